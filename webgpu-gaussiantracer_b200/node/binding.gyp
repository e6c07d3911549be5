{
  "targets": [
    {
      "target_name": "gtrace_napi",
      "sources": ["gtrace_napi.cc"],
      "include_dirs": ["../../include"],
      "libraries": ["-L<(module_root_dir)/../gtrace", "-lgtrace", "-Wl,-rpath,<(module_root_dir)/../gtrace"],
      "cflags_cc": ["-std=c++17", "-O2"]
    }
  ]
}
