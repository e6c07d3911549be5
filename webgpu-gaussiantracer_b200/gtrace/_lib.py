"""ctypes binding of libgtrace.so (the C ABI of include/gtrace.h).

The library is built in-tree (``make -C webgpu-gaussiantracer_b200/csrc``)
and loaded from this directory.  There is no fallback: every call goes to
the CUDA library, and a missing library is an error.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libgtrace.so")

GT_OK = 0
GT_ERR_INVALID_ARG = 1
GT_ERR_OOM = 2
GT_ERR_CUDA = 3
GT_ERR_DEVICE_TIMEOUT = 4
GT_ERR_STACK_OVERFLOW = 5
GT_ERR_UNSUPPORTED = 6
GT_ERR_NO_DEVICE = 7

GT_FLAG_INPUT_DEVICE = 0x1
GT_FLAG_OUTPUT_DEVICE = 0x2
GT_FLAG_ASYNC = 0x4
GT_FLAG_ACCUMULATE = 0x8
GT_FLAG_CHECKPOINT = 0x10
GT_FLAG_FAST_BUILD = 0x20
GT_FLAG_ANTIALIAS = 0x40

GT_TONEMAP_HDR = 0
GT_TONEMAP_EXPOSURE = 1
GT_TONEMAP_EXPOSURE_GAMMA = 2

STATUS_NAMES = {GT_OK: "GT_OK", GT_ERR_INVALID_ARG: "GT_ERR_INVALID_ARG", GT_ERR_OOM: "GT_ERR_OOM",
                GT_ERR_CUDA: "GT_ERR_CUDA", GT_ERR_DEVICE_TIMEOUT: "GT_ERR_DEVICE_TIMEOUT",
                GT_ERR_STACK_OVERFLOW: "GT_ERR_STACK_OVERFLOW", GT_ERR_UNSUPPORTED: "GT_ERR_UNSUPPORTED",
                GT_ERR_NO_DEVICE: "GT_ERR_NO_DEVICE"}


class Uniforms(C.Structure):
    _fields_ = [("to_world", C.c_float * 16), ("camera_aspect", C.c_float * 2), ("t_min", C.c_float),
                ("t_max", C.c_float), ("T_min", C.c_float), ("alpha_min", C.c_float), ("k", C.c_uint32),
                ("sh_degree_max", C.c_uint32), ("accumulated_frames", C.c_uint32), ("early_stop", C.c_uint32),
                ("debug_mode", C.c_uint32), ("_pad", C.c_uint32)]


class RenderStats(C.Structure):
    _fields_ = [("kernel_ms", C.c_float), ("total_ms", C.c_float), ("rays", C.c_uint64), ("rounds", C.c_uint64),
                ("entries", C.c_uint64), ("contributing", C.c_uint64), ("proxy_tests", C.c_uint64),
                ("node_visits", C.c_uint64), ("anyhits", C.c_uint64), ("status_flags", C.c_uint32),
                ("handed", C.c_uint32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if not name.startswith("_")}


class SceneInfo(C.Structure):
    _fields_ = [("n_particles", C.c_uint64), ("n_kept", C.c_uint64), ("device_bytes", C.c_uint64),
                ("bvh_depth", C.c_uint32), ("_pad", C.c_uint32), ("build_ms", C.c_float),
                ("bounds", C.c_float * 6), ("upload_ms", C.c_float)]


class BwdOpts(C.Structure):
    _fields_ = [("mode", C.c_uint32), ("max_rounds", C.c_uint32), ("mem_budget", C.c_uint64),
                ("used_mode", C.c_uint32), ("_pad", C.c_uint32), ("fwd_ms", C.c_float), ("bwd_ms", C.c_float)]


class BatchItem(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("u", Uniforms), ("w", C.c_uint32), ("h", C.c_uint32),
                ("out_rgba", C.c_void_p), ("dL_drgba", C.c_void_p)]


class TuneResult(C.Structure):
    _fields_ = [("block_threads", C.c_uint32), ("blocks_per_sm", C.c_uint32), ("tile_w", C.c_uint32),
                ("tile_h", C.c_uint32), ("best_ms", C.c_float), ("default_ms", C.c_float),
                ("kbuf", C.c_uint32), ("leaf_batch", C.c_uint32), ("handoff_after", C.c_uint32),
                ("_pad", C.c_uint32)]


class BvhInfo(C.Structure):
    _fields_ = [("n_nodes8", C.c_uint32), ("n_leaves", C.c_uint32), ("root", C.c_uint32), ("depth", C.c_uint32)]


class PlyInfo(C.Structure):
    _fields_ = [("n_vertices", C.c_uint64), ("data_offset", C.c_uint64), ("sh_degree", C.c_uint32),
                ("record_stride", C.c_uint32), ("row_bytes", C.c_uint32), ("n_properties", C.c_uint32),
                ("ingest_ms", C.c_float), ("_pad", C.c_uint32)]

    def as_dict(self):
        return {name: getattr(self, name) for name, _ in self._fields_ if not name.startswith("_")}


assert C.sizeof(Uniforms) == 112

# (name, restype, argtypes) of every symbol include/gtrace.h declares
_vp, _u32, _u64, _i32 = C.c_void_p, C.c_uint32, C.c_uint64, C.c_int32
SIGNATURES = [
    ("gt_version", _u32, []),
    ("gt_context_create", _i32, [C.c_int, C.POINTER(_vp)]),
    ("gt_context_destroy", _i32, [_vp]),
    ("gt_last_error", _i32, [_vp, C.c_char_p, C.c_size_t]),
    ("gt_scene_create", _i32, [_vp, _vp, _u64, _u32, C.c_double, _u32, C.POINTER(_vp)]),
    ("gt_scene_create_ex", _i32, [_vp, _vp, _u64, _u32, C.c_double, _vp, _u32, C.POINTER(_vp)]),
    ("gt_scene_destroy", _i32, [_vp]),
    ("gt_scene_get_info", _i32, [_vp, C.POINTER(SceneInfo)]),
    ("gt_scene_export_bvh", _i32, [_vp, _vp, _u64, _vp, _u64, C.POINTER(BvhInfo)]),
    ("gt_ply_parse_header", _i32, [_vp, _u64, C.POINTER(PlyInfo)]),
    ("gt_ply_pack", _i32, [_vp, _vp, _u64, _vp, _u64, _u32, C.POINTER(PlyInfo)]),
    ("gt_scene_create_from_ply", _i32, [_vp, _vp, _u64, C.c_double, _u32, C.POINTER(_vp), C.POINTER(PlyInfo)]),
    ("gt_scene_create_from_ply_file", _i32, [_vp, C.c_char_p, C.c_double, _u32, C.POINTER(_vp),
                                             C.POINTER(PlyInfo)]),
    ("gt_render", _i32, [_vp, _vp, C.POINTER(Uniforms), _u32, _u32, _vp, _u32, C.POINTER(RenderStats)]),
    ("gt_render_hits", _i32, [_vp, _vp, C.POINTER(Uniforms), _u32, _u32, _vp, _u32, _u32, _vp, _vp, _vp, _vp, _vp,
                              _vp]),
    ("gt_backward", _i32, [_vp, _vp, C.POINTER(Uniforms), _u32, _u32, _vp, _vp, _u32, C.POINTER(BwdOpts),
                           C.POINTER(RenderStats)]),
    ("gt_render_batch", _i32, [_vp, C.POINTER(BatchItem), _u32, _u32, C.POINTER(RenderStats)]),
    ("gt_render_batch_noalloc", _i32, [_vp, C.POINTER(BatchItem), _u32, _u32, C.POINTER(RenderStats)]),
    ("gt_backward_batch", _i32, [_vp, C.POINTER(BatchItem), _u32, C.POINTER(_vp), C.POINTER(_vp), _u32, _u32,
                                 C.POINTER(BwdOpts), C.POINTER(RenderStats)]),
    ("gt_tonemap", _i32, [_vp, _vp, _u64, _u32, C.c_float, _vp, _u32]),
    ("gt_l2_loss", _i32, [_vp, _vp, _vp, _u64, _vp, C.POINTER(C.c_double)]),
    ("gt_autotune", _i32, [_vp, _vp, C.POINTER(Uniforms), _u32, _u32, C.POINTER(TuneResult)]),
    ("gt_autotune_batch", _i32, [_vp, C.POINTER(BatchItem), _u32, C.POINTER(TuneResult)]),
    ("gt_set_tune", _i32, [_vp, _vp, C.POINTER(Uniforms), _u32, _u32, C.POINTER(TuneResult)]),
    ("gt_autotune_reset", _i32, [_vp]),
    ("gt_set_limits", _i32, [_vp, _u32, _u32, _u32]),
    ("gt_device_alloc", _i32, [_vp, _u64, C.POINTER(_vp)]),
    ("gt_device_free", _i32, [_vp, _vp]),
    ("gt_host_alloc", _i32, [_vp, _u64, C.POINTER(_vp)]),
    ("gt_host_free", _i32, [_vp, _vp]),
    ("gt_memcpy", _i32, [_vp, _vp, _vp, _u64, C.c_int]),
    ("gt_synchronize", _i32, [_vp]),
    ("gt_timer_start", _i32, [_vp]),
    ("gt_timer_stop", _i32, [_vp, C.POINTER(C.c_float)]),
    ("gt_kernel_times", _i32, [_vp, C.POINTER(C.c_float), _u32, C.POINTER(_u32)]),
    ("gt_launch_count", _i32, [_vp, C.POINTER(_u64)]),
    ("gt_device_attributes", _i32, [_vp, C.POINTER(_u32), C.POINTER(_u32)]),
]

_lib = None


class GTraceError(RuntimeError):
    """A non-zero gt_status, with the library's message."""

    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status
        self.message = message


def load(path: str | None = None):
    """Loads libgtrace.so and declares every entry point."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    p = path or LIB_PATH
    if not os.path.exists(p):
        raise FileNotFoundError(f"{p} is missing: build it with `make -C webgpu-gaussiantracer_b200/csrc`")
    lib = C.CDLL(p)
    for name, res, args in SIGNATURES:
        fn = getattr(lib, name)
        fn.restype = res
        fn.argtypes = args
    if path is None:
        _lib = lib
    return lib


def last_error(ctx) -> str:
    buf = C.create_string_buffer(1024)
    load().gt_last_error(ctx, buf, len(buf))
    return buf.value.decode("utf-8", "replace")


def check(status: int, ctx=None):
    if status != GT_OK:
        raise GTraceError(status, last_error(ctx))
