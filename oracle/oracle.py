"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE).

Only the tests, the smoke check and the benchmark's CPU-baseline leg import
this module.  The product library never loads the oracle.  Parity unpinned:
see gt_oracle.h.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None


def build(force: bool = False) -> str:
    """Compiles the oracle with its Makefile (gcc, -ffp-contract=off)."""
    if force or not os.path.exists(_LIB_PATH):
        subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


class OrHits(C.Structure):
    _fields_ = [("max_entries", C.c_uint32), ("pidx", C.POINTER(C.c_uint32)), ("t", C.POINTER(C.c_float)),
                ("alpha", C.POINTER(C.c_float)), ("count", C.POINTER(C.c_uint32)),
                ("rounds", C.POINTER(C.c_uint32)), ("anyhits", C.c_uint64), ("node_visits", C.c_uint64)]


def lib():
    global _lib
    if _lib is None:
        build()
        L = C.CDLL(_LIB_PATH)
        vp, u64, u32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int
        L.or_expf.restype = C.c_float
        L.or_expf.argtypes = [C.c_float]
        L.or_log.restype = C.c_double
        L.or_log.argtypes = [C.c_double]
        L.or_ply_to_aos.restype = i32
        L.or_ply_to_aos.argtypes = [vp, C.c_size_t, C.POINTER(u32), C.POINTER(u32), C.POINTER(u32), vp, vp]
        for sfx in ("f32", "f64"):
            f = getattr(L, f"or_scene_create_{sfx}")
            f.restype = vp
            f.argtypes = [vp, u64, u32, C.c_double]
            f = getattr(L, f"or_scene_create_ex_{sfx}")
            f.restype = vp
            f.argtypes = [vp, u64, u32, C.c_double, vp]
            getattr(L, f"or_scene_destroy_{sfx}").argtypes = [vp]
            k = getattr(L, f"or_scene_kept_{sfx}")
            k.restype = u64
            k.argtypes = [vp]
            p = getattr(L, f"or_scene_proxy_{sfx}")
            p.restype = i32
            p.argtypes = [vp, u64, C.POINTER(u32), vp, vp]
            r = getattr(L, f"or_render_{sfx}")
            r.restype = i32
            r.argtypes = [vp, vp, u32, u32, vp, u32, i32, i32, vp, C.POINTER(OrHits)]
        L.or_render_accum_f32.restype = i32
        L.or_render_accum_f32.argtypes = [vp, vp, u32, u32, i32, vp]
        L.or_new_seed.restype = u32
        L.or_new_seed.argtypes = [u32, u32, u32]
        L.or_rng.restype = C.c_float
        L.or_rng.argtypes = [C.POINTER(u32)]
        L.or_tonemap.restype = i32
        L.or_tonemap.argtypes = [vp, u64, u32, C.c_float, vp]
        L.or_backward_f64.restype = i32
        L.or_backward_f64.argtypes = [vp, vp, u32, u32, vp, u32, vp, i32, vp]
        L.or_backward_lists_f64.restype = i32
        L.or_backward_lists_f64.argtypes = [vp, vp, u32, u32, vp, u32, vp, vp, vp, u32, vp, i32, vp]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


class Scene:
    """Oracle scene in float ("f32": the bit-exact specification) or double."""

    def __init__(self, packed: np.ndarray, alpha_min: float, precision: str = "f32", activated=None):
        """activated: optional (n, 8) float64 opacity, scale xyz, rotation
        wxyz, from which the proxies are built (as the reference builds them)."""
        L = lib()
        self.precision = precision
        self._aos = np.ascontiguousarray(packed, dtype=np.float32)
        n = self._aos.shape[0]
        stride = self._aos.shape[1] * 4 if n else 320
        self.n = n
        self._act = None if activated is None else np.ascontiguousarray(activated, dtype=np.float64).reshape(n, 8)
        self._h = getattr(L, f"or_scene_create_ex_{precision}")(_ptr(self._aos), n, stride, alpha_min,
                                                                _ptr(self._act))
        if not self._h:
            raise RuntimeError("oracle scene creation failed")

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            getattr(lib(), f"or_scene_destroy_{self.precision}")(h)
            self._h = None

    @property
    def n_kept(self) -> int:
        return int(getattr(lib(), f"or_scene_kept_{self.precision}")(self._h))

    def proxy(self, j: int):
        p = C.c_uint32()
        o2w = np.zeros(12, np.float32)
        w2o = np.zeros(12, np.float32)
        getattr(lib(), f"or_scene_proxy_{self.precision}")(self._h, j, C.byref(p), _ptr(o2w), _ptr(w2o))
        return int(p.value), o2w, w2o

    def render(self, uniforms, w: int, h: int, pixels=None, algo: int = 0, threads: int = 0,
               max_entries: int = 0):
        """Returns rgba (n_pix x 4) and, if max_entries > 0, a hit record dict."""
        u = np.frombuffer(bytes(uniforms), dtype=np.uint8).copy()
        pix = None if pixels is None else np.ascontiguousarray(pixels, dtype=np.uint32)
        npix = w * h if pix is None else pix.shape[0]
        dt = np.float32 if self.precision == "f32" else np.float64
        out = np.zeros((npix, 4), dtype=dt)
        hits = None
        rec = {}
        if max_entries > 0 or True:
            me = max(max_entries, 0)
            rec = {"pidx": np.zeros((npix, max(me, 1)), np.uint32), "t": np.zeros((npix, max(me, 1)), np.float32),
                   "alpha": np.zeros((npix, max(me, 1)), np.float32), "count": np.zeros(npix, np.uint32),
                   "rounds": np.zeros(npix, np.uint32)}
            hits = OrHits(me, rec["pidx"].ctypes.data_as(C.POINTER(C.c_uint32)),
                          rec["t"].ctypes.data_as(C.POINTER(C.c_float)),
                          rec["alpha"].ctypes.data_as(C.POINTER(C.c_float)),
                          rec["count"].ctypes.data_as(C.POINTER(C.c_uint32)),
                          rec["rounds"].ctypes.data_as(C.POINTER(C.c_uint32)), 0, 0)
        rc = getattr(lib(), f"or_render_{self.precision}")(self._h, _ptr(u), w, h, _ptr(pix), npix, algo, threads,
                                                           _ptr(out), C.byref(hits) if hits else None)
        if rc != 0:
            raise RuntimeError(f"oracle render failed ({rc})")
        rec["anyhits"] = int(hits.anyhits)
        rec["node_visits"] = int(hits.node_visits)
        return out, rec

    def render_accum(self, uniforms, w: int, h: int, accum: np.ndarray, threads: int = 0) -> np.ndarray:
        """Progressive anti-aliasing step: blends the jittered render of
        frame ``accumulated_frames`` into ``accum`` (w*h x 4 float32, in place)."""
        if self.precision != "f32":
            raise ValueError("the anti-aliasing restatement is the float build")
        u = np.frombuffer(bytes(uniforms), dtype=np.uint8).copy()
        assert accum.dtype == np.float32 and accum.flags.c_contiguous and accum.size == w * h * 4
        rc = lib().or_render_accum_f32(self._h, _ptr(u), w, h, threads, _ptr(accum))
        if rc != 0:
            raise RuntimeError(f"oracle accumulate failed ({rc})")
        return accum

    def backward(self, uniforms, w: int, h: int, dL_drgba: np.ndarray, pixels=None, threads: int = 0):
        if self.precision != "f64":
            raise ValueError("the oracle adjoint is FP64")
        u = np.frombuffer(bytes(uniforms), dtype=np.uint8).copy()
        pix = None if pixels is None else np.ascontiguousarray(pixels, dtype=np.uint32)
        npix = w * h if pix is None else pix.shape[0]
        g = np.ascontiguousarray(dL_drgba, dtype=np.float64).reshape(npix, 4)
        out = np.zeros((59, max(self.n, 1)), dtype=np.float64)
        rc = lib().or_backward_f64(self._h, _ptr(u), w, h, _ptr(pix), npix, _ptr(g), threads, _ptr(out))
        if rc != 0:
            raise RuntimeError(f"oracle backward failed ({rc})")
        return out[:, :self.n]


def backward_lists(scene: "Scene", uniforms, w: int, h: int, hits: dict, dL_drgba, pixels=None,
                   alpha_min: float | None = None, threads: int = 0) -> np.ndarray:
    """FP64 adjoint on the entry lists of a (float) render: `hits` holds
    pidx (n_pix x max_e), count and alpha; entries with alpha > alpha_min
    (the float decision) are the composited ones."""
    if scene.precision != "f64":
        raise ValueError("the oracle adjoint is FP64")
    u = np.frombuffer(bytes(uniforms), dtype=np.uint8).copy()
    pix = None if pixels is None else np.ascontiguousarray(pixels, dtype=np.uint32)
    npix = w * h if pix is None else pix.shape[0]
    lists = np.ascontiguousarray(hits["pidx"], dtype=np.uint32)
    max_e = lists.shape[1]
    if (np.asarray(hits["count"]) > max_e).any():
        raise ValueError("entry lists are truncated")
    contrib = None
    if alpha_min is not None:
        contrib = np.ascontiguousarray(np.asarray(hits["alpha"]) > np.float32(alpha_min), dtype=np.uint8)
    counts = np.ascontiguousarray(hits["count"], dtype=np.uint32)
    g = np.ascontiguousarray(dL_drgba, dtype=np.float64).reshape(npix, 4)
    out = np.zeros((59, max(scene.n, 1)), dtype=np.float64)
    rc = lib().or_backward_lists_f64(scene._h, _ptr(u), w, h, _ptr(pix), npix, _ptr(lists), _ptr(contrib),
                                     _ptr(counts), max_e, _ptr(g), threads, _ptr(out))
    if rc != 0:
        raise RuntimeError(f"oracle backward failed ({rc})")
    return out[:, :scene.n]


def ply_to_aos(data: bytes, activations: bool = False):
    """Packed records of a PLY blob; with activations=True also the (n, 8)
    float64 activated values (opacity, scale xyz, rotation wxyz)."""
    L = lib()
    buf = np.frombuffer(data, dtype=np.uint8)
    n, deg, stride = C.c_uint32(), C.c_uint32(), C.c_uint32()
    rc = L.or_ply_to_aos(_ptr(buf), len(data), C.byref(n), C.byref(deg), C.byref(stride), None, None)
    if rc != 0:
        raise ValueError(f"oracle PLY parse failed ({rc})")
    out = np.zeros((n.value, stride.value // 4), dtype=np.float32)
    act = np.zeros((n.value, 8), dtype=np.float64)
    rc = L.or_ply_to_aos(_ptr(buf), len(data), C.byref(n), C.byref(deg), C.byref(stride), _ptr(out), _ptr(act))
    if rc != 0:
        raise ValueError(f"oracle PLY parse failed ({rc})")
    return (out, act) if activations else out


def tonemap(rgba: np.ndarray, mode: int, exposure: float = 1.66) -> np.ndarray:
    """unorm8 RGBA of an RGBA-f32 image (src/toneMapper.ts:15-24), shape (n, 4)."""
    a = np.ascontiguousarray(rgba, dtype=np.float32).reshape(-1, 4)
    out = np.zeros((a.shape[0], 4), dtype=np.uint8)
    rc = lib().or_tonemap(_ptr(a), a.shape[0], mode, exposure, _ptr(out))
    if rc != 0:
        raise ValueError(f"oracle tone map failed ({rc})")
    return out


def new_seed(p1: int, p2: int, rounds: int = 8) -> int:
    return int(lib().or_new_seed(p1, p2, rounds))


def rng(seed: int):
    s = C.c_uint32(seed)
    v = float(lib().or_rng(C.byref(s)))
    return v, int(s.value)


def expf(x: float) -> float:
    return float(lib().or_expf(x))


def log(x: float) -> float:
    return float(lib().or_log(x))
