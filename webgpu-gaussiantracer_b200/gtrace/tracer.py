"""Host API of the tracer: the drop-in for the reference's render path.

The reference drives its WebGPU pipeline like this (src/main.ts:469-577)::

    const tlas = await gaussianSceneToBvh(device, gsData, alpha_min, GaussianIndices);
    const rtPipeline = await createRayTracingPipeline(device, tlas, hit_array_size);
    const sbt = createShaderBindingTable(device, rtPipeline, GaussianIndices);
    ...
    passEncoder.traceRays(device, sbt, width, height);

Here the same steps are::

    ctx = Context(0)                                   # adapter + device
    scene = gaussian_scene_to_bvh(ctx, gs_data, alpha_min, gaussian_indices)
    rgba = ctx.trace_rays(scene, uniforms, width, height)   # (H, W, 4) float32

The acceleration structure, pipeline and shader binding table collapse into
one scene handle built on the GPU; ``trace_rays`` takes the reference's
112-byte uniform block and returns its RGBA-f32 pixel buffer.  Errors are
raised as ``GTraceError`` (the reference throws strings).
"""
from __future__ import annotations

import ctypes as C
import weakref

import numpy as np

from . import _lib as L
from .ply import PackedGaussians


def _uniforms(u) -> L.Uniforms:
    if isinstance(u, L.Uniforms):
        return u
    b = bytes(np.asarray(u, dtype=np.uint8).tobytes() if not isinstance(u, (bytes, bytearray)) else u)
    if len(b) != 112:
        raise ValueError("the uniform block is 112 bytes")
    return L.Uniforms.from_buffer_copy(b)


class Context:
    """A CUDA device, its stream and the library state (one per GPU)."""

    def __init__(self, device: int = 0):
        self._lib = L.load()
        h = C.c_void_p()
        L.check(self._lib.gt_context_create(device, C.byref(h)), None)
        self._h = h
        self.device = device
        self._scenes = weakref.WeakSet()

    @property
    def handle(self):
        return self._h

    def close(self):
        """Destroys the context; scenes built on it are released with it."""
        if getattr(self, "_h", None):
            for s in list(self._scenes):
                s._h = None  # freed by gt_context_destroy
            self._lib.gt_context_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def check(self, status: int):
        L.check(status, self._h)

    # ------------------------------------------------------------- render
    def render(self, scene: "Scene", uniforms, width: int, height: int, out: np.ndarray | None = None,
               stats: bool = False, checkpoint: bool = False, antialias: bool = False):
        """Renders one view to a host array of shape (height, width, 4).
        checkpoint=True keeps the round checkpoint for a following backward.
        antialias=True takes the jittered sample of frame
        ``uniforms.accumulated_frames`` and blends it into ``out`` (the
        reference's progressive average; frame 0 replaces it)."""
        u = _uniforms(uniforms)
        if out is None:
            if antialias and u.accumulated_frames != 0:
                raise ValueError("antialias frames after the first blend into `out`: pass it")
            out = np.empty((height, width, 4), dtype=np.float32)
        if out.dtype != np.float32 or not out.flags.c_contiguous or out.size != width * height * 4:
            raise ValueError("out must be a C-contiguous float32 array of width*height*4 values")
        st = L.RenderStats()
        flags = (L.GT_FLAG_CHECKPOINT if checkpoint else 0) | (L.GT_FLAG_ANTIALIAS if antialias else 0)
        self.check(self._lib.gt_render(self._h, scene.handle, C.byref(u), width, height,
                                       out.ctypes.data_as(C.c_void_p), flags, C.byref(st)))
        return (out, st.as_dict()) if stats else out

    trace_rays = render

    def render_device(self, scene: "Scene", uniforms, width: int, height: int, out_dev: int, asynchronous=False,
                      checkpoint: bool = False):
        """Renders into a device buffer (pointer from ``device_alloc``)."""
        u = _uniforms(uniforms)
        flags = L.GT_FLAG_OUTPUT_DEVICE | (L.GT_FLAG_ASYNC if asynchronous else 0) | \
            (L.GT_FLAG_CHECKPOINT if checkpoint else 0)
        st = L.RenderStats()
        self.check(self._lib.gt_render(self._h, scene.handle, C.byref(u), width, height, C.c_void_p(out_dev), flags,
                                       None if asynchronous else C.byref(st)))
        return None if asynchronous else st.as_dict()

    def render_hits(self, scene: "Scene", uniforms, width: int, height: int, pixels, max_entries: int = 64):
        """Composited hit sequences of the listed pixels (see gt_render_hits)."""
        u = _uniforms(uniforms)
        pix = np.ascontiguousarray(pixels, dtype=np.uint32)
        n = pix.shape[0]
        me = max(int(max_entries), 1)
        rec = {"pidx": np.zeros((n, me), np.uint32), "t": np.zeros((n, me), np.float32),
               "alpha": np.zeros((n, me), np.float32), "count": np.zeros(n, np.uint32),
               "rounds": np.zeros(n, np.uint32), "rgba": np.zeros((n, 4), np.float32)}
        vp = lambda a: a.ctypes.data_as(C.c_void_p)  # noqa: E731
        self.check(self._lib.gt_render_hits(self._h, scene.handle, C.byref(u), width, height, vp(pix), n, me,
                                            vp(rec["pidx"]), vp(rec["t"]), vp(rec["alpha"]), vp(rec["count"]),
                                            vp(rec["rounds"]), vp(rec["rgba"])))
        return rec

    def backward(self, scene: "Scene", uniforms, width: int, height: int, dL_drgba: np.ndarray, mode: int = 0,
                 max_rounds: int = 0, mem_budget: int = 0, out: np.ndarray | None = None, accumulate=False,
                 reuse_checkpoint: bool = False):
        """dLoss/dparams (59 x n, parameter-major) from dLoss/drgba (h, w, 4)."""
        u = _uniforms(uniforms)
        g = np.ascontiguousarray(dL_drgba, dtype=np.float32)
        if g.size != width * height * 4:
            raise ValueError("dL_drgba must hold width*height*4 values")
        if out is None:
            out = np.zeros((59, scene.n), dtype=np.float32)
        opts = L.BwdOpts(mode, max_rounds, mem_budget, 0, 0, 0.0, 0.0)
        st = L.RenderStats()
        flags = (L.GT_FLAG_ACCUMULATE if accumulate else 0) | (L.GT_FLAG_CHECKPOINT if reuse_checkpoint else 0)
        self.check(self._lib.gt_backward(self._h, scene.handle, C.byref(u), width, height,
                                         g.ctypes.data_as(C.c_void_p), out.ctypes.data_as(C.c_void_p), flags,
                                         C.byref(opts), C.byref(st)))
        info = st.as_dict()
        info.update(used_mode=opts.used_mode, fwd_ms=opts.fwd_ms, bwd_ms=opts.bwd_ms, max_rounds=opts.max_rounds)
        return out, info

    def backward_batch(self, views, mode: int = 0, max_rounds: int = 0, mem_budget: int = 0):
        """views: list of (scene, uniforms, width, height, dL_drgba) -> {scene: (59 x n) gradient}, info.
        Gradients of all views of a scene are summed in one adjoint launch."""
        items = (L.BatchItem * len(views))()
        keep = []
        scenes = []
        for i, (scene, uniforms, w, h, g) in enumerate(views):
            ga = np.ascontiguousarray(g, dtype=np.float32)
            if ga.size != w * h * 4:
                raise ValueError("dL_drgba must hold width*height*4 values")
            keep.append(ga)
            items[i].scene = scene.handle
            items[i].u = _uniforms(uniforms)
            items[i].w, items[i].h = w, h
            items[i].out_rgba = None
            items[i].dL_drgba = ga.ctypes.data
            if scene not in scenes:
                scenes.append(scene)
        outs = [np.zeros((59, s.n), dtype=np.float32) for s in scenes]
        sc = (C.c_void_p * len(scenes))(*[s.handle.value for s in scenes])
        op = (C.c_void_p * len(scenes))(*[o.ctypes.data for o in outs])
        opts = L.BwdOpts(mode, max_rounds, mem_budget, 0, 0, 0.0, 0.0)
        st = L.RenderStats()
        self.check(self._lib.gt_backward_batch(self._h, items, len(views), sc, op, len(scenes), 0, C.byref(opts),
                                               C.byref(st)))
        info = st.as_dict()
        info.update(used_mode=opts.used_mode, fwd_ms=opts.fwd_ms, bwd_ms=opts.bwd_ms, max_rounds=opts.max_rounds)
        return dict(zip(scenes, outs)), info

    def render_batch(self, views, outs=None, device_outputs=False, asynchronous=False):
        """views: list of (scene, uniforms, width, height[, out]) -> list of outputs, stats."""
        items = (L.BatchItem * len(views))()
        results = []
        for i, v in enumerate(views):
            scene, uniforms, w, h = v[:4]
            if device_outputs:
                ptr = v[4]
                results.append(ptr)
            else:
                arr = outs[i] if outs is not None else np.empty((h, w, 4), dtype=np.float32)
                results.append(arr)
                ptr = arr.ctypes.data
            items[i].scene = scene.handle
            items[i].u = _uniforms(uniforms)
            items[i].w = w
            items[i].h = h
            items[i].out_rgba = ptr
            items[i].dL_drgba = None
        flags = (L.GT_FLAG_OUTPUT_DEVICE if device_outputs else 0) | (L.GT_FLAG_ASYNC if asynchronous else 0)
        st = L.RenderStats()
        self.check(self._lib.gt_render_batch(self._h, items, len(views), flags, None if asynchronous else C.byref(st)))
        return results, st.as_dict()

    def backward_device(self, scene: "Scene", uniforms, width: int, height: int, dL_dev: int, out_dev: int,
                        reuse_checkpoint: bool = True, mode: int = 0):
        """Device-buffer backward (gradient 59 x n at out_dev); returns the info dict."""
        u = _uniforms(uniforms)
        opts = L.BwdOpts(mode, 0, 0, 0, 0, 0.0, 0.0)
        st = L.RenderStats()
        flags = L.GT_FLAG_INPUT_DEVICE | L.GT_FLAG_OUTPUT_DEVICE | (L.GT_FLAG_CHECKPOINT if reuse_checkpoint else 0)
        self.check(self._lib.gt_backward(self._h, scene.handle, C.byref(u), width, height, C.c_void_p(dL_dev),
                                         C.c_void_p(out_dev), flags, C.byref(opts), C.byref(st)))
        info = st.as_dict()
        info.update(used_mode=opts.used_mode, fwd_ms=opts.fwd_ms, bwd_ms=opts.bwd_ms, max_rounds=opts.max_rounds)
        return info

    def l2_loss(self, rgba_dev: int, target_dev: int, n_pixels: int, dL_dev: int) -> float:
        loss = C.c_double()
        self.check(self._lib.gt_l2_loss(self._h, C.c_void_p(rgba_dev), C.c_void_p(target_dev), n_pixels,
                                        C.c_void_p(dL_dev), C.byref(loss)))
        return loss.value

    def autotune(self, scene: "Scene", uniforms, width: int, height: int):
        r = L.TuneResult()
        self.check(self._lib.gt_autotune(self._h, scene.handle, C.byref(_uniforms(uniforms)), width, height,
                                         C.byref(r)))
        return {name: getattr(r, name) for name, _ in r._fields_ if not name.startswith("_")}

    def autotune_batch(self, views):
        """views: list of (scene, uniforms, width, height) -> the fastest launch
        shape of that batch, cached for later render_batch calls of its shape."""
        items = (L.BatchItem * len(views))()
        for i, (scene, uniforms, w, h) in enumerate(views):
            items[i].scene = scene.handle
            items[i].u = _uniforms(uniforms)
            items[i].w, items[i].h = w, h
        r = L.TuneResult()
        self.check(self._lib.gt_autotune_batch(self._h, items, len(views), C.byref(r)))
        return {name: getattr(r, name) for name, _ in r._fields_ if not name.startswith("_")}

    def set_tune(self, scene: "Scene", uniforms, width: int, height: int, blocks_per_sm: int = 4,
                 kbuf: int = 32, leaf_batch: int = 32, block_threads: int = 128, handoff_after: int = 0):
        """Installs a launch shape for this (scene, k, image size) bucket:
        block_threads 32 traces 8x4 tiles of rays per warp (kbuf entries per
        ray, rays handed to a warp-per-ray launch after handoff_after
        traversals, 0: the default), 128 one ray per warp (gt_set_tune)."""
        r = L.TuneResult(block_threads, blocks_per_sm, 8, 4, 0.0, 0.0, kbuf, leaf_batch, handoff_after, 0)
        self.check(self._lib.gt_set_tune(self._h, scene.handle, C.byref(_uniforms(uniforms)), width, height,
                                         C.byref(r)))

    # ------------------------------------------------------------ display
    def tonemap(self, rgba: np.ndarray, mode: int = L.GT_TONEMAP_HDR, exposure: float = 1.66) -> np.ndarray:
        """The reference's tone-map pass (src/toneMapper.ts:15-24) into a
        headless RGBA8 image of the same height and width."""
        a = np.ascontiguousarray(rgba, dtype=np.float32)
        if a.size % 4:
            raise ValueError("rgba holds 4 floats per pixel")
        n = a.size // 4
        out = np.zeros(a.shape[:-1] + (4,) if a.ndim > 1 and a.shape[-1] == 4 else (n, 4), dtype=np.uint8)
        self.check(self._lib.gt_tonemap(self._h, a.ctypes.data_as(C.c_void_p), n, mode, exposure,
                                        out.ctypes.data_as(C.c_void_p), 0))
        return out

    # --------------------------------------------------------- PLY ingest
    def pack_ply(self, data: bytes):
        """Native ``PackedGaussians(arrayBuffer).gaussiansBuffer``: the PLY
        blob decoded, activated and packed on the GPU.  Returns the records as
        a float32 array of shape (n, record_stride / 4) and the header info."""
        buf = np.frombuffer(bytes(data), dtype=np.uint8)
        info = ply_header(buf)
        out = np.zeros((info["n_vertices"], info["record_stride"] // 4), dtype=np.float32)
        pi = L.PlyInfo()
        self.check(self._lib.gt_ply_pack(self._h, buf.ctypes.data_as(C.c_void_p), buf.size,
                                         out.ctypes.data_as(C.c_void_p), out.nbytes, 0, C.byref(pi)))
        return out, pi.as_dict()

    # ----------------------------------------------------------- helpers
    def device_alloc(self, nbytes: int) -> int:
        p = C.c_void_p()
        self.check(self._lib.gt_device_alloc(self._h, nbytes, C.byref(p)))
        return p.value

    def device_free(self, ptr: int):
        self.check(self._lib.gt_device_free(self._h, C.c_void_p(ptr)))

    def host_alloc(self, nbytes: int, dtype=np.float32, shape=None) -> np.ndarray:
        """Page-locked host array (freed with host_free)."""
        p = C.c_void_p()
        self.check(self._lib.gt_host_alloc(self._h, nbytes, C.byref(p)))
        buf = (C.c_uint8 * nbytes).from_address(p.value)
        arr = np.frombuffer(buf, dtype=dtype)
        return arr.reshape(shape) if shape is not None else arr

    def host_free(self, arr: np.ndarray):
        self.check(self._lib.gt_host_free(self._h, C.c_void_p(arr.ctypes.data)))

    def memcpy(self, dst: int, src: int, nbytes: int, kind: int):
        self.check(self._lib.gt_memcpy(self._h, C.c_void_p(dst), C.c_void_p(src), nbytes, kind))

    def synchronize(self):
        self.check(self._lib.gt_synchronize(self._h))

    def timer_start(self):
        self.check(self._lib.gt_timer_start(self._h))

    def timer_stop(self) -> float:
        ms = C.c_float()
        self.check(self._lib.gt_timer_stop(self._h, C.byref(ms)))
        return ms.value

    def kernel_times(self, max_n: int = 256):
        buf = (C.c_float * max_n)()
        n = C.c_uint32()
        self.check(self._lib.gt_kernel_times(self._h, buf, max_n, C.byref(n)))
        return [buf[i] for i in range(n.value)]

    def device_attributes(self) -> dict:
        """SM count and the maximum SM clock (MHz) of the context's GPU."""
        n, khz = C.c_uint32(), C.c_uint32()
        self.check(self._lib.gt_device_attributes(self._h, C.byref(n), C.byref(khz)))
        return {"sm_count": int(n.value), "max_sm_mhz": khz.value / 1000.0}

    def launch_count(self) -> int:
        n = C.c_uint64()
        self.check(self._lib.gt_launch_count(self._h, C.byref(n)))
        return n.value


class Scene:
    """Proxies + BVH + shading records of one packed particle buffer, on the GPU."""

    def __init__(self, ctx: Context, packed: np.ndarray, alpha_min: float, device_ptr: int | None = None,
                 n: int | None = None, stride: int | None = None, fast_build: bool = False, activated=None):
        """fast_build: Karras LBVH hierarchy (quicker build, slower traversal).
        activated: optional (n, 8) float64 opacity, scale xyz, rotation wxyz
        (PackedGaussians.activations()): the proxies are then built from these
        double values, as the reference builds them (gt_scene_create_ex)."""
        self.ctx = ctx
        self._lib = ctx._lib
        h = C.c_void_p()
        fb = L.GT_FLAG_FAST_BUILD if fast_build else 0
        if device_ptr is not None:
            if activated is not None:
                raise ValueError("activated values go with a host packed buffer")
            self.n = int(n)
            ctx.check(self._lib.gt_scene_create(ctx.handle, C.c_void_p(device_ptr), self.n, int(stride),
                                                float(alpha_min), L.GT_FLAG_INPUT_DEVICE | fb, C.byref(h)))
        else:
            arr = np.ascontiguousarray(packed, dtype=np.float32)
            self.n = arr.shape[0]
            stride = arr.shape[1] * 4 if arr.ndim == 2 and self.n else 320
            act = None
            if activated is not None:
                act = np.ascontiguousarray(activated, dtype=np.float64)
                if act.shape != (self.n, 8):
                    raise ValueError("activated must have shape (n, 8)")
            ctx.check(self._lib.gt_scene_create_ex(ctx.handle, arr.ctypes.data_as(C.c_void_p) if self.n else None,
                                                   self.n, stride, float(alpha_min),
                                                   act.ctypes.data_as(C.c_void_p) if act is not None and self.n
                                                   else None, fb, C.byref(h)))
        self._h = h
        self.alpha_min = alpha_min
        ctx._scenes.add(self)

    @classmethod
    def from_ply(cls, ctx: Context, source, alpha_min: float, fast_build: bool = False) -> "Scene":
        """Builds a scene straight from a 3DGS PLY (bytes, or a file path as
        str): loadGaussianSplatting + PackedGaussians + gaussianSceneToBvh,
        with decoding, activation and packing done natively.  The header info
        is kept in ``ply_info``."""
        self = cls.__new__(cls)
        self.ctx = ctx
        self._lib = ctx._lib
        h = C.c_void_p()
        pi = L.PlyInfo()
        fb = L.GT_FLAG_FAST_BUILD if fast_build else 0
        if isinstance(source, str):
            ctx.check(self._lib.gt_scene_create_from_ply_file(ctx.handle, source.encode(), float(alpha_min), fb,
                                                              C.byref(h), C.byref(pi)))
        else:
            buf = np.frombuffer(bytes(source), dtype=np.uint8)
            ctx.check(self._lib.gt_scene_create_from_ply(ctx.handle, buf.ctypes.data_as(C.c_void_p), buf.size,
                                                         float(alpha_min), fb, C.byref(h), C.byref(pi)))
        self._h = h
        self.n = int(pi.n_vertices)
        self.alpha_min = alpha_min
        self.ply_info = pi.as_dict()
        ctx._scenes.add(self)
        return self

    @property
    def handle(self):
        if not self._h:
            raise ValueError("scene is closed (or its context was closed)")
        return self._h

    def info(self) -> dict:
        i = L.SceneInfo()
        self.ctx.check(self._lib.gt_scene_get_info(self._h, C.byref(i)))
        d = {name: getattr(i, name) for name, _ in i._fields_ if not name.startswith("_")}
        d["bounds"] = list(i.bounds)
        return d

    def export_bvh(self):
        """(nodes8 as a float32 array (n_nodes8, 8, 8), leaf particle indices,
        info dict) of the built hierarchy (gt_scene_export_bvh)."""
        info = L.BvhInfo()
        self.ctx.check(self._lib.gt_scene_export_bvh(self.handle, None, 0, None, 0, C.byref(info)))
        nodes = np.zeros((info.n_nodes8, 8, 8), dtype=np.float32)
        leaves = np.zeros(info.n_leaves, dtype=np.uint32)
        self.ctx.check(self._lib.gt_scene_export_bvh(self.handle, nodes.ctypes.data_as(C.c_void_p), nodes.nbytes,
                                                     leaves.ctypes.data_as(C.c_void_p), leaves.size, C.byref(info)))
        return nodes, leaves, {name: getattr(info, name) for name, _ in info._fields_}

    def close(self):
        if getattr(self, "_h", None) and getattr(self.ctx, "_h", None):
            self._lib.gt_scene_destroy(self._h)
        self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def ply_header(data) -> dict:
    """Header of a 3DGS PLY blob as the native loader decodes it (no GPU
    work): n_vertices, data_offset, sh_degree, record_stride, row_bytes,
    n_properties."""
    lib = L.load()
    buf = np.frombuffer(bytes(data), dtype=np.uint8) if not isinstance(data, np.ndarray) else data
    pi = L.PlyInfo()
    L.check(lib.gt_ply_parse_header(buf.ctypes.data_as(C.c_void_p), buf.size, C.byref(pi)), None)
    d = pi.as_dict()
    d.pop("ingest_ms")
    return d


def gaussian_scene_to_bvh(ctx: Context, gs_data: PackedGaussians, alpha_min: float,
                          gaussian_indices: list | None = None) -> Scene:
    """gaussianSceneToBvh (src/main.ts:30-111): one proxy per Gaussian with
    opacity > alpha_min, built from the double-precision gaussianData values
    as the reference builds it; fills ``gaussian_indices`` with the kept
    particle indices in order, as the reference does for its shader binding
    table."""
    if gaussian_indices is not None:
        op = gs_data.gaussianData["opacity"]
        gaussian_indices.extend(np.nonzero(op > alpha_min)[0].tolist())
    return Scene(ctx, gs_data.gaussiansBuffer, alpha_min, activated=gs_data.activations())
