"""Display-side rows on the GPU, bit for bit against the oracle:
progressive anti-aliasing (GT_FLAG_ANTIALIAS: the reference's `antialiasing`
path, src/GS_shader.ts:275-308) through gt_render with host and device
outputs and through gt_render_batch, and the tone map (gt_tonemap,
src/toneMapper.ts:15-24)."""
import os
import tempfile

import numpy as np
import pytest

from conftest import small_scene, view
from gtrace import _lib as L
from gtrace.image import read_ppm, write_ppm
from gtrace.tracer import Scene
from oracle import oracle

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 4).view(np.uint32)


@pytest.mark.parametrize("debug_mode", [0, 1, 2])
def test_antialias_frames_match_oracle(ctx, debug_mode):
    pg = small_scene(n=3000, seed=41)
    w, h = 61, 37
    scene = Scene(ctx, pg.gaussiansBuffer, 0.01)
    osc = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32")
    acc_gpu = np.zeros((h, w, 4), np.float32)
    acc_ref = np.zeros((w * h, 4), np.float32)
    dev = ctx.device_alloc(w * h * 16)
    try:
        for f in range(4):
            v = view(w, h, k=5, accumulated_frames=f, debug_mode=debug_mode)
            ctx.render(scene, v.uniforms, w, h, out=acc_gpu, antialias=True)
            osc.render_accum(v.uniforms, w, h, acc_ref)
            assert np.array_equal(_bits(acc_gpu), acc_ref.view(np.uint32)), f
            # the same frame into a device buffer that holds the previous average
            if f == 0:
                ctx.memcpy(dev, acc_gpu.ctypes.data, w * h * 16, 0)
            else:
                u = np.frombuffer(bytes(v.uniforms), np.uint8)
                st = ctx._lib.gt_render(ctx.handle, scene.handle, L.Uniforms.from_buffer_copy(u.tobytes()), w, h,
                                        L.C.c_void_p(dev), L.GT_FLAG_OUTPUT_DEVICE | L.GT_FLAG_ANTIALIAS, None)
                ctx.check(st)
                back = np.zeros((h, w, 4), np.float32)
                ctx.memcpy(back.ctypes.data, dev, w * h * 16, 1)
                assert np.array_equal(_bits(back), acc_ref.view(np.uint32)), f
    finally:
        ctx.device_free(dev)
        scene.close()


def test_antialias_batch_matches_single(ctx):
    pg = small_scene(n=2500, seed=42)
    scene = Scene(ctx, pg.gaussiansBuffer, 0.01)
    sizes = [(40, 24), (33, 17)]
    singles = [np.zeros((h, w, 4), np.float32) for w, h in sizes]
    batched = [np.zeros((h, w, 4), np.float32) for w, h in sizes]
    for f in range(3):
        views = [view(w, h, pos=(0.3 * i, 0.0, 4.0), k=6, accumulated_frames=f) for i, (w, h) in enumerate(sizes)]
        for v, out in zip(views, singles):
            ctx.render(scene, v.uniforms, v.width, v.height, out=out, antialias=True)
        items = (L.BatchItem * len(views))()
        for i, (v, out) in enumerate(zip(views, batched)):
            items[i].scene = scene.handle
            items[i].u = L.Uniforms.from_buffer_copy(bytes(v.uniforms))
            items[i].w, items[i].h = v.width, v.height
            items[i].out_rgba = out.ctypes.data
            items[i].dL_drgba = None
        ctx.check(ctx._lib.gt_render_batch(ctx.handle, items, len(views), L.GT_FLAG_ANTIALIAS, None))
        for a, b in zip(singles, batched):
            assert np.array_equal(_bits(a), _bits(b)), f
    scene.close()


def test_antialias_rejects_checkpoint(ctx):
    pg = small_scene(n=500, seed=43)
    scene = Scene(ctx, pg.gaussiansBuffer, 0.01)
    v = view(16, 16, k=4)
    out = np.zeros((16, 16, 4), np.float32)
    u = L.Uniforms.from_buffer_copy(bytes(v.uniforms))
    st = ctx._lib.gt_render(ctx.handle, scene.handle, u, 16, 16, out.ctypes.data_as(L.C.c_void_p),
                            L.GT_FLAG_ANTIALIAS | L.GT_FLAG_CHECKPOINT, None)
    assert st == L.GT_ERR_INVALID_ARG
    ctx.render(scene, v.uniforms, 16, 16)  # the context is still usable
    scene.close()


@pytest.mark.parametrize("mode", [L.GT_TONEMAP_HDR, L.GT_TONEMAP_EXPOSURE, L.GT_TONEMAP_EXPOSURE_GAMMA])
def test_tonemap_matches_oracle(ctx, mode):
    pg = small_scene(n=3000, seed=44)
    scene = Scene(ctx, pg.gaussiansBuffer, 0.01)
    v = view(97, 65, k=6)
    img = ctx.render(scene, v.uniforms, v.width, v.height)
    rs = np.random.Generator(np.random.PCG64(6))
    edge = np.concatenate([rs.uniform(-1.0, 4.0, (4000, 4)),
                           [[np.nan, np.inf, -np.inf, 0.0], [0.5 / 255, 1.5 / 255, 1.0, 254.5 / 255]]])
    for data in (img, edge.astype(np.float32)):
        got = ctx.tonemap(data, mode, 1.66)
        want = oracle.tonemap(data, mode, 1.66)
        assert np.array_equal(got.reshape(-1, 4), want)
    # device buffers, asynchronous
    n = v.width * v.height
    src, dst = ctx.device_alloc(n * 16), ctx.device_alloc(n * 4)
    ctx.memcpy(src, img.ctypes.data, n * 16, 0)
    ctx.check(ctx._lib.gt_tonemap(ctx.handle, L.C.c_void_p(src), n, mode, 1.66, L.C.c_void_p(dst),
                                  L.GT_FLAG_INPUT_DEVICE | L.GT_FLAG_OUTPUT_DEVICE | L.GT_FLAG_ASYNC))
    ctx.synchronize()
    back = np.zeros((n, 4), np.uint8)
    ctx.memcpy(back.ctypes.data, dst, n * 4, 1)
    assert np.array_equal(back, oracle.tonemap(img, mode, 1.66))
    ctx.device_free(src)
    ctx.device_free(dst)
    with tempfile.TemporaryDirectory() as d:
        p = os.path.join(d, "frame.ppm")
        rgba8 = ctx.tonemap(img, mode)
        write_ppm(p, rgba8)
        assert np.array_equal(read_ppm(p), rgba8[:, :, :3])
    scene.close()
