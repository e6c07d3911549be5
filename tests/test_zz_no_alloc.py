"""gt_render_batch_noalloc: the batched render for callers that cannot
allocate while they render (a frame loop that must not stall on
cudaMalloc/cudaFree, which synchronise the device; a process whose GPU memory
is owned by another allocator).  Its scratch lives in a fixed device array,
so this test calls it through the C ABI twice in a row and checks each result
against gt_render_batch on the same views, bit for bit (the tolerance of the
other parity tests).  The file name sorts last so that a run stopping at the
first failure has run every other test already; it also passes alone."""
import ctypes as C
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
for p in (ROOT, os.path.join(ROOT, "webgpu-gaussiantracer_b200")):
    if p not in sys.path:
        sys.path.insert(0, p)

from gtrace import _lib as L  # noqa: E402
from gtrace import synth  # noqa: E402

pytestmark = pytest.mark.gpu


def _scene(lib, ctx, n, seed, alpha_min):
    rec = np.ascontiguousarray(synth.pack(synth.raw_small(n=n, seed=seed)).gaussiansBuffer)
    h = C.c_void_p()
    assert lib.gt_scene_create(ctx, rec.ctypes.data_as(C.c_void_p), rec.shape[0], 320, alpha_min, 0,
                               C.byref(h)) == L.GT_OK, L.last_error(ctx)
    return h


def test_noalloc_batch_matches_gt_render_batch():
    lib = L.load()
    ctx = C.c_void_p()
    assert lib.gt_context_create(0, C.byref(ctx)) == L.GT_OK, L.last_error(None)
    buffers = []
    try:
        s1 = _scene(lib, ctx, 1200, 31, 0.01)
        s2 = _scene(lib, ctx, 2000, 32, 0.05)
        shapes = [(s1, synth.view(37, 21, (0.0, 0.0, 4.0), k=6), 37, 21),
                  (s2, synth.view(64, 40, (1.0, 2.0, 3.5), k=16), 64, 40),
                  (s1, synth.view(16, 16, (0.5, -3.0, 2.0), k=3), 16, 16)]
        count = len(shapes)

        def items_for(outs):
            items = (L.BatchItem * count)()
            for i, (sc, v, w, h) in enumerate(shapes):
                items[i].scene = sc
                items[i].u = L.Uniforms.from_buffer_copy(v.uniforms.tobytes())
                items[i].w, items[i].h = w, h
                items[i].out_rgba = outs[i]
                items[i].dL_drgba = None
            return items

        def device_buffers():
            outs = []
            for _, _, w, h in shapes:
                p = C.c_void_p()
                assert lib.gt_device_alloc(ctx, w * h * 16, C.byref(p)) == L.GT_OK
                buffers.append(p.value)
                outs.append(p.value)
            return outs

        def download(outs):
            res = []
            for (_, _, w, h), p in zip(shapes, outs):
                a = np.empty((h, w, 4), np.float32)
                assert lib.gt_memcpy(ctx, a.ctypes.data_as(C.c_void_p), C.c_void_p(p), w * h * 16, 1) == L.GT_OK
                res.append(a)
            return res

        ref_outs = device_buffers()
        st = L.RenderStats()
        assert lib.gt_render_batch(ctx, items_for(ref_outs), count, L.GT_FLAG_OUTPUT_DEVICE,
                                   C.byref(st)) == L.GT_OK, L.last_error(ctx)
        ref = download(ref_outs)
        assert st.rays == sum(w * h for _, _, w, h in shapes)

        na_outs = device_buffers()
        for call in range(2):  # the static scratch is reused: two calls in a row
            for p, (_, _, w, h) in zip(na_outs, shapes):
                zero = np.zeros(w * h * 4, np.float32)
                assert lib.gt_memcpy(ctx, C.c_void_p(p), zero.ctypes.data_as(C.c_void_p), w * h * 16, 0) == L.GT_OK
            st2 = L.RenderStats()
            rc = lib.gt_render_batch_noalloc(ctx, items_for(na_outs), count, L.GT_FLAG_OUTPUT_DEVICE, C.byref(st2))
            assert rc == L.GT_OK, L.last_error(ctx)
            got = download(na_outs)
            for a, b in zip(got, ref):
                np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
            assert st2.rays == st.rays and st2.entries == st.entries and st2.status_flags == 0

        assert st2.kernel_ms > 0.0 and st2.total_ms >= st2.kernel_ms

        # progressive anti-aliasing: frame 0 replaces the image, frame 1 blends
        # into it, as gt_render_batch does
        aa_ref, aa_na = device_buffers(), device_buffers()
        for frame in range(2):
            for outs, fn in ((aa_ref, lib.gt_render_batch), (aa_na, lib.gt_render_batch_noalloc)):
                its = items_for(outs)
                for i in range(count):
                    its[i].u.accumulated_frames = frame
                assert fn(ctx, its, count, L.GT_FLAG_OUTPUT_DEVICE | L.GT_FLAG_ANTIALIAS, None) == L.GT_OK, \
                    L.last_error(ctx)
            for a, b in zip(download(aa_na), download(aa_ref)):
                np.testing.assert_array_equal(a.view(np.uint32), b.view(np.uint32))
        assert not all(np.array_equal(a, b) for a, b in zip(download(aa_na), ref))  # jittered samples

        # sizes beyond the fixed scratch, host outputs and checkpoints are rejected
        big = (L.BatchItem * 257)()
        assert lib.gt_render_batch_noalloc(ctx, big, 257, L.GT_FLAG_OUTPUT_DEVICE, None) == L.GT_ERR_INVALID_ARG
        assert "256" in L.last_error(ctx)
        assert lib.gt_render_batch_noalloc(ctx, items_for(na_outs), count, 0, None) == L.GT_ERR_INVALID_ARG
        assert lib.gt_render_batch_noalloc(ctx, items_for(na_outs), count,
                                           L.GT_FLAG_OUTPUT_DEVICE | L.GT_FLAG_CHECKPOINT, None) == L.GT_ERR_INVALID_ARG
    finally:
        for p in buffers:
            lib.gt_device_free(ctx, C.c_void_p(p))
        lib.gt_context_destroy(ctx)


def test_noalloc_tile_packet_path_matches_gt_render_batch():
    """A view of at least 80 8x4 tiles per SM: the call runs the tile-packet
    kernel, which here has no handoff buffer (every packet finishes its own
    rays), while gt_render_batch hands the long rays to the warp-per-ray
    kernel.  Same image bits, same counters; pixels of a stratified subset
    equal the oracle's."""
    from oracle import oracle
    lib = L.load()
    ctx = C.c_void_p()
    assert lib.gt_context_create(0, C.byref(ctx)) == L.GT_OK, L.last_error(None)
    buffers = []
    try:
        pg = synth.pack(synth.raw_clusters(50_000, synth.SEED_BASE + 71))
        rec = np.ascontiguousarray(pg.gaussiansBuffer)
        sc = C.c_void_p()
        assert lib.gt_scene_create(ctx, rec.ctypes.data_as(C.c_void_p), rec.shape[0], 320, 0.01, 0,
                                   C.byref(sc)) == L.GT_OK, L.last_error(ctx)
        w, h = 1280, 720
        v = synth.view(w, h, (0.0, 0.0, 9.0), k=16)
        imgs = []
        for fn in (lib.gt_render_batch, lib.gt_render_batch_noalloc, lib.gt_render_batch_noalloc):
            p = C.c_void_p()
            assert lib.gt_device_alloc(ctx, w * h * 16, C.byref(p)) == L.GT_OK
            buffers.append(p.value)
            items = (L.BatchItem * 1)()
            items[0].scene = sc
            items[0].u = L.Uniforms.from_buffer_copy(v.uniforms.tobytes())
            items[0].w, items[0].h = w, h
            items[0].out_rgba = p.value
            st = L.RenderStats()
            assert fn(ctx, items, 1, L.GT_FLAG_OUTPUT_DEVICE, C.byref(st)) == L.GT_OK, L.last_error(ctx)
            assert st.rays == w * h and st.status_flags == 0
            a = np.empty((h, w, 4), np.float32)
            assert lib.gt_memcpy(ctx, a.ctypes.data_as(C.c_void_p), C.c_void_p(p.value), w * h * 16, 1) == L.GT_OK
            imgs.append((a, st.entries, st.contributing))
        ref, na, na2 = imgs
        for got in (na, na2):
            np.testing.assert_array_equal(got[0].view(np.uint32), ref[0].view(np.uint32))
            assert got[1:] == ref[1:]
        pix = (np.arange(7, h, 24)[:, None] * w + np.arange(5, w, 24)[None, :]).reshape(-1).astype(np.uint32)
        oref, _ = oracle.Scene(rec, 0.01, "f32").render(v.uniforms, w, h, pixels=pix)
        np.testing.assert_array_equal(na[0].reshape(-1, 4)[pix].view(np.uint32), oref.view(np.uint32))
        lib.gt_scene_destroy(sc)
    finally:
        for p in buffers:
            lib.gt_device_free(ctx, C.c_void_p(p))
        lib.gt_context_destroy(ctx)
