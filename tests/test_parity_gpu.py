"""GPU parity: the CUDA tracer against the oracle's float build.

The tracer and the oracle follow the same binary32 operation order, so
images, hit sequences, hit t values and alphas must match bit for bit.  The
oracle's double build gives the FP64 error statistics."""
import ctypes as C

import numpy as np
import pytest

from conftest import small_scene, view
from oracle import oracle
from gtrace import synth
from gtrace import _lib as L
from gtrace.tracer import Scene, _uniforms
from gtrace.uniforms import with_fields

pytestmark = pytest.mark.gpu


def _both(ctx, packed, amin):
    return Scene(ctx, packed, amin), oracle.Scene(packed, amin, "f32")


def _assert_hits_equal(got, ref, max_entries):
    np.testing.assert_array_equal(got["count"], ref["count"])
    np.testing.assert_array_equal(got["rounds"], ref["rounds"])
    n = np.minimum(got["count"], max_entries)
    for q in range(len(n)):
        m = n[q]
        np.testing.assert_array_equal(got["pidx"][q, :m], ref["pidx"][q, :m])
        np.testing.assert_array_equal(got["t"][q, :m].view(np.uint32), ref["t"][q, :m].view(np.uint32))
        np.testing.assert_array_equal(got["alpha"][q, :m].view(np.uint32), ref["alpha"][q, :m].view(np.uint32))


@pytest.mark.parametrize("k", [1, 2, 4, 6, 8, 11, 16, 24, 32])
def test_image_bit_exact_across_k(ctx, k):
    pg = small_scene(n=2048, seed=7)
    g, o = _both(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 64, 48
    v = view(w, h, k=k)
    img = ctx.render(g, v.uniforms, w, h)
    ref, _ = o.render(v.uniforms, w, h)
    np.testing.assert_array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))


@pytest.mark.parametrize("k", [1, 6, 16])
def test_hit_sequences_bit_exact(ctx, k):
    pg = small_scene(n=2048, seed=9)
    g, o = _both(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 40, 30
    v = view(w, h, k=k)
    pix = np.arange(w * h, dtype=np.uint32)
    got = ctx.render_hits(g, v.uniforms, w, h, pix, max_entries=256)
    _, ref = o.render(v.uniforms, w, h, pixels=pix, max_entries=256)
    _assert_hits_equal(got, ref, 256)
    assert got["rounds"].max() >= 2  # several rounds happened


def test_small_config_full_image(ctx):
    """16,384 Gaussians, 256x256, k = 6, alpha_min 0.01, T_min 0.01: every
    pixel bit-exact; hit sequences of a stratified subset equal; FP64 RMSE."""
    pg, amin, v = synth.small_config()
    g, o = _both(ctx, pg.gaussiansBuffer, amin)
    img, st = ctx.render(g, v.uniforms, v.width, v.height, stats=True)
    ref, rh = o.render(v.uniforms, v.width, v.height, max_entries=0)
    np.testing.assert_array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))
    assert st["rays"] == v.width * v.height
    assert st["entries"] == int(rh["count"].sum())
    pix = np.arange(0, v.width * v.height, 97, dtype=np.uint32)
    got = ctx.render_hits(g, v.uniforms, v.width, v.height, pix, max_entries=256)
    _, ref_h = o.render(v.uniforms, v.width, v.height, pixels=pix, max_entries=256)
    _assert_hits_equal(got, ref_h, 256)
    o64 = oracle.Scene(pg.gaussiansBuffer, amin, "f64")
    r64, _ = o64.render(v.uniforms, v.width, v.height)
    rmse = float(np.sqrt(np.mean((img.reshape(-1, 4)[:, :3] - r64[:, :3]) ** 2)))
    assert rmse < 1e-4


@pytest.mark.parametrize("w,h", [(1, 1), (37, 23), (9, 5), (130, 7)])
def test_any_image_size(ctx, w, h):
    """Sizes need not be multiples of 8 (the reference requires that,
    webrtx/src/pass_encoder.ts:52-56)."""
    pg = small_scene(n=800, seed=4)
    g, o = _both(ctx, pg.gaussiansBuffer, 0.01)
    v = view(w, h, k=4)
    img = ctx.render(g, v.uniforms, w, h)
    ref, _ = o.render(v.uniforms, w, h)
    np.testing.assert_array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))


def test_empty_and_culled_scenes(ctx):
    v = view(16, 16)
    empty = Scene(ctx, np.zeros((0, 80), np.float32), 0.01)
    img = ctx.render(empty, v.uniforms, 16, 16)
    assert (img[..., :3] == 0).all() and (img[..., 3] == 1).all()
    pg = small_scene(n=100, seed=1)
    rec = pg.gaussiansBuffer.copy()
    rec[:, 12] = 0.005  # every opacity below alpha_min: no proxies
    culled = Scene(ctx, rec, 0.01)
    assert culled.info()["n_kept"] == 0
    img = ctx.render(culled, v.uniforms, 16, 16)
    assert (img[..., :3] == 0).all()


def test_single_proxy_scene(ctx):
    rec = np.zeros((1, 80), np.float32)
    rec[0, 4:7] = 0.3
    rec[0, 8] = 1.0
    rec[0, 12] = 0.9
    rec[0, 16:19] = (0.5, 0.1, -0.3)
    g, o = _both(ctx, rec, 0.01)
    assert g.info()["n_kept"] == 1
    v = view(32, 32, k=2)
    img = ctx.render(g, v.uniforms, 32, 32)
    ref, _ = o.render(v.uniforms, 32, 32)
    np.testing.assert_array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))
    assert img[..., :3].max() > 0


@pytest.mark.parametrize("mode", [1, 2])
def test_debug_modes(ctx, mode):
    """debugMode 1 (closest proxy hit coloured by SH along the ray) and 2
    (front-face hit count, bucketed) against the oracle."""
    pg = small_scene(n=1500, seed=8)
    g, o = _both(ctx, pg.gaussiansBuffer, 0.2)
    v = view(48, 32, k=6, debug_mode=mode)
    img = ctx.render(g, v.uniforms, 48, 32)
    ref, _ = o.render(v.uniforms, 48, 32)
    np.testing.assert_array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))


def test_uniform_variants(ctx):
    pg = small_scene(n=1500, seed=12)
    g, o = _both(ctx, pg.gaussiansBuffer, 0.05)
    base = view(32, 24, k=4).uniforms
    for u in [with_fields(base, early_stop=1), with_fields(base, early_stop=3), with_fields(base, T_min=0.5),
              with_fields(base, sh_degree_max=0), with_fields(base, sh_degree_max=1),
              with_fields(base, sh_degree_max=2), with_fields(base, alpha_min=0.3),
              with_fields(base, t_min=3.9), with_fields(base, t_max=4.2)]:
        img = ctx.render(g, u, 32, 24)
        ref, _ = o.render(u, 32, 24)
        np.testing.assert_array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))


def test_camera_inside_scene(ctx):
    """Proxies containing the camera give no front-face hit (skipped)."""
    pg = small_scene(n=2000, seed=13)
    g, o = _both(ctx, pg.gaussiansBuffer, 0.01)
    v = view(40, 40, pos=(0.05, -0.02, 0.1), target=(1.0, 0.3, -2.0), k=6)
    img = ctx.render(g, v.uniforms, 40, 40)
    ref, _ = o.render(v.uniforms, 40, 40)
    np.testing.assert_array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))


def test_invalid_arguments(ctx):
    pg = small_scene(n=10, seed=1)
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    v = view(8, 8)
    for bad in [with_fields(v.uniforms, k=0), with_fields(v.uniforms, k=33), with_fields(v.uniforms, debug_mode=3)]:
        with pytest.raises(L.GTraceError) as e:
            ctx.render(g, bad, 8, 8)
        assert e.value.status == L.GT_ERR_INVALID_ARG
    with pytest.raises(L.GTraceError):
        ctx.render(g, v.uniforms, 0, 8, out=np.zeros(0, np.float32))
    with pytest.raises(L.GTraceError) as e:
        Scene(ctx, pg.gaussiansBuffer, 1.5)
    assert e.value.status == L.GT_ERR_INVALID_ARG
    # at most 2^31 pixels, and at most 2^31 work slots once the 8x4 tile grid
    # is padded to 16x16-tile blocks (a 2^31 x 1 image has 2^31 pixels but
    # 2^37 slots); both are rejected before anything is launched
    u = _uniforms(v.uniforms)
    dev = ctx.device_alloc(64)
    try:
        for w, h in [(1 << 31, 1), (1 << 28, 8), (65544, 32760)]:
            assert ctx._lib.gt_render(ctx.handle, g.handle, C.byref(u), w, h, C.c_void_p(dev),
                                      L.GT_FLAG_OUTPUT_DEVICE, None) == L.GT_ERR_INVALID_ARG
    finally:
        ctx.device_free(dev)


def test_device_output_and_async(ctx):
    pg = small_scene(n=1000, seed=14)
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 33, 17
    v = view(w, h, k=6)
    host = ctx.render(g, v.uniforms, w, h)
    dev = ctx.device_alloc(w * h * 16)
    try:
        ctx.render_device(g, v.uniforms, w, h, dev, asynchronous=True)
        ctx.synchronize()
        out = np.zeros((h, w, 4), np.float32)
        ctx.memcpy(out.ctypes.data, dev, w * h * 16, 1)
    finally:
        ctx.device_free(dev)
    np.testing.assert_array_equal(out, host)


@pytest.mark.parametrize("block_threads", [128, 32])
def test_page_locked_host_output(ctx, block_threads):
    """A page-locked host buffer is written by the trace kernels directly
    (no staging copy); the image equals the one a pageable buffer receives
    through the copy, bit for bit, for both forward kernels, with pixels
    handed between them, and for an anti-aliased frame (which takes the
    staging path)."""
    pg = small_scene(n=6000, seed=16)
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 45, 29
    v = view(w, h, k=4, T_min=0.0001)
    ctx.set_tune(g, v.uniforms, w, h, kbuf=8 if block_threads == 32 else 64, block_threads=block_threads,
                 handoff_after=1)
    pinned = ctx.host_alloc(w * h * 16, np.float32, (h, w, 4))
    try:
        ref = ctx.render(g, v.uniforms, w, h)
        pinned[...] = np.nan
        st = ctx.render(g, v.uniforms, w, h, out=pinned, stats=True)[1]
        assert st["rays"] == w * h
        np.testing.assert_array_equal(pinned.view(np.uint32), ref.view(np.uint32))
        if block_threads == 32:
            assert st["handed"] > 0
        # anti-aliased frames 0 and 1 into the page-locked buffer
        page = np.zeros((h, w, 4), np.float32)
        for f in (0, 1):
            u = with_fields(v.uniforms, accumulated_frames=f)
            ctx.render(g, u, w, h, out=page, antialias=True)
            ctx.render(g, u, w, h, out=pinned, antialias=True)
        np.testing.assert_array_equal(pinned.view(np.uint32), page.view(np.uint32))
    finally:
        ctx._lib.gt_autotune_reset(ctx._h)
        ctx.host_free(pinned)


def test_scene_from_device_buffer(ctx):
    pg = small_scene(n=700, seed=15)
    rec = np.ascontiguousarray(pg.gaussiansBuffer)
    dev = ctx.device_alloc(rec.nbytes)
    try:
        ctx.memcpy(dev, rec.ctypes.data, rec.nbytes, 0)
        g1 = Scene(ctx, None, 0.01, device_ptr=dev, n=rec.shape[0], stride=320)
    finally:
        pass
    g2 = Scene(ctx, rec, 0.01)
    v = view(24, 24)
    a = ctx.render(g1, v.uniforms, 24, 24)
    b = ctx.render(g2, v.uniforms, 24, 24)
    ctx.device_free(dev)
    np.testing.assert_array_equal(a, b)


def test_batch_equals_single_views(ctx):
    """Views of several scenes and sizes in one persistent launch (replayed
    from a captured graph on the second call) equal separate renders."""
    s1 = Scene(ctx, small_scene(n=900, seed=21).gaussiansBuffer, 0.01)
    s2 = Scene(ctx, small_scene(n=1700, seed=22).gaussiansBuffer, 0.05)
    views = [(s1, view(31, 17, k=4).uniforms, 31, 17), (s2, view(20, 40, pos=(1.0, 2.0, 3.5), k=16).uniforms, 20, 40),
             (s1, view(8, 8, k=1).uniforms, 8, 8)]
    for _ in range(2):
        outs, st = ctx.render_batch(views)
        for (sc, u, w, h), out in zip(views, outs):
            np.testing.assert_array_equal(out, ctx.render(sc, u, w, h))
        assert st["rays"] == 31 * 17 + 20 * 40 + 64


def test_autotune_keeps_results(ctx):
    pg = small_scene(n=1200, seed=23)
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    v = view(64, 64, k=6)
    before = ctx.render(g, v.uniforms, 64, 64)
    r = ctx.autotune(g, v.uniforms, 64, 64)
    assert r["blocks_per_sm"] >= 1 and r["best_ms"] > 0 and r["block_threads"] in (32, 128)
    assert r["kbuf"] >= 6 and (r["block_threads"] == 128 or r["kbuf"] <= 64)
    after = ctx.render(g, v.uniforms, 64, 64)
    np.testing.assert_array_equal(before, after)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 5, 16])
def test_tuned_shapes_are_bit_exact(ctx, k):
    """Every k-buffer size and leaf batch gives the same image, bit for bit."""
    pg = small_scene(n=3000, seed=31)
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 48, 40
    v = view(w, h, k=k)
    ref = ctx.render(g, v.uniforms, w, h)
    for kbuf, lb, b in [(k, 8, 4), (min(32, k + 3), 16, 2), (32, 24, 8), (k, 32, 1), (32, 1, 4), (33, 32, 4),
                         (48, 16, 4), (64, 32, 4), (64, 5, 2), (80, 32, 4), (128, 32, 4), (100, 12, 3)]:
        ctx.set_tune(g, v.uniforms, w, h, blocks_per_sm=b, kbuf=kbuf, leaf_batch=lb)
        np.testing.assert_array_equal(ctx.render(g, v.uniforms, w, h), ref, err_msg=f"kbuf={kbuf} lb={lb}")
    with pytest.raises(RuntimeError):
        ctx.set_tune(g, v.uniforms, w, h, kbuf=129)
    ctx._lib.gt_autotune_reset(ctx._h)


@pytest.mark.gpu
@pytest.mark.parametrize("k", [1, 7, 16, 32])
def test_both_kernels_and_packet_kbufs_are_bit_exact(ctx, k):
    """The tile-packet kernel (block_threads 32) at every k-buffer size and
    the warp-per-ray kernel (128) give the oracle's image, bit for bit."""
    pg = small_scene(n=3000, seed=33)
    g, o = _both(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 45, 37
    v = view(w, h, k=k)
    ref, _ = o.render(v.uniforms, w, h)
    for bt, kbuf in [(32, k), (32, 24), (32, 32), (32, 40), (32, 48), (32, 64), (32, 100), (128, 64)]:
        ctx.set_tune(g, v.uniforms, w, h, kbuf=kbuf, block_threads=bt)
        img = ctx.render(g, v.uniforms, w, h)
        np.testing.assert_array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32),
                                      err_msg=f"block_threads={bt} kbuf={kbuf}")
    with pytest.raises(RuntimeError):
        ctx.set_tune(g, v.uniforms, w, h, block_threads=64)
    ctx._lib.gt_autotune_reset(ctx._h)


@pytest.mark.gpu
def test_hierarchies_give_identical_images(ctx):
    """The PLOC and LBVH hierarchies change the traversal order only."""
    pg = small_scene(n=5000, seed=37)
    w, h = 56, 40
    for k in (3, 16):
        v = view(w, h, k=k)
        a = ctx.render(Scene(ctx, pg.gaussiansBuffer, 0.01), v.uniforms, w, h)
        b = ctx.render(Scene(ctx, pg.gaussiansBuffer, 0.01, fast_build=True), v.uniforms, w, h)
        np.testing.assert_array_equal(a, b)
        ref, _ = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32").render(v.uniforms, w, h)
        np.testing.assert_array_equal(a.reshape(-1, 4), ref)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 3, 40])
def test_clustering_with_coincident_particles(ctx, n):
    """Identical particles tie in every merge distance; the build must still
    finish and render what the oracle renders."""
    pg = small_scene(n=1, seed=38)
    rec = np.repeat(pg.gaussiansBuffer[:1], n, axis=0)
    rec[:, 0:3] = 0.0    # at the origin
    rec[:, 4:7] = 0.3    # scales (activated)
    rec[:, 12] = 0.9     # opacity well above alpha_min
    w, h = 24, 20
    v = view(w, h, pos=(0.0, 0.0, 3.0), k=4)
    s = Scene(ctx, rec, 0.01)
    assert s.info()["n_kept"] == n
    img = ctx.render(s, v.uniforms, w, h)
    ref, _ = oracle.Scene(rec, 0.01, "f32").render(v.uniforms, w, h)
    np.testing.assert_array_equal(img.reshape(-1, 4), ref)


def test_clusters_1m_stratified_subset(ctx):
    """1M clustered Gaussians at 1920x1080, k = 16: every 8th pixel in x and y
    (32,400 rays) bit-exact against the oracle's float build, hit sequences
    of every 64th of those equal, and the subset's RMSE against the FP64
    render below 1e-4."""
    pg, amin, v = synth.clusters_1m_config()
    w, h = v.width, v.height
    g = Scene(ctx, pg.gaussiansBuffer, amin)
    img = ctx.render(g, v.uniforms, w, h).reshape(-1, 4)
    ys, xs = np.meshgrid(np.arange(0, h, 8), np.arange(0, w, 8), indexing="ij")
    pix = (ys * w + xs).ravel().astype(np.uint32)
    o = oracle.Scene(pg.gaussiansBuffer, amin, "f32")
    ref, _ = o.render(v.uniforms, w, h, pixels=pix)
    np.testing.assert_array_equal(img[pix].view(np.uint32), ref.view(np.uint32))
    sub = pix[::64]
    got = ctx.render_hits(g, v.uniforms, w, h, sub, max_entries=512)
    _, ref_h = o.render(v.uniforms, w, h, pixels=sub, max_entries=512)
    _assert_hits_equal(got, ref_h, 512)
    del o
    r64, _ = oracle.Scene(pg.gaussiansBuffer, amin, "f64").render(v.uniforms, w, h, pixels=pix)
    rmse = float(np.sqrt(np.mean((img[pix, :3] - r64[:, :3]) ** 2)))
    assert rmse < 1e-4, rmse
    # the tile packets' later hand-off points (the tuner's choices at this
    # size) give the whole image of the default bit for bit
    for ha in (6, 64):
        ctx.set_tune(g, v.uniforms, w, h, kbuf=32, block_threads=32, handoff_after=ha)
        try:
            other = ctx.render(g, v.uniforms, w, h).reshape(-1, 4)
        finally:
            ctx._lib.gt_autotune_reset(ctx._h)
        np.testing.assert_array_equal(other.view(np.uint32), img.view(np.uint32), err_msg=f"handoff_after={ha}")


def test_batched_config_shape(ctx):
    """The batched configuration's structure at 2% of its Gaussian counts:
    8 scenes, 64 views of uneven sizes, per-scene alpha_min; one batched
    launch equals the 64 single renders bit for bit."""
    scenes_raw, views = synth.batched_scenes_config(scale=0.02)
    scenes = [Scene(ctx, synth.pack(r).gaussiansBuffer, a) for r, a in scenes_raw]
    items = [(scenes[s], synth.view(w, h, pos, k=16, alpha_min=scenes_raw[s][1]).uniforms, w, h)
             for s, w, h, pos in views]
    outs, st = ctx.render_batch(items)
    assert st["rays"] == sum(w * h for _, w, h, _ in views)
    for (sc, u, w, h), out in zip(items, outs):
        np.testing.assert_array_equal(out, ctx.render(sc, u, w, h))


@pytest.mark.parametrize("n_pix", [1, 7, 507])
def test_render_hits_any_pixel_count(ctx, n_pix):
    """Pixel lists of any length (the per-pixel output parts of the call's
    device buffer each start on their own aligned boundary)."""
    pg = small_scene(n=2048, seed=12)
    g, o = _both(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 40, 30
    v = view(w, h, k=5)
    pix = np.random.default_rng(n_pix).integers(0, w * h, size=n_pix).astype(np.uint32)
    got = ctx.render_hits(g, v.uniforms, w, h, pix, max_entries=33)
    _, ref = o.render(v.uniforms, w, h, pixels=pix, max_entries=33)
    _assert_hits_equal(got, ref, 33)


@pytest.mark.gpu
def test_batch_debug_modes_after_render_batch_of_same_shape(ctx):
    """Render-only launches use a kernel without the debug modes; a batch of
    the same shape that holds a debug view must still get the kernel that
    has them (the batch graphs are keyed on it)."""
    pg = small_scene(n=3000, seed=71)
    s = Scene(ctx, pg.gaussiansBuffer, 0.01)
    views = [view(40, 32, pos=(0.2 * i, 0.0, 4.0), k=5) for i in range(2)]
    plain = [(s, v.uniforms, v.width, v.height) for v in views]
    out1, _ = ctx.render_batch(plain)
    for v, o in zip(views, out1):
        np.testing.assert_array_equal(o, ctx.render(s, v.uniforms, v.width, v.height))
    for mode in (1, 2):
        dv = view(40, 32, pos=(0.0, 0.0, 4.0), k=5, debug_mode=mode)
        mixed = [(s, dv.uniforms, dv.width, dv.height), plain[1]]
        out2, _ = ctx.render_batch(mixed)
        np.testing.assert_array_equal(out2[0], ctx.render(s, dv.uniforms, dv.width, dv.height))
        np.testing.assert_array_equal(out2[1], out1[1])
        ref, _ = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32").render(dv.uniforms, dv.width, dv.height)
        np.testing.assert_array_equal(out2[0].reshape(-1, 4), ref)
    s.close()
