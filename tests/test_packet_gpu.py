"""The tile-packet kernel (one warp per 8x4 tile of rays, gt_packet.cu)
against the oracle on the cases the other parity tests cover with the
default choice.  At test image sizes the default is the warp-per-ray kernel,
so every case here installs block_threads = 32 for its view first
(gt_set_tune); the results must be the oracle's, bit for bit.  The last
test renders the full-size batched configuration, where the default is the
tile packets."""
import numpy as np
import pytest

from conftest import small_scene, view
from oracle import oracle
from gtrace import synth
from gtrace.tracer import Scene
from gtrace.uniforms import with_fields

pytestmark = pytest.mark.gpu


def _bits(a):
    return np.ascontiguousarray(a, dtype=np.float32).reshape(-1, 4).view(np.uint32)


def _packet_render(ctx, scene, u, w, h, kbuf=32, **kw):
    ctx.set_tune(scene, u, w, h, kbuf=kbuf, block_threads=32)
    try:
        return ctx.render(scene, u, w, h, **kw)
    finally:
        ctx._lib.gt_autotune_reset(ctx._h)


def test_uniform_variants_and_sizes(ctx):
    pg = small_scene(n=2500, seed=51)
    g = Scene(ctx, pg.gaussiansBuffer, 0.05)
    o = oracle.Scene(pg.gaussiansBuffer, 0.05, "f32")
    base = view(40, 28, k=5).uniforms
    for u in [base, with_fields(base, early_stop=1), with_fields(base, early_stop=3), with_fields(base, T_min=0.5),
              with_fields(base, sh_degree_max=0), with_fields(base, sh_degree_max=2),
              with_fields(base, alpha_min=0.3), with_fields(base, t_min=3.9), with_fields(base, t_max=4.2)]:
        img = _packet_render(ctx, g, u, 40, 28)
        ref, _ = o.render(u, 40, 28)
        assert np.array_equal(_bits(img), ref.view(np.uint32))
    for w, h in [(1, 1), (9, 5), (130, 7), (33, 65)]:
        v = view(w, h, k=7)
        img = _packet_render(ctx, g, v.uniforms, w, h)
        ref, _ = o.render(v.uniforms, w, h)
        assert np.array_equal(_bits(img), ref.view(np.uint32)), (w, h)


def test_camera_inside_and_small_scenes(ctx):
    pg = small_scene(n=2000, seed=52)
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    o = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32")
    v = view(40, 40, pos=(0.05, -0.02, 0.1), target=(1.0, 0.3, -2.0), k=6)
    img = _packet_render(ctx, g, v.uniforms, 40, 40)
    ref, _ = o.render(v.uniforms, 40, 40)
    assert np.array_equal(_bits(img), ref.view(np.uint32))
    empty = Scene(ctx, np.zeros((0, 80), np.float32), 0.01)
    img = _packet_render(ctx, empty, view(16, 16).uniforms, 16, 16)
    assert (img[..., :3] == 0).all() and (img[..., 3] == 1).all()
    rec = np.zeros((1, 80), np.float32)
    rec[0, 4:7] = 0.3
    rec[0, 8] = 1.0
    rec[0, 12] = 0.9
    rec[0, 16:19] = (0.5, 0.1, -0.3)
    one = Scene(ctx, rec, 0.01)
    v = view(32, 32, k=2)
    img = _packet_render(ctx, one, v.uniforms, 32, 32)
    ref, _ = oracle.Scene(rec, 0.01, "f32").render(v.uniforms, 32, 32)
    assert np.array_equal(_bits(img), ref.view(np.uint32)) and img[..., :3].max() > 0


def test_dense_scene_many_rounds(ctx):
    """Many rounds per ray and k-buffers that run out several times."""
    pg = small_scene(n=12000, seed=53)
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    o = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32")
    for k, kbuf in [(1, 24), (3, 32), (16, 32), (32, 64)]:
        v = view(48, 40, k=k, T_min=0.0001)
        img = _packet_render(ctx, g, v.uniforms, 48, 40, kbuf=kbuf)
        ref, _ = o.render(v.uniforms, 48, 40)
        assert np.array_equal(_bits(img), ref.view(np.uint32)), (k, kbuf)


def test_antialias_frames(ctx):
    pg = small_scene(n=3000, seed=54)
    w, h = 45, 29
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    o = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32")
    acc_gpu = np.zeros((h, w, 4), np.float32)
    acc_ref = np.zeros((w * h, 4), np.float32)
    for f in range(3):
        v = view(w, h, k=5, accumulated_frames=f)
        _packet_render(ctx, g, v.uniforms, w, h, out=acc_gpu, antialias=True)
        o.render_accum(v.uniforms, w, h, acc_ref)
        assert np.array_equal(_bits(acc_gpu), acc_ref.view(np.uint32)), f


def test_batch_of_views_and_scenes(ctx):
    pa = small_scene(n=1500, seed=55)
    pb = small_scene(n=2500, seed=56)
    ga, gb = Scene(ctx, pa.gaussiansBuffer, 0.01), Scene(ctx, pb.gaussiansBuffer, 0.02)
    oa, ob = oracle.Scene(pa.gaussiansBuffer, 0.01, "f32"), oracle.Scene(pb.gaussiansBuffer, 0.02, "f32")
    views = [(ga, view(37, 21, k=4).uniforms, 37, 21), (gb, view(24, 40, k=9).uniforms, 24, 40),
             (ga, view(16, 16, pos=(1.0, 2.0, 3.5), k=16).uniforms, 16, 16)]
    ctx.set_tune(views[0][0], views[0][1], 37, 21, kbuf=32, block_threads=32)  # the batch takes item 0's shape
    try:
        outs, st = ctx.render_batch(views)
    finally:
        ctx._lib.gt_autotune_reset(ctx._h)
    for (sc, u, w, h), out in zip(views, outs):
        ref, _ = (oa if sc is ga else ob).render(u, w, h)
        assert np.array_equal(_bits(out), ref.view(np.uint32))
    assert st["rays"] == 37 * 21 + 24 * 40 + 16 * 16


@pytest.mark.parametrize("handoff_after", [0, 1, 6, 64])
def test_handoff_across_views(ctx, handoff_after):
    """Rays that reach the packets' traversal limit go to the warp-per-ray
    kernel with their compositing state, in a batch of views of two scenes.
    Dense scenes, k = 2 and 8-entry buffers make most rays reach it; every
    view must equal the oracle bit for bit, for the default hand-off point
    (0: after 3 traversals) and others the tuner may choose."""
    pa = small_scene(n=12000, seed=57)
    pb = small_scene(n=9000, seed=58)
    ga, gb = Scene(ctx, pa.gaussiansBuffer, 0.01), Scene(ctx, pb.gaussiansBuffer, 0.01)
    oa, ob = oracle.Scene(pa.gaussiansBuffer, 0.01, "f32"), oracle.Scene(pb.gaussiansBuffer, 0.01, "f32")
    views = [(ga, view(40, 24, k=2, T_min=0.0001).uniforms, 40, 24),
             (gb, view(24, 40, k=2, T_min=0.0001).uniforms, 24, 40),
             (ga, view(33, 17, pos=(1.0, 2.0, 3.5), k=2, T_min=0.0001).uniforms, 33, 17),
             (gb, view(16, 24, pos=(-2.0, 0.5, 3.0), k=2, T_min=0.0001).uniforms, 16, 24)]
    ctx.set_tune(views[0][0], views[0][1], 40, 24, kbuf=8, block_threads=32, handoff_after=handoff_after)
    try:
        outs, st = ctx.render_batch(views)
    finally:
        ctx._lib.gt_autotune_reset(ctx._h)
    for (sc, u, w, h), out in zip(views, outs):
        ref, _ = (oa if sc is ga else ob).render(u, w, h)
        assert np.array_equal(_bits(out), ref.view(np.uint32))
    rays = sum(w * h for _, _, w, h in views)
    assert st["rays"] == rays
    # (the packets hand over once every tile of the launch is taken, so even
    # the latest hand-off point hands rays over at these sizes)
    assert st["handed"] > rays // 4, st["handed"]


@pytest.mark.parametrize("mode", [1, 2])
def test_checkpointing_forward_and_gradients(ctx, mode):
    """gt_backward's checkpointing forward as tile packets (with rays handed
    to the warp-per-ray kernel after three traversals): the image is the
    oracle's and the gradients match the FP64 oracle's adjoint."""
    from test_backward_gpu import _check, _ref_grad
    pg = small_scene(n=4000, seed=57)
    rec = pg.gaussiansBuffer
    w, h = 48, 40
    v = view(w, h, k=6, T_min=0.001)
    s = Scene(ctx, rec, 0.01)
    ctx.set_tune(s, v.uniforms, w, h, kbuf=32, block_threads=32)
    try:
        img = ctx.render(s, v.uniforms, w, h, checkpoint=True)
        ref, _ = oracle.Scene(rec, 0.01, "f32").render(v.uniforms, w, h)
        assert np.array_equal(_bits(img), ref.view(np.uint32))
        g = np.random.default_rng(11).normal(size=(h, w, 4)).astype(np.float32)
        got, info = ctx.backward(s, v.uniforms, w, h, g, mode=mode)
    finally:
        ctx._lib.gt_autotune_reset(ctx._h)
    assert info["used_mode"] == mode
    _check(got, _ref_grad(rec, 0.01, v.uniforms, w, h, g))


@pytest.mark.parametrize("pos", [(0.0, 0.0, 40.0), (0.3, 0.2, 0.9), (2.5, -1.5, 2.0)])
def test_entry_face_test_across_distances(ctx, pos):
    """Near and far cameras (object-space origins from ~1 to ~10^4 proxy
    radii): the tile packets give the oracle's image, bit for bit."""
    pg = small_scene(n=6000, seed=58)
    g = Scene(ctx, pg.gaussiansBuffer, 0.01)
    o = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32")
    v = view(56, 44, pos=pos, k=8, T_min=0.001)
    img = _packet_render(ctx, g, v.uniforms, 56, 44)
    ref, _ = o.render(v.uniforms, 56, 44)
    assert np.array_equal(_bits(img), ref.view(np.uint32))


def test_batched_config_full_size_equals_single_renders(ctx):
    """The batched configuration at full size (8 scenes of 100k-1M Gaussians,
    64 views up to 1920x1080, 44.7M rays in one launch: tile packets, and a
    handoff buffer that fills up): every view equals its own single render
    bit for bit."""
    raw_scenes, views = synth.batched_scenes_config()
    scenes = [Scene(ctx, synth.pack(raw).gaussiansBuffer, amin) for raw, amin in raw_scenes]
    items = []
    try:
        for s, w, h, pos in views:
            v = synth.view(w, h, pos, k=16, alpha_min=raw_scenes[s][1])
            items.append((scenes[s], v.uniforms, w, h, ctx.device_alloc(w * h * 16)))
        _, st = ctx.render_batch(items, device_outputs=True)
        assert st["rays"] == sum(w * h for _, _, w, h, _ in items)
        for sc, u, w, h, ptr in items:
            got = np.zeros((h, w, 4), np.float32)
            ctx.memcpy(got.ctypes.data, ptr, w * h * 16, 1)
            assert np.array_equal(_bits(got), _bits(ctx.render(sc, u, w, h)))
    finally:
        for it in items:
            ctx.device_free(it[4])
        for s in scenes:
            s.close()
