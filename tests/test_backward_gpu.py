"""GPU adjoint: gt_backward against the oracle's FP64 adjoint (itself checked
against central finite differences in test_backward_cpu.py), both
checkpoint and replay modes, batches and accumulation.  The FP64 reference
runs on the composited entry lists of the float render (which the CUDA
forward reproduces bit for bit), so both sides differentiate the same
piecewise-smooth function.

Tolerance: relative error <= 1e-3 per parameter row in the 2-norm, and per
element |cuda - fp64| <= 1e-3 |fp64| + 1e-4 max|row| (float arithmetic and
atomic summation order against double)."""
import numpy as np
import pytest

from conftest import small_scene, view
from oracle import oracle
from gtrace.tracer import Scene

pytestmark = pytest.mark.gpu


def _ref_grad(rec, amin, uniforms, w, h, g):
    from gtrace.uniforms import unpack_uniforms
    _, hits = oracle.Scene(rec, amin, "f32").render(uniforms, w, h, max_entries=1024)
    s64 = oracle.Scene(rec, amin, "f64")
    return oracle.backward_lists(s64, uniforms, w, h, hits, np.asarray(g, np.float64).reshape(-1, 4),
                                 alpha_min=unpack_uniforms(uniforms)["alpha_min"])


def _check(got, ref, rel=1e-3):
    for i in range(59):
        r = ref[i]
        scale = np.abs(r).max()
        if scale == 0:
            assert np.abs(got[i]).max() <= 1e-6
            continue
        assert np.linalg.norm(got[i] - r) <= rel * np.linalg.norm(r) + 1e-6 * scale, i
        assert (np.abs(got[i] - r) <= rel * np.abs(r) + 1e-4 * scale).mean() >= 0.999, i


@pytest.mark.parametrize("mode", [1, 2])
@pytest.mark.parametrize("k", [4, 16])
def test_gradient_matches_fp64_oracle(ctx, mode, k):
    pg = small_scene(n=1500, seed=41)
    rec = pg.gaussiansBuffer
    w, h = 48, 40
    v = view(w, h, k=k)
    rng = np.random.default_rng(k)
    g = rng.normal(size=(h, w, 4)).astype(np.float32)
    s = Scene(ctx, rec, 0.01)
    got, info = ctx.backward(s, v.uniforms, w, h, g, mode=mode)
    assert info["used_mode"] == mode
    ref = _ref_grad(rec, 0.01, v.uniforms, w, h, g)
    _check(got, ref)
    assert np.abs(got).sum() > 0


def test_checkpoint_and_replay_agree_and_grow(ctx):
    pg = small_scene(n=2000, seed=42)
    s = Scene(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 40, 30
    v = view(w, h, k=2)  # many rounds per ray
    g = np.random.default_rng(3).normal(size=(h, w, 4)).astype(np.float32)
    a, ia = ctx.backward(s, v.uniforms, w, h, g, mode=1, max_rounds=1)
    b, ib = ctx.backward(s, v.uniforms, w, h, g, mode=2, max_rounds=1)
    assert ia["used_mode"] == 1 and ib["used_mode"] == 2
    # replay records one per round (> 1 a ray); checkpoint records hold up to
    # 16 contributing entries each, across rounds, so there are fewer
    assert ib["max_rounds"] > w * h and 0 < ia["max_rounds"] < ib["max_rounds"]
    np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6 * np.abs(a).max())


def test_checkpoint_records_across_handoff_and_pool_growth(ctx):
    """Checkpoint records take a ray's contributing entries across round
    boundaries, and a ray's open record passes from its tile packet to the
    warp-per-ray kernel at the handoff: forced tile packets with 8-entry
    buffers and k = 2 hand rays over after three traversals.  A fresh context
    sizes its first pool from the call before (one pixel), so the forward
    overflows it, counts the records it needed and runs again.  The gradient
    equals the warp-per-ray path's and the FP64 oracle's."""
    from gtrace.tracer import Context
    pg = small_scene(n=2000, seed=42)
    rec = pg.gaussiansBuffer
    w, h = 64, 48
    v = view(w, h, k=2)
    g = np.random.default_rng(5).normal(size=(h, w, 4)).astype(np.float32)
    ref_cuda, _ = ctx.backward(Scene(ctx, rec, 0.01), v.uniforms, w, h, g, mode=1)
    c2 = Context(0)
    try:
        s2 = Scene(c2, rec, 0.01)
        one = view(1, 1, k=2)
        c2.backward(s2, one.uniforms, 1, 1, np.zeros((1, 1, 4), np.float32), mode=1)
        c2.set_tune(s2, v.uniforms, w, h, kbuf=8, block_threads=32)
        got, info = c2.backward(s2, v.uniforms, w, h, g, mode=1)
        assert info["used_mode"] == 1
        assert info["max_rounds"] > 1025  # more records than the first pool held
        got = got.copy()
    finally:
        c2.close()
    np.testing.assert_allclose(got, ref_cuda, rtol=1e-5, atol=1e-6 * np.abs(ref_cuda).max())
    _check(got, _ref_grad(rec, 0.01, v.uniforms, w, h, g))


def test_l2_loss_against_perturbed_target(ctx):
    """The differentiable configuration in miniature: L = sum (rgb - target)^2."""
    from gtrace import synth
    raw = synth.raw_clusters(3000, seed=77)
    target_raw = synth.perturb(raw, seed=78)
    pg, tg = synth.pack(raw), synth.pack(target_raw)
    w, h = 56, 56
    v = view(w, h, pos=(0.0, 0.0, 12.0), k=8)
    s, st = Scene(ctx, pg.gaussiansBuffer, 0.01), Scene(ctx, tg.gaussiansBuffer, 0.01)
    img = ctx.render(s, v.uniforms, w, h)
    tgt = ctx.render(st, v.uniforms, w, h)
    g = np.zeros_like(img)
    g[..., :3] = 2.0 * (img[..., :3] - tgt[..., :3])
    got, _ = ctx.backward(s, v.uniforms, w, h, g)
    ref = _ref_grad(pg.gaussiansBuffer, 0.01, v.uniforms, w, h, g)
    _check(got, ref)


def test_batch_sums_views_and_accumulate_flag(ctx):
    pg = small_scene(n=1200, seed=43)
    s = Scene(ctx, pg.gaussiansBuffer, 0.01)
    v1 = view(32, 24, k=6)
    v2 = view(20, 36, pos=(1.5, 0.5, 3.5), k=6)
    rng = np.random.default_rng(5)
    g1 = rng.normal(size=(24, 32, 4)).astype(np.float32)
    g2 = rng.normal(size=(36, 20, 4)).astype(np.float32)
    a, _ = ctx.backward(s, v1.uniforms, 32, 24, g1)
    b, _ = ctx.backward(s, v2.uniforms, 20, 36, g2)
    res, info = ctx.backward_batch([(s, v1.uniforms, 32, 24, g1), (s, v2.uniforms, 20, 36, g2)])
    np.testing.assert_allclose(res[s], a + b, rtol=1e-5, atol=1e-6 * np.abs(a + b).max())
    acc = a.copy()
    acc2, _ = ctx.backward(s, v2.uniforms, 20, 36, g2, out=acc, accumulate=True)
    np.testing.assert_allclose(acc2, a + b, rtol=1e-5, atol=1e-6 * np.abs(a + b).max())


def test_render_checkpoint_reused_by_backward(ctx):
    """A render with GT_FLAG_CHECKPOINT leaves the round checkpoint in the
    context; the following backward of the same view skips its own forward."""
    pg = small_scene(n=1500, seed=44)
    s = Scene(ctx, pg.gaussiansBuffer, 0.01)
    w, h = 36, 28
    v = view(w, h, k=8)
    g = np.random.default_rng(9).normal(size=(h, w, 4)).astype(np.float32)
    plain = ctx.render(s, v.uniforms, w, h)
    img = ctx.render(s, v.uniforms, w, h, checkpoint=True)
    np.testing.assert_array_equal(img, plain)
    a, ia = ctx.backward(s, v.uniforms, w, h, g, reuse_checkpoint=True)
    assert ia["fwd_ms"] == 0.0
    b, ib = ctx.backward(s, v.uniforms, w, h, g)
    assert ib["fwd_ms"] > 0.0
    np.testing.assert_allclose(a, b, rtol=1e-5, atol=1e-6 * np.abs(b).max())
    # a different view does not reuse the stored checkpoint
    v2 = view(w, h, pos=(0.3, 0.2, 4.0), k=8)
    c, ic = ctx.backward(s, v2.uniforms, w, h, g, reuse_checkpoint=True)
    assert ic["fwd_ms"] > 0.0


def test_l2_loss_helper(ctx):
    n = 1000
    rng = np.random.default_rng(1)
    a = rng.normal(size=(n, 4)).astype(np.float32)
    b = rng.normal(size=(n, 4)).astype(np.float32)
    da, db, dg = (ctx.device_alloc(n * 16) for _ in range(3))
    try:
        ctx.memcpy(da, a.ctypes.data, n * 16, 0)
        ctx.memcpy(db, b.ctypes.data, n * 16, 0)
        loss = ctx.l2_loss(da, db, n, dg)
        g = np.zeros((n, 4), np.float32)
        ctx.memcpy(g.ctypes.data, dg, n * 16, 1)
    finally:
        for p in (da, db, dg):
            ctx.device_free(p)
    d = a[:, :3].astype(np.float64) - b[:, :3]
    assert abs(loss - (d ** 2).sum()) <= 1e-6 * (d ** 2).sum()
    np.testing.assert_allclose(g[:, :3], 2 * (a[:, :3] - b[:, :3]), rtol=1e-6)
    assert (g[:, 3] == 0).all()


@pytest.mark.parametrize("mode", [1, 2])
def test_gradient_with_wide_kbuffer(ctx, mode):
    """A 64-entry k-buffer and a small leaf batch change nothing but speed."""
    pg = small_scene(n=1500, seed=43)
    rec = pg.gaussiansBuffer
    w, h = 48, 40
    v = view(w, h, k=12)
    g = np.random.default_rng(5).normal(size=(h, w, 4)).astype(np.float32)
    s = Scene(ctx, rec, 0.01)
    ctx.set_tune(s, v.uniforms, w, h, kbuf=64, leaf_batch=8)
    got, info = ctx.backward(s, v.uniforms, w, h, g, mode=mode)
    ctx._lib.gt_autotune_reset(ctx._h)
    assert info["used_mode"] == mode
    _check(got, _ref_grad(rec, 0.01, v.uniforms, w, h, g))


def test_differentiable_config_subset(ctx):
    """The differentiable configuration on a 2,048-Gaussian subset of its
    200k scene (200x200 view of the same camera, k = 8): the full gradient
    of the L2 loss against the perturbed-scene target, CUDA against the FP64
    adjoint on the same entry lists."""
    from gtrace import synth
    from gtrace.uniforms import unpack_uniforms
    raw, amin, v0 = synth.clusters_200k_config()
    sub = {k: np.asarray(a)[:2048] for k, a in raw.items()}
    rec = synth.pack(sub).gaussiansBuffer
    tgt_rec = synth.pack(synth.perturb(sub, synth.SEED_BASE + 33)).gaussiansBuffer
    w, h = 200, 200
    v = synth.view(w, h, (0.0, 0.0, 12.0), k=8, alpha_min=amin)
    s, t = Scene(ctx, rec, amin), Scene(ctx, tgt_rec, amin)
    img = ctx.render(s, v.uniforms, w, h)
    target = ctx.render(t, v.uniforms, w, h)
    g = 2.0 * (img - target)
    g[..., 3] = 0.0
    got, info = ctx.backward(s, v.uniforms, w, h, g.astype(np.float32))
    _, hits = oracle.Scene(rec, amin, "f32").render(v.uniforms, w, h, max_entries=256)
    ref = oracle.backward_lists(oracle.Scene(rec, amin, "f64"), v.uniforms, w, h, hits,
                                g.reshape(-1, 4).astype(np.float64),
                                alpha_min=unpack_uniforms(v.uniforms)["alpha_min"])
    _check(got, ref)
    assert np.abs(got).sum() > 0


@pytest.mark.parametrize("budget", [0, 1])
def test_batch_of_two_scenes_matches_fp64_oracle(ctx, budget):
    """Interleaved views of two scenes in one gt_backward_batch: each scene's
    gradient is the sum of the FP64 adjoints of its views.  budget = 1 byte
    puts every view in an adjoint launch of its own (the per-view colour sums
    then never fit together), which must give the same sums."""
    pa, pb = small_scene(n=1200, seed=45), small_scene(n=900, seed=46)
    sa, sb = Scene(ctx, pa.gaussiansBuffer, 0.01), Scene(ctx, pb.gaussiansBuffer, 0.01)
    rng = np.random.default_rng(7)
    specs = [(sa, pa, view(32, 24, k=6)), (sb, pb, view(28, 20, pos=(1.0, 0.5, 3.6), k=4)),
             (sa, pa, view(20, 36, pos=(-1.5, 0.5, 3.5), k=8))]
    views, refs = [], {sa: 0.0, sb: 0.0}
    for sc, pg, v in specs:
        g = rng.normal(size=(v.height, v.width, 4)).astype(np.float32)
        views.append((sc, v.uniforms, v.width, v.height, g))
        refs[sc] = refs[sc] + _ref_grad(pg.gaussiansBuffer, 0.01, v.uniforms, v.width, v.height, g)
    got, info = ctx.backward_batch(views, mode=1, mem_budget=budget)
    assert info["used_mode"] == 1
    for sc in (sa, sb):
        _check(got[sc], refs[sc])
