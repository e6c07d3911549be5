"""CUDA gradients at the sizes of the differentiable configurations.

1. The 200k-Gaussian, 800x800, k = 8 configuration: the CUDA adjoint of the
   L2 loss against the perturbed-scene target, checked against central
   finite differences (h = 1e-4, and h/2 for a Richardson extrapolation) of
   the FP64 oracle render on 256 random (particle, parameter) pairs.  Each
   perturbed render covers only the pixels
   whose rays can reach the particle's proxy (its circumscribed sphere,
   sized for the perturbed parameter), which holds every pixel the
   parameter can change; the oracle scene is rebuilt for each.  Pixels
   whose perturbed or float hit sequences differ (entry lists, which entries
   pass alpha_min, round counts) straddle a discontinuity of the
   piecewise-smooth image and are left out of both sides of the comparison;
   the test reports how many and bounds the samples left without pixels.
   Relative error <= 1e-3 is required of 98 % of the samples and, for all,
   |fd - cuda| <= 1e-3 max(|fd|, |cuda|) + 1e-4 sum|pixel terms|: a
   gradient that is a small residue of per-pixel terms of both signs carries
   the float32 summation error of those terms.
2. The batched forward + backward configuration: views of the 1M-Gaussian
   scene rendered in one checkpointing gt_render_batch and differentiated by
   one gt_backward_batch that sums all views, against the FP64 oracle
   adjoint summed over the same views.  dL/dpixel is the L2 loss gradient
   on a stratified pixel subset and zero elsewhere, which keeps the FP64
   side to a few thousand rays a view.

The function differentiated is the reference's tracePath
(src/GS_shader.ts:192-273); the reference itself has no backward pass."""
import concurrent.futures as cf
import ctypes as C
import math
import os
import threading

import numpy as np
import pytest

from oracle import oracle
from gtrace import _lib as L
from gtrace import synth
from gtrace.tracer import Scene, _uniforms
from gtrace.uniforms import unpack_uniforms

pytestmark = pytest.mark.gpu

# record column of each of the 59 gradient rows: position, scale, rotation
# (w, x, y, z), opacity, 16 x 3 SH coefficients
REC_INDEX = [0, 1, 2, 4, 5, 6, 8, 9, 10, 11, 12] + [16 + 4 * c + ch for c in range(16) for ch in range(3)]
H_STEP = 1e-4


def ray_dirs(uniforms, w, h):
    """Camera origin and the w*h primary ray directions in double (the
    ray generation of src/GS_shader.ts:275-285 without its float rounding)."""
    f = np.frombuffer(bytes(uniforms), np.float32).astype(np.float64)
    tw, asp = f[:16], f[16:18]
    cx, cy, cz, o = -tw[0:3], tw[4:7], -tw[8:11], tw[12:15]
    ax = ((np.arange(w) + 0.5) / w * 2.0 - 1.0) * asp[0]
    ay = ((np.arange(h) + 0.5) / h * 2.0 - 1.0) * asp[1]
    v = ax[None, :, None] * cx + ay[:, None, None] * cy + cz
    d = v / np.linalg.norm(v, axis=-1, keepdims=True)
    return o, d.reshape(-1, 3)


def footprint(o, dirs, rec_row, amin, h):
    """Pixels whose rays pass within the circumscribed sphere of the
    particle's proxy (circumradius 1.2584 of the unit-inradius icosahedron,
    scaled by sqrt(2 ln(opacity / alpha_min)) and the largest scale), for
    parameters up to h larger than the record's."""
    mu = rec_row[0:3].astype(np.float64)
    op = float(rec_row[12]) + h
    if not op > amin:
        return np.zeros(0, np.int64)
    r = 1.3 * math.sqrt(2.0 * math.log(op / amin)) * (float(np.abs(rec_row[4:7]).max()) + h) + h + 1e-4
    m = mu - o
    t = dirs @ m
    d2 = float(m @ m) - t * t
    return np.nonzero((d2 <= r * r) & (t > -r))[0]


def signature(hits, amin, n):
    out = []
    for q in range(n):
        m = int(hits["count"][q])
        out.append((tuple(hits["pidx"][q, :m]), tuple(hits["alpha"][q, :m] > np.float32(amin)),
                    int(hits["rounds"][q])))
    return out


def fd_samples(rec, amin, u, w, h, g, picks, workers=None):
    """Central differences of sum over S of g * rgba for each (particle, row)
    pick, with steps h and h/2, and their Richardson extrapolation
    (4 D(h/2) - D(h)) / 3, S being the pixels of the particle's footprint
    whose hit sequence (entries, which pass alpha_min, rounds) is the same in
    the four FP64 renders and in the float render (the one the CUDA kernels
    reproduce and differentiate).  Pixels outside S sit on a discontinuity of
    the piecewise-smooth image (or order two hits differently in float and
    double).  The extrapolation matters for the smallest Gaussians: with
    scales of e^-5 and rays at a few standard deviations, the h^2 term of a
    plain central difference alone reaches 1e-3.  g: (w*h, 4) float64
    weights.  Returns (particle, row, D(h), extrapolated, S) per pick with a
    non-empty S, and the numbers of excluded pixels and of picks left
    without pixels."""
    o, dirs = ray_dirs(u, w, h)
    base = oracle.Scene(rec, amin, "f32")
    max_e = 1024
    workers = workers or min(16, os.cpu_count() or 1)
    local = threading.local()

    def one(pick):
        p, i = pick
        col = REC_INDEX[i]
        pix = footprint(o, dirs, rec[p], amin, H_STEP).astype(np.uint32)
        if len(pix) == 0:
            return None
        if not hasattr(local, "rec"):
            local.rec = rec.copy()
        r = local.rec
        x = rec[p, col]
        _, h0 = base.render(u, w, h, pixels=pix, threads=1, max_entries=max_e)
        res = []
        for step in (H_STEP, -H_STEP, 0.5 * H_STEP, -0.5 * H_STEP):
            r[p, col] = np.float32(x + step)
            s64 = oracle.Scene(r, amin, "f64")
            img, hh = s64.render(u, w, h, pixels=pix, threads=1, max_entries=max_e)
            res.append((float(r[p, col]), img, signature(hh, amin, len(pix)), int(hh["count"].max())))
            del s64
        r[p, col] = x
        if max([m for *_, m in res] + [int(h0["count"].max())]) > max_e:
            return None
        sig0 = signature(h0, amin, len(pix))
        keep = np.array([all(rr[2][q] == sig0[q] for rr in res) for q in range(len(pix))], bool)
        gk = g[pix[keep]]
        per_px = ((res[0][1] - res[1][1])[keep] * gk).sum(axis=1) / (res[0][0] - res[1][0])
        d1 = float(per_px.sum())
        d2 = float(((res[2][1] - res[3][1])[keep] * gk).sum()) / (res[2][0] - res[3][0])
        return (p, i, d1, (4.0 * d2 - d1) / 3.0, pix[keep], int((~keep).sum()), float(np.abs(per_px).sum()))

    out, excluded, empty = [], 0, 0
    with cf.ThreadPoolExecutor(workers) as ex:
        for res in ex.map(one, picks):
            if res is None:
                continue
            p, i, d1, dx, keep, nx, asum = res
            excluded += nx
            if len(keep) == 0:
                empty += 1
            else:
                out.append((p, i, d1, dx, keep, asum))
    return out, excluded, empty


def test_fd_differentiable_config(ctx):
    raw, amin, v = synth.clusters_200k_config()
    rec = np.ascontiguousarray(synth.pack(raw).gaussiansBuffer, dtype=np.float32)
    tgt = synth.pack(synth.perturb(raw, synth.SEED_BASE + 33)).gaussiansBuffer
    w, h = v.width, v.height
    s, t = Scene(ctx, rec, amin), Scene(ctx, tgt, amin)
    try:
        img = ctx.render(s, v.uniforms, w, h, checkpoint=True)
        target = ctx.render(t, v.uniforms, w, h)
        g = 2.0 * (img - target)
        g[..., 3] = 0.0
        g = g.reshape(-1, 4).astype(np.float32)
        grad, _ = ctx.backward(s, v.uniforms, w, h, g, reuse_checkpoint=True)
        contributing = np.nonzero(np.abs(grad[10]) > 0)[0]
        assert len(contributing) > 10000
        rng = np.random.default_rng(synth.SEED_BASE + 303)
        picks = [(int(p), int(i)) for p, i in zip(rng.choice(contributing, 256, replace=False),
                                                  rng.integers(0, 59, 256))]
        samples, excluded, empty = fd_samples(rec, amin, v.uniforms, w, h, g.astype(np.float64), picks)
        # the CUDA gradient of the same sum: dL/dpixel on S only, the
        # checkpoint of the render above reused
        gm = np.zeros_like(g)
        row_max = np.abs(grad).max(axis=1)
        err_c, err_x, cond_ok, worst = [], [], [], []
        for p, i, d1, dx, keep, asum in samples:
            gm[keep] = g[keep]
            an = float(ctx.backward(s, v.uniforms, w, h, gm, reuse_checkpoint=True)[0][i, p])
            gm[keep] = 0.0
            floor = 1e-4 * row_max[i]
            err_c.append(abs(d1 - an) / max(abs(d1), abs(an), floor))
            err_x.append(abs(dx - an) / max(abs(dx), abs(an), floor))
            # a gradient that is a small residue of per-pixel terms of both
            # signs carries the float32 summation error of those terms
            cond_ok.append(abs(dx - an) <= 1e-3 * max(abs(dx), abs(an)) + 1e-4 * asum)
            worst.append((err_x[-1], p, i, dx, an, asum))
    finally:
        s.close()
        t.close()
    err_c, err_x = np.array(err_c), np.array(err_x)
    n_rel = int((err_x <= 1e-3).sum())
    print(f"FD at 200k/800x800: {len(samples)} of {len(picks)} samples, {excluded} footprint pixels excluded, "
          f"{empty} samples without pixels; relative error, central h = 1e-4: max {err_c.max():.2e}, median "
          f"{np.median(err_c):.2e}; extrapolated from h and h/2: max {err_x.max():.2e}, median {np.median(err_x):.2e}; "
          f"{n_rel} samples within 1e-3")
    assert len(samples) >= 0.9 * len(picks), (len(samples), empty)
    assert all(cond_ok), sorted(worst, reverse=True)[:5]
    assert n_rel >= 0.98 * len(samples), sorted(worst, reverse=True)[:5]
    assert np.median(err_c) <= 1e-4


def _check_rows(got, ref, rel=1e-3):
    """Per parameter row: 2-norm relative error <= rel, and 99.9 % of the
    elements within rel |ref| + 1e-4 max|row|."""
    for i in range(59):
        r = ref[i]
        scale = np.abs(r).max()
        if scale == 0:
            assert np.abs(got[i]).max() <= 1e-6, i
            continue
        assert np.linalg.norm(got[i] - r) <= rel * np.linalg.norm(r) + 1e-6 * scale, i
        assert (np.abs(got[i] - r) <= rel * np.abs(r) + 1e-4 * scale).mean() >= 0.999, i


def test_batched_adjoint_matches_fp64_oracle(ctx):
    pg, amin, _ = synth.clusters_1m_config()
    rec = pg.gaussiansBuffer
    target_raw = synth.perturb(synth.raw_clusters(1_000_000, synth.SEED_BASE + 1), synth.SEED_BASE + 44)
    views = synth.batched_fwd_bwd_views()[:6]
    lib = ctx._lib
    s = Scene(ctx, rec, amin)
    t = Scene(ctx, synth.pack(target_raw).gaussiansBuffer, amin)
    stride = 12
    try:
        imgs = [np.zeros((v.height, v.width, 4), np.float32) for v in views]
        items = (L.BatchItem * len(views))()
        for i, v in enumerate(views):
            items[i].scene = s.handle
            items[i].u = _uniforms(v.uniforms)
            items[i].w, items[i].h = v.width, v.height
            items[i].out_rgba = imgs[i].ctypes.data
        ctx.check(lib.gt_render_batch(ctx.handle, items, len(views), L.GT_FLAG_CHECKPOINT, None))
        gs, pixsets = [], []
        for i, v in enumerate(views):
            tgt = ctx.render(t, v.uniforms, v.width, v.height)
            mask = np.zeros((v.height, v.width), bool)
            mask[(i % stride)::stride, (i * 5 % stride)::stride] = True
            gi = np.where(mask[..., None], 2.0 * (imgs[i] - tgt), 0.0).astype(np.float32)
            gi[..., 3] = 0.0
            gs.append(gi)
            pixsets.append(np.nonzero(mask.reshape(-1))[0].astype(np.uint32))
            items[i].out_rgba = None
            items[i].dL_drgba = gi.ctypes.data
        got = np.zeros((59, s.n), np.float32)
        sc = (C.c_void_p * 1)(s.handle.value)
        op = (C.c_void_p * 1)(got.ctypes.data)
        opts = L.BwdOpts(0, 0, 0, 0, 0, 0.0, 0.0)
        ctx.check(lib.gt_backward_batch(ctx.handle, items, len(views), sc, op, 1, L.GT_FLAG_CHECKPOINT,
                                        C.byref(opts), None))
        assert opts.fwd_ms == 0.0  # the render's checkpoint was used
    finally:
        s.close()
        t.close()
    o32 = oracle.Scene(rec, amin, "f32")
    o64 = oracle.Scene(rec, amin, "f64")
    ref = np.zeros((59, pg.gaussiansBuffer.shape[0]), np.float64)
    for v, img, gi, pix in zip(views, imgs, gs, pixsets):
        img_ref, hits = o32.render(v.uniforms, v.width, v.height, pixels=pix, max_entries=1024)
        # the batch rendered these pixels exactly as the oracle does
        got_px = img.reshape(-1, 4)[pix]
        np.testing.assert_array_equal(got_px.view(np.uint32), img_ref.view(np.uint32))
        ref += oracle.backward_lists(o64, v.uniforms, v.width, v.height, hits,
                                     gi.reshape(-1, 4)[pix].astype(np.float64), pixels=pix,
                                     alpha_min=unpack_uniforms(v.uniforms)["alpha_min"])
    assert np.abs(ref[10]).max() > 0
    _check_rows(got, ref)
