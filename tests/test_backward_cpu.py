"""CPU check of the adjoint formulas: the oracle's FP64 analytic gradient
against central finite differences of its FP64 render (h = 1e-4) on 256
randomly chosen (particle, parameter) pairs.

Samples whose +h and -h renders differ in any hit sequence or in which
entries pass alpha_min straddle a discontinuity of the piecewise-smooth
image and are rejected; the test reports and bounds how many."""
import numpy as np
import pytest

from conftest import small_scene, view
from oracle import oracle

PARAM_NAMES = ["px", "py", "pz", "s0", "s1", "s2", "qw", "qx", "qy", "qz", "opacity"] + \
              [f"sh{c}_{ch}" for c in range(16) for ch in "rgb"]
REC_INDEX = [0, 1, 2, 4, 5, 6, 8, 9, 10, 11, 12] + [16 + 4 * c + ch for c in range(16) for ch in range(3)]


def _render(rec, amin, u, w, h):
    s = oracle.Scene(rec, amin, "f64")
    img, hits = s.render(u, w, h, algo=0, max_entries=128)
    return img, hits


def _signature(hits, alpha_min):
    n = hits["count"]
    sig = []
    for q in range(len(n)):
        m = min(int(n[q]), hits["pidx"].shape[1])
        sig.append((tuple(hits["pidx"][q, :m]), tuple(hits["alpha"][q, :m] > alpha_min), int(hits["rounds"][q])))
    return sig


@pytest.mark.parametrize("seed", [3, 4])
def test_fp64_adjoint_matches_central_differences(seed):
    pg = small_scene(n=300, seed=seed)
    rec = pg.gaussiansBuffer.astype(np.float32).copy()
    w, h = 20, 16
    v = view(w, h, k=4, alpha_min=0.01, T_min=0.01)
    u = v.uniforms
    amin = 0.01
    rng = np.random.default_rng(seed)
    wgt = rng.normal(size=(w * h, 4))
    wgt[:, 3] = 0.0
    base_img, base_hits = _render(rec, amin, u, w, h)
    s64 = oracle.Scene(rec, amin, "f64")
    grad = s64.backward(u, w, h, wgt)  # (59, n)
    # particles that contribute to the image
    contributing = sorted({int(p) for q in range(w * h) for p, a in
                           zip(base_hits["pidx"][q, :min(base_hits["count"][q], 128)],
                               base_hits["alpha"][q, :min(base_hits["count"][q], 128)]) if a > 0.01})
    assert len(contributing) > 10
    # 128 (particle, parameter) pairs per seed: 256 over both seeds
    pairs = [(int(p), int(i)) for p in contributing for i in range(59)]
    picks = [pairs[q] for q in rng.choice(len(pairs), size=min(128, len(pairs)), replace=False)]
    hstep = 1e-4
    checked = rejected = 0
    errs = []
    for p, i in picks:
        col = REC_INDEX[i]
        rp, rm = rec.copy(), rec.copy()
        rp[p, col] = np.float32(rec[p, col] + hstep)
        rm[p, col] = np.float32(rec[p, col] - hstep)
        ip, hp = _render(rp, amin, u, w, h)
        im, hm = _render(rm, amin, u, w, h)
        if _signature(hp, 0.01) != _signature(hm, 0.01):
            rejected += 1
            continue
        fd = float(((ip - im) * wgt).sum()) / float(np.float64(rp[p, col]) - np.float64(rm[p, col]))
        an = float(grad[i, p])
        scale = max(abs(fd), abs(an), 1e-3 * np.abs(grad).max())
        errs.append(abs(fd - an) / scale)
        checked += 1
    assert checked >= 0.7 * len(picks), (checked, rejected)
    assert max(errs) <= 1e-3, (max(errs), PARAM_NAMES)
