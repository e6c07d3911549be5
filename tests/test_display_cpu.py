"""Oracle restatements of the display-side rows: the anti-aliasing jitter
(getNewSeed / rng, src/GS_shader.ts:6-31), the progressive blend
(src/GS_shader.ts:300-308) and the tone map (src/toneMapper.ts:15-24)."""
import numpy as np
import pytest

from conftest import small_scene, view
from oracle import oracle

M32 = 0xFFFFFFFF


def tea(p1, p2, rounds=8):
    """getNewSeed written out in Python integers (src/GS_shader.ts:9-23)."""
    s0, v0, v1 = 0, p1, p2
    for _ in range(rounds):
        s0 = (s0 + 0x9E3779B9) & M32
        v0 = (v0 + ((((v1 << 4) & M32) + 0xA341316C) & M32 ^ ((v1 + s0) & M32) ^ (((v1 >> 5) + 0xC8013EA4) & M32))) & M32
        v1 = (v1 + ((((v0 << 4) & M32) + 0xAD90777D) & M32 ^ ((v0 + s0) & M32) ^ (((v0 >> 5) + 0x7E95761E) & M32))) & M32
    return v0


def test_seed_and_rng_known_answers():
    rs = np.random.Generator(np.random.PCG64(3))
    for p1, p2 in [(0, 0), (1, 0), (0, 1), (M32, M32)] + [tuple(int(x) for x in rs.integers(0, 2**32, 2))
                                                            for _ in range(50)]:
        assert oracle.new_seed(p1, p2, 8) == tea(p1, p2)
    seed = 12345
    for _ in range(20):
        v, s2 = oracle.rng(seed)
        seed_py = (1664525 * seed + 1013904223) & M32
        assert s2 == seed_py and v == (seed_py & 0xFFFFFF) / 16777216.0 and 0.0 <= v < 1.0
        seed = s2


def test_accumulate_blend_is_the_reference_mix():
    pg = small_scene(n=1500, seed=21)
    s = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32")
    w, h = 24, 16
    v0 = view(w, h, k=6)
    acc = np.zeros((w * h, 4), np.float32)
    s.render_accum(v0.uniforms, w, h, acc)
    centre, _ = s.render(v0.uniforms, w, h)
    assert not np.array_equal(acc, centre)           # jittered, not the pixel centre
    # nearby samples: the image mean moves by a few percent at most
    assert abs(acc[:, :3].mean() - centre[:, :3].mean()) < 0.1 * centre[:, :3].mean()
    for f in (1, 2, 7):
        vf = view(w, h, k=6, accumulated_frames=f)
        old = acc.copy()
        s.render_accum(vf.uniforms, w, h, acc)
        z = np.zeros_like(acc)
        s.render_accum(vf.uniforms, w, h, z)          # = new * a, rounded once
        a = np.float32(1.0) / (np.float32(f) + np.float32(1.0))
        want = old * (np.float32(1.0) - a) + z
        want[:, 3] = 1.0
        assert np.array_equal(acc.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("mode", [0, 1, 2])
def test_tonemap_restatement(mode):
    rs = np.random.Generator(np.random.PCG64(5))
    hdr = np.concatenate([rs.uniform(-0.5, 3.0, (500, 4)),
                          np.array([[np.nan, np.inf, -np.inf, 0.0], [0.5 / 255, 1.5 / 255, 1.0, 254.5 / 255]])])
    hdr = hdr.astype(np.float32)
    out = oracle.tonemap(hdr, mode, 1.66)
    assert (out[:, 3] == 255).all()
    with np.errstate(all="ignore"):
        x = hdr[:, :3].astype(np.float64)
        if mode >= 1:
            x = 1.0 - np.exp(-1.66 * x)
        if mode == 2:
            x = np.where(x > 0, np.power(np.maximum(x, 0), 1 / 2.2), x)
        want = np.where(np.isnan(x), 0, np.rint(np.clip(x, 0, 1) * 255))
    assert np.abs(out[:, :3].astype(int) - want).max() <= 1
    assert out[-2, 0] == 0  # NaN -> 0
    if mode == 0:
        assert out[-2, 1] == 255 and out[-2, 2] == 0 and out[-1, 2] == 255
        assert out[-1, 0] == 0 and out[-1, 1] == 2 and out[-1, 3] == 255  # ties to even
