"""CPU tests of the oracle: its elementary functions, known answers derived
from the reference's formulas, and agreement of its two render algorithms."""
import math

import numpy as np
import pytest

from conftest import small_scene, view
from oracle import oracle
from gtrace import synth
from gtrace.uniforms import look_at, pack_uniforms, with_fields


def ulp_diff(a, b):
    a = np.asarray(a, np.float32).view(np.int32).astype(np.int64)
    b = np.asarray(b, np.float32).view(np.int32).astype(np.int64)
    return np.abs(a - b)


def test_expf_within_two_ulp():
    xs = np.concatenate([np.linspace(-87.0, 88.0, 20001, dtype=np.float32),
                         np.float32([-1e-7, 0.0, 1e-7, -0.5, -20.25])])
    got = np.array([oracle.expf(float(x)) for x in xs], np.float32)
    ref = np.exp(xs.astype(np.float64)).astype(np.float32)
    assert ulp_diff(got, ref).max() <= 2
    assert oracle.expf(-87.5) == 0.0
    assert math.isinf(oracle.expf(89.0))


def test_log_matches_math_log():
    for x in [1e-300, 0.01, 0.5, 0.7071, 1.0, 1.0000001, 2.0, 99.0, 1e300]:
        assert abs(oracle.log(x) - math.log(x)) <= 4e-16 * max(1.0, abs(math.log(x)))


def _isotropic_particle(pos=(0, 0, 0), scale=0.05, opacity=0.8, dc=(0.3, -0.2, 0.1), rest=0.0):
    rec = np.zeros((1, 80), np.float32)
    rec[0, 0:3] = pos
    rec[0, 4:7] = scale
    rec[0, 8:12] = (1.0, 0.0, 0.0, 0.0)
    rec[0, 12] = opacity
    rec[0, 16:19] = dc
    for k in range(1, 16):
        rec[0, 16 + 4 * k:19 + 4 * k] = rest
    return rec


def _sh_reference(sh, d, deg=3):
    """shToRadiance restated from src/GS_shader.ts:138-177 in float64."""
    C0, C1 = 0.28209479177387814, 0.4886025119029199
    C2 = [1.0925484305920792, -1.0925484305920792, 0.31539156525252005, -1.0925484305920792, 0.5462742152960396]
    C3 = [-0.5900435899266435, 2.890611442640554, -0.4570457994644658, 0.3731763325901154, -0.4570457994644658,
          1.445305721320277, -0.5900435899266435]
    x, y, z = d
    L = 0.5 + C0 * sh[0]
    if deg >= 1:
        L = L + C1 * (-y * sh[1] + z * sh[2] - x * sh[3])
    if deg >= 2:
        xx, yy, zz = x * x, y * y, z * z
        L = L + (C2[0] * x * y * sh[4] + C2[1] * y * z * sh[5] + C2[2] * (2 * zz - xx - yy) * sh[6]
                 + C2[3] * x * z * sh[7] + C2[4] * (xx - yy) * sh[8])
    if deg >= 3:
        L = L + (C3[0] * y * (3 * xx - yy) * sh[9] + C3[1] * x * y * z * sh[10] + C3[2] * y * (4 * zz - xx - yy) * sh[11]
                 + C3[3] * z * (2 * zz - 3 * xx - 3 * yy) * sh[12] + C3[4] * x * (4 * zz - xx - yy) * sh[13]
                 + C3[5] * z * (xx - yy) * sh[14] + C3[6] * x * (xx - 3 * yy) * sh[15])
    return L


def _ray(px, py, w, h, tanh, origin=(0.0, 0.0, 4.0)):
    nx = ((px + 0.5) / w) * 2 - 1
    ny = ((py + 0.5) / h) * 2 - 1
    d = np.array([-nx * tanh, ny * tanh, -1.0])  # camX = -right = (-1,0,0), camZ = -back
    return np.asarray(origin), d / np.linalg.norm(d)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_single_gaussian_known_answer(precision):
    """One isotropic Gaussian in front of the camera: alpha = o exp(-r^2/s^2)
    at the ray's closest approach r (no 1/2 factor, src/GS_shader.ts:135) and
    colour max(0, SH(normalize(mu - origin))) (:264)."""
    mu = np.array([0.0013, 0.0007, 0.0])
    sh = np.zeros((16, 3))
    sh[0] = (0.3, -0.2, 0.1)
    sh[1:] = 0.02
    rec = _isotropic_particle(pos=mu, rest=0.02)
    s = oracle.Scene(rec, 0.01, precision)
    assert s.n_kept == 1
    w = h = 33
    u = pack_uniforms(look_at((0.0, 0.0, 4.0)), w, h, T_min=0.01, alpha_min=0.01, k=4)
    img, hits = s.render(u, w, h, algo=0, max_entries=4)
    img = img.reshape(h, w, 4)
    tanh = float(np.frombuffer(u.tobytes(), np.float32)[16])
    dirc = mu - np.array([0.0, 0.0, 4.0])
    col = np.maximum(0.0, _sh_reference(sh, dirc / np.linalg.norm(dirc)))
    s_proxy = math.sqrt(2 * math.log(0.8 / 0.01)) * 0.05  # proxy scale; inradius 1, circumradius 1.2584
    inside = outside = 0
    for py in range(h):
        for px in range(w):
            o, d = _ray(px, py, w, h, tanh)
            r2 = np.sum(np.cross(mu - o, d) ** 2)
            q = py * w + px
            if r2 < (0.999 * s_proxy) ** 2:  # through the inscribed sphere: one front-face hit
                alpha = 0.8 * math.exp(-r2 / 0.05 ** 2)
                assert hits["count"][q] == 1
                np.testing.assert_allclose(hits["alpha"][q, 0], alpha, rtol=2e-5, atol=1e-7)
                expect = alpha * col if alpha > 0.01 else np.zeros(3)
                np.testing.assert_allclose(img[py, px, :3], expect, rtol=5e-5, atol=1e-6)
                inside += 1
            elif r2 > (1.2584 * 1.001 * s_proxy) ** 2:  # misses the circumscribed sphere
                assert hits["count"][q] == 0
                assert (img[py, px, :3] == 0).all()
                outside += 1
    assert inside >= 5 and outside > 900
    assert (img[..., 3] == 1.0).all()


def test_shared_edge_hit_is_composited_twice():
    """A ray through a shared edge of two front faces reports the particle
    twice: the barycentric test is inclusive and nothing removes duplicates
    (webrtx/src/glsl/intersect.glsl:91, src/GS_shader.ts:250-269).  The ray
    along -z through the centre crosses the edge between vertices 4 and 5."""
    rec = _isotropic_particle()
    s = oracle.Scene(rec, 0.01, "f64")
    w = h = 33
    u = pack_uniforms(look_at((0.0, 0.0, 4.0)), w, h, T_min=0.01, alpha_min=0.01, k=4)
    img, hits = s.render(u, w, h, pixels=[16 * 33 + 16], algo=0, max_entries=4)
    assert hits["count"][0] == 2
    assert hits["pidx"][0, 0] == hits["pidx"][0, 1] == 0
    sh = np.zeros((16, 3))
    sh[0] = (0.3, -0.2, 0.1)
    c = np.maximum(0.0, _sh_reference(sh, (0.0, 0.0, -1.0)))
    np.testing.assert_allclose(img[0, :3], 0.8 * c * (2 - 0.8), rtol=1e-6)


def test_proxy_cut_and_scale():
    """Proxies exist only for opacity > alpha_min (strict), scaled by
    sqrt(2 ln(o/alpha_min)) (src/main.ts:79-87)."""
    rec = np.concatenate([_isotropic_particle(opacity=0.5), _isotropic_particle(pos=(1, 0, 0), opacity=0.01),
                          _isotropic_particle(pos=(2, 0, 0), opacity=0.0099)])
    s = oracle.Scene(rec, 0.01, "f64")
    assert s.n_kept == 1
    p, o2w, w2o = s.proxy(0)
    assert p == 0
    s_expect = math.sqrt(2 * math.log(0.5 / 0.01))
    np.testing.assert_allclose(o2w[[0, 4, 8]], 0.05 * s_expect, rtol=1e-6)
    m = np.eye(4)
    m[:3, :3] = o2w[:9].reshape(3, 3).T
    m[:3, 3] = o2w[9:]
    wi = np.eye(4)
    wi[:3, :3] = w2o[:9].reshape(3, 3).T
    wi[:3, 3] = w2o[9:]
    np.testing.assert_allclose(m @ wi, np.eye(4), atol=1e-5)


def test_icosahedron_inradius_one():
    """The proxy of a unit-scale particle with s = 1 has its faces at
    distance 1 from the centre (src/main.ts:12-14)."""
    a = 0.01
    o = a * math.exp(0.5)  # s = sqrt(2 ln(o/a)) = 1
    rec = _isotropic_particle(scale=1.0, opacity=o)
    s = oracle.Scene(rec, a, "f64")
    w = h = 16
    u = pack_uniforms(look_at((0.0, 0.0, 5.0)), w, h, T_min=0.01, alpha_min=0.5, k=4)
    _, hits = s.render(u, w, h, pixels=[8 * 16 + 8], algo=0, max_entries=4)
    # the central ray enters the proxy between distance 1 (inradius) and the circumradius
    t_entry = hits["t"][0, 0]
    assert 5.0 - 1.2584 - 1e-6 <= t_entry <= 5.0 - 1.0 + 1e-6


@pytest.mark.parametrize("k", [1, 3, 6])
def test_algorithms_agree(k):
    """The sort-all-hits checker and the restated reference traversal (per
    round k-buffer with the commit rule) produce the same hit sequences."""
    pg = small_scene(n=1500, seed=11)
    s = oracle.Scene(pg.gaussiansBuffer, 0.01)
    v = view(48, 40, k=k)
    a, ha = s.render(v.uniforms, 48, 40, algo=0, max_entries=64)
    b, hb = s.render(v.uniforms, 48, 40, algo=1, max_entries=64)
    np.testing.assert_array_equal(ha["count"], hb["count"])
    np.testing.assert_array_equal(ha["rounds"], hb["rounds"])
    np.testing.assert_array_equal(ha["pidx"], hb["pidx"])
    np.testing.assert_array_equal(ha["t"], hb["t"])
    np.testing.assert_array_equal(a, b)


def test_early_stop_and_transmittance_cut():
    pg = small_scene(n=1500, seed=3)
    s = oracle.Scene(pg.gaussiansBuffer, 0.01)
    v = view(24, 24, k=2)
    _, full = s.render(v.uniforms, 24, 24, algo=0, max_entries=128)
    _, one = s.render(with_fields(v.uniforms, early_stop=1), 24, 24, algo=0, max_entries=128)
    assert one["rounds"].max() <= 1
    assert (one["count"] <= 2).all()
    assert full["rounds"].max() > 1
    # T_min = 1: no round starts
    _, none = s.render(with_fields(v.uniforms, T_min=1.0), 24, 24, algo=0, max_entries=4)
    assert none["rounds"].max() == 0


def test_empty_scene_renders_black():
    rec = np.zeros((0, 80), np.float32)
    s = oracle.Scene(rec, 0.01)
    v = view(16, 8)
    img, h = s.render(v.uniforms, 16, 8, algo=0, max_entries=2)
    assert (img[:, :3] == 0).all() and (img[:, 3] == 1).all()


def test_ply_ingest_matches_host_mirror():
    """The oracle's C restatement of GS_ply and the numpy mirror agree to 1 ulp
    (both activate in double; exp implementations may differ in the last bit)."""
    raw = synth.raw_small(n=300, seed=5)
    from gtrace.ply import write_ply, PackedGaussians
    data = write_ply(raw)
    a = oracle.ply_to_aos(data)
    b = PackedGaussians(data).gaussiansBuffer
    assert a.shape == b.shape == (300, 80)
    assert ulp_diff(a, b).max() <= 1


def test_fp64_render_close_to_fp32():
    pg = small_scene(n=1000, seed=21)
    s32 = oracle.Scene(pg.gaussiansBuffer, 0.01, "f32")
    s64 = oracle.Scene(pg.gaussiansBuffer, 0.01, "f64")
    v = view(32, 32)
    a, _ = s32.render(v.uniforms, 32, 32)
    b, _ = s64.render(v.uniforms, 32, 32)
    rmse = float(np.sqrt(np.mean((a[:, :3] - b[:, :3]) ** 2)))
    assert rmse < 1e-3
