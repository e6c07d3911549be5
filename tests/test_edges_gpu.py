"""Adversarial geometry for the exact prefilters of the CUDA kernels.

Both forward kernels put exact filters in front of the reference's triangle
test (webrtx/src/glsl/intersect.glsl:73-92) and facing rule
(webrtx/src/glsl/trace.glsl:154-164): a padded slab test on the world boxes,
the proxy's bounding sphere, an object-space facing test with a tolerance
tau, and a t-range test.  Each is meant to skip only work whose outcome is
known; if a margin were too tight a hit would vanish silently.  The cases
here aim rays at those margins:

* a ray through a shared edge of two front faces (the particle is composited
  twice: inclusive barycentric test, no de-duplication, src/GS_shader.ts:250-269);
* rays grazing proxy silhouettes and the box-touching vertices;
* rays within a few tau of a face's plane that still cross the face;
* needle and disc proxies (scale ratio 1e3 and more);
* tiny proxies about 1e3 from the origin.

Every image is compared bit for bit with the oracle for both kernels (a warp
per ray: block_threads 128; a warp per 8x4 tile: block_threads 32), and the
warp-per-ray kernel's hit sequences, t and alpha bits (gt_render_hits) with
the oracle's."""
import itertools
import math

import numpy as np
import pytest

from oracle import oracle
from gtrace.tracer import Scene
from gtrace.uniforms import pack_uniforms

pytestmark = pytest.mark.gpu

KERNELS = (("warp per ray", 128, 64), ("warp per 8x4 tile", 32, 32))


def _records(pos, scale, rot, opacity, seed=0):
    n = len(pos)
    rng = np.random.default_rng(seed)
    rec = np.zeros((n, 80), np.float32)
    rec[:, 0:3] = pos
    rec[:, 4:7] = scale
    rec[:, 8:12] = rot
    rec[:, 12] = opacity
    rec[:, 16:19] = rng.normal(0.0, 0.5, size=(n, 3))
    for c in range(1, 16):
        rec[:, 16 + 4 * c:19 + 4 * c] = rng.normal(0.0, 0.05, size=(n, 3))
    return rec


def _unit_quats(rng, n):
    q = rng.normal(size=(n, 4))
    return q / np.linalg.norm(q, axis=1, keepdims=True)


def _camera(origin, forward, up_hint):
    """Column-major camera matrix (right, up, back, position) whose central
    ray (odd image sizes: the middle pixel) points along `forward`."""
    f = np.asarray(forward, np.float64)
    f = f / np.linalg.norm(f)
    back = -f
    right = np.cross(np.asarray(up_hint, np.float64), back)
    if np.linalg.norm(right) < 1e-9:
        right = np.cross(np.array([0.3, 0.5, 0.8]), back)
    right /= np.linalg.norm(right)
    up = np.cross(back, right)
    m = np.eye(4)
    m[:3, 0], m[:3, 1], m[:3, 2], m[:3, 3] = right, up, back, origin
    return m.T.reshape(16).astype(np.float32)


def _uniforms(origin, forward, up_hint, w, h, half_angle, k=6, alpha_min=0.01):
    hfov = 2.0 * math.degrees(math.atan(half_angle))
    return pack_uniforms(_camera(origin, forward, up_hint), w, h, hfov=hfov, t_min=1e-3, t_max=1e5, T_min=0.01,
                         alpha_min=alpha_min, k=k)


def _icosahedron():
    """Vertices of the proxy's unit icosahedron (inradius 1, the reference's
    construction of src/main.ts:12-25) and its 20 faces as vertex triples."""
    r = (3.0 + math.sqrt(5.0)) / (2.0 * math.sqrt(3.0))
    s, t = 1.0 / r, (1.0 + math.sqrt(5.0)) / (2.0 * r)
    v = []
    for a, b in itertools.product((-1, 1), repeat=2):
        v += [(a * s, b * t, 0.0), (0.0, a * s, b * t), (b * t, 0.0, a * s)]
    v = np.array(v)
    edge = min(np.linalg.norm(v[i] - v[j]) for i in range(12) for j in range(i))
    faces = [f for f in itertools.combinations(range(12), 3)
             if all(abs(np.linalg.norm(v[a] - v[b]) - edge) < 1e-9 for a, b in itertools.combinations(f, 2))]
    assert len(faces) == 20
    return v, faces


def _proxy_map(osc, j):
    """Object-to-world 4x4 matrix of kept proxy j (float64 of the oracle's float values)."""
    p, o2w, _ = osc.proxy(j)
    m = np.eye(4)
    m[:3, :3] = np.asarray(o2w[:9], np.float64).reshape(3, 3).T
    m[:3, 3] = o2w[9:]
    return p, m


def _bits(a):
    """uint32 view of a float32 array with every NaN as one pattern: the
    reference's float arithmetic turns some extreme proxies' alpha into NaN
    on both implementations, whose default NaN payloads differ (the CPU's
    0xFFC00000, the GPU's 0x7FFFFFFF)."""
    a = np.ascontiguousarray(a, dtype=np.float32).copy()
    b = a.view(np.uint32)
    b[np.isnan(a)] = 0x7FC00000
    return b


def _check_views(ctx, rec, amin, views, need_hits=1):
    """Renders every (uniforms, w, h) view with both kernels and the oracle;
    images bit for bit, hit records of the warp-per-ray kernel bit for bit
    (NaNs as one pattern).  Returns the total count of composited entries
    seen."""
    g = Scene(ctx, rec, amin)
    o = oracle.Scene(rec, amin, "f32")
    total = 0
    try:
        for u, w, h in views:
            ref, hits = o.render(u, w, h, max_entries=64)
            for name, bt, kbuf in KERNELS:
                ctx.set_tune(g, u, w, h, kbuf=kbuf, block_threads=bt)
                try:
                    img = ctx.render(g, u, w, h)
                finally:
                    ctx._lib.gt_autotune_reset(ctx._h)
                np.testing.assert_array_equal(_bits(img.reshape(-1, 4)), _bits(ref), err_msg=name)
            pix = np.arange(w * h, dtype=np.uint32)
            got = ctx.render_hits(g, u, w, h, pix, max_entries=64)
            np.testing.assert_array_equal(got["count"], hits["count"])
            np.testing.assert_array_equal(got["rounds"], hits["rounds"])
            for q in range(w * h):
                m = min(int(hits["count"][q]), 64)
                np.testing.assert_array_equal(got["pidx"][q, :m], hits["pidx"][q, :m])
                np.testing.assert_array_equal(_bits(got["t"][q, :m]), _bits(hits["t"][q, :m]))
                np.testing.assert_array_equal(_bits(got["alpha"][q, :m]), _bits(hits["alpha"][q, :m]))
            total += int(hits["count"].sum())
    finally:
        g.close()
    assert total >= need_hits
    return total


def test_shared_edge_duplicate_on_both_kernels(ctx):
    """The ray along -z through the centre of an isotropic particle crosses
    the edge between two front faces: two entries of the same particle."""
    rec = _records([(0.0, 0.0, 0.0)], [(0.05, 0.05, 0.05)], [(1.0, 0.0, 0.0, 0.0)], [0.8])
    rec[0, 20:] = 0.0  # DC only
    w = h = 33
    u = pack_uniforms(_camera((0.0, 0.0, 4.0), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0)), w, h, hfov=60.0, t_min=1e-3,
                      t_max=1e5, T_min=0.01, alpha_min=0.01, k=4)
    g = Scene(ctx, rec, 0.01)
    try:
        got = ctx.render_hits(g, u, w, h, np.array([16 * 33 + 16], np.uint32), max_entries=4)
        assert got["count"][0] == 2 and got["pidx"][0, 0] == got["pidx"][0, 1] == 0
        assert got["t"][0, 0] == got["t"][0, 1]
    finally:
        g.close()
    _check_views(ctx, rec, 0.01, [(u, w, h)], need_hits=2)


def test_rays_grazing_silhouettes_and_box_vertices(ctx):
    """Narrow pinhole views (image span 1e-4 rad) aimed at silhouette edges
    and at the vertices that touch the proxies' world boxes, for isotropic,
    rotated and anisotropic particles: rays hit, miss and graze."""
    rng = np.random.default_rng(61)
    v, faces = _icosahedron()
    pos = [(0.0, 0.0, 0.0), (1.0, -0.5, 0.3), (-0.7, 0.4, -0.2)]
    scale = [(0.1, 0.1, 0.1), (0.12, 0.05, 0.03), (0.02, 0.09, 0.2)]
    rot = [(1.0, 0.0, 0.0, 0.0)] + list(_unit_quats(rng, 2))
    rec = _records(pos, scale, rot, [0.9, 0.7, 0.95], seed=61)
    osc = oracle.Scene(rec, 0.01, "f64")
    views = []
    for j in range(osc.n_kept):
        _, m = _proxy_map(osc, j)
        wv = (m[:3, :3] @ v.T).T + m[:3, 3]
        for _ in range(4):
            d = rng.normal(size=3)
            d /= np.linalg.norm(d)
            # silhouette edges: faces on both sides face opposite ways
            normals = []
            for f in faces:
                a, b, c = wv[list(f)]
                n = np.cross(b - a, c - a)
                if np.dot(n, a - m[:3, 3]) < 0:
                    n = -n
                normals.append(n)
            sil = []
            for fa, fb in itertools.combinations(range(20), 2):
                shared = set(faces[fa]) & set(faces[fb])
                if len(shared) == 2 and np.dot(normals[fa], d) * np.dot(normals[fb], d) < 0:
                    sil.append(sorted(shared))
            e = sil[rng.integers(len(sil))]
            for target in (0.5 * (wv[e[0]] + wv[e[1]]), wv[e[0]]):
                views.append((_uniforms(target - 2.0 * d, d, (0.0, 1.0, 0.0), 17, 17, 1e-4), 17, 17))
        # the vertices at the extremes of the world box, seen along each axis
        for a in range(3):
            for idx in (int(np.argmin(wv[:, a])), int(np.argmax(wv[:, a]))):
                d = np.zeros(3)
                d[(a + 1) % 3] = 1.0
                d += 1e-3 * rng.normal(size=3)
                views.append((_uniforms(wv[idx] - 2.0 * d, d, (0.0, 0.0, 1.0), 15, 15, 2e-5), 15, 15))
    total = _check_views(ctx, rec, 0.01, views, need_hits=50)
    assert total < sum(w * h for _, w, h in views)  # some rays miss


def test_rays_nearly_in_a_face_plane(ctx):
    """Rays at angles of 1e-7 to 1e-4 rad to a face's plane, aimed at a
    point inside the face, from both sides (front- and back-facing by a hair):
    the facing tolerance tau of the kernels is ~1e-5 of these products."""
    rng = np.random.default_rng(62)
    v, faces = _icosahedron()
    rec = _records([(0.2, -0.1, 0.4), (0.0, 0.0, 0.0)], [(0.15, 0.07, 0.04), (0.1, 0.1, 0.1)],
                   [tuple(_unit_quats(rng, 1)[0]), (1.0, 0.0, 0.0, 0.0)], [0.9, 0.8], seed=62)
    osc = oracle.Scene(rec, 0.01, "f64")
    views = []
    for j in range(osc.n_kept):
        _, m = _proxy_map(osc, j)
        lin = m[:3, :3]
        for f in rng.choice(20, size=3, replace=False):
            a, b, c = (lin @ v[list(faces[f])].T).T + m[:3, 3]
            n = np.cross(b - a, c - a)
            n /= np.linalg.norm(n)
            if np.dot(n, a - m[:3, 3]) < 0:
                n = -n  # outward
            tan = (b - a) / np.linalg.norm(b - a)
            x = 0.5 * a + 0.3 * b + 0.2 * c  # inside the face
            for eps in (1e-7, 1e-6, 4e-6, 1e-5, 2e-5, 5e-5, 1e-4):
                for sgn in (1.0, -1.0):
                    d = math.cos(eps) * tan - sgn * math.sin(eps) * n
                    # rows vary the angle to the plane by +-20 %, columns lie in it
                    views.append((_uniforms(x - 0.3 * d, d, n, 9, 9, 0.2 * eps), 9, 9))
    _check_views(ctx, rec, 0.01, views, need_hits=20)


def test_rays_through_edges_and_vertices(ctx):
    """Narrow views (image span 1e-5 of the distance) aimed at points 1e-7 to
    1e-2 (in units of the face) from an edge or a vertex of a face, seen from
    random directions: the face test keeps for the exact triangle test only
    the faces whose plane crossing lies within its rounding reach of the
    latest one, and near an edge or a vertex two or more faces do."""
    rng = np.random.default_rng(64)
    v, faces = _icosahedron()
    rec = _records([(0.0, 0.0, 0.0), (0.6, 0.2, -0.3), (-0.5, -0.4, 0.2)],
                   [(0.1, 0.1, 0.1), (0.15, 0.05, 0.02), (0.01, 0.12, 0.06)],
                   [(1.0, 0.0, 0.0, 0.0)] + list(_unit_quats(rng, 2)), [0.9, 0.6, 0.99], seed=64)
    osc = oracle.Scene(rec, 0.01, "f64")
    views = []
    for j in range(osc.n_kept):
        _, m = _proxy_map(osc, j)
        lin = m[:3, :3]
        for f in rng.choice(20, size=5, replace=False):
            a, b, c = (lin @ v[list(faces[f])].T).T + m[:3, 3]
            for off in (1e-7, 1e-5, 1e-3, 1e-2):
                s_ = off * rng.choice([-1.0, 1.0])
                edge = a + 0.4 * (b - a) + s_ * (c - a)            # beside edge ab
                vert = a + off * (b - a) + abs(s_) * (c - a)         # beside vertex a
                for x in (edge, vert):
                    d = rng.normal(size=3)
                    d /= np.linalg.norm(d)
                    n = np.cross(b - a, c - a)
                    if np.dot(d, n) * np.dot(n, a - m[:3, 3]) > 0:
                        d = -d  # towards the face from outside
                    views.append((_uniforms(x - 2.0 * d, d, (0.0, 1.0, 0.0), 9, 9, 1e-5), 9, 9))
    _check_views(ctx, rec, 0.01, views, need_hits=50)


@pytest.mark.parametrize("ratio", [1e3, 1e4])
def test_needle_and_disc_proxies(ctx, ratio):
    """Scale ratios of 1e3 and 1e4 (needles and discs), random orientations.
    At 1e4 the response's float arithmetic (src/GS_shader.ts:111-136: the
    precision matrix holds 1/s^2 ~ 1e10) loses E to cancellation, so some
    entries get alpha > 1 and a few pixels NaN, identically on both sides
    (the FP64 render has none)."""
    rng = np.random.default_rng(int(ratio))
    n = 600
    pos = rng.uniform(-0.6, 0.6, size=(n, 3))
    big = rng.uniform(0.05, 0.2, size=n)
    scale = np.stack([big, big / ratio, big / ratio], axis=1)
    scale[n // 2:, 1] = big[n // 2:]  # discs
    for i in range(n):
        scale[i] = rng.permutation(scale[i])
    rec = _records(pos, scale, _unit_quats(rng, n), rng.uniform(0.05, 0.99, size=n), seed=int(ratio))
    views = []
    for cam in ((0.0, 0.0, 2.5), (1.7, 1.1, -1.3)):
        c = np.asarray(cam)
        views.append((_uniforms(c, -c, (0.0, 1.0, 0.0), 64, 48, math.tan(math.radians(25.0)), k=8), 64, 48))
    _check_views(ctx, rec, 0.01, views, need_hits=1000)


def test_tiny_proxies_far_from_the_origin(ctx):
    """Particles of scale ~1e-4 about 1.4e3 from the origin, seen from 0.02
    away: the world-space box padding and the object-space margins at large
    |origin| relative to the proxy size."""
    rng = np.random.default_rng(63)
    n = 300
    c0 = np.array([1000.0, 500.0, -800.0])
    pos = c0 + rng.normal(0.0, 1e-3, size=(n, 3))
    scale = rng.uniform(0.5e-4, 3e-4, size=(n, 3))
    rec = _records(pos, scale, _unit_quats(rng, n), rng.uniform(0.05, 0.99, size=n), seed=63)
    views = []
    for off in ((0.0, 0.0, 0.02), (0.015, -0.01, 0.0), (-0.01, 0.012, -0.01)):
        o = c0 + np.asarray(off)
        views.append((_uniforms(o, c0 - o, (0.0, 1.0, 0.0), 48, 40, math.tan(math.radians(10.0)), k=6), 48, 40))
    _check_views(ctx, rec, 0.01, views, need_hits=500)
