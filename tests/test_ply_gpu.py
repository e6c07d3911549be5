"""Native PLY ingest on the GPU (gt_ply_pack, gt_scene_create_from_ply*):
packed records equal to the oracle's restatement of PackedGaussians
(src/GS_ply.ts:39-253) bit for bit, except words whose double value sits
within 4 double ulps of a binary32 rounding boundary (two correct `exp`
implementations may round those apart); scenes built from the PLY render
exactly like scenes built from the packed buffer."""
import os
import tempfile

import numpy as np
import pytest

import ply_cases as P
from gtrace import ply, synth
from gtrace._lib import GTraceError
from gtrace.tracer import Scene
from oracle import oracle

pytestmark = pytest.mark.gpu

ACCEPTED = [c for c in P.cases() if c[2]]
REJECTED = [c for c in P.cases() if not c[2]]


@pytest.mark.parametrize("name,blob,accepted", ACCEPTED, ids=[c[0] for c in ACCEPTED])
def test_pack_matches_oracle(ctx, name, blob, accepted):
    got, info = ctx.pack_ply(blob)
    pg = ply.PackedGaussians(blob)
    assert info["n_vertices"] == pg.numGaussians and info["sh_degree"] == pg.sphericalHarmonicsDegree
    if pg.numGaussians == 0:
        assert got.size == 0
        return
    want = oracle.ply_to_aos(blob)
    assert got.shape == want.shape
    P.check_activation(got, want, P.exact_words(pg))


@pytest.mark.parametrize("name,blob,accepted", REJECTED, ids=[c[0] for c in REJECTED])
def test_rejects_like_the_reference(ctx, name, blob, accepted):
    with pytest.raises(GTraceError) as ei:
        ctx.pack_ply(blob)
    assert ei.value.status == 1 and ei.value.message.startswith("PLY")
    with pytest.raises(GTraceError):
        Scene.from_ply(ctx, blob, 0.01)


def test_pack_large_unaligned(ctx):
    """200k vertices behind a uchar column (every float unaligned), several
    tiles per block of the packing kernel."""
    std3 = [("float", nm) for nm in P._names(3)]
    blob = P.build([("uchar", "red")] + std3 + [("uchar", "green")], 200_000, seed=31)
    got, info = ctx.pack_ply(blob)
    assert info["row_bytes"] == 250
    pg = ply.PackedGaussians(blob)
    ties = P.check_activation(got, oracle.ply_to_aos(blob), P.exact_words(pg))
    assert ties <= 8


def test_scene_from_ply_renders_like_packed(ctx):
    """A PLY scene's proxies come from the double activations (as the
    reference's do): the same image as gt_scene_create_ex with the oracle's
    activations, and as the oracle's scene built from them."""
    blob = ply.write_ply(synth.raw_small(n=6000, seed=synth.SEED_BASE + 5))
    packed, act = oracle.ply_to_aos(blob, activations=True)
    v = synth.view(128, 96, (0.0, 0.0, 4.0), k=6)
    a = Scene.from_ply(ctx, blob, 0.01)
    b = Scene(ctx, packed, 0.01, activated=act)
    assert a.n == 6000 and a.ply_info["sh_degree"] == 3
    ia = ctx.render(a, v.uniforms, v.width, v.height)
    ib = ctx.render(b, v.uniforms, v.width, v.height)
    assert np.array_equal(ia.view(np.uint32), ib.view(np.uint32))
    ref, _ = oracle.Scene(packed, 0.01, "f32", activated=act).render(v.uniforms, v.width, v.height)
    assert np.array_equal(ia.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))
    # the mirror's gaussianData gives the same proxies
    c = Scene(ctx, ply.PackedGaussians(blob).gaussiansBuffer, 0.01,
              activated=ply.PackedGaussians(blob).activations())
    ic = ctx.render(c, v.uniforms, v.width, v.height)
    assert np.array_equal(ia.view(np.uint32), ic.view(np.uint32))
    c.close()
    with tempfile.TemporaryDirectory() as d:
        path = os.path.join(d, "scene.ply")
        with open(path, "wb") as fh:
            fh.write(blob)
        c = Scene.from_ply(ctx, path, 0.01, fast_build=True)
        ic = ctx.render(c, v.uniforms, v.width, v.height)
        assert np.array_equal(ia.view(np.uint32), ic.view(np.uint32))
        c.close()
        with pytest.raises(GTraceError):
            Scene.from_ply(ctx, os.path.join(d, "missing.ply"), 0.01)
    a.close()
    b.close()


def test_lower_degree_scene(ctx):
    """A degree-1 file packs 128-byte records; the missing SH bands read as
    zero (the reference's shader would read the next record there)."""
    raw = synth.raw_small(n=3000, seed=synth.SEED_BASE + 6)
    raw1 = dict(raw)
    raw1["sh"] = raw["sh"][:, :4, :]
    blob = ply.write_ply(raw1, sh_degree=1)
    s = Scene.from_ply(ctx, blob, 0.01)
    assert s.ply_info["record_stride"] == 128
    packed, act = oracle.ply_to_aos(blob, activations=True)
    v = synth.view(96, 64, (0.0, 0.0, 4.0), k=6)
    img = ctx.render(s, v.uniforms, v.width, v.height)
    ref, _ = oracle.Scene(packed, 0.01, "f32", activated=act).render(v.uniforms, v.width, v.height)
    assert np.array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))
    s.close()


def test_opacity_cut_in_double_like_the_reference(ctx):
    """The reference cuts proxies on the double opacity (src/main.ts:79). With
    alpha_min between a Gaussian's double opacity and its binary32 rounding,
    the Gaussian keeps its proxy from a PLY (or with gt_scene_create_ex) and
    loses it with gt_scene_create on the packed records.  Its proxy's hits
    then take k-buffer slots in the rounds of the rays through it, as in the
    reference, and the image equals the oracle's built the same way."""
    x = np.float32(-4.6)
    while True:  # a binary32 logit whose double opacity rounds down to binary32
        o = 1.0 / (1.0 + np.exp(-np.float64(x)))
        if np.float64(np.float32(o)) < o:
            break
        x = np.nextafter(x, np.float32(0))
    alpha_min = (float(np.float32(o)) + o) / 2.0
    raw = synth.raw_small(n=400, seed=synth.SEED_BASE + 8)
    raw["opacity_logit"][:50] = x
    blob = ply.write_ply(raw)
    pg = ply.PackedGaussians(blob)
    assert (pg.gaussianData["opacity"][:50] > alpha_min).all()
    assert (pg.gaussiansBuffer[:50, 12].astype(np.float64) < alpha_min).all()
    a = Scene.from_ply(ctx, blob, alpha_min)
    b = Scene(ctx, pg.gaussiansBuffer, alpha_min)
    assert a.info()["n_kept"] == b.info()["n_kept"] + 50
    packed, act = oracle.ply_to_aos(blob, activations=True)
    v = synth.view(80, 60, (0.0, 0.0, 4.0), k=3)
    img = ctx.render(a, v.uniforms, v.width, v.height)
    ref, _ = oracle.Scene(packed, alpha_min, "f32", activated=act).render(v.uniforms, v.width, v.height)
    assert np.array_equal(img.reshape(-1, 4).view(np.uint32), ref.view(np.uint32))
    a.close()
    b.close()
