"""CPU tests of the C-ABI surface and the host-side mirror of the reference
(uniform block, camera, PLY ingest).  No kernel runs here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT
from gtrace import _lib as L
from gtrace.ply import PackedGaussians, record_stride, write_ply
from gtrace.uniforms import look_at, pack_uniforms, unpack_uniforms
from gtrace import synth

HEADER = os.path.join(ROOT, "include", "gtrace.h")
# the reference's sample file (data/pc_short.ply of its checkout), when available
REF_PLY = os.environ.get("GTRACE_REFERENCE_PLY", "")
GOLDEN = os.path.join(ROOT, "tests", "golden")


def declared_symbols():
    text = open(HEADER).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(gt_[a-z_0-9]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = L.load()
    names = declared_symbols()
    assert len(names) >= 20
    for name in names:
        assert hasattr(lib, name), name
    # and the binding declares exactly the header's entry points
    assert sorted(n for n, _, _ in L.SIGNATURES) == names


def test_version_and_struct_layouts():
    lib = L.load()
    assert lib.gt_version() == 2
    assert C.sizeof(L.Uniforms) == 112
    assert C.sizeof(L.TuneResult) == 40 and L.TuneResult.handoff_after.offset == 32
    assert C.sizeof(L.SceneInfo) == 64 and L.SceneInfo.upload_ms.offset == 60
    assert L.Uniforms.k.offset == 88 and L.Uniforms.debug_mode.offset == 104
    assert L.Uniforms.camera_aspect.offset == 64 and L.Uniforms.T_min.offset == 80


def test_context_without_gpu_fails_cleanly():
    """gt_context_create reports GT_ERR_NO_DEVICE (never aborts) when no GPU is
    visible; on a GPU host it succeeds."""
    lib = L.load()
    h = C.c_void_p()
    rc = lib.gt_context_create(0, C.byref(h))
    if rc == L.GT_OK:
        assert lib.gt_context_destroy(h) == L.GT_OK
    else:
        assert rc == L.GT_ERR_NO_DEVICE
        assert L.last_error(None)
    assert lib.gt_context_create(-1, C.byref(h)) in (L.GT_ERR_NO_DEVICE,)


def test_null_arguments_rejected():
    lib = L.load()
    assert lib.gt_context_create(0, None) == L.GT_ERR_INVALID_ARG
    assert lib.gt_render(None, None, None, 1, 1, None, 0, None) == L.GT_ERR_INVALID_ARG
    assert lib.gt_scene_create(None, None, 0, 320, 0.01, 0, None) == L.GT_ERR_INVALID_ARG
    assert lib.gt_scene_get_info(None, None) == L.GT_ERR_INVALID_ARG
    assert lib.gt_context_destroy(None) == L.GT_OK
    assert lib.gt_scene_destroy(None) == L.GT_OK


def test_uniform_block_matches_reference_packing():
    """src/main.ts:520-534: toWorld at 0, aspect at 64 (tan(hfov/2), then that
    f32 value times H/W), t_min 72, t_max 76, T_min 80, alpha_min 84, k 88,
    sh_degree_max 92, accumulatedFrames 96, earlyStop 100 (<= 0 -> 0xFFFFFFFF),
    debugMode 104."""
    tw = look_at((0.0, 0.0, 3.0))
    u = pack_uniforms(tw, 960, 640, hfov=60.0, t_min=1e-3, t_max=1e5, T_min=0.03, alpha_min=0.2, k=6,
                      sh_degree_max=3, early_stop=0, debug_mode=1)
    assert u.nbytes == 112
    d = unpack_uniforms(u)
    assert d["k"] == 6 and d["debug_mode"] == 1 and d["early_stop"] == 0xFFFFFFFF
    a0 = np.float32(np.tan(np.pi / 6))
    assert d["camera_aspect"][0] == a0
    assert d["camera_aspect"][1] == np.float32(float(a0) * (640 / 960))
    np.testing.assert_array_equal(d["to_world"], tw)
    # the WASD camera at (0,0,3) looking at the origin is the identity rotation
    np.testing.assert_allclose(tw.reshape(4, 4).T[:3, :3], np.eye(3), atol=1e-7)
    assert unpack_uniforms(pack_uniforms(tw, 8, 8, early_stop=3))["early_stop"] == 3


def test_look_at_back_axis_points_away_from_target():
    tw = look_at((3.0, 4.0, 12.0), (1.0, 0.0, 0.0)).reshape(4, 4)  # rows of this view are columns
    back = tw[2, :3]
    v = np.array([2.0, 4.0, 12.0])
    np.testing.assert_allclose(back, v / np.linalg.norm(v), atol=1e-6)
    np.testing.assert_allclose(tw[3, :3], (3.0, 4.0, 12.0))
    r = tw[:3, :3]
    np.testing.assert_allclose(r @ r.T, np.eye(3), atol=1e-6)


def test_packed_layout_and_activation():
    raw = synth.raw_small(n=5, seed=1)
    pg = PackedGaussians(write_ply(raw))
    assert pg.numGaussians == 5 and pg.sphericalHarmonicsDegree == 3
    assert record_stride(3) == 320 and pg.gaussiansBuffer.shape == (5, 80)
    rec = pg.gaussiansBuffer
    np.testing.assert_array_equal(rec[:, 0:3], np.float32(raw["xyz"]))
    np.testing.assert_allclose(rec[:, 4:7], np.exp(np.float32(raw["log_scale"]).astype(np.float64)), rtol=1e-7)
    q = np.float32(raw["rot"]).astype(np.float64)
    np.testing.assert_allclose(rec[:, 8:12], q / np.linalg.norm(q, axis=1, keepdims=True), rtol=1e-6)
    np.testing.assert_allclose(rec[:, 12], 1 / (1 + np.exp(-np.float32(raw["opacity_logit"]).astype(np.float64))),
                               rtol=1e-7)
    # sh[0] = f_dc, sh[i+1] = (f_rest_i, f_rest_{15+i}, f_rest_{30+i})
    np.testing.assert_array_equal(rec[:, 16:19], np.float32(raw["sh"][:, 0, :]))
    np.testing.assert_array_equal(rec[:, 16 + 4 * 7:19 + 4 * 7], np.float32(raw["sh"][:, 7, :]))
    assert (rec[:, [3, 7, 13, 14, 15, 19]] == 0).all()


def test_lower_sh_degree_stride():
    raw = synth.raw_small(n=3, seed=2)
    raw["sh"] = raw["sh"][:, :4, :]
    pg = PackedGaussians(write_ply(raw, sh_degree=1))
    assert pg.sphericalHarmonicsDegree == 1 and pg.gaussiansBuffer.shape == (3, (64 + 16 * 4) // 4)


@pytest.mark.skipif(not (REF_PLY and os.path.exists(REF_PLY)), reason="GTRACE_REFERENCE_PLY not set")
def test_reference_sample_ply_golden():
    """The reference's own sample file (data/pc_short.ply, 100 SH-3 Gaussians)
    ingests to the committed golden summary (tests/golden/make_golden.py)."""
    import json
    with open(REF_PLY, "rb") as fh:
        pg = PackedGaussians(fh.read())
    g = json.load(open(os.path.join(GOLDEN, "pc_short_ingest.json")))
    assert pg.numGaussians == g["n"] and pg.sphericalHarmonicsDegree == g["degree"]
    rec = pg.gaussiansBuffer
    np.testing.assert_allclose(rec.astype(np.float64).sum(axis=0), np.array(g["column_sums"]), rtol=1e-6, atol=1e-6)
    np.testing.assert_array_equal(rec[:3].view(np.uint32).tolist(), g["first3_bits"])


def test_golden_ingest_fixture_selfconsistent():
    """Fixture committed from the reference sample (works without the mount)."""
    import json
    g = json.load(open(os.path.join(GOLDEN, "pc_short_ingest.json")))
    first = np.array(g["first3_bits"], dtype=np.uint32).view(np.float32)
    assert first.shape == (3, 80)
    # activated fields: unit quaternions, opacity in (0,1), positive scales
    np.testing.assert_allclose(np.linalg.norm(first[:, 8:12], axis=1), 1.0, rtol=1e-6)
    assert ((first[:, 12] > 0) & (first[:, 12] < 1)).all() and (first[:, 4:7] > 0).all()
