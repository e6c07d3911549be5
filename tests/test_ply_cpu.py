"""PLY ingest on the CPU: the native header decoder of libgtrace.so (host
code, no GPU), the Python mirror of PackedGaussians and the oracle's C
restatement must accept and reject the same files and agree on every field
of the header and every packed word (src/GS_ply.ts:58-253)."""
import numpy as np
import pytest

import ply_cases as P
from gtrace import ply
from gtrace.tracer import ply_header
from oracle import oracle


def _mirror(blob):
    try:
        return ply.PackedGaussians(blob)
    except ply.PlyError:
        return None


def _native(blob):
    from gtrace._lib import GTraceError
    try:
        return ply_header(blob)
    except GTraceError as e:
        assert e.status == 1, e  # GT_ERR_INVALID_ARG
        return None


def _oracle(blob):
    try:
        return oracle.ply_to_aos(blob)
    except ValueError:
        return None


@pytest.mark.parametrize("name,blob,accepted", P.cases(), ids=[c[0] for c in P.cases()])
def test_header_rules_agree(name, blob, accepted):
    pg, hdr, aos = _mirror(blob), _native(blob), _oracle(blob)
    assert (pg is not None, hdr is not None, aos is not None) == (accepted,) * 3
    if not accepted:
        return
    assert hdr["n_vertices"] == pg.numGaussians == aos.shape[0]
    assert hdr["sh_degree"] == pg.sphericalHarmonicsDegree
    assert hdr["record_stride"] == ply.record_stride(pg.sphericalHarmonicsDegree)
    assert hdr["data_offset"] == blob.index(b"end_header") + 11
    if pg.numGaussians:
        assert hdr["record_stride"] == pg.gaussiansBuffer.shape[1] * 4
        P.check_activation(pg.gaussiansBuffer, aos, P.exact_words(pg))


def test_key_order_rules():
    """Array-index names first (ascending), repeated names keep their place."""
    blob = P.build([("float", "b"), ("float", "12"), ("uchar", "a"), ("float", "3"), ("float", "b")], 0)
    count, props, _ = ply._decode_header(blob)
    assert props == [("3", "float"), ("12", "float"), ("b", "float"), ("a", "uchar")]


def test_mirror_matches_oracle_large():
    blob = P.standard(20000, 3, seed=99)
    pg = ply.PackedGaussians(blob)
    aos = oracle.ply_to_aos(blob)
    ties = P.check_activation(pg.gaussiansBuffer, aos, P.exact_words(pg))
    assert ties <= 2



def test_oracle_activations_match_mirror():
    """The double activations behind the packed records (the values the
    reference builds its proxies from) agree between the oracle's loader and
    the mirror to an ulp of exp, and round to the packed words."""
    blob = P.standard(3000, 3, seed=77)
    pg = ply.PackedGaussians(blob)
    aos, act = oracle.ply_to_aos(blob, activations=True)
    mirror = pg.activations()
    assert act.shape == mirror.shape == (3000, 8)
    assert np.all(np.abs(act - mirror) <= 2 * np.spacing(np.abs(mirror)))
    assert np.array_equal(act[:, 4:].astype(np.float32), aos[:, 8:12])
    assert np.array_equal(act[:, 0].astype(np.float32), aos[:, 12])
