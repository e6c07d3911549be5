"""Regenerates tests/golden/pc_short_ingest.json from the reference's sample
file data/pc_short.ply (100 SH-3 Gaussians) through gtrace.ply.PackedGaussians,
cross-checked against the oracle's C restatement of the same loader.

Run with the path of that file (in the reference's checkout) as the argument
or in the GTRACE_REFERENCE_PLY environment variable:
    python tests/golden/make_golden.py <reference checkout>/data/pc_short.ply
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "webgpu-gaussiantracer_b200"))

from gtrace.ply import PackedGaussians  # noqa: E402
from oracle import oracle  # noqa: E402


def main(path):
    data = open(path, "rb").read()
    pg = PackedGaussians(data)
    rec = pg.gaussiansBuffer
    ref = oracle.ply_to_aos(data)
    ulps = np.abs(rec.view(np.int32).astype(np.int64) - ref.view(np.int32).astype(np.int64)).max()
    assert ulps <= 1, ulps
    out = {"source": "data/pc_short.ply of the reference", "n": pg.numGaussians,
           "degree": pg.sphericalHarmonicsDegree, "column_sums": rec.astype(np.float64).sum(axis=0).tolist(),
           "first3_bits": rec[:3].view(np.uint32).tolist(), "max_ulp_vs_oracle": int(ulps)}
    with open(os.path.join(HERE, "pc_short_ingest.json"), "w") as fh:
        json.dump(out, fh)
    print("wrote", os.path.join(HERE, "pc_short_ingest.json"), "n =", pg.numGaussians, "ulps =", ulps)


if __name__ == "__main__":
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("GTRACE_REFERENCE_PLY", "")
    if not src:
        raise SystemExit("usage: make_golden.py <reference checkout>/data/pc_short.ply")
    main(src)
