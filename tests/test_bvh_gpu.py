"""Structural invariants of the hierarchy built on the GPU (Morton codes,
radix sort, PLOC or Karras, 8-wide collapse), read back with
gt_scene_export_bvh: every proxy is a leaf exactly once, every node but the
root has exactly one parent and is reachable from the root, each child box
contains its subtree's boxes, each leaf box contains its proxy (the world
box of the icosahedron under the proxy transform the oracle computes), and
the leaves are exactly the particles with opacity > alpha_min."""
import math

import numpy as np
import pytest

from conftest import small_scene
from gtrace import synth
from gtrace.tracer import Scene
from oracle import oracle

pytestmark = pytest.mark.gpu

LEAF, EMPTY = 0x80000000, 0xFFFFFFFF


def _ico_vertices():
    rr = (3.0 + math.sqrt(5.0)) / (2.0 * math.sqrt(3.0))
    ss, tt = 1.0 / rr, (1.0 + math.sqrt(5.0)) / (2.0 * rr)
    v = [(-ss, tt, 0), (ss, tt, 0), (-ss, -tt, 0), (ss, -tt, 0), (0, -ss, tt), (0, ss, tt), (0, -ss, -tt),
         (0, ss, -tt), (tt, 0, -ss), (tt, 0, ss), (-tt, 0, -ss), (-tt, 0, ss)]
    return np.array(v, dtype=np.float64).astype(np.float32)


def _proxy_boxes(packed, alpha_min):
    """Particle index -> world box (lo, hi) of its proxy, from the oracle."""
    s = oracle.Scene(packed, alpha_min, "f32")
    L = oracle.lib()
    verts = _ico_vertices()
    boxes = {}
    for j in range(int(L.or_scene_kept_f32(s._h))):
        p, o2w, _ = s.proxy(j)
        M = np.asarray(o2w, dtype=np.float32).reshape(4, 3)  # columns
        w = ((M[0] * verts[:, :1] + M[1] * verts[:, 1:2]) + M[2] * verts[:, 2:3]) + M[3]
        boxes[p] = (w.min(axis=0), w.max(axis=0))
    return boxes


def _check(scene, packed, alpha_min):
    nodes, leaves, info = scene.export_bvh()
    n8, m = info["n_nodes8"], info["n_leaves"]
    boxes = _proxy_boxes(packed, alpha_min)
    assert m == len(boxes)
    assert sorted(leaves.tolist()) == sorted(boxes)          # the kept particles, each once
    if info["root"] & LEAF:  # a one-proxy scene: the root is the leaf
        assert m == 1 and info["root"] == LEAF
        return
    refs = nodes[:, :, 6].view(np.uint32)
    lo, hi = nodes[:, :, 0:3], nodes[:, :, 3:6]
    is_empty = refs == EMPTY
    is_leaf = ~is_empty & ((refs & LEAF) != 0)
    is_node = ~is_empty & ~is_leaf
    # every leaf referenced once, every node but the root referenced once
    assert np.array_equal(np.sort(refs[is_leaf] & 0x7FFFFFFF), np.arange(m, dtype=np.uint32))
    assert np.array_equal(np.sort(refs[is_node]), np.arange(1, n8, dtype=np.uint32))
    # reachable from the root without revisits
    seen, todo = np.zeros(n8, bool), [0]
    while todo:
        i = todo.pop()
        assert not seen[i]
        seen[i] = True
        todo.extend(int(r) for r in refs[i][is_node[i]])
    assert seen.all()
    # child boxes contain their subtree; leaf boxes contain their proxy
    for i in range(n8):
        for c in np.nonzero(is_node[i])[0]:
            k = int(refs[i, c])
            occ = ~is_empty[k]
            assert (lo[k][occ] >= lo[i, c]).all() and (hi[k][occ] <= hi[i, c]).all()
        for c in np.nonzero(is_leaf[i])[0]:
            p = int(leaves[refs[i, c] & 0x7FFFFFFF])
            blo, bhi = boxes[p]
            assert (blo >= lo[i, c]).all() and (bhi <= hi[i, c]).all()


@pytest.mark.parametrize("fast_build", [False, True])
def test_hierarchy_invariants(ctx, fast_build):
    pg = small_scene(n=20000, seed=61)
    s = Scene(ctx, pg.gaussiansBuffer, 0.05, fast_build=fast_build)
    _check(s, pg.gaussiansBuffer, 0.05)
    s.close()


def test_hierarchy_invariants_clusters(ctx):
    pg = synth.pack(synth.raw_clusters(30000, synth.SEED_BASE + 9))
    s = Scene(ctx, pg.gaussiansBuffer, 0.01)
    _check(s, pg.gaussiansBuffer, 0.01)
    s.close()


@pytest.mark.parametrize("n", [1, 2, 9, 40])
def test_hierarchy_invariants_coincident(ctx, n):
    pg = small_scene(n=1, seed=38)
    rec = np.repeat(pg.gaussiansBuffer[:1], n, axis=0)
    rec[:, 0:3] = 0.0
    rec[:, 4:7] = 0.3
    rec[:, 12] = 0.9
    s = Scene(ctx, rec, 0.01)
    _check(s, rec, 0.01)
    s.close()
