"""How far the build's canonical arithmetic is from the alternatives, counted
on the benchmarked scenes and asserted, so that a change cannot move the
numbers silently.

* Plane-test cell centres.  The canonical build accumulates the centres
  "+= cellSize" from the first candidate cell, as the reference does
  (src/Control/Algorithm/FastBuildKernels.h:144-164,
  src/Control/Algorithm/TwoLevelBuildKernels.h:396-420).  An earlier form
  computed them per cell as (i*s + o) + s/2; the two give the same pairs on
  the plain 65,536-triangle soup and on the 1M-triangle cluster; on the
  4.2M-triangle heightfield the accumulated centres keep one (cell, triangle)
  pair more (10,747,835 against 10,747,834).
* Leaf resolution.  The canonical rule is the exact floor of the cube root
  (largest r with r^3 <= cs^3 * lambda * refs / V, clamped to [1, 255]); the
  reference evaluates cs * powf(lambda * refs / V, 0.3333333f) and truncates
  (src/Control/Algorithm/TwoLevelBuildKernels.h:48-81).  With host powf the
  two agree on every top cell of the cluster (top lambda 1/16, leaf lambda 4)
  and of the reference's default two-level grid on the soup and the cluster;
  the reference rule gives no zero resolution and none above 255 there.
"""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes


def _pair_diff(a, b):
    sa, sb = set(a.tolist()), set(b.tolist())
    return len(sa - sb), len(sb - sa)


def _uniform(sc, flags):
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 5.0)
    oracle.set_reference_arithmetic(flags)
    try:
        return oracle.build_uniform(sc.vertices, sc.indices, b, res)
    finally:
        oracle.set_reference_arithmetic(0)


def _two_level(sc, lam_top, lam_leaf, divisor, min_res, flags):
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, lam_top, divisor, min_res)
    oracle.set_reference_arithmetic(flags)
    try:
        return oracle.build_two_level(sc.vertices, sc.indices, b, res, lam_leaf, 16)
    finally:
        oracle.set_reference_arithmetic(0)


def _same_two_level(g, h):
    return (np.array_equal(g.cells, h.cells) and np.array_equal(g.leaves, h.leaves)
            and np.array_equal(g.indices, h.indices) and np.array_equal(g.top_pairs, h.top_pairs))


def test_centres_plain_soup():
    sc = scenes.uniform_soup(65536, seed=0)
    g, d = _uniform(sc, 0), _uniform(sc, oracle.DIRECT_CENTRES)
    assert g.top_pairs.size == 258_680
    assert _pair_diff(g.top_pairs, d.top_pairs) == (0, 0)
    assert np.array_equal(g.cells, d.cells)


@pytest.mark.parametrize("lam_top,lam_leaf,divisor,min_res", [(1.0 / 16.0, 4.0, 1, 2), (5.0, 1.2, 6, 2)])
def test_cluster_two_level_centres_and_leaf_rule(lam_top, lam_leaf, divisor, min_res):
    sc = scenes.cluster_in_field(1 << 20, seed=1)
    g = _two_level(sc, lam_top, lam_leaf, divisor, min_res, 0)
    for flags in (oracle.DIRECT_CENTRES, oracle.REF_LEAF_POW, oracle.DIRECT_CENTRES | oracle.REF_LEAF_POW):
        assert _same_two_level(g, _two_level(sc, lam_top, lam_leaf, divisor, min_res, flags)), flags
    raw = oracle.leaf_res_reference(g, lam_leaf, 16)
    assert int((raw == 0).any(axis=1).sum()) == 0
    assert int((raw > 255).any(axis=1).sum()) == 0
    mine = np.stack([g.cells[:, 1] & 0xFF, (g.cells[:, 1] >> 8) & 0xFF, (g.cells[:, 1] >> 16) & 0xFF], axis=1)
    assert np.array_equal(mine, raw)


def test_leaf_rule_reference_defaults_plain_soup():
    sc = scenes.uniform_soup(65536, seed=0)
    g = _two_level(sc, 5.0, 1.2, 6, 2, 0)
    assert _same_two_level(g, _two_level(sc, 5.0, 1.2, 6, 2, oracle.REF_LEAF_POW))


def test_centres_heightfield():
    sc = scenes.heightfield_boxes(2048, 1024, nboxes=1000)
    g, d = _uniform(sc, 0), _uniform(sc, oracle.DIRECT_CENTRES)
    assert g.top_pairs.size == 10_747_835
    assert d.top_pairs.size == 10_747_834
    assert _pair_diff(g.top_pairs, d.top_pairs) == (1, 0)
