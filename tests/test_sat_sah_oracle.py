"""The oracle's precise (SAT) insertion and SAH resolution search, on the CPU.

* SAT (src/Control/Algorithm/BuildKernels.h:117-201): the plane test plus the
  nine edge-cross-axis tests.  Every pair it keeps the plane rule keeps too,
  every triangle keeps at least one cell, and the pairs it drops are cells
  whose box a float64 separating-axis test also separates from the triangle
  by more than the tolerance.
* SAH (src/Control/Algorithm/SAHGridBuilder.h:117-202): the refs of every
  tested resolution equal a numpy float32 restatement of countRefs'
  arithmetic, and the chosen resolution is the first least-cost one.
"""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

EPS = np.float32(1e-5)


def _sat_scene():
    return scenes.uniform_soup(2000, seed=11, offset_scale=0.2)


def test_sat_pairs_are_a_subset_of_the_plane_pairs():
    sc = _sat_scene()
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 5.0)
    plane = oracle.build_uniform(sc.vertices, sc.indices, b, res)
    sat = oracle.build_uniform(sc.vertices, sc.indices, b, res, insertion=1)
    ps, ss = set(plane.top_pairs.tolist()), set(sat.top_pairs.tolist())
    assert ss <= ps
    assert len(ss) < len(ps)  # large triangles: the edge tests cut cells
    tris = {p & 0xFFFFFFFF for p in ss}
    assert tris == set(range(sc.num_triangles))


def _overlap64(tri, centre, half):
    """Float64 triangle/box overlap with a relative margin (Akenine-Moller axes)."""
    v = tri.astype(np.float64) - centre
    e = [v[1] - v[0], v[2] - v[1], v[0] - v[2]]
    axes = [np.eye(3)[i] for i in range(3)] + [np.cross(e[0], e[1])]
    axes += [np.cross(np.eye(3)[i], ed) for ed in e for i in range(3)]
    for a in axes:
        if not np.any(a):
            continue
        p = v @ a
        r = np.abs(a) @ half
        tol = 1e-4 * (np.abs(a).sum() * (np.abs(v).max() + half.max()))
        if p.min() > r + tol or p.max() < -r - tol:
            return False
    return True


def test_sat_drops_only_separated_cells():
    sc = _sat_scene()
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 5.0)
    plane = oracle.build_uniform(sc.vertices, sc.indices, b, res)
    sat = oracle.build_uniform(sc.vertices, sc.indices, b, res, insertion=1)
    dropped = sorted(set(plane.top_pairs.tolist()) - set(sat.top_pairs.tolist()))
    cs = (b[3:].astype(np.float64) - b[:3]) / res
    tri = sc.vertices[sc.indices]
    rng = np.random.default_rng(0)
    for p in rng.choice(len(dropped), size=min(400, len(dropped)), replace=False):
        c, t = dropped[p] >> 32, dropped[p] & 0xFFFFFFFF
        x, y, z = c % res[0], (c // res[0]) % res[1], c // (res[0] * res[1])
        centre = b[:3] + (np.array([x, y, z]) + 0.5) * cs
        assert not _overlap64(tri[t], centre, cs / 2), (t, (x, y, z))


def _refs_numpy(sc, b, res):
    tri = sc.vertices[sc.indices]
    bmin, bmax = tri.min(1), tri.max(1)
    g0 = b[:3]
    out = np.ones(sc.num_triangles, np.uint64)
    for a in range(3):
        r = np.float32(res[a])
        cs = np.float32((b[3 + a] - b[a]) / r)
        rcp = np.float32(np.float32(1) / cs)
        mn = np.maximum(np.float32(0), (bmin[:, a] - g0[a]) * rcp + (-EPS)).astype(np.float32)
        mx = np.minimum(r - np.float32(1), (bmax[:, a] - g0[a]) * rcp + EPS).astype(np.float32)
        lo, hi = mn.astype(np.uint32), mx.astype(np.uint32)
        out *= np.where(hi >= lo, hi - lo + 1, 0).astype(np.uint64)
    return int(out.sum())


@pytest.mark.parametrize("n,seed,scale", [(300, 1, 0.05), (1500, 2, 0.2)])
def test_sah_counts_match_countrefs_arithmetic(n, seed, scale):
    sc = scenes.uniform_soup(n, seed=seed, offset_scale=scale)
    b = oracle.bounds(sc.vertices, sc.indices)
    r = oracle.sah_resolution(sc.vertices, sc.indices, b)
    lo, hi = np.array(r["res_min"]), np.array(r["res_max"])
    cnt = r["counts"]
    assert cnt.shape == tuple((hi - lo + 1)[::-1])
    rng = np.random.default_rng(seed)
    for _ in range(12):
        res = [int(rng.integers(lo[a], hi[a] + 1)) for a in range(3)]
        assert cnt[res[2] - lo[2], res[1] - lo[1], res[0] - lo[0]] == _refs_numpy(sc, b, res)
    # the first least cost in z, y, x order
    costs = np.array([[[oracle.sah_cost(sc.vertices, sc.indices, b, (x, y, z))[1]
                        for x in range(lo[0], hi[0] + 1)] for y in range(lo[1], hi[1] + 1)]
                      for z in range(lo[2], hi[2] + 1)], np.float32)
    k = int(np.argmin(costs.ravel()))
    best = np.unravel_index(k, costs.shape)
    assert r["res"] == (lo[0] + best[2], lo[1] + best[1], lo[2] + best[0])
    assert np.float32(r["cost"]) == costs.ravel()[k]


def test_sah_window_brackets_the_lambda_estimate():
    sc = scenes.uniform_soup(5000, seed=3)
    b = oracle.bounds(sc.vertices, sc.indices)
    est = oracle.resolution(sc.num_triangles, b, 5.0)
    lo, hi = oracle.sah_window(sc.num_triangles, b)
    assert np.all(lo <= est) and np.all(est <= hi)
    assert np.all(lo >= 1) and np.all(hi <= 2048)
