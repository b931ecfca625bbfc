"""SAT insertion and the SAH resolution search on the GPU against the oracle.

Grids built with SHN_INSERT_SAT must equal oracle.build_uniform /
build_two_level with insertion=1 bit for bit; the SAH search must return the
oracle's counts for every tested resolution, and the same resolution, cost
and refs.
"""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu


def _grid_equal(g, og):
    ex = g.export()
    assert np.array_equal(ex["res"], og.res)
    assert np.array_equal(ex["top_pairs"], og.top_pairs), "sorted pairs differ"
    assert np.array_equal(ex["cells"], og.cells), "cells differ"
    assert np.array_equal(ex["indices"], og.indices), "indices differ"
    if og.kind == 1:
        assert np.array_equal(ex["leaves"], og.leaves), "leaves differ"


@pytest.mark.parametrize("n,seed,scale", [(1, 2, 0.3), (2000, 11, 0.2), (65536, 0, 0.05)])
def test_uniform_sat(gpu, n, seed, scale):
    import shinobi_b200 as shn
    sc = scenes.uniform_soup(n, seed=seed, offset_scale=scale)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 5.0)
    g = shn.Grid().build(soup, shn.grid_params(shn.SHN_GRID_UNIFORM, res=res, insertion=shn.SHN_INSERT_SAT))
    og = oracle.build_uniform(sc.vertices, sc.indices, b, res, insertion=1)
    _grid_equal(g, og)
    plane = shn.Grid().build(soup, shn.grid_params(shn.SHN_GRID_UNIFORM, res=res))
    assert g.info().num_refs <= plane.info().num_refs


def test_two_level_sat_top(gpu):
    import shinobi_b200 as shn
    sc = scenes.cluster_in_field(131072, seed=1)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 1.0 / 16.0)
    p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL, lambda_=1.0 / 16.0, lambda_leaf=4.0, res=res,
                        insertion=shn.SHN_INSERT_SAT)
    g = shn.Grid().build(soup, p)
    og = oracle.build_two_level(sc.vertices, sc.indices, b, res, 4.0, 16, insertion=1)
    _grid_equal(g, og)


@pytest.mark.parametrize("n,seed,scale", [(300, 1, 0.05), (20000, 4, 0.02)])
def test_sah_resolution(gpu, n, seed, scale):
    import shinobi_b200 as shn
    sc = scenes.uniform_soup(n, seed=seed, offset_scale=scale)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    got = soup.sah_resolution(5.0, counts=True)
    want = oracle.sah_resolution(sc.vertices, sc.indices, b)
    assert got["res_min"] == want["res_min"] and got["res_max"] == want["res_max"]
    assert np.array_equal(got["counts"], want["counts"])
    assert got["res"] == want["res"]
    assert got["refs"] == want["refs"]
    assert np.float32(got["cost"]) == np.float32(want["cost"])
    assert got["num_tested"] == want["counts"].size


def test_sah_cost_list(gpu):
    import shinobi_b200 as shn
    sc = scenes.cluster_in_field(50000, seed=2)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    cands = [oracle.resolution(sc.num_triangles, b, lam) for lam in (0.5, 1.0, 2.0, 5.0, 9.0)]
    cands.append(np.array([1, 1, 1], np.int32))
    refs, cost = soup.sah_cost(np.stack(cands))
    for i, r in enumerate(cands):
        wr, wc = oracle.sah_cost(sc.vertices, sc.indices, b, r)
        assert int(refs[i]) == wr
        assert np.float32(cost[i]) == np.float32(wc)
    assert int(refs[-1]) == sc.num_triangles
