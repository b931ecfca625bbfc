"""Failure detection without a GPU fault: bounded device waits that run out
report SHN_ERR_TIMEOUT and leave the context usable; invalid inputs, unbuilt
grids and budget overruns are refused on the host with a status."""
import ctypes as C

import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu


def test_bounded_lookback_wait_reports_timeout_and_context_survives(gpu):
    import torch

    import shinobi_b200 as shn
    ctx = shn.Context(0)
    rc = ctx.lib.shn_selftest_lookback_timeout(ctx.handle, None)
    assert rc == shn._abi.SHN_ERR_TIMEOUT
    # the context still works: a scan right after gives the right answer
    x = torch.arange(5000, dtype=torch.int32, device="cuda")
    out = shn.exclusive_scan(x, ctx=ctx)
    ref = np.concatenate([[0], np.cumsum(np.arange(5000, dtype=np.int64))])
    assert np.array_equal(out.cpu().numpy().astype(np.int64), ref)
    ctx.close()


def test_invalid_scene_inputs_are_refused(gpu):
    import shinobi_b200 as shn
    v = np.random.default_rng(0).random((30, 3), dtype=np.float32)
    idx = np.arange(30, dtype=np.uint32).reshape(10, 3)
    bad_v = v.copy()
    bad_v[4, 1] = np.nan
    with pytest.raises(shn.ShinobiError) as e:
        shn.FaceSoup(bad_v, idx)
    assert e.value.status == shn._abi.SHN_ERR_INVALID
    bad_i = idx.copy()
    bad_i[3, 2] = 30
    with pytest.raises(shn.ShinobiError) as e:
        shn.FaceSoup(v, bad_i)
    assert e.value.status == shn._abi.SHN_ERR_INVALID


def test_rejected_vertex_update_leaves_the_scene_unchanged(gpu):
    """Host vertices are checked on the device before they replace the
    scene's: an update holding inf/NaN is refused and the scene still builds
    the same grid as before."""
    import shinobi_b200 as shn
    sc = scenes.uniform_soup(2000, seed=4)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    p = shn.grid_params(shn.SHN_GRID_UNIFORM, lambda_=5.0)
    before = shn.Grid().build(soup, p).export()
    for bad in (np.nan, np.inf):
        v = sc.vertices.copy()
        v[17, 2] = bad
        with pytest.raises(shn.ShinobiError) as e:
            soup.update_vertices(v)
        assert e.value.status == shn._abi.SHN_ERR_INVALID
    after = shn.Grid().build(soup, p).export()
    for k in ("cells", "indices", "top_pairs"):
        assert np.array_equal(before[k], after[k]), k
    moved = sc.vertices * np.float32(1.5)
    soup.update_vertices(moved)                 # a valid update still goes through
    assert np.allclose(soup.bounds[3:], oracle.bounds(moved, sc.indices)[3:])


def test_trace_before_build_is_refused(gpu):
    import shinobi_b200 as shn
    g = shn.Grid()
    cam = scenes.Camera((0.5, 0.5, -1.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 16, 16)
    with pytest.raises(shn.ShinobiError) as e:
        g.trace_primary(cam)
    assert e.value.status == shn._abi.SHN_ERR_NOT_BUILT


def test_build_over_budget_is_refused_and_context_survives(gpu):
    import shinobi_b200 as shn
    ctx = shn.Context(0, hbm_budget_bytes=8 << 20)
    sc = scenes.uniform_soup(1 << 18, seed=3)
    with pytest.raises(shn.ShinobiError) as e:
        soup = shn.FaceSoup(sc.vertices, sc.indices, ctx=ctx)
        shn.Grid(ctx).build(soup, shn.grid_params(shn.SHN_GRID_UNIFORM))
    assert e.value.status == shn._abi.SHN_ERR_BUDGET
    used, budget = ctx.memory()
    assert used <= budget
    small = scenes.uniform_soup(500, seed=4)
    soup = shn.FaceSoup(small.vertices, small.indices, ctx=ctx)
    g = shn.Grid(ctx).build(soup, shn.grid_params(shn.SHN_GRID_UNIFORM))
    assert g.info().num_refs > 0
    ctx.close()
