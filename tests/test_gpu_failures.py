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


def test_forced_timeout_inside_compact_is_reported_and_context_survives(gpu):
    """shn_compact_u32 with its first tile withheld: the other tiles' bounded
    look-back waits run out, shn_ctx_sync_status reports SHN_ERR_TIMEOUT, and
    the next compaction on the same context is correct and clean."""
    import torch

    import shinobi_b200 as shn
    ctx = shn.Context(0)
    rng = np.random.default_rng(5)
    f = (rng.random(100_000) < 0.3).astype(np.uint32)
    d = torch.from_numpy(f.view(np.int32)).cuda()
    assert ctx.lib.shn_debug_force_lookback_timeout(shn._abi.SHN_FORCE_CTX_SCAN, ctx.handle, None) == 0
    shn.compact(d, ctx=ctx)
    with pytest.raises(shn.ShinobiError) as e:
        ctx.sync_status()
    assert e.value.status == shn._abi.SHN_ERR_TIMEOUT
    out = shn.compact(d, ctx=ctx)
    ctx.sync_status()                       # cleared by the report above
    assert np.array_equal(out.cpu().numpy().view(np.uint32), oracle.compact(f))
    ctx.close()


def test_forced_timeout_inside_ao_compaction_is_reported_and_grid_survives(gpu):
    """The hit compaction of shn_trace_ao with its first tile withheld:
    shn_grid_sync_status reports SHN_ERR_TIMEOUT (no access left the
    buffers), and the next AO call on the same grid matches the oracle."""
    import shinobi_b200 as shn
    ctx = shn.default_context()
    sc = scenes.cluster_in_field(32768, seed=1)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 1.0 / 16.0, 1, 2)
    g = shn.Grid().build(soup, shn.grid_params(shn.SHN_GRID_TWO_LEVEL, lambda_=1.0 / 16.0, top_divisor=1,
                                               min_res=2, lambda_leaf=4.0, res=res))
    cam = scenes.Camera((0.0, 0.0, -0.25), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 256, 144)
    h = g.trace_primary(cam)
    g.sync_status()
    assert ctx.lib.shn_debug_force_lookback_timeout(shn._abi.SHN_FORCE_GRID_COMPACTION, None, g.handle) == 0
    g.trace_ao(cam, h, spp=4, length=0.1, offset=1e-4, seed=1)
    with pytest.raises(shn.ShinobiError) as e:
        g.sync_status()
    assert e.value.status == shn._abi.SHN_ERR_TIMEOUT
    ao = g.trace_ao(cam, h, spp=4, length=0.1, offset=1e-4, seed=1)
    g.sync_status()
    og = oracle.build_two_level(sc.vertices, sc.indices, b, res, 4.0, 16)
    org, d = oracle.primary_rays(cam)
    rt, rtt, _, _, _ = oracle.trace_closest(og, org, d)
    ro, rd, rpix = oracle.ao_rays(sc.vertices, sc.indices, org, d, rt, rtt, 4, 1, 1e-4)
    occ, _ = oracle.trace_any(og, ro, rd, np.full(ro.shape[0], 0.1, np.float32))
    cnt = np.zeros(org.shape[0], np.int64)
    np.add.at(cnt, rpix, occ.astype(np.int64))
    ref = np.where(rt == shn.SHN_MISS, np.float32(1.0),
                   np.float32(1.0) - cnt.astype(np.float32) / np.float32(4.0)).astype(np.float32)
    assert np.array_equal(ao.cpu().numpy(), ref)


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
