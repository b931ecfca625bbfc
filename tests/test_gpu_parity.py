"""Parity of the CUDA path (through the C ABI) against the oracle.

Grids (cell ranges, cell words, leaf ranges, sorted pair arrays, indices[])
must be bit-exact; closest-hit triangle ids, t, u, v and any-hit flags are
compared exactly as well (both sides evaluate the same IEEE operations in the
same order; the library is built with -fmad=false).  t is additionally
checked against an FP64 evaluation with a 1e-5 relative tolerance.
"""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu

T_REL_TOL = 1e-5


def _torch():
    import torch
    return torch


def build_both(shn, sc, kind, lam, divisor=1, min_res=1, lam_leaf=1.2, thr=16, res=None):
    torch = _torch()
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    assert np.array_equal(soup.bounds.view(np.uint32), b.view(np.uint32))
    if res is None:
        res = oracle.resolution(sc.num_triangles, b, lam, divisor, min_res)
    p = shn.grid_params(kind, lambda_=lam, top_divisor=divisor, min_res=min_res,
                        lambda_leaf=lam_leaf, leaf_threshold=thr, res=res)
    g = shn.Grid().build(soup, p)
    torch.cuda.synchronize()
    if kind == shn.SHN_GRID_UNIFORM:
        og = oracle.build_uniform(sc.vertices, sc.indices, b, res)
    else:
        og = oracle.build_two_level(sc.vertices, sc.indices, b, res, lam_leaf, thr)
    return soup, g, og


def assert_grid_equal(shn, g, og):
    ex = g.export()
    assert np.array_equal(ex["res"], og.res)
    assert np.array_equal(ex["cells"], og.cells), "cells differ"
    assert np.array_equal(ex["indices"], og.indices), "indices differ"
    assert np.array_equal(ex["top_pairs"], og.top_pairs), "sorted pairs differ"
    if og.kind == 1:
        assert np.array_equal(ex["leaves"], og.leaves), "leaves differ"


def test_uniform_build_soup(gpu):
    import shinobi_b200 as shn
    sc = scenes.uniform_soup(65536, seed=0)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_UNIFORM, 5.0)
    assert_grid_equal(shn, g, og)


@pytest.mark.parametrize("n,seed,scale", [(1, 3, 0.01), (7, 4, 0.2), (3000, 5, 0.05), (20000, 6, 0.002)])
def test_uniform_build_ragged(gpu, n, seed, scale):
    import shinobi_b200 as shn
    sc = scenes.uniform_soup(n, seed=seed, offset_scale=scale)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_UNIFORM, 5.0)
    assert_grid_equal(shn, g, og)


def test_two_level_build_cluster(gpu):
    import shinobi_b200 as shn
    sc = scenes.cluster_in_field(131072, seed=1)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_TWO_LEVEL, 1.0 / 16.0, lam_leaf=4.0)
    assert_grid_equal(shn, g, og)


def test_two_level_build_reference_defaults(gpu):
    import shinobi_b200 as shn
    sc = scenes.uniform_soup(65536, seed=0)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_TWO_LEVEL, 5.0, divisor=6, min_res=2, lam_leaf=1.2)
    assert_grid_equal(shn, g, og)


def _check_hits(h, ref_tri, ref_t, ref_u, ref_v):
    tri = h.tri.cpu().numpy().view(np.uint32)
    t = h.t.cpu().numpy()
    u = h.u.cpu().numpy()
    v = h.v.cpu().numpy()
    assert np.array_equal(tri, ref_tri), f"{np.count_nonzero(tri != ref_tri)} tri mismatches"
    assert np.array_equal(t.view(np.uint32), ref_t.view(np.uint32))
    assert np.array_equal(u.view(np.uint32), ref_u.view(np.uint32))
    assert np.array_equal(v.view(np.uint32), ref_v.view(np.uint32))
    return tri, t


def test_trace_primary_uniform(gpu):
    import shinobi_b200 as shn
    sc = scenes.uniform_soup(65536, seed=0)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_UNIFORM, 5.0)
    cam = scenes.CAMERA_SOUP
    h = g.trace_primary(cam)
    org, d = oracle.primary_rays(cam)
    rt, rtt, ru, rv, _ = oracle.trace_closest(og, org, d)
    tri, t = _check_hits(h, rt, rtt, ru, rv)
    hit = tri != shn.SHN_MISS
    assert hit.sum() > 50000
    t64 = oracle.t_fp64(sc.vertices, sc.indices, tri, org, d)
    rel = np.abs(t[hit] - t64[hit]) / np.abs(t64[hit])
    assert rel.max() < T_REL_TOL


def test_trace_primary_two_level(gpu):
    import shinobi_b200 as shn
    sc = scenes.cluster_in_field(131072, seed=1)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_TWO_LEVEL, 1.0 / 16.0, lam_leaf=4.0)
    cam = scenes.Camera((0.0, 0.0, -0.25), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 320, 180)
    h = g.trace_primary(cam)
    org, d = oracle.primary_rays(cam)
    rt, rtt, ru, rv, _ = oracle.trace_closest(og, org, d)
    _check_hits(h, rt, rtt, ru, rv)


def test_trace_soa_closest_and_any(gpu):
    import shinobi_b200 as shn
    torch = _torch()
    sc = scenes.uniform_soup(20000, seed=7, offset_scale=0.03)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_UNIFORM, 5.0)
    org, d = scenes.random_rays(50000, seed=8)
    tmax = np.full(50000, 0.7, np.float32)
    h = g.trace_closest(torch.from_numpy(org).cuda(), torch.from_numpy(d).cuda(),
                        torch.from_numpy(tmax).cuda())
    rt, rtt, ru, rv, _ = oracle.trace_closest(og, org, d, tmax)
    _check_hits(h, rt, rtt, ru, rv)
    occ = g.trace_any(torch.from_numpy(org).cuda(), torch.from_numpy(d).cuda(),
                      torch.from_numpy(tmax).cuda())
    ro, _ = oracle.trace_any(og, org, d, tmax)
    assert np.array_equal(occ.cpu().numpy(), ro)
    assert np.array_equal(ro.astype(bool), rt != shn.SHN_MISS)


def test_ao_two_level(gpu):
    import shinobi_b200 as shn
    torch = _torch()
    sc = scenes.cluster_in_field(131072, seed=1)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_TWO_LEVEL, 1.0 / 16.0, lam_leaf=4.0)
    cam = scenes.Camera((0.0, 0.0, -0.25), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 256, 144)
    h = g.trace_primary(cam)
    nrays = torch.zeros(1, dtype=torch.int32, device="cuda")
    ao = g.trace_ao(cam, h, spp=4, length=0.1, offset=1e-4, seed=1, num_rays=nrays)
    org, d = oracle.primary_rays(cam)
    rt, rtt, _, _, _ = oracle.trace_closest(og, org, d)
    ro, rd, rpix = oracle.ao_rays(sc.vertices, sc.indices, org, d, rt, rtt, 4, 1, 1e-4)
    occ, _ = oracle.trace_any(og, ro, rd, np.full(ro.shape[0], 0.1, np.float32))
    assert int(nrays.item()) == ro.shape[0]
    cnt = np.zeros(org.shape[0], np.int64)
    np.add.at(cnt, rpix, occ.astype(np.int64))
    ref = np.where(rt == shn.SHN_MISS, np.float32(1.0),
                   (np.float32(1.0) - cnt.astype(np.float32) / np.float32(4.0)).astype(np.float32))
    got = ao.cpu().numpy()
    assert np.array_equal(got, ref.astype(np.float32))
    assert occ.mean() > 0.05


@pytest.mark.parametrize("n", [0, 1, 2047, 2048, 2049, 100003, 3_000_000])
def test_exclusive_scan(gpu, n):
    import shinobi_b200 as shn
    torch = _torch()
    rng = np.random.default_rng(n)
    x = rng.integers(0, 50, size=n, dtype=np.uint32)
    out = shn.exclusive_scan(torch.from_numpy(x.view(np.int32)).cuda()).cpu().numpy().view(np.uint32)
    ref = np.concatenate([[0], np.cumsum(x, dtype=np.uint64)]).astype(np.uint32)
    assert np.array_equal(out, ref)


@pytest.mark.parametrize("n", [0, 1, 5000, 1_000_001])
def test_compact(gpu, n):
    import shinobi_b200 as shn
    torch = _torch()
    rng = np.random.default_rng(n + 1)
    f = (rng.random(n) < 0.3).astype(np.uint32)
    out = shn.compact(torch.from_numpy(f.view(np.int32)).cuda()).cpu().numpy().view(np.uint32)
    assert np.array_equal(out, oracle.compact(f))


@pytest.mark.parametrize("n,bits", [(1, 8), (4095, 8), (4096, 16), (4097, 19), (1_000_000, 22),
                                    (3_000_001, 32), (8191, 9), (8193, 17), (100_000, 18), (2_000_000, 25),
                                    (700_001, 26), (5_000_000, 27)])
def test_sort_keys(gpu, n, bits):
    """Stable sort on bits [32, 32 + bits) (8- or 9-bit digit passes, the
    last one narrower when bits is not a multiple of the width); the bits
    above the range are random and must not change the order."""
    import shinobi_b200 as shn
    torch = _torch()
    rng = np.random.default_rng(bits)
    field = rng.integers(0, 1 << bits, size=n, dtype=np.uint64)
    above = rng.integers(0, 1 << (32 - bits), size=n, dtype=np.uint64) if bits < 32 else np.zeros(n, np.uint64)
    lo = np.arange(n, dtype=np.uint64)
    keys = (((above << np.uint64(bits)) | field) << np.uint64(32)) | lo
    t = torch.from_numpy(keys.view(np.int64)).cuda()
    shn.sort_keys(t, 32, 32 + bits)
    shn.default_context().sync_status()
    got = t.cpu().numpy().view(np.uint64)
    assert np.array_equal(got, keys[np.argsort(field, kind="stable")])


@pytest.mark.parametrize("case", [0, 1, 2])
def test_builds_match_reference_hostbuild_fixture(gpu, case):
    """The CUDA uniform and two-level builds against the grids the reference's
    own TwoLevelGridBuilderHost::hostBuild produced (tests/golden), with
    empty ranges canonicalised to [0, 0]."""
    import os
    import shinobi_b200 as shn
    z = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "hostbuild_uniform.npz"))
    vtx, idx, res = (z[f"c{case}_{n}"] for n in ("vertices", "indices", "res"))

    def canon(r):
        r = r.copy()
        r[r[:, 0] == r[:, 1]] = 0
        return r

    soup = shn.FaceSoup(vtx, idx)
    assert np.array_equal(soup.bounds.view(np.uint32), z[f"c{case}_bounds"].view(np.uint32))
    g = shn.Grid().build(soup, shn.grid_params(shn.SHN_GRID_UNIFORM, res=res))
    ex = g.export()
    assert np.array_equal(canon(ex["cells"]), canon(z[f"c{case}_leaves"]))
    assert np.array_equal(ex["indices"], z[f"c{case}_refs"])
    g2 = shn.Grid().build(soup, shn.grid_params(shn.SHN_GRID_TWO_LEVEL, lambda_leaf=4.0, leaf_threshold=16, res=res))
    ex2 = g2.export()
    assert np.array_equal(ex2["cells"], z[f"c{case}_cellwords"])
    assert np.array_equal(canon(ex2["leaves"]), canon(z[f"c{case}_leaves"]))
    assert np.array_equal(ex2["indices"], z[f"c{case}_refs"])
