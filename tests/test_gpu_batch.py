"""Batched multi-scene build/trace (one fused pipeline, one launch) against the
oracle built scene by scene; CUDA-graph replay; measured lambda autotuner."""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu


def _scenes():
    out = []
    for i, (n, s) in enumerate([(1000, 0.05), (4000, 0.001), (20000, 0.01), (1, 0.02), (7000, 0.03), (60000, 0.004)]):
        out.append(scenes.uniform_soup(n, seed=100 + i, offset_scale=s))
    return out


def _rays(counts, seed):
    orgs, dirs = [], []
    for i, c in enumerate(counts):
        o, d = scenes.random_rays(c, seed=seed, stream=i)
        orgs.append(o)
        dirs.append(d)
    off = np.concatenate([[0], np.cumsum(counts)]).astype(np.uint32)
    return np.concatenate(orgs), np.concatenate(dirs), off


def _oracle_grids(scs, lambdas):
    grids = []
    for sc, lam in zip(scs, lambdas):
        b = oracle.bounds(sc.vertices, sc.indices)
        res = oracle.resolution(sc.num_triangles, b, float(lam))
        grids.append(oracle.build_uniform(sc.vertices, sc.indices, b, res))
    return grids


def test_batch_build_matches_per_scene_oracle(gpu):
    import shinobi_b200 as shn
    scs = _scenes()
    lam = np.array([5, 3, 2, 5, 8, 1.5], np.float32)
    bt = shn.Batch(scs)
    bt.set_lambdas(lam)
    bt.build()
    for s, og in enumerate(_oracle_grids(scs, lam)):
        ex = bt.export_scene(s, og.cells.shape[0], og.indices.size)
        assert np.array_equal(ex["res"], og.res)
        assert np.array_equal(ex["cells"], og.cells), f"scene {s} cells"
        assert np.array_equal(ex["indices"], og.indices), f"scene {s} indices"


def test_batch_trace_matches_oracle_and_graph_replay(gpu):
    import torch

    import shinobi_b200 as shn
    scs = _scenes()
    lam = np.full(len(scs), 5.0, np.float32)
    bt = shn.Batch(scs)
    bt.set_lambdas(lam)
    bt.build()
    counts = [3000, 5000, 1, 2000, 8000, 4000]
    org, d, off = _rays(counts, seed=3)
    torg, td = torch.from_numpy(org).cuda(), torch.from_numpy(d).cuda()
    h = bt.trace(torg, td, off)
    tri = h.tri.cpu().numpy().view(np.uint32)
    t = h.t.cpu().numpy()
    for s, og in enumerate(_oracle_grids(scs, lam)):
        a, b = off[s], off[s + 1]
        rt, rtt, _, _, _ = oracle.trace_closest(og, org[a:b], d[a:b])
        assert np.array_equal(tri[a:b], rt), f"scene {s}"
        assert np.array_equal(t[a:b].view(np.uint32), rtt.view(np.uint32))
    occ = bt.trace(torg, td, off, tmax=torch.full((org.shape[0],), 0.5, device="cuda"), any_hit=True)
    occ = occ.cpu().numpy()
    for s, og in enumerate(_oracle_grids(scs, lam)):
        a, b = off[s], off[s + 1]
        ro, _ = oracle.trace_any(og, org[a:b], d[a:b], np.full(b - a, 0.5, np.float32))
        assert np.array_equal(occ[a:b], ro)
    # graph: build + trace captured once, replayed twice
    out = shn.alloc_hits(org.shape[0])
    bt.capture(torg, td, off, out)
    for _ in range(2):
        out.tri.fill_(-7)
        bt.replay()
        torch.cuda.synchronize()
        assert np.array_equal(out.tri.cpu().numpy().view(np.uint32), tri)
        assert np.array_equal(out.t.cpu().numpy().view(np.uint32), t.view(np.uint32))


def test_batch_autotune_picks_candidates(gpu):
    import shinobi_b200 as shn
    scs = _scenes()[:4]
    bt = shn.Batch(scs)
    cands = np.array([1.0, 3.0, 8.0], np.float32)
    chosen = bt.autotune(cands, expected_rays=[100000] * 4, sample_rays=8192)
    assert set(chosen.tolist()) <= set(cands.tolist())
    bt.build()
    for s, og in enumerate(_oracle_grids(scs, chosen)):
        ex = bt.export_scene(s, og.cells.shape[0], og.indices.size)
        assert np.array_equal(ex["cells"], og.cells)


def test_batch_autotune_sah_and_block_shapes(gpu):
    import shinobi_b200 as shn
    scs = _scenes()[:4]
    bt = shn.Batch(scs)
    cands = np.array([0.5, 1.0, 3.0, 8.0], np.float32)
    chosen, sah, rep = bt.autotune_ex(cands, expected_rays=[100000] * 4, sample_rays=8192, sah_keep=2,
                                      blocks_per_sm=(0, 4, 6), sort_tiles=(6144, 4096))
    assert set(chosen.tolist()) <= set(cands.tolist())
    nonempty = sum(1 for sc in scs if sc.num_triangles)
    assert rep["timed_candidates"] == 2 * nonempty
    assert rep["blocks_per_sm"] in (0, 4, 6) and all(ms > 0 for ms in rep["shape_ms"])
    assert rep["sort_tile_keys"] in (4096, 6144) and all(ms > 0 for ms in rep["sort_tile_ms"])
    # the chosen candidate is one of the two of least SAH cost, and its cost is the oracle's
    for s, sc in enumerate(scs):
        if not sc.num_triangles:
            continue
        b = oracle.bounds(sc.vertices, sc.indices)
        costs = [oracle.sah_cost(sc.vertices, sc.indices, b, oracle.resolution(sc.num_triangles, b, float(l)))[1]
                 for l in cands]
        kept = np.argsort(np.array(costs, np.float32), kind="stable")[:2]
        assert chosen[s] in cands[kept]
        assert np.float32(sah[s]) == np.float32(costs[int(np.where(cands == chosen[s])[0][0])])
    bt.build()
    for s, og in enumerate(_oracle_grids(scs, chosen)):
        ex = bt.export_scene(s, og.cells.shape[0], og.indices.size)
        assert np.array_equal(ex["cells"], og.cells)


def test_batch_build_with_4096_key_sort_tiles(gpu):
    """The autotuner's other onesweep tile shape gives the same grids."""
    import shinobi_b200 as shn
    scs = _scenes()
    bt = shn.Batch(scs)
    cands = np.array([1.5], np.float32)
    chosen, _, rep = bt.autotune_ex(cands, expected_rays=[100000] * len(scs), sample_rays=4096,
                                    sort_tiles=(4096,))
    assert rep["sort_tile_keys"] == 4096
    bt.build()
    for s, og in enumerate(_oracle_grids(scs, chosen)):
        ex = bt.export_scene(s, og.cells.shape[0], og.indices.size)
        assert np.array_equal(ex["cells"], og.cells)
        assert np.array_equal(ex["indices"], og.indices)
