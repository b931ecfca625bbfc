"""Parity at the full sizes of the benchmarked workloads.

* Cluster in a field (the headline step): the 1,048,576-triangle scene, the
  two-level grid with top lambda 1/16 and leaf lambda 4 -- cell words, leaf
  ranges, indices[] and sorted top pairs bit-exact -- then the 1920x1080
  primary closest hits and 4 ambient-occlusion rays per hit, compared on every
  16th pixel of the frame (tri, t, u, v and the AO value bit-exact).
* Heightfield path tracer: the 4,206,304-triangle heightfield + boxes, the
  uniform grid at lambda 5 bit-exact, and the 1920x1080 x 16 spp render
  compared on a spread of pixels (bit-exact, RMSE stated).
* Batched scenes: all 256 scenes of the batched workload (about 63M
  triangles) built by one fused pipeline; 256 random rays per scene through
  the single batched trace launch against each scene's oracle grid, and the
  grids of every 16th scene bit-exact.

The oracle traces run on the host cores; the samples are sized so that each
test finishes in well under a minute there.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu

AO_SPP, AO_LEN, AO_OFFSET, AO_SEED = 4, 0.1, 1e-4, 1
RMSE_TOL = 1e-6
PT_LIGHT = dict(light_pos=(0.3, 0.3, 1.0), light_e1=(0.0, 0.4, 0.0), light_e2=(0.4, 0.0, 0.0),
                light_radiance=(20.0, 20.0, 20.0), background=(0.15, 0.2, 0.3))


def _mismatch(a, b):
    return int(np.count_nonzero(np.asarray(a) != np.asarray(b)))


def test_cluster_headline_full_size(gpu):
    import shinobi_b200 as shn
    oracle.set_threads(os.cpu_count() or 1)
    sc = scenes.cluster_in_field(1 << 20, seed=1)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 1.0 / 16.0, 1, 2)
    p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL, lambda_=1.0 / 16.0, top_divisor=1, min_res=2,
                        lambda_leaf=4.0, leaf_threshold=16)
    g = shn.Grid().build(soup, p)
    og = oracle.build_two_level(sc.vertices, sc.indices, b, res, 4.0, 16)
    ex = g.export()
    assert np.array_equal(ex["res"], og.res)
    for k in ("cells", "leaves", "indices", "top_pairs"):
        assert ex[k].shape == getattr(og, k).shape, k
        assert np.array_equal(ex[k], getattr(og, k)), f"{k}: {_mismatch(ex[k], getattr(og, k))} words differ"

    cam = scenes.CAMERA_CLUSTER
    h = g.trace_primary(cam)
    ao = g.trace_ao(cam, h, AO_SPP, AO_LEN, AO_OFFSET, AO_SEED)
    g.sync_status()
    org, d = oracle.primary_rays(cam)
    sel = np.arange(0, org.shape[0], 16, dtype=np.int64)
    rt, rtt, ru, rv, _ = oracle.trace_closest(og, org[sel], d[sel])
    tri = h.tri.cpu().numpy().view(np.uint32)[sel]
    assert np.array_equal(tri, rt), f"{_mismatch(tri, rt)} of {sel.size} primary hits differ"
    for got, ref in ((h.t, rtt), (h.u, ru), (h.v, rv)):
        g_ = got.cpu().numpy()[sel]
        assert np.array_equal(g_.view(np.uint32), ref.view(np.uint32))
    hit = rt != shn.SHN_MISS
    assert hit.sum() > sel.size // 4
    t64 = oracle.t_fp64(sc.vertices, sc.indices, rt, org[sel], d[sel])
    assert (np.abs(rtt[hit] - t64[hit]) / np.abs(t64[hit])).max() < 1e-5
    ro, rd, rpix = oracle.ao_rays(sc.vertices, sc.indices, org[sel], d[sel], rt, rtt, AO_SPP, AO_SEED,
                                  AO_OFFSET, pix=sel)
    occ, _ = oracle.trace_any(og, ro, rd, np.full(ro.shape[0], AO_LEN, np.float32))
    cnt = np.zeros(sel.size, np.int64)
    np.add.at(cnt, rpix, occ.astype(np.int64))
    ref = np.where(rt == shn.SHN_MISS, np.float32(1.0),
                   np.float32(1.0) - cnt.astype(np.float32) / np.float32(AO_SPP)).astype(np.float32)
    got = ao.cpu().numpy()[sel]
    assert np.array_equal(got, ref), f"{_mismatch(got, ref)} of {sel.size} AO values differ"
    assert 0.05 < occ.mean() < 0.95


def test_heightfield_path_tracer_full_size(gpu):
    import shinobi_b200 as shn
    oracle.set_threads(os.cpu_count() or 1)
    sc = scenes.heightfield_boxes(2048, 1024, nboxes=1000)
    assert sc.num_triangles == 4_206_304
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 5.0)
    g = shn.Grid().build(soup, shn.grid_params(shn.SHN_GRID_UNIFORM, lambda_=5.0))
    og = oracle.build_uniform(sc.vertices, sc.indices, b, res)
    ex = g.export()
    assert np.array_equal(ex["res"], og.res)
    for k in ("cells", "indices", "top_pairs"):
        assert np.array_equal(ex[k], getattr(og, k)), f"{k}: {_mismatch(ex[k], getattr(og, k))} words differ"
    del ex
    cam = scenes.CAMERA_HEIGHTFIELD
    params = shn.pt_params(spp=16, max_depth=4, rr_depth=2, albedo=0.7, offset=1e-4, seed=2, **PT_LIGHT)
    img = g.pt_render(soup, cam, params)
    g.sync_status()
    img = img.cpu().numpy().reshape(-1, 3)
    sel = np.arange(7, cam.res_x * cam.res_y, 211, dtype=np.uint32)
    ref = oracle.pt_render_pixels(og, cam, sel, 16, 4, 2, 0.7, PT_LIGHT["light_pos"], PT_LIGHT["light_e1"],
                                  PT_LIGHT["light_e2"], PT_LIGHT["light_radiance"], PT_LIGHT["background"],
                                  1e-4, 2)
    got = img[sel]
    rmse = float(np.sqrt(np.mean((got.astype(np.float64) - ref) ** 2)))
    assert rmse <= RMSE_TOL
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), f"{_mismatch(got, ref)} values differ"
    assert float(ref.mean()) > 0.0


def test_batched_256_scenes_full_size(gpu):
    import ctypes as C

    import torch

    import shinobi_b200 as shn
    ns = 256
    tris, scales, _ = scenes.batch_workload_sizes(ns)
    vs, ix = [], []
    for i in range(ns):
        v, t = scenes.uniform_soup_device(int(tris[i]), seed=1000 + i, offset_scale=float(scales[i]))
        vs.append(v)
        ix.append(t)
    vo = np.concatenate([[0], np.cumsum(3 * tris)]).astype(np.uint32)
    to = np.concatenate([[0], np.cumsum(tris)]).astype(np.uint32)
    V = torch.cat(vs)
    I = torch.cat(ix)
    del vs, ix
    ctx = shn.default_context()
    lib = ctx.lib
    h = C.c_void_p()
    ctx.check(lib.shn_batch_create(ctx.handle, ns, shn._ptr(V), vo.ctypes.data_as(C.c_void_p), shn._ptr(I),
                                   to.ctypes.data_as(C.c_void_p), shn.SHN_MEM_DEVICE, shn._stream(None),
                                   C.byref(h)), "shn_batch_create")
    bt = shn.Batch.__new__(shn.Batch)
    bt.ctx, bt.handle, bt.num_scenes, bt.tri_offsets = ctx, h, ns, to
    cands = np.array([0.5, 0.75, 1.0, 1.5, 2.0, 3.0], np.float32)
    lam = cands[np.random.default_rng(5).integers(0, cands.size, ns)]
    bt.set_lambdas(lam)
    bt.build()
    per = 256
    orgs, dirs = [], []
    for i in range(ns):
        o, d = scenes.random_rays_device(per, seed=77, stream=i)
        orgs.append(o)
        dirs.append(d)
    org = torch.cat(orgs)
    dr = torch.cat(dirs)
    ro = np.arange(0, (ns + 1) * per, per, dtype=np.uint32)
    hits = bt.trace(org, dr, ro)
    bt.sync_status()
    tri = hits.tri.cpu().numpy().view(np.uint32)
    tt = hits.t.cpu().numpy()
    org_h, dir_h = org.cpu().numpy(), dr.cpu().numpy()

    def check(s):
        oracle.set_threads(1)   # scenes run in parallel, one host thread each
        vh = V[vo[s]:vo[s + 1]].cpu().numpy()
        ih = I[to[s]:to[s + 1]].cpu().numpy().astype(np.uint32)   # local to the scene
        bb = oracle.bounds(vh, ih)
        res = oracle.resolution(int(tris[s]), bb, float(lam[s]))
        og = oracle.build_uniform(vh, ih, bb, res)
        a, b_ = ro[s], ro[s + 1]
        rt, rtt, _, _, _ = oracle.trace_closest(og, org_h[a:b_], dir_h[a:b_])
        bad = _mismatch(tri[a:b_], rt) + _mismatch(tt[a:b_].view(np.uint32), rtt.view(np.uint32))
        return s, bad, int((rt != shn.SHN_MISS).sum()), (og if s % 16 == 0 else None)

    workers = max(1, min(16, os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=workers) as pool:
        results = list(pool.map(check, range(ns)))
    bad = [(s, b_) for s, b_, _, _ in results if b_]
    assert not bad, f"scenes with hit mismatches (scene, words): {bad[:10]}"
    assert sum(r[2] for r in results) > 0
    for s, _, _, og in results:
        if og is None:
            continue
        ex = bt.export_scene(s, og.cells.shape[0], og.indices.size)
        assert np.array_equal(ex["res"], og.res), f"scene {s} res"
        assert np.array_equal(ex["cells"], og.cells), f"scene {s} cells"
        assert np.array_equal(ex["indices"], og.indices), f"scene {s} indices"
    bt.close()
