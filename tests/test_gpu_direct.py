"""Direct illumination from an area light (DirectIlluminationIntegrator::shade and
computeDirectIllumination, src/Integrator/DirectIlluminationIntegrator.h:46-338)
through the C ABI against the oracle.

Shadow segments, their blocked flags, the per-pixel frame and the progressive
final image are compared bit for bit: both sides evaluate the same IEEE FP32
operations in the same order (the library is built with -fmad=false, the
oracle with -ffp-contract=off).
"""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

from test_gpu_parity import build_both

pytestmark = pytest.mark.gpu

LIGHT_CLUSTER = dict(position=(-0.05, 0.2, -0.05), edge1=(0.1, 0.0, 0.0), edge2=(0.0, 0.0, 0.1),
                     normal=(0.0, -1.0, 0.0), intensity=(10.0, 9.0, 8.0))
LIGHT_SOUP = dict(position=(0.3, 1.2, 0.3), edge1=(0.4, 0.0, 0.0), edge2=(0.0, 0.0, 0.4),
                  normal=(0.0, -1.0, 0.0), intensity=(4.0, 4.0, 4.0))


def _oracle_direct(sc, og, cam, spp, seed, image_id, light, **kw):
    org, d = oracle.primary_rays(cam, image_id)
    tri, t, _, _, _ = oracle.trace_closest(og, org, d)
    ro, rd, rpix = oracle.direct_rays(org, d, tri, t, spp, seed, image_id, light)
    occ, _ = oracle.trace_any(og, ro, rd, np.full(ro.shape[0], 0.9999, np.float32))
    frame, fin = oracle.shade_direct(sc.vertices, sc.indices, org, d, tri, t, spp, seed, image_id, light,
                                     occ, **kw)
    return tri, occ, frame, fin


def test_direct_two_level(gpu):
    import shinobi_b200 as shn
    import torch
    sc = scenes.cluster_in_field(131072, seed=1)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_TWO_LEVEL, 1.0 / 16.0, lam_leaf=4.0)
    cam = scenes.Camera((0.0, 0.0, -0.25), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 256, 144)
    h = g.trace_primary(cam)
    nrays = torch.zeros(1, dtype=torch.int32, device="cuda")
    p = shn.di_params(light=LIGHT_CLUSTER, samples=4, seed=7)
    frame = g.shade_direct(cam, h, p, num_rays=nrays).cpu().numpy().reshape(-1, 3)
    tri, occ, ref, _ = _oracle_direct(sc, og, cam, 4, 7, 0, LIGHT_CLUSTER)
    assert int(nrays.item()) == occ.shape[0] == int(np.count_nonzero(tri != shn.SHN_MISS)) * 4
    assert np.array_equal(frame.view(np.uint32), ref.view(np.uint32))
    hit = tri != shn.SHN_MISS
    lit = (frame[hit] > 0).any(axis=1)
    assert 0.05 < lit.mean() < 0.95            # lit and shadowed or back-facing pixels both occur
    assert 0.0 < occ.mean() < 1.0


def test_direct_uniform_materials_progressive(gpu):
    import shinobi_b200 as shn
    import torch
    sc = scenes.uniform_soup(65536, seed=0)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_UNIFORM, 5.0)
    cam = scenes.Camera((0.5, 0.5, -1.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 192, 160)
    rng = np.random.default_rng(11)
    mats = rng.integers(0, 6, size=sc.num_triangles, dtype=np.uint32)   # ids 4, 5 are out of range
    table = rng.uniform(0.1, 0.9, size=(4, 4)).astype(np.float32)
    d_mats = torch.from_numpy(mats.view(np.int32)).cuda()
    d_table = torch.from_numpy(table).cuda()
    n = cam.res_x * cam.res_y
    final = torch.zeros(cam.res_y, cam.res_x, 3, dtype=torch.float32, device="cuda")
    ref_final = np.zeros((n, 3), np.float32)
    for image_id in range(3):
        h = g.trace_primary(cam, image_id)
        p = shn.di_params(light=LIGHT_SOUP, tri_material=d_mats, diffuse=d_table, samples=3, seed=5,
                          image_id=image_id)
        frame = g.shade_direct(cam, h, p, final=final).cpu().numpy().reshape(-1, 3)
        tri, occ, ref, ref_final = _oracle_direct(sc, og, cam, 3, 5, image_id, LIGHT_SOUP,
                                                  tri_material=mats, diffuse=table, final=ref_final)
        assert np.array_equal(frame.view(np.uint32), ref.view(np.uint32)), image_id
        got_final = final.cpu().numpy().reshape(-1, 3)
        assert np.array_equal(got_final.view(np.uint32), ref_final.view(np.uint32)), image_id
    assert (ref_final > 0).any()


def test_direct_all_miss_is_background(gpu):
    import shinobi_b200 as shn
    import torch
    sc = scenes.uniform_soup(4096, seed=2)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_UNIFORM, 5.0)
    cam = scenes.Camera((0.5, 0.5, -1.5), (0.0, 0.0, -1.0), (0.0, 1.0, 0.0), 45.0, 64, 48)
    h = g.trace_primary(cam)
    nrays = torch.full((1,), 77, dtype=torch.int32, device="cuda")
    frame = g.shade_direct(cam, h, shn.di_params(samples=5), num_rays=nrays).cpu().numpy().reshape(-1, 3)
    _, occ, ref, _ = _oracle_direct(sc, og, cam, 5, 1, 0, dict(
        position=(-0.05, 0.2, -0.05), edge1=(0.1, 0.0, 0.0), edge2=(0.0, 0.0, 0.1), normal=(0.0, -1.0, 0.0),
        intensity=(10.0, 10.0, 10.0)))
    assert int(nrays.item()) == 0 and occ.shape[0] == 0
    assert np.array_equal(frame.view(np.uint32), ref.view(np.uint32))
    np.testing.assert_allclose(frame, np.tile([0.15, 0.2, 0.3], (frame.shape[0], 1)), rtol=1e-6)


def test_direct_invalid_arguments(gpu):
    import shinobi_b200 as shn
    import torch
    sc = scenes.uniform_soup(1024, seed=3)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_UNIFORM, 5.0)
    cam = scenes.Camera((0.5, 0.5, -1.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 32, 32)
    h = g.trace_primary(cam)
    with pytest.raises(shn.ShinobiError):
        g.shade_direct(cam, h, shn.di_params(samples=0))
    table = torch.ones(2, 4, dtype=torch.float32, device="cuda")
    with pytest.raises(shn.ShinobiError):
        g.shade_direct(cam, h, shn.di_params(diffuse=table, num_materials=0))
