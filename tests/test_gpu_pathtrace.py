"""Wavefront path tracer (compaction after every bounce) against the oracle's
path-by-path restatement: same counter-based Philox streams, same arithmetic,
so the images agree exactly; the stated per-pixel RMSE bound (1e-6) is also
checked for the record."""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu

RMSE_TOL = 1e-6
LIGHT = dict(light_pos=(0.3, 0.3, 1.0), light_e1=(0.0, 0.4, 0.0), light_e2=(0.4, 0.0, 0.0),
             light_radiance=(20.0, 20.0, 20.0), background=(0.15, 0.2, 0.3))


@pytest.mark.parametrize("kind", [0, 1])
def test_pt_matches_oracle(gpu, kind):
    import torch

    import shinobi_b200 as shn
    sc = scenes.heightfield_boxes(128, 64, nboxes=40)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    if kind == 0:
        res = oracle.resolution(sc.num_triangles, b, 5.0)
        og = oracle.build_uniform(sc.vertices, sc.indices, b, res)
        p = shn.grid_params(shn.SHN_GRID_UNIFORM, res=res)
    else:
        res = oracle.resolution(sc.num_triangles, b, 5.0, 6, 2)
        og = oracle.build_two_level(sc.vertices, sc.indices, b, res, 1.2, 16)
        p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL, res=res)
    g = shn.Grid().build(soup, p)
    cam = scenes.Camera(scenes.CAMERA_HEIGHTFIELD.eye, scenes.CAMERA_HEIGHTFIELD.forward,
                        scenes.CAMERA_HEIGHTFIELD.up, 45.0, 96, 54)
    params = shn.pt_params(spp=8, max_depth=4, rr_depth=2, albedo=0.7, offset=1e-4, seed=2, **LIGHT)
    stats = torch.zeros(5, dtype=torch.int32, device="cuda")
    img = g.pt_render(soup, cam, params, stats=stats).cpu().numpy()
    ref = oracle.pt_render(og, cam, 8, 4, 2, 0.7, LIGHT["light_pos"], LIGHT["light_e1"], LIGHT["light_e2"],
                           LIGHT["light_radiance"], LIGHT["background"], 1e-4, 2)
    rmse = float(np.sqrt(np.mean((img.astype(np.float64) - ref) ** 2)))
    assert rmse <= RMSE_TOL
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
    live = stats.cpu().numpy()
    assert live[0] == 96 * 54 * 8
    assert np.all(np.diff(live[:4]) <= 0) and live[3] > 0   # compaction shrinks the wavefront
    assert 0 < live[4] <= live[:4].sum()                     # next-event shadow rays


def test_pt_large_wave_chunks(gpu):
    """More paths than one wavefront chunk: the chunked waves give the same image."""
    import shinobi_b200 as shn
    sc = scenes.heightfield_boxes(64, 32, nboxes=10)
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, 5.0)
    og = oracle.build_uniform(sc.vertices, sc.indices, b, res)
    g = shn.Grid().build(soup, shn.grid_params(shn.SHN_GRID_UNIFORM, res=res))
    cam = scenes.Camera(scenes.CAMERA_HEIGHTFIELD.eye, scenes.CAMERA_HEIGHTFIELD.forward,
                        scenes.CAMERA_HEIGHTFIELD.up, 45.0, 512, 512)
    params = shn.pt_params(spp=40, max_depth=3, rr_depth=1, **LIGHT)   # 10.5M paths > 2^23 per wave
    img = g.pt_render(soup, cam, params).cpu().numpy()
    ref = oracle.pt_render(og, cam, 40, 3, 1, 0.7, LIGHT["light_pos"], LIGHT["light_e1"], LIGHT["light_e2"],
                           LIGHT["light_radiance"], LIGHT["background"], 1e-4, 2)
    assert np.array_equal(img.view(np.uint32), ref.view(np.uint32))
