"""Dynamic scenes (DynamicRTEngine): the rebuild of frame N+1 on its own
stream while frame N renders gives exactly the frames of the sequential
interpolate -> rebuild -> render loop, one frame behind as in the reference."""
import numpy as np
import pytest

from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("kind", [0, 1])
def test_dynamic_frames_equal_sequential_rebuild_then_render(gpu, kind):
    import torch

    import shinobi_b200 as shn
    sc = scenes.cluster_in_field(32768, seed=1)
    base = sc.vertices
    move = scenes.uniform_draws(base.shape[0], 3, 7, scenes.TAG_RAYS)
    kf2 = (base + (move - np.float32(0.5)) * np.float32(0.004)).astype(np.float32)
    base_t = torch.from_numpy(base).cuda()
    kf2_t = torch.from_numpy(kf2).cuda()
    if kind == 0:
        p = shn.grid_params(shn.SHN_GRID_UNIFORM, lambda_=5.0)
    else:
        p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL, lambda_=1.0 / 16.0, top_divisor=1, min_res=2, lambda_leaf=4.0)
    cam = scenes.Camera((0.0, 0.0, -0.25), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 160, 90)
    di = shn.di_params(samples=4, seed=3)
    coeffs = [0.25, 0.5, 1.0, 0.75]
    eng = shn.DynamicEngine(base, sc.indices, p)
    hits = shn.alloc_hits(cam.res_x * cam.res_y)
    frame = torch.empty(cam.res_y, cam.res_x, 3, dtype=torch.float32, device="cuda")
    dyn = []
    for c in coeffs:
        eng.render_frame(base_t, kf2_t, c, cam, di, hits, frame)
        dyn.append((hits.tri.clone(), hits.t.clone(), frame.clone()))
    eng.close()
    # sequential: frame k shows the geometry of the previous call's coefficient
    soup = shn.FaceSoup(base, sc.indices)
    g = shn.Grid()
    for k, c_prev in enumerate([None] + coeffs[:-1]):
        if c_prev is not None:
            soup.interpolate_vertices(base_t, kf2_t, c_prev)
        g.build(soup, p)
        h = g.trace_primary(cam)
        f = g.shade_direct(cam, h, di)
        g.sync_status()
        tri, t, fr = dyn[k]
        assert torch.equal(h.tri, tri), f"frame {k}: hits differ"
        assert torch.equal(h.t.view(torch.int32), t.view(torch.int32)), f"frame {k}: t differs"
        assert torch.equal(f.view(torch.int32), fr.view(torch.int32)), f"frame {k}: shading differs"
    assert not torch.equal(dyn[0][0], dyn[-1][0])   # the geometry did move
