"""Keyframe interpolation on the device (FaceSoup::uploadVertices of the
reference's DynamicRTEngine, src/Control/Structure/FaceSoup.h:249-339):
vertices kf1 * (1 - c) + kf2 * c in FP32, the rest from kf2 when the first
keyframe is shorter; the rebuilt grid, the bounds and the primary hits must
equal the oracle's on the same interpolated vertices."""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

from test_gpu_parity import assert_grid_equal

pytestmark = pytest.mark.gpu


def _lerp(kf1, kf2, c):
    c = np.float32(c)
    out = kf2.copy()
    m = kf1.shape[0]
    out[:m] = kf1 * (np.float32(1.0) - c) + kf2[:m] * c
    return out.astype(np.float32)


@pytest.mark.parametrize("kind,short", [(0, False), (1, False), (1, True)])
def test_interpolated_frame_matches_oracle(gpu, kind, short):
    import torch
    import shinobi_b200 as shn
    sc = scenes.cluster_in_field(20000, seed=9) if kind else scenes.uniform_soup(20000, seed=9)
    rng = np.random.default_rng(2)
    kf1 = sc.vertices.copy()
    kf2 = (sc.vertices + rng.normal(scale=0.003, size=sc.vertices.shape)).astype(np.float32)
    if short:
        kf1 = kf1[: kf1.shape[0] // 2]
    soup = shn.FaceSoup(sc.vertices, sc.indices)
    for c in (0.37, 1.0):
        soup.interpolate_vertices(torch.from_numpy(kf1).cuda(), torch.from_numpy(kf2).cuda(), c)
        v = _lerp(kf1, kf2, c)
        b = oracle.bounds(v, sc.indices)
        assert np.array_equal(soup.bounds.view(np.uint32), b.view(np.uint32))
        if kind:
            res = oracle.resolution(sc.num_triangles, b, 1.0 / 16.0, 1, 2)
            p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL, lambda_=1.0 / 16.0, top_divisor=1, min_res=2,
                                lambda_leaf=4.0, res=res)
            og = oracle.build_two_level(v, sc.indices, b, res, 4.0, 16)
            cam = scenes.Camera((0.0, 0.0, -0.25), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 96, 64)
        else:
            res = oracle.resolution(sc.num_triangles, b, 5.0)
            p = shn.grid_params(shn.SHN_GRID_UNIFORM, lambda_=5.0, res=res)
            og = oracle.build_uniform(v, sc.indices, b, res)
            cam = scenes.Camera((0.5, 0.5, -1.5), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 96, 64)
        g = shn.Grid().build(soup, p)
        assert_grid_equal(shn, g, og)
        h = g.trace_primary(cam)
        org, d = oracle.primary_rays(cam)
        rt, rtt = oracle.trace_closest(og, org, d)[:2]
        assert np.array_equal(h.tri.cpu().numpy().view(np.uint32), rt)
        assert np.array_equal(h.t.cpu().numpy().view(np.uint32), rtt.view(np.uint32))
