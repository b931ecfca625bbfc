"""Block culling inside the leaf cells of a two-level grid, at the full size of
the dense-cluster workload (1,048,576 triangles, leaf cells of tens of
thousands of references), against the oracle, which tests every reference.

The two-level build runs on the triangles in Morton order and the traversal
skips 32-reference blocks whose box the ray's segment cannot meet.  Closest
hits (triangle id and t) and any-hit flags must equal the oracle's bit for
bit, for rays from a common eye (the grouped same-origin path), rays starting
inside the cluster in random directions, axis-aligned rays (zero direction
components), and short segments; the exported grid must be the oracle's.
"""
import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

from test_gpu_parity import assert_grid_equal, build_both

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def cluster():
    import shinobi_b200 as shn
    sc = scenes.cluster_in_field(1 << 20, seed=1)
    soup, g, og = build_both(shn, sc, shn.SHN_GRID_TWO_LEVEL, 1.0 / 16.0, divisor=1, min_res=2, lam_leaf=4.0)
    return shn, sc, soup, g, og


def _rays(n, seed):
    rng = np.random.default_rng(seed)
    # eye rays through the cluster (one origin)
    eye = np.tile(np.array([0.0, 0.0, -0.25], np.float32), (n, 1))
    tgt = rng.uniform(-0.06, 0.06, size=(n, 3)).astype(np.float32)
    d_eye = (tgt - eye).astype(np.float32)
    # rays starting inside the cluster, random directions
    o_in = rng.uniform(-0.05, 0.05, size=(n, 3)).astype(np.float32)
    d_in = rng.normal(size=(n, 3)).astype(np.float32)
    # axis-aligned rays through the cluster
    o_ax = rng.uniform(-0.05, 0.05, size=(n, 3)).astype(np.float32)
    axis = rng.integers(0, 3, size=n)
    sign = rng.choice([-1.0, 1.0], size=n)
    d_ax = np.zeros((n, 3), np.float32)
    d_ax[np.arange(n), axis] = sign
    o_ax[np.arange(n), axis] = -0.2 * sign            # start outside, pointing in
    org = np.concatenate([eye, o_in, o_ax])
    dirs = np.concatenate([d_eye, d_in, d_ax])
    return org, dirs


def test_exported_grid_is_canonical(cluster):
    shn, sc, soup, g, og = cluster
    assert_grid_equal(shn, g, og)


def test_closest_hits_with_culling(cluster):
    import torch
    shn, sc, soup, g, og = cluster
    org, dirs = _rays(12000, seed=3)
    h = g.trace_closest(torch.from_numpy(org).cuda(), torch.from_numpy(dirs).cuda())
    tri = h.tri.cpu().numpy().view(np.uint32)
    t = h.t.cpu().numpy()
    rt, rtt = oracle.trace_closest(og, org, dirs)[:2]
    assert np.count_nonzero(rt != shn.SHN_MISS) > 20000
    assert np.array_equal(tri, rt)
    assert np.array_equal(t.view(np.uint32), rtt.view(np.uint32))


@pytest.mark.parametrize("tmax", [1e-4, 0.01, 0.1])
def test_any_hit_with_culling(cluster, tmax):
    import torch
    shn, sc, soup, g, og = cluster
    org, dirs = _rays(8000, seed=5)
    tm = np.full(org.shape[0], tmax, np.float32)
    occ = g.trace_any(torch.from_numpy(org).cuda(), torch.from_numpy(dirs).cuda(),
                      torch.from_numpy(tm).cuda()).cpu().numpy()
    ro, _ = oracle.trace_any(og, org, dirs, tm)
    assert np.array_equal(occ, ro)
    assert 0 < ro.sum() < ro.size


def test_camera_and_ao_full_frame_sample(cluster):
    """The C1 camera at a reduced resolution: every primary hit and AO flag."""
    import torch
    shn, sc, soup, g, og = cluster
    cam = scenes.Camera((0.0, 0.0, -0.25), (0.0, 0.0, 1.0), (0.0, 1.0, 0.0), 45.0, 320, 180)
    h = g.trace_primary(cam)
    nrays = torch.zeros(1, dtype=torch.int32, device="cuda")
    ao = g.trace_ao(cam, h, spp=4, length=0.1, offset=1e-4, seed=1, num_rays=nrays).cpu().numpy()
    org, d = oracle.primary_rays(cam)
    rt, rtt = oracle.trace_closest(og, org, d)[:2]
    assert np.array_equal(h.tri.cpu().numpy().view(np.uint32), rt)
    assert np.array_equal(h.t.cpu().numpy().view(np.uint32), rtt.view(np.uint32))
    ro, rd, rpix = oracle.ao_rays(sc.vertices, sc.indices, org, d, rt, rtt, 4, 1, 1e-4)
    occ, _ = oracle.trace_any(og, ro, rd, np.full(ro.shape[0], 0.1, np.float32))
    cnt = np.zeros(org.shape[0], np.int64)
    np.add.at(cnt, rpix, occ.astype(np.int64))
    ref = np.where(rt == shn.SHN_MISS, np.float32(1.0),
                   (np.float32(1.0) - cnt.astype(np.float32) / np.float32(4.0)).astype(np.float32))
    assert np.array_equal(ao, ref.astype(np.float32))
