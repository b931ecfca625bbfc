"""The reference's only real scene, ruins (38,665 triangles of uneven sizes
with shared vertices and 10 materials), as the reference's own readers load
it (tests/golden/ruins.npz), through the CUDA path against the oracle:
uniform and two-level grids bit-exact, primary hits from the scene's camera
and direct illumination from its area light with its materials, compared on
a spread of pixels of the 1024x1024 frame (bit-exact)."""
import os

import numpy as np
import pytest

import oracle
from shinobi_b200 import scenes

pytestmark = pytest.mark.gpu

HERE = os.path.dirname(os.path.abspath(__file__))


def _ruins():
    z = np.load(os.path.join(HERE, "golden", "ruins.npz"))
    c = z["camera"]
    cam = scenes.Camera(tuple(c[0:3]), tuple(c[3:6]), tuple(c[6:9]), float(c[9]), int(c[10]), int(c[11]))
    l = z["light"]
    light = {k: tuple(l[3 * i:3 * i + 3]) for i, k in enumerate(("position", "edge1", "edge2", "normal", "intensity"))}
    diffuse = np.zeros((z["materials"].shape[0], 4), np.float32)
    diffuse[:, :3] = z["materials"][:, 0:3]
    return z["vertices"], z["indices"], z["face_material"], diffuse, cam, light


def _build(shn, vtx, idx, kind):
    soup = shn.FaceSoup(vtx, idx)
    b = oracle.bounds(vtx, idx)
    if kind == shn.SHN_GRID_UNIFORM:
        res = oracle.resolution(idx.shape[0], b, 5.0)
        og = oracle.build_uniform(vtx, idx, b, res)
        p = shn.grid_params(shn.SHN_GRID_UNIFORM, lambda_=5.0)
    else:
        res = oracle.resolution(idx.shape[0], b, 5.0, 6, 2)
        og = oracle.build_two_level(vtx, idx, b, res, 1.2, 16)
        p = shn.grid_params(shn.SHN_GRID_TWO_LEVEL)
    g = shn.Grid().build(soup, p)
    return soup, g, og


@pytest.mark.parametrize("kind", [0, 1])
def test_ruins_grids_bit_exact(gpu, kind):
    import shinobi_b200 as shn
    vtx, idx, _, _, _, _ = _ruins()
    soup, g, og = _build(shn, vtx, idx, kind)
    ex = g.export()
    assert np.array_equal(ex["res"], og.res)
    keys = ("cells", "indices", "top_pairs") + (("leaves",) if kind == 1 else ())
    for k in keys:
        assert np.array_equal(ex[k], getattr(og, k)), k


@pytest.mark.parametrize("kind", [0, 1])
def test_ruins_primary_hits_and_direct_illumination(gpu, kind):
    import torch

    import shinobi_b200 as shn
    oracle.set_threads(os.cpu_count() or 1)
    vtx, idx, fmat, diffuse, cam, light = _ruins()
    soup, g, og = _build(shn, vtx, idx, kind)
    h = g.trace_primary(cam)
    tm = torch.from_numpy(fmat.view(np.int32)).cuda()
    dt = torch.from_numpy(diffuse).cuda()
    prm = shn.di_params(light=light, tri_material=tm, diffuse=dt, samples=4, seed=1)
    frame = g.shade_direct(cam, h, prm)
    g.sync_status()
    org, d = oracle.primary_rays(cam)
    sel = np.arange(3, org.shape[0], 5, dtype=np.int64)
    rt, rtt, ru, rv, _ = oracle.trace_closest(og, org[sel], d[sel])
    tri = h.tri.cpu().numpy().view(np.uint32)[sel]
    assert np.array_equal(tri, rt), f"{np.count_nonzero(tri != rt)} of {sel.size} hits differ"
    assert np.array_equal(h.t.cpu().numpy()[sel].view(np.uint32), rtt.view(np.uint32))
    hit = rt != shn.SHN_MISS
    assert hit.mean() > 0.5
    ro, rd, _ = oracle.direct_rays(org[sel], d[sel], rt, rtt, 4, 1, 0, light, pix=sel)
    occ, _ = oracle.trace_any(og, ro, rd, np.full(ro.shape[0], 0.9999, np.float32))
    ref, _ = oracle.shade_direct(vtx, idx, org[sel], d[sel], rt, rtt, 4, 1, 0, light, occ, tri_material=fmat,
                                 diffuse=diffuse, pix=sel)
    got = frame.cpu().numpy().reshape(-1, 3)[sel]
    assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), \
        f"{np.count_nonzero((got != ref).any(axis=1))} of {sel.size} shaded pixels differ"
    assert 0.05 < occ.mean() < 0.95
    assert float(ref.max()) > 0.0
