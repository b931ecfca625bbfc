"""The oracle's direct-illumination restatement (computeDirectIllumination,
src/Integrator/DirectIlluminationIntegrator.h:46-168; AreaLightShadowRayGenerator,
src/Engine/RayGenerators.h:106-139) against an independent float64 evaluation
of the same formula, on the CPU."""
import numpy as np

import oracle

MISS = 0xFFFFFFFF
LIGHT = dict(position=(-0.2, 1.0, -0.2), edge1=(0.4, 0.0, 0.0), edge2=(0.0, 0.0, 0.4),
             normal=(0.0, -1.0, 0.0), intensity=(5.0, 4.0, 3.0))


def _scene():
    # two triangles in the plane y = 0: the first faces +y, the second (reversed winding) faces -y
    vtx = np.array([[0, 0, 0], [0, 0, 1], [1, 0, 0], [0, 0, 0], [1, 0, 0], [0, 0, 1]], np.float32)
    idx = np.array([[0, 1, 2], [3, 4, 5]], np.uint32)
    return vtx, idx


def _primary(n=64, seed=0):
    rng = np.random.default_rng(seed)
    org = np.tile(np.array([0.3, 2.0, 0.3], np.float32), (n, 1))
    tgt = np.stack([rng.uniform(0.05, 0.6, n), np.zeros(n), rng.uniform(0.05, 0.3, n)], 1).astype(np.float32)
    d = (tgt - org).astype(np.float32)
    t = np.ones(n, np.float32)
    tri = (np.arange(n) % 3).astype(np.uint32)
    tri[tri == 2] = MISS
    return org, d, tri, t


def _ref64(vtx, idx, org, d, tri, t, ro, rd, occ, spp, diff, bg):
    n = org.shape[0]
    out = np.zeros((n, 3))
    li = np.array(LIGHT["intensity"], np.float64)
    ln = np.array(LIGHT["normal"], np.float64)
    area = np.linalg.norm(np.cross(LIGHT["edge1"], LIGHT["edge2"]))
    k = 0
    for p in range(n):
        if tri[p] == MISS:
            out[p] = np.asarray(bg, np.float64)
            continue
        v = vtx[idx[tri[p]]].astype(np.float64)
        nrm = np.cross(v[1] - v[0], v[2] - v[0])
        nrm /= np.linalg.norm(nrm)
        for s in range(spp):
            L = rd[k].astype(np.float64)
            assert np.allclose(ro[k], org[p] + (t[p] - 1e-5) * d[p], atol=1e-6)
            if not occ[k]:
                lh = L / np.linalg.norm(L)
                out[p] += li * area * np.asarray(diff) * max(0.0, -ln @ lh) * max(0.0, nrm @ lh) / (L @ L) / spp
            k += 1
    return out


def test_direct_shading_matches_float64():
    vtx, idx = _scene()
    org, d, tri, t = _primary()
    spp = 4
    ro, rd, rpix = oracle.direct_rays(org, d, tri, t, spp, 3, 0, LIGHT)
    assert ro.shape[0] == int(np.count_nonzero(tri != MISS)) * spp
    # light points lie on the light's parallelogram
    lp = ro + rd
    assert np.allclose(lp[:, 1], 1.0, atol=1e-5)
    assert (lp[:, 0] >= -0.2 - 1e-6).all() and (lp[:, 0] <= 0.2 + 1e-6).all()
    rng = np.random.default_rng(1)
    occ = (rng.random(ro.shape[0]) < 0.3).astype(np.uint8)
    frame, _ = oracle.shade_direct(vtx, idx, org, d, tri, t, spp, 3, 0, LIGHT, occ)
    ref = _ref64(vtx, idx, org, d, tri, t, ro, rd, occ, spp, (0.7, 0.7, 0.7), (0.15, 0.2, 0.3))
    np.testing.assert_allclose(frame, ref, rtol=2e-5, atol=1e-7)
    # the back-facing triangle (id 1) receives nothing; the front-facing one is lit where unblocked
    assert (frame[tri == 1] == 0).all()
    assert (frame[tri == 0] > 0).any()


def test_direct_all_blocked_and_materials():
    vtx, idx = _scene()
    org, d, tri, t = _primary(seed=2)
    ro, rd, _ = oracle.direct_rays(org, d, tri, t, 2, 9, 0, LIGHT)
    frame, _ = oracle.shade_direct(vtx, idx, org, d, tri, t, 2, 9, 0, LIGHT, np.ones(ro.shape[0], np.uint8))
    assert (frame[tri != MISS] == 0).all()
    table = np.array([[0.5, 0.5, 0.5, 0], [0.9, 0.1, 0.2, 0]], np.float32)
    mats = np.array([1, 0], np.uint32)
    occ0 = np.zeros(ro.shape[0], np.uint8)
    f_mat, _ = oracle.shade_direct(vtx, idx, org, d, tri, t, 2, 9, 0, LIGHT, occ0, tri_material=mats,
                                   diffuse=table)
    ref = _ref64(vtx, idx, org, d, tri, t, ro, rd, occ0, 2, table[1, :3], (0.15, 0.2, 0.3))
    sel = tri == 0
    np.testing.assert_allclose(f_mat[sel], ref[sel], rtol=2e-5, atol=1e-7)
    # an out-of-range material id reads material 0
    f_oor, _ = oracle.shade_direct(vtx, idx, org, d, tri, t, 2, 9, 0, LIGHT, occ0,
                                   tri_material=np.array([7, 7], np.uint32), diffuse=table)
    ref0 = _ref64(vtx, idx, org, d, tri, t, ro, rd, occ0, 2, table[0, :3], (0.15, 0.2, 0.3))
    np.testing.assert_allclose(f_oor[sel], ref0[sel], rtol=2e-5, atol=1e-7)


def test_progressive_blend():
    vtx, idx = _scene()
    org, d, tri, t = _primary(seed=3)
    fin = np.zeros((org.shape[0], 3), np.float32)
    frames = []
    for image_id in range(4):
        ro, rd, _ = oracle.direct_rays(org, d, tri, t, 1, 4, image_id, LIGHT)
        f, fin = oracle.shade_direct(vtx, idx, org, d, tri, t, 1, 4, image_id, LIGHT,
                                     np.zeros(ro.shape[0], np.uint8), final=fin)
        frames.append(f.astype(np.float64))
    np.testing.assert_allclose(fin, np.mean(frames, axis=0), rtol=1e-5, atol=1e-7)
    # different image ids draw different light points
    assert not np.array_equal(frames[0], frames[1])
