"""Generate the golden fixtures that pin the oracle to the reference's own code.

Runs where the reference tree is available (it builds oracle/_ref from the
reference sources in place, see oracle/Makefile) and writes small .npz files
next to this script.  The tests compare the oracle against these files
without needing the reference tree.

  python tests/golden/make_golden.py

Fixtures
  hostbuild_uniform.npz  TwoLevelGridBuilderHost::hostBuild on scenes where
                         every top cell holds <= 16 references (so each top
                         cell is one leaf: a uniform grid) and every triangle's
                         candidate range is either one cell on all axes or
                         >= 2 cells on all axes (there the reference's host
                         insertion rule and its GPU rule coincide)
  camera.npz             Camera::init + RegularPixelSampler + getDirection
  mt_closest.npz         SimpleIntersector (Moller-Trumbore) brute-force closest hits
  cosine.npz             CosineHemisphereSampler directions
  cellword.npz           TwoLevelGridCell packing
  ruins.npz              the reference's ruins scene as its own scene-file
                         readers load it (FWObject::read, CameraManager::read,
                         LightSourceLoader::loadFromFile on scenes/ruins):
                         vertices, triangle indices, face materials, the
                         Phong-normalised diffuse / specular table, camera
                         and area light

  python tests/golden/make_golden.py --only ruins    (that fixture alone)
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

import oracle  # noqa: E402
from shinobi_b200 import scenes  # noqa: E402

EPS = np.float32(1e-5)


def candidate_spans(vtx, idx, b, res):
    """Per-triangle candidate cell counts per axis, float32 like countRefs."""
    v = vtx[idx]                                  # (n, 3, 3)
    bmin = v.min(axis=1).astype(np.float32)
    bmax = v.max(axis=1).astype(np.float32)
    gmin = b[:3].astype(np.float32)
    gmax = b[3:].astype(np.float32)
    resf = res.astype(np.float32)
    cs = (gmax - gmin) / resf
    rcp = np.float32(1.0) / cs
    minf = np.maximum(np.float32(0), (bmin - gmin) * rcp + (-EPS))
    maxf = np.minimum(resf - np.float32(1), (bmax - gmin) * rcp + EPS)
    lo = minf.astype(np.uint32)
    hi = maxf.astype(np.uint32)
    return hi.astype(np.int64) - lo.astype(np.int64)


def hostbuild_case(n, seed, scale, lam):
    sc = scenes.uniform_soup(n, seed=seed, offset_scale=scale)
    b = oracle.bounds(sc.vertices, sc.indices)
    res = oracle.resolution(sc.num_triangles, b, lam)
    tris = sc.indices
    # drop triangles until the rule holds under the kept set's own bounds, so
    # that a build which derives its bounds from the scene sees the same grid
    for _ in range(20):
        span = candidate_spans(sc.vertices, tris, b, res)
        keep = np.all(span == 0, axis=1) | np.all(span >= 1, axis=1)
        tris = tris[keep]
        b2 = oracle.bounds(sc.vertices, tris)
        if keep.all() and np.array_equal(b2, b):
            break
        b = b2
    else:
        raise RuntimeError("filter did not converge")
    used, inv = np.unique(tris, return_inverse=True)
    vtx = np.ascontiguousarray(sc.vertices[used])
    idx = np.ascontiguousarray(inv.reshape(-1, 3).astype(np.uint32))
    cells, leaves, refs = oracle.ref_host_build(vtx, idx, b, res)
    C = cells.shape[0]
    assert leaves.shape[0] == C, "a top cell was refined; pick a finer resolution"
    return dict(vertices=vtx, indices=idx, bounds=b, res=res, leaves=leaves, refs=refs,
                cellwords=cells)


def main():
    if oracle.ref_lib() is None:
        oracle.build()
    R = oracle.ref_lib()
    assert R is not None, "oracle/_ref not built: the reference tree is required"
    import ctypes as C

    def p(a):
        return a.ctypes.data_as(C.c_void_p)

    # ---- host builder on rule-coincident scenes --------------------------------
    cases = [hostbuild_case(20000, 11, 0.003, 5.0), hostbuild_case(6000, 12, 0.02, 5.0),
             hostbuild_case(3000, 13, 0.05, 2.0)]
    out = {}
    for k, c in enumerate(cases):
        for key, val in c.items():
            out[f"c{k}_{key}"] = val
    out["num_cases"] = np.array(len(cases))
    np.savez_compressed(os.path.join(HERE, "hostbuild_uniform.npz"), **out)

    # ---- camera + pixel sampler ------------------------------------------------------
    cams = [scenes.CAMERA_SOUP, scenes.CAMERA_CLUSTER, scenes.CAMERA_HEIGHTFIELD,
            scenes.Camera((1.0, -2.0, 0.5), (0.3, 0.9, -0.1), (0.0, 0.0, 1.0), 60.0, 333, 77)]
    cam_out = {}
    rng = np.random.default_rng(0)
    for k, cam in enumerate(cams):
        c9 = np.zeros(9, np.float32)
        R.ref_camera(p(np.array(cam.eye, np.float32)), p(np.array(cam.forward, np.float32)),
                     p(np.array(cam.up, np.float32)), cam.fov_deg, cam.res_x, cam.res_y, p(c9))
        ids = np.unique(np.concatenate([np.arange(64), rng.integers(0, cam.res_x * cam.res_y, 4000)])).astype(np.uint32)
        dirs = np.zeros((ids.size, 3), np.float32)
        R.ref_primary_dirs(p(c9), cam.res_x, cam.res_y, 0, p(ids), ids.size, p(dirs))
        cam_out[f"cam{k}"] = np.array([*cam.eye, *cam.forward, *cam.up, cam.fov_deg, cam.res_x, cam.res_y], np.float64)
        cam_out[f"c9_{k}"] = c9
        cam_out[f"ids_{k}"] = ids
        cam_out[f"dirs_{k}"] = dirs
    cam_out["num"] = np.array(len(cams))
    np.savez_compressed(os.path.join(HERE, "camera.npz"), **cam_out)

    # ---- Moller-Trumbore closest hits (brute force) -----------------------------------
    sc = scenes.uniform_soup(2000, seed=21, offset_scale=0.15)
    org0, d0 = scenes.random_rays(3000, seed=22)
    # plus rays aimed at random interior points of random triangles (mostly hits)
    rng = np.random.default_rng(23)
    pick = rng.integers(0, sc.num_triangles, 3000)
    bary = rng.dirichlet([1.0, 1.0, 1.0], 3000).astype(np.float32)
    target = np.einsum("nk,nkd->nd", bary, sc.vertices[sc.indices[pick]]).astype(np.float32)
    org1 = rng.random((3000, 3), dtype=np.float32)
    d1 = (target - org1).astype(np.float32)
    org = np.ascontiguousarray(np.concatenate([org0, org1]), np.float32)
    d = np.ascontiguousarray(np.concatenate([d0, d1]), np.float32)
    tri = np.zeros(org.shape[0], np.uint32)
    t = np.zeros(org.shape[0], np.float32)
    R.ref_mt_closest(p(sc.vertices), p(np.ascontiguousarray(sc.indices)), sc.num_triangles, p(org), p(d),
                     org.shape[0], p(tri), p(t))
    np.savez_compressed(os.path.join(HERE, "mt_closest.npz"), vertices=sc.vertices, indices=sc.indices,
                        org=org, dir=d, tri=tri, t=t)

    # ---- cosine hemisphere sampler ------------------------------------------------------
    u = scenes.uniform_draws(5000, 2, 31, scenes.TAG_RAYS)
    u1 = np.ascontiguousarray(u[:, 0])
    u2 = np.ascontiguousarray(u[:, 1])
    dirs = np.zeros((5000, 3), np.float32)
    R.ref_cosine_sample(p(u1), p(u2), 5000, p(dirs))
    np.savez_compressed(os.path.join(HERE, "cosine.npz"), u1=u1, u2=u2, dirs=dirs)

    # ---- TwoLevelGridCell packing --------------------------------------------------------------
    rows = []
    for rx, ry, rz, ne, lb in [(1, 1, 1, 0, 0), (1, 1, 1, 1, 7), (87, 87, 87, 1, 123456), (255, 3, 9, 1, 4000000000),
                               (2, 200, 17, 0, 42), (16, 16, 16, 1, 1 << 31)]:
        w = np.zeros(2, np.uint32)
        R.ref_cell_word(rx, ry, rz, ne, lb, p(w))
        rows.append([rx, ry, rz, ne, lb, w[0], w[1]])
    np.savez_compressed(os.path.join(HERE, "cellword.npz"), rows=np.array(rows, np.uint64))
    print("fixtures written to", HERE)


def ruins_fixture():
    """The ruins scene through the reference's own readers (compiled in place)."""
    oracle.build()
    ref = os.environ.get("SHINOBI_REFERENCE", "/root/reference")
    d = os.path.join(ref, "scenes", "ruins")
    o = oracle.ref_read_obj(os.path.join(d, "ruins.obj"))
    cam = oracle.ref_read_camera(os.path.join(d, "camera.cfg"))
    light = oracle.ref_read_light(os.path.join(d, "light.cfg"))
    np.savez_compressed(os.path.join(HERE, "ruins.npz"), vertices=o["vertices"],
                        indices=o["indices"].astype(np.uint32), face_material=o["face_material"].astype(np.uint32),
                        materials=o["materials"], camera=cam, light=light)
    print("ruins.npz:", o["vertices"].shape[0], "vertices,", o["indices"].shape[0], "triangles,",
          o["materials"].shape[0], "materials")


if __name__ == "__main__":
    if "--only" in sys.argv and sys.argv[sys.argv.index("--only") + 1] == "ruins":
        ruins_fixture()
    else:
        main()
        ruins_fixture()
