"""Oracle (test infrastructure only).

Python bindings for ``liboracle.so`` -- the CPU restatement of Shinobi's
grid build, DDA traversal and ray generation -- and for ``_ref/`` -- the
reference's own host-compilable code compiled in place.  Only ``tests/``,
``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` import
this package; the product never does.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libshinobi_ref.so")
MISS = 0xFFFFFFFF

_lib = None
_ref = None


def build(force: bool = False) -> None:
    """Compile the oracle (and the reference checker when its tree is present)."""
    args = ["make", "-C", HERE]
    if force:
        args.insert(1, "-B")
    subprocess.run(args, check=True, stdout=subprocess.DEVNULL)


def _f32(a):
    return np.ascontiguousarray(a, dtype=np.float32)


def _u32(a):
    return np.ascontiguousarray(a, dtype=np.uint32)


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB) or os.path.getmtime(LIB) < os.path.getmtime(os.path.join(HERE, "oracle.cpp")):
            build()
        L = C.CDLL(LIB)
        vp, u32, i32, f32 = C.c_void_p, C.c_uint32, C.c_int, C.c_float
        L.orc_bounds.argtypes = [vp, vp, u32, vp]
        L.orc_resolution.argtypes = [u32, vp, f32, i32, i32, vp]
        L.orc_sah_window.argtypes = [u32, vp, f32, f32, f32, vp, vp]
        L.orc_sah_refs.argtypes = [vp, vp, u32, vp, vp]
        L.orc_sah_refs.restype = C.c_uint64
        L.orc_sah_cost.argtypes = [vp, vp, C.c_uint64]
        L.orc_sah_cost.restype = f32
        L.orc_sah_resolution.argtypes = [vp, vp, u32, vp, f32, f32, f32, vp, vp, vp, vp]
        L.orc_build_uniform.argtypes = [vp, u32, vp, u32, vp, vp]
        L.orc_build_uniform.restype = vp
        L.orc_build_two_level.argtypes = [vp, u32, vp, u32, vp, vp, f32, u32]
        L.orc_build_two_level.restype = vp
        L.orc_build_uniform_ex.argtypes = [vp, u32, vp, u32, vp, vp, i32]
        L.orc_build_uniform_ex.restype = vp
        L.orc_build_two_level_ex.argtypes = [vp, u32, vp, u32, vp, vp, f32, u32, i32]
        L.orc_build_two_level_ex.restype = vp
        L.orc_grid_free.argtypes = [vp]
        L.orc_set_reference_arithmetic.argtypes = [i32]
        L.orc_leaf_res_reference.argtypes = [vp, f32, u32, vp]
        L.orc_grid_from_arrays.argtypes = [i32, vp, vp, vp, vp, C.c_uint64, vp, C.c_uint64, vp, u32, vp, u32]
        L.orc_grid_from_arrays.restype = vp
        L.orc_grid_info.argtypes = [vp, vp]
        for nm in ("orc_grid_cells", "orc_grid_leaves", "orc_grid_indices", "orc_grid_top_pairs"):
            getattr(L, nm).argtypes = [vp]
            getattr(L, nm).restype = vp
        L.orc_num_threads.restype = i32
        L.orc_set_threads.argtypes = [i32]
        L.orc_trace_closest.argtypes = [vp] + [vp] * 7 + [u32] + [vp] * 5
        L.orc_trace_any.argtypes = [vp] + [vp] * 7 + [u32, vp, vp]
        L.orc_trace_brute.argtypes = [vp, vp, u32] + [vp] * 6 + [u32, vp, vp]
        L.orc_t_fp64.argtypes = [vp, vp, vp] + [vp] * 6 + [u32, vp]
        L.orc_sincos_2pi.argtypes = [vp, u32, vp, vp]
        L.orc_cosine_local.argtypes = [vp, vp, u32, vp]
        L.orc_philox.argtypes = [vp, u32, u32, u32, vp]
        L.orc_camera.argtypes = [vp, vp, vp, f32, u32, u32, vp]
        L.orc_primary_rays.argtypes = [vp, u32, u32, u32, vp, vp, vp]
        L.orc_ao_rays.argtypes = [vp, vp] + [vp] * 8 + [u32, u32, u32, f32] + [vp] * 8
        L.orc_ao_rays.restype = u32
        L.orc_direct_rays.argtypes = [vp] * 8 + [u32, u32, u32, u32, vp] + [vp] * 8
        L.orc_direct_rays.restype = u32
        L.orc_shade_direct.argtypes = [vp] * 10 + [u32, u32, u32, u32] + [vp] * 3 + [u32] + [vp] * 6
        L.orc_pt_render.argtypes = [vp, vp, vp, u32, u32, u32, u32, u32, f32, vp, vp, vp, vp, vp, f32, u32, vp]
        L.orc_pt_render_pixels.argtypes = [vp, vp, vp, u32, u32, u32, u32, u32, f32, vp, vp, vp, vp, vp, f32,
                                           u32, vp, u32, vp]
        L.orc_compact.argtypes = [vp, u32, vp]
        L.orc_compact.restype = u32
        _lib = L
    return _lib


def ref_lib():
    """The reference's own code compiled in place, or None when it was not built here."""
    global _ref
    if _ref is None and os.path.exists(REF_LIB):
        R = C.CDLL(REF_LIB)
        vp, u32, i32, f32 = C.c_void_p, C.c_uint32, C.c_int, C.c_float
        R.ref_host_build.argtypes = [vp, u32, vp, u32, i32, i32, i32, vp, vp]
        R.ref_host_build.restype = vp
        R.ref_host_build_copy.argtypes = [vp, vp, vp, vp]
        R.ref_host_build_free.argtypes = [vp]
        R.ref_camera.argtypes = [vp, vp, vp, f32, u32, u32, vp]
        R.ref_primary_dirs.argtypes = [vp, u32, u32, u32, vp, u32, vp]
        R.ref_mt_closest.argtypes = [vp, vp, u32, vp, vp, u32, vp, vp]
        R.ref_cosine_sample.argtypes = [vp, vp, u32, vp]
        R.ref_cell_word.argtypes = [u32, u32, u32, i32, u32, vp]
        R.ref_obj_read.argtypes = [C.c_char_p, vp]
        R.ref_obj_read.restype = vp
        R.ref_obj_copy.argtypes = [vp, vp, vp, vp, vp]
        R.ref_obj_free.argtypes = [vp]
        R.ref_camera_read.argtypes = [C.c_char_p, vp]
        R.ref_light_read.argtypes = [C.c_char_p, vp]
        _ref = R
    return _ref


def bounds(vtx, idx) -> np.ndarray:
    vtx, idx = _f32(vtx), _u32(idx)
    out = np.zeros(6, np.float32)
    lib().orc_bounds(_p(vtx), _p(idx), idx.shape[0], _p(out))
    return out


def resolution(nt: int, b, lam: float, divisor: int = 1, min_res: int = 1) -> np.ndarray:
    b = _f32(b)
    out = np.zeros(3, np.int32)
    lib().orc_resolution(nt, _p(b), lam, divisor, min_res, _p(out))
    return out


def sah_window(nt: int, b, lam: float = 5.0, wlo: float = 0.75, whi: float = 1.25):
    b = _f32(b)
    lo, hi = np.zeros(3, np.int32), np.zeros(3, np.int32)
    lib().orc_sah_window(nt, _p(b), lam, wlo, whi, _p(lo), _p(hi))
    return lo, hi


def sah_cost(vtx, idx, b, res):
    """(refs, cost) of one resolution (SAHGridBuilder.h:164-175)."""
    vtx, idx, b = _f32(vtx), _u32(idx), _f32(b)
    r = np.ascontiguousarray(res, np.int32)
    refs = int(lib().orc_sah_refs(_p(vtx), _p(idx), idx.shape[0], _p(b), _p(r)))
    return refs, float(np.float32(lib().orc_sah_cost(_p(b), _p(r), refs)))


def sah_resolution(vtx, idx, b, lam: float = 5.0, wlo: float = 0.75, whi: float = 1.25):
    """SAHGridBuilder::computeResolution: dict(res, cost, refs, res_min, res_max, counts[z, y, x])."""
    vtx, idx, b = _f32(vtx), _u32(idx), _f32(b)
    lo, hi = sah_window(idx.shape[0], b, lam, wlo, whi)
    n = hi - lo + 1
    counts = np.zeros(int(np.prod(n.astype(np.int64))), np.uint64)
    res = np.zeros(3, np.int32)
    cost = np.zeros(1, np.float32)
    refs = np.zeros(1, np.uint64)
    lib().orc_sah_resolution(_p(vtx), _p(idx), idx.shape[0], _p(b), lam, wlo, whi, _p(res), _p(cost), _p(refs),
                             _p(counts))
    return {"res": tuple(int(x) for x in res), "cost": float(cost[0]), "refs": int(refs[0]),
            "res_min": tuple(int(x) for x in lo), "res_max": tuple(int(x) for x in hi),
            "counts": counts.reshape(int(n[2]), int(n[1]), int(n[0]))}


@dataclass
class Grid:
    kind: int
    res: np.ndarray
    bounds: np.ndarray
    cells: np.ndarray       # (C, 2) uint32: ranges (uniform) or cell words (two-level)
    leaves: np.ndarray      # (L, 2) uint32 (two-level)
    indices: np.ndarray     # (K,) uint32
    top_pairs: np.ndarray   # sorted (cell<<32 | tri) uint64
    handle: object = None

    def __del__(self):
        if self.handle:
            lib().orc_grid_free(self.handle)
            self.handle = None


def _wrap(h, kind, res, b) -> Grid:
    L = lib()
    info = np.zeros(8, np.uint64)
    L.orc_grid_info(h, _p(info))
    nc, nk, nl, ntp = int(info[1]), int(info[2]), int(info[3]), int(info[4])

    def arr(ptr, n, dt):
        if n == 0:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(C.cast(ptr, C.POINTER(np.ctypeslib.as_ctypes_type(dt))), (n,)).copy()

    cells = arr(L.orc_grid_cells(h), 2 * nc, np.uint32).reshape(-1, 2)
    leaves = arr(L.orc_grid_leaves(h), 2 * nl, np.uint32).reshape(-1, 2)
    indices = arr(L.orc_grid_indices(h), nk, np.uint32)
    tp = arr(L.orc_grid_top_pairs(h), ntp, np.uint64)
    return Grid(kind, np.asarray(res, np.int32), np.asarray(b, np.float32), cells, leaves, indices, tp, h)


def build_uniform(vtx, idx, b, res, insertion: int = 0) -> Grid:
    """insertion 0: plane test (the GPU sort path); 1: the precise SAT insertion."""
    vtx, idx, b = _f32(vtx), _u32(idx), _f32(b)
    r = np.ascontiguousarray(res, np.int32)
    h = lib().orc_build_uniform_ex(_p(vtx), vtx.shape[0], _p(idx), idx.shape[0], _p(b), _p(r), insertion)
    return _wrap(h, 0, r, b)


def build_two_level(vtx, idx, b, res, lambda_leaf: float, leaf_threshold: int = 16, insertion: int = 0) -> Grid:
    vtx, idx, b = _f32(vtx), _u32(idx), _f32(b)
    r = np.ascontiguousarray(res, np.int32)
    h = lib().orc_build_two_level_ex(_p(vtx), vtx.shape[0], _p(idx), idx.shape[0], _p(b), _p(r),
                                     lambda_leaf, leaf_threshold, insertion)
    return _wrap(h, 1, r, b)


def grid_from_arrays(kind, b, res, cells, leaves, indices, vtx, idx) -> Grid:
    """Oracle traversal over grid arrays built elsewhere (e.g. by the reference builder)."""
    b, vtx, idx = _f32(b), _f32(vtx), _u32(idx)
    r = np.ascontiguousarray(res, np.int32)
    cells, indices = _u32(cells), _u32(indices)
    leaves = _u32(leaves) if leaves is not None else np.zeros((0, 2), np.uint32)
    h = lib().orc_grid_from_arrays(kind, _p(b), _p(r), _p(cells), _p(leaves), leaves.size // 2,
                                   _p(indices), indices.size, _p(vtx), vtx.shape[0], _p(idx), idx.shape[0])
    return Grid(kind, r, b, cells.reshape(-1, 2), leaves.reshape(-1, 2), indices, np.zeros(0, np.uint64), h)


def ref_host_build(vtx, idx, b, res):
    """The reference's TwoLevelGridBuilderHost::hostBuild (compiled in place) -> (cells, leaves, refs)."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("reference checker library not built (oracle/_ref)")
    vtx, idx, b = _f32(vtx), _u32(idx), _f32(b)
    sizes = np.zeros(3, np.uint64)
    h = R.ref_host_build(_p(vtx), vtx.shape[0], _p(idx), idx.shape[0], int(res[0]), int(res[1]),
                         int(res[2]), _p(b), _p(sizes))
    cells = np.zeros((int(sizes[0]), 2), np.uint32)
    leaves = np.zeros((int(sizes[1]), 2), np.uint32)
    refs = np.zeros(int(sizes[2]), np.uint32)
    R.ref_host_build_copy(h, _p(cells), _p(leaves), _p(refs))
    R.ref_host_build_free(h)
    return cells, leaves, refs


def ref_read_obj(path: str) -> dict:
    """The reference's FWObject::read (compiled in place): vertices, indices,
    face_material, and per material diffuse rgb, specular rgb, Ns."""
    R = ref_lib()
    if R is None:
        raise RuntimeError("reference checker library not built (oracle/_ref)")
    sizes = np.zeros(3, np.uint64)
    h = R.ref_obj_read(str(path).encode(), _p(sizes))
    nv, nf, nm = (int(x) for x in sizes)
    v = np.zeros((nv, 3), np.float32)
    f = np.zeros((nf, 3), np.uint64)
    fm = np.zeros(nf, np.uint64)
    mt = np.zeros((nm, 7), np.float32)
    R.ref_obj_copy(h, _p(v), _p(f), _p(fm), _p(mt))
    R.ref_obj_free(h)
    return {"vertices": v, "indices": f, "face_material": fm, "materials": mt}


def ref_read_camera(path: str) -> np.ndarray:
    """CameraManager::read from its defaults: position, orientation, up, FOV, resX, resY."""
    out = np.zeros(12, np.float32)
    ref_lib().ref_camera_read(str(path).encode(), _p(out))
    return out


def ref_read_light(path: str) -> np.ndarray:
    """LightSourceLoader::loadFromFile: position, edge1, edge2, normal, intensity (15 floats)."""
    out = np.zeros(15, np.float32)
    ref_lib().ref_light_read(str(path).encode(), _p(out))
    return out


def trace_closest(g: Grid, org, dirs, tmax=None):
    """Returns (tri, t, u, v, stats[steps, tests])."""
    org, dirs = _f32(org), _f32(dirs)
    n = org.shape[0]
    ox, oy, oz = (np.ascontiguousarray(org[:, k]) for k in range(3))
    dx, dy, dz = (np.ascontiguousarray(dirs[:, k]) for k in range(3))
    tm = _f32(tmax) if tmax is not None else None
    tri = np.zeros(n, np.uint32)
    t = np.zeros(n, np.float32)
    u = np.zeros(n, np.float32)
    v = np.zeros(n, np.float32)
    st = np.zeros(2, np.uint64)
    lib().orc_trace_closest(g.handle, _p(ox), _p(oy), _p(oz), _p(dx), _p(dy), _p(dz), _p(tm), n,
                            _p(tri), _p(t), _p(u), _p(v), _p(st))
    return tri, t, u, v, st


def trace_any(g: Grid, org, dirs, tmax):
    org, dirs = _f32(org), _f32(dirs)
    n = org.shape[0]
    ox, oy, oz = (np.ascontiguousarray(org[:, k]) for k in range(3))
    dx, dy, dz = (np.ascontiguousarray(dirs[:, k]) for k in range(3))
    tm = _f32(tmax)
    occ = np.zeros(n, np.uint8)
    st = np.zeros(2, np.uint64)
    lib().orc_trace_any(g.handle, _p(ox), _p(oy), _p(oz), _p(dx), _p(dy), _p(dz), _p(tm), n,
                        _p(occ), _p(st))
    return occ, st


def trace_brute(vtx, idx, org, dirs):
    vtx, idx, org, dirs = _f32(vtx), _u32(idx), _f32(org), _f32(dirs)
    n = org.shape[0]
    cols = [np.ascontiguousarray(org[:, k]) for k in range(3)] + [np.ascontiguousarray(dirs[:, k]) for k in range(3)]
    tri = np.zeros(n, np.uint32)
    t = np.zeros(n, np.float32)
    lib().orc_trace_brute(_p(vtx), _p(idx), idx.shape[0], *[_p(c) for c in cols], n, _p(tri), _p(t))
    return tri, t


def t_fp64(vtx, idx, tri, org, dirs) -> np.ndarray:
    vtx, idx, tri, org, dirs = _f32(vtx), _u32(idx), _u32(tri), _f32(org), _f32(dirs)
    n = org.shape[0]
    cols = [np.ascontiguousarray(org[:, k]) for k in range(3)] + [np.ascontiguousarray(dirs[:, k]) for k in range(3)]
    out = np.zeros(n, np.float64)
    lib().orc_t_fp64(_p(vtx), _p(idx), _p(tri), *[_p(c) for c in cols], n, _p(out))
    return out


def sincos_2pi(u):
    u = _f32(u)
    s = np.zeros_like(u)
    c = np.zeros_like(u)
    lib().orc_sincos_2pi(_p(u), u.size, _p(s), _p(c))
    return s, c


def cosine_local(u1, u2) -> np.ndarray:
    """Cosine-weighted hemisphere directions in the local frame (z = normal)."""
    u1, u2 = _f32(u1), _f32(u2)
    out = np.zeros((u1.shape[0], 3), np.float32)
    lib().orc_cosine_local(_p(u1), _p(u2), u1.shape[0], _p(out))
    return out


def philox(ctr, k0: int, k1: int) -> np.ndarray:
    ctr = _u32(ctr).reshape(-1, 4)
    out = np.zeros_like(ctr)
    lib().orc_philox(_p(ctr), ctr.shape[0], k0, k1, _p(out))
    return out


def camera(cam) -> np.ndarray:
    out = np.zeros(9, np.float32)
    lib().orc_camera(_p(_f32(cam.eye)), _p(_f32(cam.forward)), _p(_f32(cam.up)), cam.fov_deg,
                     cam.res_x, cam.res_y, _p(out))
    return out


def primary_rays(cam, image_id: int = 0):
    """(org (n,3), dir (n,3)) of the camera's primary rays, pixel-major."""
    c = camera(cam)
    n = cam.res_x * cam.res_y
    dx, dy, dz = (np.zeros(n, np.float32) for _ in range(3))
    lib().orc_primary_rays(_p(c), cam.res_x, cam.res_y, image_id, _p(dx), _p(dy), _p(dz))
    org = np.tile(_f32(cam.eye), (n, 1))
    return org, np.stack([dx, dy, dz], axis=1)


def ao_rays(vtx, idx, org, dirs, tri, t, spp: int, seed: int, offset: float, pix=None):
    """AO rays from primary hits; returns (org, dir, pixel) for hit pixels only.
    pix: the frame's pixel id of each input ray (a sample of a frame), which keys
    the random numbers; default 0..n-1.  The returned pixel is the input index."""
    vtx, idx, org, dirs, tri, t = _f32(vtx), _u32(idx), _f32(org), _f32(dirs), _u32(tri), _f32(t)
    pix = _u32(pix) if pix is not None else None
    n = org.shape[0]
    m_max = int(np.count_nonzero(tri != MISS)) * spp
    outs = [np.zeros(m_max, np.float32) for _ in range(6)] + [np.zeros(m_max, np.uint32)]
    cols = [np.ascontiguousarray(org[:, k]) for k in range(3)] + [np.ascontiguousarray(dirs[:, k]) for k in range(3)]
    m = lib().orc_ao_rays(_p(vtx), _p(idx), *[_p(c) for c in cols], _p(tri), _p(t), n, spp, seed,
                          offset, *[_p(o) for o in outs], _p(pix))
    assert m == m_max
    ro = np.stack(outs[0:3], axis=1)
    rd = np.stack(outs[3:6], axis=1)
    return ro, rd, outs[6]


def _light15(light) -> np.ndarray:
    return np.concatenate([_f32(light[k]) for k in ("position", "edge1", "edge2", "normal", "intensity")])


def direct_rays(org, dirs, tri, t, spp: int, seed: int, image_id: int, light, pix=None):
    """Shadow segments of the hit pixels; returns (org, dir, pixel) in pixel-major order.
    pix: frame pixel ids of the inputs (keys the random numbers), default 0..n-1."""
    org, dirs, tri, t = _f32(org), _f32(dirs), _u32(tri), _f32(t)
    pix = _u32(pix) if pix is not None else None
    n = org.shape[0]
    m_max = int(np.count_nonzero(tri != MISS)) * spp
    outs = [np.zeros(m_max, np.float32) for _ in range(6)] + [np.zeros(m_max, np.uint32)]
    cols = [np.ascontiguousarray(org[:, k]) for k in range(3)] + [np.ascontiguousarray(dirs[:, k]) for k in range(3)]
    m = lib().orc_direct_rays(*[_p(c) for c in cols], _p(tri), _p(t), n, spp, seed, image_id,
                              _p(_light15(light)), *[_p(o) for o in outs], _p(pix))
    assert m == m_max
    return np.stack(outs[0:3], axis=1), np.stack(outs[3:6], axis=1), outs[6]


def shade_direct(vtx, idx, org, dirs, tri, t, spp, seed, image_id, light, occ, tri_material=None,
                 diffuse=None, default_diffuse=(0.7, 0.7, 0.7), background=(0.15, 0.2, 0.3), final=None,
                 pix=None):
    """(frame (n,3), final (n,3) or None) with the semantics of shn_shade_direct;
    occ = blocked flags of direct_rays' segments, in its order."""
    vtx, idx, org, dirs, tri, t = _f32(vtx), _u32(idx), _f32(org), _f32(dirs), _u32(tri), _f32(t)
    n = org.shape[0]
    cols = [np.ascontiguousarray(org[:, k]) for k in range(3)] + [np.ascontiguousarray(dirs[:, k]) for k in range(3)]
    occ = np.ascontiguousarray(occ, dtype=np.uint8)
    tm = _u32(tri_material) if tri_material is not None else None
    df = _f32(diffuse).reshape(-1) if diffuse is not None else None
    nmat = df.size // 4 if df is not None else 0
    frame = np.zeros(3 * n, np.float32)
    fin = _f32(final).reshape(-1).copy() if final is not None else None
    lib().orc_shade_direct(_p(vtx), _p(idx), *[_p(c) for c in cols], _p(tri), _p(t), n, spp, seed, image_id,
                           _p(_light15(light)), _p(tm) if tm is not None else None,
                           _p(df) if df is not None else None, nmat, _p(_f32(default_diffuse)),
                           _p(_f32(background)), _p(occ), _p(frame), _p(fin) if fin is not None else None,
                           _p(_u32(pix)) if pix is not None else None)
    return frame.reshape(n, 3), (fin.reshape(n, 3) if fin is not None else None)


def pt_render(g: Grid, cam, spp, max_depth, rr_depth, albedo, light_pos, light_e1, light_e2,
              light_radiance, background, offset, seed) -> np.ndarray:
    """Path-traced image (resy, resx, 3) with the same semantics as shn_pt_render."""
    c = camera(cam)
    img = np.zeros(cam.res_x * cam.res_y * 3, np.float32)
    lib().orc_pt_render(g.handle, _p(c), _p(_f32(cam.eye)), cam.res_x, cam.res_y, spp, max_depth,
                        rr_depth, albedo, _p(_f32(light_pos)), _p(_f32(light_e1)), _p(_f32(light_e2)),
                        _p(_f32(light_radiance)), _p(_f32(background)), offset, seed, _p(img))
    return img.reshape(cam.res_y, cam.res_x, 3)


def pt_render_pixels(g: Grid, cam, pix, spp, max_depth, rr_depth, albedo, light_pos, light_e1, light_e2,
                     light_radiance, background, offset, seed) -> np.ndarray:
    """pt_render's values at the frame pixels pix only: (len(pix), 3)."""
    c = camera(cam)
    pix = _u32(pix)
    out = np.zeros(pix.size * 3, np.float32)
    lib().orc_pt_render_pixels(g.handle, _p(c), _p(_f32(cam.eye)), cam.res_x, cam.res_y, spp, max_depth,
                               rr_depth, albedo, _p(_f32(light_pos)), _p(_f32(light_e1)), _p(_f32(light_e2)),
                               _p(_f32(light_radiance)), _p(_f32(background)), offset, seed, _p(pix), pix.size,
                               _p(out))
    return out.reshape(-1, 3)


def compact(flags) -> np.ndarray:
    flags = _u32(flags)
    out = np.zeros(flags.size, np.uint32)
    m = lib().orc_compact(_p(flags), flags.size, _p(out))
    return out[:m]


DIRECT_CENTRES, REF_LEAF_POW = 1, 2


def set_reference_arithmetic(flags: int) -> None:
    """Switch the oracle's build to other arithmetic in the given places, to
    count how far it is from the canonical build: DIRECT_CENTRES (plane-test
    centres computed per cell instead of accumulated as the reference does),
    REF_LEAF_POW (the reference's powf leaf-resolution rule instead of the exact
    cube root); 0 restores the canonical build."""
    lib().orc_set_reference_arithmetic(int(flags))


def leaf_res_reference(g: Grid, lambda_leaf: float, threshold: int = 16) -> np.ndarray:
    """(C_top, 3) leaf resolutions as the reference's powf rule gives them, unclamped."""
    out = np.zeros((int(np.prod(g.res)), 3), np.uint32)
    lib().orc_leaf_res_reference(g.handle, lambda_leaf, threshold, _p(out))
    return out


def set_threads(n: int) -> None:
    lib().orc_set_threads(n)


def num_threads() -> int:
    return lib().orc_num_threads()
