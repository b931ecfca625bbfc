"""shinobi_b200: B200-native grid ray tracing (Python bindings of the C ABI).

The compute path lives in ``libshinobi_b200.so`` (hand-written sm_100a CUDA
behind the C ABI of ``include/shinobi_b200.h``).  This module is a thin
ctypes binding for tests, the benchmark and Python users; torch is used only
to hold device buffers and streams.  There is no CPU fallback: every call
goes to the CUDA library and raises ``ShinobiError`` on failure.

Names follow the reference's operator surface: a ``FaceSoup`` holds the
triangles (FaceSoup<frame>), ``Grid.build`` plays FastSimpleGridBuilder /
FastTwoLevelGridBuilder, ``Grid.trace_*`` play the grid traversers with the
intersector, and ``Grid.trace_primary`` / ``Grid.trace_ao`` / ``Grid.shade_direct`` the ray
generators with the trace<> kernel.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _abi
from ._abi import (SHN_GRID_TWO_LEVEL, SHN_GRID_UNIFORM, SHN_INSERT_PLANE, SHN_INSERT_SAT, SHN_MEM_DEVICE,
                   SHN_MEM_HOST, SHN_MISS, GridInfo, GridParams)

__all__ = ["ShinobiError", "Context", "FaceSoup", "Grid", "grid_params", "SHN_MISS",
           "SHN_GRID_UNIFORM", "SHN_GRID_TWO_LEVEL", "SHN_INSERT_PLANE", "SHN_INSERT_SAT", "exclusive_scan", "compact", "sort_keys",
           "camera_struct", "default_context", "read_obj", "read_camera", "read_light"]


class ShinobiError(RuntimeError):
    def __init__(self, status: int, msg: str = ""):
        self.status = status
        super().__init__(f"{_abi.STATUS.get(status, status)}: {msg}")


def _torch():
    import torch  # noqa: PLC0415  (torch is plumbing: device buffers and streams)
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def _stream(stream):
    torch = _torch()
    if stream is None:
        stream = torch.cuda.current_stream()
    return C.c_void_p(stream.cuda_stream)


class Context:
    """One library context (device, stream-ordered memory pool, HBM budget)."""

    def __init__(self, device: int = 0, hbm_budget_bytes: int = 0):
        self.lib = _abi.load()
        h = C.c_void_p()
        st = self.lib.shn_ctx_create(device, hbm_budget_bytes, C.byref(h))
        if st != 0:
            raise ShinobiError(st, "shn_ctx_create")
        self.handle = h
        self.device = device

    def check(self, st: int, what: str):
        if st != 0:
            msg = self.lib.shn_ctx_last_error(self.handle)
            raise ShinobiError(st, f"{what}: {msg.decode() if msg else ''}")

    def sync_status(self, stream=None):
        """Synchronise the stream and raise ShinobiError (SHN_ERR_TIMEOUT) if a
        bounded device wait gave up in a scan, compaction or sort on this
        context since the last check."""
        self.check(self.lib.shn_ctx_sync_status(self.handle, _stream(stream)), "shn_ctx_sync_status")

    def memory(self):
        used, budget = C.c_uint64(), C.c_uint64()
        self.check(self.lib.shn_ctx_memory(self.handle, C.byref(used), C.byref(budget)), "memory")
        return used.value, budget.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.shn_ctx_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_default_ctx = None


def default_context() -> Context:
    global _default_ctx
    if _default_ctx is None:
        _default_ctx = Context(0)
    return _default_ctx


class FaceSoup:
    """Triangle storage on the device (FaceSoup::upload / uploadVertices)."""

    def __init__(self, vertices, indices, ctx: Context | None = None, stream=None):
        self.ctx = ctx or default_context()
        lib = self.ctx.lib
        h = C.c_void_p()
        if isinstance(vertices, np.ndarray):
            v = np.ascontiguousarray(vertices, np.float32)
            i = np.ascontiguousarray(indices, np.uint32)
            st = lib.shn_scene_create(self.ctx.handle, v.ctypes.data_as(C.c_void_p), v.shape[0],
                                      i.ctypes.data_as(C.c_void_p), i.shape[0], SHN_MEM_HOST,
                                      _stream(stream), C.byref(h))
        else:
            v, i = vertices.contiguous(), indices.contiguous()
            st = lib.shn_scene_create(self.ctx.handle, _ptr(v), v.shape[0], _ptr(i), i.shape[0],
                                      SHN_MEM_DEVICE, _stream(stream), C.byref(h))
        self.ctx.check(st, "shn_scene_create")
        self.handle = h
        self.num_triangles = int(indices.shape[0])
        self.num_vertices = int(vertices.shape[0])

    def update_vertices(self, vertices, stream=None):
        lib = self.ctx.lib
        if isinstance(vertices, np.ndarray):
            v = np.ascontiguousarray(vertices, np.float32)
            st = lib.shn_scene_update_vertices(self.handle, v.ctypes.data_as(C.c_void_p), v.shape[0],
                                               SHN_MEM_HOST, _stream(stream))
        else:
            v = vertices.contiguous()
            st = lib.shn_scene_update_vertices(self.handle, _ptr(v), v.shape[0], SHN_MEM_DEVICE,
                                               _stream(stream))
        self.ctx.check(st, "shn_scene_update_vertices")

    def interpolate_vertices(self, kf1, kf2, coeff: float, stream=None):
        """Vertices = kf1 * (1 - coeff) + kf2 * coeff on the device (FaceSoup::uploadVertices of
        the reference's dynamic engine); kf1 (n1, 3) may be shorter than kf2 (nv, 3): the rest
        take kf2.  Both are device tensors."""
        kf1 = kf1.contiguous()
        kf2 = kf2.contiguous()
        self.ctx.check(self.ctx.lib.shn_scene_interpolate_vertices(
            self.handle, _ptr(kf1), kf1.shape[0], _ptr(kf2), float(coeff), _stream(stream)),
            "shn_scene_interpolate_vertices")

    @property
    def bounds(self) -> np.ndarray:
        out = (C.c_float * 6)()
        self.ctx.check(self.ctx.lib.shn_scene_bounds(self.handle, out), "bounds")
        return np.array(out[:], np.float32)

    def sah_resolution(self, lambda_: float = 5.0, window=(0.75, 1.25), counts: bool = False, stream=None):
        """SAHGridBuilder::computeResolution: the least-cost resolution of the window around the
        lambda estimate.  Returns a dict (res, res_min, res_max, cost, refs, num_tested[, counts]);
        counts is indexed [z, y, x] over the window."""
        r = _abi.SahResult()
        buf, cap = None, 0
        if counts:
            probe = _abi.SahResult()
            self.ctx.check(self.ctx.lib.shn_grid_sah_resolution(self.handle, lambda_, window[0], window[1], None,
                                                                 0, C.byref(probe), _stream(stream)),
                           "shn_grid_sah_resolution")
            cap = int(probe.num_tested)
            buf = np.zeros(cap, np.uint64)
        self.ctx.check(self.ctx.lib.shn_grid_sah_resolution(
            self.handle, lambda_, window[0], window[1],
            None if buf is None else buf.ctypes.data_as(C.c_void_p), cap, C.byref(r), _stream(stream)),
            "shn_grid_sah_resolution")
        out = {"res": tuple(r.res), "res_min": tuple(r.res_min), "res_max": tuple(r.res_max),
               "cost": float(r.cost), "refs": int(r.refs), "num_tested": int(r.num_tested)}
        if buf is not None:
            n = [out["res_max"][a] - out["res_min"][a] + 1 for a in range(3)]
            out["counts"] = buf.reshape(n[2], n[1], n[0])
        return out

    def sah_cost(self, resolutions, stream=None):
        """(refs, cost) arrays of the SAH cost of each (rx, ry, rz) in `resolutions` (<= 32)."""
        res = np.ascontiguousarray(np.asarray(resolutions, np.int32).reshape(-1, 3))
        k = res.shape[0]
        refs = np.zeros(k, np.uint64)
        cost = np.zeros(k, np.float32)
        self.ctx.check(self.ctx.lib.shn_grid_sah_cost(self.handle, res.ctypes.data_as(C.c_void_p), k,
                                                      refs.ctypes.data_as(C.c_void_p),
                                                      cost.ctypes.data_as(C.c_void_p), _stream(stream)),
                       "shn_grid_sah_cost")
        return refs, cost

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.shn_scene_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def grid_params(kind: int = SHN_GRID_UNIFORM, lambda_: float | None = None, top_divisor=None,
                min_res=None, lambda_leaf=None, leaf_threshold=None, res=None, insertion=None) -> GridParams:
    p = GridParams()
    _abi.load().shn_grid_params_default(kind, C.byref(p))
    if lambda_ is not None:
        p.lambda_ = lambda_
    if top_divisor is not None:
        p.top_divisor = top_divisor
    if min_res is not None:
        p.min_res = min_res
    if lambda_leaf is not None:
        p.lambda_leaf = lambda_leaf
    if leaf_threshold is not None:
        p.leaf_threshold = leaf_threshold
    if res is not None:
        for k in range(3):
            p.res[k] = int(res[k])
    if insertion is not None:
        p.insertion = int(insertion)
    return p


def pt_params(**kw) -> _abi.PtParams:
    """Path tracer parameters (defaults: 16 spp, depth 4, roulette from depth 2, albedo 0.7)."""
    p = _abi.PtParams()
    _abi.load().shn_pt_params_default(C.byref(p))
    for k, v in kw.items():
        if isinstance(v, (tuple, list)):
            arr = getattr(p, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(p, k, v)
    return p


def di_params(light=None, tri_material=None, diffuse=None, **kw) -> _abi.DiParams:
    """Direct-illumination parameters (defaults: 4 shadow rays per pixel, seed 1,
    a 0.1 x 0.1 light facing down at y = 0.2, diffuse 0.7, the reference's
    background).  ``light`` is a dict of AreaLight fields; ``tri_material``
    (uint32 per triangle) and ``diffuse`` ((num_materials, 4) float32) are
    device tensors that must stay alive until the call's work has run."""
    p = _abi.DiParams()
    _abi.load().shn_di_params_default(C.byref(p))
    for k, v in (light or {}).items():
        arr = getattr(p.light, k)
        for i, x in enumerate(v):
            arr[i] = x
    if tri_material is not None:
        p.tri_material = _ptr(tri_material)
    if diffuse is not None:
        p.diffuse = _ptr(diffuse)
        p.num_materials = int(diffuse.shape[0])
    for k, v in kw.items():
        if isinstance(v, (tuple, list)):
            arr = getattr(p, k)
            for i, x in enumerate(v):
                arr[i] = x
        else:
            setattr(p, k, v)
    return p


def camera_struct(cam) -> _abi.Camera:
    c = _abi.Camera()
    for k in range(3):
        c.eye[k] = cam.eye[k]
        c.forward[k] = cam.forward[k]
        c.up[k] = cam.up[k]
    c.fov_deg = cam.fov_deg
    c.res_x = cam.res_x
    c.res_y = cam.res_y
    return c


@dataclass
class HitBuffers:
    tri: object
    t: object
    u: object
    v: object

    def struct(self) -> _abi.Hits:
        return _abi.Hits(_ptr(self.tri), _ptr(self.t), _ptr(self.u), _ptr(self.v))


def alloc_hits(n: int, device="cuda", uv: bool = True) -> HitBuffers:
    torch = _torch()
    return HitBuffers(torch.empty(n, dtype=torch.int32, device=device),
                      torch.empty(n, dtype=torch.float32, device=device),
                      torch.empty(n, dtype=torch.float32, device=device) if uv else None,
                      torch.empty(n, dtype=torch.float32, device=device) if uv else None)


class Grid:
    """Uniform or two-level grid over a FaceSoup (build + traversal)."""

    def __init__(self, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.shn_grid_create(self.ctx.handle, C.byref(h)), "shn_grid_create")
        self.handle = h
        self.scene = None

    def build(self, scene: FaceSoup, params: GridParams, stream=None) -> "Grid":
        self.ctx.check(self.ctx.lib.shn_grid_build(self.handle, scene.handle, C.byref(params),
                                                   _stream(stream)), "shn_grid_build")
        self.scene = scene  # traces read the scene's triangles (hit records, AO and shading normals)
        return self

    def sync_status(self, stream=None):
        """Synchronise the stream and raise ShinobiError (SHN_ERR_TIMEOUT) if a
        bounded device wait gave up in a trace, AO, direct-illumination or
        path-tracer call on this grid since the last check."""
        self.ctx.check(self.ctx.lib.shn_grid_sync_status(self.handle, _stream(stream)), "shn_grid_sync_status")

    def info(self) -> GridInfo:
        inf = GridInfo()
        self.ctx.check(self.ctx.lib.shn_grid_get_info(self.handle, C.byref(inf)), "shn_grid_get_info")
        return inf

    def export(self):
        """-> dict(cells (C,2), leaves (L,2), indices (K,), top_pairs) as numpy uint arrays."""
        inf = self.info()
        cells = np.zeros((inf.num_cells, 2), np.uint32)
        leaves = np.zeros((inf.num_leaves, 2), np.uint32)
        indices = np.zeros(inf.num_refs, np.uint32)
        ntp = inf.num_top_refs if inf.kind == SHN_GRID_TWO_LEVEL else inf.num_refs
        top = np.zeros(ntp, np.uint64)
        self.ctx.check(self.ctx.lib.shn_grid_export(
            self.handle, cells.ctypes.data_as(C.c_void_p), leaves.ctypes.data_as(C.c_void_p),
            indices.ctypes.data_as(C.c_void_p), top.ctypes.data_as(C.c_void_p)), "shn_grid_export")
        return {"cells": cells, "leaves": leaves, "indices": indices, "top_pairs": top,
                "res": np.array(inf.res[:], np.int32), "bounds": np.array(inf.bounds[:], np.float32)}

    @staticmethod
    def _rays(org, dirs, tmax):
        cols = [org[:, k].contiguous() for k in range(3)] + [dirs[:, k].contiguous() for k in range(3)]
        r = _abi.Rays(*[_ptr(c) for c in cols], _ptr(tmax.contiguous()) if tmax is not None else None)
        return r, cols

    def trace_closest(self, org, dirs, tmax=None, out: HitBuffers | None = None, stream=None) -> HitBuffers:
        n = org.shape[0]
        out = out or alloc_hits(n, org.device)
        r, keep = self._rays(org, dirs, tmax)
        h = out.struct()
        self.ctx.check(self.ctx.lib.shn_trace_closest(self.handle, C.byref(r), n, C.byref(h),
                                                      _stream(stream)), "shn_trace_closest")
        return out

    def trace_any(self, org, dirs, tmax, out=None, stream=None):
        torch = _torch()
        n = org.shape[0]
        out = out if out is not None else torch.empty(n, dtype=torch.uint8, device=org.device)
        r, keep = self._rays(org, dirs, tmax)
        self.ctx.check(self.ctx.lib.shn_trace_any(self.handle, C.byref(r), n, _ptr(out),
                                                  _stream(stream)), "shn_trace_any")
        return out

    def trace_primary(self, cam, image_id: int = 0, out: HitBuffers | None = None, stream=None) -> HitBuffers:
        n = cam.res_x * cam.res_y
        out = out or alloc_hits(n)
        c = camera_struct(cam)
        h = out.struct()
        self.ctx.check(self.ctx.lib.shn_trace_primary(self.handle, C.byref(c), image_id, C.byref(h),
                                                      _stream(stream)), "shn_trace_primary")
        return out

    def trace_ao(self, cam, primary: HitBuffers, spp: int, length: float, offset: float, seed: int,
                 out=None, num_rays=None, stream=None):
        torch = _torch()
        n = cam.res_x * cam.res_y
        out = out if out is not None else torch.empty(n, dtype=torch.float32, device="cuda")
        c = camera_struct(cam)
        h = primary.struct()
        self.ctx.check(self.ctx.lib.shn_trace_ao(self.handle, C.byref(c), C.byref(h), spp, length,
                                                 offset, seed, _ptr(out), _ptr(num_rays),
                                                 _stream(stream)), "shn_trace_ao")
        return out

    def shade_direct(self, cam, primary: HitBuffers, params=None, frame=None, final=None, num_rays=None,
                     stream=None):
        """Area-light direct illumination of the primary hits; returns the
        (res_y, res_x, 3) frame (device).  ``final``, when given, receives the
        progressive blend with weight 1 / (image_id + 1)."""
        torch = _torch()
        p = params or di_params()
        frame = frame if frame is not None else torch.empty(cam.res_y, cam.res_x, 3, dtype=torch.float32,
                                                            device="cuda")
        c = camera_struct(cam)
        h = primary.struct()
        self.ctx.check(self.ctx.lib.shn_shade_direct(self.handle, C.byref(c), C.byref(h), C.byref(p),
                                                     _ptr(frame), _ptr(final), _ptr(num_rays),
                                                     _stream(stream)), "shn_shade_direct")
        return frame

    def pt_render(self, scene: FaceSoup, cam, params=None, out=None, stats=None, stream=None):
        """Wavefront path tracer; returns the (res_y, res_x, 3) mean-radiance image (device)."""
        torch = _torch()
        p = params or pt_params()
        out = out if out is not None else torch.empty(cam.res_y, cam.res_x, 3, dtype=torch.float32,
                                                      device="cuda")
        c = camera_struct(cam)
        self.ctx.check(self.ctx.lib.shn_pt_render(self.handle, scene.handle, C.byref(c), C.byref(p),
                                                  _ptr(out), _ptr(stats), _stream(stream)),
                       "shn_pt_render")
        return out

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.shn_grid_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class DynamicEngine:
    """Rebuild of the next frame overlapped with the render of the current one
    (DynamicRTEngine): two frame slots with their own scene, grid and stream."""

    def __init__(self, vertices, indices, params: GridParams, ctx: Context | None = None):
        self.ctx = ctx or default_context()
        h = C.c_void_p()
        if isinstance(vertices, np.ndarray):
            v = np.ascontiguousarray(vertices, np.float32)
            i = np.ascontiguousarray(indices, np.uint32)
            st = self.ctx.lib.shn_dynamic_create(self.ctx.handle, v.ctypes.data_as(C.c_void_p), v.shape[0],
                                                 i.ctypes.data_as(C.c_void_p), i.shape[0], SHN_MEM_HOST,
                                                 C.byref(params), C.byref(h))
        else:
            v, i = vertices.contiguous(), indices.contiguous()
            st = self.ctx.lib.shn_dynamic_create(self.ctx.handle, _ptr(v), v.shape[0], _ptr(i), i.shape[0],
                                                 SHN_MEM_DEVICE, C.byref(params), C.byref(h))
        self.ctx.check(st, "shn_dynamic_create")
        self.handle = h

    def render_frame(self, kf1, kf2, coeff: float, cam, di, hits: HitBuffers, frame, final=None):
        """Renders the previous call's geometry and prepares kf1*(1-coeff)+kf2*coeff
        (device tensors (n, 3)); returns (render_ms, build_ms, frame_ms)."""
        kf1 = kf1.contiguous()
        kf2 = kf2.contiguous()
        c = camera_struct(cam)
        hs = hits.struct()
        t = [C.c_float(), C.c_float(), C.c_float()]
        self.ctx.check(self.ctx.lib.shn_dynamic_render_frame(
            self.handle, _ptr(kf1), kf1.shape[0], _ptr(kf2), float(coeff), C.byref(c), C.byref(di), C.byref(hs),
            _ptr(frame), _ptr(final), C.byref(t[0]), C.byref(t[1]), C.byref(t[2])), "shn_dynamic_render_frame")
        return t[0].value, t[1].value, t[2].value

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.shn_dynamic_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Batch:
    """Many scenes built by one fused pipeline and traced by one launch (uniform grids)."""

    def __init__(self, scenes_list, ctx: Context | None = None, stream=None):
        self.ctx = ctx or default_context()
        vo = np.zeros(len(scenes_list) + 1, np.uint32)
        to = np.zeros(len(scenes_list) + 1, np.uint32)
        for i, sc in enumerate(scenes_list):
            vo[i + 1] = vo[i] + sc.vertices.shape[0]
            to[i + 1] = to[i] + sc.indices.shape[0]
        v = np.ascontiguousarray(np.concatenate([sc.vertices for sc in scenes_list]), np.float32)
        ix = np.ascontiguousarray(np.concatenate([sc.indices for sc in scenes_list]), np.uint32)
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.shn_batch_create(
            self.ctx.handle, len(scenes_list), v.ctypes.data_as(C.c_void_p), vo.ctypes.data_as(C.c_void_p),
            ix.ctypes.data_as(C.c_void_p), to.ctypes.data_as(C.c_void_p), SHN_MEM_HOST, _stream(stream),
            C.byref(h)), "shn_batch_create")
        self.handle = h
        self.num_scenes = len(scenes_list)
        self.tri_offsets = to

    def set_lambdas(self, lambdas):
        a = np.ascontiguousarray(lambdas, np.float32)
        self.ctx.check(self.ctx.lib.shn_batch_set_lambdas(self.handle, a.ctypes.data_as(C.c_void_p)),
                       "shn_batch_set_lambdas")

    def autotune(self, candidates, expected_rays, sample_rays=16384, seed=7, stream=None):
        c = np.ascontiguousarray(candidates, np.float32)
        e = np.ascontiguousarray(expected_rays, np.uint32)
        out = np.zeros(self.num_scenes, np.float32)
        self.ctx.check(self.ctx.lib.shn_batch_autotune(
            self.handle, c.ctypes.data_as(C.c_void_p), c.size, e.ctypes.data_as(C.c_void_p), sample_rays,
            seed, out.ctypes.data_as(C.c_void_p), _stream(stream)), "shn_batch_autotune")
        return out

    def autotune_ex(self, candidates, expected_rays, sample_rays=16384, seed=7, sah_keep=0,
                    blocks_per_sm=(), sort_tiles=(), stream=None):
        """The autotuner with the SAH pruning term (time only the sah_keep candidates of least SAH
        cost per scene) and the trace kernel's blocks per SM as a timed term.
        -> (chosen lambdas, SAH cost of each, report dict)."""
        c = np.ascontiguousarray(candidates, np.float32)
        e = np.ascontiguousarray(expected_rays, np.uint32)
        cfg = _abi.AutotuneConfig()
        cfg.sah_keep = sah_keep
        cfg.num_block_shapes = len(blocks_per_sm)
        for i, v in enumerate(blocks_per_sm):
            cfg.blocks_per_sm[i] = int(v)
        cfg.num_sort_tiles = len(sort_tiles)
        for i, v in enumerate(sort_tiles):
            cfg.sort_tile_keys[i] = int(v)
        rep = _abi.AutotuneReport()
        out = np.zeros(self.num_scenes, np.float32)
        sah = np.zeros(self.num_scenes, np.float32)
        self.ctx.check(self.ctx.lib.shn_batch_autotune_ex(
            self.handle, c.ctypes.data_as(C.c_void_p), c.size, e.ctypes.data_as(C.c_void_p), sample_rays,
            seed, C.byref(cfg), out.ctypes.data_as(C.c_void_p), sah.ctypes.data_as(C.c_void_p), C.byref(rep),
            _stream(stream)), "shn_batch_autotune_ex")
        report = {"timed_candidates": int(rep.timed_candidates), "blocks_per_sm": int(rep.blocks_per_sm),
                  "shape_ms": [float(x) for x in rep.shape_ms[:len(blocks_per_sm)]],
                  "sort_tile_keys": int(rep.sort_tile_keys),
                  "sort_tile_ms": [float(x) for x in rep.sort_tile_ms[:len(sort_tiles)]]}
        return out, sah, report

    def build(self, stream=None):
        self.ctx.check(self.ctx.lib.shn_batch_build(self.handle, _stream(stream)), "shn_batch_build")
        return self

    def info(self):
        p, c, ms = C.c_uint64(), C.c_uint64(), C.c_float()
        self.ctx.check(self.ctx.lib.shn_batch_info(self.handle, C.byref(p), C.byref(c), C.byref(ms)),
                       "shn_batch_info")
        return {"num_pairs": p.value, "total_cells": c.value, "build_ms": ms.value}

    def trace(self, org, dirs, ray_offsets, tmax=None, out: HitBuffers | None = None, any_hit=False,
              stream=None):
        torch = _torch()
        n = org.shape[0]
        r, keep = Grid._rays(org, dirs, tmax)
        ro = np.ascontiguousarray(ray_offsets, np.uint32)
        if any_hit:
            occ = torch.empty(n, dtype=torch.uint8, device=org.device)
            self.ctx.check(self.ctx.lib.shn_batch_trace(self.handle, C.byref(r), ro.ctypes.data_as(C.c_void_p),
                                                        None, _ptr(occ), _stream(stream)), "shn_batch_trace")
            return occ
        out = out or alloc_hits(n, org.device)
        h = out.struct()
        self.ctx.check(self.ctx.lib.shn_batch_trace(self.handle, C.byref(r), ro.ctypes.data_as(C.c_void_p),
                                                    C.byref(h), None, _stream(stream)), "shn_batch_trace")
        return out

    def capture(self, org, dirs, ray_offsets, out: HitBuffers, stream=None):
        """Capture build + trace into a CUDA graph; keeps the ray columns alive."""
        r, self._graph_cols = Grid._rays(org, dirs, None)
        self._graph_ro = np.ascontiguousarray(ray_offsets, np.uint32)
        h = out.struct()
        self.ctx.check(self.ctx.lib.shn_batch_capture(self.handle, C.byref(r),
                                                      self._graph_ro.ctypes.data_as(C.c_void_p),
                                                      C.byref(h), _stream(stream)), "shn_batch_capture")

    def replay(self, stream=None):
        self.ctx.check(self.ctx.lib.shn_batch_replay(self.handle, _stream(stream)), "shn_batch_replay")

    def sync_status(self, stream=None):
        """Synchronise and raise ShinobiError if a bounded wait gave up (or a replay
        overflowed its planned pairs) in this batch since the last check."""
        self.ctx.check(self.ctx.lib.shn_batch_sync_status(self.handle, _stream(stream)), "shn_batch_sync_status")

    def export_scene(self, s: int, max_cells: int, max_refs: int):
        res = (C.c_int32 * 3)()
        b = (C.c_float * 6)()
        cells = np.zeros(2 * max_cells, np.uint32)
        idx = np.zeros(max(1, max_refs), np.uint32)
        nref = C.c_uint64()
        self.ctx.check(self.ctx.lib.shn_batch_export_scene(self.handle, s, res, b, cells.ctypes.data_as(C.c_void_p),
                                                           idx.ctypes.data_as(C.c_void_p), C.byref(nref)),
                       "shn_batch_export_scene")
        r = np.array(res[:], np.int32)
        nc = int(np.prod(r))
        return {"res": r, "bounds": np.array(b[:], np.float32), "cells": cells[:2 * nc].reshape(-1, 2),
                "indices": idx[:nref.value]}

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.shn_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Ray-query server (continuous batching over resident grids)."""

    def __init__(self, ctx: Context | None = None, num_slots=64, max_batch_rays=4 << 20,
                 max_requests_per_launch=4096, max_queue=0, coalesce=True):
        self.ctx = ctx or default_context()
        cfg = _abi.ServerConfig()
        self.ctx.lib.shn_server_config_default(C.byref(cfg))
        cfg.num_slots, cfg.max_batch_rays = num_slots, max_batch_rays
        cfg.max_requests_per_launch, cfg.max_queue, cfg.coalesce = max_requests_per_launch, max_queue, int(coalesce)
        h = C.c_void_p()
        self.ctx.check(self.ctx.lib.shn_server_create(self.ctx.handle, C.byref(cfg), C.byref(h)), "shn_server_create")
        self.handle = h
        self._keep = {}

    def load_scene(self, slot, scene, lambda_=5.0):
        v = np.ascontiguousarray(scene.vertices, np.float32)
        i = np.ascontiguousarray(scene.indices, np.uint32)
        self.ctx.check(self.ctx.lib.shn_server_load_scene(self.handle, slot, v.ctypes.data_as(C.c_void_p), v.shape[0],
                                                          i.ctypes.data_as(C.c_void_p), i.shape[0], lambda_),
                       "shn_server_load_scene")

    @staticmethod
    def ray_request(kind, slot, rays8, out_tri=None, out_t=None) -> _abi.Request:
        """rays8: (n, 8) float32 host array (pinned for overlap): ox oy oz dx dy dz tmax pad."""
        r = _abi.Request()
        r.kind, r.scene, r.num_rays = kind, slot, rays8.shape[0]
        r.rays = rays8.ctypes.data_as(C.c_void_p) if isinstance(rays8, np.ndarray) else C.c_void_p(rays8.data_ptr())
        if out_tri is not None:
            r.out_tri = out_tri.ctypes.data_as(C.c_void_p) if isinstance(out_tri, np.ndarray) else C.c_void_p(out_tri.data_ptr())
        if out_t is not None:
            r.out_t = out_t.ctypes.data_as(C.c_void_p) if isinstance(out_t, np.ndarray) else C.c_void_p(out_t.data_ptr())
        return r

    def update_request(self, slot, scene, lambda_=5.0) -> _abi.Request:
        v = np.ascontiguousarray(scene.vertices, np.float32)
        i = np.ascontiguousarray(scene.indices, np.uint32)
        self._keep[id(v)] = (v, i)
        r = _abi.Request()
        r.kind, r.scene = _abi.SHN_REQ_UPDATE, slot
        r.vtx, r.nv = v.ctypes.data_as(C.c_void_p), v.shape[0]
        r.idx, r.nt = i.ctypes.data_as(C.c_void_p), i.shape[0]
        r.lambda_ = lambda_
        return r

    def submit(self, req) -> int:
        t = C.c_uint64()
        self.ctx.check(self.ctx.lib.shn_server_submit(self.handle, C.byref(req), C.byref(t)), "shn_server_submit")
        return t.value

    def wait(self, ticket, timeout_ms=60000) -> int:
        res = C.c_int32()
        st = self.ctx.lib.shn_server_wait(self.handle, ticket, timeout_ms, C.byref(res))
        self.ctx.check(st, "shn_server_wait")
        return res.value

    def run_schedule(self, reqs, arrival_s):
        arr = (_abi.Request * len(reqs))(*reqs)
        t = np.ascontiguousarray(arrival_s, np.float64)
        res = np.zeros(len(reqs), np.int32)
        self.ctx.lib.shn_server_run_schedule(self.handle, len(reqs), arr, t.ctypes.data_as(C.c_void_p),
                                            res.ctypes.data_as(C.c_void_p))
        return res

    def stats(self, reset=False) -> dict:
        st = _abi.ServerStats()
        self.ctx.check(self.ctx.lib.shn_server_get_stats(self.handle, C.byref(st), int(reset)), "shn_server_get_stats")
        return {k: getattr(st, k) for k, _ in _abi.ServerStats._fields_}

    def records(self):
        """Per-request records since the last stats reset (completion order) as a numpy
        structured array: submit_s, latency_us, kind, scene, num_rays, status."""
        n = C.c_uint32()
        self.ctx.check(self.ctx.lib.shn_server_get_records(self.handle, 0, None, C.byref(n)), "records")
        buf = (_abi.RequestRecord * max(1, n.value))()
        self.ctx.check(self.ctx.lib.shn_server_get_records(self.handle, n.value, buf, C.byref(n)), "records")
        dt = np.dtype([("submit_s", "f8"), ("latency_us", "f8"), ("kind", "u4"), ("scene", "u4"),
                       ("num_rays", "u4"), ("status", "i4")])
        return np.frombuffer(bytes(buf), dtype=dt, count=n.value).copy()

    def drain(self, timeout_ms=600000):
        self.ctx.check(self.ctx.lib.shn_server_drain(self.handle, timeout_ms), "shn_server_drain")

    def close(self):
        if getattr(self, "handle", None):
            self.ctx.lib.shn_server_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---- scene files ------------------------------------------------------------------
def read_obj(path: str) -> dict:
    """Wavefront OBJ + MTL with the reference's parsing rules (FWObject::read):
    dict(vertices (nv,3) float32, indices (nf,3) uint32, face_material (nf,)
    uint32, diffuse (nm,4) float32 (Phong-normalised, .w 0), specular (nm,4)
    (.w = Ns), material_names, skipped_lines)."""
    lib = _abi.load()
    h = C.c_void_p()
    st = lib.shn_obj_read(str(path).encode(), C.byref(h))
    if st != 0:
        raise ShinobiError(st, f"shn_obj_read {path}")
    try:
        inf = _abi.ObjInfo()
        lib.shn_obj_get_info(h, C.byref(inf))
        v = np.zeros((inf.num_vertices, 3), np.float32)
        f = np.zeros((inf.num_faces, 3), np.uint32)
        fm = np.zeros(inf.num_faces, np.uint32)
        d = np.zeros((inf.num_materials, 4), np.float32)
        sp = np.zeros((inf.num_materials, 4), np.float32)
        lib.shn_obj_copy(h, v.ctypes.data_as(C.c_void_p), f.ctypes.data_as(C.c_void_p),
                         fm.ctypes.data_as(C.c_void_p), d.ctypes.data_as(C.c_void_p), sp.ctypes.data_as(C.c_void_p))
        names = [lib.shn_obj_material_name(h, m).decode() for m in range(inf.num_materials)]
        return {"vertices": v, "indices": f, "face_material": fm, "diffuse": d, "specular": sp,
                "material_names": names, "skipped_lines": int(inf.skipped_lines),
                "num_normals": int(inf.num_normals), "num_texcoords": int(inf.num_texcoords)}
    finally:
        lib.shn_obj_destroy(h)


def read_camera(path: str, defaults=None):
    """camera.cfg with the reference's rules (CameraManager::read): returns a
    scenes.Camera; entries missing from the file keep the defaults' values."""
    from .scenes import Camera
    lib = _abi.load()
    # the reference's CameraManager defaults: position 0, orientation +z, up -y, 512x512, 66 degrees
    defaults = defaults or Camera((0.0, 0.0, 0.0), (0.0, 0.0, 1.0), (0.0, -1.0, 0.0), 66.0, 512, 512)
    c = camera_struct(defaults)
    st = lib.shn_camera_read(str(path).encode(), C.byref(c))
    if st != 0:
        raise ShinobiError(st, f"shn_camera_read {path}")
    return Camera(tuple(c.eye), tuple(c.forward), tuple(c.up), float(c.fov_deg), int(c.res_x), int(c.res_y))


def read_light(path: str) -> dict:
    """light.cfg with the reference's rules (LightSourceLoader::loadFromFile): a
    dict of the area light's fields, usable as di_params(light=...)."""
    lib = _abi.load()
    l = _abi.AreaLight()
    st = lib.shn_light_read(str(path).encode(), C.byref(l))
    if st != 0:
        raise ShinobiError(st, f"shn_light_read {path}")
    return {k: tuple(getattr(l, k)) for k in ("position", "edge1", "edge2", "normal", "intensity")}


def exclusive_scan(x, ctx: Context | None = None, stream=None):
    """uint32 exclusive scan; returns n+1 values (last = total)."""
    torch = _torch()
    ctx = ctx or default_context()
    out = torch.empty(x.numel() + 1, dtype=torch.int32, device=x.device)
    ctx.check(ctx.lib.shn_exclusive_scan_u32(ctx.handle, _ptr(x), _ptr(out), x.numel(), _stream(stream)),
              "shn_exclusive_scan_u32")
    return out


def compact(flags, ctx: Context | None = None, stream=None):
    torch = _torch()
    ctx = ctx or default_context()
    out = torch.empty(max(1, flags.numel()), dtype=torch.int32, device=flags.device)
    cnt = torch.zeros(1, dtype=torch.int32, device=flags.device)
    ctx.check(ctx.lib.shn_compact_u32(ctx.handle, _ptr(flags), flags.numel(), _ptr(out), _ptr(cnt),
                                      _stream(stream)), "shn_compact_u32")
    return out[: int(cnt.item())]


def sort_keys(keys, lo_bit: int, hi_bit: int, ctx: Context | None = None, stream=None):
    """In-place stable radix sort of int64 keys on bits [lo_bit, hi_bit)."""
    torch = _torch()
    ctx = ctx or default_context()
    tmp = torch.empty_like(keys)
    ctx.check(ctx.lib.shn_sort_keys_u64(ctx.handle, _ptr(keys), _ptr(tmp), keys.numel(), lo_bit, hi_bit,
                                        _stream(stream)), "shn_sort_keys_u64")
    return keys
