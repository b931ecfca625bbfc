"""ctypes declarations of the C ABI in include/shinobi_b200.h."""
from __future__ import annotations

import ctypes as C
import os

from . import build as _build

vp = C.c_void_p
u32 = C.c_uint32
u64 = C.c_uint64
i32 = C.c_int
f32 = C.c_float

STATUS = {
    0: "SHN_OK", 1: "SHN_ERR_INVALID", 2: "SHN_ERR_CUDA", 3: "SHN_ERR_OOM", 4: "SHN_ERR_TIMEOUT",
    5: "SHN_ERR_BUDGET", 6: "SHN_ERR_NOT_BUILT", 7: "SHN_ERR_BUSY", 8: "SHN_ERR_CANCELLED",
}

SHN_OK, SHN_ERR_INVALID, SHN_ERR_CUDA, SHN_ERR_OOM, SHN_ERR_TIMEOUT = 0, 1, 2, 3, 4
SHN_ERR_BUDGET, SHN_ERR_NOT_BUILT, SHN_ERR_BUSY, SHN_ERR_CANCELLED = 5, 6, 7, 8

SHN_MISS = 0xFFFFFFFF
SHN_FORCE_CTX_SCAN, SHN_FORCE_GRID_COMPACTION, SHN_FORCE_NOALLOC_SCAN = 1, 2, 3
SHN_INSERT_PLANE, SHN_INSERT_SAT = 0, 1
SHN_MEM_HOST = 0
SHN_MEM_DEVICE = 1
SHN_GRID_UNIFORM = 0
SHN_GRID_TWO_LEVEL = 1


class GridParams(C.Structure):
    _fields_ = [("kind", u32), ("lambda_", f32), ("top_divisor", i32), ("min_res", i32),
                ("lambda_leaf", f32), ("leaf_threshold", u32), ("res", i32 * 3), ("insertion", u32)]


class GridInfo(C.Structure):
    _fields_ = [("kind", u32), ("res", i32 * 3), ("bounds", f32 * 6), ("cell_size", f32 * 3),
                ("num_cells", u64), ("num_top_refs", u64), ("num_leaves", u64), ("num_refs", u64),
                ("device_bytes", u64), ("build_ms", f32)]


class Rays(C.Structure):
    _fields_ = [("ox", vp), ("oy", vp), ("oz", vp), ("dx", vp), ("dy", vp), ("dz", vp), ("tmax", vp)]


class Hits(C.Structure):
    _fields_ = [("tri", vp), ("t", vp), ("u", vp), ("v", vp)]


class Camera(C.Structure):
    _fields_ = [("eye", f32 * 3), ("forward", f32 * 3), ("up", f32 * 3), ("fov_deg", f32),
                ("res_x", u32), ("res_y", u32)]


class PtParams(C.Structure):
    _fields_ = [("spp", u32), ("max_depth", u32), ("rr_depth", u32), ("albedo", f32),
                ("light_pos", f32 * 3), ("light_e1", f32 * 3), ("light_e2", f32 * 3),
                ("light_radiance", f32 * 3), ("background", f32 * 3), ("offset", f32), ("seed", u32)]


class AreaLight(C.Structure):
    _fields_ = [("position", f32 * 3), ("edge1", f32 * 3), ("edge2", f32 * 3), ("normal", f32 * 3),
                ("intensity", f32 * 3)]


class ObjInfo(C.Structure):
    _fields_ = [("num_vertices", u32), ("num_faces", u32), ("num_materials", u32), ("num_normals", u32),
                ("num_texcoords", u32), ("skipped_lines", u64)]


class SahResult(C.Structure):
    _fields_ = [("res", i32 * 3), ("res_min", i32 * 3), ("res_max", i32 * 3), ("cost", f32), ("refs", u64),
                ("num_tested", u64)]


class AutotuneConfig(C.Structure):
    _fields_ = [("sah_keep", u32), ("num_block_shapes", u32), ("blocks_per_sm", u32 * 8),
                ("num_sort_tiles", u32), ("sort_tile_keys", u32 * 4)]


class AutotuneReport(C.Structure):
    _fields_ = [("timed_candidates", u32), ("blocks_per_sm", u32), ("shape_ms", f32 * 8),
                ("sort_tile_keys", u32), ("sort_tile_ms", f32 * 4)]


class DiParams(C.Structure):
    _fields_ = [("light", AreaLight), ("samples", u32), ("seed", u32), ("image_id", u32),
                ("tri_material", vp), ("diffuse", vp), ("num_materials", u32),
                ("default_diffuse", f32 * 3), ("background", f32 * 3)]


class ServerConfig(C.Structure):
    _fields_ = [("num_slots", u32), ("max_batch_rays", u32), ("max_requests_per_launch", u32),
                ("max_queue", u32), ("coalesce", u32)]


class Request(C.Structure):
    _fields_ = [("kind", u32), ("scene", u32), ("num_rays", u32), ("rays", vp), ("out_tri", vp),
                ("out_t", vp), ("vtx", vp), ("nv", u32), ("idx", vp), ("nt", u32), ("lambda_", f32)]


class ServerStats(C.Structure):
    _fields_ = [("requests", u64), ("updates", u64), ("rays", u64), ("launches", u64),
                ("max_requests_per_launch", u64), ("p50_us", C.c_double), ("p99_us", C.c_double),
                ("max_us", C.c_double), ("mean_us", C.c_double), ("wall_s", C.c_double),
                ("mrays_per_s", C.c_double)]


class RequestRecord(C.Structure):
    _fields_ = [("submit_s", C.c_double), ("latency_us", C.c_double), ("kind", u32), ("scene", u32),
                ("num_rays", u32), ("status", C.c_int32)]


SHN_REQ_CLOSEST = 0
SHN_REQ_ANY = 1
SHN_REQ_UPDATE = 2

# name -> (argtypes, restype)
SIGNATURES = {
    "shn_abi_version": ([], u32),
    "shn_status_string": ([i32], C.c_char_p),
    "shn_ctx_create": ([i32, u64, C.POINTER(vp)], i32),
    "shn_ctx_destroy": ([vp], None),
    "shn_ctx_last_error": ([vp], C.c_char_p),
    "shn_ctx_memory": ([vp, C.POINTER(u64), C.POINTER(u64)], i32),
    "shn_scene_create": ([vp, vp, u32, vp, u32, u32, vp, C.POINTER(vp)], i32),
    "shn_scene_update_vertices": ([vp, vp, u32, u32, vp], i32),
    "shn_scene_bounds": ([vp, C.POINTER(f32)], i32),
    "shn_scene_interpolate_vertices": ([vp, vp, u32, vp, f32, vp], i32),
    "shn_scene_num_triangles": ([vp], u32),
    "shn_scene_destroy": ([vp], None),
    "shn_grid_params_default": ([u32, C.POINTER(GridParams)], None),
    "shn_grid_create": ([vp, C.POINTER(vp)], i32),
    "shn_grid_build": ([vp, vp, C.POINTER(GridParams), vp], i32),
    "shn_grid_sah_resolution": ([vp, f32, f32, f32, vp, u64, C.POINTER(SahResult), vp], i32),
    "shn_grid_sah_cost": ([vp, vp, u32, vp, vp, vp], i32),
    "shn_grid_get_info": ([vp, C.POINTER(GridInfo)], i32),
    "shn_grid_export": ([vp, vp, vp, vp, vp], i32),
    "shn_grid_destroy": ([vp], None),
    "shn_trace_closest": ([vp, C.POINTER(Rays), u32, C.POINTER(Hits), vp], i32),
    "shn_trace_any": ([vp, C.POINTER(Rays), u32, vp, vp], i32),
    "shn_trace_primary": ([vp, C.POINTER(Camera), u32, C.POINTER(Hits), vp], i32),
    "shn_trace_ao": ([vp, C.POINTER(Camera), C.POINTER(Hits), u32, f32, f32, u32, vp, vp, vp], i32),
    "shn_grid_set_stats": ([vp, vp], i32),
    "shn_batch_create": ([vp, u32, vp, vp, vp, vp, u32, vp, C.POINTER(vp)], i32),
    "shn_batch_set_lambdas": ([vp, vp], i32),
    "shn_batch_autotune": ([vp, vp, u32, vp, u32, u32, vp, vp], i32),
    "shn_batch_autotune_ex": ([vp, vp, u32, vp, u32, u32, C.POINTER(AutotuneConfig), vp, vp,
                               C.POINTER(AutotuneReport), vp], i32),
    "shn_batch_build": ([vp, vp], i32),
    "shn_batch_trace": ([vp, C.POINTER(Rays), vp, C.POINTER(Hits), vp, vp], i32),
    "shn_batch_capture": ([vp, C.POINTER(Rays), vp, C.POINTER(Hits), vp], i32),
    "shn_batch_replay": ([vp, vp], i32),
    "shn_batch_info": ([vp, vp, vp, vp], i32),
    "shn_batch_export_scene": ([vp, u32, vp, vp, vp, vp, vp], i32),
    "shn_batch_destroy": ([vp], None),
    "shn_server_config_default": ([C.POINTER(ServerConfig)], None),
    "shn_server_create": ([vp, C.POINTER(ServerConfig), C.POINTER(vp)], i32),
    "shn_server_load_scene": ([vp, u32, vp, u32, vp, u32, f32], i32),
    "shn_server_submit": ([vp, C.POINTER(Request), C.POINTER(u64)], i32),
    "shn_server_wait": ([vp, u64, u32, C.POINTER(i32)], i32),
    "shn_server_poll": ([vp, u64, C.POINTER(i32)], i32),
    "shn_server_drain": ([vp, u32], i32),
    "shn_server_get_stats": ([vp, C.POINTER(ServerStats), i32], i32),
    "shn_server_run_schedule": ([vp, u32, vp, vp, vp], i32),
    "shn_server_destroy": ([vp], None),
    "shn_di_params_default": ([C.POINTER(DiParams)], None),
    "shn_shade_direct": ([vp, C.POINTER(Camera), C.POINTER(Hits), C.POINTER(DiParams), vp, vp, vp, vp], i32),
    "shn_pt_params_default": ([C.POINTER(PtParams)], None),
    "shn_pt_render": ([vp, vp, C.POINTER(Camera), C.POINTER(PtParams), vp, vp, vp], i32),
    "shn_exclusive_scan_u32": ([vp, vp, vp, u32, vp], i32),
    "shn_exclusive_scan_u32_noalloc": ([vp, vp, u32, vp], i32),
    "shn_compact_u32": ([vp, vp, u32, vp, vp, vp], i32),
    "shn_selftest_lookback_timeout": ([vp, vp], i32),
    "shn_exclusive_scan_u32_noalloc_status": ([vp], i32),
    "shn_ctx_sync_status": ([vp, vp], i32),
    "shn_grid_sync_status": ([vp, vp], i32),
    "shn_batch_sync_status": ([vp, vp], i32),
    "shn_debug_force_lookback_timeout": ([u32, vp, vp], i32),
    "shn_dynamic_create": ([vp, vp, u32, vp, u32, u32, C.POINTER(GridParams), C.POINTER(vp)], i32),
    "shn_dynamic_render_frame": ([vp, vp, u32, vp, f32, C.POINTER(Camera), C.POINTER(DiParams), C.POINTER(Hits),
                                  vp, vp, vp, vp, vp], i32),
    "shn_dynamic_get_grid": ([vp, u32, C.POINTER(vp), C.POINTER(vp)], i32),
    "shn_dynamic_destroy": ([vp], None),
    "shn_obj_read": ([C.c_char_p, C.POINTER(vp)], i32),
    "shn_obj_get_info": ([vp, C.POINTER(ObjInfo)], i32),
    "shn_obj_copy": ([vp, vp, vp, vp, vp, vp], i32),
    "shn_obj_material_name": ([vp, u32], C.c_char_p),
    "shn_obj_destroy": ([vp], None),
    "shn_camera_read": ([C.c_char_p, C.POINTER(Camera)], i32),
    "shn_light_read": ([C.c_char_p, C.POINTER(AreaLight)], i32),
    "shn_server_get_records": ([vp, u32, vp, vp], i32),
    "shn_sort_keys_u64": ([vp, vp, vp, u32, u32, u32, vp], i32),
}

_lib = None


def load(auto_build: bool = True):
    """Load libshinobi_b200.so (building it first when missing or stale).

    SHINOBI_B200_LIB may name another build of the library to load instead."""
    global _lib
    if _lib is None:
        path = os.environ.get("SHINOBI_B200_LIB") or _build.LIB
        if path == _build.LIB and auto_build and _build.stale():
            _build.build()
        if not os.path.exists(path):
            raise RuntimeError(f"libshinobi_b200.so not built ({path})")
        lib = C.CDLL(path)
        for name, (args, res) in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = res
        _lib = lib
    return _lib
