/*
 * shinobi_b200 -- C ABI of the B200-native (sm_100a) grid ray-tracing path:
 * sort-based uniform and two-level grid construction, 3D-DDA traversal with a
 * watertight ray/triangle test, camera / ambient-occlusion ray generation and
 * the wavefront path tracer with stream compaction.
 *
 * Conventions
 *  - every call returns shn_status; shn_ctx_last_error() gives a message;
 *  - bounded device-side waits (look-back scans, bulk copies) that give up
 *    set an error bit instead of hanging.  Calls that synchronise (exports,
 *    builds up to their last stage) report it themselves; asynchronous calls
 *    (a build's last stage, traces, AO, direct
 *    illumination, the path tracer, scans, compaction, sorts, batch replays)
 *    leave it in a device word that shn_grid_sync_status /
 *    shn_ctx_sync_status / shn_batch_sync_status /
 *    shn_exclusive_scan_u32_noalloc_status report (SHN_ERR_TIMEOUT) and
 *    clear; the reference aborted through cutil's check macros instead;
 *  - pointers named d_* are device pointers owned by the caller; objects
 *    created by shn_*_create are owned by the library and released by the
 *    matching shn_*_destroy;
 *  - "stream" is a cudaStream_t (NULL = legacy default stream); all work of a
 *    call is ordered on it and calls return without synchronising unless a
 *    size must come back to the host (documented per call);
 *  - no global textures or __constant__ state: several grids and scenes may
 *    be alive and used concurrently from different streams; a ctx serialises
 *    its own bookkeeping with an internal lock.
 *
 * Reference interfaces replaced (jckarter/shinobi, paths within that tree):
 *  - FaceSoup<frame>::upload / uploadVertices      -> shn_scene_create / shn_scene_update_vertices
 *      (src/Control/Structure/FaceSoup.h:171-339)
 *  - FastSimpleGridBuilder::init/build/rebuild     -> shn_grid_build (SHN_GRID_UNIFORM)
 *      (src/Control/Algorithm/FastSimpleGridBuilder.h:59-452)
 *  - FastTwoLevelGridBuilder::init/build/rebuild   -> shn_grid_build (SHN_GRID_TWO_LEVEL)
 *      (src/Control/Algorithm/FastTwoLevelGridBuilder.h:61-740)
 *  - UniformGridTraverser / TwoLevelGridTraverser  -> shn_trace_closest
 *      (src/Control/Algorithm/SimpleGridTraverser.h:274-401,
 *       src/Control/Algorithm/TwoLevelGridTraverser.h:445-671)
 *  - *ShadowTraverser                               -> shn_trace_any
 *      (src/Control/Algorithm/SimpleGridTraverser.h:405-469,
 *       src/Control/Algorithm/TwoLevelGridTraverser.h:677-828)
 *  - trace<RegularPrimaryRayGenerator,...>          -> shn_trace_primary
 *      (src/Engine/RayTracingKernels.h:37-136, src/Engine/RayGenerators.h:36-61)
 *  - DirectIlluminationIntegrator::shade occlusion  -> shn_trace_ao (ambient occlusion)
 *    and shn_shade_direct (area light + computeDirectIllumination)
 *      (src/Integrator/DirectIlluminationIntegrator.h:254-315)
 *  - DynamicRTEngine::init / renderFrame          -> shn_dynamic_create / shn_dynamic_render_frame
 *      (src/Engine/DynamicRTEngine.h:49-158)
 *  - FWObject::read, CameraManager::read,
 *    LightSourceLoader::loadFromFile               -> shn_obj_read, shn_camera_read, shn_light_read
 *      (src/Loaders/FWObjectReader.cpp:96-502, src/Loaders/CameraManager.cpp:94-158,
 *       src/Loaders/LightSourceLoader.cpp:26-89)
 *  - SimplePathTracer / render megakernel           -> shn_pt_render
 *      (src/Integrator/SimplePathTracer.hpp:65-241, src/Shinobi.h:152-230)
 *  - InclusiveScan / ExclusiveScan / Sort           -> shn_exclusive_scan_u32 / shn_sort_keys_u64
 *      (src/Utils/Scan.h:35-68, src/Utils/Sort.h:33-48)
 *  - chag::pp::compact (present, unused by the ref) -> shn_compact_u32
 *      (src/Utils/chag/pp/compact.cuh:52-90)
 */
#ifndef SHINOBI_B200_H
#define SHINOBI_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SHN_ABI_VERSION 1u
#define SHN_MISS 0xFFFFFFFFu

typedef enum shn_status {
  SHN_OK = 0,
  SHN_ERR_INVALID = 1,      /* bad argument, size beyond a stated maximum, non-finite input */
  SHN_ERR_CUDA = 2,         /* a CUDA runtime call failed */
  SHN_ERR_OOM = 3,          /* device allocation failed */
  SHN_ERR_TIMEOUT = 4,      /* a bounded device-side wait gave up (result is not valid) */
  SHN_ERR_BUDGET = 5,       /* the context's HBM budget would be exceeded */
  SHN_ERR_NOT_BUILT = 6,    /* grid used before a successful build */
  SHN_ERR_BUSY = 7,         /* server queue full / request not finished */
  SHN_ERR_CANCELLED = 8     /* server request cancelled */
} shn_status;

typedef struct shn_ctx shn_ctx;
typedef struct shn_scene shn_scene;
typedef struct shn_grid shn_grid;

/* ---- context -------------------------------------------------------------
 * One per device.  hbm_budget_bytes = 0 means no limit.  Device memory of
 * scenes, grids and build workspaces comes from a stream-ordered pool that
 * the context owns. */
shn_status shn_ctx_create(int device, uint64_t hbm_budget_bytes, shn_ctx** out);
/* Releases the caller's handle.  Scenes, grids, batches and servers created
 * on the context keep it alive: its memory pool is destroyed when the last
 * of them is destroyed, in any order. */
void shn_ctx_destroy(shn_ctx* ctx);
const char* shn_status_string(shn_status s);
const char* shn_ctx_last_error(const shn_ctx* ctx);
shn_status shn_ctx_memory(const shn_ctx* ctx, uint64_t* used_bytes, uint64_t* budget_bytes);
uint32_t shn_abi_version(void);

/* ---- scene (FaceSoup) ----------------------------------------------------- */
#define SHN_MEM_HOST 0u
#define SHN_MEM_DEVICE 1u
/* vtx_xyz: nv float xyz triples; idx: nt uint32 index triples.  mem says
 * whether both pointers are host or device memory.  Host input is validated
 * (finite vertices, indices < nv); device input is copied as is.  Blocks
 * until the bounds are known on the host (one small read-back for device
 * input). */
shn_status shn_scene_create(shn_ctx* ctx, const float* vtx_xyz, uint32_t nv, const uint32_t* idx,
                            uint32_t nt, uint32_t mem, void* stream, shn_scene** out);
/* Replace vertex positions (same counts); recomputes bounds.  Host vertices
 * are staged on the device and checked there for inf/NaN before they replace
 * the scene's (SHN_ERR_INVALID leaves the scene unchanged); synchronises the
 * stream once for that check and once for the bounds. */
shn_status shn_scene_update_vertices(shn_scene* s, const float* vtx_xyz, uint32_t nv, uint32_t mem,
                                     void* stream);
/* Keyframe interpolation on the device (FaceSoup::uploadVertices as used by
 * DynamicRTEngine, src/Control/Structure/FaceSoup.h:249-339,
 * src/Engine/DynamicRTEngine.h:73-158): vertex coordinate i becomes
 * kf1[i] * (1 - coeff) + kf2[i] * coeff (FP32, in that order) for the first
 * n1 vertices and kf2[i] for the rest, as the reference does when the first
 * keyframe is shorter.  d_kf1 (3*n1 floats) and d_kf2 (3*nv floats, nv the
 * scene's count) are device arrays; recomputes bounds (one stream
 * synchronisation).  Inputs are not checked for inf/NaN beyond the bounds. */
shn_status shn_scene_interpolate_vertices(shn_scene* s, const float* d_kf1, uint32_t n1, const float* d_kf2,
                                          float coeff, void* stream);
shn_status shn_scene_bounds(const shn_scene* s, float out_min_max[6]);
uint32_t shn_scene_num_triangles(const shn_scene* s);
void shn_scene_destroy(shn_scene* s);

/* ---- scene files -------------------------------------------------------------
 * Wavefront OBJ + MTL, camera and area-light configuration files, read with
 * the reference's parsing rules so that a scene loads into the same
 * vertices, faces, materials, camera and light:
 *  - FWObject::read / readMtlLib      -> shn_obj_read
 *      (src/Loaders/FWObjectReader.cpp:96-502): v / vn / vt, f with v, v/t,
 *      v//n or v/t/n references (1-based), polygons fanned around their
 *      first vertex, usemtl (material 0 is "Default", diffuse 0.9774; others
 *      in order of first use), mtllib files (read after the OBJ, relative to
 *      its directory; Kd / Ks / Ka / Ns of used materials), then diffuse /= pi
 *      and specular *= (Ns + 2) / (2 pi) (Material::setupPhongCoefficients,
 *      src/Loaders/FWObject.hpp:87-91).  Lines the reference rejects are
 *      skipped and counted.  A face index that is not positive or names a
 *      missing vertex, or an .mtl file that cannot be opened, makes the call
 *      fail with SHN_ERR_INVALID (the reference reads out of bounds / throws).
 *  - CameraManager::read               -> shn_camera_read
 *      (src/Loaders/CameraManager.cpp:94-158, rotation: :29-63): position,
 *      orientation, up, rotation (degrees, applied to orientation and up),
 *      resX, resY, FOV; lines holding '#' are skipped; entries missing from
 *      the file keep the values *cam holds on entry.
 *  - LightSourceLoader::loadFromFile   -> shn_light_read
 *      (src/Loaders/LightSourceLoader.cpp:26-89): position, normal,
 *      intensity, edge1, edge2; a missing normal is normalize(edge1 x edge2). */
typedef struct shn_obj shn_obj;
typedef struct shn_obj_info {
  uint32_t num_vertices, num_faces, num_materials, num_normals, num_texcoords;
  uint64_t skipped_lines;
} shn_obj_info;
shn_status shn_obj_read(const char* path, shn_obj** out);
shn_status shn_obj_get_info(const shn_obj* o, shn_obj_info* info);
/* Copies (any pointer may be NULL): vertices 3*num_vertices floats, faces
 * 3*num_faces vertex indices (0-based), face_material num_faces material ids,
 * diffuse and specular 4*num_materials floats (rgb after the Phong setup;
 * diffuse .w = 0, specular .w = Ns). */
shn_status shn_obj_copy(const shn_obj* o, float* vertices, uint32_t* faces, uint32_t* face_material,
                        float* diffuse, float* specular);
/* Name of material m (valid until shn_obj_destroy), NULL if out of range. */
const char* shn_obj_material_name(const shn_obj* o, uint32_t m);
void shn_obj_destroy(shn_obj* o);

/* ---- grid build ------------------------------------------------------------ */
#define SHN_GRID_UNIFORM 0u
#define SHN_GRID_TWO_LEVEL 1u

typedef struct shn_grid_params {
  uint32_t kind;            /* SHN_GRID_UNIFORM or SHN_GRID_TWO_LEVEL */
  float lambda;             /* cells per triangle of the (top) grid: res = diag*cbrt(lambda*N/V) */
  int32_t top_divisor;      /* integer divisor applied to that resolution (reference two-level: 6) */
  int32_t min_res;          /* lower clamp per axis after the divisor (reference two-level: 2) */
  float lambda_leaf;        /* two-level: leaf cells per reference in a top cell (reference: 1.2) */
  uint32_t leaf_threshold;  /* two-level: top cells with <= this many references stay one leaf (16) */
  int32_t res[3];           /* if all > 0: use this resolution instead of the lambda rule */
  uint32_t insertion;       /* SHN_INSERT_PLANE (default) or SHN_INSERT_SAT, for the uniform grid / top level */
} shn_grid_params;

/* Insertion rules.  PLANE: a candidate cell of a triangle whose box spans two
 * or more cells on every axis is kept if the triangle's plane passes within
 * half a cell of its centre (the reference's sort-based builders,
 * src/Control/Algorithm/FastBuildKernels.h:137-212).  SAT: the plane test and
 * the nine edge-cross-axis tests of the triangle/box separating-axis test
 * (the precise insertion of the reference's other builder,
 * src/Control/Algorithm/BuildKernels.h:117-201): tighter grids, a slower
 * build.  The leaf level of two-level grids always uses PLANE, as in the
 * reference. */
#define SHN_INSERT_PLANE 0u
#define SHN_INSERT_SAT 1u

/* Reference defaults: uniform lambda=5; two-level lambda=5, divisor 6, min 2,
 * lambda_leaf 1.2, threshold 16 (src/Control/Algorithm/GridBuilder.h:48,
 * src/Control/Algorithm/FastTwoLevelGridBuilder.h:87-102,
 * src/Control/Algorithm/TwoLevelBuildKernels.h:49,73). */
void shn_grid_params_default(uint32_t kind, shn_grid_params* p);

/* ---- SAH resolution search ------------------------------------------------- */
typedef struct shn_sah_result {
  int32_t res[3];       /* resolution of least cost (the first one in z, y, x order) */
  int32_t res_min[3];   /* the searched window, inclusive */
  int32_t res_max[3];
  float cost;           /* its cost */
  uint64_t refs;        /* its bounding-box cell references */
  uint64_t num_tested;  /* resolutions in the window */
} shn_sah_result;

/* SAHGridBuilder::computeResolution (src/Control/Algorithm/SAHGridBuilder.h:117-202):
 * every resolution from window_lo to window_hi times the lambda estimate of
 * GridBuilder::computeResolution (reference: lambda 5, window 0.75 .. 1.25),
 * each bound clamped to [1, 2048], costed as
 *   0.85 * refs * cellArea / sceneArea + 0.15 * (resX + resY + resZ)
 * with refs the triangles' bounding-box cell count at that resolution
 * (countRefs, src/Control/Algorithm/FastBuildKernels.h:31-86), counted
 * exactly in 64 bits.  counts (optional, host, x fastest then y then z)
 * receives every tested resolution's refs.  Synchronous on `stream`.
 * SHN_ERR_INVALID when the window holds more than 2^24 resolutions or
 * resolutions x triangles exceeds 2e13. */
shn_status shn_grid_sah_resolution(const shn_scene* scene, float lambda, float window_lo, float window_hi,
                                   uint64_t* counts, uint64_t counts_capacity, shn_sah_result* out,
                                   void* stream);

/* The same refs and cost for k <= 32 explicit resolutions res[3*i .. 3*i+2]
 * (each axis in [1, 2048]); refs or cost may be NULL.  Synchronous. */
shn_status shn_grid_sah_cost(const shn_scene* scene, const int32_t* res, uint32_t k, uint64_t* refs,
                             float* cost, void* stream);

typedef struct shn_grid_info {
  uint32_t kind;
  int32_t res[3];
  float bounds[6];
  float cell_size[3];
  uint64_t num_cells;      /* uniform cells, or top cells */
  uint64_t num_top_refs;   /* two-level: (top cell, tri) pairs */
  uint64_t num_leaves;     /* two-level: leaf cells */
  uint64_t num_refs;       /* entries of indices[] (the reference array) */
  uint64_t device_bytes;   /* grid-owned device memory */
  float build_ms;          /* device time of the last build (CUDA events) */
} shn_grid_info;

shn_status shn_grid_create(shn_ctx* ctx, shn_grid** out);
/* Builds (or rebuilds) the grid over the scene on stream.  Synchronises the
 * stream once (uniform: the pair count) or twice (two-level: the pair count,
 * then the leaf and leaf-reference counts) to size buffers from device-side
 * counts, as the reference does, and returns SHN_ERR_TIMEOUT if a bounded
 * device wait gave up before those points.  The last stage (sort, ranges and
 * what follows) runs asynchronously on stream: traces, exports and info calls
 * of the grid, on any stream, are ordered after it, and a wait that gives up
 * there is reported by shn_grid_sync_status.  Traces of the grid read the
 * scene's triangles (hit records, normals), so the scene must outlive them. */
shn_status shn_grid_build(shn_grid* g, const shn_scene* s, const shn_grid_params* p, void* stream);
shn_status shn_grid_get_info(const shn_grid* g, shn_grid_info* out);
/* Copies the grid to host buffers (any may be NULL): cells = 2*num_cells
 * uint32 (uniform: [begin,end) ranges; two-level: cell words in the
 * TwoLevelGridCell layout), leaves = 2*num_leaves, indices = num_refs,
 * top_pairs = num_top_refs sorted (cell<<32 | tri) keys (two-level) or
 * num_refs (uniform), all in (cell, triangle id) order.  A two-level grid
 * keeps the references of each leaf in spatial order on the device, and its
 * empty leaves hold [D, D) with D the distance to the nearest non-empty leaf;
 * the export puts the references back in (cell, triangle id) order and
 * returns empty leaves as [0, 0).  Uniform grids of 2^22 cells or more keep
 * the same distances in their empty cells, exported as [0, 0).
 * Synchronises. */
shn_status shn_grid_export(const shn_grid* g, uint32_t* cells, uint32_t* leaves, uint32_t* indices,
                           uint64_t* top_pairs);
/* Frees the grid's device memory (stream-ordered, pool); every launch that
 * reads the grid must have completed. */
void shn_grid_destroy(shn_grid* g);
/* Synchronises stream, then reports and clears the grid's device error word:
 * SHN_ERR_TIMEOUT if a bounded wait gave up in any trace, AO,
 * direct-illumination or path-tracer call on the grid since the last check
 * (their results are then not valid), else SHN_OK.  The word also clears at
 * the start of each build, which reports its own waits.  No counterpart in
 * the reference (its cutil macros aborted the process). */
shn_status shn_grid_sync_status(const shn_grid* g, void* stream);

/* ---- traversal -------------------------------------------------------------- */
typedef struct shn_rays {
  const float *ox, *oy, *oz;  /* device SoA origins */
  const float *dx, *dy, *dz;  /* device SoA directions (need not be unit length) */
  const float* tmax;          /* device; NULL = FLT_MAX */
} shn_rays;

typedef struct shn_hits {
  uint32_t* tri;  /* device; SHN_MISS when nothing was hit */
  float* t;       /* device; tmax when nothing was hit */
  float* u;       /* device, may be NULL: barycentric weight of vertex 1 */
  float* v;       /* device, may be NULL: barycentric weight of vertex 2 */
} shn_hits;

/* Closest hit with t in (1e-5, tmax). */
shn_status shn_trace_closest(const shn_grid* g, const shn_rays* rays, uint32_t n, shn_hits* hits,
                             void* stream);
/* Any hit with t in (1e-5, tmax): occluded[i] = 1 if blocked, else 0. */
shn_status shn_trace_any(const shn_grid* g, const shn_rays* rays, uint32_t n, uint8_t* d_occluded,
                         void* stream);

typedef struct shn_camera {
  float eye[3], forward[3], up[3];
  float fov_deg;            /* vertical opening angle */
  uint32_t res_x, res_y;
} shn_camera;

/* Pinhole primary rays (Camera + RegularPixelSampler<1,1>, generated in the
 * kernel) traced for closest hit; hits are pixel-major (res_x*res_y). */
shn_status shn_trace_primary(const shn_grid* g, const shn_camera* cam, uint32_t image_id,
                             shn_hits* hits, void* stream);

/* Ambient occlusion from primary hits: spp cosine-distributed any-hit rays
 * of length `length` per hit pixel, origin offset `offset` along the facing
 * normal, Philox4x32-10 stream (pixel, sample) keyed by seed.  d_ao[p] =
 * fraction of unoccluded samples (1 for pixels without a primary hit).
 * If d_num_rays != NULL it receives the number of AO rays traced (device). */
shn_status shn_trace_ao(const shn_grid* g, const shn_camera* cam, const shn_hits* primary,
                        uint32_t spp, float length, float offset, uint32_t seed, float* d_ao,
                        uint32_t* d_num_rays, void* stream);

/* Direct illumination from one parallelogram light (DirectIlluminationIntegrator::shade
 * and computeDirectIllumination, src/Integrator/DirectIlluminationIntegrator.h:46-168,
 * src/Integrator/DirectIlluminationIntegrator.h:254-338; AreaLightSource,
 * src/Primitive/LightSource.hpp:35-51; MaterialContainer, src/Primitive/Material.h:36-46).
 * Per primary hit pixel p and sample s < samples:
 *   origin  = eye + (t - 1e-5) * d          (SimpleRayBuffer::store, src/Engine/RayBuffers.h:52-55)
 *   L       = position + r1 * edge1 + r2 * edge2 - origin, (r1, r2) from the
 *             Philox4x32-10 counter (p, s, image_id, 0x444C) keyed by seed
 *   any-hit shadow segment with t in (1e-5, 0.9999)   (OcclusionRayBuffer::store, src/Engine/RayBuffers.h:156-168)
 *   value_s = 0 if blocked, else intensity * |edge1 x edge2| * diffuse(material(tri))
 *             * max(0, -normal_light . L^) * max(0, n . L^) / (L . L), n the
 *             unflipped geometric normal of the hit triangle;
 * pixels without a hit take `background` for every sample.
 * frame[p] = sum_s value_s / samples (RGB, 3 floats per pixel), and
 * final[p] = final[p] * (1 - w) + frame[p] * w with w = 1 / (image_id + 1).
 * tri_material (per scene triangle) may be NULL: material 0 everywhere; diffuse
 * (4 floats per material, .w unused) may be NULL: default_diffuse everywhere.
 * Material ids >= num_materials read material 0.  d_final may be NULL.
 * If d_num_rays != NULL it receives the number of shadow rays traced (device). */
typedef struct shn_area_light {
  float position[3];   /* corner */
  float edge1[3], edge2[3];
  float normal[3];     /* the light emits towards -normal */
  float intensity[3];
} shn_area_light;

typedef struct shn_di_params {
  shn_area_light light;
  uint32_t samples;              /* shadow rays per pixel (NUMOCCLUSIONSAMPLES = 4) */
  uint32_t seed;
  uint32_t image_id;             /* progressive accumulation index */
  const uint32_t* tri_material;  /* device, per scene triangle, or NULL */
  const float* diffuse;          /* device, 4 floats per material, or NULL */
  uint32_t num_materials;
  float default_diffuse[3];
  float background[3];           /* BACKGROUND_R/G/B, src/CUDAConfig.h:57-59 */
} shn_di_params;

void shn_di_params_default(shn_di_params* p);
/* Scene files of the camera and the area light (see "scene files" above). */
shn_status shn_camera_read(const char* path, shn_camera* cam);
shn_status shn_light_read(const char* path, shn_area_light* light);
shn_status shn_shade_direct(const shn_grid* g, const shn_camera* cam, const shn_hits* primary,
                            const shn_di_params* p, float* d_frame, float* d_final,
                            uint32_t* d_num_rays, void* stream);

/* Work counters: when d_counters (2 x uint64, device) is non-NULL, later
 * trace calls on this grid run counting variants of their kernels and add
 * {cell visits, triangle tests} to it (for roofline accounting); NULL turns
 * counting off.  Not part of the reference interface. */
shn_status shn_grid_set_stats(shn_grid* g, uint64_t* d_counters);

/* ---- dynamic scenes (DynamicRTEngine, src/Engine/DynamicRTEngine.h:49-158) -------
 * Two frame slots, each a scene with its own grid and stream.  A frame
 * renders the slot built during the previous frame (primary rays + direct
 * illumination, shn_trace_primary + shn_shade_direct) on that slot's stream
 * while, on the other slot's stream, the vertices are interpolated between
 * two keyframes (shn_scene_interpolate_vertices, FaceSoup::uploadVertices)
 * and that slot's grid is rebuilt (shn_grid_build), so the rebuild of frame
 * N+1 overlaps the render of frame N on the GPU.  As in the reference, the
 * frame a call renders shows the previous call's keyframe geometry (the
 * first call renders the geometry given to shn_dynamic_create).  Unlike the
 * reference (one global grid-parameter constant and global textures for
 * both slots), the two slots share no state. */
typedef struct shn_dynamic shn_dynamic;
/* vtx/idx as for shn_scene_create (host or device, mem); builds slot 0.
 * Synchronises. */
shn_status shn_dynamic_create(shn_ctx* ctx, const float* vtx_xyz, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              uint32_t mem, const shn_grid_params* p, shn_dynamic** out);
/* DynamicRTEngine::renderFrame: renders into hits / d_frame / d_final (as for
 * shn_shade_direct, with di->image_id) and prepares the next frame from the
 * device keyframes d_kf1 (3*n1 floats) and d_kf2 (3*nv floats) with coeff
 * (vertex = kf1 * (1 - coeff) + kf2 * coeff).  Returns when both the render
 * and the rebuild are done; render_ms, build_ms (device time of each stream)
 * and frame_ms (first to last, the two overlapping) may be NULL. */
shn_status shn_dynamic_render_frame(shn_dynamic* e, const float* d_kf1, uint32_t n1, const float* d_kf2,
                                    float coeff, const shn_camera* cam, const shn_di_params* di,
                                    shn_hits* hits, float* d_frame, float* d_final, float* render_ms,
                                    float* build_ms, float* frame_ms);
/* The grid and scene the next call renders (next = 1) or the last call
 * rendered (next = 0); owned by the engine. */
shn_status shn_dynamic_get_grid(const shn_dynamic* e, uint32_t next, shn_grid** grid, shn_scene** scene);
void shn_dynamic_destroy(shn_dynamic* e);

/* ---- batched multi-scene build and trace ----------------------------------------
 * Many independent scenes, each with its own uniform grid, built by one
 * fused pipeline (one count/scan, emit, sort and range pass over all
 * triangles) and traced by one persistent launch over all scenes' rays.
 * Not a reference interface: the reference builds one scene per engine. */
typedef struct shn_batch shn_batch;
/* Scenes are concatenated: scene s has vertices [vtx_offsets[s], vtx_offsets[s+1])
 * and triangles [tri_offsets[s], tri_offsets[s+1]) whose indices are local to
 * the scene's vertices.  Offsets are host arrays of num_scenes+1 entries
 * starting at 0; vertices/indices are host or device memory (mem).  Synchronises. */
shn_status shn_batch_create(shn_ctx* ctx, uint32_t num_scenes, const float* vtx_xyz,
                            const uint32_t* vtx_offsets, const uint32_t* idx,
                            const uint32_t* tri_offsets, uint32_t mem, void* stream, shn_batch** out);
/* Per-scene cell density (num_scenes floats, default 5). */
shn_status shn_batch_set_lambdas(shn_batch* b, const float* lambdas);
/* Measured autotuner: for every scene and candidate lambda, builds the scene's
 * grid and traces min(sample_rays, expected_rays[s]) uniformly random rays
 * (origins in [-1,2]^3, unit directions, Philox seed), and keeps the lambda
 * with the smallest build + scaled trace time.  chosen (optional) receives
 * the lambdas; they are also applied to the batch.  Synchronises. */
shn_status shn_batch_autotune(shn_batch* b, const float* candidates, uint32_t num_candidates,
                              const uint32_t* expected_rays, uint32_t sample_rays, uint32_t seed,
                              float* chosen, void* stream);
/* The autotuner with two more terms.
 *  sah_keep > 0: per scene, every candidate's resolution is costed with the
 *    SAH cost of shn_grid_sah_cost (SAHGridBuilder.h:164-175) and only the
 *    sah_keep cheapest are built and timed; 0 times them all.
 *  blocks_per_sm[0 .. num_block_shapes): resident blocks per SM of the
 *    batch's persistent closest-hit trace kernel (block of 128 threads) to
 *    time on the chosen grids with max(sample_rays, 2^21) random rays
 *    spread over the scenes like expected_rays (median of three launches
 *    each); the fastest is kept for later traces and captures.
 *    0 entries: the occupancy limit.
 *  sort_tile_keys[0 .. num_sort_tiles): keys per tile of the batch's
 *    onesweep passes (4096 or 6144), each timed as the batch's whole build
 *    (median of three) on the chosen grids; the fastest is kept.
 * sah_cost (optional, num_scenes) receives the chosen candidate's SAH cost;
 * report (optional) the work done and the shape timings.  Synchronises. */
typedef struct shn_autotune_config {
  uint32_t sah_keep;
  uint32_t num_block_shapes;  /* <= 8 */
  uint32_t blocks_per_sm[8];
  uint32_t num_sort_tiles;    /* <= 4: onesweep tile shapes to time on the batch's build */
  uint32_t sort_tile_keys[4]; /* keys per tile: 4096 or 6144 (0: 6144) */
} shn_autotune_config;
typedef struct shn_autotune_report {
  uint32_t timed_candidates;  /* (scene, lambda) builds timed */
  uint32_t blocks_per_sm;     /* chosen (0: occupancy limit) */
  float shape_ms[8];          /* median sample trace time per blocks_per_sm entry */
  uint32_t sort_tile_keys;    /* chosen keys per onesweep tile */
  float sort_tile_ms[4];      /* median whole-build time per sort_tile_keys entry */
} shn_autotune_report;
shn_status shn_batch_autotune_ex(shn_batch* b, const float* candidates, uint32_t num_candidates,
                                 const uint32_t* expected_rays, uint32_t sample_rays, uint32_t seed,
                                 const shn_autotune_config* cfg, float* chosen, float* sah_cost,
                                 shn_autotune_report* report, void* stream);
/* Builds every scene's grid (plans buffers with one read-back on the first
 * call or after a lambda change).  Synchronises. */
shn_status shn_batch_build(shn_batch* b, void* stream);
/* Traces rays of all scenes in one launch: device SoA rays concatenated in
 * scene order, ray_offsets = host array of num_scenes+1.  Closest hits into
 * hits (triangle ids local to their scene) or, if d_occluded != NULL, any-hit
 * flags. */
shn_status shn_batch_trace(shn_batch* b, const shn_rays* rays, const uint32_t* ray_offsets,
                           shn_hits* hits, uint8_t* d_occluded, void* stream);
/* Captures build + closest-hit trace into a CUDA graph (ray and hit buffers
 * are baked in and must stay valid); shn_batch_replay launches it. */
shn_status shn_batch_capture(shn_batch* b, const shn_rays* rays, const uint32_t* ray_offsets,
                             shn_hits* hits, void* stream);
shn_status shn_batch_replay(shn_batch* b, void* stream);
shn_status shn_batch_info(const shn_batch* b, uint64_t* num_pairs, uint64_t* total_cells, float* build_ms);
/* One scene's grid rebased to local indices: cells 2*res product uint32,
 * indices num_refs uint32 (triangle ids local to the scene).  Synchronises. */
shn_status shn_batch_export_scene(const shn_batch* b, uint32_t scene, int32_t res[3], float bounds[6],
                                  uint32_t* cells, uint32_t* indices, uint64_t* num_refs);
void shn_batch_destroy(shn_batch* b);
/* Synchronises stream, then reports and clears the batch's device error word
 * (set by the build, trace or graph replay of the batch since the last check;
 * each build clears it first): SHN_ERR_TIMEOUT for a bounded wait that gave
 * up, SHN_ERR_INVALID when a replay found more pairs than planned. */
shn_status shn_batch_sync_status(shn_batch* b, void* stream);

/* ---- ray-query server ------------------------------------------------------------
 * Resident uniform grids in scene slots, requests admitted by the context's
 * HBM budget, continuous batching: consecutive ray requests (any scenes,
 * closest or any hit) are packed into one launch while the previous launch
 * runs; scene updates rebuild a slot's grid after the requests queued before
 * them.  coalesce = 0 gives the plain path: one launch per request, no overlap.
 * A replaced slot keeps its previous scene and grid (once no launch reads
 * them) and builds its next replacement into their device buffers, so
 * replacements of similar size allocate no device memory; that memory counts
 * against the HBM budget, and an update the budget would refuse releases it
 * and tries once more. */
#define SHN_REQ_CLOSEST 0u
#define SHN_REQ_ANY 1u
#define SHN_REQ_UPDATE 2u

typedef struct shn_server shn_server;
typedef struct shn_server_config {
  uint32_t num_slots;                /* scene slots (default 64) */
  uint32_t max_batch_rays;           /* rays per launch and per request (default 4M) */
  uint32_t max_requests_per_launch;  /* default 4096 */
  uint32_t max_queue;                /* 0 = unbounded; else submit returns SHN_ERR_BUSY when full */
  uint32_t coalesce;                 /* 1 = continuous batching (default), 0 = one launch per request */
} shn_server_config;

typedef struct shn_request {
  uint32_t kind;       /* SHN_REQ_CLOSEST / SHN_REQ_ANY / SHN_REQ_UPDATE */
  uint32_t scene;      /* slot */
  uint32_t num_rays;
  const float* rays;   /* host, 8 floats per ray: ox oy oz dx dy dz tmax (unused); pinned for overlap */
  uint32_t* out_tri;   /* host, may be NULL: hit triangle (closest) / any hit (SHN_MISS = not occluded) */
  float* out_t;        /* host, may be NULL */
  /* SHN_REQ_UPDATE: new scene for the slot (host arrays, read during processing) */
  const float* vtx;
  uint32_t nv;
  const uint32_t* idx;
  uint32_t nt;
  float lambda;
} shn_request;

typedef struct shn_server_stats {
  uint64_t requests, updates, rays, launches, max_requests_per_launch;
  double p50_us, p99_us, max_us, mean_us;  /* submit -> completion latency */
  double wall_s;                           /* first submit -> last completion */
  double mrays_per_s;
} shn_server_stats;

void shn_server_config_default(shn_server_config* c);
shn_status shn_server_create(shn_ctx* ctx, const shn_server_config* cfg, shn_server** out);
/* Synchronous initial load of a slot (only while no request is pending). */
shn_status shn_server_load_scene(shn_server* s, uint32_t slot, const float* vtx_xyz, uint32_t nv,
                                 const uint32_t* idx, uint32_t nt, float lambda);
shn_status shn_server_submit(shn_server* s, const shn_request* r, uint64_t* ticket);
/* Waits up to timeout_ms; SHN_OK with *result set when done (the ticket is
 * released), SHN_ERR_BUSY if still pending. */
shn_status shn_server_wait(shn_server* s, uint64_t ticket, uint32_t timeout_ms, shn_status* result);
shn_status shn_server_poll(shn_server* s, uint64_t ticket, shn_status* result);
shn_status shn_server_drain(shn_server* s, uint32_t timeout_ms);
shn_status shn_server_get_stats(shn_server* s, shn_server_stats* out, int reset);
/* Per-request records since the last stats reset, in completion order:
 * submit time (steady clock, seconds), latency, kind, scene, rays, status.
 * Copies min(max_records, *count) of them; *count = how many exist. */
typedef struct shn_request_record {
  double submit_s;
  double latency_us;
  uint32_t kind, scene, num_rays;
  int32_t status;
} shn_request_record;
shn_status shn_server_get_records(shn_server* s, uint32_t max_records, shn_request_record* out,
                                  uint32_t* count);
/* Load generator: submits reqs[i] at arrival_s[i] seconds after the call
 * (from the calling thread), then waits for all; results (optional) per request. */
shn_status shn_server_run_schedule(shn_server* s, uint32_t n, const shn_request* reqs,
                                   const double* arrival_s, shn_status* results);
void shn_server_destroy(shn_server* s);

/* ---- path tracer --------------------------------------------------------------- */
typedef struct shn_pt_params {
  uint32_t spp;              /* samples per pixel */
  uint32_t max_depth;        /* bounces (path segments) per sample */
  uint32_t rr_depth;         /* Russian roulette from this depth on */
  float albedo;              /* diffuse albedo of every surface */
  float light_pos[3];        /* area light: corner, two edges, emitted radiance */
  float light_e1[3];
  float light_e2[3];
  float light_radiance[3];
  float background[3];
  float offset;              /* ray origin offset along the normal */
  uint32_t seed;
} shn_pt_params;

void shn_pt_params_default(shn_pt_params* p);
/* Wavefront path tracer: camera rays -> extend -> shade/next-event -> compact
 * after each bounce.  d_image: res_x*res_y*3 floats (mean radiance).  If
 * d_stats != NULL (max_depth+1 uint32, device) it receives the number of paths
 * traced at each bounce d < max_depth, summed over all wavefront chunks, and
 * in d_stats[max_depth] the number of next-event shadow rays traced. */
shn_status shn_pt_render(const shn_grid* g, const shn_scene* s, const shn_camera* cam,
                         const shn_pt_params* p, float* d_image, uint32_t* d_stats, void* stream);

/* ---- parallel primitives ------------------------------------------------------- */
/* d_out[0..n] = exclusive prefix sums of d_in[0..n-1], d_out[n] = total.
 * Single-pass decoupled look-back.  n < 2^31. */
shn_status shn_exclusive_scan_u32(shn_ctx* ctx, const uint32_t* d_in, uint32_t* d_out, uint32_t n,
                                  void* stream);
/* Same result as shn_exclusive_scan_u32, for callers that cannot allocate
 * device memory on this path (an engine that has pre-claimed all device
 * memory for its own allocator, or a loop whose memory budget is already
 * committed): the look-back scratch lives in a fixed file-scope device array
 * of about 64 KiB held by every GPU that loads the library, not in a pool.
 * n <= 2^24 (SHN_SCAN_NOALLOC_MAX_N), larger n returns SHN_ERR_INVALID.  All
 * calls on a device share that array: calls whose work overlaps on the GPU
 * race, so order them on one stream.  Each call clears the words it uses
 * (8 * (ceil(n / 2048) + 1) bytes, one cudaMemsetAsync on the stream).  A
 * look-back wait that gives up is reported by
 * shn_exclusive_scan_u32_noalloc_status.  The first call on each device looks
 * up the array's device address (cudaGetSymbolAddress, with that device
 * current) and caches it for the life of the process; make it before any
 * stream capture, and do not call after a cudaDeviceReset, which invalidates
 * the cached address.  No counterpart in the reference. */
#define SHN_SCAN_NOALLOC_MAX_N (1u << 24)
shn_status shn_exclusive_scan_u32_noalloc(const uint32_t* d_in, uint32_t* d_out, uint32_t n,
                                          void* stream);
/* Synchronises stream, then reports and clears the error word of the
 * allocation-free scan: SHN_ERR_TIMEOUT if a look-back wait gave up in any
 * shn_exclusive_scan_u32_noalloc call on the current device since the last
 * check (those calls' outputs are not valid), else SHN_OK.  Allocates
 * nothing (it reads the same fixed array).  No counterpart in the reference. */
shn_status shn_exclusive_scan_u32_noalloc_status(void* stream);
/* Synchronises stream, then reports and clears the error word of the
 * context-level primitives (shn_exclusive_scan_u32, shn_compact_u32,
 * shn_sort_keys_u64): SHN_ERR_TIMEOUT if a bounded wait gave up in any of
 * them since the last check.  No counterpart in the reference. */
shn_status shn_ctx_sync_status(shn_ctx* ctx, void* stream);
/* Failure-detection self test of the look-back scans that run inside other
 * calls.  Arms the next look-back scan of the chosen kind to launch without
 * its first tile, which then never publishes, so every other tile's bounded
 * wait runs out (about a second) and records SHN_ERR_TIMEOUT for the status
 * call above; the output of that one call is not valid, and no access leaves
 * its buffers.  The arm is used by the first call with at least two tiles
 * (more than 2048 elements / pixels):
 *   SHN_FORCE_CTX_SCAN         shn_exclusive_scan_u32 or shn_compact_u32 on ctx;
 *   SHN_FORCE_GRID_COMPACTION  the hit compaction of shn_trace_ao or
 *                              shn_shade_direct on g;
 *   SHN_FORCE_NOALLOC_SCAN     shn_exclusive_scan_u32_noalloc (any device).
 * No counterpart in the reference. */
#define SHN_FORCE_CTX_SCAN 1u
#define SHN_FORCE_GRID_COMPACTION 2u
#define SHN_FORCE_NOALLOC_SCAN 3u
shn_status shn_debug_force_lookback_timeout(uint32_t target, shn_ctx* ctx, shn_grid* g);
/* Failure-detection self test: runs the look-back scan kernel with tile 0
 * never published, so tile 1's bounded wait must run out (about a second)
 * and report it.  Returns SHN_ERR_TIMEOUT when the wait ran out and the
 * context is still usable (the expected result).  No counterpart in the
 * reference. */
shn_status shn_selftest_lookback_timeout(shn_ctx* ctx, void* stream);
/* Stable compaction: d_out_idx[0..m) = indices i with d_flags[i] != 0, in
 * order; *d_count = m (device). */
shn_status shn_compact_u32(shn_ctx* ctx, const uint32_t* d_flags, uint32_t n, uint32_t* d_out_idx,
                           uint32_t* d_count, void* stream);
/* Stable LSD radix sort of 64-bit keys on bits [lo_bit, hi_bit), at most 32
 * bits (one onesweep pass per 8- or 9-bit digit, whichever width needs fewer
 * passes; bits outside the range do not affect the order).  d_tmp has n
 * entries; the sorted keys end in d_keys.  n < 2^30. */
shn_status shn_sort_keys_u64(shn_ctx* ctx, uint64_t* d_keys, uint64_t* d_tmp, uint32_t n,
                             uint32_t lo_bit, uint32_t hi_bit, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SHINOBI_B200_H */
