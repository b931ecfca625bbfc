// Batched multi-scene build and trace.
//
// Many independent scenes (uniform grids) are built by ONE pipeline over the
// concatenated triangles -- count/scan, emit, onesweep sort, ranges -- with a
// global cell-id space (scene s owns cells [cell_offset_s, + C_s)), and all
// scenes' rays are traced by ONE persistent launch in which every lane looks
// its scene up in a device table.  The whole build + trace can be captured
// into a CUDA graph and replayed without host synchronisation once the pair
// count has been planned.  Per-scene cell density lambda comes from
// shn_batch_set_lambdas or from the measured autotuner shn_batch_autotune.
//
// The per-scene result is bit-identical to shn_grid_build on that scene
// alone (same cell arithmetic, same stable order); ranges and indices are
// global and shn_batch_export_scene rebases them.
#include <chrono>

#include "internal.h"
#include "trace_coop.cuh"

struct shn_batch {
  shn_ctx* ctx = nullptr;
  uint32_t ns = 0;
  uint32_t T = 0;                      // total triangles
  std::vector<uint32_t> tri_off, vtx_off;
  std::vector<float> bounds;           // 6 per scene
  std::vector<float> lambdas;
  std::vector<shn::BatchScene> scenes;
  // device
  float* vtx = nullptr;
  uint32_t* idx = nullptr;
  float4* tri = nullptr;
  uint32_t* d_tri_off = nullptr;
  uint32_t* d_vtx_off = nullptr;
  shn::BatchScene* d_scenes = nullptr;
  uint32_t* offs = nullptr;
  void* scan_ws = nullptr;
  uint64_t* keys[2] = {nullptr, nullptr};
  void* sort_ws = nullptr;
  uint2* cells = nullptr;
  uint32_t* indices = nullptr;
  uint32_t* d_err = nullptr;           // [0] error bits, [1..] scratch words
  uint32_t* h_pinned = nullptr;
  uint64_t total_cells = 0;
  uint32_t P = 0;                      // planned pair count
  shn::SortPlan plan{0, 8, 0};             // digit plan of the sort over the global cell bits
  uint64_t* sorted = nullptr;
  bool planned = false, built = false;
  std::vector<std::pair<void*, size_t>> owned;   // (ptr, bytes) of plan-time buffers
  size_t bytes_vtx = 0, bytes_idx = 0, bytes_tri = 0;
  // graph
  cudaGraphExec_t exec = nullptr;
  cudaGraph_t graph = nullptr;
  uint32_t* d_ray_off = nullptr;
  uint32_t ray_off_cap = 0;
  uint32_t* d_counter = nullptr;
  float build_ms = 0.f;
  int blocks_closest = 0, blocks_any = 0;  // persistent grid sizes (computed before any capture)
  uint32_t bps_closest = 0;                // autotuned blocks per SM of the closest-hit trace (0: occupancy)
  uint32_t sort_tile = 0;                  // autotuned keys per onesweep tile (0: 6144)
};

namespace shn {
namespace {

constexpr int kBatchTraceBlock = 128;

struct BatchAcc {
  const BatchScene* sc;
  const uint2* cells;
  SHN_D const Geom& geom(uint32_t s) const { return sc[s].g; }
  SHN_D const uint2* cells_of(uint32_t s) const { return cells + sc[s].cell_offset; }
};

struct BatchAccW {
  static constexpr bool kIndirect = true;  // no reference-ordered copy: triangles through indices[]
  BatchAcc a;
  Refs r;
  SHN_D const Geom& geom(uint32_t s) const { return a.geom(s); }
  SHN_D const uint2* cells(uint32_t s) const { return a.cells_of(s); }
  SHN_D const uint2* leaves(uint32_t) const { return nullptr; }
  SHN_D Refs refs(uint32_t) const { return r; }
};

struct RaysV {
  const float *ox, *oy, *oz, *dx, *dy, *dz, *tmax;
};

template <bool ANY>
__global__ void __launch_bounds__(kBatchTraceBlock, 8) k_batch_trace(GridView G, BatchAcc A, RaysV R,
                                                                 const uint32_t* __restrict__ ray_off,
                                                                 uint32_t ns, uint32_t n, uint32_t* counter,
                                                                 uint32_t* otri, float* ot, float* ou,
                                                                 float* ov, uint8_t* occ) {
  // incoherent rays rarely share a cell range: no grouping (measured slower here)
  warp_trace_acc<0, ANY, false>(
      BatchAccW{A, refs_of(G)}, n, counter,
      [&](uint32_t i, V3& o, V3& d, float& tmax, uint32_t& scene, uint32_t&) {
        uint32_t lo = 0, hi = ns;
        while (hi - lo > 1) {
          const uint32_t mid = (lo + hi) >> 1;
          if (__ldg(ray_off + mid) <= i) lo = mid; else hi = mid;
        }
        scene = lo;
        o = mk(R.ox[i], R.oy[i], R.oz[i]);
        d = mk(R.dx[i], R.dy[i], R.dz[i]);
        tmax = R.tmax ? R.tmax[i] : FLT_MAX;
      },
      [&](uint32_t i, const Hit& h, uint32_t, uint32_t, uint32_t scene) {
        if (ANY) {
          occ[i] = h.tri != kMiss ? 1 : 0;
        } else {
          otri[i] = h.tri == kMiss ? kMiss : h.tri - A.sc[scene].tri_offset;
          ot[i] = h.t;
          if (ou) ou[i] = h.u;
          if (ov) ov[i] = h.v;
        }
      });
}

// Uniformly random rays for the autotuner: origins in [lo,hi]^3, unit directions.
__global__ void k_random_rays(uint32_t n, uint32_t seed, float lo, float hi, float* ox, float* oy,
                              float* oz, float* dx, float* dy, float* dz) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const uint4 w = philox4x32(make_uint4(i, 0u, 0u, 0x4155u), seed, 0x5455u);
  const uint4 w2 = philox4x32(make_uint4(i, 1u, 0u, 0x4155u), seed, 0x5455u);
  const float span = hi - lo;
  ox[i] = u01(w.x) * span + lo;
  oy[i] = u01(w.y) * span + lo;
  oz[i] = u01(w.z) * span + lo;
  const float z = u01(w.w) * 2.f - 1.f;
  float sn, cs;
  sincos_2pi(u01(w2.x), sn, cs);
  const float r = sqrtf(fmaxf(0.f, 1.f - z * z));
  dx[i] = r * cs;
  dy[i] = r * sn;
  dz[i] = z;
}

template <class K>
int batch_blocks(K kernel, int num_sms) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kBatchTraceBlock, 0);
  return std::max(1, per_sm) * num_sms;
}

cudaError_t own(shn_batch* b, void** p, size_t bytes, cudaStream_t st) {
  bytes = std::max<size_t>(bytes, 16);
  cudaError_t e = dev_alloc(b->ctx, p, bytes, st);
  if (e == cudaSuccess) b->owned.emplace_back(*p, bytes);
  return e;
}

void release_plan(shn_batch* b, cudaStream_t st) {
  for (auto& it : b->owned) dev_free(b->ctx, it.first, it.second, st);
  b->owned.clear();
  b->offs = nullptr;
  b->scan_ws = b->sort_ws = nullptr;
  b->keys[0] = b->keys[1] = nullptr;
  b->cells = nullptr;
  b->indices = nullptr;
  b->d_scenes = nullptr;
  b->d_ray_off = nullptr;
  b->ray_off_cap = 0;
  b->d_counter = nullptr;
  b->planned = b->built = false;
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
}

shn_status alloc_err(shn_batch* b, cudaError_t e, const char* what) {
  if (e == cudaErrorNotPermitted) return set_error(b->ctx, SHN_ERR_BUDGET, std::string(what) + ": HBM budget exceeded");
  return set_error(b->ctx, SHN_ERR_OOM, std::string(what) + ": out of device memory");
}

// Per-scene geometry from lambdas; plans the pair count (one sync) and the buffers.
shn_status plan(shn_batch* b, cudaStream_t st) {
  release_plan(b, st);
  b->scenes.assign(b->ns, BatchScene{});
  uint64_t co = 0;
  for (uint32_t s = 0; s < b->ns; ++s) {
    int res[3];
    const uint32_t nt = b->tri_off[s + 1] - b->tri_off[s];
    compute_resolution(nt, &b->bounds[6 * s], b->lambdas[s], 1, 1, res);
    if (nt == 0) res[0] = res[1] = res[2] = 1;
    BatchScene& sc = b->scenes[s];
    sc.g = make_geom(&b->bounds[6 * s], res);
    sc.tri_offset = b->tri_off[s];
    sc.nt = nt;
    sc.cell_offset = co;
    sc.ncells = (uint32_t)((uint64_t)res[0] * res[1] * res[2]);
    co += sc.ncells;
  }
  if (co >= (1ull << 32)) return set_error(b->ctx, SHN_ERR_INVALID, "batch has more than 2^32 cells");
  b->total_cells = co;
  b->blocks_closest = b->bps_closest ? (int)b->bps_closest * b->ctx->num_sms
                                      : batch_blocks(k_batch_trace<false>, b->ctx->num_sms);
  b->blocks_any = batch_blocks(k_batch_trace<true>, b->ctx->num_sms);
  cudaError_t e = own(b, (void**)&b->d_scenes, sizeof(BatchScene) * b->ns, st);
  if (e == cudaSuccess) e = own(b, (void**)&b->offs, ((size_t)b->T + 1) * 4, st);
  if (e == cudaSuccess) e = own(b, &b->scan_ws, batch_scan_bytes(b->T), st);
  if (e == cudaSuccess) e = own(b, (void**)&b->d_counter, 64, st);
  if (e != cudaSuccess) return alloc_err(b, e, "batch plan");
  cudaMemcpyAsync(b->d_scenes, b->scenes.data(), sizeof(BatchScene) * b->ns, cudaMemcpyHostToDevice, st);
  cudaMemsetAsync(b->d_err, 0, 64, st);
  launch_batch_count(b->tri, b->T, b->d_tri_off, b->d_scenes, b->ns, b->scan_ws, b->d_err, b->offs, st);
  cudaMemcpyAsync(b->h_pinned, b->offs + b->T, 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(b->h_pinned + 1, b->d_err, 4, cudaMemcpyDeviceToHost, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(b->ctx, e, "batch plan");
  if (b->h_pinned[1]) return set_error(b->ctx, SHN_ERR_TIMEOUT, "bounded device wait gave up (batch plan)");
  b->P = b->h_pinned[0];
  if (b->P >= (1u << 30)) return set_error(b->ctx, SHN_ERR_INVALID, "more than 2^30 cell references in the batch");
  b->plan = sort_plan(key_bits_for(co ? co - 1 : 0));
  e = own(b, (void**)&b->keys[0], (size_t)b->P * 8, st);
  if (e == cudaSuccess) e = own(b, (void**)&b->keys[1], (size_t)b->P * 8, st);
  if (e == cudaSuccess) e = own(b, &b->sort_ws, sort_workspace_bytes(b->P), st);
  if (e == cudaSuccess) e = own(b, (void**)&b->cells, co * 8, st);
  if (e == cudaSuccess) e = own(b, (void**)&b->indices, (size_t)b->P * 4, st);
  if (e != cudaSuccess) return alloc_err(b, e, "batch buffers");
  b->planned = true;
  return SHN_OK;
}

// The build as a sequence of launches with fixed sizes (no host sync): capturable.
void enqueue_build(shn_batch* b, cudaStream_t st) {
  cudaMemsetAsync(b->d_err, 0, 4, st);
  launch_batch_count(b->tri, b->T, b->d_tri_off, b->d_scenes, b->ns, b->scan_ws, b->d_err, b->offs, st);
  sort_prepare(b->sort_ws, st);
  launch_batch_emit(b->tri, b->T, b->d_tri_off, b->d_scenes, b->ns, b->offs, b->keys[0], b->P, b->d_err,
                    sort_hist_counts(b->sort_ws), b->plan, st);
  b->sorted = onesweep_sort(b->keys[0], b->keys[1], b->P, 32, b->plan, b->sort_ws, b->d_err, st, true,
                            b->sort_tile);
  // no reference-ordered triangle copy: the batch's cells hold a few
  // references each and the trace reads a reference's triangle through its
  // id (indices[]), which measured cheaper than gathering and writing 96 bytes
  // per reference in the build; the ranges are written by tiles of cells
  launch_cell_ranges(b->sorted, b->P, b->total_cells, b->cells, b->indices, st);
}

GridView batch_view(const shn_batch* b) {
  GridView v{};
  v.kind = 0;
  v.src = b->tri;
  v.ridx = b->indices;
  return v;
}

void enqueue_trace(shn_batch* b, const shn_rays* rays, uint32_t n, shn_hits* hits, uint8_t* occ,
                   cudaStream_t st) {
  cudaMemsetAsync(b->d_counter, 0, 4, st);
  const GridView G = batch_view(b);
  const BatchAcc A{b->d_scenes, b->cells};
  const RaysV R{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz, rays->tmax};
  if (occ) {
    k_batch_trace<true><<<b->blocks_any, kBatchTraceBlock, 0, st>>>(G, A, R, b->d_ray_off, b->ns, n, b->d_counter,
                                                             nullptr, nullptr, nullptr, nullptr, occ);
  } else {
    k_batch_trace<false><<<b->blocks_closest, kBatchTraceBlock, 0, st>>>(G, A, R, b->d_ray_off, b->ns, n, b->d_counter,
                                                              hits->tri, hits->t, hits->u, hits->v, nullptr);
  }
}

shn_status upload_ray_offsets(shn_batch* b, const uint32_t* ray_offsets, cudaStream_t st) {
  if (b->ray_off_cap < b->ns + 1) {
    cudaError_t e = own(b, (void**)&b->d_ray_off, ((size_t)b->ns + 1) * 4, st);
    if (e != cudaSuccess) return alloc_err(b, e, "ray offsets");
    b->ray_off_cap = b->ns + 1;
  }
  cudaMemcpyAsync(b->d_ray_off, ray_offsets, ((size_t)b->ns + 1) * 4, cudaMemcpyHostToDevice, st);
  return SHN_OK;
}

shn_status check_rays(shn_batch* b, const shn_rays* rays, const uint32_t* ray_offsets) {
  if (!rays || !ray_offsets || !rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz)
    return set_error(b->ctx, SHN_ERR_INVALID, "null rays / offsets");
  if (ray_offsets[0] != 0) return set_error(b->ctx, SHN_ERR_INVALID, "ray_offsets[0] must be 0");
  for (uint32_t s = 0; s < b->ns; ++s)
    if (ray_offsets[s + 1] < ray_offsets[s]) return set_error(b->ctx, SHN_ERR_INVALID, "ray_offsets not monotone");
  return SHN_OK;
}

}  // namespace
}  // namespace shn

using namespace shn;

extern "C" {

shn_status shn_batch_create(shn_ctx* ctx, uint32_t num_scenes, const float* vtx_xyz,
                            const uint32_t* vtx_offsets, const uint32_t* idx,
                            const uint32_t* tri_offsets, uint32_t mem, void* stream, shn_batch** out) {
  if (!ctx || !out || num_scenes == 0 || !vtx_offsets || !tri_offsets || mem > SHN_MEM_DEVICE)
    return SHN_ERR_INVALID;
  *out = nullptr;
  const uint32_t nv = vtx_offsets[num_scenes], T = tri_offsets[num_scenes];
  if ((nv && !vtx_xyz) || (T && !idx)) return SHN_ERR_INVALID;
  if (vtx_offsets[0] != 0 || tri_offsets[0] != 0) return set_error(ctx, SHN_ERR_INVALID, "offsets must start at 0");
  for (uint32_t s = 0; s < num_scenes; ++s)
    if (vtx_offsets[s + 1] < vtx_offsets[s] || tri_offsets[s + 1] < tri_offsets[s])
      return set_error(ctx, SHN_ERR_INVALID, "offsets not monotone");
  if (T >= (1u << 30) || nv >= (1u << 30)) return set_error(ctx, SHN_ERR_INVALID, "batch larger than 2^30 elements");
  if (mem == SHN_MEM_HOST) {
    for (size_t i = 0; i < 3 * (size_t)nv; ++i)
      if (!std::isfinite(vtx_xyz[i])) return set_error(ctx, SHN_ERR_INVALID, "non-finite vertex coordinate");
    for (uint32_t s = 0; s < num_scenes; ++s) {
      const uint32_t snv = vtx_offsets[s + 1] - vtx_offsets[s];
      for (size_t i = 3 * (size_t)tri_offsets[s]; i < 3 * (size_t)tri_offsets[s + 1]; ++i)
        if (idx[i] >= snv) return set_error(ctx, SHN_ERR_INVALID, "triangle index out of range of its scene");
    }
  }
  cudaStream_t st = (cudaStream_t)stream;
  shn_batch* b = new shn_batch();
  b->ctx = ctx;
  ctx_retain(ctx);
  b->ns = num_scenes;
  b->T = T;
  b->tri_off.assign(tri_offsets, tri_offsets + num_scenes + 1);
  b->vtx_off.assign(vtx_offsets, vtx_offsets + num_scenes + 1);
  b->lambdas.assign(num_scenes, 5.f);
  b->bytes_vtx = std::max<size_t>(12 * (size_t)nv, 16);
  b->bytes_idx = std::max<size_t>(12 * (size_t)T, 16);
  b->bytes_tri = std::max<size_t>(48 * (size_t)T, 16);
  cudaError_t e = dev_alloc(ctx, (void**)&b->vtx, b->bytes_vtx, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, (void**)&b->idx, b->bytes_idx, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, (void**)&b->tri, b->bytes_tri, st);
  if (e == cudaSuccess) e = cudaMalloc(&b->d_tri_off, 4 * ((size_t)num_scenes + 1));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_vtx_off, 4 * ((size_t)num_scenes + 1));
  if (e == cudaSuccess) e = cudaMalloc(&b->d_err, 64);
  if (e == cudaSuccess) e = cudaMallocHost(&b->h_pinned, 64);
  if (e != cudaSuccess) {
    shn_batch_destroy(b);
    return set_error(ctx, e == cudaErrorNotPermitted ? SHN_ERR_BUDGET : SHN_ERR_OOM, "batch scenes");
  }
  const cudaMemcpyKind kind = mem == SHN_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  if (nv) cudaMemcpyAsync(b->vtx, vtx_xyz, 12 * (size_t)nv, kind, st);
  if (T) cudaMemcpyAsync(b->idx, idx, 12 * (size_t)T, kind, st);
  cudaMemcpyAsync(b->d_tri_off, tri_offsets, 4 * ((size_t)num_scenes + 1), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(b->d_vtx_off, vtx_offsets, 4 * ((size_t)num_scenes + 1), cudaMemcpyHostToDevice, st);
  launch_batch_pack(b->vtx, b->d_vtx_off, b->idx, b->d_tri_off, num_scenes, T, b->tri, st);
  float* d_b = nullptr;
  e = dev_alloc(ctx, (void**)&d_b, 24 * (size_t)num_scenes, st);
  if (e != cudaSuccess) {
    shn_batch_destroy(b);
    return set_error(ctx, SHN_ERR_OOM, "batch bounds");
  }
  launch_batch_bounds(b->tri, b->d_tri_off, num_scenes, T, d_b, st);
  b->bounds.resize(6 * (size_t)num_scenes);
  cudaMemcpyAsync(b->bounds.data(), d_b, 24 * (size_t)num_scenes, cudaMemcpyDeviceToHost, st);
  dev_free(ctx, d_b, 24 * (size_t)num_scenes, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    shn_batch_destroy(b);
    return cuda_status(ctx, e, "batch create");
  }
  *out = b;
  return SHN_OK;
}

shn_status shn_batch_set_lambdas(shn_batch* b, const float* lambdas) {
  if (!b || !lambdas) return SHN_ERR_INVALID;
  for (uint32_t s = 0; s < b->ns; ++s)
    if (!(lambdas[s] > 0.f)) return set_error(b->ctx, SHN_ERR_INVALID, "lambda must be > 0");
  b->lambdas.assign(lambdas, lambdas + b->ns);
  b->planned = false;
  return SHN_OK;
}

shn_status shn_batch_build(shn_batch* b, void* stream) {
  if (!b) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  shn_status rc;
  if (!b->planned && (rc = plan(b, st))) return rc;
  cudaEvent_t e0, e1;
  cudaEventCreate(&e0);
  cudaEventCreate(&e1);
  cudaEventRecord(e0, st);
  enqueue_build(b, st);
  cudaEventRecord(e1, st);
  cudaMemcpyAsync(b->h_pinned, b->d_err, 4, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  cudaEventElapsedTime(&b->build_ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  if (e != cudaSuccess) return cuda_status(b->ctx, e, "batch build");
  if (b->h_pinned[0] & kErrCapacity) {
    b->planned = false;
    return set_error(b->ctx, SHN_ERR_INVALID, "pair count changed since planning; build again to re-plan");
  }
  if (b->h_pinned[0]) return set_error(b->ctx, SHN_ERR_TIMEOUT, "bounded device wait gave up (batch build)");
  b->built = true;
  return SHN_OK;
}

shn_status shn_batch_trace(shn_batch* b, const shn_rays* rays, const uint32_t* ray_offsets,
                           shn_hits* hits, uint8_t* d_occluded, void* stream) {
  if (!b) return SHN_ERR_INVALID;
  if (!b->built) return set_error(b->ctx, SHN_ERR_NOT_BUILT, "batch not built");
  shn_status rc = check_rays(b, rays, ray_offsets);
  if (rc) return rc;
  if (!d_occluded && (!hits || !hits->tri || !hits->t)) return set_error(b->ctx, SHN_ERR_INVALID, "no output");
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = upload_ray_offsets(b, ray_offsets, st))) return rc;
  const uint32_t n = ray_offsets[b->ns];
  if (n) enqueue_trace(b, rays, n, hits, d_occluded, st);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SHN_OK : cuda_status(b->ctx, e, "batch trace");
}

shn_status shn_batch_capture(shn_batch* b, const shn_rays* rays, const uint32_t* ray_offsets,
                             shn_hits* hits, void* stream) {
  if (!b || !hits || !hits->tri || !hits->t) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  shn_status rc;
  if (!b->planned && (rc = plan(b, st))) return rc;
  if ((rc = check_rays(b, rays, ray_offsets))) return rc;
  if ((rc = upload_ray_offsets(b, ray_offsets, st))) return rc;
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(b->ctx, e, "batch capture");
  if (b->exec) {
    cudaGraphExecDestroy(b->exec);
    b->exec = nullptr;
  }
  if (b->graph) {
    cudaGraphDestroy(b->graph);
    b->graph = nullptr;
  }
  cudaStream_t cs;
  cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking);
  e = cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal);
  if (e == cudaSuccess) {
    enqueue_build(b, cs);
    const uint32_t n = ray_offsets[b->ns];
    if (n) enqueue_trace(b, rays, n, hits, nullptr, cs);
    e = cudaStreamEndCapture(cs, &b->graph);
  }
  if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
  cudaStreamDestroy(cs);
  if (e != cudaSuccess) return cuda_status(b->ctx, e, "batch graph capture");
  b->built = true;
  return SHN_OK;
}

shn_status shn_batch_replay(shn_batch* b, void* stream) {
  if (!b || !b->exec) return b ? set_error(b->ctx, SHN_ERR_NOT_BUILT, "no captured graph") : SHN_ERR_INVALID;
  cudaError_t e = cudaGraphLaunch(b->exec, (cudaStream_t)stream);
  return e == cudaSuccess ? SHN_OK : cuda_status(b->ctx, e, "batch graph launch");
}

shn_status shn_batch_sync_status(shn_batch* b, void* stream) {
  if (!b) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  cudaError_t e = cudaMemcpyAsync(b->h_pinned + 2, b->d_err, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(b->ctx, e, "batch status");
  const uint32_t bits = b->h_pinned[2];
  if (!bits) return SHN_OK;
  e = cudaMemsetAsync(b->d_err, 0, 4, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(b->ctx, e, "batch status");
  if (bits & (kErrLookbackTimeout | kErrTmaTimeout))
    return set_error(b->ctx, SHN_ERR_TIMEOUT, "a bounded device wait gave up in a batch build, trace or replay");
  return set_error(b->ctx, SHN_ERR_INVALID, "pair capacity exceeded in a batch replay; build again to re-plan");
}

shn_status shn_batch_autotune(shn_batch* b, const float* candidates, uint32_t num_candidates,
                              const uint32_t* expected_rays, uint32_t sample_rays, uint32_t seed,
                              float* chosen, void* stream) {
  return shn_batch_autotune_ex(b, candidates, num_candidates, expected_rays, sample_rays, seed, nullptr, chosen,
                               nullptr, nullptr, stream);
}

shn_status shn_batch_autotune_ex(shn_batch* b, const float* candidates, uint32_t num_candidates,
                                 const uint32_t* expected_rays, uint32_t sample_rays, uint32_t seed,
                                 const shn_autotune_config* cfg, float* chosen, float* sah_out,
                                 shn_autotune_report* report, void* stream) {
  if (!b || !candidates || num_candidates == 0 || !expected_rays || sample_rays == 0) return SHN_ERR_INVALID;
  const uint32_t keep = cfg ? cfg->sah_keep : 0u;
  const uint32_t nshapes = cfg ? cfg->num_block_shapes : 0u;
  if (nshapes > 8 || (keep && num_candidates > 32)) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  shn_ctx* ctx = b->ctx;
  // sample rays (same distribution as the batched workload)
  float* rb = nullptr;
  const size_t rbytes = (size_t)sample_rays * 4 * 8;
  cudaError_t e = dev_alloc(ctx, (void**)&rb, rbytes, st);
  if (e != cudaSuccess) return alloc_err(b, e, "autotune rays");
  float* cols[8];
  for (int k = 0; k < 8; ++k) cols[k] = rb + (size_t)k * sample_rays;
  k_random_rays<<<(sample_rays + 255) / 256, 256, 0, st>>>(sample_rays, seed, -1.f, 2.f, cols[0], cols[1],
                                                           cols[2], cols[3], cols[4], cols[5]);
  shn_rays rays{cols[0], cols[1], cols[2], cols[3], cols[4], cols[5], nullptr};
  shn_hits hits{(uint32_t*)cols[6], cols[7], nullptr, nullptr};
  shn_status rc = SHN_OK;
  cudaEvent_t e1, e2;
  cudaEventCreate(&e1);
  cudaEventCreate(&e2);
  shn_grid* g = nullptr;
  shn_grid_create(ctx, &g);
  std::vector<float> best(b->ns, candidates[0]), best_sah(b->ns, 0.f);
  std::vector<int32_t> cres(3 * (size_t)num_candidates);
  std::vector<float> ccost(num_candidates);
  std::vector<uint32_t> order(num_candidates);
  uint32_t timed = 0;
  for (uint32_t s = 0; s < b->ns && rc == SHN_OK; ++s) {
    const uint32_t nt = b->tri_off[s + 1] - b->tri_off[s];
    if (nt == 0) continue;
    // a scene view over the batch's packed triangles
    shn_scene sc;
    sc.ctx = ctx;
    sc.nt = nt;
    sc.nv = 0;
    sc.tri = b->tri + 3 * (size_t)b->tri_off[s];  // the scene's records, in place
    sc.ids = b->tri;                               // their ids count from the batch's first record
    memcpy(sc.bounds, &b->bounds[6 * s], 24);
    for (uint32_t c = 0; c < num_candidates; ++c) {
      compute_resolution(nt, sc.bounds, candidates[c], 1, 1, &cres[3 * (size_t)c]);
      order[c] = c;
    }
    if (keep || sah_out) {
      // the SAH term: one counting launch over the scene for all candidates
      for (uint32_t c0 = 0; c0 < num_candidates && rc == SHN_OK; c0 += 32)
        rc = sah_refs_list(ctx, sc.tri, nt, sc.bounds, &cres[3 * (size_t)c0], std::min(32u, num_candidates - c0),
                           nullptr, &ccost[c0], st);
      if (rc) break;
      if (keep)
        std::stable_sort(order.begin(), order.end(), [&](uint32_t x, uint32_t y) { return ccost[x] < ccost[y]; });
    }
    const uint32_t ntime = keep ? std::min(keep, num_candidates) : num_candidates;
    double best_cost = 1e300;
    for (uint32_t k = 0; k < ntime; ++k) {
      const uint32_t c = order[k];
      shn_grid_params p;
      shn_grid_params_default(SHN_GRID_UNIFORM, &p);
      p.lambda = candidates[c];
      rc = build_grid(g, &sc, &p, st);
      if (rc) break;
      const uint32_t m = std::min(sample_rays, std::max<uint32_t>(expected_rays[s], 1024u));
      cudaEventRecord(e1, st);
      rc = shn_trace_closest(g, &rays, m, &hits, st);
      cudaEventRecord(e2, st);
      cudaEventSynchronize(e2);
      if (rc) break;
      ++timed;
      float trace_ms = 0.f;
      cudaEventElapsedTime(&trace_ms, e1, e2);
      const double cost = (double)grid_build_ms(g) + (double)trace_ms * ((double)expected_rays[s] / (double)m);
      if (cost < best_cost) {
        best_cost = cost;
        best[s] = candidates[c];
        best_sah[s] = ccost[c];
      }
    }
  }
  shn_grid_destroy(g);
  if (rc == SHN_OK) rc = shn_batch_set_lambdas(b, best.data());
  // the block-shape term: the persistent trace's resident blocks per SM, timed
  // on the chosen grids with the sample rays spread over the scenes like the
  // expected rays
  float shape_ms[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (rc == SHN_OK && nshapes) {
    rc = shn_batch_build(b, st);
    // a launch that fills the GPU many times over: at least 2^21 rays
    const uint32_t m = std::max<uint32_t>(sample_rays, 1u << 21);
    float* sb = nullptr;
    const size_t sbytes = (size_t)m * 4 * 8;
    if (rc == SHN_OK) {
      e = dev_alloc(ctx, (void**)&sb, sbytes, st);
      if (e != cudaSuccess) rc = alloc_err(b, e, "autotune shape rays");
    }
    float* sc8[8];
    for (int k = 0; k < 8; ++k) sc8[k] = sb ? sb + (size_t)k * m : nullptr;
    shn_rays srays{sc8[0], sc8[1], sc8[2], sc8[3], sc8[4], sc8[5], nullptr};
    shn_hits shits{(uint32_t*)sc8[6], sc8[7], nullptr, nullptr};
    if (rc == SHN_OK)
      k_random_rays<<<(m + 255) / 256, 256, 0, st>>>(m, seed + 1u, -1.f, 2.f, sc8[0], sc8[1], sc8[2], sc8[3],
                                                     sc8[4], sc8[5]);
    double total = 0.0;
    for (uint32_t s = 0; s < b->ns; ++s) total += expected_rays[s];
    std::vector<uint32_t> offs(b->ns + 1, 0u);
    double acc = 0.0;
    for (uint32_t s = 0; s < b->ns; ++s) {
      acc += expected_rays[s];
      offs[s + 1] = total > 0.0 ? (uint32_t)std::min<double>(m, std::floor(m * (acc / total))) : m;
    }
    offs[b->ns] = m;
    if (rc == SHN_OK) rc = upload_ray_offsets(b, offs.data(), st);
    float best_ms = FLT_MAX;
    uint32_t best_bps = 0;
    for (uint32_t i = 0; i < nshapes && rc == SHN_OK; ++i) {
      const uint32_t bps = cfg->blocks_per_sm[i];
      b->blocks_closest = bps ? (int)bps * ctx->num_sms : batch_blocks(k_batch_trace<false>, ctx->num_sms);
      float t[3];
      for (int r = 0; r < 3; ++r) {
        cudaEventRecord(e1, st);
        enqueue_trace(b, &srays, m, &shits, nullptr, st);
        cudaEventRecord(e2, st);
        e = cudaEventSynchronize(e2);
        if (e != cudaSuccess) {
          rc = cuda_status(ctx, e, "autotune shapes");
          break;
        }
        cudaEventElapsedTime(&t[r], e1, e2);
      }
      if (rc) break;
      std::sort(t, t + 3);
      shape_ms[i] = t[1];
      if (t[1] < best_ms) {
        best_ms = t[1];
        best_bps = bps;
      }
    }
    b->bps_closest = best_bps;
    b->blocks_closest = best_bps ? (int)best_bps * ctx->num_sms : batch_blocks(k_batch_trace<false>, ctx->num_sms);
    if (report) report->blocks_per_sm = best_bps;
    if (sb) dev_free(ctx, sb, sbytes, st);
  }
  // the sort-tile term: the batch's whole build timed with each tile shape
  const uint32_t ntiles = cfg ? cfg->num_sort_tiles : 0u;
  float tile_ms[4] = {0, 0, 0, 0};
  if (rc == SHN_OK && ntiles) {
    if (ntiles > 4) rc = set_error(ctx, SHN_ERR_INVALID, "at most 4 sort tile shapes");
    if (rc == SHN_OK && !b->planned) rc = plan(b, st);
    float best_ms = FLT_MAX;
    uint32_t best_tile = 0;
    for (uint32_t i = 0; i < ntiles && rc == SHN_OK; ++i) {
      const uint32_t tk = cfg->sort_tile_keys[i];
      if (tk != 0 && tk != 4096 && tk != 6144) {
        rc = set_error(ctx, SHN_ERR_INVALID, "sort tile shapes: 4096 or 6144 keys (0: 6144)");
        break;
      }
      b->sort_tile = tk == 6144 ? 0u : tk;
      float t[3];
      for (int r = 0; r < 3 && rc == SHN_OK; ++r) {
        cudaEventRecord(e1, st);
        enqueue_build(b, st);
        cudaEventRecord(e2, st);
        e = cudaEventSynchronize(e2);
        if (e != cudaSuccess) rc = cuda_status(ctx, e, "autotune sort tiles");
        else cudaEventElapsedTime(&t[r], e1, e2);
      }
      if (rc) break;
      std::sort(t, t + 3);
      tile_ms[i] = t[1];
      if (t[1] < best_ms) {
        best_ms = t[1];
        best_tile = b->sort_tile;
      }
    }
    b->sort_tile = best_tile;
    // the last timed build used the last shape: build once more with the chosen one
    if (rc == SHN_OK) rc = shn_batch_build(b, st);
  }
  cudaEventDestroy(e1);
  cudaEventDestroy(e2);
  dev_free(ctx, rb, rbytes, st);
  cudaStreamSynchronize(st);
  if (rc) return rc;
  if (chosen) memcpy(chosen, best.data(), 4 * (size_t)b->ns);
  if (sah_out) memcpy(sah_out, best_sah.data(), 4 * (size_t)b->ns);
  if (report) {
    report->timed_candidates = timed;
    if (!nshapes) report->blocks_per_sm = b->bps_closest;
    memcpy(report->shape_ms, shape_ms, sizeof(shape_ms));
    report->sort_tile_keys = b->sort_tile ? b->sort_tile : 6144u;
    memcpy(report->sort_tile_ms, tile_ms, sizeof(tile_ms));
  }
  return SHN_OK;
}

shn_status shn_batch_info(const shn_batch* b, uint64_t* num_pairs, uint64_t* total_cells, float* build_ms) {
  if (!b) return SHN_ERR_INVALID;
  if (num_pairs) *num_pairs = b->P;
  if (total_cells) *total_cells = b->total_cells;
  if (build_ms) *build_ms = b->build_ms;
  return b->planned ? SHN_OK : SHN_ERR_NOT_BUILT;
}

shn_status shn_batch_export_scene(const shn_batch* b, uint32_t scene, int32_t res[3], float bounds[6],
                                  uint32_t* cells, uint32_t* indices, uint64_t* num_refs) {
  if (!b || scene >= b->ns) return SHN_ERR_INVALID;
  if (!b->built) return set_error(b->ctx, SHN_ERR_NOT_BUILT, "batch not built");
  const BatchScene& sc = b->scenes[scene];
  if (res)
    for (int i = 0; i < 3; ++i) res[i] = sc.g.res[i];
  if (bounds) memcpy(bounds, &b->bounds[6 * scene], 24);
  std::vector<uint32_t> h(2 * (size_t)sc.ncells);
  cudaError_t e = cudaMemcpy(h.data(), b->cells + sc.cell_offset, 8 * (size_t)sc.ncells, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_status(b->ctx, e, "export");
  // the scene's references are one contiguous block of the global sorted array
  uint32_t lo = 0xFFFFFFFFu, hi = 0;
  for (uint32_t c = 0; c < sc.ncells; ++c)
    if (h[2 * c + 1] > h[2 * c]) {
      lo = std::min(lo, h[2 * c]);
      hi = std::max(hi, h[2 * c + 1]);
    }
  if (lo == 0xFFFFFFFFu) lo = hi = 0;
  for (uint32_t c = 0; c < sc.ncells; ++c) {
    if (h[2 * c + 1] > h[2 * c]) {
      h[2 * c] -= lo;
      h[2 * c + 1] -= lo;
    } else {
      h[2 * c] = h[2 * c + 1] = 0;
    }
  }
  if (cells) memcpy(cells, h.data(), h.size() * 4);
  if (num_refs) *num_refs = hi - lo;
  if (indices && hi > lo) {
    e = cudaMemcpy(indices, b->indices + lo, 4 * (size_t)(hi - lo), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return cuda_status(b->ctx, e, "export");
    for (uint32_t i = 0; i < hi - lo; ++i) indices[i] -= sc.tri_offset;
  }
  return SHN_OK;
}

void shn_batch_destroy(shn_batch* b) {
  if (!b) return;
  cudaStream_t st = 0;
  release_plan(b, st);
  dev_free(b->ctx, b->vtx, b->bytes_vtx, st);
  dev_free(b->ctx, b->idx, b->bytes_idx, st);
  dev_free(b->ctx, b->tri, b->bytes_tri, st);
  if (b->d_tri_off) cudaFree(b->d_tri_off);
  if (b->d_vtx_off) cudaFree(b->d_vtx_off);
  if (b->d_err) cudaFree(b->d_err);
  if (b->h_pinned) cudaFreeHost(b->h_pinned);
  shn_ctx* c = b->ctx;
  delete b;
  ctx_release(c);
}

}  // extern "C"
