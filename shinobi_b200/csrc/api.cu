// C ABI: context, scene (FaceSoup) and grid lifecycle, error reporting,
// stream-ordered device memory with an HBM budget, and the primitive entry
// points.  See include/shinobi_b200.h for the contract of every call.
#include <cmath>
#include <cstdio>

#include "internal.h"

namespace shn {

cudaError_t dev_alloc(shn_ctx* ctx, void** p, size_t bytes, cudaStream_t st) {
  if (ctx->budget) {
    const uint64_t now = ctx->used.fetch_add(bytes) + bytes;
    if (now > ctx->budget) {
      ctx->used.fetch_sub(bytes);
      return cudaErrorNotPermitted;
    }
  } else {
    ctx->used.fetch_add(bytes);
  }
  cudaError_t e = cudaMallocFromPoolAsync(p, bytes, ctx->pool, st);
  if (e != cudaSuccess) {
    ctx->used.fetch_sub(bytes);
    cudaGetLastError();
  }
  return e;
}

void dev_free(shn_ctx* ctx, void* p, size_t bytes, cudaStream_t st) {
  if (!p) return;
  cudaFreeAsync(p, st);
  ctx->used.fetch_sub(bytes);
}

shn_status set_error(shn_ctx* ctx, shn_status s, const std::string& msg) {
  if (ctx) {
    std::lock_guard<std::mutex> lk(ctx->mu);
    ctx->last_error = msg;
  }
  return s;
}

shn_status cuda_status(shn_ctx* ctx, cudaError_t e, const char* where) {
  std::string m = std::string(where) + ": " + cudaGetErrorString(e);
  return set_error(ctx, e == cudaErrorMemoryAllocation ? SHN_ERR_OOM : SHN_ERR_CUDA, m);
}

}  // namespace shn

using namespace shn;

namespace {

shn_status alloc_status(shn_ctx* ctx, cudaError_t e, const char* what) {
  if (e == cudaErrorNotPermitted) return set_error(ctx, SHN_ERR_BUDGET, std::string(what) + ": HBM budget exceeded");
  if (e == cudaErrorMemoryAllocation) return set_error(ctx, SHN_ERR_OOM, std::string(what) + ": out of device memory");
  return cuda_status(ctx, e, what);
}

shn_status copy_in(shn_ctx* ctx, void* dst, const void* src, size_t bytes, uint32_t mem,
                   cudaStream_t st) {
  cudaError_t e = cudaMemcpyAsync(dst, src, bytes,
                                  mem == SHN_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
  return e == cudaSuccess ? SHN_OK : cuda_status(ctx, e, "copy");
}

// Branch-free reductions (vectorised by the host compiler): any exponent
// field of all ones marks an inf/NaN coordinate; the largest index must be
// below nv.
shn_status validate_host(shn_ctx* ctx, const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt) {
  const uint32_t* bits = reinterpret_cast<const uint32_t*>(vtx);
  uint32_t bad = 0;
  for (size_t i = 0; i < 3 * (size_t)nv; ++i) bad |= (uint32_t)((bits[i] & 0x7F800000u) == 0x7F800000u);
  if (bad) return set_error(ctx, SHN_ERR_INVALID, "non-finite vertex coordinate");
  if (idx && nt) {
    uint32_t mx = 0;
    for (size_t i = 0; i < 3 * (size_t)nt; ++i) mx = idx[i] > mx ? idx[i] : mx;
    if (mx >= nv) return set_error(ctx, SHN_ERR_INVALID, "triangle index out of range");
  }
  return SHN_OK;
}

// Sets *flag when any of the n words is an inf/NaN float (exponent all ones).
__global__ void k_nonfinite(const uint32_t* __restrict__ bits, size_t n, uint32_t* flag) {
  uint32_t bad = 0;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    bad |= (uint32_t)((__ldg(bits + i) & 0x7F800000u) == 0x7F800000u);
  if (__any_sync(0xFFFFFFFFu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1u);
}

// kf1 * (1 - c) + kf2 * c for the first m coordinates, kf2 for the rest.
__global__ void k_lerp_vertices(const float* __restrict__ kf1, const float* __restrict__ kf2, size_t m, size_t n,
                                float omc, float c, float* __restrict__ out) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    out[i] = i < m ? __ldg(kf1 + i) * omc + __ldg(kf2 + i) * c : __ldg(kf2 + i);
}

shn_status refresh_bounds(shn_scene* s, cudaStream_t st) {
  float* d6 = nullptr;
  cudaError_t e = dev_alloc(s->ctx, (void**)&d6, 64, st);
  if (e != cudaSuccess) return alloc_status(s->ctx, e, "bounds");
  launch_bounds_reduce(s->tri, s->nt, d6, st);
  float h6[6];
  cudaMemcpyAsync(h6, d6, sizeof(h6), cudaMemcpyDeviceToHost, st);
  dev_free(s->ctx, d6, 64, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(s->ctx, e, "scene bounds");
  for (int i = 0; i < 3; ++i)
    if (!(h6[i] <= h6[i + 3]) && s->nt) return set_error(s->ctx, SHN_ERR_INVALID, "empty or non-finite scene bounds");
  memcpy(s->bounds, h6, sizeof(h6));
  return SHN_OK;
}

}  // namespace

namespace shn {
void ctx_retain(shn_ctx* c) { c->refs.fetch_add(1); }

uint32_t* pinned_take(shn_ctx* c) {
  std::lock_guard<std::mutex> lk(c->pin_mu);
  if (c->pin_free.empty()) {
    constexpr size_t kSlab = 64 << 10;
    void* slab = nullptr;
    if (cudaMallocHost(&slab, kSlab) != cudaSuccess) return nullptr;
    c->pin_slabs.push_back(slab);
    for (size_t off = 0; off < kSlab; off += 64) c->pin_free.push_back((uint32_t*)((char*)slab + off));
  }
  uint32_t* p = c->pin_free.back();
  c->pin_free.pop_back();
  return p;
}

void pinned_give(shn_ctx* c, uint32_t* p) {
  if (!p) return;
  std::lock_guard<std::mutex> lk(c->pin_mu);
  c->pin_free.push_back(p);
}

void ctx_release(shn_ctx* c) {
  if (!c || c->refs.fetch_sub(1) != 1) return;
  cudaSetDevice(c->device);
  cudaDeviceSynchronize();
  if (c->d_err) cudaFree(c->d_err);
  if (c->pool) cudaMemPoolDestroy(c->pool);
  for (void* slab : c->pin_slabs) cudaFreeHost(slab);
  delete c;
}
}  // namespace shn

namespace shn {
shn_status scene_reload(shn_scene* s, const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                        cudaStream_t st) {
  if (!s || (nv && !vtx) || (nt && !idx)) return SHN_ERR_INVALID;
  shn_ctx* ctx = s->ctx;
  if (nt >= (1u << 30) || nv >= (1u << 30)) return set_error(ctx, SHN_ERR_INVALID, "scene larger than 2^30 elements");
  shn_status rc = validate_host(ctx, vtx, nv, idx, nt);
  if (rc) return rc;
  struct Buf {
    void** p;
    size_t* cap;
    size_t need;
  } bufs[3] = {{(void**)&s->vtx, &s->cap_v, std::max<size_t>(12 * (size_t)nv, 16)},
               {(void**)&s->idx, &s->cap_i, std::max<size_t>(12 * (size_t)nt, 16)},
               {(void**)&s->tri, &s->cap_t, std::max<size_t>(48 * (size_t)nt, 16)}};
  for (Buf& b : bufs) {
    if (*b.cap >= b.need) continue;
    dev_free(ctx, *b.p, *b.cap, st);
    *b.p = nullptr;
    *b.cap = 0;
    const cudaError_t e = dev_alloc(ctx, b.p, b.need, st);
    if (e != cudaSuccess) return alloc_status(ctx, e, "scene");
    *b.cap = b.need;
  }
  s->nv = nv;
  s->nt = nt;
  s->bytes = s->cap_v + s->cap_i + s->cap_t;
  if (nv) rc = copy_in(ctx, s->vtx, vtx, 12 * (size_t)nv, SHN_MEM_HOST, st);
  if (!rc && nt) rc = copy_in(ctx, s->idx, idx, 12 * (size_t)nt, SHN_MEM_HOST, st);
  if (rc) return rc;
  launch_pack_triangles(s->vtx, s->idx, nt, s->tri, st);
  return refresh_bounds(s, st);
}
}  // namespace shn

extern "C" {

uint32_t shn_abi_version(void) { return SHN_ABI_VERSION; }

const char* shn_status_string(shn_status s) {
  switch (s) {
    case SHN_OK: return "ok";
    case SHN_ERR_INVALID: return "invalid argument";
    case SHN_ERR_CUDA: return "CUDA error";
    case SHN_ERR_OOM: return "out of device memory";
    case SHN_ERR_TIMEOUT: return "bounded device wait gave up";
    case SHN_ERR_BUDGET: return "HBM budget exceeded";
    case SHN_ERR_NOT_BUILT: return "grid not built";
    case SHN_ERR_BUSY: return "busy";
    case SHN_ERR_CANCELLED: return "cancelled";
  }
  return "unknown status";
}

shn_status shn_ctx_create(int device, uint64_t hbm_budget_bytes, shn_ctx** out) {
  if (!out) return SHN_ERR_INVALID;
  *out = nullptr;
  cudaError_t e = cudaSetDevice(device);
  if (e != cudaSuccess) return SHN_ERR_CUDA;
  shn_ctx* c = new shn_ctx();
  c->device = device;
  c->budget = hbm_budget_bytes;
  cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, device);
  cudaMemPoolProps props = {};
  props.allocType = cudaMemAllocationTypePinned;
  props.location.type = cudaMemLocationTypeDevice;
  props.location.id = device;
  e = cudaMemPoolCreate(&c->pool, &props);
  if (e != cudaSuccess) {
    delete c;
    return SHN_ERR_CUDA;
  }
  uint64_t thr = UINT64_MAX;
  cudaMemPoolSetAttribute(c->pool, cudaMemPoolAttrReleaseThreshold, &thr);
  if (cudaMalloc(&c->d_err, 64) != cudaSuccess) {
    cudaMemPoolDestroy(c->pool);
    delete c;
    return SHN_ERR_OOM;
  }
  cudaMemset(c->d_err, 0, 64);
  *out = c;
  return SHN_OK;
}

void shn_ctx_destroy(shn_ctx* c) { ctx_release(c); }

const char* shn_ctx_last_error(const shn_ctx* c) { return c ? c->last_error.c_str() : ""; }

shn_status shn_ctx_memory(const shn_ctx* c, uint64_t* used, uint64_t* budget) {
  if (!c) return SHN_ERR_INVALID;
  if (used) *used = c->used.load();
  if (budget) *budget = c->budget;
  return SHN_OK;
}

// ---- scene -----------------------------------------------------------------------
shn_status shn_scene_create(shn_ctx* ctx, const float* vtx, uint32_t nv, const uint32_t* idx,
                            uint32_t nt, uint32_t mem, void* stream, shn_scene** out) {
  if (!ctx || !out || (nv && !vtx) || (nt && !idx) || mem > SHN_MEM_DEVICE) return SHN_ERR_INVALID;
  *out = nullptr;
  if (nt >= (1u << 30) || nv >= (1u << 30)) return set_error(ctx, SHN_ERR_INVALID, "scene larger than 2^30 elements");
  if (mem == SHN_MEM_HOST) {
    shn_status v = validate_host(ctx, vtx, nv, idx, nt);
    if (v) return v;
  }
  cudaStream_t st = (cudaStream_t)stream;
  shn_scene* s = new shn_scene();
  s->ctx = ctx;
  ctx_retain(ctx);
  s->nv = nv;
  s->nt = nt;
  const size_t bv = std::max<size_t>(12 * (size_t)nv, 16), bi = std::max<size_t>(12 * (size_t)nt, 16),
               bt = std::max<size_t>(48 * (size_t)nt, 16);
  cudaError_t e = dev_alloc(ctx, (void**)&s->vtx, bv, st);
  if (e == cudaSuccess) {
    s->cap_v = bv;
    e = dev_alloc(ctx, (void**)&s->idx, bi, st);
  }
  if (e == cudaSuccess) {
    s->cap_i = bi;
    e = dev_alloc(ctx, (void**)&s->tri, bt, st);
  }
  if (e != cudaSuccess) {
    shn_scene_destroy(s);
    return alloc_status(ctx, e, "scene");
  }
  s->cap_t = bt;
  s->bytes = bv + bi + bt;
  shn_status rc = SHN_OK;
  if (nv) rc = copy_in(ctx, s->vtx, vtx, 12 * (size_t)nv, mem, st);
  if (!rc && nt) rc = copy_in(ctx, s->idx, idx, 12 * (size_t)nt, mem, st);
  if (!rc) {
    launch_pack_triangles(s->vtx, s->idx, nt, s->tri, st);
    rc = refresh_bounds(s, st);
  }
  if (rc) {
    shn_scene_destroy(s);
    return rc;
  }
  *out = s;
  return SHN_OK;
}

shn_status shn_scene_update_vertices(shn_scene* s, const float* vtx, uint32_t nv, uint32_t mem,
                                     void* stream) {
  if (!s || !vtx || nv != s->nv || mem > SHN_MEM_DEVICE) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  shn_status rc;
  if (mem == SHN_MEM_HOST) {
    // host vertices are checked on the device: copied to a staging buffer,
    // scanned for inf/NaN, and only then copied over the scene's vertices,
    // so a rejected update leaves the scene as it was
    const size_t vb = 12 * (size_t)nv;
    char* stage = nullptr;
    cudaError_t e = dev_alloc(s->ctx, (void**)&stage, vb + 256, st);
    if (e != cudaSuccess) return alloc_status(s->ctx, e, "vertex staging");
    uint32_t* flag = (uint32_t*)(stage + ((vb + 255) & ~(size_t)255));
    uint32_t* h = pinned_take(s->ctx);
    if (!h) {
      dev_free(s->ctx, stage, vb + 256, st);
      return set_error(s->ctx, SHN_ERR_OOM, "pinned");
    }
    cudaMemsetAsync(flag, 0, 4, st);
    rc = copy_in(s->ctx, stage, vtx, vb, mem, st);
    if (!rc && nv) {
      const size_t n = 3 * (size_t)nv;
      const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 8);
      k_nonfinite<<<blocks, 256, 0, st>>>((const uint32_t*)stage, n, flag);
    }
    cudaMemcpyAsync(h, flag, 4, cudaMemcpyDeviceToHost, st);
    if (!rc) {
      e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) rc = cuda_status(s->ctx, e, "vertex check");
    }
    const uint32_t bad = rc ? 0u : h[0];
    pinned_give(s->ctx, h);
    if (!rc && bad) rc = set_error(s->ctx, SHN_ERR_INVALID, "non-finite vertex coordinate");
    if (!rc) rc = copy_in(s->ctx, s->vtx, stage, vb, SHN_MEM_DEVICE, st);
    dev_free(s->ctx, stage, vb + 256, st);
    if (rc) return rc;
  } else {
    rc = copy_in(s->ctx, s->vtx, vtx, 12 * (size_t)nv, mem, st);
    if (rc) return rc;
  }
  launch_pack_triangles(s->vtx, s->idx, s->nt, s->tri, st);
  return refresh_bounds(s, st);
}

shn_status shn_scene_interpolate_vertices(shn_scene* s, const float* kf1, uint32_t n1, const float* kf2,
                                          float coeff, void* stream) {
  if (!s || !kf2 || (n1 && !kf1) || n1 > s->nv) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  const size_t n = 3 * (size_t)s->nv;
  if (n) {
    const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 148 * 8);
    k_lerp_vertices<<<blocks, 256, 0, st>>>(kf1, kf2, 3 * (size_t)n1, n, 1.f - coeff, coeff, s->vtx);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(s->ctx, e, "interpolate vertices");
  }
  launch_pack_triangles(s->vtx, s->idx, s->nt, s->tri, st);
  return refresh_bounds(s, st);
}

shn_status shn_scene_bounds(const shn_scene* s, float out[6]) {
  if (!s || !out) return SHN_ERR_INVALID;
  memcpy(out, s->bounds, sizeof(s->bounds));
  return SHN_OK;
}

uint32_t shn_scene_num_triangles(const shn_scene* s) { return s ? s->nt : 0; }

void shn_scene_destroy(shn_scene* s) {
  if (!s) return;
  cudaStream_t st = 0;
  dev_free(s->ctx, s->vtx, s->cap_v, st);
  dev_free(s->ctx, s->idx, s->cap_i, st);
  dev_free(s->ctx, s->tri, s->cap_t, st);
  shn_ctx* c = s->ctx;
  delete s;
  ctx_release(c);
}


// ---- grid --------------------------------------------------------------------------
void shn_grid_params_default(uint32_t kind, shn_grid_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->kind = kind;
  p->lambda = 5.f;
  p->lambda_leaf = 1.2f;
  p->leaf_threshold = 16;
  if (kind == SHN_GRID_TWO_LEVEL) {
    p->top_divisor = 6;
    p->min_res = 2;
  } else {
    p->top_divisor = 1;
    p->min_res = 1;
  }
}

shn_status shn_grid_create(shn_ctx* ctx, shn_grid** out) {
  if (!ctx || !out) return SHN_ERR_INVALID;
  shn_grid* g = new shn_grid();
  g->ctx = ctx;
  ctx_retain(ctx);
  *out = g;
  return SHN_OK;
}

shn_status shn_grid_build(shn_grid* g, const shn_scene* s, const shn_grid_params* p, void* stream) {
  if (!g || !s || !p) return SHN_ERR_INVALID;
  if (p->kind > SHN_GRID_TWO_LEVEL || !(p->lambda > 0.f) || (p->kind == SHN_GRID_TWO_LEVEL && !(p->lambda_leaf > 0.f)))
    return set_error(g->ctx, SHN_ERR_INVALID, "bad grid parameters");
  if (s->ctx != g->ctx) return set_error(g->ctx, SHN_ERR_INVALID, "scene and grid belong to different contexts");
  shn_status rc = build_grid(g, s, p, (cudaStream_t)stream);
  if (rc == SHN_OK) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_status(g->ctx, e, "grid build");
  }
  return rc;
}

shn_status shn_grid_get_info(const shn_grid* g, shn_grid_info* o) {
  if (!g || !o) return SHN_ERR_INVALID;
  memset(o, 0, sizeof(*o));
  o->kind = g->kind;
  for (int i = 0; i < 3; ++i) {
    o->res[i] = g->geom.res[i];
    o->cell_size[i] = comp(g->geom.cs, i);
  }
  o->bounds[0] = g->geom.gmin.x; o->bounds[1] = g->geom.gmin.y; o->bounds[2] = g->geom.gmin.z;
  o->bounds[3] = g->geom.gmax.x; o->bounds[4] = g->geom.gmax.y; o->bounds[5] = g->geom.gmax.z;
  o->num_cells = g->num_cells;
  o->num_top_refs = g->num_top_refs;
  o->num_leaves = g->num_leaves;
  o->num_refs = g->num_refs;
  o->device_bytes = g->cap_cells + g->cap_leaves + g->cap_refs + g->cap_rtri + g->offs_tri.bytes +
                    g->offs_pair.bytes + g->scan.bytes + g->top_ranges.bytes + g->keys[0].bytes +
                    g->keys[1].bytes + g->keys[2].bytes + g->sortws.bytes + g->mhi.bytes + g->perm_tri.bytes +
                    g->cbox.bytes + g->sbox.bytes + g->ldist.bytes;
  o->build_ms = g->built ? grid_build_ms(g) : 0.f;
  return g->built ? SHN_OK : SHN_ERR_NOT_BUILT;
}

shn_status shn_grid_export(const shn_grid* g, uint32_t* cells, uint32_t* leaves, uint32_t* indices,
                           uint64_t* top_pairs) {
  if (!g) return SHN_ERR_INVALID;
  if (!g->built) return set_error(g->ctx, SHN_ERR_NOT_BUILT, "grid not built");
  cudaError_t e = g->ev1 ? cudaEventSynchronize(g->ev1) : cudaSuccess;  // the build's end
  if (e == cudaSuccess && cells && g->num_cells) e = cudaMemcpy(cells, g->cells, g->num_cells * 8, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && leaves && g->num_leaves) e = cudaMemcpy(leaves, g->leaves, g->num_leaves * 8, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && indices && g->num_refs) e = cudaMemcpy(indices, g->indices, g->num_refs * 4, cudaMemcpyDeviceToHost);
  const uint64_t np = g->kind == SHN_GRID_TWO_LEVEL ? g->num_top_refs : g->num_refs;
  if (e == cudaSuccess && top_pairs && np) e = cudaMemcpy(top_pairs, g->top_pairs, np * 8, cudaMemcpyDeviceToHost);
  if (e == cudaSuccess && cells && g->cell_dist) {
    // empty cells of a large uniform grid carry their distance to the nearest
    // non-empty cell on the device; exported, an empty cell is [0, 0)
    for (uint64_t i = 0; i < g->num_cells; ++i)
      if (cells[2 * i] == cells[2 * i + 1]) cells[2 * i] = cells[2 * i + 1] = 0;
  }
  if (e == cudaSuccess && leaves && g->spatial) {
    // empty leaves carry their distance to the nearest non-empty leaf on the
    // device; exported, an empty leaf is [0, 0)
    for (uint64_t i = 0; i < g->num_leaves; ++i)
      if (leaves[2 * i] == leaves[2 * i + 1]) leaves[2 * i] = leaves[2 * i + 1] = 0;
  }
  if (e == cudaSuccess && g->spatial) {
    // a two-level grid was built on the triangles in Morton order: the
    // references of a leaf are in that order and the pairs' low words are
    // positions in it; both are put back in (cell, triangle id) order
    if (indices && g->num_refs) {
      std::vector<uint2> lv(g->num_leaves);
      e = cudaMemcpy(lv.data(), g->leaves, g->num_leaves * 8, cudaMemcpyDeviceToHost);
      for (size_t i = 0; e == cudaSuccess && i < lv.size(); ++i)
        if (lv[i].y > lv[i].x) std::sort(indices + lv[i].x, indices + lv[i].y);
    }
    if (e == cudaSuccess && top_pairs && np) {
      std::vector<float4> pt((size_t)g->src_nt * 3);
      e = cudaMemcpy(pt.data(), g->perm_tri.ptr, pt.size() * sizeof(float4), cudaMemcpyDeviceToHost);
      for (uint64_t i = 0; e == cudaSuccess && i < np; ++i) {
        uint32_t id;
        memcpy(&id, &pt[3 * (size_t)(uint32_t)top_pairs[i]].w, 4);
        top_pairs[i] = (top_pairs[i] & 0xFFFFFFFF00000000ull) | id;
      }
      if (e == cudaSuccess) std::sort(top_pairs, top_pairs + np);
    }
  }
  return e == cudaSuccess ? SHN_OK : cuda_status(g->ctx, e, "grid export");
}

void shn_grid_destroy(shn_grid* g) {
  if (!g) return;
  if (g->ev1) cudaEventSynchronize(g->ev1);  // the last build may still run on its stream
  cudaStream_t st = 0;
  shn_ctx* c = g->ctx;
  dev_free(c, g->cells, g->cap_cells, st);
  dev_free(c, g->leaves, g->cap_leaves, st);
  dev_free(c, g->indices, g->cap_refs, st);
  dev_free(c, g->rtri, g->cap_rtri, st);
  DevBuf* bufs[] = {&g->offs_tri, &g->offs_pair, &g->scan,     &g->top_ranges, &g->keys[0], &g->keys[1],
                    &g->keys[2],   &g->sortws,    &g->mhi,      &g->perm_tri,   &g->cbox,    &g->sbox,
                    &g->ldist};
  for (DevBuf* b : bufs) dev_free(c, b->ptr, b->bytes, st);
  dev_free(c, g->d_err, 64, st);
  pinned_give(c, g->h_pinned);
  if (g->ev0) cudaEventDestroy(g->ev0);
  if (g->ev1) cudaEventDestroy(g->ev1);
  delete g;
  ctx_release(c);
}

// ---- primitives -------------------------------------------------------------------------
shn_status shn_exclusive_scan_u32(shn_ctx* ctx, const uint32_t* in, uint32_t* out, uint32_t n,
                                  void* stream) {
  if (!ctx || !out || (n && !in)) return SHN_ERR_INVALID;
  if (n >= (1u << 31)) return set_error(ctx, SHN_ERR_INVALID, "n >= 2^31");
  cudaStream_t st = (cudaStream_t)stream;
  void* ws = nullptr;
  const size_t wb = scan_workspace_bytes(n);
  cudaError_t e = dev_alloc(ctx, &ws, wb, st);
  if (e != cudaSuccess) return alloc_status(ctx, e, "scan workspace");
  const uint32_t armed = ctx->force_lookback.exchange(0);
  if (!launch_exclusive_scan(in, out, n, ws, ctx->d_err, st, armed != 0) && armed) ctx->force_lookback.store(armed);
  dev_free(ctx, ws, wb, st);
  e = cudaGetLastError();
  return e == cudaSuccess ? SHN_OK : cuda_status(ctx, e, "exclusive_scan");
}

shn_status shn_compact_u32(shn_ctx* ctx, const uint32_t* flags, uint32_t n, uint32_t* out_idx,
                           uint32_t* d_count, void* stream) {
  if (!ctx || !d_count || (n && (!flags || !out_idx))) return SHN_ERR_INVALID;
  if (n >= (1u << 31)) return set_error(ctx, SHN_ERR_INVALID, "n >= 2^31");
  cudaStream_t st = (cudaStream_t)stream;
  void* ws = nullptr;
  const size_t wb = scan_workspace_bytes(n);
  cudaError_t e = dev_alloc(ctx, &ws, wb, st);
  if (e != cudaSuccess) return alloc_status(ctx, e, "compact workspace");
  const uint32_t armed = ctx->force_lookback.exchange(0);
  if (!launch_compact(flags, n, out_idx, d_count, ws, ctx->d_err, st, armed != 0) && armed)
    ctx->force_lookback.store(armed);
  dev_free(ctx, ws, wb, st);
  e = cudaGetLastError();
  return e == cudaSuccess ? SHN_OK : cuda_status(ctx, e, "compact");
}

shn_status shn_sort_keys_u64(shn_ctx* ctx, uint64_t* keys, uint64_t* tmp, uint32_t n,
                             uint32_t lo_bit, uint32_t hi_bit, void* stream) {
  if (!ctx || (n && (!keys || !tmp)) || hi_bit > 64 || lo_bit > hi_bit) return SHN_ERR_INVALID;
  if (n >= (1u << 30)) return set_error(ctx, SHN_ERR_INVALID, "n >= 2^30");
  if (hi_bit - lo_bit > 32) return set_error(ctx, SHN_ERR_INVALID, "at most 32 key bits per sort");
  const SortPlan plan = sort_plan(hi_bit - lo_bit);
  cudaStream_t st = (cudaStream_t)stream;
  void* ws = nullptr;
  const size_t wb = sort_workspace_bytes(n);
  cudaError_t e = dev_alloc(ctx, &ws, wb, st);
  if (e != cudaSuccess) return alloc_status(ctx, e, "sort workspace");
  uint64_t* res = onesweep_sort(keys, tmp, n, lo_bit, plan, ws, ctx->d_err, st);
  if (res != keys && n) cudaMemcpyAsync(keys, res, (size_t)n * 8, cudaMemcpyDeviceToDevice, st);
  dev_free(ctx, ws, wb, st);
  e = cudaGetLastError();
  return e == cudaSuccess ? SHN_OK : cuda_status(ctx, e, "sort");
}

// ---- device-side status -------------------------------------------------------------
}  // extern "C"

namespace {

// Synchronises the stream, then reads and clears the error word.
shn_status read_and_clear(shn_ctx* ctx, uint32_t* d_word, cudaStream_t st, const char* what) {
  uint32_t* h = pinned_take(ctx);
  if (!h) return set_error(ctx, SHN_ERR_OOM, "pinned");
  h[0] = 0;
  cudaError_t e = cudaMemcpyAsync(h, d_word, 4, cudaMemcpyDeviceToHost, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  const uint32_t bits = h[0];
  pinned_give(ctx, h);
  if (e != cudaSuccess) return cuda_status(ctx, e, what);
  if (!bits) return SHN_OK;
  e = cudaMemsetAsync(d_word, 0, 4, st);
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(ctx, e, what);
  std::string m = std::string(what) + ": a bounded device wait gave up (";
  if (bits & kErrLookbackTimeout) m += "look-back";
  if (bits & kErrTmaTimeout) m += (bits & kErrLookbackTimeout) ? ", bulk copy" : "bulk copy";
  if (bits & kErrCapacity) m += (bits & (kErrLookbackTimeout | kErrTmaTimeout)) ? ", capacity" : "capacity";
  m += "); the results of the calls since the last check are not valid";
  return set_error(ctx, (bits & (kErrLookbackTimeout | kErrTmaTimeout)) ? SHN_ERR_TIMEOUT : SHN_ERR_INVALID, m);
}

}  // namespace

extern "C" {

shn_status shn_ctx_sync_status(shn_ctx* ctx, void* stream) {
  if (!ctx) return SHN_ERR_INVALID;
  return read_and_clear(ctx, ctx->d_err, (cudaStream_t)stream, "context primitives");
}

shn_status shn_grid_sync_status(const shn_grid* g, void* stream) {
  if (!g) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  if (!g->d_err) {  // never built: nothing of this grid ran on the device
    const cudaError_t e = cudaStreamSynchronize(st);
    return e == cudaSuccess ? SHN_OK : cuda_status(g->ctx, e, "grid status");
  }
  if (g->ev1) cudaEventSynchronize(g->ev1);  // the build's tail, whatever its stream
  return read_and_clear(g->ctx, g->d_err, st, "grid");
}

shn_status shn_debug_force_lookback_timeout(uint32_t target, shn_ctx* ctx, shn_grid* g) {
  if (target == SHN_FORCE_CTX_SCAN) {
    if (!ctx) return SHN_ERR_INVALID;
    ctx->force_lookback.store(1);
    return SHN_OK;
  }
  if (target == SHN_FORCE_GRID_COMPACTION) {
    if (!g) return SHN_ERR_INVALID;
    g->force_lookback.store(1);
    return SHN_OK;
  }
  if (target == SHN_FORCE_NOALLOC_SCAN) return noalloc_force_lookback_timeout();
  return SHN_ERR_INVALID;
}

}  // extern "C"
