// Persistent, warp-scheduled trace kernels: each warp takes 32 rays at a time
// from a global atomic pool (the reference's trace<> kernel took 96-ray
// batches per warp, src/Engine/RayTracingKernels.h:60-100) and traces them to
// completion.  Variants: SoA rays (closest / any), in-kernel camera rays
// (RegularPrimaryRayGenerator) and in-kernel ambient-occlusion rays
// generated from compacted primary hits, and the shadow segments of direct
// illumination from an area light with their per-pixel shading.
#include "internal.h"
#include "trace.cuh"
#include "trace_coop.cuh"

namespace shn {

namespace {

constexpr int kTraceBlock = 128;

struct RaysView {
  const float *ox, *oy, *oz, *dx, *dy, *dz, *tmax;
};

// Work counters of the stats variants: {cell visits, triangle tests}, warp-aggregated.
template <bool STATS>
SHN_D void add_stats(unsigned long long* stats, const Hit& h, bool valid) {
  if (!STATS) return;
  unsigned long long s = valid ? h.steps : 0u, t = valid ? h.tests : 0u;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    s += __shfl_xor_sync(0xFFFFFFFFu, s, o);
    t += __shfl_xor_sync(0xFFFFFFFFu, t, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(stats, s);
    atomicAdd(stats + 1, t);
  }
}

template <bool STATS>
SHN_D void add_counts(unsigned long long* stats, uint32_t steps, uint32_t tests) {
  if (!STATS) return;
  atomicAdd(stats, (unsigned long long)steps);
  atomicAdd(stats + 1, (unsigned long long)tests);
}

template <int KIND, bool ANY, bool STATS>
__global__ void __launch_bounds__(kTraceBlock, 8) k_trace_rays(GridView G, RaysView R, uint32_t n,
                                                            uint32_t* counter, uint32_t* otri,
                                                            float* ot, float* ou, float* ov,
                                                            uint8_t* occ, unsigned long long* stats,
                                                            uint32_t* err) {
  warp_trace<KIND, ANY>(
      G, n, counter,
      [&](uint32_t i, V3& o, V3& d, float& tmax) {
        o = mk(R.ox[i], R.oy[i], R.oz[i]);
        d = mk(R.dx[i], R.dy[i], R.dz[i]);
        tmax = R.tmax ? R.tmax[i] : FLT_MAX;
      },
      [&](uint32_t i, const Hit& h, uint32_t steps, uint32_t tests) {
        if (ANY) {
          occ[i] = h.tri != kMiss ? 1 : 0;
        } else {
          otri[i] = h.tri;
          ot[i] = h.t;
          if (ou) ou[i] = h.u;
          if (ov) ov[i] = h.v;
        }
        add_counts<STATS>(stats, steps, tests);
      });
}

template <int KIND, bool STATS>
__global__ void __launch_bounds__(kTraceBlock, 8) k_trace_camera(GridView G, CamView cam,
                                                              uint32_t image_id, uint32_t n,
                                                              uint32_t* counter, uint32_t* otri,
                                                              float* ot, float* ou, float* ov,
                                                              unsigned long long* stats,
                                                              uint32_t* err) {
  warp_trace<KIND, false, true>(
      G, n, counter,
      [&](uint32_t i, V3& o, V3& d, float& tmax) {
        o = cam.eye;
        d = primary_dir(cam, tile_pixel(cam, i), image_id);
        tmax = FLT_MAX;
      },
      [&](uint32_t r, const Hit& h, uint32_t steps, uint32_t tests) {
        const uint32_t i = tile_pixel(cam, r);
        otri[i] = h.tri;
        ot[i] = h.t;
        if (ou) ou[i] = h.u;
        if (ov) ov[i] = h.v;
        add_counts<STATS>(stats, steps, tests);
      });
}

// Compaction of hit pixels: hit_idx[k] = k-th pixel with a hit, pos[p] = its rank.
__global__ void __launch_bounds__(256) k_compact_hits(const uint32_t* __restrict__ tri, uint32_t n,
                                                      uint32_t* __restrict__ hit_idx,
                                                      uint32_t* __restrict__ pos, uint32_t* d_m,
                                                      LookbackState st) {
  __shared__ TileScanSmem<256, 8> sm;
  tile_scan<256, 8>(
      st, n, sm, [&](uint32_t i) { return tri[i] != kMiss ? 1u : 0u; },
      [&](uint32_t i, uint32_t ex) {
        pos[i] = ex;
        if (tri[i] != kMiss) hit_idx[ex] = i;
      },
      d_m);
}

struct AoParams {
  CamView cam;
  uint32_t image_id, spp, seed;
  float len, offset;
  const float4* stri;  // scene triangles, 48-byte records (v0, v1, v2)
  uint32_t snt;
  uint32_t npix;
};

template <int KIND, bool STATS>
__global__ void __launch_bounds__(kTraceBlock, 6) k_trace_ao(GridView G, AoParams A,
                                                          const uint32_t* __restrict__ ptri,
                                                          const float* __restrict__ pt,
                                                          const uint32_t* __restrict__ hit_idx,
                                                          const uint32_t* d_m, uint32_t* counter,
                                                          uint8_t* __restrict__ occ,
                                                          unsigned long long* stats,
                                                          uint32_t* err) {
  const uint32_t n = (*d_m) * A.spp;
  warp_trace<KIND, true, true>(
      G, n, counter,
      [&](uint32_t r, V3& o, V3& dir, float& tmax) {
        const uint32_t k = r / A.spp, s = r - k * A.spp;
        const uint32_t p = hit_idx[k];
        // a compaction whose look-back gave up (error bit set) can leave a
        // slot unwritten: such a ray becomes an empty segment, no access leaves
        // the pixel and triangle arrays
        const uint32_t tri = p < A.npix ? ptri[p] : kMiss;
        if (tri >= A.snt) {
          o = A.cam.eye;
          dir = mk(0.f, 0.f, 1.f);
          tmax = 0.f;
          return;
        }
        const float t = pt[p];
        const V3 d = primary_dir(A.cam, p, A.image_id);
        const float4* rec = A.stri + 3 * (size_t)tri;
        const V3 v0 = f4v(__ldg(rec));
        const V3 v1 = f4v(__ldg(rec + 1));
        const V3 v2 = f4v(__ldg(rec + 2));
        const V3 e1 = sub(v1, v0);
        V3 nn = normalize(cross(e1, sub(v2, v0)));
        if (dot(nn, d) > 0.f) nn = mk(-nn.x, -nn.y, -nn.z);
        const V3 tx = normalize(e1);
        const V3 ty = cross(nn, tx);
        const V3 hp = add(A.cam.eye, muls(d, t));
        o = add(hp, muls(nn, A.offset));
        const uint4 w = philox4x32(make_uint4(p, s, 0u, 0x414Fu), A.seed, 0u);
        const float u1 = u01(w.x), u2 = u01(w.y);
        float sn, cs;
        sincos_2pi(u1, sn, cs);
        const float rr = sqrtf(1.f - u2);
        const float lx = sn * rr, ly = cs * rr, lz = sqrtf(u2);
        dir = mk(tx.x * lx + ty.x * ly + nn.x * lz, tx.y * lx + ty.y * ly + nn.y * lz,
                 tx.z * lx + ty.z * ly + nn.z * lz);
        tmax = A.len;
      },
      [&](uint32_t r, const Hit& h, uint32_t steps, uint32_t tests) {
        occ[r] = h.tri != kMiss ? 1 : 0;
        add_counts<STATS>(stats, steps, tests);
      });
}

__global__ void k_ao_finalize(const uint32_t* __restrict__ ptri, const uint32_t* __restrict__ pos,
                              const uint8_t* __restrict__ occ, uint32_t n, uint32_t spp,
                              const uint32_t* d_m, float* __restrict__ ao, uint32_t* d_num_rays) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && d_num_rays) *d_num_rays = (*d_m) * spp;
  if (p >= n) return;
  if (ptri[p] == kMiss) {
    ao[p] = 1.0f;
    return;
  }
  const uint32_t q = pos[p];
  if (q >= *d_m) {  // only after a look-back that gave up (error bit set)
    ao[p] = 1.0f;
    return;
  }
  const uint32_t b = q * spp;
  uint32_t c = 0;
  for (uint32_t s = 0; s < spp; ++s) c += occ[b + s];
  ao[p] = 1.0f - (float)c / (float)spp;
}

// Direct illumination from a parallelogram light (DirectIlluminationIntegrator::shade,
// src/Integrator/DirectIlluminationIntegrator.h:254-315, and computeDirectIllumination,
// src/Integrator/DirectIlluminationIntegrator.h:46-168).
struct DiParams {
  CamView cam;
  V3 lpos, le1, le2, lnrm, lint, ddef, bg;
  float larea;
  uint32_t spp, seed, image_id, nmat, npix;
  const float4* stri;        // scene triangles, 48-byte records (v0, v1, v2)
  const uint32_t* tri_mat;   // per scene triangle, or null
  const float4* diffuse;     // per material, or null
};

// Shadow segment of sample s of hit pixel p: the origin is the stored hit point
// eye + (t - EPS) d (SimpleRayBuffer::store, src/Engine/RayBuffers.h:52-55), the
// direction runs to a uniform point of the light (AreaLightShadowRayGenerator,
// src/Engine/RayGenerators.h:106-139; AreaLightSource::getPoint,
// src/Primitive/LightSource.hpp:40-43); Philox replaces the KISS generator.
SHN_D void di_segment(const DiParams& P, uint32_t p, uint32_t s, float t, V3& o, V3& L) {
  const V3 d = primary_dir(P.cam, p, P.image_id);
  o = add(P.cam.eye, muls(d, t - 1e-5f));
  const uint4 w = philox4x32(make_uint4(p, s, P.image_id, 0x444Cu), P.seed, 0u);
  const V3 lp = add(add(P.lpos, muls(P.le1, u01(w.x))), muls(P.le2, u01(w.y)));
  L = sub(lp, o);
}

template <int KIND, bool STATS>
__global__ void __launch_bounds__(kTraceBlock, 6) k_trace_direct(GridView G, DiParams P,
                                                              const float* __restrict__ pt,
                                                              const uint32_t* __restrict__ hit_idx,
                                                              const uint32_t* d_m, uint32_t* counter,
                                                              uint8_t* __restrict__ occ,
                                                              unsigned long long* stats,
                                                              uint32_t* err) {
  const uint32_t n = (*d_m) * P.spp;
  warp_trace<KIND, true, true>(
      G, n, counter,
      [&](uint32_t r, V3& o, V3& dir, float& tmax) {
        const uint32_t k = r / P.spp, s = r - k * P.spp;
        const uint32_t p = hit_idx[k];
        if (p >= P.npix) {  // slot left unwritten by a look-back that gave up
          o = P.cam.eye;
          dir = mk(0.f, 0.f, 1.f);
          tmax = 0.f;
          return;
        }
        di_segment(P, p, s, pt[p], o, dir);
        tmax = 0.9999f;
      },
      [&](uint32_t r, const Hit& h, uint32_t steps, uint32_t tests) {
        occ[r] = h.tri != kMiss ? 1 : 0;
        add_counts<STATS>(stats, steps, tests);
      });
}

// Per pixel: the mean over samples of the light's contribution
// (computeDirectIllumination, src/Integrator/DirectIlluminationIntegrator.h:97-159),
// then the progressive blend into the final image.
__global__ void __launch_bounds__(256) k_shade_direct(DiParams P, const uint32_t* __restrict__ ptri,
                                                      const float* __restrict__ pt,
                                                      const uint32_t* __restrict__ pos,
                                                      const uint8_t* __restrict__ occ, uint32_t n,
                                                      const uint32_t* d_m, float* __restrict__ frame,
                                                      float* __restrict__ fin, uint32_t* d_num_rays) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p == 0 && d_num_rays) *d_num_rays = (*d_m) * P.spp;
  if (p >= n) return;
  const float inv_s = 1.0f / (float)P.spp;
  const uint32_t tri = ptri[p];
  V3 rad = mk(0.f, 0.f, 0.f);
  if (tri == kMiss) {
    for (uint32_t s = 0; s < P.spp; ++s) rad = add(rad, muls(P.bg, inv_s));
  } else {
    const float t = pt[p];
    const float4* rec = P.stri + 3 * (size_t)tri;
    const V3 v0 = f4v(__ldg(rec));
    const V3 nrm = normalize(cross(sub(f4v(__ldg(rec + 1)), v0), sub(f4v(__ldg(rec + 2)), v0)));
    V3 diff = P.ddef;
    if (P.diffuse) {
      uint32_t m = P.tri_mat ? __ldg(P.tri_mat + tri) : 0u;
      if (m >= P.nmat) m = 0u;
      diff = f4v(__ldg(P.diffuse + m));
    }
    const V3 k = mul(muls(P.lint, P.larea), diff);
    const uint32_t q = pos[p];
    const bool valid = q < *d_m;  // false only after a look-back that gave up
    const uint8_t* oc = occ + (size_t)q * P.spp;
    for (uint32_t s = 0; s < P.spp; ++s) {
      if (!valid || oc[s]) continue;
      V3 o, L;
      di_segment(P, p, s, t, o, L);
      const V3 ln = normalize(L);
      const float att = 1.0f / dot(L, L);
      const float a = fmaxf(0.f, -dot(P.lnrm, ln));
      const float b = fmaxf(0.f, dot(nrm, ln));
      rad = add(rad, muls(muls(muls(muls(k, a), b), att), inv_s));
    }
  }
  float* f = frame + 3 * (size_t)p;
  f[0] = rad.x;
  f[1] = rad.y;
  f[2] = rad.z;
  if (fin) {
    const float wn = 1.0f / (float)(P.image_id + 1u);
    const float wo = 1.0f - wn;
    float* g = fin + 3 * (size_t)p;
    g[0] = g[0] * wo + rad.x * wn;
    g[1] = g[1] * wo + rad.y * wn;
    g[2] = g[2] * wo + rad.z * wn;
  }
}

template <class K>
int persistent_blocks(K kernel, int num_sms) {
  int per_sm = 0;
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kTraceBlock, 0);
  return std::max(1, per_sm) * num_sms;
}

GridView view_of(const shn_grid* g) {
  GridView v;
  v.g = g->geom;
  v.kind = g->kind;
  v.cells = g->cells;
  v.leaves = g->leaves;
  v.rv0 = g->rtri;
  v.rv1 = g->rtri + g->num_refs;
  v.rv2 = g->rtri + 2 * g->num_refs;
  v.src = g->src_tri;
  v.cbox = g->num_blocks ? (const float4*)g->cbox.ptr : nullptr;
  v.sbox = g->num_blocks ? (const float4*)g->sbox.ptr : nullptr;
  v.ridx = nullptr;
  return v;
}

// Per-call scratch from the context pool, released stream-ordered.
struct Scratch {
  shn_ctx* ctx;
  cudaStream_t st;
  std::vector<std::pair<void*, size_t>> items;
  cudaError_t err = cudaSuccess;
  template <class T>
  T* get(size_t count) {
    void* p = nullptr;
    const size_t bytes = std::max<size_t>(count * sizeof(T), 16);
    cudaError_t e = dev_alloc(ctx, &p, bytes, st);
    if (e != cudaSuccess) {
      err = e;
      return nullptr;
    }
    items.emplace_back(p, bytes);
    return (T*)p;
  }
  ~Scratch() {
    for (auto& it : items) dev_free(ctx, it.first, it.second, st);
  }
};

shn_status check_launch(shn_ctx* ctx, const char* what) {
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SHN_OK : cuda_status(ctx, e, what);
}

}  // namespace

CamView make_camera(const shn_camera* c) {
  // Camera::init (src/Primitive/Camera.h:41-60), host FP32 as in the reference.
  const float aspect = (float)c->res_x / (float)c->res_y;
  const V3 f = normalize(mk(c->forward[0], c->forward[1], c->forward[2]));
  const V3 r = normalize(cross(f, mk(c->up[0], c->up[1], c->up[2])));
  const V3 u = normalize(cross(f, r));
  const float ang = c->fov_deg * 3.14159265358979323846f / 180.f;
  const float tn = tanf(ang / 2.f);
  const V3 row = muls(muls(muls(r, 2.f), tn), aspect);
  const V3 col = muls(muls(u, 2.f), tn);
  CamView v;
  v.eye = mk(c->eye[0], c->eye[1], c->eye[2]);
  v.sx = mk(row.x / (float)c->res_x, row.y / (float)c->res_x, row.z / (float)c->res_x);
  v.sy = mk(col.x / (float)c->res_y, col.y / (float)c->res_y, col.z / (float)c->res_y);
  v.tl = sub(sub(f, mk(row.x / 2.f, row.y / 2.f, row.z / 2.f)), mk(col.x / 2.f, col.y / 2.f, col.z / 2.f));
  v.resx = (float)c->res_x;
  v.res_x = c->res_x;
  v.res_y = c->res_y;
  return v;
}

}  // namespace shn

using namespace shn;

extern "C" {

shn_status shn_grid_set_stats(shn_grid* g, uint64_t* d_counters) {
  if (!g) return SHN_ERR_INVALID;
  g->stats = (unsigned long long*)d_counters;
  return SHN_OK;
}

shn_status shn_trace_closest(const shn_grid* g, const shn_rays* rays, uint32_t n, shn_hits* hits,
                             void* stream) {
  if (!g || !rays || !hits) return SHN_ERR_INVALID;
  if (!g->built) return set_error(g->ctx, SHN_ERR_NOT_BUILT, "grid not built");
  grid_fence(g, (cudaStream_t)stream);
  if (n == 0) return SHN_OK;
  if (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz || !hits->tri || !hits->t)
    return set_error(g->ctx, SHN_ERR_INVALID, "null ray or hit array");
  cudaStream_t st = (cudaStream_t)stream;
  Scratch S{g->ctx, st};
  uint32_t* counter = S.get<uint32_t>(1);
  if (!counter) return set_error(g->ctx, SHN_ERR_OOM, "trace scratch");
  cudaMemsetAsync(counter, 0, 4, st);
  const GridView G = view_of(g);
  const RaysView R{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz, rays->tmax};
#define SHN_LAUNCH_RAYS(K, S)                                                                   \
  {                                                                                             \
    static int blocks = persistent_blocks(k_trace_rays<K, false, S>, g->ctx->num_sms);          \
    k_trace_rays<K, false, S><<<blocks, kTraceBlock, 0, st>>>(G, R, n, counter, hits->tri,      \
                                                            hits->t, hits->u, hits->v, nullptr, \
                                                            g->stats, g->d_err);                          \
  }
  if (g->kind == SHN_GRID_UNIFORM) {
    if (g->stats) SHN_LAUNCH_RAYS(0, true) else SHN_LAUNCH_RAYS(0, false)
  } else {
    if (g->stats) SHN_LAUNCH_RAYS(1, true) else SHN_LAUNCH_RAYS(1, false)
  }
#undef SHN_LAUNCH_RAYS
  return check_launch(g->ctx, "trace_closest");
}

shn_status shn_trace_any(const shn_grid* g, const shn_rays* rays, uint32_t n, uint8_t* d_occluded,
                         void* stream) {
  if (!g || !rays || !d_occluded) return SHN_ERR_INVALID;
  if (!g->built) return set_error(g->ctx, SHN_ERR_NOT_BUILT, "grid not built");
  grid_fence(g, (cudaStream_t)stream);
  if (n == 0) return SHN_OK;
  if (!rays->ox || !rays->oy || !rays->oz || !rays->dx || !rays->dy || !rays->dz)
    return set_error(g->ctx, SHN_ERR_INVALID, "null ray array");
  cudaStream_t st = (cudaStream_t)stream;
  Scratch S{g->ctx, st};
  uint32_t* counter = S.get<uint32_t>(1);
  if (!counter) return set_error(g->ctx, SHN_ERR_OOM, "trace scratch");
  cudaMemsetAsync(counter, 0, 4, st);
  const GridView G = view_of(g);
  const RaysView R{rays->ox, rays->oy, rays->oz, rays->dx, rays->dy, rays->dz, rays->tmax};
#define SHN_LAUNCH_ANY(K, S)                                                                    \
  {                                                                                             \
    static int blocks = persistent_blocks(k_trace_rays<K, true, S>, g->ctx->num_sms);           \
    k_trace_rays<K, true, S><<<blocks, kTraceBlock, 0, st>>>(G, R, n, counter, nullptr, nullptr, \
                                                           nullptr, nullptr, d_occluded,        \
                                                           g->stats, g->d_err);                           \
  }
  if (g->kind == SHN_GRID_UNIFORM) {
    if (g->stats) SHN_LAUNCH_ANY(0, true) else SHN_LAUNCH_ANY(0, false)
  } else {
    if (g->stats) SHN_LAUNCH_ANY(1, true) else SHN_LAUNCH_ANY(1, false)
  }
#undef SHN_LAUNCH_ANY
  return check_launch(g->ctx, "trace_any");
}

shn_status shn_trace_primary(const shn_grid* g, const shn_camera* cam, uint32_t image_id,
                             shn_hits* hits, void* stream) {
  if (!g || !cam || !hits || !hits->tri || !hits->t) return SHN_ERR_INVALID;
  if (!g->built) return set_error(g->ctx, SHN_ERR_NOT_BUILT, "grid not built");
  grid_fence(g, (cudaStream_t)stream);
  const uint64_t n64 = (uint64_t)cam->res_x * cam->res_y;
  if (n64 == 0) return SHN_OK;
  if (n64 > (1u << 24)) return set_error(g->ctx, SHN_ERR_INVALID, "more than 2^24 pixels");
  const uint32_t n = (uint32_t)n64;
  cudaStream_t st = (cudaStream_t)stream;
  Scratch S{g->ctx, st};
  uint32_t* counter = S.get<uint32_t>(1);
  if (!counter) return set_error(g->ctx, SHN_ERR_OOM, "trace scratch");
  cudaMemsetAsync(counter, 0, 4, st);
  const GridView G = view_of(g);
  const CamView C = make_camera(cam);
#define SHN_LAUNCH_CAM(K, S)                                                                    \
  {                                                                                             \
    static int blocks = persistent_blocks(k_trace_camera<K, S>, g->ctx->num_sms);               \
    k_trace_camera<K, S><<<blocks, kTraceBlock, 0, st>>>(G, C, image_id, n, counter, hits->tri, \
                                                       hits->t, hits->u, hits->v, g->stats, \
                                                       g->d_err);    \
  }
  if (g->kind == SHN_GRID_UNIFORM) {
    if (g->stats) SHN_LAUNCH_CAM(0, true) else SHN_LAUNCH_CAM(0, false)
  } else {
    if (g->stats) SHN_LAUNCH_CAM(1, true) else SHN_LAUNCH_CAM(1, false)
  }
#undef SHN_LAUNCH_CAM
  return check_launch(g->ctx, "trace_primary");
}

shn_status shn_trace_ao(const shn_grid* g, const shn_camera* cam, const shn_hits* primary,
                        uint32_t spp, float length, float offset, uint32_t seed, float* d_ao,
                        uint32_t* d_num_rays, void* stream) {
  if (!g || !cam || !primary || !primary->tri || !primary->t || !d_ao || spp == 0) return SHN_ERR_INVALID;
  if (!g->built) return set_error(g->ctx, SHN_ERR_NOT_BUILT, "grid not built");
  grid_fence(g, (cudaStream_t)stream);
  if (!g->src_tri) return set_error(g->ctx, SHN_ERR_INVALID, "grid has no scene");
  const uint64_t n64 = (uint64_t)cam->res_x * cam->res_y;
  if (n64 == 0) return SHN_OK;
  if (n64 > (1u << 24) || n64 * spp >= (1ull << 32)) return set_error(g->ctx, SHN_ERR_INVALID, "too many AO rays");
  const uint32_t n = (uint32_t)n64;
  cudaStream_t st = (cudaStream_t)stream;
  Scratch S{g->ctx, st};
  uint32_t* counter = S.get<uint32_t>(4);
  uint32_t* hit_idx = S.get<uint32_t>(n);
  uint32_t* pos = S.get<uint32_t>(n);
  uint8_t* occ = S.get<uint8_t>((size_t)n * spp);
  const size_t tiles = (n + 2047) / 2048;
  uint64_t* status = S.get<uint64_t>(tiles + 2);
  if (S.err != cudaSuccess) return set_error(g->ctx, SHN_ERR_OOM, "ao scratch");
  cudaMemsetAsync(counter, 0, 16, st);
  cudaMemsetAsync(status, 0, (tiles + 2) * 8, st);
  LookbackState ls{status, (uint32_t*)(status + tiles + 1), g->d_err};
  uint32_t* d_m = counter + 1;
  const uint32_t armed = g->force_lookback.exchange(0);
  const uint32_t cblocks = lookback_blocks((uint32_t)tiles, ls.ticket, armed != 0, st);
  if (armed && cblocks == tiles) g->force_lookback.store(armed);
  k_compact_hits<<<cblocks, 256, 0, st>>>(primary->tri, n, hit_idx, pos, d_m, ls);
  const GridView G = view_of(g);
  AoParams A;
  A.cam = make_camera(cam);
  A.image_id = 0;
  A.spp = spp;
  A.seed = seed;
  A.len = length;
  A.offset = offset;
  A.stri = g->src_tri;
  A.snt = g->src_nt;
  A.npix = n;
#define SHN_LAUNCH_AO(K, S)                                                                       \
  {                                                                                               \
    static int blocks = persistent_blocks(k_trace_ao<K, S>, g->ctx->num_sms);                     \
    k_trace_ao<K, S><<<blocks, kTraceBlock, 0, st>>>(G, A, primary->tri, primary->t, hit_idx, d_m, \
                                                   counter, occ, g->stats, g->d_err);                       \
  }
  if (g->kind == SHN_GRID_UNIFORM) {
    if (g->stats) SHN_LAUNCH_AO(0, true) else SHN_LAUNCH_AO(0, false)
  } else {
    if (g->stats) SHN_LAUNCH_AO(1, true) else SHN_LAUNCH_AO(1, false)
  }
#undef SHN_LAUNCH_AO
  k_ao_finalize<<<(n + 255) / 256, 256, 0, st>>>(primary->tri, pos, occ, n, spp, d_m, d_ao, d_num_rays);
  return check_launch(g->ctx, "trace_ao");
}

void shn_di_params_default(shn_di_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  const float pos[3] = {-0.05f, 0.2f, -0.05f}, e1[3] = {0.1f, 0.f, 0.f}, e2[3] = {0.f, 0.f, 0.1f},
              nrm[3] = {0.f, -1.f, 0.f}, inten[3] = {10.f, 10.f, 10.f};
  memcpy(p->light.position, pos, 12);
  memcpy(p->light.edge1, e1, 12);
  memcpy(p->light.edge2, e2, 12);
  memcpy(p->light.normal, nrm, 12);
  memcpy(p->light.intensity, inten, 12);
  p->samples = 4;
  p->seed = 1;
  for (int i = 0; i < 3; ++i) p->default_diffuse[i] = 0.7f;
  p->background[0] = 0.15f;
  p->background[1] = 0.2f;
  p->background[2] = 0.3f;
}

shn_status shn_shade_direct(const shn_grid* g, const shn_camera* cam, const shn_hits* primary,
                            const shn_di_params* prm, float* d_frame, float* d_final,
                            uint32_t* d_num_rays, void* stream) {
  if (!g || !cam || !primary || !primary->tri || !primary->t || !prm || !d_frame || prm->samples == 0)
    return SHN_ERR_INVALID;
  if (!g->built) return set_error(g->ctx, SHN_ERR_NOT_BUILT, "grid not built");
  grid_fence(g, (cudaStream_t)stream);
  if (!g->src_tri) return set_error(g->ctx, SHN_ERR_INVALID, "grid has no scene");
  if (prm->diffuse && prm->num_materials == 0)
    return set_error(g->ctx, SHN_ERR_INVALID, "diffuse table without materials");
  const uint64_t n64 = (uint64_t)cam->res_x * cam->res_y;
  if (n64 == 0) return SHN_OK;
  if (n64 > (1u << 24) || n64 * prm->samples >= (1ull << 32))
    return set_error(g->ctx, SHN_ERR_INVALID, "too many shadow rays");
  const uint32_t n = (uint32_t)n64;
  cudaStream_t st = (cudaStream_t)stream;
  Scratch S{g->ctx, st};
  uint32_t* counter = S.get<uint32_t>(4);
  uint32_t* hit_idx = S.get<uint32_t>(n);
  uint32_t* pos = S.get<uint32_t>(n);
  uint8_t* occ = S.get<uint8_t>((size_t)n * prm->samples);
  const size_t tiles = (n + 2047) / 2048;
  uint64_t* status = S.get<uint64_t>(tiles + 2);
  if (S.err != cudaSuccess) return set_error(g->ctx, SHN_ERR_OOM, "direct-illumination scratch");
  cudaMemsetAsync(counter, 0, 16, st);
  cudaMemsetAsync(status, 0, (tiles + 2) * 8, st);
  LookbackState ls{status, (uint32_t*)(status + tiles + 1), g->d_err};
  uint32_t* d_m = counter + 1;
  const uint32_t armed = g->force_lookback.exchange(0);
  const uint32_t cblocks = lookback_blocks((uint32_t)tiles, ls.ticket, armed != 0, st);
  if (armed && cblocks == tiles) g->force_lookback.store(armed);
  k_compact_hits<<<cblocks, 256, 0, st>>>(primary->tri, n, hit_idx, pos, d_m, ls);
  const GridView G = view_of(g);
  const shn_area_light& l = prm->light;
  DiParams P;
  P.cam = make_camera(cam);
  P.lpos = mk(l.position[0], l.position[1], l.position[2]);
  P.le1 = mk(l.edge1[0], l.edge1[1], l.edge1[2]);
  P.le2 = mk(l.edge2[0], l.edge2[1], l.edge2[2]);
  P.lnrm = mk(l.normal[0], l.normal[1], l.normal[2]);
  P.lint = mk(l.intensity[0], l.intensity[1], l.intensity[2]);
  const V3 ln = cross(P.le1, P.le2);
  P.larea = sqrtf(dot(ln, ln));  // AreaLightSource::getArea, src/Primitive/LightSource.hpp:45-48
  P.ddef = mk(prm->default_diffuse[0], prm->default_diffuse[1], prm->default_diffuse[2]);
  P.bg = mk(prm->background[0], prm->background[1], prm->background[2]);
  P.spp = prm->samples;
  P.seed = prm->seed;
  P.image_id = prm->image_id;
  P.nmat = prm->num_materials;
  P.npix = n;
  P.stri = g->src_tri;
  P.tri_mat = prm->tri_material;
  P.diffuse = (const float4*)prm->diffuse;
#define SHN_LAUNCH_DI(K, S)                                                                          \
  {                                                                                                  \
    static int blocks = persistent_blocks(k_trace_direct<K, S>, g->ctx->num_sms);                    \
    k_trace_direct<K, S><<<blocks, kTraceBlock, 0, st>>>(G, P, primary->t, hit_idx, d_m, counter,   \
                                                       occ, g->stats, g->d_err);                     \
  }
  if (g->kind == SHN_GRID_UNIFORM) {
    if (g->stats) SHN_LAUNCH_DI(0, true) else SHN_LAUNCH_DI(0, false)
  } else {
    if (g->stats) SHN_LAUNCH_DI(1, true) else SHN_LAUNCH_DI(1, false)
  }
#undef SHN_LAUNCH_DI
  k_shade_direct<<<(n + 255) / 256, 256, 0, st>>>(P, primary->tri, primary->t, pos, occ, n, d_m, d_frame,
                                                  d_final, d_num_rays);
  return check_launch(g->ctx, "shade_direct");
}

}  // extern "C"
