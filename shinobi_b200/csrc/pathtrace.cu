// Wavefront path tracer with stream compaction after every bounce.
//
// The reference runs its path tracer as a persistent megakernel in which
// finished paths leave their lanes idle until the whole warp is done
// (src/Integrator/SimplePathTracer.hpp:65-241, src/Shinobi.h:152-230).  Here
// every bounce is one persistent trace+shade kernel over the live paths,
// followed by a decoupled look-back compaction that packs the survivors
// (64-byte records) for the next bounce, so warps only ever see live paths.
//
// Semantics (restated by the oracle path for path):
//  * path g = sample * npix + (the pixel's number in 8x4-tile order); camera ray through the pixel with a
//    Philox jitter (RandomPixelSampler, src/Primitive/PixelSampler.h:56-70);
//  * at a hit: facing geometric normal n; next-event estimation to one
//    point of the parallelogram light (shadow segment, any hit, t < 0.9999
//    as in OcclusionRayBuffer, src/Engine/RayBuffers.h:156-169); Russian
//    roulette with continuation probability = albedo from depth rr_depth
//    on; cosine-weighted bounce (CosineHemisphereSampler,
//    src/Utils/HemisphereSamplers.hpp:54-72) in the frame {e1, n x e1, n};
//  * a miss adds throughput * background;
//  * each path writes its radiance to its own slot; the image is the
//    per-pixel mean over samples summed in sample order (deterministic).
// Random numbers: Philox4x32-10, counter (pixel, sample, depth, tag), key (seed, 0).
#include "internal.h"
#include "trace.cuh"

namespace shn {

namespace {

constexpr int kPtBlock = 128;
constexpr uint32_t kTagJitter = 0x4A49u, kTagLight = 0x4C54u, kTagDir = 0x4449u;

struct PtView {
  CamView cam;
  uint32_t npix, spp, max_depth, rr_depth, seed;
  float albedo, offset;
  V3 lpos, le1, le2, lrad, lnrm, bg;
  float larea;
  const float4* stri;
  uint32_t snt;
};

// Path record: r0 = org.xyz, beta.x; r1 = dir.xyz, beta.y; r2 = L.xyz, beta.z;
// r3 = (pixel, sample, depth, 0) bits.
struct PathRec {
  float4 r0, r1, r2, r3;
};

__global__ void k_pt_camera(PtView P, uint64_t g0, uint32_t count, PathRec* __restrict__ out,
                            uint32_t* d_n) {
  const uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k == 0) *d_n = count;
  if (k >= count) return;
  const uint64_t g = g0 + k;
  // path g = sample s, camera ray number g - s * npix, numbered by 8x4 pixel
  // tiles: a warp's 32 paths are one compact tile of one sample
  const uint32_t s = (uint32_t)(g / P.npix);
  const uint32_t p = tile_pixel(P.cam, (uint32_t)(g - (uint64_t)s * P.npix));
  const uint4 w = philox4x32(make_uint4(p, s, 0u, kTagJitter), P.seed, 0u);
  float ox = u01(w.x), oy = u01(w.y);
  const float tmp = (float)p / P.cam.resx;
  oy = truncf(tmp) + oy;
  ox = (tmp - truncf(tmp)) * P.cam.resx + ox;
  const CamView& c = P.cam;
  const V3 d = mk(c.tl.x + ox * c.sx.x + oy * c.sy.x, c.tl.y + ox * c.sx.y + oy * c.sy.y,
                  c.tl.z + ox * c.sx.z + oy * c.sy.z);
  PathRec r;
  r.r0 = make_float4(c.eye.x, c.eye.y, c.eye.z, 1.f);
  r.r1 = make_float4(d.x, d.y, d.z, 1.f);
  r.r2 = make_float4(0.f, 0.f, 0.f, 1.f);
  r.r3 = make_float4(__uint_as_float(p), __uint_as_float(s), __uint_as_float(0u), 0.f);
  out[k] = r;
}

template <int KIND>
__global__ void __launch_bounds__(kPtBlock, 10) k_pt_bounce(GridView G, PtView P, PathRec* __restrict__ paths,
                                                        const uint32_t* d_n, uint32_t depth,
                                                        uint32_t* counter, uint32_t* __restrict__ alive,
                                                        float4* __restrict__ slots, uint64_t g0,
                                                        uint32_t* d_shadow) {
  const uint32_t n = *d_n;
  const int lane = threadIdx.x & 31;
  uint32_t shadow_rays = 0;
  while (true) {
    uint32_t b = 0;
    if (lane == 0) b = atomicAdd(counter, 32u);
    const uint32_t base = __shfl_sync(0xFFFFFFFFu, b, 0);
    if (base >= n) break;
    const uint32_t i = base + lane;
    if (i >= n) continue;
    PathRec r = paths[i];
    const V3 org = mk(r.r0.x, r.r0.y, r.r0.z);
    const V3 dir = mk(r.r1.x, r.r1.y, r.r1.z);
    V3 beta = mk(r.r0.w, r.r1.w, r.r2.w);
    V3 L = mk(r.r2.x, r.r2.y, r.r2.z);
    const uint32_t p = __float_as_uint(r.r3.x), s = __float_as_uint(r.r3.y);
    if (p >= P.npix || s >= P.spp) {  // record left unwritten by a look-back that gave up
      alive[i] = 0u;
      continue;
    }
    Hit h{FLT_MAX, kMiss, 0.f, 0.f};
    trace_ray<KIND, false>(G, org, dir, h);
    bool live = false;
    if (h.tri == kMiss) {
      L = add(L, mul(beta, P.bg));
    } else {
      const float4* rec = P.stri + 3 * (size_t)h.tri;
      const V3 v0 = f4v(__ldg(rec));
      const V3 v1 = f4v(__ldg(rec + 1));
      const V3 v2 = f4v(__ldg(rec + 2));
      const V3 e1 = sub(v1, v0);
      V3 nn = normalize(cross(e1, sub(v2, v0)));
      if (dot(nn, dir) > 0.f) nn = mk(-nn.x, -nn.y, -nn.z);
      const V3 hp = add(org, muls(dir, h.t));
      const V3 o = add(hp, muls(nn, P.offset));
      // next-event estimation
      const uint4 wl = philox4x32(make_uint4(p, s, depth, kTagLight), P.seed, 0u);
      const float lu = u01(wl.x), lv = u01(wl.y), urr = u01(wl.z);
      const V3 lp = add(add(P.lpos, muls(P.le1, lu)), muls(P.le2, lv));
      const V3 wv = sub(lp, o);
      const float d2 = dot(wv, wv);
      const V3 l = muls(wv, 1.0f / sqrtf(d2));
      const float cs = dot(nn, l);
      const float cl = -dot(P.lnrm, l);
      if (cs > 0.f && cl > 0.f) {
        Hit sh{0.9999f, kMiss, 0.f, 0.f};
        trace_ray<KIND, true>(G, o, wv, sh);
        ++shadow_rays;
        if (sh.tri == kMiss) {
          const float f = ((((P.albedo * 0.31830988618379067f) * cs) * cl) * P.larea) / d2;
          L = add(L, muls(mul(beta, P.lrad), f));
        }
      }
      // continuation
      live = depth + 1 < P.max_depth;
      if (live && depth >= P.rr_depth) {
        if (urr < P.albedo) beta = muls(beta, 1.0f / P.albedo);
        else live = false;
      }
      if (live) {
        const uint4 wd = philox4x32(make_uint4(p, s, depth, kTagDir), P.seed, 0u);
        const float u1 = u01(wd.x), u2 = u01(wd.y);
        float sn, cn;
        sincos_2pi(u1, sn, cn);
        const float rr = sqrtf(1.f - u2);
        const float lx = sn * rr, ly = cn * rr, lz = sqrtf(u2);
        const V3 tx = normalize(e1);
        const V3 ty = cross(nn, tx);
        const V3 nd = mk(tx.x * lx + ty.x * ly + nn.x * lz, tx.y * lx + ty.y * ly + nn.y * lz,
                         tx.z * lx + ty.z * ly + nn.z * lz);
        beta = muls(beta, P.albedo);
        r.r0 = make_float4(o.x, o.y, o.z, beta.x);
        r.r1 = make_float4(nd.x, nd.y, nd.z, beta.y);
        r.r2 = make_float4(L.x, L.y, L.z, beta.z);
        r.r3.z = __uint_as_float(depth + 1);
        paths[i] = r;
      }
    }
    alive[i] = live ? 1u : 0u;
    if (!live) slots[(uint64_t)s * P.npix + p - g0] = make_float4(L.x, L.y, L.z, 0.f);
  }
  if (d_shadow) {  // every lane leaves the loop at the same iteration
    const uint32_t c = __reduce_add_sync(0xFFFFFFFFu, shadow_rays);
    if (lane == 0 && c) atomicAdd(d_shadow, c);
  }
}

__global__ void __launch_bounds__(256) k_pt_compact(const PathRec* __restrict__ in,
                                                    const uint32_t* __restrict__ alive,
                                                    const uint32_t* d_n, PathRec* __restrict__ out,
                                                    uint32_t* d_next, LookbackState st) {
  __shared__ TileScanSmem<256, 8> sm;
  const uint32_t n = *d_n;
  // one tile per block; blocks beyond the live count only publish nothing
  if ((uint64_t)blockIdx.x * 2048 >= n) {
    if (blockIdx.x == 0 && threadIdx.x == 0) *d_next = 0;
    return;
  }
  tile_scan<256, 8>(
      st, n, sm, [&](uint32_t i) { return alive[i]; },
      [&](uint32_t i, uint32_t ex) {
        if (alive[i]) out[ex] = in[i];
      },
      d_next);
}

__global__ void k_pt_resolve(const float4* __restrict__ slots, uint32_t npix, uint32_t spp,
                             float* __restrict__ img) {
  const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= npix) return;
  float r = 0.f, g = 0.f, b = 0.f;
  for (uint32_t s = 0; s < spp; ++s) {
    const float4 v = slots[(uint64_t)s * npix + p];
    r += v.x;
    g += v.y;
    b += v.z;
  }
  img[3 * (size_t)p] = r / (float)spp;
  img[3 * (size_t)p + 1] = g / (float)spp;
  img[3 * (size_t)p + 2] = b / (float)spp;
}

__global__ void k_copy_u32(const uint32_t* src, uint32_t* dst) { *dst = *src; }
__global__ void k_add_u32(const uint32_t* src, uint32_t* dst) { *dst += *src; }

}  // namespace

}  // namespace shn

using namespace shn;

extern "C" {

void shn_pt_params_default(shn_pt_params* p) {
  if (!p) return;
  memset(p, 0, sizeof(*p));
  p->spp = 16;
  p->max_depth = 4;
  p->rr_depth = 2;
  p->albedo = 0.7f;
  const float pos[3] = {0.3f, 0.3f, 1.0f}, e1[3] = {0.f, 0.4f, 0.f}, e2[3] = {0.4f, 0.f, 0.f};
  const float rad[3] = {20.f, 20.f, 20.f}, bg[3] = {0.15f, 0.2f, 0.3f};
  memcpy(p->light_pos, pos, 12);
  memcpy(p->light_e1, e1, 12);
  memcpy(p->light_e2, e2, 12);
  memcpy(p->light_radiance, rad, 12);
  memcpy(p->background, bg, 12);
  p->offset = 1e-4f;
  p->seed = 2;
}

shn_status shn_pt_render(const shn_grid* g, const shn_scene* s, const shn_camera* cam,
                         const shn_pt_params* prm, float* d_image, uint32_t* d_stats, void* stream) {
  if (!g || !s || !cam || !prm || !d_image || prm->spp == 0 || prm->max_depth == 0) return SHN_ERR_INVALID;
  if (!g->built) return set_error(g->ctx, SHN_ERR_NOT_BUILT, "grid not built");
  grid_fence(g, (cudaStream_t)stream);
  if (!(prm->albedo > 0.f && prm->albedo <= 1.f)) return set_error(g->ctx, SHN_ERR_INVALID, "albedo must be in (0,1]");
  const uint64_t npix = (uint64_t)cam->res_x * cam->res_y;
  if (npix == 0) return SHN_OK;
  if (npix > (1u << 24)) return set_error(g->ctx, SHN_ERR_INVALID, "more than 2^24 pixels");
  const uint64_t total = npix * prm->spp;
  cudaStream_t st = (cudaStream_t)stream;
  shn_ctx* ctx = g->ctx;

  PtView P;
  P.cam = make_camera(cam);
  P.npix = (uint32_t)npix;
  P.spp = prm->spp;
  P.max_depth = prm->max_depth;
  P.rr_depth = prm->rr_depth;
  P.seed = prm->seed;
  P.albedo = prm->albedo;
  P.offset = prm->offset;
  P.lpos = mk(prm->light_pos[0], prm->light_pos[1], prm->light_pos[2]);
  P.le1 = mk(prm->light_e1[0], prm->light_e1[1], prm->light_e1[2]);
  P.le2 = mk(prm->light_e2[0], prm->light_e2[1], prm->light_e2[2]);
  P.lrad = mk(prm->light_radiance[0], prm->light_radiance[1], prm->light_radiance[2]);
  P.bg = mk(prm->background[0], prm->background[1], prm->background[2]);
  const V3 ln = cross(P.le1, P.le2);
  P.larea = sqrtf(dot(ln, ln));
  P.lnrm = normalize(ln);
  P.stri = s->tri;
  P.snt = s->nt;
  const GridView G = [&] {
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
  }();

  // Waves of at most kWave paths bound the state memory (2 x 64 B per path + slots).
  const uint64_t kWave = 1ull << 23;
  const uint32_t wave = (uint32_t)std::min<uint64_t>(total, kWave);
  const size_t tiles = (wave + 2047) / 2048;
  void *pa = nullptr, *pb = nullptr, *alive = nullptr, *slots = nullptr, *cnt = nullptr, *status = nullptr;
  const size_t bRec = (size_t)wave * sizeof(PathRec), bAl = (size_t)wave * 4, bSl = (size_t)total * 16,
               bCnt = 64 * 4, bSt = (tiles + 2) * 8;
  cudaError_t e = dev_alloc(ctx, &pa, bRec, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, &pb, bRec, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, &alive, bAl, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, &slots, bSl, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, &cnt, bCnt, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, &status, bSt, st);
  auto release = [&] {
    dev_free(ctx, pa, bRec, st);
    dev_free(ctx, pb, bRec, st);
    dev_free(ctx, alive, bAl, st);
    dev_free(ctx, slots, bSl, st);
    dev_free(ctx, cnt, bCnt, st);
    dev_free(ctx, status, bSt, st);
  };
  if (e != cudaSuccess) {
    release();
    return set_error(ctx, e == cudaErrorNotPermitted ? SHN_ERR_BUDGET : SHN_ERR_OOM, "path tracer state");
  }
  uint32_t* counters = (uint32_t*)cnt;  // [0..15] work counters, [16..31] live counts
  int blocks = 0;
  {
    static int b0 = [&] { int v = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_pt_bounce<0>, kPtBlock, 0); return v; }();
    static int b1 = [&] { int v = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&v, k_pt_bounce<1>, kPtBlock, 0); return v; }();
    blocks = std::max(1, g->kind == SHN_GRID_UNIFORM ? b0 : b1) * ctx->num_sms;
  }
  if (d_stats) cudaMemsetAsync(d_stats, 0, (prm->max_depth + 1) * 4, st);
  for (uint64_t g0 = 0; g0 < total; g0 += wave) {
    const uint32_t count = (uint32_t)std::min<uint64_t>(wave, total - g0);
    PathRec* cur = (PathRec*)pa;
    PathRec* nxt = (PathRec*)pb;
    uint32_t* d_n = counters + 16;
    k_pt_camera<<<(count + 255) / 256, 256, 0, st>>>(P, g0, count, cur, d_n);
    for (uint32_t d = 0; d < prm->max_depth; ++d) {
      cudaMemsetAsync(counters, 0, 4, st);
      if (d_stats) k_add_u32<<<1, 1, 0, st>>>(d_n, d_stats + d);
      uint32_t* d_shadow = d_stats ? d_stats + prm->max_depth : nullptr;
      float4* slot_base = (float4*)slots;
      if (g->kind == SHN_GRID_UNIFORM)
        k_pt_bounce<0><<<blocks, kPtBlock, 0, st>>>(G, P, cur, d_n, d, counters, (uint32_t*)alive, slot_base, 0,
                                                    d_shadow);
      else
        k_pt_bounce<1><<<blocks, kPtBlock, 0, st>>>(G, P, cur, d_n, d, counters, (uint32_t*)alive, slot_base, 0,
                                                    d_shadow);
      if (d + 1 < prm->max_depth) {
        cudaMemsetAsync(status, 0, bSt, st);
        LookbackState ls{(uint64_t*)status, (uint32_t*)((uint64_t*)status + tiles + 1), g->d_err};
        uint32_t* d_next = d_n + 1;
        k_pt_compact<<<(unsigned)tiles, 256, 0, st>>>(cur, (uint32_t*)alive, d_n, nxt, d_next, ls);
        k_copy_u32<<<1, 1, 0, st>>>(d_next, d_n);
        std::swap(cur, nxt);
      }
    }
  }
  k_pt_resolve<<<(unsigned)((npix + 255) / 256), 256, 0, st>>>((const float4*)slots, (uint32_t)npix,
                                                               prm->spp, d_image);
  release();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHN_OK : cuda_status(ctx, e, "pt_render");
}

}  // extern "C"
