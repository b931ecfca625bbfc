// SAH resolution search and the SAH cost of candidate grid resolutions.
//
// SAHGridBuilder::computeResolution (src/Control/Algorithm/SAHGridBuilder.h:117-202)
// tries every resolution between 0.75 and 1.25 times the lambda = 5 estimate
// on each axis and keeps the first one (z outer, then y, then x) of least
// cost
//   0.85 * refs * cellArea / sceneArea + 0.15 * (resX + resY + resZ),
// cellArea = 2 (cx^2 + cy^2 + cz^2) of the cell size and sceneArea the same
// of the scene box, where refs counts every triangle's bounding-box cells
// (countRefs, src/Control/Algorithm/FastBuildKernels.h:31-86).  The reference
// launches one counting kernel and reads it back per resolution; here one
// kernel counts a whole tile of resolutions per block: each staged triangle's
// per-axis cell spans for the tile's resolutions go to shared memory once and
// every thread sums span_x * span_y * span_z for a 2 x 2 x 2 block of
// resolutions.  The counts are exact 64-bit sums.  (The reference adds up its
// per-block partial counts over the block size, 256, instead of the number
// of blocks, 128, reading past its array (SAHGridBuilder.h:80-84), and
// counts in 32 bits; both are left out.)
#include <cmath>

#include "internal.h"

namespace shn {
namespace {

constexpr int kSahBlock = 256;
constexpr int kTX = 16, kTY = 16, kTZ = 8;  // resolutions per block tile; 2 x 2 x 2 per thread
constexpr int kSahChunk = 256;              // triangles staged per step (one per thread)
constexpr int kMaxCandidates = 32;

// Cells of [lo, hi] along one axis at resolution res (countRefs' arithmetic,
// src/Control/Algorithm/FastBuildKernels.h:53-69): 0 when the range is empty.
SHN_D uint32_t axis_span(float lo, float hi, float g0, float rcp, float rm1) {
  if (!(rm1 >= 0.f)) return 0u;
  const float mnf = fmaxf(0.f, (lo - g0) * rcp + -kEps);
  const float mxf = fminf(rm1, (hi - g0) * rcp + kEps);
  const uint32_t a = (uint32_t)mnf, b = (uint32_t)mxf;
  return b >= a ? b - a + 1u : 0u;
}

struct AxisTable {
  float rcp[kTX + kTY + kTZ];  // 1 / cellSize per resolution of the tile
  float rm1[kTX + kTY + kTZ];  // resolution - 1; -1 past the window (span 0)
};

__global__ void __launch_bounds__(kSahBlock) k_sah_counts(const float4* __restrict__ tri, uint32_t nt, V3 gmin,
                                                          V3 gmax, int3 rmin, int3 cnt, int3 tiles,
                                                          unsigned long long* counts) {
  __shared__ __align__(16) uint16_t s_x[kSahChunk][kTX];
  __shared__ __align__(16) uint16_t s_y[kSahChunk][kTY];
  __shared__ __align__(16) uint16_t s_z[kSahChunk][kTZ];
  __shared__ AxisTable tab;
  const int tile = blockIdx.x;
  const int tx = tile % tiles.x, ty = (tile / tiles.x) % tiles.y, tz = tile / (tiles.x * tiles.y);
  if (threadIdx.x < kTX + kTY + kTZ) {
    const int j = threadIdx.x;
    const int ax = j < kTX ? 0 : (j < kTX + kTY ? 1 : 2);
    const int i = ax == 0 ? tx * kTX + j : (ax == 1 ? ty * kTY + j - kTX : tz * kTZ + j - kTX - kTY);
    const int n = ax == 0 ? cnt.x : (ax == 1 ? cnt.y : cnt.z);
    const int r0 = ax == 0 ? rmin.x : (ax == 1 ? rmin.y : rmin.z);
    const float res = (float)(r0 + i);
    const float cs = (comp(gmax, ax) - comp(gmin, ax)) / res;  // cellSize, then its reciprocal
    tab.rcp[j] = 1.f / cs;
    tab.rm1[j] = i < n ? res - 1.f : -1.f;  // -1: every span 0
  }
  const int lx = threadIdx.x % 8, ly = (threadIdx.x / 8) % 8, lz = threadIdx.x / 64;
  unsigned long long acc[8] = {0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull, 0ull};
  for (uint32_t t0 = blockIdx.y * kSahChunk; t0 < nt; t0 += gridDim.y * kSahChunk) {
    __syncthreads();  // the table, or the previous chunk's readers
    {
      const uint32_t t = t0 + threadIdx.x;
      uint32_t px[kTX / 2], py[kTY / 2], pz[kTZ / 2];
      if (t < nt) {
        const float4* r = tri + 3 * (size_t)t;
        const V3 a = f4v(__ldg(r)), b = f4v(__ldg(r + 1)), c = f4v(__ldg(r + 2));
        const V3 bmin = vmin(vmin(a, b), c), bmax = vmax(vmax(a, b), c);
#pragma unroll
        for (int j = 0; j < kTX; j += 2)
          px[j / 2] = axis_span(bmin.x, bmax.x, gmin.x, tab.rcp[j], tab.rm1[j]) |
                      axis_span(bmin.x, bmax.x, gmin.x, tab.rcp[j + 1], tab.rm1[j + 1]) << 16;
#pragma unroll
        for (int j = 0; j < kTY; j += 2)
          py[j / 2] = axis_span(bmin.y, bmax.y, gmin.y, tab.rcp[kTX + j], tab.rm1[kTX + j]) |
                      axis_span(bmin.y, bmax.y, gmin.y, tab.rcp[kTX + j + 1], tab.rm1[kTX + j + 1]) << 16;
#pragma unroll
        for (int j = 0; j < kTZ; j += 2)
          pz[j / 2] = axis_span(bmin.z, bmax.z, gmin.z, tab.rcp[kTX + kTY + j], tab.rm1[kTX + kTY + j]) |
                      axis_span(bmin.z, bmax.z, gmin.z, tab.rcp[kTX + kTY + j + 1], tab.rm1[kTX + kTY + j + 1])
                          << 16;
      } else {
#pragma unroll
        for (int j = 0; j < kTX / 2; ++j) px[j] = 0u;
#pragma unroll
        for (int j = 0; j < kTY / 2; ++j) py[j] = 0u;
#pragma unroll
        for (int j = 0; j < kTZ / 2; ++j) pz[j] = 0u;
      }
      uint4* dx = reinterpret_cast<uint4*>(s_x[threadIdx.x]);
      uint4* dy = reinterpret_cast<uint4*>(s_y[threadIdx.x]);
      dx[0] = make_uint4(px[0], px[1], px[2], px[3]);
      dx[1] = make_uint4(px[4], px[5], px[6], px[7]);
      dy[0] = make_uint4(py[0], py[1], py[2], py[3]);
      dy[1] = make_uint4(py[4], py[5], py[6], py[7]);
      *reinterpret_cast<uint4*>(s_z[threadIdx.x]) = make_uint4(pz[0], pz[1], pz[2], pz[3]);
    }
    __syncthreads();
    const uint32_t kn = min((uint32_t)kSahChunk, nt - t0);
    for (uint32_t k = 0; k < kn; ++k) {
      const uint32_t wx = reinterpret_cast<const uint32_t*>(s_x[k])[lx];
      const uint32_t wy = reinterpret_cast<const uint32_t*>(s_y[k])[ly];
      const uint32_t wz = reinterpret_cast<const uint32_t*>(s_z[k])[lz];
      const uint32_t x0 = wx & 0xFFFFu, x1 = wx >> 16, y0 = wy & 0xFFFFu, y1 = wy >> 16;
      const uint32_t z0 = wz & 0xFFFFu, z1 = wz >> 16;
      const uint32_t p00 = x0 * y0, p10 = x1 * y0, p01 = x0 * y1, p11 = x1 * y1;  // <= 2^22
      acc[0] += (unsigned long long)p00 * z0;
      acc[1] += (unsigned long long)p10 * z0;
      acc[2] += (unsigned long long)p01 * z0;
      acc[3] += (unsigned long long)p11 * z0;
      acc[4] += (unsigned long long)p00 * z1;
      acc[5] += (unsigned long long)p10 * z1;
      acc[6] += (unsigned long long)p01 * z1;
      acc[7] += (unsigned long long)p11 * z1;
    }
  }
#pragma unroll
  for (int q = 0; q < 8; ++q) {
    const int ix = tx * kTX + 2 * lx + (q & 1), iy = ty * kTY + 2 * ly + ((q >> 1) & 1),
              iz = tz * kTZ + 2 * lz + (q >> 2);
    if (ix < cnt.x && iy < cnt.y && iz < cnt.z && acc[q])
      atomicAdd(counts + ((size_t)iz * cnt.y + iy) * cnt.x + ix, acc[q]);
  }
}

struct Candidates {
  int res[kMaxCandidates][3];
};

// refs of each of k explicit resolutions: grid-stride over the triangles,
// a warp sum per candidate, one atomic per warp and candidate.
__global__ void __launch_bounds__(256) k_sah_list(const float4* __restrict__ tri, uint32_t nt, V3 gmin, V3 gmax,
                                                  Candidates cand, int k, unsigned long long* counts) {
  __shared__ float s_rcp[kMaxCandidates][3], s_rm1[kMaxCandidates][3];
  if (threadIdx.x < 3 * k) {
    const int c = threadIdx.x / 3, ax = threadIdx.x % 3;
    const float res = (float)cand.res[c][ax];
    const float cs = (comp(gmax, ax) - comp(gmin, ax)) / res;
    s_rcp[c][ax] = 1.f / cs;
    s_rm1[c][ax] = res - 1.f;
  }
  __syncthreads();
  for (int c = 0; c < k; ++c) {
    unsigned long long sum = 0ull;
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
      const float4* r = tri + 3 * (size_t)t;
      const V3 a = f4v(__ldg(r)), b = f4v(__ldg(r + 1)), cc = f4v(__ldg(r + 2));
      const V3 bmin = vmin(vmin(a, b), cc), bmax = vmax(vmax(a, b), cc);
      const uint32_t sx = axis_span(bmin.x, bmax.x, gmin.x, s_rcp[c][0], s_rm1[c][0]);
      const uint32_t sy = axis_span(bmin.y, bmax.y, gmin.y, s_rcp[c][1], s_rm1[c][1]);
      const uint32_t sz = axis_span(bmin.z, bmax.z, gmin.z, s_rcp[c][2], s_rm1[c][2]);
      sum += (unsigned long long)(sx * sy) * sz;
    }
    for (int o = 16; o; o >>= 1) sum += __shfl_down_sync(0xFFFFFFFFu, sum, o);
    if ((threadIdx.x & 31) == 0 && sum) atomicAdd(counts + c, sum);
  }
}

// The reference's cost of one resolution (SAHGridBuilder.h:164-175), in
// its order of float operations.
float sah_cost(const float b[6], const int res[3], uint64_t refs) {
  const V3 bs = sub(mk(b[3], b[4], b[5]), mk(b[0], b[1], b[2]));
  const float scene_area = 2.f * (bs.x * bs.x + bs.y * bs.y + bs.z * bs.z);
  const V3 r = mk((float)res[0], (float)res[1], (float)res[2]);
  const V3 cs = divv(bs, r);
  const float cell_area = 2.f * (cs.x * cs.x + cs.y * cs.y + cs.z * cs.z);
  return 0.85f * (float)refs * cell_area / scene_area + 0.15f * (r.x + r.y + r.z);
}

int window_res(float v) {
  if (!(v == v) || v >= 2048.f) return 2048;
  return std::min(std::max((int)v, 1), 2048);
}

}  // namespace
}  // namespace shn

using namespace shn;

extern "C" shn_status shn_grid_sah_resolution(const shn_scene* s, float lambda, float window_lo, float window_hi,
                                              uint64_t* counts, uint64_t counts_capacity, shn_sah_result* out,
                                              void* stream) {
  if (!s || !out || !(lambda > 0.f) || !(window_lo > 0.f) || !(window_hi >= window_lo)) return SHN_ERR_INVALID;
  shn_ctx* ctx = s->ctx;
  const uint32_t nt = s->nt;
  if (nt == 0) return set_error(ctx, SHN_ERR_INVALID, "empty scene");
  cudaStream_t st = (cudaStream_t)stream;
  // GridBuilder::computeResolution's estimate, then the search window
  // (SAHGridBuilder.h:121-136), each bound clamped to [1, 2048]
  const V3 bmin = mk(s->bounds[0], s->bounds[1], s->bounds[2]), bmax = mk(s->bounds[3], s->bounds[4], s->bounds[5]);
  V3 diag = sub(bmax, bmin);
  const float volume = diag.x * diag.y * diag.z;
  const float magic = powf(lambda * (float)nt / volume, 0.3333333f);
  diag = muls(diag, magic);
  int rmin[3], rmax[3], n[3];
  for (int a = 0; a < 3; ++a) {
    const float d = comp(diag, a);
    rmin[a] = window_res(window_lo * d);
    rmax[a] = std::max(rmin[a], window_res(window_hi * d));
    n[a] = rmax[a] - rmin[a] + 1;
  }
  const uint64_t N = (uint64_t)n[0] * n[1] * n[2];
  if (N > (1ull << 24) || (double)N * nt > 2e13)
    return set_error(ctx, SHN_ERR_INVALID, "SAH search space too large for this scene: narrow the window");
  if (counts && counts_capacity < N) return set_error(ctx, SHN_ERR_INVALID, "counts array too small");
  const size_t cnt_bytes = N * 8;
  void* ws = nullptr;
  cudaError_t e = dev_alloc(ctx, &ws, cnt_bytes, st);
  if (e != cudaSuccess)
    return set_error(ctx, e == cudaErrorNotPermitted ? SHN_ERR_BUDGET : SHN_ERR_OOM, "SAH counts");
  unsigned long long* d_cnt = (unsigned long long*)ws;
  cudaMemsetAsync(d_cnt, 0, cnt_bytes, st);
  const int3 tiles = make_int3((n[0] + kTX - 1) / kTX, (n[1] + kTY - 1) / kTY, (n[2] + kTZ - 1) / kTZ);
  const uint32_t ntiles = (uint32_t)tiles.x * tiles.y * tiles.z;
  // about four blocks per SM over the tiles and the triangle splits
  const uint32_t chunks = (nt + kSahChunk - 1) / kSahChunk;
  const uint32_t splits = std::max(1u, std::min(chunks, (148u * 4u + ntiles - 1) / ntiles));
  k_sah_counts<<<dim3(ntiles, splits), kSahBlock, 0, st>>>(s->tri, nt, bmin, bmax,
                                                           make_int3(rmin[0], rmin[1], rmin[2]),
                                                           make_int3(n[0], n[1], n[2]), tiles, d_cnt);
  std::vector<uint64_t> h(N);
  cudaMemcpyAsync(h.data(), d_cnt, cnt_bytes, cudaMemcpyDeviceToHost, st);
  dev_free(ctx, ws, cnt_bytes, st);
  e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(ctx, e, "SAH search");
  // the reference's loop order: z, y, x; the first least cost wins
  float best = FLT_MAX;
  int bi[3] = {rmin[0], rmin[1], rmin[2]};
  uint64_t bref = 0;
  for (int z = 0; z < n[2]; ++z)
    for (int y = 0; y < n[1]; ++y)
      for (int x = 0; x < n[0]; ++x) {
        const int res[3] = {rmin[0] + x, rmin[1] + y, rmin[2] + z};
        const uint64_t refs = h[((size_t)z * n[1] + y) * n[0] + x];
        const float cost = sah_cost(s->bounds, res, refs);
        if (cost < best) {
          best = cost;
          bi[0] = res[0];
          bi[1] = res[1];
          bi[2] = res[2];
          bref = refs;
        }
      }
  for (int a = 0; a < 3; ++a) {
    out->res[a] = bi[a];
    out->res_min[a] = rmin[a];
    out->res_max[a] = rmax[a];
  }
  out->cost = best;
  out->refs = bref;
  out->num_tested = N;
  if (counts) memcpy(counts, h.data(), cnt_bytes);
  return SHN_OK;
}

namespace shn {

shn_status sah_refs_list(shn_ctx* ctx, const float4* tri, uint32_t nt, const float b[6], const int32_t* res,
                         uint32_t k, uint64_t* refs, float* cost, cudaStream_t st) {
  if (k == 0 || k > (uint32_t)kMaxCandidates) return set_error(ctx, SHN_ERR_INVALID, "1 to 32 resolutions");
  Candidates c{};
  for (uint32_t i = 0; i < k; ++i)
    for (int a = 0; a < 3; ++a) {
      if (res[3 * i + a] < 1 || res[3 * i + a] > 2048)
        return set_error(ctx, SHN_ERR_INVALID, "resolution outside [1, 2048]");
      c.res[i][a] = res[3 * i + a];
    }
  std::vector<uint64_t> h(k, 0ull);
  if (nt) {
    void* ws = nullptr;
    cudaError_t e = dev_alloc(ctx, &ws, 8 * (size_t)k, st);
    if (e != cudaSuccess)
      return set_error(ctx, e == cudaErrorNotPermitted ? SHN_ERR_BUDGET : SHN_ERR_OOM, "SAH counts");
    cudaMemsetAsync(ws, 0, 8 * (size_t)k, st);
    const V3 bmin = mk(b[0], b[1], b[2]), bmax = mk(b[3], b[4], b[5]);
    const unsigned blocks = std::min<unsigned>((nt + 255) / 256, 148u * 8u);
    k_sah_list<<<blocks, 256, 0, st>>>(tri, nt, bmin, bmax, c, (int)k, (unsigned long long*)ws);
    cudaMemcpyAsync(h.data(), ws, 8 * (size_t)k, cudaMemcpyDeviceToHost, st);
    dev_free(ctx, ws, 8 * (size_t)k, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_status(ctx, e, "SAH cost");
  }
  for (uint32_t i = 0; i < k; ++i) {
    if (refs) refs[i] = h[i];
    if (cost) cost[i] = sah_cost(b, res + 3 * i, h[i]);
  }
  return SHN_OK;
}

}  // namespace shn

extern "C" shn_status shn_grid_sah_cost(const shn_scene* s, const int32_t* res, uint32_t k, uint64_t* refs,
                                        float* cost, void* stream) {
  if (!s || !res || (!refs && !cost) || k == 0 || k > (uint32_t)kMaxCandidates) return SHN_ERR_INVALID;
  return sah_refs_list(s->ctx, s->tri, s->nt, s->bounds, res, k, refs, cost, (cudaStream_t)stream);
}
