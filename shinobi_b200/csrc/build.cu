// Sort-based uniform and two-level grid construction for sm_100a.
//
// Pipeline (uniform grid, and the top level of the two-level grid):
//   k_count_groups      exact per-triangle cell counts (bbox range + plane
//                       test, by row intervals: rows.cuh), warps pulling
//                       32 triangles at a time
//   k_scan_inplace      decoupled look-back exclusive scan of the counts ->
//                       per-triangle output offsets and the pair total
//   k_emit_units        packed (cell << 32 | tri) keys, triangle order
//   onesweep_sort       stable 8-bit-digit LSD sort on the cell bits
//   k_ranges            [begin,end) per cell, indices[] and the
//                       reference-ordered SoA float4 triangle copy
// Two-level leaf stage:
//   k_leaf_cells_scan   leaf resolution per top cell fused with the scan of
//                       leaf-cell counts -> TwoLevelGridCell words
//   k_count_groups + k_scan_inplace: exact leaf-cell counts per sorted top pair
//   k_emit_units        (leafId << 32 | tri) keys
//   onesweep_sort + k_ranges on the leaf keys.
//
// The cell arithmetic restates src/Control/Algorithm/FastBuildKernels.h:31-313
// and src/Control/Algorithm/TwoLevelBuildKernels.h:40-536 operation by
// operation (see the oracle for the list of canonicalisations); the library
// is compiled with -fmad=false so the results are bit-identical to it.
#include <cmath>

#include "internal.h"
#include "rows.cuh"

namespace shn {

namespace {

constexpr int kScanBlock = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanBlock * kScanItems;

// Scene triangles, one 48-byte record per triangle: v0 (w = triangle id
// bits), v1, v2.  A record spans at most two 32-byte sectors, so the gather
// of a triangle by id (reference-ordered copy, AO and path-tracer normals)
// touches 2 sectors instead of 3 for three separate arrays.
struct TriArr {
  const float4* p;
};

SHN_D void load_tri(const TriArr& t, uint32_t i, V3& a, V3& b, V3& c) {
  const float4* r = t.p + 3 * (size_t)i;
  a = f4v(__ldg(r));
  b = f4v(__ldg(r + 1));
  c = f4v(__ldg(r + 2));
}

SHN_D void tri_bounds(V3 a, V3 b, V3 c, V3& bmin, V3& bmax) {
  bmin = mk(FLT_MAX, FLT_MAX, FLT_MAX);
  bmax = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  bmin = vmin(bmin, a); bmax = vmax(bmax, a);
  bmin = vmin(bmin, b); bmax = vmax(bmax, b);
  bmin = vmin(bmin, c); bmax = vmax(bmax, c);
}

// countRefs / buildUnsortedGrid cell range (FastBuildKernels.h:47-69, 110-133).
SHN_D void cell_range(V3 a, V3 b, V3 c, const Geom& g, uint32_t lo[3], uint32_t hi[3]) {
  V3 bmin, bmax;
  tri_bounds(a, b, c, bmin, bmax);
  const V3 minf = vmax(mk(0.f, 0.f, 0.f), add(mul(sub(bmin, g.gmin), g.rcpBuild), mk(-kEps, -kEps, -kEps)));
  const V3 maxf = vmin(sub(g.resf, mk(1.f, 1.f, 1.f)), add(mul(sub(bmax, g.gmin), g.rcpBuild), mk(kEps, kEps, kEps)));
  lo[0] = (uint32_t)minf.x; lo[1] = (uint32_t)minf.y; lo[2] = (uint32_t)minf.z;
  hi[0] = (uint32_t)maxf.x; hi[1] = (uint32_t)maxf.y; hi[2] = (uint32_t)maxf.z;
}

// Pair-generation unit of a triangle against the top grid: candidate box
// from countRefs (FastBuildKernels.h:47-69), plane test when the box spans
// two or more cells on every axis (FastBuildKernels.h:137-212).
SHN_D void top_unit(V3 a, V3 b, V3 c, const Geom& g, uint32_t id, uint32_t base, Unit& U) {
  uint32_t lo[3], hi[3];
  cell_range(a, b, c, g, lo, hi);
  const bool plane = hi[0] - lo[0] > 0 && hi[1] - lo[1] > 0 && hi[2] - lo[2] > 0;
  V3 n = mk(0.f, 0.f, 0.f);
  if (plane) n = normalize(cross(sub(b, a), sub(c, a)));
  U.a[0] = a.x; U.a[1] = a.y; U.a[2] = a.z;
  U.n[0] = n.x; U.n[1] = n.y; U.n[2] = n.z;
  U.s[0] = g.cs.x; U.s[1] = g.cs.y; U.s[2] = g.cs.z;
  U.o[0] = g.gmin.x; U.o[1] = g.gmin.y; U.o[2] = g.gmin.z;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    U.lo[k] = lo[k];
    U.span[k] = hi[k] - lo[k] + 1u;
  }
  U.id = id;
  U.base = base;
  U.stride[0] = (uint32_t)g.resf.x;
  U.stride[1] = (uint32_t)(g.resf.x * g.resf.y);
  unit_finish(U, plane);
}

// Leaf resolution: largest r with r^3 <= cs_a^3 * lambda * refs / V, clamped
// to [1, 255] (see the header comment of the oracle for the reasoning).
SHN_D uint32_t cube_floor(double q) {
  if (!(q > 0.0)) return 0u;
  if (__dmul_rn(__dmul_rn(256.0, 256.0), 256.0) <= q) return 256u;
  uint32_t lo = 0, hi = 256;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    const double m = (double)mid;
    if (__dmul_rn(__dmul_rn(m, m), m) <= q) lo = mid; else hi = mid;
  }
  return lo;
}

SHN_D uint32_t leaf_word(const Geom& g, float lambda, uint32_t refs, uint32_t threshold,
                         uint32_t* count) {
  uint32_t r[3] = {1u, 1u, 1u};
  if (refs > threshold) {
    const double vol = __dmul_rn(__dmul_rn((double)g.cs.x, (double)g.cs.y), (double)g.cs.z);
    const double lr = __dmul_rn((double)lambda, (double)refs);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
      const double c = (double)comp(g.cs, a);
      const double q = __ddiv_rn(__dmul_rn(__dmul_rn(__dmul_rn(c, c), c), lr), vol);
      r[a] = min(255u, max(1u, cube_floor(q)));
    }
  }
  *count = r[0] * r[1] * r[2];
  uint32_t y = (r[0] & 0xFFu) | ((r[1] & 0xFFu) << 8) | ((r[2] & 0xFFu) << 16);
  if (refs > 0) y |= kNotEmpty;
  return y;
}

// Pair-generation unit of a (top cell, triangle) pair against the cell's leaf
// grid (countLeafLevelRefs / writeLeafLevelRefs, TwoLevelBuildKernels.h:175-222,
// 327-451): candidate box [lo, hp) clamped to the leaf resolution, plane test
// when it spans two or more leaf cells on every axis.
SHN_D void leaf_unit(V3 a, V3 b, V3 c, const Geom& g, uint32_t topCell, uint32_t cellY,
                     uint32_t leafBegin, uint32_t id, Unit& U) {
  const uint32_t rX = (uint32_t)g.res[0], rY = (uint32_t)g.res[1];
  const uint32_t tx = topCell % rX;
  const uint32_t ty = (topCell % (rX * rY)) / rX;
  const uint32_t tz = topCell / (rX * rY);
  V3 bmin, bmax;
  tri_bounds(a, b, c, bmin, bmax);
  const V3 cres = mk((float)(cellY & 0xFFu), (float)((cellY >> 8) & 0xFFu), (float)((cellY >> 16) & 0xFFu));
  V3 origin;
  origin.x = (float)tx * g.cs.x + g.gmin.x;
  origin.y = (float)ty * g.cs.y + g.gmin.y;
  origin.z = (float)tz * g.cs.z + g.gmin.z;
  const V3 subRCP = divv(cres, g.cs);
  const V3 minf = add(mul(sub(bmin, origin), subRCP), mk(-0.001f, -0.001f, -0.001f));
  const V3 maxf = add(mul(sub(bmax, origin), subRCP), mk(1.001f, 1.001f, 1.001f));
  int lo[3], hp[3];
  lo[0] = max(0, (int)minf.x); lo[1] = max(0, (int)minf.y); lo[2] = max(0, (int)minf.z);
  hp[0] = min((int)cres.x, (int)maxf.x);
  hp[1] = min((int)cres.y, (int)maxf.y);
  hp[2] = min((int)cres.z, (int)maxf.z);
  const bool plane = hp[0] - lo[0] > 1 && hp[1] - lo[1] > 1 && hp[2] - lo[2] > 1;
  V3 n = mk(0.f, 0.f, 0.f);
  if (plane) n = normalize(cross(sub(b, a), sub(c, a)));
  const V3 scs = divv(g.cs, cres);
  U.a[0] = a.x; U.a[1] = a.y; U.a[2] = a.z;
  U.n[0] = n.x; U.n[1] = n.y; U.n[2] = n.z;
  U.s[0] = scs.x; U.s[1] = scs.y; U.s[2] = scs.z;
  U.o[0] = origin.x; U.o[1] = origin.y; U.o[2] = origin.z;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    U.lo[k] = (uint32_t)lo[k];
    U.span[k] = hp[k] > lo[k] ? (uint32_t)(hp[k] - lo[k]) : 0u;
  }
  U.id = id;
  U.base = leafBegin;
  U.stride[0] = (uint32_t)cres.x;
  U.stride[1] = (uint32_t)(cres.x * cres.y);
  unit_finish(U, plane);
}

// ---- unit makers: item index -> unit ------------------------------------------------
struct TopMaker {
  TriArr tri;
  Geom g;
  SHN_D bool operator()(uint32_t t, Unit& U) const {
    V3 a, b, c;
    load_tri(tri, t, a, b, c);
    top_unit(a, b, c, g, t, 0u, U);
    return true;
  }
};

struct LeafMaker {
  TriArr tri;
  const uint64_t* top;  // sorted (top cell << 32 | tri)
  const uint2* cells;   // top cell words
  Geom g;
  SHN_D bool operator()(uint32_t i, Unit& U) const {
    const uint64_t k = top[i];
    const uint32_t c = (uint32_t)(k >> 32), t = (uint32_t)k;
    V3 a, b, cc;
    load_tri(tri, t, a, b, cc);
    const uint2 w = cells[c];
    leaf_unit(a, b, cc, g, c, w.y, w.x, t, U);
    return true;
  }
};

// ---- generic count (fused with the offsets scan) and emit kernels --------------------
constexpr int kUnitWarps = kScanBlock / 32;

// Exact pair count of every item into counts[i].  Warps take 32 items at a
// time from a global counter: no block-wide barrier, so warps whose items
// span many rows do not hold up the others (the tile-fused form above spent
// most of its time waiting at the tile barrier).
template <class Maker>
__global__ void __launch_bounds__(kScanBlock) k_count_groups(Maker mk, uint32_t n, uint32_t* __restrict__ counts,
                                                            uint32_t* group_counter) {
  __shared__ Unit su[kUnitWarps][32];
  __shared__ uint32_t acc[kUnitWarps][32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t groups = (n + 31u) / 32u;
  while (true) {
    uint32_t gidx = 0;
    if (lane == 0) gidx = atomicAdd(group_counter, 1u);
    gidx = __shfl_sync(0xFFFFFFFFu, gidx, 0);
    if (gidx >= groups) break;
    const uint32_t i = gidx * 32u + lane;
    const bool valid = i < n && mk(i, su[warp][lane]);
    __syncwarp();
    const uint32_t c = warp_count_units(su[warp], acc[warp], valid);
    if (i < n) counts[i] = c;
    __syncwarp();
  }
}

// In-place exclusive scan: data[0..n) -> prefixes, data[n] = total.  Each
// tile reads all of its items before it writes any.
__global__ void __launch_bounds__(kScanBlock) k_scan_inplace(uint32_t* data, uint32_t n, LookbackState st) {
  __shared__ TileScanSmem<kScanBlock, kScanItems> sm;
  tile_scan<kScanBlock, kScanItems>(
      st, n, sm, [&](uint32_t i) { return data[i]; }, [&](uint32_t i, uint32_t ex) { data[i] = ex; }, data + n);
}

// Keys of every item at offs[item]: 32 items per warp step, coalesced stores.
// hist (optional): the sort's digit counts ([pass][512]) of the keys' cell
// bits under the sort plan hp, counted here so that the sort needs no
// histogram pass over the keys.
template <class Maker>
__global__ void __launch_bounds__(kScanBlock) k_emit_units(Maker mk, uint32_t n,
                                                          const uint32_t* __restrict__ offs,
                                                          uint64_t* __restrict__ keys, uint32_t cap,
                                                          uint32_t* err, uint32_t* hist, SortPlan hp) {
  __shared__ Unit su[kUnitWarps][32];
  __shared__ uint32_t shist[4 * 512];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (hist) {
    for (int i = threadIdx.x; i < 4 * 512; i += kScanBlock) shist[i] = 0u;
    __syncthreads();
  }
  const uint32_t groups = (n + 31u) / 32u;
  for (uint32_t gi = blockIdx.x * kUnitWarps + warp; gi < groups; gi += gridDim.x * kUnitWarps) {
    const uint32_t i = gi * 32u + lane;
    const bool valid = i < n && mk(i, su[warp][lane]);
    const uint32_t out = offs[gi * 32u];
    __syncwarp();
    warp_emit_units(su[warp], valid, out, keys, cap, err, hist ? shist : nullptr, hist ? hp.passes : 0u, hp.width);
    __syncwarp();
  }
  if (hist) {
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < hp.passes * 512; i += kScanBlock)
      if (shist[i]) atomicAdd(hist + i, shist[i]);
  }
}

// ---- precise (SAT) insertion --------------------------------------------------------
// The reference's other uniform-grid builder keeps a candidate cell only if
// the plane test AND the nine edge-cross-axis tests of the triangle/box
// separating-axis test pass (GridOperator with taPreciseInsertion,
// src/Control/Algorithm/BuildKernels.h:41-201); cell centres are accumulated
// as in the plane-test path.  One thread walks one triangle's candidates
// (this insertion is a build option, not the hot path).
SHN_D bool sat_axis(float a, float b, float fa, float fb, float v0a, float v0b, float v1a, float v1b, float ha,
                    float hb) {
  const float p0 = a * v0a + b * v0b;
  const float p1 = a * v1a + b * v1b;
  const float mn = fminf(p0, p1);
  const float mx = fmaxf(p0, p1);
  const float rad = fa * ha + fb * hb;
  return !(mn > rad + kEps || mx + kEps < -rad);
}

SHN_D bool sat_edges(V3 t0, V3 t1, V3 t2, V3 c, V3 h) {
  const V3 v0 = sub(t0, c), v1 = sub(t1, c), v2 = sub(t2, c);
  const V3 e[3] = {sub(v1, v0), sub(v2, v1), sub(v0, v2)};
  bool ok = true;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const V3 ed = e[k];
    const V3 fe = mk(fabsf(ed.x), fabsf(ed.y), fabsf(ed.z));
    ok = ok && (k < 2 ? sat_axis(ed.z, -ed.y, fe.z, fe.y, v0.y, v0.z, v2.y, v2.z, h.y, h.z)
                      : sat_axis(ed.z, -ed.y, fe.z, fe.y, v0.y, v0.z, v1.y, v1.z, h.y, h.z));
    ok = ok && (k < 2 ? sat_axis(-ed.z, ed.x, fe.z, fe.x, v0.x, v0.z, v2.x, v2.z, h.x, h.z)
                      : sat_axis(-ed.z, ed.x, fe.z, fe.x, v0.x, v0.z, v1.x, v1.z, h.x, h.z));
    ok = ok && (k == 1 ? sat_axis(ed.y, -ed.x, fe.y, fe.x, v0.x, v0.y, v1.x, v1.y, h.x, h.y)
                       : sat_axis(ed.y, -ed.x, fe.y, fe.x, v1.x, v1.y, v2.x, v2.y, h.x, h.y));
  }
  return ok;
}

// Cells of triangle t in (z, y, x) order; emit(cell) for each kept one.
template <class F>
SHN_D void sat_cells(const TriArr& tri, const Geom& g, uint32_t t, F&& emit) {
  V3 a, b, c;
  load_tri(tri, t, a, b, c);
  uint32_t lo[3], hi[3];
  cell_range(a, b, c, g, lo, hi);
  const uint32_t rx = (uint32_t)g.resf.x, rxy = (uint32_t)(g.resf.x * g.resf.y);
  if (!(hi[0] - lo[0] > 0 && hi[1] - lo[1] > 0 && hi[2] - lo[2] > 0)) {
    for (uint32_t z = lo[2]; z <= hi[2]; ++z)
      for (uint32_t y = lo[1]; y <= hi[1]; ++y)
        for (uint32_t x = lo[0]; x <= hi[0]; ++x) emit(x + y * rx + z * rxy);
    return;
  }
  const V3 n = normalize(cross(sub(b, a), sub(c, a)));
  const V3 h = muls(g.cs, 0.5f);
  float cz = (((float)lo[2] * g.cs.z + g.gmin.z) + h.z) - g.cs.z;
  for (uint32_t z = lo[2]; z <= hi[2]; ++z) {
    cz += g.cs.z;
    float cy = (((float)lo[1] * g.cs.y + g.gmin.y) + h.y) - g.cs.y;
    for (uint32_t y = lo[1]; y <= hi[1]; ++y) {
      cy += g.cs.y;
      float cx = (((float)lo[0] * g.cs.x + g.gmin.x) + h.x) - g.cs.x;
      for (uint32_t x = lo[0]; x <= hi[0]; ++x) {
        cx += g.cs.x;
        const V3 cc = mk(cx, cy, cz);
        const float d = dot(sub(cc, a), n);
        const V3 dist = muls(n, d);
        if (sat_edges(a, b, c, cc, h) && fabsf(dist.x) <= h.x + kEps && fabsf(dist.y) <= h.y + kEps &&
            fabsf(dist.z) <= h.z + kEps)
          emit(x + y * rx + z * rxy);
      }
    }
  }
}

__global__ void k_count_sat(TriArr tri, uint32_t n, Geom g, uint32_t* __restrict__ counts) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint32_t k = 0;
    sat_cells(tri, g, t, [&](uint32_t) { ++k; });
    counts[t] = k;
  }
}

__global__ void __launch_bounds__(kScanBlock) k_emit_sat(TriArr tri, uint32_t n, Geom g,
                                                        const uint32_t* __restrict__ offs,
                                                        uint64_t* __restrict__ keys, uint32_t cap, uint32_t* err,
                                                        uint32_t* hist, SortPlan hp) {
  __shared__ uint32_t shist[4 * 512];
  for (int i = threadIdx.x; i < 4 * 512; i += kScanBlock) shist[i] = 0u;
  __syncthreads();
  const uint32_t hmask = (1u << hp.width) - 1u;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    uint32_t o = offs[t];
    sat_cells(tri, g, t, [&](uint32_t cell) {
      if (o < cap) keys[o] = ((uint64_t)cell << 32) | t;
      else atomicOr(err, kErrCapacity);
      ++o;
      for (uint32_t p = 0; p < hp.passes; ++p) atomicAdd(shist + p * 512 + ((cell >> (hp.width * p)) & hmask), 1u);
    });
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < hp.passes * 512; i += kScanBlock)
    if (shist[i]) atomicAdd(hist + i, shist[i]);
}

// ---------------------------------------------------------------------------
__global__ void k_pack_triangles(const float* __restrict__ vtx, const uint32_t* __restrict__ idx,
                                 uint32_t nt, float4* __restrict__ tri) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < nt; t += gridDim.x * blockDim.x) {
    const uint32_t i0 = idx[3 * (size_t)t], i1 = idx[3 * (size_t)t + 1], i2 = idx[3 * (size_t)t + 2];
    const float* a = vtx + 3 * (size_t)i0;
    const float* b = vtx + 3 * (size_t)i1;
    const float* c = vtx + 3 * (size_t)i2;
    float4* r = tri + 3 * (size_t)t;
    r[0] = make_float4(a[0], a[1], a[2], __uint_as_float(t));
    r[1] = make_float4(b[0], b[1], b[2], 0.f);
    r[2] = make_float4(c[0], c[1], c[2], 0.f);
  }
}

// Order-preserving float <-> uint mapping for atomic min/max of bounds.
SHN_D uint32_t fkey(float f) {
  const uint32_t u = __float_as_uint(f);
  return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
SHN_HD float fval(uint32_t k) {
  const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
  float f;
  memcpy(&f, &u, 4);
  return f;
}

__global__ void k_bounds(const float4* __restrict__ tri, uint32_t nt, uint32_t* out6) {
  V3 mn = mk(FLT_MAX, FLT_MAX, FLT_MAX), mx = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < 3ull * nt;
       i += (uint64_t)gridDim.x * blockDim.x) {
    const V3 p = f4v(tri[i]);
    mn = vmin(mn, p);
    mx = vmax(mx, p);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    mn.x = fminf(mn.x, __shfl_xor_sync(0xFFFFFFFFu, mn.x, o));
    mn.y = fminf(mn.y, __shfl_xor_sync(0xFFFFFFFFu, mn.y, o));
    mn.z = fminf(mn.z, __shfl_xor_sync(0xFFFFFFFFu, mn.z, o));
    mx.x = fmaxf(mx.x, __shfl_xor_sync(0xFFFFFFFFu, mx.x, o));
    mx.y = fmaxf(mx.y, __shfl_xor_sync(0xFFFFFFFFu, mx.y, o));
    mx.z = fmaxf(mx.z, __shfl_xor_sync(0xFFFFFFFFu, mx.z, o));
  }
  if ((threadIdx.x & 31) == 0) {
    atomicMin(out6 + 0, fkey(mn.x)); atomicMin(out6 + 1, fkey(mn.y)); atomicMin(out6 + 2, fkey(mn.z));
    atomicMax(out6 + 3, fkey(mx.x)); atomicMax(out6 + 4, fkey(mx.y)); atomicMax(out6 + 5, fkey(mx.z));
  }
}

__global__ void k_bounds_decode(uint32_t* io6) {
  if (threadIdx.x < 6) {
    const float f = fval(io6[threadIdx.x]);
    io6[threadIdx.x] = __float_as_uint(f);
  }
}

// Cell ranges from sorted keys (prepareCellRanges, FastBuildKernels.h:243-311)
// plus indices[] and the reference-ordered triangle copy.  Every thread
// handles kRangeItems keys per step (block-strided, so each load and store
// instruction is coalesced) to keep several gathers in flight; cell
// boundaries are found with warp shuffles of the neighbouring keys.
constexpr int kRangeItems = 1;
constexpr int kRangeBlock = 256;

__global__ void __launch_bounds__(kRangeBlock) k_ranges(const uint64_t* __restrict__ keys, uint32_t n,
                                                        uint2* __restrict__ ranges,
                                                        uint32_t* __restrict__ indices, TriArr tri,
                                                        float4* __restrict__ rtri) {
  const int lane = threadIdx.x & 31;
  constexpr uint32_t kStep = kRangeBlock * kRangeItems;
  for (uint64_t b0 = (uint64_t)blockIdx.x * kStep; b0 < n; b0 += (uint64_t)gridDim.x * kStep) {
    uint32_t c[kRangeItems], t[kRangeItems];
#pragma unroll
    for (int q = 0; q < kRangeItems; ++q) {
      const uint64_t i = b0 + q * kRangeBlock + threadIdx.x;
      const uint64_t k = i < n ? __ldcs(keys + i) : ~0ull;
      c[q] = (uint32_t)(k >> 32);
      t[q] = (uint32_t)k;
    }
    float4 a[kRangeItems], b[kRangeItems], d[kRangeItems];
    if (rtri) {
#pragma unroll
      for (int q = 0; q < kRangeItems; ++q) {
        const uint64_t i = b0 + q * kRangeBlock + threadIdx.x;
        if (i < n) {
          const float4* r = tri.p + 3 * (size_t)t[q];
          a[q] = __ldg(r);
          b[q] = __ldg(r + 1);
          d[q] = __ldg(r + 2);
        }
      }
    }
#pragma unroll
    for (int q = 0; q < kRangeItems; ++q) {
      const uint64_t i = b0 + q * kRangeBlock + threadIdx.x;
      uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, c[q], 1);
      uint32_t next = __shfl_down_sync(0xFFFFFFFFu, c[q], 1);
      if (i < n) {
        if (lane == 0) prev = i > 0 ? (uint32_t)(keys[i - 1] >> 32) : ~c[q];
        if (lane == 31) next = i + 1 < n ? (uint32_t)(keys[i + 1] >> 32) : ~c[q];
        if (i + 1 == n) next = ~c[q];
        if (i == 0) prev = ~c[q];
        if (prev != c[q]) ranges[c[q]].x = (uint32_t)i;
        if (next != c[q]) ranges[c[q]].y = (uint32_t)i + 1;
        // streaming (evict-first) stores: the output must not push the
        // triangles being gathered out of L2
        // the record's id: the triangle id whether or not the build ran on a
        // reordered copy of the triangles
        if (indices) __stcs(indices + i, rtri ? __float_as_uint(a[q].w) : t[q]);
        if (rtri) {
          __stcs(rtri + i, a[q]);
          __stcs(rtri + (size_t)n + i, b[q]);
          __stcs(rtri + 2 * (size_t)n + i, d[q]);
        }
      }
    }
  }
}

// Cell ranges by tiles of cells (grids whose range pass writes no triangle
// copy): block b owns cells [c0, c0 + kCellTile) and their keys [k0, k1)
// (two binary searches over the sorted keys).  Run starts and ends go to
// shared memory, then the tile's ranges are written as whole 8-byte words in
// cell order -- coalesced, every cell written once (empty ones as (0, 0)),
// so the cell array needs no clearing and no sector of it is written in
// part -- together with indices[] for its keys.
constexpr uint32_t kCellTile = 2048;

__global__ void __launch_bounds__(kRangeBlock) k_cell_ranges(const uint64_t* __restrict__ keys, uint32_t n,
                                                             uint64_t C, uint2* __restrict__ ranges,
                                                             uint32_t* __restrict__ indices) {
  __shared__ uint32_t s_b[kCellTile], s_e[kCellTile];
  __shared__ uint32_t s_k[2];
  const int lane = threadIdx.x & 31;
  for (uint64_t c0 = (uint64_t)blockIdx.x * kCellTile; c0 < C; c0 += (uint64_t)gridDim.x * kCellTile) {
    const uint64_t c1 = c0 + kCellTile < C ? c0 + kCellTile : C;
    for (uint32_t i = threadIdx.x; i < kCellTile; i += kRangeBlock) {
      s_b[i] = 0u;
      s_e[i] = 0u;
    }
    if (threadIdx.x < 2) {
      const uint64_t target = threadIdx.x == 0 ? c0 : c1;
      uint32_t lo = 0, hi = n;  // first key whose cell >= target
      while (lo < hi) {
        const uint32_t mid = lo + (hi - lo) / 2;
        if ((__ldg(keys + mid) >> 32) < target) lo = mid + 1;
        else hi = mid;
      }
      s_k[threadIdx.x] = lo;
    }
    __syncthreads();
    const uint32_t k0 = s_k[0], k1 = s_k[1];
    // whole warps step through [k0, k1) so that neighbours come by shuffles
    for (uint32_t w0 = k0 + (threadIdx.x & ~31u); w0 < k1; w0 += kRangeBlock) {
      const uint32_t i = w0 + lane;
      const bool in = i < k1;
      const uint64_t k = in ? __ldcs(keys + i) : 0ull;
      const uint32_t c = (uint32_t)(k >> 32);
      uint32_t prev = __shfl_up_sync(0xFFFFFFFFu, c, 1);
      uint32_t next = __shfl_down_sync(0xFFFFFFFFu, c, 1);
      if (in) {
        if (lane == 0) prev = i > k0 ? (uint32_t)(__ldg(keys + i - 1) >> 32) : ~c;
        if (lane == 31 || i + 1 == k1) next = i + 1 < k1 ? (uint32_t)(__ldg(keys + i + 1) >> 32) : ~c;
        if (prev != c) s_b[c - (uint32_t)c0] = i;
        if (next != c) s_e[c - (uint32_t)c0] = i + 1;
        __stcs(indices + i, (uint32_t)k);
      }
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < (uint32_t)(c1 - c0); j += kRangeBlock)
      __stcs(reinterpret_cast<uint2*>(ranges) + c0 + j, make_uint2(s_b[j], s_e[j]));
    __syncthreads();
  }
}

// ---- spatial order and block boxes (two-level grids) -------------------------
// The build of a two-level grid runs on a copy of the triangles sorted by the
// Morton code of their vertex sum in the scene box (20 bits per axis), so that
// the references inside each leaf cell come out in spatial order; the cells,
// their ranges and the set of references in each are the same as in triangle
// order.  The 60-bit code is sorted as two stable 30-bit passes of the key
// sort (low half first), each key carrying the triangle's position.
SHN_HD uint32_t spread10(uint32_t v) {
  v &= 0x3FFu;
  v = (v | (v << 16)) & 0x030000FFu;
  v = (v | (v << 8)) & 0x0300F00Fu;
  v = (v | (v << 4)) & 0x030C30C3u;
  v = (v | (v << 2)) & 0x09249249u;
  return v;
}

SHN_D uint32_t quant20(float q) { return q > 0.f ? (uint32_t)fminf(q, 1048575.f) : 0u; }

__global__ void k_morton_keys(TriArr tri, uint32_t n, V3 lo3, V3 scale, uint32_t tb, uint64_t* __restrict__ keys,
                              uint32_t* __restrict__ hi) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const float4* r = tri.p + 3 * (size_t)i;
    const V3 a = f4v(__ldg(r)), b = f4v(__ldg(r + 1)), c = f4v(__ldg(r + 2));
    const V3 q = mul(sub(add(add(a, b), c), lo3), scale);
    const uint32_t x = quant20(q.x), y = quant20(q.y), z = quant20(q.z);
    const uint32_t mlo = spread10(x) | (spread10(y) << 1) | (spread10(z) << 2);
    const uint32_t mhi = spread10(x >> 10) | (spread10(y >> 10) << 1) | (spread10(z >> 10) << 2);
    keys[i] = ((uint64_t)mlo << tb) | i;
    hi[i] = mhi;
  }
}

__global__ void k_morton_second(const uint64_t* __restrict__ sorted, const uint32_t* __restrict__ hi, uint32_t n,
                                uint32_t tb, uint64_t* __restrict__ keys) {
  const uint64_t mask = (1ull << tb) - 1ull;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(sorted[j] & mask);
    keys[j] = ((uint64_t)__ldg(hi + i) << tb) | i;
  }
}

__global__ void k_permute_tris(const uint64_t* __restrict__ sorted, TriArr tri, uint32_t n, uint32_t tb,
                               float4* __restrict__ out) {
  const uint64_t mask = (1ull << tb) - 1ull;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n; j += gridDim.x * blockDim.x) {
    const uint32_t i = (uint32_t)(sorted[j] & mask);
    const float4* r = tri.p + 3 * (size_t)i;
    float4* o = out + 3 * (size_t)j;
    o[0] = __ldg(r);
    o[1] = __ldg(r + 1);
    o[2] = __ldg(r + 2);
  }
}

// Box (min, max) of the three vertices of references [32k, 32k + 32) of the
// reference-ordered arrays, one warp per block; then boxes of 32 blocks.
__global__ void k_block_boxes(const float4* __restrict__ v0, const float4* __restrict__ v1,
                              const float4* __restrict__ v2, uint32_t n, uint32_t nblocks,
                              float4* __restrict__ box) {
  const int lane = threadIdx.x & 31;
  const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t k = w0; k < nblocks; k += nw) {
    const uint32_t i = 32u * k + lane;
    V3 mn = mk(INFINITY, INFINITY, INFINITY), mx = mk(-INFINITY, -INFINITY, -INFINITY);
    if (i < n) {
      const V3 a = f4v(__ldg(v0 + i)), b = f4v(__ldg(v1 + i)), c = f4v(__ldg(v2 + i));
      mn = vmin(vmin(a, b), c);
      mx = vmax(vmax(a, b), c);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn = vmin(mn, mk(__shfl_xor_sync(0xFFFFFFFFu, mn.x, o), __shfl_xor_sync(0xFFFFFFFFu, mn.y, o),
                       __shfl_xor_sync(0xFFFFFFFFu, mn.z, o)));
      mx = vmax(mx, mk(__shfl_xor_sync(0xFFFFFFFFu, mx.x, o), __shfl_xor_sync(0xFFFFFFFFu, mx.y, o),
                       __shfl_xor_sync(0xFFFFFFFFu, mx.z, o)));
    }
    if (lane == 0) {
      box[2 * (size_t)k] = make_float4(mn.x, mn.y, mn.z, 0.f);
      box[2 * (size_t)k + 1] = make_float4(mx.x, mx.y, mx.z, 0.f);
    }
  }
}

__global__ void k_super_boxes(const float4* __restrict__ box, uint32_t nblocks, uint32_t nsuper,
                              float4* __restrict__ sbox) {
  const int lane = threadIdx.x & 31;
  const uint32_t w0 = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, nw = (gridDim.x * blockDim.x) >> 5;
  for (uint32_t s = w0; s < nsuper; s += nw) {
    const uint32_t k = 32u * s + lane;
    V3 mn = mk(INFINITY, INFINITY, INFINITY), mx = mk(-INFINITY, -INFINITY, -INFINITY);
    if (k < nblocks) {
      mn = f4v(__ldg(box + 2 * (size_t)k));
      mx = f4v(__ldg(box + 2 * (size_t)k + 1));
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      mn = vmin(mn, mk(__shfl_xor_sync(0xFFFFFFFFu, mn.x, o), __shfl_xor_sync(0xFFFFFFFFu, mn.y, o),
                       __shfl_xor_sync(0xFFFFFFFFu, mn.z, o)));
      mx = vmax(mx, mk(__shfl_xor_sync(0xFFFFFFFFu, mx.x, o), __shfl_xor_sync(0xFFFFFFFFu, mx.y, o),
                       __shfl_xor_sync(0xFFFFFFFFu, mx.z, o)));
    }
    if (lane == 0) {
      sbox[2 * (size_t)s] = make_float4(mn.x, mn.y, mn.z, 0.f);
      sbox[2 * (size_t)s + 1] = make_float4(mx.x, mx.y, mx.z, 0.f);
    }
  }
}

// ---- distance to the nearest non-empty leaf (two-level grids) ---------------------
// For every leaf of a top cell with a leaf grid of more than one cell: D = the
// L-infinity distance (in leaf cells, capped at kLeafDistCap + 1) to the
// nearest non-empty leaf of the same grid, computed as three separable min-max
// passes (x, then y, then z).  An empty leaf stores [D, D): its range stays
// empty, and a DDA that fetched it may take its next D - 1 steps without
// fetching, since every cell within those steps lies closer than D.
constexpr uint32_t kLeafDistCap = 7;

// top cell owning leaf li: the last cell whose leaf offset is <= li (offsets
// are the exclusive scan of the leaf counts, so empty cells never match last)
SHN_D uint32_t leaf_owner(const uint2* __restrict__ cells, uint32_t C, uint32_t li) {
  uint32_t lo = 0, hi = C;
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(&cells[mid].x) <= li) lo = mid; else hi = mid;
  }
  return lo;
}

// pass: axis 0 reads occupancy from the leaves, axes 1 and 2 the previous pass
// (the first pass finds each leaf's top cell and keeps it in owner[])
template <int AXIS>
__global__ void k_leaf_dist(const uint2* __restrict__ cells, uint32_t C, uint2* __restrict__ leaves, uint32_t L,
                            uint32_t* __restrict__ owner, const uint8_t* __restrict__ din,
                            uint8_t* __restrict__ dout) {
  for (uint32_t li = blockIdx.x * blockDim.x + threadIdx.x; li < L; li += gridDim.x * blockDim.x) {
    uint32_t c;
    if (AXIS == 0) {
      c = leaf_owner(cells, C, li);
      owner[li] = c;
    } else {
      c = __ldg(owner + li);
    }
    const uint2 cw = __ldg(cells + c);
    const uint32_t rx = cw.y & 0xFFu, ry = (cw.y >> 8) & 0xFFu, rz = (cw.y >> 16) & 0xFFu;
    if (!(cw.y & kNotEmpty) || rx * ry * rz <= 1u) continue;
    const uint32_t k = li - cw.x;
    const uint32_t x = k % rx, y = (k / rx) % ry, z = k / (rx * ry);
    const uint32_t pos = AXIS == 0 ? x : (AXIS == 1 ? y : z);
    const uint32_t len = AXIS == 0 ? rx : (AXIS == 1 ? ry : rz);
    const uint32_t stride = AXIS == 0 ? 1u : (AXIS == 1 ? rx : rx * ry);
    uint32_t best = kLeafDistCap + 1;
    const uint32_t lo = pos >= kLeafDistCap ? pos - kLeafDistCap : 0u;
    const uint32_t hi = min(len - 1u, pos + kLeafDistCap);
    for (uint32_t q = lo; q <= hi; ++q) {
      const uint32_t j = li - pos * stride + q * stride;
      const uint32_t dq = q > pos ? q - pos : pos - q;
      uint32_t v;
      if (AXIS == 0) {
        const uint2 r = leaves[j];
        v = r.y > r.x ? dq : kLeafDistCap + 1;
      } else {
        v = max(dq, (uint32_t)__ldg(din + j));
      }
      best = min(best, v);
    }
    if (AXIS < 2) {
      dout[li] = (uint8_t)best;
    } else {
      const uint2 r = leaves[li];
      if (r.y <= r.x) leaves[li] = make_uint2(best, best);
    }
  }
}

// The same distances for the cells of a large uniform grid (one grid, no
// owner search); an empty cell stores [D, D).
constexpr uint64_t kCellDistMin = 1ull << 22;  // uniform grids with at least this many cells

// Uniform grids keep the larger cap: the path tracer's long walks through the
// empty space above a heightfield gain more from it (C2 784 -> 798 Mrays/s)
// than the wider windows cost its build.
constexpr uint32_t kCellDistCap = 15;

template <int AXIS>
__global__ void k_cell_dist(uint2* __restrict__ cells, uint32_t rx, uint32_t ry, uint32_t rz,
                            const uint8_t* __restrict__ din, uint8_t* __restrict__ dout) {
  const uint64_t n = (uint64_t)rx * ry * rz;
  for (uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; c < n; c += (uint64_t)gridDim.x * blockDim.x) {
    const uint32_t x = (uint32_t)(c % rx), y = (uint32_t)((c / rx) % ry), z = (uint32_t)(c / ((uint64_t)rx * ry));
    const uint32_t pos = AXIS == 0 ? x : (AXIS == 1 ? y : z);
    const uint32_t len = AXIS == 0 ? rx : (AXIS == 1 ? ry : rz);
    const uint64_t stride = AXIS == 0 ? 1ull : (AXIS == 1 ? (uint64_t)rx : (uint64_t)rx * ry);
    uint32_t best = kCellDistCap + 1;
    const uint32_t lo = pos >= kCellDistCap ? pos - kCellDistCap : 0u;
    const uint32_t hi = min(len - 1u, pos + kCellDistCap);
    for (uint32_t q = lo; q <= hi; ++q) {
      const uint64_t j = c - (uint64_t)pos * stride + (uint64_t)q * stride;
      const uint32_t dq = q > pos ? q - pos : pos - q;
      uint32_t v;
      if (AXIS == 0) {
        const uint2 r = cells[j];
        v = r.y > r.x ? dq : kCellDistCap + 1;
      } else {
        v = max(dq, (uint32_t)__ldg(din + j));
      }
      best = min(best, v);
    }
    if (AXIS < 2) {
      dout[c] = (uint8_t)best;
    } else {
      const uint2 r = cells[c];
      if (r.y <= r.x) cells[c] = make_uint2(best, best);
    }
  }
}

__global__ void __launch_bounds__(kScanBlock) k_leaf_cells_scan(const uint2* __restrict__ top_ranges,
                                                               uint32_t C, Geom g, float lambda,
                                                               uint32_t threshold, LookbackState st,
                                                               uint2* __restrict__ cells,
                                                               uint32_t* d_total) {
  __shared__ TileScanSmem<kScanBlock, kScanItems> sm;
  tile_scan<kScanBlock, kScanItems>(
      st, C, sm,
      [&](uint32_t c) {
        const uint2 r = top_ranges[c];
        uint32_t cnt;
        leaf_word(g, lambda, r.y - r.x, threshold, &cnt);
        return cnt;
      },
      [&](uint32_t c, uint32_t ex) {
        const uint2 r = top_ranges[c];
        uint32_t cnt;
        const uint32_t y = leaf_word(g, lambda, r.y - r.x, threshold, &cnt);
        cells[c] = make_uint2(ex, y);
      },
      d_total);
}

// ---- batched multi-scene build ---------------------------------------------------
// All scenes' triangles are one array (global triangle ids); scene s owns
// triangles [tri_off[s], tri_off[s+1]) and global cells
// [scenes[s].cell_offset, + res product).  One count/scan, one emit, one sort
// and one range pass serve every scene.
SHN_D uint32_t find_segment(const uint32_t* __restrict__ off, uint32_t nseg, uint32_t i) {
  uint32_t lo = 0, hi = nseg;  // off[lo] <= i < off[hi]
  while (hi - lo > 1) {
    const uint32_t mid = (lo + hi) >> 1;
    if (__ldg(off + mid) <= i) lo = mid; else hi = mid;
  }
  return lo;
}

__global__ void k_batch_pack(const float* __restrict__ vtx, const uint32_t* __restrict__ vtx_off,
                             const uint32_t* __restrict__ idx, const uint32_t* __restrict__ tri_off,
                             uint32_t ns, uint32_t T, float4* __restrict__ tri) {
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < T; t += gridDim.x * blockDim.x) {
    const uint32_t s = find_segment(tri_off, ns, t);
    const uint32_t vb = __ldg(vtx_off + s);
    const uint32_t i0 = vb + idx[3 * (size_t)t], i1 = vb + idx[3 * (size_t)t + 1], i2 = vb + idx[3 * (size_t)t + 2];
    const float* a = vtx + 3 * (size_t)i0;
    const float* b = vtx + 3 * (size_t)i1;
    const float* c = vtx + 3 * (size_t)i2;
    float4* r = tri + 3 * (size_t)t;
    r[0] = make_float4(a[0], a[1], a[2], __uint_as_float(t));
    r[1] = make_float4(b[0], b[1], b[2], 0.f);
    r[2] = make_float4(c[0], c[1], c[2], 0.f);
  }
}

__global__ void k_batch_bounds(const float4* __restrict__ tri, const uint32_t* __restrict__ tri_off,
                               uint32_t ns, uint32_t T, uint32_t* __restrict__ out) {
  for (uint32_t t0 = blockIdx.x * blockDim.x; t0 < T; t0 += gridDim.x * blockDim.x) {
    const uint32_t t = t0 + threadIdx.x;
    const bool valid = t < T;
    const uint32_t s = valid ? find_segment(tri_off, ns, t) : 0xFFFFFFFFu;
    V3 mn = mk(FLT_MAX, FLT_MAX, FLT_MAX), mx = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    if (valid) {
      for (int k = 0; k < 3; ++k) {
        const V3 p = f4v(tri[3 * (size_t)t + k]);
        mn = vmin(mn, p);
        mx = vmax(mx, p);
      }
    }
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, s);
    const int lane = threadIdx.x & 31;
    if (peers == 0xFFFFFFFFu) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        mn.x = fminf(mn.x, __shfl_xor_sync(0xFFFFFFFFu, mn.x, o));
        mn.y = fminf(mn.y, __shfl_xor_sync(0xFFFFFFFFu, mn.y, o));
        mn.z = fminf(mn.z, __shfl_xor_sync(0xFFFFFFFFu, mn.z, o));
        mx.x = fmaxf(mx.x, __shfl_xor_sync(0xFFFFFFFFu, mx.x, o));
        mx.y = fmaxf(mx.y, __shfl_xor_sync(0xFFFFFFFFu, mx.y, o));
        mx.z = fmaxf(mx.z, __shfl_xor_sync(0xFFFFFFFFu, mx.z, o));
      }
      if (lane != 0) continue;
    }
    if (!valid) continue;
    uint32_t* o6 = out + 6 * (size_t)s;
    atomicMin(o6 + 0, fkey(mn.x)); atomicMin(o6 + 1, fkey(mn.y)); atomicMin(o6 + 2, fkey(mn.z));
    atomicMax(o6 + 3, fkey(mx.x)); atomicMax(o6 + 4, fkey(mx.y)); atomicMax(o6 + 5, fkey(mx.z));
  }
}

__global__ void k_batch_bounds_decode(uint32_t* io, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) io[i] = __float_as_uint(fval(io[i]));
}

struct BatchMaker {
  TriArr tri;
  const uint32_t* tri_off;
  const BatchScene* scenes;
  uint32_t ns;
  SHN_D bool operator()(uint32_t t, Unit& U) const {
    const uint32_t s = find_segment(tri_off, ns, t);
    V3 a, b, c;
    load_tri(tri, t, a, b, c);
    top_unit(a, b, c, scenes[s].g, t, (uint32_t)scenes[s].cell_offset, U);
    return true;
  }
};

int grid_for(uint64_t n, int block, int max_blocks) {
  const uint64_t b = (n + block - 1) / block;
  return (int)std::max<uint64_t>(1, std::min<uint64_t>(b, (uint64_t)max_blocks));
}

// Exact counts of n items into offs[0..n) then the in-place scan: offs[i] =
// first output slot of item i, offs[n] = total.  ws: (tiles + 2) * 8 bytes
// (look-back status, scan ticket, count group counter), zeroed here.
template <class Maker>
void launch_counts(Maker mk, uint32_t n, uint32_t* offs, void* ws, uint32_t* err, cudaStream_t st) {
  const size_t tiles = ((size_t)n + kScanTile - 1) / kScanTile;
  uint64_t* status = (uint64_t*)ws;
  cudaMemsetAsync(status, 0, (tiles + 2) * 8, st);
  uint32_t* ticket = (uint32_t*)(status + tiles + 1);
  const int blocks = grid_for((n + 31) / 32, kUnitWarps, 148 * 7);
  k_count_groups<<<blocks, kScanBlock, 0, st>>>(mk, n, offs, ticket + 1);
  k_scan_inplace<<<(unsigned)tiles, kScanBlock, 0, st>>>(offs, n, LookbackState{status, ticket, err});
}

// The counts and offsets of the precise insertion (as launch_counts).
void launch_counts_sat(TriArr tri, Geom g, uint32_t n, uint32_t* offs, void* ws, uint32_t* err, cudaStream_t st) {
  const size_t tiles = ((size_t)n + kScanTile - 1) / kScanTile;
  uint64_t* status = (uint64_t*)ws;
  cudaMemsetAsync(status, 0, (tiles + 2) * 8, st);
  uint32_t* ticket = (uint32_t*)(status + tiles + 1);
  k_count_sat<<<grid_for(n, 128, 148 * 16), 128, 0, st>>>(tri, n, g, offs);
  k_scan_inplace<<<(unsigned)tiles, kScanBlock, 0, st>>>(offs, n, LookbackState{status, ticket, err});
}

shn_status ensure(shn_grid* g, void** p, size_t* cap, size_t bytes, cudaStream_t st) {
  if (*cap >= bytes && *p) return SHN_OK;
  if (*p) dev_free(g->ctx, *p, *cap, st);
  *p = nullptr;
  *cap = 0;
  size_t want = std::max<size_t>(bytes + bytes / 8, 256);
  cudaError_t e = dev_alloc(g->ctx, p, want, st);
  if (e != cudaSuccess) {
    *p = nullptr;
    return e == cudaErrorMemoryAllocation ? set_error(g->ctx, SHN_ERR_OOM, "device allocation failed")
                                          : (e == cudaErrorNotPermitted ? set_error(g->ctx, SHN_ERR_BUDGET, "HBM budget exceeded")
                                                                        : cuda_status(g->ctx, e, "alloc"));
  }
  *cap = want;
  return SHN_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
Geom make_geom(const float b[6], const int res[3]) {
  Geom g;
  g.gmin = mk(b[0], b[1], b[2]);
  g.gmax = mk(b[3], b[4], b[5]);
  for (int i = 0; i < 3; ++i) g.res[i] = res[i];
  g.resf = mk((float)res[0], (float)res[1], (float)res[2]);
  const V3 diag = sub(g.gmax, g.gmin);
  g.cs = divv(diag, g.resf);
  g.rcpBuild = divv(mk(1.f, 1.f, 1.f), g.cs);
  g.rcpTrav = divv(g.resf, diag);
  return g;
}

// GridBuilder::computeResolution (GridBuilder.h:41-62) and the two-level top
// rule (FastTwoLevelGridBuilder.h:87-102), each axis clamped to [1, 2048].
void compute_resolution(uint32_t nt, const float b[6], float lambda, int divisor, int min_res,
                        int out[3]) {
  V3 diag = sub(mk(b[3], b[4], b[5]), mk(b[0], b[1], b[2]));
  const float volume = diag.x * diag.y * diag.z;
  const float magic = powf(lambda * (float)nt / volume, 0.3333333f);
  diag = muls(diag, magic);
  const float d[3] = {diag.x, diag.y, diag.z};
  for (int a = 0; a < 3; ++a) {
    const float v = d[a];
    int r = (v >= 2048.f || !(v == v)) ? 2048 : (int)v;
    if (divisor > 1) r = r / divisor;
    r = std::max(r, min_res);
    r = std::min(std::max(r, 1), 2048);
    out[a] = r;
  }
}

void launch_pack_triangles(const float* vtx, const uint32_t* idx, uint32_t nt, float4* tri,
                           cudaStream_t st) {
  if (!nt) return;
  k_pack_triangles<<<grid_for(nt, 256, 148 * 16), 256, 0, st>>>(vtx, idx, nt, tri);
}

void launch_bounds_reduce(const float4* tri, uint32_t nt, float* d_out6, cudaStream_t st) {
  uint32_t init[6];
  for (int i = 0; i < 3; ++i) init[i] = 0xFFFFFFFFu;
  for (int i = 3; i < 6; ++i) init[i] = 0u;
  cudaMemcpyAsync(d_out6, init, sizeof(init), cudaMemcpyHostToDevice, st);
  if (nt) k_bounds<<<grid_for(3ull * nt, 256, 148 * 8), 256, 0, st>>>(tri, nt, (uint32_t*)d_out6);
  k_bounds_decode<<<1, 32, 0, st>>>((uint32_t*)d_out6);
}

namespace {

shn_status ensure_buf(shn_grid* g, DevBuf& b, size_t bytes, cudaStream_t st) {
  return ensure(g, &b.ptr, &b.bytes, bytes, st);
}

LookbackState scan_state(shn_grid* g, uint64_t n, cudaStream_t st, shn_status* rc) {
  const size_t tiles = ((size_t)n + kScanTile - 1) / kScanTile;
  *rc = ensure_buf(g, g->scan, (tiles + 2) * 8, st);
  uint64_t* status = (uint64_t*)g->scan.ptr;
  uint32_t* ticket = (uint32_t*)(status + tiles + 1);
  if (*rc == SHN_OK) cudaMemsetAsync(status, 0, (tiles + 2) * 8, st);
  return LookbackState{status, ticket, g->d_err};
}

int range_blocks(uint64_t n) { return grid_for(n, kRangeBlock * kRangeItems, 148 * 8); }

// Emit grid: groups of 32 items, kUnitWarps groups per block step.
int emit_blocks(uint64_t n) { return grid_for((n + 31) / 32, kUnitWarps, 148 * 8); }

uint32_t scan_tiles(uint64_t n) { return (uint32_t)std::max<uint64_t>(1, (n + kScanTile - 1) / kScanTile); }

shn_status read_words(shn_grid* g, const uint32_t* d_src[], int k, uint32_t* out,
                      cudaStream_t st) {
  for (int i = 0; i < k; ++i)
    cudaMemcpyAsync(g->h_pinned + i, d_src[i], 4, cudaMemcpyDeviceToHost, st);
  cudaMemcpyAsync(g->h_pinned + 7, g->d_err, 4, cudaMemcpyDeviceToHost, st);
  cudaError_t e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) return cuda_status(g->ctx, e, "build sync");
  if (g->h_pinned[7] != 0u)
    return set_error(g->ctx, SHN_ERR_TIMEOUT, "a bounded device wait gave up during the build");
  for (int i = 0; i < k; ++i) out[i] = g->h_pinned[i];
  return SHN_OK;
}

// The build's last stage is not waited for: the end event orders every
// consumer (traces on any stream, exports, info), and a bounded wait that
// gives up in it is reported through the grid's error word
// (shn_grid_sync_status), like the traces' own.  The two size read-backs
// before it have already checked the word for the earlier stages.
shn_status finish(shn_grid* g, cudaStream_t st) {
  cudaEventRecord(g->ev1, st);
  g->build_ms_pending = true;
  g->built = true;
  return SHN_OK;
}

}  // namespace

void grid_fence(const shn_grid* g, cudaStream_t st) {
  if (g->ev1) cudaStreamWaitEvent(st, g->ev1, 0);
}

float grid_build_ms(const shn_grid* g) {
  if (g->build_ms_pending && g->ev1 && cudaEventSynchronize(g->ev1) == cudaSuccess) {
    cudaEventElapsedTime(&g->build_ms, g->ev0, g->ev1);
    g->build_ms_pending = false;
  }
  return g->build_ms;
}

shn_status build_grid(shn_grid* g, const shn_scene* s, const shn_grid_params* p, cudaStream_t st) {
  shn_ctx* ctx = g->ctx;
  const uint32_t nt = s->nt;
  int res[3];
  if (p->res[0] > 0 && p->res[1] > 0 && p->res[2] > 0) {
    for (int i = 0; i < 3; ++i) res[i] = std::min(p->res[i], 2048);
  } else {
    compute_resolution(nt, s->bounds, p->lambda, p->top_divisor, p->min_res, res);
  }
  const uint64_t C = (uint64_t)res[0] * res[1] * res[2];
  if (C >= (1ull << 31)) return set_error(ctx, SHN_ERR_INVALID, "grid resolution too large");
  g->kind = p->kind;
  g->geom = make_geom(s->bounds, res);
  const bool sat = p->insertion == SHN_INSERT_SAT;
  g->built = false;
  g->src_tri = s->ids ? s->ids : s->tri;
  g->src_nt = s->nt;
  if (!g->d_err) {
    // stream-ordered pool memory and a pinned block from the context's slab:
    // no device-wide synchronisation while other streams are running
    cudaError_t e = dev_alloc(ctx, (void**)&g->d_err, 64, st);
    if (e != cudaSuccess) {
      g->d_err = nullptr;
      return e == cudaErrorNotPermitted ? set_error(ctx, SHN_ERR_BUDGET, "HBM budget exceeded")
                                        : set_error(ctx, SHN_ERR_OOM, "err word");
    }
    g->h_pinned = pinned_take(ctx);
    if (!g->h_pinned) return set_error(ctx, SHN_ERR_OOM, "pinned");
    cudaEventCreate(&g->ev0);
    cudaEventCreate(&g->ev1);
  }
  cudaMemsetAsync(g->d_err, 0, 64, st);
  cudaEventRecord(g->ev0, st);
  TriArr tri{s->tri};
  shn_status rc;
  g->num_blocks = g->num_super = 0;
  g->cell_dist = false;

  // ---- two-level: build on the triangles in Morton order ------------------------
  g->spatial = p->kind == SHN_GRID_TWO_LEVEL && nt > 1;
  if (g->spatial) {
    const uint32_t tb = 32u - (uint32_t)__builtin_clz(nt - 1);
    for (int i = 0; i < 2; ++i)
      if ((rc = ensure_buf(g, g->keys[i], (size_t)nt * 8, st))) return rc;
    if ((rc = ensure_buf(g, g->mhi, (size_t)nt * 4, st))) return rc;
    if ((rc = ensure_buf(g, g->perm_tri, (size_t)nt * 48, st))) return rc;
    if ((rc = ensure_buf(g, g->sortws, sort_workspace_bytes(nt), st))) return rc;
    const V3 lo = mk(s->bounds[0], s->bounds[1], s->bounds[2]);
    const V3 hi = mk(s->bounds[3], s->bounds[4], s->bounds[5]);
    const V3 lo3 = muls(lo, 3.f), ext3 = sub(muls(hi, 3.f), lo3);
    const V3 scale = mk(ext3.x > 0.f ? 1048576.f / ext3.x : 0.f, ext3.y > 0.f ? 1048576.f / ext3.y : 0.f,
                        ext3.z > 0.f ? 1048576.f / ext3.z : 0.f);
    uint64_t* m0 = (uint64_t*)g->keys[0].ptr;
    uint64_t* m1 = (uint64_t*)g->keys[1].ptr;
    uint32_t* mh = (uint32_t*)g->mhi.ptr;
    const int blocks = grid_for(nt, 256, 148 * 16);
    k_morton_keys<<<blocks, 256, 0, st>>>(tri, nt, lo3, scale, tb, m0, mh);
    uint64_t* s1 = onesweep_sort(m0, m1, nt, tb, sort_plan(30), g->sortws.ptr, g->d_err, st);
    uint64_t* o1 = s1 == m0 ? m1 : m0;
    k_morton_second<<<blocks, 256, 0, st>>>(s1, mh, nt, tb, o1);
    uint64_t* s2 = onesweep_sort(o1, s1, nt, tb, sort_plan(30), g->sortws.ptr, g->d_err, st);
    k_permute_tris<<<blocks, 256, 0, st>>>(s2, tri, nt, tb, (float4*)g->perm_tri.ptr);
    tri = TriArr{(const float4*)g->perm_tri.ptr};
  }

  // ---- counts + offsets ------------------------------------------------------
  if ((rc = ensure_buf(g, g->offs_tri, ((size_t)nt + 1) * 4, st))) return rc;
  uint32_t* offs = (uint32_t*)g->offs_tri.ptr;
  uint32_t P = 0;
  if (nt) {
    if ((rc = ensure_buf(g, g->scan, (((size_t)nt + kScanTile - 1) / kScanTile + 2) * 8, st))) return rc;
    if (sat) launch_counts_sat(tri, g->geom, nt, offs, g->scan.ptr, g->d_err, st);
    else launch_counts(TopMaker{tri, g->geom}, nt, offs, g->scan.ptr, g->d_err, st);
    const uint32_t* src[1] = {offs + nt};
    if ((rc = read_words(g, src, 1, &P, st))) return rc;
  }
  if (P >= (1u << 30)) return set_error(ctx, SHN_ERR_INVALID, "more than 2^30 cell references");

  // ---- emit + sort (uniform grid / top level) ----------------------------------
  for (int i = 0; i < 2; ++i)
    if ((rc = ensure_buf(g, g->keys[i], (size_t)std::max<uint32_t>(P, 1) * 8, st))) return rc;
  if ((rc = ensure_buf(g, g->sortws, sort_workspace_bytes(P), st))) return rc;
  uint64_t* k0 = (uint64_t*)g->keys[0].ptr;
  uint64_t* k1 = (uint64_t*)g->keys[1].ptr;
  const SortPlan top_plan = sort_plan(key_bits_for(C ? C - 1 : 0));
  sort_prepare(g->sortws.ptr, st);
  if (nt && sat)
    k_emit_sat<<<grid_for(nt, kScanBlock, 148 * 8), kScanBlock, 0, st>>>(tri, nt, g->geom, offs, k0, P, g->d_err,
                                                                        sort_hist_counts(g->sortws.ptr), top_plan);
  else if (nt)
    k_emit_units<<<emit_blocks(nt), kScanBlock, 0, st>>>(TopMaker{tri, g->geom}, nt, offs, k0, P, g->d_err,
                                                        sort_hist_counts(g->sortws.ptr), top_plan);
  uint64_t* sortedTop = onesweep_sort(k0, k1, P, 32, top_plan, g->sortws.ptr, g->d_err, st, true);
  const int topBuf = sortedTop == k0 ? 0 : 1;

  g->num_cells = C;
  g->num_top_refs = (p->kind == SHN_GRID_TWO_LEVEL) ? P : 0;
  if ((rc = ensure(g, (void**)&g->cells, &g->cap_cells, C * 8, st))) return rc;

  if (p->kind == SHN_GRID_UNIFORM) {
    if ((rc = ensure(g, (void**)&g->indices, &g->cap_refs, (size_t)std::max<uint32_t>(P, 1) * 4, st))) return rc;
    if ((rc = ensure(g, (void**)&g->rtri, &g->cap_rtri, (size_t)std::max<uint32_t>(P, 1) * 48, st))) return rc;
    cudaMemsetAsync(g->cells, 0, C * 8, st);
    if (P) k_ranges<<<range_blocks(P), kRangeBlock, 0, st>>>(sortedTop, P, g->cells, g->indices, tri, g->rtri);
    g->cell_dist = C >= kCellDistMin;
    if (g->cell_dist) {
      if ((rc = ensure_buf(g, g->ldist, 2 * (size_t)C, st))) return rc;
      uint8_t* d1 = (uint8_t*)g->ldist.ptr;
      uint8_t* d2 = d1 + C;
      const int blocks = grid_for(C, 256, 148 * 8);
      k_cell_dist<0><<<blocks, 256, 0, st>>>(g->cells, res[0], res[1], res[2], nullptr, d1);
      k_cell_dist<1><<<blocks, 256, 0, st>>>(g->cells, res[0], res[1], res[2], d1, d2);
      k_cell_dist<2><<<blocks, 256, 0, st>>>(g->cells, res[0], res[1], res[2], d2, nullptr);
    }
    g->num_refs = P;
    g->num_leaves = 0;
    g->top_pairs = sortedTop;
    return finish(g, st);
  }

  // ---- two-level leaf stage ------------------------------------------------------
  if ((rc = ensure_buf(g, g->top_ranges, C * 8, st))) return rc;
  uint2* topRanges = (uint2*)g->top_ranges.ptr;
  cudaMemsetAsync(topRanges, 0, C * 8, st);
  if (P) k_ranges<<<range_blocks(P), kRangeBlock, 0, st>>>(sortedTop, P, topRanges, nullptr, tri, nullptr);
  uint32_t* d_L = g->d_err + 1;
  {
    LookbackState ls = scan_state(g, C, st, &rc);
    if (rc) return rc;
    k_leaf_cells_scan<<<scan_tiles(C), kScanBlock, 0, st>>>(topRanges, (uint32_t)C, g->geom,
                                                           p->lambda_leaf, p->leaf_threshold, ls,
                                                           g->cells, d_L);
  }
  if ((rc = ensure_buf(g, g->offs_pair, ((size_t)P + 1) * 4, st))) return rc;
  uint32_t* pairOffs = (uint32_t*)g->offs_pair.ptr;
  if (P) {
    if ((rc = ensure_buf(g, g->scan, (((size_t)P + kScanTile - 1) / kScanTile + 2) * 8, st))) return rc;
    launch_counts(LeafMaker{tri, sortedTop, g->cells, g->geom}, P, pairOffs, g->scan.ptr, g->d_err, st);
  } else {
    cudaMemsetAsync(pairOffs, 0, 4, st);
  }
  uint32_t sizes[2];
  {
    const uint32_t* src[2] = {d_L, pairOffs + P};
    if ((rc = read_words(g, src, 2, sizes, st))) return rc;
  }
  const uint32_t Lc = sizes[0], R = sizes[1];
  if (R >= (1u << 30)) return set_error(ctx, SHN_ERR_INVALID, "more than 2^30 leaf references");
  const int bA = (topBuf + 1) % 3, bB = (topBuf + 2) % 3;
  if ((rc = ensure_buf(g, g->keys[bA], (size_t)std::max<uint32_t>(R, 1) * 8, st))) return rc;
  if ((rc = ensure_buf(g, g->keys[bB], (size_t)std::max<uint32_t>(R, 1) * 8, st))) return rc;
  if ((rc = ensure_buf(g, g->sortws, sort_workspace_bytes(R), st))) return rc;
  uint64_t* lk0 = (uint64_t*)g->keys[bA].ptr;
  uint64_t* lk1 = (uint64_t*)g->keys[bB].ptr;
  const SortPlan leaf_plan = sort_plan(key_bits_for(Lc ? Lc - 1 : 0));
  sort_prepare(g->sortws.ptr, st);
  if (P)
    k_emit_units<<<emit_blocks(P), kScanBlock, 0, st>>>(LeafMaker{tri, sortedTop, g->cells, g->geom}, P,
                                                       pairOffs, lk0, R, g->d_err,
                                                       sort_hist_counts(g->sortws.ptr), leaf_plan);
  uint64_t* sortedLeaf = onesweep_sort(lk0, lk1, R, 32, leaf_plan, g->sortws.ptr, g->d_err, st, true);
  if ((rc = ensure(g, (void**)&g->leaves, &g->cap_leaves, (size_t)std::max<uint32_t>(Lc, 1) * 8, st))) return rc;
  if ((rc = ensure(g, (void**)&g->indices, &g->cap_refs, (size_t)std::max<uint32_t>(R, 1) * 4, st))) return rc;
  if ((rc = ensure(g, (void**)&g->rtri, &g->cap_rtri, (size_t)std::max<uint32_t>(R, 1) * 48, st))) return rc;
  cudaMemsetAsync(g->leaves, 0, (size_t)Lc * 8, st);
  if (R) k_ranges<<<range_blocks(R), kRangeBlock, 0, st>>>(sortedLeaf, R, g->leaves, g->indices, tri, g->rtri);
  if (g->spatial && Lc) {
    if ((rc = ensure_buf(g, g->ldist, 6 * (size_t)Lc, st))) return rc;
    uint32_t* own = (uint32_t*)g->ldist.ptr;
    uint8_t* d1 = (uint8_t*)(own + Lc);
    uint8_t* d2 = d1 + Lc;
    const int blocks = grid_for(Lc, 256, 148 * 8);
    k_leaf_dist<0><<<blocks, 256, 0, st>>>(g->cells, (uint32_t)C, g->leaves, Lc, own, nullptr, d1);
    k_leaf_dist<1><<<blocks, 256, 0, st>>>(g->cells, (uint32_t)C, g->leaves, Lc, own, d1, d2);
    k_leaf_dist<2><<<blocks, 256, 0, st>>>(g->cells, (uint32_t)C, g->leaves, Lc, own, d2, nullptr);
  }
  if (g->spatial && R) {
    const uint64_t nb = (R + 31) / 32, ns = (nb + 31) / 32;
    if ((rc = ensure_buf(g, g->cbox, nb * 32, st))) return rc;
    if ((rc = ensure_buf(g, g->sbox, ns * 32, st))) return rc;
    const float4* rv = g->rtri;
    k_block_boxes<<<grid_for(nb * 32, 256, 148 * 8), 256, 0, st>>>(rv, rv + R, rv + 2 * (size_t)R, R, (uint32_t)nb,
                                                                  (float4*)g->cbox.ptr);
    k_super_boxes<<<grid_for(ns * 32, 256, 148 * 8), 256, 0, st>>>((const float4*)g->cbox.ptr, (uint32_t)nb,
                                                                  (uint32_t)ns, (float4*)g->sbox.ptr);
    g->num_blocks = nb;
    g->num_super = ns;
  }
  g->num_leaves = Lc;
  g->num_refs = R;
  g->top_pairs = sortedTop;
  return finish(g, st);
}


// ---- batch launch wrappers (host) ------------------------------------------------------
void launch_batch_pack(const float* vtx, const uint32_t* vtx_off, const uint32_t* idx,
                       const uint32_t* tri_off, uint32_t ns, uint32_t T, float4* tri, cudaStream_t st) {
  if (T) k_batch_pack<<<grid_for(T, 256, 148 * 16), 256, 0, st>>>(vtx, vtx_off, idx, tri_off, ns, T, tri);
}

void launch_batch_bounds(const float4* tri, const uint32_t* tri_off, uint32_t ns, uint32_t T,
                         float* d_out6ns, cudaStream_t st) {
  std::vector<uint32_t> init(6 * (size_t)ns);
  for (uint32_t s = 0; s < ns; ++s)
    for (int i = 0; i < 6; ++i) init[6 * s + i] = i < 3 ? 0xFFFFFFFFu : 0u;
  cudaMemcpyAsync(d_out6ns, init.data(), init.size() * 4, cudaMemcpyHostToDevice, st);
  cudaStreamSynchronize(st);  // init lives on the host stack
  if (T) k_batch_bounds<<<grid_for(T, 256, 148 * 16), 256, 0, st>>>(tri, tri_off, ns, T, (uint32_t*)d_out6ns);
  k_batch_bounds_decode<<<(6 * ns + 255) / 256, 256, 0, st>>>((uint32_t*)d_out6ns, 6 * ns);
}

size_t batch_scan_bytes(uint32_t T) { return (((size_t)T + kScanTile - 1) / kScanTile + 2) * 8; }

void launch_batch_count(const float4* tri, uint32_t T, const uint32_t* tri_off, const BatchScene* scenes,
                        uint32_t ns, void* scan_ws, uint32_t* err, uint32_t* offs, cudaStream_t st) {
  if (!T) {
    cudaMemsetAsync(offs, 0, 4, st);
    return;
  }
  const TriArr ts{tri};
  launch_counts(BatchMaker{ts, tri_off, scenes, ns}, T, offs, scan_ws, err, st);
}

void launch_batch_emit(const float4* tri, uint32_t T, const uint32_t* tri_off, const BatchScene* scenes,
                       uint32_t ns, const uint32_t* offs, uint64_t* keys, uint32_t capacity,
                       uint32_t* err, uint32_t* hist, SortPlan hplan, cudaStream_t st) {
  const TriArr ts{tri};
  if (T)
    k_emit_units<<<emit_blocks(T), kScanBlock, 0, st>>>(BatchMaker{ts, tri_off, scenes, ns}, T, offs, keys,
                                                       capacity, err, hist, hplan);
}

void launch_cell_ranges(const uint64_t* keys, uint32_t n, uint64_t C, uint2* ranges, uint32_t* indices,
                        cudaStream_t st) {
  if (!C) return;
  const uint64_t tiles = (C + kCellTile - 1) / kCellTile;
  k_cell_ranges<<<(unsigned)std::min<uint64_t>(tiles, 148u * 16u), kRangeBlock, 0, st>>>(keys, n, C, ranges,
                                                                                         indices);
}

void launch_ranges(const uint64_t* keys, uint32_t n, uint2* ranges, uint32_t* indices,
                   const float4* tri, uint32_t T, float4* rtri, cudaStream_t st) {
  const TriArr ts{tri};
  if (n) k_ranges<<<range_blocks(n), kRangeBlock, 0, st>>>(keys, n, ranges, indices, ts, rtri);
}

}  // namespace shn
