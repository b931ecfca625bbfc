// Warp-cooperative traversal engine.
//
// Every lane owns one ray and walks the grid with an explicit DDA state
// machine, so the lanes of a warp reach "here is my next cell range" at the
// same point of the loop.  The ranges are then tested in two phases:
//  * small ranges (<= kCoopThreshold references): each lane tests its own
//    range, as the reference's SimpleIntersector does;
//  * large ranges: the whole warp tests one lane's range, 32 triangles per
//    instruction, with that lane's ray broadcast (warp-uniform, so the
//    watertight test's axis permutation is a compile-time constant), and the
//    closest hit is reduced across the warp.  This generalises the
//    reference's HybridIntersector work donation
//    (src/Intersector/HybridIntersector.hpp:472-704) and keeps lanes busy
//    when one ray sits in a cell with tens of thousands of references.
//    When several lanes wait on the same large range, each 32-reference chunk
//    is loaded once and tested against all of their rays (group_range).
// Lanes whose ray has finished take a new ray from the global pool at the
// top of the loop (persistent threads), one by one or, for coherent rays, as
// a warp of 32 once all lanes are done (PACKET).
//
// The per-ray sequence of cell visits, tests and continuation decisions is
// exactly that of trace_uniform / trace_two_level (trace.cuh) (block culling
// and the empty-leaf skips only leave out work that cannot change the result);
// the closest hit of a range is the least (t, triangle id) of its candidates,
// the winner the reference's strict-< loop keeps over references in (cell,
// triangle) order, so results are identical.
#pragma once
#include <type_traits>

#include "trace.cuh"

namespace shn {

constexpr uint32_t kCoopThreshold = 32;
constexpr int kCoopBlock = 128;  // threads per block of every kernel that runs the engine

// Reference-ordered triangle arrays of one grid, and the scene's records
// indexed by triangle id (for the final hit record).
struct Refs {
  const float4* __restrict__ rv0;
  const float4* __restrict__ rv1;
  const float4* __restrict__ rv2;
  const float4* __restrict__ src;
  const float4* __restrict__ cbox;  // block boxes (see GridView), or null
  const float4* __restrict__ sbox;
  const uint32_t* __restrict__ ridx;  // not null: reference i is src[3 * ridx[i]] (no rv*)
};
SHN_D Refs refs_of(const GridView& G) { return Refs{G.rv0, G.rv1, G.rv2, G.src, G.cbox, G.sbox, G.ridx}; }

// Triangle of reference i: from the reference-ordered arrays, or (IND: grids
// that keep no reference-ordered copy) through the reference's triangle id.
template <bool IND>
SHN_D void ref_load(const Refs& G, uint32_t i, float4& p0, float4& p1, float4& p2) {
  if (IND) {
    const float4* r = G.src + 3 * (size_t)__ldg(G.ridx + i);
    p0 = __ldg(r);
    p1 = __ldg(r + 1);
    p2 = __ldg(r + 2);
  } else {
    p0 = __ldg(G.rv0 + i);
    p1 = __ldg(G.rv1 + i);
    p2 = __ldg(G.rv2 + i);
  }
}

// Ranges longer than this are tested block by block with box culling when the
// grid has block boxes.
constexpr uint32_t kCullMin = 64;

// Reciprocal direction for box tests: infinities (zero direction components)
// become +-1e30, so that a box face through the origin gives 0, not NaN.
SHN_D V3 cull_rcp(V3 r) {
  return mk(isinf(r.x) ? copysignf(1e30f, r.x) : r.x, isinf(r.y) ? copysignf(1e30f, r.y) : r.y,
            isinf(r.z) ? copysignf(1e30f, r.z) : r.z);
}

// Whether the segment t in (0, tb] of the ray o + t d (cr = cull_rcp(1/d)) can
// meet a triangle inside the box [mn, mx].  The slab distances carry a margin
// of 2^-8 of their magnitude, far above the rounding of the slab arithmetic
// and of the watertight test's t, so a block holding a triangle that the
// watertight test hits below tb is never skipped.  Overflowing distances
// (no finite margin) keep the box.
SHN_D bool box_meets(V3 o, V3 cr, float4 mn, float4 mx, float tb) {
  const float x1 = (mn.x - o.x) * cr.x, x2 = (mx.x - o.x) * cr.x;
  const float y1 = (mn.y - o.y) * cr.y, y2 = (mx.y - o.y) * cr.y;
  const float z1 = (mn.z - o.z) * cr.z, z2 = (mx.z - o.z) * cr.z;
  const float tn = fmaxf(fmaxf(fminf(x1, x2), fminf(y1, y2)), fminf(z1, z2));
  const float tf = fminf(fminf(fmaxf(x1, x2), fmaxf(y1, y2)), fmaxf(z1, z2));
  const float m = (fabsf(tn) + fabsf(tf)) * 0x1p-8f + 1e-30f;
  if (!(m < INFINITY)) return true;
  return tn - m <= tf + m && tf + m >= 0.f && tn - m <= tb;
}

// Number of references of block k inside [b, e).
SHN_D uint32_t block_refs(uint32_t k, uint32_t b, uint32_t e) {
  return min(e, 32u * k + 32u) - max(b, 32u * k);
}

enum : uint32_t { ST_DONE = 0, ST_TOP = 1, ST_LEAF = 2, ST_LEAF_TESTED = 3, ST_TOP_NEXT = 4, ST_U_TESTED = 5 };

struct Lane {
  V3 org, rcp;
  float Sx, Sy, Sz;
  uint32_t perm;          // kx | ky << 2 | kz << 4
  float tbest;
  uint32_t best;          // triangle id of the best hit, kMiss if none
  V3 cell, tMax;
  float tEntry;
  int vis, cap;
  V3 sc, sMax, scs, cres;
  uint32_t lb;
  int vis2;
  uint32_t b, e;
  uint32_t st;
  uint32_t anyhit;        // runtime any-hit flag (mixed launches)
};

// The same state for kernels that test shared ranges as a group: the first
// eight words hold what a group test reads of another lane's ray (origin and
// shear, then the permutation and the bound) as two 16-byte words.  The
// kernels without grouping keep the layout above, measured faster for them.
struct __align__(16) LaneG {
  V3 org;
  float Sx;
  float Sy, Sz;
  uint32_t perm;
  float tbest;
  uint32_t best;
  V3 rcp;
  V3 cell, tMax;
  float tEntry;
  int vis, cap;
  V3 sc, sMax, scs, cres;
  uint32_t lb;
  int vis2;
  uint32_t b, e;
  uint32_t st;
  uint32_t anyhit;
};

template <class LT>
SHN_D RayWT lane_ray(const LT& L) {
  RayWT r;
  r.org = L.org;
  r.kx = L.perm & 3;
  r.ky = (L.perm >> 2) & 3;
  r.kz = (L.perm >> 4) & 3;
  r.Sx = L.Sx;
  r.Sy = L.Sy;
  r.Sz = L.Sz;
  return r;
}

template <int KIND, class LT>
SHN_D void lane_init(const Geom& g, LT& L, V3 org, V3 dir, float tmax) {
  L.org = org;
  L.rcp = divv(mk(1.f, 1.f, 1.f), dir);
  const RayWT w = wt_setup(org, dir);
  L.Sx = w.Sx;
  L.Sy = w.Sy;
  L.Sz = w.Sz;
  L.perm = (uint32_t)w.kx | ((uint32_t)w.ky << 2) | ((uint32_t)w.kz << 4);
  L.tbest = tmax;
  L.best = kMiss;
  L.anyhit = 0;
  L.st = ST_DONE;
  L.b = L.e = 0;
  if (!(L.tbest > 0.f)) return;
  const V3 rcp = L.rcp;
  const V3 t1 = mul(sub(g.gmin, org), rcp);
  V3 t2 = mul(sub(g.gmax, org), rcp);
  const V3 tmn = vmin(t1, t2);
  t2 = vmax(t1, t2);
  float tEntry = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
  const float tExit = fminf(fminf(t2.x, t2.y), t2.z);
  if (tExit <= tEntry || tExit < 0.f) return;
  V3 entry;
  if (KIND == 0) {
    const float te = tEntry + kEps;
    entry = (tEntry >= 0.f) ? add(org, divv(mk(te, te, te), rcp)) : org;
  } else {
    tEntry = fmaxf(0.f, tEntry);
    const float te = tEntry + kEps;
    entry = add(org, divv(mk(te, te, te), rcp));
  }
  L.tEntry = tEntry;
  V3 cell = mul(sub(entry, g.gmin), g.rcpTrav);
  cell = mk(floorf(cell.x), floorf(cell.y), floorf(cell.z));
  const V3 tmp = mk(rcp.x > 0.f ? 1.f : 0.f, rcp.y > 0.f ? 1.f : 0.f, rcp.z > 0.f ? 1.f : 0.f);
  L.cell = cell;
  L.tMax = mul(sub(add(mul(add(cell, tmp), g.cs), g.gmin), org), rcp);
  const bool valid = (cell.x != (rcp.x > 0.f ? g.resf.x : -1.f)) &&
                     (cell.y != (rcp.y > 0.f ? g.resf.y : -1.f)) &&
                     (cell.z != (rcp.z > 0.f ? g.resf.z : -1.f));
  L.vis = 0;
  L.cap = g.res[0] + g.res[1] + g.res[2] + 3;
  L.st = valid ? ST_TOP : ST_DONE;
}

// Runs the lane's state machine until it has a non-empty range to test
// (returns true, range in L.b/L.e) or the ray is finished (returns false).
template <int KIND, bool ANY, class LT>
SHN_D bool lane_advance(const Geom& g, const uint2* __restrict__ cells, const uint2* __restrict__ leaves,
                        LT& L, uint32_t& steps) {
  while (true) {
    switch (L.st) {
      case ST_TOP: {
        L.vis++;
        const uint32_t cx = (uint32_t)clampf(L.cell.x, 0.f, g.resf.x - 1.f);
        const uint32_t cy = (uint32_t)clampf(L.cell.y, 0.f, g.resf.y - 1.f);
        const uint32_t cz = (uint32_t)clampf(L.cell.z, 0.f, g.resf.z - 1.f);
        const uint2 cw = __ldg(cells + (cx + cy * (uint32_t)g.res[0] + cz * (uint32_t)g.res[0] * (uint32_t)g.res[1]));
        steps++;
        if (KIND == 0) {
          L.b = cw.x;
          L.e = cw.y;
          L.st = ST_U_TESTED;
          if (L.e > L.b) return true;
          break;
        }
        if ((cw.y & kNotEmpty) && (cw.y & 0xFFFFFFu) == 0x010101u) {
          // a top cell with one leaf: its leaf DDA visits that leaf and then
          // always leaves the cell, so the range goes straight to the top step
          const uint2 range = __ldg(leaves + cw.x);
          steps++;
          L.b = range.x;
          L.e = range.y;
          L.st = ST_TOP_NEXT;
          if (L.e > L.b) return true;
          break;
        }
        if (cw.y & kNotEmpty) {
          const V3 rcp = L.rcp, org = L.org;
          const float te = L.tEntry;
          const V3 ent = add(org, divv(mk(te, te, te), rcp));
          const V3 cres = mk((float)(cw.y & 0xFFu), (float)((cw.y >> 8) & 0xFFu), (float)((cw.y >> 16) & 0xFFu));
          const V3 subRCP = mul(g.rcpTrav, cres);
          const V3 minB = add(mul(L.cell, g.cs), g.gmin);
          V3 sc;
          sc.x = floorf((ent.x - minB.x) * subRCP.x);
          sc.y = floorf((ent.y - minB.y) * subRCP.y);
          sc.z = floorf((ent.z - minB.z) * subRCP.z);
          const V3 scs = divv(mk(1.f, 1.f, 1.f), subRCP);
          sc = vmin(sub(cres, mk(1.f, 1.f, 1.f)), vmax(sc, mk(0.f, 0.f, 0.f)));
          const V3 tmp = mk(rcp.x > 0.f ? 1.f : 0.f, rcp.y > 0.f ? 1.f : 0.f, rcp.z > 0.f ? 1.f : 0.f);
          L.sMax.x = ((sc.x + tmp.x) * scs.x + minB.x - org.x) * rcp.x;
          L.sMax.y = ((sc.y + tmp.y) * scs.y + minB.y - org.y) * rcp.y;
          L.sMax.z = ((sc.z + tmp.z) * scs.z + minB.z - org.z) * rcp.z;
          L.sc = sc;
          L.scs = scs;
          L.cres = cres;
          L.lb = cw.x;
          L.vis2 = 0;
          L.st = ST_LEAF;
        } else {
          L.st = ST_TOP_NEXT;
        }
        break;
      }
      case ST_LEAF: {
        // runs of empty leaf cells are walked here, each with the step of
        // ST_LEAF_TESTED (nothing was tested, so its any-hit exit cannot fire)
        // An empty leaf of a two-level grid built here holds [D, D), D its
        // distance to the nearest non-empty leaf: the next D - 1 cells of the
        // walk are empty too and are stepped through without fetching.
        const float tb = L.tbest;
        const int cap2 = (int)L.cres.x + (int)L.cres.y + (int)L.cres.z + 3;
        uint32_t skip = 0;
        while (true) {
          L.vis2++;
          steps++;
          if (skip == 0) {
            const uint32_t li = L.lb + (uint32_t)(L.sc.x + L.cres.x * L.sc.y + L.cres.x * L.cres.y * L.sc.z);
            const uint2 range = __ldg(leaves + li);
            if (range.y > range.x) {
              L.b = range.x;
              L.e = range.y;
              L.st = ST_LEAF_TESTED;
              return true;
            }
            skip = range.x > 0u ? range.x - 1u : 0u;
          } else {
            --skip;
          }
          if (!(tb > L.sMax.x || tb > L.sMax.y || tb > L.sMax.z)) {
            L.st = ST_TOP_NEXT;
            break;
          }
          const int d = min_dim(L.sMax);
          const float rd = sel(d, L.rcp);
          bump(L.sc, d, rd > 0.f ? 1.f : -1.f);
          bump(L.sMax, d, sel(d, L.scs) * fabsf(rd));
          const float cd = sel(d, L.sc);
          const bool v2 = !(fabsf(cd - sel(d, L.cres)) < 0.1f || fabsf(cd + 1.f) < 0.1f);
          if (!(v2 && L.vis2 < cap2)) {
            L.st = ST_TOP_NEXT;
            break;
          }
        }
        break;
      }
      case ST_LEAF_TESTED: {
        if ((ANY || L.anyhit) && L.best != kMiss) {
          L.st = ST_DONE;
          return false;
        }
        const float tb = L.tbest;
        bool v2 = tb > L.sMax.x || tb > L.sMax.y || tb > L.sMax.z;
        if (!v2) {
          L.st = ST_TOP_NEXT;
          break;
        }
        const int d = min_dim(L.sMax);
        const float rd = sel(d, L.rcp);
        bump(L.sc, d, rd > 0.f ? 1.f : -1.f);
        bump(L.sMax, d, sel(d, L.scs) * fabsf(rd));
        const float cd = sel(d, L.sc);
        v2 = !(fabsf(cd - sel(d, L.cres)) < 0.1f || fabsf(cd + 1.f) < 0.1f);
        const int cap2 = (int)L.cres.x + (int)L.cres.y + (int)L.cres.z + 3;
        L.st = (v2 && L.vis2 < cap2) ? ST_LEAF : ST_TOP_NEXT;
        break;
      }
      case ST_U_TESTED:
      case ST_TOP_NEXT: {
        if ((ANY || L.anyhit) && L.best != kMiss) {
          L.st = ST_DONE;
          return false;
        }
        const float tb = L.tbest;
        bool valid = tb > L.tMax.x || tb > L.tMax.y || tb > L.tMax.z;
        if (!valid) {
          L.st = ST_DONE;
          return false;
        }
        const int d = min_dim(L.tMax);
        if (KIND == 1) L.tEntry = sel(d, L.tMax);
        const float rd = sel(d, L.rcp);
        bump(L.cell, d, rd > 0.f ? 1.f : -1.f);
        bump(L.tMax, d, sel(d, g.cs) * fabsf(rd));
        const float cd = sel(d, L.cell);
        valid = !(fabsf(cd - sel(d, g.resf)) < 0.1f || fabsf(cd + 1.f) < 0.1f);
        L.st = (valid && L.vis < L.cap) ? ST_TOP : ST_DONE;
        if (L.st == ST_DONE) return false;
        break;
      }
      default:
        return false;
    }
  }
}

// ---- watertight test with a compile-time axis permutation ---------------------
// Component K of v; K == 3: component k, chosen at run time (one copy of the
// code for every axis permutation, for kernels whose rays take all six).
template <int K>
SHN_D float pget(V3 v, uint32_t k) {
  return K == 0 ? v.x : (K == 1 ? v.y : (K == 2 ? v.z : sel((int)k, v)));
}

template <int K>
SHN_D float cget(V3 v) {
  return K == 0 ? v.x : (K == 1 ? v.y : v.z);
}

// The test on vertices already translated by the ray origin.
template <int KX, int KY, int KZ>
SHN_D bool wt_test_t(V3 A, V3 B, V3 C, float Sx, float Sy, float Sz, float tmin, float tbest, float& t,
                     uint32_t perm) {
  const uint32_t kx = perm & 3u, ky = (perm >> 2) & 3u, kz = (perm >> 4) & 3u;
  const float Akz = pget<KZ>(A, kz), Bkz = pget<KZ>(B, kz), Ckz = pget<KZ>(C, kz);
  const float Ax = __fmaf_rn(-Sx, Akz, pget<KX>(A, kx));
  const float Ay = __fmaf_rn(-Sy, Akz, pget<KY>(A, ky));
  const float Bx = __fmaf_rn(-Sx, Bkz, pget<KX>(B, kx));
  const float By = __fmaf_rn(-Sy, Bkz, pget<KY>(B, ky));
  const float Cx = __fmaf_rn(-Sx, Ckz, pget<KX>(C, kx));
  const float Cy = __fmaf_rn(-Sy, Ckz, pget<KY>(C, ky));
  float U = __fmaf_rn(Cx, By, -(Cy * Bx));
  float V = __fmaf_rn(Ax, Cy, -(Ay * Cx));
  float W = __fmaf_rn(Bx, Ay, -(By * Ax));
  // "some edge function is exactly zero" and "the signs differ", written with
  // min/max (fminf/fmaxf skip a NaN operand exactly as the or-chains of
  // comparisons do, so the outcome is that of the generic wt_test)
  if (fminf(fminf(fabsf(U), fabsf(V)), fabsf(W)) == 0.f) {
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if (fminf(fminf(U, V), W) < 0.f && fmaxf(fmaxf(U, V), W) > 0.f) return false;
  const float det = U + V + W;
  if (det == 0.f) return false;
  const float T = __fmaf_rn(W, Sz * Ckz, __fmaf_rn(V, Sz * Bkz, U * (Sz * Akz)));
  const float tt = T / det;
  if (!(tt > tmin && tt < tbest)) return false;
  t = tt;
  return true;
}

template <int KX, int KY, int KZ>
SHN_D bool wt_test_p(V3 org, float Sx, float Sy, float Sz, float4 p0, float4 p1, float4 p2,
                     float tmin, float tbest, float& t, uint32_t perm) {
  return wt_test_t<KX, KY, KZ>(sub(f4v(p0), org), sub(f4v(p1), org), sub(f4v(p2), org), Sx, Sy, Sz, tmin,
                               tbest, t, perm);
}

// Whole warp tests references [b, e) against one (warp-uniform) ray.
// Closest: returns the packed argmin key (t bits << 32 | triangle id) in every
// lane, or ~0 when nothing beats tbest.  Any: returns a hit's key or ~0.  A
// lane's candidate must beat tbest strictly and may tie the lane's running
// minimum (the least (t, id) wins, as in test_range).
// L2 latency is covered by the other resident warps: the kernels that run
// this engine are limited to 64 registers (8 blocks of 128 threads per SM),
// which measured faster than staging the next chunk in registers or in
// shared memory (cp.async) at lower occupancy.
template <bool ANY, int KX, int KY, int KZ, bool IND>
SHN_D uint64_t warp_range_p(const Refs& G, V3 org, float Sx, float Sy, float Sz, float tbest,
                            uint32_t b, uint32_t e, uint32_t& tests, uint32_t perm) {
  const int lane = threadIdx.x & 31;
  uint64_t key = ~0ull;
  float tb = tbest;
  const float4* q0 = G.rv0 + b + lane;
  const float4* q1 = G.rv1 + b + lane;
  const float4* q2 = G.rv2 + b + lane;
  uint32_t tested_end = e;
  uint32_t base = b;
  if (!ANY) {
    // closest hit: two references per lane per step (independent tests in
    // flight); each lane keeps its least (t, triangle id), and the warp's
    // least key is the range's
    for (; base + 32 < e; base += 64, q0 += 64, q1 += 64, q2 += 64) {
      const uint32_t it = base + lane, it2 = it + 32;
      float4 a0, a1, a2;
      if (IND) {
        ref_load<IND>(G, it, a0, a1, a2);
      } else {
        a0 = __ldg(q0);
        a1 = __ldg(q1);
        a2 = __ldg(q2);
      }
      const bool has2 = it2 < e;
      float4 c0 = a0, c1 = a1, c2 = a2;
      if (has2) {
        if (IND) {
          ref_load<IND>(G, it2, c0, c1, c2);
        } else {
          c0 = __ldg(q0 + 32);
          c1 = __ldg(q1 + 32);
          c2 = __ldg(q2 + 32);
        }
      }
      float t;
      if (it < e && wt_test_p<KX, KY, KZ>(org, Sx, Sy, Sz, a0, a1, a2, kEps, key == ~0ull ? tb : next_up(tb), t, perm)) {
        const uint64_t c = ((uint64_t)__float_as_uint(t) << 32) | __float_as_uint(a0.w);
        if (c < key) {
          key = c;
          tb = t;
        }
      }
      if (has2 && wt_test_p<KX, KY, KZ>(org, Sx, Sy, Sz, c0, c1, c2, kEps, key == ~0ull ? tb : next_up(tb), t, perm)) {
        const uint64_t c = ((uint64_t)__float_as_uint(t) << 32) | __float_as_uint(c0.w);
        if (c < key) {
          key = c;
          tb = t;
        }
      }
    }
  }
  // any hit (stops after the first 32-reference chunk holding a hit), and the
  // last chunk of a closest-hit range
  for (; base < e; base += 32, q0 += 32, q1 += 32, q2 += 32) {
    const uint32_t it = base + lane;
    bool hit = false;
    if (it < e) {
      float4 p0, p1, p2;
      if (IND) {
        ref_load<IND>(G, it, p0, p1, p2);
      } else {
        p0 = __ldg(q0);
        p1 = __ldg(q1);
        p2 = __ldg(q2);
      }
      float t;
      if (wt_test_p<KX, KY, KZ>(org, Sx, Sy, Sz, p0, p1, p2, kEps, key == ~0ull ? tb : next_up(tb), t, perm)) {
        const uint64_t c = ((uint64_t)__float_as_uint(t) << 32) | __float_as_uint(p0.w);
        if (c < key) {
          key = c;
          tb = t;
        }
        hit = true;
      }
    }
    if (ANY && __any_sync(0xFFFFFFFFu, hit)) {
      tested_end = min(e, base + 32u);
      break;
    }
  }
  tests += tested_end - b;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, key, o);
    key = other < key ? other : key;
  }
  return key;
}

// warp_range_p on a grid with block boxes: the blocks of 32 references that
// overlap [b, e) are visited in order, 1024 at a time; a block whose box the
// ray's segment (0, best so far] cannot meet (box_meets), or whose 1024-block
// box it cannot meet, is skipped.  Every triangle the ray can hit below the
// bound is in a visited block, so the result is that of warp_range_p.  Closest
// hit takes two blocks per step (one reference of each per lane); any hit
// stops after the first block holding a hit.  tests counts the references
// tested.
template <bool ANY, int KX, int KY, int KZ>
SHN_D uint64_t warp_range_cull_p(const Refs& G, V3 org, V3 cr, float Sx, float Sy, float Sz, float tbest,
                                 uint32_t b, uint32_t e, uint32_t& tests, uint32_t perm) {
  const int lane = threadIdx.x & 31;
  uint64_t key = ~0ull;
  float tb = tbest;
  const uint32_t kb = b >> 5, ke = (e - 1) >> 5;
  uint32_t ntest = 0;
  bool done = false;
  for (uint32_t s = kb >> 5; s <= (ke >> 5) && !done; ++s) {
    uint64_t wk = key;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, wk, o);
      wk = other < wk ? other : wk;
    }
    const float tw = wk == ~0ull ? tbest : __uint_as_float((uint32_t)(wk >> 32));
    if (!box_meets(org, cr, __ldg(G.sbox + 2 * (size_t)s), __ldg(G.sbox + 2 * (size_t)s + 1), tw)) continue;
    const uint32_t k = 32u * s + lane;
    const bool need = k >= kb && k <= ke &&
                      box_meets(org, cr, __ldg(G.cbox + 2 * (size_t)k), __ldg(G.cbox + 2 * (size_t)k + 1), tw);
    uint32_t m = __ballot_sync(0xFFFFFFFFu, need);
    while (m) {
      const uint32_t k1 = 32u * s + (uint32_t)(__ffs(m) - 1);
      m &= m - 1;
      uint32_t k2 = ~0u;
      if (!ANY && m) {
        k2 = 32u * s + (uint32_t)(__ffs(m) - 1);
        m &= m - 1;
      }
      ntest += block_refs(k1, b, e) + (k2 != ~0u ? block_refs(k2, b, e) : 0u);
      const uint32_t it = 32u * k1 + lane, it2 = 32u * k2 + lane;
      const bool ok = it >= b && it < e;
      const bool ok2 = !ANY && k2 != ~0u && it2 >= b && it2 < e;
      bool hit = false;
      float t;
      if (ok) {
        const float4 p0 = __ldg(G.rv0 + it), p1 = __ldg(G.rv1 + it), p2 = __ldg(G.rv2 + it);
        if (wt_test_p<KX, KY, KZ>(org, Sx, Sy, Sz, p0, p1, p2, kEps, key == ~0ull ? tb : next_up(tb), t, perm)) {
          const uint64_t c = ((uint64_t)__float_as_uint(t) << 32) | __float_as_uint(p0.w);
          if (c < key) {
            key = c;
            tb = t;
          }
          hit = true;
        }
      }
      if (ok2) {
        const float4 p0 = __ldg(G.rv0 + it2), p1 = __ldg(G.rv1 + it2), p2 = __ldg(G.rv2 + it2);
        if (wt_test_p<KX, KY, KZ>(org, Sx, Sy, Sz, p0, p1, p2, kEps, key == ~0ull ? tb : next_up(tb), t, perm)) {
          const uint64_t c = ((uint64_t)__float_as_uint(t) << 32) | __float_as_uint(p0.w);
          if (c < key) {
            key = c;
            tb = t;
          }
        }
      }
      if (ANY && __any_sync(0xFFFFFFFFu, hit)) {
        done = true;
        break;
      }
    }
  }
  tests += ntest;
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    const uint64_t other = __shfl_xor_sync(0xFFFFFFFFu, key, o);
    key = other < key ? other : key;
  }
  return key;
}

template <bool ANY, int KX, int KY, int KZ, bool IND>
SHN_D uint64_t warp_range_q(const Refs& G, V3 org, V3 rcp, float Sx, float Sy, float Sz, float tbest,
                            uint32_t b, uint32_t e, uint32_t& tests, uint32_t perm) {
  if (!IND && G.cbox && e - b > kCullMin)
    return warp_range_cull_p<ANY, KX, KY, KZ>(G, org, cull_rcp(rcp), Sx, Sy, Sz, tbest, b, e, tests, perm);
  return warp_range_p<ANY, KX, KY, KZ, IND>(G, org, Sx, Sy, Sz, tbest, b, e, tests, perm);
}

template <bool ANY, bool IND>
SHN_D uint64_t warp_range(const Refs& G, uint32_t perm, V3 org, V3 rcp, float Sx, float Sy, float Sz,
                          float tbest, uint32_t b, uint32_t e, uint32_t& tests) {
  // any-hit kernels: one copy with the permutation chosen at run time
  if (ANY) return warp_range_q<ANY, 3, 3, 3, IND>(G, org, rcp, Sx, Sy, Sz, tbest, b, e, tests, perm);
  switch (perm) {
    case (1u | 2u << 2 | 0u << 4): return warp_range_q<ANY, 1, 2, 0, IND>(G, org, rcp, Sx, Sy, Sz, tbest, b, e, tests, perm);
    case (2u | 1u << 2 | 0u << 4): return warp_range_q<ANY, 2, 1, 0, IND>(G, org, rcp, Sx, Sy, Sz, tbest, b, e, tests, perm);
    case (2u | 0u << 2 | 1u << 4): return warp_range_q<ANY, 2, 0, 1, IND>(G, org, rcp, Sx, Sy, Sz, tbest, b, e, tests, perm);
    case (0u | 2u << 2 | 1u << 4): return warp_range_q<ANY, 0, 2, 1, IND>(G, org, rcp, Sx, Sy, Sz, tbest, b, e, tests, perm);
    case (0u | 1u << 2 | 2u << 4): return warp_range_q<ANY, 0, 1, 2, IND>(G, org, rcp, Sx, Sy, Sz, tbest, b, e, tests, perm);
    default:                        return warp_range_q<ANY, 1, 0, 2, IND>(G, org, rcp, Sx, Sy, Sz, tbest, b, e, tests, perm);
  }
}

// Several lanes wait on the same large range (same scene, same first
// reference, same axis permutation): each lane loads one reference of every
// 32-reference chunk once and tests it against each of those rays in turn,
// reading the ray's origin and shear from its parked state (a broadcast), so
// a chunk crosses L2 once for the group instead of once per ray.  Candidates
// of ray r go to gkey[r] (t bits << 32 | triangle id, ~0 = none) by atomicMin.
// A candidate must beat the ray's bound from earlier cells strictly and may
// tie the range's running minimum (bound = next float above it), so gkey[r]
// ends as the least (t, triangle id) of the range's candidates below the
// earlier bound -- what warp_range_p returns -- in whatever order the lanes'
// updates land.  An any-hit ray leaves after the first chunk holding a hit
// (gend[r] = end of that chunk), as in warp_range_p.  SAME: every ray of the
// group has the same origin (camera rays), so the vertices are translated
// once per chunk instead of once per ray (the same operations, the same bits).
template <int KX, int KY, int KZ, bool SAME, bool ANY>
SHN_D void group_range_p(const Refs& G, const LaneG* park, unsigned long long* gkey, uint32_t* gend,
                         uint32_t gmask, uint32_t b, uint32_t e, uint32_t perm) {
  // closest hit: two references per lane per chunk (64-reference chunks), so a
  // ray's parameters are read once per two tests; any hit: 32-reference chunks,
  // the granularity of warp_range_p's early exit
  constexpr uint32_t kStep = ANY ? 32u : 64u;
  const int lane = threadIdx.x & 31;
  uint32_t live = gmask;
  const float4* q0 = G.rv0 + b + lane;
  const float4* q1 = G.rv1 + b + lane;
  const float4* q2 = G.rv2 + b + lane;
  const V3 o0 = park[__ffs(gmask) - 1].org;
  for (uint32_t base = b; base < e && live; base += kStep, q0 += kStep, q1 += kStep, q2 += kStep) {
    const uint32_t it = base + lane, it2 = it + 32u;
    const bool ok = it < e, ok2 = !ANY && it2 < e;
    float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0, p2 = p0, c0 = p0, c1 = p0, c2 = p0;
    if (ok) {
      p0 = __ldg(q0);
      p1 = __ldg(q1);
      p2 = __ldg(q2);
    }
    if (ok2) {
      c0 = __ldg(q0 + 32);
      c1 = __ldg(q1 + 32);
      c2 = __ldg(q2 + 32);
    }
    V3 A, B, C, A2, B2, C2;
    if (SAME) {
      A = sub(f4v(p0), o0);
      B = sub(f4v(p1), o0);
      C = sub(f4v(p2), o0);
      if (!ANY) {
        A2 = sub(f4v(c0), o0);
        B2 = sub(f4v(c1), o0);
        C2 = sub(f4v(c2), o0);
      }
    }
    uint32_t m = live;
    while (m) {
      const int r = __ffs(m) - 1;
      m &= m - 1;
      const float4 ra = *reinterpret_cast<const float4*>(&park[r].org);  // org, Sx
      const float4 rb = *reinterpret_cast<const float4*>(&park[r].Sy);   // Sy, Sz, perm, tbest
      const unsigned long long k = *reinterpret_cast<volatile const unsigned long long*>(gkey + r);
      const float bound = k == ~0ull ? rb.w : __uint_as_float((uint32_t)(k >> 32) + 1u);
      float t;
      const bool hit =
          ok && (SAME ? wt_test_t<KX, KY, KZ>(A, B, C, ra.w, rb.x, rb.y, kEps, bound, t, perm)
                      : wt_test_p<KX, KY, KZ>(mk(ra.x, ra.y, ra.z), ra.w, rb.x, rb.y, p0, p1, p2, kEps, bound, t,
                                                 KX == 3 ? __float_as_uint(rb.z) : perm));
      unsigned long long cand = hit ? (((unsigned long long)__float_as_uint(t) << 32) | __float_as_uint(p0.w)) : ~0ull;
      if (!ANY) {
        float t2;
        const bool hit2 =
            ok2 && (SAME ? wt_test_t<KX, KY, KZ>(A2, B2, C2, ra.w, rb.x, rb.y, kEps, bound, t2, perm)
                         : wt_test_p<KX, KY, KZ>(mk(ra.x, ra.y, ra.z), ra.w, rb.x, rb.y, c0, c1, c2, kEps, bound,
                                                 t2, perm));
        if (hit2) {
          const unsigned long long c2k = ((unsigned long long)__float_as_uint(t2) << 32) | __float_as_uint(c0.w);
          cand = c2k < cand ? c2k : cand;
        }
      }
      if (cand != ~0ull) atomicMin(gkey + r, cand);
      if (ANY) {
        if (__any_sync(0xFFFFFFFFu, hit)) {
          live &= ~(1u << r);
          if (lane == 0) gend[r] = min(e, base + 32u);
        }
      }
    }
  }
  __syncwarp();
}

// group_range_p on a grid with block boxes: per 1024-reference super-block,
// each lane tests its own ray against the super-block's box; then each lane
// takes one block of the super-block and tests its box against every ray
// still in, giving per block the set of rays that must test it; a block is
// loaded once for those rays.  Skipped blocks hold no triangle a ray can hit
// below its bound, so the keys are those of group_range_p.  gend[r] = b +
// number of references ray r tested.
template <int KX, int KY, int KZ, bool SAME, bool ANY>
SHN_D void group_cull_p(const Refs& G, const LaneG* park, unsigned long long* gkey, uint32_t* gend,
                        uint32_t gmask, uint32_t b, uint32_t e, uint32_t perm) {
  const int lane = threadIdx.x & 31;
  uint32_t live = gmask;
  const uint32_t kb = b >> 5, ke = (e - 1) >> 5;
  const V3 o0 = park[__ffs(gmask) - 1].org;
  const bool mine = (gmask >> lane) & 1u;
  const V3 myo = park[lane].org;
  const V3 mycr = cull_rcp(park[lane].rcp);
  const float mytb0 = park[lane].tbest;
  uint32_t mycount = 0;
  for (uint32_t s = kb >> 5; s <= (ke >> 5) && live; ++s) {
    bool in = false;
    if (mine && ((live >> lane) & 1u)) {
      const unsigned long long k = *reinterpret_cast<volatile const unsigned long long*>(gkey + lane);
      const float tb = k == ~0ull ? mytb0 : __uint_as_float((uint32_t)(k >> 32));
      in = box_meets(myo, mycr, __ldg(G.sbox + 2 * (size_t)s), __ldg(G.sbox + 2 * (size_t)s + 1), tb);
    }
    const uint32_t rs = __ballot_sync(0xFFFFFFFFu, in);
    if (!rs) continue;
    const uint32_t kl = 32u * s + lane;
    const bool kval = kl >= kb && kl <= ke;
    float4 bmn = make_float4(0.f, 0.f, 0.f, 0.f), bmx = bmn;
    if (kval) {
      bmn = __ldg(G.cbox + 2 * (size_t)kl);
      bmx = __ldg(G.cbox + 2 * (size_t)kl + 1);
    }
    uint32_t need = 0;  // rays that must test block kl
    for (uint32_t m = rs; m; m &= m - 1) {
      const int r = __ffs(m) - 1;
      const unsigned long long k = *reinterpret_cast<volatile const unsigned long long*>(gkey + r);
      const float tb = k == ~0ull ? park[r].tbest : __uint_as_float((uint32_t)(k >> 32));
      if (kval && box_meets(park[r].org, cull_rcp(park[r].rcp), bmn, bmx, tb)) need |= 1u << r;
    }
    uint32_t U = __ballot_sync(0xFFFFFFFFu, need != 0u);
    while (U && live) {
      const int bl = __ffs(U) - 1;
      U &= U - 1;
      const uint32_t rays = __shfl_sync(0xFFFFFFFFu, need, bl) & live;
      if (!rays) continue;
      const uint32_t kk = 32u * s + (uint32_t)bl;
      if ((rays >> lane) & 1u) mycount += block_refs(kk, b, e);
      const uint32_t it = 32u * kk + lane;
      const bool ok = it >= b && it < e;
      float4 p0 = make_float4(0.f, 0.f, 0.f, 0.f), p1 = p0, p2 = p0;
      if (ok) {
        p0 = __ldg(G.rv0 + it);
        p1 = __ldg(G.rv1 + it);
        p2 = __ldg(G.rv2 + it);
      }
      V3 A, B, C;
      if (SAME) {
        A = sub(f4v(p0), o0);
        B = sub(f4v(p1), o0);
        C = sub(f4v(p2), o0);
      }
      for (uint32_t m = rays; m; m &= m - 1) {
        const int r = __ffs(m) - 1;
        const float4 ra = *reinterpret_cast<const float4*>(&park[r].org);  // org, Sx
        const float4 rb = *reinterpret_cast<const float4*>(&park[r].Sy);   // Sy, Sz, perm, tbest
        const unsigned long long k = *reinterpret_cast<volatile const unsigned long long*>(gkey + r);
        const float bound = k == ~0ull ? rb.w : __uint_as_float((uint32_t)(k >> 32) + 1u);
        float t;
        const bool hit =
            ok && (SAME ? wt_test_t<KX, KY, KZ>(A, B, C, ra.w, rb.x, rb.y, kEps, bound, t, perm)
                        : wt_test_p<KX, KY, KZ>(mk(ra.x, ra.y, ra.z), ra.w, rb.x, rb.y, p0, p1, p2, kEps, bound, t,
                                                 KX == 3 ? __float_as_uint(rb.z) : perm));
        if (hit) atomicMin(gkey + r, ((unsigned long long)__float_as_uint(t) << 32) | __float_as_uint(p0.w));
        if (ANY) {
          if (__any_sync(0xFFFFFFFFu, hit)) live &= ~(1u << r);
        }
      }
    }
  }
  if (mine) gend[lane] = b + mycount;
  __syncwarp();
}

template <int KX, int KY, int KZ, bool SAME, bool ANY>
SHN_D void group_range_q(const Refs& G, const LaneG* park, unsigned long long* gkey, uint32_t* gend,
                         uint32_t gmask, uint32_t b, uint32_t e, uint32_t perm) {
  if (G.cbox && e - b > kCullMin) group_cull_p<KX, KY, KZ, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm);
  else group_range_p<KX, KY, KZ, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm);
}

template <bool SAME, bool ANY>
SHN_D void group_range_s(const Refs& G, uint32_t perm, const LaneG* park, unsigned long long* gkey,
                         uint32_t* gend, uint32_t gmask, uint32_t b, uint32_t e) {
  if (ANY) {
    group_range_q<3, 3, 3, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm);
    return;
  }
  switch (perm) {
    case (1u | 2u << 2 | 0u << 4): group_range_q<1, 2, 0, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm); break;
    case (2u | 1u << 2 | 0u << 4): group_range_q<2, 1, 0, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm); break;
    case (2u | 0u << 2 | 1u << 4): group_range_q<2, 0, 1, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm); break;
    case (0u | 2u << 2 | 1u << 4): group_range_q<0, 2, 1, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm); break;
    case (0u | 1u << 2 | 2u << 4): group_range_q<0, 1, 2, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm); break;
    default:                        group_range_q<1, 0, 2, SAME, ANY>(G, park, gkey, gend, gmask, b, e, perm); break;
  }
}

// ANY: the kernel's rays are all any-hit (lanes with a per-ray any-hit flag in
// a closest-hit kernel never join a group).  SAME is used by closest-hit
// kernels only (camera rays share the eye); the any-hit kernels' rays start
// from per-pixel hit points.
template <bool ANY>
SHN_D void group_range(const Refs& G, uint32_t perm, const LaneG* park, unsigned long long* gkey,
                       uint32_t* gend, uint32_t gmask, uint32_t b, uint32_t e) {
  if (ANY) {
    group_range_s<false, true>(G, perm, park, gkey, gend, gmask, b, e);
    return;
  }
  // do all rays of the group share the first one's origin (bit for bit)?
  const V3 o0 = park[__ffs(gmask) - 1].org;
  bool same = true;
  for (uint32_t m = gmask; m; m &= m - 1) {
    const V3 o = park[__ffs(m) - 1].org;
    same = same && __float_as_uint(o.x) == __float_as_uint(o0.x) && __float_as_uint(o.y) == __float_as_uint(o0.y) &&
           __float_as_uint(o.z) == __float_as_uint(o0.z);
  }
  if (same) group_range_s<true, false>(G, perm, park, gkey, gend, gmask, b, e);
  else group_range_s<false, false>(G, perm, park, gkey, gend, gmask, b, e);
}

// Per-lane test of its own (small) range with the generic watertight test.
template <bool ANY, bool IND, class LT>
SHN_D void lane_range(const Refs& G, LT& L, uint32_t& tests) {
  const RayWT w = lane_ray(L);
  const float t0 = L.tbest;
  bool found = false;
  for (uint32_t it = L.b; it < L.e; ++it) {
    tests++;
    float4 p0, p1, p2;
    ref_load<IND>(G, it, p0, p1, p2);
    float t, u, v;
    if (wt_test(w, p0, p1, p2, kEps, found ? next_up(L.tbest) : t0, t, u, v)) {
      const uint32_t id = __float_as_uint(p0.w);
      if (!found || t < L.tbest || id < L.best) {
        L.tbest = t;
        L.best = id;
        found = true;
      }
      if (ANY || L.anyhit) return;
    }
  }
}

// Final hit record of a lane: triangle id and barycentrics of the best
// triangle, recomputed with the same arithmetic from the scene's record.
template <class LT>
SHN_D void lane_result(const Refs& G, const LT& L, Hit& h) {
  h.t = L.tbest;
  h.tri = kMiss;
  h.u = h.v = 0.f;
  if (L.best == kMiss) return;
  const float4* rec = G.src + 3 * (size_t)L.best;
  const float4 p0 = __ldg(rec);
  const float4 p1 = __ldg(rec + 1);
  const float4 p2 = __ldg(rec + 2);
  float t, u, v;
  wt_test(lane_ray(L), p0, p1, p2, kEps, INFINITY, t, u, v);
  h.tri = L.best;
  h.u = u;
  h.v = v;
}

// The warp loop.  acc gives the lane's grid (geometry, cells, leaves) by its
// scene id; G holds the reference-ordered triangle arrays shared by all
// scenes.  src(i, org, dir, tmax, scene) generates ray i; sink(i, hit, steps,
// tests) consumes its result.  n rays are taken from *counter (pre-zeroed).
// GROUP: lanes waiting on the same large range test it together
// (group_range); worth it for coherent rays (camera, AO, shadow segments).
// PACKET: the warp takes its next 32 rays only when all 32 lanes are idle,
// so a warp traces 32 consecutive rays (neighbouring pixels, or the samples
// of neighbouring hits) side by side from their start: their DDA walks stay
// in step, where lanes refilled one by one drift apart.  On the 1M-triangle
// cluster at 1920x1080 the camera kernel went from 5.24 to 2.22 ms and the AO
// kernel from 2.91 to 2.47 ms (identical results); lanes whose ray ends early
// wait for the warp's last ray instead of starting a new one.
template <int KIND, bool ANY, bool GROUP = true, bool PACKET = false, class Acc, class Src, class Sink>
SHN_D void warp_trace_acc(const Acc& acc, uint32_t n, uint32_t* counter, Src&& src, Sink&& sink) {
  using LaneT = typename std::conditional<GROUP, LaneG, Lane>::type;
  // grids without a reference-ordered triangle copy (batched scenes)
  constexpr bool IND = Acc::kIndirect;
  static_assert(!(GROUP && IND), "grouped range tests read the reference-ordered copy");
  __shared__ LaneT lane_park[kCoopBlock];
  __shared__ unsigned long long grp_key[kCoopBlock];
  __shared__ uint32_t grp_end[kCoopBlock];
  const int lane = threadIdx.x & 31;
  const uint32_t lt = (1u << lane) - 1u;
  LaneT L;
  L.st = ST_DONE;
  bool has = false;
  uint32_t rid = 0, steps = 0, tests = 0, scene = 0;
  bool pool_empty = false;
  while (true) {
    const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !has);
    if ((PACKET ? idle == 0xFFFFFFFFu : idle != 0u) && !pool_empty) {
      const uint32_t cnt = __popc(idle);
      uint32_t base = 0;
      if (lane == 0) base = atomicAdd(counter, cnt);
      base = __shfl_sync(0xFFFFFFFFu, base, 0);
      if (base + cnt >= n) pool_empty = true;
      if (!has) {
        const uint32_t r = base + __popc(idle & lt);
        if (r < n) {
          rid = r;
          has = true;
          steps = tests = 0;
          V3 o, d;
          float tmax;
          uint32_t anyhit = 0;
          src(r, o, d, tmax, scene, anyhit);
          lane_init<KIND>(acc.geom(scene), L, o, d, tmax);
          L.anyhit = anyhit;
        }
      }
    }
    bool pending = false;
    if (has) {
      pending = lane_advance<KIND, ANY>(acc.geom(scene), acc.cells(scene), acc.leaves(scene), L, steps);
      if (!pending) {
        Hit h;
        lane_result(acc.refs(scene), L, h);
        sink(rid, h, steps, tests, scene);
        has = false;
      }
    }
    const uint32_t pmask = __ballot_sync(0xFFFFFFFFu, pending);
    if (pmask == 0) {
      if (pool_empty && __ballot_sync(0xFFFFFFFFu, has) == 0) break;
      continue;
    }
    const bool big = pending && (L.e - L.b > kCoopThreshold);
    if (pending && !big) lane_range<ANY, IND>(acc.refs(scene), L, tests);
    uint32_t bmask = __ballot_sync(0xFFFFFFFFu, big);
    if (bmask) {
      // The lanes' traversal state waits in shared memory while the warp tests
      // the large ranges, so the test loops have the registers to themselves.
      const uint32_t wb = threadIdx.x & ~31u;
      LaneT* park = lane_park + wb;
      unsigned long long* gkey = grp_key + wb;
      uint32_t* gend = grp_end + wb;
      park[lane] = L;
      // lanes waiting on the same range: same scene and first reference (closest
      // hit: and the same axis permutation, a compile-time constant of the group
      // test; any hit: the test takes each ray's own permutation at run time, so
      // rays of any direction share the range's loads -- AO kernel on the
      // 1M-triangle cluster 2.46 -> 2.12 ms)
      const unsigned long long rkey = (big && (ANY || !L.anyhit))
                                          ? (((unsigned long long)scene << 38) | ((unsigned long long)(ANY ? 0u : L.perm) << 32) | L.b)
                                          : ~0ull - lane;
      const uint32_t same = GROUP ? __match_any_sync(0xFFFFFFFFu, rkey) : (1u << lane);
      if (GROUP) {
        gkey[lane] = ~0ull;
        gend[lane] = L.e;
      }
      __syncwarp();
      uint32_t grouped = 0;
      while (bmask) {
        const int j = __ffs(bmask) - 1;
        const uint32_t gm = __shfl_sync(0xFFFFFFFFu, same, j) & bmask;
        bmask &= ~gm;
        const LaneT& Lj = park[j];
        const uint32_t sj = __shfl_sync(0xFFFFFFFFu, scene, j);
        const Refs R = acc.refs(sj);
        if constexpr (GROUP) {
          if (gm & (gm - 1)) {
            grouped |= gm;
            group_range<ANY>(R, Lj.perm, park, gkey, gend, gm, Lj.b, Lj.e);
            continue;
          }
        }
        const V3 org = Lj.org;
        const float Sx = Lj.Sx, Sy = Lj.Sy, Sz = Lj.Sz;
        const uint32_t perm = Lj.perm;
        const float tb = Lj.tbest;
        const uint32_t b = Lj.b, e = Lj.e;
        const uint32_t aj = Lj.anyhit;
        uint32_t wt = 0;
        const V3 rcp = Lj.rcp;
        const uint64_t key = (ANY || aj) ? warp_range<true, IND>(R, perm, org, rcp, Sx, Sy, Sz, tb, b, e, wt)
                                         : warp_range<false, IND>(R, perm, org, rcp, Sx, Sy, Sz, tb, b, e, wt);
        if (lane == j) {
          tests += wt;
          if (key != ~0ull) {
            park[j].tbest = __uint_as_float((uint32_t)(key >> 32));
            park[j].best = (uint32_t)key;
          }
        }
        __syncwarp();
      }
      if (GROUP && ((grouped >> lane) & 1u)) {
        tests += gend[lane] - park[lane].b;
        const unsigned long long k = gkey[lane];
        if (k != ~0ull) {
          park[lane].tbest = __uint_as_float((uint32_t)(k >> 32));
          park[lane].best = (uint32_t)k;
        }
      }
      __syncwarp();
      L = park[lane];
      __syncwarp();
    }
  }
}

// Grid access of a lane: the single-grid kernels use one GridView for every lane.
struct OneGrid {
  static constexpr bool kIndirect = false;
  const GridView* G;
  SHN_D const Geom& geom(uint32_t) const { return G->g; }
  SHN_D const uint2* cells(uint32_t) const { return G->cells; }
  SHN_D const uint2* leaves(uint32_t) const { return G->leaves; }
  SHN_D Refs refs(uint32_t) const { return refs_of(*G); }
};

template <int KIND, bool ANY, bool PACKET = false, class Src, class Sink>
SHN_D void warp_trace(const GridView& G, uint32_t n, uint32_t* counter, Src&& src, Sink&& sink) {
  warp_trace_acc<KIND, ANY, true, PACKET>(
      OneGrid{&G}, n, counter,
      [&](uint32_t i, V3& o, V3& d, float& tmax, uint32_t& scene, uint32_t&) {
        scene = 0;
        src(i, o, d, tmax);
      },
      [&](uint32_t i, const Hit& h, uint32_t steps, uint32_t tests, uint32_t) { sink(i, h, steps, tests); });
}

}  // namespace shn
