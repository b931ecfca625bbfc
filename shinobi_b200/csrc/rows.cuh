// Triangle -> cell pair generation by rows, warp-cooperative.
//
// A "unit" is one triangle against a regular lattice of cells: the top grid
// (countRefs / buildUnsortedGrid, src/Control/Algorithm/FastBuildKernels.h:31-215)
// or the leaf grid of one top cell (countLeafLevelRefs / writeLeafLevelRefs,
// src/Control/Algorithm/TwoLevelBuildKernels.h:129-455).  Its candidate cells
// are the index box [lo, lo + span) of the triangle's bounding box; when the
// box spans two or more cells on every axis a candidate is kept only if the
// plane-distance test passes at the cell centre.
//
// Cell centres.  As in the reference, the centres along each axis are
// accumulated from the first candidate cell: c(lo - 1) = ((lo*s + o) + s/2) - s,
// then c(i + 1) = c(i) + s, in FP32 (FastBuildKernels.h:144-164,
// TwoLevelBuildKernels.h:396-420).  Each axis restarts its sequence for every
// row of the enclosing loops, so the centre of index i along an axis depends
// on i and lo only.
//
// Row intervals.  Fix the two indices of a row and let i run along the third
// axis r.  Adding a positive s to a float never decreases it, so the centre is
// non-decreasing in i, and the plane distance
//   d = ((c0 - a0)*n0 + (c1 - a1)*n1) + (c2 - a2)*n2
// is monotone in i (direction = sign of n_r; every IEEE operation is
// monotone), and the test
//   |n_k * d| <= s_k/2 + eps  for k = 0, 1, 2
// holds on an interval of d values that contains 0.  The cells of the row
// that pass are therefore one interval of i, and every cell before it fails
// on one side of the plane and every cell after it on the other.  The row's
// interval is found by walking the accumulated centres from lo: a
// real-arithmetic estimate says how far the walk may go by additions alone
// (one test confirms that the cell before the estimate still fails on the
// near side; if not, the walk restarts from lo and tests every cell), then
// cells are tested until the first one on the far side.  The result is
// bit-identical to testing every candidate (the oracle does the latter).
//
// Work is balanced across the 32 lanes of a warp: the rows of 32 units are
// flattened and processed 32 at a time, and the emitted pairs of 32 rows are
// flattened again so that every store instruction writes 32 consecutive keys.
#pragma once
#include "common.cuh"

namespace shn {

constexpr uint32_t kWarpFull = 0xFFFFFFFFu;

// 27 words: an odd stride, so lanes reading different units from shared
// memory hit different banks.
struct Unit {
  float a[3];          // triangle vertex 0
  float n[3];          // unit normal (plane units)
  float s[3];          // lattice cell size
  float o[3];          // lattice origin: centres start at ((lo_k*s_k + o_k) + s_k*0.5) - s_k
  uint32_t lo[3];      // first candidate index per axis
  uint32_t span[3];    // number of candidate indices per axis (0 = none)
  uint32_t meta;       // bits 0-1: row axis r; bit 2: plane test applies
  uint32_t id;         // low key word (triangle id)
  uint32_t base;       // cell id of index (0, 0, 0)
  uint32_t stride[2];  // cell id = base + x + y*stride[0] + z*stride[1]
  float R;             // min_k (s_k/2 + eps)/|n_k|  (estimate only)
  float inv_nr;        // 1/n_r                      (estimate only)
  float inv_sr;        // 1/s_r                      (estimate only)
  uint32_t pad;
};

SHN_HD void unit_axes(int r, int& u, int& v) {
  u = r == 0 ? 1 : 0;
  v = r == 2 ? 1 : 2;
}

// Fills the derived fields; the row axis is the one with the most cells.
SHN_HD void unit_finish(Unit& U, bool plane) {
  int r = 0;
  if (U.span[1] > U.span[r]) r = 1;
  if (U.span[2] > U.span[r]) r = 2;
  U.meta = (uint32_t)r | (plane ? 4u : 0u);
  if (plane) {
    const float t0 = U.s[0] * 0.5f + kEps, t1 = U.s[1] * 0.5f + kEps, t2 = U.s[2] * 0.5f + kEps;
    U.R = fminf(t0 / fabsf(U.n[0]), fminf(t1 / fabsf(U.n[1]), t2 / fabsf(U.n[2])));
    const float nr = r == 0 ? U.n[0] : (r == 1 ? U.n[1] : U.n[2]);
    const float sr = r == 0 ? U.s[0] : (r == 1 ? U.s[1] : U.s[2]);
    U.inv_nr = 1.0f / nr;
    U.inv_sr = 1.0f / sr;
  } else {
    U.R = 0.f;
    U.inv_nr = 0.f;
    U.inv_sr = 0.f;
  }
  U.pad = 0u;
}

SHN_HD uint32_t unit_rows(const Unit& U) {
  const uint32_t r = U.meta & 3u;
  return r == 0u ? U.span[1] * U.span[2] : (r == 1u ? U.span[0] * U.span[2] : U.span[0] * U.span[1]);
}

SHN_HD uint32_t unit_cells(const Unit& U) { return U.span[0] * U.span[1] * U.span[2]; }

// Accumulated centre of index i >= lo_k along axis k (see the header).
SHN_HD float acc_centre(const Unit& U, int k, uint32_t i) {
  const float s = U.s[k];
  float c = (((float)U.lo[k] * s + U.o[k]) + s * 0.5f) - s;
  for (uint32_t q = U.lo[k]; q <= i; ++q) c += s;
  return c;
}

// (c_k(i) - a_k) * n_k
SHN_HD float unit_term(const Unit& U, int k, uint32_t i) { return (acc_centre(U, k, i) - U.a[k]) * U.n[k]; }

SHN_HD float combine(int r, float tr, float tu, float tv) {
  if (r == 0) return (tr + tu) + tv;
  if (r == 1) return (tu + tr) + tv;
  return (tu + tv) + tr;
}

// Class of the cell whose centre along the row axis is c:
// 0 = passes, -1 = fails with d < 0 (or NaN), +1 = fails with d > 0.
SHN_HD int class_at(const Unit& U, int r, float c, float tu, float tv) {
  const float d = combine(r, (c - U.a[r]) * U.n[r], tu, tv);
  const bool pass = fabsf(U.n[0] * d) <= U.s[0] * 0.5f + kEps &&
                    fabsf(U.n[1] * d) <= U.s[1] * 0.5f + kEps &&
                    fabsf(U.n[2] * d) <= U.s[2] * 0.5f + kEps;
  return pass ? 0 : (d > 0.f ? 1 : -1);
}

SHN_HD uint32_t clamp_index(float x, uint32_t lo, uint32_t hi1) {
  const float c = fminf(fmaxf(x, (float)lo), (float)hi1);  // NaN -> lo
  uint32_t i = (uint32_t)c;
  return i < lo ? lo : (i > hi1 ? hi1 : i);
}

// Passing cells [f, e) of row j of a plane unit.
SHN_HD void row_interval(const Unit& U, uint32_t j, uint32_t& f, uint32_t& e) {
  const int r = (int)(U.meta & 3u);
  int u, v;
  unit_axes(r, u, v);
  const uint32_t su = U.span[u];
  const uint32_t iu = U.lo[u] + j % su, iv = U.lo[v] + j / su;
  const float tu = unit_term(U, u, iu), tv = unit_term(U, v, iv);
  const uint32_t lo = U.lo[r], hi1 = U.lo[r] + U.span[r];  // [lo, hi1)
  const float s = U.s[r];
  const float c0 = ((((float)lo * s + U.o[r]) + s * 0.5f) - s) + s;  // centre of lo
  const float nr = U.n[r];
  if (!(nr > 0.f) && !(nr < 0.f)) {  // the class is the same along the whole row
    if (class_at(U, r, c0, tu, tv) == 0) { f = lo; e = hi1; }
    else { f = lo; e = lo; }
    return;
  }
  const int before = nr > 0.f ? -1 : 1;
  const int after = -before;
  // real-arithmetic estimate of the interval: |d| <= R
  const float S = tu + tv;
  const float ca = (U.a[r] - U.o[r]) - s * 0.5f;
  const float x1 = ((-U.R - S) * U.inv_nr + ca) * U.inv_sr;
  const float x2 = ((U.R - S) * U.inv_nr + ca) * U.inv_sr;
  const uint32_t xs = clamp_index(ceilf(fminf(x1, x2)) - 1.0f, lo, hi1);  // walk without tests up to here
  // f: first index whose class is not `before`
  uint32_t x = lo;
  float c = c0;
  if (xs > lo + 1) {
    while (x + 1 < xs) {  // centre of xs - 1
      c += s;
      ++x;
    }
    if (class_at(U, r, c, tu, tv) != before) {  // the estimate overshot: test every cell from lo
      x = lo;
      c = c0;
    } else {
      c += s;
      ++x;
    }
  }
  while (x < hi1 && class_at(U, r, c, tu, tv) == before) {
    c += s;
    ++x;
  }
  f = x;
  if (x == hi1) { e = x; return; }
  // e: first index >= f whose class is `after`; cells between pass
  const float cf = c;
  const uint32_t ys = clamp_index(floorf(fmaxf(x1, x2)), x, hi1);
  if (ys > x + 1) {
    while (x + 1 < ys) {  // centre of ys - 1
      c += s;
      ++x;
    }
    if (class_at(U, r, c, tu, tv) == after) {  // overshot: test every cell from f
      x = f;
      c = cf;
    }
  }
  while (x < hi1 && class_at(U, r, c, tu, tv) != after) {
    c += s;
    ++x;
  }
  e = x;
}

// Largest lane l with v_l <= q (v non-decreasing across lanes, v_0 <= q).
SHN_D int warp_search(uint32_t v, uint32_t q) {
  int o = 0;
#pragma unroll
  for (int s = 16; s > 0; s >>= 1) {
    const uint32_t c = __shfl_sync(kWarpFull, v, o + s);
    if (c <= q) o += s;
  }
  return o;
}

SHN_D uint32_t warp_incl_sum(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(kWarpFull, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

// Candidate count of every lane's unit (after the plane test).  su: the
// warp's 32 unit slots in shared memory, slot `lane` filled by this lane when
// `valid`; acc: 32 words of shared memory.
SHN_D uint32_t warp_count_units(Unit* su, uint32_t* acc, bool valid) {
  const int lane = threadIdx.x & 31;
  const bool plane = valid && (su[lane].meta & 4u);
  const uint32_t direct = (valid && !plane) ? unit_cells(su[lane]) : 0u;
  const uint32_t rows = plane ? unit_rows(su[lane]) : 0u;
  acc[lane] = 0u;
  const uint32_t incl = warp_incl_sum(rows);
  const uint32_t tot = __shfl_sync(kWarpFull, incl, 31);
  const uint32_t pre = incl - rows;
  __syncwarp();
  for (uint32_t j0 = 0; j0 < tot; j0 += 32) {
    const uint32_t j = j0 + lane;
    const int ow = warp_search(pre, j);
    const uint32_t opre = __shfl_sync(kWarpFull, pre, ow);
    uint32_t len = 0;
    if (j < tot) {
      uint32_t f, e;
      row_interval(su[ow], j - opre, f, e);
      len = e - f;
    }
    // segmented sum over lanes with the same owner (owners are non-decreasing)
    uint32_t sum = len;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const uint32_t y = __shfl_up_sync(kWarpFull, sum, o);
      const int w = __shfl_up_sync(kWarpFull, ow, o);
      if (lane >= o && w == ow) sum += y;
    }
    const int nxt = __shfl_down_sync(kWarpFull, ow, 1);
    if ((lane == 31 || nxt != ow) && sum) acc[ow] += sum;  // one writer per owner
    __syncwarp();
  }
  return direct + acc[lane];
}

// Writes the keys (cell << 32 | id) of the 32 lanes' units (slots filled as
// for warp_count_units), unit after unit and row after row, to keys[out ...].
// Stores beyond `cap` are dropped and flagged with kErrCapacity.  When shist
// is non-null, the hwidth-bit digits (cell >> hwidth*p) of every key, p <
// hpasses, are counted into shist[p * 512 + digit] (shared memory).
SHN_D void warp_emit_units(Unit* su, bool valid, uint32_t out, uint64_t* __restrict__ keys, uint32_t cap,
                           uint32_t* err, uint32_t* shist = nullptr, uint32_t hpasses = 0,
                           uint32_t hwidth = 8) {
  const int lane = threadIdx.x & 31;
  const uint32_t rows = valid ? unit_rows(su[lane]) : 0u;
  const uint32_t incl = warp_incl_sum(rows);
  const uint32_t tot = __shfl_sync(kWarpFull, incl, 31);
  const uint32_t pre = incl - rows;
  __syncwarp();
  for (uint32_t j0 = 0; j0 < tot; j0 += 32) {
    const uint32_t j = j0 + lane;
    const int ow = warp_search(pre, j);
    const uint32_t opre = __shfl_sync(kWarpFull, pre, ow);
    uint32_t len = 0, c0 = 0, st = 0, id = 0;
    if (j < tot) {
      const Unit& W = su[ow];
      const uint32_t jr = j - opre;
      const int r = (int)(W.meta & 3u);
      int u, v;
      unit_axes(r, u, v);
      uint32_t f, e;
      if (W.meta & 4u) {
        row_interval(W, jr, f, e);
      } else {
        f = W.lo[r];
        e = W.lo[r] + W.span[r];
      }
      len = e - f;
      const uint32_t iu = W.lo[u] + jr % W.span[u], iv = W.lo[v] + jr / W.span[u];
      uint32_t x, y, z;
      if (r == 0) { x = f; y = iu; z = iv; }
      else if (r == 1) { x = iu; y = f; z = iv; }
      else { x = iu; y = iv; z = f; }
      c0 = W.base + x + y * W.stride[0] + z * W.stride[1];
      st = r == 0 ? 1u : W.stride[r - 1];
      id = W.id;
    }
    const uint32_t pincl = warp_incl_sum(len);
    const uint32_t L = __shfl_sync(kWarpFull, pincl, 31);
    const uint32_t pos = pincl - len;
    for (uint32_t q0 = 0; q0 < L; q0 += 32) {
      const uint32_t q = q0 + lane;
      const int src = warp_search(pos, q);
      const uint32_t sc = __shfl_sync(kWarpFull, c0, src);
      const uint32_t ss = __shfl_sync(kWarpFull, st, src);
      const uint32_t sid = __shfl_sync(kWarpFull, id, src);
      const uint32_t sp = __shfl_sync(kWarpFull, pos, src);
      if (q < L) {
        const uint32_t o = out + q;
        const uint32_t cell = sc + (q - sp) * ss;
        if (o < cap) __stcs(keys + o, ((uint64_t)cell << 32) | sid);
        else atomicOr(err, kErrCapacity);
        // the cells are below 2^bits of the sort plan: the last pass's digit
        // needs no narrower mask
        const uint32_t hmask = (1u << hwidth) - 1u;
        for (uint32_t p = 0; p < hpasses; ++p) atomicAdd(shist + p * 512 + ((cell >> (hwidth * p)) & hmask), 1u);
      }
    }
    out += L;
    __syncwarp();
  }
}

}  // namespace shn
