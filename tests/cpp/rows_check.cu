// Host check of the row-interval search of the pair generation (rows.cuh):
// for random triangles against random lattices, the passing cells of every row
// found by row_interval equal those of testing every cell in the oracle's form
// (dot(centre - v0, n) and the per-axis half-cell comparison), and they are
// one contiguous interval.  Prints the counts; exits non-zero on a mismatch.
#include <cstdio>
#include <random>
#include <cstdlib>
#include "rows.cuh"
using namespace shn;
int main(int argc, char** argv) {
  std::mt19937 rng(1);
  std::uniform_real_distribution<float> U01(0.f, 1.f);
  long rows = 0, cells = 0, bad = 0, noncontig = 0;
  const int iters = argc > 1 ? atoi(argv[1]) : 20000;
  for (int it = 0; it < iters; ++it) {
    Unit u{};
    float sc = powf(10.f, -3.f + 2.f * U01(rng));
    float cs[3], o[3];
    for (int k = 0; k < 3; ++k) { cs[k] = (0.001f + U01(rng)) * 0.05f; o[k] = -1.f + 2.f * U01(rng); }
    V3 a = mk(o[0] + U01(rng), o[1] + U01(rng), o[2] + U01(rng));
    V3 b = add(a, mk((U01(rng) - .5f) * sc * 40, (U01(rng) - .5f) * sc * 40, (U01(rng) - .5f) * sc * 40));
    V3 c = add(a, mk((U01(rng) - .5f) * sc * 40, (U01(rng) - .5f) * sc * 40, (U01(rng) - .5f) * sc * 40));
    if (it % 7 == 0) c = add(a, mk(b.x - a.x, 0.f, 0.f));  // axis-aligned-ish
    V3 n = normalize(cross(sub(b, a), sub(c, a)));
    u.a[0] = a.x; u.a[1] = a.y; u.a[2] = a.z; u.n[0] = n.x; u.n[1] = n.y; u.n[2] = n.z;
    for (int k = 0; k < 3; ++k) {
      u.s[k] = cs[k]; u.o[k] = o[k];
      float mn = fminf(comp(a, k), fminf(comp(b, k), comp(c, k))), mx = fmaxf(comp(a, k), fmaxf(comp(b, k), comp(c, k)));
      int l = (int)((mn - o[k]) / cs[k]) - 1, h = (int)((mx - o[k]) / cs[k]) + 1;
      if (l < 0) l = 0;
      u.lo[k] = l; u.span[k] = (uint32_t)(h - l + 1);
      if (u.span[k] < 2) u.span[k] = 2;
      if (u.span[k] > 64) u.span[k] = 64;
    }
    unit_finish(u, true);
    const uint32_t R = unit_rows(u);
    const int r = u.meta & 3; int uu, vv; unit_axes(r, uu, vv);
    for (uint32_t j = 0; j < R; ++j) {
      uint32_t f, e; row_interval(u, j, f, e);
      const uint32_t iu = u.lo[uu] + j % u.span[uu], iv = u.lo[vv] + j / u.span[uu];
      const float tu = unit_term(u, uu, iu), tv = unit_term(u, vv, iv);
      // brute force in the oracle's form: centres accumulated from lo per
      // axis as the reference loops do, dot(sub(centre, a), n)
      float acc[3][64];
      for (int k = 0; k < 3; ++k) {
        float cc = (((float)u.lo[k] * u.s[k] + u.o[k]) + u.s[k] * 0.5f) - u.s[k];
        for (uint32_t q = 0; q < u.span[k] && q < 64; ++q) { cc += u.s[k]; acc[k][q] = cc; }
      }
      int first = -1, last = -1, cnt = 0;
      for (uint32_t i = u.lo[r]; i < u.lo[r] + u.span[r]; ++i) {
        uint32_t idx[3]; idx[r] = i; idx[uu] = iu; idx[vv] = iv;
        V3 cc = mk(acc[0][idx[0] - u.lo[0]], acc[1][idx[1] - u.lo[1]], acc[2][idx[2] - u.lo[2]]);
        const float d = dot(sub(cc, a), n);
        const V3 dist = muls(n, d);
        const bool pass = fabsf(dist.x) <= u.s[0] * 0.5f + kEps && fabsf(dist.y) <= u.s[1] * 0.5f + kEps &&
                          fabsf(dist.z) <= u.s[2] * 0.5f + kEps;
        if (pass) { if (first < 0) first = i; last = i; ++cnt; }
      }
      (void)tu; (void)tv;
      ++rows; cells += u.span[r];
      if (cnt && (uint32_t)(last - first + 1) != (uint32_t)cnt) ++noncontig;
      const bool ok = cnt == 0 ? (e == f) : (f == (uint32_t)first && e == (uint32_t)last + 1);
      if (!ok) { if (bad < 5) printf("mismatch it=%d j=%u got [%u,%u) want [%d,%d] cnt=%d\n", it, j, f, e, first, last, cnt); ++bad; }
    }
  }
  printf("rows %ld cells %ld mismatches %ld noncontiguous %ld\n", rows, cells, bad, noncontig);
  return bad != 0;
}
