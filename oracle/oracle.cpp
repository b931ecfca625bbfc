// Oracle: CPU restatement of Shinobi's grid build, 3D-DDA traversal and
// ray generation, used ONLY as the checker by tests/, the smoke check and
// the bench's CPU-baseline leg.  It is not part of the product and the
// product never links it.
//
// Every routine states the reference file:line it restates (paths are
// relative to the jckarter/shinobi tree).  Floating point follows the
// reference's operation order exactly; the library is compiled with
// -ffp-contract=off so no multiply-add is fused, which makes every result
// reproducible bit for bit by the CUDA kernels (compiled with -fmad=false).
//
// Documented, deliberate deviations from the reference (shared with the
// CUDA path, so both compute the same canonical result):
//  * pairs are ordered by (cell, tri); the reference order inside a cell is
//    whatever its shared-memory atomicAdd produced
//    (src/Control/Algorithm/FastBuildKernels.h:135);
//  * candidate cells rejected by the plane test are not emitted at all, so
//    no sentinel pairs reach the sorted arrays or indices[]
//    (reference: src/Control/Algorithm/FastBuildKernels.h:185-192);
//  * normals use 1/sqrtf instead of rsqrtf, divisions are IEEE instead of
//    __fdividef;
//  * leaf resolution is floor(cbrt(cs_a^3 * lambda * refs / V)) evaluated
//    exactly (largest r with r^3 <= q in double) and clamped to [1,255]
//    (reference: powf(..., 0.3333333f) on the device with 8-bit wrap,
//    src/Control/Algorithm/TwoLevelBuildKernels.h:48-81,
//    src/Control/Structure/TwoLevelGrid.hpp:88-101);
//  * ray-triangle test is the watertight test of Woop, Benthin and Wald
//    (JCGT 2013) instead of Moller-Trumbore
//    (src/Intersector/SimpleIntersector.hpp:38-124);
//  * DDA loops carry a step cap of res.x+res.y+res.z+3 (a legitimate ray
//    visits at most res.x+res.y+res.z-2 cells) so a NaN state cannot loop.
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {
#include "oracle.h"
}

namespace {

const float kEps = 0.00001f;  // src/CUDAStdAfx.h:96
const uint32_t kMiss = 0xFFFFFFFFu;

struct V3 {
  float x, y, z;
};
inline V3 mk(float x, float y, float z) { return V3{x, y, z}; }
inline V3 add(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
inline V3 sub(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
inline V3 mul(V3 a, V3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
inline V3 divv(V3 a, V3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
inline V3 muls(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
inline float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline V3 cross(V3 a, V3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
inline V3 normalize(V3 a) {
  float r = 1.0f / sqrtf(dot(a, a));
  return muls(a, r);
}
inline float& at(V3& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
inline float at(const V3& v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
inline V3 vmin(V3 a, V3 b) { return mk(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
inline V3 vmax(V3 a, V3 b) { return mk(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }

struct Tri {
  V3 v[3];
};

inline Tri load_tri(const float* vtx, const uint32_t* idx, uint32_t t) {
  Tri r;
  for (int k = 0; k < 3; ++k) {
    const float* p = vtx + 3 * (size_t)idx[3 * (size_t)t + k];
    r.v[k] = mk(p[0], p[1], p[2]);
  }
  return r;
}

// BBox::empty + extend x3 (src/Primitive/BBox.hpp:78-82, 109-119).
inline void tri_bounds(const Tri& t, V3& bmin, V3& bmax) {
  bmin = mk(FLT_MAX, FLT_MAX, FLT_MAX);
  bmax = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  for (int k = 0; k < 3; ++k) {
    bmin = vmin(bmin, t.v[k]);
    bmax = vmax(bmax, t.v[k]);
  }
}

struct Geom {
  V3 gmin, gmax;
  int res[3];
  V3 resf;
  V3 cs;        // (max-min)/res  (SimpleGrid::getCellSize, SimpleGrid.h:98-101)
  V3 rcpBuild;  // 1/cs          (FastSimpleGridBuilder.h:114-117)
  V3 rcpTrav;   // res/(max-min) (SimpleGrid::getCellSizeRCP, SimpleGrid.h:103-106)
};

Geom make_geom(const float b[6], const int res[3]) {
  Geom g;
  g.gmin = mk(b[0], b[1], b[2]);
  g.gmax = mk(b[3], b[4], b[5]);
  for (int i = 0; i < 3; ++i) g.res[i] = res[i];
  g.resf = mk((float)res[0], (float)res[1], (float)res[2]);
  V3 diag = sub(g.gmax, g.gmin);
  g.cs = divv(diag, g.resf);
  g.rcpBuild = divv(mk(1.f, 1.f, 1.f), g.cs);
  g.rcpTrav = divv(g.resf, diag);
  return g;
}

// ---------------------------------------------------------------------------
// Cell centres for the plane test, as the reference computes them: along each
// axis the centre of the first candidate cell is (lo*s + o) + s/2, the loop
// starts one cell before it and adds "+= cellSize" per cell
// (src/Control/Algorithm/FastBuildKernels.h:144-164,
// src/Control/Algorithm/TwoLevelBuildKernels.h:396-420).
inline void accumulated_centres(uint32_t lo, uint32_t hi, float s, float o, float half, std::vector<float>& out) {
  out.resize(hi - lo + 1);
  float c = (((float)lo * s + o) + half) - s;
  for (uint32_t i = lo; i <= hi; ++i) {
    c += s;
    out[i - lo] = c;
  }
}

// The same centre computed directly per cell, (i*s + o) + s/2: an earlier
// canonical form of this build, kept to count how far it was from the
// reference's (kDirectCentres).
inline float lattice_centre(uint32_t i, float s, float o) { return ((float)i * s + o) + s * 0.5f; }

// Variants, used only to count how far other arithmetic is from the build
// above (the counts are asserted by a test so that a change cannot move them
// silently):
//  kDirectCentres: centres computed per cell instead of accumulated;
//  kRefLeafPow: leaf resolution cs_a * powf(lambda * refs / V, 0.3333333f)
//    truncated, as countLeafLevelCells evaluates it (host powf), then clamped
//    to [1, 255] like the canonical rule (the reference's zero and 8-bit-wrap
//    cases are counted separately by orc_leaf_res_reference).
const int kDirectCentres = 1, kRefLeafPow = 2;
int g_ref_arith = 0;

// ---------------------------------------------------------------------------
// Candidate cell range of a triangle in a uniform grid.
// Restates countRefs / buildUnsortedGrid, src/Control/Algorithm/FastBuildKernels.h:47-69, 110-133.
inline void cell_range(const Tri& tri, const Geom& g, uint32_t lo[3], uint32_t hi[3]) {
  V3 bmin, bmax;
  tri_bounds(tri, bmin, bmax);
  V3 minf = vmax(mk(0.f, 0.f, 0.f), add(mul(sub(bmin, g.gmin), g.rcpBuild), mk(-kEps, -kEps, -kEps)));
  V3 maxf = vmin(sub(g.resf, mk(1.f, 1.f, 1.f)), add(mul(sub(bmax, g.gmin), g.rcpBuild), mk(kEps, kEps, kEps)));
  lo[0] = (uint32_t)minf.x; lo[1] = (uint32_t)minf.y; lo[2] = (uint32_t)minf.z;
  hi[0] = (uint32_t)maxf.x; hi[1] = (uint32_t)maxf.y; hi[2] = (uint32_t)maxf.z;
}

// Separating-axis test of one triangle edge against the cell box (the axisTest
// of src/Control/Algorithm/BuildKernels.h:41-61): the triangle's projection
// p0/p1 onto the axis against the box's radius rad.
inline bool sat_axis(float a, float b, float fa, float fb, float v0a, float v0b, float v1a, float v1b, float ha,
                     float hb) {
  const float p0 = a * v0a + b * v0b;
  const float p1 = a * v1a + b * v1b;
  const float mn = fminf(p0, p1);
  const float mx = fmaxf(p0, p1);
  const float rad = fa * ha + fb * hb;
  return !(mn > rad + kEps || mx + kEps < -rad);
}

// The nine edge-cross-axis tests of the precise insertion (GridOperator with
// taPreciseInsertion, src/Control/Algorithm/BuildKernels.h:143-185), in the
// cell-centred frame: vertices minus the cell centre c, h = half cell size.
inline bool sat_edges(const Tri& tri, V3 c, V3 h) {
  const V3 v0 = sub(tri.v[0], c), v1 = sub(tri.v[1], c), v2 = sub(tri.v[2], c);
  const V3 e[3] = {sub(v1, v0), sub(v2, v1), sub(v0, v2)};
  bool ok = true;
  for (int k = 0; k < 3; ++k) {
    const V3 ed = e[k];
    const V3 fe = mk(fabsf(ed.x), fabsf(ed.y), fabsf(ed.z));
    // X axis: X01 for edges 0 and 1, X2 for edge 2
    if (k < 2) ok = ok && sat_axis(ed.z, -ed.y, fe.z, fe.y, v0.y, v0.z, v2.y, v2.z, h.y, h.z);
    else ok = ok && sat_axis(ed.z, -ed.y, fe.z, fe.y, v0.y, v0.z, v1.y, v1.z, h.y, h.z);
    // Y axis: Y02 for edges 0 and 1, Y1 for edge 2
    if (k < 2) ok = ok && sat_axis(-ed.z, ed.x, fe.z, fe.x, v0.x, v0.z, v2.x, v2.z, h.x, h.z);
    else ok = ok && sat_axis(-ed.z, ed.x, fe.z, fe.x, v0.x, v0.z, v1.x, v1.z, h.x, h.z);
    // Z axis: Z12 for edges 0 and 2, Z0 for edge 1
    if (k == 1) ok = ok && sat_axis(ed.y, -ed.x, fe.y, fe.x, v0.x, v0.y, v1.x, v1.y, h.x, h.y);
    else ok = ok && sat_axis(ed.y, -ed.x, fe.y, fe.x, v1.x, v1.y, v2.x, v2.y, h.x, h.y);
  }
  return ok;
}

// Visit the cells of one triangle in the reference's emission order (z, y, x)
// applying the plane-distance test when the bbox spans >= 2 cells on every axis.
// Restates buildUnsortedGrid, src/Control/Algorithm/FastBuildKernels.h:137-212;
// with sat set, the precise insertion of the reference's other builder adds
// the nine edge tests to the plane test (src/Control/Algorithm/BuildKernels.h:117-201).
template <class F>
inline void for_each_cell(const Tri& tri, const Geom& g, F&& emit, bool sat = false) {
  uint32_t lo[3], hi[3];
  cell_range(tri, g, lo, hi);
  const uint32_t rx = (uint32_t)g.resf.x;
  const uint32_t rxy = (uint32_t)(g.resf.x * g.resf.y);
  if (hi[0] - lo[0] > 0 && hi[1] - lo[1] > 0 && hi[2] - lo[2] > 0) {
    const V3 n = normalize(cross(sub(tri.v[1], tri.v[0]), sub(tri.v[2], tri.v[0])));
    const V3 half = muls(g.cs, 0.5f);
    const bool acc = (g_ref_arith & kDirectCentres) == 0;
    thread_local std::vector<float> ax, ay, az;
    if (acc) {
      accumulated_centres(lo[0], hi[0], g.cs.x, g.gmin.x, half.x, ax);
      accumulated_centres(lo[1], hi[1], g.cs.y, g.gmin.y, half.y, ay);
      accumulated_centres(lo[2], hi[2], g.cs.z, g.gmin.z, half.z, az);
    }
    for (uint32_t z = lo[2]; z <= hi[2]; ++z) {
      const float cz = acc ? az[z - lo[2]] : lattice_centre(z, g.cs.z, g.gmin.z);
      for (uint32_t y = lo[1]; y <= hi[1]; ++y) {
        const float cy = acc ? ay[y - lo[1]] : lattice_centre(y, g.cs.y, g.gmin.y);
        for (uint32_t x = lo[0]; x <= hi[0]; ++x) {
          const float cx = acc ? ax[x - lo[0]] : lattice_centre(x, g.cs.x, g.gmin.x);
          const float d = dot(sub(mk(cx, cy, cz), tri.v[0]), n);
          const V3 dist = muls(n, d);
          if ((!sat || sat_edges(tri, mk(cx, cy, cz), half)) && fabsf(dist.x) <= half.x + kEps &&
              fabsf(dist.y) <= half.y + kEps && fabsf(dist.z) <= half.z + kEps)
            emit(x + y * rx + z * rxy);
        }
      }
    }
  } else {
    for (uint32_t z = lo[2]; z <= hi[2]; ++z)
      for (uint32_t y = lo[1]; y <= hi[1]; ++y)
        for (uint32_t x = lo[0]; x <= hi[0]; ++x) emit(x + y * rx + z * rxy);
  }
}

// ---------------------------------------------------------------------------
// Two-level grid cell word, same bit layout as TwoLevelGridCell
// (src/Control/Structure/TwoLevelGrid.hpp:34-152): x = leaf begin,
// y = resX | resY<<8 | resZ<<16 | 0x40000000 (not empty).
const uint32_t kNotEmpty = 0x40000000u;

uint32_t largest_cube_root_floor(double q) {
  if (!(q > 0.0)) return 0;
  uint32_t lo = 0, hi = 256;  // invariant: lo^3 <= q, hi^3 > q (or hi = cap)
  if ((double)hi * (double)hi * (double)hi <= q) return hi;
  while (hi - lo > 1) {
    uint32_t mid = (lo + hi) / 2;
    double m = (double)mid;
    if (m * m * m <= q) lo = mid; else hi = mid;
  }
  return lo;
}

// Leaf resolution per axis.  Restates countLeafLevelCells,
// src/Control/Algorithm/TwoLevelBuildKernels.h:48-81, with the exact cube
// root and clamping described in the file header.
void leaf_res(const Geom& g, float lambda, uint32_t refs, uint32_t threshold, uint32_t out[3]) {
  if (refs <= threshold) {
    out[0] = out[1] = out[2] = 1;
    return;
  }
  if (g_ref_arith & kRefLeafPow) {
    const float vol = (g.cs.x * g.cs.y) * g.cs.z;
    const float magic = powf(lambda * (float)refs / vol, 0.3333333f);
    for (int a = 0; a < 3; ++a) {
      const float r = at(g.cs, a) * magic;
      const uint32_t ri = r >= 4294967296.f ? 0xFFFFFFFFu : (uint32_t)r;
      out[a] = std::min<uint32_t>(255u, std::max<uint32_t>(1u, ri));
    }
    return;
  }
  const double vol = ((double)g.cs.x * (double)g.cs.y) * (double)g.cs.z;
  const double lr = (double)lambda * (double)refs;
  for (int a = 0; a < 3; ++a) {
    const double c = (double)at(g.cs, a);
    const double q = (((c * c) * c) * lr) / vol;
    uint32_t r = largest_cube_root_floor(q);
    out[a] = std::min<uint32_t>(255u, std::max<uint32_t>(1u, r));
  }
}

// Candidate leaf cells of one (top cell, tri) pair in emission order.
// Restates countLeafLevelRefs / writeLeafLevelRefs,
// src/Control/Algorithm/TwoLevelBuildKernels.h:175-222, 327-451.
template <class F>
inline void for_each_leaf(const Tri& tri, const Geom& g, uint32_t topCell, uint32_t cellY,
                          uint32_t leafBegin, F&& emit) {
  const uint32_t rX = (uint32_t)g.res[0], rY = (uint32_t)g.res[1];
  const uint32_t tx = topCell % rX;
  const uint32_t ty = (topCell % (rX * rY)) / rX;
  const uint32_t tz = topCell / (rX * rY);
  V3 bmin, bmax;
  tri_bounds(tri, bmin, bmax);
  const V3 cres = mk((float)(cellY & 0xFF), (float)((cellY >> 8) & 0xFF), (float)((cellY >> 16) & 0xFF));
  V3 origin;
  origin.x = (float)tx * g.cs.x + g.gmin.x;
  origin.y = (float)ty * g.cs.y + g.gmin.y;
  origin.z = (float)tz * g.cs.z + g.gmin.z;
  const V3 subRCP = divv(cres, g.cs);
  const V3 minf = add(mul(sub(bmin, origin), subRCP), mk(-0.001f, -0.001f, -0.001f));
  const V3 maxf = add(mul(sub(bmax, origin), subRCP), mk(1.001f, 1.001f, 1.001f));
  int lo[3], hp[3];
  lo[0] = std::max(0, (int)minf.x); lo[1] = std::max(0, (int)minf.y); lo[2] = std::max(0, (int)minf.z);
  hp[0] = std::min((int)cres.x, (int)maxf.x);
  hp[1] = std::min((int)cres.y, (int)maxf.y);
  hp[2] = std::min((int)cres.z, (int)maxf.z);
  const uint32_t crx = (uint32_t)cres.x;
  const uint32_t crxy = (uint32_t)(cres.x * cres.y);
  if (hp[0] - lo[0] > 1 && hp[1] - lo[1] > 1 && hp[2] - lo[2] > 1) {
    const V3 n = normalize(cross(sub(tri.v[1], tri.v[0]), sub(tri.v[2], tri.v[0])));
    const V3 scs = divv(g.cs, cres);
    const bool acc = (g_ref_arith & kDirectCentres) == 0;
    thread_local std::vector<float> ax, ay, az;
    if (acc) {
      accumulated_centres((uint32_t)lo[0], (uint32_t)hp[0] - 1, scs.x, origin.x, scs.x * 0.5f, ax);
      accumulated_centres((uint32_t)lo[1], (uint32_t)hp[1] - 1, scs.y, origin.y, scs.y * 0.5f, ay);
      accumulated_centres((uint32_t)lo[2], (uint32_t)hp[2] - 1, scs.z, origin.z, scs.z * 0.5f, az);
    }
    for (int z = lo[2]; z < hp[2]; ++z) {
      const float cz = acc ? az[z - lo[2]] : lattice_centre((uint32_t)z, scs.z, origin.z);
      for (int y = lo[1]; y < hp[1]; ++y) {
        const float cy = acc ? ay[y - lo[1]] : lattice_centre((uint32_t)y, scs.y, origin.y);
        for (int x = lo[0]; x < hp[0]; ++x) {
          const float cx = acc ? ax[x - lo[0]] : lattice_centre((uint32_t)x, scs.x, origin.x);
          const float d = dot(sub(mk(cx, cy, cz), tri.v[0]), n);
          const V3 dist = muls(n, d);
          if (fabsf(dist.x) <= scs.x * 0.5f + kEps && fabsf(dist.y) <= scs.y * 0.5f + kEps &&
              fabsf(dist.z) <= scs.z * 0.5f + kEps)
            emit((uint32_t)x + (uint32_t)y * crx + (uint32_t)z * crxy + leafBegin);
        }
      }
    }
  } else {
    for (int z = lo[2]; z < hp[2]; ++z)
      for (int y = lo[1]; y < hp[1]; ++y)
        for (int x = lo[0]; x < hp[0]; ++x)
          emit((uint32_t)x + (uint32_t)y * crx + (uint32_t)z * crxy + leafBegin);
  }
}

}  // namespace

// ===========================================================================
// Grid handle
struct orc_grid {
  int kind;  // 0 uniform, 1 two-level
  Geom g;
  std::vector<uint32_t> cells;       // uniform: 2*C ranges; two-level: 2*C_top cell words
  std::vector<uint32_t> leaves;      // two-level: 2*L ranges
  std::vector<uint32_t> indices;     // tri id per reference
  std::vector<uint64_t> top_pairs;   // two-level: sorted (cell<<32|tri) top pairs
  std::vector<uint32_t> leaf_counts; // two-level: leaf cells per top cell
  std::vector<float> vtx;            // copy of the scene for traversal
  std::vector<uint32_t> idx;
};

extern "C" {

void orc_bounds(const float* vtx, const uint32_t* idx, uint32_t nt, float out[6]) {
  // src/Control/Algorithm/FastSimpleGridBuilder.h:73-79 (BBox::extend over face vertices)
  V3 bmin = mk(FLT_MAX, FLT_MAX, FLT_MAX), bmax = mk(-FLT_MAX, -FLT_MAX, -FLT_MAX);
  for (uint32_t t = 0; t < nt; ++t) {
    Tri tr = load_tri(vtx, idx, t);
    for (int k = 0; k < 3; ++k) {
      bmin = vmin(bmin, tr.v[k]);
      bmax = vmax(bmax, tr.v[k]);
    }
  }
  out[0] = bmin.x; out[1] = bmin.y; out[2] = bmin.z;
  out[3] = bmax.x; out[4] = bmax.y; out[5] = bmax.z;
}

// GridBuilder::computeResolution (src/Control/Algorithm/GridBuilder.h:41-62) and the
// two-level top rule (src/Control/Algorithm/FastTwoLevelGridBuilder.h:87-102):
// res = (int)(diag * powf(lambda*N/V, 0.3333333f)), then /divisor, then >= min_res.
// Each axis is additionally clamped to [1, 2048].
void orc_resolution(uint32_t nt, const float b[6], float lambda, int divisor, int min_res, int out[3]) {
  V3 diag = sub(mk(b[3], b[4], b[5]), mk(b[0], b[1], b[2]));
  const float volume = diag.x * diag.y * diag.z;
  const float magic = powf(lambda * (float)nt / volume, 0.3333333f);
  diag = muls(diag, magic);
  float d[3] = {diag.x, diag.y, diag.z};
  for (int a = 0; a < 3; ++a) {
    float v = d[a];
    int r = (v >= 2048.f || !(v == v)) ? 2048 : (int)v;
    if (divisor > 1) r = r / divisor;
    r = std::max(r, min_res);
    r = std::min(std::max(r, 1), 2048);
    out[a] = r;
  }
}

// ---------------------------------------------------------------------------
// SAH resolution search, SAHGridBuilder::computeResolution
// (src/Control/Algorithm/SAHGridBuilder.h:117-202): the window of resolutions
// from wlo to whi times the lambda estimate (each bound clamped to [1, 2048]),
// refs = sum over the triangles of their bounding-box cells (countRefs,
// src/Control/Algorithm/FastBuildKernels.h:31-86, summed exactly in 64 bits),
// cost = 0.85 refs cellArea / sceneArea + 0.15 (rx + ry + rz); the first
// least cost in z, y, x order wins.
static int sah_window_res(float v) {
  if (!(v == v) || v >= 2048.f) return 2048;
  return std::min(std::max((int)v, 1), 2048);
}

void orc_sah_window(uint32_t nt, const float b[6], float lambda, float wlo, float whi, int rmin[3], int rmax[3]) {
  V3 diag = sub(mk(b[3], b[4], b[5]), mk(b[0], b[1], b[2]));
  const float volume = diag.x * diag.y * diag.z;
  const float magic = powf(lambda * (float)nt / volume, 0.3333333f);
  diag = muls(diag, magic);
  for (int a = 0; a < 3; ++a) {
    rmin[a] = sah_window_res(wlo * at(diag, a));
    rmax[a] = std::max(rmin[a], sah_window_res(whi * at(diag, a)));
  }
}

uint64_t orc_sah_refs(const float* vtx, const uint32_t* idx, uint32_t nt, const float b[6], const int res[3]) {
  const Geom g = make_geom(b, res);
  uint64_t sum = 0;
  for (uint32_t t = 0; t < nt; ++t) {
    uint32_t lo[3], hi[3];
    cell_range(load_tri(vtx, idx, t), g, lo, hi);
    uint64_t p = 1;
    for (int a = 0; a < 3; ++a) p *= hi[a] >= lo[a] ? (uint64_t)(hi[a] - lo[a] + 1) : 0;
    sum += p;
  }
  return sum;
}

float orc_sah_cost(const float b[6], const int res[3], uint64_t refs) {
  const V3 bs = sub(mk(b[3], b[4], b[5]), mk(b[0], b[1], b[2]));
  const float scene_area = 2.f * (bs.x * bs.x + bs.y * bs.y + bs.z * bs.z);
  const V3 r = mk((float)res[0], (float)res[1], (float)res[2]);
  const V3 cs = divv(bs, r);
  const float cell_area = 2.f * (cs.x * cs.x + cs.y * cs.y + cs.z * cs.z);
  return 0.85f * (float)refs * cell_area / scene_area + 0.15f * (r.x + r.y + r.z);
}

void orc_sah_resolution(const float* vtx, const uint32_t* idx, uint32_t nt, const float b[6], float lambda,
                        float wlo, float whi, int res_out[3], float* cost_out, uint64_t* refs_out,
                        uint64_t* counts) {
  int rmin[3], rmax[3];
  orc_sah_window(nt, b, lambda, wlo, whi, rmin, rmax);
  const int n[3] = {rmax[0] - rmin[0] + 1, rmax[1] - rmin[1] + 1, rmax[2] - rmin[2] + 1};
  const int64_t N = (int64_t)n[0] * n[1] * n[2];
  std::vector<uint64_t> refs(N);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t i = 0; i < N; ++i) {
    const int res[3] = {rmin[0] + (int)(i % n[0]), rmin[1] + (int)((i / n[0]) % n[1]), rmin[2] + (int)(i / ((int64_t)n[0] * n[1]))};
    refs[i] = orc_sah_refs(vtx, idx, nt, b, res);
  }
  float best = FLT_MAX;
  for (int64_t i = 0; i < N; ++i) {
    const int res[3] = {rmin[0] + (int)(i % n[0]), rmin[1] + (int)((i / n[0]) % n[1]), rmin[2] + (int)(i / ((int64_t)n[0] * n[1]))};
    const float c = orc_sah_cost(b, res, refs[i]);
    if (c < best) {
      best = c;
      for (int a = 0; a < 3; ++a) res_out[a] = res[a];
      *cost_out = c;
      *refs_out = refs[i];
    }
  }
  if (counts) std::copy(refs.begin(), refs.end(), counts);
}

orc_grid* orc_build_uniform_ex(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                               const float bounds[6], const int res[3], int insertion) {
  orc_grid* G = new orc_grid();
  G->kind = 0;
  G->g = make_geom(bounds, res);
  G->vtx.assign(vtx, vtx + 3 * (size_t)nv);
  G->idx.assign(idx, idx + 3 * (size_t)nt);
  const size_t C = (size_t)res[0] * res[1] * res[2];
  std::vector<uint64_t> pairs;
  for (uint32_t t = 0; t < nt; ++t) {
    Tri tr = load_tri(vtx, idx, t);
    for_each_cell(tr, G->g, [&](uint32_t c) { pairs.push_back(((uint64_t)c << 32) | t); }, insertion == 1);
  }
  std::sort(pairs.begin(), pairs.end());  // == stable sort on the cell key (emission is tri ordered)
  G->cells.assign(2 * C, 0u);
  G->indices.resize(pairs.size());
  // prepareCellRanges, src/Control/Algorithm/FastBuildKernels.h:243-311
  for (size_t i = 0; i < pairs.size(); ++i) {
    uint32_t c = (uint32_t)(pairs[i] >> 32);
    if (i == 0 || (uint32_t)(pairs[i - 1] >> 32) != c) G->cells[2 * (size_t)c] = (uint32_t)i;
    if (i + 1 == pairs.size() || (uint32_t)(pairs[i + 1] >> 32) != c) G->cells[2 * (size_t)c + 1] = (uint32_t)(i + 1);
    G->indices[i] = (uint32_t)pairs[i];
  }
  G->top_pairs.swap(pairs);
  return G;
}

orc_grid* orc_build_uniform(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                            const float bounds[6], const int res[3]) {
  return orc_build_uniform_ex(vtx, nv, idx, nt, bounds, res, 0);
}

// insertion 1: the precise (SAT) insertion for the top grid; the leaf
// level keeps the plane test (the reference's two-level kernels have no other)
orc_grid* orc_build_two_level_ex(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                                 const float bounds[6], const int res[3], float lambda_leaf,
                                 uint32_t leaf_threshold, int insertion) {
  orc_grid* G = orc_build_uniform_ex(vtx, nv, idx, nt, bounds, res, insertion);
  G->kind = 1;
  const Geom& g = G->g;
  const size_t C = (size_t)res[0] * res[1] * res[2];
  std::vector<uint32_t> ranges;
  ranges.swap(G->cells);
  G->cells.assign(2 * C, 0u);
  G->leaf_counts.resize(C);
  // countLeafLevelCells + ExclusiveScan + prepareTopLevelCellRanges
  // (src/Control/Algorithm/TwoLevelBuildKernels.h:40-127,
  //  src/Control/Algorithm/FastTwoLevelGridBuilder.h:256-330)
  uint64_t L = 0;
  for (size_t c = 0; c < C; ++c) {
    const uint32_t refs = ranges[2 * c + 1] - ranges[2 * c];
    uint32_t r[3];
    leaf_res(g, lambda_leaf, refs, leaf_threshold, r);
    uint32_t y = (r[0] & 0xFF) | ((r[1] & 0xFF) << 8) | ((r[2] & 0xFF) << 16);
    if (refs > 0) y |= kNotEmpty;
    G->leaf_counts[c] = r[0] * r[1] * r[2];
    G->cells[2 * c] = (uint32_t)L;
    G->cells[2 * c + 1] = y;
    L += G->leaf_counts[c];
  }
  // countLeafLevelRefs / writeLeafLevelRefs / Sort / prepareLeafCellRanges
  // (src/Control/Algorithm/FastTwoLevelGridBuilder.h:345-531)
  std::vector<uint64_t> lp;
  for (size_t i = 0; i < G->top_pairs.size(); ++i) {
    const uint32_t c = (uint32_t)(G->top_pairs[i] >> 32);
    const uint32_t t = (uint32_t)G->top_pairs[i];
    Tri tr = load_tri(vtx, idx, t);
    for_each_leaf(tr, g, c, G->cells[2 * (size_t)c + 1], G->cells[2 * (size_t)c],
                  [&](uint32_t l) { lp.push_back(((uint64_t)l << 32) | t); });
  }
  std::sort(lp.begin(), lp.end());
  G->leaves.assign(2 * (size_t)L, 0u);
  G->indices.resize(lp.size());
  for (size_t i = 0; i < lp.size(); ++i) {
    uint32_t l = (uint32_t)(lp[i] >> 32);
    if (i == 0 || (uint32_t)(lp[i - 1] >> 32) != l) G->leaves[2 * (size_t)l] = (uint32_t)i;
    if (i + 1 == lp.size() || (uint32_t)(lp[i + 1] >> 32) != l) G->leaves[2 * (size_t)l + 1] = (uint32_t)(i + 1);
    G->indices[i] = (uint32_t)lp[i];
  }
  return G;
}

orc_grid* orc_build_two_level(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              const float bounds[6], const int res[3], float lambda_leaf,
                              uint32_t leaf_threshold) {
  return orc_build_two_level_ex(vtx, nv, idx, nt, bounds, res, lambda_leaf, leaf_threshold, 0);
}

// Wrap grid arrays built elsewhere (e.g. by the reference's host builder) so
// the DDA traversal can run over them.  kind 0: cells are [begin,end) ranges;
// kind 1: cells are TwoLevelGridCell words and leaves are ranges.
orc_grid* orc_grid_from_arrays(int kind, const float bounds[6], const int res[3],
                               const uint32_t* cells, const uint32_t* leaves, uint64_t nleaves,
                               const uint32_t* indices, uint64_t nrefs, const float* vtx,
                               uint32_t nv, const uint32_t* idx, uint32_t nt) {
  orc_grid* G = new orc_grid();
  G->kind = kind;
  G->g = make_geom(bounds, res);
  const size_t C = (size_t)res[0] * res[1] * res[2];
  G->cells.assign(cells, cells + 2 * C);
  if (kind == 1) G->leaves.assign(leaves, leaves + 2 * nleaves);
  G->indices.assign(indices, indices + nrefs);
  G->vtx.assign(vtx, vtx + 3 * (size_t)nv);
  G->idx.assign(idx, idx + 3 * (size_t)nt);
  return G;
}

void orc_grid_free(orc_grid* G) { delete G; }

void orc_set_reference_arithmetic(int flags) { g_ref_arith = flags; }

// The reference's leaf resolution of every top cell of a two-level grid
// exactly as countLeafLevelCells evaluates it on the host (powf, truncation,
// no clamping: src/Control/Algorithm/TwoLevelBuildKernels.h:48-81): out
// receives 3 uint32 per top cell (1,1,1 for cells of <= threshold refs).
void orc_leaf_res_reference(const orc_grid* G, float lambda, uint32_t threshold, uint32_t* out) {
  const Geom& g = G->g;
  const size_t C = (size_t)g.res[0] * g.res[1] * g.res[2];
  std::vector<uint32_t> refs(C, 0u);
  for (uint64_t k : G->top_pairs) ++refs[(size_t)(k >> 32)];
  const float vol = (g.cs.x * g.cs.y) * g.cs.z;
  for (size_t c = 0; c < C; ++c) {
    if (refs[c] <= threshold) {
      out[3 * c] = out[3 * c + 1] = out[3 * c + 2] = 1u;
      continue;
    }
    const float magic = powf(lambda * (float)refs[c] / vol, 0.3333333f);
    for (int a = 0; a < 3; ++a) {
      const float r = at(g.cs, a) * magic;
      out[3 * c + a] = r >= 4294967296.f ? 0xFFFFFFFFu : (uint32_t)r;
    }
  }
}

void orc_grid_info(const orc_grid* G, uint64_t out[8]) {
  out[0] = (uint64_t)G->kind;
  out[1] = (uint64_t)G->g.res[0] * G->g.res[1] * G->g.res[2];
  out[2] = G->indices.size();
  out[3] = G->leaves.size() / 2;
  out[4] = G->top_pairs.size();
  out[5] = (uint64_t)G->g.res[0];
  out[6] = (uint64_t)G->g.res[1];
  out[7] = (uint64_t)G->g.res[2];
}

const uint32_t* orc_grid_cells(const orc_grid* G) { return G->cells.data(); }
const uint32_t* orc_grid_leaves(const orc_grid* G) { return G->leaves.data(); }
const uint32_t* orc_grid_indices(const orc_grid* G) { return G->indices.data(); }
const uint64_t* orc_grid_top_pairs(const orc_grid* G) { return G->top_pairs.data(); }

}  // extern "C"

// ===========================================================================
// Traversal
namespace {

struct Ray {
  V3 org, dir;
};

// Watertight ray/triangle test (Woop, Benthin, Wald: "Watertight Ray/Triangle
// Intersection", JCGT 2(1), 2013).  Per-ray shear constants.
struct WT {
  int kx, ky, kz;
  float Sx, Sy, Sz;
};

inline WT wt_setup(V3 d) {
  WT w;
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  w.kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
  w.kx = w.kz + 1 == 3 ? 0 : w.kz + 1;
  w.ky = w.kx + 1 == 3 ? 0 : w.kx + 1;
  if (at(d, w.kz) < 0.f) std::swap(w.kx, w.ky);
  w.Sx = at(d, w.kx) / at(d, w.kz);
  w.Sy = at(d, w.ky) / at(d, w.kz);
  w.Sz = 1.0f / at(d, w.kz);
  return w;
}

// Returns true and updates t/u/v when the hit lies in (tmin, tbest).
inline bool wt_intersect(const WT& w, V3 org, const Tri& tri, float tmin, float tbest, float& t,
                         float& u, float& v) {
  const V3 A = sub(tri.v[0], org), B = sub(tri.v[1], org), C = sub(tri.v[2], org);
  // shear with one fused multiply-add per coordinate; edge functions as one
  // rounded product plus a fused multiply-add (fmaf is correctly rounded)
  const float Ax = fmaf(-w.Sx, at(A, w.kz), at(A, w.kx));
  const float Ay = fmaf(-w.Sy, at(A, w.kz), at(A, w.ky));
  const float Bx = fmaf(-w.Sx, at(B, w.kz), at(B, w.kx));
  const float By = fmaf(-w.Sy, at(B, w.kz), at(B, w.ky));
  const float Cx = fmaf(-w.Sx, at(C, w.kz), at(C, w.kx));
  const float Cy = fmaf(-w.Sy, at(C, w.kz), at(C, w.ky));
  float U = fmaf(Cx, By, -(Cy * Bx));
  float V = fmaf(Ax, Cy, -(Ay * Cx));
  float W = fmaf(Bx, Ay, -(By * Ax));
  if (U == 0.f || V == 0.f || W == 0.f) {
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if ((U < 0.f || V < 0.f || W < 0.f) && (U > 0.f || V > 0.f || W > 0.f)) return false;
  const float det = U + V + W;
  if (det == 0.f) return false;
  const float Az = w.Sz * at(A, w.kz);
  const float Bz = w.Sz * at(B, w.kz);
  const float Cz = w.Sz * at(C, w.kz);
  const float T = fmaf(W, Cz, fmaf(V, Bz, U * Az));
  const float tt = T / det;
  if (!(tt > tmin && tt < tbest)) return false;
  t = tt;
  u = V / det;
  v = W / det;
  return true;
}

struct Stats {
  uint64_t steps = 0, tests = 0;
};

struct Hit {
  float t;
  uint32_t ref;
  float u, v;
};

// Test all references of one cell range; any-hit returns on the first hit.
inline bool test_range(const orc_grid* G, const WT& w, V3 org, uint32_t b, uint32_t e, Hit& h,
                       bool any, Stats& st) {
  for (uint32_t it = b; it < e; ++it) {
    Tri tr = load_tri(G->vtx.data(), G->idx.data(), G->indices[it]);
    ++st.tests;
    float t, u, v;
    if (wt_intersect(w, org, tr, kEps, h.t, t, u, v)) {
      h.t = t; h.ref = it; h.u = u; h.v = v;
      if (any) return true;
    }
  }
  return false;
}

inline int min_dim(V3 t) { return (t.x < t.y) ? ((t.x < t.z) ? 0 : 2) : ((t.y < t.z) ? 1 : 2); }

inline float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }

// UniformGridTraverser::traverse / traverseInit / traverseCell,
// src/Control/Algorithm/SimpleGridTraverser.h:274-401.  Closest-hit keeps
// going while the best t exceeds the current cell's exit; any-hit stops at
// the first hit in (EPS, tmax).
void trace_uniform(const orc_grid* G, const Ray& r, Hit& h, bool any, Stats& st) {
  const Geom& g = G->g;
  const V3 rcp = divv(mk(1.f, 1.f, 1.f), r.dir);
  const WT w = wt_setup(r.dir);
  if (!(h.t > 0.f)) return;
  // BBox::fastClip, src/Primitive/BBox.hpp:60-75
  const V3 t1 = mul(sub(g.gmin, r.org), rcp);
  V3 t2 = mul(sub(g.gmax, r.org), rcp);
  const V3 tmn = vmin(t1, t2);
  t2 = vmax(t1, t2);
  const float tEntry = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
  const float tExit = fminf(fminf(t2.x, t2.y), t2.z);
  if (tExit <= tEntry || tExit < 0.f) return;
  const V3 entry = (tEntry >= 0.f) ? add(r.org, divv(mk(tEntry + kEps, tEntry + kEps, tEntry + kEps), rcp)) : r.org;
  V3 cell = mul(sub(entry, g.gmin), g.rcpTrav);
  cell = mk(floorf(cell.x), floorf(cell.y), floorf(cell.z));
  const V3 tmp = mk(rcp.x > 0.f ? 1.f : 0.f, rcp.y > 0.f ? 1.f : 0.f, rcp.z > 0.f ? 1.f : 0.f);
  V3 tMax = mul(sub(add(mul(add(cell, tmp), g.cs), g.gmin), r.org), rcp);
  bool valid = (cell.x != (rcp.x > 0.f ? (float)g.res[0] : -1.f)) &&
               (cell.y != (rcp.y > 0.f ? (float)g.res[1] : -1.f)) &&
               (cell.z != (rcp.z > 0.f ? (float)g.res[2] : -1.f));
  const int cap = g.res[0] + g.res[1] + g.res[2] + 3;
  for (int step = 0; valid && step < cap; ++step) {
    // tex3D clamps out-of-range coordinates; the lookup does the same.
    const uint32_t cx = (uint32_t)clampf(cell.x, 0.f, g.resf.x - 1.f);
    const uint32_t cy = (uint32_t)clampf(cell.y, 0.f, g.resf.y - 1.f);
    const uint32_t cz = (uint32_t)clampf(cell.z, 0.f, g.resf.z - 1.f);
    const size_t ci = cx + (size_t)cy * g.res[0] + (size_t)cz * g.res[0] * g.res[1];
    ++st.steps;
    if (test_range(G, w, r.org, G->cells[2 * ci], G->cells[2 * ci + 1], h, any, st)) return;
    valid = h.t > tMax.x || h.t > tMax.y || h.t > tMax.z;
    if (!valid) break;
    const int d = min_dim(tMax);
    at(cell, d) += at(rcp, d) > 0.f ? 1.f : -1.f;
    at(tMax, d) += at(g.cs, d) * fabsf(at(rcp, d));
    valid = !(fabsf(at(cell, d) - (float)g.res[d]) < 0.1f || fabsf(at(cell, d) + 1.f) < 0.1f);
  }
}

// TwoLevelGridTraverser::traverse / traverseInit / traverseMacroCell / traverseCell,
// src/Control/Algorithm/TwoLevelGridTraverser.h:445-671 (fastDivide -> IEEE division).
void trace_two_level(const orc_grid* G, const Ray& r, Hit& h, bool any, Stats& st) {
  const Geom& g = G->g;
  const V3 rcp = divv(mk(1.f, 1.f, 1.f), r.dir);
  const WT w = wt_setup(r.dir);
  if (!(h.t > 0.f)) return;
  const V3 t1 = mul(sub(g.gmin, r.org), rcp);
  V3 t2 = mul(sub(g.gmax, r.org), rcp);
  const V3 tmn = vmin(t1, t2);
  t2 = vmax(t1, t2);
  float tEntry = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
  const float tExit = fminf(fminf(t2.x, t2.y), t2.z);
  if (tExit <= tEntry || tExit < 0.f) return;
  tEntry = fmaxf(0.f, tEntry);
  const V3 entry = add(r.org, divv(mk(tEntry + kEps, tEntry + kEps, tEntry + kEps), rcp));
  V3 cell = mul(sub(entry, g.gmin), g.rcpTrav);
  cell = mk(floorf(cell.x), floorf(cell.y), floorf(cell.z));
  const V3 tmp = mk(rcp.x > 0.f ? 1.f : 0.f, rcp.y > 0.f ? 1.f : 0.f, rcp.z > 0.f ? 1.f : 0.f);
  V3 tMax = mul(sub(add(mul(add(cell, tmp), g.cs), g.gmin), r.org), rcp);
  bool valid = (cell.x != (rcp.x > 0.f ? (float)g.res[0] : -1.f)) &&
               (cell.y != (rcp.y > 0.f ? (float)g.res[1] : -1.f)) &&
               (cell.z != (rcp.z > 0.f ? (float)g.res[2] : -1.f));
  const int cap = g.res[0] + g.res[1] + g.res[2] + 3;
  for (int step = 0; valid && step < cap; ++step) {
    const uint32_t cx = (uint32_t)clampf(cell.x, 0.f, g.resf.x - 1.f);
    const uint32_t cy = (uint32_t)clampf(cell.y, 0.f, g.resf.y - 1.f);
    const uint32_t cz = (uint32_t)clampf(cell.z, 0.f, g.resf.z - 1.f);
    const size_t ci = cx + (size_t)cy * g.res[0] + (size_t)cz * g.res[0] * g.res[1];
    const uint32_t leafBegin = G->cells[2 * ci];
    const uint32_t cy_word = G->cells[2 * ci + 1];
    ++st.steps;
    if (cy_word & kNotEmpty) {
      const V3 ent = add(r.org, divv(mk(tEntry, tEntry, tEntry), rcp));
      const V3 cres = mk((float)(cy_word & 0xFF), (float)((cy_word >> 8) & 0xFF), (float)((cy_word >> 16) & 0xFF));
      const V3 subRCP = mul(g.rcpTrav, cres);
      const V3 minB = add(mul(cell, g.cs), g.gmin);
      V3 sc;
      sc.x = floorf((ent.x - minB.x) * subRCP.x);
      sc.y = floorf((ent.y - minB.y) * subRCP.y);
      sc.z = floorf((ent.z - minB.z) * subRCP.z);
      const V3 scs = divv(mk(1.f, 1.f, 1.f), subRCP);
      sc = vmin(sub(cres, mk(1.f, 1.f, 1.f)), vmax(sc, mk(0.f, 0.f, 0.f)));
      V3 sMax;
      sMax.x = ((sc.x + (rcp.x > 0.f ? 1.f : 0.f)) * scs.x + minB.x - r.org.x) * rcp.x;
      sMax.y = ((sc.y + (rcp.y > 0.f ? 1.f : 0.f)) * scs.y + minB.y - r.org.y) * rcp.y;
      sMax.z = ((sc.z + (rcp.z > 0.f ? 1.f : 0.f)) * scs.z + minB.z - r.org.z) * rcp.z;
      bool v2 = true;
      const int cap2 = (int)cres.x + (int)cres.y + (int)cres.z + 3;
      for (int s2 = 0; v2 && s2 < cap2; ++s2) {
        const uint32_t li = leafBegin + (uint32_t)(sc.x + cres.x * sc.y + cres.x * cres.y * sc.z);
        ++st.steps;
        if (test_range(G, w, r.org, G->leaves[2 * (size_t)li], G->leaves[2 * (size_t)li + 1], h, any, st))
          return;
        v2 = h.t > sMax.x || h.t > sMax.y || h.t > sMax.z;
        if (!v2) break;
        const int d = min_dim(sMax);
        at(sc, d) += at(rcp, d) > 0.f ? 1.f : -1.f;
        at(sMax, d) += at(scs, d) * fabsf(at(rcp, d));
        v2 = !(fabsf(at(sc, d) - at(cres, d)) < 0.1f || fabsf(at(sc, d) + 1.f) < 0.1f);
      }
    }
    valid = h.t > tMax.x || h.t > tMax.y || h.t > tMax.z;
    if (!valid) break;
    const int d = min_dim(tMax);
    tEntry = at(tMax, d);
    at(cell, d) += at(rcp, d) > 0.f ? 1.f : -1.f;
    at(tMax, d) += at(g.cs, d) * fabsf(at(rcp, d));
    valid = !(fabsf(at(cell, d) - (float)g.res[d]) < 0.1f || fabsf(at(cell, d) + 1.f) < 0.1f);
  }
}

inline void trace_one(const orc_grid* G, const Ray& r, Hit& h, bool any, Stats& st) {
  if (G->kind == 0) trace_uniform(G, r, h, any, st);
  else trace_two_level(G, r, h, any, st);
}

}  // namespace

extern "C" {

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

// Closest hit for SoA rays.  tmax may be NULL (FLT_MAX, as the primary ray
// generators return, src/Engine/RayGenerators.h:59,94).  Misses report
// tri = 0xFFFFFFFF and t = tmax.  stats (optional) receives {cell steps, tri tests}.
void orc_trace_closest(const orc_grid* G, const float* ox, const float* oy, const float* oz,
                       const float* dx, const float* dy, const float* dz, const float* tmax,
                       uint32_t n, uint32_t* tri, float* t, float* u, float* v, uint64_t* stats) {
  uint64_t S = 0, T = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : S, T)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    Ray r{mk(ox[i], oy[i], oz[i]), mk(dx[i], dy[i], dz[i])};
    Hit h{tmax ? tmax[i] : FLT_MAX, kMiss, 0.f, 0.f};
    Stats st;
    trace_one(G, r, h, false, st);
    tri[i] = h.ref == kMiss ? kMiss : G->indices[h.ref];
    t[i] = h.t;
    if (u) u[i] = h.u;
    if (v) v[i] = h.v;
    S += st.steps;
    T += st.tests;
  }
  if (stats) { stats[0] = S; stats[1] = T; }
}

// Any hit in (EPS, tmax): occluded[i] = 1 when the segment is blocked.
void orc_trace_any(const orc_grid* G, const float* ox, const float* oy, const float* oz,
                   const float* dx, const float* dy, const float* dz, const float* tmax, uint32_t n,
                   uint8_t* occluded, uint64_t* stats) {
  uint64_t S = 0, T = 0;
#pragma omp parallel for schedule(dynamic, 256) reduction(+ : S, T)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    Ray r{mk(ox[i], oy[i], oz[i]), mk(dx[i], dy[i], dz[i])};
    Hit h{tmax ? tmax[i] : FLT_MAX, kMiss, 0.f, 0.f};
    Stats st;
    trace_one(G, r, h, true, st);
    occluded[i] = h.ref != kMiss ? 1 : 0;
    S += st.steps;
    T += st.tests;
  }
  if (stats) { stats[0] = S; stats[1] = T; }
}

// Brute-force closest hit over all triangles (no grid), same watertight test.
void orc_trace_brute(const float* vtx, const uint32_t* idx, uint32_t nt, const float* ox,
                     const float* oy, const float* oz, const float* dx, const float* dy,
                     const float* dz, uint32_t n, uint32_t* tri, float* t) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    V3 org = mk(ox[i], oy[i], oz[i]), dir = mk(dx[i], dy[i], dz[i]);
    WT w = wt_setup(dir);
    float best = FLT_MAX, tt, uu, vv;
    uint32_t bh = kMiss;
    for (uint32_t k = 0; k < nt; ++k) {
      Tri tr = load_tri(vtx, idx, k);
      if (wt_intersect(w, org, tr, kEps, best, tt, uu, vv)) { best = tt; bh = k; }
    }
    tri[i] = bh;
    t[i] = best;
  }
}

// FP64 ray/plane distance of the reported triangle, for the 1e-5 t check.
void orc_t_fp64(const float* vtx, const uint32_t* idx, const uint32_t* tri, const float* ox,
                const float* oy, const float* oz, const float* dx, const float* dy, const float* dz,
                uint32_t n, double* t64) {
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < (int64_t)n; ++i) {
    if (tri[i] == kMiss) { t64[i] = NAN; continue; }
    double p[3][3];
    for (int k = 0; k < 3; ++k) {
      const float* q = vtx + 3 * (size_t)idx[3 * (size_t)tri[i] + k];
      p[k][0] = q[0]; p[k][1] = q[1]; p[k][2] = q[2];
    }
    double e1[3] = {p[1][0] - p[0][0], p[1][1] - p[0][1], p[1][2] - p[0][2]};
    double e2[3] = {p[2][0] - p[0][0], p[2][1] - p[0][1], p[2][2] - p[0][2]};
    double nn[3] = {e1[1] * e2[2] - e1[2] * e2[1], e1[2] * e2[0] - e1[0] * e2[2], e1[0] * e2[1] - e1[1] * e2[0]};
    double o[3] = {ox[i], oy[i], oz[i]}, d[3] = {dx[i], dy[i], dz[i]};
    double num = (p[0][0] - o[0]) * nn[0] + (p[0][1] - o[1]) * nn[1] + (p[0][2] - o[2]) * nn[2];
    double den = d[0] * nn[0] + d[1] * nn[1] + d[2] * nn[2];
    t64[i] = num / den;
  }
}

}  // extern "C"

// ===========================================================================
// Ray generation
namespace {

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw: "Parallel Random Numbers: As
// Easy as 1, 2, 3", SC'11).
inline void philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t h0 = (uint32_t)(p0 >> 32), l0 = (uint32_t)p0;
    const uint32_t h1 = (uint32_t)(p1 >> 32), l1 = (uint32_t)p1;
    const uint32_t n0 = h1 ^ c[1] ^ k0, n2 = h0 ^ c[3] ^ k1;
    c[0] = n0; c[1] = l1; c[2] = n2; c[3] = l0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

inline float u01(uint32_t w) { return (float)(w >> 8) * (1.0f / 16777216.0f); }

// sin/cos of 2*pi*u for u in [0,1): quadrant reduction and Taylor polynomials
// of degree 11 (sin) / 12 (cos) on [0, pi/2], evaluated with basic IEEE
// operations only so that host and device agree bit for bit.
inline void sincos_2pi(float u, float& s, float& c) {
  const float x = u * 4.0f;
  int q = (int)x;
  const float f = x - (float)q;
  q &= 3;
  const float th = f * 1.57079632679489662f;
  const float z = th * th;
  float ps = -2.50521083854417188e-08f;            // -1/11!
  ps = ps * z + 2.75573192239858907e-06f;           //  1/9!
  ps = ps * z + -1.98412698412698413e-04f;          // -1/7!
  ps = ps * z + 8.33333333333333333e-03f;           //  1/5!
  ps = ps * z + -1.66666666666666667e-01f;          // -1/3!
  ps = ps * z + 1.0f;
  const float sv = th * ps;
  float pc = 2.08767569878680990e-09f;              //  1/12!
  pc = pc * z + -2.75573192239858907e-07f;          // -1/10!
  pc = pc * z + 2.48015873015873016e-05f;           //  1/8!
  pc = pc * z + -1.38888888888888889e-03f;          // -1/6!
  pc = pc * z + 4.16666666666666667e-02f;           //  1/4!
  pc = pc * z + -0.5f;                              // -1/2!
  pc = pc * z + 1.0f;
  const float cv = pc;
  switch (q) {
    case 0: s = sv; c = cv; break;
    case 1: s = cv; c = -sv; break;
    case 2: s = -sv; c = -cv; break;
    default: s = -cv; c = sv; break;
  }
}

}  // namespace

extern "C" {

void orc_sincos_2pi(const float* u, uint32_t n, float* s, float* c) {
  for (uint32_t i = 0; i < n; ++i) sincos_2pi(u[i], s[i], c[i]);
}

// CosineHemisphereSampler (src/Utils/HemisphereSamplers.hpp:54-72) in the
// local frame: (sin 2pi u1 * sqrt(1-u2), cos 2pi u1 * sqrt(1-u2), sqrt(u2)),
// with the deterministic sincos_2pi above.
void orc_cosine_local(const float* u1, const float* u2, uint32_t n, float* out) {
  for (uint32_t i = 0; i < n; ++i) {
    float sn, cs;
    sincos_2pi(u1[i], sn, cs);
    const float r = sqrtf(1.f - u2[i]);
    out[3 * i] = sn * r;
    out[3 * i + 1] = cs * r;
    out[3 * i + 2] = sqrtf(u2[i]);
  }
}

void orc_philox(const uint32_t* ctr, uint32_t n, uint32_t k0, uint32_t k1, uint32_t* out) {
  for (uint32_t i = 0; i < n; ++i) {
    uint32_t c[4] = {ctr[4 * i], ctr[4 * i + 1], ctr[4 * i + 2], ctr[4 * i + 3]};
    philox(c, k0, k1);
    for (int j = 0; j < 4; ++j) out[4 * i + j] = c[j];
  }
}

// Camera::init (src/Primitive/Camera.h:41-60): out = {topLeft, stepX, stepY}.
void orc_camera(const float eye[3], const float fwd[3], const float up[3], float fov_deg,
                uint32_t resx, uint32_t resy, float out[9]) {
  (void)eye;
  const float aspect = (float)resx / (float)resy;
  const V3 f = normalize(mk(fwd[0], fwd[1], fwd[2]));
  const V3 r = normalize(cross(f, mk(up[0], up[1], up[2])));
  const V3 u = normalize(cross(f, r));
  const float ang = fov_deg * 3.14159265358979323846f / 180.f;
  const float tn = tanf(ang / 2.f);
  const V3 row = muls(muls(muls(r, 2.f), tn), aspect);
  const V3 col = muls(muls(u, 2.f), tn);
  const V3 sx = mk(row.x / (float)resx, row.y / (float)resx, row.z / (float)resx);
  const V3 sy = mk(col.x / (float)resy, col.y / (float)resy, col.z / (float)resy);
  const V3 tl = sub(sub(f, mk(row.x / 2.f, row.y / 2.f, row.z / 2.f)), mk(col.x / 2.f, col.y / 2.f, col.z / 2.f));
  out[0] = tl.x; out[1] = tl.y; out[2] = tl.z;
  out[3] = sx.x; out[4] = sx.y; out[5] = sx.z;
  out[6] = sy.x; out[7] = sy.y; out[8] = sy.z;
}

// RegularPrimaryRayGenerator with RegularPixelSampler<1,1>
// (src/Engine/RayGenerators.h:36-61, src/Primitive/PixelSampler.h:34-54):
// direction = topLeft + px*stepX + py*stepY (not normalised).
void orc_primary_rays(const float cam[9], uint32_t resx, uint32_t resy, uint32_t image_id,
                      float* dx, float* dy, float* dz) {
  const float rx = (float)resx;
  const uint32_t n = resx * resy;
  for (uint32_t id = 0; id < n; ++id) {
    float tmp = (float)image_id / 1.0f;
    float py = (truncf(tmp) + 0.5f) / 1.0f;
    float px = tmp - truncf(tmp) + 0.5f / 1.0f;
    tmp = (float)id / rx;
    py += truncf(tmp);
    px += (tmp - truncf(tmp)) * rx;
    dx[id] = cam[0] + px * cam[3] + py * cam[6];
    dy[id] = cam[1] + px * cam[4] + py * cam[7];
    dz[id] = cam[2] + px * cam[5] + py * cam[8];
  }
}

// Ambient-occlusion rays from primary hits: for every hit pixel p and sample
// s < spp, origin = hit point + offset * n (n faces the incoming ray),
// direction = cosine-weighted about n (CosineHemisphereSampler,
// src/Utils/HemisphereSamplers.hpp:54-72) in the frame {normalize(e1),
// n x normalize(e1), n}, random numbers from Philox4x32-10 with counter
// (p, s, 0, 0x414F) and key (seed, 0).  Output rays are in pixel-major
// order over hit pixels only; returns the number of rays written.
uint32_t orc_ao_rays(const float* vtx, const uint32_t* idx, const float* ox, const float* oy,
                     const float* oz, const float* dx, const float* dy, const float* dz,
                     const uint32_t* tri, const float* t, uint32_t n, uint32_t spp, uint32_t seed,
                     float offset, float* rox, float* roy, float* roz, float* rdx, float* rdy,
                     float* rdz, uint32_t* rpix, const uint32_t* pix) {
  uint32_t m = 0;
  for (uint32_t p = 0; p < n; ++p) {
    if (tri[p] == kMiss) continue;
    const uint32_t pid = pix ? pix[p] : p;  // the pixel's id in the full frame
    const Tri tr = load_tri(vtx, idx, tri[p]);
    const V3 d = mk(dx[p], dy[p], dz[p]);
    const V3 e1 = sub(tr.v[1], tr.v[0]);
    V3 nn = normalize(cross(e1, sub(tr.v[2], tr.v[0])));
    if (dot(nn, d) > 0.f) nn = mk(-nn.x, -nn.y, -nn.z);
    const V3 tx = normalize(e1);
    const V3 ty = cross(nn, tx);
    const V3 hp = add(mk(ox[p], oy[p], oz[p]), muls(d, t[p]));
    const V3 o = add(hp, muls(nn, offset));
    for (uint32_t s = 0; s < spp; ++s) {
      uint32_t c[4] = {pid, s, 0u, 0x414Fu};
      philox(c, seed, 0u);
      const float u1 = u01(c[0]), u2 = u01(c[1]);
      float sn, cs;
      sincos_2pi(u1, sn, cs);
      const float r = sqrtf(1.f - u2);
      const float lx = sn * r, ly = cs * r, lz = sqrtf(u2);
      rox[m] = o.x; roy[m] = o.y; roz[m] = o.z;
      rdx[m] = tx.x * lx + ty.x * ly + nn.x * lz;
      rdy[m] = tx.y * lx + ty.y * ly + nn.y * lz;
      rdz[m] = tx.z * lx + ty.z * ly + nn.z * lz;
      rpix[m] = p;
      ++m;
    }
  }
  return m;
}

// Direct illumination from a parallelogram light (DirectIlluminationIntegrator::shade,
// src/Integrator/DirectIlluminationIntegrator.h:254-315).  light15 = position,
// edge1, edge2, normal, intensity.  Shadow segment of sample s of hit pixel p:
// origin = o + (t - 1e-5) d, the stored hit point of SimpleRayBuffer::store
// (src/Engine/RayBuffers.h:52-55); direction = a uniform point of the light
// (AreaLightSource::getPoint, src/Primitive/LightSource.hpp:40-43) minus the
// origin, its (r1, r2) from Philox4x32-10 with counter (p, s, image_id, 0x444C)
// and key (seed, 0) in place of AreaLightShadowRayGenerator's KISS generator
// (src/Engine/RayGenerators.h:106-139).  The segment is blocked by a hit with
// t in (1e-5, 0.9999) (OcclusionRayBuffer::store, src/Engine/RayBuffers.h:156-168).
static void di_segment(V3 org, V3 d, float t, const float* light15, uint32_t p, uint32_t s,
                       uint32_t image_id, uint32_t seed, V3& o, V3& L) {
  const V3 LP = mk(light15[0], light15[1], light15[2]), E1 = mk(light15[3], light15[4], light15[5]),
           E2 = mk(light15[6], light15[7], light15[8]);
  o = add(org, muls(d, t - 1e-5f));
  uint32_t c[4] = {p, s, image_id, 0x444Cu};
  philox(c, seed, 0u);
  const V3 lp = add(add(LP, muls(E1, u01(c[0]))), muls(E2, u01(c[1])));
  L = sub(lp, o);
}

// Shadow segments of every hit pixel, pixel-major over hit pixels, spp per
// pixel; returns the number written.
uint32_t orc_direct_rays(const float* ox, const float* oy, const float* oz, const float* dx,
                         const float* dy, const float* dz, const uint32_t* tri, const float* t,
                         uint32_t n, uint32_t spp, uint32_t seed, uint32_t image_id,
                         const float* light15, float* rox, float* roy, float* roz, float* rdx,
                         float* rdy, float* rdz, uint32_t* rpix, const uint32_t* pix) {
  uint32_t m = 0;
  for (uint32_t p = 0; p < n; ++p) {
    if (tri[p] == kMiss) continue;
    const uint32_t pid = pix ? pix[p] : p;
    for (uint32_t s = 0; s < spp; ++s) {
      V3 o, L;
      di_segment(mk(ox[p], oy[p], oz[p]), mk(dx[p], dy[p], dz[p]), t[p], light15, pid, s, image_id, seed, o, L);
      rox[m] = o.x; roy[m] = o.y; roz[m] = o.z;
      rdx[m] = L.x; rdy[m] = L.y; rdz[m] = L.z;
      rpix[m] = p;
      ++m;
    }
  }
  return m;
}

// computeDirectIllumination (src/Integrator/DirectIlluminationIntegrator.h:46-168):
// per unblocked sample intensity * area * diffuse * max(0, -n_light . L^) *
// max(0, n . L^) / (L . L) with n the unflipped geometric normal, summed as
// value / spp in sample order; pixels without a hit sum background / spp.
// occ holds the blocked flags of orc_direct_rays' segments in its order.  The
// final image blends with weight 1 / (image_id + 1).  Material ids >=
// num_materials read material 0; diffuse == nullptr means ddef everywhere.
void orc_shade_direct(const float* vtx, const uint32_t* idx, const float* ox, const float* oy,
                      const float* oz, const float* dx, const float* dy, const float* dz,
                      const uint32_t* tri, const float* t, uint32_t n, uint32_t spp, uint32_t seed,
                      uint32_t image_id, const float* light15, const uint32_t* tri_mat,
                      const float* diffuse, uint32_t nmat, const float* ddef, const float* bg,
                      const uint8_t* occ, float* frame, float* fin, const uint32_t* pix) {
  const V3 E1 = mk(light15[3], light15[4], light15[5]), E2 = mk(light15[6], light15[7], light15[8]);
  const V3 LN = mk(light15[9], light15[10], light15[11]), LI = mk(light15[12], light15[13], light15[14]);
  const V3 lc = cross(E1, E2);
  const float larea = sqrtf(dot(lc, lc));
  const V3 BG = mk(bg[0], bg[1], bg[2]);
  const float inv_s = 1.0f / (float)spp;
  uint32_t k = 0;
  for (uint32_t p = 0; p < n; ++p) {
    V3 rad = mk(0.f, 0.f, 0.f);
    if (tri[p] == kMiss) {
      for (uint32_t s = 0; s < spp; ++s) rad = add(rad, muls(BG, inv_s));
    } else {
      const Tri tr = load_tri(vtx, idx, tri[p]);
      const V3 nrm = normalize(cross(sub(tr.v[1], tr.v[0]), sub(tr.v[2], tr.v[0])));
      V3 diff = mk(ddef[0], ddef[1], ddef[2]);
      if (diffuse) {
        uint32_t m = tri_mat ? tri_mat[tri[p]] : 0u;
        if (m >= nmat) m = 0u;
        diff = mk(diffuse[4 * m], diffuse[4 * m + 1], diffuse[4 * m + 2]);
      }
      const V3 kk = mul(muls(LI, larea), diff);
      const uint32_t pid = pix ? pix[p] : p;
      for (uint32_t s = 0; s < spp; ++s, ++k) {
        if (occ[k]) continue;
        V3 o, L;
        di_segment(mk(ox[p], oy[p], oz[p]), mk(dx[p], dy[p], dz[p]), t[p], light15, pid, s, image_id, seed, o, L);
        const V3 ln = normalize(L);
        const float att = 1.0f / dot(L, L);
        const float a = fmaxf(0.f, -dot(LN, ln));
        const float b = fmaxf(0.f, dot(nrm, ln));
        rad = add(rad, muls(muls(muls(muls(kk, a), b), att), inv_s));
      }
    }
    frame[3 * p] = rad.x;
    frame[3 * p + 1] = rad.y;
    frame[3 * p + 2] = rad.z;
    if (fin) {
      const float wn = 1.0f / (float)(image_id + 1u);
      const float wo = 1.0f - wn;
      fin[3 * p] = fin[3 * p] * wo + rad.x * wn;
      fin[3 * p + 1] = fin[3 * p + 1] * wo + rad.y * wn;
      fin[3 * p + 2] = fin[3 * p + 2] * wo + rad.z * wn;
    }
  }
}

// Path tracer, path by path (the CUDA side runs it as a wavefront with
// compaction; results are per path and independent of the schedule).
// Semantics: SimplePathTracer (src/Integrator/SimplePathTracer.hpp:65-241)
// restated with next-event estimation at every vertex to a parallelogram
// light, Russian roulette with continuation probability = albedo from depth
// rr_depth on, cosine-weighted bounces (CosineHemisphereSampler,
// src/Utils/HemisphereSamplers.hpp:54-72), camera jitter as in
// RandomPixelSampler (src/Primitive/PixelSampler.h:56-70), Philox4x32-10
// counters (pixel, sample, depth, tag) with key (seed, 0).  The image is the
// per-pixel mean of the per-path radiance summed in sample order.
// pix (may be null): render only pixels pix[0..npix_sel) of the frame into
// image[3k..3k+3) (a sample of a frame); null renders every pixel.
void orc_pt_render_pixels(const orc_grid* G, const float cam9[9], const float eye[3], uint32_t resx,
                          uint32_t resy, uint32_t spp, uint32_t max_depth, uint32_t rr_depth, float albedo,
                          const float lpos[3], const float le1[3], const float le2[3], const float lrad[3],
                          const float bg[3], float offset, uint32_t seed, const uint32_t* pix,
                          uint32_t npix_sel, float* image) {
  const uint32_t npix = pix ? npix_sel : resx * resy;
  const V3 LP = mk(lpos[0], lpos[1], lpos[2]), E1 = mk(le1[0], le1[1], le1[2]),
           E2 = mk(le2[0], le2[1], le2[2]), LR = mk(lrad[0], lrad[1], lrad[2]), BG = mk(bg[0], bg[1], bg[2]);
  const V3 ln = cross(E1, E2);
  const float larea = sqrtf(dot(ln, ln));
  const V3 lnrm = normalize(ln);
  const V3 tl = mk(cam9[0], cam9[1], cam9[2]), sx = mk(cam9[3], cam9[4], cam9[5]), sy = mk(cam9[6], cam9[7], cam9[8]);
  const V3 E = mk(eye[0], eye[1], eye[2]);
  const float rxf = (float)resx;
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t pi = 0; pi < (int64_t)npix; ++pi) {
    const uint32_t p = pix ? pix[pi] : (uint32_t)pi;
    float ir = 0.f, ig = 0.f, ib = 0.f;
    for (uint32_t s = 0; s < spp; ++s) {
      uint32_t c[4] = {p, s, 0u, 0x4A49u};
      philox(c, seed, 0u);
      float ox = u01(c[0]), oy = u01(c[1]);
      const float tmp = (float)p / rxf;
      oy = truncf(tmp) + oy;
      ox = (tmp - truncf(tmp)) * rxf + ox;
      V3 d = mk(tl.x + ox * sx.x + oy * sy.x, tl.y + ox * sx.y + oy * sy.y, tl.z + ox * sx.z + oy * sy.z);
      V3 org = E;
      V3 beta = mk(1.f, 1.f, 1.f), L = mk(0.f, 0.f, 0.f);
      for (uint32_t depth = 0; depth < max_depth; ++depth) {
        Hit h{FLT_MAX, kMiss, 0.f, 0.f};
        Stats st;
        trace_one(G, Ray{org, d}, h, false, st);
        if (h.ref == kMiss) {
          L = add(L, mul(beta, BG));
          break;
        }
        const Tri tr = load_tri(G->vtx.data(), G->idx.data(), G->indices[h.ref]);
        const V3 e1 = sub(tr.v[1], tr.v[0]);
        V3 nn = normalize(cross(e1, sub(tr.v[2], tr.v[0])));
        if (dot(nn, d) > 0.f) nn = mk(-nn.x, -nn.y, -nn.z);
        const V3 hp = add(org, muls(d, h.t));
        const V3 o = add(hp, muls(nn, offset));
        uint32_t cl4[4] = {p, s, depth, 0x4C54u};
        philox(cl4, seed, 0u);
        const float lu = u01(cl4[0]), lv = u01(cl4[1]), urr = u01(cl4[2]);
        const V3 lp = add(add(LP, muls(E1, lu)), muls(E2, lv));
        const V3 wv = sub(lp, o);
        const float d2 = dot(wv, wv);
        const V3 l = muls(wv, 1.0f / sqrtf(d2));
        const float cs = dot(nn, l);
        const float clg = -dot(lnrm, l);
        if (cs > 0.f && clg > 0.f) {
          Hit sh{0.9999f, kMiss, 0.f, 0.f};
          Stats st2;
          trace_one(G, Ray{o, wv}, sh, true, st2);
          if (sh.ref == kMiss) {
            const float f = ((((albedo * 0.31830988618379067f) * cs) * clg) * larea) / d2;
            L = add(L, muls(mul(beta, LR), f));
          }
        }
        bool live = depth + 1 < max_depth;
        if (live && depth >= rr_depth) {
          if (urr < albedo) beta = muls(beta, 1.0f / albedo);
          else live = false;
        }
        if (!live) break;
        uint32_t cd[4] = {p, s, depth, 0x4449u};
        philox(cd, seed, 0u);
        const float u1 = u01(cd[0]), u2 = u01(cd[1]);
        float sn, cn;
        sincos_2pi(u1, sn, cn);
        const float rr = sqrtf(1.f - u2);
        const float lx = sn * rr, ly = cn * rr, lz = sqrtf(u2);
        const V3 tx = normalize(e1);
        const V3 ty = cross(nn, tx);
        d = mk(tx.x * lx + ty.x * ly + nn.x * lz, tx.y * lx + ty.y * ly + nn.y * lz,
               tx.z * lx + ty.z * ly + nn.z * lz);
        beta = muls(beta, albedo);
        org = o;
      }
      ir += L.x;
      ig += L.y;
      ib += L.z;
    }
    image[3 * (size_t)pi] = ir / (float)spp;
    image[3 * (size_t)pi + 1] = ig / (float)spp;
    image[3 * (size_t)pi + 2] = ib / (float)spp;
  }
}

void orc_pt_render(const orc_grid* G, const float cam9[9], const float eye[3], uint32_t resx,
                   uint32_t resy, uint32_t spp, uint32_t max_depth, uint32_t rr_depth, float albedo,
                   const float lpos[3], const float le1[3], const float le2[3], const float lrad[3],
                   const float bg[3], float offset, uint32_t seed, float* image) {
  orc_pt_render_pixels(G, cam9, eye, resx, resy, spp, max_depth, rr_depth, albedo, lpos, le1, le2, lrad, bg,
                       offset, seed, nullptr, 0, image);
}

// Stable stream compaction: indices of non-zero flags in order.
uint32_t orc_compact(const uint32_t* flags, uint32_t n, uint32_t* out) {
  uint32_t m = 0;
  for (uint32_t i = 0; i < n; ++i)
    if (flags[i]) out[m++] = i;
  return m;
}

}  // extern "C"
