// Device-side building blocks shared by the build, traversal and path-tracing
// kernels.  All float arithmetic here is written in an explicit operation
// order; the library is compiled with -fmad=false so that no multiply-add is
// contracted and every result is reproducible bit for bit on the host.
#pragma once
#include <cfloat>
#include <cstdint>
#include <cuda_runtime.h>

#define SHN_HD __host__ __device__ __forceinline__
#define SHN_D __device__ __forceinline__

namespace shn {

constexpr float kEps = 0.00001f;      // EPS, src/CUDAStdAfx.h:96
constexpr uint32_t kMiss = 0xFFFFFFFFu;
constexpr uint32_t kNotEmpty = 0x40000000u;  // TwoLevelGridCell LARGENOTEMPTYMASK

// Device error word bits (grid->err / ctx->err): set by bounded waits that gave up.
constexpr uint32_t kErrLookbackTimeout = 1u;
constexpr uint32_t kErrTmaTimeout = 2u;
constexpr uint32_t kErrCapacity = 4u;

struct V3 {
  float x, y, z;
};
SHN_HD V3 mk(float x, float y, float z) { return V3{x, y, z}; }
SHN_HD V3 add(V3 a, V3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
SHN_HD V3 sub(V3 a, V3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
SHN_HD V3 mul(V3 a, V3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
SHN_HD V3 divv(V3 a, V3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
SHN_HD V3 muls(V3 a, float s) { return mk(a.x * s, a.y * s, a.z * s); }
SHN_HD float dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
SHN_HD V3 cross(V3 a, V3 b) {
  return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
SHN_HD V3 normalize(V3 a) {
  const float r = 1.0f / sqrtf(dot(a, a));
  return muls(a, r);
}
SHN_HD V3 vmin(V3 a, V3 b) { return mk(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
SHN_HD V3 vmax(V3 a, V3 b) { return mk(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
SHN_HD float comp(V3 v, int i) { return i == 0 ? v.x : (i == 1 ? v.y : v.z); }
SHN_HD V3 f4v(float4 a) { return mk(a.x, a.y, a.z); }

// Grid geometry (GridParameters + the build-time reciprocal).
struct Geom {
  V3 gmin, gmax;
  int res[3];
  V3 resf;
  V3 cs;        // (max-min)/res              SimpleGrid::getCellSize
  V3 rcpBuild;  // 1/cs                       FastSimpleGridBuilder.h:117
  V3 rcpTrav;   // res/(max-min)              SimpleGrid::getCellSizeRCP
};

// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, SC'11).
SHN_HD uint4 philox4x32(uint4 c, uint32_t k0, uint32_t k1) {
#pragma unroll
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)0xD2511F53u * c.x;
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c.z;
    const uint32_t h0 = (uint32_t)(p0 >> 32), l0 = (uint32_t)p0;
    const uint32_t h1 = (uint32_t)(p1 >> 32), l1 = (uint32_t)p1;
    c = make_uint4(h1 ^ c.y ^ k0, l1, h0 ^ c.w ^ k1, l0);
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
  return c;
}

SHN_HD float u01(uint32_t w) { return (float)(w >> 8) * (1.0f / 16777216.0f); }

// sin/cos of 2*pi*u, u in [0,1): quadrant reduction plus Taylor polynomials
// of degree 11 / 12 on [0, pi/2] (coefficients 1/n!), basic IEEE operations
// only, so the host restatement reproduces it exactly.
SHN_HD void sincos_2pi(float u, float& s, float& c) {
  const float x = u * 4.0f;
  int q = (int)x;
  const float f = x - (float)q;
  q &= 3;
  const float th = f * 1.57079632679489662f;
  const float z = th * th;
  float ps = -2.50521083854417188e-08f;
  ps = ps * z + 2.75573192239858907e-06f;
  ps = ps * z + -1.98412698412698413e-04f;
  ps = ps * z + 8.33333333333333333e-03f;
  ps = ps * z + -1.66666666666666667e-01f;
  ps = ps * z + 1.0f;
  const float sv = th * ps;
  float pc = 2.08767569878680990e-09f;
  pc = pc * z + -2.75573192239858907e-07f;
  pc = pc * z + 2.48015873015873016e-05f;
  pc = pc * z + -1.38888888888888889e-03f;
  pc = pc * z + 4.16666666666666667e-02f;
  pc = pc * z + -0.5f;
  pc = pc * z + 1.0f;
  const float cv = pc;
  if (q == 0) { s = sv; c = cv; }
  else if (q == 1) { s = cv; c = -sv; }
  else if (q == 2) { s = -sv; c = -cv; }
  else { s = -cv; c = sv; }
}

// ---- memory-model helpers (look-back publication) ---------------------------
SHN_D uint32_t ld_acquire(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
SHN_D uint32_t ld_relaxed(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
SHN_D void st_relaxed(uint32_t* p, uint32_t v) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
SHN_D void st_release(uint32_t* p, uint32_t v) {
  asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}
SHN_D uint64_t ld_acquire64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
SHN_D void st_release64(uint64_t* p, uint64_t v) {
  asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Bounded spin budget for look-back and barrier waits: after this many polls
// (each followed by a short sleep) a wait records an error and gives up.
constexpr uint32_t kSpinLimit = 1u << 22;

}  // namespace shn
