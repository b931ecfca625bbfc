// 3D-DDA traversal of uniform and two-level grids with the watertight
// ray/triangle test, as device functions shared by the trace, AO and
// path-tracing kernels.
//
// Traversal restates UniformGridTraverser (src/Control/Algorithm/SimpleGridTraverser.h:274-401)
// and TwoLevelGridTraverser (src/Control/Algorithm/TwoLevelGridTraverser.h:445-671):
// float cell coordinates, continuation while the best t exceeds the current
// cell's exit (min of tMax), exit when a coordinate reaches res or -1 within
// 0.1.  Cell lookups clamp the coordinates like the reference's tex3D did;
// each DDA level carries a step cap of res.x+res.y+res.z+3.  Any-hit stops at
// the first hit in (EPS, tmax).
//
// Triangles are read from the grid's reference-ordered SoA float4 copy
// (v0[ref], v1[ref], v2[ref]; v0.w carries the triangle id), so a cell's
// candidates are contiguous and no indices[] indirection is needed.
#pragma once
#include "common.cuh"

namespace shn {

struct GridView {
  Geom g;
  uint32_t kind;
  const uint2* __restrict__ cells;
  const uint2* __restrict__ leaves;
  const float4* __restrict__ rv0;
  const float4* __restrict__ rv1;
  const float4* __restrict__ rv2;
  // the scene's triangle records (48 bytes: v0 with the id in w, v1, v2),
  // indexed by the id that rv0[].w holds
  const float4* __restrict__ src;
  // boxes (min, max) of references [32k, 32k + 32) and [1024s, 1024s + 1024)
  // of rv*, or null (no culling)
  const float4* __restrict__ cbox;
  const float4* __restrict__ sbox;
  // when not null: no reference-ordered copy; reference i is src[3 * ridx[i]]
  const uint32_t* __restrict__ ridx;
};

struct Hit {
  float t;
  uint32_t tri;
  float u, v;
  uint32_t steps = 0, tests = 0;  // work counters (only read by the stats variants)
};

// Watertight ray/triangle test (Woop, Benthin, Wald, JCGT 2(1), 2013).
struct RayWT {
  V3 org;
  int kx, ky, kz;
  float Sx, Sy, Sz;
};

SHN_D float sel(int k, V3 v) { return k == 0 ? v.x : (k == 1 ? v.y : v.z); }

SHN_D RayWT wt_setup(V3 org, V3 d) {
  RayWT r;
  r.org = org;
  const float ax = fabsf(d.x), ay = fabsf(d.y), az = fabsf(d.z);
  r.kz = (ax > ay) ? ((ax > az) ? 0 : 2) : ((ay > az) ? 1 : 2);
  r.kx = r.kz + 1 == 3 ? 0 : r.kz + 1;
  r.ky = r.kx + 1 == 3 ? 0 : r.kx + 1;
  if (sel(r.kz, d) < 0.f) {
    const int t = r.kx;
    r.kx = r.ky;
    r.ky = t;
  }
  const float dz = sel(r.kz, d);
  r.Sx = sel(r.kx, d) / dz;
  r.Sy = sel(r.ky, d) / dz;
  r.Sz = 1.0f / dz;
  return r;
}

SHN_D bool wt_test(const RayWT& r, float4 p0, float4 p1, float4 p2, float tmin, float tbest,
                   float& t, float& u, float& v) {
  const V3 A = sub(f4v(p0), r.org), B = sub(f4v(p1), r.org), C = sub(f4v(p2), r.org);
  const float Akz = sel(r.kz, A), Bkz = sel(r.kz, B), Ckz = sel(r.kz, C);
  // shear: one fused multiply-add per coordinate; edge functions: one product
  // rounded, then a fused multiply-add (the oracle uses fmaf identically)
  const float Ax = __fmaf_rn(-r.Sx, Akz, sel(r.kx, A));
  const float Ay = __fmaf_rn(-r.Sy, Akz, sel(r.ky, A));
  const float Bx = __fmaf_rn(-r.Sx, Bkz, sel(r.kx, B));
  const float By = __fmaf_rn(-r.Sy, Bkz, sel(r.ky, B));
  const float Cx = __fmaf_rn(-r.Sx, Ckz, sel(r.kx, C));
  const float Cy = __fmaf_rn(-r.Sy, Ckz, sel(r.ky, C));
  float U = __fmaf_rn(Cx, By, -(Cy * Bx));
  float V = __fmaf_rn(Ax, Cy, -(Ay * Cx));
  float W = __fmaf_rn(Bx, Ay, -(By * Ax));
  // exact zero of an edge function -> recompute in double; mixed signs -> miss
  // (min/max skip a NaN operand exactly as or-chains of comparisons do)
  if (fminf(fminf(fabsf(U), fabsf(V)), fabsf(W)) == 0.f) {
    U = (float)((double)Cx * (double)By - (double)Cy * (double)Bx);
    V = (float)((double)Ax * (double)Cy - (double)Ay * (double)Cx);
    W = (float)((double)Bx * (double)Ay - (double)By * (double)Ax);
  }
  if (fminf(fminf(U, V), W) < 0.f && fmaxf(fmaxf(U, V), W) > 0.f) return false;
  const float det = U + V + W;
  if (det == 0.f) return false;
  const float T = __fmaf_rn(W, r.Sz * Ckz, __fmaf_rn(V, r.Sz * Bkz, U * (r.Sz * Akz)));
  const float tt = T / det;
  if (!(tt > tmin && tt < tbest)) return false;
  t = tt;
  u = V / det;
  v = W / det;
  return true;
}

// Closest hit in a range: the least (t, triangle id) below the bound from
// earlier cells, i.e. the first minimum in triangle-id order, which is what a
// strict-< loop over the references in (cell, triangle) order keeps.  The
// references of a range may be stored in another order, so a candidate may
// tie the range's running minimum (bound = next float above it) and wins on
// the smaller id.
SHN_D float next_up(float t) { return __uint_as_float(__float_as_uint(t) + 1u); }

template <bool ANY>
SHN_D bool test_range(const GridView& G, const RayWT& r, uint32_t b, uint32_t e, Hit& h) {
  h.steps += 1;
  const float t0 = h.t;
  bool found = false;
  for (uint32_t it = b; it < e; ++it) {
    h.tests += 1;
    const float4 p0 = __ldg(G.rv0 + it);
    const float4 p1 = __ldg(G.rv1 + it);
    const float4 p2 = __ldg(G.rv2 + it);
    float t, u, v;
    if (wt_test(r, p0, p1, p2, kEps, found ? next_up(h.t) : t0, t, u, v)) {
      const uint32_t id = __float_as_uint(p0.w);
      if (!found || t < h.t || id < h.tri) {
        h.t = t;
        h.tri = id;
        h.u = u;
        h.v = v;
        found = true;
      }
      if (ANY) return true;
    }
  }
  return false;
}

SHN_D int min_dim(V3 t) { return (t.x < t.y) ? ((t.x < t.z) ? 0 : 2) : ((t.y < t.z) ? 1 : 2); }
SHN_D float clampf(float v, float lo, float hi) { return fminf(fmaxf(v, lo), hi); }
SHN_D void bump(V3& v, int d, float a) {
  if (d == 0) v.x += a; else if (d == 1) v.y += a; else v.z += a;
}

template <bool ANY>
SHN_D void trace_uniform(const GridView& G, V3 org, V3 dir, Hit& h) {
  const Geom& g = G.g;
  const V3 rcp = divv(mk(1.f, 1.f, 1.f), dir);
  const RayWT w = wt_setup(org, dir);
  if (!(h.t > 0.f)) return;
  const V3 t1 = mul(sub(g.gmin, org), rcp);
  V3 t2 = mul(sub(g.gmax, org), rcp);
  const V3 tmn = vmin(t1, t2);
  t2 = vmax(t1, t2);
  const float tEntry = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
  const float tExit = fminf(fminf(t2.x, t2.y), t2.z);
  if (tExit <= tEntry || tExit < 0.f) return;
  const float te = tEntry + kEps;
  const V3 entry = (tEntry >= 0.f) ? add(org, divv(mk(te, te, te), rcp)) : org;
  V3 cell = mul(sub(entry, g.gmin), g.rcpTrav);
  cell = mk(floorf(cell.x), floorf(cell.y), floorf(cell.z));
  const V3 tmp = mk(rcp.x > 0.f ? 1.f : 0.f, rcp.y > 0.f ? 1.f : 0.f, rcp.z > 0.f ? 1.f : 0.f);
  V3 tMax = mul(sub(add(mul(add(cell, tmp), g.cs), g.gmin), org), rcp);
  bool valid = (cell.x != (rcp.x > 0.f ? g.resf.x : -1.f)) && (cell.y != (rcp.y > 0.f ? g.resf.y : -1.f)) &&
               (cell.z != (rcp.z > 0.f ? g.resf.z : -1.f));
  const int cap = g.res[0] + g.res[1] + g.res[2] + 3;
  // An empty cell of a large uniform grid holds [D, D), D its distance to the
  // nearest non-empty cell: the next D - 1 cells are empty and are stepped
  // through without fetching (counted as visits all the same).
  uint32_t skip = 0;
  for (int step = 0; valid && step < cap; ++step) {
    if (skip == 0) {
      const uint32_t cx = (uint32_t)clampf(cell.x, 0.f, g.resf.x - 1.f);
      const uint32_t cy = (uint32_t)clampf(cell.y, 0.f, g.resf.y - 1.f);
      const uint32_t cz = (uint32_t)clampf(cell.z, 0.f, g.resf.z - 1.f);
      const uint2 range = __ldg(G.cells + (cx + cy * (uint32_t)g.res[0] + cz * (uint32_t)g.res[0] * (uint32_t)g.res[1]));
      if (test_range<ANY>(G, w, range.x, range.y, h)) return;
      if (range.y <= range.x && range.x > 0u) skip = range.x - 1u;
    } else {
      --skip;
      h.steps += 1;
    }
    valid = h.t > tMax.x || h.t > tMax.y || h.t > tMax.z;
    if (!valid) break;
    const int d = min_dim(tMax);
    const float rd = sel(d, rcp);
    bump(cell, d, rd > 0.f ? 1.f : -1.f);
    bump(tMax, d, sel(d, g.cs) * fabsf(rd));
    const float cd = sel(d, cell);
    valid = !(fabsf(cd - sel(d, g.resf)) < 0.1f || fabsf(cd + 1.f) < 0.1f);
  }
}

template <bool ANY>
SHN_D void trace_two_level(const GridView& G, V3 org, V3 dir, Hit& h) {
  const Geom& g = G.g;
  const V3 rcp = divv(mk(1.f, 1.f, 1.f), dir);
  const RayWT w = wt_setup(org, dir);
  if (!(h.t > 0.f)) return;
  const V3 t1 = mul(sub(g.gmin, org), rcp);
  V3 t2 = mul(sub(g.gmax, org), rcp);
  const V3 tmn = vmin(t1, t2);
  t2 = vmax(t1, t2);
  float tEntry = fmaxf(fmaxf(tmn.x, tmn.y), tmn.z);
  const float tExit = fminf(fminf(t2.x, t2.y), t2.z);
  if (tExit <= tEntry || tExit < 0.f) return;
  tEntry = fmaxf(0.f, tEntry);
  const float te = tEntry + kEps;
  const V3 entry = add(org, divv(mk(te, te, te), rcp));
  V3 cell = mul(sub(entry, g.gmin), g.rcpTrav);
  cell = mk(floorf(cell.x), floorf(cell.y), floorf(cell.z));
  const V3 tmp = mk(rcp.x > 0.f ? 1.f : 0.f, rcp.y > 0.f ? 1.f : 0.f, rcp.z > 0.f ? 1.f : 0.f);
  V3 tMax = mul(sub(add(mul(add(cell, tmp), g.cs), g.gmin), org), rcp);
  bool valid = (cell.x != (rcp.x > 0.f ? g.resf.x : -1.f)) && (cell.y != (rcp.y > 0.f ? g.resf.y : -1.f)) &&
               (cell.z != (rcp.z > 0.f ? g.resf.z : -1.f));
  const int cap = g.res[0] + g.res[1] + g.res[2] + 3;
  for (int step = 0; valid && step < cap; ++step) {
    const uint32_t cx = (uint32_t)clampf(cell.x, 0.f, g.resf.x - 1.f);
    const uint32_t cy = (uint32_t)clampf(cell.y, 0.f, g.resf.y - 1.f);
    const uint32_t cz = (uint32_t)clampf(cell.z, 0.f, g.resf.z - 1.f);
    const uint2 cw = __ldg(G.cells + (cx + cy * (uint32_t)g.res[0] + cz * (uint32_t)g.res[0] * (uint32_t)g.res[1]));
    if (cw.y & kNotEmpty) {
      const V3 ent = add(org, divv(mk(tEntry, tEntry, tEntry), rcp));
      const V3 cres = mk((float)(cw.y & 0xFFu), (float)((cw.y >> 8) & 0xFFu), (float)((cw.y >> 16) & 0xFFu));
      const V3 subRCP = mul(g.rcpTrav, cres);
      const V3 minB = add(mul(cell, g.cs), g.gmin);
      V3 sc;
      sc.x = floorf((ent.x - minB.x) * subRCP.x);
      sc.y = floorf((ent.y - minB.y) * subRCP.y);
      sc.z = floorf((ent.z - minB.z) * subRCP.z);
      const V3 scs = divv(mk(1.f, 1.f, 1.f), subRCP);
      sc = vmin(sub(cres, mk(1.f, 1.f, 1.f)), vmax(sc, mk(0.f, 0.f, 0.f)));
      V3 sMax;
      sMax.x = ((sc.x + tmp.x) * scs.x + minB.x - org.x) * rcp.x;
      sMax.y = ((sc.y + tmp.y) * scs.y + minB.y - org.y) * rcp.y;
      sMax.z = ((sc.z + tmp.z) * scs.z + minB.z - org.z) * rcp.z;
      bool v2 = true;
      const int cap2 = (int)cres.x + (int)cres.y + (int)cres.z + 3;
      for (int s2 = 0; v2 && s2 < cap2; ++s2) {
        const uint32_t li = cw.x + (uint32_t)(sc.x + cres.x * sc.y + cres.x * cres.y * sc.z);
        const uint2 range = __ldg(G.leaves + li);
        if (test_range<ANY>(G, w, range.x, range.y, h)) return;
        v2 = h.t > sMax.x || h.t > sMax.y || h.t > sMax.z;
        if (!v2) break;
        const int d = min_dim(sMax);
        const float rd = sel(d, rcp);
        bump(sc, d, rd > 0.f ? 1.f : -1.f);
        bump(sMax, d, sel(d, scs) * fabsf(rd));
        const float cd = sel(d, sc);
        v2 = !(fabsf(cd - sel(d, cres)) < 0.1f || fabsf(cd + 1.f) < 0.1f);
      }
    }
    valid = h.t > tMax.x || h.t > tMax.y || h.t > tMax.z;
    if (!valid) break;
    const int d = min_dim(tMax);
    tEntry = sel(d, tMax);
    const float rd = sel(d, rcp);
    bump(cell, d, rd > 0.f ? 1.f : -1.f);
    bump(tMax, d, sel(d, g.cs) * fabsf(rd));
    const float cd = sel(d, cell);
    valid = !(fabsf(cd - sel(d, g.resf)) < 0.1f || fabsf(cd + 1.f) < 0.1f);
  }
}

template <int KIND, bool ANY>
SHN_D void trace_ray(const GridView& G, V3 org, V3 dir, Hit& h) {
  if (KIND == 0) trace_uniform<ANY>(G, org, dir, h);
  else trace_two_level<ANY>(G, org, dir, h);
}

// Camera::init result + RegularPixelSampler<1,1> (src/Primitive/Camera.h:67-70,
// src/Primitive/PixelSampler.h:40-52).
struct CamView {
  V3 eye, tl, sx, sy;
  float resx;
  uint32_t res_x, res_y;
};

SHN_D V3 primary_dir(const CamView& c, uint32_t id, uint32_t image_id) {
  float tmp = (float)image_id / 1.0f;
  float py = (truncf(tmp) + 0.5f) / 1.0f;
  float px = tmp - truncf(tmp) + 0.5f / 1.0f;
  tmp = (float)id / c.resx;
  py += truncf(tmp);
  px += (tmp - truncf(tmp)) * c.resx;
  return mk(c.tl.x + px * c.sx.x + py * c.sy.x, c.tl.y + px * c.sx.y + py * c.sy.y,
            c.tl.z + px * c.sx.z + py * c.sy.z);
}

// Camera ray r -> pixel: rays 32k .. 32k+31 (one warp's packet) cover the
// 8x4 pixel tile k of the image (tiles row by row); the pixels right of the
// last full tile column and below the last full tile row follow in row
// order.  A bijection of [0, resx*resy).  With packet refill the 32 rays of
// a warp are one compact tile: camera kernel 2.22 -> 2.06 ms on the
// 1M-triangle cluster at 1920x1080 (32x1 rows before).
SHN_D uint32_t tile_pixel(const CamView& c, uint32_t r) {
  const uint32_t rx = c.res_x, ry = c.res_y;
  const uint32_t W = rx & ~7u, H = ry & ~3u;
  if (r < W * H) {
    const uint32_t t = r >> 5, q = r & 31u, tw = W >> 3;
    const uint32_t ty = t / tw, tx = t - ty * tw;
    return (ty * 4 + (q >> 3)) * rx + tx * 8 + (q & 7u);
  }
  r -= W * H;
  const uint32_t sw = rx - W;
  if (r < sw * H) {
    const uint32_t y = r / sw;
    return y * rx + W + (r - y * sw);
  }
  r -= sw * H;
  return H * rx + r;
}

}  // namespace shn
