// Checker-only driver around the reference's own host-compilable code.
//
// Built by oracle/Makefile from the reference sources where they lie (never
// copied): it links src/Control/Algorithm/TwoLevelGridBuilder.cpp
// (TwoLevelGridBuilderHost::hostBuild, the reference CPU builder) and
// instantiates the reference's host-usable headers (Camera, pixel sampler,
// Moller-Trumbore intersector, cosine hemisphere sampler, two-level cell
// word) behind a C ABI.  The output lands in oracle/_ref/ and is used by
// tests/golden/make_golden.py to pin the oracle, and by the bench's
// reference arm as the CPU baseline of the grid build.
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <vector>

#include "Control/Algorithm/TwoLevelGridBuilder.hpp"
#include "Loaders/CameraManager.hpp"
#include "Loaders/FWObject.hpp"
#include "Loaders/LightSourceLoader.hpp"
#include "Intersector/SimpleIntersector.hpp"
#include "Primitive/Camera.h"
#include "Primitive/PixelSampler.h"
#include "Primitive/Triangle.hpp"
#include "Utils/HemisphereSamplers.hpp"

int gRESX = 0;
int gRESY = 0;

namespace {
// Storage adapter so that SimpleIntersector's Moller-Trumbore test can read
// triangles from plain host arrays (FaceSoup::operator[] semantics:
// src/Control/Structure/FaceSoup.h:54-105, reference index == tri id here).
struct HostSoup {
  const float* vtx;
  const uint32_t* idx;
  Triangle operator[](uint i) const {
    Triangle t;
    for (int k = 0; k < 3; ++k) {
      const float* p = vtx + 3 * (size_t)idx[3 * (size_t)i + k];
      t.vertices[k].x = p[0];
      t.vertices[k].y = p[1];
      t.vertices[k].z = p[2];
    }
    return t;
  }
};

FWObject* make_object(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt) {
  FWObject* o = new FWObject();
  o->allocateVertices(nv);
  for (uint32_t i = 0; i < nv; ++i) {
    o->getVertex(i).x = vtx[3 * i];
    o->getVertex(i).y = vtx[3 * i + 1];
    o->getVertex(i).z = vtx[3 * i + 2];
  }
  o->allocateFaces(nt);
  for (uint32_t t = 0; t < nt; ++t) {
    FWObject::Face& f = o->getFace(t);
    f.vert1 = idx[3 * t];
    f.vert2 = idx[3 * t + 1];
    f.vert3 = idx[3 * t + 2];
    f.material = 0;
  }
  return o;
}

struct RefGrid {
  std::vector<uint32_t> cells, leaves, refs;
};
}  // namespace

extern "C" {

// TwoLevelGridBuilderHost::hostBuild on a caller-chosen top resolution and
// bounds (src/Control/Algorithm/TwoLevelGridBuilder.cpp:28-213).
void* ref_host_build(const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt, int rx,
                     int ry, int rz, const float bounds[6], uint64_t sizes[3]) {
  FWObject* o = make_object(vtx, nv, idx, nt);
  TwoLevelGridCell* cells = new TwoLevelGridCell[(size_t)rx * ry * rz];
  uint2* leaves = NULL;
  uint numLeaves = 0;
  uint* soup = NULL;
  uint numRefs = 0;
  vec3f res;
  res.x = (float)rx; res.y = (float)ry; res.z = (float)rz;
  vec3f mn, mx;
  mn.x = bounds[0]; mn.y = bounds[1]; mn.z = bounds[2];
  mx.x = bounds[3]; mx.y = bounds[4]; mx.z = bounds[5];
  TwoLevelGridBuilderHost::hostBuild(cells, leaves, numLeaves, soup, numRefs, rx, ry, rz, res, mn,
                                     mx, o->facesBegin(), o->facesEnd(), *o);
  RefGrid* g = new RefGrid();
  const size_t C = (size_t)rx * ry * rz;
  g->cells.resize(2 * C);
  for (size_t c = 0; c < C; ++c) {
    g->cells[2 * c] = cells[c].data.x;
    g->cells[2 * c + 1] = cells[c].data.y;
  }
  g->leaves.resize(2 * (size_t)numLeaves);
  for (size_t l = 0; l < numLeaves; ++l) {
    g->leaves[2 * l] = leaves[l].x;
    g->leaves[2 * l + 1] = leaves[l].y;
  }
  g->refs.assign(soup, soup + numRefs);
  delete[] cells;
  delete[] leaves;
  delete[] soup;
  delete o;
  sizes[0] = C;
  sizes[1] = numLeaves;
  sizes[2] = numRefs;
  return g;
}

void ref_host_build_copy(void* h, uint32_t* cells, uint32_t* leaves, uint32_t* refs) {
  RefGrid* g = (RefGrid*)h;
  memcpy(cells, g->cells.data(), g->cells.size() * 4);
  memcpy(leaves, g->leaves.data(), g->leaves.size() * 4);
  memcpy(refs, g->refs.data(), g->refs.size() * 4);
}

void ref_host_build_free(void* h) { delete (RefGrid*)h; }

// Camera::init (src/Primitive/Camera.h:41-60): {topLeft, stepX, stepY}.
void ref_camera(const float eye[3], const float fwd[3], const float up[3], float fov,
                uint32_t resx, uint32_t resy, float out[9]) {
  Camera c;
  vec3f e, f, u;
  e.x = eye[0]; e.y = eye[1]; e.z = eye[2];
  f.x = fwd[0]; f.y = fwd[1]; f.z = fwd[2];
  u.x = up[0]; u.y = up[1]; u.z = up[2];
  c.init(e, f, u, fov, resx, resy);
  out[0] = c.mTopLeft.x; out[1] = c.mTopLeft.y; out[2] = c.mTopLeft.z;
  out[3] = c.mStepX.x; out[4] = c.mStepX.y; out[5] = c.mStepX.z;
  out[6] = c.mStepY.x; out[7] = c.mStepY.y; out[8] = c.mStepY.z;
}

// RegularPixelSampler<1,1>::getPixelCoords + Camera::getDirection
// (src/Primitive/PixelSampler.h:40-52, src/Primitive/Camera.h:67-70).
void ref_primary_dirs(const float cam[9], uint32_t resx, uint32_t resy, uint32_t image_id,
                      const uint32_t* ids, uint32_t n, float* out) {
  Camera c;
  c.mTopLeft.x = cam[0]; c.mTopLeft.y = cam[1]; c.mTopLeft.z = cam[2];
  c.mStepX.x = cam[3]; c.mStepX.y = cam[4]; c.mStepX.z = cam[5];
  c.mStepY.x = cam[6]; c.mStepY.y = cam[7]; c.mStepY.z = cam[8];
  RegularPixelSampler<1, 1> s;
  s.resX = (float)resx;
  s.resY = (float)resy;
  for (uint32_t i = 0; i < n; ++i) {
    float px, py;
    s.getPixelCoords((float)ids[i], (float)image_id, px, py);
    vec3f d = c.getDirection(px, py);
    out[3 * i] = d.x; out[3 * i + 1] = d.y; out[3 * i + 2] = d.z;
  }
}

// Brute-force closest hit with the reference's Moller-Trumbore test, in the
// reciprocal-direction form the traversers call
// (src/Intersector/SimpleIntersector.hpp:38-89, 326-337).
void ref_mt_closest(const float* vtx, const uint32_t* idx, uint32_t nt, const float* org,
                    const float* dir, uint32_t n, uint32_t* tri, float* t) {
  HostSoup soup{vtx, idx};
  SimpleIntersector<HostSoup> isect;
  uint2 range;
  range.x = 0;
  range.y = nt;
  for (uint32_t i = 0; i < n; ++i) {
    vec3f o, rcp;
    o.x = org[3 * i]; o.y = org[3 * i + 1]; o.z = org[3 * i + 2];
    rcp.x = 1.f / dir[3 * i]; rcp.y = 1.f / dir[3 * i + 1]; rcp.z = 1.f / dir[3 * i + 2];
    float rt = FLT_MAX;
    uint best = 0xFFFFFFFFu;
    isect(o, rcp, rt, range, soup, NULL, best);
    tri[i] = best;
    t[i] = rt;
  }
}

// CosineHemisphereSampler (src/Utils/HemisphereSamplers.hpp:54-72) on host.
void ref_cosine_sample(const float* u1, const float* u2, uint32_t n, float* out) {
  CosineHemisphereSampler s;
  for (uint32_t i = 0; i < n; ++i) {
    vec3f d = s(u1[i], u2[i]);
    out[3 * i] = d.x; out[3 * i + 1] = d.y; out[3 * i + 2] = d.z;
  }
}

// TwoLevelGridCell packing (src/Control/Structure/TwoLevelGrid.hpp:72-151).
void ref_cell_word(uint32_t rx, uint32_t ry, uint32_t rz, int not_empty, uint32_t leaf_begin,
                   uint32_t out[2]) {
  TwoLevelGridCell c;
  c.clear();
  c.setNotEmpty();
  if (!not_empty) c.setEmpty();
  c.setX(rx);
  c.setY(ry);
  c.setZ(rz);
  c.setLeafRangeBegin(leaf_begin);
  out[0] = c.data.x;
  out[1] = c.data.y;
}

// FWObject::read (src/Loaders/FWObjectReader.cpp:193-502): sizes = {vertices,
// faces, materials}; the object is returned for ref_obj_copy.
void* ref_obj_read(const char* path, uint64_t sizes[3]) {
  FWObject* o = new FWObject();
  o->read(path);
  sizes[0] = o->getNumVertices();
  sizes[1] = o->getNumFaces();
  sizes[2] = o->getNumMaterials();
  return o;
}

// vertices 3*nv, faces 3*nf (vert1..3), face material nf, per material
// diffuse rgb + specular rgb + Ns (7 floats).
void ref_obj_copy(void* h, float* vertices, uint64_t* faces, uint64_t* face_material, float* materials) {
  FWObject* o = (FWObject*)h;
  for (size_t i = 0; i < o->getNumVertices(); ++i) {
    const vec3f v = o->getVertex(i);
    vertices[3 * i] = v.x; vertices[3 * i + 1] = v.y; vertices[3 * i + 2] = v.z;
  }
  for (size_t i = 0; i < o->getNumFaces(); ++i) {
    const FWObject::Face f = o->getFace(i);
    faces[3 * i] = f.vert1; faces[3 * i + 1] = f.vert2; faces[3 * i + 2] = f.vert3;
    face_material[i] = f.material;
  }
  for (size_t m = 0; m < o->getNumMaterials(); ++m) {
    const FWObject::Material& mt = o->getMaterial(m);
    float* d = materials + 7 * m;
    d[0] = mt.diffuseCoeff.x; d[1] = mt.diffuseCoeff.y; d[2] = mt.diffuseCoeff.z;
    d[3] = mt.specularCoeff.x; d[4] = mt.specularCoeff.y; d[5] = mt.specularCoeff.z;
    d[6] = mt.specularExp;
  }
}

void ref_obj_free(void* h) { delete (FWObject*)h; }

// CameraManager::read (src/Loaders/CameraManager.cpp:94-158) from the
// CameraManager defaults: out = position, orientation, up (after the file's
// rotation), FOV, resX, resY.
void ref_camera_read(const char* path, float out[12]) {
  CameraManager c;
  c.read(path);
  const vec3f p = c.getPosition(), o = c.getOrientation(), u = c.getUp();
  out[0] = p.x; out[1] = p.y; out[2] = p.z;
  out[3] = o.x; out[4] = o.y; out[5] = o.z;
  out[6] = u.x; out[7] = u.y; out[8] = u.z;
  out[9] = c.getFOV();
  out[10] = (float)c.getResX();
  out[11] = (float)c.getResY();
}

// LightSourceLoader::loadFromFile (src/Loaders/LightSourceLoader.cpp:26-89):
// out = position, edge1, edge2, normal, intensity.
void ref_light_read(const char* path, float out[15]) {
  LightSourceLoader l;
  const AreaLightSource a = l.loadFromFile(path);
  const vec3f v[5] = {a.position, a.edge1, a.edge2, a.normal, a.intensity};
  for (int k = 0; k < 5; ++k) {
    out[3 * k] = v[k].x; out[3 * k + 1] = v[k].y; out[3 * k + 2] = v[k].z;
  }
}

}  // extern "C"
