// C++ adapters with the reference's class and method names, forwarding to
// the C ABI in shinobi_b200.h (header only; link libshinobi_b200.so).
//
// The reference composes its ray tracer from compile-time policies
// (src/Engine/RayTracingTypes.h:76-128, src/Shinobi.h:49-116): a primitive
// storage (FaceSoup), a builder (FastSimpleGridBuilder /
// FastTwoLevelGridBuilder), a traverser + intersector pair running inside a
// persistent trace kernel, and an integrator (DirectIlluminationIntegrator,
// SimplePathTracer) driven by StaticRTEngine.  The classes below keep those
// names and the host-side method names and argument meanings, so an engine
// written against the reference's host interface moves over by changing its
// includes and its typedefs.  Differences that a caller sees:
//  * errors throw shinobi::Error (the reference aborts through cutil's
//    CUDA_SAFE_CALL);
//  * there is no global texture or constant state: grids are objects, any
//    number of them may live at once, and every call names its grid;
//  * traversal and intersection are fused in the library's kernels (the
//    watertight test replaces Moller-Trumbore), so UniformGridTraverser /
//    TwoLevelGridTraverser are host objects that launch a trace over a ray
//    buffer instead of device functors;
//  * FWObject is a minimal host mesh with the reference's accessors
//    (src/Loaders/FWObject.hpp:40-285), without the OBJ reader.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <ostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "../shinobi_b200.h"

// Same declaration as the CUDA runtime's (driver_types.h), so this header
// needs no CUDA include path; streams are passed through as void*.
struct CUstream_st;
typedef CUstream_st* cudaStream_t;

namespace shinobi {

class Error : public std::runtime_error {
 public:
  Error(shn_status s, const std::string& what)
      : std::runtime_error(what + ": " + shn_status_string(s)), status(s) {}
  shn_status status;
};

inline void check(shn_status s, const char* what, const shn_ctx* ctx = nullptr) {
  if (s == SHN_OK) return;
  std::string w(what);
  if (ctx) {
    const char* e = shn_ctx_last_error(ctx);
    if (e && *e) w += std::string(" (") + e + ")";
  }
  throw Error(s, w);
}

struct vec3f {
  float x, y, z;
};

struct BBox {
  vec3f min, max;
};

// ---- host mesh (src/Loaders/FWObject.hpp:40-285) ------------------------------
class FWObject {
 public:
  struct Face {
    size_t vert1, vert2, vert3;
    size_t material = 0;
  };
  // after Material::setupPhongCoefficients, as FWObject::read leaves them
  struct Material {
    std::string name;
    vec3f diffuseCoeff{0.f, 0.f, 0.f}, specularCoeff{0.f, 0.f, 0.f};
    float specularExp = 0.f;
  };
  typedef const Face* t_FaceIterator;

  void allocateVertices(size_t n) { mVertices.resize(n); }
  void allocateFaces(size_t n) { mFaces.resize(n); }
  size_t getNumVertices() const { return mVertices.size(); }
  size_t getNumFaces() const { return mFaces.size(); }
  size_t getNumMaterials() const { return mMaterials.size(); }
  vec3f getVertex(size_t i) const { return mVertices[i]; }
  vec3f& getVertex(size_t i) { return mVertices[i]; }
  Face getFace(size_t i) const { return mFaces[i]; }
  Face& getFace(size_t i) { return mFaces[i]; }
  const Material& getMaterial(size_t i) const { return mMaterials[i]; }
  t_FaceIterator facesBegin() const { return mFaces.data(); }
  t_FaceIterator facesEnd() const { return mFaces.data() + mFaces.size(); }

  // FWObject::read (src/Loaders/FWObjectReader.cpp:193-502): Wavefront OBJ
  // with its MTL libraries, through shn_obj_read.
  void read(const char* aFileName) {
    shn_obj* o = nullptr;
    if (shn_obj_read(aFileName, &o) != SHN_OK) throw Error(SHN_ERR_INVALID, std::string("FWObject::read: ") + aFileName);
    shn_obj_info inf;
    shn_obj_get_info(o, &inf);
    std::vector<float> v(3 * (size_t)inf.num_vertices), d(4 * (size_t)inf.num_materials),
        sp(4 * (size_t)inf.num_materials);
    std::vector<uint32_t> f(3 * (size_t)inf.num_faces), fm(inf.num_faces);
    shn_obj_copy(o, v.data(), f.data(), fm.data(), d.data(), sp.data());
    mVertices.resize(inf.num_vertices);
    for (size_t i = 0; i < mVertices.size(); ++i) mVertices[i] = vec3f{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    mFaces.resize(inf.num_faces);
    for (size_t i = 0; i < mFaces.size(); ++i) mFaces[i] = Face{f[3 * i], f[3 * i + 1], f[3 * i + 2], fm[i]};
    mMaterials.resize(inf.num_materials);
    for (size_t m = 0; m < mMaterials.size(); ++m) {
      const char* name = shn_obj_material_name(o, (uint32_t)m);
      mMaterials[m].name = name ? name : "";
      mMaterials[m].diffuseCoeff = vec3f{d[4 * m], d[4 * m + 1], d[4 * m + 2]};
      mMaterials[m].specularCoeff = vec3f{sp[4 * m], sp[4 * m + 1], sp[4 * m + 2]};
      mMaterials[m].specularExp = sp[4 * m + 3];
    }
    shn_obj_destroy(o);
  }

 private:
  std::vector<vec3f> mVertices;
  std::vector<Face> mFaces;
  std::vector<Material> mMaterials;
};

// ---- device context ------------------------------------------------------------
// The reference uses the current CUDA device implicitly; the adapters share
// one library context per process unless a Context is passed explicitly.
class Context {
 public:
  explicit Context(int device = 0, uint64_t hbm_budget_bytes = 0) {
    check(shn_ctx_create(device, hbm_budget_bytes, &mCtx), "shn_ctx_create");
  }
  ~Context() { shn_ctx_destroy(mCtx); }
  Context(const Context&) = delete;
  Context& operator=(const Context&) = delete;
  shn_ctx* get() const { return mCtx; }

  static Context& instance() {
    static Context c;
    return c;
  }

 private:
  shn_ctx* mCtx = nullptr;
};

// ---- primitive storage (src/Control/Structure/FaceSoup.h:41-346) ------------------
class FaceSoup {
 public:
  explicit FaceSoup(Context& ctx = Context::instance()) : mCtx(&ctx) {}
  ~FaceSoup() { cleanup(); }
  FaceSoup(const FaceSoup&) = delete;
  FaceSoup& operator=(const FaceSoup&) = delete;

  // FaceSoup::upload (FaceSoup.h:171-247): triangles [aBegin, aEnd) of aData.
  void upload(FWObject::t_FaceIterator aBegin, FWObject::t_FaceIterator aEnd, const FWObject& aData,
              cudaStream_t aStream = 0) {
    cleanup();
    flatten(aData, &mVtx);
    mIdx.clear();
    for (FWObject::t_FaceIterator it = aBegin; it != aEnd; ++it) {
      mIdx.push_back((uint32_t)it->vert1);
      mIdx.push_back((uint32_t)it->vert2);
      mIdx.push_back((uint32_t)it->vert3);
    }
    check(shn_scene_create(mCtx->get(), mVtx.data(), (uint32_t)(mVtx.size() / 3), mIdx.data(),
                           (uint32_t)(mIdx.size() / 3), SHN_MEM_HOST, aStream, &mScene),
          "FaceSoup::upload", mCtx->get());
  }

  // FaceSoup::uploadVertices (FaceSoup.h:249-339): vertices interpolated
  // between two key frames, new bounds returned.
  void uploadVertices(const FWObject& aKeyFrame1, const FWObject& aKeyFrame2, float aCoeff,
                      cudaStream_t aStream, vec3f& oMinBound, vec3f& oMaxBound) {
    if (!mScene) throw Error(SHN_ERR_NOT_BUILT, "FaceSoup::uploadVertices before upload");
    const size_t nv = aKeyFrame1.getNumVertices();
    if (aKeyFrame2.getNumVertices() != nv || 3 * nv != mVtx.size())
      throw Error(SHN_ERR_INVALID, "FaceSoup::uploadVertices: vertex counts differ");
    const float omc = 1.f - aCoeff;
    for (size_t i = 0; i < nv; ++i) {
      const vec3f a = aKeyFrame1.getVertex(i), b = aKeyFrame2.getVertex(i);
      mVtx[3 * i + 0] = a.x * omc + b.x * aCoeff;  // the reference's order of operations
      mVtx[3 * i + 1] = a.y * omc + b.y * aCoeff;
      mVtx[3 * i + 2] = a.z * omc + b.z * aCoeff;
    }
    check(shn_scene_update_vertices(mScene, mVtx.data(), (uint32_t)nv, SHN_MEM_HOST, aStream),
          "FaceSoup::uploadVertices", mCtx->get());
    const BBox b = getBounds();
    oMinBound = b.min;
    oMaxBound = b.max;
  }

  void cleanup() {
    if (mScene) shn_scene_destroy(mScene);
    mScene = nullptr;
  }

  BBox getBounds() const {
    float b[6];
    check(shn_scene_bounds(mScene, b), "FaceSoup::getBounds");
    return BBox{{b[0], b[1], b[2]}, {b[3], b[4], b[5]}};
  }
  uint32_t getNumPrimitives() const { return mScene ? shn_scene_num_triangles(mScene) : 0u; }
  shn_scene* handle() const { return mScene; }
  Context& context() const { return *mCtx; }

 private:
  static void flatten(const FWObject& o, std::vector<float>* out) {
    out->resize(3 * o.getNumVertices());
    for (size_t i = 0; i < o.getNumVertices(); ++i) {
      const vec3f v = o.getVertex(i);
      (*out)[3 * i] = v.x;
      (*out)[3 * i + 1] = v.y;
      (*out)[3 * i + 2] = v.z;
    }
  }
  Context* mCtx;
  shn_scene* mScene = nullptr;
  std::vector<float> mVtx;
  std::vector<uint32_t> mIdx;
};

// ---- grids (src/Control/Structure/SimpleGrid.h, TwoLevelGrid.h) ---------------------
class GridBase {
 public:
  explicit GridBase(Context& ctx) : mCtx(&ctx) { check(shn_grid_create(ctx.get(), &mGrid), "shn_grid_create"); }
  ~GridBase() { shn_grid_destroy(mGrid); }
  GridBase(const GridBase&) = delete;
  GridBase& operator=(const GridBase&) = delete;

  shn_grid_info info() const {
    shn_grid_info i;
    check(shn_grid_get_info(mGrid, &i), "grid info");
    return i;
  }
  vec3f getResolution() const {
    const shn_grid_info i = info();
    return vec3f{(float)i.res[0], (float)i.res[1], (float)i.res[2]};
  }
  BBox bounds() const {
    const shn_grid_info i = info();
    return BBox{{i.bounds[0], i.bounds[1], i.bounds[2]}, {i.bounds[3], i.bounds[4], i.bounds[5]}};
  }
  shn_grid* handle() const { return mGrid; }
  Context& context() const { return *mCtx; }

 protected:
  Context* mCtx;
  shn_grid* mGrid = nullptr;
};

class SimpleGrid : public GridBase {
 public:
  explicit SimpleGrid(Context& ctx = Context::instance()) : GridBase(ctx) {}
};

class TwoLevelGrid : public GridBase {
 public:
  explicit TwoLevelGrid(Context& ctx = Context::instance()) : GridBase(ctx) {}
};

// ---- builders (src/Control/Algorithm/FastSimpleGridBuilder.h:44-470,
//                FastTwoLevelGridBuilder.h:46-760) -------------------------------------
template <class Grid, uint32_t KIND>
class GridBuilderT {
 public:
  GridBuilderT() { shn_grid_params_default(KIND, &mParams); }

  void setNumPrimitives(uint32_t aNum) { mNumPrimitives = aNum; }
  // Parameters the reference fixes at compile time.
  shn_grid_params& params() { return mParams; }

  // init: uploads the faces into the storage (and measures the bounds).
  void init(Grid& oGrid, FaceSoup& oFaceSoup, FWObject::t_FaceIterator aBegin,
            FWObject::t_FaceIterator aEnd, const FWObject& aData) {
    (void)oGrid;
    oFaceSoup.upload(aBegin, aEnd, aData);
    mNumPrimitives = oFaceSoup.getNumPrimitives();
  }

  // build: the whole grid construction on the default stream.
  void build(Grid& oGrid, FaceSoup& oFaceSoup) { rebuild(oGrid, oFaceSoup, nullptr); }

  // rebuild: construction over the storage's current vertices on aStream
  // (the reference's dynamic-scene path).
  void rebuild(Grid& oGrid, FaceSoup& oFaceSoup, cudaStream_t aStream) {
    check(shn_grid_build(oGrid.handle(), oFaceSoup.handle(), &mParams, aStream), "grid build",
          oGrid.context().get());
    mLastGrid = &oGrid;  // statistics are read when asked for (the build's last stage runs on)
  }

  void cleanup() {}

  void outputStats(std::ostream& os) const {
    const shn_grid_info last = mLastGrid ? mLastGrid->info() : shn_grid_info{};
    os << "Grid resolution: " << last.res[0] << " " << last.res[1] << " " << last.res[2] << "\n"
       << "Number of references: " << last.num_refs << "\n";
    if (KIND == SHN_GRID_TWO_LEVEL) os << "Number of leaf cells: " << last.num_leaves << "\n";
    os << "Build time (ms): " << last.build_ms << "\n";
  }

 protected:
  uint32_t mNumPrimitives = 0;
  shn_grid_params mParams;
  const Grid* mLastGrid = nullptr;
};

typedef GridBuilderT<SimpleGrid, SHN_GRID_UNIFORM> FastSimpleGridBuilder;
typedef GridBuilderT<TwoLevelGrid, SHN_GRID_TWO_LEVEL> FastTwoLevelGridBuilder;

// SAHGridBuilder (src/Control/Algorithm/SAHGridBuilder.h:38-202): the uniform
// sort-based build at the resolution of least SAH cost in the window 0.75 ..
// 1.25 around the lambda = 5 estimate (computeResolution), counted on the
// device in one launch.
class SAHGridBuilder : public GridBuilderT<SimpleGrid, SHN_GRID_UNIFORM> {
 public:
  // computeResolution: fixes params().res for the builds that follow.
  shn_sah_result computeResolution(FaceSoup& oFaceSoup, cudaStream_t aStream = nullptr) {
    shn_sah_result r{};
    check(shn_grid_sah_resolution(oFaceSoup.handle(), 5.f, 0.75f, 1.25f, nullptr, 0, &r, aStream),
          "SAH resolution", oFaceSoup.context().get());
    for (int k = 0; k < 3; ++k) mParams.res[k] = r.res[k];
    return r;
  }
  void build(SimpleGrid& oGrid, FaceSoup& oFaceSoup) {
    computeResolution(oFaceSoup);
    rebuild(oGrid, oFaceSoup, nullptr);
  }
};

// ---- traversers (SimpleGridTraverser.h:249-469, TwoLevelGridTraverser.h:430-828) ------
// The reference's traverser + SimpleIntersector pair, fused: closest hit for
// the *Traverser classes, any hit for the *ShadowTraverser classes.  Rays and
// results are device SoA buffers (shn_rays / shn_hits).
struct ClosestTraverser {
  void traverse(const GridBase& aGrid, const shn_rays& aRays, uint32_t aNumRays, shn_hits& oHits,
                cudaStream_t aStream = 0) const {
    check(shn_trace_closest(aGrid.handle(), &aRays, aNumRays, &oHits, aStream), "traverse",
          aGrid.context().get());
  }
};
struct ShadowTraverser {
  void traverse(const GridBase& aGrid, const shn_rays& aRays, uint32_t aNumRays, uint8_t* oOccluded,
                cudaStream_t aStream = 0) const {
    check(shn_trace_any(aGrid.handle(), &aRays, aNumRays, oOccluded, aStream), "traverse (any hit)",
          aGrid.context().get());
  }
};
typedef ClosestTraverser UniformGridTraverser;
typedef ClosestTraverser TwoLevelGridTraverser;
typedef ShadowTraverser UniformGridShadowTraverser;
typedef ShadowTraverser TwoLevelGridShadowTraverser;

// ---- camera (src/Primitive/Camera.h:34-70) --------------------------------------------
class Camera {
 public:
  void init(const vec3f& aCenter, const vec3f& aForward, const vec3f& aUp, float aVertOpeningAngInGrad,
            uint32_t aResX, uint32_t aResY) {
    const float c[9] = {aCenter.x, aCenter.y, aCenter.z, aForward.x, aForward.y, aForward.z, aUp.x, aUp.y, aUp.z};
    memcpy(mCam.eye, c, sizeof(mCam.eye));
    memcpy(mCam.forward, c + 3, sizeof(mCam.forward));
    memcpy(mCam.up, c + 6, sizeof(mCam.up));
    mCam.fov_deg = aVertOpeningAngInGrad;
    mCam.res_x = aResX;
    mCam.res_y = aResY;
  }
  const shn_camera& params() const { return mCam; }
  uint32_t resX() const { return mCam.res_x; }
  uint32_t resY() const { return mCam.res_y; }

 private:
  shn_camera mCam{};
};

// CameraManager::read (src/Loaders/CameraManager.cpp:94-158): the camera of a
// camera.cfg file, from the reference's CameraManager defaults.
class CameraManager {
 public:
  void read(const char* aFileName) {
    shn_camera c{};
    c.forward[2] = 1.f;
    c.up[1] = -1.f;
    c.fov_deg = 66.f;
    c.res_x = c.res_y = 512u;
    if (shn_camera_read(aFileName, &c) != SHN_OK) throw Error(SHN_ERR_INVALID, std::string("CameraManager::read: ") + aFileName);
    mCam = c;
  }
  vec3f getPosition() const { return vec3f{mCam.eye[0], mCam.eye[1], mCam.eye[2]}; }
  vec3f getOrientation() const { return vec3f{mCam.forward[0], mCam.forward[1], mCam.forward[2]}; }
  vec3f getUp() const { return vec3f{mCam.up[0], mCam.up[1], mCam.up[2]}; }
  float getFOV() const { return mCam.fov_deg; }
  uint32_t getResX() const { return mCam.res_x; }
  uint32_t getResY() const { return mCam.res_y; }

 private:
  shn_camera mCam{};
};

// ---- integrators (src/Integrator/DirectIlluminationIntegrator.h:197-362,
//                   src/Integrator/SimplePathTracer.hpp:65-241) ------------------------
// Device buffers (cudaMalloc'd by the caller) for one frame.
struct FrameBuffer {
  float* deviceData = nullptr;  // resX*resY floats (ambient occlusion) or *3 (radiance)
  uint32_t resX = 0, resY = 0;
};

// AreaLightSource (src/Primitive/LightSource.hpp:35-51): a parallelogram
// position + a*edge1 + b*edge2, emitting towards -normal.
struct AreaLightSource {
  vec3f position{-0.05f, 0.2f, -0.05f}, normal{0.f, -1.f, 0.f}, intensity{10.f, 10.f, 10.f},
      edge1{0.1f, 0.f, 0.f}, edge2{0.f, 0.f, 0.1f};
};

// LightSourceLoader::loadFromFile (src/Loaders/LightSourceLoader.cpp:26-89).
struct LightSourceLoader {
  AreaLightSource loadFromFile(const char* aFileName) {
    shn_area_light l;
    if (shn_light_read(aFileName, &l) != SHN_OK) throw Error(SHN_ERR_INVALID, std::string("LightSourceLoader: ") + aFileName);
    AreaLightSource a;
    a.position = vec3f{l.position[0], l.position[1], l.position[2]};
    a.normal = vec3f{l.normal[0], l.normal[1], l.normal[2]};
    a.intensity = vec3f{l.intensity[0], l.intensity[1], l.intensity[2]};
    a.edge1 = vec3f{l.edge1[0], l.edge1[1], l.edge1[2]};
    a.edge2 = vec3f{l.edge2[0], l.edge2[1], l.edge2[2]};
    return a;
  }
};

// MaterialContainer (src/Primitive/Material.h:36-46) with the per-face
// material ids of FaceSoup::getMaterialId (src/Control/Structure/FaceSoup.h:165).
// Device pointers owned by the caller; null diffuse = defaultDiffuse everywhere.
struct MaterialContainer {
  const float* diffuseDevice = nullptr;        // 4 floats per material (.w unused)
  uint32_t numMaterials = 0;
  const uint32_t* faceMaterialDevice = nullptr;  // per triangle; null = material 0
  vec3f defaultDiffuse{0.7f, 0.7f, 0.7f};
};

// DirectIlluminationIntegrator: primary closest-hit rays, then
// numOcclusionSamples shadow rays per hit pixel to the area light and the
// per-pixel shading of computeDirectIllumination with the progressive blend
// into the final image.  ambientOcclusion() is the C1 form: cosine-weighted
// any-hit rays of occlusionLength, one visibility fraction per pixel.
class DirectIlluminationIntegrator {
 public:
  uint32_t numOcclusionSamples = 4;  // NUMOCCLUSIONSAMPLES
  uint32_t seed = 1;
  AreaLightSource lightSource;
  float occlusionLength = 0.1f;
  float originOffset = 1e-4f;

  // tracePrimary: hits (device, resX*resY) for the camera.
  void tracePrimary(const GridBase& aGrid, const Camera& aCamera, shn_hits& oHits, int aImageId,
                    cudaStream_t aStream = 0) {
    check(shn_trace_primary(aGrid.handle(), &aCamera.params(), (uint32_t)aImageId, &oHits, aStream),
          "tracePrimary", aGrid.context().get());
  }
  // shade: oFrameBuffer = this image's radiance (RGB per pixel); oFinalImage
  // (may have null deviceData) = running mean over image ids 0..aImageId.
  // the shading parameters of this integrator for one image
  shn_di_params params(const MaterialContainer& aMaterials, int aImageId) const {
    shn_di_params p;
    shn_di_params_default(&p);
    const vec3f* lv[5] = {&lightSource.position, &lightSource.edge1, &lightSource.edge2, &lightSource.normal,
                          &lightSource.intensity};
    float* dst[5] = {p.light.position, p.light.edge1, p.light.edge2, p.light.normal, p.light.intensity};
    for (int i = 0; i < 5; ++i) {
      dst[i][0] = lv[i]->x;
      dst[i][1] = lv[i]->y;
      dst[i][2] = lv[i]->z;
    }
    p.samples = numOcclusionSamples;
    p.seed = seed;
    p.image_id = (uint32_t)aImageId;
    p.tri_material = aMaterials.faceMaterialDevice;
    p.diffuse = aMaterials.diffuseDevice;
    p.num_materials = aMaterials.numMaterials;
    p.default_diffuse[0] = aMaterials.defaultDiffuse.x;
    p.default_diffuse[1] = aMaterials.defaultDiffuse.y;
    p.default_diffuse[2] = aMaterials.defaultDiffuse.z;
    return p;
  }
  void shade(const GridBase& aGrid, const Camera& aCamera, const shn_hits& aPrimary,
             const MaterialContainer& aMaterials, FrameBuffer& oFrameBuffer, FrameBuffer& oFinalImage,
             int aImageId, cudaStream_t aStream = 0) {
    const shn_di_params p = params(aMaterials, aImageId);
    check(shn_shade_direct(aGrid.handle(), &aCamera.params(), &aPrimary, &p, oFrameBuffer.deviceData,
                           oFinalImage.deviceData, nullptr, aStream),
          "shade", aGrid.context().get());
  }
  void integrate(const GridBase& aGrid, const Camera& aCamera, shn_hits& oHits, const MaterialContainer& aMaterials,
                 FrameBuffer& oFrameBuffer, FrameBuffer& oFinalImage, int aImageId, cudaStream_t aStream = 0) {
    tracePrimary(aGrid, aCamera, oHits, aImageId, aStream);
    shade(aGrid, aCamera, oHits, aMaterials, oFrameBuffer, oFinalImage, aImageId, aStream);
  }
  // ambientOcclusion: oFrame = visible fraction of the occlusion rays per pixel.
  void ambientOcclusion(const GridBase& aGrid, const Camera& aCamera, const shn_hits& aPrimary, FrameBuffer& oFrame,
                        cudaStream_t aStream = 0) {
    check(shn_trace_ao(aGrid.handle(), &aCamera.params(), &aPrimary, numOcclusionSamples, occlusionLength,
                       originOffset, seed, oFrame.deviceData, nullptr, aStream),
          "ambientOcclusion", aGrid.context().get());
  }
  void cleanup() {}
};

// Wavefront path tracer with compaction after every bounce.
class SimplePathTracer {
 public:
  SimplePathTracer() { shn_pt_params_default(&mParams); }
  shn_pt_params& params() { return mParams; }
  void integrate(const GridBase& aGrid, const FaceSoup& aStorage, const Camera& aCamera, FrameBuffer& oFrame,
                 cudaStream_t aStream = 0, uint32_t* oBounceStats = nullptr) {
    check(shn_pt_render(aGrid.handle(), aStorage.handle(), &aCamera.params(), &mParams, oFrame.deviceData,
                        oBounceStats, aStream),
          "SimplePathTracer::integrate", aGrid.context().get());
  }
  void cleanup() {}

 private:
  shn_pt_params mParams;
};

// ---- engine (src/Engine/StaticRTEngine.h:34-237) ---------------------------------------
template <class Builder, class Grid>
class StaticRTEngine {
 public:
  void init(const FWObject& aScene, Context& ctx = Context::instance()) {
    mStorage.reset(new FaceSoup(ctx));
    mGrid.reset(new Grid(ctx));
    mBuilder.init(*mGrid, *mStorage, aScene.facesBegin(), aScene.facesEnd(), aScene);
  }
  void build() { mBuilder.build(*mGrid, *mStorage); }
  void renderImage(DirectIlluminationIntegrator& aIntegrator, const Camera& aCamera, shn_hits& oHits,
                   const MaterialContainer& aMaterials, FrameBuffer& oFrameBuffer, FrameBuffer& oFinalImage,
                   int aImageId, cudaStream_t aStream = 0) {
    aIntegrator.integrate(*mGrid, aCamera, oHits, aMaterials, oFrameBuffer, oFinalImage, aImageId, aStream);
  }
  Builder& builder() { return mBuilder; }
  Grid& grid() { return *mGrid; }
  FaceSoup& storage() { return *mStorage; }

 private:
  Builder mBuilder;
  std::unique_ptr<FaceSoup> mStorage;
  std::unique_ptr<Grid> mGrid;
};

// ---- dynamic engine (src/Engine/DynamicRTEngine.h:49-158) -----------------------------
// Two frame slots: renderFrame renders the geometry prepared by the previous
// call while the keyframe interpolation of the next frame and its rebuild run
// on the other slot's stream.  The keyframes are device arrays (3 floats per
// vertex); FaceSoup::uploadVertices's host upload is the caller's copy.
class DynamicRTEngine {
 public:
  DynamicRTEngine() = default;
  ~DynamicRTEngine() { shn_dynamic_destroy(mEngine); }
  DynamicRTEngine(const DynamicRTEngine&) = delete;
  DynamicRTEngine& operator=(const DynamicRTEngine&) = delete;

  void init(const FWObject& aScene, const shn_grid_params& aParams, Context& ctx = Context::instance()) {
    std::vector<float> v(3 * aScene.getNumVertices());
    for (size_t i = 0; i < aScene.getNumVertices(); ++i) {
      const vec3f p = aScene.getVertex(i);
      v[3 * i] = p.x;
      v[3 * i + 1] = p.y;
      v[3 * i + 2] = p.z;
    }
    std::vector<uint32_t> idx(3 * aScene.getNumFaces());
    for (size_t i = 0; i < aScene.getNumFaces(); ++i) {
      const FWObject::Face f = aScene.getFace(i);
      idx[3 * i] = (uint32_t)f.vert1;
      idx[3 * i + 1] = (uint32_t)f.vert2;
      idx[3 * i + 2] = (uint32_t)f.vert3;
    }
    shn_dynamic_destroy(mEngine);
    mEngine = nullptr;
    mCtx = &ctx;
    check(shn_dynamic_create(ctx.get(), v.data(), (uint32_t)aScene.getNumVertices(), idx.data(),
                             (uint32_t)aScene.getNumFaces(), SHN_MEM_HOST, &aParams, &mEngine),
          "DynamicRTEngine::init", ctx.get());
  }
  // renderFrame: oHits / oFrameBuffer / oFinalImage as for
  // DirectIlluminationIntegrator::integrate; oRenderTime / oBuildTime in ms.
  void renderFrame(const float* aKeyFrame1Device, uint32_t aNumVertices1, const float* aKeyFrame2Device,
                   float aCoeff, DirectIlluminationIntegrator& aIntegrator, const Camera& aCamera,
                   const MaterialContainer& aMaterials, shn_hits& oHits, FrameBuffer& oFrameBuffer,
                   FrameBuffer& oFinalImage, int aImageId, float& oRenderTime, float& oBuildTime) {
    shn_di_params p = aIntegrator.params(aMaterials, aImageId);
    check(shn_dynamic_render_frame(mEngine, aKeyFrame1Device, aNumVertices1, aKeyFrame2Device, aCoeff,
                                   &aCamera.params(), &p, &oHits, oFrameBuffer.deviceData, oFinalImage.deviceData,
                                   &oRenderTime, &oBuildTime, nullptr),
          "DynamicRTEngine::renderFrame", mCtx ? mCtx->get() : nullptr);
  }

 private:
  shn_dynamic* mEngine = nullptr;
  Context* mCtx = nullptr;
};

}  // namespace shinobi
