// Drives the C++ adapters (include/shinobi/shinobi.hpp) the way an engine
// written against the reference's host interface would: FWObject ->
// FaceSoup::upload -> Fast*GridBuilder / SAHGridBuilder::init/build ->
// StaticRTEngine::renderImage (DirectIlluminationIntegrator::tracePrimary +
// shade).  Usage:
//   adapter_example <scene.bin> <out.bin> <kind 0|1|2> <res_x> <res_y>
// kind 0: uniform grid, 1: two-level grid, 2: uniform grid at the SAH resolution.
// scene.bin: uint32 nv, uint32 nt, nv*3 float, nt*3 uint32.
// out.bin:   res_x*res_y uint32 triangle ids, res_x*res_y float t, then the
//            res_x*res_y*3 float direct-illumination frame.
// Exit code 3 (after printing "no device") when no CUDA device is usable.
#include <cstdio>
#include <cstdlib>
#include <iostream>
#include <type_traits>
#include <vector>

#include "shinobi/shinobi.hpp"

#include <cuda_runtime_api.h>

template <class Builder, class Grid>
static int run(shinobi::FWObject& obj, const char* out_path, uint32_t rx, uint32_t ry) {
  shinobi::Context& ctx = shinobi::Context::instance();
  shinobi::StaticRTEngine<Builder, Grid> engine;
  engine.init(obj, ctx);
  if (std::is_same<Grid, shinobi::TwoLevelGrid>::value) {
    engine.builder().params().lambda = 1.0f / 16.0f;
    engine.builder().params().top_divisor = 1;
    engine.builder().params().min_res = 2;
    engine.builder().params().lambda_leaf = 4.0f;
  }
  engine.build();
  shinobi::Camera cam;
  cam.init(shinobi::vec3f{0.5f, 0.5f, -1.5f}, shinobi::vec3f{0.f, 0.f, 1.f}, shinobi::vec3f{0.f, 1.f, 0.f}, 45.f,
           rx, ry);
  const size_t n = (size_t)rx * ry;
  uint32_t* d_tri = nullptr;
  float* d_t = nullptr;
  cudaMalloc((void**)&d_tri, 4 * n);
  cudaMalloc((void**)&d_t, 4 * n);
  shn_hits hits{d_tri, d_t, nullptr, nullptr};
  float* d_frame = nullptr;
  float* d_final = nullptr;
  cudaMalloc((void**)&d_frame, 12 * n);
  cudaMalloc((void**)&d_final, 12 * n);
  cudaMemset(d_final, 0, 12 * n);
  shinobi::DirectIlluminationIntegrator integ;
  integ.lightSource.position = shinobi::vec3f{0.3f, 1.2f, 0.3f};
  integ.lightSource.edge1 = shinobi::vec3f{0.4f, 0.f, 0.f};
  integ.lightSource.edge2 = shinobi::vec3f{0.f, 0.f, 0.4f};
  integ.lightSource.intensity = shinobi::vec3f{4.f, 4.f, 4.f};
  shinobi::MaterialContainer materials;
  shinobi::FrameBuffer frame{d_frame, rx, ry}, final_image{d_final, rx, ry};
  engine.renderImage(integ, cam, hits, materials, frame, final_image, 0);
  cudaDeviceSynchronize();
  std::vector<uint32_t> tri(n);
  std::vector<float> t(n), rgb(3 * n), acc(3 * n);
  cudaMemcpy(tri.data(), d_tri, 4 * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(t.data(), d_t, 4 * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(rgb.data(), d_frame, 12 * n, cudaMemcpyDeviceToHost);
  cudaMemcpy(acc.data(), d_final, 12 * n, cudaMemcpyDeviceToHost);
  cudaFree(d_tri);
  cudaFree(d_t);
  cudaFree(d_frame);
  cudaFree(d_final);
  for (size_t i = 0; i < 3 * n; ++i)
    if (acc[i] != rgb[i]) return 4;  // image 0: the final image equals the frame
  FILE* f = fopen(out_path, "wb");
  if (!f) return 1;
  fwrite(tri.data(), 4, n, f);
  fwrite(t.data(), 4, n, f);
  fwrite(rgb.data(), 4, 3 * n, f);
  fclose(f);
  engine.builder().outputStats(std::cout);
  return 0;
}

int main(int argc, char** argv) {
  if (argc != 6) {
    fprintf(stderr, "usage: %s scene.bin out.bin kind res_x res_y\n", argv[0]);
    return 2;
  }
  FILE* f = fopen(argv[1], "rb");
  if (!f) return 2;
  uint32_t nv = 0, nt = 0;
  if (fread(&nv, 4, 1, f) != 1 || fread(&nt, 4, 1, f) != 1) return 2;
  std::vector<float> v(3 * (size_t)nv);
  std::vector<uint32_t> idx(3 * (size_t)nt);
  if (fread(v.data(), 4, v.size(), f) != v.size() || fread(idx.data(), 4, idx.size(), f) != idx.size()) return 2;
  fclose(f);
  shinobi::FWObject obj;
  obj.allocateVertices(nv);
  for (uint32_t i = 0; i < nv; ++i) obj.getVertex(i) = shinobi::vec3f{v[3 * i], v[3 * i + 1], v[3 * i + 2]};
  obj.allocateFaces(nt);
  for (uint32_t i = 0; i < nt; ++i) obj.getFace(i) = shinobi::FWObject::Face{idx[3 * i], idx[3 * i + 1], idx[3 * i + 2]};
  const int kind = atoi(argv[3]);
  const uint32_t rx = (uint32_t)atoi(argv[4]), ry = (uint32_t)atoi(argv[5]);
  try {
    if (kind == 0) return run<shinobi::FastSimpleGridBuilder, shinobi::SimpleGrid>(obj, argv[2], rx, ry);
    if (kind == 2) return run<shinobi::SAHGridBuilder, shinobi::SimpleGrid>(obj, argv[2], rx, ry);
    return run<shinobi::FastTwoLevelGridBuilder, shinobi::TwoLevelGrid>(obj, argv[2], rx, ry);
  } catch (const shinobi::Error& e) {
    if (e.status == SHN_ERR_CUDA) {
      printf("no device: %s\n", e.what());
      return 3;
    }
    fprintf(stderr, "error: %s\n", e.what());
    return 1;
  }
}
