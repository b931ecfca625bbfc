// Dynamic scenes: the rebuild of the next frame overlapped with the render
// of the current one (DynamicRTEngine, src/Engine/DynamicRTEngine.h:49-158).
//
// Two frame slots, each a scene (FaceSoup) with its own grid, a render
// stream and a rebuild stream.  A frame renders the slot built during the previous frame (primary
// rays + direct illumination from an area light, DirectIlluminationIntegrator)
// on that slot's stream while, on the other slot's stream, the next frame's
// vertices are interpolated between two keyframes (FaceSoup::uploadVertices)
// and that slot's grid is rebuilt.  The GPU runs the two streams side by
// side; events order every reuse of a slot or of the caller's output
// buffers.  As in the reference, the frame rendered by a call shows the
// geometry of the previous call's keyframes (the first call renders the
// geometry the engine was created with).
//
// The reference binds one global grid-parameter constant and global
// textures, so its two slots share state; here each slot is a separate grid
// handle and the two never alias.
#include "internal.h"

struct shn_dynamic {
  shn_ctx* ctx = nullptr;
  shn_scene* scene[2] = {nullptr, nullptr};
  shn_grid* grid[2] = {nullptr, nullptr};
  cudaStream_t stream[2] = {nullptr, nullptr};   // per slot: its renders (lowest priority)
  cudaStream_t bstream[2] = {nullptr, nullptr};  // per slot: its rebuilds (highest priority)
  cudaEvent_t rendered[2] = {nullptr, nullptr};  // the slot's last render (outputs written, grid read)
  cudaEvent_t built[2] = {nullptr, nullptr};     // the slot's last rebuild
  cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};
  shn_grid_params params{};
  uint32_t nv = 0;
  uint32_t render_slot = 0;
};

using namespace shn;

namespace {

void destroy(shn_dynamic* e) {
  for (int s = 0; s < 2; ++s) {
    if (e->stream[s]) cudaStreamSynchronize(e->stream[s]);
    if (e->bstream[s]) cudaStreamSynchronize(e->bstream[s]);
  }
  for (int s = 0; s < 2; ++s) {
    if (e->grid[s]) shn_grid_destroy(e->grid[s]);
    if (e->scene[s]) shn_scene_destroy(e->scene[s]);
    if (e->rendered[s]) cudaEventDestroy(e->rendered[s]);
    if (e->built[s]) cudaEventDestroy(e->built[s]);
    if (e->stream[s]) cudaStreamDestroy(e->stream[s]);
    if (e->bstream[s]) cudaStreamDestroy(e->bstream[s]);
  }
  for (cudaEvent_t v : e->ev)
    if (v) cudaEventDestroy(v);
  if (e->ctx) ctx_release(e->ctx);
  delete e;
}

}  // namespace

extern "C" {

shn_status shn_dynamic_create(shn_ctx* ctx, const float* vtx_xyz, uint32_t nv, const uint32_t* idx, uint32_t nt,
                              uint32_t mem, const shn_grid_params* p, shn_dynamic** out) {
  if (!ctx || !p || !out) return SHN_ERR_INVALID;
  *out = nullptr;
  shn_dynamic* e = new shn_dynamic();
  e->ctx = ctx;
  ctx_retain(ctx);
  e->params = *p;
  e->nv = nv;
  shn_status rc = SHN_OK;
  // rebuilds get the device's highest stream priority, renders its lowest:
  // at every boundary between the render's kernels the pending rebuild
  // blocks are scheduled first, so the rebuild advances while the frame
  // renders instead of waiting for it to end
  int least = 0, greatest = 0;
  cudaDeviceGetStreamPriorityRange(&least, &greatest);
  for (int s = 0; s < 2 && rc == SHN_OK; ++s) {
    if (cudaStreamCreateWithPriority(&e->stream[s], cudaStreamNonBlocking, least) != cudaSuccess ||
        cudaStreamCreateWithPriority(&e->bstream[s], cudaStreamNonBlocking, greatest) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->rendered[s], cudaEventDisableTiming) != cudaSuccess ||
        cudaEventCreateWithFlags(&e->built[s], cudaEventDisableTiming) != cudaSuccess) {
      rc = set_error(ctx, SHN_ERR_CUDA, "dynamic engine streams");
      break;
    }
    rc = shn_scene_create(ctx, vtx_xyz, nv, idx, nt, mem, e->bstream[s], &e->scene[s]);
    if (rc == SHN_OK) rc = shn_grid_create(ctx, &e->grid[s]);
  }
  for (int i = 0; i < 4 && rc == SHN_OK; ++i)
    if (cudaEventCreate(&e->ev[i]) != cudaSuccess) rc = set_error(ctx, SHN_ERR_CUDA, "dynamic engine events");
  // DynamicRTEngine::init: slot 0 is built now and rendered by the first frame
  if (rc == SHN_OK) rc = shn_grid_build(e->grid[0], e->scene[0], &e->params, e->bstream[0]);
  for (int s = 0; s < 2 && rc == SHN_OK; ++s) {
    if (cudaEventRecord(e->built[s], e->bstream[s]) != cudaSuccess ||
        cudaEventRecord(e->rendered[s], e->stream[s]) != cudaSuccess)
      rc = set_error(ctx, SHN_ERR_CUDA, "dynamic engine events");
  }
  if (rc == SHN_OK && cudaStreamSynchronize(e->bstream[0]) != cudaSuccess)
    rc = set_error(ctx, SHN_ERR_CUDA, "dynamic engine initial build");
  if (rc != SHN_OK) {
    destroy(e);
    return rc;
  }
  *out = e;
  return SHN_OK;
}

shn_status shn_dynamic_render_frame(shn_dynamic* e, const float* d_kf1, uint32_t n1, const float* d_kf2,
                                    float coeff, const shn_camera* cam, const shn_di_params* di,
                                    shn_hits* hits, float* d_frame, float* d_final, float* render_ms,
                                    float* build_ms, float* frame_ms) {
  if (!e || !d_kf2 || !cam || !di || !hits || !d_frame || (n1 && !d_kf1) || n1 > e->nv) return SHN_ERR_INVALID;
  const uint32_t r = e->render_slot, u = 1u - r;
  cudaStream_t sr = e->stream[r], su = e->bstream[u];
  // slot r's grid comes from its last rebuild; the outputs were last written
  // by the other slot's render
  cudaStreamWaitEvent(sr, e->built[r], 0);
  cudaStreamWaitEvent(sr, e->rendered[u], 0);
  cudaEventRecord(e->ev[0], sr);
  shn_status rc = shn_trace_primary(e->grid[r], cam, di->image_id, hits, sr);
  if (rc == SHN_OK) rc = shn_shade_direct(e->grid[r], cam, hits, di, d_frame, d_final, nullptr, sr);
  cudaEventRecord(e->ev[1], sr);
  cudaEventRecord(e->rendered[r], sr);
  if (rc != SHN_OK) return rc;
  // the next frame's geometry and grid in the other slot, on that slot's
  // rebuild stream, after its last render (one frame ago) has read them
  cudaStreamWaitEvent(su, e->rendered[u], 0);
  cudaEventRecord(e->ev[2], su);
  rc = shn_scene_interpolate_vertices(e->scene[u], d_kf1, n1, d_kf2, coeff, su);
  if (rc == SHN_OK) rc = shn_grid_build(e->grid[u], e->scene[u], &e->params, su);
  cudaEventRecord(e->ev[3], su);
  cudaEventRecord(e->built[u], su);
  if (rc != SHN_OK) return rc;
  cudaError_t ce = cudaEventSynchronize(e->ev[1]);
  if (ce == cudaSuccess) ce = cudaEventSynchronize(e->ev[3]);
  if (ce != cudaSuccess) return cuda_status(e->ctx, ce, "dynamic frame");
  rc = shn_grid_sync_status(e->grid[r], sr);
  if (rc != SHN_OK) return rc;
  // render: ev0 -> ev1 (slot r's stream); rebuild: ev2 -> ev3 (slot u's);
  // the frame: from the earlier start to the later end
  float rd = 0.f, bd = 0.f, r_to_b_end = 0.f, r_to_b_start = 0.f;
  cudaEventElapsedTime(&rd, e->ev[0], e->ev[1]);
  cudaEventElapsedTime(&bd, e->ev[2], e->ev[3]);
  cudaEventElapsedTime(&r_to_b_end, e->ev[0], e->ev[3]);
  cudaEventElapsedTime(&r_to_b_start, e->ev[0], e->ev[2]);
  if (render_ms) *render_ms = rd;
  if (build_ms) *build_ms = bd;
  if (frame_ms) *frame_ms = std::max(rd, r_to_b_end) - std::min(0.f, r_to_b_start);
  e->render_slot = u;
  return SHN_OK;
}

shn_status shn_dynamic_get_grid(const shn_dynamic* e, uint32_t next, shn_grid** grid, shn_scene** scene) {
  if (!e) return SHN_ERR_INVALID;
  const uint32_t s = next ? e->render_slot : 1u - e->render_slot;
  if (grid) *grid = e->grid[s];
  if (scene) *scene = e->scene[s];
  return SHN_OK;
}

void shn_dynamic_destroy(shn_dynamic* e) {
  if (e) destroy(e);
}

}  // extern "C"
