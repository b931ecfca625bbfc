// Host-side internals shared by the translation units of libshinobi_b200.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/shinobi_b200.h"
#include "common.cuh"
#include "lookback.cuh"

namespace shn {

// Device buffer from the context's stream-ordered pool.
struct DevBuf {
  void* ptr = nullptr;
  size_t bytes = 0;
};

}  // namespace shn

struct shn_ctx {
  int device = 0;
  int num_sms = 148;
  uint64_t budget = 0;
  std::atomic<uint64_t> used{0};
  cudaMemPool_t pool = nullptr;
  std::mutex mu;
  std::string last_error;
  uint32_t* d_err = nullptr;    // device error word of context-level primitives
  // failure-detection self test: the next context-level look-back scan
  // withholds its first tile (shn_debug_force_lookback_timeout)
  std::atomic<uint32_t> force_lookback{0};
  // One reference for the handle returned by shn_ctx_create and one per live
  // scene / grid / batch / server: the context (and its memory pool) is torn
  // down when the last of them is released, whatever the destruction order.
  std::atomic<int> refs{1};
  // 64-byte pinned host blocks for status read-backs, carved from slabs so
  // that creating or destroying a grid never calls cudaMallocHost /
  // cudaFreeHost (both synchronise the whole device).
  std::mutex pin_mu;
  std::vector<void*> pin_slabs;
  std::vector<uint32_t*> pin_free;
};

struct shn_scene {
  shn_ctx* ctx = nullptr;
  uint32_t nv = 0, nt = 0;
  float* vtx = nullptr;      // 3*nv
  uint32_t* idx = nullptr;   // 3*nt
  float4* tri = nullptr;     // 3*nt: per triangle a 48-byte record v0, v1, v2 (w of v0 = tri id bits)
  // records indexed by the id in v0.w: tri itself, except for a view into a
  // larger array whose ids count from that array's start
  const float4* ids = nullptr;
  float bounds[6] = {0, 0, 0, 0, 0, 0};
  size_t bytes = 0;
  size_t cap_v = 0, cap_i = 0, cap_t = 0;  // allocated bytes of vtx, idx, tri
};

struct shn_grid {
  shn_ctx* ctx = nullptr;
  bool built = false;
  uint32_t kind = 0;
  shn::Geom geom{};
  uint64_t num_cells = 0, num_top_refs = 0, num_leaves = 0, num_refs = 0;
  // results
  uint2* cells = nullptr;       // uniform ranges / two-level cell words
  uint2* leaves = nullptr;      // two-level leaf ranges
  uint32_t* indices = nullptr;  // tri id per reference
  float4* rtri = nullptr;       // 3*num_refs: reference-ordered v0[], v1[], v2[]
  uint64_t* top_pairs = nullptr;  // two-level: sorted top pairs; uniform: sorted pairs
  // two-level grids: the build runs on the triangles in Morton order (perm_tri,
  // w = original id), so the pairs' low words are positions in that order;
  // boxes of every 32 references (cbox) and every 1024 (sbox) of rtri, two
  // float4 (min, max) each, let the traversal skip blocks a ray cannot hit
  bool spatial = false;
  // large uniform grids: empty cells hold [D, D), D their distance to the
  // nearest non-empty cell (see k_cell_dist)
  bool cell_dist = false;
  uint64_t num_blocks = 0, num_super = 0;
  shn::DevBuf mhi, perm_tri, cbox, sbox, ldist;
  size_t cap_cells = 0, cap_leaves = 0, cap_refs = 0, cap_rtri = 0;
  // grow-only build workspace
  shn::DevBuf offs_tri, offs_pair, scan, top_ranges, keys[3], sortws;
  // word 0: error bits of bounded waits that gave up, set by this grid's build
  // and by every trace call on it; cleared by shn_grid_sync_status (which
  // reports them) and at the start of each build.  Words 1.. are build scratch.
  uint32_t* d_err = nullptr;
  uint32_t* h_pinned = nullptr; // pinned host words for size read-backs
  // failure-detection self test: the next hit compaction of an AO or
  // direct-illumination call withholds its first tile
  mutable std::atomic<uint32_t> force_lookback{0};
  // ev1: end of the last build on its stream (the build's tail runs
  // asynchronously; every consumer waits for it, see grid_fence)
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  mutable float build_ms = 0.f;
  mutable bool build_ms_pending = false;
  size_t bytes = 0;
  // scene the grid was built over (triangles by id, for shading / AO frames)
  const float4* src_tri = nullptr;
  uint32_t src_nt = 0;
  // optional device counters {cell visits, triangle tests} of the stats kernels
  unsigned long long* stats = nullptr;
};

namespace shn {

// api.cu
cudaError_t dev_alloc(shn_ctx* ctx, void** p, size_t bytes, cudaStream_t st);
void dev_free(shn_ctx* ctx, void* p, size_t bytes, cudaStream_t st);
uint32_t* pinned_take(shn_ctx* ctx);
void pinned_give(shn_ctx* ctx, uint32_t* p);
void ctx_retain(shn_ctx* ctx);
// Replaces a scene's geometry with new host arrays (checked as
// shn_scene_create checks them), reusing its device buffers when they are
// large enough.  On an error the scene's contents are undefined.
shn_status scene_reload(shn_scene* s, const float* vtx, uint32_t nv, const uint32_t* idx, uint32_t nt,
                        cudaStream_t st);
void ctx_release(shn_ctx* ctx);
shn_status set_error(shn_ctx* ctx, shn_status s, const std::string& msg);
shn_status cuda_status(shn_ctx* ctx, cudaError_t e, const char* where);

// sort.cu
// Digit plan of a stable LSD sort: `passes` passes of `width`-bit digits (8 or 9).
struct SortPlan {
  uint32_t passes, width, bits;  // the last pass takes only the bits left of `bits`
};
SortPlan sort_plan(uint32_t bits);          // fewest passes for `bits` key bits (<= 32)
uint32_t key_bits_for(uint64_t max_key_value);
size_t sort_workspace_bytes(uint32_t n);
uint32_t sort_tiles(uint32_t n);
// tile_keys: keys per onesweep tile, 6144 (default, 0) or 4096
uint64_t* onesweep_sort(uint64_t* buf0, uint64_t* buf1, uint32_t n, uint32_t lo_bit, SortPlan plan,
                        void* ws, uint32_t* d_err, cudaStream_t st, bool counts_ready = false,
                        uint32_t tile_keys = 0);
// digit counts [pass][512] in the sort workspace, for producers that count
// the digits of the keys they write (sort_prepare zeroes them first)
uint32_t* sort_hist_counts(void* ws);
void sort_prepare(void* ws, cudaStream_t st);

// build.cu
Geom make_geom(const float b[6], const int res[3]);
void compute_resolution(uint32_t nt, const float b[6], float lambda, int divisor, int min_res,
                        int out[3]);
shn_status build_grid(shn_grid* g, const shn_scene* s, const shn_grid_params* p, cudaStream_t st);
// Orders work on st after the grid's last build (a no-op on the build's own stream).
void grid_fence(const shn_grid* g, cudaStream_t st);
// Device time of the last build; waits for its end.
float grid_build_ms(const shn_grid* g);
// Bounding-box cell references (countRefs) and SAH cost of k <= 32
// resolutions res[3*i..3*i+2] over nt 48-byte triangle records; synchronous.
shn_status sah_refs_list(shn_ctx* ctx, const float4* tri, uint32_t nt, const float b[6], const int32_t* res,
                         uint32_t k, uint64_t* refs, float* cost, cudaStream_t st);
void launch_pack_triangles(const float* vtx, const uint32_t* idx, uint32_t nt, float4* tri,
                           cudaStream_t st);
void launch_bounds_reduce(const float4* tri, uint32_t nt, float* d_out6, cudaStream_t st);

// batched multi-scene build (build.cu)
struct BatchScene {
  Geom g;
  uint32_t tri_offset, nt;
  uint64_t cell_offset;
  uint32_t ncells, pad;
};
void launch_batch_pack(const float* vtx, const uint32_t* vtx_off, const uint32_t* idx,
                       const uint32_t* tri_off, uint32_t ns, uint32_t T, float4* tri, cudaStream_t st);
void launch_batch_bounds(const float4* tri, const uint32_t* tri_off, uint32_t ns, uint32_t T,
                         float* d_out6ns, cudaStream_t st);
size_t batch_scan_bytes(uint32_t T);
void launch_batch_count(const float4* tri, uint32_t T, const uint32_t* tri_off, const BatchScene* scenes,
                        uint32_t ns, void* scan_ws, uint32_t* err, uint32_t* offs, cudaStream_t st);
void launch_batch_emit(const float4* tri, uint32_t T, const uint32_t* tri_off, const BatchScene* scenes,
                       uint32_t ns, const uint32_t* offs, uint64_t* keys, uint32_t capacity,
                       uint32_t* err, uint32_t* hist, SortPlan hplan, cudaStream_t st);
// Ranges of all C cells (empty ones (0, 0)) and indices[], written by tiles
// of cells: needs no cleared cell array.
void launch_cell_ranges(const uint64_t* keys, uint32_t n, uint64_t C, uint2* ranges, uint32_t* indices,
                        cudaStream_t st);
void launch_ranges(const uint64_t* keys, uint32_t n, uint2* ranges, uint32_t* indices,
                   const float4* tri, uint32_t T, float4* rtri, cudaStream_t st);

// trace.cu
struct CamView;
CamView make_camera(const shn_camera* c);

// scan.cu (context-level primitives)
// withhold_first: failure-detection self test -- the launch leaves out tile 0
// (which then never publishes), so the other tiles' look-back waits run out;
// only honoured when there are at least two tiles (returns whether it was).
bool launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, void* ws, uint32_t* err,
                           cudaStream_t st, bool withhold_first = false);
size_t scan_workspace_bytes(uint32_t n);
bool launch_compact(const uint32_t* flags, uint32_t n, uint32_t* out_idx, uint32_t* d_count,
                    void* ws, uint32_t* err, cudaStream_t st, bool withhold_first = false);
// Look-back launch shape with tile 0 optionally withheld: sets the ticket
// word to 1 when withholding and returns the number of blocks to launch.
uint32_t lookback_blocks(uint32_t tiles, uint32_t* ticket, bool withhold_first, cudaStream_t st);

// scan_noalloc.cu: arms the failure-detection self test of the allocation-free scan
shn_status noalloc_force_lookback_timeout();

}  // namespace shn
