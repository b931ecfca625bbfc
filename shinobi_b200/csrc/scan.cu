// Context-level parallel primitives: single-pass exclusive scan and stable
// stream compaction (decoupled look-back).  Replace the reference's
// three-level InclusiveScan with a cudaMalloc per call (src/Utils/Scan.cu:124-252),
// chag::pp::prefix (src/Utils/chag/pp/detail/prefix.cu.inl:59-239) and the
// unused chag::pp::compact (src/Utils/chag/pp/detail/compact.cu.inl:57-200).
#include "internal.h"

namespace shn {

namespace {
constexpr int kBlock = 256;
constexpr int kItems = 8;
constexpr int kTile = kBlock * kItems;

__global__ void __launch_bounds__(kBlock) k_exclusive_scan(const uint32_t* __restrict__ in,
                                                          uint32_t* __restrict__ out, uint32_t n,
                                                          LookbackState st) {
  __shared__ TileScanSmem<kBlock, kItems> sm;
  tile_scan<kBlock, kItems>(
      st, n, sm, [&](uint32_t i) { return in[i]; }, [&](uint32_t i, uint32_t ex) { out[i] = ex; },
      out + n);
}

__global__ void __launch_bounds__(kBlock) k_compact(const uint32_t* __restrict__ flags,
                                                   uint32_t* __restrict__ out, uint32_t n,
                                                   uint32_t* d_count, LookbackState st) {
  __shared__ TileScanSmem<kBlock, kItems> sm;
  tile_scan<kBlock, kItems>(
      st, n, sm, [&](uint32_t i) { return flags[i] ? 1u : 0u; },
      [&](uint32_t i, uint32_t ex) {
        if (flags[i]) out[ex] = i;
      },
      d_count);
}
}  // namespace

size_t scan_workspace_bytes(uint32_t n) {
  const size_t tiles = ((size_t)n + kTile - 1) / kTile;
  return (tiles + 2) * 8;
}

static LookbackState prep(void* ws, uint32_t n, uint32_t* err, cudaStream_t st) {
  const size_t tiles = ((size_t)n + kTile - 1) / kTile;
  uint64_t* status = (uint64_t*)ws;
  cudaMemsetAsync(status, 0, (tiles + 2) * 8, st);
  return LookbackState{status, (uint32_t*)(status + tiles + 1), err};
}

uint32_t lookback_blocks(uint32_t tiles, uint32_t* ticket, bool withhold_first, cudaStream_t st) {
  if (!withhold_first || tiles < 2) return tiles;
  static const uint32_t one = 1u;  // tickets start at 1: tile 0 is never taken
  cudaMemcpyAsync(ticket, &one, 4, cudaMemcpyHostToDevice, st);
  return tiles - 1;
}

bool launch_exclusive_scan(const uint32_t* in, uint32_t* out, uint32_t n, void* ws, uint32_t* err,
                           cudaStream_t st, bool withhold_first) {
  if (n == 0) {
    cudaMemsetAsync(out, 0, 4, st);
    return false;
  }
  LookbackState ls = prep(ws, n, err, st);
  const uint32_t tiles = (n + kTile - 1) / kTile;
  const uint32_t blocks = lookback_blocks(tiles, ls.ticket, withhold_first, st);
  k_exclusive_scan<<<blocks, kBlock, 0, st>>>(in, out, n, ls);
  return blocks != tiles;
}

bool launch_compact(const uint32_t* flags, uint32_t n, uint32_t* out_idx, uint32_t* d_count,
                    void* ws, uint32_t* err, cudaStream_t st, bool withhold_first) {
  if (n == 0) {
    cudaMemsetAsync(d_count, 0, 4, st);
    return false;
  }
  LookbackState ls = prep(ws, n, err, st);
  const uint32_t tiles = (n + kTile - 1) / kTile;
  const uint32_t blocks = lookback_blocks(tiles, ls.ticket, withhold_first, st);
  k_compact<<<blocks, kBlock, 0, st>>>(flags, out_idx, n, d_count, ls);
  return blocks != tiles;
}

}  // namespace shn

using namespace shn;

extern "C" {

// Failure-detection self test: a single block scans tile 1 of a two-tile
// input while tile 0 is never published, so the block's look-back must give
// up after its bounded wait and flag kErrLookbackTimeout.
shn_status shn_selftest_lookback_timeout(shn_ctx* ctx, void* stream) {
  if (!ctx) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  const uint32_t n = 2 * kTile;
  uint32_t *in = nullptr, *out = nullptr, *err = nullptr;
  void* ws = nullptr;
  cudaError_t e = dev_alloc(ctx, (void**)&in, n * 4, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, (void**)&out, (n + 1) * 4, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, (void**)&err, 4, st);
  if (e == cudaSuccess) e = dev_alloc(ctx, &ws, scan_workspace_bytes(n), st);
  shn_status rc = SHN_OK;
  if (e != cudaSuccess) {
    rc = cuda_status(ctx, e, "selftest alloc");
  } else {
    cudaMemsetAsync(in, 0, n * 4, st);
    cudaMemsetAsync(err, 0, 4, st);
    LookbackState ls = prep(ws, n, err, st);
    const uint32_t one = 1u;  // the only block takes ticket 1: tile 0 never runs
    cudaMemcpyAsync(ls.ticket, &one, 4, cudaMemcpyHostToDevice, st);
    k_exclusive_scan<<<1, kBlock, 0, st>>>(in, out, n, ls);
    uint32_t h = 0;
    cudaMemcpyAsync(&h, err, 4, cudaMemcpyDeviceToHost, st);
    e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) rc = cuda_status(ctx, e, "selftest");
    else if (h & kErrLookbackTimeout) rc = set_error(ctx, SHN_ERR_TIMEOUT, "look-back wait gave up (expected)");
  }
  if (in) dev_free(ctx, in, n * 4, st);
  if (out) dev_free(ctx, out, (n + 1) * 4, st);
  if (err) dev_free(ctx, err, 4, st);
  if (ws) dev_free(ctx, ws, scan_workspace_bytes(n), st);
  cudaStreamSynchronize(st);
  return rc;
}

}  // extern "C"
