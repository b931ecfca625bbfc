// Exclusive scan that allocates nothing (shn_exclusive_scan_u32_noalloc).
//
// Some callers cannot take a device allocation on their hot path: an engine
// that has claimed all device memory up front for its own allocator, or a
// serving loop whose memory budget is already committed, where an allocation
// may block, may fail under memory pressure and would be charged against a
// budget the caller has already spent.  This variant keeps its look-back
// scratch (an error word, the tile ticket and the per-tile status words) in
// one fixed, file-scope device array instead of the context's memory pool;
// the caller still passes its own input and output buffers.
//
// Limits and sharing rules:
//  * at most kNoAllocMaxN = 2^24 elements per call (bigger sizes are
//    rejected with SHN_ERR_INVALID before anything is launched);
//  * the array is shared by every call in the process on a given device and
//    keeps the last call's contents: each call clears the words it uses
//    (the ticket and its tiles' status words, one cudaMemsetAsync of
//    8 * (tiles + 1) bytes on its stream) before its kernel runs, so two
//    calls whose work overlaps on the GPU (different streams, no ordering
//    between them) race on it -- order such calls on one stream;
//  * the error word is not cleared per call: a look-back wait that gave up
//    in any call leaves a bit there until shn_exclusive_scan_u32_noalloc_status
//    reports and clears it;
//  * every GPU that loads the library holds the array (about 64 KiB) until
//    the process exits;
//  * the host cannot use the array's name as a device address, so the first
//    call on each device looks the address up with cudaGetSymbolAddress
//    (with that device current) and caches it for the life of the process;
//    make that first call before any stream capture on that device.  A
//    cudaDeviceReset (or anything else that destroys the device's primary
//    context) invalidates the cached address.
#include <atomic>
#include <mutex>

#include "internal.h"

namespace shn {
namespace {

constexpr int kNaBlock = 256;
constexpr int kNaItems = 8;
constexpr int kNaTile = kNaBlock * kNaItems;
constexpr uint32_t kNoAllocMaxN = 1u << 24;
constexpr uint32_t kNaMaxTiles = kNoAllocMaxN / kNaTile;          // 8192
// word 0: error bits (sticky), word 1: tile ticket, words 2..: tile status
constexpr size_t kNaScratchWords = kNaMaxTiles + 2;

static __device__ __align__(256) uint64_t g_scan_scratch[kNaScratchWords];

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
void* g_addr[kMaxDevices] = {nullptr};
// failure-detection self test: the next call withholds its first tile
std::atomic<uint32_t> g_force_lookback{0};

__global__ void __launch_bounds__(kNaBlock) k_exclusive_scan_noalloc(const uint32_t* __restrict__ in,
                                                                    uint32_t* __restrict__ out,
                                                                    uint32_t n, uint64_t* scratch) {
  __shared__ TileScanSmem<kNaBlock, kNaItems> sm;
  LookbackState st{scratch + 2, (uint32_t*)(scratch + 1), (uint32_t*)scratch};
  tile_scan<kNaBlock, kNaItems>(
      st, n, sm, [&](uint32_t i) { return in[i]; }, [&](uint32_t i, uint32_t ex) { out[i] = ex; },
      out + n);
}

// Device address of the scratch array on the current device (looked up once).
cudaError_t scratch_address(void** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_scan_scratch);
    if (e != cudaSuccess) return e;
    g_addr[dev] = p;
  }
  *out = g_addr[dev];
  return cudaSuccess;
}

}  // namespace
}  // namespace shn

namespace shn {
shn_status noalloc_force_lookback_timeout() {
  g_force_lookback.store(1);
  return SHN_OK;
}
}  // namespace shn

using namespace shn;

extern "C" shn_status shn_exclusive_scan_u32_noalloc(const uint32_t* d_in, uint32_t* d_out,
                                                     uint32_t n, void* stream) {
  if (!d_out || (n && !d_in)) return SHN_ERR_INVALID;
  if (n > kNoAllocMaxN) return SHN_ERR_INVALID;
  cudaStream_t st = (cudaStream_t)stream;
  if (n == 0) {
    return cudaMemsetAsync(d_out, 0, sizeof(uint32_t), st) == cudaSuccess ? SHN_OK : SHN_ERR_CUDA;
  }
  void* scratch = nullptr;
  if (scratch_address(&scratch) != cudaSuccess) return SHN_ERR_CUDA;
  uint64_t* words = (uint64_t*)scratch;
  const uint32_t tiles = (n + kNaTile - 1) / kNaTile;
  // the ticket and the status words of the tiles used start at zero; the
  // error word (word 0) keeps what earlier calls recorded
  if (cudaMemsetAsync(words + 1, 0, (size_t)(tiles + 1) * sizeof(uint64_t), st) != cudaSuccess)
    return SHN_ERR_CUDA;
  const uint32_t armed = g_force_lookback.exchange(0);
  const uint32_t blocks = lookback_blocks(tiles, (uint32_t*)(words + 1), armed != 0, st);
  if (armed && blocks == tiles) g_force_lookback.store(armed);
  k_exclusive_scan_noalloc<<<blocks, kNaBlock, 0, st>>>(d_in, d_out, n, words);
  return cudaGetLastError() == cudaSuccess ? SHN_OK : SHN_ERR_CUDA;
}

extern "C" shn_status shn_exclusive_scan_u32_noalloc_status(void* stream) {
  cudaStream_t st = (cudaStream_t)stream;
  void* scratch = nullptr;
  if (scratch_address(&scratch) != cudaSuccess) return SHN_ERR_CUDA;
  if (cudaStreamSynchronize(st) != cudaSuccess) return SHN_ERR_CUDA;
  uint32_t bits = 0;
  if (cudaMemcpy(&bits, scratch, sizeof(bits), cudaMemcpyDeviceToHost) != cudaSuccess) return SHN_ERR_CUDA;
  if (!bits) return SHN_OK;
  if (cudaMemset(scratch, 0, sizeof(uint64_t)) != cudaSuccess) return SHN_ERR_CUDA;
  return SHN_ERR_TIMEOUT;
}
