// Onesweep LSD radix sort of 64-bit keys on an 8-bit digit per pass
// (Adinets and Merrill, "Onesweep: A Faster Least Significant Digit Radix
// Sort for GPUs", 2022), written for sm_100a:
//  * one histogram kernel computes the digit counts of every pass in a
//    single read of the keys;
//  * each pass is ONE kernel: a 4096-key tile is staged into shared memory
//    with a bulk asynchronous copy (cp.async.bulk + mbarrier), ranked with
//    warp match/popc (stable), its per-digit counts are combined across
//    tiles with decoupled look-back, the tile is reordered in shared memory
//    and written out with coalesced stores.
// Replaces the reference's 2-bit split radix sort with three launches per
// pass (src/Utils/Sort.cu:28-56, src/Utils/chag/pp/detail/sort.cu.inl:436-597).
// Stability makes the result identical to a stable sort on the digit bits,
// so keys emitted in triangle order come out ordered by (cell, tri).
#include "internal.h"

namespace shn {

namespace {

constexpr int kSortBlock = 256;
constexpr int kSortItems = 16;
constexpr int kSortTile = kSortBlock * kSortItems;  // 4096 keys, 32 KB
constexpr int kSortWarps = kSortBlock / 32;
constexpr uint32_t kDigFlagAgg = 1u << 30;
constexpr uint32_t kDigFlagPrefix = 2u << 30;
// A tile that gave up (its staged keys never arrived, or its own look-back
// ran out) publishes this for its digits: later tiles stop looking back,
// record the error and publish it in turn.
constexpr uint32_t kDigFlagPoison = 3u << 30;
constexpr uint32_t kDigValueMask = (1u << 30) - 1u;
constexpr int kLookback = 8;

__global__ void __launch_bounds__(kSortBlock) k_sort_hist(const uint64_t* __restrict__ keys,
                                                          uint32_t n, uint32_t lo_bit,
                                                          uint32_t passes, uint32_t* hist) {
  __shared__ uint32_t sh[kSortWarps][4][256];
  const int warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kSortWarps * 4 * 256; i += kSortBlock) (&sh[0][0][0])[i] = 0u;
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * kSortBlock;
  for (uint64_t i = (uint64_t)blockIdx.x * kSortBlock + threadIdx.x; i < n; i += stride) {
    const uint64_t k = keys[i];
    for (uint32_t p = 0; p < passes; ++p) {
      const uint32_t d = (uint32_t)(k >> (lo_bit + 8u * p)) & 255u;
      atomicAdd(&sh[warp][p][d], 1u);
    }
  }
  __syncthreads();
  for (uint32_t p = 0; p < passes; ++p) {
    uint32_t s = 0;
    for (int w = 0; w < kSortWarps; ++w) s += sh[w][p][threadIdx.x];
    if (s) atomicAdd(&hist[p * 256 + threadIdx.x], s);
  }
}

// Exclusive scan of each pass's 256 digit counts (one block per pass).
__global__ void __launch_bounds__(256) k_sort_hist_scan(uint32_t* hist) {
  __shared__ ScanSmem<256> sm;
  uint32_t* h = hist + blockIdx.x * 256;
  const uint32_t v = h[threadIdx.x];
  uint32_t tot;
  const uint32_t ex = block_excl_scan<256>(v, sm, &tot);
  h[threadIdx.x] = ex;
}

SHN_D uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

SHN_D uint32_t mbar_try_wait(uint32_t bar) {
  uint32_t done;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0;\n selp.u32 %0, 1, 0, p;\n}"
      : "=r"(done)
      : "r"(bar)
      : "memory");
  return done;
}

__global__ void __launch_bounds__(kSortBlock, 3) k_onesweep(const uint64_t* __restrict__ in,
                                                         uint64_t* __restrict__ out, uint32_t n,
                                                         uint32_t shift,
                                                         const uint32_t* __restrict__ digit_base,
                                                         uint32_t* status, uint32_t* ticket,
                                                         uint32_t* err, int use_bulk) {
  __shared__ alignas(128) uint64_t s_keys[kSortTile];
  __shared__ uint32_t s_whist[kSortWarps][256];
  __shared__ uint32_t s_gbase[256];
  __shared__ ScanSmem<kSortBlock> s_scan;
  __shared__ alignas(8) uint64_t s_mbar;
  __shared__ uint32_t s_tile;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  for (int i = threadIdx.x; i < kSortWarps * 256; i += kSortBlock) (&s_whist[0][0])[i] = 0u;
  __syncthreads();
  const uint32_t tile = s_tile;
  const uint64_t base = (uint64_t)tile * kSortTile;
  const uint64_t left = (uint64_t)n - base;
  const uint32_t count = left < (uint64_t)kSortTile ? (uint32_t)left : (uint32_t)kSortTile;
  // Bulk copies need 16-byte aligned addresses and sizes: an even number of
  // keys from a 16-byte aligned buffer (the host checks the buffer).
  const uint32_t bulk_keys = use_bulk ? (count & ~1u) : 0u;
  const uint32_t bar = smem_u32(&s_mbar);

  // ---- stage the tile with a bulk async copy ------------------------------
  if (threadIdx.x == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(bar) : "memory");
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    if (bulk_keys) {
      asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar),
                   "r"(bulk_keys * 8u)
                   : "memory");
      asm volatile(
          "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
              smem_u32(s_keys)),
          "l"(in + base), "r"(bulk_keys * 8u), "r"(bar)
          : "memory");
    } else {
      asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
    }
  }
  // keys not covered by the bulk copy are staged with plain loads
  for (uint32_t i = bulk_keys + threadIdx.x; i < count; i += kSortBlock) s_keys[i] = in[base + i];
  __syncthreads();
  // Bounded wait for the staged tile, taken by the whole block: if any
  // thread's wait runs out, every thread leaves together.  The tile then
  // publishes a poisoned status for all 256 digits, so later tiles stop
  // looking back at once instead of spending their own wait budget on it.
  int timed_out = 0;
  {
    uint32_t done = 0, spins = 0;
    while (!done) {
      done = mbar_try_wait(bar);
      if (!done && ++spins > kSpinLimit) {
        timed_out = 1;
        break;
      }
    }
  }
  if (__syncthreads_or(timed_out)) {
    if (threadIdx.x == 0) atomicOr(err, kErrTmaTimeout);
    st_release(status + (uint64_t)tile * 256 + threadIdx.x, kDigFlagPoison);
    // the copy may still be in flight into this block's shared memory: wait
    // for it once more (bounded) before the block exits
    uint32_t spins = 0;
    while (!mbar_try_wait(bar) && ++spins <= kSpinLimit) __nanosleep(64);
    __syncthreads();
    return;
  }

  // ---- stable rank within each warp's 512-key slice ------------------------
  uint64_t key[kSortItems];
  uint32_t rank[kSortItems];
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t idx = warp * (32 * kSortItems) + k * 32 + lane;
    const bool valid = idx < count;
    key[k] = valid ? s_keys[idx] : 0ull;
    const uint32_t d = valid ? ((uint32_t)(key[k] >> shift) & 255u) : 256u;
    const uint32_t peers = __match_any_sync(0xFFFFFFFFu, d);
    const int leader = __ffs(peers) - 1;
    uint32_t old = 0;
    if (lane == leader && d < 256u) old = s_whist[warp][d];
    old = __shfl_sync(0xFFFFFFFFu, old, leader);
    rank[k] = old + __popc(peers & ((1u << lane) - 1u));
    if (lane == leader && d < 256u) s_whist[warp][d] = old + __popc(peers);
    __syncwarp();
  }
  __syncthreads();

  // ---- per digit: warp prefixes and tile count; publish the tile count ------
  const uint32_t dgt = threadIdx.x;  // 256 threads <-> 256 digits
  uint32_t tcount = 0;
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) {
    const uint32_t c = s_whist[w][dgt];
    s_whist[w][dgt] = tcount;
    tcount += c;
  }
  uint32_t* my = status + (uint64_t)tile * 256 + dgt;
  st_release(my, (tile == 0 ? kDigFlagPrefix : kDigFlagAgg) | tcount);
  uint32_t tot;
  const uint32_t bstart = block_excl_scan<kSortBlock>(tcount, s_scan, &tot);
  // s_whist[w][d] becomes the tile-local start of warp w's digit-d keys
#pragma unroll
  for (int w = 0; w < kSortWarps; ++w) s_whist[w][dgt] += bstart;
  __syncthreads();

  // ---- reorder the tile in shared memory (digit order, stable) -------------
#pragma unroll
  for (int k = 0; k < kSortItems; ++k) {
    const uint32_t idx = warp * (32 * kSortItems) + k * 32 + lane;
    if (idx < count) {
      const uint32_t d = (uint32_t)(key[k] >> shift) & 255u;
      s_keys[s_whist[warp][d] + rank[k]] = key[k];
    }
  }

  // ---- look-back across tiles for this digit ----------------------------------
  uint32_t excl = 0;
  bool poisoned = false;
  if (tile != 0) {
    // kLookback predecessors per round trip: the status word carries flag
    // and value together, so relaxed loads suffice and all of a round's
    // loads are in flight at once.
    int64_t j = (int64_t)tile - 1;
    bool done = false;
    while (!done) {
      uint32_t w[kLookback];
#pragma unroll
      for (int q = 0; q < kLookback; ++q)
        w[q] = (j - q >= 0) ? ld_relaxed(status + (uint64_t)(j - q) * 256 + dgt) : kDigFlagPrefix;
#pragma unroll
      for (int q = 0; q < kLookback; ++q) {
        if (done) break;
        uint32_t v = w[q];
        if ((v >> 30) == 0u) {  // not published yet: poll this one
          const uint32_t* p = status + (uint64_t)(j - q) * 256 + dgt;
          uint32_t spins = 0;
          while (((v = ld_relaxed(p)) >> 30) == 0u) {
            if (++spins > kSpinLimit) {
              v = kDigFlagPoison;
              break;
            }
            __nanosleep(20);
          }
        }
        if ((v >> 30) == 3u) {  // a predecessor gave up, or this wait ran out
          atomicOr(err, kErrLookbackTimeout);
          poisoned = true;
          done = true;
          break;
        }
        excl += v & kDigValueMask;
        if ((v >> 30) == 2u) done = true;
      }
      j -= kLookback;
    }
    st_release(my, poisoned ? kDigFlagPoison : (kDigFlagPrefix | (excl + tcount)));
  }
  s_gbase[dgt] = digit_base[dgt] + excl - bstart;  // global index = s_gbase[d] + local index
  __syncthreads();

  // ---- coalesced write-out ---------------------------------------------------
  for (uint32_t i = threadIdx.x; i < count; i += kSortBlock) {
    const uint64_t k = s_keys[i];
    const uint32_t d = (uint32_t)(k >> shift) & 255u;
    __stcs(out + s_gbase[d] + i, k);
  }
}

}  // namespace

size_t sort_workspace_bytes(uint32_t n) {
  const size_t tiles = ((size_t)n + kSortTile - 1) / kSortTile;
  return (4 * 256 + 8) * sizeof(uint32_t) + tiles * 256 * sizeof(uint32_t);
}

uint32_t sort_tiles(uint32_t n) { return (uint32_t)(((size_t)n + kSortTile - 1) / kSortTile); }

// Sorts keys held in buf0 on bits [lo_bit, lo_bit + 8*passes); returns the
// buffer holding the result (buf0 or buf1).  ws: sort_workspace_bytes(n).
uint64_t* onesweep_sort(uint64_t* buf0, uint64_t* buf1, uint32_t n, uint32_t lo_bit,
                        uint32_t passes, void* ws, uint32_t* d_err, cudaStream_t st) {
  if (n <= 1 || passes == 0) return buf0;
  uint32_t* hist = (uint32_t*)ws;
  uint32_t* tickets = hist + 4 * 256;
  uint32_t* status = tickets + 8;
  const uint32_t tiles = sort_tiles(n);
  cudaMemsetAsync(hist, 0, (4 * 256 + 8) * sizeof(uint32_t), st);
  const int hist_blocks = (int)std::min<uint32_t>(tiles, 4 * 148u);
  k_sort_hist<<<hist_blocks, kSortBlock, 0, st>>>(buf0, n, lo_bit, passes, hist);
  k_sort_hist_scan<<<passes, 256, 0, st>>>(hist);
  uint64_t* src = buf0;
  uint64_t* dst = buf1;
  for (uint32_t p = 0; p < passes; ++p) {
    cudaMemsetAsync(status, 0, (size_t)tiles * 256 * sizeof(uint32_t), st);
    const int bulk = (((uintptr_t)src) & 15u) == 0u;
    k_onesweep<<<tiles, kSortBlock, 0, st>>>(src, dst, n, lo_bit + 8u * p, hist + p * 256, status,
                                            tickets + p, d_err, bulk);
    std::swap(src, dst);
  }
  return src;
}

uint32_t sort_passes_for(uint64_t max_key_value) {
  uint32_t bits = 0;
  while (bits < 32 && (max_key_value >> bits) != 0) ++bits;
  return (bits + 7) / 8;
}

}  // namespace shn
