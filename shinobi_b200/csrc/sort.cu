// Onesweep LSD radix sort of 64-bit keys (Adinets and Merrill, "Onesweep: A
// Faster Least Significant Digit Radix Sort for GPUs", 2022), written for
// sm_100a:
//  * digits are 8 or 9 bits wide, whichever sorts the key bits in fewer
//    passes (27 cell bits: three 9-bit passes instead of four 8-bit ones);
//  * the digit counts of every pass come from one histogram kernel over the
//    keys, or from the producer of the keys while it writes them (the grid
//    build's key emission does this; see sort_hist_counts);
//  * each pass is ONE kernel over 6144-key tiles (two per SM): a tile is staged into
//    shared memory with a bulk asynchronous copy (cp.async.bulk +
//    mbarrier), each warp's digit counts are taken with order-free shared
//    atomics, the tile's counts are published at once and combined across
//    tiles with decoupled look-back, then every key is ranked stably (in
//    input order; the lanes of a warp holding the same digit find each other
//    through a shared match word per digit) straight into its digit-ordered
//    place in shared memory, and the tile is written out with coalesced
//    stores.  Publishing before ranking lets the look-back of later tiles
//    find this tile's counts early.  Ordinary stores: a digit's run of a
//    tile ends in a sector that the next tile's run of the same digit
//    completes, and the two merge in L2 instead of reaching DRAM as partial
//    writes.
// Replaces the reference's 2-bit split radix sort with three launches per
// pass (src/Utils/Sort.cu:28-56, src/Utils/chag/pp/detail/sort.cu.inl:436-597).
// Stability makes the result identical to a stable sort on the digit bits,
// so keys emitted in triangle order come out ordered by (cell, tri).
#include "internal.h"

namespace shn {

namespace {

constexpr int kSortBlock = 512;
constexpr int kSortWarps = kSortBlock / 32;
constexpr int kPassItems = 12;            // keys per thread: 6144-key tiles, two per SM
constexpr int kMinTile = kSortBlock * 8;  // sizes the look-back status array
constexpr int kMaxBins = 512;             // 9-bit digits
constexpr int kHistBlock = 256;
constexpr uint32_t kDigFlagAgg = 1u << 30;
constexpr uint32_t kDigFlagPrefix = 2u << 30;
// A tile that gave up (its staged keys never arrived, or its own look-back
// ran out) publishes this for its digits: later tiles stop looking back,
// record the error and publish it in turn.
constexpr uint32_t kDigFlagPoison = 3u << 30;
constexpr uint32_t kDigValueMask = (1u << 30) - 1u;
constexpr int kLookback = 8;

__global__ void __launch_bounds__(kHistBlock) k_sort_hist(const uint64_t* __restrict__ keys,
                                                          uint32_t n, uint32_t lo_bit,
                                                          uint32_t passes, uint32_t width, uint32_t bits,
                                                          uint32_t* hist) {
  __shared__ uint32_t sh[4 * kMaxBins];
  for (int i = threadIdx.x; i < 4 * kMaxBins; i += kHistBlock) sh[i] = 0u;
  __syncthreads();
  const uint64_t stride = (uint64_t)gridDim.x * kHistBlock;
  for (uint64_t i = (uint64_t)blockIdx.x * kHistBlock + threadIdx.x; i < n; i += stride) {
    const uint64_t k = keys[i];
    for (uint32_t p = 0; p < passes; ++p) {
      const uint32_t w = min(width, bits - width * p);
      const uint32_t d = (uint32_t)(k >> (lo_bit + width * p)) & ((1u << w) - 1u);
      atomicAdd(&sh[p * kMaxBins + d], 1u);
    }
  }
  __syncthreads();
  for (uint32_t i = threadIdx.x; i < passes * kMaxBins; i += kHistBlock)
    if (sh[i]) atomicAdd(&hist[i], sh[i]);
}

// Exclusive scan of each pass's digit counts (one block per pass).
__global__ void __launch_bounds__(kMaxBins) k_sort_hist_scan(uint32_t* hist) {
  __shared__ ScanSmem<kMaxBins> sm;
  uint32_t* h = hist + blockIdx.x * kMaxBins;
  const uint32_t v = h[threadIdx.x];
  uint32_t tot;
  const uint32_t ex = block_excl_scan<kMaxBins>(v, sm, &tot);
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

// Per tile: stage the keys, count the digits of every warp's slice (shared
// atomics, order-free), publish the tile's digit counts at once, look back
// for the tile's global digit offsets, then rank every key stably
// (warp match in input order) straight into its digit-ordered place in
// shared memory and write the tile out.  Publishing before ranking lets the
// look-back of later tiles find this tile's counts early, so the prefix
// front does not wait on ranking; status words are published with relaxed
// stores (flag and value share one word, nothing else is read through them).
template <int ITEMS, int MINB, int BITS>
__global__ void __launch_bounds__(kSortBlock, MINB) k_onesweep(const uint64_t* __restrict__ in,
                                                            uint64_t* __restrict__ out, uint32_t n,
                                                            uint32_t shift, uint32_t kMask,
                                                            const uint32_t* __restrict__ digit_base,
                                                            uint32_t* status, uint32_t* ticket,
                                                            uint32_t* err, int use_bulk) {
  // kMask: the pass's digit mask (BITS bits, fewer in the last pass when the
  // sorted bits are not a multiple of BITS; bits above the range never count)
  constexpr int kSortTile = kSortBlock * ITEMS;
  constexpr int kWarpSlice = 32 * ITEMS;  // keys ranked per warp (<= 512: 16-bit counters)
  constexpr uint32_t kBins = 1u << BITS;
  constexpr int kPerThread = (int)kBins / kSortBlock > 0 ? (int)kBins / kSortBlock : 1;
  static_assert(kBins <= kSortBlock, "one digit per thread");
  // dynamic: the tile's keys, then per-warp match words (the lane bits of
  // the keys holding each digit)
  extern __shared__ __align__(128) uint64_t s_keys[];
  uint32_t(*s_match)[kBins] = reinterpret_cast<uint32_t(*)[kBins]>(s_keys + kSortTile);
  // per-warp digit counts, then each warp's running position per digit
  // (both <= the tile size): two 16-bit counters per word, so that the
  // counting can use 32-bit shared atomics
  __shared__ uint32_t s_wcnt[kSortWarps][kBins / 2];
  __shared__ uint32_t s_gbase[kBins];
  __shared__ ScanSmem<kSortBlock> s_scan;
  __shared__ alignas(8) uint64_t s_mbar;
  __shared__ uint32_t s_tile;
  uint16_t(*s_w16)[kBins] = reinterpret_cast<uint16_t(*)[kBins]>(s_wcnt);
  (void)kPerThread;

  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (threadIdx.x == 0) s_tile = atomicAdd(ticket, 1u);
  for (int i = threadIdx.x; i < kSortWarps * (int)kBins / 2; i += kSortBlock) (&s_wcnt[0][0])[i] = 0u;
  for (int i = threadIdx.x; i < kSortWarps * (int)kBins; i += kSortBlock) (&s_match[0][0])[i] = 0u;
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
  // publishes a poisoned status for all its digits, so later tiles stop
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
    if (threadIdx.x < kBins) st_relaxed(status + (uint64_t)tile * kBins + threadIdx.x, kDigFlagPoison);
    // the copy may still be in flight into this block's shared memory: wait
    // for it once more (bounded) before the block exits
    uint32_t spins = 0;
    while (!mbar_try_wait(bar) && ++spins <= kSpinLimit) __nanosleep(64);
    __syncthreads();
    return;
  }

  // ---- keys into registers; count each warp slice's digits ------------------
  uint64_t key[ITEMS];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint32_t idx = warp * kWarpSlice + k * 32 + lane;
    key[k] = idx < count ? s_keys[idx] : 0ull;
    if (idx < count) {
      const uint32_t d = (uint32_t)(key[k] >> shift) & kMask;
      atomicAdd(&s_wcnt[warp][d >> 1], 1u << (16u * (d & 1u)));
    }
  }
  __syncthreads();

  // ---- per digit: warp starts, tile count, publish, look back -------------------
  const uint32_t dgt = threadIdx.x;  // threads 0..kBins-1 <-> digits
  const bool has_digit = dgt < kBins;
  uint32_t tcount = 0;
  uint32_t* my = status + (uint64_t)tile * kBins + dgt;
  if (has_digit) {
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) {
      const uint32_t c = s_w16[w][dgt];
      s_w16[w][dgt] = (uint16_t)tcount;
      tcount += c;
    }
    st_relaxed(my, (tile == 0 ? kDigFlagPrefix : kDigFlagAgg) | tcount);
  }
  uint32_t tot;
  const uint32_t bstart = block_excl_scan<kSortBlock>(tcount, s_scan, &tot);
  uint32_t excl = 0;
  if (has_digit) {
    // warp w's digit-d keys go to tile-local positions from here on
#pragma unroll
    for (int w = 0; w < kSortWarps; ++w) s_w16[w][dgt] = (uint16_t)(s_w16[w][dgt] + bstart);
    if (tile != 0) {
      // kLookback predecessors per round trip; relaxed loads suffice (see above)
      bool poisoned = false;
      int64_t j = (int64_t)tile - 1;
      bool done = false;
      while (!done) {
        uint32_t w[kLookback];
#pragma unroll
        for (int q = 0; q < kLookback; ++q)
          w[q] = (j - q >= 0) ? ld_relaxed(status + (uint64_t)(j - q) * kBins + dgt) : kDigFlagPrefix;
#pragma unroll
        for (int q = 0; q < kLookback; ++q) {
          if (done) break;
          uint32_t v = w[q];
          if ((v >> 30) == 0u) {  // not published yet: poll this one
            const uint32_t* p = status + (uint64_t)(j - q) * kBins + dgt;
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
      st_relaxed(my, poisoned ? kDigFlagPoison : (kDigFlagPrefix | (excl + tcount)));
    }
    s_gbase[dgt] = digit_base[dgt] + excl - bstart;  // global index = s_gbase[d] + tile-local index
  }
  __syncthreads();

  // ---- stable rank straight into digit order (input order (warp, k, lane)) --
  // The lanes holding the same digit find each other through the warp's
  // match word of that digit (shared atomicOr of the lane bits); the lowest
  // of them advances the warp's running position and clears the word.
  const uint32_t lbit = 1u << lane, lt = lbit - 1u;
  uint32_t* wm = s_match[warp];
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const uint32_t idx = warp * kWarpSlice + k * 32 + lane;
    const bool valid = idx < count;
    const uint32_t d = (uint32_t)(key[k] >> shift) & kMask;
    if (valid) atomicOr(wm + d, lbit);
    __syncwarp();
    const uint32_t peers = valid ? wm[d] : lbit;
    __syncwarp();
    const bool leader = valid && (peers & lt) == 0u;
    uint32_t pos0 = 0;
    if (leader) {
      wm[d] = 0u;
      pos0 = s_w16[warp][d];
      s_w16[warp][d] = (uint16_t)(pos0 + __popc(peers));
    }
    pos0 = __shfl_sync(0xFFFFFFFFu, pos0, __ffs(peers) - 1);
    if (valid) s_keys[pos0 + __popc(peers & lt)] = key[k];
    __syncwarp();
  }
  __syncthreads();

  // ---- coalesced write-out ---------------------------------------------------
  for (uint32_t i = threadIdx.x; i < count; i += kSortBlock) {
    const uint64_t k = s_keys[i];
    const uint32_t d = (uint32_t)(k >> shift) & kMask;
    out[s_gbase[d] + i] = k;
  }
}

}  // namespace

size_t sort_workspace_bytes(uint32_t n) {
  const size_t tiles = ((size_t)n + kMinTile - 1) / kMinTile;
  return (4 * kMaxBins + 8) * sizeof(uint32_t) + tiles * kMaxBins * sizeof(uint32_t);
}

uint32_t sort_tiles(uint32_t n) { return (uint32_t)(((size_t)n + kMinTile - 1) / kMinTile); }

uint32_t* sort_hist_counts(void* ws) { return (uint32_t*)ws; }

void sort_prepare(void* ws, cudaStream_t st) {
  cudaMemsetAsync(ws, 0, (4 * kMaxBins + 8) * sizeof(uint32_t), st);
}

uint32_t key_bits_for(uint64_t max_key_value) {
  uint32_t bits = 0;
  while (bits < 32 && (max_key_value >> bits) != 0) ++bits;
  return bits;
}

SortPlan sort_plan(uint32_t bits) {
  SortPlan p;
  p.bits = bits;
  p.width = 8;
  p.passes = (bits + 7) / 8;
  const uint32_t p9 = (bits + 8) / 9;
  if (p9 < p.passes) {
    p.width = 9;
    p.passes = p9;
  }
  return p;
}

namespace {

template <int ITEMS, int MINB, int BITS>
void launch_pass(const uint64_t* src, uint64_t* dst, uint32_t n, uint32_t shift, uint32_t mask,
                 const uint32_t* digit_base, uint32_t* status, uint32_t* ticket, uint32_t* err, cudaStream_t st) {
  constexpr int tile = kSortBlock * ITEMS;
  constexpr size_t smem = (size_t)tile * sizeof(uint64_t) + (size_t)kSortWarps * (1u << BITS) * sizeof(uint32_t);
  // the dynamic shared-memory limit is a per-device attribute: set it once per device
  static std::atomic<uint64_t> done_mask{0};
  int dev = 0;
  cudaGetDevice(&dev);
  const uint64_t bit = 1ull << (dev & 63);
  if (!(done_mask.load() & bit)) {
    cudaFuncSetAttribute(k_onesweep<ITEMS, MINB, BITS>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    done_mask.fetch_or(bit);
  }
  const uint32_t tiles = (uint32_t)(((size_t)n + tile - 1) / tile);
  cudaMemsetAsync(status, 0, (size_t)tiles * (1u << BITS) * sizeof(uint32_t), st);
  const int bulk = (((uintptr_t)src) & 15u) == 0u;
  k_onesweep<ITEMS, MINB, BITS><<<tiles, kSortBlock, smem, st>>>(src, dst, n, shift, mask, digit_base, status,
                                                                 ticket, err, bulk);
}

}  // namespace

// Sorts keys held in buf0 on the plan's digits of bits [lo_bit, ...);
// returns the buffer holding the result (buf0 or buf1).  ws:
// sort_workspace_bytes(n).  counts_ready: the caller ran sort_prepare(ws)
// before producing the keys and its producer added every key's digits to
// sort_hist_counts(ws) ([pass][512]).
uint64_t* onesweep_sort(uint64_t* buf0, uint64_t* buf1, uint32_t n, uint32_t lo_bit, SortPlan plan, void* ws,
                        uint32_t* d_err, cudaStream_t st, bool counts_ready, uint32_t tile_keys) {
  if (n <= 1 || plan.passes == 0) return buf0;
  uint32_t* hist = (uint32_t*)ws;
  uint32_t* tickets = hist + 4 * kMaxBins;
  uint32_t* status = tickets + 8;
  if (!counts_ready) {
    sort_prepare(ws, st);
    const int hist_blocks = (int)std::min<uint32_t>((n + 4095) / 4096, 4 * 148u);
    k_sort_hist<<<hist_blocks, kHistBlock, 0, st>>>(buf0, n, lo_bit, plan.passes, plan.width, plan.bits, hist);
  }
  k_sort_hist_scan<<<plan.passes, kMaxBins, 0, st>>>(hist);
  uint64_t* src = buf0;
  uint64_t* dst = buf1;
  for (uint32_t p = 0; p < plan.passes; ++p) {
    const uint32_t shift = lo_bit + plan.width * p;
    const uint32_t w = std::min(plan.width, plan.bits - plan.width * p);
    const uint32_t mask = (1u << w) - 1u;
    // 4096-key tiles (8 per thread) are the autotuner's alternative tile shape
    const bool t4k = tile_keys == 4096u;
    if (plan.width == 9) {
      if (t4k) launch_pass<8, 2, 9>(src, dst, n, shift, mask, hist + p * kMaxBins, status, tickets + p, d_err, st);
      else launch_pass<kPassItems, 2, 9>(src, dst, n, shift, mask, hist + p * kMaxBins, status, tickets + p, d_err, st);
    } else {
      if (t4k) launch_pass<8, 2, 8>(src, dst, n, shift, mask, hist + p * kMaxBins, status, tickets + p, d_err, st);
      else launch_pass<kPassItems, 2, 8>(src, dst, n, shift, mask, hist + p * kMaxBins, status, tickets + p, d_err, st);
    }
    std::swap(src, dst);
  }
  return src;
}

}  // namespace shn
