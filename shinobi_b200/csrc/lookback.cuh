// Single-pass exclusive prefix scan with decoupled look-back (Merrill and
// Garland, "Single-pass Parallel Prefix Scan with Decoupled Look-back",
// NVIDIA tech report NVR-2016-002), as a block-level device template so
// that producers (per-triangle candidate counts, per-top-cell leaf counts,
// live-path flags) and consumers (offset writes, compaction scatters) are
// fused into the same kernel.
//
// Tile status words are 64-bit: high 32 bits = flag (0 empty, 1 aggregate,
// 2 inclusive prefix), low 32 bits = value.  Tiles are numbered by an atomic
// ticket taken at block start, so every tile a block waits on belongs to a
// block that is already running; waits are still bounded (kSpinLimit polls)
// and record kErrLookbackTimeout instead of hanging.
#pragma once
#include "common.cuh"

namespace shn {

constexpr uint64_t kFlagAgg = 1ull << 32;
constexpr uint64_t kFlagPrefix = 2ull << 32;

struct LookbackState {
  uint64_t* status;    // one word per tile, zeroed before the launch
  uint32_t* ticket;    // zeroed before the launch
  uint32_t* err;       // error bits (may be shared)
};

template <int BLOCK>
struct ScanSmem {
  uint32_t warp_tot[BLOCK / 32];
  uint32_t tile_excl;
  uint32_t tile_id;
};

SHN_D uint32_t warp_incl_scan(uint32_t v) {
  const int lane = threadIdx.x & 31;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const uint32_t y = __shfl_up_sync(0xFFFFFFFFu, v, o);
    if (lane >= o) v += y;
  }
  return v;
}

SHN_D uint32_t warp_sum(uint32_t v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xFFFFFFFFu, v, o);
  return v;
}

SHN_D uint32_t take_tile(LookbackState st, uint32_t* smem_tile) {
  if (threadIdx.x == 0) *smem_tile = atomicAdd(st.ticket, 1u);
  __syncthreads();
  return *smem_tile;
}

// Block-wide exclusive scan of one value per thread; returns this thread's
// exclusive prefix within the block and writes the block total to *total.
template <int BLOCK>
SHN_D uint32_t block_excl_scan(uint32_t v, ScanSmem<BLOCK>& sm, uint32_t* total) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const uint32_t incl = warp_incl_scan(v);
  if (lane == 31) sm.warp_tot[warp] = incl;
  __syncthreads();
  if (warp == 0) {
    uint32_t w = lane < BLOCK / 32 ? sm.warp_tot[lane] : 0u;
    const uint32_t wi = warp_incl_scan(w);
    if (lane < BLOCK / 32) sm.warp_tot[lane] = wi - w;
    if (lane == 31) sm.tile_excl = wi;  // block total (temporarily)
  }
  __syncthreads();
  *total = sm.tile_excl;
  const uint32_t r = sm.warp_tot[warp] + incl - v;
  __syncthreads();
  return r;
}

// Look-back for tile `tile` whose aggregate is `agg`; executed by warp 0.
// Returns the exclusive prefix of the tile (valid in lane 0 and broadcast).
SHN_D uint32_t lookback_warp(LookbackState st, uint32_t tile, uint32_t agg) {
  const int lane = threadIdx.x & 31;
  if (tile == 0) {
    if (lane == 0) st_release64(st.status, kFlagPrefix | agg);
    return 0u;
  }
  if (lane == 0) st_release64(st.status + tile, kFlagAgg | agg);
  uint32_t excl = 0;
  int64_t j = (int64_t)tile - 1;
  while (true) {
    const int64_t k = j - lane;
    uint64_t w = kFlagPrefix;  // lanes past tile 0 contribute nothing and stop
    if (k >= 0) {
      uint32_t spins = 0;
      while (true) {
        w = ld_acquire64(st.status + k);
        if ((w >> 32) != 0u) break;
        if (++spins > kSpinLimit) {
          atomicOr(st.err, kErrLookbackTimeout);
          w = kFlagAgg;  // give up: count as zero
          break;
        }
        __nanosleep(32);
      }
    } else {
      w = kFlagPrefix;  // virtual prefix 0 before tile 0
    }
    const uint32_t pmask = __ballot_sync(0xFFFFFFFFu, (w >> 32) == 2u);
    const int first = pmask ? __ffs(pmask) - 1 : 32;  // closest tile carrying a prefix
    const uint32_t contrib = (lane <= first && k >= 0) ? (uint32_t)w : 0u;
    excl += warp_sum(contrib);
    if (pmask) break;
    j -= 32;
  }
  if (lane == 0) st_release64(st.status + tile, kFlagPrefix | (excl + agg));
  return excl;
}

// Full tile scan over ITEMS values per thread.
//   load(i)  -> uint32 value of item i (only called for i < n)
//   store(i, excl) called for every i < n with the global exclusive prefix
// The tile's items are produced in striped order (coalesced producer reads),
// transposed through shared memory, scanned in blocked order and handed to
// the consumer in striped order again.  The block holding the last tile
// writes the grand total to *d_total when d_total is non-null.
template <int BLOCK, int ITEMS>
struct TileScanSmem {
  uint32_t items[BLOCK * ITEMS + (BLOCK * ITEMS) / 32];
  ScanSmem<BLOCK> scan;
  uint32_t tile_prefix;
};

SHN_D int pad_idx(int i) { return i + (i >> 5); }

// Split form for producers that fill the tile cooperatively: take the tile
// with tile_begin, write item li (0 <= li < BLOCK*ITEMS) of the tile to
// sm.items[pad_idx(li)] in any order, then call tile_finish, which scans,
// looks back and hands every item's global exclusive prefix to store().
template <int BLOCK, int ITEMS>
SHN_D uint32_t tile_begin(LookbackState st, TileScanSmem<BLOCK, ITEMS>& sm) {
  return take_tile(st, &sm.scan.tile_id);
}

template <int BLOCK, int ITEMS, class Store>
SHN_D void tile_finish(LookbackState st, uint32_t n, uint32_t tile, TileScanSmem<BLOCK, ITEMS>& sm,
                       Store&& store, uint32_t* d_total) {
  constexpr int TILE = BLOCK * ITEMS;
  const uint64_t base = (uint64_t)tile * TILE;
  __syncthreads();
  uint32_t v[ITEMS];
  uint32_t tsum = 0;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    v[k] = sm.items[pad_idx(threadIdx.x * ITEMS + k)];
    tsum += v[k];
  }
  uint32_t agg;
  uint32_t texcl = block_excl_scan<BLOCK>(tsum, sm.scan, &agg);
  if (threadIdx.x < 32) {
    const uint32_t ex = lookback_warp(st, tile, agg);
    if (threadIdx.x == 0) sm.tile_prefix = ex;
  }
  __syncthreads();
  const uint32_t tp = sm.tile_prefix;
  uint32_t run = tp + texcl;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    sm.items[pad_idx(threadIdx.x * ITEMS + k)] = run;
    run += v[k];
  }
  __syncthreads();
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const int li = k * BLOCK + threadIdx.x;
    const uint64_t i = base + li;
    if (i < n) store((uint32_t)i, sm.items[pad_idx(li)]);
  }
  if (d_total && base + TILE >= n && threadIdx.x == 0) *d_total = tp + agg;
}

template <int BLOCK, int ITEMS, class Load, class Store>
SHN_D void tile_scan(LookbackState st, uint32_t n, TileScanSmem<BLOCK, ITEMS>& sm, Load&& load,
                     Store&& store, uint32_t* d_total) {
  constexpr int TILE = BLOCK * ITEMS;
  const uint32_t tile = tile_begin(st, sm);
  const uint64_t base = (uint64_t)tile * TILE;
#pragma unroll
  for (int k = 0; k < ITEMS; ++k) {
    const int li = k * BLOCK + threadIdx.x;
    const uint64_t i = base + li;
    sm.items[pad_idx(li)] = (i < n) ? load((uint32_t)i) : 0u;
  }
  tile_finish(st, n, tile, sm, store, d_total);
}

}  // namespace shn
