// utl_kernels.cu -- batched and per-call kernels of the UTL-PFOR codec.
//
// Batched pack: a persistent kernel whose CTAs take tiles of kTile blocks
// from a device work counter.  Each warp packs its blocks into shared-memory
// slots, warp 0 scans the tile's block lengths and resolves the tile's
// global byte offset with a decoupled look-back over the tiles before it,
// and the warps then copy their blocks to HBM at the final offsets: one
// pass over the values, packed bytes written once, block index written as
// a by-product.  The result is byte-identical to calling the reference's
// PackUint32(flag|Append, ...) block after block (pack.go:76-97).
//
// Batched unpack: one CTA per tile; the tile's contiguous packed bytes are
// staged into shared memory with 16-byte loads, then each warp decodes its
// blocks (warp_unpack_block) and writes 128-byte coalesced rows of values.
#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>

#include "utl_device.cuh"
#include "utl_launch.h"
#include "utl_lane.cuh"
#include "utl_quad.cuh"
#include "utl_unpack.cuh"
#include "utl_pair.cuh"
#include "utl_unlane.cuh"

namespace utl {

constexpr int kWarps = 8;
constexpr int kBlocksPerWarp = 2;
constexpr int kTile = kWarps * kBlocksPerWarp;  // blocks per CTA tile
constexpr int kThreads = kWarps * 32;

template <bool U64> struct Shape;
template <> struct Shape<false> {
  static constexpr int kMax = kMaxBlock32;
  static constexpr int kSlot = 1024;   // pack slot (>= kMax, multiple of 16)
  // unpack per-block staging: a block starts up to 15 bytes into its first
  // 16-byte chunk and its last chunk may run 15 bytes past its end
  static constexpr int kStage = 1056;  // >= kMax + 30, multiple of 16
};
template <> struct Shape<true> {
  static constexpr int kMax = kMaxBlock64;
  static constexpr int kSlot = 2048;
  static constexpr int kStage = 2080;
};

// ------------------------------------------------------------------------
// small helpers
// ------------------------------------------------------------------------
__device__ __forceinline__ uint64_t ld_relaxed_u64(const uint64_t* p) {
  uint64_t v;
  asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void st_relaxed_u64(uint64_t* p, uint64_t v) {
  asm volatile("st.relaxed.gpu.global.b64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ uint64_t shfl_up64(uint64_t v, int d) {
  const uint32_t lo = __shfl_up_sync(kFull, (uint32_t)v, d), hi = __shfl_up_sync(kFull, (uint32_t)(v >> 32), d);
  return ((uint64_t)hi << 32) | lo;
}

__device__ __forceinline__ uint64_t warp_sum_u64(uint64_t v) {
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) v += shfl_xor64(v, d);
  return v;
}

// Stream of block b: largest s with block_start[s] <= b (that stream is
// non-empty).  Returns the first value index and the block's value count.
__device__ __forceinline__ void block_span(const uint64_t* val_off, const uint64_t* bstart, int n_streams, int64_t b,
                                           uint64_t* first, int* n) {
  int lo = 0, hi = n_streams;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if ((int64_t)bstart[mid] <= b) lo = mid;
    else hi = mid;
  }
  uint64_t f = val_off[lo] + (uint64_t)(b - (int64_t)bstart[lo]) * kBlock;
  uint64_t e = val_off[lo + 1];
  *first = f;
  *n = (int)min((uint64_t)kBlock, e - f);
}

// Stream of block b (largest s with block_start[s] <= b).
__device__ __forceinline__ int stream_of(const uint64_t* bstart, int n_streams, int64_t b) {
  int lo = 0, hi = n_streams;
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if ((int64_t)bstart[mid] <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}
// The same, knowing the stream s0 of an earlier block: galloping from s0
// (consecutive blocks are nearly always in the same or the next stream).
__device__ __forceinline__ int stream_from(const uint64_t* bstart, int n_streams, int s0, int64_t b) {
  int lo = s0, step = 1;
  while (lo + step < n_streams && (int64_t)bstart[lo + step] <= b) {
    lo += step;
    step <<= 1;
  }
  int hi = min(n_streams, lo + step);
  while (hi - lo > 1) {
    int mid = (lo + hi) >> 1;
    if ((int64_t)bstart[mid] <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}
// First value index and value count of block b of stream s.
__device__ __forceinline__ void span_in(const uint64_t* val_off, const uint64_t* bstart, int s, int64_t b,
                                        uint64_t* first, int* n) {
  const uint64_t f = val_off[s] + (uint64_t)(b - (int64_t)bstart[s]) * kBlock;
  *first = f;
  *n = (int)min((uint64_t)kBlock, val_off[s + 1] - f);
}

// Copy len bytes of a shared-memory slot (word aligned) to out[g..g+len):
// whole 32-bit words where the global word lies inside the range, single
// bytes at the two edges (those words are shared with neighbouring blocks).
__device__ __forceinline__ void warp_copy_out(const uint32_t* sw, int len, uint8_t* out, uint64_t g, int lane) {
  if (len <= 0) return;
  const uint64_t ge = g + (uint64_t)len;
  const uint64_t q0 = g >> 2, q1 = (ge + 3) >> 2;
  for (uint64_t q = q0 + lane; q < q1; q += 32) {
    const int64_t sb = (int64_t)(q * 4) - (int64_t)g;
    if (sb >= 0 && sb + 4 <= len) {
      const int qi = (int)(sb >> 2);
      *(uint32_t*)(out + q * 4) = __funnelshift_r(sw[qi], sw[qi + 1], (int)(sb & 3) * 8);
    } else {
      for (int b = 0; b < 4; b++) {
        const int64_t s = sb + b;
        if (s >= 0 && s < len) out[q * 4 + b] = (uint8_t)(sw[s >> 2] >> ((s & 3) * 8));
      }
    }
  }
}

// Stage global bytes [g0, g1) of buf (readable range [0, buf_len)) into
// shared memory at dst16 (16-byte aligned) so that byte g0 lands at
// dst16 + ((buf + g0) & 15).  Bytes outside the buffer read as zero.
__device__ __forceinline__ void stage_bytes(uint4* dst16, const uint8_t* buf, uint64_t buf_len, uint64_t g0, uint64_t g1,
                                            int tid, int nthr) {
  const uintptr_t lo = (uintptr_t)buf, hi = lo + buf_len;
  const uintptr_t a0 = (lo + g0) & ~(uintptr_t)15;
  const uintptr_t a1 = (lo + g1 + 15) & ~(uintptr_t)15;
  const int nch = (int)((a1 - a0) >> 4);
  for (int c = tid; c < nch; c += nthr) {
    const uintptr_t a = a0 + 16 * (uintptr_t)c;
    uint4 v;
    if (a >= lo && a + 16 <= hi) {
      v = __ldcs((const uint4*)a);
    } else {
      uint32_t w[4] = {0, 0, 0, 0};
      for (int b = 0; b < 16; b++) {
        const uintptr_t x = a + b;
        if (x >= lo && x < hi) w[b >> 2] |= (uint32_t)(*(const uint8_t*)x) << ((b & 3) * 8);
      }
      v = make_uint4(w[0], w[1], w[2], w[3]);
    }
    dst16[c] = v;
  }
}

// ------------------------------------------------------------------------
// planning
// ------------------------------------------------------------------------
__global__ void __launch_bounds__(1024) plan_kernel(const uint64_t* __restrict__ val_off, int n,
                                                    uint64_t* __restrict__ bstart) {
  __shared__ uint64_t warp_tot[32];
  const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5, T = blockDim.x;
  const int64_t per = ((int64_t)n + T - 1) / T;
  const int64_t s0 = min((int64_t)n, (int64_t)tid * per), s1 = min((int64_t)n, s0 + per);
  uint64_t sum = 0;
  for (int64_t s = s0; s < s1; s++) sum += (val_off[s + 1] - val_off[s] + kBlock - 1) / kBlock;
  uint64_t incl = sum;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    uint32_t lo = __shfl_up_sync(kFull, (uint32_t)incl, d), hi = __shfl_up_sync(kFull, (uint32_t)(incl >> 32), d);
    if (lane >= d) incl += ((uint64_t)hi << 32) | lo;
  }
  if (lane == 31) warp_tot[wid] = incl;
  __syncthreads();
  if (wid == 0) {
    uint64_t t = lane < (T >> 5) ? warp_tot[lane] : 0, ti = t;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
      uint32_t lo = __shfl_up_sync(kFull, (uint32_t)ti, d), hi = __shfl_up_sync(kFull, (uint32_t)(ti >> 32), d);
      if (lane >= d) ti += ((uint64_t)hi << 32) | lo;
    }
    warp_tot[lane] = ti - t;
  }
  __syncthreads();
  uint64_t acc = warp_tot[wid] + incl - sum;
  for (int64_t s = s0; s < s1; s++) {
    bstart[s] = acc;
    acc += (val_off[s + 1] - val_off[s] + kBlock - 1) / kBlock;
  }
  if (tid == T - 1) bstart[n] = acc;
}

__global__ void stream_off_kernel(const uint64_t* __restrict__ block_off, const uint64_t* __restrict__ bstart, int n,
                                  uint64_t* __restrict__ sbo) {
  int s = blockIdx.x * blockDim.x + threadIdx.x;
  if (s <= n) sbo[s] = block_off[bstart[s]];
}

// ------------------------------------------------------------------------
// batched pack with single-pass decoupled look-back
// ------------------------------------------------------------------------
// Tile state word: bits 0-1 flag (0 empty, 1 aggregate, 2 inclusive
// prefix), bits 2-63 value.  Waits are bounded (PackArgs::spin_limit polls,
// each after a 64 ns sleep); on expiry the kernel records UTL_ERR_TIMEOUT
// and carries on with a zero contribution so it always terminates.  Tiles
// are handed out in launch order by an atomic counter, so every
// predecessor of a waiting tile is already running.

// Each lane inspects 8 consecutive predecessors per round (lane 0 the 8
// nearest), so one round covers 256 tiles: with hundreds of tiles in flight
// the nearest inclusive prefix is normally found in one or two rounds.
constexpr int kLookPerLane = 8;

// Publish a tile's aggregate (tile 0 publishes its inclusive prefix).
__device__ __forceinline__ void tile_publish(uint64_t* status, int64_t tile, uint64_t agg) {
  st_relaxed_u64(&status[tile], (agg << 2) | (tile == 0 ? 2u : 1u));
}

// Exclusive prefix of a tile whose aggregate is already published; then
// publishes the tile's inclusive prefix.  Whole warp.
__device__ uint64_t tile_resolve(uint64_t* status, int64_t tile, uint64_t agg, int lane, uint32_t* err, uint32_t lim) {
  if (tile == 0) return 0;
  uint64_t excl = 0;
  int64_t j = tile - 1;
  bool timed_out = false;
  for (;;) {
    uint64_t st[kLookPerLane];
#pragma unroll
    for (int i = 0; i < kLookPerLane; i++) {
      const int64_t idx = j - (int64_t)lane * kLookPerLane - i;
      st[i] = idx >= 0 ? ld_relaxed_u64(&status[idx]) : 2u;  // before tile 0: prefix 0
    }
#pragma unroll
    for (int i = 0; i < kLookPerLane; i++) {
      const int64_t idx = j - (int64_t)lane * kLookPerLane - i;
      uint32_t it = 0;
      while ((st[i] & 3u) == 0) {
        if (++it > lim) {
          timed_out = true;
          st[i] = 2u;
          break;
        }
        __nanosleep(64);
        st[i] = ld_relaxed_u64(&status[idx]);
      }
    }
    // this lane's nearest inclusive prefix (index into st), or none
    int fi = kLookPerLane;
#pragma unroll
    for (int i = kLookPerLane - 1; i >= 0; i--)
      if ((st[i] & 3u) == 2u) fi = i;
    uint64_t part = 0;
#pragma unroll
    for (int i = 0; i < kLookPerLane; i++)
      if (i <= fi) part += st[i] >> 2;
    const unsigned pm = __ballot_sync(kFull, fi < kLookPerLane);
    const int first = pm ? __ffs(pm) - 1 : 32;
    excl += warp_sum_u64(lane <= first ? part : 0ull);
    if (pm) break;
    j -= 32 * kLookPerLane;
  }
  if (__any_sync(kFull, timed_out) && lane == 0 && err) atomicOr(err, 1u << 10);
  if (lane == 0) st_relaxed_u64(&status[tile], ((excl + agg) << 2) | 2u);
  return excl;
}

// The first round of a look-back, issued early: the loads complete in the
// background while the caller does other work.
struct LookRound {
  uint64_t st[kLookPerLane];
};
__device__ __forceinline__ void tile_resolve_issue(const uint64_t* status, int64_t tile, int lane, LookRound& r) {
#pragma unroll
  for (int i = 0; i < kLookPerLane; i++) {
    const int64_t idx = tile - 1 - (int64_t)lane * kLookPerLane - i;
    r.st[i] = (tile > 0 && idx >= 0) ? ld_relaxed_u64(&status[idx]) : 2u;
  }
}
// Finish the look-back started by tile_resolve_issue (whole warp) and
// publish the tile's inclusive prefix.
__device__ __forceinline__ uint64_t tile_resolve_finish(uint64_t* status, int64_t tile, uint64_t agg, int lane,
                                                       uint32_t* err, LookRound& r, uint32_t lim) {
  if (tile == 0) return 0;
  uint64_t excl = 0;
  int64_t j = tile - 1;
  bool timed_out = false;
  bool first_round = true;
  for (;;) {
    uint64_t st[kLookPerLane];
#pragma unroll
    for (int i = 0; i < kLookPerLane; i++) {
      const int64_t idx = j - (int64_t)lane * kLookPerLane - i;
      st[i] = first_round ? r.st[i] : (idx >= 0 ? ld_relaxed_u64(&status[idx]) : 2u);
    }
    first_round = false;
#pragma unroll
    for (int i = 0; i < kLookPerLane; i++) {
      const int64_t idx = j - (int64_t)lane * kLookPerLane - i;
      uint32_t it = 0;
      while ((st[i] & 3u) == 0) {
        if (++it > lim) {
          timed_out = true;
          st[i] = 2u;
          break;
        }
        __nanosleep(64);
        st[i] = ld_relaxed_u64(&status[idx]);
      }
    }
    int fi = kLookPerLane;
#pragma unroll
    for (int i = kLookPerLane - 1; i >= 0; i--)
      if ((st[i] & 3u) == 2u) fi = i;
    uint64_t part = 0;
#pragma unroll
    for (int i = 0; i < kLookPerLane; i++)
      if (i <= fi) part += st[i] >> 2;
    const unsigned pm = __ballot_sync(kFull, fi < kLookPerLane);
    const int first = pm ? __ffs(pm) - 1 : 32;
    excl += warp_sum_u64(lane <= first ? part : 0ull);
    if (pm) break;
    j -= 32 * kLookPerLane;
  }
  if (__any_sync(kFull, timed_out) && lane == 0 && err) atomicOr(err, 1u << 10);
  if (lane == 0) st_relaxed_u64(&status[tile], ((excl + agg) << 2) | 2u);
  return excl;
}

// Look-back of a tile whose aggregate is already published, in one go (out
// of line: used only for tiles too large for the pack's image).
__device__ __noinline__ uint64_t tile_resolve_now(uint64_t* status, int64_t tile, uint64_t agg, int lane,
                                                  uint32_t* err, uint32_t lim) {
  LookRound r;
  tile_resolve_issue(status, tile, lane, r);
  return tile_resolve_finish(status, tile, agg, lane, err, r, lim);
}

__device__ uint64_t tile_lookback(uint64_t* status, int64_t tile, uint64_t agg, int lane, uint32_t* err, uint32_t lim) {
  if (lane == 0) tile_publish(status, tile, agg);
  return tile_resolve(status, tile, agg, lane, err, lim);
}

template <bool U64>
__global__ void __launch_bounds__(kThreads) pack_kernel(PackArgs a) {
  extern __shared__ uint4 smem4[];
  constexpr int kSlot = Shape<U64>::kSlot;
  uint8_t* slots = (uint8_t*)smem4;
  uint32_t* hb_all = (uint32_t*)(slots + kTile * kSlot + 16);
  __shared__ int s_len[kTile];
  __shared__ int s_off[kTile];
  __shared__ int64_t s_tile;
  __shared__ uint64_t s_prefix;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* hb = hb_all + warp * kBlock;

  for (;;) {
    if (tid == 0) s_tile = (int64_t)atomicAdd((unsigned long long*)a.counter, 1ull);
    __syncthreads();
    const int64_t tile = s_tile;
    if (tile >= a.n_tiles) break;
    const int64_t b0 = tile * kTile;

#pragma unroll
    for (int j = 0; j < kBlocksPerWarp; j++) {
      const int lb = warp * kBlocksPerWarp + j;
      const int64_t b = b0 + lb;
      int len = 0;
      if (b < a.n_blocks) {
        uint64_t first;
        int n;
        block_span(a.val_off, a.block_start, a.n_streams, b, &first, &n);
        if (U64) {
          const uint64_t* vp = (const uint64_t*)a.values + first;
          uint64_t x[4];
#pragma unroll
          for (int k = 0; k < 4; k++) x[k] = (lane + 32 * k < n) ? __ldcs(vp + lane + 32 * k) : 0ull;
          len = warp_pack_block64(x, n, a.flag, slots, lb * kSlot, hb, lane);
        } else {
          const uint32_t* vp = (const uint32_t*)a.values + first;
          uint32_t v[4];
#pragma unroll
          for (int k = 0; k < 4; k++) v[k] = (lane + 32 * k < n) ? __ldcs(vp + lane + 32 * k) : 0u;
          len = warp_pack_block(v, n, a.flag, kTypeU32, kModePlain, 0, slots, lb * kSlot, hb, lane);
        }
      }
      if (lane == 0) s_len[lb] = len;
    }
    __syncthreads();

    if (warp == 0) {
      const int l = lane < kTile ? s_len[lane] : 0;
      const int incl = warp_incl_scan(l, lane);
      if (lane < kTile) s_off[lane] = incl - l;
      const uint64_t agg = (uint64_t)__shfl_sync(kFull, incl, 31);
      const uint64_t prefix = tile_lookback(a.tile_status, tile, agg, lane, a.err, a.spin_limit);
      if (lane == 0) s_prefix = prefix;
    }
    __syncthreads();

    const uint64_t prefix = s_prefix;
#pragma unroll
    for (int j = 0; j < kBlocksPerWarp; j++) {
      const int lb = warp * kBlocksPerWarp + j;
      const int64_t b = b0 + lb;
      if (b < a.n_blocks) {
        const uint64_t g = prefix + (uint64_t)s_off[lb];
        const int len = s_len[lb];
        if (g + (uint64_t)len <= a.out_cap) {
          warp_copy_out((const uint32_t*)(slots + lb * kSlot), len, a.out, g, lane);
        } else if (lane == 0 && a.err) {
          atomicOr(a.err, 1u << 9);
        }
        if (lane == 0) {
          a.block_off[b] = g;
          if (b == a.n_blocks - 1) a.block_off[a.n_blocks] = g + (uint64_t)len;
        }
      }
    }
    __syncthreads();
  }
}

// ------------------------------------------------------------------------
// batched unpack
// ------------------------------------------------------------------------
template <bool U64>
__global__ void __launch_bounds__(kThreads) unpack_kernel(UnpackArgs a) {
  extern __shared__ uint4 smem4[];
  constexpr int kStage = Shape<U64>::kStage;
  constexpr int kMax = Shape<U64>::kMax;
  uint8_t* stage = (uint8_t*)smem4;
  uint32_t* hb_all = (uint32_t*)(stage + kTile * kStage + 64);
  __shared__ uint64_t s_boff[kTile + 1];
  __shared__ int s_contig;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  uint32_t* hb = hb_all + warp * kBlock;
  const int64_t b0 = (int64_t)blockIdx.x * kTile;
  const int nb = (int)min((int64_t)kTile, a.n_blocks - b0);

  if (tid <= nb) s_boff[tid] = a.block_off[b0 + tid];
  __syncthreads();
  if (tid == 0) {
    int ok = 1;
    for (int j = 0; j < nb; j++) {
      const uint64_t s = s_boff[j], e = s_boff[j + 1];
      if (e < s || e - s > (uint64_t)kMax || e > a.packed_len) ok = 0;
    }
    s_contig = ok;
  }
  __syncthreads();
  const bool contig = s_contig != 0;
  if (contig) {
    stage_bytes(smem4, a.packed, a.packed_len, s_boff[0], s_boff[nb], tid, kThreads);
  } else {
    for (int j = warp; j < nb; j += kWarps) {
      const uint64_t s = s_boff[j], e = s_boff[j + 1];
      if (e >= s && e - s <= (uint64_t)kMax && e <= a.packed_len)
        stage_bytes((uint4*)(stage + j * kStage), a.packed, a.packed_len, s, e, lane, 32);
    }
  }
  __syncthreads();

  const SmemBytes sb{(const uint32_t*)stage};
  const int base0 = (int)(((uintptr_t)a.packed + s_boff[0]) & 15);
#pragma unroll
  for (int j = 0; j < kBlocksPerWarp; j++) {
    const int lb = warp * kBlocksPerWarp + j;
    if (lb >= nb) break;
    const int64_t b = b0 + lb;
    const uint64_t s = s_boff[lb], e = s_boff[lb + 1];
    uint64_t first;
    int want;
    block_span(a.val_off, a.block_start, a.n_streams, b, &first, &want);
    int status = kOK, ovf = 0;
    if (e < s || e - s > (uint64_t)kMax || e > a.packed_len) {
      status = kErrCountMismatch;
    } else {
      const int len = (int)(e - s);
      const int blk = contig ? base0 + (int)(s - s_boff[0])
                             : lb * kStage + (int)(((uintptr_t)a.packed + s) & 15);
      UnpackResult r;
      if (U64) {
        uint64_t x[4];
        r = warp_unpack_block64(sb, blk, len, x, hb, lane);
        if (r.status == kOK && (r.count != want || r.consumed != len)) r.status = kErrCountMismatch;
        if (r.status == kOK) {
          uint64_t* op = (uint64_t*)a.values + first;
#pragma unroll
          for (int k = 0; k < 4; k++)
            if (lane + 32 * k < want) __stcs(op + lane + 32 * k, x[k]);
        }
      } else {
        uint32_t v[4];
        r = warp_unpack_block(sb, blk, len, false, v, hb, lane);
        if (r.status == kOK && (r.count != want || r.consumed != len)) r.status = kErrCountMismatch;
        if (r.status == kOK) {
          uint32_t* op = (uint32_t*)a.values + first;
#pragma unroll
          for (int k = 0; k < 4; k++)
            if (lane + 32 * k < want) __stcs(op + lane + 32 * k, v[k]);
        }
      }
      status = r.status;
      ovf = r.ovf;
    }
    if (lane == 0) {
      if (a.block_status) a.block_status[b] = status | (ovf << 8);
      if (status != kOK && a.err) atomicOr(a.err, 1u << status);
    }
  }
}

// ------------------------------------------------------------------------
// quad-per-block batched kernels (uint32): a warp codes 8 blocks at once
// ------------------------------------------------------------------------
constexpr int kQWarps = 4;                 // warps per CTA
constexpr int kQTile = kQWarps * 8;        // blocks per CTA tile
constexpr int kQThreads = kQWarps * 32;
constexpr int kQStage = 8 * 528;           // per-warp staging budget (8 blocks up to 528 B)
constexpr int kQStagePad = 128;            // readable slack past the staged bytes
constexpr int kQImage = kQTile * 288;      // pack tile image budget

struct QuadUnpackSmem {
  uint4 stage[kQWarps][(kQStage + kQStagePad) / 16];
  uint4 patch[kQWarps][8][kBlock / 4 + 1];  // +16 B: quads start on different banks
};

__global__ void __launch_bounds__(kQThreads) unpack_quad_kernel(UnpackArgs a) {
  extern __shared__ uint4 smem4[];
  QuadUnpackSmem& S = *(QuadUnpackSmem*)smem4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int q = lane >> 2, j = lane & 3;
  const unsigned qm = quad::quad_mask(lane);
  const int64_t b0 = ((int64_t)blockIdx.x * kQWarps + warp) * 8;
  if (b0 >= a.n_blocks) return;
  const int nb = (int)min((int64_t)8, a.n_blocks - b0);
  // block offsets of the warp's 8 blocks
  const uint64_t my_off = lane <= nb ? a.block_off[b0 + lane] : 0ull;
  const uint64_t off0 = __shfl_sync(kFull, my_off, 0);
  const uint64_t off1 = __shfl_sync(kFull, my_off, nb);
  const uint64_t next_off = __shfl_down_sync(kFull, my_off, 1);
  const bool ok = lane >= nb ||
                  (next_off >= my_off && next_off - my_off <= (uint64_t)kMaxBlock32 && next_off <= a.packed_len);
  const bool all_ok = __all_sync(kFull, ok);
  // this quad's block bounds (read by every lane before quads diverge)
  const uint64_t s = __shfl_sync(kFull, my_off, q), e = __shfl_sync(kFull, my_off, q + 1);
  const uintptr_t gbase = (uintptr_t)a.packed;
  const int ph = (int)((gbase + off0) & 15);
  const bool staged = all_ok && (int64_t)(off1 - off0) + ph + 16 <= kQStage;
  if (staged) stage_bytes(S.stage[warp], a.packed, a.packed_len, off0, off1, lane, 32);
  __syncwarp();
  if (q >= nb) return;
  const int64_t b = b0 + q;
  uint64_t first;
  int want;
  block_span(a.val_off, a.block_start, a.n_streams, b, &first, &want);
  int status = kOK, ovf = 0;
  if (e < s || e - s > (uint64_t)kMaxBlock32 || e > a.packed_len) {
    status = kErrCountMismatch;
  } else {
    const int len = (int)(e - s);
    uint32_t x[8][4];
    uint32_t* patch = (uint32_t*)S.patch[warp][q];
    quad::QResult r;
    if (staged) {
      r = quad::quad_unpack_block(SmemBytes{(const uint32_t*)S.stage[warp]}, ph + (int64_t)(s - off0), len, false, x,
                                  patch, j, qm);
    } else {
      r = quad::quad_unpack_block(GlobalBytes{a.packed + s, len}, 0, len, false, x, patch, j, qm);
    }
    if (r.status == kOK && (r.count != want || r.consumed != len)) r.status = kErrCountMismatch;
    if (r.status == kOK) {
      uint32_t* op = (uint32_t*)a.values + first;
      if (want == kBlock) {
        quad::quad_store_full(op, x, patch, j, qm);
      } else {
#pragma unroll
        for (int v = 0; v < 8; v++)
#pragma unroll
          for (int k = 0; k < 4; k++)
            if (16 * v + 4 * j + k < want) op[16 * v + 4 * j + k] = x[v][k];
      }
    }
    status = r.status;
    ovf = r.ovf;
  }
  if (j == 0) {
    if (a.block_status) a.block_status[b] = status | (ovf << 8);
    if (status != kOK && a.err) atomicOr(a.err, 1u << status);
  }
}

// Pipelined variant: persistent warps walk groups of 8 blocks with a stride
// of the whole grid; while a warp decodes group g its next group's bytes
// are already in flight into the second staging buffer (cp.async, 16-byte
// chunks, no registers held) and the block offsets of the group after
// that are loading.  Groups that do not fit a buffer take the one-block-
// per-round path of unpack_quad_kernel.
// per-buffer budget: 8 blocks of up to 264 bytes (narrow batches) or of up
// to 528 bytes (batches whose blocks are wide)
constexpr int kPStageNarrow = 8 * 264;
constexpr int kPStageWide = 8 * 528;
template <int STAGE, int NBUF = 2>
struct QuadPipeSmem {
  uint4 stage[kQWarps][NBUF][(STAGE + kQStagePad) / 16];
  uint4 patch[kQWarps][8][kBlock / 4 + 1];  // +16 B: quads start on different banks
};

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

// Issue the staging of bytes [g0, g1) of buf as stage_bytes lays them out;
// chunks that are not wholly inside the buffer are copied synchronously.
__device__ __forceinline__ void stage_bytes_async(uint4* dst16, const uint8_t* buf, uint64_t buf_len, uint64_t g0,
                                                  uint64_t g1, int lane) {
  const uintptr_t lo = (uintptr_t)buf, hi = lo + buf_len;
  const uintptr_t a0 = (lo + g0) & ~(uintptr_t)15;
  const uintptr_t a1 = (lo + g1 + 15) & ~(uintptr_t)15;
  const int nch = (int)((a1 - a0) >> 4);
  for (int c = lane; c < nch; c += 32) {
    const uintptr_t a = a0 + 16 * (uintptr_t)c;
    if (a >= lo && a + 16 <= hi) {
      cp_async16(&dst16[c], (const void*)a);
    } else {
      uint32_t w[4] = {0, 0, 0, 0};
      for (int bb = 0; bb < 16; bb++) {
        const uintptr_t x = a + bb;
        if (x >= lo && x < hi) w[bb >> 2] |= (uint32_t)(*(const uint8_t*)x) << ((bb & 3) * 8);
      }
      dst16[c] = make_uint4(w[0], w[1], w[2], w[3]);
    }
  }
}

struct GroupInfo {
  uint64_t off;   // lane l <= nb: block_off[b0 + l]
  int64_t b0;
  int nb;
  int s0;         // stream of block b0 (lane 0; broadcast when used)
};

__device__ __forceinline__ GroupInfo group_load(const UnpackArgs& a, int64_t g, int lane) {
  GroupInfo gi;
  gi.b0 = g * 8;
  gi.nb = gi.b0 < a.n_blocks ? (int)min((int64_t)8, a.n_blocks - gi.b0) : 0;
  gi.off = (gi.nb > 0 && lane <= gi.nb) ? a.block_off[gi.b0 + lane] : 0ull;
  gi.s0 = (gi.nb > 0 && lane == 0) ? stream_of(a.block_start, a.n_streams, gi.b0) : 0;
  return gi;
}

// whether a group's contiguous bytes fit one staging buffer (warp-uniform)
template <int STAGE, int MAXB = kMaxBlock32>
__device__ __forceinline__ bool group_fits(const UnpackArgs& a, const GroupInfo& gi, int lane) {
  const uint64_t next = __shfl_down_sync(kFull, gi.off, 1);
  const bool ok = lane >= gi.nb || (next >= gi.off && next - gi.off <= (uint64_t)MAXB && next <= a.packed_len);
  const uint64_t o0 = __shfl_sync(kFull, gi.off, 0), o1 = __shfl_sync(kFull, gi.off, gi.nb);
  const int ph = (int)(((uintptr_t)a.packed + o0) & 15);
  return __all_sync(kFull, ok) && (int64_t)(o1 - o0) + ph + 16 <= STAGE;
}

// Mean packed block length above which a batch takes the wide staging.
constexpr uint64_t kWideMean = 240;
// The uint64 staging: groups of 8 single-sub-block blocks (narrow, the
// uint32 wide budget) or of 8 two-block pairs of up to 1056 bytes (wide).
constexpr int kP64StageWide = 8 * 1056;
constexpr uint64_t kWideMean64 = 500;

// Decode and store uint64 block at staging offset blk (len bytes) by a quad
// (unpackUint64Block, uint64.go:191-266): the first uint32 sub-block, then
// for a two-block pair the upper-halves sub-block after it, both through
// one quad decode call in a rolled loop (one copy of the decoder in the
// kernel: three inlined copies overflowed the instruction cache); values
// are joined in registers and stored as 16-byte pairs where the output
// allows.  status / ovf are quad-uniform; nothing is stored for a block
// that fails.
__device__ __forceinline__ void quad64_block(const SmemBytes& sb, int blk, int len, uint64_t* op, int want,
                                             uint32_t* patch, int j, unsigned qm, int& status, int& ovf) {
  status = kOK;
  ovf = 0;
  if (len < 4) { status = kErrInvalidBuffer; return; }
  const uint32_t h = sb.u32(blk);
  if (((h >> 13) & 3) != 3) { status = kErrUnsupportedType; return; }
  const int forw = (int)((h >> 15) & 3);
  const int exc = (int)(h >> 24);
  const bool two = (h & kHdrCombine) != 0;
  // FOR64 (8-byte base in front of the payload) or fit-32: one sub-block
  uint64_t base = 0;
  if (!two && forw == 3) {
    const int off = 4 + (exc > 0 ? 2 : 0);
    if (len < off + 8) { status = kErrInvalidBuffer; return; }
    base = sb.u64(blk + off);
  }
  uint32_t x[8][4], xl[8][4];
  int sub = blk, avail = len, count = 0, c1 = 0;
#pragma unroll 1
  for (int part = 0; part < (two ? 2 : 1); part++) {
    // the width-generic payload loop: the per-width copies of the payload
    // code cost this kernel more in instruction-cache misses than they save
    const quad::QResult r = quad::quad_unpack_block<SmemBytes, false>(sb, sub, avail, true, x, patch, j, qm);
    if (r.status != kOK) { status = r.status; ovf = r.ovf; return; }
    if (part == 0) {
      count = r.count;
      c1 = r.consumed;
      if (two) {
        // the reference's order of checks for a pair (uint64.go:226-262)
        const int meta = 4 + (exc > 0 ? 2 : 0) + ((1 << forw) >> 1) + 2;  // its block2Len field ends here
        if (len < meta) { status = kErrInvalidBuffer; return; }
        const int b2len = (int)sb.u16(blk + meta - 2);
        if (c1 + b2len > len) { status = kErrInvalidBuffer; return; }
        sub = blk + c1;
        avail = b2len;
#pragma unroll
        for (int v = 0; v < 8; v++)
#pragma unroll
          for (int k = 0; k < 4; k++) xl[v][k] = x[v][k];
      }
    } else {
      if (r.count != count) { status = kErrInvalidBuffer; return; }
      c1 += avail;
    }
  }
  if (count != want || c1 != len) { status = kErrCountMismatch; return; }
  const bool full = want == kBlock && ((uintptr_t)op & 15) == 0;
#pragma unroll
  for (int v = 0; v < 8; v++) {
    const int i = 16 * v + 4 * j;
    uint64_t y[4];
#pragma unroll
    for (int k = 0; k < 4; k++) y[k] = two ? (((uint64_t)x[v][k] << 32) | xl[v][k]) : base + x[v][k];
    if (full) {
      __stcs((ulonglong2*)(op + i), make_ulonglong2(y[0], y[1]));
      __stcs((ulonglong2*)(op + i + 2), make_ulonglong2(y[2], y[3]));
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (i + k < want) op[i + k] = y[k];
    }
  }
}

// AUTO: the narrow and the wide instance are both launched; each works out
// from the block offsets which of them the batch's mean block length calls
// for, and the other returns at once (same inputs, same answer).  U64: a
// quad per uint64 block (quad64_block), everything else as for uint32.
// NBUF 1: one staging buffer per warp, filled and waited for at the top of
// each group (twice the resident warps of the double buffer for the large
// uint64 budget, which hides the wait instead).
template <int STAGE, bool U64, int NBUF>
__device__ __forceinline__ void pipe_body(const UnpackArgs& a, uint4* smem4) {
  QuadPipeSmem<STAGE, NBUF>& S = *(QuadPipeSmem<STAGE, NBUF>*)smem4;
  constexpr int kMaxB = U64 ? kMaxBlock64 : kMaxBlock32;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int q = lane >> 2, j = lane & 3;
  const unsigned qm = quad::quad_mask(lane);
  const int64_t n_groups = (a.n_blocks + 7) / 8;
  const int64_t stride = (int64_t)gridDim.x * kQWarps;
  int64_t g = (int64_t)blockIdx.x * kQWarps + warp;
  if (g >= n_groups) return;
  uint32_t* patch = (uint32_t*)S.patch[warp][q];

  GroupInfo cur = group_load(a, g, lane);
  bool cur_fits = group_fits<STAGE, kMaxB>(a, cur, lane);
  if (NBUF == 2) {
    if (cur_fits)
      stage_bytes_async(S.stage[warp][0], a.packed, a.packed_len, __shfl_sync(kFull, cur.off, 0),
                        __shfl_sync(kFull, cur.off, cur.nb), lane);
    cp_async_commit();
  }
  GroupInfo nxt = group_load(a, g + stride, lane);
  for (int it = 0; g < n_groups; it++, g += stride) {
    const int buf = NBUF == 2 ? (it & 1) : 0;
    bool nxt_fits = false;
    GroupInfo nn;
    if constexpr (NBUF == 2) {
      // put the next group in flight, and start loading the one after it
      nxt_fits = nxt.nb > 0 && group_fits<STAGE, kMaxB>(a, nxt, lane);
      if (nxt_fits)
        stage_bytes_async(S.stage[warp][buf ^ 1], a.packed, a.packed_len, __shfl_sync(kFull, nxt.off, 0),
                          __shfl_sync(kFull, nxt.off, nxt.nb), lane);
      cp_async_commit();
      nn = group_load(a, g + 2 * stride, lane);
      cp_async_wait1();
    } else {
      // this group now; the next group's offsets are already loading
      if (cur_fits)
        stage_bytes_async(S.stage[warp][0], a.packed, a.packed_len, __shfl_sync(kFull, cur.off, 0),
                          __shfl_sync(kFull, cur.off, cur.nb), lane);
      cp_async_commit();
      asm volatile("cp.async.wait_all;" ::: "memory");
    }
    __syncwarp();

    const int nb = cur.nb;
    const uint64_t off0 = __shfl_sync(kFull, cur.off, 0);
    const uint64_t s = __shfl_sync(kFull, cur.off, q), e = __shfl_sync(kFull, cur.off, q + 1);
    const bool bad = e < s || e - s > (uint64_t)kMaxB || e > a.packed_len;
    const int64_t b = cur.b0 + q;
    const int s0 = __shfl_sync(kFull, cur.s0, 0);
    const int rounds = cur_fits ? 1 : nb;
    const uint4* stg = S.stage[warp][buf];
#pragma unroll 1
    for (int rd = 0; rd < rounds; rd++) {
      if (!cur_fits) {
        // one block per round, synchronously, through this group's buffer
        const uint64_t rs = __shfl_sync(kFull, cur.off, rd), re = __shfl_sync(kFull, cur.off, rd + 1);
        __syncwarp();
        if (re >= rs && re - rs <= (uint64_t)kMaxB && re <= a.packed_len)
          stage_bytes(S.stage[warp][buf], a.packed, a.packed_len, rs, re, lane, 32);
        __syncwarp();
      }
      if (cur_fits ? q < nb : q == rd) {
        uint64_t first;
        int want;
        span_in(a.val_off, a.block_start, stream_from(a.block_start, a.n_streams, s0, b), b, &first, &want);
        int status = kOK, ovf = 0;
        if (bad) {
          status = kErrCountMismatch;
        } else {
          const int len = (int)(e - s);
          const int blk = cur_fits ? (int)(((uintptr_t)a.packed + off0) & 15) + (int)(s - off0)
                                   : (int)(((uintptr_t)a.packed + s) & 15);
          if constexpr (U64) {
            quad64_block(SmemBytes{(const uint32_t*)stg}, blk, len, (uint64_t*)a.values + first, want, patch, j, qm,
                         status, ovf);
          } else {
            uint32_t x[8][4];
            const quad::QResult r =
                quad::quad_unpack_block(SmemBytes{(const uint32_t*)stg}, blk, len, false, x, patch, j, qm);
            status = r.status;
            ovf = r.ovf;
            if (status == kOK && (r.count != want || r.consumed != len)) status = kErrCountMismatch;
            if (status == kOK) {
              uint32_t* op = (uint32_t*)a.values + first;
              if (want == kBlock) {
                quad::quad_store_full(op, x, patch, j, qm);
              } else {
#pragma unroll
                for (int v = 0; v < 8; v++)
#pragma unroll
                  for (int k = 0; k < 4; k++)
                    if (16 * v + 4 * j + k < want) op[16 * v + 4 * j + k] = x[v][k];
              }
            }
          }
        }
        if (j == 0) {
          if (a.block_status) a.block_status[b] = status | (ovf << 8);
          if (status != kOK && a.err) atomicOr(a.err, 1u << status);
        }
      }
    }
    __syncwarp();
    if constexpr (NBUF == 2) {
      cur = nxt;
      cur_fits = nxt_fits;
      nxt = nn;
    } else {
      cur = nxt;
      cur_fits = cur.nb > 0 && group_fits<STAGE, kMaxB>(a, cur, lane);
      nxt = group_load(a, g + 2 * stride, lane);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

template <int STAGE, bool AUTO, bool U64 = false, int NBUF = 2>
__global__ void __launch_bounds__(kQThreads, U64 ? 4 : 5) unpack_quad_pipe_kernel(UnpackArgs a) {
  extern __shared__ uint4 smem4[];
  if (AUTO) {
    const uint64_t span = a.block_off[a.n_blocks] - a.block_off[0];
    const bool wide = span > (U64 ? kWideMean64 : kWideMean) * (uint64_t)a.n_blocks;
    if (wide != (STAGE == (U64 ? kP64StageWide : kPStageWide))) return;
    if (!wide && span <= a.lane_mean * (uint64_t)a.n_blocks) return;
  }
  pipe_body<STAGE, U64, NBUF>(a, smem4);
}

// Thread-per-block uint32 unpack (utl_unlane.cuh): persistent warps over
// tiles of 32 blocks.  AUTO: launched next to the two pipe instances; each
// of the three works out from the block offsets whether the batch's mean
// block length is its class, the other two return at once.
constexpr int kLUStage1 = 32 * 264;  // one buffer: a tile of 32 blocks of up to 264 bytes
constexpr int kLUStage2 = 5120;      // two buffers: tiles of up to 160 bytes a block
template <int NBUF, int STAGE, int W>
struct LaneUnpackSmem {
  uint4 stage[W][NBUF][(STAGE + kQStagePad) / 16];
  // the output chunk of the tile's 32 blocks; after the chunks, the quads'
  // exception scratch of the fallback (8 x 132 words)
  uint4 tile[W][32 * unlane::kTileStride / 16];
};
static_assert(32 * unlane::kTileStride >= 8 * (kBlock + 4) * 4, "fallback scratch");

// The quad decoder on the blocks of `todo` (bit i: block b0 + i).  staged:
// the tile's bytes are in stg with block i at ph + (s_i - s_0); otherwise
// rounds of consecutive blocks that fit are staged here one after the
// other.  Per-lane inputs are lane i's block values (s, e, first, want, ok).
template <int STAGE>
__device__ __forceinline__ void unlane_fallback(const UnpackArgs& a, uint4* stg, uint32_t* scratch, int64_t b0, int nb,
                                             uint32_t todo, bool staged, int ph, uint64_t s, uint64_t e,
                                             uint64_t first, int want, bool ok, int lane) {
  const int q = lane >> 2, j = lane & 3;
  const unsigned qm = quad::quad_mask(lane);
  uint32_t* patch = scratch + q * (kBlock + 4);
  const uint64_t s0 = __shfl_sync(kFull, s, 0);
  int next = 0;  // unstaged mode: first block of the next round
  while (staged ? todo != 0u : next < nb) {
    // this round's blocks: quad q takes block bi (or none)
    int bi = -1, rph = 0;
    uint64_t rbase = 0;
    if (staged) {
      const int cnt = min(8, __popc(todo));
      if (q < cnt) bi = (int)__fns(todo, 0, q + 1);
      const uint32_t cut = cnt < __popc(todo) ? (uint32_t)__fns(todo, 0, 9) : 32u;
      todo &= cut >= 32u ? 0u : ~((1u << cut) - 1u);
      rph = ph;
      rbase = s0;
    } else {
      // consecutive blocks from `next` whose bytes fit the buffer together
      const uint64_t rs = __shfl_sync(kFull, s, next);
      const int p0 = (int)(((uintptr_t)a.packed + rs) & 15);
      const bool fit = lane >= next && lane < next + 8 && lane < nb && ok && e >= rs &&
                       (int64_t)(e - rs) + p0 + 16 <= STAGE;
      const unsigned fm = __ballot_sync(kFull, fit) >> next;
      const int cnt = max(1, __ffs(~fm) - 1);  // a bad first block is a round of its own
      const bool any = (fm & 1u) != 0;
      if (any) {
        const uint64_t re = __shfl_sync(kFull, e, next + cnt - 1);
        stage_bytes(stg, a.packed, a.packed_len, rs, re, lane, 32);
      }
      if (q < cnt) bi = next + q;
      next += cnt;
      rph = p0;
      rbase = rs;
      __syncwarp();
    }
    const int src = bi >= 0 ? bi : 0;
    const uint64_t bs = __shfl_sync(kFull, s, src), be = __shfl_sync(kFull, e, src);
    const uint64_t bf = __shfl_sync(kFull, first, src);
    const int bw = __shfl_sync(kFull, want, src);
    const bool bok = __shfl_sync(kFull, ok ? 1 : 0, src) != 0;
    if (bi >= 0) {
      int status = kOK, ovf = 0;
      if (!bok) {
        status = kErrCountMismatch;
      } else {
        const int len = (int)(be - bs);
        const int blk = rph + (int)(bs - rbase);
        uint32_t x[8][4];
        const quad::QResult r = quad::quad_unpack_block(SmemBytes{(const uint32_t*)stg}, blk, len, false, x, patch, j, qm);
        status = r.status;
        ovf = r.ovf;
        if (status == kOK && (r.count != bw || r.consumed != len)) status = kErrCountMismatch;
        if (status == kOK) {
          uint32_t* op = (uint32_t*)a.values + bf;
          if (bw == kBlock) {
            quad::quad_store_full(op, x, patch, j, qm);
          } else {
#pragma unroll
            for (int v = 0; v < 8; v++)
#pragma unroll
              for (int k = 0; k < 4; k++)
                if (16 * v + 4 * j + k < bw) op[16 * v + 4 * j + k] = x[v][k];
          }
        }
      }
      if (j == 0) {
        if (a.block_status) a.block_status[b0 + bi] = status | (ovf << 8);
        if (status != kOK && a.err) atomicOr(a.err, 1u << status);
      }
    }
    __syncwarp();
  }
}

// The blocks of tile t as each lane sees its own (lane i: block 32t + i)
// and whether the tile's bytes fit one staging buffer of STAGE bytes.
struct LaneTile {
  uint64_t s, e, first;
  int want;
  bool ok, fits;
};
__device__ __forceinline__ int lane_tile_nb(const UnpackArgs& a, int64_t t) {
  return (int)min((int64_t)32, a.n_blocks - t * 32);
}
template <int STAGE>
__device__ __forceinline__ LaneTile lane_tile(const UnpackArgs& a, int64_t t, int lane) {
  LaneTile q;
  const int64_t b0 = t * 32;
  const int nb = lane_tile_nb(a, t);
  const bool mine = lane < nb;
  q.s = mine ? a.block_off[b0 + lane] : 0ull;
  q.e = mine ? a.block_off[b0 + lane + 1] : 0ull;
  q.ok = mine && q.e >= q.s && q.e - q.s <= (uint64_t)kMaxBlock32 && q.e <= a.packed_len;
  const uint64_t o0 = __shfl_sync(kFull, q.s, 0), oN = __shfl_sync(kFull, q.e, nb - 1);
  const int ph = (int)(((uintptr_t)a.packed + o0) & 15);
  // contiguous and in bounds: every block's end is the next one's start
  const uint64_t nxt_s = __shfl_down_sync(kFull, q.s, 1);
  const bool chain = !mine || lane == nb - 1 || nxt_s == q.e;
  q.fits = __all_sync(kFull, !mine || (q.ok && chain)) && (int64_t)(oN - o0) + ph + 16 <= STAGE;
  // the values each block decodes to
  const int s0 = __shfl_sync(kFull, lane == 0 ? stream_of(a.block_start, a.n_streams, b0) : 0, 0);
  q.first = 0;
  q.want = 0;
  if (mine)
    span_in(a.val_off, a.block_start, stream_from(a.block_start, a.n_streams, s0, b0 + lane), b0 + lane, &q.first,
            &q.want);
  return q;
}
// Stage tile q's bytes (when they fit) into stg.
__device__ __forceinline__ void lane_tile_stage(const UnpackArgs& a, const LaneTile& q, int nb, uint4* stg, int lane) {
  if (q.fits)
    stage_bytes_async(stg, a.packed, a.packed_len, __shfl_sync(kFull, q.s, 0), __shfl_sync(kFull, q.e, nb - 1), lane);
}

// Decode tile q (its bytes in stg when q.fits): the thread path's blocks
// row by row through the chunk tile, then the quad decoder on the rest.
template <int STAGE>
__device__ __forceinline__ void lane_tile_decode(const UnpackArgs& a, const LaneTile& q, int64_t b0, int nb,
                                                 uint4* stg, uint8_t* tileb, int lane) {
  using namespace unlane;
  const SmemBytes sb{(const uint32_t*)stg};
  uint8_t* T = tileb + lane * kTileStride;
  const bool mine = lane < nb;
  const uint64_t o0 = __shfl_sync(kFull, q.s, 0);
  const int ph = (int)(((uintptr_t)a.packed + o0) & 15);
  Plan f;
  const bool fast = q.fits && mine && plan(sb, ph + (int)(q.s - o0), (int)(q.e - q.s), q.want, f);
  const uint32_t fastm = __ballot_sync(kFull, fast);
  // the block's first value index, in the padding after its chunk rows: the
  // copy-out reads it with one shared load instead of two shuffles
  *(uint64_t*)(T + 64 * kRows) = q.first;
  if (fastm) {
      uint32_t cur[16], nxt[16];
      int wi = 0, ex = 0, np = 256, doff = 0;
#pragma unroll
      for (int i = 0; i < 16; i++) cur[i] = nxt[i] = 0;
      if (fast) {
        if (f.bw > 0) load_words(sb, f.pay, cur);
        if (f.bw > 4) load_words(sb, f.pay + 64, nxt);
        if (f.exc > 0) np = (int)sb.u8(f.xo);
        doff = f.nc;
      }
#pragma unroll 1
      for (int c = 0; c < 8 / kRows; c++) {
        if (fast) {
#pragma unroll
          for (int r = 0; r < kRows; r++) {
            const int v = c * kRows + r;
            const int sh = v * f.bw - 32 * wi;
            uint32_t y[16];
#pragma unroll
            for (int i = 0; i < 16; i++) y[i] = __funnelshift_r(cur[i], nxt[i], sh) & f.mask;
            if (f.delta) {
              // delta (delta.go:50-115): the per-lane running sum;
              // the previous row is still in the chunk tile's other slot
              // (the chunk copy-out only reads it), with the FOR base added
              const uint8_t* pr = T + 64 * ((r + kRows - 1) % kRows);
#pragma unroll
              for (int i = 0; i < 4; i++) {
                const uint4 p4 = *(const uint4*)(pr + 16 * i);
                const uint32_t pv[4] = {p4.x, p4.y, p4.z, p4.w};
#pragma unroll
                for (int k = 0; k < 4; k++)
                  y[4 * i + k] = (v == 0 ? 0u : pv[k] - f.base) + (f.zz ? zz_dec(y[4 * i + k]) : y[4 * i + k]);
              }
            }
#pragma unroll
            for (int i = 0; i < 16; i++) y[i] += f.base;
#pragma unroll
            for (int i = 0; i < 4; i++)
              *(uint4*)(T + 64 * r + 16 * i) = make_uint4(y[4 * i], y[4 * i + 1], y[4 * i + 2], y[4 * i + 3]);
            if ((v + 1) * f.bw >= 32 * (wi + 1)) {
#pragma unroll
              for (int i = 0; i < 16; i++) cur[i] = nxt[i];
              wi++;
              if (4 * (wi + 1) < f.bw) load_words(sb, f.pay + 64 * (wi + 1), nxt);
            }
          }
          // this chunk's exceptions (applyExceptions, exceptions.go:194-284):
          // the high bits above the FOR-added low bits, in list order
          while (np < 16 * kRows * (c + 1)) {
            const int code = (int)((f.cw >> (2 * ex)) & 3);
            uint32_t hv = sb.u32(f.svb + doff);
            if (code < 3) hv &= (1u << (8 * (code + 1))) - 1u;
            doff += code + 1;
            uint32_t* tp = (uint32_t*)(T + 64 * ((np >> 4) - c * kRows) + 4 * (np & 15));
            *tp = ((*tp - f.base) | shl32(hv, f.bw)) + f.base;
            ex++;
            np = ex < f.exc ? (int)sb.u8(f.xo + ex) : 256;
          }
        }
        __syncwarp();
        // the chunk's rows of every thread-path block, 16 bytes per lane
        const int part = lane % kLanesPerBlock;
#pragma unroll 4
        for (int it = 0; it < 32 / kBlocksPerStore; it++) {
          const int i = it * kBlocksPerStore + lane / kLanesPerBlock;
          const uint64_t fi = *(const uint64_t*)(tileb + i * kTileStride + 64 * kRows);
          if ((fastm >> i) & 1u) {
            const uint4 val = *(const uint4*)(tileb + i * kTileStride + 16 * part);
            uint32_t* op = (uint32_t*)a.values + fi + 16 * kRows * c + 4 * part;
            // 16-byte stores only at 16-byte addresses (the host pipeline's
            // pieces start their values at any value index)
            if (((uintptr_t)op & 15) == 0) {
              __stcs((uint4*)op, val);
            } else {
              op[0] = val.x;
              op[1] = val.y;
              op[2] = val.z;
              op[3] = val.w;
            }
          }
        }
        __syncwarp();
      }
    if (fast && a.block_status) a.block_status[b0 + lane] = kOK;
  }
  const uint32_t todo = __ballot_sync(kFull, mine && !fast);
  if (todo)
    unlane_fallback<STAGE>(a, stg, (uint32_t*)tileb, b0, nb, todo, q.fits, ph, q.s, q.e, q.first, q.want, q.ok, lane);
}

// NBUF 1: each tile is staged and waited for at the top of its turn; NBUF
// 2: the next tile's bytes are in flight while this one decodes (smaller
// buffers, tiles of up to 160 bytes a block; larger tiles take the quad
// decoder with their own staging).  W warps per CTA.
template <int NBUF, int STAGE, int W>
__device__ __forceinline__ void lane_body(const UnpackArgs& a, uint4* smem4) {
  LaneUnpackSmem<NBUF, STAGE, W>& S = *(LaneUnpackSmem<NBUF, STAGE, W>*)smem4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t n_tiles = (a.n_blocks + 31) / 32;
  const int64_t stride = (int64_t)gridDim.x * W;
  uint8_t* tileb = (uint8_t*)S.tile[warp];
  int64_t t = (int64_t)blockIdx.x * W + warp;
  if (t >= n_tiles) return;
  LaneTile cur = lane_tile<STAGE>(a, t, lane);
  if (NBUF == 2) {
    lane_tile_stage(a, cur, lane_tile_nb(a, t), S.stage[warp][0], lane);
    cp_async_commit();
  }
  for (int it = 0; t < n_tiles; it++, t += stride) {
    const int buf = NBUF == 2 ? (it & 1) : 0;
    LaneTile nxt;
    if constexpr (NBUF == 2) {
      if (t + stride < n_tiles) {
        nxt = lane_tile<STAGE>(a, t + stride, lane);
        lane_tile_stage(a, nxt, lane_tile_nb(a, t + stride), S.stage[warp][buf ^ 1], lane);
      }
      cp_async_commit();
      cp_async_wait1();
    } else {
      lane_tile_stage(a, cur, lane_tile_nb(a, t), S.stage[warp][0], lane);
      cp_async_commit();
      asm volatile("cp.async.wait_all;" ::: "memory");
    }
    __syncwarp();
    lane_tile_decode<STAGE>(a, cur, t * 32, lane_tile_nb(a, t), S.stage[warp][buf], tileb, lane);
    __syncwarp();
    if constexpr (NBUF == 2) {
      cur = nxt;
    } else {
      if (t + stride < n_tiles) cur = lane_tile<STAGE>(a, t + stride, lane);
    }
  }
  asm volatile("cp.async.wait_all;" ::: "memory");
}

template <bool AUTO, int NBUF, int STAGE, int W>
__global__ void __launch_bounds__(32 * W, 16 / W) unpack_lane_kernel(UnpackArgs a) {
  extern __shared__ uint4 smem4[];
  if (AUTO) {
    const uint64_t span = a.block_off[a.n_blocks] - a.block_off[0];
    if (span > a.lane_mean * (uint64_t)a.n_blocks) return;
  }
  lane_body<NBUF, STAGE, W>(a, smem4);
}

// The default uint32 unpack in one launch: the thread-per-block path for
// batches of at most kWideMean bytes a block on average, the quad pipeline
// with the large staging otherwise (both persistent, 4 warps per CTA, at
// most as much shared memory as the launch provides), chosen from the
// block offsets by every CTA alike.
constexpr size_t kAutoSmem = sizeof(LaneUnpackSmem<1, kLUStage1, 4>) > sizeof(QuadPipeSmem<kPStageWide, 2>)
                                 ? sizeof(LaneUnpackSmem<1, kLUStage1, 4>)
                                 : sizeof(QuadPipeSmem<kPStageWide, 2>);
__global__ void __launch_bounds__(kQThreads, 4) unpack_auto_kernel(UnpackArgs a) {
  extern __shared__ uint4 smem4[];
  const uint64_t span = a.block_off[a.n_blocks] - a.block_off[0];
  if (span <= kWideMean * (uint64_t)a.n_blocks) lane_body<1, kLUStage1, 4>(a, smem4);
  else pipe_body<kPStageWide, false, 2>(a, smem4);
}

// TMA-staged pipelined unpack (utl_unpack.cuh): persistent warps over
// groups of 8 blocks, NSTAGE groups in flight per warp, each group's bytes
// brought in by one bulk copy on its stage's mbarrier.
template <int STAGE, int NSTAGE>
struct QuadTmaSmem {
  uint4 stage[kQWarps][NSTAGE][(STAGE + kQStagePad) / 16];
  uint4 patch[kQWarps][8][kBlock / 4 + 1];  // +16 B: quads start on different banks
  uint64_t bar[kQWarps][NSTAGE];
};

// Offsets of group g for the TMA pipeline: lane l <= nb holds
// block_off[8g + l]; lane 0 also the stream of block 8g (in `s0`).
struct TmaGroup {
  uint64_t off;
  int s0;
};
__device__ __forceinline__ TmaGroup tma_group_load(const UnpackArgs& a, int64_t g, int lane) {
  TmaGroup t;
  const int64_t b0 = g * 8;
  const int nb = b0 < a.n_blocks ? (int)min((int64_t)8, a.n_blocks - b0) : 0;
  t.off = (nb > 0 && lane <= nb) ? a.block_off[b0 + lane] : 0ull;
  t.s0 = (nb > 0 && lane == 0) ? stream_of(a.block_start, a.n_streams, b0) : 0;
  return t;
}
__device__ __forceinline__ int tma_group_nb(const UnpackArgs& a, int64_t g) {
  const int64_t b0 = g * 8;
  return b0 < a.n_blocks ? (int)min((int64_t)8, a.n_blocks - b0) : 0;
}
template <int STAGE>
__device__ __forceinline__ bool tma_group_fits(const UnpackArgs& a, const TmaGroup& t, int nb, int lane) {
  if (nb <= 0) return false;
  GroupInfo gi;
  gi.off = t.off;
  gi.b0 = 0;
  gi.nb = nb;
  gi.s0 = 0;
  return group_fits<STAGE>(a, gi, lane);
}

// Copy the 16-byte chunks [c0, c1) of the aligned range starting at a0 (the
// chunks of buf's ends that the bulk copy leaves out) with plain loads;
// bytes outside the buffer read as zero.
__device__ __forceinline__ void stage_edge(uint4* dst16, uintptr_t a0, uintptr_t lo, uintptr_t hi, int c0, int c1,
                                           int lane) {
  for (int c = c0 + lane; c < c1; c += 32) {
    const uintptr_t a = a0 + 16 * (uintptr_t)c;
    uint32_t w[4] = {0, 0, 0, 0};
    for (int bb = 0; bb < 16; bb++) {
      const uintptr_t x = a + bb;
      if (x >= lo && x < hi) w[bb >> 2] |= (uint32_t)(*(const uint8_t*)x) << ((bb & 3) * 8);
    }
    dst16[c] = make_uint4(w[0], w[1], w[2], w[3]);
  }
}

// Put group gi (which fits the stage) in flight into dst: one bulk copy of
// the buffer's aligned interior part, plain loads for the edge chunks.
// Returns whether a bulk copy was issued (then bar completes with it).
__device__ __forceinline__ bool stage_issue(const UnpackArgs& a, const TmaGroup& gi, int nb, uint4* dst16,
                                            uint64_t* bar, int lane) {
  const uint64_t o0 = __shfl_sync(kFull, gi.off, 0), o1 = __shfl_sync(kFull, gi.off, nb);
  const uintptr_t lo = (uintptr_t)a.packed, hi = lo + a.packed_len;
  const uintptr_t a0 = (lo + o0) & ~(uintptr_t)15, a1 = (lo + o1 + 15) & ~(uintptr_t)15;
  const uintptr_t lo16 = (lo + 15) & ~(uintptr_t)15, hi16 = hi & ~(uintptr_t)15;
  const uintptr_t t0 = a0 > lo16 ? a0 : lo16, t1 = a1 < hi16 ? a1 : hi16;
  const int nch = (int)((a1 - a0) >> 4);
  if (t1 > t0) {
    if (lane == 0) {
      tma::proxy_fence();
      tma::mbar_expect_tx(bar, (uint32_t)(t1 - t0));
      tma::bulk_load((uint8_t*)dst16 + (t0 - a0), (const void*)t0, (uint32_t)(t1 - t0), bar);
    }
    const int c0 = (int)((t0 - a0) >> 4), c1 = (int)((t1 - a0) >> 4);
    if (c0 > 0) stage_edge(dst16, a0, lo, hi, 0, c0, lane);
    if (c1 < nch) stage_edge(dst16, a0, lo, hi, c1, nch, lane);
    return true;
  }
  stage_edge(dst16, a0, lo, hi, 0, nch, lane);
  return false;
}

template <int STAGE, int NSTAGE, bool AUTO, bool FAST>
__global__ void __launch_bounds__(kQThreads, 5) unpack_quad_tma_kernel(UnpackArgs a) {
  extern __shared__ uint4 smem4[];
  QuadTmaSmem<STAGE, NSTAGE>& S = *(QuadTmaSmem<STAGE, NSTAGE>*)smem4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (AUTO) {
    const uint64_t span = a.block_off[a.n_blocks] - a.block_off[0];
    const bool wide = span > kWideMean * (uint64_t)a.n_blocks;
    if (wide != (STAGE == kPStageWide)) return;
  }
  const int q = lane >> 2, j = lane & 3;
  const unsigned qm = quad::quad_mask(lane);
  const int64_t n_groups = (a.n_blocks + 7) / 8;
  const int64_t stride = (int64_t)gridDim.x * kQWarps;
  int64_t g = (int64_t)blockIdx.x * kQWarps + warp;
  if (g >= n_groups) return;
  uint32_t* patch = (uint32_t*)S.patch[warp][q];
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NSTAGE; s++) tma::mbar_init(&S.bar[warp][s], 1);
    tma::mbar_init_fence();
  }
  __syncwarp();
  const uint32_t lim = a.spin_limit;
  uint32_t pend = 0, phase = 0, fits = 0;  // per stage slot: copy in flight, parity of its next completion; per group: fits

  // groups in flight: gq[0] is the current group (stage st), gq[k] the
  // k-th after it
  TmaGroup gq[NSTAGE];
#pragma unroll
  for (int k = 0; k < NSTAGE; k++) {
    gq[k] = tma_group_load(a, g + k * stride, lane);
    if (tma_group_fits<STAGE>(a, gq[k], tma_group_nb(a, g + k * stride), lane)) fits |= 1u << k;
  }
#pragma unroll
  for (int k = 0; k < NSTAGE - 1; k++)
    if (((fits >> k) & 1u) && stage_issue(a, gq[k], tma_group_nb(a, g + k * stride), S.stage[warp][k],
                                          &S.bar[warp][k], lane))
      pend |= 1u << k;
  bool timed_out = false;
  int st = 0;  // stage of the current group
  for (; g < n_groups; g += stride) {
    // the group NSTAGE-1 ahead goes in flight into the stage freed last round
    const int sn = st == 0 ? NSTAGE - 1 : st - 1;
    if (((fits >> (NSTAGE - 1)) & 1u) &&
        stage_issue(a, gq[NSTAGE - 1], tma_group_nb(a, g + (NSTAGE - 1) * stride), S.stage[warp][sn],
                    &S.bar[warp][sn], lane))
      pend |= 1u << sn;
    if ((pend >> st) & 1u) {
      if (!tma::mbar_wait(&S.bar[warp][st], (phase >> st) & 1u, lim)) {
        timed_out = true;
        break;
      }
      pend &= ~(1u << st);
      phase ^= 1u << st;
    }
    __syncwarp();

    const int nb = tma_group_nb(a, g);
    const bool cur_fits = fits & 1u;
    const uint64_t off0 = __shfl_sync(kFull, gq[0].off, 0);
    const uint64_t s = __shfl_sync(kFull, gq[0].off, q), e = __shfl_sync(kFull, gq[0].off, q + 1);
    const bool bad = e < s || e - s > (uint64_t)kMaxBlock32 || e > a.packed_len;
    const int64_t b = g * 8 + q;
    const int s0 = __shfl_sync(kFull, gq[0].s0, 0);
    const int rounds = cur_fits ? 1 : nb;
    uint4* stg = S.stage[warp][st];
#pragma unroll 1
    for (int rd = 0; rd < rounds; rd++) {
      if (!cur_fits) {
        // one block per round, synchronously, through this group's buffer
        const uint64_t rs = __shfl_sync(kFull, gq[0].off, rd), re = __shfl_sync(kFull, gq[0].off, rd + 1);
        __syncwarp();
        if (re >= rs && re - rs <= (uint64_t)kMaxBlock32 && re <= a.packed_len)
          stage_bytes(stg, a.packed, a.packed_len, rs, re, lane, 32);
        __syncwarp();
      }
      if (cur_fits ? q < nb : q == rd) {
        uint64_t first;
        int want;
        span_in(a.val_off, a.block_start, stream_from(a.block_start, a.n_streams, s0, b), b, &first, &want);
        int status = kOK, ovf = 0;
        if (bad) {
          status = kErrCountMismatch;
        } else {
          const int len = (int)(e - s);
          const int blk = cur_fits ? (int)(((uintptr_t)a.packed + off0) & 15) + (int)(s - off0)
                                   : (int)(((uintptr_t)a.packed + s) & 15);
          uint32_t* op = (uint32_t*)a.values + first;
          const SmemBytes sb{(const uint32_t*)stg};
          quad::QFast f;
          uint32_t x[8][4];
          quad::QResult r;
          if (FAST && quad::fast_plan(sb, blk, len, j, qm, f)) r = quad::fast_decode(sb, blk, f, x, patch, j, qm);
          else r = quad::quad_unpack_block(sb, blk, len, false, x, patch, j, qm);
          status = r.status;
          ovf = r.ovf;
          if (status == kOK && (r.count != want || r.consumed != len)) status = kErrCountMismatch;
          if (status == kOK) {
            if (want == kBlock) {
              quad::quad_store_full(op, x, patch, j, qm);
            } else {
#pragma unroll
              for (int v = 0; v < 8; v++)
#pragma unroll
                for (int k = 0; k < 4; k++)
                  if (16 * v + 4 * j + k < want) op[16 * v + 4 * j + k] = x[v][k];
            }
          }
        }
        if (j == 0) {
          if (a.block_status) a.block_status[b] = status | (ovf << 8);
          if (status != kOK && a.err) atomicOr(a.err, 1u << status);
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < NSTAGE - 1; k++) gq[k] = gq[k + 1];
    fits >>= 1;
    gq[NSTAGE - 1] = tma_group_load(a, g + NSTAGE * stride, lane);
    if (tma_group_fits<STAGE>(a, gq[NSTAGE - 1], tma_group_nb(a, g + NSTAGE * stride), lane))
      fits |= 1u << (NSTAGE - 1);
    st = st == NSTAGE - 1 ? 0 : st + 1;
  }
  if (timed_out) {
    // record it, then let every copy still in flight land (bounded) before
    // the warp leaves
    if (lane == 0 && a.err) atomicOr(a.err, 1u << 10);
#pragma unroll
    for (int s2 = 0; s2 < NSTAGE; s2++)
      if ((pend >> s2) & 1u) tma::mbar_wait(&S.bar[warp][s2], (phase >> s2) & 1u, lim);
  }
}

// ------------------------------------------------------------------------
// uint64 unpack with TMA staging: an octet of lanes per uint64 block, 4
// blocks per warp.  The octet's first quad decodes the block's first
// uint32 sub-block (the only one of a FOR64 or fit-32 block), its second
// quad the upper-halves sub-block of a two-block pair at the same time
// (unpackUint64Block, uint64.go:191-266); the halves meet by one shuffle
// per pair of values and every lane stores 16-byte pairs of uint64.
// ------------------------------------------------------------------------
constexpr int kO64Stage = 4224;  // a group of 4 blocks of up to ~1 KB (two-block pairs of width 32)

__device__ __forceinline__ TmaGroup tma_group_load4(const UnpackArgs& a, int64_t g, int lane) {
  TmaGroup t;
  const int64_t b0 = g * 4;
  const int nb = b0 < a.n_blocks ? (int)min((int64_t)4, a.n_blocks - b0) : 0;
  t.off = (nb > 0 && lane <= nb) ? a.block_off[b0 + lane] : 0ull;
  t.s0 = (nb > 0 && lane == 0) ? stream_of(a.block_start, a.n_streams, b0) : 0;
  return t;
}
__device__ __forceinline__ int tma_group_nb4(const UnpackArgs& a, int64_t g) {
  const int64_t b0 = g * 4;
  return b0 < a.n_blocks ? (int)min((int64_t)4, a.n_blocks - b0) : 0;
}
template <int STAGE>
__device__ __forceinline__ bool tma_group_fits64(const UnpackArgs& a, const TmaGroup& t, int nb, int lane) {
  if (nb <= 0) return false;
  const uint64_t next = __shfl_down_sync(kFull, t.off, 1);
  const bool ok = lane >= nb || (next >= t.off && next - t.off <= (uint64_t)kMaxBlock64 && next <= a.packed_len);
  const uint64_t o0 = __shfl_sync(kFull, t.off, 0), o1 = __shfl_sync(kFull, t.off, nb);
  const int ph = (int)(((uintptr_t)a.packed + o0) & 15);
  return __all_sync(kFull, ok) && (int64_t)(o1 - o0) + ph + 16 <= STAGE;
}

// Decode and store uint64 block at staging offset blk (len bytes) by an
// octet (quad qh of it: 0 first sub-block, 1 upper halves).  Returns the
// status (octet-uniform) and overflow position.
__device__ __forceinline__ void oct64_block(const SmemBytes& sb, int blk, int len, uint64_t* op, int want,
                                            uint32_t* patch, int qh, int j, int lane, int& status, int& ovf) {
  const unsigned qm = quad::quad_mask(lane);
  const unsigned om = 0xFFu << (lane & 24);
  status = kOK;
  ovf = 0;
  if (len < 4) { status = kErrInvalidBuffer; return; }
  const uint32_t h = sb.u32(blk);
  if (((h >> 13) & 3) != 3) { status = kErrUnsupportedType; return; }
  const int forw = (int)((h >> 15) & 3);
  const int exc = (int)(h >> 24);
  uint32_t x[8][4];
  if (!(h & kHdrCombine)) {
    // FOR64 or fit-32: one sub-block, decoded by the first quad
    uint64_t base = 0;
    if (forw == 3) {
      const int off = 4 + (exc > 0 ? 2 : 0);
      if (len < off + 8) { status = kErrInvalidBuffer; return; }
      base = sb.u64(blk + off);
    }
    quad::QResult r{kOK, 0, 0, 0};
    if (qh == 0) r = quad::quad_unpack_block(sb, blk, len, true, x, patch, j, qm);
    int st = r.status, ov = r.ovf;
    if (st == kOK && (r.count != want || r.consumed != len)) st = kErrCountMismatch;
    st = __shfl_sync(om, st, lane & 24);
    ov = __shfl_sync(om, ov, lane & 24);
    status = st;
    ovf = ov;
    if (st != kOK || qh != 0) return;
    // 16-byte stores only where the output is 16-byte aligned (a stream may
    // start at any value index)
    if (want == kBlock && ((uintptr_t)op & 15) == 0) {
#pragma unroll
      for (int v = 0; v < 8; v++) {
        const int i = 16 * v + 4 * j;
        __stcs((ulonglong2*)(op + i), make_ulonglong2(base + x[v][0], base + x[v][1]));
        __stcs((ulonglong2*)(op + i + 2), make_ulonglong2(base + x[v][2], base + x[v][3]));
      }
    } else {
#pragma unroll
      for (int v = 0; v < 8; v++)
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (16 * v + 4 * j + k < want) op[16 * v + 4 * j + k] = base + x[v][k];
    }
    return;
  }
  // two-block pair: the first sub-block's length from its header (what its
  // decode consumes when it is valid), then both sub-blocks at once
  const int p1 = 4 + (exc > 0 ? 2 : 0) + ((1 << forw) >> 1) + 2;  // meta: its block2Len field ends here
  const int bw1 = (int)((h >> 8) & 31) * 4;
  const int c1 = (h & 0xFF) == 0 ? 4 : p1 + 16 * bw1 + (exc > 0 ? min(exc, 16) + (int)sb.u16(blk + 4) : 0);
  const int b2len = len >= p1 ? (int)sb.u16(blk + p1 - 2) : 0;
  const bool hi_ok = len >= p1 && c1 + b2len <= len;  // (an empty first sub-block consumes its header only)
  quad::QResult r{kOK, 0, 0, 0};
  if (qh == 0) r = quad::quad_unpack_block(sb, blk, len, true, x, patch, j, qm);
  else if (hi_ok) r = quad::quad_unpack_block(sb, blk + c1, b2len, true, x, patch, j, qm);
  const int st1 = __shfl_sync(om, r.status, lane & 24), ov1 = __shfl_sync(om, r.ovf, lane & 24);
  const int n1 = __shfl_sync(om, r.count, lane & 24), cons1 = __shfl_sync(om, r.consumed, lane & 24);
  const int st2 = __shfl_sync(om, r.status, (lane & 24) + 4), ov2 = __shfl_sync(om, r.ovf, (lane & 24) + 4);
  const int n2 = __shfl_sync(om, r.count, (lane & 24) + 4);
  // the reference's order: first sub-block, bounds of the pair, second
  // sub-block, equal counts (uint64.go:226-262)
  if (st1 != kOK) { status = st1; ovf = ov1; return; }
  if (len < p1 || cons1 + b2len > len) { status = kErrInvalidBuffer; return; }
  if (st2 != kOK) { status = st2; ovf = ov2; return; }
  if (n2 != n1) { status = kErrInvalidBuffer; return; }
  if (n1 != want || cons1 + b2len != len) { status = kErrCountMismatch; return; }
  // lane j of the first quad stores values 4j, 4j+1 of each row, lane j of
  // the second quad 4j+2, 4j+3: each sends the partner the halves it needs
  const int i0 = (qh == 0) ? 0 : 2;
#pragma unroll
  for (int v = 0; v < 8; v++) {
    const uint32_t a0 = __shfl_xor_sync(om, qh == 0 ? x[v][2] : x[v][0], 4);
    const uint32_t a1 = __shfl_xor_sync(om, qh == 0 ? x[v][3] : x[v][1], 4);
    const uint64_t v0 = qh == 0 ? ((uint64_t)a0 << 32 | x[v][0]) : ((uint64_t)x[v][2] << 32 | a0);
    const uint64_t v1 = qh == 0 ? ((uint64_t)a1 << 32 | x[v][1]) : ((uint64_t)x[v][3] << 32 | a1);
    const int i = 16 * v + 4 * j + i0;
    if (want == kBlock && ((uintptr_t)op & 15) == 0) {
      __stcs((ulonglong2*)(op + i), make_ulonglong2(v0, v1));
    } else {
      if (i < want) op[i] = v0;
      if (i + 1 < want) op[i + 1] = v1;
    }
  }
}

template <int NSTAGE>
struct Oct64Smem {
  uint4 stage[kQWarps][NSTAGE][(kO64Stage + kQStagePad) / 16];
  uint4 patch[kQWarps][8][kBlock / 4 + 1];
  uint64_t bar[kQWarps][NSTAGE];
};

template <int NSTAGE>
__global__ void __launch_bounds__(kQThreads, 4) unpack_oct64_tma_kernel(UnpackArgs a) {
  extern __shared__ uint4 smem4[];
  Oct64Smem<NSTAGE>& S = *(Oct64Smem<NSTAGE>*)smem4;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int ob = lane >> 3, qh = (lane >> 2) & 1, j = lane & 3;  // octet = block of the group
  const int64_t n_groups = (a.n_blocks + 3) / 4;
  const int64_t stride = (int64_t)gridDim.x * kQWarps;
  int64_t g = (int64_t)blockIdx.x * kQWarps + warp;
  if (g >= n_groups) return;
  uint32_t* patch = (uint32_t*)S.patch[warp][lane >> 2];
  if (lane == 0) {
#pragma unroll
    for (int s = 0; s < NSTAGE; s++) tma::mbar_init(&S.bar[warp][s], 1);
    tma::mbar_init_fence();
  }
  __syncwarp();
  const uint32_t lim = a.spin_limit;
  uint32_t pend = 0, phase = 0, fits = 0;
  TmaGroup gq[NSTAGE];
#pragma unroll
  for (int k = 0; k < NSTAGE; k++) {
    gq[k] = tma_group_load4(a, g + k * stride, lane);
    if (tma_group_fits64<kO64Stage>(a, gq[k], tma_group_nb4(a, g + k * stride), lane)) fits |= 1u << k;
  }
#pragma unroll
  for (int k = 0; k < NSTAGE - 1; k++)
    if (((fits >> k) & 1u) && stage_issue(a, gq[k], tma_group_nb4(a, g + k * stride), S.stage[warp][k],
                                          &S.bar[warp][k], lane))
      pend |= 1u << k;
  bool timed_out = false;
  int st = 0;
  for (; g < n_groups; g += stride) {
    const int sn = st == 0 ? NSTAGE - 1 : st - 1;
    if (((fits >> (NSTAGE - 1)) & 1u) &&
        stage_issue(a, gq[NSTAGE - 1], tma_group_nb4(a, g + (NSTAGE - 1) * stride), S.stage[warp][sn],
                    &S.bar[warp][sn], lane))
      pend |= 1u << sn;
    if ((pend >> st) & 1u) {
      if (!tma::mbar_wait(&S.bar[warp][st], (phase >> st) & 1u, lim)) {
        timed_out = true;
        break;
      }
      pend &= ~(1u << st);
      phase ^= 1u << st;
    }
    __syncwarp();
    const int nb = tma_group_nb4(a, g);
    const bool cur_fits = fits & 1u;
    const uint64_t off0 = __shfl_sync(kFull, gq[0].off, 0);
    const uint64_t s = __shfl_sync(kFull, gq[0].off, ob), e = __shfl_sync(kFull, gq[0].off, ob + 1);
    const bool bad = e < s || e - s > (uint64_t)kMaxBlock64 || e > a.packed_len;
    const int64_t b = g * 4 + ob;
    const int s0 = __shfl_sync(kFull, gq[0].s0, 0);
    const int rounds = cur_fits ? 1 : nb;
    uint4* stg = S.stage[warp][st];
#pragma unroll 1
    for (int rd = 0; rd < rounds; rd++) {
      if (!cur_fits) {
        const uint64_t rs = __shfl_sync(kFull, gq[0].off, rd), re = __shfl_sync(kFull, gq[0].off, rd + 1);
        __syncwarp();
        if (re >= rs && re - rs <= (uint64_t)kMaxBlock64 && re <= a.packed_len)
          stage_bytes(stg, a.packed, a.packed_len, rs, re, lane, 32);
        __syncwarp();
      }
      if (cur_fits ? ob < nb : ob == rd) {
        uint64_t first;
        int want;
        span_in(a.val_off, a.block_start, stream_from(a.block_start, a.n_streams, s0, b), b, &first, &want);
        int status = kOK, ovf = 0;
        if (bad) {
          status = kErrCountMismatch;
        } else {
          const int len = (int)(e - s);
          const int blk = cur_fits ? (int)(((uintptr_t)a.packed + off0) & 15) + (int)(s - off0)
                                   : (int)(((uintptr_t)a.packed + s) & 15);
          oct64_block(SmemBytes{(const uint32_t*)stg}, blk, len, (uint64_t*)a.values + first, want, patch, qh, j,
                      lane, status, ovf);
        }
        if ((lane & 7) == 0) {
          if (a.block_status) a.block_status[b] = status | (ovf << 8);
          if (status != kOK && a.err) atomicOr(a.err, 1u << status);
        }
      }
    }
    __syncwarp();
#pragma unroll
    for (int k = 0; k < NSTAGE - 1; k++) gq[k] = gq[k + 1];
    fits >>= 1;
    gq[NSTAGE - 1] = tma_group_load4(a, g + NSTAGE * stride, lane);
    if (tma_group_fits64<kO64Stage>(a, gq[NSTAGE - 1], tma_group_nb4(a, g + NSTAGE * stride), lane))
      fits |= 1u << (NSTAGE - 1);
    st = st == NSTAGE - 1 ? 0 : st + 1;
  }
  if (timed_out) {
    if (lane == 0 && a.err) atomicOr(a.err, 1u << 10);
#pragma unroll
    for (int s2 = 0; s2 < NSTAGE; s2++)
      if ((pend >> s2) & 1u) tma::mbar_wait(&S.bar[warp][s2], (phase >> s2) & 1u, lim);
  }
}

struct QuadPackSmem {
  uint32_t hb[kQTile][kBlock];
  uint32_t xs[kQTile][kBlock];
  uint8_t idx[kQTile][16];
  uint4 image[2][kQImage / 16 + 2];
  int len[2][kQTile];
  int off[2][kQTile + 1];
  int64_t tile[2];
  uint64_t prefix;
  uint64_t direct_prefix;
  int64_t next;
};

// Phase D of a tile whose image is complete and whose byte offset G is
// known: this warp's image bytes [r0, r1) go to out[G + r] in aligned
// 16-byte chunks assembled with funnel shifts; partial chunks at the two
// ends are shared with neighbours and written bytewise.
__device__ __forceinline__ void image_copy_out(const uint4* img4, int r0, int r1, uint8_t* out, uint64_t G, int lane) {
  if (r1 <= r0) return;
  const uint8_t* img = (const uint8_t*)img4;
  const uint64_t A0 = (uint64_t)(uintptr_t)out + G;  // address of image byte 0
  const uint64_t c0 = (A0 + (uint64_t)r0) >> 4, c1 = (A0 + (uint64_t)r1 + 15) >> 4;
  const int sh = (int)((16 - (A0 & 15)) & 3) * 8;
  const uint32_t* iw = (const uint32_t*)img4;
  for (uint64_t c = c0 + lane; c < c1; c += 32) {
    const int64_t o = (int64_t)(c * 16 - A0);  // image offset of this chunk
    uint8_t* gp = (uint8_t*)(uintptr_t)(c * 16);
    if (o >= r0 && o + 16 <= r1) {
      const int wq = (int)(o >> 2);
      const uint32_t w0 = iw[wq], w1 = iw[wq + 1], w2 = iw[wq + 2], w3 = iw[wq + 3], w4 = iw[wq + 4];
      __stcs((uint4*)gp, make_uint4(__funnelshift_r(w0, w1, sh), __funnelshift_r(w1, w2, sh),
                                    __funnelshift_r(w2, w3, sh), __funnelshift_r(w3, w4, sh)));
    } else {
      for (int bb = 0; bb < 16; bb++) {
        const int64_t io = o + bb;
        if (io >= r0 && io < r1) gp[bb] = img[io];
      }
    }
  }
}

// Pack, software-pipelined over tiles of kQTile blocks.  Iteration i:
// take tile t_i; warp 0 issues the look-back loads of t_{i-1}; (A) every
// quad plans its block of t_i; warp 0 scans t_i's lengths and publishes
// t_i's aggregate, then finishes t_{i-1}'s look-back (its loads have
// landed during phase A); (D) every warp streams its part of t_{i-1}'s
// image to HBM at the resolved offset; (C) every quad writes t_i's bytes
// into the other image.  Tiles are taken from the work counter just before
// their phase A, so predecessors are always at least as far along.  A tile
// too large for the image is resolved and written straight to HBM in its
// own iteration.
__global__ void __launch_bounds__(kQThreads, 4) pack_quad_kernel(PackArgs a) {
  extern __shared__ uint4 smem4[];
  QuadPackSmem& S = *(QuadPackSmem*)smem4;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int q = lane >> 2, j = lane & 3;
  const unsigned qm = quad::quad_mask(lane);
  const int lb = warp * 8 + q;  // block within the tile

  if (tid == 0) {
    S.tile[1] = -1;  // no pending tile
    S.next = (int64_t)atomicAdd((unsigned long long*)a.counter, 1ull);
  }
  for (int it = 0;; it++) {
    const int cb = it & 1, pb = cb ^ 1;  // buffers of this and the pending tile
    __syncthreads();
    const int64_t tile = S.next < a.n_tiles ? S.next : -1;
    const int64_t ptile = S.tile[pb];
    if (tid == 0) S.tile[cb] = tile;
    LookRound lr;
    if (warp == 0 && ptile >= 0) tile_resolve_issue(a.tile_status, ptile, lane, lr);

    // phase A: decisions and lengths of tile t_i
    const int64_t b = tile * kQTile + lb;
    const bool live = tile >= 0 && b < a.n_blocks;
    uint32_t x[8][4];
    quad::QPlan plan;
    plan.len = 0;
    if (live) {
      uint64_t first;
      int n;
      block_span(a.val_off, a.block_start, a.n_streams, b, &first, &n);
      const uint32_t* vp = (const uint32_t*)a.values + first;
      if (n == kBlock && ((uintptr_t)vp & 15) == 0) {
#pragma unroll
        for (int v = 0; v < 8; v++) {
          const uint4 t = __ldcs((const uint4*)(vp + 16 * v + 4 * j));
          x[v][0] = t.x; x[v][1] = t.y; x[v][2] = t.z; x[v][3] = t.w;
        }
      } else {
#pragma unroll
        for (int v = 0; v < 8; v++)
#pragma unroll
          for (int k = 0; k < 4; k++) x[v][k] = (16 * v + 4 * j + k < n) ? __ldcs(vp + 16 * v + 4 * j + k) : 0u;
      }
      plan = quad::quad_plan_block(x, n, a.flag, kTypeU32, kModePlain, S.hb[lb], S.idx[lb], S.xs[lb], j, qm);
    }
    if (j == 0) S.len[cb][lb] = plan.len;
    __syncthreads();
    if (tile < 0 && ptile < 0) break;

    // warp 0: scan of t_i and its aggregate first (no tile's publication
    // ever waits on a look-back), then the look-back of t_{i-1}, whose
    // loads have landed during phase A
    if (warp == 0) {
      if (tile >= 0) {
        const int l = S.len[cb][lane];
        const int incl = warp_incl_scan(l, lane);
        S.off[cb][lane] = incl - l;
        if (lane == 31) {
          S.off[cb][kQTile] = incl;
          tile_publish(a.tile_status, tile, (uint64_t)incl);
        }
      }
      if (ptile >= 0) {
        const uint64_t pre = tile_resolve_finish(a.tile_status, ptile, (uint64_t)S.off[pb][kQTile], lane, a.err, lr, a.spin_limit);
        if (lane == 0) S.prefix = pre;
      }
    }
    __syncthreads();

    // a tile too large for the image is resolved now and written straight
    // to HBM in phase C
    const int total = tile >= 0 ? S.off[cb][kQTile] : 0;
    const bool direct = total > kQImage;
    if (direct) {
      if (warp == 0) {
        const uint64_t pre = tile_resolve_now(a.tile_status, tile, (uint64_t)total, lane, a.err, a.spin_limit);
        if (lane == 0) S.direct_prefix = pre;
      }
      __syncthreads();
    }

    // phase D of t_{i-1}
    if (ptile >= 0) {
      const uint64_t G = S.prefix;
      const int ptotal = S.off[pb][kQTile];
      const bool fits = G + (uint64_t)ptotal <= a.out_cap;
      const int64_t pbk = ptile * kQTile + lb;
      if (pbk < a.n_blocks && j == 0) {
        const uint64_t g = G + (uint64_t)S.off[pb][lb];
        a.block_off[pbk] = g;
        if (pbk == a.n_blocks - 1) a.block_off[a.n_blocks] = g + (uint64_t)S.len[pb][lb];
      }
      if (fits) image_copy_out(S.image[pb], S.off[pb][warp * 8], S.off[pb][warp * 8 + 8], a.out, G, lane);
      else if (tid == 0 && a.err) atomicOr(a.err, 1u << 9);
    }

    // phase C of t_i: into the image, or straight to HBM
    if (tile >= 0) {
      uint8_t* o = (uint8_t*)S.image[cb] + S.off[cb][lb];
      bool write = live;
      if (direct) {
        const uint64_t G = S.direct_prefix;
        const bool fits = G + (uint64_t)total <= a.out_cap;
        if (live && j == 0) {
          const uint64_t g = G + (uint64_t)S.off[cb][lb];
          a.block_off[b] = g;
          if (b == a.n_blocks - 1) a.block_off[a.n_blocks] = g + (uint64_t)plan.len;
        }
        if (!fits && tid == 0 && a.err) atomicOr(a.err, 1u << 9);
        write = live && fits;
        o = a.out + G + S.off[cb][lb];
      }
      if (write) quad::quad_write_block(plan, x, kModePlain, 0, S.hb[lb], S.idx[lb], o, j, qm);
      if (direct && tid == 0) S.tile[cb] = -1;  // nothing pending
    }
    // the next tile is taken last: its phase A follows at once
    if (tid == 0) S.next = (int64_t)atomicAdd((unsigned long long*)a.counter, 1ull);
  }
}

// ------------------------------------------------------------------------
// Pack, one thread per block: every warp runs on its own over tiles of 32
// consecutive blocks (no CTA barriers).  A warp takes a tile, loads it
// (cp.async into 528-byte slots), plans every block (one per thread),
// scans the lengths and publishes the tile's aggregate at once -- nothing
// between taking a tile and publishing it waits on another warp.  Then
// each thread writes its block into the warp's image; the next tile is
// taken, loaded, planned and published while the look-back loads of the
// current one are in flight; finally the current tile's look-back is
// finished and its image streamed to HBM at the resolved offset.
// The uint64 pack runs the same loop over tiles of 16 uint64 blocks, a lane
// pair per block and a lane per uint32 sub-block (SHAPE 2); the uint32 pack
// picks its image window per launch (SHAPE 0 or 1, utl_lane.cuh).
// ------------------------------------------------------------------------
constexpr int kLWarps = 1;
constexpr int kLThreads = kLWarps * 32;
template <int SHAPE>
struct LaneWarpSmem {
  uint4 in[32 * lane::kSlot / 16];
  uint4 img[lane::Window<SHAPE>::kImageBytes / 16];
};
static_assert(lane::kSlot % 16 == 0, "16-byte slots");

__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Issue the loads of tile `tile` into the slots; returns this lane's block
// value count (0 past the last block).  Whole, contiguous, 16-byte aligned
// tiles go through cp.async; others are loaded and zero-padded per block.
// The 33 aligned chunks per slot of a misaligned contiguous tile (out of
// line: the aligned tiles' loop stays small).
__device__ __noinline__ void lane_issue_shifted(uint8_t* inb, const uint8_t* src, int lane) {
  for (int c = lane; c < 32 * 33; c += 32) {
    const int k = c / 33, q = c - 33 * k;
    cp_async16(inb + k * lane::kSlot + 16 * q, src + 512 * k + 16 * q);
  }
}

__device__ __forceinline__ int lane_load_tile(const PackArgs& a, int64_t tile, uint8_t* inb, int lane, int& shift) {
  const int64_t gb = tile * 32 + lane;
  uint64_t first = 0;
  int n = 0;
  shift = 0;
  const int s0 = __shfl_sync(kFull, lane == 0 ? stream_of(a.block_start, a.n_streams, tile * 32) : 0, 0);
  if (gb < a.n_blocks) span_in(a.val_off, a.block_start, stream_from(a.block_start, a.n_streams, s0, gb), gb, &first, &n);
  const uint32_t* vals = (const uint32_t*)a.values;
  const uint64_t f0 = __shfl_sync(kFull, first, 0);
  const bool whole = __all_sync(kFull, n == kBlock && first == f0 + (uint64_t)kBlock * lane);
  const int mis = (int)(((uintptr_t)(vals + f0) >> 2) & 3);  // words past a 16-byte boundary
  if (whole && mis == 0) {
    const uint8_t* src = (const uint8_t*)(vals + f0) + 16 * lane;
    uint8_t* dst = inb + 16 * lane;
#pragma unroll 8
    for (int k = 0; k < 32; k++) cp_async16(dst + k * lane::kSlot, src + 512 * k);
  } else if (whole && (((uintptr_t)vals) & 15) == 0 && f0 - (uint64_t)mis >= a.val_off[0] &&
             f0 - (uint64_t)mis + 32 * kBlock + 4 <= a.val_off[a.n_streams]) {
    // one contiguous run that starts mis words into a 16-byte chunk: each
    // slot takes the 33 aligned chunks that cover its block (the 33rd fills
    // the bank stagger) and is shifted down by mis words once loaded
    // (lane_realign_slot).  The chunks stay inside the values the stream
    // table describes.
    lane_issue_shifted(inb, (const uint8_t*)(vals + f0 - mis), lane);
    shift = mis;
  } else {
    // block by block: whole 16-byte aligned blocks in 16-byte copies, the
    // others value by value; positions past the block's count are zeroed
    for (int k = 0; k < 32; k++) {
      const uint64_t fk = __shfl_sync(kFull, first, k);
      const int nk = __shfl_sync(kFull, n, k);
      uint8_t* dst = inb + k * lane::kSlot + 16 * lane;
      const uint32_t* src = vals + fk + 4 * lane;
      if (nk == kBlock && (((uintptr_t)(vals + fk)) & 15) == 0) {
        cp_async16(dst, src);
      } else {
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (4 * lane + q < nk) cp_async4(dst + 4 * q, src + q);
          else *(uint32_t*)(dst + 4 * q) = 0u;
        }
      }
    }
  }
  cp_async_commit();
  return n;
}

// Shift a slot loaded mis (1..3) words late down to word 0: chunk c takes
// words mis..mis+3 of chunks c and c+1 (in place, ascending; 33 chunks in).
template <int M>
__device__ __forceinline__ void realign_chunks(uint4* s4) {
  uint4 a = s4[0];
  for (int c = 0; c < 32; c++) {
    const uint4 b = s4[c + 1];
    const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    s4[c] = make_uint4(w[M], w[M + 1], w[M + 2], w[M + 3]);
    a = b;
  }
}
__device__ __noinline__ void lane_realign_slot(uint4* slot, int shift) {
  if (shift == 1) realign_chunks<1>(slot);
  else if (shift == 2) realign_chunks<2>(slot);
  else if (shift == 3) realign_chunks<3>(slot);
}

// A tile of the uint64 lane pack is 16 uint64 blocks; block k's low words
// go to slot 2k and its high words to slot 2k+1 (zero past the block's
// count), so each slot holds one uint32 sub-block candidate.  The raw
// block is first copied (cp.async, all blocks in flight at once) to the
// start of its slot pair, then split in place: the warp holds a block in
// registers between a read and a write separated by a barrier.  Returns
// the value count of this lane's block (lane >> 1; 0 past the last block).
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned sa = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(sa), "l"(gmem) : "memory");
}
__device__ __forceinline__ int lane_load_tile64(const PackArgs& a, int64_t tile, uint8_t* inb, int lane) {
  const int64_t gb = tile * 16 + (lane & 15);
  uint64_t first = 0;
  int n = 0;
  const int s0 = __shfl_sync(kFull, lane == 0 ? stream_of(a.block_start, a.n_streams, tile * 16) : 0, 0);
  if (lane < 16 && gb < a.n_blocks)
    span_in(a.val_off, a.block_start, stream_from(a.block_start, a.n_streams, s0, gb), gb, &first, &n);
  const uint64_t* vals = (const uint64_t*)a.values;
  constexpr int kPair = 2 * lane::kSlot;  // a block's slot pair; its raw 1 KB fits at the start
  for (int k = 0; k < 16; k++) {
    const uint64_t fk = __shfl_sync(kFull, first, k);
    const int nk = __shfl_sync(kFull, n, k);
    uint8_t* dst = inb + k * kPair;
    const uint64_t* src = vals + fk;
    if (nk == kBlock && ((uintptr_t)src & 15) == 0) {
      cp_async16(dst + 16 * lane, src + 2 * lane);
      cp_async16(dst + 16 * (lane + 32), src + 2 * (lane + 32));
    } else {
#pragma unroll
      for (int r = 0; r < 4; r++) {
        const int i = lane + 32 * r;
        if (i < nk) cp_async8(dst + 8 * i, src + i);
        else *(uint2*)(dst + 8 * i) = make_uint2(0u, 0u);
      }
    }
  }
  cp_async_commit();
  cp_async_wait0();
  __syncwarp();
  // split: lane l's values 4l..4l+3 are raw bytes 32l..32l+31 of the pair
  for (int k0 = 0; k0 < 16; k0 += 4) {
    uint4 A[4], B[4];
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint8_t* b = inb + (k0 + q) * kPair + 32 * lane;
      A[q] = *(const uint4*)b;
      B[q] = *(const uint4*)(b + 16);
    }
    __syncwarp();
#pragma unroll
    for (int q = 0; q < 4; q++) {
      uint8_t* b = inb + (k0 + q) * kPair;
      *(uint4*)(b + 16 * lane) = make_uint4(A[q].x, A[q].z, B[q].x, B[q].z);
      *(uint4*)(b + lane::kSlot + 16 * lane) = make_uint4(A[q].y, A[q].w, B[q].y, B[q].w);
    }
  }
  return __shfl_sync(kFull, n, lane >> 1);
}

// The shape of uint64 block lane >> 1 (packUint64Scalar, uint64.go:302-333),
// worked out by the lane pair from the two slots, and this lane's sub-block:
// FOR64 when !NoFOR && min > 0 && max - min < 2^32 (the low words become
// x - min in place, packed with FOR off inside), else one block of the low
// words when every value fits in 32 bits, else the low words (combine
// bit, block2Len field) followed by the high words.  The pair splits the
// 128 values; lane h reads its chunks rotated by h so the pair's 16-byte
// reads fall in distinct banks.
struct Shape64 {
  int n;           // this lane's sub-block value count (0: none)
  int mode;
  uint32_t type_flags;
  int flag;
  uint64_t base64;
  bool two;        // the block is written as two sub-blocks
};
__device__ __forceinline__ Shape64 lane_shape64(uint8_t* inb, int nk, int flag, int lane) {
  const int t = lane >> 1, h = lane & 1;
  uint32_t* lo = (uint32_t*)(inb + (2 * t) * lane::kSlot);
  const uint32_t* hi = (const uint32_t*)(inb + (2 * t + 1) * lane::kSlot);
  uint64_t mn = ~0ull, mx = 0ull;
  uint32_t acc = 0;
  for (int c = 0; c < 16; c++) {
    const int i0 = 64 * h + 4 * ((c + h) & 15);
    const uint4 L = *(const uint4*)(lo + i0), H = *(const uint4*)(hi + i0);
    const uint32_t l4[4] = {L.x, L.y, L.z, L.w}, h4[4] = {H.x, H.y, H.z, H.w};
#pragma unroll
    for (int q = 0; q < 4; q++) {
      const uint64_t x = ((uint64_t)h4[q] << 32) | l4[q];
      if (i0 + q < nk) {
        mn = min(mn, x);
        mx = max(mx, x);
      }
      acc |= h4[q];  // zero past the count
    }
  }
  mn = min(mn, (uint64_t)__shfl_xor_sync(kFull, (unsigned long long)mn, 1));
  mx = max(mx, (uint64_t)__shfl_xor_sync(kFull, (unsigned long long)mx, 1));
  acc |= __shfl_xor_sync(kFull, acc, 1);
  Shape64 sh;
  const bool for64 = nk > 0 && !(flag & kNoFOR) && mn > 0 && (mx - mn) < (1ull << 32);
  sh.two = nk > 0 && !for64 && acc != 0;
  sh.n = (h == 0 || sh.two) ? nk : 0;
  sh.mode = h ? kModePlain : (for64 ? kModeFor64 : (sh.two ? kModeCombine : kModePlain));
  sh.type_flags = kTypeU64 | ((h == 0 && sh.two) ? kHdrCombine : 0u);
  sh.flag = flag | (for64 ? kNoFOR : 0);
  sh.base64 = for64 ? mn : 0;
  if (for64) {
    // the low 32 bits of x - min are the low word minus the low word of min
    const uint32_t m32 = (uint32_t)mn;
    for (int c = 0; c < 16; c++) {
      const int i0 = 64 * h + 4 * ((c + h) & 15);
#pragma unroll
      for (int q = 0; q < 4; q++)
        if (i0 + q < nk) lo[i0 + q] -= m32;
    }
  }
  __syncwarp();
  return sh;
}

// Tile offsets of the lane pack.  Every tile publishes its aggregate (its
// byte length) twice: in its own word agg[t] (length + 1; 0 = not yet) and
// added into the word of its group of 32 tiles (sum << 6 | count; the
// group is complete at count 32).  Nothing is overwritten later.  A warp
// knows the inclusive prefix of the last tile it packed, so the exclusive
// prefix of its current tile t is that plus the aggregates of the tiles in
// between: whole groups by their group words, the ragged ends by the tile
// words.  All these loads go out at once, one round trip.  Tiles are taken
// in order and every taken tile is published right after its plan, so
// every wait ends; waits are still bounded (UTL_ERR_TIMEOUT).
struct LaneScan {
  uint32_t* agg;  // n_tiles words
  uint32_t* grp;  // ceil(n_tiles / 32) words
  uint32_t lim;   // spin limit of each wait
};
__device__ __forceinline__ uint32_t ld_relaxed_u32(const uint32_t* p) {
  uint32_t v;
  asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
  return v;
}
__device__ __forceinline__ void lane_publish(const LaneScan& sc, int64_t t, uint32_t total) {
  asm volatile("st.relaxed.gpu.global.u32 [%0], %1;" ::"l"(sc.agg + t), "r"(total + 1u) : "memory");
  atomicAdd(&sc.grp[t >> 5], (total << 6) | 1u);
}

// The loads of a window sum over tiles lo < j < t, issued early.
struct LaneWin {
  int64_t a, b;      // tiles a..b (a > b: empty)
  int64_t ga, gb;    // whole groups ga..gb (ga > gb: none)
  uint32_t head, tail, g0, g1;
};
__device__ __forceinline__ void lane_win_issue(const LaneScan& sc, int64_t lo, int64_t t, int lane, LaneWin& w) {
  w.a = lo + 1;
  w.b = t - 1;
  w.ga = (w.a + 31) >> 5;
  w.gb = ((w.b + 1) >> 5) - 1;
  if (w.ga > w.gb) {  // no whole group: every tile on its own (at most 62)
    w.ga = 1;
    w.gb = 0;
  }
  const bool groups = w.ga <= w.gb;
  const int64_t head_end = groups ? 32 * w.ga - 1 : w.b;     // last head tile
  const int64_t tail_beg = groups ? 32 * (w.gb + 1) : w.b + 1;
  const int64_t h = w.a + lane, h2 = w.a + 32 + lane, tl = tail_beg + lane;
  // head tiles a..head_end (up to 62 without groups: two per lane)
  w.head = (w.a <= w.b && h <= head_end) ? ld_relaxed_u32(sc.agg + h) : 1u;
  w.tail = (!groups && h2 <= head_end) ? ld_relaxed_u32(sc.agg + h2)
                                       : ((groups && tl <= w.b) ? ld_relaxed_u32(sc.agg + tl) : 1u);
  w.g0 = (groups && w.ga + lane <= w.gb) ? ld_relaxed_u32(sc.grp + w.ga + lane) : 32u;
  w.g1 = (groups && w.ga + 32 + lane <= w.gb) ? ld_relaxed_u32(sc.grp + w.ga + 32 + lane) : 32u;
}
__device__ __forceinline__ uint32_t lane_wait_tile(const LaneScan& sc, int64_t j, uint32_t v, bool& to) {
  for (uint32_t it = 0; v == 0; it++) {
    if (it > sc.lim) {
      to = true;
      return 1u;
    }
    __nanosleep(64);
    v = ld_relaxed_u32(sc.agg + j);
  }
  return v;
}
__device__ __forceinline__ uint32_t lane_wait_group(const LaneScan& sc, int64_t g, uint32_t v, bool& to) {
  for (uint32_t it = 0; (v & 63u) != 32u; it++) {
    if (it > sc.lim) {
      to = true;
      return 32u;
    }
    __nanosleep(64);
    v = ld_relaxed_u32(sc.grp + g);
  }
  return v;
}
// Sum of the window issued by lane_win_issue (whole warp).
__device__ __forceinline__ uint64_t lane_win_finish(const LaneScan& sc, LaneWin& w, int lane, uint32_t* err) {
  if (w.a > w.b) return 0;
  bool to = false;
  const bool groups = w.ga <= w.gb;
  const int64_t head_end = groups ? 32 * w.ga - 1 : w.b;
  const int64_t tail_beg = groups ? 32 * (w.gb + 1) : w.b + 1;
  const int64_t h = w.a + lane, h2 = w.a + 32 + lane, tl = tail_beg + lane;
  uint64_t sum = 0;
  if (h <= head_end) sum += lane_wait_tile(sc, h, w.head, to) - 1u;
  if (!groups && h2 <= head_end) sum += lane_wait_tile(sc, h2, w.tail, to) - 1u;
  if (groups && tl <= w.b) sum += lane_wait_tile(sc, tl, w.tail, to) - 1u;
  if (groups) {
    if (w.ga + lane <= w.gb) sum += lane_wait_group(sc, w.ga + lane, w.g0, to) >> 6;
    if (w.ga + 32 + lane <= w.gb) sum += lane_wait_group(sc, w.ga + 32 + lane, w.g1, to) >> 6;
    for (int64_t g = w.ga + 64 + lane; g <= w.gb; g += 32)  // very wide windows
      sum += lane_wait_group(sc, g, ld_relaxed_u32(sc.grp + g), to) >> 6;
  }
  if (__any_sync(kFull, to) && lane == 0 && err) atomicOr(err, 1u << 10);
  return warp_sum_u64(sum);
}

// Take a tile, load it, plan its blocks and publish its aggregate.  U64:
// lane pair 2k, 2k+1 holds uint64 block k as one or two sub-blocks.
template <bool DELTA, bool U64>
__device__ __forceinline__ void lane_take_and_plan(const PackArgs& a, const LaneScan& sc, uint8_t* inb, uint4* slot,
                                                   int lane, int64_t& t, int& n, lane::Plan& p, int& incl,
                                                   int& total) {
  unsigned long long tv = 0;
  if (lane == 0) tv = atomicAdd((unsigned long long*)a.counter, 1ull);
  t = (int64_t)__shfl_sync(kFull, tv, 0);
  if (t >= a.n_tiles) return;
  p.len = 0;
  p.exc = 0;
  if (U64) {
    const int nk = lane_load_tile64(a, t, inb, lane);
    __syncwarp();
    const Shape64 sh = lane_shape64(inb, nk, a.flag, lane);
    n = sh.n;
    if (n > 0) {
      p = lane::plan_block<DELTA>(slot, n, sh.flag, sh.type_flags, sh.mode);
      p.base64 = sh.base64;
    }
    // block2Len of a combined pair: the upper-halves block's length
    const int l_hi = __shfl_xor_sync(kFull, p.len, 1);
    if (n > 0 && p.mode == kModeCombine) p.blk2 = l_hi;
  } else {
    int shift;
    n = lane_load_tile(a, t, inb, lane, shift);
    cp_async_wait0();
    __syncwarp();
    if (shift) lane_realign_slot(slot, shift);  // warp-uniform; each lane its own slot
    if (n > 0) p = lane::plan_block<DELTA>(slot, n, a.flag);
  }
  incl = warp_incl_scan(p.len, lane);
  total = __shfl_sync(kFull, incl, 31);
  if (lane == 31) lane_publish(sc, t, (uint32_t)total);
}

// out[G + r] = img[r] for r in [0, len).  The destination's aligned 16-byte
// chunks start at image offset s + 16i (s = the misalignment, the same for
// the whole tile); each is assembled from the two aligned image chunks i
// and i+1 with a funnel shift (a loop per word shift Q).  The bytes before
// the first and after the last whole chunk (fewer than 16 each) are shared
// with the neighbouring tiles and go out one byte per lane.  The image has
// 32 readable bytes past len.
template <int Q>
__device__ __forceinline__ void lane_copy_chunks(const uint4* img4, uint4* dst, int nf, int b, int lane) {
  // unrolled: several chunks' shared loads in flight before their stores
  // (measured c3 pack 0.535 -> 0.506 ms)
#pragma unroll 4
  for (int i = lane; i < nf; i += 32) {
    const uint4 I0 = img4[i], I1 = img4[i + 1];
    const uint32_t v[8] = {I0.x, I0.y, I0.z, I0.w, I1.x, I1.y, I1.z, I1.w};
    __stcs(dst + i, make_uint4(__funnelshift_r(v[Q], v[Q + 1], b), __funnelshift_r(v[Q + 1], v[Q + 2], b),
                               __funnelshift_r(v[Q + 2], v[Q + 3], b), __funnelshift_r(v[Q + 3], v[Q + 4], b)));
  }
}
__device__ __forceinline__ void lane_copy_out(const uint4* img4, int len, uint8_t* out, uint64_t G, int lane) {
  if (len <= 0) return;
  const uint8_t* img = (const uint8_t*)img4;
  uint8_t* o = out + G;
  const int s = (int)((0u - (uint32_t)(uintptr_t)o) & 15u);
  const int nf = len >= s ? (len - s) >> 4 : 0;
  uint4* dst = (uint4*)(o + s);
  const int b = (s & 3) * 8;
  switch (s >> 2) {
    case 0: lane_copy_chunks<0>(img4, dst, nf, b, lane); break;
    case 1: lane_copy_chunks<1>(img4, dst, nf, b, lane); break;
    case 2: lane_copy_chunks<2>(img4, dst, nf, b, lane); break;
    default: lane_copy_chunks<3>(img4, dst, nf, b, lane); break;
  }
  const int t0 = s + 16 * nf;  // first byte after the whole chunks
  if (lane < 16) {
    if (lane < s && lane < len) o[lane] = img[lane];
    if (t0 + lane < len) o[t0 + lane] = img[t0 + lane];
  }
}

// block_off of the tile's blocks, once the tile's byte offset G is known
// (a uint64 block's offset is its first sub-block's; its end, the pair's).
template <bool U64>
__device__ __forceinline__ void lane_block_offsets(const PackArgs& a, int64_t tile, int lane, int n, int off,
                                                   int incl, uint64_t G) {
  if (U64) {
    const int pair_end = __shfl_xor_sync(kFull, incl, 1);
    const int64_t gb = tile * 16 + (lane >> 1);
    if (!(lane & 1) && n > 0) {
      a.block_off[gb] = G + (uint64_t)off;
      if (gb == a.n_blocks - 1) a.block_off[a.n_blocks] = G + (uint64_t)pair_end;
    }
  } else {
    const int64_t gb = tile * 32 + lane;
    if (n > 0) {
      a.block_off[gb] = G + (uint64_t)off;
      if (gb == a.n_blocks - 1) {
        a.block_off[a.n_blocks] = G + (uint64_t)incl;
        if (a.stats) {  // the batch's packed bytes and blocks, for the next launch's shape
          a.stats[0] = G + (uint64_t)incl;
          a.stats[1] = (uint64_t)a.n_blocks;
        }
      }
    }
  }
}

template <bool DELTA>
__device__ __forceinline__ void lane_write(const lane::Plan& p, const uint4* slot, uint8_t* o) {
  if (__any_sync(__activemask(), p.exc > 0)) lane::write_block<DELTA, true>(p, slot, o);
  else lane::write_block<DELTA, false>(p, slot, o);
}
// One copy of the writer, with the runtime-width payload packer (the
// uint64 kernel, whose instruction cache missed: measured c4 pack 1.16 ->
// 1.06 ms with a single writer call site and -> 0.98 with one payload
// packer for all widths; the uint32 kernels measured faster with the two
// specialised writers and the per-width packers, c3 0.533 against 0.597).
template <bool DELTA>
__device__ __forceinline__ void lane_write1(const lane::Plan& p, const uint4* slot, uint8_t* o) {
  lane::write_block<DELTA, true, true>(p, slot, o);
}

template <bool DELTA, int SHAPE>
__global__ void __launch_bounds__(kLThreads, 8) pack_lane_kernel(PackArgs a) {
  constexpr bool U64 = SHAPE == 2;
  extern __shared__ uint4 smem4[];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  LaneWarpSmem<SHAPE>& W = ((LaneWarpSmem<SHAPE>*)smem4)[warp];
  uint8_t* inb = (uint8_t*)W.in;
  uint8_t* img = (uint8_t*)W.img;
  uint4* slot = (uint4*)(inb + lane * lane::kSlot);
  LaneScan sc;
  sc.agg = (uint32_t*)a.tile_status;
  sc.grp = sc.agg + a.n_tiles;
  sc.lim = a.spin_limit;
  int64_t prev = -1;       // the last tile this warp finished
  uint64_t prev_incl = 0;  // its inclusive prefix
  // the current tile (planned and published; -1: none yet) and its layout
  int64_t cur = -1;
  int n = 0, incl = 0, total = 0, n_rounds = 0;
  lane::Plan p;
  p.len = 0;
  LaneWin win;
  for (;;) {
    const int off = incl - p.len;
    if (cur >= 0) {
      lane_win_issue(sc, prev, cur, lane, win);
      if constexpr (U64) {
        // one call site of the writer: a tile that fits the image is one
        // round whose copy-out waits for the next tile's planning; a larger
        // tile resolves its offset first, then one window of blocks at a
        // time is written and streamed out
        const bool multi = n_rounds > 1;
        uint64_t G = 0;
        bool fits = false;
        int my_round = n > 0 ? 0 : -1;
        if (multi) {
          G = prev_incl + lane_win_finish(sc, win, lane, a.err);
          fits = G + (uint64_t)total <= a.out_cap;
          if (!fits && lane == 0 && a.err) atomicOr(a.err, 1u << 9);
          my_round = n > 0 ? off / lane::Window<SHAPE>::kBytes : -1;
        }
        for (int r = 0; r < (multi ? n_rounds : 1); r++) {
          int base = 0, end = 0;
          if (multi) {
            const unsigned in_r = __ballot_sync(kFull, my_round == r);
            const unsigned in_next = __ballot_sync(kFull, my_round == r + 1);
            base = __shfl_sync(kFull, off, __ffs(in_r) - 1);
            end = in_next ? __shfl_sync(kFull, off, __ffs(in_next) - 1) : total;
          }
          if (my_round == r) lane_write1<DELTA>(p, slot, img + (off - base));
          if (multi) {
            __syncwarp();
            if (fits) lane_copy_out(W.img, end - base, a.out, G + (uint64_t)base, lane);
            __syncwarp();
          }
        }
        if (multi) {
          lane_block_offsets<U64>(a, cur, lane, n, off, incl, G);
          prev = cur;
          prev_incl = G + (uint64_t)total;
        }
      } else if (n_rounds <= 1) {
        if (n > 0) lane_write<DELTA>(p, slot, img + off);
      } else {
        // a tile larger than the image: its offset first, then one window
        // of blocks at a time is written and streamed out
        const uint64_t G = prev_incl + lane_win_finish(sc, win, lane, a.err);
        const bool fits = G + (uint64_t)total <= a.out_cap;
        if (!fits && lane == 0 && a.err) atomicOr(a.err, 1u << 9);
        const int my_round = n > 0 ? off / lane::Window<SHAPE>::kBytes : -1;
        for (int r = 0; r < n_rounds; r++) {
          const unsigned in_r = __ballot_sync(kFull, my_round == r);
          const unsigned in_next = __ballot_sync(kFull, my_round == r + 1);
          const int base = __shfl_sync(kFull, off, __ffs(in_r) - 1);
          const int end = in_next ? __shfl_sync(kFull, off, __ffs(in_next) - 1) : total;
          if (my_round == r) lane_write<DELTA>(p, slot, img + (off - base));
          __syncwarp();
          if (fits) lane_copy_out(W.img, end - base, a.out, G + (uint64_t)base, lane);
          __syncwarp();
        }
        lane_block_offsets<U64>(a, cur, lane, n, off, incl, G);
        prev = cur;
        prev_incl = G + (uint64_t)total;
      }
      __syncwarp();
    }
    // the slots are free: the next tile is taken, loaded, planned and
    // published while the current tile's window loads are in flight
    const int64_t done = cur;
    const int d_n = n, d_off = off, d_incl = incl, d_total = total, d_rounds = n_rounds;
    lane_take_and_plan<DELTA, U64>(a, sc, inb, slot, lane, cur, n, p, incl, total);
    if (done >= 0 && d_rounds <= 1) {
      const uint64_t G = prev_incl + lane_win_finish(sc, win, lane, a.err);
      if (G + (uint64_t)d_total <= a.out_cap) lane_copy_out(W.img, d_total, a.out, G, lane);
      else if (lane == 0 && a.err) atomicOr(a.err, 1u << 9);
      lane_block_offsets<U64>(a, done, lane, d_n, d_off, d_incl, G);
      prev = done;
      prev_incl = G + (uint64_t)d_total;
      __syncwarp();
    }
    if (cur >= a.n_tiles) break;
    // the last lane with a block (a prefix of the lanes, or every even lane
    // and some odd ones for uint64) and the start offsets pick the rounds
    const unsigned act = __ballot_sync(kFull, n > 0);
    const int last = act ? 31 - __clz(act) : 0;
    n_rounds = act ? __shfl_sync(kFull, incl - p.len, last) / lane::Window<SHAPE>::kBytes + 1 : 0;
  }
}

// ------------------------------------------------------------------------
// Pack, a lane pair per block (utl_pair.cuh): the lane pack's loop over
// tiles of 16 blocks.  Each warp works alone: take a tile, load it (16-byte
// cp.async into 544-byte slots), plan every block (a pair per block), scan
// the lengths and publish the tile's aggregate at once; write the blocks
// into the warp's image while the window loads of the tile's offset are in
// flight; take, load, plan and publish the next tile; then stream the image
// out at the resolved offset.
// ------------------------------------------------------------------------
template <int SHAPE>
struct PairWarpSmem {
  uint4 in[16 * pair::kSlot / 16];
  uint4 img[pair::Window<SHAPE>::kImageBytes / 16];
};
static_assert(pair::kSlot % 16 == 0, "16-byte slots");

// Issue the loads of tile `tile` (16 blocks) into the slots; returns this
// lane's block value count (0 past the last block); shift as for the lane
// pack (whole tiles one contiguous run 1..3 words past a 16-byte boundary).
__device__ __noinline__ void pair_issue_shifted(uint8_t* inb, const uint8_t* src, int lane) {
  for (int c = lane; c < 16 * 33; c += 32) {
    const int k = c / 33, q = c - 33 * k;
    cp_async16(inb + k * pair::kSlot + 16 * q, src + 512 * k + 16 * q);
  }
}
__device__ __forceinline__ int pair_load_tile(const PackArgs& a, int64_t tile, uint8_t* inb, int lane, int& shift) {
  const int kb = lane >> 1;
  const int64_t gb = tile * 16 + kb;
  uint64_t first = 0;
  int n = 0;
  shift = 0;
  const int s0 = __shfl_sync(kFull, lane == 0 ? stream_of(a.block_start, a.n_streams, tile * 16) : 0, 0);
  if (gb < a.n_blocks) span_in(a.val_off, a.block_start, stream_from(a.block_start, a.n_streams, s0, gb), gb, &first, &n);
  const uint32_t* vals = (const uint32_t*)a.values;
  const uint64_t f0 = __shfl_sync(kFull, first, 0);
  const bool whole = __all_sync(kFull, n == kBlock && first == f0 + (uint64_t)kBlock * kb);
  const int mis = (int)(((uintptr_t)(vals + f0) >> 2) & 3);
  if (whole && mis == 0) {
    const uint8_t* src = (const uint8_t*)(vals + f0) + 16 * lane;
    uint8_t* dst = inb + 16 * lane;
    // block k's 32 chunks, chunk l from lane l
#pragma unroll 8
    for (int k = 0; k < 16; k++) cp_async16(dst + k * pair::kSlot, src + 512 * k);
  } else if (whole && (((uintptr_t)vals) & 15) == 0 && f0 - (uint64_t)mis >= a.val_off[0] &&
             f0 - (uint64_t)mis + 16 * kBlock + 4 <= a.val_off[a.n_streams]) {
    pair_issue_shifted(inb, (const uint8_t*)(vals + f0 - mis), lane);
    shift = mis;
  } else {
    for (int k = 0; k < 16; k++) {
      const uint64_t fk = __shfl_sync(kFull, first, 2 * k);
      const int nk = __shfl_sync(kFull, n, 2 * k);
      const uint32_t* blk = vals + fk;
      // 32 chunks of the block: lane l takes chunk l
      uint8_t* d = inb + k * pair::kSlot + 16 * lane;
      const uint32_t* sp = blk + 4 * lane;
      if (nk == kBlock && (((uintptr_t)blk) & 15) == 0) {
        cp_async16(d, sp);
      } else {
#pragma unroll
        for (int q = 0; q < 4; q++) {
          if (4 * lane + q < nk) cp_async4(d + 4 * q, sp + q);
          else *(uint32_t*)(d + 4 * q) = 0u;
        }
      }
    }
  }
  cp_async_commit();
  return n;
}

template <bool DELTA>
__device__ __forceinline__ void pair_take_and_plan(const PackArgs& a, const LaneScan& sc, uint8_t* inb, uint4* slot,
                                                   int lane, unsigned pm, int64_t& t, int& n, lane::Plan& p,
                                                   int& incl, int& total) {
  unsigned long long tv = 0;
  if (lane == 0) tv = atomicAdd((unsigned long long*)a.counter, 1ull);
  t = (int64_t)__shfl_sync(kFull, tv, 0);
  if (t >= a.n_tiles) return;
  p.len = 0;
  p.exc = 0;
  int shift;
  n = pair_load_tile(a, t, inb, lane, shift);
  cp_async_wait0();
  __syncwarp();
  const int h = lane & 1;
  if (shift) pair::realign_slot(slot, shift, h, pm);  // warp-uniform
  if (n > 0) p = pair::plan_block<DELTA>(slot, n, a.flag, h, pm);
  incl = warp_incl_scan(h == 0 ? p.len : 0, lane);
  total = __shfl_sync(kFull, incl, 31);
  if (lane == 31) lane_publish(sc, t, (uint32_t)total);
}

template <bool DELTA>
__device__ __forceinline__ void pair_write(const lane::Plan& p, const uint4* slot, uint8_t* o, int h, unsigned pm) {
  if (__any_sync(__activemask(), p.exc > 0)) pair::write_block<DELTA, true>(p, slot, o, h, pm);
  else pair::write_block<DELTA, false>(p, slot, o, h, pm);
}

__device__ __forceinline__ void pair_block_offsets(const PackArgs& a, int64_t tile, int lane, int n, int off,
                                                   int incl, uint64_t G) {
  const int64_t gb = tile * 16 + (lane >> 1);
  if (!(lane & 1) && n > 0) {
    a.block_off[gb] = G + (uint64_t)off;
    if (gb == a.n_blocks - 1) {
      a.block_off[a.n_blocks] = G + (uint64_t)incl;
      if (a.stats) {  // the batch's packed bytes and blocks, for the next launch's shape
        a.stats[0] = G + (uint64_t)incl;
        a.stats[1] = (uint64_t)a.n_blocks;
      }
    }
  }
}

template <bool DELTA, int SHAPE>
__global__ void __launch_bounds__(32, SHAPE == 1 ? 18 : 16) pack_pair_kernel(PackArgs a) {
  extern __shared__ uint4 smem4[];
  constexpr int kW = pair::Window<SHAPE>::kBytes;
  const int lane = threadIdx.x & 31;
  const int h = lane & 1;
  const unsigned pm = pair::pair_mask(lane);
  PairWarpSmem<SHAPE>& W = *(PairWarpSmem<SHAPE>*)smem4;
  uint8_t* inb = (uint8_t*)W.in;
  uint8_t* img = (uint8_t*)W.img;
  uint4* slot = (uint4*)(inb + (lane >> 1) * pair::kSlot);
  LaneScan sc;
  sc.agg = (uint32_t*)a.tile_status;
  sc.grp = sc.agg + a.n_tiles;
  sc.lim = a.spin_limit;
  int64_t prev = -1;       // the last tile this warp finished
  uint64_t prev_incl = 0;  // its inclusive prefix
  int64_t cur = -1;        // the current tile (planned and published)
  int n = 0, incl = 0, total = 0, n_rounds = 0;
  lane::Plan p;
  p.len = 0;
  LaneWin win;
  for (;;) {
    const int off = incl - p.len;
    if (cur >= 0) {
      lane_win_issue(sc, prev, cur, lane, win);
      if (n_rounds <= 1) {
        if (n > 0) pair_write<DELTA>(p, slot, img + off, h, pm);
      } else {
        // a tile larger than the image: its offset first, then one window
        // of blocks at a time is written and streamed out
        const uint64_t G = prev_incl + lane_win_finish(sc, win, lane, a.err);
        const bool fits = G + (uint64_t)total <= a.out_cap;
        if (!fits && lane == 0 && a.err) atomicOr(a.err, 1u << 9);
        const int my_round = n > 0 ? off / kW : -1;
        for (int r = 0; r < n_rounds; r++) {
          const unsigned in_r = __ballot_sync(kFull, my_round == r);
          const unsigned in_next = __ballot_sync(kFull, my_round == r + 1);
          const int base = __shfl_sync(kFull, off, __ffs(in_r) - 1);
          const int end = in_next ? __shfl_sync(kFull, off, __ffs(in_next) - 1) : total;
          if (my_round == r) pair_write<DELTA>(p, slot, img + (off - base), h, pm);
          __syncwarp();
          if (fits) lane_copy_out(W.img, end - base, a.out, G + (uint64_t)base, lane);
          __syncwarp();
        }
        pair_block_offsets(a, cur, lane, n, off, incl, G);
        prev = cur;
        prev_incl = G + (uint64_t)total;
      }
      __syncwarp();
    }
    const int64_t done = cur;
    const int d_n = n, d_off = off, d_incl = incl, d_total = total, d_rounds = n_rounds;
    pair_take_and_plan<DELTA>(a, sc, inb, slot, lane, pm, cur, n, p, incl, total);
    if (done >= 0 && d_rounds <= 1) {
      const uint64_t G = prev_incl + lane_win_finish(sc, win, lane, a.err);
      if (G + (uint64_t)d_total <= a.out_cap) lane_copy_out(W.img, d_total, a.out, G, lane);
      else if (lane == 0 && a.err) atomicOr(a.err, 1u << 9);
      pair_block_offsets(a, done, lane, d_n, d_off, d_incl, G);
      prev = done;
      prev_incl = G + (uint64_t)d_total;
      __syncwarp();
    }
    if (cur >= a.n_tiles) break;
    const unsigned act = __ballot_sync(kFull, n > 0);
    const int last = act ? 31 - __clz(act) : 0;
    n_rounds = act ? __shfl_sync(kFull, incl - p.len, last) / kW + 1 : 0;
  }
}

// ------------------------------------------------------------------------
// Get: one thread per query; queries that need the reference's full-block
// fallback (delta blocks, deep positions) are resolved by the whole warp.
// ------------------------------------------------------------------------
struct SubGet {
  const uint8_t* p;  // sub-block start
  int64_t rd;        // readable bytes
  int64_t len;       // the reference's len(src)
  int pos;
};

// Resolve every lane whose r.need_full is set with a warp-wide unpack of
// its block (getUint32FullUnpack / getFullUnpackViaBlock, get.go:198-218,
// 339-349), bounded by the block end the thread validated.
template <bool U64>
__device__ __forceinline__ void resolve_full(bool active, const SubGet& q, GetResult& r, uint32_t* hb, int lane) {
  unsigned m = __ballot_sync(kFull, active && r.need_full);
  while (m) {
    const int src = __ffs(m) - 1;
    m &= m - 1;
    const uint8_t* p = (const uint8_t*)__shfl_sync(kFull, (unsigned long long)q.p, src);
    const int64_t rd = (int64_t)__shfl_sync(kFull, (unsigned long long)q.rd, src);
    const int64_t len = (int64_t)__shfl_sync(kFull, (unsigned long long)r.end, src);
    const int pos = __shfl_sync(kFull, q.pos, src);
    uint32_t v[4];
    const GlobalBytes g{p, rd};
    const UnpackResult u = warp_unpack_block(g, 0, len, U64, v, hb, lane);
    const int slot = pos >> 5;
    uint32_t mine = slot == 0 ? v[0] : slot == 1 ? v[1] : slot == 2 ? v[2] : v[3];
    const uint32_t val = __shfl_sync(kFull, mine, pos & 31);
    if (lane == src) {
      r.need_full = false;
      r.status = u.status;
      r.ovf = u.ovf;
      r.value = val;
    }
  }
}

template <bool U64>
__global__ void __launch_bounds__(kThreads) get_kernel(GetArgs a) {
  __shared__ uint32_t hb_all[kWarps * kBlock];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  uint32_t* hb = hb_all + warp * kBlock;
  const int64_t q = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = q < a.n_queries;

  int status = kOK, ovf = 0;
  uint64_t result = 0;
  SubGet sg{nullptr, 0, 0, 0};
  bool live = false;
  if (act) {
    const uint32_t s = a.q_stream[q];
    const uint64_t p = a.q_pos[q];
    if (s >= (uint32_t)a.n_streams || p >= a.val_off[s + 1] - a.val_off[s]) {
      status = kErrPositionOutOfRange;
    } else {
      const int64_t b = (int64_t)a.block_start[s] + (int64_t)(p / kBlock);
      const uint64_t off = a.block_off[b], end = a.block_off[b + 1];
      const uint64_t e2 = min(end, a.packed_len);
      const int64_t rd = (e2 > off) ? (int64_t)(e2 - off) : 0;
      sg = SubGet{a.packed + off, rd, (end >= off) ? (int64_t)(end - off) : 0, (int)(p % kBlock)};
      live = true;
    }
  }

  if (!U64) {
    GetResult r{kOK, 0, 0u, false};
    if (live) r = thread_get_u32(GlobalBytes{sg.p, sg.rd}, sg.len, sg.pos, false);
    resolve_full<false>(live, sg, r, hb, lane);
    if (live) {
      status = r.status;
      ovf = r.ovf;
      result = r.value;
    }
  } else {
    // getUint64Scalar, uint64.go:372-436
    const GlobalBytes g{sg.p, sg.rd};
    uint32_t h = 0;
    bool go = live;
    if (go) {
      if (sg.len < 4) { status = kErrInvalidBuffer; go = false; }
      else {
        h = g.u32(0);
        if (((h >> 13) & 3) != 3) { status = kErrUnsupportedType; go = false; }
      }
    }
    GetResult r{kOK, 0, 0u, false};
    if (go) r = thread_get_u32(g, sg.len, sg.pos, true);
    resolve_full<true>(go, sg, r, hb, lane);
    if (go && r.status != kOK) { status = r.status; ovf = r.ovf; go = false; }
    const uint32_t lower = r.value;
    const int forw = (int)((h >> 15) & 3), exc = (int)(h >> 24);
    SubGet sg2{nullptr, 0, 0, sg.pos};
    bool second = false;
    if (go) {
      if (!(h & kHdrCombine)) {
        uint64_t base = 0;
        if (forw == 3) {
          const int off = 4 + (exc > 0 ? 2 : 0);
          if (sg.len < off + 8) { status = kErrInvalidBuffer; go = false; }
          else base = g.u64(off);
        }
        if (go) result = (uint64_t)lower + base;
      } else {
        const int64_t meta = 4 + (exc > 0 ? 2 : 0) + ((1 << forw) >> 1) + 2;
        if (sg.len < meta) { status = kErrInvalidBuffer; go = false; }
        else {
          const int64_t b2len = g.u16(meta - 2);
          int64_t b1 = meta + (int64_t)(((h >> 8) & 31) * 4) * 16;
          if (exc > 0) b1 += min(exc, 16) + (int64_t)g.u16(4);
          if (b1 + b2len > sg.len) { status = kErrInvalidBuffer; go = false; }
          else {
            const int64_t rd2 = max((int64_t)0, min(b2len, sg.rd - b1));
            sg2 = SubGet{sg.p + b1, rd2, b2len, sg.pos};
            second = true;
          }
        }
      }
    }
    GetResult r2{kOK, 0, 0u, false};
    if (second) r2 = thread_get_u32(GlobalBytes{sg2.p, sg2.rd}, sg2.len, sg2.pos, true);
    resolve_full<true>(second, sg2, r2, hb, lane);
    if (second) {
      if (r2.status != kOK) { status = r2.status; ovf = r2.ovf; }
      else result = ((uint64_t)r2.value << 32) | lower;
    }
  }

  if (act) {
    if (U64) ((uint64_t*)a.out)[q] = status == kOK ? result : 0ull;
    else ((uint32_t*)a.out)[q] = status == kOK ? (uint32_t)result : 0u;
    if (a.status) a.status[q] = status | (ovf << 8);
    if (status != kOK && a.err) atomicOr(a.err, 1u << status);
  }
}

// ------------------------------------------------------------------------
// per-call kernels (one warp): inputs and outputs live in mapped pinned
// host memory, so a call is one launch and one synchronize.
// ------------------------------------------------------------------------
template <bool U64>
__global__ void __launch_bounds__(32) plain_pack_kernel(int flag, const void* vals, int n, uint8_t* out,
                                                        PlainResult* res) {
  __shared__ uint4 slot4[(Shape<U64>::kSlot + 16) / 16];
  __shared__ uint32_t hb[kBlock];
  const int lane = threadIdx.x;
  uint8_t* slot = (uint8_t*)slot4;
  int len;
  if (U64) {
    const uint64_t* vp = (const uint64_t*)vals;
    uint64_t x[4];
#pragma unroll
    for (int k = 0; k < 4; k++) x[k] = (lane + 32 * k < n) ? vp[lane + 32 * k] : 0ull;
    len = warp_pack_block64(x, n, flag, slot, 0, hb, lane);
  } else {
    const uint32_t* vp = (const uint32_t*)vals;
    uint32_t v[4];
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = (lane + 32 * k < n) ? vp[lane + 32 * k] : 0u;
    len = warp_pack_block(v, n, flag, kTypeU32, kModePlain, 0, slot, 0, hb, lane);
  }
  __syncwarp();
  warp_copy_out((const uint32_t*)slot, len, out, 0, lane);
  if (lane == 0) {
    res->status = kOK;
    res->len = len;
  }
}

// Copy staged bytes from mapped host memory into device scratch, then
// decode from device memory.
__device__ __forceinline__ void warp_stage_dev(const uint8_t* src, int64_t n, uint8_t* tmp, int lane) {
  for (int64_t i = lane; i < n; i += 32) tmp[i] = src[i];
  __syncwarp();
  __threadfence_block();
}

template <bool U64>
__global__ void __launch_bounds__(32) plain_unpack_kernel(const uint8_t* src, int64_t staged, int64_t avail,
                                                          uint8_t* tmp, void* vals, PlainResult* res) {
  __shared__ uint32_t hb[kBlock];
  const int lane = threadIdx.x;
  warp_stage_dev(src, staged, tmp, lane);
  const GlobalBytes g{tmp, staged};
  UnpackResult r;
  if (U64) {
    uint64_t x[4];
    r = warp_unpack_block64(g, 0, avail, x, hb, lane);
    if (r.status == kOK) {
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (lane + 32 * k < r.count) ((uint64_t*)vals)[lane + 32 * k] = x[k];
    }
  } else {
    uint32_t v[4];
    r = warp_unpack_block(g, 0, avail, false, v, hb, lane);
    if (r.status == kOK) {
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (lane + 32 * k < r.count) ((uint32_t*)vals)[lane + 32 * k] = v[k];
    }
  }
  if (lane == 0) {
    res->status = r.status;
    res->count = r.count;
    res->len = r.consumed;
    res->ovf = r.ovf;
  }
}

template <bool U64>
__global__ void __launch_bounds__(32) plain_get_kernel(int pos, const uint8_t* src, int64_t staged, int64_t avail,
                                                       uint8_t* tmp, PlainResult* res) {
  __shared__ uint32_t hb[kBlock];
  const int lane = threadIdx.x;
  warp_stage_dev(src, staged, tmp, lane);
  const GlobalBytes g{tmp, staged};
  const bool me = lane == 0;
  int status = kOK, ovf = 0;
  uint64_t result = 0;
  if (!U64) {
    SubGet sg{tmp, staged, avail, pos};
    GetResult r{kOK, 0, 0u, false};
    if (me) r = thread_get_u32(g, avail, pos, false);
    resolve_full<false>(me, sg, r, hb, lane);
    status = r.status;
    ovf = r.ovf;
    result = r.value;
  } else {
    uint32_t h = 0;
    bool go = true;
    if (avail < 4) { status = kErrInvalidBuffer; go = false; }
    else {
      h = g.u32(0);
      if (((h >> 13) & 3) != 3) { status = kErrUnsupportedType; go = false; }
    }
    SubGet sg{tmp, staged, avail, pos};
    GetResult r{kOK, 0, 0u, false};
    if (go && me) r = thread_get_u32(g, avail, pos, true);
    resolve_full<true>(go && me, sg, r, hb, lane);
    if (go && r.status != kOK) { status = r.status; ovf = r.ovf; go = false; }
    const int forw = (int)((h >> 15) & 3), exc = (int)(h >> 24);
    bool second = false;
    SubGet sg2{nullptr, 0, 0, pos};
    if (go) {
      if (!(h & kHdrCombine)) {
        uint64_t base = 0;
        if (forw == 3) {
          const int off = 4 + (exc > 0 ? 2 : 0);
          if (avail < off + 8) { status = kErrInvalidBuffer; go = false; }
          else base = g.u64(off);
        }
        if (go) result = (uint64_t)r.value + base;
      } else {
        const int64_t meta = 4 + (exc > 0 ? 2 : 0) + ((1 << forw) >> 1) + 2;
        if (avail < meta) { status = kErrInvalidBuffer; go = false; }
        else {
          const int64_t b2len = g.u16(meta - 2);
          int64_t b1 = meta + (int64_t)(((h >> 8) & 31) * 4) * 16;
          if (exc > 0) b1 += min(exc, 16) + (int64_t)g.u16(4);
          if (b1 + b2len > avail) { status = kErrInvalidBuffer; go = false; }
          else {
            sg2 = SubGet{tmp + b1, max((int64_t)0, min(b2len, staged - b1)), b2len, pos};
            second = true;
          }
        }
      }
    }
    GetResult r2{kOK, 0, 0u, false};
    if (second && me) r2 = thread_get_u32(GlobalBytes{sg2.p, sg2.rd}, sg2.len, pos, true);
    resolve_full<true>(second && me, sg2, r2, hb, lane);
    if (second) {
      if (r2.status != kOK) { status = r2.status; ovf = r2.ovf; }
      else result = ((uint64_t)r2.value << 32) | r.value;
    }
  }
  if (me) {
    res->status = status;
    res->ovf = ovf;
    res->value = status == kOK ? result : 0ull;
  }
}

// ------------------------------------------------------------------------
// host launchers
// ------------------------------------------------------------------------
namespace launch {

// Launch configuration of one device: kernel attributes set and resident
// CTAs per SM queried once per device (with that device current), under a
// lock, and published through `ready` only after every field is written.
// Setting attributes and querying occupancy allocates nothing (the CUDA
// runtime may load this library's kernels onto the device the first time).
constexpr int kMaxDevices = 64;
struct DevCfg {
  std::atomic<int> ready{0};
  cudaError_t err = cudaSuccess;
  int sms = 0;
  int lane_ctas[3] = {0, 0, 0};  // pack_lane_kernel, per window shape
  int pair_ctas[2] = {0, 0};     // pack_pair_kernel, per window shape
  int quad_pack_ctas = 0;        // pack_quad_kernel
  int pipe_ctas = 0;             // unpack_quad_pipe_kernel, narrow staging
  int pipe_wide_ctas = 0;        // unpack_quad_pipe_kernel, wide staging
  int tma_ctas = 0;              // unpack_quad_tma_kernel, narrow staging (3 stages)
  int tma_wide_ctas = 0;         // unpack_quad_tma_kernel, wide staging (2 stages)
  int oct64_ctas[2] = {0, 0};    // unpack_oct64_tma_kernel, 2 / 3 stages
  int lane_unpack_ctas[2] = {0, 0};  // unpack_lane_kernel, one / two staging buffers
  int auto_unpack_ctas = 0;          // unpack_auto_kernel
  int pipe64_ctas[3] = {0, 0, 0};  // unpack_quad_pipe_kernel for uint64: narrow, wide, wide single buffer
  int pack_ctas[2] = {0, 0};     // pack_kernel<false/true>
  // Mapped pinned pair the uint32 lane pack's last block fills with the
  // batch's packed bytes and block count; the next allocating launch on
  // this device reads it (without waiting) to pick its window shape.  Only
  // a performance hint: a stale or torn pair picks the other shape, whose
  // output is the same.  Allocated by the first pack that may allocate.
  std::atomic<uint64_t*> stats{nullptr};
  uint64_t* stats_dev = nullptr;
};
static DevCfg g_dev[kMaxDevices];
static std::mutex g_setup_mu;

template <class K>
static cudaError_t set_smem(K kern, size_t bytes) {
  cudaError_t e = cudaFuncSetAttribute((const void*)kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
  if (e != cudaSuccess) return e;
  cudaFuncSetAttribute((const void*)kern, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
  return cudaSuccess;
}
template <class K>
static int occupancy(K kern, int threads, size_t bytes) {
  int n = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, threads, bytes) != cudaSuccess || n <= 0) n = 1;
  return n;
}

static cudaError_t setup_device(int dev, DevCfg& c);

// The current device's configuration, set up on first use.
static cudaError_t dev_cfg(DevCfg** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  DevCfg& c = g_dev[dev];
  if (!c.ready.load(std::memory_order_acquire)) {
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!c.ready.load(std::memory_order_relaxed)) {
      e = setup_device(dev, c);
      if (e != cudaSuccess) return e;
      c.ready.store(1, std::memory_order_release);
    }
  }
  *out = &c;
  return cudaSuccess;
}

// The mapped pinned stats pair of a device (allocating; once per device).
static uint64_t* lane_stats_dev(DevCfg& c) {
  if (c.stats.load(std::memory_order_acquire)) return c.stats_dev;
  std::lock_guard<std::mutex> lk(g_setup_mu);
  if (c.stats.load(std::memory_order_relaxed)) return c.stats_dev;
  uint64_t* h = nullptr;
  if (cudaHostAlloc((void**)&h, 2 * sizeof(uint64_t), cudaHostAllocMapped | cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    return nullptr;
  }
  h[0] = h[1] = 0;
  uint64_t* d = nullptr;
  if (cudaHostGetDevicePointer((void**)&d, h, 0) != cudaSuccess) {
    cudaGetLastError();
    cudaFreeHost(h);
    return nullptr;
  }
  c.stats_dev = d;
  c.stats.store(h, std::memory_order_release);
  return d;
}

static int num_sms() {
  DevCfg* c = nullptr;
  return dev_cfg(&c) == cudaSuccess ? c->sms : 148;
}

size_t pack_smem(bool u64) {
  return (size_t)kTile * (u64 ? Shape<true>::kSlot : Shape<false>::kSlot) + 16 + (size_t)kWarps * kBlock * 4;
}
size_t unpack_smem(bool u64) {
  return (size_t)kTile * (u64 ? Shape<true>::kStage : Shape<false>::kStage) + 64 + (size_t)kWarps * kBlock * 4;
}

int64_t tiles_for(int64_t n_blocks) { return (n_blocks + kTile - 1) / kTile; }

cudaError_t plan(const uint64_t* val_off, int n, uint64_t* bstart, cudaStream_t st) {
  plan_kernel<<<1, 1024, 0, st>>>(val_off, n, bstart);
  note_launch(1);
  return cudaGetLastError();
}

cudaError_t stream_offsets(const uint64_t* block_off, const uint64_t* bstart, int n, uint64_t* sbo, cudaStream_t st) {
  int threads = 256, blocks = (n + 1 + threads - 1) / threads;
  stream_off_kernel<<<blocks, threads, 0, st>>>(block_off, bstart, n, sbo);
  note_launch(1);
  return cudaGetLastError();
}

// UTL_KNOB_UNPACK64_SCHEDULE: 0 = warp per block, 1 / 2 = an octet per
// block with TMA staging, two / three groups in flight per warp, 3-7 = a
// quad per block through the cp.async pipeline (7, the default: double
// buffered small budget or single large buffer by the batch's mean block
// length).
static std::atomic<int> g_unpack64_schedule{7};
// UTL_KNOB_UNPACK_CTAS_PER_SM: cap on resident unpack CTAs (of 4 warps) per
// SM of the persistent unpack kernels (0 = the occupancy maximum).
static std::atomic<int> g_unpack_cap{0};
static int unpack_ctas(int occ) {
  const int cap = g_unpack_cap.load(std::memory_order_relaxed);
  return (cap > 0 && cap < occ) ? cap : occ;
}

template <int STAGE, bool AUTO, bool U64 = false, int NBUF = 2>
static cudaError_t unpack_pipe(const UnpackArgs& a, cudaStream_t st, int ctas) {
  const size_t psmem = sizeof(QuadPipeSmem<STAGE, NBUF>);
  const int64_t groups = (a.n_blocks + 7) / 8;
  int64_t grid = (int64_t)num_sms() * unpack_ctas(ctas);
  const int64_t need = (groups + kQWarps - 1) / kQWarps;
  if (grid > need) grid = need;
  unpack_quad_pipe_kernel<STAGE, AUTO, U64, NBUF><<<(unsigned)grid, kQThreads, psmem, st>>>(a);
  note_launch(1);
  return cudaGetLastError();
}
static cudaError_t unpack_auto(const UnpackArgs& a, cudaStream_t st, int ctas) {
  // persistent over the finer of the two paths' work items (8-block groups)
  const int64_t groups = (a.n_blocks + 7) / 8;
  int64_t grid = (int64_t)num_sms() * unpack_ctas(ctas);
  const int64_t need = (groups + kQWarps - 1) / kQWarps;
  if (grid > need) grid = need;
  unpack_auto_kernel<<<(unsigned)grid, kQThreads, kAutoSmem, st>>>(a);
  note_launch(1);
  return cudaGetLastError();
}
template <bool AUTO, int NBUF, int STAGE, int W>
static cudaError_t unpack_lane(const UnpackArgs& a, cudaStream_t st, int ctas) {
  const int64_t tiles = (a.n_blocks + 31) / 32;
  int64_t grid = (int64_t)num_sms() * unpack_ctas(ctas);
  const int64_t need = (tiles + W - 1) / W;
  if (grid > need) grid = need;
  unpack_lane_kernel<AUTO, NBUF, STAGE, W><<<(unsigned)grid, 32 * W, sizeof(LaneUnpackSmem<NBUF, STAGE, W>), st>>>(a);
  note_launch(1);
  return cudaGetLastError();
}
template <int STAGE, int NSTAGE, bool AUTO, bool FAST = false>
static cudaError_t unpack_tma(const UnpackArgs& a, cudaStream_t st, int ctas) {
  const size_t smem = sizeof(QuadTmaSmem<STAGE, NSTAGE>);
  const int64_t groups = (a.n_blocks + 7) / 8;
  int64_t grid = (int64_t)num_sms() * unpack_ctas(ctas);
  const int64_t need = (groups + kQWarps - 1) / kQWarps;
  if (grid > need) grid = need;
  unpack_quad_tma_kernel<STAGE, NSTAGE, AUTO, FAST><<<(unsigned)grid, kQThreads, smem, st>>>(a);
  note_launch(1);
  return cudaGetLastError();
}
// UTL_KNOB_UNPACK_SCHEDULE (include/utlpfor.h)
static int g_unpack_schedule = 8;
static int g_pack_cap = 0;
static int g_pack_schedule = 1;
// Test knobs: the polls of every bounded wait (0 = the default 2^22), and
// whether the pack leaves the caller's scratch as it finds it.
static std::atomic<uint32_t> g_spin_limit{0};
// UTL_KNOB_PACK_WINDOW: 0 = by the previous allocating uint32 pack on this
// device, 1 = the large image window, 2 = the small one.
static std::atomic<int> g_pack_window{0};
static std::atomic<int> g_keep_scratch{0};
uint32_t spin_limit() {
  const uint32_t v = g_spin_limit.load(std::memory_order_relaxed);
  return v ? v : (1u << 22);
}
bool keep_scratch() { return g_keep_scratch.load(std::memory_order_relaxed) != 0; }

template <bool DELTA, int SHAPE>
static void launch_lane(const PackArgs& a, int64_t grid, cudaStream_t st) {
  pack_lane_kernel<DELTA, SHAPE><<<(unsigned)grid, kLThreads, sizeof(LaneWarpSmem<SHAPE>) * kLWarps, st>>>(a);
}

static cudaError_t setup_device(int dev, DevCfg& c) {
  cudaError_t e = cudaDeviceGetAttribute(&c.sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (c.sms <= 0) c.sms = 148;
  const size_t lsm[3] = {sizeof(LaneWarpSmem<0>) * kLWarps, sizeof(LaneWarpSmem<1>) * kLWarps,
                         sizeof(LaneWarpSmem<2>) * kLWarps};
  if ((e = set_smem(pack_lane_kernel<false, 0>, lsm[0])) != cudaSuccess) return e;
  if ((e = set_smem(pack_lane_kernel<true, 0>, lsm[0])) != cudaSuccess) return e;
  if ((e = set_smem(pack_lane_kernel<false, 1>, lsm[1])) != cudaSuccess) return e;
  if ((e = set_smem(pack_lane_kernel<true, 1>, lsm[1])) != cudaSuccess) return e;
  if ((e = set_smem(pack_lane_kernel<false, 2>, lsm[2])) != cudaSuccess) return e;
  if ((e = set_smem(pack_lane_kernel<true, 2>, lsm[2])) != cudaSuccess) return e;
  c.lane_ctas[0] = occupancy(pack_lane_kernel<false, 0>, kLThreads, lsm[0]);
  c.lane_ctas[1] = occupancy(pack_lane_kernel<false, 1>, kLThreads, lsm[1]);
  c.lane_ctas[2] = occupancy(pack_lane_kernel<false, 2>, kLThreads, lsm[2]);
  const size_t psm[2] = {sizeof(PairWarpSmem<0>), sizeof(PairWarpSmem<1>)};
  if ((e = set_smem(pack_pair_kernel<false, 0>, psm[0])) != cudaSuccess) return e;
  if ((e = set_smem(pack_pair_kernel<true, 0>, psm[0])) != cudaSuccess) return e;
  if ((e = set_smem(pack_pair_kernel<false, 1>, psm[1])) != cudaSuccess) return e;
  if ((e = set_smem(pack_pair_kernel<true, 1>, psm[1])) != cudaSuccess) return e;
  c.pair_ctas[0] = occupancy(pack_pair_kernel<false, 0>, 32, psm[0]);
  c.pair_ctas[1] = occupancy(pack_pair_kernel<false, 1>, 32, psm[1]);
  if ((e = set_smem(pack_quad_kernel, sizeof(QuadPackSmem))) != cudaSuccess) return e;
  c.quad_pack_ctas = occupancy(pack_quad_kernel, kQThreads, sizeof(QuadPackSmem));
  if ((e = set_smem(pack_kernel<false>, pack_smem(false))) != cudaSuccess) return e;
  if ((e = set_smem(pack_kernel<true>, pack_smem(true))) != cudaSuccess) return e;
  c.pack_ctas[0] = occupancy(pack_kernel<false>, kThreads, pack_smem(false));
  c.pack_ctas[1] = occupancy(pack_kernel<true>, kThreads, pack_smem(true));
  if ((e = set_smem(unpack_quad_kernel, sizeof(QuadUnpackSmem))) != cudaSuccess) return e;
  const size_t pn = sizeof(QuadPipeSmem<kPStageNarrow>), pw = sizeof(QuadPipeSmem<kPStageWide>);
  if ((e = set_smem(unpack_quad_pipe_kernel<kPStageNarrow, true>, pn)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_pipe_kernel<kPStageNarrow, false>, pn)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_pipe_kernel<kPStageWide, true>, pw)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_pipe_kernel<kPStageWide, false>, pw)) != cudaSuccess) return e;
  c.pipe_ctas = occupancy(unpack_quad_pipe_kernel<kPStageNarrow, false>, kQThreads, pn);
  c.pipe_wide_ctas = occupancy(unpack_quad_pipe_kernel<kPStageWide, false>, kQThreads, pw);
  const size_t tn = sizeof(QuadTmaSmem<kPStageNarrow, 3>), tw = sizeof(QuadTmaSmem<kPStageWide, 2>);
  if ((e = set_smem(unpack_quad_tma_kernel<kPStageNarrow, 3, true, false>, tn)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_tma_kernel<kPStageNarrow, 3, false, false>, tn)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_tma_kernel<kPStageWide, 2, true, false>, tw)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_tma_kernel<kPStageWide, 2, false, false>, tw)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_tma_kernel<kPStageNarrow, 3, false, true>, tn)) != cudaSuccess) return e;
  c.tma_ctas = occupancy(unpack_quad_tma_kernel<kPStageNarrow, 3, false, false>, kQThreads, tn);
  c.tma_wide_ctas = occupancy(unpack_quad_tma_kernel<kPStageWide, 2, false, false>, kQThreads, tw);
  if ((e = set_smem(unpack_oct64_tma_kernel<2>, sizeof(Oct64Smem<2>))) != cudaSuccess) return e;
  if ((e = set_smem(unpack_oct64_tma_kernel<3>, sizeof(Oct64Smem<3>))) != cudaSuccess) return e;
  c.oct64_ctas[0] = occupancy(unpack_oct64_tma_kernel<2>, kQThreads, sizeof(Oct64Smem<2>));
  c.oct64_ctas[1] = occupancy(unpack_oct64_tma_kernel<3>, kQThreads, sizeof(Oct64Smem<3>));
  const size_t qn = sizeof(QuadPipeSmem<kPStageWide>), qw = sizeof(QuadPipeSmem<kP64StageWide>);
  if ((e = set_smem(unpack_quad_pipe_kernel<kPStageWide, true, true>, qn)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_pipe_kernel<kP64StageWide, true, true>, qw)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_pipe_kernel<kPStageWide, false, true>, qn)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_pipe_kernel<kP64StageWide, false, true>, qw)) != cudaSuccess) return e;
  c.pipe64_ctas[0] = occupancy(unpack_quad_pipe_kernel<kPStageWide, false, true>, kQThreads, qn);
  c.pipe64_ctas[1] = occupancy(unpack_quad_pipe_kernel<kP64StageWide, false, true>, kQThreads, qw);
  const size_t lu1 = sizeof(LaneUnpackSmem<1, kLUStage1, 4>), lu2 = sizeof(LaneUnpackSmem<2, kLUStage2, 2>);
  if ((e = set_smem(unpack_lane_kernel<true, 1, kLUStage1, 4>, lu1)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_lane_kernel<false, 1, kLUStage1, 4>, lu1)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_lane_kernel<true, 2, kLUStage2, 2>, lu2)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_lane_kernel<false, 2, kLUStage2, 2>, lu2)) != cudaSuccess) return e;
  c.lane_unpack_ctas[0] = occupancy(unpack_lane_kernel<false, 1, kLUStage1, 4>, 128, lu1);
  c.lane_unpack_ctas[1] = occupancy(unpack_lane_kernel<false, 2, kLUStage2, 2>, 64, lu2);
  if ((e = set_smem(unpack_auto_kernel, kAutoSmem)) != cudaSuccess) return e;
  c.auto_unpack_ctas = occupancy(unpack_auto_kernel, kQThreads, kAutoSmem);
  const size_t q1 = sizeof(QuadPipeSmem<kP64StageWide, 1>);
  if ((e = set_smem(unpack_quad_pipe_kernel<kP64StageWide, true, true, 1>, q1)) != cudaSuccess) return e;
  if ((e = set_smem(unpack_quad_pipe_kernel<kP64StageWide, false, true, 1>, q1)) != cudaSuccess) return e;
  c.pipe64_ctas[2] = occupancy(unpack_quad_pipe_kernel<kP64StageWide, false, true, 1>, kQThreads, q1);
  if ((e = set_smem(unpack_kernel<false>, unpack_smem(false))) != cudaSuccess) return e;
  if ((e = set_smem(unpack_kernel<true>, unpack_smem(true))) != cudaSuccess) return e;
  return cudaSuccess;
}

// Window shape of a uint32 pack (0 large, 1 small): the knob, or the block
// density of the previous allocating pack on this device, read from the
// mapped pair without waiting (a performance hint only).  Sets a.stats for
// the kernel to record this batch's density (allocating calls only).
static int pick_window(PackArgs& a, bool may_alloc, DevCfg& c, uint64_t small_block) {
  a.stats = may_alloc ? lane_stats_dev(c) : nullptr;
  const int kn = g_pack_window.load(std::memory_order_relaxed);
  if (kn == 1) return 0;
  if (kn == 2) return 1;
  if (!a.stats) return 0;
  const volatile uint64_t* hv = c.stats.load(std::memory_order_acquire);
  const uint64_t bytes = hv[0], blocks = hv[1];
  return (blocks > 0 && bytes <= blocks * small_block) ? 1 : 0;
}

template <bool DELTA, int SHAPE>
static void launch_pair(const PackArgs& a, int64_t grid, cudaStream_t st) {
  pack_pair_kernel<DELTA, SHAPE><<<(unsigned)grid, 32, sizeof(PairWarpSmem<SHAPE>), st>>>(a);
}

static cudaError_t pack_pair(const PackArgs& a_in, cudaStream_t st, bool may_alloc, DevCfg& c) {
  PackArgs a = a_in;
  a.n_tiles = (a.n_blocks + 15) / 16;
  const int shape = pick_window(a, may_alloc, c, (uint64_t)pair::kSmallBlock);
  const int occ = c.pair_ctas[shape];
  const int per_sm = (g_pack_cap > 0 && g_pack_cap < occ) ? g_pack_cap : occ;
  int64_t grid = (int64_t)c.sms * per_sm;
  if (grid > a.n_tiles) grid = a.n_tiles;
  if (grid < 1) grid = 1;
  const bool d = (a.flag & kDelta) != 0;
  if (shape == 1) d ? launch_pair<true, 1>(a, grid, st) : launch_pair<false, 1>(a, grid, st);
  else d ? launch_pair<true, 0>(a, grid, st) : launch_pair<false, 0>(a, grid, st);
  note_launch(1);
  return cudaGetLastError();
}

static cudaError_t pack_lane(const PackArgs& a_in, cudaStream_t st, bool u64, bool may_alloc, DevCfg& c) {
  PackArgs a = a_in;
  a.n_tiles = u64 ? (a.n_blocks + 15) / 16 : (a.n_blocks + 31) / 32;
  int shape = 2;
  a.stats = nullptr;
  if (!u64) shape = pick_window(a, may_alloc, c, (uint64_t)lane::kSmallBlock);
  const int occ = c.lane_ctas[shape];
  const int per_sm = (g_pack_cap > 0 && g_pack_cap < occ) ? g_pack_cap : occ;
  int64_t grid = (int64_t)c.sms * per_sm;
  if (grid * kLWarps > a.n_tiles) grid = (a.n_tiles + kLWarps - 1) / kLWarps;
  if (grid < 1) grid = 1;
  const bool d = (a.flag & kDelta) != 0;
  switch (shape) {
    case 0: d ? launch_lane<true, 0>(a, grid, st) : launch_lane<false, 0>(a, grid, st); break;
    case 1: d ? launch_lane<true, 1>(a, grid, st) : launch_lane<false, 1>(a, grid, st); break;
    default: d ? launch_lane<true, 2>(a, grid, st) : launch_lane<false, 2>(a, grid, st); break;
  }
  note_launch(1);
  return cudaGetLastError();
}

cudaError_t pack(bool u64, const PackArgs& a_in, cudaStream_t st, bool may_alloc) {
  DevCfg* c = nullptr;
  cudaError_t e = dev_cfg(&c);
  if (e != cudaSuccess) return e;
  if (g_pack_schedule == 2 && !u64) return pack_pair(a_in, st, may_alloc, *c);
  if (g_pack_schedule >= 1) return pack_lane(a_in, st, u64, may_alloc, *c);
  if (!u64) {
    PackArgs a = a_in;
    a.n_tiles = (a.n_blocks + kQTile - 1) / kQTile;
    const int per_sm = (g_pack_cap > 0 && g_pack_cap < c->quad_pack_ctas) ? g_pack_cap : c->quad_pack_ctas;
    int64_t grid = (int64_t)c->sms * per_sm;
    if (grid > a.n_tiles) grid = a.n_tiles;
    if (grid < 1) grid = 1;
    pack_quad_kernel<<<(unsigned)grid, kQThreads, sizeof(QuadPackSmem), st>>>(a);
    note_launch(1);
    return cudaGetLastError();
  }
  const PackArgs& a = a_in;
  int64_t grid = (int64_t)c->sms * c->pack_ctas[1];
  if (grid > a.n_tiles) grid = a.n_tiles;
  if (grid < 1) grid = 1;
  pack_kernel<true><<<(unsigned)grid, kThreads, pack_smem(true), st>>>(a);
  note_launch(1);
  return cudaGetLastError();
}

cudaError_t unpack(bool u64, const UnpackArgs& a, cudaStream_t st) {
  if (a.n_blocks <= 0) return cudaSuccess;
  DevCfg* c = nullptr;
  cudaError_t e = dev_cfg(&c);
  if (e != cudaSuccess) return e;
  if (!u64) {
    // thread per block or the wide pipeline by the mean block length, on the device, in one launch
    if (g_unpack_schedule == 8) return unpack_auto(a, st, c->auto_unpack_ctas);
    if (g_unpack_schedule == 9) return unpack_lane<false, 1, kLUStage1, 4>(a, st, c->lane_unpack_ctas[0]);
    if (g_unpack_schedule == 10) return unpack_lane<false, 2, kLUStage2, 2>(a, st, c->lane_unpack_ctas[1]);
    if (g_unpack_schedule == 1) {  // by the batch's mean block length, decided on the device
      e = unpack_pipe<kPStageNarrow, true>(a, st, c->pipe_ctas);
      if (e != cudaSuccess) return e;
      return unpack_pipe<kPStageWide, true>(a, st, c->pipe_wide_ctas);
    }
    if (g_unpack_schedule == 4) {  // TMA staging, by the batch's mean block length on the device
      e = unpack_tma<kPStageNarrow, 3, true>(a, st, c->tma_ctas);
      if (e != cudaSuccess) return e;
      return unpack_tma<kPStageWide, 2, true>(a, st, c->tma_wide_ctas);
    }
    if (g_unpack_schedule == 5) return unpack_tma<kPStageNarrow, 3, false>(a, st, c->tma_ctas);
    if (g_unpack_schedule == 6) return unpack_tma<kPStageWide, 2, false>(a, st, c->tma_wide_ctas);
    if (g_unpack_schedule == 7) return unpack_tma<kPStageNarrow, 3, false, true>(a, st, c->tma_ctas);
    if (g_unpack_schedule == 2) return unpack_pipe<kPStageWide, false>(a, st, c->pipe_wide_ctas);
    if (g_unpack_schedule == 3) return unpack_pipe<kPStageNarrow, false>(a, st, c->pipe_ctas);
    const int64_t grid = (a.n_blocks + kQTile - 1) / kQTile;
    unpack_quad_kernel<<<(unsigned)grid, kQThreads, sizeof(QuadUnpackSmem), st>>>(a);
    note_launch(1);
    return cudaGetLastError();
  }
  const int sched64 = g_unpack64_schedule.load(std::memory_order_relaxed);
  if (sched64 == 3) {  // quad per block, staging by the batch's mean block length on the device
    e = unpack_pipe<kPStageWide, true, true>(a, st, c->pipe64_ctas[0]);
    if (e != cudaSuccess) return e;
    return unpack_pipe<kP64StageWide, true, true>(a, st, c->pipe64_ctas[1]);
  }
  if (sched64 == 4) return unpack_pipe<kPStageWide, false, true>(a, st, c->pipe64_ctas[0]);
  if (sched64 == 5) return unpack_pipe<kP64StageWide, false, true>(a, st, c->pipe64_ctas[1]);
  if (sched64 == 6) return unpack_pipe<kP64StageWide, false, true, 1>(a, st, c->pipe64_ctas[2]);
  if (sched64 == 7) {  // as 3, the large budget with a single buffer
    e = unpack_pipe<kPStageWide, true, true>(a, st, c->pipe64_ctas[0]);
    if (e != cudaSuccess) return e;
    return unpack_pipe<kP64StageWide, true, true, 1>(a, st, c->pipe64_ctas[2]);
  }
  if (sched64 == 1 || sched64 == 2) {
    const int64_t groups = (a.n_blocks + 3) / 4;
    int64_t grid = (int64_t)c->sms * unpack_ctas(c->oct64_ctas[sched64 - 1]);
    const int64_t need = (groups + kQWarps - 1) / kQWarps;
    if (grid > need) grid = need;
    if (sched64 == 1) unpack_oct64_tma_kernel<2><<<(unsigned)grid, kQThreads, sizeof(Oct64Smem<2>), st>>>(a);
    else unpack_oct64_tma_kernel<3><<<(unsigned)grid, kQThreads, sizeof(Oct64Smem<3>), st>>>(a);
    note_launch(1);
    return cudaGetLastError();
  }
  const int64_t grid = tiles_for(a.n_blocks);
  unpack_kernel<true><<<(unsigned)grid, kThreads, unpack_smem(true), st>>>(a);
  note_launch(1);
  return cudaGetLastError();
}

cudaError_t get(bool u64, const GetArgs& a, cudaStream_t st) {
  if (a.n_queries <= 0) return cudaSuccess;
  const int64_t grid = (a.n_queries + kThreads - 1) / kThreads;
  if (u64) get_kernel<true><<<(unsigned)grid, kThreads, 0, st>>>(a);
  else get_kernel<false><<<(unsigned)grid, kThreads, 0, st>>>(a);
  note_launch(1);
  return cudaGetLastError();
}

cudaError_t plain_pack(bool u64, int flag, const void* vals, int n, uint8_t* out, PlainResult* res, cudaStream_t st) {
  if (u64) plain_pack_kernel<true><<<1, 32, 0, st>>>(flag, vals, n, out, res);
  else plain_pack_kernel<false><<<1, 32, 0, st>>>(flag, vals, n, out, res);
  note_launch(1);
  return cudaGetLastError();
}

cudaError_t plain_unpack(bool u64, const uint8_t* src, int64_t staged, int64_t avail, uint8_t* tmp, void* vals,
                         PlainResult* res, cudaStream_t st) {
  if (u64) plain_unpack_kernel<true><<<1, 32, 0, st>>>(src, staged, avail, tmp, vals, res);
  else plain_unpack_kernel<false><<<1, 32, 0, st>>>(src, staged, avail, tmp, vals, res);
  note_launch(1);
  return cudaGetLastError();
}

cudaError_t plain_get(bool u64, int pos, const uint8_t* src, int64_t staged, int64_t avail, uint8_t* tmp,
                      PlainResult* res, cudaStream_t st) {
  if (u64) plain_get_kernel<true><<<1, 32, 0, st>>>(pos, src, staged, avail, tmp, res);
  else plain_get_kernel<false><<<1, 32, 0, st>>>(pos, src, staged, avail, tmp, res);
  note_launch(1);
  return cudaGetLastError();
}

int set_knob(int knob, int value) {
  switch (knob) {
    case 0:  // UTL_KNOB_UNPACK_SCHEDULE
      if (value < 0 || value > 10) return -1;
      g_unpack_schedule = value;
      return 0;
    case 1:  // UTL_KNOB_PACK_CTAS_PER_SM (0 = occupancy maximum)
      if (value < 0 || value > 32) return -1;
      g_pack_cap = value;
      return 0;
    case 2:  // UTL_KNOB_PACK_SCHEDULE
      if (value < 0 || value > 2) return -1;
      g_pack_schedule = value;
      return 0;
    case 7:  // UTL_KNOB_UNPACK_CTAS_PER_SM (0 = occupancy maximum)
      if (value < 0 || value > 32) return -1;
      g_unpack_cap.store(value, std::memory_order_relaxed);
      return 0;
    case 8:  // UTL_KNOB_UNPACK64_SCHEDULE
      if (value < 0 || value > 7) return -1;
      g_unpack64_schedule.store(value, std::memory_order_relaxed);
      return 0;
    case 6:  // UTL_KNOB_PACK_WINDOW
      if (value < 0 || value > 2) return -1;
      g_pack_window.store(value, std::memory_order_relaxed);
      return 0;
    case 4:  // UTL_KNOB_SPIN_LIMIT (0 = default)
      if (value < 0 || value > (1 << 30)) return -1;
      g_spin_limit.store((uint32_t)value, std::memory_order_relaxed);
      return 0;
    case 5:  // UTL_KNOB_KEEP_SCRATCH
      if (value != 0 && value != 1) return -1;
      g_keep_scratch.store(value, std::memory_order_relaxed);
      return 0;
  }
  return -1;
}
int get_knob(int knob) {
  switch (knob) {
    case 0: return g_unpack_schedule;
    case 1: return g_pack_cap;
    case 2: return g_pack_schedule;
    case 4: return (int)g_spin_limit.load(std::memory_order_relaxed);
    case 5: return g_keep_scratch.load(std::memory_order_relaxed);
    case 6: return g_pack_window.load(std::memory_order_relaxed);
    case 7: return g_unpack_cap.load(std::memory_order_relaxed);
    case 8: return g_unpack64_schedule.load(std::memory_order_relaxed);
  }
  return -1;
}

}  // namespace launch
}  // namespace utl
