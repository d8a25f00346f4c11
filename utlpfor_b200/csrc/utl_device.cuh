// utl_device.cuh -- warp-level UTL-PFOR block codec for sm_100a.
//
// One warp owns one 128-value block.  Lane t of the warp holds the values
// at block positions i = t + 32k (k = 0..3); in the UTL layout (value i in
// lane i%16, row i/16) these are the four rows v = 2k + (t>>4) of UTL lane
// t%16, so a lane pair (t, t^16) holds one whole UTL lane and every global
// load/store of values is a coalesced 128-byte warp access.
//
// The byte-level format and every decision follow the Go reference
// github.com/Akron/utlpfor; each routine cites the file:line it matches.
#pragma once
#include <stdint.h>

namespace utl {

constexpr int kBlock = 128;
constexpr int kMaxBlock32 = 1018;  // MaxBlockLength32(0), scalar.go:336
constexpr int kMaxBlock64 = 2038;  // MaxBlockLength64(0), uint64.go:451
constexpr unsigned kFull = 0xFFFFFFFFu;

// Status codes shared with include/utlpfor.h.
enum : int {
  kOK = 0,
  kErrInvalidBuffer = 1,
  kErrPositionOutOfRange = 2,
  kErrInvalidBlockLength = 3,
  kErrInvalidFlags = 4,
  kErrUnsupportedType = 5,
  kErrNotImplemented = 6,
  kErrOverflow = 7,
  kErrCountMismatch = 8,
};

// Flag bits, utlpfor.go:24-68.
enum : int { kDelta = 1, kNoFOR = 2, kNoPatch = 4, kSpecial = 8, kAppend = 16, kNoInPlace = 32 };

// Header layout, header.go:8-87.
constexpr uint32_t kTypeU32 = 2u << 13;
constexpr uint32_t kTypeU64 = 3u << 13;
constexpr uint32_t kHdrCombine = 1u << 19;
constexpr uint32_t kHdrDelta = 1u << 22;
constexpr uint32_t kHdrZigZag = 1u << 23;

// Block shapes of the pack modes (uint64.go:124-189).
enum PackMode : int { kModePlain = 0, kModeCombine = 1, kModeFor64 = 2 };

__device__ __forceinline__ int len32(uint32_t x) { return 32 - __clz(x); }
__device__ __forceinline__ int round_step(int bw) { return (bw + 3) & ~3; }
// Go semantics of uint32 << s: zero for s >= 32.
__device__ __forceinline__ uint32_t shl32(uint32_t v, int s) { return s >= 32 ? 0u : v << s; }
__device__ __forceinline__ uint32_t zz_enc(uint32_t v) { return (v << 1) ^ (uint32_t)((int32_t)v >> 31); }
__device__ __forceinline__ uint32_t zz_dec(uint32_t v) { return (v >> 1) ^ (0u - (v & 1u)); }
__device__ __forceinline__ int svb_len_of(uint32_t x) {
  return x < (1u << 8) ? 1 : x < (1u << 16) ? 2 : x < (1u << 24) ? 3 : 4;
}
__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Warp inclusive prefix sum.
__device__ __forceinline__ int warp_incl_scan(int x, int lane) {
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    int y = __shfl_up_sync(kFull, x, d);
    if (lane >= d) x += y;
  }
  return x;
}

__device__ __forceinline__ uint64_t shfl_xor64(uint64_t v, int m) {
  uint32_t lo = __shfl_xor_sync(kFull, (uint32_t)v, m);
  uint32_t hi = __shfl_xor_sync(kFull, (uint32_t)(v >> 32), m);
  return ((uint64_t)hi << 32) | lo;
}

// ---------------------------------------------------------------------------
// Byte sources.  The unpack routine is written against a byte source so the
// same code decodes blocks staged in shared memory (batched kernels) and
// blocks read straight from global memory (Get).
// ---------------------------------------------------------------------------

// Shared-memory bytes: a word-aligned buffer with at least two readable
// padding words past the last byte any caller asks for.
struct SmemBytes {
  const uint32_t* w;
  __device__ __forceinline__ uint32_t u32(int off) const {
    int q = off >> 2;
    return __funnelshift_r(w[q], w[q + 1], (off & 3) * 8);
  }
  __device__ __forceinline__ uint32_t u8(int off) const { return (w[off >> 2] >> ((off & 3) * 8)) & 0xFFu; }
  __device__ __forceinline__ uint32_t u16(int off) const { return u32(off) & 0xFFFFu; }
  __device__ __forceinline__ uint64_t u64(int off) const { return (uint64_t)u32(off) | ((uint64_t)u32(off + 4) << 32); }
};

// Global-memory bytes with a hard bound: reads at or past `len` return zero,
// so a corrupt header can never steer a load outside the caller's buffer.
struct GlobalBytes {
  const uint8_t* p;
  int64_t len;
  __device__ __forceinline__ uint32_t u8(int64_t off) const {
    return (off >= 0 && off < len) ? (uint32_t)p[off] : 0u;
  }
  __device__ __forceinline__ uint32_t u16(int64_t off) const { return u8(off) | (u8(off + 1) << 8); }
  __device__ __forceinline__ uint32_t u32(int64_t off) const {
    if (off >= 0 && off + 4 <= len) {
      const uint8_t* q = p + off;
      if (((uintptr_t)q & 3) == 0) return *(const uint32_t*)q;
      return (uint32_t)q[0] | ((uint32_t)q[1] << 8) | ((uint32_t)q[2] << 16) | ((uint32_t)q[3] << 24);
    }
    return u8(off) | (u8(off + 1) << 8) | (u8(off + 2) << 16) | (u8(off + 3) << 24);
  }
  __device__ __forceinline__ uint64_t u64(int64_t off) const { return (uint64_t)u32(off) | ((uint64_t)u32(off + 4) << 32); }
};

// ---------------------------------------------------------------------------
// Bit-width selection, select_bitwidth.go:56-121 / chooseBestFromExcCounts.
// exc[si] = number of values above 2^(4*si)-1; ties keep the wider width.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void choose_best_packed(uint64_t c, int* best_w, int* best_exc) {
  // byte si of c is exc[si]; counts do not increase with si, so the
  // non-zero bytes form a prefix and their number is maxStepIdx
  int max_si = 0;
#pragma unroll
  for (int si = 0; si < 8; si++) max_si += ((c >> (8 * si)) & 0xFF) != 0;
  int bw = max_si * 4, be = 0;
  int best = 4 + (max_si << 6);
#pragma unroll
  for (int si = 7; si >= 0; si--) {
    const int e = (int)((c >> (8 * si)) & 0xFF);
    // excCostBytesPerValue (select_bitwidth.go:35) is {1,1,1,2,2,3,3,4,4}:
    // for the step deltas 1..8 that occur, (delta + 1) / 2
    const int bpv = (max_si - si + 1) >> 1;
    const int cost = 4 + (si << 6) + 2 + min(e, 16) + ((e + 3) >> 2) + e * bpv;
    if (si < max_si && cost < best) {
      best = cost;
      bw = si * 4;
      be = e;
    }
  }
  *best_w = bw;
  *best_exc = be;
}

__device__ __forceinline__ void choose_best(const int exc[8], int* best_w, int* best_exc) {
  uint64_t c = 0;
#pragma unroll
  for (int si = 0; si < 8; si++) c |= (uint64_t)(exc[si] & 0xFF) << (8 * si);
  choose_best_packed(c, best_w, best_exc);
}

// Warp-wide exception counts at the eight step thresholds.  Each value adds
// one to the byte lanes si < bin(x) of a 64-bit counter; a warp add of the
// two halves cannot carry between bytes (at most 128 per byte).
__device__ __forceinline__ void warp_exc_counts(const uint32_t w[4], const bool valid[4], int exc[8]) {
  uint64_t c = 0;
#pragma unroll
  for (int k = 0; k < 4; k++) {
    int bin = (len32(w[k]) + 3) >> 2;
    uint64_t add = bin ? (0x0101010101010101ull >> (8 * (8 - bin))) : 0ull;
    c += valid[k] ? add : 0ull;
  }
  uint32_t lo = __reduce_add_sync(kFull, (uint32_t)c);
  uint32_t hi = __reduce_add_sync(kFull, (uint32_t)(c >> 32));
#pragma unroll
  for (int si = 0; si < 4; si++) {
    exc[si] = (lo >> (8 * si)) & 0xFF;
    exc[si + 4] = (hi >> (8 * si)) & 0xFF;
  }
}

// ---------------------------------------------------------------------------
// Pack one uint32 block into shared memory.
//
// Follows packBlockScalar (scalar.go:126-235): FOR decision on the raw
// values (for.go:95-126), FOR subtract, per-lane delta with block-global
// zigzag (delta.go:23-48), width selection on the work values, header,
// UTL payload (scalar.go:7-59), exception index + StreamVByte high bits
// (exceptions.go:138-186).  mode adds the uint64 shapes: kModeCombine
// reserves the block2Len field (filled by the caller), kModeFor64 writes the
// 8-byte FOR64 base and forWidth=3 (uint64.go:124-157).
//
// v[k] is the value at position lane+32k (ignored at positions >= n).
// The block is written at byte offset dst of sm; hb is a 128-word per-warp
// scratch.  Returns the block length (warp-uniform).
// ---------------------------------------------------------------------------
__device__ int warp_pack_block(const uint32_t v[4], int n, int flag, uint32_t type_flags, int mode,
                               uint64_t base64, uint8_t* sm, int dst, uint32_t* hb, int lane) {
  bool valid[4];
  uint32_t w[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    valid[k] = lane + 32 * k < n;
    w[k] = valid[k] ? v[k] : 0u;
  }
  uint32_t hflags = type_flags | ((uint32_t)(flag & kSpecial) << 14);

  // Step 1: FOR on the raw values (for.go:95-126).
  bool use_for = false;
  uint32_t base = 0;
  int fw = 0;
  if (!(flag & kNoFOR)) {
    uint32_t mn = 0xFFFFFFFFu, mx = 0u;
#pragma unroll
    for (int k = 0; k < 4; k++)
      if (valid[k]) {
        mn = min(mn, w[k]);
        mx = max(mx, w[k]);
      }
    mn = __reduce_min_sync(kFull, mn);
    mx = __reduce_max_sync(kFull, mx);
    if (mn != 0) {
      int for_max = round_step(len32(mx - mn));
      int raw_max = round_step(len32(mx));
      if (for_max < raw_max) {
        int exc[8], std_w, dummy;
        warp_exc_counts(w, valid, exc);
        choose_best(exc, &std_w, &dummy);
        if (for_max < std_w) {
          use_for = true;
          base = mn;
          int nb = (len32(mn) + 7) >> 3;  // for.go:11-13
          fw = nb >= 3 ? 3 : nb;
        }
      }
    }
    if (use_for) {
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (valid[k]) w[k] -= base;
      hflags |= (uint32_t)fw << 15;
    }
  }

  const int hh = lane >> 4;
  // Step 2: per-lane delta along the rows, zigzag if any lane borrowed.
  if (flag & kDelta) {
    uint32_t p[4];
#pragma unroll
    for (int k = 0; k < 4; k++) p[k] = __shfl_xor_sync(kFull, w[k], 16);
    bool borrow = false;
    uint32_t nw[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      // row 2k+hh; the previous row lives in the partner lane
      bool has_prev = hh || k > 0;
      uint32_t prev = hh ? p[k] : (k > 0 ? p[k - 1] : 0u);
      if (valid[k] && has_prev) {
        borrow |= w[k] < prev;
        nw[k] = w[k] - prev;
      } else {
        nw[k] = w[k];
      }
    }
    bool zz = __any_sync(kFull, borrow);
#pragma unroll
    for (int k = 0; k < 4; k++) w[k] = (zz && valid[k]) ? zz_enc(nw[k]) : nw[k];
    hflags |= kHdrDelta | (zz ? kHdrZigZag : 0u);
  }

  // Step 3: step width and exception count.
  int bw, exc_n = 0;
  if (flag & kNoPatch) {
    uint32_t o = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) o |= w[k];
    o = __reduce_or_sync(kFull, o);
    bw = round_step(len32(o));
  } else {
    int exc[8];
    warp_exc_counts(w, valid, exc);
    choose_best(exc, &bw, &exc_n);
  }

  // Layout: header [svbLen] [FOR base | FOR64 base] [block2Len] payload [index] [svb].
  const int pb = bw * 16;
  const int forb = use_for ? ((1 << fw) >> 1) : 0;
  const int meta = 4 + (exc_n ? 2 : 0);
  const int p_off = meta + (mode == kModeFor64 ? 8 : forb) + (mode == kModeCombine ? 2 : 0);
  if (mode == kModeFor64) hflags |= 3u << 15;
  if (lane == 0) {
    uint32_t h = (uint32_t)(n & 0xFF) | ((uint32_t)(bw >> 2) << 8) | hflags | ((uint32_t)exc_n << 24);
    uint8_t* o = sm + dst;
    o[0] = (uint8_t)h; o[1] = (uint8_t)(h >> 8); o[2] = (uint8_t)(h >> 16); o[3] = (uint8_t)(h >> 24);
    if (mode == kModeFor64) {
#pragma unroll
      for (int b = 0; b < 8; b++) o[meta + b] = (uint8_t)(base64 >> (8 * b));
    } else {
      for (int b = 0; b < forb; b++) o[meta + b] = (uint8_t)(base >> (8 * b));
    }
    if (mode == kModeCombine) { o[meta + forb] = 0; o[meta + forb + 1] = 0; }
  }

  // Step 4: UTL payload.  Each lane pair rebuilds its UTL lane's eight
  // masked rows; the pair splits the lane's bw/4 words between them.
  if (bw > 0) {
    const uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);
    uint32_t m[4], p[4], rows[8];
#pragma unroll
    for (int k = 0; k < 4; k++) m[k] = w[k] & mask;
#pragma unroll
    for (int k = 0; k < 4; k++) p[k] = __shfl_xor_sync(kFull, m[k], 16);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      rows[2 * k] = hh ? p[k] : m[k];
      rows[2 * k + 1] = hh ? m[k] : p[k];
    }
    const int L = lane & 15;
    const int nwords = bw >> 2;
    for (int wd = hh; wd < nwords; wd += 2) {
      uint32_t word = 0;
#pragma unroll
      for (int r = 0; r < 8; r++) {
        int s = r * bw - 32 * wd;
        if (s > -bw && s < 32) word |= s >= 0 ? (rows[r] << s) : (rows[r] >> (-s));
      }
      uint8_t* o = sm + dst + p_off + wd * 64 + L * 4;
      o[0] = (uint8_t)word; o[1] = (uint8_t)(word >> 8); o[2] = (uint8_t)(word >> 16); o[3] = (uint8_t)(word >> 24);
    }
  }

  if (exc_n == 0) return p_off + pb;

  // Step 5: exceptions (bw < 32 here).  Ranks follow ascending position.
  const uint32_t emask = (1u << bw) - 1u;
  const int idx_off = dst + p_off + pb;
  const int idx_sz = exc_n <= 16 ? exc_n : 16;
  __syncwarp();  // hb may still be read by the previous block's SVB step
  int rank_base = 0;
  unsigned bal[4];
#pragma unroll
  for (int k = 0; k < 4; k++) {
    bool e = valid[k] && w[k] > emask;
    bal[k] = __ballot_sync(kFull, e);
    if (e) {
      int r = rank_base + __popc(bal[k] & lanemask_lt());
      hb[r] = w[k] >> bw;
      if (exc_n <= 16) sm[idx_off + r] = (uint8_t)(lane + 32 * k);
    }
    rank_base += __popc(bal[k]);
  }
  if (exc_n > 16 && lane < 16) {
    // 128-bit LSB-first bitmap: bit i of ballot word i/32 is position i
    const int q = lane >> 2;
    const unsigned word = q == 0 ? bal[0] : q == 1 ? bal[1] : q == 2 ? bal[2] : bal[3];
    sm[idx_off + lane] = (uint8_t)(word >> (8 * (lane & 3)));
  }
  __syncwarp();

  // StreamVByte: lane g encodes ranks 4g..4g+3 (control byte g).
  const int nc = (exc_n + 3) >> 2;
  int gsz = 0;
  uint32_t ctrl = 0;
  int slots = 0;
  if (lane < nc) {
    slots = min(4, exc_n - 4 * lane);
    for (int s = 0; s < slots; s++) {
      int l = svb_len_of(hb[4 * lane + s]);
      ctrl |= (uint32_t)(l - 1) << (2 * s);
      gsz += l;
    }
  }
  int incl = warp_incl_scan(gsz, lane);
  int total = __shfl_sync(kFull, incl, 31);
  const int svb_off = idx_off + idx_sz;
  if (lane < nc) {
    sm[svb_off + lane] = (uint8_t)ctrl;
    int d = svb_off + nc + incl - gsz;
    for (int s = 0; s < slots; s++) {
      uint32_t x = hb[4 * lane + s];
      int l = ((ctrl >> (2 * s)) & 3) + 1;
      for (int b = 0; b < l; b++) sm[d + b] = (uint8_t)(x >> (8 * b));
      d += l;
    }
  }
  const int svb_len = nc + total;
  if (lane == 0) {
    sm[dst + 4] = (uint8_t)svb_len;
    sm[dst + 5] = (uint8_t)(svb_len >> 8);
  }
  return p_off + pb + idx_sz + svb_len;
}

// Pack one uint64 block (packUint64Scalar, uint64.go:302-333): FOR64 when
// !NoFOR && min>0 && max-min<2^32, else one block when every value fits in
// 32 bits, else a lower-halves block (combine) followed by an upper-halves
// block.  Returns the total length.
__device__ int warp_pack_block64(const uint64_t x[4], int n, int flag, uint8_t* sm, int dst, uint32_t* hb, int lane) {
  uint64_t mn = ~0ull, mx = 0ull, acc = 0ull;
#pragma unroll
  for (int k = 0; k < 4; k++)
    if (lane + 32 * k < n) {
      mn = min(mn, x[k]);
      mx = max(mx, x[k]);
      acc |= x[k];
    }
#pragma unroll
  for (int d = 16; d > 0; d >>= 1) {
    mn = min(mn, shfl_xor64(mn, d));
    mx = max(mx, shfl_xor64(mx, d));
    acc |= shfl_xor64(acc, d);
  }
  const int inner = flag & ~kAppend;
  uint32_t lo[4], hi[4];
  if (!(inner & kNoFOR) && mn > 0 && (mx - mn) < (1ull << 32)) {
#pragma unroll
    for (int k = 0; k < 4; k++) lo[k] = (uint32_t)(x[k] - mn);
    return warp_pack_block(lo, n, inner | kNoFOR, kTypeU64, kModeFor64, mn, sm, dst, hb, lane);
  }
#pragma unroll
  for (int k = 0; k < 4; k++) {
    lo[k] = (uint32_t)x[k];
    hi[k] = (uint32_t)(x[k] >> 32);
  }
  if ((acc >> 32) == 0) return warp_pack_block(lo, n, inner, kTypeU64, kModePlain, 0, sm, dst, hb, lane);
  int l1 = warp_pack_block(lo, n, inner, kTypeU64 | kHdrCombine, kModeCombine, 0, sm, dst, hb, lane);
  int l2 = warp_pack_block(hi, n, inner, kTypeU64, kModePlain, 0, sm, dst + l1, hb, lane);
  if (lane == 0) {
    // block1's header was written by this lane; uint64.go:180-182
    uint32_t h = (uint32_t)sm[dst] | ((uint32_t)sm[dst + 1] << 8) | ((uint32_t)sm[dst + 2] << 16) |
                 ((uint32_t)sm[dst + 3] << 24);
    int fw = (h >> 15) & 3;
    int off = dst + 4 + ((h >> 24) ? 2 : 0) + ((1 << fw) >> 1);
    sm[off] = (uint8_t)l2;
    sm[off + 1] = (uint8_t)(l2 >> 8);
  }
  return l1 + l2;
}

// ---------------------------------------------------------------------------
// Unpack one block (unpackUint32Scalar, scalar.go:260-309, with the
// decodeUnpackHeader prologue of unpack_block.go:62-172 and applyExceptions
// of exceptions.go:194-284).  avail is the byte count the caller hands in
// (the reference's len(src)).  On success v[k] holds position lane+32k for
// positions < count.  Result fields are warp-uniform.
// ---------------------------------------------------------------------------
struct UnpackResult {
  int status;
  int count;
  int consumed;
  int ovf;
};

template <class Src>
__device__ UnpackResult warp_unpack_block(const Src& sb, int64_t blk, int64_t avail, bool for_u64, uint32_t v[4],
                                          uint32_t* hb, int lane) {
  UnpackResult r{kOK, 0, 0, 0};
  if (avail < 4) { r.status = kErrInvalidBuffer; return r; }
  const uint32_t h = sb.u32(blk);
  const int count = (int)(h & 0xFF);
  const int bw = (int)((h >> 8) & 31) * 4;
  const int itype = (int)((h >> 13) & 3);
  const int forw = (int)((h >> 15) & 3);
  const int exc = (int)(h >> 24);
  const bool has_exc = exc > 0;
  const bool delta = (h & kHdrDelta) != 0;
  const bool zz = (h & kHdrZigZag) != 0;
  bool combine = (h & kHdrCombine) != 0;
  if (for_u64) {
    if (itype != 3) { r.status = kErrUnsupportedType; return r; }
  } else {
    if (itype != 2 && itype != 1) { r.status = kErrUnsupportedType; return r; }
    combine = false;
  }
  if ((unsigned)(count - 1) >= (unsigned)kBlock || bw > 32) {
    if (count == 0) { r.consumed = 4; return r; }
    r.status = count > kBlock ? kErrInvalidBlockLength : kErrInvalidBuffer;
    return r;
  }
  const bool u64s = for_u64 && itype == 3 && forw == 3 && !combine;
  int p_off = 4 + (has_exc ? 2 : 0);
  const int for_off = p_off;
  if (forw > 0) p_off += u64s ? 8 : ((1 << forw) >> 1);
  if (combine) p_off += 2;
  const int pb = bw * 16;
  int64_t end = p_off + pb + (has_exc ? (exc <= 16 ? exc : 16) : 0);
  if (avail < end) { r.status = kErrInvalidBuffer; return r; }
  int svb_len = 0;
  if (has_exc) {
    svb_len = (int)sb.u16(blk + 4);
    if (end + svb_len > avail) { r.status = kErrInvalidBuffer; return r; }
    end += svb_len;
  }
  uint32_t fbase = 0;
  if (forw > 0 && !u64s) {
    fbase = forw == 1 ? sb.u8(blk + for_off) : forw == 2 ? sb.u16(blk + for_off) : sb.u32(blk + for_off);
  }
  int consumed = p_off + pb;

  // UTL unpack of all 128 slots (scalar.go:65-116).
  const int L = lane & 15, hh = lane >> 4;
  const uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);
#pragma unroll
  for (int k = 0; k < 4; k++) {
    uint32_t x = 0;
    if (bw > 0) {
      int bitpos = (2 * k + hh) * bw;
      int boff = bitpos & 31;
      int64_t o = blk + p_off + (bitpos >> 5) * 64 + L * 4;
      uint32_t lo = sb.u32(o);
      uint32_t hi = (boff + bw > 32) ? sb.u32(o + 64) : 0u;
      x = (uint32_t)((((uint64_t)hi << 32) | lo) >> boff) & mask;
    }
    v[k] = x;
  }

  if (has_exc) {
    if (exc > count) { r.status = kErrInvalidBuffer; return r; }
    const int64_t svb_start = blk + consumed + (exc <= 16 ? exc : 16);
    const int nc = (exc + 3) >> 2;
    if (nc > svb_len) { r.status = kErrInvalidBuffer; return r; }
    // Control-byte validation, exceptions.go:63-80: lane g sizes group g.
    int gsz = 0, slots = 0;
    uint32_t c = 0;
    if (lane < nc) {
      c = sb.u8(svb_start + lane);
      slots = min(4, exc - 4 * lane);
      for (int s = 0; s < slots; s++) gsz += (int)((c >> (2 * s)) & 3) + 1;
    }
    int incl = warp_incl_scan(gsz, lane);
    int total = __shfl_sync(kFull, incl, 31);
    if (nc + total > svb_len) { r.status = kErrInvalidBuffer; return r; }
    __syncwarp();  // hb reuse across blocks
    if (lane < nc) {
      int64_t d = svb_start + nc + incl - gsz;
      for (int s = 0; s < slots; s++) {
        int l = (int)((c >> (2 * s)) & 3) + 1;
        uint32_t x = 0;
        for (int b = 0; b < l; b++) x |= sb.u8(d + b) << (8 * b);
        hb[4 * lane + s] = x;
        d += l;
      }
    }
    __syncwarp();
    const int64_t xo = blk + consumed;
    if (exc <= 16) {
      // Sorted position list; full blocks mask the position to 7 bits.
      for (int j = 0; j < exc; j++) {
        int p = (int)sb.u8(xo + j);
        int tgt = count == kBlock ? (p & 127) : (p < count ? p : -1);
        if (tgt >= 0 && (tgt & 31) == lane) {
          uint32_t add = shl32(hb[j], bw);
          int slot = tgt >> 5;
#pragma unroll
          for (int k = 0; k < 4; k++)
            if (slot == k) v[k] |= add;
        }
      }
    } else {
      uint32_t B[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        B[k] = sb.u32(xo + 4 * k);
        int lo = 32 * k;  // stale bits past count are masked (exceptions.go:251-260)
        if (count <= lo) B[k] = 0;
        else if (count < lo + 32) B[k] &= (1u << (count - lo)) - 1u;
      }
      int pop = __popc(B[0]) + __popc(B[1]) + __popc(B[2]) + __popc(B[3]);
      if (pop <= exc) {
        int pre = 0;
#pragma unroll
        for (int k = 0; k < 4; k++) {
          if ((B[k] >> lane) & 1u) v[k] |= shl32(hb[pre + __popc(B[k] & lanemask_lt())], bw);
          pre += __popc(B[k]);
        }
      }
    }
    consumed = (int)(svb_start - blk) + svb_len;
  }

  if (delta) {
    // Per-lane prefix sum; the pair exchange gives each lane all 8 rows.
    uint32_t d[4], p[4], rows[8];
#pragma unroll
    for (int k = 0; k < 4; k++) d[k] = zz ? zz_dec(v[k]) : v[k];
#pragma unroll
    for (int k = 0; k < 4; k++) p[k] = __shfl_xor_sync(kFull, d[k], 16);
#pragma unroll
    for (int k = 0; k < 4; k++) {
      rows[2 * k] = hh ? p[k] : d[k];
      rows[2 * k + 1] = hh ? d[k] : p[k];
    }
    uint32_t acc = rows[0];
    int first = 0x7FFFFFFF;
#pragma unroll
    for (int r2 = 1; r2 < 8; r2++) {
      int idx = L + 16 * r2;
      if (idx < count) {
        uint32_t nx = acc + rows[r2];
        if (nx < acc && idx < first) first = idx;
        acc = nx;
        rows[r2] = acc;
      }
    }
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] = (lane + 32 * k < count) ? (hh ? rows[2 * k + 1] : rows[2 * k]) : v[k];  // static indices: rows stays in registers
    if (!zz) {
      // ErrOverflow.Position: first wrap in v-major order = lowest index.
      int m = __reduce_min_sync(kFull, (unsigned)first);
      if (m != 0x7FFFFFFF) {
        r.status = kErrOverflow;
        r.ovf = m;
        return r;
      }
    }
  }
  if (forw > 0 && !u64s) {
#pragma unroll
    for (int k = 0; k < 4; k++) v[k] += fbase;
  }
  r.count = count;
  r.consumed = consumed;
  return r;
}

// Unpack one uint64 block (unpackUint64Block, uint64.go:191-266).
template <class Src>
__device__ UnpackResult warp_unpack_block64(const Src& sb, int64_t blk, int64_t avail, uint64_t out[4], uint32_t* hb,
                                            int lane) {
  UnpackResult r{kOK, 0, 0, 0};
  if (avail < 4) { r.status = kErrInvalidBuffer; return r; }
  const uint32_t h = sb.u32(blk);
  if (((h >> 13) & 3) != 3) { r.status = kErrUnsupportedType; return r; }
  const int forw = (int)((h >> 15) & 3);
  const int exc = (int)(h >> 24);
  uint32_t lo[4], hi[4];
  if (!(h & kHdrCombine)) {
    uint64_t base = 0;
    if (forw == 3) {
      int off = 4 + (exc > 0 ? 2 : 0);
      if (avail < off + 8) { r.status = kErrInvalidBuffer; return r; }
      base = sb.u64(blk + off);
    }
    r = warp_unpack_block(sb, blk, avail, true, lo, hb, lane);
    if (r.status != kOK) return r;
#pragma unroll
    for (int k = 0; k < 4; k++) out[k] = (uint64_t)lo[k] + base;
    return r;
  }
  UnpackResult r1 = warp_unpack_block(sb, blk, avail, true, lo, hb, lane);
  if (r1.status != kOK) return r1;
  const int meta = 4 + (exc > 0 ? 2 : 0) + ((1 << forw) >> 1) + 2;
  if (avail < meta) { r.status = kErrInvalidBuffer; return r; }
  const int b2len = (int)sb.u16(blk + meta - 2);
  if (r1.consumed + b2len > avail) { r.status = kErrInvalidBuffer; return r; }
  UnpackResult r2 = warp_unpack_block(sb, blk + r1.consumed, b2len, true, hi, hb, lane);
  if (r2.status != kOK) return r2;
  if (r2.count != r1.count) { r.status = kErrInvalidBuffer; return r; }
#pragma unroll
  for (int k = 0; k < 4; k++) out[k] = ((uint64_t)hi[k] << 32) | lo[k];
  r.count = r1.count;
  r.consumed = r1.consumed + b2len;
  return r;
}

// ---------------------------------------------------------------------------
// Single-value Get, one thread (get.go:81-190 and helpers).
// ---------------------------------------------------------------------------

// get.go:34-67
__device__ __forceinline__ uint32_t extract_packed(const GlobalBytes& g, int64_t payload, int64_t plen, int pos, int bw) {
  int lane = pos & 15, pil = pos >> 4;
  int bitpos = pil * bw, word = bitpos >> 5, boff = bitpos & 31;
  int64_t off = (int64_t)word * 64 + lane * 4;
  uint64_t acc = 0;
  if (off + 4 <= plen) acc = g.u32(payload + off);
  if (bw > 32 - boff) {
    int64_t n2 = off + 64;
    if (n2 + 4 <= plen) acc |= (uint64_t)g.u32(payload + n2) << 32;
  }
  acc >>= boff;
  uint64_t mask = bw >= 32 ? 0xFFFFFFFFull : ((1ull << bw) - 1ull);
  return (uint32_t)(acc & mask);
}

// svb.go:40-100: region [x, x+len) of g.
__device__ uint32_t svb_decode_one(const GlobalBytes& g, int64_t x, int64_t len, int count, int index) {
  if (count <= 0 || index < 0 || index >= count) return 0;
  int64_t off = (count + 3) >> 2;
  int tcb = index >> 2, slot = index & 3;
  for (int cb = 0; cb < tcb; cb++) {
    if (cb >= len) return 0;
    uint32_t c = g.u8(x + cb);
    off += (int64_t)((c & 3) + ((c >> 2) & 3) + ((c >> 4) & 3) + ((c >> 6) & 3) + 4);
  }
  if (tcb >= len) return 0;
  uint32_t c = g.u8(x + tcb);
  for (int s = 0; s < slot; s++) off += (int64_t)((c >> (2 * s)) & 3) + 1;
  int bl = (int)((c >> (2 * slot)) & 3) + 1;
  if (off >= len) return 0;
  int64_t end = min(off + bl, len);
  uint32_t acc = 0;
  for (int64_t i = off; i < end; i++) acc |= g.u8(x + i) << (8 * (int)(i - off));
  return acc;
}

// get.go:363-381
__device__ __forceinline__ int bitmap_rank128(const GlobalBytes& g, int64_t bm, int64_t blen, int byte_idx, int bit_idx) {
  if (blen < 16) return 0;
  uint64_t w0 = g.u64(bm), w1 = g.u64(bm + 8);
  if (byte_idx < 8) return __popcll(w0 & ((1ull << (8 * byte_idx + bit_idx)) - 1ull));
  return __popcll(w0) + __popcll(w1 & ((1ull << (8 * (byte_idx - 8) + bit_idx)) - 1ull));
}

// Whether a block's exceptions apply as the full unpack applies them when
// each is looked up by its own position: a position list strictly
// increasing below the count, or a bitmap (bits past the count dropped)
// with no more bits than exceptions.  x: the exception index, xlen bytes
// from there to the block's end.
__device__ __forceinline__ bool exc_in_order(const GlobalBytes& g, int64_t x, int64_t xlen, int exc, int count) {
  if (exc <= 16) {
    if (xlen < exc) return false;
    int prev = -1;
    for (int i = 0; i < exc; i++) {
      const int p = (int)g.u8(x + i);
      if (p <= prev || p >= count) return false;
      prev = p;
    }
    return true;
  }
  if (xlen < 16) return false;
  int pop = 0;
  for (int k = 0; k < 4; k++) {
    uint32_t m = g.u32(x + 4 * k);
    const int lo = 32 * k;
    if (count <= lo) m = 0;
    else if (count < lo + 32) m &= (1u << (count - lo)) - 1u;
    pop += __popc(m);
  }
  return pop <= exc;
}

// exceptions.go:63-80: the StreamVByte control bytes (at x, len bytes of
// control and data) and the data they size fit.
__device__ __forceinline__ bool svb_controls_fit(const GlobalBytes& g, int64_t x, int64_t len, int exc) {
  const int nc = (exc + 3) >> 2;
  int64_t total = 0;
  for (int c = 0; c < nc; c++) {
    const uint32_t b = g.u8(x + c);
    const int slots = min(4, exc - 4 * c);
    for (int s2 = 0; s2 < slots; s2++) total += (int64_t)((b >> (2 * s2)) & 3) + 1;
  }
  return nc + total <= len;
}

// Result of a thread-level Get on one (sub-)block.  need_full asks the warp
// to resolve the value with a full block unpack (get.go:174-181).
struct GetResult {
  int status;
  int ovf;
  uint32_t value;
  bool need_full;
  int64_t end;  // validated block end, set with need_full
};

// get.go:18-28 at the reference's AVX2/AVX-512 level
__device__ __forceinline__ int delta_full_unpack_threshold(int bw) { return bw >= 20 ? 4 : 8; }

// getUint32Scalar (get.go:81-190).  len is the caller's buffer length (the
// reference's len(src)); g bounds the bytes actually readable.
__device__ GetResult thread_get_u32(const GlobalBytes& g, int64_t len, int pos, bool for_u64) {
  GetResult r{kOK, 0, 0u, false, 0};
  if (len < 4) { r.status = kErrInvalidBuffer; return r; }
  const uint32_t h = g.u32(0);
  const int count = (int)(h & 0xFF), bw = (int)((h >> 8) & 31) * 4, itype = (int)((h >> 13) & 3);
  const int forw = (int)((h >> 15) & 3), exc = (int)(h >> 24);
  const bool has_exc = exc > 0, delta = (h & kHdrDelta) != 0, zz = (h & kHdrZigZag) != 0;
  bool combine = (h & kHdrCombine) != 0;
  if (for_u64) {
    if (itype != 3) { r.status = kErrUnsupportedType; return r; }
  } else {
    if (itype != 2 && itype != 1) { r.status = kErrUnsupportedType; return r; }
    combine = false;
  }
  if (pos < 0 || pos >= count) { r.status = kErrPositionOutOfRange; return r; }
  if (bw > 32) { r.status = kErrInvalidBuffer; return r; }
  const bool u64s = for_u64 && itype == 3 && forw == 3 && !combine;
  int64_t p_off = 4 + (has_exc ? 2 : 0);
  int forb = 0;
  if (forw > 0) {
    if (u64s) p_off += 8;
    else { forb = (1 << forw) >> 1; p_off += forb; }
  }
  if (combine) p_off += 2;
  const int64_t pb = bw * 16;
  int64_t end = p_off + pb;
  if (len < end) { r.status = kErrInvalidBuffer; return r; }
  const int isz = exc <= 16 ? exc : 16;
  if (has_exc) {
    if (exc > count) { r.status = kErrInvalidBuffer; return r; }
    int64_t svb_len = g.u16(4);
    if (svb_len < ((exc + 3) >> 2) || end + isz + svb_len > len) { r.status = kErrInvalidBuffer; return r; }
    end += isz + svb_len;
  }
  GlobalBytes gb{g.p, min(end, g.len)};  // src = src[:blockEnd]
  uint32_t fbase = forb == 1 ? gb.u8(p_off - 1) : forb == 2 ? gb.u16(p_off - 2) : forb == 4 ? gb.u32(p_off - 4) : 0u;
  const int64_t xs = p_off + pb;  // exception region start
  if (!delta) {
    uint32_t val = bw > 0 ? extract_packed(gb, p_off, pb, pos, bw) : 0u;
    if (has_exc) {
      // findExceptionIndex, exceptions.go:293-325
      int64_t xlen = end - xs;
      int ei = -1;
      if (exc <= 16) {
        int nn = (int)min((int64_t)exc, xlen);
        for (int i = 0; i < nn; i++) {
          uint32_t b = gb.u8(xs + i);
          if (b == (uint32_t)(pos & 0xFF)) { ei = i; break; }
          if (b > (uint32_t)(pos & 0xFF)) break;
        }
      } else {
        int64_t bl = min(xlen, (int64_t)16);
        int bi = pos >> 3, bit = pos & 7;
        if (bl > 0 && bi < bl && ((gb.u8(xs + bi) >> bit) & 1u)) ei = bitmap_rank128(gb, xs, bl, bi, bit);
      }
      if (ei >= 0) val |= shl32(svb_decode_one(gb, xs + isz, xlen - isz, exc, ei), bw);
    }
    r.value = val + fbase;
    return r;
  }
  const int pil = pos >> 4;
  if (pil > delta_full_unpack_threshold(bw)) {
    // The reference unpacks the whole block here (get.go:174-181), for speed
    // only.  For a zigzag delta block (no overflow is possible) whose
    // exceptions are in order, the lane walk below gives the value the full
    // unpack gives, and of the full unpack's checks only the StreamVByte
    // control validation (exceptions.go:63-80) is not already done above.
    // Other blocks -- plain delta, whose overflow anywhere in the block the
    // full unpack reports, or exceptions out of order -- go to the warp.
    if (!zz || (has_exc && !exc_in_order(gb, xs, end - xs, exc, count))) {
      r.need_full = true;
      r.end = end;
      return r;
    }
    if (has_exc && !svb_controls_fit(gb, xs + isz, end - xs - isz, exc)) {
      r.status = kErrInvalidBuffer;
      return r;
    }
  }
  // getValueWithDelta, get.go:250-285
  const int lane = pos & 15;
  uint32_t lv[8];
#pragma unroll
  for (int vv = 0; vv < 8; vv++) lv[vv] = 0;
  for (int vv = 0; vv <= pil; vv++) {
    int s = lane + vv * 16;
    if (s >= count) break;
    if (bw > 0) lv[vv] = extract_packed(gb, p_off, pb, s, bw);
  }
  if (has_exc) {
    // applyLaneExceptions, get.go:297-334
    const int64_t xlen = end - xs, svb = xs + isz, svb_len = xlen - isz;
    if (exc <= 16) {
      for (int i = 0; i < exc; i++) {
        int p = (int)gb.u8(xs + i);
        if ((p & 15) != lane) continue;
        int vv = p >> 4;
        if (vv > pil) break;
        uint32_t add = shl32(svb_decode_one(gb, svb, svb_len, exc, i), bw);
#pragma unroll
        for (int q = 0; q < 8; q++)
          if (q == vv) lv[q] |= add;
      }
    } else {
      for (int vv = 0; vv <= pil; vv++) {
        int s = lane + vv * 16;
        if (s >= count) break;
        int bi = s >> 3, bit = s & 7;
        if (!((gb.u8(xs + bi) >> bit) & 1u)) continue;
        int rank = bitmap_rank128(gb, xs, 16, bi, bit);
        uint32_t add = shl32(svb_decode_one(gb, svb, svb_len, exc, rank), bw);
#pragma unroll
        for (int q = 0; q < 8; q++)
          if (q == vv) lv[q] |= add;
      }
    }
  }
  if (zz) lv[0] = zz_dec(lv[0]);
#pragma unroll
  for (int vv = 1; vv < 8; vv++) {
    if (vv <= pil && lane + vv * 16 < count) lv[vv] = lv[vv - 1] + (zz ? zz_dec(lv[vv]) : lv[vv]);
  }
  uint32_t val = 0;
#pragma unroll
  for (int q = 0; q < 8; q++)
    if (q == pil) val = lv[q];
  r.value = val + fbase;
  return r;
}

}  // namespace utl
