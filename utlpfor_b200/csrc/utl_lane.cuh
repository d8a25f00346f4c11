// utl_lane.cuh -- thread-per-block UTL-PFOR pack of uint32 blocks (and of
// the uint32 sub-blocks a uint64 block is written as).
//
// One thread owns one 128-value block end to end.  The block's values sit
// in a 528-byte shared-memory slot (natural order: value i at word i, so
// 16-byte chunk c holds row c/4, lanes 4(c%4)..4(c%4)+3 of the UTL layout);
// slots are 528 bytes apart so 16-byte reads of the same chunk by 32
// threads fall in distinct banks.  The thread reads its slot in passes
// (statistics, work-value histogram when FOR or delta change the values,
// payload), plans the block exactly as PackUint32 does (pack.go:76-97,
// scalar.go:7-59) and writes the block's bytes into its warp's tile image.
// Nothing is shared between threads except the image, where every byte is
// owned by exactly one block; words that straddle two owners are written
// bytewise.
#pragma once
#include "utl_device.cuh"
#include "utl_quad.cuh"

namespace utl {
namespace lane {

constexpr int kSlot = 528;        // one block's 512 value bytes + a 16-byte bank stagger
// Largest block the pack emits: header + 512 payload bytes + a FOR base (a
// uint64 sub-block: the 8-byte FOR64 base, or a FOR base and the 2-byte
// block2Len field), rounded up.
constexpr int kMaxLen = 528;
// A tile's image holds the blocks that start in a window of kWindow bytes
// (a tile whose blocks are larger is written and copied out in rounds),
// plus the last block's overhang and the slack the copy-out reads.  The
// window trades occupancy against rounds, so there are three shapes:
//   0: uint32, 7 KB (9 warps per SM);
//   1: uint32 batches of small blocks, 4752 bytes, the largest window at
//      which 10 warps fit an SM (227 KB of shared memory, 1 KB reserved per
//      CTA); chosen when the previous uint32 pack averaged at most
//      kSmallBlock bytes a block;
//   2: uint64, 10 KB: its tiles run to 32 sub-blocks of up to 528 bytes.
constexpr int kWindow = 7168;
constexpr int kWindowSmall = 4752;
constexpr int kWindow64 = 10240;
constexpr int kSmallBlock = kWindowSmall / 32;
template <int SHAPE>
struct Window {
  static constexpr int kBytes = SHAPE == 2 ? kWindow64 : (SHAPE == 1 ? kWindowSmall : kWindow);
  static constexpr int kImageBytes = (kBytes + kMaxLen + 32 + 15) / 16 * 16;
};

// 4-bit bucket counter of a value: bucket b = clz/4 (zero values drop out).
__device__ __forceinline__ uint32_t nib(uint32_t x) { return quad::shl_clamp(1u, (uint32_t)__clz(x) & ~3u); }

// Nibble counters (at most 15 values each) widened into byte counters:
// E holds buckets 0,2,4,6 and O buckets 1,3,5,7.
__device__ __forceinline__ void widen(uint32_t a, uint32_t& E, uint32_t& O) {
  E += a & 0x0F0F0F0Fu;
  O += (a >> 4) & 0x0F0F0F0Fu;
}

// exc[si] (byte si) = values in buckets < 8 - si, i.e. values wider than
// 4*si bits (the counts chooseBestFromExcCounts works on,
// select_bitwidth.go:46-72).  Every byte stays at or below 128.
__device__ __forceinline__ uint64_t exc_from_hist(uint32_t E, uint32_t O) {
  const uint32_t b03 = __byte_perm(E, O, 0x5140);  // buckets 0,1,2,3
  const uint32_t b47 = __byte_perm(E, O, 0x7362);  // buckets 4,5,6,7
  const uint32_t p03 = b03 * 0x01010101u;
  const uint32_t p47 = b47 * 0x01010101u + (p03 >> 24) * 0x01010101u;
  const uint32_t e_lo = __byte_perm(p47, 0, 0x0123);
  const uint32_t e_hi = __byte_perm(p03, 0, 0x0123);
  return ((uint64_t)e_hi << 32) | e_lo;
}

// StreamVByte data bytes of the exceptions at width bw, from the bucket
// counts: a value of bucket b has its top bit in nibble 8-b, so its high
// part value >> bw takes ceil((32 - 4b - bw) / 8) bytes (svb.go:10-45;
// bw is a multiple of 4, so the count is the same for the whole bucket).
__device__ __forceinline__ int svb_data_bytes(uint32_t E, uint32_t O, int bw) {
  int tot = 0;
#pragma unroll
  for (int b = 0; b < 8; b++) {
    const int c = (int)((((b & 1) ? O : E) >> (8 * (b >> 1))) & 0xFFu);
    const int r = 32 - 4 * b - bw;
    if (r > 0) tot += c * ((r + 7) >> 3);
  }
  return tot;
}

struct Plan {
  uint32_t header;
  uint32_t base;  // FOR base, 0 without FOR
  uint64_t base64;  // FOR64 base (mode kModeFor64)
  int mode;       // kModePlain, or a uint64 sub-block shape (kModeCombine, kModeFor64)
  int blk2;       // kModeCombine: the upper-halves block's length (block2Len)
  int bw;
  int exc;
  int forb;       // FOR base bytes (0/1/2/4; 8 for the FOR64 base)
  int p_off;      // payload offset in the block
  int idx_sz;
  int svb_len;    // StreamVByte bytes (control + data)
  int len;
  bool zz;
};

// Rows 0..7 of lane group g (UTL lanes 4g..4g+3) as work values: FOR
// (for.go:95-126) then per-lane delta and, when the block needs it, zigzag
// (delta.go:23-48).  Padding positions hold values that map to zero.
template <bool DELTA>
__device__ __forceinline__ void group_work(const uint4* s4, int g, uint32_t base, bool zz, uint32_t (&w)[8][4],
                                           bool& borrow) {
  uint4 t[8];
#pragma unroll
  for (int r = 0; r < 8; r++) t[r] = s4[4 * r + g];
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const uint32_t v[4] = {t[r].x, t[r].y, t[r].z, t[r].w};
#pragma unroll
    for (int k = 0; k < 4; k++) {
      if (DELTA && r > 0) {
        const uint32_t pv = k == 0 ? t[r - 1].x : k == 1 ? t[r - 1].y : k == 2 ? t[r - 1].z : t[r - 1].w;
        borrow |= v[k] < pv;
        w[r][k] = v[k] - pv;  // the FOR base cancels
      } else {
        w[r][k] = v[k] - base;
      }
      if (DELTA) w[r][k] = zz ? zz_enc(w[r][k]) : w[r][k];
    }
  }
}

// Bucket histogram of the work values (and the delta borrow flag).  An
// out-of-line routine returns its results by value: they come back in
// registers, where reference parameters would put the caller's variables
// in local memory.
struct Hist {
  uint32_t E, O;
  bool borrow;
};
template <bool DELTA>
__device__ __noinline__ Hist work_hist(const uint4* s4, uint32_t base, bool zz) {
  Hist h{0u, 0u, false};
  for (int g = 0; g < 4; g++) {
    uint32_t w[8][4];
    group_work<DELTA>(s4, g, base, zz, w, h.borrow);
#pragma unroll
    for (int rp = 0; rp < 4; rp++) {
      uint32_t a = 0;
#pragma unroll
      for (int k = 0; k < 4; k++) a += nib(w[2 * rp][k]) + nib(w[2 * rp + 1][k]);
      widen(a, h.E, h.O);
    }
  }
  return h;
}

// Work value at block position pos (exception high bits).
template <bool DELTA>
__device__ __forceinline__ uint32_t work_at(const uint32_t* s, int pos, uint32_t base, bool zz) {
  const uint32_t a = s[pos];
  uint32_t w = (DELTA && pos >= 16) ? a - s[pos - 16] : a - base;
  if (DELTA && zz) w = zz_enc(w);
  return w;
}

// Partial block (n < 128) whose values FOR or delta transform: the padding
// is set so that its work values are zero, as the reference leaves them
// (scalar.go:34-40, delta.go:23-48): base in row 0, the lane's value one
// row up below it.
__device__ __noinline__ void fill_padding(uint32_t* s, int n, uint32_t base) {
  for (int i = n; i < kBlock; i++) s[i] = i >= 16 ? s[i - 16] : base;
}

// Statistics of the raw values: min/max (FOR decision) and bucket counts.
template <bool MM, bool HI>
__device__ __forceinline__ void raw_stats(const uint4* s4, uint32_t& mn, uint32_t& mx, uint32_t& E, uint32_t& O) {
  mn = 0xFFFFFFFFu;
  mx = 0u;
  E = 0u;
  O = 0u;
#pragma unroll 1
  for (int c8 = 0; c8 < 8; c8++) {
    uint4 t[4];
#pragma unroll
    for (int q = 0; q < 4; q++) t[q] = s4[4 * c8 + q];
    if (MM) {
      const uint32_t m01 = __vimin3_u32(__vimin3_u32(t[0].x, t[0].y, t[0].z), t[0].w, t[1].x);
      const uint32_t m23 = __vimin3_u32(__vimin3_u32(t[2].x, t[2].y, t[2].z), t[2].w, t[3].x);
      const uint32_t n01 = __vimin3_u32(t[1].y, t[1].z, t[1].w);
      const uint32_t n23 = __vimin3_u32(t[3].y, t[3].z, t[3].w);
      mn = __vimin3_u32(mn, __vimin3_u32(m01, m23, n01), n23);
      const uint32_t x01 = __vimax3_u32(__vimax3_u32(t[0].x, t[0].y, t[0].z), t[0].w, t[1].x);
      const uint32_t x23 = __vimax3_u32(__vimax3_u32(t[2].x, t[2].y, t[2].z), t[2].w, t[3].x);
      const uint32_t y01 = __vimax3_u32(t[1].y, t[1].z, t[1].w);
      const uint32_t y23 = __vimax3_u32(t[3].y, t[3].z, t[3].w);
      mx = __vimax3_u32(mx, __vimax3_u32(x01, x23, y01), y23);
    }
    if (HI) {
      const uint32_t a0 = nib(t[0].x) + nib(t[0].y) + nib(t[0].z) + nib(t[0].w) + nib(t[1].x) + nib(t[1].y) +
                          nib(t[1].z) + nib(t[1].w);
      const uint32_t a1 = nib(t[2].x) + nib(t[2].y) + nib(t[2].z) + nib(t[2].w) + nib(t[3].x) + nib(t[3].y) +
                          nib(t[3].z) + nib(t[3].w);
      widen(a0, E, O);
      widen(a1, E, O);
    }
  }
}

// The block's decisions and length (PackUint32: for.go:95-126 FOR,
// delta.go:23-48 delta/zigzag, select_bitwidth.go:20-72 width and
// exceptions, exceptions.go:138-186 exception index, svb.go StreamVByte).
// type_flags and mode describe uint64 sub-blocks (uint64.go:124-182): the
// header's integer type and combine bit, and the FOR64 base or block2Len
// field in front of the payload.
template <bool DELTA>
__device__ Plan plan_block(uint4* s4, int n, int flag, uint32_t type_flags = kTypeU32, int mode = kModePlain) {
  uint32_t* s = (uint32_t*)s4;
  const bool need_mm = !(flag & kNoFOR);
  const bool need_raw_hist = !(flag & kNoFOR) || !DELTA;
  uint32_t mn, mx, E, O;
  if (need_mm) raw_stats<true, true>(s4, mn, mx, E, O);
  else if (need_raw_hist) raw_stats<false, true>(s4, mn, mx, E, O);
  else mn = mx = E = O = 0;
  if (need_mm && n < kBlock) {
    mn = 0xFFFFFFFFu;
    for (int i = 0; i < n; i++) mn = min(mn, s[i]);
  }
  uint32_t hflags = type_flags | ((uint32_t)(flag & kSpecial) << 14);
  bool use_for = false;
  uint32_t base = 0;
  int fw = 0;
  if (need_mm && mn != 0) {
    const int for_max = round_step(len32(mx - mn));
    const int raw_max = round_step(len32(mx));
    if (for_max < raw_max) {
      int std_w, dummy;
      choose_best_packed(exc_from_hist(E, O), &std_w, &dummy);
      if (for_max < std_w) {
        use_for = true;
        base = mn;
        const int nb = (len32(mn) + 7) >> 3;
        fw = nb >= 3 ? 3 : nb;
        hflags |= (uint32_t)fw << 15;
      }
    }
  }
  bool zz = false;
  if (DELTA || use_for) {
    if (n < kBlock) fill_padding(s, n, base);
    if (DELTA || mx != mn) {
      Hist hs = work_hist<DELTA>(s4, base, false);
      if (DELTA && hs.borrow) {
        zz = true;
        hs = work_hist<DELTA>(s4, base, true);
      }
      E = hs.E;
      O = hs.O;
    } else {
      E = O = 0;  // a constant block under FOR: every work value is zero
    }
  }
  if (DELTA) hflags |= kHdrDelta | (zz ? kHdrZigZag : 0u);
  const uint64_t ec = exc_from_hist(E, O);
  int bw, exc = 0;
  if (flag & kNoPatch) {
    int max_si = 0;
#pragma unroll
    for (int si = 0; si < 8; si++) max_si += ((ec >> (8 * si)) & 0xFF) != 0;
    bw = 4 * max_si;
  } else {
    choose_best_packed(ec, &bw, &exc);
  }
  Plan p;
  p.bw = bw;
  p.exc = exc;
  p.base = base;
  p.zz = zz;
  p.base64 = 0;
  p.mode = mode;
  p.blk2 = 0;
  p.forb = mode == kModeFor64 ? 8 : (use_for ? ((1 << fw) >> 1) : 0);
  if (mode == kModeFor64) hflags |= 3u << 15;
  p.p_off = 4 + (exc ? 2 : 0) + p.forb + (mode == kModeCombine ? 2 : 0);
  p.header = (uint32_t)(n & 0xFF) | ((uint32_t)(bw >> 2) << 8) | hflags | ((uint32_t)exc << 24);
  p.idx_sz = exc == 0 ? 0 : (exc <= 16 ? exc : 16);
  p.svb_len = exc ? ((exc + 3) >> 2) + svb_data_bytes(E, O, bw) : 0;
  p.len = p.p_off + 16 * bw + p.idx_sz + p.svb_len;
  return p;
}

__device__ __forceinline__ void put_bytes(uint8_t* p, uint32_t v, int nb) {
  p[0] = (uint8_t)v;
  if (nb > 1) p[1] = (uint8_t)(v >> 8);
  if (nb > 2) p[2] = (uint8_t)(v >> 16);
  if (nb > 3) p[3] = (uint8_t)(v >> 24);
}

// 16 payload bytes (lanes 4g..4g+3 of word w) at pw + 16w + 4g words plus
// d4 bytes: whole words inside, single bytes in the two straddling words.
__device__ __forceinline__ void put_seg(uint32_t* pw, int d4, int sh, int w, int g, const uint32_t (&x)[4]) {
  uint32_t* q = pw + 16 * w + 4 * g;
  if (d4 == 0) {
    if (((uintptr_t)q & 15) == 0) {
      *(uint4*)q = make_uint4(x[0], x[1], x[2], x[3]);
    } else {
      q[0] = x[0]; q[1] = x[1]; q[2] = x[2]; q[3] = x[3];
    }
    return;
  }
  uint8_t* b = (uint8_t*)q;
  if (d4 <= 1) b[1] = (uint8_t)x[0];
  if (d4 <= 2) b[2] = (uint8_t)(x[0] >> (8 * (2 - d4)));
  b[3] = (uint8_t)(x[0] >> (8 * (3 - d4)));
  q[1] = __funnelshift_r(x[0], x[1], sh);
  q[2] = __funnelshift_r(x[1], x[2], sh);
  q[3] = __funnelshift_r(x[2], x[3], sh);
  b[16] = (uint8_t)(x[3] >> sh);
  if (d4 >= 2) b[17] = (uint8_t)(x[3] >> (sh + 8));
  if (d4 >= 3) b[18] = (uint8_t)(x[3] >> (sh + 16));
}

// The payload words of lanes 4g..4g+3 at width BW (scalar.go:7-59): lane
// k's eight work values, masked to BW bits, packed LSB first into BW/4
// words; word w of the four lanes is one 16-byte segment.  The bit
// positions are constants, so each value costs a mask and a shift-or.
template <int BW>
__device__ __forceinline__ void pack_group(const uint32_t (&w)[8][4], uint32_t* pw, int d4, int sh, int g) {
  constexpr int NW = BW / 4;
  constexpr uint32_t MASK = BW >= 32 ? 0xFFFFFFFFu : ((1u << (BW & 31)) - 1u);
  uint32_t x[NW][4];
#pragma unroll
  for (int i = 0; i < NW; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) x[i][k] = 0;
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const int pos = r * BW, wi = pos >> 5, s = pos & 31;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t m = w[r][k] & MASK;
      x[wi][k] |= m << s;
      if (s + BW > 32) x[wi + 1][k] |= m >> (32 - s);
    }
  }
#pragma unroll
  for (int i = 0; i < NW; i++) put_seg(pw, d4, sh, i, g, x[i]);
}

// Widths 8 and 16 take whole bytes of each value: a word is the low bytes
// of four (two) consecutive rows, gathered with byte permutes.
template <>
__device__ __forceinline__ void pack_group<8>(const uint32_t (&w)[8][4], uint32_t* pw, int d4, int sh, int g) {
  uint32_t x[2][4];
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) {
      const uint32_t lo = __byte_perm(w[4 * i][k], w[4 * i + 1][k], 0x0040);
      const uint32_t hi = __byte_perm(w[4 * i + 2][k], w[4 * i + 3][k], 0x0040);
      x[i][k] = __byte_perm(lo, hi, 0x5410);
    }
  put_seg(pw, d4, sh, 0, g, x[0]);
  put_seg(pw, d4, sh, 1, g, x[1]);
}
template <>
__device__ __forceinline__ void pack_group<16>(const uint32_t (&w)[8][4], uint32_t* pw, int d4, int sh, int g) {
  uint32_t x[4][4];
#pragma unroll
  for (int i = 0; i < 4; i++)
#pragma unroll
    for (int k = 0; k < 4; k++) x[i][k] = __byte_perm(w[2 * i][k], w[2 * i + 1][k], 0x5410);
#pragma unroll
  for (int i = 0; i < 4; i++) put_seg(pw, d4, sh, i, g, x[i]);
}

// The same at any width (multiple of 4, at most 32) with runtime shifts:
// a word of the four lanes is complete when a row reaches its end, and the
// part of that row's value above it starts the next word.  Eight copies of
// the segment store instead of the 36 of the per-width code.
__device__ __forceinline__ void pack_group_any(const uint32_t (&w)[8][4], int bw, uint32_t* pw, int d4, int sh,
                                               int g) {
  if (bw == 0) return;
  const uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);
  uint32_t acc[4] = {0, 0, 0, 0};
  int pos = 0, wi = 0;
#pragma unroll
  for (int r = 0; r < 8; r++) {
    uint32_t m[4];
#pragma unroll
    for (int k = 0; k < 4; k++) {
      m[k] = w[r][k] & mask;
      acc[k] |= m[k] << pos;
    }
    pos += bw;
    if (pos >= 32) {
      put_seg(pw, d4, sh, wi, g, acc);
      wi++;
      pos -= 32;
#pragma unroll
      for (int k = 0; k < 4; k++) acc[k] = pos ? (m[k] >> (bw - pos)) : 0u;
    }
  }
}

// Write the block at o (shared memory): header, StreamVByte length, FOR
// base, the UTL payload (scalar.go:7-59: lane L's eight values packed LSB
// first into bw/4 words, word w of lane L at byte 64w + 4L), then the
// exception index and StreamVByte data (exceptions.go:138-186).
template <bool DELTA, bool EXC, bool ANY_WIDTH = false>
__device__ void write_block(const Plan& p, const uint4* s4, uint8_t* o) {
  put_bytes(o, p.header, 4);
  int m = 4;
  if (p.exc) {
    put_bytes(o + 4, (uint32_t)p.svb_len, 2);
    m = 6;
  }
  if (p.mode == kModeFor64) {
    put_bytes(o + m, (uint32_t)p.base64, 4);
    put_bytes(o + m + 4, (uint32_t)(p.base64 >> 32), 4);
  } else if (p.forb) {
    put_bytes(o + m, p.base, p.forb);
  }
  if (p.mode == kModeCombine) put_bytes(o + m + p.forb, (uint32_t)p.blk2, 2);
  const int bw = p.bw;
  uint8_t* pay = o + p.p_off;
  const uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);  // exceptions are above it
  const int d4 = (int)((uintptr_t)pay & 3);
  uint32_t* pw = (uint32_t*)(pay - d4);
  const int sh = 32 - 8 * d4;
  uint32_t bm[4] = {0, 0, 0, 0};
  // rolled: a smaller loop body keeps the pack's hot code in the
  // instruction cache (measured: c3 pack 0.575 -> 0.539 ms with the rolled
  // statistics loop below)
#pragma unroll 1
  for (int g = 0; g < 4; g++) {
    uint32_t w[8][4];
    bool borrow = false;
    group_work<DELTA>(s4, g, p.base, p.zz, w, borrow);
    if (EXC) {
      uint32_t f[4] = {0, 0, 0, 0};
#pragma unroll
      for (int r = 0; r < 8; r++)
#pragma unroll
        for (int k = 0; k < 4; k++)
          if (w[r][k] > mask) f[r >> 1] |= 1u << ((r & 1) * 16 + k);
#pragma unroll
      for (int q = 0; q < 4; q++) bm[q] |= f[q] << (4 * g);
    }
    if constexpr (ANY_WIDTH) {
      pack_group_any(w, bw, pw, d4, sh, g);
    } else {
      switch (bw) {
        case 4: pack_group<4>(w, pw, d4, sh, g); break;
        case 8: pack_group<8>(w, pw, d4, sh, g); break;
        case 12: pack_group<12>(w, pw, d4, sh, g); break;
        case 16: pack_group<16>(w, pw, d4, sh, g); break;
        case 20: pack_group<20>(w, pw, d4, sh, g); break;
        case 24: pack_group<24>(w, pw, d4, sh, g); break;
        case 28: pack_group<28>(w, pw, d4, sh, g); break;
        case 32: pack_group<32>(w, pw, d4, sh, g); break;
        default: break;  // bw 0: no payload
      }
    }
  }
  if (EXC && p.exc) {
    const uint32_t* s = (const uint32_t*)s4;
    uint8_t* xi = pay + 16 * bw;
    uint8_t* svb = xi + p.idx_sz;
    const int nc = (p.exc + 3) >> 2;
    if (p.exc > 16) {
#pragma unroll
      for (int q = 0; q < 4; q++) put_bytes(xi + 4 * q, bm[q], 4);
    }
    // exceptions in position order: the lowest set bit of the bitmap each time
    uint32_t b0 = bm[0], b1 = bm[1], b2 = bm[2], b3 = bm[3];
    int dd = nc, rank = 0;
    uint32_t ctrl = 0;
    for (; rank < p.exc; rank++) {
      const int q = b0 ? 0 : b1 ? 1 : b2 ? 2 : 3;
      const uint32_t wq = q == 0 ? b0 : q == 1 ? b1 : q == 2 ? b2 : b3;
      const uint32_t rest = wq & (wq - 1);
      b0 = q == 0 ? rest : b0;
      b1 = q == 1 ? rest : b1;
      b2 = q == 2 ? rest : b2;
      b3 = q == 3 ? rest : b3;
      const int pos = 32 * q + __ffs(wq) - 1;
      const uint32_t hv = work_at<DELTA>(s, pos & 127, p.base, p.zz) >> bw;  // bw < 32 with exceptions
      const int l = svb_len_of(hv);
      if (p.exc <= 16) xi[rank] = (uint8_t)pos;
      ctrl |= (uint32_t)(l - 1) << (2 * (rank & 3));
      if (dd + l <= p.svb_len) put_bytes(svb + dd, hv, l);
      dd += l;
      if ((rank & 3) == 3) {
        svb[rank >> 2] = (uint8_t)ctrl;
        ctrl = 0;
      }
    }
    if ((rank & 3) && (rank >> 2) < nc) svb[rank >> 2] = (uint8_t)ctrl;
  }
}

}  // namespace lane
}  // namespace utl
