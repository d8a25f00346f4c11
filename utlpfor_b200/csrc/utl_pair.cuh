// utl_pair.cuh -- lane-pair UTL-PFOR pack of uint32 blocks.
//
// Two threads own one 128-value block: thread h of the pair holds UTL lane
// groups h and h+2 (UTL lanes 4h..4h+3 and 8+4h..8+4h+3; group g is the
// 16-byte chunk g of every row), so a warp packs 16 blocks at a time with
// half the staging a thread-per-block pack needs per warp -- which is what
// lets twice as many warps reside on an SM.  Everything per value is
// thread-local and streamed row by row (few registers): statistics, work
// values (FOR, per-lane delta, zigzag), payload words and exception flags;
// only block-wide facts cross the pair, with one shuffle each (min, max,
// bucket counts, borrow, exception bitmap, StreamVByte control codes).
//
// Decisions and bytes follow PackUint32 (pack.go:76-97, scalar.go:126-235):
// FOR on the raw values (for.go:95-126), per-lane delta with block-global
// zigzag (delta.go:23-48), step width and exception count by the cost model
// (select_bitwidth.go:20-72), UTL payload (scalar.go:7-59), exception index
// and StreamVByte high bits (exceptions.go:138-186).
#pragma once
#include "utl_device.cuh"
#include "utl_lane.cuh"

namespace utl {
namespace pair {

// Staging slot of one block: 512 value bytes + 32 bytes of stagger, so the
// 16-byte reads of a quarter warp (4 pairs, both groups) hit 8 distinct
// bank groups.
constexpr int kSlot = 544;
// Image windows of a 16-block tile (lane::Window's roles, half the size):
// 0 = 3584 bytes (16 warps per SM), 1 = 2304 bytes for batches of small
// blocks (18 warps per SM).
constexpr int kWindow = 3584;
constexpr int kWindowSmall = 2304;
constexpr int kSmallBlock = kWindowSmall / 16;
template <int SHAPE>
struct Window {
  static constexpr int kBytes = SHAPE == 1 ? kWindowSmall : kWindow;
  static constexpr int kImageBytes = (kBytes + lane::kMaxLen + 32 + 15) / 16 * 16;
};

// Shift a slot loaded `shift` (1..3) words late down to word 0, the pair
// splitting its 32 chunks in halves (thread 0 takes its last input chunk
// before thread 1 overwrites it).
template <int M>
__device__ __forceinline__ uint4 shift_chunk(const uint4& a, const uint4& b) {
  const uint32_t w[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
  return make_uint4(w[M], w[M + 1], w[M + 2], w[M + 3]);
}
template <int M>
__device__ __forceinline__ void realign_half(uint4* s4, int h, const uint4& edge) {
  const int c0 = 16 * h;
  uint4 a = s4[c0];
  for (int c = c0; c < c0 + 16; c++) {
    const uint4 b = (h == 0 && c == 15) ? edge : s4[c + 1];
    s4[c] = shift_chunk<M>(a, b);
    a = b;
  }
}
__device__ __noinline__ void realign_slot(uint4* s4, int shift, int h, unsigned pm) {
  const uint4 edge = s4[16];
  __syncwarp(pm);
  if (shift == 1) realign_half<1>(s4, h, edge);
  else if (shift == 2) realign_half<2>(s4, h, edge);
  else realign_half<3>(s4, h, edge);
  __syncwarp(pm);
}

__device__ __forceinline__ unsigned pair_mask(int lane) { return 3u << (lane & 30); }
__device__ __forceinline__ uint32_t padd(uint32_t x, unsigned pm) { return x + __shfl_xor_sync(pm, x, 1); }
__device__ __forceinline__ uint32_t por(uint32_t x, unsigned pm) { return x | __shfl_xor_sync(pm, x, 1); }
__device__ __forceinline__ uint32_t pmin(uint32_t x, unsigned pm) { return min(x, __shfl_xor_sync(pm, x, 1)); }
__device__ __forceinline__ uint32_t pmax(uint32_t x, unsigned pm) { return max(x, __shfl_xor_sync(pm, x, 1)); }

// Work value (FOR / delta / zigzag) of one row chunk: cur holds row r of a
// group, prv row r-1 (DELTA; the FOR base cancels in a delta).
template <bool DELTA>
__device__ __forceinline__ void work4(const uint4& cur, const uint4& prv, int r, uint32_t base, bool zz,
                                      uint32_t (&w)[4], bool& borrow) {
  const uint32_t c[4] = {cur.x, cur.y, cur.z, cur.w}, p[4] = {prv.x, prv.y, prv.z, prv.w};
#pragma unroll
  for (int k = 0; k < 4; k++) {
    if (DELTA && r > 0) {
      borrow |= c[k] < p[k];
      w[k] = c[k] - p[k];
    } else {
      w[k] = c[k] - base;
    }
    if (DELTA && zz) w[k] = zz_enc(w[k]);
  }
}

// Statistics of the thread's two groups of raw values: min/max and bucket
// counts (lane::raw_stats over half the chunks).
template <bool MM, bool HI>
__device__ __forceinline__ void raw_stats(const uint4* s4, int h, uint32_t& mn, uint32_t& mx, uint32_t& E,
                                          uint32_t& O) {
  mn = 0xFFFFFFFFu;
  mx = 0u;
  E = 0u;
  O = 0u;
#pragma unroll 2
  for (int r2 = 0; r2 < 4; r2++) {
    uint4 t[4];
    t[0] = s4[8 * r2 + h];
    t[1] = s4[8 * r2 + h + 2];
    t[2] = s4[8 * r2 + 4 + h];
    t[3] = s4[8 * r2 + 4 + h + 2];
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
      using lane::nib;
      const uint32_t a0 = nib(t[0].x) + nib(t[0].y) + nib(t[0].z) + nib(t[0].w) + nib(t[1].x) + nib(t[1].y) +
                          nib(t[1].z) + nib(t[1].w);
      const uint32_t a1 = nib(t[2].x) + nib(t[2].y) + nib(t[2].z) + nib(t[2].w) + nib(t[3].x) + nib(t[3].y) +
                          nib(t[3].z) + nib(t[3].w);
      lane::widen(a0, E, O);
      lane::widen(a1, E, O);
    }
  }
}

// Bucket counts of the thread's work values (and the delta borrow).
template <bool DELTA>
__device__ __noinline__ lane::Hist work_hist(const uint4* s4, int h, uint32_t base, bool zz) {
  uint32_t E = 0, O = 0;
  bool borrow = false;
#pragma unroll
  for (int gi = 0; gi < 2; gi++) {
    const int g = h + 2 * gi;
    uint4 prv = s4[g];
#pragma unroll
    for (int r = 0; r < 8; r += 2) {
      const uint4 c0 = s4[4 * r + g], c1 = s4[4 * (r + 1) + g];
      uint32_t w0[4], w1[4];
      work4<DELTA>(c0, prv, r, base, zz, w0, borrow);
      work4<DELTA>(c1, c0, r + 1, base, zz, w1, borrow);
      prv = c1;
      using lane::nib;
      const uint32_t a = nib(w0[0]) + nib(w0[1]) + nib(w0[2]) + nib(w0[3]) + nib(w1[0]) + nib(w1[1]) + nib(w1[2]) +
                         nib(w1[3]);
      lane::widen(a, E, O);
    }
  }
  return lane::Hist{E, O, borrow};
}

// The padding of a partial block (n < 128) holds values whose work values
// are zero, as the reference leaves them (scalar.go:34-40, delta.go:
// 23-48): the base in row 0, the lane's value one row up below it.  Each
// thread fills its own UTL lanes, row by row.
__device__ __forceinline__ void fill_padding(uint32_t* s, int n, uint32_t base, int h) {
  for (int v = 0; v < 8; v++)
#pragma unroll
    for (int gi = 0; gi < 2; gi++)
#pragma unroll
      for (int k = 0; k < 4; k++) {
        const int i = 16 * v + 4 * (h + 2 * gi) + k;
        if (i >= n) s[i] = v > 0 ? s[i - 16] : base;
      }
}

// The block's decisions and length: lane::plan_block computed over the
// pair (each thread's statistics of its half, combined across the pair).
template <bool DELTA>
__device__ lane::Plan plan_block(uint4* s4, int n, int flag, int h, unsigned pm) {
  uint32_t* s = (uint32_t*)s4;
  const bool need_mm = !(flag & kNoFOR);
  const bool need_raw_hist = !(flag & kNoFOR) || !DELTA;
  uint32_t mn, mx, E, O;
  if (need_mm) raw_stats<true, true>(s4, h, mn, mx, E, O);
  else if (need_raw_hist) raw_stats<false, true>(s4, h, mn, mx, E, O);
  else mn = mx = E = O = 0;
  if (need_mm && n < kBlock) {
    mn = 0xFFFFFFFFu;
    for (int i = h; i < n; i += 2) mn = min(mn, s[i]);  // padding is zero: only the minimum needs the count
  }
  if (need_mm) {
    mn = pmin(mn, pm);
    mx = pmax(mx, pm);
  }
  if (need_raw_hist) {
    E = padd(E, pm);
    O = padd(O, pm);
  }
  uint32_t hflags = kTypeU32 | ((uint32_t)(flag & kSpecial) << 14);
  bool use_for = false;
  uint32_t base = 0;
  int fw = 0;
  if (need_mm && mn != 0) {
    const int for_max = round_step(len32(mx - mn));
    const int raw_max = round_step(len32(mx));
    if (for_max < raw_max) {
      int std_w, dummy;
      choose_best_packed(lane::exc_from_hist(E, O), &std_w, &dummy);
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
    if (n < kBlock) {
      fill_padding(s, n, base, h);
      __syncwarp(pm);
    }
    if (DELTA || mx != mn) {
      lane::Hist hs = work_hist<DELTA>(s4, h, base, false);
      E = padd(hs.E, pm);
      O = padd(hs.O, pm);
      if (DELTA && por(hs.borrow ? 1u : 0u, pm)) {
        zz = true;
        hs = work_hist<DELTA>(s4, h, base, true);
        E = padd(hs.E, pm);
        O = padd(hs.O, pm);
      }
    } else {
      E = O = 0;  // a constant block under FOR: every work value is zero
    }
  }
  if (DELTA) hflags |= kHdrDelta | (zz ? kHdrZigZag : 0u);
  const uint64_t ec = lane::exc_from_hist(E, O);
  int bw, exc = 0;
  if (flag & kNoPatch) {
    int max_si = 0;
#pragma unroll
    for (int si = 0; si < 8; si++) max_si += ((ec >> (8 * si)) & 0xFF) != 0;
    bw = 4 * max_si;
  } else {
    choose_best_packed(ec, &bw, &exc);
  }
  lane::Plan p;
  p.bw = bw;
  p.exc = exc;
  p.base = base;
  p.zz = zz;
  p.base64 = 0;
  p.mode = kModePlain;
  p.blk2 = 0;
  p.forb = use_for ? ((1 << fw) >> 1) : 0;
  p.p_off = 4 + (exc ? 2 : 0) + p.forb;
  p.header = (uint32_t)(n & 0xFF) | ((uint32_t)(bw >> 2) << 8) | hflags | ((uint32_t)exc << 24);
  p.idx_sz = exc == 0 ? 0 : (exc <= 16 ? exc : 16);
  p.svb_len = exc ? ((exc + 3) >> 2) + lane::svb_data_bytes(E, O, bw) : 0;
  p.len = p.p_off + 16 * bw + p.idx_sz + p.svb_len;
  return p;
}

// Payload of group g at width BW, streamed row by row: each row's four
// work values, masked to BW bits, shift into the group's word accumulator;
// a completed word of the four lanes is one 16-byte segment (lane::put_seg).
// Exception flags (work value above the mask) land in f: bit 16(r&1)+k of
// f[r>>1] for row r, lane k of the group.
template <int BW, bool DELTA, bool EXC>
__device__ __forceinline__ void write_group(const uint4* s4, int g, uint32_t base, bool zz, uint32_t* pw, int d4,
                                            int sh, uint32_t (&f)[4]) {
  constexpr uint32_t MASK = BW >= 32 ? 0xFFFFFFFFu : ((1u << (BW & 31)) - 1u);
  uint32_t acc[4] = {0, 0, 0, 0};
  int wi = 0;
  bool borrow = false;
  uint4 prv = s4[g];
#pragma unroll
  for (int r = 0; r < 8; r++) {
    const uint4 cur = s4[4 * r + g];
    uint32_t w[4];
    work4<DELTA>(cur, prv, r, base, zz, w, borrow);
    prv = cur;
    if (EXC) {
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (w[k] > MASK) f[r >> 1] |= 1u << ((r & 1) * 16 + k);
    }
    if (BW == 0) continue;
    const int pos = r * BW, s = pos & 31;
    if (BW == 8) {
      // byte r&3 of the word takes the value's low byte
#pragma unroll
      for (int k = 0; k < 4; k++)
        acc[k] = (r & 3) == 0 ? (w[k] & 0xFFu) : __byte_perm(acc[k], w[k], (r & 3) == 1 ? 0x3240 : (r & 3) == 2 ? 0x3410 : 0x4210);
    } else if (BW == 16) {
#pragma unroll
      for (int k = 0; k < 4; k++) acc[k] = (r & 1) == 0 ? (w[k] & 0xFFFFu) : __byte_perm(acc[k], w[k], 0x5410);
    } else {
#pragma unroll
      for (int k = 0; k < 4; k++) acc[k] |= (w[k] & MASK) << s;
    }
    if (s + BW >= 32) {
      lane::put_seg(pw, d4, sh, wi, g, acc);
      wi++;
#pragma unroll
      for (int k = 0; k < 4; k++) acc[k] = (s + BW > 32) ? ((w[k] & MASK) >> (32 - s)) : 0u;
    }
  }
}

template <bool DELTA, bool EXC>
__device__ __forceinline__ void write_groups(int bw, const uint4* s4, int h, uint32_t base, bool zz, uint32_t* pw,
                                             int d4, int sh, uint32_t (&f)[4]) {
#pragma unroll
  for (int gi = 0; gi < 2; gi++) {
    const int g = h + 2 * gi;
    uint32_t fg[4] = {0, 0, 0, 0};
    switch (bw) {
      case 0: write_group<0, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
      case 4: write_group<4, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
      case 8: write_group<8, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
      case 12: write_group<12, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
      case 16: write_group<16, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
      case 20: write_group<20, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
      case 24: write_group<24, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
      case 28: write_group<28, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
      default: write_group<32, DELTA, EXC>(s4, g, base, zz, pw, d4, sh, fg); break;
    }
    if (EXC) {
#pragma unroll
      for (int q = 0; q < 4; q++) f[q] |= fg[q] << (4 * g);
    }
  }
}

// Set bits of m below position p.
__device__ __forceinline__ int rank_below(const uint32_t (&m)[4], int p) {
  const int q = p >> 5;
  const uint32_t low = (1u << (p & 31)) - 1u;
  int r = 0;
#pragma unroll
  for (int t = 0; t < 4; t++) r += t < q ? __popc(m[t]) : (t == q ? __popc(m[t] & low) : 0);
  return r;
}

// The exception index and StreamVByte high bits of a block whose payload
// starts at pay; own holds the exception flags of the thread's positions.
template <bool DELTA>
__device__ __forceinline__ void write_exceptions(const lane::Plan& p, const uint4* s4, uint8_t* pay,
                                                 const uint32_t (&own)[4], int h, unsigned pm) {
  const int bw = p.bw;
  uint32_t bm[4];
#pragma unroll
  for (int q = 0; q < 4; q++) bm[q] = por(own[q], pm);
  const uint32_t* s = (const uint32_t*)s4;
  uint8_t* xi = pay + 16 * bw;
  uint8_t* svb = xi + p.idx_sz;
  const int nc = (p.exc + 3) >> 2;
  if (p.exc <= 16) {
    // codes of the own exceptions, shared across the pair: the control word
    uint32_t cw = 0;
    for (uint32_t q0 = 0; q0 < 4; q0++) {
      for (uint32_t m = own[q0]; m; m &= m - 1) {
        const int pos = 32 * (int)q0 + __ffs(m) - 1;
        const int rk = rank_below(bm, pos);
        const uint32_t hv = lane::work_at<DELTA>(s, pos, p.base, p.zz) >> bw;
        cw |= (uint32_t)(svb_len_of(hv) - 1) << (2 * rk);
      }
    }
    cw = por(cw, pm);
    for (uint32_t q0 = 0; q0 < 4; q0++) {
      for (uint32_t m = own[q0]; m; m &= m - 1) {
        const int pos = 32 * (int)q0 + __ffs(m) - 1;
        const int rk = rank_below(bm, pos);
        const uint32_t hv = lane::work_at<DELTA>(s, pos, p.base, p.zz) >> bw;
        const int l = svb_len_of(hv);
        const int dd = nc + rk + quad::sum2bit(cw & ((1u << (2 * rk)) - 1u));
        xi[rk] = (uint8_t)pos;
        if (dd + l <= p.svb_len) lane::put_bytes(svb + dd, hv, l);
      }
    }
    if (h == 0)
      for (int c = 0; c < nc; c++) svb[c] = (uint8_t)(cw >> (8 * c));
  } else {
    if (h == 0) {
#pragma unroll
      for (int q = 0; q < 2; q++) lane::put_bytes(xi + 4 * q, bm[q], 4);
    } else {
#pragma unroll
      for (int q = 2; q < 4; q++) lane::put_bytes(xi + 4 * q, bm[q], 4);
    }
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
      const uint32_t hv = lane::work_at<DELTA>(s, pos & 127, p.base, p.zz) >> bw;
      const int l = svb_len_of(hv);
      ctrl |= (uint32_t)(l - 1) << (2 * (rank & 3));
      if ((rank & 1) == h && dd + l <= p.svb_len) lane::put_bytes(svb + dd, hv, l);
      dd += l;
      if ((rank & 3) == 3) {
        if (h == 0) svb[rank >> 2] = (uint8_t)ctrl;
        ctrl = 0;
      }
    }
    if (h == 0 && (rank & 3) && (rank >> 2) < nc) svb[rank >> 2] = (uint8_t)ctrl;
  }
}

// Write the block at o (shared memory): header, StreamVByte length, FOR
// base (thread 0 of the pair), the payload of the thread's two groups, then
// the exception index and StreamVByte high bits.  Up to 16 exceptions (a
// position list): each thread handles the exceptions at its own positions
// (rank = set bits of the block's bitmap below the position), the pair
// shares the 2-bit length codes (the control bytes) with one shuffle.  More
// than 16 (a bitmap): the pair walks the bitmap in position order and
// splits the stores by rank parity.
template <bool DELTA, bool EXC>
__device__ void write_block(const lane::Plan& p, const uint4* s4, uint8_t* o, int h, unsigned pm) {
  if (h == 0) {
    lane::put_bytes(o, p.header, 4);
    int m = 4;
    if (p.exc) {
      lane::put_bytes(o + 4, (uint32_t)p.svb_len, 2);
      m = 6;
    }
    if (p.forb) lane::put_bytes(o + m, p.base, p.forb);
  }
  const int bw = p.bw;
  uint8_t* pay = o + p.p_off;
  const int d4 = (int)((uintptr_t)pay & 3);
  uint32_t* pw = (uint32_t*)(pay - d4);
  const int sh = 32 - 8 * d4;
  uint32_t own[4] = {0, 0, 0, 0};
  write_groups<DELTA, EXC>(bw, s4, h, p.base, p.zz, pw, d4, sh, own);
  if constexpr (EXC) {
    if (p.exc) write_exceptions<DELTA>(p, s4, pay, own, h, pm);
  }
}

}  // namespace pair
}  // namespace utl
