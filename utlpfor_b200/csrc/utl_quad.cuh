// utl_quad.cuh -- quad-per-block UTL-PFOR codec for the batched kernels.
//
// A warp codes eight 128-value blocks at once: lanes 4q..4q+3 (a "quad")
// own block q.  Quad lane j holds UTL lanes 4j..4j+3 of every row, i.e.
// the values at positions 16v + 4j + c (row v = 0..7, c = 0..3): one
// 16-byte vector per row, so value loads and stores are 128-bit and each
// quad touches whole 64-byte rows.  Row-wise work (delta, zigzag, bit
// packing along a UTL lane) stays inside one thread; only block-wide
// decisions (min/max, exception counts, ranks, scans) cross the quad, with
// two shuffle steps.  Per-block control work is thereby shared by four
// lanes instead of thirty-two, which is what keeps the codec within the
// instruction budget of the HBM roofline.
//
// Decisions and byte layout follow the Go reference github.com/Akron/utlpfor
// exactly; each step cites the file:line it matches.
#pragma once
#include <type_traits>

#include "utl_device.cuh"

namespace utl {
namespace quad {

// ---------------------------------------------------------------- helpers
// Every quad primitive names only the quad's four lanes (qm), as a
// cooperative-groups tile of four would: quads of one warp may take
// different branches, and a full-warp mask inside such a branch is
// undefined behaviour.
__device__ __forceinline__ unsigned quad_mask(int lane) { return 0xFu << (lane & 28); }
__device__ __forceinline__ uint32_t qmin(uint32_t x, unsigned qm) {
  x = min(x, __shfl_xor_sync(qm, x, 1));
  return min(x, __shfl_xor_sync(qm, x, 2));
}
__device__ __forceinline__ uint32_t qmax(uint32_t x, unsigned qm) {
  x = max(x, __shfl_xor_sync(qm, x, 1));
  return max(x, __shfl_xor_sync(qm, x, 2));
}
__device__ __forceinline__ uint32_t qor(uint32_t x, unsigned qm) {
  x |= __shfl_xor_sync(qm, x, 1);
  return x | __shfl_xor_sync(qm, x, 2);
}
__device__ __forceinline__ uint32_t qsum(uint32_t x, unsigned qm) {
  x += __shfl_xor_sync(qm, x, 1);
  return x + __shfl_xor_sync(qm, x, 2);
}
// exclusive prefix sum over the quad (lane order j = 0..3)
__device__ __forceinline__ uint32_t qexcl(uint32_t x, int j, unsigned qm) {
  uint32_t incl = x;
  uint32_t y = __shfl_up_sync(qm, incl, 1, 4);
  if (j >= 1) incl += y;
  y = __shfl_up_sync(qm, incl, 2, 4);
  if (j >= 2) incl += y;
  return incl - x;
}
// PTX shifts clamp the amount to the register width (shift >= 64 gives 0).
__device__ __forceinline__ uint64_t shr64_clamp(uint64_t x, uint32_t s) {
  uint64_t r;
  asm("shr.b64 %0, %1, %2;" : "=l"(r) : "l"(x), "r"(s));
  return r;
}
// Sum of the 2-bit fields of x.
__device__ __forceinline__ int sum2bit(uint32_t x) { return __popc(x & 0x55555555u) + 2 * __popc(x & 0xAAAAAAAAu); }

// ---------------------------------------------------------------- unpack
struct QResult {
  int status;
  int count;
  int consumed;
  int ovf;
};

// Load 16 payload bytes at byte offset a of a byte source as four words.
template <class Src>
__device__ __forceinline__ void load16(const Src& s, int64_t a, uint32_t w[4]) {
#pragma unroll
  for (int k = 0; k < 4; k++) w[k] = s.u32(a + 4 * k);
}
template <>
__device__ __forceinline__ void load16<SmemBytes>(const SmemBytes& s, int64_t a, uint32_t w[4]) {
  const int q = (int)(a >> 2), sh = (int)(a & 3) * 8;
  const uint32_t w0 = s.w[q], w1 = s.w[q + 1], w2 = s.w[q + 2], w3 = s.w[q + 3], w4 = s.w[q + 4];
  w[0] = __funnelshift_r(w0, w1, sh);
  w[1] = __funnelshift_r(w1, w2, sh);
  w[2] = __funnelshift_r(w2, w3, sh);
  w[3] = __funnelshift_r(w3, w4, sh);
}

// UTL payload of one quad lane at a bit width known at compile time
// (scalar.go:65-116): the lane's BW/4 words of UTL lanes 4j..4j+3 are the
// 16-byte windows at pbase + 64i; all are loaded first, then every row is
// cut out with constant shifts (a value straddling words i and i+1 joins
// them), so the loop has no branches and no loads between its rows.
template <int BW>
__device__ __forceinline__ void utl_rows(const SmemBytes& sb, int pbase, uint32_t (&x)[8][4]) {
  constexpr int NW = BW / 4;
  uint32_t w[NW][4];
#pragma unroll
  for (int i = 0; i < NW; i++) load16(sb, pbase + 64 * i, w[i]);
#pragma unroll
  for (int v = 0; v < 8; v++) {
    const int pos = v * BW, wi = pos >> 5, sh = pos & 31;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t val = w[wi][k] >> sh;
      if (sh + BW > 32) val |= w[wi + 1][k] << (32 - sh);
      if (BW < 32) val &= (1u << (BW & 31)) - 1u;
      x[v][k] = val;
    }
  }
}

// The same for any width (multiple of 4, at most 32) of a staged block.
__device__ __forceinline__ void utl_rows_any(const SmemBytes& sb, int pbase, int bw, uint32_t (&x)[8][4]) {
  switch (bw) {
    case 4: utl_rows<4>(sb, pbase, x); break;
    case 8: utl_rows<8>(sb, pbase, x); break;
    case 12: utl_rows<12>(sb, pbase, x); break;
    case 16: utl_rows<16>(sb, pbase, x); break;
    case 20: utl_rows<20>(sb, pbase, x); break;
    case 24: utl_rows<24>(sb, pbase, x); break;
    case 28: utl_rows<28>(sb, pbase, x); break;
    case 32: utl_rows<32>(sb, pbase, x); break;
    default:
#pragma unroll
      for (int v = 0; v < 8; v++)
#pragma unroll
        for (int k = 0; k < 4; k++) x[v][k] = 0;
  }
}

// Bitmap-mode high bits (more than 16 exceptions): lane j sizes control
// bytes 8j..8j+7 (exceptions.go:63-80 validation), then decodes its values
// into patch[rank], pre-shifted by bw.  Returns false on a corrupt region.
template <class Src>
__device__ __forceinline__ bool decode_bitmap_high_bits(const Src& sb, int64_t svb, int exc, int nc, int svb_len,
                                                     int bw, uint32_t* patch, int j, unsigned qm) {
  int tot = 0;
  for (int g8 = 0; g8 < 8; g8++) {
    const int g = 8 * j + g8;
    if (g < nc) {
      const uint32_t c = sb.u8(svb + g);
      const int sl = min(4, exc - 4 * g);
      const uint32_t m = sl >= 4 ? 0xFFu : ((1u << (2 * sl)) - 1u);
      tot += sl + sum2bit(c & m);
    }
  }
  const int before = (int)qexcl((uint32_t)tot, j, qm);
  const int needed = nc + (int)qsum((uint32_t)tot, qm);
  if (needed > svb_len) return false;
  __syncwarp(qm);
  int64_t d = svb + nc + before;
  for (int g8 = 0; g8 < 8; g8++) {
    const int g = 8 * j + g8;
    if (g < nc) {
      const uint32_t c = sb.u8(svb + g);
      const int sl = min(4, exc - 4 * g);
      for (int s2 = 0; s2 < sl; s2++) {
        const int l = (int)((c >> (2 * s2)) & 3) + 1;
        uint32_t hv = sb.u32(d);
        if (l < 4) hv &= (1u << (8 * l)) - 1u;
        patch[4 * g + s2] = shl32(hv, bw);
        d += l;
      }
    }
  }
  __syncwarp(qm);
  return true;
}

// Unpack one uint32 block (unpackUint32Scalar, scalar.go:260-309, with
// decodeUnpackHeader unpack_block.go:62-172 and applyExceptions
// exceptions.go:194-284).  x[v][c] receives position 16v+4j+c.  patch is
// the quad's 128-word shared scratch.  Results are quad-uniform.
template <class Src, bool WIDTH_SPEC = true>
__device__ QResult quad_unpack_block(const Src& sb, int64_t blk, int64_t avail, bool for_u64, uint32_t (&x)[8][4],
                                     uint32_t* patch, int j, unsigned qm) {
  QResult r{kOK, 0, 0, 0};
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
  const int isz = has_exc ? (exc <= 16 ? exc : 16) : 0;
  int64_t end = p_off + pb + isz;
  if (avail < end) { r.status = kErrInvalidBuffer; return r; }
  int svb_len = 0;
  if (has_exc) {
    svb_len = (int)sb.u16(blk + 4);
    if (end + svb_len > avail) { r.status = kErrInvalidBuffer; return r; }
    end += svb_len;
  }
  uint32_t fbase = 0;
  if (forw > 0 && !u64s)
    fbase = forw == 1 ? sb.u8(blk + for_off) : forw == 2 ? sb.u16(blk + for_off) : sb.u32(blk + for_off);
  int consumed = p_off + pb;

  // UTL payload (scalar.go:65-116): the four lanes 4j..4j+3 of a word
  // index w are 16 contiguous bytes at 64w + 16j; a value straddling two
  // words is joined with a funnel shift.
  if constexpr (std::is_same<Src, SmemBytes>::value && WIDTH_SPEC) {
    utl_rows_any(sb, (int)blk + p_off + 16 * j, bw, x);
  } else if (bw == 0) {
#pragma unroll
    for (int v = 0; v < 8; v++)
#pragma unroll
      for (int k = 0; k < 4; k++) x[v][k] = 0;
  } else {
    const uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);
    const int64_t pbase = blk + p_off + 16 * j;
    uint32_t cur[4], nxt[4];
    load16(sb, pbase, cur);
    int wi = 1;
    int pos = 0;
    // At most one word past the lane's last word is loaded (wi <= bw/4);
    // its bits are never used but it must be readable: it lies inside the
    // block or the staging padding.
    load16(sb, pbase + 64, nxt);
#pragma unroll
    for (int v = 0; v < 8; v++) {
#pragma unroll
      for (int k = 0; k < 4; k++) x[v][k] = __funnelshift_r(cur[k], nxt[k], pos) & mask;
      pos += bw;
      if (pos >= 32 && v < 7) {
        pos -= 32;
#pragma unroll
        for (int k = 0; k < 4; k++) cur[k] = nxt[k];
        wi++;
        load16(sb, pbase + 64 * wi, nxt);
      }
    }
  }

  if (has_exc) {
    if (exc > count) { r.status = kErrInvalidBuffer; return r; }
    const int64_t xo = blk + consumed;             // exception index
    const int64_t svb = xo + isz;                  // StreamVByte region
    const int nc = (exc + 3) >> 2;
    if (nc > svb_len) { r.status = kErrInvalidBuffer; return r; }
    if (exc <= 16) {
      // <= 4 control bytes: one word.  exceptions.go:63-80 validation.
      const uint32_t cw = sb.u32(svb) & (nc >= 4 ? 0xFFFFFFFFu : ((1u << (8 * nc)) - 1u));
      const uint32_t slots = exc >= 16 ? 0xFFFFFFFFu : ((1u << (2 * exc)) - 1u);
      const int needed = nc + exc + sum2bit(cw & slots);
      if (needed > svb_len) { r.status = kErrInvalidBuffer; return r; }
      // patch through shared memory: positions are arbitrary
      __syncwarp(qm);
#pragma unroll
      for (int v = 0; v < 8; v++)
        *(uint4*)&patch[16 * v + 4 * j] = make_uint4(x[v][0], x[v][1], x[v][2], x[v][3]);
      __syncwarp(qm);
      for (int e = j; e < exc; e += 4) {
        const int p = (int)sb.u8(xo + e);
        const int tgt = count == kBlock ? (p & 127) : (p < count ? p : -1);
        const int code = (int)((cw >> (2 * e)) & 3);
        const int off = nc + e + sum2bit(cw & ((1u << (2 * e)) - 1u));
        uint32_t hv = sb.u32(svb + off);
        if (code < 3) hv &= (1u << (8 * (code + 1))) - 1u;
        if (tgt >= 0) atomicOr(&patch[tgt], shl32(hv, bw));
      }
      __syncwarp(qm);
#pragma unroll
      for (int v = 0; v < 8; v++) {
        const uint4 t = *(const uint4*)&patch[16 * v + 4 * j];
        x[v][0] = t.x; x[v][1] = t.y; x[v][2] = t.z; x[v][3] = t.w;
      }
    } else {
      // Bitmap mode: decode every high-bit value into patch[] (out of
      // line: rare), then each lane ORs the ranks of its own positions.
      if (!decode_bitmap_high_bits(sb, svb, exc, nc, svb_len, bw, patch, j, qm)) {
        r.status = kErrInvalidBuffer;
        return r;
      }
      uint32_t rowbits[8];
      int pop = 0;
#pragma unroll
      for (int v = 0; v < 8; v++) {
        uint32_t m = sb.u16(xo + 2 * v);
        const int lo = 16 * v;  // stale bits past count are masked (exceptions.go:251-260)
        if (count <= lo) m = 0;
        else if (count < lo + 16) m &= (1u << (count - lo)) - 1u;
        rowbits[v] = m;
        pop += __popc(m);
      }
      if (pop <= exc) {
        int pre = 0;
#pragma unroll
        for (int v = 0; v < 8; v++) {
          const uint32_t m = rowbits[v];
          const int mine = pre + __popc(m & ((1u << (4 * j)) - 1u));
          const uint32_t nib = (m >> (4 * j)) & 0xFu;
#pragma unroll
          for (int k = 0; k < 4; k++)
            if ((nib >> k) & 1u) x[v][k] |= patch[mine + __popc(nib & ((1u << k) - 1u))];
          pre += __popc(m);
        }
      }
      __syncwarp(qm);
    }
    consumed = (int)(svb - blk) + svb_len;
  }

  if (delta) {
    // per-lane prefix sum down the rows (delta.go:50-115); the first wrap
    // in v-major order is the lowest flat index
    int first = 0x7FFFFFFF;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t acc = zz ? zz_dec(x[0][k]) : x[0][k];
      if (zz && 4 * j + k < count) x[0][k] = acc;
#pragma unroll
      for (int v = 1; v < 8; v++) {
        const int idx = 16 * v + 4 * j + k;
        if (idx < count) {
          const uint32_t d = zz ? zz_dec(x[v][k]) : x[v][k];
          const uint32_t nx = acc + d;
          if (nx < acc && idx < first) first = idx;
          acc = nx;
          x[v][k] = acc;
        }
      }
    }
    if (!zz) {
      const int m = (int)qmin((uint32_t)first, qm);
      if (m != 0x7FFFFFFF) {
        r.status = kErrOverflow;
        r.ovf = m;
        return r;
      }
    }
  }
  if (forw > 0 && !u64s) {
#pragma unroll
    for (int v = 0; v < 8; v++)
#pragma unroll
      for (int k = 0; k < 4; k++) x[v][k] += fbase;
  }
  r.count = count;
  r.consumed = consumed;
  return r;
}

// ---------------------------------------------------------------- pack
// Decisions of one uint32 block, phase A of the pack (scalar.go:126-235).
// Store a full decoded block (quad layout: lane j holds words 16v+4j+k) at
// op (4-byte aligned).  When op is 16-byte aligned each row is four 16-byte
// stores.  Otherwise (m = op's word misalignment) the block goes through the
// quad's 128-word shared buffer and lane j writes the aligned chunk that
// starts at word 16v+4j+4-m; the first 4-m and last m words are stored
// singly.
__device__ __forceinline__ void quad_store_full(uint32_t* op, const uint32_t (&x)[8][4], uint32_t* buf, int j,
                                                unsigned qm) {
  const int m = (int)(((uintptr_t)op >> 2) & 3);
  if (m == 0) {
#pragma unroll
    for (int v = 0; v < 8; v++) __stcs((uint4*)(op + 16 * v + 4 * j), make_uint4(x[v][0], x[v][1], x[v][2], x[v][3]));
    return;
  }
  __syncwarp(qm);
#pragma unroll
  for (int v = 0; v < 8; v++) *(uint4*)(buf + 16 * v + 4 * j) = make_uint4(x[v][0], x[v][1], x[v][2], x[v][3]);
  __syncwarp(qm);
  const int sh = 4 - m;
#pragma unroll
  for (int v = 0; v < 8; v++) {
    const int r = 16 * v + 4 * j + sh;
    if (r + 4 <= kBlock) __stcs((uint4*)(op + r), make_uint4(buf[r], buf[r + 1], buf[r + 2], buf[r + 3]));
  }
  if (j == 0)
    for (int k = 0; k < sh; k++) op[k] = buf[k];
  if (j == 3)
    for (int k = kBlock - m; k < kBlock; k++) op[k] = buf[k];
  __syncwarp(qm);
}

struct QPlan {
  uint32_t header;
  uint32_t base;   // FOR base (u32 FOR)
  int bw;
  int exc;
  int forb;        // FOR base bytes written (0/1/2/4; 8 for FOR64)
  int p_off;
  int idx_sz;
  int svb_len;
  int len;
};

__device__ __forceinline__ uint32_t shl_clamp(uint32_t x, uint32_t s) {
  uint32_t r;
  asm("shl.b32 %0, %1, %2;" : "=r"(r) : "r"(x), "r"(s));
  return r;
}

// Per-thread histogram of the values' leading-zero buckets b = clz/4
// (b = 8 - bin, bin = ceil(len/4) of select_bitwidth.go:46; zero values
// fall in bucket 8 and are dropped by the clamped shift).  Each value adds
// 1 << (clz & ~3) to a word of eight 4-bit counters; the values are split
// over three words so no counter exceeds 15, then the nibbles are widened
// to bytes: E holds buckets 0,2,4,6 and O buckets 1,3,5,7.
// Positions past the block's count hold zero and land in the dropped
// bucket 8.
__device__ __forceinline__ void bucket_hist(const uint32_t (&x)[8][4], uint32_t& E, uint32_t& O) {
  uint32_t acc[3] = {0, 0, 0};
#pragma unroll
  for (int v = 0; v < 8; v++)
#pragma unroll
    for (int k = 0; k < 4; k++) acc[(4 * v + k) / 11] += shl_clamp(1u, (uint32_t)__clz(x[v][k]) & ~3u);
  E = (acc[0] & 0x0F0F0F0Fu) + (acc[1] & 0x0F0F0F0Fu) + (acc[2] & 0x0F0F0F0Fu);
  O = ((acc[0] >> 4) & 0x0F0F0F0Fu) + ((acc[1] >> 4) & 0x0F0F0F0Fu) + ((acc[2] >> 4) & 0x0F0F0F0Fu);
}

// exc[si] (byte si) = values with bin > si = values in buckets < 8 - si:
// the quad's bucket counts in order, prefix-summed, read back to front.
// Every byte stays at or below 128.
__device__ __forceinline__ uint64_t quad_exc_from_buckets(uint32_t E, uint32_t O, unsigned qm) {
  E = qsum(E, qm);
  O = qsum(O, qm);
  const uint32_t b03 = __byte_perm(E, O, 0x5140);  // buckets 0,1,2,3
  const uint32_t b47 = __byte_perm(E, O, 0x7362);  // buckets 4,5,6,7
  const uint32_t p03 = b03 * 0x01010101u;          // byte k: buckets 0..k
  const uint32_t p47 = b47 * 0x01010101u + (p03 >> 24) * 0x01010101u;
  // exc[si] = prefix byte 7 - si
  const uint32_t e_lo = __byte_perm(p47, 0, 0x0123);  // si 0..3 <- prefix bytes 7..4
  const uint32_t e_hi = __byte_perm(p03, 0, 0x0123);  // si 4..7 <- prefix bytes 3..0
  return ((uint64_t)e_hi << 32) | e_lo;
}

// Phase A: FOR (for.go:95-126), delta/zigzag (delta.go:23-48), width
// (select_bitwidth.go:20-72), exception ranks and high bits (exceptions.go:
// 138-186) and the StreamVByte length.  x[v][c] holds the block's values,
// zero past position n (the reference packs zeros there, scalar.go:34-40),
// and is turned into the work values in place.  hb (128 words, 16-byte
// aligned) receives the high bits in rank order and idx (16 bytes) the
// position list or bitmap.  mode as in warp_pack_block.  Partial blocks
// (n < 128) take masked variants of the steps that must skip padding.
__device__ QPlan quad_plan_block(uint32_t (&x)[8][4], int n, int flag, uint32_t type_flags, int mode,
                                 uint32_t* hb, uint8_t* idx, uint32_t* xs, int j, unsigned qm) {
  const bool full = n == kBlock;
#define QVALID(v, k) (16 * (v) + 4 * j + (k) < n)
  uint32_t hflags = type_flags | ((uint32_t)(flag & kSpecial) << 14);
  bool use_for = false;
  uint32_t base = 0;
  int fw = 0;
  uint32_t h_e = 0, h_o = 0;
  bool have_hist = false;
  if (!(flag & kNoFOR)) {
    uint32_t mn = 0xFFFFFFFFu, mx = 0u;
    if (full) {
#pragma unroll
      for (int v = 0; v < 8; v++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
          mn = min(mn, x[v][k]);
          mx = max(mx, x[v][k]);
        }
    } else {
#pragma unroll
      for (int v = 0; v < 8; v++)
#pragma unroll
        for (int k = 0; k < 4; k++) {
          if (QVALID(v, k)) mn = min(mn, x[v][k]);
          mx = max(mx, x[v][k]);  // padding is zero
        }
    }
    mn = qmin(mn, qm);
    mx = qmax(mx, qm);
    if (mn != 0) {
      const int for_max = round_step(len32(mx - mn));
      const int raw_max = round_step(len32(mx));
      if (for_max < raw_max) {
        bucket_hist(x, h_e, h_o);
        have_hist = true;
        int std_w, dummy;
        choose_best_packed(quad_exc_from_buckets(h_e, h_o, qm), &std_w, &dummy);
        if (for_max < std_w) {
          use_for = true;
          base = mn;
          const int nb = (len32(mn) + 7) >> 3;
          fw = nb >= 3 ? 3 : nb;
        }
      }
    }
    if (use_for) {
#pragma unroll
      for (int v = 0; v < 8; v++)
#pragma unroll
        for (int k = 0; k < 4; k++) x[v][k] = (full || QVALID(v, k)) ? x[v][k] - base : 0u;
      hflags |= (uint32_t)fw << 15;
      have_hist = false;
    }
  }
  if (flag & kDelta) {
    bool borrow = false;
#pragma unroll
    for (int k = 0; k < 4; k++)
#pragma unroll
      for (int v = 7; v >= 1; v--)
        if (full || QVALID(v, k)) {
          borrow |= x[v][k] < x[v - 1][k];
          x[v][k] -= x[v - 1][k];
        }
    const bool zz = qor(borrow ? 1u : 0u, qm) != 0;
    if (zz) {
#pragma unroll
      for (int v = 0; v < 8; v++)
#pragma unroll
        for (int k = 0; k < 4; k++) x[v][k] = zz_enc(x[v][k]);  // zz_enc(0) == 0 keeps the padding
    }
    hflags |= kHdrDelta | (zz ? kHdrZigZag : 0u);
    have_hist = false;
  }
  int bw, exc_n = 0;
  if (flag & kNoPatch) {
    uint32_t o = 0;
#pragma unroll
    for (int v = 0; v < 8; v++)
#pragma unroll
      for (int k = 0; k < 4; k++) o |= x[v][k];
    bw = round_step(len32(qor(o, qm)));
  } else {
    if (!have_hist) bucket_hist(x, h_e, h_o);
    choose_best_packed(quad_exc_from_buckets(h_e, h_o, qm), &bw, &exc_n);
  }
  QPlan p;
  p.bw = bw;
  p.exc = exc_n;
  p.base = base;
  p.forb = mode == kModeFor64 ? 8 : (use_for ? ((1 << fw) >> 1) : 0);
  if (mode == kModeFor64) hflags |= 3u << 15;
  const int meta = 4 + (exc_n ? 2 : 0);
  p.p_off = meta + p.forb + (mode == kModeCombine ? 2 : 0);
  p.header = (uint32_t)(n & 0xFF) | ((uint32_t)(bw >> 2) << 8) | hflags | ((uint32_t)exc_n << 24);
  p.idx_sz = exc_n == 0 ? 0 : (exc_n <= 16 ? exc_n : 16);
  p.svb_len = 0;
  if (exc_n > 0) {
    // Exception flags: nibble v of nibs = this lane's four flags of row v.
    const uint32_t emask = (1u << bw) - 1u;  // bw < 32 when there are exceptions
    uint32_t nibs = 0;
#pragma unroll
    for (int v = 0; v < 8; v++)
#pragma unroll
      for (int k = 0; k < 4; k++)
        if (x[v][k] > emask) nibs |= 1u << (4 * v + k);  // padding is zero
    // per-row flag counts, one byte per row (rows 0-3 in cl, 4-7 in ch)
    uint32_t t = nibs - ((nibs >> 1) & 0x55555555u);
    t = (t & 0x33333333u) + ((t >> 2) & 0x33333333u);
    uint32_t cl = t & 0xFFFFu, ch = t >> 16;
    cl = (cl & 0x00FFu) | ((cl & 0xFF00u) << 8);
    cl = (cl & 0x000F000Fu) | ((cl & 0x00F000F0u) << 4);
    ch = (ch & 0x00FFu) | ((ch & 0xFF00u) << 8);
    ch = (ch & 0x000F000Fu) | ((ch & 0x00F000F0u) << 4);
    // rank of (v, j, k) = exceptions in earlier rows + in earlier lanes of
    // row v + earlier flags of this lane in row v (ascending positions)
    const uint32_t el = qexcl(cl, j, qm), eh = qexcl(ch, j, qm);
    const uint32_t tl = qsum(cl, qm), th = qsum(ch, qm);
    const uint32_t sl = (tl * 0x01010101u) >> 24;  // all rows 0-3
    const uint32_t bl = tl * 0x01010100u + el;      // byte v: rank base of row v
    const uint32_t bh = th * 0x01010100u + sl * 0x01010101u + eh;
    // the work values go through shared memory so that only the set flag
    // bits are visited (about 0.1 per lane for typical data)
    __syncwarp(qm);
#pragma unroll
    for (int v = 0; v < 8; v++) *(uint4*)(xs + 16 * v + 4 * j) = make_uint4(x[v][0], x[v][1], x[v][2], x[v][3]);
    for (uint32_t m = nibs; m; m &= m - 1) {
      const int i = __ffs(m) - 1;
      const int v = i >> 2, k = i & 3;
      const uint32_t nib = (nibs >> (4 * v)) & 0xFu;
      const int rb = (int)(((v < 4 ? bl : bh) >> (8 * (v & 3))) & 0xFF);
      const int r = rb + __popc(nib & ((1u << k) - 1u));
      const int pos = 16 * v + 4 * j + k;
      hb[r] = xs[pos] >> bw;
      if (exc_n <= 16) idx[r] = (uint8_t)pos;
    }
    if (exc_n > 16) {
      // bitmap: bytes 2v, 2v+1 hold row v's 16 lane flags, LSB first
#pragma unroll
      for (int pr = 0; pr < 4; pr++) {
        const uint32_t n0 = (nibs >> (8 * pr)) & 0xFu, n1 = (nibs >> (8 * pr + 4)) & 0xFu;
        const uint32_t wrd = qor((n0 << (4 * j)) | (n1 << (16 + 4 * j)), qm);
        if (j == 0) *(uint32_t*)(idx + 4 * pr) = wrd;
      }
    }
    __syncwarp(qm);
    // StreamVByte data length (control bytes + minimal little-endian bytes)
    const int nc = (exc_n + 3) >> 2;
    int tot = 0;
    if (exc_n <= 16) {
      if (j < nc) {
        const uint4 g = *(const uint4*)(hb + 4 * j);
        const int sl4 = exc_n - 4 * j;
        tot = svb_len_of(g.x) + (sl4 > 1 ? svb_len_of(g.y) : 0) + (sl4 > 2 ? svb_len_of(g.z) : 0) +
              (sl4 > 3 ? svb_len_of(g.w) : 0);
      }
    } else {
      const int G = (nc + 3) >> 2;
      for (int g = G * j; g < min(nc, G * j + G); g++)
        for (int s2 = 0; s2 < 4 && 4 * g + s2 < exc_n; s2++) tot += svb_len_of(hb[4 * g + s2]);
    }
    p.svb_len = nc + (int)qsum((uint32_t)tot, qm);
  }
  p.len = p.p_off + bw * 16 + p.idx_sz + p.svb_len;
  return p;
#undef QVALID
}

// Phase C: write the block's bytes at o (shared or global memory).  x holds
// the work values of phase A, hb/idx its exception data.  base64 is the
// FOR64 base.
__device__ void quad_write_block(const QPlan& p, const uint32_t (&x)[8][4], int mode, uint64_t base64,
                                 const uint32_t* hb, const uint8_t* idx, uint8_t* o, int j, unsigned qm) {
  const int bw = p.bw;
  if (j == 0) {
    const uint32_t h = p.header;
    o[0] = (uint8_t)h; o[1] = (uint8_t)(h >> 8); o[2] = (uint8_t)(h >> 16); o[3] = (uint8_t)(h >> 24);
    const int meta = 4 + (p.exc ? 2 : 0);
    if (p.exc) { o[4] = (uint8_t)p.svb_len; o[5] = (uint8_t)(p.svb_len >> 8); }
    if (mode == kModeFor64) {
#pragma unroll
      for (int b = 0; b < 8; b++) o[meta + b] = (uint8_t)(base64 >> (8 * b));
    } else if (p.forb) {
      o[meta] = (uint8_t)p.base;
      if (p.forb > 1) o[meta + 1] = (uint8_t)(p.base >> 8);
      if (p.forb > 2) { o[meta + 2] = (uint8_t)(p.base >> 16); o[meta + 3] = (uint8_t)(p.base >> 24); }
    }
    if (mode == kModeCombine) { o[meta + p.forb] = 0; o[meta + p.forb + 1] = 0; }
  }
  // UTL payload (scalar.go:7-59): lanes 4j..4j+3 advance together, so each
  // completed word index w yields the 16 payload bytes at 64w + 16j.  The
  // payload is one contiguous run of such chunks in (w, j) order; when it
  // is not word aligned, each lane stores the aligned words ending inside
  // its chunk, joining the previous chunk's last word (from lane j-1, or
  // lane 3 of the previous word index) with a funnel shift.  Only the
  // bytes of the run's first and last partial word are stored singly.
  if (bw > 0) {
    const uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);
    uint8_t* pay = o + p.p_off;
    const int d = (int)((uintptr_t)pay & 3);
    const int sh = 8 * (4 - d);
    const int nrow = bw >> 2;
    uint32_t cur[4] = {0, 0, 0, 0};
    uint32_t prev3 = 0;
    int bits = 0, w = 0;
#pragma unroll
    for (int v = 0; v < 8; v++) {
      uint32_t m[4];
#pragma unroll
      for (int k = 0; k < 4; k++) {
        m[k] = x[v][k] & mask;
        cur[k] |= m[k] << bits;
      }
      if (bits + bw >= 32) {
        uint8_t* c = pay + 64 * w + 16 * j;
        const uint32_t up = __shfl_up_sync(qm, cur[3], 1, 4);
        const uint32_t last3 = __shfl_sync(qm, cur[3], 3, 4);
        if (d == 0) {
          if (((uintptr_t)c & 15) == 0) {
            *(uint4*)c = make_uint4(cur[0], cur[1], cur[2], cur[3]);
          } else {
            uint32_t* cw = (uint32_t*)c;
            cw[0] = cur[0]; cw[1] = cur[1]; cw[2] = cur[2]; cw[3] = cur[3];
          }
        } else {
          const uint32_t prevw = j == 0 ? prev3 : up;
          uint32_t* aw = (uint32_t*)(c - d);
          if (w == 0 && j == 0) {
            for (int b = 0; b < 4 - d; b++) c[b] = (uint8_t)(cur[0] >> (8 * b));
          } else {
            aw[0] = __funnelshift_r(prevw, cur[0], sh);
          }
          aw[1] = __funnelshift_r(cur[0], cur[1], sh);
          aw[2] = __funnelshift_r(cur[1], cur[2], sh);
          aw[3] = __funnelshift_r(cur[2], cur[3], sh);
          if (w == nrow - 1 && j == 3) {
            for (int b = 16 - d; b < 16; b++) c[b] = (uint8_t)(cur[3] >> (8 * (b - 12)));
          }
        }
        prev3 = last3;
        w++;
#pragma unroll
        for (int k = 0; k < 4; k++) cur[k] = __funnelshift_rc(m[k], 0u, 32 - bits);
        bits = bits + bw - 32;
      } else {
        bits += bw;
      }
    }
  }
  if (p.exc) {
    uint8_t* xi = o + p.p_off + bw * 16;
    for (int b = j; b < p.idx_sz; b += 4) xi[b] = idx[b];
    uint8_t* svb = xi + p.idx_sz;
    const int nc = (p.exc + 3) >> 2;
    if (p.exc <= 16) {
      // one control group per lane
      uint4 g = make_uint4(0, 0, 0, 0);
      int sl4 = 0, tot = 0;
      if (j < nc) {
        g = *(const uint4*)(hb + 4 * j);
        sl4 = min(4, p.exc - 4 * j);
        tot = svb_len_of(g.x) + (sl4 > 1 ? svb_len_of(g.y) : 0) + (sl4 > 2 ? svb_len_of(g.z) : 0) +
              (sl4 > 3 ? svb_len_of(g.w) : 0);
      }
      int dd = nc + (int)qexcl((uint32_t)tot, j, qm);
      if (j < nc) {
        const uint32_t gv[4] = {g.x, g.y, g.z, g.w};
        uint32_t ctrl = 0;
#pragma unroll
        for (int s2 = 0; s2 < 4; s2++) {
          if (s2 < sl4) {
            const uint32_t hv = gv[s2];
            const int l = svb_len_of(hv);
            ctrl |= (uint32_t)(l - 1) << (2 * s2);
            svb[dd] = (uint8_t)hv;
            if (l > 1) svb[dd + 1] = (uint8_t)(hv >> 8);
            if (l > 2) svb[dd + 2] = (uint8_t)(hv >> 16);
            if (l > 3) svb[dd + 3] = (uint8_t)(hv >> 24);
            dd += l;
          }
        }
        svb[j] = (uint8_t)ctrl;
      }
    } else {
      const int G = (nc + 3) >> 2;
      const int g0 = G * j, g1 = min(nc, G * j + G);
      int tot = 0;
      for (int g = g0; g < g1; g++)
        for (int s2 = 0; s2 < 4 && 4 * g + s2 < p.exc; s2++) tot += svb_len_of(hb[4 * g + s2]);
      int dd = nc + (int)qexcl((uint32_t)tot, j, qm);
      for (int g = g0; g < g1; g++) {
        uint32_t ctrl = 0;
        for (int s2 = 0; s2 < 4 && 4 * g + s2 < p.exc; s2++) {
          const uint32_t hv = hb[4 * g + s2];
          const int l = svb_len_of(hv);
          ctrl |= (uint32_t)(l - 1) << (2 * s2);
          for (int b = 0; b < l; b++) svb[dd + b] = (uint8_t)(hv >> (8 * b));
          dd += l;
        }
        svb[g] = (uint8_t)ctrl;
      }
    }
  }
}

}  // namespace quad
}  // namespace utl
