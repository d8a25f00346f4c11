// utl_unpack.cuh -- the batched uint32 unpack with TMA bulk staging.
//
// A warp decodes groups of 8 consecutive blocks, a quad of 4 lanes per
// block (lane j of the quad holds UTL lanes 4j..4j+3 of every row, so a row
// is one 16-byte vector), as the other quad kernels do.  What is new here:
//
//  * staging: a group's contiguous packed bytes (rounded out to 16-byte
//    chunks) go to shared memory by one cp.async.bulk copy issued by one
//    lane, completing on an mbarrier; a warp keeps NSTAGE groups in flight
//    (the one it decodes and the NSTAGE-1 after it).  Only chunks at the very
//    ends of the packed buffer, outside its 16-byte aligned interior, are
//    copied by plain loads.  Every wait is bounded (UTL_ERR_TIMEOUT).
//  * a fast path for the common block (header and bounds valid, at most 16
//    exceptions in strictly increasing positions below the count): the
//    exception positions become a 128-bit mask, each lane ORs the high bits
//    of its own positions into its registers by rank (popcounts of the
//    mask), with no shared-memory round trip of the values; anything else
//    (bitmap exception index, corrupt or unusual blocks) takes the general
//    routine, which reports the reference's exact error.
//
// Decode steps and validation follow unpackUint32Scalar (scalar.go:260-309),
// decodeUnpackHeader (unpack_block.go:62-172), applyExceptions
// (exceptions.go:194-284) and deltaDecodePerLane*WithOverflow (delta.go:
// 50-115).
#pragma once
#include "utl_device.cuh"
#include "utl_quad.cuh"

namespace utl {
namespace tma {

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_init_fence() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
      "selp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// One bulk copy global -> this CTA's shared memory, completing on bar.
// Both addresses 16-byte aligned, bytes a multiple of 16.
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(smem_u32(dst)),
      "l"(src), "r"(bytes), "r"(smem_u32(bar))
      : "memory");
}
// Bounded wait for the phase of the given parity (whole warp; uniform).
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, uint32_t lim) {
  bool ok = false;
  for (uint32_t it = 0; it < lim && !ok; it++) ok = mbar_try_wait(bar, parity);
  return __all_sync(kFull, ok);
}

}  // namespace tma

namespace quad {

// Header facts and checks of the fast path.
struct QFast {
  int count, bw, exc, nc, svb_len;
  int xo, svb;      // exception index and StreamVByte offsets (staging bytes)
  uint32_t cw;      // control bytes (at most 4)
  uint32_t m[4];    // exception positions as a 128-bit mask
  uint32_t fbase;
  int consumed;
  bool delta, zz, has_for;
};

// Whether the block at staging offset blk (length avail) takes the fast
// path; quad-uniform.  Every condition mirrors a check of the general
// routine, so a block that passes decodes exactly as the reference
// decodes it and a block that fails goes to the general routine.
__device__ __forceinline__ bool fast_plan(const SmemBytes& sb, int blk, int avail, int j, unsigned qm, QFast& f) {
  const uint32_t h = sb.u32(blk);
  f.count = (int)(h & 0xFF);
  const int bwf = (int)((h >> 8) & 31);
  const int itype = (int)((h >> 13) & 3);
  const int forw = (int)((h >> 15) & 3);
  f.exc = (int)(h >> 24);
  f.bw = 4 * bwf;
  f.delta = (h & kHdrDelta) != 0;
  f.zz = (h & kHdrZigZag) != 0;
  f.has_for = forw > 0;
  const int p_off = 4 + (f.exc ? 2 : 0) + ((1 << forw) >> 1);
  const int isz = f.exc ? min(f.exc, 16) : 0;
  f.svb_len = f.exc ? (int)sb.u16(blk + 4) : 0;
  f.consumed = p_off + 16 * f.bw + (f.exc ? isz + f.svb_len : 0);
  // unpack_block.go:62-172: type, count, width and every region in bounds
  bool ok = avail >= 4 && (itype == 1 || itype == 2) && (unsigned)(f.count - 1) < (unsigned)kBlock && bwf <= 8 &&
            f.consumed <= avail && f.exc <= 16 && f.exc <= f.count;
  const int fo = blk + 4 + (f.exc ? 2 : 0);
  f.fbase = forw == 1 ? sb.u8(fo) : forw == 2 ? sb.u16(fo) : forw == 3 ? sb.u32(fo) : 0u;
  f.xo = blk + p_off + 16 * f.bw;
  f.svb = f.xo + isz;
  f.m[0] = f.m[1] = f.m[2] = f.m[3] = 0u;
  f.cw = 0u;
  f.nc = (f.exc + 3) >> 2;
  if (ok && f.exc > 0) {
    // exceptions.go:63-80: the control bytes and the data they size fit
    f.cw = sb.u32(f.svb) & (f.nc >= 4 ? 0xFFFFFFFFu : ((1u << (8 * f.nc)) - 1u));
    const uint32_t slots = f.exc >= 16 ? 0xFFFFFFFFu : ((1u << (2 * f.exc)) - 1u);
    ok = f.nc <= f.svb_len && f.nc + f.exc + sum2bit(f.cw & slots) <= f.svb_len;
    // positions 4j..4j+3 of the list, strictly increasing and below the
    // count (then each applies to its own position, as applyExceptions
    // does, and its rank in the list is its rank in the mask)
    const uint32_t q = sb.u32(f.xo + 4 * j);
    const uint32_t qp = __shfl_up_sync(qm, q, 1, 4);
    int prev = j == 0 ? -1 : (int)(qp >> 24);
    bool bad = false;
    uint32_t m0 = 0, m1 = 0, m2 = 0, m3 = 0;
#pragma unroll
    for (int b = 0; b < 4; b++) {
      if (4 * j + b < f.exc) {
        const int p = (int)((q >> (8 * b)) & 0xFF);
        bad |= p <= prev || p >= f.count;
        prev = p;
        const uint32_t bit = 1u << (p & 31);
        const int wsel = (p >> 5) & 3;
        m0 |= wsel == 0 ? bit : 0u;
        m1 |= wsel == 1 ? bit : 0u;
        m2 |= wsel == 2 ? bit : 0u;
        m3 |= wsel == 3 ? bit : 0u;
      }
    }
    f.m[0] = qor(m0, qm);
    f.m[1] = qor(m1, qm);
    f.m[2] = qor(m2, qm);
    f.m[3] = qor(m3, qm);
    ok = ok && qor(bad ? 1u : 0u, qm) == 0;
  }
  return ok;
}

// Decode a block that fast_plan accepted.  x[v][c] receives position
// 16v+4j+c; patch is the quad's shared scratch (16 words used).  Returns
// kOK or kErrOverflow (with its position).
__device__ __forceinline__ QResult fast_decode(const SmemBytes& sb, int blk, const QFast& f, uint32_t (&x)[8][4],
                                               uint32_t* patch, int j, unsigned qm) {
  QResult r{kOK, f.count, f.consumed, 0};
  const int bw = f.bw;
  // UTL payload (scalar.go:65-116)
  if (bw == 0) {
#pragma unroll
    for (int v = 0; v < 8; v++)
#pragma unroll
      for (int k = 0; k < 4; k++) x[v][k] = 0;
  } else {
    const uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1u);
    const int pbase = f.xo - 16 * bw + 16 * j;
    uint32_t cur[4], nxt[4];
    load16(sb, pbase, cur);
    load16(sb, pbase + 64, nxt);
    int wi = 1, pos = 0;
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
  if (f.exc > 0) {
    // high bits of exceptions j, j+4, ... (exceptions.go:32-88) in rank order
    for (int e = j; e < f.exc; e += 4) {
      const int code = (int)((f.cw >> (2 * e)) & 3);
      const int off = f.nc + e + sum2bit(f.cw & ((1u << (2 * e)) - 1u));
      uint32_t hv = sb.u32(f.svb + off);
      if (code < 3) hv &= (1u << (8 * (code + 1))) - 1u;
      patch[e] = shl32(hv, bw);
    }
    __syncwarp(qm);
    // each lane ORs the high bits of its own positions: rank = set bits of
    // the mask below the position
    int pre = 0;
#pragma unroll
    for (int v = 0; v < 8; v++) {
      const uint32_t row = (f.m[v >> 1] >> (16 * (v & 1))) & 0xFFFFu;
      const uint32_t nib = (row >> (4 * j)) & 0xFu;
      if (nib) {
        int rk = pre + __popc(row & ((1u << (4 * j)) - 1u));
#pragma unroll
        for (int k = 0; k < 4; k++)
          if ((nib >> k) & 1u) x[v][k] |= patch[rk++];
      }
      pre += __popc(row);
    }
    __syncwarp(qm);
  }
  if (f.delta) {
    // per-lane prefix sums down the rows (delta.go:50-115); the first wrap
    // in row-major order is the lowest flagged index
    int first = 0x7FFFFFFF;
#pragma unroll
    for (int k = 0; k < 4; k++) {
      uint32_t acc = f.zz ? zz_dec(x[0][k]) : x[0][k];
      if (f.zz && 4 * j + k < f.count) x[0][k] = acc;
#pragma unroll
      for (int v = 1; v < 8; v++) {
        const int idx = 16 * v + 4 * j + k;
        if (idx < f.count) {
          const uint32_t d = f.zz ? zz_dec(x[v][k]) : x[v][k];
          const uint32_t nx = acc + d;
          if (nx < acc && idx < first) first = idx;
          acc = nx;
          x[v][k] = acc;
        }
      }
    }
    if (!f.zz) {
      const int m = (int)qmin((uint32_t)first, qm);
      if (m != 0x7FFFFFFF) {
        r.status = kErrOverflow;
        r.ovf = m;
        return r;
      }
    }
  }
  if (f.has_for) {
#pragma unroll
    for (int v = 0; v < 8; v++)
#pragma unroll
      for (int k = 0; k < 4; k++) x[v][k] += f.fbase;
  }
  return r;
}

}  // namespace quad
}  // namespace utl
