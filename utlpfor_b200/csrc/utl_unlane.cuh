// utl_unlane.cuh -- batched uint32 unpack, one thread per block.
//
// A warp takes a tile of 32 consecutive blocks (one per lane), stages the
// tile's packed bytes in shared memory (16-byte cp.async), and every lane
// decodes its own block row by row: the sixteen UTL lanes' current payload
// words sit in registers, each row is cut out with one funnel shift and a
// mask per value, the FOR base (or the zigzag delta sum) is applied in the
// thread, and the rows go to a small per-warp tile (two rows of each of
// the 32 blocks) from which the whole warp writes them out as 16-byte
// stores.  Per-block control work (header, validation, exceptions) is done
// once per block instead of by four or thirty-two lanes, so the warp
// issues a fraction of the quad decoder's instructions per value.
//
// The thread path takes the common blocks only: a valid header of integer
// type 1 or 2, a full block (128 values) whose length and count agree with
// the batch's tables, at most 16 exceptions in strictly increasing
// positions, exceptions only without delta, plain (not zigzag) delta only
// at widths whose sums cannot wrap (no overflow is possible, so no block
// the thread path takes can fail).  Every other block -- bitmap
// exceptions, delta with exceptions, partial or corrupt blocks -- goes to
// the quad decoder (utl_quad.cuh) after the tile's rows are out, from the
// same staged bytes, which reports the reference's exact status.  Decode steps follow unpackUint32Scalar (scalar.go:260-309),
// decodeUnpackHeader (unpack_block.go:62-172), applyExceptions
// (exceptions.go:194-284) and deltaDecodePerLane* (delta.go:50-115).
#pragma once
#include "utl_quad.cuh"

namespace utl {
namespace unlane {

constexpr int kRows = 2;                        // rows of every block per output chunk
constexpr int kTileStride = 64 * kRows + 16;    // bytes per block in the chunk tile (+16: conflict-free stores;
                                                // its first 8 bytes hold the block's first value index)
constexpr int kLanesPerBlock = 64 * kRows / 16;  // lanes that write one block's chunk
constexpr int kBlocksPerStore = 32 / kLanesPerBlock;

// Header facts of a block the thread path takes.
struct Plan {
  int bw, exc, nc, pay, xo, svb;
  uint32_t base, cw, mask;
  bool delta, zz;
};

// Whether the block at staging offset blk (len bytes; want values expected)
// takes the thread path.  Each condition is one the quad decoder checks
// too, so a block that passes decodes to exactly what the quad decoder
// gives it.  Reads stay inside the block plus four bytes (the staging
// buffer is padded).
__device__ __forceinline__ bool plan(const SmemBytes& sb, int blk, int len, int want, Plan& f) {
  if (len < 4 || want != kBlock) return false;
  const uint32_t h = sb.u32(blk);
  const int count = (int)(h & 0xFF);
  const int bwf = (int)((h >> 8) & 31);
  const int itype = (int)((h >> 13) & 3);
  const int forw = (int)((h >> 15) & 3);
  const int exc = (int)(h >> 24);
  const bool delta = (h & kHdrDelta) != 0, zz = (h & kHdrZigZag) != 0;
  // unpack_block.go:62-172: type, count and width; exceptions in list mode
  if (!(itype == 1 || itype == 2) || count != kBlock || bwf > 8 || exc > 16) return false;
  // plain delta: at width 28 or less eight values cannot wrap a uint32 sum
  // (so no overflow to report); delta blocks with exceptions go to the quads
  if (delta && (exc > 0 || (!zz && bwf > 7))) return false;
  f.zz = zz;
  f.bw = 4 * bwf;
  f.exc = exc;
  f.delta = delta;
  const int fo = 4 + (exc ? 2 : 0);
  f.pay = blk + fo + ((1 << forw) >> 1);
  const int svb_len = exc ? (int)sb.u16(blk + 4) : 0;
  if (f.pay - blk + 16 * f.bw + (exc ? exc + svb_len : 0) != len) return false;
  f.base = forw == 1 ? sb.u8(blk + fo) : forw == 2 ? sb.u16(blk + fo) : forw == 3 ? sb.u32(blk + fo) : 0u;
  f.mask = f.bw >= 32 ? 0xFFFFFFFFu : ((1u << f.bw) - 1u);
  f.xo = f.pay + 16 * f.bw;
  f.svb = f.xo + exc;
  f.nc = (exc + 3) >> 2;
  f.cw = 0;
  if (exc > 0) {
    // exceptions.go:63-80: the control bytes and the data they size fit
    f.cw = sb.u32(f.svb) & (f.nc >= 4 ? 0xFFFFFFFFu : ((1u << (8 * f.nc)) - 1u));
    const uint32_t slots = exc >= 16 ? 0xFFFFFFFFu : ((1u << (2 * exc)) - 1u);
    if (f.nc + exc + quad::sum2bit(f.cw & slots) > svb_len) return false;
    // strictly increasing positions below the count: each applies to its
    // own position, in list order
    int prev = -1;
    for (int e = 0; e < exc; e++) {
      const int p = (int)sb.u8(f.xo + e);
      if (p <= prev) return false;
      prev = p;
    }
    if (prev >= kBlock) return false;  // the last is the largest
  }
  return true;
}

// The sixteen UTL lanes' payload word at byte offset a (any alignment): 17
// aligned words joined by funnel shifts.
__device__ __forceinline__ void load_words(const SmemBytes& sb, int a, uint32_t (&w)[16]) {
  const int q = a >> 2, sh = (a & 3) * 8;
  uint32_t t[17];
#pragma unroll
  for (int i = 0; i < 17; i++) t[i] = sb.w[q + i];
#pragma unroll
  for (int i = 0; i < 16; i++) w[i] = __funnelshift_r(t[i], t[i + 1], sh);
}

}  // namespace unlane
}  // namespace utl
