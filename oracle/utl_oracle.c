/*
 * utl_oracle.c -- CPU oracle for the UTL-PFOR block codec.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA implementation, and
 * the CPU restatement timed as the CPU baseline.  It is never linked into
 * or called by the product library.
 *
 * A plain-C restatement of the scalar path of github.com/Akron/utlpfor
 * (Go).  Citations are file:line in that project.  The reference's
 * StreamVByte dependency (github.com/mhr3/streamvbyte v0.4.0, go.mod:7)
 * is not available; its published format (control bytes first, 2 bits per
 * value LSB-first holding byte-length-1, then minimal little-endian data
 * bytes, unused slots zero) is restated in svb_encode/svb_decode below and
 * pinned by the reference's golden block testdata/exceptions_128.bin.
 *
 * Get() uses the delta full-unpack threshold of the reference's AVX2 /
 * AVX-512 level (get.go:18-28), the level it runs at on current x86
 * servers.  The threshold changes which validation runs on corrupt
 * blocks, never the value returned for a valid block.
 */
#include "utl_oracle.h"
#include "utl_oracle_int.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>

#define BLOCK 128
#define HDR 4
#define SVBLEN_BYTES 2
#define B2LEN_BYTES 2
#define EXC_BITMAP_THRESHOLD 16
#define FOR64_BASE 8

/* header.go:8-87 */
#define H_TYPE_SHIFT 13
#define H_FORW_SHIFT 15
#define H_SPECIAL (1u << 17)
#define H_RESERVED (1u << 18)
#define H_COMBINE (1u << 19)
#define H_BLK256 (1u << 20)
#define H_DELTA (1u << 22)
#define H_ZIGZAG (1u << 23)
#define H_EXC_SHIFT 24
#define T_U16 1
#define T_U32 2
#define T_U64 3

static inline uint32_t ld16(const uint8_t *p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); }
static inline uint32_t ld32(const uint8_t *p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}
static inline uint64_t ld64(const uint8_t *p) { return (uint64_t)ld32(p) | ((uint64_t)ld32(p + 4) << 32); }
static inline void st16(uint8_t *p, uint32_t v) { p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); }
static inline void st32(uint8_t *p, uint32_t v) {
  p[0] = (uint8_t)v; p[1] = (uint8_t)(v >> 8); p[2] = (uint8_t)(v >> 16); p[3] = (uint8_t)(v >> 24);
}
static inline void st64(uint8_t *p, uint64_t v) { st32(p, (uint32_t)v); st32(p + 4, (uint32_t)(v >> 32)); }

/* math/bits.Len32 */
static inline int len32(uint32_t x) { return x ? 32 - __builtin_clz(x) : 0; }
/* select_bitwidth.go:10 */
static inline int round_up_step(int bw) { return ((bw + 3) / 4) * 4; }
/* header.go:93 */
static inline int payload_bytes(int bw) { return ((bw + 3) >> 2) << 6; }
/* header.go:97 */
static inline int for_base_bytes(int fw) { return (1 << fw) >> 1; }
/* exceptions.go:10 */
static inline int exc_index_size(int exc) { return exc <= EXC_BITMAP_THRESHOLD ? exc : 16; }
/* svb.go:4 */
static inline int svb_ctrl_count(int n) { return (n + 3) >> 2; }
/* assumed streamvbyte.MaxEncodedLen: control bytes + 4 bytes per value;
 * consistent with MaxBlockLength32(0) == 1018 (scalar.go:327). */
static inline int max_svb_len(int n) { return svb_ctrl_count(n) + 4 * n; }
/* Go's uint32 << s yields 0 for s >= 32. */
static inline uint32_t shl32(uint32_t v, int s) { return s >= 32 ? 0u : v << s; }

typedef struct {
  int count, bw, int_type, exc, forw, has_exc, delta, zigzag, special, combine;
} hdr_t;

/* header.go:110-130 */
static hdr_t decode_header(uint32_t h) {
  hdr_t d;
  d.count = (int)(h & 0xFF);
  d.bw = (int)((h >> 8) & 0x1F) * 4;
  d.int_type = (int)((h >> H_TYPE_SHIFT) & 3);
  d.forw = (int)((h >> H_FORW_SHIFT) & 3);
  d.exc = (int)((h >> H_EXC_SHIFT) & 0xFF);
  d.has_exc = d.exc > 0;
  d.delta = (h & H_DELTA) != 0;
  d.zigzag = (h & H_ZIGZAG) != 0;
  d.special = (h & H_SPECIAL) != 0;
  d.combine = (h & H_COMBINE) != 0;
  return d;
}

/* header.go:102-108 */
static uint32_t encode_header(int count, int bw, int exc, uint32_t flags) {
  uint32_t h = (uint32_t)(count & 0xFF) | ((uint32_t)((bw / 4) & 0x1F) << 8) | flags;
  h |= (uint32_t)(exc & 0xFF) << H_EXC_SHIFT;
  return h;
}

/* ---------------- bit-width selection: select_bitwidth.go ---------------- */

static const int exc_cost_bpv[9] = {1, 1, 1, 2, 2, 3, 3, 4, 4}; /* :35 */

/* select_bitwidth.go:117-121 */
static int estimate_exc_cost(int exc, int step_delta) {
  int bpv = exc_cost_bpv[step_delta];
  int ctrl = (exc + 3) >> 2;
  int idx = exc < EXC_BITMAP_THRESHOLD ? exc : EXC_BITMAP_THRESHOLD;
  return SVBLEN_BYTES + idx + ctrl + exc * bpv;
}

/* select_bitwidth.go:56-72: ties keep the wider width (strict <). */
static void choose_best_from_hist(const int hist[9], int max_si, int *best_w, int *best_exc) {
  int bw = max_si * 4, be = 0;
  int best_cost = HDR + (max_si << 6);
  int above = 0;
  for (int si = max_si - 1; si >= 0; si--) {
    above += hist[si + 1];
    int cost = HDR + (si << 6) + estimate_exc_cost(above, max_si - si);
    if (cost < best_cost) { best_cost = cost; bw = si * 4; be = above; }
  }
  *best_w = bw;
  *best_exc = be;
}

/* select_bitwidth.go:41-51 */
static void select_bitwidth(const uint32_t *v, int n, int *bw, int *exc) {
  int hist[9] = {0};
  uint32_t orv = 0;
  for (int i = 0; i < n; i++) { orv |= v[i]; hist[(len32(v[i]) + 3) >> 2]++; }
  choose_best_from_hist(hist, (len32(orv) + 3) >> 2, bw, exc);
}

/* select_bitwidth.go:20-26 */
static int select_bitwidth_nopatch(const uint32_t *v, int n) {
  uint32_t orv = 0;
  for (int i = 0; i < n; i++) orv |= v[i];
  return round_up_step(len32(orv));
}

/* ---------------- FOR: for.go ---------------- */

/* for.go:11-13 */
static int select_for_width(uint32_t m) {
  static const int lut[5] = {0, 1, 2, 3, 3};
  return lut[(len32(m) + 7) >> 3];
}

/* for.go:95-126 (findMinMaxScalar + decideFORFull) */
static void select_with_for(const uint32_t *v, int n, int *use, uint32_t *base, int *fw) {
  uint32_t mn = v[0], mx = v[0];
  for (int i = 1; i < n; i++) { if (v[i] < mn) mn = v[i]; if (v[i] > mx) mx = v[i]; }
  *use = 0; *base = 0; *fw = 0;
  if (mn == 0) return;
  int for_max = round_up_step(len32(mx - mn));
  int raw_max = round_up_step(len32(mx));
  if (for_max >= raw_max) return;
  int std_w, dummy;
  select_bitwidth(v, n, &std_w, &dummy);
  if (for_max >= std_w) return;
  *use = 1; *base = mn; *fw = select_for_width(mn);
}

/* ---------------- delta / zigzag: delta.go ---------------- */

static inline uint32_t zz_enc(uint32_t v) { return (v << 1) ^ (uint32_t)((int32_t)v >> 31); }
static inline uint32_t zz_dec(uint32_t v) { return (v >> 1) ^ (uint32_t)(-(int32_t)(v & 1)); }

/* delta.go:23-48 */
static int delta_encode(uint32_t *v, int n) {
  int zz = 0;
  for (int lane = 0; lane < 16; lane++)
    for (int r = 7; r > 0; r--) {
      int cur = lane + r * 16, prev = cur - 16;
      if (cur >= n || prev >= n) continue;
      if (v[cur] < v[prev]) zz = 1;
      v[cur] = v[cur] - v[prev];
    }
  if (zz)
    for (int i = 0; i < n; i++) v[i] = zz_enc(v[i]);
  return zz;
}

/* delta.go:50-77 */
static void delta_decode(uint32_t *v, int n, int use_zz) {
  for (int lane = 0; lane < 16; lane++) {
    if (lane >= n) break;
    if (use_zz) v[lane] = zz_dec(v[lane]);
    for (int r = 1; r < 8; r++) {
      int cur = lane + r * 16;
      if (cur >= n) break;
      v[cur] = v[cur - 16] + (use_zz ? zz_dec(v[cur]) : v[cur]);
    }
  }
}

/* delta.go:83-115: first wrap in v-major order, 0 if none. */
static int delta_decode_overflow(uint32_t *v, int n) {
  int pos = 0;
  for (int r = 1; r < 8; r++)
    for (int lane = 0; lane < 16; lane++) {
      int cur = lane + r * 16, prev = cur - 16;
      if (cur >= n) break;
      uint32_t next = v[prev] + v[cur];
      if (pos == 0 && next < v[prev]) pos = cur;
      v[cur] = next;
    }
  return pos;
}

/* ---------------- UTL bit packing: scalar.go:7-116 ---------------- */

/* Value i sits in lane i%16, row i/16; lane L's bit stream is a run of
 * 32-bit words, word w at byte w*64 + L*4 (scalar.go:19-59). */
static void pack_lanes(uint8_t *dst, const uint32_t *v, int n, int bw) {
  if (bw == 0) return;
  uint64_t mask = bw >= 32 ? 0xFFFFFFFFull : ((1ull << bw) - 1);
  for (int lane = 0; lane < 16; lane++) {
    uint64_t acc = 0;
    int bits = 0, out = lane * 4;
    for (int r = 0; r < 8; r++) {
      int i = lane + r * 16;
      uint32_t x = i < n ? v[i] : 0;
      acc |= ((uint64_t)x & mask) << bits;
      bits += bw;
      while (bits >= 32) { st32(dst + out, (uint32_t)acc); out += 64; acc >>= 32; bits -= 32; }
    }
    if (bits > 0) st32(dst + out, (uint32_t)acc);
  }
}

/* scalar.go:65-116; always decodes all 128 slots. */
static void unpack_lanes(uint32_t *dst, const uint8_t *payload, size_t plen, int bw) {
  if (bw == 0) { memset(dst, 0, BLOCK * 4); return; }
  uint32_t mask = bw >= 32 ? 0xFFFFFFFFu : ((1u << bw) - 1);
  for (int lane = 0; lane < 16; lane++) {
    uint64_t acc = 0;
    int bits = 0;
    size_t in = (size_t)lane * 4;
    for (int r = 0; r < 8; r++) {
      while (bits < bw) {
        /* the pair-lane loader reads 8 bytes at the even lane's offset */
        size_t pair = in - (size_t)(lane & 1) * 4;
        if (pair + 8 > plen) { bits = bw; break; }
        acc |= (uint64_t)ld32(payload + in) << bits;
        in += 64;
        bits += 32;
      }
      dst[lane + r * 16] = (uint32_t)acc & mask;
      acc >>= bw;
      bits -= bw;
    }
  }
}

/* ---------------- StreamVByte (github.com/mhr3/streamvbyte format) ---------------- */

static inline int svb_len_of(uint32_t x) { return x < (1u << 8) ? 1 : x < (1u << 16) ? 2 : x < (1u << 24) ? 3 : 4; }

static int svb_encode(uint8_t *dst, const uint32_t *v, int n) {
  int nc = svb_ctrl_count(n);
  memset(dst, 0, (size_t)nc);
  int off = nc;
  for (int i = 0; i < n; i++) {
    int l = svb_len_of(v[i]);
    dst[i >> 2] |= (uint8_t)((l - 1) << ((i & 3) * 2));
    for (int b = 0; b < l; b++) dst[off + b] = (uint8_t)(v[i] >> (8 * b));
    off += l;
  }
  return off;
}

static void svb_decode(const uint8_t *src, int n, uint32_t *out) {
  int off = svb_ctrl_count(n);
  for (int i = 0; i < n; i++) {
    int l = ((src[i >> 2] >> ((i & 3) * 2)) & 3) + 1;
    uint32_t x = 0;
    for (int b = 0; b < l; b++) x |= (uint32_t)src[off + b] << (8 * b);
    out[i] = x;
    off += l;
  }
}

/* svb.go:9-26 */
static int svb_group_size(uint8_t c) {
  return (c & 3) + ((c >> 2) & 3) + ((c >> 4) & 3) + ((c >> 6) & 3) + 4;
}

/* svb.go:72-100 */
static uint32_t svb_read_value(const uint8_t *d, size_t len, size_t off, int bl) {
  if (off >= len) return 0;
  size_t end = off + (size_t)bl < len ? off + (size_t)bl : len;
  uint32_t acc = 0;
  for (size_t i = off; i < end; i++) acc |= (uint32_t)d[i] << ((i - off) * 8);
  return acc;
}

/* svb.go:40-70 */
static uint32_t svb_decode_one(const uint8_t *enc, size_t len, int count, int index) {
  if (count <= 0 || index < 0 || index >= count) return 0;
  size_t off = (size_t)svb_ctrl_count(count);
  int tcb = index >> 2, slot = index & 3;
  for (int cb = 0; cb < tcb; cb++) {
    if ((size_t)cb >= len) return 0;
    off += (size_t)svb_group_size(enc[cb]);
  }
  if ((size_t)tcb >= len) return 0;
  uint8_t c = enc[tcb];
  for (int s = 0; s < slot; s++) off += (size_t)((c >> (s * 2)) & 3) + 1;
  return svb_read_value(enc, len, off, ((c >> (slot * 2)) & 3) + 1);
}

/* ---------------- block pack: scalar.go:126-235 ---------------- */

static int pack_block(uint8_t flag, const uint32_t *values, int n, uint8_t *dst, uint32_t type_flags,
                      int has_combine, size_t *out_len) {
  if (n <= 0 || n > BLOCK) return UTLO_ERR_INVALID_BUFFER;
  uint32_t work[BLOCK];
  memcpy(work, values, (size_t)n * 4);
  uint32_t hflags = type_flags | ((uint32_t)(flag & UTLO_SPECIAL) << 14);

  int use_for = 0, fw = 0;
  uint32_t base = 0;
  if (!(flag & UTLO_NOFOR)) {
    select_with_for(values, n, &use_for, &base, &fw);
    if (use_for) {
      for (int i = 0; i < n; i++) work[i] -= base;
      hflags |= (uint32_t)fw << H_FORW_SHIFT;
    }
  }
  if (flag & UTLO_DELTA) {
    if (delta_encode(work, n)) hflags |= H_ZIGZAG;
    hflags |= H_DELTA;
  }
  int bw, exc = 0;
  if (flag & UTLO_NOPATCH) bw = select_bitwidth_nopatch(work, n);
  else select_bitwidth(work, n, &bw, &exc);

  int pbytes = payload_bytes(bw);
  int forb = for_base_bytes(fw);
  int p_off = HDR + (exc ? SVBLEN_BYTES : 0) + forb + (has_combine ? B2LEN_BYTES : 0);
  if (has_combine) st16(dst + p_off - B2LEN_BYTES, 0); /* filled by the uint64 caller */
  st32(dst, encode_header(n, bw, exc, hflags));
  if (use_for) {
    uint8_t *b = dst + HDR + (exc ? SVBLEN_BYTES : 0);
    if (fw == 1) b[0] = (uint8_t)base;
    else if (fw == 2) st16(b, base);
    else if (fw == 3) st32(b, base);
  }
  memset(dst + p_off, 0, (size_t)pbytes);
  pack_lanes(dst + p_off, work, n, bw);
  if (!exc) { *out_len = (size_t)(p_off + pbytes); return UTLO_OK; }

  /* exceptions.go:138-186 */
  uint32_t high[BLOCK];
  uint32_t mask = (1u << bw) - 1; /* bw < 32 whenever exc > 0 */
  uint8_t *idx = dst + p_off + pbytes;
  int k = 0;
  if (exc <= EXC_BITMAP_THRESHOLD) {
    for (int i = 0; i < n; i++)
      if (work[i] > mask) { idx[k] = (uint8_t)i; high[k++] = work[i] >> bw; }
  } else {
    memset(idx, 0, 16);
    for (int i = 0; i < n; i++)
      if (work[i] > mask) { idx[i >> 3] |= (uint8_t)(1u << (i & 7)); high[k++] = work[i] >> bw; }
  }
  uint8_t *svb = idx + exc_index_size(exc);
  int svb_len = svb_encode(svb, high, exc);
  st16(dst + HDR, (uint32_t)svb_len);
  *out_len = (size_t)(svb - dst) + (size_t)svb_len;
  return UTLO_OK;
}

int utlo_pack_u32(uint8_t flag, const uint32_t *values, int n, uint8_t *dst, size_t *out_len) {
  /* pack.go:76-97 and scalar.go:239-255: Append only moves the write
   * position, which the caller owns here. */
  return pack_block(flag, values, n, dst, (uint32_t)T_U32 << H_TYPE_SHIFT, 0, out_len);
}

/* ---------------- block unpack: unpack_block.go + scalar.go:260-309 ---------------- */

typedef utlo_uhdr_t uhdr_t;

static int check_int_type(int t, int for_u64) {
  if (for_u64) return t == T_U64 ? UTLO_OK : UTLO_ERR_UNSUPPORTED_TYPE; /* header.go:187 */
  return (t == T_U32 || t == T_U16) ? UTLO_OK : UTLO_ERR_UNSUPPORTED_TYPE; /* header.go:175 */
}

/* unpack_block.go:62-172 */
static int decode_unpack_header(const uint8_t *buf, size_t len, int for_u64, uhdr_t *o) {
  memset(o, 0, sizeof(*o));
  if (len < HDR) return UTLO_ERR_INVALID_BUFFER;
  hdr_t h = decode_header(ld32(buf));
  int err = check_int_type(h.int_type, for_u64);
  if (err) return err;
  if (!for_u64) h.combine = 0;
  if ((unsigned)(h.count - 1) >= BLOCK || (unsigned)h.bw > 32) {
    if (h.count == 0) { o->empty = 1; return UTLO_OK; }
    if (h.count > BLOCK) return UTLO_ERR_INVALID_BLOCK_LENGTH;
    return UTLO_ERR_INVALID_BUFFER;
  }
  int u64s = for_u64 && h.int_type == T_U64 && h.forw == 3 && !h.combine;
  size_t p_off = HDR + (h.has_exc ? SVBLEN_BYTES : 0);
  size_t for_off = p_off;
  if (h.forw > 0) p_off += u64s ? FOR64_BASE : (size_t)for_base_bytes(h.forw);
  if (h.combine) p_off += B2LEN_BYTES;
  size_t pb = (size_t)payload_bytes(h.bw);
  size_t end = p_off + pb + (h.has_exc ? (size_t)exc_index_size(h.exc) : 0);
  if (len < end) return UTLO_ERR_INVALID_BUFFER;
  if (h.has_exc) {
    size_t svb_len = ld16(buf + HDR);
    if (end + svb_len > len) return UTLO_ERR_INVALID_BUFFER;
    end += svb_len;
  }
  uint32_t fb = 0;
  if (h.forw > 0 && !u64s) {
    if (h.forw == 1) fb = buf[for_off];
    else if (h.forw == 2) fb = ld16(buf + for_off);
    else fb = ld32(buf + for_off);
  }
  o->consumed = p_off + pb;
  o->p_off = p_off;
  o->block_end = end;
  o->for_base = fb;
  o->count = h.count;
  o->bw = h.bw;
  o->exc = h.exc;
  o->has_exc = h.has_exc;
  o->delta = h.delta;
  o->zigzag = h.zigzag;
  o->has_for = h.forw > 0;
  o->u64single = u64s;
  return UTLO_OK;
}

/* exceptions.go:32-88; buf is limited to the block end. */
static int decode_exc_high_bits(uint32_t *dst, const uint8_t *buf, size_t len, size_t exc_start, int exc,
                                size_t *consumed) {
  if (len < HDR + SVBLEN_BYTES) return UTLO_ERR_INVALID_BUFFER;
  size_t svb_len = ld16(buf + HDR);
  size_t svb_start = exc_start + (size_t)exc_index_size(exc);
  if (svb_start + svb_len > len) return UTLO_ERR_INVALID_BUFFER;
  size_t nc = (size_t)svb_ctrl_count(exc);
  if (nc > svb_len) return UTLO_ERR_INVALID_BUFFER;
  const uint8_t *ctrl = buf + svb_start;
  size_t need = nc;
  for (int g = 0; g < exc / 4; g++) need += (size_t)svb_group_size(ctrl[g]);
  int k = exc % 4;
  if (k > 0) {
    uint8_t c = ctrl[exc / 4];
    for (int s = 0; s < k; s++) need += (size_t)((c >> (s * 2)) & 3) + 1;
  }
  if (need > svb_len) return UTLO_ERR_INVALID_BUFFER;
  svb_decode(ctrl, exc, dst);
  *consumed = svb_start + svb_len;
  return UTLO_OK;
}

/* exceptions.go:194-284 */
static int apply_exceptions(uint32_t *dst, const uint8_t *buf, size_t len, size_t exc_start, int count, int bw,
                            int exc, size_t *consumed) {
  if (exc > count) return UTLO_ERR_INVALID_BUFFER;
  uint32_t hb[BLOCK];
  int err = decode_exc_high_bits(hb, buf, len, exc_start, exc, consumed);
  if (err) return err;
  if (exc <= EXC_BITMAP_THRESHOLD) {
    const uint8_t *pos = buf + exc_start;
    for (int i = 0; i < exc; i++) {
      if (count == BLOCK) dst[pos[i] & 0x7F] |= shl32(hb[i], bw);
      else if (pos[i] < count) dst[pos[i]] |= shl32(hb[i], bw);
    }
  } else {
    for (int i = 0; i < exc; i++) hb[i] = shl32(hb[i], bw);
    uint64_t w0 = ld64(buf + exc_start), w1 = ld64(buf + exc_start + 8);
    if (count < BLOCK) {
      if (count < 64) { w1 = 0; w0 &= (1ull << count) - 1; }
      else w1 &= (1ull << (count - 64)) - 1;
    }
    if (__builtin_popcountll(w0) + __builtin_popcountll(w1) > exc) return UTLO_OK;
    int k = 0;
    for (; w0; w0 &= w0 - 1) dst[__builtin_ctzll(w0)] |= hb[k++];
    for (; w1; w1 &= w1 - 1) dst[64 + __builtin_ctzll(w1)] |= hb[k++];
  }
  return UTLO_OK;
}

/* scalar.go:260-309; out receives all 128 slots, the first *count valid. */
static int unpack_block(const uint8_t *buf, size_t len, int for_u64, uint32_t *out, int *count, size_t *consumed,
                        int *ovf, int *u64single) {
  uhdr_t h;
  int err = decode_unpack_header(buf, len, for_u64, &h);
  if (err) return err;
  if (u64single) *u64single = h.u64single;
  if (h.empty) { *count = 0; *consumed = HDR; return UTLO_OK; }
  len = h.block_end;
  unpack_lanes(out, buf + h.p_off, (size_t)payload_bytes(h.bw), h.bw);
  size_t cons = h.consumed;
  if (h.has_exc) {
    err = apply_exceptions(out, buf, len, h.consumed, h.count, h.bw, h.exc, &cons);
    if (err) return err;
  }
  if (h.delta) {
    if (h.zigzag) delta_decode(out, h.count, 1);
    else {
      int p = delta_decode_overflow(out, h.count);
      if (p > 0) { if (ovf) *ovf = p; return UTLO_ERR_OVERFLOW; }
    }
  }
  if (h.has_for && !h.u64single)
    for (int i = 0; i < h.count; i++) out[i] += h.for_base;
  *count = h.count;
  *consumed = cons;
  return UTLO_OK;
}

int utlo_unpack_u32(const uint8_t *src, size_t src_len, uint32_t *out, int *count, size_t *consumed, int *ovf_pos) {
  uint32_t tmp[BLOCK];
  int n = 0;
  size_t c = 0;
  int err = unpack_block(src, src_len, 0, tmp, &n, &c, ovf_pos, NULL);
  if (err) return err;
  memcpy(out, tmp, (size_t)n * 4);
  *count = n;
  *consumed = c;
  return UTLO_OK;
}

/* ---------------- shared internals (utl_oracle_int.h) ---------------- */

const utlo_block_impl utlo_scalar_impl = {pack_block, unpack_block};

uint32_t utlo_i_encode_header(int count, int bw, int exc, uint32_t flags) { return encode_header(count, bw, exc, flags); }
int utlo_i_estimate_exc_cost(int exc, int step_delta) { return estimate_exc_cost(exc, step_delta); }
int utlo_i_select_for_width(uint32_t m) { return select_for_width(m); }
int utlo_i_delta_encode(uint32_t *v, int n) { return delta_encode(v, n); }
void utlo_i_delta_decode(uint32_t *v, int n, int use_zz) { delta_decode(v, n, use_zz); }
int utlo_i_delta_decode_overflow(uint32_t *v, int n) { return delta_decode_overflow(v, n); }
int utlo_i_svb_encode(uint8_t *dst, const uint32_t *v, int n) { return svb_encode(dst, v, n); }
int utlo_i_decode_unpack_header(const uint8_t *buf, size_t len, int for_u64, utlo_uhdr_t *o) {
  return decode_unpack_header(buf, len, for_u64, o);
}
int utlo_i_apply_exceptions(uint32_t *dst, const uint8_t *buf, size_t len, size_t exc_start, int count, int bw,
                            int exc, size_t *consumed) {
  return apply_exceptions(dst, buf, len, exc_start, count, bw, exc, consumed);
}

/* ---------------- Get: get.go ---------------- */

/* get.go:18-28 at the AVX2/AVX-512 level */
static int delta_full_unpack_threshold(int bw) { return bw >= 20 ? 4 : 8; }

/* get.go:34-67 */
static uint32_t extract_packed(int pos, const uint8_t *payload, size_t plen, int bw) {
  int lane = pos % 16, pil = pos / 16;
  int bitpos = pil * bw, word = bitpos / 32, boff = bitpos % 32;
  size_t off = (size_t)word * 64 + (size_t)lane * 4;
  uint64_t acc = 0;
  if (off + 4 <= plen) acc = ld32(payload + off);
  if (bw > 32 - boff) {
    size_t n2 = off + 64;
    if (n2 + 4 <= plen) acc |= (uint64_t)ld32(payload + n2) << 32;
  }
  acc >>= boff;
  uint64_t mask = bw >= 32 ? 0xFFFFFFFFull : ((1ull << bw) - 1);
  return (uint32_t)(acc & mask);
}

/* get.go:363-381 */
static int bitmap_rank128(const uint8_t *bm, size_t len, int byte_idx, int bit_idx) {
  if (len < 16) return 0;
  uint64_t w0 = ld64(bm), w1 = ld64(bm + 8);
  if (byte_idx < 8) return __builtin_popcountll(w0 & ((1ull << (8 * byte_idx + bit_idx)) - 1));
  return __builtin_popcountll(w0) + __builtin_popcountll(w1 & ((1ull << (8 * (byte_idx - 8) + bit_idx)) - 1));
}

/* exceptions.go:293-325 */
static int find_exception_index(const uint8_t *x, size_t len, int exc, int pos) {
  if (exc <= EXC_BITMAP_THRESHOLD) {
    int n = (size_t)exc < len ? exc : (int)len;
    for (int i = 0; i < n; i++) {
      if (x[i] == (uint8_t)pos) return i;
      if (x[i] > (uint8_t)pos) return -1;
    }
    return -1;
  }
  size_t bl = len < 16 ? len : 16;
  if (bl == 0) return -1;
  int bi = pos / 8, bit = pos % 8;
  if ((size_t)bi >= bl) return -1;
  if (!(x[bi] & (1u << bit))) return -1;
  return bitmap_rank128(x, bl, bi, bit);
}

/* get.go:297-334 */
static void apply_lane_exceptions(uint32_t *lv, const uint8_t *x, size_t xlen, int exc, int lane, int pil,
                                  int count, int bw) {
  size_t isz = (size_t)exc_index_size(exc);
  const uint8_t *svb = x + isz;
  size_t svb_len = xlen - isz;
  if (exc <= EXC_BITMAP_THRESHOLD) {
    for (int i = 0; i < exc; i++) {
      int p = x[i];
      if (p % 16 != lane) continue;
      int v = p / 16;
      if (v > pil) break;
      lv[v] |= shl32(svb_decode_one(svb, svb_len, exc, i), bw);
    }
  } else {
    for (int v = 0; v <= pil; v++) {
      int s = lane + v * 16;
      if (s >= count) break;
      int bi = s / 8, bit = s % 8;
      if (!(x[bi] & (1u << bit))) continue;
      int rank = bitmap_rank128(x, 16, bi, bit);
      lv[v] |= shl32(svb_decode_one(svb, svb_len, exc, rank), bw);
    }
  }
}

/* get.go:81-190 */
static int get_u32_impl(int pos, const uint8_t *src, size_t len, int for_u64, uint32_t *value, int *ovf) {
  if (len < HDR) return UTLO_ERR_INVALID_BUFFER;
  hdr_t h = decode_header(ld32(src));
  int err = check_int_type(h.int_type, for_u64);
  if (err) return err;
  if (!for_u64) h.combine = 0;
  if (pos < 0 || pos >= h.count) return UTLO_ERR_POSITION_OUT_OF_RANGE;
  if (h.bw > 32) return UTLO_ERR_INVALID_BUFFER;
  int u64s = for_u64 && h.int_type == T_U64 && h.forw == 3 && !h.combine;
  size_t p_off = HDR + (h.has_exc ? SVBLEN_BYTES : 0);
  int forb = 0;
  if (h.forw > 0) {
    if (u64s) p_off += FOR64_BASE;
    else { forb = for_base_bytes(h.forw); p_off += (size_t)forb; }
  }
  if (h.combine) p_off += B2LEN_BYTES;
  size_t pb = (size_t)payload_bytes(h.bw);
  size_t end = p_off + pb;
  if (len < end) return UTLO_ERR_INVALID_BUFFER;
  if (h.has_exc) {
    if (h.exc > h.count) return UTLO_ERR_INVALID_BUFFER;
    size_t svb_len = ld16(src + HDR);
    size_t isz = (size_t)exc_index_size(h.exc);
    if (svb_len < (size_t)svb_ctrl_count(h.exc) || end + isz + svb_len > len) return UTLO_ERR_INVALID_BUFFER;
    end += isz + svb_len;
  }
  len = end;
  uint32_t fb = 0;
  if (forb == 1) fb = src[p_off - 1];
  else if (forb == 2) fb = ld16(src + p_off - 2);
  else if (forb == 4) fb = ld32(src + p_off - 4);
  const uint8_t *payload = src + p_off;
  size_t exc_start = p_off + pb;

  if (!h.delta) { /* get.go:228-244 */
    uint32_t v = h.bw > 0 ? extract_packed(pos, payload, pb, h.bw) : 0;
    if (h.has_exc) {
      const uint8_t *x = src + exc_start;
      size_t xlen = len - exc_start;
      int ei = find_exception_index(x, xlen, h.exc, pos);
      if (ei >= 0) {
        size_t isz = (size_t)exc_index_size(h.exc);
        v |= shl32(svb_decode_one(x + isz, xlen - isz, h.exc, ei), h.bw);
      }
    }
    *value = v + fb;
    return UTLO_OK;
  }

  int pil = pos / 16;
  if (pil > delta_full_unpack_threshold(h.bw)) { /* get.go:198-218, 339-349 */
    uint32_t tmp[BLOCK];
    int n = 0;
    size_t c = 0;
    err = unpack_block(src, len, for_u64, tmp, &n, &c, ovf, NULL);
    if (err) return err;
    *value = tmp[pos];
    return UTLO_OK;
  }

  /* get.go:250-285 */
  int lane = pos % 16;
  uint32_t lv[8] = {0};
  for (int v = 0; v <= pil; v++) {
    int s = lane + v * 16;
    if (s >= h.count) break;
    if (h.bw > 0) lv[v] = extract_packed(s, payload, pb, h.bw);
  }
  if (h.has_exc) apply_lane_exceptions(lv, src + exc_start, len - exc_start, h.exc, lane, pil, h.count, h.bw);
  if (h.zigzag) lv[0] = zz_dec(lv[0]);
  for (int v = 1; v <= pil; v++) {
    int s = lane + v * 16;
    if (s >= h.count) break;
    lv[v] = lv[v - 1] + (h.zigzag ? zz_dec(lv[v]) : lv[v]);
  }
  *value = lv[pil] + fb;
  return UTLO_OK;
}

int utlo_get_u32(int pos, const uint8_t *src, size_t src_len, uint32_t *value, int *ovf_pos) {
  return get_u32_impl(pos, src, src_len, 0, value, ovf_pos);
}

/* ---------------- BlockLength / Header / MaxBlockLength ---------------- */

/* block_length.go:8-65 */
int utlo_block_length(const uint8_t *src, size_t len, size_t *out) {
  if (len < HDR) return UTLO_ERR_INVALID_BUFFER;
  uint32_t word = ld32(src);
  hdr_t h = decode_header(word);
  if (h.count > BLOCK) return UTLO_ERR_INVALID_BLOCK_LENGTH;
  if (h.bw > 32) return UTLO_ERR_INVALID_BUFFER;
  int combine = h.combine && h.int_type == T_U64;
  if (h.int_type == T_U64) {
    if (word & (H_RESERVED | H_BLK256)) return UTLO_ERR_INVALID_FLAGS;
  } else if (word & (H_RESERVED | H_COMBINE | H_BLK256)) {
    return UTLO_ERR_INVALID_FLAGS;
  }
  int forb = (h.int_type == T_U64 && !combine && h.forw == 3) ? FOR64_BASE : for_base_bytes(h.forw);
  size_t p_off = HDR + (h.has_exc ? SVBLEN_BYTES : 0) + (size_t)forb + (combine ? B2LEN_BYTES : 0);
  size_t b1 = p_off + ((size_t)h.bw << 4);
  if (h.has_exc) {
    if (len < HDR + SVBLEN_BYTES) return UTLO_ERR_INVALID_BUFFER;
    b1 += (size_t)exc_index_size(h.exc) + ld16(src + HDR);
  }
  if (!combine) { *out = b1; return UTLO_OK; }
  if (len < p_off) return UTLO_ERR_INVALID_BUFFER;
  *out = b1 + ld16(src + p_off - B2LEN_BYTES);
  return UTLO_OK;
}

/* header.go:135-153 */
int utlo_header(const uint8_t *src, size_t len, int *count, int *bw, int *exc, int *delta, int *has_for, int *zz,
                int *special) {
  *count = *bw = *exc = *delta = *has_for = *zz = *special = 0;
  if (len < HDR) return UTLO_ERR_INVALID_BUFFER;
  hdr_t h = decode_header(ld32(src));
  if (check_int_type(h.int_type, 0)) return UTLO_ERR_UNSUPPORTED_TYPE;
  *count = h.count; *bw = h.bw; *exc = h.exc; *delta = h.delta;
  *has_for = h.forw > 0; *zz = h.zigzag; *special = h.special;
  return UTLO_OK;
}

/* scalar.go:336-357 */
int utlo_max_block_length32(uint8_t flag) {
  int for_b = (flag & UTLO_NOFOR) ? 0 : 4;
  if (flag & UTLO_NOPATCH) return HDR + for_b + payload_bytes(32);
  return HDR + SVBLEN_BYTES + for_b + payload_bytes(28) + EXC_BITMAP_THRESHOLD + max_svb_len(BLOCK);
}

/* uint64.go:451-453 */
int utlo_max_block_length64(uint8_t flag) { return 2 * utlo_max_block_length32(flag) + B2LEN_BYTES; }

/* ---------------- uint64: uint64.go ---------------- */

/* uint64.go:302-333 with packFor64 (:147) and packUint64TwoBlock (:161) */
int utlo_i_pack_u64(const utlo_block_impl *im, uint8_t flag, const uint64_t *v, int n, uint8_t *dst,
                    size_t *out_len) {
  if (n <= 0 || n > BLOCK) return UTLO_ERR_INVALID_BUFFER;
  uint8_t inner = (uint8_t)(flag & ~UTLO_APPEND);
  uint64_t mn = v[0], mx = v[0], acc = 0;
  for (int i = 0; i < n; i++) { acc |= v[i]; if (v[i] < mn) mn = v[i]; if (v[i] > mx) mx = v[i]; }
  uint32_t lo[BLOCK], hi[BLOCK];
  const uint32_t t64 = (uint32_t)T_U64 << H_TYPE_SHIFT;
  int err;
  if (!(inner & UTLO_NOFOR) && mn > 0 && (mx - mn) < (1ull << 32)) {
    for (int i = 0; i < n; i++) lo[i] = (uint32_t)(v[i] - mn);
    size_t ilen;
    err = im->pack((uint8_t)(inner | UTLO_NOFOR), lo, n, dst + FOR64_BASE, t64, 0, &ilen);
    if (err) return err;
    /* uint64.go:124-142: move header(+svbLen) forward, insert the base */
    uint32_t hw = ld32(dst + FOR64_BASE);
    int ins = HDR + (((hw >> H_EXC_SHIFT) & 0xFF) > 0 ? SVBLEN_BYTES : 0);
    memmove(dst, dst + FOR64_BASE, (size_t)ins);
    st64(dst + ins, mn);
    st32(dst, hw | (3u << H_FORW_SHIFT));
    *out_len = ilen + FOR64_BASE;
    return UTLO_OK;
  }
  if ((acc >> 32) == 0) {
    for (int i = 0; i < n; i++) lo[i] = (uint32_t)v[i];
    return im->pack(inner, lo, n, dst, t64, 0, out_len);
  }
  for (int i = 0; i < n; i++) { lo[i] = (uint32_t)v[i]; hi[i] = (uint32_t)(v[i] >> 32); }
  size_t l1, l2;
  err = im->pack(inner, lo, n, dst, t64 | H_COMBINE, 1, &l1);
  if (err) return err;
  err = im->pack(inner, hi, n, dst + l1, t64, 0, &l2);
  if (err) return err;
  hdr_t h1 = decode_header(ld32(dst));
  st16(dst + HDR + (h1.has_exc ? SVBLEN_BYTES : 0) + for_base_bytes(h1.forw), (uint32_t)l2);
  *out_len = l1 + l2;
  return UTLO_OK;
}

int utlo_pack_u64(uint8_t flag, const uint64_t *v, int n, uint8_t *dst, size_t *out_len) {
  return utlo_i_pack_u64(&utlo_scalar_impl, flag, v, n, dst, out_len);
}

/* uint64.go:191-266 */
int utlo_i_unpack_u64(const utlo_block_impl *im, const uint8_t *buf, size_t len, uint64_t *out, int *count,
                      size_t *consumed, int *ovf) {
  if (len < HDR) return UTLO_ERR_INVALID_BUFFER;
  hdr_t h = decode_header(ld32(buf));
  if (h.int_type != T_U64) return UTLO_ERR_UNSUPPORTED_TYPE;
  uint32_t lo[BLOCK], hi[BLOCK];
  int n = 0, n2 = 0;
  size_t c1 = 0, c2 = 0;
  int err;
  if (!h.combine) {
    uint64_t base = 0;
    if (h.forw == 3) {
      size_t off = HDR + (h.exc > 0 ? SVBLEN_BYTES : 0);
      if (len < off + FOR64_BASE) return UTLO_ERR_INVALID_BUFFER;
      base = ld64(buf + off);
    }
    err = im->unpack(buf, len, 1, lo, &n, &c1, ovf, NULL);
    if (err) return err;
    for (int i = 0; i < n; i++) out[i] = (uint64_t)lo[i] + base;
    *count = n;
    *consumed = c1;
    return UTLO_OK;
  }
  err = im->unpack(buf, len, 1, lo, &n, &c1, ovf, NULL);
  if (err) return err;
  int forb = for_base_bytes(h.forw);
  size_t meta = HDR + (h.has_exc ? SVBLEN_BYTES : 0) + (size_t)forb + B2LEN_BYTES;
  if (len < meta) return UTLO_ERR_INVALID_BUFFER;
  size_t b2len = ld16(buf + meta - B2LEN_BYTES);
  if (c1 + b2len > len) return UTLO_ERR_INVALID_BUFFER;
  err = im->unpack(buf + c1, b2len, 1, hi, &n2, &c2, ovf, NULL);
  if (err) return err;
  if (n2 != n) return UTLO_ERR_INVALID_BUFFER;
  for (int i = 0; i < n; i++) out[i] = ((uint64_t)hi[i] << 32) | lo[i];
  *count = n;
  *consumed = c1 + b2len;
  return UTLO_OK;
}

int utlo_unpack_u64(const uint8_t *buf, size_t len, uint64_t *out, int *count, size_t *consumed, int *ovf) {
  return utlo_i_unpack_u64(&utlo_scalar_impl, buf, len, out, count, consumed, ovf);
}

/* uint64.go:372-436 */
int utlo_get_u64(int pos, const uint8_t *buf, size_t len, uint64_t *value, int *ovf) {
  if (len < HDR) return UTLO_ERR_INVALID_BUFFER;
  hdr_t h = decode_header(ld32(buf));
  if (h.int_type != T_U64) return UTLO_ERR_UNSUPPORTED_TYPE;
  uint32_t lo, hi;
  int err = get_u32_impl(pos, buf, len, 1, &lo, ovf);
  if (err) return err;
  if (!h.combine) {
    uint64_t base = 0;
    if (h.forw == 3) {
      size_t off = HDR + (h.exc > 0 ? SVBLEN_BYTES : 0);
      if (len < off + FOR64_BASE) return UTLO_ERR_INVALID_BUFFER;
      base = ld64(buf + off);
    }
    *value = (uint64_t)lo + base;
    return UTLO_OK;
  }
  int forb = for_base_bytes(h.forw);
  size_t meta = HDR + (h.has_exc ? SVBLEN_BYTES : 0) + (size_t)forb + B2LEN_BYTES;
  if (len < meta) return UTLO_ERR_INVALID_BUFFER;
  size_t b2len = ld16(buf + meta - B2LEN_BYTES);
  size_t b1 = meta + ((size_t)h.bw << 4);
  if (h.has_exc) {
    if (len < HDR + SVBLEN_BYTES) return UTLO_ERR_INVALID_BUFFER;
    b1 += (size_t)(h.exc < EXC_BITMAP_THRESHOLD ? h.exc : EXC_BITMAP_THRESHOLD) + ld16(buf + HDR);
  }
  if (b1 + b2len > len) return UTLO_ERR_INVALID_BUFFER;
  err = get_u32_impl(pos, buf + b1, b2len, 1, &hi, ovf);
  if (err) return err;
  *value = ((uint64_t)hi << 32) | lo;
  return UTLO_OK;
}

/* ---------------- multi-threaded stream helpers ---------------- */

static int64_t n_blocks_of(uint64_t n) { return (int64_t)((n + BLOCK - 1) / BLOCK); }

typedef struct {
  const utlo_block_impl *im;
  int is64;
  uint8_t flag;
  const void *values;
  const uint64_t *val_off;
  const int64_t *bstart; /* per-stream first block index, n_streams+1 */
  int n_streams;
  int64_t b0, b1;        /* this worker's block range */
  uint8_t *buf;          /* private output */
  size_t used;
  uint32_t *lens;        /* per-block lengths, b1-b0 */
  int err;
  struct pack_shared *shared;
} pack_job_t;

static int stream_of_block(const int64_t *bstart, int n_streams, int64_t b) {
  int lo = 0, hi = n_streams; /* bstart[lo] <= b < bstart[hi] */
  while (hi - lo > 1) {
    int mid = (lo + hi) / 2;
    if (bstart[mid] <= b) lo = mid; else hi = mid;
  }
  return lo;
}

/* Shared state of one pack_streams call: each worker packs its block range
 * into its own buffer, waits for all, then copies its bytes to their final
 * place and writes its blocks' offsets (both phases run in parallel). */
typedef struct pack_shared {
  pthread_barrier_t bar;
  pack_job_t *jobs;
  int n_threads;
  uint8_t *out;
  size_t out_cap;
  uint64_t *block_off;
  int64_t nb;
} pack_shared_t;

static void *pack_worker(void *arg) {
  pack_job_t *j = (pack_job_t *)arg;
  if (j->b0 < j->b1) {
    int s = stream_of_block(j->bstart, j->n_streams, j->b0);
    for (int64_t b = j->b0; b < j->b1; b++) {
      while (b >= j->bstart[s + 1]) s++;
      uint64_t first = j->val_off[s] + (uint64_t)(b - j->bstart[s]) * BLOCK;
      uint64_t last = j->val_off[s + 1];
      int n = (int)((last - first) < BLOCK ? (last - first) : BLOCK);
      size_t l = 0;
      int err = j->is64 ? utlo_i_pack_u64(j->im, j->flag, (const uint64_t *)j->values + first, n, j->buf + j->used, &l)
                        : j->im->pack(j->flag, (const uint32_t *)j->values + first, n, j->buf + j->used,
                                      (uint32_t)T_U32 << H_TYPE_SHIFT, 0, &l);
      if (err) { j->err = err; break; }
      j->lens[b - j->b0] = (uint32_t)l;
      j->used += l;
    }
  }
  pack_shared_t *sh = j->shared;
  pthread_barrier_wait(&sh->bar);
  size_t off = 0, total = 0;
  int err = 0;
  for (int t = 0; t < sh->n_threads; t++) {
    if (sh->jobs[t].err) err = 1;
    if (&sh->jobs[t] < j) off += sh->jobs[t].used;
    total += sh->jobs[t].used;
  }
  if (err || total > sh->out_cap) return NULL;
  memcpy(sh->out + off, j->buf, j->used);
  if (sh->block_off) {
    uint64_t acc = off;
    for (int64_t b = j->b0; b < j->b1; b++) { sh->block_off[b] = acc; acc += j->lens[b - j->b0]; }
    if (j->b1 == sh->nb) sh->block_off[sh->nb] = acc;
  }
  return NULL;
}

static int64_t *block_starts(const uint64_t *val_off, int n_streams) {
  int64_t *bs = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n_streams + 1));
  bs[0] = 0;
  for (int s = 0; s < n_streams; s++) bs[s + 1] = bs[s] + n_blocks_of(val_off[s + 1] - val_off[s]);
  return bs;
}

static size_t stream_pack_bound(uint8_t flag, const uint64_t *val_off, int n_streams, int is64) {
  int64_t nb = 0;
  for (int s = 0; s < n_streams; s++) nb += n_blocks_of(val_off[s + 1] - val_off[s]);
  return (size_t)nb * (size_t)(is64 ? utlo_max_block_length64(flag) : utlo_max_block_length32(flag));
}

size_t utlo_stream_pack_bound_u32(uint8_t flag, const uint64_t *val_off, int n_streams) {
  return stream_pack_bound(flag, val_off, n_streams, 0);
}
size_t utlo_stream_pack_bound_u64(uint8_t flag, const uint64_t *val_off, int n_streams) {
  return stream_pack_bound(flag, val_off, n_streams, 1);
}

/* Per-thread output buffers kept from call to call (grown on demand), so
 * that a timed call does not pay for fresh pages. */
#define MAX_WS 1024
static pthread_mutex_t g_ws_mu = PTHREAD_MUTEX_INITIALIZER;
static uint8_t *g_ws_buf[MAX_WS];
static size_t g_ws_cap[MAX_WS];

int utlo_i_pack_streams(const utlo_block_impl *im, int is64, uint8_t flag, const void *values,
                        const uint64_t *val_off, int n_streams, uint8_t *out, size_t out_cap, uint64_t *block_off,
                        uint64_t *stream_byte_off, int n_threads) {
  if (n_threads < 1) n_threads = 1;
  if (n_threads > MAX_WS) n_threads = MAX_WS;
  int64_t *bs = block_starts(val_off, n_streams);
  int64_t nb = bs[n_streams];
  pack_job_t *jobs = (pack_job_t *)calloc((size_t)n_threads, sizeof(pack_job_t));
  pthread_t *th = (pthread_t *)calloc((size_t)n_threads, sizeof(pthread_t));
  size_t maxb = (size_t)(is64 ? utlo_max_block_length64(flag) : utlo_max_block_length32(flag));
  uint32_t *lens = (uint32_t *)malloc(sizeof(uint32_t) * (size_t)(nb > 0 ? nb : 1));
  int err = UTLO_OK;
  pack_shared_t sh;
  sh.jobs = jobs; sh.n_threads = n_threads; sh.out = out; sh.out_cap = out_cap; sh.block_off = block_off; sh.nb = nb;
  pthread_barrier_init(&sh.bar, NULL, (unsigned)n_threads);
  pthread_mutex_lock(&g_ws_mu);
  for (int t = 0; t < n_threads; t++) {
    pack_job_t *j = &jobs[t];
    j->im = im; j->is64 = is64; j->flag = flag; j->values = values; j->val_off = val_off; j->bstart = bs;
    j->n_streams = n_streams;
    j->b0 = nb * t / n_threads; j->b1 = nb * (t + 1) / n_threads;
    const size_t need = maxb * (size_t)(j->b1 - j->b0) + 1;
    if (g_ws_cap[t] < need) {
      free(g_ws_buf[t]);
      g_ws_buf[t] = (uint8_t *)malloc(need);
      g_ws_cap[t] = g_ws_buf[t] ? need : 0;
    }
    j->buf = g_ws_buf[t];
    j->lens = lens + j->b0;
    j->shared = &sh;
    if (!j->buf) err = UTLO_ERR_INVALID_BUFFER;
  }
  if (!err) {
    for (int t = 1; t < n_threads; t++) pthread_create(&th[t], NULL, pack_worker, &jobs[t]);
    pack_worker(&jobs[0]);
    for (int t = 1; t < n_threads; t++) pthread_join(th[t], NULL);
    size_t total = 0;
    for (int t = 0; t < n_threads; t++) { if (jobs[t].err && !err) err = jobs[t].err; total += jobs[t].used; }
    if (!err && total > out_cap) err = UTLO_ERR_INVALID_BUFFER;
  }
  pthread_mutex_unlock(&g_ws_mu);
  if (!err && block_off && nb == 0) block_off[0] = 0;
  if (!err && stream_byte_off) {
    /* stream s starts where its first block does */
    uint64_t a = 0;
    int64_t b = 0;
    for (int s = 0; s <= n_streams; s++) {
      while (b < bs[s]) a += lens[b++];
      stream_byte_off[s] = a;
    }
  }
  pthread_barrier_destroy(&sh.bar);
  free(jobs); free(th); free(lens); free(bs);
  return err;
}

int utlo_pack_streams_u32(uint8_t flag, const uint32_t *values, const uint64_t *val_off, int n_streams, uint8_t *out,
                          size_t out_cap, uint64_t *block_off, uint64_t *stream_byte_off, int n_threads) {
  return utlo_i_pack_streams(&utlo_scalar_impl, 0, flag, values, val_off, n_streams, out, out_cap, block_off,
                             stream_byte_off, n_threads);
}
int utlo_pack_streams_u64(uint8_t flag, const uint64_t *values, const uint64_t *val_off, int n_streams, uint8_t *out,
                          size_t out_cap, uint64_t *block_off, uint64_t *stream_byte_off, int n_threads) {
  return utlo_i_pack_streams(&utlo_scalar_impl, 1, flag, values, val_off, n_streams, out, out_cap, block_off,
                             stream_byte_off, n_threads);
}

typedef struct {
  const utlo_block_impl *im;
  int is64;
  const uint8_t *packed;
  const uint64_t *block_off, *val_off;
  const int64_t *bstart;
  int n_streams;
  int64_t b0, b1;
  void *values;
  int err;
} unpack_job_t;

/* Each worker unpacks a contiguous range of blocks; a block must consume
 * exactly its indexed length and hold the expected value count, as a
 * caller walking the stream (example_test.go:171-186) would see it. */
static void *unpack_worker(void *arg) {
  unpack_job_t *j = (unpack_job_t *)arg;
  if (j->b0 >= j->b1) return NULL;
  int s = stream_of_block(j->bstart, j->n_streams, j->b0);
  for (int64_t b = j->b0; b < j->b1; b++) {
    while (b >= j->bstart[s + 1]) s++;
    uint64_t first = j->val_off[s] + (uint64_t)(b - j->bstart[s]) * BLOCK;
    uint64_t last = j->val_off[s + 1];
    int want = (int)((last - first) < BLOCK ? (last - first) : BLOCK);
    size_t off = j->block_off[b], blen = j->block_off[b + 1] - off;
    int n = 0, ovf = 0;
    size_t c = 0;
    int err;
    if (j->is64) {
      err = utlo_i_unpack_u64(j->im, j->packed + off, blen, (uint64_t *)j->values + first, &n, &c, &ovf);
    } else if (want == BLOCK) {
      err = j->im->unpack(j->packed + off, blen, 0, (uint32_t *)j->values + first, &n, &c, &ovf, NULL);
    } else {
      uint32_t tmp[BLOCK];
      err = j->im->unpack(j->packed + off, blen, 0, tmp, &n, &c, &ovf, NULL);
      if (!err && n == want) memcpy((uint32_t *)j->values + first, tmp, (size_t)n * 4);
    }
    if (!err && (n != want || c != blen)) err = UTLO_ERR_INVALID_BUFFER;
    if (err) { j->err = err; return NULL; }
  }
  return NULL;
}

int utlo_i_unpack_streams(const utlo_block_impl *im, int is64, const uint8_t *packed, const uint64_t *block_off,
                          const uint64_t *val_off, int n_streams, void *values, int n_threads) {
  if (n_threads < 1) n_threads = 1;
  int64_t *bs = block_starts(val_off, n_streams);
  int64_t nb = bs[n_streams];
  unpack_job_t *jobs = (unpack_job_t *)calloc((size_t)n_threads, sizeof(unpack_job_t));
  pthread_t *th = (pthread_t *)calloc((size_t)n_threads, sizeof(pthread_t));
  for (int t = 0; t < n_threads; t++) {
    unpack_job_t *j = &jobs[t];
    j->im = im; j->is64 = is64; j->packed = packed; j->block_off = block_off; j->val_off = val_off; j->bstart = bs;
    j->n_streams = n_streams; j->values = values;
    j->b0 = nb * t / n_threads; j->b1 = nb * (t + 1) / n_threads;
  }
  for (int t = 1; t < n_threads; t++) pthread_create(&th[t], NULL, unpack_worker, &jobs[t]);
  unpack_worker(&jobs[0]);
  for (int t = 1; t < n_threads; t++) pthread_join(th[t], NULL);
  int err = UTLO_OK;
  for (int t = 0; t < n_threads; t++) if (jobs[t].err && !err) err = jobs[t].err;
  free(jobs); free(th); free(bs);
  return err;
}

int utlo_unpack_streams_u32(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off, int n_streams,
                            uint32_t *values, int n_threads) {
  return utlo_i_unpack_streams(&utlo_scalar_impl, 0, packed, block_off, val_off, n_streams, values, n_threads);
}
int utlo_unpack_streams_u64(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off, int n_streams,
                            uint64_t *values, int n_threads) {
  return utlo_i_unpack_streams(&utlo_scalar_impl, 1, packed, block_off, val_off, n_streams, values, n_threads);
}

/* Batched Get over packed streams: the block index of stream s's first
 * block is the running sum of ceil(n/128) over the streams before it. */
static void get_streams(int is64, const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off,
                        int n_streams, const uint32_t *q_stream, const uint64_t *q_pos, int64_t n_queries, void *out,
                        int32_t *status) {
  int64_t *bs = block_starts(val_off, n_streams);
  for (int64_t i = 0; i < n_queries; i++) {
    const uint32_t s = q_stream[i];
    const uint64_t p = q_pos[i];
    int err = UTLO_ERR_POSITION_OUT_OF_RANGE, ovf = 0;
    uint64_t v = 0;
    if ((int64_t)s < n_streams && p < val_off[s + 1] - val_off[s]) {
      const int64_t b = bs[s] + (int64_t)(p / BLOCK);
      const uint8_t *blk = packed + block_off[b];
      const size_t len = (size_t)(block_off[b + 1] - block_off[b]);
      if (is64) {
        err = utlo_get_u64((int)(p % BLOCK), blk, len, &v, &ovf);
      } else {
        uint32_t v32 = 0;
        err = utlo_get_u32((int)(p % BLOCK), blk, len, &v32, &ovf);
        v = v32;
      }
    }
    if (is64) ((uint64_t *)out)[i] = err ? 0 : v;
    else ((uint32_t *)out)[i] = err ? 0 : (uint32_t)v;
    status[i] = err | (err == UTLO_ERR_OVERFLOW ? ovf << 8 : 0);
  }
  free(bs);
}

void utlo_get_streams_u32(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off, int n_streams,
                          const uint32_t *q_stream, const uint64_t *q_pos, int64_t n_queries, uint32_t *out,
                          int32_t *status) {
  get_streams(0, packed, block_off, val_off, n_streams, q_stream, q_pos, n_queries, out, status);
}
void utlo_get_streams_u64(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off, int n_streams,
                          const uint32_t *q_stream, const uint64_t *q_pos, int64_t n_queries, uint64_t *out,
                          int32_t *status) {
  get_streams(1, packed, block_off, val_off, n_streams, q_stream, q_pos, n_queries, out, status);
}
