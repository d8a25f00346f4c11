/*
 * utl_simd.c -- CPU restatement of the reference's vectorized block
 * pipelines: packBlockAVX512 / unpackBlockAVX512 (simd_avx512_amd64.go:
 * 617-735, 821-888) with their per-bit-width kernels (simd_spec_amd64.go)
 * and fused width/FOR selection (:215-308), and the same pipelines eight
 * lanes at a time for AVX2 (simd_avx2_amd64.go), picked at run time as the
 * reference's dispatch does (dispatch.go:47-78: AVX-512 before AVX2).
 *
 * TEST INFRASTRUCTURE ONLY: the timed CPU baseline of the benchmark and of
 * its reference arm (the Go reference needs a Go 1.27 toolchain, absent
 * here).  Its bytes equal the scalar restatement's (utl_oracle.c) for
 * every input, as the reference's own SIMD and scalar paths do
 * (fuzz_simd_test.go:13-40); the tests check that.  Never linked into or
 * called by the product library.
 */
#include <immintrin.h>
#include <stdint.h>
#include <string.h>

#include "utl_oracle.h"
#include "utl_oracle_int.h"

/* ------------------------------------------------------------- AVX-512 */
#pragma GCC push_options
#pragma GCC target("avx512f,avx512bw,avx512vl,avx512dq,avx2,bmi,bmi2,popcnt,lzcnt")

typedef __m512i V;
#define V_LOAD(p) _mm512_loadu_si512((const void *)(p))
#define V_STORE(p, v) _mm512_storeu_si512((void *)(p), (v))
#define V_SET1(x) _mm512_set1_epi32((int)(uint32_t)(x))
#define V_ZERO() _mm512_setzero_si512()
#define V_AND(a, b) _mm512_and_si512((a), (b))
#define V_OR(a, b) _mm512_or_si512((a), (b))
#define V_XOR(a, b) _mm512_xor_si512((a), (b))
#define V_ADD(a, b) _mm512_add_epi32((a), (b))
#define V_SUB(a, b) _mm512_sub_epi32((a), (b))
#define V_SLL(a, n) _mm512_slli_epi32((a), (unsigned)(n))
#define V_SRL(a, n) _mm512_srli_epi32((a), (unsigned)(n))
#define V_SRA(a, n) _mm512_srai_epi32((a), (unsigned)(n))
#define V_MINU(a, b) _mm512_min_epu32((a), (b))
#define V_MAXU(a, b) _mm512_max_epu32((a), (b))
#define V_GTU_MASK(a, b) ((uint32_t)_mm512_cmpgt_epu32_mask((a), (b)))
#define V_HMINU(v) ((uint32_t)_mm512_reduce_min_epu32(v))
#define V_HMAXU(v) ((uint32_t)_mm512_reduce_max_epu32(v))
#define V_HOR(v) ((uint32_t)_mm512_reduce_or_epi32(v))
#define FN(x) x##_avx512
#include "utl_simd_body.inc"
#undef FN
#undef V_LOAD
#undef V_STORE
#undef V_SET1
#undef V_ZERO
#undef V_AND
#undef V_OR
#undef V_XOR
#undef V_ADD
#undef V_SUB
#undef V_SLL
#undef V_SRL
#undef V_SRA
#undef V_MINU
#undef V_MAXU
#undef V_GTU_MASK
#undef V_HMINU
#undef V_HMAXU
#undef V_HOR
#pragma GCC pop_options

/* ---------------------------------------------------------------- AVX2 */
#pragma GCC push_options
#pragma GCC target("avx2,bmi,bmi2,popcnt,lzcnt")

/* a row of 16 lanes as two 8-lane halves */
typedef struct {
  __m256i a, b;
} V2;
#define V V2
static inline V2 v2_load(const void *p) {
  V2 r = {_mm256_loadu_si256((const __m256i *)p), _mm256_loadu_si256((const __m256i *)p + 1)};
  return r;
}
static inline void v2_store(void *p, V2 v) {
  _mm256_storeu_si256((__m256i *)p, v.a);
  _mm256_storeu_si256((__m256i *)p + 1, v.b);
}
static inline V2 v2_set1(uint32_t x) {
  V2 r = {_mm256_set1_epi32((int)x), _mm256_set1_epi32((int)x)};
  return r;
}
#define V2_BIN(name, op)                       \
  static inline V2 name(V2 x, V2 y) {          \
    V2 r = {op(x.a, y.a), op(x.b, y.b)};       \
    return r;                                  \
  }
V2_BIN(v2_and, _mm256_and_si256)
V2_BIN(v2_or, _mm256_or_si256)
V2_BIN(v2_xor, _mm256_xor_si256)
V2_BIN(v2_add, _mm256_add_epi32)
V2_BIN(v2_sub, _mm256_sub_epi32)
V2_BIN(v2_minu, _mm256_min_epu32)
V2_BIN(v2_maxu, _mm256_max_epu32)
static inline V2 v2_sll(V2 x, unsigned n) {
  V2 r = {_mm256_slli_epi32(x.a, (int)n), _mm256_slli_epi32(x.b, (int)n)};
  return r;
}
static inline V2 v2_srl(V2 x, unsigned n) {
  V2 r = {_mm256_srli_epi32(x.a, (int)n), _mm256_srli_epi32(x.b, (int)n)};
  return r;
}
static inline V2 v2_sra(V2 x, unsigned n) {
  V2 r = {_mm256_srai_epi32(x.a, (int)n), _mm256_srai_epi32(x.b, (int)n)};
  return r;
}
/* unsigned a > b per lane as a 16-bit mask: signed compare after flipping
 * the sign bits */
static inline uint32_t v2_gtu_mask(V2 x, V2 y) {
  const __m256i s = _mm256_set1_epi32((int)0x80000000u);
  const __m256i ga = _mm256_cmpgt_epi32(_mm256_xor_si256(x.a, s), _mm256_xor_si256(y.a, s));
  const __m256i gb = _mm256_cmpgt_epi32(_mm256_xor_si256(x.b, s), _mm256_xor_si256(y.b, s));
  return (uint32_t)_mm256_movemask_ps(_mm256_castsi256_ps(ga)) |
         ((uint32_t)_mm256_movemask_ps(_mm256_castsi256_ps(gb)) << 8);
}
static inline uint32_t v2_hred(V2 x, int op) {
  uint32_t t[16];
  v2_store(t, x);
  uint32_t r = t[0];
  for (int i = 1; i < 16; i++) r = op == 0 ? (t[i] < r ? t[i] : r) : op == 1 ? (t[i] > r ? t[i] : r) : (r | t[i]);
  return r;
}
#define V_LOAD(p) v2_load((const void *)(p))
#define V_STORE(p, v) v2_store((void *)(p), (v))
#define V_SET1(x) v2_set1((uint32_t)(x))
#define V_ZERO() v2_set1(0u)
#define V_AND(a, b) v2_and((a), (b))
#define V_OR(a, b) v2_or((a), (b))
#define V_XOR(a, b) v2_xor((a), (b))
#define V_ADD(a, b) v2_add((a), (b))
#define V_SUB(a, b) v2_sub((a), (b))
#define V_SLL(a, n) v2_sll((a), (unsigned)(n))
#define V_SRL(a, n) v2_srl((a), (unsigned)(n))
#define V_SRA(a, n) v2_sra((a), (unsigned)(n))
#define V_MINU(a, b) v2_minu((a), (b))
#define V_MAXU(a, b) v2_maxu((a), (b))
#define V_GTU_MASK(a, b) v2_gtu_mask((a), (b))
#define V_HMINU(v) v2_hred((v), 0)
#define V_HMAXU(v) v2_hred((v), 1)
#define V_HOR(v) v2_hred((v), 2)
#define FN(x) x##_avx2
#include "utl_simd_body.inc"
#undef FN
#undef V
#pragma GCC pop_options

/* ------------------------------------------------------------ dispatch */
static int g_level = -1; /* 2 AVX-512, 1 AVX2, 0 none */

int utlo_simd_level(void) {
  if (g_level < 0) {
    __builtin_cpu_init();
    if (__builtin_cpu_supports("avx512f") && __builtin_cpu_supports("avx512bw") &&
        __builtin_cpu_supports("avx512vl") && __builtin_cpu_supports("avx512dq"))
      g_level = 2;
    else if (__builtin_cpu_supports("avx2"))
      g_level = 1;
    else
      g_level = 0;
  }
  return g_level;
}

/* Lower the level (tests run the AVX2 pipeline on AVX-512 hosts); a level
 * above what the CPU has is refused.  Returns the level in force. */
int utlo_simd_set_level(int level) {
  g_level = -1;
  const int have = utlo_simd_level();
  if (level >= 0 && level <= have) g_level = level;
  return g_level;
}

static const utlo_block_impl impl_avx512 = {pack_block_avx512, unpack_block_avx512};
static const utlo_block_impl impl_avx2 = {pack_block_avx2, unpack_block_avx2};

static const utlo_block_impl *impl(void) {
  const int l = utlo_simd_level();
  return l >= 2 ? &impl_avx512 : l == 1 ? &impl_avx2 : &utlo_scalar_impl;
}

int utlo_simd_pack_u32(uint8_t flag, const uint32_t *values, int n, uint8_t *dst, size_t *out_len) {
  return impl()->pack(flag, values, n, dst, 2u << UTLO_TYPE_SHIFT, 0, out_len);
}
int utlo_simd_unpack_u32(const uint8_t *src, size_t src_len, uint32_t *out, int *count, size_t *consumed,
                         int *ovf_pos) {
  uint32_t tmp[UTLO_BLOCK];
  int n = 0;
  size_t c = 0;
  const int err = impl()->unpack(src, src_len, 0, tmp, &n, &c, ovf_pos, NULL);
  if (err) return err;
  memcpy(out, tmp, (size_t)n * 4);
  *count = n;
  *consumed = c;
  return UTLO_OK;
}
int utlo_simd_pack_u64(uint8_t flag, const uint64_t *values, int n, uint8_t *dst, size_t *out_len) {
  return utlo_i_pack_u64(impl(), flag, values, n, dst, out_len);
}
int utlo_simd_unpack_u64(const uint8_t *src, size_t src_len, uint64_t *out, int *count, size_t *consumed,
                         int *ovf_pos) {
  return utlo_i_unpack_u64(impl(), src, src_len, out, count, consumed, ovf_pos);
}
int utlo_simd_pack_streams_u32(uint8_t flag, const uint32_t *values, const uint64_t *val_off, int n_streams,
                               uint8_t *out, size_t out_cap, uint64_t *block_off, uint64_t *stream_byte_off,
                               int n_threads) {
  return utlo_i_pack_streams(impl(), 0, flag, values, val_off, n_streams, out, out_cap, block_off, stream_byte_off,
                             n_threads);
}
int utlo_simd_pack_streams_u64(uint8_t flag, const uint64_t *values, const uint64_t *val_off, int n_streams,
                               uint8_t *out, size_t out_cap, uint64_t *block_off, uint64_t *stream_byte_off,
                               int n_threads) {
  return utlo_i_pack_streams(impl(), 1, flag, values, val_off, n_streams, out, out_cap, block_off, stream_byte_off,
                             n_threads);
}
int utlo_simd_unpack_streams_u32(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off,
                                 int n_streams, uint32_t *values, int n_threads) {
  return utlo_i_unpack_streams(impl(), 0, packed, block_off, val_off, n_streams, values, n_threads);
}
int utlo_simd_unpack_streams_u64(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off,
                                 int n_streams, uint64_t *values, int n_threads) {
  return utlo_i_unpack_streams(impl(), 1, packed, block_off, val_off, n_streams, values, n_threads);
}
