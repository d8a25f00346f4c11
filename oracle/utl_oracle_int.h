/*
 * utl_oracle_int.h -- internals shared by the two CPU restatements of the
 * reference codec: the scalar path (utl_oracle.c) and the vectorized
 * AVX-512 / AVX2 path (utl_simd.c).  TEST INFRASTRUCTURE ONLY.
 *
 * The reference shares the same pieces between its scalar and SIMD block
 * pipelines: the header codec (header.go), the exception index and
 * StreamVByte coding (exceptions.go), the unpack prologue
 * (unpack_block.go:62-172), the partial-block delta kernels (delta.go) and
 * the uint64 wrappers (uint64.go), which take the block packer as an
 * argument (packFor64 / packUint64TwoBlock, uint64.go:147-189).
 */
#ifndef UTL_ORACLE_INT_H
#define UTL_ORACLE_INT_H

#include <stddef.h>
#include <stdint.h>

#define UTLO_BLOCK 128
#define UTLO_HDR 4
#define UTLO_SVBLEN_BYTES 2
#define UTLO_B2LEN_BYTES 2
#define UTLO_EXC_BITMAP_THRESHOLD 16
#define UTLO_TYPE_SHIFT 13
#define UTLO_FORW_SHIFT 15
#define UTLO_H_DELTA (1u << 22)
#define UTLO_H_ZIGZAG (1u << 23)

/* Output of the unpack prologue (decodeUnpackHeader, unpack_block.go). */
typedef struct {
  size_t consumed, p_off, block_end;
  uint32_t for_base;
  int count, bw, exc, has_exc, delta, zigzag, has_for, u64single, empty;
} utlo_uhdr_t;

/* A block pipeline: pack one block of n <= 128 uint32 values with the
 * given header type flags (and the block2Len field of a combined uint64
 * pair), or unpack one (all 128 slots written, the first *count valid). */
typedef struct {
  int (*pack)(uint8_t flag, const uint32_t *v, int n, uint8_t *dst, uint32_t type_flags, int has_combine,
              size_t *out_len);
  int (*unpack)(const uint8_t *buf, size_t len, int for_u64, uint32_t *out, int *count, size_t *consumed, int *ovf,
                int *u64single);
} utlo_block_impl;

extern const utlo_block_impl utlo_scalar_impl;

uint32_t utlo_i_encode_header(int count, int bw, int exc, uint32_t flags);
int utlo_i_estimate_exc_cost(int exc, int step_delta);
int utlo_i_select_for_width(uint32_t m);
int utlo_i_delta_encode(uint32_t *v, int n);
void utlo_i_delta_decode(uint32_t *v, int n, int use_zz);
int utlo_i_delta_decode_overflow(uint32_t *v, int n);
int utlo_i_svb_encode(uint8_t *dst, const uint32_t *v, int n);
int utlo_i_decode_unpack_header(const uint8_t *buf, size_t len, int for_u64, utlo_uhdr_t *o);
int utlo_i_apply_exceptions(uint32_t *dst, const uint8_t *buf, size_t len, size_t exc_start, int count, int bw,
                            int exc, size_t *consumed);

/* uint64.go:302-333 / :191-266 over a block pipeline. */
int utlo_i_pack_u64(const utlo_block_impl *im, uint8_t flag, const uint64_t *v, int n, uint8_t *dst,
                    size_t *out_len);
int utlo_i_unpack_u64(const utlo_block_impl *im, const uint8_t *buf, size_t len, uint64_t *out, int *count,
                      size_t *consumed, int *ovf);

/* Many streams on n_threads host threads over a block pipeline (the
 * utlo_pack_streams / utlo_unpack_streams contract). */
int utlo_i_pack_streams(const utlo_block_impl *im, int is64, uint8_t flag, const void *values,
                        const uint64_t *val_off, int n_streams, uint8_t *out, size_t out_cap, uint64_t *block_off,
                        uint64_t *stream_byte_off, int n_threads);
int utlo_i_unpack_streams(const utlo_block_impl *im, int is64, const uint8_t *packed, const uint64_t *block_off,
                          const uint64_t *val_off, int n_streams, void *values, int n_threads);

#endif
