/*
 * utl_oracle.h -- CPU oracle for the UTL-PFOR block codec.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of the scalar
 * code path of the Go library github.com/Akron/utlpfor, used as the
 * checker for the CUDA implementation (tests, smoke check, and the timed
 * CPU baseline of bench.py).  The product library never links, loads or
 * calls anything in this directory.
 *
 * Every function cites the reference file:line it follows.  Error codes
 * mirror the reference's sentinel errors (utlpfor.go:70-115).
 */
#ifndef UTL_ORACLE_H
#define UTL_ORACLE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Status codes, same numbering as the product C-ABI (include/utlpfor.h). */
enum {
  UTLO_OK = 0,
  UTLO_ERR_INVALID_BUFFER = 1,       /* ErrInvalidBuffer        */
  UTLO_ERR_POSITION_OUT_OF_RANGE = 2,/* ErrPositionOutOfRange   */
  UTLO_ERR_INVALID_BLOCK_LENGTH = 3, /* ErrInvalidBlockLength   */
  UTLO_ERR_INVALID_FLAGS = 4,        /* ErrInvalidFlags         */
  UTLO_ERR_UNSUPPORTED_TYPE = 5,     /* ErrUnsupportedType      */
  UTLO_ERR_NOT_IMPLEMENTED = 6,      /* ErrNotImplemented       */
  UTLO_ERR_OVERFLOW = 7              /* *ErrOverflow{Position}  */
};

/* Flag bits (utlpfor.go:24-68). */
enum {
  UTLO_DELTA = 1, UTLO_NOFOR = 2, UTLO_NOPATCH = 4, UTLO_SPECIAL = 8,
  UTLO_APPEND = 16, UTLO_NOINPLACE = 32
};

/* Pack one uint32 block (1..128 values) at dst[0..).  dst must hold
 * utlo_max_block_length32(flag) bytes.  Returns the status; *out_len gets
 * the block length.  values is not modified. */
int utlo_pack_u32(uint8_t flag, const uint32_t *values, int n, uint8_t *dst,
                  size_t *out_len);

/* Unpack one uint32 block.  out must hold 128 values.  On UTLO_ERR_OVERFLOW
 * *ovf_pos holds ErrOverflow.Position. */
int utlo_unpack_u32(const uint8_t *src, size_t src_len, uint32_t *out,
                    int *count, size_t *consumed, int *ovf_pos);

/* GetUint32.  *ovf_pos as above (full-unpack path only). */
int utlo_get_u32(int pos, const uint8_t *src, size_t src_len, uint32_t *value,
                 int *ovf_pos);

int utlo_block_length(const uint8_t *src, size_t src_len, size_t *len);

int utlo_header(const uint8_t *src, size_t src_len, int *count, int *bit_width,
                int *exc_count, int *has_delta, int *has_for, int *has_zigzag,
                int *has_special);

int utlo_max_block_length32(uint8_t flag);
int utlo_max_block_length64(uint8_t flag);

int utlo_pack_u64(uint8_t flag, const uint64_t *values, int n, uint8_t *dst,
                  size_t *out_len);
int utlo_unpack_u64(const uint8_t *src, size_t src_len, uint64_t *out,
                    int *count, size_t *consumed, int *ovf_pos);
int utlo_get_u64(int pos, const uint8_t *src, size_t src_len, uint64_t *value,
                 int *ovf_pos);

/* Stream helpers used by the tests and the CPU baseline: pack/unpack many
 * streams block by block exactly as repeated Append calls would, on
 * n_threads host threads (each thread owns a contiguous range of streams).
 *
 * values: all streams' values back to back; stream s is
 *   values[val_off[s] .. val_off[s+1]).
 * pack: out receives the packed streams back to back; block_off (optional,
 *   n_blocks+1 entries) receives each block's byte offset and stream_byte_off
 *   (n_streams+1) each stream's.  out_cap must be >= the exact size; use
 *   utlo_stream_pack_bound for a safe bound.  Returns first error or OK.
 * unpack: block b of stream s is packed[block_off[b] .. block_off[b+1]) and
 *   its values land at values[val_off[s] + 128*(b - first block of s)]. */
size_t utlo_stream_pack_bound_u32(uint8_t flag, const uint64_t *val_off,
                                  int n_streams);
size_t utlo_stream_pack_bound_u64(uint8_t flag, const uint64_t *val_off,
                                  int n_streams);
int utlo_pack_streams_u32(uint8_t flag, const uint32_t *values,
                          const uint64_t *val_off, int n_streams, uint8_t *out,
                          size_t out_cap, uint64_t *block_off,
                          uint64_t *stream_byte_off, int n_threads);
int utlo_unpack_streams_u32(const uint8_t *packed, const uint64_t *block_off,
                            const uint64_t *val_off, int n_streams,
                            uint32_t *values, int n_threads);
int utlo_pack_streams_u64(uint8_t flag, const uint64_t *values,
                          const uint64_t *val_off, int n_streams, uint8_t *out,
                          size_t out_cap, uint64_t *block_off,
                          uint64_t *stream_byte_off, int n_threads);
int utlo_unpack_streams_u64(const uint8_t *packed, const uint64_t *block_off,
                            const uint64_t *val_off, int n_streams,
                            uint64_t *values, int n_threads);

/* GetUint32/GetUint64 for n_queries (stream, position-in-stream) pairs
 * over packed streams laid out as utlo_pack_streams writes them: query i
 * reads block pos/128 of stream q_stream[i] and calls utlo_get_u32/u64 on
 * it.  status[i] = error | (overflow position << 8); a stream or position
 * out of range is UTLO_ERR_POSITION_OUT_OF_RANGE. */
void utlo_get_streams_u32(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off, int n_streams,
                          const uint32_t *q_stream, const uint64_t *q_pos, int64_t n_queries, uint32_t *out,
                          int32_t *status);
void utlo_get_streams_u64(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off, int n_streams,
                          const uint32_t *q_stream, const uint64_t *q_pos, int64_t n_queries, uint64_t *out,
                          int32_t *status);

/* The reference's vectorized pipelines (utl_simd.c): AVX-512 when the CPU
 * has it, else AVX2, else the scalar path.  Same contracts and bytes as
 * the functions above.  utlo_simd_set_level lowers the level for tests
 * (2 AVX-512, 1 AVX2, 0 scalar) and returns the level in force. */
int utlo_simd_level(void);
int utlo_simd_set_level(int level);
int utlo_simd_pack_u32(uint8_t flag, const uint32_t *values, int n, uint8_t *dst, size_t *out_len);
int utlo_simd_unpack_u32(const uint8_t *src, size_t src_len, uint32_t *out, int *count, size_t *consumed,
                         int *ovf_pos);
int utlo_simd_pack_u64(uint8_t flag, const uint64_t *values, int n, uint8_t *dst, size_t *out_len);
int utlo_simd_unpack_u64(const uint8_t *src, size_t src_len, uint64_t *out, int *count, size_t *consumed,
                         int *ovf_pos);
int utlo_simd_pack_streams_u32(uint8_t flag, const uint32_t *values, const uint64_t *val_off, int n_streams,
                               uint8_t *out, size_t out_cap, uint64_t *block_off, uint64_t *stream_byte_off,
                               int n_threads);
int utlo_simd_pack_streams_u64(uint8_t flag, const uint64_t *values, const uint64_t *val_off, int n_streams,
                               uint8_t *out, size_t out_cap, uint64_t *block_off, uint64_t *stream_byte_off,
                               int n_threads);
int utlo_simd_unpack_streams_u32(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off,
                                 int n_streams, uint32_t *values, int n_threads);
int utlo_simd_unpack_streams_u64(const uint8_t *packed, const uint64_t *block_off, const uint64_t *val_off,
                                 int n_streams, uint64_t *values, int n_threads);

#ifdef __cplusplus
}
#endif
#endif
