/*
 * utlpfor.h -- C ABI of the B200 (sm_100a) UTL-PFOR block codec.
 *
 * Drop-in boundary for the Go package github.com/Akron/utlpfor: each
 * per-call entry point below is what that package's cgo shim binds in
 * place of the Go function named beside it (file:line in the reference).
 * All compute runs on the GPU; there is no CPU code path for pack, unpack
 * or get.  Header parsing helpers (utl_block_length, utl_header,
 * utl_max_block_length*) read a few header bytes on the host, as the
 * reference does.
 *
 * Conventions
 *  - Every function returns a status: 0 on success, else one of UTL_ERR_*.
 *    Codes 1..7 are the reference's errors (utlpfor.go:70-115); the cgo
 *    shim maps them back to the same Go error values.
 *  - Per-call functions take HOST pointers and block until the result is
 *    back on the host.  They are safe to call from several threads; each
 *    host thread gets its own CUDA stream and staging buffers on the
 *    current device.  A utl_codec handle (the Compressor32/64 counterpart)
 *    carries its own stream and buffers.
 *  - utl_*_batch_* functions take DEVICE pointers, enqueue work on the
 *    given cudaStream_t (passed as void*, NULL = legacy default stream) and
 *    return without synchronizing.  Device buffers must be 16-byte aligned.
 *  - Streams: stream s of a batch holds values[val_off[s] .. val_off[s+1])
 *    and packs to ceil(n_s/128) blocks laid out back to back exactly as
 *    repeated PackUint32(flag|Append, block, dst, ...) calls would lay them
 *    out (pack.go:76-97); streams follow each other in the packed buffer.
 *    block_start[s] is the index of stream s's first block (utl_batch_plan).
 */
#ifndef UTLPFOR_H
#define UTLPFOR_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define UTL_API __attribute__((visibility("default")))
#else
#define UTL_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define UTL_OK 0
#define UTL_ERR_INVALID_BUFFER 1        /* ErrInvalidBuffer       utlpfor.go:71 */
#define UTL_ERR_POSITION_OUT_OF_RANGE 2 /* ErrPositionOutOfRange  utlpfor.go:74 */
#define UTL_ERR_INVALID_BLOCK_LENGTH 3  /* ErrInvalidBlockLength  utlpfor.go:77 */
#define UTL_ERR_INVALID_FLAGS 4         /* ErrInvalidFlags        utlpfor.go:80 */
#define UTL_ERR_UNSUPPORTED_TYPE 5      /* ErrUnsupportedType     utlpfor.go:86 */
#define UTL_ERR_NOT_IMPLEMENTED 6       /* ErrNotImplemented      utlpfor.go:83 */
#define UTL_ERR_OVERFLOW 7              /* *ErrOverflow{Position} utlpfor.go:108 */
#define UTL_ERR_COUNT_MISMATCH 8 /* batch: block count/length disagrees with the stream table */
#define UTL_ERR_CAPACITY 9       /* batch: output buffer too small */
#define UTL_ERR_TIMEOUT 10       /* device wait gave up (never expected) */
#define UTL_ERR_ARG 11           /* bad argument (NULL, size, alignment) */
#define UTL_ERR_CUDA 12          /* CUDA runtime error; see utl_last_cuda_error */
#define UTL_ERR_SCRATCH_LIMIT 13 /* batch too large for the built-in scratch of a _noalloc call */

/* ---- flags (utlpfor.go:24-68) ---- */
#define UTL_DELTA 1
#define UTL_NOFOR 2
#define UTL_NOPATCH 4
#define UTL_SPECIAL 8
#define UTL_APPEND 16
#define UTL_NOINPLACE 32

#define UTL_BLOCK_SIZE 128

/* ==================== per-call drop-in (host buffers) ==================== */

/* PackUint32 (pack.go:76).  Packs n (1..128) values into one block at dst.
 * Append and NoInPlace only affect where the Go caller places the block and
 * whether it may reuse values as scratch; the bytes are the same, and the
 * caller's values are never modified.  dst_cap >= utl_max_block_length32
 * (flag) always suffices; *out_len receives the block length. */
UTL_API int utl_pack_u32(uint8_t flag, const uint32_t *values, int n, uint8_t *dst,
                 size_t dst_cap, size_t *out_len);

/* UnpackUint32 (unpack.go:5).  values must hold 128 entries; *count values
 * are valid on success, *consumed is the block's byte length.  On
 * UTL_ERR_OVERFLOW *overflow_pos is ErrOverflow.Position. */
UTL_API int utl_unpack_u32(const uint8_t *src, size_t src_len, uint32_t *values,
                   int *count, size_t *consumed, int *overflow_pos);

/* GetUint32 (get.go:74). */
UTL_API int utl_get_u32(int pos, const uint8_t *src, size_t src_len, uint32_t *value,
                int *overflow_pos);

/* PackUint64 (uint64.go:279), UnpackUint64 (uint64.go:338),
 * GetUint64 (uint64.go:364).  dst_cap >= utl_max_block_length64(flag). */
UTL_API int utl_pack_u64(uint8_t flag, const uint64_t *values, int n, uint8_t *dst,
                 size_t dst_cap, size_t *out_len);
UTL_API int utl_unpack_u64(const uint8_t *src, size_t src_len, uint64_t *values,
                   int *count, size_t *consumed, int *overflow_pos);
UTL_API int utl_get_u64(int pos, const uint8_t *src, size_t src_len, uint64_t *value,
                int *overflow_pos);

/* BlockLength (block_length.go:8). */
UTL_API int utl_block_length(const uint8_t *src, size_t src_len, size_t *block_len);

/* Header (header.go:135); boolean outputs are 0/1. */
UTL_API int utl_header(const uint8_t *src, size_t src_len, int *count, int *bit_width,
               int *exc_count, int *has_delta, int *has_for, int *has_zigzag,
               int *has_special);

/* MaxBlockLength32 (scalar.go:336), MaxBlockLength64 (uint64.go:451). */
UTL_API int utl_max_block_length32(uint8_t flag);
UTL_API int utl_max_block_length64(uint8_t flag);

/* Compressor32/Compressor64 (compressor.go:16-107): a handle owning its own
 * CUDA stream and staging buffers; not safe for concurrent use, like the
 * reference's type.  is64 selects the 64-bit entry points below. */
typedef struct utl_codec utl_codec;
UTL_API int utl_codec_new(int is64, utl_codec **out);
UTL_API void utl_codec_free(utl_codec *c);
UTL_API int utl_codec_pack_u32(utl_codec *c, uint8_t flag, const uint32_t *values,
                       int n, uint8_t *dst, size_t dst_cap, size_t *out_len);
UTL_API int utl_codec_unpack_u32(utl_codec *c, const uint8_t *src, size_t src_len,
                         uint32_t *values, int *count, size_t *consumed,
                         int *overflow_pos);
UTL_API int utl_codec_get_u32(utl_codec *c, int pos, const uint8_t *src,
                      size_t src_len, uint32_t *value, int *overflow_pos);
UTL_API int utl_codec_pack_u64(utl_codec *c, uint8_t flag, const uint64_t *values,
                       int n, uint8_t *dst, size_t dst_cap, size_t *out_len);
UTL_API int utl_codec_unpack_u64(utl_codec *c, const uint8_t *src, size_t src_len,
                         uint64_t *values, int *count, size_t *consumed,
                         int *overflow_pos);
UTL_API int utl_codec_get_u64(utl_codec *c, int pos, const uint8_t *src,
                      size_t src_len, uint64_t *value, int *overflow_pos);

/* A pool of per-call contexts for servers that call from many host threads
 * at once (the reference's Compressor32/64 are not safe for concurrent use,
 * compressor.go:8,63, so a Go server keeps one per goroutine or a
 * sync.Pool of them; this is that pool on the C side).  Each of the
 * n_contexts contexts owns a CUDA stream and mapped pinned staging; a call
 * takes a free one, runs the per-call kernel on its stream and returns it,
 * so calls from different threads overlap on the GPU.  All calls are
 * thread-safe and behave exactly as utl_pack_u32 etc.  The pool belongs to
 * the device current at utl_pool_new; calls switch to it for their
 * duration.  No counterpart function in the reference. */
typedef struct utl_pool utl_pool;
UTL_API int utl_pool_new(int n_contexts, utl_pool **out);
UTL_API void utl_pool_free(utl_pool *p);
UTL_API int utl_pool_pack_u32(utl_pool *p, uint8_t flag, const uint32_t *values, int n, uint8_t *dst,
                              size_t dst_cap, size_t *out_len);
UTL_API int utl_pool_unpack_u32(utl_pool *p, const uint8_t *src, size_t src_len, uint32_t *values, int *count,
                                size_t *consumed, int *overflow_pos);
UTL_API int utl_pool_get_u32(utl_pool *p, int pos, const uint8_t *src, size_t src_len, uint32_t *value,
                             int *overflow_pos);
UTL_API int utl_pool_pack_u64(utl_pool *p, uint8_t flag, const uint64_t *values, int n, uint8_t *dst,
                              size_t dst_cap, size_t *out_len);
UTL_API int utl_pool_unpack_u64(utl_pool *p, const uint8_t *src, size_t src_len, uint64_t *values, int *count,
                                size_t *consumed, int *overflow_pos);
UTL_API int utl_pool_get_u64(utl_pool *p, int pos, const uint8_t *src, size_t src_len, uint64_t *value,
                             int *overflow_pos);

/* ==================== batched (device buffers) ==================== */
/* One launch packs, unpacks or queries the blocks of many streams of
 * uneven length.  The reference has no batched form; these replace the
 * caller's loop of Append / BlockLength-walk calls (example_test.go:171-186)
 * with one device-wide pass whose block offsets come from an exclusive scan
 * of the block lengths. */

/* Total blocks of a stream table given on the host (val_off: n_streams+1). */
UTL_API int64_t utl_count_blocks(const uint64_t *h_val_off, int n_streams);

/* block_start[s] = sum over t<s of ceil(n_t/128), s = 0..n_streams. */
UTL_API int utl_batch_plan(const uint64_t *d_val_off, int n_streams,
                   uint64_t *d_block_start, void *stream);

/* Device scratch the pack needs for n_blocks blocks (tile states of the
 * single-pass offset scan). */
UTL_API size_t utl_pack_scratch_bytes(int64_t n_blocks);

/* Pack every block of every stream.  d_block_off (n_blocks+1) receives each
 * block's byte offset in d_out and the total at [n_blocks];
 * d_stream_byte_off (n_streams+1, optional) each stream's start.
 * d_err (optional, one uint32, zero it first) receives UTL_ERR_CAPACITY
 * or UTL_ERR_TIMEOUT bits (1<<code) for the host to check after the stream
 * synchronizes.  out_cap >= n_blocks*utl_max_block_length32(flag) always
 * suffices. */
UTL_API int utl_pack_batch_u32(uint8_t flag, const uint32_t *d_values,
                       const uint64_t *d_val_off, const uint64_t *d_block_start,
                       int n_streams, int64_t n_blocks, uint8_t *d_out,
                       size_t out_cap, uint64_t *d_block_off,
                       uint64_t *d_stream_byte_off, void *d_scratch,
                       size_t scratch_bytes, uint32_t *d_err, void *stream);
UTL_API int utl_pack_batch_u64(uint8_t flag, const uint64_t *d_values,
                       const uint64_t *d_val_off, const uint64_t *d_block_start,
                       int n_streams, int64_t n_blocks, uint8_t *d_out,
                       size_t out_cap, uint64_t *d_block_off,
                       uint64_t *d_stream_byte_off, void *d_scratch,
                       size_t scratch_bytes, uint32_t *d_err, void *stream);

/* utl_pack_batch_u32 for callers that cannot allocate device memory while
 * they pack: latency-bound serving loops that cannot take the device-wide
 * synchronisation of cudaMalloc/cudaFree, and hosts that own a fixed device
 * memory budget and hand out no allocation rights (a Go process calling
 * through cgo that manages every device byte itself).  It has no counterpart in the reference (the Go library
 * never touches device memory).  Same arguments as utl_pack_batch_u32
 * without the scratch: the look-back tile states live in a 2 MiB array
 * built into the library, which every GPU that loads the library keeps
 * until the process exits.  Batches above
 * utl_pack_batch_u32_noalloc_max_blocks() blocks (about 4.2 million, i.e.
 * 5.4e8 values) are rejected with UTL_ERR_SCRATCH_LIMIT.  The first call
 * on a device (of this or any other batched entry point) sets the
 * kernels' launch attributes and queries their occupancy on that device,
 * and the first call of this entry point on a device looks up the array's
 * device address (with that device current); make that first call before
 * any stream capture.  The address lookup does not survive a
 * cudaDeviceReset of that device.  All calls on a device share the array,
 * so calls that overlap on the GPU (different streams, or threads without
 * ordering) race: serialise them.  Calls no cudaMalloc, cudaFree,
 * cudaHostAlloc or other allocating routine, on the first call too (the
 * CUDA runtime itself may load the library's kernels onto the device on
 * first use). */
UTL_API int utl_pack_batch_u32_noalloc(uint8_t flag, const uint32_t *d_values,
                               const uint64_t *d_val_off,
                               const uint64_t *d_block_start, int n_streams,
                               int64_t n_blocks, uint8_t *d_out,
                               size_t out_cap, uint64_t *d_block_off,
                               uint64_t *d_stream_byte_off, uint32_t *d_err,
                               void *stream);
UTL_API int64_t utl_pack_batch_u32_noalloc_max_blocks(void);

/* Unpack every block.  Block b is d_packed[d_block_off[b] .. d_block_off[b+1])
 * and must decode to the stream table's count, consuming exactly its
 * length.  d_block_status (optional, n_blocks int32) receives per block
 * code | (overflow_pos << 8); d_err (optional) gets 1<<code for every code
 * seen.  Blocks that fail write no values. */
UTL_API int utl_unpack_batch_u32(const uint8_t *d_packed, size_t packed_len,
                         const uint64_t *d_block_off, const uint64_t *d_val_off,
                         const uint64_t *d_block_start, int n_streams,
                         int64_t n_blocks, uint32_t *d_values,
                         int32_t *d_block_status, uint32_t *d_err,
                         void *stream);
UTL_API int utl_unpack_batch_u64(const uint8_t *d_packed, size_t packed_len,
                         const uint64_t *d_block_off, const uint64_t *d_val_off,
                         const uint64_t *d_block_start, int n_streams,
                         int64_t n_blocks, uint64_t *d_values,
                         int32_t *d_block_status, uint32_t *d_err,
                         void *stream);

/* GetUint32/GetUint64 for n_queries (stream, position-in-stream) pairs.
 * d_status (optional) as for unpack, per query. */
UTL_API int utl_get_batch_u32(const uint8_t *d_packed, size_t packed_len,
                      const uint64_t *d_block_off, const uint64_t *d_val_off,
                      const uint64_t *d_block_start, int n_streams,
                      const uint32_t *d_q_stream, const uint64_t *d_q_pos,
                      int64_t n_queries, uint32_t *d_out, int32_t *d_status,
                      uint32_t *d_err, void *stream);
UTL_API int utl_get_batch_u64(const uint8_t *d_packed, size_t packed_len,
                      const uint64_t *d_block_off, const uint64_t *d_val_off,
                      const uint64_t *d_block_start, int n_streams,
                      const uint32_t *d_q_stream, const uint64_t *d_q_pos,
                      int64_t n_queries, uint64_t *d_out, int32_t *d_status,
                      uint32_t *d_err, void *stream);

/* ==================== batched (host buffers) ==================== */
/* Same batches end to end from host memory: copies in, batched passes,
 * copies out, on the calling thread's context.  Large batches run in
 * pieces whose copies in, kernels and copies out overlap
 * (UTL_KNOB_HOST_PIPELINE).  Pinned host buffers give full PCIe bandwidth
 * and the overlap; pageable ones work at the speed of CUDA's staged copies.
 * *out_len receives the packed size; h_block_off (n_blocks+1) and
 * h_stream_byte_off (n_streams+1, optional) as above. */
UTL_API int utl_pack_streams_u32(uint8_t flag, const uint32_t *h_values,
                         const uint64_t *h_val_off, int n_streams,
                         uint8_t *h_out, size_t out_cap, uint64_t *h_block_off,
                         uint64_t *h_stream_byte_off, size_t *out_len);
UTL_API int utl_unpack_streams_u32(const uint8_t *h_packed, size_t packed_len,
                           const uint64_t *h_block_off,
                           const uint64_t *h_val_off, int n_streams,
                           uint32_t *h_values);
UTL_API int utl_pack_streams_u64(uint8_t flag, const uint64_t *h_values,
                         const uint64_t *h_val_off, int n_streams,
                         uint8_t *h_out, size_t out_cap, uint64_t *h_block_off,
                         uint64_t *h_stream_byte_off, size_t *out_len);
UTL_API int utl_unpack_streams_u64(const uint8_t *h_packed, size_t packed_len,
                           const uint64_t *h_block_off,
                           const uint64_t *h_val_off, int n_streams,
                           uint64_t *h_values);

/* ==================== stream indexer ==================== */
/* Block offsets of a packed stream that carries no index: the walk a
 * caller does with BlockLength block after block from offset 0
 * (block_length.go:8-65, caller pattern example_test.go:171-186), done on
 * the device.  d_packed[0, packed_len) holds whole blocks back to back;
 * d_block_off receives n_blocks + 1 offsets (capacity max_blocks + 1, the
 * last entry is packed_len).  Synchronizes `stream`.  Returns UTL_OK, the
 * BlockLength error of the first bad block (UTL_ERR_INVALID_BUFFER also
 * when a block runs past the end) with *n_blocks = that block's index, or
 * UTL_ERR_CAPACITY with *n_blocks = the block count. */
UTL_API int utl_index_stream(const uint8_t *d_packed, size_t packed_len,
                             uint64_t *d_block_off, int64_t max_blocks,
                             int64_t *n_blocks, void *stream);

/* ==================== tuning ==================== */
/* Process-wide knobs of the batched kernels, set by the autotuner
 * (utlpfor_b200.tune); no counterpart in the reference.  Defaults are
 * sound on any B200.
 *   UTL_KNOB_UNPACK_SCHEDULE: the uint32 unpack kernel.  0 = one CTA per
 *     32 blocks; 2 = persistent warps with the next group's bytes in
 *     flight (cp.async double buffer), staging up to 528 bytes a block;
 *     3 = the same staging up to 264 bytes a block (more warps resident);
 *     1 = 3 or 2 by the batch's mean block length, decided on the device;
 *     5 = persistent warps staging each group of 8 blocks with one TMA bulk
 *     copy, three groups in flight, up to 264 bytes a block; 6 = the same
 *     with two groups of up to 528 bytes a block in flight; 4 = 5 or 6 by
 *     the batch's mean block length, decided on the device; 7 = 5 with a
 *     register fast path for blocks of at most 16 exceptions (positions
 *     turned into a bitmask, high bits ORed by rank, no shared-memory round
 *     trip of the values); 9 = one thread per block (tiles of 32 blocks per
 *     warp, rows written out through a shared-memory chunk), the quad decoder
 *     for blocks it does not take (bitmap exceptions, plain delta, partial,
 *     corrupt or oversized blocks); 10 = 9 with the next tile's bytes in
 *     flight in a second, smaller buffer; 8 = 9 for batches of at most 240
 *     bytes a block on average, else 2, decided on the device (the default).
 *   UTL_KNOB_PACK_CTAS_PER_SM: cap on resident pack CTAs per SM (0 = the
 *     occupancy maximum).
 *   UTL_KNOB_PACK_SCHEDULE: uint32 pack kernel, 0 = four threads per block
 *     (CTA tiles), 1 = one thread per block (independent warp tiles of 32
 *     blocks), 2 = a lane pair per block (independent warp tiles of 16
 *     blocks, half the shared memory per warp, more warps per SM).
 *   UTL_KNOB_PACK_WINDOW: the tile image of the one-thread and lane-pair
 *     packs, 0 = by the block density of the previous pack on this device
 *     that may allocate (a hint read without waiting), 1 = the large window,
 *     2 = the small window (for batches of at most about 144 bytes a block).
 *     Outputs are the same for every value.
 *   UTL_KNOB_UNPACK_CTAS_PER_SM: cap on resident CTAs (4 warps each) per SM
 *     of the persistent unpack kernels, schedules 1-6 (0 = the occupancy
 *     maximum).
 *   UTL_KNOB_UNPACK64_SCHEDULE: the uint64 unpack kernel, 0 = a warp per
 *     block; 1 = an octet of lanes per block (one quad per
 *     uint32 sub-block, both decoded at once), 4 blocks per warp staged by
 *     TMA bulk copies, two groups in flight; 2 = the same with three;
 *     3 = a quad of lanes per block (the two sub-blocks of a pair one after
 *     the other), 8 blocks per warp, cp.async double buffer sized by the
 *     batch's mean block length; 4 / 5 = the same with the small / large
 *     buffer always; 6 = the large budget in a single buffer per warp
 *     (twice the resident warps); 7 = as 3 with the large budget single
 *     buffered (the default).
 *   UTL_KNOB_HOST_PIPELINE: the host-buffer batch calls, 0 = one pass
 *     (all copies in, kernels, all copies out); 1 = batches of 64 MiB of
 *     values or more are cut at block boundaries into pieces of
 *     max(16 MiB, batch/32) whose copies in, kernels and copies out overlap
 *     (the default); 2 = every batch in eighths (for tests).  Outputs are
 *     the same in every mode.
 * Two knobs exist for tests of the pack's bounded waits only:
 *   UTL_KNOB_SPIN_LIMIT: polls (64 ns sleep each) a waiting tile makes
 *     before it gives up, records UTL_ERR_TIMEOUT in d_err and carries on
 *     with a zero contribution (0 = the default, 2^22).
 *   UTL_KNOB_KEEP_SCRATCH: 1 = the batched pack does not clear the caller's
 *     scratch before its launch, so a test can preset the tile states
 *     (for instance a work counter past tile 0, whose tile then never
 *     publishes).  Output is undefined unless the scratch is zeroed. */
#define UTL_KNOB_UNPACK_SCHEDULE 0
#define UTL_KNOB_PACK_CTAS_PER_SM 1
#define UTL_KNOB_PACK_SCHEDULE 2
#define UTL_KNOB_HOST_PIPELINE 3
#define UTL_KNOB_SPIN_LIMIT 4
#define UTL_KNOB_KEEP_SCRATCH 5
#define UTL_KNOB_PACK_WINDOW 6
#define UTL_KNOB_UNPACK_CTAS_PER_SM 7
#define UTL_KNOB_UNPACK64_SCHEDULE 8
UTL_API int utl_set_knob(int knob, int value);
UTL_API int utl_get_knob(int knob);

/* ==================== diagnostics ==================== */
/* Number of this library's kernels launched so far in this process. */
UTL_API uint64_t utl_launch_count(void);
/* Last CUDA error seen by this thread's calls (cudaError_t value). */
UTL_API int utl_last_cuda_error(void);
/* Library version string. */
UTL_API const char *utl_version(void);

#ifdef __cplusplus
}
#endif
#endif /* UTLPFOR_H */
