// utl_launch.h -- internal interface between the C ABI and the kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace utl {

struct PackArgs {
  const void* values;
  const uint64_t* val_off;
  const uint64_t* block_start;
  int n_streams;
  int flag;
  int64_t n_blocks;
  int64_t n_tiles;
  uint8_t* out;
  uint64_t out_cap;
  uint64_t* block_off;
  unsigned long long* counter;  // tile work counter (scratch)
  uint64_t* tile_status;        // look-back states (scratch)
  uint32_t* err;
  uint64_t* stats = nullptr;    // set by the launcher: packed bytes and blocks of the batch
  uint32_t spin_limit = 1u << 22;  // polls of each bounded wait (UTL_KNOB_SPIN_LIMIT)
};

struct UnpackArgs {
  const uint8_t* packed;
  uint64_t packed_len;
  const uint64_t* block_off;
  const uint64_t* val_off;
  const uint64_t* block_start;
  int n_streams;
  int64_t n_blocks;
  void* values;
  int32_t* block_status;
  uint32_t* err;
  uint32_t spin_limit = 1u << 22;  // polls of each bounded wait (UTL_KNOB_SPIN_LIMIT)
  uint64_t lane_mean = 0;  // > 0: the small-staging pipe instance leaves batches of at most this mean block length
                           // to the thread-per-block kernel launched beside it
};

struct GetArgs {
  const uint8_t* packed;
  uint64_t packed_len;
  const uint64_t* block_off;
  const uint64_t* val_off;
  const uint64_t* block_start;
  int n_streams;
  const uint32_t* q_stream;
  const uint64_t* q_pos;
  int64_t n_queries;
  void* out;
  int32_t* status;
  uint32_t* err;
};

// Result record of a per-call kernel, written to mapped host memory.
struct PlainResult {
  int32_t status;
  int32_t count;
  int64_t len;
  int32_t ovf;
  int32_t pad;
  uint64_t value;
};

void note_launch(int n);

// The batched pack behind utl_pack_batch_u32/u64 (argument checks, scratch
// clearing, launch); may_alloc as for launch::pack.  Returns a UTL_* status.
int pack_batch_device(bool u64, bool may_alloc, uint8_t flag, const void* d_values, const uint64_t* d_val_off,
                      const uint64_t* d_block_start, int n_streams, int64_t n_blocks, uint8_t* d_out, size_t out_cap,
                      uint64_t* d_block_off, uint64_t* d_sbo, void* d_scratch, size_t scratch_bytes, uint32_t* d_err,
                      cudaStream_t st);

namespace launch {
size_t pack_smem(bool u64);
size_t unpack_smem(bool u64);
int64_t tiles_for(int64_t n_blocks);
// scratch layout of the pack: [0,8) work counter, [16, 16+8*tiles) tile states
inline size_t pack_scratch_bytes(int64_t n_blocks) { return 16 + 8 * (size_t)tiles_for(n_blocks); }
cudaError_t plan(const uint64_t* val_off, int n, uint64_t* bstart, cudaStream_t st);
cudaError_t stream_offsets(const uint64_t* block_off, const uint64_t* bstart, int n, uint64_t* sbo, cudaStream_t st);
// may_alloc false: the launch makes no allocation of any kind (the uint32
// lane pack then skips its mapped-memory window hint).
cudaError_t pack(bool u64, const PackArgs& a, cudaStream_t st, bool may_alloc);
cudaError_t unpack(bool u64, const UnpackArgs& a, cudaStream_t st);
cudaError_t get(bool u64, const GetArgs& a, cudaStream_t st);
cudaError_t plain_pack(bool u64, int flag, const void* vals, int n, uint8_t* out, PlainResult* res, cudaStream_t st);
cudaError_t plain_unpack(bool u64, const uint8_t* src, int64_t staged, int64_t avail, uint8_t* tmp, void* vals,
                         PlainResult* res, cudaStream_t st);
cudaError_t plain_get(bool u64, int pos, const uint8_t* src, int64_t staged, int64_t avail, uint8_t* tmp,
                      PlainResult* res, cudaStream_t st);
size_t index_scratch_bytes(uint64_t len);
int index_stream(const uint8_t* p, uint64_t len, uint64_t* block_off, int64_t max_blocks, int64_t* n_blocks,
                 void* scratch, cudaStream_t st, cudaError_t* cerr);
int set_knob(int knob, int value);
int get_knob(int knob);
uint32_t spin_limit();     // UTL_KNOB_SPIN_LIMIT as a poll count
bool keep_scratch();       // UTL_KNOB_KEEP_SCRATCH
}  // namespace launch
}  // namespace utl
