// utl_noalloc.cu -- batched pack that allocates nothing.
//
// Some callers cannot allocate device memory when they pack: serving loops
// whose latency budget cannot absorb the device-wide synchronisation a
// cudaMalloc/cudaFree may cause, and hosts that hand this library a fixed
// memory budget up front (a Go process calling through cgo that manages
// every device byte itself).
// utl_pack_batch_u32_noalloc serves them: the caller passes only inputs and
// outputs, and the look-back tile states live in the fixed-size array
// below instead of caller-provided or library-allocated scratch.
#include <cuda_runtime.h>
#include <stdint.h>

#include <mutex>

#include "../../include/utlpfor.h"
#include "utl_launch.h"

namespace utl {

// Scratch of the no-allocation pack (2 MiB): the tile work counter and one
// 8-byte look-back state per tile, laid out as utl_pack_scratch_bytes
// describes.  Every GPU that loads this library holds these bytes until
// the process exits.  In host code the name is only a host-side stand-in
// for the device array; its device address comes from cudaGetSymbolAddress.
constexpr size_t kNoAllocScratchBytes = (size_t)2 << 20;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

namespace {
constexpr int kMaxDevices = 64;
std::mutex g_mu;
// Device address of g_noalloc_scratch, looked up once per device.  A
// cudaDeviceReset on that device unloads this library's module there, so
// the cached address does not survive it: callers that reset a device must
// not call this entry point on it afterwards.
void* g_addr[kMaxDevices];
}  // namespace

}  // namespace utl

using namespace utl;

extern "C" int64_t utl_pack_batch_u32_noalloc_max_blocks(void) {
  // largest n with utl_pack_scratch_bytes(n) <= kNoAllocScratchBytes
  int64_t lo = 0, hi = (int64_t)kNoAllocScratchBytes * 16;
  while (lo < hi) {
    const int64_t mid = (lo + hi + 1) / 2;
    if (utl_pack_scratch_bytes(mid) <= kNoAllocScratchBytes) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

extern "C" int utl_pack_batch_u32_noalloc(uint8_t flag, const uint32_t* d_values, const uint64_t* d_val_off,
                                          const uint64_t* d_block_start, int n_streams, int64_t n_blocks,
                                          uint8_t* d_out, size_t out_cap, uint64_t* d_block_off,
                                          uint64_t* d_stream_byte_off, uint32_t* d_err, void* stream) {
  if (n_blocks < 0 || n_streams < 0) return UTL_ERR_ARG;
  if (n_blocks > utl_pack_batch_u32_noalloc_max_blocks()) return UTL_ERR_SCRATCH_LIMIT;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return UTL_ERR_CUDA;
  void* scratch = nullptr;
  {
    // once per device, with that device current: the symbol's device address
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
      void* p = nullptr;
      if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) return UTL_ERR_CUDA;
      g_addr[dev] = p;
    }
    scratch = g_addr[dev];
  }
  // The array keeps the previous call's contents; the pack clears the
  // counter and tile states it uses on `stream` before its kernel runs.
  // may_alloc = false: the launch takes no allocating step at all (the
  // uint32 pack's mapped-memory window hint is skipped).
  return pack_batch_device(false, false, flag, d_values, d_val_off, d_block_start, n_streams, n_blocks, d_out, out_cap,
                           d_block_off, d_stream_byte_off, scratch, kNoAllocScratchBytes, d_err, (cudaStream_t)stream);
}
