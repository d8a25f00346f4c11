// utl_index.cu -- device stream indexer: the block offsets of a packed
// stream that carries no index, i.e. what a caller gets by walking the
// stream with BlockLength block after block (block_length.go:8-65, caller
// pattern example_test.go:171-186).
//
// The walk is a chain: each block's start follows from the previous one's
// header.  It is done speculatively in parallel.  The stream is cut into
// partitions of kPart bytes; one thread per partition finds a position
// where kSync consecutive headers parse and stay inside the stream (a true
// block start lies within the first kMaxBlock bytes of every partition),
// walks from there to the partition's end and records where its chain
// leaves the partition.  A second pass checks, in parallel, that the chain
// entering each partition (the previous partition's exit) meets that
// partition's chain -- two chains that share one position share all later
// ones -- and derives the partition's true block count.  Partitions whose
// check fails (a false start, or a stream error) are walked again one after
// the other from the true entry, which also finds the first bad block.  A
// scan of the counts places each partition's blocks, and a last pass walks
// every partition from its true entry and writes the offsets.
#include <cuda_runtime.h>
#include <stdint.h>

#include "utl_launch.h"

namespace utl {
namespace index {

// Status codes of include/utlpfor.h and the block size (utlpfor.go).
constexpr int kOK = 0;
constexpr int kErrInvalidBuffer = 1;
constexpr int kErrInvalidBlockLength = 3;
constexpr int kErrInvalidFlags = 4;
constexpr int kBlock = 128;

constexpr int64_t kPart = 8192;      // partition bytes (>= kMaxBlock)
constexpr int64_t kMaxBlock = 2048;  // every block is at most MaxBlockLength64(0) = 2038 bytes
constexpr int kSync = 6;             // headers that must parse in a row to accept a start
constexpr int kThreads = 256;
constexpr int kErrCapacity = 9;  // UTL_ERR_CAPACITY

__device__ __forceinline__ uint32_t byte_at(const uint8_t* p, uint64_t len, uint64_t i) {
  return i < len ? (uint32_t)p[i] : 0u;
}

// BlockLength of the block at byte off (block_length.go:8-65); on success
// also requires the block to end inside the stream, as the caller's next
// Unpack would (ErrInvalidBuffer otherwise).  Returns a status code.
__device__ int block_length_at(const uint8_t* p, uint64_t len, uint64_t off, uint64_t* out) {
  if (off + 4 > len) return kErrInvalidBuffer;
  const uint32_t h = byte_at(p, len, off) | (byte_at(p, len, off + 1) << 8) | (byte_at(p, len, off + 2) << 16) |
                     (byte_at(p, len, off + 3) << 24);
  const int count = (int)(h & 0xFFu), bw = (int)((h >> 8) & 0x1Fu) * 4, type = (int)((h >> 13) & 3u);
  const int forw = (int)((h >> 15) & 3u), exc = (int)(h >> 24);
  if (count > kBlock) return kErrInvalidBlockLength;
  if (bw > 32) return kErrInvalidBuffer;
  const bool combine = (h & (1u << 19)) && type == 3;
  if (type == 3) {
    if (h & ((1u << 18) | (1u << 20))) return kErrInvalidFlags;
  } else if (h & ((1u << 18) | (1u << 19) | (1u << 20))) {
    return kErrInvalidFlags;
  }
  const int forb = (type == 3 && !combine && forw == 3) ? 8 : ((1 << forw) >> 1);
  const uint64_t p_off = 4 + (exc ? 2 : 0) + forb + (combine ? 2 : 0);
  uint64_t b1 = p_off + ((uint64_t)bw << 4);
  if (exc) {
    if (off + 6 > len) return kErrInvalidBuffer;
    b1 += (uint64_t)(exc <= 16 ? exc : 16) + (byte_at(p, len, off + 4) | (byte_at(p, len, off + 5) << 8));
  }
  if (combine) {
    if (off + p_off > len) return kErrInvalidBuffer;
    b1 += byte_at(p, len, off + p_off - 2) | (byte_at(p, len, off + p_off - 1) << 8);
  }
  if (off + b1 > len) return kErrInvalidBuffer;
  *out = b1;
  return kOK;
}

struct Part {
  int64_t entry;   // first block start of the thread's chain (-1: none found)
  int64_t exit;    // where the chain leaves the partition (-1: it hit an error)
  int64_t count;   // blocks of the chain that start in the partition
  int64_t tcount;  // true block count (after the check)
  int32_t ok;      // the partition's chain is the stream's chain
  int32_t pad;
};

// Walk from `pos` while the block start is below `end`; counts the blocks.
// Returns the first start at or past `end`, or -1 on an error (err/epos set).
__device__ int64_t walk(const uint8_t* p, uint64_t len, int64_t pos, int64_t end, int64_t* count, int* err,
                        int64_t* epos) {
  int64_t c = 0;
  while (pos < end && (uint64_t)pos < len) {
    uint64_t L;
    const int st = block_length_at(p, len, (uint64_t)pos, &L);
    if (st != kOK) {
      *err = st;
      *epos = pos;
      *count = c;
      return -1;
    }
    pos += (int64_t)L;
    c++;
  }
  *count = c;
  return pos;
}

// Walk the chains from x (the stream's) and y (a partition's) forward, the
// one behind each time, until they meet before `end`.  On a meeting
// returns true with hx/hy = blocks each chain took to get there.
__device__ bool meet(const uint8_t* p, uint64_t len, int64_t x, int64_t y, int64_t end, int64_t* hx, int64_t* hy) {
  int64_t cx = 0, cy = 0;
  while (x != y) {
    if (x >= end || y >= end) return false;
    uint64_t L;
    if (x < y) {
      if (block_length_at(p, len, (uint64_t)x, &L) != kOK) return false;
      x += (int64_t)L;
      cx++;
    } else {
      if (block_length_at(p, len, (uint64_t)y, &L) != kOK) return false;
      y += (int64_t)L;
      cy++;
    }
  }
  *hx = cx;
  *hy = cy;
  return x < end;
}

__global__ void __launch_bounds__(kThreads) speculate_kernel(const uint8_t* p, uint64_t len, int64_t n_parts,
                                                             Part* parts) {
  const int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= n_parts) return;
  const int64_t start = k * kPart, end = min((int64_t)len, start + kPart);
  int64_t entry = -1;
  if (k == 0) {
    entry = 0;
  } else {
    const int64_t stop = min(end, start + kMaxBlock);
    for (int64_t x = start; x < stop && entry < 0; x++) {
      int64_t q = x;
      int good = 0;
      for (; good < kSync && (uint64_t)q < len; good++) {
        uint64_t L;
        // a start is accepted only on blocks a packer can emit (no block is
        // longer than kMaxBlock); the walks keep BlockLength's own rules
        if (block_length_at(p, len, (uint64_t)q, &L) != kOK || L > (uint64_t)kMaxBlock) break;
        q += (int64_t)L;
      }
      if (good == kSync || (uint64_t)q == len) entry = x;
    }
  }
  Part r;
  r.entry = entry;
  r.count = 0;
  r.exit = -1;
  r.tcount = 0;
  r.ok = 0;
  r.pad = 0;
  if (entry >= 0) {
    int err = 0;
    int64_t epos = 0;
    r.exit = walk(p, len, entry, end, &r.count, &err, &epos);
  }
  parts[k] = r;
}

// Partition k's chain is the stream's chain when the chain entering it (the
// previous partition's exit, assumed true) meets it; the true count then
// differs from the chain's count by the blocks between the two positions.
__global__ void __launch_bounds__(kThreads) check_kernel(const uint8_t* p, uint64_t len, int64_t n_parts,
                                                         Part* parts, int64_t* first_bad) {
  const int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= n_parts) return;
  Part& r = parts[k];
  if (k == 0) {
    r.ok = r.exit >= 0;
    r.tcount = r.count;
  } else {
    const int64_t x = parts[k - 1].exit, y = r.entry;
    const int64_t end = min((int64_t)len, k * kPart + kPart);
    bool ok = false;
    int64_t tc = 0;
    if (x >= 0 && r.exit >= 0) {
      if (x >= end) {  // only at the stream's end (partitions are longer than any block)
        ok = true;
        tc = 0;
      } else if (y >= 0) {
        int64_t hx, hy;
        if (meet(p, len, x, y, end, &hx, &hy)) {  // the chains share every block from the meeting on
          ok = true;
          tc = hx + r.count - hy;
        }
      }
    }
    r.ok = ok;
    r.tcount = tc;
  }
  if (!r.ok) atomicMin((unsigned long long*)first_bad, (unsigned long long)k);
}

// Walk one partition after another from the first unchecked one, whose
// entry is true, until a partition's own chain meets the true chain again
// (it and the partitions after it are then right) or the stream ends or
// fails.  err_info: code, partition, blocks of that partition before the
// bad block.
__global__ void fixup_kernel(const uint8_t* p, uint64_t len, int64_t n_parts, Part* parts, int64_t k0,
                             int64_t* err_info) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  int64_t k = k0;
  int64_t x = k == 0 ? 0 : parts[k - 1].exit;
  while (k < n_parts) {
    const int64_t end = min((int64_t)len, k * kPart + kPart);
    int64_t c;
    int err = 0;
    int64_t epos = 0;
    const int64_t e = walk(p, len, x, end, &c, &err, &epos);
    Part& r = parts[k];
    if (e < 0) {
      err_info[0] = err;
      err_info[1] = k;
      err_info[2] = c;
      r.tcount = c;
      r.exit = -1;
      for (int64_t j = k; j < n_parts; j++) parts[j].ok = 1;  // nothing past the error is used
      return;
    }
    r.tcount = c;
    r.exit = e;
    r.ok = 1;
    k++;
    if (k >= n_parts) return;
    Part& q = parts[k];
    const int64_t nend = min((int64_t)len, k * kPart + kPart);
    if (e >= nend) {
      q.tcount = 0;
      q.exit = e;
      q.ok = 1;
      return;
    }
    if (q.entry >= 0 && q.exit >= 0) {
      int64_t hx, hy;
      if (meet(p, len, e, q.entry, nend, &hx, &hy)) {
        q.tcount = hx + q.count - hy;
        q.ok = 1;
        return;
      }
    }
    x = e;
  }
}

__global__ void __launch_bounds__(kThreads) unchecked_kernel(int64_t n_parts, const Part* parts, int64_t* first_bad) {
  const int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k < n_parts && !parts[k].ok) atomicMin((unsigned long long*)first_bad, (unsigned long long)k);
}

// Exclusive scan of the true counts into base[] (one CTA); base[n] = total.
__global__ void __launch_bounds__(1024) scan_kernel(int64_t n_parts, const Part* parts, int64_t* base) {
  __shared__ int64_t sums[1024];
  const int t = threadIdx.x;
  const int64_t per = (n_parts + 1023) / 1024;
  const int64_t lo = min(n_parts, per * t), hi = min(n_parts, lo + per);
  int64_t s = 0;
  for (int64_t k = lo; k < hi; k++) s += parts[k].tcount;
  sums[t] = s;
  __syncthreads();
  for (int d = 1; d < 1024; d <<= 1) {
    const int64_t v = t >= d ? sums[t - d] : 0;
    __syncthreads();
    sums[t] += v;
    __syncthreads();
  }
  int64_t run = sums[t] - s;
  for (int64_t k = lo; k < hi; k++) {
    base[k] = run;
    run += parts[k].tcount;
  }
  if (t == 1023) base[n_parts] = sums[1023];
}

// Each partition's true blocks, from its true entry: their offsets.
__global__ void __launch_bounds__(kThreads) write_kernel(const uint8_t* p, uint64_t len, int64_t n_parts,
                                                         const Part* parts, const int64_t* base, uint64_t* block_off) {
  const int64_t k = (int64_t)blockIdx.x * kThreads + threadIdx.x;
  if (k >= n_parts) return;
  const int64_t end = min((int64_t)len, k * kPart + kPart);
  int64_t pos = k == 0 ? 0 : parts[k - 1].exit;
  int64_t i = base[k];
  const int64_t stop = base[k + 1];
  while (pos < end && i < stop) {
    uint64_t L;
    if (block_length_at(p, len, (uint64_t)pos, &L) != kOK) break;
    block_off[i++] = (uint64_t)pos;
    pos += (int64_t)L;
  }
  if (k == n_parts - 1) block_off[stop] = len;
}

}  // namespace index

namespace launch {

size_t index_scratch_bytes(uint64_t len) {
  const int64_t n_parts = (int64_t)((len + index::kPart - 1) / index::kPart);
  return (size_t)n_parts * sizeof(index::Part) + (size_t)(n_parts + 1) * 8 + 64;
}

// Block offsets of the packed stream p[0, len) into block_off (capacity
// max_blocks + 1).  Synchronizes st.  Returns a status; *n_blocks is the
// block count, or on an error the index of the bad block.
int index_stream(const uint8_t* p, uint64_t len, uint64_t* block_off, int64_t max_blocks, int64_t* n_blocks,
                 void* scratch, cudaStream_t st, cudaError_t* cerr) {
  using namespace index;
  *n_blocks = 0;
  *cerr = cudaSuccess;
  const int64_t n_parts = (int64_t)((len + kPart - 1) / kPart);
  int64_t* ctl = (int64_t*)scratch;  // first_bad, err code, err partition, err count
  Part* parts = (Part*)((uint8_t*)scratch + 64);
  int64_t* base = (int64_t*)(parts + n_parts);
  if (len == 0) {
    if (max_blocks < 0) return kErrCapacity;
    *cerr = cudaMemsetAsync(block_off, 0, 8, st);
    if (*cerr == cudaSuccess) *cerr = cudaStreamSynchronize(st);
    return *cerr == cudaSuccess ? kOK : -1;
  }
  const int64_t init[4] = {INT64_MAX, 0, -1, 0};
  if ((*cerr = cudaMemcpyAsync(ctl, init, sizeof(init), cudaMemcpyHostToDevice, st)) != cudaSuccess) return -1;
  const unsigned grid = (unsigned)((n_parts + kThreads - 1) / kThreads);
  speculate_kernel<<<grid, kThreads, 0, st>>>(p, len, n_parts, parts);
  check_kernel<<<grid, kThreads, 0, st>>>(p, len, n_parts, parts, ctl);
  note_launch(2);
  for (;;) {
    int64_t h[4];
    if ((*cerr = cudaMemcpyAsync(h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return -1;
    if ((*cerr = cudaStreamSynchronize(st)) != cudaSuccess) return -1;
    if (h[1] != 0 || h[0] == INT64_MAX) break;  // an error found, or every partition checked
    const int64_t reset = INT64_MAX;
    if ((*cerr = cudaMemcpyAsync(ctl, &reset, 8, cudaMemcpyHostToDevice, st)) != cudaSuccess) return -1;
    fixup_kernel<<<1, 32, 0, st>>>(p, len, n_parts, parts, h[0], ctl + 1);
    unchecked_kernel<<<grid, kThreads, 0, st>>>(n_parts, parts, ctl);
    note_launch(2);
  }
  scan_kernel<<<1, 1024, 0, st>>>(n_parts, parts, base);
  note_launch(1);
  int64_t h[4], total = 0;
  if ((*cerr = cudaMemcpyAsync(h, ctl, sizeof(h), cudaMemcpyDeviceToHost, st)) != cudaSuccess) return -1;
  if ((*cerr = cudaMemcpyAsync(&total, base + n_parts, 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return -1;
  if ((*cerr = cudaStreamSynchronize(st)) != cudaSuccess) return -1;
  if (h[1] != 0) {  // the walk failed at block base[partition] + count
    int64_t b = 0;
    if ((*cerr = cudaMemcpyAsync(&b, base + h[2], 8, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return -1;
    if ((*cerr = cudaStreamSynchronize(st)) != cudaSuccess) return -1;
    *n_blocks = b + h[3];
    return (int)h[1];
  }
  *n_blocks = total;
  if (total > max_blocks) return kErrCapacity;
  write_kernel<<<grid, kThreads, 0, st>>>(p, len, n_parts, parts, base, block_off);
  note_launch(1);
  if ((*cerr = cudaGetLastError()) != cudaSuccess) return -1;
  if ((*cerr = cudaStreamSynchronize(st)) != cudaSuccess) return -1;
  return kOK;
}

}  // namespace launch
}  // namespace utl
