// utl_capi.cu -- C ABI of the UTL-PFOR codec (declared in include/utlpfor.h).
//
// Per-call entry points run one single-warp kernel per call.  Inputs are
// copied into a mapped, pinned staging buffer that the kernel reads over
// PCIe, and the kernel writes its result record and output back into the
// same buffer, so a call costs one launch and one stream synchronize.
// Each host thread owns one context (stream + staging) per device; a
// utl_codec handle owns its own.
#include <cuda_runtime.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <atomic>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/utlpfor.h"
#include "utl_launch.h"
#include "utl_pieces.h"

namespace utl {

using pieces::Piece;
using pieces::cut_pieces;

static std::atomic<uint64_t> g_launches{0};
void note_launch(int n) { g_launches.fetch_add((uint64_t)n, std::memory_order_relaxed); }

static thread_local int t_last_cuda = 0;

static int cuda_fail(cudaError_t e) {
  t_last_cuda = (int)e;
  return UTL_ERR_CUDA;
}
#define UTL_CUDA(x)                          \
  do {                                       \
    cudaError_t _e = (x);                    \
    if (_e != cudaSuccess) return cuda_fail(_e); \
  } while (0)

static inline uint32_t ld16(const uint8_t* p) { return (uint32_t)p[0] | ((uint32_t)p[1] << 8); }
static inline uint32_t ld32(const uint8_t* p) {
  return (uint32_t)p[0] | ((uint32_t)p[1] << 8) | ((uint32_t)p[2] << 16) | ((uint32_t)p[3] << 24);
}

// Staging layout of a context's mapped buffer.
constexpr size_t kStageIn = 144 * 1024;  // covers the largest span a corrupt block can name
constexpr size_t kStageOut = 4096;       // one packed block (<= 2038 B) or 128 values
constexpr size_t kStageRes = 256;
constexpr size_t kStageBytes = kStageIn + kStageOut + kStageRes;

struct Grow {
  void* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(n, (size_t)256);
    cudaError_t e = cudaMalloc(&p, want);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFree(p);
    p = nullptr;
    cap = 0;
  }
};

// Pinned host memory that grows on demand.
struct HostGrow {
  uint8_t* p = nullptr;
  size_t cap = 0;
  cudaError_t ensure(size_t n) {
    if (n <= cap) return cudaSuccess;
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
    size_t want = std::max(n, (size_t)4096);
    cudaError_t e = cudaHostAlloc((void**)&p, want, cudaHostAllocDefault);
    if (e == cudaSuccess) cap = want;
    return e;
  }
  void release() {
    if (p) cudaFreeHost(p);
    p = nullptr;
    cap = 0;
  }
};

// Most pieces one host-buffer batch is cut into (one event pair each).
constexpr int kMaxPieces = 64;

struct Ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  uint8_t* h_stage = nullptr;  // mapped pinned
  uint8_t* d_stage = nullptr;  // device alias of h_stage
  uint8_t* d_tmp = nullptr;    // device copy of staged input
  // buffers of the host-buffer batch path
  Grow values, val_off, bstart, packed, block_off, sbo, scratch, err, index;
  // the piecewise host-buffer pipeline: copies in on h2d, kernels on
  // stream, copies out on d2h; ev_in[k] / ev_run[k] mark piece k's input
  // resident / its kernels done
  cudaStream_t h2d = nullptr, d2h = nullptr;
  cudaEvent_t ev_in[kMaxPieces] = {}, ev_run[kMaxPieces] = {};
  HostGrow h_meta;  // pinned landing area of the pack's block offsets

  int init() {
    UTL_CUDA(cudaGetDevice(&device));
    UTL_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    UTL_CUDA(cudaHostAlloc((void**)&h_stage, kStageBytes, cudaHostAllocMapped | cudaHostAllocPortable));
    UTL_CUDA(cudaHostGetDevicePointer((void**)&d_stage, h_stage, 0));
    UTL_CUDA(cudaMalloc((void**)&d_tmp, kStageIn));
    return UTL_OK;
  }
  int init_pipe() {
    if (h2d) return UTL_OK;
    for (int k = 0; k < kMaxPieces; k++) {
      UTL_CUDA(cudaEventCreateWithFlags(&ev_in[k], cudaEventDisableTiming));
      UTL_CUDA(cudaEventCreateWithFlags(&ev_run[k], cudaEventDisableTiming));
    }
    UTL_CUDA(cudaStreamCreateWithFlags(&d2h, cudaStreamNonBlocking));
    UTL_CUDA(cudaStreamCreateWithFlags(&h2d, cudaStreamNonBlocking));
    return UTL_OK;
  }
  void destroy() {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(device);
    cudaStream_t ss[] = {stream, h2d, d2h};
    for (cudaStream_t s : ss)
      if (s) cudaStreamSynchronize(s);
    Grow* gs[] = {&values, &val_off, &bstart, &packed, &block_off, &sbo, &scratch, &err, &index};
    for (Grow* g : gs) g->release();
    h_meta.release();
    for (int k = 0; k < kMaxPieces; k++) {
      if (ev_in[k]) cudaEventDestroy(ev_in[k]);
      if (ev_run[k]) cudaEventDestroy(ev_run[k]);
    }
    if (d_tmp) cudaFree(d_tmp);
    if (h_stage) cudaFreeHost(h_stage);
    for (cudaStream_t s : ss)
      if (s) cudaStreamDestroy(s);
    cudaSetDevice(cur);
  }
  uint8_t* in_h() { return h_stage; }
  uint8_t* in_d() { return d_stage; }
  uint8_t* out_h() { return h_stage + kStageIn; }
  uint8_t* out_d() { return d_stage + kStageIn; }
  PlainResult* res_h() { return (PlainResult*)(h_stage + kStageIn + kStageOut); }
  PlainResult* res_d() { return (PlainResult*)(d_stage + kStageIn + kStageOut); }
};

// One context per (host thread, device), released at thread exit.
struct ThreadCtxs {
  std::unordered_map<int, Ctx*> m;
  ~ThreadCtxs() {
    for (auto& kv : m) {
      kv.second->destroy();
      delete kv.second;
    }
  }
};
static thread_local ThreadCtxs t_ctxs;

static int thread_ctx(Ctx** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cuda_fail(e);
  auto it = t_ctxs.m.find(dev);
  if (it != t_ctxs.m.end()) {
    *out = it->second;
    return UTL_OK;
  }
  Ctx* c = new Ctx();
  int rc = c->init();
  if (rc != UTL_OK) {
    c->destroy();
    delete c;
    return rc;
  }
  t_ctxs.m[dev] = c;
  *out = c;
  return UTL_OK;
}

// ---------------------------------------------------------------------------
// header helpers (host): block_length.go:8-65, header.go:135-153,
// scalar.go:336-357, uint64.go:451-453
// ---------------------------------------------------------------------------
static int block_length_host(const uint8_t* src, size_t len, size_t* out) {
  if (!src && len) return UTL_ERR_ARG;
  if (len < 4) return UTL_ERR_INVALID_BUFFER;
  const uint32_t h = ld32(src);
  const int count = (int)(h & 0xFF), bw = (int)((h >> 8) & 31) * 4, itype = (int)((h >> 13) & 3);
  const int forw = (int)((h >> 15) & 3), exc = (int)(h >> 24);
  if (count > UTL_BLOCK_SIZE) return UTL_ERR_INVALID_BLOCK_LENGTH;
  if (bw > 32) return UTL_ERR_INVALID_BUFFER;
  const bool combine = (h & (1u << 19)) && itype == 3;
  if (itype == 3) {
    if (h & ((1u << 18) | (1u << 20))) return UTL_ERR_INVALID_FLAGS;
  } else if (h & ((1u << 18) | (1u << 19) | (1u << 20))) {
    return UTL_ERR_INVALID_FLAGS;
  }
  const size_t forb = (itype == 3 && !combine && forw == 3) ? 8 : (size_t)((1 << forw) >> 1);
  const size_t p_off = 4 + (exc ? 2 : 0) + forb + (combine ? 2 : 0);
  size_t b1 = p_off + ((size_t)bw << 4);
  if (exc) {
    if (len < 6) return UTL_ERR_INVALID_BUFFER;
    b1 += (size_t)(exc <= 16 ? exc : 16) + ld16(src + 4);
  }
  if (!combine) {
    *out = b1;
    return UTL_OK;
  }
  if (len < p_off) return UTL_ERR_INVALID_BUFFER;
  *out = b1 + ld16(src + p_off - 2);
  return UTL_OK;
}

// Upper bound of the bytes a decode of src may touch, from header fields
// alone (no validation): the per-call kernels stage only this much.
static size_t staged_extent(const uint8_t* src, size_t len) {
  if (len < 6) return len;
  const uint32_t h = ld32(src);
  const int bw = (int)((h >> 8) & 31) * 4, forw = (int)((h >> 15) & 3), exc = (int)(h >> 24);
  const bool combine = (h & (1u << 19)) != 0;
  size_t p_off = 4 + (exc ? 2 : 0) + (forw ? 8 : 0) + (combine ? 2 : 0);
  size_t e = p_off + (size_t)bw * 16 + (exc ? 16 + ld16(src + 4) : 0);
  if (combine) {
    size_t b2 = 4 + (exc ? 2 : 0) + (size_t)((1 << forw) >> 1);
    if (b2 + 2 <= len) e += ld16(src + b2);
  }
  return std::min(len, e + 64);
}

}  // namespace utl

using namespace utl;

// ---------------------------------------------------------------------------
// per-call entry points
// ---------------------------------------------------------------------------
static int pack_call(Ctx* c, bool u64, uint8_t flag, const void* values, int n, uint8_t* dst, size_t dst_cap,
                     size_t* out_len) {
  if (n <= 0 || n > UTL_BLOCK_SIZE) return UTL_ERR_INVALID_BUFFER;  // pack.go / scalar.go:240
  if (!values || !dst || !out_len) return UTL_ERR_ARG;
  memcpy(c->in_h(), values, (size_t)n * (u64 ? 8 : 4));
  c->res_h()->status = -1;
  cudaError_t e = launch::plain_pack(u64, flag, c->in_d(), n, c->out_d(), c->res_d(), c->stream);
  if (e != cudaSuccess) return cuda_fail(e);
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e);
  const PlainResult r = *c->res_h();
  if (r.status != UTL_OK) return r.status;
  if ((size_t)r.len > dst_cap) return UTL_ERR_CAPACITY;
  memcpy(dst, c->out_h(), (size_t)r.len);
  *out_len = (size_t)r.len;
  return UTL_OK;
}

static int unpack_call(Ctx* c, bool u64, const uint8_t* src, size_t src_len, void* values, int* count,
                       size_t* consumed, int* ovf) {
  if ((!src && src_len) || !values || !count || !consumed) return UTL_ERR_ARG;
  const size_t staged = staged_extent(src, src_len);
  if (staged > kStageIn) return UTL_ERR_ARG;
  if (staged) memcpy(c->in_h(), src, staged);
  c->res_h()->status = -1;
  cudaError_t e = launch::plain_unpack(u64, c->in_d(), (int64_t)staged, (int64_t)src_len, c->d_tmp, c->out_d(),
                                       c->res_d(), c->stream);
  if (e != cudaSuccess) return cuda_fail(e);
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e);
  const PlainResult r = *c->res_h();
  if (r.status != UTL_OK) {
    if (r.status == UTL_ERR_OVERFLOW && ovf) *ovf = r.ovf;
    return r.status;
  }
  memcpy(values, c->out_h(), (size_t)r.count * (u64 ? 8 : 4));
  *count = r.count;
  *consumed = (size_t)r.len;
  return UTL_OK;
}

static int get_call(Ctx* c, bool u64, int pos, const uint8_t* src, size_t src_len, uint64_t* value, int* ovf) {
  if ((!src && src_len) || !value) return UTL_ERR_ARG;
  const size_t staged = staged_extent(src, src_len);
  if (staged > kStageIn) return UTL_ERR_ARG;
  if (staged) memcpy(c->in_h(), src, staged);
  c->res_h()->status = -1;
  cudaError_t e = launch::plain_get(u64, pos, c->in_d(), (int64_t)staged, (int64_t)src_len, c->d_tmp, c->res_d(),
                                    c->stream);
  if (e != cudaSuccess) return cuda_fail(e);
  e = cudaStreamSynchronize(c->stream);
  if (e != cudaSuccess) return cuda_fail(e);
  const PlainResult r = *c->res_h();
  if (r.status != UTL_OK) {
    if (r.status == UTL_ERR_OVERFLOW && ovf) *ovf = r.ovf;
    return r.status;
  }
  *value = r.value;
  return UTL_OK;
}

#define WITH_CTX(expr)                 \
  Ctx* c_ = nullptr;                   \
  int rc_ = thread_ctx(&c_);           \
  if (rc_ != UTL_OK) return rc_;       \
  return (expr)

struct utl_codec {
  Ctx ctx;
};

extern "C" {

int utl_pack_u32(uint8_t flag, const uint32_t* values, int n, uint8_t* dst, size_t dst_cap, size_t* out_len) {
  WITH_CTX(pack_call(c_, false, flag, values, n, dst, dst_cap, out_len));
}
int utl_pack_u64(uint8_t flag, const uint64_t* values, int n, uint8_t* dst, size_t dst_cap, size_t* out_len) {
  WITH_CTX(pack_call(c_, true, flag, values, n, dst, dst_cap, out_len));
}
int utl_unpack_u32(const uint8_t* src, size_t src_len, uint32_t* values, int* count, size_t* consumed,
                   int* overflow_pos) {
  WITH_CTX(unpack_call(c_, false, src, src_len, values, count, consumed, overflow_pos));
}
int utl_unpack_u64(const uint8_t* src, size_t src_len, uint64_t* values, int* count, size_t* consumed,
                   int* overflow_pos) {
  WITH_CTX(unpack_call(c_, true, src, src_len, values, count, consumed, overflow_pos));
}
int utl_get_u32(int pos, const uint8_t* src, size_t src_len, uint32_t* value, int* overflow_pos) {
  if (!value) return UTL_ERR_ARG;
  uint64_t v = 0;
  Ctx* c = nullptr;
  int rc = thread_ctx(&c);
  if (rc != UTL_OK) return rc;
  rc = get_call(c, false, pos, src, src_len, &v, overflow_pos);
  if (rc == UTL_OK) *value = (uint32_t)v;
  return rc;
}
int utl_get_u64(int pos, const uint8_t* src, size_t src_len, uint64_t* value, int* overflow_pos) {
  WITH_CTX(get_call(c_, true, pos, src, src_len, value, overflow_pos));
}

int utl_block_length(const uint8_t* src, size_t src_len, size_t* block_len) {
  if (!block_len) return UTL_ERR_ARG;
  return block_length_host(src, src_len, block_len);
}

int utl_header(const uint8_t* src, size_t src_len, int* count, int* bit_width, int* exc_count, int* has_delta,
               int* has_for, int* has_zigzag, int* has_special) {
  int* outs[] = {count, bit_width, exc_count, has_delta, has_for, has_zigzag, has_special};
  for (int* o : outs)
    if (!o) return UTL_ERR_ARG;
  for (int* o : outs) *o = 0;
  if (src_len < 4 || !src) return UTL_ERR_INVALID_BUFFER;
  const uint32_t h = ld32(src);
  const int itype = (int)((h >> 13) & 3);
  if (itype != 2 && itype != 1) return UTL_ERR_UNSUPPORTED_TYPE;
  *count = (int)(h & 0xFF);
  *bit_width = (int)((h >> 8) & 31) * 4;
  *exc_count = (int)(h >> 24);
  *has_delta = (h >> 22) & 1;
  *has_for = ((h >> 15) & 3) > 0;
  *has_zigzag = (h >> 23) & 1;
  *has_special = (h >> 17) & 1;
  return UTL_OK;
}

int utl_max_block_length32(uint8_t flag) {
  const int forb = (flag & UTL_NOFOR) ? 0 : 4;
  if (flag & UTL_NOPATCH) return 4 + forb + 32 * 16;
  return 4 + 2 + forb + 28 * 16 + 16 + (32 + 4 * 128);
}
int utl_max_block_length64(uint8_t flag) { return 2 * utl_max_block_length32(flag) + 2; }

int utl_codec_new(int is64, utl_codec** out) {
  (void)is64;
  if (!out) return UTL_ERR_ARG;
  utl_codec* c = new utl_codec();
  int rc = c->ctx.init();
  if (rc != UTL_OK) {
    c->ctx.destroy();
    delete c;
    return rc;
  }
  *out = c;
  return UTL_OK;
}
void utl_codec_free(utl_codec* c) {
  if (!c) return;
  c->ctx.destroy();
  delete c;
}
int utl_codec_pack_u32(utl_codec* c, uint8_t flag, const uint32_t* values, int n, uint8_t* dst, size_t dst_cap,
                       size_t* out_len) {
  if (!c) return UTL_ERR_ARG;
  return pack_call(&c->ctx, false, flag, values, n, dst, dst_cap, out_len);
}
int utl_codec_unpack_u32(utl_codec* c, const uint8_t* src, size_t src_len, uint32_t* values, int* count,
                         size_t* consumed, int* overflow_pos) {
  if (!c) return UTL_ERR_ARG;
  return unpack_call(&c->ctx, false, src, src_len, values, count, consumed, overflow_pos);
}
int utl_codec_get_u32(utl_codec* c, int pos, const uint8_t* src, size_t src_len, uint32_t* value, int* overflow_pos) {
  if (!c || !value) return UTL_ERR_ARG;
  uint64_t v = 0;
  int rc = get_call(&c->ctx, false, pos, src, src_len, &v, overflow_pos);
  if (rc == UTL_OK) *value = (uint32_t)v;
  return rc;
}
int utl_codec_pack_u64(utl_codec* c, uint8_t flag, const uint64_t* values, int n, uint8_t* dst, size_t dst_cap,
                       size_t* out_len) {
  if (!c) return UTL_ERR_ARG;
  return pack_call(&c->ctx, true, flag, values, n, dst, dst_cap, out_len);
}
int utl_codec_unpack_u64(utl_codec* c, const uint8_t* src, size_t src_len, uint64_t* values, int* count,
                         size_t* consumed, int* overflow_pos) {
  if (!c) return UTL_ERR_ARG;
  return unpack_call(&c->ctx, true, src, src_len, values, count, consumed, overflow_pos);
}
int utl_codec_get_u64(utl_codec* c, int pos, const uint8_t* src, size_t src_len, uint64_t* value, int* overflow_pos) {
  if (!c) return UTL_ERR_ARG;
  return get_call(&c->ctx, true, pos, src, src_len, value, overflow_pos);
}

// ---------------------------------------------------------------------------
// pool of per-call contexts for many host threads
// ---------------------------------------------------------------------------
}  // extern "C"

// A fixed set of contexts (each: CUDA stream, mapped pinned staging, device
// scratch) shared by any number of host threads.  A call takes a free
// context (try-lock, starting at a rotating index so callers spread over
// the set), runs the per-call kernel on its stream and gives it back; calls
// on different contexts overlap on the GPU.
struct utl_pool {
  int device = 0;
  int n = 0;
  Ctx* ctx = nullptr;
  std::atomic<int>* busy = nullptr;
  std::atomic<uint32_t> next{0};
};

namespace {
struct PoolLease {
  utl_pool* p;
  int i = -1;
  int prev_dev = -1;
  explicit PoolLease(utl_pool* pool) : p(pool) {
    const uint32_t start = p->next.fetch_add(1, std::memory_order_relaxed);
    for (uint64_t t = 0;; t++) {
      const int k = (int)((start + t) % (uint32_t)p->n);
      int z = 0;
      if (p->busy[k].load(std::memory_order_relaxed) == 0 &&
          p->busy[k].compare_exchange_strong(z, 1, std::memory_order_acquire)) {
        i = k;
        break;
      }
      if ((t + 1) % (uint64_t)p->n == 0) std::this_thread::yield();
    }
    int cur = 0;
    if (cudaGetDevice(&cur) == cudaSuccess && cur != p->device) {
      prev_dev = cur;
      cudaSetDevice(p->device);
    }
  }
  ~PoolLease() {
    if (prev_dev >= 0) cudaSetDevice(prev_dev);
    p->busy[i].store(0, std::memory_order_release);
  }
  Ctx* ctx() { return &p->ctx[i]; }
};
}  // namespace

extern "C" {

int utl_pool_new(int n_contexts, utl_pool** out) {
  if (!out || n_contexts <= 0 || n_contexts > 1024) return UTL_ERR_ARG;
  *out = nullptr;
  utl_pool* p = new utl_pool();
  p->n = n_contexts;
  p->ctx = new Ctx[n_contexts];
  p->busy = new std::atomic<int>[n_contexts];
  int rc = UTL_OK;
  cudaError_t e = cudaGetDevice(&p->device);
  if (e != cudaSuccess) rc = cuda_fail(e);
  for (int k = 0; k < n_contexts; k++) {
    p->busy[k].store(0);
    if (rc == UTL_OK) rc = p->ctx[k].init();
  }
  if (rc != UTL_OK) {
    utl_pool_free(p);
    return rc;
  }
  *out = p;
  return UTL_OK;
}
void utl_pool_free(utl_pool* p) {
  if (!p) return;
  for (int k = 0; k < p->n; k++) p->ctx[k].destroy();
  delete[] p->ctx;
  delete[] p->busy;
  delete p;
}
int utl_pool_pack_u32(utl_pool* p, uint8_t flag, const uint32_t* values, int n, uint8_t* dst, size_t dst_cap,
                      size_t* out_len) {
  if (!p) return UTL_ERR_ARG;
  PoolLease l(p);
  return pack_call(l.ctx(), false, flag, values, n, dst, dst_cap, out_len);
}
int utl_pool_unpack_u32(utl_pool* p, const uint8_t* src, size_t src_len, uint32_t* values, int* count,
                        size_t* consumed, int* overflow_pos) {
  if (!p) return UTL_ERR_ARG;
  PoolLease l(p);
  return unpack_call(l.ctx(), false, src, src_len, values, count, consumed, overflow_pos);
}
int utl_pool_get_u32(utl_pool* p, int pos, const uint8_t* src, size_t src_len, uint32_t* value, int* overflow_pos) {
  if (!p || !value) return UTL_ERR_ARG;
  uint64_t v = 0;
  PoolLease l(p);
  const int rc = get_call(l.ctx(), false, pos, src, src_len, &v, overflow_pos);
  if (rc == UTL_OK) *value = (uint32_t)v;
  return rc;
}
int utl_pool_pack_u64(utl_pool* p, uint8_t flag, const uint64_t* values, int n, uint8_t* dst, size_t dst_cap,
                      size_t* out_len) {
  if (!p) return UTL_ERR_ARG;
  PoolLease l(p);
  return pack_call(l.ctx(), true, flag, values, n, dst, dst_cap, out_len);
}
int utl_pool_unpack_u64(utl_pool* p, const uint8_t* src, size_t src_len, uint64_t* values, int* count,
                        size_t* consumed, int* overflow_pos) {
  if (!p) return UTL_ERR_ARG;
  PoolLease l(p);
  return unpack_call(l.ctx(), true, src, src_len, values, count, consumed, overflow_pos);
}
int utl_pool_get_u64(utl_pool* p, int pos, const uint8_t* src, size_t src_len, uint64_t* value, int* overflow_pos) {
  if (!p) return UTL_ERR_ARG;
  PoolLease l(p);
  return get_call(l.ctx(), true, pos, src, src_len, value, overflow_pos);
}

// ---------------------------------------------------------------------------
// batched, device buffers
// ---------------------------------------------------------------------------
int64_t utl_count_blocks(const uint64_t* h_val_off, int n_streams) {
  if (!h_val_off || n_streams < 0) return -1;
  int64_t nb = 0;
  for (int s = 0; s < n_streams; s++) {
    if (h_val_off[s + 1] < h_val_off[s]) return -1;
    nb += (int64_t)((h_val_off[s + 1] - h_val_off[s] + UTL_BLOCK_SIZE - 1) / UTL_BLOCK_SIZE);
  }
  return nb;
}

int utl_batch_plan(const uint64_t* d_val_off, int n_streams, uint64_t* d_block_start, void* stream) {
  if (!d_val_off || !d_block_start || n_streams < 0) return UTL_ERR_ARG;
  cudaError_t e = launch::plan(d_val_off, n_streams, d_block_start, (cudaStream_t)stream);
  return e == cudaSuccess ? UTL_OK : cuda_fail(e);
}

size_t utl_pack_scratch_bytes(int64_t n_blocks) { return launch::pack_scratch_bytes(n_blocks < 0 ? 0 : n_blocks); }

}  // extern "C"

int utl::pack_batch_device(bool u64, bool may_alloc, uint8_t flag, const void* d_values, const uint64_t* d_val_off,
                      const uint64_t* d_block_start, int n_streams, int64_t n_blocks, uint8_t* d_out, size_t out_cap,
                      uint64_t* d_block_off, uint64_t* d_sbo, void* d_scratch, size_t scratch_bytes, uint32_t* d_err,
                      cudaStream_t st) {
  if (n_streams < 0 || n_blocks < 0 || !d_val_off || !d_block_start || !d_block_off) return UTL_ERR_ARG;
  if (n_blocks > 0 && (!d_values || !d_out || !d_scratch)) return UTL_ERR_ARG;
  if (((uintptr_t)d_out & 3) != 0) return UTL_ERR_ARG;
  if (n_blocks == 0) {
    UTL_CUDA(cudaMemsetAsync(d_block_off, 0, sizeof(uint64_t), st));
  } else {
    if (scratch_bytes < launch::pack_scratch_bytes(n_blocks)) return UTL_ERR_ARG;
    if (!launch::keep_scratch()) UTL_CUDA(cudaMemsetAsync(d_scratch, 0, launch::pack_scratch_bytes(n_blocks), st));
    PackArgs a;
    a.values = d_values;
    a.val_off = d_val_off;
    a.block_start = d_block_start;
    a.n_streams = n_streams;
    a.flag = flag;
    a.n_blocks = n_blocks;
    a.n_tiles = launch::tiles_for(n_blocks);
    a.out = d_out;
    a.out_cap = out_cap;
    a.block_off = d_block_off;
    a.counter = (unsigned long long*)d_scratch;
    a.tile_status = (uint64_t*)((uint8_t*)d_scratch + 16);
    a.err = d_err;
    a.spin_limit = launch::spin_limit();
    cudaError_t e = launch::pack(u64, a, st, may_alloc);
    if (e != cudaSuccess) return cuda_fail(e);
  }
  if (d_sbo) {
    cudaError_t e = launch::stream_offsets(d_block_off, d_block_start, n_streams, d_sbo, st);
    if (e != cudaSuccess) return cuda_fail(e);
  }
  return UTL_OK;
}

extern "C" {

int utl_pack_batch_u32(uint8_t flag, const uint32_t* d_values, const uint64_t* d_val_off,
                       const uint64_t* d_block_start, int n_streams, int64_t n_blocks, uint8_t* d_out, size_t out_cap,
                       uint64_t* d_block_off, uint64_t* d_stream_byte_off, void* d_scratch, size_t scratch_bytes,
                       uint32_t* d_err, void* stream) {
  return pack_batch_device(false, true, flag, d_values, d_val_off, d_block_start, n_streams, n_blocks, d_out, out_cap,
                           d_block_off, d_stream_byte_off, d_scratch, scratch_bytes, d_err, (cudaStream_t)stream);
}
int utl_pack_batch_u64(uint8_t flag, const uint64_t* d_values, const uint64_t* d_val_off,
                       const uint64_t* d_block_start, int n_streams, int64_t n_blocks, uint8_t* d_out, size_t out_cap,
                       uint64_t* d_block_off, uint64_t* d_stream_byte_off, void* d_scratch, size_t scratch_bytes,
                       uint32_t* d_err, void* stream) {
  return pack_batch_device(true, true, flag, d_values, d_val_off, d_block_start, n_streams, n_blocks, d_out, out_cap,
                           d_block_off, d_stream_byte_off, d_scratch, scratch_bytes, d_err, (cudaStream_t)stream);
}

static int unpack_batch(bool u64, const uint8_t* d_packed, size_t packed_len, const uint64_t* d_block_off,
                        const uint64_t* d_val_off, const uint64_t* d_block_start, int n_streams, int64_t n_blocks,
                        void* d_values, int32_t* d_status, uint32_t* d_err, cudaStream_t st) {
  if (n_streams < 0 || n_blocks < 0) return UTL_ERR_ARG;
  if (n_blocks == 0) return UTL_OK;
  if (!d_packed || !d_block_off || !d_val_off || !d_block_start || !d_values) return UTL_ERR_ARG;
  UnpackArgs a;
  a.packed = d_packed;
  a.packed_len = packed_len;
  a.block_off = d_block_off;
  a.val_off = d_val_off;
  a.block_start = d_block_start;
  a.n_streams = n_streams;
  a.n_blocks = n_blocks;
  a.values = d_values;
  a.block_status = d_status;
  a.err = d_err;
  a.spin_limit = launch::spin_limit();
  cudaError_t e = launch::unpack(u64, a, st);
  return e == cudaSuccess ? UTL_OK : cuda_fail(e);
}

int utl_unpack_batch_u32(const uint8_t* d_packed, size_t packed_len, const uint64_t* d_block_off,
                         const uint64_t* d_val_off, const uint64_t* d_block_start, int n_streams, int64_t n_blocks,
                         uint32_t* d_values, int32_t* d_block_status, uint32_t* d_err, void* stream) {
  return unpack_batch(false, d_packed, packed_len, d_block_off, d_val_off, d_block_start, n_streams, n_blocks,
                      d_values, d_block_status, d_err, (cudaStream_t)stream);
}
int utl_unpack_batch_u64(const uint8_t* d_packed, size_t packed_len, const uint64_t* d_block_off,
                         const uint64_t* d_val_off, const uint64_t* d_block_start, int n_streams, int64_t n_blocks,
                         uint64_t* d_values, int32_t* d_block_status, uint32_t* d_err, void* stream) {
  return unpack_batch(true, d_packed, packed_len, d_block_off, d_val_off, d_block_start, n_streams, n_blocks,
                      d_values, d_block_status, d_err, (cudaStream_t)stream);
}

static int get_batch(bool u64, const uint8_t* d_packed, size_t packed_len, const uint64_t* d_block_off,
                     const uint64_t* d_val_off, const uint64_t* d_block_start, int n_streams,
                     const uint32_t* d_q_stream, const uint64_t* d_q_pos, int64_t n_queries, void* d_out,
                     int32_t* d_status, uint32_t* d_err, cudaStream_t st) {
  if (n_queries < 0 || n_streams < 0) return UTL_ERR_ARG;
  if (n_queries == 0) return UTL_OK;
  if (!d_block_off || !d_val_off || !d_block_start || !d_q_stream || !d_q_pos || !d_out) return UTL_ERR_ARG;
  GetArgs a;
  a.packed = d_packed;
  a.packed_len = packed_len;
  a.block_off = d_block_off;
  a.val_off = d_val_off;
  a.block_start = d_block_start;
  a.n_streams = n_streams;
  a.q_stream = d_q_stream;
  a.q_pos = d_q_pos;
  a.n_queries = n_queries;
  a.out = d_out;
  a.status = d_status;
  a.err = d_err;
  cudaError_t e = launch::get(u64, a, st);
  return e == cudaSuccess ? UTL_OK : cuda_fail(e);
}

int utl_get_batch_u32(const uint8_t* d_packed, size_t packed_len, const uint64_t* d_block_off,
                      const uint64_t* d_val_off, const uint64_t* d_block_start, int n_streams,
                      const uint32_t* d_q_stream, const uint64_t* d_q_pos, int64_t n_queries, uint32_t* d_out,
                      int32_t* d_status, uint32_t* d_err, void* stream) {
  return get_batch(false, d_packed, packed_len, d_block_off, d_val_off, d_block_start, n_streams, d_q_stream, d_q_pos,
                   n_queries, d_out, d_status, d_err, (cudaStream_t)stream);
}
int utl_get_batch_u64(const uint8_t* d_packed, size_t packed_len, const uint64_t* d_block_off,
                      const uint64_t* d_val_off, const uint64_t* d_block_start, int n_streams,
                      const uint32_t* d_q_stream, const uint64_t* d_q_pos, int64_t n_queries, uint64_t* d_out,
                      int32_t* d_status, uint32_t* d_err, void* stream) {
  return get_batch(true, d_packed, packed_len, d_block_off, d_val_off, d_block_start, n_streams, d_q_stream, d_q_pos,
                   n_queries, d_out, d_status, d_err, (cudaStream_t)stream);
}

// ---------------------------------------------------------------------------
// batched, host buffers
// ---------------------------------------------------------------------------
static int first_error(uint32_t bits) {
  for (int c = 1; c < 32; c++)
    if (bits & (1u << c)) return c;
  return UTL_OK;
}

// Host-buffer batches go through the piecewise pipeline when the knob
// allows: 0 = never, 1 = batches of at least kPipeMinBytes of values, in
// pieces of max(kPieceMinBytes, batch / 32), 2 = any batch, in eighths.
static std::atomic<int> g_host_pipe{1};
constexpr uint64_t kPipeMinBytes = 64ull << 20;
constexpr uint64_t kPieceMinBytes = 16ull << 20;

// Values per piece for a batch of nv values of esz bytes (0 = one piece).
static uint64_t piece_target(uint64_t nv, size_t esz) {
  const uint64_t B = UTL_BLOCK_SIZE;
  const int mode = g_host_pipe.load(std::memory_order_relaxed);
  uint64_t t = 0;
  if (mode == 1 && nv * esz >= kPipeMinBytes) t = std::max(kPieceMinBytes, nv * esz / 32) / esz;
  if (mode == 2) t = (nv + 7) / 8;
  return t ? (t + B - 1) / B * B : 0;
}


// Pack through the pipeline: piece k's values go in on h2d while piece
// k-1 packs on the compute stream into its own worst-case region; when a
// piece is done the host reads its packed size, places its block offsets
// after the pieces before it and copies its bytes out on d2h, so the two
// copy directions and the kernels overlap.
static int pack_streams_piped(Ctx* c, bool u64, uint8_t flag, const void* h_values, const uint64_t* h_val_off,
                              int n_streams, int64_t nb, const std::vector<Piece>& ps,
                              const std::vector<uint64_t>& tab, uint8_t* h_out, size_t out_cap,
                              uint64_t* h_block_off, uint64_t* h_sbo, size_t* out_len) {
  const int P = (int)ps.size();
  const size_t esz = u64 ? 8 : 4;
  const uint64_t v0 = h_val_off[0], nv = h_val_off[n_streams] - v0;
  const size_t maxb = (size_t)(u64 ? utl_max_block_length64(flag) : utl_max_block_length32(flag));
  std::vector<size_t> reg(P + 1, 0);  // piece k packs into packed[reg[k], reg[k+1])
  int64_t nb_max = 0;
  for (int k = 0; k < P; k++) {
    const int64_t n = ps[k].b1 - ps[k].b0;
    nb_max = std::max(nb_max, n);
    reg[k + 1] = reg[k] + (((size_t)n * maxb + 16 + 255) & ~(size_t)255);
  }
  int rc = c->init_pipe();
  if (rc != UTL_OK) return rc;
  UTL_CUDA(c->values.ensure(nv * esz));
  UTL_CUDA(c->val_off.ensure(tab.size() * 8));
  UTL_CUDA(c->bstart.ensure(tab.size() * 8));
  UTL_CUDA(c->packed.ensure(reg[P]));
  UTL_CUDA(c->block_off.ensure(((size_t)nb + P) * 8));  // piece k's nb_k + 1 offsets at b0 + k
  UTL_CUDA(c->scratch.ensure(launch::pack_scratch_bytes(nb_max)));
  UTL_CUDA(c->err.ensure(8));
  UTL_CUDA(c->h_meta.ensure(((size_t)nb + P) * 8));
  const cudaStream_t st = c->stream;
  uint64_t* dtab = (uint64_t*)c->val_off.p;
  uint64_t* dbs = (uint64_t*)c->bstart.p;
  uint64_t* dbo = (uint64_t*)c->block_off.p;
  const uint64_t* hbo = (const uint64_t*)c->h_meta.p;
  UTL_CUDA(cudaMemsetAsync(c->err.p, 0, 4, st));
  UTL_CUDA(cudaMemcpyAsync(dtab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, c->h2d));

  int next = 0;        // first piece whose bytes are not yet placed
  uint64_t base = 0;   // packed bytes of the pieces before it
  // place pieces [next, upto) that are done (all of them when wait): only
  // pieces already enqueued, since an event not yet recorded in this call
  // still reports an earlier call's completion
  auto place = [&](int upto, bool wait) -> int {
    while (next < upto) {
      cudaError_t e = wait ? cudaEventSynchronize(c->ev_run[next]) : cudaEventQuery(c->ev_run[next]);
      if (e == cudaErrorNotReady) return UTL_OK;
      if (e != cudaSuccess) return cuda_fail(e);
      const Piece& q = ps[next];
      const int64_t n = q.b1 - q.b0;
      const uint64_t* rel = hbo + q.b0 + next;
      for (int64_t i = 0; i < n; i++) h_block_off[q.b0 + i] = rel[i] + base;
      const uint64_t len = rel[n];
      if (len && h_out && base + len <= out_cap)
        UTL_CUDA(cudaMemcpyAsync(h_out + base, (uint8_t*)c->packed.p + reg[next], len, cudaMemcpyDeviceToHost,
                                 c->d2h));
      base += len;
      next++;
    }
    return UTL_OK;
  };

  for (int k = 0; k < P; k++) {
    const Piece& q = ps[k];
    const int64_t n = q.b1 - q.b0;
    uint8_t* dv = (uint8_t*)c->values.p + (q.v0 - v0) * esz;
    UTL_CUDA(cudaMemcpyAsync(dv, (const uint8_t*)h_values + q.v0 * esz, (q.v1 - q.v0) * esz, cudaMemcpyHostToDevice,
                             c->h2d));
    UTL_CUDA(cudaEventRecord(c->ev_in[k], c->h2d));
    UTL_CUDA(cudaStreamWaitEvent(st, c->ev_in[k], 0));
    cudaError_t e = launch::plan(dtab + q.t0, q.ns, dbs + q.t0, st);
    if (e != cudaSuccess) return cuda_fail(e);
    rc = pack_batch_device(u64, true, flag, dv, dtab + q.t0, dbs + q.t0, q.ns, n, (uint8_t*)c->packed.p + reg[k],
                    reg[k + 1] - reg[k], dbo + q.b0 + k, nullptr, c->scratch.p, c->scratch.cap, (uint32_t*)c->err.p,
                    st);
    if (rc != UTL_OK) return rc;
    UTL_CUDA(cudaMemcpyAsync(c->h_meta.p + (q.b0 + k) * 8, dbo + q.b0 + k, ((size_t)n + 1) * 8,
                             cudaMemcpyDeviceToHost, st));
    UTL_CUDA(cudaEventRecord(c->ev_run[k], st));
    rc = place(k + 1, false);
    if (rc != UTL_OK) return rc;
  }
  rc = place(P, true);
  if (rc != UTL_OK) return rc;
  uint32_t errbits = 0;
  UTL_CUDA(cudaMemcpyAsync(&errbits, c->err.p, 4, cudaMemcpyDeviceToHost, st));
  UTL_CUDA(cudaStreamSynchronize(st));
  UTL_CUDA(cudaStreamSynchronize(c->d2h));
  if (errbits) return first_error(errbits);
  h_block_off[nb] = base;
  if (h_sbo) {
    int64_t b = 0;
    for (int s = 0; s < n_streams; s++) {
      h_sbo[s] = h_block_off[b];
      b += (int64_t)((h_val_off[s + 1] - h_val_off[s] + UTL_BLOCK_SIZE - 1) / UTL_BLOCK_SIZE);
    }
    h_sbo[n_streams] = base;
  }
  *out_len = (size_t)base;
  if (base > out_cap || (base && !h_out)) return UTL_ERR_CAPACITY;
  return UTL_OK;
}

// Unpack through the pipeline: every piece's packed bytes and block
// offsets are queued on h2d first; piece k unpacks once its bytes are in
// and its values go out on d2h while later pieces still come in.  Piece k
// reads bytes below round_up(block_off[b1], 16) when its offsets rise
// monotonically, and all of them are in once its own copy is; a piece
// whose offsets do not rise waits for the whole buffer, so its blocks
// decode (or fail) exactly as in a single pass.
static int unpack_streams_piped(Ctx* c, bool u64, const uint8_t* h_packed, size_t packed_len,
                                const uint64_t* h_block_off, const uint64_t* h_val_off, int n_streams, int64_t nb,
                                const std::vector<Piece>& ps, const std::vector<uint64_t>& tab, void* h_values) {
  const int P = (int)ps.size();
  const size_t esz = u64 ? 8 : 4;
  const uint64_t v0 = h_val_off[0], nv = h_val_off[n_streams] - v0;
  int rc = c->init_pipe();
  if (rc != UTL_OK) return rc;
  UTL_CUDA(c->values.ensure(nv * esz));
  UTL_CUDA(c->val_off.ensure(tab.size() * 8));
  UTL_CUDA(c->bstart.ensure(tab.size() * 8));
  UTL_CUDA(c->packed.ensure(packed_len + 16));
  UTL_CUDA(c->block_off.ensure(((size_t)nb + 1) * 8));
  UTL_CUDA(c->err.ensure(8));
  const cudaStream_t st = c->stream;
  uint64_t* dtab = (uint64_t*)c->val_off.p;
  uint64_t* dbs = (uint64_t*)c->bstart.p;
  uint64_t* dbo = (uint64_t*)c->block_off.p;
  uint8_t* dp = (uint8_t*)c->packed.p;
  UTL_CUDA(cudaMemsetAsync(c->err.p, 0, 4, st));
  UTL_CUDA(cudaMemcpyAsync(dtab, tab.data(), tab.size() * 8, cudaMemcpyHostToDevice, c->h2d));
  // piece k copies bytes [cut[k], cut[k+1]) of the packed buffer
  std::vector<uint64_t> cut(P + 1, 0);
  cut[P] = packed_len;
  for (int k = 1; k < P; k++) {
    const uint64_t o = std::min<uint64_t>(h_block_off[ps[k].b0], packed_len);
    cut[k] = std::max(cut[k - 1], std::min<uint64_t>((o + 15) & ~(uint64_t)15, packed_len));
  }
  for (int k = 0; k < P; k++) {
    const Piece& q = ps[k];
    UTL_CUDA(cudaMemcpyAsync(dbo + q.b0, h_block_off + q.b0, ((size_t)(q.b1 - q.b0) + 1) * 8,
                             cudaMemcpyHostToDevice, c->h2d));
    if (cut[k + 1] > cut[k])
      UTL_CUDA(cudaMemcpyAsync(dp + cut[k], h_packed + cut[k], cut[k + 1] - cut[k], cudaMemcpyHostToDevice, c->h2d));
    UTL_CUDA(cudaEventRecord(c->ev_in[k], c->h2d));
  }
  for (int k = 0; k < P; k++) {
    const Piece& q = ps[k];
    bool rising = true;
    for (int64_t b = q.b0; b < q.b1 && rising; b++) rising = h_block_off[b + 1] >= h_block_off[b];
    UTL_CUDA(cudaStreamWaitEvent(st, c->ev_in[rising ? k : P - 1], 0));
    cudaError_t e = launch::plan(dtab + q.t0, q.ns, dbs + q.t0, st);
    if (e != cudaSuccess) return cuda_fail(e);
    const size_t vb = (q.v0 - v0) * esz;
    rc = unpack_batch(u64, dp, packed_len, dbo + q.b0, dtab + q.t0, dbs + q.t0, q.ns, q.b1 - q.b0,
                      (uint8_t*)c->values.p + vb, nullptr, (uint32_t*)c->err.p, st);
    if (rc != UTL_OK) return rc;
    UTL_CUDA(cudaEventRecord(c->ev_run[k], st));
    UTL_CUDA(cudaStreamWaitEvent(c->d2h, c->ev_run[k], 0));
    UTL_CUDA(cudaMemcpyAsync((uint8_t*)h_values + q.v0 * esz, (uint8_t*)c->values.p + vb, (q.v1 - q.v0) * esz,
                             cudaMemcpyDeviceToHost, c->d2h));
  }
  uint32_t errbits = 0;
  UTL_CUDA(cudaMemcpyAsync(&errbits, c->err.p, 4, cudaMemcpyDeviceToHost, c->d2h));
  UTL_CUDA(cudaStreamSynchronize(c->d2h));
  return errbits ? first_error(errbits) : UTL_OK;
}

static int pack_streams(bool u64, uint8_t flag, const void* h_values, const uint64_t* h_val_off, int n_streams,
                        uint8_t* h_out, size_t out_cap, uint64_t* h_block_off, uint64_t* h_sbo, size_t* out_len) {
  if (!h_val_off || n_streams < 0 || !out_len || !h_block_off) return UTL_ERR_ARG;
  const int64_t nb = utl_count_blocks(h_val_off, n_streams);
  if (nb < 0) return UTL_ERR_ARG;
  Ctx* c = nullptr;
  int rc = thread_ctx(&c);
  if (rc != UTL_OK) return rc;
  const size_t esz = u64 ? 8 : 4;
  const uint64_t v0 = h_val_off[0], nv = h_val_off[n_streams] - v0;
  const uint64_t target = piece_target(nv, esz);
  if (target && nv > target) {
    std::vector<Piece> ps;
    std::vector<uint64_t> tab;
    cut_pieces(h_val_off, n_streams, target, ps, tab);
    if (ps.size() >= 2 && ps.size() <= (size_t)kMaxPieces)
      return pack_streams_piped(c, u64, flag, h_values, h_val_off, n_streams, nb, ps, tab, h_out, out_cap,
                                h_block_off, h_sbo, out_len);
  }
  const size_t maxb = (size_t)(u64 ? utl_max_block_length64(flag) : utl_max_block_length32(flag));
  UTL_CUDA(c->values.ensure(nv * esz));
  UTL_CUDA(c->val_off.ensure(((size_t)n_streams + 1) * 8));
  UTL_CUDA(c->bstart.ensure(((size_t)n_streams + 1) * 8));
  UTL_CUDA(c->packed.ensure((size_t)nb * maxb + 16));
  UTL_CUDA(c->block_off.ensure(((size_t)nb + 1) * 8));
  UTL_CUDA(c->sbo.ensure(((size_t)n_streams + 1) * 8));
  UTL_CUDA(c->scratch.ensure(launch::pack_scratch_bytes(nb)));
  UTL_CUDA(c->err.ensure(8));
  cudaStream_t st = c->stream;
  if (nv) UTL_CUDA(cudaMemcpyAsync(c->values.p, (const uint8_t*)h_values + v0 * esz, nv * esz, cudaMemcpyHostToDevice, st));
  UTL_CUDA(cudaMemsetAsync(c->err.p, 0, 4, st));
  // value offsets are rebased to the copied range when the table does not start at zero
  uint64_t* dvo = (uint64_t*)c->val_off.p;
  if (v0) {
    uint64_t* tmp = new uint64_t[(size_t)n_streams + 1];
    for (int s = 0; s <= n_streams; s++) tmp[s] = h_val_off[s] - v0;
    cudaError_t e = cudaMemcpyAsync(dvo, tmp, ((size_t)n_streams + 1) * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    delete[] tmp;
    if (e != cudaSuccess) return cuda_fail(e);
  } else {
    UTL_CUDA(cudaMemcpyAsync(dvo, h_val_off, ((size_t)n_streams + 1) * 8, cudaMemcpyHostToDevice, st));
  }
  cudaError_t e = launch::plan(dvo, n_streams, (uint64_t*)c->bstart.p, st);
  if (e != cudaSuccess) return cuda_fail(e);
  rc = pack_batch_device(u64, true, flag, c->values.p, dvo, (const uint64_t*)c->bstart.p, n_streams, nb, (uint8_t*)c->packed.p,
                  c->packed.cap, (uint64_t*)c->block_off.p, h_sbo ? (uint64_t*)c->sbo.p : nullptr, c->scratch.p,
                  c->scratch.cap, (uint32_t*)c->err.p, st);
  if (rc != UTL_OK) return rc;
  UTL_CUDA(cudaMemcpyAsync(h_block_off, c->block_off.p, ((size_t)nb + 1) * 8, cudaMemcpyDeviceToHost, st));
  uint32_t errbits = 0;
  UTL_CUDA(cudaMemcpyAsync(&errbits, c->err.p, 4, cudaMemcpyDeviceToHost, st));
  if (h_sbo) UTL_CUDA(cudaMemcpyAsync(h_sbo, c->sbo.p, ((size_t)n_streams + 1) * 8, cudaMemcpyDeviceToHost, st));
  UTL_CUDA(cudaStreamSynchronize(st));
  if (errbits) return first_error(errbits);
  const size_t total = (size_t)h_block_off[nb];
  *out_len = total;
  if (total > out_cap || (total && !h_out)) return UTL_ERR_CAPACITY;
  if (total) {
    UTL_CUDA(cudaMemcpyAsync(h_out, c->packed.p, total, cudaMemcpyDeviceToHost, st));
    UTL_CUDA(cudaStreamSynchronize(st));
  }
  return UTL_OK;
}

static int unpack_streams(bool u64, const uint8_t* h_packed, size_t packed_len, const uint64_t* h_block_off,
                          const uint64_t* h_val_off, int n_streams, void* h_values) {
  if (!h_val_off || !h_block_off || n_streams < 0) return UTL_ERR_ARG;
  const int64_t nb = utl_count_blocks(h_val_off, n_streams);
  if (nb < 0) return UTL_ERR_ARG;
  if (nb == 0) return UTL_OK;
  if (!h_packed || !h_values) return UTL_ERR_ARG;
  Ctx* c = nullptr;
  int rc = thread_ctx(&c);
  if (rc != UTL_OK) return rc;
  const size_t esz = u64 ? 8 : 4;
  const uint64_t v0 = h_val_off[0], nv = h_val_off[n_streams] - v0;
  const uint64_t target = piece_target(nv, esz);
  if (target && nv > target) {
    std::vector<Piece> ps;
    std::vector<uint64_t> tab;
    cut_pieces(h_val_off, n_streams, target, ps, tab);
    if (ps.size() >= 2 && ps.size() <= (size_t)kMaxPieces)
      return unpack_streams_piped(c, u64, h_packed, packed_len, h_block_off, h_val_off, n_streams, nb, ps, tab,
                                  h_values);
  }
  UTL_CUDA(c->values.ensure(nv * esz));
  UTL_CUDA(c->val_off.ensure(((size_t)n_streams + 1) * 8));
  UTL_CUDA(c->bstart.ensure(((size_t)n_streams + 1) * 8));
  UTL_CUDA(c->packed.ensure(packed_len + 16));
  UTL_CUDA(c->block_off.ensure(((size_t)nb + 1) * 8));
  UTL_CUDA(c->err.ensure(8));
  cudaStream_t st = c->stream;
  UTL_CUDA(cudaMemcpyAsync(c->packed.p, h_packed, packed_len, cudaMemcpyHostToDevice, st));
  UTL_CUDA(cudaMemcpyAsync(c->block_off.p, h_block_off, ((size_t)nb + 1) * 8, cudaMemcpyHostToDevice, st));
  UTL_CUDA(cudaMemsetAsync(c->err.p, 0, 4, st));
  uint64_t* dvo = (uint64_t*)c->val_off.p;
  if (v0) {
    uint64_t* tmp = new uint64_t[(size_t)n_streams + 1];
    for (int s = 0; s <= n_streams; s++) tmp[s] = h_val_off[s] - v0;
    cudaError_t e = cudaMemcpyAsync(dvo, tmp, ((size_t)n_streams + 1) * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    delete[] tmp;
    if (e != cudaSuccess) return cuda_fail(e);
  } else {
    UTL_CUDA(cudaMemcpyAsync(dvo, h_val_off, ((size_t)n_streams + 1) * 8, cudaMemcpyHostToDevice, st));
  }
  cudaError_t e = launch::plan(dvo, n_streams, (uint64_t*)c->bstart.p, st);
  if (e != cudaSuccess) return cuda_fail(e);
  rc = unpack_batch(u64, (const uint8_t*)c->packed.p, packed_len, (const uint64_t*)c->block_off.p, dvo,
                    (const uint64_t*)c->bstart.p, n_streams, nb, c->values.p, nullptr, (uint32_t*)c->err.p, st);
  if (rc != UTL_OK) return rc;
  uint32_t errbits = 0;
  UTL_CUDA(cudaMemcpyAsync(&errbits, c->err.p, 4, cudaMemcpyDeviceToHost, st));
  UTL_CUDA(cudaMemcpyAsync((uint8_t*)h_values + v0 * esz, c->values.p, nv * esz, cudaMemcpyDeviceToHost, st));
  UTL_CUDA(cudaStreamSynchronize(st));
  return errbits ? first_error(errbits) : UTL_OK;
}

int utl_pack_streams_u32(uint8_t flag, const uint32_t* h_values, const uint64_t* h_val_off, int n_streams,
                         uint8_t* h_out, size_t out_cap, uint64_t* h_block_off, uint64_t* h_stream_byte_off,
                         size_t* out_len) {
  return pack_streams(false, flag, h_values, h_val_off, n_streams, h_out, out_cap, h_block_off, h_stream_byte_off,
                      out_len);
}
int utl_pack_streams_u64(uint8_t flag, const uint64_t* h_values, const uint64_t* h_val_off, int n_streams,
                         uint8_t* h_out, size_t out_cap, uint64_t* h_block_off, uint64_t* h_stream_byte_off,
                         size_t* out_len) {
  return pack_streams(true, flag, h_values, h_val_off, n_streams, h_out, out_cap, h_block_off, h_stream_byte_off,
                      out_len);
}
int utl_unpack_streams_u32(const uint8_t* h_packed, size_t packed_len, const uint64_t* h_block_off,
                           const uint64_t* h_val_off, int n_streams, uint32_t* h_values) {
  return unpack_streams(false, h_packed, packed_len, h_block_off, h_val_off, n_streams, h_values);
}
int utl_unpack_streams_u64(const uint8_t* h_packed, size_t packed_len, const uint64_t* h_block_off,
                           const uint64_t* h_val_off, int n_streams, uint64_t* h_values) {
  return unpack_streams(true, h_packed, packed_len, h_block_off, h_val_off, n_streams, h_values);
}

int utl_index_stream(const uint8_t* d_packed, size_t packed_len, uint64_t* d_block_off, int64_t max_blocks,
                     int64_t* n_blocks, void* stream) {
  if (!n_blocks || !d_block_off || max_blocks < 0 || (packed_len && !d_packed)) return UTL_ERR_ARG;
  *n_blocks = 0;
  Ctx* c = nullptr;
  int rc = thread_ctx(&c);
  if (rc != UTL_OK) return rc;
  UTL_CUDA(c->index.ensure(launch::index_scratch_bytes(packed_len)));
  cudaError_t ce = cudaSuccess;
  rc = launch::index_stream(d_packed, packed_len, d_block_off, max_blocks, n_blocks, c->index.p, (cudaStream_t)stream,
                            &ce);
  if (rc < 0) return cuda_fail(ce);
  return rc;
}

int utl_set_knob(int knob, int value) {
  if (knob == UTL_KNOB_HOST_PIPELINE) {
    if (value < 0 || value > 2) return UTL_ERR_ARG;
    g_host_pipe.store(value, std::memory_order_relaxed);
    return UTL_OK;
  }
  return launch::set_knob(knob, value) == 0 ? UTL_OK : UTL_ERR_ARG;
}
int utl_get_knob(int knob) {
  if (knob == UTL_KNOB_HOST_PIPELINE) return g_host_pipe.load(std::memory_order_relaxed);
  return launch::get_knob(knob);
}

uint64_t utl_launch_count(void) { return g_launches.load(std::memory_order_relaxed); }
int utl_last_cuda_error(void) { return t_last_cuda; }
const char* utl_version(void) { return "utlpfor-b200 0.1 (sm_100a)"; }

}  // extern "C"
