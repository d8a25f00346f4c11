"""Batched device API: one launch packs, unpacks or queries all blocks of
many streams of uneven length.  Tensors are torch CUDA tensors used as raw
device memory (uint32/uint64 data carried in int32/int64 tensors is fine);
work is enqueued on torch's current CUDA stream.

A batch is described by a stream table val_off (n_streams+1 value offsets):
stream s holds values[val_off[s]:val_off[s+1]] and packs into
ceil(n_s/128) blocks laid out back to back, exactly as repeated
PackUint32(flag|Append, block, ...) calls lay them out (pack.go:76-97).
"""
import ctypes as C
from dataclasses import dataclass

import numpy as np

from ._lib import load

_ERRBITS = {8: "block count or length disagrees with the stream table", 9: "output capacity too small",
            10: "device wait timed out"}


def _torch():
    import torch
    return torch


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def _stream():
    return C.c_void_p(_torch().cuda.current_stream().cuda_stream)


def _check(rc):
    if rc != 0:
        from . import _raise
        _raise(rc)


def count_blocks(val_off_host):
    vo = np.ascontiguousarray(val_off_host, dtype=np.uint64)
    n = load().utl_count_blocks(vo.ctypes.data_as(C.POINTER(C.c_uint64)), len(vo) - 1)
    if n < 0:
        raise ValueError("stream table must be non-decreasing")
    return int(n)


@dataclass
class PackedBatch:
    packed: object          # uint8 tensor (capacity >= packed_len)
    block_off: object       # int64 tensor, n_blocks+1
    stream_byte_off: object  # int64 tensor, n_streams+1
    val_off: object         # int64 tensor, n_streams+1
    block_start: object     # int64 tensor, n_streams+1
    n_streams: int
    n_blocks: int
    is64: bool
    err: object = None      # int32 tensor, error bits of the pack

    @property
    def packed_len(self):
        return int(self.block_off[self.n_blocks].item())


def plan(val_off):
    """block_start[s] = blocks of streams before s (device, int64)."""
    torch = _torch()
    n = val_off.numel() - 1
    bs = torch.empty(n + 1, dtype=torch.int64, device=val_off.device)
    _check(load().utl_batch_plan(_ptr(val_off), n, _ptr(bs), _stream()))
    return bs


def pack_batch(values, val_off, flag=0, n_blocks=None, out=None, block_start=None, is64=None, check=True):
    """Pack every stream; returns a PackedBatch.

    values: CUDA tensor (int32/uint32 -> PackUint32, int64/uint64 -> PackUint64).
    val_off: host array or CUDA int64 tensor of n_streams+1 offsets.  With a
    CUDA tensor n_blocks must be given.  check=True synchronizes and raises
    on device-reported errors.
    """
    torch = _torch()
    dev = values.device
    if is64 is None:
        is64 = values.element_size() == 8
    if not isinstance(val_off, torch.Tensor):
        vo_host = np.ascontiguousarray(val_off, dtype=np.uint64)
        n_blocks = count_blocks(vo_host)
        val_off = torch.from_numpy(vo_host.view(np.int64)).to(dev)
    elif n_blocks is None:
        n_blocks = count_blocks(val_off.cpu().numpy().view(np.uint64))
    n = val_off.numel() - 1
    L = load()
    if block_start is None:
        block_start = plan(val_off)
    maxb = L.utl_max_block_length64(flag) if is64 else L.utl_max_block_length32(flag)
    if out is None:
        out = torch.empty(max(n_blocks * maxb, 16), dtype=torch.uint8, device=dev)
    block_off = torch.empty(n_blocks + 1, dtype=torch.int64, device=dev)
    sbo = torch.empty(n + 1, dtype=torch.int64, device=dev)
    sbytes = L.utl_pack_scratch_bytes(n_blocks)
    scratch = torch.empty(max(sbytes, 16), dtype=torch.uint8, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    fn = L.utl_pack_batch_u64 if is64 else L.utl_pack_batch_u32
    _check(fn(flag & 0xFF, _ptr(values), _ptr(val_off), _ptr(block_start), n, n_blocks, _ptr(out), out.numel(),
              _ptr(block_off), _ptr(sbo), _ptr(scratch), sbytes, _ptr(err), _stream()))
    pb = PackedBatch(out, block_off, sbo, val_off, block_start, n, n_blocks, is64, err)
    if check:
        bits = int(err.item())
        for code, msg in _ERRBITS.items():
            if bits & (1 << code):
                from . import BatchError
                raise BatchError(msg)
    return pb


def unpack_batch(pb, out=None, block_status=None, check=True, packed=None, block_off=None):
    """Unpack every block of a PackedBatch (or of packed/block_off given
    explicitly with pb's stream table).  Returns the values tensor."""
    torch = _torch()
    packed = pb.packed if packed is None else packed
    block_off = pb.block_off if block_off is None else block_off
    dev = packed.device
    total = None
    if out is None:
        total = int(pb.val_off[pb.n_streams].item())
        out = torch.empty(max(total, 1), dtype=torch.int64 if pb.is64 else torch.int32, device=dev)
    err = torch.zeros(1, dtype=torch.int32, device=dev)
    L = load()
    fn = L.utl_unpack_batch_u64 if pb.is64 else L.utl_unpack_batch_u32
    _check(fn(_ptr(packed), packed.numel(), _ptr(block_off), _ptr(pb.val_off), _ptr(pb.block_start), pb.n_streams,
              pb.n_blocks, _ptr(out), _ptr(block_status), _ptr(err), _stream()))
    if check:
        bits = int(err.item())
        if bits:
            from . import _raise
            code = min(c for c in range(1, 32) if bits & (1 << c))
            _raise(code)
    return out if total is None else out[:total]


def get_batch(pb, q_stream, q_pos, out=None, status=None):
    """GetUint32/GetUint64 at (stream, position) pairs; returns (values, status)."""
    torch = _torch()
    dev = pb.packed.device
    nq = q_stream.numel()
    if out is None:
        out = torch.empty(max(nq, 1), dtype=torch.int64 if pb.is64 else torch.int32, device=dev)
    if status is None:
        status = torch.empty(max(nq, 1), dtype=torch.int32, device=dev)
    L = load()
    fn = L.utl_get_batch_u64 if pb.is64 else L.utl_get_batch_u32
    _check(fn(_ptr(pb.packed), pb.packed.numel(), _ptr(pb.block_off), _ptr(pb.val_off), _ptr(pb.block_start),
              pb.n_streams, _ptr(q_stream), _ptr(q_pos), nq, _ptr(out), _ptr(status), C.c_void_p(0), _stream()))
    return out[:nq], status[:nq]


def pack_streams(flag, values, val_off):
    """Host-buffer batch: numpy in, numpy out (copies, one batched pass).
    Returns (packed uint8 array, block_off, stream_byte_off)."""
    L = load()
    is64 = values.dtype.itemsize == 8
    v = np.ascontiguousarray(values)
    vo = np.ascontiguousarray(val_off, dtype=np.uint64)
    n = len(vo) - 1
    nb = count_blocks(vo)
    maxb = L.utl_max_block_length64(flag) if is64 else L.utl_max_block_length32(flag)
    out = np.empty(max(nb * maxb, 1), dtype=np.uint8)
    bo = np.zeros(nb + 1, dtype=np.uint64)
    so = np.zeros(n + 1, dtype=np.uint64)
    olen = C.c_size_t(0)
    fn = L.utl_pack_streams_u64 if is64 else L.utl_pack_streams_u32
    _check(fn(flag & 0xFF, C.c_void_p(v.ctypes.data), vo.ctypes.data_as(C.POINTER(C.c_uint64)), n,
              C.c_void_p(out.ctypes.data), out.nbytes, bo.ctypes.data_as(C.POINTER(C.c_uint64)),
              so.ctypes.data_as(C.POINTER(C.c_uint64)), C.byref(olen)))
    return out[:olen.value], bo, so


def unpack_streams(packed, block_off, val_off, is64=False):
    """Host-buffer batch unpack; returns the values array."""
    L = load()
    pk = np.ascontiguousarray(packed, dtype=np.uint8)
    bo = np.ascontiguousarray(block_off, dtype=np.uint64)
    vo = np.ascontiguousarray(val_off, dtype=np.uint64)
    out = np.empty(max(int(vo[-1]), 1), dtype=np.uint64 if is64 else np.uint32)
    fn = L.utl_unpack_streams_u64 if is64 else L.utl_unpack_streams_u32
    _check(fn(C.c_void_p(pk.ctypes.data), pk.nbytes, bo.ctypes.data_as(C.POINTER(C.c_uint64)),
              vo.ctypes.data_as(C.POINTER(C.c_uint64)), len(vo) - 1, C.c_void_p(out.ctypes.data)))
    return out[:int(vo[-1])]


class BatchCodec:
    """Preallocated batch over a fixed stream table: pack() and unpack()
    enqueue work on torch's current stream without allocating, so they can
    run back to back or be captured in a CUDA graph.

    values/out are CUDA tensors of the element size (4 or 8 bytes).
    """

    def __init__(self, val_off_host, flag=0, is64=False, device="cuda", out_cap=None, tuned=True):
        torch = _torch()
        L = load()
        if tuned:
            from .tune import apply
            apply(device)
        vo = np.ascontiguousarray(val_off_host, dtype=np.uint64)
        self.n_streams = len(vo) - 1
        self.n_blocks = count_blocks(vo)
        self.n_values = int(vo[-1])
        self.flag = flag & 0xFF
        self.is64 = is64
        self.val_off = torch.from_numpy(vo.view(np.int64)).to(device)
        self.block_start = plan(self.val_off)
        maxb = L.utl_max_block_length64(flag) if is64 else L.utl_max_block_length32(flag)
        cap = out_cap if out_cap is not None else max(self.n_blocks * maxb, 16)
        self.packed = torch.empty(cap, dtype=torch.uint8, device=device)
        self.block_off = torch.zeros(self.n_blocks + 1, dtype=torch.int64, device=device)
        self.stream_byte_off = torch.zeros(self.n_streams + 1, dtype=torch.int64, device=device)
        self.scratch_bytes = L.utl_pack_scratch_bytes(self.n_blocks)
        self.scratch = torch.empty(max(self.scratch_bytes, 16), dtype=torch.uint8, device=device)
        self.err = torch.zeros(1, dtype=torch.int32, device=device)
        self.block_status = None
        self._pack_fn = L.utl_pack_batch_u64 if is64 else L.utl_pack_batch_u32
        self._unpack_fn = L.utl_unpack_batch_u64 if is64 else L.utl_unpack_batch_u32
        self._get_fn = L.utl_get_batch_u64 if is64 else L.utl_get_batch_u32

    def pack(self, values, stream_offsets=False):
        _check(self._pack_fn(self.flag, _ptr(values), _ptr(self.val_off), _ptr(self.block_start), self.n_streams,
                             self.n_blocks, _ptr(self.packed), self.packed.numel(), _ptr(self.block_off),
                             _ptr(self.stream_byte_off) if stream_offsets else C.c_void_p(0), _ptr(self.scratch),
                             self.scratch_bytes, _ptr(self.err), _stream()))

    def unpack(self, out, block_status=None):
        _check(self._unpack_fn(_ptr(self.packed), self.packed.numel(), _ptr(self.block_off), _ptr(self.val_off),
                               _ptr(self.block_start), self.n_streams, self.n_blocks, _ptr(out),
                               _ptr(block_status), _ptr(self.err), _stream()))

    def get(self, q_stream, q_pos, out, status=None):
        _check(self._get_fn(_ptr(self.packed), self.packed.numel(), _ptr(self.block_off), _ptr(self.val_off),
                            _ptr(self.block_start), self.n_streams, _ptr(q_stream), _ptr(q_pos), q_stream.numel(),
                            _ptr(out), _ptr(status), _ptr(self.err), _stream()))

    def capture(self, values, out):
        """Record pack(values) + unpack(out) into a CUDA graph (one warm-up
        pass runs first so no first-use setup happens during capture);
        returns the torch.cuda.CUDAGraph to replay()."""
        torch = _torch()
        self.pack(values)
        self.unpack(out)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            self.pack(values)
            self.unpack(out)
        return g

    @property
    def packed_len(self):
        return int(self.block_off[self.n_blocks].item())

    def error_bits(self):
        return int(self.err.item())


def index_stream(packed, max_blocks=None):
    """Block offsets of a packed stream without an index (a CUDA uint8
    tensor of whole blocks back to back): the BlockLength walk of
    block_length.go:8-65 done on the device.  Returns an int64 tensor of
    n_blocks + 1 offsets (the last is the stream length); raises the
    reference's error of the first bad block (its index in .block)."""
    torch = _torch()
    L = load()
    nbytes = packed.numel()
    cap = max_blocks if max_blocks is not None else nbytes // 64 + 16
    while True:
        out = torch.empty(cap + 1, dtype=torch.int64, device=packed.device)
        n = C.c_int64(0)
        rc = L.utl_index_stream(_ptr(packed), nbytes, _ptr(out), cap, C.byref(n), _stream())
        if rc == 9 and max_blocks is None:  # capacity: n holds the block count
            cap = n.value
            continue
        if rc != 0:
            from . import _raise
            try:
                _raise(rc)
            except Exception as e:
                e.block = n.value
                raise
        return out[:n.value + 1]
