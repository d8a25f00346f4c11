"""ctypes access to the CPU oracle (oracle/liboracle.so) for the tests.

The oracle is the checker: the tests compare the CUDA library against it.
Builds the oracle with make on first use when the shared object is missing.
"""
import ctypes as C
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ODIR = os.path.join(ROOT, "oracle")
SO = os.path.join(ODIR, "liboracle.so")

OK, INVALID_BUFFER, POS_RANGE, INVALID_BLOCK_LENGTH, INVALID_FLAGS, UNSUPPORTED_TYPE, \
    NOT_IMPLEMENTED, OVERFLOW = range(8)
DELTA, NOFOR, NOPATCH, SPECIAL, APPEND, NOINPLACE = 1, 2, 4, 8, 16, 32

_lib = None


def lib():
    global _lib
    if _lib is None:
        srcs = [os.path.join(ODIR, f) for f in ("utl_oracle.c", "utl_simd.c", "utl_simd_body.inc", "utl_oracle.h",
                                                 "utl_oracle_int.h", "Makefile")]
        if not os.path.exists(SO) or any(os.path.getmtime(SO) < os.path.getmtime(f) for f in srcs):
            subprocess.check_call(["make", "-s", "-C", ODIR])
        L = C.CDLL(SO)
        P8, PU32, PU64, SZ = C.POINTER(C.c_uint8), C.POINTER(C.c_uint32), C.POINTER(C.c_uint64), C.POINTER(C.c_size_t)
        PI = C.POINTER(C.c_int)
        L.utlo_pack_u32.argtypes = [C.c_uint8, PU32, C.c_int, P8, SZ]
        L.utlo_pack_u64.argtypes = [C.c_uint8, PU64, C.c_int, P8, SZ]
        L.utlo_unpack_u32.argtypes = [P8, C.c_size_t, PU32, PI, SZ, PI]
        L.utlo_unpack_u64.argtypes = [P8, C.c_size_t, PU64, PI, SZ, PI]
        L.utlo_get_u32.argtypes = [C.c_int, P8, C.c_size_t, PU32, PI]
        L.utlo_get_u64.argtypes = [C.c_int, P8, C.c_size_t, PU64, PI]
        L.utlo_block_length.argtypes = [P8, C.c_size_t, SZ]
        L.utlo_header.argtypes = [P8, C.c_size_t] + [PI] * 7
        L.utlo_max_block_length32.argtypes = [C.c_uint8]
        L.utlo_max_block_length64.argtypes = [C.c_uint8]
        L.utlo_stream_pack_bound_u32.argtypes = [C.c_uint8, PU64, C.c_int]
        L.utlo_stream_pack_bound_u32.restype = C.c_size_t
        L.utlo_stream_pack_bound_u64.argtypes = [C.c_uint8, PU64, C.c_int]
        L.utlo_stream_pack_bound_u64.restype = C.c_size_t
        L.utlo_pack_streams_u32.argtypes = [C.c_uint8, PU32, PU64, C.c_int, P8, C.c_size_t, PU64, PU64, C.c_int]
        L.utlo_pack_streams_u64.argtypes = [C.c_uint8, PU64, PU64, C.c_int, P8, C.c_size_t, PU64, PU64, C.c_int]
        L.utlo_unpack_streams_u32.argtypes = [P8, PU64, PU64, C.c_int, PU32, C.c_int]
        L.utlo_unpack_streams_u64.argtypes = [P8, PU64, PU64, C.c_int, PU64, C.c_int]
        for pre in ("utlo_simd_",):
            getattr(L, pre + "pack_u32").argtypes = [C.c_uint8, PU32, C.c_int, P8, SZ]
            getattr(L, pre + "pack_u64").argtypes = [C.c_uint8, PU64, C.c_int, P8, SZ]
            getattr(L, pre + "unpack_u32").argtypes = [P8, C.c_size_t, PU32, PI, SZ, PI]
            getattr(L, pre + "unpack_u64").argtypes = [P8, C.c_size_t, PU64, PI, SZ, PI]
            getattr(L, pre + "pack_streams_u32").argtypes = [C.c_uint8, PU32, PU64, C.c_int, P8, C.c_size_t, PU64,
                                                             PU64, C.c_int]
            getattr(L, pre + "pack_streams_u64").argtypes = [C.c_uint8, PU64, PU64, C.c_int, P8, C.c_size_t, PU64,
                                                             PU64, C.c_int]
            getattr(L, pre + "unpack_streams_u32").argtypes = [P8, PU64, PU64, C.c_int, PU32, C.c_int]
            getattr(L, pre + "unpack_streams_u64").argtypes = [P8, PU64, PU64, C.c_int, PU64, C.c_int]
        L.utlo_simd_level.argtypes = []
        L.utlo_simd_set_level.argtypes = [C.c_int]
        PI32 = C.POINTER(C.c_int32)
        L.utlo_get_streams_u32.argtypes = [P8, PU64, PU64, C.c_int, PU32, PU64, C.c_int64, PU32, PI32]
        L.utlo_get_streams_u32.restype = None
        L.utlo_get_streams_u64.argtypes = [P8, PU64, PU64, C.c_int, PU32, PU64, C.c_int64, PU64, PI32]
        L.utlo_get_streams_u64.restype = None
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _bytes(src):
    b = np.frombuffer(bytes(src), dtype=np.uint8).copy()
    if b.size == 0:
        b = np.zeros(1, dtype=np.uint8)[:0]
    return b


def _fn(name, simd):
    return getattr(lib(), ("utlo_simd_" if simd else "utlo_") + name)


def simd_level(level=None):
    """The vectorized pipelines' level (2 AVX-512, 1 AVX2, 0 scalar); with
    an argument, lower it first (None: leave it)."""
    if level is not None:
        return lib().utlo_simd_set_level(level)
    return lib().utlo_simd_level()


def pack_u32(flag, values, simd=False):
    v = np.ascontiguousarray(values, dtype=np.uint32)
    dst = np.zeros(2048, dtype=np.uint8)
    n = C.c_size_t(0)
    err = _fn("pack_u32", simd)(flag, _p(v, C.c_uint32), len(v), _p(dst, C.c_uint8), C.byref(n))
    return (bytes(dst[:n.value]) if err == 0 else None), err


def pack_u64(flag, values, simd=False):
    v = np.ascontiguousarray(values, dtype=np.uint64)
    dst = np.zeros(4096, dtype=np.uint8)
    n = C.c_size_t(0)
    err = _fn("pack_u64", simd)(flag, _p(v, C.c_uint64), len(v), _p(dst, C.c_uint8), C.byref(n))
    return (bytes(dst[:n.value]) if err == 0 else None), err


def unpack_u32(src, simd=False):
    b = _bytes(src)
    out = np.zeros(128, dtype=np.uint32)
    cnt, cons, ovf = C.c_int(0), C.c_size_t(0), C.c_int(0)
    err = _fn("unpack_u32", simd)(_p(b, C.c_uint8), len(b), _p(out, C.c_uint32), C.byref(cnt), C.byref(cons), C.byref(ovf))
    if err:
        return None, 0, err, ovf.value
    return out[:cnt.value].copy(), cons.value, 0, 0


def unpack_u64(src, simd=False):
    b = _bytes(src)
    out = np.zeros(128, dtype=np.uint64)
    cnt, cons, ovf = C.c_int(0), C.c_size_t(0), C.c_int(0)
    err = _fn("unpack_u64", simd)(_p(b, C.c_uint8), len(b), _p(out, C.c_uint64), C.byref(cnt), C.byref(cons), C.byref(ovf))
    if err:
        return None, 0, err, ovf.value
    return out[:cnt.value].copy(), cons.value, 0, 0


def get_u32(pos, src):
    b = _bytes(src)
    v, ovf = C.c_uint32(0), C.c_int(0)
    err = lib().utlo_get_u32(pos, _p(b, C.c_uint8), len(b), C.byref(v), C.byref(ovf))
    return (v.value if err == 0 else 0), err, ovf.value


def get_u64(pos, src):
    b = _bytes(src)
    v, ovf = C.c_uint64(0), C.c_int(0)
    err = lib().utlo_get_u64(pos, _p(b, C.c_uint8), len(b), C.byref(v), C.byref(ovf))
    return (v.value if err == 0 else 0), err, ovf.value


def block_length(src):
    b = _bytes(src)
    n = C.c_size_t(0)
    err = lib().utlo_block_length(_p(b, C.c_uint8), len(b), C.byref(n))
    return (n.value if err == 0 else 0), err


def header(src):
    b = _bytes(src)
    f = [C.c_int(0) for _ in range(7)]
    err = lib().utlo_header(_p(b, C.c_uint8), len(b), *[C.byref(x) for x in f])
    return [x.value for x in f], err


def max_block_length32(flag):
    return lib().utlo_max_block_length32(flag)


def max_block_length64(flag):
    return lib().utlo_max_block_length64(flag)


def pack_streams(flag, values, val_off, n_threads=4, simd=False, out=None, bo=None, want_so=True):
    """Returns (packed bytes ndarray, block_off, stream_byte_off).  simd:
    through the vectorized pipelines (the same bytes).  out / bo: buffers
    to reuse (capacity at least the stream bound / n_blocks + 1)."""
    is64 = values.dtype == np.uint64
    L = lib()
    vo = np.ascontiguousarray(val_off, dtype=np.uint64)
    ns = len(vo) - 1
    bound_fn = L.utlo_stream_pack_bound_u64 if is64 else L.utlo_stream_pack_bound_u32
    cap = bound_fn(flag, _p(vo, C.c_uint64), ns)
    if out is None or out.size < cap:
        out = np.empty(max(cap, 1), dtype=np.uint8)
    nb = int(np.sum((vo[1:] - vo[:-1] + np.uint64(127)) // np.uint64(128))) if ns else 0
    if bo is None or bo.size < nb + 1:
        bo = np.zeros(nb + 1, dtype=np.uint64)
    so = np.zeros(ns + 1, dtype=np.uint64) if want_so else None
    pso = _p(so, C.c_uint64) if want_so else None
    if is64:
        err = _fn("pack_streams_u64", simd)(flag, _p(values, C.c_uint64), _p(vo, C.c_uint64), ns, _p(out, C.c_uint8),
                                            cap, _p(bo, C.c_uint64), pso, n_threads)
    else:
        err = _fn("pack_streams_u32", simd)(flag, _p(values, C.c_uint32), _p(vo, C.c_uint64), ns, _p(out, C.c_uint8),
                                            cap, _p(bo, C.c_uint64), pso, n_threads)
    assert err == 0, err
    return out[:int(bo[nb])], bo[:nb + 1], so


def unpack_streams(packed, block_off, val_off, dtype=np.uint32, n_threads=4, simd=False, out=None):
    L = lib()
    vo = np.ascontiguousarray(val_off, dtype=np.uint64)
    bo = np.ascontiguousarray(block_off, dtype=np.uint64)
    pk = np.ascontiguousarray(packed, dtype=np.uint8)
    if out is None:
        out = np.zeros(int(vo[-1]), dtype=dtype)
    if dtype == np.uint64:
        err = _fn("unpack_streams_u64", simd)(_p(pk, C.c_uint8), _p(bo, C.c_uint64), _p(vo, C.c_uint64), len(vo) - 1,
                                              _p(out, C.c_uint64), n_threads)
    else:
        err = _fn("unpack_streams_u32", simd)(_p(pk, C.c_uint8), _p(bo, C.c_uint64), _p(vo, C.c_uint64), len(vo) - 1,
                                              _p(out, C.c_uint32), n_threads)
    return out, err


def get_streams(packed, block_off, val_off, q_stream, q_pos, is64=False):
    """GetUint32/GetUint64 per (stream, position) query over packed
    streams: (values, status = error | overflow position << 8)."""
    L = lib()
    vo = np.ascontiguousarray(val_off, dtype=np.uint64)
    bo = np.ascontiguousarray(block_off, dtype=np.uint64)
    pk = np.ascontiguousarray(packed, dtype=np.uint8)
    qs = np.ascontiguousarray(q_stream, dtype=np.uint32)
    qp = np.ascontiguousarray(q_pos, dtype=np.uint64)
    out = np.zeros(qs.size, dtype=np.uint64 if is64 else np.uint32)
    st = np.zeros(qs.size, dtype=np.int32)
    fn = L.utlo_get_streams_u64 if is64 else L.utlo_get_streams_u32
    fn(_p(pk, C.c_uint8), _p(bo, C.c_uint64), _p(vo, C.c_uint64), len(vo) - 1, _p(qs, C.c_uint32),
       _p(qp, C.c_uint64), qs.size, _p(out, C.c_uint64 if is64 else C.c_uint32), _p(st, C.c_int32))
    return out, st


def index_stream(packed):
    """The caller's BlockLength walk over a packed stream (block_length.go:
    8-65, example_test.go:171-186): (offsets incl. the end, error code,
    index of the bad block).  A block running past the end is
    ErrInvalidBuffer, as the caller's Unpack of it would report."""
    pk = np.ascontiguousarray(packed, dtype=np.uint8)
    L = lib()
    offs, pos = [], 0
    n = C.c_size_t(0)
    while pos < pk.size:
        sub = pk[pos:]
        err = L.utlo_block_length(_p(sub, C.c_uint8), sub.size, C.byref(n))
        if err == 0 and pos + n.value > pk.size:
            err = INVALID_BUFFER
        if err != 0:
            return offs, err, len(offs)
        offs.append(pos)
        pos += n.value
    offs.append(pos)
    return offs, OK, len(offs) - 1
