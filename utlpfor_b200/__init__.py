"""utlpfor_b200 -- the UTL-PFOR block codec on NVIDIA B200 (sm_100a).

Python mirror of the Go API of github.com/Akron/utlpfor (names, argument
meaning and errors kept), running every pack/unpack/get on the GPU through
the C ABI of libutlpfor_b200.so.  Go returns (value, error); here the value
is returned and the error is raised as the exception class of the same
name.  Batched device entry points (pack_batch, unpack_batch, get_batch)
work on torch CUDA tensors.
"""
import ctypes as C

import numpy as np

from ._lib import load

__all__ = [
    "Delta", "NoFOR", "NoPatch", "Special", "Append", "NoInPlace",
    "UTLError", "ErrInvalidBuffer", "ErrPositionOutOfRange", "ErrInvalidBlockLength",
    "ErrInvalidFlags", "ErrUnsupportedType", "ErrNotImplemented", "ErrOverflow",
    "PackUint32", "UnpackUint32", "GetUint32", "PackUint64", "UnpackUint64", "GetUint64",
    "BlockLength", "Header", "MaxBlockLength32", "MaxBlockLength64",
    "ScratchLen", "ScratchLenNoInPlace", "ScratchLen64",
    "Compressor32", "Compressor64", "NewUint32", "NewUint64", "CompressorPool",
]

# Flags, utlpfor.go:24-68
Delta, NoFOR, NoPatch, Special, Append, NoInPlace = 1, 2, 4, 8, 16, 32
# scratch sizes of the reference API (pack.go:5-12, uint64.go:15); accepted, unused
ScratchLen, ScratchLenNoInPlace, ScratchLen64 = 128, 256, 384


class UTLError(Exception):
    code = -1


class ErrInvalidBuffer(UTLError):
    code = 1


class ErrPositionOutOfRange(UTLError):
    code = 2


class ErrInvalidBlockLength(UTLError):
    code = 3


class ErrInvalidFlags(UTLError):
    code = 4


class ErrUnsupportedType(UTLError):
    code = 5


class ErrNotImplemented(UTLError):
    code = 6


class ErrOverflow(UTLError):
    """Delta decode wrapped past 2^32 at flat index Position (utlpfor.go:108)."""
    code = 7

    def __init__(self, position):
        super().__init__("UTLpfor: delta decode overflow at index %d" % position)
        self.Position = position


class BatchError(UTLError):
    """Error of a batched call that has no reference counterpart."""


_ERR = {c.code: c for c in (ErrInvalidBuffer, ErrPositionOutOfRange, ErrInvalidBlockLength,
                            ErrInvalidFlags, ErrUnsupportedType, ErrNotImplemented)}
_MSG = {1: "UTLpfor: invalid buffer", 2: "UTLpfor: position out of range",
        3: "UTLpfor: invalid block length", 4: "UTLpfor: invalid header flags",
        5: "UTLpfor: unsupported integer type", 6: "UTLpfor: not implemented",
        8: "block count or length disagrees with the stream table", 9: "output capacity too small",
        10: "device wait timed out", 11: "invalid argument", 12: "CUDA error",
        13: "batch exceeds the built-in scratch of the no-allocation pack"}


def _raise(code, ovf=0):
    if code == 0:
        return
    if code == 7:
        raise ErrOverflow(ovf)
    if code in _ERR:
        raise _ERR[code](_MSG[code])
    msg = _MSG.get(code, "error %d" % code)
    if code == 12:
        msg += " (cudaError %d)" % load().utl_last_cuda_error()
    raise BatchError(msg)


def _u8(src):
    b = np.frombuffer(bytes(src), dtype=np.uint8) if not isinstance(src, np.ndarray) else \
        np.ascontiguousarray(src, dtype=np.uint8)
    return b, b.ctypes.data_as(C.POINTER(C.c_uint8))


def _pack(is64, flag, values, dst, codec=None, kind="codec"):
    L = load()
    dt, P = (np.uint64, C.c_uint64) if is64 else (np.uint32, C.c_uint32)
    v = np.ascontiguousarray(values, dtype=dt)
    cap = L.utl_max_block_length64(flag) if is64 else L.utl_max_block_length32(flag)
    out = np.zeros(cap, dtype=np.uint8)
    n = C.c_size_t(0)
    args = (flag & 0xFF, v.ctypes.data_as(C.POINTER(P)), len(v), out.ctypes.data_as(C.POINTER(C.c_uint8)),
            cap, C.byref(n))
    if codec is not None:
        rc = getattr(L, "utl_%s_pack_%s" % (kind, "u64" if is64 else "u32"))(codec, *args)
    else:
        rc = (L.utl_pack_u64 if is64 else L.utl_pack_u32)(*args)
    _raise(rc)
    block = bytes(out[:n.value])
    if flag & Append:
        # pack.go:14-55: the block goes after the existing content of dst
        base = bytearray(dst) if dst is not None else bytearray()
        base += block
        return base
    return bytearray(block)


def _unpack(is64, src, codec=None, kind="codec"):
    L = load()
    b, p = _u8(src)
    dt, P = (np.uint64, C.c_uint64) if is64 else (np.uint32, C.c_uint32)
    out = np.zeros(128, dtype=dt)
    cnt, cons, ovf = C.c_int(0), C.c_size_t(0), C.c_int(0)
    args = (p, len(b), out.ctypes.data_as(C.POINTER(P)), C.byref(cnt), C.byref(cons), C.byref(ovf))
    if codec is not None:
        rc = getattr(L, "utl_%s_unpack_%s" % (kind, "u64" if is64 else "u32"))(codec, *args)
    else:
        rc = (L.utl_unpack_u64 if is64 else L.utl_unpack_u32)(*args)
    _raise(rc, ovf.value)
    return out[:cnt.value].copy(), cons.value


def _get(is64, pos, src, codec=None, kind="codec"):
    L = load()
    b, p = _u8(src)
    val = C.c_uint64(0) if is64 else C.c_uint32(0)
    ovf = C.c_int(0)
    args = (int(pos), p, len(b), C.byref(val), C.byref(ovf))
    if codec is not None:
        rc = getattr(L, "utl_%s_get_%s" % (kind, "u64" if is64 else "u32"))(codec, *args)
    else:
        rc = (L.utl_get_u64 if is64 else L.utl_get_u32)(*args)
    _raise(rc, ovf.value)
    return val.value


def PackUint32(flag, values, dst=None, scratch=None):
    """PackUint32 (pack.go:76): returns the packed block (after dst's content with Append)."""
    return _pack(False, flag, values, dst)


def UnpackUint32(src, values=None, scratch=None):
    """UnpackUint32 (unpack.go:5): returns (values, consumed)."""
    return _unpack(False, src)


def GetUint32(pos, src, scratch=None):
    """GetUint32 (get.go:74)."""
    return _get(False, pos, src)


def PackUint64(flag, values, dst=None, scratch=None):
    """PackUint64 (uint64.go:279)."""
    return _pack(True, flag, values, dst)


def UnpackUint64(src, values=None, scratch=None):
    """UnpackUint64 (uint64.go:338): returns (values, consumed)."""
    return _unpack(True, src)


def GetUint64(pos, src, scratch=None):
    """GetUint64 (uint64.go:364)."""
    return _get(True, pos, src)


def BlockLength(src):
    """BlockLength (block_length.go:8)."""
    b, p = _u8(src)
    n = C.c_size_t(0)
    _raise(load().utl_block_length(p, len(b), C.byref(n)))
    return n.value


def Header(src):
    """Header (header.go:135): (count, bitWidth, excCount, hasDelta, hasFOR, hasZigZag, hasSpecial)."""
    b, p = _u8(src)
    f = [C.c_int(0) for _ in range(7)]
    _raise(load().utl_header(p, len(b), *[C.byref(x) for x in f]))
    c, bw, e, d, fo, z, s = [x.value for x in f]
    return c, bw, e, bool(d), bool(fo), bool(z), bool(s)


def MaxBlockLength32(flag):
    return load().utl_max_block_length32(flag & 0xFF)


def MaxBlockLength64(flag):
    return load().utl_max_block_length64(flag & 0xFF)


class _Codec:
    _is64 = False

    def __init__(self):
        h = C.c_void_p()
        _raise(load().utl_codec_new(1 if self._is64 else 0, C.byref(h)))
        self._h = h

    def __del__(self):
        h = getattr(self, "_h", None)
        if h:
            load().utl_codec_free(h)
            self._h = None

    def Compress(self, flags, dst, values):
        return _pack(self._is64, flags, values, dst, self._h)

    def Decompress(self, dst, src):
        return _unpack(self._is64, src, self._h)

    def Get(self, pos, src):
        return _get(self._is64, pos, src, self._h)


class Compressor32(_Codec):
    """Compressor32 (compressor.go:16): owns its own CUDA stream and staging."""
    _is64 = False


class Compressor64(_Codec):
    """Compressor64 (compressor.go:63)."""
    _is64 = True


class CompressorPool:
    """A pool of per-call GPU contexts shared by any number of threads.

    The reference's Compressor32/64 must not be used concurrently
    (compressor.go:8,63); a server calling from many threads would keep one
    per thread or a pool of them.  This is that pool: n contexts, each with
    its own CUDA stream and mapped pinned staging; every call takes a free
    one, so calls from different threads overlap on the GPU.  Methods are
    thread-safe and return exactly what PackUint32/UnpackUint32/GetUint32
    (and the 64-bit forms) return."""

    def __init__(self, n_contexts=8):
        h = C.c_void_p()
        _raise(load().utl_pool_new(int(n_contexts), C.byref(h)))
        self._h = h
        self.n_contexts = int(n_contexts)

    def close(self):
        h = getattr(self, "_h", None)
        if h:
            load().utl_pool_free(h)
            self._h = None

    def __del__(self):
        self.close()

    def PackUint32(self, flag, values, dst=None):
        return _pack(False, flag, values, dst, self._h, "pool")

    def UnpackUint32(self, src):
        return _unpack(False, src, self._h, "pool")

    def GetUint32(self, pos, src):
        return _get(False, pos, src, self._h, "pool")

    def PackUint64(self, flag, values, dst=None):
        return _pack(True, flag, values, dst, self._h, "pool")

    def UnpackUint64(self, src):
        return _unpack(True, src, self._h, "pool")

    def GetUint64(self, pos, src):
        return _get(True, pos, src, self._h, "pool")


def NewUint32():
    return Compressor32()


def NewUint64():
    return Compressor64()


from .batch import (BatchCodec, PackedBatch, get_batch, index_stream, pack_batch, pack_streams, plan,  # noqa: E402
                    unpack_batch, unpack_streams)
