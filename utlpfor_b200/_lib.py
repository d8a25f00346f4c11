"""ctypes binding of libutlpfor_b200.so (include/utlpfor.h).

The library is built in-tree by utlpfor_b200.build.  There is no fallback:
if the shared object is missing or a GPU is absent, calls fail loudly.
"""
import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libutlpfor_b200.so")

P8 = C.POINTER(C.c_uint8)
PU32 = C.POINTER(C.c_uint32)
PU64 = C.POINTER(C.c_uint64)
PI32 = C.POINTER(C.c_int32)
PI = C.POINTER(C.c_int)
SZ = C.POINTER(C.c_size_t)
VP = C.c_void_p

# (name, restype, argtypes) for every symbol of include/utlpfor.h
SIGNATURES = [
    ("utl_pack_u32", C.c_int, [C.c_uint8, PU32, C.c_int, P8, C.c_size_t, SZ]),
    ("utl_unpack_u32", C.c_int, [P8, C.c_size_t, PU32, PI, SZ, PI]),
    ("utl_get_u32", C.c_int, [C.c_int, P8, C.c_size_t, PU32, PI]),
    ("utl_pack_u64", C.c_int, [C.c_uint8, PU64, C.c_int, P8, C.c_size_t, SZ]),
    ("utl_unpack_u64", C.c_int, [P8, C.c_size_t, PU64, PI, SZ, PI]),
    ("utl_get_u64", C.c_int, [C.c_int, P8, C.c_size_t, PU64, PI]),
    ("utl_block_length", C.c_int, [P8, C.c_size_t, SZ]),
    ("utl_header", C.c_int, [P8, C.c_size_t] + [PI] * 7),
    ("utl_max_block_length32", C.c_int, [C.c_uint8]),
    ("utl_max_block_length64", C.c_int, [C.c_uint8]),
    ("utl_codec_new", C.c_int, [C.c_int, C.POINTER(VP)]),
    ("utl_codec_free", None, [VP]),
    ("utl_codec_pack_u32", C.c_int, [VP, C.c_uint8, PU32, C.c_int, P8, C.c_size_t, SZ]),
    ("utl_codec_unpack_u32", C.c_int, [VP, P8, C.c_size_t, PU32, PI, SZ, PI]),
    ("utl_codec_get_u32", C.c_int, [VP, C.c_int, P8, C.c_size_t, PU32, PI]),
    ("utl_codec_pack_u64", C.c_int, [VP, C.c_uint8, PU64, C.c_int, P8, C.c_size_t, SZ]),
    ("utl_codec_unpack_u64", C.c_int, [VP, P8, C.c_size_t, PU64, PI, SZ, PI]),
    ("utl_codec_get_u64", C.c_int, [VP, C.c_int, P8, C.c_size_t, PU64, PI]),
    ("utl_pool_new", C.c_int, [C.c_int, C.POINTER(VP)]),
    ("utl_pool_free", None, [VP]),
    ("utl_pool_pack_u32", C.c_int, [VP, C.c_uint8, PU32, C.c_int, P8, C.c_size_t, SZ]),
    ("utl_pool_unpack_u32", C.c_int, [VP, P8, C.c_size_t, PU32, PI, SZ, PI]),
    ("utl_pool_get_u32", C.c_int, [VP, C.c_int, P8, C.c_size_t, PU32, PI]),
    ("utl_pool_pack_u64", C.c_int, [VP, C.c_uint8, PU64, C.c_int, P8, C.c_size_t, SZ]),
    ("utl_pool_unpack_u64", C.c_int, [VP, P8, C.c_size_t, PU64, PI, SZ, PI]),
    ("utl_pool_get_u64", C.c_int, [VP, C.c_int, P8, C.c_size_t, PU64, PI]),
    ("utl_count_blocks", C.c_int64, [PU64, C.c_int]),
    ("utl_batch_plan", C.c_int, [VP, C.c_int, VP, VP]),
    ("utl_pack_scratch_bytes", C.c_size_t, [C.c_int64]),
    ("utl_pack_batch_u32", C.c_int, [C.c_uint8, VP, VP, VP, C.c_int, C.c_int64, VP, C.c_size_t, VP, VP, VP,
                                     C.c_size_t, VP, VP]),
    ("utl_pack_batch_u64", C.c_int, [C.c_uint8, VP, VP, VP, C.c_int, C.c_int64, VP, C.c_size_t, VP, VP, VP,
                                     C.c_size_t, VP, VP]),
    ("utl_pack_batch_u32_noalloc", C.c_int, [C.c_uint8, VP, VP, VP, C.c_int, C.c_int64, VP, C.c_size_t, VP, VP, VP,
                                             VP]),
    ("utl_pack_batch_u32_noalloc_max_blocks", C.c_int64, []),
    ("utl_unpack_batch_u32", C.c_int, [VP, C.c_size_t, VP, VP, VP, C.c_int, C.c_int64, VP, VP, VP, VP]),
    ("utl_unpack_batch_u64", C.c_int, [VP, C.c_size_t, VP, VP, VP, C.c_int, C.c_int64, VP, VP, VP, VP]),
    ("utl_get_batch_u32", C.c_int, [VP, C.c_size_t, VP, VP, VP, C.c_int, VP, VP, C.c_int64, VP, VP, VP, VP]),
    ("utl_get_batch_u64", C.c_int, [VP, C.c_size_t, VP, VP, VP, C.c_int, VP, VP, C.c_int64, VP, VP, VP, VP]),
    ("utl_pack_streams_u32", C.c_int, [C.c_uint8, VP, PU64, C.c_int, VP, C.c_size_t, PU64, PU64, SZ]),
    ("utl_pack_streams_u64", C.c_int, [C.c_uint8, VP, PU64, C.c_int, VP, C.c_size_t, PU64, PU64, SZ]),
    ("utl_unpack_streams_u32", C.c_int, [VP, C.c_size_t, PU64, PU64, C.c_int, VP]),
    ("utl_unpack_streams_u64", C.c_int, [VP, C.c_size_t, PU64, PU64, C.c_int, VP]),
    ("utl_index_stream", C.c_int, [VP, C.c_size_t, VP, C.c_int64, C.POINTER(C.c_int64), VP]),
    ("utl_set_knob", C.c_int, [C.c_int, C.c_int]),
    ("utl_get_knob", C.c_int, [C.c_int]),
    ("utl_launch_count", C.c_uint64, []),
    ("utl_last_cuda_error", C.c_int, []),
    ("utl_version", C.c_char_p, []),
]

_lib = None


def load():
    """Load (not build) the shared library; raises if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(
                "libutlpfor_b200.so not built; run `python -m utlpfor_b200.build` (needs nvcc)")
        L = C.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib
