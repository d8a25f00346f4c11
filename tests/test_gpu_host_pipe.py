"""GPU parity of the host-buffer batch calls (utl_pack_streams_*,
utl_unpack_streams_*) in every UTL_KNOB_HOST_PIPELINE mode: the batch cut
into pieces at block boundaries, with overlapped copies, must give the same
bytes, block offsets, stream offsets, values and error codes as one pass
and as the oracle."""
import ctypes as C

import numpy as np
import pytest

import oracle_ref as O
from gen import streams

pytestmark = pytest.mark.gpu

KNOB = 3  # UTL_KNOB_HOST_PIPELINE
ERR_CAPACITY = 9
P64 = C.POINTER(C.c_uint64)


@pytest.fixture(scope="module")
def L():
    import torch

    from utlpfor_b200._lib import load
    assert torch.cuda.is_available()
    return load()


@pytest.fixture(params=[0, 1, 2], ids=["one_pass", "auto", "eighths"])
def mode(L, request):
    old = L.utl_get_knob(KNOB)
    assert L.utl_set_knob(KNOB, request.param) == 0
    yield request.param
    L.utl_set_knob(KNOB, old)


def set_mode(L, m):
    assert L.utl_set_knob(KNOB, m) == 0


def c_pack(L, flag, vals, vo, cap=None):
    is64 = vals.dtype.itemsize == 8
    vo = np.ascontiguousarray(vo, dtype=np.uint64)
    ns = len(vo) - 1
    nb = L.utl_count_blocks(vo.ctypes.data_as(P64), ns)
    maxb = L.utl_max_block_length64(flag) if is64 else L.utl_max_block_length32(flag)
    if cap is None:
        cap = max(nb * maxb, 1)
    out = np.zeros(max(cap, 1), dtype=np.uint8)
    bo = np.zeros(nb + 1, dtype=np.uint64)
    so = np.zeros(ns + 1, dtype=np.uint64)
    olen = C.c_size_t(0)
    fn = L.utl_pack_streams_u64 if is64 else L.utl_pack_streams_u32
    rc = fn(flag, C.c_void_p(vals.ctypes.data), vo.ctypes.data_as(P64), ns, C.c_void_p(out.ctypes.data), cap,
            bo.ctypes.data_as(P64), so.ctypes.data_as(P64), C.byref(olen))
    return rc, out[:min(olen.value, cap)], bo, so, olen.value


def c_unpack(L, packed, bo, vo, dtype):
    vo = np.ascontiguousarray(vo, dtype=np.uint64)
    bo = np.ascontiguousarray(bo, dtype=np.uint64)
    pk = np.ascontiguousarray(packed, dtype=np.uint8)
    out = np.zeros(max(int(vo[-1]), 1), dtype=dtype)
    fn = L.utl_unpack_streams_u64 if dtype == np.uint64 else L.utl_unpack_streams_u32
    rc = fn(C.c_void_p(pk.ctypes.data), pk.nbytes, bo.ctypes.data_as(P64), vo.ctypes.data_as(P64), len(vo) - 1,
            C.c_void_p(out.ctypes.data))
    return rc, out[:int(vo[-1])]


# ragged streams; the long ones get cut inside when the batch is in eighths
LENS = [1, 128, 300, 0, 257, 5000, 5, 129, 0, 4096, 77, 3001, 640]


@pytest.mark.parametrize("is64,kind,flag", [(False, "exc", 0), (False, "sorted", 1), (False, "walk", 6),
                                            (True, "walk", 1), (True, "full", 0)])
def test_oracle_parity(L, mode, is64, kind, flag):
    rng = np.random.default_rng(77)
    vals, vo = streams(rng, LENS, kind, is64=is64)
    want, wbo, wso = O.pack_streams(flag, vals, vo)
    rc, got, bo, so, olen = c_pack(L, flag, vals, vo)
    assert rc == 0 and olen == len(want)
    assert got.tobytes() == want.tobytes()
    assert np.array_equal(bo, wbo) and np.array_equal(so, wso)
    rc, out = c_unpack(L, got, bo, vo, vals.dtype)
    assert rc == 0 and np.array_equal(out, vals)


def test_offset_table_not_at_zero(L, mode):
    """A stream table that starts inside the value array packs and unpacks
    the named range only."""
    rng = np.random.default_rng(5)
    vals, vo = streams(rng, LENS, "exc")
    pad = 333
    big = np.concatenate([rng.integers(0, 2**32, pad, dtype=np.uint64).astype(np.uint32), vals])
    vo2 = vo + np.uint64(pad)
    want, wbo, wso = O.pack_streams(2, vals, vo)
    rc, got, bo, so, _ = c_pack(L, 2, big, vo2)
    assert rc == 0 and got.tobytes() == want.tobytes()
    assert np.array_equal(bo, wbo) and np.array_equal(so, wso)
    rc, out = c_unpack(L, got, bo, vo2, np.uint32)
    assert rc == 0 and np.array_equal(out[pad:], vals)


def test_capacity_error(L, mode):
    rng = np.random.default_rng(9)
    vals, vo = streams(rng, LENS, "exc")
    want, wbo, _ = O.pack_streams(0, vals, vo)
    rc, _, bo, _, olen = c_pack(L, 0, vals, vo, cap=len(want) - 1)
    assert rc == ERR_CAPACITY and olen == len(want)
    assert np.array_equal(bo, wbo)
    rc, got, _, _, olen = c_pack(L, 0, vals, vo, cap=len(want))
    assert rc == 0 and got.tobytes() == want.tobytes()


def test_corrupt_inputs_same_in_every_mode(L):
    """Damaged blocks and offsets that do not rise: the same return code and
    the same values for the blocks that still decode, one pass or pieces."""
    rng = np.random.default_rng(31)
    vals, vo = streams(rng, LENS, "exc")
    packed, bo, _ = O.pack_streams(1, vals, vo)
    nb = len(bo) - 1
    cases = []
    bad = packed.copy()
    b = nb // 2
    bad[int(bo[b]) + 1] ^= 0x1F  # bit width field of one block in the middle
    cases.append((bad, bo))
    bo2 = bo.copy()
    bo2[nb // 3], bo2[nb // 3 + 1] = bo2[nb // 3 + 1], bo2[nb // 3]
    cases.append((packed, bo2))
    bo3 = bo.copy()
    bo3[-2] = bo3[-1] + 5  # past the end of the buffer
    cases.append((packed, bo3))
    old = L.utl_get_knob(KNOB)
    try:
        for pk, offs in cases:
            results = []
            for m in (0, 2):
                set_mode(L, m)
                results.append(c_unpack(L, pk, offs, vo, np.uint32))
            (rc0, out0), (rc2, out2) = results
            assert rc0 == rc2 != 0
            # blocks whose bytes and offsets are intact decode the same
            bl = 0
            for s in range(len(vo) - 1):
                for p in range(int(vo[s]), int(vo[s + 1]), 128):
                    e = min(p + 128, int(vo[s + 1]))
                    intact = (offs[bl] == bo[bl] and offs[bl + 1] == bo[bl + 1]
                              and pk[int(bo[bl]):int(bo[bl + 1])].tobytes() == packed[int(bo[bl]):int(bo[bl + 1])].tobytes())
                    if intact:
                        assert np.array_equal(out0[p:e], vals[p:e]), bl
                        assert np.array_equal(out2[p:e], vals[p:e]), bl
                    bl += 1
    finally:
        set_mode(L, old)


@pytest.mark.parametrize("flag", [0, 1])
def test_large_batch_pieces_match_one_pass(L, flag):
    """About 40 M values over 400 ragged streams (160 MB: the default mode
    cuts it into pieces, some inside streams): every output is the same as
    one pass, and the values come back."""
    import hashlib
    rng = np.random.default_rng(4242)
    lens = rng.integers(1, 200000, 400)
    vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    n = int(vo[-1])
    v = rng.integers(0, 2**8, n, dtype=np.uint32)
    m = rng.random(n) < 0.02
    v[m] = rng.integers(2**8, 2**32, int(m.sum()), dtype=np.uint64).astype(np.uint32)
    old = L.utl_get_knob(KNOB)
    try:
        res = {}
        for md in (0, 1):
            set_mode(L, md)
            rc, got, bo, so, _ = c_pack(L, flag, v, vo)
            assert rc == 0
            res[md] = (hashlib.sha256(got.tobytes()).digest(), bo, so)
            rc, out = c_unpack(L, got, bo, vo, np.uint32)
            assert rc == 0 and np.array_equal(out, v)
        assert res[0][0] == res[1][0]
        assert np.array_equal(res[0][1], res[1][1]) and np.array_equal(res[0][2], res[1][2])
    finally:
        set_mode(L, old)


def test_knob_range(L):
    old = L.utl_get_knob(KNOB)
    assert old == 1
    assert L.utl_set_knob(KNOB, 3) != 0 and L.utl_set_knob(KNOB, -1) != 0
    assert L.utl_get_knob(KNOB) == old
