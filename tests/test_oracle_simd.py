"""The vectorized CPU pipelines (AVX-512 and AVX2 restatements of the
reference's packBlockAVX512 / unpackBlockAVX512, oracle/utl_simd.c) give
the scalar restatement's bytes, values and error classes for every input,
as the reference's SIMD and scalar paths do (fuzz_simd_test.go:13-40).
The vectorized pipelines are the timed CPU baseline; the scalar one is
pinned to the reference's golden data (test_oracle_golden.py)."""
import json
import os

import numpy as np
import pytest

import oracle_ref as O
from gen import KINDS32, KINDS64, block_values, block_values64, streams

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
LEVELS = [lv for lv in (2, 1) if lv <= O.simd_level()]


@pytest.fixture(params=LEVELS, ids=lambda lv: {2: "avx512", 1: "avx2"}[lv])
def level(request):
    have = O.simd_level()
    O.simd_level(request.param)
    yield request.param
    O.simd_level(have)


def test_cpu_has_a_vector_level():
    assert O.simd_level() >= 1


def test_golden_blocks(level):
    for g in GOLDEN["golden_blocks"]:
        blk, err = O.pack_u32(g["flag"], np.array(g["values"], dtype=np.uint32), simd=True)
        assert err == 0 and blk.hex() == g["packed_hex"], g["name"]
        v, c, err, _ = O.unpack_u32(bytes.fromhex(g["packed_hex"]), simd=True)
        assert err == 0 and list(v) == g["values"]


@pytest.mark.parametrize("flag", range(16))
def test_u32_blocks_match_scalar(level, flag):
    rng = np.random.default_rng(700 + flag)
    for kind in KINDS32:
        for n in (1, 2, 15, 16, 17, 31, 64, 100, 127, 128, 128, 128):
            v = block_values(rng, n, kind)
            want, werr = O.pack_u32(flag, v)
            got, gerr = O.pack_u32(flag, v, simd=True)
            assert (got, gerr) == (want, werr), (kind, n)
            wv, wc, werr, wovf = O.unpack_u32(want)
            gv, gc, gerr, govf = O.unpack_u32(want, simd=True)
            assert (gc, gerr, govf) == (wc, werr, wovf)
            assert np.array_equal(gv, wv)


@pytest.mark.parametrize("flag", [0, 1, 2, 3, 4, 5, 9, 13])
def test_u64_blocks_match_scalar(level, flag):
    rng = np.random.default_rng(800 + flag)
    for kind in KINDS64:
        for n in (1, 16, 77, 128):
            v = block_values64(rng, n, kind)
            want, werr = O.pack_u64(flag, v)
            got, gerr = O.pack_u64(flag, v, simd=True)
            assert (got, gerr) == (want, werr), (kind, n)
            wv, wc, werr, wovf = O.unpack_u64(want)
            gv, gc, gerr, govf = O.unpack_u64(want, simd=True)
            assert (gc, gerr, govf) == (wc, werr, wovf)
            assert np.array_equal(gv, wv)


def test_corrupt_and_overflow_match_scalar(level):
    """Damaged blocks and delta overflows: the same error class and
    overflow position from both pipelines."""
    rng = np.random.default_rng(42)
    for flag in (0, 1, 3, 5):
        for kind in ("exc", "dense_exc", "sorted", "walk", "full"):
            v = block_values(rng, 128, kind)
            blk, _ = O.pack_u32(flag, v)
            for _ in range(60):
                b = bytearray(blk)
                i = int(rng.integers(0, len(b)))
                b[i] ^= int(rng.integers(1, 256))
                cut = int(rng.integers(0, len(b) + 1)) if rng.random() < 0.3 else len(b)
                b = bytes(b[:cut])
                wv, wc, werr, wovf = O.unpack_u32(b)
                gv, gc, gerr, govf = O.unpack_u32(b, simd=True)
                assert (gc, gerr, govf) == (wc, werr, wovf)
                if werr == 0:
                    assert np.array_equal(gv, wv)
    # every overflow position of a full delta block
    for pos in range(16, 128):
        v = np.zeros(128, dtype=np.uint32)
        v[pos - 16] = 0xFFFFFFF0
        v[pos] = 0x20
        blk, err = O.pack_u32(O.DELTA | O.NOFOR, v)
        assert err == 0
        b = bytearray(blk)
        h = int.from_bytes(b[:4], "little") & ~(1 << 23)  # clear zigzag: the wrap becomes an overflow
        b[:4] = h.to_bytes(4, "little")
        assert O.unpack_u32(bytes(b), simd=True)[2:] == O.unpack_u32(bytes(b))[2:]


@pytest.mark.parametrize("is64", [False, True])
def test_streams_match_scalar(level, is64):
    rng = np.random.default_rng(9)
    lens = [1, 128, 300, 0, 257, 1000, 5, 129, 4096, 77]
    for kind in (("exc", "sorted", "walk") if not is64 else ("for64", "full", "walk")):
        vals, vo = streams(rng, lens, kind, is64=is64)
        for flag in (0, 1, 4):
            want, wbo, wso = O.pack_streams(flag, vals, vo)
            got, gbo, gso = O.pack_streams(flag, vals, vo, n_threads=3, simd=True)
            assert got.tobytes() == want.tobytes()
            assert np.array_equal(gbo, wbo) and np.array_equal(gso, wso)
            out, err = O.unpack_streams(want, wbo, vo, dtype=vals.dtype, n_threads=3, simd=True)
            assert err == 0 and np.array_equal(out, vals)
