"""GPU parity of the per-call drop-in (C ABI through the Go-API mirror)
against the CPU oracle and the reference's golden data: packed bytes
identical, unpacked and Get values identical, identical error classes and
overflow positions on corrupt input (corrupt_test.go, fuzz_simd_test.go)."""
import json
import os

import numpy as np
import pytest

import oracle_ref as O
from gen import KINDS32, KINDS64, block_values, block_values64

pytestmark = pytest.mark.gpu

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))


@pytest.fixture(scope="module")
def U():
    import utlpfor_b200 as U
    return U


def code_of(fn):
    import utlpfor_b200 as U
    try:
        return fn(), 0, 0
    except U.ErrOverflow as e:
        return None, 7, e.Position
    except U.UTLError as e:
        return None, e.code, 0


@pytest.mark.parametrize("g", GOLDEN["golden_blocks"], ids=lambda g: g["name"])
def test_golden_vectors(U, g):
    packed = U.PackUint32(g["flag"], g["values"])
    assert bytes(packed).hex() == g["packed_hex"]
    vals, consumed = U.UnpackUint32(bytes.fromhex(g["packed_hex"]))
    assert list(vals) == g["values"] and consumed == len(packed)
    assert U.BlockLength(packed) == len(packed)
    for pos in range(0, 128, 5):
        assert U.GetUint32(pos, packed) == g["values"][pos]


@pytest.mark.parametrize("ex", GOLDEN["examples"], ids=lambda e: e["name"])
def test_examples(U, ex):
    k = ex["kind"]
    if k == "pack32_len":
        assert len(U.PackUint32(ex["flag"], ex["values"])) == ex["want"]
    elif k == "pack64_len":
        p = U.PackUint64(ex["flag"], ex["values"])
        assert len(p) == ex["want"]
        assert [int(x) for x in U.UnpackUint64(p)[0]] == ex["values"]
        assert U.GetUint64(1, p) == ex["values"][1]
    elif k == "append32_lens":
        dst = bytearray()
        lens = []
        for b in ex["blocks"]:
            before = len(dst)
            dst = U.PackUint32(ex["flag"], b, dst)
            lens.append(len(dst) - before)
        assert lens == ex["want"]
    elif k == "append32_total":
        dst = bytearray()
        for b in ex["blocks"]:
            dst = U.PackUint32(ex["flag"], b, dst)
        assert len(dst) == ex["want"]
    elif k == "skip_blocks":
        dst = bytearray()
        for b in ex["blocks"]:
            dst = U.PackUint32(ex["flag"], b, dst)
        bl = U.BlockLength(dst)
        assert bl == ex["want"]
        assert list(U.UnpackUint32(bytes(dst[bl:]))[0]) == ex["blocks"][1]
    elif k == "header32":
        c, bw, e, d, f, z, s = U.Header(U.PackUint32(ex["flag"], ex["values"]))
        w = ex["want"]
        assert (c, bw, e, d, f) == (w["count"], w["bit_width"], w["exc_count"], w["delta"], w["for"])
    elif k == "max32":
        for f, want in ex["want"].items():
            assert U.MaxBlockLength32(int(f)) == want
    elif k == "max64":
        for f, want in ex["want"].items():
            assert U.MaxBlockLength64(int(f)) == want


@pytest.mark.parametrize("flag", list(range(16)) + [16, 32, 48])
def test_pack_bytes_match_oracle_u32(U, flag):
    rng = np.random.default_rng(4242 + flag)
    for n in (1, 3, 16, 17, 31, 32, 33, 64, 100, 127, 128):
        for kind in KINDS32:
            v = block_values(rng, n, kind)
            want, err = O.pack_u32(flag, v)
            assert err == 0
            got = bytes(U.PackUint32(flag & ~16, v))
            assert got == want, (flag, n, kind)
            vals, cons = U.UnpackUint32(got)
            assert np.array_equal(vals, v) and cons == len(got)
            for pos in (0, n // 2, n - 1):
                assert U.GetUint32(pos, got) == int(v[pos])


@pytest.mark.parametrize("flag", range(8))
def test_pack_bytes_match_oracle_u64(U, flag):
    rng = np.random.default_rng(99 + flag)
    for n in (1, 2, 33, 100, 128):
        for kind in KINDS64:
            v = block_values64(rng, n, kind)
            want, err = O.pack_u64(flag, v)
            assert err == 0
            got = bytes(U.PackUint64(flag, v))
            assert got == want, (flag, n, kind)
            ov, oc, oerr, oovf = O.unpack_u64(want)
            r = code_of(lambda: U.UnpackUint64(got))
            assert r[1] == oerr and r[2] == oovf
            if oerr == 0:
                assert np.array_equal(r[0][0], ov) and r[0][1] == oc
            for pos in (0, n - 1, 77 % n):
                gv, gerr, govf = O.get_u64(pos, want)
                r = code_of(lambda: U.GetUint64(pos, got))
                assert (r[1], r[2]) == (gerr, govf)
                if gerr == 0:
                    assert r[0] == gv


def corruptions(rng, packed, n_flip=40):
    out = [packed[:cut] for cut in range(0, len(packed))]
    for _ in range(n_flip):
        b = bytearray(packed)
        i = int(rng.integers(0, len(b)))
        b[i] ^= int(rng.integers(1, 256))
        out.append(bytes(b))
    return out


def corrupt_targets32(rng):
    t = []
    t.append((0, np.arange(128, dtype=np.uint32) % 200))
    few = (np.arange(128) % 50).astype(np.uint32)
    few[7], few[50] = 0xFFFF0000, 0x00FF0000
    t.append((0, few))
    many = (np.arange(128) % 50).astype(np.uint32)
    for j in range(48):
        many[(j * 11) % 128] = 0xFF000000 | int(rng.integers(0, 0xFFFFFF))
    t.append((0, many))
    t.append((1, (1000 + 3 * np.arange(128)).astype(np.uint32)))
    t.append((1, (1000000 + 3 * np.arange(128)).astype(np.uint32)))
    t.append((1, block_values(rng, 128, "walk")))
    t.append((1, block_values(rng, 128, "exc")))
    t.append((1 | 2, (rng.integers(0, 2**28, 128, dtype=np.uint64) << np.uint64(4)).astype(np.uint32)))
    t.append((0, block_values(rng, 77, "dense_exc")))
    return t


def test_corrupt_u32_matches_oracle(U):
    """corrupt_test.go: truncations at every length and byte flips; the GPU
    path returns the oracle's error class, overflow position and values."""
    rng = np.random.default_rng(7)
    for flag, v in corrupt_targets32(rng):
        packed, err = O.pack_u32(flag, v)
        for data in corruptions(rng, packed):
            ov, oc, oerr, oovf = O.unpack_u32(data)
            r = code_of(lambda: U.UnpackUint32(data))
            assert (r[1], r[2]) == (oerr, oovf), (flag, len(data))
            if oerr == 0:
                assert np.array_equal(r[0][0], ov) and r[0][1] == oc
            for pos in (0, 7, 64, 100, 127):
                gv, gerr, govf = O.get_u32(pos, data)
                r = code_of(lambda: U.GetUint32(pos, data))
                assert (r[1], r[2]) == (gerr, govf), (flag, len(data), pos)
                if gerr == 0:
                    assert r[0] == gv
            bl, berr = O.block_length(data)
            r = code_of(lambda: U.BlockLength(data))
            assert r[1] == berr and (berr or r[0] == bl)


def test_corrupt_u64_matches_oracle(U):
    rng = np.random.default_rng(11)
    for flag in (0, 1):
        for kind in ("for64", "full", "walk", "upper_for"):
            v = block_values64(rng, 128, kind)
            packed, _ = O.pack_u64(flag, v)
            for data in corruptions(rng, packed, 20)[::3]:
                ov, oc, oerr, oovf = O.unpack_u64(data)
                r = code_of(lambda: U.UnpackUint64(data))
                assert (r[1], r[2]) == (oerr, oovf), (flag, kind, len(data))
                if oerr == 0:
                    assert np.array_equal(r[0][0], ov) and r[0][1] == oc
                for pos in (0, 64, 127):
                    gv, gerr, govf = O.get_u64(pos, data)
                    r = code_of(lambda: U.GetUint64(pos, data))
                    assert (r[1], r[2]) == (gerr, govf)
                    if gerr == 0:
                        assert r[0] == gv


def test_fuzz_corpus(U):
    for case in GOLDEN["fuzz_corpus"]:
        data = bytes(case["args"][0])
        for pos in (0, 7, 64, 127):
            assert code_of(lambda: U.GetUint32(pos, data))[1] == O.get_u32(pos, data)[1]
            assert code_of(lambda: U.GetUint64(pos, data))[1] == O.get_u64(pos, data)[1]
        assert code_of(lambda: U.UnpackUint32(data))[1] == O.unpack_u32(data)[2]
        assert code_of(lambda: U.UnpackUint64(data))[1] == O.unpack_u64(data)[2]


def test_overflow_positions(U):
    import struct
    for v in range(1, 8):
        for lane in range(16):
            d = [0] * 128
            d[lane + (v - 1) * 16] = 0xFFFFFFFF
            d[lane + v * 16] = 1
            h = 128 | (8 << 8) | (2 << 13) | (1 << 22)
            payload = bytearray(512)
            for i in range(128):
                struct.pack_into("<I", payload, (i // 16) * 64 + (i % 16) * 4, d[i])
            blk = struct.pack("<I", h) + bytes(payload)
            r = code_of(lambda: U.UnpackUint32(blk))
            assert r[1] == 7 and r[2] == lane + v * 16
            # Get at a deep position of a bw-32 delta block takes the full-unpack path
            r = code_of(lambda: U.GetUint32(127, blk))
            assert (r[1], r[2]) == O.get_u32(127, blk)[1:]


def test_compressor_objects(U):
    c = U.NewUint32()
    vals = [10, 20, 30, 40, 50]
    p = c.Compress(0, None, vals)
    assert list(c.Decompress(None, p)[0]) == vals
    assert c.Get(2, p) == 30
    c64 = U.NewUint64()
    v64 = [10**12, 10**12 + 1, 10**12 + 2]
    p = c64.Compress(0, None, v64)
    assert len(p) == 19 and c64.Get(1, p) == v64[1]
    assert [int(x) for x in c64.Decompress(None, p)[0]] == v64


def test_invalid_lengths(U):
    with pytest.raises(U.ErrInvalidBuffer):
        U.PackUint32(0, [])
    with pytest.raises(U.ErrInvalidBuffer):
        U.PackUint32(0, list(range(129)))
    with pytest.raises(U.ErrInvalidBuffer):
        U.PackUint64(0, [])
