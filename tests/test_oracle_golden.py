"""Pins the CPU oracle to the reference's own golden data.

Mirrors format_conformance_test.go:727-790 (golden blocks byte-exact plus
Unpack/BlockLength/Get round trip), the Example known answers of
example_test.go, the overflow position table of
simd_delta_overflow_test.go:177-205, and the corrupt-input error contract
of corrupt_test.go:150-168 on the reference's fuzz corpus.
"""
import json
import os
import struct

import numpy as np
import pytest

import oracle_ref as O

GOLDEN = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "golden.json")))
KNOWN_ERRORS = {O.INVALID_BUFFER, O.POS_RANGE, O.INVALID_BLOCK_LENGTH, O.INVALID_FLAGS,
                O.UNSUPPORTED_TYPE, O.OVERFLOW}


@pytest.mark.parametrize("g", GOLDEN["golden_blocks"], ids=lambda g: g["name"])
def test_golden_vectors(g):
    packed, err = O.pack_u32(g["flag"], g["values"])
    assert err == 0
    assert packed.hex() == g["packed_hex"]


@pytest.mark.parametrize("g", GOLDEN["golden_blocks"], ids=lambda g: g["name"])
def test_golden_vectors_round_trip(g):
    packed = bytes.fromhex(g["packed_hex"])
    vals, consumed, err, _ = O.unpack_u32(packed)
    assert err == 0
    assert list(vals) == g["values"]
    bl, err = O.block_length(packed)
    assert err == 0 and bl == consumed == len(packed)
    for pos, want in enumerate(g["values"]):
        v, err, _ = O.get_u32(pos, packed)
        assert err == 0 and v == want, pos


@pytest.mark.parametrize("ex", GOLDEN["examples"], ids=lambda e: e["name"])
def test_example_known_answers(ex):
    k = ex["kind"]
    if k == "pack32_len":
        packed, err = O.pack_u32(ex["flag"], ex["values"])
        assert err == 0 and len(packed) == ex["want"]
        vals, cons, err, _ = O.unpack_u32(packed)
        assert err == 0 and list(vals) == ex["values"] and cons == len(packed)
    elif k == "pack64_len":
        packed, err = O.pack_u64(ex["flag"], ex["values"])
        assert err == 0 and len(packed) == ex["want"]
        vals, cons, err, _ = O.unpack_u64(packed)
        assert err == 0 and [int(x) for x in vals] == ex["values"]
    elif k in ("append32_lens", "append32_total"):
        lens = []
        for b in ex["blocks"]:
            packed, err = O.pack_u32(ex["flag"], b)
            assert err == 0
            lens.append(len(packed))
        if k == "append32_lens":
            assert lens == ex["want"]
        else:
            assert sum(lens) == ex["want"]
    elif k == "skip_blocks":
        stream = b"".join(O.pack_u32(ex["flag"], b)[0] for b in ex["blocks"])
        bl, err = O.block_length(stream)
        assert err == 0 and bl == ex["want"]
        vals, _, err, _ = O.unpack_u32(stream[bl:])
        assert err == 0 and list(vals) == ex["blocks"][1]
    elif k == "header32":
        packed, err = O.pack_u32(ex["flag"], ex["values"])
        (count, bw, exc, delta, has_for, zz, special), err = O.header(packed)
        w = ex["want"]
        assert err == 0 and (count, bw, exc, bool(delta), bool(has_for)) == (
            w["count"], w["bit_width"], w["exc_count"], w["delta"], w["for"])
    elif k == "max32":
        for f, want in ex["want"].items():
            assert O.max_block_length32(int(f)) == want
    elif k == "max64":
        for f, want in ex["want"].items():
            assert O.max_block_length64(int(f)) == want
    else:
        raise AssertionError(k)


def test_exceptions_golden_layout():
    # format_conformance_test.go: bw 8, 10 exceptions in list mode, svbLen 33,
    # control bytes aa aa 0a.
    g = [x for x in GOLDEN["golden_blocks"] if x["name"] == "exceptions_128"][0]
    b = bytes.fromhex(g["packed_hex"])
    h = struct.unpack_from("<I", b)[0]
    assert (h >> 8) & 31 == 2 and h >> 24 == 10
    assert struct.unpack_from("<H", b, 4)[0] == 33
    assert list(b[6 + 128:6 + 138]) == [5, 15, 25, 35, 45, 55, 65, 75, 85, 95]
    assert b[6 + 138:6 + 141] == bytes([0xAA, 0xAA, 0x0A])


def raw_block_bw32(values, delta=True, count=128):
    """A hand-built uint32 block at bit width 32 (one 32-bit word per row)."""
    h = count | (8 << 8) | (2 << 13) | ((1 << 22) if delta else 0)
    payload = bytearray(512)
    for i in range(128):
        lane, row = i % 16, i // 16
        struct.pack_into("<I", payload, row * 64 + lane * 4, values[i] if i < count else 0)
    return struct.pack("<I", h) + bytes(payload)


def test_overflow_position_every_row_lane():
    # simd_delta_overflow_test.go:177-205 through the full unpack path
    for v in range(1, 8):
        for lane in range(16):
            d = [0] * 128
            d[lane + (v - 1) * 16] = 0xFFFFFFFF
            d[lane + v * 16] = 1
            vals, _, err, pos = O.unpack_u32(raw_block_bw32(d))
            assert err == O.OVERFLOW and pos == lane + v * 16


def test_overflow_first_in_v_major_order():
    rng = np.random.default_rng(20260907)
    for _ in range(200):
        d = [int(x) for x in rng.integers(0, 2**32, 128, dtype=np.uint64)]
        # v-major reference restated in Python (delta.go:83-115)
        x = list(d)
        want = 0
        for r in range(1, 8):
            for lane in range(16):
                cur, prev = lane + r * 16, lane + (r - 1) * 16
                nxt = (x[prev] + x[cur]) & 0xFFFFFFFF
                if want == 0 and nxt < x[prev]:
                    want = cur
                x[cur] = nxt
        _, _, err, pos = O.unpack_u32(raw_block_bw32(d))
        if want:
            assert err == O.OVERFLOW and pos == want
        else:
            assert err == 0


@pytest.mark.parametrize("case", GOLDEN["fuzz_corpus"], ids=lambda c: c["file"])
def test_fuzz_corpus_known_errors(case):
    data = bytes(case["args"][0])
    for pos in (0, 7, 64, 127):
        _, err, _ = O.get_u32(pos, data)
        assert err in KNOWN_ERRORS | {O.OK}
        _, err, _ = O.get_u64(pos, data)
        assert err in KNOWN_ERRORS | {O.OK}
    assert O.unpack_u32(data)[2] in KNOWN_ERRORS | {O.OK}
    assert O.unpack_u64(data)[2] in KNOWN_ERRORS | {O.OK}
    assert O.block_length(data)[1] in KNOWN_ERRORS | {O.OK}
    assert O.header(data)[1] in KNOWN_ERRORS | {O.OK}


def test_empty_block_and_errors():
    # unpack_block.go:87-91: count 0 decodes to nothing and consumes 4 bytes
    empty = struct.pack("<I", 2 << 13)
    vals, cons, err, _ = O.unpack_u32(empty)
    assert err == 0 and len(vals) == 0 and cons == 4
    assert O.unpack_u32(b"\x00\x00")[2] == O.INVALID_BUFFER
    assert O.unpack_u32(struct.pack("<I", 200 | (2 << 13)))[2] == O.INVALID_BLOCK_LENGTH
    assert O.unpack_u32(struct.pack("<I", 5 | (3 << 13)))[2] == O.UNSUPPORTED_TYPE
    assert O.pack_u32(0, [])[1] == O.INVALID_BUFFER
    assert O.pack_u32(0, list(range(129)))[1] == O.INVALID_BUFFER
    packed, _ = O.pack_u32(0, [1, 2, 3])
    assert O.get_u32(3, packed)[1] == O.POS_RANGE
    assert O.get_u32(-1, packed)[1] == O.POS_RANGE
