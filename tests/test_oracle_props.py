"""Oracle self-consistency: round trips over every stored flag combination,
partial lengths and the three uint64 paths (fuzz_test.go round-trip
properties, Get == Unpack, BlockLength == consumed)."""
import numpy as np
import pytest

import oracle_ref as O


def gen_block(rng, n, kind):
    if kind == "small":
        return rng.integers(0, 2**11, n, dtype=np.uint64).astype(np.uint32)
    if kind == "exc":
        v = rng.integers(0, 2**8, n, dtype=np.uint64)
        m = rng.random(n) < 0.05
        v[m] = rng.integers(2**8, 2**32, m.sum(), dtype=np.uint64)
        return v.astype(np.uint32)
    if kind == "sorted":
        return np.cumsum(1 + rng.geometric(1 / 64, n)).astype(np.uint32)
    if kind == "const":
        return np.full(n, rng.integers(0, 2**32, dtype=np.uint64), dtype=np.uint32)
    if kind == "full":
        return rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    raise ValueError(kind)


@pytest.mark.parametrize("flag", range(16))
def test_round_trip_all_flags_u32(flag):
    rng = np.random.default_rng(1000 + flag)
    for n in (1, 2, 15, 16, 17, 63, 64, 65, 100, 127, 128):
        for kind in ("small", "exc", "sorted", "const", "full"):
            v = gen_block(rng, n, kind)
            packed, err = O.pack_u32(flag, v)
            assert err == 0
            got, cons, err, _ = O.unpack_u32(packed)
            assert err == 0 and cons == len(packed) and np.array_equal(got, v), (flag, n, kind)
            assert O.block_length(packed) == (len(packed), 0)
            for pos in range(n):
                assert O.get_u32(pos, packed)[:2] == (int(v[pos]), 0)


def gen64(rng, n, kind):
    if kind == "for64":
        return (2**40 + rng.integers(0, 2**20, n, dtype=np.uint64)).astype(np.uint64)
    if kind == "full":
        return rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)
    if kind == "walk":
        steps = rng.integers(-1000, 1001, n)
        return (np.int64(2**62) + np.cumsum(steps)).astype(np.uint64)
    if kind == "fit32":
        return rng.integers(0, 2**32, n, dtype=np.uint64)
    raise ValueError(kind)


@pytest.mark.parametrize("flag", range(8))
def test_round_trip_u64(flag):
    rng = np.random.default_rng(77 + flag)
    for n in (1, 5, 64, 127, 128):
        for kind in ("for64", "full", "walk", "fit32"):
            v = gen64(rng, n, kind)
            packed, err = O.pack_u64(flag, v)
            assert err == 0
            got, cons, err, _ = O.unpack_u64(packed)
            assert err == 0 and cons == len(packed) and np.array_equal(got, v), (flag, n, kind)
            assert O.block_length(packed) == (len(packed), 0)
            for pos in range(0, n, 7):
                assert O.get_u64(pos, packed)[:2] == (int(v[pos]), 0)


def test_stream_helpers_match_block_calls():
    rng = np.random.default_rng(5)
    lens = [1, 128, 300, 0, 257, 1000]
    vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    vals = gen_block(rng, int(vo[-1]), "exc")
    packed, bo, so = O.pack_streams(0, vals, vo, n_threads=3)
    ref = b""
    for s in range(len(lens)):
        for j in range(0, lens[s], 128):
            ref += O.pack_u32(0, vals[int(vo[s]) + j:int(vo[s]) + min(j + 128, lens[s])])[0]
    assert packed.tobytes() == ref
    out, err = O.unpack_streams(packed, bo, vo, n_threads=3)
    assert err == 0 and np.array_equal(out, vals)
