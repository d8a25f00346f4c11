"""GPU parity of the device stream indexer (utl_index_stream) with the
caller's BlockLength walk on the host (the oracle): offsets of packed
streams of every shape, mixed integer widths, errors at the first bad
block, and payloads that hold runs of bytes which parse as headers (so
that partitions start on false chains and the merge and re-walk paths
run)."""
import numpy as np
import pytest

import oracle_ref as O
from gen import streams

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch

    import utlpfor_b200 as U
    assert torch.cuda.is_available()
    return U, torch


def dev(torch, a):
    return torch.from_numpy(np.ascontiguousarray(a, dtype=np.uint8)).cuda()


def check(U, torch, packed):
    want, err, nb = O.index_stream(packed)
    if err == O.OK:
        got = U.index_stream(dev(torch, packed)).cpu().numpy()
        assert got.size == len(want)
        assert np.array_equal(got, np.array(want, dtype=np.int64))
    else:
        with pytest.raises(Exception) as ei:
            U.index_stream(dev(torch, packed))
        assert ei.value.block == nb
        from utlpfor_b200 import _raise
        with pytest.raises(type(ei.value)):
            _raise(err)
    return want, err, nb


@pytest.mark.parametrize("flag", [0, 1, 2, 4, 5])
@pytest.mark.parametrize("kind", ["small", "exc", "dense_exc", "sorted", "const", "zero", "full", "wide"])
def test_index_u32_streams(env, flag, kind):
    U, torch = env
    rng = np.random.default_rng(flag * 7 + len(kind))
    lens = list(rng.integers(1, 20000, 12)) + [128, 1, 129]
    vals, vo = streams(rng, lens, kind)
    packed, bo, _ = O.pack_streams(flag, vals, vo)
    want, err, _ = check(U, torch, packed)
    assert err == O.OK and want == list(bo.astype(np.int64))


@pytest.mark.parametrize("kind", ["for64", "full", "walk", "fit32", "zero"])
def test_index_u64_and_mixed(env, kind):
    U, torch = env
    rng = np.random.default_rng(len(kind))
    v64, vo64 = streams(rng, list(rng.integers(1, 9000, 6)), kind, is64=True)
    p64, _, _ = O.pack_streams(1, v64, vo64)
    v32, vo32 = streams(rng, list(rng.integers(1, 9000, 6)), "exc")
    p32, _, _ = O.pack_streams(0, v32, vo32)
    check(U, torch, p64)
    _, err, _ = check(U, torch, np.concatenate([p32, p64, p32]))
    assert err == O.OK


def test_index_empty_and_large(env):
    U, torch = env
    got = U.index_stream(dev(torch, np.zeros(0, np.uint8))).cpu().numpy()
    assert list(got) == [0]
    rng = np.random.default_rng(5)
    vals, vo = streams(rng, [1 << 22], "exc")
    packed, bo, _ = O.pack_streams(0, vals, vo, n_threads=8)
    got = U.index_stream(dev(torch, packed)).cpu().numpy()
    assert np.array_equal(got, bo.astype(np.int64))


def test_index_errors(env):
    U, torch = env
    rng = np.random.default_rng(9)
    vals, vo = streams(rng, [50000], "exc")
    packed, bo, _ = O.pack_streams(0, vals, vo)
    nb = len(bo) - 1
    _, err, at = check(U, torch, packed[:-1])  # the last block runs past the end
    assert err == O.INVALID_BUFFER and at == nb - 1
    for b, how in [(7, "reserved"), (nb // 2, "count"), (nb - 3, "bw")]:
        bad = packed.copy()
        o = int(bo[b])
        if how == "reserved":
            bad[o + 2] |= 0x04    # header bit 18
        elif how == "count":
            bad[o] = 200          # count > 128
        else:
            bad[o + 1] |= 0x1F    # bit width field 31 -> 124
        _, err, at = check(U, torch, bad)
        assert err != O.OK and at == b


def fake_header_blocks(n_blocks, tail):
    """bw-32 blocks (NoPatch, a zero value so no FOR): their payload is the
    values in order, here 4-byte words that parse as 4-byte blocks (count 1,
    bw 0, uint32).  tail: the last value -- a fake header (the false chain
    meets the next true block), or one that fails to parse."""
    v = np.full((n_blocks, 128), 0x00004001, dtype=np.uint32)
    v[:, 0] = 0
    v[:, 1] = 0xFFFFFFFF
    v[:, 127] = tail
    return v.reshape(-1)


@pytest.mark.parametrize("tail", [0x00004001, 0xFFFFFFFF, 0x00014001])
def test_index_false_chains(env, tail):
    U, torch = env
    vals = fake_header_blocks(3000, tail)
    vo = np.array([0, vals.size], dtype=np.uint64)
    packed, bo, _ = O.pack_streams(4, vals, vo)  # NoPatch
    assert np.all(np.diff(bo) == 516)
    want, err, _ = check(U, torch, packed)
    assert err == O.OK and want == list(bo.astype(np.int64))
