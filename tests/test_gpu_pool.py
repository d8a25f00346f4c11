"""The per-call context pool (utl_pool_*, utlpfor_b200.CompressorPool):
many host threads pack, unpack and query blocks at once through a few
contexts; every result equals the oracle's (bytes, values, errors)."""
import threading

import numpy as np
import pytest

import oracle_ref as O
from gen import KINDS32, block_values, block_values64

pytestmark = pytest.mark.gpu


def _worker(pool, seed, errors, is64):
    rng = np.random.default_rng(seed)
    try:
        for it in range(60):
            flag = int(rng.integers(0, 16))
            n = int(rng.integers(1, 129))
            if is64:
                v = block_values64(rng, n, ("for64", "full", "walk", "fit32")[it % 4])
                want, err = O.pack_u64(flag, v)
                got = bytes(pool.PackUint64(flag, v))
                vals, cons = pool.UnpackUint64(got)
                g = pool.GetUint64(n - 1, got)
            else:
                v = block_values(rng, n, KINDS32[it % len(KINDS32)])
                want, err = O.pack_u32(flag, v)
                got = bytes(pool.PackUint32(flag, v))
                vals, cons = pool.UnpackUint32(got)
                g = pool.GetUint32(n - 1, got)
            assert err == 0 and got == want, (seed, it, flag)
            assert np.array_equal(vals, v) and cons == len(got)
            assert g == int(v[-1])
    except Exception as e:  # reported by the main thread
        errors.append(repr(e))


@pytest.mark.parametrize("is64", [False, True])
def test_pool_many_threads_match_oracle(is64):
    import utlpfor_b200 as U
    pool = U.CompressorPool(4)
    errors = []
    ts = [threading.Thread(target=_worker, args=(pool, 100 + k, errors, is64)) for k in range(12)]
    for t in ts:
        t.start()
    for t in ts:
        t.join()
    pool.close()
    assert not errors, errors[:3]


def test_pool_errors_match_oracle():
    import utlpfor_b200 as U
    pool = U.CompressorPool(2)
    rng = np.random.default_rng(5)
    blk, _ = O.pack_u32(1, block_values(rng, 128, "walk"))
    for cut in range(0, len(blk), 7):
        b = blk[:cut]
        _, _, oerr, _ = O.unpack_u32(b)
        try:
            pool.UnpackUint32(b)
            code = 0
        except U.UTLError as e:
            code = e.code
        assert code == oerr, cut
    pool.close()
