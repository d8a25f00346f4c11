"""GPU tests of the serving loop: every request of a mixed run -- compress,
decompress and Get of uneven sizes, batched together and overlapping on
several CUDA streams -- gives exactly the result of the same request served
alone, and both equal the oracle (the codec is integer: the tolerance is
zero).  Also: admission holds the device-memory budget, and requests on a
released stream or over the budget fail on their own."""
import numpy as np
import pytest

import oracle_ref as O
from gen import block_values, block_values64

pytestmark = pytest.mark.gpu

KINDS32 = ("small", "exc", "sorted", "walk", "const", "dense_exc", "wide", "zero")
KINDS64 = ("for64", "full", "walk", "fit32")


def make_inputs(seed, n):
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        ln = int(np.exp(rng.uniform(0, np.log(40000))))
        if i % 5 == 4:
            out.append((block_values64(rng, ln, KINDS64[i % 4]), int(rng.choice([0, 1, 2, 4]))))
        else:
            out.append((block_values(rng, ln, KINDS32[i % len(KINDS32)]), int(rng.integers(0, 8))))
    return out


def oracle_stream(values, flag):
    vo = np.array([0, values.size], dtype=np.uint64)
    packed, bo, _ = O.pack_streams(flag, values, vo)
    return packed, bo


def run_alone(S, inputs, positions):
    """Each request on an idle server, one at a time."""
    srv = S.CodecServer(budget_bytes=4 << 30, slots=1)
    try:
        res = []
        for (v, flag), pos in zip(inputs, positions):
            h = srv.submit_compress(v, flag).result(timeout=60)
            packed = h.packed.cpu().numpy().copy()
            dec = srv.submit_decompress(h).result(timeout=60).copy()
            got = srv.submit_get(h, pos).result(timeout=60).copy()
            res.append((packed, h.block_off.cpu().numpy().copy(), dec, got))
            srv.release(h)
        return res
    finally:
        srv.close()


def test_mixed_requests_equal_alone_and_oracle():
    import utlpfor_b200.serve as S
    inputs = make_inputs(11, 40)
    rng = np.random.default_rng(3)
    positions = [rng.integers(0, max(v.size, 1), 50).astype(np.int64) for v, _ in inputs]
    alone = run_alone(S, inputs, positions)

    srv = S.CodecServer(budget_bytes=4 << 30, slots=3, max_batch_requests=8)
    try:
        # the first half is compressed up front; then the second half's
        # compresses arrive interleaved with decompress/Get of the first half
        half = len(inputs) // 2
        handles = [None] * len(inputs)
        for i in range(half):
            handles[i] = srv.submit_compress(*inputs[i])
        for i in range(half):
            handles[i] = handles[i].result(timeout=60)
        futs = []
        for i in range(half, len(inputs)):
            futs.append(("c", i, srv.submit_compress(*inputs[i])))
            j = i - half
            futs.append(("d", j, srv.submit_decompress(handles[j])))
            futs.append(("g", j, srv.submit_get(handles[j], positions[j])))
        mixed = {}
        for kind, i, f in futs:
            mixed[(kind, i)] = f.result(timeout=120)
        for i in range(half, len(inputs)):
            handles[i] = mixed[("c", i)]
        more = [(i, srv.submit_decompress(handles[i]), srv.submit_get(handles[i], positions[i]))
                for i in range(half, len(inputs))]
        for i, fd, fg in more:
            mixed[("d", i)] = fd.result(timeout=60)
            mixed[("g", i)] = fg.result(timeout=60)
        st = srv.stats()
        assert st["batches"] < 3 * len(inputs)  # requests were batched together
        for i, (v, flag) in enumerate(inputs):
            want, wbo = oracle_stream(v, flag)
            a_packed, a_bo, a_dec, a_get = alone[i]
            h = handles[i]
            m_packed = h.packed.cpu().numpy()
            assert np.array_equal(a_packed, want), i
            assert np.array_equal(m_packed, want), i
            assert np.array_equal(a_bo.view(np.uint64), wbo) and np.array_equal(h.block_off.cpu().numpy(), a_bo)
            assert np.array_equal(a_dec, v) and np.array_equal(mixed[("d", i)], v), i
            assert np.array_equal(a_get, v[positions[i]]) and np.array_equal(mixed[("g", i)], a_get), i
        for h in handles:
            srv.release(h)
        assert srv.stats()["resident_bytes"] == 0
    finally:
        srv.close()


def test_admission_budget_and_failures():
    import utlpfor_b200.serve as S
    from utlpfor_b200 import ErrPositionOutOfRange
    rng = np.random.default_rng(9)
    vals = [block_values(rng, 20000, "exc") for _ in range(12)]
    from utlpfor_b200._lib import load
    one = 20000 * 4 + 157 * load().utl_max_block_length32(0) + 16 * 159   # a compress request's device bytes
    srv = S.CodecServer(budget_bytes=3 * one + 100, slots=3)
    try:
        # over the budget on its own: rejected at once
        with pytest.raises(S.ServerError):
            srv.submit_compress(np.zeros(1 << 20, np.uint32)).result(timeout=10)
        futs = [srv.submit_compress(v) for v in vals]
        hs = [f.result(timeout=60) for f in futs]
        st = srv.stats()
        assert st["admitted"] == 12 and st["rejected"] == 1
        for v, h in zip(vals, hs):
            assert np.array_equal(srv.submit_decompress(h).result(timeout=60), v)
        # a Get past the end fails its own request only
        bad = srv.submit_get(hs[0], np.array([5, 20000], dtype=np.int64))
        good = srv.submit_get(hs[1], np.array([5, 19999], dtype=np.int64))
        with pytest.raises(ErrPositionOutOfRange):
            bad.result(timeout=60)
        assert np.array_equal(good.result(timeout=60), vals[1][[5, 19999]])
        srv.release(hs[2])
        with pytest.raises(S.ServerError):
            srv.submit_decompress(hs[2]).result(timeout=60)
    finally:
        srv.close()
