"""Host logic of the serving loop's admission (no GPU): batches are the
longest arrival-order prefix of one integer width that fits the memory left
and the batch limits."""
from types import SimpleNamespace as NS

import numpy as np

from utlpfor_b200.serve import select_batch


def req(kind, n, cost, is64=False):
    if kind == "compress":
        return NS(kind=kind, values=np.zeros(n, np.uint64 if is64 else np.uint32), cost=cost)
    h = NS(n_values=n, is64=is64)
    return NS(kind=kind, handle=h, positions=np.zeros(n, np.int64), cost=cost)


def test_prefix_under_budget():
    q = [req("decompress", 100, 10) for _ in range(5)]
    assert select_batch(q, 35, 100, 1 << 20) == q[:3]
    assert select_batch(q, 9, 100, 1 << 20) == []
    assert select_batch(q, 1000, 100, 1 << 20) == q


def test_batch_limits():
    q = [req("compress", 1000, 1) for _ in range(10)]
    assert select_batch(q, 100, 4, 1 << 20) == q[:4]
    assert select_batch(q, 100, 100, 2500) == q[:2]
    big = [req("compress", 5000, 1)] + q
    assert select_batch(big, 100, 100, 2500) == big[:1]  # an oversized first request goes alone


def test_one_width_per_batch():
    q = [req("get", 10, 1), req("get", 10, 1, is64=True), req("get", 10, 1), req("get", 10, 1, is64=True)]
    assert select_batch(q, 100, 100, 1 << 20) == [q[0], q[2]]
    assert select_batch(q[1:], 100, 100, 1 << 20) == [q[1], q[3]]


def test_empty_queue():
    assert select_batch([], 100, 10, 10) == []
