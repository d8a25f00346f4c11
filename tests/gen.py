"""Seeded synthetic inputs shaped like the benchmark workloads, small."""
import numpy as np


def block_values(rng, n, kind):
    if kind == "small":      # uniform [0, 2^11)
        return rng.integers(0, 2**11, n, dtype=np.uint64).astype(np.uint32)
    if kind == "exc":        # [0,2^8) with 2% outliers in [2^8, 2^32)
        v = rng.integers(0, 2**8, n, dtype=np.uint64)
        m = rng.random(n) < 0.02
        v[m] = rng.integers(2**8, 2**32, int(m.sum()), dtype=np.uint64)
        return v.astype(np.uint32)
    if kind == "dense_exc":  # many exceptions: bitmap index mode
        v = rng.integers(0, 2**6, n, dtype=np.uint64)
        m = rng.random(n) < 0.4
        v[m] = rng.integers(2**6, 2**32, int(m.sum()), dtype=np.uint64)
        return v.astype(np.uint32)
    if kind == "sorted":     # posting list gaps 1+Geom(1/64)
        return np.cumsum(1 + rng.geometric(1 / 64, n)).astype(np.uint32)
    if kind == "const":
        return np.full(n, rng.integers(0, 2**32, dtype=np.uint64), dtype=np.uint32)
    if kind == "zero":
        return np.zeros(n, dtype=np.uint32)
    if kind == "full":
        return rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
    if kind == "walk":       # signed random walk, forces zigzag under Delta
        return (np.int64(2**31) + np.cumsum(rng.integers(-1000, 1001, n))).astype(np.uint32)
    if kind == "wide":       # every step width
        bw = int(rng.integers(0, 33))
        hi = 2**bw if bw < 32 else 2**32
        return rng.integers(0, max(hi, 1), n, dtype=np.uint64).astype(np.uint32)
    raise ValueError(kind)


KINDS32 = ("small", "exc", "dense_exc", "sorted", "const", "zero", "full", "walk", "wide")


def block_values64(rng, n, kind):
    if kind == "for64":
        return (2**40 + rng.integers(0, 2**20, n, dtype=np.uint64)).astype(np.uint64)
    if kind == "full":
        return rng.integers(0, 2**64 - 1, n, dtype=np.uint64, endpoint=True)
    if kind == "walk":
        return (np.int64(2**62) + np.cumsum(rng.integers(-1000, 1001, n))).astype(np.uint64)
    if kind == "fit32":
        return rng.integers(0, 2**32, n, dtype=np.uint64)
    if kind == "upper_for":  # two-block whose upper halves take a 4-byte FOR base
        return ((np.uint64(2**30) + rng.integers(0, 16, n, dtype=np.uint64)) << np.uint64(32)) | \
            rng.integers(0, 2**32, n, dtype=np.uint64)
    if kind == "zero":
        return np.zeros(n, dtype=np.uint64)
    raise ValueError(kind)


KINDS64 = ("for64", "full", "walk", "fit32", "upper_for", "zero")


def streams(rng, lens, kind, is64=False):
    vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    parts = []
    for n in lens:
        parts.append(block_values64(rng, n, kind) if is64 else block_values(rng, n, kind))
    dt = np.uint64 if is64 else np.uint32
    vals = np.concatenate(parts).astype(dt) if parts else np.zeros(0, dt)
    return vals, vo
