"""Multi-process host logic on CPU (gloo, world size 2): each rank packs its
shard of a batch of streams (the oracle stands in for the rank's GPU), the
ranks' byte offsets come from one all-gather, and the shards laid rank after
rank equal the whole batch packed at once, block offsets included.  Also
the maximum-over-ranks timing reduction."""
import os
import socket

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    sys.path.insert(0, ROOT)
    import torch.distributed as dist

    import oracle_ref as O
    from gen import streams
    from utlpfor_b200.dist import exclusive_offsets, global_block_offsets, max_over_ranks, shard_streams
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    try:
        rng = np.random.default_rng(42)  # every rank builds the same batch
        lens = list(rng.integers(1, 3000, 17)) + [128, 1]
        vals, vo = streams(rng, lens, "exc")
        s0, s1 = shard_streams(vo, rank, world)
        lvo = vo[s0:s1 + 1] - vo[s0]
        lvals = vals[int(vo[s0]):int(vo[s1])]
        packed, bo, _ = O.pack_streams(0, lvals, lvo) if s1 > s0 else (np.zeros(0, np.uint8), np.zeros(1, np.uint64), None)
        off, total = exclusive_offsets(len(packed))
        gbo = global_block_offsets(bo, off)
        t = max_over_ranks([1.0 + rank, 5.0 - rank])
        parts = [None] * world
        dist.all_gather_object(parts, (s0, s1, packed.tobytes(), gbo.tolist(), off, total, t))
        q.put((rank, parts))
    finally:
        dist.destroy_process_group()


def test_sharded_pack_joins_into_the_whole_stream():
    import multiprocessing as mp
    import sys
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ref as O
    from gen import streams
    world = 2
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    try:
        results = dict(q.get(timeout=120) for _ in range(world))
    finally:
        for p in procs:
            p.join(timeout=60)
    for p in procs:
        assert p.exitcode == 0
    parts = results[0]
    assert parts == results[1]
    rng = np.random.default_rng(42)
    lens = list(rng.integers(1, 3000, 17)) + [128, 1]
    vals, vo = streams(rng, lens, "exc")
    want, wbo, _ = O.pack_streams(0, vals, vo)
    joined = b"".join(p[2] for p in parts)
    assert joined == want.tobytes()
    assert parts[0][0] == 0 and parts[-1][1] == len(lens) and parts[0][1] == parts[1][0]
    assert all(p[5] == len(want) for p in parts)
    gbo = []
    for p in parts:
        gbo += p[3][:-1]
    gbo.append(len(want))
    assert gbo == list(wbo.astype(int))
    assert all(p[6] == [2.0, 5.0] for p in parts)


@pytest.mark.parametrize("world", [1, 2, 3, 8])
def test_shard_streams_covers_every_stream_once(world):
    from utlpfor_b200.dist import shard_streams
    rng = np.random.default_rng(world)
    vo = np.concatenate([[0], np.cumsum(rng.integers(0, 5000, 40))]).astype(np.uint64)
    cuts = [shard_streams(vo, r, world) for r in range(world)]
    assert cuts[0][0] == 0 and cuts[-1][1] == 40
    for a, b in zip(cuts, cuts[1:]):
        assert a[1] == b[0] and a[0] <= a[1]
