"""GPU parity of the batched device path against the oracle: one launch
packs many uneven streams byte-identically to block-by-block Append calls,
unpacks them, and answers Get queries; plus large-size properties."""
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


def to_dev(torch, a):
    a = np.ascontiguousarray(a)
    return torch.from_numpy(a.view(np.int64 if a.dtype.itemsize == 8 else np.int32)).cuda()


LENS = [1, 128, 300, 0, 257, 1000, 5, 129, 0, 4096, 77]


UNPACK_SCHEDULES = {0: "unpack_tiles", 1: "unpack_pipelined", 2: "unpack_pipelined_wide",
                    3: "unpack_pipelined_narrow", 4: "unpack_tma", 5: "unpack_tma_narrow", 6: "unpack_tma_wide",
                    7: "unpack_tma_fast", 8: "unpack_thread_auto", 9: "unpack_thread",
                    10: "unpack_thread_double"}


@pytest.fixture(params=sorted(UNPACK_SCHEDULES), ids=[UNPACK_SCHEDULES[k] for k in sorted(UNPACK_SCHEDULES)])
def sched(request):
    from utlpfor_b200._lib import load
    L = load()
    old = L.utl_get_knob(0)
    assert L.utl_set_knob(0, request.param) == 0
    yield request.param
    L.utl_set_knob(0, old)


@pytest.fixture(params=[0, 1, 3, 4, 5, 6, 7],
                ids=["unpack64_warp", "unpack64_octet", "unpack64_quad", "unpack64_quad_narrow", "unpack64_quad_wide",
                     "unpack64_quad_wide1", "unpack64_quad_auto1"])
def u64sched(request):
    from utlpfor_b200._lib import load
    L = load()
    old = L.utl_get_knob(8)
    assert L.utl_set_knob(8, request.param) == 0
    yield request.param
    L.utl_set_knob(8, old)


@pytest.fixture(params=[0, 1, 2], ids=["pack_quad", "pack_lane", "pack_pair"])
def psched(request):
    from utlpfor_b200._lib import load
    L = load()
    old = L.utl_get_knob(2)
    assert L.utl_set_knob(2, request.param) == 0
    yield request.param
    L.utl_set_knob(2, old)


KINDS = ["small", "exc", "dense_exc", "sorted", "walk", "wide", "const", "zero", "full"]


@pytest.mark.parametrize("flag", list(range(16)))
@pytest.mark.parametrize("kind", KINDS)
def test_pack_unpack_batch_u32(env, flag, kind, psched):
    """Every combination of the four stored flag bits (Delta, NoFOR,
    NoPatch, Special) under every pack schedule, each result unpacked
    under every unpack schedule."""
    _batch_u32_case(env, flag, kind, all_unpack=True)


@pytest.mark.parametrize("flag", [f | extra for extra in (16, 32, 48) for f in range(16)])
@pytest.mark.parametrize("kind", KINDS)
def test_pack_unpack_batch_u32_placement_flags(env, flag, kind, psched):
    """Append and NoInPlace (placement only: the same bytes) on top of every
    stored-bit combination, under both pack schedules."""
    _batch_u32_case(env, flag, kind)


def _batch_u32_case(env, flag, kind, all_unpack=False):
    U, torch = env
    rng = np.random.default_rng(flag * 31 + len(kind))
    vals, vo = streams(rng, LENS, kind)
    want, wbo, wso = O.pack_streams(flag, vals, vo)
    pb = U.pack_batch(to_dev(torch, vals), vo, flag)
    got_len = pb.packed_len
    assert got_len == len(want)
    assert np.array_equal(pb.packed[:got_len].cpu().numpy(), want)
    assert np.array_equal(pb.block_off.cpu().numpy().view(np.uint64), wbo)
    assert np.array_equal(pb.stream_byte_off.cpu().numpy().view(np.uint64), wso)
    from utlpfor_b200._lib import load
    L = load()
    old = L.utl_get_knob(0)
    try:
        for sc in (sorted(UNPACK_SCHEDULES) if all_unpack else [old]):
            assert L.utl_set_knob(0, sc) == 0
            out = U.unpack_batch(pb)
            assert np.array_equal(out.cpu().numpy().view(np.uint32), vals), UNPACK_SCHEDULES[sc]
    finally:
        L.utl_set_knob(0, old)


@pytest.mark.parametrize("flag", list(range(16)) + [16 | 5, 32 | 9, 48 | 15])
@pytest.mark.parametrize("kind", ["for64", "full", "walk", "fit32", "upper_for", "zero"])
def test_pack_unpack_batch_u64(env, flag, kind, psched, u64sched):
    U, torch = env
    rng = np.random.default_rng(500 + flag)
    vals, vo = streams(rng, LENS, kind, is64=True)
    want, wbo, wso = O.pack_streams(flag, vals, vo)
    pb = U.pack_batch(to_dev(torch, vals), vo, flag)
    assert pb.packed_len == len(want)
    assert np.array_equal(pb.packed[:pb.packed_len].cpu().numpy(), want)
    assert np.array_equal(pb.block_off.cpu().numpy().view(np.uint64), wbo)
    # unpack goes through the reference's decode rules, including its
    # reading of two-block upper halves with a 4-byte FOR base
    ref, err = O.unpack_streams(want, wbo, vo, dtype=np.uint64)
    status = torch.empty(pb.n_blocks, dtype=torch.int32, device="cuda")
    out = U.unpack_batch(pb, block_status=status, check=False)
    st = status.cpu().numpy()
    for s in range(len(LENS)):
        b0 = int(pb.block_start[s].item())
        for j in range((LENS[s] + 127) // 128):
            blk = want[int(wbo[b0 + j]):int(wbo[b0 + j + 1])]
            ov, oc, oerr, oovf = O.unpack_u64(blk)
            if oerr == 0 and (len(ov) != min(128, LENS[s] - 128 * j) or oc != len(blk)):
                oerr = 8
            assert st[b0 + j] & 0xFF == oerr, (s, j)
            if oerr == 0:
                lo = int(vo[s]) + 128 * j
                assert np.array_equal(out[lo:lo + len(ov)].cpu().numpy().view(np.uint64), ov)


@pytest.mark.parametrize("is64", [False, True])
@pytest.mark.parametrize("flag", list(range(8)) + [8])
def test_get_batch(env, is64, flag, psched):
    U, torch = env
    rng = np.random.default_rng(77 + flag)
    kinds = ("sorted", "exc", "walk", "full") if not is64 else ("for64", "full", "walk")
    for kind in kinds:
        vals, vo = streams(rng, LENS, kind, is64=is64)
        packed, bo, so = O.pack_streams(flag, vals, vo)
        pb = U.pack_batch(to_dev(torch, vals), vo, flag)
        ns = len(LENS)
        qs = rng.integers(0, ns + 1, 3000).astype(np.uint32)  # includes an out-of-range stream
        lens = np.array(LENS + [0])
        qp = (rng.random(3000) * (lens[qs] + 3)).astype(np.uint64)  # some past the end
        out, st = U.get_batch(pb, to_dev(torch, qs), to_dev(torch, qp))
        out = out.cpu().numpy().view(np.uint64 if is64 else np.uint32)
        st = st.cpu().numpy()
        for i in range(3000):
            s, p = int(qs[i]), int(qp[i])
            if s >= ns or p >= LENS[s]:
                assert st[i] & 0xFF == 2
                continue
            b = int(pb.block_start[s].item()) + p // 128
            blk = packed[int(bo[b]):int(bo[b + 1])]
            gv, gerr, govf = (O.get_u64 if is64 else O.get_u32)(p % 128, blk)
            assert (st[i] & 0xFF, st[i] >> 8) == (gerr, govf)
            if gerr == 0:
                assert out[i] == gv == vals[int(vo[s]) + p]


def test_unpack_batch_corrupt_blocks(env, sched):
    """A corrupt block fails its own status only; the others decode."""
    U, torch = env
    rng = np.random.default_rng(3)
    lens = [128 * 40]
    vals, vo = streams(rng, lens, "exc")
    packed, bo, _ = O.pack_streams(1, vals, vo)
    bad = packed.copy()
    victims = [3, 17, 29]
    for b in victims:
        bad[int(bo[b]) + int(rng.integers(0, int(bo[b + 1] - bo[b])))] ^= 0x5A
    pb = U.pack_batch(to_dev(torch, vals), vo, 1)
    dev_bad = torch.from_numpy(bad).cuda()
    status = torch.zeros(pb.n_blocks, dtype=torch.int32, device="cuda")
    out = U.unpack_batch(pb, block_status=status, check=False, packed=dev_bad)
    st = status.cpu().numpy()
    outv = out.cpu().numpy().view(np.uint32)
    for b in range(pb.n_blocks):
        blk = bad[int(bo[b]):int(bo[b + 1])]
        ov, oc, oerr, oovf = O.unpack_u32(blk)
        if oerr == 0 and (len(ov) != 128 or oc != len(blk)):
            oerr = 8
        assert (st[b] & 0xFF, st[b] >> 8) == (oerr, oovf), b
        if oerr == 0:
            assert np.array_equal(outv[128 * b:128 * b + 128], ov)


@pytest.mark.parametrize("flag", [0, 1])
def test_unpack_batch_corrupt_blocks_u64(env, u64sched, flag):
    """uint64 blocks (two-block and FOR64 shapes) with a damaged byte fail
    their own status with the reference's error class; the others decode."""
    U, torch = env
    rng = np.random.default_rng(7 + flag)
    parts, vo = [], [0]
    for kind in ("full", "for64", "walk"):
        v, _ = streams(rng, [128 * 20], kind, is64=True)
        parts.append(v)
        vo.append(vo[-1] + len(v))
    vals = np.concatenate(parts)
    vo = np.array(vo, dtype=np.uint64)
    packed, bo, _ = O.pack_streams(flag, vals, vo)
    bad = packed.copy()
    victims = [2, 11, 19, 23, 35, 44, 58]
    for b in victims:
        bad[int(bo[b]) + int(rng.integers(0, int(bo[b + 1] - bo[b])))] ^= 0x5A
    pb = U.pack_batch(to_dev(torch, vals), vo, flag)
    dev_bad = torch.from_numpy(bad).cuda()
    status = torch.zeros(pb.n_blocks, dtype=torch.int32, device="cuda")
    out = U.unpack_batch(pb, block_status=status, check=False, packed=dev_bad)
    st = status.cpu().numpy()
    outv = out.cpu().numpy().view(np.uint64)
    for b in range(pb.n_blocks):
        blk = bad[int(bo[b]):int(bo[b + 1])]
        ov, oc, oerr, oovf = O.unpack_u64(blk)
        if oerr == 0 and (len(ov) != 128 or oc != len(blk)):
            oerr = 8
        assert (st[b] & 0xFF, st[b] >> 8) == (oerr, oovf), b
        if oerr == 0:
            assert np.array_equal(outv[128 * b:128 * b + 128], ov)


def test_host_buffer_streams(env):
    U, torch = env
    rng = np.random.default_rng(12)
    for is64, kind in ((False, "exc"), (True, "walk")):
        vals, vo = streams(rng, LENS, kind, is64=is64)
        want, wbo, wso = O.pack_streams(1, vals, vo)
        packed, bo, so = U.pack_streams(1, vals, vo)
        assert packed.tobytes() == want.tobytes()
        assert np.array_equal(bo, wbo) and np.array_equal(so, wso)
        out = U.unpack_streams(packed, bo, vo, is64=is64)
        assert np.array_equal(out, vals)


def test_large_round_trip_properties(env, sched, psched):
    """2^24 values with the exception-heavy shape: pack is byte-identical to
    the oracle (checked by digest), unpack restores every value."""
    U, torch = env
    import hashlib
    rng = np.random.default_rng(2024)
    n = 1 << 24
    v = rng.integers(0, 2**8, n, dtype=np.uint64)
    m = rng.random(n) < 0.02
    v[m] = rng.integers(2**8, 2**32, int(m.sum()), dtype=np.uint64)
    v = v.astype(np.uint32)
    v[: 128 * 1000] = 7  # some all-equal blocks
    vo = np.array([0, n], dtype=np.uint64)
    want, wbo, _ = O.pack_streams(0, v, vo, n_threads=8)
    pb = U.pack_batch(to_dev(torch, v), vo, 0)
    assert pb.packed_len == len(want)
    got = pb.packed[:pb.packed_len].cpu().numpy()
    assert hashlib.sha256(got.tobytes()).digest() == hashlib.sha256(want.tobytes()).digest()
    out = U.unpack_batch(pb)
    assert torch.equal(out, to_dev(torch, v))


@pytest.mark.parametrize("flag", [0, 1, 3, 4])
def test_large_u64_mix(env, flag, psched, u64sched):
    """2^21 uint64 values over 96 ragged streams mixing the three uint64
    shapes (FOR64, two-block, delta walk): the pack is byte-identical to the
    oracle under both pack schedules and the unpack restores every value."""
    U, torch = env
    rng = np.random.default_rng(64 + flag)
    lens = rng.integers(1, 40000, 96)
    lens[-1] = max(1, (1 << 21) - int(lens[:-1].sum())) if int(lens[:-1].sum()) < (1 << 21) else lens[-1]
    kinds = ["for64", "full", "walk"]
    vals, vo = [], [0]
    for i, n in enumerate(lens):
        v, _ = streams(rng, [int(n)], kinds[i % 3], is64=True)
        vals.append(v)
        vo.append(vo[-1] + int(n))
    vals = np.concatenate(vals)
    vo = np.array(vo, dtype=np.uint64)
    want, wbo, _ = O.pack_streams(flag, vals, vo, n_threads=8)
    pb = U.pack_batch(to_dev(torch, vals), vo, flag)
    assert pb.packed_len == len(want)
    assert np.array_equal(pb.packed[:pb.packed_len].cpu().numpy(), want)
    assert np.array_equal(pb.block_off.cpu().numpy().view(np.uint64), wbo)
    out = U.unpack_batch(pb)
    assert torch.equal(out, to_dev(torch, vals))


@pytest.mark.parametrize("flag", [0, 1, 2, 6])
@pytest.mark.parametrize("kind", ["exc", "sorted", "walk"])
def test_misaligned_whole_tiles(env, flag, kind, psched):
    """Long streams that start 1, 2 or 3 values past a 16-byte boundary, so
    whole tiles of 32 blocks load misaligned; the last tile ends at the end
    of the values.  Bytes and offsets equal the oracle's."""
    U, torch = env
    rng = np.random.default_rng(900 + flag)
    lens = [5, 128 * 100, 3, 128 * 70 + 17, 1, 128 * 64, 2, 128 * 33 + 1, 128 * 65]
    vals, vo = streams(rng, lens, kind)
    want, wbo, wso = O.pack_streams(flag, vals, vo)
    pb = U.pack_batch(to_dev(torch, vals), vo, flag)
    assert pb.packed_len == len(want)
    assert np.array_equal(pb.packed[:pb.packed_len].cpu().numpy(), want)
    assert np.array_equal(pb.block_off.cpu().numpy().view(np.uint64), wbo)
    out = U.unpack_batch(pb)
    assert torch.equal(out, to_dev(torch, vals))


def test_pack_window_shapes(env):
    """The uint32 lane pack picks its image window from the previous pack's
    block density.  Small blocks twice (the second pack takes the small
    window), then large blocks right after (the small window with many
    rounds), then again (the large window): every output equals the
    oracle's."""
    U, torch = env
    from utlpfor_b200._lib import load
    L = load()
    old = L.utl_get_knob(2)
    assert L.utl_set_knob(2, 1) == 0
    try:
        rng = np.random.default_rng(55)
        n = 1 << 18
        small = rng.integers(0, 2**8, n, dtype=np.uint64)
        m = rng.random(n) < 0.02
        small[m] = rng.integers(2**8, 2**32, int(m.sum()), dtype=np.uint64)
        small = small.astype(np.uint32)
        large = rng.integers(0, 2**32, n, dtype=np.uint64).astype(np.uint32)
        vo = np.array([0, n], dtype=np.uint64)
        for vals, flag in ((small, 0), (small, 0), (large, 4), (large, 4), (small, 0)):
            want, wbo, _ = O.pack_streams(flag, vals, vo, n_threads=8)
            pb = U.pack_batch(to_dev(torch, vals), vo, flag)
            assert pb.packed_len == len(want)
            assert np.array_equal(pb.packed[:pb.packed_len].cpu().numpy(), want)
            assert np.array_equal(pb.block_off.cpu().numpy().view(np.uint64), wbo)
    finally:
        L.utl_set_knob(2, old)
