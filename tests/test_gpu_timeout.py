"""A bounded wait of the batched pack run to expiry, on purpose and safely.

The pack's tiles learn their byte offsets from the tiles before them; a
tile waits (polling, 64 ns sleeps) for its predecessors to publish.  Every
wait is bounded: after UTL_KNOB_SPIN_LIMIT polls the kernel records
UTL_ERR_TIMEOUT (bit 10 of d_err), counts the missing tile as empty and
carries on, so the launch always ends.  Here the test presets the pack's
scratch (UTL_KNOB_KEEP_SCRATCH) with the work counter already past tile 0:
tile 0 is never taken, never publishes, and every tile that needs it gives
up after a short limit.  The call must return, the stream must
synchronise, and d_err must carry the timeout bit; a normal pack right
after it on the same process must be byte-identical to the oracle again.
"""
import ctypes as C

import numpy as np
import pytest

import oracle_ref as O
from gen import streams

pytestmark = pytest.mark.gpu

SPIN_LIMIT, KEEP_SCRATCH, PACK_SCHEDULE = 4, 5, 2
TIMEOUT_BIT = 1 << 10


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


@pytest.mark.parametrize("is64,schedule", [(False, 2), (False, 1), (False, 0), (True, 1), (True, 0)],
                         ids=["u32_pair", "u32_lane", "u32_quad", "u64_lane", "u64_warp"])
def test_pack_wait_expires_and_reports_timeout(is64, schedule):
    import time

    import torch

    from utlpfor_b200._lib import load
    L = load()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(1010)
    lens = [128 * 32 * 12 + 5]  # a dozen tiles and a ragged tail
    vals, vo = streams(rng, lens, "walk" if is64 else "exc", is64=is64)
    want, wbo, _ = O.pack_streams(0, vals, vo)
    nb = len(wbo) - 1
    d_vals = torch.from_numpy(vals.view(np.int64 if is64 else np.int32)).cuda()
    d_vo = torch.from_numpy(vo.view(np.int64)).cuda()
    d_bs = torch.empty(2, dtype=torch.int64, device="cuda")
    assert L.utl_batch_plan(_p(d_vo), 1, _p(d_bs), stream) == 0
    mx = L.utl_max_block_length64(0) if is64 else L.utl_max_block_length32(0)
    cap = nb * mx
    sb = L.utl_pack_scratch_bytes(nb)
    pack = L.utl_pack_batch_u64 if is64 else L.utl_pack_batch_u32
    olds = [L.utl_get_knob(k) for k in (SPIN_LIMIT, KEEP_SCRATCH, PACK_SCHEDULE)]
    try:
        assert L.utl_set_knob(PACK_SCHEDULE, schedule) == 0
        assert L.utl_set_knob(SPIN_LIMIT, 1024) == 0
        assert L.utl_set_knob(KEEP_SCRATCH, 1) == 0
        scratch = torch.zeros(sb, dtype=torch.uint8, device="cuda")
        scratch[:8].view(torch.int64).fill_(1)  # the work counter: tile 0 is never handed out
        out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        bo = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        rc = pack(0, _p(d_vals), _p(d_vo), _p(d_bs), 1, nb, _p(out), cap, _p(bo), None, _p(scratch), sb, _p(err),
                  stream)
        assert rc == 0
        torch.cuda.synchronize()  # the launch ends on its own
        elapsed = time.perf_counter() - t0
        assert int(err.item()) & TIMEOUT_BIT, "no timeout recorded"
        assert elapsed < 30.0
    finally:
        for k, v in zip((SPIN_LIMIT, KEEP_SCRATCH, PACK_SCHEDULE), olds):
            L.utl_set_knob(k, v)

    # the same process packs normally afterwards
    scratch = torch.empty(sb, dtype=torch.uint8, device="cuda")
    out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
    bo = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = pack(0, _p(d_vals), _p(d_vo), _p(d_bs), 1, nb, _p(out), cap, _p(bo), None, _p(scratch), sb, _p(err), stream)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    assert np.array_equal(bo.cpu().numpy().view(np.uint64), wbo)
    n = int(wbo[-1])
    assert out[:n].cpu().numpy().tobytes() == want.tobytes()


def test_test_knobs_round_trip():
    from utlpfor_b200._lib import load
    L = load()
    for k, vals in ((SPIN_LIMIT, (0, 1, 1 << 22)), (KEEP_SCRATCH, (0, 1))):
        old = L.utl_get_knob(k)
        for v in vals:
            assert L.utl_set_knob(k, v) == 0 and L.utl_get_knob(k) == v
        assert L.utl_set_knob(k, -1) != 0
        L.utl_set_knob(k, old)
