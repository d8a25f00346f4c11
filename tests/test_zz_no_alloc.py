"""GPU check of utl_pack_batch_u32_noalloc, the batched pack for callers
that cannot allocate device memory while packing -- serving loops whose
latency budget cannot absorb the device-wide synchronisation of
cudaMalloc/cudaFree, and hosts that manage a fixed device-memory budget
themselves.  The entry point keeps its look-back scratch in a fixed array
inside the library, so its packed bytes and block offsets must equal those
of utl_pack_batch_u32 given caller scratch -- exactly, since packing is
byte-exact -- on two calls in a row (the second call reuses the array the
first one left behind).  Runs alone or after the other tests.
"""
import ctypes as C
import os
import subprocess
import sys

import numpy as np
import pytest

from gen import streams

pytestmark = pytest.mark.gpu


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


def test_noalloc_pack_matches_allocating_pack():
    import torch

    from utlpfor_b200._lib import load
    L = load()
    assert torch.cuda.is_available()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    rng = np.random.default_rng(31337)
    cases = [([1 << 20], "exc", 0), ([1, 300, 4096, 0, 128 * 77 + 5, 129], "sorted", 1), ([5000, 7], "walk", 5)]
    for lens, kind, flag in cases:
        vals, vo = streams(rng, lens, kind)
        nb = L.utl_count_blocks(vo.ctypes.data_as(C.POINTER(C.c_uint64)), len(lens))
        assert nb > 0
        d_vals = torch.from_numpy(vals.view(np.int32)).cuda()
        d_vo = torch.from_numpy(vo.view(np.int64)).cuda()
        d_bs = torch.empty(len(lens) + 1, dtype=torch.int64, device="cuda")
        assert L.utl_batch_plan(_p(d_vo), len(lens), _p(d_bs), stream) == 0
        cap = nb * L.utl_max_block_length32(flag)

        # reference: the allocating entry point with caller scratch
        ref_out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
        ref_bo = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
        sb = L.utl_pack_scratch_bytes(nb)
        scratch = torch.empty(sb, dtype=torch.uint8, device="cuda")
        err = torch.zeros(1, dtype=torch.int32, device="cuda")
        rc = L.utl_pack_batch_u32(flag, _p(d_vals), _p(d_vo), _p(d_bs), len(lens), nb, _p(ref_out), cap, _p(ref_bo),
                                  None, _p(scratch), sb, _p(err), stream)
        assert rc == 0
        torch.cuda.synchronize()
        assert int(err.item()) == 0
        n = int(ref_bo[nb].item())

        for _ in range(2):
            out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
            bo = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
            err2 = torch.zeros(1, dtype=torch.int32, device="cuda")
            rc = L.utl_pack_batch_u32_noalloc(flag, _p(d_vals), _p(d_vo), _p(d_bs), len(lens), nb, _p(out), cap,
                                              _p(bo), None, _p(err2), stream)
            assert rc == 0
            torch.cuda.synchronize()
            assert int(err2.item()) == 0
            assert torch.equal(bo, ref_bo)
            assert torch.equal(out[:n], ref_out[:n])


def test_noalloc_rejects_oversized_batches():
    from utlpfor_b200._lib import load
    L = load()
    mx = L.utl_pack_batch_u32_noalloc_max_blocks()
    assert mx >= 1 << 21  # at least the 2^28-value benchmark batch
    # rejected before any device work: no pointer is touched
    rc = L.utl_pack_batch_u32_noalloc(0, None, None, None, 1, mx + 1, None, 0, None, None, None, None)
    assert rc == 13


_FIRST_CALL = r"""
import ctypes as C, sys
import numpy as np, torch
sys.path[:0] = [sys.argv[1], sys.argv[2]]
import oracle_ref as O
from gen import streams
from utlpfor_b200._lib import load
L = load()
assert L.utl_launch_count() == 0
torch.cuda.set_device(0)
p = lambda t: C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)
rng = np.random.default_rng(4242)
lens = [3000, 1, 128 * 40 + 9, 0, 700]
vals, vo = streams(rng, lens, "exc")
want, wbo, _ = O.pack_streams(0, vals, vo)
nb = len(wbo) - 1
d_vals = torch.from_numpy(vals.view(np.int32)).cuda()
d_vo = torch.from_numpy(vo.view(np.int64)).cuda()
d_bs = torch.empty(len(lens) + 1, dtype=torch.int64, device="cuda")
stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
assert L.utl_batch_plan(p(d_vo), len(lens), p(d_bs), stream) == 0
cap = nb * L.utl_max_block_length32(0)
out = torch.zeros(cap, dtype=torch.uint8, device="cuda")
bo = torch.zeros(nb + 1, dtype=torch.int64, device="cuda")
err = torch.zeros(1, dtype=torch.int32, device="cuda")
assert L.utl_launch_count() == 1  # only the plan kernel so far: this is the first pack
rc = L.utl_pack_batch_u32_noalloc(0, p(d_vals), p(d_vo), p(d_bs), len(lens), nb, p(out), cap, p(bo), None, p(err),
                                  stream)
assert rc == 0, rc
torch.cuda.synchronize()
assert int(err.item()) == 0
got_bo = bo.cpu().numpy().view(np.uint64)
assert np.array_equal(got_bo, wbo), "block offsets differ from the oracle"
n = int(got_bo[-1])
assert out[:n].cpu().numpy().tobytes() == want.tobytes(), "packed bytes differ from the oracle"
print("first-call noalloc pack ok")
"""


def test_noalloc_as_first_pack_matches_oracle():
    """The entry point as the very first pack of a fresh process (so its
    first-call set-up runs inside it): packed bytes and block offsets equal
    the oracle's."""
    tests = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(tests)
    r = subprocess.run([sys.executable, "-c", _FIRST_CALL, root, tests], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-4000:]
    assert "first-call noalloc pack ok" in r.stdout
