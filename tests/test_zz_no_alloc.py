"""GPU check of utl_pack_batch_u32_noalloc, the batched pack for callers
that cannot allocate device memory while packing -- code being recorded
into a CUDA graph (allocation is illegal during stream capture), serving
loops whose latency budget cannot absorb the device-wide synchronisation
of cudaMalloc/cudaFree, and hosts that manage a fixed device-memory budget
themselves.  The entry point keeps its look-back scratch in a fixed array
inside the library, so its packed bytes and block offsets must equal those
of utl_pack_batch_u32 given caller scratch -- exactly, since packing is
byte-exact -- on two calls in a row (the second call reuses the array the
first one left behind).  Runs alone or after the other tests.
"""
import ctypes as C

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
