"""Byte parity with the oracle at the benchmark configurations' full sizes.

Each case generates the exact seeded workload bench.py measures (on the
device, with bench.make_workload), packs it with the batched pack, and
compares the packed bytes (length and SHA-256), every block offset and
every stream offset with the oracle's block-by-block Append packing of
the same values on the host; then unpacks on the device and compares with
the values.  A round trip alone cannot catch a wrong width, FOR or
exception decision that still decodes; byte equality does.  The delta
posting-list configuration is also queried with 2^20 random Get queries,
checked against the oracle's GetUint32 on the oracle's bytes.

    c1  2^20 u32 uniform [0, 2^11), flag 0
    c2  1000 posting lists (log-uniform lengths in [128, 2^20], gaps
        1+Geom(1/64)), flags Delta and Delta|NoFOR
    c3  2^28 u32 in 2^21 blocks, U[0,2^8) with 2% U[2^8,2^32) and 10% of
        blocks all-equal, flags 0, NoFOR and NoPatch
    c4  2^26 u64 in 512 streams (FOR-reducible, full-range, random walks),
        flag Delta
"""
import hashlib
import os

import numpy as np
import pytest

import oracle_ref as O

pytestmark = pytest.mark.gpu

DELTA, NOFOR, NOPATCH = 1, 2, 4
CASES = [("c1", 0), ("c2", DELTA), ("c2", DELTA | NOFOR), ("c3", 0), ("c3", NOFOR), ("c3", NOPATCH), ("c4", DELTA)]


def _threads():
    try:
        return max(1, len(os.sched_getaffinity(0)))
    except AttributeError:
        return os.cpu_count() or 1


@pytest.fixture(scope="module")
def env():
    import torch

    import bench
    import utlpfor_b200 as U
    assert torch.cuda.is_available()
    return U, torch, bench


def _sha(a):
    return hashlib.sha256(memoryview(np.ascontiguousarray(a))).hexdigest()


@pytest.mark.parametrize("name,flag", CASES, ids=["%s-flag%d" % c for c in CASES])
def test_full_size_bytes_match_oracle(env, name, flag):
    U, torch, bench = env
    dev = torch.device("cuda", 0)
    values, vo = bench.make_workload(torch, name, 0, dev)
    is64 = values.element_size() == 8
    host = values.cpu().numpy().view(np.uint64 if is64 else np.uint32)
    want, wbo, wso = O.pack_streams(flag, host, vo, n_threads=_threads())
    pb = U.pack_batch(values, vo, flag)
    assert pb.packed_len == len(want)
    got = pb.packed[:pb.packed_len].cpu().numpy()
    assert _sha(got) == _sha(want), "packed bytes differ from the oracle"
    assert np.array_equal(pb.block_off.cpu().numpy().view(np.uint64), wbo)
    assert np.array_equal(pb.stream_byte_off.cpu().numpy().view(np.uint64), wso)
    del got
    out = U.unpack_batch(pb)
    assert torch.equal(out, values)
    if name == "c2":
        nq = 1 << 20
        rng = np.random.default_rng(2020 + flag)
        lens = (vo[1:] - vo[:-1]).astype(np.int64)
        qs = rng.integers(0, lens.size, nq).astype(np.uint32)
        qp = (rng.random(nq) * lens[qs]).astype(np.uint64)
        ov, ost = O.get_streams(want, wbo, vo, qs, qp)
        assert np.all(ost == 0)
        gv, gst = U.get_batch(pb, torch.from_numpy(qs.view(np.int32)).to(dev),
                              torch.from_numpy(qp.view(np.int64)).to(dev))
        assert np.array_equal(gst.cpu().numpy(), ost)
        assert np.array_equal(gv.cpu().numpy().view(np.uint32), ov)
        assert np.array_equal(ov, host[vo[qs].astype(np.int64) + qp.astype(np.int64)])
