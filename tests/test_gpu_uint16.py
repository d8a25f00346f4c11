"""Blocks whose header names the uint16 integer type (IntTypeUint16).

No encoder in the reference writes them, but its uint32 decoders accept
them (validateIntType, header.go:169-180; decodeUnpackHeader,
unpack_block.go:62-172): the payload is read exactly as for uint32.  The
blocks here are hand-built from oracle-packed uint32 blocks by rewriting
the header's integer-type field (bits 13-14) from 2 to 1.  UnpackUint32,
GetUint32, BlockLength and Header on the GPU (per call) and the batched
unpack and Get must give what the oracle gives for the same bytes; the
uint64 decoders must reject them (validateIntType64) with the oracle's
error.
"""
import numpy as np
import pytest

import oracle_ref as O
from gen import block_values

pytestmark = pytest.mark.gpu


def as_u16(block):
    b = bytearray(block)
    h = int.from_bytes(b[:4], "little")
    h = (h & ~(3 << 13)) | (1 << 13)
    b[:4] = h.to_bytes(4, "little")
    return bytes(b)


def code_of(fn):
    import utlpfor_b200 as U
    try:
        return fn(), 0, 0
    except U.ErrOverflow as e:
        return None, 7, e.Position
    except U.UTLError as e:
        return None, e.code, 0


def cases(rng):
    for flag in range(16):
        for kind in ("small", "exc", "dense_exc", "sorted", "walk", "const", "zero"):
            for n in (1, 77, 128):
                v = block_values(rng, n, kind)
                blk, err = O.pack_u32(flag, v)
                assert err == 0
                yield flag, kind, v, as_u16(blk)


def test_uint16_blocks_per_call():
    import utlpfor_b200 as U
    rng = np.random.default_rng(16)
    for flag, kind, v, blk in cases(rng):
        ov, oc, oerr, oovf = O.unpack_u32(blk)
        assert oerr == 0 and np.array_equal(ov, v), (flag, kind)
        got, gerr, govf = code_of(lambda: U.UnpackUint32(blk))
        assert (gerr, govf) == (oerr, oovf)
        assert np.array_equal(got[0], ov) and got[1] == oc
        assert U.BlockLength(blk) == O.block_length(blk)[0] == len(blk)
        hdr, herr = O.header(blk)
        assert herr == 0
        assert list(U.Header(blk)) == [hdr[0], hdr[1], hdr[2], bool(hdr[3]), bool(hdr[4]), bool(hdr[5]),
                                       bool(hdr[6])]
        for pos in range(0, len(v), 7):
            gv, gerr, govf = O.get_u32(pos, blk)
            assert gerr == 0
            assert U.GetUint32(pos, blk) == gv == v[pos]
        # the uint64 decoders reject the type as the oracle does
        _, uerr, _ = code_of(lambda: U.UnpackUint64(blk))
        assert uerr == O.unpack_u64(blk)[2] == 5
        _, uerr, _ = code_of(lambda: U.GetUint64(0, blk))
        assert uerr == O.get_u64(0, blk)[1] == 5


def test_uint16_blocks_batched():
    import torch

    import utlpfor_b200 as U
    rng = np.random.default_rng(61)
    blocks, vals, lens = [], [], []
    for flag, kind, v, blk in cases(rng):
        blocks.append(blk)
        vals.append(v)
        lens.append(len(v))
    packed = np.frombuffer(b"".join(blocks), dtype=np.uint8).copy()
    bo = np.concatenate([[0], np.cumsum([len(b) for b in blocks])]).astype(np.uint64)
    vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
    values = np.concatenate(vals).astype(np.uint32)
    want, err = O.unpack_streams(packed, bo, vo)
    assert err == 0 and np.array_equal(want, values)
    dev_vals = torch.from_numpy(values.view(np.int32)).cuda()
    pb = U.pack_batch(dev_vals, vo, 0)  # the stream table; the bytes are replaced below
    d_packed = torch.from_numpy(packed).cuda()
    d_bo = torch.from_numpy(bo.view(np.int64)).cuda()
    status = torch.full((pb.n_blocks,), -1, dtype=torch.int32, device="cuda")
    out = U.unpack_batch(pb, block_status=status, packed=d_packed, block_off=d_bo)
    assert np.array_equal(status.cpu().numpy(), np.zeros(pb.n_blocks, dtype=np.int32))
    assert np.array_equal(out.cpu().numpy().view(np.uint32), values)
    # batched Get over the same bytes
    qs = rng.integers(0, len(lens), 5000).astype(np.uint32)
    qp = (rng.random(5000) * np.array(lens)[qs]).astype(np.uint64)
    ov, ost = O.get_streams(packed, bo, vo, qs, qp)
    pb.packed, pb.block_off = d_packed, d_bo
    gv, gst = U.get_batch(pb, torch.from_numpy(qs.view(np.int32)).cuda(), torch.from_numpy(qp.view(np.int64)).cuda())
    assert np.array_equal(gst.cpu().numpy(), ost)
    assert np.array_equal(gv.cpu().numpy().view(np.uint32), ov)
