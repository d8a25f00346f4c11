"""The batched pack + unpack recorded into a CUDA graph replays to the same
bytes and values as eager launches; and the autotuner's candidates all
give identical results."""
import numpy as np
import pytest

from gen import streams

pytestmark = pytest.mark.gpu


def test_graph_replay_matches_eager():
    import torch

    import utlpfor_b200 as U
    rng = np.random.default_rng(99)
    vals, vo = streams(rng, [128 * 300 + 17, 5, 4096], "exc")
    d = torch.from_numpy(vals.view(np.int32)).cuda()
    codec = U.BatchCodec(vo, flag=0)
    out = torch.empty_like(d)
    codec.pack(d)
    torch.cuda.synchronize()
    n = codec.packed_len
    eager = codec.packed[:n].clone()
    bo = codec.block_off.clone()
    g = codec.capture(d, out)
    for _ in range(2):
        codec.packed.zero_()
        out.zero_()
        g.replay()
        torch.cuda.synchronize()
        assert torch.equal(codec.packed[:n], eager)
        assert torch.equal(codec.block_off, bo)
        assert torch.equal(out, d)
    assert codec.error_bits() == 0


def test_tuner_candidates_agree():
    """Every candidate of every knob the tuner sweeps (pack tile size and
    window, pack and unpack warps per SM, unpack schedule) gives the same
    bytes and values; the tuner reports a choice for each knob and leaves
    the knobs as it found them."""
    from utlpfor_b200._lib import load
    from utlpfor_b200.tune import KNOBS, tune
    L = load()
    before = {k: L.utl_get_knob(int(k)) for k in KNOBS}
    cfg = tune(log2n=18, write=False)
    assert set(cfg["knobs"]) == set(KNOBS)
    assert {k: L.utl_get_knob(int(k)) for k in KNOBS} == before
