"""Autotuner of the batched kernels' knobs.

Measures every candidate knob setting on a synthetic batch of the
exception-heavy shape on the current GPU (CUDA events, after warm-up) and
stores the fastest in utlpfor_b200/tuned/<gpu name>.json; apply() loads
that file (if any) for the current GPU and sets the knobs.  Knobs
(include/utlpfor.h):
  2 UTL_KNOB_PACK_SCHEDULE       blocks per warp tile: 2 = 16 (lane pair per
                                 block), 1 = 32 (one thread per block),
                                 0 = four threads per block, CTA tiles
  6 UTL_KNOB_PACK_WINDOW         1 large / 2 small tile image (warps per SM)
  1 UTL_KNOB_PACK_CTAS_PER_SM    0 occupancy maximum, else a cap
  0 UTL_KNOB_UNPACK_SCHEDULE     0 tiles; 1-3 cp.async double buffer (auto,
                                 wide, narrow staging); 4-6 TMA bulk staging
                                 (auto, three narrow groups, two wide groups
                                 in flight per warp); 8 a thread per block
                                 for small blocks, else the wide cp.async
                                 pipeline
  7 UTL_KNOB_UNPACK_CTAS_PER_SM  warps per SM of the unpack (4 per CTA):
                                 0 occupancy maximum, else a cap
The pack schedule (with the window left to its per-batch choice) is swept
first, then the CTA cap of the winner; every pack candidate must give the
same bytes, every unpack candidate the same values.

    python -m utlpfor_b200.tune [--log2n 26] [--out PATH]
"""
import argparse
import json
import os
import re

from ._lib import load

HERE = os.path.dirname(os.path.abspath(__file__))
TUNED = os.path.join(HERE, "tuned")
# Candidates are the settings that suit any batch: the window and the
# unpack staging size stay chosen per batch (window 0, unpack schedules 1,
# 4 and 8 pick by block density), so a setting tuned on one workload cannot
# slow down a batch of much larger blocks.
PACK_SHAPES = [(1, 0), (2, 0), (0, 0)]  # (schedule, window)
PACK_CAPS = [0, 16, 12, 8]
UNPACK_SCHEDULES = [8, 1, 4, 0]
UNPACK_CAPS = [0, 4, 3, 2]
KNOBS = ("0", "1", "2", "6", "7")


def _gpu_name(torch, dev=None):
    return torch.cuda.get_device_name(dev)


def config_path(name):
    return os.path.join(TUNED, re.sub(r"[^A-Za-z0-9]+", "_", name).strip("_") + ".json")


def apply(dev=None):
    """Set the knobs stored for this GPU; returns the applied dict or None."""
    import torch
    p = config_path(_gpu_name(torch, dev))
    if not os.path.exists(p):
        return None
    with open(p) as f:
        cfg = json.load(f)
    L = load()
    for k, v in cfg.get("knobs", {}).items():
        L.utl_set_knob(int(k), int(v))
    return cfg["knobs"]


def _time(fn, torch, reps=5):
    for _ in range(2):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / reps


def _workload(torch, log2n):
    """U[0,2^8) with 2% outliers in [2^8, 2^31) and 10% all-equal blocks."""
    n = 1 << log2n
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    v = torch.randint(0, 256, (n,), device="cuda", dtype=torch.int32, generator=g)
    m = torch.rand(n, device="cuda", generator=g) < 0.02
    v = torch.where(m, torch.randint(256, 2**31, (n,), device="cuda", dtype=torch.int32, generator=g), v)
    nb = n // 128
    sel = torch.rand(nb, device="cuda", generator=g) < 0.10
    c = torch.randint(0, 256, (nb,), device="cuda", dtype=torch.int32, generator=g)
    vb = v.view(nb, 128)
    vb.copy_(torch.where(sel[:, None], c[:, None], vb))
    return v


def tune(log2n=26, flag=0, write=True, out=None):
    import numpy as np
    import torch

    from .batch import BatchCodec
    L = load()
    v = _workload(torch, log2n)
    vo = np.array([0, v.numel()], dtype=np.uint64)
    codec = BatchCodec(vo, flag=flag, device="cuda", tuned=False)
    dst = torch.empty_like(v)
    old = {k: L.utl_get_knob(int(k)) for k in KNOBS}
    results = {}
    ref = None

    def pack_time():
        nonlocal ref
        t = _time(lambda: codec.pack(v), torch)
        codec.pack(v)
        torch.cuda.synchronize()
        got = codec.packed[:codec.packed_len].clone()
        if ref is None:
            ref = got
        assert torch.equal(got, ref), "a pack knob changed the packed bytes"
        return t

    def unpack_time():
        t = _time(lambda: codec.unpack(dst), torch)
        codec.unpack(dst)
        torch.cuda.synchronize()
        assert torch.equal(dst, v), "an unpack knob changed the values"
        return t

    try:
        # pack: schedule and window together, then the CTA cap
        times = {}
        for sc, win in PACK_SHAPES:
            assert L.utl_set_knob(2, sc) == 0 and L.utl_set_knob(6, win) == 0 and L.utl_set_knob(1, 0) == 0
            times["%d/%d" % (sc, win)] = pack_time()
        best_shape = min(times, key=times.get)
        results["pack schedule/window"] = times
        sc, win = (int(x) for x in best_shape.split("/"))
        L.utl_set_knob(2, sc)
        L.utl_set_knob(6, win)
        times = {}
        for cap in PACK_CAPS:
            assert L.utl_set_knob(1, cap) == 0
            times[str(cap)] = pack_time()
        results["pack ctas per SM"] = times
        pcap = int(min(times, key=times.get))
        L.utl_set_knob(1, pcap)
        codec.pack(v)
        # unpack: schedule, then the CTA cap
        times = {}
        for us in UNPACK_SCHEDULES:
            assert L.utl_set_knob(0, us) == 0 and L.utl_set_knob(7, 0) == 0
            times[str(us)] = unpack_time()
        results["unpack schedule"] = times
        us = int(min(times, key=times.get))
        L.utl_set_knob(0, us)
        times = {}
        for cap in UNPACK_CAPS:
            assert L.utl_set_knob(7, cap) == 0
            times[str(cap)] = unpack_time()
        results["unpack ctas per SM"] = times
        ucap = int(min(times, key=times.get))
    finally:
        for k, val in old.items():
            L.utl_set_knob(int(k), val)
    best = {"0": us, "1": pcap, "2": sc, "6": win, "7": ucap}
    cfg = {"gpu": _gpu_name(torch), "knobs": best, "ms": results,
           "workload": "2^%d u32, U[0,2^8) with 2%% outliers in [2^8,2^31), 10%% all-equal blocks, flag %d"
                       % (log2n, flag)}
    if write or out:
        path = out or config_path(cfg["gpu"])
        os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
        with open(path, "w") as f:
            json.dump(cfg, f, indent=1)
    return cfg


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--log2n", type=int, default=26)
    ap.add_argument("--flag", type=int, default=0)
    ap.add_argument("--no-write", action="store_true")
    ap.add_argument("--out", default=None, help="write the config here instead of the package's tuned/ folder")
    a = ap.parse_args()
    print(json.dumps(tune(a.log2n, a.flag, not a.no_write, a.out)))
