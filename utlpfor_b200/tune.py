"""Autotuner of the batched kernels' schedule knobs.

Measures every candidate knob setting on a synthetic batch with the given
shape on the current GPU and stores the fastest in
utlpfor_b200/tuned/<gpu name>.json; apply() loads that file (if any) for
the current GPU and sets the knobs.  Knobs (include/utlpfor.h):
  0 UTL_KNOB_UNPACK_SCHEDULE   0 tiles, 1 persistent pipelined (staging by block size), 2/3 wide/narrow only
  1 UTL_KNOB_PACK_CTAS_PER_SM  0 occupancy maximum, else a cap
  2 UTL_KNOB_PACK_SCHEDULE     0 four threads per block, 1 one thread per block

    python -m utlpfor_b200.tune [--log2n 26]
"""
import argparse
import json
import os
import re

from ._lib import load

HERE = os.path.dirname(os.path.abspath(__file__))
TUNED = os.path.join(HERE, "tuned")
CANDIDATES = {0: [0, 1], 2: [1, 0], 1: [0, 3, 2]}  # pack schedule before its CTA cap


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


def tune(log2n=26, flag=0, write=True):
    import numpy as np
    import torch

    from .batch import BatchCodec
    L = load()
    n = 1 << log2n
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    v = torch.randint(0, 256, (n,), device="cuda", dtype=torch.int32, generator=g)
    m = torch.rand(n, device="cuda", generator=g) < 0.02
    v = torch.where(m, torch.randint(256, 2**31, (n,), device="cuda", dtype=torch.int32, generator=g), v)
    vo = np.array([0, n], dtype=np.uint64)
    codec = BatchCodec(vo, flag=flag, device="cuda")
    out = torch.empty_like(v)
    codec.pack(v)
    best, results = {}, {}
    ref = None
    for knob, cands in CANDIDATES.items():
        times = {}
        for c in cands:
            assert L.utl_set_knob(knob, c) == 0
            if knob == 0:
                t = _time(lambda: codec.unpack(out), torch)
                codec.unpack(out)
                torch.cuda.synchronize()
                assert torch.equal(out, v), "unpack schedule %d gave wrong values" % c
            else:
                t = _time(lambda: codec.pack(v), torch)
                codec.pack(v)
                torch.cuda.synchronize()
                got = codec.packed[:codec.packed_len].clone()
                if ref is None:
                    ref = got
                assert torch.equal(got, ref), "pack knob %d=%d changed the packed bytes" % (knob, c)
            times[c] = t
        pick = min(times, key=times.get)
        L.utl_set_knob(knob, pick)
        best[str(knob)] = pick
        results[str(knob)] = {str(c): t for c, t in times.items()}
    cfg = {"gpu": _gpu_name(torch), "knobs": best, "ms": results,
           "workload": "2^%d u32, U[0,2^8) with 2%% outliers, flag %d" % (log2n, flag)}
    if write:
        os.makedirs(TUNED, exist_ok=True)
        with open(config_path(cfg["gpu"]), "w") as f:
            json.dump(cfg, f, indent=1)
    return cfg


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--log2n", type=int, default=26)
    ap.add_argument("--flag", type=int, default=0)
    ap.add_argument("--no-write", action="store_true")
    a = ap.parse_args()
    print(json.dumps(tune(a.log2n, a.flag, not a.no_write)))
