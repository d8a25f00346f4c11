#!/usr/bin/env python
"""Benchmark of the batched UTL-PFOR codec on B200.

One step = one batched PackUint32 pass over the whole workload followed by
one batched UnpackUint32 pass over the packed result (a round trip),
inputs resident in HBM.  The default workload is the exception-heavy
configuration: 2^28 uint32 values in 2^21 blocks of 128, values uniform in
[0, 2^8) except with probability 0.02 uniform in [2^8, 2^32), and 10% of
blocks all-equal (constant drawn uniform in [0, 2^8)), flag 0, seeded
synthetic data.  The working set (1 GiB of values in, 1 GiB out) is far
larger than L2, so no L2 flush is needed between steps.

Printed: ONE JSON line (rank 0).  value = uncompressed round-trip
throughput (bytes of values packed + bytes of values unpacked) / step
time, summed over ranks.  e2e = the same metric through the host-buffer
C-ABI calls (utl_pack_streams_u32 / utl_unpack_streams_u32) with pinned
host memory, copies included.  get = 2^20 random GetUint32 queries over the
packed result in one batched launch (queries/s).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                    [--workload c3|c3-nofor|c3-nopatch|c1|c2|c4|c5]

The c5 workload measures the serving loop instead (utlpfor_b200.serve):
requests with host buffers arrive open-loop at swept Poisson rates; the
line reports per-rate p50/p99 latency and sustained uncompressed GB/s, and
the same request mix through the plain per-call C-ABI on a sample.
"""
import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

DELTA, NOFOR, NOPATCH = 1, 2, 4
L2_BYTES = 126 * 2**20


# --------------------------------------------------------------------------
# workloads (seeded synthetic data with the configs' shapes)
# --------------------------------------------------------------------------
WORKLOADS = {
    "c3": dict(desc="pfor_exception_heavy: 2^28 u32 in 2^21 blocks, U[0,2^8) + 2% U[2^8,2^32), "
                    "10% all-equal blocks", flag=0, is64=False),
    "c3-nofor": dict(desc="pfor_exception_heavy (flag NoFOR)", flag=NOFOR, is64=False),
    "c3-nopatch": dict(desc="pfor_exception_heavy (flag NoPatch)", flag=NOPATCH, is64=False),
    "c1": dict(desc="plain_round_trip: 2^20 u32 uniform [0,2^11), flag 0", flag=0, is64=False),
    "c2": dict(desc="delta_posting_lists: 1000 lists log-uniform [128,2^20], gaps 1+Geom(1/64), flag Delta",
               flag=DELTA, is64=False),
    "c4": dict(desc="uint64_streams: 2^26 u64 in 512 streams, 1/3 FOR-reducible, 1/3 full-range, "
                    "1/3 random walks from 2^62 (flag Delta)", flag=DELTA, is64=True),
    "c5": dict(desc="served_mixed_requests: Poisson arrivals, 60/30/10 decompress/compress/Get, sizes "
                    "log-uniform [128,2^22] u32 drawn from the c1/c2/c3 distributions, 64 GB admission budget",
               flag=0, is64=False),
}


def gen_c3_torch(torch, n, gen, dev):
    v = torch.randint(0, 256, (n,), device=dev, dtype=torch.int32, generator=gen)
    m = torch.rand(n, device=dev, generator=gen) < 0.02
    big = torch.randint(256, 2**32, (n,), device=dev, dtype=torch.int64, generator=gen).to(torch.int32)
    v = torch.where(m, big, v)
    del big, m
    nb = n // 128
    sel = torch.rand(nb, device=dev, generator=gen) < 0.10
    c = torch.randint(0, 256, (nb,), device=dev, dtype=torch.int32, generator=gen)
    vb = v.view(nb, 128)
    vb.copy_(torch.where(sel[:, None], c[:, None], vb))
    return v


def loguniform_lengths(rng, n, lo, hi):
    return np.exp(rng.uniform(np.log(lo), np.log(hi), n)).astype(np.int64)


def make_workload(torch, name, rank, dev, log2n=28):
    """Returns (values CUDA tensor, val_off numpy uint64)."""
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234 + rank)
    rng = np.random.default_rng(1234 + rank)
    if name.startswith("c3"):
        n = 1 << log2n
        return gen_c3_torch(torch, n, gen, dev), np.array([0, n], dtype=np.uint64)
    if name == "c1":
        n = 1 << 20
        v = torch.randint(0, 2**11, (n,), device=dev, dtype=torch.int32, generator=gen)
        return v, np.array([0, n], dtype=np.uint64)
    if name == "c2":
        lens = loguniform_lengths(rng, 1000, 128, 2**20)
        vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
        n = int(vo[-1])
        gaps = 1 + torch.distributions.Geometric(probs=torch.tensor(1 / 64, device=dev)).sample((n,)).to(torch.int64)
        # per-list cumulative sums: global cumsum minus the list's starting prefix
        cs = torch.cumsum(gaps, 0)
        starts = torch.from_numpy(vo[:-1].astype(np.int64)).to(dev)
        base = torch.where(starts > 0, cs[(starts - 1).clamp(min=0)], torch.zeros_like(starts))
        rep = torch.repeat_interleave(base, torch.from_numpy(lens).to(dev))
        v = (cs - rep).to(torch.int32)
        return v, vo
    if name == "c4":
        lens = loguniform_lengths(rng, 512, 128, 2**18).astype(np.float64)
        lens = np.maximum(128, np.round(lens * (2**26 / lens.sum()))).astype(np.int64)
        vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
        parts = []
        for s, ln in enumerate(lens):
            ln = int(ln)
            kind = s % 3
            if kind == 0:
                x = (2**40 + torch.randint(0, 2**20, (ln,), device=dev, dtype=torch.int64, generator=gen))
            elif kind == 1:
                x = torch.randint(-2**63, 2**63 - 1, (ln,), device=dev, dtype=torch.int64, generator=gen)
            else:
                steps = torch.randint(-1000, 1001, (ln,), device=dev, dtype=torch.int64, generator=gen)
                x = 2**62 + torch.cumsum(steps, 0)
            parts.append(x)
        return torch.cat(parts), vo
    raise ValueError(name)


# --------------------------------------------------------------------------
# clocks sampled during the timed region
# --------------------------------------------------------------------------
class ClockSampler:
    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_id):
        self.gpu_id = gpu_id
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu_id), "--query-gpu=" + self.QUERY, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except OSError:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        self.t.join(timeout=2)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for nm, val in zip(names, f[5:9]):
                if val.lower().startswith("active"):
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def gpu_smi_id(torch, dev_index):
    """nvidia-smi -i id of a torch device: its UUID, else its PCI bus id."""
    try:
        props = torch.cuda.get_device_properties(dev_index)
        u = getattr(props, "uuid", None)
        if u:
            u = str(u)
            return u if u.startswith("GPU-") else "GPU-" + u
        return "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
    except Exception:
        pass
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        return vis.split(",")[dev_index]
    return dev_index


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def profiled_traffic():
    """dram bytes per value of the pack and unpack kernels from the
    committed ncu summary (profiles/*.txt lines 'traffic_per_value <kernel> <bytes>')."""
    out = {}
    d = os.path.join(ROOT, "profiles")
    if os.path.isdir(d):
        for fn in sorted(os.listdir(d)):
            if not fn.endswith(".txt"):
                continue
            with open(os.path.join(d, fn)) as f:
                for ln in f:
                    p = ln.split()
                    if len(p) == 3 and p[0] == "traffic_per_value":
                        try:
                            out[p[1]] = float(p[2])
                        except ValueError:
                            pass
    return out


# --------------------------------------------------------------------------
# CPU side: the oracle restatement timed on the host cores
# --------------------------------------------------------------------------
def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_round_trip(values_np, val_off, flag, threads, min_seconds=10.0, max_rounds=50, rounds=None):
    """Pack + unpack the values on `threads` host threads with the CPU
    restatement of the reference's vectorized pipelines (AVX-512, else
    AVX2: oracle/utl_simd.c), into output buffers allocated once (as a
    caller packing into preallocated slices would).  Returns the per-round
    seconds."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ref as O
    times = []
    out = bo = None
    vals_out = np.empty_like(values_np)
    t_start = time.perf_counter()
    while True:
        t0 = time.perf_counter()
        packed, bo, _ = O.pack_streams(flag, values_np, val_off, n_threads=threads, simd=True, out=out, bo=bo,
                                       want_so=False)
        _, err = O.unpack_streams(packed, bo, val_off, dtype=values_np.dtype, n_threads=threads, simd=True,
                                  out=vals_out)
        t1 = time.perf_counter()
        assert err == 0
        if out is None:
            out = packed.base if packed.base is not None else packed
            assert np.array_equal(vals_out, values_np), "CPU round trip mismatch"
        times.append(t1 - t0)
        if rounds is not None:
            if len(times) >= rounds:
                break
        elif time.perf_counter() - t_start >= min_seconds or len(times) >= max_rounds:
            break
    return times


def cpu_kind():
    """Which CPU pipeline the baseline times, for the JSON line."""
    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import oracle_ref as O
    lv = O.simd_level()
    name = {2: "AVX-512", 1: "AVX2"}.get(lv, "scalar")
    return ("%s restatement of the reference's packBlockAVX512/unpackBlockAVX512 pipelines "
            "(oracle/utl_simd.c; AVX-512 before AVX2 as the reference dispatches)" % name)


def c3_sample_host(n, seed):
    rng = np.random.default_rng(seed)
    v = rng.integers(0, 256, n, dtype=np.uint32)
    m = rng.random(n, dtype=np.float32) < 0.02
    v[m] = rng.integers(256, 2**32, int(m.sum()), dtype=np.uint64).astype(np.uint32)
    nb = n // 128
    sel = rng.random(nb) < 0.10
    c = rng.integers(0, 256, nb, dtype=np.uint32)
    vb = v.reshape(nb, 128)
    vb[sel] = c[sel][:, None]
    return v


def make_workload_host(name, seed, log2n=28):
    """Host (numpy) version of make_workload: the same shapes and
    distributions (other random draws), for the CPU reference arm."""
    rng = np.random.default_rng(seed)
    if name.startswith("c3"):
        n = 1 << log2n
        return c3_sample_host(n, seed), np.array([0, n], dtype=np.uint64)
    if name == "c1":
        n = 1 << 20
        return rng.integers(0, 2**11, n, dtype=np.uint32), np.array([0, n], dtype=np.uint64)
    if name == "c2":
        lens = loguniform_lengths(rng, 1000, 128, 2**20)
        vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
        v = np.empty(int(vo[-1]), dtype=np.uint32)
        for s, ln in enumerate(lens):
            v[int(vo[s]):int(vo[s + 1])] = np.cumsum(rng.geometric(1 / 64, int(ln)), dtype=np.int64).astype(np.uint32)
        return v, vo
    if name == "c4":
        lens = loguniform_lengths(rng, 512, 128, 2**18).astype(np.float64)
        lens = np.maximum(128, np.round(lens * (2**26 / lens.sum()))).astype(np.int64)
        vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
        parts = []
        for s, ln in enumerate(lens):
            kind = s % 3
            if kind == 0:
                x = np.uint64(2**40) + rng.integers(0, 2**20, int(ln), dtype=np.uint64)
            elif kind == 1:
                x = rng.integers(0, 2**64 - 1, int(ln), dtype=np.uint64, endpoint=True)
            else:
                x = (np.int64(2**62) + np.cumsum(rng.integers(-1000, 1001, int(ln)))).astype(np.uint64)
            parts.append(x)
        return np.concatenate(parts), vo
    raise ValueError(name)


def workload_config(name, n, n_blocks, world):
    """The config object both arms print (the workload, not its packed
    size, which depends on the random draws)."""
    wl = WORKLOADS[name]
    return {"workload": wl["desc"], "flag": wl["flag"], "values_per_gpu": n, "blocks_per_gpu": n_blocks,
            "l2": "inputs larger than L2 (no flush)" if n * (8 if wl["is64"] else 4) > L2_BYTES else "inputs fit L2",
            "parallelism": "replicas" if world > 1 else "1 GPU"}


# --------------------------------------------------------------------------
def run_reference(args):
    """The reference arm: the reference's CPU algorithm on the host cores
    (the Go module needs a Go 1.27 toolchain, absent here, so its AVX-512 /
    AVX2 pipelines run as restated in C), on this arm's workload at full
    size, all host threads, same metric."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    wl = WORKLOADS[args.workload]
    threads = host_threads()
    vals, vo = make_workload_host(args.workload, 1234, args.log2n)
    n = int(vo[-1])
    esz = vals.dtype.itemsize
    nb = int(sum((int(vo[s + 1] - vo[s]) + 127) // 128 for s in range(len(vo) - 1)))
    cpu_round_trip(vals, vo, wl["flag"], threads, rounds=max(args.warmup, 1))
    times = cpu_round_trip(vals, vo, wl["flag"], threads, rounds=args.steps)
    t = sum(times) / len(times)
    gbps = 2 * esz * n / t / 1e9
    sample = "the whole workload (%d values, %d MiB) per step" % (n, esz * n >> 20)
    line = {"metric": "round-trip uncompressed GB/s (batched PackUint32 + UnpackUint32)", "value": gbps,
            "unit": "GB/s", "impl": "reference", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t * 1e3, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64" if esz == 8 else "u32", "data": "synthetic (seeded, the workload's distribution, on host)",
            "config": workload_config(args.workload, n, nb, 1),
            "cpu_baseline": {"value": gbps, "unit": "GB/s", "cores": threads, "kind": "port", "impl": cpu_kind(),
                             "sample": sample},
            "e2e": {"value": gbps, "unit": "GB/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# --------------------------------------------------------------------------
# serving workload (c5)
# --------------------------------------------------------------------------
def c5_pools(seed, n=1 << 23):
    """Host value pools of the c1/c2/c3 distributions; a request's values
    are a contiguous slice of one pool."""
    rng = np.random.default_rng(seed)
    c1 = rng.integers(0, 2**11, n, dtype=np.uint64).astype(np.uint32)
    c2 = np.cumsum(1 + rng.geometric(1 / 64, n)).astype(np.uint32)
    c3 = c3_sample_host(n, seed + 1)
    return [(c1, 0), (c2, DELTA), (c3, 0)]


def c5_requests(rng, count, pools, n_resident):
    """(kind, pool, start, size, handle index) per request: 60% decompress,
    30% compress, 10% Get; sizes log-uniform in [128, 2^22]; a Get asks for
    min(size/128, 4096) uniform positions of a resident stream."""
    kinds = rng.choice(3, count, p=[0.6, 0.3, 0.1])
    sizes = np.exp(rng.uniform(np.log(128), np.log(2**22), count)).astype(np.int64)
    out = []
    for k, sz in zip(kinds, sizes):
        pi = int(rng.integers(0, len(pools)))
        start = int(rng.integers(0, pools[pi][0].size - sz))
        out.append((("decompress", "compress", "get")[k], pi, start, int(sz), int(rng.integers(0, n_resident))))
    return out


def run_serving(args):
    import torch

    import utlpfor_b200.serve as S
    from utlpfor_b200._lib import load
    L = load()
    torch.cuda.set_device(0)
    pools = c5_pools(5)
    rng = np.random.default_rng(6)
    budget = 64 << 30
    srv = S.CodecServer(budget_bytes=budget, slots=args.serve_slots)
    # resident streams the decompress/Get requests read
    n_res = 64
    res_specs = c5_requests(rng, n_res, pools, 1)
    handles = [srv.submit_compress(pools[pi][0][st:st + sz], pools[pi][1]) for _, pi, st, sz, _ in res_specs]
    handles = [f.result(timeout=300) for f in handles]
    for h, (_, pi, st, sz, _) in zip(handles, res_specs):  # resident streams decode to their values
        assert np.array_equal(srv.submit_decompress(h).result(timeout=300), pools[pi][0][st:st + sz])
    errors = []

    def submit(spec):
        kind, pi, st, sz, hi = spec
        if kind == "compress":
            f = srv.submit_compress(pools[pi][0][st:st + sz], pools[pi][1])

            def drop(fut):
                if fut.exception() is not None:
                    errors.append(repr(fut.exception()))
                else:
                    srv.release(fut.result())
            f.add_done_callback(drop)
            return
        if kind == "decompress":
            f = srv.submit_decompress(handles[hi])
        else:
            h = handles[hi]
            q = min(max(sz // 128, 1), 4096)
            f = srv.submit_get(h, (np.arange(q, dtype=np.int64) * 7919) % h.n_values)
        f.add_done_callback(lambda fut: fut.exception() is not None and errors.append(repr(fut.exception())))

    def run_point(specs, rate):
        """Open-loop arrivals at `rate` requests/s (None: all at once)."""
        srv.reset_stats()
        t0 = time.perf_counter()
        gaps = rng.exponential(1.0 / rate, len(specs)) if rate else np.zeros(len(specs))
        due = t0 + np.cumsum(gaps)
        for spec, d in zip(specs, due):
            w = d - time.perf_counter()
            if w > 0:
                time.sleep(w)
            submit(spec)
        srv.drain()
        wall = time.perf_counter() - t0
        st = srv.stats()
        return {"offered_req_per_s": rate, "requests": len(specs), "wall_s": round(wall, 3),
                "served_req_per_s": round(len(specs) / wall, 1),
                "sustained_GBps": round(st["uncompressed_bytes"] / wall / 1e9, 3),
                "p50_ms": round(st["all"]["p50_ms"], 3), "p99_ms": round(st["all"]["p99_ms"], 3),
                "by_kind": {k: {"p50_ms": round(st[k]["p50_ms"], 3), "p99_ms": round(st[k]["p99_ms"], 3)}
                            for k in ("compress", "decompress", "get") if k in st},
                "batches": st["batches"], "max_batches_in_flight": st["max_batches_in_flight"],
                "admitted": st["admitted"], "rejected": st["rejected"]}

    run_point(c5_requests(rng, 200, pools, n_res), None)   # warm-up: allocator caches, first launches
    nreq = args.serve_requests
    burst = run_point(c5_requests(rng, nreq, pools, n_res), None)
    cap = burst["served_req_per_s"]
    points = [run_point(c5_requests(rng, nreq, pools, n_res), round(cap * f, 1)) for f in (0.25, 0.5, 0.9)]
    srv.close()

    # the same mix through the plain per-call C-ABI (one call per block / position), on a sample
    sample = c5_requests(np.random.default_rng(7), 40, pools, n_res)
    res_bytes = []
    for _, pi, st, sz, _ in res_specs:
        pk, bo, _ = U_pack_host(pools[pi][0][st:st + sz], pools[pi][1])
        res_bytes.append((pk, bo, sz))
    t0 = time.perf_counter()
    moved = 0
    for kind, pi, st, sz, hi in sample:
        if kind == "compress":
            U_pack_host(pools[pi][0][st:st + sz], pools[pi][1], plain=L)
            moved += 4 * sz
        elif kind == "decompress":
            pk, bo, n = res_bytes[hi]
            U_unpack_host(pk, bo, n, L)
            moved += 4 * n
        else:
            pk, bo, n = res_bytes[hi]
            q = min(max(sz // 128, 1), 4096)
            U_get_host(pk, bo, (np.arange(q, dtype=np.int64) * 7919) % n, L)
            moved += 4 * q
    plain_wall = time.perf_counter() - t0
    best = max([burst] + points, key=lambda p: p["sustained_GBps"])
    line = {"metric": "served sustained uncompressed GB/s (p50/p99 latency per offered rate)",
            "value": best["sustained_GBps"], "unit": "GB/s", "n_gpus": 1, "steps": len(points) + 1,
            "warmup": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32",
            "data": "synthetic (seeded pools of the c1/c2/c3 distributions)",
            "config": {"workload": WORKLOADS["c5"]["desc"], "requests_per_point": nreq,
                       "resident_streams": n_res, "slots": args.serve_slots, "budget_bytes": budget,
                       "results": "to host (numpy), inputs from host"},
            "serving": {"burst": burst, "rates": points},
            "plain_per_call": {"requests": len(sample), "GBps": round(moved / plain_wall / 1e9, 4),
                               "wall_s": round(plain_wall, 2),
                               "calls": "utl_pack_u32 / utl_unpack_u32 per 128-value block, utl_get_u32 per position"},
            "errors": errors[:5], "gpu_launches": None}
    print(json.dumps(line))
    return 0


def U_pack_host(values, flag, plain=None):
    """Pack one stream block by block through the per-call C-ABI (plain) or
    the batched host-buffer call; returns (packed, block_off, stream_off)."""
    from utlpfor_b200 import batch
    if plain is None:
        return batch.pack_streams(flag, values, np.array([0, values.size], dtype=np.uint64))
    buf = np.empty(600, dtype=np.uint8)
    n = C.c_size_t(0)
    pu8 = buf.ctypes.data_as(C.POINTER(C.c_uint8))
    for i in range(0, values.size, 128):
        blk = values[i:i + 128]
        rc = plain.utl_pack_u32(flag, blk.ctypes.data_as(C.POINTER(C.c_uint32)), blk.size, pu8, buf.size,
                                C.byref(n))
        assert rc == 0, rc


def U_unpack_host(packed, block_off, n, L):
    out = np.empty(128, dtype=np.uint32)
    cnt, ovf = C.c_int(0), C.c_int(0)
    cons = C.c_size_t(0)
    po = out.ctypes.data_as(C.POINTER(C.c_uint32))
    for b in range(block_off.size - 1):
        a, e = int(block_off[b]), int(block_off[b + 1])
        blk = packed[a:e]
        rc = L.utl_unpack_u32(blk.ctypes.data_as(C.POINTER(C.c_uint8)), blk.size, po, C.byref(cnt), C.byref(cons),
                              C.byref(ovf))
        assert rc == 0, rc


def U_get_host(packed, block_off, positions, L):
    v, ovf = C.c_uint32(0), C.c_int(0)
    for p in positions:
        b = int(p) // 128
        a, e = int(block_off[b]), int(block_off[b + 1])
        blk = packed[a:e]
        rc = L.utl_get_u32(int(p) % 128, blk.ctypes.data_as(C.POINTER(C.c_uint8)), blk.size, C.byref(v), C.byref(ovf))
        assert rc == 0, rc


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c3", choices=sorted(WORKLOADS))
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-plain", action="store_true", help="skip the per-call drop-in sample")
    ap.add_argument("--no-index", action="store_true", help="skip timing the stream indexer")
    ap.add_argument("--no-get", action="store_true", help="skip timing the batched Get")
    ap.add_argument("--log2n", type=int, default=28, help="values per GPU of the c3 workloads (2^log2n)")
    ap.add_argument("--knob", action="append", default=[], help="kernel knob id=value (see utl_set_knob)")
    ap.add_argument("--serve-requests", type=int, default=10000, help="c5: requests per offered rate")
    ap.add_argument("--serve-slots", type=int, default=3, help="c5: batches in flight (CUDA streams)")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "c5":
        return run_serving(args)

    import torch
    import torch.distributed as dist

    import utlpfor_b200 as U
    from utlpfor_b200._lib import load

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=dev)

    wl = WORKLOADS[args.workload]
    flag, is64 = wl["flag"], wl["is64"]
    esz = 8 if is64 else 4
    L = load()
    values, vo = make_workload(torch, args.workload, rank, dev, args.log2n)
    n = int(vo[-1])
    codec = U.BatchCodec(vo, flag=flag, is64=is64, device=dev)  # applies the tuned knobs of this GPU
    for kv in args.knob:  # explicit knobs override them
        k, v = kv.split("=")
        assert L.utl_set_knob(int(k), int(v)) == 0, kv
    out = torch.empty_like(values)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize()

    # correctness of the timed path: one checked round trip
    codec.pack(values)
    codec.unpack(out)
    torch.cuda.synchronize()
    assert codec.error_bits() == 0, "device reported errors"
    assert torch.equal(out, values), "round trip mismatch"
    packed_len = codec.packed_len

    for _ in range(args.warmup):
        codec.pack(values)
        codec.unpack(out)
    barrier()
    sampler = ClockSampler(gpu_smi_id(torch, local))
    sampler.start()
    time.sleep(0.3)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True),
           torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    launches0 = L.utl_launch_count()
    barrier()
    t_all0 = torch.cuda.Event(enable_timing=True)
    t_all1 = torch.cuda.Event(enable_timing=True)
    t_all0.record()
    for e0, e1, e2 in ev:
        e0.record()
        codec.pack(values)
        e1.record()
        codec.unpack(out)
        e2.record()
    t_all1.record()
    barrier()
    launches = L.utl_launch_count() - launches0
    clocks = sampler.stop()
    total_ms = t_all0.elapsed_time(t_all1)
    pack_ms = sum(a.elapsed_time(b) for a, b, _ in ev) / args.steps
    unpack_ms = sum(b.elapsed_time(c) for _, b, c in ev) / args.steps
    step_ms = total_ms / args.steps
    if world > 1:
        from utlpfor_b200.dist import max_over_ranks
        step_ms, pack_ms, unpack_ms = max_over_ranks([step_ms, pack_ms, unpack_ms])
    assert torch.equal(out, values)

    value_bytes = n * esz
    value = world * 2 * value_bytes / (step_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak()
    pack_bytes = value_bytes + packed_len
    unpack_bytes = packed_len + value_bytes
    pack_gbs = pack_bytes / (pack_ms * 1e-3) / 1e9
    unpack_gbs = unpack_bytes / (unpack_ms * 1e-3) / 1e9
    traffic = profiled_traffic()
    dom = "pack" if pack_ms >= unpack_ms else "unpack"
    dom_achieved = pack_gbs if dom == "pack" else unpack_gbs
    pack_names = {0: "pack_quad_kernel", 1: "pack_lane_kernel", 2: "pack_pair_kernel"}
    if dom == "pack":
        kname = ("pack_kernel" if L.utl_get_knob(2) == 0 else "pack_lane_kernel") if is64 else \
            pack_names.get(L.utl_get_knob(2), "pack_lane_kernel")
    elif is64:
        s64 = L.utl_get_knob(8)
        kname = "unpack_kernel" if s64 == 0 else "unpack_oct64_tma_kernel" if s64 in (1, 2) else "unpack_quad_pipe_kernel"
    else:
        s32 = L.utl_get_knob(0)
        # schedule 8: one kernel, the thread-per-block path on batches of small blocks (the exception-heavy one)
        kname = ("unpack_auto_kernel" if s32 == 8 else "unpack_lane_kernel" if s32 in (9, 10)
                 else "unpack_quad_pipe_kernel" if s32 in (1, 2, 3) else "unpack_quad_kernel" if s32 == 0
                 else "unpack_quad_tma_kernel")
    dom_traffic = traffic.get(kname + ("_u64" if is64 else ""))  # per-value DRAM bytes of that kernel on that width
    roofline = {"bound": "hbm", "achieved": dom_achieved, "peak": peak, "unit": "GB/s",
                "frac": dom_achieved / peak, "traffic": (dom_traffic * n) if dom_traffic else None,
                "kernel": kname, "peak_source": peak_kind + " (MEASURED_PEAKS.json hbm_gbs)"
                if peak_kind == "measured" else "fallback 6650 GB/s",
                "algorithmic_bytes": pack_bytes if dom == "pack" else unpack_bytes}

    # end to end through the host-buffer C ABI, pinned host memory
    e2e = None
    if not args.no_e2e:
        h_vals = torch.empty(n * esz, dtype=torch.uint8, pin_memory=True)
        h_vals.copy_(values.view(torch.uint8))
        h_out = torch.empty(n * esz, dtype=torch.uint8, pin_memory=True)
        h_packed = torch.empty(packed_len + 4096, dtype=torch.uint8, pin_memory=True)
        nb = codec.n_blocks
        h_bo = torch.zeros(nb + 1, dtype=torch.int64, pin_memory=True).numpy().view(np.uint64)
        h_vo = np.ascontiguousarray(vo, dtype=np.uint64)
        ns = len(vo) - 1
        olen = C.c_size_t(0)
        pk = L.utl_pack_streams_u64 if is64 else L.utl_pack_streams_u32
        up = L.utl_unpack_streams_u64 if is64 else L.utl_unpack_streams_u32
        P64 = C.POINTER(C.c_uint64)

        def e2e_step():
            rc = pk(flag, C.c_void_p(h_vals.data_ptr()), h_vo.ctypes.data_as(P64), ns, C.c_void_p(h_packed.data_ptr()),
                    h_packed.numel(), h_bo.ctypes.data_as(P64), None, C.byref(olen))
            assert rc == 0, rc
            rc = up(C.c_void_p(h_packed.data_ptr()), olen.value, h_bo.ctypes.data_as(P64), h_vo.ctypes.data_as(P64), ns,
                    C.c_void_p(h_out.data_ptr()))
            assert rc == 0, rc

        e2e_step()
        assert torch.equal(h_out, h_vals), "e2e round trip mismatch"
        e_steps = max(3, min(args.steps, 5))
        barrier()
        t0 = time.perf_counter()
        for _ in range(e_steps):
            e2e_step()
        e2e_s = (time.perf_counter() - t0) / e_steps
        if world > 1:
            from utlpfor_b200.dist import max_over_ranks
            e2e_s = max_over_ranks([e2e_s])[0]
        meta = 8 * (ns + 1)
        h2d = value_bytes + meta + packed_len + 8 * (nb + 1) + meta
        d2h = 8 * (nb + 1) + packed_len + value_bytes + 8
        e2e = {"value": world * 2 * value_bytes / e2e_s / 1e9, "unit": "GB/s", "h2d_bytes_per_step": h2d,
               "d2h_bytes_per_step": d2h, "ms_per_step": e2e_s * 1e3,
               "timing": "host wall clock around synchronous C-ABI calls (pinned host buffers)"}

    # the stream indexer over the packed result (outside the timed region):
    # block offsets recovered from the bytes alone, checked against the pack's
    index = None
    if rank == 0 and not args.no_index:
        pk_t = codec.packed[:packed_len]
        bo_t = torch.empty(codec.n_blocks + 1, dtype=torch.int64, device=dev)
        nbv = C.c_int64(0)
        sp = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        rc = L.utl_index_stream(C.c_void_p(pk_t.data_ptr()), packed_len, C.c_void_p(bo_t.data_ptr()), codec.n_blocks,
                                C.byref(nbv), sp)
        assert rc == 0 and nbv.value == codec.n_blocks, (rc, nbv.value)
        assert torch.equal(bo_t, codec.block_off), "indexer offsets differ from the pack's"
        reps = 5
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(reps):
            L.utl_index_stream(C.c_void_p(pk_t.data_ptr()), packed_len, C.c_void_p(bo_t.data_ptr()), codec.n_blocks,
                               C.byref(nbv), sp)
        ims = (time.perf_counter() - t0) / reps * 1e3
        index = {"ms": ims, "packed_GBps": packed_len / (ims * 1e-3) / 1e9, "blocks": codec.n_blocks,
                 "timing": "host wall clock around the synchronous call"}

    # GetUint32 / GetUint64 over the packed result: 2^20 queries, a stream
    # drawn uniformly among the non-empty ones and a position uniformly in
    # it, one batched launch; checked against the values, timed with CUDA
    # events (reported as queries/s: a query reads a few bytes of a block)
    get = None
    if rank == 0 and not args.no_get:
        nq = 1 << 20
        gq = torch.Generator(device=dev)
        gq.manual_seed(4321)
        starts_t = torch.from_numpy(vo[:-1].astype(np.int64)).to(dev)
        lens_t = torch.from_numpy((vo[1:] - vo[:-1]).astype(np.int64)).to(dev)
        live = torch.nonzero(lens_t > 0).flatten()
        q_s = live[torch.randint(0, live.numel(), (nq,), device=dev, generator=gq)]
        q_p = (torch.rand(nq, device=dev, generator=gq, dtype=torch.float64) * lens_t[q_s].double()).long()
        q_p = torch.minimum(q_p, lens_t[q_s] - 1)
        q_stream = q_s.to(torch.int32)
        q_out = torch.empty(nq, dtype=values.dtype, device=dev)
        codec.get(q_stream, q_p, q_out)
        assert torch.equal(q_out, values[starts_t[q_s] + q_p]), "Get results differ from the values"
        g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        reps = 10
        torch.cuda.synchronize()
        g0.record()
        for _ in range(reps):
            codec.get(q_stream, q_p, q_out)
        g1.record()
        torch.cuda.synchronize()
        gms = g0.elapsed_time(g1) / reps
        get = {"queries": nq, "ms": gms, "queries_per_s": nq / (gms * 1e-3),
               "queries_drawn": "stream uniform among non-empty streams, position uniform in it",
               "timing": "CUDA events, one batched launch per call"}

    # the plain per-call drop-in on the same data: one utl_pack_u32 and one
    # utl_unpack_u32 call per 128-value block (host buffers), the way a Go
    # caller would use the per-call API block after block; a bounded sample
    plain = None
    if rank == 0 and not args.no_plain and not is64:
        nblk = min(codec.n_blocks, 2000)
        hv = values[:nblk * 128].cpu().numpy().view(np.uint32).copy()
        hv_n = min(hv.size, n)
        buf = np.zeros(L.utl_max_block_length32(flag), dtype=np.uint8)
        outb = np.zeros(128, dtype=np.uint32)
        olen, cnt, cons, ovf = C.c_size_t(0), C.c_int(0), C.c_size_t(0), C.c_int(0)
        pu8 = buf.ctypes.data_as(C.POINTER(C.c_uint8))
        pout = outb.ctypes.data_as(C.POINTER(C.c_uint32))
        lat_p, lat_u = [], []
        for rep in range(2):  # the first pass warms the per-thread context
            lat_p.clear()
            lat_u.clear()
            for i in range(0, hv_n, 128):
                blk = hv[i:i + 128]
                t0 = time.perf_counter()
                rc = L.utl_pack_u32(flag, blk.ctypes.data_as(C.POINTER(C.c_uint32)), blk.size, pu8, buf.size,
                                    C.byref(olen))
                t1 = time.perf_counter()
                assert rc == 0, rc
                rc = L.utl_unpack_u32(pu8, olen.value, pout, C.byref(cnt), C.byref(cons), C.byref(ovf))
                t2 = time.perf_counter()
                assert rc == 0 and cnt.value == blk.size and np.array_equal(outb[:blk.size], blk)
                lat_p.append(t1 - t0)
                lat_u.append(t2 - t1)
        tot = sum(lat_p) + sum(lat_u)
        # the same calls from 8 host threads through a pool of 8 contexts
        # (raw C-ABI calls on buffers prepared per thread; ctypes releases
        # the interpreter lock for the duration of each call)
        pool = C.c_void_p()
        assert L.utl_pool_new(8, C.byref(pool)) == 0
        n_thr = 8
        per = max(1, (hv_n // 128) // n_thr)

        def pool_worker(k, reps):
            pb = np.zeros(L.utl_max_block_length32(flag), dtype=np.uint8)
            po = np.zeros(128, dtype=np.uint32)
            n_, c_, cs_, ov_ = C.c_size_t(0), C.c_int(0), C.c_size_t(0), C.c_int(0)
            pbp = pb.ctypes.data_as(C.POINTER(C.c_uint8))
            pop = po.ctypes.data_as(C.POINTER(C.c_uint32))
            blocks = [hv[128 * i:128 * i + 128] for i in range(k * per, (k + 1) * per)]
            ptrs = [bl.ctypes.data_as(C.POINTER(C.c_uint32)) for bl in blocks]
            for _ in range(reps):
                for bl, bp in zip(blocks, ptrs):
                    assert L.utl_pool_pack_u32(pool, flag, bp, bl.size, pbp, pb.size, C.byref(n_)) == 0
                    assert L.utl_pool_unpack_u32(pool, pbp, n_.value, pop, C.byref(c_), C.byref(cs_),
                                                 C.byref(ov_)) == 0

        pool_worker(0, 1)  # warm the contexts
        ths = [threading.Thread(target=pool_worker, args=(k, 1)) for k in range(n_thr)]
        tp0 = time.perf_counter()
        for t_ in ths:
            t_.start()
        for t_ in ths:
            t_.join()
        pool_s = time.perf_counter() - tp0
        L.utl_pool_free(pool)
        plain = {"GBps": 2 * 4 * hv_n / tot / 1e9, "unit": "GB/s (round-trip uncompressed)", "blocks": hv_n // 128,
                 "pooled_8_threads_GBps": 2 * 4 * 128 * per * n_thr / pool_s / 1e9,
                 "pack_us_p50": 1e6 * float(np.median(lat_p)), "pack_us_p99": 1e6 * float(np.percentile(lat_p, 99)),
                 "unpack_us_p50": 1e6 * float(np.median(lat_u)),
                 "unpack_us_p99": 1e6 * float(np.percentile(lat_u, 99)),
                 "calls": "utl_pack_u32 + utl_unpack_u32 per 128-value block, host buffers, one thread",
                 "sample": "the workload's first %d blocks" % (hv_n // 128)}

    cpu = None
    if rank == 0 and not args.no_cpu:
        # the same values, copied to the host, through the CPU restatement
        # of the reference's vectorized pipelines on every host thread
        threads = host_threads()
        host_vals = values.cpu().numpy().view(np.uint64 if is64 else np.uint32)
        times = cpu_round_trip(host_vals, vo, flag, threads, min_seconds=10.0, max_rounds=10)
        del host_vals
        t = sum(times) / len(times)
        cpu = {"value": 2 * value_bytes / t / 1e9, "unit": "GB/s", "cores": threads, "kind": "port",
               "impl": cpu_kind(),
               "sample": "the whole workload (%d values, %d MiB), %d rounds" % (n, value_bytes >> 20, len(times))}

    if rank == 0:
        line = {
            "metric": "round-trip uncompressed GB/s (batched PackUint32 + UnpackUint32)",
            "value": value, "unit": "GB/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64" if is64 else "u32", "data": "synthetic (seeded on device)",
            "config": workload_config(args.workload, n, codec.n_blocks, world),
            "packed": {"bytes_per_gpu": packed_len, "bytes_per_value": packed_len / n},
            "pack": {"ms": pack_ms, "uncompressed_GBps": value_bytes / (pack_ms * 1e-3) / 1e9,
                     "hbm_GBps": pack_gbs, "hbm_frac": pack_gbs / peak},
            "unpack": {"ms": unpack_ms, "uncompressed_GBps": value_bytes / (unpack_ms * 1e-3) / 1e9,
                       "hbm_GBps": unpack_gbs, "hbm_frac": unpack_gbs / peak},
            "roofline": roofline,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "plain_per_call": plain,
            "batched_e2e_over_plain": (e2e["value"] / plain["GBps"]) if (e2e and plain) else None,
            "index": index,
            "get": get,
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
