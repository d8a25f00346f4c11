"""Continuous-batching codec server over HBM-resident packed streams.

Requests -- compress (values -> a resident packed stream), decompress (a
resident stream -> values) and get (positions of a resident stream ->
values) -- arrive on any thread through submit_*() and return futures.
One scheduler thread batches them: whenever one of its CUDA stream slots
is free it forms a batch from the oldest waiting requests of one kind,
admitting requests in arrival order while the device-memory budget holds
(resident streams + buffers of batches in flight), and launches the batch
with the batched kernels (copies in, one pack/unpack/get launch, copies
out) on that slot's stream.  Requests that arrive while batches are on the
GPU join the next batch as slots and memory free up, and batches on
different slots overlap on the device.  Completed batches are retired by
polling their events; each request records its submit-to-result latency.

A packed stream lives in HBM as its bytes and its block offsets (relative
to its first byte); its bytes are exactly those of PackUint32/PackUint64
with Append, block after block (pack.go:76-97).
"""
import ctypes as C
import queue
import threading
import time
from concurrent.futures import Future
from dataclasses import dataclass, field

import numpy as np

from ._lib import load


def _t():
    import torch
    return torch


def _p(t):
    return C.c_void_p(t.data_ptr()) if t is not None else C.c_void_p(0)


class ServerError(RuntimeError):
    pass


@dataclass
class Handle:
    """A packed stream resident in HBM."""
    id: int
    n_values: int
    is64: bool
    flag: int
    packed: object      # uint8 device tensor, exactly the stream's bytes
    block_off: object   # int64 device tensor, n_blocks + 1, starting at 0
    released: bool = False
    nbytes: int = 0     # device bytes held (packed + block offsets)

    def __post_init__(self):
        self.n_blocks = self.block_off.numel() - 1
        self.nbytes = self.packed.numel() + 8 * self.block_off.numel()


@dataclass
class _Req:
    kind: str
    fut: Future
    t_submit: float
    values: object = None       # compress: numpy array
    flag: int = 0
    handle: Handle = None       # decompress / get
    positions: object = None    # get: numpy int64
    cost: int = 0               # device bytes the request needs while in flight
    bytes_done: int = 0         # uncompressed bytes it moves


@dataclass
class _Batch:
    kind: str
    reqs: list
    slot: int
    event: object
    cost: int
    keep: list = field(default_factory=list)   # device/pinned tensors alive until retired
    finish: object = None                       # callable run at retirement


def _req_values(r):
    if r.kind == "compress":
        return r.values.size
    if r.kind == "decompress":
        return r.handle.n_values
    return r.positions.size


def _req_group(r):
    """Requests of one batch share the integer width (and, to pack, nothing
    else: flags may differ inside a compress batch)."""
    if r.kind == "compress":
        return r.values.dtype == np.uint64
    return r.handle.is64


def select_batch(queue_, budget_left, max_reqs, max_vals):
    """Continuous-batching admission: the longest prefix, in arrival order,
    of the requests of the oldest one's width whose device bytes fit the
    budget left and whose sizes fit the batch limits.  The first request is
    taken alone if it exceeds max_vals by itself.  Returns [] when even the
    oldest request does not fit the memory left."""
    if not queue_:
        return []
    g = _req_group(queue_[0])
    take, cost, vals = [], 0, 0
    for r in queue_:
        if _req_group(r) != g:
            continue
        n = _req_values(r)
        if take and (len(take) >= max_reqs or vals + n > max_vals):
            break
        if cost + r.cost > budget_left:
            break
        take.append(r)
        cost += r.cost
        vals += n
    return take


class CodecServer:
    def __init__(self, budget_bytes=64 << 30, slots=3, max_batch_requests=256, max_batch_values=1 << 25,
                 device="cuda"):
        torch = _t()
        self.L = load()
        dev = torch.device(device)
        if dev.type != "cuda":
            raise ValueError("the server runs on a CUDA device")
        self.dev = torch.device("cuda", dev.index if dev.index is not None else torch.cuda.current_device())
        self.budget = int(budget_bytes)
        self.max_reqs = max_batch_requests
        self.max_vals = max_batch_values
        self.streams = [torch.cuda.Stream(device=self.dev) for _ in range(slots)]
        self.slot_busy = [None] * slots
        self.inbox = queue.Queue()
        self.pending = {"compress": [], "decompress": [], "get": []}
        self.resident = 0
        self.in_flight = 0
        self.latencies = {"compress": [], "decompress": [], "get": []}
        self.bytes_done = 0
        self.batches = 0
        self.max_overlap = 0
        self.admitted = 0
        self.rejected = 0
        self._next_id = 0
        self._submitted = 0
        self._completed = 0
        self._lock = threading.Lock()
        self._stop = False
        self._dead = None
        self._t0 = time.perf_counter()
        self._thread = threading.Thread(target=self._run, daemon=True)
        self._thread.start()

    # ------------------------------------------------------------ client API
    def _submit(self, r):
        if self._dead is not None:
            raise ServerError("scheduler stopped: %r" % (self._dead,))
        with self._lock:
            self._submitted += 1
        r.fut.add_done_callback(self._done)
        if r.handle is not None and r.handle.released:
            r.fut.set_exception(ServerError("stream was released"))
        elif r.cost > self.budget:
            self.rejected += 1
            r.fut.set_exception(ServerError("request needs %d bytes, over the %d-byte budget" % (r.cost, self.budget)))
        else:
            self.inbox.put(r)
        return r.fut

    def submit_compress(self, values, flag=0):
        v = np.ascontiguousarray(values)
        if v.dtype not in (np.uint32, np.uint64):
            raise TypeError("values must be uint32 or uint64")
        maxb = (self.L.utl_max_block_length64 if v.dtype == np.uint64 else self.L.utl_max_block_length32)(flag)
        nb = (v.size + 127) // 128
        r = _Req("compress", Future(), time.perf_counter(), values=v, flag=flag & 0xFF,
                 cost=v.nbytes + nb * maxb + 16 * (nb + 2), bytes_done=v.nbytes)
        return self._submit(r)

    def submit_decompress(self, handle):
        esz = 8 if handle.is64 else 4
        r = _Req("decompress", Future(), time.perf_counter(), handle=handle,
                 cost=handle.nbytes + handle.n_values * esz + 64, bytes_done=handle.n_values * esz)
        return self._submit(r)

    def submit_get(self, handle, positions):
        pos = np.ascontiguousarray(positions, dtype=np.int64)
        esz = 8 if handle.is64 else 4
        r = _Req("get", Future(), time.perf_counter(), handle=handle, positions=pos,
                 cost=handle.nbytes + pos.size * (16 + esz) + 64, bytes_done=pos.size * esz)
        return self._submit(r)

    def release(self, handle):
        """Free a resident stream (its memory returns to the budget)."""
        with self._lock:
            if not handle.released:
                handle.released = True
                self.resident -= handle.nbytes
                handle.packed = None
                handle.block_off = None

    def _done(self, _fut):
        with self._lock:
            self._completed += 1

    def drain(self, timeout=None):
        """Wait until every request submitted so far has its result."""
        t_end = None if timeout is None else time.perf_counter() + timeout
        while self._completed < self._submitted:
            if t_end is not None and time.perf_counter() > t_end:
                raise TimeoutError("requests still pending")
            time.sleep(50e-6)

    def close(self):
        self._stop = True
        self._thread.join()

    def reset_stats(self):
        for v in self.latencies.values():
            v.clear()
        self.bytes_done = 0
        self.batches = self.admitted = self.rejected = self.max_overlap = 0
        self._t0 = time.perf_counter()

    def stats(self):
        out = {}
        for k, v in self.latencies.items():
            if v:
                a = np.array(v) * 1e3
                out[k] = {"n": len(v), "p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99))}
        allv = [x for v in self.latencies.values() for x in v]
        if allv:
            a = np.array(allv) * 1e3
            out["all"] = {"n": len(allv), "p50_ms": float(np.percentile(a, 50)), "p99_ms": float(np.percentile(a, 99))}
        wall = time.perf_counter() - self._t0
        out["uncompressed_bytes"] = self.bytes_done
        out["uncompressed_GBps"] = self.bytes_done / wall / 1e9 if wall > 0 else 0.0
        out["batches"] = self.batches
        out["admitted"] = self.admitted
        out["rejected"] = self.rejected
        out["queued"] = sum(len(v) for v in self.pending.values()) + self.inbox.qsize()
        out["max_batches_in_flight"] = self.max_overlap
        out["resident_bytes"] = self.resident
        return out

    # ------------------------------------------------------------ scheduler
    def _run(self):
        try:
            self._loop()
        except BaseException as e:  # noqa: BLE001 - the thread must not die silently
            self._dead = e
            for q in self.pending.values():
                for r in q:
                    if not r.fut.done():
                        r.fut.set_exception(ServerError("scheduler stopped: %r" % (e,)))
            raise

    def _loop(self):
        torch = _t()
        torch.cuda.set_device(self.dev)
        while True:
            drained = False
            try:
                while True:
                    r = self.inbox.get_nowait()
                    self.pending[r.kind].append(r)
                    drained = True
            except queue.Empty:
                pass
            try:
                retired = self._retire()
                launched = self._launch_ready()
            except Exception as e:  # noqa: BLE001 - keep serving; fail what was waiting
                retired = launched = True
                for q in self.pending.values():
                    for r in q:
                        if not r.fut.done():
                            r.fut.set_exception(ServerError("scheduler error: %r" % (e,)))
                    q.clear()
            if self._stop and not any(self.pending.values()) and not any(self.slot_busy) and self.inbox.empty():
                return
            if not (drained or retired or launched):
                time.sleep(20e-6)

    def _retire(self):
        done = False
        for s, b in enumerate(self.slot_busy):
            if b is not None and b.event.query():
                try:
                    b.finish()
                except Exception as e:  # noqa: BLE001 - surfaced on the futures
                    for r in b.reqs:
                        if not r.fut.done():
                            r.fut.set_exception(e)
                now = time.perf_counter()
                for r in b.reqs:
                    self.latencies[r.kind].append(now - r.t_submit)
                    self.bytes_done += r.bytes_done
                self.in_flight -= b.cost
                self.slot_busy[s] = None
                done = True
        return done

    def _launch_ready(self):
        launched = False
        while True:
            free = [s for s, b in enumerate(self.slot_busy) if b is None]
            if not free:
                return launched
            kinds = [k for k, v in self.pending.items() if v]
            if not kinds:
                return launched
            # the kind whose oldest request has waited longest goes first
            kind = min(kinds, key=lambda k: self.pending[k][0].t_submit)
            q = self.pending[kind]
            for r in q:
                if kind != "compress" and r.handle.released and not r.fut.done():
                    r.fut.set_exception(ServerError("stream was released"))
            q = [r for r in q if not r.fut.done()]
            self.pending[kind] = q
            if not q:
                continue
            take = select_batch(q, self.budget - self.resident - self.in_flight, self.max_reqs, self.max_vals)
            if not take:
                if not any(self.slot_busy):
                    # nothing in flight will free memory: the oldest request cannot be served
                    r = q.pop(0)
                    self.rejected += 1
                    r.fut.set_exception(ServerError(
                        "request needs %d bytes; budget %d, resident streams hold %d" % (r.cost, self.budget,
                                                                                          self.resident)))
                    continue
                return launched
            ids = set(id(r) for r in take)
            self.pending[kind] = [r for r in q if id(r) not in ids]
            cost = sum(r.cost for r in take)
            slot = free[0]
            self.in_flight += cost
            try:
                b = self._launch(kind, take, slot, cost)
            except Exception as e:  # noqa: BLE001 - a launch that fails fails its requests
                self.in_flight -= cost
                for r in take:
                    r.fut.set_exception(e)
                continue
            self.slot_busy[slot] = b
            self.batches += 1
            self.admitted += len(take)
            self.max_overlap = max(self.max_overlap, sum(x is not None for x in self.slot_busy))
            launched = True

    def _check(self, rc):
        if rc != 0:
            raise ServerError("codec call failed with status %d" % rc)

    def _launch(self, kind, reqs, slot, cost):
        torch = _t()
        st = self.streams[slot]
        with torch.cuda.stream(st):
            if kind == "compress":
                b = self._launch_compress(reqs, st)
            elif kind == "decompress":
                b = self._launch_decompress(reqs, st)
            else:
                b = self._launch_get(reqs, st)
            ev = torch.cuda.Event()
            ev.record(st)
        b.slot, b.event, b.cost, b.kind, b.reqs = slot, ev, cost, kind, reqs
        return b

    # each request kind: copies in, one batched launch, copies out
    def _launch_compress(self, reqs, st):
        torch = _t()
        L = self.L
        groups = {}
        for r in reqs:
            groups.setdefault((r.values.dtype == np.uint64, r.flag), []).append(r)
        keep, finals = [], []
        for (is64, flag), rs in groups.items():
            esz = 8 if is64 else 4
            lens = np.array([r.values.size for r in rs], dtype=np.uint64)
            vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
            nb = int(L.utl_count_blocks(vo.ctypes.data_as(C.POINTER(C.c_uint64)), len(rs)))
            n = int(vo[-1])
            h_vals = torch.empty(max(n * esz, 1), dtype=torch.uint8, pin_memory=True)
            hv = h_vals.numpy()
            pos = 0
            for r in rs:
                hv[pos:pos + r.values.nbytes] = r.values.view(np.uint8)
                pos += r.values.nbytes
            d_vals = h_vals.to(self.dev, non_blocking=True)
            d_vo = torch.from_numpy(vo.view(np.int64)).pin_memory().to(self.dev, non_blocking=True)
            d_bs = torch.empty(len(rs) + 1, dtype=torch.int64, device=self.dev)
            s_ptr = C.c_void_p(st.cuda_stream)
            self._check(L.utl_batch_plan(_p(d_vo), len(rs), _p(d_bs), s_ptr))
            maxb = (L.utl_max_block_length64 if is64 else L.utl_max_block_length32)(flag)
            out = torch.empty(max(nb * maxb, 16), dtype=torch.uint8, device=self.dev)
            bo = torch.empty(nb + 1, dtype=torch.int64, device=self.dev)
            sbo = torch.empty(len(rs) + 1, dtype=torch.int64, device=self.dev)
            sb = L.utl_pack_scratch_bytes(nb)
            scratch = torch.empty(max(sb, 16), dtype=torch.uint8, device=self.dev)
            err = torch.zeros(1, dtype=torch.int32, device=self.dev)
            fn = L.utl_pack_batch_u64 if is64 else L.utl_pack_batch_u32
            self._check(fn(flag, _p(d_vals), _p(d_vo), _p(d_bs), len(rs), nb, _p(out), out.numel(), _p(bo), _p(sbo),
                           _p(scratch), sb, _p(err), s_ptr))
            h_sbo = torch.empty(len(rs) + 1, dtype=torch.int64, pin_memory=True)
            h_sbo.copy_(sbo, non_blocking=True)
            h_bs = torch.empty(len(rs) + 1, dtype=torch.int64, pin_memory=True)
            h_bs.copy_(d_bs, non_blocking=True)
            h_err = torch.empty(1, dtype=torch.int32, pin_memory=True)
            h_err.copy_(err, non_blocking=True)
            keep += [h_vals, d_vals, d_vo, d_bs, out, bo, sbo, scratch, err, h_sbo, h_bs, h_err]
            finals.append((rs, is64, flag, out, bo, h_sbo, h_bs, h_err))

        def finish():
            with torch.cuda.stream(st):
                for rs, is64, flag, out, bo, h_sbo, h_bs, h_err in finals:
                    if int(h_err[0]):
                        raise ServerError("pack reported error bits %#x" % int(h_err[0]))
                    so, bs = h_sbo.numpy(), h_bs.numpy()
                    for i, r in enumerate(rs):
                        a, e = int(so[i]), int(so[i + 1])
                        packed = out[a:e].clone()
                        boff = bo[int(bs[i]):int(bs[i + 1]) + 1] - a
                        with self._lock:
                            self._next_id += 1
                            h = Handle(self._next_id, r.values.size, is64, flag, packed, boff.clone())
                            self.resident += h.nbytes
                        r.fut.set_result(h)
                st.synchronize()
        return _Batch("compress", reqs, -1, None, 0, keep, finish)

    def _gather(self, reqs):
        """One packed buffer and block-offset table over the requests' streams."""
        torch = _t()
        packed = torch.cat([r.handle.packed for r in reqs]) if len(reqs) > 1 else reqs[0].handle.packed
        parts, base = [], 0
        for r in reqs:
            parts.append(r.handle.block_off[:-1] + base)
            base += r.handle.packed.numel()
        parts.append(torch.tensor([base], dtype=torch.int64, device=self.dev))
        bo = torch.cat(parts)
        lens = np.array([r.handle.n_values for r in reqs], dtype=np.uint64)
        vo = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint64)
        return packed, bo, vo

    def _launch_decompress(self, reqs, st):
        torch = _t()
        L = self.L
        is64 = reqs[0].handle.is64
        packed, bo, vo = self._gather(reqs)
        n = int(vo[-1])
        d_vo = torch.from_numpy(vo.view(np.int64)).pin_memory().to(self.dev, non_blocking=True)
        d_bs = torch.empty(len(reqs) + 1, dtype=torch.int64, device=self.dev)
        s_ptr = C.c_void_p(st.cuda_stream)
        self._check(L.utl_batch_plan(_p(d_vo), len(reqs), _p(d_bs), s_ptr))
        out = torch.empty(max(n, 1), dtype=torch.int64 if is64 else torch.int32, device=self.dev)
        err = torch.zeros(1, dtype=torch.int32, device=self.dev)
        fn = L.utl_unpack_batch_u64 if is64 else L.utl_unpack_batch_u32
        self._check(fn(_p(packed), packed.numel(), _p(bo), _p(d_vo), _p(d_bs), len(reqs), bo.numel() - 1, _p(out),
                       None, _p(err), s_ptr))
        h_out = torch.empty(max(n, 1), dtype=out.dtype, pin_memory=True)
        h_out.copy_(out, non_blocking=True)
        h_err = torch.empty(1, dtype=torch.int32, pin_memory=True)
        h_err.copy_(err, non_blocking=True)

        def finish():
            if int(h_err[0]):
                raise ServerError("unpack reported error bits %#x" % int(h_err[0]))
            # results are views of the pinned output (kept alive by the arrays)
            arr = h_out.numpy().view(np.uint64 if is64 else np.uint32)
            for i, r in enumerate(reqs):
                r.fut.set_result(arr[int(vo[i]):int(vo[i + 1])])
        return _Batch("decompress", reqs, -1, None, 0, [packed, bo, d_vo, d_bs, out, err, h_out, h_err], finish)

    def _launch_get(self, reqs, st):
        torch = _t()
        L = self.L
        is64 = reqs[0].handle.is64
        packed, bo, vo = self._gather(reqs)
        qs = np.concatenate([np.full(r.positions.size, i, dtype=np.uint32) for i, r in enumerate(reqs)])
        qp = np.concatenate([r.positions for r in reqs]).astype(np.uint64)
        qo = np.concatenate([[0], np.cumsum([r.positions.size for r in reqs])]).astype(np.int64)
        d_vo = torch.from_numpy(vo.view(np.int64)).pin_memory().to(self.dev, non_blocking=True)
        d_qs = torch.from_numpy(qs.view(np.int32)).pin_memory().to(self.dev, non_blocking=True)
        d_qp = torch.from_numpy(qp.view(np.int64)).pin_memory().to(self.dev, non_blocking=True)
        d_bs = torch.empty(len(reqs) + 1, dtype=torch.int64, device=self.dev)
        s_ptr = C.c_void_p(st.cuda_stream)
        self._check(L.utl_batch_plan(_p(d_vo), len(reqs), _p(d_bs), s_ptr))
        nq = qs.size
        out = torch.empty(max(nq, 1), dtype=torch.int64 if is64 else torch.int32, device=self.dev)
        status = torch.empty(max(nq, 1), dtype=torch.int32, device=self.dev)
        fn = L.utl_get_batch_u64 if is64 else L.utl_get_batch_u32
        self._check(fn(_p(packed), packed.numel(), _p(bo), _p(d_vo), _p(d_bs), len(reqs), _p(d_qs), _p(d_qp), nq,
                       _p(out), _p(status), None, s_ptr))
        h_out = torch.empty(max(nq, 1), dtype=out.dtype, pin_memory=True)
        h_out.copy_(out, non_blocking=True)
        h_st = torch.empty(max(nq, 1), dtype=torch.int32, pin_memory=True)
        h_st.copy_(status, non_blocking=True)

        def finish():
            from . import _raise
            arr = h_out.numpy().view(np.uint64 if is64 else np.uint32)
            stv = h_st.numpy()
            for i, r in enumerate(reqs):
                a, e = int(qo[i]), int(qo[i + 1])
                bad = np.nonzero(stv[a:e] & 0xFF)[0]
                if bad.size:
                    try:
                        _raise(int(stv[a + bad[0]] & 0xFF), int(stv[a + bad[0]] >> 8))
                    except Exception as ex:  # noqa: BLE001
                        r.fut.set_exception(ex)
                    continue
                r.fut.set_result(arr[a:e].copy())
        return _Batch("get", reqs, -1, None, 0, [packed, bo, d_vo, d_qs, d_qp, d_bs, out, status, h_out, h_st],
                      finish)
