"""Continuous-batching MSM server over resident base tables.

The base sets (for example an SRS-like table of G1 points and one of G2
points) stay resident on the device.  Clients submit scalar vectors; request
i of group g asks for  sum_j k_j * T_g[offset + j]  over a prefix (or any
slice) of the group's table.

A worker thread keeps up to ``slots`` batches in flight, each on its own CUDA
stream.  Whenever a slot is free it admits the oldest pending requests of one
group -- as many as fit the batch limits and the device-memory budget -- and
launches them as one flattened batch (``gm_batch_run``): scalars are staged
through the slot's pinned buffer, the batch runs, and the results come back
through pinned memory.  Requests that arrive while batches run wait in the
queue and are admitted as soon as a slot and memory free up, so their work
overlaps with batches already on the device.

Admission by device memory: at start the server measures the free device
memory and keeps ``budget = free - reserve``.  Every slot owns a fixed device
workspace of ``slot_bytes`` (by default twice the largest workspace of a
batch at the server's limits, and at most budget / slots), allocated once, and
runs its batches in it (``gm_batch_run_ws``): no batch takes an allocation
from the library's stream-ordered pool, whose growth under load was measured
to stall a launch for up to a second.  A batch is admitted only if its
workspace (``gm_batch_workspace_bytes``) fits a slot; a single request that
cannot fit even alone is rejected with an error.

Latency of a request = completion time - submission time (host clock); the
server records both for p50/p99.
"""
from __future__ import annotations

import collections
import threading
import time
from dataclasses import dataclass, field

import numpy as np

import gpu_msm_b200 as gm


@dataclass
class Request:
    rid: int
    group: int
    scalars: np.ndarray          # (n, limbs) uint64
    offset: int = 0
    t_submit: float = 0.0
    t_done: float = 0.0
    result: np.ndarray = None    # projective point (numpy structured, 1 element)
    error: str = None
    batch_id: int = -1
    done: threading.Event = field(default_factory=threading.Event)

    @property
    def latency(self) -> float:
        return self.t_done - self.t_submit


class _Slot:
    def __init__(self, torch, dev, max_points, limbs, max_batch):
        self.stream = torch.cuda.Stream(device=dev)
        self.h_sc = torch.empty((max_points, limbs), dtype=torch.int64, pin_memory=True)
        self.d_sc = torch.empty((max_points, limbs), dtype=torch.int64, device=dev)
        self.d_out = torch.empty(max_batch * gm.G2P_WORDS, dtype=torch.int64, device=dev)
        self.h_out = torch.empty(max_batch * gm.G2P_WORDS, dtype=torch.int64, pin_memory=True)
        self.ws = None
        self.event = None
        self.reqs = []
        self.bytes = 0
        self.group = 1


class MsmServer:
    def __init__(self, tables: dict, max_batch: int = 64, max_points: int = 1 << 22, slots: int = 2,
                 mem_reserve: int = 2 << 30, mem_budget: int = None, scalar_limbs: int = 5, slot_bytes: int = None):
        import torch
        self.torch = torch
        self.tables = tables
        self.dev = next(iter(tables.values())).device
        self.max_batch = max_batch
        self.max_points = max_points
        self.limbs = scalar_limbs
        free, _ = torch.cuda.mem_get_info(self.dev)
        self.budget = mem_budget if mem_budget is not None else max(0, free - mem_reserve)
        self.slots = [_Slot(torch, self.dev, max_points, scalar_limbs, max_batch) for _ in range(slots)]
        if slot_bytes is None:
            need = max((gm.batch_workspace_bytes(t, sz, scalar_limbs=scalar_limbs) for _, t, sz in self._limit_shapes()),
                       default=0)
            slot_bytes = min(self.budget // max(1, slots), 2 * need)
        self.slot_bytes = int(slot_bytes) // 256 * 256
        for sl in self.slots:
            sl.ws = torch.empty(max(256, self.slot_bytes), dtype=torch.uint8, device=self.dev)
        self.pending = collections.deque()
        self.cv = threading.Condition()
        self.stop_flag = False
        self.thread = None
        self.next_id = 0
        self.batches = []       # (batch id, group, n requests, points)
        self.completed = []

    # ---------------------------------------------------------------- client
    def submit(self, group: int, scalars: np.ndarray, offset: int = 0) -> Request:
        sc = np.ascontiguousarray(scalars, dtype=np.uint64)
        if sc.ndim != 2 or sc.shape[1] != self.limbs or len(sc) == 0:
            raise ValueError(f"scalars must be (n, {self.limbs}) uint64 with n > 0")
        if group not in self.tables or offset < 0 or offset + len(sc) > self.tables[group].n:
            raise ValueError("request outside the resident table")
        if len(sc) > self.max_points:
            raise ValueError("request larger than the server's max_points")
        with self.cv:
            r = Request(self.next_id, group, sc, offset, t_submit=time.perf_counter())
            self.next_id += 1
            self.pending.append(r)
            self.cv.notify()
        return r

    def start(self, warmup: bool = True):
        """Start the worker thread.  warmup: first run, on every slot at once,
        batches of each group at the server's limits (one MSM of max_points,
        and max_batch MSMs sharing max_points) with zero scalars.  Their
        workspaces and kernels are those of real batches, so the library's
        stream-ordered memory pool already holds the memory of concurrent
        batches and every kernel is loaded: no request waits for the pool to
        grow (tens of milliseconds, occasionally far more, under load) or for a
        first launch."""
        if warmup:
            self._warmup()
        self.stop_flag = False
        self.thread = threading.Thread(target=self._loop, name="msm-server", daemon=True)
        self.thread.start()
        return self

    def stop(self, drain: bool = True):
        with self.cv:
            if not drain:
                self.pending.clear()
            self.stop_flag = True
            self.cv.notify()
        if self.thread is not None:
            self.thread.join()
            self.thread = None

    # ---------------------------------------------------------------- worker
    def _limit_shapes(self):
        """(group, table, sizes) of batches at the server's limits: the
        largest requests the table allows, as many as max_points holds, and
        max_batch equal requests sharing max_points."""
        for group, table in self.tables.items():
            n = min(self.max_points, table.n)
            yield group, table, [n] * max(1, min(self.max_batch, self.max_points // n))
            per = max(1, min(n, self.max_points // self.max_batch))
            yield group, table, [per] * max(1, min(self.max_batch, self.max_points // per))

    def _warmup(self):
        torch = self.torch
        for group, table, sizes in self._limit_shapes():
            if gm.batch_workspace_bytes(table, sizes, scalar_limbs=self.limbs) > self.slot_bytes:
                continue
            words = gm.G1P_WORDS if group == 1 else gm.G2P_WORDS
            total = int(sum(sizes))
            for slot in self.slots:
                with torch.cuda.stream(slot.stream):
                    slot.d_sc[:total].zero_()
                    out = slot.d_out[:len(sizes) * words].view(len(sizes), words)
                    gm.batch_run(table, sizes, slot.d_sc[:total], out=out, stream=slot.stream, workspace=slot.ws)
            for slot in self.slots:
                slot.stream.synchronize()

    def _reap(self):
        """Complete the slots whose batch finished."""
        now_any = False
        for s in self.slots:
            if s.event is not None and s.event.query():
                t = time.perf_counter()
                host = s.h_out.numpy().view(np.uint64)
                for i, r in enumerate(s.reqs):
                    words = gm.G1P_WORDS if r.group == 1 else gm.G2P_WORDS
                    dt = gm.G1P if r.group == 1 else gm.G2P
                    r.result = np.ascontiguousarray(host[i * words:(i + 1) * words]).view(dt).reshape(1).copy()
                    r.t_done = t
                    self.completed.append(r)
                    r.done.set()
                s.event, s.reqs, s.bytes = None, [], 0
                now_any = True
        return now_any

    def _form_batch(self):
        """Oldest pending requests of one group that fit the limits and the
        memory budget; None if nothing can be admitted now."""
        if not self.pending:
            return None
        group = self.pending[0].group
        table = self.tables[group]
        take, sizes, points = [], [], 0
        for r in list(self.pending):
            if r.group != group:
                continue
            n = len(r.scalars)
            if len(take) == self.max_batch or points + n > self.max_points:
                break
            trial = sizes + [n]
            need = gm.batch_workspace_bytes(table, trial, scalar_limbs=self.limbs)
            if need > self.slot_bytes:
                if not take:
                    # cannot fit even alone in a slot's workspace
                    self.pending.remove(r)
                    r.error = "request does not fit the device-memory budget"
                    r.t_done = time.perf_counter()
                    r.done.set()
                    return None
                break
            take.append(r)
            sizes = trial
            points += n
        if not take:
            return None
        for r in take:
            self.pending.remove(r)
        return group, take, gm.batch_workspace_bytes(table, sizes, scalar_limbs=self.limbs)

    def _launch(self, slot, group, reqs, nbytes):
        torch = self.torch
        sizes = np.array([len(r.scalars) for r in reqs], dtype=np.int64)
        offs = np.array([r.offset for r in reqs], dtype=np.int64)
        total = int(sizes.sum())
        h = slot.h_sc.numpy().view(np.uint64)
        row = 0
        for r in reqs:
            h[row:row + len(r.scalars)] = r.scalars
            row += len(r.scalars)
        words = gm.G1P_WORDS if group == 1 else gm.G2P_WORDS
        with torch.cuda.stream(slot.stream):
            slot.d_sc[:total].copy_(slot.h_sc[:total], non_blocking=True)
            out = slot.d_out[:len(reqs) * words].view(len(reqs), words)
            gm.batch_run(self.tables[group], sizes, slot.d_sc[:total], base_offsets=offs, out=out,
                         stream=slot.stream, workspace=slot.ws)
            slot.h_out[:len(reqs) * words].copy_(slot.d_out[:len(reqs) * words], non_blocking=True)
            ev = torch.cuda.Event()
            ev.record(slot.stream)
        bid = len(self.batches)
        for r in reqs:
            r.batch_id = bid
        self.batches.append((bid, group, len(reqs), total))
        slot.reqs, slot.bytes, slot.group, slot.event = reqs, nbytes, group, ev

    def _loop(self):
        torch = self.torch
        torch.cuda.set_device(self.dev)
        while True:
            with self.cv:
                self._reap()
                if self.stop_flag and not self.pending and all(s.event is None for s in self.slots):
                    return
                free = [s for s in self.slots if s.event is None]
                batch = self._form_batch() if free else None
                if batch is None:
                    self.cv.wait(timeout=0.0002)
                    continue
            group, reqs, nbytes = batch
            self._launch(free[0], group, reqs, nbytes)


def percentiles(latencies):
    a = np.sort(np.asarray(latencies, dtype=np.float64))
    if len(a) == 0:
        return {"p50_ms": None, "p99_ms": None, "mean_ms": None}
    return {"p50_ms": float(np.percentile(a, 50) * 1e3), "p99_ms": float(np.percentile(a, 99) * 1e3),
            "mean_ms": float(a.mean() * 1e3)}


def poisson_trace(count, rate, seed, groups=(1, 2), group_p=(0.7, 0.3), log2_range=None):
    """Arrival offsets (seconds), groups and sizes of `count` requests:
    exponential inter-arrival times at `rate` per second, group drawn with
    probabilities group_p, size floor(2^U) with U ~ U[lo, hi] of its group."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate, size=count)
    t = np.cumsum(gaps) - gaps[0]
    g = rng.choice(groups, size=count, p=group_p)
    sizes = np.empty(count, dtype=np.int64)
    for i in range(count):
        lo, hi = log2_range[int(g[i])]
        sizes[i] = int(np.floor(2.0 ** rng.uniform(lo, hi)))
    return t, g, sizes


def serve_trace(server: MsmServer, t, groups, scalars_list):
    """Submit requests at the trace's arrival times (real time); wait for all."""
    reqs = []
    t0 = time.perf_counter()
    for ti, g, sc in zip(t, groups, scalars_list):
        delay = t0 + ti - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        reqs.append(server.submit(int(g), sc))
    for r in reqs:
        r.done.wait()
    return reqs, time.perf_counter() - t0


def plain_trace(tables, t, groups, scalars_list, dev):
    """The same trace served one request at a time by plain launches (FIFO):
    H2D of the scalars, one MSM over the table prefix, D2H of the result."""
    import torch
    lat, results = [], []
    t0 = time.perf_counter()
    for ti, g, sc in zip(t, groups, scalars_list):
        arrival = t0 + ti
        delay = arrival - time.perf_counter()
        if delay > 0:
            time.sleep(delay)
        d = torch.from_numpy(sc.view(np.int64)).to(dev, non_blocking=False)
        out = tables[int(g)].msm(d)
        host = out.cpu()
        results.append(host)
        lat.append(time.perf_counter() - arrival)
    return lat, results, time.perf_counter() - t0
