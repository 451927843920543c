"""Serving loops: symbolic factorizations as a request stream on one GPU.

ContinuousServer (the serving path) serves by size class.  Small requests
(fewer than LARGE_REQUEST_N lines) go to the persistent kernel of
StreamServer: each is uploaded and published as soon as it arrives and fits,
and its work pieces run on whichever CTAs free up, overlapping with every
request already on the device -- many small matrices share the GPU, where
alone each would leave most SMs idle.  A large request fills the GPU on its
own: it runs alone on the factorization kernel (shared-memory state, all
warps of an SM on two traversals) once the requests on the device finish,
instead of inside the serving kernel's smaller global-state traversals.

Server batches at launch granularity instead: whenever the GPU finishes a
persistent launch, every request that has arrived in the meantime and fits
the memory budget is uploaded and joins the next launch.  It is kept for
comparison and for matrices larger than the serving kernel's limit.

Admission is by predicted device bytes (the matrix's own storage plus the
per-line state and frontier queues, n x concurrent sources x per-source
state); a request whose result is delivered releases its bytes.

Latency is measured per request from its arrival to the moment its result is
on the host; the report gives p50/p99 and sustained factorizations/s, and
`one_at_a_time` runs the same stream with batches of one for comparison.
Every result is the same whether the request ran alone or in a mix (the
launch processes each matrix independently; the test-suite checks it).
"""
from __future__ import annotations

import collections
import dataclasses
import time
from typing import Callable, Dict, List, Optional, Sequence

import numpy as np

from . import Context, Params, Result
from .matgen import Graph


# Lines from which a request runs alone on the factorization kernel instead of
# sharing the persistent serving kernel (the serving kernel's own priority
# classes split at the same size).
LARGE_REQUEST_N = 65536


@dataclasses.dataclass
class Request:
    rid: int
    arrival_s: float          # offset from the start of the stream
    graph: object             # a Graph, or a PendingGraph still being generated


class PendingGraph:
    """A request's matrix that a process pool is still generating."""

    def __init__(self, async_result):
        self._r = async_result
        self._g = None

    def ready(self) -> bool:
        return self._g is not None or self._r.ready()

    def get(self) -> Graph:
        if self._g is None:
            self._g = self._r.get()
            self._r = None
        return self._g


class LazyStream:
    """Generates the matrices of a long request stream in a process pool, in
    arrival order and at most `ahead` at a time, so a stream of thousands of
    large requests needs neither the memory nor the wait of building them all
    first.  Iterate over it for the requests; a request whose matrix is not
    ready yet arrives when it is (its latency counts from the later time)."""

    def __init__(self, pool, make: Callable, specs: Sequence, arrivals: Sequence[float], ahead: int = 256):
        self.pool, self.make, self.specs, self.arrivals = pool, make, list(specs), list(arrivals)
        self.ahead = ahead
        self.reqs: List[Request] = []
        self._next = 0

    def __len__(self):
        return len(self.specs)

    def top_up(self, consumed: int) -> None:
        """Keeps `ahead` requests generating beyond the first `consumed`."""
        while self._next < len(self.specs) and self._next < consumed + self.ahead:
            i = self._next
            pg = PendingGraph(self.pool.apply_async(self.make, (self.specs[i],)))
            self.reqs.append(Request(i, float(self.arrivals[i]), pg))
            self._next += 1


@dataclasses.dataclass
class Completion:
    rid: int
    arrival_s: float
    start_s: float            # when its launch began
    done_s: float             # when its result was on the host
    result: Result

    @property
    def latency_s(self) -> float:
        return self.done_s - self.arrival_s


def matrix_bytes(g: Graph) -> int:
    """Device bytes of an uploaded matrix: G and G^T (int32 CSR) plus the
    per-line counts kept with it."""
    return 8 * (g.n + 1) + 8 * g.nnz + 12 * g.n


class Server:
    """Continuous-batching factorization server on one device."""

    def __init__(self, ctx: Context, params: Optional[Params] = None,
                 mem_budget_bytes: int = 120 << 30, max_batch: int = 64,
                 max_lines_per_launch: int = 4_000_000):
        self.ctx = ctx
        self.params = params if params is not None else Params.default(want_pattern=0)
        self.budget = int(mem_budget_bytes)
        self.max_batch = int(max_batch)
        self.max_lines = int(max_lines_per_launch)

    def predicted_bytes(self, g: Graph) -> int:
        return matrix_bytes(g) + self.ctx.predict_scratch_bytes(g.n, g.nnz, self.params)

    def run(self, requests: Sequence[Request], clock: Callable[[], float] = time.perf_counter,
            on_result: Optional[Callable[[Completion], None]] = None) -> Dict:
        """Serves `requests` (sorted by arrival) in real time; returns the
        report and the completions (with results)."""
        reqs = sorted(requests, key=lambda r: r.arrival_s)
        for r in reqs:
            if self.predicted_bytes(r.graph) > self.budget:
                raise ValueError(f"request {r.rid} (n={r.graph.n}) exceeds the memory budget by itself")
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        pending = collections.deque(reqs)   # not yet arrived
        waiting: collections.deque = collections.deque()
        done: List[Completion] = []
        launches = 0
        batch_sizes: List[int] = []
        in_use = 0
        while pending or waiting:
            t = now()
            while pending and pending[0].arrival_s <= t:
                waiting.append(pending.popleft())
            if not waiting:
                # idle: sleep until the next arrival
                time.sleep(max(0.0, min(pending[0].arrival_s - t, 0.05)))
                continue
            # admit in arrival order while the budget and the launch size allow
            batch: List[Request] = []
            lines = 0
            in_use = 0
            while waiting and len(batch) < self.max_batch:
                r = waiting[0]
                b = self.predicted_bytes(r.graph)
                if batch and (in_use + b > self.budget or lines + r.graph.n > self.max_lines):
                    break
                waiting.popleft()
                batch.append(r)
                in_use += b
                lines += r.graph.n
            start = now()
            mats = [self.ctx.upload(r.graph) for r in batch]
            results = self.ctx.symbfact_batch(mats, self.params)
            for m in mats:
                m.free()          # releases the request's bytes
            fin = now()
            launches += 1
            batch_sizes.append(len(batch))
            for r, res in zip(batch, results):
                c = Completion(r.rid, r.arrival_s, start, fin, res)
                done.append(c)
                if on_result:
                    on_result(c)
        lat = np.array([c.latency_s for c in done])
        span = max(c.done_s for c in done) - min(c.arrival_s for c in done) if done else 0.0
        report = {
            "requests": len(done),
            "launches": launches,
            "mean_batch": float(np.mean(batch_sizes)) if batch_sizes else 0.0,
            "p50_ms": float(np.percentile(lat, 50) * 1000) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99) * 1000) if len(lat) else None,
            "mean_ms": float(lat.mean() * 1000) if len(lat) else None,
            "factorizations_per_s": len(done) / span if span > 0 else None,
            "nnz_lu_per_s": sum(c.result.nnz_lu for c in done) / span if span > 0 else None,
            "span_s": span,
        }
        return {"report": report, "completions": sorted(done, key=lambda c: c.rid)}


class ContinuousServer:
    """Serves a request stream on the persistent kernel (StreamServer):
    every request is published as soon as it arrives and fits, and runs
    alongside whatever is already on the device.  Requests that do not fit
    wait (admission by device bytes) until finished ones are fetched.
    Requests of more than max_n lines (the large class) run alone through
    `oversize` once the device is drained; later requests wait behind them in
    arrival order."""

    def __init__(self, server, poll_interval_s: float = 0.0005,
                 oversize: Optional[Callable[[Graph], Result]] = None, max_n: Optional[int] = None,
                 stall_s: float = 300.0):
        self.server = server
        self.poll_interval = poll_interval_s
        self.oversize = oversize      # runs requests above max_n (after draining)
        self.max_n = max_n
        self.stall_s = stall_s        # no completion for this long while work is in flight: error

    def run(self, requests, clock: Callable[[], float] = time.perf_counter,
            on_result: Optional[Callable[[Completion], None]] = None, keep_graphs: int = -1) -> Dict:
        """Serves the stream (a list of Requests, or a LazyStream); a
        request's latency runs from its arrival -- or, when its matrix was
        still being generated then, from the moment it was ready -- to its
        result on the host.  keep_graphs >= 0: only the first keep_graphs
        requests keep their matrices after submission (long streams)."""
        lazy = requests if isinstance(requests, LazyStream) else None
        if lazy is not None:
            lazy.top_up(0)
            reqs = lazy.reqs
            total = len(lazy)
        else:
            reqs = sorted(requests, key=lambda r: r.arrival_s)
            total = len(reqs)
        t0 = clock()
        now = lambda: clock() - t0  # noqa: E731
        pending = collections.deque(reqs)
        nxt = len(reqs)
        waiting: collections.deque = collections.deque()
        inflight: Dict[int, Request] = {}
        started: Dict[int, float] = {}
        arrived: Dict[int, float] = {}
        done: List[Completion] = []
        alone = 0                                  # large-class requests run on their own
        last_progress = now()
        while pending or waiting or inflight or (lazy is not None and nxt < total):
            t = now()
            if inflight and t - last_progress > self.stall_s:
                raise RuntimeError(f"serving stalled: {len(inflight)} requests in flight, "
                                   f"no completion for {self.stall_s:.0f} s")
            if lazy is not None:
                lazy.top_up(len(done) + len(inflight) + len(waiting))
                while nxt < len(lazy.reqs):
                    pending.append(lazy.reqs[nxt])
                    nxt += 1
            while pending and pending[0].arrival_s <= t:
                r = pending[0]
                if isinstance(r.graph, PendingGraph):
                    if not r.graph.ready():
                        break                      # arrives when its matrix exists
                    r.graph = r.graph.get()
                arrived[r.rid] = max(r.arrival_s, t)
                waiting.append(pending.popleft())
            # admit waiting requests in arrival order while they fit
            while waiting:
                r = waiting[0]
                st = now()
                if self.max_n is not None and r.graph.n > self.max_n:
                    if inflight:
                        break                      # finish what runs, then take it alone
                    self.server.drain()
                    res = self.oversize(r.graph)
                    alone += 1
                    waiting.popleft()
                    c = Completion(r.rid, arrived.pop(r.rid, r.arrival_s), st, now(), res)
                    done.append(c)
                    if on_result:
                        on_result(c)
                    continue
                rid = self.server.submit(r.graph)
                if rid is None:
                    break
                waiting.popleft()
                if 0 <= keep_graphs <= r.rid:
                    r.graph = None                 # uploaded: the host copy can go
                inflight[rid] = r
                started[rid] = st
            for rid in self.server.poll():
                last_progress = now()
                res = self.server.result(rid)
                r = inflight.pop(rid)
                c = Completion(r.rid, arrived.pop(r.rid, r.arrival_s), started.pop(rid), now(), res)
                done.append(c)
                if on_result:
                    on_result(c)
            if not waiting and inflight:
                time.sleep(self.poll_interval)
            elif not inflight and not waiting and pending:
                time.sleep(max(0.0005, min(pending[0].arrival_s - now(), 0.05)))
            elif not inflight and not waiting and not pending:
                time.sleep(0.001)                  # the next matrix is still being generated
        lat = np.array([c.latency_s for c in done])
        span = max(c.done_s for c in done) - min(c.arrival_s for c in done) if done else 0.0
        report = {
            "requests": len(done),
            "p50_ms": float(np.percentile(lat, 50) * 1000) if len(lat) else None,
            "p99_ms": float(np.percentile(lat, 99) * 1000) if len(lat) else None,
            "mean_ms": float(lat.mean() * 1000) if len(lat) else None,
            "factorizations_per_s": len(done) / span if span > 0 else None,
            "nnz_lu_per_s": sum(c.result.nnz_lu for c in done) / span if span > 0 else None,
            "span_s": span,
            "run_alone": alone,
        }
        return {"report": report, "completions": sorted(done, key=lambda c: c.rid)}


def run_alone(ctx: Context, g: Graph, params: Optional[Params] = None) -> Result:
    """One request alone on the factorization kernel (the large class):
    upload, factorize, free the matrix."""
    with ctx.upload(g) as m:
        return ctx.symbfact(m, params if params is not None else Params.default(want_pattern=0))


def one_at_a_time(ctx: Context, requests: Sequence[Request], params: Optional[Params] = None,
                  clock: Callable[[], float] = time.perf_counter) -> Dict:
    """The same stream served one request per launch (no batching)."""
    srv = Server(ctx, params, max_batch=1)
    return srv.run(requests, clock)


def make_stream(count: int, n_lo: int, n_hi: int, rate_hz: float, seed: int,
                build: Callable[[str, int, int], Graph]) -> List[Request]:
    """A seeded Poisson stream of `count` requests of the mixed kinds."""
    from . import matgen
    spec = matgen.mixed_spec(count, n_lo, n_hi, seed)
    rng = np.random.default_rng(seed + 1)
    t = np.cumsum(rng.exponential(1.0 / rate_hz, size=count))
    return [Request(i, float(a), build(k, n, s)) for i, (a, (k, n, s)) in enumerate(zip(t, spec))]
