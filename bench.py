"""Benchmark: symbolic LU factorization throughput on the B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload nd3d|plain2d|circuit|bundled]

A step is one full symbolic factorization (fill pattern of L and U, per-line
counts, supernode partition) of the workload matrix.  The default workload is
the 80^3 7-point stencil in geometric nested-dissection order with a seeded
10% of one-sided drops (n = 512,000), the single-GPU configuration the
headline metric is quoted on.  Inputs are seeded synthetic matrices.

Printed (rank 0, one JSON line):
  value  -- nnz(L+U)/s over all ranks, matrix resident in HBM, pattern kept on
            the device, CUDA events on the launching stream, max over ranks;
  e2e    -- the same metric through the public API from pinned host buffers:
            upload (H2D + graph build), factorization, and download of every
            result array including the pattern, all inside the timed region;
  roofline, cpu_baseline, clocks, gpu_launches as documented in the keys.

Multi-GPU (torchrun): ONE matrix is split into contiguous source-line ranges
of equal predicted work, one per rank; each rank factorizes its range with
traversal reuse and the per-line arrays are summed over NCCL.  Total work is
fixed as N grows: strong scaling.

--impl reference times the CPU restatement of the reference algorithm (the
reference has no CPU path of its own) on a bounded, evenly strided sample of
the workload's sources, with all host threads, in the same metric.
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=["nd3d", "plain2d", "circuit", "bundled", "batch", "serve", "order"],
                    default="nd3d")
    ap.add_argument("--batch-count", type=int, default=256,
                    help="matrices in the batch workload (also measured beside the default line; 0: skip)")
    ap.add_argument("--serve-count", type=int, default=120, help="requests in the serving stream")
    ap.add_argument("--serve-nmax", type=int, default=1_000_000, help="largest n of the serving stream")
    ap.add_argument("--serve-rate", type=float, default=20.0, help="Poisson arrival rate (1/s)")
    ap.add_argument("--serve-default", type=int, default=240,
                    help="requests of the short serving stream measured beside the default line (0: skip)")
    ap.add_argument("--serve-default-rate", type=float, default=60.0, help="its Poisson rate (1/s)")
    ap.add_argument("--serve-compare", type=int, default=120,
                    help="first requests served again, continuously and one at a time, for the comparison")
    ap.add_argument("--side", type=int, default=80, help="grid side of the nd3d workload")
    ap.add_argument("--reuse", type=int, default=-1,
                    help="reuse traversals along s-1 -> s chains (-1: library default, on)")
    ap.add_argument("--block", type=int, default=0)
    ap.add_argument("--lanes", type=int, default=0)
    ap.add_argument("--ctas-per-sm", type=int, default=0)
    ap.add_argument("--chunk", type=int, default=0, help="sources per work piece (0: library default)")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU baseline sample budget")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--wide-regs", action="store_true",
                    help="512-thread CTAs with up to 128 registers a thread (GSOFA_FLAG_WIDE_REGS)")
    ap.add_argument("--form", choices=["ranges", "csr"], default="ranges",
                    help="pattern form: begin/end ranges into a pool (no compaction) or CSR")
    ap.add_argument("--state", choices=["auto", "global", "shared"], default="auto",
                    help="where the traversals keep their visited bitmaps")
    ap.add_argument("--partitions", type=int, default=4,
                    help="one GPU: also time the matrix as this many work-predicted line ranges, "
                         "one after another (the multi-GPU split, measured on one device; 0: skip)")
    ap.add_argument("--host-pool-gb", type=float, default=16.0,
                    help="circuit workload: host buffer the pattern streams into, range by range (0: skip)")
    ap.add_argument("--pattern", type=int, default=-1,
                    help="materialize the L+U pattern (-1: yes except for the circuit workload, "
                         "whose pattern does not fit in memory)")
    return ap.parse_args()


def workload(args):
    from gsofa_b200 import matgen
    if args.workload == "nd3d":
        g = matgen.config_nd3d(args.side)
        cfg = {"workload": f"grid3d_{args.side}^3_7pt_nd_drop0.1", "n": g.n, "nnz": g.nnz,
               "ordering": "geometric nested dissection", "seed": matgen.SEEDS["nd3d"]}
    elif args.workload == "plain2d":
        g = matgen.config_plain2d()
        cfg = {"workload": "grid2d_64x64_5pt_natural", "n": g.n, "nnz": g.nnz, "ordering": "natural"}
    elif args.workload == "circuit":
        g = matgen.config_circuit()
        cfg = {"workload": "powerlaw_659033_rcm", "n": g.n, "nnz": g.nnz, "ordering": "random+RCM",
               "seed": matgen.SEEDS["circuit"]}
    else:
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        from tests.common import bundled
        g = bundled()
        cfg = {"workload": "superlu_dump_11948", "n": g.n, "nnz": g.nnz}
    return g, cfg


class ClockSampler:
    """SM clock, power and clock-event reasons sampled through NVML (in
    process: no child processes, so the timed loop is not disturbed) every
    200 ms while the timed region runs.  Only reads device state."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"),
               ("hw_power_brake", "nvmlClocksEventReasonHwPowerBrakeSlowdown"))

    def __init__(self, device_index: int):
        self.dev = device_index
        self.samples = []
        self._stop = threading.Event()
        self._t = None
        self._nvml = None
        self._h = None
        self.max_mhz = None
        try:
            import pynvml
            pynvml.nvmlInit()
            vis = os.environ.get("CUDA_VISIBLE_DEVICES")
            idx = device_index
            if vis:
                ids = [x.strip() for x in vis.split(",") if x.strip()]
                if device_index < len(ids) and ids[device_index].isdigit():
                    idx = int(ids[device_index])
            self._h = pynvml.nvmlDeviceGetHandleByIndex(idx)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
            self._nvml = pynvml
        except Exception:
            self._nvml = None

    def _run(self):
        n = self._nvml
        while not self._stop.is_set():
            try:
                sm = n.nvmlDeviceGetClockInfo(self._h, n.NVML_CLOCK_SM)
                try:
                    rs = n.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                except Exception:
                    rs = n.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
                pw = n.nvmlDeviceGetPowerUsage(self._h) / 1000.0
                self.samples.append((sm, rs, pw))
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        if self._nvml is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        if self._t is not None:
            self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": self.max_mhz, "reasons": ["unsampled"]}
        reasons = set()
        for _, rs, _ in self.samples:
            for name, const in self.REASONS:
                bit = getattr(self._nvml, const, 0)
                if bit and (rs & bit):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(s[0] for s in self.samples), "sm_max_mhz": self.max_mhz,
                "reasons": sorted(reasons), "power_w_max": max(s[2] for s in self.samples),
                "samples": len(self.samples)}


def hbm_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def traffic_per_launch(cfg_name, form):
    """DRAM bytes per factorization launch from the committed ncu summary
    (profiles/traffic.json, keyed by workload and pattern form)."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(p) as f:
            d = json.load(f)
        e = d.get(f"{cfg_name}/{form}")
        return None if e is None else float(e["dram_bytes_per_launch"])
    except Exception:
        return None


def _line_orig(g, src):
    """Distinct off-diagonal original entries of each listed line."""
    out = np.zeros(src.shape[0], np.int64)
    for i, s in enumerate(src.tolist()):
        row = np.unique(g.adj[g.beg[s]:g.end[s]])
        out[i] = row.shape[0] - int(np.any(row == s))
    return out


def cpu_sample(g, budget_s, step_hint=None, extras=True):
    """Times the CPU oracle on every k-th line of the workload (the highest
    line included), both reachability passes, all OpenMP threads, one line per
    scheduling step with the heaviest lines first.  k is calibrated so the
    timed run takes at least a quarter of budget_s (or given as step_hint).

    Returns a dict: rate (nnz(L+U) of the sampled lines per second), the
    sample, the oracle's per-line counts (c0: U rows, c1: L columns) for the
    parity check, and -- with extras -- the same sample timed on one thread
    (serial) and with the max-id restatement of the reference's own algorithm
    (OpenMP) on a sub-sample."""
    import oracle
    n = g.n
    threads = oracle.threads()

    def run(k):
        src = np.arange(n - 1, -1, -k, dtype=np.int32)   # includes the heaviest line
        t0 = time.perf_counter()
        c0, _, _, _ = oracle.counts(g.beg, g.end, g.adj, 0, nthreads=0, sources=src)
        c1, _, _, _ = oracle.counts(g.beg, g.end, g.adj, 1, nthreads=0, sources=src)
        dt = time.perf_counter() - t0
        nnz = int(c0[src].sum(dtype=np.int64) + c1[src].sum(dtype=np.int64) + src.shape[0])
        return nnz, dt, src, c0, c1

    k = step_hint or max(1, n // 64)
    nnz, dt, src, c0, c1 = run(k)
    while step_hint is None and dt < budget_s / 4 and k > 1:
        k = max(1, min(n, int(k * max(dt, 1e-3) / (budget_s / 2))))
        nnz, dt, src, c0, c1 = run(k)
    out = {"rate": nnz / dt, "seconds": dt, "k": k, "sources": src, "c0": c0, "c1": c1,
           "threads": threads, "cores": os.cpu_count() or 1,
           "omp_num_threads": os.environ.get("OMP_NUM_THREADS"),
           "desc": f"every {k}-th line of both passes ({src.shape[0]} of {n} sources), {dt:.2f} s"}
    if not extras:
        return out
    # one thread on every m-th sampled line (about a quarter of the budget)
    m = max(1, int(round(threads * dt / max(budget_s / 4, 1e-3))))
    sub = src[::m]
    t0 = time.perf_counter()
    s0, _, _, _ = oracle.counts(g.beg, g.end, g.adj, 0, nthreads=1, sources=sub)
    s1, _, _, _ = oracle.counts(g.beg, g.end, g.adj, 1, nthreads=1, sources=sub)
    ts = time.perf_counter() - t0
    out["serial"] = {"value": int(s0[sub].sum(dtype=np.int64) + s1[sub].sum(dtype=np.int64) + sub.shape[0]) / ts,
                     "unit": "nnz/s", "cores": 1, "sample": f"every {k * m}-th line ({sub.shape[0]} sources), "
                     f"{ts:.2f} s"}
    # the reference's algorithm (max-id label propagation) on every 4th
    # sampled line: nnz of a line = its fills + its distinct originals + 1
    sub = src[::4]
    t0 = time.perf_counter()
    fills, _, _ = oracle.maxid_counts(g.beg, g.end, g.adj, sub)
    tm = time.perf_counter() - t0
    nnz_m = fills + int(_line_orig(g, sub).sum()) + sub.shape[0]
    out["maxid"] = {"value": nnz_m / tm, "unit": "nnz/s", "cores": threads,
                    "sample": f"every {4 * k}-th line ({sub.shape[0]} sources), {tm:.2f} s"}
    return out


def cpu_baseline_obj(cs):
    """The JSON object of a CPU sample: the OpenMP reachability restatement is
    the divisor; the serial run and the max-id restatement ride along."""
    o = {"value": cs["rate"], "unit": "nnz/s", "cores": cs["threads"], "host_cores": cs["cores"],
         "omp_num_threads": cs["omp_num_threads"], "kind": "port",
         "algorithm": "two-pass reachability restatement, OpenMP, one line per scheduling step",
         "sample": cs["desc"], "sample_sources": int(cs["sources"].shape[0])}
    for key in ("serial", "maxid"):
        if key in cs:
            o[key] = cs[key]
    return o


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    g, cfg = workload(args)
    # one calibration (which also times the serial and max-id runs), then
    # warm-up and timed steps on the same sample as the GPU arm's baseline
    cs = cpu_sample(g, args.cpu_seconds)
    for _ in range(max(args.warmup - 1, 0)):
        cpu_sample(g, args.cpu_seconds, step_hint=cs["k"], extras=False)
    rates = []
    t0 = time.perf_counter()
    for _ in range(args.steps):
        rates.append(cpu_sample(g, args.cpu_seconds, step_hint=cs["k"], extras=False)["rate"])
    wall = time.perf_counter() - t0
    value = statistics.mean(rates)
    base = cpu_baseline_obj(cs)
    base["value"] = value
    line = {
        "metric": "nnz(L+U)/s", "value": value, "unit": "nnz/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * wall / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32",
        "data": "synthetic (seeded generator)", "impl": "reference",
        "config": dict(cfg, sample=cs["desc"]),
        "cpu_baseline": base,
        "e2e": {"value": value, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def batch_main(args):
    """The mixed-size batch: 256 matrices (n log-uniform in [2,000, 200,000];
    2-D natural, 3-D nested dissection and power-law RCM patterns) factorized
    in one persistent launch, against the plain loop of one launch per matrix
    on the same GPU.  Counts and supernodes are produced (the power-law
    members' patterns, ~0.25 n^2 entries each, do not fit in memory)."""
    import torch
    import gsofa_b200
    from gsofa_b200 import autotune, matgen

    torch.cuda.set_device(0)
    spec = matgen.config_batch(args.batch_count)
    graphs = [matgen.make(k, n, sd) for k, n, sd in spec]
    ctx = gsofa_b200.Context(0)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    mats = [ctx.upload(g) for g in graphs]
    base = gsofa_b200.Params.default(want_pattern=0, flags=gsofa_b200.FLAG_NO_DOWNLOAD)
    sample = mats[:: max(1, len(mats) // 32)]
    tuned, report = autotune.autotune(ctx, sample, base, use_cache=False)

    def timed(fn, k):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = None
        for _ in range(k):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1), out

    # plain: one launch per matrix
    plain_once = lambda: [ctx.symbfact(m, tuned) for m in mats]  # noqa: E731
    plain_once()
    t_plain, plain_res = timed(plain_once, 1)
    # batched: one persistent launch (captured in a CUDA graph, replayed)
    bp = gsofa_b200.Params()
    autotune.ctypes_copy(bp, tuned)
    bp.flags |= gsofa_b200.FLAG_GRAPH
    batch_once = lambda: ctx.symbfact_batch(mats, bp)  # noqa: E731
    for _ in range(max(args.warmup, 1)):
        batch_once()
    with ClockSampler(0) as clk:
        t_batch, batch_res = timed(batch_once, args.steps)
    for a, b in zip(plain_res, batch_res):
        assert (a.fill_count, a.nnz_lu, a.n_supernodes) == (b.fill_count, b.nnz_lu, b.n_supernodes)
    nnz = sum(r.nnz_lu for r in batch_res)
    value = args.steps * nnz / (t_batch / 1000.0)
    plain_value = nnz / (t_plain / 1000.0)
    line = {
        "metric": "nnz(L+U)/s", "value": value, "unit": "nnz/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_batch / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)",
        "config": {"workload": f"batch_{len(mats)}_mixed_2k-200k", "matrices": len(mats),
                   "lines": int(sum(g.n for g in graphs)), "nnz": int(sum(g.nnz for g in graphs)),
                   "nnz_lu": int(nnz), "pattern": "counts only", "seed": matgen.SEEDS["batch"],
                   "autotune": report, "graph": "CUDA graph replay of the persistent launch"},
        "factorizations_per_s": args.steps * len(mats) / (t_batch / 1000.0),
        "plain_loop": {"value": plain_value, "ms": t_plain,
                       "factorizations_per_s": len(mats) / (t_plain / 1000.0)},
        "batched_vs_plain": value / plain_value,
        "clocks": clk.summary(), "gpu_launches": args.steps,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0


def _make_graph(spec):
    from gsofa_b200 import matgen
    kind, n, seed = spec
    return matgen.make(kind, n, seed)


def serving_run(ctx, count, nmax, rate, compare, pool_procs=16):
    """Continuous batching on the persistent serving kernel over a seeded
    Poisson stream of `count` mixed-kind requests (n log-uniform in [1,000,
    nmax]) under a 120 GB admission budget, the matrices generated in a
    process pool while they are served.  The first `compare` requests are then
    served again, continuously and one request per launch, for the
    comparison; the results must be identical request by request."""
    import multiprocessing as mp
    import gsofa_b200
    from gsofa_b200 import matgen, serve

    spec = matgen.mixed_spec(count, 1000, nmax, matgen.SEEDS["serve"])
    rng = np.random.default_rng(matgen.SEEDS["serve"] + 1)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=len(spec)))
    k = min(compare, len(spec))
    pool = mp.get_context("spawn").Pool(min(pool_procs, os.cpu_count() or 1))
    params = gsofa_b200.Params.default(want_pattern=0)
    srv = gsofa_b200.StreamServer(0, mem_budget_bytes=120 << 30)
    oversize = lambda g: serve.run_alone(ctx, g, params)  # noqa: E731
    # size classes: small requests share the persistent serving kernel, large
    # ones run alone on the factorization kernel
    cs = serve.ContinuousServer(srv, oversize=oversize, max_n=min(srv.max_n, serve.LARGE_REQUEST_N - 1))
    warm = [serve.Request(-1 - i, 0.0, matgen.make("grid3d", 2000, i)) for i in range(4)]
    cs.run(warm)
    stream = serve.LazyStream(pool, _make_graph, spec, arrivals, ahead=256)
    with ClockSampler(0) as clk:
        full = cs.run(stream, keep_graphs=k)
    srv.drain()
    sub = [serve.Request(r.rid, r.arrival_s, r.graph) for r in stream.reqs[:k]]
    cont = cs.run(sub)
    srv.drain()
    max_n = srv.max_n
    srv.close()
    single = serve.one_at_a_time(ctx, sub, params)
    pool.close()
    by_id = {c.rid: c for c in full["completions"]}
    same = True
    for a, b in zip(cont["completions"], single["completions"]):
        c = by_id[a.rid]
        same &= (a.result.fill_count, a.result.nnz_lu, a.result.n_supernodes) == \
                (b.result.fill_count, b.result.nnz_lu, b.result.n_supernodes) == \
                (c.result.fill_count, c.result.nnz_lu, c.result.n_supernodes)
        same &= bool(np.array_equal(a.result.u_row_count, b.result.u_row_count))
        same &= bool(np.array_equal(a.result.sn_start, c.result.sn_start))
    return {"workload": f"serve_{len(spec)}_poisson_{rate:g}hz_n1k-{nmax}", "requests": len(spec),
            "admission_budget_gb": 120, "pattern": "counts only", "seed": matgen.SEEDS["serve"],
            "serving": full["report"],
            "comparison": {"requests": k, "continuous": cont["report"], "one_at_a_time": single["report"]},
            "results_identical": bool(same), "serving_kernel_max_n": max_n,
            "size_classes": {"serving_kernel": f"n < {serve.LARGE_REQUEST_N}",
                             "alone_on_factorization_kernel": f"n >= {serve.LARGE_REQUEST_N}"},
            "clocks": clk.summary(),
            "generation": "process pool, in arrival order, while serving (a request arrives when both "
                          "its time and its matrix have come)"}


def order_main(args):
    """The step before the path: reverse Cuthill-McKee on the GPU
    (gsofa_order_rcm) of the power-law circuit pattern before it is ordered
    (n = 659,033, the same shuffle the circuit workload's generator orders
    with scipy), timed end to end through the public call (host arrays in,
    permutation out), against the oracle's sequential restatement on one
    host core; parity is bit-exact, and the ordered pattern is factorized
    (counts) to report the fill the ordering leaves."""
    import torch
    import gsofa_b200
    import oracle
    from gsofa_b200 import matgen
    torch.cuda.set_device(0)
    g = matgen.powerlaw(659_033, seed=matgen.SEEDS["circuit"], ordering="random")
    ctx = gsofa_b200.Context(0)
    for _ in range(args.warmup):
        perm = ctx.order_rcm(g)
    times = []
    with ClockSampler(0) as clk:
        for _ in range(args.steps):
            t0 = time.perf_counter()
            perm = ctx.order_rcm(g)
            times.append((time.perf_counter() - t0) * 1000.0)
    t_cpu = time.perf_counter()
    want = oracle.rcm(g.beg, g.end, g.adj)
    t_cpu = (time.perf_counter() - t_cpu) * 1000.0
    same = bool(np.array_equal(perm, want))
    inv = np.empty(g.n, np.int64)
    inv[perm] = np.arange(g.n)
    rows = np.repeat(np.arange(g.n), g.end - g.beg)
    band_in = int(np.abs(rows - g.adj.astype(np.int64)).max())
    band_out = int(np.abs(inv[rows] - inv[g.adj]).max())
    h = gsofa_b200.permute_lines(g, perm)
    with ctx.upload(h) as m:
        ordered = ctx.symbfact(m, gsofa_b200.Params.default(want_pattern=0, flags=gsofa_b200.FLAG_NO_DOWNLOAD))
    ms = float(np.median(times))
    line = {
        "metric": "ordering time", "value": ms, "unit": "ms", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)",
        "config": {"workload": f"rcm_{g.name}", "n": g.n, "nnz": g.nnz,
                   "ordering": "reverse Cuthill-McKee of A + A^T, George-Liu start, (degree, id) ties"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": int(4 * (2 * g.n + g.nnz)),
                "d2h_bytes_per_step": int(4 * g.n)},
        "cpu_baseline": {"value": t_cpu, "unit": "ms", "cores": 1, "kind": "port",
                         "sample": "the whole matrix, once (sequential restatement)"},
        "parity": {"perm_identical_to_oracle": same},
        "bandwidth": {"input": band_in, "ordered": band_out},
        "fill_after_ordering": {"nnz_lu": int(ordered.nnz_lu), "fill_count": int(ordered.fill_count),
                                "factorization_kernel_ms": float(ordered.kernel_ms)},
        "clocks": clk.summary(), "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0 if same else 1


def serve_main(args):
    """The serving configuration as its own line: --serve-count requests
    (10,000 for the full stream), n up to --serve-nmax, at --serve-rate."""
    import torch
    import gsofa_b200
    torch.cuda.set_device(0)
    ctx = gsofa_b200.Context(0)
    out = serving_run(ctx, args.serve_count, args.serve_nmax, args.serve_rate, args.serve_compare)
    rep = out["serving"]
    line = {
        "metric": "nnz(L+U)/s", "value": rep["nnz_lu_per_s"], "unit": "nnz/s", "n_gpus": 1,
        "steps": 1, "warmup": 1, "ms_per_step": rep["span_s"] * 1000.0, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)",
        "config": {k: out[k] for k in ("workload", "requests", "admission_budget_gb", "pattern", "seed",
                                       "generation")},
        "serving": rep, "comparison": out["comparison"], "results_identical": out["results_identical"],
        "serving_kernel_max_n": out["serving_kernel_max_n"], "size_classes": out["size_classes"],
        "factorizations_per_s": rep["factorizations_per_s"],
        "clocks": out["clocks"], "gpu_launches": None,
    }
    print(json.dumps(line), flush=True)
    ctx.close()
    return 0 if out["results_identical"] else 1


def _sha(a, dtype) -> str:
    import hashlib
    return hashlib.sha256(np.ascontiguousarray(a, dtype=dtype).tobytes()).hexdigest()


def check_parity(g, workload_name, res, cs, want_pattern):
    """Compares a GPU result (per-line arrays downloaded through the public
    API) with the CPU oracle: the U row and L column counts of every sampled
    line, the sorted lists of every 8th sampled line (pattern mode), and --
    where tests/golden/large.json holds the workload -- the SHA-256 digests of
    the full per-line arrays and supernode starts from a full oracle run."""
    import oracle
    src = cs["sources"]
    bad = int(np.count_nonzero(res.u_row_count[src] != cs["c0"][src]))
    bad += int(np.count_nonzero(res.l_col_count[src] != cs["c1"][src]))
    out = {"lines_checked": int(src.shape[0]), "fields": ["u_row_count", "l_col_count"],
           "sample": cs["desc"]}
    if want_pattern and (res.u_ptr is not None or res.u_beg is not None):
        sub = src[::8]
        for pass_, cnt, row in ((0, cs["c0"], res.u_row), (1, cs["c1"], res.l_col)):
            rp, ri = oracle.lists(g.beg, g.end, g.adj, pass_, sub, cnt)
            for i, s_ in enumerate(sub.tolist()):
                if not np.array_equal(row(s_), ri[rp[i]:rp[i + 1]]):
                    bad += 1
        out["lists_checked"] = int(2 * sub.shape[0])
        out["fields"].append("sorted U row / L column lists")
    gold = None
    try:
        with open(os.path.join(ROOT, "tests", "golden", "large.json")) as f:
            gold = json.load(f).get(workload_name)
    except (OSError, ValueError):
        gold = None
    if gold is not None:
        flags = res.line_flags if res.line_flags is not None else None
        got = {"u_row_count": _sha(res.u_row_count, "<i4"), "l_col_count": _sha(res.l_col_count, "<i4"),
               "sn_start": _sha(res.sn_start, "<i4")}
        if flags is not None:
            got["line_flags"] = _sha(flags, "u1")
        gm = [k for k, v in got.items() if v != gold["sha256"][k]]
        gm += [k for k in ("fill_count", "nnz_lu", "n_supernodes") if int(getattr(res, k)) != int(gold[k])]
        bad += len(gm)
        out["golden"] = {"file": "tests/golden/large.json", "compared": sorted(got) + ["fill_count", "nnz_lu",
                         "n_supernodes"], "mismatched": gm}
    out["mismatches"] = bad
    return out


def link_gbs(torch, stream, nbytes=1 << 30):
    """Device-to-host copy rate of this box's host link: 1 GiB from device
    memory into page-locked host memory, best of three, CUDA events."""
    src = torch.empty(nbytes, dtype=torch.uint8, device="cuda")
    dst = torch.empty(nbytes, dtype=torch.uint8).pin_memory()
    best = None
    for _ in range(3):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dst.copy_(src, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        best = ms if best is None else min(best, ms)
    return nbytes / (best / 1000.0) / 1e9


def _params(gsofa_b200, args, **kw):
    """Library parameters from the command line (plus overrides)."""
    flags = {"auto": 0, "global": gsofa_b200.FLAG_GLOBAL_STATE, "shared": gsofa_b200.FLAG_SHARED_STATE}[args.state]
    if args.wide_regs:
        flags |= gsofa_b200.FLAG_WIDE_REGS
    base = dict(reuse=args.reuse, block_size=args.block, src_chunk=args.chunk, threads_per_source=args.lanes,
                ctas_per_sm=args.ctas_per_sm, flags=flags)
    extra_flags = kw.pop("flags", 0)
    base.update(kw)
    base["flags"] = flags | extra_flags
    return gsofa_b200.Params.default(**base)


def _device_timed(torch, stream, flush, steps, fn):
    """Runs fn() `steps` times between CUDA events on the launching stream,
    flushing L2 between steps; returns (ms, results)."""
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = []
    for i in range(steps):
        if i:
            flush.fill_(i & 0xff)
        out.append(fn())
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1), out


def batched_vs_plain(args, ctx, torch, stream, gsofa_b200):
    """The mixed-size batch (256 matrices, n log-uniform in [2,000, 200,000],
    2-D natural / 3-D nested-dissection / power-law RCM) in one persistent
    launch replayed from a CUDA graph, against the plain loop of one launch
    per matrix on the same GPU; counts and supernodes (the power-law members'
    patterns hold ~0.25 n^2 entries each).  Also per matrix kind, so the
    ratio's make-up is visible.  Results are compared matrix by matrix."""
    import multiprocessing as mp
    from gsofa_b200 import matgen
    spec = matgen.config_batch(args.batch_count)
    with mp.get_context("spawn").Pool(min(16, os.cpu_count() or 1)) as pool:
        graphs = pool.map(_make_graph, spec, chunksize=4)
    mats = [ctx.upload(g) for g in graphs]
    flags = {"auto": 0, "global": gsofa_b200.FLAG_GLOBAL_STATE, "shared": gsofa_b200.FLAG_SHARED_STATE}[args.state]
    p = gsofa_b200.Params.default(want_pattern=0, flags=gsofa_b200.FLAG_NO_DOWNLOAD | flags)
    pg = gsofa_b200.Params.default(want_pattern=0, flags=gsofa_b200.FLAG_NO_DOWNLOAD | gsofa_b200.FLAG_GRAPH | flags)

    def timed(fn, k):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = None
        for _ in range(k):
            out = fn()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / k, out

    def plain(ms):
        return [ctx.symbfact(m, p) for m in ms]

    plain(mats)
    t_plain, rp = timed(lambda: plain(mats), 1)
    ctx.symbfact_batch(mats, pg)
    t_batch, rb = timed(lambda: ctx.symbfact_batch(mats, pg), 2)
    same = all((a.fill_count, a.nnz_lu, a.n_supernodes) == (b.fill_count, b.nnz_lu, b.n_supernodes)
               for a, b in zip(rp, rb))
    per_kind = {}
    for kind in ("grid2d", "grid3d", "powerlaw"):
        sel = [m for m, (k, _, _) in zip(mats, spec) if k == kind]
        if not sel:
            continue
        tp, _ = timed(lambda: plain(sel), 1)
        ctx.symbfact_batch(sel, p)
        tb, _ = timed(lambda: ctx.symbfact_batch(sel, p), 1)
        per_kind[kind] = {"matrices": len(sel), "lines": int(sum(m.n for m in sel)), "plain_ms": tp,
                          "batched_ms": tb, "batched_vs_plain": tp / tb}
    nnz = sum(r.nnz_lu for r in rb)
    for m in mats:
        m.free()
    return {"workload": f"batch_{len(mats)}_mixed_2k-200k", "matrices": len(mats),
            "lines": int(sum(g.n for g in graphs)), "nnz_lu": int(nnz), "seed": matgen.SEEDS["batch"],
            "pattern": "counts only", "batched_ms": t_batch, "plain_ms": t_plain,
            "batched_value": nnz / (t_batch / 1000.0), "plain_value": nnz / (t_plain / 1000.0),
            "batched_vs_plain": t_plain / t_batch,
            "batched_factorizations_per_s": len(mats) / (t_batch / 1000.0),
            "plain_factorizations_per_s": len(mats) / (t_plain / 1000.0),
            "graph": "one persistent launch replayed from a CUDA graph", "results_identical": same,
            "per_kind": per_kind}


def streamed_pattern(args, ctx, m, torch, gsofa_b200, g):
    """The whole pattern of a matrix whose pattern no device holds (the
    659,033-line power-law matrix: ~1.2e11 entries, ~480 GB), produced in
    contiguous line ranges, each written as begin/end ranges into one
    page-locked host buffer of --host-pool-gb while its traversals run (the
    staged form: full blocks leave the device during the kernel).  The ranges
    are cut from the exact per-line counts of a counts-only run so that each
    fills most of the buffer.  A consumer would take each range's lists before
    the next range overwrites the buffer; here every range's per-line counts
    are checked against the counts-only run and its lists against the oracle
    on sampled lines.  Timed end to end (device events around all ranges,
    copies included)."""
    import oracle
    counts = ctx.symbfact(m, want_pattern=0)
    per_line = counts.u_row_count.astype(np.int64) + counts.l_col_count.astype(np.int64)
    cum = np.concatenate([[0], np.cumsum(per_line)])
    need = int(cum[-1])
    cap = int(args.host_pool_gb * (1 << 30) // 4)
    if per_line.max() > cap:
        raise ValueError("one line's lists exceed the host buffer")
    cuts = [0]
    while cuts[-1] < g.n:
        lo = cuts[-1]
        hi = int(np.searchsorted(cum, cum[lo] + cap, side="right")) - 1
        cuts.append(max(lo + 1, min(hi, g.n)))
    hpool = torch.empty(cap, dtype=torch.int32).pin_memory().numpy()
    stream = torch.cuda.current_stream()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    bad, checked, written, kms, total_ms = 0, 0, 0, 0.0, 0.0
    rng = np.random.default_rng(7)
    for k in range(len(cuts) - 1):
        lo, hi = cuts[k], cuts[k + 1]
        p = gsofa_b200.Params.default(line_lo=lo, line_hi=hi)
        torch.cuda.synchronize()
        e0.record(stream)
        r = ctx.symbfact_ranges(m, hpool, p)
        e1.record(stream)
        torch.cuda.synchronize()
        total_ms += e0.elapsed_time(e1)
        written += r.pool_used
        kms += r.kernel_ms
        if not (np.array_equal(r.u_row_count[lo:hi], counts.u_row_count[lo:hi]) and
                np.array_equal(r.l_col_count[lo:hi], counts.l_col_count[lo:hi])):
            bad += 1
        src = np.unique(rng.integers(lo, hi, size=3).astype(np.int32))
        for pass_, row, cnt in ((0, r.u_row, counts.u_row_count), (1, r.l_col, counts.l_col_count)):
            rp, ri = oracle.lists(g.beg, g.end, g.adj, pass_, src, cnt)
            for i, s_ in enumerate(src.tolist()):
                checked += 1
                if not np.array_equal(row(s_), ri[rp[i]:rp[i + 1]]):
                    bad += 1
    return {"entries": int(written), "expected_entries": need, "ranges": len(cuts) - 1,
            "host_pool_gb": args.host_pool_gb, "ms": total_ms, "kernel_ms": kms,
            "value": (written + g.n) / (total_ms / 1000.0), "unit": "nnz/s",
            "d2h_bytes": int(4 * written), "lists_checked": checked, "mismatches": bad,
            "note": "the whole pattern produced in host memory range by range, each range's lists "
                    "streamed out of the device while its traversals ran"}


def sharded_main(args, world, rank, local):
    """N GPUs (torchrun): ONE matrix split over the ranks as contiguous line
    ranges of equal predicted work (gsofa_partition_lines), each rank
    factorizing its range with traversal reuse; the per-line arrays are then
    summed over NCCL (distributed.symbfact_sharded).  Total work is fixed as N
    grows: strong scaling.  value = nnz(L+U) of the whole matrix per second
    (whole-matrix factorizations x nnz(L+U)), timed on the device as the max
    over ranks."""
    import torch
    import torch.distributed as dist
    import gsofa_b200
    from gsofa_b200 import distributed

    g, cfg = workload(args)
    want_pattern = args.pattern if args.pattern >= 0 else int(args.workload != "circuit")
    ctx = gsofa_b200.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    m = ctx.upload(g)
    nd = gsofa_b200.FLAG_NO_DOWNLOAD
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    cuts, pred = gsofa_b200.partition_lines(g, world)
    lo, hi = int(cuts[rank]), int(cuts[rank + 1])
    rp = distributed.rank_params(rank, world, cuts, _params(gsofa_b200, args, flags=nd))
    share = ctx.symbfact(m, rp)
    need = int(share.nnz_u + share.nnz_l)
    if want_pattern:
        dpool = torch.empty(max(need, 1), dtype=torch.int32, device="cuda")
        pr = distributed.rank_params(rank, world, cuts, _params(gsofa_b200, args, flags=nd))
        pr.want_pattern = 2
        step = lambda: ctx.symbfact_ranges(m, dpool, pr)  # noqa: E731
    else:
        step = lambda: ctx.symbfact(m, rp)  # noqa: E731
    for i in range(max(args.warmup, 1)):
        if i:
            flush.fill_(i & 0xff)
        step()

    def max_over_ranks(t):
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    dist.barrier()
    with ClockSampler(local) as clk:
        t_ms, rs = _device_timed(torch, stream, flush, args.steps, step)
    dist.barrier()
    t_max = max_over_ranks(t_ms)
    # assemble the whole factorization once (one sum-all-reduce over NCCL)
    full = distributed.symbfact_sharded(ctx, m, rank, world, distributed.torch_allreduce(), 0,
                                        params=_params(gsofa_b200, args), cuts=cuts)
    nnz_lu = full["nnz_lu"]
    value = args.steps * nnz_lu / (t_max / 1000.0)

    # end to end: upload from pinned host buffers, this rank's range (counts
    # and link flags to pinned buffers, lists to a pinned host pool), the NCCL
    # sum of the per-line arrays and the host supernode scan, every step
    pb = torch.from_numpy(g.beg).pin_memory()
    pe = torch.from_numpy(g.end).pin_memory()
    pa = torch.from_numpy(g.adj).pin_memory()
    allred = distributed.torch_allreduce()
    hpool = torch.empty(max(need, 1), dtype=torch.int32).pin_memory().numpy() if want_pattern else None

    def e2e_step():
        mm = ctx.upload(pb.numpy(), pe.numpy(), pa.numpy())
        if want_pattern:
            pp = distributed.rank_params(rank, world, cuts, _params(gsofa_b200, args))
            pp.want_pattern = 2
            r = ctx.symbfact_ranges(mm, hpool, pp)
        else:
            r = ctx.symbfact(mm, distributed.rank_params(rank, world, cuts, _params(gsofa_b200, args)))
        mm.free()
        return distributed.combine(g.n, r.u_row_count, r.l_col_count, r.line_flags, r.fill_count, allred)

    e2e_step()
    dist.barrier()
    te, outs = _device_timed(torch, stream, flush, args.steps, e2e_step)
    dist.barrier()
    te = max_over_ranks(te)
    assert outs[-1]["nnz_lu"] == nnz_lu
    parity = None
    if rank == 0:
        gold = None
        try:
            with open(os.path.join(ROOT, "tests", "golden", "large.json")) as f:
                gold = json.load(f).get(cfg["workload"])
        except (OSError, ValueError):
            gold = None
        if gold is not None:
            got = {"u_row_count": _sha(full["u_row_count"], "<i4"), "l_col_count": _sha(full["l_col_count"], "<i4"),
                   "line_flags": _sha(full["line_flags"], "u1"), "sn_start": _sha(full["sn_start"], "<i4")}
            bad = [k for k, v in got.items() if v != gold["sha256"][k]]
            bad += [k for k in ("fill_count", "nnz_lu") if int(full[k]) != int(gold[k])]
            parity = {"golden": "tests/golden/large.json", "mismatched": bad, "mismatches": len(bad)}
        line = {
            "metric": "nnz(L+U)/s", "value": value, "unit": "nnz/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int32", "data": "synthetic (seeded generator)",
            "config": dict(cfg, nnz_lu=int(nnz_lu), fill_count=int(full["fill_count"]),
                           supernodes=int(len(full["sn_start"])),
                           pattern="begin/end ranges into a device pool per rank" if want_pattern else "counts only",
                           l2="flushed between steps (256 MiB write)",
                           parallelism=f"one matrix in {world} contiguous work-predicted line ranges, "
                                       "one per rank; per-line arrays summed over NCCL"),
            "cuts": [int(c) for c in cuts], "predicted_work": [float(w) for w in pred],
            "factorizations_per_s": args.steps / (t_max / 1000.0),
            "e2e": {"value": args.steps * nnz_lu / (te / 1000.0), "unit": "nnz/s", "ms_per_step": te / args.steps,
                    "h2d_bytes_per_step": int((2 * g.n + g.nnz) * 4),
                    "d2h_bytes_per_step": int(4 * need + 12 * g.n + 16 * g.n * int(bool(want_pattern))),
                    "note": "per rank: its range's lists and per-line arrays; the NCCL sum is inside"},
            "parity": parity, "clocks": clk.summary(), "gpu_launches": args.steps,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    dist.destroy_process_group()
    return 1 if parity is not None and parity["mismatches"] else 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batch":
        return batch_main(args)
    if args.workload == "serve":
        return serve_main(args)
    if args.workload == "order":
        return order_main(args)

    import torch
    import torch.distributed as dist
    import gsofa_b200

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        return sharded_main(args, world, rank, local)

    g, cfg = workload(args)
    want_pattern = args.pattern if args.pattern >= 0 else int(args.workload != "circuit")
    form = args.form if want_pattern else "counts"
    ctx = gsofa_b200.Context(local)
    stream = torch.cuda.current_stream()
    ctx.set_stream(stream.cuda_stream)
    m = ctx.upload(g)
    nd = gsofa_b200.FLAG_NO_DOWNLOAD
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    # one counts-only run sizes the pattern pool exactly
    first = ctx.symbfact(m, _params(gsofa_b200, args, want_pattern=0, flags=nd))
    need = int(first.nnz_u + first.nnz_l)
    dpool = torch.empty(max(need, 1), dtype=torch.int32, device="cuda") if form == "ranges" else None
    if form == "ranges":
        params = _params(gsofa_b200, args, flags=nd)
        step = lambda: ctx.symbfact_ranges(m, dpool, params)  # noqa: E731
    else:
        params = _params(gsofa_b200, args, want_pattern=int(form == "csr"), flags=nd)
        step = lambda: ctx.symbfact(m, params)  # noqa: E731

    res = None
    # warm-up steps are timed steps untimed: the L2 flush runs too, so its
    # kernel is loaded before the timed region starts
    for i in range(max(args.warmup, 1)):
        if i:
            flush.fill_(i & 0xff)
        res = step()

    def barrier():
        if world > 1:
            dist.barrier()

    def max_over_ranks(t):
        if world == 1:
            return t
        tt = torch.tensor([t], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        return float(tt.item())

    # ---- device-resident timed region ------------------------------------
    barrier()
    with ClockSampler(local) as clk:
        t_ms, rs = _device_timed(torch, stream, flush, args.steps, step)
    barrier()
    kernel_ms = [r.kernel_ms for r in rs]
    t_max = max_over_ranks(t_ms)
    nnz_lu = res.nnz_lu
    value = world * args.steps * nnz_lu / (t_max / 1000.0)
    facts = world * args.steps / (t_max / 1000.0)

    # the other output forms of the same matrix, a few steps each (side numbers)
    forms = {}
    if want_pattern:
        k3 = max(1, min(args.steps, 5))
        for name, p in (("csr", _params(gsofa_b200, args, want_pattern=1, flags=nd)),
                        ("counts", _params(gsofa_b200, args, want_pattern=0, flags=nd))):
            if name == form:
                continue
            ctx.symbfact(m, p)
            tf, rf = _device_timed(torch, stream, flush, k3, lambda: ctx.symbfact(m, p))
            forms[name] = {"ms_per_step": tf / k3, "kernel_ms": statistics.mean(r.kernel_ms for r in rf),
                           "value": k3 * nnz_lu / (tf / 1000.0)}

    # the multi-GPU split measured on this device: the matrix as K contiguous
    # line ranges of equal predicted work, one launch each, back to back
    split = None
    if world == 1 and args.partitions > 1:
        cuts, pred = gsofa_b200.partition_lines(g, args.partitions)
        part_ms, part_nnz = [], 0
        for k in range(args.partitions):
            lo, hi = int(cuts[k]), int(cuts[k + 1])
            if form == "ranges":
                pk = _params(gsofa_b200, args, flags=nd, line_lo=lo, line_hi=hi)
                fn = lambda pk=pk: ctx.symbfact_ranges(m, dpool, pk)  # noqa: E731
            else:
                pk = _params(gsofa_b200, args, want_pattern=int(form == "csr"), flags=nd, line_lo=lo, line_hi=hi)
                fn = lambda pk=pk: ctx.symbfact(m, pk)  # noqa: E731
            fn()
            k3 = max(1, min(args.steps, 5))
            _, rk = _device_timed(torch, stream, flush, k3, fn)
            part_ms.append(statistics.mean(r.kernel_ms for r in rk))
            part_nnz += rk[-1].nnz_u + rk[-1].nnz_l
        full_ms = statistics.mean(kernel_ms)
        split = {"parts": args.partitions, "cuts": [int(c) for c in cuts], "predicted_work": [float(w) for w in pred],
                 "kernel_ms": part_ms, "summed_kernel_ms": sum(part_ms), "unsplit_kernel_ms": full_ms,
                 "summed_over_unsplit": sum(part_ms) / full_ms,
                 "slowest_over_mean": max(part_ms) / statistics.mean(part_ms),
                 "entries_match": bool(part_nnz == res.nnz_u + res.nnz_l)}

    # ---- end-to-end through the public API ----------------------------------
    e2e = None
    out = None
    if not args.no_e2e:
        pb = torch.from_numpy(g.beg).pin_memory()
        pe = torch.from_numpy(g.end).pin_memory()
        pa = torch.from_numpy(g.adj).pin_memory()
        n1 = g.n + 1

        def pinned(count, dt):
            return torch.empty(max(int(count), 1), dtype=dt).pin_memory().numpy()

        # page-locked result buffers, sized from the counts run, reused
        bufs = {"u_row_count": pinned(g.n, torch.int32), "l_col_count": pinned(g.n, torch.int32),
                "l_row_count": pinned(g.n, torch.int32), "sn_start": pinned(g.n, torch.int32)}
        if form == "ranges":
            # the lists stream into page-locked host memory while the
            # traversals run; per-line begins come back with the counts
            hpool = pinned(need, torch.int32)
            bufs.update(u_beg=pinned(g.n, torch.int64), l_beg=pinned(g.n, torch.int64))
            pe2e = _params(gsofa_b200, args)
            run = lambda mm: ctx.symbfact_ranges(mm, hpool, pe2e, out=bufs)  # noqa: E731
        else:
            if form == "csr":
                bufs.update(u_ptr=pinned(n1, torch.int64), l_ptr=pinned(n1, torch.int64),
                            u_idx=pinned(first.nnz_u, torch.int32), l_idx=pinned(first.nnz_l, torch.int32))
            pe2e = _params(gsofa_b200, args, want_pattern=int(form == "csr"))
            run = lambda mm: ctx.symbfact_into(mm, pe2e, bufs)  # noqa: E731
        for _ in range(2):   # warm the host-side allocations
            flush.fill_(1)
            mm = ctx.upload(pb.numpy(), pe.numpy(), pa.numpy())
            out = run(mm)
            mm.free()
        k2 = args.steps
        phases = {"upload_ms": 0.0, "factor_and_fetch_ms": 0.0, "free_ms": 0.0}

        def e2e_step():
            h0 = time.perf_counter()
            mm = ctx.upload(pb.numpy(), pe.numpy(), pa.numpy())
            h1 = time.perf_counter()
            o = run(mm)
            h2 = time.perf_counter()
            mm.free()
            h3 = time.perf_counter()
            phases["upload_ms"] += 1000 * (h1 - h0) / k2
            phases["factor_and_fetch_ms"] += 1000 * (h2 - h1) / k2
            phases["free_ms"] += 1000 * (h3 - h2) / k2
            return o

        barrier()
        te, outs = _device_timed(torch, stream, flush, k2, e2e_step)
        barrier()
        te = max_over_ranks(te)
        out = outs[-1]
        assert out.nnz_lu == nnz_lu and out.fill_count == res.fill_count
        h2d = (2 * g.n + g.nnz) * 4
        d2h = 3 * 4 * g.n + 4 * out.n_supernodes
        if form == "csr":
            d2h += 4 * (out.nnz_u + out.nnz_l) + 2 * 8 * n1
        elif form == "ranges":
            d2h += 4 * out.pool_used + 2 * 8 * g.n
        e2e = {"value": world * k2 * nnz_lu / (te / 1000.0), "unit": "nnz/s", "steps": k2,
               "ms_per_step": te / k2, "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
               "form": form, "host_phases": phases, "kernel_ms": out.kernel_ms,
               # the step moves d2h bytes over PCIe: their rate against the
               # host link's copy rate shows how close e2e is to its bound
               "d2h_gbs": d2h / (te / k2 / 1000.0) / 1e9, "d2h_link_gbs": link_gbs(torch, stream)}
        if want_pattern:
            # the same steps for a consumer of the supernodal structure: the
            # pattern stays on the device and only the per-supernode index
            # lists come back
            pcsr = _params(gsofa_b200, args)
            mm = ctx.upload(pb.numpy(), pe.numpy(), pa.numpy())
            _, sup = ctx.symbfact_supernodal(mm, pcsr)
            mm.free()
            snb = {k: torch.empty(max(getattr(sup, k).size, 1),
                                  dtype=torch.int64 if k in ("xlsub", "xusub") else torch.int32).pin_memory().numpy()
                   for k in ("xsup", "supno", "xlsub", "lsub", "xusub", "usub")}

            def sn_step():
                mm = ctx.upload(pb.numpy(), pe.numpy(), pa.numpy())
                o = ctx.symbfact_supernodal(mm, pcsr, out=snb)
                mm.free()
                return o

            ts, sns = _device_timed(torch, stream, flush, k2, sn_step)
            rs_, sup = sns[-1]
            assert rs_.nnz_lu == nnz_lu and sup.nsuper == res.n_supernodes
            d2h_sn = sum(int(getattr(sup, k).nbytes) for k in ("xsup", "supno", "xlsub", "lsub", "xusub", "usub"))
            e2e["supernodal"] = {"value": world * k2 * nnz_lu / (ts / 1000.0), "unit": "nnz/s",
                                 "ms_per_step": ts / k2, "h2d_bytes_per_step": int(h2d),
                                 "d2h_bytes_per_step": d2h_sn, "lsub": int(sup.lsub.size),
                                 "usub": int(sup.usub.size)}

    # ---- roofline of the factorization kernel --------------------------------
    # Algorithmic bytes follow the per-source traversal model: every source
    # expands all of X(s).  With reuse the kernel expands fewer vertices, so
    # the model's |X| and E_insp come from one untimed run without reuse.
    ideal = res
    if args.reuse != 0:
        ideal = ctx.symbfact(m, _params(gsofa_b200, args, want_pattern=0, flags=nd, reuse=0, src_chunk=0))
        assert ideal.nnz_lu == nnz_lu
    peak, peak_kind = hbm_peak()
    kms = statistics.mean(kernel_ms)
    n = g.n
    b_alg = 8 * ideal.x_total + 8 * ideal.e_insp + (4 * nnz_lu if want_pattern else 0) + 8 * n
    achieved = b_alg / (kms / 1000.0) / 1e9
    traffic = traffic_per_launch(cfg["workload"], form)
    # the same byte model over the work this kernel actually did (expansions of
    # both passes, edges it inspected): how close the traversal it runs comes
    # to the bandwidth bound, as opposed to the per-source model above
    b_act = 8 * 2 * res.x_total + 8 * res.edges_inspected + (4 * nnz_lu if want_pattern else 0) + 8 * n
    roof = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak, "traffic": traffic, "peak_kind": peak_kind,
            "actual_work_bytes": int(b_act), "frac_of_actual_work": b_act / (kms / 1000.0) / 1e9 / peak,
            "algorithmic_bytes": int(b_alg), "kernel_ms": kms, "x_total": ideal.x_total,
            "e_insp": ideal.e_insp, "edges_inspected": res.edges_inspected,
            "edges_inspected_without_reuse": ideal.edges_inspected,
            "work_ratio": res.edges_inspected / max(ideal.edges_inspected, 1),
            "levels": res.levels, "reused_sources": res.reused_sources, "sources": res.sources,
            "cycles": dict(zip(("seed", "levels", "fold", "count", "lists", "clear", "pair_wait"),
                               res.cycles)), "ctas": res.ctas}

    batched = None
    if world == 1 and args.batch_count > 0 and args.workload == "nd3d":
        batched = batched_vs_plain(args, ctx, torch, stream, gsofa_b200)
    serving = None
    if world == 1 and args.workload == "nd3d" and args.serve_default > 0:
        # a short serving stream beside the headline line (the 10,000-request
        # stream is its own run: --workload serve --serve-count 10000)
        serving = serving_run(ctx, args.serve_default, 200_000, args.serve_default_rate,
                              min(args.serve_default, 120))
    streamed = None
    if world == 1 and args.workload == "circuit" and args.host_pool_gb > 0:
        streamed = streamed_pattern(args, ctx, m, torch, gsofa_b200, g)

    cpu = None
    parity = None
    if rank == 0:
        # the oracle on a strided sample of the lines: timed as the CPU
        # baseline, and its per-line results checked against the GPU's
        cs = cpu_sample(g, args.cpu_seconds, extras=(world == 1))
        if world == 1 and not args.no_cpu_baseline:
            cpu = cpu_baseline_obj(cs)
        chk = out
        if chk is None:
            chk = ctx.symbfact(m, _params(gsofa_b200, args, want_pattern=int(want_pattern != 0)))
        parity = check_parity(g, cfg["workload"], chk, cs, want_pattern)

    if rank == 0:
        line = {
            "metric": "nnz(L+U)/s", "value": value, "unit": "nnz/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t_max / args.steps,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int32",
            "data": "synthetic (seeded generator)",
            "config": dict(cfg, nnz_lu=int(nnz_lu), fill_count=int(res.fill_count),
                           supernodes=int(res.n_supernodes),
                           pattern={"ranges": "begin/end ranges into a device pool", "csr": "CSR on the device",
                                    "counts": "counts only"}[form],
                           state=args.state, reuse=args.reuse, l2="flushed between steps (256 MiB write)",
                           parallelism=("one matrix on one GPU (--gpus N splits it into N contiguous "
                                        "work-predicted line ranges)" if world == 1 else
                                        f"independent factorization per rank x{world}")),
            "factorizations_per_s": facts,
            "other_forms": forms,
            "split_on_one_gpu": split,
            "batched": batched,
            "pattern_streamed_to_host": streamed,
            "serving": serving,
            "e2e": e2e,
            "roofline": roof,
            "cpu_baseline": cpu,
            "parity": parity,
            "clocks": clk.summary(),
            "gpu_launches": args.steps,
        }
        print(json.dumps(line), flush=True)
    ctx.close()
    if world > 1:
        dist.destroy_process_group()
    if parity is not None and parity["mismatches"]:
        print(f"parity check failed: {parity}", file=sys.stderr)
        return 1
    if streamed is not None and streamed["mismatches"]:
        print(f"streamed pattern check failed: {streamed}", file=sys.stderr)
        return 1
    return 0


if __name__ == "__main__":
    sys.exit(main())
