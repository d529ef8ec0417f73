#!/usr/bin/env python
"""Benchmark of the dielectric BIE hot path on B200.

Workload (default `cfg3`): box 1.5 x 1.0 x 0.8, n_quad = 6, l_ec = 0.08,
eps_in = 4, eps_out = 1 (N = 42,048 nodes, near-field corrections at
up_tol = 1e-9, max_order = 8). One step = one block solve of k = 64 point-source
right-hand sides (positions uniform in the box interior, charges ~ N(0, 1),
seeded) to a relative residual of 1e-10: RHS assembly on the device + the
refined solver (split-BF16 three-term tensor-core direct sum, FP64 corrections,
FP64 Krylov and iterative refinement). The same steps are also timed on the
plain FP64 GPU path for the comparison the metric names.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload cfg3]

Under torchrun (N > 1) every rank solves its own request stream on its own GPU
(replicas; no collective on the data path): value = all ranks' solves / the
slowest rank's time. `--impl reference` times the CPU restatement of the
reference's path (oracle/, C + OpenMP on all host cores) on the same workload.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG_DIR = os.path.join(ROOT, "dielectricbie.jl_b200")
METRIC = "solves/s + p50/p99 latency at 1e-8 rel σ err: refined/batched vs plain FP64 GPU"

WORKLOADS = {
    "cfg3": dict(box=(1.5, 1.0, 0.8), nq=6, l_ec=0.08, eps_in=4.0, eps_out=1.0, k=64, seed=3, rtol=1e-10,
                 up_tol=1e-9, max_order=8, probes=1000, charges="normal"),
    "cfg2": dict(box=(2.0, 1.0, 1.0), nq=6, l_ec=0.05, eps_in=10.0, eps_out=1.0, k=8, seed=2, rtol=1e-10,
                 up_tol=1e-9, max_order=8, probes=0, charges="pm1", inner=0.8),
    "cfg1": dict(box=(1.2, 0.8, 0.6), nq=4, l_ec=0.2, eps_in=4.0, eps_out=1.0, k=1, seed=1, rtol=1e-12,
                 up_tol=1e-9, max_order=8, probes=0, charges="one"),
    # serving stream of uneven geometries (sides U[0.5, 2], eps_in log-U[2, 80], n_quad 4 or 6, node
    # counts log-U[n_min, n_max], geometry repeats with p = 0.5, 1-32 point sources per request)
    "cfg4": dict(requests=2000, n_min=2000, n_max=200000, repeat=0.5, rate=20.0, seed=4, rtol=1e-8,
                 up_tol=1e-9, max_order=8, k=0, restart=60, resident_fraction=0.45, builders=2),
}

# lattice of 4 x 4 x 2 cubes (side 0.5, gap 0.2), 16 sources at cell-corner centres between cubes
WORKLOADS["cfg5"] = dict(lattice=(4, 4, 2), side=0.5, gap=0.2, nq=6, l_ec=0.05, eps_in=4.0, eps_out=1.0, k=16,
                         seed=5, rtol=1e-8, up_tol=1e-9, max_order=8)

# serving stream: single-source requests spread over three resident geometries (the cfg3
# box and two other boxes), Poisson arrivals
SERVE_STREAM = dict(requests=1024, rate=1500.0, repeats=2,
                    extra_boxes=[(1.2, 1.0, 0.6, 6, 0.08, 10.0, 1.0), (1.0, 1.0, 0.5, 4, 0.06, 20.0, 1.0)])


def load_package():
    name = "dielectricbie_jl_b200"
    if name in sys.modules:
        return sys.modules[name]
    sys.path.insert(0, PKG_DIR)
    import build as pkg_build  # in-tree build of libbie_b200.so (no-op when up to date)
    pkg_build.build()
    spec = importlib.util.spec_from_file_location(name, os.path.join(PKG_DIR, "__init__.py"),
                                                  submodule_search_locations=[PKG_DIR])
    mod = importlib.util.module_from_spec(spec)
    sys.modules[name] = mod
    spec.loader.exec_module(mod)
    return mod


def make_sources(wl, nbatch, k):
    """Point sources uniform in the box interior (inner fraction `inner`), charges per workload."""
    rng = np.random.default_rng(wl["seed"])
    half = np.array(wl["box"]) / 2 * wl.get("inner", 0.9)
    out = []
    for _ in range(nbatch):
        pos = rng.uniform(-half, half, size=(k, 3))
        if wl["charges"] == "normal":
            q = rng.standard_normal(k)
        elif wl["charges"] == "pm1":
            q = rng.choice([-1.0, 1.0], size=k)
        else:
            q = np.ones(k)
        out.append((np.ascontiguousarray(pos), np.ascontiguousarray(q)))
    return out


def make_probes(bie, itf, m, seed):
    """Exterior probes: a random surface node pushed 0.1-0.5 along its outward normal."""
    rng = np.random.default_rng(seed)
    idx = rng.integers(0, itf.n, size=m)
    d = rng.uniform(0.1, 0.5, size=m)
    return np.ascontiguousarray(itf.points[idx] + itf.normals[idx] * d[:, None])


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except (OSError, FileNotFoundError):
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 8:
                continue
            try:
                sm.append(float(parts[0]))
                mx = float(parts[1])
            except ValueError:
                continue
            for nm, v in zip(names, parts[4:8]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


class CpuReference:
    """CPU restatement of the reference path (oracle: FP64 direct sum + CSC near
    corrections + GMRES, C/OpenMP on all host cores), built once per workload."""

    def __init__(self, wl, threads=0):
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import oracle as orc
        orc.build()
        self.orc, self.wl, self.threads = orc, wl, threads or os.cpu_count()
        self.m = orc.Mesh.single_box(*wl["box"], wl["nq"], wl["l_ec"], wl["eps_in"], wl["eps_out"])
        ups, adp = orc.build_neighbor_list(self.m, wl["max_order"], wl["up_tol"], True)
        self.C = orc.DT_corrections(self.m, ups, adp, wl["up_tol"], nthreads=self.threads)
        self.sources = make_sources(wl, 64, 1)

    def solve(self, step, max_seconds=30.0):
        """One right-hand side (a different seeded source per step), GMRES to the
        workload's rtol; bounded to about max_seconds (then not converged)."""
        orc, wl, m = self.orc, self.wl, self.m
        pos, q = self.sources[step % len(self.sources)]
        b = orc.rhs_point(m.pts, m.nrm, pos[0], q[0], wl["eps_in"])
        t0 = time.perf_counter()
        orc.op_apply(m, b, self.C, nthreads=self.threads)
        t_mv = time.perf_counter() - t0
        itmax = max(2, int(max_seconds / max(t_mv, 1e-6)))
        t0 = time.perf_counter()
        x, it, res = orc.gmres(m, b, self.C, atol=0.0, rtol=wl["rtol"], itmax=itmax, nthreads=self.threads)
        t = time.perf_counter() - t0
        converged = res <= wl["rtol"] * np.linalg.norm(b) * (1 + 1e-9)
        return dict(seconds=t, iterations=it, converged=bool(converged), matvec_s=t_mv, n=m.n, cores=self.threads)


def run_reference_arm(args, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if "box" not in wl:
        print(json.dumps({"impl": "reference", "unavailable": f"the CPU arm times single-geometry workloads; "
                                                               f"{args.workload} is a multi-geometry stream"}))
        return 0
    ref = CpuReference(wl)
    times, info = [], None
    for step in range(args.warmup + args.steps):
        info = ref.solve(step)
        if step >= args.warmup:
            times.append(info["seconds"])
    per_solve = float(np.mean(times))
    value = 1.0 / per_solve
    sample = (f"one RHS column of the {args.workload} workload per step (a different seeded point source each "
              f"step): oracle FP64 direct sum + CSC near corrections + GMRES (rtol {wl['rtol']:g}), N={info['n']}, "
              f"{info['iterations']} iterations{'' if info['converged'] else ' (time-bounded, not converged)'}")
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": per_solve * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded point sources)",
            "config": workload_config(args.workload, wl, info["n"]),
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": info["cores"], "kind": "port",
                             "sample": sample},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def max_over_ranks(dist, values, device=None):
    """Element-wise maximum of per-rank timings over the process group (the
    slowest replica sets the job's time). Device tensors for NCCL, host tensors
    for gloo."""
    import torch
    on_dev = dist.get_backend() == "nccl"
    t = torch.tensor(values, dtype=torch.float64, device=(f"cuda:{device}" if on_dev else "cpu"))
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.cpu()]


def replica_value(per_rank_units, world, time_ms):
    """Whole-job throughput of independent replicas: all ranks' units over the
    slowest rank's time."""
    return per_rank_units * world / (time_ms * 1e-3)


def profiled_traffic(name):
    """DRAM bytes (read + written) per launch of a kernel, from the ncu summary
    committed under profiles/ (its `dram_bytes_per_launch:` line); None if absent."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None
    import re
    m = re.search(r"dram_bytes_per_launch:\s*([0-9.eE+]+)", open(path).read())
    return float(m.group(1)) if m else None


def poisson_arrivals(rng, count, rate):
    return np.cumsum(rng.exponential(1.0 / rate, size=count)) - 0.0


def rhs_columns(rhs):
    """Columns of a request's right-hand side: an N x k block, or ("point", sources, eps_src)."""
    return len(rhs[1]) if isinstance(rhs, tuple) else rhs.shape[1]


def serve_stream(bie, requests, precision, rtol, slots=4, batch=128, restart=200, block=False):
    """Serves `requests` = [(op, rhs, arrival_s)] through the library's request server
    (continuous batching), submitting each at its arrival time from a separate thread; rhs is
    an N x k block or ("point", sources, eps_src) (bie_server_submit_point: only the sources
    are queued, the right-hand sides are built on the device). Latency = completion -
    arrival; throughput = RHS columns / (last completion - first arrival). block: the merged
    batches are solved by block GMRES."""
    srv = bie.SolveServer(max_slots=slots, max_batch_rhs=batch)
    nreq = len(requests)
    tickets, sub_t = [None] * nreq, [0.0] * nreq
    ready = [threading.Event() for _ in range(nreq)]
    t0 = time.perf_counter() + 0.01

    def submitter():
        for i, (op, rhs, arr) in enumerate(requests):
            dt = t0 + arr - time.perf_counter()
            if dt > 0:
                time.sleep(dt)
            sub_t[i] = time.perf_counter()
            if isinstance(rhs, tuple):
                tickets[i] = srv.submit_sources(op, rhs[1], rhs[2], rtol=rtol, precision=precision, restart=restart,
                                                block=block)
            else:
                tickets[i] = srv.submit(op, rhs, rtol=rtol, precision=precision, restart=restart, block=block)
            ready[i].set()

    th = threading.Thread(target=submitter)
    th.start()
    lat, done, cols, unsolved = [], [], 0, 0
    for i in range(nreq):
        ready[i].wait()
        _, st, l_ms = srv.result(tickets[i], sigma=False)
        t_done = sub_t[i] + l_ms * 1e-3
        done.append(t_done)
        lat.append((t_done - (t0 + requests[i][2])) * 1e3)
        cols += rhs_columns(requests[i][1])
        unsolved += int(not st.solved)
    th.join()
    cnt = srv.counters()
    srv.close()
    span = max(done) - (t0 + requests[0][2])
    # batch composition: the requests of one batch complete together
    order = np.argsort(done)
    widths, last = [], None
    for i in order:
        if last is None or done[i] - last > 5e-4:
            widths.append(0)
        widths[-1] += rhs_columns(requests[i][1])
        last = done[i]
    return {"solves_per_s": cols / span, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "makespan_s": span, "requests": nreq, "solves": cols,
            "unconverged_requests": unsolved, "batches": cnt["batches"], "merged_requests": cnt["merged_requests"],
            "batch_columns": widths if len(widths) <= 64 else f"{len(widths)} completion groups",
            "peak_inflight": cnt["peak_inflight"], "hbm_peak_bytes": cnt["hbm_peak"],
            "workspace_releases": cnt["workspace_releases"], "enomem_retries": cnt["enomem_retries"],
            "group_solves": cnt["groups"], "grouped_batches": cnt["grouped_batches"]}


def plain_sequential(bie, requests, rtol, restart=200):
    """The plain FP64 GPU path one request at a time in arrival order (a request starts when
    it has arrived and the previous one is done); same host API as the server's requests
    (point-source requests through bie_solve_point, blocks through bie_solve)."""
    t_free, lat, cols = 0.0, [], 0
    for op, rhs, arr in requests:
        start = max(arr, t_free)
        t1 = time.perf_counter()
        if isinstance(rhs, tuple):
            bie.gpu_solve_sources(op, rhs[1], rhs[2], rtol=rtol, precision="fp64", restart=restart)
        else:
            bie.gpu_solve(op, rhs, rtol=rtol, precision="fp64", restart=restart)
        t_free = start + (time.perf_counter() - t1)
        lat.append((t_free - arr) * 1e3)
        cols += rhs_columns(rhs)
    span = t_free - requests[0][2]
    return {"solves_per_s": cols / span, "p50_ms": float(np.percentile(lat, 50)),
            "p99_ms": float(np.percentile(lat, 99)), "makespan_s": span, "requests": len(requests), "solves": cols}


def request_stream(bie, itf, op, wl, precision, device, block=False):
    """Single-point-source requests over three resident geometries (the workload's box and
    two other boxes of 23k-24k nodes, their correction blocks on the device), Poisson
    arrivals (seeded). Untimed warm-up first, as warm-up steps precede the block solves: one
    full-width (128-column) batch per geometry, then a warm-up stream (another seed); they meet
    the batch widths' first-use costs (launch-shape tuning per kernel instance, workspace
    growth, graph capture). The timed stream is served
    `repeats` times (the spread of the figures between the runs is reported), then solved
    by the plain FP64 path one request at a time."""
    cnt, rate = SERVE_STREAM["requests"], SERVE_STREAM["rate"]
    geoms = [(itf, op, wl["eps_in"], np.array(wl["box"]) / 2 * 0.9)]
    for b in SERVE_STREAM["extra_boxes"]:
        it2 = bie.single_dielectric_box3d(*b)
        op2 = bie.lhs_dielectric_box3d_fmm3d_corrected(it2, 1e-12, wl["up_tol"], wl["max_order"], precision=precision,
                                                       device=device, keep_host_blocks=False)
        geoms.append((it2, op2, b[5], np.array(b[:3]) / 2 * 0.9))

    def stream(seed):
        rng = np.random.default_rng(seed)
        arr = poisson_arrivals(rng, cnt, rate)
        reqs = []
        for i in range(cnt):
            g_itf, g_op, eps, half = geoms[int(rng.integers(len(geoms)))]
            src = bie.PointSource(tuple(rng.uniform(-half, half)), float(rng.standard_normal()))
            reqs.append((g_op, ("point", [src], eps), float(arr[i])))
        return reqs

    # untimed: a full-width batch (the server's 128 columns) per geometry, so that the widest
    # kernel instance's tuning and workspace are in place whatever widths the warm-up stream's
    # timing produces; then the warm-up stream
    rng_w = np.random.default_rng(wl["seed"] + 98)
    with bie.SolveServer(max_slots=1, max_batch_rhs=128) as srv:
        for g_itf, g_op, eps, half in geoms:
            src = [bie.PointSource(tuple(rng_w.uniform(-half, half)), float(rng_w.standard_normal()))
                   for _ in range(128)]
            srv.result(srv.submit_sources(g_op, src, eps, rtol=wl["rtol"], precision=precision, restart=200,
                                          block=block), sigma=False)
    serve_stream(bie, stream(wl["seed"] + 99), precision, wl["rtol"], block=block)
    reqs = stream(wl["seed"] + 100)
    runs = [serve_stream(bie, reqs, precision, wl["rtol"], block=block) for _ in range(SERVE_STREAM["repeats"])]
    plain = plain_sequential(bie, reqs, wl["rtol"])
    sps = [r["solves_per_s"] for r in runs]
    served = dict(runs[0])
    served["repeats"] = [{k: r[k] for k in ("solves_per_s", "p50_ms", "p99_ms", "makespan_s", "peak_inflight",
                                            "batches")} for r in runs]
    served["solves_per_s_spread"] = (max(sps) - min(sps)) / max(sps)
    return {"workload": f"request stream: {cnt} single-source requests over {len(geoms)} resident geometries "
                        f"(N = {', '.join(str(g[0].n) for g in geoms)}), Poisson arrivals at {rate:g}/s (seeded), "
                        f"rtol {wl['rtol']:g}, after one untimed warm-up stream; served {len(runs)} times",
            "served_krylov": "block GMRES per merged batch" if block else "GMRES, one Arnoldi process per column",
            "refined_served": served, "plain_fp64_sequential": plain,
            "speedup_solves_per_s": served["solves_per_s"] / plain["solves_per_s"]}


def box_for_nodes(bie, sides, nq, eps_in, target):
    """l_ec by bisection on the mesher so that the box has about `target` nodes (the value
    used is kept on the interface as l_ec_used)."""
    lo, hi = 1e-3, 2.0 * max(sides)
    best = None
    for _ in range(30):
        mid = math.sqrt(lo * hi)
        itf = bie.single_dielectric_box3d(*sides, nq, mid, eps_in, 1.0)
        itf.l_ec_used = mid
        if best is None or abs(math.log(itf.n / target)) < abs(math.log(best.n / target)):
            best = itf
        if itf.n > target:
            lo = mid
        else:
            hi = mid
        if hi / lo < 1.01:
            break
    return best


class GeometryCache:
    """Resident geometries (mesh + near-field blocks on the device, host copy of the blocks
    released) under a device-memory budget. A request's geometry is built when first needed
    (its set-up time falls on that request); least recently used geometries without pending
    requests are destroyed to make room and built again when a later request repeats them.
    Thread-safe: builder threads build and pin (a geometry requested while it is being built
    waits for that build), the polling thread unpins."""

    def __init__(self, bie, wl, device, budget_bytes, nthreads=0):
        import collections
        self.bie, self.wl, self.device, self.budget, self.nthreads = bie, wl, device, budget_bytes, nthreads
        self.live = collections.OrderedDict()  # key -> (itf, op, bytes)
        self.building = {}                     # key -> Event set when its build ends
        self.lec = {}                          # key -> l_ec found by the first build
        self.pins = collections.Counter()
        self.lock = threading.Lock()
        self.used = self.peak = 0
        self.builds = self.rebuilds = self.evictions = 0
        self.setup = []  # (nodes, seconds, rebuild)

    def _evict_for(self, need):
        while self.used + need > self.budget:
            victim = next((k for k in self.live if self.pins[k] == 0), None)
            if victim is None:
                return
            itf, op, b = self.live.pop(victim)
            for gm in list(itf._geoms.values()):
                gm.close()
            itf._geoms.clear()
            self.used -= b
            self.evictions += 1

    def get(self, key, spec):
        """(itf, op) of the request's geometry, built if it is not resident; pins it."""
        while True:
            with self.lock:
                if key in self.live:
                    self.live.move_to_end(key)
                    self.pins[key] += 1
                    return self.live[key][:2]
                ev = self.building.get(key)
                if ev is None:  # this thread builds it
                    ev = self.building[key] = threading.Event()
                    break
            ev.wait()  # another thread is building it
        try:
            return self._build(key, spec)
        finally:
            with self.lock:
                del self.building[key]
            ev.set()

    def resident(self, key):
        with self.lock:
            return key in self.live

    def _build(self, key, spec):
        import ctypes as C
        import torch
        from dielectricbie_jl_b200 import _abi
        sides, nq, eps_in, target = spec
        t1 = time.perf_counter()
        if key in self.lec:
            itf = self.bie.single_dielectric_box3d(*sides, nq, self.lec[key], eps_in, 1.0)
        else:
            itf = box_for_nodes(self.bie, sides, nq, eps_in, target)
        # room for this geometry's blocks, reserved before the build so that concurrent builders
        # do not all claim the same free budget (the set-up's transient device memory included)
        reserve = int(1.25 * self.live_estimate(itf))
        with self.lock:
            self._evict_for(reserve)
            self.used += reserve
        # and room on the device beside the solves in flight: a build waits (at most 60 s) until
        # its reservation and a margin are free, so that it does not take the memory of batches
        # the server has admitted
        t_gate = time.perf_counter()
        while time.perf_counter() - t_gate < 60.0:
            free, _ = torch.cuda.mem_get_info(self.device)
            if free >= reserve + (8 << 30):
                break
            time.sleep(0.05)
        try:
            op = self.bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, self.wl["up_tol"], self.wl["max_order"],
                                                               device=self.device, keep_host_blocks=False,
                                                               nthreads=self.nthreads)
            n, nb, b = C.c_int64(), C.c_int64(), C.c_size_t()
            _abi.check(_abi.lib().bie_geom_info(op.geom._h, C.byref(n), C.byref(nb), C.byref(b)))
        finally:
            with self.lock:
                self.used -= reserve
        dt = time.perf_counter() - t1
        with self.lock:
            rebuild = key in self.lec
            if not rebuild:
                self.lec[key] = itf.l_ec_used
            self.setup.append((itf.n, dt, rebuild))
            self.builds += 1
            self.rebuilds += int(rebuild)
            self.live[key] = (itf, op, b.value)
            self.used += b.value
            self.peak = max(self.peak, self.used)
            self.pins[key] += 1
            return itf, op

    def live_estimate(self, itf):
        # blocks of nq^4 doubles; about 48 source-target pairs per panel at n_quad 4 and 8 at 6
        # (up_tol 1e-9), plus the node arrays
        per_panel = 48 if itf.n_quad == 4 else 8
        return itf.npanels * per_panel * itf.n_quad ** 4 * 8 + itf.n * 80

    def unpin(self, key):
        with self.lock:
            self.pins[key] -= 1


def run_serving_workload(args, wl, bie, device):
    """`--workload cfg4`: the uneven serving stream; served refined solver vs the plain FP64
    path one request at a time. Requests carry their point sources only (the right-hand
    sides are built on the device). Geometries are built when a request first needs them and
    kept resident (correction blocks on the device only) under a device-memory budget: all
    distinct geometries of the stream need about 170 GB of blocks, more than fits beside the
    solver workspaces, so the least recently used idle geometries are destroyed and built
    again when repeated. Set-up time is on the request path of both arms."""
    import resource
    import torch
    rng = np.random.default_rng(wl["seed"])
    specs, reqs = [], []
    arr = poisson_arrivals(rng, wl["requests"], wl["rate"])
    for i in range(wl["requests"]):
        if specs and rng.random() < wl["repeat"]:
            key = int(rng.integers(len(specs)))
        else:
            sides = tuple(float(v) for v in rng.uniform(0.5, 2.0, size=3))
            eps_in = float(math.exp(rng.uniform(math.log(2.0), math.log(80.0))))
            nq = int(rng.choice([4, 6]))
            target = math.exp(rng.uniform(math.log(wl["n_min"]), math.log(wl["n_max"])))
            specs.append((sides, nq, eps_in, target))
            key = len(specs) - 1
        k = int(rng.integers(1, 33))
        half = 0.45 * np.array(specs[key][0])
        src = [bie.PointSource(tuple(rng.uniform(-half, half)), float(rng.standard_normal())) for _ in range(k)]
        reqs.append((key, src, float(arr[i])))
    total = torch.cuda.get_device_properties(device).total_memory
    budget = int(wl["resident_fraction"] * total)

    builders = wl["builders"]

    def run_arm(served):
        # the served arm builds new geometries on a pool of threads (each with its share of
        # the host cores), so requests on resident geometries are not held behind set-up; the
        # plain arm does everything in turn
        cache = GeometryCache(bie, wl, device, budget,
                              nthreads=max(2, (os.cpu_count() or 8) // builders) if served else 0)
        nreq = len(reqs)
        lat, done, cols, unsolved = [0.0] * nreq, [0.0] * nreq, 0, 0
        t0 = time.perf_counter() + 0.01
        failed = []
        if served:
            # the server's workspace budget: the device memory the resident geometries leave
            srv = bie.SolveServer(max_slots=4, max_batch_rhs=128, hbm_fraction=max(0.1, 0.7 - wl["resident_fraction"]))
            tickets = [None] * nreq
            sub_t = [0.0] * nreq
            ready = [threading.Event() for _ in range(nreq)]

            def submit_one(i):
                key, src, a = reqs[i]
                try:
                    itf, op = cache.get(key, specs[key])
                    sub_t[i] = time.perf_counter()
                    tickets[i] = srv.submit_sources(op, src, specs[key][2], rtol=wl["rtol"],
                                                    precision=args.precision, restart=wl["restart"])
                except Exception as e:  # recorded; the stream goes on
                    failed.append((i, repr(e)))
                ready[i].set()

            from concurrent.futures import ThreadPoolExecutor
            pool = ThreadPoolExecutor(max_workers=builders)

            def submitter():
                for i, (key, src, a) in enumerate(reqs):
                    dt = t0 + a - time.perf_counter()
                    if dt > 0:
                        time.sleep(dt)
                    if cache.resident(key):
                        submit_one(i)
                    else:
                        pool.submit(submit_one, i)

            th = threading.Thread(target=submitter)
            th.start()
            for i in range(nreq):
                ready[i].wait()
                if tickets[i] is None:
                    done[i] = time.perf_counter()
                    lat[i] = (done[i] - (t0 + reqs[i][2])) * 1e3
                    continue
                _, st, l_ms = srv.result(tickets[i], sigma=False)
                cache.unpin(reqs[i][0])
                done[i] = sub_t[i] + l_ms * 1e-3
                lat[i] = (done[i] - (t0 + reqs[i][2])) * 1e3
                unsolved += int(not st.solved)
            th.join()
            pool.shutdown()
            cnt = srv.counters()
            srv.close()
        else:
            t_free = t0
            for i, (key, src, a) in enumerate(reqs):
                t_free = max(t_free, t0 + a)
                now = time.perf_counter()
                if now < t_free:
                    time.sleep(t_free - now)
                try:
                    itf, op = cache.get(key, specs[key])
                    _, st = bie.gpu_solve_sources(op, src, specs[key][2], rtol=wl["rtol"], precision="fp64",
                                                  restart=wl["restart"])
                    cache.unpin(key)
                    unsolved += int(not st.solved)
                except Exception as e:  # recorded; the stream goes on
                    failed.append((i, repr(e)))
                t_free = time.perf_counter()
                done[i] = t_free
                lat[i] = (t_free - (t0 + a)) * 1e3
            cnt = None
        bad = {i for i, _ in failed}
        cols = sum(len(src) for i, (_, src, _) in enumerate(reqs) if i not in bad)
        span = max(done) - (t0 + reqs[0][2])
        su = np.array([(n, t) for n, t, _ in cache.setup])
        out = {"solves_per_s": cols / span, "p50_ms": float(np.percentile(lat, 50)),
               "p99_ms": float(np.percentile(lat, 99)), "makespan_s": span, "requests": nreq, "solves": cols,
               "unconverged_requests": unsolved, "failed_requests": len(failed),
               "first_failures": failed[:3],
               "geometry_builds": cache.builds, "geometry_rebuilds": cache.rebuilds,
               "geometry_evictions": cache.evictions, "resident_peak_gb": cache.peak / 1e9,
               "setup_s_total": float(su[:, 1].sum()), "setup_s_median": float(np.median(su[:, 1])),
               "setup_s_max": float(su[:, 1].max()), "setup_s_at_max_nodes": float(su[np.argmax(su[:, 0]), 1])}
        if cnt is not None:
            out.update({"batches": cnt["batches"], "merged_requests": cnt["merged_requests"],
                        "peak_inflight": cnt["peak_inflight"], "group_solves": cnt["groups"],
                        "grouped_batches": cnt["grouped_batches"], "workspace_releases": cnt["workspace_releases"],
                        "enomem_retries": cnt["enomem_retries"], "hbm_peak_bytes": cnt["hbm_peak"]})
        for key, (itf, op, b) in list(cache.live.items()):
            for gm in list(itf._geoms.values()):
                gm.close()
        return out

    served = run_arm(True)
    plain = run_arm(False)
    line = {"metric": METRIC, "value": served["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
            "steps": wl["requests"], "warmup": 0, "ms_per_step": served["makespan_s"] * 1e3 / wl["requests"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"{args.precision} tensor-core direct sum + fp64",
            "data": "synthetic (seeded boxes and point sources, Poisson arrivals)",
            "config": {"workload": f"cfg4 serving stream: {wl['requests']} requests, node counts log-uniform "
                                   f"in [{wl['n_min']}, {wl['n_max']}], {len(specs)} distinct geometries "
                                   f"(repeat p = {wl['repeat']}), 1-32 point sources each, Poisson arrivals "
                                   f"{wl['rate']:g}/s, rtol {wl['rtol']:g}, Krylov restart {wl['restart']}",
                       "geometries": len(specs),
                       "geometry_residency": f"built on first use, least recently used idle geometries destroyed "
                                             f"above {wl['resident_fraction']:.0%} of device memory and rebuilt "
                                             f"when repeated; set-up on the request path of both arms (served: "
                                             f"{builders} builder threads; plain: in turn)",
                       "host_peak_rss_gb": resource.getrusage(resource.RUSAGE_SELF).ru_maxrss / 2**20},
            "p50_ms": served["p50_ms"], "p99_ms": served["p99_ms"],
            "refined_served": served, "plain_fp64_sequential": plain,
            "speedup_vs_plain_fp64": served["solves_per_s"] / plain["solves_per_s"]}
    print(json.dumps(line), flush=True)
    return 0


def run_lattice_workload(args, wl, bie, device):
    """`--workload cfg5`: one solve of 16 right-hand sides on the cube lattice. The refined
    solver runs to rtol 1e-8; the plain FP64 path runs to rtol 1e-10 as the accuracy
    reference. Reports time per GMRES iteration (device time on the solver's stream),
    iteration counts, the sigma error and the tensor-core kernel's FP32-issue fraction."""
    import ctypes as C
    import torch
    from dielectricbie_jl_b200 import _abi
    L = _abi.lib()
    nx, ny, nz = wl["lattice"]
    pitch = wl["side"] + wl["gap"]
    boxes = [{"center": ((i - (nx - 1) / 2) * pitch, (j - (ny - 1) / 2) * pitch, (l - (nz - 1) / 2) * pitch),
              "Lx": wl["side"], "Ly": wl["side"], "Lz": wl["side"]}
             for i in range(nx) for j in range(ny) for l in range(nz)]
    t0 = time.perf_counter()
    itf = bie.multi_dielectric_box3d(wl["nq"], wl["l_ec"], boxes, [wl["eps_in"]] * len(boxes), wl["eps_out"])
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, wl["up_tol"], wl["max_order"], device=device)
    setup_s = time.perf_counter() - t0
    rng = np.random.default_rng(wl["seed"])
    corners = [((i - (nx - 2) / 2) * pitch, (j - (ny - 2) / 2) * pitch, (l - (nz - 2) / 2) * pitch)
               for i in range(nx - 1) for j in range(ny - 1) for l in range(max(nz - 1, 1))]
    pick = rng.integers(len(corners), size=wl["k"])
    jit = rng.uniform(-0.05, 0.05, size=(wl["k"], 3))  # stays inside the 0.2-wide gaps
    q = rng.choice([-1.0, 1.0], size=wl["k"])
    srcs = [bie.PointSource(tuple(np.array(corners[p]) + d), float(c)) for p, d, c in zip(pick, jit, q)]
    F = bie.rhs_dielectric_box3d(itf, srcs, wl["eps_out"])
    n, k = itf.n, wl["k"]
    g = op.geom._h
    dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).to(f"cuda:{device}")  # noqa: E731
    Fd = dev(F)
    Sd = torch.empty((n, k), dtype=torch.float64, device=f"cuda:{device}")
    stream = torch.cuda.ExternalStream(op.geom.stream, device=device)

    def solve(precision, rtol, itmax):
        o = _abi.SolveOpts()
        L.bie_solve_opts_default(C.byref(o))
        o.rtol, o.itmax, o.restart, o.precision = rtol, itmax, 200, _abi.PRECISIONS[precision]
        st = _abi.Stats()
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        with torch.cuda.stream(stream):
            ev0.record(stream)
            rc = L.bie_solve_device(g, C.c_void_p(Fd.data_ptr()), C.c_void_p(Sd.data_ptr()), k, C.byref(o),
                                    C.byref(st), None)
            ev1.record(stream)
        ev1.synchronize()
        if rc not in (_abi.BIE_OK, _abi.BIE_ENOCONV):
            _abi.check(rc)
        return ev0.elapsed_time(ev1), st, Sd.cpu().numpy().copy()

    solve(args.precision, 1e-2, 3)  # warm-up (workspace, kernel attributes)
    _abi.check(L.bie_profile_enable(g, 1))
    ms_ref, st_ref, S_ref = solve(args.precision, wl["rtol"], 400)
    tc = _abi.KernelTime()
    _abi.check(L.bie_profile_read(g, _abi.KERNEL_KINDS["direct_tc"], C.byref(tc)))
    _abi.check(L.bie_profile_enable(g, 0))
    ms_plain, st_plain, S_plain = solve("fp64", 1e-10, 400)
    err = max(np.linalg.norm(S_ref[:, c] - S_plain[:, c]) / np.linalg.norm(S_plain[:, c]) for c in range(k))
    pairs_per_s = tc.pairs / (tc.launches / 2) / (tc.ms / (tc.launches / 2) * 1e-3) if tc.launches else 0.0
    it_ref, it_plain = max(st_ref.iterations, 1), max(st_plain.iterations, 1)
    line = {"metric": METRIC, "value": k / (ms_ref * 1e-3), "unit": "solves/s", "n_gpus": 1, "steps": 1,
            "warmup": 1, "ms_per_step": ms_ref, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": f"{args.precision} tensor-core direct sum + fp64", "data": "synthetic (seeded sources)",
            "config": {"workload": f"cfg5: lattice {nx}x{ny}x{nz} cubes of side {wl['side']}, gap {wl['gap']}, "
                                   f"n_quad={wl['nq']}, l_ec={wl['l_ec']}, eps {wl['eps_in']}/{wl['eps_out']}, "
                                   f"N={n}, {k} RHS", "nodes": n, "rhs_per_solve": k, "rtol": wl["rtol"],
                       "near_blocks": op.near.nblocks, "host_setup_s": setup_s},
            "refined": {"ms": ms_ref, "iterations": st_ref.iterations, "outer": st_ref.outer,
                        "ms_per_iteration": ms_ref / it_ref, "fp64_matvecs": st_ref.fp64_matvecs,
                        "lowp_matvecs": st_ref.lowp_matvecs},
            "plain_fp64": {"ms": ms_plain, "iterations": st_plain.iterations, "ms_per_iteration": ms_plain / it_plain,
                           "rtol": 1e-10, "value": k / (ms_plain * 1e-3)},
            "speedup_vs_plain_fp64": ms_plain / ms_ref,
            "speedup_per_iteration": (ms_plain / it_plain) / (ms_ref / it_ref),
            "accuracy": {"sigma_rel_err_max": err, "reference_sigma": "plain FP64 GPU solve at rtol 1e-10"},
            "roofline": {"kernel": "k_dt_tc", "pairs_per_s": pairs_per_s,
                         "fp32_issue_frac": pairs_per_s * 12 / (148 * 128 * 1965e6)}}
    print(json.dumps(line), flush=True)
    return 0


def workload_config(name, wl, n):
    return {"workload": f"{name}: block {wl['k']}-RHS solve, box {'x'.join(str(v) for v in wl['box'])}, "
                        f"n_quad={wl['nq']}, l_ec={wl['l_ec']}, eps {wl['eps_in']}/{wl['eps_out']}, N={n}",
            "nodes": n, "rhs_per_solve": wl["k"], "rtol": wl["rtol"], "up_tol": wl["up_tol"],
            "max_order": wl["max_order"], "l2": "flushed between steps (256 MB write)"}


def run_peaks(L, device):
    """Arithmetic ceilings of the direct sums on this device, three probe rounds each
    (the best kept), with the SM clock sampled meanwhile; per-SM-per-clock rates use the
    median sampled clock."""
    import ctypes as C
    import torch
    names = ["fp32_fma", "fp32x2_fma", "mufu_rsqrt", "fp64_fma", "fp64_mma_m8n8k4", "cvt_f32x2_bf16x2"]
    units = ["lane-FMA/s", "lane-FMA/s", "lane-op/s", "lane-FMA/s", "flop/s", "lane-op/s"]
    best = {}
    with ClockSampler(device) as clk:
        for _ in range(3):
            for w, nm in enumerate(names):
                ps, ms = C.c_double(), C.c_double()
                rc = L.bie_peak_probe(device, w, C.byref(ps), C.byref(ms))
                if rc != 0:
                    raise RuntimeError(f"bie_peak_probe({w}) failed: {rc}")
                best[nm] = max(best.get(nm, 0.0), ps.value)
    clocks = clk.summary()
    sms = torch.cuda.get_device_properties(device).multi_processor_count
    mhz = clocks.get("sm_mhz") or 1965.0
    lat = {}
    for w, nm in ((6, "fp64_mma_m8n8k4"), (7, "fp64_fma")):
        ps, ms = C.c_double(), C.c_double()
        if L.bie_peak_probe(device, w, C.byref(ps), C.byref(ms)) != 0:
            raise RuntimeError(f"bie_peak_probe({w}) failed")
        lat[nm] = ps.value
    out = {"peaks": {nm: {"value": best[nm], "unit": u, "per_sm_per_clock": best[nm] / (sms * mhz * 1e6)}
                     for nm, u in zip(names, units)},
           "latency_cycles": lat, "sms": sms, "clocks": clocks}
    print(json.dumps(out), flush=True)
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=8)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="cfg3", choices=sorted(WORKLOADS))
    ap.add_argument("--precision", default="bf16x3", choices=["bf16x3", "fp32"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--block", type=int, default=1, choices=[0, 1],
                    help="1 (default): block GMRES, one Krylov space shared by the block's columns, the "
                         "method of solve_dielectric_box3d_block; 0: one Arnoldi process per column")
    ap.add_argument("--no-serving", action="store_true", help="skip the request-stream measurement")
    ap.add_argument("--profile-matvec", action="store_true",
                    help="apply the refined and the FP64 operator once each to k columns and exit "
                         "(small case for ncu captures)")
    ap.add_argument("--columns", type=int, default=0, help="--profile-matvec: columns (default: the workload's k)")
    ap.add_argument("--cfg4-requests", type=int, default=0, help="--workload cfg4: requests (default 2000)")
    ap.add_argument("--cfg4-nmax", type=int, default=0, help="--workload cfg4: largest node count (default 200000)")
    ap.add_argument("--cfg4-rate", type=float, default=0.0, help="--workload cfg4: arrivals per second (default 20)")
    ap.add_argument("--peaks", action="store_true",
                    help="measure the arithmetic ceilings of the direct sums (FP32 FMA, packed FP32 FMA, "
                         "MUFU rsqrt, FP64 FMA, FP64 tensor-core MMA, FP32 -> bf16x2 conversion) on this "
                         "device and exit")
    args = ap.parse_args()
    wl = WORKLOADS[args.workload]
    if args.impl == "reference":
        return run_reference_arm(args, wl)

    import torch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    device = local
    torch.cuda.set_device(device)
    bie = load_package()
    from dielectricbie_jl_b200 import _abi  # noqa: E402
    import ctypes as C
    L = _abi.lib()
    if args.peaks:
        return run_peaks(L, device)
    if args.workload == "cfg4":
        wl = dict(wl)
        if args.cfg4_requests:
            wl["requests"] = args.cfg4_requests
        if args.cfg4_nmax:
            wl["n_max"] = args.cfg4_nmax
        if args.cfg4_rate:
            wl["rate"] = args.cfg4_rate
        return run_serving_workload(args, wl, bie, device)
    if args.workload == "cfg5":
        return run_lattice_workload(args, wl, bie, device)

    # ---------------- setup (untimed): mesh, near-field blocks, device geometry -------
    itf = bie.single_dielectric_box3d(*wl["box"], wl["nq"], wl["l_ec"], wl["eps_in"], wl["eps_out"])
    op = bie.lhs_dielectric_box3d_fmm3d_corrected(itf, 1e-12, wl["up_tol"], wl["max_order"],
                                                  precision=args.precision, device=device)
    g = op.geom._h
    n, k = itf.n, wl["k"]
    if args.profile_matvec:
        k = args.columns or k
        X = np.asfortranarray(np.random.default_rng(0).standard_normal((n, k)))
        op.mul(X, precision=args.precision)
        op.mul(X, precision="fp64")
        torch.cuda.synchronize(device)
        print(json.dumps({"profile_matvec": args.workload, "n": n, "k": k}), flush=True)
        return 0
    nsteps = args.warmup + args.steps
    batches = make_sources(wl, nsteps + 1, k)
    stream = torch.cuda.ExternalStream(op.geom.stream, device=device)

    def dev(a):
        return torch.from_numpy(np.ascontiguousarray(a)).to(f"cuda:{device}")

    src_d = [dev(p) for p, _ in batches]
    q_d = [dev(q) for _, q in batches]
    eps_d = dev(np.full(k, wl["eps_in"]))
    F = torch.empty((n, k), dtype=torch.float64, device=device)
    S = torch.empty((n, k), dtype=torch.float64, device=device)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=device)  # 256 MB > L2 (126 MB)

    def opts(precision, rtol, verify=False):
        o = _abi.SolveOpts()
        L.bie_solve_opts_default(C.byref(o))
        o.rtol, o.itmax, o.restart = rtol, 600, 200
        o.precision = _abi.PRECISIONS[precision]
        o.flags = 0 if verify else _abi.BIE_NO_VERIFY
        o.block = int(args.block)
        return o

    def solve_step(i, precision, rtol, verify=False, st=None, allow_noconv=False):
        _abi.check(L.bie_rhs_point_device(g, C.c_void_p(src_d[i].data_ptr()), C.c_void_p(q_d[i].data_ptr()),
                                          C.c_void_p(eps_d.data_ptr()), k, C.c_void_p(F.data_ptr()), None))
        o = opts(precision, rtol, verify)
        if allow_noconv:
            o.itmax = 1500
        rc = L.bie_solve_device(g, C.c_void_p(F.data_ptr()), C.c_void_p(S.data_ptr()), k, C.byref(o),
                                C.byref(st) if st is not None else None, None)
        if rc != _abi.BIE_OK and not (allow_noconv and rc == _abi.BIE_ENOCONV):
            _abi.check(rc)

    def timed_loop(precision, rtol, tag, profile=False):
        ms = []
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        for i in range(nsteps):
            flush.zero_()
            torch.cuda.synchronize(device)
            if i == args.warmup and profile:
                _abi.check(L.bie_profile_enable(g, 1))
            if i >= args.warmup:  # NVTX range of a timed step (ncu --nvtx-include "<tag>_step/")
                torch.cuda.nvtx.range_push(f"{tag}_step")
            with torch.cuda.stream(stream):
                ev0.record(stream)
                solve_step(i, precision, rtol)
                ev1.record(stream)
            ev1.synchronize()
            if i >= args.warmup:
                torch.cuda.nvtx.range_pop()
            if i >= args.warmup:
                ms.append(ev0.elapsed_time(ev1))
        return ms

    # ---------------- accuracy (untimed) ---------------------------------------------
    # The oracle's sigma columns (tests/golden/<workload>_sigma.npz, made by
    # tests/golden/make_large.py: the CPU restatement's corrected operator solved to a true
    # relative residual < 1e-13) are the first columns of the accuracy batch; the other
    # columns are compared with a plain FP64 GPU solve of the same batch at rtol 1e-13.
    acc = nsteps
    gold_path = os.path.join(ROOT, "tests", "golden", f"{args.workload}_sigma.npz")
    gold = dict(np.load(gold_path)) if os.path.exists(gold_path) else None
    pos, qs = (a.copy() for a in batches[acc])
    if gold is not None:
        assert gold["n"] == n, "the oracle fixture was made on another mesh"
        ng = len(gold["q"])
        pos[:ng], qs[:ng] = gold["src"], gold["q"]
        src_d[acc].copy_(torch.from_numpy(np.ascontiguousarray(pos)))
        q_d[acc].copy_(torch.from_numpy(np.ascontiguousarray(qs)))
    st = _abi.Stats()
    # plain FP64 at rtol 1e-13 (at high contrast it may stop at its FP64 floor first; the
    # residual it reached is reported)
    solve_step(acc, "fp64", 1e-13, verify=True, st=st, allow_noconv=True)
    torch.cuda.synchronize(device)
    S_plain = S.cpu().numpy().copy()
    plain_ref_iters = st.iterations
    ref_resid = st.max_rel_resid
    solve_step(acc, args.precision, wl["rtol"], verify=True, st=st)
    torch.cuda.synchronize(device)
    S_refined = S.cpu().numpy().copy()

    def relerr(a, b):
        return float(np.linalg.norm(a - b) / np.linalg.norm(b))

    accuracy = {"refined_true_rel_resid": st.max_rel_resid, "refined_iterations": st.iterations,
                "refined_outer": st.outer, "refined_fp64_matvecs": st.fp64_matvecs,
                "refined_lowp_matvecs": st.lowp_matvecs,
                "sigma_rel_err_max_vs_plain_fp64": max(relerr(S_refined[:, c], S_plain[:, c]) for c in range(k)),
                "plain_fp64_rtol": 1e-13, "plain_fp64_true_rel_resid": ref_resid}
    if gold is not None:
        ng = len(gold["q"])
        Sg = gold["sigma"]
        accuracy.update({
            "sigma_rel_err_max": max(relerr(S_refined[:, c], Sg[:, c]) for c in range(ng)),
            "reference_sigma": f"FP64 oracle (CPU restatement of the reference's corrected operator, "
                               f"GMRES to a true relative residual <= {float(gold['true_rel_resid'].max()):.1e}), "
                               f"{ng} columns of the batch ({os.path.relpath(gold_path, ROOT)})",
            "plain_fp64_sigma_rel_err_max_vs_oracle": max(relerr(S_plain[:, c], Sg[:, c]) for c in range(ng))})
    else:
        accuracy.update({"sigma_rel_err_max": accuracy["sigma_rel_err_max_vs_plain_fp64"],
                         "reference_sigma": "plain FP64 GPU solve at rtol 1e-13 (no oracle fixture)"})
    if wl["probes"]:
        # total potential q/(4 pi eps_src r) + S[sigma] at exterior probes
        # (test/solver/dielectric_box3d.jl:285-294) and the polarisation energy, each with the
        # FP64 single layer of the library; the reference is the oracle's sigma where the
        # fixture has it, else the plain FP64 solve
        T = make_probes(bie, itf, wl["probes"], wl["seed"])
        P = bie.laplace3d_pottrg(itf, T)
        ncol = len(gold["q"]) if gold is not None else k
        S_cmp = np.asfortranarray(gold["sigma"] if gold is not None else S_plain)
        r = np.linalg.norm(T[:, None, :] - pos[None, :ncol, :], axis=-1)
        phi_inc = qs[None, :ncol] / (4 * math.pi * wl["eps_in"] * r)
        tot_ref = phi_inc + P @ S_cmp
        tot = phi_inc + P @ np.asfortranarray(S_refined[:, :ncol])
        accuracy["probe_potential_rel_err_max"] = max(relerr(tot[:, c], tot_ref[:, c]) for c in range(ncol))
        srcs = [bie.PointSource(tuple(p), float(qq)) for p, qq in zip(pos[:ncol], qs[:ncol])]
        W_ref = bie.polarization_energy(itf, S_cmp, srcs)
        W = bie.polarization_energy(itf, np.asfortranarray(S_refined[:, :ncol]), srcs)
        accuracy["energy_rel_err_max"] = float(np.max(np.abs(W - W_ref) / np.abs(W_ref)))

    # ---------------- timed: refined (profiled) and plain FP64 ----------------------
    if dist is not None:
        dist.barrier()
    with ClockSampler(device) as clk:
        ms_ref = timed_loop(args.precision, wl["rtol"], "refined")
    # the last timed refined step's sigma (its steps skip the solver's own final check):
    # FP64 true residual ||F - A sigma|| / ||F|| per column, untimed
    Y = torch.empty_like(S)
    _abi.check(L.bie_matvec_device(g, C.c_void_p(S.data_ptr()), C.c_void_p(Y.data_ptr()), k, _abi.BIE_FP64, 0,
                                   C.c_void_p(op.geom.stream)))
    torch.cuda.synchronize(device)
    accuracy["timed_step_true_rel_resid_max"] = float(((F - Y).norm(dim=0) / F.norm(dim=0)).max())
    ms_plain = timed_loop("fp64", wl["rtol"], "plain")
    # kernel breakdown: the same refined steps again with per-kernel event timing (eager
    # launches; the timed loops above replay captured GMRES iterations as CUDA graphs)
    timed_loop(args.precision, wl["rtol"], "profiled", profile=True)
    kt = {}
    for name, kind in _abi.KERNEL_KINDS.items():
        t = _abi.KernelTime()
        _abi.check(L.bie_profile_read(g, kind, C.byref(t)))
        kt[name] = t
    _abi.check(L.bie_profile_enable(g, 0))

    total_ms = float(np.sum(ms_ref))
    total_plain = float(np.sum(ms_plain))
    if dist is not None:
        total_ms, total_plain = max_over_ranks(dist, [total_ms, total_plain], device)
    solves = k * args.steps * world
    value = replica_value(k * args.steps, world, total_ms)
    plain_value = replica_value(k * args.steps, world, total_plain)

    # ---------------- e2e: reference-shaped host API with host buffers ---------------
    # bie_solve_point: the k point sources (pinned host memory) go to the device, the
    # right-hand sides are built there, and Sigma (N x k column-major, pinned) comes back;
    # the host clock spans the whole call. Phases: the solve's device time (stats.seconds,
    # events inside the call) and the rest of the call (copies, layout conversion, host).
    pin = lambda shape: torch.empty(shape, dtype=torch.float64, pin_memory=True).numpy()  # noqa: E731
    Sh = np.asfortranarray(pin((k, n)).T)   # N x k column-major, pinned
    src_h, q_h, eps_h = pin((k, 3)), pin((k,)), pin((k,))
    e2e_ms, e2e_solve_ms = [], []
    o = opts(args.precision, wl["rtol"])
    st_e2e = _abi.Stats()
    for i in range(nsteps):
        pos_i, q_i = batches[i]
        src_h[:], q_h[:], eps_h[:] = pos_i, q_i, wl["eps_in"]
        flush.zero_()
        torch.cuda.synchronize(device)
        t0 = time.perf_counter()
        rc = L.bie_solve_point(g, _abi.dptr(src_h), _abi.dptr(q_h), _abi.dptr(eps_h), k, _abi.dptr(Sh), C.byref(o),
                               C.byref(st_e2e))
        t1 = time.perf_counter()
        if rc != _abi.BIE_OK:
            _abi.check(rc)
        if i >= args.warmup:
            e2e_ms.append((t1 - t0) * 1e3)
            e2e_solve_ms.append(st_e2e.seconds * 1e3)
    e2e_total = float(np.sum(e2e_ms))
    if dist is not None:
        (e2e_total,) = max_over_ranks(dist, [e2e_total], device)
    e2e_value = solves / (e2e_total * 1e-3)
    e2e_phases = {"call_ms_mean": float(np.mean(e2e_ms)), "solve_device_ms_mean": float(np.mean(e2e_solve_ms)),
                  "outside_solve_ms_mean": float(np.mean(e2e_ms) - np.mean(e2e_solve_ms)),
                  "call_ms_p99": float(np.percentile(e2e_ms, 99))}

    # ---------------- serving: cfg3 request stream, continuous batching vs plain ------
    serving = None
    if args.workload == "cfg3" and world == 1 and not args.no_serving:
        # the served batches keep one Arnoldi process per column: measured on the cfg3 stream,
        # block GMRES per merged batch (up to 128 columns, converging together) served 532
        # solves/s against 1,135
        serving = request_stream(bie, itf, op, wl, args.precision, device, block=False)

    # ---------------- roofline of the dominant kernel ------------------------------
    peaks = {}
    pk_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(pk_path):
        with open(pk_path) as f:
            peaks = json.load(f)
    # denominators: the driver-measured peaks when present (the sustained bf16 figure: the
    # kernel is timed inside long solve steps), else the pool's fallback figures (6.65 TB/s
    # copy, 1.59 PFLOP/s bf16 burst)
    if "bf16_tflops_sustained" in peaks:
        bf16_peak, bf16_src = peaks["bf16_tflops_sustained"], "bf16_tflops_sustained of measured"
    elif "bf16_tflops" in peaks:
        bf16_peak, bf16_src = peaks["bf16_tflops"], "bf16_tflops of measured"
    else:
        bf16_peak, bf16_src = 1590.0, "bf16 1.59 PFLOP/s of fallback"
    hbm_peak = peaks.get("hbm_gbs", 6650.0)
    hbm_src = "hbm_gbs of measured" if "hbm_gbs" in peaks else "6.65 TB/s of fallback"
    clocks = clk.summary()
    kinds_ms = {nm: t.ms for nm, t in kt.items() if nm != "all"}
    dominant = max(kinds_ms, key=kinds_ms.get)
    tc = kt["direct_tc"]
    roofline = None
    if tc.launches:
        per_launch_ms = tc.ms / (tc.launches / 2)  # pack + tensor-core kernel per column block
        flops = 6.0 * tc.pair_cols / (tc.launches / 2)  # three bf16 MMAs (2 flops each) per pair and column
        achieved = flops / (per_launch_ms * 1e-3) / 1e12
        roofline = {"kernel": "k_dt_tc (tcgen05 split-BF16 x3 block direct sum, incl. Q packing)", "bound": "tensor",
                    "achieved": achieved, "peak": bf16_peak, "unit": "TFLOP/s", "frac": achieved / bf16_peak,
                    "peak_source": bf16_src,
                    "traffic": profiled_traffic(f"k_dt_tc_{args.workload}.md"),
                    "traffic_source": f"profiles/k_dt_tc_{args.workload}.md (ncu dram bytes read + written per launch)",
                    "per_launch_ms": per_launch_ms,
                    "autotuned_launch": bie.tuned_launch(op, "tensor_core", k)}
        sm_mhz = clocks.get("sm_mhz") or 1965.0
        fp32_issue_peak = 148 * 128 * sm_mhz * 1e6  # FP32 lane-instructions/s at the sampled clock
        pairs_per_s = tc.pairs / (tc.launches / 2) / (per_launch_ms * 1e-3)
        roofline["fp32_issue_frac"] = pairs_per_s * 12 / fp32_issue_peak
        roofline["pairs_per_s"] = pairs_per_s
    comb = kt["combine"]
    extra = {}
    for nm, t in kt.items():
        if nm == "all" or not t.launches:
            continue
        extra[nm] = {"ms": t.ms, "launches": t.launches, "share": t.ms / max(kt["all"].ms, 1e-9)}
    if comb.launches:
        gbs = comb.bytes / (comb.ms * 1e-3) / 1e9
        extra["combine"].update({"achieved_GBps": gbs, "hbm_frac": gbs / hbm_peak, "peak_source": hbm_src})
    f64 = kt["direct_fp64"]
    if f64.launches:
        extra["direct_fp64"]["pair_cols_per_s"] = f64.pair_cols / (f64.ms * 1e-3)

    # ---------------- CPU baseline (rank 0, N = 1) ----------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        info = CpuReference(wl).solve(0, max_seconds=20.0)
        cpu = {"value": 1.0 / info["seconds"], "unit": "solves/s", "cores": info["cores"], "kind": "port",
               "sample": f"one RHS column of the workload: oracle FP64 direct sum + CSC corrections + GMRES, "
                         f"{info['iterations']} iterations, {info['seconds']:.2f} s"
                         f"{'' if info['converged'] else ' (time-bounded, not converged)'}"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": f"{args.precision} tensor-core direct sum + fp64",
            "data": "synthetic (seeded point sources, uniform in the box interior)",
            "config": dict(workload_config(args.workload, wl, n),
                           krylov="block GMRES (one Krylov space per block)" if args.block
                           else "GMRES, one Arnoldi process per column"),
            "p50_ms": float(np.percentile(ms_ref, 50)), "p99_ms": float(np.percentile(ms_ref, 99)),
            "plain_fp64": {"value": plain_value, "unit": "solves/s", "ms_per_step": total_plain / args.steps,
                           "p50_ms": float(np.percentile(ms_plain, 50)),
                           "p99_ms": float(np.percentile(ms_plain, 99)), "iterations": plain_ref_iters},
            "speedup_vs_plain_fp64": value / plain_value,
            "accuracy": accuracy,
            "roofline": roofline,
            "kernels": extra,
            "dominant_kernel_kind": dominant,
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_value, "unit": "solves/s", "h2d_bytes_per_step": 5 * k * 8,
                    "d2h_bytes_per_step": n * k * 8, "api": "bie_solve_point (host sources in, host Sigma out)",
                    "phases": e2e_phases},
            "serving": serving,
            "gpu_launches": int(kt["all"].launches),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
