#!/usr/bin/env python
"""Benchmark of the dense density-matrix step on the 512-H2O box (ndim 11776).

One step = one SCF iteration's density step: packed H, S -> filter (1e-5) ->
Cholesky orthogonalisation -> trace-correcting purification -> packed P.

  value  device-resident packed inputs (libptbgpu ptbgpu_tc_purify_device),
         seconds per step from the library's CUDA events on its stream;
  e2e    the C-ABI call with pinned host buffers (ptbgpu_tc_purify), host->device
         and device->host copies inside the timed region, host wall clock around
         every one of the timed calls.
  cpu_baseline  one whole call of the oracle's dense solve2 on the same problem
         (all host cores), no scaling.

Inputs (2 x 555 MB packed, plus ~8 GB of working matrices per step) are far
larger than the 126 MB L2, so no L2 flush is needed between steps.
N > 1 runs independent replicas (the dense step does not shard); the per-step
time reported is the maximum over ranks.

--impl reference times the reference's dense FP64 density step (the check-mode
solve2: LAPACK dsygvd + Fermi occupations + P = C f C^T, restated in the CPU
oracle with scipy's multithreaded OpenBLAS) on the host cores, whole calls
only: where the requested steps do not fit --ref-budget seconds, fewer whole
calls run and the line's "steps" says how many (the request is kept beside it).

--workload sm_water32 / sm_alkane / sm_water512 measure the submatrix method
(the density step twoscf calls, source/sm.f90): the 32-H2O cluster and the
C200H402 chain with per-atom columns, the 512-H2O box with seeded k-means
columns, all with filter 1e-4; value = device time of the call (inputs copied
in first), e2e = the whole host call.

--workload purify_types measures the reference's full-matrix purification
module (dormant in twoscf: McWeeny, Pade, Newton-Schulz and eigen-sign solvers
with the chemical-potential search, source/purification.f90) in FP64 on the
32-H2O cluster, one call per solver type; the oracle is the CPU baseline.

--workload lattice256 measures the uneven multi-instance batch instead: 256
synthetic cubic-lattice systems (20-400 atoms, ndim 166-3064), every system's
dense projector by the FP64 eigensolver in one launch
(ptbgpu_eig_density_batch); one step = the whole batch, host buffers in and
out (value and e2e are the same call).  The trace-correcting purification of
the same systems (ptbgpu_tc_purify_batch, mixed and FP64, host worker threads)
and the grouped entry are reported beside it.  With N > 1 the 256 systems are
split over the ranks (size-balanced, no collective) and the batch's time is the
maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

import numpy as np  # noqa: E402

METRIC = "P-build s/SCF iter & TFLOP/s: mixed-prec vs FP64 GPU at max|dP|<=1e-6"
UNIT = "s/SCF-iter"
FILTER = 1e-5


def load_peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return d.get("bf16_tflops", 1590.0), d.get("bf16_tflops_sustained", 1400.0), d.get("hbm_gbs", 6650.0), "measured"
    return 1590.0, 1400.0, 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except (FileNotFoundError, OSError):
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        if not self.path or not os.path.exists(self.path):
            return None
        rows = [r.split(",") for r in open(self.path).read().strip().splitlines() if r.strip()]
        os.unlink(self.path)
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx = max(mx, float(r[2]))
                for k, nm in enumerate(names):
                    if r[5 + k].strip().lower() == "active":
                        reasons.add(nm)
            except (ValueError, IndexError):
                continue
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def dist_setup(gpus: int):
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
        pg = dist
    return rank, world, local, pg


def reduce_max(pg, value: float) -> float:
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], device="cuda", dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def reduce_sum(pg, value: float) -> float:
    if pg is None:
        return value
    import torch
    t = torch.tensor([value], device="cuda", dtype=torch.float64)
    pg.all_reduce(t, op=pg.ReduceOp.SUM)
    return float(t.item())


def barrier(pg):
    if pg is not None:
        pg.barrier()


def cpu_dense_full(sysobj):
    """One call of the oracle's dense FP64 density step (the check-mode solve2:
    dsygvd + Fermi occupations + P = C f C^T) on the whole workload, filtered as
    the GPU path filters it; returns its wall-clock seconds."""
    from oracle import ptb_oracle as O
    Hv = O.filter_matrix_sym(sysobj.Hvec, FILTER)
    Sv = O.filter_matrix_sym(sysobj.Svec, FILTER)
    t0 = time.perf_counter()
    O.solve2(1, sysobj.ndim, sysobj.nel, 0, 300.0, Hv, Sv)
    return time.perf_counter() - t0


def timed_calls(call, steps: int, warm, warmups: int, budget_s: float):
    """The reference arm's timing loop: `warmups` untimed calls of `warm` (a
    cheap call of the same code path), then whole calls of `call` until `steps`
    have run or `budget_s` of wall clock is spent (at least one).  Returns the
    per-call seconds actually measured and the warm-up count actually run."""
    t_start = time.perf_counter()
    for _ in range(warmups):
        warm()
    times = []
    while len(times) < steps:
        t0 = time.perf_counter()
        call()
        times.append(time.perf_counter() - t0)
        if time.perf_counter() - t_start + times[-1] > budget_s:
            break
    return times, warmups


def reference_line(args, value, unit, desc, ndim, batch, sample, times, warmups):
    cores = os.cpu_count()
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": unit, "n_gpus": args.gpus,
        "steps": len(times), "warmup": warmups, "requested_steps": args.steps, "requested_warmup": args.warmup,
        "ms_per_step": value * 1e3, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "global_batch": batch, "seq_len": ndim, "parallelism": "replicas"},
        "cpu_baseline": {"value": value, "unit": unit, "cores": cores, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "timed_calls_s": times,
    }


def run_reference(args, rank):
    """The reference arm: the oracle's CPU restatement of the same workload on
    all host cores, whole calls only (no scaling of samples).  Where the
    requested steps do not fit the time budget, fewer whole calls are timed and
    the line says how many ran."""
    from ptb_b200 import synth
    if rank != 0:
        return
    budget = args.ref_budget
    cores = os.cpu_count()
    if args.workload in SM_WORKLOADS:
        cfg, cols, desc = SM_WORKLOADS[args.workload]
        if synth.CONFIGS[cfg].get("nmol", 0) * 23 > SM_ORACLE_MAX_NDIM:
            print(json.dumps({"impl": "reference", "unavailable": "the CPU restatement of the submatrix method works "
                              "on full ndim x ndim matrices, which at ndim 47104 need about 70 GB of host memory"}),
                  flush=True)
            return
        sysobj = synth.make_config(cfg)
        cpu = SmCpu(sysobj, cols)
        times, w = timed_calls(cpu.call, args.steps, cpu.call, min(args.warmup, 1), budget)
        v = statistics.median(times)
        line = reference_line(args, v, UNIT, desc, sysobj.ndim, 1, cpu.sample(cores, len(times)), times, w)
        print(json.dumps(line), flush=True)
        return
    if args.workload == "purify_types":
        s = synth.make_config(0)
        sweep = lambda: [purify_oracle(s, pt, me, it) for pt, me, it, _ in PURIFY_TYPES]
        times, w = timed_calls(sweep, args.steps, sweep, min(args.warmup, 1), budget)
        v = statistics.median(times)
        line = reference_line(args, v, PURIFY_UNIT, PURIFY_DESC, s.ndim, 1,
                              f"oracle purification (numpy / scipy OpenBLAS, {cores} threads), one call per type, "
                              f"whole workload, median of {len(times)} sweeps", times, w)
        print(json.dumps(line), flush=True)
        return
    if args.workload == "lattice256":
        from oracle import ptb_oracle as O
        systems = synth.make_config(4)

        def batch():
            for x in systems:
                O.solve2(1, x.ndim, x.nel, 0, 300.0, x.Hvec, x.Svec)

        small = min(systems, key=lambda x: x.ndim)
        warm = lambda: O.solve2(1, small.ndim, small.nel, 0, 300.0, small.Hvec, small.Svec)
        times, w = timed_calls(batch, args.steps, warm, args.warmup, budget)
        v = statistics.median(times)
        line = reference_line(args, v, "s/batch-of-256",
                              "uneven multi-instance batch: 256 cubic-lattice systems (20-400 atoms)", 
                              max(x.ndim for x in systems), 256,
                              f"oracle solve2 (dsygvd + Fermi + C f C^T, OpenBLAS {cores} threads) on all 256 "
                              f"systems, median of {len(times)} whole batches", times, w)
        print(json.dumps(line), flush=True)
        return
    s = synth.water_cluster(args.nmol, seed=1)
    n = s.ndim
    from oracle import ptb_oracle as O
    lead = min(n, 2048)
    Hl = O.packsym(O.blowsym(n, s.Hvec)[:lead, :lead])
    Sl = O.packsym(O.blowsym(n, s.Svec)[:lead, :lead])
    warm = lambda: O.solve2(1, lead, min(s.nel, lead), 0, 300.0, Hl, Sl)
    times, w = timed_calls(lambda: cpu_dense_full(s), args.steps, warm, min(args.warmup, 1), budget)
    v = statistics.median(times)
    line = reference_line(args, v, UNIT,
                          f"dense density step, {args.nmol}-H2O box ({s.nat} atoms, ndim {n}, nel {s.nel}), "
                          "filter 1e-5", n, 1,
                          f"oracle solve2 (dsygvd + Fermi + C f C^T, OpenBLAS {cores} threads) on the whole "
                          f"ndim {n} problem, median of {len(times)} whole calls (warm-up: one call on the leading "
                          f"{lead} basis functions)", times, w)
    print(json.dumps(line), flush=True)


SM_WORKLOADS = {
    "sm_water32": (0, 2, "submatrix method, 32-H2O cluster (96 atoms, ndim 736), per-atom columns, filter 1e-4"),
    "sm_alkane": (2, 2, "submatrix method, C200H402 (602 atoms, ndim 4610), per-atom columns, filter 1e-4"),
    "sm_water512": (1, 4, "submatrix method, 512-H2O box (1536 atoms, ndim 11776), seeded k-means columns, "
                          "filter 1e-4"),
    "sm_water2048": (3, 4, "submatrix method, 2048-H2O box (6144 atoms, ndim 47104), seeded k-means columns, "
                           "filter 1e-4"),
}
# The oracle restates the submatrix method on full n x n matrices: above this order
# (the 2048-H2O box: two 17.7 GB full matrices plus their filtered copies) it does
# not fit a host, so those workloads have no CPU baseline.
SM_ORACLE_MAX_NDIM = 20000
SM_FILTER = 1e-4


class SmCpu:
    """The oracle's submatrix method on the host cores, whole calls.  With
    k-means columns the grouping (the oracle's seeded k-means, a slow
    pure-Python restatement; the reference's own k-means took 2.0 s of its
    logged 45.2 s) runs once outside the timed call and its partition is
    passed in, as the library's benchmark call receives it."""

    def __init__(self, s, cols):
        from oracle import ptb_oracle as O
        self.O, self.s, self.cols = O, s, cols
        self.Hv = O.filter_matrix_sym(s.Hvec, SM_FILTER)
        self.Sv = O.filter_matrix_sym(s.Svec, SM_FILTER)
        self.part = None
        if cols == 4:
            H, S = O.blowsym(s.ndim, self.Hv), O.blowsym(s.ndim, self.Sv)
            self.part, _, _ = O.kmeans_partition(s.ndim, H, S, s.nat, s.xyz, s.aoat, seed=42)
        self.last = None

    def call(self):
        O, s = self.O, self.s
        self.last = O.sm_stupid_simple(s.ndim, s.nel, self.Hv, self.Sv, s.nat, s.xyz, s.aoat, self.cols, 2,
                                       self.part)
        return self.last

    def sample(self, cores, count):
        what = "oracle sm_stupid_simple (scipy OpenBLAS dsygvd, " + str(cores) + " threads), whole workload"
        if self.cols == 4:
            what += " with the seeded k-means partition computed outside the timed call"
        return what + f", median of {count} whole calls"

    def step(self):
        """Returns (seconds, sample text, oracle result) of one whole call."""
        t0 = time.perf_counter()
        ref = self.call()
        return time.perf_counter() - t0, self.sample(os.cpu_count(), 1), ref


def run_sm(args, rank, world, local, pg):
    import torch

    from ptb_b200 import Context, Options, synth

    cfg, cols, desc = SM_WORKLOADS[args.workload]
    s = synth.make_config(cfg)
    torch.cuda.set_device(local)
    ctx = Context(local)
    o = Options(filter=SM_FILTER)
    part = None
    if cols == 4:   # the library's seeded k-means (also what the call itself runs without a partition)
        part, _, _ = ctx.kmeans_partition(s.ndim, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, seed=42, opts=o)
    pinned = False
    if world == 1:
        # end to end from pinned host buffers (H, S in, P out), as the dense line;
        # pageable arrays where the host cannot pin that much (2048 H2O: 3 x 8.9 GB)
        try:
            hH = torch.from_numpy(s.Hvec).pin_memory().numpy()
            hS = torch.from_numpy(s.Svec).pin_memory().numpy()
            hP = torch.empty(s.ndim * (s.ndim + 1) // 2, dtype=torch.float64).pin_memory().numpy()
            pinned = True
        except RuntimeError:
            hH, hS, hP = s.Hvec, s.Svec, None
        call = lambda: ctx.sm_stupid_simple(s.ndim, s.nel, hH, hS, s.nat, s.xyz, s.aoat, cols, 2, None, o, out=hP)
    else:
        # one system over the ranks: a size-balanced share of the submatrices per GPU,
        # one all-reduce of the electron count per bisection step, one of P at the end
        from ptb_b200.distributed import DeviceShard, sm_stupid_simple_sharded

        class Shard(DeviceShard):
            launches = 0

            def prepare(self, ids):
                st_ = super().prepare(ids)
                Shard.launches = int(st_.kernel_launches)
                return st_

        shard = Shard(ctx)
        call = lambda: sm_stupid_simple_sharded(shard, s.ndim, s.nel, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, cols, 2,
                                                None, o)
    for _ in range(args.warmup):
        call()
    barrier(pg)
    stats, walls, evms = [], [], []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            torch.cuda.synchronize()
            barrier(pg)
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            t0 = time.perf_counter()
            e0.record()
            P, st = call()
            e1.record()
            torch.cuda.synchronize()
            walls.append(time.perf_counter() - t0)
            evms.append(e0.elapsed_time(e1))
            stats.append(st)
    clocks = clk.summary()
    # one GPU: the library's device time of the call; several: the whole sharded
    # call between events (the ranks wait on each other inside it), max over ranks
    ms = reduce_max(pg, statistics.median(x.ms_solve for x in stats) if world == 1 else statistics.median(evms))
    wall = reduce_max(pg, statistics.median(walls))
    if rank != 0:
        ctx.close()
        return
    if world > 1:
        info = stats[-1]
        stats = [type("S", (), {"nsm": info.nsm, "sum_dims": int(np.sum(info.dims)), "max_dim": int(np.max(info.dims)),
                                "mu_iterations": len(info.trace), "kernel_launches": Shard.launches,
                                "mu": info.mu, "nel": info.nel})()]
    dims = ctx.sm_plan(s.ndim, s.Hvec, s.Svec, s.nat, s.xyz, s.aoat, cols, 2, part, o)
    feig = float(np.sum(7.0 * np.asarray(dims, dtype=np.float64) ** 3))
    cpu, acc = None, {}
    if world == 1 and not args.no_cpu_baseline and s.ndim <= SM_ORACLE_MAX_NDIM:
        tc, sample, ref = SmCpu(s, cols).step()
        cpu = {"value": tc, "unit": UNIT, "cores": os.cpu_count(), "kind": "port", "sample": sample}
        if ref is not None:
            acc = {"max_abs_dP_vs_oracle": float(np.max(np.abs(P - ref.Pvec))), "mu": stats[-1].mu,
                   "mu_oracle": ref.mu, "nel": stats[-1].nel, "nel_oracle": ref.nel}
    last = stats[-1]
    npk = s.ndim * (s.ndim + 1) // 2
    line = {
        "metric": METRIC, "value": ms / 1e3, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak" if world == 1 else "strong",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": desc, "global_batch": 1, "seq_len": s.ndim,
                   "parallelism": "one GPU" if world == 1 else f"submatrices sharded over {world} ranks",
                   "l2": "per call the packed inputs are copied in and unpacked afresh"},
        "submatrices": {"nsm": int(last.nsm), "sum_dims": int(last.sum_dims), "max_dim": int(last.max_dim),
                        "mu_iterations": int(last.mu_iterations)},
        "e2e": {"value": wall, "unit": UNIT, "h2d_bytes_per_step": 2 * npk * 8, "d2h_bytes_per_step": npk * 8,
                "timing": "host wall clock of the whole call, median of the timed calls; "
                          + ("pinned host H, S and P" if pinned else "pageable host arrays")
                          + ("" if world == 1 else ", max over ranks")},
        "gpu_launches": int(sum(x.kernel_launches for x in stats)),
        "roofline": {"bound": "fp64", "kernel": "the library's FP64 generalized eigensolver (Cholesky, reduction, "
                     "tridiagonalisation, divide and conquer, owned rows; DMMA tile products): k_eig_fused, one "
                     "persistent launch for submatrices of order <= 1024, and k_eig_cluster, one thread-block "
                     "cluster per larger submatrix, side by side",
                     "achieved": feig / (ms / 1e3) / 1e12,
                     "peak": 37.0, "unit": "TFLOP/s", "frac": feig / (ms / 1e3) / 1e12 / 37.0, "traffic": None,
                     "peak_kind": "nominal B200 FP64 (no measured FP64 figure on this pool)",
                     "work": "7 m^3 per submatrix (dsygvd with vectors), the whole call's device time"},
        "cpu_baseline": cpu, "clocks": clocks,
    }
    if acc:
        line["accuracy"] = acc
    print(json.dumps(line), flush=True)
    ctx.close()


# The solver types of the reference's full-matrix purification module
# (source/purification_settings.f90:6-27): type, metric, iterative metric, label.
PURIFY_TYPES = [
    (1, 2, False, "mcweeny, inverse_sqrt"),
    (1, 1, False, "mcweeny, inverse"),
    (2, 2, False, "pade, inverse_sqrt"),
    (3, 2, False, "newton, inverse_sqrt"),
    (3, 1, True, "newton, inverse, iterative_inversion"),
    (4, 2, False, "diag, inverse_sqrt"),
]
PURIFY_DESC = ("full-matrix purification module (mu search with McWeeny / Pade / Newton-Schulz / eigen-sign "
               "solvers), 32-H2O cluster (96 atoms, ndim 736, nel 256), filter 1e-4, one call per solver type")
PURIFY_UNIT = "s/sweep-of-6-types"


def purify_oracle(s, ptype, metric, it):
    """One oracle call of the purification module with the workload's filter."""
    from oracle import ptb_oracle as O
    pur = O.PurificationSettings(type=ptype, metric_type=metric, metric_iterative=it, nel=s.nel)
    t0 = time.perf_counter()
    P, mu, steps = O.purification(pur, s.ndim, O.filter_matrix_sym(s.Hvec, SM_FILTER),
                                  O.filter_matrix_sym(s.Svec, SM_FILTER))
    return time.perf_counter() - t0, P, mu, steps


def run_purify_types(args, rank, world, local, pg):
    """The reference's dormant full-matrix purification (purification_wrapper,
    source/purification.f90:28-782) in FP64 on the device, once per solver type;
    one step = the six calls.  N > 1 runs replicas."""
    import torch

    from ptb_b200 import Context, Options, PurificationSettings, synth

    s = synth.make_config(0)
    torch.cuda.set_device(local)
    ctx = Context(local)
    o = Options(filter=SM_FILTER)
    npk = s.ndim * (s.ndim + 1) // 2
    per, step_ms, step_wall, launches, flops = [], 0.0, 0.0, 0, 0.0
    with ClockSampler(local) as clk:
        for ptype, metric, it, label in PURIFY_TYPES:
            pur = PurificationSettings(type=ptype, metric_type=metric, metric_iterative=it, nel=s.nel)
            for _ in range(args.warmup):
                ctx.purification(pur, s.ndim, s.Hvec, s.Svec, o)
            ms, walls, sts = [], [], []
            for _ in range(args.steps):
                torch.cuda.synchronize()
                barrier(pg)
                t0 = time.perf_counter()
                P, st = ctx.purification(pur, s.ndim, s.Hvec, s.Svec, o)
                walls.append(time.perf_counter() - t0)
                ms.append(st.ms_solve)
                sts.append(st)
            m = reduce_max(pg, statistics.median(ms))
            w = reduce_max(pg, statistics.median(walls))
            step_ms += m
            step_wall += w
            launches += sum(x.kernel_launches for x in sts)
            flops += sts[-1].flops
            per.append({"type": label, "ms": m, "mu_steps": int(sts[-1].mu_iterations),
                        "sign_iterations": int(sts[-1].iterations), "mu": sts[-1].mu,
                        "dgemm_tflops": sts[-1].flops / (m / 1e3) / 1e12, "P": P})
    clocks = clk.summary()
    if rank != 0:
        ctx.close()
        return
    cpu_s = 0.0
    if not args.no_cpu_baseline:
        for (ptype, metric, it, _), d in zip(PURIFY_TYPES, per):
            t, Pref, mu, steps = purify_oracle(s, ptype, metric, it)
            cpu_s += t
            d.update({"oracle_s": t, "max_abs_dP_vs_oracle": float(np.max(np.abs(d["P"] - Pref))),
                      "mu_oracle": mu, "mu_steps_oracle": int(steps)})
    for d in per:
        d.pop("P")
    tf = flops / (step_ms / 1e3) / 1e12
    line = {
        "metric": METRIC, "value": step_ms / 1e3, "unit": PURIFY_UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": PURIFY_DESC, "global_batch": 1, "seq_len": s.ndim,
                   "parallelism": "one GPU" if world == 1 else f"replicas x{world}",
                   "l2": "small case: inputs (4.3 MB packed) fit in L2; latency-bound"},
        "e2e": {"value": step_wall, "unit": PURIFY_UNIT, "h2d_bytes_per_step": len(PURIFY_TYPES) * 2 * npk * 8,
                "d2h_bytes_per_step": len(PURIFY_TYPES) * npk * 8},
        "gpu_launches": launches,
        "roofline": {"bound": "fp64", "kernel": "FP64-class products on the int8 tensor cores (oz_dgemm) and the "
                     "library's eigensolver (eig_full) with the library's kernels",
                     "achieved": tf, "peak": 37.0, "unit": "TFLOP/s", "frac": tf / 37.0, "traffic": None,
                     "peak_kind": "nominal B200 FP64 (no measured FP64 figure on this pool)",
                     "work": "2 n^3 per FP64-class product issued, eigensolves not counted, over the six calls' "
                             "device time"},
        "cpu_baseline": ({"value": cpu_s, "unit": PURIFY_UNIT, "cores": os.cpu_count(), "kind": "port",
                          "sample": "oracle purification (numpy / scipy OpenBLAS), one call per type, whole workload"}
                         if cpu_s else None),
        "clocks": clocks, "types": per,
    }
    print(json.dumps(line), flush=True)
    ctx.close()


def run_batch(args, rank, world, local, pg):
    """The multi-instance batch of 256 independent systems.  The timed path is
    the library's FP64 eigensolver with every system in one launch
    (ptbgpu_eig_density_batch: one CTA per system up to order 1024, one
    thread-block cluster per larger system, P formed in the same launch).  On
    one GPU the trace-correcting purification of the same systems (mixed
    precision and FP64, host worker streams) and the grouped entry are reported
    beside it.  With N ranks the systems are split size-balanced (decreasing
    ndim^3 to the least-loaded rank, the submatrix shards' rule) and each rank
    solves its share in one launch: no collective, the batch's time is the
    maximum over ranks (strong scaling of the fixed batch)."""
    import torch

    from ptb_b200 import PREC_FP64, PREC_MIXED, Context, Options, synth

    all_systems = synth.make_config(4)
    if world > 1:
        from ptb_b200.distributed import assign_submatrices
        share = assign_submatrices([s.ndim for s in all_systems], world)[rank]
        systems = [all_systems[k] for k in share]
    else:
        systems = all_systems
    args_b = [(s.ndim, s.nel, s.Hvec, s.Svec) for s in systems]
    torch.cuda.set_device(local)
    ctx = Context(local)
    for _ in range(args.warmup):
        ctx.eig_density_batch(args_b)
    barrier(pg)
    walls, stats = [], None
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            Ps, stats, wall = ctx.eig_density_batch(args_b)
            walls.append(wall)
    clocks = clk.summary()
    ms = reduce_max(pg, statistics.median(walls))
    comparisons = {}
    if args.compare_fp64 and world == 1:
        Pm, stm, wallm = ctx.tc_purify_batch(args_b, Options(precision=PREC_MIXED), workers=args.workers)
        P64, st64, wall64 = ctx.tc_purify_batch(args_b, Options(precision=PREC_FP64), workers=args.workers)
        Pg, stg, wallg = ctx.tc_purify_grouped(args_b, Options(precision=PREC_MIXED))
        dmax = lambda X, Y: float(max(np.max(np.abs(a - b)) for a, b in zip(X, Y)))
        comparisons = {
            "purify_mixed": {"entry": "ptbgpu_tc_purify_batch (bf16x3 trace-correcting purification, FP64-class "
                                      f"refinement, {args.workers} worker streams)", "s_per_step": wallm / 1e3,
                             "max_abs_dP_vs_eig_batch": dmax(Pm, Ps),
                             "refine_rounds": {str(r): sum(1 for x in stm if x.refine_rounds == r) for r in range(6)},
                             "fp64_fallbacks": sum(x.fp64_fallback for x in stm),
                             "gpu_launches": int(sum(x.kernel_launches for x in stm))},
            "purify_fp64": {"entry": "ptbgpu_tc_purify_batch, FP64", "s_per_step": wall64 / 1e3,
                            "max_abs_dP_vs_eig_batch": dmax(P64, Ps)},
            "purify_grouped": {"entry": "ptbgpu_tc_purify_grouped", "s_per_step": wallg / 1e3,
                               "max_abs_dP_vs_eig_batch": dmax(Pg, Ps)},
            "speedup_eig_batch_vs_purify_mixed": wallm / ms, "speedup_eig_batch_vs_purify_fp64": wall64 / ms,
        }
    launches = reduce_sum(pg, float(sum(x.kernel_launches for x in stats)) * args.steps)
    if rank != 0:
        ctx.close()
        return
    feig = float(sum(7.0 * float(s.ndim) ** 3 for s in all_systems))
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        from oracle import ptb_oracle as O
        t0 = time.perf_counter()
        for s in systems:
            O.solve2(1, s.ndim, s.nel, 0, 300.0, s.Hvec, s.Svec)
        t = time.perf_counter() - t0
        cpu = {"value": t, "unit": "s/batch-of-256", "cores": os.cpu_count(), "kind": "port",
               "sample": f"oracle solve2 (dsygvd + Fermi + C f C^T, scipy OpenBLAS, {os.cpu_count()} threads) on "
                         "all 256 systems, one whole batch"}
    npk = sum(s.ndim * (s.ndim + 1) // 2 for s in all_systems)
    line = {
        "metric": METRIC, "value": ms / 1e3, "unit": "s/batch-of-256", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak" if world == 1 else "strong", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "uneven multi-instance batch: 256 cubic-lattice systems (20-400 atoms, ndim "
                               f"{min(s.ndim for s in all_systems)}-{max(s.ndim for s in all_systems)}), dense "
                               "projector per system by the FP64 eigensolver, all systems (of a rank's share) in one "
                               "launch",
                   "global_batch": 256, "seq_len": max(s.ndim for s in all_systems),
                   "parallelism": "one GPU" if world == 1 else
                   f"systems sharded over {world} ranks (size-balanced by ndim^3, no collective)",
                   "l2": "inputs (6.2 GB packed) far larger than L2"},
        "e2e": {"value": ms / 1e3, "unit": "s/batch-of-256", "h2d_bytes_per_step": 2 * npk * 8,
                "d2h_bytes_per_step": npk * 8,
                "timing": "host wall clock of the whole C call (packed host arrays in and out, copies inside), "
                          "median of the timed calls"},
        "gpu_launches": int(launches),
        "roofline": {"bound": "fp64", "kernel": "k_eig_fused / k_eig_cluster (FP64 generalized eigensolver, DMMA "
                                                "tile products)",
                     "achieved": feig / (ms / 1e3) / 1e12, "peak": 37.0 * world, "unit": "TFLOP/s",
                     "frac": feig / (ms / 1e3) / 1e12 / (37.0 * world), "traffic": None,
                     "peak_kind": "nominal B200 FP64 (no measured FP64 figure on this pool)"
                                  + ("" if world == 1 else f", times {world} GPUs"),
                     "work": "7 m^3 per system (dsygvd with vectors), the whole call's wall time"},
        "cpu_baseline": cpu,
        "clocks": clocks,
    }
    if comparisons:
        line["comparisons"] = comparisons
    print(json.dumps(line), flush=True)
    ctx.close()


def run_ours(args, rank, world, local, pg):
    import torch

    from ptb_b200 import PREC_FP64, PREC_MIXED, Context, Options, synth

    peak_burst, peak_sust, hbm, peak_kind = load_peaks()
    s = synth.water_cluster(args.nmol, seed=1)
    n, nel = s.ndim, s.nel
    npk = n * (n + 1) // 2
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    dH = torch.from_numpy(s.Hvec).to(dev)
    dS = torch.from_numpy(s.Svec).to(dev)
    dP = torch.empty(npk, dtype=torch.float64, device=dev)
    hH = torch.from_numpy(s.Hvec).pin_memory()
    hS = torch.from_numpy(s.Svec).pin_memory()
    hP = torch.empty(npk, dtype=torch.float64).pin_memory()
    hHn, hSn, hPn = hH.numpy(), hS.numpy(), hP.numpy()
    prec = PREC_FP64 if args.precision == "fp64" else PREC_MIXED
    opts = Options(filter=FILTER, precision=prec)
    ctx = Context(local)
    torch.cuda.synchronize()

    def dev_step(o=opts):
        return ctx.tc_purify_device(n, nel, dH.data_ptr(), dS.data_ptr(), dP.data_ptr(), o)

    for _ in range(args.warmup):
        dev_step()
    torch.cuda.synchronize()
    barrier(pg)
    stats = []
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier(pg)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            stats.append(dev_step())
        torch.cuda.synchronize()
        wall = time.perf_counter() - t0
        barrier(pg)
        # end to end through the host C-ABI: pinned host H, S in and P out, host
        # wall clock around every call (each returns after its P is on the host)
        e2e_walls = []
        for _ in range(args.steps):
            barrier(pg)
            t1 = time.perf_counter()
            ctx.tc_purify(n, nel, hHn, hSn, opts, out=hPn)
            e2e_walls.append(time.perf_counter() - t1)
        torch.cuda.synchronize()
    clocks = clk.summary()
    ms_dev = sum(st.ms_total for st in stats) / len(stats)
    ms_dev = reduce_max(pg, ms_dev)
    ms_e2e = reduce_max(pg, 1e3 * sum(e2e_walls) / len(e2e_walls))

    # accuracy against the plain FP64 GPU path, and its time (the 10x comparator)
    fp64 = {}
    if args.compare_fp64 and rank == 0:
        Pmix = dP.cpu().numpy().copy()
        st64 = ctx.tc_purify_device(n, nel, dH.data_ptr(), dS.data_ptr(), dP.data_ptr(),
                                    Options(filter=FILTER, precision=PREC_FP64))
        P64 = dP.cpu().numpy()
        fp64 = {"s_per_step": st64.ms_total / 1e3, "iterations": st64.iterations,
                "max_abs_dP_mixed_vs_fp64": float(np.max(np.abs(Pmix - P64)))}
        chk = ctx.check_density(n, Pmix, ctx.filter_matrix_sym(s.Svec, n, FILTER),
                                ctx.filter_matrix_sym(s.Hvec, n, FILTER))
        chk64 = ctx.check_density(n, P64, ctx.filter_matrix_sym(s.Svec, n, FILTER),
                                  ctx.filter_matrix_sym(s.Hvec, n, FILTER))
        fp64.update({"nel_mixed": chk.nel, "band_energy_mixed": chk.band_energy,
                     "band_energy_fp64": chk64.band_energy,
                     "dE_band_mixed_vs_fp64": chk.band_energy - chk64.band_energy,
                     "idempotency_frob_mixed": chk.idempotency_frob,
                     "speedup_mixed_vs_fp64": (st64.ms_total / 1e3) / (ms_dev / 1e3)})

    last = stats[-1]
    # roofline of the dominant kernel: the tcgen05 product (both epilogues)
    tc_ms = (sum(x.ms_tc_sp2 + x.ms_tc_full for x in stats)) / len(stats)
    tc_n = (sum(x.n_tc_sp2 + x.n_tc_full for x in stats)) / len(stats)
    # algorithmic flops: SP2 step = symmetric square, n^2 (n+1) ~ n^3; general product 2 n^3
    alg = last.n_tc_sp2 * float(n) ** 3 + last.n_tc_full * 2.0 * float(n) ** 3
    executed = last.tc_flops   # every product of the split, every tile that ran (reported by the library)
    achieved = alg / (last.ms_tc_sp2 + last.ms_tc_full) / 1e9 if (last.ms_tc_sp2 + last.ms_tc_full) > 0 else 0.0
    exec_tf = executed / (last.ms_tc_sp2 + last.ms_tc_full) / 1e9 if (last.ms_tc_sp2 + last.ms_tc_full) > 0 else 0.0
    # measured DRAM bytes per launch of each epilogue (ncu at ndim 11776), weighted
    # by this step's launches of each; only for the workload they were measured on
    traffic = None
    tp = ROOT / "profiles" / "traffic.json"
    if tp.exists():
        tj = json.loads(tp.read_text())
        if tj.get("ndim") == n and (last.n_tc_sp2 + last.n_tc_full) > 0:
            traffic = (last.n_tc_sp2 * tj["sp2_bytes_per_launch"] + last.n_tc_full * tj["full_bytes_per_launch"]) / (
                last.n_tc_sp2 + last.n_tc_full)
    # the FP64-class products of the mixed path on the int8 tensor cores (Ozaki slices)
    oz = None
    if last.n_oz > 0 and last.ms_oz > 0:
        oz = {"kernel": "k_oz_product (tcgen05 kind::i8, exact int32 slice-pair sums)",
              "slices": opts.fp64_slices, "launches_per_step": last.n_oz, "ms_per_step_in_kernel": last.ms_oz,
              "int8_executed_tops": last.oz_ops / (last.ms_oz / 1e3) / 1e12}

    if rank != 0:
        return
    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        t = cpu_dense_full(s)
        cpu = {"value": t, "unit": UNIT, "cores": os.cpu_count(), "kind": "port",
               "sample": f"one whole call of the oracle solve2 (dsygvd + Fermi + C f C^T, scipy OpenBLAS, "
                         f"{os.cpu_count()} threads) on the ndim {n} problem"}
    line = {
        "metric": METRIC, "value": ms_dev / 1e3, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_dev, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None,
        "dtype": ("bf16x3+i8-sliced-f64+f64" if oz else "bf16x3+f64") if prec == PREC_MIXED else "f64",
        "data": "synthetic",
        "config": {"workload": f"dense density step, {args.nmol}-H2O box ({s.nat} atoms, ndim {n}, nel {nel}), "
                               "filter 1e-5, trace-correcting purification",
                   "global_batch": world, "seq_len": n, "parallelism": f"replicas x{world}",
                   "l2": "inputs and working set far larger than L2 (no flush)"},
        "tflops_algorithmic": last.flops / (last.ms_solve / 1e3) / 1e12 if last.ms_solve > 0 else None,
        "iterations": last.iterations,
        "e2e": {"value": ms_e2e / 1e3, "unit": UNIT, "h2d_bytes_per_step": 2 * npk * 8, "d2h_bytes_per_step": npk * 8,
                "timing": f"host wall clock around ptbgpu_tc_purify (pinned host buffers), mean of {args.steps} calls"},
        "gpu_launches": int(sum(x.kernel_launches for x in stats)),
        "roofline": {"bound": "tensor", "kernel": "k_tc_product (tcgen05 bf16x3)",
                     "achieved": achieved, "peak": peak_sust, "unit": "TFLOP/s",
                     "frac": achieved / peak_sust if peak_sust else None, "traffic": traffic,
                     "peak_kind": f"{peak_kind} bf16 sustained",
                     "executed_tflops": exec_tf, "executed_frac": exec_tf / peak_sust if peak_sust else None,
                     "launches_per_step": tc_n, "ms_per_step_in_kernel": tc_ms},
        "cpu_baseline": cpu,
        "clocks": clocks,
        "wall_s_timed": wall,
    }
    if oz:
        line["int8_fp64_products"] = oz
    if fp64:
        line["fp64_gpu"] = fp64
    print(json.dumps(line), flush=True)
    ctx.close()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--precision", choices=["mixed", "fp64"], default="mixed")
    ap.add_argument("--no-compare-fp64", dest="compare_fp64", action="store_false")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--workload", choices=["water512", "lattice256", "purify_types"] + sorted(SM_WORKLOADS),
                    default="water512")
    ap.add_argument("--workers", type=int, default=8, help="worker streams of the lattice256 batch")
    ap.add_argument("--ref-budget", type=float, default=240.0,
                    help="wall-clock seconds the reference arm may spend on whole timed calls (at least one runs)")
    ap.add_argument("--nmol", type=int, default=512,
                    help="water molecules in the box (512 = the benchmark workload; smaller boxes for profiling)")
    args = ap.parse_args()
    if args.impl == "reference":
        rank = int(os.environ.get("RANK", "0"))
        run_reference(args, rank)
        return
    # libptbgpu first: its cuBLAS / cuSOLVER dependencies then resolve to the CUDA
    # toolkit it was built against rather than to the copies bundled with torch.
    from ptb_b200 import load_library
    load_library()
    rank, world, local, pg = dist_setup(args.gpus)
    try:
        if args.workload == "lattice256":
            run_batch(args, rank, world, local, pg)
        elif args.workload in SM_WORKLOADS:
            run_sm(args, rank, world, local, pg)
        elif args.workload == "purify_types":
            run_purify_types(args, rank, world, local, pg)
        else:
            run_ours(args, rank, world, local, pg)
    finally:
        if pg is not None:
            pg.destroy_process_group()


if __name__ == "__main__":
    main()
