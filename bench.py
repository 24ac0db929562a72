"""Benchmark: time to a 1e-8 FP64 relative residual of AMG-preconditioned CG
and BiCGStab on the 3-D 7-point variable-coefficient heat-conduction
problem, 256^3 cells (16,777,216 rows, 117,047,296 nonzeros), log-normal
conductivity, Dirichlet on one face, Neumann elsewhere (seeded synthetic
input), mixed precision (FP32 AMG hierarchy and V-cycle, FP64 outer Krylov
loop) against plain FP64 on the same GPU.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl thermofem|reference] [--size M]

A step is one solve (Solver::apply) from a zero initial guess with the
hierarchy already built.  `value` is seconds per solve of the mixed PCG;
`plain_fp64` is PCG with an FP64 hierarchy; `bicgstab` holds the same pair
for BiCGStab; `speedup_mixed_vs_fp64` is the PCG ratio.  Inputs stay resident
in HBM (the 1.4 GB FP64 operator is far larger than the 126 MB L2, so nothing
is flushed between steps).  `e2e` runs the mixed PCG through the C ABI with
pinned host buffers (rhs upload, x upload and download inside the timed
region).  `reference_gpu` is the reference's own CUDA build (compiled for
sm_100a from its sources) on the same inputs, where that build is present;
`heat3d_128` repeats the mixed/plain PCG pair on 128^3 with the error of each
solution against the CPU oracle's FP64 solve.  With N > 1 every rank solves
its own replica (a single system does not shard) and the time is the max
over ranks.  `--impl reference` times the CPU oracle (the reference has no
CPU solver; its host restatement is the baseline) on the host cores.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SIZE = 256
EXTRA_SIZE = 128
SEED_MATRIX, SEED_RHS = 1001, 1002
AMG = dict(jacobi_weight=2.0 / 3.0, pre_sweeps=1, post_sweeps=1, cycle="v", coarse_rows=64)
METRIC = "time-to-1e-8 FP64 relative residual (s), AMG-PCG V-cycle, FP32 hierarchy / FP64 outer"
# DRAM bytes (read + write) per algorithmic byte of one launch, from ncu
# captures of the same kernel and layout on a smaller case of the same
# stencil (FP64 Krylov operator, FP32 finest level of the mixed hierarchy;
# sliced and CSR row tiles on 128^3, the staged banded kernel on 192^3).  The
# operators are one stencil at every size, so traffic grows with the bytes;
# layouts without a capture report null.
TRAFFIC_RATIO = {
    ("f64", "sliced"): (163197184 + 4258048) / 179961860,
    ("f64", "csr"): (171013632 + 13778176) / 187760644,
    ("f32", "sliced"): (96349184 + 4392704) / 104726532,
    ("f32", "csr"): (104301056 + 5819136) / 112656388,
    ("f64", "banded"): 516795905 / 521662468,
    ("f32", "banded"): 262385128 / 267448324,
}
TRAFFIC_SOURCE = {"banded": "192^3"}


def traffic_source(layout):
    return (f"ncu DRAM bytes per algorithmic byte of the same kernel and layout on "
            f"{TRAFFIC_SOURCE.get(layout, '128^3')}, times this launch's algorithmic bytes")


SOLVER = "PCG / BiCGStab + aggregation AMG V(1,1), Jacobi w=2/3, coarse LU <= 64 rows, rtol 1e-8"


def workload_name(m):
    return (f"heat3d {m}^3 7-point FV, log-normal k (seed {SEED_MATRIX}), Dirichlet x=0, "
            f"rhs U[-1,1] (seed {SEED_RHS})")


def spmv_bytes(n, nnz, vsize=8, isize=4, csize=None):
    """Algorithmic bytes of one CSR SpMV: values + column entries (csize
    bytes each, default the index size), row offsets, x and y each once."""
    csize = isize if csize is None else csize
    return nnz * (vsize + csize) + n * (isize + 2 * vsize) + isize


def layout_bytes(layout, n, entries, vsize):
    """Algorithmic bytes of one SpMV over the storage it streams, x and y once:
    sliced / sorted copy: entries incl. padding x (value + 2-byte column
    offset), one 4-byte start per 32-row slice; banded copy: entries incl.
    padding x value, one 8-byte {offset, mask} per 32 entries, the slice
    starts; CSR: row offsets and per entry the value and a 2-byte column
    offset ("csr") or a 4-byte column index ("csr32")."""
    slices = ((n + 31) // 32 + 1) * 4
    if layout in ("sliced", "sorted"):
        return entries * (vsize + 2) + slices + 2 * n * vsize
    if layout == "banded":
        return entries * vsize + (entries // 32) * 8 + slices + 2 * n * vsize
    if layout == "csr32":
        return spmv_bytes(n, entries, vsize, 4, 4)
    return spmv_bytes(n, entries, vsize, 4, 2)


def kernel_name(layout, t, entries):
    """The kernel that streams a layout, and what it streams."""
    return {
        "sliced": f"sliced_kernel<{t}> over the sliced copy (32-row slices, 2-byte column offsets, {entries} entries)",
        "sorted": f"sliced_kernel<{t}> over the sorted sliced copy ({entries} entries)",
        "banded": f"the banded copy's tuned kernel over {entries} entries (32-row slices, one shared column offset "
                  f"per entry slot): sliced_pipe_kernel<{t}, group, ..., StagedBand> (values and slots bulk-copied "
                  f"into shared memory) or sliced_kernel<{t}, ..., BandCols>",
        "csr": f"csr_pipe_kernel<{t},int,short> over the CSR arrays (2-byte column offsets)",
        "csr32": f"csr_pipe_kernel<{t},int,int> over the CSR arrays (4-byte column indices)",
    }[layout]


def iteration_bytes(solver, n, op_layout, op_entries):
    """Algorithmic bytes of one PCG iteration of the mixed solve: the bytes
    model of every kernel it launches, summed.  FP64 outer loop: operator
    SpMV with p.Ap (operator bytes + p), x/r update (6 vectors), r.z fused
    with the cycle output conversion (r, z, FP32 x), p update (3 vectors),
    cycle input conversion fused with the finest zero-guess sweep (r in; dinv,
    rhs, x).  FP32 V(1,1) cycle, per level of n_d rows in the layout the cycle
    streams: residual (SpMV bytes + b), post-smooth (SpMV bytes + b + D^-1),
    prolongation (x read and written, map, coarse x), and below the finest
    level the restriction fused with the zero-guess sweep (fine residual and
    members, offsets, D^-1, b and x written); the dense coarse solve reads
    its inverse."""
    stats = solver.level_statistics()
    nb = layout_bytes(op_layout, n, op_entries, 8) + 8 * n  # SpMV with p.Ap
    nb += 6 * 8 * n + (8 + 8 + 4) * n + 3 * 8 * n + (8 + 4 + 4 + 4) * n
    for d, st in enumerate(stats):
        nd = st["rows"]
        if d + 1 == len(stats):
            nb += nd * nd * 8 + 2 * 4 * nd  # dense coarse solve
            break
        layout, entries = solver.level_spmv_layout(d)
        spmv = layout_bytes(layout, nd, entries, 4)
        nc = stats[d + 1]["rows"]
        nb += (spmv + 4 * nd) + (spmv + 8 * nd) + (8 * nd + 4 * nd + 4 * nc)
        if d > 0:
            nf = stats[d - 1]["rows"]
            nb += 4 * nf + 4 * nf + 4 * (nd + 1) + 4 * nd + 8 * nd
    return nb


def measured_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during a region."""

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = os.path.join(tempfile.gettempdir(), f"thermofem_b200_clocks_{os.getpid()}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index),
                 "--query-gpu=clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                 "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
                 "clocks_event_reasons.sw_power_cap", "--format=csv,noheader,nounits", "-lms", "100"],
                stdout=self.f, stderr=subprocess.DEVNULL)
            # the timed region starts once the sampler is producing (at most 3 s)
            deadline = time.monotonic() + 3.0
            while time.monotonic() < deadline and self.proc.poll() is None and os.path.getsize(self.path) == 0:
                time.sleep(0.02)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        rows = []
        with open(self.path) as f:
            for line in f:
                parts = [p.strip() for p in line.split(",")]
                if len(parts) >= 7:
                    try:
                        rows.append((float(parts[0]), float(parts[1]), float(parts[2]), parts[3:7]))
                    except ValueError:
                        pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k, v in enumerate(r[3]) if v.lower() == "active"})
        return {"sm_mhz": float(np.median([r[0] for r in rows])), "sm_max_mhz": max(r[1] for r in rows),
                "power_w_max": max(r[2] for r in rows), "samples": len(rows), "reasons": reasons}


def oracle_baseline(A, b, iterations, sample_iterations=10, repeats=1):
    """The CPU oracle's FP64 AMG-PCG on the host cores: its setup, then
    `repeats` bounded samples of `sample_iterations` PCG iterations, each
    scaled to `iterations` (the full solve's count).  Returns (setup_s,
    [seconds per full solve, one per sample], threads)."""
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    from oracle import oracle as O
    t0 = time.perf_counter()
    amg = O.Amg(A, jacobi_weight=AMG["jacobi_weight"], coarse_rows=AMG["coarse_rows"])
    setup_s = time.perf_counter() - t0
    k = min(sample_iterations, iterations)
    times = []
    for _ in range(repeats):
        t0 = time.perf_counter()
        O.cg(A, amg, b, np.zeros(A.rows), max_iterations=k)
        times.append((time.perf_counter() - t0) * iterations / k)
    return setup_s, times, O.num_threads()


def run_reference(args):
    """The CPU oracle (OpenMP, all host cores) on the same workload and metric:
    the reference has no CPU solver, so its host restatement is the baseline.
    A step is a bounded sample of 10 PCG iterations scaled to the iteration
    count of the full FP64 solve (one full solve first, where it fits the
    time budget, gives that count; otherwise the count the FP64 solve takes on
    the GPU on this problem)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
    from oracle import oracle as O
    from thermofem_b200 import problems as P
    m = args.size or SIZE
    off, idx, val = P.heat3d(m, SEED_MATRIX)
    n = len(off) - 1
    b = P.rhs_uniform(n, SEED_RHS)
    A = O.Csr(n, off, idx, val)
    t0 = time.perf_counter()
    amg = O.Amg(A, jacobi_weight=AMG["jacobi_weight"], coarse_rows=AMG["coarse_rows"])
    setup_s = time.perf_counter() - t0
    # the full solve's iteration count: solved here when that is cheap (small
    # sizes), else the count of the FP64 hierarchy on this problem (the GPU's
    # FP64 solve takes the oracle's iterations: same hierarchy, same recurrence)
    known = {128: 99, 256: 138}
    if m in known:
        iterations = known[m]
        how = f"{iterations} iterations (the FP64 solve's count on this problem)"
    else:
        _, rep = O.cg(A, amg, b, np.zeros(n))
        iterations = rep["iterations"]
        how = f"{iterations} iterations (one full solve)"
    k = min(10, iterations)
    times = []
    for step in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        O.cg(A, amg, b, np.zeros(n), max_iterations=k)
        t = (time.perf_counter() - t0) * iterations / k
        if step >= args.warmup:
            times.append(t)
    value = float(np.median(times))
    cores = O.num_threads()
    sample = f"{k} PCG iterations per step, scaled to the full solve's {how}"
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": "s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": value * 1e3, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded generator)",
            "config": {"workload": workload_name(m), "rows": n, "nnz": int(len(idx)), "solver": SOLVER,
                       "parallelism": f"host OpenMP, {cores} threads (CPU oracle, FP64 hierarchy)"},
            "iterations": iterations, "setup_s": setup_s,
            "cpu_baseline": {"value": value, "unit": "s", "cores": cores, "kind": "port", "sample": sample},
            "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_workload(args):
    """Measurements of the other benchmark configurations (synthetic inputs of the
    stated shapes; device times from CUDA events).  The batched workload
    shards its systems over the ranks of a torchrun launch (longest first to
    the least loaded rank, no data-path collective; the time is the max over
    ranks); the single-system workloads run on one GPU."""
    import torch
    import thermofem_b200 as tf
    from thermofem_b200 import problems as P
    from thermofem_b200 import shard

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if args.workload == "batched" and world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    elif rank != 0:
        return
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ctx = tf.Context(local)

    def events():
        return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)

    if args.workload == "batched":
        count, steps = 48, 20
        params = P.batched_transient_params(count, seed=1004)
        weights = [P.transient3d_nnz(m) for m, _ in params]
        mine = shard.assign(weights, world)[rank]
        probs = P.batched_transient(count, seed=1004, only=mine)
        solvers = []
        t0 = time.perf_counter()
        for m, r, mat, _ in probs:
            s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(hierarchy_type="f32", **AMG, **_small(args)),
                      ctx=ctx)
            s.setup(tf.DeviceCsr.from_host(*mat, device=dev))
            solvers.append(s)
        setup_s = time.perf_counter() - t0
        batch = tf.Batch(solvers, ctx=ctx) if solvers else None
        t_init = [torch.tensor(p[3], device=dev) for p in probs]

        def maxover(v):
            if dist is None:
                return v
            t = torch.tensor([v], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            return float(t.item())

        out = {}
        reports = []
        for mode in ("batched", "one_by_one", "batched"):
            temps = [t.clone() for t in t_init]
            its = [0] * len(probs)
            ok = [True] * len(probs)
            if dist is not None:
                dist.barrier()
            torch.cuda.synchronize(dev)
            e0, e1 = events()
            e0.record(ctx.stream)
            for _ in range(steps):
                rhs = [t / p[1] for t, p in zip(temps, probs)]
                xs = [t.clone() for t in temps]
                if not solvers:
                    reps = []
                elif mode == "batched":
                    reps = batch.apply(rhs, xs)
                else:
                    reps = [s.apply(b, x) for s, b, x in zip(solvers, rhs, xs)]
                for i, rep in enumerate(reps):
                    its[i] += rep["iterations"]
                    ok[i] = ok[i] and rep["status"] == "Converged"
                temps = xs
            e1.record(ctx.stream)
            torch.cuda.synchronize(dev)
            if dist is not None:
                dist.barrier()
            s_step = maxover(e0.elapsed_time(e1) / 1e3 / steps)
            reports = [{"iterations": it, "converged": c} for it, c in zip(its, ok)]
            out[mode] = {"s_per_step": s_step}
        everything = shard.gather_reports(reports, mine, count)
        setup_s = maxover(setup_s)
        for mode in out:
            out[mode]["iterations"] = sum(r["iterations"] for r in everything)
            out[mode]["converged"] = all(r["converged"] for r in everything)
        if rank == 0:
            rows = sum(m ** 3 for m, _ in params)
            print(json.dumps({
                "workload": f"batched transient: {count} backward-Euler 3-D 7-point problems, sides U{{16..96}} "
                            f"({rows} rows in all), r = dt k/h^2 U[0.1,10], {steps} steps, AMG-PCG V FP32 / FP64 "
                            "outer, rtol 1e-8",
                "metric": f"seconds per time step (all {count} systems)", "unit": "s", "n_gpus": world,
                "scaling": "strong",
                "parallelism": "systems sharded over ranks by nonzeros (longest first), no data-path collective"
                               if world > 1 else "single GPU",
                "imbalance": shard.imbalance(weights, shard.assign(weights, world)),
                "batched": out["batched"], "one_by_one": out["one_by_one"],
                "speedup_batched": out["one_by_one"]["s_per_step"] / out["batched"]["s_per_step"],
                "setup_s": setup_s, "data": "synthetic (seeded generator)"}), flush=True)
        del batch, solvers
        if dist is not None:
            dist.destroy_process_group()
        return
    if args.workload == "learned":
        from thermofem_b200 import learned as L
        m = args.size or 256
        res = L.evaluate(L.load(ctx=ctx), m, ctx=ctx)
        print(json.dumps({
            "workload": f"heat3d {m}^3 (seed 9000, held out), AMG F(1,1) FP32 hierarchy / FP64 outer, rtol 1e-8; "
                        "learned per-row Jacobi damping (trained on 200 problems of sides 32..64) vs fixed w=2/3",
            "metric": "time-to-1e-8 FP64 relative residual (ms) and iterations", "unit": "ms",
            **res, "data": "synthetic (seeded generator)"}), flush=True)
        return
    if args.workload == "convdiff":
        m = args.size or 192
        off, idx, val = P.convdiff3d(m, 1003)
        kind, label, cycle = tf.BiCgStab, "BiCGStab + AMG W-cycle", "w"
    else:
        m = args.size or 256
        off, idx, val = P.heat3d(m, SEED_MATRIX)
        kind, label, cycle = tf.Cg, "PCG + AMG V-cycle", "v"
    n = len(off) - 1
    a = tf.DeviceCsr.from_host(off, idx, val)
    del off, idx, val
    b = torch.tensor(P.rhs_uniform(n, SEED_RHS), device="cuda")
    res = {}
    for hier in ("f32", "f64", "f32v"):
        opts = dict(AMG, cycle=cycle)
        s = kind(tf.solver_options(), "amg", tf.amg_options(hierarchy_type=hier, **opts, **_small(args)), ctx=ctx)
        t0 = time.perf_counter()
        s.setup(a)
        torch.cuda.synchronize()
        setup_s = time.perf_counter() - t0
        times = []
        for k in range(1 + args.steps):
            x = torch.zeros(n, dtype=torch.float64, device="cuda")
            e0, e1 = events()
            e0.record(ctx.stream)
            rep = s.apply(b, x)
            e1.record(ctx.stream)
            torch.cuda.synchronize()
            if k:
                times.append(e0.elapsed_time(e1) / 1e3)
        r = tf.residual(a, b, x, ctx=ctx)
        true_rel = float(torch.linalg.norm(r) / torch.linalg.norm(b))
        res[hier] = {"s": sorted(times)[len(times) // 2], "iterations": rep["iterations"], "status": rep["status"],
                     "true_relative_residual": true_rel, "setup_s": setup_s}
        del s
    print(json.dumps({
        "workload": f"{args.workload} {m}^3 ({n} rows, {a.nnz} nnz), {label}, Jacobi w=2/3 V/W(1,1), rtol 1e-8",
        "metric": "time-to-1e-8 FP64 relative residual (s), median", "unit": "s",
        "mixed_f32_hierarchy": res["f32"], "plain_fp64": res["f64"],
        "speedup_mixed_vs_fp64": res["f64"]["s"] / res["f32"]["s"],
        "f32_operators_f64_cycle": res["f32v"], "speedup_f32_operators_vs_fp64": res["f64"]["s"] / res["f32v"]["s"],
        "data": "synthetic (seeded generator)"}),
        flush=True)


def _small(args):
    return {} if args.small_level_rows is None else {"small_level_rows": args.small_level_rows}


def run_profile(args):
    """The kernels of whole solves, for an ncu launch list: setup and warm-up
    solves first (skip their launches with ncu -s), then args.steps solves.
    --profile spmv: the FP64 operator SpMV instead (NVTX range "spmv")."""
    import torch
    import thermofem_b200 as tf
    from thermofem_b200 import problems as P
    off, idx, val = P.heat3d(args.size or SIZE, SEED_MATRIX)
    n = len(off) - 1
    ctx = tf.Context(0)
    a = tf.DeviceCsr.from_host(off, idx, val)
    b = torch.tensor(P.rhs_uniform(n, SEED_RHS), device="cuda")
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    if args.profile == "spmv":
        s = tf.Cg(tf.solver_options(), "identity", ctx=ctx)
        s.setup(a)
        for _ in range(args.warmup):
            s.spmv(b, x)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("spmv")  # ncu --nvtx --nvtx-include "spmv/"
        for _ in range(args.steps):
            s.spmv(b, x)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile": "spmv", "rows": n, "nnz": len(idx), "layout": s.spmv_layout()}), flush=True)
        return
    if args.profile == "spmv32":
        # the FP32 finest level of the mixed hierarchy, as level_spmv streams it
        s = tf.Cg(tf.solver_options(), "amg", tf.amg_options(hierarchy_type="f32", **AMG, **_small(args)), ctx=ctx)
        s.setup(a)
        x32, y32 = b.float(), torch.empty(n, dtype=torch.float32, device="cuda")
        for _ in range(args.warmup):
            s.level_spmv(0, x32, y32)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("spmv")  # ncu --nvtx --nvtx-include "spmv/"
        for _ in range(args.steps):
            s.level_spmv(0, x32, y32)
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_pop()
        print(json.dumps({"profile": "spmv32", "rows": n, "nnz": len(idx), "layout": s.level_spmv_layout(0)}),
              flush=True)
        return
    s = tf.Cg(tf.solver_options(), "amg",
              tf.amg_options(hierarchy_type="f32" if args.profile == "mixed" else "f64", **AMG, **_small(args)),
              ctx=ctx)
    s.setup(a)
    s.set_graph_mode(0)  # per-iteration graphs: ncu cannot profile inside conditional graph nodes
    ctx.synchronize()
    l0 = ctx.launches
    for _ in range(args.warmup):
        x.zero_()
        s.apply(b, x)
    l1 = ctx.launches
    for _ in range(args.steps):
        x.zero_()
        torch.cuda.synchronize()
        torch.cuda.nvtx.range_push("solve")  # ncu --nvtx --nvtx-include "solve/"
        rep = s.apply(b, x)
        torch.cuda.nvtx.range_pop()
    ctx.synchronize()
    print(json.dumps({"profile": args.profile, "setup_launches": l0, "warmup_launches": l1 - l0,
                      "timed_launches": ctx.launches - l1, "iterations": rep["iterations"]}), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="thermofem", choices=["thermofem", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the cpu_baseline leg")
    ap.add_argument("--no-reference-gpu", action="store_true", help="skip the reference GPU build leg")
    ap.add_argument("--small-level-rows", type=int, default=None,
                    help="tf_amg_options.small_level_rows (default: the library default)")
    ap.add_argument("--profile", choices=["mixed", "fp64", "spmv", "spmv32"], default=None,
                    help="profiling run: setup, --warmup solves, then --steps solves of one path (spmv: the FP64 "
                         "operator SpMV; spmv32: the FP32 finest level's)")
    ap.add_argument("--workload", choices=["batched", "convdiff", "heat", "learned"], default=None,
                    help="the other benchmark configurations (one JSON line each, not the headline): batched = 48 "
                         "transient systems x 20 steps; convdiff = 192^3 BiCGStab W-cycle; heat = --size^3 heat; "
                         "learned = shipped damping model vs w=2/3 on --size^3 (default 256), F-cycle")
    ap.add_argument("--size", type=int, default=None,
                    help="grid side (headline and reference arm: default 256; --workload convdiff/heat/learned)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.profile:
        return run_profile(args)
    if args.workload:
        return run_workload(args)
    return headline(args)


def headline(args):
    import torch
    import thermofem_b200 as tf
    from thermofem_b200 import problems as P

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    m = args.size or SIZE
    lead = rank == 0 and world == 1  # the host-side legs run once, on a single-GPU run

    off, idx, val = P.heat3d(m, SEED_MATRIX)
    n, nnz = len(off) - 1, len(idx)
    b_host = torch.tensor(P.rhs_uniform(n, SEED_RHS))
    ctx = tf.Context(local)
    a = tf.DeviceCsr.from_host(off, idx, val, device=dev)
    b = b_host.to(dev)
    x = torch.zeros(n, dtype=torch.float64, device=dev)

    def barrier():
        if dist is not None:
            dist.barrier()

    def maxover(v):
        if dist is None:
            return v
        t = torch.tensor([v], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def make(kind, hier, a=a):
        cls = tf.Cg if kind == "cg" else tf.BiCgStab
        s = cls(tf.solver_options(torch.float64), "amg", tf.amg_options(hierarchy_type=hier, **AMG, **_small(args)),
                ctx=ctx)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        s.setup(a)
        ctx.synchronize()
        return s, time.perf_counter() - t0

    def timed(s, b, x, steps):
        def solve():
            x.zero_()
            rep = s.apply(b, x)
            assert rep["status"] == "Converged", rep
            return rep
        for _ in range(args.warmup):
            solve()
        barrier()
        torch.cuda.synchronize(dev)
        launches0 = ctx.launches
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ctx.stream)
        for _ in range(steps):
            rep = solve()
        e1.record(ctx.stream)
        torch.cuda.synchronize(dev)
        barrier()
        ms = e0.elapsed_time(e1) / steps
        return maxover(ms), rep, ctx.launches - launches0

    def true_residual(a, b, x):
        r = tf.residual(a, b, x, ctx=ctx)
        return float(torch.linalg.norm(r) / torch.linalg.norm(b))

    # ---- the four solves: {PCG, BiCGStab} x {FP32 hierarchy, FP64 hierarchy}
    runs = {}
    keep = {}
    with Clocks(local) as clk:
        for kind in ("cg", "bicgstab"):
            for hier in ("f32", "f64"):
                s, setup_s = make(kind, hier)
                ms, rep, launches = timed(s, b, x, args.steps)
                runs[(kind, hier)] = {"ms": ms, "iterations": rep["iterations"], "setup_s": setup_s,
                                      "true_relative_residual": true_residual(a, b, x),
                                      "setup_phases_ms": {k: round(v, 3) for k, v in s.setup_phases().items()},
                                      "launches": launches}
                if kind == "cg":
                    keep[hier] = s
                else:
                    del s
    clocks = clk.summary()
    mixed, plain = keep["f32"], keep["f64"]
    pcg_mixed = runs[("cg", "f32")]

    # ---- e2e: the public C ABI call with pinned host buffers, the copies inside
    # the timed region (a zeroed pinned initial guess per step, prepared outside it)
    hb = b_host.pin_memory()
    hxs = [torch.zeros(n, dtype=torch.float64).pin_memory() for _ in range(args.steps + 2)]
    for hx in hxs[:2]:
        mixed.apply(hb, hx)
    barrier()
    t0 = time.perf_counter()
    for hx in hxs[2:]:
        rep_e2e = mixed.apply(hb, hx)
    e2e_s = maxover((time.perf_counter() - t0) / args.steps)
    del hxs
    assert rep_e2e["status"] == "Converged"

    # ---- roofline of the dominant kernel family of the mixed solve, the FP32
    # level SpMV, on its finest level as the cycle streams it; beside it the
    # FP64 Krylov operator SpMV
    def time_launch(fn, reps=50):
        for _ in range(5):
            fn()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ctx.stream)
        for _ in range(reps):
            fn()
        e1.record(ctx.stream)
        torch.cuda.synchronize(dev)
        return e0.elapsed_time(e1) / reps

    # In the cycle, other levels and the outer loop run between two launches
    # of the finest level, so it is timed cold: before every launch a 192 MB
    # READ leaves the 126 MB L2 holding other, clean lines (a written flush
    # would leave dirty lines for the timed kernel to write back).
    flush = torch.ones(48 << 20, dtype=torch.int32, device=dev)

    def time_launch_cold(fn, reps=20):
        for _ in range(3):
            fn()
        pairs = []
        for _ in range(reps):
            with torch.cuda.stream(ctx.stream):
                flush.sum()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(ctx.stream)
            fn()
            e1.record(ctx.stream)
            pairs.append((e0, e1))
        torch.cuda.synchronize(dev)
        return sum(e0.elapsed_time(e1) for e0, e1 in pairs) / reps

    y = torch.empty_like(b)
    b32 = b.float()
    y32 = torch.empty_like(b32)
    spmv_ms = time_launch(lambda: plain.spmv(b, y))
    spmv32_ms = time_launch_cold(lambda: mixed.level_spmv(0, b32, y32))
    del flush
    csr_ms = time_launch(lambda: tf.spmv(a, b, y, ctx=ctx))
    peak, peak_kind = measured_peaks()
    layout, entries = plain.spmv_layout()
    layout32, entries32 = mixed.level_spmv_layout(0)
    algo = layout_bytes(layout, n, entries, 8)
    achieved = algo / (spmv_ms * 1e-3) / 1e9
    algo32 = layout_bytes(layout32, n, entries32, 4)
    achieved32 = algo32 / (spmv32_ms * 1e-3) / 1e9
    achieved_csr = spmv_bytes(n, nnz) / (csr_ms * 1e-3) / 1e9
    traffic = TRAFFIC_RATIO[("f64", layout)] * algo if ("f64", layout) in TRAFFIC_RATIO else None
    traffic32 = TRAFFIC_RATIO[("f32", layout32)] * algo32 if ("f32", layout32) in TRAFFIC_RATIO else None

    # solve-level effective bandwidth: the bytes model of one iteration over
    # the measured time per iteration
    it_bytes = iteration_bytes(mixed, n, *mixed.spmv_layout())
    solve_gbs = it_bytes * pcg_mixed["iterations"] / (pcg_mixed["ms"] * 1e-3) / 1e9
    del mixed, plain, keep

    # ---- 128^3: the same pair, and each solution against the CPU oracle's
    # FP64 solve (the oracle finishes that size in seconds)
    extra = None
    if m != EXTRA_SIZE:
        off2, idx2, val2 = P.heat3d(EXTRA_SIZE, SEED_MATRIX)
        n2 = len(off2) - 1
        a2 = tf.DeviceCsr.from_host(off2, idx2, val2, device=dev)
        b2_host = P.rhs_uniform(n2, SEED_RHS)
        b2 = torch.tensor(b2_host, device=dev)
        x2 = torch.zeros(n2, dtype=torch.float64, device=dev)
        extra = {"workload": workload_name(EXTRA_SIZE), "rows": n2, "nnz": int(len(idx2))}
        xs2 = {}
        for hier in ("f32", "f64"):
            s, setup_s = make("cg", hier, a=a2)
            ms, rep, _ = timed(s, b2, x2, args.steps)
            extra["mixed" if hier == "f32" else "plain_fp64"] = {
                "value": ms / 1e3, "unit": "s", "iterations": rep["iterations"], "setup_s": setup_s,
                "true_relative_residual": true_residual(a2, b2, x2)}
            xs2[hier] = x2.cpu().numpy()
            del s
        extra["speedup_mixed_vs_fp64"] = extra["plain_fp64"]["value"] / extra["mixed"]["value"]
        if lead and not args.no_cpu:
            try:
                subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "oracle")], check=True)
                from oracle import oracle as O
                A2 = O.Csr(n2, off2, idx2, val2)
                xo, orep = O.cg(A2, O.Amg(A2, jacobi_weight=AMG["jacobi_weight"], coarse_rows=AMG["coarse_rows"]),
                                b2_host, np.zeros(n2))
                for hier, key in (("f32", "mixed"), ("f64", "plain_fp64")):
                    extra[key]["relative_error_vs_oracle"] = float(np.linalg.norm(xs2[hier] - xo) /
                                                                   np.linalg.norm(xo))
                extra["oracle_iterations"] = orep["iterations"]
            except Exception as e:  # reported, never required
                extra["oracle"] = f"failed: {e}"
        del a2

    # ---- the reference's own CUDA build on the same inputs
    reference_gpu = None
    if lead and not args.no_reference_gpu:
        try:
            from oracle import oracle as O
            if O.ref_gpu_available():
                torch.cuda.synchronize(dev)
                r = O.ref_gpu_solve_pair(O.Csr(n, off, idx, val), b_host.numpy(),
                                         jacobi_weight=AMG["jacobi_weight"], coarse_rows=AMG["coarse_rows"],
                                         repeats=2)
                reference_gpu = {
                    "build": "the reference's library sources compiled with nvcc for sm_100a (cuSPARSE, cuBLAS, CUB)",
                    "setup_s": r["setup_s"], "timing": "host clock around device-synchronised calls, best of 2",
                    "pcg": {k: r["pcg"][k] for k in ("solve_s", "iterations", "relative_residual")},
                    "bicgstab": {k: r["bicgstab"][k] for k in ("solve_s", "iterations", "relative_residual")}}
                reference_gpu["pcg_speedup"] = {
                    "mixed": r["pcg"]["solve_s"] / (runs[("cg", "f32")]["ms"] / 1e3),
                    "plain_fp64": r["pcg"]["solve_s"] / (runs[("cg", "f64")]["ms"] / 1e3)}
                reference_gpu["bicgstab_speedup"] = {
                    "mixed": r["bicgstab"]["solve_s"] / (runs[("bicgstab", "f32")]["ms"] / 1e3),
                    "plain_fp64": r["bicgstab"]["solve_s"] / (runs[("bicgstab", "f64")]["ms"] / 1e3)}
            else:
                reference_gpu = {"unavailable": "oracle/_ref/libref_gpu.so was not built (reference sources absent)"}
        except Exception as e:  # reported, never required
            reference_gpu = {"unavailable": f"failed: {e}"}

    # ---- the CPU oracle on the host cores (bounded sample)
    cpu = None
    if lead and not args.no_cpu:
        try:
            from oracle import oracle as O
            setup_cpu, times, cores = oracle_baseline(O.Csr(n, off, idx, val), b_host.numpy(),
                                                      runs[("cg", "f64")]["iterations"])
            cpu = {"value": times[0], "unit": "s", "cores": cores, "kind": "port",
                   "sample": f"10 FP64 AMG-PCG iterations of the same {m}^3 problem on the oracle's hierarchy "
                             f"(built in {setup_cpu:.1f} s, not counted), scaled to the FP64 solve's "
                             f"{runs[('cg', 'f64')]['iterations']} iterations"}
        except Exception as e:  # the baseline is reported, never required
            cpu = {"value": None, "unit": "s", "cores": None, "kind": "port", "sample": f"failed: {e}"}

    if rank == 0:
        def pair(kind):
            mx, pl = runs[(kind, "f32")], runs[(kind, "f64")]
            return {"mixed": {"value": mx["ms"] / 1e3, "unit": "s", "iterations": mx["iterations"],
                              "true_relative_residual": mx["true_relative_residual"], "setup_s": mx["setup_s"]},
                    "plain_fp64": {"value": pl["ms"] / 1e3, "unit": "s", "iterations": pl["iterations"],
                                   "true_relative_residual": pl["true_relative_residual"], "setup_s": pl["setup_s"]},
                    "speedup_mixed_vs_fp64": pl["ms"] / mx["ms"]}
        kernel32 = f"SpMV, FP32 finest AMG level: {kernel_name(layout32, 'float', entries32)}"
        kernel64 = f"SpMV, FP64 Krylov operator: {kernel_name(layout, 'double', entries)}"
        line = {
            "metric": METRIC, "value": pcg_mixed["ms"] / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": pcg_mixed["ms"], "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64 outer / f32 hierarchy", "data": "synthetic (seeded generator)",
            "config": {"workload": workload_name(m), "rows": n, "nnz": nnz, "solver": SOLVER,
                       "parallelism": "replicas" if world > 1 else "single GPU",
                       "l2": "inputs larger than L2 (1.4 GB FP64 operator), no flush"},
            "iterations": pcg_mixed["iterations"], "true_relative_residual": pcg_mixed["true_relative_residual"],
            "setup_s": pcg_mixed["setup_s"], "setup_phases_ms": pcg_mixed["setup_phases_ms"],
            "plain_fp64": {"value": runs[("cg", "f64")]["ms"] / 1e3, "unit": "s",
                           "iterations": runs[("cg", "f64")]["iterations"],
                           "true_relative_residual": runs[("cg", "f64")]["true_relative_residual"],
                           "setup_s": runs[("cg", "f64")]["setup_s"],
                           "setup_phases_ms": runs[("cg", "f64")]["setup_phases_ms"]},
            "speedup_mixed_vs_fp64": runs[("cg", "f64")]["ms"] / pcg_mixed["ms"],
            "pcg": pair("cg"), "bicgstab": pair("bicgstab"),
            "reference_gpu": reference_gpu,
            "heat3d_128": extra,
            "spmv_gbs": {"f64_operator": achieved, "f32_level0": achieved32, "f64_int32_csr": achieved_csr},
            "solve_effective_gbs": {"value": solve_gbs, "bytes_per_iteration": it_bytes,
                                    "model": "sum over one iteration's kernels of their algorithmic bytes"},
            "roofline": {"bound": "hbm", "achieved": achieved32, "peak": peak, "unit": "GB/s",
                         "frac": achieved32 / peak, "traffic": traffic32, "kernel": kernel32,
                         "share": "the FP32 level SpMV family takes the largest share of the mixed solve's "
                                  "device time in its ncu launch list",
                         "peak_source": peak_kind, "algorithmic_bytes": algo32, "launch_ms": spmv32_ms,
                         "timing": "cold (L2 evicted by a read before each launch), CUDA events",
                         "traffic_source": traffic_source(layout32)},
            "roofline_fp64_operator": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                                       "frac": achieved / peak, "traffic": traffic, "kernel": kernel64,
                                       "peak_source": peak_kind, "algorithmic_bytes": algo, "launch_ms": spmv_ms,
                                       "traffic_source": traffic_source(layout)},
            "cpu_baseline": cpu,
            "e2e": {"value": e2e_s, "unit": "s", "h2d_bytes_per_step": 2 * n * 8, "d2h_bytes_per_step": n * 8},
            "gpu_launches": int(pcg_mixed["launches"]),
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
