"""Benchmark of the PDHG path: LP solves per second at relative KKT 1e-6.

Workload (default): the 60-case refinery-shaped case stack - 24 period blocks
of 115 rows x 160 columns (2,760 x 3,840, 43,412 nonzeros), every case
sharing the matrix and differing from the base in one cost, supply bound,
demand or capacity - solved by the engine as one batched FP32 run with FP64
restart/termination checks, to relative KKT 1e-6. A step is one solve of the
whole stack; `value` is cases solved per second with the stack's data already
on the device; `e2e` is the same metric through the C ABI from host arrays
(create + solve + download inside the timed region).

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]
                    [--workload stack|spmv|packed|adjoint|powerlaw|seam]

Two side measurements ride on the stack line:
  * `spmv`: the single-LP iteration (the two fused SpMV kernels) on the
    200,000 x 300,000 power-law LP (2.4M nonzeros), FP32 and FP64, timed over
    a fixed number of iterations with CUDA events - per-iteration time,
    iterations/s and algorithmic GB/s against the measured HBM peak.
    `--workload spmv` runs this leg alone (for profiling).
  * `fp64_single_case`: the same 60 cases solved one at a time by the
    engine's plain FP64 mode - the plain FP64 single-case GPU PDHG the batched
    mixed-precision run is compared with.
  * `stream`: 240 cases (the 60, four times) through a rolling stack of 64
    slots, each freed slot admitting the next case in place.

`--workload packed` times the packed batch of 256 unequal LPs instead,
`--workload adjoint` the unrolled-PDHG sensitivities of the 60-case stack, and
`--workload powerlaw --tolerance T` whole solves of the power-law LP in FP32
(with refinement) and FP64, and `--workload seam` the reference's own
solve_pdhg on its own CUDA backend against the same solver on this engine's
kernels (through the LinAlgBackend adapter); each prints its own JSON line.

Under torchrun every rank solves its own copy of the stack (weak scaling, no
collective on the data path); rank 0 prints one JSON line. `--impl reference`
times the reference's own CPU PDHG (oracle/_ref, compiled from the reference
sources; the oracle port where that is absent) on the host cores, solving the
same cases concurrently on all threads.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM = 6650.0
TOL = 1e-6
# The case stack runs to relative KKT 1e-6 with the duality gap held to 5e-7:
# the gap is relative to 1 + |c'x| + |q'y|, about twice the objective, and at
# 5e-7 every case's objective lands within 1e-6 of the dual simplex optimum
# (at 1e-6 one case of the 60 ends 1.3e-6 away, in the reference's PDHG as
# here). The hardest case's iteration count, which sets the stack's time, is
# the same. Every arm of the stack line uses these settings.
STACK_GAP_TOL = 5e-7
STACK_OPTS = dict(tolerance=TOL, gap_tolerance=STACK_GAP_TOL)
# Side legs of the default stack line, in the order they run.
SIDE_LEGS = ("spmv", "fp64_single_case", "stream", "exact_stack", "adjoint", "packed", "powerlaw",
             "powerlaw_1e8")
# The power-law LP toward relative KKT 1e-8 (FP32 with refinement, relabelled)
# under this time cap: the leg reports how far it got.
POWERLAW_1E8_SECONDS = 45.0
# DRAM bytes (read + write) per fused seg_kernel launch of 30 cases (one
# half of the split stack), mean of the primal and dual kernels, from one
# cold-cache ncu capture (profiles/seg_kernel_refinery_stack.md): 3.04 MB
# and 2.84 MB.
SEG_KERNEL_TRAFFIC = 2.94e6


def hbm_peak():
    try:
        with open(PEAKS) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM, "fallback"


# ----------------------------------------------------------------- clocks

class ClockSampler:
    """nvidia-smi clock/throttle samples every 200 ms while running."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int = 0):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------- workloads

def stack_workload(cases=None):
    from anukulan_b200 import lpgen
    st = lpgen.refinery_stack()
    if cases is not None and cases < st.num_cases:
        # The first `cases` cases: a profiling case with one launch's case
        # count of the split stack, on one stream.
        idx = list(range(cases))
        st = lpgen.CaseStack(st.base, [st.names[i] for i in idx], st.c[idx], st.q[idx],
                             st.lower[idx], st.upper[idx])
    cfg = {"workload": "refinery_case_stack", "cases": st.num_cases,
           "rows": st.base.num_rows, "cols": st.base.num_cols, "nnz": st.base.k.nnz,
           "tolerance": TOL, "gap_tolerance": STACK_GAP_TOL,
           "precision": "fp32 iterates, fp64 checks",
           "l2": "flushed (256 MiB write) before every step"}
    return st, cfg


def algorithmic_bytes_per_iteration(nnz, m, n, cases, s_a, s_x):
    """Minimum bytes one PDHG iteration moves (both fused kernels): A and A'
    read once (value + int32 index) with their row starts, and per case x
    read/written, c, l, u, anchor_x, x_bar written and read (8n) and y
    read/written, q, Kx read/written, anchor_y, anchor_kx (7m)."""
    return 2 * nnz * (s_a + 4) + 4 * (m + n + 2) + cases * s_x * (8 * n + 7 * m)


def flush_l2(torch, buf):
    buf.zero_()


def spmv_leg(iterations, device, peak, only=None, tile_threads=0):
    """Per-iteration time of the single-LP path on the power-law LP: two fused
    SpMV + step kernels per iteration, graph-captured, timed by the engine's
    CUDA events around every iteration chunk (`profile`). tile_threads: the
    products' CTA size (0: chosen by the engine's trial solves)."""
    from anukulan_b200 import lpgen, pdhg
    from anukulan_b200.abi import PRECISION_FP32, PRECISION_FP64, make_options
    lp, _ = lpgen.power_law_lp()
    m, n, nnz = lp.num_rows, lp.num_cols, lp.k.nnz
    out = {"workload": "powerlaw_lp", "rows": m, "cols": n, "nnz": nnz,
           "row_length_max": int(lp.k.row_lengths().max()), "iterations": iterations,
           "peak_GBps": peak,
           "note": "algorithmic bytes = 2 nnz (s_a + 4) + 4 (m + n + 2) + s_x (8n + 7m); "
                   "each gathered x or y element also moves a 32-byte sector through L1"}
    # *_relabelled: the same with options.locality_order (rows by length,
    # columns grouped under their first row), which gives the gathers cache
    # locality; the arithmetic and its summation order are unchanged.
    legs = (("fp32", PRECISION_FP32, 4, 0), ("fp64", PRECISION_FP64, 8, 0),
            ("fp32_relabelled", PRECISION_FP32, 4, 1), ("fp64_relabelled", PRECISION_FP64, 8, 1))
    for name, prec, size, relabel in legs:
        if only and name not in only:
            continue
        opts = make_options(tolerance=1e-12, precision=prec, max_iterations=iterations,
                            profile=1, polish_feasibility=0, polish_on_exit=0, device=device,
                            locality_order=relabel, tile_threads=tile_threads)
        r = pdhg.solve_pdhg(lp, opts)
        per_it = r.device_iteration_seconds / max(r.device_iterations, 1)
        b = algorithmic_bytes_per_iteration(nnz, m, n, 1, size, size)
        out[name] = {"setup_ms": {k: round(r.phases[k] * 1e3, 2)
                                  for k in ("scaling", "matrix_norm")},
                     "tile_trial_ms": round(r.tile_trial_seconds * 1e3, 2),
                     "product_threads": [r.row_product_threads, r.column_product_threads],
                     "us_per_iteration": per_it * 1e6, "iterations_per_second": 1.0 / per_it,
                     "algorithmic_bytes_per_iteration": b,
                     "achieved_GBps": b / per_it / 1e9, "frac": b / per_it / 1e9 / peak,
                     "kernel_launches": int(r.kernel_launches)}
    if not only or "host_scaling" in only:
        # The same set-up with scale_lp's sweeps on the host instead.
        r = pdhg.solve_pdhg(lp, make_options(max_iterations=1, polish_feasibility=0,
                                             polish_on_exit=0, device=device,
                                             scaling_on_device=0))
        out["host_scaling_setup_ms"] = {k: round(r.phases[k] * 1e3, 2)
                                        for k in ("scaling", "matrix_norm")}
    return out


def packed_leg(local_rank, steps, warmup, workers=0, cpu=True, cpu_sample=32):
    """The packed batch: 256 independent LPs, rows log-uniform in
    [500, 50,000], 1.5x as many columns, 8 nonzeros per column, FP32 with
    FP64 checks and refinement to relative KKT 1e-6. A step solves the whole
    batch, timed with CUDA events."""
    import torch
    from anukulan_b200 import lpgen, pdhg
    from anukulan_b200.abi import OPTIMAL, PRECISION_FP32, make_options
    batch = lpgen.packed_batch()
    lps = [lp for lp, _ in batch]
    opts = make_options(tolerance=TOL, precision=PRECISION_FP32, device=local_rank)
    t0 = time.perf_counter()
    solver = pdhg.PackedBatchSolver(lps, opts, workers=workers)
    create_s = time.perf_counter() - t0
    for _ in range(warmup):
        solver.solve()
    clocks = ClockSampler(local_rank)
    clocks.start()
    step_ms, solved, iters = [], 0, 0
    for _ in range(steps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        res = solver.solve()
        e1.record()
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        solved += sum(int(r.status == OPTIMAL) for r in res)
        iters += sum(r.iterations for r in res)
    clk = clocks.stop()
    used = solver.workers
    tile = int(res[0].row_product_threads) if steps else None
    solver.close()
    total = float(np.sum(step_ms))
    nnz = sum(lp.k.nnz for lp in lps)
    out = {
        "value": solved / (total / 1e3), "unit": "solves/s", "steps": steps, "warmup": warmup,
        "ms_per_step": total / steps,
        "config": {"workload": "packed_batch", "lps": len(lps),
                   "rows_total": int(sum(lp.num_rows for lp in lps)), "nnz_total": int(nnz),
                   "rows_range": [int(min(lp.num_rows for lp in lps)),
                                  int(max(lp.num_rows for lp in lps))],
                   "tolerance": TOL, "workers": used, "product_threads": tile},
        "cases_optimal": solved, "cases_attempted": len(lps) * steps,
        "iterations_per_second": iters / (total / 1e3),
        "step_ms": [round(v, 1) for v in step_ms], "create_seconds": create_s, "clocks": clk,
    }
    if cpu:
        # The reference's CPU PDHG on a uniform random sample of the batch,
        # one LP per host thread.
        import oracle
        from concurrent.futures import ThreadPoolExecutor
        rng = np.random.default_rng(0)
        sample = [lps[i] for i in rng.choice(len(lps), size=min(cpu_sample, len(lps)),
                                             replace=False)]
        threads = os.cpu_count() or 1
        use_ref = oracle.have_reference()
        fn = (lambda lp: oracle.ref_solve(lp, tolerance=TOL)) if use_ref else \
            (lambda lp: oracle.oracle_solve(lp, tolerance=TOL))
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=threads) as ex:
            ok = sum(int(r.status == OPTIMAL) for r in ex.map(fn, sample))
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": ok / dt, "unit": "solves/s", "cores": threads,
                               "kind": "reference" if use_ref else "port",
                               "sample": f"{len(sample)} LPs drawn uniformly from the batch, "
                                         f"one per host thread (cpu_backend), {dt:.1f} s"}
    return out


def run_packed(args, rank, world, local_rank):
    """--workload packed: the packed batch as the line's own workload. Rank 0
    only (the batch does not shard here)."""
    if rank != 0:
        return None
    import torch
    torch.cuda.set_device(local_rank)
    leg = packed_leg(local_rank, args.steps, args.warmup, args.packed_workers, args.cpu_baseline)
    out = {
        "metric": "LP solves/s to relative KKT 1e-6 (packed batch of unequal LPs, FP32 + FP64 checks)",
        "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32",
        "data": "synthetic (seeded generator, 256 LPs of the random known-optimum construction)",
    }
    out.update(leg)
    return out


def adjoint_leg(local_rank, steps, warmup, cpu=True, unrolled_steps=2000):
    """Sensitivities through the unrolled program: the 60-case refinery stack,
    2,000 FP32 iterations with checkpoints every 100, loss c_hat'x_T per
    case with c_hat = c (1 + 0.05 N(0,1)). A step is one forward pass (x_T
    and the losses) and one backward pass (dL/dc, dL/dq for every case)."""
    import torch
    from anukulan_b200 import lpgen, pdhg
    from anukulan_b200.abi import PRECISION_FP32, make_options
    stack, c_hat = lpgen.adjoint_case()
    ratio = c_hat / np.where(stack.base.c != 0, stack.base.c, 1.0)
    loss = stack.c * ratio
    T, R = unrolled_steps, 100
    opts = make_options(precision=PRECISION_FP32, device=local_rank)
    u = pdhg.UnrolledPdhg(stack.base, stack.c, stack.q, stack.lower, stack.upper,
                          iterations=T, checkpoint_every=R, options=opts)
    for _ in range(warmup):
        x, _ = u.forward()
        u.backward(loss)
    clocks = ClockSampler(local_rank)
    clocks.start()
    step_ms = []
    for _ in range(steps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        x, _ = u.forward()
        gc, gq = u.backward(loss)
        e1.record()
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
    clk = clocks.stop()
    tau, sigma = u.step_sizes()
    u.close()
    total = float(np.sum(step_ms))
    K = stack.num_cases
    out = {
        "value": K * steps / (total / 1e3), "unit": "case gradients/s", "steps": steps,
        "warmup": warmup, "ms_per_step": total / steps,
        "config": {"workload": "unrolled_adjoint", "cases": K, "iterations": T,
                   "checkpoint_every": R, "rows": stack.base.num_rows,
                   "cols": stack.base.num_cols},
        "step_ms": [round(v, 2) for v in step_ms], "clocks": clk,
    }
    if cpu:
        # The float64 numpy restatement of the same program and reverse mode,
        # one case on one host thread.
        from oracle import unrolled as U
        slp = U.ScaledLp(stack.case(0))
        t0 = time.perf_counter()
        U.adjoint(slp, stack.c[0], stack.q[0], loss[0], tau[0], sigma[0], T, R)
        dt = time.perf_counter() - t0
        out["cpu_baseline"] = {"value": 1.0 / dt, "unit": "case gradients/s", "cores": 1,
                               "kind": "port",
                               "sample": f"case 0, forward + reverse in numpy/scipy FP64, {dt:.2f} s"}
    return out


def run_adjoint(args, rank, world, local_rank):
    """--workload adjoint: the unrolled adjoint as the line's own workload."""
    if rank != 0:
        return None
    import torch
    torch.cuda.set_device(local_rank)
    leg = adjoint_leg(local_rank, args.steps, args.warmup, args.cpu_baseline, args.unrolled_steps)
    out = {
        "metric": f"unrolled-PDHG sensitivities/s (dL/dc, dL/dq per case, {args.unrolled_steps:,} FP32 iterations)",
        "n_gpus": 1, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32", "data": "synthetic (seeded generator, refinery-shaped 60-case stack)",
    }
    out.update(leg)
    return out


def stream_leg(st, opts, copies=4):
    """A stack of copies x 60 cases (more than one run's 64 slots), solved as a
    rolling stack: a slot freed by a converged case admits the next waiting
    case at once. Timed after one warm-up solve; device-resident handle."""
    import torch
    from anukulan_b200 import pdhg
    from anukulan_b200.abi import OPTIMAL
    c = np.concatenate([st.c] * copies)
    q = np.concatenate([st.q] * copies)
    lo = np.concatenate([st.lower] * copies)
    hi = np.concatenate([st.upper] * copies)
    solver = pdhg.CaseStackSolver(st.base, c, q, lo, hi, opts)
    solver.solve()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    res = solver.solve()
    torch.cuda.synchronize()
    dt = time.perf_counter() - t0
    solver.close()
    ok = sum(int(r.status == OPTIMAL) for r in res)
    return {"cases": len(res), "slots": 64, "optimal": ok, "seconds": dt, "value": ok / dt,
            "unit": "solves/s",
            "mode": "rolling stack: retired slots admit waiting cases at termination checks"}


def powerlaw_leg(local_rank, tolerance, precisions, locality, time_limit, peak,
                 cpu=True, cpu_iterations=2000):
    """Whole solves of the 200,000 x 300,000 power-law LP to `tolerance`, one
    per precision (FP32 iterates with FP64 checks and refinement; FP64), no
    warm-up: each solve is long. Per solve: seconds, iterations, the device
    time per iteration and its fraction of the HBM roofline (algorithmic
    bytes of one iteration), the residuals and the objective's distance from
    the planted optimum c'x0."""
    from anukulan_b200 import lpgen, pdhg
    from anukulan_b200.abi import PRECISION_FP32, PRECISION_FP64, make_options
    lp, objective = lpgen.power_law_lp()
    nnz, m, n = lp.k.nnz, lp.num_rows, lp.num_cols
    out = {"config": {"workload": "powerlaw_lp", "rows": m, "cols": n, "nnz": nnz,
                      "tolerance": tolerance, "locality_order": locality}}
    for name, prec, size in (("fp32", PRECISION_FP32, 4), ("fp64", PRECISION_FP64, 8)):
        if name not in precisions:
            continue
        opts = make_options(tolerance=tolerance, precision=prec, device=local_rank,
                            max_iterations=5_000_000, time_limit_seconds=time_limit,
                            profile=1, locality_order=locality)
        clocks = ClockSampler(local_rank)
        clocks.start()
        t0 = time.perf_counter()
        r = pdhg.solve_pdhg(lp, opts)
        dt = time.perf_counter() - t0
        clk = clocks.stop()
        us = 1e6 * r.device_iteration_seconds / max(r.device_iterations, 1)
        bytes_it = algorithmic_bytes_per_iteration(nnz, m, n, 1, size, size)
        achieved = bytes_it / (us * 1e-6) / 1e9 if r.device_iterations else None
        out[name] = {"status": r.status, "iterations": r.iterations, "seconds": dt,
                     "solves_per_second": 1.0 / dt,
                     "iterations_per_second": r.iterations / dt,
                     "restarts": r.restarts, "polished": bool(r.polished),
                     "relative_primal": r.residual.relative_primal,
                     "relative_dual": r.residual.relative_dual,
                     "relative_gap": r.residual.relative_gap,
                     "objective_error": abs(r.objective - objective) / abs(objective),
                     "setup_ms": {k: round(r.phases[k] * 1e3, 2)
                                  for k in ("scaling", "matrix_norm")},
                     "tile_trial_ms": round(r.tile_trial_seconds * 1e3, 2),
                     "product_threads": [r.row_product_threads, r.column_product_threads],
                     "us_per_iteration_device": us,
                     "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak,
                                  "unit": "GB/s", "frac": achieved / peak if achieved else None,
                                  "algorithmic_bytes_per_iteration": bytes_it},
                     "clocks": clk}
    if cpu:
        # The reference's CPU PDHG (threaded_cpu_backend with the reference's
        # own default thread count) run for a bounded number of iterations:
        # its time per iteration, and that time over the engine's iteration
        # count as a projection of its whole solve.
        import oracle
        if oracle.have_reference():
            r = oracle.ref_solve(lp, threads=-1, tolerance=tolerance,
                                 max_iterations=cpu_iterations, time_limit_seconds=600.0)
            per_it = r.phases["iterating"] / max(r.iterations, 1)
            first = out.get(precisions[0], {})
            out["cpu_baseline"] = {
                "value": 1.0 / per_it, "unit": "iterations/s",
                "cores": int(oracle.ref_lib().ref_default_thread_count()), "kind": "reference",
                "sample": f"{r.iterations} iterations of solve_pdhg on threaded_cpu_backend, "
                          f"{r.phases['iterating']:.1f} s iterating, "
                          f"{r.phases['scaling'] + r.phases['matrix_norm']:.1f} s set-up",
                "projected_solve_seconds": per_it * first.get("iterations", 0)}
    return out


def run_powerlaw(args, rank, world, local_rank):
    """--workload powerlaw: whole solves of the power-law LP as the line's
    own workload, to --tolerance."""
    if rank != 0:
        return None
    import torch
    torch.cuda.set_device(local_rank)
    peak, kind = hbm_peak()
    wanted = args.precisions.split(",")
    out = {"metric": f"power-law LP solve to relative KKT {args.tolerance:g}",
           "unit": "seconds", "higher_is_better": False, "n_gpus": 1,
           "data": "synthetic (seeded generator, planted optimum c'x0)", "peak_source": kind}
    out.update(powerlaw_leg(local_rank, args.tolerance, wanted, args.locality, args.time_limit,
                            peak, args.cpu_baseline))
    out["value"] = out[wanted[0]]["seconds"]
    return out


def run_seam(args, rank, world, local_rank):
    """The reference's own solve_pdhg, unchanged, on the power-law LP and on
    one refinery case, with the seam's arithmetic on (a) the reference's own
    cuda_backend.cu and (b) this engine's kernels through the LinAlgBackend
    adapter. Same solver, same calls, one launch per seam operation: the
    per-iteration time compares the kernels under the seam. FP64, a fixed
    number of iterations; the two arms' iterates are compared too."""
    if rank != 0:
        return None
    import torch
    import oracle
    from anukulan_b200 import lpgen
    torch.cuda.set_device(local_rank)
    kw = dict(tolerance=1e-12, max_iterations=args.seam_iterations, polish_on_exit=0,
              polish_feasibility=0)
    out = {"metric": "reference solve_pdhg, us per iteration, by backend", "unit": "us",
           "higher_is_better": False, "n_gpus": 1, "dtype": "f64",
           "config": {"workload": "seam", "iterations": args.seam_iterations},
           "data": "synthetic (seeded generators)"}
    problems = (("powerlaw_lp", lpgen.power_law_lp()[0]),
                ("refinery_case_0", lpgen.refinery_stack().case(0)))
    for name, lp in problems:
        leg = {"rows": lp.num_rows, "cols": lp.num_cols, "nnz": lp.k.nnz}
        runs = {}
        for arm, solve in (("reference_cuda_backend", oracle.ref_cuda_solve),
                           ("engine_adapter", oracle.ref_b200_solve)):
            solve(lp, **dict(kw, max_iterations=40))  # context, module load, first uploads
            r = solve(lp, **kw)
            runs[arm] = r
            leg[arm] = {"iterations": r.iterations,
                        "us_per_iteration": 1e6 * r.phases["iterating"] / max(r.iterations, 1),
                        "iterating_s": r.phases["iterating"], "checks_s": r.phases["checks"],
                        "scaling_s": r.phases["scaling"]}
        a, b = runs["reference_cuda_backend"], runs["engine_adapter"]
        leg["iterate_rel_diff"] = float(max(
            np.max(np.abs(a.x - b.x)) / max(1.0, float(np.max(np.abs(a.x)))),
            np.max(np.abs(a.y - b.y)) / max(1.0, float(np.max(np.abs(a.y))))))
        leg["speedup"] = (leg["reference_cuda_backend"]["us_per_iteration"]
                          / leg["engine_adapter"]["us_per_iteration"])
        out[name] = leg
    out["value"] = out["powerlaw_lp"]["engine_adapter"]["us_per_iteration"]
    return out


def exact_stack_leg(st, device):
    """The case stack answered exactly, the reference's stated design for
    case stacks (README.md:81-86): the engine bounds every case at once (the
    FP32 stack to relative KKT 1e-6), the engine's point for the base LP goes
    through the reference's crossover_basis and simplex, and every case is
    finished by the reference's warm dual simplex from that basis, on all
    host threads (a case whose warm start misses is finished from its own
    engine point). Beside it, the reference's family --from-first
    (app/anukulan_cli.cpp:1065-1230): a cold dual simplex on the base, then
    every case warm from its basis, on the same threads. Crossover and the
    simplex are the reference's host code, built from its sources."""
    import oracle
    from concurrent.futures import ThreadPoolExecutor
    from anukulan_b200 import pdhg
    from anukulan_b200.abi import OPTIMAL, PRECISION_FP32
    if not oracle.have_reference_b200():
        return {"unavailable": "oracle/_ref adapter build absent"}
    threads = os.cpu_count() or 1
    K = st.num_cases
    cases = [st.case(k) for k in range(K)]
    pdhg.solve_pdhg(st.base, precision=PRECISION_FP32, device=device, **STACK_OPTS)  # warm-up

    def warm_all(basis):
        def one(k):
            d, _ = oracle.ref_simplex_basis(cases[k], basis)
            return d
        with ThreadPoolExecutor(max_workers=threads) as ex:
            return list(ex.map(one, range(K)))

    t0 = time.perf_counter()
    bounds = pdhg.solve_case_stack(st, precision=PRECISION_FP32, device=device, **STACK_OPTS)
    t1 = time.perf_counter()
    base = pdhg.solve_pdhg(st.base, precision=PRECISION_FP32, device=device, **STACK_OPTS)
    t2 = time.perf_counter()
    fin = oracle.ref_finish_simplex(st.base, base.x, base.y)
    t3 = time.perf_counter()
    warm = warm_all(fin["basis"])
    misses = [k for k, d in enumerate(warm) if d["status"] != 0]
    for k in misses:
        own = oracle.ref_finish_simplex(cases[k], bounds[k].x, bounds[k].y)
        warm[k] = {"status": own["status"], "objective": own["objective"], "pivots": own["pivots"]}
    t4 = time.perf_counter()
    r0 = time.perf_counter()
    ref_base, ref_basis = oracle.ref_simplex_basis(st.base)
    ref_warm = warm_all(ref_basis)
    r1 = time.perf_counter()
    exact = sum(int(d["status"] == 0) for d in warm)
    agree = sum(int(a["status"] == 0 and b["status"] == 0 and
                    abs(a["objective"] - b["objective"]) <= 1e-9 * max(1.0, abs(b["objective"])))
                for a, b in zip(warm, ref_warm))
    bound_err = max(abs(bounds[k].objective - ref_warm[k]["objective"])
                    / max(1.0, abs(ref_warm[k]["objective"])) for k in range(K))
    return {
        "value": exact / (t4 - t0), "unit": "exact solves/s", "cases": K, "exact": exact,
        # The exact answers alone (base point, crossover, warm simplex), without
        # the stack's first-order bounds, which the reference's route does not
        # produce: the like-for-like rate against reference_family_from_first.
        "exact_only_value": exact / (t4 - t1),
        "agree_with_reference_1e-9": agree, "threads": threads,
        "seconds": {"engine_stack_bounds": t1 - t0, "engine_base_point": t2 - t1,
                    "crossover_and_base_simplex": t3 - t2, "warm_dual_simplex": t4 - t3,
                    "total": t4 - t0},
        "base_pivots": {"from_crossover": fin["pivots"], "cold": ref_base["pivots"]},
        "warm_pivots_median": float(np.median([d["pivots"] for d in warm])),
        "warm_misses": len(misses),
        "bounds_all_optimal": all(r.status == OPTIMAL for r in bounds),
        "bound_objective_max_rel_error": bound_err,
        "reference_family_from_first": {
            "value": sum(int(d["status"] == 0) for d in ref_warm) / (r1 - r0),
            "unit": "exact solves/s", "seconds": r1 - r0,
            "cold_base_seconds": ref_base["seconds"],
            "mode": "cold dual simplex on the base, every case warm from its basis, "
                    f"{threads} host threads"},
    }


def fp64_single_case(st, device):
    """The stack's cases solved one after another by the engine's plain FP64
    single-case mode, host arrays in and results out: (a) a fresh
    anu_pdhg_solve per case, (b) one handle whose scaled matrix and ||K|| are
    kept, each case swapped in by anu_pdhg_set_case (the reference's backends
    keep a prepared matrix per SparseMatrix::id() the same way)."""
    from anukulan_b200 import pdhg
    from anukulan_b200.abi import OPTIMAL, PRECISION_FP32, PRECISION_FP64, make_options
    opts = make_options(precision=PRECISION_FP64, device=device, **STACK_OPTS)
    pdhg.solve_pdhg(st.case(0), opts)  # warm-up: context, module load
    t0 = time.perf_counter()
    ok = 0
    iters = 0
    for k in range(st.num_cases):
        r = pdhg.solve_pdhg(st.case(k), opts)
        ok += int(r.status == OPTIMAL)
        iters += r.iterations
    dt = time.perf_counter() - t0
    t1 = time.perf_counter()
    h = pdhg.PdhgHandle(st.base, opts)
    ok_h = 0
    for k in range(st.num_cases):
        h.set_case(st.c[k], st.q[k], st.lower[k], st.upper[k])
        ok_h += int(h.run().status == OPTIMAL)
    h.close()
    dt_h = time.perf_counter() - t1
    # The same handle loop with FP32 iterates, FP64 checks and refinement:
    # what a caller with one LP at a time (a crossover seed, a node) gets.
    opts32 = make_options(precision=PRECISION_FP32, device=device, **STACK_OPTS)
    t2 = time.perf_counter()
    h = pdhg.PdhgHandle(st.base, opts32)
    ok_32 = 0
    for k in range(st.num_cases):
        h.set_case(st.c[k], st.q[k], st.lower[k], st.upper[k])
        ok_32 += int(h.run().status == OPTIMAL)
    h.close()
    dt_32 = time.perf_counter() - t2
    return {"value": ok_h / dt_h, "unit": "solves/s", "cases": st.num_cases, "optimal": ok_h,
            "seconds": dt_h, "iterations_per_second": iters / dt_h,
            "mode": "engine FP64, one case per run on one handle (matrix prepared once)",
            "fresh_solve_per_case": {"value": ok / dt, "unit": "solves/s", "seconds": dt,
                                     "mode": "engine FP64, anu_pdhg_solve per case"},
            "fp32_handle": {"value": ok_32 / dt_32, "unit": "solves/s", "seconds": dt_32,
                            "optimal": ok_32,
                            "mode": "engine FP32 + FP64 checks and refinement, one case per "
                                    "run on one handle"}}


# -------------------------------------------------------------- our arm

def run_engine(args, rank, world, local_rank):
    import torch
    from anukulan_b200 import pdhg
    from anukulan_b200.abi import OPTIMAL, PRECISION_FP32, make_options

    torch.cuda.set_device(local_rank)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local_rank))
    st, cfg = stack_workload(args.cases)
    opts = make_options(precision=PRECISION_FP32, device=local_rank, profile=1, **STACK_OPTS,
                        split_stacks=0 if args.no_split else 1,
                        persistent_chunks=1 if args.persistent else 0)
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device="cuda")
    # Under torchrun the workload is the stack taken `world` times, sharded by
    # case across the ranks (anukulan_b200.distributed): each rank solves its
    # contiguous slice on its own GPU and one all-gather of the results gives
    # every rank every case's answer. One rank: the stack itself, no gather.
    full = st
    if dist is not None:
        from anukulan_b200 import distributed as D
        from anukulan_b200.lpgen import CaseStack
        full = CaseStack(st.base, st.names * world, np.tile(st.c, (world, 1)),
                         np.tile(st.q, (world, 1)), np.tile(st.lower, (world, 1)),
                         np.tile(st.upper, (world, 1)))
        st = D.sub_stack(full, D.case_shard(full.num_cases, rank, world))
        cfg = dict(cfg, cases=full.num_cases)

    def barrier():
        if dist is not None:
            dist.barrier()

    def solve_all(local_solver):
        """This rank's slice, then (several ranks) the results of every case."""
        if dist is None:
            return local_solver.solve(), local_solver.solve
        res = D.solve_stack_sharded(full, solve=lambda _: local_solver.solve())
        return res, None

    # The engine runs a stack of 16 or more cases as two half-stacks of
    # alternate cases.
    split_run = st.num_cases >= 16 and not args.no_split and not args.persistent
    # value: data resident (handle created once), one solve per step
    solver = pdhg.CaseStackSolver(st.base, st.c, st.q, st.lower, st.upper, opts)
    for _ in range(args.warmup):
        res = solver.solve()
    torch.cuda.synchronize()
    clocks = ClockSampler(local_rank)
    clocks.start()
    step_ms = []
    phases = []
    dev_iter_s = 0.0
    dev_iters = 0
    launches = 0
    solved = 0
    total_iterations = 0
    for _ in range(args.steps):
        flush_l2(torch, flush)
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        res, _ = solve_all(solver)
        e1.record()
        torch.cuda.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        phases.append(res[0].phases)
        solved += sum(1 for r in res if r.status == OPTIMAL)
        dev_iter_s += res[0].device_iteration_seconds
        dev_iters += res[0].device_iterations
        # Each result counts its own half-stack's launches up to the moment it
        # was finalized; the last one of each half has them all. Under torchrun
        # the results are every rank's slice, in rank order.
        for r0 in range(0, len(res), st.num_cases):
            mine = res[r0:r0 + st.num_cases]
            halves = (mine[0::2], mine[1::2]) if (split_run and len(mine) > 1) else (mine,)
            launches += sum(max(r.kernel_launches for r in h) for h in halves if h)
        total_iterations += max(r.iterations for r in res)
    clk = clocks.stop()
    solver.close()
    # e2e: from host arrays through the C ABI, every step
    e2e_ms = []
    e2e_parts = []
    for i in range(args.warmup + args.steps if args.e2e else 0):
        flush_l2(torch, flush)
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        h0 = time.perf_counter()
        s2 = pdhg.CaseStackSolver(st.base, st.c, st.q, st.lower, st.upper, opts)
        h1 = time.perf_counter()
        r2, _ = solve_all(s2)
        h2 = time.perf_counter()
        s2.close()
        h3 = time.perf_counter()
        e1.record()
        torch.cuda.synchronize()
        if i >= args.warmup:
            e2e_ms.append(e0.elapsed_time(e1))
            e2e_parts.append((h1 - h0, h2 - h1, h3 - h2))
    total_ms = float(np.sum(step_ms))
    total_e2e = float(np.sum(e2e_ms)) if e2e_ms else float("nan")
    if dist is not None:
        t = torch.tensor([total_ms, total_e2e], device="cuda", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        total_ms, total_e2e = float(t[0]), float(t[1])
    # After the gather every rank holds every case's result.
    solved_all = solved
    cases_all = full.num_cases * args.steps
    out = None
    if rank == 0:
        peak, peak_kind = hbm_peak()
        nnz, m, n = st.base.k.nnz, st.base.num_rows, st.base.num_cols
        # The engine runs a stack of 16 or more cases as two half-stacks at
        # once (two streams): a launch carries half the cases, and two are in
        # flight at a time.
        split = st.num_cases >= 16 and not args.no_split and not args.persistent
        per_launch_cases = (st.num_cases + 1) // 2 if split else st.num_cases
        bytes_it = algorithmic_bytes_per_iteration(nnz, m, n, per_launch_cases, 4, 4)
        per_launch_s = dev_iter_s / max(dev_iters, 1) / 2.0
        achieved = (bytes_it / 2.0) / per_launch_s / 1e9 if dev_iters else None
        h2d = (st.base.k.nnz * 12 + (st.base.num_rows + 1) * 4
               + st.num_cases * 8 * (3 * n + m))
        d2h = st.num_cases * 8 * (n + m)
        out = {
            "metric": "LP solves/s to relative KKT 1e-6 (batched FP32 PDHG, FP64 checks)",
            "value": solved_all / (total_ms / 1e3),
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps,
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f32",
            "data": "synthetic (seeded generator, refinery-shaped 60-case stack)",
            "config": dict(cfg, parallelism=(f"cases sharded over {world} GPUs, one result "
                                             f"all-gather per step" if world > 1
                                             else "one GPU")),
            "cases_optimal": solved_all,
            "cases_attempted": cases_all,
            "iterations_per_solve": total_iterations / args.steps,
            "step_ms": [round(v, 2) for v in step_ms],
            "phases_ms_median": {k: round(1e3 * float(np.median([ph[k] for ph in phases])), 2)
                                 for k in phases[0]},
            "e2e": {"value": solved_all / (total_e2e / 1e3), "unit": "solves/s",
                    "h2d_bytes_per_step": int(h2d) * world, "d2h_bytes_per_step": int(d2h) * world,
                    "parts_ms_median": ({k: round(1e3 * float(np.median([p[i] for p in e2e_parts])), 2)
                                         for i, k in enumerate(("create", "solve", "close"))}
                                        if e2e_parts else None),
                    "step_ms": [round(v, 2) for v in e2e_ms]},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None,
                         "traffic": SEG_KERNEL_TRAFFIC,
                         "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                                           "cold cache, profiles/seg_kernel_refinery_stack.md",
                         "peak_source": peak_kind,
                         "kernel": "seg_kernel (fused case-stack SpMM + primal/dual step), mean per launch",
                         "algorithmic_bytes_per_launch": bytes_it / 2.0,
                         "cases_per_launch": per_launch_cases,
                         "launches_in_flight": 2 if per_launch_cases < st.num_cases else 1,
                         "launch_seconds": per_launch_s},
            "clocks": clk,
        }
        if args.cpu_baseline:
            out["cpu_baseline"] = cpu_baseline(st, seconds=args.cpu_seconds)
        legs = set(args.side_legs.split(",")) if args.side else set()
        if world > 1:
            # The other ranks would wait at the closing barrier, holding their
            # GPUs; the side legs are single-GPU measurements, taken at N=1.
            legs = set()
        if "spmv" in legs:
            out["spmv"] = spmv_leg(args.spmv_iterations, local_rank, peak)
        if "fp64_single_case" in legs:
            out["fp64_single_case"] = fp64_single_case(st, local_rank)
        if "stream" in legs:
            out["stream"] = stream_leg(st, opts)
        if "exact_stack" in legs:
            out["exact_stack"] = exact_stack_leg(st, local_rank)
        if "adjoint" in legs:
            out["adjoint"] = adjoint_leg(local_rank, steps=3, warmup=2, cpu=args.cpu_baseline)
        if "packed" in legs:
            out["packed"] = packed_leg(local_rank, steps=1, warmup=1, workers=args.packed_workers,
                                       cpu=args.cpu_baseline, cpu_sample=16)
        if "powerlaw" in legs:
            out["powerlaw"] = powerlaw_leg(local_rank, TOL, ["fp32", "fp64"], 1, 300.0, peak,
                                           cpu=args.cpu_baseline)
        if "powerlaw_1e8" in legs:
            out["powerlaw_1e8"] = powerlaw_leg(local_rank, 1e-8, ["fp32"], 1,
                                               POWERLAW_1E8_SECONDS, peak, cpu=False)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return out


def cpu_baseline(st, seconds=15.0, threads=None, prefer_reference=True):
    """The reference's CPU PDHG (or the oracle port) solving cases of the stack
    concurrently, one case per host thread, for about `seconds`."""
    import oracle
    from concurrent.futures import ThreadPoolExecutor
    from anukulan_b200.abi import OPTIMAL
    threads = threads or os.cpu_count() or 1
    use_ref = prefer_reference and oracle.have_reference()
    solve = (lambda lp: oracle.ref_solve(lp, **STACK_OPTS)) if use_ref else \
        (lambda lp: oracle.oracle_solve(lp, **STACK_OPTS))
    done = 0
    ok = 0
    t0 = time.perf_counter()
    k = 0
    with ThreadPoolExecutor(max_workers=threads) as ex:
        while time.perf_counter() - t0 < seconds or done == 0:
            batch = [st.case((k + i) % st.num_cases) for i in range(threads)]
            k += threads
            for r in ex.map(solve, batch):
                done += 1
                ok += int(r.status == OPTIMAL)
    dt = time.perf_counter() - t0
    return {"value": ok / dt, "unit": "solves/s", "cores": threads,
            "kind": "reference" if use_ref else "port",
            "sample": f"{done} cases of the stack, {threads} concurrent single-thread solves "
                      f"(cpu_backend), {dt:.1f} s"}


# ---------------------------------------------------------- reference arm

def run_reference(args, rank, world):
    if rank != 0:
        return None
    try:
        import oracle  # noqa: F401
    except Exception as e:  # pragma: no cover
        return {"impl": "reference", "unavailable": f"oracle package missing: {e}"}
    from concurrent.futures import ThreadPoolExecutor
    from anukulan_b200.abi import OPTIMAL
    st, cfg = stack_workload()
    threads = os.cpu_count() or 1
    use_ref = oracle.have_reference()
    solve = (lambda lp: oracle.ref_solve(lp, **STACK_OPTS)) if use_ref else \
        (lambda lp: oracle.oracle_solve(lp, **STACK_OPTS))
    cases = [st.case(k) for k in range(st.num_cases)]
    # A step is the engine's step: every case of the stack solved once, here
    # by single-thread solves spread over all host threads.
    step_s = []
    optimal = []
    with ThreadPoolExecutor(max_workers=threads) as ex:
        for i in range(args.warmup + args.steps):
            t0 = time.perf_counter()
            ok = sum(int(r.status == OPTIMAL) for r in ex.map(solve, cases))
            dt = time.perf_counter() - t0
            if i >= args.warmup:
                step_s.append(dt)
                optimal.append(ok)
    total = float(np.sum(step_s))
    value = float(np.sum(optimal)) / total
    kind = "reference" if use_ref else "port"
    sample = (f"the {st.num_cases}-case stack per step, {threads} concurrent single-thread "
              f"solves (cpu_backend), {args.steps} timed steps, {total:.1f} s")
    out = {
        "impl": "reference",
        "metric": "LP solves/s to relative KKT 1e-6 (batched FP32 PDHG, FP64 checks)",
        "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": total * 1e3 / args.steps,
        "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded generator, refinery-shaped 60-case stack)",
        "config": cfg,
        "cases_optimal": int(np.min(optimal)),
        "cpu_baseline": {"value": value, "unit": "solves/s", "cores": threads, "kind": kind,
                         "sample": sample},
        "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    if args.gpu_reference and oracle.have_reference_cuda():
        # A side leg: without a usable device it records why instead of
        # ending the reference arm's line.
        try:
            out["gpu_reference"] = reference_gpu_leg(st)
        except RuntimeError as e:
            out["gpu_reference"] = {"unavailable": str(e)}
    return out


def reference_gpu_leg(st, cases=None):
    """The reference's own FP64 GPU PDHG (its cuda_backend.cu, built for
    sm_100a into oracle/_ref) solving the stack's cases one at a time: the
    plain FP64 single-case GPU PDHG."""
    import oracle
    from anukulan_b200.abi import OPTIMAL
    ks = range(st.num_cases) if cases is None else cases
    oracle.ref_cuda_solve(st.case(0), **STACK_OPTS)  # context and module load
    t0 = time.perf_counter()
    ok = 0
    iters = 0
    for k in ks:
        r = oracle.ref_cuda_solve(st.case(k), **STACK_OPTS)
        ok += int(r.status == OPTIMAL)
        iters += r.iterations
    dt = time.perf_counter() - t0
    return {"value": ok / dt, "unit": "solves/s", "cases": len(ks), "optimal": ok,
            "seconds": dt, "iterations_per_second": iters / dt,
            "mode": "reference solve_pdhg on its cuda_backend, FP64, one case per call"}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="engine", choices=["engine", "reference"])
    ap.add_argument("--no-cpu-baseline", dest="cpu_baseline", action="store_false")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--cases", type=int, default=None,
                    help="solve only the first N cases of the stack (profiling)")
    ap.add_argument("--no-gpu-reference", dest="gpu_reference", action="store_false",
                    help="reference arm: skip the reference's own CUDA backend leg")
    ap.add_argument("--no-e2e", dest="e2e", action="store_false",
                    help="skip the end-to-end pass (profiling runs)")
    ap.add_argument("--no-split", action="store_true",
                    help="run the stack as one stack on one stream (profiling)")
    ap.add_argument("--persistent", action="store_true",
                    help="run each iteration chunk of the stack as one cooperative kernel")
    ap.add_argument("--workload", default="stack",
                    choices=["stack", "spmv", "packed", "adjoint", "powerlaw", "seam"])
    ap.add_argument("--tolerance", type=float, default=1e-6,
                    help="--workload powerlaw: relative KKT tolerance")
    ap.add_argument("--time-limit", type=float, default=300.0,
                    help="--workload powerlaw: seconds per solve")
    ap.add_argument("--unrolled-steps", type=int, default=2000,
                    help="--workload adjoint: unrolled PDHG steps (profiling runs use fewer)")
    ap.add_argument("--packed-workers", type=int, default=0,
                    help="LPs in flight for --workload packed (0: autotune)")
    ap.add_argument("--spmv-iterations", type=int, default=2000)
    ap.add_argument("--seam-iterations", type=int, default=400,
                    help="--workload seam: iterations of the reference's solve_pdhg per arm")
    ap.add_argument("--locality", type=int, default=0,
                    help="--workload powerlaw: options.locality_order (relabelled rows/columns)")
    ap.add_argument("--precisions", default="fp32,fp64",
                    help="--workload powerlaw: comma list of fp32, fp64")
    ap.add_argument("--spmv-legs", default="",
                    help="comma list of spmv legs to run with --workload spmv "
                         "(fp32, fp64, fp32_relabelled, fp64_relabelled; default all)")
    ap.add_argument("--tile-threads", type=int, default=0,
                    help="--workload spmv: options.tile_threads (0 = tuned, 128, 256)")
    ap.add_argument("--no-side", dest="side", action="store_false",
                    help="skip every side leg of the stack line")
    ap.add_argument("--side-legs", default=",".join(SIDE_LEGS),
                    help="comma list of the stack line's side legs: " + ", ".join(SIDE_LEGS))
    args = ap.parse_args(argv)
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        out = run_reference(args, rank, world)
    elif args.workload == "packed":
        out = run_packed(args, rank, world, local_rank)
    elif args.workload == "adjoint":
        out = run_adjoint(args, rank, world, local_rank)
    elif args.workload == "powerlaw":
        out = run_powerlaw(args, rank, world, local_rank)
    elif args.workload == "seam":
        out = run_seam(args, rank, world, local_rank)
    elif args.workload == "spmv":
        out = None
        if rank == 0:
            import torch
            torch.cuda.set_device(local_rank)
            peak, kind = hbm_peak()
            out = spmv_leg(args.spmv_iterations, local_rank, peak,
                           args.spmv_legs.split(",") if args.spmv_legs else None,
                           args.tile_threads)
            out["peak_source"] = kind
    else:
        out = run_engine(args, rank, world, local_rank)
    if rank == 0 and out is not None:
        print(json.dumps(out), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
