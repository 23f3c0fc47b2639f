"""Benchmark: DC operating points per second of the 500x500 diode mesh
(250,002 unknowns, 1.25 M nonzeros, 25,000 diodes) on one B200, mixed
precision (FP32 Krylov bulk, FP64 device evaluation / residual / update)
against the plain FP64 path, each checked against the FP64 oracle.

One step = one complete DC Newton solve from x = 0: device evaluation,
stamp-map assembly, BiCGSTAB, limiting and convergence, all inside one
persistent kernel launch.  `value` uses a device-resident plan (inputs
already in HBM); `e2e` calls the public C ABI entry point ohm_newton_solve
with pinned host arrays every step (upload, solve, download).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
Multi-GPU: one process per GPU (torchrun); every rank solves its own replica
(the path has no exchange step), value = all ranks' solves / max time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solves/s & SpMV HBM GB/s: mixed-prec batched vs plain FP64 GPU at 1e-9 rel err"
def workload(sysm, rows, cols):
    """Name of the headline workload with its sizes (500x500: 250,002
    unknowns, 25,000 diodes)."""
    return (f"diode-mesh {rows}x{cols} DC operating point ({sysm.size:,} unknowns, "
            f"{len(sysm.diode_descriptors):,} diodes, seed 1)")
L2_FLUSH_BYTES = 512 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--rows", type=int, default=500)
    p.add_argument("--cols", type=int, default=500)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--batch", type=int, default=4096,
                   help="Monte Carlo batch size for the batched measurement (0 skips it)")
    p.add_argument("--batch-mixed", action="store_true",
                   help="also time the batch with the FP32 Krylov bulk")
    p.add_argument("--tran-stages", type=int, default=100_000,
                   help="inverter-chain stages of the transient measurement (0 skips it)")
    p.add_argument("--tran-steps", type=int, default=2000)
    p.add_argument("--adjoint-rows", type=int, default=1000,
                   help="RC-diode mesh size of the adjoint measurement (0 skips it)")
    p.add_argument("--ac-rows", type=int, default=100,
                   help="RC mesh size of the AC sweep measurement (0 skips it)")
    p.add_argument("--grid-rows", type=int, default=1000,
                   help="mesh size of the large-grid DC measurement (0 skips it)")
    p.add_argument("--compile-small", action="store_true",
                   help="compile section on 100x100 meshes and a 2,000-stage chain (for profiling)")
    p.add_argument("--ladder-nodes", type=int, default=10_000,
                   help="resistor-ladder nodes of the linear DC measurement (0 skips it)")
    p.add_argument("--sections", default="dc,ladder,batch,transient,adjoint,grid,compile,ac",
                   help="comma list of dc (the headline), ladder, batch, transient, adjoint, grid, compile, ac, "
                        "and gradcheck (not a default: ~130 forward transients of the 1M-row mesh); a run "
                        "without dc "
                        "prints only the chosen sections (for profiling small cases); 'spmv' alone "
                        "runs the backend SpMV measurement")
    p.add_argument("--profile", choices=["fp64", "mixed", "grid"], default=None,
                   help="one warm-up and one timed solve only (for an ncu capture); 'grid': the "
                        "--grid-rows RC-diode mesh at 1 V, one Newton iteration with BiCGSTAB capped at "
                        "40 iterations (a launch of a few ms on a working set larger than L2)")
    return p.parse_args()


def guarded(section, *args):
    """A secondary section that fails is reported in the line ({"error":
    ...}) instead of ending the run before the headline is printed."""
    try:
        return section(*args)
    except Exception as e:  # noqa: BLE001
        return {"error": f"{type(e).__name__}: {e}"}


def newton_params(mixed: bool, precond: int = 0):
    """Newton stops at max|dx| < 1e-9 V; each linear solve is inexact with an
    Eisenstat-Walker tolerance in [1e-4, 0.7] on the diagonally scaled
    residual, above an absolute floor of 1e-14 ||W b||.  The same settings for
    the FP64 and the mixed path; precond 0 = block Jacobi, 2 = ISAI(1)."""
    from ohmnivore_b200 import solver as S
    return S.NewtonParams(max_iterations=200, abs_tol=1e-9, bicgstab_max_iterations=20000,
                          bicgstab_tolerance=1e-14, precision=1 if mixed else 0, inner_rtol=1e-4,
                          forcing=1, eta_max=0.7, precond=precond)


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.FIELDS}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *exc):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        finally:
            os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def spmv_bytes(n, nnz, wa, wv):
    """Algorithmic SpMV bytes: values + column indices + row pointers + x read once + y write."""
    return nnz * (wa + 4) + 4 * (n + 1) + 2 * n * wv


def solve_bytes(info, n, nnz, nd, mixed):
    """Algorithmic bytes of one persistent-kernel launch (one Newton solve).

    Per Newton iteration: device evaluation + stamp map (descriptor 48 B,
    anode voltage 8 B, 6 stamp values written and read 16 B each, the touched
    slot's base + value 16 B, rhs base + value 16 B); the FP64 residual
    b - J x (SpMV at FP64 + b read + r64 write + Krylov vectors initialised:
    r, r_hat, p, v, d); the limiter (x, x_prev, scale, d: 4 n*8 + proposals).
    Per BiCGSTAB iteration (Jacobi): 2 SpMV + 21 length-n vector streams +
    2 diagonal reads, in the Krylov precision (4 B mixed, 8 B FP64).
    """
    w = 4 if mixed else 8
    newton_it = int(info["iterations"])
    kry = int(info["krylov_iterations"])
    b_eval = nd * (48 + 8 + 6 * 16 + 16 + 16)
    b_setup = spmv_bytes(n, nnz, 8, 8) + 2 * n * 8 + n * 8 + 5 * n * w + 2 * n * w
    b_limit = 4 * n * 8 + nd * (48 + 16)
    b_it = 2 * spmv_bytes(n, nnz, w, w) + 21 * n * w + 2 * n * w
    return newton_it * (b_eval + b_setup + b_limit) + kry * b_it, kry


def measured_peaks():
    try:
        return json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        return None


def run_reference(args, rank):
    """Reference arm: the oracle port of the reference CPU path (FP64 Newton
    with a sparse LU per iteration, newton.rs CpuSparseLu mode) on the host."""
    if rank != 0:
        return
    from ohmnivore_b200 import circuits, mna
    from oracle import newton_ref
    sysm = mna.compile_circuit(circuits.diode_mesh(args.rows, args.cols, seed=1))
    t_w = time.perf_counter()
    for _ in range(args.warmup):                       # warm-up: one Newton iteration each
        try:
            newton_ref.newton(sysm, max_iterations=1)
        except Exception:
            pass
    t_w = time.perf_counter() - t_w
    times = []
    iters = 0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, it = newton_ref.newton(sysm)
        times.append(time.perf_counter() - t0)
        iters = it
    total = sum(times)
    value = args.steps / total
    line = {"metric": METRIC, "value": value, "unit": "solves/s", "impl": "reference", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic", "config": {"workload": workload(sysm, args.rows, args.cols),
                                            "newton_iterations": iters},
            "cpu_baseline": {"value": value, "unit": "solves/s", "cores": 1, "host_cores": os.cpu_count(), "kind": "port",
                             "sample": f"{args.steps} full DC solves of the workload (FP64 Newton + "
                                       "SuperLU per iteration, single thread); warm-up = 1 Newton "
                                       "iteration each"},
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return
    if args.profile:
        run_profile_case(args)
        return

    import torch
    import torch.distributed as dist
    from ohmnivore_b200 import circuits, mna
    from ohmnivore_b200 import solver as S

    torch.cuda.set_device(local_rank)
    if world > 1:
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300),
                                device_id=torch.device("cuda", local_rank))

    sysm = mna.compile_circuit(circuits.diode_mesh(args.rows, args.cols, seed=1))
    n, nnz, nd = sysm.size, sysm.g.nnz, len(sysm.diode_descriptors)
    ctx = S.Context(local_rank)
    stream = torch.cuda.ExternalStream(ctx.lib.ohm_ctx_stream(ctx.handle), device=local_rank)
    plan = S.NewtonPlan(sysm, ctx)
    x = torch.zeros(n, dtype=torch.float64, device=f"cuda:{local_rank}")
    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=f"cuda:{local_rank}")

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()

    sections = set(args.sections.split(","))
    if "dc" not in sections:
        line = {"metric": METRIC, "sections_only": sorted(sections)}
        if "spmv" in sections:
            line["spmv"] = spmv_roofline(S, ctx, sysm, stream, flush)
        if "ladder" in sections and args.ladder_nodes > 0:
            line["ladder"] = guarded(ladder_section, args, S, ctx, stream, barrier, world, rank, local_rank)
        if "batch" in sections and args.batch > 0:
            line["batch"] = guarded(batch_section, args, S, ctx, stream, barrier, world, rank, local_rank)
        if "transient" in sections and args.tran_stages > 0:
            line["transient"] = guarded(transient_section, args, S, ctx, stream, barrier, world, rank, local_rank)
        if "adjoint" in sections and args.adjoint_rows > 0:
            line["adjoint"] = guarded(adjoint_section, args, S, ctx, stream, barrier, world, rank, local_rank)
        if "grid" in sections and args.grid_rows > 0:
            line["grid"] = guarded(grid_section, args, S, ctx, stream, barrier, world, rank, local_rank)
        if "compile" in sections:
            line["compile"] = guarded(compile_section, args, S, ctx, stream, barrier, world, rank, local_rank)
        if "ac" in sections and args.ac_rows > 0:
            line["ac"] = guarded(ac_section, args, S, ctx, stream, barrier, world, rank, local_rank)
        if "gradcheck" in sections and args.adjoint_rows > 0:
            line["gradcheck"] = guarded(gradcheck_section, args, S, ctx, stream, barrier, world, rank, local_rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
        plan.close()
        ctx.close()
        if world > 1:
            dist.destroy_process_group()
        return

    def timed_solves(mixed, steps, warmup, precond=0):
        params = newton_params(mixed, precond)
        infos = []
        for _ in range(warmup):
            with torch.cuda.stream(stream):
                x.zero_()
            plan.newton_device(x.data_ptr(), params)
        barrier()
        total_ms = 0.0
        for _ in range(steps):
            with torch.cuda.stream(stream):
                flush.zero_()                       # L2 flush outside the timed interval
                x.zero_()
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            infos.append(plan.newton_device(x.data_ptr(), params))
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            total_ms += e0.elapsed_time(e1)
        barrier()
        t = torch.tensor([total_ms], dtype=torch.float64, device=x.device)
        if world > 1:
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), infos, x.cpu().numpy()

    # ---- FP64 path (headline: faster on this latency-bound single circuit)
    #      and the mixed-precision path, both device-resident ----
    with ClockSampler(local_rank) as clk:
        fp64_ms, fp64_infos, x_fp64 = timed_solves(False, args.steps, args.warmup)
    clocks = clk.summary()
    mixed_ms, mixed_infos, x_mixed = timed_solves(True, args.steps, args.warmup)
    # FP32 Krylov + FP64 Newton with the ISAI(1) preconditioner (the
    # reference's choice for matrices with a zero diagonal, gpu.rs:139-168)
    isai_steps = min(args.steps, 3)
    isai_ms, isai_infos, x_isai = timed_solves(True, isai_steps, 1, precond=2)

    # ---- e2e: public C ABI, pinned host arrays, upload + solve + download ----
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory().numpy()  # noqa: E731
    h_vals = pin(sysm.g.val.astype(np.float64))
    h_col = pin(sysm.g.col.astype(np.uint32))
    h_rp = pin(sysm.g.row_ptr.astype(np.uint32))
    h_b = pin(sysm.b_dc.astype(np.float64))
    h_dd = torch.from_numpy(sysm.diode_descriptors.view(np.uint8)).pin_memory().numpy().view(mna.DIODE_DTYPE)
    h_x = pin(np.zeros(n))
    params = newton_params(False)

    def e2e_call():
        return S.newton_solve(ctx, h_vals, h_col, h_rp, h_b, h_dd, sysm.bjt_descriptors,
                              sysm.mosfet_descriptors, n, nnz, params)

    for _ in range(max(1, args.warmup)):
        e2e_call()
    barrier()
    e2e_ms = 0.0
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        h_x[:] = e2e_call()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    barrier()
    t = torch.tensor([e2e_ms], dtype=torch.float64, device=x.device)
    if world > 1:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    e2e_ms = float(t.item())
    h2d = h_vals.nbytes + h_col.nbytes + h_rp.nbytes + h_b.nbytes + h_dd.nbytes
    d2h = n * 8

    # ---- SpMV bandwidth (cold L2, FP64 and FP32 values) ----
    spmv = spmv_roofline(S, ctx, sysm, stream, flush)

    # ---- roofline of the persistent kernel (dominant: the only kernel of a solve) ----
    peaks = measured_peaks()
    hbm_peak = peaks["hbm_gbs"] if peaks else 6650.0
    peak_src = "measured" if peaks else "fallback"
    info0 = fp64_infos[-1]
    algo_bytes, kry = solve_bytes(info0, n, nnz, nd, mixed=False)
    per_launch_ms = fp64_ms / args.steps
    achieved = algo_bytes / (per_launch_ms * 1e-3) / 1e9

    value = world * args.steps / (fp64_ms * 1e-3)
    mixed_value = world * args.steps / (mixed_ms * 1e-3)
    line = {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": fp64_ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": workload(sysm, args.rows, args.cols),
                   "precision": "FP64 (BiCGSTAB, device eval, residual, update)",
                   "preconditioner": "block Jacobi (2x2 for the source branch row)",
                   "newton_abs_tol": 1e-9, "krylov_tol_floor": 1e-14,
                   "inner_tolerance": "Eisenstat-Walker in [1e-4, 0.7], scaled residual",
                   "l2": "flushed (512 MiB write) before every timed step",
                   "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
        "mixed_precision": {"value": mixed_value, "unit": "solves/s", "ms_per_step": mixed_ms / args.steps,
                            "newton_iterations": mixed_infos[-1]["iterations"],
                            "krylov_iterations": mixed_infos[-1]["krylov_iterations"],
                            "fp64_fallbacks": mixed_infos[-1]["fp64_fallbacks"],
                            "note": "FP32 BiCGSTAB bulk; on this single L2-resident circuit the loop is "
                                    "latency-bound, so FP32 iterations cost the same as FP64 ones"},
        "mixed_isai1": {"value": world * isai_steps / (isai_ms * 1e-3), "unit": "solves/s",
                        "ms_per_step": isai_ms / isai_steps, "steps": isai_steps,
                        "newton_iterations": isai_infos[-1]["iterations"],
                        "krylov_iterations": isai_infos[-1]["krylov_iterations"],
                        "fp64_fallbacks": isai_infos[-1]["fp64_fallbacks"],
                        "note": "FP32 BiCGSTAB preconditioned by ISAI(1) of the device ILU(0) factors, rebuilt "
                                "every Newton iteration; FP64 device evaluation, residual and update"},
        "mixed_vs_fp64": mixed_value / value,
        "newton_iterations": info0["iterations"], "krylov_iterations": kry,
        "krylov_restarts": info0["krylov_restarts"],
        "e2e": {"value": world * args.steps / (e2e_ms * 1e-3), "unit": "solves/s",
                "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
                "api": "ohm_newton_solve (host arrays in pinned memory)"},
        "gpu_launches": args.steps,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                     "frac": achieved / hbm_peak,
                     "traffic": 7.64e6 * (n / 40002.0),
                     "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum of the same kernel on the "
                                       "200x200 mesh (7.64 MB per solve, 40,002 unknowns), scaled by unknowns: the "
                                       "working set stays in L2, so DRAM sees the inputs about once per solve",
                     "peak_source": peak_src,
                     "kernel": "persistent_solver<1> (FP64 Krylov)",
                     "algorithmic_bytes_per_launch": algo_bytes,
                     "note": "working set (~40 MB) is L2-resident inside a solve"},
        "spmv": spmv,
        "clocks": clocks,
    }

    # ---- accuracy vs the FP64 oracle and the CPU baseline (rank 0, N = 1) ----
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        from oracle import newton_ref
        t0 = time.perf_counter()
        ref, it_ref = newton_ref.newton(sysm)
        cpu_s = time.perf_counter() - t0
        nn = slice(0, sysm.n_nodes)
        br = slice(sysm.n_nodes, n)
        err = lambda a, sl: float(np.max(np.abs(a[sl] - ref[sl])) / np.max(np.abs(ref[sl])))  # noqa: E731
        line["rel_err_vs_oracle"] = {
            "mixed": {"voltages": err(x_mixed, nn), "currents": err(x_mixed, br)},
            "mixed_isai1": {"voltages": err(x_isai, nn), "currents": err(x_isai, br)},
            "fp64": {"voltages": err(x_fp64, nn), "currents": err(x_fp64, br)},
            "e2e_fp64": {"voltages": err(h_x, nn), "currents": err(h_x, br)}}
        line["cpu_baseline"] = {"value": 1.0 / cpu_s, "unit": "solves/s", "cores": 1, "host_cores": os.cpu_count(), "kind": "port",
                                "sample": f"1 full DC solve of the workload ({it_ref} FP64 Newton "
                                          "iterations, SuperLU per iteration), single thread"}
    if "ladder" in sections and args.ladder_nodes > 0:
        line["ladder"] = guarded(ladder_section, args, S, ctx, stream, barrier, world, rank, local_rank)
    if "batch" in sections and args.batch > 0:
        line["batch"] = guarded(batch_section, args, S, ctx, stream, barrier, world, rank, local_rank)
    if "transient" in sections and args.tran_stages > 0:
        line["transient"] = guarded(transient_section, args, S, ctx, stream, barrier, world, rank, local_rank)
    if "adjoint" in sections and args.adjoint_rows > 0:
        line["adjoint"] = guarded(adjoint_section, args, S, ctx, stream, barrier, world, rank, local_rank)
    if "grid" in sections and args.grid_rows > 0:
        line["grid"] = guarded(grid_section, args, S, ctx, stream, barrier, world, rank, local_rank)
    if "compile" in sections:
        line["compile"] = guarded(compile_section, args, S, ctx, stream, barrier, world, rank, local_rank)
    if "ac" in sections and args.ac_rows > 0:
        line["ac"] = guarded(ac_section, args, S, ctx, stream, barrier, world, rank, local_rank)
    if rank == 0:
        print(json.dumps(line), flush=True)
    plan.close()
    ctx.close()
    if world > 1:
        dist.destroy_process_group()


def batch_params(mixed: bool):
    """Monte Carlo batch: Newton to max|dx| < 1e-10 V, constant inner
    tolerance 1e-4 on the scaled residual, DC continuation on failure."""
    from ohmnivore_b200 import solver as S
    return S.NewtonParams(max_iterations=100, abs_tol=1e-10, bicgstab_max_iterations=20000,
                          bicgstab_tolerance=1e-14, precision=1 if mixed else 0, inner_rtol=1e-4,
                          continuation=True)


def batch_section(args, S, ctx, stream, barrier, world, rank, local_rank):
    """Batched Monte Carlo DC (BJT differential-pair meshes, 50-20,000
    nodes, seed 3, VAF 100 V): one launch over the packed batch, against the
    plain FP64 single-circuit path on a size-stratified sample, and the
    error of a sample against the FP64 oracle."""
    import torch
    from ohmnivore_b200 import circuits, mna
    t0 = time.perf_counter()
    ckts = circuits.monte_carlo_batch(args.batch, seed=3, vaf=100.0)
    if world > 1:
        # instances shard over the ranks (LPT on component count); no exchange
        # during the solve, one status gather at the end
        from ohmnivore_b200.shard import lpt_partition
        mine = lpt_partition([c.n_components for c in ckts], world)[rank]
    else:
        mine = np.arange(len(ckts))
    t_gen = time.perf_counter()
    systems = [S.compile_circuit_device(ckts[int(i)], ctx) for i in mine]
    setup_s = time.perf_counter() - t0
    compile_s = time.perf_counter() - t_gen
    batch = S.NewtonBatch(systems, ctx)
    rows = batch.rows
    nnz = int(batch.nnz_off[-1])
    x = torch.zeros(rows, dtype=torch.float64, device=f"cuda:{local_rank}")
    t0 = time.perf_counter()
    choice = batch.autotune(batch_params(False), sample_size=256)
    tune_s = time.perf_counter() - t0

    def timed(mixed):
        with torch.cuda.stream(stream):
            x.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        info = batch.newton_device(x.data_ptr(), batch_params(mixed), check=False)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        barrier()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=x.device)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), info

    with ClockSampler(local_rank) as clk:
        ms, info = timed(False)
    per = batch.instance_info()
    from ohmnivore_b200.shard import gather_status
    status_all = gather_status([q["status"] for q in per], mine, args.batch)
    cont = torch.tensor([sum(1 for q in per if q["continuation_steps"] > 0), rows, nnz], dtype=torch.float64,
                        device=x.device)
    if world > 1:
        import torch.distributed as dist
        dist.all_reduce(cont)
    out = {"workload": f"Monte Carlo batch: {args.batch} BJT differential-pair meshes, 50-20,000 nodes "
                       f"(seed 3, VAF 100 V), {int(cont[1].item())} unknowns, {int(cont[2].item())} nonzeros",
           "value": args.batch / (ms * 1e-3), "unit": "solves/s", "ms": ms,
           "scaling": "strong: the instances are sharded over the GPUs (LPT), one batch launch per GPU"
                      if world > 1 else "1 GPU",
           "precision": "FP64", "kernel_launches": info["kernel_launches"],
           "split": "circuits whose one-block solve would outlast the rest run alone on the whole GPU first "
                    "(ohm_batch_set_split); kernel_launches counts those solves and the batch launch",
           "failed_instances": int(np.count_nonzero(status_all != 0)),
           "continuation_instances": int(cont[0].item()),
           "krylov_iterations": info["krylov_iterations"], "autotune": choice,
           "autotune_s": tune_s, "host_setup_s": setup_s, "device_compile_s": compile_s, "clocks": clk.summary()}
    xs = batch.split(x.cpu().numpy())
    if args.batch_mixed:
        ms_m, info_m = timed(True)
        per_m = batch.instance_info()
        out["mixed_precision"] = {"value": args.batch / (ms_m * 1e-3), "ms": ms_m,
                                  "failed_instances": sum(1 for q in per_m if q["status"] != 0),
                                  "fp64_fallbacks": info_m["fp64_fallbacks"]}
    batch.close()

    # plain FP64 one-circuit-at-a-time GPU path on a size-stratified sample
    order = np.argsort([-s.size for s in systems], kind="stable")
    sample = sorted({int(order[(k * len(order)) // 32]) for k in range(32)})
    single_ms = 0.0
    for i in sample:
        s = systems[i]
        plan = S.NewtonPlan(s, ctx)
        xi = torch.zeros(s.size, dtype=torch.float64, device=x.device)
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        try:
            plan.newton_device(xi.data_ptr(), batch_params(False))
        except S.OhmnivoreError:
            pass
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        single_ms += e0.elapsed_time(e1)
        plan.close()
    single_rate = len(sample) / (single_ms * 1e-3)
    out["single_fp64"] = {"value": world * single_rate, "unit": "solves/s",
                          "sample": "32 instances of this GPU's share, spread by size, one persistent-kernel "
                                    "solve each (x GPUs)"}
    out["batched_vs_single"] = out["value"] / (world * single_rate)
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import newton_ref
        ev, ei = 0.0, 0.0
        check = sorted({int(order[(k * len(order)) // 64]) for k in range(64)})   # size-stratified
        for i in check:
            s = systems[i]
            ref, _ = newton_ref.dc_operating_point(s)
            nn = slice(0, s.n_nodes)
            br = slice(s.n_nodes, s.size)
            ev = max(ev, float(np.max(np.abs(xs[i][nn] - ref[nn])) / np.max(np.abs(ref[nn]))))
            if s.size > s.n_nodes:
                ei = max(ei, float(np.max(np.abs(xs[i][br] - ref[br])) / max(np.max(np.abs(ref[br])), 1e-300)))
        out["rel_err_vs_oracle"] = {"voltages": ev, "currents": ei, "instances": len(check),
                                    "sample": "size-stratified: every (len/64)-th instance by size"}
    return out


def transient_section(args, S, ctx, stream, barrier, world, rank, local_rank):
    """CMOS inverter chain (100,000 stages, 200,000 level-1 MOSFETs, 10 fF
    loads, PULSE input 0-1.8 V, 50 ps edges, 2 ns period): 2000 backward-Euler
    steps of 5 ps, a Newton solve per step started from the linear
    extrapolation of the last two steps, all steps on the device, replayed
    as one CUDA graph of 20 persistent launches.  Precision: FP32 Krylov bulk
    with FP64 residual / update (and the plain FP64 path beside it).  The
    first 50 steps are checked against the oracle (LU Newton per step)."""
    import torch
    from ohmnivore_b200 import circuits, mna
    stages, nsteps, h = args.tran_stages, args.tran_steps, 5e-12
    sysm = mna.compile_circuit(circuits.inverter_chain(stages=stages, seed=2))
    n = sysm.size
    # DC operating point from logic levels (input low), then the transient
    x0 = np.zeros(n)
    x0[sysm.node_index(1)] = 1.8
    out = np.array([sysm.node_index(2 + k) for k in range(1, stages + 1)])
    x0[out] = np.where(np.arange(1, stages + 1) % 2 == 1, 1.8, 0.0)
    plan = S.NewtonPlan(sysm, ctx)
    x = torch.from_numpy(x0).to(f"cuda:{local_rank}")
    dc_params = S.NewtonParams(max_iterations=100, abs_tol=1e-10, bicgstab_max_iterations=20000,
                               bicgstab_tolerance=1e-14, inner_rtol=1e-4, continuation=True)
    plan.newton_device(x.data_ptr(), dc_params)
    xdc = x.clone()
    probes = [sysm.node_index(k) for k in (2, 3, 4, 5, 102, 1002, 2 + stages)]
    tr = S.Transient(plan, probes)
    tr.set_predictor(2)

    def step_params(mixed):
        return S.NewtonParams(max_iterations=50, abs_tol=1e-9, bicgstab_max_iterations=20000,
                              bicgstab_tolerance=1e-14, inner_rtol=1e-4, precision=1 if mixed else 0)

    def timed(mixed, clk=None):
        with torch.cuda.stream(stream):
            x.copy_(xdc)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        wave = tr.run(x.data_ptr(), 0.0, h, nsteps, step_params(mixed), steps_per_launch=100, graph=True)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        barrier()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=x.device)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), dict(tr.last_info), wave

    timed(True)                                     # warm-up (graph instantiation, caches)
    with ClockSampler(local_rank) as clk:
        ms_m, info_m, wave_m = timed(True)
    ms_d, info_d, wave_d = timed(False)
    res = {"workload": f"CMOS inverter chain, {stages} stages ({2 * stages} MOSFETs), {nsteps} BE steps of 5 ps",
           "value": world * nsteps / (ms_m * 1e-3), "unit": "timesteps/s", "ms_full_run": ms_m,
           "precision": "FP32 Krylov bulk, FP64 device evaluation / residual / update",
           "newton_start": "quadratic extrapolation 3 x_{n-1} - 3 x_{n-2} + x_{n-3} (ohm_transient_set_predictor(2))",
           "newton_iterations": info_m["newton_iterations"], "krylov_iterations": info_m["krylov_iterations"],
           "fp64_fallbacks": info_m["fp64_fallbacks"], "kernel_launches": info_m["launches"],
           "cuda_graph": bool(info_m["graph"]), "clocks": clk.summary(),
           "fp64": {"value": world * nsteps / (ms_d * 1e-3), "ms_full_run": ms_d,
                    "newton_iterations": info_d["newton_iterations"]},
           "mixed_vs_fp64_max_abs_diff_V": float(np.max(np.abs(wave_m - wave_d)))}
    # the reference's own stepping policy on the same chain: adaptive BE / TRAP
    # with LTE control (tstep 5 ps, one 2 ns input period), one launch
    tstop_ad = 2e-9
    with torch.cuda.stream(stream):          # untimed warm-up run (first-call set-up)
        x.copy_(xdc)
    tr.run_adaptive(x.data_ptr(), h, tstop_ad, 0.0, step_params(True))
    with torch.cuda.stream(stream):
        x.copy_(xdc)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
    times_ad, _ = tr.run_adaptive(x.data_ptr(), h, tstop_ad, 0.0, step_params(True))
    with torch.cuda.stream(stream):
        e1.record(stream)
    e1.synchronize()
    ia = dict(tr.last_info)
    ms_a = e0.elapsed_time(e1)
    res["adaptive"] = {"workload": f"same chain, adaptive BE/TRAP, tstep 5 ps, tstop {tstop_ad * 1e9:g} ns",
                       "ms_full_run": ms_a, "accepted": ia["accepted"], "rejected": ia["rejected"],
                       "linear_solves": ia["linear_solves"], "newton_iterations": ia["newton_iterations"],
                       "krylov_iterations": ia["krylov_iterations"], "points": ia["points"],
                       "accepted_steps_per_s": ia["accepted"] / (ms_a * 1e-3),
                       "min_step_ps": float(np.min(np.diff(times_ad))) * 1e12 if len(times_ad) > 1 else None}
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import newton_ref, transient_ref
        xd = xdc.cpu().numpy()
        ref_dc, _ = newton_ref.newton(sysm, x0=xd)
        k = 50
        t0 = time.perf_counter()
        _, ref_wave, _ = transient_ref.be_transient(sysm, ref_dc, 0.0, h, k, probes)
        cpu_s = time.perf_counter() - t0
        res["rel_err_vs_oracle"] = {
            "first_steps": k,
            "mixed": float(np.max(np.abs(wave_m[:k] - ref_wave)) / np.max(np.abs(ref_wave))),
            "fp64": float(np.max(np.abs(wave_d[:k] - ref_wave)) / np.max(np.abs(ref_wave))),
            "dc_start": float(np.max(np.abs(xd[:sysm.n_nodes] - ref_dc[:sysm.n_nodes])) / 1.8)}
        res["cpu_baseline"] = {"value": k / cpu_s, "unit": "timesteps/s", "cores": 1, "host_cores": os.cpu_count(), "kind": "port",
                               "sample": f"{k} BE steps of the same chain, LU Newton per step, single thread"}
    tr.close()
    plan.close()
    return res


def compile_section(args, S, ctx, stream, barrier, world, rank, local_rank):
    """Device-side MNA compile (ohm_compile) against the host compiler on the
    workloads' circuits: wall time of each (the device figure includes the
    upload of the component arrays, the download of the system and its
    assembly into the same Python object), and a bit-for-bit check."""
    from ohmnivore_b200 import circuits, mna
    work = [("diode mesh 500x500 (headline)", lambda: circuits.diode_mesh(500, 500, seed=1)),
            ("RC-diode mesh 1000x1000", lambda: circuits.rc_diode_mesh(1000, 1000, seed=4)),
            ("inverter chain, 100,000 stages", lambda: circuits.inverter_chain(stages=100_000, seed=2))]
    if args.compile_small:
        work = [("diode mesh 100x100", lambda: circuits.diode_mesh(100, 100, seed=1)),
                ("RC-diode mesh 100x100", lambda: circuits.rc_diode_mesh(100, 100, seed=4)),
                ("inverter chain, 2,000 stages", lambda: circuits.inverter_chain(stages=2000, seed=2))]
    S.compile_circuit_device(circuits.diode_mesh(8, 8, seed=1), ctx)        # module load, memory cache
    res = {}
    for name, mk in work:
        ckt = mk()
        t0 = time.perf_counter()
        host = mna.compile_circuit(ckt)
        t1 = time.perf_counter()
        dev = S.compile_circuit_device(ckt, ctx)
        t2 = time.perf_counter()
        same = (np.array_equal(dev.g.col, host.g.col) and np.array_equal(dev.g.row_ptr, host.g.row_ptr)
                and np.array_equal(dev.g.val.view(np.uint64), host.g.val.view(np.uint64))
                and np.array_equal(dev.b_dc.view(np.uint64), host.b_dc.view(np.uint64))
                and np.array_equal(dev.diode_descriptors.view(np.uint8), host.diode_descriptors.view(np.uint8))
                and np.array_equal(dev.mosfet_descriptors.view(np.uint8), host.mosfet_descriptors.view(np.uint8)))
        res[name] = {"rows": host.size, "nonzeros": host.g.nnz, "components": ckt.n_components,
                     "host_s": t1 - t0, "device_s": t2 - t1, "speedup": (t1 - t0) / (t2 - t1),
                     "bit_identical": bool(same)}
    # many small circuits: 32 Monte Carlo instances, one call each
    ckts = circuits.monte_carlo_batch(32, seed=3, vaf=100.0)
    t0 = time.perf_counter()
    hs = [mna.compile_circuit(c) for c in ckts]
    t1 = time.perf_counter()
    ds = [S.compile_circuit_device(c, ctx) for c in ckts]
    t2 = time.perf_counter()
    same = all(np.array_equal(d.g.val.view(np.uint64), h.g.val.view(np.uint64)) for d, h in zip(ds, hs))
    res["32 Monte Carlo circuits, one call each"] = {
        "rows": int(sum(h.size for h in hs)), "host_s": t1 - t0, "device_s": t2 - t1,
        "speedup": (t1 - t0) / (t2 - t1), "bit_identical": bool(same)}
    return res


def ladder_section(args, S, ctx, stream, barrier, world, rank, local_rank):
    """Linear DC operating point of the 10,000-node resistor ladder (series R
    log-uniform 100-100k ohm, shunt R 1k-1M ohm to ground, 10 V at node 1,
    seed 0): FP64 block-Jacobi BiCGSTAB at the configured tolerance 1e-12
    (||r|| < 1e-12 ||b||) and at 1e-13, device-resident (ohm_solve_real_device)
    and end to end through ohm_solve_real (host arrays), each checked against
    the oracle's dense Gaussian elimination (CpuSolver, cpu.rs:28-96) on the
    full system.  The CPU baseline times that dense GE as the reference runs
    it (every row update, no zero skipping) on a bounded 2,500-node ladder and
    scales the time by (n / 2,500)^3, the operation count of the elimination."""
    import torch
    from ohmnivore_b200 import circuits, mna
    n_nodes = args.ladder_nodes
    sysm = mna.compile_circuit(circuits.resistor_ladder(n_nodes, seed=0))
    n, nnz = sysm.size, sysm.g.nnz
    be = S.SolverBackend(ctx)
    A = be.upload_matrix(sysm.g)
    bb, bx = be.new_buffer(n), be.new_buffer(n)
    bb.upload(sysm.b_dc)
    reps = max(3, args.steps)

    def timed(fn):
        for _ in range(2):
            fn()                                     # warm-up
        barrier()
        ms = []
        for _ in range(reps):
            with torch.cuda.stream(stream):
                e0 = torch.cuda.Event(enable_timing=True)
                e1 = torch.cuda.Event(enable_timing=True)
                e0.record(stream)
            out = fn()
            with torch.cuda.stream(stream):
                e1.record(stream)
            e1.synchronize()
            ms.append(e0.elapsed_time(e1))
        barrier()
        t = torch.tensor([sum(ms) / len(ms)], dtype=torch.float64, device=f"cuda:{local_rank}")
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), out

    peaks = measured_peaks()
    hbm_peak = peaks["hbm_gbs"] if peaks else 6650.0
    res = {"workload": f"resistor ladder {n_nodes:,} nodes, linear DC ({n:,} rows, {nnz:,} nonzeros, seed 0)",
           "precision": "FP64", "preconditioner": "block Jacobi (2x2 for the source branch row)"}
    xs = {}
    for tol in (1e-12, 1e-13):
        params = S.BiCgStabParams(tolerance=tol, max_iterations=50000)
        ms_dev, info = timed(lambda: be.solve_real_device(A, bb, bx, params))
        x_dev = bx.download()
        solver = S.GpuSolver(ctx, params)
        ms_e2e, x_e2e = timed(lambda: solver.solve_real(sysm.g, sysm.b_dc))
        kry = int(info["krylov_iterations"])
        b_it = 2 * spmv_bytes(n, nnz, 8, 8) + 21 * n * 8 + 2 * n * 8
        achieved = kry * b_it / (ms_dev * 1e-3) / 1e9
        xs[tol] = (x_dev, x_e2e)
        res[f"tol_{tol:g}"] = {
            "value": world * 1e3 / ms_dev, "unit": "solves/s", "ms": ms_dev,
            "krylov_iterations": kry, "us_per_iteration": 1e3 * ms_dev / max(kry, 1),
            "e2e": {"value": world * 1e3 / ms_e2e, "unit": "solves/s", "ms": ms_e2e,
                    "api": "ohm_solve_real (host CSR, b, x)",
                    "h2d_bytes_per_step": int(4 * (n + 1) + 12 * nnz + 8 * n), "d2h_bytes_per_step": int(8 * n)},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm_peak, "unit": "GB/s",
                         "frac": achieved / hbm_peak,
                         "note": "working set ~1.4 MB, L2-resident: the loop is bound by grid synchronisation"}}
    A.close(); bb.close(); bx.close()
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import linear_ref
        ref = linear_ref.dense_solve_real(n, n, sysm.g.row_ptr, sysm.g.col, sysm.g.val, sysm.b_dc)
        nn, br = slice(0, sysm.n_nodes), slice(sysm.n_nodes, n)
        err = lambda a, sl: float(np.max(np.abs(a[sl] - ref[sl])) / np.max(np.abs(ref[sl])))  # noqa: E731
        for tol, (xd, xe) in xs.items():
            res[f"tol_{tol:g}"]["rel_err_vs_dense_ge"] = {"voltages": err(xd, nn), "currents": err(xd, br),
                                                          "e2e_voltages": err(xe, nn)}
        m = 2500
        small = mna.compile_circuit(circuits.resistor_ladder(m, seed=0))
        t0 = time.perf_counter()
        linear_ref.dense_solve_real(small.size, small.size, small.g.row_ptr, small.g.col, small.g.val,
                                    small.b_dc, skip_zero_factors=False)
        cpu_small = time.perf_counter() - t0
        cpu_full = cpu_small * (n / small.size) ** 3
        res["cpu_baseline"] = {"value": 1.0 / cpu_full, "unit": "solves/s", "cores": 1,
                               "host_cores": os.cpu_count(), "kind": "port",
                               "sample": f"dense GE (cpu.rs:28-96, every row update) on the {m:,}-node ladder: "
                                         f"{cpu_small:.2f} s, scaled by ({n}/{small.size})^3 to {cpu_full:.0f} s"}
    return res


def ac_section(args, S, ctx, stream, barrier, world, rank, local_rank):
    """AC sweep (ac::run) of a 100x100 RC mesh (R log-uniform 10-10k ohm, C
    log-uniform 1 fF-1 pF to ground, seed 4) driven by a 1 V AC source
    through 50 ohm: 10 points per decade from 1 kHz to 1 THz (90 points),
    all points in one launch through ohm_ac_sweep (host arrays in and out),
    complex FP64 BiCGSTAB to 1e-15 (relative residual; the low-frequency
    points are ill-conditioned); the oracle's complex LU per point on a
    sample of the points."""
    from ohmnivore_b200 import circuits, mna
    rows = args.ac_rows
    ckt = circuits.rc_diode_mesh(rows, rows, seed=4, diode_frac=0.0)
    src = int(np.flatnonzero(ckt.kind == circuits.V)[0])
    ckt.ac[src] = (1.0, 0.0)
    sysm = mna.compile_circuit(ckt)
    freqs = S.ac_frequencies("dec", 10, 1e3, 1e12)
    params = S.BiCgStabParams(max_iterations=50000, tolerance=1e-15)
    S.ac_sweep(sysm, freqs[:4], params, ctx)                 # warm-up
    barrier()
    t0 = time.perf_counter()
    x, infos = S.ac_sweep(sysm, freqs, params, ctx)
    wall = time.perf_counter() - t0
    its = [p["iterations"] for p in infos]
    res = {"workload": f"AC sweep, {rows}x{rows} RC mesh ({sysm.size} rows, {sysm.g.nnz} nonzeros), "
                       f"{len(freqs)} points 1 kHz-1 THz",
           "value": world * len(freqs) / wall, "unit": "frequency points/s", "ms_sweep": wall * 1e3,
           "api": "ohm_ac_sweep (host arrays; upload, one launch, download)",
           "iterations_mean": float(np.mean(its)), "iterations_max": int(np.max(its)),
           "failed_points": int(sum(1 for p in infos if p["krylov_code"] != 1))}   # 1: converged
    if rank == 0 and not args.no_cpu_baseline:
        from oracle import ac_ref
        sample = list(range(0, len(freqs), 18))
        t0 = time.perf_counter()
        ref = ac_ref.ac_sweep(sysm, freqs[sample])
        cpu = time.perf_counter() - t0
        err = max(float(np.max(np.abs(x[k] - ref[j])) / np.max(np.abs(ref[j]))) for j, k in enumerate(sample))
        res["rel_err_vs_oracle"] = {"max": err, "points": len(sample)}
        res["cpu_baseline"] = {"value": len(sample) / cpu, "unit": "frequency points/s", "cores": 1, "host_cores": os.cpu_count(), "kind": "port",
                               "sample": f"{len(sample)} of the points, complex sparse LU each, single thread"}
    return res


def grid_section(args, S, ctx, stream, barrier, world, rank, local_rank):
    """DC operating point of the 1000x1000 RC mesh with diodes at 5 % of the
    nodes (seed 4; the adjoint workload's circuit, capacitors open at DC,
    the source at its step's final value, 1 V through 50 ohm):
    one FP64 and one mixed-precision solve after a warm-up, with the
    headline's Newton settings.  One large circuit fills the GPU, so the
    batched kernel (one block per circuit) does not apply; the mixed path
    is compared with the FP64 one."""
    import torch
    from ohmnivore_b200 import circuits, mna
    rows = args.grid_rows
    ckt = circuits.rc_diode_mesh(rows, rows, seed=4)
    src = int(np.flatnonzero(ckt.kind == circuits.V)[0])
    ckt.value[src] = 1.0                           # DC at the step's final value
    ckt.tran.pop(src, None)
    sysm = mna.compile_circuit(ckt)
    plan = S.NewtonPlan(sysm, ctx)
    x = torch.zeros(sysm.size, dtype=torch.float64, device=f"cuda:{local_rank}")

    def solve(mixed):
        with torch.cuda.stream(stream):
            x.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        info = plan.newton_device(x.data_ptr(), newton_params(mixed))
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        barrier()
        t = torch.tensor([e0.elapsed_time(e1)], dtype=torch.float64, device=x.device)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item()), info, x.cpu().numpy()

    solve(False)                                   # warm-up
    ms_d, info_d, x_d = solve(False)
    ms_m, info_m, x_m = solve(True)
    nn = sysm.n_nodes
    res = {"workload": f"DC operating point, {rows}x{rows} RC-diode mesh, 1 V through 50 ohm ({sysm.size} rows, "
                       f"{sysm.g.nnz} nonzeros, {len(sysm.diode_descriptors)} diodes)",
           "fp64": {"value": world * 1e3 / ms_d, "unit": "solves/s", "ms": ms_d,
                    "newton_iterations": info_d["iterations"], "krylov_iterations": info_d["krylov_iterations"]},
           "mixed": {"value": world * 1e3 / ms_m, "unit": "solves/s", "ms": ms_m,
                     "newton_iterations": info_m["iterations"], "krylov_iterations": info_m["krylov_iterations"],
                     "fp64_fallbacks": info_m["fp64_fallbacks"]},
           "mixed_vs_fp64": ms_d / ms_m,
           "mixed_vs_fp64_rel_err_voltages": float(np.max(np.abs(x_m[:nn] - x_d[:nn])) / np.max(np.abs(x_d[:nn])))}
    plan.close()
    return res


def adjoint_section(args, S, ctx, stream, barrier, world, rank, local_rank):
    """Adjoint sensitivities on the 1000x1000 RC mesh with diodes at 5% of the
    nodes (seed 4), driven by a 1 V step through 50 ohm: the gradient of one
    node voltage at t = 1 ns (500 BE steps of 2 ps) w.r.t. every R, C and Is,
    by the transient adjoint (every forward state kept in HBM, 500 x 1 M
    doubles = 4 GB, so the reverse sweep recomputes nothing; DC start
    included).  Outputs: the corner opposite the drive (the configured
    one) and node (10, 10) near the drive, where the response is nonzero;
    GPU central differences (relative step 1e-6) on the three resistors with
    the largest gradients of the latter."""
    import copy
    import torch
    from ohmnivore_b200 import circuits, mna
    rows, nsteps, h = args.adjoint_rows, 500, 2e-12
    ckt = circuits.rc_diode_mesh(rows, rows, seed=4)
    sysm = mna.compile_circuit(ckt)
    comps = S.ComponentTable(ckt, sysm)
    pn = S.NewtonParams(max_iterations=100, abs_tol=1e-10, bicgstab_max_iterations=20000,
                        bicgstab_tolerance=1e-14, inner_rtol=1e-6)
    plan = S.NewtonPlan(sysm, ctx)
    x = torch.zeros(sysm.size, dtype=torch.float64, device=f"cuda:{local_rank}")
    plan.newton_device(x.data_ptr(), pn)
    far = sysm.node_index(2 + rows * rows - 1)
    near = sysm.node_index(2 + 10 * rows + 10)
    tr = S.Transient(plan, [far, near])

    def ev_time(fn):
        with torch.cuda.stream(stream):
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        r = fn()
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        barrier()
        return e0.elapsed_time(e1), r

    xs = x.clone()
    fwd_ms, wave = ev_time(lambda: tr.run(xs.data_ptr(), 0.0, h, nsteps, pn, steps_per_launch=100))
    res = {"workload": f"RC mesh {rows}x{rows} with diodes at 5% of nodes, {sysm.size} unknowns, "
                       f"{len(comps.r_ohms)} R + {len(comps.c_farads)} C + {len(sysm.diode_descriptors)} Is "
                       f"parameters, {nsteps} BE steps of 2 ps",
           "forward_ms": fwd_ms, "unit": "gradients/s"}
    out = {}
    for name, row in (("opposite_corner", far), ("node_10_10", near)):
        w = np.zeros(sysm.size)
        w[row] = 1.0
        with ClockSampler(local_rank) as clk:
            ms, (g, info) = ev_time(lambda: tr.adjoint(x.data_ptr(), 0.0, h, nsteps, w, comps, pn, 0))
        out[name] = {"output_V": info["output"], "adjoint_ms": ms, "linear_solves": info["linear_solves"],
                     "krylov_iterations": info["krylov_iterations"],
                     "max_abs_grad": {k: float(np.max(np.abs(v))) for k, v in g.items() if len(v)},
                     "nonzero_grads": {k: int(np.count_nonzero(v)) for k, v in g.items()},
                     "clocks": clk.summary()}
        if name == "node_10_10":
            fd_err = []
            for j in np.argsort(-np.abs(g["R"]))[:3]:
                idx = comps.r_index[j]
                v = ckt.value[idx]
                outs = []
                for sign in (1, -1):
                    c2 = copy.deepcopy(ckt)
                    c2.value[idx] = v * (1 + sign * 1e-6)
                    s2 = mna.compile_circuit(c2)
                    p2 = S.NewtonPlan(s2, ctx)
                    t2 = S.Transient(p2, [near])
                    x2 = torch.zeros(s2.size, dtype=torch.float64, device=x.device)
                    p2.newton_device(x2.data_ptr(), pn)
                    outs.append(t2.run(x2.data_ptr(), 0.0, h, nsteps, pn, steps_per_launch=100)[-1, 0])
                    t2.close()
                    p2.close()
                fd = (outs[0] - outs[1]) / (2e-6 * v)
                fd_err.append(abs(g["R"][j] - fd) / abs(fd))
            out[name]["rel_err_vs_central_differences"] = {"resistors": 3, "max": float(max(fd_err))}
    res.update(out)
    res["value"] = world * 1000.0 / out["node_10_10"]["adjoint_ms"]
    if rank == 0 and not args.no_cpu_baseline:
        import scipy.sparse as sp
        import scipy.sparse.linalg as spl
        from oracle import adjoint_ref, transient_ref
        xh = x.cpu().numpy()
        t0 = time.perf_counter()
        A = transient_ref.companion(sysm, h)
        J = adjoint_ref._jacobian(sysm, A, xh)
        w = np.zeros(sysm.size)
        w[near] = 1.0
        lam = spl.splu(J.T.tocsc()).solve(w)
        adjoint_ref.backstamp(sysm, comps, xh, xh, lam, h)
        one = time.perf_counter() - t0
        res["cpu_baseline"] = {"value": 1.0 / (one * (nsteps + 1)), "unit": "gradients/s", "cores": 1, "host_cores": os.cpu_count(),
                               "kind": "port", "sample": "1 reverse step (assemble J, LU of J^T, back-stamp) "
                                                         f"timed and scaled to {nsteps + 1} solves, no forward pass"}
    tr.close()
    plan.close()
    return res


def gradcheck_section(args, S, ctx, stream, barrier, world, rank, local_rank):
    """Full-size check of the config-5 gradient (not in the default sections:
    ~130 forward transients of the 1M-row mesh): the transient adjoint of
    V(node (10, 10)) at t = 1 ns (500 BE steps of 2 ps) against GPU central
    differences (relative step 1e-6, over the values actually used) on a
    seeded subset of 64 parameters, 24 R, 24 C and 16 Is, drawn among those
    whose relative sensitivity |p dO/dp| is at least 1e-2 of the largest of
    their kind (a 1e-6 change of a weaker one moves the output by less than
    the forward solves resolve).  Every solve stops at max|dx| < 1e-13 V.
    The output's dependence on Is is weak (|Is dO/dIs| <= ~3e-9 V), so Is
    takes a relative step of 1e-3; a 1e-6 step moves the output by ~1e-14 V.
    R perturbs the plan's conductance base, C a new transient object's C
    values, Is a new plan's descriptors (f32, as the descriptors store it)."""
    import copy
    import torch
    from ohmnivore_b200 import circuits, mna
    rows, nsteps, h = args.adjoint_rows, 500, 2e-12
    ckt = circuits.rc_diode_mesh(rows, rows, seed=4)
    sysm = mna.compile_circuit(ckt)
    comps = S.ComponentTable(ckt, sysm)
    pn = S.NewtonParams(max_iterations=100, abs_tol=1e-13, bicgstab_max_iterations=20000,
                        bicgstab_tolerance=1e-15, inner_rtol=1e-8)
    plan = S.NewtonPlan(sysm, ctx)
    dev = f"cuda:{local_rank}"
    x = torch.zeros(sysm.size, dtype=torch.float64, device=dev)
    plan.newton_device(x.data_ptr(), pn)
    near = sysm.node_index(2 + 10 * rows + 10)
    tr = S.Transient(plan, [near])
    w = np.zeros(sysm.size)
    w[near] = 1.0
    t0 = time.perf_counter()
    try:
        g, info = tr.adjoint(x.data_ptr(), 0.0, h, nsteps, w, comps, pn, 0)
    except S.OhmnivoreError as e:
        raise RuntimeError(f"adjoint: {e}") from e
    adj_s = time.perf_counter() - t0
    x0 = x.clone()

    def forward(p, t):
        xs = torch.zeros(sysm.size, dtype=torch.float64, device=dev)
        try:
            p.newton_device(xs.data_ptr(), pn)
        except S.OhmnivoreError as e:
            raise RuntimeError(f"forward DC: {e}") from e
        try:
            return float(t.run(xs.data_ptr(), 0.0, h, nsteps, pn, steps_per_launch=100)[-1, 0])
        except S.OhmnivoreError as e:
            raise RuntimeError(f"forward transient: {e} {t.last_info}") from e

    rng = np.random.default_rng(7)
    picks = {}
    pval = {"R": comps.r_ohms, "C": comps.c_farads,
            "Is": sysm.diode_descriptors["is_val"].astype(np.float64)}
    step = {"R": 1e-6, "C": 1e-6, "Is": 1e-3}
    for kind, cnt in (("R", 24), ("C", 24), ("Is", 16)):
        rs = np.abs(g[kind] * pval[kind])
        cand = np.flatnonzero(rs >= 1e-2 * np.max(rs))
        picks[kind] = np.sort(rng.choice(cand, size=min(cnt, len(cand)), replace=False))
    gv = sysm.g.val.copy()
    res = {"workload": f"RC-diode mesh {rows}x{rows} ({sysm.size} unknowns), d V(node 10,10)(1 ns)/dp, "
                       f"{nsteps} BE steps of 2 ps", "adjoint_s": adj_s, "output_V": info["output"]}
    t0 = time.perf_counter()
    for kind in ("R", "C", "Is"):
        errs = []
        for j in picks[kind]:
            outs, vals = [], []
            for sign in (1, -1):
                if kind == "R":
                    r0_ = comps.r_ohms[j]
                    r1_ = r0_ * (1 + sign * step["R"])
                    dg = 1.0 / r1_ - 1.0 / r0_
                    a_, b_ = int(comps.r_a[j]), int(comps.r_b[j])
                    v2 = gv.copy()
                    for (ri, ci, sg) in ((a_, a_, 1), (b_, b_, 1), (a_, b_, -1), (b_, a_, -1)):
                        if ri >= 0 and ci >= 0:
                            v2[sysm.g.value_index(ri, ci)] += sg * dg
                    plan.set_base(v2)
                    outs.append(forward(plan, tr))
                    vals.append(r1_)
                elif kind == "C":
                    c0_ = comps.c_farads[j]
                    c1_ = c0_ * (1 + sign * step["C"])
                    s2 = copy.copy(sysm)
                    cc = copy.copy(sysm.c)
                    cc.val = sysm.c.val.copy()
                    a_, b_ = int(comps.c_a[j]), int(comps.c_b[j])
                    for (ri, ci, sg) in ((a_, a_, 1), (b_, b_, 1), (a_, b_, -1), (b_, a_, -1)):
                        if ri >= 0 and ci >= 0:
                            cc.val[cc.value_index(ri, ci)] += sg * (c1_ - c0_)
                    s2.c = cc
                    plan.sysm = s2
                    t2 = S.Transient(plan, [near])
                    plan.sysm = sysm
                    outs.append(forward(plan, t2))
                    t2.close()
                    vals.append(c1_)
                else:
                    s2 = copy.copy(sysm)
                    dd = sysm.diode_descriptors.copy()
                    dd["is_val"][j] = np.float32(float(dd["is_val"][j]) * (1 + sign * step["Is"]))
                    s2.diode_descriptors = dd
                    p2 = S.NewtonPlan(s2, ctx)
                    t2 = S.Transient(p2, [near])
                    outs.append(forward(p2, t2))
                    t2.close()
                    p2.close()
                    vals.append(float(dd["is_val"][j]))
            plan.set_base(gv)
            fd = (outs[0] - outs[1]) / (vals[0] - vals[1])
            errs.append(abs(g[kind][j] - fd) / max(abs(fd), 1e-3 * float(np.max(np.abs(g[kind])))))
        res[kind] = {"parameters": len(picks[kind]), "relative_step": step[kind],
                     "max_rel_err": float(max(errs)), "median_rel_err": float(np.median(errs)),
                     "within_1e-6": int(sum(e <= 1e-6 for e in errs))}
    res["fd_wall_s"] = time.perf_counter() - t0
    tr.close()
    plan.close()
    del x0
    return res


def run_profile_case(args):
    """Profiling case: one warm-up solve and one solve of the workload."""
    import torch
    from ohmnivore_b200 import circuits, mna
    from ohmnivore_b200 import solver as S
    if args.profile == "grid":
        ckt = circuits.rc_diode_mesh(args.grid_rows, args.grid_rows, seed=4)
        src = int(np.flatnonzero(ckt.kind == circuits.V)[0])
        ckt.value[src] = 1.0
        ckt.tran.pop(src, None)
        sysm = mna.compile_circuit(ckt)
        ctx = S.Context(0)
        plan = S.NewtonPlan(sysm, ctx)
        x = torch.zeros(sysm.size, dtype=torch.float64, device="cuda")
        params = S.NewtonParams(max_iterations=1, abs_tol=1e-9, bicgstab_max_iterations=40,
                                bicgstab_tolerance=1e-14, inner_rtol=1e-12)
        for _ in range(2):
            x.zero_()
            torch.cuda.synchronize()
            try:
                plan.newton_device(x.data_ptr(), params)
            except (S.SolveError, S.NewtonNotConverged):
                pass                     # the capped Krylov solve is expected to stop unconverged
        print(json.dumps({"profile_case": f"RC-diode mesh {args.grid_rows}x{args.grid_rows} at 1 V, one Newton "
                                          "iteration, 40 BiCGSTAB iterations", **plan.last_info}))
        plan.close()
        ctx.close()
        return
    sysm = mna.compile_circuit(circuits.diode_mesh(args.rows, args.cols, seed=1))
    ctx = S.Context(0)
    plan = S.NewtonPlan(sysm, ctx)
    x = torch.zeros(sysm.size, dtype=torch.float64, device="cuda")
    params = newton_params(args.profile == "mixed")
    for _ in range(2):
        x.zero_()
        torch.cuda.synchronize()
        info = plan.newton_device(x.data_ptr(), params)
    print(json.dumps({"profile_case": f"diode-mesh {args.rows}x{args.cols}", "precision": args.profile,
                      **info}))
    plan.close()
    ctx.close()


def spmv_roofline(S, ctx, sysm, stream, flush):
    """Stand-alone CSR SpMV (the backend op) on the workload matrix, L2
    flushed before every launch; algorithmic bytes / event time."""
    import torch
    be = S.SolverBackend(ctx)
    A = be.upload_matrix(sysm.g)
    bx = be.new_buffer(sysm.size)
    by = be.new_buffer(sysm.size)
    bx.upload(np.ones(sysm.size))
    reps = 20
    ms = []
    for r in range(reps + 3):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        be.spmv(A, bx, by)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        if r >= 3:
            ms.append(e0.elapsed_time(e1))
    t = statistics.median(ms) * 1e-3
    byt = spmv_bytes(sysm.size, sysm.g.nnz, 8, 8)
    peaks = measured_peaks()
    peak = peaks["hbm_gbs"] if peaks else 6650.0
    out = {"kernel": "spmv_row_kernel (FP64, one thread per row)", "bytes": byt, "us": t * 1e6,
           "achieved_gbs": byt / t / 1e9, "frac": byt / t / 1e9 / peak, "cold_l2": True,
           "note": "the workload matrix (20 MB): launch latency dominates at this size"}
    # HBM-bound size: a 4096 x 4096 five-point mesh matrix (the structure of
    # the MNA meshes), 16.8 M rows, 83.9 M nonzeros, random values
    m = 4096
    n = m * m
    idx = np.arange(n, dtype=np.int64)
    i, j = idx // m, idx % m
    nbr = [idx - m, idx - 1, idx, idx + 1, idx + m]
    ok = [i > 0, j > 0, np.ones(n, bool), j < m - 1, i < m - 1]
    cnt = np.sum(ok, axis=0)
    rp = np.concatenate([[0], np.cumsum(cnt)]).astype(np.int64)
    col = np.stack([np.where(o, c, -1) for c, o in zip(nbr, ok)], axis=1).reshape(-1)
    col = col[col >= 0]
    del nbr, ok, idx, i, j
    val = np.random.default_rng(9).uniform(-1.0, 1.0, len(col))
    big = type(sysm.g)(n, n, rp, col, val)
    A2 = be.upload_matrix(big)
    bx2, by2 = be.new_buffer(n), be.new_buffer(n)
    bx2.upload(np.ones(n))
    ms2 = []
    for r in range(8):
        with torch.cuda.stream(stream):
            flush.zero_()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
        be.spmv(A2, bx2, by2)
        with torch.cuda.stream(stream):
            e1.record(stream)
        e1.synchronize()
        if r >= 3:
            ms2.append(e0.elapsed_time(e1))
    t2 = statistics.median(ms2) * 1e-3
    byt2 = spmv_bytes(n, len(col), 8, 8)
    out["hbm_bound"] = {"matrix": f"5-point mesh 4096x4096: {n} rows, {len(col)} nonzeros",
                        "bytes": byt2, "us": t2 * 1e6, "achieved_gbs": byt2 / t2 / 1e9,
                        "frac": byt2 / t2 / 1e9 / peak, "peak_gbs": peak}
    for h in (A2, bx2, by2):
        h.close()
    return out


if __name__ == "__main__":
    main()
