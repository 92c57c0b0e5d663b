#!/usr/bin/env python
"""Benchmark of the sparse iterative-solve path on B200.

Headline step: one Csr SpMV (FP64 values, int32 indices, 1 right-hand side)
on the 3D 7-point Poisson matrix of a 128^3 grid (n = 2,097,152,
nnz = 14,581,760), x ~ N(0, 1) from a seed.  value = algorithmic bytes of
one SpMV / device time, in GB/s; the roofline fraction is against the
measured HBM copy bandwidth.  The matrix and vectors (217 MB) exceed the
126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
                  [--sweep] [--no-solve] [--no-extra] [--mtx] [--profile-tour]

The same line carries the time-to-1e-10 GMRES section (FP64, IR+FP32,
IR+BF16, CB-GMRES with an FP32 basis) and, unless --no-extra, the CG,
batched BiCGStab, differentiable-solve and block Jacobi sections.  --mtx
times the host matrix I/O instead (no GPU).

--impl reference times the CPU restatement of the reference executor's
SpMV (oracle/, OpenMP over all host cores) on the same workload.  Under
torchrun every rank runs its own replica (the path does not shard); rank 0
prints one JSON line.
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

METRIC = ("time-to-1e-10 rel. residual, mixed vs FP64 on GPU; "
          "SpMV GB/s as % of HBM peak")
GRID = 128
SEED = 0


def csr_bytes(n, nnz, k, vb, ib=4, beta=False):
    """Compulsory bytes of one Csr SpMV: values + col_idxs + row_ptrs + x
    read once + y written once (+ y read when beta != 0)."""
    return nnz * (vb + ib) + (n + 1) * ib + k * n * (vb + vb) + (k * n * vb if beta else 0)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_traffic(name):
    """DRAM bytes per launch of the named kernel from the committed ncu
    summary (profiles/traffic.json), or None."""
    p = os.path.join(ROOT, "profiles", "traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f).get(name)
    return None


class ClockSampler:
    """Samples nvidia-smi clocks and throttle reasons in the background."""

    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,"
              "clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.samples = []
        self._stop = threading.Event()
        self._t = None

    def __enter__(self):
        def loop():
            while not self._stop.is_set():
                try:
                    out = subprocess.run(
                        ["nvidia-smi", "-i", str(self.index),
                         "--query-gpu=" + self.FIELDS,
                         "--format=csv,noheader,nounits"],
                        capture_output=True, text=True, timeout=5).stdout
                    parts = [p.strip() for p in out.strip().split(",")]
                    if len(parts) == 7:
                        self.samples.append(parts)
                except Exception:
                    pass
                self._stop.wait(0.1)
        self._t = threading.Thread(target=loop, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *exc):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = [float(s[0]) for s in self.samples if s[0].replace(".", "").isdigit()]
        mx = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown",
                 "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4)
                          if s[3 + i].lower().startswith("active")})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(self.samples)}


def dist_env():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def max_over_ranks(values, device):
    """Each per-rank time replaced by its maximum over all ranks of the
    default process group (every rank gets the result): the whole job is as
    slow as its slowest rank."""
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(v) for v in values], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return [float(v) for v in t.tolist()]


def build_matrix():
    from ginkgo_b200 import stencils
    rp, ci, v = stencils.poisson_3d_7pt(GRID)
    return rp, ci, v


def run_reference(args):
    """CPU restatement of the reference's Csr SpMV (oracle, OpenMP)."""
    world, rank, _ = dist_env()
    if rank != 0:
        return
    from oracle import oracle as orc
    rp, ci, v = build_matrix()
    n, nnz = len(rp) - 1, len(ci)
    x = np.random.default_rng(SEED).standard_normal(n)
    y = np.empty(n)
    threads = os.cpu_count() or 1
    for _ in range(max(args.warmup, 1)):
        orc.csr_spmv_par(rp, ci, v, x, y, threads)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        orc.csr_spmv_par(rp, ci, v, x, y, threads)
    dt = (time.perf_counter() - t0) / args.steps
    gbs = csr_bytes(n, nnz, 1, 8) / dt / 1e9
    out = {
        "impl": "reference", "metric": METRIC, "value": round(gbs, 2),
        "unit": "GB/s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": round(dt * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic",
        "config": {"workload": "csr_spmv_poisson3d_7pt_128", "n": n,
                   "nnz": nnz, "num_rhs": 1, "format": "csr",
                   "value_type": "f64", "index_type": "int32"},
        "cpu_baseline": {"value": round(gbs, 2), "unit": "GB/s",
                         "cores": threads, "kind": "port",
                         "sample": f"{args.steps} full SpMVs (n={n})"},
        "e2e": {"value": round(gbs, 2), "unit": "GB/s",
                "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out), flush=True)


def cpu_baseline(rp, ci, v, budget_s=12.0):
    from oracle import oracle as orc
    n, nnz = len(rp) - 1, len(ci)
    x = np.random.default_rng(SEED).standard_normal(n)
    y = np.empty(n)
    threads = os.cpu_count() or 1
    orc.csr_spmv_par(rp, ci, v, x, y, threads)
    reps, t0 = 0, time.perf_counter()
    while time.perf_counter() - t0 < budget_s and reps < 2000:
        orc.csr_spmv_par(rp, ci, v, x, y, threads)
        reps += 1
    dt = (time.perf_counter() - t0) / reps
    return {"value": round(csr_bytes(n, nnz, 1, 8) / dt / 1e9, 2),
            "unit": "GB/s", "cores": threads, "kind": "port",
            "sample": f"{reps} full Csr FP64 SpMVs of the same matrix "
                      f"({dt * 1e3:.2f} ms each), oracle with OpenMP"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", default="b200")
    ap.add_argument("--strategy", default="auto",
                    choices=["auto", "classical", "load_balance"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sweep", action="store_true",
                    help="also time every format / precision / k on matrix A")
    ap.add_argument("--no-solve", action="store_true",
                    help="skip the time-to-1e-10 mixed vs FP64 GMRES section")
    ap.add_argument("--no-extra", action="store_true",
                    help="skip the batched BiCGStab and differentiable-solve sections")
    ap.add_argument("--solve-case", choices=["f64", "ir_f32", "ir_bf16", "cb_f32"],
                    help="profiling aid: run one GMRES variant on the 27-point "
                    "operator for --solve-iters iterations and exit")
    ap.add_argument("--solve-iters", type=int, default=60)
    ap.add_argument("--profile-tour", action="store_true",
                    help="profiling aid: one capped invocation of every kernel "
                    "family (SpMV formats, conversions, CG, BiCGStab, batch, "
                    "transpose + SDDMM) and exit")
    ap.add_argument("--profile-op", choices=sorted(PROFILE_OPS),
                    help="profiling aid: three launches of one operation on the "
                    "7-point 128^3 matrix (inputs larger than L2) and exit, the "
                    "small case for a single-kernel ncu capture")
    ap.add_argument("--mtx", action="store_true",
                    help="host-side matrix I/O: MatrixMarket text and binary "
                    "read/write of the 128^3 matrix (no GPU needed) and exit")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    if args.mtx:
        return mtx_section(args.steps if "--steps" in sys.argv else 3)
    if args.impl == "reference":
        return run_reference(args)
    if args.solve_case:
        return solve_case(args.solve_case, args.solve_iters)
    if args.profile_tour:
        return profile_tour()
    if args.profile_op:
        return profile_op(args.profile_op)

    import torch
    world, rank, local = dist_env()
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from ginkgo_b200.matrix import Csr, CudaExecutor

    exe = CudaExecutor.create(local)
    rp, ci, v = build_matrix()
    n, nnz = len(rp) - 1, len(ci)
    A = Csr.read(exe, rp, ci, v)
    x = torch.from_numpy(np.random.default_rng(SEED).standard_normal(n)).cuda()
    y = torch.empty(n, dtype=torch.float64, device="cuda")
    stream = torch.cuda.current_stream()

    def time_op(op, steps, warmup):
        for _ in range(warmup):
            op()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            op()
        e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / 1e3 / steps

    def time_graph(op, steps, warmup):
        """Device time of op (one library call): the call is captured once in
        a CUDA graph (the library launches on the current stream) and the
        graph replayed, so the host cost of the Python binding (tensor
        checks, ctypes marshalling: comparable to the 40 us kernel) does not
        leave the GPU idle between steps.  The same kernel with the same
        arguments runs every step."""
        op()  # first-use set-up (occupancy queries) outside the capture
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            op()
        out = time_op(g.replay, steps, warmup)
        del g
        return out

    # pick the faster Csr strategy for the headline (both are reported)
    per_strategy = {}
    for strat in ("classical", "load_balance"):
        A.set_strategy(strat)
        per_strategy[strat] = time_graph(lambda: A.apply(x, y), 20, 3)
    strategy = (min(per_strategy, key=per_strategy.get)
                if args.strategy == "auto" else args.strategy)
    A.set_strategy(strategy)

    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        t_step = time_graph(lambda: A.apply(x, y), args.steps, args.warmup)
        # end-to-end through the public API with host buffers: every step
        # copies its x from pinned host memory and its y back, pipelined over
        # three streams (the next step's upload and the previous step's
        # download overlap this step's product, the two copy directions run
        # at once), with two device and host buffers per vector
        t_e2e = time_e2e(A, n, max(args.steps, 20), 3)
    if world > 1:
        t_step, t_e2e = max_over_ranks([t_step, t_e2e], "cuda")

    nbytes = csr_bytes(n, nnz, 1, 8)
    gbs = nbytes / t_step / 1e9
    peak, peak_kind = measured_peaks()
    kernel = f"csr_{strategy}"
    result = {
        "metric": METRIC,
        "value": round(gbs * world, 2),
        "unit": "GB/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": round(t_step * 1e3, 5),
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f64",
        "data": "synthetic",
        "config": {"workload": "csr_spmv_poisson3d_7pt_128", "n": n, "nnz": nnz,
                   "num_rhs": 1, "format": "csr", "strategy": strategy,
                   "value_type": "f64", "index_type": "int32",
                   "l2": "inputs (217 MB) larger than L2 (126 MB), no flush",
                   "timing": "device: CUDA-graph replays of one A.apply call; "
                             "e2e: A.apply calls, each step's x uploaded from and y "
                             "downloaded to pinned host memory, the copies of "
                             "neighbouring steps overlapped on two copy streams",
                   "parallelism": f"replicas{world}"},
        "roofline": {"bound": "hbm", "achieved": round(gbs, 1),
                     "peak": peak, "unit": "GB/s",
                     "frac": round(gbs / peak, 4),
                     "peak_kind": peak_kind,
                     "frac_of_8tbs_spec": round(gbs / 8000.0, 4),
                     "traffic": committed_traffic(kernel),
                     "algorithmic_bytes": nbytes, "kernel": kernel},
        "strategies_ms": {k: round(t * 1e3, 5) for k, t in per_strategy.items()},
        "e2e": {"value": round(nbytes / t_e2e / 1e9 * world, 2), "unit": "GB/s",
                "h2d_bytes_per_step": n * 8, "d2h_bytes_per_step": n * 8,
                "ms_per_step": round(t_e2e * 1e3, 4)},
        "gpu_launches": args.steps + max(args.steps // 4, 5),
        "clocks": clk.summary(),
    }
    if args.sweep:
        result["sweep"] = sweep(exe, rp, ci, v, time_graph)
    if not args.no_solve:
        solve = ir_gmres_section(exe, stream)
        result["ir_gmres"] = solve
        result["gpu_launches"] += solve.pop("gpu_launches")
    if not args.no_extra:
        for key, fn in (("cg", cg_section), ("krylov_iteration", krylov_iteration_section),
                        ("batch_bicgstab", batch_section),
                        ("autograd", autograd_section),
                        ("block_jacobi", block_jacobi_section)):
            try:
                result[key] = fn(exe, stream)
            except Exception as e:  # a failed optional section is reported, not fatal
                result[key] = {"error": f"{type(e).__name__}: {e}"[:300]}
    if rank == 0 and not args.no_cpu_baseline:
        result["cpu_baseline"] = cpu_baseline(rp, ci, v)
    if rank == 0:
        print(json.dumps(result), flush=True)
    if world > 1:
        torch.distributed.destroy_process_group()


def gmres_variants(max_iters):
    """GMRES(30) + scalar Jacobi to 1e-10: plain FP64, iterative refinement
    around an FP32 / BF16-basis inner cycle, and compressed-basis GMRES
    (FP64 arithmetic over an FP32 basis)."""
    from ginkgo_b200.solver import CbGmres, Gmres, Ir, Iteration, Jacobi, ResidualNorm
    crit = (Iteration.build().with_max_iters(max_iters),
            ResidualNorm.build().with_reduction_factor(1e-10))
    jac = Jacobi.build().with_max_block_size(1)
    return {
        "f64": Gmres.build().with_krylov_dim(30).with_criteria(*crit)
        .with_preconditioner(jac),
        "ir_f32": Ir.build().with_criteria(*crit).with_solver(
            Gmres.build().with_krylov_dim(30).with_storage_precision("f32")
            .with_preconditioner(jac)),
        "ir_bf16": Ir.build().with_criteria(*crit).with_solver(
            Gmres.build().with_krylov_dim(30).with_storage_precision("bf16")
            .with_preconditioner(jac)),
        "cb_f32": CbGmres.build().with_krylov_dim(30).with_storage_precision("reduce1")
        .with_criteria(*crit).with_preconditioner(jac),
    }


def solve_case(name, iters, grid=96):
    """One capped solve of one variant on the 27-point operator, untimed:
    the workload of the GMRES kernel profiles."""
    import torch
    from ginkgo_b200 import stencils
    from ginkgo_b200.matrix import Csr, CudaExecutor
    exe = CudaExecutor.create(0)
    rp, ci, v = stencils.anisotropic_27pt(grid)
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    b = torch.from_numpy(np.random.default_rng(3).standard_normal(n)).cuda()
    s = gmres_variants(iters)[name].on(exe).generate(A)
    x = torch.zeros(n, dtype=torch.float64, device="cuda")
    s.apply(b, x)
    torch.cuda.synchronize()
    print(json.dumps({"solve_case": name, "workload": f"aniso27_{grid}",
                      "iterations": s.logger.num_iterations,
                      "residual_norm": np.asarray(s.logger.residual_norm,
                                                 dtype=float).tolist()}))


def mtx_section(steps):
    """Host-side matrix I/O on the 7-point 128^3 matrix (14.6M entries): the
    library's MatrixMarket text and binary readers and writers through the
    Python API (bytes in and out, numpy arrays), best of `steps` runs each,
    checked bit-exact against the source arrays; and the oracle
    restatement on a bounded sample as the CPU-port baseline."""
    from ginkgo_b200 import mtx_io as M
    from oracle import mtx as O
    rp, ci, v = build_matrix()
    n = len(rp) - 1
    rows = np.repeat(np.arange(n, dtype=np.int32), np.diff(rp))
    data = M.MatrixData((n, n), rows, np.asarray(ci, np.int32), np.asarray(v, np.float64))
    lower = np.asarray(ci) <= rows
    perm = np.random.default_rng(SEED).permutation(int(lower.sum()))
    sym = M.MatrixData((n, n), rows[lower][perm], np.asarray(ci, np.int32)[lower][perm],
                       np.asarray(v, np.float64)[lower][perm])

    def best(f):
        ts = []
        for _ in range(max(steps, 1)):
            t0 = time.perf_counter()
            out = f()
            ts.append(time.perf_counter() - t0)
        return min(ts), out

    t_w, text = best(lambda: M.write_raw(data).encode())
    t_r, back = best(lambda: M.read_raw(text))
    t_bw, binary = best(lambda: M.write_binary_raw(data))
    t_br, bback = best(lambda: M.read_binary_raw(binary))
    sym_text = M.write_raw(sym).replace("real general", "real symmetric", 1).encode()
    t_s, sback = best(lambda: M.read_raw(sym_text))
    for d in (back, bback, sback):
        assert np.array_equal(d.row_idxs, rows) and np.array_equal(d.col_idxs, ci) \
            and np.array_equal(d.values, v), "matrix I/O round trip differs"
    k = 200_000
    sample = M.write_raw(M.MatrixData((n, n), rows[:k], np.asarray(ci[:k], np.int32),
                                      np.asarray(v[:k], np.float64)))
    t0 = time.perf_counter()
    O.read_raw(sample)
    t_o = time.perf_counter() - t0
    nnz = len(ci)
    mb = lambda nbytes, t: round(nbytes / t / 1e6, 1)  # noqa: E731
    print(json.dumps({
        "mtx_io": {"workload": "poisson3d_7pt_128", "entries": nnz,
                   "host_threads": os.cpu_count(),
                   "text_bytes": len(text), "binary_bytes": len(binary),
                   "read_text_s": round(t_r, 3), "read_text_mb_s": mb(len(text), t_r),
                   "read_text_mentries_s": round(nnz / t_r / 1e6, 2),
                   "write_text_s": round(t_w, 3), "write_text_mb_s": mb(len(text), t_w),
                   "read_binary_s": round(t_br, 3), "read_binary_mb_s": mb(len(binary), t_br),
                   "write_binary_s": round(t_bw, 3),
                   "read_symmetric_shuffled_s": round(t_s, 3),
                   "symmetric_text_bytes": len(sym_text),
                   "cpu_baseline": {"kind": "port", "cores": 1,
                                    "value": round(k / t_o / 1e6, 3), "unit": "M entries/s",
                                    "sample": f"oracle read of the first {k} entries"},
                   "steps": steps}}), flush=True)


def time_e2e(A, n, steps, warmup):
    """Seconds per step of y_i = A x_i through A.apply with host buffers:
    step i uploads x_i (pinned host -> device) on a copy stream, multiplies
    on the compute stream once its upload is done, and downloads y_i on a
    second copy stream once its product is done; buffers alternate between
    two slots, each reused only after the step two before has released it.
    Timed with CUDA events from before the first upload to after the last
    download, the steps after `warmup` untimed ones."""
    import torch
    rng = np.random.default_rng(SEED)
    xh = [torch.from_numpy(rng.standard_normal(n)).pin_memory() for _ in range(2)]
    yh = [torch.empty(n, dtype=torch.float64).pin_memory() for _ in range(2)]
    xd = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    yd = [torch.empty(n, dtype=torch.float64, device="cuda") for _ in range(2)]
    s_in, s_comp, s_out = torch.cuda.Stream(), torch.cuda.Stream(), torch.cuda.Stream()
    ev = lambda: torch.cuda.Event()
    up, done, down = [ev(), ev()], [ev(), ev()], [ev(), ev()]
    for e in up + done + down:
        e.record(torch.cuda.current_stream())

    def step(i):
        k = i % 2
        with torch.cuda.stream(s_in):
            s_in.wait_event(done[k])        # the product of step i - 2 read xd[k]
            xd[k].copy_(xh[k], non_blocking=True)
            up[k].record(s_in)
        with torch.cuda.stream(s_comp):
            s_comp.wait_event(up[k])
            s_comp.wait_event(down[k])      # the download of step i - 2 read yd[k]
            A.apply(xd[k], yd[k])
            done[k].record(s_comp)
        with torch.cuda.stream(s_out):
            s_out.wait_event(done[k])
            yh[k].copy_(yd[k], non_blocking=True)
            down[k].record(s_out)

    for i in range(warmup):
        step(i)
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(s_in)
    s_comp.wait_event(e0)
    s_out.wait_event(e0)
    for i in range(warmup, warmup + steps):
        step(i)
    s_in.wait_stream(s_out)
    s_in.wait_stream(s_comp)
    e1.record(s_in)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / steps


def profile_tour():
    """One capped invocation of every kernel family on inputs larger than
    L2, for the ncu launch list: SpMV in every format (FP64, one and four
    right-hand sides) on the 7-point 128^3 matrix, the Ell and Sellp
    conversions, 20 CG and 20 BiCGStab iterations (one and sixteen
    right-hand sides), the batched BiCGStab on 1024 systems, the transpose +
    SDDMM of the differentiable solve, mixed-type Csr/Ell SpMV, block Jacobi
    (blocks of 8), 10 Arnoldi steps of GMRES and of every CB-GMRES basis
    format, CG / BiCGStab / GMRES with block Jacobi inside (blocks of 8),
    CG with adaptive-precision blocks and their apply, SpGEMM (A^2), SpGEAM
    and the Hybrid conversions and SpMV."""
    import torch
    from ginkgo_b200 import stencils
    from ginkgo_b200._lib import call
    from ginkgo_b200.batch import BatchBicgstab, convection_diffusion_batch
    from ginkgo_b200.matrix import Csr, CudaExecutor, _p, _stream
    from ginkgo_b200.solver import Bicgstab, Cg, Iteration, Jacobi, ResidualNorm
    exe = CudaExecutor.create(0)
    rp, ci, v = stencils.poisson_3d_7pt(128)
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    E = A.convert_to_ell()
    S = A.convert_to_sellp(32, 1)
    rng = np.random.default_rng(0)
    for k in (1, 4):
        x = torch.from_numpy(rng.standard_normal((n, k))).cuda()
        y = torch.empty((n, k), dtype=torch.float64, device="cuda")
        for name in ("classical", "load_balance", "ell", "sellp"):
            op = E if name == "ell" else S if name == "sellp" else A.set_strategy(name)
            op.apply(x, y)
    A.set_strategy("classical")
    crit = (Iteration.build().with_max_iters(20), ResidualNorm.build().with_reduction_factor(1e-14))
    jac = Jacobi.build().with_max_block_size(1)
    for k in (1, 16):
        b = torch.from_numpy(rng.standard_normal((n, k))).cuda()
        for fac in (Cg, Bicgstab):
            s = fac.build().with_criteria(*crit).with_preconditioner(jac).on(exe).generate(A)
            x = torch.zeros_like(b)
            s.apply(b, x)
    Ab, _ = convection_diffusion_batch(exe, 1024, lo=32, hi=1024, seed=3)
    bb = torch.from_numpy(rng.standard_normal(Ab.total_rows)).cuda()
    sb = (BatchBicgstab.build().with_max_iterations(500).with_tolerance(1e-8)
          .with_tolerance_type("relative").with_preconditioner("jacobi").on(exe).generate(Ab))
    sb.apply(bb, torch.zeros_like(bb))
    At = A.transpose()
    lam = torch.from_numpy(rng.standard_normal((n, 16))).cuda()
    xx = torch.from_numpy(rng.standard_normal((n, 16))).cuda()
    g = torch.empty_like(A.values)
    call("b2s_csr_sddmm_f64", n, _p(At.row_ptrs), _p(At.col_idxs), At.max_row_nnz, _p(lam),
         lam.stride(0), _p(xx), xx.stride(0), 16, -1.0, _p(g), _stream(g))
    # mixed value types: FP32 matrix with FP64 vectors (Csr and Ell)
    A32 = A.convert_to_precision(torch.float32)
    x1 = torch.from_numpy(rng.standard_normal((n, 1))).cuda()
    y1 = torch.empty_like(x1)
    A32.apply(x1, y1)
    A32.convert_to_ell().apply(x1, y1)
    # block Jacobi (blocks of 8), generate and apply
    from ginkgo_b200.solver import BlockJacobi, CbGmres, Gmres
    bj = BlockJacobi(A, 8)
    bj.apply(x1, y1)
    # 10 Arnoldi steps of GMRES and of each CB-GMRES basis format
    crit10 = (Iteration.build().with_max_iters(10), ResidualNorm.build().with_reduction_factor(1e-14))
    for fac in [Gmres.build().with_krylov_dim(30)] + [
            CbGmres.build().with_krylov_dim(30).with_storage_precision(sp)
            for sp in ("reduce1", "reduce2", "integer", "ireduce1", "ireduce2")]:
        s = fac.with_criteria(*crit10).with_preconditioner(jac).on(exe).generate(A)
        s.apply(x1[:, 0].contiguous(), torch.zeros(n, dtype=torch.float64, device="cuda"))
    # block Jacobi inside CG, BiCGStab and GMRES (blocks of 8 consecutive rows)
    jb = Jacobi.build().with_max_block_size(8).with_block_pointers(np.arange(0, n + 1, 8))
    b1 = x1[:, 0].contiguous()
    for fac in (Cg.build().with_criteria(*crit), Bicgstab.build().with_criteria(*crit),
                Gmres.build().with_krylov_dim(30).with_criteria(*crit10)):
        s = fac.with_preconditioner(jb).on(exe).generate(A)
        s.apply(b1, torch.zeros(n, dtype=torch.float64, device="cuda"))
    # adaptive-precision blocks (autodetection: FP16 storage on this matrix)
    # inside CG, and their stand-alone apply
    jba = (Jacobi.build().with_max_block_size(8).with_block_pointers(np.arange(0, n + 1, 8))
           .with_storage_optimization(0xFF))
    s = Cg.build().with_criteria(*crit).with_preconditioner(jba).on(exe).generate(A)
    s.apply(b1, torch.zeros(n, dtype=torch.float64, device="cuda"))
    s.precond.apply(x1, y1)
    # sparse products: A^2 (SpGEMM), A + A (SpGEAM), Csr -> Hybrid -> SpMV, Csr
    from ginkgo_b200.matrix import spgeam, spgemm
    spgemm(A, A)
    spgeam(1.0, A, -0.5, A)
    H = A.convert_to_hybrid("imbalance_limit", percent=0.5)
    H.apply(x1, y1)
    H.convert_to_csr()
    torch.cuda.synchronize()
    print(json.dumps({"profile_tour": "done", "n": n}))


# operations of --profile-op: the kernel each one runs three times
PROFILE_OPS = {
    "lb1": "csr_lb_kernel (load_balance, one right-hand side)",
    "lb16": "csr_lb_lanes_kernel (load_balance, 16 right-hand sides)",
    "cg_block": "cg_block_kernel (CG update pass with 8-row block Jacobi)",
    "cg_block_f16": "cg_block_kernel (CG update pass, 8-row blocks stored in FP16)",
    "lb1_b": "csr_lb1_kernel (load_balance, one column, power-law matrix B)",
    "classical_b": "csr classical (one column, power-law matrix B)",
    "bicg_block": "bicg_block_vec_kernel (BiCGStab with 8-row block Jacobi)",
    "sddmm16": "sddmm_lanes_kernel (16 columns)",
    "spgemm": "gemm_*_rows_kernel (A^2)",
    "mixed": "csr_mixed_kernel (FP32 matrix, FP64 vectors)",
    "jacobi_apply": "jacobi_block_apply_kernel (8-row blocks)",
    "ell4": "rhs_lanes_kernel (Ell, 4 right-hand sides)",
    "bicg16": "bicg_vec_lanes_kernel / bicg_update_lanes_kernel (BiCGStab, 16 RHS)",
}


def profile_op(op):
    """Three launches of one operation on the 7-point 128^3 matrix (217 MB of
    Csr, larger than L2; matrix B for the *_b operations), for a
    single-kernel ncu capture with -k and -c."""
    import torch
    from ginkgo_b200 import stencils
    from ginkgo_b200._lib import call
    from ginkgo_b200.matrix import Csr, CudaExecutor, _p, _stream, spgemm
    from ginkgo_b200.solver import Bicgstab, BlockJacobi, Cg, Iteration, Jacobi, ResidualNorm
    exe = CudaExecutor.create(0)
    if op.endswith("_b"):
        # matrix B: power-law, n = 4M, 80M entries (1 GB of Csr)
        rp, ci, v = stencils.power_law(4_000_000, seed=0, mu=2.5, sigma=1.0, max_len=4096)
    else:
        rp, ci, v = stencils.poisson_3d_7pt(128)
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    rng = np.random.default_rng(0)
    k = 16 if op in ("lb16", "sddmm16", "bicg16") else 4 if op == "ell4" else 1
    x = torch.from_numpy(rng.standard_normal((n, k))).cuda()
    y = torch.empty_like(x)
    crit = (Iteration.build().with_max_iters(3), ResidualNorm.build().with_reduction_factor(1e-14))
    jb = Jacobi.build().with_max_block_size(8).with_block_pointers(np.arange(0, n + 1, 8))
    for _ in range(3):
        if op in ("lb1", "lb16", "lb1_b"):
            A.set_strategy("load_balance").apply(x, y)
        elif op == "classical_b":
            A.apply(x, y)
        elif op in ("cg_block", "bicg_block", "cg_block_f16"):
            fac = Bicgstab if op == "bicg_block" else Cg
            if op == "cg_block_f16":
                jb = jb.with_storage_optimization(0x02)  # precision_reduction(0, 2)
            s = fac.build().with_criteria(*crit).with_preconditioner(jb).on(exe).generate(A)
            s.apply(x[:, 0].contiguous(), torch.zeros(n, dtype=torch.float64, device="cuda"))
        elif op == "sddmm16":
            g = torch.empty_like(A.values)
            call("b2s_csr_sddmm_f64", n, _p(A.row_ptrs), _p(A.col_idxs), A.max_row_nnz, _p(x),
                 x.stride(0), _p(y), y.stride(0), 16, -1.0, _p(g), _stream(g))
        elif op == "spgemm":
            spgemm(A, A)
        elif op == "mixed":
            A.convert_to_precision(torch.float32).apply(x, y)
        elif op == "jacobi_apply":
            BlockJacobi(A, 8, np.arange(0, n + 1, 8)).apply(x, y)
        elif op == "ell4":
            A.convert_to_ell().apply(x, y)
        elif op == "bicg16":
            s = (Bicgstab.build().with_criteria(*crit)
                 .with_preconditioner(Jacobi.build().with_max_block_size(1)).on(exe).generate(A))
            s.apply(x, torch.zeros_like(x))
    torch.cuda.synchronize()
    print(json.dumps({"profile_op": op, "kernel": PROFILE_OPS[op], "n": n}))


def ir_gmres_section(exe, stream, grid=96, reps=3):
    """Time to a relative residual of 1e-10 (verified on the explicit FP64
    residual) on the 3D 27-point anisotropic operator (96^3, coefficients
    1, 1e-2, 1e-4), GMRES(30) + scalar Jacobi: plain FP64 GMRES against
    iterative refinement with an FP32 and a BF16-basis inner cycle.  Each
    timed solve starts from x = 0 and includes the graph set-up and the
    host convergence checks; the median of `reps` solves is reported."""
    import torch
    from ginkgo_b200 import stencils
    from ginkgo_b200.matrix import Csr
    rp, ci, v = stencils.anisotropic_27pt(grid)
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    b = torch.from_numpy(np.random.default_rng(3).standard_normal(n)).cuda()
    variants = gmres_variants(20000)
    out = {"workload": f"aniso27_{grid}", "n": n, "nnz": len(ci),
           "krylov_dim": 30, "goal": 1e-10}
    sols = {}
    launches = 0
    bnorm = float(b.norm())
    for name, fac in variants.items():
        s = fac.on(exe).generate(A)
        times = []
        for rep in range(reps + 1):
            x = torch.zeros(n, dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            s.apply(b, x)
            e1.record(stream)
            torch.cuda.synchronize()
            if rep > 0:
                times.append(e0.elapsed_time(e1))
        r = torch.empty_like(x)
        A.apply(-1.0, x, 0.0, r)
        r += b
        rel = float(r.norm()) / bnorm
        it = s.logger.num_iterations
        launches += reps * (4 * it + 3 * s.logger.restarts + 4)
        sols[name] = x
        out[name] = {"ms": round(float(np.median(times)), 3),
                     "iterations": it, "restarts": s.logger.restarts,
                     "converged": s.logger.has_converged,
                     "explicit_rel_residual": rel}
    for name in ("ir_f32", "ir_bf16", "cb_f32"):
        out[name]["error_vs_f64"] = float((sols[name] - sols["f64"]).norm() /
                                          sols["f64"].norm())
        out[name]["speedup_vs_f64"] = round(out["f64"]["ms"] / out[name]["ms"], 3)
    out["gpu_launches"] = launches
    return out


def block_jacobi_section(exe, stream, block_size=8):
    """Block Jacobi on the 7-point 128^3 matrix: blocks of up to block_size
    rows (consecutive single-row natural blocks merged), device generate
    (pivoted Gauss-Jordan per block) and apply with one right-hand side.
    Apply bytes: the stored blocks (block_size^2 values each) + b + x +
    the block pointers."""
    import torch
    from ginkgo_b200.matrix import Csr
    from ginkgo_b200.solver import BlockJacobi
    rp, ci, v = build_matrix()
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    bj = BlockJacobi(A, block_size)
    gen_ms = _event_ms(lambda: BlockJacobi(A, block_size, bj.block_pointers), stream)
    b = torch.from_numpy(np.random.default_rng(SEED).standard_normal(n)).cuda()
    x = torch.empty_like(b)
    apply_ms = _graph_ms(lambda: bj.apply(b, x), stream)
    nbytes = bj.num_blocks * block_size * block_size * 8 + 2 * n * 8 + (bj.num_blocks + 1) * 4
    peak, _ = measured_peaks()
    # adaptive precision (autodetection): the blocks of this matrix are
    # stored in FP16, two bytes per value
    ba = BlockJacobi(A, block_size, bj.block_pointers, storage_optimization=0xFF)
    gen_a_ms = _event_ms(lambda: BlockJacobi(A, block_size, bj.block_pointers,
                                             storage_optimization=0xFF), stream)
    prec = np.unique(ba.block_precisions).tolist()
    value_bytes = {0x00: 8, 0x01: 4, 0x02: 2, 0x10: 4, 0x11: 2, 0x20: 2}
    abytes = (bj.num_blocks * block_size * block_size * value_bytes.get(prec[0], 8)
              + 2 * n * 8 + (bj.num_blocks + 1) * 4 + bj.num_blocks)
    apply_a_ms = _graph_ms(lambda: ba.apply(b, x), stream)
    return {"workload": "poisson3d_7pt_128", "max_block_size": block_size,
            "num_blocks": bj.num_blocks, "generate_ms": round(gen_ms, 3),
            "apply_ms": round(apply_ms, 4),
            "apply_gbs": round(nbytes / (apply_ms * 1e-3) / 1e9, 1),
            "apply_frac_of_measured": round(nbytes / (apply_ms * 1e-3) / 1e9 / peak, 3),
            "adaptive": {"precisions": prec, "generate_ms": round(gen_a_ms, 3),
                         "apply_ms": round(apply_a_ms, 4),
                         "apply_gbs": round(abytes / (apply_a_ms * 1e-3) / 1e9, 1),
                         "apply_frac_of_measured":
                             round(abytes / (apply_a_ms * 1e-3) / 1e9 / peak, 3)},
            "timing": "apply: CUDA-graph replays of one apply call"}


def _graph_ms(fn, stream, reps=20):
    """Device time of fn (one library call) per replay of a CUDA graph that
    holds it, after a warm-up call outside the capture (first-use set-up)."""
    import torch
    fn()
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        fn()
    for _ in range(3):
        g.replay()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        g.replay()
    e1.record(stream)
    torch.cuda.synchronize()
    del g
    return e0.elapsed_time(e1) / reps


def _event_ms(fn, stream, reps=3):
    """Median CUDA-event time of fn() over reps runs after one warm-up."""
    import torch
    fn()
    times = []
    for _ in range(reps):
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        times.append(e0.elapsed_time(e1))
    return float(np.median(times))


def cg_section(exe, stream, grid=256):
    """The reference's CPU-runnable case on the GPU: CG + scalar Jacobi on
    the 2D 5-point Poisson matrix (256^2), b = A x_true with x_true ~
    U[-1, 1] drawn as the reference run drew it (mt19937(1234)), to a
    relative residual of 1e-10 or 1000 iterations.  The reference executors
    take 710 iterations to 9.777e-11 on this system."""
    import torch
    from ginkgo_b200 import stencils
    from ginkgo_b200.matrix import Csr
    from ginkgo_b200.solver import Cg, Iteration, Jacobi, ResidualNorm
    rp, ci, v = stencils.poisson_2d_5pt(grid)
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    xt = torch.from_numpy(stencils.std_uniform(1234, n, -1.0, 1.0)).cuda()
    b = torch.empty_like(xt)
    A.apply(xt, b)
    s = (Cg.build().with_criteria(Iteration.build().with_max_iters(1000),
                                  ResidualNorm.build().with_reduction_factor(1e-10))
         .with_preconditioner(Jacobi.build().with_max_block_size(1)).on(exe).generate(A))
    x = torch.zeros_like(b)
    ms = _event_ms(lambda: (x.zero_(), s.apply(b, x)), stream)
    r = b.clone()
    A.apply(-1.0, x, 1.0, r)
    return {"workload": f"poisson2d_5pt_{grid}", "n": n, "nnz": len(ci), "ms": round(ms, 3),
            "iterations": s.logger.num_iterations,
            "explicit_rel_residual": float(r.norm() / b.norm()),
            "reference_iterations": 710}


def krylov_iteration_section(exe, stream, iters=40):
    """Time per iteration of the fused CG and BiCGStab (scalar Jacobi, one
    right-hand side) on the 3D 7-point 128^3 matrix: `iters` iterations with
    the residual goal out of reach (reduction 1e-30), median of 3 solves,
    set-up included, divided by the iteration count."""
    import torch
    from ginkgo_b200.matrix import Csr
    from ginkgo_b200.solver import Bicgstab, Cg, Iteration, Jacobi, ResidualNorm
    rp, ci, v = build_matrix()
    n = len(rp) - 1
    A = Csr.read(exe, rp, ci, v)
    b = torch.from_numpy(np.random.default_rng(SEED).standard_normal(n)).cuda()
    out = {"workload": "poisson3d_7pt_128", "n": n, "iterations": iters}
    for name, f in (("cg", Cg), ("bicgstab", Bicgstab)):
        s = (f.build().with_criteria(Iteration.build().with_max_iters(iters),
                                     ResidualNorm.build().with_reduction_factor(1e-30))
             .with_preconditioner(Jacobi.build().with_max_block_size(1)).on(exe).generate(A))
        x = torch.zeros_like(b)
        ms = _event_ms(lambda: (x.zero_(), s.apply(b, x)), stream)
        out[name] = {"ms": round(ms, 3), "us_per_iteration": round(ms * 1e3 / iters, 1),
                     "iterations": s.logger.num_iterations}
    return out


def batch_section(exe, stream, num_systems=8192, seed=3):
    """Batched BiCGStab + scalar Jacobi over 8192 convection-diffusion
    systems of n ~ U[32, 1024] rows (batch Ell, ragged), relative tolerance
    1e-8, at most 500 iterations; the autotuner runs once (untimed) and the
    timed solves reuse its table.  Reported per precision: median solve time
    of 3, systems per second, iterations, the largest logged relative
    residual and the fraction of systems that converged."""
    import torch
    from ginkgo_b200.batch import BatchBicgstab, convection_diffusion_batch
    out = {"workload": f"convection_diffusion_batch_{num_systems}", "tol": 1e-8,
           "max_iters": 500}
    for dt, name in ((torch.float64, "f64"), (torch.float32, "f32")):
        A, _ = convection_diffusion_batch(exe, num_systems, lo=32, hi=1024, seed=seed,
                                          dtype=dt)
        b = torch.from_numpy(np.random.default_rng(seed).standard_normal(A.total_rows)).to(dt).cuda()
        s = (BatchBicgstab.build().with_max_iterations(500).with_tolerance(1e-8)
             .with_tolerance_type("relative").with_preconditioner("jacobi")
             .on(exe).generate(A))
        x = torch.zeros_like(b)
        table = s.tune(b, x)
        ms = _event_ms(lambda: (x.zero_(), s.apply(b, x)), stream)
        it = s.logger.iterations.double()
        bn = torch.zeros(A.num_systems, dtype=torch.float64, device=b.device)
        seg = torch.repeat_interleave(torch.arange(A.num_systems, device=b.device),
                                      torch.from_numpy(np.diff(A.host_row_offsets)).cuda())
        bn.index_add_(0, seg, b.double() ** 2)
        rel = s.logger.residual_norms / bn.sqrt()
        vb = 8 if dt == torch.float64 else 4
        # two matrix reads per iteration (5 slots per row, value + index)
        mat_bytes = float((it * torch.from_numpy(np.diff(A.host_row_offsets)).cuda()
                           .double()).sum()) * 2 * 5 * (vb + 4)
        buckets = {f"<={1 << k}": {"threads_per_system": int(table[2 * k]),
                                   "vectors_in_smem": bool(table[2 * k + 1])}
                   for k in range(12) if table[2 * k] > 0}
        out[name] = {"ms": round(ms, 3), "systems_per_s": round(A.num_systems / ms * 1e3, 1),
                     "matrix_gbs": round(mat_bytes / (ms * 1e-3) / 1e9, 1),
                     "tuned_buckets": buckets,
                     "total_rows": int(A.total_rows),
                     "mean_iterations": round(float(it.mean()), 1),
                     "max_iterations": int(it.max()),
                     "max_logged_rel_residual": float(rel.max()),
                     "converged_fraction": float((rel <= 1e-8 * 1.0001).double().mean())}
    return out


def autograd_section(exe, stream, nx=64, k=16, seed=5):
    """Differentiable solve x = A(theta)^-1 b on the 64^3 variable-conductivity
    operator (theta ~ lognormal(0, 0.5)), 16 right-hand sides, loss
    sum ||x - x_target||^2: median time of 3 forward solves and of 3
    backward passes (adjoint CG on the GPU transpose + SDDMM)."""
    import torch
    from ginkgo_b200.autograd import ConductivityOperator
    g = torch.Generator(device="cuda").manual_seed(seed)
    op = ConductivityOperator(nx)
    theta = torch.exp(0.5 * torch.randn(op.num_edges, dtype=torch.float64, device="cuda",
                                        generator=g)).requires_grad_(True)
    b = torch.randn(op.n, k, dtype=torch.float64, device="cuda", generator=g)
    xt = torch.randn(op.n, k, dtype=torch.float64, device="cuda", generator=g)
    state = {}

    def fwd():
        state["x"] = op.solve(theta, b, tol=1e-10)

    def bwd():
        theta.grad = None
        loss = ((state["x"] - xt) ** 2).sum()
        loss.backward(retain_graph=True)

    fwd_ms = _event_ms(fwd, stream)
    bwd_ms = _event_ms(bwd, stream)
    return {"workload": f"conductivity_{nx}^3_k{k}", "n": op.n, "nnz": op.nnz,
            "forward_ms": round(fwd_ms, 3), "backward_ms": round(bwd_ms, 3),
            "grad_norm": float(theta.grad.norm())}


def sweep(exe, rp, ci, v, time_op, include_b=True):
    """Every format x precision x k in {1, 4, 16} on matrix A (the 7-point
    128^3 Poisson matrix) and matrix B (power-law, n = 4M, row lengths
    round(lognormal(2.5, 1)) clipped to [1, 4096], seed 0).  gbs counts the
    bytes of the format as stored (padding included), useful_gbs the Csr
    bytes of the same product; Ell on B is not built (its padding would
    need n * max_row slots)."""
    import torch
    from ginkgo_b200 import stencils
    from ginkgo_b200.matrix import Csr
    peak, _ = measured_peaks()
    out = {}
    mats = [("A", rp, ci, v)]
    if include_b:
        mats.append(("B",) + stencils.power_law(4_000_000, seed=0, mu=2.5, sigma=1.0,
                                                max_len=4096))
    rng = np.random.default_rng(1)
    for mname, mrp, mci, mv in mats:
        n, nnz = len(mrp) - 1, len(mci)
        out[f"{mname}_shape"] = {"n": n, "nnz": nnz}
        for dt, vb in ((torch.float64, 8), (torch.float32, 4)):
            A = Csr.read(exe, mrp, mci, mv, dtype=dt)
            ops = [("csr_classical", None), ("csr_load_balance", None)]
            width = A.max_row_nnz
            if mname == "A":
                ops.append(("ell", A.convert_to_ell()))
            else:
                out[f"{mname}_ell_{'f64' if vb == 8 else 'f32'}"] = {
                    "not_applicable": f"storage: {n} x {width} slots = "
                                      f"{n * width * (vb + 4) / 1e9:.0f} GB"}
            S = A.convert_to_sellp(32, 1)
            ops.append(("sellp32", S))
            for k in (1, 4, 16):
                x = torch.from_numpy(rng.standard_normal((n, k))).to(dt).cuda()
                y = torch.empty((n, k), dtype=dt, device="cuda")
                useful = csr_bytes(n, nnz, k, vb)
                for name, op in ops:
                    if name.startswith("csr"):
                        A.set_strategy(name[4:])
                        op, nb = A, useful
                    elif name == "ell":
                        nb = op.width * op.stride * (vb + 4) + k * n * 2 * vb
                    else:
                        nb = (op.num_stored_elements * (vb + 4) +
                              (op.slice_sets.numel() + op.slice_lengths.numel()) * 8 +
                              k * n * 2 * vb)
                    t = time_op(lambda: op.apply(x, y), 20, 3)
                    out[f"{mname}_{name}_{'f64' if vb == 8 else 'f32'}_k{k}"] = {
                        "ms": round(t * 1e3, 5), "gbs": round(nb / t / 1e9, 1),
                        "useful_gbs": round(useful / t / 1e9, 1),
                        "frac_of_measured": round(nb / t / 1e9 / peak, 3)}
                del x, y
            del A, S, ops
            torch.cuda.empty_cache()
    return out


if __name__ == "__main__":
    main()
