"""Benchmark: time to true-residual rtol 1e-8 of plain FP64 GMRES(30) + block-Jacobi
ILU(0) on the 2M-vertex Poisson-disk/Delaunay disk mesh (RCM-ordered, bs 3),
plus the SpMV / ILU-apply kernels' achieved HBM bandwidth.

One step = one complete solve from x0 = 0 with the matrix and the ILU(0)
factors resident in HBM (setup timed separately).  N GPUs run N independent
replicas (the path has no exchange step on one rank's system): every rank
solves its own copy, steps are timed with CUDA events on the library's stream
between barriers, and the slowest rank's time is reported.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

REPO = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(REPO, "owt-krylov_b200")
for _p in (REPO, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "time-to-rtol 1e-8 on B200, learned/mixed vs plain FP64 ILU-GMRES; SpMV HBM GB/s"
WORKLOAD = "plain-fp64-gmres30-ilu0"


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--vertices", type=int, default=2_000_000)
    p.add_argument("--seed", type=int, default=1)
    p.add_argument("--no-cpu-baseline", action="store_true")
    return p.parse_args()


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, index: int):
        self.index = index
        self.proc = None

    def __enter__(self):
        cmd = ["nvidia-smi", f"--id={self.index}",
               "--query-gpu=clocks.sm,clocks.max.sm,clocks_event_reasons.active,"
               "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
               "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
               "--format=csv,noheader,nounits", "-lms", "200"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            out, _ = self.proc.communicate(timeout=10)
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            try:
                sm.append(float(f[0]))
                mx = max(mx, float(f[1]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, f[3:7]):
                if v.lower() == "active":
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx or None,
                "reasons": sorted(reasons), "samples": len(sm)}


def build_system(n_vertices: int, seed: int):
    from owtk_b200 import problems

    t = time.time()
    s = problems.config1(n_vertices, seed=seed)
    return s, time.time() - t


def algorithmic_bytes(s, ilu_entries: int):
    n, bs, nnz = s.owned, s.bs, s.nnz
    spmv = nnz * (bs * 8 + 4) + (n + 1) * 4 + 2 * n * bs * 8
    # Forward + backward ILU sweep: factor values + columns once, row offsets
    # and diagonal positions, inverse diagonal, input read, output written and
    # re-read by the backward sweep.
    ilu = ilu_entries * (bs * 8 + 4) + 2 * (n + 1) * 4 + n * 4 + n * bs * 8 + 3 * n * bs * 8
    return spmv, ilu


def cpu_reference_solve(s, reps: int, native_build: bool = False):
    """The reference's own CPU GMRES(30)+ILU(0) (oracle/_ref), one host thread."""
    import oracle

    try:
        ref = oracle.Reference(native=native_build)
        kind = "reference"
    except FileNotFoundError:
        return None
    m = ref.matrix("bsr", s.owned, 0, s.bs, s.rowptr, s.cols, s.vals)
    t = time.time()
    pc = ref.pc("ilu", m, 0)
    setup = time.time() - t
    opts = oracle.default_options(restart=30)
    times, last = [], None
    for _ in range(reps):
        t = time.time()
        r, x = ref.solve("gmres", m, pc, opts, s.rhs, np.zeros(s.owned * s.bs))
        times.append(time.time() - t)
        last = r
    return {"kind": kind, "seconds": times, "setup_seconds": setup, "iterations": int(last.iterations),
            "status": int(last.status), "true_residual": float(last.true_residual_norm)}


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    s, gen = build_system(args.vertices, args.seed)
    res = cpu_reference_solve(s, args.warmup + args.steps)
    if res is None:
        print(json.dumps({"impl": "reference", "unavailable": "reference harness oracle/_ref not built"}))
        return 0
    timed = res["seconds"][args.warmup:]
    v = statistics.mean(timed)
    line = {
        "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "vertices": s.owned, "entries": s.nnz, "block_size": s.bs,
                   "solver": "gmres(30)+ilu(0)", "rtol": 1e-8, "ordering": "rcm"},
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": res["kind"],
                         "sample": f"full solve of the {s.owned}-vertex system, {res['iterations']} iterations, "
                                   "one thread (the reference is single-threaded)"},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "reference_iterations": res["iterations"], "reference_setup_s": res["setup_seconds"],
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    from owtk_b200 import native

    s, gen_s = build_system(args.vertices, args.seed + 0)   # replicas share the system
    n, bs = s.owned, s.bs
    ctx = native.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    t = time.time()
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    ctx.synchronize()
    setup_s = time.time() - t
    opts = native.default_options(restart=30, relative_tolerance=1e-8)
    ws = native.Workspace(ctx)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    x = native.Vector(ctx, n, 0, bs)

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(local)
        ctx.synchronize()

    def step():
        x.fill(0.0)
        r = native.solve(native.FGMRES, m, pc, b, x, opts, ws)
        if r.status != 0:
            raise RuntimeError(f"solve did not converge: {r.as_dict()}")
        return r

    for _ in range(args.warmup):
        last = step()
    barrier()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0 = ctx.kernel_launches
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            last = step()
        e1.record(stream)
        e1.synchronize()
    barrier()
    launches = ctx.kernel_launches - launches0
    ms = e0.elapsed_time(e1) / args.steps
    if world > 1:
        tt = torch.tensor([ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        ms = float(tt.item())

    # End to end through the reference-facing host-buffer call: pinned rhs/x
    # copied in, solved, x copied back, every step.
    hb = torch.from_numpy(s.rhs.astype(np.float64)).pin_memory()
    hx = torch.zeros(n * bs, dtype=torch.float64).pin_memory()
    for _ in range(1):
        hx.zero_()
        native.solve_host(native.FGMRES, m, pc, hb.data_ptr(), hx.data_ptr(), opts, ws)
    barrier()
    e2, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e2.record(stream)
    for _ in range(args.steps):
        hx.zero_()
        r = native.solve_host(native.FGMRES, m, pc, hb.data_ptr(), hx.data_ptr(), opts, ws)
        assert r.status == 0
    e3.record(stream)
    e3.synchronize()
    e2e_ms = e2.elapsed_time(e3) / args.steps
    if world > 1:
        tt = torch.tensor([e2e_ms], device=f"cuda:{local}")
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(tt.item())

    # Kernel rooflines, live: average launch time of the dominant kernel (the
    # ILU(0) forward+backward sweep pair) and of the SpMV, CUDA events on the
    # library's stream.  The matrix (336 MB) exceeds L2, so each launch streams
    # it from HBM.
    ilu_entries = int(pc.ilu_factors()[1].size)
    spmv_bytes, ilu_bytes = algorithmic_bytes(s, ilu_entries)
    y = native.Vector(ctx, n, 0, bs)

    def time_op(fn, reps):
        fn()
        ctx.synchronize()
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        c.record(stream)
        c.synchronize()
        return a.elapsed_time(c) / reps

    spmv_ms = time_op(lambda: m.apply(b, y), 50)
    ilu_ms = time_op(lambda: pc.apply(b, y), 10)
    peak, peak_kind = measured_peaks()
    clocks = clk.summary()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_reference_solve(s, 1)
    if rank == 0:
        line = {
            "metric": METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "vertices": n, "entries": s.nnz, "block_size": bs,
                       "solver": "gmres(30)+ilu(0)", "rtol": 1e-8, "ordering": "rcm", "parallelism": f"replicas{world}",
                       "l2": "inputs larger than L2 (matrix 336 MB, Krylov basis 2.9 GB)",
                       "iterations": int(last.iterations), "setup_s": setup_s, "mesh_gen_s": gen_s},
            "e2e": {"value": e2e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": 2 * n * bs * 8,
                    "d2h_bytes_per_step": n * bs * 8},
            "roofline": {"bound": "hbm", "kernel": "ilu0 forward+backward sweep", "achieved": ilu_bytes / (ilu_ms * 1e-3) / 1e9,
                         "peak": peak, "unit": "GB/s", "frac": ilu_bytes / (ilu_ms * 1e-3) / 1e9 / peak,
                         "traffic": None, "bytes_per_launch": ilu_bytes, "ms_per_launch": ilu_ms,
                         "peak_source": peak_kind},
            "spmv": {"achieved": spmv_bytes / (spmv_ms * 1e-3) / 1e9, "unit": "GB/s",
                     "frac": spmv_bytes / (spmv_ms * 1e-3) / 1e9 / peak, "us_per_launch": spmv_ms * 1e3,
                     "bytes_per_launch": spmv_bytes},
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["seconds"][0], "unit": "s", "cores": 1, "kind": cpu["kind"],
                                    "sample": f"one full reference solve of the same system "
                                              f"({cpu['iterations']} iterations, ILU setup {cpu['setup_seconds']:.2f} s excluded)"}
        print(json.dumps(line))
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
