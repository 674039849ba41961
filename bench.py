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

# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per vertex from one
# ncu capture on the 1M-vertex disk mesh (profiles/ilu0_sweeps_fp64_1m_vertices.md,
# profiles/spmv_bulk_bsr3_fp64_1m_vertices.md); traffic grows with the vertex
# count, so the benchmark's per-launch traffic is this times its vertices.
PROFILED_TRAFFIC_PER_VERTEX = {"ilu0 sweep pair": (255.98e6 + 20.01e6 + 279.70e6 + 21.33e6) / 999_573,
                               "spmv": (224.46e6 + 5.60e6) / 999_573}
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
    p.add_argument("--kernels", action="store_true",
                   help="standalone kernel throughput sweep (one JSON line per kernel) instead of the solve")
    p.add_argument("--bs", default="3", help="block sizes of the kernel sweep, comma separated")
    p.add_argument("--orders", default="rcm", help="vertex orders of the kernel sweep: rcm,hilbert")
    p.add_argument("--only", default="", help="kernel sweep: comma-separated subset of "
                   "spmv,split,spmv32,dense,dense32,ilu,ssor,dot,norm,axpy,gnn (default) and fgmres_learned")
    p.add_argument("--reps", type=int, default=20, help="kernel sweep: timed launches per kernel")
    p.add_argument("--form", choices=["plain", "mixed", "batching", "learned"], default="plain",
                   help="plain: the FP64 GMRES(30)+ILU(0) headline; mixed / batching / learned: the three "
                        "other forms, one JSON line each")
    p.add_argument("--systems", type=int, default=256, help="batching: number of systems")
    p.add_argument("--draws", type=int, default=32, help="learned: coefficient draws of the training mesh")
    p.add_argument("--train-vertices", type=int, default=200_000, help="learned: training mesh size")
    p.add_argument("--epochs", type=int, default=20, help="learned: passes over the training pairs (rate 3e-3 decaying to 3e-4)")
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
               "--format=csv,noheader,nounits", "-lms", "50"]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            time.sleep(0.5)   # the sampler is running before the timed region starts
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
    return kernel_bytes("spmv", n, bs, nnz), kernel_bytes("ilu", n, bs, nnz, factor_entries=ilu_entries)


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
                         "traffic": PROFILED_TRAFFIC_PER_VERTEX["ilu0 sweep pair"] * n,
                         "traffic_source": "ncu DRAM bytes per vertex on the 1M-vertex mesh, scaled to this mesh",
                         "bytes_per_launch": ilu_bytes, "ms_per_launch": ilu_ms, "peak_source": peak_kind},
            "spmv": {"achieved": spmv_bytes / (spmv_ms * 1e-3) / 1e9, "unit": "GB/s",
                     "frac": spmv_bytes / (spmv_ms * 1e-3) / 1e9 / peak, "us_per_launch": spmv_ms * 1e3,
                     "bytes_per_launch": spmv_bytes, "traffic": PROFILED_TRAFFIC_PER_VERTEX["spmv"] * n},
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


def kernel_bytes(kind: str, n: int, bs: int, nnz: int, sv: int = 8, factor_entries: int = 0, k: int = 16,
                 off_entries: int = 0) -> int:
    """Algorithmic HBM bytes of one launch (values, 32-bit indices, vectors
    each read or written once)."""
    vec = n * bs * sv
    if kind in ("spmv", "spmv32"):
        return nnz * (bs * sv + 4) + (n + 1) * 4 + 2 * vec
    if kind in ("dense", "dense32"):
        return nnz * (bs * bs * sv + 4) + (n + 1) * 4 + 2 * vec
    if kind == "split":
        return vec + off_entries * (bs * sv + 4) + (n + 1) * 4 + 2 * vec
    if kind == "ilu":
        return algorithmic_bytes_ilu(n, bs, factor_entries)
    if kind == "ssor":
        return 2 * (nnz * (bs * sv + 4) + (n + 1) * 4) + 3 * vec
    if kind == "dot":
        return (k + 1) * vec
    if kind == "norm":
        return vec
    if kind == "axpy":
        return 3 * vec
    raise ValueError(kind)


def algorithmic_bytes_ilu(n: int, bs: int, factor_entries: int) -> int:
    # Forward + backward ILU sweep: factor values + columns once, row offsets
    # and diagonal positions, inverse diagonal, input read, output written and
    # re-read by the backward sweep.
    return factor_entries * (bs * 8 + 4) + 2 * (n + 1) * 4 + n * 4 + n * bs * 8 + 3 * n * bs * 8


def run_kernels(args):
    """Standalone throughput sweep of the hot kernels on the Poisson-disk /
    Delaunay disk mesh: each kernel launched `--reps` times back to back on the
    library's stream and timed with CUDA events; the matrices exceed L2, so
    every launch streams them from HBM.  One JSON line per (order, bs, kernel)."""
    import torch
    from owtk_b200 import native, problems

    peak, peak_kind = measured_peaks()
    only = set(filter(None, args.only.split(","))) or {"spmv", "split", "spmv32", "dense", "dense32", "ilu", "ssor",
                                                        "dot", "norm", "axpy", "gnn"}
    t = time.time()
    xy, edges = problems.disk_mesh(args.vertices, args.seed)
    gen_s = time.time() - t
    ctx = native.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))

    def timed(fn, reps):
        fn()
        ctx.synchronize()
        a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        c.record(stream)
        c.synchronize()
        return a.elapsed_time(c) / reps * 1e3   # microseconds per launch

    for order in args.orders.split(","):
        for bs in [int(b) for b in args.bs.split(",")]:
            s = problems.component_diagonal_system(xy, edges, bs, np.random.default_rng(args.seed), order=order)
            n, nnz = s.owned, s.nnz
            m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
            x = native.Vector(ctx, n, 0, bs).upload(s.rhs)
            y = native.Vector(ctx, n, 0, bs)
            results = []

            def emit(kind, us, nbytes, **extra):
                gbs = nbytes / (us * 1e-6) / 1e9
                line = {"kernel": kind, "order": order, "block_size": bs, "vertices": n, "entries": nnz,
                        "us_per_launch": round(us, 2), "bytes_per_launch": int(nbytes), "achieved_gbs": round(gbs, 1),
                        "peak_gbs": peak, "frac": round(gbs / peak, 4), "peak_source": peak_kind,
                        "reps": args.reps, "mesh_gen_s": round(gen_s, 1)}
                line.update(extra)
                results.append(line)
                print(json.dumps(line), flush=True)

            if "spmv" in only:
                emit("spmv", timed(lambda: m.apply(x, y), args.reps), kernel_bytes("spmv", n, bs, nnz))
            if "split" in only:
                orp, oci, diag, off = s.split()
                d = native.Vector(ctx, n, 0, bs).upload(diag)
                o = native.Vector(ctx, max(off.size // bs, 1), 0, bs).upload(off)
                sm = native.Matrix(ctx, "split", n, 0, bs, orp, oci, diag_ptr=d.data_ptr, off_ptr=o.data_ptr)
                emit("split", timed(lambda: sm.apply(x, y), args.reps),
                     kernel_bytes("split", n, bs, nnz, off_entries=int(orp[-1])))
            if "spmv32" in only:
                m32 = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals, dtype=np.float32)
                x32 = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(s.rhs)
                y32 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
                emit("spmv32", timed(lambda: m32.apply(x32, y32), args.reps), kernel_bytes("spmv32", n, bs, nnz, sv=4))
            if ("dense" in only or "dense32" in only) and bs <= 4:
                # Dense bs x bs blocks on the same mesh (the precision form's
                # matrix): FP64, and FP32 as its inner SpMV.
                sd = problems.dense_block_system(xy, edges, bs, np.random.default_rng(args.seed), order=order)
                if "dense" in only:
                    md = native.Matrix(ctx, "dense", n, 0, bs, sd.rowptr, sd.cols, sd.vals)
                    xd = native.Vector(ctx, n, 0, bs).upload(sd.rhs)
                    emit("dense", timed(lambda: md.apply(xd, y), args.reps), kernel_bytes("dense", n, bs, sd.nnz))
                    del md
                if "dense32" in only:
                    md32 = native.Matrix(ctx, "dense", n, 0, bs, sd.rowptr, sd.cols, sd.vals, dtype=np.float32)
                    xd32 = native.Vector(ctx, n, 0, bs, dtype=np.float32).upload(sd.rhs)
                    yd32 = native.Vector(ctx, n, 0, bs, dtype=np.float32)
                    emit("dense32", timed(lambda: md32.apply(xd32, yd32), args.reps),
                         kernel_bytes("dense32", n, bs, sd.nnz, sv=4))
                    del md32
            if "ilu" in only:
                pc = native.Preconditioner(m, native.PC_ILU, 0)
                fe = int(pc.ilu_factors()[1].size)
                _, _, depth_lower, depth_upper = pc.levels()
                emit("ilu", timed(lambda: pc.apply(x, y), max(2, args.reps // 4)),
                     kernel_bytes("ilu", n, bs, nnz, factor_entries=fe),
                     lower_levels=int(depth_lower), upper_levels=int(depth_upper))
            if "ssor" in only:
                ps = native.Preconditioner(m, native.PC_SSOR, 1.0)
                emit("ssor", timed(lambda: ps.apply(x, y), max(2, args.reps // 4)), kernel_bytes("ssor", n, bs, nnz))
            if "dot" in only:
                basis = [native.Vector(ctx, n, 0, bs).upload(s.rhs) for _ in range(16)]
                emit("dot", timed(lambda: native.dot_batch(x, basis), args.reps), kernel_bytes("dot", n, bs, nnz, k=16),
                     note="16 dot products against one vector, result read on the host")
            if "norm" in only:
                emit("norm", timed(lambda: native.norm(x), args.reps), kernel_bytes("norm", n, bs, nnz),
                     note="one-pass scaled norm, result read on the host")
            if "axpy" in only:
                emit("axpy", timed(lambda: native.axpy(0.5, x, y), args.reps), kernel_bytes("axpy", n, bs, nnz))
            if "gnn" in only and bs <= 8:
                # One application of the learned preconditioner: q = r/d with
                # both norms, the encoder, three layers, the last layer with
                # the decoder fused.  Algorithmic bytes per vertex: FP64 r
                # twice, FP32 1/d, q written and read twice; BF16 features
                # (128 B) written by the encoder and layers 1-3, read by layers
                # 1-4; each layer's 8-slot neighbour list (32-bit column and
                # BF16 weight per slot, 48 B); FP64 output.
                net = native.Learned(m, seed=1)
                per_vertex = (2 * bs * 8 + bs * 4 + 3 * bs * 4 + 4 * 128 + 4 * 128 + 4 * 48 + bs * 8)
                flops = 4 * 2 * 2 * 64 * 64 * n
                us = timed(lambda: net.apply(x, y), max(2, args.reps // 2))
                emit("gnn", us, per_vertex * n, tensor_tflops=round(flops / (us * 1e-6) / 1e12, 2),
                     note="one learned-preconditioner application (65 kFLOP on the tensor cores vs ~1.3 kB per vertex)")
            if "fgmres_learned" in only and bs <= 8:
                # One FGMRES solve with the (untrained) network and the ILU(0)
                # fallback, 14 iterations fixed: the per-iteration mix of
                # network, SpMV, residual check and Gram-Schmidt kernels.
                ilu = native.Preconditioner(m, native.PC_ILU, 0)
                pcl = native.LearnedPreconditioner(native.Learned(m, seed=1), ilu)
                xs = native.Vector(ctx, n, 0, bs)
                ws = native.Workspace(ctx)
                opts = native.default_options(relative_tolerance=0.0, maximum_iterations=14, restart=30)

                def solve():
                    xs.fill(0.0)
                    native.solve(native.FGMRES, m, pcl, x, xs, opts, ws)

                us = timed(solve, 1)
                emit("fgmres_learned", us, 0, iterations=14, fallbacks=pcl.counts()[1],
                     note="one learned-preconditioned FGMRES solve, 14 iterations")
            ctx.synchronize()
    return 0

# ---------------------------------------------------------------- other forms
def _event_time(stream, fn, steps):
    import torch

    a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    c.record(stream)
    c.synchronize()
    return a.elapsed_time(c) / steps


def _line(args, workload, value_s, e2e_s, cfg, dtype, extra):
    line = {"metric": METRIC, "value": value_s, "unit": "s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": value_s * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": dict({"workload": workload}, **cfg)}
    if e2e_s is not None:
        line["e2e"] = e2e_s
    line.update(extra)
    return line


def run_batching(args):
    """256 uneven systems (log-uniform 5k-200k vertices, aspect U(1,4), bs in
    {1,2,3,4}) by BiCGSTAB + Jacobi to rtol 1e-8 in one persistent,
    graph-captured launch after the autotuner picked the launch shape."""
    import torch
    from owtk_b200 import native, problems

    t = time.time()
    systems = problems.batch_systems(count=args.systems, seed=3)
    gen_s = time.time() - t
    ctx = native.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    t = time.time()
    batch = native.Batch(ctx, systems)
    create_s = time.time() - t
    t = time.time()
    bps, vpw = batch.autotune()
    tune_s = time.time() - t
    rhs = np.concatenate([y.rhs for y in systems])
    rv = native.Vector(ctx, rhs.size, 0, 1).upload(rhs)
    xv = native.Vector(ctx, rhs.size, 0, 1)
    opts = native.default_options()
    res = None

    def step():
        nonlocal res
        xv.fill(0.0)
        res = batch.solve(rv, xv, opts)

    for _ in range(args.warmup):
        step()
    launches0 = ctx.kernel_launches
    with Clocks(0) as clk:
        ms = _event_time(stream, step, args.steps)
    launches = (ctx.kernel_launches - launches0) // args.steps
    status = [r.status for r in res]
    its = np.array([r.iterations for r in res])
    # e2e: pinned host rhs / x copied in and x copied out inside the call.
    hb = torch.from_numpy(rhs).pin_memory()
    hx = torch.zeros(rhs.size, dtype=torch.float64).pin_memory()

    def host_step():
        hx.zero_()
        batch.solve_host(hb.data_ptr(), hx.data_ptr(), opts)

    host_step()
    e2e_ms = _event_time(stream, host_step, args.steps)
    # Algorithmic bytes: per iteration two SpMV passes and ~21 vector passes
    # (element-wise phases and the fused dot operands); setup SpMV + 3 passes.
    total = 0
    for y, k in zip(systems, its):
        n, bs, nnz = y.owned, y.bs, y.nnz
        spmv = nnz * (bs * 8 + 4) + (n + 1) * 4 + 2 * n * bs * 8
        total += int(k) * (2 * spmv + 21 * n * bs * 8) + spmv + 3 * n * bs * 8
    peak, peak_kind = measured_peaks()
    achieved = total / (ms * 1e-3) / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        cpu = _cpu_batch_sample(systems, its)
    extra = {"e2e": {"value": e2e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": 2 * rhs.size * 8,
                     "d2h_bytes_per_step": rhs.size * 8},
             "roofline": {"bound": "hbm", "kernel": "k_batch_bicgstab (whole persistent launch)", "achieved": achieved,
                          "peak": peak, "unit": "GB/s", "frac": achieved / peak, "traffic": None,
                          "bytes_per_launch": total, "ms_per_launch": ms, "peak_source": peak_kind},
             "batch": {"systems": len(systems), "vertices": int(sum(y.owned for y in systems)),
                       "unknowns": int(rhs.size), "entries": int(sum(y.nnz for y in systems)),
                       "converged": int(sum(1 for v in status if v == 0)), "iterations_min": int(its.min()),
                       "iterations_max": int(its.max()), "iterations_mean": float(its.mean()),
                       "blocks_per_sm": bps, "vertices_per_warp": {str(b): vpw[b] for b in (1, 2, 3, 4)},
                       "generate_s": gen_s, "create_s": create_s, "autotune_s": tune_s,
                       "graph_captures_launches": list(batch.graph_counts())},
             "gpu_launches": int(launches), "clocks": clk.summary()}
    if cpu is not None:
        extra["cpu_baseline"] = cpu
    print(json.dumps(_line(args, "batch-256-bicgstab-jacobi", ms / 1e3, None,
                           {"systems": len(systems), "solver": "bicgstab+jacobi", "rtol": 1e-8,
                            "l2": "inputs larger than L2 (matrices 2.8 GB)"}, "f64", extra)))
    return 0


def _cpu_batch_sample(systems, its, budget_s: float = 20.0):
    """The reference's bicgstab + Jacobi (oracle/_ref, one thread) on the first
    systems until ~budget_s, extrapolated to the whole batch by
    sum(unknowns x iterations)."""
    import oracle

    try:
        ref = oracle.Reference()
    except FileNotFoundError:
        return None
    spent, work_done, done = 0.0, 0, 0
    for y, k in zip(systems, its):
        m = ref.matrix("bsr", y.owned, 0, y.bs, y.rowptr, y.cols, y.vals)
        pc = ref.pc("jacobi", m, 0.0)
        t = time.time()
        r, _ = ref.solve("bicgstab", m, pc, oracle.default_options(), y.rhs, np.zeros(y.owned * y.bs))
        spent += time.time() - t
        work_done += y.owned * y.bs * int(r.iterations)
        done += 1
        if spent >= budget_s:
            break
    total_work = sum(y.owned * y.bs * int(k) for y, k in zip(systems, its))
    value = spent * total_work / max(work_done, 1)
    return {"value": value, "unit": "s", "cores": 1, "kind": "reference",
            "sample": f"reference bicgstab+jacobi on the first {done} of {len(systems)} systems ({spent:.1f} s), "
                      f"scaled by unknowns x iterations to the whole batch"}


def run_mixed(args):
    """Dense 3x3 blocks on the 2M-vertex disk mesh: FP64 FGMRES(30) outer
    refinement to rtol 1e-10 around block-ILU(0) factors stored in FP32 and in
    BF16 with an FP32 inner solve, against the plain FP64 block-ILU(0) FGMRES;
    errors against the FP64 solution."""
    import torch
    from owtk_b200 import native, problems

    t = time.time()
    s = problems.config2(args.vertices)
    gen_s = time.time() - t
    n, bs = s.owned, s.bs
    ctx = native.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    m = native.Matrix(ctx, "dense", n, 0, bs, s.rowptr, s.cols, s.vals)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    opts = native.default_options(relative_tolerance=1e-10, restart=30)
    out = {}
    xref = None
    for name, storage, inner in (("fp64", native.F64, None), ("fp32", native.F32, 4), ("bf16", native.BF16, 4)):
        t = time.time()
        pc = native.Preconditioner(m, native.PC_BLOCK_ILU, 0, storage=storage, mixed_inner=inner)
        ctx.synchronize()
        setup_s = time.time() - t
        x = native.Vector(ctx, n, 0, bs)
        ws = native.Workspace(ctx)
        res = None

        def step():
            nonlocal res
            x.fill(0.0)
            res = native.solve(native.FGMRES, m, pc, b, x, opts, ws)

        for _ in range(args.warmup):
            step()
        ms = _event_time(stream, step, args.steps)
        xs = x.download()
        if xref is None:
            xref = xs
        out[name] = {"ms": ms, "iterations": int(res.iterations), "status": int(res.status),
                     "true_relative_residual": float(res.true_residual_norm / np.linalg.norm(s.rhs)),
                     "error_vs_fp64": float(np.linalg.norm(xs - xref) / np.linalg.norm(xref)), "setup_s": setup_s}
    best = min(out["fp32"]["ms"], out["bf16"]["ms"])
    extra = {"mixed": out, "speedup_vs_fp64": out["fp64"]["ms"] / best}
    print(json.dumps(_line(args, "mixed-dense3x3-fgmres-blockilu0", best / 1e3, None,
                           {"vertices": n, "entries": s.nnz, "block_size": bs, "rtol": 1e-10,
                            "solver": "fgmres(30) fp64 outer, block-ilu(0) fp32/bf16 factors, fp32 inner",
                            "mesh_gen_s": gen_s}, "f64+f32", extra)))
    return 0


def run_learned(args):
    """Anisotropic unit-square mesh (--vertices, default 8M): the network is
    trained on the GPU on ILU(0)-GMRES residual/error pairs of --draws
    coefficient draws of a --train-vertices mesh, then FGMRES(30) with the
    network (ILU(0) fallback; FP64 outer, BF16/FP32 network) is timed against
    plain FP64 ILU(0)-GMRES(30) on the same system, both to rtol 1e-8."""
    import torch
    from owtk_b200 import learned, native, problems

    ctx = native.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    # Training.
    t = time.time()
    train = [sys_ for _, sys_ in problems.anisotropic_draws(args.train_vertices, 41, range(args.draws))]
    gen_train_s = time.time() - t
    m0 = native.Matrix(ctx, "bsr", train[0].owned, 0, 3, train[0].rowptr, train[0].cols, train[0].vals)
    net = native.Learned(m0, seed=1)
    t = time.time()
    hist = learned.train(ctx, net, train, epochs=args.epochs, learning_rate=3e-3, pairs_per_system=6,
                         final_learning_rate=3e-4)
    train_s = time.time() - t
    weights = net.parameters()
    # The large system.
    t = time.time()
    s = problems.config4(args.vertices)
    gen_s = time.time() - t
    n, bs = s.owned, s.bs
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    t = time.time()
    ilu = native.Preconditioner(m, native.PC_ILU, 0)
    ctx.synchronize()
    ilu_setup_s = time.time() - t
    netL = native.Learned(m, seed=1)
    netL.set_parameters(weights)
    pcl = native.LearnedPreconditioner(netL, ilu)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    x = native.Vector(ctx, n, 0, bs)
    ws = native.Workspace(ctx)
    opts = native.default_options(relative_tolerance=1e-8, restart=30)
    results = {}
    for name, pc in (("ilu0_gmres_fp64", ilu), ("learned_fgmres", pcl)):
        res = None

        def step():
            nonlocal res
            x.fill(0.0)
            res = native.solve(native.FGMRES, m, pc, b, x, opts, ws)

        step()
        ms = _event_time(stream, step, max(1, args.steps))
        results[name] = {"ms": ms, "iterations": int(res.iterations), "status": int(res.status),
                         "true_relative_residual": float(res.true_residual_norm / np.linalg.norm(s.rhs))}
    apps, falls = pcl.counts()
    results["learned_fgmres"]["network_applications"] = apps
    results["learned_fgmres"]["fallbacks"] = falls
    speed = results["ilu0_gmres_fp64"]["ms"] / results["learned_fgmres"]["ms"]
    extra = {"learned": results, "speedup_vs_plain_fp64_ilu_gmres": speed,
             "training": {"draws": args.draws, "vertices": train[0].owned, "epochs": args.epochs,
                          "loss_history": hist, "train_s": train_s, "generate_s": gen_train_s},
             "setup": {"mesh_gen_s": gen_s, "ilu_setup_s": ilu_setup_s}}
    print(json.dumps(_line(args, "learned-anisotropic-fgmres", results["learned_fgmres"]["ms"] / 1e3, None,
                           {"vertices": n, "entries": s.nnz, "block_size": bs, "rtol": 1e-8,
                            "solver": "fgmres(30) + learned network (ilu(0) fallback) vs gmres(30)+ilu(0)"},
                           "f64+bf16", extra)))
    return 0



def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.kernels:
        return run_kernels(args)
    if args.form == "batching":
        return run_batching(args)
    if args.form == "mixed":
        return run_mixed(args)
    if args.form == "learned":
        return run_learned(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
