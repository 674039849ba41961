"""Benchmark: time to true-residual rtol 1e-8 on one B200 of the learned-
preconditioned FGMRES(30) against plain FP64 ILU(0)-GMRES(30), on the
8M-vertex anisotropic Poisson-disk/Delaunay unit-square mesh (RCM, bs 3).

One step = one complete solve from x0 = 0 with the matrix, the ILU(0)
factors and the trained network resident in HBM (setup timed separately).
`value` is the learned solve; the plain FP64 ILU(0)-GMRES(30) solve of the
same system on the same GPU, their ratio, the network's layer roofline and
the 2M-vertex plain workload are extra keys.  N GPUs run N independent
replicas (the path has no exchange step on one rank's system): every rank
solves its own copy, steps are timed with CUDA events on the library's stream
between barriers, and the slowest rank's time is reported.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--form learned|plain|mixed|batching] [--kernels]

--impl reference times the reference's own CPU GMRES(30) + ILU(0)
(oracle/_ref, built from the unmodified reference headers) on the same
system, which that process builds with the reference's own RCM ordering and
without loading this project's library.
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
WEIGHTS = os.path.join(PKG, "weights", "learned_anisotropic_bs3.owtkgnn")
TRAFFIC_FILE = os.path.join(REPO, "profiles", "dram_traffic_per_vertex.txt")
MESH_CACHE = os.path.join(REPO, ".bench_cache")
WORKLOADS = {"learned": "learned-fgmres30-vs-ilu0-gmres30-anisotropic-8m",
             "plain": "plain-fp64-gmres30-ilu0"}


def parse(argv=None):
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", choices=["ours", "reference"], default="ours")
    p.add_argument("--vertices", type=int, default=None,
                   help="mesh size (default: 8M for the learned form, 2M otherwise)")
    p.add_argument("--seed", type=int, default=None, help="mesh seed (default: 4 learned, 1 otherwise)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-plain-2m", action="store_true", help="learned form: skip the 2M-vertex plain keys")
    p.add_argument("--ref-budget", type=float, default=900.0,
                   help="reference arm: seconds of timed full solves at most (the first solve is the warm-up)")
    p.add_argument("--kernels", action="store_true",
                   help="standalone kernel throughput sweep (one JSON line per kernel) instead of the solve")
    p.add_argument("--bs", default="3", help="block sizes of the kernel sweep, comma separated")
    p.add_argument("--orders", default="rcm", help="vertex orders of the kernel sweep: rcm,hilbert")
    p.add_argument("--only", default="", help="kernel sweep: comma-separated subset of "
                   "spmv,split,spmv32,dense,dense32,ilu,ssor,dot,norm,axpy,gnn (default), fgmres_jacobi and fgmres_learned")
    p.add_argument("--reps", type=int, default=20, help="kernel sweep: timed launches per kernel")
    p.add_argument("--form", choices=["learned", "plain", "mixed", "batching"], default="learned",
                   help="learned: the headline (8M anisotropic, learned FGMRES vs plain FP64 ILU(0)-GMRES); "
                        "plain: FP64 GMRES(30)+ILU(0) on the 2M disk mesh; mixed / batching: the other forms")
    p.add_argument("--systems", type=int, default=256, help="batching: number of systems")
    p.add_argument("--jacobi-correction", default="1,0.7",
                   help="learned: STEPS[,OMEGA] damped Jacobi corrections after each accepted network step "
                        "(0: the network alone)")
    p.add_argument("--weights", default=WEIGHTS, help="learned: checkpoint of the trained network")
    a = p.parse_args(argv)
    if a.vertices is None:
        a.vertices = 8_000_000 if a.form == "learned" else 2_000_000
    if a.seed is None:
        a.seed = 4 if a.form == "learned" else 1
    return a


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def measured_peaks():
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def measured_tensor_peak():
    """Dense BF16 TFLOP/s sustained (a kernel timed inside a long solve)."""
    path = os.path.join(REPO, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        if "bf16_tflops_sustained" in d:
            return float(d["bf16_tflops_sustained"]), "measured sustained"
    return 1400.0, "fallback sustained"


def profiled_traffic():
    """DRAM bytes per vertex of each kernel from ncu captures, kept as
    "name: bytes_per_vertex" lines in the profiles' traffic table."""
    out = {}
    if os.path.exists(TRAFFIC_FILE):
        for line in open(TRAFFIC_FILE):
            line = line.split("#", 1)[0].strip()
            if ":" in line:
                k, v = line.rsplit(":", 1)
                out[k.strip()] = float(v)
    return out


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


# ---------------------------------------------------------------- systems
def cached_mesh(n_target: int, seed: int, domain: str):
    """Poisson-disk points and Delaunay edges, kept in .bench_cache/ so the
    second arm run on the same host reuses the first one's mesh."""
    from owtk_b200 import problems

    os.makedirs(MESH_CACHE, exist_ok=True)
    stem = os.path.join(MESH_CACHE, f"{domain}-{n_target}-{seed}")
    try:
        meta = json.load(open(stem + ".json"))
        xy = np.load(stem + "-xy.npy")
        edges = np.load(stem + "-edges.npy")
        if xy.shape == (meta["points"], 2) and edges.shape == (meta["edges"], 2):
            return xy, edges
    except (OSError, ValueError, KeyError):
        pass
    xy, edges = problems.disk_mesh(n_target, seed, domain=domain)
    # Written under a private name and renamed into place, so replicas that
    # build the same mesh at once never leave a torn file for a later reader.
    tag = f".{os.getpid()}.tmp"
    for name, arr in (("-xy.npy", xy), ("-edges.npy", edges)):
        with open(stem + name + tag, "wb") as f:
            np.save(f, arr)
        os.replace(stem + name + tag, stem + name)
    with open(stem + ".json" + tag, "w") as f:
        json.dump({"points": int(xy.shape[0]), "edges": int(edges.shape[0])}, f)
    os.replace(stem + ".json" + tag, stem + ".json")
    return xy, edges


def build_system(form: str, n_vertices: int, seed: int, rcm=None):
    """The workload's system; `rcm` computes the RCM order (default: this
    library's; the reference arm passes the reference's own)."""
    from owtk_b200 import problems

    t = time.time()
    if form == "learned":
        xy, edges = cached_mesh(n_vertices, seed, "square")
        rng = np.random.default_rng([seed, 0])
        s = problems.anisotropic_system(xy, edges, 3, rng, order="rcm", rcm=rcm)
    else:
        xy, edges = cached_mesh(n_vertices, seed, "disk")
        rng = np.random.default_rng(seed)
        s = problems.component_diagonal_system(xy, edges, 3, rng, order="rcm", rcm=rcm)
    return s, time.time() - t


def correction_of(args) -> tuple:
    """--jacobi-correction STEPS[,OMEGA]: damped Jacobi corrections after
    each accepted network step of the learned preconditioner."""
    parts = str(getattr(args, "jacobi_correction", "0")).split(",")
    return int(parts[0]), float(parts[1]) if len(parts) > 1 else 1.0


def workload_config(form: str, s, world: int, correction: tuple = (0, 1.0)) -> dict:
    """The `config` both arms print for one workload (same keys and values)."""
    if form == "learned":
        steps, omega = correction
        net = "learned network" + (f" + {steps} damped jacobi correction(s) (omega {omega:g})" if steps else "")
        return {"workload": WORKLOADS["learned"], "vertices": s.owned, "entries": s.nnz, "block_size": s.bs,
                "mesh": "poisson-disk unit square, delaunay, anisotropic w=1+1e4(e.d)^2, skew U(-0.3,0.3)",
                "solver": f"ours: fgmres(30) + {net} (ilu(0) fallback), fp64 outer; "
                          "reference: gmres(30) + ilu(0) fp64",
                "rtol": 1e-8, "ordering": "rcm", "parallelism": f"replicas{world}",
                "l2": "inputs larger than L2 (matrix 1.3 GB, Krylov basis 11.5 GB)"}
    return {"workload": WORKLOADS["plain"], "vertices": s.owned, "entries": s.nnz, "block_size": s.bs,
            "mesh": "poisson-disk unit disk, delaunay, component-diagonal", "solver": "gmres(30)+ilu(0)",
            "rtol": 1e-8, "ordering": "rcm", "parallelism": f"replicas{world}",
            "l2": "inputs larger than L2 (matrix 336 MB, Krylov basis 2.9 GB)"}


def algorithmic_bytes(s, ilu_entries: int):
    n, bs, nnz = s.owned, s.bs, s.nnz
    return kernel_bytes("spmv", n, bs, nnz), kernel_bytes("ilu", n, bs, nnz, factor_entries=ilu_entries)


def first_layer_roofline(n, ms, peak, peak_kind):
    """The encoder folded into the first layer: per vertex the 32-byte input
    record, the 8-slot list (4-byte columns, 2-byte weights) and the new
    128-byte BF16 row."""
    if ms <= 0:
        return None
    b = n * (32 + 8 * 6 + 128)
    return {"kernel": "k_gnn_first_layer", "ms_per_launch": ms, "bytes_per_launch": b,
            "achieved": b / (ms * 1e-3) / 1e9, "unit": "GB/s", "frac": b / (ms * 1e-3) / 1e9 / peak,
            "peak_source": peak_kind}


def gnn_layer_bytes(n: int) -> int:
    """One fused message-passing layer (k_gnn_layer): each vertex's BF16 row of
    64 features read once and its new row written once (128 B each), and its
    padded 8-slot neighbour list (32-bit column + BF16 weight per slot, 48 B)."""
    return n * (2 * 128 + 48)


def gnn_layer_flops(n: int) -> int:
    """[h | m] (n x 128) times Wl^T (128 x 64) on the tensor cores."""
    return 2 * n * 128 * 64


# ---------------------------------------------------------------- CPU reference
def cpu_reference_solve(s, reps: int, native_build: bool = False, restart: int = 30):
    """The reference's own CPU GMRES(restart)+ILU(0) (oracle/_ref), one host
    thread; returns None when that build is absent."""
    import oracle

    try:
        ref = oracle.Reference(native=native_build)
    except FileNotFoundError:
        return None
    m = ref.matrix("bsr", s.owned, 0, s.bs, s.rowptr, s.cols, s.vals)
    t = time.time()
    pc = ref.pc("ilu", m, 0)
    setup = time.time() - t
    opts = oracle.default_options(restart=restart)
    times, last = [], None
    for _ in range(reps):
        t = time.time()
        r, x = ref.solve("gmres", m, pc, opts, s.rhs, np.zeros(s.owned * s.bs))
        times.append(time.time() - t)
        last = r
    return {"kind": "reference", "isa": ref.isa or "as shipped (no -march)", "seconds": times,
            "setup_seconds": setup, "iterations": int(last.iterations), "status": int(last.status),
            "true_residual": float(last.true_residual_norm)}


def run_reference(args):
    """The reference's CPU GMRES(30)+ILU(0) on the workload's system, built in
    this process with the reference's own RCM (oracle/_ref); this project's
    library is not loaded.  One step = one full solve from x0 = 0.  --warmup
    warm-up solves (fewer if they would exceed a third of --ref-budget, at
    least one), then timed solves until --steps or until --ref-budget seconds
    of them are spent, whichever comes first."""
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    import oracle

    try:
        ref = oracle.Reference()
    except FileNotFoundError:
        print(json.dumps({"impl": "reference", "unavailable": "reference harness oracle/_ref not built"}))
        return 0
    form = "learned" if args.form == "learned" else "plain"
    s, gen_s = build_system(form, args.vertices, args.seed, rcm=ref.rcm)
    m = ref.matrix("bsr", s.owned, 0, s.bs, s.rowptr, s.cols, s.vals)
    t = time.time()
    pc = ref.pc("ilu", m, 0)
    setup_s = time.time() - t
    opts = oracle.default_options(restart=30)
    x0 = np.zeros(s.owned * s.bs)
    warm, timed, last = [], [], None
    # The requested warm-up solves, unless they would take more than a third
    # of the timed budget (then one).
    while len(warm) < max(1, args.warmup) and (not warm or sum(warm) + warm[-1] <= args.ref_budget / 3):
        t = time.time()
        last, _x = ref.solve("gmres", m, pc, opts, s.rhs, x0)
        warm.append(time.time() - t)
    spent = 0.0
    while len(timed) < args.steps and (not timed or spent + timed[-1] <= args.ref_budget):
        t = time.time()
        last, _x = ref.solve("gmres", m, pc, opts, s.rhs, x0)
        timed.append(time.time() - t)
        spent += timed[-1]
    v = statistics.mean(timed)
    cpu = oracle.host_cpu()
    line = {
        "metric": METRIC, "value": v, "unit": "s", "n_gpus": args.gpus, "steps": len(timed),
        "warmup": len(warm), "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(form, s, world, correction_of(args)),
        "impl": "reference",
        "cpu_baseline": {"value": v, "unit": "s", "cores": 1, "kind": "reference",
                         "sample": f"{len(timed)} full reference GMRES(30)+ILU(0) solves of the "
                                   f"{s.owned}-vertex system ({int(last.iterations)} iterations each), one thread "
                                   f"(the reference is single-threaded); steps requested {args.steps}, "
                                   f"timed solves capped at {args.ref_budget:.0f} s",
                         "cpu": cpu},
        "e2e": {"value": v, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "steps_requested": args.steps, "warmup_requested": args.warmup,
        "reference_iterations": int(last.iterations), "reference_status": int(last.status),
        "reference_true_relative_residual": float(last.true_residual_norm / np.linalg.norm(s.rhs)),
        "reference_setup_s": setup_s, "system_build_s": gen_s, "warmup_seconds": warm,
        "ordering_by": "reference reverse_cuthill_mckee_order",
    }
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------- our arm
class _ZeroGuesses:
    """Pinned zero initial guesses for the host-buffer (end-to-end) steps,
    one per call and zeroed before the timed region: zeroing x0 on the host
    is input preparation, not part of the call being timed.  Beyond 6 GB of
    buffers the last one is re-zeroed before each further call (inside the
    timed region; `rezeroed` counts those calls)."""

    def __init__(self, elems, calls):
        import torch

        count = max(1, min(calls, (6 << 30) // max(1, elems * 8)))
        self.bufs = [torch.zeros(elems, dtype=torch.float64).pin_memory() for _ in range(count)]
        self.i = 0
        self.rezeroed = 0

    def next(self):
        if self.i < len(self.bufs):
            b = self.bufs[self.i]
        else:
            b = self.bufs[-1]
            b.zero_()
            self.rezeroed += 1
        self.i += 1
        return b


def _events(stream, fn, steps):
    import torch

    a, c = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        fn()
    c.record(stream)
    c.synchronize()
    return a.elapsed_time(c) / steps


def _max_over_ranks(ms, world, local):
    """The slowest rank's time (all ranks take part; NCCL reduces on the
    device, gloo on the host)."""
    if world > 1:
        import torch

        dev = "cpu" if torch.distributed.get_backend() == "gloo" else f"cuda:{local}"
        tt = torch.tensor([ms], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        return float(tt.item())
    return ms


def _checked(r, rhs_norm, rtol=1e-8, what="solve"):
    """A timed step counts only if it converged with the true residual at
    rtol (x0 = 0: the initial residual is the right-hand side)."""
    if r.status != 0 or not (r.true_residual_norm <= rtol * rhs_norm * (1 + 1e-12)):
        raise RuntimeError(f"{what} did not reach rtol {rtol}: {r.as_dict()}")
    return r


def run_learned(args):
    """The headline: learned-preconditioned FGMRES(30) vs plain FP64
    ILU(0)-GMRES(30) on the 8M-vertex anisotropic mesh, both to true-residual
    rtol 1e-8 from x0 = 0.  The network's weights come from the committed
    checkpoint (trained on 500 coefficient draws of a 200k-vertex mesh)."""
    import torch
    from owtk_b200 import checkpoint, native

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    s, gen_s = build_system("learned", args.vertices, args.seed)
    n, bs = s.owned, s.bs
    bnorm = float(np.linalg.norm(s.rhs))
    ctx = native.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", local))
    t = time.time()
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    ilu = native.Preconditioner(m, native.PC_ILU, 0)
    net = native.Learned(m, seed=1)
    ck = checkpoint.load_network(args.weights, net, with_optimizer=False)
    pcl = native.LearnedPreconditioner(net, ilu)
    pcl.set_correction(*correction_of(args))
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

    last = {}

    def step(pc, name):
        x.fill(0.0)
        last[name] = _checked(native.solve(native.FGMRES, m, pc, b, x, opts, ws), bnorm, what=name)

    for _ in range(args.warmup):
        step(pcl, "learned")
    barrier()
    apps0, falls0 = pcl.counts()
    launches0 = ctx.kernel_launches
    with Clocks(local) as clk:
        ms = _events(stream, lambda: step(pcl, "learned"), args.steps)
    barrier()
    launches = ctx.kernel_launches - launches0
    apps1, falls1 = pcl.counts()
    ms = _max_over_ranks(ms, world, local)
    learned_x = x.download()

    # Plain FP64 ILU(0)-GMRES(30) on the same system and GPU.
    for _ in range(max(1, args.warmup // 2)):
        step(ilu, "plain")
    barrier()
    plain_ms = _max_over_ranks(_events(stream, lambda: step(ilu, "plain"), args.steps), world, local)

    # End to end through the reference-facing host-buffer call: pinned rhs/x
    # copied in, solved, x copied back, every step.
    hb = torch.from_numpy(s.rhs.astype(np.float64)).pin_memory()
    guesses = _ZeroGuesses(n * bs, args.steps + 1)

    def host_step():
        hx = guesses.next()
        _checked(native.solve_host(native.FGMRES, m, pcl, hb.data_ptr(), hx.data_ptr(), opts, ws), bnorm,
                 what="learned (host buffers)")

    host_step()
    barrier()
    e2e_ms = _max_over_ranks(_events(stream, host_step, args.steps), world, local)

    # Roofline of the dominant kernel, live: the fused message-passing layer
    # (k_gnn_layer: layers 2-3 when the encoder is folded into the first
    # layer, else 1-3) timed per launch with CUDA events on the library's
    # stream over a network application on the right-hand side; the folded
    # first layer beside it (per vertex its 32-byte input record, the 8-slot
    # list and the new 128-byte row).
    y = native.Vector(ctx, n, 0, bs)
    st = net.stage_times(b, y, 20)
    peak, peak_kind = measured_peaks()
    tpeak, tpeak_kind = measured_tensor_peak()
    lb, lf = gnn_layer_bytes(n), gnn_layer_flops(n)
    layer_s = st["layer"] * 1e-3
    traffic = profiled_traffic()
    per_solve_apps = (apps1 - apps0) / args.steps
    clocks = clk.summary()
    cpu = plain2m = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        cpu = cpu_reference_solve(s, 1)
        vec = cpu_reference_solve(s, 1, native_build=True) if cpu else None
    if not args.no_plain_2m:
        plain2m = plain_2m_keys(ctx, stream, world, local)
    if rank == 0:
        line = {
            "metric": METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64+bf16", "data": "synthetic",
            "config": workload_config("learned", s, world, correction_of(args)),
            "e2e": {"value": e2e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": 2 * n * bs * 8,
                    "d2h_bytes_per_step": n * bs * 8,
                    "x0": "one pinned zero buffer per step, zeroed before the timed region",
                    "x0_rezeroed_in_timing": guesses.rezeroed},
            "roofline": {"bound": "hbm",
                         "kernel": "k_gnn_layer (fused message-passing layer, "
                                   + ("layers 2-3; layer 1 runs with the encoder folded in)"
                                      if st["encoder_first_layer"] > 0 else "layers 1-3)"),
                         "achieved": lb / layer_s / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": lb / layer_s / 1e9 / peak,
                         "traffic": traffic["k_gnn_layer"] * n if "k_gnn_layer" in traffic else None,
                         "traffic_source": "ncu DRAM bytes per vertex of one captured launch, scaled to this mesh",
                         "bytes_per_launch": lb, "ms_per_launch": st["layer"], "peak_source": peak_kind,
                         "tensor": {"achieved": lf / layer_s / 1e12, "peak": tpeak, "unit": "TFLOP/s",
                                    "frac": lf / layer_s / 1e12 / tpeak, "flops_per_launch": lf,
                                    "peak_source": tpeak_kind},
                         "network_stages_ms": st,
                         "first_layer": first_layer_roofline(n, st["encoder_first_layer"], peak, peak_kind),
                         "network_share_of_solve": per_solve_apps * st["application"] / ms},
            "learned": {"iterations": int(last["learned"].iterations),
                        "true_relative_residual": float(last["learned"].true_residual_norm / bnorm),
                        "network_applications_per_solve": per_solve_apps,
                        "fallbacks_per_solve": (falls1 - falls0) / args.steps,
                        "weights": os.path.relpath(args.weights, REPO),
                        "training": {k: ck["metadata"].get(k) for k in ("draws", "train_vertices", "epochs",
                                                                        "pairs_per_draw", "command")}},
            "plain_fp64_ilu0_gmres30": {"ms": plain_ms, "iterations": int(last["plain"].iterations),
                                        "true_relative_residual": float(last["plain"].true_residual_norm / bnorm)},
            "speedup_vs_plain_fp64_ilu_gmres": plain_ms / ms,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "setup_s": setup_s, "system_build_s": gen_s,
        }
        if cpu is not None:
            line["cpu_baseline"] = {
                "value": cpu["seconds"][0], "unit": "s", "cores": 1, "kind": "reference",
                "sample": f"one full reference GMRES(30)+ILU(0) solve of the same system "
                          f"({cpu['iterations']} iterations, ILU setup {cpu['setup_seconds']:.1f} s excluded), "
                          "reference built as shipped (-O3, no -march)",
                "cpu": oracle.host_cpu(),
                "vector_build": None if vec is None else {
                    "value": vec["seconds"][0], "isa": vec["isa"], "iterations": vec["iterations"]}}
            line["parity"] = {"plain_iterations": int(last["plain"].iterations),
                              "reference_iterations": cpu["iterations"],
                              "within_2": abs(int(last["plain"].iterations) - cpu["iterations"]) <= 2,
                              "reference_true_relative_residual": cpu["true_residual"] / bnorm}
        if plain2m is not None:
            line["plain_2m"] = plain2m
        print(json.dumps(line))
    del learned_x
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def plain_2m_keys(ctx, stream, world, local, steps: int = 5):
    """The 2M-vertex disk workload (FP64 GMRES(30)+ILU(0)): solve time, e2e,
    and the live rooflines of the ILU(0) sweep pair and the SpMV."""
    import torch
    from owtk_b200 import native

    s, gen_s = build_system("plain", 2_000_000, 1)
    n, bs = s.owned, s.bs
    bnorm = float(np.linalg.norm(s.rhs))
    m = native.Matrix(ctx, "bsr", n, 0, bs, s.rowptr, s.cols, s.vals)
    pc = native.Preconditioner(m, native.PC_ILU, 0)
    opts = native.default_options(restart=30, relative_tolerance=1e-8)
    ws = native.Workspace(ctx)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    x = native.Vector(ctx, n, 0, bs)
    res = {}

    def step():
        x.fill(0.0)
        res["r"] = _checked(native.solve(native.FGMRES, m, pc, b, x, opts, ws), bnorm, what="plain 2M")

    for _ in range(2):
        step()
    ctx.synchronize()
    ms = _max_over_ranks(_events(stream, step, steps), world, local)
    hb = torch.from_numpy(s.rhs.astype(np.float64)).pin_memory()
    guesses = _ZeroGuesses(n * bs, steps + 1)

    def host_step():
        hx = guesses.next()
        _checked(native.solve_host(native.FGMRES, m, pc, hb.data_ptr(), hx.data_ptr(), opts, ws), bnorm)

    host_step()
    e2e_ms = _max_over_ranks(_events(stream, host_step, steps), world, local)
    ilu_entries = int(pc.ilu_factors()[1].size)
    spmv_bytes, ilu_bytes = algorithmic_bytes(s, ilu_entries)
    y = native.Vector(ctx, n, 0, bs)
    m.apply(b, y)
    pc.apply(b, y)
    ctx.synchronize()
    spmv_ms = _events(stream, lambda: m.apply(b, y), 50)
    ilu_ms = _events(stream, lambda: pc.apply(b, y), 10)
    peak, _ = measured_peaks()
    traffic = profiled_traffic()
    return {"config": workload_config("plain", s, world), "ms": ms, "iterations": int(res["r"].iterations),
            "true_relative_residual": float(res["r"].true_residual_norm / bnorm),
            "e2e_ms": e2e_ms, "system_build_s": gen_s,
            "ilu0_sweep_pair": {"ms_per_launch": ilu_ms, "bytes_per_launch": ilu_bytes,
                                "achieved": ilu_bytes / (ilu_ms * 1e-3) / 1e9,
                                "frac": ilu_bytes / (ilu_ms * 1e-3) / 1e9 / peak,
                                "traffic": traffic["ilu0 sweep pair"] * n if "ilu0 sweep pair" in traffic else None},
            "spmv": {"us_per_launch": spmv_ms * 1e3, "bytes_per_launch": spmv_bytes,
                     "achieved": spmv_bytes / (spmv_ms * 1e-3) / 1e9,
                     "frac": spmv_bytes / (spmv_ms * 1e-3) / 1e9 / peak,
                     "traffic": traffic["spmv"] * n if "spmv" in traffic else None}}


def run_plain(args):
    """FP64 GMRES(30)+ILU(0) on the 2M-vertex disk mesh (the plain drop-in at
    scale) with the sweep-pair and SpMV rooflines."""
    import torch
    from owtk_b200 import native

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    s, gen_s = build_system("plain", args.vertices, args.seed)
    n, bs = s.owned, s.bs
    bnorm = float(np.linalg.norm(s.rhs))
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
    last = {}

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize(local)
        ctx.synchronize()

    def step():
        x.fill(0.0)
        last["r"] = _checked(native.solve(native.FGMRES, m, pc, b, x, opts, ws), bnorm)

    for _ in range(args.warmup):
        step()
    barrier()
    launches0 = ctx.kernel_launches
    with Clocks(local) as clk:
        ms = _events(stream, step, args.steps)
    barrier()
    launches = ctx.kernel_launches - launches0
    ms = _max_over_ranks(ms, world, local)
    hb = torch.from_numpy(s.rhs.astype(np.float64)).pin_memory()
    guesses = _ZeroGuesses(n * bs, args.steps + 1)

    def host_step():
        hx = guesses.next()
        _checked(native.solve_host(native.FGMRES, m, pc, hb.data_ptr(), hx.data_ptr(), opts, ws), bnorm)

    host_step()
    barrier()
    e2e_ms = _max_over_ranks(_events(stream, host_step, args.steps), world, local)
    ilu_entries = int(pc.ilu_factors()[1].size)
    spmv_bytes, ilu_bytes = algorithmic_bytes(s, ilu_entries)
    y = native.Vector(ctx, n, 0, bs)
    m.apply(b, y)
    pc.apply(b, y)
    ctx.synchronize()
    spmv_ms = _events(stream, lambda: m.apply(b, y), 50)
    ilu_ms = _events(stream, lambda: pc.apply(b, y), 10)
    peak, peak_kind = measured_peaks()
    traffic = profiled_traffic()
    clocks = clk.summary()
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        import oracle

        cpu = cpu_reference_solve(s, 1)
    if rank == 0:
        line = {
            "metric": METRIC, "value": ms / 1e3, "unit": "s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": workload_config("plain", s, world),
            "e2e": {"value": e2e_ms / 1e3, "unit": "s", "h2d_bytes_per_step": 2 * n * bs * 8,
                    "d2h_bytes_per_step": n * bs * 8,
                    "x0": "one pinned zero buffer per step, zeroed before the timed region",
                    "x0_rezeroed_in_timing": guesses.rezeroed},
            "roofline": {"bound": "hbm", "kernel": "ilu0 forward+backward sweep",
                         "achieved": ilu_bytes / (ilu_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                         "frac": ilu_bytes / (ilu_ms * 1e-3) / 1e9 / peak,
                         "traffic": traffic["ilu0 sweep pair"] * n if "ilu0 sweep pair" in traffic else None,
                         "traffic_source": "ncu DRAM bytes per vertex of one captured launch, scaled to this mesh",
                         "bytes_per_launch": ilu_bytes, "ms_per_launch": ilu_ms, "peak_source": peak_kind},
            "spmv": {"achieved": spmv_bytes / (spmv_ms * 1e-3) / 1e9, "unit": "GB/s",
                     "frac": spmv_bytes / (spmv_ms * 1e-3) / 1e9 / peak, "us_per_launch": spmv_ms * 1e3,
                     "bytes_per_launch": spmv_bytes,
                     "traffic": traffic["spmv"] * n if "spmv" in traffic else None},
            "iterations": int(last["r"].iterations), "setup_s": setup_s, "system_build_s": gen_s,
            "gpu_launches": int(launches),
            "clocks": clocks,
        }
        if cpu is not None:
            line["cpu_baseline"] = {"value": cpu["seconds"][0], "unit": "s", "cores": 1, "kind": cpu["kind"],
                                    "sample": f"one full reference solve of the same system "
                                              f"({cpu['iterations']} iterations, ILU setup "
                                              f"{cpu['setup_seconds']:.2f} s excluded)",
                                    "cpu": oracle.host_cpu()}
            line["parity"] = {"iterations": int(last["r"].iterations), "reference_iterations": cpu["iterations"],
                              "within_2": abs(int(last["r"].iterations) - cpu["iterations"]) <= 2}
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
    xy, edges = cached_mesh(args.vertices, args.seed, "disk")
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
            if "fgmres_jacobi" in only:
                # FGMRES(30) + Jacobi, 14 iterations fixed: the Gram-Schmidt
                # kernels with one SpMV and one element-wise apply per
                # iteration.  Algorithmic bytes: per iteration k (1..14) the
                # basis dots read w and k basis vectors, the fused second pass
                # reads k + 1 and writes w, the last pass reads k + 1 and
                # writes V_k (3k + 5 vector passes); the SpMV; Jacobi reads
                # two vectors and writes one.
                pj = native.Preconditioner(m, native.PC_JACOBI, 0)
                xs = native.Vector(ctx, n, 0, bs)
                ws = native.Workspace(ctx)
                opts = native.default_options(relative_tolerance=0.0, maximum_iterations=14, restart=30)

                def solve_j():
                    xs.fill(0.0)
                    native.solve(native.FGMRES, m, pj, x, xs, opts, ws)

                vec = n * bs * 8
                gs_bytes = sum((3 * k + 5) * vec for k in range(1, 15))
                us = timed(solve_j, max(2, args.reps // 4))
                emit("fgmres_jacobi", us, gs_bytes + 14 * (kernel_bytes("spmv", n, bs, nnz) + 3 * vec),
                     iterations=14, gram_schmidt_bytes=gs_bytes,
                     note="FGMRES(30) + Jacobi, 14 iterations: Gram-Schmidt, SpMV and Jacobi bytes over the solve")
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
    return _events(stream, fn, steps)


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
    guesses = _ZeroGuesses(rhs.size, args.steps + 1)

    def host_step():
        hx = guesses.next()
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
                     "d2h_bytes_per_step": rhs.size * 8,
                     "x0": "one pinned zero buffer per step, zeroed before the timed region",
                     "x0_rezeroed_in_timing": guesses.rezeroed},
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


def reference_dense_solution(s, rtol: float = 1e-13, budget_s: float = 300.0):
    """FP64 solution of a dense-block system by the reference's own GMRES(30)
    on its DenseBlockCsrMatrix (the reference has no preconditioner for dense
    blocks, so none is used), one host thread; None when oracle/_ref is absent."""
    import oracle

    try:
        ref = oracle.Reference()
    except FileNotFoundError:
        return None, None
    m = ref.matrix("dense", s.owned, 0, s.bs, s.rowptr, s.cols, s.vals)
    pc = ref.pc("identity", m, 0.0)
    t = time.time()
    r, x = ref.solve("gmres", m, pc, oracle.default_options(relative_tolerance=rtol, maximum_iterations=5000,
                                                            restart=30), s.rhs, np.zeros(s.owned * s.bs))
    info = {"solver": "reference gmres(30), no preconditioner", "rtol": rtol, "iterations": int(r.iterations),
            "status": int(r.status), "true_relative_residual": float(r.true_residual_norm / np.linalg.norm(s.rhs)),
            "seconds": time.time() - t}
    return (x if r.status == 0 else None), info


def run_mixed(args):
    """Dense 3x3 blocks on the 2M-vertex disk mesh: FP64 FGMRES(30) outer
    refinement to rtol 1e-10 around block-ILU(0) factors stored in FP32 and in
    BF16 with an FP32 inner solve of 0, 1, 2 or 4 GMRES steps, against the
    plain FP64 block-ILU(0) FGMRES; each solution's error is taken against
    the reference's own FP64 solution of the same system (rtol 1e-13)."""
    import torch
    from owtk_b200 import native, problems

    t = time.time()
    s = problems.config2(args.vertices)
    gen_s = time.time() - t
    n, bs = s.owned, s.bs
    bnorm = float(np.linalg.norm(s.rhs))
    ctx = native.Context(0)
    stream = torch.cuda.ExternalStream(ctx.stream, device=torch.device("cuda", 0))
    m = native.Matrix(ctx, "dense", n, 0, bs, s.rowptr, s.cols, s.vals)
    b = native.Vector(ctx, n, 0, bs).upload(s.rhs)
    opts = native.default_options(relative_tolerance=1e-10, restart=30)
    xref, ref_info = (None, None) if args.no_cpu_baseline else reference_dense_solution(s)
    out = {}
    runs = [("fp64", native.F64, None)]
    for storage_name, storage in (("fp32", native.F32), ("bf16", native.BF16)):
        for inner in (0, 1, 2, 4):
            runs.append((f"{storage_name}_inner{inner}", storage, inner))
    xs64 = None
    for name, storage, inner in runs:
        t = time.time()
        pc = native.Preconditioner(m, native.PC_BLOCK_ILU, 0, storage=storage, mixed_inner=inner)
        ctx.synchronize()
        setup_s = time.time() - t
        x = native.Vector(ctx, n, 0, bs)
        ws = native.Workspace(ctx)
        res = {}

        def step():
            x.fill(0.0)
            res["r"] = _checked(native.solve(native.FGMRES, m, pc, b, x, opts, ws), bnorm, rtol=1e-10, what=name)

        for _ in range(args.warmup):
            step()
        ms = _event_time(stream, step, args.steps)
        xs = x.download()
        if xs64 is None:
            xs64 = xs
        out[name] = {"ms": ms, "iterations": int(res["r"].iterations),
                     "preconditioner_applications": int(res["r"].preconditioner_applications),
                     "true_relative_residual": float(res["r"].true_residual_norm / bnorm),
                     "error_vs_gpu_fp64": float(np.linalg.norm(xs - xs64) / np.linalg.norm(xs64)),
                     "setup_s": setup_s}
        if xref is not None:
            out[name]["error_vs_reference_fp64"] = float(np.linalg.norm(xs - xref) / np.linalg.norm(xref))
        del pc, ws, x
    mixed = {k: v for k, v in out.items() if k != "fp64"}
    best = min(mixed, key=lambda k: mixed[k]["ms"])
    extra = {"mixed": out, "best_mixed": best, "speedup_vs_fp64": out["fp64"]["ms"] / mixed[best]["ms"],
             "reference_solution": ref_info}
    print(json.dumps(_line(args, "mixed-dense3x3-fgmres-blockilu0", mixed[best]["ms"] / 1e3, None,
                           {"vertices": n, "entries": s.nnz, "block_size": bs, "rtol": 1e-10,
                            "solver": "fgmres(30) fp64 outer, block-ilu(0) fp32/bf16 factors, fp32 inner",
                            "mesh_gen_s": gen_s}, "f64+f32", extra)))
    return 0


def main(argv=None):
    args = parse(argv)
    if args.impl == "reference":
        return run_reference(args)
    if args.kernels:
        return run_kernels(args)
    if args.form == "batching":
        return run_batching(args)
    if args.form == "mixed":
        return run_mixed(args)
    if args.form == "plain":
        return run_plain(args)
    return run_learned(args)


if __name__ == "__main__":
    sys.exit(main())
