"""ORACLE — test infrastructure only (tests/, __graft_entry__.smoke(), bench.py's
CPU-baseline and reference legs).  Never imported by the product.

Two CPU checkers behind one interface:
  * ``Restatement`` — oracle/owtk_oracle.c, a plain-C restatement of the
    reference path (built into oracle/_build/ by oracle/Makefile);
  * ``Reference``   — the unmodified reference headers behind
    oracle/ref_harness.cpp (built into oracle/_ref/ from the read-only
    reference tree; the built .so travels with the repository snapshot).
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from ctypes import POINTER, c_char_p, c_double, c_int, c_int64, c_size_t, c_uint64, c_void_p

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
RESTATEMENT_SO = os.path.join(HERE, "_build", "libowtk_oracle.so")
REFERENCE_SO = os.path.join(HERE, "_ref", "libowtk_ref.so")
REFERENCE_VECTOR_SO = {"avx512": os.path.join(HERE, "_ref", "libowtk_ref_avx512.so"),
                       "avx2": os.path.join(HERE, "_ref", "libowtk_ref_avx2.so")}


def host_vector_isa() -> str | None:
    """Highest x86-64 ISA level of the running CPU that a vector build of the
    reference targets: "avx512" (x86-64-v4), "avx2" (x86-64-v3) or None."""
    try:
        flags = set()
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("flags"):
                    flags = set(line.split(":", 1)[1].split())
                    break
    except OSError:
        return None
    if {"avx512f", "avx512bw", "avx512cd", "avx512dq", "avx512vl", "avx2", "fma"} <= flags:
        return "avx512"
    if {"avx2", "fma", "bmi1", "bmi2", "movbe"} <= flags:
        return "avx2"
    return None


def host_cpu() -> dict:
    """CPU model name and logical CPU count of this host."""
    model = None
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name"):
                    model = line.split(":", 1)[1].strip()
                    break
    except OSError:
        pass
    return {"model": model, "nproc": os.cpu_count(), "usable_cpus": len(os.sched_getaffinity(0))}


class Options(ctypes.Structure):
    _fields_ = [("relative_tolerance", c_double), ("absolute_tolerance", c_double),
                ("breakdown_tolerance", c_double), ("maximum_iterations", c_uint64),
                ("convergence_check_interval", c_uint64), ("restart", c_uint64),
                ("residual_replacement_interval", c_uint64), ("idr_shadow_space", c_uint64),
                ("relaxation", c_double), ("verify_true_residual", ctypes.c_int32),
                ("gmres_orthogonalization", ctypes.c_int32)]


class Result(ctypes.Structure):
    _fields_ = [("status", ctypes.c_int32), ("breakdown_reason", ctypes.c_int32), ("iterations", c_uint64),
                ("operator_applications", c_uint64), ("preconditioner_applications", c_uint64),
                ("global_reductions", c_uint64), ("reorthogonalizations", c_uint64),
                ("arnoldi_norm_verifications", c_uint64), ("initial_residual_norm", c_double),
                ("recursive_residual_norm", c_double), ("true_residual_norm", c_double),
                ("relative_residual_norm", c_double), ("converged_by_application", ctypes.c_int32),
                ("pad", ctypes.c_int32), ("solve_seconds", c_double)]

    def as_dict(self) -> dict:
        return {name: getattr(self, name) for name, _ in self._fields_ if name != "pad"}


def default_options(**kw) -> Options:
    o = Options(1e-8, 0.0, 64 * np.finfo(np.float64).eps, 1000, 10, 30, 50, 4, 1.0, 1, 0)
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


def reference_root() -> str | None:
    """The reference checkout the harness compiles against: $OWTK_REFERENCE_ROOT,
    else baseline/_ref beside the repository; None when neither holds it."""
    for root in (os.environ.get("OWTK_REFERENCE_ROOT"), os.path.join(os.path.dirname(HERE), "baseline", "_ref")):
        if root and os.path.exists(os.path.join(root, "include", "owt", "krylov", "core.hpp")):
            return root
    return None


def build(reference: bool = True) -> None:
    """Compile the checkers (gcc/g++ only; the reference leg needs its sources)."""
    subprocess.run(["make", "-s", "-C", HERE, "oracle"], check=True)
    root = reference_root()
    if reference and root is not None:
        subprocess.run(["make", "-s", "-C", HERE, "ref", f"REF={root}"], check=True)


def _p(a):
    return a.ctypes.data_as(c_void_p)


def _i64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int64))


def _u64(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


# --------------------------------------------------------------- restatement
class Restatement:
    """ctypes over oracle/owtk_oracle.c (double precision, int64 indices)."""

    def __init__(self):
        if not os.path.exists(RESTATEMENT_SO):
            build(reference=False)
        L = ctypes.CDLL(RESTATEMENT_SO)
        vp = c_void_p
        for name, res, args in [
            ("orc_bsr_spmv", None, [c_int64, c_int64, vp, vp, vp, vp, vp]),
            ("orc_split_spmv", None, [c_int64, c_int64, vp, vp, vp, vp, vp, vp]),
            ("orc_dense_spmv", None, [c_int64, c_int64, vp, vp, vp, vp, vp]),
            ("orc_dot", c_double, [c_int64, vp, vp]),
            ("orc_norm", c_double, [c_int64, vp]),
            ("orc_jacobi_inverse", c_int, [c_int64, c_int64, vp, vp, vp, vp, c_double, vp]),
            ("orc_jacobi_apply", None, [c_int64, vp, vp, vp]),
            ("orc_ssor_apply", c_int, [c_int64, c_int64, vp, vp, vp, c_double, vp, vp, vp]),
            ("orc_split_ssor_apply", None, [c_int64, c_int64, vp, vp, vp, vp, c_double, vp, vp, vp]),
            ("orc_ilu_create", vp, [c_int64, c_int64, vp, vp, vp, c_int64, POINTER(c_int)]),
            ("orc_ilu_update", c_int, [vp, vp, vp, vp]),
            ("orc_ilu_apply", None, [vp, vp, vp]),
            ("orc_ilu_entries", c_int64, [vp]),
            ("orc_ilu_copy", None, [vp, vp, vp, vp, vp, vp, vp]),
            ("orc_ilu_destroy", None, [vp]),
            ("orc_levels", None, [c_int64, vp, vp, vp, vp]),
            ("orc_rcm", c_int, [c_int64, vp, vp, vp]),
            ("orc_hilbert", c_int, [c_int64, vp, vp]),
            ("orc_block_ilu_create", vp, [c_int64, c_int64, vp, vp, vp, POINTER(c_int)]),
            ("orc_block_ilu_apply", None, [vp, vp, vp]),
            ("orc_block_ilu_copy", None, [vp, vp, vp]),
            ("orc_block_ilu_entries", c_int64, [vp]),
            ("orc_block_ilu_destroy", None, [vp]),
            ("orc_bicgstab", None, [vp, vp, POINTER(Options), vp, vp, POINTER(Result)]),
            ("orc_gmres", None, [vp, vp, POINTER(Options), vp, vp, POINTER(Result)]),
        ]:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        self.L = L

    def bsr_spmv(self, owned, bs, rp, ci, v, x):
        rp, ci = _i64(rp), _i64(ci)
        v, x = np.ascontiguousarray(v, np.float64), np.ascontiguousarray(x, np.float64)
        y = np.zeros(owned * bs)
        self.L.orc_bsr_spmv(owned, bs, _p(rp), _p(ci), _p(v), _p(x), _p(y))
        return y

    def split_spmv(self, owned, bs, rp, ci, diag, off, x):
        rp, ci = _i64(rp), _i64(ci)
        diag, off, x = (np.ascontiguousarray(a, np.float64) for a in (diag, off, x))
        y = np.zeros(owned * bs)
        self.L.orc_split_spmv(owned, bs, _p(rp), _p(ci), _p(diag), _p(off), _p(x), _p(y))
        return y

    def dense_spmv(self, owned, bs, rp, ci, v, x):
        rp, ci = _i64(rp), _i64(ci)
        v, x = np.ascontiguousarray(v, np.float64), np.ascontiguousarray(x, np.float64)
        y = np.zeros(owned * bs)
        self.L.orc_dense_spmv(owned, bs, _p(rp), _p(ci), _p(v), _p(x), _p(y))
        return y

    def dot(self, a, b):
        a, b = np.ascontiguousarray(a, np.float64), np.ascontiguousarray(b, np.float64)
        return self.L.orc_dot(a.size, _p(a), _p(b))

    def norm(self, a):
        a = np.ascontiguousarray(a, np.float64)
        return self.L.orc_norm(a.size, _p(a))

    def jacobi_inverse(self, owned, bs, rp, ci, v, split_diag=None, minimum=64 * np.finfo(float).eps):
        rp, ci = _i64(rp), _i64(ci)
        v = np.ascontiguousarray(v if v is not None else np.zeros(1), np.float64)
        inv = np.zeros(owned * bs)
        sd = None if split_diag is None else np.ascontiguousarray(split_diag, np.float64)
        code = self.L.orc_jacobi_inverse(owned, bs, _p(rp), _p(ci), _p(v), _p(sd) if sd is not None else None,
                                         minimum, _p(inv))
        return code, inv

    def ssor_apply(self, owned, bs, rp, ci, v, omega, x):
        rp, ci = _i64(rp), _i64(ci)
        v, x = np.ascontiguousarray(v, np.float64), np.ascontiguousarray(x, np.float64)
        out = np.zeros(owned * bs)
        work = np.zeros(owned * bs)
        code = self.L.orc_ssor_apply(owned, bs, _p(rp), _p(ci), _p(v), omega, _p(x), _p(out), _p(work))
        return code, out

    def split_ssor_apply(self, owned, bs, rp, ci, diag, off, omega, x):
        rp, ci = _i64(rp), _i64(ci)
        diag, off, x = (np.ascontiguousarray(a, np.float64) for a in (diag, off, x))
        out = np.zeros(owned * bs)
        work = np.zeros(owned * bs)
        self.L.orc_split_ssor_apply(owned, bs, _p(rp), _p(ci), _p(diag), _p(off), omega, _p(x), _p(out), _p(work))
        return out

    def ilu(self, owned, bs, rp, ci, v, fill=0):
        return RestatedIlu(self, owned, bs, rp, ci, v, fill)

    def block_ilu(self, owned, bs, rp, ci, v):
        return RestatedBlockIlu(self, owned, bs, rp, ci, v)

    def levels(self, owned, rp, ci):
        rp, ci = _i64(rp), _i64(ci)
        lo = np.zeros(owned, np.int64)
        up = np.zeros(owned, np.int64)
        self.L.orc_levels(owned, _p(rp), _p(ci), _p(lo), _p(up))
        return lo, up

    def rcm(self, owned, rp, ci):
        rp, ci = _i64(rp), _i64(ci)
        out = np.zeros(owned, np.int64)
        self.L.orc_rcm(owned, _p(rp), _p(ci), _p(out))
        return out

    def hilbert(self, xy):
        xy = np.ascontiguousarray(xy, np.float64)
        out = np.zeros(xy.shape[0], np.int64)
        self.L.orc_hilbert(xy.shape[0], _p(xy), _p(out))
        return out

    def solve(self, solver: str, matrix: dict, pc: dict, options: Options, rhs, x0):
        """solver 'gmres' | 'bicgstab'; matrix/pc dicts as built by make_matrix/make_pc."""
        x = np.array(x0, dtype=np.float64, copy=True)
        b = np.ascontiguousarray(rhs, np.float64)
        r = Result()
        fn = self.L.orc_gmres if solver == "gmres" else self.L.orc_bicgstab
        fn(ctypes.byref(matrix["struct"]), ctypes.byref(pc["struct"]), ctypes.byref(options), _p(b), _p(x),
           ctypes.byref(r))
        return r, x

    class _Matrix(ctypes.Structure):
        _fields_ = [("kind", c_int), ("owned", c_int64), ("ghost", c_int64), ("bs", c_int64),
                    ("rp", c_void_p), ("ci", c_void_p), ("v", c_void_p), ("diag", c_void_p), ("off", c_void_p)]

    class _Pc(ctypes.Structure):
        _fields_ = [("kind", c_int), ("omega", c_double), ("inv", c_void_p), ("ilu", c_void_p),
                    ("work", c_void_p)]

    def make_matrix(self, kind, owned, ghost, bs, rp, ci, v=None, diag=None, off=None):
        keep = {"rp": _i64(rp), "ci": _i64(ci)}
        for k, a in (("v", v), ("diag", diag), ("off", off)):
            if a is not None:
                keep[k] = np.ascontiguousarray(a, np.float64)
        st = self._Matrix({"bsr": 0, "split": 1, "dense": 2}[kind], owned, ghost, bs, _p(keep["rp"]),
                          _p(keep["ci"]), _p(keep["v"]) if "v" in keep else None,
                          _p(keep["diag"]) if "diag" in keep else None,
                          _p(keep["off"]) if "off" in keep else None)
        return {"struct": st, "keep": keep, "owned": owned, "bs": bs}

    def make_pc(self, kind, matrix, parameter=1.0, ilu=None):
        owned, bs = matrix["owned"], matrix["bs"]
        keep = {}
        st = self._Pc({"identity": 0, "jacobi": 1, "ssor": 2, "split_ssor": 3, "ilu": 4}[kind], parameter,
                      None, None, None)
        if kind == "jacobi":
            k = matrix["keep"]
            code, inv = self.jacobi_inverse(owned, bs, k["rp"], k["ci"], k.get("v"), k.get("diag"))
            if code:
                raise ValueError("singular Jacobi diagonal")
            keep["inv"] = inv
            st.inv = _p(inv)
        if kind in ("ssor", "split_ssor"):
            keep["work"] = np.zeros(owned * bs)
            st.work = _p(keep["work"])
        if kind == "ilu":
            st.ilu = ilu.h
            keep["ilu"] = ilu
        return {"struct": st, "keep": keep}


class RestatedIlu:
    def __init__(self, o: Restatement, owned, bs, rp, ci, v, fill):
        self.o, self.owned, self.bs = o, owned, bs
        rp, ci = _i64(rp), _i64(ci)
        v = np.ascontiguousarray(v, np.float64)
        st = c_int(0)
        self.h = o.L.orc_ilu_create(owned, bs, _p(rp), _p(ci), _p(v), fill, ctypes.byref(st))
        self.status = st.value

    def factors(self):
        n = self.o.L.orc_ilu_entries(self.h)
        rp = np.zeros(self.owned + 1, np.int64)
        ci = np.zeros(max(n, 1), np.int64)
        val = np.zeros(max(n * self.bs, 1))
        inv = np.zeros(self.owned * self.bs)
        dp = np.zeros(self.owned, np.int64)
        src = np.zeros(max(n, 1), np.int64)
        self.o.L.orc_ilu_copy(self.h, _p(rp), _p(ci), _p(val), _p(inv), _p(dp), _p(src))
        return rp, ci[:n], val[:n * self.bs], inv, dp, src[:n]

    def update(self, rp, ci, v):
        rp, ci = _i64(rp), _i64(ci)
        v = np.ascontiguousarray(v, np.float64)
        return self.o.L.orc_ilu_update(self.h, _p(rp), _p(ci), _p(v))

    def apply(self, x):
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros(self.owned * self.bs)
        self.o.L.orc_ilu_apply(self.h, _p(x), _p(out))
        return out

    def __del__(self):
        try:
            self.o.L.orc_ilu_destroy(self.h)
        except Exception:
            pass


class RestatedBlockIlu:
    """Dense-block ILU(0) (no reference counterpart; see owtk_oracle.c)."""

    def __init__(self, o: Restatement, owned, bs, rp, ci, v):
        self.o, self.owned, self.bs = o, owned, bs
        rp, ci = _i64(rp), _i64(ci)
        v = np.ascontiguousarray(v, np.float64)
        st = c_int(0)
        self.h = o.L.orc_block_ilu_create(owned, bs, _p(rp), _p(ci), _p(v), ctypes.byref(st))
        self.status = st.value

    def factors(self):
        n = self.o.L.orc_block_ilu_entries(self.h)
        b2 = self.bs * self.bs
        val = np.zeros(max(n * b2, 1))
        dinv = np.zeros(self.owned * b2)
        self.o.L.orc_block_ilu_copy(self.h, _p(val), _p(dinv))
        return val[: n * b2], dinv

    def apply(self, x):
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros(self.owned * self.bs)
        self.o.L.orc_block_ilu_apply(self.h, _p(x), _p(out))
        return out

    def __del__(self):
        try:
            self.o.L.orc_block_ilu_destroy(self.h)
        except Exception:
            pass


# ----------------------------------------------------------------- reference
class Reference:
    """ctypes over oracle/ref_harness.cpp compiled against the reference headers."""

    PC = {"identity": 0, "jacobi": 1, "ssor": 2, "split_ssor": 3, "ilu": 4}
    SOLVER = {"gmres": 0, "fgmres": 0, "bicgstab": 1, "pipelined_bicgstab": 2,
              "comm_hiding_bicgstab": 3, "idrs": 4}

    def __init__(self, native: bool = False):
        """native=False: the build as the reference ships (no -march).  native=True:
        the vector build for the running CPU's ISA level (AVX-512 or AVX2 paths
        of the reference's simd.hpp); FileNotFoundError when there is none."""
        self.isa = None
        if native:
            self.isa = host_vector_isa()
            if self.isa is None:
                raise FileNotFoundError("no AVX2 or AVX-512 on this CPU for a vector build of the reference")
            path = REFERENCE_VECTOR_SO[self.isa]
        else:
            path = REFERENCE_SO
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        L = ctypes.CDLL(path)
        vp, sz = c_void_p, c_size_t
        for name, res, args in [
            ("ref_last_error", c_char_p, []),
            ("ref_default_options", None, [POINTER(Options)]),
            ("ref_bsr_create", c_int, [sz, sz, sz, vp, vp, vp, POINTER(vp)]),
            ("ref_dense_create", c_int, [sz, sz, sz, vp, vp, vp, POINTER(vp)]),
            ("ref_split_create", c_int, [sz, sz, sz, vp, vp, vp, vp, POINTER(vp)]),
            ("ref_split_set_values", c_int, [vp, vp, vp]),
            ("ref_bsr_set_values", c_int, [vp, vp]),
            ("ref_matrix_destroy", None, [vp]),
            ("ref_matrix_apply", c_int, [vp, vp, vp]),
            ("ref_matrix_diagonal", c_int, [vp, vp]),
            ("ref_pc_create", c_int, [c_int, vp, c_double, POINTER(vp)]),
            ("ref_pc_destroy", None, [vp]),
            ("ref_pc_apply", c_int, [vp, vp, vp]),
            ("ref_pc_update_values", c_int, [vp]),
            ("ref_pc_numeric_updates", c_uint64, [vp]),
            ("ref_ilu_factors", c_int, [vp, POINTER(c_uint64), vp, vp, vp, vp]),
            ("ref_workspace_create", vp, []),
            ("ref_workspace_destroy", None, [vp]),
            ("ref_workspace_epochs", c_uint64, [vp]),
            ("ref_workspace_vector", c_int, [vp, sz, vp]),
            ("ref_solve", c_int, [c_int, c_int, vp, vp, POINTER(Options), vp, vp, vp, POINTER(Result)]),
            ("ref_dot", c_double, [sz, sz, sz, vp, vp]),
            ("ref_norm", c_double, [sz, sz, sz, vp]),
            ("ref_solve_ex", c_int, [c_int, c_int, vp, vp, POINTER(Options), vp, vp, c_uint64, vp, vp, vp,
                                     POINTER(Result)]),
            ("ref_solve_specwave", c_int, [c_int, vp, POINTER(Options), vp, vp, POINTER(Result)]),
            ("ref_dot_kind", c_double, [c_int, sz, sz, sz, vp, vp, vp]),
            ("ref_norm_kind", c_double, [c_int, sz, sz, sz, vp]),
            ("ref_rcm", c_int, [sz, sz, vp, vp, vp]),
            ("ref_hilbert", c_int, [sz, vp, vp]),
            ("ref_inverse_permutation", c_int, [sz, vp, vp]),
        ]:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        self.L = L

    def check(self, code):
        if code != 0:
            raise ReferenceError_(code, self.L.ref_last_error().decode())

    def matrix(self, kind, owned, ghost, bs, rp, ci, v=None, diag=None, off=None):
        return RefMatrix(self, kind, owned, ghost, bs, rp, ci, v, diag, off)

    def pc(self, kind, matrix, parameter=0.0):
        return RefPc(self, kind, matrix, parameter)

    def solve(self, solver, matrix, pc, options, rhs, x0, reduction=0, workspace=None):
        x = np.array(x0, dtype=np.float64, copy=True)
        b = np.ascontiguousarray(rhs, np.float64)
        r = Result()
        self.check(self.L.ref_solve(self.SOLVER[solver], reduction, matrix.h, pc.h, ctypes.byref(options), _p(b),
                                    _p(x), workspace, ctypes.byref(r)))
        return r, x

    REDUCTION = {"serial": 0, "compensated": 1, "mixed": 2}

    def solve_ex(self, solver, matrix, pc, options, rhs, x0, reduction="serial", stop_at=0, snapshot=False):
        """ref_solve_ex: optional convergence test stopping at iteration
        `stop_at` and (FGMRES) the Arnoldi snapshot: returns (result, x,
        snapshot dict or None)."""
        x = np.array(x0, dtype=np.float64, copy=True)
        b = np.ascontiguousarray(rhs, np.float64)
        r = Result()
        cols = ctypes.c_uint64(0)
        R = int(options.restart)
        n = b.size
        h = np.zeros((R + 1) * max(R, 1)) if snapshot else None
        z = np.zeros(max(R, 1) * n) if snapshot else None
        self.check(self.L.ref_solve_ex(self.SOLVER[solver], self.REDUCTION[reduction], matrix.h, pc.h,
                                       ctypes.byref(options), _p(b), _p(x), int(stop_at),
                                       ctypes.byref(cols) if snapshot else None, _p(h) if snapshot else None,
                                       _p(z) if snapshot else None, ctypes.byref(r)))
        snap = None
        if snapshot:
            c = int(cols.value)
            snap = {"columns": c, "h": h.reshape(max(R, 1), R + 1)[:c, : c + 1].T.copy(),
                    "basis": z[: c * n].reshape(c, n).copy()}
        return r, x, snap

    def solve_specwave(self, solver_id, matrix, options, rhs, x0):
        x = np.array(x0, dtype=np.float64, copy=True)
        b = np.ascontiguousarray(rhs, np.float64)
        r = Result()
        self.check(self.L.ref_solve_specwave(int(solver_id), matrix.h, ctypes.byref(options), _p(b), _p(x),
                                             ctypes.byref(r)))
        return r, x

    def dot_kind(self, reduction, owned, ghost, bs, a, b):
        """(hi, lo) of the reference dot with the named reduction."""
        a, b = np.ascontiguousarray(a, np.float64), np.ascontiguousarray(b, np.float64)
        lo = ctypes.c_double(0)
        hi = self.L.ref_dot_kind(self.REDUCTION[reduction], owned, ghost, bs, _p(a), _p(b), ctypes.byref(lo))
        return hi, lo.value

    def norm_kind(self, reduction, owned, ghost, bs, a):
        a = np.ascontiguousarray(a, np.float64)
        return self.L.ref_norm_kind(self.REDUCTION[reduction], owned, ghost, bs, _p(a))

    def dot(self, owned, ghost, bs, a, b):
        a, b = np.ascontiguousarray(a, np.float64), np.ascontiguousarray(b, np.float64)
        return self.L.ref_dot(owned, ghost, bs, _p(a), _p(b))

    def norm(self, owned, ghost, bs, a):
        a = np.ascontiguousarray(a, np.float64)
        return self.L.ref_norm(owned, ghost, bs, _p(a))

    def rcm(self, owned, rp, ci, ghost=0):
        rp, ci = _u64(rp), _u64(ci)
        out = np.zeros(owned, np.uint64)
        self.check(self.L.ref_rcm(owned, ghost, _p(rp), _p(ci), _p(out)))
        return out.astype(np.int64)

    def inverse_permutation(self, new_to_old):
        p = _u64(new_to_old)
        out = np.zeros(p.size, np.uint64)
        self.check(self.L.ref_inverse_permutation(p.size, _p(p), _p(out)))
        return out.astype(np.int64)

    def hilbert(self, xy):
        xy = np.ascontiguousarray(xy, np.float64)
        out = np.zeros(xy.shape[0], np.uint64)
        self.check(self.L.ref_hilbert(xy.shape[0], _p(xy), _p(out)))
        return out.astype(np.int64)


class ReferenceError_(RuntimeError):
    KIND = {1: "invalid_argument", 2: "zero_pivot", 3: "out_of_range", 7: "runtime_error"}

    def __init__(self, code, message):
        super().__init__(f"{self.KIND.get(code, code)}: {message}")
        self.code = code
        self.kind = self.KIND.get(code, str(code))
        self.message = message


class RefMatrix:
    def __init__(self, ref: Reference, kind, owned, ghost, bs, rp, ci, v, diag, off):
        self.ref, self.kind, self.owned, self.ghost, self.bs = ref, kind, owned, ghost, bs
        rp, ci = _u64(rp), _u64(ci)
        if ci.size == 0:
            ci = np.zeros(1, np.uint64)
        h = c_void_p()
        if kind == "bsr":
            v = np.ascontiguousarray(v, np.float64)
            ref.check(ref.L.ref_bsr_create(owned, ghost, bs, _p(rp), _p(ci), _p(v), ctypes.byref(h)))
        elif kind == "dense":
            v = np.ascontiguousarray(v, np.float64)
            ref.check(ref.L.ref_dense_create(owned, ghost, bs, _p(rp), _p(ci), _p(v), ctypes.byref(h)))
        else:
            diag, off = np.ascontiguousarray(diag, np.float64), np.ascontiguousarray(off, np.float64)
            if off.size == 0:
                off = np.zeros(1)
            ref.check(ref.L.ref_split_create(owned, ghost, bs, _p(rp), _p(ci), _p(diag), _p(off), ctypes.byref(h)))
        self.h = h

    @property
    def local(self):
        return (self.owned + self.ghost) * self.bs

    def apply(self, x, y=None):
        x = np.ascontiguousarray(x, np.float64)
        y = np.zeros(self.local) if y is None else np.array(y, dtype=np.float64, copy=True)
        self.ref.check(self.ref.L.ref_matrix_apply(self.h, _p(x), _p(y)))
        return y

    def set_values(self, v=None, diag=None, off=None):
        if self.kind == "split":
            diag, off = np.ascontiguousarray(diag, np.float64), np.ascontiguousarray(off, np.float64)
            self.ref.check(self.ref.L.ref_split_set_values(self.h, _p(diag), _p(off)))
        else:
            v = np.ascontiguousarray(v, np.float64)
            self.ref.check(self.ref.L.ref_bsr_set_values(self.h, _p(v)))

    def __del__(self):
        try:
            self.ref.L.ref_matrix_destroy(self.h)
        except Exception:
            pass


class RefPc:
    def __init__(self, ref: Reference, kind, matrix: RefMatrix, parameter):
        self.ref, self.matrix = ref, matrix
        h = c_void_p()
        ref.check(ref.L.ref_pc_create(Reference.PC[kind], matrix.h, parameter, ctypes.byref(h)))
        self.h = h

    def apply(self, x, out=None, inplace=False):
        m = self.matrix
        if inplace:
            buf = np.array(x, dtype=np.float64, copy=True)
            self.ref.check(self.ref.L.ref_pc_apply(self.h, _p(buf), _p(buf)))
            return buf
        x = np.ascontiguousarray(x, np.float64)
        out = np.zeros(m.local) if out is None else np.array(out, dtype=np.float64, copy=True)
        self.ref.check(self.ref.L.ref_pc_apply(self.h, _p(x), _p(out)))
        return out

    def update_values(self):
        self.ref.check(self.ref.L.ref_pc_update_values(self.h))

    @property
    def numeric_updates(self):
        return self.ref.L.ref_pc_numeric_updates(self.h)

    def ilu_factors(self):
        n = c_uint64()
        self.ref.check(self.ref.L.ref_ilu_factors(self.h, ctypes.byref(n), None, None, None, None))
        m = self.matrix
        rp = np.zeros(m.owned + 1, np.uint64)
        ci = np.zeros(max(n.value, 1), np.uint64)
        v = np.zeros(max(n.value * m.bs, 1))
        inv = np.zeros(m.owned * m.bs)
        self.ref.check(self.ref.L.ref_ilu_factors(self.h, ctypes.byref(n), _p(rp), _p(ci), _p(v), _p(inv)))
        return rp.astype(np.int64), ci[:n.value].astype(np.int64), v[:n.value * m.bs], inv

    def __del__(self):
        try:
            self.ref.L.ref_pc_destroy(self.h)
        except Exception:
            pass
