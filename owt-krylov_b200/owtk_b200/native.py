"""ctypes binding of the C ABI in include/owtk.h (lib/libowtk_b200.so).

The library is the product: this module only marshals arguments.  Loading
fails loudly when the shared object is missing — there is no fallback.
"""
from __future__ import annotations

import ctypes
import os
from ctypes import POINTER, c_char_p, c_double, c_int, c_int32, c_size_t, c_uint64, c_void_p

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(os.path.dirname(_HERE), "lib", "libowtk_b200.so")

F64, F32, BF16 = 0, 1, 2
PC_IDENTITY, PC_JACOBI, PC_SSOR, PC_SPLIT_SSOR, PC_ILU, PC_BLOCK_ILU, PC_MIXED, PC_LEARNED = 0, 1, 2, 3, 4, 5, 6, 7
FGMRES, BICGSTAB, PIPELINED_BICGSTAB, COMM_HIDING_BICGSTAB, IDRS = 0, 1, 2, 3, 4

STATUS = {0: "ok", 1: "invalid_argument", 2: "zero_pivot", 3: "out_of_range", 4: "cuda_error",
          5: "timeout", 6: "no_device", 7: "runtime_error"}
SOLVER_STATUS = ["converged", "maximum_iterations", "breakdown", "diverged", "invalid_input"]
BREAKDOWN = ["none", "arnoldi_invariant_subspace", "singular_projected_system",
             "biorthogonality_loss", "alpha_denominator", "omega_denominator", "omega_zero",
             "idr_shadow_space", "idr_small_system", "non_finite_scalar"]


class OwtkError(RuntimeError):
    def __init__(self, code: int, message: str):
        super().__init__(f"{STATUS.get(code, code)}: {message}")
        self.code = code
        self.kind = STATUS.get(code, str(code))
        self.message = message


class SolverOptions(ctypes.Structure):
    _fields_ = [("relative_tolerance", c_double), ("absolute_tolerance", c_double),
                ("breakdown_tolerance", c_double), ("maximum_iterations", c_uint64),
                ("convergence_check_interval", c_uint64), ("restart", c_uint64),
                ("residual_replacement_interval", c_uint64), ("idr_shadow_space", c_uint64),
                ("relaxation", c_double), ("verify_true_residual", c_int32),
                ("gmres_orthogonalization", c_int32)]


class SolverResult(ctypes.Structure):
    _fields_ = [("status", c_int32), ("breakdown_reason", c_int32), ("iterations", c_uint64),
                ("operator_applications", c_uint64), ("preconditioner_applications", c_uint64),
                ("global_reductions", c_uint64), ("reorthogonalizations", c_uint64),
                ("arnoldi_norm_verifications", c_uint64), ("initial_residual_norm", c_double),
                ("recursive_residual_norm", c_double), ("true_residual_norm", c_double),
                ("relative_residual_norm", c_double), ("converged_by_application", c_int32),
                ("reserved", c_int32), ("solve_seconds", c_double)]

    def as_dict(self) -> dict:
        d = {name: getattr(self, name) for name, _ in self._fields_ if name != "reserved"}
        d["status_name"] = SOLVER_STATUS[self.status] if 0 <= self.status < 5 else str(self.status)
        d["breakdown_name"] = BREAKDOWN[self.breakdown_reason] if 0 <= self.breakdown_reason < 10 else "?"
        return d


CONVERGENCE_TEST = ctypes.CFUNCTYPE(c_int, c_void_p, c_uint64, c_void_p, c_size_t)
HOST_APPLY = ctypes.CFUNCTYPE(c_int, c_void_p, c_void_p, c_void_p, c_size_t)
REDUCTION = {"serial": 0, "compensated": 1, "mixed": 2}


class SolveExtras(ctypes.Structure):
    _fields_ = [("reduction", c_int32), ("reserved", c_int32), ("convergence_test", CONVERGENCE_TEST),
                ("convergence_user", c_void_p), ("arnoldi_snapshot", c_void_p)]


class BatchSystem(ctypes.Structure):
    _fields_ = [("owned", c_size_t), ("bs", c_size_t), ("rowptr", c_void_p), ("cols", c_void_p),
                ("values", c_void_p)]


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise OSError(f"owtk CUDA library not built: {LIB_PATH} (run `make -C owt-krylov_b200`)")
        L = ctypes.CDLL(LIB_PATH)
        vp, sz, u64p = c_void_p, c_size_t, POINTER(c_uint64)
        sig = {
            "owtk_last_error": (c_char_p, []),
            "owtk_abi_version": (c_int, []),
            "owtk_context_create": (c_int, [c_int, POINTER(vp)]),
            "owtk_context_destroy": (c_int, [vp]),
            "owtk_context_synchronize": (c_int, [vp]),
            "owtk_context_stream": (vp, [vp]),
            "owtk_context_kernel_launches": (c_uint64, [vp]),
            "owtk_vector_create": (c_int, [vp, c_int, sz, sz, sz, POINTER(vp)]),
            "owtk_vector_view": (c_int, [vp, c_int, sz, sz, sz, vp, sz, POINTER(vp)]),
            "owtk_vector_destroy": (c_int, [vp]),
            "owtk_vector_data": (vp, [vp]),
            "owtk_vector_upload": (c_int, [vp, vp, sz]),
            "owtk_vector_download": (c_int, [vp, vp, sz]),
            "owtk_vector_fill": (c_int, [vp, c_double, c_int]),
            "owtk_copy_owned": (c_int, [vp, vp]),
            "owtk_axpy": (c_int, [c_double, vp, vp]),
            "owtk_scale": (c_int, [c_double, vp]),
            "owtk_assign_linear_combination": (c_int, [vp, c_double, vp, c_double, vp]),
            "owtk_dot": (c_int, [vp, vp, POINTER(c_double)]),
            "owtk_norm": (c_int, [vp, POINTER(c_double)]),
            "owtk_dot_batch": (c_int, [vp, POINTER(vp), sz, POINTER(c_double)]),
            "owtk_bsr_create": (c_int, [vp, c_int, sz, sz, sz, vp, vp, vp, POINTER(vp)]),
            "owtk_bsr_update_values": (c_int, [vp, vp]),
            "owtk_split_view_create": (c_int, [vp, c_int, sz, sz, sz, vp, vp, vp, vp, POINTER(vp)]),
            "owtk_dense_bsr_create": (c_int, [vp, c_int, sz, sz, sz, vp, vp, vp, POINTER(vp)]),
            "owtk_matrix_destroy": (c_int, [vp]),
            "owtk_matrix_info": (c_int, [vp, POINTER(c_int), POINTER(sz), POINTER(sz), POINTER(sz), POINTER(sz)]),
            "owtk_spmv": (c_int, [vp, vp, vp]),
            "owtk_spmv_rows": (c_int, [vp, vp, vp, vp, sz]),
            "owtk_matrix_diagonal": (c_int, [vp, vp]),
            "owtk_pc_create": (c_int, [vp, c_int, c_double, POINTER(vp)]),
            "owtk_pc_destroy": (c_int, [vp]),
            "owtk_pc_create_stored": (c_int, [vp, c_int, c_double, c_int, POINTER(vp)]),
            "owtk_pc_create_mixed": (c_int, [vp, c_int, c_double, c_int, ctypes.c_uint32, POINTER(vp)]),
            "owtk_pc_apply": (c_int, [vp, vp, vp]),
            "owtk_pc_update_values": (c_int, [vp, vp]),
            "owtk_pc_numeric_updates": (c_uint64, [vp]),
            "owtk_ilu_factors": (c_int, [vp, u64p, vp, vp, vp, vp]),
            "owtk_pc_levels": (c_int, [vp, vp, vp, u64p, u64p]),
            "owtk_rcm_order": (c_int, [sz, sz, vp, vp, vp]),
            "owtk_hilbert_order": (c_int, [sz, vp, vp]),
            "owtk_inverse_permutation": (c_int, [sz, vp, vp]),
            "owtk_level_sets": (c_int, [sz, vp, vp, vp, vp, u64p, u64p]),
            "owtk_default_options": (None, [POINTER(SolverOptions)]),
            "owtk_workspace_create": (c_int, [vp, POINTER(vp)]),
            "owtk_workspace_destroy": (c_int, [vp]),
            "owtk_workspace_allocation_epochs": (c_uint64, [vp]),
            "owtk_workspace_vector": (vp, [vp, sz]),
            "owtk_solve": (c_int, [c_int, vp, vp, vp, vp, POINTER(SolverOptions), vp, POINTER(SolverResult)]),
            "owtk_solve_host": (c_int, [c_int, vp, vp, vp, vp, POINTER(SolverOptions), vp, POINTER(SolverResult)]),
            "owtk_batch_create": (c_int, [vp, sz, POINTER(BatchSystem), POINTER(vp)]),
            "owtk_batch_destroy": (c_int, [vp]),
            "owtk_batch_layout": (c_int, [vp, POINTER(sz), vp]),
            "owtk_batch_config": (c_int, [vp, POINTER(ctypes.c_uint32), POINTER(ctypes.c_uint32)]),
            "owtk_batch_set_config": (c_int, [vp, ctypes.c_uint32, sz, ctypes.c_uint32]),
            "owtk_batch_autotune": (c_int, [vp, POINTER(SolverOptions), POINTER(ctypes.c_uint32),
                                            POINTER(ctypes.c_uint32)]),
            "owtk_batch_use_graph": (c_int, [vp, c_int]),
            "owtk_batch_graph_counts": (c_int, [vp, u64p, u64p]),
            "owtk_batch_solve": (c_int, [vp, vp, vp, POINTER(SolverOptions), POINTER(SolverResult)]),
            "owtk_batch_solve_host": (c_int, [vp, vp, vp, POINTER(SolverOptions), POINTER(SolverResult)]),
            "owtk_bf16_gemm_nt": (c_int, [vp, sz, sz, sz, vp, vp, vp]),
            "owtk_solve_specwave": (c_int, [c_int, vp, vp, vp, POINTER(SolverOptions), vp, POINTER(SolverResult)]),
            "owtk_debug_unpublished_dependency": (c_int, [vp, ctypes.c_uint32]),
            "owtk_pc_sweep_schedule": (c_int, [vp, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]),
            "owtk_pc_chain_schedule": (c_int, [vp, POINTER(c_int32)]),
            "owtk_pc_lockstep_schedule": (c_int, [vp, POINTER(c_int32), POINTER(c_int32), POINTER(c_int32)]),
            "owtk_permutation_create": (c_int, [vp, sz, vp, POINTER(vp)]),
            "owtk_permutation_destroy": (c_int, [vp]),
            "owtk_vector_permute": (c_int, [vp, vp, vp, c_int]),
            "owtk_bsr_create_permuted_split": (c_int, [vp, c_int, sz, vp, vp, vp, vp, POINTER(vp)]),
            "owtk_bsr_update_permuted_split": (c_int, [vp, vp, vp]),
            "owtk_dot_ex": (c_int, [vp, vp, c_int, POINTER(c_double), POINTER(c_double)]),
            "owtk_norm_ex": (c_int, [vp, c_int, POINTER(c_double)]),
            "owtk_arnoldi_snapshot_create": (c_int, [vp, POINTER(vp)]),
            "owtk_arnoldi_snapshot_destroy": (c_int, [vp]),
            "owtk_arnoldi_snapshot_clear": (c_int, [vp]),
            "owtk_arnoldi_snapshot_columns": (sz, [vp]),
            "owtk_arnoldi_snapshot_h": (c_int, [vp, sz, sz, POINTER(c_double)]),
            "owtk_arnoldi_snapshot_basis": (c_int, [vp, sz, POINTER(vp)]),
            "owtk_solve_ex": (c_int, [c_int, vp, vp, vp, vp, POINTER(SolverOptions), vp, POINTER(SolveExtras),
                                      POINTER(SolverResult)]),
            "owtk_solve_host_ex": (c_int, [c_int, vp, vp, vp, vp, POINTER(SolverOptions), vp, POINTER(SolveExtras),
                                           POINTER(SolverResult)]),
            "owtk_solve_specwave_ex": (c_int, [c_int, vp, vp, vp, POINTER(SolverOptions), vp, c_int,
                                               POINTER(SolverResult)]),
            "owtk_callback_operator_create": (c_int, [vp, c_int, sz, sz, sz, HOST_APPLY, vp, POINTER(vp)]),
            "owtk_pc_create_callback": (c_int, [vp, c_int, sz, sz, sz, HOST_APPLY, vp, POINTER(vp)]),
            "owtk_learned_create": (c_int, [vp, c_uint64, POINTER(vp)]),
            "owtk_learned_destroy": (c_int, [vp]),
            "owtk_learned_update_matrix": (c_int, [vp, vp]),
            "owtk_learned_parameter_count": (sz, []),
            "owtk_learned_uses_tma": (c_int, [vp]),
            "owtk_learned_get_parameters": (c_int, [vp, vp, sz]),
            "owtk_learned_set_parameters": (c_int, [vp, vp, sz]),
            "owtk_learned_get_adam_state": (c_int, [vp, vp, vp, sz, u64p]),
            "owtk_learned_set_adam_state": (c_int, [vp, vp, vp, sz, c_uint64]),
            "owtk_learned_apply": (c_int, [vp, vp, vp]),
            "owtk_learned_stage_times": (c_int, [vp, vp, vp, ctypes.c_uint32, POINTER(c_double)]),
            "owtk_learned_loss_grad": (c_int, [vp, vp, vp, POINTER(c_double), vp]),
            "owtk_learned_adam_step": (c_int, [vp, c_double]),
            "owtk_learned_set_loss_weights": (c_int, [vp, c_double, c_double]),
            "owtk_pc_create_learned": (c_int, [vp, vp, POINTER(vp)]),
            "owtk_pc_learned_counts": (c_int, [vp, u64p, u64p]),
            "owtk_pc_learned_set_correction": (c_int, [vp, ctypes.c_uint32, c_double]),
        }
        for name, (res, args) in sig.items():
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def check(code: int):
    if code != 0:
        raise OwtkError(code, lib().owtk_last_error().decode())


def _ptr(a: np.ndarray):
    return a.ctypes.data_as(c_void_p)


def _u64(a) -> np.ndarray:
    return np.ascontiguousarray(np.asarray(a, dtype=np.uint64))


def default_options(**kw) -> SolverOptions:
    o = SolverOptions()
    lib().owtk_default_options(ctypes.byref(o))
    for k, v in kw.items():
        if not hasattr(o, k):
            raise KeyError(k)
        setattr(o, k, v)
    return o


class Context:
    def __init__(self, device: int = 0):
        h = c_void_p()
        check(lib().owtk_context_create(device, ctypes.byref(h)))
        self.h = h

    def synchronize(self):
        check(lib().owtk_context_synchronize(self.h))

    @property
    def stream(self) -> int:
        return lib().owtk_context_stream(self.h) or 0

    @property
    def kernel_launches(self) -> int:
        return lib().owtk_context_kernel_launches(self.h)

    def close(self):
        if self.h:
            lib().owtk_context_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _dtype_code(dt) -> int:
    return F64 if np.dtype(dt) == np.float64 else F32


def _np_dtype(code: int):
    return np.float64 if code == F64 else np.float32


class Vector:
    def __init__(self, ctx: Context, owned: int, ghost: int, bs: int, dtype=np.float64, handle=None,
                 owner=True):
        self.ctx, self.owned, self.ghost, self.bs = ctx, owned, ghost, bs
        self.dtype = np.dtype(dtype)
        self.owner = owner
        if handle is None:
            h = c_void_p()
            check(lib().owtk_vector_create(ctx.h, _dtype_code(dtype), owned, ghost, bs, ctypes.byref(h)))
            handle = h
        self.h = handle

    @classmethod
    def view(cls, ctx, owned, ghost, bs, device_ptr: int, count: int, dtype=np.float64):
        h = c_void_p()
        check(lib().owtk_vector_view(ctx.h, _dtype_code(dtype), owned, ghost, bs, c_void_p(device_ptr),
                                     count, ctypes.byref(h)))
        return cls(ctx, owned, ghost, bs, dtype, handle=h)

    @property
    def size(self) -> int:
        return (self.owned + self.ghost) * self.bs

    @property
    def data_ptr(self) -> int:
        return lib().owtk_vector_data(self.h) or 0

    def upload(self, a: np.ndarray):
        a = np.ascontiguousarray(a, dtype=self.dtype)
        check(lib().owtk_vector_upload(self.h, _ptr(a), a.size))
        return self

    def download(self, count: int | None = None) -> np.ndarray:
        count = self.size if count is None else count
        out = np.empty(count, dtype=self.dtype)
        check(lib().owtk_vector_download(self.h, _ptr(out), count))
        return out

    def fill(self, value: float, owned_only: bool = False):
        check(lib().owtk_vector_fill(self.h, value, 1 if owned_only else 0))

    def close(self):
        if self.h is not None and self.owner:
            lib().owtk_vector_destroy(self.h)
        self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dot(a: Vector, b: Vector) -> float:
    r = c_double()
    check(lib().owtk_dot(a.h, b.h, ctypes.byref(r)))
    return r.value


def norm(a: Vector) -> float:
    r = c_double()
    check(lib().owtk_norm(a.h, ctypes.byref(r)))
    return r.value


def dot_batch(w: Vector, basis: list[Vector]) -> np.ndarray:
    arr = (c_void_p * max(1, len(basis)))(*[v.h for v in basis])
    out = (c_double * (len(basis) + 1))()
    check(lib().owtk_dot_batch(w.h, arr, len(basis), out))
    return np.array(out[:])


def axpy(alpha: float, x: Vector, y: Vector):
    check(lib().owtk_axpy(alpha, x.h, y.h))


def scale(alpha: float, x: Vector):
    check(lib().owtk_scale(alpha, x.h))


def copy_owned(src: Vector, dst: Vector):
    check(lib().owtk_copy_owned(src.h, dst.h))


def assign_linear_combination(out: Vector, a: float, x: Vector, b: float, y: Vector):
    check(lib().owtk_assign_linear_combination(out.h, a, x.h, b, y.h))


class Matrix:
    """Device matrix: kind 'bsr', 'split' (borrowed device coefficients) or 'dense'."""

    def __init__(self, ctx: Context, kind: str, owned: int, ghost: int, bs: int, rowptr, cols,
                 values=None, diag_ptr: int = 0, off_ptr: int = 0, dtype=np.float64):
        self.ctx, self.kind, self.owned, self.ghost, self.bs = ctx, kind, owned, ghost, bs
        self.dtype = np.dtype(dtype)
        rp, ci = _u64(rowptr), _u64(cols)
        if ci.size == 0:
            ci = np.zeros(1, dtype=np.uint64)
        h = c_void_p()
        code = _dtype_code(dtype)
        if kind == "bsr":
            v = np.ascontiguousarray(values, dtype=self.dtype)
            check(lib().owtk_bsr_create(ctx.h, code, owned, ghost, bs, _ptr(rp), _ptr(ci), _ptr(v), ctypes.byref(h)))
        elif kind == "dense":
            v = np.ascontiguousarray(values, dtype=self.dtype)
            check(lib().owtk_dense_bsr_create(ctx.h, code, owned, ghost, bs, _ptr(rp), _ptr(ci), _ptr(v),
                                              ctypes.byref(h)))
        elif kind == "split":
            check(lib().owtk_split_view_create(ctx.h, code, owned, ghost, bs, _ptr(rp), _ptr(ci),
                                               c_void_p(diag_ptr), c_void_p(off_ptr), ctypes.byref(h)))
        else:
            raise ValueError(kind)
        self.h = h

    def update_values(self, values):
        v = np.ascontiguousarray(values, dtype=self.dtype)
        check(lib().owtk_bsr_update_values(self.h, _ptr(v)))

    def diagonal(self) -> np.ndarray:
        out = np.empty(self.owned * self.bs, dtype=self.dtype)
        check(lib().owtk_matrix_diagonal(self.h, _ptr(out)))
        return out

    def apply(self, x: Vector, y: Vector):
        check(lib().owtk_spmv(self.h, x.h, y.h))

    def apply_rows(self, x: Vector, y: Vector, rows):
        """The listed rows of y = A x, as apply computes them; other rows untouched."""
        r = np.ascontiguousarray(rows, dtype=np.uint64)
        check(lib().owtk_spmv_rows(self.h, x.h, y.h, _ptr(r) if r.size else None, r.size))

    def close(self):
        if self.h is not None:
            lib().owtk_matrix_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Preconditioner:
    """storage F32/BF16: factors kept in that precision (FP32 applies);
    mixed_inner >= 0: FP64 wrapper around an FP32 inner solve of that many
    GMRES steps (0: one factor apply)."""

    def __init__(self, matrix: Matrix, kind: int, parameter: float = 0.0, storage: int = F64,
                 mixed_inner: int | None = None):
        h = c_void_p()
        if mixed_inner is not None:
            check(lib().owtk_pc_create_mixed(matrix.h, kind, parameter, storage, mixed_inner, ctypes.byref(h)))
        elif storage != F64:
            check(lib().owtk_pc_create_stored(matrix.h, kind, parameter, storage, ctypes.byref(h)))
        else:
            check(lib().owtk_pc_create(matrix.h, kind, parameter, ctypes.byref(h)))
        self.h, self.matrix, self.kind = h, matrix, kind

    def apply(self, x: Vector, y: Vector):
        check(lib().owtk_pc_apply(self.h, x.h, y.h))

    def update_values(self, matrix: Matrix | None = None):
        check(lib().owtk_pc_update_values(self.h, (matrix or self.matrix).h))

    @property
    def numeric_updates(self) -> int:
        return lib().owtk_pc_numeric_updates(self.h)

    def ilu_factors(self):
        n = c_uint64()
        check(lib().owtk_ilu_factors(self.h, ctypes.byref(n), None, None, None, None))
        m = self.matrix
        per = m.bs * m.bs if self.kind == PC_BLOCK_ILU else m.bs
        rp = np.empty(m.owned + 1, dtype=np.uint64)
        ci = np.empty(max(1, n.value), dtype=np.uint64)
        vals = np.empty(n.value * per, dtype=m.dtype)
        inv = np.empty(m.owned * per, dtype=m.dtype)
        check(lib().owtk_ilu_factors(self.h, ctypes.byref(n), _ptr(rp), _ptr(ci), _ptr(vals), _ptr(inv)))
        return rp, ci[:n.value], vals, inv

    def sweep_schedule(self):
        """(cluster CTAs or 0, levels per epoch, ring rows per CTA)."""
        c, k, r = c_int32(), c_int32(), c_int32()
        check(lib().owtk_pc_sweep_schedule(self.h, ctypes.byref(c), ctypes.byref(k), ctypes.byref(r)))
        return c.value, k.value, r.value

    def lockstep_schedule(self):
        """(cluster CTAs or 0, forward levels, backward levels) of the lockstep sweep."""
        c, lo, up = c_int32(), c_int32(), c_int32()
        check(lib().owtk_pc_lockstep_schedule(self.h, ctypes.byref(c), ctypes.byref(lo), ctypes.byref(up)))
        return c.value, lo.value, up.value

    def chain_windows(self):
        """Row windows of the chain sweep (0: the applies take another sweep)."""
        w = c_int32()
        check(lib().owtk_pc_chain_schedule(self.h, ctypes.byref(w)))
        return w.value

    def levels(self):
        m = self.matrix
        lo = np.empty(m.owned, dtype=np.int32)
        up = np.empty(m.owned, dtype=np.int32)
        dl, du = c_uint64(), c_uint64()
        check(lib().owtk_pc_levels(self.h, _ptr(lo), _ptr(up), ctypes.byref(dl), ctypes.byref(du)))
        return lo, up, dl.value, du.value

    def close(self):
        if self.h is not None:
            lib().owtk_pc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Workspace:
    def __init__(self, ctx: Context):
        h = c_void_p()
        check(lib().owtk_workspace_create(ctx.h, ctypes.byref(h)))
        self.h, self.ctx = h, ctx

    @property
    def allocation_epochs(self) -> int:
        return lib().owtk_workspace_allocation_epochs(self.h)

    def vector_data(self, index: int, count: int, dtype=np.float64) -> np.ndarray:
        vh = lib().owtk_workspace_vector(self.h, index)
        if not vh:
            raise IndexError(index)
        out = np.empty(count, dtype=dtype)
        check(lib().owtk_vector_download(c_void_p(vh), _ptr(out), count))
        return out

    def close(self):
        if self.h is not None:
            lib().owtk_workspace_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve(kind: int, matrix: Matrix, pc: Preconditioner | None, rhs: Vector, x: Vector,
          options: SolverOptions | None = None, workspace: Workspace | None = None) -> SolverResult:
    o = options or default_options()
    r = SolverResult()
    check(lib().owtk_solve(kind, matrix.h, pc.h if pc else None, rhs.h, x.h, ctypes.byref(o),
                           workspace.h if workspace else None, ctypes.byref(r)))
    return r


def solve_specwave(solver_id: int, matrix: Matrix, rhs: Vector, x: Vector, options: SolverOptions | None = None,
                   workspace: Workspace | None = None, reduction: str = "serial") -> SolverResult:
    """solve_specwave_native: a legacy SpecWave solver id (owtk_solve_specwave_ex)."""
    o = options or default_options()
    r = SolverResult()
    check(lib().owtk_solve_specwave_ex(solver_id, matrix.h, rhs.h, x.h, ctypes.byref(o),
                                       workspace.h if workspace else None, REDUCTION[reduction], ctypes.byref(r)))
    return r


class Permutation:
    """owtk_permutation_*: a node permutation applied on the device."""

    def __init__(self, ctx: Context, new_to_old):
        p = _u64(new_to_old)
        h = c_void_p()
        check(lib().owtk_permutation_create(ctx.h, p.size, _ptr(p), ctypes.byref(h)))
        self.h, self.ctx, self.n = h, ctx, p.size

    def apply(self, src: Vector, dst: Vector, inverse: bool = False):
        check(lib().owtk_vector_permute(self.h, src.h, dst.h, 1 if inverse else 0))

    def permuted_split_matrix(self, bs: int, off_rowptr, off_cols, diag: Vector, off: Vector, dtype=np.float64):
        """P A P^T from a split layout whose coefficient arrays are device vectors."""
        rp, ci = _u64(off_rowptr), _u64(off_cols)
        if ci.size == 0:
            ci = np.zeros(1, dtype=np.uint64)
        h = c_void_p()
        check(lib().owtk_bsr_create_permuted_split(self.h, _dtype_code(dtype), bs, _ptr(rp), _ptr(ci),
                                                   c_void_p(diag.data_ptr), c_void_p(off.data_ptr), ctypes.byref(h)))
        m = Matrix.__new__(Matrix)
        m.ctx, m.kind, m.owned, m.ghost, m.bs, m.dtype, m.h = self.ctx, "bsr", self.n, 0, bs, np.dtype(dtype), h
        return m

    def __del__(self):
        try:
            if self.h is not None:
                lib().owtk_permutation_destroy(self.h)
                self.h = None
        except Exception:
            pass


def update_permuted_split(matrix: Matrix, diag: Vector, off: Vector):
    check(lib().owtk_bsr_update_permuted_split(matrix.h, c_void_p(diag.data_ptr), c_void_p(off.data_ptr)))


class ArnoldiSnapshot:
    """owtk_arnoldi_snapshot_*: the last unrotated Arnoldi relation of FGMRES."""

    def __init__(self, ctx: Context):
        h = c_void_p()
        check(lib().owtk_arnoldi_snapshot_create(ctx.h, ctypes.byref(h)))
        self.h, self.ctx = h, ctx

    @property
    def columns(self) -> int:
        return int(lib().owtk_arnoldi_snapshot_columns(self.h))

    def h_entry(self, row: int, column: int) -> float:
        v = c_double()
        check(lib().owtk_arnoldi_snapshot_h(self.h, row, column, ctypes.byref(v)))
        return v.value

    def basis(self, column: int, owned: int, ghost: int, bs: int, dtype=np.float64) -> np.ndarray:
        v = c_void_p()
        check(lib().owtk_arnoldi_snapshot_basis(self.h, column, ctypes.byref(v)))
        out = np.empty((owned + ghost) * bs, dtype=dtype)
        check(lib().owtk_vector_download(v, _ptr(out), out.size))
        return out

    def clear(self):
        check(lib().owtk_arnoldi_snapshot_clear(self.h))

    def __del__(self):
        try:
            if self.h is not None:
                lib().owtk_arnoldi_snapshot_destroy(self.h)
                self.h = None
        except Exception:
            pass


def solve_ex(kind: int, matrix, pc, rhs: Vector, x: Vector, options: SolverOptions | None = None,
             workspace: Workspace | None = None, reduction: str = "serial", convergence_test=None,
             snapshot: ArnoldiSnapshot | None = None) -> SolverResult:
    """owtk_solve_ex.  convergence_test(iteration, candidate ndarray) -> bool."""
    o = options or default_options()
    r = SolverResult()
    ex = SolveExtras()
    ex.reduction = REDUCTION[reduction]
    errors = []
    if convergence_test is not None:
        dtype = rhs.dtype

        def _test(_user, iteration, candidate, count):
            try:
                arr = np.ctypeslib.as_array(ctypes.cast(candidate, POINTER(ctypes.c_double if dtype == np.float64
                                                                             else ctypes.c_float)), (count,))
                return 1 if convergence_test(int(iteration), arr.copy()) else 0
            except Exception as exc:   # kept and re-raised after the call
                errors.append(exc)
                return -1

        cb = CONVERGENCE_TEST(_test)
        ex.convergence_test = cb
    ex.arnoldi_snapshot = snapshot.h if snapshot is not None else None
    code = lib().owtk_solve_ex(kind, matrix.h, pc.h if pc else None, rhs.h, x.h, ctypes.byref(o),
                               workspace.h if workspace else None, ctypes.byref(ex), ctypes.byref(r))
    if errors:
        raise errors[0]
    check(code)
    return r


def dot_ex(a: Vector, b: Vector, reduction: str = "serial"):
    """(result, low) of owtk_dot_ex."""
    hi, lo = c_double(), c_double()
    check(lib().owtk_dot_ex(a.h, b.h, REDUCTION[reduction], ctypes.byref(hi), ctypes.byref(lo)))
    return hi.value, lo.value


def norm_ex(a: Vector, reduction: str = "serial") -> float:
    r = c_double()
    check(lib().owtk_norm_ex(a.h, REDUCTION[reduction], ctypes.byref(r)))
    return r.value


class _HostApply:
    """A Python function fn(in ndarray, out ndarray) behind HOST_APPLY."""

    def __init__(self, fn, dtype):
        self.fn, self.errors = fn, []
        ct = ctypes.c_double if np.dtype(dtype) == np.float64 else ctypes.c_float

        def _call(_user, pin, pout, count):
            try:
                vin = np.ctypeslib.as_array(ctypes.cast(pin, POINTER(ct)), (count,))
                vout = np.ctypeslib.as_array(ctypes.cast(pout, POINTER(ct)), (count,))
                fn(vin, vout)
                return 0
            except Exception as exc:
                self.errors.append(exc)
                return 1

        self.cb = HOST_APPLY(_call)


class CallbackOperator:
    """owtk_callback_operator_create: an application operator fn(in, out) on
    host arrays ((owned + ghost) * bs values), usable wherever a Matrix is."""

    def __init__(self, ctx: Context, owned: int, ghost: int, bs: int, fn, dtype=np.float64):
        self.ctx, self.owned, self.ghost, self.bs, self.dtype = ctx, owned, ghost, bs, np.dtype(dtype)
        self._apply = _HostApply(fn, dtype)
        h = c_void_p()
        check(lib().owtk_callback_operator_create(ctx.h, _dtype_code(dtype), owned, ghost, bs, self._apply.cb, None,
                                                  ctypes.byref(h)))
        self.h = h

    def apply(self, x: Vector, y: Vector):
        check(lib().owtk_spmv(self.h, x.h, y.h))

    def __del__(self):
        try:
            if self.h is not None:
                lib().owtk_matrix_destroy(self.h)
                self.h = None
        except Exception:
            pass


class CallbackPreconditioner:
    """owtk_pc_create_callback: an application preconditioner fn(in, out)."""

    def __init__(self, ctx: Context, owned: int, ghost: int, bs: int, fn, dtype=np.float64):
        self._apply = _HostApply(fn, dtype)
        h = c_void_p()
        check(lib().owtk_pc_create_callback(ctx.h, _dtype_code(dtype), owned, ghost, bs, self._apply.cb, None,
                                            ctypes.byref(h)))
        self.h = h
        self.kind = 8

    def apply(self, x: Vector, y: Vector):
        check(lib().owtk_pc_apply(self.h, x.h, y.h))

    def __del__(self):
        try:
            if self.h is not None:
                lib().owtk_pc_destroy(self.h)
                self.h = None
        except Exception:
            pass


def solve_host(kind: int, matrix: Matrix, pc: Preconditioner | None, rhs_ptr: int, x_ptr: int,
               options: SolverOptions | None = None, workspace: Workspace | None = None) -> SolverResult:
    o = options or default_options()
    r = SolverResult()
    check(lib().owtk_solve_host(kind, matrix.h, pc.h if pc else None, c_void_p(rhs_ptr), c_void_p(x_ptr),
                                ctypes.byref(o), workspace.h if workspace else None, ctypes.byref(r)))
    return r


# ---------------------------------------------------------------- tensor cores
def bf16_gemm_nt(ctx: Context, a_ptr: int, b_ptr: int, d_ptr: int, m: int, n: int, k: int):
    """D (m x n FP32) = A (m x k BF16) * B (n x k BF16)^T on the tensor cores;
    device pointers (e.g. torch tensors' data_ptr())."""
    check(lib().owtk_bf16_gemm_nt(ctx.h, m, n, k, c_void_p(a_ptr), c_void_p(b_ptr), c_void_p(d_ptr)))


# ---------------------------------------------------------------- learned preconditioner
class Learned:
    """The message-passing network on a matrix's graph (owtk_learned_* in
    include/owtk.h): forward, loss/gradient, Adam, and its use as a
    preconditioner with a fallback."""

    def __init__(self, matrix: Matrix, seed: int = 0):
        self.matrix = matrix
        self.h = None
        h = c_void_p()
        check(lib().owtk_learned_create(matrix.h, seed, ctypes.byref(h)))
        self.h = h

    @property
    def uses_tma(self) -> bool:
        return bool(lib().owtk_learned_uses_tma(self.h))

    @staticmethod
    def parameter_count() -> int:
        return int(lib().owtk_learned_parameter_count())

    def update_matrix(self, matrix: Matrix):
        check(lib().owtk_learned_update_matrix(self.h, matrix.h))
        self.matrix = matrix

    def parameters(self) -> np.ndarray:
        out = np.empty(self.parameter_count(), dtype=np.float32)
        check(lib().owtk_learned_get_parameters(self.h, _ptr(out), out.size))
        return out

    def set_parameters(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        check(lib().owtk_learned_set_parameters(self.h, _ptr(p), p.size))

    def adam_state(self):
        """(first moment, second moment, step) of the Adam optimiser."""
        m = np.empty(self.parameter_count(), dtype=np.float32)
        v = np.empty_like(m)
        t = c_uint64()
        check(lib().owtk_learned_get_adam_state(self.h, _ptr(m), _ptr(v), m.size, ctypes.byref(t)))
        return m, v, int(t.value)

    def set_adam_state(self, m, v, step: int):
        m = np.ascontiguousarray(m, dtype=np.float32)
        v = np.ascontiguousarray(v, dtype=np.float32)
        check(lib().owtk_learned_set_adam_state(self.h, _ptr(m), _ptr(v), m.size, int(step)))

    def apply(self, x: Vector, y: Vector):
        check(lib().owtk_learned_apply(self.h, x.h, y.h))

    def stage_times(self, x: Vector, y: Vector, repetitions: int = 10) -> dict:
        """Mean milliseconds per stage of y = M(x) (CUDA events on the stream)."""
        ms = (c_double * 5)()
        check(lib().owtk_learned_stage_times(self.h, x.h, y.h, repetitions, ms))
        return {"norms_encoder": ms[0], "layer": ms[1], "last_layer_decoder": ms[2], "application": ms[3],
                "encoder_first_layer": ms[4]}

    def loss_grad(self, r: Vector, e: Vector, want_grads: bool = False):
        loss = c_double()
        g = np.empty(self.parameter_count(), dtype=np.float32) if want_grads else None
        check(lib().owtk_learned_loss_grad(self.h, r.h, e.h, ctypes.byref(loss), _ptr(g) if g is not None else None))
        return (loss.value, g) if want_grads else loss.value

    def adam_step(self, learning_rate: float):
        check(lib().owtk_learned_adam_step(self.h, learning_rate))

    def set_loss_weights(self, error_weight: float = 1.0, residual_weight: float = 1.0):
        check(lib().owtk_learned_set_loss_weights(self.h, error_weight, residual_weight))

    def close(self):
        if self.h is not None:
            lib().owtk_learned_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class LearnedPreconditioner(Preconditioner):
    """owtk_pc_create_learned: the network judged by the FP64 residual, the
    fallback (e.g. an ILU(0) Preconditioner) taking the steps it fails."""

    def __init__(self, net: Learned, fallback: "Preconditioner | None" = None):
        self.matrix = net.matrix
        self.net = net
        self.fallback = fallback
        self.kind = PC_LEARNED
        self.h = None
        h = c_void_p()
        check(lib().owtk_pc_create_learned(net.h, fallback.h if fallback else None, ctypes.byref(h)))
        self.h = h

    def counts(self):
        a, f = c_uint64(), c_uint64()
        check(lib().owtk_pc_learned_counts(self.h, ctypes.byref(a), ctypes.byref(f)))
        return a.value, f.value

    def set_correction(self, steps: int, omega: float = 1.0):
        """Damped Jacobi corrections z += omega D^-1 (v - A z) after each
        accepted network step."""
        check(lib().owtk_pc_learned_set_correction(self.h, steps, omega))


# ---------------------------------------------------------------- batching
class Batch:
    """Many independent FP64 component-diagonal systems solved together by
    BiCGSTAB + Jacobi in one persistent graph-captured launch
    (owtk_batch_* in include/owtk.h).  `systems` holds objects with owned, bs,
    rowptr, cols, vals (a BlockSystem) or (owned, bs, rowptr, cols, vals) tuples."""

    MAX_BS = 32

    def __init__(self, ctx: Context, systems):
        self.ctx = ctx
        self.h = None
        keep, descs = [], []
        for y in systems:
            owned, bs, rp, ci, vals = ((y.owned, y.bs, y.rowptr, y.cols, y.vals) if hasattr(y, "owned") else y)
            rp, ci = _u64(rp), _u64(ci)
            vals = np.ascontiguousarray(vals, dtype=np.float64)
            keep += [rp, ci, vals]
            descs.append(BatchSystem(owned, bs, _ptr(rp), _ptr(ci), _ptr(vals)))
        arr = (BatchSystem * len(descs))(*descs)
        h = c_void_p()
        check(lib().owtk_batch_create(ctx.h, len(descs), arr, ctypes.byref(h)))
        self.h = h
        self.count = len(descs)
        self.unknowns, self.offsets = self.layout()

    def layout(self):
        n = c_size_t()
        off = np.empty(self.count + 1, dtype=np.uint64)
        check(lib().owtk_batch_layout(self.h, ctypes.byref(n), _ptr(off)))
        return n.value, off.astype(np.int64)

    def config(self):
        bps = ctypes.c_uint32()
        vpw = (ctypes.c_uint32 * (self.MAX_BS + 1))()
        check(lib().owtk_batch_config(self.h, ctypes.byref(bps), vpw))
        return bps.value, list(vpw)

    def set_config(self, blocks_per_sm: int = 0, bs: int = 0, vertices_per_warp: int = 0):
        check(lib().owtk_batch_set_config(self.h, blocks_per_sm, bs, vertices_per_warp))

    def autotune(self, options: SolverOptions | None = None):
        bps = ctypes.c_uint32()
        vpw = (ctypes.c_uint32 * (self.MAX_BS + 1))()
        check(lib().owtk_batch_autotune(self.h, ctypes.byref(options) if options else None, ctypes.byref(bps), vpw))
        return bps.value, list(vpw)

    def use_graph(self, enable: bool):
        check(lib().owtk_batch_use_graph(self.h, int(enable)))

    def graph_counts(self):
        c, l = c_uint64(), c_uint64()
        check(lib().owtk_batch_graph_counts(self.h, ctypes.byref(c), ctypes.byref(l)))
        return c.value, l.value

    def solve(self, rhs: Vector, x: Vector, options: SolverOptions | None = None) -> list:
        o = options or default_options()
        res = (SolverResult * self.count)()
        check(lib().owtk_batch_solve(self.h, c_void_p(rhs.data_ptr), c_void_p(x.data_ptr), ctypes.byref(o), res))
        return list(res)

    def solve_host(self, rhs_ptr: int, x_ptr: int, options: SolverOptions | None = None) -> list:
        o = options or default_options()
        res = (SolverResult * self.count)()
        check(lib().owtk_batch_solve_host(self.h, c_void_p(rhs_ptr), c_void_p(x_ptr), ctypes.byref(o), res))
        return list(res)

    def close(self):
        if self.h is not None:
            lib().owtk_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


# ---------------------------------------------------------------- host setup
def rcm_order(owned: int, rowptr, cols, ghost: int = 0) -> np.ndarray:
    rp, ci = _u64(rowptr), _u64(cols)
    out = np.empty(owned, dtype=np.uint64)
    check(lib().owtk_rcm_order(owned, ghost, _ptr(rp), _ptr(ci), _ptr(out)))
    return out.astype(np.int64)


def hilbert_order(xy: np.ndarray) -> np.ndarray:
    xy = np.ascontiguousarray(xy, dtype=np.float64)
    out = np.empty(xy.shape[0], dtype=np.uint64)
    check(lib().owtk_hilbert_order(xy.shape[0], _ptr(xy), _ptr(out)))
    return out.astype(np.int64)


def inverse_permutation(p) -> np.ndarray:
    p = _u64(p)
    out = np.empty(p.size, dtype=np.uint64)
    check(lib().owtk_inverse_permutation(p.size, _ptr(p), _ptr(out)))
    return out.astype(np.int64)


def level_sets(owned: int, rowptr, cols):
    rp, ci = _u64(rowptr), _u64(cols)
    lo = np.empty(owned, dtype=np.int32)
    up = np.empty(owned, dtype=np.int32)
    dl, du = c_uint64(), c_uint64()
    check(lib().owtk_level_sets(owned, _ptr(rp), _ptr(ci), _ptr(lo), _ptr(up), ctypes.byref(dl), ctypes.byref(du)))
    return lo, up, dl.value, du.value
