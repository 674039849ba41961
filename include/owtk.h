/*
 * owtk.h — C ABI of the B200 (sm_100a) single-rank OWT-Krylov solve path.
 *
 * Plain pointers, sizes and opaque handles; no C++ or CUDA types in any
 * signature.  Every call returns an owtk_status; owtk_last_error() gives the
 * message of the last failure on the calling thread.  The status codes map
 * one-to-one onto the exceptions of the reference's header-only API:
 *   std::invalid_argument -> OWTK_ERR_INVALID_ARGUMENT
 *   std::runtime_error("zero pivot in ILU(0)") -> OWTK_ERR_ZERO_PIVOT
 *   std::out_of_range     -> OWTK_ERR_OUT_OF_RANGE
 * Solver failures are not errors: they are reported in owtk_solver_result,
 * exactly like the reference's SolverResult (core.hpp:118-146).
 *
 * Reference anchors (file:line) are into include/owt/krylov/ of OWT-Krylov.
 * Vectors, matrices and preconditioners live in device memory (HBM) and
 * every operation is enqueued on the context's CUDA stream; *_host entry
 * points take host buffers and include the host<->device copies.
 */
#ifndef OWTK_H
#define OWTK_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum owtk_status {
    OWTK_OK = 0,
    OWTK_ERR_INVALID_ARGUMENT = 1,
    OWTK_ERR_ZERO_PIVOT = 2,
    OWTK_ERR_OUT_OF_RANGE = 3,
    OWTK_ERR_CUDA = 4,
    OWTK_ERR_TIMEOUT = 5,     /* a bounded device-side wait gave up */
    OWTK_ERR_NO_DEVICE = 6,
    OWTK_ERR_RUNTIME = 7
} owtk_status;

/* OWTK_BF16 is a factor-storage type only (owtk_pc_create_stored/_mixed). */
typedef enum owtk_dtype { OWTK_F64 = 0, OWTK_F32 = 1, OWTK_BF16 = 2 } owtk_dtype;

typedef struct owtk_context owtk_context;
typedef struct owtk_vector owtk_vector;
typedef struct owtk_matrix owtk_matrix;
typedef struct owtk_preconditioner owtk_preconditioner;
typedef struct owtk_workspace owtk_workspace;

const char* owtk_last_error(void);
int owtk_abi_version(void);

/* ---- context: one device, one stream ------------------------------------ */
owtk_status owtk_context_create(int device, owtk_context** out);
owtk_status owtk_context_destroy(owtk_context* ctx);
owtk_status owtk_context_synchronize(owtk_context* ctx);
/* The cudaStream_t every call of this context is enqueued on. */
void* owtk_context_stream(owtk_context* ctx);
/* Kernels this library has launched on the context so far. */
uint64_t owtk_context_kernel_launches(owtk_context* ctx);

/* ---- BlockVector<T> (core.hpp:197-395): owned nodes then ghost nodes,
 *      bs contiguous values per node.  *_view wraps caller device memory
 *      without copying (core.hpp:223-230).  Invalid layouts are rejected as
 *      in core.hpp:371-377. -------------------------------------------------- */
owtk_status owtk_vector_create(owtk_context* ctx, owtk_dtype dtype, size_t owned_nodes,
                               size_t ghost_nodes, size_t block_size, owtk_vector** out);
owtk_status owtk_vector_view(owtk_context* ctx, owtk_dtype dtype, size_t owned_nodes,
                             size_t ghost_nodes, size_t block_size, void* device_values,
                             size_t value_count, owtk_vector** out);
owtk_status owtk_vector_destroy(owtk_vector* v);
void* owtk_vector_data(owtk_vector* v);
/* Copy `count` values from/to the start of the vector (host memory). */
owtk_status owtk_vector_upload(owtk_vector* v, const void* host, size_t count);
owtk_status owtk_vector_download(owtk_vector* v, void* host, size_t count);
/* fill_owned / fill (core.hpp:339-340). */
owtk_status owtk_vector_fill(owtk_vector* v, double value, int owned_only);

/* ---- owned-only BLAS-1 (core.hpp:562-601, simd.hpp:15-202) --------------- */
owtk_status owtk_copy_owned(owtk_vector* source, owtk_vector* destination);
owtk_status owtk_axpy(double alpha, owtk_vector* x, owtk_vector* y);
owtk_status owtk_scale(double alpha, owtk_vector* x);
owtk_status owtk_assign_linear_combination(owtk_vector* out, double alpha, owtk_vector* x,
                                           double beta, owtk_vector* y);
/* SerialReduction::dot / norm (reduction.hpp:114-150). */
owtk_status owtk_dot(owtk_vector* lhs, owtk_vector* rhs, double* result);
owtk_status owtk_norm(owtk_vector* v, double* result);
/* k dots of w against basis[0..k) and w.w in one pass (krylov_solvers.hpp:273-281). */
owtk_status owtk_dot_batch(owtk_vector* w, owtk_vector* const* basis, size_t k, double* results);

/* ---- matrices ------------------------------------------------------------
 * Index arrays are host size_t-compatible (uint64), values host arrays in
 * the matrix dtype; they are validated (block_csr.hpp:281-300), narrowed to
 * int32 and uploaded once. */
/* BlockCsrMatrix<T> (block_csr.hpp:22-360): values [entry][component]. */
owtk_status owtk_bsr_create(owtk_context* ctx, owtk_dtype dtype, size_t owned_nodes,
                            size_t ghost_nodes, size_t block_size, const uint64_t* row_offsets,
                            const uint64_t* column_indices, const void* values,
                            owtk_matrix** out);
/* New numeric values for the same pattern (host array). */
owtk_status owtk_bsr_update_values(owtk_matrix* m, const void* values);
/* SplitBlockCsrMatrixView<T> (split_block_csr.hpp:29-196): diagonal[node][c]
 * and off_diagonal[edge][c].  The coefficient arrays are BORROWED device
 * memory: writes to them are seen by the next apply without any update call
 * (split_block_csr.hpp:25-27); only the structure is copied. */
owtk_status owtk_split_view_create(owtk_context* ctx, owtk_dtype dtype, size_t owned_nodes,
                                   size_t ghost_nodes, size_t block_size,
                                   const uint64_t* off_diagonal_row_offsets,
                                   const uint64_t* off_diagonal_columns,
                                   const void* device_diagonal, const void* device_off_diagonal,
                                   owtk_matrix** out);
/* DenseBlockCsrMatrix<T> (dense_block_csr.hpp:15-330): row-major bs x bs blocks. */
owtk_status owtk_dense_bsr_create(owtk_context* ctx, owtk_dtype dtype, size_t owned_nodes,
                                  size_t ghost_nodes, size_t block_size,
                                  const uint64_t* row_offsets, const uint64_t* column_indices,
                                  const void* values, owtk_matrix** out);
owtk_status owtk_matrix_destroy(owtk_matrix* m);
/* kind: 0 component-diagonal BSR, 1 split view, 2 dense BSR, 3 host callback. */
owtk_status owtk_matrix_info(owtk_matrix* m, int* kind, size_t* owned_nodes,
                             size_t* ghost_nodes, size_t* block_size, size_t* entries);
/* Matrix::apply (block_csr.hpp:192-215, split_block_csr.hpp:89-119,
 * dense_block_csr.hpp:173-205): owned rows of out are overwritten. */
owtk_status owtk_spmv(owtk_matrix* m, owtk_vector* in, owtk_vector* out);

/* BlockCsrMatrix / SplitBlockCsrMatrixView / DenseBlockCsrMatrix::apply_rows
 * (block_csr.hpp:198-215, split_block_csr.hpp:95-119,
 * dense_block_csr.hpp:179-204): out rows listed in host_rows (count entries,
 * any order, repeats allowed) computed as apply computes them, bit for bit;
 * other rows untouched.  A row >= owned gives OWTK_ERR_OUT_OF_RANGE. */
owtk_status owtk_spmv_rows(owtk_matrix* m, owtk_vector* in, owtk_vector* out, const uint64_t* host_rows,
                           size_t count);
/* BlockCsrMatrix::diagonal (block_csr.hpp:217-236), host output. */
owtk_status owtk_matrix_diagonal(owtk_matrix* m, void* host_out);

/* ---- preconditioners (preconditioner.hpp, split_block_csr.hpp:205-332) ---- */
typedef enum owtk_pc_kind {
    OWTK_PC_IDENTITY = 0,    /* IdentityPreconditioner (preconditioner.hpp:17-23) */
    OWTK_PC_JACOBI = 1,      /* JacobiPreconditioner (:25-113); parameter = minimum diagonal (<= 0: 64 eps) */
    OWTK_PC_SSOR = 2,        /* LocalSsorPreconditioner (:124-247); parameter = omega */
    OWTK_PC_SPLIT_SSOR = 3,  /* SplitLocalSsorPreconditioner (split_block_csr.hpp:205-332); parameter = omega */
    OWTK_PC_ILU = 4,         /* IluLevelPreconditioner / Ilu0Preconditioner (:253-508); parameter = fill level */
    /* No reference counterpart: ILU(0) of a dense-block BSR (bs <= 4), block
     * IKJ factorisation with inverted diagonal blocks; parameter unused. */
    OWTK_PC_BLOCK_ILU = 5,
    /* Created only by owtk_pc_create_mixed. */
    OWTK_PC_MIXED = 6,
    /* Created only by owtk_pc_create_learned. */
    OWTK_PC_LEARNED = 7,
    /* Created only by owtk_pc_create_callback. */
    OWTK_PC_CALLBACK = 8
} owtk_pc_kind;

owtk_status owtk_pc_create(owtk_matrix* m, owtk_pc_kind kind, double parameter,
                           owtk_preconditioner** out);
/* Mixed precision (no reference counterpart).  owtk_pc_create_stored: an
 * ILU / block ILU of an FP64 matrix, factorised in FP64 on the device, whose
 * factors are kept in `storage` (OWTK_F32 or OWTK_BF16); its applies take
 * FP32 vectors and compute in FP32.  owtk_pc_create_mixed: a preconditioner
 * for FP64 (flexible) solves that hands its FP64 input to an FP32 inner
 * solve — `inner_iterations` GMRES steps with an FP32 copy of the matrix and
 * the stored-precision factors (0: one factor apply) — and returns the FP64
 * result.  owtk_pc_update_values refreshes both from the FP64 matrix. */
owtk_status owtk_pc_create_stored(owtk_matrix* m, owtk_pc_kind kind, double parameter, owtk_dtype storage,
                                  owtk_preconditioner** out);
owtk_status owtk_pc_create_mixed(owtk_matrix* m, owtk_pc_kind inner_kind, double parameter, owtk_dtype storage,
                                 uint32_t inner_iterations, owtk_preconditioner** out);
owtk_status owtk_pc_destroy(owtk_preconditioner* pc);
/* apply(const in, out); in == out is allowed for ILU and split SSOR. */
owtk_status owtk_pc_apply(owtk_preconditioner* pc, owtk_vector* in, owtk_vector* out);
/* update_values(matrix) — re-validates the pattern and refactors; SSOR
 * refreshes its diagonal cache from the same matrix (preconditioner.hpp:142). */
owtk_status owtk_pc_update_values(owtk_preconditioner* pc, owtk_matrix* m);
uint64_t owtk_pc_numeric_updates(owtk_preconditioner* pc);
/* ILU factor storage (preconditioner.hpp:367-370); pass NULL arrays to query
 * the entry count first.  Values and inverse diagonal in the PC's dtype (the
 * FP64 factors for stored-precision PCs); for a block ILU the values hold
 * bs*bs per entry and the inverse diagonal bs*bs per row. */
owtk_status owtk_ilu_factors(owtk_preconditioner* pc, uint64_t* entries, uint64_t* row_offsets,
                             uint64_t* columns, void* values, void* inverse_diagonal);
/* Level sets the sweeps were scheduled with (no reference counterpart): per
 * owned row its lower (forward-sweep) and upper (backward-sweep) level. */
owtk_status owtk_pc_levels(owtk_preconditioner* pc, int32_t* lower_level, int32_t* upper_level,
                           uint64_t* lower_depth, uint64_t* upper_depth);

/* How an ILU preconditioner's applies are scheduled (no reference
 * counterpart): cluster_ctas > 0 when they run on one thread-block cluster of
 * that many CTAs (dependency values through distributed shared memory, epochs
 * of epoch_levels levels, ring_rows rows of results per CTA), 0 for the
 * level-scheduled sweep over the whole GPU.  Both give the same bits.  The
 * cluster schedule is opt-in (environment variable OWTK_CLUSTER_SWEEP=1 at
 * preconditioner creation): on a 2M-vertex RCM-ordered mesh it measured
 * slower than the level-scheduled sweep. */
owtk_status owtk_pc_sweep_schedule(owtk_preconditioner* pc, int32_t* cluster_ctas, int32_t* epoch_levels,
                                   int32_t* ring_rows);

/* Whether an ILU preconditioner's applies run as the chain sweep (no
 * reference counterpart): *windows > 0 (the number of row windows) when both
 * factor DAGs average fewer than 8 rows per level, as on a Hilbert-curve
 * order, and the applies run one warp per component through windows of up
 * to 32 consecutive rows; 0 otherwise.  The same bits either way.  The
 * environment variable OWTK_CHAIN_SWEEP=0 at preconditioner creation turns
 * it off. */
owtk_status owtk_pc_chain_schedule(owtk_preconditioner* pc, int32_t* windows);

/* Whether an ILU preconditioner's applies run level by level on one
 * thread-block cluster (no reference counterpart): *cluster_ctas > 0 (the
 * cluster's CTAs) with the two sweeps' level counts, 0 otherwise.  The
 * lockstep schedule is opt-in (the environment variable OWTK_LOCKSTEP_SWEEP=1
 * at preconditioner creation; it is slower than the level-scheduled sweep on
 * the meshes measured) and is taken when every level fits the cluster's lanes
 * (512 per CTA, one per row and component) and the DAGs are not
 * near-sequential; the same bits as every other schedule. */
owtk_status owtk_pc_lockstep_schedule(owtk_preconditioner* pc, int32_t* cluster_ctas, int32_t* lower_levels,
                                      int32_t* upper_levels);

/* ---- host setup (ordering.hpp) -------------------------------------------- */
/* reverse_cuthill_mckee_order (ordering.hpp:138-180); new_to_old[owned]. */
owtk_status owtk_rcm_order(size_t owned_nodes, size_t ghost_nodes, const uint64_t* row_offsets,
                           const uint64_t* column_indices, uint64_t* new_to_old);
/* hilbert_order (ordering.hpp:231-261); xy holds n (x, y) pairs. */
owtk_status owtk_hilbert_order(size_t n, const double* xy, uint64_t* new_to_old);
/* inverse_permutation (ordering.hpp:263-277). */
owtk_status owtk_inverse_permutation(size_t n, const uint64_t* new_to_old, uint64_t* old_to_new);
/* Level sets of a pattern (no reference counterpart); depths are max level + 1. */
owtk_status owtk_level_sets(size_t owned_nodes, const uint64_t* row_offsets,
                            const uint64_t* column_indices, int32_t* lower_level,
                            int32_t* upper_level, uint64_t* lower_depth, uint64_t* upper_depth);

/* ---- solvers (krylov_solvers.hpp, pipelined_bicgstab.hpp, idrs.hpp) ------- */
typedef enum owtk_solver_kind {
    OWTK_SOLVER_FGMRES = 0,                   /* fgmres / gmres (krylov_solvers.hpp:159-540) */
    OWTK_SOLVER_BICGSTAB = 1,                 /* bicgstab (:542-809) */
    OWTK_SOLVER_PIPELINED_BICGSTAB = 2,       /* pipelined_bicgstab (pipelined_bicgstab.hpp:20-313) */
    OWTK_SOLVER_COMM_HIDING_BICGSTAB = 3,     /* communication_hiding_bicgstab (:321-661) */
    OWTK_SOLVER_IDRS = 4                      /* idrs (idrs.hpp:128-506) */
} owtk_solver_kind;

/* SolverOptions<T> (core.hpp:88-111) without the callback. */
typedef struct owtk_solver_options {
    double relative_tolerance;
    double absolute_tolerance;
    double breakdown_tolerance;
    uint64_t maximum_iterations;
    uint64_t convergence_check_interval;
    uint64_t restart;
    uint64_t residual_replacement_interval;
    uint64_t idr_shadow_space;
    double relaxation;
    int32_t verify_true_residual;
    int32_t gmres_orthogonalization;  /* 0 iterated CGS, 1 adaptive CGS, 2 one-sync CGS */
} owtk_solver_options;

/* SolverResult<T> (core.hpp:118-146); status / breakdown_reason carry the
 * numeric values of SolverStatus (:24-30) and BreakdownReason (:41-52). */
typedef struct owtk_solver_result {
    int32_t status;
    int32_t breakdown_reason;
    uint64_t iterations;
    uint64_t operator_applications;
    uint64_t preconditioner_applications;
    uint64_t global_reductions;
    uint64_t reorthogonalizations;
    uint64_t arnoldi_norm_verifications;
    double initial_residual_norm;
    double recursive_residual_norm;
    double true_residual_norm;
    double relative_residual_norm;
    int32_t converged_by_application;
    int32_t reserved;
    double solve_seconds;
} owtk_solver_result;

void owtk_default_options(owtk_solver_options* options);

/* SolverWorkspace<T> (core.hpp:402-459): device vectors reused across solves
 * of the same layout; allocation_epochs() counts (re)allocations. */
owtk_status owtk_workspace_create(owtk_context* ctx, owtk_workspace** out);
owtk_status owtk_workspace_destroy(owtk_workspace* ws);
uint64_t owtk_workspace_allocation_epochs(owtk_workspace* ws);
/* Workspace vector `index` (same slot order as the reference solver), or NULL. */
owtk_vector* owtk_workspace_vector(owtk_workspace* ws, size_t index);

/* Device-resident solve: rhs and x are device vectors with the matrix layout.
 * pc may be NULL (identity); workspace may be NULL (a temporary is used). */
owtk_status owtk_solve(owtk_solver_kind kind, owtk_matrix* m, owtk_preconditioner* pc,
                       owtk_vector* rhs, owtk_vector* x, const owtk_solver_options* options,
                       owtk_workspace* workspace, owtk_solver_result* result);
/* The reference-facing call on HOST buffers ((owned+ghost)*bs values each):
 * copies rhs and x in, solves on the device, copies x back. */
owtk_status owtk_solve_host(owtk_solver_kind kind, owtk_matrix* m, owtk_preconditioner* pc,
                            const void* host_rhs, void* host_x,
                            const owtk_solver_options* options, owtk_workspace* workspace,
                            owtk_solver_result* result);

/* ---- reductions, application convergence tests, Arnoldi snapshots ---------
 * The reference's solvers take a Reduction, an optional
 * SolverOptions::convergence_test callback and (FGMRES) an optional
 * ArnoldiSnapshot; owtk_solve_ex / owtk_solve_host_ex take them as extras. */
typedef enum owtk_reduction_kind {
    OWTK_REDUCTION_SERIAL = 0,          /* SerialReduction (reduction.hpp:103-168) */
    /* CompensatedSerialReduction (reduction.hpp:175-226): Neumaier-compensated
     * sums of the rounded products, partial pairs merged exactly. */
    OWTK_REDUCTION_COMPENSATED = 1,
    /* MixedPrecisionSerialReduction (reduction.hpp:228-299): products split
     * exactly by FMA and summed in doubled precision (Dot2 of Ogita, Rump and
     * Oishi), at least as accurate as the reference's long double sums; the
     * 2-norm in doubled precision too. */
    OWTK_REDUCTION_MIXED_PRECISION = 2
} owtk_reduction_kind;

/* dot / norm with a chosen reduction.  `low` (may be NULL) receives the low
 * part of the compensated result: result + low is the exact sum of the
 * device's (sum, correction) pair, the analogue of the reference's
 * long double local_dot. */
owtk_status owtk_dot_ex(owtk_vector* lhs, owtk_vector* rhs, owtk_reduction_kind reduction, double* result,
                        double* low);
owtk_status owtk_norm_ex(owtk_vector* v, owtk_reduction_kind reduction, double* result);

/* SolverOptions::convergence_test (core.hpp:102-108, called as in
 * krylov_solvers.hpp:122-143): called at iteration zero and after each
 * complete iterate with the iteration count and a HOST copy of the candidate
 * solution ((owned + ghost) * bs values in the solve's dtype).  Return 1 to
 * stop (the solver then measures the true residual and reports
 * converged_by_application), 0 to continue, a negative value to abort the
 * solve with OWTK_ERR_RUNTIME.  While a test is set, the residual tolerance
 * is replaced by it, as in the reference. */
typedef int (*owtk_convergence_test_fn)(void* user, uint64_t iteration, const void* candidate, size_t count);

/* ArnoldiSnapshot<T> (core.hpp:462-534): the last unrotated Arnoldi relation
 * FGMRES produced — the Hessenberg entries h(row, column) of the last cycle
 * and its preconditioned basis vectors (device vectors owned by the snapshot). */
typedef struct owtk_arnoldi_snapshot owtk_arnoldi_snapshot;
owtk_status owtk_arnoldi_snapshot_create(owtk_context* ctx, owtk_arnoldi_snapshot** out);
owtk_status owtk_arnoldi_snapshot_destroy(owtk_arnoldi_snapshot* snapshot);
owtk_status owtk_arnoldi_snapshot_clear(owtk_arnoldi_snapshot* snapshot);
size_t owtk_arnoldi_snapshot_columns(const owtk_arnoldi_snapshot* snapshot);
/* OWTK_ERR_OUT_OF_RANGE unless column < columns and row <= columns. */
owtk_status owtk_arnoldi_snapshot_h(const owtk_arnoldi_snapshot* snapshot, size_t row, size_t column,
                                    double* value);
/* Borrowed handle of preconditioned basis vector `column` (< columns). */
owtk_status owtk_arnoldi_snapshot_basis(owtk_arnoldi_snapshot* snapshot, size_t column, owtk_vector** out);

typedef struct owtk_solve_extras {
    int32_t reduction;                          /* owtk_reduction_kind */
    int32_t reserved;                           /* 0 */
    owtk_convergence_test_fn convergence_test;  /* NULL: none */
    void* convergence_user;
    owtk_arnoldi_snapshot* arnoldi_snapshot;    /* FGMRES only; NULL: none */
} owtk_solve_extras;

/* owtk_solve / owtk_solve_host with extras (NULL extras: the plain call). */
owtk_status owtk_solve_ex(owtk_solver_kind kind, owtk_matrix* m, owtk_preconditioner* pc, owtk_vector* rhs,
                          owtk_vector* x, const owtk_solver_options* options, owtk_workspace* workspace,
                          const owtk_solve_extras* extras, owtk_solver_result* result);
owtk_status owtk_solve_host_ex(owtk_solver_kind kind, owtk_matrix* m, owtk_preconditioner* pc,
                               const void* host_rhs, void* host_x, const owtk_solver_options* options,
                               owtk_workspace* workspace, const owtk_solve_extras* extras,
                               owtk_solver_result* result);

/* solve_specwave_native (specwave_compat.hpp:99-249) for the legacy SpecWave
 * solver IDs: 3, 4, 10, 22 communication-hiding BiCGSTAB + SSOR (4: residual
 * replacement 50 when unset); 5, 8, 11 BiCGSTAB + SSOR; 7 GMRES + SSOR;
 * 9, 13 BiCGSTAB + ILU(0); 12, 15 pipelined BiCGSTAB + SSOR; 14 IDR(s) + SSOR;
 * 21 pipelined BiCGSTAB + ILU(0); SSOR with omega = options->relaxation.  ID 10
 * uses the mixed-precision reduction and ID 22 the compensated one, as in the
 * reference; the other IDs use `reduction` (serial for owtk_solve_specwave).
 * ID 6 (PETSc) returns the default result (invalid_input); the stationary and
 * multigrid IDs are rejected with OWTK_ERR_INVALID_ARGUMENT. */
owtk_status owtk_solve_specwave(int solver_id, owtk_matrix* m, owtk_vector* rhs, owtk_vector* x,
                                const owtk_solver_options* options, owtk_workspace* workspace,
                                owtk_solver_result* result);
owtk_status owtk_solve_specwave_ex(int solver_id, owtk_matrix* m, owtk_vector* rhs, owtk_vector* x,
                                   const owtk_solver_options* options, owtk_workspace* workspace,
                                   owtk_reduction_kind reduction, owtk_solver_result* result);

/* ---- host-callback operators and preconditioners ----------------------------
 * The reference's solvers are templates over duck-typed operators and
 * preconditioners (docs/MANUAL.tex:676-712): any type with apply(in, out).
 * These wrap such an application-supplied host function so the device
 * solvers can use it: each application copies `in` ((owned + ghost) * bs
 * values) and the current `out` to host buffers, calls apply(user, in, out,
 * count) and copies out's owned values (and in's ghost values, which a halo
 * exchange may write) back.  apply returns 0 on success; anything else fails
 * the call with OWTK_ERR_RUNTIME.  Every application synchronises the
 * stream, so these suit matrix-free operators and prototypes, not speed. */
typedef int (*owtk_host_apply_fn)(void* user, void* in, void* out, size_t count);
/* A matrix of kind 3 usable wherever an operator is (owtk_spmv, solves);
 * preconditioners that need coefficients (Jacobi, SSOR, ILU) reject it. */
owtk_status owtk_callback_operator_create(owtk_context* ctx, owtk_dtype dtype, size_t owned_nodes,
                                          size_t ghost_nodes, size_t block_size, owtk_host_apply_fn apply,
                                          void* user, owtk_matrix** out);
/* A preconditioner of kind OWTK_PC_CALLBACK (8) for vectors of this layout. */
owtk_status owtk_pc_create_callback(owtk_context* ctx, owtk_dtype dtype, size_t owned_nodes, size_t ghost_nodes,
                                    size_t block_size, owtk_host_apply_fn apply, void* user,
                                    owtk_preconditioner** out);

/* ---- permutations and device ingestion of a split layout -------------------
 * The orderings above give new_to_old; these apply one on the device.  No
 * reference counterpart (the reference orders but never permutes; its
 * inverse_permutation, ordering.hpp:263-277, defines the validation). */
typedef struct owtk_permutation owtk_permutation;
/* new_to_old[i] = old index of new node i; every index in [0, n) once. */
owtk_status owtk_permutation_create(owtk_context* ctx, size_t n, const uint64_t* new_to_old, owtk_permutation** out);
owtk_status owtk_permutation_destroy(owtk_permutation* p);
/* Owned nodes of dst from src (same layout, n owned nodes, dst != src):
 * inverse 0: dst.node(i) = src.node(new_to_old[i]); inverse 1:
 * dst.node(new_to_old[i]) = src.node(i).  Ghost entries are untouched. */
owtk_status owtk_vector_permute(owtk_permutation* p, owtk_vector* src, owtk_vector* dst, int inverse);
/* P A P^T as a component-diagonal BSR matrix, built from an application's
 * split layout (SplitBlockCsrMatrixView, split_block_csr.hpp:17-28): the
 * diagonal[node][c] and off_diagonal[edge][c] arrays in DEVICE memory, the
 * edge structure (off-diagonal row offsets and columns, n owned nodes, no
 * ghosts) on the host.  Row i of the result is old row new_to_old[i] with
 * its diagonal and edges relabelled and sorted by new column; the values are
 * gathered on the device.  owtk_bsr_update_permuted_split re-gathers them
 * from the same-shaped arrays (a numeric update with no host copy). */
owtk_status owtk_bsr_create_permuted_split(owtk_permutation* p, owtk_dtype dtype, size_t bs,
                                           const uint64_t* off_rowptr, const uint64_t* off_cols,
                                           const void* device_diagonal, const void* device_off_diagonal,
                                           owtk_matrix** out);
owtk_status owtk_bsr_update_permuted_split(owtk_matrix* m, const void* device_diagonal,
                                           const void* device_off_diagonal);

/* ---- bounded device waits (no reference counterpart) ----------------------
 * Every device-side wait of this library (sweep dependencies, the batched
 * solver's grid barrier, pipeline stages) gives up after a bounded number of
 * polls, sets a status bit and lets its launch end; the call then returns
 * OWTK_ERR_TIMEOUT and the context stays usable.  This hook runs a two-row
 * ILU forward sweep whose only dependency is never published, with the given
 * poll limit (1 .. 2^22), so the timeout path can be exercised without any
 * fault: it returns OWTK_ERR_TIMEOUT. */
owtk_status owtk_debug_unpublished_dependency(owtk_context* ctx, uint32_t spin_limit);

/* ---- allocation-free variant (no counterpart in the reference) ----------
 * The batched dot product of owtk_dot_batch for callers that cannot allocate
 * device memory (a host framework that owns the device allocator, code where
 * a cudaMalloc would be forbidden or would synchronise the device).  It needs
 * no context and allocates nothing: w, the k basis vectors (a host array of
 * device pointers, n doubles each) and results (k + 1 doubles: w.basis_j, then
 * w.w) are caller-owned device memory; stream is a cudaStream_t (NULL: the
 * legacy default stream).  Its reduction scratch is one static device array
 * of about 148 KiB that every GPU loading the library holds until exit, so:
 * k <= 31 (larger batches return OWTK_ERR_INVALID_ARGUMENT); calls that
 * overlap on the GPU race on that array and must be serialised; and the
 * first call on a device looks up the array's address with that device
 * current, so make it before any stream capture.  The address is kept for the
 * life of the process: do not call it again on a device after
 * cudaDeviceReset, which invalidates that address. */
owtk_status owtk_dot_batch_f64_noalloc(const double* w, const double* const* basis, size_t k,
                                       size_t n, double* results, void* stream);

/* ---------------------------------------------------------------- batching
 * Many independent FP64 component-diagonal block-CSR systems (uneven sizes,
 * block sizes 1..32, ghosts 0) solved together by BiCGSTAB with a Jacobi
 * preconditioner in ONE persistent cooperative launch with per-system
 * convergence masks, captured once in a CUDA graph and replayed.  No single
 * reference counterpart: each system follows the reference's bicgstab
 * (krylov_solvers.hpp:546-745) with JacobiPreconditioner
 * (preconditioner.hpp:25-113), result counters included; the structure of each
 * system is validated like BlockCsrMatrix (block_csr.hpp:281-300). */
typedef struct owtk_batch owtk_batch;

typedef struct owtk_batch_system {
    size_t owned;               /* vertices (rows) */
    size_t bs;                  /* block size, 1..32 */
    const uint64_t* rowptr;     /* host, owned + 1 */
    const uint64_t* cols;       /* host, rowptr[owned] local columns < owned */
    const double* values;       /* host, rowptr[owned] * bs, [entry][component] */
} owtk_batch_system;

owtk_status owtk_batch_create(owtk_context* ctx, size_t count, const owtk_batch_system* systems, owtk_batch** out);
owtk_status owtk_batch_destroy(owtk_batch* batch);
/* Total unknowns and the first unknown of each system (count + 1 entries):
 * right-hand sides and solutions are single device arrays in system order. */
owtk_status owtk_batch_layout(const owtk_batch* batch, size_t* unknowns, uint64_t* offsets);
/* Current launch shape: resident blocks per SM and vertices per warp pass for
 * block sizes 0..32 (33 entries; index = block size). */
owtk_status owtk_batch_config(const owtk_batch* batch, uint32_t* blocks_per_sm, uint32_t* vertices_per_warp);
/* Override the shape (0 leaves a field unchanged).  Blocks per SM run from 1
 * to 8 (clamped to what is resident); each count launches the solver build
 * whose register budget allows it. */
owtk_status owtk_batch_set_config(owtk_batch* batch, uint32_t blocks_per_sm, size_t bs, uint32_t vertices_per_warp);
/* Autotuner: times one SpMV pass per vertices-per-warp candidate and block
 * size present, then a few solver iterations per blocks-per-SM count (every
 * resident count), and keeps the fastest; outputs as owtk_batch_config (either
 * may be NULL). */
owtk_status owtk_batch_autotune(owtk_batch* batch, const owtk_solver_options* options, uint32_t* blocks_per_sm,
                                uint32_t* vertices_per_warp);
/* 1 (default): each solve replays a CUDA graph holding the whole launch
 * (re-captured when the vectors, options or shape change); 0: plain launches. */
owtk_status owtk_batch_use_graph(owtk_batch* batch, int enable);
owtk_status owtk_batch_graph_counts(const owtk_batch* batch, uint64_t* captures, uint64_t* launches);
/* Solve every system from the initial guess in x; results has count entries.
 * Device arrays of owtk_batch_layout's total length. */
owtk_status owtk_batch_solve(owtk_batch* batch, const double* device_rhs, double* device_x,
                             const owtk_solver_options* options, owtk_solver_result* results);
/* Same with host arrays (copied in and out inside the call). */
owtk_status owtk_batch_solve_host(owtk_batch* batch, const double* host_rhs, double* host_x,
                                  const owtk_solver_options* options, owtk_solver_result* results);

/* ---------------------------------------------------------------- tensor cores
 * D (m x n, FP32, row-major) = A (m x k, BF16, row-major) * B (n x k, BF16,
 * row-major)^T on the sm_100a tensor cores (tcgen05.mma, FP32 accumulation in
 * tensor memory); m % 128 == 0, n in {64, 128}, k % 64 == 0, 16-byte aligned
 * device pointers.  The building block of the learned preconditioner's dense
 * products, exposed to check that path in isolation.  No reference
 * counterpart. */
owtk_status owtk_bf16_gemm_nt(owtk_context* ctx, size_t m, size_t n, size_t k, const void* device_a,
                              const void* device_b, float* device_d);

/* ---------------------------------------------------------------- learned preconditioner
 * A message-passing network on the graph of an FP64 component-diagonal BSR
 * matrix (ghosts 0, block size <= 8): hidden width 64, 4 layers, BF16 weights
 * and activations on the tensor cores with FP32 accumulation, no biases (so
 * M(a r) = a M(r) for a > 0); its decoder adds the Jacobi step, so untrained
 * weights give the Jacobi preconditioner.  The FP64 restatement of the
 * network is oracle/gnn.py.  No reference counterpart.  The matrix is
 * borrowed and must outlive the network. */
typedef struct owtk_learned owtk_learned;

owtk_status owtk_learned_create(owtk_matrix* m, uint64_t seed, owtk_learned** out);
owtk_status owtk_learned_destroy(owtk_learned* net);
/* Re-read the coefficients of a matrix with the same pattern (edge weights
 * and diagonal of the graph); the weights are kept. */
owtk_status owtk_learned_update_matrix(owtk_learned* net, owtk_matrix* m);
/* 1 when the layers gather neighbours with TMA (tile::gather4) into shared
 * memory (environment OWTK_GNN_TMA=1 at creation, with tensor-map support),
 * 0 for the default register-gather path; both give bit-identical results. */
int owtk_learned_uses_tma(const owtk_learned* net);
/* Flat FP32 parameters: encoder 64x16, 4 layers 64x128, decoder 8x64. */
size_t owtk_learned_parameter_count(void);
owtk_status owtk_learned_get_parameters(owtk_learned* net, float* host, size_t count);
owtk_status owtk_learned_set_parameters(owtk_learned* net, const float* host, size_t count);
/* Adam optimiser state (first and second moments, count = parameter count,
 * and the step number of the bias correction), so training can be saved to
 * a checkpoint and resumed. */
owtk_status owtk_learned_get_adam_state(owtk_learned* net, float* first_moment, float* second_moment, size_t count,
                                        uint64_t* step);
owtk_status owtk_learned_set_adam_state(owtk_learned* net, const float* first_moment, const float* second_moment,
                                        size_t count, uint64_t step);
/* out = M(in), FP64 vectors of the matrix layout. */
owtk_status owtk_learned_apply(owtk_learned* net, owtk_vector* in, owtk_vector* out);
/* Profiling: `repetitions` applications out = M(in), each stage bracketed by
 * CUDA events on the context's stream.  milliseconds[5] receives the mean
 * time of (0) the norms and the encoder (with the encoder folded into the
 * first layer: the norms and the input records), (1) one fused
 * message-passing layer (k_gnn_layer) before the last, (2) the last layer
 * with the decoder fused, (3) the whole application, (4) the first layer
 * with the encoder folded in (0 when the encoder runs on its own: training
 * builds, block sizes above 4, OWTK_GNN_FUSED_FIRST=0). */
owtk_status owtk_learned_stage_times(owtk_learned* net, owtk_vector* in, owtk_vector* out, uint32_t repetitions,
                                     double* milliseconds);
/* Forward + backward of one training pair: the loss (weights below) and
 * its gradient, kept on the device for owtk_learned_adam_step (and copied
 * to host_grads when it is not NULL). */
owtk_status owtk_learned_loss_grad(owtk_learned* net, owtk_vector* r, owtk_vector* e, double* loss,
                                   float* host_grads);
owtk_status owtk_learned_adam_step(owtk_learned* net, double learning_rate);
/* Loss = error_weight ||M(r) - e||^2 / ||e||^2
 *      + residual_weight ||r - A M(r)||^2 / ||r||^2   (default 0.1 and 1). */
owtk_status owtk_learned_set_loss_weights(owtk_learned* net, double error_weight, double residual_weight);
/* The network as a preconditioner of its matrix: each application z = M(v)
 * is judged by the FP64 residual ||v - A z||; when that does not fall below
 * ||v|| the fallback (e.g. ILU(0), may be NULL) computes z instead.  Both
 * handles are borrowed. */
owtk_status owtk_pc_create_learned(owtk_learned* net, owtk_preconditioner* fallback, owtk_preconditioner** out);
owtk_status owtk_pc_learned_counts(owtk_preconditioner* p, uint64_t* applications, uint64_t* fallbacks);
/* No reference counterpart (the learned form is new).  After each accepted
 * network step z = M(v), `steps` (0..8, default 0) damped Jacobi corrections
 * z += omega D^-1 (v - A z), 0 < omega < 2, with D^-1 the FP32 reciprocal
 * diagonal; each costs one element-wise pass and one SpMV, and the solver
 * reuses the last product A z as its next operator application. */
owtk_status owtk_pc_learned_set_correction(owtk_preconditioner* p, uint32_t steps, double omega);

#ifdef __cplusplus
}
#endif

#endif /* OWTK_H */
