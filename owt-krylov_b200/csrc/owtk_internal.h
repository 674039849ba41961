// Internal declarations shared by the kernels (*.cu) and the host runtime
// (capi.cu, setup.cpp, solvers.cpp).  Not part of the public ABI.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <exception>
#include <memory>
#include <new>
#include <string>
#include <vector>

#include "../../include/owtk.h"

namespace owtk {

// ---------------------------------------------------------------- errors
struct Error {
    owtk_status code;
    std::string message;
};
[[noreturn]] void fail(owtk_status code, const std::string& message);
void cuda_check(cudaError_t e, const char* what);
#define OWTK_CUDA(call) ::owtk::cuda_check((call), #call)
void record_error(const std::string& message);   // text returned by owtk_last_error()

inline void require(bool ok, const char* message)
{
    if (!ok) fail(OWTK_ERR_INVALID_ARGUMENT, message);
}

// Runs an entry point's body, mapping exceptions to status codes.
template<class F>
owtk_status guarded(F&& f)
{
    try {
        f();
        return OWTK_OK;
    } catch (const Error& e) {
        record_error(e.message);
        return e.code;
    } catch (const std::bad_alloc&) {
        record_error("host allocation failed");
        return OWTK_ERR_RUNTIME;
    } catch (const std::exception& e) {
        record_error(e.what());
        return OWTK_ERR_RUNTIME;
    }
}

// ---------------------------------------------------------------- device buffers
// Owning device allocation (cudaMalloc) released on destruction.
struct DeviceBuffer {
    void* ptr = nullptr;
    std::size_t bytes = 0;
    DeviceBuffer() = default;
    explicit DeviceBuffer(std::size_t n) { allocate(n); }
    DeviceBuffer(const DeviceBuffer&) = delete;
    DeviceBuffer& operator=(const DeviceBuffer&) = delete;
    DeviceBuffer(DeviceBuffer&& o) noexcept : ptr(o.ptr), bytes(o.bytes) { o.ptr = nullptr; o.bytes = 0; }
    DeviceBuffer& operator=(DeviceBuffer&& o) noexcept;
    ~DeviceBuffer();
    void allocate(std::size_t n);
    template<class T> T* as() const { return static_cast<T*>(ptr); }
};

// Upload a host vector into a fresh device buffer (synchronous on the stream).
template<class T>
DeviceBuffer upload(cudaStream_t s, const std::vector<T>& host)
{
    DeviceBuffer b(host.size() * sizeof(T) + 16);
    if (!host.empty())
        OWTK_CUDA(cudaMemcpyAsync(b.ptr, host.data(), host.size() * sizeof(T),
                                  cudaMemcpyHostToDevice, s));
    return b;
}

// ---------------------------------------------------------------- context
// Scalar results of reductions land in a mapped pinned block the host reads
// after one stream synchronisation.
constexpr int kScalarSlots = 512;
constexpr int kMaxBatch = 128;           // largest dot batch (GMRES restart + 2)
constexpr int kReduceBlocks = 4 * 148;   // two-stage reductions: max first-stage blocks

struct Context {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    double* host_scalars = nullptr;      // mapped pinned, kScalarSlots
    double* dev_scalars = nullptr;       // device alias of host_scalars
    DeviceBuffer dev_scalar_copy;        // device-resident copies for kernels
    DeviceBuffer partials;               // kReduceBlocks * kMaxBatch * 2 doubles
    DeviceBuffer tickets;                // reduction tickets (self-resetting)
    DeviceBuffer status;                 // device error word(s)
    std::uint64_t launches = 0;
    ~Context();
    void sync();
    void launched(int n = 1) { launches += static_cast<std::uint64_t>(n); }
    // Device error word: set by bounded waits (timeout) and the device factorisation.
    void check_device_status();
};

// ---------------------------------------------------------------- objects
struct Vector {
    Context* ctx = nullptr;
    owtk_dtype dtype = OWTK_F64;
    std::size_t owned = 0, ghost = 0, bs = 0;
    void* data = nullptr;
    DeviceBuffer storage;      // empty for views
    bool is_view = false;
    std::size_t owned_size() const { return owned * bs; }
    std::size_t local_size() const { return (owned + ghost) * bs; }
    std::size_t elem() const { return dtype == OWTK_F64 ? 8 : 4; }
    bool same_layout(const Vector& o) const
    {
        return owned == o.owned && ghost == o.ghost && bs == o.bs;
    }
};

// Row tiles for the SpMV kernels: a tile is a run of consecutive rows whose
// work fits one CTA's shared-memory stage; a row that does not fit alone is a
// "long" tile handled component-parallel.
struct TilePlan {
    DeviceBuffer tile_rows;    // int32, tiles + 1
    DeviceBuffer tile_meta;    // int4 per tile: first row, end row, first entry, end entry
    int tiles = 0;
    int tile_values = 0;       // stage capacity used to build the plan
};

// Row-slice copy of a component-diagonal or dense-block BSR (bs <= 4), read
// by its SpMV.  Slices of 32 consecutive rows, one warp each; a slice's lanes
// take its rows longest first.  Step k of a slice holds entry k of the n_k
// rows longer than k: their columns [lane] and values [value of the entry]
// [lane] (bs values, or bs * bs for dense blocks), packed with no padding
// (step k + 1 starts n_k entries later).  Rows longer than kSliceMaxRow have
// length 0 in their slice and are listed in long_rows.
constexpr int kSliceMaxRow = 48;
struct RowSlices {
    int slices = 0;
    std::size_t packed = 0;    // entries held (all but the long rows')
    DeviceBuffer base;         // int32 per slice + 1: first packed entry
    DeviceBuffer lanes;        // uint16 per slice lane: row in slice | length << 8 (row 255: none)
    DeviceBuffer cols;         // int32 per packed entry
    DeviceBuffer vals;         // element per packed entry and component
    DeviceBuffer long_rows;    // int32
    int long_count = 0;
    bool filled = false;       // cols and vals hold the matrix's current values
};

struct Matrix {
    Context* ctx = nullptr;
    int kind = 0;              // 0 component-diagonal BSR, 1 split view, 2 dense BSR
    owtk_dtype dtype = OWTK_F64;
    std::size_t owned = 0, ghost = 0, bs = 0, entries = 0;
    // Host copies of the structure (needed for setup and pattern checks).
    std::vector<std::int32_t> h_rowptr, h_cols;
    DeviceBuffer rowptr, cols;       // int32
    DeviceBuffer values;             // owning kinds: nnz*bs (BSR) / nnz*bs*bs (dense)
    const void* diag = nullptr;      // split view: borrowed device diagonal
    const void* off = nullptr;       // split view: borrowed device off-diagonal
    TilePlan plan;
    RowSlices slices;
    // Kind 3 (owtk_callback_operator_create): an application function applied
    // on host copies of the vectors.
    owtk_host_apply_fn host_apply = nullptr;
    void* host_user = nullptr;
    std::vector<unsigned char> host_in, host_out;
    // BSR built from a permuted split layout: per entry its source in the
    // split arrays (node < owned: diagonal, else owned + edge), for updates.
    DeviceBuffer split_map;
    std::size_t split_edges = 0;
    // apply_rows: the last row list's device copy, reused while it fits.
    DeviceBuffer row_list;
    const void* value_ptr() const { return kind == 1 ? off : values.ptr; }
    std::size_t local_size() const { return (owned + ghost) * bs; }
};

struct Workspace {
    Context* ctx = nullptr;
    std::vector<std::unique_ptr<Vector>> vectors;
    std::vector<std::unique_ptr<Vector>> stage;   // host-buffer solve staging (rhs, x)
    std::size_t scalar_capacity = 0;              // host scalar arrays (Hessenberg etc.)
    std::uint64_t epochs = 0;
    // core.hpp:405-423: (re)allocate when the layout changes or more vectors /
    // scalars are needed; each growth counts one allocation epoch.
    void prepare(const Vector& layout, std::size_t count, std::size_t scalars = 0);
};

// A scheduled triangular sweep: rows ordered by (level, row), cut into warp
// tasks that never straddle a level; dependencies are the row's entries whose
// column lies on the solved side.
struct Sweep {
    DeviceBuffer order;        // int32 rows
    DeviceBuffer task_start;   // int32, tasks + 1 (positions in order)
    int tasks = 0;
    int depth = 0;             // number of levels
    int rows_per_task = 1;
    std::vector<std::int32_t> h_level;
    std::vector<std::int32_t> h_order;
    // ILU applies: the rows' lower (forward) or upper (backward) factor
    // entries packed in task order, so a task's columns and values are
    // contiguous.  seg: int32, rows + 1 (positions in order); psrc: int64
    // factor entry of each packed entry; pvals refreshed by every numeric
    // factorisation.
    bool packed = false;
    std::size_t pentries = 0;
    DeviceBuffer seg, pcols, psrc, pvals;
};

// The same sweep run by one thread-block cluster (kernels_cluster_sweep.cu):
// tasks dealt round-robin to C CTAs, levels cut into epochs of K levels,
// a ring of R rows per CTA.
struct ClusterSweep {
    bool ready = false;
    int C = 0, K = 0, E = 0, R = 0, tasks = 0;
    DeviceBuffer rows, recs, task_ptr, epoch_task, cta_first;
};

// The ILU applies level by level on one thread-block cluster
// (kernels_lockstep_sweep.cu): per level and CTA a chunk of lanes ((row,
// component) pairs) with a record each (output index, entries, dependency
// locations), their factor values (gathered after every numeric
// factorisation) and the chunk's list of older dependencies.
struct LockstepSweep {
    bool ready = false;
    int C = 0, D = 0, max_lanes = 0, max_far = 0;
    std::size_t values = 0, ovf_values = 0;
    std::uint64_t gathered = ~0ull;   // numeric_updates the gathered values belong to
    DeviceBuffer blk, recs, vsrc, vals, far_src, ovf_loc, ovf_src, ovf_val;
};

// The ILU applies of a near-sequential DAG by one warp per component
// (kernels_chain_sweep.cu): windows of up to 32 consecutive rows.
struct ChainSweep {
    bool ready = false;
    int count = 0;
    DeviceBuffer windows;   // int4 {first row, end row, first entry, end entry}
};
// Rows per level (both DAGs) below which the ILU applies take the chain sweep.
constexpr int kChainRowsPerLevel = 8;

struct Preconditioner {
    Context* ctx = nullptr;
    owtk_pc_kind kind = OWTK_PC_IDENTITY;
    owtk_dtype dtype = OWTK_F64;
    Matrix* matrix = nullptr;
    std::size_t owned = 0, ghost = 0, bs = 0;
    double parameter = 0;
    std::uint64_t numeric_updates = 0;
    DeviceBuffer inv_diag;     // Jacobi, ILU
    DeviceBuffer diag_cache;   // BSR SSOR diagonal cache
    DeviceBuffer work;         // SSOR forward-sweep scratch
    // ILU factor pattern (host copies + device).
    std::vector<std::int32_t> f_rowptr, f_cols, f_diagpos;
    std::vector<std::int64_t> f_source;     // matrix entry or -1 (fill)
    std::vector<std::int32_t> row_counts;   // local entries per matrix row
    DeviceBuffer d_frowptr, d_fcols, d_fdiagpos, d_fsource, d_fvalues;
    // IKJ update list of the numeric factorisation: for every lower entry l,
    // the (target, upper) entry pairs it updates, in reference order.
    DeviceBuffer d_upd_start, d_upd_target, d_upd_upper;
    // SSOR dependency patterns reuse the matrix structure.
    Sweep lower, upper;
    // Cluster schedules of the ILU applies and, per factor entry, where its
    // dependency is read (owner CTA and ring slot, or global memory).
    ClusterSweep c_lower, c_upper;
    ChainSweep chain;
    LockstepSweep l_lower, l_upper;
    DeviceBuffer d_floc;
    DeviceBuffer flags;        // uint32 per row, epoch-stamped
    DeviceBuffer ticket;       // uint64 monotone task counter
    std::uint32_t epoch = 0;
    std::uint64_t ticket_base = 0;
    // Dense-block ILU: bs x bs factor blocks, inverse diagonal blocks.
    bool block = false;
    // Factor storage precision; F32 / BF16 copies are applied to FP32 vectors.
    owtk_dtype storage = OWTK_F64;
    DeviceBuffer lp_vals, lp_inv, work32;
    // Mixed-precision wrapper: FP64 in/out, FP32 inner solve.
    std::unique_ptr<Matrix> m32;
    std::unique_ptr<Preconditioner> inner;
    std::unique_ptr<Workspace> inner_ws;
    unsigned inner_iterations = 0;
    DeviceBuffer v32, z32;
    // Learned preconditioner: the network (borrowed) and the preconditioner
    // that takes a step whenever the network's step does not reduce the FP64
    // residual (borrowed, may be null).
    struct Gnn* net = nullptr;
    Preconditioner* fallback = nullptr;
    std::uint64_t learned_applications = 0, learned_fallbacks = 0;
    // Damped Jacobi corrections after each accepted network step
    // (owtk_pc_learned_set_correction): z += omega D^-1 (v - A z).
    int learned_correction_steps = 0;
    double learned_correction_omega = 1.0;
    DeviceBuffer check_work, alias_copy;
    // OWTK_PC_CALLBACK: an application function applied on host copies.
    owtk_host_apply_fn host_apply = nullptr;
    void* host_user = nullptr;
    std::vector<unsigned char> host_in, host_out;
};
// gnn.cu.  With `product` non-null, returns true when it also holds A z for
// the network's own matrix (no fallback was taken).
bool learned_apply(Preconditioner& p, struct Vector& in, struct Vector& out, double* product = nullptr);
const Matrix* learned_matrix(const Preconditioner& p);


// ---------------------------------------------------------------- setup (setup.cpp)
void build_tile_plan(Matrix& m);
void build_row_slices(Matrix& m);
void levels_of(std::size_t owned, const std::int32_t* rowptr, const std::int32_t* cols,
               std::vector<std::int32_t>& lower, std::vector<std::int32_t>& upper);
void build_sweep(Context& ctx, Sweep& s, std::size_t owned, std::size_t bs,
                 const std::vector<std::int32_t>& level, bool descending_rows);
void pack_sweep(Context& ctx, Sweep& s, std::size_t bs, std::size_t element_size,
                const std::vector<std::int32_t>& rowptr, const std::vector<std::int32_t>& cols,
                const std::vector<std::int32_t>& diagpos, bool backward);
void build_lockstep_sweep(Context& ctx, LockstepSweep& s, std::size_t owned, std::size_t bs, owtk_dtype dtype,
                          const std::vector<std::int32_t>& level, const std::vector<std::int32_t>& rowptr,
                          const std::vector<std::int32_t>& cols, const std::vector<std::int32_t>& diagpos,
                          bool backward);
void build_chain_sweep(Context& ctx, ChainSweep& s, std::size_t owned, int depth_lower, int depth_upper,
                       const std::vector<std::int32_t>& rowptr);
void build_cluster_sweep(Context& ctx, ClusterSweep& s, std::size_t owned, std::size_t bs, owtk_dtype dtype,
                         const std::vector<std::int32_t>& level, const std::vector<std::int32_t>& rowptr,
                         const std::vector<std::int32_t>& cols, const std::vector<std::int32_t>& diagpos,
                         bool backward, std::vector<std::uint32_t>& loc);
void rcm_order(std::size_t owned, const std::int32_t* rowptr, const std::int32_t* cols,
               std::uint64_t* out);
void hilbert_order(std::size_t n, const double* xy, std::uint64_t* out);

// ---------------------------------------------------------------- kernels
namespace kern {

template<class T> void fill(Context& c, std::size_t n, T value, T* x);
template<class T> void copy(Context& c, std::size_t n, const T* x, T* y);
template<class T> void axpy(Context& c, std::size_t n, T alpha, const T* x, T* y);
template<class T> void scale(Context& c, std::size_t n, T alpha, T* x);
template<class T> void lincomb(Context& c, std::size_t n, T a, const T* x, T b, const T* y, T* out);
// out = b - a (true residual)
template<class T> void sub(Context& c, std::size_t n, const T* b, const T* a, T* out);
// out = x / s (GMRES first basis vector)
template<class T> void divide(Context& c, std::size_t n, const T* x, T s, T* out);
// BiCGSTAB search update: p = r + beta*(p - omega*v)
template<class T> void bicg_p(Context& c, std::size_t n, const T* r, T beta, T omega, const T* v, T* p);
// x += alpha*ph; x += omega*sh; r = s - omega*t
template<class T> void bicg_xr(Context& c, std::size_t n, T alpha, const T* ph, T omega, const T* sh,
                               const T* s, const T* t, T* x, T* r);
// Communication-hiding recurrences (pipelined_bicgstab.hpp:436-451, :506-512).
template<class T> void ch_pszupdate(Context& c, std::size_t n, T beta, T omega, const T* r2, const T* w,
                                    const T* w2, const T* t, const T* z2, const T* v,
                                    T* p2, T* s, T* s2, T* z);
template<class T> void ch_qy(Context& c, std::size_t n, T alpha, const T* r, const T* s, const T* r2,
                             const T* s2, const T* w, const T* z, T* q, T* q2, T* y);
template<class T> void ch_rw(Context& c, std::size_t n, T alpha, T omega, const T* q, const T* y,
                             const T* q2, const T* w2, const T* z2, const T* t, const T* v,
                             T* r, T* r2, T* w);
// GMRES: w -= sum_i h_i V_i in reference order (h on device, negated inside).
template<class T> void cgs_update(Context& c, std::size_t n, int k, const T* const* basis,
                                  const double* h, T* w);
// GMRES: out = (w - sum_i h_i V_i) * s (the last pass and the normalisation
// in one; w is not written).
template<class T> void cgs_update_scale(Context& c, std::size_t n, int k, const T* const* basis,
                                        const double* h, const T* w, T s, T* out);
// GMRES: dots of x with V_i (i < k) and x.x, each vector read once (the same
// values as multidot on those pairs); k + 1 <= 32.
template<class T> void basis_dots(Context& c, std::size_t n, int k, const T* const* basis, const T* x,
                                  double* out_dev, double* out_host);
// GMRES fused: w -= sum_i h_i V_i, then dots of the new w with V_i and w.w.
template<class T> void cgs_update_dot(Context& c, std::size_t n, int k, const T* const* basis,
                                      const double* h, T* w, double* out_dev, double* out_host);
// Compensated GMRES update (krylov_solvers.hpp:24-40).
template<class T> void gmres_update(Context& c, std::size_t n, int k, const T* const* dirs,
                                    const double* coef, const T* base, T* out);
// k dot products a_i . b_i (FP64 accumulation); results to out_dev and out_host.
template<class T> void multidot(Context& c, std::size_t n, int k, const T* const* a,
                                const T* const* b, double* out_dev, double* out_host);
template<class T> void norm(Context& c, std::size_t n, const T* x, double* out_dev, double* out_host);
// Accurate reductions: mode 1 compensated (Neumaier over rounded products),
// mode 2 doubled precision (TwoProduct + TwoSum, the Dot2 algorithm).  out_lo
// (host, may be null) receives the low part: out + out_lo is the pair's exact sum.
template<class T> void multidot_accurate(Context& c, std::size_t n, int k, int mode, const T* const* a,
                                         const T* const* b, double* out_dev, double* out_host, double* out_lo);
// Node permutation of owned vector values (forward: dst[new] = src[n2o[new]]).
template<class T> void permute_nodes(Context& c, std::size_t n, std::size_t bs, const std::int64_t* n2o, const T* src,
                                     T* dst, bool inverse);
// values[e] = map[e] < n ? diag[map[e]] : off[map[e] - n] (bs values per entry).
template<class T> void gather_split(Context& c, std::size_t entries, std::size_t bs, std::size_t n,
                                    const std::int64_t* map, const T* diag, const T* off, T* values);
// Doubled-precision 2-norm; scratch: two device doubles.
template<class T> void norm_accurate(Context& c, std::size_t n, const T* x, double* scratch, double* out_dev,
                                     double* out_host);
// ||x - w|| and ||x|| (two results) in one pass.
void residual_norms(Context& c, std::size_t n, const double* x, const double* w, double* out_dev, double* out_host);
// q = r / d (FP32 q, FP32 1/d) with norms[0] = norms[1] = ||r||, norms[2] = norms[3] = ||q||.
template<class T>
void prepare_norms(Context& c, std::size_t n, const T* r, const float* dinv, float* q, double* norms);
template<class T> void jacobi(Context& c, std::size_t n, const T* inv, const T* in, T* out);
template<class T> void spmv(Context& c, const Matrix& m, const T* x, T* y);
template<class T> void spmv_rows(Context& c, const Matrix& m, const int* rows, int count, const T* x, T* y);
// Copy the matrix's current columns and values into its row-slice layout
// (a no-op for matrices without one); called after every write of the values.
void slices_fill(Context& c, Matrix& m);
template<class T> void gather_values(Context& c, std::size_t entries, std::size_t bs,
                                     const std::int64_t* source, const T* values, T* out);
// ILU(0)/SSOR sweeps.
template<class T> void ilu_factorize(Context& c, Preconditioner& p, const T* matrix_values);
template<class T> void ilu_apply(Context& c, Preconditioner& p, const T* in, T* out);
template<class T> bool cluster_ilu_apply(Context& c, Preconditioner& p, const T* in, T* out);
template<class T> bool chain_ilu_apply(Context& c, Preconditioner& p, const T* in, T* out);
template<class T> bool lockstep_ilu_apply(Context& c, Preconditioner& p, const T* in, T* out);
// Test hook: a sweep whose only dependency is never published (bounded wait).
void debug_unpublished_dependency(Context& c, int spin_limit);
template<class T> void ssor_apply(Context& c, Preconditioner& p, const T* in, T* out);
template<class T> void reciprocal_checked(Context& c, std::size_t n, const T* d, T minimum, T* inv);
template<class T> void bsr_diagonal(Context& c, const Matrix& m, T* out);

template<class T> void scaled_copy(Context& c, std::size_t n, const T* x, T s, T* out);
template<class To, class From> void convert(Context& c, std::size_t n, const From* src, To* dst);
template<class F> void ilu_apply_lp(Context& c, Preconditioner& p, const float* in, float* out);
void block_ilu_factorize(Context& c, Preconditioner& p, const double* matrix_values);
void block_ilu_apply(Context& c, Preconditioner& p, const double* in, double* out);

}  // namespace kern

// Operator / preconditioner application on device vectors (capi.cu).
void apply_operator(Matrix& m, Vector& in, Vector& out);
void apply_preconditioner(Preconditioner* p, Vector& in, Vector& out);
// apply_preconditioner that may also return A out (see learned_apply).
bool apply_preconditioner_product(Preconditioner* p, Vector& in, Vector& out, double* product);
void matrix_layout_check_f64(Matrix& m, Vector& in, Vector& out);

// Last unrotated Arnoldi relation of FGMRES (core.hpp:462-534): the
// Hessenberg columns as recorded before the Givens rotations (column-major,
// (max_columns + 1) rows) and device copies of the preconditioned basis.
struct ArnoldiSnapshot {
    Context* ctx = nullptr;
    std::size_t max_columns = 0, columns = 0;
    std::vector<double> h;
    std::vector<std::unique_ptr<Vector>> basis;
    void begin_cycle(const Vector& layout, std::size_t maximum_columns);
    void record_column(std::size_t column, const double* values, std::size_t count);
    void finish_cycle(const std::vector<Vector*>& preconditioned, std::size_t count);
    void clear();
};

// Optional parts of a solve (owtk_solve_ex): the reduction (0 serial,
// 1 compensated, 2 mixed precision), the application convergence test
// (SolverOptions::convergence_test, core.hpp:102-108) and the FGMRES snapshot.
struct SolveExtras {
    int reduction = 0;
    owtk_convergence_test_fn test = nullptr;
    void* user = nullptr;
    ArnoldiSnapshot* snapshot = nullptr;
};

// A device vector with its own storage and the layout and dtype of `like`.
std::unique_ptr<Vector> make_vector_like(const Vector& like);

// Solver recurrences (solvers.cpp).
void solve(owtk_solver_kind kind, Matrix& m, Preconditioner* pc, Vector& rhs, Vector& x,
           const owtk_solver_options& options, Workspace& ws, owtk_solver_result& result,
           const SolveExtras* extras = nullptr);

}  // namespace owtk

// The opaque handles of the C ABI are the runtime objects themselves.
struct owtk_context : owtk::Context {};
struct owtk_vector : owtk::Vector {};
struct owtk_matrix : owtk::Matrix {};
struct owtk_preconditioner : owtk::Preconditioner {};
struct owtk_workspace : owtk::Workspace {};
struct owtk_arnoldi_snapshot : owtk::ArnoldiSnapshot {};
struct owtk_permutation {
    owtk::Context* ctx = nullptr;
    std::size_t n = 0;
    std::vector<std::int64_t> new_to_old, old_to_new;
    owtk::DeviceBuffer d_new_to_old;
};
