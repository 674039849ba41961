// Test infrastructure only: a C-ABI harness around the UNMODIFIED OWT-Krylov
// reference headers.  It is compiled (never copied) from the read-only
// reference tree by oracle/Makefile into oracle/_ref/, and it is loaded only by
// tests, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm.
// Nothing in the product library links or calls it.
//
// Every entry point catches the reference's exceptions and turns them into the
// same status codes the product's C ABI uses (include/owtk.h), so a parity test
// can compare error behaviour as well as numbers.

#include <owt/krylov/block_csr.hpp>
#include <owt/krylov/core.hpp>
#include <owt/krylov/dense_block_csr.hpp>
#include <owt/krylov/execution.hpp>
#include <owt/krylov/idrs.hpp>
#include <owt/krylov/krylov_solvers.hpp>
#include <owt/krylov/ordering.hpp>
#include <owt/krylov/pipelined_bicgstab.hpp>
#include <owt/krylov/preconditioner.hpp>
#include <owt/krylov/reduction.hpp>
#include <owt/krylov/specwave_compat.hpp>
#include <owt/krylov/split_block_csr.hpp>

#include <cstdint>
#include <cstring>
#include <memory>
#include <optional>
#include <stdexcept>
#include <string>
#include <utility>
#include <variant>
#include <vector>

namespace ok = owt::krylov;

namespace {

thread_local std::string g_error;

enum Code {
    OK = 0,
    INVALID_ARGUMENT = 1,
    ZERO_PIVOT = 2,
    OUT_OF_RANGE = 3,
    RUNTIME = 7,
};

template<class F>
int guarded(F&& f)
{
    try {
        f();
        return OK;
    } catch (const std::invalid_argument& e) {
        g_error = e.what();
        return INVALID_ARGUMENT;
    } catch (const std::out_of_range& e) {
        g_error = e.what();
        return OUT_OF_RANGE;
    } catch (const std::runtime_error& e) {
        g_error = e.what();
        return std::string(e.what()).find("zero pivot") != std::string::npos
            ? ZERO_PIVOT : RUNTIME;
    } catch (const std::exception& e) {
        g_error = e.what();
        return RUNTIME;
    }
}

using Bsr = ok::BlockCsrMatrix<double>;
using Split = ok::SplitBlockCsrMatrixView<double>;
using Dense = ok::DenseBlockCsrMatrix<double>;

struct Matrix {
    int kind = 0;  // 0 component-diagonal BSR, 1 split view, 2 dense BSR
    std::size_t owned = 0, ghost = 0, bs = 0;
    // Split views borrow; keep their storage alive here.
    std::vector<std::size_t> rowptr, cols;
    std::vector<double> diag, off;
    std::unique_ptr<Bsr> bsr;
    std::unique_ptr<Split> split;
    std::unique_ptr<Dense> dense;
};

struct Pc {
    int kind = 0;  // 0 identity, 1 jacobi, 2 ssor, 3 split ssor, 4 ilu(k)
    Matrix* matrix = nullptr;
    std::unique_ptr<ok::JacobiPreconditioner<double>> jacobi;
    std::unique_ptr<ok::LocalSsorPreconditioner<double>> ssor;
    std::unique_ptr<ok::SplitLocalSsorPreconditioner<double>> split_ssor;
    std::unique_ptr<ok::IluLevelPreconditioner<double>> ilu;

    void apply(const ok::BlockVector<double>& in, ok::BlockVector<double>& out) const
    {
        switch (kind) {
        case 0: ok::IdentityPreconditioner{}.apply(in, out); break;
        case 1: jacobi->apply(in, out); break;
        case 2: ssor->apply(in, out); break;
        case 3: split_ssor->apply(in, out); break;
        case 4: ilu->apply(in, out); break;
        default: throw std::invalid_argument("unknown preconditioner kind");
        }
    }
};

// Forwarding preconditioner so the reference solvers see a plain object.
struct PcRef {
    const Pc* pc;
    void apply(const ok::BlockVector<double>& in, ok::BlockVector<double>& out) const
    {
        pc->apply(in, out);
    }
};

// Operator over whichever matrix form the handle holds (halo is a no-op).
struct Op {
    Matrix* m;
    void apply(ok::BlockVector<double>& in, ok::BlockVector<double>& out)
    {
        switch (m->kind) {
        case 0: ok::DistributedBlockOperator<Bsr&>(*m->bsr).apply(in, out); break;
        case 1: m->split->apply(in, out); break;
        case 2: m->dense->apply(in, out); break;
        default: throw std::invalid_argument("unknown matrix kind");
        }
    }
};

ok::BlockVector<double> view(const Matrix* m, const double* data)
{
    return ok::BlockVector<double>::view(
        m->owned, m->ghost, m->bs,
        std::span<double>(const_cast<double*>(data), (m->owned + m->ghost) * m->bs));
}

}  // namespace

extern "C" {

// Same field layout as owtk_solver_options / owtk_solver_result in include/owtk.h.
struct ref_options {
    double relative_tolerance;
    double absolute_tolerance;
    double breakdown_tolerance;
    std::uint64_t maximum_iterations;
    std::uint64_t convergence_check_interval;
    std::uint64_t restart;
    std::uint64_t residual_replacement_interval;
    std::uint64_t idr_shadow_space;
    double relaxation;
    std::int32_t verify_true_residual;
    std::int32_t gmres_orthogonalization;
};

struct ref_result {
    std::int32_t status;
    std::int32_t breakdown_reason;
    std::uint64_t iterations;
    std::uint64_t operator_applications;
    std::uint64_t preconditioner_applications;
    std::uint64_t global_reductions;
    std::uint64_t reorthogonalizations;
    std::uint64_t arnoldi_norm_verifications;
    double initial_residual_norm;
    double recursive_residual_norm;
    double true_residual_norm;
    double relative_residual_norm;
    std::int32_t converged_by_application;
    std::int32_t pad;
    double solve_seconds;
};

const char* ref_last_error() { return g_error.c_str(); }

void ref_default_options(ref_options* o)
{
    ok::SolverOptions<double> d;
    o->relative_tolerance = d.relative_tolerance;
    o->absolute_tolerance = d.absolute_tolerance;
    o->breakdown_tolerance = d.breakdown_tolerance;
    o->maximum_iterations = d.maximum_iterations;
    o->convergence_check_interval = d.convergence_check_interval;
    o->restart = d.restart;
    o->residual_replacement_interval = d.residual_replacement_interval;
    o->idr_shadow_space = d.idr_shadow_space;
    o->relaxation = d.relaxation;
    o->verify_true_residual = d.verify_true_residual ? 1 : 0;
    o->gmres_orthogonalization = static_cast<int>(d.gmres_orthogonalization);
}

int ref_bsr_create(std::size_t owned, std::size_t ghost, std::size_t bs,
                   const std::uint64_t* rowptr, const std::uint64_t* cols,
                   const double* vals, void** out)
{
    return guarded([&] {
        auto m = std::make_unique<Matrix>();
        m->kind = 0; m->owned = owned; m->ghost = ghost; m->bs = bs;
        const std::size_t nnz = rowptr[owned];
        m->bsr = std::make_unique<Bsr>(
            owned, ghost, bs,
            std::vector<std::size_t>(rowptr, rowptr + owned + 1),
            std::vector<std::size_t>(cols, cols + nnz),
            std::vector<double>(vals, vals + nnz * bs));
        *out = m.release();
    });
}

int ref_dense_create(std::size_t owned, std::size_t ghost, std::size_t bs,
                     const std::uint64_t* rowptr, const std::uint64_t* cols,
                     const double* vals, void** out)
{
    return guarded([&] {
        auto m = std::make_unique<Matrix>();
        m->kind = 2; m->owned = owned; m->ghost = ghost; m->bs = bs;
        const std::size_t nnz = rowptr[owned];
        m->dense = std::make_unique<Dense>(
            owned, ghost, bs,
            std::vector<std::size_t>(rowptr, rowptr + owned + 1),
            std::vector<std::size_t>(cols, cols + nnz),
            std::vector<double>(vals, vals + nnz * bs * bs));
        *out = m.release();
    });
}

int ref_split_create(std::size_t owned, std::size_t ghost, std::size_t bs,
                     const std::uint64_t* rowptr, const std::uint64_t* cols,
                     const double* diag, const double* off, void** out)
{
    return guarded([&] {
        auto m = std::make_unique<Matrix>();
        m->kind = 1; m->owned = owned; m->ghost = ghost; m->bs = bs;
        const std::size_t edges = rowptr[owned];
        m->rowptr.assign(rowptr, rowptr + owned + 1);
        m->cols.assign(cols, cols + edges);
        m->diag.assign(diag, diag + owned * bs);
        m->off.assign(off, off + edges * bs);
        m->split = std::make_unique<Split>(
            owned, ghost, bs, std::span<const std::size_t>(m->rowptr),
            std::span<const std::size_t>(m->cols), std::span<const double>(m->diag),
            std::span<const double>(m->off));
        *out = m.release();
    });
}

// Overwrite the borrowed split coefficients in place (visible without update).
int ref_split_set_values(void* h, const double* diag, const double* off)
{
    return guarded([&] {
        auto* m = static_cast<Matrix*>(h);
        if (m->kind != 1) throw std::invalid_argument("not a split view");
        std::memcpy(m->diag.data(), diag, m->diag.size() * sizeof(double));
        std::memcpy(m->off.data(), off, m->off.size() * sizeof(double));
    });
}

// Overwrite the values of an owning BSR matrix in place.
int ref_bsr_set_values(void* h, const double* vals)
{
    return guarded([&] {
        auto* m = static_cast<Matrix*>(h);
        if (m->kind != 0) throw std::invalid_argument("not a BSR matrix");
        auto values = m->bsr->values();
        std::memcpy(values.data(), vals, values.size() * sizeof(double));
    });
}

void ref_matrix_destroy(void* h) { delete static_cast<Matrix*>(h); }

int ref_matrix_apply(void* h, const double* x, double* y)
{
    return guarded([&] {
        auto* m = static_cast<Matrix*>(h);
        auto in = view(m, x);
        auto out = view(m, y);
        Op{m}.apply(in, out);
    });
}

int ref_matrix_diagonal(void* h, double* out)
{
    return guarded([&] {
        auto* m = static_cast<Matrix*>(h);
        std::vector<double> d;
        if (m->kind == 0) d = m->bsr->diagonal();
        else if (m->kind == 1) d = m->split->diagonal();
        else throw std::invalid_argument("dense BSR has no diagonal()");
        std::memcpy(out, d.data(), d.size() * sizeof(double));
    });
}

int ref_pc_create(int kind, void* matrix, double parameter, void** out)
{
    return guarded([&] {
        auto* m = static_cast<Matrix*>(matrix);
        auto pc = std::make_unique<Pc>();
        pc->kind = kind;
        pc->matrix = m;
        switch (kind) {
        case 0: break;
        case 1:
            if (m->kind == 0) pc->jacobi = std::make_unique<ok::JacobiPreconditioner<double>>(*m->bsr);
            else if (m->kind == 1) pc->jacobi = std::make_unique<ok::JacobiPreconditioner<double>>(*m->split);
            else throw std::invalid_argument("Jacobi needs a matrix with diagonal()");
            break;
        case 2:
            if (m->kind != 0) throw std::invalid_argument("SSOR needs a component-diagonal BSR");
            pc->ssor = std::make_unique<ok::LocalSsorPreconditioner<double>>(*m->bsr, parameter);
            break;
        case 3:
            if (m->kind != 1) throw std::invalid_argument("split SSOR needs a split view");
            pc->split_ssor = std::make_unique<ok::SplitLocalSsorPreconditioner<double>>(*m->split, parameter);
            break;
        case 4:
            if (m->kind != 0) throw std::invalid_argument("ILU needs a component-diagonal BSR");
            pc->ilu = std::make_unique<ok::IluLevelPreconditioner<double>>(
                *m->bsr, static_cast<std::size_t>(parameter));
            break;
        default: throw std::invalid_argument("unknown preconditioner kind");
        }
        *out = pc.release();
    });
}

void ref_pc_destroy(void* h) { delete static_cast<Pc*>(h); }

int ref_pc_apply(void* h, const double* in, double* out)
{
    return guarded([&] {
        auto* pc = static_cast<Pc*>(h);
        auto vin = view(pc->matrix, in);
        auto vout = view(pc->matrix, out);
        pc->apply(vin, vout);
    });
}

int ref_pc_update_values(void* h)
{
    return guarded([&] {
        auto* pc = static_cast<Pc*>(h);
        Matrix* m = pc->matrix;
        switch (pc->kind) {
        case 1:
            if (m->kind == 0) pc->jacobi->update_values(*m->bsr);
            else pc->jacobi->update_values(*m->split);
            break;
        case 2: pc->ssor->update_values(); break;
        case 3: pc->split_ssor->update_values(*m->split); break;
        case 4: pc->ilu->update_values(*m->bsr); break;
        default: break;
        }
    });
}

std::uint64_t ref_pc_numeric_updates(void* h)
{
    auto* pc = static_cast<Pc*>(h);
    switch (pc->kind) {
    case 1: return pc->jacobi->numeric_updates();
    case 2: return pc->ssor->numeric_updates();
    case 3: return pc->split_ssor->numeric_updates();
    case 4: return pc->ilu->numeric_updates();
    default: return 0;
    }
}

// ILU factor storage; call with null arrays first to learn the entry count.
int ref_ilu_factors(void* h, std::uint64_t* entries, std::uint64_t* rowptr,
                    std::uint64_t* cols, double* vals, double* inverse_diagonal)
{
    return guarded([&] {
        auto* pc = static_cast<Pc*>(h);
        if (pc->kind != 4) throw std::invalid_argument("not an ILU preconditioner");
        auto r = pc->ilu->factor_row_offsets();
        auto c = pc->ilu->factor_columns();
        auto v = pc->ilu->factor_values();
        auto d = pc->ilu->inverse_diagonal();
        *entries = c.size();
        if (rowptr) for (std::size_t i = 0; i < r.size(); ++i) rowptr[i] = r[i];
        if (cols) for (std::size_t i = 0; i < c.size(); ++i) cols[i] = c[i];
        if (vals) std::memcpy(vals, v.data(), v.size() * sizeof(double));
        if (inverse_diagonal) std::memcpy(inverse_diagonal, d.data(), d.size() * sizeof(double));
    });
}

void* ref_workspace_create() { return new ok::SolverWorkspace<double>(); }
void ref_workspace_destroy(void* w) { delete static_cast<ok::SolverWorkspace<double>*>(w); }
std::uint64_t ref_workspace_epochs(void* w)
{
    return static_cast<ok::SolverWorkspace<double>*>(w)->allocation_epochs();
}
int ref_workspace_vector(void* w, std::size_t index, double* out)
{
    return guarded([&] {
        auto& v = static_cast<ok::SolverWorkspace<double>*>(w)->vector(index);
        std::memcpy(out, v.data(), v.owned_size() * sizeof(double));
    });
}

// solver: 0 gmres/fgmres, 1 bicgstab, 2 pipelined bicgstab,
//         3 communication-hiding bicgstab, 4 idrs
// reduction: 0 serial, 1 compensated, 2 mixed precision (long double)
int ref_solve(int solver, int reduction, void* matrix, void* pc_handle,
              const ref_options* o, const double* rhs, double* x, void* workspace,
              ref_result* out)
{
    return guarded([&] {
        auto* m = static_cast<Matrix*>(matrix);
        const Pc* pc = static_cast<Pc*>(pc_handle);
        ok::SolverOptions<double> opt;
        opt.relative_tolerance = o->relative_tolerance;
        opt.absolute_tolerance = o->absolute_tolerance;
        opt.breakdown_tolerance = o->breakdown_tolerance;
        opt.maximum_iterations = o->maximum_iterations;
        opt.convergence_check_interval = o->convergence_check_interval;
        opt.restart = o->restart;
        opt.residual_replacement_interval = o->residual_replacement_interval;
        opt.idr_shadow_space = o->idr_shadow_space;
        opt.relaxation = o->relaxation;
        opt.verify_true_residual = o->verify_true_residual != 0;
        opt.collect_timings = true;
        opt.gmres_orthogonalization =
            static_cast<ok::GmresOrthogonalization>(o->gmres_orthogonalization);
        auto vb = view(m, rhs);
        auto vx = view(m, x);
        Op op{m};
        auto* ws = static_cast<ok::SolverWorkspace<double>*>(workspace);
        ok::SolverResult<double> r;
        auto run = [&](auto red) {
            switch (solver) {
            case 0: r = ok::fgmres(op, vb, vx, opt, PcRef{pc}, red, ws); break;
            case 1: r = ok::bicgstab(op, vb, vx, opt, PcRef{pc}, red, ws); break;
            case 2: r = ok::pipelined_bicgstab(op, vb, vx, opt, PcRef{pc}, red, ws); break;
            case 3: r = ok::communication_hiding_bicgstab(op, vb, vx, opt, PcRef{pc}, red, ws); break;
            case 4: r = ok::idrs(op, vb, vx, opt, PcRef{pc}, red); break;
            default: throw std::invalid_argument("unknown solver");
            }
        };
        if (reduction == 1) run(ok::CompensatedSerialReduction<double>{});
        else if (reduction == 2) run(ok::MixedPrecisionSerialReduction<double>{});
        else run(ok::SerialReduction<double>{});
        out->status = static_cast<std::int32_t>(r.status);
        out->breakdown_reason = static_cast<std::int32_t>(r.breakdown_reason);
        out->iterations = r.iterations;
        out->operator_applications = r.operator_applications;
        out->preconditioner_applications = r.preconditioner_applications;
        out->global_reductions = r.global_reductions;
        out->reorthogonalizations = r.reorthogonalizations;
        out->arnoldi_norm_verifications = r.arnoldi_norm_verifications;
        out->initial_residual_norm = r.initial_residual_norm;
        out->recursive_residual_norm = r.recursive_residual_norm;
        out->true_residual_norm = r.true_residual_norm;
        out->relative_residual_norm = r.relative_residual_norm;
        out->converged_by_application = r.converged_by_application ? 1 : 0;
        out->solve_seconds = r.solve_seconds();
    });
}

namespace {
ok::SolverOptions<double> options_of(const ref_options* o)
{
    ok::SolverOptions<double> opt;
    opt.relative_tolerance = o->relative_tolerance;
    opt.absolute_tolerance = o->absolute_tolerance;
    opt.breakdown_tolerance = o->breakdown_tolerance;
    opt.maximum_iterations = o->maximum_iterations;
    opt.convergence_check_interval = o->convergence_check_interval;
    opt.restart = o->restart;
    opt.residual_replacement_interval = o->residual_replacement_interval;
    opt.idr_shadow_space = o->idr_shadow_space;
    opt.relaxation = o->relaxation;
    opt.verify_true_residual = o->verify_true_residual != 0;
    opt.collect_timings = true;
    opt.gmres_orthogonalization = static_cast<ok::GmresOrthogonalization>(o->gmres_orthogonalization);
    return opt;
}

void result_of(const ok::SolverResult<double>& r, ref_result* out)
{
    out->status = static_cast<std::int32_t>(r.status);
    out->breakdown_reason = static_cast<std::int32_t>(r.breakdown_reason);
    out->iterations = r.iterations;
    out->operator_applications = r.operator_applications;
    out->preconditioner_applications = r.preconditioner_applications;
    out->global_reductions = r.global_reductions;
    out->reorthogonalizations = r.reorthogonalizations;
    out->arnoldi_norm_verifications = r.arnoldi_norm_verifications;
    out->initial_residual_norm = r.initial_residual_norm;
    out->recursive_residual_norm = r.recursive_residual_norm;
    out->true_residual_norm = r.true_residual_norm;
    out->relative_residual_norm = r.relative_residual_norm;
    out->converged_by_application = r.converged_by_application ? 1 : 0;
    out->solve_seconds = r.solve_seconds();
}
}  // namespace

// ref_solve with the two optional inputs of the reference's solvers: an
// application convergence test that stops at iteration `stop_at` (0: none;
// core.hpp:102-108) and, for FGMRES, an ArnoldiSnapshot (core.hpp:462-534)
// whose columns, Hessenberg entries h(row, col) (column-major, restart + 1
// rows) and owned preconditioned-basis values are copied out.
int ref_solve_ex(int solver, int reduction, void* matrix, void* pc_handle, const ref_options* o,
                 const double* rhs, double* x, std::uint64_t stop_at, std::uint64_t* snapshot_columns,
                 double* snapshot_h, double* snapshot_basis, ref_result* out)
{
    return guarded([&] {
        auto* m = static_cast<Matrix*>(matrix);
        const Pc* pc = static_cast<Pc*>(pc_handle);
        ok::SolverOptions<double> opt = options_of(o);
        if (stop_at > 0)
            opt.convergence_test = [stop_at](std::size_t it, const ok::BlockVector<double>&) { return it >= stop_at; };
        auto vb = view(m, rhs);
        auto vx = view(m, x);
        Op op{m};
        ok::ArnoldiSnapshot<double> snap;
        ok::SolverResult<double> r;
        auto run = [&](auto red) {
            switch (solver) {
            case 0: r = ok::fgmres(op, vb, vx, opt, PcRef{pc}, red, static_cast<ok::SolverWorkspace<double>*>(nullptr), snapshot_columns ? &snap : nullptr); break;
            case 1: r = ok::bicgstab(op, vb, vx, opt, PcRef{pc}, red); break;
            case 2: r = ok::pipelined_bicgstab(op, vb, vx, opt, PcRef{pc}, red); break;
            case 3: r = ok::communication_hiding_bicgstab(op, vb, vx, opt, PcRef{pc}, red); break;
            case 4: r = ok::idrs(op, vb, vx, opt, PcRef{pc}, red); break;
            default: throw std::invalid_argument("unknown solver");
            }
        };
        if (reduction == 1) run(ok::CompensatedSerialReduction<double>{});
        else if (reduction == 2) run(ok::MixedPrecisionSerialReduction<double>{});
        else run(ok::SerialReduction<double>{});
        result_of(r, out);
        if (snapshot_columns) {
            const std::size_t cols = snap.columns(), R = o->restart, n = m->owned * m->bs;
            *snapshot_columns = cols;
            for (std::size_t c = 0; c < cols; ++c) {
                for (std::size_t row = 0; row <= cols; ++row) snapshot_h[c * (R + 1) + row] = snap.h(row, c);
                const auto& z = snap.preconditioned_basis(c);
                std::copy(z.owned().begin(), z.owned().end(), snapshot_basis + c * n);
            }
        }
    });
}

// solve_specwave_native (specwave_compat.hpp:99-249) on a component-diagonal
// BSR handle with its operator and no halo.
int ref_solve_specwave(int solver_id, void* matrix, const ref_options* o, const double* rhs, double* x,
                       ref_result* out)
{
    return guarded([&] {
        auto* m = static_cast<Matrix*>(matrix);
        if (m->kind != 0) throw std::invalid_argument("SpecWave dispatch needs a component-diagonal BSR");
        auto vb = view(m, rhs);
        auto vx = view(m, x);
        ok::DistributedBlockOperator<Bsr&> op(*m->bsr);
        ok::NoHaloExchange halo;
        const auto r = ok::solve_specwave_native(static_cast<ok::SpecWaveSolver>(solver_id), *m->bsr, op, halo, vb,
                                                 vx, options_of(o));
        result_of(r, out);
    });
}

// dot and norm with a chosen reduction (0 serial, 1 compensated, 2 mixed
// precision); the mixed local_dot's long double is returned as hi + lo.
double ref_dot_kind(int kind, std::size_t owned, std::size_t ghost, std::size_t bs, const double* a,
                    const double* b, double* low)
{
    const std::size_t n = (owned + ghost) * bs;
    auto va = ok::BlockVector<double>::view(owned, ghost, bs, std::span<double>(const_cast<double*>(a), n));
    auto vb = ok::BlockVector<double>::view(owned, ghost, bs, std::span<double>(const_cast<double*>(b), n));
    if (low) *low = 0.0;
    if (kind == 1) return ok::CompensatedSerialReduction<double>{}.dot(va, vb);
    if (kind == 2) {
        const long double w = ok::MixedPrecisionSerialReduction<double>{}.local_dot(va, vb);
        const double hi = static_cast<double>(w);
        if (low) *low = static_cast<double>(w - static_cast<long double>(hi));
        return hi;
    }
    return ok::SerialReduction<double>{}.dot(va, vb);
}

double ref_norm_kind(int kind, std::size_t owned, std::size_t ghost, std::size_t bs, const double* a)
{
    const std::size_t n = (owned + ghost) * bs;
    auto va = ok::BlockVector<double>::view(owned, ghost, bs, std::span<double>(const_cast<double*>(a), n));
    if (kind == 1) return ok::CompensatedSerialReduction<double>{}.norm(va);
    if (kind == 2) return ok::MixedPrecisionSerialReduction<double>{}.norm(va);
    return ok::SerialReduction<double>{}.norm(va);
}

double ref_dot(std::size_t owned, std::size_t ghost, std::size_t bs,
               const double* a, const double* b)
{
    const std::size_t n = (owned + ghost) * bs;
    auto va = ok::BlockVector<double>::view(owned, ghost, bs,
        std::span<double>(const_cast<double*>(a), n));
    auto vb = ok::BlockVector<double>::view(owned, ghost, bs,
        std::span<double>(const_cast<double*>(b), n));
    return ok::SerialReduction<double>{}.dot(va, vb);
}

double ref_norm(std::size_t owned, std::size_t ghost, std::size_t bs, const double* a)
{
    const std::size_t n = (owned + ghost) * bs;
    auto va = ok::BlockVector<double>::view(owned, ghost, bs,
        std::span<double>(const_cast<double*>(a), n));
    return ok::SerialReduction<double>{}.norm(va);
}

// Reverse Cuthill-McKee over the owned graph of a BSR pattern (bs irrelevant).
int ref_rcm(std::size_t owned, std::size_t ghost, const std::uint64_t* rowptr,
            const std::uint64_t* cols, std::uint64_t* out)
{
    return guarded([&] {
        const std::size_t nnz = rowptr[owned];
        Bsr m(owned, ghost, 1, std::vector<std::size_t>(rowptr, rowptr + owned + 1),
              std::vector<std::size_t>(cols, cols + nnz), std::vector<double>(nnz, 0.0));
        const auto order = ok::reverse_cuthill_mckee_order(m);
        for (std::size_t i = 0; i < order.size(); ++i) out[i] = order[i];
    });
}

int ref_hilbert(std::size_t n, const double* xy, std::uint64_t* out)
{
    return guarded([&] {
        std::vector<std::pair<double, double>> c(n);
        for (std::size_t i = 0; i < n; ++i) c[i] = {xy[2 * i], xy[2 * i + 1]};
        const auto order = ok::hilbert_order(c);
        for (std::size_t i = 0; i < order.size(); ++i) out[i] = order[i];
    });
}

int ref_inverse_permutation(std::size_t n, const std::uint64_t* in, std::uint64_t* out)
{
    return guarded([&] {
        std::vector<std::size_t> p(in, in + n);
        const auto inv = ok::inverse_permutation(p);
        for (std::size_t i = 0; i < n; ++i) out[i] = inv[i];
    });
}

}  // extern "C"
