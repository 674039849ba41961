// A reference-style consumer of the header-only API: the same calls an
// OWT-Krylov application makes (BlockCsrMatrix, PolicyBlockOperator, Ilu0 /
// Jacobi / split SSOR preconditioners, gmres / bicgstab / idrs, RCM), with
// the device execution policy.  Reads a system written by the test, writes the
// results back for comparison with the CPU oracle.
//
//   consumer <dir>   (dir holds meta.txt, rowptr.u64, cols.u64, vals.f64, rhs.f64)
#include <owtk/krylov.hpp>

#include <cstdio>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

using namespace owt::krylov;

template<class V>
V read(const std::string& path, std::size_t n)
{
    V v(n);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char*>(v.data()), static_cast<std::streamsize>(n * sizeof(typename V::value_type)));
    if (!f) throw std::runtime_error("cannot read " + path);
    return v;
}

template<class V>
void write(const std::string& path, const V& v)
{
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), static_cast<std::streamsize>(v.size() * sizeof(v[0])));
}

template<class R>
void report(std::ostream& out, const char* name, const R& r)
{
    out << name << ' ' << static_cast<int>(r.status) << ' ' << static_cast<int>(r.breakdown_reason) << ' '
        << r.iterations << ' ' << r.operator_applications << ' ' << r.preconditioner_applications << ' '
        << r.global_reductions << ' ' << r.true_residual_norm << '\n';
}

int main(int argc, char** argv)
{
    if (argc < 2) return 2;
    const std::string dir = argv[1];
    std::size_t n = 0, bs = 0, nnz = 0;
    {
        std::ifstream meta(dir + "/meta.txt");
        meta >> n >> bs >> nnz;
    }
    BlockCsrMatrix<double> A(n, 0, bs, read<std::vector<std::size_t>>(dir + "/rowptr.u64", n + 1),
                             read<std::vector<std::size_t>>(dir + "/cols.u64", nnz),
                             read<std::vector<double>>(dir + "/vals.f64", nnz * bs));
    BlockVector<double> rhs(n, 0, bs);
    const auto b = read<std::vector<double>>(dir + "/rhs.f64", n * bs);
    std::copy(b.begin(), b.end(), rhs.data());

    // The only change from a host consumer: the execution policy.
    PolicyBlockOperator op(A, CudaExecutionPolicy{});

    std::ofstream results(dir + "/results.txt");
    BlockVector<double> y = rhs.clone_layout();
    op.apply(rhs, y);
    write(dir + "/spmv.f64", std::vector<double>(y.owned().begin(), y.owned().end()));
    // apply_rows (block_csr.hpp:198-215): every third row, last to first;
    // the other rows keep the 7.0 they start with.
    {
        BlockVector<double> z = rhs.clone_layout();
        std::fill(z.data(), z.data() + z.local_size(), 7.0);
        std::vector<std::size_t> rows;
        for (std::size_t r = n; r-- > 0;)
            if (r % 3 == 0) rows.push_back(r);
        A.apply_rows(rhs, z, rows);
        write(dir + "/spmv_rows.f64", std::vector<double>(z.owned().begin(), z.owned().end()));
    }

    Ilu0Preconditioner ilu(A);
    SolverOptions<double> options;
    SolverWorkspace<double> workspace;
    BlockVector<double> x1 = rhs.clone_layout();
    const auto r1 = gmres(op, rhs, x1, options, ilu, SerialReduction<double>{}, &workspace);
    report(results, "gmres_ilu0", r1);
    write(dir + "/x_gmres.f64", std::vector<double>(x1.owned().begin(), x1.owned().end()));

    JacobiPreconditioner jacobi(A);
    SolverOptions<double> bench = options;
    bench.convergence_check_interval = 1;
    BlockVector<double> x2 = rhs.clone_layout();
    const auto r2 = bicgstab_with_workspace(op, rhs, x2, workspace, bench, jacobi);
    report(results, "bicgstab_jacobi", r2);
    write(dir + "/x_bicgstab.f64", std::vector<double>(x2.owned().begin(), x2.owned().end()));

    BlockVector<double> x3 = rhs.clone_layout();
    const auto r3 = idrs(op, rhs, x3, bench, jacobi);
    report(results, "idrs_jacobi", r3);

    // Split diagonal/edge view and split SSOR over borrowed host arrays.
    std::vector<std::size_t> off_rp{0}, off_ci;
    std::vector<double> diag(n * bs), off;
    for (std::size_t r = 0; r < n; ++r) {
        for (std::size_t e = A.row_offsets()[r]; e < A.row_offsets()[r + 1]; ++e) {
            const std::size_t c = A.column_indices()[e];
            const double* v = A.values().data() + e * bs;
            if (c == r) std::copy(v, v + bs, diag.data() + r * bs);
            else {
                off_ci.push_back(c);
                off.insert(off.end(), v, v + bs);
            }
        }
        off_rp.push_back(off_ci.size());
    }
    SplitBlockCsrMatrixView<double> split(n, 0, bs, std::span<const std::size_t>(off_rp),
                                          std::span<const std::size_t>(off_ci), std::span<const double>(diag),
                                          std::span<const double>(off));
    SplitLocalSsorPreconditioner<double> ssor(split, 1.2);
    BlockVector<double> z = rhs.clone_layout();
    ssor.apply(rhs, z);
    write(dir + "/split_ssor.f64", std::vector<double>(z.owned().begin(), z.owned().end()));

    // The SpecWave dispatcher with the same operator (legacy id 9).
    NoHaloExchange halo;
    BlockVector<double> x4 = rhs.clone_layout();
    const auto r4 = solve_specwave_native(SpecWaveSolver::bicgstab_ilu0, A, op, halo, rhs, x4, options);
    report(results, "specwave_bicgstab_ilu0", r4);
    write(dir + "/x_specwave.f64", std::vector<double>(x4.owned().begin(), x4.owned().end()));
    try {
        BlockVector<double> x5 = rhs.clone_layout();
        (void)solve_specwave_native(SpecWaveSolver::multigrid_w, A, op, halo, rhs, x5, options);
        results << "specwave_multigrid accepted\n";
    } catch (const std::invalid_argument&) {
        results << "specwave_multigrid invalid_argument\n";
    }

    // The stability variants (krylov_solvers.hpp:766-809,
    // pipelined_bicgstab.hpp:275-313, :620-661).
    auto variant = [&](const std::string& name, auto&& solve) {
        BlockVector<double> xv = rhs.clone_layout();
        const auto r = solve(xv);
        report(results, name.c_str(), r);
        write(dir + "/x_" + name + ".f64", std::vector<double>(xv.owned().begin(), xv.owned().end()));
    };
    variant("bicgstab_stable", [&](auto& xv) { return bicgstab_stable(op, rhs, xv, options, ilu); });
    variant("bicgstab_residual_replacement",
            [&](auto& xv) { return bicgstab_residual_replacement(op, rhs, xv, options, 7, ilu); });
    variant("bicgstab_mixed_precision", [&](auto& xv) { return bicgstab_mixed_precision(op, rhs, xv, options, ilu); });
    variant("pipelined_bicgstab_stable", [&](auto& xv) { return pipelined_bicgstab_stable(op, rhs, xv, options, ilu); });
    variant("pipelined_bicgstab_residual_replacement",
            [&](auto& xv) { return pipelined_bicgstab_residual_replacement(op, rhs, xv, options, 7, ilu); });
    variant("pipelined_bicgstab_mixed_precision",
            [&](auto& xv) { return pipelined_bicgstab_mixed_precision(op, rhs, xv, options, ilu); });
    variant("communication_hiding_bicgstab_stable",
            [&](auto& xv) { return communication_hiding_bicgstab_stable(op, rhs, xv, options, ilu); });
    variant("communication_hiding_bicgstab_residual_replacement",
            [&](auto& xv) { return communication_hiding_bicgstab_residual_replacement(op, rhs, xv, options, 7, ilu); });
    variant("communication_hiding_bicgstab_mixed_precision",
            [&](auto& xv) { return communication_hiding_bicgstab_mixed_precision(op, rhs, xv, options, ilu); });

    // FGMRES recording its last Arnoldi relation (restart 6: several cycles).
    ArnoldiSnapshot<double> snapshot;
    SolverOptions<double> small = options;
    small.restart = 6;
    BlockVector<double> x6 = rhs.clone_layout();
    const auto r6 = fgmres(op, rhs, x6, small, ilu, SerialReduction<double>{}, static_cast<SolverWorkspace<double>*>(nullptr), &snapshot);
    report(results, "fgmres_snapshot", r6);
    results << "snapshot_columns " << snapshot.columns() << '\n';
    {
        std::vector<double> h, z;
        for (std::size_t c = 0; c < snapshot.columns(); ++c) {
            for (std::size_t row = 0; row <= c + 1; ++row) h.push_back(snapshot.h(row, c));
            const auto& v = snapshot.preconditioned_basis(c);
            z.insert(z.end(), v.owned().begin(), v.owned().end());
        }
        write(dir + "/snapshot_h.f64", h);
        write(dir + "/snapshot_basis.f64", z);
        try {
            (void)snapshot.h(0, snapshot.columns());
            results << "snapshot_range none\n";
        } catch (const std::out_of_range&) {
            results << "snapshot_range out_of_range\n";
        }
    }

    // An application convergence test that stops at iteration 5.
    SolverOptions<double> app = options;
    std::size_t calls = 0;
    app.convergence_test = [&calls](std::size_t iteration, const BlockVector<double>&) {
        ++calls;
        return iteration >= 5;
    };
    BlockVector<double> x7 = rhs.clone_layout();
    const auto r7 = bicgstab(op, rhs, x7, app, ilu);
    report(results, "bicgstab_application_test", r7);
    results << "application " << (r7.converged_by_application ? 1 : 0) << ' ' << calls << '\n';

    // A matrix-free operator and a host preconditioner of the application's
    // own types (any type with apply), as the reference's templates accept.
    struct HostSpmv {
        const BlockCsrMatrix<double>* A;
        void apply(BlockVector<double>& in, BlockVector<double>& out) const
        {
            const std::size_t b = A->block_size();
            for (std::size_t r = 0; r < A->owned_nodes(); ++r)
                for (std::size_t c = 0; c < b; ++c) {
                    double sum = 0;
                    for (std::size_t e = A->row_offsets()[r]; e < A->row_offsets()[r + 1]; ++e)
                        sum += A->values()[e * b + c] * in.data()[A->column_indices()[e] * b + c];
                    out.data()[r * b + c] = sum;
                }
        }
    };
    struct HostJacobi {
        std::vector<double> inverse;
        void apply(const BlockVector<double>& in, BlockVector<double>& out) const
        {
            for (std::size_t i = 0; i < inverse.size(); ++i) out.data()[i] = inverse[i] * in.data()[i];
        }
    };
    HostJacobi host_jacobi;
    for (double d : A.diagonal()) host_jacobi.inverse.push_back(1.0 / d);
    HostSpmv host_op{&A};
    BlockVector<double> x8 = rhs.clone_layout();
    const auto r8 = bicgstab(host_op, rhs, x8, bench, host_jacobi);
    report(results, "bicgstab_matrix_free", r8);
    write(dir + "/x_matrix_free.f64", std::vector<double>(x8.owned().begin(), x8.owned().end()));

    // Owned-only vector operations (core.hpp:562-601).
    BlockVector<double> u = rhs.clone_layout();
    for (std::size_t i = 0; i < u.owned_size(); ++i) u.data()[i] = 0.25 * static_cast<double>(i % 17) - 1.5;
    axpy(0.37, rhs, u);
    scale(-1.7, u);
    BlockVector<double> w = rhs.clone_layout();
    assign_linear_combination(w, 0.5, rhs, -1.25, u);
    write(dir + "/blas_u.f64", std::vector<double>(u.owned().begin(), u.owned().end()));
    write(dir + "/blas_w.f64", std::vector<double>(w.owned().begin(), w.owned().end()));

    // The three reductions on the same pair.
    results << std::hexfloat;
    results << "dot_serial " << SerialReduction<double>{}.dot(rhs, u) << '\n';
    results << "dot_compensated " << CompensatedSerialReduction<double>{}.dot(rhs, u) << '\n';
    results << "dot_mixed " << MixedPrecisionSerialReduction<double>{}.dot(rhs, u) << '\n';
    results << "norm_mixed " << MixedPrecisionSerialReduction<double>{}.norm(u) << '\n';
    results << std::defaultfloat;

    const auto order = reverse_cuthill_mckee_order(A);
    write(dir + "/rcm.u64", order);
    results << "epochs " << workspace.allocation_epochs() << '\n';
    results << "ilu_updates " << ilu.numeric_updates() << '\n';
    try {
        BlockVector<double> wrong(n + 1, 0, bs);
        ilu.apply(rhs, wrong);
        results << "layout_error none\n";
    } catch (const std::invalid_argument&) {
        results << "layout_error invalid_argument\n";
    }
    return 0;
}
