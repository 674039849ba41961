// Krylov solver recurrences over device-resident vectors.
//
// The control flow, breakdown guards and work counters follow the reference
// solvers statement by statement (anchors below); every vector operation is a
// device kernel and every reduction a device two-stage reduction whose scalar
// result the host reads after one stream synchronisation, at exactly the
// points where the reference branches on it.  Scalars stay in T like the
// reference's.  Workspace slot order matches the reference, so a caller can
// inspect the same vectors.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <random>
#include <vector>

#include "owtk_internal.h"

namespace owtk {
namespace {

enum Status { kConverged = 0, kMaxIterations = 1, kBreakdown = 2, kDiverged = 3, kInvalid = 4 };
enum Reason {
    kNone = 0, kArnoldi = 1, kSingular = 2, kBiorthogonality = 3, kAlphaDen = 4, kOmegaDen = 5,
    kOmegaZero = 6, kIdrShadow = 7, kIdrSmall = 8, kNonFinite = 9
};

// Scalar slots in the context's mapped block.
constexpr int kSlotA = 0;      // first reduction batch
constexpr int kSlotB = 128;    // second Gram-Schmidt batch
constexpr int kSlotCoef = 256; // coefficients uploaded for update kernels
constexpr int kSlotScratch = 508;   // two device doubles for the accurate norm

template<class T>
struct Engine {
    Context& c;
    Matrix& A;
    Preconditioner* M;
    std::size_t n;                 // owned values
    owtk_solver_result& res;
    const owtk_solver_options& o;
    const SolveExtras* ex = nullptr;
    std::vector<unsigned char> candidate_host;          // host copy for the convergence test
    std::unique_ptr<Vector> app_residual, app_work;     // its true-residual vectors

    int mode() const { return ex ? ex->reduction : 0; }
    bool has_test() const { return ex != nullptr && ex->test != nullptr; }

    T* p(Vector& v) const { return static_cast<T*>(v.data); }
    const T* p(const Vector& v) const { return static_cast<const T*>(v.data); }
    T scalar(int slot) const { return static_cast<T>(c.host_scalars[slot]); }
    double* dslot(int slot) const { return c.dev_scalar_copy.as<double>() + slot; }
    double* hslot(int slot) const { return c.dev_scalars + slot; }

    void op(Vector& in, Vector& out) { apply_operator(A, in, out); ++res.operator_applications; }
    void pc(Vector& in, Vector& out) { apply_preconditioner(M, in, out); ++res.preconditioner_applications; }
    // out = M in, then az = A out.  The learned preconditioner bound to this
    // operator forms A out for its residual check; it then writes it to az
    // (the same SpMV, so the same bits) and the second product is skipped.
    void pc_op(Vector& in, Vector& out, Vector& az)
    {
        if (M != nullptr && M->kind == OWTK_PC_LEARNED && learned_matrix(*M) == &A && A.dtype == OWTK_F64
            && az.dtype == OWTK_F64 && az.same_layout(in)) {
            matrix_layout_check_f64(A, out, az);
            ++res.preconditioner_applications;
            if (apply_preconditioner_product(M, in, out, static_cast<double*>(az.data))) {
                ++res.operator_applications;
                return;
            }
            op(out, az);
            return;
        }
        pc(in, out);
        op(out, az);
    }

    // k dot products of (a[j], b[j]) in one pass; values in slots [slot, slot+k).
    void dots(int k, Vector* const* a, Vector* const* b, int slot = kSlotA)
    {
        const T* pa[kMaxBatch];
        const T* pb[kMaxBatch];
        for (int j = 0; j < k; ++j) { pa[j] = p(*a[j]); pb[j] = p(*b[j]); }
        if (mode() != 0) kern::multidot_accurate<T>(c, n, k, mode(), pa, pb, dslot(slot), hslot(slot), nullptr);
        else kern::multidot<T>(c, n, k, pa, pb, dslot(slot), hslot(slot));
        c.sync();
    }
    T dot(Vector& a, Vector& b)
    {
        ++res.global_reductions;
        Vector* pa[1] = {&a};
        Vector* pb[1] = {&b};
        dots(1, pa, pb);
        return scalar(kSlotA);
    }
    T norm_nocount(Vector& v)
    {
        // The compensated reduction keeps the serial scaled norm
        // (reduction.hpp:217-220); the mixed-precision one widens it (:283-286).
        if (mode() == 2) kern::norm_accurate<T>(c, n, p(v), dslot(kSlotScratch), dslot(kSlotA), hslot(kSlotA));
        else kern::norm<T>(c, n, p(v), dslot(kSlotA), hslot(kSlotA));
        c.sync();
        return scalar(kSlotA);
    }
    T norm(Vector& v)
    {
        ++res.global_reductions;
        return norm_nocount(v);
    }
    // krylov_solvers.hpp:95-108
    T norm_from_squared(Vector& v, T squared)
    {
        if (std::isfinite(squared) && squared >= std::numeric_limits<T>::min()) return std::sqrt(squared);
        return norm(v);
    }
    // krylov_solvers.hpp:62-74
    void true_residual(Vector& b, Vector& x, Vector& r, Vector& work)
    {
        op(x, work);
        kern::sub<T>(c, n, p(b), p(work), p(r));
    }
    void copy(Vector& s, Vector& d) { kern::copy<T>(c, n, p(s), p(d)); }
    void fill(Vector& v, T value) { kern::fill<T>(c, n, value, p(v)); }
    void axpy(T a, Vector& x, Vector& y) { kern::axpy<T>(c, n, a, p(x), p(y)); }
    void scale(T a, Vector& x) { kern::scale<T>(c, n, a, p(x)); }

    void breakdown(int reason)
    {
        res.status = kBreakdown;
        res.breakdown_reason = reason;
    }
    // krylov_solvers.hpp:110-120
    void set_residuals(T recursive, T true_norm, T rhs_norm)
    {
        res.recursive_residual_norm = recursive;
        res.true_residual_norm = true_norm;
        res.relative_residual_norm = static_cast<double>(true_norm / (rhs_norm > T(0) ? rhs_norm : T(1)));
    }
    // core.hpp:549-560: an application convergence test replaces the tolerance.
    T threshold(T rhs_norm) const
    {
        const T rel = static_cast<T>(o.relative_tolerance) * (rhs_norm > T(0) ? rhs_norm : T(1));
        if (!std::isfinite(rhs_norm) || !std::isfinite(rel)) return std::numeric_limits<T>::quiet_NaN();
        if (has_test()) return T(0);
        return std::max(static_cast<T>(o.absolute_tolerance), rel);
    }
    // krylov_solvers.hpp:122-143: ask the application whether `candidate`
    // solves the problem; if so, measure its true residual (one operator
    // application, two norms) and finish as converged by the application.
    bool app_converged(Vector& b, Vector& candidate)
    {
        if (!has_test()) return false;
        const std::size_t count = candidate.local_size();
        candidate_host.resize(count * candidate.elem());
        OWTK_CUDA(cudaMemcpyAsync(candidate_host.data(), candidate.data, candidate_host.size(),
                                  cudaMemcpyDeviceToHost, c.stream));
        c.sync();
        const int answer = ex->test(ex->user, res.iterations, candidate_host.data(), count);
        if (answer < 0) fail(OWTK_ERR_RUNTIME, "application convergence test failed");
        if (answer == 0) return false;
        if (!app_residual) {
            app_residual = make_vector_like(candidate);
            app_work = make_vector_like(candidate);
        }
        true_residual(b, candidate, *app_residual, *app_work);
        const T rhs_norm = norm(b);
        const T true_norm = norm(*app_residual);
        set_residuals(static_cast<T>(res.recursive_residual_norm), true_norm, rhs_norm);
        if (!std::isfinite(true_norm) || !std::isfinite(rhs_norm)) {
            breakdown(kNonFinite);
        } else {
            res.status = kConverged;
            res.converged_by_application = 1;
        }
        return true;
    }
    T tiny() const { return T(1024) * std::numeric_limits<T>::min(); }
    T btol() const { return static_cast<T>(o.breakdown_tolerance); }
};

// core.hpp:536-547
template<class T> bool valid_options(const owtk_solver_options& o)
{
    const T rt = static_cast<T>(o.relative_tolerance), at = static_cast<T>(o.absolute_tolerance),
            bt = static_cast<T>(o.breakdown_tolerance);
    return std::isfinite(rt) && std::isfinite(at) && std::isfinite(bt) && rt >= T(0) && at >= T(0)
        && bt > T(0) && o.maximum_iterations > 0 && o.convergence_check_interval > 0;
}

// ------------------------------------------------------------------ BiCGSTAB
// krylov_solvers.hpp:546-745
template<class T>
void bicgstab(Engine<T>& e, Vector& b, Vector& x, Workspace& ws)
{
    auto& res = e.res;
    const auto& o = e.o;
    ws.prepare(b, 9);
    Vector& r = *ws.vectors[0];
    Vector& shadow = *ws.vectors[1];
    Vector& search = *ws.vectors[2];
    Vector& psearch = *ws.vectors[3];
    Vector& osearch = *ws.vectors[4];
    Vector& mid = *ws.vectors[5];
    Vector& pmid = *ws.vectors[6];
    Vector& omid = *ws.vectors[7];
    Vector& work = *ws.vectors[8];

    if (e.app_converged(b, x)) return;
    e.true_residual(b, x, r, work);
    e.copy(r, shadow);
    const T bnorm = e.norm(b);
    const T r0 = e.norm(r);
    const T thr = e.threshold(bnorm);
    const T tiny = e.tiny();
    res.initial_residual_norm = r0;
    e.set_residuals(r0, r0, bnorm);
    if (!std::isfinite(r0) || !std::isfinite(thr)) { e.breakdown(kNonFinite); return; }
    if (r0 <= thr) { res.status = kConverged; return; }

    T rho_prev = 1, alpha = 1, omega = 1;
    bool first = true;
    auto restart = [&]() {
        e.copy(r, shadow);
        e.fill(search, T(0));
        e.fill(osearch, T(0));
        rho_prev = 1; alpha = 1; omega = 1;
        first = true;
    };
    for (std::uint64_t it = 1; it <= o.maximum_iterations; ++it) {
        res.iterations = it;
        const T rho = e.dot(shadow, r);
        if (!std::isfinite(rho) || std::abs(rho) <= tiny) {
            e.breakdown(std::isfinite(rho) ? kBiorthogonality : kNonFinite);
            return;
        }
        if (first) {
            e.copy(r, search);
            first = false;
        } else {
            if (std::abs(omega) <= tiny) { e.breakdown(kOmegaZero); return; }
            const T beta = (rho / rho_prev) * (alpha / omega);
            kern::bicg_p<T>(e.c, e.n, e.p(r), beta, omega, e.p(osearch), e.p(search));
        }
        e.pc(search, psearch);
        e.op(psearch, osearch);
        const T sv = e.dot(shadow, osearch);
        if (!std::isfinite(sv) || std::abs(sv) <= tiny) {
            e.breakdown(std::isfinite(sv) ? kAlphaDen : kNonFinite);
            return;
        }
        alpha = rho / sv;
        kern::lincomb<T>(e.c, e.n, T(1), e.p(r), -alpha, e.p(osearch), e.p(mid));
        const T mnorm = e.norm(mid);
        if (mnorm <= thr) {
            e.axpy(alpha, psearch, x);
            if (e.app_converged(b, x)) return;
            e.true_residual(b, x, r, work);
            const T tn = e.norm(r);
            e.set_residuals(mnorm, tn, bnorm);
            if (tn <= thr) { res.status = kConverged; return; }
            restart();
            continue;
        }
        e.pc(mid, pmid);
        e.op(pmid, omid);
        Vector* da[2] = {&omid, &omid};
        Vector* db[2] = {&mid, &omid};
        res.global_reductions += 2;
        e.dots(2, da, db);
        const T num = e.scalar(kSlotA), den = e.scalar(kSlotA + 1);
        if (!std::isfinite(den) || std::abs(den) <= tiny) {
            e.breakdown(std::isfinite(den) ? kOmegaDen : kNonFinite);
            return;
        }
        omega = num / den;
        const T angle = std::abs(num) / std::sqrt(den) / mnorm;
        if (!std::isfinite(omega) || omega == T(0) || angle <= e.btol()) {
            e.breakdown(std::isfinite(omega) ? kOmegaZero : kNonFinite);
            return;
        }
        kern::bicg_xr<T>(e.c, e.n, alpha, e.p(psearch), omega, e.p(pmid), e.p(mid), e.p(omid), e.p(x), e.p(r));
        if (e.app_converged(b, x)) return;
        const bool replace = o.residual_replacement_interval > 0 && it % o.residual_replacement_interval == 0;
        const bool check = !e.has_test() && it % o.convergence_check_interval == 0;
        if (replace || check) {
            const T rn = e.norm(r);
            if (replace || rn <= thr) {
                e.true_residual(b, x, r, work);
                const T tn = e.norm(r);
                e.set_residuals(rn, tn, bnorm);
                if (tn <= thr) { res.status = kConverged; return; }
                restart();
                continue;
            }
            res.recursive_residual_norm = rn;
        }
        rho_prev = rho;
    }
    e.true_residual(b, x, r, work);
    const T tn = e.norm(r);
    e.set_residuals(static_cast<T>(res.recursive_residual_norm), tn, bnorm);
    res.status = tn <= thr ? kConverged : kMaxIterations;
    if (!std::isfinite(tn)) e.breakdown(kNonFinite);
}

// -------------------------------------------------------- pipelined BiCGSTAB
// pipelined_bicgstab.hpp:24-253
template<class T>
void pipelined_bicgstab(Engine<T>& e, Vector& b, Vector& x, Workspace& ws)
{
    auto& res = e.res;
    const auto& o = e.o;
    ws.prepare(b, 9);
    Vector& r = *ws.vectors[0];
    Vector& shadow = *ws.vectors[1];
    Vector& search = *ws.vectors[2];
    Vector& osearch = *ws.vectors[3];
    Vector& mid = *ws.vectors[4];
    Vector& omid = *ws.vectors[5];
    Vector& psearch = *ws.vectors[6];
    Vector& pmid = *ws.vectors[7];
    Vector& work = *ws.vectors[8];

    if (e.app_converged(b, x)) return;
    e.true_residual(b, x, r, work);
    e.copy(r, shadow);
    e.copy(r, search);
    {
        Vector* a[2] = {&b, &r};
        e.dots(2, a, a);
        ++res.global_reductions;
    }
    const T bsq = e.scalar(kSlotA), rsq = e.scalar(kSlotA + 1);
    const T bnorm = e.norm_from_squared(b, bsq);
    T rnorm = e.norm_from_squared(r, rsq);
    const T thr = e.threshold(bnorm);
    const T tiny = e.tiny();
    res.initial_residual_norm = rnorm;
    e.set_residuals(rnorm, rnorm, bnorm);
    if (!std::isfinite(rnorm) || !std::isfinite(thr)) { e.breakdown(kNonFinite); return; }
    if (rnorm <= thr) { res.status = kConverged; return; }

    T rho = e.dot(shadow, r);
    T alpha = 1, omega = 1;
    auto restart = [&]() {
        e.copy(r, shadow);
        e.copy(r, search);
        rho = e.dot(shadow, r);
        alpha = 1;
        omega = 1;
    };
    for (std::uint64_t it = 1; it <= o.maximum_iterations; ++it) {
        res.iterations = it;
        e.pc(search, psearch);
        e.op(psearch, osearch);
        const T so = e.dot(shadow, osearch);
        if (!std::isfinite(so) || std::abs(so) <= tiny) { e.breakdown(kAlphaDen); return; }
        alpha = rho / so;
        kern::lincomb<T>(e.c, e.n, T(1), e.p(r), -alpha, e.p(osearch), e.p(mid));
        e.pc(mid, pmid);
        e.op(pmid, omid);
        Vector* da[3] = {&omid, &omid, &mid};
        Vector* db[3] = {&mid, &omid, &mid};
        e.dots(3, da, db);
        ++res.global_reductions;
        const T g0 = e.scalar(kSlotA), g1 = e.scalar(kSlotA + 1), g2 = e.scalar(kSlotA + 2);
        const T mnorm = e.norm_from_squared(mid, g2);
        if (!std::isfinite(mnorm)) { e.breakdown(kNonFinite); return; }
        if (mnorm <= thr || !std::isfinite(g1) || std::abs(g1) <= tiny) {
            if (mnorm <= thr) {
                e.axpy(alpha, psearch, x);
                if (e.app_converged(b, x)) return;
                e.true_residual(b, x, r, work);
                const T tn = e.norm(r);
                e.set_residuals(mnorm, tn, bnorm);
                if (tn <= thr) { res.status = kConverged; return; }
                restart();
                continue;
            }
            e.breakdown(kOmegaDen);
            return;
        }
        omega = g0 / g1;
        const T angle = std::abs(g0) / std::sqrt(g1) / mnorm;
        if (!std::isfinite(omega) || omega == T(0) || angle <= e.btol()) { e.breakdown(kOmegaZero); return; }
        kern::bicg_xr<T>(e.c, e.n, alpha, e.p(psearch), omega, e.p(pmid), e.p(mid), e.p(omid), e.p(x), e.p(r));
        Vector* na[2] = {&shadow, &r};
        Vector* nb[2] = {&r, &r};
        e.dots(2, na, nb);
        ++res.global_reductions;
        const T prev = rho;
        rho = e.scalar(kSlotA);
        const T rsq2 = e.scalar(kSlotA + 1);
        rnorm = e.norm_from_squared(r, rsq2);
        res.recursive_residual_norm = rnorm;
        if (e.app_converged(b, x)) return;
        if (rnorm <= thr) {
            e.true_residual(b, x, r, work);
            const T tn = e.norm(r);
            e.set_residuals(rnorm, tn, bnorm);
            if (tn <= thr) { res.status = kConverged; return; }
            restart();
            continue;
        }
        if (!std::isfinite(prev) || std::abs(prev) <= tiny) { e.breakdown(kBiorthogonality); return; }
        const T beta = (rho / prev) * (alpha / omega);
        kern::bicg_p<T>(e.c, e.n, e.p(r), beta, omega, e.p(osearch), e.p(search));
        if (o.residual_replacement_interval > 0 && it % o.residual_replacement_interval == 0) {
            e.true_residual(b, x, r, work);
            restart();
        }
    }
    e.true_residual(b, x, r, work);
    const T tn = e.norm(r);
    e.set_residuals(rnorm, tn, bnorm);
    res.status = tn <= thr ? kConverged : kMaxIterations;
    if (!std::isfinite(tn)) e.breakdown(kNonFinite);
}

// ------------------------------------------- communication-hiding BiCGSTAB
// pipelined_bicgstab.hpp:321-598
template<class T>
void comm_hiding_bicgstab(Engine<T>& e, Vector& b, Vector& x, Workspace& ws)
{
    auto& res = e.res;
    const auto& o = e.o;
    ws.prepare(b, 16);
    Vector& r = *ws.vectors[0];
    Vector& rp = *ws.vectors[1];
    Vector& s = *ws.vectors[2];
    Vector& s2 = *ws.vectors[3];
    Vector& p2 = *ws.vectors[4];
    Vector& r2 = *ws.vectors[5];
    Vector& w = *ws.vectors[6];
    Vector& w2 = *ws.vectors[7];
    Vector& z = *ws.vectors[8];
    Vector& z2 = *ws.vectors[9];
    Vector& t = *ws.vectors[10];
    Vector& v = *ws.vectors[11];
    Vector& q = *ws.vectors[12];
    Vector& q2 = *ws.vectors[13];
    Vector& y = *ws.vectors[14];
    Vector& work = *ws.vectors[15];

    if (e.app_converged(b, x)) return;
    e.true_residual(b, x, r, work);
    e.copy(r, rp);
    {
        Vector* a[2] = {&b, &r};
        e.dots(2, a, a);
        ++res.global_reductions;
    }
    const T bsq = e.scalar(kSlotA), rsq = e.scalar(kSlotA + 1);
    const T bnorm = e.norm_from_squared(b, bsq);
    T rnorm = e.norm_from_squared(r, rsq);
    const T thr = e.threshold(bnorm);
    const T tiny = e.tiny();
    res.initial_residual_norm = rnorm;
    e.set_residuals(rnorm, rnorm, bnorm);
    if (!std::isfinite(rnorm) || !std::isfinite(thr)) { e.breakdown(kNonFinite); return; }
    if (rnorm <= thr) { res.status = kConverged; return; }

    T rho = 0, alpha = 0, beta = 0, omega = 0;
    auto init = [&]() -> bool {
        e.copy(r, rp);
        rho = e.dot(r, rp);
        if (!std::isfinite(rho) || std::abs(rho) <= tiny) return false;
        e.pc(r, r2);
        e.op(r2, w);
        const T d2 = e.dot(w, rp);
        if (!std::isfinite(d2) || std::abs(d2) <= tiny) return false;
        e.pc(w, w2);
        e.op(w2, t);
        alpha = rho / d2;
        beta = 0;
        omega = 0;
        return true;
    };
    if (!init()) { e.breakdown(kBiorthogonality); return; }
    bool first = true;
    for (std::uint64_t it = 1; it <= o.maximum_iterations; ++it) {
        res.iterations = it;
        if (first) {
            e.copy(r2, p2);
            e.copy(w, s);
            e.copy(w2, s2);
            e.copy(t, z);
            first = false;
        } else {
            kern::ch_pszupdate<T>(e.c, e.n, beta, omega, e.p(r2), e.p(w), e.p(w2), e.p(t), e.p(z2), e.p(v),
                                  e.p(p2), e.p(s), e.p(s2), e.p(z));
        }
        kern::ch_qy<T>(e.c, e.n, alpha, e.p(r), e.p(s), e.p(r2), e.p(s2), e.p(w), e.p(z), e.p(q), e.p(q2), e.p(y));
        // First batch (q.y, y.y, q.q), overlapped in the reference with PC+SpMV;
        // on one device the batch is simply issued before them.
        Vector* fa[3] = {&q, &y, &q};
        Vector* fb[3] = {&y, &y, &q};
        e.dots(3, fa, fb);
        ++res.global_reductions;
        const T f0 = e.scalar(kSlotA), f1 = e.scalar(kSlotA + 1), f2 = e.scalar(kSlotA + 2);
        e.pc(z, z2);
        e.op(z2, v);
        const T mnorm = e.norm_from_squared(q, f2);
        if (!std::isfinite(mnorm)) { e.breakdown(kNonFinite); return; }
        if (mnorm <= thr || !std::isfinite(f1) || std::abs(f1) <= tiny) {
            if (mnorm <= thr) {
                e.axpy(alpha, p2, x);
                if (e.app_converged(b, x)) return;
                e.true_residual(b, x, r, work);
                const T tn = e.norm(r);
                e.set_residuals(mnorm, tn, bnorm);
                if (tn <= thr) { res.status = kConverged; return; }
                if (!init()) { e.breakdown(kBiorthogonality); return; }
                first = true;
                continue;
            }
            e.breakdown(std::isfinite(f1) ? kOmegaDen : kNonFinite);
            return;
        }
        omega = f0 / f1;
        const T angle = std::abs(f0) / std::sqrt(f1) / mnorm;
        if (!std::isfinite(omega) || omega == T(0) || angle <= e.btol()) { e.breakdown(kOmegaZero); return; }
        e.axpy(alpha, p2, x);
        e.axpy(omega, q2, x);
        kern::ch_rw<T>(e.c, e.n, alpha, omega, e.p(q), e.p(y), e.p(q2), e.p(w2), e.p(z2), e.p(t), e.p(v),
                       e.p(r), e.p(r2), e.p(w));
        const T prev = rho;
        Vector* sa[5] = {&r, &r, &s, &w, &z};
        Vector* sb[5] = {&r, &rp, &rp, &rp, &rp};
        e.dots(5, sa, sb);
        ++res.global_reductions;
        const T g0 = e.scalar(kSlotA), g1 = e.scalar(kSlotA + 1), g2 = e.scalar(kSlotA + 2),
                g3 = e.scalar(kSlotA + 3), g4 = e.scalar(kSlotA + 4);
        e.pc(w, w2);
        e.op(w2, t);
        rnorm = e.norm_from_squared(r, g0);
        rho = g1;
        res.recursive_residual_norm = rnorm;
        if (e.app_converged(b, x)) return;
        if (rnorm <= thr) {
            e.true_residual(b, x, r, work);
            const T tn = e.norm(r);
            e.set_residuals(rnorm, tn, bnorm);
            if (tn <= thr) { res.status = kConverged; return; }
            if (!init()) { e.breakdown(kBiorthogonality); return; }
            first = true;
            continue;
        }
        if (o.residual_replacement_interval > 0 && it % o.residual_replacement_interval == 0) {
            e.true_residual(b, x, r, work);
            if (!init()) { e.breakdown(kBiorthogonality); return; }
            first = true;
            continue;
        }
        if (!std::isfinite(rho) || !std::isfinite(prev) || std::abs(rho) <= tiny || std::abs(prev) <= tiny) {
            e.breakdown(std::isfinite(rho) && std::isfinite(prev) ? kBiorthogonality : kNonFinite);
            return;
        }
        beta = (rho / prev) * (alpha / omega);
        const T den = g3 + beta * g2 - beta * omega * g4;
        if (!std::isfinite(den) || std::abs(den) <= tiny) {
            e.breakdown(std::isfinite(den) ? kAlphaDen : kNonFinite);
            return;
        }
        alpha = rho / den;
    }
    e.true_residual(b, x, r, work);
    const T tn = e.norm(r);
    e.set_residuals(rnorm, tn, bnorm);
    res.status = tn <= thr ? kConverged : kMaxIterations;
    if (!std::isfinite(tn)) e.breakdown(kNonFinite);
}

// --------------------------------------------------------------------- GMRES
// krylov_solvers.hpp:159-486
template<class T>
void fgmres(Engine<T>& e, Vector& b, Vector& x, Workspace& ws)
{
    auto& res = e.res;
    const auto& o = e.o;
    const std::size_t R = o.restart;
    if (R + 2 > static_cast<std::size_t>(kMaxBatch)) fail(OWTK_ERR_INVALID_ARGUMENT, "restart too large");
    // krylov_solvers.hpp:183-201: vectors and the scalar block it sizes.
    ws.prepare(b, 2 + (R + 1) + R, (R + 1) * R + R + R + (R + 1) + (R + 2) + (R + 2));
    Vector& r = *ws.vectors[0];
    Vector& w = *ws.vectors[1];
    std::vector<Vector*> V(R + 1), Z(R);
    for (std::size_t j = 0; j <= R; ++j) V[j] = ws.vectors[2 + j].get();
    for (std::size_t j = 0; j < R; ++j) Z[j] = ws.vectors[2 + R + 1 + j].get();
    std::vector<const T*> vptr(R + 1), zptr(R);
    for (std::size_t j = 0; j <= R; ++j) vptr[j] = e.p(*V[j]);
    for (std::size_t j = 0; j < R; ++j) zptr[j] = e.p(*Z[j]);
    ArnoldiSnapshot* snap = e.ex ? e.ex->snapshot : nullptr;

    if (e.app_converged(b, x)) {
        if (snap) snap->clear();
        return;
    }
    e.true_residual(b, x, r, w);
    const T bnorm = e.norm(b);
    const T r0 = e.norm(r);
    const T thr = e.threshold(bnorm);
    res.initial_residual_norm = r0;
    e.set_residuals(r0, r0, bnorm);
    if (!std::isfinite(r0) || !std::isfinite(thr)) { e.breakdown(kNonFinite); return; }
    if (r0 <= thr) {
        if (snap) snap->clear();
        res.status = kConverged;
        return;
    }

    // krylov_solvers.hpp:232: the candidate iterate of the convergence test.
    std::unique_ptr<Vector> candidate = e.has_test() ? make_vector_like(b) : nullptr;
    std::vector<T> H((R + 1) * R), cs(R), sn(R), g(R + 1), coef(R + 1);
    std::vector<double> column(R + 2);
    auto h = [&](std::size_t row, std::size_t col) -> T& { return H[col * (R + 1) + row]; };
    // The fused Gram-Schmidt kernels sum in the serial reduction's order; the
    // accurate reductions take the general path (pair dots, then updates).
    const bool fusable = e.mode() == 0;
    while (res.iterations < o.maximum_iterations) {
        if (snap) snap->begin_cycle(b, R);
        const T beta = e.norm(r);
        kern::divide<T>(e.c, e.n, e.p(r), beta, e.p(*V[0]));
        std::fill(H.begin(), H.end(), T(0));
        std::fill(g.begin(), g.end(), T(0));
        g[0] = beta;
        std::size_t cols = 0;
        bool arnoldi_breakdown = false;
        for (; cols < R && res.iterations < o.maximum_iterations; ++cols, ++res.iterations) {
            e.pc_op(*V[cols], *Z[cols], w);
            const std::size_t k = cols + 1;
            const T* vb[kMaxBatch];
            for (std::size_t j = 0; j < k; ++j) vb[j] = vptr[j];
            ++res.global_reductions;
            const bool iterated = o.gmres_orthogonalization == 0;
            // w.V_j (j < k) and w.w as one batch of pair dots into `slot`.
            const auto pair_dots = [&](int slot) {
                const T* pa[kMaxBatch];
                const T* pb[kMaxBatch];
                for (std::size_t j = 0; j < k; ++j) { pa[j] = e.p(w); pb[j] = vptr[j]; }
                pa[k] = e.p(w);
                pb[k] = e.p(w);
                if (e.mode() != 0)
                    kern::multidot_accurate<T>(e.c, e.n, static_cast<int>(k + 1), e.mode(), pa, pb, e.dslot(slot),
                                               e.hslot(slot), nullptr);
                else
                    kern::multidot<T>(e.c, e.n, static_cast<int>(k + 1), pa, pb, e.dslot(slot), e.hslot(slot));
            };
            if (fusable && k + 1 <= 32) {
                // First projection batch: w.V_j (j < k) and w.w, w read once.
                kern::basis_dots<T>(e.c, e.n, static_cast<int>(k), vb, e.p(w), e.dslot(kSlotA), e.hslot(kSlotA));
            } else {
                pair_dots(kSlotA);
            }
            if (iterated) {
                // w -= V h1, fused with the second batch (one pass over V while
                // the batch fits the fused kernel); then w -= V h2.
                if (fusable && k + 1 <= 32) {
                    kern::cgs_update_dot<T>(e.c, e.n, static_cast<int>(k), vb, e.dslot(kSlotA), e.p(w),
                                            e.dslot(kSlotB), e.hslot(kSlotB));
                } else {
                    kern::cgs_update<T>(e.c, e.n, static_cast<int>(k), vb, e.dslot(kSlotA), e.p(w));
                    pair_dots(kSlotB);
                }
                // The last pass, w -= V h2, waits for the norm: it is fused
                // with the normalisation into V[cols + 1] below.
            } else {
                kern::cgs_update<T>(e.c, e.n, static_cast<int>(k), vb, e.dslot(kSlotA), e.p(w));
            }
            bool last_pass_pending = iterated;
            const auto finish_last_pass = [&] {
                if (!last_pass_pending) return;
                kern::cgs_update<T>(e.c, e.n, static_cast<int>(k), vb, e.dslot(kSlotB), e.p(w));
                last_pass_pending = false;
            };
            e.c.sync();
            const T original = e.scalar(kSlotA + static_cast<int>(k));
            T projected = original;
            for (std::size_t row = 0; row < k; ++row) {
                h(row, cols) = e.scalar(kSlotA + static_cast<int>(row));
                projected -= h(row, cols) * h(row, cols);
            }
            const T nonneg = std::max(projected, T(0));
            const bool adaptive = o.gmres_orthogonalization == 1
                && (projected <= T(0) || nonneg < T(0.5) * original);
            T nsq = nonneg;
            if (iterated || adaptive) {
                if (adaptive) {
                    pair_dots(kSlotB);
                    kern::cgs_update<T>(e.c, e.n, static_cast<int>(k), vb, e.dslot(kSlotB), e.p(w));
                    e.c.sync();
                }
                ++res.global_reductions;
                ++res.reorthogonalizations;
                nsq = e.scalar(kSlotB + static_cast<int>(k));
                for (std::size_t row = 0; row < k; ++row) {
                    const T corr = e.scalar(kSlotB + static_cast<int>(row));
                    h(row, cols) += corr;
                    nsq -= corr * corr;
                }
            }
            if (original < std::numeric_limits<T>::min() || !std::isfinite(nsq)
                || nsq <= std::numeric_limits<T>::epsilon() * original
                || (nsq > T(0) && nsq < std::numeric_limits<T>::min())) {
                finish_last_pass();
                h(cols + 1, cols) = e.norm(w);
                ++res.arnoldi_norm_verifications;
            } else {
                h(cols + 1, cols) = std::sqrt(std::max(nsq, T(0)));
            }
            if (!std::isfinite(h(cols + 1, cols))) {
                finish_last_pass();
                e.breakdown(kNonFinite);
                return;
            }
            T cscale = 0;
            for (std::size_t row = 0; row <= cols + 1; ++row) cscale = std::max(cscale, std::abs(h(row, cols)));
            if (h(cols + 1, cols) > e.btol() * cscale) {
                if (last_pass_pending)
                    kern::cgs_update_scale<T>(e.c, e.n, static_cast<int>(k), vb, e.dslot(kSlotB), e.p(w),
                                              T(1) / h(cols + 1, cols), e.p(*V[cols + 1]));
                else
                    kern::scaled_copy<T>(e.c, e.n, e.p(w), T(1) / h(cols + 1, cols), e.p(*V[cols + 1]));
                last_pass_pending = false;
            } else {
                finish_last_pass();
                arnoldi_breakdown = true;
            }
            if (snap) {
                for (std::size_t row = 0; row <= cols + 1; ++row) column[row] = static_cast<double>(h(row, cols));
                snap->record_column(cols, column.data(), cols + 2);
            }
            for (std::size_t row = 0; row < cols; ++row) {
                const T first = cs[row] * h(row, cols) + sn[row] * h(row + 1, cols);
                h(row + 1, cols) = -sn[row] * h(row, cols) + cs[row] * h(row + 1, cols);
                h(row, cols) = first;
            }
            const T den = std::hypot(h(cols, cols), h(cols + 1, cols));
            if (!std::isfinite(den)) { e.breakdown(kNonFinite); return; }
            if (den == T(0)) {
                arnoldi_breakdown = true;
                cs[cols] = 1;
                sn[cols] = 0;
            } else {
                cs[cols] = h(cols, cols) / den;
                sn[cols] = h(cols + 1, cols) / den;
            }
            h(cols, cols) = cs[cols] * h(cols, cols) + sn[cols] * h(cols + 1, cols);
            h(cols + 1, cols) = 0;
            g[cols + 1] = -sn[cols] * g[cols];
            g[cols] *= cs[cols];
            const T est = std::abs(g[cols + 1]);
            res.recursive_residual_norm = est;
            if (candidate) {
                // krylov_solvers.hpp:399-425: x_k = x + Z c without ending the
                // cycle, c from the rotated system so far; offered to the test.
                bool nonsingular = true;
                for (std::size_t row = cols + 1; row-- > 0;) {
                    T value = g[row];
                    for (std::size_t j = row + 1; j <= cols; ++j) value -= h(row, j) * coef[j];
                    if (h(row, row) == T(0)) {
                        nonsingular = false;
                        break;
                    }
                    coef[row] = value / h(row, row);
                }
                if (nonsingular) {
                    for (std::size_t j = 0; j <= cols; ++j) e.c.host_scalars[kSlotCoef + j] = static_cast<double>(coef[j]);
                    OWTK_CUDA(cudaMemcpyAsync(e.dslot(kSlotCoef), e.c.host_scalars + kSlotCoef,
                                              (cols + 1) * sizeof(double), cudaMemcpyHostToDevice, e.c.stream));
                    kern::gmres_update<T>(e.c, e.n, static_cast<int>(cols + 1), zptr.data(), e.dslot(kSlotCoef),
                                          e.p(x), e.p(*candidate));
                    ++res.iterations;
                    if (e.app_converged(b, *candidate)) {
                        if (snap) snap->finish_cycle(Z, cols + 1);
                        e.copy(*candidate, x);
                        e.c.sync();
                        return;
                    }
                    --res.iterations;
                }
            }
            if (est <= thr || arnoldi_breakdown) {
                ++cols;
                ++res.iterations;
                break;
            }
        }
        if (snap) snap->finish_cycle(Z, cols);
        std::fill(coef.begin(), coef.end(), T(0));
        for (std::size_t rv = cols; rv-- > 0;) {
            T val = g[rv];
            for (std::size_t col = rv + 1; col < cols; ++col) val -= h(rv, col) * coef[col];
            T cscale = 0;
            for (std::size_t row = 0; row <= rv; ++row) cscale = std::max(cscale, std::abs(h(row, rv)));
            if (std::abs(h(rv, rv)) <= e.btol() * cscale) { e.breakdown(kSingular); return; }
            coef[rv] = val / h(rv, rv);
        }
        for (std::size_t j = 0; j < cols; ++j) e.c.host_scalars[kSlotCoef + j] = static_cast<double>(coef[j]);
        OWTK_CUDA(cudaMemcpyAsync(e.dslot(kSlotCoef), e.c.host_scalars + kSlotCoef, cols * sizeof(double),
                                  cudaMemcpyHostToDevice, e.c.stream));
        kern::gmres_update<T>(e.c, e.n, static_cast<int>(cols), zptr.data(), e.dslot(kSlotCoef), e.p(x), e.p(x));
        e.true_residual(b, x, r, w);
        const T tn = e.norm(r);
        e.set_residuals(static_cast<T>(res.recursive_residual_norm), tn, bnorm);
        if (!std::isfinite(tn)) { e.breakdown(kNonFinite); return; }
        if (tn <= thr) { res.status = kConverged; return; }
        if (arnoldi_breakdown && !(tn < beta)) { e.breakdown(kArnoldi); return; }
    }
    res.status = kMaxIterations;
}

// --------------------------------------------------------------------- IDR(s)
// idrs.hpp:33-76 — partial-pivoting dense solve of the small system.
template<class T>
bool solve_dense(std::vector<T> a, std::vector<T> rhs, std::vector<T>& sol, T tol)
{
    const std::size_t n = rhs.size();
    sol.assign(n, T(0));
    for (std::size_t col = 0; col < n; ++col) {
        std::size_t piv = col;
        for (std::size_t row = col + 1; row < n; ++row)
            if (std::abs(a[row * n + col]) > std::abs(a[piv * n + col])) piv = row;
        if (!std::isfinite(a[piv * n + col]) || std::abs(a[piv * n + col]) <= tol) return false;
        if (piv != col) {
            for (std::size_t k = col; k < n; ++k) std::swap(a[col * n + k], a[piv * n + k]);
            std::swap(rhs[col], rhs[piv]);
        }
        for (std::size_t row = col + 1; row < n; ++row) {
            const T f = a[row * n + col] / a[col * n + col];
            for (std::size_t k = col; k < n; ++k) a[row * n + k] -= f * a[col * n + k];
            rhs[row] -= f * rhs[col];
        }
    }
    for (std::size_t rv = n; rv-- > 0;) {
        T v = rhs[rv];
        for (std::size_t k = rv + 1; k < n; ++k) v -= a[rv * n + k] * sol[k];
        sol[rv] = v / a[rv * n + rv];
    }
    return true;
}

// idrs.hpp:128-506
template<class T>
void idrs(Engine<T>& e, Vector& b, Vector& x, Workspace& ws)
{
    auto& res = e.res;
    const auto& o = e.o;
    const std::size_t s = o.idr_shadow_space;
    ws.prepare(b, 4 + 3 * s);
    Vector& r = *ws.vectors[0];
    Vector& proj = *ws.vectors[1];
    Vector& prec = *ws.vectors[2];
    Vector& work = *ws.vectors[3];
    std::vector<Vector*> G(s), U(s), P(s);
    for (std::size_t k = 0; k < s; ++k) {
        G[k] = ws.vectors[4 + k].get();
        U[k] = ws.vectors[4 + s + k].get();
        P[k] = ws.vectors[4 + 2 * s + k].get();
    }
    if (e.app_converged(b, x)) return;
    e.true_residual(b, x, r, work);
    const T bnorm = e.norm(b);
    T rnorm = e.norm(r);
    const T thr = e.threshold(bnorm);
    res.initial_residual_norm = rnorm;
    e.set_residuals(rnorm, rnorm, bnorm);
    if (!std::isfinite(rnorm) || !std::isfinite(thr)) { e.breakdown(kNonFinite); return; }
    if (rnorm <= thr) { res.status = kConverged; return; }

    std::vector<T> Mm(s * s, T(0)), f(s, T(0)), am, ar, cf;
    std::size_t epoch = 0, restarts = 0;
    T omega = 1;
    std::vector<T> host_shadow(e.n);
    // idrs.hpp:78-119: deterministic shadow space from mt19937_64 and the
    // standard normal distribution of the host C++ library, orthonormalised.
    auto init_shadow = [&](std::uint64_t shift) -> bool {
        std::mt19937_64 gen(42ULL + 0ULL + shift * 0x9e3779b97f4a7c15ULL);
        std::normal_distribution<T> dist(T(0), T(1));
        const std::size_t first = s == 1 ? 1 : 0;
        if (s == 1) {
            e.copy(r, *P[0]);
            const T nv = e.norm(*P[0]);
            if (nv <= e.btol()) return false;
            e.scale(T(1) / nv, *P[0]);
        }
        for (std::size_t k = first; k < s; ++k) {
            for (std::size_t i = 0; i < e.n; ++i) host_shadow[i] = dist(gen);
            OWTK_CUDA(cudaMemcpyAsync(P[k]->data, host_shadow.data(), e.n * sizeof(T), cudaMemcpyHostToDevice, e.c.stream));
            for (std::size_t prev = 0; prev < k; ++prev) {
                const T pr = e.dot(*P[prev], *P[k]);
                e.axpy(-pr, *P[prev], *P[k]);
            }
            const T nv = e.norm(*P[k]);
            if (nv <= e.btol()) return false;
            e.scale(T(1) / nv, *P[k]);
        }
        e.c.sync();
        return true;
    };
    auto restart_basis = [&]() -> bool {
        if (!init_shadow(epoch++)) return false;
        std::fill(Mm.begin(), Mm.end(), T(0));
        for (std::size_t k = 0; k < s; ++k) {
            Mm[k * s + k] = 1;
            e.fill(*G[k], T(0));
            e.fill(*U[k], T(0));
            f[k] = e.dot(*P[k], r);
        }
        omega = 1;
        return true;
    };
    auto restart_or_fail = [&]() -> bool {
        ++restarts;
        return restarts <= 4 && restart_basis();
    };
    auto pivot_small = [&](std::size_t col) -> bool {
        T cscale = 0;
        for (std::size_t row = col; row < s; ++row) cscale = std::max(cscale, std::abs(Mm[row * s + col]));
        const T piv = Mm[col * s + col];
        const T tol = std::max(std::numeric_limits<T>::min(), e.btol() * cscale);
        return !std::isfinite(piv) || std::abs(piv) <= tol;
    };
    if (!restart_basis()) { e.breakdown(kIdrShadow); return; }

    bool restarted = false;
    while (res.iterations < o.maximum_iterations) {
        restarted = false;
        for (std::size_t k = 0; k < s && res.iterations < o.maximum_iterations; ++k) {
            const std::size_t act = s - k;
            am.assign(act * act, T(0));
            ar.assign(act, T(0));
            T mscale = 0;
            for (std::size_t row = 0; row < act; ++row) {
                ar[row] = f[k + row];
                for (std::size_t col = 0; col < act; ++col) {
                    const T v = Mm[(k + row) * s + (k + col)];
                    am[row * act + col] = v;
                    mscale = std::max(mscale, std::abs(v));
                }
            }
            const T dtol = std::max(std::numeric_limits<T>::min(), T(64) * std::numeric_limits<T>::epsilon() * mscale);
            if (!solve_dense<T>(am, ar, cf, dtol)) {
                if (!restart_or_fail()) { e.breakdown(kIdrSmall); return; }
                restarted = true;
                break;
            }
            e.copy(r, proj);
            for (std::size_t col = k; col < s; ++col) e.axpy(-cf[col - k], *G[col], proj);
            e.pc(proj, prec);
            e.scale(omega, prec);
            for (std::size_t col = k; col < s; ++col) e.axpy(cf[col - k], *U[col], prec);
            e.op(prec, work);
            for (std::size_t prev = 0; prev < k; ++prev) {
                const T piv = Mm[prev * s + prev];
                if (pivot_small(prev)) {
                    if (!restart_or_fail()) { e.breakdown(kIdrSmall); return; }
                    restarted = true;
                    break;
                }
                const T al = e.dot(*P[prev], work) / piv;
                e.axpy(-al, *G[prev], work);
                e.axpy(-al, *U[prev], prec);
            }
            if (restarted) break;
            for (std::size_t row = 0; row < k; ++row) Mm[row * s + k] = 0;
            for (std::size_t row = k; row < s; ++row) Mm[row * s + k] = e.dot(*P[row], work);
            const T piv = Mm[k * s + k];
            if (pivot_small(k)) {
                if (!restart_or_fail()) { e.breakdown(kIdrSmall); return; }
                restarted = true;
                break;
            }
            e.copy(work, *G[k]);
            e.copy(prec, *U[k]);
            const T be = f[k] / piv;
            e.axpy(be, *U[k], x);
            e.axpy(-be, *G[k], r);
            for (std::size_t row = k + 1; row < s; ++row) f[row] -= be * Mm[row * s + k];
            f[k] = 0;
            ++res.iterations;
            restarts = 0;
            if (e.app_converged(b, x)) return;
            rnorm = e.norm(r);
            res.recursive_residual_norm = rnorm;
            if (!std::isfinite(rnorm)) { e.breakdown(kNonFinite); return; }
            if (rnorm <= thr) {
                e.true_residual(b, x, r, work);
                const T tn = e.norm(r);
                e.set_residuals(rnorm, tn, bnorm);
                if (tn <= thr) { res.status = kConverged; return; }
                rnorm = tn;
                if (!restart_or_fail()) { res.status = kDiverged; return; }
                restarted = true;
                break;
            }
            if (o.residual_replacement_interval > 0 && res.iterations % o.residual_replacement_interval == 0) {
                e.true_residual(b, x, r, work);
                rnorm = e.norm(r);
                e.set_residuals(rnorm, rnorm, bnorm);
                if (rnorm <= thr) { res.status = kConverged; return; }
                if (!restart_basis()) { e.breakdown(kIdrShadow); return; }
                restarted = true;
                break;
            }
        }
        if (restarted) continue;
        if (res.iterations >= o.maximum_iterations) break;
        e.pc(r, prec);
        e.op(prec, work);
        Vector* da[2] = {&work, &work};
        Vector* db[2] = {&r, &work};
        res.global_reductions += 2;
        e.dots(2, da, db);
        const T num = e.scalar(kSlotA), den = e.scalar(kSlotA + 1);
        if (!std::isfinite(den) || den <= std::numeric_limits<T>::min()) { e.breakdown(kOmegaDen); return; }
        omega = num / den;
        const T adn = std::sqrt(std::max(T(0), den)) * std::max(rnorm, std::numeric_limits<T>::min());
        const T angle = adn > T(0) ? std::abs(num) / adn : T(1);
        constexpr T min_angle = T(0.7);
        if (angle > T(0) && angle < min_angle) omega *= min_angle / angle;
        if (!std::isfinite(omega) || std::abs(omega) <= std::numeric_limits<T>::min()) {
            e.breakdown(kOmegaDen);
            return;
        }
        e.axpy(omega, prec, x);
        e.axpy(-omega, work, r);
        ++res.iterations;
        restarts = 0;
        if (e.app_converged(b, x)) return;
        rnorm = e.norm(r);
        res.recursive_residual_norm = rnorm;
        if (!std::isfinite(rnorm)) { e.breakdown(kNonFinite); return; }
        if (rnorm <= thr) {
            e.true_residual(b, x, r, work);
            const T tn = e.norm(r);
            e.set_residuals(rnorm, tn, bnorm);
            if (tn <= thr) { res.status = kConverged; return; }
            rnorm = tn;
            if (!restart_or_fail()) { res.status = kDiverged; return; }
            continue;
        }
        if (o.residual_replacement_interval > 0 && res.iterations % o.residual_replacement_interval == 0) {
            e.true_residual(b, x, r, work);
            rnorm = e.norm(r);
            e.set_residuals(rnorm, rnorm, bnorm);
            if (rnorm <= thr) { res.status = kConverged; return; }
            if (!restart_basis()) { e.breakdown(kIdrShadow); return; }
            continue;
        }
        for (std::size_t row = 0; row < s; ++row) f[row] = e.dot(*P[row], r);
    }
    e.true_residual(b, x, r, work);
    const T tn = e.norm(r);
    e.set_residuals(rnorm, tn, bnorm);
    res.status = kMaxIterations;
}

template<class T>
void run(owtk_solver_kind kind, Matrix& m, Preconditioner* pc, Vector& b, Vector& x,
         const owtk_solver_options& o, Workspace& ws, owtk_solver_result& res, const SolveExtras* ex)
{
    Engine<T> e{*m.ctx, m, pc, b.owned_size(), res, o};
    e.ex = ex;
    switch (kind) {
    case OWTK_SOLVER_FGMRES:
        if (o.restart == 0) {
            if (ex && ex->snapshot) ex->snapshot->clear();
            return;
        }
        fgmres<T>(e, b, x, ws);
        break;
    case OWTK_SOLVER_BICGSTAB: bicgstab<T>(e, b, x, ws); break;
    case OWTK_SOLVER_PIPELINED_BICGSTAB: pipelined_bicgstab<T>(e, b, x, ws); break;
    case OWTK_SOLVER_COMM_HIDING_BICGSTAB: comm_hiding_bicgstab<T>(e, b, x, ws); break;
    case OWTK_SOLVER_IDRS: {
        const std::size_t s = o.idr_shadow_space;
        if (s == 0 || s > b.owned_size()) return;
        if (s == 1) {  // idrs.hpp:164-170: IDR(1) is BiCGSTAB
            bicgstab<T>(e, b, x, ws);
            break;
        }
        idrs<T>(e, b, x, ws);
        break;
    }
    default: fail(OWTK_ERR_INVALID_ARGUMENT, "unknown solver");
    }
}

}  // namespace

void solve(owtk_solver_kind kind, Matrix& m, Preconditioner* pc, Vector& b, Vector& x,
           const owtk_solver_options& o, Workspace& ws, owtk_solver_result& res, const SolveExtras* ex)
{
    if (ex && (ex->reduction < 0 || ex->reduction > 2)) fail(OWTK_ERR_INVALID_ARGUMENT, "unknown reduction kind");
    std::memset(&res, 0, sizeof(res));
    res.status = kInvalid;
    res.breakdown_reason = kNone;
    const double nan = std::numeric_limits<double>::quiet_NaN();
    res.initial_residual_norm = res.recursive_residual_norm = nan;
    res.true_residual_norm = res.relative_residual_norm = nan;
    const auto t0 = std::chrono::steady_clock::now();
    const bool bad = !b.same_layout(x) || b.dtype != x.dtype
        || (m.dtype == OWTK_F64 ? !valid_options<double>(o) : !valid_options<float>(o));
    if (!bad) {
        if (m.dtype == OWTK_F64) run<double>(kind, m, pc, b, x, o, ws, res, ex);
        else run<float>(kind, m, pc, b, x, o, ws, res, ex);
    } else if (kind == OWTK_SOLVER_FGMRES && ex && ex->snapshot) {
        ex->snapshot->clear();   // krylov_solvers.hpp:177-182
    }
    m.ctx->check_device_status();
    res.solve_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

}  // namespace owtk

using namespace owtk;

extern "C" {

void owtk_default_options(owtk_solver_options* o)
{
    if (!o) return;
    o->relative_tolerance = 1e-8;
    o->absolute_tolerance = 0;
    o->breakdown_tolerance = 64 * std::numeric_limits<double>::epsilon();
    o->maximum_iterations = 1000;
    o->convergence_check_interval = 10;
    o->restart = 30;
    o->residual_replacement_interval = 50;
    o->idr_shadow_space = 4;
    o->relaxation = 1;
    o->verify_true_residual = 1;
    o->gmres_orthogonalization = 0;
}

}  // extern "C"
