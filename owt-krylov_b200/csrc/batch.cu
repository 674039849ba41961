// Batched BiCGSTAB + Jacobi: many independent component-diagonal BSR systems
// of uneven sizes and block sizes solved together in ONE persistent
// cooperative launch, with per-system convergence masks, replayed from a CUDA
// graph.
//
// Every system runs the reference's preconditioned BiCGSTAB
// (krylov_solvers.hpp:546-745) with a Jacobi preconditioner
// (preconditioner.hpp:25-113): the same element-wise arithmetic (explicitly
// rounded, bit-identical SpMV and vector updates), the same breakdown guards,
// early exit, residual replacement, convergence checks, restarts and work
// counters.  Reductions use this kernel's own fixed summation order.
//
// Execution.  The grid is co-resident (cooperative launch) and walks a fixed
// cycle of phases separated by a bounded grid barrier:
//   SP0 EW0 | { EW1 SP1 EW2 EW3 SP2 EW4 SP3 EW5 }*
// EW phases are element-wise passes over a static partition of all systems'
// unknowns (block b owns a contiguous range, cut at system boundaries into
// segments); SP phases are SpMV passes over a static partition of vertices
// (warp w owns a contiguous vertex range balanced by entry count, cut at
// system boundaries), in passes of `vpw` vertices per warp (the tuned
// vertices-per-warp of the system's block size), lanes over (vertex,
// component) outputs, entries in row order.  A phase that ends in a
// reduction writes one partial per segment; the segment that arrives last for
// its system (ticket) combines that system's partials in segment order and
// advances the system's state machine.  Systems that are not in a phase's
// branch skip it; finished systems skip everything, and the launch ends when
// none is left.

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace batch {

using namespace dev;

constexpr int kBlock = 256;
constexpr int kWarps = kBlock / 32;
constexpr int kEwSlot = 8;          // doubles per element-wise partial: norm A (3), norm B (3), dot
constexpr int kSpSlot = 2;          // doubles per SpMV partial: two dots
constexpr int kVectors = 9;         // workspace slot order of the reference's bicgstab
constexpr int kMaxBlockSize = 32;
constexpr int kBarrierSpin = 1 << 24;

enum Vec { kR = 0, kShadow = 1, kSearch = 2, kPsearch = 3, kOsearch = 4, kMid = 5, kPmid = 6, kOmid = 7, kWork = 8 };
enum Mode : int { kRun = 0, kFinal = 1, kDone = 2 };
enum Flag : int { kFirst = 1, kRestart = 2, kEarly = 4, kTrue = 8 };
enum Phase : int { kSp0, kEw0, kEw1, kSp1, kEw2, kEw3, kSp2, kEw4, kSp3, kEw5, kSpBench };
enum Status { kConverged = 0, kMaxIterations = 1, kBreakdown = 2, kInvalid = 4 };
enum Reason { kNone = 0, kBiorthogonality = 3, kAlphaDen = 4, kOmegaDen = 5, kOmegaZero = 6, kNonFinite = 9 };

struct Sys {                 // immutable layout of one system
    long long u0;            // first unknown
    long long val0;          // first value
    int v0;                  // first vertex
    int e0;                  // first entry
    int owned, bs, vpw, pad;
    int ew_slot0, ew_nseg, sp_slot0, sp_nseg;
};

struct State {               // mutable solver state of one system
    double rho, rho_prev, alpha, omega, beta, bnorm, thr, mnorm, rn;
    double initial, recursive, true_norm, relative;
    long long it, op_apps, pc_apps, reductions;
    int mode, flags, status, reason;
};
static_assert(sizeof(State) % 8 == 0, "State is copied as 8-byte words");

struct Grid {                // grid barrier
    unsigned count, gen, abort, pad;
};

struct Options {
    double rtol, atol, btol;
    long long maxit, check, replace;
};

struct Args {
    int nsys;
    const Sys* sys;
    State* st;
    unsigned* tickets;       // per system: element-wise, SpMV arrival counters
    owtk_solver_result* results;
    const int* rowptr;       // all systems' rows, global entry numbers
    const int* xoff;         // per entry: first unknown of the column's block
    const double* vals;
    const double* inv;       // Jacobi inverse diagonal per unknown
    const double* b;
    double* x;
    double* vec;             // kVectors * U
    long long U;
    const int* ew_first;     // per block: first segment
    const int4* ew_seg;      // (system, u0, u1, slot)
    double* ew_part;
    const int* sp_first;     // per warp: first segment
    const int4* sp_seg;      // (system, v0, v1, slot)
    double* sp_part;
    Grid* grid;
    unsigned* remaining;
    unsigned* status;
    Options o;
    int bench_bs;            // SpMV bench only: block size to run (0 = all)
};

__device__ __forceinline__ int ld_cg(const int* p) { return __ldcg(p); }
__device__ __forceinline__ double ld_cg(const double* p) { return __ldcg(p); }

__device__ __forceinline__ double* vecp(const Args& a, int v) { return a.vec + static_cast<long long>(v) * a.U; }

// ---------------------------------------------------------------- barrier
__device__ bool grid_sync(const Args& a)
{
    __shared__ int ok_s;
    __syncthreads();
    if (threadIdx.x == 0) {
        int ok = 1;
        Grid* g = a.grid;
        const unsigned gen = ld_acquire(&g->gen);
        __threadfence();
        if (atomicAdd(&g->count, 1u) + 1 == gridDim.x) {
            atomicExch(&g->count, 0u);
            __threadfence();
            st_release(&g->gen, gen + 1);
        } else {
            int i = 0;
            for (; i < kBarrierSpin; ++i) {
                if (ld_acquire(&g->gen) != gen) break;
                if (ld_acquire(&g->abort)) break;
                __nanosleep(64);
            }
            if (i == kBarrierSpin) {
                atomicOr(a.status, kErrTimeout);
                st_release(&g->abort, 1u);
            }
        }
        if (ld_acquire(&g->abort)) ok = 0;
        __threadfence();
        ok_s = ok;
    }
    __syncthreads();
    return ok_s != 0;
}

// ---------------------------------------------------------------- state machine
// All of it runs in one thread per system: the last segment to arrive.

__device__ double norm_value(const ScaledSum& s)
{
    if (s.nan) return __longlong_as_double(0x7ff8000000000000LL);
    if (s.scale == 0.0 || isinf(s.scale)) return s.scale;
    return s.scale * sqrt(s.ssq);
}

__device__ void set_residuals(State& s, double recursive, double true_norm)
{
    s.recursive = recursive;
    s.true_norm = true_norm;
    s.relative = true_norm / (s.bnorm > 0.0 ? s.bnorm : 1.0);
}

__device__ void finish(const Args& a, int sys, State& s, int status, int reason)
{
    s.mode = kDone;
    s.status = status;
    s.reason = reason;
    owtk_solver_result r{};
    r.status = status;
    r.breakdown_reason = reason;
    r.iterations = static_cast<std::uint64_t>(s.it);
    r.operator_applications = static_cast<std::uint64_t>(s.op_apps);
    r.preconditioner_applications = static_cast<std::uint64_t>(s.pc_apps);
    r.global_reductions = static_cast<std::uint64_t>(s.reductions);
    r.initial_residual_norm = s.initial;
    r.recursive_residual_norm = s.recursive;
    r.true_residual_norm = s.true_norm;
    r.relative_residual_norm = s.relative;
    a.results[sys] = r;
    __threadfence();
    atomicSub(a.remaining, 1u);
}

__device__ double tiny() { return 1024.0 * 2.2250738585072014e-308; }

// Loop top of the reference's iteration it+1 with rho = dot(shadow, r).
__device__ void begin_iteration(const Args& a, int sys, State& s, double rho)
{
    const long long it = s.it + 1;
    if (it > a.o.maxit) {
        s.mode = kFinal;
        return;
    }
    s.it = it;
    s.reductions += 1;
    if (!isfinite(rho) || fabs(rho) <= tiny()) {
        finish(a, sys, s, kBreakdown, isfinite(rho) ? kBiorthogonality : kNonFinite);
        return;
    }
    s.rho = rho;
    if (!(s.flags & kFirst)) {
        if (fabs(s.omega) <= tiny()) {
            finish(a, sys, s, kBreakdown, kOmegaZero);
            return;
        }
        s.beta = (rho / s.rho_prev) * (s.alpha / s.omega);
    }
    s.mode = kRun;
}

__device__ void restart(const Args& a, int sys, State& s, double rho)
{
    s.flags = kFirst | kRestart;
    s.rho_prev = 1.0;
    s.alpha = 1.0;
    s.omega = 1.0;
    begin_iteration(a, sys, s, rho);
}

struct Reduced {
    ScaledSum n0, n1;
    double d0, d1;
};

__device__ Reduced combine_ew(const Args& a, const Sys& y)
{
    Reduced r{{0.0, 0.0, 0}, {0.0, 0.0, 0}, 0.0, 0.0};
    for (int k = 0; k < y.ew_nseg; ++k) {
        const double* p = a.ew_part + static_cast<long long>(y.ew_slot0 + k) * kEwSlot;
        r.n0 = norm_merge(r.n0, ScaledSum{ld_cg(p + 0), ld_cg(p + 1), ld_cg(p + 2) != 0.0});
        r.n1 = norm_merge(r.n1, ScaledSum{ld_cg(p + 3), ld_cg(p + 4), ld_cg(p + 5) != 0.0});
        r.d0 = add_rn(r.d0, ld_cg(p + 6));
    }
    return r;
}

__device__ Reduced combine_sp(const Args& a, const Sys& y)
{
    Reduced r{{0.0, 0.0, 0}, {0.0, 0.0, 0}, 0.0, 0.0};
    for (int k = 0; k < y.sp_nseg; ++k) {
        const double* p = a.sp_part + static_cast<long long>(y.sp_slot0 + k) * kSpSlot;
        r.d0 = add_rn(r.d0, ld_cg(p + 0));
        r.d1 = add_rn(r.d1, ld_cg(p + 1));
    }
    return r;
}

// State written by other SMs: read through L2, never a stale L1 line.
__device__ State load_state(const State* p)
{
    State s;
    const long long* src = reinterpret_cast<const long long*>(p);
    long long* dst = reinterpret_cast<long long*>(&s);
#pragma unroll
    for (int i = 0; i < static_cast<int>(sizeof(State) / 8); ++i) dst[i] = __ldcg(src + i);
    return s;
}

__device__ void finalize(const Args& a, int phase, int sys)
{
    const Sys y = a.sys[sys];
    State s = load_state(a.st + sys);
    const auto& o = a.o;
    switch (phase) {
    case kEw0: {   // r = b - A x, shadow = r; norms of b and r, r.r
        const Reduced r = combine_ew(a, y);
        s.op_apps += 1;
        s.reductions += 2;
        s.bnorm = norm_value(r.n0);
        const double r0 = norm_value(r.n1);
        const double rel = o.rtol * (s.bnorm > 0.0 ? s.bnorm : 1.0);
        s.thr = (!isfinite(s.bnorm) || !isfinite(rel)) ? __longlong_as_double(0x7ff8000000000000LL)
                                                       : fmax(o.atol, rel);
        s.initial = r0;
        set_residuals(s, r0, r0);
        if (!isfinite(r0) || !isfinite(s.thr)) {
            finish(a, sys, s, kBreakdown, kNonFinite);
            break;
        }
        if (r0 <= s.thr) {
            finish(a, sys, s, kConverged, kNone);
            break;
        }
        s.rho_prev = s.alpha = s.omega = 1.0;
        s.flags = kFirst;
        begin_iteration(a, sys, s, r.d0);
        break;
    }
    case kSp1: {   // sv = shadow . A psearch
        const Reduced r = combine_sp(a, y);
        s.pc_apps += 1;
        s.op_apps += 1;
        s.reductions += 1;
        s.flags &= ~(kFirst | kRestart);
        const double sv = r.d0;
        if (!isfinite(sv) || fabs(sv) <= tiny()) {
            finish(a, sys, s, kBreakdown, isfinite(sv) ? kAlphaDen : kNonFinite);
            break;
        }
        s.alpha = s.rho / sv;
        break;
    }
    case kEw2: {   // ||mid||
        const Reduced r = combine_ew(a, y);
        s.reductions += 1;
        s.mnorm = norm_value(r.n0);
        if (s.mnorm <= s.thr) s.flags |= kEarly;
        break;
    }
    case kSp2: {   // omid.mid, omid.omid
        const Reduced r = combine_sp(a, y);
        s.pc_apps += 1;
        s.op_apps += 1;
        s.reductions += 2;
        const double num = r.d0, den = r.d1;
        if (!isfinite(den) || fabs(den) <= tiny()) {
            finish(a, sys, s, kBreakdown, isfinite(den) ? kOmegaDen : kNonFinite);
            break;
        }
        s.omega = num / den;
        const double angle = fabs(num) / sqrt(den) / s.mnorm;
        if (!isfinite(s.omega) || s.omega == 0.0 || angle <= o.btol) {
            finish(a, sys, s, kBreakdown, isfinite(s.omega) ? kOmegaZero : kNonFinite);
            break;
        }
        break;
    }
    case kEw4: {
        const Reduced r = combine_ew(a, y);
        if (s.flags & kEarly) {       // early exit: true residual of x + alpha psearch
            s.op_apps += 1;
            s.reductions += 1;
            const double tn = norm_value(r.n0);
            set_residuals(s, s.mnorm, tn);
            if (tn <= s.thr) {
                finish(a, sys, s, kConverged, kNone);
                break;
            }
            restart(a, sys, s, r.d0);
            break;
        }
        const bool replace = o.replace > 0 && s.it % o.replace == 0;
        const bool check = s.it % o.check == 0;
        if (replace || check) {
            s.reductions += 1;
            const double rn = norm_value(r.n0);
            if (replace || rn <= s.thr) {
                s.rn = rn;
                s.flags |= kTrue;
                break;
            }
            s.recursive = rn;
        }
        s.rho_prev = s.rho;
        begin_iteration(a, sys, s, r.d0);
        break;
    }
    case kEw5: {   // true residual: replacement / check, or after the last iteration
        const Reduced r = combine_ew(a, y);
        s.op_apps += 1;
        s.reductions += 1;
        const double tn = norm_value(r.n0);
        if (s.mode == kFinal) {
            set_residuals(s, s.recursive, tn);
            if (!isfinite(tn)) finish(a, sys, s, kBreakdown, kNonFinite);
            else finish(a, sys, s, tn <= s.thr ? kConverged : kMaxIterations, kNone);
            break;
        }
        set_residuals(s, s.rn, tn);
        s.flags &= ~kTrue;
        if (tn <= s.thr) {
            finish(a, sys, s, kConverged, kNone);
            break;
        }
        restart(a, sys, s, r.d0);
        break;
    }
    default:
        break;
    }
    a.st[sys] = s;
}

// ---------------------------------------------------------------- SpMV phases
// Which systems take part, and what the pass computes.
__device__ __forceinline__ bool sp_role(const Args& a, int phase, int mode, int flags, int bs, int& in, int& out,
                                        int& dots)
{
    dots = 0;
    switch (phase) {
    case kSp0: in = -1; out = kWork; return mode == kRun;
    case kSp1: in = kPsearch; out = kOsearch; dots = 1; return mode == kRun;
    case kSp2:
        if (mode != kRun) return false;
        if (flags & kEarly) { in = -1; out = kWork; return true; }
        in = kPmid; out = kOmid; dots = 2; return true;
    case kSp3: in = -1; out = kWork; return (mode == kRun && (flags & kTrue)) || mode == kFinal;
    case kSpBench: in = kPsearch; out = kOsearch; return a.bench_bs == 0 || a.bench_bs == bs;
    default: return false;
    }
}

__device__ void sp_phase(const Args& a, int phase)
{
    const int wg = blockIdx.x * kWarps + (threadIdx.x >> 5), lane = threadIdx.x & 31;
    const int s_end = a.sp_first[wg + 1];
    for (int sg = a.sp_first[wg]; sg < s_end; ++sg) {
        const int4 seg = a.sp_seg[sg];
        const int sys = seg.x;
        const State* stp = a.st + sys;
        const int mode = ld_cg(&stp->mode), flags = ld_cg(&stp->flags);
        const Sys y = a.sys[sys];
        int vin, vout, dots;
        if (!sp_role(a, phase, mode, flags, y.bs, vin, vout, dots)) continue;
        const double* in = vin < 0 ? a.x : vecp(a, vin);
        double* out = vecp(a, vout);
        const double* da = dots ? vecp(a, phase == kSp1 ? kShadow : kMid) : nullptr;
        const int bs = y.bs, vpw = y.vpw;
        double d0 = 0.0, d1 = 0.0;
        for (int v = seg.y; v < seg.z; v += vpw) {
            const int outs = min(vpw, seg.z - v) * bs;
            for (int o = lane; o < outs; o += 32) {
                const int vl = o / bs, c = o - vl * bs;
                const int vg = v + vl;
                const int eb = __ldg(a.rowptr + vg), ee = __ldg(a.rowptr + vg + 1);
                const double* vv = a.vals + y.val0 + static_cast<long long>(eb - y.e0) * bs + c;
                double acc = 0.0;
                int e = eb;
                for (; e + 4 <= ee; e += 4) {
                    const int x0 = __ldg(a.xoff + e), x1 = __ldg(a.xoff + e + 1), x2 = __ldg(a.xoff + e + 2),
                              x3 = __ldg(a.xoff + e + 3);
                    const double p0 = mul_rn(__ldg(vv + (e - eb) * bs), ld_cg(in + x0 + c));
                    const double p1 = mul_rn(__ldg(vv + (e + 1 - eb) * bs), ld_cg(in + x1 + c));
                    const double p2 = mul_rn(__ldg(vv + (e + 2 - eb) * bs), ld_cg(in + x2 + c));
                    const double p3 = mul_rn(__ldg(vv + (e + 3 - eb) * bs), ld_cg(in + x3 + c));
                    acc = add_rn(add_rn(add_rn(add_rn(acc, p0), p1), p2), p3);
                }
                for (; e < ee; ++e) acc = add_rn(acc, mul_rn(__ldg(vv + (e - eb) * bs), ld_cg(in + __ldg(a.xoff + e) + c)));
                const long long u = y.u0 + static_cast<long long>(vg - y.v0) * bs + c;
                out[u] = acc;
                if (dots == 1) d0 = add_rn(d0, mul_rn(ld_cg(da + u), acc));
                if (dots == 2) {
                    d0 = add_rn(d0, mul_rn(acc, ld_cg(da + u)));
                    d1 = add_rn(d1, mul_rn(acc, acc));
                }
            }
        }
        if (dots) {
            d0 = warp_sum(d0);
            d1 = warp_sum(d1);
            if (lane == 0) {
                double* p = a.sp_part + static_cast<long long>(seg.w) * kSpSlot;
                p[0] = d0;
                p[1] = d1;
                __threadfence();
                const unsigned old = atomicAdd(a.tickets + 2 * sys + 1, 1u);
                if ((old + 1) % static_cast<unsigned>(y.sp_nseg) == 0) {
                    __threadfence();
                    finalize(a, phase, sys);
                }
            }
            __syncwarp();
        }
    }
}

// ---------------------------------------------------------------- element-wise phases
// What a system does in an element-wise phase: 0 = nothing.
__device__ __forceinline__ int ew_role(int phase, int mode, int flags)
{
    switch (phase) {
    case kEw0: return mode == kRun ? 1 : 0;
    case kEw1: return mode == kRun ? 1 : 0;
    case kEw2: return mode == kRun ? 1 : 0;
    case kEw3: return mode == kRun ? ((flags & kEarly) ? 2 : 1) : 0;
    case kEw4: return mode == kRun ? ((flags & kEarly) ? 2 : 1) : 0;
    case kEw5: return ((mode == kRun && (flags & kTrue)) || mode == kFinal) ? 1 : 0;
    default: return 0;
    }
}

__device__ void ew_phase(const Args& a, int phase)
{
    __shared__ double red[kWarps][kEwSlot];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double* r = vecp(a, kR);
    double* shadow = vecp(a, kShadow);
    double* search = vecp(a, kSearch);
    double* psearch = vecp(a, kPsearch);
    double* osearch = vecp(a, kOsearch);
    double* mid = vecp(a, kMid);
    double* pmid = vecp(a, kPmid);
    double* omid = vecp(a, kOmid);
    double* work = vecp(a, kWork);
    const int s_end = a.ew_first[blockIdx.x + 1];
    for (int sg = a.ew_first[blockIdx.x]; sg < s_end; ++sg) {
        const int4 seg = a.ew_seg[sg];
        const int sys = seg.x;
        const State* stp = a.st + sys;
        const int mode = ld_cg(&stp->mode), flags = ld_cg(&stp->flags);
        const int role = ew_role(phase, mode, flags);
        if (role == 0) continue;
        const double alpha = ld_cg(&stp->alpha), omega = ld_cg(&stp->omega), beta = ld_cg(&stp->beta);
        ScaledSum n0{0.0, 0.0, 0}, n1{0.0, 0.0, 0};
        double d0 = 0.0;
        bool reduce = true;
        for (long long u = seg.y + threadIdx.x; u < seg.z; u += kBlock) {
            switch (phase) {
            case kEw0: {
                const double bv = __ldg(a.b + u), rv = sub_rn(bv, ld_cg(work + u));
                r[u] = rv;
                shadow[u] = rv;
                norm_push(n0, bv);
                norm_push(n1, rv);
                d0 = add_rn(d0, mul_rn(rv, rv));
                break;
            }
            case kEw1: {
                const double rv = ld_cg(r + u);
                double sv;
                if (flags & kRestart) {
                    shadow[u] = rv;
                    osearch[u] = 0.0;
                }
                if (flags & kFirst) {
                    sv = rv;
                } else {
                    sv = add_rn(rv, mul_rn(beta, sub_rn(ld_cg(search + u), mul_rn(omega, ld_cg(osearch + u)))));
                }
                search[u] = sv;
                psearch[u] = mul_rn(__ldg(a.inv + u), sv);
                break;
            }
            case kEw2: {
                const double m = add_rn(mul_rn(1.0, ld_cg(r + u)), mul_rn(-alpha, ld_cg(osearch + u)));
                mid[u] = m;
                norm_push(n0, m);
                break;
            }
            case kEw3:
                if (role == 2) a.x[u] = add_rn(ld_cg(a.x + u), mul_rn(alpha, ld_cg(psearch + u)));
                else pmid[u] = mul_rn(__ldg(a.inv + u), ld_cg(mid + u));
                break;
            case kEw4:
                if (role == 2) {
                    const double rv = sub_rn(__ldg(a.b + u), ld_cg(work + u));
                    r[u] = rv;
                    norm_push(n0, rv);
                    d0 = add_rn(d0, mul_rn(rv, rv));
                } else {
                    const double xv = add_rn(add_rn(ld_cg(a.x + u), mul_rn(alpha, ld_cg(psearch + u))),
                                             mul_rn(omega, ld_cg(pmid + u)));
                    const double rv = sub_rn(ld_cg(mid + u), mul_rn(omega, ld_cg(omid + u)));
                    a.x[u] = xv;
                    r[u] = rv;
                    norm_push(n0, rv);
                    d0 = add_rn(d0, mul_rn(ld_cg(shadow + u), rv));
                }
                break;
            case kEw5: {
                const double rv = sub_rn(__ldg(a.b + u), ld_cg(work + u));
                r[u] = rv;
                norm_push(n0, rv);
                d0 = add_rn(d0, mul_rn(rv, rv));
                break;
            }
            default:
                break;
            }
        }
        if (phase == kEw1 || phase == kEw3) reduce = false;
        if (!reduce) continue;
        // Block reduction in a fixed order, then the system's ticket.
        n0 = norm_warp(n0);
        n1 = norm_warp(n1);
        d0 = warp_sum(d0);
        if (lane == 0) {
            red[warp][0] = n0.scale;
            red[warp][1] = n0.ssq;
            red[warp][2] = n0.nan;
            red[warp][3] = n1.scale;
            red[warp][4] = n1.ssq;
            red[warp][5] = n1.nan;
            red[warp][6] = d0;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            ScaledSum m0{red[0][0], red[0][1], red[0][2] != 0.0}, m1{red[0][3], red[0][4], red[0][5] != 0.0};
            double dd = red[0][6];
            for (int w = 1; w < kWarps; ++w) {
                m0 = norm_merge(m0, ScaledSum{red[w][0], red[w][1], red[w][2] != 0.0});
                m1 = norm_merge(m1, ScaledSum{red[w][3], red[w][4], red[w][5] != 0.0});
                dd = add_rn(dd, red[w][6]);
            }
            double* p = a.ew_part + static_cast<long long>(seg.w) * kEwSlot;
            p[0] = m0.scale;
            p[1] = m0.ssq;
            p[2] = m0.nan;
            p[3] = m1.scale;
            p[4] = m1.ssq;
            p[5] = m1.nan;
            p[6] = dd;
            __threadfence();
            const Sys y = a.sys[sys];
            const unsigned old = atomicAdd(a.tickets + 2 * sys, 1u);
            if ((old + 1) % static_cast<unsigned>(y.ew_nseg) == 0) {
                __threadfence();
                finalize(a, phase, sys);
            }
        }
        __syncthreads();
    }
}

// MINB: resident CTAs per SM the register budget is cut for (2, 3, 4, 5, 6:
// 128, 80, 64, 48, 40 registers, the leaner ones with some state spilled).
// The launch is latency-bound, so more resident warps can outweigh the
// spills; the autotuner times every count.
template<int MINB>
__global__ void __launch_bounds__(kBlock, MINB) k_batch_bicgstab(Args a)
{
    sp_phase(a, kSp0);
    if (!grid_sync(a)) return;
    ew_phase(a, kEw0);
    if (!grid_sync(a)) return;
    const long long cap = a.o.maxit + 8;
    for (long long cycle = 0;; ++cycle) {
        if (ld_acquire(a.remaining) == 0) break;
        if (cycle > cap) {
            if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(a.status, kErrTimeout);
            break;
        }
        ew_phase(a, kEw1);
        if (!grid_sync(a)) return;
        sp_phase(a, kSp1);
        if (!grid_sync(a)) return;
        ew_phase(a, kEw2);
        if (!grid_sync(a)) return;
        ew_phase(a, kEw3);
        if (!grid_sync(a)) return;
        sp_phase(a, kSp2);
        if (!grid_sync(a)) return;
        ew_phase(a, kEw4);
        if (!grid_sync(a)) return;
        sp_phase(a, kSp3);
        if (!grid_sync(a)) return;
        ew_phase(a, kEw5);
        if (!grid_sync(a)) return;
    }
}

// One SpMV pass (psearch -> osearch) over the systems of one block size; the
// autotuner times it per vertices-per-warp candidate.
__global__ void __launch_bounds__(kBlock) k_batch_spmv_bench(Args a) { sp_phase(a, kSpBench); }

__global__ void k_batch_init(int nsys, State* st, unsigned* tickets, owtk_solver_result* results, Grid* grid,
                             unsigned* remaining)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < nsys) {
        State s{};
        s.mode = kRun;
        st[i] = s;
        tickets[2 * i] = 0u;
        tickets[2 * i + 1] = 0u;
        results[i] = owtk_solver_result{};
    }
    if (i == 0) {
        *grid = Grid{0u, 0u, 0u, 0u};
        *remaining = static_cast<unsigned>(nsys);
    }
}

// Jacobi inverse diagonal per unknown (preconditioner.hpp:62-69): first
// diagonal entry of each row, 1/d, singular when not finite or |d| <= 64 eps.
__global__ void k_batch_jacobi(int nsys, const Sys* sys, const int* sys_of_vertex, int nv, const int* rowptr,
                               const int* xoff, const double* vals, double* inv, unsigned* status)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= nv) return;
    const Sys y = sys[sys_of_vertex[v]];
    const long long u = y.u0 + static_cast<long long>(v - y.v0) * y.bs;
    for (int e = rowptr[v]; e < rowptr[v + 1]; ++e) {
        if (xoff[e] == u) {
            const double* d = vals + y.val0 + static_cast<long long>(e - y.e0) * y.bs;
            for (int c = 0; c < y.bs; ++c) {
                const double dv = d[c];
                if (!isfinite(dv) || fabs(dv) <= 64.0 * 2.220446049250313e-16) atomicOr(status, kErrSingularDiagonal);
                inv[u + c] = div_rn(1.0, dv);
            }
            return;
        }
    }
    atomicOr(status, kErrMissingDiagonal);
}

}  // namespace batch
}  // namespace owtk

// ====================================================================== host
namespace owtk {

struct Batch {
    Context* ctx = nullptr;
    int nsys = 0;
    long long V = 0, E = 0, U = 0, NV = 0;
    std::vector<batch::Sys> h_sys;
    std::vector<std::int32_t> h_rowptr;      // global
    std::vector<int> sys_of_vertex;
    DeviceBuffer rowptr, xoff, vals, inv, vec, sys, st, tickets, results, ew_first, ew_seg, ew_part, sp_first, sp_seg,
        sp_part, grid, remaining, scratch_b, scratch_x, stage_b, stage_x;
    int blocks_per_sm = 0, max_blocks_per_sm = 0, grid_blocks = 0;
    int vpw[batch::kMaxBlockSize + 1] = {};
    std::uint64_t config_version = 1;
    owtk_solver_result* h_results = nullptr;  // pinned
    bool use_graph = true;
    // Captured graph and its key.
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    const void* key_b = nullptr;
    void* key_x = nullptr;
    batch::Options key_o{};
    std::uint64_t key_version = 0;
    std::uint64_t graph_launches = 0, graph_captures = 0;

    ~Batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        if (h_results) cudaFreeHost(h_results);
    }
};

namespace {

using batch::kBlock;
using batch::kWarps;

int default_vpw(int bs) { return std::max(1, 32 / bs); }

// Static partitions for the current grid size.
void build_partition(Batch& B)
{
    const int G = B.grid_blocks, W = G * kWarps;
    // Element-wise: block b owns unknowns [b*U/G, (b+1)*U/G).
    std::vector<std::int32_t> ew_first(G + 1, 0);
    std::vector<std::int32_t> ew_seg;
    std::vector<int> ew_count(B.nsys, 0), ew_slot0(B.nsys, -1);
    int nseg = 0;
    int s = 0;
    for (int b = 0; b < G; ++b) {
        ew_first[b] = nseg;
        const long long lo = B.U * b / G, hi = B.U * (b + 1) / G;
        long long u = lo;
        while (u < hi) {
            while (B.h_sys[s].u0 + static_cast<long long>(B.h_sys[s].owned) * B.h_sys[s].bs <= u) ++s;
            const long long send = B.h_sys[s].u0 + static_cast<long long>(B.h_sys[s].owned) * B.h_sys[s].bs;
            const long long e = std::min(hi, send);
            if (ew_slot0[s] < 0) ew_slot0[s] = nseg;
            ew_seg.insert(ew_seg.end(), {s, static_cast<std::int32_t>(u), static_cast<std::int32_t>(e), nseg});
            ++ew_count[s];
            ++nseg;
            u = e;
        }
    }
    ew_first[G] = nseg;
    // SpMV: warp w owns a vertex range balanced by (entries + 1) * bs.
    std::vector<double> prefix(B.V + 1, 0.0);
    {
        int sv = 0;
        for (long long v = 0; v < B.V; ++v) {
            while (B.h_sys[sv].v0 + B.h_sys[sv].owned <= v) ++sv;
            prefix[v + 1] = prefix[v] + static_cast<double>(B.h_rowptr[v + 1] - B.h_rowptr[v] + 1) * B.h_sys[sv].bs;
        }
    }
    std::vector<std::int32_t> sp_first(W + 1, 0);
    std::vector<std::int32_t> sp_seg;
    std::vector<int> sp_count(B.nsys, 0), sp_slot0(B.nsys, -1);
    int nsp = 0;
    s = 0;
    long long v = 0;
    for (int w = 0; w < W; ++w) {
        sp_first[w] = nsp;
        const double target = prefix[B.V] * (w + 1) / W;
        long long hi = w + 1 == W ? B.V : std::lower_bound(prefix.begin() + v, prefix.end(), target) - prefix.begin();
        hi = std::min<long long>(std::max(hi, v), B.V);
        while (v < hi) {
            while (B.h_sys[s].v0 + B.h_sys[s].owned <= v) ++s;
            const long long e = std::min<long long>(hi, B.h_sys[s].v0 + B.h_sys[s].owned);
            if (sp_slot0[s] < 0) sp_slot0[s] = nsp;
            sp_seg.insert(sp_seg.end(), {s, static_cast<std::int32_t>(v), static_cast<std::int32_t>(e), nsp});
            ++sp_count[s];
            ++nsp;
            v = e;
        }
    }
    sp_first[W] = nsp;
    for (int i = 0; i < B.nsys; ++i) {
        B.h_sys[i].ew_slot0 = ew_slot0[i];
        B.h_sys[i].ew_nseg = ew_count[i];
        B.h_sys[i].sp_slot0 = sp_slot0[i];
        B.h_sys[i].sp_nseg = sp_count[i];
        B.h_sys[i].vpw = B.vpw[B.h_sys[i].bs];
    }
    cudaStream_t st = B.ctx->stream;
    B.ew_first = upload(st, ew_first);
    B.ew_seg = upload(st, ew_seg);
    B.sp_first = upload(st, sp_first);
    B.sp_seg = upload(st, sp_seg);
    B.ew_part.allocate(static_cast<std::size_t>(std::max(nseg, 1)) * batch::kEwSlot * sizeof(double));
    B.sp_part.allocate(static_cast<std::size_t>(std::max(nsp, 1)) * batch::kSpSlot * sizeof(double));
    B.sys = upload(st, B.h_sys);
    B.ctx->sync();
}

void refresh_sys(Batch& B)
{
    for (auto& y : B.h_sys) y.vpw = B.vpw[y.bs];
    B.sys = upload(B.ctx->stream, B.h_sys);
    B.ctx->sync();
    ++B.config_version;
}

void set_grid(Batch& B, int blocks_per_sm)
{
    B.blocks_per_sm = std::max(1, std::min(blocks_per_sm, B.max_blocks_per_sm));
    B.grid_blocks = B.ctx->sm_count * B.blocks_per_sm;
    build_partition(B);
    ++B.config_version;
}

batch::Args make_args(Batch& B, const double* b, double* x, const batch::Options& o)
{
    batch::Args a{};
    a.nsys = B.nsys;
    a.sys = B.sys.as<batch::Sys>();
    a.st = B.st.as<batch::State>();
    a.tickets = B.tickets.as<unsigned>();
    a.results = B.results.as<owtk_solver_result>();
    a.rowptr = B.rowptr.as<int>();
    a.xoff = B.xoff.as<int>();
    a.vals = B.vals.as<double>();
    a.inv = B.inv.as<double>();
    a.b = b;
    a.x = x;
    a.vec = B.vec.as<double>();
    a.U = B.U;
    a.ew_first = B.ew_first.as<int>();
    a.ew_seg = B.ew_seg.as<int4>();
    a.ew_part = B.ew_part.as<double>();
    a.sp_first = B.sp_first.as<int>();
    a.sp_seg = B.sp_seg.as<int4>();
    a.sp_part = B.sp_part.as<double>();
    a.grid = B.grid.as<batch::Grid>();
    a.remaining = B.remaining.as<unsigned>();
    a.status = B.ctx->status.as<unsigned>();
    a.o = o;
    return a;
}

// The solver instance whose register budget allows k resident CTAs per SM
// (k = 1 takes the two-CTA budget).
using SolveKernel = void (*)(batch::Args);
SolveKernel solve_kernel(int k)
{
    switch (k) {
    case 1:
    case 2: return batch::k_batch_bicgstab<2>;
    case 3: return batch::k_batch_bicgstab<3>;
    case 4: return batch::k_batch_bicgstab<4>;
    case 5: return batch::k_batch_bicgstab<5>;
    case 6: return batch::k_batch_bicgstab<6>;
    case 7: return batch::k_batch_bicgstab<7>;
    default: return batch::k_batch_bicgstab<8>;
    }
}

void enqueue_solve(Batch& B, const batch::Args& a)
{
    cudaStream_t st = B.ctx->stream;
    batch::k_batch_init<<<(B.nsys + 255) / 256, 256, 0, st>>>(B.nsys, a.st, a.tickets, a.results, a.grid,
                                                               a.remaining);
    OWTK_CUDA(cudaGetLastError());
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(B.grid_blocks));
    cfg.blockDim = dim3(kBlock);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    OWTK_CUDA(cudaLaunchKernelEx(&cfg, solve_kernel(B.blocks_per_sm), a));
    OWTK_CUDA(cudaMemcpyAsync(B.h_results, a.results, sizeof(owtk_solver_result) * B.nsys, cudaMemcpyDeviceToHost,
                              st));
}

bool same_options(const batch::Options& p, const batch::Options& q) { return std::memcmp(&p, &q, sizeof p) == 0; }

void run_solve(Batch& B, const double* b, double* x, const owtk_solver_options& opt, owtk_solver_result* out)
{
    batch::Options o{opt.relative_tolerance, opt.absolute_tolerance, opt.breakdown_tolerance,
                     static_cast<long long>(opt.maximum_iterations), static_cast<long long>(opt.convergence_check_interval),
                     static_cast<long long>(opt.residual_replacement_interval)};
    const bool valid = std::isfinite(o.rtol) && std::isfinite(o.atol) && std::isfinite(o.btol) && o.rtol >= 0
        && o.atol >= 0 && o.btol > 0 && opt.maximum_iterations > 0 && opt.convergence_check_interval > 0
        && opt.maximum_iterations < (1ull << 40);
    if (!valid) {
        for (int i = 0; i < B.nsys; ++i) {
            out[i] = owtk_solver_result{};
            out[i].status = batch::kInvalid;
        }
        return;
    }
    const auto t0 = std::chrono::steady_clock::now();
    const batch::Args a = make_args(B, b, x, o);
    if (B.use_graph) {
        if (!B.exec || B.key_b != b || B.key_x != x || !same_options(B.key_o, o) || B.key_version != B.config_version) {
            if (B.exec) cudaGraphExecDestroy(B.exec);
            if (B.graph) cudaGraphDestroy(B.graph);
            B.exec = nullptr;
            B.graph = nullptr;
            OWTK_CUDA(cudaStreamBeginCapture(B.ctx->stream, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_solve(B, a);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(B.ctx->stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            OWTK_CUDA(cudaStreamEndCapture(B.ctx->stream, &B.graph));
            OWTK_CUDA(cudaGraphInstantiate(&B.exec, B.graph, 0));
            B.key_b = b;
            B.key_x = x;
            B.key_o = o;
            B.key_version = B.config_version;
            ++B.graph_captures;
        }
        OWTK_CUDA(cudaGraphLaunch(B.exec, B.ctx->stream));
        ++B.graph_launches;
    } else {
        enqueue_solve(B, a);
    }
    B.ctx->launched(2);   // initialisation + the persistent solver kernel
    B.ctx->sync();
    B.ctx->check_device_status();
    const double secs = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    for (int i = 0; i < B.nsys; ++i) {
        out[i] = B.h_results[i];
        out[i].solve_seconds = secs;
    }
}

float time_spmv_bench(Batch& B, int bs_filter, int reps)
{
    batch::Options o{};
    batch::Args a = make_args(B, B.scratch_b.as<double>(), B.scratch_x.as<double>(), o);
    a.bench_bs = bs_filter;
    cudaStream_t st = B.ctx->stream;
    batch::k_batch_spmv_bench<<<B.grid_blocks, kBlock, 0, st>>>(a);
    OWTK_CUDA(cudaGetLastError());
    cudaEvent_t e0, e1;
    OWTK_CUDA(cudaEventCreate(&e0));
    OWTK_CUDA(cudaEventCreate(&e1));
    OWTK_CUDA(cudaEventRecord(e0, st));
    for (int r = 0; r < reps; ++r) batch::k_batch_spmv_bench<<<B.grid_blocks, kBlock, 0, st>>>(a);
    OWTK_CUDA(cudaGetLastError());
    OWTK_CUDA(cudaEventRecord(e1, st));
    OWTK_CUDA(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return ms / reps;
}

}  // namespace

}  // namespace owtk

// ====================================================================== C ABI
using owtk::Batch;
using owtk::DeviceBuffer;
using owtk::fail;
using owtk::guarded;

struct owtk_batch : owtk::Batch {};

extern "C" {

owtk_status owtk_batch_create(owtk_context* ctx, size_t count, const owtk_batch_system* systems, owtk_batch** out)
{
    return guarded([&] {
        owtk::require(ctx != nullptr && out != nullptr && systems != nullptr, "null handle");
        if (count == 0 || count > (1u << 20)) fail(OWTK_ERR_INVALID_ARGUMENT, "batch needs 1..2^20 systems");
        auto B = std::make_unique<owtk_batch>();
        B->ctx = ctx;
        B->nsys = static_cast<int>(count);
        B->h_sys.resize(count);
        long long V = 0, E = 0, U = 0, NV = 0;
        for (size_t i = 0; i < count; ++i) {
            const auto& y = systems[i];
            if (y.owned == 0 || y.bs == 0 || y.bs > static_cast<size_t>(owtk::batch::kMaxBlockSize)
                || y.rowptr == nullptr || y.cols == nullptr || y.values == nullptr || y.rowptr[0] != 0)
                fail(OWTK_ERR_INVALID_ARGUMENT, "invalid batch system storage");
            auto& h = B->h_sys[i];
            h.u0 = U;
            h.val0 = NV;
            h.v0 = static_cast<int>(V);
            h.e0 = static_cast<int>(E);
            h.owned = static_cast<int>(y.owned);
            h.bs = static_cast<int>(y.bs);
            V += static_cast<long long>(y.owned);
            E += static_cast<long long>(y.rowptr[y.owned]);
            U += static_cast<long long>(y.owned * y.bs);
            NV += static_cast<long long>(y.rowptr[y.owned] * y.bs);
        }
        if (V >= (1ll << 31) || E >= (1ll << 31) || U >= (1ll << 31))
            fail(OWTK_ERR_INVALID_ARGUMENT, "batch too large for 32-bit vertex, entry or unknown indices");
        B->V = V;
        B->E = E;
        B->U = U;
        B->NV = NV;
        std::vector<std::int32_t> rowptr(V + 1), xoff(E);
        std::vector<double> vals(NV);
        B->sys_of_vertex.resize(V);
        for (size_t i = 0; i < count; ++i) {
            const auto& y = systems[i];
            const auto& h = B->h_sys[i];
            for (size_t r = 0; r < y.owned; ++r) {
                if (y.rowptr[r + 1] < y.rowptr[r]) fail(OWTK_ERR_INVALID_ARGUMENT, "rowptr must be non-decreasing");
                rowptr[h.v0 + r] = static_cast<std::int32_t>(h.e0 + y.rowptr[r]);
                B->sys_of_vertex[h.v0 + r] = static_cast<int>(i);
            }
            const size_t nnz = y.rowptr[y.owned];
            for (size_t e = 0; e < nnz; ++e) {
                if (y.cols[e] >= y.owned) fail(OWTK_ERR_OUT_OF_RANGE, "batch column index out of range");
                xoff[h.e0 + e] = static_cast<std::int32_t>(h.u0 + static_cast<long long>(y.cols[e]) * h.bs);
            }
            std::memcpy(vals.data() + h.val0, y.values, sizeof(double) * nnz * y.bs);
        }
        rowptr[V] = static_cast<std::int32_t>(E);
        B->h_rowptr = rowptr;
        cudaStream_t st = ctx->stream;
        B->rowptr = owtk::upload(st, rowptr);
        B->xoff = owtk::upload(st, xoff);
        B->vals = owtk::upload(st, vals);
        B->inv.allocate(U * sizeof(double) + 16);
        B->vec.allocate(static_cast<std::size_t>(owtk::batch::kVectors) * U * sizeof(double) + 16);
        OWTK_CUDA(cudaMemsetAsync(B->vec.ptr, 0, static_cast<std::size_t>(owtk::batch::kVectors) * U * sizeof(double),
                                  st));
        B->st.allocate(count * sizeof(owtk::batch::State));
        B->tickets.allocate(count * 2 * sizeof(unsigned));
        B->results.allocate(count * sizeof(owtk_solver_result));
        B->grid.allocate(sizeof(owtk::batch::Grid));
        B->remaining.allocate(16);
        B->scratch_b.allocate(U * sizeof(double) + 16);
        B->scratch_x.allocate(U * sizeof(double) + 16);
        OWTK_CUDA(cudaMallocHost(reinterpret_cast<void**>(&B->h_results), count * sizeof(owtk_solver_result)));
        for (int bs = 1; bs <= owtk::batch::kMaxBlockSize; ++bs) B->vpw[bs] = owtk::default_vpw(bs);
        // Counts 1..8 whose instance is resident at that count.
        B->max_blocks_per_sm = 0;
        for (int k = 1; k <= 8; ++k) {
            int resident = 0;
            OWTK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&resident, owtk::solve_kernel(k),
                                                                    owtk::batch::kBlock, 0));
            if (resident < k) break;
            B->max_blocks_per_sm = k;
        }
        if (B->max_blocks_per_sm < 1) fail(OWTK_ERR_CUDA, "batched solver kernel cannot be resident");
        owtk::set_grid(*B, std::min(B->max_blocks_per_sm, 4));
        // Jacobi inverse diagonal on the device.
        auto sov = owtk::upload(st, B->sys_of_vertex);
        owtk::batch::k_batch_jacobi<<<static_cast<unsigned>((V + 255) / 256), 256, 0, st>>>(
            B->nsys, B->sys.as<owtk::batch::Sys>(), sov.as<int>(), static_cast<int>(V), B->rowptr.as<int>(),
            B->xoff.as<int>(), B->vals.as<double>(), B->inv.as<double>(), ctx->status.as<unsigned>());
        OWTK_CUDA(cudaGetLastError());
        ctx->launched();
        ctx->sync();
        try {
            ctx->check_device_status();
        } catch (const owtk::Error& e) {
            fail(OWTK_ERR_INVALID_ARGUMENT, std::string("batch Jacobi setup: ") + e.message);
        }
        // Scratch right-hand side of ones for tuning runs.
        std::vector<double> ones(U, 1.0);
        OWTK_CUDA(cudaMemcpyAsync(B->scratch_b.ptr, ones.data(), U * sizeof(double), cudaMemcpyHostToDevice, st));
        ctx->sync();
        *out = B.release();
    });
}

owtk_status owtk_batch_destroy(owtk_batch* batch)
{
    return guarded([&] { delete batch; });
}

owtk_status owtk_batch_layout(const owtk_batch* batch, size_t* unknowns, uint64_t* offsets)
{
    return guarded([&] {
        owtk::require(batch != nullptr, "null handle");
        if (unknowns) *unknowns = static_cast<size_t>(batch->U);
        if (offsets) {
            for (int i = 0; i < batch->nsys; ++i) offsets[i] = static_cast<uint64_t>(batch->h_sys[i].u0);
            offsets[batch->nsys] = static_cast<uint64_t>(batch->U);
        }
    });
}

owtk_status owtk_batch_config(const owtk_batch* batch, uint32_t* blocks_per_sm, uint32_t* vertices_per_warp)
{
    return guarded([&] {
        owtk::require(batch != nullptr, "null handle");
        if (blocks_per_sm) *blocks_per_sm = static_cast<uint32_t>(batch->blocks_per_sm);
        if (vertices_per_warp)
            for (int bs = 0; bs <= owtk::batch::kMaxBlockSize; ++bs) vertices_per_warp[bs] = batch->vpw[bs];
    });
}

owtk_status owtk_batch_set_config(owtk_batch* batch, uint32_t blocks_per_sm, size_t bs, uint32_t vertices_per_warp)
{
    return guarded([&] {
        owtk::require(batch != nullptr, "null handle");
        if (bs > static_cast<size_t>(owtk::batch::kMaxBlockSize) || vertices_per_warp > 4096)
            fail(OWTK_ERR_INVALID_ARGUMENT, "invalid batch configuration");
        if (bs > 0 && vertices_per_warp > 0) {
            batch->vpw[bs] = static_cast<int>(vertices_per_warp);
            owtk::refresh_sys(*batch);
        }
        if (blocks_per_sm > 0 && static_cast<int>(blocks_per_sm) != batch->blocks_per_sm)
            owtk::set_grid(*batch, static_cast<int>(blocks_per_sm));
    });
}

owtk_status owtk_batch_use_graph(owtk_batch* batch, int enable)
{
    return guarded([&] {
        owtk::require(batch != nullptr, "null handle");
        batch->use_graph = enable != 0;
    });
}

owtk_status owtk_batch_graph_counts(const owtk_batch* batch, uint64_t* captures, uint64_t* launches)
{
    return guarded([&] {
        owtk::require(batch != nullptr, "null handle");
        if (captures) *captures = batch->graph_captures;
        if (launches) *launches = batch->graph_launches;
    });
}

owtk_status owtk_batch_autotune(owtk_batch* batch, const owtk_solver_options* options, uint32_t* blocks_per_sm,
                                uint32_t* vertices_per_warp)
{
    return guarded([&] {
        owtk::require(batch != nullptr, "null handle");
        Batch& B = *batch;
        // 1. Vertices per warp, per block size present: time one SpMV pass
        //    over that block size's systems for each candidate.
        bool present[owtk::batch::kMaxBlockSize + 1] = {};
        for (const auto& y : B.h_sys) present[y.bs] = true;
        for (int bs = 1; bs <= owtk::batch::kMaxBlockSize; ++bs) {
            if (!present[bs]) continue;
            const int base = owtk::default_vpw(bs);
            std::vector<int> cand;
            for (int v : {std::max(1, base / 4), std::max(1, base / 2), base, 2 * base, 4 * base, 8 * base})
                if (std::find(cand.begin(), cand.end(), v) == cand.end()) cand.push_back(v);
            float best = 1e30f;
            int pick = base;
            for (int v : cand) {
                B.vpw[bs] = v;
                owtk::refresh_sys(B);
                // Best of three timings: one timing alone picked differently
                // from run to run.
                float ms = owtk::time_spmv_bench(B, bs, 5);
                for (int trial = 0; trial < 2; ++trial) ms = std::min(ms, owtk::time_spmv_bench(B, bs, 5));
                if (ms < best) {
                    best = ms;
                    pick = v;
                }
            }
            B.vpw[bs] = pick;
            owtk::refresh_sys(B);
        }
        // 2. Resident blocks per SM: time a few iterations of the whole solve.
        owtk_solver_options o;
        if (options) o = *options;
        else owtk_default_options(&o);
        o.maximum_iterations = 4;
        o.relative_tolerance = 0.0;
        o.absolute_tolerance = 0.0;
        std::vector<owtk_solver_result> res(B.nsys);
        float best = 1e30f;
        int pick = B.blocks_per_sm;
        const bool graph = B.use_graph;
        B.use_graph = false;
        for (int k = 1; k <= B.max_blocks_per_sm; ++k) {
            owtk::set_grid(B, k);
            float ms = 1e30f;
            for (int rep = 0; rep < 4; ++rep) {   // the first is a warm-up; best of the other three
                OWTK_CUDA(cudaMemsetAsync(B.scratch_x.ptr, 0, B.U * sizeof(double), B.ctx->stream));
                const auto t0 = std::chrono::steady_clock::now();
                owtk::run_solve(B, B.scratch_b.as<double>(), B.scratch_x.as<double>(), o, res.data());
                const float t = std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
                if (rep > 0) ms = std::min(ms, t);
            }
            if (ms < best) {
                best = ms;
                pick = k;
            }
        }
        B.use_graph = graph;
        owtk::set_grid(B, pick);
        if (blocks_per_sm) *blocks_per_sm = static_cast<uint32_t>(B.blocks_per_sm);
        if (vertices_per_warp)
            for (int bs = 0; bs <= owtk::batch::kMaxBlockSize; ++bs) vertices_per_warp[bs] = B.vpw[bs];
    });
}

owtk_status owtk_batch_solve(owtk_batch* batch, const double* device_rhs, double* device_x,
                             const owtk_solver_options* options, owtk_solver_result* results)
{
    return guarded([&] {
        owtk::require(batch != nullptr && device_rhs != nullptr && device_x != nullptr && options != nullptr
                          && results != nullptr,
                      "null argument");
        owtk::run_solve(*batch, device_rhs, device_x, *options, results);
    });
}

owtk_status owtk_batch_solve_host(owtk_batch* batch, const double* host_rhs, double* host_x,
                                  const owtk_solver_options* options, owtk_solver_result* results)
{
    return guarded([&] {
        owtk::require(batch != nullptr && host_rhs != nullptr && host_x != nullptr && options != nullptr
                          && results != nullptr,
                      "null argument");
        Batch& B = *batch;
        const std::size_t bytes = B.U * sizeof(double);
        if (!B.stage_b.ptr) {
            B.stage_b.allocate(bytes + 16);
            B.stage_x.allocate(bytes + 16);
        }
        cudaStream_t st = B.ctx->stream;
        OWTK_CUDA(cudaMemcpyAsync(B.stage_b.ptr, host_rhs, bytes, cudaMemcpyHostToDevice, st));
        OWTK_CUDA(cudaMemcpyAsync(B.stage_x.ptr, host_x, bytes, cudaMemcpyHostToDevice, st));
        owtk::run_solve(B, B.stage_b.as<double>(), B.stage_x.as<double>(), *options, results);
        OWTK_CUDA(cudaMemcpyAsync(host_x, B.stage_x.ptr, bytes, cudaMemcpyDeviceToHost, st));
        B.ctx->sync();
    });
}

}  // extern "C"
