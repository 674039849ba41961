// Level-scheduled triangular sweeps (sm_100a): ILU(k) numeric factorisation,
// ILU forward/backward solves and SSOR forward/backward sweeps.
//
// Schedule (built once at symbolic setup, reused by every numeric update and
// apply): rows are ordered by (level, row) and cut into warp tasks of up to
// 32/bs rows from a single level, so rows inside a task never depend on each
// other.  Warps take tasks in order from a monotone 64-bit ticket; a task's
// lanes are (row, component) pairs.  Before reading a dependency a lane waits
// for that row's epoch flag (acquire); after a task's rows are written the
// warp publishes their flags (fence + release).  Every dependency lies in an
// earlier task, held by a warp that is already running, so the sweep always
// makes progress; each wait is still bounded (kSpinLimit polls) and a wait
// that gives up sets the timeout bit of the device status word and carries
// on, so a kernel can never hang the GPU.
//
// Per (row, component) the arithmetic is the reference's, term by term and
// in entry order, with explicit rounding (device_common.cuh), so results equal
// the CPU path bit for bit whatever order the rows complete in.

#include <cfloat>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

constexpr int kSpinLimit = 1 << 22;

enum Mode { kIluForward, kIluBackward, kSsorForward, kSsorBackward, kIluFactor };

template<class T>
struct SweepArgs {
    const int* order;
    const int* task_start;
    int tasks;
    const int* rowptr;      // dependency pattern (ILU factor pattern or matrix pattern)
    const int* cols;
    const int* diagpos;     // ILU only
    T* vals;                // ILU factor values (written by the factorisation) or matrix/edge values
    const T* diag;          // SSOR diagonal
    T* inv;                 // ILU inverse diagonal (written by the factorisation)
    const T* in;
    T* out;
    T* work;                // SSOR forward result
    T omega;
    int owned;
    int bs;
    unsigned* flags;
    unsigned epoch;
    unsigned long long* ticket;
    unsigned long long base;
    unsigned* status;
    const int* upd_start;   // factorisation update lists
    const int* upd_target;
    const int* upd_upper;
};

__device__ __forceinline__ void wait_row(const unsigned* flags, int row, unsigned epoch, unsigned* status)
{
    if (ld_acquire(flags + row) == epoch) return;
    for (int it = 0; it < kSpinLimit; ++it) {
        __nanosleep(32);
        if (ld_acquire(flags + row) == epoch) return;
    }
    atomicOr(status, kErrTimeout);
}

template<class T> __device__ __forceinline__ T pivot_tolerance();
template<> __device__ __forceinline__ double pivot_tolerance<double>() { return 64.0 * DBL_EPSILON; }
template<> __device__ __forceinline__ float pivot_tolerance<float>() { return 64.0f * FLT_EPSILON; }

template<class T, int MODE>
__device__ __forceinline__ void row_body(const SweepArgs<T>& a, int row, int c0, int cstep)
{
    const int bs = a.bs;
    const std::size_t rb = static_cast<std::size_t>(row) * bs;
    if (MODE == kIluForward) {
        const int b = a.rowptr[row], d = a.diagpos[row];
        for (int e = b; e < d; ++e) wait_row(a.flags, a.cols[e], a.epoch, a.status);
        for (int c = c0; c < bs; c += cstep) {
            T y = a.in[rb + c];
            for (int e = b; e < d; ++e)
                y = sub_rn(y, mul_rn(a.vals[static_cast<std::size_t>(e) * bs + c],
                                     __ldcg(a.out + static_cast<std::size_t>(a.cols[e]) * bs + c)));
            a.out[rb + c] = y;
        }
    } else if (MODE == kIluBackward) {
        const int d = a.diagpos[row], end = a.rowptr[row + 1];
        for (int e = d + 1; e < end; ++e) wait_row(a.flags, a.cols[e], a.epoch, a.status);
        for (int c = c0; c < bs; c += cstep) {
            T x = a.out[rb + c];
            for (int e = d + 1; e < end; ++e)
                x = sub_rn(x, mul_rn(a.vals[static_cast<std::size_t>(e) * bs + c],
                                     __ldcg(a.out + static_cast<std::size_t>(a.cols[e]) * bs + c)));
            a.out[rb + c] = mul_rn(x, a.inv[rb + c]);
        }
    } else if (MODE == kSsorForward) {
        const int b = a.rowptr[row], end = a.rowptr[row + 1];
        for (int e = b; e < end; ++e) {
            const int col = a.cols[e];
            if (col < row) wait_row(a.flags, col, a.epoch, a.status);
        }
        for (int c = c0; c < bs; c += cstep) {
            T y = a.in[rb + c];
            for (int e = b; e < end; ++e) {
                const int col = a.cols[e];
                if (col >= row || col >= a.owned) continue;
                y = sub_rn(y, mul_rn(mul_rn(a.omega, a.vals[static_cast<std::size_t>(e) * bs + c]),
                                     __ldcg(a.work + static_cast<std::size_t>(col) * bs + c)));
            }
            a.work[rb + c] = div_rn(y, a.diag[rb + c]);
        }
    } else if (MODE == kSsorBackward) {
        const int b = a.rowptr[row], end = a.rowptr[row + 1];
        for (int e = b; e < end; ++e) {
            const int col = a.cols[e];
            if (col > row && col < a.owned) wait_row(a.flags, col, a.epoch, a.status);
        }
        for (int c = c0; c < bs; c += cstep) {
            T z = mul_rn(a.diag[rb + c], a.work[rb + c]);
            for (int e = b; e < end; ++e) {
                const int col = a.cols[e];
                if (col <= row || col >= a.owned) continue;
                z = sub_rn(z, mul_rn(mul_rn(a.omega, a.vals[static_cast<std::size_t>(e) * bs + c]),
                                     __ldcg(a.out + static_cast<std::size_t>(col) * bs + c)));
            }
            a.out[rb + c] = div_rn(z, a.diag[rb + c]);
        }
    } else {  // kIluFactor: IKJ elimination of one row (preconditioner.hpp:442-469)
        const int b = a.rowptr[row], d = a.diagpos[row];
        for (int l = b; l < d; ++l) wait_row(a.flags, a.cols[l], a.epoch, a.status);
        const T tol = pivot_tolerance<T>();
        for (int c = c0; c < bs; c += cstep) {
            for (int l = b; l < d; ++l) {
                const int p = a.cols[l];
                const T piv = __ldcg(a.vals + static_cast<std::size_t>(a.diagpos[p]) * bs + c);
                if (fabs(piv) <= tol) atomicOr(a.status, kErrZeroPivot);
                const T lv = div_rn(a.vals[static_cast<std::size_t>(l) * bs + c], piv);
                a.vals[static_cast<std::size_t>(l) * bs + c] = lv;
                for (int u = a.upd_start[l]; u < a.upd_start[l + 1]; ++u) {
                    const std::size_t t = static_cast<std::size_t>(a.upd_target[u]) * bs + c;
                    const T uv = __ldcg(a.vals + static_cast<std::size_t>(a.upd_upper[u]) * bs + c);
                    a.vals[t] = sub_rn(a.vals[t], mul_rn(lv, uv));
                }
            }
            const T dv = a.vals[static_cast<std::size_t>(d) * bs + c];
            if (!isfinite(dv) || fabs(dv) <= tol) atomicOr(a.status, kErrZeroPivot);
            a.inv[rb + c] = div_rn(T(1), dv);
        }
    }
}

template<class T, int MODE>
__global__ void __launch_bounds__(kThreads) k_sweep(SweepArgs<T> a)
{
    const int lane = threadIdx.x & 31;
    const int bs = a.bs;
    for (;;) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(a.ticket, 1ull) - a.base;
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= static_cast<unsigned long long>(a.tasks)) break;
        const int s = a.task_start[t], nrows = a.task_start[t + 1] - s;
        int rl, c0, cstep;
        if (bs <= 32) {
            rl = lane / bs;
            c0 = lane - rl * bs;
            cstep = bs;
        } else {
            rl = 0;
            c0 = lane;
            cstep = 32;
        }
        if (rl < nrows) row_body<T, MODE>(a, a.order[s + rl], c0, cstep);
        __syncwarp();
        if (lane < nrows) {
            __threadfence();
            st_release(a.flags + a.order[s + lane], a.epoch);
        }
    }
}

template<class T, int MODE>
void launch(Context& c, Preconditioner& p, Sweep& s, SweepArgs<T>& a)
{
    if (s.tasks == 0) return;
    if (++p.epoch == 0xffffffffu) {
        OWTK_CUDA(cudaMemsetAsync(p.flags.ptr, 0, p.owned * sizeof(unsigned), c.stream));
        p.epoch = 1;
    }
    const int warps_per_block = kThreads / 32;
    int blocks = (s.tasks + warps_per_block - 1) / warps_per_block;
    const int cap = c.sm_count * 8;
    if (blocks > cap) blocks = cap;
    a.order = s.order.as<int>();
    a.task_start = s.task_start.as<int>();
    a.tasks = s.tasks;
    a.flags = p.flags.as<unsigned>();
    a.epoch = p.epoch;
    a.ticket = p.ticket.as<unsigned long long>();
    a.base = p.ticket_base;
    a.status = c.status.as<unsigned>();
    a.owned = static_cast<int>(p.owned);
    a.bs = static_cast<int>(p.bs);
    k_sweep<T, MODE><<<blocks, kThreads, 0, c.stream>>>(a);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
    p.ticket_base += static_cast<unsigned long long>(s.tasks)
        + static_cast<unsigned long long>(blocks) * warps_per_block;
}

}  // namespace

namespace kern {

template<class T> void ilu_factorize(Context& c, Preconditioner& p, const T* matrix_values)
{
    gather_values<T>(c, p.f_cols.size(), p.bs, p.d_fsource.as<std::int64_t>(), matrix_values,
                     p.d_fvalues.as<T>());
    SweepArgs<T> a{};
    a.rowptr = p.d_frowptr.as<int>();
    a.cols = p.d_fcols.as<int>();
    a.diagpos = p.d_fdiagpos.as<int>();
    a.vals = p.d_fvalues.as<T>();
    a.inv = p.inv_diag.as<T>();
    a.upd_start = p.d_upd_start.as<int>();
    a.upd_target = p.d_upd_target.as<int>();
    a.upd_upper = p.d_upd_upper.as<int>();
    launch<T, kIluFactor>(c, p, p.lower, a);
}

template<class T> void ilu_apply(Context& c, Preconditioner& p, const T* in, T* out)
{
    SweepArgs<T> a{};
    a.rowptr = p.d_frowptr.as<int>();
    a.cols = p.d_fcols.as<int>();
    a.diagpos = p.d_fdiagpos.as<int>();
    a.vals = p.d_fvalues.as<T>();
    a.inv = p.inv_diag.as<T>();
    a.in = in;
    a.out = out;
    launch<T, kIluForward>(c, p, p.lower, a);
    launch<T, kIluBackward>(c, p, p.upper, a);
}

template<class T> void ssor_apply(Context& c, Preconditioner& p, const T* in, T* out)
{
    const Matrix& m = *p.matrix;
    SweepArgs<T> a{};
    a.rowptr = m.rowptr.as<int>();
    a.cols = m.cols.as<int>();
    a.vals = const_cast<T*>(static_cast<const T*>(m.value_ptr()));
    a.diag = p.kind == OWTK_PC_SPLIT_SSOR ? static_cast<const T*>(m.diag) : p.diag_cache.as<T>();
    a.in = in;
    a.out = out;
    a.work = p.work.as<T>();
    a.omega = static_cast<T>(p.parameter);
    launch<T, kSsorForward>(c, p, p.lower, a);
    launch<T, kSsorBackward>(c, p, p.upper, a);
    const T omega = static_cast<T>(p.parameter);
    if (omega != T(1)) scale<T>(c, p.owned * p.bs, omega * (T(2) - omega), out);
}

template void ilu_factorize<double>(Context&, Preconditioner&, const double*);
template void ilu_factorize<float>(Context&, Preconditioner&, const float*);
template void ilu_apply<double>(Context&, Preconditioner&, const double*, double*);
template void ilu_apply<float>(Context&, Preconditioner&, const float*, float*);
template void ssor_apply<double>(Context&, Preconditioner&, const double*, double*);
template void ssor_apply<float>(Context&, Preconditioner&, const float*, float*);

}  // namespace kern
}  // namespace owtk
