// Level-scheduled triangular sweeps (sm_100a): ILU(k) numeric factorisation,
// ILU forward/backward solves and SSOR forward/backward sweeps.
//
// Schedule (built once at symbolic setup, reused by every numeric update and
// apply): rows are ordered by (level, row) and cut into warp tasks of up to
// 32/bs rows from a single level, so rows inside a task never depend on each
// other.  Warps take tasks in order from a monotone 64-bit ticket; a task's
// lanes are (row, component) pairs.  Every dependency lies in an earlier task,
// held by a warp that is already running, so a sweep always makes progress.
//
// Applies (ILU and SSOR sweeps) synchronise on the data itself: the sweep's
// output is first filled with a signalling-NaN sentinel that no arithmetic
// result can equal (NaN results are stored as the canonical quiet NaN), and a
// lane reads a dependency with a relaxed 8-byte load until it is no longer
// the sentinel.  One load both waits and fetches, so a level costs about one
// L2 round trip.  For block sizes up to 32 a lane publishes its (row,
// component) from inside its polling loop, so a row waits for its own
// dependencies only, not for those of the other rows of its warp's task
// (2M-vertex mesh, bs 3: ILU(0) apply 5.75 -> 5.02 ms, SSOR 8.44 -> 6.00 ms);
// the dense-block sweeps publish a block row, or in the backward sweep a row
// once all of its block rows are final (FP64 dense-block ILU(0)-FGMRES on
// that mesh 150.6 -> 92.3 ms).  A second poll round in flight, half a round
// trip behind the first, was slower (5.0 -> 9.6 ms): the polls and the spin
// that staggers them cost more issue and L2 traffic than they save.
// The numeric factorisation, which updates factor entries in
// place, publishes per-row epoch flags instead (fence + release / relaxed
// loads + fence).  Every wait is bounded (kSpinLimit polls): a wait that gives
// up sets the timeout bit of the device status word and carries on, and later
// waits of the launch then return at once, so a kernel can never hang the GPU.
//
// Per (row, component) the arithmetic is the reference's, term by term and
// in entry order, with explicit rounding (device_common.cuh), so results equal
// the CPU path bit for bit whatever order the rows complete in.

#include <cfloat>
#include <cmath>
#include <cstdlib>

#include <cuda_bf16.h>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

constexpr int kSpinLimit = 1 << 22;

enum Mode {
    kIluForward, kIluBackward, kSsorForward, kSsorBackward, kIluFactor,
    kBlockForward, kBlockBackward, kBlockFactor
};

constexpr bool is_factor(int mode) { return mode == kIluFactor || mode == kBlockFactor; }
constexpr int kMaxBlock = 4;   // dense-block ILU handles bs <= 4

// T: vector / arithmetic type.  F: factor storage type (T, or float / bf16
// storage under FP32 arithmetic).
template<class T, class F = T>
struct SweepArgs {
    const int* order;
    const int* task_start;
    int tasks;
    const int* rowptr;      // dependency pattern (ILU factor pattern or matrix pattern)
    const int* cols;
    const int* diagpos;     // ILU only
    const int* seg;         // ILU applies on packed segments: entries of order position q in [seg[q], seg[q+1])
    F* vals;                // ILU factor values (written by the factorisation) or matrix/edge values
    const T* diag;          // SSOR diagonal
    F* inv;                 // ILU inverse diagonal (blocks for the dense-block ILU)
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
    int spin_limit;         // polls before an apply's dependency wait gives up (0: kSpinLimit)
};

constexpr int kChunk = 8;   // dependency entries handled per unrolled step

__device__ __forceinline__ unsigned ld_relaxed(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

template<class T> struct Bits;
template<> struct Bits<double> {
    using U = unsigned long long;
    static constexpr U kSentinel = 0x7ff0dead5eed0badull;   // signalling NaN
    static constexpr U kQuietNan = 0x7ff8000000000000ull;
};
template<> struct Bits<float> {
    using U = unsigned;
    static constexpr U kSentinel = 0x7f80deadu;              // signalling NaN
    static constexpr U kQuietNan = 0x7fc00000u;
};

__device__ __forceinline__ unsigned long long ld_relaxed_bits(const double* p)
{
    unsigned long long v;
    asm volatile("ld.relaxed.gpu.global.b64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_relaxed_bits(const float* p)
{
    unsigned v;
    asm volatile("ld.relaxed.gpu.global.b32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}
__device__ __forceinline__ void st_relaxed(double* p, double v)
{
    asm volatile("st.relaxed.gpu.global.f64 [%0], %1;" ::"l"(p), "d"(v) : "memory");
}
__device__ __forceinline__ void st_relaxed(float* p, float v)
{
    asm volatile("st.relaxed.gpu.global.f32 [%0], %1;" ::"l"(p), "f"(v) : "memory");
}
__device__ __forceinline__ double from_bits(unsigned long long u) { return __longlong_as_double(static_cast<long long>(u)); }
__device__ __forceinline__ float from_bits(unsigned u) { return __uint_as_float(u); }

// Publish a sweep result: NaN is stored canonically so it can never equal the sentinel.
template<class T>
__device__ __forceinline__ void publish(T* p, T v)
{
    if (v != v) v = from_bits(Bits<T>::kQuietNan);
    st_relaxed(p, v);
}

template<class T>
__global__ void k_fill_sentinel(std::size_t n, T* x)
{
    const std::size_t i = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) reinterpret_cast<typename Bits<T>::U*>(x)[i] = Bits<T>::kSentinel;
}

// Bounded spin on one dependency flag.  Once any wait of the launch has given
// up (status timeout bit), later waits return at once, so a sweep with a
// broken schedule ends after one timeout instead of one per dependency.
__device__ __noinline__ void spin_until(const unsigned* flag, unsigned epoch, unsigned* status)
{
    for (int it = 0; it < kSpinLimit; ++it) {
        if (ld_relaxed(flag) == epoch) return;
        if (it >= 256) __nanosleep(64);
        if ((it & 1023) == 1023 && (*reinterpret_cast<volatile unsigned*>(status) & kErrTimeout)) return;
    }
    atomicOr(status, kErrTimeout);
}

// Wait until every dependency of a row is published.  `filter`: 0 all
// entries of [b, e) are dependencies (ILU factor rows), 1 columns < row
// (SSOR forward), 2 row < column < owned (SSOR backward).  Flags are loaded
// kChunk at a time with relaxed loads; one fence afterwards gives acquire
// ordering for the dependency values read next.
template<int FILTER>
__device__ __forceinline__ void wait_deps(const unsigned* flags, const int* cols, int b, int e, int row,
                                          int owned, unsigned epoch, unsigned* status)
{
    for (int k0 = b; k0 < e; k0 += kChunk) {
        int cc[kChunk];
        unsigned f[kChunk];
#pragma unroll
        for (int j = 0; j < kChunk; ++j) {
            int c = k0 + j < e ? cols[k0 + j] : -1;
            if (FILTER == 1 && c >= row) c = -1;
            if (FILTER == 2 && (c <= row || c >= owned)) c = -1;
            cc[j] = c;
        }
#pragma unroll
        for (int j = 0; j < kChunk; ++j) f[j] = cc[j] >= 0 ? ld_relaxed(flags + cc[j]) : epoch;
#pragma unroll
        for (int j = 0; j < kChunk; ++j)
            if (f[j] != epoch) spin_until(flags + cc[j], epoch, status);
    }
    __threadfence();
}

template<class T> __device__ __forceinline__ T pivot_tolerance();
template<> __device__ __forceinline__ double pivot_tolerance<double>() { return 64.0 * DBL_EPSILON; }
template<> __device__ __forceinline__ float pivot_tolerance<float>() { return 64.0f * FLT_EPSILON; }

template<class T> __device__ __forceinline__ T cvt(double v) { return static_cast<T>(v); }
template<class T> __device__ __forceinline__ T cvt(float v) { return static_cast<T>(v); }
template<class T> __device__ __forceinline__ T cvt(__nv_bfloat16 v) { return static_cast<T>(__bfloat162float(v)); }

// y -= sum_e vals[e][c] * dep[col_e][c] over e in [b, e) in entry order;
// FILTER as in wait_deps, OMEGA multiplies each coefficient first (SSOR).
// POLL: dependency values are read with relaxed loads and waited on until
// they differ from the sentinel (applies); otherwise they are already final
// (the caller waited on flags) and read through L2.
template<class T, class F, int FILTER, bool OMEGA, bool POLL>
__device__ __forceinline__ T eliminate(T y, const SweepArgs<T, F>& a, const T* dep, int b, int e, int row, int c)
{
    using U = typename Bits<T>::U;
    const int bs = a.bs;
    for (int k0 = b; k0 < e; k0 += kChunk) {
        T fv[kChunk], xv[kChunk];
        U xb[kChunk];
        const T* src[kChunk];
        bool on[kChunk];
#pragma unroll
        for (int j = 0; j < kChunk; ++j) {
            const int k = k0 + j;
            int col = k < e ? a.cols[k] : -1;
            if (FILTER == 1 && col >= row) col = -1;
            if (FILTER == 2 && (col <= row || col >= a.owned)) col = -1;
            on[j] = col >= 0;
            src[j] = dep + static_cast<std::size_t>(on[j] ? col : 0) * bs + c;
            if (on[j]) {
                fv[j] = cvt<T>(a.vals[static_cast<std::size_t>(k) * bs + c]);
                if (POLL) xb[j] = ld_relaxed_bits(src[j]);
                else xv[j] = __ldcg(src[j]);
            }
        }
        if (POLL) {
            // Re-poll every still-pending dependency together: one L2 round
            // trip per round however many are pending.
            for (int it = 0;; ++it) {
                bool pending = false;
#pragma unroll
                for (int j = 0; j < kChunk; ++j) pending |= on[j] && xb[j] == Bits<T>::kSentinel;
                if (!pending) break;
                if (it >= a.spin_limit) {
                    atomicOr(a.status, kErrTimeout);
                    break;
                }
                if ((it & 1023) == 1023 && (*reinterpret_cast<volatile unsigned*>(a.status) & kErrTimeout)) break;
                if (it >= 256) __nanosleep(32);
#pragma unroll
                for (int j = 0; j < kChunk; ++j)
                    if (on[j] && xb[j] == Bits<T>::kSentinel) xb[j] = ld_relaxed_bits(src[j]);
            }
#pragma unroll
            for (int j = 0; j < kChunk; ++j) xv[j] = from_bits(xb[j]);
        }
#pragma unroll
        for (int j = 0; j < kChunk; ++j) {
            if (on[j]) {
                const T coef = OMEGA ? mul_rn(a.omega, fv[j]) : fv[j];
                y = sub_rn(y, mul_rn(coef, xv[j]));
            }
        }
    }
    return y;
}

// eliminate() for one (row, component) per lane (block size <= 32), with the
// result published from inside the polling loop: a lane publishes as soon as
// its own dependencies have arrived instead of when the whole warp's have, so
// a level waits for a row's dependencies, not for its task's.  The loop is
// warp-uniform (all 32 lanes take part; `valid` false for lanes without a
// row) and ends when every lane is done.  FIN: 0 publish y, 1 y * fin, 2 y /
// fin.  Same operations in the same order as eliminate() + publish().
template<class T, class F, int FILTER, bool OMEGA, int FIN>
__device__ __forceinline__ void eliminate_publish(bool valid, T y, const SweepArgs<T, F>& a, const T* dep, int b,
                                                  int e, int row, int c, T fin, T* dst)
{
    using U = typename Bits<T>::U;
    const int bs = a.bs;
    T fv[kChunk];
    U xb[kChunk];
    const T* src[kChunk];
    bool on[kChunk];
    int k0 = b, it = 0;
    bool loaded = false, done = !valid;
    for (;;) {
        if (!done) {
            if (!loaded && k0 >= e) {
                publish(dst, FIN == 1 ? mul_rn(y, fin) : FIN == 2 ? div_rn(y, fin) : y);
                done = true;
            } else {
                if (!loaded) {
#pragma unroll
                    for (int j = 0; j < kChunk; ++j) {
                        const int k = k0 + j;
                        int col = k < e ? a.cols[k] : -1;
                        if (FILTER == 1 && col >= row) col = -1;
                        if (FILTER == 2 && (col <= row || col >= a.owned)) col = -1;
                        on[j] = col >= 0;
                        src[j] = dep + static_cast<std::size_t>(on[j] ? col : 0) * bs + c;
                        if (on[j]) {
                            fv[j] = cvt<T>(a.vals[static_cast<std::size_t>(k) * bs + c]);
                            xb[j] = ld_relaxed_bits(src[j]);
                        }
                    }
                    loaded = true;
                }
                bool pending = false;
#pragma unroll
                for (int j = 0; j < kChunk; ++j) pending |= on[j] && xb[j] == Bits<T>::kSentinel;
                if (pending) {
                    if (it >= a.spin_limit) {
                        atomicOr(a.status, kErrTimeout);
                        pending = false;
                    } else if ((it & 1023) == 1023
                               && (*reinterpret_cast<volatile unsigned*>(a.status) & kErrTimeout)) {
                        pending = false;
                    }
                }
                if (!pending) {
#pragma unroll
                    for (int j = 0; j < kChunk; ++j) {
                        if (on[j]) {
                            const T coef = OMEGA ? mul_rn(a.omega, fv[j]) : fv[j];
                            y = sub_rn(y, mul_rn(coef, from_bits(xb[j])));
                        }
                    }
                    k0 += kChunk;
                    loaded = false;
                    if (k0 >= e) {
                        publish(dst, FIN == 1 ? mul_rn(y, fin) : FIN == 2 ? div_rn(y, fin) : y);
                        done = true;
                    }
                } else {
                    if (it >= 256) __nanosleep(32);
                    ++it;
#pragma unroll
                    for (int j = 0; j < kChunk; ++j)
                        if (on[j] && xb[j] == Bits<T>::kSentinel) xb[j] = ld_relaxed_bits(src[j]);
                }
            }
        }
        if (!__any_sync(0xffffffffu, !done)) break;
    }
}

// ILU / SSOR apply of (row, component c) with early publication; row < 0:
// a lane without a row, which only takes part in the warp's votes.  q: the
// row's position in the task order (its packed segment, when a.seg is set).
template<class T, class F, int MODE>
__device__ __forceinline__ void apply_lane(const SweepArgs<T, F>& a, int row, int q, int c)
{
    const bool valid = row >= 0;
    const std::size_t o = valid ? static_cast<std::size_t>(row) * a.bs + c : 0;
    if constexpr (MODE == kIluForward) {
        int b = 0, d = 0;
        if (valid) {
            b = a.seg ? a.seg[q] : a.rowptr[row];
            d = a.seg ? a.seg[q + 1] : a.diagpos[row];
        }
        const T own = valid ? a.in[o] : T(0);
        eliminate_publish<T, F, 0, false, 0>(valid, own, a, a.work, b, d, row, c, T(1), a.work + o);
    } else if constexpr (MODE == kIluBackward) {
        int b = 0, end = 0;
        if (valid) {
            b = a.seg ? a.seg[q] : a.diagpos[row] + 1;
            end = a.seg ? a.seg[q + 1] : a.rowptr[row + 1];
        }
        const T own = valid ? a.work[o] : T(0), inv = valid ? cvt<T>(a.inv[o]) : T(1);
        eliminate_publish<T, F, 0, false, 1>(valid, own, a, a.out, b, end, row, c, inv, a.out + o);
    } else if constexpr (MODE == kSsorForward) {
        const int b = valid ? a.rowptr[row] : 0, end = valid ? a.rowptr[row + 1] : 0;
        const T own = valid ? a.in[o] : T(0), dg = valid ? a.diag[o] : T(1);
        eliminate_publish<T, F, 1, true, 2>(valid, own, a, a.work, b, end, row, c, dg, a.work + o);
    } else if constexpr (MODE == kSsorBackward) {
        const int b = valid ? a.rowptr[row] : 0, end = valid ? a.rowptr[row + 1] : 0;
        const T dg = valid ? a.diag[o] : T(1);
        const T z0 = valid ? mul_rn(dg, a.work[o]) : T(0);
        eliminate_publish<T, F, 2, true, 2>(valid, z0, a, a.out, b, end, row, c, dg, a.out + o);
    }
}

constexpr bool is_scalar_apply(int mode)
{
    return mode == kIluForward || mode == kIluBackward || mode == kSsorForward || mode == kSsorBackward;
}

constexpr bool is_lane_apply(int mode)
{
    return is_scalar_apply(mode) || mode == kBlockForward || mode == kBlockBackward;
}

// Dense-block rows: acc -= sum_k (sum_j B_k[i][j] dep[col_k][j]) over k in
// [b, e), each block-row product summed from +0 over j (the dense SpMV's
// order); dependency values are polled until published.
template<class T, class F>
__device__ __forceinline__ T block_eliminate(T acc, const SweepArgs<T, F>& a, const T* dep, int b, int e, int i)
{
    using U = typename Bits<T>::U;
    const int bs = a.bs;
    constexpr int kQ = 4;   // block entries per round
    for (int k0 = b; k0 < e; k0 += kQ) {
        T co[kQ][kMaxBlock], xv[kQ][kMaxBlock];
        U xb[kQ][kMaxBlock];
        const T* src[kQ];
        bool on[kQ];
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            const int k = k0 + q;
            on[q] = k < e;
            src[q] = dep + static_cast<std::size_t>(on[q] ? a.cols[k] : 0) * bs;
#pragma unroll
            for (int j = 0; j < kMaxBlock; ++j) {
                if (on[q] && j < bs) {
                    co[q][j] = cvt<T>(a.vals[(static_cast<std::size_t>(k) * bs + i) * bs + j]);
                    xb[q][j] = ld_relaxed_bits(src[q] + j);
                }
            }
        }
        for (int it = 0;; ++it) {
            bool pending = false;
#pragma unroll
            for (int q = 0; q < kQ; ++q)
#pragma unroll
                for (int j = 0; j < kMaxBlock; ++j)
                    pending |= on[q] && j < bs && xb[q][j] == Bits<T>::kSentinel;
            if (!pending) break;
            if (it >= a.spin_limit) {
                atomicOr(a.status, kErrTimeout);
                break;
            }
            if ((it & 1023) == 1023 && (*reinterpret_cast<volatile unsigned*>(a.status) & kErrTimeout)) break;
            if (it >= 256) __nanosleep(32);
#pragma unroll
            for (int q = 0; q < kQ; ++q)
#pragma unroll
                for (int j = 0; j < kMaxBlock; ++j)
                    if (on[q] && j < bs && xb[q][j] == Bits<T>::kSentinel) xb[q][j] = ld_relaxed_bits(src[q] + j);
        }
#pragma unroll
        for (int q = 0; q < kQ; ++q) {
            if (!on[q]) continue;
            T sum = 0;
#pragma unroll
            for (int j = 0; j < kMaxBlock; ++j) {
                if (j < bs) {
                    xv[q][j] = from_bits(xb[q][j]);
                    sum = add_rn(sum, mul_rn(co[q][j], xv[q][j]));
                }
            }
            acc = sub_rn(acc, sum);
        }
    }
    return acc;
}

// Dense-block apply of block row i of `row` with early publication (the
// counterpart of eliminate_publish): the forward sweep publishes each block
// row as soon as its own dependencies have arrived; the backward sweep forms
// w = y - sum U x per block row, and a row publishes x = Dinv w (shuffles
// over its bs lanes, the same sum order as the warp path) once all of its
// lanes hold their w.  Warp-uniform loop; row < 0 for lanes without a row.
template<class T, class F, bool BACK>
__device__ __forceinline__ void block_apply_lane(const SweepArgs<T, F>& a, int row, int i, int rl)
{
    using U = typename Bits<T>::U;
    const int bs = a.bs;
    const bool valid = row >= 0;
    const std::size_t rb = valid ? static_cast<std::size_t>(row) * bs : 0;
    const T* dep = BACK ? a.out : a.work;
    int b = 0, e = 0;
    T acc = 0, dinv[kMaxBlock];
#pragma unroll
    for (int j = 0; j < kMaxBlock; ++j) dinv[j] = 0;
    if (valid) {
        if (BACK) {
            b = a.diagpos[row] + 1;
            e = a.rowptr[row + 1];
            acc = a.work[rb + i];
#pragma unroll
            for (int j = 0; j < kMaxBlock; ++j)
                if (j < bs) dinv[j] = cvt<T>(a.inv[static_cast<std::size_t>(row) * bs * bs + i * bs + j]);
        } else {
            b = a.rowptr[row];
            e = a.diagpos[row];
            acc = a.in[rb + i];
        }
    }
    constexpr int kQ = 4;   // block entries per round
    T co[kQ][kMaxBlock];
    U xb[kQ][kMaxBlock];
    const T* src[kQ];
    bool on[kQ];
    int k0 = b, it = 0;
    bool loaded = false, ready = !valid, done = !valid;
    const int base = (rl * bs) & 31;
    const unsigned rowmask = (bs < 32 ? ((1u << bs) - 1u) : 0xffffffffu) << base;
    for (;;) {
        if (!ready) {
            if (!loaded && k0 >= e) {
                ready = true;
            } else {
                if (!loaded) {
#pragma unroll
                    for (int q = 0; q < kQ; ++q) {
                        const int k = k0 + q;
                        on[q] = k < e;
                        src[q] = dep + static_cast<std::size_t>(on[q] ? a.cols[k] : 0) * bs;
#pragma unroll
                        for (int j = 0; j < kMaxBlock; ++j) {
                            if (on[q] && j < bs) {
                                co[q][j] = cvt<T>(a.vals[(static_cast<std::size_t>(k) * bs + i) * bs + j]);
                                xb[q][j] = ld_relaxed_bits(src[q] + j);
                            }
                        }
                    }
                    loaded = true;
                }
                bool pending = false;
#pragma unroll
                for (int q = 0; q < kQ; ++q)
#pragma unroll
                    for (int j = 0; j < kMaxBlock; ++j)
                        pending |= on[q] && j < bs && xb[q][j] == Bits<T>::kSentinel;
                if (pending) {
                    if (it >= a.spin_limit) {
                        atomicOr(a.status, kErrTimeout);
                        pending = false;
                    } else if ((it & 1023) == 1023
                               && (*reinterpret_cast<volatile unsigned*>(a.status) & kErrTimeout)) {
                        pending = false;
                    }
                }
                if (!pending) {
#pragma unroll
                    for (int q = 0; q < kQ; ++q) {
                        if (!on[q]) continue;
                        T sum = 0;
#pragma unroll
                        for (int j = 0; j < kMaxBlock; ++j)
                            if (j < bs) sum = add_rn(sum, mul_rn(co[q][j], from_bits(xb[q][j])));
                        acc = sub_rn(acc, sum);
                    }
                    k0 += kQ;
                    loaded = false;
                    if (k0 >= e) ready = true;
                } else {
                    if (it >= 256) __nanosleep(32);
                    ++it;
#pragma unroll
                    for (int q = 0; q < kQ; ++q)
#pragma unroll
                        for (int j = 0; j < kMaxBlock; ++j)
                            if (on[q] && j < bs && xb[q][j] == Bits<T>::kSentinel)
                                xb[q][j] = ld_relaxed_bits(src[q] + j);
                }
            }
        }
        if constexpr (!BACK) {
            if (ready && !done) {
                publish(a.work + rb + i, acc);
                done = true;
            }
        } else {
            const unsigned rdy = __ballot_sync(0xffffffffu, ready);
            const bool row_ready = (rdy & rowmask) == rowmask;
            if (__any_sync(0xffffffffu, row_ready && !done)) {
                T x = 0;
#pragma unroll
                for (int j = 0; j < kMaxBlock; ++j) {
                    if (j < bs) {
                        const T wj = __shfl_sync(0xffffffffu, acc, (base + j) & 31);
                        x = add_rn(x, mul_rn(dinv[j], wj));
                    }
                }
                if (row_ready && !done) {
                    publish(a.out + rb + i, x);
                    done = true;
                }
            }
        }
        if (!__any_sync(0xffffffffu, !done)) break;
    }
}

// In-place Gauss-Jordan inverse of a bs x bs block with partial pivoting
// (the dense-block ILU's diagonal); returns false on a zero pivot.
__device__ bool block_inverse(int bs, const double* a, double* inv)
{
    double m[kMaxBlock * kMaxBlock], r[kMaxBlock * kMaxBlock];
    for (int i = 0; i < bs * bs; ++i) { m[i] = a[i]; r[i] = 0.0; }
    for (int i = 0; i < bs; ++i) r[i * bs + i] = 1.0;
    for (int c = 0; c < bs; ++c) {
        int p = c;
        for (int i = c + 1; i < bs; ++i)
            if (fabs(m[i * bs + c]) > fabs(m[p * bs + c])) p = i;
        if (!isfinite(m[p * bs + c]) || fabs(m[p * bs + c]) <= 64.0 * DBL_EPSILON) return false;
        if (p != c) {
            for (int j = 0; j < bs; ++j) {
                double t = m[c * bs + j]; m[c * bs + j] = m[p * bs + j]; m[p * bs + j] = t;
                t = r[c * bs + j]; r[c * bs + j] = r[p * bs + j]; r[p * bs + j] = t;
            }
        }
        const double piv = m[c * bs + c];
        for (int j = 0; j < bs; ++j) {
            m[c * bs + j] = div_rn(m[c * bs + j], piv);
            r[c * bs + j] = div_rn(r[c * bs + j], piv);
        }
        for (int i = 0; i < bs; ++i) {
            if (i == c) continue;
            const double f = m[i * bs + c];
            for (int j = 0; j < bs; ++j) {
                m[i * bs + j] = sub_rn(m[i * bs + j], mul_rn(f, m[c * bs + j]));
                r[i * bs + j] = sub_rn(r[i * bs + j], mul_rn(f, r[c * bs + j]));
            }
        }
    }
    for (int i = 0; i < bs * bs; ++i) inv[i] = r[i];
    return true;
}

template<class T, class F, int MODE>
__device__ __forceinline__ T row_body(const SweepArgs<T, F>& a, int row, int c0, int cstep)
{
    const int bs = a.bs;
    const std::size_t rb = static_cast<std::size_t>(row) * bs;
    // Row-local operands are loaded before the dependency wait so their
    // latency is not added to the level-to-level critical path.
    if constexpr (MODE == kIluForward) {          // in -> work (unit lower solve)
        const int b = a.rowptr[row], d = a.diagpos[row];
        for (int c = c0; c < bs; c += cstep) {
            const T own = a.in[rb + c];
            publish(a.work + rb + c, eliminate<T, F, 0, false, true>(own, a, a.work, b, d, row, c));
        }
    } else if constexpr (MODE == kIluBackward) {  // work -> out (upper solve, times the inverse diagonal)
        const int d = a.diagpos[row], end = a.rowptr[row + 1];
        for (int c = c0; c < bs; c += cstep) {
            const T own = a.work[rb + c], inv = cvt<T>(a.inv[rb + c]);
            publish(a.out + rb + c, mul_rn(eliminate<T, F, 0, false, true>(own, a, a.out, d + 1, end, row, c), inv));
        }
    } else if constexpr (MODE == kSsorForward) {  // in -> work
        const int b = a.rowptr[row], end = a.rowptr[row + 1];
        for (int c = c0; c < bs; c += cstep) {
            const T own = a.in[rb + c], dg = a.diag[rb + c];
            publish(a.work + rb + c, div_rn(eliminate<T, F, 1, true, true>(own, a, a.work, b, end, row, c), dg));
        }
    } else if constexpr (MODE == kSsorBackward) { // work -> out
        const int b = a.rowptr[row], end = a.rowptr[row + 1];
        for (int c = c0; c < bs; c += cstep) {
            const T dg = a.diag[rb + c];
            const T z0 = mul_rn(dg, a.work[rb + c]);
            publish(a.out + rb + c, div_rn(eliminate<T, F, 2, true, true>(z0, a, a.out, b, end, row, c), dg));
        }
    } else if constexpr (MODE == kBlockForward) {  // in -> work, block row c0 of the row
        const int b = a.rowptr[row], d = a.diagpos[row];
        const T own = a.in[rb + c0];
        publish(a.work + rb + c0, block_eliminate<T, F>(own, a, a.work, b, d, c0));
    } else if constexpr (MODE == kBlockBackward) { // returns w = y - sum U x; the caller applies Dinv
        const int d = a.diagpos[row], end = a.rowptr[row + 1];
        const T own = a.work[rb + c0];
        return block_eliminate<T, F>(own, a, a.out, d + 1, end, c0);
    } else if constexpr (MODE == kBlockFactor) {   // block IKJ of one row; lane = block row c0
        const int b = a.rowptr[row], d = a.diagpos[row];
        wait_deps<0>(a.flags, a.cols, b, d, row, a.owned, a.epoch, a.status);
        const int i = c0;
        const std::size_t b2 = static_cast<std::size_t>(bs) * bs;
        for (int l = b; l < d; ++l) {
            const int p = a.cols[l];
            T arow[kMaxBlock], lrow[kMaxBlock];
            for (int j = 0; j < bs; ++j) arow[j] = a.vals[l * b2 + i * bs + j];
            const F* dp = a.inv + static_cast<std::size_t>(p) * b2;
            for (int k = 0; k < bs; ++k) {
                T sum = 0;
                for (int j = 0; j < bs; ++j) sum = add_rn(sum, mul_rn(arow[j], __ldcg(dp + j * bs + k)));
                lrow[k] = sum;
            }
            for (int k = 0; k < bs; ++k) a.vals[l * b2 + i * bs + k] = lrow[k];
            for (int u = a.upd_start[l]; u < a.upd_start[l + 1]; ++u) {
                const F* ub = a.vals + static_cast<std::size_t>(a.upd_upper[u]) * b2;
                F* tb = a.vals + static_cast<std::size_t>(a.upd_target[u]) * b2 + i * bs;
                for (int k = 0; k < bs; ++k) {
                    T sum = 0;
                    for (int j = 0; j < bs; ++j) sum = add_rn(sum, mul_rn(lrow[j], __ldcg(ub + j * bs + k)));
                    tb[k] = sub_rn(tb[k], sum);
                }
            }
        }
    } else if constexpr (MODE == kIluFactor) {  // IKJ elimination of one row (preconditioner.hpp:442-469)
        const int b = a.rowptr[row], d = a.diagpos[row];
        wait_deps<0>(a.flags, a.cols, b, d, row, a.owned, a.epoch, a.status);
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
    return T(0);
}

// LANE: applies with block size <= 32 through apply_lane / block_apply_lane
// (early publication); otherwise row_body.
template<class T, class F, int MODE, bool LANE = false>
__global__ void __launch_bounds__(kThreads) k_sweep(SweepArgs<T, F> a)
{
    const int lane = threadIdx.x & 31;
    const int bs = a.bs;
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
    unsigned long long t = 0;
    if (lane == 0) t = atomicAdd(a.ticket, 1ull) - a.base;
    for (;;) {
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= static_cast<unsigned long long>(a.tasks)) break;
        // Reserve the next task now; the atomic's latency overlaps this task.
        unsigned long long next = 0;
        if (lane == 0) next = atomicAdd(a.ticket, 1ull) - a.base;
        const int s = a.task_start[t], nrows = a.task_start[t + 1] - s;
        const int row = rl < nrows ? a.order[s + rl] : -1;
        T w = 0;
        if constexpr (LANE && (MODE == kBlockForward || MODE == kBlockBackward))
            block_apply_lane<T, F, MODE == kBlockBackward>(a, row, c0, rl);
        else if constexpr (LANE) apply_lane<T, F, MODE>(a, row, s + rl, c0);
        else if (row >= 0) w = row_body<T, F, MODE>(a, row, c0, cstep);
        if constexpr (MODE == kBlockBackward && !LANE) {
            // x_r[i] = sum_j Dinv_r[i][j] w_j: the row's w_j live in the
            // lanes rl*bs + j of this warp.
            __syncwarp();
            const int base = (rl * bs) & 31;
            T x = 0;
            for (int j = 0; j < bs; ++j) {
                const T wj = __shfl_sync(0xffffffffu, w, (base + j) & 31);
                if (row >= 0)
                    x = add_rn(x, mul_rn(cvt<T>(a.inv[static_cast<std::size_t>(row) * bs * bs + c0 * bs + j]), wj));
            }
            if (row >= 0) publish(a.out + static_cast<std::size_t>(row) * bs + c0, x);
        }
        if constexpr (MODE == kBlockFactor) {
            // The row's diagonal block is final: invert it (one lane per row).
            __syncwarp();
            if (row >= 0 && c0 == 0) {
                const std::size_t b2 = static_cast<std::size_t>(bs) * bs;
                double blk[kMaxBlock * kMaxBlock], inv[kMaxBlock * kMaxBlock];
                const F* dblk = a.vals + static_cast<std::size_t>(a.diagpos[row]) * b2;
                for (std::size_t q = 0; q < b2; ++q) blk[q] = static_cast<double>(dblk[q]);
                if (!block_inverse(bs, blk, inv)) atomicOr(a.status, kErrZeroPivot);
                for (std::size_t q = 0; q < b2; ++q) a.inv[static_cast<std::size_t>(row) * b2 + q] = static_cast<F>(inv[q]);
            }
        }
        if constexpr (is_factor(MODE)) {
            __syncwarp();
            if (lane < nrows) {
                __threadfence();
                st_release(a.flags + a.order[s + lane], a.epoch);
            }
        }
        t = next;
    }
}

// Warps per sweep launch: enough to hold a few levels' worth of tasks in
// flight.  More warps only add polling traffic on the dependency flags while
// the sweep is bound by its level-to-level latency.
int sweep_warps(const Context& c, const Sweep& s)
{
    const char* env = std::getenv("OWTK_SWEEP_WARPS_PER_LEVEL");
    const double factor = env ? std::atof(env) : 16.0;
    const double per_level = s.depth > 0 ? static_cast<double>(s.tasks) / s.depth : s.tasks;
    long long warps = factor > 0 ? static_cast<long long>(std::ceil(factor * per_level)) : s.tasks;
    const long long cap = static_cast<long long>(c.sm_count) * 64;
    if (warps < 32) warps = 32;
    if (warps > cap) warps = cap;
    if (warps > s.tasks) warps = s.tasks;
    return static_cast<int>(warps);
}

template<class T, class F, int MODE>
void launch(Context& c, Preconditioner& p, Sweep& s, SweepArgs<T, F>& a)
{
    if (s.tasks == 0) return;
    if (is_factor(MODE) && ++p.epoch == 0xffffffffu) {
        OWTK_CUDA(cudaMemsetAsync(p.flags.ptr, 0, p.owned * sizeof(unsigned), c.stream));
        p.epoch = 1;
    }
    const int warps_per_block = kThreads / 32;
    const int blocks = (sweep_warps(c, s) + warps_per_block - 1) / warps_per_block;
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
    if (a.spin_limit <= 0) a.spin_limit = kSpinLimit;
    bool lane = false;
    if constexpr (is_lane_apply(MODE)) {
        if (p.bs <= 32) {
            k_sweep<T, F, MODE, true><<<blocks, kThreads, 0, c.stream>>>(a);
            lane = true;
        }
    }
    if (!lane) k_sweep<T, F, MODE><<<blocks, kThreads, 0, c.stream>>>(a);
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
    launch<T, T, kIluFactor>(c, p, p.lower, a);
    for (Sweep* s : {&p.lower, &p.upper})
        if (s->packed)
            gather_values<T>(c, s->pentries, p.bs, s->psrc.as<std::int64_t>(), p.d_fvalues.as<T>(), s->pvals.as<T>());
}

template<class T> void fill_sentinel(Context& c, std::size_t n, T* x)
{
    if (n == 0) return;
    k_fill_sentinel<T><<<static_cast<unsigned>((n + 255) / 256), 256, 0, c.stream>>>(n, x);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

// preconditioner.hpp:320-363.  The forward result goes to the PC's work
// vector, so in == out is allowed: `in` is fully read before `out` is reset.
template<class T> void ilu_apply(Context& c, Preconditioner& p, const T* in, T* out)
{
    if (chain_ilu_apply<T>(c, p, in, out)) return;
    if (lockstep_ilu_apply<T>(c, p, in, out)) return;
    if (cluster_ilu_apply<T>(c, p, in, out)) return;
    SweepArgs<T> a{};
    a.rowptr = p.d_frowptr.as<int>();
    a.cols = p.d_fcols.as<int>();
    a.diagpos = p.d_fdiagpos.as<int>();
    a.vals = p.d_fvalues.as<T>();
    a.inv = p.inv_diag.as<T>();
    a.in = in;
    a.out = out;
    a.work = p.work.as<T>();
    const std::size_t n = p.owned * p.bs;
    const bool packed = p.lower.packed && p.upper.packed;
    if (packed) {
        a.seg = p.lower.seg.as<int>();
        a.cols = p.lower.pcols.as<int>();
        a.vals = p.lower.pvals.as<T>();
    }
    fill_sentinel<T>(c, n, a.work);
    launch<T, T, kIluForward>(c, p, p.lower, a);
    if (packed) {
        a.seg = p.upper.seg.as<int>();
        a.cols = p.upper.pcols.as<int>();
        a.vals = p.upper.pvals.as<T>();
    }
    fill_sentinel<T>(c, n, out);
    launch<T, T, kIluBackward>(c, p, p.upper, a);
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
    const std::size_t n = p.owned * p.bs;
    fill_sentinel<T>(c, n, a.work);
    launch<T, T, kSsorForward>(c, p, p.lower, a);
    fill_sentinel<T>(c, n, out);
    launch<T, T, kSsorBackward>(c, p, p.upper, a);
    const T omega = static_cast<T>(p.parameter);
    if (omega != T(1)) scale<T>(c, p.owned * p.bs, omega * (T(2) - omega), out);
}

// ILU(k) with low-precision factor storage F (float or bf16) and FP32
// vectors / arithmetic: the inner preconditioner of mixed-precision solves.
template<class F> void ilu_apply_lp(Context& c, Preconditioner& p, const float* in, float* out)
{
    SweepArgs<float, F> a{};
    a.rowptr = p.d_frowptr.as<int>();
    a.cols = p.d_fcols.as<int>();
    a.diagpos = p.d_fdiagpos.as<int>();
    a.vals = p.lp_vals.as<F>();
    a.inv = p.lp_inv.as<F>();
    a.in = in;
    a.out = out;
    a.work = p.work32.as<float>();
    const std::size_t n = p.owned * p.bs;
    fill_sentinel<float>(c, n, a.work);
    if (p.block) {
        launch<float, F, kBlockForward>(c, p, p.lower, a);
        fill_sentinel<float>(c, n, out);
        launch<float, F, kBlockBackward>(c, p, p.upper, a);
    } else {
        launch<float, F, kIluForward>(c, p, p.lower, a);
        fill_sentinel<float>(c, n, out);
        launch<float, F, kIluBackward>(c, p, p.upper, a);
    }
}

// Dense-block ILU(0): FP64 factorisation (bs <= 4) reusing the symbolic
// pattern, update lists and level sets of the component-diagonal ILU.
void block_ilu_factorize(Context& c, Preconditioner& p, const double* matrix_values)
{
    gather_values<double>(c, p.f_cols.size(), p.bs * p.bs, p.d_fsource.as<std::int64_t>(), matrix_values,
                          p.d_fvalues.as<double>());
    SweepArgs<double> a{};
    a.rowptr = p.d_frowptr.as<int>();
    a.cols = p.d_fcols.as<int>();
    a.diagpos = p.d_fdiagpos.as<int>();
    a.vals = p.d_fvalues.as<double>();
    a.inv = p.inv_diag.as<double>();
    a.upd_start = p.d_upd_start.as<int>();
    a.upd_target = p.d_upd_target.as<int>();
    a.upd_upper = p.d_upd_upper.as<int>();
    launch<double, double, kBlockFactor>(c, p, p.lower, a);
}

void block_ilu_apply(Context& c, Preconditioner& p, const double* in, double* out)
{
    SweepArgs<double> a{};
    a.rowptr = p.d_frowptr.as<int>();
    a.cols = p.d_fcols.as<int>();
    a.diagpos = p.d_fdiagpos.as<int>();
    a.vals = p.d_fvalues.as<double>();
    a.inv = p.inv_diag.as<double>();
    a.in = in;
    a.out = out;
    a.work = p.work.as<double>();
    const std::size_t n = p.owned * p.bs;
    fill_sentinel<double>(c, n, a.work);
    launch<double, double, kBlockForward>(c, p, p.lower, a);
    fill_sentinel<double>(c, n, out);
    launch<double, double, kBlockBackward>(c, p, p.upper, a);
}

template void ilu_apply_lp<float>(Context&, Preconditioner&, const float*, float*);
template void ilu_apply_lp<__nv_bfloat16>(Context&, Preconditioner&, const float*, float*);
template void ilu_factorize<double>(Context&, Preconditioner&, const double*);
template void ilu_factorize<float>(Context&, Preconditioner&, const float*);
// A two-row ILU forward apply whose schedule holds row 1 only: row 1 waits
// for row 0, which nothing computes, so its wait runs out after
// `spin_limit` polls, sets the timeout bit and the launch ends.  Lets a test
// check the bounded wait and the host's OWTK_ERR_TIMEOUT without any fault.
void debug_unpublished_dependency(Context& c, int spin_limit)
{
    const std::vector<int> rowptr{0, 1, 3}, cols{0, 0, 1}, diagpos{0, 2}, order{1}, task_start{0, 1};
    const std::vector<double> vals{2.0, -1.0, 2.0}, in{1.0, 1.0}, inv{0.5, 0.5};
    DeviceBuffer d_rp = upload(c.stream, rowptr), d_ci = upload(c.stream, cols), d_dp = upload(c.stream, diagpos),
                 d_order = upload(c.stream, order), d_ts = upload(c.stream, task_start),
                 d_v = upload(c.stream, vals), d_in = upload(c.stream, in), d_inv = upload(c.stream, inv);
    DeviceBuffer work(2 * sizeof(double) + 16), ticket(sizeof(unsigned long long));
    OWTK_CUDA(cudaMemsetAsync(ticket.ptr, 0, sizeof(unsigned long long), c.stream));
    k_fill_sentinel<double><<<1, 32, 0, c.stream>>>(2, work.as<double>());
    SweepArgs<double> a{};
    a.order = d_order.as<int>();
    a.task_start = d_ts.as<int>();
    a.tasks = 1;
    a.rowptr = d_rp.as<int>();
    a.cols = d_ci.as<int>();
    a.diagpos = d_dp.as<int>();
    a.vals = d_v.as<double>();
    a.inv = d_inv.as<double>();
    a.in = d_in.as<double>();
    a.out = work.as<double>();
    a.work = work.as<double>();
    a.owned = 2;
    a.bs = 1;
    a.ticket = ticket.as<unsigned long long>();
    a.status = c.status.as<unsigned>();
    a.spin_limit = spin_limit > 0 ? spin_limit : kSpinLimit;
    k_sweep<double, double, kIluForward, true><<<1, kThreads, 0, c.stream>>>(a);
    OWTK_CUDA(cudaGetLastError());
    c.launched(2);
    c.sync();
}

template void ilu_apply<double>(Context&, Preconditioner&, const double*, double*);
template void ilu_apply<float>(Context&, Preconditioner&, const float*, float*);
template void ssor_apply<double>(Context&, Preconditioner&, const double*, double*);
template void ssor_apply<float>(Context&, Preconditioner&, const float*, float*);

}  // namespace kern
}  // namespace owtk
