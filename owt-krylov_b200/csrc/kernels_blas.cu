// Vector updates and reductions of the Krylov solvers (sm_100a).
//
// Element-wise kernels: each thread owns kIlp elements spaced one CTA apart,
// loads them all before computing (independent 8-byte loads, fully coalesced
// per warp), and evaluates the reference expression with the same rounding
// sequence (device_common.cuh).
//
// Reductions: fixed-size first stage (one partial per CTA and dot), then the
// last CTA to finish (atomic ticket) combines the partials in a fixed order.
// Results are deterministic run to run and land both in device memory (for
// kernels that consume them) and in mapped pinned memory (for the host).

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <mutex>
#include <utility>
#include <vector>

#include <cuda_bf16.h>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;
constexpr int kIlp = 4;
constexpr int kPerBlock = kThreads * kIlp;

inline unsigned ew_blocks(std::size_t n)
{
    return static_cast<unsigned>((n + kPerBlock - 1) / kPerBlock);
}

#define EW_PROLOGUE                                                            \
    const std::size_t i0 = static_cast<std::size_t>(blockIdx.x) * kPerBlock   \
        + threadIdx.x;

template<class T>
__global__ void __launch_bounds__(kThreads) k_fill(std::size_t n, T v, T* __restrict__ x)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) x[i] = v;
    }
}

template<class T>
__global__ void __launch_bounds__(kThreads) k_copy(std::size_t n, const T* __restrict__ x, T* __restrict__ y)
{
    EW_PROLOGUE
    T a[kIlp];
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) a[k] = x[i];
    }
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) y[i] = a[k];
    }
}

// y[i] += alpha * x[i]   (simd.hpp:533-535 scalar form)
template<class T>
__global__ void __launch_bounds__(kThreads) k_axpy(std::size_t n, T alpha, const T* __restrict__ x, T* __restrict__ y)
{
    EW_PROLOGUE
    T a[kIlp], b[kIlp];
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) { a[k] = x[i]; b[k] = y[i]; }
    }
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) y[i] = add_rn(b[k], mul_rn(alpha, a[k]));
    }
}

template<class T>
__global__ void __launch_bounds__(kThreads) k_scale(std::size_t n, T alpha, T* __restrict__ x)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) x[i] = mul_rn(x[i], alpha);
    }
}

// out = a*x + b*y   (core.hpp:598-600)
template<class T>
__global__ void __launch_bounds__(kThreads) k_lincomb(std::size_t n, T a, const T* __restrict__ x, T b,
                                                      const T* __restrict__ y, T* __restrict__ out)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) out[i] = add_rn(mul_rn(a, x[i]), mul_rn(b, y[i]));
    }
}

// out = b - a   (krylov_solvers.hpp:71-73)
template<class T>
__global__ void __launch_bounds__(kThreads) k_sub(std::size_t n, const T* __restrict__ b, const T* __restrict__ a,
                                                  T* __restrict__ out)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) out[i] = sub_rn(b[i], a[i]);
    }
}

// out = x / s   (krylov_solvers.hpp:256-258)
template<class T>
__global__ void __launch_bounds__(kThreads) k_divide(std::size_t n, const T* __restrict__ x, T s, T* __restrict__ out)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) out[i] = div_rn(x[i], s);
    }
}

// p = r + beta*(p - omega*v)   (krylov_solvers.hpp:629-632)
template<class T>
__global__ void __launch_bounds__(kThreads) k_bicg_p(std::size_t n, const T* __restrict__ r, T beta, T omega,
                                                     const T* __restrict__ v, T* __restrict__ p)
{
    EW_PROLOGUE
    T rr[kIlp], pp[kIlp], vv[kIlp];
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) { rr[k] = r[i]; pp[k] = p[i]; vv[k] = v[i]; }
    }
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) p[i] = add_rn(rr[k], mul_rn(beta, sub_rn(pp[k], mul_rn(omega, vv[k]))));
    }
}

// x += alpha*ph; x += omega*sh; r = s - omega*t   (krylov_solvers.hpp:703-708)
template<class T>
__global__ void __launch_bounds__(kThreads) k_bicg_xr(std::size_t n, T alpha, const T* __restrict__ ph, T omega,
                                                      const T* __restrict__ sh, const T* __restrict__ s,
                                                      const T* __restrict__ t, T* __restrict__ x,
                                                      T* __restrict__ r)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) {
            const T xv = add_rn(add_rn(x[i], mul_rn(alpha, ph[i])), mul_rn(omega, sh[i]));
            const T rv = sub_rn(s[i], mul_rn(omega, t[i]));
            x[i] = xv;
            r[i] = rv;
        }
    }
}

// pipelined_bicgstab.hpp:436-445
template<class T>
__global__ void __launch_bounds__(kThreads) k_ch_psz(std::size_t n, T beta, T omega, const T* __restrict__ r2,
                                                     const T* __restrict__ w, const T* __restrict__ w2,
                                                     const T* __restrict__ t, const T* __restrict__ z2,
                                                     const T* __restrict__ v, T* __restrict__ p2,
                                                     T* __restrict__ s, T* __restrict__ s2, T* __restrict__ z)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) {
            p2[i] = add_rn(r2[i], mul_rn(beta, sub_rn(p2[i], mul_rn(omega, s2[i]))));
            s[i] = add_rn(w[i], mul_rn(beta, sub_rn(s[i], mul_rn(omega, z[i]))));
            s2[i] = add_rn(w2[i], mul_rn(beta, sub_rn(s2[i], mul_rn(omega, z2[i]))));
            z[i] = add_rn(t[i], mul_rn(beta, sub_rn(z[i], mul_rn(omega, v[i]))));
        }
    }
}

// pipelined_bicgstab.hpp:447-451
template<class T>
__global__ void __launch_bounds__(kThreads) k_ch_qy(std::size_t n, T alpha, const T* __restrict__ r,
                                                    const T* __restrict__ s, const T* __restrict__ r2,
                                                    const T* __restrict__ s2, const T* __restrict__ w,
                                                    const T* __restrict__ z, T* __restrict__ q,
                                                    T* __restrict__ q2, T* __restrict__ y)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) {
            q[i] = sub_rn(r[i], mul_rn(alpha, s[i]));
            q2[i] = sub_rn(r2[i], mul_rn(alpha, s2[i]));
            y[i] = sub_rn(w[i], mul_rn(alpha, z[i]));
        }
    }
}

// pipelined_bicgstab.hpp:506-512
template<class T>
__global__ void __launch_bounds__(kThreads) k_ch_rw(std::size_t n, T alpha, T omega, const T* __restrict__ q,
                                                    const T* __restrict__ y, const T* __restrict__ q2,
                                                    const T* __restrict__ w2, const T* __restrict__ z2,
                                                    const T* __restrict__ t, const T* __restrict__ v,
                                                    T* __restrict__ r, T* __restrict__ r2, T* __restrict__ w)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) {
            r[i] = sub_rn(q[i], mul_rn(omega, y[i]));
            r2[i] = sub_rn(q2[i], mul_rn(omega, sub_rn(w2[i], mul_rn(alpha, z2[i]))));
            w[i] = sub_rn(y[i], mul_rn(omega, sub_rn(t[i], mul_rn(alpha, v[i]))));
        }
    }
}

// out = x * s   (copy_owned + scale, krylov_solvers.hpp:355-356)
template<class T>
__global__ void __launch_bounds__(kThreads) k_scaled_copy(std::size_t n, const T* __restrict__ x, T s,
                                                          T* __restrict__ out)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) out[i] = mul_rn(x[i], s);
    }
}

template<class T>
__global__ void __launch_bounds__(kThreads) k_jacobi(std::size_t n, const T* __restrict__ inv,
                                                     const T* __restrict__ in, T* __restrict__ out)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) out[i] = mul_rn(inv[i], in[i]);
    }
}

// inv = 1/d with the singular-diagonal check (preconditioner.hpp:62-69).
template<class T>
__global__ void __launch_bounds__(kThreads) k_reciprocal(std::size_t n, const T* __restrict__ d, T minimum,
                                                         T* __restrict__ inv, unsigned* status)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) {
            const T v = d[i];
            if (!isfinite(v) || fabs(v) <= minimum) atomicOr(status, kErrSingularDiagonal);
            inv[i] = div_rn(T(1), v);
        }
    }
}

// Element-wise precision conversion (factor storage and mixed-precision
// vector hand-off).
__device__ __forceinline__ void cvt_store(float* d, double v) { *d = __double2float_rn(v); }
__device__ __forceinline__ void cvt_store(double* d, float v) { *d = static_cast<double>(v); }
__device__ __forceinline__ void cvt_store(__nv_bfloat16* d, double v) { *d = __double2bfloat16(v); }

template<class To, class From>
__global__ void __launch_bounds__(kThreads) k_convert(std::size_t n, const From* __restrict__ src,
                                                      To* __restrict__ dst)
{
    EW_PROLOGUE
#pragma unroll
    for (int k = 0; k < kIlp; ++k) {
        const std::size_t i = i0 + static_cast<std::size_t>(k) * kThreads;
        if (i < n) cvt_store(dst + i, src[i]);
    }
}

// --------------------------------------------------------------- pointer packs
struct PtrPack {
    const void* p[kMaxBatch];
};

// w -= sum_j h_j V_j in the reference's axpy order (krylov_solvers.hpp:286-290).
template<class T>
__global__ void __launch_bounds__(kThreads) k_cgs_update(std::size_t n, int k, PtrPack basis,
                                                         const double* __restrict__ h, T* __restrict__ w)
{
    __shared__ const T* sp[kMaxBatch];
    __shared__ T sh[kMaxBatch];
    for (int j = threadIdx.x; j < k; j += kThreads) {
        sp[j] = static_cast<const T*>(basis.p[j]);
        sh[j] = -static_cast<T>(h[j]);
    }
    __syncthreads();
    EW_PROLOGUE
#pragma unroll
    for (int u = 0; u < kIlp; ++u) {
        const std::size_t i = i0 + static_cast<std::size_t>(u) * kThreads;
        if (i >= n) continue;
        T wv = w[i];
        for (int j = 0; j < k; ++j) wv = add_rn(wv, mul_rn(sh[j], sp[j][i]));
        w[i] = wv;
    }
}

// The last Gram-Schmidt pass fused with the normalisation: out = (w - V h) * s,
// with the sum of k_cgs_update and the product of k_scaled_copy in the same
// order, so the bits equal those two launches; w itself is left as it was.
template<class T>
__global__ void __launch_bounds__(kThreads) k_cgs_update_scale(std::size_t n, int k, PtrPack basis,
                                                               const double* __restrict__ h,
                                                               const T* __restrict__ w, T s, T* __restrict__ out)
{
    __shared__ const T* sp[kMaxBatch];
    __shared__ T sh[kMaxBatch];
    for (int j = threadIdx.x; j < k; j += kThreads) {
        sp[j] = static_cast<const T*>(basis.p[j]);
        sh[j] = -static_cast<T>(h[j]);
    }
    __syncthreads();
    EW_PROLOGUE
#pragma unroll
    for (int u = 0; u < kIlp; ++u) {
        const std::size_t i = i0 + static_cast<std::size_t>(u) * kThreads;
        if (i >= n) continue;
        T wv = w[i];
        for (int j = 0; j < k; ++j) wv = add_rn(wv, mul_rn(sh[j], sp[j][i]));
        out[i] = mul_rn(wv, s);
    }
}

// Neumaier-compensated correction sum (krylov_solvers.hpp:24-40).
template<class T>
__global__ void __launch_bounds__(kThreads) k_gmres_update(std::size_t n, int k, PtrPack dirs,
                                                           const double* __restrict__ coef,
                                                           const T* base, T* out)
{
    __shared__ const T* sp[kMaxBatch];
    __shared__ T sc[kMaxBatch];
    for (int j = threadIdx.x; j < k; j += kThreads) {
        sp[j] = static_cast<const T*>(dirs.p[j]);
        sc[j] = static_cast<T>(coef[j]);
    }
    __syncthreads();
    EW_PROLOGUE
#pragma unroll
    for (int u = 0; u < kIlp; ++u) {
        const std::size_t i = i0 + static_cast<std::size_t>(u) * kThreads;
        if (i >= n) continue;
        T sum = 0, comp = 0;
        for (int j = 0; j < k; ++j) {
            const T term = mul_rn(sc[j], sp[j][i]);
            const T upd = add_rn(sum, term);
            comp = add_rn(comp, fabs(sum) >= fabs(term) ? add_rn(sub_rn(sum, upd), term)
                                                        : add_rn(sub_rn(term, upd), sum));
            sum = upd;
        }
        out[i] = add_rn(base[i], add_rn(sum, comp));
    }
}

// --------------------------------------------------------------- reductions
unsigned reduce_blocks(const Context& c, std::size_t n)
{
    const std::size_t want = (n + kThreads * 8 - 1) / (kThreads * 8);
    std::size_t cap = static_cast<std::size_t>(c.sm_count) * 4;
    if (cap > static_cast<std::size_t>(kReduceBlocks)) cap = kReduceBlocks;
    return static_cast<unsigned>(want < 1 ? 1 : (want > cap ? cap : want));
}

// CTAs of `kernel` that fit on the device at once (one wave), at most `want`:
// the Gram-Schmidt kernels hold many basis streams in registers, so fewer
// CTAs fit per SM than the element-wise kernels and a grid sized for those
// would run in several waves.
template<class K>
unsigned resident_blocks(const Context& c, K kernel, unsigned want)
{
    static std::mutex mutex;
    static std::vector<std::pair<const void*, int>> cache;   // kernel -> resident CTAs per SM
    const void* key = reinterpret_cast<const void*>(kernel);
    int per_sm = 0;
    {
        std::lock_guard<std::mutex> lock(mutex);
        for (const auto& [k, v] : cache)
            if (k == key) per_sm = v;
        if (per_sm == 0) {
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, kThreads, 0) != cudaSuccess
                || per_sm < 1) {
                cudaGetLastError();
                return want;
            }
            cache.emplace_back(key, per_sm);
        }
    }
    const unsigned cap = static_cast<unsigned>(per_sm) * static_cast<unsigned>(c.sm_count);
    return want < cap ? want : cap;
}

// Reduce G per-thread accumulators across the CTA; thread j < G writes the
// CTA's partial for accumulator j.
template<int G>
__device__ __forceinline__ void block_partials(const double (&acc)[G], int count, double* partials,
                                               int slot0)
{
    __shared__ double red[G][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < G; ++j) {
        const double v = warp_sum(acc[j]);
        if (lane == 0) red[j][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x < count) {
        double s = 0;
#pragma unroll
        for (int w = 0; w < kThreads / 32; ++w) s += red[threadIdx.x][w];
        partials[static_cast<std::size_t>(slot0 + threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
    __syncthreads();
}

// Last CTA: sum each accumulator's partials over CTAs in a fixed order.
__device__ __forceinline__ bool last_block(unsigned* ticket)
{
    __shared__ bool is_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) is_last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    return is_last;
}

__device__ __forceinline__ void combine(int count, const double* partials, double* out_dev,
                                        double* out_host)
{
    __threadfence();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int j = warp; j < count; j += kThreads / 32) {
        double s = 0;
        for (unsigned b = lane; b < gridDim.x; b += 32)
            s += __ldcg(partials + static_cast<std::size_t>(j) * gridDim.x + b);
        s = warp_sum(s);
        if (lane == 0) {
            out_dev[j] = s;
            out_host[j] = s;
        }
    }
}

// k dots a_j . b_j, FP64 accumulation (float inputs are widened as the
// reference's SerialReduction<float> does, reduction.hpp:123-133).  G dots are
// accumulated per pass; U elements per thread are loaded before use, so each
// thread keeps 2*G*U independent loads in flight.
template<class T, int G, int U>
__global__ void __launch_bounds__(kThreads) k_multidot(std::size_t n, int k, PtrPack a, PtrPack b,
                                                       double* partials, unsigned* ticket,
                                                       double* out_dev, double* out_host)
{
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * kThreads;
    __shared__ const T* sa[kMaxBatch];
    __shared__ const T* sb[kMaxBatch];
    for (int j = threadIdx.x; j < k; j += kThreads) {
        sa[j] = static_cast<const T*>(a.p[j]);
        sb[j] = static_cast<const T*>(b.p[j]);
    }
    __syncthreads();
    for (int g0 = 0; g0 < k; g0 += G) {
        double acc[G];
        const T* pa[G];
        const T* pb[G];
#pragma unroll
        for (int j = 0; j < G; ++j) {
            acc[j] = 0;
            pa[j] = g0 + j < k ? sa[g0 + j] : nullptr;
            pb[j] = g0 + j < k ? sb[g0 + j] : nullptr;
        }
        for (std::size_t i = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += U * stride) {
            T va[U][G], vb[U][G];
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const std::size_t idx = i + u * stride;
#pragma unroll
                for (int j = 0; j < G; ++j) {
                    const bool on = g0 + j < k && idx < n;
                    va[u][j] = on ? pa[j][idx] : T(0);
                    vb[u][j] = on ? pb[j][idx] : T(0);
                }
            }
#pragma unroll
            for (int u = 0; u < U; ++u)
#pragma unroll
                for (int j = 0; j < G; ++j)
                    acc[j] += static_cast<double>(va[u][j]) * static_cast<double>(vb[u][j]);
        }
        block_partials<G>(acc, k - g0 < G ? k - g0 : G, partials, g0);
    }
    if (last_block(ticket)) {
        combine(k, partials, out_dev, out_host);
        if (threadIdx.x == 0) *ticket = 0;
    }
}

// Dots of x with every V_j (j < k) and x.x in one pass: x and each V_j are
// read once per element.  The grid, the per-thread element order and the CTA
// and over-CTA sums follow k_multidot on the pairs (x, V_j) and (x, x); the
// results agree with it to FP64 rounding (a few ulps, measured), not always
// bit for bit, so a caller keeps to one of the two kernels for a given dot.
// Gram-Schmidt kernels: three CTAs per SM, one element per thread and pass
// (2M-vertex mesh, FGMRES(30)+Jacobi 14 iterations: 6.44 ms against 6.60 ms
// for two CTAs with two elements and 6.80 ms for four with one).
constexpr int kGsBlocks = 3;
template<class T, int G>
__global__ void __launch_bounds__(kThreads, kGsBlocks) k_basis_dots(std::size_t n, int k, PtrPack basis,
                                                         const T* __restrict__ x, double* partials, unsigned* ticket,
                                                         double* out_dev, double* out_host)
{
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * kThreads;
    double acc[G];
#pragma unroll
    for (int j = 0; j < G; ++j) acc[j] = 0;
    double self = 0.0;
    const T* const* bp = reinterpret_cast<const T* const*>(basis.p);
    // U elements per pass, all loads first (the basis is read-only here).
    constexpr int U = 1;
    for (std::size_t i0 = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i0 < n; i0 += U * stride) {
        T xv[U], vj[U][G - 1];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const std::size_t i = i0 + u * stride;
            const bool in = i < n;
            xv[u] = in ? x[i] : T(0);
#pragma unroll
            for (int j = 0; j < G - 1; ++j) vj[u][j] = (in && j < k) ? __ldg(bp[j] + i) : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (i0 + u * stride >= n) break;
#pragma unroll
            for (int j = 0; j < G - 1; ++j)
                if (j < k) acc[j] += static_cast<double>(xv[u]) * static_cast<double>(vj[u][j]);
            self += static_cast<double>(xv[u]) * static_cast<double>(xv[u]);
        }
    }
    {
        // block_partials<G>, written out so that acc stays in registers.
        __shared__ double red[G][kThreads / 32];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const double v = warp_sum(j == k ? self : acc[j]);
            if (lane == 0) red[j][warp] = v;
        }
        __syncthreads();
        if (threadIdx.x <= k) {
            double t = 0;
#pragma unroll
            for (int w = 0; w < kThreads / 32; ++w) t += red[threadIdx.x][w];
            partials[static_cast<std::size_t>(threadIdx.x) * gridDim.x + blockIdx.x] = t;
        }
        __syncthreads();
    }
    if (last_block(ticket)) {
        combine(k + 1, partials, out_dev, out_host);
        if (threadIdx.x == 0) *ticket = 0;
    }
}

// w -= V h (reference axpy order), then dots of the updated w with every V_j
// and w.w, in one pass over V (second Gram-Schmidt pass, krylov_solvers.hpp:310-322).
template<class T, int G>
__global__ void __launch_bounds__(kThreads, kGsBlocks) k_cgs_update_dot(std::size_t n, int k, PtrPack basis,
                                                             const double* __restrict__ h, T* __restrict__ w,
                                                             double* partials, unsigned* ticket,
                                                             double* out_dev, double* out_host)
{
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * kThreads;
    const T* const* bp = reinterpret_cast<const T* const*>(basis.p);
    double acc[G];
#pragma unroll
    for (int j = 0; j < G; ++j) acc[j] = 0;
    double self = 0.0;
    T coef[G - 1];
#pragma unroll
    for (int j = 0; j < G - 1; ++j) coef[j] = j < k ? -static_cast<T>(h[j]) : T(0);
    // U elements per pass, all loads first; each basis value is read once
    // (read-only path), for the update and for its dot.
    constexpr int U = 1;
    for (std::size_t i0 = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i0 < n; i0 += U * stride) {
        T wv[U], vj[U][G - 1];
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const std::size_t i = i0 + u * stride;
            const bool in = i < n;
            wv[u] = in ? w[i] : T(0);
#pragma unroll
            for (int j = 0; j < G - 1; ++j) vj[u][j] = (in && j < k) ? __ldg(bp[j] + i) : T(0);
        }
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const std::size_t i = i0 + u * stride;
            if (i >= n) break;
            T v = wv[u];
#pragma unroll
            for (int j = 0; j < G - 1; ++j)
                if (j < k) v = add_rn(v, mul_rn(coef[j], vj[u][j]));
            w[i] = v;
            const double wd = static_cast<double>(v);
#pragma unroll
            for (int j = 0; j < G - 1; ++j)
                if (j < k) acc[j] += wd * static_cast<double>(vj[u][j]);
            self += wd * wd;
        }
    }
    {
        // The CTA's partials (block_partials written out: acc stays in registers).
        __shared__ double red[G][kThreads / 32];
        const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const double v = warp_sum(j == k ? self : acc[j]);
            if (lane == 0) red[j][warp] = v;
        }
        __syncthreads();
        if (threadIdx.x <= k) {
            double t = 0;
#pragma unroll
            for (int wi = 0; wi < kThreads / 32; ++wi) t += red[threadIdx.x][wi];
            partials[static_cast<std::size_t>(threadIdx.x) * gridDim.x + blockIdx.x] = t;
        }
        __syncthreads();
    }
    if (last_block(ticket)) {
        combine(k + 1, partials, out_dev, out_host);
        if (threadIdx.x == 0) *ticket = 0;
    }
}

// One-pass scaled 2-norm: each thread keeps (scale, sum of squares relative
// to scale) and rescales when a larger magnitude arrives; pairs combine the
// same way.  NaN anywhere gives NaN and an infinite entry gives infinity,
// as the reference's two-pass scaled norm does (reduction.hpp:64-89).
template<class T>
__global__ void __launch_bounds__(kThreads) k_norm(std::size_t n, const T* __restrict__ x, double* partials,
                                                   unsigned* ticket, double* out_dev, double* out_host)
{
    ScaledSum a{0.0, 0.0, 0};
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * kThreads;
    constexpr int kU = 8;   // loads in flight per thread
    for (std::size_t i = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += kU * stride) {
        double v[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const std::size_t idx = i + u * stride;
            v[u] = idx < n ? static_cast<double>(x[idx]) : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) norm_push(a, v[u]);
    }
    a = norm_warp(a);
    __shared__ ScaledSum red[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = a;
    __syncthreads();
    if (threadIdx.x == 0) {
        ScaledSum s = red[0];
        for (int w = 1; w < kThreads / 32; ++w) s = norm_merge(s, red[w]);
        partials[3 * blockIdx.x + 0] = s.scale;
        partials[3 * blockIdx.x + 1] = s.ssq;
        partials[3 * blockIdx.x + 2] = s.nan;
    }
    if (last_block(ticket)) {
        __threadfence();
        // Every thread merges a strided share of the CTA partials, then the
        // CTA merges the threads' results (fixed order: deterministic).
        ScaledSum t{0.0, 0.0, 0};
        for (unsigned b = threadIdx.x; b < gridDim.x; b += kThreads) {
            const ScaledSum p{__ldcg(partials + 3 * b), __ldcg(partials + 3 * b + 1),
                              __ldcg(partials + 3 * b + 2) != 0.0};
            t = norm_merge(t, p);
        }
        t = norm_warp(t);
        __syncthreads();
        if (lane == 0) red[warp] = t;
        __syncthreads();
        if (threadIdx.x == 0) {
            ScaledSum s = red[0];
            for (int w = 1; w < kThreads / 32; ++w) s = norm_merge(s, red[w]);
            double r;
            if (s.nan) r = __longlong_as_double(0x7ff8000000000000LL);
            else if (s.scale == 0.0 || isinf(s.scale)) r = s.scale;
            else r = s.scale * sqrt(s.ssq);
            *out_dev = r;
            *out_host = r;
            *ticket = 0;
        }
    }
}

// ---------------------------------------------------------- permutations
// Node permutation of a vector (owned nodes, bs values each): forward
// dst[new] = src[new_to_old[new]], inverse dst[new_to_old[new]] = src[new].
template<class T>
__global__ void __launch_bounds__(kThreads) k_permute_nodes(std::size_t n, int bs, const std::int64_t* __restrict__ n2o,
                                                            const T* __restrict__ src, T* __restrict__ dst,
                                                            int inverse)
{
    const std::size_t total = n * static_cast<std::size_t>(bs);
    for (std::size_t i = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i < total;
         i += static_cast<std::size_t>(gridDim.x) * kThreads) {
        const std::size_t node = i / bs, c = i - node * bs;
        const std::size_t old = static_cast<std::size_t>(n2o[node]);
        if (inverse) dst[old * bs + c] = src[i];
        else dst[i] = src[old * bs + c];
    }
}

// Values of a permuted matrix gathered from a split layout: entry e takes
// node s = map[e] of the diagonal when s < n, else off-diagonal edge s - n.
template<class T>
__global__ void __launch_bounds__(kThreads) k_gather_split(std::size_t entries, int bs, std::int64_t n,
                                                           const std::int64_t* __restrict__ map,
                                                           const T* __restrict__ diag, const T* __restrict__ off,
                                                           T* __restrict__ values)
{
    const std::size_t total = entries * static_cast<std::size_t>(bs);
    for (std::size_t i = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i < total;
         i += static_cast<std::size_t>(gridDim.x) * kThreads) {
        const std::size_t e = i / bs, c = i - e * bs;
        const std::int64_t s = map[e];
        values[i] = s < n ? diag[static_cast<std::size_t>(s) * bs + c] : off[static_cast<std::size_t>(s - n) * bs + c];
    }
}

// ---------------------------------------------------------- accurate reductions
// The reference's CompensatedSerialReduction sums the rounded products with
// Neumaier's compensated summation, and MixedPrecisionSerialReduction sums in
// long double (reduction.hpp:175-299).  The device forms below keep those
// accuracy classes with a parallel order:
//   mode 1 (compensated): rounded products, each thread a Neumaier pair
//     (sum, correction);
//   mode 2 (mixed precision): each product split exactly by an FMA
//     (TwoProduct) and summed with TwoSum into (sum, correction) -- the Dot2
//     algorithm of Ogita, Rump and Oishi ("Accurate sum and dot product",
//     SIAM J. Sci. Comput. 26, 2005): as accurate as a computation in twice
//     the working precision rounded once, and at least as accurate as the
//     reference's 80-bit long double sum.
// Pairs from threads, warps and CTAs merge exactly: (s1, c1) + (s2, c2) =
// (TwoSum(s1, s2).sum, c1 + c2 + TwoSum(s1, s2).error).  Merges run in a
// fixed order, so results are deterministic.  Float inputs are widened to
// FP64 first (products of floats are exact in FP64).
struct CompPair {
    double s, c;
};

__device__ __forceinline__ void two_sum(double a, double b, double& sum, double& err)
{
    sum = __dadd_rn(a, b);
    const double bb = __dsub_rn(sum, a);
    err = __dadd_rn(__dsub_rn(a, __dsub_rn(sum, bb)), __dsub_rn(b, bb));
}

__device__ __forceinline__ CompPair comp_merge(CompPair x, CompPair y)
{
    double s, e;
    two_sum(x.s, y.s, s, e);
    return {s, __dadd_rn(__dadd_rn(x.c, y.c), e)};
}

template<int MODE>
__device__ __forceinline__ void comp_push(CompPair& a, double x, double y)
{
    if constexpr (MODE == 1) {
        const double p = __dmul_rn(x, y);
        const double t = __dadd_rn(a.s, p);
        a.c = __dadd_rn(a.c, fabs(a.s) >= fabs(p) ? __dadd_rn(__dsub_rn(a.s, t), p)
                                                   : __dadd_rn(__dsub_rn(p, t), a.s));
        a.s = t;
    } else {
        const double h = __dmul_rn(x, y);
        const double r = __fma_rn(x, y, -h);   // exact: x*y = h + r
        double s, q;
        two_sum(a.s, h, s, q);
        a.s = s;
        a.c = __dadd_rn(a.c, __dadd_rn(q, r));
    }
}

__device__ __forceinline__ CompPair comp_warp(CompPair v)
{
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        const CompPair o{__shfl_down_sync(0xffffffffu, v.s, off), __shfl_down_sync(0xffffffffu, v.c, off)};
        v = comp_merge(v, o);
    }
    return v;
}

// k accurate dots a_j . b_j, G per pass.  Partials: two doubles per (dot, CTA).
template<class T, int MODE, int G>
__global__ void __launch_bounds__(kThreads) k_multidot_acc(std::size_t n, int k, PtrPack a, PtrPack b,
                                                           double* partials, unsigned* ticket, double* out_dev,
                                                           double* out_host, double* out_lo)
{
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * kThreads;
    __shared__ CompPair red[G][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int g0 = 0; g0 < k; g0 += G) {
        CompPair acc[G];
        const T* pa[G];
        const T* pb[G];
#pragma unroll
        for (int j = 0; j < G; ++j) {
            acc[j] = {0.0, 0.0};
            pa[j] = g0 + j < k ? static_cast<const T*>(a.p[g0 + j]) : nullptr;
            pb[j] = g0 + j < k ? static_cast<const T*>(b.p[g0 + j]) : nullptr;
        }
        for (std::size_t i = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
#pragma unroll
            for (int j = 0; j < G; ++j)
                if (g0 + j < k)
                    comp_push<MODE>(acc[j], static_cast<double>(pa[j][i]), static_cast<double>(pb[j][i]));
        }
#pragma unroll
        for (int j = 0; j < G; ++j) {
            const CompPair v = comp_warp(acc[j]);
            if (lane == 0) red[j][warp] = v;
        }
        __syncthreads();
        if (threadIdx.x < G && g0 + static_cast<int>(threadIdx.x) < k) {
            CompPair t = red[threadIdx.x][0];
            for (int w = 1; w < kThreads / 32; ++w) t = comp_merge(t, red[threadIdx.x][w]);
            const std::size_t d = static_cast<std::size_t>(g0) + threadIdx.x;
            partials[(2 * d) * gridDim.x + blockIdx.x] = t.s;
            partials[(2 * d + 1) * gridDim.x + blockIdx.x] = t.c;
        }
        __syncthreads();
    }
    if (last_block(ticket)) {
        __threadfence();
        for (int j = warp; j < k; j += kThreads / 32) {
            const std::size_t d = static_cast<std::size_t>(j);
            CompPair t{0.0, 0.0};
            for (unsigned bb = lane; bb < gridDim.x; bb += 32)
                t = comp_merge(t, {__ldcg(partials + (2 * d) * gridDim.x + bb),
                                   __ldcg(partials + (2 * d + 1) * gridDim.x + bb)});
            t = comp_warp(t);
            if (lane == 0) {
                double hi, lo;
                two_sum(t.s, t.c, hi, lo);   // hi + lo == s + c exactly
                out_dev[j] = hi;
                out_host[j] = hi;
                if (out_lo != nullptr) out_lo[j] = lo;
            }
        }
        if (threadIdx.x == 0) *ticket = 0;
    }
}

// Largest magnitude with NaN detection: scratch[0] = max |x|, scratch[1] = 1
// when a NaN was seen.
template<class T>
__global__ void __launch_bounds__(kThreads) k_absmax(std::size_t n, const T* __restrict__ x, double* partials,
                                                     unsigned* ticket, double* scratch)
{
    double m = 0.0, bad = 0.0;
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * kThreads;
    for (std::size_t i = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
        const double v = fabs(static_cast<double>(x[i]));
        if (isnan(v)) bad = 1.0;
        else m = fmax(m, v);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        m = fmax(m, __shfl_down_sync(0xffffffffu, m, off));
        bad = fmax(bad, __shfl_down_sync(0xffffffffu, bad, off));
    }
    __shared__ double rm[kThreads / 32], rb[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        rm[warp] = m;
        rb[warp] = bad;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < kThreads / 32; ++w) {
            m = fmax(m, rm[w]);
            bad = fmax(bad, rb[w]);
        }
        partials[2 * blockIdx.x] = m;
        partials[2 * blockIdx.x + 1] = bad;
    }
    if (last_block(ticket)) {
        __threadfence();
        if (threadIdx.x == 0) {
            double mm = 0.0, bb = 0.0;
            for (unsigned b = 0; b < gridDim.x; ++b) {
                mm = fmax(mm, __ldcg(partials + 2 * b));
                bb = fmax(bb, __ldcg(partials + 2 * b + 1));
            }
            scratch[0] = mm;
            scratch[1] = bb;
            *ticket = 0;
        }
    }
}

// Doubled-precision 2-norm: entries scaled by the power of two of max |x|
// (exact), squares split by TwoProduct and summed as in Dot2, the square
// root of the (sum, correction) pair refined by one Newton step.  NaN gives
// NaN; an infinite or zero maximum is returned as is.
template<class T>
__global__ void __launch_bounds__(kThreads) k_norm_acc(std::size_t n, const T* __restrict__ x,
                                                       const double* __restrict__ scratch, double* partials,
                                                       unsigned* ticket, double* out_dev, double* out_host)
{
    const double mx = scratch[0];
    const bool special = scratch[1] != 0.0 || mx == 0.0 || isinf(mx);
    const int e = special ? 0 : ilogb(mx);
    CompPair acc{0.0, 0.0};
    if (!special) {
        const std::size_t stride = static_cast<std::size_t>(gridDim.x) * kThreads;
        for (std::size_t i = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
            const double y = scalbn(static_cast<double>(x[i]), -e);
            comp_push<2>(acc, y, y);
        }
    }
    acc = comp_warp(acc);
    __shared__ CompPair red[kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) red[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        CompPair t = red[0];
        for (int w = 1; w < kThreads / 32; ++w) t = comp_merge(t, red[w]);
        partials[2 * blockIdx.x] = t.s;
        partials[2 * blockIdx.x + 1] = t.c;
    }
    if (last_block(ticket)) {
        __threadfence();
        if (threadIdx.x == 0) {
            CompPair t{0.0, 0.0};
            for (unsigned b = 0; b < gridDim.x; ++b)
                t = comp_merge(t, {__ldcg(partials + 2 * b), __ldcg(partials + 2 * b + 1)});
            double r;
            if (scratch[1] != 0.0) {
                r = __longlong_as_double(0x7ff8000000000000LL);
            } else if (special) {
                r = mx;
            } else {
                double hi, lo;
                two_sum(t.s, t.c, hi, lo);
                const double r0 = sqrt(hi);
                const double resid = __dadd_rn(__fma_rn(-r0, r0, hi), lo);   // (hi + lo) - r0^2
                r = scalbn(__dadd_rn(r0, __ddiv_rn(resid, __dmul_rn(2.0, r0))), e);
            }
            *out_dev = r;
            *out_host = r;
            *ticket = 0;
        }
    }
}

// q = r / d (FP32) with ||r|| and ||q|| in the same pass: the learned
// preconditioner's input scaling.  Plain FP64 sums of squares (the inputs
// are residuals; the network needs the norms to FP32 accuracy only), summed
// per thread, per CTA and over CTAs in a fixed order: deterministic.
template<class T>
__global__ void __launch_bounds__(256) k_prepare_norms(std::size_t n, const T* __restrict__ r,
                                                       const float* __restrict__ dinv, float* __restrict__ q,
                                                       double* partials, unsigned* ticket, double* norms)
{
    constexpr int kU = 4;
    double a = 0.0, b = 0.0;
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * 256;
    for (std::size_t i0 = static_cast<std::size_t>(blockIdx.x) * 256 + threadIdx.x; i0 < n; i0 += kU * stride) {
        T rv[kU];
        float dv[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const std::size_t i = i0 + u * stride;
            rv[u] = i < n ? r[i] : T(0);
            dv[u] = i < n ? dinv[i] : 0.0f;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const std::size_t i = i0 + u * stride;
            if (i < n) {
                const float qv = static_cast<float>(rv[u]) * dv[u];
                q[i] = qv;
                const double rd = static_cast<double>(rv[u]), qd = static_cast<double>(qv);
                a = fma(rd, rd, a);
                b = fma(qd, qd, b);
            }
        }
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, m);
        b += __shfl_xor_sync(0xffffffffu, b, m);
    }
    __shared__ double red[2][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0;
        for (int w = 0; w < 8; ++w) {
            sa += red[0][w];
            sb += red[1][w];
        }
        partials[2 * blockIdx.x] = sa;
        partials[2 * blockIdx.x + 1] = sb;
    }
    if (last_block(ticket)) {
        __threadfence();
        double ta = 0.0, tb = 0.0;
        for (unsigned k = threadIdx.x; k < gridDim.x; k += 256) {
            ta += __ldcg(partials + 2 * k);
            tb += __ldcg(partials + 2 * k + 1);
        }
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) {
            ta += __shfl_xor_sync(0xffffffffu, ta, m);
            tb += __shfl_xor_sync(0xffffffffu, tb, m);
        }
        __syncthreads();
        if (lane == 0) {
            red[0][warp] = ta;
            red[1][warp] = tb;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double sa = 0.0, sb = 0.0;
            for (int w = 0; w < 8; ++w) {
                sa += red[0][w];
                sb += red[1][w];
            }
            norms[0] = norms[1] = sqrt(sa);
            norms[2] = norms[3] = sqrt(sb);
            *ticket = 0;
        }
    }
}

// ||x - w|| and ||x|| in one pass (the learned preconditioner's residual
// check, which only compares the two): plain FP64 sums of squares, loads four
// deep per thread, summed per thread, per CTA and over CTAs in a fixed order
// (every thread of the last CTA takes a strided share of the partials).
__global__ void __launch_bounds__(256) k_residual_norms(std::size_t n, const double* __restrict__ x,
                                                        const double* __restrict__ w, double* partials,
                                                        unsigned* ticket, double* out_dev, double* out_host)
{
    constexpr int kU = 4;
    double a = 0.0, b = 0.0;
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * 256;
    for (std::size_t i0 = static_cast<std::size_t>(blockIdx.x) * 256 + threadIdx.x; i0 < n; i0 += kU * stride) {
        double xv[kU], wv[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const std::size_t i = i0 + u * stride;
            xv[u] = i < n ? x[i] : 0.0;
            wv[u] = i < n ? w[i] : 0.0;
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const double d = xv[u] - wv[u];
            a = fma(d, d, a);
            b = fma(xv[u], xv[u], b);
        }
    }
#pragma unroll
    for (int m = 16; m > 0; m >>= 1) {
        a += __shfl_xor_sync(0xffffffffu, a, m);
        b += __shfl_xor_sync(0xffffffffu, b, m);
    }
    __shared__ double red[2][8];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0;
        for (int k = 0; k < 8; ++k) {
            sa += red[0][k];
            sb += red[1][k];
        }
        partials[2 * blockIdx.x] = sa;
        partials[2 * blockIdx.x + 1] = sb;
    }
    if (last_block(ticket)) {
        __threadfence();
        double ta = 0.0, tb = 0.0;
        for (unsigned k = threadIdx.x; k < gridDim.x; k += 256) {
            ta += __ldcg(partials + 2 * k);
            tb += __ldcg(partials + 2 * k + 1);
        }
#pragma unroll
        for (int m = 16; m > 0; m >>= 1) {
            ta += __shfl_xor_sync(0xffffffffu, ta, m);
            tb += __shfl_xor_sync(0xffffffffu, tb, m);
        }
        __syncthreads();
        if (lane == 0) {
            red[0][warp] = ta;
            red[1][warp] = tb;
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            double sa = 0.0, sb = 0.0;
            for (int k = 0; k < 8; ++k) {
                sa += red[0][k];
                sb += red[1][k];
            }
            out_dev[0] = out_host[0] = sqrt(sa);
            out_dev[1] = out_host[1] = sqrt(sb);
            *ticket = 0;
        }
    }
}

inline PtrPack pack(const void* const* p, int k)
{
    PtrPack pk{};
    for (int i = 0; i < k; ++i) pk.p[i] = p[i];
    return pk;
}

double* partials_of(Context& c) { return c.partials.as<double>(); }
unsigned* ticket_of(Context& c) { return c.tickets.as<unsigned>(); }

}  // namespace

namespace kern {

#define LAUNCH_EW(kernel, n, ...)                                                  \
    do {                                                                           \
        if ((n) == 0) break;                                                       \
        kernel<<<ew_blocks(n), kThreads, 0, c.stream>>>((n), __VA_ARGS__);         \
        OWTK_CUDA(cudaGetLastError());                                             \
        c.launched();                                                              \
    } while (0)

template<class T> void fill(Context& c, std::size_t n, T value, T* x) { LAUNCH_EW(k_fill<T>, n, value, x); }
template<class T> void copy(Context& c, std::size_t n, const T* x, T* y)
{
    if (x == y) return;
    LAUNCH_EW(k_copy<T>, n, x, y);
}
template<class T> void axpy(Context& c, std::size_t n, T alpha, const T* x, T* y) { LAUNCH_EW(k_axpy<T>, n, alpha, x, y); }
template<class T> void scale(Context& c, std::size_t n, T alpha, T* x) { LAUNCH_EW(k_scale<T>, n, alpha, x); }
template<class T> void lincomb(Context& c, std::size_t n, T a, const T* x, T b, const T* y, T* out)
{
    LAUNCH_EW(k_lincomb<T>, n, a, x, b, y, out);
}
template<class T> void sub(Context& c, std::size_t n, const T* b, const T* a, T* out) { LAUNCH_EW(k_sub<T>, n, b, a, out); }
template<class T> void divide(Context& c, std::size_t n, const T* x, T s, T* out) { LAUNCH_EW(k_divide<T>, n, x, s, out); }
template<class T> void bicg_p(Context& c, std::size_t n, const T* r, T beta, T omega, const T* v, T* p)
{
    LAUNCH_EW(k_bicg_p<T>, n, r, beta, omega, v, p);
}
template<class T> void bicg_xr(Context& c, std::size_t n, T alpha, const T* ph, T omega, const T* sh,
                               const T* s, const T* t, T* x, T* r)
{
    LAUNCH_EW(k_bicg_xr<T>, n, alpha, ph, omega, sh, s, t, x, r);
}
template<class T> void ch_pszupdate(Context& c, std::size_t n, T beta, T omega, const T* r2, const T* w,
                                    const T* w2, const T* t, const T* z2, const T* v,
                                    T* p2, T* s, T* s2, T* z)
{
    LAUNCH_EW(k_ch_psz<T>, n, beta, omega, r2, w, w2, t, z2, v, p2, s, s2, z);
}
template<class T> void ch_qy(Context& c, std::size_t n, T alpha, const T* r, const T* s, const T* r2,
                             const T* s2, const T* w, const T* z, T* q, T* q2, T* y)
{
    LAUNCH_EW(k_ch_qy<T>, n, alpha, r, s, r2, s2, w, z, q, q2, y);
}
template<class T> void ch_rw(Context& c, std::size_t n, T alpha, T omega, const T* q, const T* y,
                             const T* q2, const T* w2, const T* z2, const T* t, const T* v,
                             T* r, T* r2, T* w)
{
    LAUNCH_EW(k_ch_rw<T>, n, alpha, omega, q, y, q2, w2, z2, t, v, r, r2, w);
}
template<class T> void scaled_copy(Context& c, std::size_t n, const T* x, T s, T* out)
{
    LAUNCH_EW(k_scaled_copy<T>, n, x, s, out);
}
template<class T> void jacobi(Context& c, std::size_t n, const T* inv, const T* in, T* out)
{
    LAUNCH_EW(k_jacobi<T>, n, inv, in, out);
}
template<class T> void reciprocal_checked(Context& c, std::size_t n, const T* d, T minimum, T* inv)
{
    LAUNCH_EW(k_reciprocal<T>, n, d, minimum, inv, c.status.as<unsigned>());
}
template<class T> void cgs_update(Context& c, std::size_t n, int k, const T* const* basis, const double* h, T* w)
{
    LAUNCH_EW(k_cgs_update<T>, n, k, pack(reinterpret_cast<const void* const*>(basis), k), h, w);
}
template<class T> void cgs_update_scale(Context& c, std::size_t n, int k, const T* const* basis, const double* h,
                                        const T* w, T s, T* out)
{
    LAUNCH_EW(k_cgs_update_scale<T>, n, k, pack(reinterpret_cast<const void* const*>(basis), k), h, w, s, out);
}
template<class T> void gmres_update(Context& c, std::size_t n, int k, const T* const* dirs,
                                    const double* coef, const T* base, T* out)
{
    LAUNCH_EW(k_gmres_update<T>, n, k, pack(reinterpret_cast<const void* const*>(dirs), k), coef, base, out);
}

template<class T> void multidot(Context& c, std::size_t n, int k, const T* const* a,
                                const T* const* b, double* out_dev, double* out_host)
{
    if (k <= 0) return;
    if (k > kMaxBatch) fail(OWTK_ERR_INVALID_ARGUMENT, "dot batch too large");
    const unsigned blocks = reduce_blocks(c, n);
    const PtrPack pa = pack(reinterpret_cast<const void* const*>(a), k);
    const PtrPack pb = pack(reinterpret_cast<const void* const*>(b), k);
    double* pp = partials_of(c);
    unsigned* tk = ticket_of(c);
    if (k == 1)
        k_multidot<T, 1, 8><<<blocks, kThreads, 0, c.stream>>>(n, k, pa, pb, pp, tk, out_dev, out_host);
    else if (k == 2)
        k_multidot<T, 2, 4><<<blocks, kThreads, 0, c.stream>>>(n, k, pa, pb, pp, tk, out_dev, out_host);
    else if (k <= 4)
        k_multidot<T, 4, 2><<<blocks, kThreads, 0, c.stream>>>(n, k, pa, pb, pp, tk, out_dev, out_host);
    else
        k_multidot<T, 8, 1><<<blocks, kThreads, 0, c.stream>>>(n, k, pa, pb, pp, tk, out_dev, out_host);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void basis_dots(Context& c, std::size_t n, int k, const T* const* basis, const T* x,
                                  double* out_dev, double* out_host)
{
    if (k + 1 > 32) fail(OWTK_ERR_INVALID_ARGUMENT, "basis dots take at most 31 basis vectors");
    const unsigned want = reduce_blocks(c, n);
    const PtrPack pb = pack(reinterpret_cast<const void* const*>(basis), k);
    // Register tiers of the basis size: fewer registers, more resident CTAs.
    if (k + 1 <= 4)
        k_basis_dots<T, 4><<<resident_blocks(c, k_basis_dots<T, 4>, want), kThreads, 0, c.stream>>>(
            n, k, pb, x, partials_of(c), ticket_of(c), out_dev, out_host);
    else if (k + 1 <= 8)
        k_basis_dots<T, 8><<<resident_blocks(c, k_basis_dots<T, 8>, want), kThreads, 0, c.stream>>>(
            n, k, pb, x, partials_of(c), ticket_of(c), out_dev, out_host);
    else if (k + 1 <= 12)
        k_basis_dots<T, 12><<<resident_blocks(c, k_basis_dots<T, 12>, want), kThreads, 0, c.stream>>>(
            n, k, pb, x, partials_of(c), ticket_of(c), out_dev, out_host);
    else if (k + 1 <= 16)
        k_basis_dots<T, 16><<<resident_blocks(c, k_basis_dots<T, 16>, want), kThreads, 0, c.stream>>>(
            n, k, pb, x, partials_of(c), ticket_of(c), out_dev, out_host);
    else if (k + 1 <= 24)
        k_basis_dots<T, 24><<<resident_blocks(c, k_basis_dots<T, 24>, want), kThreads, 0, c.stream>>>(
            n, k, pb, x, partials_of(c), ticket_of(c), out_dev, out_host);
    else
        k_basis_dots<T, 32><<<resident_blocks(c, k_basis_dots<T, 32>, want), kThreads, 0, c.stream>>>(
            n, k, pb, x, partials_of(c), ticket_of(c), out_dev, out_host);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void cgs_update_dot(Context& c, std::size_t n, int k, const T* const* basis,
                                      const double* h, T* w, double* out_dev, double* out_host)
{
    if (k + 1 > 32) fail(OWTK_ERR_INVALID_ARGUMENT, "fused Gram-Schmidt pass takes at most 31 basis vectors");
    const unsigned want = reduce_blocks(c, n);
    const PtrPack pb = pack(reinterpret_cast<const void* const*>(basis), k);
    // Register tiers of the basis size: fewer registers, more resident CTAs.
    if (k + 1 <= 4)
        k_cgs_update_dot<T, 4><<<resident_blocks(c, k_cgs_update_dot<T, 4>, want), kThreads, 0, c.stream>>>(
            n, k, pb, h, w, partials_of(c), ticket_of(c), out_dev, out_host);
    else if (k + 1 <= 8)
        k_cgs_update_dot<T, 8><<<resident_blocks(c, k_cgs_update_dot<T, 8>, want), kThreads, 0, c.stream>>>(
            n, k, pb, h, w, partials_of(c), ticket_of(c), out_dev, out_host);
    else if (k + 1 <= 12)
        k_cgs_update_dot<T, 12><<<resident_blocks(c, k_cgs_update_dot<T, 12>, want), kThreads, 0, c.stream>>>(
            n, k, pb, h, w, partials_of(c), ticket_of(c), out_dev, out_host);
    else if (k + 1 <= 16)
        k_cgs_update_dot<T, 16><<<resident_blocks(c, k_cgs_update_dot<T, 16>, want), kThreads, 0, c.stream>>>(
            n, k, pb, h, w, partials_of(c), ticket_of(c), out_dev, out_host);
    else if (k + 1 <= 24)
        k_cgs_update_dot<T, 24><<<resident_blocks(c, k_cgs_update_dot<T, 24>, want), kThreads, 0, c.stream>>>(
            n, k, pb, h, w, partials_of(c), ticket_of(c), out_dev, out_host);
    else
        k_cgs_update_dot<T, 32><<<resident_blocks(c, k_cgs_update_dot<T, 32>, want), kThreads, 0, c.stream>>>(
            n, k, pb, h, w, partials_of(c), ticket_of(c), out_dev, out_host);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void norm(Context& c, std::size_t n, const T* x, double* out_dev, double* out_host)
{
    const unsigned blocks = reduce_blocks(c, n);
    k_norm<T><<<blocks, kThreads, 0, c.stream>>>(n, x, partials_of(c), ticket_of(c), out_dev, out_host);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void permute_nodes(Context& c, std::size_t n, std::size_t bs, const std::int64_t* n2o, const T* src,
                                     T* dst, bool inverse)
{
    const std::size_t total = n * bs;
    if (total == 0) return;
    const unsigned blocks = static_cast<unsigned>(std::min<std::size_t>((total + kThreads - 1) / kThreads,
                                                                       static_cast<std::size_t>(c.sm_count) * 16));
    k_permute_nodes<T><<<blocks, kThreads, 0, c.stream>>>(n, static_cast<int>(bs), n2o, src, dst, inverse ? 1 : 0);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void gather_split(Context& c, std::size_t entries, std::size_t bs, std::size_t n, const std::int64_t* map,
                                    const T* diag, const T* off, T* values)
{
    const std::size_t total = entries * bs;
    if (total == 0) return;
    const unsigned blocks = static_cast<unsigned>(std::min<std::size_t>((total + kThreads - 1) / kThreads,
                                                                       static_cast<std::size_t>(c.sm_count) * 16));
    k_gather_split<T><<<blocks, kThreads, 0, c.stream>>>(entries, static_cast<int>(bs), static_cast<std::int64_t>(n),
                                                         map, diag, off, values);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void multidot_accurate(Context& c, std::size_t n, int k, int mode, const T* const* a,
                                         const T* const* b, double* out_dev, double* out_host, double* out_lo)
{
    if (k <= 0) return;
    if (k > kMaxBatch) fail(OWTK_ERR_INVALID_ARGUMENT, "dot batch too large");
    if (mode != 1 && mode != 2) fail(OWTK_ERR_INVALID_ARGUMENT, "unknown reduction mode");
    const unsigned blocks = reduce_blocks(c, n);
    const PtrPack pa = pack(reinterpret_cast<const void* const*>(a), k);
    const PtrPack pb = pack(reinterpret_cast<const void* const*>(b), k);
    if (mode == 1)
        k_multidot_acc<T, 1, 4><<<blocks, kThreads, 0, c.stream>>>(n, k, pa, pb, partials_of(c), ticket_of(c),
                                                                    out_dev, out_host, out_lo);
    else
        k_multidot_acc<T, 2, 4><<<blocks, kThreads, 0, c.stream>>>(n, k, pa, pb, partials_of(c), ticket_of(c),
                                                                    out_dev, out_host, out_lo);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void norm_accurate(Context& c, std::size_t n, const T* x, double* scratch, double* out_dev,
                                     double* out_host)
{
    const unsigned blocks = reduce_blocks(c, n);
    k_absmax<T><<<blocks, kThreads, 0, c.stream>>>(n, x, partials_of(c), ticket_of(c), scratch);
    k_norm_acc<T><<<blocks, kThreads, 0, c.stream>>>(n, x, scratch, partials_of(c), ticket_of(c), out_dev,
                                                     out_host);
    OWTK_CUDA(cudaGetLastError());
    c.launched(2);
}

template<class T>
void prepare_norms(Context& c, std::size_t n, const T* r, const float* dinv, float* q, double* norms)
{
    const std::size_t want = (n + 256 * 4 - 1) / (256 * 4);
    const unsigned blocks = static_cast<unsigned>(std::min<std::size_t>(std::max<std::size_t>(want, 1),
                                                                       std::min(c.sm_count * 8, kReduceBlocks)));
    k_prepare_norms<T><<<blocks, 256, 0, c.stream>>>(n, r, dinv, q, partials_of(c), ticket_of(c), norms);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}
template void prepare_norms<double>(Context&, std::size_t, const double*, const float*, float*, double*);

void residual_norms(Context& c, std::size_t n, const double* x, const double* w, double* out_dev, double* out_host)
{
    const std::size_t want = (n + 256 * 4 - 1) / (256 * 4);
    const unsigned blocks = static_cast<unsigned>(std::min<std::size_t>(std::max<std::size_t>(want, 1),
                                                                       std::min(c.sm_count * 8, kReduceBlocks)));
    k_residual_norms<<<blocks, 256, 0, c.stream>>>(n, x, w, partials_of(c), ticket_of(c), out_dev, out_host);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class To, class From> void convert(Context& c, std::size_t n, const From* src, To* dst)
{
    LAUNCH_EW((k_convert<To, From>), n, src, dst);
}
template void convert<float, double>(Context&, std::size_t, const double*, float*);
template void convert<double, float>(Context&, std::size_t, const float*, double*);
template void convert<__nv_bfloat16, double>(Context&, std::size_t, const double*, __nv_bfloat16*);

#define INSTANTIATE(T)                                                                              \
    template void fill<T>(Context&, std::size_t, T, T*);                                           \
    template void copy<T>(Context&, std::size_t, const T*, T*);                                    \
    template void axpy<T>(Context&, std::size_t, T, const T*, T*);                                 \
    template void scale<T>(Context&, std::size_t, T, T*);                                          \
    template void lincomb<T>(Context&, std::size_t, T, const T*, T, const T*, T*);                 \
    template void sub<T>(Context&, std::size_t, const T*, const T*, T*);                           \
    template void divide<T>(Context&, std::size_t, const T*, T, T*);                               \
    template void bicg_p<T>(Context&, std::size_t, const T*, T, T, const T*, T*);                  \
    template void bicg_xr<T>(Context&, std::size_t, T, const T*, T, const T*, const T*, const T*, T*, T*); \
    template void ch_pszupdate<T>(Context&, std::size_t, T, T, const T*, const T*, const T*, const T*,    \
                                  const T*, const T*, T*, T*, T*, T*);                             \
    template void ch_qy<T>(Context&, std::size_t, T, const T*, const T*, const T*, const T*, const T*,    \
                           const T*, T*, T*, T*);                                                  \
    template void ch_rw<T>(Context&, std::size_t, T, T, const T*, const T*, const T*, const T*, const T*, \
                           const T*, const T*, T*, T*, T*);                                        \
    template void jacobi<T>(Context&, std::size_t, const T*, const T*, T*);                        \
    template void scaled_copy<T>(Context&, std::size_t, const T*, T, T*);                          \
    template void reciprocal_checked<T>(Context&, std::size_t, const T*, T, T*);                   \
    template void cgs_update<T>(Context&, std::size_t, int, const T* const*, const double*, T*);   \
    template void cgs_update_scale<T>(Context&, std::size_t, int, const T* const*, const double*, const T*, T, T*); \
    template void basis_dots<T>(Context&, std::size_t, int, const T* const*, const T*, double*, double*); \
    template void gmres_update<T>(Context&, std::size_t, int, const T* const*, const double*, const T*, T*); \
    template void multidot<T>(Context&, std::size_t, int, const T* const*, const T* const*, double*, double*); \
    template void cgs_update_dot<T>(Context&, std::size_t, int, const T* const*, const double*, T*, double*, double*); \
    template void norm<T>(Context&, std::size_t, const T*, double*, double*);                       \
    template void multidot_accurate<T>(Context&, std::size_t, int, int, const T* const*, const T* const*,  \
                                       double*, double*, double*);                                 \
    template void norm_accurate<T>(Context&, std::size_t, const T*, double*, double*, double*);      \
    template void permute_nodes<T>(Context&, std::size_t, std::size_t, const std::int64_t*, const T*, T*, bool); \
    template void gather_split<T>(Context&, std::size_t, std::size_t, std::size_t, const std::int64_t*, const T*, \
                                  const T*, T*);

INSTANTIATE(double)
INSTANTIATE(float)

}  // namespace kern
}  // namespace owtk
