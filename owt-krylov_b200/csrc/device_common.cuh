// Device helpers shared by the kernel translation units.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace owtk::dev {

// Explicitly rounded arithmetic.  The reference's CPU path as shipped (-O3,
// no -march) never contracts a*b+c into an FMA, so every product that the
// reference rounds is rounded here too; with these intrinsics nvcc cannot
// contract them, and element-wise results match the CPU bit for bit.
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double add_rn(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ float add_rn(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ double sub_rn(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ float sub_rn(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ double div_rn(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float div_rn(float a, float b) { return __fdiv_rn(a, b); }

__device__ __forceinline__ double warp_sum(double v)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// Device error word bits (read by the host after a stream synchronisation).
enum : unsigned {
    kErrMissingDiagonal = 1u,
    kErrSingularDiagonal = 2u,
    kErrZeroPivot = 4u,
    kErrTimeout = 8u,
};

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p)
{
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release(unsigned* p, unsigned v)
{
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v) : "memory");
}

constexpr int kThreads = 256;

// One-pass scaled sum of squares (the dnrm2 recurrence): |x| = scale * sqrt(ssq).
// Partial states merge exactly like the sequential recurrence would rescale.
struct ScaledSum {
    double scale, ssq;
    int nan;
};

__device__ __forceinline__ void norm_push(ScaledSum& a, double x)
{
    const double m = fabs(x);
    if (isnan(m)) { a.nan = 1; return; }
    if (m == 0.0 || isinf(a.scale)) return;
    if (m > a.scale) {
        if (isinf(m)) { a.scale = m; a.ssq = 1.0; return; }
        const double r = a.scale / m;
        a.ssq = 1.0 + a.ssq * r * r;
        a.scale = m;
    } else {
        const double r = m / a.scale;
        a.ssq += r * r;
    }
}

__device__ __forceinline__ ScaledSum norm_merge(ScaledSum a, ScaledSum b)
{
    ScaledSum r;
    r.nan = a.nan | b.nan;
    if (a.scale < b.scale) { const ScaledSum t = a; a = b; b = t; }
    r.scale = a.scale;
    if (a.scale == 0.0) { r.ssq = 0.0; return r; }
    if (isinf(a.scale)) { r.ssq = 1.0; return r; }
    const double q = b.scale / a.scale;
    r.ssq = a.ssq + b.ssq * q * q;
    return r;
}

__device__ __forceinline__ ScaledSum norm_warp(ScaledSum a)
{
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        ScaledSum b;
        b.scale = __shfl_xor_sync(0xffffffffu, a.scale, o);
        b.ssq = __shfl_xor_sync(0xffffffffu, a.ssq, o);
        b.nan = __shfl_xor_sync(0xffffffffu, a.nan, o);
        a = norm_merge(a, b);
    }
    return a;
}

// ---------------------------------------------------------------- bulk copies
// One-dimensional bulk copies global -> shared (cp.async.bulk, the TMA unit's
// untiled form) completing on a shared-memory mbarrier.  Source and
// destination must be 16-byte aligned and the size a multiple of 16.  No
// multicast form is used anywhere in this library.

__device__ __forceinline__ std::uint32_t smem_u32(const void* p)
{
    return static_cast<std::uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(std::uint32_t bar, std::uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

// Makes barrier initialisation and prior shared-memory writes visible to the
// async proxy (the bulk-copy engine).
__device__ __forceinline__ void fence_proxy_async_smem()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_arrive(std::uint32_t bar)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(std::uint32_t bar, std::uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(std::uint32_t bar, std::uint32_t parity)
{
    std::uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(bar), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait for the phase of parity `parity` to complete.
__device__ __forceinline__ bool mbar_wait_bounded(std::uint32_t bar, std::uint32_t parity, int limit)
{
    for (int i = 0; i < limit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ std::uint64_t l2_policy_evict_first()
{
    std::uint64_t p;
    asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
    return p;
}

// Hint: bring `bytes` (a multiple of 16) from a 16-byte aligned address into L2.
__device__ __forceinline__ void prefetch_l2(const void* src, std::uint32_t bytes)
{
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(src), "r"(bytes) : "memory");
}

__device__ __forceinline__ void bulk_load(std::uint32_t dst, const void* src, std::uint32_t bytes,
                                          std::uint32_t bar, std::uint64_t policy)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes.L2::cache_hint"
        " [%0], [%1], %2, [%3], %4;" ::"r"(dst),
        "l"(src), "r"(bytes), "r"(bar), "l"(policy)
        : "memory");
}

// Granule-aligned copy of elements [b, e) of an array of `total` elements of
// `sz` bytes starting at a 16-byte aligned base.  Returns the bytes to copy
// (0: nothing), the copy's first byte `lo`, the index of element b in the
// destination and how many of the run's elements the copy holds.
__device__ __forceinline__ std::uint32_t bulk_segment(std::size_t b, std::size_t e, std::size_t total, int sz,
                                                      std::size_t& lo, int& off, int& avail)
{
    const std::size_t bb = b * sz, eb = e * sz, tb = (total * sz) & ~std::size_t(15);
    lo = bb & ~std::size_t(15);
    std::size_t hi = (eb + 15) & ~std::size_t(15);
    if (hi > tb) hi = tb;
    off = static_cast<int>((bb - lo) / sz);
    if (hi <= bb) {
        avail = 0;
        return 0;
    }
    avail = static_cast<int>((hi - bb) / sz);
    return static_cast<std::uint32_t>(hi - lo);
}

// OR of `pred` over the `count` threads that meet at named barrier `id`.
__device__ __forceinline__ bool bar_any(int id, int count, bool pred)
{
    std::uint32_t out;
    asm volatile(
        "{\n\t.reg .pred pi, po;\n\t"
        "setp.ne.u32 pi, %1, 0;\n\t"
        "bar.red.or.pred po, %2, %3, pi;\n\t"
        "selp.u32 %0, 1, 0, po;\n\t}"
        : "=r"(out)
        : "r"(static_cast<std::uint32_t>(pred)), "r"(id), "r"(count)
        : "memory");
    return out != 0;
}

}  // namespace owtk::dev
