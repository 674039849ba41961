// Device helpers shared by the kernel translation units.
#pragma once

#include <cuda_runtime.h>

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

}  // namespace owtk::dev
