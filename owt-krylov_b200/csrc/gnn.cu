// Learned preconditioner: a message-passing network on the matrix graph
// (hidden 64, 4 layers, no biases) whose dense products run on the sm_100a
// tensor cores (tcgen05.mma, BF16 operands in shared memory, FP32
// accumulators in TMEM), with hand-written forward, backward and Adam
// kernels.  The network (FP64 restatement in oracle/gnn.py):
//
//   q = r/d (the Jacobi step);  x_v = [r_v/rms(r), q_v/rms(q), 0...] (16 features)
//   h0 = x We^T;  per layer: m_v = sum_u w_vu h_u,  h += relu([h | m] Wl^T)
//   out = q + rms(q) * (h4 Wd^T)       (an untrained decoder is Jacobi)
//
// Device layouts: node features h are BF16 rows of 64 (128 bytes); the layer
// kernel gathers a 128-row tile of [h | m] into swizzled shared memory, runs
// eight K=16 MMAs against the resident layer weight and applies the
// ReLU/residual epilogue straight from TMEM.

#include <cuda.h>
#include <cuda_bf16.h>
#include <cudaTypedefs.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <random>
#include <string>
#include <vector>

#include "device_common.cuh"
#include "owtk_internal.h"
#include "umma.cuh"

namespace owtk {
namespace gnn {

using namespace dev;
using bf16 = __nv_bfloat16;

constexpr int kH = 64;             // hidden width
constexpr int kF = 16;             // input features
constexpr int kLayers = 4;
constexpr int kTile = 128;         // rows per tensor-core tile
constexpr int kMmaSpin = 1 << 22;

// ---------------------------------------------------------------- shared pieces
__device__ __forceinline__ std::uint32_t align1024(std::uint32_t a) { return (a + 1023u) & ~1023u; }

// Bounded wait on an mbarrier phase; false if it gave up.
__device__ __forceinline__ bool wait_phase(std::uint32_t bar, std::uint32_t parity)
{
    return mbar_wait_bounded(bar, parity, kMmaSpin);
}

// 16 bytes of a BF16 row (8 features) to / from FP32.
__device__ __forceinline__ void bf16x8_to_f32(const uint4& u, float (&f)[8])
{
    const bf16* b = reinterpret_cast<const bf16*>(&u);
#pragma unroll
    for (int i = 0; i < 8; ++i) f[i] = __bfloat162float(b[i]);
}

__device__ __forceinline__ uint4 f32_to_bf16x8(const float (&f)[8])
{
    uint4 u;
    bf16* b = reinterpret_cast<bf16*>(&u);
#pragma unroll
    for (int i = 0; i < 8; ++i) b[i] = __float2bfloat16_rn(f[i]);
    return u;
}

// Edge weights enter the aggregation rounded to BF16: the product of a BF16
// weight and a BF16 feature is exact in FP32, so s = fma(w, x, s) in FP32 is
// the same operation as the mixed-precision fma.rn.f32.bf16 used here.
__device__ __forceinline__ float bf16_round(float w) { return __bfloat162float(__float2bfloat16_rn(w)); }

// acc += w * f for the 8 BF16 features of f; w holds BF16 bits.
__device__ __forceinline__ void accumulate_row(unsigned short w, const uint4& f, float2 (&acc)[4])
{
    const std::uint32_t x[4] = {f.x, f.y, f.z, f.w};
#pragma unroll
    for (int k = 0; k < 4; ++k)
        asm("{\n\t.reg .b16 lo, hi;\n\tmov.b32 {lo, hi}, %2;\n\t"
            "fma.rn.f32.bf16 %0, lo, %3, %0;\n\t"
            "fma.rn.f32.bf16 %1, hi, %3, %1;\n\t}"
            : "+f"(acc[k].x), "+f"(acc[k].y)
            : "r"(x[k]), "h"(w));
}

__device__ __forceinline__ uint4 pack_bf16x8(const float2 (&acc)[4])
{
    uint4 u;
    std::uint32_t* p = reinterpret_cast<std::uint32_t*>(&u);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const __nv_bfloat162 b = __floats2bfloat162_rn(acc[k].x, acc[k].y);
        p[k] = *reinterpret_cast<const std::uint32_t*>(&b);
    }
    return u;
}

// ---------------------------------------------------------------- generic GEMM
// D (M x N, FP32, row-major) = A (M x K, BF16, row-major) * B (N x K, BF16,
// row-major)^T with M % 128 == 0, N in {64, 128}, K % 64 == 0.  One CTA (4
// warps) per 128-row tile; K in 64-element blocks staged through swizzled
// shared memory.  Used to check the tensor-core path in isolation.
template<int N>
__global__ void __launch_bounds__(128, 1) k_umma_gemm_nt(int K, const bf16* __restrict__ A,
                                                          const bf16* __restrict__ B, float* __restrict__ D,
                                                          unsigned* status)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) std::uint64_t bar_storage;
    __shared__ std::uint32_t tmem_base_s;
    const std::uint32_t base = align1024(smem_u32(smem_raw));
    const std::uint32_t a_tile = base, b_tile = base + kTile * 128;
    unsigned char* gen = smem_raw + (base - smem_u32(smem_raw));
    const std::uint32_t bar = smem_u32(&bar_storage);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const long long row0 = static_cast<long long>(blockIdx.x) * kTile;
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_proxy_async_smem();
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base_s), N);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const std::uint32_t tmem = tmem_base_s;
    constexpr std::uint32_t idesc = umma_idesc_bf16(kTile, N);
    bool ok = true;
    for (int kb = 0; kb < K / 64; ++kb) {
        // Stage A (128 x 64) and B (N x 64): thread t copies 16-byte chunks.
        for (int i = threadIdx.x; i < kTile * 8; i += 128) {
            const int r = i >> 3, c = i & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(A + (row0 + r) * K + kb * 64 + c * 8);
            *reinterpret_cast<uint4*>(gen + sw128(r, c)) = v;
        }
        for (int i = threadIdx.x; i < N * 8; i += 128) {
            const int r = i >> 3, c = i & 7;
            const uint4 v = *reinterpret_cast<const uint4*>(B + static_cast<long long>(r) * K + kb * 64 + c * 8);
            *reinterpret_cast<uint4*>(gen + kTile * 128 + sw128(r, c)) = v;
        }
        fence_proxy_async_smem();
        __syncthreads();
        if (threadIdx.x == 0) {
            tmem_fence_after_sync();
#pragma unroll
            for (int k = 0; k < 4; ++k)
                umma_bf16(tmem, umma_desc_sw128(a_tile + 32 * k), umma_desc_sw128(b_tile + 32 * k), idesc,
                          kb > 0 || k > 0);
            umma_commit(bar);
        }
        ok = ok && wait_phase(bar, kb & 1);
        tmem_fence_after_sync();
        if (!__syncthreads_and(ok)) break;
    }
    if (ok) {
        // Epilogue: warp w reads TMEM lanes 32w..32w+31 = rows of the tile.
#pragma unroll
        for (int c0 = 0; c0 < N; c0 += 32) {
            float v[32];
            tmem_ld32(tmem + (static_cast<std::uint32_t>(32 * warp) << 16) + c0, v);
            float* out = D + (row0 + 32 * warp + lane) * N + c0;
#pragma unroll
            for (int i = 0; i < 32; ++i) out[i] = v[i];
        }
    } else if (threadIdx.x == 0) {
        atomicOr(status, kErrTimeout);
    }
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, N);
}

// ---------------------------------------------------------------- network kernels
struct GraphArgs {
    int n, bs;
    const int* nb_ptr;       // off-diagonal neighbours of v (row v of the matrix)
    const int* nb_col;
    const float* nb_w;       // w_vu = -mean_c a_vu,c / d_v,c
    const int* tr_ptr;       // transposed: the v with u in N(v), for vertex u
    const int* tr_col;
    const float* tr_w;       // w_vu of that edge
    const int* tr_edge;      // index of that edge in the forward (nb) order
    const float* dinv;       // 1 / diagonal, n * bs
    const int* ell_col;      // first 8 neighbours of v at 8 v.. (padding: -1)
    const unsigned short* ell_w;   // their weights as BF16 bits (padding: 0)
    const unsigned char* tile_ovf;   // 128-row tile holds a row with more than 8 neighbours
};

// q = r / d in FP32 (the Jacobi step; its norm scales the network's output).
template<class T>
__global__ void __launch_bounds__(256) k_gnn_prepare(long long count, const T* __restrict__ r,
                                                     const float* __restrict__ dinv, float* __restrict__ q)
{
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) q[i] = static_cast<float>(r[i]) * dinv[i];
}

// Encoder: h0 = x We^T with x = [r / rms(r), q / rms(q), 0...].  A warp
// takes 32 vertices per round: lane j loads vertex j's 2 BS inputs (coalesced;
// the next round's inputs are loaded before this round's arithmetic), then in
// 8 passes of 4 vertices an 8-lane group per vertex computes it, lane `c8`
// features 8*c8..8*c8+7 from its own weights held in registers, the inputs
// shared by shuffles; one coalesced 16-byte store per lane.  The sums are
// packed f32x2 FMAs over the 2 BS nonzero inputs in ascending order; the zero
// inputs are skipped, which leaves every sum bit-identical to the full
// 16-term one (fma(w, 0, s) = s, s never -0).
template<class T, int BS>
__global__ void __launch_bounds__(256) k_gnn_encode(GraphArgs g, const T* __restrict__ r, const float* __restrict__ q,
                                                    const double* norms, const float* __restrict__ we,
                                                    bf16* __restrict__ h0)
{
    constexpr int NF = 2 * BS;
    const int lane = threadIdx.x & 31, grp = lane >> 3, c8 = lane & 7;
    float2 w[NF][4];   // w[f][k] = (We[8 c8 + 2k][f], We[8 c8 + 2k + 1][f])
#pragma unroll
    for (int f = 0; f < NF; ++f)
#pragma unroll
        for (int k = 0; k < 4; ++k)
            w[f][k] = make_float2(we[(8 * c8 + 2 * k) * kF + f], we[(8 * c8 + 2 * k + 1) * kF + f]);
    const double root = sqrt(static_cast<double>(g.n) * g.bs), nr = norms[0], nq = norms[2];
    const float inv_r = nr > 0.0 ? static_cast<float>(root / nr) : 0.0f;
    const float inv_q = nq > 0.0 ? static_cast<float>(root / nq) : 0.0f;
    const long long n = g.n;
    const long long step = static_cast<long long>(gridDim.x) * (blockDim.x / 32) * 32;
    const auto load = [&](long long v0, float (&x)[NF]) {
        const long long v = min(v0 + lane, n - 1);
#pragma unroll
        for (int c = 0; c < BS; ++c) {
            x[c] = static_cast<float>(r[v * BS + c]) * inv_r;
            x[BS + c] = q[v * BS + c] * inv_q;
        }
    };
    long long v0 = (static_cast<long long>(blockIdx.x) * (blockDim.x / 32) + (threadIdx.x >> 5)) * 32;
    float x[NF], xn[NF];
    if (v0 < n) load(v0, x);
    for (; v0 < n; v0 += step) {
        if (v0 + step < n) load(v0 + step, xn);
#pragma unroll
        for (int p = 0; p < 8; ++p) {
            const int src = 4 * p + grp;
            float2 acc[4] = {make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f), make_float2(0.0f, 0.0f),
                             make_float2(0.0f, 0.0f)};
#pragma unroll
            for (int f = 0; f < NF; ++f) {
                const float xf = __shfl_sync(0xffffffffu, x[f], src);
                const float2 xx = make_float2(xf, xf);
#pragma unroll
                for (int k = 0; k < 4; ++k) acc[k] = __ffma2_rn(w[f][k], xx, acc[k]);
            }
            const long long v = v0 + src;
            if (v < n) reinterpret_cast<uint4*>(h0 + v * kH)[c8] = pack_bf16x8(acc);
        }
#pragma unroll
        for (int f = 0; f < NF; ++f) x[f] = xn[f];
    }
}

template<class T>
void launch_encode(unsigned grid, cudaStream_t st, const GraphArgs& g, const T* r, const float* q, const double* norms,
                   const float* we, bf16* h0)
{
    switch (g.bs) {
    case 1: k_gnn_encode<T, 1><<<grid, 256, 0, st>>>(g, r, q, norms, we, h0); break;
    case 2: k_gnn_encode<T, 2><<<grid, 256, 0, st>>>(g, r, q, norms, we, h0); break;
    case 3: k_gnn_encode<T, 3><<<grid, 256, 0, st>>>(g, r, q, norms, we, h0); break;
    case 4: k_gnn_encode<T, 4><<<grid, 256, 0, st>>>(g, r, q, norms, we, h0); break;
    case 5: k_gnn_encode<T, 5><<<grid, 256, 0, st>>>(g, r, q, norms, we, h0); break;
    case 6: k_gnn_encode<T, 6><<<grid, 256, 0, st>>>(g, r, q, norms, we, h0); break;
    case 7: k_gnn_encode<T, 7><<<grid, 256, 0, st>>>(g, r, q, norms, we, h0); break;
    default: k_gnn_encode<T, 8><<<grid, 256, 0, st>>>(g, r, q, norms, we, h0); break;
    }
}

// Decoder: out = q + rms(q) * (h Wd^T).  An 8-lane group per vertex reads the
// row as one coalesced 128-byte load; each lane's partial dot products are
// summed across the group with three shuffles.
template<class O>
__global__ void __launch_bounds__(256) k_gnn_decode(GraphArgs g, const float* __restrict__ q, const double* norms,
                                                    const float* __restrict__ wd, const bf16* __restrict__ h,
                                                    O* __restrict__ out)
{
    // Row c, features 8*c8..8*c8+7 at c * 72 + c8 * 9: conflict-free across a group.
    __shared__ float w[8 * 72];
    for (int i = threadIdx.x; i < 8 * kH; i += blockDim.x) w[(i / kH) * 72 + ((i % kH) / 8) * 9 + i % 8] = wd[i];
    __syncthreads();
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int v = static_cast<int>(t >> 3), c8 = static_cast<int>(t & 7);
    const bool live = v < g.n;
    const float s = static_cast<float>(norms[2] / sqrt(static_cast<double>(g.n) * g.bs));
    float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (live) bf16x8_to_f32(reinterpret_cast<const uint4*>(h + static_cast<long long>(v) * kH)[c8], f);
    float mine = 0.0f;
    for (int c = 0; c < g.bs; ++c) {
        float acc = 0.0f;
#pragma unroll
        for (int i = 0; i < 8; ++i) acc = fmaf(w[c * 72 + c8 * 9 + i], f[i], acc);
        acc += __shfl_xor_sync(0xffffffffu, acc, 1);
        acc += __shfl_xor_sync(0xffffffffu, acc, 2);
        acc += __shfl_xor_sync(0xffffffffu, acc, 4);
        if (c8 == c) mine = acc;
    }
    if (live && c8 < g.bs) {
        const long long o = static_cast<long long>(v) * g.bs + c8;
        out[o] = static_cast<O>(norms[0] > 0.0 ? fmaf(s, mine, q[o]) : 0.0f);
    }
}

// One message-passing layer, fused.  Per 128-row tile:
//  * the tile's own rows h arrive by one 2D TMA load whose 128-byte swizzle
//    is the MMA's K-major operand layout, issued while the previous tile
//    finishes (and the tile after next has its index rows prefetched to L2);
//  * each of the 8 warps aggregates m_v = sum_u w_vu h_u for 16 rows, four at a time
//    (an 8-lane group per row, lane `chunk` owning features 8*chunk..+7), over
//    the rows' padded 8-slot neighbour lists: lane `chunk` loads slot
//    `chunk`'s index and BF16 weight two row steps ahead and the group shares
//    them by shuffles; the neighbours' 16-byte feature chunks are gathered in
//    quarter steps of two slots through a register ring kGatherDepth quarter
//    steps ahead of their use; the sums run in FP32 as mixed-precision FMAs
//    straight from the BF16 halves (each product exact) and m is rounded to
//    BF16 into the swizzled second operand block;
//  * eight K=16 MMAs give Y = [h | m] Wl^T in TMEM; the epilogue writes
//    h + relu(Y) into A0 and one TMA tile store moves it out (for the last
//    layer of an inference pass, four more MMAs of the rounded rows against
//    the BF16 decoder weights, N = 16, give out = q + rms(q) (h Wd^T)).
// Padding slots (index -1) load nothing and carry weight 0: fma(0, x, s) = s
// for the finite chunk x their registers still hold and a running sum that
// is never -0, so the sums are bit-identical to skipping the slot.  Rows with
// more than 8 neighbours continue from their CSR list in the same edge order
// (their tiles are flagged on the host).  Training also keeps m (BF16) and
// the sign mask of Y (one 64-bit word per row) for the backward pass.
constexpr int kEll = 8;            // padded neighbour slots per row
#ifndef OWTK_GNN_DEPTH
#define OWTK_GNN_DEPTH 1
#endif
constexpr int kGatherDepth = OWTK_GNN_DEPTH;   // quarter steps (2 slots) in flight per warp
constexpr int kLayerThreads = 128;   // backward kernels
#ifndef OWTK_GNN_WARPS
#define OWTK_GNN_WARPS 8
#endif
constexpr int kFwdWarps = OWTK_GNN_WARPS;          // forward layer: 4 or 8 warps per tile
constexpr int kFwdThreads = 32 * kFwdWarps;
constexpr int kRowsPerWarp = kTile / kFwdWarps;    // gather rows per warp
constexpr int kRowSteps = kRowsPerWarp / 4;        // row steps of 4 rows
constexpr int kEpiHalves = 8 / kFwdWarps;          // epilogue column halves per thread
static_assert(kFwdWarps == 4 || kFwdWarps == 8, "forward layer: 4 or 8 warps");
constexpr int kLayerSmem = 1024 + 2 * kTile * 128 + 2 * kH * 128;   // A: [h | m], B: Wl
constexpr int kDecodeRows = 16;                                      // Wd padded to N = 16
constexpr int kLayerSmemDec = kLayerSmem + kDecodeRows * 128;        // + Wd (BF16, swizzled)

#ifndef OWTK_GNN_LDOP
#define OWTK_GNN_LDOP ".nc"
#endif
// Chunk `chunk` of feature row u into d when u >= 0 (a padding slot, u < 0,
// leaves d as it is).
__device__ __forceinline__ void load_slot(uint4& d, const bf16* h, int u, int chunk)
{
    const uint4* p = reinterpret_cast<const uint4*>(h + static_cast<long long>(u) * kH) + chunk;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ge.s32 p, %4, 0;\n\t"
        "@p ld.global" OWTK_GNN_LDOP ".v4.u32 {%0, %1, %2, %3}, [%5];\n\t}"
        : "+r"(d.x), "+r"(d.y), "+r"(d.z), "+r"(d.w)
        : "r"(u), "l"(p));
}

// The decoder fused into the last layer (inference): out = q + rms(q) (h Wd^T)
// from the epilogue's rounded rows, with the sums of k_gnn_decode in the same
// order (per 8-feature chunk, then the pairwise tree over the chunks).
template<class O>
struct DecodeArgs {
    const float* q;
    const double* norms;
    const float* wd;
    O* out;
};

#ifndef OWTK_GNN_DEC_BLOCKS
#define OWTK_GNN_DEC_BLOCKS 4
#endif
template<bool TRAIN, bool DECODE = false, class O = float>
__global__ void __launch_bounds__(kFwdThreads, DECODE ? OWTK_GNN_DEC_BLOCKS : 4)
    k_gnn_layer(GraphArgs g, const __grid_constant__ CUtensorMap tmap_in, const __grid_constant__ CUtensorMap tmap_out,
                const bf16* __restrict__ h_in, const bf16* __restrict__ wl, bf16* __restrict__ m_out,
                unsigned long long* __restrict__ mask_out, DecodeArgs<O> dec, unsigned* status)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) std::uint64_t bar_storage[2];   // [0] MMAs done, [1] own rows landed
    __shared__ std::uint32_t tmem_base_s;
    const std::uint32_t raw = smem_u32(smem_raw), base = align1024(raw);
    unsigned char* tile = smem_raw + (base - raw);                 // A0 (h), A1 (m), B0, B1
    const std::uint32_t a0 = base, a1 = base + kTile * 128, b0 = base + 2 * kTile * 128, b1 = b0 + kH * 128;
    const std::uint32_t bar = smem_u32(&bar_storage[0]), bar_h = smem_u32(&bar_storage[1]);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (g.n + kTile - 1) / kTile;

    // Layer weight (64 x 128, row-major = K-major) into the two B blocks.
    for (int i = threadIdx.x; i < kH * 16; i += kFwdThreads) {
        const int r = i >> 4, c16 = i & 15;
        const uint4 v = *reinterpret_cast<const uint4*>(wl + r * 128 + c16 * 8);
        *reinterpret_cast<uint4*>(tile + 2 * kTile * 128 + (c16 >> 3) * kH * 128 + sw128(r, c16 & 7)) = v;
    }
    float dec_scale = 0.0f;
    bool dec_live = false;
    const std::uint32_t wdt = b1 + kH * 128;   // decoder weight tile (DECODE)
    if (DECODE) {
        // Wd (bs x 64, FP32) as a 16-row BF16 operand, rows past bs zero.
        for (int i = threadIdx.x; i < kDecodeRows * 8; i += kFwdThreads) {
            const int c = i >> 3, c8 = i & 7;
            float f[8];
#pragma unroll
            for (int k = 0; k < 8; ++k) f[k] = c < g.bs ? dec.wd[c * kH + c8 * 8 + k] : 0.0f;
            *reinterpret_cast<uint4*>(tile + (wdt - base) + sw128(c, c8)) = f32_to_bf16x8(f);
        }
        dec_scale = static_cast<float>(dec.norms[2] / sqrt(static_cast<double>(g.n) * g.bs));
        dec_live = dec.norms[0] > 0.0;
    }
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        mbar_init(bar_h, 1);
        fence_proxy_async_smem();
    }
    constexpr std::uint32_t kCols = DECODE ? 2 * kH : kH;   // Y (64) and the decoder's 16
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base_s), kCols);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const std::uint32_t tmem = tmem_base_s;
    constexpr std::uint32_t idesc = umma_idesc_bf16(kTile, kH);
    constexpr std::uint32_t idesc_dec = umma_idesc_bf16(kTile, kDecodeRows);
    std::uint32_t mma_waits = 0;   // completions of `bar` so far
    // Own rows of `t` into A0 (rows past n read as zeros); the index rows of
    // the tile after it towards L2.
    const auto stage_tile = [&](int t) {
        if (t < ntiles) {
            mbar_arrive_expect_tx(bar_h, kTile * 128);
            tma_load_2d(a0, &tmap_in, 0, t * kTile, bar_h);
        }
        const int tn = t + static_cast<int>(gridDim.x);
        if (tn < ntiles) {
            const std::uint32_t rows = static_cast<std::uint32_t>(min(kTile, g.n - tn * kTile));
            prefetch_l2(g.ell_col + static_cast<long long>(tn) * kTile * kEll, rows * kEll * 4);
            prefetch_l2(g.ell_w + static_cast<long long>(tn) * kTile * kEll, rows * kEll * 2);
        }
    };
    if (threadIdx.x == 0) stage_tile(blockIdx.x);
    const int grp = lane >> 3, chunk = lane & 7;   // 4 rows at a time, 8 lanes x 16 bytes per row
    int iter = 0;
    bool ok = true, h_pending = blockIdx.x < ntiles;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++iter) {
        const int row0 = t * kTile;
        const bool overflow = g.tile_ovf[t] != 0;
        // ---- m: row step s (0..7) covers rows 32*warp + 4*s + grp; its 8
        // slots are gathered as 4 quarter steps of 2 slots, issued kGatherDepth
        // quarter steps ahead of their accumulation through a register ring.
        // Lane `chunk` of a group loads the row's slot `chunk` (index and
        // weight, two row steps ahead of its first gather) and shares it by
        // shuffles.
        const int first = row0 + kRowsPerWarp * warp + grp;
        const auto ell_at = [&](int s) { return static_cast<long long>(min(first + 4 * s, g.n - 1)) * kEll + chunk; };
        constexpr int kQuarters = 4 * kRowSteps;
        int ecol[8];
        unsigned ew[8];   // BF16 weight bits
        // A padding slot loads nothing (weight 0): it keeps a chunk gathered
        // earlier in this tile or these zeros.
        uint4 ring[kGatherDepth + 1][2];
#pragma unroll
        for (int i = 0; i <= kGatherDepth; ++i) ring[i][0] = ring[i][1] = make_uint4(0, 0, 0, 0);
        const auto load_ell = [&](int s) {
            ecol[s & 7] = __ldg(g.ell_col + ell_at(s));
            ew[s & 7] = __ldg(g.ell_w + ell_at(s));
        };
        const auto issue = [&](int k) {   // quarter k: slots 2*(k&3), +1 of row step k>>2
            const int s = k >> 2;
#pragma unroll
            for (int j = 0; j < 2; ++j) {
                const int u = __shfl_sync(0xffffffffu, ecol[s & 7], (lane & ~7) + 2 * (k & 3) + j);
                load_slot(ring[k % (kGatherDepth + 1)][j], h_in, u, chunk);
            }
        };
        static_assert(kGatherDepth >= 1 && kGatherDepth <= 20, "index ring holds 8 row steps");
        load_ell(0);
        load_ell(1);
        load_ell(2);
#pragma unroll
        for (int k = 0; k < kGatherDepth; ++k) {
            if ((k & 3) == 0 && k > 0 && (k >> 2) + 2 < kRowSteps) load_ell((k >> 2) + 2);
            issue(k);
        }
        float2 acc[4];
#pragma unroll
        for (int k = 0; k < kQuarters; ++k) {
            const int kn = k + kGatherDepth;
            if (kn < kQuarters) {
                if ((kn & 3) == 0 && (kn >> 2) + 2 < kRowSteps) load_ell((kn >> 2) + 2);
                issue(kn);
            }
            const int s = k >> 2;
            if ((k & 3) == 0)
#pragma unroll
                for (int i = 0; i < 4; ++i) acc[i] = make_float2(0.0f, 0.0f);
#pragma unroll
            for (int j = 0; j < 2; ++j)
                accumulate_row(static_cast<unsigned short>(
                                   __shfl_sync(0xffffffffu, ew[s & 7], (lane & ~7) + 2 * (k & 3) + j)),
                               ring[k % (kGatherDepth + 1)][j], acc);
            if ((k & 3) == 3) {
                const int r = kRowsPerWarp * warp + 4 * s + grp, v = row0 + r;
                if (overflow && v < g.n) {   // rows with more than 8 neighbours
                    const int e1 = g.nb_ptr[v + 1];
                    for (int e = g.nb_ptr[v] + kEll; e < e1; ++e)
                        accumulate_row(__bfloat16_as_ushort(__float2bfloat16_rn(g.nb_w[e])),
                                       __ldg(reinterpret_cast<const uint4*>(
                                                            h_in + static_cast<long long>(g.nb_col[e]) * kH) + chunk),
                                       acc);
                }
                uint4 mv = make_uint4(0, 0, 0, 0);
                if (v < g.n) {
                    mv = pack_bf16x8(acc);
                    if (TRAIN) *reinterpret_cast<uint4*>(m_out + static_cast<long long>(v) * kH + chunk * 8) = mv;
                }
                *reinterpret_cast<uint4*>(tile + kTile * 128 + sw128(r, chunk)) = mv;
            }
        }
        fence_proxy_async_smem();
        ok = wait_phase(bar_h, iter & 1);
        h_pending = !ok;
        tmem_fence_before_sync();
        if (!__syncthreads_and(ok)) break;
        // ---- Y = [h | m] Wl^T
        if (threadIdx.x == 0) {
            tmem_fence_after_sync();
#pragma unroll
            for (int k = 0; k < 4; ++k)
                umma_bf16(tmem, umma_desc_sw128(a0 + 32 * k), umma_desc_sw128(b0 + 32 * k), idesc, k > 0);
#pragma unroll
            for (int k = 0; k < 4; ++k)
                umma_bf16(tmem, umma_desc_sw128(a1 + 32 * k), umma_desc_sw128(b1 + 32 * k), idesc, true);
            umma_commit(bar);
        }
        ok = wait_phase(bar, mma_waits++ & 1);
        tmem_fence_after_sync();
        if (!__syncthreads_and(ok)) break;
        // ---- epilogue: row = tile row 32*(warp % 4) + lane (the warp's TMEM
        // lane quarter); with 8 warps each thread takes one half of the row.
        const int quad = warp & 3, r = 32 * quad + lane, v = row0 + r;
#pragma unroll
        for (int hh = 0; hh < kEpiHalves; ++hh) {
            const int half = kFwdWarps == 8 ? (warp >> 2) : hh;
            std::uint32_t mask = 0;
            float y[16];
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) {
                const int c8 = half * 4 + c4;
                if ((c4 & 1) == 0) tmem_ld16(tmem + (static_cast<std::uint32_t>(32 * quad) << 16) + 8 * c8, y);
                uint4* cell = reinterpret_cast<uint4*>(tile + sw128(r, c8));
                float hf[8];
                bf16x8_to_f32(*cell, hf);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float yv = y[(c4 & 1) * 8 + i];
                    if (yv > 0.0f) mask |= 1u << (c4 * 8 + i);
                    hf[i] += fmaxf(yv, 0.0f);
                }
                // The new rows replace the old ones in A0 (each thread its own
                // row and chunks): the operand of the decoder's MMA, or the
                // source of one TMA store.
                *cell = f32_to_bf16x8(hf);
            }
            if (TRAIN && v < g.n) reinterpret_cast<std::uint32_t*>(mask_out + v)[half] = mask;
        }
        fence_proxy_async_smem();
        if constexpr (DECODE) {
            // out = q + rms(q) (h Wd^T): four K=16 MMAs into TMEM columns 64..79.
            tmem_fence_before_sync();
            __syncthreads();
            if (threadIdx.x == 0) {
                tmem_fence_after_sync();
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    umma_bf16(tmem + kH, umma_desc_sw128(a0 + 32 * k), umma_desc_sw128(wdt + 32 * k), idesc_dec, k > 0);
                umma_commit(bar);
            }
            ok = wait_phase(bar, mma_waits++ & 1);
            tmem_fence_after_sync();
            if (!__syncthreads_and(ok)) break;
            float y[kDecodeRows];
            if (warp < 4) tmem_ld16(tmem + (static_cast<std::uint32_t>(32 * quad) << 16) + kH, y);
            if (warp < 4 && v < g.n) {
                const long long o0 = static_cast<long long>(v) * g.bs;
#pragma unroll
                for (int c = 0; c < 8; ++c)
                    if (c < g.bs) dec.out[o0 + c] = static_cast<O>(dec_live ? fmaf(dec_scale, y[c], dec.q[o0 + c]) : 0.0f);
            }
        }
        tmem_fence_before_sync();
        __syncthreads();
        // A0 is free once the store has read it: the next tile's own rows.
        if (threadIdx.x == 0) {
            if (!DECODE) {
                tma_store_2d(&tmap_out, a0, 0, row0);
                bulk_wait_read();
            }
            fence_proxy_async_smem();
            stage_tile(t + static_cast<int>(gridDim.x));
        }
        h_pending = t + static_cast<int>(gridDim.x) < ntiles;
    }
    if (!ok && threadIdx.x == 0) {
        atomicOr(status, kErrTimeout);
        if (h_pending) wait_phase(bar_h, iter & 1);   // let an own-row copy in flight land
    }
    if (!DECODE && threadIdx.x == 0) bulk_wait_all();
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, kCols);
}

// ---------------------------------------------------------------- fused first layer
// Inference, block size <= 4: the encoder folded into the first layer.  Both
// are linear up to the first ReLU, so with x_v = [r_v / rms(r), q_v / rms(q)]
// (2 bs <= 8 nonzero inputs) and s_v = sum_u w_vu x_u,
//   h0_v = x_v We^T,   Y1_v = [h0_v | sum_u w_vu h0_u] Wl1^T
//        = x_v (Wl1_h We)^T + s_v (Wl1_m We)^T,   h1_v = h0_v + relu(Y1_v).
// k_gnn_first_weights folds the weights into one BF16 operand B1 (N = 128,
// K = 16): rows 0-63 [Wl1_h We | Wl1_m We] (Y1), rows 64-127 [We | 0] (h0).
// The layer then gathers the neighbours' 32-byte input records (FP32
// [r_u, q_u, 0...], unnormalised: the norms scale the sums afterwards)
// instead of their 128-byte feature rows, and one M=128, N=128, K=16 MMA of
// the tile's [x | s] rows gives Y1 and h0 together in TMEM.
constexpr int kFirstThreads = 128;   // a thread per tile row (its TMEM lane)
constexpr int kFirstCols = 128;      // TMEM columns: Y1 (0-63), h0 (64-127)
// B1 and two A/out tiles (alternate tiles, so a tile's store drains while
// the next is built), 16 KB each after up to 1 KB of alignment; the request
// also keeps at most four CTAs on an SM: 4 x 128 TMEM columns fill its 512.
constexpr int kFirstSmem = 1024 + 3 * kTile * 128;
static_assert(5 * kFirstSmem > 228 * 1024, "first layer: at most 4 CTAs per SM");

// rec[v] = [r_v (BS values rounded to FP32), q_v (BS), 0...] as 8 floats: a
// thread per vertex, two 16-byte stores.
template<class T, int BS>
__global__ void __launch_bounds__(256) k_gnn_records(long long n, const T* __restrict__ r,
                                                     const float* __restrict__ q, float4* __restrict__ rec)
{
    const long long v = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (v >= n) return;
    float x[8];
#pragma unroll
    for (int f = 0; f < 8; ++f) x[f] = 0.0f;
#pragma unroll
    for (int c = 0; c < BS; ++c) {
        x[c] = static_cast<float>(r[v * BS + c]);
        x[BS + c] = q[v * BS + c];
    }
    rec[2 * v] = make_float4(x[0], x[1], x[2], x[3]);
    rec[2 * v + 1] = make_float4(x[4], x[5], x[6], x[7]);
}

template<class T>
void launch_records(unsigned grid, cudaStream_t st, long long n, int bs, const T* r, const float* q, float4* rec)
{
    switch (bs) {
    case 1: k_gnn_records<T, 1><<<grid, 256, 0, st>>>(n, r, q, rec); break;
    case 2: k_gnn_records<T, 2><<<grid, 256, 0, st>>>(n, r, q, rec); break;
    case 3: k_gnn_records<T, 3><<<grid, 256, 0, st>>>(n, r, q, rec); break;
    default: k_gnn_records<T, 4><<<grid, 256, 0, st>>>(n, r, q, rec); break;
    }
}

// B1 (128 rows of 16 BF16, K-major) from the FP32 master weights; each sum
// in FP32 over k in ascending order.
__global__ void k_gnn_first_weights(const float* __restrict__ we, const float* __restrict__ wl1, bf16* __restrict__ b1)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;    // over 128 * 16
    if (i >= 2 * kH * 16) return;
    const int row = i >> 4, j = i & 15;
    float v = 0.0f;
    if (row < kH) {
        const int f = j & 7, half = j >> 3;   // half 0: Wl1_h We, half 1: Wl1_m We
        for (int k = 0; k < kH; ++k) v = fmaf(wl1[row * 2 * kH + half * kH + k], we[k * kF + f], v);
    } else if (j < 8) {
        v = we[(row - kH) * kF + j];
    }
    b1[i] = __float2bfloat16_rn(v);
}

__global__ void __launch_bounds__(kFirstThreads, 4)
    k_gnn_first_layer(GraphArgs g, const __grid_constant__ CUtensorMap tmap_out, const float4* __restrict__ rec,
                      const double* norms, const bf16* __restrict__ b1, unsigned* status)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) std::uint64_t bar_storage[1];
    __shared__ std::uint32_t tmem_base_s;
    const std::uint32_t raw = smem_u32(smem_raw), base = align1024(raw);
    unsigned char* tiles = smem_raw + (base - raw);   // B1, then A0 and A1 (rows [x | s], then output rows)
    const std::uint32_t b = base;
    const std::uint32_t bar = smem_u32(&bar_storage[0]);
    const int warp = threadIdx.x >> 5, r = threadIdx.x;
    const int ntiles = (g.n + kTile - 1) / kTile;

    // B1: two 16-byte chunks per row into the swizzled block.
    for (int i = threadIdx.x; i < 2 * kH * 2; i += kFirstThreads)
        *reinterpret_cast<uint4*>(tiles + sw128(i >> 1, i & 1)) = reinterpret_cast<const uint4*>(b1)[i];
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_proxy_async_smem();
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base_s), kFirstCols);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const std::uint32_t tmem = tmem_base_s;
    constexpr std::uint32_t idesc = umma_idesc_bf16(kTile, 2 * kH);
    const double root = sqrt(static_cast<double>(g.n) * g.bs), nr = norms[0], nq = norms[2];
    const float inv_r = nr > 0.0 ? static_cast<float>(root / nr) : 0.0f;
    const float inv_q = nq > 0.0 ? static_cast<float>(root / nq) : 0.0f;
    const int bs = g.bs;
    const auto fma_record = [](float w, const float4& lo, const float4& hi, float (&s)[8]) {
        s[0] = fmaf(w, lo.x, s[0]);
        s[1] = fmaf(w, lo.y, s[1]);
        s[2] = fmaf(w, lo.z, s[2]);
        s[3] = fmaf(w, lo.w, s[3]);
        s[4] = fmaf(w, hi.x, s[4]);
        s[5] = fmaf(w, hi.y, s[5]);
        s[6] = fmaf(w, hi.z, s[6]);
        s[7] = fmaf(w, hi.w, s[7]);
    };
    // A row's 8 slots (columns, BF16 weights) and its own record, loaded one
    // tile ahead of their use.
    int4 c0 = make_int4(-1, -1, -1, -1), c1 = c0;
    uint4 wv = make_uint4(0, 0, 0, 0);
    float4 own0 = make_float4(0.0f, 0.0f, 0.0f, 0.0f), own1 = own0;
    const auto load_row = [&](int t) {
        const int v = t * kTile + r;
        if (t < ntiles && v < g.n) {
            c0 = __ldg(reinterpret_cast<const int4*>(g.ell_col) + 2ll * v);
            c1 = __ldg(reinterpret_cast<const int4*>(g.ell_col) + 2ll * v + 1);
            wv = __ldg(reinterpret_cast<const uint4*>(g.ell_w) + v);
            own0 = __ldg(rec + 2ll * v);
            own1 = __ldg(rec + 2ll * v + 1);
        }
    };
    load_row(blockIdx.x);
    std::uint32_t phase = 0;
    bool ok = true;
    int buf = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, buf ^= 1) {
        const int row0 = t * kTile, v = row0 + r;
        const std::uint32_t a = base + static_cast<std::uint32_t>(1 + buf) * kTile * 128;
        unsigned char* tile = tiles + (1 + buf) * kTile * 128;
        float x[8], s[8];
#pragma unroll
        for (int f = 0; f < 8; ++f) x[f] = s[f] = 0.0f;
        if (v < g.n) {
            // All eight neighbour records before the sums (slot order,
            // padding slots skipped), then the next tile's row data.
            const int col[8] = {c0.x, c0.y, c0.z, c0.w, c1.x, c1.y, c1.z, c1.w};
            const std::uint32_t wp[4] = {wv.x, wv.y, wv.z, wv.w};
            const float own[8] = {own0.x, own0.y, own0.z, own0.w, own1.x, own1.y, own1.z, own1.w};
            float4 lo[8], hi[8];
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                lo[j] = hi[j] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
                if (col[j] >= 0) {
                    lo[j] = __ldg(rec + 2ll * col[j]);
                    hi[j] = __ldg(rec + 2ll * col[j] + 1);
                }
            }
            load_row(t + static_cast<int>(gridDim.x));
#pragma unroll
            for (int j = 0; j < 8; ++j)
                if (col[j] >= 0)
                    fma_record(__uint_as_float((j & 1 ? wp[j >> 1] >> 16 : wp[j >> 1] & 0xffffu) << 16), lo[j], hi[j],
                               s);
            if (g.tile_ovf[t]) {   // more than 8 neighbours: the rest in CSR order
                const int e1 = g.nb_ptr[v + 1];
                for (int e = g.nb_ptr[v] + kEll; e < e1; ++e) {
                    const int u = g.nb_col[e];
                    fma_record(bf16_round(g.nb_w[e]), __ldg(rec + 2ll * u), __ldg(rec + 2ll * u + 1), s);
                }
            }
#pragma unroll
            for (int f = 0; f < 8; ++f) {
                const float sc = f < bs ? inv_r : (f < 2 * bs ? inv_q : 0.0f);
                x[f] = own[f] * sc;
                s[f] *= sc;
            }
        } else {
            load_row(t + static_cast<int>(gridDim.x));
        }
        *reinterpret_cast<uint4*>(tile + sw128(r, 0)) = f32_to_bf16x8(x);
        *reinterpret_cast<uint4*>(tile + sw128(r, 1)) = f32_to_bf16x8(s);
        fence_proxy_async_smem();
        tmem_fence_before_sync();
        __syncthreads();
        // ---- [Y1 | h0] = [x | s] B1^T
        if (threadIdx.x == 0) {
            tmem_fence_after_sync();
            umma_bf16(tmem, umma_desc_sw128(a), umma_desc_sw128(b), idesc, false);
            umma_commit(bar);
        }
        ok = wait_phase(bar, phase);
        phase ^= 1;
        tmem_fence_after_sync();
        if (!__syncthreads_and(ok)) break;
        // ---- epilogue: h1 = h0 + relu(Y1) over the tile's row r (TMEM lane r)
        const std::uint32_t trow = tmem + (static_cast<std::uint32_t>(32 * warp) << 16);
#pragma unroll
        for (int c16 = 0; c16 < 4; ++c16) {
            float y[16], h[16];
            tmem_ld16(trow + 16 * c16, y);
            tmem_ld16(trow + kH + 16 * c16, h);
#pragma unroll
            for (int half = 0; half < 2; ++half) {
                float o[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) o[i] = h[8 * half + i] + fmaxf(y[8 * half + i], 0.0f);
                *reinterpret_cast<uint4*>(tile + sw128(r, 2 * c16 + half)) = f32_to_bf16x8(o);
            }
        }
        fence_proxy_async_smem();
        tmem_fence_before_sync();
        __syncthreads();
        // Store this tile; the other buffer, written next, is free once the
        // store before this one has read it.
        if (threadIdx.x == 0) {
            tma_store_2d(&tmap_out, a, 0, row0);
            bulk_wait_read_all_but_one();
        }
        __syncthreads();
    }
    if (!ok && threadIdx.x == 0) atomicOr(status, kErrTimeout);
    if (threadIdx.x == 0) bulk_wait_all();
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, kFirstCols);
}

// ---------------------------------------------------------------- TMA-fed layer
// The same layer, warp-specialised.  A producer warp streams, per 16-row
// sub-tile, the neighbours' feature rows with TMA gathers (tile::gather4, box
// one row high) into a 3-stage shared-memory ring together with the rows'
// gather plan entries and edge weights (bulk copies), and per 128-row tile the
// tile's own rows with one 2D TMA load whose 128-byte swizzle is exactly the
// K-major operand layout of the MMA.  The four consumer warps aggregate m from
// shared memory (no global loads on the common path), write the swizzled m
// block, run the eight MMAs and the epilogue.  Rows whose neighbours do not fit
// a sub-tile's 128 slots are gathered from global memory by the consumers.
constexpr int kSubRows = 16;                     // rows per gather sub-tile
constexpr int kSubsPerTile = kTile / kSubRows;   // 8
constexpr int kSlots = 128;                      // staged neighbour rows per sub-tile
constexpr int kGStages = 3;
constexpr int kSubWeights = 512;                 // staged edge weights per sub-tile
constexpr int kTmaThreads = 160;                 // 4 consumer warps + 1 producer warp
constexpr int kStageSlots = kSlots * 128;                        // 16 KB
constexpr int kStageMeta = kStageSlots;                          // 16 int4 = 256 B
constexpr int kStageHead = kStageMeta + 256;                     // woff, wavail, nq
constexpr int kStageW = kStageHead + 64;                         // weights
constexpr int kStageBytes = (kStageW + kSubWeights * 4 + 16 + 1023) / 1024 * 1024;
constexpr int kTmaSmem = 1024 + 2 * kTile * 128 + 2 * kH * 128 + kGStages * kStageBytes;

template<bool TRAIN>
__global__ void __launch_bounds__(kTmaThreads, 2)
    k_gnn_layer_tma(GraphArgs g, const __grid_constant__ CUtensorMap gmap, const __grid_constant__ CUtensorMap tmap,
                    const bf16* __restrict__ h_in, const bf16* __restrict__ wl, bf16* __restrict__ h_out,
                    bf16* __restrict__ m_out, unsigned long long* __restrict__ mask_out, const int4* __restrict__ quads,
                    const int* __restrict__ quad_ptr, const int4* __restrict__ metas, int edges, unsigned* status)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) std::uint64_t bars[2 * kGStages + 3];   // full, empty, a_full, a_free, mma
    __shared__ std::uint32_t tmem_base_s;
    const std::uint32_t raw = smem_u32(smem_raw), base = align1024(raw);
    unsigned char* sm = smem_raw + (base - raw);
    const std::uint32_t a0 = base, a1 = base + kTile * 128, b0 = base + 2 * kTile * 128, b1 = b0 + kH * 128;
    const std::uint32_t st0 = b0 + 2 * kH * 128;
    unsigned char* stg = sm + (st0 - base);
    const std::uint32_t bar0 = smem_u32(bars);
    const auto full = [&](int s) { return bar0 + 8 * s; };
    const auto empty = [&](int s) { return bar0 + 8 * (kGStages + s); };
    const std::uint32_t a_full = bar0 + 8 * (2 * kGStages), a_free = a_full + 8, mma_bar = a_full + 16;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (g.n + kTile - 1) / kTile;

    // Layer weight into the two B blocks.
    for (int i = threadIdx.x; i < kH * 16; i += kTmaThreads) {
        const int r = i >> 4, c16 = i & 15;
        *reinterpret_cast<uint4*>(sm + 2 * kTile * 128 + (c16 >> 3) * kH * 128 + sw128(r, c16 & 7)) =
            *reinterpret_cast<const uint4*>(wl + r * 128 + c16 * 8);
    }
    if (threadIdx.x == 0) {
        for (int s = 0; s < kGStages; ++s) {
            mbar_init(full(s), 1);
            mbar_init(empty(s), 4);
        }
        mbar_init(a_full, 1);
        mbar_init(a_free, 1);
        mbar_init(mma_bar, 1);
        fence_proxy_async_smem();
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base_s), kH);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const std::uint32_t tmem = tmem_base_s;

    if (warp == 4) {
        // ------------------------------------------------------------ producer
        const std::uint64_t policy = l2_policy_evict_normal();
        int gsub = 0, it = 0;
        bool ok = true;
        for (int t = blockIdx.x; t < ntiles && ok; t += gridDim.x, ++it) {
            const int row0 = t * kTile;
            // The tile's plan in one round of loads: lane s < 9 holds sub-tile
            // s's first quad and first edge; lane q holds quad q of each
            // sub-tile (at most 32 per sub-tile).
            int my_q = 0, my_e = 0;
            if (lane <= kSubsPerTile) {
                const int sub = min(t * kSubsPerTile + lane, (g.n + kSubRows - 1) / kSubRows);
                my_q = quad_ptr[sub];
                my_e = g.nb_ptr[min(row0 + lane * kSubRows, g.n)];
            }
            int4 myquad[kSubsPerTile];
            int qs[kSubsPerTile + 1], es[kSubsPerTile + 1];
#pragma unroll
            for (int s = 0; s <= kSubsPerTile; ++s) {
                qs[s] = __shfl_sync(0xffffffffu, my_q, s);
                es[s] = __shfl_sync(0xffffffffu, my_e, s);
            }
#pragma unroll
            for (int s = 0; s < kSubsPerTile; ++s) {
                myquad[s] = make_int4(0, 0, 0, 0);
                if (lane < qs[s + 1] - qs[s]) myquad[s] = quads[qs[s] + lane];
            }
#pragma unroll
            for (int s = 0; s < kSubsPerTile; ++s, ++gsub) {
                if (!ok) break;
                const int st = gsub % kGStages, use = gsub / kGStages;
                const int sub = t * kSubsPerTile + s;
                const int r0 = row0 + s * kSubRows;
                unsigned char* sp = stg + st * kStageBytes;
                const std::uint32_t sb = st0 + st * kStageBytes;
                const int nq = r0 < g.n ? qs[s + 1] - qs[s] : 0;
                int good = 1;
                if (lane == 0) {
                    if (!mbar_wait_bounded(empty(st), (use & 1) ^ 1, kMmaSpin)) {
                        good = 0;
                    } else if (r0 >= g.n) {
                        mbar_arrive(full(st));
                    } else {
                        const int e_first = es[s], e_last = es[s + 1];
                        std::size_t lo = 0;
                        int woff = 0, wavail = 0;
                        std::uint32_t wb = bulk_segment(e_first, e_last, edges, 4, lo, woff, wavail);
                        if (wb > static_cast<std::uint32_t>(kSubWeights * 4 + 16)) {   // keep within the stage
                            wb = 0;
                            wavail = 0;
                        }
                        int* head = reinterpret_cast<int*>(sp + kStageHead);
                        head[0] = woff;
                        head[1] = wavail;
                        head[2] = e_first;
                        mbar_arrive_expect_tx(full(st), static_cast<std::uint32_t>(nq) * 512u + 256u + wb);
                        bulk_load(sb + kStageMeta, metas + static_cast<std::size_t>(sub) * kSubRows, 256, full(st),
                                  policy);
                        if (wb) bulk_load(sb + kStageW, reinterpret_cast<const unsigned char*>(g.nb_w) + lo, wb, full(st),
                                          policy);
                    }
                }
                good = __shfl_sync(0xffffffffu, good, 0);
                if (!good) {
                    atomicOr(status, kErrTimeout);
                    ok = false;
                    break;
                }
                if (lane < nq) {
                    const int4 q = myquad[s];
                    tma_gather4(sb + lane * 512, &gmap, 0, q.x, q.y, q.z, q.w, full(st), policy);
                }
                __syncwarp();
            }
            if (!ok) break;
            // The tile's own rows (swizzled) once the previous tile's epilogue is done.
            if (lane == 0) {
                if (it > 0 && !mbar_wait_bounded(a_free, (it - 1) & 1, kMmaSpin)) {
                    atomicOr(status, kErrTimeout);
                    ok = false;
                } else {
                    mbar_arrive_expect_tx(a_full, kTile * 128);
                    tma_load_2d(a0, &tmap, 0, row0, a_full);
                }
            }
            ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
        }
        // Leave after the last copies landed.
        if (lane == 0) {
            for (int k = max(0, gsub - kGStages); k < gsub; ++k)
                mbar_wait_bounded(full(k % kGStages), (k / kGStages) & 1, kMmaSpin);
            if (it > 0) mbar_wait_bounded(a_full, (it - 1) & 1, kMmaSpin);
        }
        return;
    }

    // ---------------------------------------------------------------- consumers
    constexpr std::uint32_t idesc = umma_idesc_bf16(kTile, kH);
    const int grp = lane >> 3, chunk = lane & 7;
    int gsub = 0, it = 0;
    bool failed = false;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
        const int row0 = t * kTile;
        for (int s = 0; s < kSubsPerTile; ++s, ++gsub) {
            const int st = gsub % kGStages, use = gsub / kGStages;
            const unsigned char* sp = stg + st * kStageBytes;
            const bool ready = !failed && __all_sync(0xffffffffu, mbar_wait_bounded(full(st), use & 1, kMmaSpin));
            failed = failed || !ready;
            const int rl = 4 * warp + grp;                 // row within the sub-tile
            const int r = s * kSubRows + rl, v = row0 + r;
            uint4 mv = make_uint4(0, 0, 0, 0);
            if (ready && v < g.n) {
                const int4 meta = reinterpret_cast<const int4*>(sp + kStageMeta)[rl];
                const int* head = reinterpret_cast<const int*>(sp + kStageHead);
                const int woff = head[0], wavail = head[1], e_first = head[2];
                const float* sw = reinterpret_cast<const float*>(sp + kStageW);
                float acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
                for (int k = 0; k < meta.y; ++k) {
                    const int wi = meta.z + k;
                    const float w = bf16_round(wi < wavail ? sw[woff + wi] : g.nb_w[e_first + wi]);
                    uint4 u;
                    if (meta.x >= 0) u = *reinterpret_cast<const uint4*>(sp + (meta.x + k) * 128 + chunk * 16);
                    else u = *reinterpret_cast<const uint4*>(h_in + static_cast<long long>(g.nb_col[e_first + wi]) * kH
                                                             + chunk * 8);
                    float f[8];
                    bf16x8_to_f32(u, f);
#pragma unroll
                    for (int i = 0; i < 8; ++i) acc[i] = fmaf(w, f[i], acc[i]);
                }
                mv = f32_to_bf16x8(acc);
                if (TRAIN) *reinterpret_cast<uint4*>(m_out + static_cast<long long>(v) * kH + chunk * 8) = mv;
            }
            *reinterpret_cast<uint4*>(sm + kTile * 128 + sw128(r, chunk)) = mv;
            __syncwarp();
            if (lane == 0) mbar_arrive(empty(st));
        }
        fence_proxy_async_smem();
        tmem_fence_before_sync();
        if (bar_any(1, 128, failed)) {
            failed = true;
            break;
        }
        if (threadIdx.x == 0) {
            bool aok = mbar_wait_bounded(a_full, it & 1, kMmaSpin);
            if (aok) {
                tmem_fence_after_sync();
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    umma_bf16(tmem, umma_desc_sw128(a0 + 32 * k), umma_desc_sw128(b0 + 32 * k), idesc, k > 0);
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    umma_bf16(tmem, umma_desc_sw128(a1 + 32 * k), umma_desc_sw128(b1 + 32 * k), idesc, true);
                umma_commit(mma_bar);
            } else {
                atomicOr(status, kErrTimeout);
                mbar_arrive(mma_bar);
            }
        }
        const bool mok = mbar_wait_bounded(mma_bar, it & 1, kMmaSpin);
        tmem_fence_after_sync();
        if (bar_any(1, 128, !mok)) {
            failed = true;
            break;
        }
        // Epilogue: row = 32*warp + lane; h_old from the swizzled A0 block.
        const int r = 32 * warp + lane, v = row0 + r;
        unsigned long long mask = 0;
        uint4 outv[8];
#pragma unroll
        for (int half = 0; half < 2; ++half) {
            float y[32];
            tmem_ld32(tmem + (static_cast<std::uint32_t>(32 * warp) << 16) + 32 * half, y);
#pragma unroll
            for (int c4 = 0; c4 < 4; ++c4) {
                const int c8 = half * 4 + c4;
                float hf[8];
                bf16x8_to_f32(*reinterpret_cast<const uint4*>(sm + sw128(r, c8)), hf);
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float yv = y[c4 * 8 + i];
                    if (yv > 0.0f) mask |= 1ull << (c8 * 8 + i);
                    hf[i] += fmaxf(yv, 0.0f);
                }
                outv[c8] = f32_to_bf16x8(hf);
            }
        }
        if (v < g.n) {
            uint4* o = reinterpret_cast<uint4*>(h_out + static_cast<long long>(v) * kH);
#pragma unroll
            for (int c8 = 0; c8 < 8; ++c8) o[c8] = outv[c8];
            if (TRAIN) mask_out[v] = mask;
        }
        tmem_fence_before_sync();
        asm volatile("bar.sync 1, 128;" ::: "memory");
        if (threadIdx.x == 0) mbar_arrive(a_free);
    }
    if (failed && threadIdx.x == 0) atomicOr(status, kErrTimeout);
    tmem_fence_before_sync();
    asm volatile("bar.sync 1, 128;" ::: "memory");
    if (warp == 0) tmem_free(tmem, kH);
}

// ---------------------------------------------------------------- backward kernels
// Loss  we ||out - e||^2 / ||e||^2 + wr ||r - A out||^2 / ||r||^2  (partials
// per block, combined in block order by the last block) and
// dz = s * (2 we (out - e) / ||e||^2 - 2 wr A^T (r - A out) / ||r||^2), where
// res = r - A out and g = A^T res are precomputed.
__global__ void __launch_bounds__(256) k_gnn_out_grad(long long count, const float* __restrict__ out,
                                                      const double* __restrict__ e, const float* __restrict__ res,
                                                      const float* __restrict__ g, const double* enorm,
                                                      const double* norms, double scale_n, double we, double wr,
                                                      float* __restrict__ dz, double* partials, unsigned* ticket,
                                                      double* loss)
{
    const double ee = (*enorm) * (*enorm), rr = norms[0] * norms[0];
    const double s = norms[2] / scale_n;   // rms of the Jacobi step
    const float ge = ee > 0.0 ? static_cast<float>(2.0 * we * s / ee) : 0.0f;
    const float gr = rr > 0.0 ? static_cast<float>(2.0 * wr * s / rr) : 0.0f;
    double acc_e = 0.0, acc_r = 0.0;
    for (long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x; i < count;
         i += static_cast<long long>(gridDim.x) * blockDim.x) {
        const double d = static_cast<double>(out[i]) - e[i];
        acc_e += d * d;
        acc_r += static_cast<double>(res[i]) * res[i];
        dz[i] = ge * static_cast<float>(d) - gr * g[i];
    }
    acc_e = warp_sum(acc_e);
    acc_r = warp_sum(acc_r);
    __shared__ double red[2][8];
    if ((threadIdx.x & 31) == 0) {
        red[0][threadIdx.x >> 5] = acc_e;
        red[1][threadIdx.x >> 5] = acc_r;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double be = 0.0, br = 0.0;
        for (int w = 0; w < 8; ++w) {
            be += red[0][w];
            br += red[1][w];
        }
        partials[2 * blockIdx.x] = be;
        partials[2 * blockIdx.x + 1] = br;
        __threadfence();
        if (atomicAdd(ticket, 1u) == gridDim.x - 1) {
            __threadfence();
            double te = 0.0, tr = 0.0;
            for (unsigned k = 0; k < gridDim.x; ++k) {
                te += __ldcg(partials + 2 * k);
                tr += __ldcg(partials + 2 * k + 1);
            }
            *loss = (ee > 0.0 ? we * te / ee : 0.0) + (rr > 0.0 ? wr * tr / rr : 0.0);
            *ticket = 0;
        }
    }
}

__global__ void k_gnn_residual(long long count, const double* __restrict__ r, const float* __restrict__ ax,
                               float* __restrict__ res)
{
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) res[i] = static_cast<float>(r[i] - static_cast<double>(ax[i]));
}

// dh4 = dz Wd (FP32 rows of 64).
__global__ void __launch_bounds__(256) k_gnn_decode_bwd(int n, int bs, const float* __restrict__ dz,
                                                        const float* __restrict__ wd, float* __restrict__ dh)
{
    __shared__ float w[8 * kH];
    for (int i = threadIdx.x; i < 8 * kH; i += blockDim.x) w[i] = wd[i];
    __syncthreads();
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    float d[8];
    for (int c = 0; c < 8; ++c) d[c] = c < bs ? dz[static_cast<long long>(v) * bs + c] : 0.0f;
    float4* o = reinterpret_cast<float4*>(dh + static_cast<long long>(v) * kH);
#pragma unroll
    for (int k4 = 0; k4 < kH / 4; ++k4) {
        float r[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            float acc = 0.0f;
            for (int c = 0; c < bs; ++c) acc = fmaf(d[c], w[c * kH + k4 * 4 + i], acc);
            r[i] = acc;
        }
        o[k4] = make_float4(r[0], r[1], r[2], r[3]);
    }
}

// Per-block partials of G[i][j] = sum_v a[v][i] * b[v][j] (a: FP32 rows of pa,
// b: rows of pb in BF16 or FP32), i < pa, j < pb, pa * pb <= 1024; rows split
// into contiguous block ranges, summed in row order.
template<class B>
__global__ void __launch_bounds__(256) k_gnn_outer(int n, int pa, int pb, const float* __restrict__ a,
                                                   const B* __restrict__ b, float* __restrict__ partials)
{
    const int rows = (n + gridDim.x - 1) / gridDim.x;
    const int v0 = blockIdx.x * rows, v1 = min(n, v0 + rows);
    for (int t = threadIdx.x; t < pa * pb; t += blockDim.x) {
        const int i = t / pb, j = t - i * pb;
        float acc = 0.0f;
        for (int v = v0; v < v1; ++v)
            acc = fmaf(a[static_cast<long long>(v) * pa + i], static_cast<float>(b[static_cast<long long>(v) * pb + j]),
                       acc);
        partials[static_cast<long long>(blockIdx.x) * pa * pb + t] = acc;
    }
}

// Sum `blocks` partial arrays of `count` floats in block order into out[]
// (optionally transposed: out[j * rows + i] for element i * cols + j).
__global__ void k_gnn_reduce(int blocks, int count, const float* __restrict__ partials, float* __restrict__ out,
                             int rows, int cols, int transpose)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= count) return;
    float acc = 0.0f;
    for (int b = 0; b < blocks; ++b) acc += partials[static_cast<long long>(b) * count + t];
    if (transpose) {
        const int i = t / cols, j = t - i * cols;
        out[j * rows + i] = acc;
    } else {
        out[t] = acc;
    }
}

// Layer backward, part 1 (tensor cores): dy = dh (.) [y > 0] (kept in BF16
// for the weight gradient), dcat = dy Wl (128 x 128 per tile, K = 64), then
// dh += dcat[:, :64] in place and dm = dcat[:, 64:].
constexpr int kBwdSmem = 1024 + kTile * 128 + 2 * kH * 128;

__global__ void __launch_bounds__(kLayerThreads, 4)
    k_gnn_layer_bwd(int n, float* __restrict__ dh, const unsigned long long* __restrict__ mask,
                    const bf16* __restrict__ wlt, bf16* __restrict__ dy_out, float* __restrict__ dm, unsigned* status)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) std::uint64_t bar_storage;
    __shared__ std::uint32_t tmem_base_s;
    const std::uint32_t raw = smem_u32(smem_raw), base = align1024(raw);
    unsigned char* tile = smem_raw + (base - raw);     // A: dy (128 x 64), B: Wl^T (128 x 64)
    const std::uint32_t a0 = base, b0 = base + kTile * 128;
    const std::uint32_t bar = smem_u32(&bar_storage);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (n + kTile - 1) / kTile;
    for (int i = threadIdx.x; i < 2 * kH * 8; i += kLayerThreads) {
        const int r = i >> 3, c = i & 7;
        *reinterpret_cast<uint4*>(tile + kTile * 128 + sw128(r, c)) =
            *reinterpret_cast<const uint4*>(wlt + r * kH + c * 8);
    }
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_proxy_async_smem();
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base_s), 2 * kH);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const std::uint32_t tmem = tmem_base_s;
    constexpr std::uint32_t idesc = umma_idesc_bf16(kTile, 2 * kH);
    int iter = 0;
    bool ok = true;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++iter) {
        const int row0 = t * kTile;
        // dy tile: thread handles (row, chunk) pairs.
        for (int i = threadIdx.x; i < kTile * 8; i += kLayerThreads) {
            const int r = i >> 3, c = i & 7, v = row0 + r;
            float f[8] = {0, 0, 0, 0, 0, 0, 0, 0};
            if (v < n) {
                const unsigned long long mk = mask[v];
                const float4* src = reinterpret_cast<const float4*>(dh + static_cast<long long>(v) * kH + c * 8);
                const float4 p = src[0], q = src[1];
                const float x[8] = {p.x, p.y, p.z, p.w, q.x, q.y, q.z, q.w};
#pragma unroll
                for (int k = 0; k < 8; ++k) f[k] = ((mk >> (c * 8 + k)) & 1ull) ? x[k] : 0.0f;
            }
            const uint4 u = f32_to_bf16x8(f);
            *reinterpret_cast<uint4*>(tile + sw128(r, c)) = u;
            if (v < n) *reinterpret_cast<uint4*>(dy_out + static_cast<long long>(v) * kH + c * 8) = u;
        }
        fence_proxy_async_smem();
        tmem_fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0) {
            tmem_fence_after_sync();
#pragma unroll
            for (int k = 0; k < 4; ++k)
                umma_bf16(tmem, umma_desc_sw128(a0 + 32 * k), umma_desc_sw128(b0 + 32 * k), idesc, k > 0);
            umma_commit(bar);
        }
        ok = wait_phase(bar, iter & 1);
        tmem_fence_after_sync();
        if (!__syncthreads_and(ok)) break;
        const int v = row0 + 32 * warp + lane;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            float y[32];
            tmem_ld32(tmem + (static_cast<std::uint32_t>(32 * warp) << 16) + 32 * q, y);
            if (v < n) {
                float* dst = q < 2 ? dh + static_cast<long long>(v) * kH + 32 * q
                                   : dm + static_cast<long long>(v) * kH + 32 * (q - 2);
#pragma unroll
                for (int i = 0; i < 32; ++i) dst[i] = q < 2 ? dst[i] + y[i] : y[i];
            }
        }
        tmem_fence_before_sync();
        __syncthreads();
    }
    if (!ok && threadIdx.x == 0) atomicOr(status, kErrTimeout);
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, 2 * kH);
}

// Layer backward, part 2: dh_u += sum over edges (v -> u) of w_vu dm_v, a
// gather over the transposed graph (deterministic).
__global__ void __launch_bounds__(256) k_gnn_agg_t(GraphArgs g, const float* __restrict__ dm, float* __restrict__ dh)
{
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    const int u = static_cast<int>(t >> 4), c4 = static_cast<int>(t & 15);
    if (u >= g.n) return;
    float4 acc = reinterpret_cast<const float4*>(dh + static_cast<long long>(u) * kH)[c4];
    for (int k = g.tr_ptr[u]; k < g.tr_ptr[u + 1]; ++k) {
        const float w = g.tr_w[k];
        const float4 d = reinterpret_cast<const float4*>(dm + static_cast<long long>(g.tr_col[k]) * kH)[c4];
        acc.x = fmaf(w, d.x, acc.x);
        acc.y = fmaf(w, d.y, acc.y);
        acc.z = fmaf(w, d.z, acc.z);
        acc.w = fmaf(w, d.w, acc.w);
    }
    reinterpret_cast<float4*>(dh + static_cast<long long>(u) * kH)[c4] = acc;
}

// Layer weight gradient on the tensor cores: dWl^T (128 x 64) = [h | m]^T dy,
// K = vertices.  Each CTA accumulates its tiles in TMEM (operands transposed
// into K-major shared tiles) and writes one FP32 partial; k_gnn_reduce sums
// the partials in CTA order.
constexpr int kWgradSmem = 1024 + 2 * kTile * 128 + 2 * kH * 128;

__global__ void __launch_bounds__(kLayerThreads, 4)
    k_gnn_wgrad(int n, const bf16* __restrict__ h, const bf16* __restrict__ m, const bf16* __restrict__ dy,
                float* __restrict__ partials, unsigned* status)
{
    extern __shared__ unsigned char smem_raw[];
    __shared__ __align__(8) std::uint64_t bar_storage;
    __shared__ std::uint32_t tmem_base_s;
    const std::uint32_t raw = smem_u32(smem_raw), base = align1024(raw);
    unsigned char* tile = smem_raw + (base - raw);
    // A: 128 feature rows x 128 vertices (two K blocks of 64); B: 64 rows x 128.
    const std::uint32_t a0 = base, b0 = base + 2 * kTile * 128;
    const std::uint32_t bar = smem_u32(&bar_storage);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (n + kTile - 1) / kTile;
    const int t0 = static_cast<int>(static_cast<long long>(ntiles) * blockIdx.x / gridDim.x);
    const int t1 = static_cast<int>(static_cast<long long>(ntiles) * (blockIdx.x + 1) / gridDim.x);
    if (threadIdx.x == 0) {
        mbar_init(bar, 1);
        fence_proxy_async_smem();
    }
    if (warp == 0) tmem_alloc(smem_u32(&tmem_base_s), kH);
    tmem_fence_before_sync();
    __syncthreads();
    tmem_fence_after_sync();
    const std::uint32_t tmem = tmem_base_s;
    constexpr std::uint32_t idesc = umma_idesc_bf16(kTile, kH);
    bf16* sa = reinterpret_cast<bf16*>(tile);
    bf16* sb = reinterpret_cast<bf16*>(tile + 2 * kTile * 128);
    int iter = 0;
    bool ok = true;
    for (int t = t0; t < t1; ++t, ++iter) {
        const int row0 = t * kTile;
        // Transpose: vertex k of the tile becomes K index k; feature f a row.
        for (int i = threadIdx.x; i < kTile * 16; i += kLayerThreads) {
            const int k = i >> 4, c16 = i & 15, v = row0 + k;     // c16: 16-byte chunk of [h | m] (8 features)
            uint4 u = make_uint4(0, 0, 0, 0);
            if (v < n) u = *reinterpret_cast<const uint4*>((c16 < 8 ? h : m) + static_cast<long long>(v) * kH
                                                          + (c16 & 7) * 8);
            const bf16* e = reinterpret_cast<const bf16*>(&u);
            const int kb = k >> 6, kc = (k & 63) >> 3, ke = k & 7;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int f = c16 * 8 + q;
                sa[(kb * kTile * 128 + sw128(f, kc)) / 2 + ke] = e[q];
            }
        }
        for (int i = threadIdx.x; i < kTile * 8; i += kLayerThreads) {
            const int k = i >> 3, c8 = i & 7, v = row0 + k;
            uint4 u = make_uint4(0, 0, 0, 0);
            if (v < n) u = *reinterpret_cast<const uint4*>(dy + static_cast<long long>(v) * kH + c8 * 8);
            const bf16* e = reinterpret_cast<const bf16*>(&u);
            const int kb = k >> 6, kc = (k & 63) >> 3, ke = k & 7;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int o = c8 * 8 + q;
                sb[(kb * kH * 128 + sw128(o, kc)) / 2 + ke] = e[q];
            }
        }
        fence_proxy_async_smem();
        tmem_fence_before_sync();
        __syncthreads();
        if (threadIdx.x == 0) {
            tmem_fence_after_sync();
#pragma unroll
            for (int kb = 0; kb < 2; ++kb)
#pragma unroll
                for (int k = 0; k < 4; ++k)
                    umma_bf16(tmem, umma_desc_sw128(a0 + kb * kTile * 128 + 32 * k),
                              umma_desc_sw128(b0 + kb * kH * 128 + 32 * k), idesc, iter > 0 || kb > 0 || k > 0);
            umma_commit(bar);
        }
        ok = wait_phase(bar, iter & 1);
        tmem_fence_after_sync();
        if (!__syncthreads_and(ok)) break;
    }
    // Partial of this CTA (zero if it had no tiles).
    const int f = 32 * warp + lane;
    float* out = partials + static_cast<long long>(blockIdx.x) * (2 * kH) * kH + static_cast<long long>(f) * kH;
#pragma unroll
    for (int half = 0; half < 2; ++half) {
        float y[32];
        if (iter > 0 && ok) {
            tmem_ld32(tmem + (static_cast<std::uint32_t>(32 * warp) << 16) + 32 * half, y);
        } else {
#pragma unroll
            for (int i = 0; i < 32; ++i) y[i] = 0.0f;
        }
#pragma unroll
        for (int i = 0; i < 32; ++i) out[32 * half + i] = y[i];
    }
    if (!ok && threadIdx.x == 0) atomicOr(status, kErrTimeout);
    tmem_fence_before_sync();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, kH);
}

// Adam (bias-corrected) on the flat FP32 parameters; refreshes the BF16
// copies of the layer weights (Wl and Wl^T) used by the tensor cores.
__global__ void __launch_bounds__(256) k_gnn_adam(int count, float* __restrict__ p, const float* __restrict__ g,
                                                  float* __restrict__ m, float* __restrict__ v, float lr, float b1,
                                                  float b2, float eps, float c1, float c2)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

__global__ void k_gnn_pack(const float* __restrict__ wl, bf16* __restrict__ wl16, bf16* __restrict__ wlt16)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;    // over kLayers * 64 * 128
    if (i >= kLayers * kH * 2 * kH) return;
    const int l = i / (kH * 2 * kH), r = (i / (2 * kH)) % kH, c = i % (2 * kH);
    const bf16 b = __float2bfloat16_rn(wl[i]);
    wl16[i] = b;
    wlt16[l * kH * 2 * kH + c * kH + r] = b;
}

// Matrix graph: weights w_vu = -mean_c a_vu,c / d_v,c of the off-diagonal
// entries, 1 / diagonal, and FP32 copies of the coefficients (for A x and
// A^T x in the residual term of the training loss).
__global__ void k_gnn_graph(int n, int bs, const int* __restrict__ nb_ptr, const int* __restrict__ nb_entry,
                            const double* __restrict__ vals, const double* __restrict__ diag, float* __restrict__ nb_w,
                            float* __restrict__ dinv, float* __restrict__ nb_a, float* __restrict__ diag_f)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n) return;
    for (int c = 0; c < bs; ++c) {
        const double d = diag[static_cast<long long>(v) * bs + c];
        dinv[static_cast<long long>(v) * bs + c] = static_cast<float>(1.0 / d);
        diag_f[static_cast<long long>(v) * bs + c] = static_cast<float>(d);
    }
    for (int k = nb_ptr[v]; k < nb_ptr[v + 1]; ++k) {
        const long long e = nb_entry[k];
        double acc = 0.0;
        for (int c = 0; c < bs; ++c) {
            const double a = vals[e * bs + c];
            acc += a / diag[static_cast<long long>(v) * bs + c];
            nb_a[static_cast<long long>(k) * bs + c] = static_cast<float>(a);
        }
        nb_w[k] = static_cast<float>(-acc / bs);
    }
}

// y = A x (transpose = false) or A^T x (true) in FP32 over the graph:
// (A x)_v = d_v x_v + sum_{u in N(v)} a_vu x_u;  (A^T x)_u = d_u x_u + sum over
// edges (v -> u) of a_vu x_v.
template<bool TRANSPOSE>
__global__ void __launch_bounds__(256) k_gnn_matvec(GraphArgs g, const float* __restrict__ nb_a,
                                                    const float* __restrict__ diag_f, const float* __restrict__ x,
                                                    float* __restrict__ y)
{
    const long long t = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= static_cast<long long>(g.n) * g.bs) return;
    const int v = static_cast<int>(t / g.bs), c = static_cast<int>(t - static_cast<long long>(v) * g.bs);
    float acc = diag_f[t] * x[t];
    if (TRANSPOSE) {
        for (int k = g.tr_ptr[v]; k < g.tr_ptr[v + 1]; ++k) {
            // tr_w's edge: the transposed slot stores the forward edge index in nb order
            const int src = g.tr_col[k];
            acc = fmaf(nb_a[static_cast<long long>(g.tr_edge[k]) * g.bs + c], x[static_cast<long long>(src) * g.bs + c],
                       acc);
        }
    } else {
        for (int k = g.nb_ptr[v]; k < g.nb_ptr[v + 1]; ++k)
            acc = fmaf(nb_a[static_cast<long long>(k) * g.bs + c], x[static_cast<long long>(g.nb_col[k]) * g.bs + c],
                       acc);
    }
    y[t] = acc;
}

__global__ void k_gnn_gather_w(int count, const int* __restrict__ idx, const float* __restrict__ src,
                               float* __restrict__ dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) dst[i] = src[idx[i]];
}

// Padded slot weights as BF16 bits (padding, idx < 0: zero).
__global__ void k_gnn_gather_wb(int count, const int* __restrict__ idx, const float* __restrict__ src,
                                unsigned short* __restrict__ dst)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < count) dst[i] = idx[i] >= 0 ? __bfloat16_as_ushort(__float2bfloat16_rn(src[idx[i]])) : 0;
}

}  // namespace gnn

// ====================================================================== host
struct Gnn {
    static constexpr int kOffWe = 0;
    static constexpr int kOffWl = gnn::kH * gnn::kF;
    static constexpr int kLayerW = gnn::kH * 2 * gnn::kH;
    static constexpr int kOffWd = kOffWl + gnn::kLayers * kLayerW;
    static constexpr int kParams = kOffWd + 8 * gnn::kH;

    Context* ctx = nullptr;
    Matrix* matrix = nullptr;
    int n = 0, bs = 0;
    DeviceBuffer nb_ptr, nb_col, nb_w, nb_entry, tr_ptr, tr_col, tr_w, tr_edge, dinv;
    DeviceBuffer ell_col, ell_src, ell_w, tile_ovf;   // padded 8-slot neighbour lists (forward layer)
    DeviceBuffer params, grads, adam_m, adam_v, wl16, wlt16;
    DeviceBuffer h[gnn::kLayers + 1], m[gnn::kLayers], mask[gnn::kLayers], x;   // training activations
    DeviceBuffer ha, hb;                                                       // inference ping-pong
    DeviceBuffer norm_r, norm_e, out32, dz, dh, dm, dy, partials, loss_partials, ticket, loss;
    DeviceBuffer qbuf;   // q = r / d (FP32); norm_r holds |r|, |q| at [0], [2]
    // Inference with the encoder folded into the first layer (bs <= 4): the
    // per-vertex input records and the folded first-layer operand B1.
    bool fused_first = false;
    DeviceBuffer rec, b1;
    // Gather plan of the TMA-fed layer (per 16-row sub-tile: neighbour rows in
    // quads, per row {slot or -1, degree, edge offset, 1}) and the tensor maps
    // of every feature buffer (gather: box 64 x 1; tile: box 64 x 128, swizzled).
    DeviceBuffer quads, quad_ptr, metas;
    bool tma = false;
    CUtensorMap gmap_a{}, tmap_a{}, gmap_b{}, tmap_b{}, gmap_h[gnn::kLayers + 1]{}, tmap_h[gnn::kLayers + 1]{};
    DeviceBuffer nb_a, diag_f, ax, res, gres;   // FP32 coefficients; A out, r - A out, A^T (r - A out)
    double loss_error_weight = 0.1, loss_residual_weight = 1.0;
    int adam_t = 0;
    bool train_ready = false;
    std::uint64_t applications = 0;
    // When set (owtk_learned_stage_times), gnn_forward records one event
    // before the first launch and one after each stage: [0] start,
    // [1] norms + encoder, [2..5] layers 1-4 (the last with the decoder).
    cudaEvent_t* stage_events = nullptr;

    gnn::GraphArgs graph() const
    {
        gnn::GraphArgs g;
        g.n = n;
        g.bs = bs;
        g.nb_ptr = nb_ptr.as<int>();
        g.nb_col = nb_col.as<int>();
        g.nb_w = nb_w.as<float>();
        g.tr_ptr = tr_ptr.as<int>();
        g.tr_col = tr_col.as<int>();
        g.tr_w = tr_w.as<float>();
        g.tr_edge = tr_edge.as<int>();
        g.dinv = dinv.as<float>();
        g.ell_col = ell_col.as<int>();
        g.ell_w = ell_w.as<unsigned short>();
        g.tile_ovf = tile_ovf.as<unsigned char>();
        return g;
    }
    unsigned blocks(long long count, int threads = 256) const
    {
        return static_cast<unsigned>((count + threads - 1) / threads);
    }
    unsigned layer_grid(int per_sm = 4) const
    {
        const int tiles = (n + gnn::kTile - 1) / gnn::kTile;
        return static_cast<unsigned>(std::min(tiles, ctx->sm_count * per_sm));
    }
};

namespace {

void gnn_pack(Gnn& G)
{
    gnn::k_gnn_pack<<<G.blocks(gnn::kLayers * Gnn::kLayerW), 256, 0, G.ctx->stream>>>(
        G.params.as<float>() + Gnn::kOffWl, G.wl16.as<gnn::bf16>(), G.wlt16.as<gnn::bf16>());
    OWTK_CUDA(cudaGetLastError());
    G.ctx->launched();
    if (G.fused_first) {
        gnn::k_gnn_first_weights<<<G.blocks(2 * gnn::kH * 16), 256, 0, G.ctx->stream>>>(
            G.params.as<float>() + Gnn::kOffWe, G.params.as<float>() + Gnn::kOffWl, G.b1.as<gnn::bf16>());
        OWTK_CUDA(cudaGetLastError());
        G.ctx->launched();
    }
}

void gnn_set_attrs()
{
    OWTK_CUDA(cudaFuncSetAttribute(gnn::k_gnn_layer<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gnn::kLayerSmem));
    OWTK_CUDA(cudaFuncSetAttribute(gnn::k_gnn_layer<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gnn::kLayerSmem));
    OWTK_CUDA(cudaFuncSetAttribute(gnn::k_gnn_layer<false, true, double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gnn::kLayerSmemDec));
    OWTK_CUDA(cudaFuncSetAttribute(gnn::k_gnn_first_layer, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gnn::kFirstSmem));
    OWTK_CUDA(cudaFuncSetAttribute(gnn::k_gnn_layer_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gnn::kBwdSmem));
    OWTK_CUDA(cudaFuncSetAttribute(gnn::k_gnn_wgrad, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gnn::kWgradSmem));
    OWTK_CUDA(cudaFuncSetAttribute(gnn::k_gnn_layer_tma<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gnn::kTmaSmem));
    OWTK_CUDA(cudaFuncSetAttribute(gnn::k_gnn_layer_tma<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   gnn::kTmaSmem));
}

// Tensor maps of a feature buffer (n rows of 64 BF16).
bool gnn_encode_maps(const void* h, int n, CUtensorMap& gmap, CUtensorMap& tmap)
{
    static PFN_cuTensorMapEncodeTiled_v12000 encode = [] {
        void* fn = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess
            || q != cudaDriverEntryPointSuccess)
            fn = nullptr;
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
    }();
    if (!encode) return false;
    const cuuint64_t dims[2] = {static_cast<cuuint64_t>(gnn::kH), static_cast<cuuint64_t>(n)};
    const cuuint64_t strides[1] = {static_cast<cuuint64_t>(gnn::kH * 2)};
    const cuuint32_t one[2] = {1, 1};
    const cuuint32_t gbox[2] = {static_cast<cuuint32_t>(gnn::kH), 1};
    const cuuint32_t tbox[2] = {static_cast<cuuint32_t>(gnn::kH), static_cast<cuuint32_t>(gnn::kTile)};
    void* addr = const_cast<void*>(h);
    if (encode(&gmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, addr, dims, strides, gbox, one, CU_TENSOR_MAP_INTERLEAVE_NONE,
               CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
        != CUDA_SUCCESS)
        return false;
    return encode(&tmap, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, addr, dims, strides, tbox, one,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE)
        == CUDA_SUCCESS;
}

// Seeded initial weights: normal draws from std::mt19937_64, scaled per
// matrix; the decoder starts at zero (the network starts as Jacobi).
std::vector<float> gnn_initial_weights(int bs, std::uint64_t seed)
{
    std::vector<float> w(Gnn::kParams, 0.0f);
    std::mt19937_64 gen(seed);
    std::normal_distribution<double> nd(0.0, 1.0);
    const double se = 1.0 / std::sqrt(2.0 * bs), sl = 0.5 / std::sqrt(2.0 * gnn::kH);
    for (int k = 0; k < gnn::kH; ++k)
        for (int f = 0; f < gnn::kF; ++f) {
            const double z = nd(gen);
            w[Gnn::kOffWe + k * gnn::kF + f] = f < 2 * bs ? static_cast<float>(se * z) : 0.0f;
        }
    for (int i = 0; i < gnn::kLayers * Gnn::kLayerW; ++i) w[Gnn::kOffWl + i] = static_cast<float>(sl * nd(gen));
    return w;
}

// Forward from r (device, T) into out (device, O).  TRAIN keeps activations.
template<class T, class O, bool TRAIN>
void gnn_forward(Gnn& G, const T* r, O* out)
{
    Context& c = *G.ctx;
    const gnn::GraphArgs g = G.graph();
    const long long nb = static_cast<long long>(G.n) * G.bs;
    double* norms = G.norm_r.as<double>();
    auto mark = [&](int k) {
        if (G.stage_events) OWTK_CUDA(cudaEventRecord(G.stage_events[k], c.stream));
    };
    mark(0);
    kern::prepare_norms<T>(c, static_cast<std::size_t>(nb), r, G.dinv.as<float>(), G.qbuf.as<float>(), norms);
    const bool fused = !TRAIN && G.fused_first;
    const gnn::bf16* hin = nullptr;
    if (fused) {
        // Input records, then the encoder and the first layer in one kernel
        // (output in hb, the buffer the second layer reads).
        gnn::launch_records<T>(G.blocks(G.n), c.stream, G.n, G.bs, r, G.qbuf.as<float>(), G.rec.as<float4>());
        OWTK_CUDA(cudaGetLastError());
        c.launched();
        mark(1);
        gnn::k_gnn_first_layer<<<G.layer_grid(4), gnn::kFirstThreads, gnn::kFirstSmem, c.stream>>>(
            g, G.tmap_b, G.rec.as<float4>(), norms, G.b1.as<gnn::bf16>(), c.status.as<unsigned>());
        OWTK_CUDA(cudaGetLastError());
        c.launched();
        mark(2);
        hin = G.hb.as<gnn::bf16>();
    } else {
        gnn::bf16* h0 = TRAIN ? G.h[0].as<gnn::bf16>() : G.ha.as<gnn::bf16>();
        gnn::launch_encode<T>(std::min(G.blocks(G.n), static_cast<unsigned>(c.sm_count * 8)), c.stream, g, r,
                              G.qbuf.as<float>(), norms, G.params.as<float>() + Gnn::kOffWe, h0);
        OWTK_CUDA(cudaGetLastError());
        c.launched();
        mark(1);
        hin = h0;
    }
    for (int l = fused ? 1 : 0; l < gnn::kLayers; ++l) {
        gnn::bf16* hout = TRAIN ? G.h[l + 1].as<gnn::bf16>() : (l % 2 == 0 ? G.hb : G.ha).as<gnn::bf16>();
        if (G.tma) {
            const CUtensorMap& gm = TRAIN ? G.gmap_h[l] : (l % 2 == 0 ? G.gmap_a : G.gmap_b);
            const CUtensorMap& tm = TRAIN ? G.tmap_h[l] : (l % 2 == 0 ? G.tmap_a : G.tmap_b);
            const int tiles = (G.n + gnn::kTile - 1) / gnn::kTile;
            const unsigned grid = static_cast<unsigned>(std::min(tiles, c.sm_count * 2));
            gnn::k_gnn_layer_tma<TRAIN><<<grid, gnn::kTmaThreads, gnn::kTmaSmem, c.stream>>>(
                g, gm, tm, hin, G.wl16.as<gnn::bf16>() + l * Gnn::kLayerW, hout,
                TRAIN ? G.m[l].as<gnn::bf16>() : nullptr, TRAIN ? G.mask[l].as<unsigned long long>() : nullptr,
                G.quads.as<int4>(), G.quad_ptr.as<int>(), G.metas.as<int4>(),
                static_cast<int>(G.nb_col.bytes / sizeof(int)), c.status.as<unsigned>());
        } else {
            const CUtensorMap& tm = TRAIN ? G.tmap_h[l] : (l % 2 == 0 ? G.tmap_a : G.tmap_b);
            const gnn::bf16* wl = G.wl16.as<gnn::bf16>() + l * Gnn::kLayerW;
            if constexpr (!TRAIN) {
              if (l == gnn::kLayers - 1) {   // last layer with the decoder fused
                const gnn::DecodeArgs<O> dec{G.qbuf.as<float>(), norms, G.params.as<float>() + Gnn::kOffWd, out};
                gnn::k_gnn_layer<false, true, O><<<G.layer_grid(OWTK_GNN_DEC_BLOCKS), gnn::kFwdThreads, gnn::kLayerSmemDec, c.stream>>>(
                    g, tm, tm, hin, wl, nullptr, nullptr, dec, c.status.as<unsigned>());
                OWTK_CUDA(cudaGetLastError());
                c.launched();
                mark(2 + l);
                ++G.applications;
                return;
              }
            }
            const CUtensorMap& tmo = TRAIN ? G.tmap_h[l + 1] : (l % 2 == 0 ? G.tmap_b : G.tmap_a);
            gnn::k_gnn_layer<TRAIN><<<G.layer_grid(4), gnn::kFwdThreads, gnn::kLayerSmem, c.stream>>>(
                g, tm, tmo, hin, wl, TRAIN ? G.m[l].as<gnn::bf16>() : nullptr,
                TRAIN ? G.mask[l].as<unsigned long long>() : nullptr, gnn::DecodeArgs<float>{},
                c.status.as<unsigned>());
        }
        OWTK_CUDA(cudaGetLastError());
        c.launched();
        if (l < gnn::kLayers - 1) mark(2 + l);
        hin = hout;
    }
    gnn::k_gnn_decode<O><<<G.blocks(8ll * G.n), 256, 0, c.stream>>>(g, G.qbuf.as<float>(), norms,
                                                               G.params.as<float>() + Gnn::kOffWd, hin, out);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
    mark(2 + gnn::kLayers - 1);
    ++G.applications;
}

void gnn_train_buffers(Gnn& G)
{
    if (G.train_ready) return;
    const std::size_t rows = static_cast<std::size_t>(G.n);
    for (auto& b : G.h) b.allocate(rows * gnn::kH * 2 + 16);
    for (int l = 0; l <= gnn::kLayers; ++l)
        if (!gnn_encode_maps(G.h[l].ptr, G.n, G.gmap_h[l], G.tmap_h[l]))
            fail(OWTK_ERR_CUDA, "tensor-map encoding of the training activations failed");
    for (auto& b : G.m) b.allocate(rows * gnn::kH * 2 + 16);
    for (auto& b : G.mask) b.allocate(rows * 8 + 16);
    G.x.allocate(rows * gnn::kF * 4 + 16);
    G.out32.allocate(rows * G.bs * 4 + 16);
    G.ax.allocate(rows * G.bs * 4 + 16);
    G.res.allocate(rows * G.bs * 4 + 16);
    G.gres.allocate(rows * G.bs * 4 + 16);
    G.dz.allocate(rows * G.bs * 4 + 16);
    G.dh.allocate(rows * gnn::kH * 4 + 16);
    G.dm.allocate(rows * gnn::kH * 4 + 16);
    G.dy.allocate(rows * gnn::kH * 2 + 16);
    G.partials.allocate(static_cast<std::size_t>(std::max(G.ctx->sm_count * 4, 256)) * 2 * gnn::kH * gnn::kH * 4);
    G.loss_partials.allocate(1024 * 8);
    G.ticket.allocate(16);
    OWTK_CUDA(cudaMemsetAsync(G.ticket.ptr, 0, 16, G.ctx->stream));
    G.loss.allocate(16);
    G.norm_e.allocate(16);
    G.train_ready = true;
}

// Features x of every vertex (kept for the encoder gradient).
__global__ void k_gnn_features(gnn::GraphArgs g, const double* __restrict__ r, const float* __restrict__ q,
                               const double* norms, float* __restrict__ x)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= g.n) return;
    const double root = sqrt(static_cast<double>(g.n) * g.bs), nr = norms[0], nq = norms[2];
    const float inv_r = nr > 0.0 ? static_cast<float>(root / nr) : 0.0f;
    const float inv_q = nq > 0.0 ? static_cast<float>(root / nq) : 0.0f;
    float* xv = x + static_cast<long long>(v) * gnn::kF;
    for (int f = 0; f < gnn::kF; ++f) xv[f] = 0.0f;
    for (int c = 0; c < g.bs; ++c) {
        const long long o = static_cast<long long>(v) * g.bs + c;
        xv[c] = static_cast<float>(r[o]) * inv_r;
        xv[g.bs + c] = q[o] * inv_q;
    }
}

// Loss and gradient of one (r, e) pair into G.grads; returns the loss.
double gnn_loss_grad(Gnn& G, const double* r, const double* e)
{
    Context& c = *G.ctx;
    gnn_train_buffers(G);
    const gnn::GraphArgs g = G.graph();
    const long long nb = static_cast<long long>(G.n) * G.bs;
    gnn_forward<double, float, true>(G, r, G.out32.as<float>());
    k_gnn_features<<<G.blocks(G.n), 256, 0, c.stream>>>(g, r, G.qbuf.as<float>(), G.norm_r.as<double>(),
                                                        G.x.as<float>());
    kern::norm<double>(c, static_cast<std::size_t>(nb), e, G.norm_e.as<double>(), G.norm_e.as<double>() + 1);
    gnn::k_gnn_matvec<false><<<G.blocks(nb), 256, 0, c.stream>>>(g, G.nb_a.as<float>(), G.diag_f.as<float>(),
                                                                 G.out32.as<float>(), G.ax.as<float>());
    gnn::k_gnn_residual<<<G.blocks(nb), 256, 0, c.stream>>>(nb, r, G.ax.as<float>(), G.res.as<float>());
    gnn::k_gnn_matvec<true><<<G.blocks(nb), 256, 0, c.stream>>>(g, G.nb_a.as<float>(), G.diag_f.as<float>(),
                                                                G.res.as<float>(), G.gres.as<float>());
    const unsigned lb = 512;
    gnn::k_gnn_out_grad<<<lb, 256, 0, c.stream>>>(nb, G.out32.as<float>(), e, G.res.as<float>(), G.gres.as<float>(),
                                                   G.norm_e.as<double>(), G.norm_r.as<double>(),
                                                   std::sqrt(static_cast<double>(nb)), G.loss_error_weight,
                                                   G.loss_residual_weight, G.dz.as<float>(),
                                                   G.loss_partials.as<double>(), G.ticket.as<unsigned>(),
                                                   G.loss.as<double>());
    c.launched(4);
    gnn::k_gnn_decode_bwd<<<G.blocks(G.n), 256, 0, c.stream>>>(G.n, G.bs, G.dz.as<float>(),
                                                                G.params.as<float>() + Gnn::kOffWd, G.dh.as<float>());
    float* grads = G.grads.as<float>();
    OWTK_CUDA(cudaMemsetAsync(grads, 0, Gnn::kParams * sizeof(float), c.stream));
    const unsigned ob = 256;
    gnn::k_gnn_outer<gnn::bf16><<<ob, 256, 0, c.stream>>>(G.n, G.bs, gnn::kH, G.dz.as<float>(),
                                                           G.h[gnn::kLayers].as<gnn::bf16>(), G.partials.as<float>());
    gnn::k_gnn_reduce<<<G.blocks(G.bs * gnn::kH), 256, 0, c.stream>>>(ob, G.bs * gnn::kH, G.partials.as<float>(),
                                                                       grads + Gnn::kOffWd, 0, 0, 0);
    c.launched(6);
    for (int l = gnn::kLayers - 1; l >= 0; --l) {
        gnn::k_gnn_layer_bwd<<<G.layer_grid(), gnn::kLayerThreads, gnn::kBwdSmem, c.stream>>>(
            G.n, G.dh.as<float>(), G.mask[l].as<unsigned long long>(), G.wlt16.as<gnn::bf16>() + l * Gnn::kLayerW,
            G.dy.as<gnn::bf16>(), G.dm.as<float>(), c.status.as<unsigned>());
        const unsigned wg = G.layer_grid();
        gnn::k_gnn_wgrad<<<wg, gnn::kLayerThreads, gnn::kWgradSmem, c.stream>>>(
            G.n, G.h[l].as<gnn::bf16>(), G.m[l].as<gnn::bf16>(), G.dy.as<gnn::bf16>(), G.partials.as<float>(),
            c.status.as<unsigned>());
        gnn::k_gnn_reduce<<<G.blocks(2 * gnn::kH * gnn::kH), 256, 0, c.stream>>>(
            wg, 2 * gnn::kH * gnn::kH, G.partials.as<float>(), grads + Gnn::kOffWl + l * Gnn::kLayerW, 2 * gnn::kH,
            gnn::kH, 1);
        gnn::k_gnn_agg_t<<<G.blocks(static_cast<long long>(G.n) * 16), 256, 0, c.stream>>>(g, G.dm.as<float>(),
                                                                                            G.dh.as<float>());
        OWTK_CUDA(cudaGetLastError());
        c.launched(4);
    }
    gnn::k_gnn_outer<float><<<ob, 256, 0, c.stream>>>(G.n, gnn::kH, gnn::kF, G.dh.as<float>(), G.x.as<float>(),
                                                       G.partials.as<float>());
    gnn::k_gnn_reduce<<<G.blocks(gnn::kH * gnn::kF), 256, 0, c.stream>>>(ob, gnn::kH * gnn::kF, G.partials.as<float>(),
                                                                          grads + Gnn::kOffWe, 0, 0, 0);
    OWTK_CUDA(cudaGetLastError());
    c.launched(3);
    double loss = 0.0;
    OWTK_CUDA(cudaMemcpyAsync(&loss, G.loss.ptr, sizeof(double), cudaMemcpyDeviceToHost, c.stream));
    c.sync();
    c.check_device_status();
    return loss;
}

void gnn_adam(Gnn& G, double lr)
{
    Context& c = *G.ctx;
    ++G.adam_t;
    const float b1 = 0.9f, b2 = 0.999f;
    const float c1 = 1.0f - std::pow(b1, static_cast<float>(G.adam_t));
    const float c2 = 1.0f - std::pow(b2, static_cast<float>(G.adam_t));
    gnn::k_gnn_adam<<<G.blocks(Gnn::kParams), 256, 0, c.stream>>>(Gnn::kParams, G.params.as<float>(),
                                                                    G.grads.as<float>(), G.adam_m.as<float>(),
                                                                    G.adam_v.as<float>(), static_cast<float>(lr), b1,
                                                                    b2, 1e-8f, c1, c2);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
    gnn_pack(G);
}

}  // namespace

namespace gnn {
}  // namespace gnn
}  // namespace owtk

// ====================================================================== C ABI
namespace owtk {

// z = M(v); judged by ||v - A z|| against ||v||, the fallback steps in when
// the network does not reduce the residual.
namespace gnn {
// One damped Jacobi correction of the network's output: z += omega D^-1 (v - A z),
// each operation rounded as written (no contraction).
__global__ void __launch_bounds__(256) k_jacobi_correct(long long count, const double* __restrict__ v,
                                                        const double* __restrict__ az,
                                                        const float* __restrict__ dinv, double omega,
                                                        double* __restrict__ z)
{
    const long long i = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count)
        z[i] = __dadd_rn(z[i], __dmul_rn(omega, __dmul_rn(static_cast<double>(dinv[i]), __dsub_rn(v[i], az[i]))));
}
}  // namespace gnn

bool learned_apply(Preconditioner& p, Vector& in, Vector& out, double* product)
{
    Gnn& G = *p.net;
    Context& c = *G.ctx;
    const std::size_t n = static_cast<std::size_t>(G.n) * G.bs;
    const double* x = static_cast<const double*>(in.data);
    double* y = static_cast<double*>(out.data);
    if (x == y) {
        if (!p.alias_copy.ptr) p.alias_copy.allocate(n * sizeof(double) + 16);
        kern::copy<double>(c, n, x, p.alias_copy.as<double>());
        x = p.alias_copy.as<double>();
    }
    gnn_forward<double, double, false>(G, x, y);
    ++p.learned_applications;
    const int corrections = p.learned_correction_steps;
    if (p.fallback == nullptr && corrections == 0) return false;
    // The check's product A z is the solver's next operator application: it
    // lands in `product` when the caller asks for it.
    double* w = product;
    if (w == nullptr) {
        if (!p.check_work.ptr) p.check_work.allocate(n * sizeof(double) + 16);
        w = p.check_work.as<double>();
    }
    kern::spmv<double>(c, *G.matrix, y, w);
    const auto correct = [&] {
        // After an accepted step: the corrections, each followed by the
        // product of the corrected z (the solver's next operator application).
        for (int k = 0; k < corrections; ++k) {
            gnn::k_jacobi_correct<<<G.blocks(static_cast<long long>(n)), 256, 0, c.stream>>>(
                static_cast<long long>(n), x, w, G.dinv.as<float>(), p.learned_correction_omega, y);
            OWTK_CUDA(cudaGetLastError());
            c.launched();
            kern::spmv<double>(c, *G.matrix, y, w);
        }
    };
    if (p.fallback == nullptr) {
        correct();
        return product != nullptr;
    }
    constexpr int kSlot = kScalarSlots - 4;
    kern::residual_norms(c, n, x, w, c.dev_scalar_copy.as<double>() + kSlot, c.dev_scalars + kSlot);
    c.sync();
    const double rho = c.host_scalars[kSlot], nu = c.host_scalars[kSlot + 1];
    if (!(rho < nu)) {
        ++p.learned_fallbacks;
        Vector src;        // non-owning description of the (possibly copied) input
        src.ctx = in.ctx;
        src.dtype = in.dtype;
        src.owned = in.owned;
        src.ghost = in.ghost;
        src.bs = in.bs;
        src.data = const_cast<double*>(x);
        src.is_view = true;
        apply_preconditioner(p.fallback, src, out);
        return false;
    }
    correct();
    return product != nullptr;
}

const Matrix* learned_matrix(const Preconditioner& p) { return p.net ? p.net->matrix : nullptr; }

namespace {

void gnn_bind_matrix(Gnn& G, Matrix& m)
{
    Context& c = *G.ctx;
    DeviceBuffer diag(static_cast<std::size_t>(G.n) * G.bs * sizeof(double) + 16);
    kern::bsr_diagonal<double>(c, m, diag.as<double>());
    c.sync();
    try {
        c.check_device_status();
    } catch (const Error&) {
        fail(OWTK_ERR_INVALID_ARGUMENT, "BlockCsrMatrix row has no diagonal");
    }
    gnn::k_gnn_graph<<<G.blocks(G.n), 256, 0, c.stream>>>(G.n, G.bs, G.nb_ptr.as<int>(), G.nb_entry.as<int>(),
                                                           static_cast<const double*>(m.values.ptr), diag.as<double>(),
                                                           G.nb_w.as<float>(), G.dinv.as<float>(), G.nb_a.as<float>(),
                                                           G.diag_f.as<float>());
    const int ne = static_cast<int>(G.tr_col.bytes / sizeof(int));
    if (ne > 0)
        gnn::k_gnn_gather_w<<<G.blocks(ne), 256, 0, c.stream>>>(ne, G.tr_edge.as<int>(), G.nb_w.as<float>(),
                                                                G.tr_w.as<float>());
    const int slots = G.n * gnn::kEll;
    gnn::k_gnn_gather_wb<<<G.blocks(slots), 256, 0, c.stream>>>(slots, G.ell_src.as<int>(), G.nb_w.as<float>(),
                                                                G.ell_w.as<unsigned short>());
    OWTK_CUDA(cudaGetLastError());
    c.launched(3);
    c.sync();
    G.matrix = &m;
}

}  // namespace
}  // namespace owtk

struct owtk_learned : owtk::Gnn {};

extern "C" {

owtk_status owtk_bf16_gemm_nt(owtk_context* ctx, size_t m, size_t n, size_t k, const void* device_a,
                              const void* device_b, float* device_d)
{
    return owtk::guarded([&] {
        owtk::require(ctx != nullptr && device_a != nullptr && device_b != nullptr && device_d != nullptr,
                      "null argument");
        if (m == 0 || m % 128 != 0 || (n != 64 && n != 128) || k == 0 || k % 64 != 0 || k > (1u << 20)
            || m > (1ull << 31))
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "bf16 gemm shape: m % 128 == 0, n in {64, 128}, k % 64 == 0");
        const auto aligned = [](const void* p) { return (reinterpret_cast<std::uintptr_t>(p) & 15u) == 0; };
        if (!aligned(device_a) || !aligned(device_b) || !aligned(device_d))
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "bf16 gemm operands must be 16-byte aligned");
        const int smem = 1024 + owtk::gnn::kTile * 128 + static_cast<int>(n) * 128;
        const auto* A = static_cast<const owtk::gnn::bf16*>(device_a);
        const auto* B = static_cast<const owtk::gnn::bf16*>(device_b);
        const unsigned grid = static_cast<unsigned>(m / 128);
        if (n == 64) {
            OWTK_CUDA(cudaFuncSetAttribute(owtk::gnn::k_umma_gemm_nt<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                           smem));
            owtk::gnn::k_umma_gemm_nt<64><<<grid, 128, smem, ctx->stream>>>(static_cast<int>(k), A, B, device_d,
                                                                             ctx->status.as<unsigned>());
        } else {
            OWTK_CUDA(cudaFuncSetAttribute(owtk::gnn::k_umma_gemm_nt<128>,
                                           cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
            owtk::gnn::k_umma_gemm_nt<128><<<grid, 128, smem, ctx->stream>>>(static_cast<int>(k), A, B, device_d,
                                                                              ctx->status.as<unsigned>());
        }
        OWTK_CUDA(cudaGetLastError());
        ctx->launched();
        ctx->sync();
        ctx->check_device_status();
    });
}

owtk_status owtk_learned_create(owtk_matrix* m, uint64_t seed, owtk_learned** out)
{
    return owtk::guarded([&] {
        owtk::require(m != nullptr && out != nullptr, "null handle");
        if (m->kind != 0 || m->dtype != OWTK_F64 || m->ghost != 0 || m->bs == 0 || m->bs > 8)
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT,
                       "the learned preconditioner needs an FP64 component-diagonal BSR matrix, no ghosts, bs <= 8");
        auto G = std::make_unique<owtk_learned>();
        G->ctx = m->ctx;
        G->n = static_cast<int>(m->owned);
        G->bs = static_cast<int>(m->bs);
        // Off-diagonal neighbour lists and their transpose (host structure).
        std::vector<std::int32_t> nb_ptr(G->n + 1, 0), nb_col, nb_entry, tr_count(G->n + 1, 0);
        for (int v = 0; v < G->n; ++v) {
            for (int e = m->h_rowptr[v]; e < m->h_rowptr[v + 1]; ++e) {
                const int u = m->h_cols[e];
                if (u == v) continue;
                nb_col.push_back(u);
                nb_entry.push_back(e);
                ++tr_count[u + 1];
            }
            nb_ptr[v + 1] = static_cast<std::int32_t>(nb_col.size());
        }
        std::vector<std::int32_t> tr_ptr(G->n + 1, 0);
        for (int u = 0; u < G->n; ++u) tr_ptr[u + 1] = tr_ptr[u] + tr_count[u + 1];
        std::vector<std::int32_t> tr_col(nb_col.size()), tr_edge(nb_col.size()), fill(tr_ptr.begin(), tr_ptr.end() - 1);
        for (int v = 0; v < G->n; ++v)
            for (int k = nb_ptr[v]; k < nb_ptr[v + 1]; ++k) {
                const int u = nb_col[k];
                tr_col[fill[u]] = v;
                tr_edge[fill[u]] = k;
                ++fill[u];
            }
        cudaStream_t st = G->ctx->stream;
        G->nb_ptr = owtk::upload(st, nb_ptr);
        G->nb_col = owtk::upload(st, nb_col);
        G->nb_entry = owtk::upload(st, nb_entry);
        G->tr_ptr = owtk::upload(st, tr_ptr);
        G->tr_col = owtk::upload(st, tr_col);
        G->tr_col.bytes = tr_col.size() * sizeof(int);
        G->tr_edge = owtk::upload(st, tr_edge);
        G->nb_w.allocate(nb_col.size() * sizeof(float) + 16);
        G->tr_w.allocate(nb_col.size() * sizeof(float) + 16);
        G->dinv.allocate(static_cast<std::size_t>(G->n) * G->bs * sizeof(float) + 16);
        G->diag_f.allocate(static_cast<std::size_t>(G->n) * G->bs * sizeof(float) + 16);
        G->nb_a.allocate(nb_col.size() * G->bs * sizeof(float) + 16);
        const std::vector<float> w0 = owtk::gnn_initial_weights(G->bs, seed);
        G->params = owtk::upload(st, w0);
        G->grads.allocate(owtk::Gnn::kParams * sizeof(float) + 16);
        G->adam_m.allocate(owtk::Gnn::kParams * sizeof(float) + 16);
        G->adam_v.allocate(owtk::Gnn::kParams * sizeof(float) + 16);
        OWTK_CUDA(cudaMemsetAsync(G->adam_m.ptr, 0, owtk::Gnn::kParams * sizeof(float), st));
        OWTK_CUDA(cudaMemsetAsync(G->adam_v.ptr, 0, owtk::Gnn::kParams * sizeof(float), st));
        G->wl16.allocate(owtk::gnn::kLayers * owtk::Gnn::kLayerW * 2 + 16);
        G->wlt16.allocate(owtk::gnn::kLayers * owtk::Gnn::kLayerW * 2 + 16);
        G->ha.allocate(static_cast<std::size_t>(G->n) * owtk::gnn::kH * 2 + 16);
        G->hb.allocate(static_cast<std::size_t>(G->n) * owtk::gnn::kH * 2 + 16);
        G->norm_r.allocate(64);
        // Gather plan of the TMA-fed layer.
        {
            const int subs = (G->n + owtk::gnn::kSubRows - 1) / owtk::gnn::kSubRows;
            std::vector<std::int32_t> quads, quad_ptr(subs + 1, 0), metas(static_cast<std::size_t>(subs) * 16 * 4, 0);
            for (int sub = 0; sub < subs; ++sub) {
                const int r0 = sub * owtk::gnn::kSubRows;
                int slots = 0;
                for (int r = r0; r < std::min(r0 + owtk::gnn::kSubRows, G->n); ++r) {
                    const int e0 = nb_ptr[r], deg = nb_ptr[r + 1] - e0, need = (deg + 3) / 4 * 4;
                    std::int32_t* meta = &metas[(static_cast<std::size_t>(r)) * 4];
                    meta[1] = deg;
                    meta[2] = e0 - nb_ptr[r0];
                    meta[3] = 1;
                    if (deg == 0) {
                        meta[0] = 0;
                    } else if (slots + need <= owtk::gnn::kSlots) {
                        meta[0] = slots;
                        for (int j = 0; j < need; ++j) quads.push_back(nb_col[e0 + (j < deg ? j : 0)]);
                        slots += need;
                    } else {
                        meta[0] = -1;
                    }
                }
                quad_ptr[sub + 1] = static_cast<std::int32_t>(quads.size() / 4);
            }
            if (quads.empty()) quads.assign(4, 0);
            G->quads = owtk::upload(st, quads);
            G->quad_ptr = owtk::upload(st, quad_ptr);
            G->metas = owtk::upload(st, metas);
        }
        G->nb_col.bytes = nb_col.size() * sizeof(int);
        // Padded 8-slot neighbour lists of the forward layer: the first 8
        // neighbours in edge order, padding slots -1 (weight 0; the weights
        // are filled from the edge weights on every matrix bind).
        {
            const int tiles = (G->n + owtk::gnn::kTile - 1) / owtk::gnn::kTile;
            std::vector<std::int32_t> ell_col(static_cast<std::size_t>(G->n) * owtk::gnn::kEll),
                ell_src(ell_col.size());
            std::vector<std::uint8_t> tile_ovf(tiles, 0);
            for (int v = 0; v < G->n; ++v) {
                const int e0 = nb_ptr[v], deg = nb_ptr[v + 1] - e0;
                for (int q = 0; q < owtk::gnn::kEll; ++q) {
                    const std::size_t i = static_cast<std::size_t>(v) * owtk::gnn::kEll + q;
                    ell_col[i] = q < deg ? nb_col[e0 + q] : -1;
                    ell_src[i] = q < deg ? e0 + q : -1;
                }
                if (deg > owtk::gnn::kEll) tile_ovf[v / owtk::gnn::kTile] = 1;
            }
            G->ell_col = owtk::upload(st, ell_col);
            G->ell_src = owtk::upload(st, ell_src);
            G->tile_ovf = owtk::upload(st, tile_ovf);
            G->ell_w.allocate(ell_col.size() * sizeof(unsigned short) + 16);
        }
        // Tensor maps of the ping-pong feature buffers (own-row tiles of the
        // layer).  The register-gather layer is the default: on the 2M-vertex
        // mesh the TMA-gather layer measured about twice its time per launch.
        if (!owtk::gnn_encode_maps(G->ha.ptr, G->n, G->gmap_a, G->tmap_a)
            || !owtk::gnn_encode_maps(G->hb.ptr, G->n, G->gmap_b, G->tmap_b))
            owtk::fail(OWTK_ERR_CUDA, "tensor-map encoding of the feature buffers failed");
        const char* tma_env = std::getenv("OWTK_GNN_TMA");
        G->tma = tma_env && tma_env[0] == '1';
        G->qbuf.allocate(static_cast<std::size_t>(G->n) * G->bs * sizeof(float) + 16);
        // The encoder folded into the first layer (inference, bs <= 4) unless
        // OWTK_GNN_FUSED_FIRST=0 or the TMA-gather layer is selected.
        const char* fused_env = std::getenv("OWTK_GNN_FUSED_FIRST");
        G->fused_first = G->bs <= 4 && !G->tma && !(fused_env && fused_env[0] == '0');
        if (G->fused_first) {
            G->rec.allocate(static_cast<std::size_t>(G->n) * 8 * sizeof(float) + 16);
            G->b1.allocate(2 * owtk::gnn::kH * 16 * 2 + 16);
        }
        owtk::gnn_set_attrs();
        owtk::gnn_pack(*G);
        owtk::gnn_bind_matrix(*G, *m);
        *out = G.release();
    });
}

owtk_status owtk_learned_destroy(owtk_learned* net)
{
    return owtk::guarded([&] { delete net; });
}

owtk_status owtk_learned_update_matrix(owtk_learned* net, owtk_matrix* m)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && m != nullptr, "null handle");
        if (m->kind != 0 || m->dtype != OWTK_F64 || static_cast<int>(m->owned) != net->n
            || static_cast<int>(m->bs) != net->bs || m->entries != net->matrix->entries)
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "matrix pattern differs from the network's graph");
        owtk::gnn_bind_matrix(*net, *m);
    });
}

size_t owtk_learned_parameter_count(void) { return owtk::Gnn::kParams; }

int owtk_learned_uses_tma(const owtk_learned* net) { return net != nullptr && net->tma ? 1 : 0; }

owtk_status owtk_learned_set_loss_weights(owtk_learned* net, double error_weight, double residual_weight)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr, "null handle");
        if (!(error_weight >= 0) || !(residual_weight >= 0) || !std::isfinite(error_weight)
            || !std::isfinite(residual_weight) || error_weight + residual_weight <= 0)
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "loss weights must be finite, non-negative, not both zero");
        net->loss_error_weight = error_weight;
        net->loss_residual_weight = residual_weight;
    });
}

owtk_status owtk_learned_get_parameters(owtk_learned* net, float* host, size_t count)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && host != nullptr && count == owtk::Gnn::kParams, "parameter count");
        OWTK_CUDA(cudaMemcpyAsync(host, net->params.ptr, count * sizeof(float), cudaMemcpyDeviceToHost,
                                  net->ctx->stream));
        net->ctx->sync();
    });
}

owtk_status owtk_learned_set_parameters(owtk_learned* net, const float* host, size_t count)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && host != nullptr && count == owtk::Gnn::kParams, "parameter count");
        OWTK_CUDA(cudaMemcpyAsync(net->params.ptr, host, count * sizeof(float), cudaMemcpyHostToDevice,
                                  net->ctx->stream));
        owtk::gnn_pack(*net);
        net->ctx->sync();
    });
}

owtk_status owtk_learned_stage_times(owtk_learned* net, owtk_vector* in, owtk_vector* out, uint32_t repetitions,
                                     double* milliseconds)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && in != nullptr && out != nullptr && milliseconds != nullptr
                          && repetitions > 0,
                      "null argument or zero repetitions");
        if (in->dtype != OWTK_F64 || out->dtype != OWTK_F64 || static_cast<int>(in->owned) != net->n
            || static_cast<int>(in->bs) != net->bs || !in->same_layout(*out) || in->data == out->data)
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "learned preconditioner vector layout mismatch");
        constexpr int kMarks = 2 + owtk::gnn::kLayers;
        cudaEvent_t ev[kMarks] = {};
        for (auto& e : ev) OWTK_CUDA(cudaEventCreate(&e));
        double acc[kMarks - 1] = {};
        std::exception_ptr failure;
        net->stage_events = ev;
        try {
            for (uint32_t rep = 0; rep < repetitions; ++rep) {
                owtk::gnn_forward<double, double, false>(*net, static_cast<const double*>(in->data),
                                                         static_cast<double*>(out->data));
                OWTK_CUDA(cudaEventSynchronize(ev[kMarks - 1]));
                for (int k = 1; k < kMarks; ++k) {
                    float ms = 0.f;
                    OWTK_CUDA(cudaEventElapsedTime(&ms, ev[k - 1], ev[k]));
                    acc[k - 1] += ms;
                }
            }
        } catch (...) {
            failure = std::current_exception();
        }
        net->stage_events = nullptr;
        for (auto& e : ev) cudaEventDestroy(e);
        if (failure) std::rethrow_exception(failure);
        net->ctx->check_device_status();
        const double r = static_cast<double>(repetitions);
        double layers = 0.0, total = 0.0;
        for (int k = 0; k < kMarks - 1; ++k) total += acc[k];
        const int first_plain = net->fused_first ? 1 : 0;   // layers before the last without the encoder
        for (int l = first_plain; l < owtk::gnn::kLayers - 1; ++l) layers += acc[1 + l];
        milliseconds[0] = acc[0] / r;
        milliseconds[1] = layers / r / (owtk::gnn::kLayers - 1 - first_plain);
        milliseconds[2] = acc[kMarks - 2] / r;
        milliseconds[3] = total / r;
        milliseconds[4] = net->fused_first ? acc[1] / r : 0.0;
    });
}

owtk_status owtk_learned_get_adam_state(owtk_learned* net, float* first_moment, float* second_moment, size_t count,
                                        uint64_t* step)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && first_moment != nullptr && second_moment != nullptr && step != nullptr
                          && count == owtk::Gnn::kParams,
                      "adam state count");
        OWTK_CUDA(cudaMemcpyAsync(first_moment, net->adam_m.ptr, count * sizeof(float), cudaMemcpyDeviceToHost,
                                  net->ctx->stream));
        OWTK_CUDA(cudaMemcpyAsync(second_moment, net->adam_v.ptr, count * sizeof(float), cudaMemcpyDeviceToHost,
                                  net->ctx->stream));
        net->ctx->sync();
        *step = static_cast<uint64_t>(net->adam_t);
    });
}

owtk_status owtk_learned_set_adam_state(owtk_learned* net, const float* first_moment, const float* second_moment,
                                        size_t count, uint64_t step)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && first_moment != nullptr && second_moment != nullptr
                          && count == owtk::Gnn::kParams && step < (1ull << 31),
                      "adam state count");
        OWTK_CUDA(cudaMemcpyAsync(net->adam_m.ptr, first_moment, count * sizeof(float), cudaMemcpyHostToDevice,
                                  net->ctx->stream));
        OWTK_CUDA(cudaMemcpyAsync(net->adam_v.ptr, second_moment, count * sizeof(float), cudaMemcpyHostToDevice,
                                  net->ctx->stream));
        net->ctx->sync();
        net->adam_t = static_cast<int>(step);
    });
}

owtk_status owtk_learned_apply(owtk_learned* net, owtk_vector* in, owtk_vector* out)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && in != nullptr && out != nullptr, "null handle");
        if (in->dtype != OWTK_F64 || out->dtype != OWTK_F64 || static_cast<int>(in->owned) != net->n
            || static_cast<int>(in->bs) != net->bs || !in->same_layout(*out))
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "learned preconditioner vector layout mismatch");
        if (in->data == out->data) owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "in and out must differ");
        owtk::gnn_forward<double, double, false>(*net, static_cast<const double*>(in->data),
                                                 static_cast<double*>(out->data));
        net->ctx->sync();
        net->ctx->check_device_status();
    });
}

owtk_status owtk_learned_loss_grad(owtk_learned* net, owtk_vector* r, owtk_vector* e, double* loss,
                                   float* host_grads)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && r != nullptr && e != nullptr && loss != nullptr, "null argument");
        if (r->dtype != OWTK_F64 || e->dtype != OWTK_F64 || static_cast<int>(r->owned) != net->n
            || static_cast<int>(r->bs) != net->bs || !r->same_layout(*e))
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "training pair layout mismatch");
        *loss = owtk::gnn_loss_grad(*net, static_cast<const double*>(r->data), static_cast<const double*>(e->data));
        if (host_grads) {
            OWTK_CUDA(cudaMemcpyAsync(host_grads, net->grads.ptr, owtk::Gnn::kParams * sizeof(float),
                                      cudaMemcpyDeviceToHost, net->ctx->stream));
            net->ctx->sync();
        }
    });
}

owtk_status owtk_learned_adam_step(owtk_learned* net, double learning_rate)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && learning_rate > 0 && std::isfinite(learning_rate), "invalid learning rate");
        owtk::gnn_adam(*net, learning_rate);
        net->ctx->sync();
    });
}

owtk_status owtk_pc_create_learned(owtk_learned* net, owtk_preconditioner* fallback, owtk_preconditioner** out)
{
    return owtk::guarded([&] {
        owtk::require(net != nullptr && out != nullptr, "null handle");
        if (fallback && (fallback->owned != static_cast<std::size_t>(net->n)
                         || fallback->bs != static_cast<std::size_t>(net->bs) || fallback->dtype != OWTK_F64))
            owtk::fail(OWTK_ERR_INVALID_ARGUMENT, "fallback preconditioner layout differs from the network's");
        auto p = std::make_unique<owtk_preconditioner>();
        p->ctx = net->ctx;
        p->kind = OWTK_PC_LEARNED;
        p->dtype = OWTK_F64;
        p->matrix = net->matrix;
        p->owned = static_cast<std::size_t>(net->n);
        p->bs = static_cast<std::size_t>(net->bs);
        p->net = net;
        p->fallback = fallback;
        *out = p.release();
    });
}

owtk_status owtk_pc_learned_set_correction(owtk_preconditioner* p, uint32_t steps, double omega)
{
    return owtk::guarded([&] {
        owtk::require(p != nullptr && p->kind == OWTK_PC_LEARNED, "not a learned preconditioner");
        owtk::require(steps <= 8 && omega > 0.0 && omega < 2.0, "correction steps must be <= 8, omega in (0, 2)");
        p->learned_correction_steps = static_cast<int>(steps);
        p->learned_correction_omega = omega;
    });
}

owtk_status owtk_pc_learned_counts(owtk_preconditioner* p, uint64_t* applications, uint64_t* fallbacks)
{
    return owtk::guarded([&] {
        owtk::require(p != nullptr && p->kind == OWTK_PC_LEARNED, "not a learned preconditioner");
        if (applications) *applications = p->learned_applications;
        if (fallbacks) *fallbacks = p->learned_fallbacks;
    });
}

}  // extern "C"
