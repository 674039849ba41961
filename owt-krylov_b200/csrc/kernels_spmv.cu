// Block-CSR SpMV kernels (sm_100a): component-diagonal BSR, the split
// diagonal/edge view and dense bs x bs BSR.
//
// Work unit: a row tile (consecutive rows whose value stream fits kStage
// elements; built once per matrix on the host).  One CTA per tile:
//   1. product phase: thread k of the tile's value stream loads value k and
//      its column (consecutive threads, consecutive addresses: the value
//      stream is read exactly once, fully coalesced, with every thread's
//      loads issued together), then gathers x[col][c] (L2-resident for
//      RCM/Hilbert-ordered meshes) and stores the rounded product in shared
//      memory;
//   2. output phase: thread o owns output (row, c) and adds that row's
//      products in entry order, writing y coalesced.
// The sum starts from +0 (or diag*x for the split view) and adds rounded
// products in entry order, which is the reference's sequence
// (block_csr.hpp:203-214, split_block_csr.hpp:100-118), so FP64 results equal
// the reference CPU path bit for bit.  A row too long to stage on its own is a
// "long" tile, processed with threads over components (coalesced for wide
// blocks such as bs = 1296).

#include <algorithm>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

constexpr int kStage = 1024;      // staged values (products) per tile: 4 per thread
constexpr int kRowCap = 1024;     // rows per tile (outputs are bounded by kStage too)

template<class T>
struct SpmvArgs {
    const int* tile_rows;
    const int* rowptr;
    const int* cols;
    const T* vals;       // BSR: [entry][c]; split: off-diagonal [edge][c]; dense: [entry][br][bc]
    const T* diag;       // split view only
    const T* x;
    T* y;
    int bs;
    unsigned long long magic;   // ceil(2^32 / bs): k / bs == (k * magic) >> 32 for k < kStage
};

__device__ __forceinline__ int div_bs(int k, unsigned long long magic)
{
    return static_cast<int>((static_cast<unsigned long long>(k) * magic) >> 32);
}

// KIND 0: component-diagonal BSR, 1: split view, 2: dense BSR.
template<class T, int KIND>
__global__ void __launch_bounds__(kThreads, 8) k_spmv_tiles(SpmvArgs<T> a)
{
    constexpr int kPer = kStage / kThreads;   // staged units per thread
    __shared__ T prod[kStage];
    const int tile = blockIdx.x;
    const int r0 = a.tile_rows[tile], r1 = a.tile_rows[tile + 1];
    const int e0 = a.rowptr[r0], e1 = a.rowptr[r1];
    const int bs = a.bs;
    const int units = (e1 - e0) * bs;   // products (KIND 0/1) or block-row contributions (KIND 2)

    if (units > kStage || (r1 - r0) * bs > kStage) {
        // Long tile: one row; threads over components.
        for (int r = r0; r < r1; ++r) {
            const int b0 = a.rowptr[r], b1 = a.rowptr[r + 1];
            for (int c = threadIdx.x; c < bs; c += kThreads) {
                const std::size_t o = static_cast<std::size_t>(r) * bs + c;
                T acc = KIND == 1 ? mul_rn(a.diag[o], a.x[o]) : T(0);
                for (int e = b0; e < b1; ++e) {
                    const std::size_t xc = static_cast<std::size_t>(a.cols[e]) * bs;
                    if (KIND == 2) {
                        const T* blk = a.vals + (static_cast<std::size_t>(e) * bs + c) * bs;
                        T contribution = 0;
                        for (int bc = 0; bc < bs; ++bc)
                            contribution = add_rn(contribution, mul_rn(blk[bc], a.x[xc + bc]));
                        acc = add_rn(acc, contribution);
                    } else {
                        acc = add_rn(acc, mul_rn(a.vals[static_cast<std::size_t>(e) * bs + c], a.x[xc + c]));
                    }
                }
                a.y[o] = acc;
            }
        }
        return;
    }

    // Row bounds of this thread's outputs, loaded early (independent of the products).
    const int outs = (r1 - r0) * bs;
    int ob[kPer], oe[kPer];
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int o = threadIdx.x + j * kThreads;
        if (o < outs) {
            const int rl = div_bs(o, a.magic);
            ob[j] = a.rowptr[r0 + rl] - e0;
            oe[j] = a.rowptr[r0 + rl + 1] - e0;
        }
    }

    if (KIND == 2) {
        // Contribution of entry e to block row br: sum_bc B[e][br][bc] x[col][bc].
        for (int k = threadIdx.x; k < units; k += kThreads) {
            const int e = div_bs(k, a.magic);
            const T* blk = a.vals + (static_cast<std::size_t>(e0) * bs + k) * bs;
            const T* xs = a.x + static_cast<std::size_t>(a.cols[e0 + e]) * bs;
            T contribution = 0;
            for (int bc = 0; bc < bs; ++bc) contribution = add_rn(contribution, mul_rn(blk[bc], xs[bc]));
            prod[k] = contribution;
        }
    } else {
        // All value and column loads first, then all x gathers: kPer
        // independent requests in flight per thread at each step.
        const T* v = a.vals + static_cast<std::size_t>(e0) * bs;
        T pv[kPer];
        int px[kPer];   // element index col*bs + c (the plan checks it fits in 31 bits)
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = threadIdx.x + j * kThreads;
            if (k < units) {
                const int e = div_bs(k, a.magic);
                pv[j] = __ldcs(v + k);
                px[j] = __ldg(a.cols + e0 + e) * bs + (k - e * bs);
            }
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = threadIdx.x + j * kThreads;
            if (k < units) prod[k] = mul_rn(pv[j], __ldg(a.x + px[j]));
        }
    }
    __syncthreads();

    const std::size_t ybase = static_cast<std::size_t>(r0) * bs;
#pragma unroll
    for (int j = 0; j < kPer; ++j) {
        const int o = threadIdx.x + j * kThreads;
        if (o < outs) {
            const int c = o - div_bs(o, a.magic) * bs;
            T acc = KIND == 1 ? mul_rn(a.diag[ybase + o], a.x[ybase + o]) : T(0);
            for (int e = ob[j]; e < oe[j]; ++e) acc = add_rn(acc, prod[e * bs + c]);
            a.y[ybase + o] = acc;
        }
    }
}

// Persistent variant for the component-diagonal and split forms: each CTA
// walks tiles blockIdx.x, +gridDim.x, ... and issues the next tile's value and
// column loads before the current tile's gather/sum/store phases, so the HBM
// stream never waits for the shared-memory phases.  Same arithmetic as
// k_spmv_tiles (bit-identical results).
template<class T, int KIND>
__global__ void __launch_bounds__(kThreads, 4) k_spmv_stream(SpmvArgs<T> a, const int4* __restrict__ meta,
                                                              int ntiles)
{
    constexpr int kPer = kStage / kThreads;
    __shared__ T prod[kStage];
    int tile = blockIdx.x;
    if (tile >= ntiles) return;
    const int bs = a.bs;
    int4 m = meta[tile];   // r0, r1, e0, e1
    T pv[kPer];
    int pc[kPer];          // column of value k (times bs plus component below)

#define OWTK_SPMV_ISSUE(t)                                                         \
    do {                                                                           \
        const int iu = ((t).w - (t).z) * bs;                                       \
        if (iu <= kStage && ((t).y - (t).x) * bs <= kStage) {                      \
            const T* iv = a.vals + static_cast<std::size_t>((t).z) * bs;           \
            _Pragma("unroll") for (int j = 0; j < kPer; ++j) {                     \
                const int k = threadIdx.x + j * kThreads;                          \
                if (k < iu) {                                                      \
                    const int e = div_bs(k, a.magic);                              \
                    pv[j] = __ldcs(iv + k);                                        \
                    pc[j] = __ldg(a.cols + (t).z + e) * bs + (k - e * bs);         \
                }                                                                  \
            }                                                                      \
        }                                                                          \
    } while (0)
    OWTK_SPMV_ISSUE(m);
    for (;;) {
        const int next = tile + static_cast<int>(gridDim.x);
        int4 mn = make_int4(0, 0, 0, 0);
        if (next < ntiles) mn = meta[next];
        const int r0 = m.x, r1 = m.y, e0 = m.z;
        const int units = (m.w - e0) * bs;
        const int outs = (r1 - r0) * bs;
        const bool longtile = units > kStage || outs > kStage;
        if (longtile) {
            for (int r = r0; r < r1; ++r) {
                const int b0 = a.rowptr[r], b1 = a.rowptr[r + 1];
                for (int c = threadIdx.x; c < bs; c += kThreads) {
                    const std::size_t o = static_cast<std::size_t>(r) * bs + c;
                    T acc = KIND == 1 ? mul_rn(a.diag[o], a.x[o]) : T(0);
                    for (int e = b0; e < b1; ++e)
                        acc = add_rn(acc, mul_rn(a.vals[static_cast<std::size_t>(e) * bs + c],
                                                 a.x[static_cast<std::size_t>(a.cols[e]) * bs + c]));
                    a.y[o] = acc;
                }
            }
            if (next >= ntiles) break;
            tile = next;
            m = mn;
            OWTK_SPMV_ISSUE(m);
            continue;
        }
        int ob[kPer], oe[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int o = threadIdx.x + j * kThreads;
            if (o < outs) {
                const int rl = div_bs(o, a.magic);
                ob[j] = a.rowptr[r0 + rl] - e0;
                oe[j] = a.rowptr[r0 + rl + 1] - e0;
            }
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = threadIdx.x + j * kThreads;
            if (k < units) prod[k] = mul_rn(pv[j], __ldg(a.x + pc[j]));
        }
        if (next < ntiles) OWTK_SPMV_ISSUE(mn);   // next tile's stream flies during the phases below
        __syncthreads();
        const std::size_t ybase = static_cast<std::size_t>(r0) * bs;
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int o = threadIdx.x + j * kThreads;
            if (o < outs) {
                const int c = o - div_bs(o, a.magic) * bs;
                T acc = KIND == 1 ? mul_rn(a.diag[ybase + o], a.x[ybase + o]) : T(0);
                for (int e = ob[j]; e < oe[j]; ++e) acc = add_rn(acc, prod[e * bs + c]);
                a.y[ybase + o] = acc;
            }
        }
        __syncthreads();
        if (next >= ntiles) break;
        tile = next;
        m = mn;
    }
#undef OWTK_SPMV_ISSUE
}

// First diagonal entry of every row (block_csr.hpp:217-236).
template<class T>
__global__ void k_bsr_diagonal(int owned, int bs, const int* rowptr, const int* cols, const T* vals,
                               T* out, unsigned* status)
{
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= owned) return;
    for (int e = rowptr[r]; e < rowptr[r + 1]; ++e) {
        if (cols[e] == r) {
            for (int c = 0; c < bs; ++c)
                out[static_cast<std::size_t>(r) * bs + c] = vals[static_cast<std::size_t>(e) * bs + c];
            return;
        }
    }
    atomicOr(status, kErrMissingDiagonal);
}

template<class T>
__global__ void k_gather_values(std::size_t entries, int bs, const std::int64_t* source, const T* values,
                                T* out)
{
    const std::size_t k = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= entries * bs) return;
    const std::size_t e = k / bs, c = k - e * bs;
    const std::int64_t s = source[e];
    out[k] = s < 0 ? T(0) : values[static_cast<std::size_t>(s) * bs + c];
}

}  // namespace

namespace kern {

template<class T> void spmv(Context& c, const Matrix& m, const T* x, T* y)
{
    if (m.plan.tiles == 0) return;
    SpmvArgs<T> a;
    a.tile_rows = m.plan.tile_rows.as<int>();
    a.rowptr = m.rowptr.as<int>();
    a.cols = m.cols.as<int>();
    a.vals = static_cast<const T*>(m.value_ptr());
    a.diag = static_cast<const T*>(m.diag);
    a.x = x;
    a.y = y;
    a.bs = static_cast<int>(m.bs);
    a.magic = ((1ull << 32) + m.bs - 1) / m.bs;
    const unsigned grid = static_cast<unsigned>(m.plan.tiles);
    const unsigned persistent = std::min<unsigned>(grid, static_cast<unsigned>(c.sm_count) * 4);
    const int4* meta = m.plan.tile_meta.as<int4>();
    if (m.kind == 0) k_spmv_stream<T, 0><<<persistent, kThreads, 0, c.stream>>>(a, meta, m.plan.tiles);
    else if (m.kind == 1) k_spmv_stream<T, 1><<<persistent, kThreads, 0, c.stream>>>(a, meta, m.plan.tiles);
    else k_spmv_tiles<T, 2><<<grid, kThreads, 0, c.stream>>>(a);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void bsr_diagonal(Context& c, const Matrix& m, T* out)
{
    const int owned = static_cast<int>(m.owned);
    k_bsr_diagonal<T><<<(owned + 255) / 256, 256, 0, c.stream>>>(
        owned, static_cast<int>(m.bs), m.rowptr.as<int>(), m.cols.as<int>(),
        static_cast<const T*>(m.values.ptr), out, c.status.as<unsigned>());
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void gather_values(Context& c, std::size_t entries, std::size_t bs,
                                     const std::int64_t* source, const T* values, T* out)
{
    const std::size_t total = entries * bs;
    if (total == 0) return;
    k_gather_values<T><<<static_cast<unsigned>((total + 255) / 256), 256, 0, c.stream>>>(
        entries, static_cast<int>(bs), source, values, out);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template void spmv<double>(Context&, const Matrix&, const double*, double*);
template void spmv<float>(Context&, const Matrix&, const float*, float*);
template void bsr_diagonal<double>(Context&, const Matrix&, double*);
template void bsr_diagonal<float>(Context&, const Matrix&, float*);
template void gather_values<double>(Context&, std::size_t, std::size_t, const std::int64_t*, const double*, double*);
template void gather_values<float>(Context&, std::size_t, std::size_t, const std::int64_t*, const float*, float*);

}  // namespace kern

// Tile plan: greedy runs of rows under the stage limits.
void build_tile_plan(Matrix& m)
{
    const int bs = static_cast<int>(m.bs);
    if ((m.owned + m.ghost) * m.bs >= (1ull << 31))
        fail(OWTK_ERR_INVALID_ARGUMENT, "vector too large for 32-bit element indices");
    std::vector<std::int32_t> tiles{0};
    int units = 0, rows = 0;
    for (std::size_t r = 0; r < m.owned; ++r) {
        const int deg = m.h_rowptr[r + 1] - m.h_rowptr[r];
        const long long row_units = static_cast<long long>(deg) * bs;
        const bool fits = units + row_units <= kStage && rows + 1 <= kRowCap
            && static_cast<long long>(rows + 1) * bs <= kStage;
        if (!fits && rows > 0) {
            tiles.push_back(static_cast<std::int32_t>(r));
            units = 0;
            rows = 0;
        }
        units += static_cast<int>(row_units > kStage ? kStage + 1 : row_units);
        rows += 1;
        if (row_units > kStage || static_cast<long long>(bs) > kStage) {
            // A row that cannot be staged is a tile of its own.
            tiles.push_back(static_cast<std::int32_t>(r + 1));
            units = 0;
            rows = 0;
        }
    }
    if (rows > 0) tiles.push_back(static_cast<std::int32_t>(m.owned));
    m.plan.tiles = static_cast<int>(tiles.size()) - 1;
    m.plan.tile_values = kStage;
    m.plan.tile_rows = upload(m.ctx->stream, tiles);
    std::vector<std::int32_t> meta(4 * static_cast<std::size_t>(m.plan.tiles));
    for (int t = 0; t < m.plan.tiles; ++t) {
        meta[4 * t + 0] = tiles[t];
        meta[4 * t + 1] = tiles[t + 1];
        meta[4 * t + 2] = m.h_rowptr[tiles[t]];
        meta[4 * t + 3] = m.h_rowptr[tiles[t + 1]];
    }
    m.plan.tile_meta = upload(m.ctx->stream, meta);
}

}  // namespace owtk
