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
#include <cstdint>
#include <cstdlib>
#include <utility>
#include <vector>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

#ifndef OWTK_SPMV_STAGE
#define OWTK_SPMV_STAGE 1024
#endif
constexpr int kStage = OWTK_SPMV_STAGE;   // staged values (products) per tile
constexpr int kRowCap = kStage < 1024 ? kStage : 1024;   // rows per tile (outputs are bounded by kStage too)

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

// KIND 0: component-diagonal BSR, 1: split view, 2: dense BSR.  BS: dense
// block size known at compile time (0: any); those instances load every
// operand of a thread's units before the first product and keep two CTAs
// per SM for the registers that takes.
template<class T, int KIND, int BS = 0>
__global__ void __launch_bounds__(kThreads, (KIND == 2 && BS > 0) ? 2 : 4) k_spmv_tiles(SpmvArgs<T> a)
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

    if (KIND == 2 && BS > 0) {
        // Contribution of entry e to block row br: sum_bc B[e][br][bc] x[col][bc]
        // (summed from +0 over bc), with all of this thread's block-row
        // values, columns and x blocks requested before the arithmetic.
        T bv[kPer][BS > 0 ? BS : 1], xv[kPer][BS > 0 ? BS : 1];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = threadIdx.x + j * kThreads;
            if (k < units) {
                const int e = div_bs(k, a.magic);
                const T* blk = a.vals + (static_cast<std::size_t>(e0) * BS + k) * BS;
                const T* xs = a.x + static_cast<std::size_t>(__ldg(a.cols + e0 + e)) * BS;
#pragma unroll
                for (int bc = 0; bc < BS; ++bc) {
                    bv[j][bc] = __ldcs(blk + bc);
                    xv[j][bc] = __ldg(xs + bc);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = threadIdx.x + j * kThreads;
            if (k < units) {
                T contribution = 0;
#pragma unroll
                for (int bc = 0; bc < BS; ++bc) contribution = add_rn(contribution, mul_rn(bv[j][bc], xv[j][bc]));
                prod[k] = contribution;
            }
        }
    } else if (KIND == 2) {
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

// ------------------------------------------------------------------ bulk
// Persistent bulk-copy pipeline for the component-diagonal and split forms.
//
// A CTA owns a contiguous run of tiles.  Its producer warp streams each tile's
// value run, column run and row offsets into a kBulkStages-deep shared-memory
// ring with cp.async.bulk (completion counted in bytes on the stage's "full"
// mbarrier; L2 evict-first on the streams so that x stays L2-resident), while
// the eight consumer warps of the previous stages gather x, form the rounded
// products in place and add them per output in entry order (the same
// arithmetic as k_spmv_tiles, bit-identical results), then release the stage
// on its "empty" mbarrier.  Every copy covers whole 16-byte granules: the
// granule-aligned superset of the tile's runs, clipped to the last whole
// granule of each array, with the at most 15 trailing bytes of an array read
// by plain loads.  Every wait is bounded; a wait that gives up sets the
// timeout bit and the consumers leave together at their next named barrier.
#ifndef OWTK_BULK_STAGES
#define OWTK_BULK_STAGES 3
#endif
#ifndef OWTK_BULK_CONSUMERS
#define OWTK_BULK_CONSUMERS 128
#endif
#ifndef OWTK_BULK_CTAS_PER_SM
#define OWTK_BULK_CTAS_PER_SM 4
#endif
constexpr int kBulkStages = OWTK_BULK_STAGES;
constexpr int kBulkConsumers = OWTK_BULK_CONSUMERS;
constexpr int kBulkThreads = kBulkConsumers + 32;
constexpr int kBulkCtasPerSm = OWTK_BULK_CTAS_PER_SM;
constexpr int kBulkSpin = 1 << 20;

struct BulkHead {          // written by the producer before the stage's arrival
    int r0, r1, e0, e1;
    int voff, vavail;      // value k of the tile sits at vals[voff + k] if k < vavail
    int coff, cavail;
    int roff, ravail;
    int longtile, pad;
};

template<class T>
struct BulkLayout {
    static constexpr int round128(int b) { return (b + 127) / 128 * 128; }
    static constexpr int kVals = round128(kStage * static_cast<int>(sizeof(T)) + 16);
    static constexpr int kCols = round128(kStage * 4 + 16);
    static constexpr int kRows = round128((kRowCap + 1) * 4 + 16);
    static constexpr int kHead = 128;
    static constexpr int kStageBytes = kVals + kCols + kRows + kHead;
    static constexpr int kBars = 128;    // 2 * kBulkStages mbarriers
    static constexpr int kTotal = kBars + kBulkStages * kStageBytes;
    static_assert(2 * kBulkStages * 8 <= kBars, "mbarrier area");
};


// Products of one staged tile, written in place over the staged values.
// BS > 0: block size known at compile time; thread t takes entries t, t+C, ...
// and all BS components of each (one column load per entry, BS independent
// gathers).  BS == 0: any block size; thread t takes values t, t+C, ...
template<class T, int BS>
__device__ __forceinline__ void bulk_products(const SpmvArgs<T>& a, const BulkHead* h, T* sv, const int* sc, int t)
{
    const int e0 = h->e0, ne = h->e1 - e0;
    const int voff = h->voff, vavail = h->vavail, coff = h->coff, cavail = h->cavail;
    const std::size_t vbase = static_cast<std::size_t>(e0) * (BS > 0 ? BS : a.bs);
    if constexpr (BS > 0) {
        constexpr int kEpt = (kStage / BS + kBulkConsumers - 1) / kBulkConsumers;
        T pv[kEpt][BS], px[kEpt][BS];
#pragma unroll
        for (int j = 0; j < kEpt; ++j) {
            const int el = t + j * kBulkConsumers;
            if (el < ne) {
                const int col = el < cavail ? sc[coff + el] : a.cols[e0 + el];
                const T* xs = a.x + col * BS;
#pragma unroll
                for (int c = 0; c < BS; ++c) {
                    const int k = el * BS + c;
                    pv[j][c] = k < vavail ? sv[voff + k] : a.vals[vbase + k];
                    px[j][c] = __ldg(xs + c);
                }
            }
        }
#pragma unroll
        for (int j = 0; j < kEpt; ++j) {
            const int el = t + j * kBulkConsumers;
            if (el < ne) {
#pragma unroll
                for (int c = 0; c < BS; ++c) sv[voff + el * BS + c] = mul_rn(pv[j][c], px[j][c]);
            }
        }
    } else {
        constexpr int kPer = (kStage + kBulkConsumers - 1) / kBulkConsumers;
        const int bs = a.bs, units = ne * bs;
        T pv[kPer], px[kPer];
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = t + j * kBulkConsumers;
            if (k < units) {
                const int e = div_bs(k, a.magic);
                pv[j] = k < vavail ? sv[voff + k] : a.vals[vbase + k];
                const int col = e < cavail ? sc[coff + e] : a.cols[e0 + e];
                px[j] = __ldg(a.x + col * bs + (k - e * bs));
            }
        }
#pragma unroll
        for (int j = 0; j < kPer; ++j) {
            const int k = t + j * kBulkConsumers;
            if (k < units) sv[voff + k] = mul_rn(pv[j], px[j]);
        }
    }
}
// Sums of one staged tile: thread t owns outputs (row, component) t, t+C, ...
// and adds its row's staged products in entry order (eight loaded ahead of
// the add chain), the reference's summation sequence.
template<class T, int KIND, int BS>
__device__ __forceinline__ void bulk_sums(const SpmvArgs<T>& a, const BulkHead* h, const T* sv, const int* sr, int t)
{
    const int bs = BS > 0 ? BS : a.bs;
    const int r0 = h->r0, e0 = h->e0, outs = (h->r1 - r0) * bs;
    const int voff = h->voff, roff = h->roff, ravail = h->ravail;
    const std::size_t ybase = static_cast<std::size_t>(r0) * bs;
    for (int o = t; o < outs; o += kBulkConsumers) {
        const int rl = BS > 0 ? o / BS : div_bs(o, a.magic), c = o - rl * bs;
        const int b0 = (rl < ravail ? sr[roff + rl] : a.rowptr[r0 + rl]) - e0;
        const int b1 = (rl + 1 < ravail ? sr[roff + rl + 1] : a.rowptr[r0 + rl + 1]) - e0;
        T acc = T(0);
        if constexpr (KIND == 1) acc = mul_rn(a.diag[ybase + o], a.x[ybase + o]);
        const T* p = sv + voff + c;
        for (int e = b0; e < b1; e += 8) {
            T q[8];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (e + i < b1) q[i] = p[(e + i) * bs];
#pragma unroll
            for (int i = 0; i < 8; ++i)
                if (e + i < b1) acc = add_rn(acc, q[i]);
        }
        a.y[ybase + o] = acc;
    }
}

template<class T, int KIND, int BS>
__global__ void __launch_bounds__(kBulkThreads, kBulkCtasPerSm)
    k_spmv_bulk(SpmvArgs<T> a, const int4* __restrict__ meta, int ntiles, std::size_t entries, std::size_t owned,
                unsigned* status)
{
    using L = BulkLayout<T>;
    extern __shared__ __align__(128) unsigned char smem[];
    const std::uint32_t bars = smem_u32(smem);     // full[0..S), empty[0..S)
    unsigned char* stages = smem + L::kBars;
    const int bs = BS > 0 ? BS : a.bs;
    const long long nb = gridDim.x;
    const int t_begin = static_cast<int>(static_cast<long long>(ntiles) * blockIdx.x / nb);
    const int t_end = static_cast<int>(static_cast<long long>(ntiles) * (blockIdx.x + 1) / nb);
    const int count = t_end - t_begin;

    if (threadIdx.x == 0) {
        for (int s = 0; s < kBulkStages; ++s) {
            mbar_init(bars + 8 * s, 1);
            mbar_init(bars + 8 * (kBulkStages + s), kBulkConsumers / 32);
        }
        fence_proxy_async_smem();
    }
    __syncthreads();

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == kBulkConsumers / 32) {
        // ------------------------------------------------------------ producer
        const std::uint64_t policy = l2_policy_evict_first();
        bool ok = true;
        int issued = 0;
        for (int i0 = 0; i0 < count && ok; i0 += 32) {
            int4 mine = make_int4(0, 0, 0, 0);
            if (i0 + lane < count) mine = meta[t_begin + i0 + lane];
            const int batch = min(32, count - i0);
            for (int j = 0; j < batch; ++j) {
                int4 m;
                m.x = __shfl_sync(0xffffffffu, mine.x, j);
                m.y = __shfl_sync(0xffffffffu, mine.y, j);
                m.z = __shfl_sync(0xffffffffu, mine.z, j);
                m.w = __shfl_sync(0xffffffffu, mine.w, j);
                const int it = i0 + j, s = it % kBulkStages, use = it / kBulkStages;
                int good = 1;
                if (lane == 0) {
                    const std::uint32_t full = bars + 8 * s, empty = bars + 8 * (kBulkStages + s);
                    if (!mbar_wait_bounded(empty, (use & 1) ^ 1, kBulkSpin)) {
                        atomicOr(status, kErrTimeout);
                        good = 0;
                    } else {
                        unsigned char* st = stages + static_cast<std::size_t>(s) * L::kStageBytes;
                        BulkHead* h = reinterpret_cast<BulkHead*>(st + L::kVals + L::kCols + L::kRows);
                        const int units = (m.w - m.z) * bs, outs = (m.y - m.x) * bs;
                        h->r0 = m.x;
                        h->r1 = m.y;
                        h->e0 = m.z;
                        h->e1 = m.w;
                        h->longtile = units > kStage || outs > kStage;
                        std::uint32_t bytes = 0, bv = 0, bc = 0, br = 0;
                        std::size_t lv = 0, lc = 0, lr = 0;
                        if (!h->longtile) {
                            bv = bulk_segment(static_cast<std::size_t>(m.z) * bs, static_cast<std::size_t>(m.w) * bs,
                                              entries * bs, sizeof(T), lv, h->voff, h->vavail);
                            bc = bulk_segment(m.z, m.w, entries, 4, lc, h->coff, h->cavail);
                            br = bulk_segment(m.x, static_cast<std::size_t>(m.y) + 1, owned + 1, 4, lr, h->roff,
                                              h->ravail);
                            bytes = bv + bc + br;
                        }
                        if (bytes == 0) {
                            mbar_arrive(full);
                        } else {
                            mbar_arrive_expect_tx(full, bytes);
                            if (bv) bulk_load(smem_u32(st), reinterpret_cast<const unsigned char*>(a.vals) + lv, bv,
                                              full, policy);
                            if (bc) bulk_load(smem_u32(st + L::kVals),
                                              reinterpret_cast<const unsigned char*>(a.cols) + lc, bc, full, policy);
                            if (br) bulk_load(smem_u32(st + L::kVals + L::kCols),
                                              reinterpret_cast<const unsigned char*>(a.rowptr) + lr, br, full, policy);
                        }
                        ++issued;
                    }
                }
                ok = __shfl_sync(0xffffffffu, good, 0) != 0;
                if (!ok) break;
            }
        }
        // Leave only after every issued copy has landed.
        if (lane == 0) {
            for (int it = max(0, issued - kBulkStages); it < issued; ++it)
                if (!mbar_wait_bounded(bars + 8 * (it % kBulkStages), (it / kBulkStages) & 1, kBulkSpin))
                    atomicOr(status, kErrTimeout);
        }
        return;
    }

    // ---------------------------------------------------------------- consumers
    // All consumers of the CTA meet at one named barrier per tile (products
    // visible before the sums); a wait that gives up is reported through that
    // barrier, so they leave together.
    const int t = threadIdx.x;
    for (int it = 0; it < count; ++it) {
        const int s = it % kBulkStages, use = it / kBulkStages;
        const bool ready = mbar_wait_bounded(bars + 8 * s, use & 1, kBulkSpin);
        unsigned char* st = stages + static_cast<std::size_t>(s) * L::kStageBytes;
        T* sv = reinterpret_cast<T*>(st);
        const int* sc = reinterpret_cast<const int*>(st + L::kVals);
        const int* sr = reinterpret_cast<const int*>(st + L::kVals + L::kCols);
        const BulkHead* h = reinterpret_cast<const BulkHead*>(st + L::kVals + L::kCols + L::kRows);
        const int longtile = ready ? h->longtile : 0;
        if (ready && longtile) {
            const int r0 = h->r0, r1 = h->r1;
            for (int r = r0; r < r1; ++r) {
                const int b0 = a.rowptr[r], b1 = a.rowptr[r + 1];
                for (int c = t; c < bs; c += kBulkConsumers) {
                    const std::size_t o = static_cast<std::size_t>(r) * bs + c;
                    T acc = KIND == 1 ? mul_rn(a.diag[o], a.x[o]) : T(0);
                    for (int e = b0; e < b1; ++e)
                        acc = add_rn(acc, mul_rn(a.vals[static_cast<std::size_t>(e) * bs + c],
                                                 a.x[static_cast<std::size_t>(a.cols[e]) * bs + c]));
                    a.y[o] = acc;
                }
            }
        } else if (ready) {
            bulk_products<T, BS>(a, h, sv, sc, t);
        }
        if (bar_any(1, kBulkConsumers, !ready)) {
            if (t == 0) atomicOr(status, kErrTimeout);
            return;
        }
        if (!longtile) bulk_sums<T, KIND, BS>(a, h, sv, sr, t);
        // The next fill of this stage is an async-proxy write after our
        // generic-proxy product writes.
        fence_proxy_async_smem();
        __syncwarp();
        if (lane == 0) mbar_arrive(bars + 8 * (kBulkStages + s));
    }
}

template<class T, int KIND, int BS>
void launch_bulk(Context& c, const SpmvArgs<T>& a, const Matrix& m)
{
    const int smem = BulkLayout<T>::kTotal;
    const unsigned grid = std::min<unsigned>(static_cast<unsigned>(m.plan.tiles),
                                             static_cast<unsigned>(c.sm_count) * kBulkCtasPerSm);
    OWTK_CUDA(cudaFuncSetAttribute(k_spmv_bulk<T, KIND, BS>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    k_spmv_bulk<T, KIND, BS><<<grid, kBulkThreads, smem, c.stream>>>(
        a, m.plan.tile_meta.as<int4>(), m.plan.tiles, m.entries, m.owned, c.status.as<unsigned>());
}

// Warp-shuffle SpMV (component-diagonal or split, block size BS <= 4): a warp
// takes 32 consecutive rows, lane l owning row 32 w + l.  The rows' entries
// are walked 32 at a time, lane l loading entry s + l (column, its BS values
// and x gathers; coalesced value loads) and forming its products; each owner
// then adds its row's products of the step in entry order, fetched from the
// producing lanes by shuffles.  Sum from +0 (split: from d x), products and
// adds rounded as written: the reference's sequence, so the bits match.
template<class T, int KIND, int BS>
__global__ void __launch_bounds__(256) k_spmv_warp(SpmvArgs<T> a, int owned)
{
    const int lane = threadIdx.x & 31;
    const long long gw = static_cast<long long>(blockIdx.x) * 8 + (threadIdx.x >> 5);
    const long long nw = static_cast<long long>(gridDim.x) * 8;
    const long long nchunks = (static_cast<long long>(owned) + 31) / 32;
    // Row offsets of the next chunk are loaded one chunk ahead; within a
    // chunk, columns two steps ahead and values and x one step ahead.
    const auto row_bounds = [&](long long ch, int& p0, int& p1) {
        const long long rr = ch * 32 + lane;
        p0 = p1 = 0;
        if (ch < nchunks && rr < owned) {
            p0 = __ldg(a.rowptr + rr);
            p1 = __ldg(a.rowptr + rr + 1);
        }
    };
    int np0, np1;
    row_bounds(gw, np0, np1);
    for (long long ch = gw; ch < nchunks; ch += nw) {
        const int r0 = static_cast<int>(ch) * 32, r = r0 + lane;
        const bool own = r < owned;
        const int rp0 = np0, rp1 = np1;
        row_bounds(ch + nw, np0, np1);
        const int last = min(31, owned - 1 - r0);
        const int ea = __shfl_sync(0xffffffffu, rp0, 0), eb = __shfl_sync(0xffffffffu, rp1, last);
        T acc[BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) {
            acc[c] = T(0);
            if constexpr (KIND == 1)
                if (own) acc[c] = mul_rn(a.diag[static_cast<std::size_t>(r) * BS + c], a.x[static_cast<std::size_t>(r) * BS + c]);
        }
        const auto load_col = [&](int s) { return s + lane < eb ? __ldg(a.cols + s + lane) : -1; };
        const auto load_vx = [&](int s, int col, T (&v)[BS], T (&xv)[BS]) {
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                v[c] = T(0);
                xv[c] = T(0);
                if (col >= 0) {
                    v[c] = __ldg(a.vals + static_cast<std::size_t>(s + lane) * BS + c);
                    xv[c] = __ldg(a.x + static_cast<std::size_t>(col) * BS + c);
                }
            }
        };
        int col1 = load_col(ea + 32);
        T v[BS], xv[BS];
        load_vx(ea, load_col(ea), v, xv);
        for (int s = ea; s < eb; s += 32) {
            // Next step's values and x (its columns arrived a step ago), then
            // the step after next's columns.
            T vn[BS], xn[BS];
            load_vx(s + 32, col1, vn, xn);
            col1 = load_col(s + 64);
            T p[BS];
#pragma unroll
            for (int c = 0; c < BS; ++c) p[c] = mul_rn(v[c], xv[c]);
            const int lo = max(rp0 - s, 0), hi = min(rp1 - s, 32);
            const int cnt = own ? max(hi - lo, 0) : 0;
            const int kmax = static_cast<int>(__reduce_max_sync(0xffffffffu, static_cast<unsigned>(cnt)));
            for (int k = 0; k < kmax; ++k) {
                const int src = min(lo + k, 31);
#pragma unroll
                for (int c = 0; c < BS; ++c) {
                    const T q = __shfl_sync(0xffffffffu, p[c], src);
                    if (k < cnt) acc[c] = add_rn(acc[c], q);
                }
            }
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                v[c] = vn[c];
                xv[c] = xn[c];
            }
        }
        if (own)
#pragma unroll
            for (int c = 0; c < BS; ++c) a.y[static_cast<std::size_t>(r) * BS + c] = acc[c];
    }
}

template<class T, int KIND>
bool launch_warp_bs(Context& c, const SpmvArgs<T>& a, const Matrix& m)
{
    const int owned = static_cast<int>(m.owned);
    const long long chunks = (static_cast<long long>(owned) + 31) / 32;
    const unsigned grid = static_cast<unsigned>(std::max<long long>(1, std::min<long long>((chunks + 7) / 8,
                                                                                          c.sm_count * 8)));
    switch (m.bs) {
    case 1: k_spmv_warp<T, KIND, 1><<<grid, 256, 0, c.stream>>>(a, owned); return true;
    case 2: k_spmv_warp<T, KIND, 2><<<grid, 256, 0, c.stream>>>(a, owned); return true;
    case 3: k_spmv_warp<T, KIND, 3><<<grid, 256, 0, c.stream>>>(a, owned); return true;
    case 4: k_spmv_warp<T, KIND, 4><<<grid, 256, 0, c.stream>>>(a, owned); return true;
    default: return false;
    }
}

template<class T, int KIND>
void launch_bulk_bs(Context& c, const SpmvArgs<T>& a, const Matrix& m)
{
    switch (m.bs) {
    case 1: launch_bulk<T, KIND, 1>(c, a, m); break;
    case 2: launch_bulk<T, KIND, 2>(c, a, m); break;
    case 3: launch_bulk<T, KIND, 3>(c, a, m); break;
    // bs 4: entry-major products put a thread's 4 staged values 32 bytes
    // apart, four threads per bank group (4-way conflicts on every access);
    // the value-major generic path is conflict-free.
    default: launch_bulk<T, KIND, 0>(c, a, m); break;
    }
}

// Row-slice SpMV (component-diagonal BSR, block size BS <= 4): a warp takes a
// slice of 32 rows, lane j the slice's j-th longest row, and walks the
// slice's packed steps: at step k the n_k lanes whose row is longer than k
// load their entry's column (one coalesced run) and BS values (BS coalesced
// runs of n_k elements), gather x from L2 and add the rounded product to
// their own sums; a row's products are added from +0 in entry order, the
// reference's sequence (block_csr.hpp:203-214), so the bits match.  Columns
// are loaded two steps ahead, x one step ahead, values VD steps ahead, and the
// next slice's lane word and first entry during this slice.  The sums are put
// back in row order through shared memory and stored as one coalesced run
// of 32 * BS elements.  Long rows (length 0 here) are written afterwards by
// the row-list kernel.
template<class T, int BS, int MINB, int VD>
__global__ void __launch_bounds__(256, MINB) k_spmv_slices(const int* __restrict__ base,
                                                           const unsigned short* __restrict__ lanes,
                                                           const int* __restrict__ scols, const T* __restrict__ svals,
                                                           const T* __restrict__ x, T* __restrict__ y, int slices,
                                                           int owned)
{
    __shared__ T out[8][32 * BS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nw = static_cast<int>(gridDim.x) * 8;
    int s = static_cast<int>(blockIdx.x) * 8 + wib;
    // This slice's lane word and first entry, loaded one slice ahead.
    unsigned meta = s < slices ? lanes[static_cast<long long>(s) * 32 + lane] : 0u;
    int off = s < slices ? base[s] : 0;
    for (; s < slices; s += nw) {
        const int len = static_cast<int>(meta >> 8), pos = static_cast<int>(meta & 255u);
        const int steps = __shfl_sync(0xffffffffu, len, 0);   // lane 0 holds the longest row
        const int sn = s + nw;
        meta = sn < slices ? lanes[static_cast<long long>(sn) * 32 + lane] : 0u;
        const int off_next = sn < slices ? base[sn] : 0;
        T acc[BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] = T(0);
        const auto count = [&](int k) { return __popc(__ballot_sync(0xffffffffu, len > k)); };
        const auto load_v = [&](int k, int o, int n, T (&vv)[BS]) {
            if (len > k) {
                const T* vp = svals + static_cast<long long>(o) * BS + lane;
#pragma unroll
                for (int c = 0; c < BS; ++c) vv[c] = __ldcs(vp + c * n);
            }
        };
        const auto load_x = [&](int k, int col, T (&xx)[BS]) {
            if (len > k) {
                const T* xp = x + static_cast<long long>(col) * BS;
#pragma unroll
                for (int c = 0; c < BS; ++c) xx[c] = __ldg(xp + c);
            }
        };
        const auto load_col = [&](int k, int o) { return len > k ? __ldcs(scols + o + lane) : 0; };
        // Values VD steps ahead, x one step ahead, columns two steps ahead.
        T v[VD + 1][BS], xv[BS];
        int o[VD + 2], n[VD + 2];
        o[0] = off;
        n[0] = count(0);
#pragma unroll
        for (int i = 1; i < VD + 2; ++i) {
            o[i] = o[i - 1] + n[i - 1];
            n[i] = count(i);
        }
#pragma unroll
        for (int i = 0; i < VD; ++i) load_v(i, o[i], n[i], v[i]);
        const int col0 = load_col(0, o[0]);
        int col1 = load_col(1, o[1]);
        load_x(0, col0, xv);
        for (int k = 0; k < steps; ++k) {
            load_v(k + VD, o[VD], n[VD], v[VD]);
            T xn[BS];
            load_x(k + 1, col1, xn);
            col1 = load_col(k + 2, o[2]);
            if (len > k)
#pragma unroll
                for (int c = 0; c < BS; ++c) acc[c] = add_rn(acc[c], mul_rn(v[0][c], xv[c]));
#pragma unroll
            for (int i = 0; i < VD; ++i)
#pragma unroll
                for (int c = 0; c < BS; ++c) v[i][c] = v[i + 1][c];
#pragma unroll
            for (int c = 0; c < BS; ++c) xv[c] = xn[c];
#pragma unroll
            for (int i = 0; i < VD + 1; ++i) {
                o[i] = o[i + 1];
                n[i] = n[i + 1];
            }
            o[VD + 1] = o[VD] + n[VD];
            n[VD + 1] = count(k + VD + 2);
        }
        if (pos < 32)
#pragma unroll
            for (int c = 0; c < BS; ++c) out[wib][pos * BS + c] = acc[c];
        __syncwarp();
        const int rows = min(32, owned - 32 * s);
        T* ys = y + static_cast<long long>(s) * 32 * BS;
        for (int i = lane; i < rows * BS; i += 32) ys[i] = out[wib][i];
        __syncwarp();
        off = off_next;
    }
}

// Dense-block BSR (DenseBlockCsrMatrix, bs <= 4) on the same row-slice
// layout with BS * BS value runs per step ([block row][block column][lane]):
// per entry and block row the contribution sums B[br][bc] x[bc] from +0 over
// bc, then adds to the row's sum — the reference's sequence
// (dense_block_csr.hpp:173-205), as k_spmv_tiles evaluates it.  Columns two
// steps ahead, values and x one step ahead.
template<class T, int BS, int MINB>
__global__ void __launch_bounds__(256, MINB) k_spmv_slices_dense(const int* __restrict__ base,
                                                                 const unsigned short* __restrict__ lanes,
                                                                 const int* __restrict__ scols,
                                                                 const T* __restrict__ svals, const T* __restrict__ x,
                                                                 T* __restrict__ y, int slices, int owned)
{
    constexpr int P = BS * BS;
    __shared__ T out[8][32 * BS];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    const int nw = static_cast<int>(gridDim.x) * 8;
    for (int s = static_cast<int>(blockIdx.x) * 8 + wib; s < slices; s += nw) {
        const unsigned meta = lanes[static_cast<long long>(s) * 32 + lane];
        const int len = static_cast<int>(meta >> 8), pos = static_cast<int>(meta & 255u);
        const int steps = __shfl_sync(0xffffffffu, len, 0);
        T acc[BS];
#pragma unroll
        for (int c = 0; c < BS; ++c) acc[c] = T(0);
        const auto count = [&](int k) { return __popc(__ballot_sync(0xffffffffu, len > k)); };
        const auto load_vx = [&](int k, int o, int n, int col, T (&vv)[P], T (&xx)[BS]) {
            if (len > k) {
                const T* vp = svals + static_cast<long long>(o) * P + lane;
                const T* xp = x + static_cast<long long>(col) * BS;
#pragma unroll
                for (int q = 0; q < P; ++q) vv[q] = __ldcs(vp + q * n);
#pragma unroll
                for (int c = 0; c < BS; ++c) xx[c] = __ldg(xp + c);
            }
        };
        const auto load_col = [&](int k, int o) { return len > k ? __ldcs(scols + o + lane) : 0; };
        int o0 = base[s], n0 = count(0);
        int o1 = o0 + n0, n1 = count(1);
        T v[P], xv[BS];
        load_vx(0, o0, n0, load_col(0, o0), v, xv);
        int col1 = load_col(1, o1);
        for (int k = 0; k < steps; ++k) {
            T vn[P], xn[BS];
            load_vx(k + 1, o1, n1, col1, vn, xn);
            const int o2 = o1 + n1, n2 = count(k + 2);
            col1 = load_col(k + 2, o2);
            if (len > k) {
#pragma unroll
                for (int br = 0; br < BS; ++br) {
                    T part = T(0);
#pragma unroll
                    for (int bc = 0; bc < BS; ++bc) part = add_rn(part, mul_rn(v[br * BS + bc], xv[bc]));
                    acc[br] = add_rn(acc[br], part);
                }
            }
#pragma unroll
            for (int q = 0; q < P; ++q) v[q] = vn[q];
#pragma unroll
            for (int c = 0; c < BS; ++c) xv[c] = xn[c];
            o1 = o2;
            n1 = n2;
        }
        if (pos < 32)
#pragma unroll
            for (int c = 0; c < BS; ++c) out[wib][pos * BS + c] = acc[c];
        __syncwarp();
        const int rows = min(32, owned - 32 * s);
        T* ys = y + static_cast<long long>(s) * 32 * BS;
        for (int i = lane; i < rows * BS; i += 32) ys[i] = out[wib][i];
        __syncwarp();
    }
}

// Fill the row-slice copy from the CSR arrays: a warp per slice walks the
// same steps as the row-slice kernels and writes each entry's `per` values
// (bs, or bs * bs for dense blocks) where they read them.
template<class T>
__global__ void __launch_bounds__(256) k_slices_fill(const int* __restrict__ base,
                                                     const unsigned short* __restrict__ lanes,
                                                     const int* __restrict__ rowptr, const int* __restrict__ cols,
                                                     const T* __restrict__ vals, int* __restrict__ scols,
                                                     T* __restrict__ svals, int slices, int per)
{
    const int lane = threadIdx.x & 31;
    const int s = static_cast<int>(blockIdx.x) * 8 + static_cast<int>(threadIdx.x >> 5);
    if (s >= slices) return;
    const unsigned meta = lanes[static_cast<long long>(s) * 32 + lane];
    const int len = static_cast<int>(meta >> 8), pos = static_cast<int>(meta & 255u);
    const int steps = __shfl_sync(0xffffffffu, len, 0);
    const int e0 = len > 0 ? rowptr[32 * s + pos] : 0;
    int off = base[s];
    for (int k = 0; k < steps; ++k) {
        const int n = __popc(__ballot_sync(0xffffffffu, len > k));
        if (len > k) {
            const int e = e0 + k;
            scols[off + lane] = cols[e];
            for (int c = 0; c < per; ++c)
                svals[static_cast<long long>(off) * per + static_cast<long long>(c) * n + lane] =
                    vals[static_cast<long long>(e) * per + c];
        }
        off += n;
    }
}

template<class T, int BS, int MINB, int VD>
void launch_slices_v(Context& c, const Matrix& m, const T* x, T* y)
{
    static int per_sm = 0;
    if (per_sm == 0) {
        OWTK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmv_slices<T, BS, MINB, VD>, 256, 0));
        per_sm = std::max(per_sm, 1);
    }
    const RowSlices& sl = m.slices;
    const unsigned grid = static_cast<unsigned>(
        std::max(1, std::min((sl.slices + 7) / 8, c.sm_count * per_sm)));
    k_spmv_slices<T, BS, MINB, VD><<<grid, 256, 0, c.stream>>>(sl.base.as<int>(), sl.lanes.as<unsigned short>(),
                                                               sl.cols.as<int>(), sl.vals.as<T>(), x, y, sl.slices,
                                                               static_cast<int>(m.owned));
}

// Resident CTAs per SM asked of the compiler for each element type and block
// size (measured on the 2M-vertex mesh, 20-30 launches each: FP64 bs 3 at 5
// CTAs 94.9 us against 107.7-147.1 us for 4 (no cap), 6 and the two-step
// value prefetch; FP64 bs 4 spills under a cap (143.7 us uncapped, 184.1 at
// 5); FP64 bs 1 took 54.1 us at 5 CTAs (48 registers) against 43.7 us for an
// earlier 32-register form, so it asks for 6 (40 registers; 8 spills); FP32
// bs 3 and 4 at 6 CTAs 61.4 and 78.0 us against 66.3 and 79.1 at 5).
template<class T, int BS>
constexpr int slice_ctas() { return sizeof(T) == 4 ? 6 : (BS == 1 ? 6 : (BS == 4 ? 1 : 5)); }

template<class T, int BS>
void launch_slices(Context& c, const Matrix& m, const T* x, T* y)
{
    launch_slices_v<T, BS, slice_ctas<T, BS>(), 1>(c, m, x, y);
}

template<class T, int BS, int kMinBlocks>
void launch_slices_dense_v(Context& c, const Matrix& m, const T* x, T* y)
{
    static int per_sm = 0;
    if (per_sm == 0) {
        OWTK_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_spmv_slices_dense<T, BS, kMinBlocks>, 256,
                                                                0));
        per_sm = std::max(per_sm, 1);
    }
    const RowSlices& sl = m.slices;
    const unsigned grid = static_cast<unsigned>(std::max(1, std::min((sl.slices + 7) / 8, c.sm_count * per_sm)));
    k_spmv_slices_dense<T, BS, kMinBlocks><<<grid, 256, 0, c.stream>>>(
        sl.base.as<int>(), sl.lanes.as<unsigned short>(), sl.cols.as<int>(), sl.vals.as<T>(), x, y, sl.slices,
        static_cast<int>(m.owned));
}

// Dense blocks at 3 resident CTAs per SM (2M-vertex mesh, 3x3 blocks: FP64
// 198.2 us against 234.0 us uncapped (92 registers) and 199.8 us at 4; FP32
// 114 us at 1, 3 and 4 alike); FP64 4x4 blocks at 2 (128 registers, 48
// bytes spilled; at 3 the 16 values per step spill 332 bytes).
template<class T, int BS>
void launch_slices_dense(Context& c, const Matrix& m, const T* x, T* y)
{
    launch_slices_dense_v<T, BS, (sizeof(T) == 8 && BS == 4) ? 2 : 3>(c, m, x, y);
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

// Rows of a listed subset (BlockCsrMatrix / SplitBlockCsrMatrixView /
// DenseBlockCsrMatrix::apply_rows, block_csr.hpp:198-215,
// split_block_csr.hpp:95-119, dense_block_csr.hpp:179-204): one thread per
// (listed row, component or block row), the reference's loop for that output
// term by term (component-diagonal: 0 + v x per entry; split: d x, then + v x;
// dense: per entry the block row's dot product from 0, then added), so the
// rows equal those of the whole-matrix apply bit for bit.  Rows not listed
// are left as they are.
template<class T>
__global__ void k_spmv_rows(int kind, int bs, const int* __restrict__ rows, int count, const int* __restrict__ rowptr,
                            const int* __restrict__ cols, const T* __restrict__ vals, const T* __restrict__ diag,
                            const T* __restrict__ x, T* __restrict__ y)
{
    const long long k = static_cast<long long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (k >= static_cast<long long>(count) * bs) return;
    const int i = static_cast<int>(k / bs), c = static_cast<int>(k - static_cast<long long>(i) * bs);
    const int row = rows[i];
    const long long o = static_cast<long long>(row) * bs + c;
    T acc = kind == 1 ? mul_rn(diag[o], x[o]) : T(0);
    for (int e = rowptr[row]; e < rowptr[row + 1]; ++e) {
        const long long xb = static_cast<long long>(cols[e]) * bs;
        if (kind == 2) {
            const T* b = vals + static_cast<long long>(e) * bs * bs + static_cast<long long>(c) * bs;
            T part = T(0);
            for (int j = 0; j < bs; ++j) part = add_rn(part, mul_rn(b[j], x[xb + j]));
            acc = add_rn(acc, part);
        } else {
            acc = add_rn(acc, mul_rn(vals[static_cast<long long>(e) * bs + c], x[xb + c]));
        }
    }
    y[o] = acc;
}

}  // namespace

namespace kern {

// OWTK_SPMV_SLICES=0 sends the component-diagonal BSR back to the bulk-copy
// pipeline (both give the same bits).
static bool slices_enabled()
{
    static const bool on = [] {
        const char* e = std::getenv("OWTK_SPMV_SLICES");
        return e == nullptr || e[0] != '0';
    }();
    return on;
}

template<class T> void spmv(Context& c, const Matrix& m, const T* x, T* y)
{
    if (m.plan.tiles == 0) return;
    if ((m.kind == 0 || m.kind == 2) && m.slices.filled && slices_enabled()) {
        if (m.kind == 0) {
            switch (m.bs) {
            case 1: launch_slices<T, 1>(c, m, x, y); break;
            case 2: launch_slices<T, 2>(c, m, x, y); break;
            case 3: launch_slices<T, 3>(c, m, x, y); break;
            default: launch_slices<T, 4>(c, m, x, y); break;
            }
        } else {
            switch (m.bs) {
            case 1: launch_slices_dense<T, 1>(c, m, x, y); break;
            case 2: launch_slices_dense<T, 2>(c, m, x, y); break;
            case 3: launch_slices_dense<T, 3>(c, m, x, y); break;
            default: launch_slices_dense<T, 4>(c, m, x, y); break;
            }
        }
        OWTK_CUDA(cudaGetLastError());
        c.launched();
        const int count = m.slices.long_count;
        if (count > 0) {
            const long long total = static_cast<long long>(count) * static_cast<long long>(m.bs);
            k_spmv_rows<T><<<static_cast<unsigned>((total + 255) / 256), 256, 0, c.stream>>>(
                m.kind, static_cast<int>(m.bs), m.slices.long_rows.as<int>(), count, m.rowptr.as<int>(),
                m.cols.as<int>(), static_cast<const T*>(m.values.ptr), nullptr, x, y);
            OWTK_CUDA(cudaGetLastError());
            c.launched();
        }
        return;
    }
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
    const auto aligned = [](const void* p) { return (reinterpret_cast<std::uintptr_t>(p) & 15u) == 0; };
    // Split views (bs <= 4) take the warp-shuffle kernel: on the 2M-vertex
    // mesh, bs 3, it measured 132 us against 160 us for the bulk pipeline,
    // which stays ahead for the component-diagonal BSR (130 vs 159 us).
    if (m.kind == 1 && m.bs <= 4 && launch_warp_bs<T, 1>(c, a, m)) {
        // launched
    } else if (m.kind != 2 && aligned(a.vals) && aligned(a.cols) && aligned(a.rowptr)) {
        if (m.kind == 0) launch_bulk_bs<T, 0>(c, a, m);
        else launch_bulk_bs<T, 1>(c, a, m);
    } else if (m.kind == 0) {
        k_spmv_tiles<T, 0><<<grid, kThreads, 0, c.stream>>>(a);
    } else if (m.kind == 1) {
        k_spmv_tiles<T, 1><<<grid, kThreads, 0, c.stream>>>(a);
    } else if (m.bs == 2) {
        k_spmv_tiles<T, 2, 2><<<grid, kThreads, 0, c.stream>>>(a);
    } else if (m.bs == 3) {
        k_spmv_tiles<T, 2, 3><<<grid, kThreads, 0, c.stream>>>(a);
    } else if (m.bs == 4) {
        k_spmv_tiles<T, 2, 4><<<grid, kThreads, 0, c.stream>>>(a);
    } else {
        k_spmv_tiles<T, 2><<<grid, kThreads, 0, c.stream>>>(a);
    }
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

template<class T> void spmv_rows(Context& c, const Matrix& m, const int* rows, int count, const T* x, T* y)
{
    if (count == 0) return;
    const long long total = static_cast<long long>(count) * static_cast<long long>(m.bs);
    k_spmv_rows<T><<<static_cast<unsigned>((total + 255) / 256), 256, 0, c.stream>>>(
        m.kind, static_cast<int>(m.bs), rows, count, m.rowptr.as<int>(), m.cols.as<int>(),
        static_cast<const T*>(m.value_ptr()), static_cast<const T*>(m.diag), x, y);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
}

void slices_fill(Context& c, Matrix& m)
{
    RowSlices& sl = m.slices;
    if (sl.slices == 0) return;
    const unsigned grid = static_cast<unsigned>((sl.slices + 7) / 8);
    const int per = static_cast<int>(m.kind == 2 ? m.bs * m.bs : m.bs);
    if (m.dtype == OWTK_F64)
        k_slices_fill<double><<<grid, 256, 0, c.stream>>>(sl.base.as<int>(), sl.lanes.as<unsigned short>(),
                                                          m.rowptr.as<int>(), m.cols.as<int>(), m.values.as<double>(),
                                                          sl.cols.as<int>(), sl.vals.as<double>(), sl.slices, per);
    else
        k_slices_fill<float><<<grid, 256, 0, c.stream>>>(sl.base.as<int>(), sl.lanes.as<unsigned short>(),
                                                         m.rowptr.as<int>(), m.cols.as<int>(), m.values.as<float>(),
                                                         sl.cols.as<int>(), sl.vals.as<float>(), sl.slices, per);
    OWTK_CUDA(cudaGetLastError());
    c.launched();
    sl.filled = true;
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
template void spmv_rows<double>(Context&, const Matrix&, const int*, int, const double*, double*);
template void spmv_rows<float>(Context&, const Matrix&, const int*, int, const float*, float*);
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
    build_row_slices(m);
}

// Row-slice layout of a component-diagonal or dense-block BSR with bs <= 4
// (FP64 or FP32): per slice of 32
// rows the lanes in order of decreasing row length (ties by row), the first
// packed entry of each slice, and the long rows; the arrays it fills are
// allocated here and written by kern::slices_fill.
void build_row_slices(Matrix& m)
{
    RowSlices& sl = m.slices;
    sl = RowSlices{};
    if ((m.kind != 0 && m.kind != 2) || m.bs > 4 || m.owned == 0 || (m.dtype != OWTK_F64 && m.dtype != OWTK_F32))
        return;
    const int owned = static_cast<int>(m.owned);
    sl.slices = (owned + 31) / 32;
    std::vector<std::uint16_t> lanes(static_cast<std::size_t>(sl.slices) * 32, 255);
    std::vector<std::int32_t> base(static_cast<std::size_t>(sl.slices) + 1, 0), long_rows;
    std::vector<std::pair<int, int>> order;   // (-length, row in slice)
    std::size_t packed = 0;
    for (int s = 0; s < sl.slices; ++s) {
        order.clear();
        const int r0 = 32 * s, r1 = std::min(owned, r0 + 32);
        for (int r = r0; r < r1; ++r) {
            int len = m.h_rowptr[r + 1] - m.h_rowptr[r];
            if (len > kSliceMaxRow) {
                long_rows.push_back(r);
                len = 0;
            }
            order.emplace_back(-len, r - r0);
        }
        std::sort(order.begin(), order.end());
        for (std::size_t j = 0; j < order.size(); ++j) {
            const int len = -order[j].first;
            lanes[static_cast<std::size_t>(s) * 32 + j] = static_cast<std::uint16_t>(order[j].second | (len << 8));
            packed += static_cast<std::size_t>(len);
        }
        base[s + 1] = static_cast<std::int32_t>(packed);
    }
    sl.packed = packed;
    sl.base = upload(m.ctx->stream, base);
    sl.lanes = upload(m.ctx->stream, lanes);
    sl.cols.allocate(packed * 4 + 16);
    const std::size_t per = m.kind == 2 ? m.bs * m.bs : m.bs;
    sl.vals.allocate(packed * per * (m.dtype == OWTK_F64 ? 8 : 4) + 16);
    sl.long_count = static_cast<int>(long_rows.size());
    if (!long_rows.empty()) sl.long_rows = upload(m.ctx->stream, long_rows);
}

}  // namespace owtk
