// ILU(k) applies for near-sequential dependency DAGs (sm_100a): the forward
// and backward triangular sweeps of IluLevelPreconditioner::apply
// (preconditioner.hpp:320-363) when the level sets hold only a few rows each.
// A Hilbert-curve order (ordering.hpp:231-261) puts mesh neighbours next to
// each other along the curve, so the factors' DAGs are about as deep as the
// matrix is long (2M rows: 1.6M levels) and the level-scheduled sweep pays
// one L2 round trip per level.
//
// The factors are component-diagonal, so the bs components are independent
// scalar solves: one warp per component, each in its own CTA (its own SM).
// Rows are taken in windows of up to 32 consecutive rows, one row per lane:
//   phase A (all lanes at once): the terms whose dependency lies outside the
//     window — final values, read from a shared-memory ring of the last
//     kRing results or, further away, from global memory through a copy
//     staged one window ahead;
//   phase B (one step per row): step t finishes row t of the window and
//     broadcasts it by a warp shuffle; the lanes whose rows depend on it use
//     it at once.
// Each window's factor rows (whole rows: columns and this component's
// values), row offsets, inputs and inverse diagonal are staged into shared
// memory by cp.async two windows ahead, its far dependency values one window
// ahead, so phase A never waits on global memory.
//
// Term order.  Forward (unit lower, y = in - sum l y): a row's terms in
// ascending column order are the ones before the window, then the in-window
// ones in step order, so phase A then phase B subtract them in the
// reference's order.  Backward (x = (y - sum u x) * inv): the in-window
// columns come first in ascending order but finish in descending step order,
// so a row's sum runs whole at its own step: phase A and the earlier steps
// only form the rounded products u * x, and step t subtracts them in column
// order and multiplies by the inverse diagonal.  Every product and
// difference is rounded separately (no contraction), as on the CPU, so
// results equal the reference bit for bit (no sentinel is involved, so NaN
// results are stored as the arithmetic produced them).
//
// There is no wait on another thread's progress anywhere: the only waits are
// for this warp's own cp.async copies.
//
// Measured on the 2M-vertex Hilbert-ordered disk mesh: 724 ms per apply
// against 1.94 s for the level-scheduled sweep.  A warp alone on its SM
// issues an instruction about every 5.5 cycles (waits on the previous
// result, on shared memory and on shuffles), so the cost is the instruction
// count per row: 29 forward, 102 backward.  Two forms with lane 0 running the
// rows from per-row records (plain, and software-pipelined) were slower:
// 1071 and 1113 ms.

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

constexpr int kRing = 8192;         // results kept in shared memory (rows)
constexpr int kStageEntries = 1024; // factor entries staged per window
constexpr int kStages = 3;          // windows in flight: phase A, far values, rows
constexpr int kChain = 5;           // backward: terms of a row held in registers

template<class T>
struct ChainArgs {
    const int4* windows;    // {first row, end row, first entry, end entry}, ascending
    int count;              // windows
    const int* rowptr;
    const int* cols;
    const int* diagpos;
    const T* vals;          // factor values, entry-major, bs per entry
    const T* inv;           // inverse diagonal (backward)
    const T* in;            // forward: the right-hand side; backward: the forward result
    T* out;                 // forward: y; backward: x
    int bs;
};

template<class T>
struct Stage {
    int cols[kStageEntries];
    T vals[kStageEntries];
    T far[kStageEntries];   // dependency values from beyond the ring, by entry
    int rowptr[33];
    int diagpos[32];
    T in[32];
    T inv[32];
};

template<class T>
struct ChainSmem {
    T ring[kRing];
    Stage<T> stage[kStages];
    T ftab[32][33];          // [step][lane]: factor of the lane's term on that step's row
    T ptab[kStageEntries];   // backward: rounded products u * x, by entry
    short etab[32][32];      // backward: [step][lane] entry of that term
    int chain_begin[32], chain_count[32];
};

__device__ __forceinline__ void cp_async(void* dst, const void* src, int bytes)
{
    const std::uint32_t d = static_cast<std::uint32_t>(__cvta_generic_to_shared(dst));
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

__device__ __forceinline__ bool staged(const int4& w) { return w.w - w.z <= kStageEntries; }

// Rows, offsets, inputs of window w into stage s (nothing for a window with
// more entries than a stage holds: it is read from global memory).
template<class T, bool BACKWARD>
__device__ __forceinline__ void stage_rows(const ChainArgs<T>& a, Stage<T>& s, const int4& w, int c, int lane)
{
    const int nw = w.y - w.x;
    if (lane == 0) cp_async(&s.rowptr[nw], a.rowptr + w.y, 4);
    if (lane < nw) {
        cp_async(&s.rowptr[lane], a.rowptr + w.x + lane, 4);
        cp_async(&s.diagpos[lane], a.diagpos + w.x + lane, 4);
        cp_async(&s.in[lane], a.in + static_cast<long long>(w.x + lane) * a.bs + c, sizeof(T));
        if (BACKWARD) cp_async(&s.inv[lane], a.inv + static_cast<long long>(w.x + lane) * a.bs + c, sizeof(T));
    }
    if (!staged(w)) return;
    for (int q = lane; q < w.w - w.z; q += 32) {
        cp_async(&s.cols[q], a.cols + w.z + q, 4);
        cp_async(&s.vals[q], a.vals + static_cast<long long>(w.z + q) * a.bs + c, sizeof(T));
    }
}

// Dependency values of window w from beyond the ring (final long before
// this window runs) into stage s; its columns are already staged.
template<class T, bool BACKWARD>
__device__ __forceinline__ void stage_far(const ChainArgs<T>& a, Stage<T>& s, const int4& w, int c, int lane)
{
    if (!staged(w)) return;
    for (int q = lane; q < w.w - w.z; q += 32) {
        const int col = s.cols[q];
        const bool far = BACKWARD ? col >= w.y + kRing : col < w.x - kRing;
        if (far) cp_async(&s.far[q], a.out + static_cast<long long>(col) * a.bs + c, sizeof(T));
    }
}

template<class T, bool BACKWARD>
__global__ void __launch_bounds__(32, 1) k_ilu_chain(ChainArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char chain_smem_raw[];
    ChainSmem<T>& S = *reinterpret_cast<ChainSmem<T>*>(chain_smem_raw);
    const int c = blockIdx.x, lane = threadIdx.x;
    const unsigned full = 0xffffffffu;
    const int W = a.count;
    // Window of processing step i (ascending forward, descending backward).
    const auto window = [&](int i) {
        if (i >= W) return make_int4(0, 0, 0, 0);
        return __ldg(a.windows + (BACKWARD ? W - 1 - i : i));
    };
    int4 w0 = window(0), w1 = window(1), w2 = window(2);
    stage_rows<T, BACKWARD>(a, S.stage[0], w0, c, lane);
    cp_async_commit();
    cp_async_wait_all();
    __syncwarp();
    stage_far<T, BACKWARD>(a, S.stage[0], w0, c, lane);
    if (W > 1) stage_rows<T, BACKWARD>(a, S.stage[1], w1, c, lane);
    cp_async_commit();
    for (int i = 0; i < W; ++i) {
        const int4 w3 = window(i + 3);
        cp_async_wait_all();
        __syncwarp();
        if (i + 1 < W) stage_far<T, BACKWARD>(a, S.stage[(i + 1) % kStages], w1, c, lane);
        if (i + 2 < W) stage_rows<T, BACKWARD>(a, S.stage[(i + 2) % kStages], w2, c, lane);
        cp_async_commit();

        Stage<T>& s = S.stage[i % kStages];
        const int r0 = w0.x, r1 = w0.y, nw = r1 - r0, e0 = w0.z;
        const bool live = lane < nw;
        const int r = r0 + lane;
        T acc = live ? s.in[lane] : T(0);
        if (!staged(w0)) {
            // A single row with more entries than a stage holds: its whole
            // sum here, from global memory.
            if (lane == 0) {
                const int b = BACKWARD ? s.diagpos[0] + 1 : s.rowptr[0];
                const int e = BACKWARD ? s.rowptr[1] : s.diagpos[0];
                for (int q = b; q < e; ++q) {
                    const int col = a.cols[q];
                    const T v = (BACKWARD ? col < r1 + kRing : col >= r0 - kRing) ? S.ring[col & (kRing - 1)]
                                                                                    : a.out[static_cast<long long>(col) * a.bs + c];
                    acc = sub_rn(acc, mul_rn(a.vals[static_cast<long long>(q) * a.bs + c], v));
                }
                if (BACKWARD) acc = mul_rn(acc, s.inv[0]);
            }
        } else if (!BACKWARD) {
            // ---- forward phase A: the terms before the window, in order.
            unsigned mask = 0;
            if (live) {
                const int qe = s.diagpos[lane] - e0;
                for (int q = s.rowptr[lane] - e0; q < qe; ++q) {
                    const int col = s.cols[q];
                    const T f = s.vals[q];
                    if (col < r0) {
                        const T v = col >= r0 - kRing ? S.ring[col & (kRing - 1)] : s.far[q];
                        acc = sub_rn(acc, mul_rn(f, v));
                    } else {
                        S.ftab[col - r0][lane] = f;
                        mask |= 1u << (col - r0);
                    }
                }
            }
            __syncwarp();
            // ---- phase B: row t is final at step t.
#pragma unroll 4
            for (int t = 0; t < nw; ++t) {
                const T f = S.ftab[t][lane];
                const T yt = __shfl_sync(full, acc, t);
                if ((mask >> t) & 1u) acc = sub_rn(acc, mul_rn(f, yt));
            }
        } else {
            // ---- backward phase A: a row's terms in column order are its
            // in-window ones (their products formed on the steps that
            // finish those rows), then the ones after the window (products
            // formed here).  They are held in a register list of kChain
            // slots; a row with more takes its products from shared memory.
            unsigned mask = 0;
            int m = 0, total = 0;
            T prods[kChain];
#pragma unroll
            for (int k = 0; k < kChain; ++k) prods[k] = T(0);
            if (live) {
                const int qb = s.diagpos[lane] + 1 - e0, qe = s.rowptr[lane + 1] - e0;
                total = qe - qb;
                for (int q = qb; q < qe; ++q) {
                    const int col = s.cols[q];
                    const T f = s.vals[q];
                    if (col < r1) {
                        S.ftab[col - r0][lane] = f;
                        S.etab[col - r0][lane] = static_cast<short>(total <= kChain ? m : q);
                        mask |= 1u << (col - r0);
                        ++m;
                    } else {
                        const T v = col < r1 + kRing ? S.ring[col & (kRing - 1)] : s.far[q];
                        const T p = mul_rn(f, v);
                        const int k = q - qb;
                        if (total <= kChain) {
#pragma unroll
                            for (int j = 0; j < kChain; ++j)
                                if (j == k) prods[j] = p;
                        } else {
                            S.ptab[q] = p;
                        }
                    }
                }
                S.chain_begin[lane] = qb;
                S.chain_count[lane] = total;
            }
            __syncwarp();
            // ---- phase B, rows in descending order: step t sums row t's
            // products in column order, scales by the inverse diagonal and
            // broadcasts the result; the rows with a term on it form that
            // product at once.
            for (int t = nw - 1; t >= 0; --t) {
                const T inv = s.inv[t];
                const int cnt = S.chain_count[t];
                if (cnt <= kChain) {
                    if (lane == t) {
#pragma unroll
                        for (int k = 0; k < kChain; ++k)
                            if (k < cnt) acc = sub_rn(acc, prods[k]);
                        acc = mul_rn(acc, inv);
                    }
                } else if (lane == t) {
                    const int qb = S.chain_begin[t];
                    for (int j = 0; j < cnt; ++j) acc = sub_rn(acc, S.ptab[qb + j]);
                    acc = mul_rn(acc, inv);
                }
                const T xt = __shfl_sync(full, acc, t);
                if ((mask >> t) & 1u) {
                    const T p = mul_rn(S.ftab[t][lane], xt);
                    const int slot = S.etab[t][lane];
                    if (total <= kChain) {
#pragma unroll
                        for (int j = 0; j < kChain; ++j)
                            if (j == slot) prods[j] = p;
                    } else {
                        S.ptab[slot] = p;
                    }
                }
            }
        }
        if (live) {
            S.ring[r & (kRing - 1)] = acc;
            a.out[static_cast<long long>(r) * a.bs + c] = acc;
        }
        w0 = w1;
        w1 = w2;
        w2 = w3;
    }
    cp_async_wait_all();
}

template<class T, bool BACKWARD>
bool launch_chain(Context& c, const Preconditioner& p, const ChainArgs<T>& a)
{
    const std::size_t smem = sizeof(ChainSmem<T>);
    static const bool configured =
        cudaFuncSetAttribute(k_ilu_chain<T, BACKWARD>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             static_cast<int>(smem)) == cudaSuccess;
    if (!configured) {
        cudaGetLastError();
        return false;
    }
    k_ilu_chain<T, BACKWARD><<<static_cast<unsigned>(p.bs), 32, smem, c.stream>>>(a);
    c.launched();
    return true;
}

}  // namespace

// Symbolic setup: windows of up to 32 consecutive rows whose factor rows fit
// one stage (a row that alone exceeds a stage gets a window of its own).
// Chosen when both DAGs average fewer than kChainRowsPerLevel rows per level.
void build_chain_sweep(Context& ctx, ChainSweep& s, std::size_t owned, int depth_lower, int depth_upper,
                       const std::vector<std::int32_t>& rowptr)
{
    s = ChainSweep{};
    const char* env = std::getenv("OWTK_CHAIN_SWEEP");
    if (env && std::atoi(env) == 0) return;
    const std::size_t n = owned;
    if (n == 0) return;
    const auto shallow = [&](int depth) {
        return static_cast<double>(n) / std::max(depth, 1) >= kChainRowsPerLevel;
    };
    if (shallow(depth_lower) || shallow(depth_upper)) return;
    std::vector<int4> windows;
    std::size_t r0 = 0;
    while (r0 < n) {
        std::size_t r1 = r0 + 1;
        while (r1 < n && r1 - r0 < 32 && rowptr[r1 + 1] - rowptr[r0] <= kStageEntries) ++r1;
        windows.push_back(int4{static_cast<int>(r0), static_cast<int>(r1), rowptr[r0], rowptr[r1]});
        r0 = r1;
    }
    s.count = static_cast<int>(windows.size());
    s.windows = upload(ctx.stream, windows);
    s.ready = true;
}

namespace kern {

// preconditioner.hpp:320-363 by one warp per component; false when the
// preconditioner has no chain schedule (the caller runs another sweep).
template<class T> bool chain_ilu_apply(Context& c, Preconditioner& p, const T* in, T* out)
{
    if (!p.chain.ready || p.block || p.storage != OWTK_F64) return false;
    ChainArgs<T> a{};
    a.windows = p.chain.windows.as<int4>();
    a.count = p.chain.count;
    a.rowptr = p.d_frowptr.as<int>();
    a.cols = p.d_fcols.as<int>();
    a.diagpos = p.d_fdiagpos.as<int>();
    a.vals = p.d_fvalues.as<T>();
    a.inv = p.inv_diag.as<T>();
    a.bs = static_cast<int>(p.bs);
    a.in = in;
    a.out = p.work.as<T>();
    if (!launch_chain<T, false>(c, p, a)) return false;
    a.in = p.work.as<T>();
    a.out = out;
    if (!launch_chain<T, true>(c, p, a)) return false;
    OWTK_CUDA(cudaGetLastError());
    return true;
}

template bool chain_ilu_apply<double>(Context&, Preconditioner&, const double*, double*);
template bool chain_ilu_apply<float>(Context&, Preconditioner&, const float*, float*);

}  // namespace kern
}  // namespace owtk
