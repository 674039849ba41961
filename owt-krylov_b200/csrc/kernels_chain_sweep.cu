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
// results equal the reference bit for bit, NaN payloads included.
//
// There is no wait on another thread's progress anywhere: the only waits are
// for this warp's own cp.async copies.

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

constexpr int kRing = 8192;        // results kept in shared memory (rows)
constexpr int kStageEntries = 512; // factor entries staged per window
constexpr int kStages = 5;         // windows staged: rows 4 ahead, far values 2 ahead
constexpr int kRec = 4;            // terms per row held in a record (more: the row's list is walked)

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

// One row of the window as the sequential phase consumes it, built in
// phase A by the row's lane.  `link` is the factor of the term on the row
// finished just before (forward: column r-1, the row's last term; backward:
// column r+1, its first term), 0 when the row has none (`linked` false).  The
// other terms in the window are slots: forward (factor, column - r0) before
// the link; backward, after it, (factor, column - r0) in the window or, beyond
// the window, (rounded product, -1).  Forward `pre` is the input minus the
// terms before the window, backward the input (y).  cnt > kRec: the row's
// list is walked instead.
template<class T>
struct Rec {
    T pre, inv, link;
    T v[kRec];
    int tags;               // kRec signed bytes
    int cnt;                // slots (the link not counted)
    int linked;
    int pad;
};

template<class T>
struct ChainSmem {
    T ring[kRing];
    Stage<T> stage[kStages];
    Rec<T> rec[32];
    T win[32];              // the window's results, in step order
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
__device__ __forceinline__ void cp_async_wait_one() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }

__device__ __forceinline__ bool staged(const int4& w) { return w.w - w.z <= kStageEntries; }
__device__ __forceinline__ int tag_of(int tags, int k) { return static_cast<signed char>((tags >> (8 * k)) & 0xff); }

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
    const int W = a.count;
    // Window of processing step i (ascending forward, descending backward).
    const auto window = [&](int i) {
        if (i >= W) return make_int4(0, 0, 0, 0);
        return __ldg(a.windows + (BACKWARD ? W - 1 - i : i));
    };
    // Descriptors of windows i .. i+4 (d[0] is the current one).
    int4 d0 = window(0), d1 = window(1), d2 = window(2), d3 = window(3), d4 = window(4);
    // Prologue: rows of windows 0-3, then the far values of windows 0 and 1.
    stage_rows<T, BACKWARD>(a, S.stage[0], d0, c, lane);
    if (W > 1) stage_rows<T, BACKWARD>(a, S.stage[1], d1, c, lane);
    if (W > 2) stage_rows<T, BACKWARD>(a, S.stage[2], d2, c, lane);
    if (W > 3) stage_rows<T, BACKWARD>(a, S.stage[3], d3, c, lane);
    cp_async_commit();
    cp_async_wait_all();
    __syncwarp();
    stage_far<T, BACKWARD>(a, S.stage[0], d0, c, lane);
    if (W > 1) stage_far<T, BACKWARD>(a, S.stage[1], d1, c, lane);
    cp_async_commit();
    cp_async_wait_all();
    __syncwarp();
    for (int i = 0; i < W; ++i) {
        const int4 d5 = window(i + 5);
        // Every copy group but the newest has landed: the rows of windows up
        // to i+3 and the far values up to i+1 (issued two iterations ago).
        cp_async_wait_one();
        __syncwarp();
        if (i + 2 < W) stage_far<T, BACKWARD>(a, S.stage[(i + 2) % kStages], d2, c, lane);
        if (i + 4 < W) stage_rows<T, BACKWARD>(a, S.stage[(i + 4) % kStages], d4, c, lane);
        cp_async_commit();

        Stage<T>& s = S.stage[i % kStages];
        const int r0 = d0.x, r1 = d0.y, nw = r1 - r0, e0 = d0.z;
        const bool live = lane < nw;
        const int r = r0 + lane;
        if (!staged(d0)) {
            // A single row with more entries than a stage holds: its whole
            // sum here, from global memory.
            if (lane == 0) {
                T acc = s.in[0];
                const int b = BACKWARD ? s.diagpos[0] + 1 : s.rowptr[0];
                const int e = BACKWARD ? s.rowptr[1] : s.diagpos[0];
                for (int q = b; q < e; ++q) {
                    const int col = a.cols[q];
                    const T v = (BACKWARD ? col < r1 + kRing : col >= r0 - kRing) ? S.ring[col & (kRing - 1)]
                                                                                    : a.out[static_cast<long long>(col) * a.bs + c];
                    acc = sub_rn(acc, mul_rn(a.vals[static_cast<long long>(q) * a.bs + c], v));
                }
                if (BACKWARD) acc = mul_rn(acc, s.inv[0]);
                S.win[0] = acc;
            }
        } else {
            // ---- phase A, one row per lane: the record of its row.
            if (live) {
                Rec<T> rc;
                rc.link = T(0);
                rc.linked = 0;
                int n = 0, tags = 0;
                const int qb = BACKWARD ? s.diagpos[lane] + 1 - e0 : s.rowptr[lane] - e0;
                const int qe = BACKWARD ? s.rowptr[lane + 1] - e0 : s.diagpos[lane] - e0;
                T acc = s.in[lane];
                for (int q = qb; q < qe; ++q) {
                    const int col = s.cols[q];
                    const T f = s.vals[q];
                    if (!BACKWARD && col < r0) {   // before the window: final, applied here in order
                        const T v = col >= r0 - kRing ? S.ring[col & (kRing - 1)] : s.far[q];
                        acc = sub_rn(acc, mul_rn(f, v));
                        continue;
                    }
                    if (col == (BACKWARD ? r + 1 : r - 1) && (BACKWARD ? col < r1 : col >= r0)) {
                        rc.link = f;   // forward: always the last term; backward: always the first
                        rc.linked = 1;
                        continue;
                    }
                    T slot = f;
                    int tag = col - r0;
                    if (BACKWARD && col >= r1) {   // after the window: the product, subtracted in turn
                        const T v = col < r1 + kRing ? S.ring[col & (kRing - 1)] : s.far[q];
                        slot = mul_rn(f, v);
                        tag = -1;
                    }
                    if (n < kRec) {
#pragma unroll
                        for (int k = 0; k < kRec; ++k)
                            if (k == n) rc.v[k] = slot;
                        tags |= (tag & 0xff) << (8 * n);
                    }
                    ++n;
                }
                rc.pre = acc;
                rc.inv = BACKWARD ? s.inv[lane] : T(0);
                rc.tags = tags;
                rc.cnt = n;
                S.rec[lane] = rc;
            }
            __syncwarp();
            // ---- phase B: lane 0 finishes the rows in order.  Step j takes
            // the row finished before (`last`) through the current row's
            // link; the next row's other terms, which need only older
            // results, are formed in the same step, off that chain.
            if (lane == 0) {
                T last = T(0);
                // The row's terms other than the link, as far as they can be
                // formed before `last` of its step is known: forward the
                // partial sum pre - slots (all before the link), backward the
                // products of the slots (subtracted after the link).
                T part = T(0);
                T prod[kRec];
#pragma unroll
                for (int k = 0; k < kRec; ++k) prod[k] = T(0);
                // Terms of record rc at step j (row t), given `last` = result of
                // the row finished at step j - 1.
                const auto prepare = [&](const Rec<T>& rc, int t, T prev_result) {
                    const int prev2 = BACKWARD ? t + 2 : t - 2;   // finished two steps before t
                    if (!BACKWARD) {
                        T acc = rc.pre;
#pragma unroll
                        for (int k = 0; k < kRec; ++k) {
                            if (k < rc.cnt) {
                                const int tag = tag_of(rc.tags, k);
                                const T v = tag == prev2 ? prev_result : S.win[tag & 31];
                                acc = sub_rn(acc, mul_rn(rc.v[k], v));
                            }
                        }
                        part = acc;
                    } else {
#pragma unroll
                        for (int k = 0; k < kRec; ++k) {
                            if (k < rc.cnt) {
                                const int tag = tag_of(rc.tags, k);
                                const T v = tag == prev2 ? prev_result : S.win[tag & 31];
                                prod[k] = tag < 0 ? rc.v[k] : mul_rn(rc.v[k], v);
                            }
                        }
                    }
                };
                Rec<T> cur = S.rec[BACKWARD ? nw - 1 : 0];
                if (cur.cnt <= kRec) prepare(cur, BACKWARD ? nw - 1 : 0, T(0));
                for (int j = 0; j < nw; ++j) {
                    const int t = BACKWARD ? nw - 1 - j : j;
                    const int tn = BACKWARD ? t - 1 : t + 1;    // the next row
                    const bool more = j + 1 < nw;
                    const Rec<T> nxt = S.rec[more ? tn : t];
                    T res;
                    if (cur.cnt <= kRec) {
                        if (!BACKWARD) {
                            res = cur.linked ? sub_rn(part, mul_rn(cur.link, last)) : part;
                        } else {
                            T acc = cur.linked ? sub_rn(cur.pre, mul_rn(cur.link, last)) : cur.pre;
#pragma unroll
                            for (int k = 0; k < kRec; ++k)
                                if (k < cur.cnt) acc = sub_rn(acc, prod[k]);
                            res = mul_rn(acc, cur.inv);
                        }
                    } else {
                        // More terms than a record holds: the row's list, in order.
                        const int prev = BACKWARD ? t + 1 : t - 1;
                        const int qb = BACKWARD ? s.diagpos[t] + 1 - e0 : s.rowptr[t] - e0;
                        const int qe = BACKWARD ? s.rowptr[t + 1] - e0 : s.diagpos[t] - e0;
                        T acc = cur.pre;
                        for (int q = qb; q < qe; ++q) {
                            const int col = s.cols[q];
                            if (!BACKWARD && col < r0) continue;   // already in pre
                            T v;
                            if (BACKWARD && col >= r1)
                                v = col < r1 + kRing ? S.ring[col & (kRing - 1)] : s.far[q];
                            else
                                v = col - r0 == prev ? last : S.win[col - r0];
                            acc = sub_rn(acc, mul_rn(s.vals[q], v));
                        }
                        res = BACKWARD ? mul_rn(acc, cur.inv) : acc;
                    }
                    // The next row's terms: they reach back two rows at most
                    // to `last` (the row before this one), older ones are in win.
                    if (more && nxt.cnt <= kRec) prepare(nxt, tn, last);
                    S.win[t] = res;
                    last = res;
                    cur = nxt;
                }
            }
        }
        __syncwarp();
        if (live) {
            const T y = S.win[lane];
            S.ring[r & (kRing - 1)] = y;
            a.out[static_cast<long long>(r) * a.bs + c] = y;
        }
        d0 = d1;
        d1 = d2;
        d2 = d3;
        d3 = d4;
        d4 = d5;
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
