// ILU(k) applies level by level on one thread-block cluster (sm_100a): the
// forward and backward triangular sweeps of IluLevelPreconditioner::apply
// (preconditioner.hpp:320-363) with the levels taken in lockstep.
//
// The level-scheduled sweep of kernels_sweep.cu lets dependants poll their
// dependencies in L2, about 0.86 us per level on the 2M-vertex RCM mesh
// (2 x 2913 levels).  Here one cluster of C CTAs (16 when the device allows
// it, else 8) of 512 threads runs the sweep one level per step:
//   * every level's rows are cut into C contiguous chunks, one per CTA, and
//     a CTA's lanes take the (row, component) pairs of its chunk — a level
//     is one step for every lane;
//   * a step ends with a cluster barrier (arrive.release / wait.acquire,
//     about 0.24 us measured), so the results of the steps before it are
//     final and visible when the next one starts: no polling, no sentinel;
//   * each CTA keeps its results of the last three levels in a shared-memory
//     ring; a dependency one or two levels back is read from its owner's
//     ring over distributed shared memory; an older one is final in global
//     memory and was loaded two steps ahead, together with the row's factor
//     values and input, into registers.
// Per (row, component) the arithmetic is the reference's, term by term in
// entry order with explicit rounding, so results equal the CPU path bit for
// bit.  Every CTA runs every step, so every barrier is met; there is no
// wait on another thread's progress other than the hardware barrier.

#include <climits>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

constexpr int kLockThreads = 512;   // lanes per CTA: (row, component) pairs of a chunk
constexpr int kLockK = 6;           // terms a row carries in registers (more: read at its step)
constexpr int kLockRing = 3;        // levels of results kept in shared memory

template<class T>
struct LockArgs {
    const int2* blk;        // D x C: first lane-task of the level's chunk, lane-tasks in it
    const int* task_io;     // per lane-task: row * bs + component (input, output, inverse diagonal)
    const int2* task_ent;   // per lane-task: first entry, entries
    const int* ent_loc;     // per entry: near (ring) or far (global index), see loc_* below
    const T* ent_val;       // per entry: the factor value of this component
    const T* inv;           // inverse diagonal (backward)
    const T* in;
    T* out;
    int D, C;
};

// Entry location: a dependency one or two levels back lives in its owner's
// ring, loc = INT_MIN | (levels back - 1) << 28 | owner << 20 | slot; an
// older one is final in global memory at index loc >= 0.
__device__ __forceinline__ bool loc_near(int loc) { return loc < 0; }
__device__ __forceinline__ int loc_back(int loc) { return ((loc >> 28) & 3) + 1; }
__device__ __forceinline__ unsigned loc_owner(int loc) { return (static_cast<unsigned>(loc) >> 20) & 0xffu; }
__device__ __forceinline__ int loc_slot(int loc) { return loc & 0xfffff; }

__device__ __forceinline__ unsigned lock_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void lock_barrier()
{
    asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

__device__ __forceinline__ unsigned lock_mapa(unsigned addr, unsigned cta)
{
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(addr), "r"(cta));
    return r;
}

__device__ __forceinline__ double lock_ld(unsigned addr, double*)
{
    double v;
    asm volatile("ld.shared::cluster.f64 %0, [%1];" : "=d"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ float lock_ld(unsigned addr, float*)
{
    float v;
    asm volatile("ld.shared::cluster.f32 %0, [%1];" : "=f"(v) : "r"(addr) : "memory");
    return v;
}

template<class T>
struct LockSlot {
    bool valid;
    int io, n, eb;
    T in, inv;
    int loc[kLockK];
    T f[kLockK];
    T far[kLockK];
};

// The lane's task of level L (two steps ahead of its use): input, inverse
// diagonal, factor values and locations, and the values of dependencies
// older than L-2, which are final by now.
template<class T, bool BACKWARD>
__device__ __forceinline__ void lock_load(const LockArgs<T>& a, LockSlot<T>& s, int L, unsigned rank, int lane)
{
    s.valid = false;
    s.n = 0;
    if (L >= a.D) return;
    const int2 b = __ldg(a.blk + static_cast<long long>(L) * a.C + rank);
    if (lane >= b.y) return;
    const int t = b.x + lane;
    s.valid = true;
    s.io = __ldg(a.task_io + t);
    const int2 e = __ldg(a.task_ent + t);
    s.eb = e.x;
    s.n = e.y;
    s.in = __ldcg(a.in + s.io);
    s.inv = BACKWARD ? __ldg(a.inv + s.io) : T(0);
#pragma unroll
    for (int k = 0; k < kLockK; ++k) {
        if (k < s.n) {
            s.loc[k] = __ldg(a.ent_loc + s.eb + k);
            s.f[k] = __ldg(a.ent_val + s.eb + k);
            s.far[k] = loc_near(s.loc[k]) ? T(0) : __ldcg(a.out + s.loc[k]);
        }
    }
}

template<class T, bool BACKWARD>
__global__ void __launch_bounds__(kLockThreads, 1) k_ilu_lockstep(LockArgs<T> a)
{
    __shared__ T ring[kLockRing][kLockThreads];
    const unsigned rank = lock_rank();
    const int lane = threadIdx.x;
    const unsigned ring_base = static_cast<unsigned>(__cvta_generic_to_shared(&ring[0][0]));
    // The ring address of (levels back, slot) on `owner` for step M.
    const auto near_addr = [&](int M, int loc) {
        const int r = (M - loc_back(loc)) % kLockRing;
        return lock_mapa(ring_base + static_cast<unsigned>((r * kLockThreads + loc_slot(loc)) * sizeof(T)),
                         loc_owner(loc));
    };
    LockSlot<T> cur, nxt;
    lock_load<T, BACKWARD>(a, cur, 0, rank, lane);
    lock_load<T, BACKWARD>(a, nxt, 1, rank, lane);
    lock_barrier();   // every CTA of the cluster has started (its ring exists)
    for (int M = 0; M < a.D; ++M) {
        if (cur.valid) {
            T acc = cur.in;
            if (cur.n <= kLockK) {
                T v[kLockK];
#pragma unroll
                for (int k = 0; k < kLockK; ++k)
                    if (k < cur.n) v[k] = loc_near(cur.loc[k]) ? lock_ld(near_addr(M, cur.loc[k]), (T*)nullptr) : cur.far[k];
#pragma unroll
                for (int k = 0; k < kLockK; ++k)
                    if (k < cur.n) acc = sub_rn(acc, mul_rn(cur.f[k], v[k]));
            } else {
                // More terms than the registers hold: read in order now.
                for (int k = 0; k < cur.n; ++k) {
                    const int loc = __ldg(a.ent_loc + cur.eb + k);
                    const T v = loc_near(loc) ? lock_ld(near_addr(M, loc), (T*)nullptr) : __ldcg(a.out + loc);
                    acc = sub_rn(acc, mul_rn(__ldg(a.ent_val + cur.eb + k), v));
                }
            }
            if (BACKWARD) acc = mul_rn(acc, cur.inv);
            ring[M % kLockRing][lane] = acc;
            a.out[cur.io] = acc;
        }
        lock_load<T, BACKWARD>(a, cur, M + 2, rank, lane);
        const LockSlot<T> t = cur;
        cur = nxt;
        nxt = t;
        lock_barrier();
    }
}

template<class T, bool BACKWARD>
bool launch_lockstep(Context& c, const LockstepSweep& s, LockArgs<T> a)
{
    auto kernel = k_ilu_lockstep<T, BACKWARD>;
    if (s.C > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    a.blk = s.blk.as<int2>();
    a.task_io = s.task_io.as<int>();
    a.task_ent = s.task_ent.as<int2>();
    a.ent_loc = s.ent_loc.as<int>();
    a.ent_val = s.ent_val.as<T>();
    a.D = s.D;
    a.C = s.C;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(s.C));
    cfg.blockDim = dim3(kLockThreads);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = c.stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(s.C);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    if (cudaLaunchKernelEx(&cfg, kernel, a) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    c.launched();
    return true;
}

template<class T>
bool lockstep_feasible(int C)
{
    auto kernel = k_ilu_lockstep<T, false>;
    if (C > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(C));
    cfg.blockDim = dim3(kLockThreads);
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = static_cast<unsigned>(C);
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int clusters = 0;
    if (cudaOccupancyMaxActiveClusters(&clusters, kernel, &cfg) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return clusters >= 1;
}

template<class T>
__global__ void k_lock_gather(std::size_t count, const long long* src, const T* vals, T* out)
{
    const std::size_t i = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) out[i] = vals[src[i]];
}

}  // namespace

// Symbolic setup of one sweep (lower: forward, upper: backward): the
// lane-tasks of every level cut into chunks, and per entry where its
// dependency is read.  Leaves s.ready false when a level is wider than the
// cluster's lanes, the DAG is shallow, or no cluster can run.
void build_lockstep_sweep(Context& ctx, LockstepSweep& s, std::size_t owned, std::size_t bs, owtk_dtype dtype,
                          const std::vector<std::int32_t>& level, const std::vector<std::int32_t>& rowptr,
                          const std::vector<std::int32_t>& cols, const std::vector<std::int32_t>& diagpos,
                          bool backward)
{
    s = LockstepSweep{};
    const char* env = std::getenv("OWTK_LOCKSTEP_SWEEP");
    if (env && std::atoi(env) == 0) return;
    const std::size_t n = owned;
    if (n < 4096 || bs == 0 || bs > 32) return;
    std::int32_t D = 0;
    for (const auto l : level) D = std::max(D, l + 1);
    if (D < 16) return;
    std::vector<std::int32_t> count(static_cast<std::size_t>(D) + 1, 0);
    for (const auto l : level) ++count[static_cast<std::size_t>(l) + 1];
    std::int32_t widest = 0;
    for (std::int32_t l = 0; l < D; ++l) widest = std::max(widest, count[static_cast<std::size_t>(l) + 1]);
    for (std::size_t i = 1; i < count.size(); ++i) count[i] += count[i - 1];
    int C = 0;
    for (const int cand : {16, 8}) {
        const std::int64_t cap = static_cast<std::int64_t>(cand) * (kLockThreads / static_cast<int>(bs));
        if (widest > cap) continue;
        if (dtype == OWTK_F64 ? lockstep_feasible<double>(cand) : lockstep_feasible<float>(cand)) {
            C = cand;
            break;
        }
    }
    if (C == 0) return;
    // Rows by (level, row); chunk k of a level: rows [k w / C, (k+1) w / C).
    std::vector<std::int32_t> order(n);
    {
        std::vector<std::int32_t> next(count.begin(), count.end() - 1);
        for (std::size_t r = 0; r < n; ++r)
            order[static_cast<std::size_t>(next[static_cast<std::size_t>(level[r])]++)] = static_cast<std::int32_t>(r);
    }
    std::vector<std::int32_t> owner(n), local(n);
    std::vector<int2> blk(static_cast<std::size_t>(D) * C);
    std::vector<std::int32_t> task_io;
    std::vector<int2> task_ent;
    std::vector<std::int32_t> ent_loc;
    std::vector<long long> ent_src;
    task_io.reserve(n * bs);
    task_ent.reserve(n * bs);
    for (std::int32_t l = 0; l < D; ++l) {
        const std::int32_t b = count[static_cast<std::size_t>(l)], w = count[static_cast<std::size_t>(l) + 1] - b;
        for (int k = 0; k < C; ++k) {
            const std::int32_t r0 = b + static_cast<std::int32_t>(static_cast<std::int64_t>(w) * k / C);
            const std::int32_t r1 = b + static_cast<std::int32_t>(static_cast<std::int64_t>(w) * (k + 1) / C);
            blk[static_cast<std::size_t>(l) * C + k] =
                int2{static_cast<int>(task_io.size()), static_cast<int>((r1 - r0) * static_cast<std::int32_t>(bs))};
            for (std::int32_t q = r0; q < r1; ++q) {
                const std::int32_t row = order[static_cast<std::size_t>(q)];
                owner[static_cast<std::size_t>(row)] = k;
                local[static_cast<std::size_t>(row)] = q - r0;
                const std::int32_t eb = backward ? diagpos[static_cast<std::size_t>(row)] + 1 : rowptr[static_cast<std::size_t>(row)];
                const std::int32_t ee = backward ? rowptr[static_cast<std::size_t>(row) + 1] : diagpos[static_cast<std::size_t>(row)];
                for (std::size_t c = 0; c < bs; ++c) {
                    task_io.push_back(static_cast<std::int32_t>(static_cast<std::size_t>(row) * bs + c));
                    task_ent.push_back(int2{static_cast<int>(ent_loc.size()), ee - eb});
                    for (std::int32_t e = eb; e < ee; ++e) {
                        const std::int32_t dep = cols[static_cast<std::size_t>(e)];
                        const std::int32_t back = level[static_cast<std::size_t>(row)] - level[static_cast<std::size_t>(dep)];
                        std::int32_t loc;
                        if (back == 1 || back == 2) {
                            const std::int32_t slot = local[static_cast<std::size_t>(dep)] * static_cast<std::int32_t>(bs) + static_cast<std::int32_t>(c);
                            loc = static_cast<std::int32_t>(static_cast<std::uint32_t>(INT_MIN)
                                                            | (static_cast<std::uint32_t>(back - 1) << 28)
                                                            | (static_cast<std::uint32_t>(owner[static_cast<std::size_t>(dep)]) << 20)
                                                            | static_cast<std::uint32_t>(slot));
                        } else {
                            loc = static_cast<std::int32_t>(static_cast<std::size_t>(dep) * bs + c);
                        }
                        ent_loc.push_back(loc);
                        ent_src.push_back(static_cast<long long>(e) * static_cast<long long>(bs) + static_cast<long long>(c));
                    }
                }
            }
        }
    }
    s.C = C;
    s.D = D;
    s.entries = ent_loc.size();
    s.blk = upload(ctx.stream, blk);
    s.task_io = upload(ctx.stream, task_io);
    s.task_ent = upload(ctx.stream, task_ent);
    s.ent_loc = upload(ctx.stream, ent_loc);
    s.ent_src = upload(ctx.stream, ent_src);
    s.ent_val.allocate(std::max<std::size_t>(1, s.entries) * (dtype == OWTK_F64 ? 8 : 4) + 16);
    s.ready = true;
}

namespace kern {

// preconditioner.hpp:320-363, one cluster, levels in lockstep; false when the
// preconditioner has no lockstep schedule or a launch was refused (the
// caller then runs another sweep).
template<class T> bool lockstep_ilu_apply(Context& c, Preconditioner& p, const T* in, T* out)
{
    if (!p.l_lower.ready || !p.l_upper.ready || p.block || p.storage != OWTK_F64) return false;
    // Factor values in task order, refreshed after every numeric factorisation.
    for (LockstepSweep* s : {&p.l_lower, &p.l_upper}) {
        if (s->gathered != p.numeric_updates && s->entries > 0) {
            k_lock_gather<T><<<static_cast<unsigned>((s->entries + 255) / 256), 256, 0, c.stream>>>(
                s->entries, s->ent_src.as<long long>(), p.d_fvalues.as<T>(), s->ent_val.as<T>());
            OWTK_CUDA(cudaGetLastError());
            c.launched();
            s->gathered = p.numeric_updates;
        }
    }
    LockArgs<T> a{};
    a.inv = p.inv_diag.as<T>();
    a.in = in;
    a.out = p.work.as<T>();
    if (!launch_lockstep<T, false>(c, p.l_lower, a)) return false;
    a.in = p.work.as<T>();
    a.out = out;
    if (!launch_lockstep<T, true>(c, p.l_upper, a)) return false;
    OWTK_CUDA(cudaGetLastError());
    return true;
}

template bool lockstep_ilu_apply<double>(Context&, Preconditioner&, const double*, double*);
template bool lockstep_ilu_apply<float>(Context&, Preconditioner&, const float*, float*);

}  // namespace kern
}  // namespace owtk
