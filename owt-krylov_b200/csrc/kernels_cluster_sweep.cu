// ILU(k) applies by one thread-block cluster (sm_100a): the forward and
// backward triangular sweeps of IluLevelPreconditioner::apply
// (preconditioner.hpp:320-363) with the dependency values passed through
// distributed shared memory instead of L2.
//
// The level-scheduled sweep of kernels_sweep.cu spreads its warps over every
// SM and publishes each result to global memory, where dependants poll it;
// on an RCM-ordered mesh every level costs about two L2 round trips
// (~0.86 us per level on the 2M-vertex mesh, 2 x 2913 levels per apply).
// Here one cluster of C CTAs (16 when the device allows it, else 8) runs the
// whole sweep:
//   * tasks (32 rows of one level, one row with all its components per
//     lane, in level order) are dealt round-robin to the CTAs; every CTA runs
//     its tasks in order with its warps taking them from a shared-memory
//     ticket.  Wide tasks keep many levels in flight with the few warps of
//     one cluster (a task of 32/bs rows, one (row, component) per lane, gave
//     ~3.7 levels in flight and lost to the sweep over the whole GPU);
//   * each CTA keeps its results in a shared-memory ring of R rows; a row
//     whose dependency is recent polls the owner CTA's ring slot over
//     distributed shared memory (ld.relaxed.cluster.shared::cluster) until the
//     slot holds a value instead of the sentinel — one DSMEM round trip;
//   * the levels are cut into epochs of K levels with a cluster barrier
//     after each, so no CTA is ever more than one epoch ahead.  A dependency
//     from the same or the previous epoch is read from its owner's ring; an
//     older one is final and, after the barriers, visible in global memory,
//     where it is read without polling.  During epoch e each CTA resets to
//     the sentinel the ring slots of its epoch e+1 rows, whose previous
//     occupants are from epoch e-2 and are read by nobody; R holds three
//     consecutive epochs of a CTA's rows, so live slots are never reused.
// Every result is also written to global memory (the sweep's output).  The
// schedule, the ring slot of every row and, for every factor entry, where
// its dependency is read from are computed once at symbolic setup.
//
// Progress: tasks are dealt in level order and every CTA runs its own in
// order, so the unfinished task with the lowest index always has its
// dependencies done and a warp working on it.  Every wait is bounded
// (spin_limit polls): a wait that gives up sets the timeout bit and the
// sweep carries on, so every thread reaches every barrier.
//
// Per (row, component) the arithmetic is the reference's, term by term in
// entry order with explicit rounding, so results equal the CPU path bit for
// bit.
//
// Status: opt-in (OWTK_CLUSTER_SWEEP=1 when the preconditioner is created).
// On the 2M-vertex RCM-ordered disk mesh (bs 3, 2 x 2913 levels) one
// cluster cannot keep enough rows in flight: an ILU(0) apply took 7.8 ms with
// tasks of 32/bs rows and 19.7 ms with one row per lane, against 5.0 ms for
// the level-scheduled sweep over the whole GPU, which stays the default.

#include <cuda.h>

#include <algorithm>
#include <cstdint>
#include <cstdlib>
#include <vector>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

constexpr int kClusterThreads = 512;
constexpr unsigned kGlobalDep = 0xffffffffu;   // dependency read from global memory
constexpr int kOwnerShift = 27;                // loc = owner << 27 | ring slot
constexpr int kSpinDefault = 1 << 22;

template<class T> struct Sent;
template<> struct Sent<double> {
    using U = unsigned long long;
    static constexpr U kSentinel = 0x7ff0dead5eed0badull;   // signalling NaN
    static constexpr U kQuietNan = 0x7ff8000000000000ull;
};
template<> struct Sent<float> {
    using U = unsigned;
    static constexpr U kSentinel = 0x7f80deadu;
    static constexpr U kQuietNan = 0x7fc00000u;
};

template<class T>
struct ClusterArgs {
    const int4* recs;         // per position: row, first and end dependency entry
    const int* rows;          // processing order, CTA-major
    const int* task_ptr;      // tasks + 1 positions in rows (CTA-major task order)
    const int* epoch_task;    // C * (E + 1): first task of each epoch per CTA
    const int* cta_first;     // C: first position of each CTA's rows
    const int* rowptr;
    const int* cols;
    const int* diagpos;
    const unsigned* loc;      // per factor entry: owner << 27 | slot, or kGlobalDep
    const T* vals;
    const T* inv;
    const T* in;              // forward: b; backward: the forward result
    T* out;                   // forward: work; backward: z
    int bs, C, E, R, spin_limit;
    unsigned* status;
};

__device__ __forceinline__ unsigned cluster_rank()
{
    unsigned r;
    asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(r));
    return r;
}

__device__ __forceinline__ void cluster_barrier()
{
    asm volatile("barrier.cluster.arrive.release;\n\tbarrier.cluster.wait.acquire;" ::: "memory");
}

__device__ __forceinline__ unsigned map_to(unsigned local_addr, unsigned cta)
{
    unsigned r;
    asm volatile("mapa.shared::cluster.u32 %0, %1, %2;" : "=r"(r) : "r"(local_addr), "r"(cta));
    return r;
}

__device__ __forceinline__ unsigned long long ld_cluster(unsigned addr, double*)
{
    unsigned long long v;
    asm volatile("ld.relaxed.cluster.shared::cluster.b64 %0, [%1];" : "=l"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ unsigned ld_cluster(unsigned addr, float*)
{
    unsigned v;
    asm volatile("ld.relaxed.cluster.shared::cluster.b32 %0, [%1];" : "=r"(v) : "r"(addr) : "memory");
    return v;
}
__device__ __forceinline__ void st_cluster(unsigned addr, unsigned long long v)
{
    asm volatile("st.relaxed.cluster.shared::cluster.b64 [%0], %1;" ::"r"(addr), "l"(v) : "memory");
}
__device__ __forceinline__ void st_cluster(unsigned addr, unsigned v)
{
    asm volatile("st.relaxed.cluster.shared::cluster.b32 [%0], %1;" ::"r"(addr), "r"(v) : "memory");
}

__device__ __forceinline__ double as_value(unsigned long long u) { return __longlong_as_double(static_cast<long long>(u)); }
__device__ __forceinline__ float as_value(unsigned u) { return __uint_as_float(u); }
__device__ __forceinline__ unsigned long long as_bits(double v) { return static_cast<unsigned long long>(__double_as_longlong(v)); }
__device__ __forceinline__ unsigned as_bits(float v) { return __float_as_uint(v); }

template<class T> __device__ __forceinline__ T ld_global_cg(const T* p) { return __ldcg(p); }

// One row per lane, all bs components: y_c = own_c - sum_e vals[e][c] *
// dep[col_e][c] over the row's dependency entries [b, e) in entry order
// (sub_rn(y, mul_rn(v, x)), the reference's rounding), then FIN: 0 y,
// 1 y * fin_c.  Recent dependencies are polled in their owner's ring, older
// ones read from `dep` in global memory.  A warp-uniform loop that ends when
// every lane has published its row.
template<class T, int BS, int FIN>
__device__ __forceinline__ void cluster_row(bool valid, const T (&own)[BS], const ClusterArgs<T>& a, const T* dep,
                                            int b, int e, const T (&fin)[BS], T* gdst, unsigned ring_dst,
                                            unsigned ring_base)
{
    using U = typename Sent<T>::U;
    constexpr int kC = 4;   // entries per round
    T y[BS];
#pragma unroll
    for (int c = 0; c < BS; ++c) y[c] = own[c];
    T fv[kC][BS];
    U xb[kC][BS];
    unsigned raddr[kC];
    bool on[kC], remote[kC];
    int k0 = b, it = 0;
    bool loaded = false, done = !valid;
    auto publish_row = [&]() {
#pragma unroll
        for (int c = 0; c < BS; ++c) {
            T r = FIN == 1 ? mul_rn(y[c], fin[c]) : y[c];
            if (r != r) r = as_value(Sent<T>::kQuietNan);
            gdst[c] = r;
            st_cluster(ring_dst + c * static_cast<unsigned>(sizeof(T)), as_bits(r));
        }
    };
    for (;;) {
        if (!done) {
            if (!loaded && k0 >= e) {
                publish_row();
                done = true;
            } else {
                if (!loaded) {
#pragma unroll
                    for (int j = 0; j < kC; ++j) {
                        const int k = k0 + j;
                        on[j] = k < e;
                        remote[j] = false;
                        if (on[j]) {
                            const int col = a.cols[k];
                            const unsigned l = a.loc[k];
#pragma unroll
                            for (int c = 0; c < BS; ++c) fv[j][c] = a.vals[static_cast<std::size_t>(k) * BS + c];
                            if (l == kGlobalDep) {
#pragma unroll
                                for (int c = 0; c < BS; ++c)
                                    xb[j][c] = as_bits(ld_global_cg(dep + static_cast<std::size_t>(col) * BS + c));
                            } else {
                                remote[j] = true;
                                const unsigned slot = l & ((1u << kOwnerShift) - 1);
                                raddr[j] = map_to(ring_base + slot * BS * static_cast<unsigned>(sizeof(T)),
                                                  l >> kOwnerShift);
#pragma unroll
                                for (int c = 0; c < BS; ++c)
                                    xb[j][c] = ld_cluster(raddr[j] + c * static_cast<unsigned>(sizeof(T)),
                                                          static_cast<T*>(nullptr));
                            }
                        }
                    }
                    loaded = true;
                }
                bool pending = false;
#pragma unroll
                for (int j = 0; j < kC; ++j)
#pragma unroll
                    for (int c = 0; c < BS; ++c) pending |= on[j] && remote[j] && xb[j][c] == Sent<T>::kSentinel;
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
                    for (int j = 0; j < kC; ++j)
                        if (on[j]) {
#pragma unroll
                            for (int c = 0; c < BS; ++c) y[c] = sub_rn(y[c], mul_rn(fv[j][c], as_value(xb[j][c])));
                        }
                    k0 += kC;
                    loaded = false;
                    if (k0 >= e) {
                        publish_row();
                        done = true;
                    }
                } else {
                    // Re-poll the first pending dependency only (the others are
                    // older and usually ready by then), backing off while it
                    // waits: polls of many lanes would otherwise crowd the
                    // cluster's shared-memory network.
                    ++it;
                    if (it >= 16) __nanosleep(it >= 256 ? 256 : 32);
                    bool first_pending = true;
#pragma unroll
                    for (int j = 0; j < kC; ++j) {
                        bool mine = false;
#pragma unroll
                        for (int c = 0; c < BS; ++c) mine |= on[j] && remote[j] && xb[j][c] == Sent<T>::kSentinel;
                        if (mine && first_pending) {
                            first_pending = false;
#pragma unroll
                            for (int c = 0; c < BS; ++c)
                                if (xb[j][c] == Sent<T>::kSentinel)
                                    xb[j][c] = ld_cluster(raddr[j] + c * static_cast<unsigned>(sizeof(T)),
                                                          static_cast<T*>(nullptr));
                        }
                    }
                }
            }
        }
        if (!__any_sync(0xffffffffu, !done)) break;
    }
}

template<class T, bool BACKWARD, int BS>
__global__ void __launch_bounds__(kClusterThreads, 1) k_cluster_sweep(ClusterArgs<T> a)
{
    using U = typename Sent<T>::U;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    U* ring = reinterpret_cast<U*>(smem_raw);
    __shared__ unsigned ticket[2];
    const unsigned k = cluster_rank();
    const int lane = threadIdx.x & 31;
    const unsigned ring_base = static_cast<unsigned>(__cvta_generic_to_shared(ring));
    const int first = a.cta_first[k];
    const int* et = a.epoch_task + static_cast<std::size_t>(k) * (a.E + 1);
    // Ring slots of this CTA's epoch-0 rows start as the sentinel; the rest
    // are reset one epoch ahead.
    {
        const int p0 = a.task_ptr[et[0]], p1 = a.task_ptr[et[a.E > 0 ? 1 : 0]];
        for (int i = threadIdx.x; i < (p1 - p0) * BS; i += blockDim.x) {
            const int p = p0 + i / BS;
            ring[((p - first) % a.R) * BS + i % BS] = Sent<T>::kSentinel;
        }
    }
    if (threadIdx.x < 2) ticket[threadIdx.x] = 0;
    cluster_barrier();
    for (int ep = 0; ep < a.E; ++ep) {
        const int t0 = et[ep], t1 = et[ep + 1];
        for (;;) {
            unsigned j = 0;
            if (lane == 0) j = atomicAdd(&ticket[ep & 1], 1u);
            j = __shfl_sync(0xffffffffu, j, 0);
            const int t = t0 + static_cast<int>(j);
            if (t >= t1) break;
            const int s = a.task_ptr[t], nrows = a.task_ptr[t + 1] - s;
            const bool valid = lane < nrows;
            const int p = s + (valid ? lane : 0);
            const int4 rec = a.recs[p];
            const int row = valid ? rec.x : 0;
            const std::size_t o = static_cast<std::size_t>(row) * BS;
            const unsigned ring_dst = ring_base + static_cast<unsigned>(((p - first) % a.R) * BS * sizeof(T));
            T own[BS], fin[BS];
#pragma unroll
            for (int c = 0; c < BS; ++c) {
                own[c] = valid ? a.in[o + c] : T(0);
                fin[c] = BACKWARD && valid ? a.inv[o + c] : T(1);
            }
            if constexpr (!BACKWARD)
                cluster_row<T, BS, 0>(valid, own, a, a.out, rec.y, rec.z, fin, a.out + o, ring_dst, ring_base);
            else
                cluster_row<T, BS, 1>(valid, own, a, a.out, rec.y, rec.z, fin, a.out + o, ring_dst, ring_base);
        }
        // Reset the slots of this CTA's next-epoch rows (their previous rows
        // are two epochs old) and the next epoch's ticket.
        if (ep + 1 < a.E) {
            const int p0 = a.task_ptr[et[ep + 1]], p1 = a.task_ptr[et[ep + 2]];
            for (int i = threadIdx.x; i < (p1 - p0) * BS; i += blockDim.x) {
                const int pp = p0 + i / BS;
                st_cluster(ring_base + static_cast<unsigned>((((pp - first) % a.R) * BS + i % BS) * sizeof(T)),
                           Sent<T>::kSentinel);
            }
            if (threadIdx.x == 0) ticket[(ep + 1) & 1] = 0;
        }
        cluster_barrier();
    }
}

template<class T, bool BACKWARD>
auto cluster_kernel(int bs)
{
    switch (bs) {
    case 1: return k_cluster_sweep<T, BACKWARD, 1>;
    case 2: return k_cluster_sweep<T, BACKWARD, 2>;
    case 3: return k_cluster_sweep<T, BACKWARD, 3>;
    default: return k_cluster_sweep<T, BACKWARD, 4>;
    }
}

template<class T, bool BACKWARD>
bool launch_cluster(Context& c, const ClusterSweep& s, ClusterArgs<T> a)
{
    auto kernel = cluster_kernel<T, BACKWARD>(a.bs);
    const std::size_t smem = static_cast<std::size_t>(s.R) * a.bs * sizeof(T);
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess
        || (s.C > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
        cudaGetLastError();
        return false;
    }
    a.rows = s.rows.as<int>();
    a.recs = s.recs.as<int4>();
    a.task_ptr = s.task_ptr.as<int>();
    a.epoch_task = s.epoch_task.as<int>();
    a.cta_first = s.cta_first.as<int>();
    a.C = s.C;
    a.E = s.E;
    a.R = s.R;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(s.C));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = smem;
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
bool cluster_feasible(int C, std::size_t smem, int bs)
{
    auto kernel = cluster_kernel<T, false>(bs);
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess
        || (C > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(C));
    cfg.blockDim = dim3(kClusterThreads);
    cfg.dynamicSmemBytes = smem;
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

}  // namespace

// Symbolic setup of one sweep (lower: forward, upper: backward) over the ILU
// factor pattern.  Fills `loc` for the sweep's dependency entries.  Leaves
// s.ready false when the sweep is too shallow to gain or its ring does not
// fit the shared memory of a cluster this device can run.
void build_cluster_sweep(Context& ctx, ClusterSweep& s, std::size_t owned, std::size_t bs, owtk_dtype dtype,
                         const std::vector<std::int32_t>& level, const std::vector<std::int32_t>& rowptr,
                         const std::vector<std::int32_t>& cols, const std::vector<std::int32_t>& diagpos,
                         bool backward, std::vector<std::uint32_t>& loc)
{
    s = ClusterSweep{};
    const char* env = std::getenv("OWTK_CLUSTER_SWEEP");
    if (env == nullptr || std::atoi(env) == 0) return;   // opt-in: slower than the level-scheduled sweep
    const std::size_t n = owned;
    if (n < 4096 || bs == 0 || bs > 4) return;
    const std::size_t es = dtype == OWTK_F64 ? 8 : 4;
    std::int32_t depth = 0;
    for (const auto l : level) depth = std::max(depth, l + 1);
    if (depth < 16 || n / static_cast<std::size_t>(depth) < 16) return;   // near-sequential DAGs: keep the plain sweep
    // Tasks: rows by (level, row), 32 rows (one per lane), never across a level.
    const int per_task = 32;
    std::vector<std::int32_t> count(static_cast<std::size_t>(depth) + 1, 0);
    for (const auto l : level) ++count[static_cast<std::size_t>(l) + 1];
    for (std::size_t i = 1; i < count.size(); ++i) count[i] += count[i - 1];
    std::vector<std::int32_t> order(n);
    {
        std::vector<std::int32_t> next(count.begin(), count.end() - 1);
        for (std::size_t r = 0; r < n; ++r) order[static_cast<std::size_t>(next[static_cast<std::size_t>(level[r])]++)] = static_cast<std::int32_t>(r);
    }
    struct Task { std::int32_t begin, end, level; };
    std::vector<Task> tasks;
    for (std::int32_t l = 0; l < depth; ++l)
        for (std::int32_t p = count[static_cast<std::size_t>(l)]; p < count[static_cast<std::size_t>(l) + 1]; p += per_task)
            tasks.push_back({p, std::min(p + per_task, count[static_cast<std::size_t>(l) + 1]), l});
    const std::size_t smem_cap = 200 * 1024;
    for (const int C : {16, 8}) {
        // Rows per CTA per level.
        std::vector<std::vector<std::int32_t>> per_level(static_cast<std::size_t>(C),
                                                         std::vector<std::int32_t>(static_cast<std::size_t>(depth), 0));
        for (std::size_t t = 0; t < tasks.size(); ++t)
            per_level[t % static_cast<std::size_t>(C)][static_cast<std::size_t>(tasks[t].level)] += tasks[t].end - tasks[t].begin;
        // The largest epoch length K whose ring (three epochs of a CTA's rows) fits.
        int K = 0, R = 0;
        for (int cand = 64; cand >= 2; cand /= 2) {
            int worst = 0;
            const int E = (depth + cand - 1) / cand;
            for (int k = 0; k < C; ++k) {
                std::vector<int> ep(static_cast<std::size_t>(E), 0);
                for (int l = 0; l < depth; ++l) ep[static_cast<std::size_t>(l / cand)] += per_level[static_cast<std::size_t>(k)][static_cast<std::size_t>(l)];
                for (int e = 0; e < E; ++e) {
                    int w = ep[static_cast<std::size_t>(e)];
                    if (e + 1 < E) w += ep[static_cast<std::size_t>(e) + 1];
                    if (e + 2 < E) w += ep[static_cast<std::size_t>(e) + 2];
                    worst = std::max(worst, w);
                }
            }
            if (static_cast<std::size_t>(worst) * bs * es <= smem_cap) {
                K = cand;
                R = std::max(worst, 1);
                break;
            }
        }
        if (K == 0) continue;
        const std::size_t smem = static_cast<std::size_t>(R) * bs * es;
        if (!(dtype == OWTK_F64 ? cluster_feasible<double>(C, smem, static_cast<int>(bs))
                                 : cluster_feasible<float>(C, smem, static_cast<int>(bs))))
            continue;
        const int E = (depth + K - 1) / K;
        // CTA-major processing order; per row its owner and ring slot.
        std::vector<std::vector<std::size_t>> cta_tasks(static_cast<std::size_t>(C));
        for (std::size_t t = 0; t < tasks.size(); ++t) cta_tasks[t % static_cast<std::size_t>(C)].push_back(t);
        std::vector<std::int32_t> rows, task_ptr{0}, epoch_task(static_cast<std::size_t>(C) * (E + 1)), cta_first(static_cast<std::size_t>(C));
        std::vector<std::int32_t> owner(n), slot(n), row_epoch(n);
        rows.reserve(n);
        std::int32_t tcount = 0;
        for (int k = 0; k < C; ++k) {
            cta_first[static_cast<std::size_t>(k)] = static_cast<std::int32_t>(rows.size());
            int e_next = 0;
            for (const std::size_t t : cta_tasks[static_cast<std::size_t>(k)]) {
                const int e = tasks[t].level / K;
                while (e_next <= e) epoch_task[static_cast<std::size_t>(k) * (E + 1) + static_cast<std::size_t>(e_next++)] = tcount;
                for (std::int32_t q = tasks[t].begin; q < tasks[t].end; ++q) {
                    const std::int32_t r = order[static_cast<std::size_t>(q)];
                    owner[static_cast<std::size_t>(r)] = k;
                    slot[static_cast<std::size_t>(r)] = static_cast<std::int32_t>((rows.size() - static_cast<std::size_t>(cta_first[static_cast<std::size_t>(k)])) % static_cast<std::size_t>(R));
                    row_epoch[static_cast<std::size_t>(r)] = e;
                    rows.push_back(r);
                }
                task_ptr.push_back(static_cast<std::int32_t>(rows.size()));
                ++tcount;
            }
            while (e_next <= E) epoch_task[static_cast<std::size_t>(k) * (E + 1) + static_cast<std::size_t>(e_next++)] = tcount;
        }
        // Where each dependency entry is read: the owner's ring when the
        // dependency is from the same or the previous epoch, else global.
        loc.resize(cols.size(), kGlobalDep);
        for (std::size_t r = 0; r < n; ++r) {
            const std::int32_t b = backward ? diagpos[r] + 1 : rowptr[r];
            const std::int32_t e = backward ? rowptr[r + 1] : diagpos[r];
            for (std::int32_t q = b; q < e; ++q) {
                const auto col = static_cast<std::size_t>(cols[static_cast<std::size_t>(q)]);
                loc[static_cast<std::size_t>(q)] =
                    row_epoch[col] + 1 >= row_epoch[r]
                        ? (static_cast<std::uint32_t>(owner[col]) << kOwnerShift) | static_cast<std::uint32_t>(slot[col])
                        : kGlobalDep;
            }
        }
        s.C = C;
        s.K = K;
        s.E = E;
        s.R = R;
        s.tasks = static_cast<int>(tasks.size());
        std::vector<int4> recs(rows.size());
        for (std::size_t q = 0; q < rows.size(); ++q) {
            const auto r = static_cast<std::size_t>(rows[q]);
            recs[q] = backward ? int4{rows[q], diagpos[r] + 1, rowptr[r + 1], 0}
                               : int4{rows[q], rowptr[r], diagpos[r], 0};
        }
        s.recs = upload(ctx.stream, recs);
        s.rows = upload(ctx.stream, rows);
        s.task_ptr = upload(ctx.stream, task_ptr);
        s.epoch_task = upload(ctx.stream, epoch_task);
        s.cta_first = upload(ctx.stream, cta_first);
        s.ready = true;
        return;
    }
}

namespace kern {

// preconditioner.hpp:320-363 on one cluster; false when the preconditioner
// has no cluster schedule or the launch was refused (the caller then runs
// the level-scheduled sweep).
template<class T> bool cluster_ilu_apply(Context& c, Preconditioner& p, const T* in, T* out)
{
    if (!p.c_lower.ready || !p.c_upper.ready || p.block || p.storage != OWTK_F64 || p.d_floc.ptr == nullptr) return false;
    ClusterArgs<T> a{};
    a.rowptr = p.d_frowptr.as<int>();
    a.cols = p.d_fcols.as<int>();
    a.diagpos = p.d_fdiagpos.as<int>();
    a.loc = p.d_floc.as<unsigned>();
    a.vals = p.d_fvalues.as<T>();
    a.inv = p.inv_diag.as<T>();
    a.bs = static_cast<int>(p.bs);
    a.status = c.status.as<unsigned>();
    a.spin_limit = kSpinDefault;
    a.in = in;
    a.out = p.work.as<T>();
    if (!launch_cluster<T, false>(c, p.c_lower, a)) return false;
    a.in = p.work.as<T>();
    a.out = out;
    if (!launch_cluster<T, true>(c, p.c_upper, a)) {
        // The forward result is in work; finish with nothing half done: the
        // caller reruns the whole apply on the plain sweep.
        return false;
    }
    OWTK_CUDA(cudaGetLastError());
    return true;
}

template bool cluster_ilu_apply<double>(Context&, Preconditioner&, const double*, double*);
template bool cluster_ilu_apply<float>(Context&, Preconditioner&, const float*, float*);

}  // namespace kern
}  // namespace owtk
