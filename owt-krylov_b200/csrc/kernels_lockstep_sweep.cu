// ILU(k) applies level by level on one thread-block cluster (sm_100a): the
// forward and backward triangular sweeps of IluLevelPreconditioner::apply
// (preconditioner.hpp:320-363) with the levels taken in lockstep.
//
// The level-scheduled sweep of kernels_sweep.cu lets dependants poll their
// dependencies in L2, about 0.86 us per level on the 2M-vertex RCM mesh
// (2 x 2913 levels).  Here one cluster of C CTAs (16 when the device allows
// it, else 8) of 512 threads runs the sweep one level per step:
//   * every level's rows are cut into C contiguous chunks, one per CTA, and
//     a CTA's lanes take the (row, component) pairs of its chunk;
//   * a step ends with a cluster barrier (arrive.release / wait.acquire,
//     about 0.24 us measured), so the results of the steps before it are
//     final and visible when the next one starts: no polling, no sentinel;
//   * each CTA keeps its results of the last three levels in a shared-memory
//     ring; a dependency one or two levels back is read from its owner's
//     ring over distributed shared memory, an older one is final in global
//     memory and is copied into shared memory one step ahead;
//   * the data of a level's chunk — per lane its output index, entry count
//     and dependency locations (a record), its factor values, and the
//     chunk's list of older dependencies — lies contiguous in global memory
//     and arrives by bulk copies (cp.async.bulk, no multicast) three steps
//     ahead into a four-stage ring, so no lane waits on global memory
//     within a step.
// Per (row, component) the arithmetic is the reference's, term by term in
// entry order with explicit rounding, so results equal the CPU path bit for
// bit.  Every CTA runs every step, so every cluster barrier is met; the only
// other waits are on this CTA's own copies, bounded.

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
constexpr int kLockK = 6;           // terms per record (more: read from global memory at the step)
constexpr int kLockRing = 3;        // levels of results kept for the other CTAs
constexpr int kLockStages = 4;      // levels of data in flight
constexpr int kLockSpin = 1 << 24;  // polls of a copy's completion before giving up
constexpr int kLockHeader = 128;    // shared memory: kLockStages mbarriers, then kLockStages chunk descriptors

// Per lane of a chunk: output (and input, inverse diagonal) index, entries,
// first overflow entry, and the first kLockK entries' locations.
struct LockRec {
    int io, n, ovf, pad;
    int loc[kLockK];
    int pad2[2];
};
static_assert(sizeof(LockRec) == 48, "records are 16-byte multiples");

template<class T>
struct LockArgs {
    const int4* blk;        // D x C: first lane (16-aligned record index), lanes, first far entry, far entries
    const LockRec* recs;
    const T* vals;          // per lane kLockK factor values (0 past n)
    const int* far_src;     // per chunk: global indices of the dependencies older than two levels
    const int* ovf_loc;     // entries past the first kLockK of a row: location (near code or global index)
    const T* ovf_val;
    const T* inv;
    const T* in;
    T* out;
    unsigned* status;
    int D, C, max_lanes, max_far;
};

// A dependency one or two levels back lives in its owner's ring:
// loc = INT_MIN | (levels back - 1) << 28 | owner << 20 | slot.  Otherwise
// loc >= 0: in a record, the index into the chunk's far list; in the
// overflow list, the global index.
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

__device__ __forceinline__ void lock_cp(void* dst, const void* src, int bytes)
{
    const std::uint32_t d = smem_u32(dst);
    if (bytes == 8)
        asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(d), "l"(src) : "memory");
    else
        asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(d), "l"(src) : "memory");
}
__device__ __forceinline__ void lock_cp_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void lock_cp_wait1() { asm volatile("cp.async.wait_group 1;" ::: "memory"); }
__device__ __forceinline__ void lock_cp_wait0() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

__host__ __device__ constexpr std::size_t lock_round16(std::size_t b) { return (b + 15) & ~std::size_t(15); }

// Shared-memory layout of one stage for chunks of up to `lanes` lanes (even)
// and `far` far entries.
template<class T>
struct LockStageLayout {
    std::size_t recs, vals, fsrc, fval, in, inv, bytes;
    __host__ __device__ LockStageLayout(int lanes, int far)
    {
        recs = 0;
        vals = recs + static_cast<std::size_t>(lanes) * sizeof(LockRec);
        fsrc = vals + lock_round16(static_cast<std::size_t>(lanes) * kLockK * sizeof(T));
        fval = fsrc + lock_round16(static_cast<std::size_t>(far) * sizeof(int));
        in = fval + lock_round16(static_cast<std::size_t>(far) * sizeof(T));
        inv = in + lock_round16(static_cast<std::size_t>(lanes) * sizeof(T));
        bytes = inv + lock_round16(static_cast<std::size_t>(lanes) * sizeof(T));
    }
};

template<class T>
std::size_t lock_smem_bytes(int lanes, int far)
{
    return kLockHeader + kLockRing * kLockThreads * sizeof(T) + kLockStages * LockStageLayout<T>(lanes, far).bytes;
}

template<class T, bool BACKWARD>
__global__ void __launch_bounds__(kLockThreads, 1) k_ilu_lockstep(LockArgs<T> a)
{
    extern __shared__ __align__(16) unsigned char lock_smem[];
    std::uint64_t* bars = reinterpret_cast<std::uint64_t*>(lock_smem);   // kLockStages mbarriers
    int4* stage_blk = reinterpret_cast<int4*>(lock_smem + 32);            // kLockStages chunk descriptors
    T* ring = reinterpret_cast<T*>(lock_smem + kLockHeader);               // [kLockRing][kLockThreads]
    unsigned char* stages = lock_smem + kLockHeader + kLockRing * kLockThreads * sizeof(T);
    const LockStageLayout<T> lay(a.max_lanes, a.max_far);
    const unsigned rank = lock_rank();
    const int lane = threadIdx.x;
    const unsigned ring_base = smem_u32(ring);
    const auto stage = [&](int L) { return stages + static_cast<std::size_t>(L % kLockStages) * lay.bytes; };
    const auto bar = [&](int L) { return smem_u32(bars + (L % kLockStages)); };
    // Bulk copies of level L's records, values and far list, and its chunk
    // descriptor b into the stage (one thread; the others read the descriptor
    // after the next CTA barrier).
    const auto descriptor = [&](int L) {
        return L < a.D ? __ldg(a.blk + static_cast<long long>(L) * a.C + rank) : int4{0, 0, 0, 0};
    };
    const auto issue = [&](int L, int4 b) {
        if (L >= a.D) return;
        stage_blk[L % kLockStages] = b;
        const int lanes = (b.y + 1) & ~1;
        const int far = (b.w + 3) & ~3;
        const std::uint32_t rb = static_cast<std::uint32_t>(lanes) * sizeof(LockRec);
        const std::uint32_t vb = static_cast<std::uint32_t>(lanes) * kLockK * sizeof(T);
        const std::uint32_t fb = static_cast<std::uint32_t>(far) * sizeof(int);
        unsigned char* s = stage(L);
        mbar_arrive_expect_tx(bar(L), rb + vb + fb);
        const std::uint64_t pol = l2_policy_evict_first();
        if (rb) bulk_load(smem_u32(s + lay.recs), a.recs + b.x, rb, bar(L), pol);
        if (vb) bulk_load(smem_u32(s + lay.vals), a.vals + static_cast<long long>(b.x) * kLockK, vb, bar(L), pol);
        if (fb) bulk_load(smem_u32(s + lay.fsrc), a.far_src + b.z, fb, bar(L), pol);
    };
    // Level L's inputs, inverse diagonal and far dependencies into its stage
    // (all final by now); its bulk copies must have landed.
    bool ok = true;
    const auto gather = [&](int L) {
        if (L >= a.D) {
            lock_cp_commit();
            return;
        }
        if (ok && !mbar_wait_bounded(bar(L), (L / kLockStages) & 1, kLockSpin)) ok = false;   // one timeout at most
        const int4 b = stage_blk[L % kLockStages];
        unsigned char* s = stage(L);
        const LockRec* recs = reinterpret_cast<const LockRec*>(s + lay.recs);
        const int* fsrc = reinterpret_cast<const int*>(s + lay.fsrc);
        T* fval = reinterpret_cast<T*>(s + lay.fval);
        if (ok) {
            if (lane < b.y) {
                const int io = recs[lane].io;
                lock_cp(reinterpret_cast<T*>(s + lay.in) + lane, a.in + io, sizeof(T));
                if (BACKWARD) lock_cp(reinterpret_cast<T*>(s + lay.inv) + lane, a.inv + io, sizeof(T));
            }
            for (int i = lane; i < b.w; i += kLockThreads) lock_cp(fval + i, a.out + fsrc[i], sizeof(T));
        }
        lock_cp_commit();
    };

    if (lane == 0) {
        for (int s = 0; s < kLockStages; ++s) mbar_init(smem_u32(bars + s), 1);
        fence_proxy_async_smem();
    }
    __syncthreads();
    int4 next{};   // lane 0: the descriptor of the level issued at the next step, loaded a step ahead
    if (lane == 0) {
        issue(0, descriptor(0));
        issue(1, descriptor(1));
        issue(2, descriptor(2));
        next = descriptor(3);
    }
    __syncthreads();   // the descriptors of levels 0-2
    gather(0);
    lock_barrier();   // every CTA of the cluster has started (its ring exists)
    for (int M = 0; M < a.D; ++M) {
        if (lane == 0) {   // into the stage of level M-1, finished before the last barrier
            issue(M + 3, next);
            next = descriptor(M + 4);
        }
        gather(M + 1);                 // level M+1's far dependencies are at most M-2: final
        lock_cp_wait1();               // this lane's copies for level M have landed,
        __syncthreads();               // and every lane's (far values are shared)
        const int4 b = stage_blk[M % kLockStages];
        if (ok && lane < b.y) {
            unsigned char* s = stage(M);
            const LockRec& r = reinterpret_cast<const LockRec*>(s + lay.recs)[lane];
            const T* val = reinterpret_cast<const T*>(s + lay.vals) + lane * kLockK;
            const T* fval = reinterpret_cast<const T*>(s + lay.fval);
            T acc = reinterpret_cast<const T*>(s + lay.in)[lane];
            T v[kLockK];
#pragma unroll
            for (int k = 0; k < kLockK; ++k) {
                if (k < r.n) {
                    const int loc = r.loc[k];
                    if (loc_near(loc)) {
                        const int rr = (M - loc_back(loc)) % kLockRing;
                        v[k] = lock_ld(lock_mapa(ring_base + static_cast<unsigned>((rr * kLockThreads + loc_slot(loc)) * sizeof(T)),
                                                 loc_owner(loc)),
                                       (T*)nullptr);
                    } else {
                        v[k] = fval[loc];
                    }
                }
            }
#pragma unroll
            for (int k = 0; k < kLockK; ++k)
                if (k < r.n) acc = sub_rn(acc, mul_rn(val[k], v[k]));
            for (int k = kLockK; k < r.n; ++k) {   // rows with more terms: the rest from global memory
                const int e = r.ovf + (k - kLockK);
                const int loc = __ldg(a.ovf_loc + e);
                T x;
                if (loc_near(loc)) {
                    const int rr = (M - loc_back(loc)) % kLockRing;
                    x = lock_ld(lock_mapa(ring_base + static_cast<unsigned>((rr * kLockThreads + loc_slot(loc)) * sizeof(T)),
                                          loc_owner(loc)),
                                (T*)nullptr);
                } else {
                    x = __ldcg(a.out + loc);
                }
                acc = sub_rn(acc, mul_rn(__ldg(a.ovf_val + e), x));
            }
            if (BACKWARD) acc = mul_rn(acc, reinterpret_cast<const T*>(s + lay.inv)[lane]);
            ring[(M % kLockRing) * kLockThreads + lane] = acc;
            a.out[r.io] = acc;
        }
        lock_barrier();
    }
    lock_cp_wait0();
    if (!ok && lane == 0) atomicOr(a.status, kErrTimeout);
    // Copies still in flight (issued for levels past the end) cannot exist:
    // issue() and gather() do nothing past level D-1.
}

template<class T, bool BACKWARD>
bool launch_lockstep(Context& c, const LockstepSweep& s, LockArgs<T> a)
{
    auto kernel = k_ilu_lockstep<T, BACKWARD>;
    const std::size_t smem = lock_smem_bytes<T>(s.max_lanes, s.max_far);
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess
        || (s.C > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
        cudaGetLastError();
        return false;
    }
    a.blk = s.blk.as<int4>();
    a.recs = s.recs.as<LockRec>();
    a.vals = s.vals.as<T>();
    a.far_src = s.far_src.as<int>();
    a.ovf_loc = s.ovf_loc.as<int>();
    a.ovf_val = s.ovf_val.as<T>();
    a.D = s.D;
    a.C = s.C;
    a.max_lanes = s.max_lanes;
    a.max_far = s.max_far;
    a.status = c.status.as<unsigned>();
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(s.C));
    cfg.blockDim = dim3(kLockThreads);
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
bool lockstep_feasible(int C, std::size_t smem)
{
    auto kernel = k_ilu_lockstep<T, true>;
    if (cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem)) != cudaSuccess
        || (C > 8 && cudaFuncSetAttribute(kernel, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)) {
        cudaGetLastError();
        return false;
    }
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(static_cast<unsigned>(C));
    cfg.blockDim = dim3(kLockThreads);
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

template<class T>
__global__ void k_lock_gather(std::size_t count, const long long* src, const T* vals, T* out)
{
    const std::size_t i = static_cast<std::size_t>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < count) out[i] = src[i] < 0 ? T(0) : vals[src[i]];
}

}  // namespace

// Symbolic setup of one sweep (lower: forward, upper: backward): the levels'
// chunks, their records and far lists, and where every factor value goes.
// Leaves s.ready false when a level is wider than the cluster's lanes, the
// DAG is shallow, the stages do not fit shared memory, or no cluster can run.
void build_lockstep_sweep(Context& ctx, LockstepSweep& s, std::size_t owned, std::size_t bs, owtk_dtype dtype,
                          const std::vector<std::int32_t>& level, const std::vector<std::int32_t>& rowptr,
                          const std::vector<std::int32_t>& cols, const std::vector<std::int32_t>& diagpos,
                          bool backward)
{
    s = LockstepSweep{};
    const char* env = std::getenv("OWTK_LOCKSTEP_SWEEP");   // opt-in: slower than the level-scheduled sweep
    if (!env || std::atoi(env) == 0) return;
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
    std::vector<std::int32_t> order(n);
    {
        std::vector<std::int32_t> next(count.begin(), count.end() - 1);
        for (std::size_t r = 0; r < n; ++r)
            order[static_cast<std::size_t>(next[static_cast<std::size_t>(level[r])]++)] = static_cast<std::int32_t>(r);
    }
    const std::size_t es = dtype == OWTK_F64 ? 8 : 4;
    for (const int C : {16, 8}) {
        if (static_cast<std::int64_t>(widest) > static_cast<std::int64_t>(C) * (kLockThreads / static_cast<int>(bs)))
            continue;
        std::vector<std::int32_t> owner(n), local(n);
        std::vector<int4> blk(static_cast<std::size_t>(D) * C);
        std::vector<LockRec> recs;
        std::vector<long long> vsrc;
        std::vector<std::int32_t> far_src, ovf_loc;
        std::vector<long long> ovf_src;
        int max_lanes = 2, max_far = 4;
        recs.reserve(n * bs + 2 * static_cast<std::size_t>(D) * C);
        for (std::int32_t l = 0; l < D; ++l) {
            const std::int32_t b = count[static_cast<std::size_t>(l)], w = count[static_cast<std::size_t>(l) + 1] - b;
            for (int k = 0; k < C; ++k) {
                const std::int32_t r0 = b + static_cast<std::int32_t>(static_cast<std::int64_t>(w) * k / C);
                const std::int32_t r1 = b + static_cast<std::int32_t>(static_cast<std::int64_t>(w) * (k + 1) / C);
                for (std::int32_t q = r0; q < r1; ++q) {
                    owner[static_cast<std::size_t>(order[static_cast<std::size_t>(q)])] = k;
                    local[static_cast<std::size_t>(order[static_cast<std::size_t>(q)])] = q - r0;
                }
            }
        }
        for (std::int32_t l = 0; l < D; ++l) {
            const std::int32_t b = count[static_cast<std::size_t>(l)], w = count[static_cast<std::size_t>(l) + 1] - b;
            for (int k = 0; k < C; ++k) {
                const std::int32_t r0 = b + static_cast<std::int32_t>(static_cast<std::int64_t>(w) * k / C);
                const std::int32_t r1 = b + static_cast<std::int32_t>(static_cast<std::int64_t>(w) * (k + 1) / C);
                const int lanes = (r1 - r0) * static_cast<int>(bs);
                const int first = static_cast<int>(recs.size());
                const int far0 = static_cast<int>(far_src.size());
                for (std::int32_t q = r0; q < r1; ++q) {
                    const std::int32_t row = order[static_cast<std::size_t>(q)];
                    const std::int32_t eb = backward ? diagpos[static_cast<std::size_t>(row)] + 1 : rowptr[static_cast<std::size_t>(row)];
                    const std::int32_t ee = backward ? rowptr[static_cast<std::size_t>(row) + 1] : diagpos[static_cast<std::size_t>(row)];
                    for (std::size_t c = 0; c < bs; ++c) {
                        LockRec rec{};
                        rec.io = static_cast<int>(static_cast<std::size_t>(row) * bs + c);
                        rec.n = ee - eb;
                        rec.ovf = static_cast<int>(ovf_loc.size());
                        for (std::int32_t e = eb; e < ee; ++e) {
                            const int kk = e - eb;
                            const std::int32_t dep = cols[static_cast<std::size_t>(e)];
                            const std::int32_t back = level[static_cast<std::size_t>(row)] - level[static_cast<std::size_t>(dep)];
                            const std::int32_t gidx = static_cast<std::int32_t>(static_cast<std::size_t>(dep) * bs + c);
                            std::int32_t near_loc = 0;
                            const bool near = back == 1 || back == 2;
                            if (near) {
                                const std::int32_t slot = local[static_cast<std::size_t>(dep)] * static_cast<std::int32_t>(bs) + static_cast<std::int32_t>(c);
                                near_loc = static_cast<std::int32_t>(static_cast<std::uint32_t>(INT_MIN)
                                                                     | (static_cast<std::uint32_t>(back - 1) << 28)
                                                                     | (static_cast<std::uint32_t>(owner[static_cast<std::size_t>(dep)]) << 20)
                                                                     | static_cast<std::uint32_t>(slot));
                            }
                            const long long src = static_cast<long long>(e) * static_cast<long long>(bs) + static_cast<long long>(c);
                            if (kk < kLockK) {
                                if (near) {
                                    rec.loc[kk] = near_loc;
                                } else {
                                    rec.loc[kk] = static_cast<int>(far_src.size()) - far0;
                                    far_src.push_back(gidx);
                                }
                                vsrc.push_back(src);
                            } else {
                                ovf_loc.push_back(near ? near_loc : gidx);
                                ovf_src.push_back(src);
                            }
                        }
                        for (int kk = rec.n; kk < kLockK; ++kk) vsrc.push_back(-1);
                        recs.push_back(rec);
                    }
                }
                if (lanes & 1) {   // chunks start at even records: bulk copies of 16-byte multiples
                    recs.push_back(LockRec{});
                    for (int kk = 0; kk < kLockK; ++kk) vsrc.push_back(-1);
                }
                const int far = static_cast<int>(far_src.size()) - far0;
                while ((far_src.size() - static_cast<std::size_t>(far0)) & 3) far_src.push_back(0);
                blk[static_cast<std::size_t>(l) * C + k] = int4{first, lanes, far0, far};
                max_lanes = std::max(max_lanes, (lanes + 1) & ~1);
                max_far = std::max(max_far, (far + 3) & ~3);
            }
        }
        const std::size_t smem = es == 8 ? lock_smem_bytes<double>(max_lanes, max_far)
                                         : lock_smem_bytes<float>(max_lanes, max_far);
        if (smem > 227 * 1024) continue;
        if (!(es == 8 ? lockstep_feasible<double>(C, smem) : lockstep_feasible<float>(C, smem))) continue;
        if (ovf_loc.empty()) {
            ovf_loc.push_back(0);
            ovf_src.push_back(-1);
        }
        if (far_src.empty()) far_src.push_back(0);
        s.C = C;
        s.D = D;
        s.max_lanes = max_lanes;
        s.max_far = max_far;
        s.values = vsrc.size();
        s.ovf_values = ovf_src.size();
        s.blk = upload(ctx.stream, blk);
        s.recs = upload(ctx.stream, recs);
        s.vsrc = upload(ctx.stream, vsrc);
        s.far_src = upload(ctx.stream, far_src);
        s.ovf_loc = upload(ctx.stream, ovf_loc);
        s.ovf_src = upload(ctx.stream, ovf_src);
        s.vals.allocate(s.values * es + 16);
        s.ovf_val.allocate(s.ovf_values * es + 16);
        s.ready = true;
        return;
    }
}

namespace kern {

// preconditioner.hpp:320-363, one cluster, levels in lockstep; false when the
// preconditioner has no lockstep schedule or a launch was refused (the
// caller then runs another sweep).
template<class T> bool lockstep_ilu_apply(Context& c, Preconditioner& p, const T* in, T* out)
{
    if (!p.l_lower.ready || !p.l_upper.ready || p.block || p.storage != OWTK_F64) return false;
    // Factor values in record order, refreshed after every numeric factorisation.
    for (LockstepSweep* s : {&p.l_lower, &p.l_upper}) {
        if (s->gathered == p.numeric_updates) continue;
        for (int part = 0; part < 2; ++part) {
            const std::size_t cnt = part ? s->ovf_values : s->values;
            if (cnt == 0) continue;
            k_lock_gather<T><<<static_cast<unsigned>((cnt + 255) / 256), 256, 0, c.stream>>>(
                cnt, (part ? s->ovf_src : s->vsrc).as<long long>(), p.d_fvalues.as<T>(),
                (part ? s->ovf_val : s->vals).as<T>());
            OWTK_CUDA(cudaGetLastError());
            c.launched();
        }
        s->gathered = p.numeric_updates;
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
