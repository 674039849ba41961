// owtk_dot_batch_f64_noalloc: the batched dot product (w . basis_j and w . w)
// for callers that must not allocate device memory — for example code that
// runs while another library owns the device allocator, or a caller in a
// setting where cudaMalloc is forbidden or would synchronise the device.
// This entry point creates no context and calls no cudaMalloc / cudaFree or
// any allocating library routine: the caller passes device inputs and a
// device output, and the reduction's scratch (per-CTA partial sums and the
// last-CTA ticket) lives in one file-scope static __device__ array below.
//
// Limits and sharing rules:
//   * at most kMaxDots = 32 dot products per call (k <= 31 basis vectors plus
//     w . w); larger batches are rejected with OWTK_ERR_INVALID_ARGUMENT;
//   * the scratch is 32 x 592 partials plus the ticket (about 148 KiB), held
//     by every GPU that loads the library until the process exits;
//   * every call shares that one array, so calls whose kernels overlap on the
//     GPU (different streams, or different host threads) race and give wrong
//     results — serialise them.  The ticket, the only state that must start at
//     zero, is cleared by each call before its kernel runs;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture begins.  The address is cached for the life
//     of the process, so the entry point must not be used on a device after
//     cudaDeviceReset (which recreates the module at a new address).

#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "device_common.cuh"
#include "owtk_internal.h"

namespace owtk {
namespace {

using namespace dev;

constexpr int kMaxDots = 32;
constexpr int kMaxBlocks = 592;
constexpr int kMaxDevices = 64;
constexpr std::size_t kTicketSlot = static_cast<std::size_t>(kMaxDots) * kMaxBlocks;

// Partials [dot][block], then one slot whose first 4 bytes are the ticket.
static __device__ __align__(256) double g_noalloc_scratch[kTicketSlot + 32];

struct Pointers {
    const double* p[kMaxDots];
};

__global__ void __launch_bounds__(kThreads) k_dot_batch_noalloc(std::size_t n, int k, const double* __restrict__ w,
                                                                Pointers basis, double* scratch,
                                                                double* __restrict__ results)
{
    double acc[kMaxDots];
#pragma unroll
    for (int j = 0; j < kMaxDots; ++j) acc[j] = 0.0;
    const std::size_t stride = static_cast<std::size_t>(gridDim.x) * kThreads;
    for (std::size_t i = static_cast<std::size_t>(blockIdx.x) * kThreads + threadIdx.x; i < n; i += stride) {
        const double wv = w[i];
#pragma unroll
        for (int j = 0; j < kMaxDots; ++j) {
            if (j < k) acc[j] += wv * basis.p[j][i];
            else if (j == k) acc[j] += wv * wv;
        }
    }
    __shared__ double red[kMaxDots][kThreads / 32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int j = 0; j < kMaxDots; ++j) {
        const double v = warp_sum(acc[j]);
        if (lane == 0) red[j][warp] = v;
    }
    __syncthreads();
    if (threadIdx.x <= k) {
        double s = 0;
        for (int q = 0; q < kThreads / 32; ++q) s += red[threadIdx.x][q];
        scratch[static_cast<std::size_t>(threadIdx.x) * gridDim.x + blockIdx.x] = s;
    }
    __threadfence();
    __syncthreads();
    __shared__ bool last;
    unsigned* ticket = reinterpret_cast<unsigned*>(scratch + kTicketSlot);
    if (threadIdx.x == 0) last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last) return;
    __threadfence();
    for (int j = warp; j <= k; j += kThreads / 32) {
        double s = 0;
        for (unsigned b = lane; b < gridDim.x; b += 32)
            s += __ldcg(scratch + static_cast<std::size_t>(j) * gridDim.x + b);
        s = warp_sum(s);
        if (lane == 0) results[j] = s;
    }
}

std::mutex g_setup_mutex;
double* g_scratch_address[kMaxDevices] = {};

// Device address of the static scratch on the current device (looked up once).
double* scratch_for_current_device()
{
    int device = 0;
    OWTK_CUDA(cudaGetDevice(&device));
    if (device < 0 || device >= kMaxDevices) fail(OWTK_ERR_INVALID_ARGUMENT, "device index out of range");
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (g_scratch_address[device] == nullptr) {
        double* ptr = nullptr;
        OWTK_CUDA(cudaGetSymbolAddress(reinterpret_cast<void**>(&ptr), g_noalloc_scratch));
        g_scratch_address[device] = ptr;
    }
    return g_scratch_address[device];
}

}  // namespace

void record_error(const std::string& message);   // owtk_last_error() text (capi.cu)

}  // namespace owtk

extern "C" owtk_status owtk_dot_batch_f64_noalloc(const double* w, const double* const* basis, size_t k,
                                                  size_t n, double* results, void* stream)
{
    using namespace owtk;
    try {
        if (w == nullptr || results == nullptr || (k > 0 && basis == nullptr))
            fail(OWTK_ERR_INVALID_ARGUMENT, "null pointer");
        if (k + 1 > static_cast<std::size_t>(kMaxDots))
            fail(OWTK_ERR_INVALID_ARGUMENT,
                 "owtk_dot_batch_f64_noalloc takes at most 31 basis vectors (32 dot products) per call");
        Pointers pack{};
        for (std::size_t j = 0; j < k; ++j) {
            if (basis[j] == nullptr) fail(OWTK_ERR_INVALID_ARGUMENT, "null basis vector");
            pack.p[j] = basis[j];
        }
        double* scratch = scratch_for_current_device();
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        OWTK_CUDA(cudaMemsetAsync(scratch + kTicketSlot, 0, sizeof(unsigned), s));
        std::size_t want = (n + kThreads * 8 - 1) / (kThreads * 8);
        if (want < 1) want = 1;
        if (want > static_cast<std::size_t>(kMaxBlocks)) want = kMaxBlocks;
        k_dot_batch_noalloc<<<static_cast<unsigned>(want), kThreads, 0, s>>>(n, static_cast<int>(k), w, pack,
                                                                              scratch, results);
        OWTK_CUDA(cudaGetLastError());
        return OWTK_OK;
    } catch (const Error& e) {
        record_error(e.message);
        return e.code;
    }
}
