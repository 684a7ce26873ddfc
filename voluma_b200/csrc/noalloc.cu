// Allocation-free exact sum.
//
// vlm_exact_sum (api.cpp) allocates its per-CTA partial bins with cudaMalloc on every call.
// Some callers cannot allocate device memory at the point where they need a sum: a host
// application whose device memory is owned by its own pool or by a fixed HBM budget (the serving
// loop of this library, or a framework's caching allocator), and latency-critical loops in which
// a cudaMalloc/cudaFree pair would synchronise the device.  This variant keeps its scratch in a
// file-scope __device__ array of fixed size and allocates nothing; the caller passes the input
// values and the output location as device pointers.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "common.h"
#include "exactsum.cuh"
#include "voluma_b200.h"

namespace vlm {
namespace {

constexpr int kNoAllocCtas = 512;      // fixed grid: every CTA owns one partial slot
constexpr int kNoAllocThreads = 256;
constexpr int kNoAllocWarps = kNoAllocThreads / 32;
constexpr int64_t kNoAllocMaxValues = (int64_t(1) << 31) - 1;
// [kNoAllocCtas partial slots of kExactStride words][1 completion counter]  = 299,016 bytes
constexpr size_t kScratchWords = size_t(kNoAllocCtas) * kExactStride + 1;
constexpr size_t kCounterWord = size_t(kNoAllocCtas) * kExactStride;

// Shared by every call on a device; holds the last call's partials until overwritten.
static __device__ __align__(256) long long g_exactScratch[kScratchWords];

constexpr int kMaxDevices = 64;
long long* g_scratchAddr[kMaxDevices] = {};  // device address of g_exactScratch, per device
std::mutex g_setupMutex;

// Grid-stride exact sum; the last CTA to finish adds the partials (int64, exact) and converts.
__global__ void __launch_bounds__(kNoAllocThreads) k_exact_sum_static(const double* __restrict__ v, int64_t n,
                                                                      long long* __restrict__ scratch,
                                                                      double* __restrict__ out) {
    __shared__ long long bins[kNoAllocWarps][kExactBins];
    __shared__ int flags[kNoAllocWarps];
    __shared__ int isLast;
    for (int q = threadIdx.x; q < kNoAllocWarps * kExactBins; q += blockDim.x) (&bins[0][0])[q] = 0;
    if (threadIdx.x < kNoAllocWarps) flags[threadIdx.x] = 0;
    __syncthreads();
    const int warp = threadIdx.x >> 5;
    for (int64_t i = int64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += int64_t(gridDim.x) * blockDim.x)
        exact_add(bins[warp], &flags[warp], v[i]);
    __syncthreads();
    long long* slot = scratch + size_t(blockIdx.x) * kExactStride;
    for (int k = threadIdx.x; k < kExactBins; k += blockDim.x) {
        long long s = 0;
        for (int w = 0; w < kNoAllocWarps; ++w) s += bins[w][k];
        slot[k] = s;
    }
    if (threadIdx.x == 0) {
        int f = 0;
        for (int w = 0; w < kNoAllocWarps; ++w) f |= flags[w];
        slot[kExactBins] = f;
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        isLast = atomicAdd((unsigned long long*)&scratch[kCounterWord], 1ull) == (unsigned long long)(gridDim.x - 1);
    __syncthreads();
    if (!isLast) return;
    __threadfence();
    __shared__ long long tot[kExactStride];
    for (int k = threadIdx.x; k < kExactStride; k += blockDim.x) {
        long long s = 0;
        for (unsigned b = 0; b < gridDim.x; ++b) {
            const long long x = __ldcg(scratch + size_t(b) * kExactStride + k);
            if (k < kExactBins)
                s += x;
            else
                s |= x;
        }
        tot[k] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        *out = exact_value(tot, int(tot[kExactBins]));
        scratch[kCounterWord] = 0;
    }
}

// Device address of the scratch array for the current device.  The first call on a device does
// the look-up (cudaGetSymbolAddress with that device current) and clears the counter.
vlm_status scratchForCurrentDevice(long long** out, std::string* err) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        *err = std::string("cudaGetDevice: ") + cudaGetErrorString(e);
        return VLM_ERR_NO_DEVICE;
    }
    if (dev < 0 || dev >= kMaxDevices) {
        *err = "device index beyond the allocation-free exact sum's table";
        return VLM_ERR_BAD_ARG;
    }
    std::lock_guard<std::mutex> lock(g_setupMutex);
    if (!g_scratchAddr[dev]) {
        long long* p = nullptr;
        e = cudaGetSymbolAddress((void**)&p, g_exactScratch);
        if (e != cudaSuccess) {
            *err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e);
            return VLM_ERR_CUDA;
        }
        g_scratchAddr[dev] = p;  // every call clears the counter on its own stream
    }
    *out = g_scratchAddr[dev];
    return VLM_OK;
}

}  // namespace
}  // namespace vlm

extern "C" {

vlm_status vlm_exact_sum_noalloc(const double* values, int64_t n, double* out, void* stream) {
    using namespace vlm;
    if (!out || (n > 0 && !values) || n < 0) {
        setThreadError("vlm_exact_sum_noalloc: invalid pointer or negative size");
        return VLM_ERR_BAD_ARG;
    }
    if (n > kNoAllocMaxValues) {
        setThreadError("vlm_exact_sum_noalloc: n = " + std::to_string(n) + " exceeds the maximum of " +
                       std::to_string(kNoAllocMaxValues) + " values");
        return VLM_ERR_BAD_ARG;
    }
    long long* scratch = nullptr;
    std::string err;
    const vlm_status st = scratchForCurrentDevice(&scratch, &err);
    if (st != VLM_OK) {
        setThreadError("vlm_exact_sum_noalloc: " + err);
        return st;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(scratch + kCounterWord, 0, sizeof(long long), s);
    if (e == cudaSuccess) {
        const int64_t want = (n + kNoAllocThreads - 1) / kNoAllocThreads;
        const int grid = int(want < 1 ? 1 : (want > kNoAllocCtas ? kNoAllocCtas : want));
        k_exact_sum_static<<<grid, kNoAllocThreads, 0, s>>>(values, n, scratch, out);
        e = cudaGetLastError();
    }
    if (e != cudaSuccess) {
        setThreadError(std::string("vlm_exact_sum_noalloc: ") + cudaGetErrorString(e));
        return VLM_ERR_CUDA;
    }
    return VLM_OK;
}

}  // extern "C"
