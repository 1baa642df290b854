// noalloc.cu -- iccg_dot_dev_noalloc: the double-double inner product of
// iccg_dot_dev with its scratch in a fixed static device array, for callers
// that may not allocate device memory.
//
// Scratch layout (one copy per device, in the library's device image):
//   [0, kSlots * 16)            per-CTA double-double partial sums
//   [kTicketOffset, +4)         arrival counter of the last-CTA reduction;
//                               it must read zero when a call starts, is set
//                               to zero by the set-up of the first call on a
//                               device, and the last CTA of every call puts
//                               it back to zero.
//
// Each CTA sums a fixed chunk of kChunk consecutive elements, so the
// partial sums, their order and the result depend only on n (not on the
// device or its occupancy).
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/iccg.h"
#include "dd.cuh"

namespace iccg {

extern thread_local std::string g_host_err;  // host_capi.cpp

namespace {

constexpr int kThreads = 256;
constexpr int kPerThread = 16;
constexpr int kChunk = kThreads * kPerThread;          // elements per CTA
constexpr int kSlots = ICCG_NOALLOC_MAX_N / kChunk;    // CTAs of the largest call
static_assert(ICCG_NOALLOC_MAX_N % kChunk == 0, "limit must be a whole number of chunks");
constexpr size_t kTicketOffset = sizeof(dd) * (size_t)kSlots;
constexpr size_t kScratchBytes = kTicketOffset + 256;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

__global__ void __launch_bounds__(kThreads) k_dot_noalloc(int n, const double* __restrict__ a,
                                                         const double* __restrict__ b, double* __restrict__ out,
                                                         unsigned char* scratch)
{
    dd* partials = reinterpret_cast<dd*>(scratch);
    unsigned int* ticket = reinterpret_cast<unsigned int*>(scratch + kTicketOffset);
    __shared__ dd sm[kThreads / 32];
    __shared__ bool last;

    acc2 s = {0.0, 0.0};
    const long long base = (long long)blockIdx.x * kChunk + threadIdx.x;
#pragma unroll
    for (int k = 0; k < kPerThread; ++k) {
        const long long i = base + (long long)k * kThreads;
        if (i < n) acc2_fma(s, a[i], b[i]);
    }
    dd v[1] = {acc2_dd(s)}, tot[1];
    block_reduce_dd<1>(v, sm, tot);
    if (threadIdx.x == 0) {
        partials[blockIdx.x] = tot[0];
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        last = (t == gridDim.x - 1u);
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    dd acc = {0.0, 0.0};
    for (int q = threadIdx.x; q < (int)gridDim.x; q += kThreads) {
        dd p;
        p.hi = __ldcg(&partials[q].hi);
        p.lo = __ldcg(&partials[q].lo);
        acc = dd_add(acc, p);
    }
    v[0] = acc;
    block_reduce_dd<1>(v, sm, tot);
    if (threadIdx.x == 0) {
        *out = dd_round(tot[0]);
        *ticket = 0u;  // every CTA has arrived: ready for the next call
    }
}

std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

int fail(int code, const std::string& msg)
{
    g_host_err = "iccg_dot_dev_noalloc: " + msg;
    return code;
}

}  // namespace
}  // namespace iccg

extern "C" int iccg_dot_dev_noalloc(int n, const double* a, const double* b, double* out, void* stream)
{
    using namespace iccg;
    if (n < 0) return fail(ICCG_ERR_ARG, "n = " + std::to_string(n) + " is negative");
    if (n > ICCG_NOALLOC_MAX_N)
        return fail(ICCG_ERR_ARG, "n = " + std::to_string(n) + " exceeds the static scratch limit ICCG_NOALLOC_MAX_N = " +
                                      std::to_string(ICCG_NOALLOC_MAX_N));
    if (!out || (n > 0 && (!a || !b))) return fail(ICCG_ERR_ARG, "null pointer argument");
    cudaStream_t st = static_cast<cudaStream_t>(stream);

    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return fail(ICCG_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
    if (dev < 0 || dev >= kMaxDevices) return fail(ICCG_ERR_ARG, "device ordinal " + std::to_string(dev) + " out of range");

    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_setup_mu);
        scratch = g_scratch_ptr[dev];
        if (!scratch) {
            // set-up, once per device: the scratch address in this device's
            // image of the library, and the arrival counter cleared
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_scratch);
            if (e != cudaSuccess)
                return fail(ICCG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
            e = cudaMemsetAsync(static_cast<unsigned char*>(p) + kTicketOffset, 0, sizeof(unsigned int), st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e != cudaSuccess) return fail(ICCG_ERR_CUDA, std::string("scratch set-up: ") + cudaGetErrorString(e));
            scratch = static_cast<unsigned char*>(p);
            g_scratch_ptr[dev] = scratch;
        }
    }

    const int grid = n == 0 ? 1 : (int)(((long long)n + kChunk - 1) / kChunk);
    k_dot_noalloc<<<grid, kThreads, 0, st>>>(n, a, b, out, scratch);
    e = cudaGetLastError();
    if (e != cudaSuccess) return fail(ICCG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    return ICCG_OK;
}
