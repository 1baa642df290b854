// devbuf.hpp -- device buffers with byte accounting, CUDA error checks.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <optional>
#include <string>

#include "host.hpp"
#include "../../include/iccg.h"

namespace iccg {

#define CK(call)                                                                                 \
    do {                                                                                         \
        cudaError_t e_ = (call);                                                                 \
        if (e_ != cudaSuccess)                                                                   \
            throw Error(ICCG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_));      \
    } while (0)

struct DevMem {
    void* p = nullptr;
    size_t bytes = 0;
    long long* counter = nullptr;
    DevMem() = default;
    DevMem(const DevMem&) = delete;
    DevMem& operator=(const DevMem&) = delete;
    ~DevMem() { release(); }
    void release()
    {
        if (p) {
            cudaFree(p);
            if (counter) *counter -= (long long)bytes;
        }
        p = nullptr;
        bytes = 0;
    }
};

// Device array of T.  Every allocation carries 16 elements of padding.
// Grow-only: a buffer keeps its allocation when it is cleared or asked for
// fewer elements, and grows with 25 % headroom, so a context that is reused
// for system after system (a serving worker's) rarely calls cudaFree, which
// synchronises the whole device, or cudaMalloc.  The memory goes back when
// the buffer is destroyed (or release() is called).
template <class T>
struct Buf {
    DevMem m;
    size_t n = 0;    // elements in use
    size_t cap = 0;  // elements allocated (plus the padding)
    T* get() const { return (T*)m.p; }
    void alloc(size_t count, long long* counter)
    {
        if (m.p && count <= cap) {
            n = count;
            return;
        }
        const size_t want = m.p ? std::max(count, cap + cap / 4) : count;
        m.release();
        n = cap = 0;
        const size_t bytes = (want + 16) * sizeof(T);
        cudaError_t e = cudaMalloc(&m.p, bytes);
        if (e != cudaSuccess) {
            m.p = nullptr;
            cudaGetLastError();
            throw Error(ICCG_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
        }
        n = count;
        cap = want;
        m.bytes = bytes;
        m.counter = counter;
        *counter += (long long)bytes;
    }
    void upload(const T* h, size_t count, long long* counter, cudaStream_t s)
    {
        alloc(count, counter);
        if (count) CK(cudaMemcpyAsync(m.p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    // clears the contents; the allocation stays for reuse
    void free() { n = 0; }
    void release()
    {
        m.release();
        n = cap = 0;
    }
};

// Set-up tracing: with ICCG_TRACE_SETUP set in the environment, each traced
// phase of a context's set-up prints its wall time to stderr as
// "[iccg setup] <phase> <ms> ms" when it ends.  Phases that end with a
// stream synchronisation include their device work.
inline bool trace_setup()
{
    static const bool on = std::getenv("ICCG_TRACE_SETUP") != nullptr;
    return on;
}

struct SetupPhase {
    const char* name;
    std::chrono::steady_clock::time_point t0;
    explicit SetupPhase(const char* n) : name(n), t0(std::chrono::steady_clock::now()) {}
    SetupPhase(const SetupPhase&) = delete;
    SetupPhase& operator=(const SetupPhase&) = delete;
    ~SetupPhase()
    {
        if (!trace_setup()) return;
        const double ms =
            std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        std::fprintf(stderr, "[iccg setup] %s %.2f ms\n", name, ms);
    }
};

}  // namespace iccg
