// devbuf.hpp -- device buffers with byte accounting, CUDA error checks.
#pragma once
#include <cuda_runtime.h>

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
template <class T>
struct Buf {
    DevMem m;
    size_t n = 0;
    T* get() const { return (T*)m.p; }
    void alloc(size_t count, long long* counter)
    {
        if (count == n && m.p) return;
        m.release();
        n = count;
        const size_t bytes = (count + 16) * sizeof(T);
        cudaError_t e = cudaMalloc(&m.p, bytes);
        if (e != cudaSuccess) {
            m.p = nullptr;
            n = 0;
            cudaGetLastError();
            throw Error(ICCG_ERR_NOMEM, "cudaMalloc of " + std::to_string(bytes) + " bytes failed");
        }
        m.bytes = bytes;
        m.counter = counter;
        *counter += (long long)bytes;
    }
    void upload(const T* h, size_t count, long long* counter, cudaStream_t s)
    {
        alloc(count, counter);
        if (count) CK(cudaMemcpyAsync(m.p, h, count * sizeof(T), cudaMemcpyHostToDevice, s));
    }
    void free()
    {
        m.release();
        n = 0;
    }
};

}  // namespace iccg
