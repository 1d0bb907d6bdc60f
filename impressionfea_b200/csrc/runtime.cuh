// runtime.cuh — device memory, error propagation and deterministic reductions for the forging kernels.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>
#include <map>
#include <mutex>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

#include "../../include/ifea_gpu.h"

namespace ifea {

// A failure surfaced through the C ABI as a status code and a message.
struct Failure : std::runtime_error {
    ifea_status status;
    Failure(ifea_status s, const std::string &m) : std::runtime_error(m), status(s) {}
};

struct CudaFailure : Failure {
    CudaFailure(const char *what, cudaError_t e)
        : Failure(IFEA_CUDA_ERROR, std::string(what) + " failed: " + cudaGetErrorString(e)) {}
};

inline void cuda_check(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw CudaFailure(what, e);
}

// Raise a kernel's dynamic shared-memory limit on the current device to at least `bytes`. The limit belongs to the
// kernel, not to a context: a context that needs less must not lower what another live context's launches rely on,
// and contexts are set up from several host threads at once, hence a monotone maximum under a lock.
inline void ensure_dynamic_smem(const void *kernel, size_t bytes)
{
    static std::mutex m;
    static std::map<std::pair<const void *, int>, size_t> done;
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    std::lock_guard<std::mutex> lock(m);
    size_t &cur = done[{kernel, dev}];
    if (bytes <= cur) return;
    cuda_check(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes), "cudaFuncSetAttribute");
    cur = bytes;
}

// Owning device buffer (cudaMalloc / cudaFree; contents undefined after resize). n is the logical length; a
// resize within the allocation keeps it (a remeshed workpiece changes every mesh-sized buffer by a few per cent),
// a larger one reallocates with an eighth of headroom.
template <typename T>
struct DBuf {
    T *p = nullptr;
    size_t n = 0, cap = 0;
    DBuf() = default;
    DBuf(const DBuf &) = delete;
    DBuf &operator=(const DBuf &) = delete;
    ~DBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        n = cap = 0;
    }
    void resize(size_t count)
    {
        if (p && count <= cap) {
            n = count;
            return;
        }
        release();
        if (count) {
            size_t c = count + count / 8;
            cuda_check(cudaMalloc((void **)&p, c * sizeof(T)), "cudaMalloc");
            cap = c;
        }
        n = count;
    }
    void upload(const T *src, size_t count, cudaStream_t s)
    {
        resize(count);
        if (count) cuda_check(cudaMemcpyAsync(p, src, count * sizeof(T), cudaMemcpyHostToDevice, s), "cudaMemcpyAsync H2D");
    }
    void upload(const std::vector<T> &v, cudaStream_t s) { upload(v.data(), v.size(), s); }
    void download(T *dst, size_t count, cudaStream_t s) const
    {
        if (count) cuda_check(cudaMemcpyAsync(dst, p, count * sizeof(T), cudaMemcpyDeviceToHost, s), "cudaMemcpyAsync D2H");
    }
    void zero(cudaStream_t s)
    {
        if (n) cuda_check(cudaMemsetAsync(p, 0, n * sizeof(T), s), "cudaMemsetAsync");
    }
    operator T *() const { return p; }
};

// Exchange two buffers' allocations (pointer, length and capacity).
template <typename T>
inline void swap_buf(DBuf<T> &a, DBuf<T> &b)
{
    std::swap(a.p, b.p);
    std::swap(a.n, b.n);
    std::swap(a.cap, b.cap);
}

// Pinned host staging for scalars read back every iteration.
template <typename T>
struct HostPinned {
    T *p = nullptr;
    size_t n = 0;
    ~HostPinned()
    {
        if (p) cudaFreeHost(p);
    }
    void resize(size_t count)
    {
        if (count <= n) return;
        if (p) cudaFreeHost(p);
        cuda_check(cudaMallocHost((void **)&p, count * sizeof(T)), "cudaMallocHost");
        n = count;
    }
};

constexpr int kReduceBlocks = 296;  // 2 x 148 SMs: fixed, so reductions are run-to-run deterministic
constexpr int kReduceThreads = 256;

// Block-wide sum of K values per thread (warp shuffles, then shared memory); result valid in thread 0.
template <int K>
__device__ __forceinline__ void block_sum(double (&v)[K], double *sh /* >= 32*K */)
{
    for (int k = 0; k < K; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0)
        for (int k = 0; k < K; k++) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
        for (int k = 0; k < K; k++) {
            v[k] = lane < nw ? sh[k * 32 + lane] : 0.0;
            for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_down_sync(0xffffffffu, v[k], o);
        }
    }
}

template <int K>
__device__ __forceinline__ void block_max(double (&v)[K], double *sh)
{
    for (int k = 0; k < K; k++)
        for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_down_sync(0xffffffffu, v[k], o));
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = (blockDim.x + 31) >> 5;
    __syncthreads();
    if (lane == 0)
        for (int k = 0; k < K; k++) sh[k * 32 + warp] = v[k];
    __syncthreads();
    if (warp == 0) {
        for (int k = 0; k < K; k++) {
            v[k] = lane < nw ? sh[k * 32 + lane] : -INFINITY;
            for (int o = 16; o > 0; o >>= 1) v[k] = fmax(v[k], __shfl_down_sync(0xffffffffu, v[k], o));
        }
    }
}

}  // namespace ifea
