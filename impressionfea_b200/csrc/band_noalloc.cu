// band_noalloc.cu — SymmetricBandMatrix.Factorize + Solve on caller-owned device buffers, with no allocation.
//
// Some callers cannot allocate device memory at the moment they need a solve: a host whose GPU memory is owned
// by its own pooling allocator (a PyTorch process, a C# host that reserves the device up front), or a
// latency-critical loop that must not pay for cudaMalloc/cudaFree. This entry point takes the band and the
// right-hand side as device pointers the caller already owns and runs the blocked band kernel (band.cuh) on them:
// its working rows sit in shared memory, or, for a band too wide for that window, in the caller's band itself,
// which is overwritten by L in any case. Its only other working memory, the two status words, sits in a fixed
// file-scope device array (kept until the process exits).
#include <algorithm>
#include <cstring>

#include "band.cuh"
#include "common.cuh"
#include "runtime.cuh"

namespace ifea {

// status: int32 row (4 bytes pad), then the double pivot
static __device__ __align__(16) double g_band_status[2];

namespace {
// Device address of the status words in the calling thread's current device context. Looked up on every call (it
// allocates nothing and costs a driver query), so that a reset device or a new primary context never sees an
// address from an earlier context.
cudaError_t status_address(double **out)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_band_status);
    if (e != cudaSuccess) return e;
    *out = (double *)p;
    return cudaSuccess;
}
}  // namespace

}  // namespace ifea

extern "C" {

// See include/ifea_gpu.h. No cudaMalloc/cudaFree or allocating library call on any path.
ifea_status ifea_band_factor_solve_noalloc(int32_t n, int32_t half_bandwidth, double *d_band, double *d_rhs,
                                           int32_t *bad_row, double *pivot, void *cuda_stream)
{
    if (n <= 0 || half_bandwidth < 0 || !d_band) return IFEA_INPUT_INVALID;
    int b = half_bandwidth < n - 1 ? half_bandwidth : n - 1;
    double *status = nullptr;
    if (ifea::status_address(&status) != cudaSuccess) return IFEA_CUDA_ERROR;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    ifea::band::Plan plan = ifea::band::plan(n, b);
    try {
        ifea::ensure_dynamic_smem(ifea::band::kernel_of(plan), plan.bytes);
    } catch (ifea::Failure &) {
        return IFEA_CUDA_ERROR;
    }
    ifea::band::launch(plan, n, b, d_band, d_rhs, (int32_t *)status, status + 1, st);
    if (cudaGetLastError() != cudaSuccess) return IFEA_CUDA_ERROR;
    struct {
        int32_t row, pad;
        double pivot;
    } out;
    if (cudaMemcpyAsync(&out, status, sizeof out, cudaMemcpyDeviceToHost, st) != cudaSuccess) return IFEA_CUDA_ERROR;
    if (cudaStreamSynchronize(st) != cudaSuccess) return IFEA_CUDA_ERROR;
    if (bad_row) *bad_row = out.row;
    if (pivot) *pivot = out.pivot;
    return out.row >= 0 ? IFEA_NOT_SPD : IFEA_OK;
}

}  // extern "C"
