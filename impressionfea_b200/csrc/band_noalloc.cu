// band_noalloc.cu — SymmetricBandMatrix.Factorize + Solve on caller-owned device buffers, with no allocation.
//
// Some callers cannot allocate device memory at the moment they need a solve: a host whose GPU memory is owned
// by its own pooling allocator (a PyTorch process, a C# host that reserves the device up front), or a
// latency-critical loop that must not pay for cudaMalloc/cudaFree. This entry point takes the band and the
// right-hand side as device pointers the caller already owns and keeps its only working memory — the window of
// band rows being factorised and two status words — in a fixed file-scope device array, sized once for every
// GPU that loads the library (kept until the process exits).
#include <algorithm>
#include <cstring>

#include "common.cuh"
#include "runtime.cuh"

namespace ifea {

// Scratch: status (int32 row, 4 bytes pad, double pivot) followed by the row window. 2 MiB in total, which admits
// half-bandwidths up to 510 (a window of at least b + 1 rows of b + 1 doubles must fit).
constexpr int64_t kBandScratchDoubles = 262144;
constexpr int64_t kBandScratchHeader = 32;  // doubles reserved for the status words (keeps the window 256-B aligned)
static __device__ __align__(256) double g_band_scratch[kBandScratchDoubles];

// Same arithmetic as k_band_factor_solve (right-looking column sweeps in the reference's subtraction order),
// with the circular row window in the scratch array instead of shared memory.
static __global__ void k_band_factor_solve_scratch(int n, int b, double *__restrict__ a, double *__restrict__ rhs, int W,
                                                   double *scratch)
{
    int32_t *err_row = (int32_t *)scratch;
    double *pivot = scratch + 1;
    double *win = scratch + kBandScratchHeader;
    __shared__ int s_bad;
    const int w = b + 1;
    int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) {
        s_bad = -1;
        *err_row = -1;
        *pivot = 0.0;
    }
    for (int64_t t = tid; t < (int64_t)min(n, W) * w; t += nt) win[t] = a[t];
    __syncthreads();
    int loaded = min(n, W);
    for (int k = 0; k < n; k++) {
        double *rk = win + (size_t)(k % W) * w;
        if (tid == 0) {
            double s = rk[b];
            if (!(s > 0) || isnan(s)) {
                s_bad = k;
                *pivot = s;
            } else {
                rk[b] = sqrt(s);
            }
        }
        __syncthreads();
        if (s_bad >= 0) break;
        double lkk = rk[b];
        int imax = min(n - 1, k + b);
        for (int i = k + 1 + tid; i <= imax; i += nt) win[(size_t)(i % W) * w + (k - i + b)] /= lkk;
        __syncthreads();
        int m = imax - k;
        int pairs = m * (m + 1) / 2;
        for (int t = tid; t < pairs; t += nt) {
            int di = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
            while ((di + 1) * (di + 2) / 2 <= t) di++;
            while (di * (di + 1) / 2 > t) di--;
            int dj = t - di * (di + 1) / 2;
            int i = k + 1 + di, j = k + 1 + dj;
            double lik = win[(size_t)(i % W) * w + (k - i + b)];
            double ljk = win[(size_t)(j % W) * w + (k - j + b)];
            win[(size_t)(i % W) * w + (j - i + b)] -= lik * ljk;
        }
        __syncthreads();
        for (int t = tid; t < w; t += nt) a[(size_t)k * w + t] = rk[t];
        __syncthreads();
        if (loaded < n) {
            double *dst = win + (size_t)(loaded % W) * w;
            for (int t = tid; t < w; t += nt) dst[t] = a[(size_t)loaded * w + t];
            loaded++;
        }
        __syncthreads();
    }
    if (s_bad >= 0) {
        if (tid == 0) *err_row = s_bad;
        return;
    }
    if (!rhs) return;
    __syncthreads();
    for (int k = 0; k < n; k++) {
        double xk = rhs[k] / a[(size_t)k * w + b];
        __syncthreads();
        if (tid == 0) rhs[k] = xk;
        int imax = min(n - 1, k + b);
        for (int i = k + 1 + tid; i <= imax; i += nt) rhs[i] -= a[(size_t)i * w + (k - i + b)] * xk;
        __syncthreads();
    }
    for (int i = n - 1; i >= 0; i--) {
        double xi = rhs[i] / a[(size_t)i * w + b];
        __syncthreads();
        if (tid == 0) rhs[i] = xi;
        for (int k = max(0, i - b) + tid; k < i; k += nt) rhs[k] -= a[(size_t)i * w + (k - i + b)] * xi;
        __syncthreads();
    }
}

namespace {
// Device address of the scratch array in the calling thread's current device context. Looked up on every call
// (it allocates nothing and costs a driver query), so that a reset device or a new primary context never sees
// an address from an earlier context.
cudaError_t scratch_address(double **out)
{
    void *p = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&p, g_band_scratch);
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
    int64_t w = (int64_t)b + 1;
    int64_t capacity = ifea::kBandScratchDoubles - ifea::kBandScratchHeader;
    if (w * w > capacity) return IFEA_INPUT_INVALID;  // half-bandwidth above 510: the row window does not fit
    int W = (int)std::min<int64_t>((int64_t)n, capacity / w);
    double *scratch = nullptr;
    if (ifea::scratch_address(&scratch) != cudaSuccess) return IFEA_CUDA_ERROR;
    cudaStream_t st = (cudaStream_t)cuda_stream;
    ifea::k_band_factor_solve_scratch<<<1, 1024, 0, st>>>(n, b, d_band, d_rhs, W, scratch);
    if (cudaGetLastError() != cudaSuccess) return IFEA_CUDA_ERROR;
    struct {
        int32_t row, pad;
        double pivot;
    } status;
    if (cudaMemcpyAsync(&status, scratch, sizeof status, cudaMemcpyDeviceToHost, st) != cudaSuccess) return IFEA_CUDA_ERROR;
    if (cudaStreamSynchronize(st) != cudaSuccess) return IFEA_CUDA_ERROR;
    if (bad_row) *bad_row = status.row;
    if (pivot) *pivot = status.pivot;
    return status.row >= 0 ? IFEA_NOT_SPD : IFEA_OK;
}

}  // extern "C"
