// mlp.cu — the learned warm start's network on the tensor cores: a per-node MLP 16 -> 128 -> 128 -> 128 -> 3 with
// GELU, BF16 weights and activations, FP32 accumulation, trained by Adam on FP32 master weights.
//
// Every layer product is one kernel, k_gemm: C (128-row tiles) = A B^T with A [M][K] and B [N][K] in BF16
// (K contiguous), staged by cp.async into shared memory as K-major core matrices without swizzle (8 rows x 16 B,
// one 16-byte K chunk of all rows after another), two stages deep, multiplied by tcgen05.mma kind::f16 issued by
// one thread into a tensor-memory accumulator, and read back by tcgen05.ld for a fused epilogue:
//   forward hidden layer  z = acc + b, h = GELU(z)        (z kept in FP32 for the backward pass, h in BF16 both
//                                                          [row][feature] and transposed)
//   backward hidden layer dz = acc * GELU'(z)             (BF16, both layouts)
//   weight gradient       partial sums over a K slice     (FP32; K = the batch, split over CTAs, summed in order)
// The 3-wide output layer, the loss and its gradient, the bias gradients and Adam are small SIMT kernels.
// Every sum runs in a fixed order, so training is bit-reproducible run to run.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>
#include <random>

#include "warmstart.h"

namespace ifea {
namespace wsm {

constexpr int BM = 128, BK = 64, SPLIT_K = 512;
typedef __nv_bfloat16 bf16;

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major, no swizzle: core matrices of 8 rows x 16 B (rows 16 B apart, 8-row groups 128 B apart: stride
// offset), the two 16-byte K chunks of one MMA a whole chunk of all rows apart (leading offset); version 1
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t chunk_bytes)
{
    return (uint64_t)((addr >> 4) & 0x3FFF) | ((uint64_t)((chunk_bytes >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((128 >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}
// instruction descriptor, kind::f16: D f32 (bits 4-5 = 1), A and B bf16 (bits 7-9, 10-12 = 1), both K-major,
// N >> 3 at bit 17, M >> 4 at bit 24
template <int N>
__host__ __device__ constexpr uint32_t idesc() { return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(BM >> 4) << 24); }

__device__ __forceinline__ void mma_bf16(uint32_t tmem, uint64_t da, uint64_t db, uint32_t id, uint32_t acc)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(tmem),
        "l"(da), "l"(db), "r"(id), "r"(acc), "r"(0), "r"(0), "r"(0), "r"(0));
}

// bounded wait on an mbarrier phase: false if it gave up (an MMA of a few microseconds ends far sooner)
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
    for (uint32_t it = 0; it < (1u << 20); it++) {
        uint32_t done;
        asm volatile(
            "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

__device__ __forceinline__ void cp_async16(uint32_t dst, const void *src, int bytes)
{
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(dst), "l"(src), "r"(bytes) : "memory");
}

#define WSM_TMEM_LD16(taddr, r)                                                                                      \
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, "  \
                 "[%16];"                                                                                            \
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),   \
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]),           \
                   "=r"(r[15])                                                                                       \
                 : "r"(taddr))

__device__ __forceinline__ float gelu(float z) { return 0.5f * z * (1.0f + erff(z * 0.70710678118654752f)); }
__device__ __forceinline__ float gelu_d(float z)
{
    return 0.5f * (1.0f + erff(z * 0.70710678118654752f)) + z * 0.39894228040143268f * expf(-0.5f * z * z);
}

enum { EPI_FWD = 0, EPI_BWD = 1, EPI_PART = 2 };

struct Gemm {
    const bf16 *A;
    int64_t lda;  // [M][K]
    const bf16 *B;
    int64_t ldb;  // [N][K]
    int M, K, kper;
    const float *bias;  // EPI_FWD
    const float *zin;   // EPI_BWD: pre-activations [M][N]
    float *zout;        // EPI_FWD: pre-activations out [M][N] (or null)
    bf16 *h;            // [M][N] (row stride N)
    bf16 *ht;           // [N][M] (row stride ldht) or null
    int64_t ldht;
    float *part;  // EPI_PART: [split][M][N]
    int *err;
};

template <int N>
constexpr int gemm_smem() { return 2 * (BM * BK * 2) + 2 * (N * BK * 2) + 64; }

template <int N, int EPI>
__global__ void __launch_bounds__(128) k_gemm(Gemm g)
{
    extern __shared__ __align__(1024) unsigned char sm[];
    constexpr int A_STAGE = BM * BK * 2, B_STAGE = N * BK * 2;
    constexpr uint32_t CHUNK_A = BM * 16, CHUNK_B = N * 16;
    constexpr int TCOLS = N < 32 ? 32 : N;
    uint64_t *bar = (uint64_t *)(sm + 2 * A_STAGE + 2 * B_STAGE);
    uint32_t *tslot = (uint32_t *)(bar + 2);
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int m0 = blockIdx.x * BM, split = blockIdx.y;
    const int k0 = split * g.kper, k1 = min(g.K, k0 + g.kper);
    const uint32_t sbase = smem_u32(sm);
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tslot)), "r"(TCOLS));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
    }
    if (tid == 0) {
        for (int s = 0; s < 2; s++) asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar + s)), "r"(1));
        asm volatile("fence.mbarrier_init.release.cluster;" ::);
    }
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::);
    const uint32_t tmem = *tslot;
    const int nblk = (k1 - k0 + BK - 1) / BK;
    uint32_t ph[2] = {0, 0};
    bool ok = true;
    for (int b = 0; b < nblk; b++) {
        const int s = b & 1;
        if (b >= 2) {
            ok = mbar_wait(smem_u32(bar + s), ph[s]);
            ph[s] ^= 1;
            if (__syncthreads_or(!ok)) break;
        }
        const int kb = k0 + b * BK, kn = min(BK, k1 - kb);
        const uint32_t sa = sbase + s * A_STAGE, sb = sbase + 2 * A_STAGE + s * B_STAGE;
        for (int q = tid; q < BM * 8; q += 128) {
            int r = q >> 3, c = q & 7, row = m0 + r;
            bool v = row < g.M && 8 * c < kn;
            const void *src = v ? (const void *)(g.A + (int64_t)row * g.lda + kb + 8 * c) : (const void *)g.A;
            cp_async16(sa + (uint32_t)(c * BM + r) * 16, src, v ? 16 : 0);
        }
        for (int q = tid; q < N * 8; q += 128) {
            int r = q >> 3, c = q & 7;
            bool v = 8 * c < kn;
            const void *src = v ? (const void *)(g.B + (int64_t)r * g.ldb + kb + 8 * c) : (const void *)g.B;
            cp_async16(sb + (uint32_t)(c * N + r) * 16, src, v ? 16 : 0);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (tid == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;" ::);
            for (int j = 0; j < kn / 16; j++)
                mma_bf16(tmem, sdesc(sa + j * 2 * CHUNK_A, CHUNK_A), sdesc(sb + j * 2 * CHUNK_B, CHUNK_B), idesc<N>(),
                         (b > 0 || j > 0) ? 1u : 0u);
            asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar + s)));
        }
    }
    if (ok && nblk > 0) {
        const int s = (nblk - 1) & 1;
        ok = mbar_wait(smem_u32(bar + s), ph[s]);
    }
    if (__syncthreads_or(!ok)) {
        if (tid == 0) atomicExch(g.err, 1);
    } else {
        asm volatile("tcgen05.fence::after_thread_sync;" ::);
        const int r = 32 * warp + lane, row = m0 + r;
#pragma unroll 1
        for (int c0 = 0; c0 < N; c0 += 16) {
            uint32_t v[16];
            WSM_TMEM_LD16(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c0, v);
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            if (row >= g.M) continue;
            if (EPI == EPI_PART) {
                float *dst = g.part + ((int64_t)split * g.M + row) * N + c0;
#pragma unroll
                for (int j = 0; j < 16; j++) dst[j] = __uint_as_float(v[j]);
                continue;
            }
            float o[16];
#pragma unroll
            for (int j = 0; j < 16; j++) {
                float a = __uint_as_float(v[j]);
                if (EPI == EPI_FWD) {
                    float z = a + g.bias[c0 + j];
                    if (g.zout) g.zout[(int64_t)row * N + c0 + j] = z;
                    o[j] = gelu(z);
                } else {
                    o[j] = a * gelu_d(g.zin[(int64_t)row * N + c0 + j]);
                }
            }
            __align__(16) bf16 hb[16];
#pragma unroll
            for (int j = 0; j < 16; j++) hb[j] = __float2bfloat16_rn(o[j]);
            uint4 *dst = (uint4 *)(g.h + (int64_t)row * N + c0);
            dst[0] = ((const uint4 *)hb)[0];
            dst[1] = ((const uint4 *)hb)[1];
            if (g.ht)
#pragma unroll
                for (int j = 0; j < 16; j++) g.ht[(int64_t)(c0 + j) * g.ldht + row] = hb[j];
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::);
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TCOLS));
}

// ------------------------------------------------------------------ SIMT parts

// rows of normalised inputs in BF16, [M][16] and transposed [16][ldt]; rows past n are zero
__global__ void k_pack_inputs(const float *__restrict__ x, const int32_t *__restrict__ idx, int64_t n, int M,
                              const float *__restrict__ norm, bf16 *__restrict__ xb, bf16 *__restrict__ xbt, int ldt,
                              const float *__restrict__ t, float *__restrict__ tb)
{
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        int64_t src = idx ? (int64_t)idx[r] : (int64_t)r;
        bool v = src < n;
        __align__(16) bf16 hb[NIN];
        for (int c = 0; c < NIN; c++) {
            float a = v ? (x[src * NIN + c] - norm[c]) / norm[NIN + c] : 0.0f;
            hb[c] = __float2bfloat16_rn(a);
            if (xbt) xbt[(int64_t)c * ldt + r] = hb[c];
        }
        uint4 *d = (uint4 *)(xb + (int64_t)r * NIN);
        d[0] = ((const uint4 *)hb)[0];
        d[1] = ((const uint4 *)hb)[1];
        if (tb)
            for (int o = 0; o < NOUT; o++)
                tb[(int64_t)r * NOUT + o] = v ? (t[src * NOUT + o] - norm[2 * NIN + o]) / norm[2 * NIN + NOUT + o] : 0.0f;
    }
}

// output layer y = W4 h3 + b4 (FP32 over the BF16 activations); denorm != 0 maps back to raw targets
__global__ void k_head_fwd(const bf16 *__restrict__ h3, int M, const float *__restrict__ par, const float *__restrict__ norm,
                           int denorm, float *__restrict__ y)
{
    __shared__ float w[NOUT * HID + NOUT];
    for (int i = threadIdx.x; i < NOUT * HID + NOUT; i += blockDim.x) w[i] = par[OFF_W4 + i];
    __syncthreads();
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < M; r += gridDim.x * blockDim.x) {
        float acc[NOUT];
        for (int o = 0; o < NOUT; o++) acc[o] = w[NOUT * HID + o];
        const uint4 *row = (const uint4 *)(h3 + (int64_t)r * HID);
        for (int q = 0; q < HID / 8; q++) {
            uint4 u = row[q];
            const bf16 *hv = (const bf16 *)&u;
            for (int j = 0; j < 8; j++) {
                float hf = __bfloat162float(hv[j]);
                for (int o = 0; o < NOUT; o++) acc[o] += w[o * HID + 8 * q + j] * hf;
            }
        }
        for (int o = 0; o < NOUT; o++)
            y[(int64_t)r * NOUT + o] = denorm ? norm[2 * NIN + o] + norm[2 * NIN + NOUT + o] * acc[o] : acc[o];
    }
}

// loss and its gradient at the output, back through the output layer: dz3 = (dy W4) * GELU'(z3); per-block
// partial sums of dW4, db4 and the loss (rows past n contribute nothing)
__global__ void __launch_bounds__(128) k_head_bwd(const bf16 *__restrict__ h3, const float *__restrict__ z3,
                                                  const float *__restrict__ y, const float *__restrict__ t, int n, int M,
                                                  const float *__restrict__ par, bf16 *__restrict__ dz3,
                                                  bf16 *__restrict__ dz3t, float *__restrict__ hpart)
{
    __shared__ float w[NOUT * HID];
    __shared__ float dys[128][NOUT];
    __shared__ float red[128];
    for (int i = threadIdx.x; i < NOUT * HID; i += blockDim.x) w[i] = par[OFF_W4 + i];
    int r = blockIdx.x * 128 + threadIdx.x;
    float dy[NOUT], l = 0;
    const float scale = 2.0f / (float)(n * NOUT);
    for (int o = 0; o < NOUT; o++) {
        float e = r < n ? y[(int64_t)r * NOUT + o] - t[(int64_t)r * NOUT + o] : 0.0f;
        l += e * e;
        dy[o] = scale * e;
        dys[threadIdx.x][o] = dy[o];
    }
    __syncthreads();
    if (r < M) {
        for (int c0 = 0; c0 < HID; c0 += 8) {
            __align__(16) bf16 hb[8];
            for (int j = 0; j < 8; j++) {
                int i = c0 + j;
                float dh = 0;
                for (int o = 0; o < NOUT; o++) dh += dy[o] * w[o * HID + i];
                hb[j] = __float2bfloat16_rn(dh * gelu_d(z3[(int64_t)r * HID + i]));
                dz3t[(int64_t)i * M + r] = hb[j];
            }
            *(uint4 *)(dz3 + (int64_t)r * HID + c0) = *(const uint4 *)hb;
        }
    }
    // dW4[o][i] = sum over this block's rows of dy[o] h3[row][i]: thread i owns column i
    float* out = hpart + (int64_t)blockIdx.x * (NOUT * HID + NOUT + 1);
    {
        int i = threadIdx.x;
        float acc[NOUT] = {0, 0, 0};
        for (int k = 0; k < 128; k++) {
            int rr = blockIdx.x * 128 + k;
            if (rr >= M) break;
            float hv = __bfloat162float(h3[(int64_t)rr * HID + i]);
            for (int o = 0; o < NOUT; o++) acc[o] += dys[k][o] * hv;
        }
        for (int o = 0; o < NOUT; o++) out[o * HID + i] = acc[o];
    }
    if (threadIdx.x < NOUT) {
        float acc = 0;
        for (int k = 0; k < 128; k++) acc += dys[k][threadIdx.x];
        out[NOUT * HID + threadIdx.x] = acc;
    }
    red[threadIdx.x] = l;
    __syncthreads();
    for (int s = 64; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[NOUT * HID + NOUT] = red[0];
}

// out[i] = sum over parts j (in order) of p[j * count + i]
__global__ void k_sum_parts(const float *__restrict__ p, int nparts, int count, int stride, float *__restrict__ out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        float acc = 0;
        for (int j = 0; j < nparts; j++) acc += p[(int64_t)j * stride + i];
        out[i] = acc;
    }
}

// bias gradients: row f of the transposed layer gradient [HID][M] summed (block per feature, fixed order)
__global__ void k_row_sums(const bf16 *__restrict__ dzt, int M, float *__restrict__ out)
{
    __shared__ float red[256];
    const bf16 *row = dzt + (int64_t)blockIdx.x * M;
    float acc = 0;
    for (int i = threadIdx.x; i < M; i += blockDim.x) acc += __bfloat162float(row[i]);
    red[threadIdx.x] = acc;
    __syncthreads();
    for (int s = 128; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[threadIdx.x] += red[threadIdx.x + s];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[blockIdx.x] = red[0];
}

__global__ void k_adam(float *__restrict__ w, const float *__restrict__ g, float *__restrict__ m, float *__restrict__ v,
                       int n, float lr, float bc1, float bc2)
{
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float gi = g[i];
        float mi = b1 * m[i] + (1 - b1) * gi, vi = b2 * v[i] + (1 - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
    }
}

// BF16 copies of the hidden layers' weights: W [out][in] for the forward products, W^T [in][out] for the backward
__global__ void k_publish(const float *__restrict__ par, bf16 *w1, bf16 *w2, bf16 *w3, bf16 *w2t, bf16 *w3t)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < HID * HID; i += gridDim.x * blockDim.x) {
        int o = i / HID, k = i % HID;
        if (i < HID * NIN) w1[i] = __float2bfloat16_rn(par[OFF_W1 + i]);
        bf16 a = __float2bfloat16_rn(par[OFF_W2 + i]), b = __float2bfloat16_rn(par[OFF_W3 + i]);
        w2[i] = a;
        w3[i] = b;
        w2t[k * HID + o] = a;
        w3t[k * HID + o] = b;
    }
}

// column sums and sums of squares of an [n][w] FP32 array, per block (double, fixed order)
__global__ void k_moments(const float *__restrict__ x, int64_t n, int w, double *__restrict__ part)
{
    __shared__ double red[2][256];
    for (int c = 0; c < w; c++) {
        double s = 0, q = 0;
        for (int64_t r = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; r < n; r += (int64_t)gridDim.x * blockDim.x) {
            double a = x[r * w + c];
            s += a;
            q += a * a;
        }
        red[0][threadIdx.x] = s;
        red[1][threadIdx.x] = q;
        __syncthreads();
        for (int k = 128; k > 0; k >>= 1) {
            if (threadIdx.x < k) {
                red[0][threadIdx.x] += red[0][threadIdx.x + k];
                red[1][threadIdx.x] += red[1][threadIdx.x + k];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            part[((int64_t)blockIdx.x * w + c) * 2] = red[0][0];
            part[((int64_t)blockIdx.x * w + c) * 2 + 1] = red[1][0];
        }
        __syncthreads();
    }
}

__global__ void k_read_err(int *err, int *out) { *out = *err; *err = 0; }

template <int N, int EPI>
void launch_gemm(const Gemm &g, int splits, cudaStream_t s)
{
    ensure_dynamic_smem((const void *)k_gemm<N, EPI>, gemm_smem<N>());
    dim3 grid((g.M + BM - 1) / BM, splits);
    k_gemm<N, EPI><<<grid, 128, gemm_smem<N>(), s>>>(g);
}

}  // namespace wsm

using namespace wsm;

WarmStartNet::WarmStartNet(uint64_t seed)
{
    cuda_check(cudaStreamCreateWithFlags(&st_, cudaStreamNonBlocking), "cudaStreamCreate");
    par_.resize(NPAR); grad_.resize(NPAR); m_.resize(NPAR); v_.resize(NPAR); norm_.resize(NNORM);
    w1_.resize(HID * NIN); w2_.resize(HID * HID); w3_.resize(HID * HID); w2t_.resize(HID * HID); w3t_.resize(HID * HID);
    loss_.resize(4);
    loss_.zero(st_);  // slots 2-3 are the tensor-core error flag and its copy: they must start at zero
    hloss_.resize(4);
    // He-uniform initial weights, zero biases (seeded)
    std::vector<float> p(NPAR, 0.0f);
    std::mt19937_64 rng(seed);
    auto fill = [&](int off, int fan_in, int count) {
        float a = std::sqrt(6.0f / (float)fan_in);
        std::uniform_real_distribution<float> u(-a, a);
        for (int i = 0; i < count; i++) p[off + i] = u(rng);
    };
    fill(OFF_W1, NIN, HID * NIN);
    fill(OFF_W2, HID, HID * HID);
    fill(OFF_W3, HID, HID * HID);
    fill(OFF_W4, HID, NOUT * HID);
    for (int i = 0; i < NOUT * HID; i++) p[OFF_W4 + i] *= 0.1f;  // a small output layer: the first guess stays near zero
    set_params(p.data());
    norm_host_.assign(NNORM, 0.0f);
    for (int c = 0; c < NIN; c++) norm_host_[NIN + c] = 1.0f;
    for (int o = 0; o < NOUT; o++) norm_host_[2 * NIN + NOUT + o] = 1.0f;
    set_norm(norm_host_.data());
}

WarmStartNet::~WarmStartNet()
{
    if (st_) {
        cudaStreamSynchronize(st_);
        cudaStreamDestroy(st_);
    }
}

void WarmStartNet::get_params(float *host) const
{
    cuda_check(cudaMemcpyAsync(host, par_.p, sizeof(float) * NPAR, cudaMemcpyDeviceToHost, st_), "D2H");
    cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
}

void WarmStartNet::set_params(const float *host)
{
    cuda_check(cudaMemcpyAsync(par_.p, host, sizeof(float) * NPAR, cudaMemcpyHostToDevice, st_), "H2D");
    m_.zero(st_);
    v_.zero(st_);
    adam_t_ = 0;
    publish(st_);
    cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
}

void WarmStartNet::get_norm(float *host) const { std::memcpy(host, norm_host_.data(), sizeof(float) * NNORM); }

void WarmStartNet::set_norm(const float *host)
{
    norm_host_.assign(host, host + NNORM);
    cuda_check(cudaMemcpyAsync(norm_.p, norm_host_.data(), sizeof(float) * NNORM, cudaMemcpyHostToDevice, st_), "H2D");
    cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
}

void WarmStartNet::publish(cudaStream_t s)
{
    k_publish<<<64, 256, 0, s>>>(par_.p, w1_.p, w2_.p, w3_.p, w2t_.p, w3t_.p);
}

void WarmStartNet::add_samples_device(const float *d_x, const float *d_t, int64_t n, cudaStream_t s)
{
    if (n <= 0) return;
    if (count_ + n > cap_) {
        int64_t cap = std::max<int64_t>(2 * cap_, std::max<int64_t>(count_ + n, 1 << 16));
        DBuf<float> nx, nt;
        nx.resize((size_t)cap * NIN);
        nt.resize((size_t)cap * NOUT);
        if (count_) {
            cuda_check(cudaMemcpyAsync(nx.p, dx_.p, sizeof(float) * count_ * NIN, cudaMemcpyDeviceToDevice, s), "D2D");
            cuda_check(cudaMemcpyAsync(nt.p, dt_.p, sizeof(float) * count_ * NOUT, cudaMemcpyDeviceToDevice, s), "D2D");
        }
        cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
        swap_buf(dx_, nx);
        swap_buf(dt_, nt);
        cap_ = cap;
    }
    cuda_check(cudaMemcpyAsync(dx_.p + count_ * NIN, d_x, sizeof(float) * n * NIN, cudaMemcpyDeviceToDevice, s), "D2D");
    cuda_check(cudaMemcpyAsync(dt_.p + count_ * NOUT, d_t, sizeof(float) * n * NOUT, cudaMemcpyDeviceToDevice, s), "D2D");
    count_ += n;
}

void WarmStartNet::add_samples_host(const float *x, const float *t, int64_t n)
{
    DBuf<float> a, b;
    a.upload(x, (size_t)n * NIN, st_);
    b.upload(t, (size_t)n * NOUT, st_);
    add_samples_device(a.p, b.p, n, st_);
    cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
}

void WarmStartNet::fit_normalisation()
{
    if (count_ < 2) throw Failure(IFEA_BAD_STATE, "The warm-start network has fewer than two training samples.");
    const int blocks = 148;
    DBuf<double> part;
    part.resize((size_t)blocks * NIN * 2);
    std::vector<double> h((size_t)blocks * NIN * 2);
    for (int pass = 0; pass < 2; pass++) {
        int w = pass == 0 ? NIN : NOUT;
        const float *src = pass == 0 ? dx_.p : dt_.p;
        k_moments<<<blocks, 256, 0, st_>>>(src, count_, w, part.p);
        cuda_check(cudaMemcpyAsync(h.data(), part.p, sizeof(double) * blocks * w * 2, cudaMemcpyDeviceToHost, st_), "D2H");
        cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
        for (int c = 0; c < w; c++) {
            double s = 0, q = 0;
            for (int b = 0; b < blocks; b++) {
                s += h[((size_t)b * w + c) * 2];
                q += h[((size_t)b * w + c) * 2 + 1];
            }
            double mean = s / count_, var = std::max(0.0, q / count_ - mean * mean);
            double sd = std::sqrt(var);
            int off = pass == 0 ? 0 : 2 * NIN;
            norm_host_[off + c] = (float)mean;
            norm_host_[off + w + c] = (float)(sd > 1e-6 ? sd : 1.0);
        }
    }
    set_norm(norm_host_.data());
}

void WarmStartNet::ensure_batch(int B)
{
    if (B <= bcap_) return;
    size_t b = (size_t)B;
    xb_.resize(b * NIN); xbt_.resize(b * NIN);
    h1_.resize(b * HID); h2_.resize(b * HID); h3_.resize(b * HID); h1t_.resize(b * HID); h2t_.resize(b * HID);
    dz1_.resize(b * HID); dz2_.resize(b * HID); dz3_.resize(b * HID); dz1t_.resize(b * HID); dz2t_.resize(b * HID);
    dz3t_.resize(b * HID);
    tb_.resize(b * NOUT); z1_.resize(b * HID); z2_.resize(b * HID); z3_.resize(b * HID); y_.resize(b * NOUT);
    int splits = (B + SPLIT_K - 1) / SPLIT_K;
    part_.resize((size_t)splits * HID * HID);
    hpart_.resize((size_t)((B + 127) / 128) * (NOUT * HID + NOUT + 1));
    idx_.resize(b);
    bcap_ = B;
}

// forward over the packed batch xb_ (B rows): z and both layouts of h kept for the backward pass when training
void WarmStartNet::forward(int B, bool train, cudaStream_t s)
{
    int *err = (int *)loss_.p + 2;
    Gemm g{};
    g.M = B; g.kper = 1 << 30; g.err = err; g.ldht = B;
    g.A = xb_.p; g.lda = NIN; g.B = w1_.p; g.ldb = NIN; g.K = NIN; g.bias = par_.p + OFF_B1;
    g.zout = train ? z1_.p : nullptr; g.h = h1_.p; g.ht = train ? h1t_.p : nullptr;
    launch_gemm<HID, EPI_FWD>(g, 1, s);
    g.A = h1_.p; g.lda = HID; g.B = w2_.p; g.ldb = HID; g.K = HID; g.bias = par_.p + OFF_B2;
    g.zout = train ? z2_.p : nullptr; g.h = h2_.p; g.ht = train ? h2t_.p : nullptr;
    launch_gemm<HID, EPI_FWD>(g, 1, s);
    g.A = h2_.p; g.B = w3_.p; g.bias = par_.p + OFF_B3;
    g.zout = train ? z3_.p : nullptr; g.h = h3_.p; g.ht = nullptr;
    launch_gemm<HID, EPI_FWD>(g, 1, s);
}

// backward over the batch (n valid rows of B) after forward(B, true) and k_head_fwd into y_; fills grad_ and,
// with apply, takes one Adam step. Returns the batch's mean squared error (reads it back).
float WarmStartNet::backward_and_step(int B, bool apply, float lr, cudaStream_t s)
{
    int *err = (int *)loss_.p + 2;
    int nblk = (B + 127) / 128;
    k_head_bwd<<<nblk, 128, 0, s>>>(h3_.p, z3_.p, y_.p, tb_.p, B, B, par_.p, dz3_.p, dz3t_.p, hpart_.p);
    int hstride = NOUT * HID + NOUT + 1;
    k_sum_parts<<<4, 128, 0, s>>>(hpart_.p, nblk, NOUT * HID + NOUT, hstride, grad_.p + OFF_W4);  // dW4, db4
    Gemm g{};
    g.M = B; g.kper = 1 << 30; g.err = err; g.ldht = B;
    // dz2 = (dz3 W3) * GELU'(z2), dz1 = (dz2 W2) * GELU'(z1)
    g.A = dz3_.p; g.lda = HID; g.B = w3t_.p; g.ldb = HID; g.K = HID; g.zin = z2_.p; g.h = dz2_.p; g.ht = dz2t_.p;
    launch_gemm<HID, EPI_BWD>(g, 1, s);
    g.A = dz2_.p; g.B = w2t_.p; g.zin = z1_.p; g.h = dz1_.p; g.ht = dz1t_.p;
    launch_gemm<HID, EPI_BWD>(g, 1, s);
    // weight gradients: dW_l = dz_l^T h_(l-1), K = the batch split over CTAs
    int splits = (B + SPLIT_K - 1) / SPLIT_K;
    Gemm w{};
    w.M = HID; w.K = B; w.kper = SPLIT_K; w.err = err; w.part = part_.p;
    w.A = dz3t_.p; w.lda = B; w.B = h2t_.p; w.ldb = B;
    launch_gemm<HID, EPI_PART>(w, splits, s);
    k_sum_parts<<<64, 256, 0, s>>>(part_.p, splits, HID * HID, HID * HID, grad_.p + OFF_W3);
    w.A = dz2t_.p; w.B = h1t_.p;
    launch_gemm<HID, EPI_PART>(w, splits, s);
    k_sum_parts<<<64, 256, 0, s>>>(part_.p, splits, HID * HID, HID * HID, grad_.p + OFF_W2);
    w.A = dz1t_.p; w.B = xbt_.p;
    launch_gemm<NIN, EPI_PART>(w, splits, s);
    k_sum_parts<<<8, 256, 0, s>>>(part_.p, splits, HID * NIN, HID * NIN, grad_.p + OFF_W1);
    k_row_sums<<<HID, 256, 0, s>>>(dz3t_.p, B, grad_.p + OFF_B3);
    k_row_sums<<<HID, 256, 0, s>>>(dz2t_.p, B, grad_.p + OFF_B2);
    k_row_sums<<<HID, 256, 0, s>>>(dz1t_.p, B, grad_.p + OFF_B1);
    if (apply) {
        adam_t_++;
        float bc1 = 1.0f - std::pow(0.9f, (float)adam_t_), bc2 = 1.0f - std::pow(0.999f, (float)adam_t_);
        k_adam<<<64, 256, 0, s>>>(par_.p, grad_.p, m_.p, v_.p, NPAR, lr, bc1, bc2);
        publish(s);
    }
    return 0.0f;
}

void WarmStartNet::infer_device(const float *d_x, int64_t n, float *d_y, cudaStream_t s)
{
    if (n <= 0) return;
    int64_t done = 0;
    while (done < n) {
        int B = (int)std::min<int64_t>(n - done, BMAX);
        int Bp = (B + 127) / 128 * 128;
        ensure_batch(Bp);
        k_pack_inputs<<<(Bp + 127) / 128, 128, 0, s>>>(d_x + done * NIN, nullptr, B, Bp, norm_.p, xb_.p, nullptr, Bp,
                                                       nullptr, nullptr);
        forward(Bp, false, s);
        k_head_fwd<<<(B + 127) / 128, 128, 0, s>>>(h3_.p, B, par_.p, norm_.p, 1, d_y + done * NOUT);
        done += B;
    }
    int e = 0;
    k_read_err<<<1, 1, 0, s>>>((int *)loss_.p + 2, (int *)loss_.p + 3);
    cuda_check(cudaMemcpyAsync(&e, (int *)loss_.p + 3, sizeof(int), cudaMemcpyDeviceToHost, s), "D2H");
    cuda_check(cudaStreamSynchronize(s), "cudaStreamSynchronize");
    if (e) throw Failure(IFEA_CUDA_ERROR, "Warm-start network: a tensor-core wait timed out.");
}

void WarmStartNet::infer_host(const float *x, int64_t n, float *y)
{
    DBuf<float> a, b;
    a.upload(x, (size_t)n * NIN, st_);
    b.resize((size_t)n * NOUT);
    infer_device(a.p, n, b.p, st_);
    b.download(y, (size_t)n * NOUT, st_);
    cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
}

float WarmStartNet::gradients_host(const float *x, const float *t, int64_t n, float *grad_host)
{
    if (n <= 0 || n % 128 || n > BMAX) throw Failure(IFEA_INPUT_INVALID, "Gradient rows must be a positive multiple of 128, at most 8192.");
    int B = (int)n;
    ensure_batch(B);
    DBuf<float> a, b;
    a.upload(x, (size_t)n * NIN, st_);
    b.upload(t, (size_t)n * NOUT, st_);
    k_pack_inputs<<<(B + 127) / 128, 128, 0, st_>>>(a.p, nullptr, n, B, norm_.p, xb_.p, xbt_.p, B, b.p, tb_.p);
    forward(B, true, st_);
    k_head_fwd<<<(B + 127) / 128, 128, 0, st_>>>(h3_.p, B, par_.p, norm_.p, 0, y_.p);
    backward_and_step(B, false, 0.0f, st_);
    std::vector<float> g(NPAR + 1);
    cuda_check(cudaMemcpyAsync(g.data(), grad_.p, sizeof(float) * NPAR, cudaMemcpyDeviceToHost, st_), "D2H");
    int e = 0;
    k_read_err<<<1, 1, 0, st_>>>((int *)loss_.p + 2, (int *)loss_.p + 3);
    cuda_check(cudaMemcpyAsync(&e, (int *)loss_.p + 3, sizeof(int), cudaMemcpyDeviceToHost, st_), "D2H");
    // the loss: the last per-block slot of the head partials, summed on the host
    int nblk = (B + 127) / 128, hstride = NOUT * HID + NOUT + 1;
    std::vector<float> hp((size_t)nblk * hstride);
    cuda_check(cudaMemcpyAsync(hp.data(), hpart_.p, sizeof(float) * hp.size(), cudaMemcpyDeviceToHost, st_), "D2H");
    cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
    if (e) throw Failure(IFEA_CUDA_ERROR, "Warm-start network: a tensor-core wait timed out.");
    std::memcpy(grad_host, g.data(), sizeof(float) * NPAR);
    double l = 0;
    for (int k = 0; k < nblk; k++) l += hp[(size_t)k * hstride + hstride - 1];
    return (float)(l / ((double)n * NOUT));
}

float WarmStartNet::train(int steps, int batch, float lr, uint64_t seed)
{
    if (count_ < 1) throw Failure(IFEA_BAD_STATE, "The warm-start network has no training samples.");
    int B = std::max(128, std::min(BMAX, batch / 128 * 128));
    ensure_batch(B);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st_);
    std::mt19937_64 rng(seed);
    std::vector<int32_t> perm((size_t)count_);
    std::iota(perm.begin(), perm.end(), 0);
    int64_t pos = count_;
    std::vector<int32_t> idx(B);
    HostPinned<int32_t> hidx;
    hidx.resize((size_t)B * 2);
    int nblk = (B + 127) / 128, hstride = NOUT * HID + NOUT + 1;
    DBuf<float> losses;
    int tail = std::max(1, steps / 10);
    losses.resize((size_t)tail);
    losses.zero(st_);
    for (int it = 0; it < steps; it++) {
        for (int r = 0; r < B; r++) {
            if (pos >= count_) {
                std::shuffle(perm.begin(), perm.end(), rng);
                pos = 0;
            }
            idx[r] = perm[pos++];
        }
        int32_t *hb = hidx.p + (it & 1) * B;
        cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");  // the pinned slot is free again
        std::memcpy(hb, idx.data(), sizeof(int32_t) * B);
        cuda_check(cudaMemcpyAsync(idx_.p, hb, sizeof(int32_t) * B, cudaMemcpyHostToDevice, st_), "H2D");
        k_pack_inputs<<<nblk, 128, 0, st_>>>(dx_.p, idx_.p, count_, B, norm_.p, xb_.p, xbt_.p, B, dt_.p, tb_.p);
        forward(B, true, st_);
        k_head_fwd<<<nblk, 128, 0, st_>>>(h3_.p, B, par_.p, norm_.p, 0, y_.p);
        backward_and_step(B, true, lr, st_);
        if (it >= steps - tail) {
            // the batch loss: the last slot of the head partials, summed into the ring of final losses
            k_sum_parts<<<1, 1, 0, st_>>>(hpart_.p + hstride - 1, nblk, 1, hstride, losses.p + (it - (steps - tail)));
        }
    }
    std::vector<float> hl((size_t)tail);
    losses.download(hl.data(), (size_t)tail, st_);
    cudaEventRecord(e1, st_);
    int e = 0;
    k_read_err<<<1, 1, 0, st_>>>((int *)loss_.p + 2, (int *)loss_.p + 3);
    cuda_check(cudaMemcpyAsync(&e, (int *)loss_.p + 3, sizeof(int), cudaMemcpyDeviceToHost, st_), "D2H");
    cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    train_ms += ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (e) throw Failure(IFEA_CUDA_ERROR, "Warm-start network: a tensor-core wait timed out.");
    double l = 0;
    for (float v : hl) l += v;
    return (float)(l / tail / ((double)B * NOUT));
}

}  // namespace ifea

// ------------------------------------------------------------------ C ABI

namespace {
template <class F>
ifea_status guard_mlp(ifea_mlp *m, F &&f)
{
    if (!m || !m->net) return IFEA_INPUT_INVALID;
    try {
        f(*m->net);
        return IFEA_OK;
    } catch (const ifea::Failure &e) {
        m->err = e.what();
        return e.status;
    } catch (const std::exception &e) {
        m->err = e.what();
        return IFEA_CUDA_ERROR;
    }
}
}  // namespace

extern "C" {

ifea_status ifea_mlp_create(uint64_t seed, ifea_mlp **out)
{
    if (!out) return IFEA_INPUT_INVALID;
    *out = nullptr;
    auto *m = new ifea_mlp;
    try {
        m->net = new ifea::WarmStartNet(seed);
    } catch (const std::exception &e) {
        delete m;
        return IFEA_CUDA_ERROR;
    }
    *out = m;
    return IFEA_OK;
}

void ifea_mlp_destroy(ifea_mlp *m)
{
    if (!m) return;
    delete m->net;
    delete m;
}

const char *ifea_mlp_last_error(const ifea_mlp *m) { return m ? m->err.c_str() : "null network"; }

int64_t ifea_mlp_param_count(void) { return ifea::wsm::NPAR; }

ifea_status ifea_mlp_get_params(ifea_mlp *m, float *host, int64_t count)
{
    if (count != ifea::wsm::NPAR || !host) return IFEA_INPUT_INVALID;
    return guard_mlp(m, [&](ifea::WarmStartNet &n) { n.get_params(host); });
}

ifea_status ifea_mlp_set_params(ifea_mlp *m, const float *host, int64_t count)
{
    if (count != ifea::wsm::NPAR || !host) return IFEA_INPUT_INVALID;
    return guard_mlp(m, [&](ifea::WarmStartNet &n) { n.set_params(host); });
}

ifea_status ifea_mlp_get_normalisation(ifea_mlp *m, float *host)
{
    if (!host) return IFEA_INPUT_INVALID;
    return guard_mlp(m, [&](ifea::WarmStartNet &n) { n.get_norm(host); });
}

ifea_status ifea_mlp_set_normalisation(ifea_mlp *m, const float *host)
{
    if (!host) return IFEA_INPUT_INVALID;
    return guard_mlp(m, [&](ifea::WarmStartNet &n) { n.set_norm(host); });
}

ifea_status ifea_mlp_add_samples(ifea_mlp *m, const float *features, const float *targets, int64_t n)
{
    if (n < 0 || (n > 0 && (!features || !targets))) return IFEA_INPUT_INVALID;
    return guard_mlp(m, [&](ifea::WarmStartNet &net) { net.add_samples_host(features, targets, n); });
}

int64_t ifea_mlp_samples(const ifea_mlp *m) { return m && m->net ? m->net->samples() : 0; }

ifea_status ifea_mlp_clear_samples(ifea_mlp *m)
{
    return guard_mlp(m, [&](ifea::WarmStartNet &n) { n.clear_samples(); });
}

ifea_status ifea_mlp_fit_normalisation(ifea_mlp *m)
{
    return guard_mlp(m, [&](ifea::WarmStartNet &n) { n.fit_normalisation(); });
}

ifea_status ifea_mlp_forward(ifea_mlp *m, const float *x, int64_t n, float *y)
{
    if (n < 0 || (n > 0 && (!x || !y))) return IFEA_INPUT_INVALID;
    return guard_mlp(m, [&](ifea::WarmStartNet &net) { net.infer_host(x, n, y); });
}

ifea_status ifea_mlp_gradients(ifea_mlp *m, const float *x, const float *t, int64_t n, float *grad, float *loss)
{
    if (!x || !t || !grad) return IFEA_INPUT_INVALID;
    return guard_mlp(m, [&](ifea::WarmStartNet &net) {
        float l = net.gradients_host(x, t, n, grad);
        if (loss) *loss = l;
    });
}

ifea_status ifea_mlp_train(ifea_mlp *m, int32_t steps, int32_t batch, float lr, uint64_t seed, float *final_loss,
                           double *gpu_ms)
{
    if (steps <= 0 || batch <= 0 || !(lr > 0)) return IFEA_INPUT_INVALID;
    return guard_mlp(m, [&](ifea::WarmStartNet &net) {
        double before = net.train_ms;
        float l = net.train(steps, batch, lr, seed);
        if (final_loss) *final_loss = l;
        if (gpu_ms) *gpu_ms = net.train_ms - before;
    });
}

}  // extern "C"
