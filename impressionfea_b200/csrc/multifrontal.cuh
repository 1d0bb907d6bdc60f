// multifrontal.cuh — GPU multifrontal sparse Cholesky (numeric factorisation and solves) behind the reference's
// ISpdSolver seam (Solver/Linear/ISpdSolver.cs:24-41; stands in for CudssSolver.cs:105-145).
//
// Every supernode owns a dense m x m column-major front in one device pool, laid out level by level. A
// factorisation assembles the matrix values into the fronts of a level (one gather), adds the children's update
// matrices (extend-add, one launch per child rank so every entry sums its children in a fixed order), then
// eliminates the supernode's pivot columns in panels of 64: a one-CTA-per-front kernel factors the panel's
// diagonal block in shared memory and solves the rows below it, and a tiled kernel subtracts the panel's
// outer product from the trailing front. What remains in the trailing block is the update matrix the parent
// reads; the pivot columns are the factor, so no copy is made. The solves walk the levels up (update vectors)
// and down (gathers from solved ancestors). Nothing uses atomics on values: results are bit-reproducible.
#pragma once
#include <cusolverSp.h>
#include <cusparse.h>

#include <algorithm>
#include <climits>
#include <string>
#include <vector>

#include "multifrontal.h"
#include "runtime.cuh"

namespace ifea {

namespace mf {

constexpr int PW = 64;  // panel width
constexpr int TT = 32;  // update tile

struct Dev {
    const int32_t *ncol, *m, *c0, *idx_start, *idx, *relmap_start, *relmap, *uvec_start, *child_start, *child_list;
    const int64_t *front_off;
    double *F, *U;
};

static __global__ void k_scatter(int64_t n, const int64_t *__restrict__ dst, const int32_t *__restrict__ src,
                          const double *__restrict__ vals, double *__restrict__ F)
{
    for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x)
        F[dst[t]] = vals[src[t]];
}

// Extend-add of the update matrices of the listed children into their parents' fronts.
static __global__ void k_extend(Dev D, const int32_t *__restrict__ children, const int32_t *__restrict__ parents)
{
    int c = children[blockIdx.y];
    int p = parents[c];
    int mc = D.m[c], nc = D.ncol[c], nr = mc - nc, mp = D.m[p];
    const double *Fc = D.F + D.front_off[c];
    double *Fp = D.F + D.front_off[p];
    const int32_t *rm = D.relmap + D.relmap_start[c];
    for (int j = blockIdx.x; j < nr; j += gridDim.x) {
        int64_t pj = (int64_t)rm[j] * mp;
        const double *col = Fc + (int64_t)(nc + j) * mc + nc;
        for (int i = j + threadIdx.x; i < nr; i += blockDim.x) Fp[pj + rm[i]] += col[i];
    }
}

// Panel k0 of every listed front: Cholesky of the diagonal block in shared memory, then rows below solved
// against it (X L11^T = F21). The lowest failing pivot column (new numbering) goes to err.
static __global__ void __launch_bounds__(256) k_panel(Dev D, const int32_t *__restrict__ fronts, int k0, int *err)
{
    __shared__ double Ds[PW][PW + 1];
    __shared__ int bad;
    int s = fronts[blockIdx.x];
    int ms = D.m[s], w = min(PW, D.ncol[s] - k0);
    double *F = D.F + D.front_off[s];
    int tid = threadIdx.x, nt = blockDim.x;
    if (tid == 0) bad = 0;
    for (int t = tid; t < w * w; t += nt) {
        int r = t / w, c = t % w;
        if (r >= c) Ds[r][c] = F[(int64_t)(k0 + c) * ms + k0 + r];
    }
    __syncthreads();
    for (int k = 0; k < w; k++) {
        if (tid == 0) {
            double d = Ds[k][k];
            if (!(d > 0)) {
                bad = 1;
                atomicMin(err, D.c0[s] + k0 + k);
            } else {
                Ds[k][k] = sqrt(d);
            }
        }
        __syncthreads();
        if (bad) return;
        double lkk = Ds[k][k];
        for (int r = k + 1 + tid; r < w; r += nt) Ds[r][k] /= lkk;
        __syncthreads();
        int mm = w - k - 1;
        for (int t = tid; t < mm * (mm + 1) / 2; t += nt) {
            int di = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
            while ((di + 1) * (di + 2) / 2 <= t) di++;
            while (di * (di + 1) / 2 > t) di--;
            int dj = t - di * (di + 1) / 2;
            int r = k + 1 + di, c = k + 1 + dj;
            Ds[r][c] -= Ds[r][k] * Ds[c][k];
        }
        __syncthreads();
    }
    for (int t = tid; t < w * w; t += nt) {
        int r = t / w, c = t % w;
        if (r >= c) F[(int64_t)(k0 + c) * ms + k0 + r] = Ds[r][c];
    }
    // rows below the block: x_k = (f_k - sum_{l<k} x_l L_kl) / L_kk
    for (int r = k0 + w + tid; r < ms; r += nt) {
        double x[PW];
        for (int k = 0; k < w; k++) {
            double v = F[(int64_t)(k0 + k) * ms + r];
            for (int l = 0; l < k; l++) v -= x[l] * Ds[k][l];
            x[k] = v / Ds[k][k];
        }
        for (int k = 0; k < w; k++) F[(int64_t)(k0 + k) * ms + r] = x[k];
    }
}

// Trailing update of every listed front after panel k0: F22 -= L21 L21^T on 32x32 lower tiles.
static __global__ void __launch_bounds__(256) k_update(Dev D, const int32_t *__restrict__ fronts, int k0)
{
    __shared__ double Ai[TT][PW + 1], Aj[TT][PW + 1];
    int s = fronts[blockIdx.y];
    int ms = D.m[s], w = min(PW, D.ncol[s] - k0), r0 = k0 + w, nt = ms - r0;
    if (nt <= 0) return;
    double *F = D.F + D.front_off[s];
    int nti = (nt + TT - 1) / TT;
    int ntiles = nti * (nti + 1) / 2;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
        while ((ti + 1) * (ti + 2) / 2 <= t) ti++;
        while (ti * (ti + 1) / 2 > t) ti--;
        int tj = t - ti * (ti + 1) / 2;
        int ri0 = r0 + ti * TT, cj0 = r0 + tj * TT;
        __syncthreads();
        for (int q = threadIdx.x; q < TT * w; q += blockDim.x) {
            int rr = q % TT, k = q / TT;
            int gi = ri0 + rr, gj = cj0 + rr;
            Ai[rr][k] = gi < ms ? F[(int64_t)(k0 + k) * ms + gi] : 0.0;
            Aj[rr][k] = gj < ms ? F[(int64_t)(k0 + k) * ms + gj] : 0.0;
        }
        __syncthreads();
        for (int q = threadIdx.x; q < TT * TT; q += blockDim.x) {
            int ii = q % TT, jj = q / TT;
            int gi = ri0 + ii, gj = cj0 + jj;
            if (gi >= ms || gj >= ms || gi < gj) continue;
            double acc = 0;
            for (int k = 0; k < w; k++) acc += Ai[ii][k] * Aj[jj][k];
            F[(int64_t)gj * ms + gi] -= acc;
        }
    }
}

static __global__ void k_permute_in(int n, const int32_t *perm, const double *b, double *y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = b[perm[i]];
}
static __global__ void k_permute_out(int n, const int32_t *perm, const double *y, double *x)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[perm[i]] = y[i];
}

// Forward elimination of the fronts of one level: y(cols) and the update vector for the parent.
static __global__ void __launch_bounds__(512) k_forward(Dev D, const int32_t *__restrict__ fronts, double *y)
{
    extern __shared__ double acc[];
    int s = fronts[blockIdx.x];
    int ms = D.m[s], nc = D.ncol[s], c0 = D.c0[s];
    const double *F = D.F + D.front_off[s];
    int tid = threadIdx.x, nt = blockDim.x;
    for (int k = tid; k < ms; k += nt) acc[k] = k < nc ? y[c0 + k] : 0.0;
    __syncthreads();
    for (int q = D.child_start[s]; q < D.child_start[s + 1]; q++) {
        int c = D.child_list[q];
        int nr = D.m[c] - D.ncol[c];
        const int32_t *rm = D.relmap + D.relmap_start[c];
        const double *u = D.U + D.uvec_start[c];
        for (int i = tid; i < nr; i += nt) acc[rm[i]] -= u[i];
        __syncthreads();
    }
    for (int kb = 0; kb < nc; kb += PW) {
        int w = min(PW, nc - kb);
        for (int k = kb; k < kb + w; k++) {
            double yk = acc[k] / F[(int64_t)k * ms + k];
            __syncthreads();
            if (tid == 0) acc[k] = yk;
            for (int r = k + 1 + tid; r < kb + w; r += nt) acc[r] -= F[(int64_t)k * ms + r] * yk;
            __syncthreads();
        }
        for (int r = kb + w + tid; r < ms; r += nt) {
            double v = acc[r];
            for (int k = kb; k < kb + w; k++) v -= F[(int64_t)k * ms + r] * acc[k];
            acc[r] = v;
        }
        __syncthreads();
    }
    for (int k = tid; k < nc; k += nt) y[c0 + k] = acc[k];
    double *u = D.U + D.uvec_start[s];
    for (int i = tid; i < ms - nc; i += nt) u[i] = -acc[nc + i];
}

// Back substitution of the fronts of one level: x(cols) from y(cols) and the solved ancestors' x.
static __global__ void __launch_bounds__(512) k_backward(Dev D, const int32_t *__restrict__ fronts, const double *y, double *x)
{
    extern __shared__ double sm[];
    int s = fronts[blockIdx.x];
    int ms = D.m[s], nc = D.ncol[s], c0 = D.c0[s], nr = ms - nc;
    const double *F = D.F + D.front_off[s];
    const int32_t *ix = D.idx + D.idx_start[s];
    double *acc = sm, *xs = sm + nc;
    int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
    for (int k = tid; k < nc; k += nt) acc[k] = y[c0 + k];
    for (int i = tid; i < nr; i += nt) xs[i] = x[ix[nc + i]];
    __syncthreads();
    for (int k = warp; k < nc; k += nw) {
        const double *col = F + (int64_t)k * ms + nc;
        double v = 0;
        for (int i = lane; i < nr; i += 32) v += col[i] * xs[i];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if (lane == 0) acc[k] -= v;
    }
    __syncthreads();
    int nblk = (nc + PW - 1) / PW;
    for (int bi = nblk - 1; bi >= 0; bi--) {
        int kb = bi * PW, w = min(PW, nc - kb), ke = kb + w;
        for (int j = kb + warp; j < ke; j += nw) {
            const double *col = F + (int64_t)j * ms;
            double v = 0;
            for (int k = ke + lane; k < nc; k += 32) v += col[k] * acc[k];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) acc[j] -= v;
        }
        __syncthreads();
        for (int k = ke - 1; k >= kb; k--) {
            double xk = acc[k] / F[(int64_t)k * ms + k];
            __syncthreads();
            if (tid == 0) acc[k] = xk;
            for (int j = kb + tid; j < k; j += nt) acc[j] -= F[(int64_t)j * ms + k] * xk;
            __syncthreads();
        }
    }
    for (int k = tid; k < nc; k += nt) x[c0 + k] = acc[k];
}

static __global__ void k_finite(int n, const double *x, int *flag)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        if (!isfinite(x[i])) atomicExch(flag, 1);
}

}  // namespace mf

class MfSolver {
public:
    explicit MfSolver(cudaStream_t s) : st_(s)
    {
        if (cusolverSpCreate(&hsp_) != CUSOLVER_STATUS_SUCCESS) throw Failure(IFEA_CUDA_ERROR, "cusolverSpCreate failed");
        if (cusparseCreateMatDescr(&descr_) != CUSPARSE_STATUS_SUCCESS) throw Failure(IFEA_CUDA_ERROR, "cusparseCreateMatDescr failed");
        cusparseSetMatType(descr_, CUSPARSE_MATRIX_TYPE_GENERAL);
        cusparseSetMatIndexBase(descr_, CUSPARSE_INDEX_BASE_ZERO);
        d_err_.resize(2);
    }
    ~MfSolver()
    {
        if (descr_) cusparseDestroyMatDescr(descr_);
        if (hsp_) cusolverSpDestroy(hsp_);
    }
    MfSolver(const MfSolver &) = delete;
    MfSolver &operator=(const MfSolver &) = delete;

    void set_stream(cudaStream_t s) { st_ = s; }
    bool analyzed() const { return analyzed_; }
    bool factored() const { return factored_; }
    int64_t factor_nonzeros() const { return sym_.factor_nnz; }
    const MfSymbolic &symbolic() const { return sym_; }
    int n() const { return sym_.n; }

    void analyze(int n, const int32_t *col_ptr, const int32_t *row_idx, int block)
    {
        analyzed_ = factored_ = false;
        std::string e = sym_.analyze(n, col_ptr, row_idx, block, hsp_, descr_);
        if (!e.empty()) throw Failure(IFEA_INPUT_INVALID, e);
        const MfSymbolic &S = sym_;
        if ((size_t)S.max_m * sizeof(double) > 200 * 1024)
            throw Failure(IFEA_INPUT_INVALID, "front larger than the solve kernels' shared-memory window");
        d_ncol_.upload(S.ncol, st_); d_m_.upload(S.m, st_); d_c0_.upload(S.c0, st_); d_idxs_.upload(S.idx_start, st_);
        d_idx_.upload(S.idx, st_); d_rms_.upload(S.relmap_start, st_); d_rm_.upload(S.relmap, st_);
        d_uvs_.upload(S.uvec_start, st_); d_off_.upload(S.front_off, st_); d_par_.upload(S.parent, st_);
        d_perm_.upload(S.perm, st_); d_adst_.upload(S.a_dst, st_); d_asrc_.upload(S.a_src, st_);
        d_ext_.upload(S.ext_child, st_);
        // children lists (ascending) for the solves
        std::vector<int32_t> cs(S.nsuper + 1, 0), cl;
        for (int s = 0; s < S.nsuper; s++)
            if (S.parent[s] >= 0) cs[S.parent[s] + 1]++;
        for (int s = 0; s < S.nsuper; s++) cs[s + 1] += cs[s];
        cl.assign(cs[S.nsuper], 0);
        {
            std::vector<int32_t> fill(cs.begin(), cs.end() - 1);
            for (int s = 0; s < S.nsuper; s++)
                if (S.parent[s] >= 0) cl[fill[S.parent[s]]++] = s;
        }
        d_cs_.upload(cs, st_);
        d_cl_.upload(cl, st_);
        // per level: fronts sorted by pivot count (descending) so each panel step's active fronts are a prefix
        lvl_sorted_.assign(S.level_list.begin(), S.level_list.end());
        for (int l = 0; l < S.nlevels; l++)
            std::stable_sort(lvl_sorted_.begin() + S.level_start[l], lvl_sorted_.begin() + S.level_start[l + 1],
                             [&](int a, int b) { return S.ncol[a] > S.ncol[b]; });
        d_lvl_.upload(lvl_sorted_, st_);
        d_F_.resize(S.pool);
        d_U_.resize(std::max<int64_t>(S.uvec_pool, 1));
        d_y_.resize(n);
        dev_.ncol = d_ncol_; dev_.m = d_m_; dev_.c0 = d_c0_; dev_.idx_start = d_idxs_; dev_.idx = d_idx_;
        dev_.relmap_start = d_rms_; dev_.relmap = d_rm_; dev_.uvec_start = d_uvs_; dev_.child_start = d_cs_;
        dev_.child_list = d_cl_; dev_.front_off = d_off_; dev_.F = d_F_; dev_.U = d_U_;
        size_t smem = (size_t)S.max_m * sizeof(double);
        cuda_check(cudaFuncSetAttribute((const void *)mf::k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "cudaFuncSetAttribute");
        cuda_check(cudaFuncSetAttribute((const void *)mf::k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "cudaFuncSetAttribute");
        cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
        analyzed_ = true;
    }

    // Numeric factorisation of device values in the order of the analysed full CSC pattern.
    void factorize(const double *d_full_vals)
    {
        if (!analyzed_) throw Failure(IFEA_BAD_STATE, "Analyze must be called first.");
        factored_ = false;
        const MfSymbolic &S = sym_;
        int32_t init[2] = {INT_MAX, 0};
        cuda_check(cudaMemcpyAsync(d_err_.p, init, sizeof init, cudaMemcpyHostToDevice, st_), "H2D");
        for (int l = 0; l < S.nlevels; l++) {
            int64_t p0 = S.level_pool_start[l], p1 = S.level_pool_start[l + 1];
            cuda_check(cudaMemsetAsync(d_F_.p + p0, 0, (size_t)(p1 - p0) * sizeof(double), st_), "memset fronts");
            int64_t a0 = S.a_level_start[l], a1 = S.a_level_start[l + 1];
            if (a1 > a0) {
                int g = (int)std::min<int64_t>((a1 - a0 + 255) / 256, 4 * 148);
                mf::k_scatter<<<g, 256, 0, st_>>>(a1 - a0, d_adst_.p + a0, d_asrc_.p + a0, d_full_vals, d_F_);
            }
            for (int r = 0; r < S.max_rank; r++) {
                int32_t e0 = S.ext_start[(size_t)l * S.max_rank + r], e1 = S.ext_start[(size_t)l * S.max_rank + r + 1];
                if (e1 <= e0) continue;
                dim3 grid(64, e1 - e0);
                mf::k_extend<<<grid, 128, 0, st_>>>(dev_, d_ext_.p + e0, d_par_);
            }
            int q0 = S.level_start[l], q1 = S.level_start[l + 1];
            int maxc = S.ncol[lvl_sorted_[q0]];
            for (int k0 = 0; k0 < maxc; k0 += mf::PW) {
                int cnt = 0, maxt = 0;
                for (int q = q0; q < q1 && S.ncol[lvl_sorted_[q]] > k0; q++) {
                    int s = lvl_sorted_[q];
                    cnt++;
                    int w = std::min(mf::PW, S.ncol[s] - k0), nt = S.m[s] - k0 - w;
                    int nti = (nt + mf::TT - 1) / mf::TT;
                    maxt = std::max(maxt, nti * (nti + 1) / 2);
                }
                mf::k_panel<<<cnt, 256, 0, st_>>>(dev_, d_lvl_.p + q0, k0, d_err_);
                if (maxt > 0) {
                    dim3 grid(std::min(maxt, 4096), cnt);
                    mf::k_update<<<grid, 256, 0, st_>>>(dev_, d_lvl_.p + q0, k0);
                }
            }
        }
        cuda_check(cudaGetLastError(), "multifrontal factorisation launch");
        int32_t e[2];
        cuda_check(cudaMemcpyAsync(e, d_err_.p, sizeof e, cudaMemcpyDeviceToHost, st_), "D2H");
        cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
        if (e[0] != INT_MAX) {
            int row = S.perm[e[0]];
            throw Failure(IFEA_NOT_SPD, "Stiffness matrix not positive definite at equation " + std::to_string(row) +
                                            ". The billet is probably unrestrained.");
        }
        factored_ = true;
    }

    // x = A^-1 b on the device (b and x may alias).
    void solve(const double *d_b, double *d_x)
    {
        if (!factored_) throw Failure(IFEA_BAD_STATE, "Factorize must be called first.");
        const MfSymbolic &S = sym_;
        int n = S.n, g = std::max(1, std::min((n + 255) / 256, 4 * 148));
        mf::k_permute_in<<<g, 256, 0, st_>>>(n, d_perm_, d_b, d_y_);
        size_t smem = (size_t)S.max_m * sizeof(double);
        for (int l = 0; l < S.nlevels; l++) {
            int q0 = S.level_start[l], cnt = S.level_start[l + 1] - q0;
            mf::k_forward<<<cnt, 512, smem, st_>>>(dev_, d_lvl_.p + q0, d_y_);
        }
        // back substitution writes x (new numbering) in place of y, top level first
        for (int l = S.nlevels - 1; l >= 0; l--) {
            int q0 = S.level_start[l], cnt = S.level_start[l + 1] - q0;
            mf::k_backward<<<cnt, 512, smem, st_>>>(dev_, d_lvl_.p + q0, d_y_, d_y_);
        }
        mf::k_permute_out<<<g, 256, 0, st_>>>(n, d_perm_, d_y_, d_x);
        cuda_check(cudaGetLastError(), "multifrontal solve launch");
    }

    void check_finite(const double *d_x)
    {
        int32_t zero = 0, f = 0;
        cuda_check(cudaMemcpyAsync(d_err_.p + 1, &zero, sizeof zero, cudaMemcpyHostToDevice, st_), "H2D");
        mf::k_finite<<<std::max(1, std::min((sym_.n + 255) / 256, 592)), 256, 0, st_>>>(sym_.n, d_x, d_err_.p + 1);
        cuda_check(cudaMemcpyAsync(&f, d_err_.p + 1, sizeof f, cudaMemcpyDeviceToHost, st_), "D2H");
        cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
        if (f) throw Failure(IFEA_NOT_SPD, "Stiffness matrix not positive definite at equation -1 (pivot NaN).");
    }

private:
    cudaStream_t st_;
    cusolverSpHandle_t hsp_ = nullptr;
    cusparseMatDescr_t descr_ = nullptr;
    MfSymbolic sym_;
    bool analyzed_ = false, factored_ = false;
    std::vector<int32_t> lvl_sorted_;
    DBuf<int32_t> d_ncol_, d_m_, d_c0_, d_idxs_, d_idx_, d_rms_, d_rm_, d_uvs_, d_par_, d_perm_, d_asrc_, d_ext_, d_cs_,
        d_cl_, d_lvl_, d_err_;
    DBuf<int64_t> d_off_, d_adst_;
    DBuf<double> d_F_, d_U_, d_y_;
    mf::Dev dev_{};
};

}  // namespace ifea
