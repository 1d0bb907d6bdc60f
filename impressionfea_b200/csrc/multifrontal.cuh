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
constexpr int UT = 64;  // update tile

struct Dev {
    const int32_t *ncol, *m, *c0, *idx_start, *idx, *relmap_start, *relmap, *uvec_start, *child_start, *child_list;
    const int64_t *front_off, *inv_off, *xinv_off;
    double *F, *U, *Inv, *Xinv, *Abig;
};

constexpr int kWideM = 192;  // fronts at least this tall get a full pivot-block inverse and multi-CTA solves

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

// Panel k0 of every listed front: Cholesky of the diagonal block in shared memory, the block's inverse (kept for
// the solves), then the rows below: X = F21 L11^-T, as a triangular matrix-vector product per row. The lowest
// failing pivot column (new numbering) goes to err.
static __global__ void __launch_bounds__(256) k_panel(Dev D, const int32_t *__restrict__ fronts, int k0, int *err)
{
    __shared__ double Ds[PW][PW + 1];
    __shared__ int bad;
    int s = fronts[blockIdx.x];
    int ms = D.m[s], w = min(PW, D.ncol[s] - k0);
    double *F = D.F + D.front_off[s];
    double *Inv = D.Inv + D.inv_off[s] + (int64_t)(k0 / PW) * PW * PW;
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
    // inverse of the lower-triangular block, column t by thread t (forward substitution on e_t)
    if (tid < w) {
        double x[PW];
        for (int i = 0; i < tid; i++) x[i] = 0.0;
        x[tid] = 1.0 / Ds[tid][tid];
        for (int i = tid + 1; i < w; i++) {
            double v = 0;
            for (int k = tid; k < i; k++) v += Ds[i][k] * x[k];
            x[i] = -v / Ds[i][i];
        }
        for (int i = 0; i < PW; i++) Inv[(int64_t)tid * PW + i] = i < w ? x[i] : 0.0;  // column-major, row i
    }
    for (int t = tid; t < PW * PW; t += nt)
        if (t / PW >= w) Inv[t] = 0.0;
    __syncthreads();
}

// Rows below the diagonal block of panel k0, 64 rows per CTA: X = F21 L11^-T = F21 Dinv^T, i.e.
// x_k = sum_{l<=k} f_l Dinv[k][l], with Dinv the stored inverse of the diagonal block.
static __global__ void __launch_bounds__(256) k_panel_trsm(Dev D, const int32_t *__restrict__ fronts, int k0)
{
    extern __shared__ double shm[];
    double (*Di)[PW + 1] = (double (*)[PW + 1])shm;
    double (*Ft)[PW + 1] = (double (*)[PW + 1])(shm + PW * (PW + 1));
    int s = fronts[blockIdx.y];
    int ms = D.m[s], w = min(PW, D.ncol[s] - k0);
    int rbeg = k0 + w + blockIdx.x * PW;
    if (rbeg >= ms) return;
    int rows = min(PW, ms - rbeg);
    double *F = D.F + D.front_off[s];
    const double *Inv = D.Inv + D.inv_off[s] + (int64_t)(k0 / PW) * PW * PW;
    for (int t = threadIdx.x; t < PW * PW; t += blockDim.x) {
        int c = t / PW, i = t % PW;
        Di[i][c] = Inv[t];  // column-major inverse: row i, column c
    }
    for (int t = threadIdx.x; t < w * PW; t += blockDim.x) {
        int l = t / PW, rr = t % PW;
        Ft[rr][l] = rr < rows ? F[(int64_t)(k0 + l) * ms + rbeg + rr] : 0.0;
    }
    __syncthreads();
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    double acc[4][4];
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
    for (int l = 0; l < w; l++) {
        double f[4], d[4];
        for (int a = 0; a < 4; a++) f[a] = Ft[tx + 16 * a][l];
        for (int b = 0; b < 4; b++) d[b] = Di[ty + 16 * b][l];
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) acc[a][b] += f[a] * d[b];
    }
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
            int rr = tx + 16 * a, k = ty + 16 * b;
            if (rr < rows && k < w) F[(int64_t)(k0 + k) * ms + rbeg + rr] = acc[a][b];
        }
}

// Block row bi of the full inverse X = L11^-1 of every listed wide supernode (column-major ncol x ncol), one CTA
// per (block column j <= bi, front): X_ii = Dinv_i, X_ij = -Dinv_i sum_{k=j}^{i-1} L_ik X_kj.
static __global__ void __launch_bounds__(256) k_inverse_row(Dev D, const int32_t *__restrict__ fronts, int bi)
{
    extern __shared__ double shm[];
    double (*A)[PW + 1] = (double (*)[PW + 1])shm;
    double (*B)[PW + 1] = (double (*)[PW + 1])(shm + PW * (PW + 1));
    int s = fronts[blockIdx.y];
    int bj = blockIdx.x;
    if (bj > bi) return;
    int ms = D.m[s], nc = D.ncol[s];
    const double *F = D.F + D.front_off[s];
    double *X = D.Xinv + D.xinv_off[s];
    int r0 = bi * PW, c0 = bj * PW, wr = min(PW, nc - r0), wc = min(PW, nc - c0);
    const double *Dinv_i = D.Inv + D.inv_off[s] + (int64_t)bi * PW * PW;
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    if (bj == bi) {
        for (int t = threadIdx.x; t < PW * PW; t += blockDim.x) {
            int c = t / PW, r = t % PW;
            if (r < wr && c < wc) X[(int64_t)(c0 + c) * nc + r0 + r] = Dinv_i[t];
        }
        return;
    }
    double acc[4][4];
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
    for (int bk = bj; bk < bi; bk++) {
        int k0 = bk * PW, wk = min(PW, nc - k0);
        __syncthreads();
        for (int t = threadIdx.x; t < PW * PW; t += blockDim.x) {
            int k = t / PW, r = t % PW;
            A[r][k] = (r < wr && k < wk) ? F[(int64_t)(k0 + k) * ms + r0 + r] : 0.0;
            B[r][k] = (r < wk && k < wc) ? X[(int64_t)(c0 + k) * nc + k0 + r] : 0.0;
        }
        __syncthreads();
        for (int k = 0; k < PW; k++) {
            double a4[4], b4[4];
            for (int a = 0; a < 4; a++) a4[a] = A[tx + 16 * a][k];
            for (int b = 0; b < 4; b++) b4[b] = B[k][ty + 16 * b];
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) acc[a][b] += a4[a] * b4[b];
        }
    }
    __syncthreads();
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) B[tx + 16 * a][ty + 16 * b] = acc[a][b];
    for (int t = threadIdx.x; t < PW * PW; t += blockDim.x) {
        int c = t / PW, r = t % PW;
        A[r][c] = Dinv_i[t];
    }
    __syncthreads();
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
    for (int k = 0; k < PW; k++) {
        double a4[4], b4[4];
        for (int a = 0; a < 4; a++) a4[a] = A[tx + 16 * a][k];
        for (int b = 0; b < 4; b++) b4[b] = B[k][ty + 16 * b];
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) acc[a][b] += a4[a] * b4[b];
    }
    for (int a = 0; a < 4; a++)
        for (int b = 0; b < 4; b++) {
            int r = tx + 16 * a, c = ty + 16 * b;
            if (r < wr && c < wc) X[(int64_t)(c0 + c) * nc + r0 + r] = -acc[a][b];
        }
}

// ---------------------------------------------------------------- solves of wide supernodes (batched multi-CTA GEMVs)
// Per-front scratch vectors live at offset idx_start[s] (length m) in Abig (assembled right-hand side), Y1, Z.

// acc = [b(cols); 0] - children's update vectors (in child order).
static __global__ void k_wide_fwd_acc(Dev D, const int32_t *__restrict__ fronts, const double *y)
{
    int s = fronts[blockIdx.x];
    int ms = D.m[s], nc = D.ncol[s], c0 = D.c0[s];
    double *acc = D.Abig + D.idx_start[s];
    for (int k = threadIdx.x; k < ms; k += blockDim.x) acc[k] = k < nc ? y[c0 + k] : 0.0;
    __syncthreads();
    for (int q = D.child_start[s]; q < D.child_start[s + 1]; q++) {
        int c = D.child_list[q];
        int nr = D.m[c] - D.ncol[c];
        const int32_t *rm = D.relmap + D.relmap_start[c];
        const double *u = D.U + D.uvec_start[c];
        for (int i = threadIdx.x; i < nr; i += blockDim.x) acc[rm[i]] -= u[i];
        __syncthreads();
    }
}

// y1 = X acc1: 32 rows per CTA (blockIdx.x), 8 warps splitting the columns; front = blockIdx.y.
static __global__ void __launch_bounds__(256) k_wide_fwd_y(Dev D, const int32_t *__restrict__ fronts, double *y, double *Y1)
{
    __shared__ double part[8][33];
    int s = fronts[blockIdx.y];
    int nc = D.ncol[s], c0 = D.c0[s];
    if (blockIdx.x * 32 >= nc) return;
    const double *X = D.Xinv + D.xinv_off[s];
    const double *acc = D.Abig + D.idx_start[s];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int r = blockIdx.x * 32 + lane;
    double v = 0;
    if (r < nc)
        for (int c = warp; c <= r; c += 8) v += X[(int64_t)c * nc + r] * acc[c];
    part[warp][lane] = v;
    __syncthreads();
    if (warp == 0 && r < nc) {
        double t = 0;
        for (int w = 0; w < 8; w++) t += part[w][lane];
        y[c0 + r] = t;
        Y1[D.idx_start[s] + r] = t;
    }
}

// update vector t = -acc2 + L21 y1: 32 rows per CTA, 8 warps splitting the pivot columns.
static __global__ void __launch_bounds__(256) k_wide_fwd_t(Dev D, const int32_t *__restrict__ fronts, const double *Y1)
{
    __shared__ double part[8][33];
    int s = fronts[blockIdx.y];
    int ms = D.m[s], nc = D.ncol[s], nr = ms - nc;
    if (blockIdx.x * 32 >= nr) return;
    const double *F = D.F + D.front_off[s];
    const double *y1 = Y1 + D.idx_start[s];
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    int i = blockIdx.x * 32 + lane;
    double v = 0;
    if (i < nr)
        for (int k = warp; k < nc; k += 8) v += F[(int64_t)k * ms + nc + i] * y1[k];
    part[warp][lane] = v;
    __syncthreads();
    if (warp == 0 && i < nr) {
        double t = 0;
        for (int w = 0; w < 8; w++) t += part[w][lane];
        D.U[D.uvec_start[s] + i] = -D.Abig[D.idx_start[s] + nc + i] + t;
    }
}

// z = y1 - L21^T x2, one warp per pivot column.
static __global__ void __launch_bounds__(256) k_wide_bwd_z(Dev D, const int32_t *__restrict__ fronts, const double *x, double *Z)
{
    int s = fronts[blockIdx.y];
    int ms = D.m[s], nc = D.ncol[s], c0 = D.c0[s], nr = ms - nc;
    int k = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (k >= nc) return;
    const double *F = D.F + D.front_off[s];
    const int32_t *ix = D.idx + D.idx_start[s];
    int lane = threadIdx.x & 31;
    const double *col = F + (int64_t)k * ms + nc;
    double v = 0;
    for (int i = lane; i < nr; i += 32) v += col[i] * x[ix[nc + i]];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) Z[D.idx_start[s] + k] = x[c0 + k] - v;
}

// x1 = X^T z, one warp per pivot column j (column j of X is contiguous).
static __global__ void __launch_bounds__(256) k_wide_bwd_x(Dev D, const int32_t *__restrict__ fronts, const double *Z, double *x)
{
    int s = fronts[blockIdx.y];
    int nc = D.ncol[s], c0 = D.c0[s];
    int j = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    if (j >= nc) return;
    const double *X = D.Xinv + D.xinv_off[s];
    const double *z = Z + D.idx_start[s];
    int lane = threadIdx.x & 31;
    const double *col = X + (int64_t)j * nc;
    double v = 0;
    for (int i = j + lane; i < nc; i += 32) v += col[i] * z[i];
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if (lane == 0) x[c0 + j] = v;
}

// Trailing update of every listed front after panel k0: F22 -= L21 L21^T on 64x64 lower tiles, each thread a
// 4x4 register block (dynamic shared memory: two 64 x PW panels).
static __global__ void __launch_bounds__(256) k_update(Dev D, const int32_t *__restrict__ fronts, int k0)
{
    extern __shared__ double sh[];
    double (*Ai)[PW + 1] = (double (*)[PW + 1])sh;
    double (*Aj)[PW + 1] = (double (*)[PW + 1])(sh + UT * (PW + 1));
    int s = fronts[blockIdx.y];
    int ms = D.m[s], w = min(PW, D.ncol[s] - k0), r0 = k0 + w, nt = ms - r0;
    if (nt <= 0) return;
    double *F = D.F + D.front_off[s];
    int nti = (nt + UT - 1) / UT;
    int ntiles = nti * (nti + 1) / 2;
    int tx = threadIdx.x % 16, ty = threadIdx.x / 16;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        int ti = (int)((sqrt(8.0 * t + 1.0) - 1.0) * 0.5);
        while ((ti + 1) * (ti + 2) / 2 <= t) ti++;
        while (ti * (ti + 1) / 2 > t) ti--;
        int tj = t - ti * (ti + 1) / 2;
        int ri0 = r0 + ti * UT, cj0 = r0 + tj * UT;
        __syncthreads();
        for (int q = threadIdx.x; q < UT * w; q += blockDim.x) {
            int rr = q % UT, k = q / UT;
            int gi = ri0 + rr, gj = cj0 + rr;
            Ai[rr][k] = gi < ms ? F[(int64_t)(k0 + k) * ms + gi] : 0.0;
            Aj[rr][k] = gj < ms ? F[(int64_t)(k0 + k) * ms + gj] : 0.0;
        }
        __syncthreads();
        double acc[4][4];
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) acc[a][b] = 0.0;
        for (int k = 0; k < w; k++) {
            double ai[4], aj[4];
            for (int a = 0; a < 4; a++) ai[a] = Ai[tx + 16 * a][k];
            for (int b = 0; b < 4; b++) aj[b] = Aj[ty + 16 * b][k];
            for (int a = 0; a < 4; a++)
                for (int b = 0; b < 4; b++) acc[a][b] += ai[a] * aj[b];
        }
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                int gi = ri0 + tx + 16 * a, gj = cj0 + ty + 16 * b;
                if (gi < ms && gj < ms && gi >= gj) F[(int64_t)gj * ms + gi] -= acc[a][b];
            }
    }
}

static __global__ void k_init_err(int *err)
{
    err[0] = INT_MAX;
    err[1] = 0;
}

static __global__ void k_permute_in(int n, const int32_t *perm, const double *b, double *y)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) y[i] = b[perm[i]];
}
static __global__ void k_permute_out(int n, const int32_t *perm, const double *y, double *x)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) x[perm[i]] = y[i];
}

// Forward elimination of the fronts of one level: y(cols) and the update vector for the parent. Each 64-pivot
// block is applied through its stored inverse (one block GEMV) instead of 64 dependent steps.
static __global__ void __launch_bounds__(512) k_forward(Dev D, const int32_t *__restrict__ fronts, double *y)
{
    extern __shared__ double acc[];
    __shared__ double yb[PW];
    int s = fronts[blockIdx.x];
    int ms = D.m[s], nc = D.ncol[s], c0 = D.c0[s];
    const double *F = D.F + D.front_off[s];
    const double *Inv = D.Inv + D.inv_off[s];
    int tid = threadIdx.x, nt = blockDim.x, lane = tid & 31, warp = tid >> 5, nw = nt >> 5;
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
        const double *I = Inv + (int64_t)(kb / PW) * PW * PW;
        // y_blk = Linv acc_blk (warp per output row, coalesced over the inverse's columns? rows: I[c*PW + i])
        for (int i = warp; i < w; i += nw) {
            double v = 0;
            for (int c = lane; c <= i; c += 32) v += I[(int64_t)c * PW + i] * acc[kb + c];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) yb[i] = v;
        }
        __syncthreads();
        for (int i = tid; i < w; i += nt) acc[kb + i] = yb[i];
        // rows below the block
        for (int r = kb + w + tid; r < ms; r += nt) {
            double v = acc[r];
            for (int k = 0; k < w; k++) v -= F[(int64_t)(kb + k) * ms + r] * yb[k];
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
    __shared__ double xb[PW];
    int s = fronts[blockIdx.x];
    int ms = D.m[s], nc = D.ncol[s], c0 = D.c0[s], nr = ms - nc;
    const double *F = D.F + D.front_off[s];
    const double *Inv = D.Inv + D.inv_off[s];
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
        // x_blk = Linv^T acc_blk: x_j = sum_{i >= j} Linv[i][j] acc_i (column j of the inverse is contiguous)
        const double *I = Inv + (int64_t)bi * PW * PW;
        for (int j = warp; j < w; j += nw) {
            double v = 0;
            for (int i = j + lane; i < w; i += 32) v += I[(int64_t)j * PW + i] * acc[kb + i];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) xb[j] = v;
        }
        __syncthreads();
        for (int j = tid; j < w; j += nt) acc[kb + j] = xb[j];
        __syncthreads();
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
        cuda_check(cudaStreamCreateWithFlags(&cap_, cudaStreamNonBlocking), "cudaStreamCreate");
        for (auto &e : ev_) cuda_check(cudaEventCreate(&e), "cudaEventCreate");
    }
    ~MfSolver()
    {
        drop_graphs();
        for (auto &e : ev_)
            if (e) cudaEventDestroy(e);
        if (cap_) cudaStreamDestroy(cap_);
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
    int big_fronts() const { return (int)big_list_.size(); }
    double factor_ms() const { return factor_ms_; }
    double solve_ms() const { return solve_ms_; }
    int64_t solves() const { return n_solves_; }
    void set_profile(bool p) { profile_ = p; }
    int n() const { return sym_.n; }

    void analyze(int n, const int32_t *col_ptr, const int32_t *row_idx, int block)
    {
        analyzed_ = factored_ = false;
        drop_graphs();
        std::string e = sym_.analyze(n, col_ptr, row_idx, block, hsp_, descr_);
        if (!e.empty()) throw Failure(IFEA_INPUT_INVALID, e);
        const MfSymbolic &S = sym_;

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
        inv_off_.assign(S.nsuper, 0);
        int64_t inv_total = 0;
        for (int q = 0; q < S.nsuper; q++) {
            inv_off_[q] = inv_total;
            inv_total += (int64_t)((S.ncol[q] + mf::PW - 1) / mf::PW) * mf::PW * mf::PW;
        }
        d_inv_off_.upload(inv_off_, st_);
        d_Inv_.resize(std::max<int64_t>(inv_total, 1));
        // big supernodes: full inverse of the pivot block and multi-CTA solves; small ones: batched per level
        xinv_off_.assign(S.nsuper, -1);
        int64_t xinv_total = 0;
        int max_small_m = 1;
        small_start_.assign(S.nlevels + 1, 0);
        small_list_.clear();
        big_start_.assign(S.nlevels + 1, 0);
        big_list_.clear();
        for (int l = 0; l < S.nlevels; l++) {
            small_start_[l] = (int32_t)small_list_.size();
            big_start_[l] = (int32_t)big_list_.size();
            for (int32_t q = S.level_start[l]; q < S.level_start[l + 1]; q++) {
                int sn = S.level_list[q];
                if (S.m[sn] >= mf::kWideM) {
                    big_list_.push_back(sn);
                    xinv_off_[sn] = xinv_total;
                    xinv_total += (int64_t)S.ncol[sn] * S.ncol[sn];
                } else {
                    small_list_.push_back(sn);
                    max_small_m = std::max(max_small_m, S.m[sn]);
                }
            }
        }
        small_start_[S.nlevels] = (int32_t)small_list_.size();
        big_start_[S.nlevels] = (int32_t)big_list_.size();
        for (int l = 0; l < S.nlevels; l++)
            std::stable_sort(big_list_.begin() + big_start_[l], big_list_.begin() + big_start_[l + 1],
                             [&](int a, int b) { return S.ncol[a] > S.ncol[b]; });
        d_big_.upload(big_list_, st_);
        d_small_.upload(small_list_, st_);
        d_xinv_off_.upload(xinv_off_, st_);
        d_Xinv_.resize(std::max<int64_t>(xinv_total, 1));
        d_Abig_.resize(S.idx_start[S.nsuper]);
        d_y1_.resize(S.idx_start[S.nsuper]);
        d_z_.resize(S.idx_start[S.nsuper]);
        small_smem_ = (size_t)max_small_m * sizeof(double);
        d_F_.resize(S.pool);
        d_U_.resize(std::max<int64_t>(S.uvec_pool, 1));
        d_y_.resize(n);
        dev_.ncol = d_ncol_; dev_.m = d_m_; dev_.c0 = d_c0_; dev_.idx_start = d_idxs_; dev_.idx = d_idx_;
        dev_.relmap_start = d_rms_; dev_.relmap = d_rm_; dev_.uvec_start = d_uvs_; dev_.child_start = d_cs_;
        dev_.child_list = d_cl_; dev_.front_off = d_off_; dev_.F = d_F_; dev_.U = d_U_;
        dev_.inv_off = d_inv_off_; dev_.Inv = d_Inv_; dev_.xinv_off = d_xinv_off_; dev_.Xinv = d_Xinv_;
        dev_.Abig = d_Abig_;
        cuda_check(cudaFuncSetAttribute((const void *)mf::k_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kUpdateSmem), "cudaFuncSetAttribute");
        cuda_check(cudaFuncSetAttribute((const void *)mf::k_panel_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kPairSmem), "cudaFuncSetAttribute");
        cuda_check(cudaFuncSetAttribute((const void *)mf::k_inverse_row, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                        (int)kPairSmem), "cudaFuncSetAttribute");
        if (small_smem_ > 200 * 1024) throw Failure(IFEA_INPUT_INVALID, "front larger than the solve kernels' shared-memory window");
        cuda_check(cudaFuncSetAttribute((const void *)mf::k_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)small_smem_), "cudaFuncSetAttribute");
        cuda_check(cudaFuncSetAttribute((const void *)mf::k_backward, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)small_smem_), "cudaFuncSetAttribute");
        cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
        analyzed_ = true;
    }

    // Numeric factorisation of device values in the order of the analysed full CSC pattern. The launch sequence
    // depends only on the pattern, so it is captured once (per values buffer) as a CUDA graph and replayed.
    void factorize(const double *d_full_vals)
    {
        if (!analyzed_) throw Failure(IFEA_BAD_STATE, "Analyze must be called first.");
        factored_ = false;
        const MfSymbolic &S = sym_;
        if (!factor_exec_ || factor_vals_ != d_full_vals) {
            if (factor_exec_) cudaGraphExecDestroy(factor_exec_);
            factor_exec_ = nullptr;
            cudaGraph_t g = nullptr;
            cuda_check(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            enqueue_factor(cap_, d_full_vals);
            cuda_check(cudaStreamEndCapture(cap_, &g), "cudaStreamEndCapture");
            cudaError_t e = cudaGraphInstantiate(&factor_exec_, g, 0);
            cudaGraphDestroy(g);
            cuda_check(e, "cudaGraphInstantiate");
            factor_vals_ = d_full_vals;
        }
        cuda_check(cudaEventRecord(ev_[0], st_), "cudaEventRecord");
        cuda_check(cudaGraphLaunch(factor_exec_, st_), "cudaGraphLaunch");
        cuda_check(cudaEventRecord(ev_[1], st_), "cudaEventRecord");
        int32_t e[2];
        cuda_check(cudaMemcpyAsync(e, d_err_.p, sizeof e, cudaMemcpyDeviceToHost, st_), "D2H");
        cuda_check(cudaStreamSynchronize(st_), "cudaStreamSynchronize");
        float ms = 0;
        if (cudaEventElapsedTime(&ms, ev_[0], ev_[1]) == cudaSuccess) factor_ms_ += ms;
        if (e[0] != INT_MAX) {
            int row = S.perm[e[0]];
            throw Failure(IFEA_NOT_SPD, "Stiffness matrix not positive definite at equation " + std::to_string(row) +
                                            ". The billet is probably unrestrained.");
        }
        factored_ = true;
    }

    void enqueue_factor(cudaStream_t st, const double *d_full_vals)
    {
        const MfSymbolic &S = sym_;
        mf::k_init_err<<<1, 1, 0, st>>>(d_err_);
        for (int l = 0; l < S.nlevels; l++) {
            int64_t p0 = S.level_pool_start[l], p1 = S.level_pool_start[l + 1];
            cuda_check(cudaMemsetAsync(d_F_.p + p0, 0, (size_t)(p1 - p0) * sizeof(double), st), "memset fronts");
            int64_t a0 = S.a_level_start[l], a1 = S.a_level_start[l + 1];
            if (a1 > a0) {
                int g = (int)std::min<int64_t>((a1 - a0 + 255) / 256, 4 * 148);
                mf::k_scatter<<<g, 256, 0, st>>>(a1 - a0, d_adst_.p + a0, d_asrc_.p + a0, d_full_vals, d_F_);
            }
            for (int r = 0; r < S.max_rank; r++) {
                int32_t e0 = S.ext_start[(size_t)l * S.max_rank + r], e1 = S.ext_start[(size_t)l * S.max_rank + r + 1];
                if (e1 <= e0) continue;
                dim3 grid(64, e1 - e0);
                mf::k_extend<<<grid, 128, 0, st>>>(dev_, d_ext_.p + e0, d_par_);
            }
            int q0 = S.level_start[l], q1 = S.level_start[l + 1];
            int maxc = S.ncol[lvl_sorted_[q0]];
            for (int k0 = 0; k0 < maxc; k0 += mf::PW) {
                int cnt = 0, maxt = 0, maxr = 0;
                for (int q = q0; q < q1 && S.ncol[lvl_sorted_[q]] > k0; q++) {
                    int sn = lvl_sorted_[q];
                    cnt++;
                    int w = std::min(mf::PW, S.ncol[sn] - k0), nt = S.m[sn] - k0 - w;
                    int nti = (nt + mf::UT - 1) / mf::UT;
                    maxt = std::max(maxt, nti * (nti + 1) / 2);
                    maxr = std::max(maxr, (nt + mf::PW - 1) / mf::PW);
                }
                mf::k_panel<<<cnt, 256, 0, st>>>(dev_, d_lvl_.p + q0, k0, d_err_);
                if (maxr > 0) mf::k_panel_trsm<<<dim3(maxr, cnt), 256, kPairSmem, st>>>(dev_, d_lvl_.p + q0, k0);
                if (maxt > 0) {
                    dim3 grid(std::min(maxt, 4096), cnt);
                    mf::k_update<<<grid, 256, kUpdateSmem, st>>>(dev_, d_lvl_.p + q0, k0);
                }
            }
            int b0 = big_start_[l], b1 = big_start_[l + 1];
            if (b1 > b0) {
                int nbmax = (S.ncol[big_list_[b0]] + mf::PW - 1) / mf::PW;
                for (int bi = 0; bi < nbmax; bi++) {
                    int cnt = 0;
                    while (b0 + cnt < b1 && (S.ncol[big_list_[b0 + cnt]] + mf::PW - 1) / mf::PW > bi) cnt++;
                    mf::k_inverse_row<<<dim3(bi + 1, cnt), 256, kPairSmem, st>>>(dev_, d_big_.p + b0, bi);
                }
            }
        }
        cuda_check(cudaGetLastError(), "multifrontal factorisation launch");
    }

    // x = A^-1 b on the device (b and x may alias). The level sweeps run as one captured CUDA graph on the
    // solver's internal vector; only the permutations in and out are launched per call.
    void solve(const double *d_b, double *d_x)
    {
        if (!factored_) throw Failure(IFEA_BAD_STATE, "Factorize must be called first.");
        const MfSymbolic &S = sym_;
        int n = S.n, g = std::max(1, std::min((n + 255) / 256, 4 * 148));
        if (!solve_exec_) {
            cudaGraph_t gr = nullptr;
            cuda_check(cudaStreamBeginCapture(cap_, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
            enqueue_sweeps(cap_);
            cuda_check(cudaStreamEndCapture(cap_, &gr), "cudaStreamEndCapture");
            cudaError_t e = cudaGraphInstantiate(&solve_exec_, gr, 0);
            cudaGraphDestroy(gr);
            cuda_check(e, "cudaGraphInstantiate");
        }
        if (profile_) cuda_check(cudaEventRecord(ev_[2], st_), "cudaEventRecord");
        mf::k_permute_in<<<g, 256, 0, st_>>>(n, d_perm_, d_b, d_y_);
        cuda_check(cudaGraphLaunch(solve_exec_, st_), "cudaGraphLaunch");
        mf::k_permute_out<<<g, 256, 0, st_>>>(n, d_perm_, d_y_, d_x);
        n_solves_++;
        if (profile_) {
            cuda_check(cudaEventRecord(ev_[3], st_), "cudaEventRecord");
            cuda_check(cudaEventSynchronize(ev_[3]), "cudaEventSynchronize");
            float ms = 0;
            if (cudaEventElapsedTime(&ms, ev_[2], ev_[3]) == cudaSuccess) solve_ms_ += ms;
        }
        cuda_check(cudaGetLastError(), "multifrontal solve launch");
    }

    void enqueue_sweeps(cudaStream_t st)
    {
        const MfSymbolic &S = sym_;
        for (int l = 0; l < S.nlevels; l++) {
            int q0 = small_start_[l], cnt = small_start_[l + 1] - q0;
            if (cnt > 0) mf::k_forward<<<cnt, 512, small_smem_, st>>>(dev_, d_small_.p + q0, d_y_);
            int b0 = big_start_[l], bc = big_start_[l + 1] - b0;
            if (bc > 0) {
                int mnc = 1, mnr = 1;
                for (int q = b0; q < b0 + bc; q++) {
                    mnc = std::max(mnc, S.ncol[big_list_[q]]);
                    mnr = std::max(mnr, S.m[big_list_[q]] - S.ncol[big_list_[q]]);
                }
                mf::k_wide_fwd_acc<<<bc, 512, 0, st>>>(dev_, d_big_.p + b0, d_y_);
                mf::k_wide_fwd_y<<<dim3((mnc + 31) / 32, bc), 256, 0, st>>>(dev_, d_big_.p + b0, d_y_, d_y1_);
                mf::k_wide_fwd_t<<<dim3((mnr + 31) / 32, bc), 256, 0, st>>>(dev_, d_big_.p + b0, d_y1_);
            }
        }
        for (int l = S.nlevels - 1; l >= 0; l--) {
            int q0 = small_start_[l], cnt = small_start_[l + 1] - q0;
            if (cnt > 0) mf::k_backward<<<cnt, 512, small_smem_, st>>>(dev_, d_small_.p + q0, d_y_, d_y_);
            int b0 = big_start_[l], bc = big_start_[l + 1] - b0;
            if (bc > 0) {
                int mnc = S.ncol[big_list_[b0]];
                mf::k_wide_bwd_z<<<dim3((mnc + 7) / 8, bc), 256, 0, st>>>(dev_, d_big_.p + b0, d_y_, d_z_);
                mf::k_wide_bwd_x<<<dim3((mnc + 7) / 8, bc), 256, 0, st>>>(dev_, d_big_.p + b0, d_z_, d_y_);
            }
        }
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
    void drop_graphs()
    {
        if (solve_exec_) cudaGraphExecDestroy(solve_exec_);
        if (factor_exec_) cudaGraphExecDestroy(factor_exec_);
        solve_exec_ = factor_exec_ = nullptr;
        factor_vals_ = nullptr;
    }
    cudaEvent_t ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    double factor_ms_ = 0, solve_ms_ = 0;
    int64_t n_solves_ = 0;
    bool profile_ = false;
    cudaStream_t cap_ = nullptr;
    cudaGraphExec_t solve_exec_ = nullptr, factor_exec_ = nullptr;
    const double *factor_vals_ = nullptr;
    static constexpr size_t kUpdateSmem = 2 * mf::UT * (mf::PW + 1) * sizeof(double);
    static constexpr size_t kPairSmem = 2 * mf::PW * (mf::PW + 1) * sizeof(double);
    cudaStream_t st_;
    cusolverSpHandle_t hsp_ = nullptr;
    std::vector<int64_t> inv_off_, xinv_off_;
    std::vector<int32_t> small_start_, small_list_, big_start_, big_list_;
    size_t small_smem_ = 8;
    DBuf<int64_t> d_inv_off_, d_xinv_off_;
    DBuf<int32_t> d_small_, d_big_;
    DBuf<double> d_Inv_, d_Xinv_, d_Abig_, d_y1_, d_z_;
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
