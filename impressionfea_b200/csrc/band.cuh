// band.cuh — SymmetricBandMatrix.Factorize + Solve (Solver/SymmetricBandMatrix.cs:60-111) in one CTA, blocked.
//
// The band is stored row-major, row i holding L[i][i-b .. i] at offsets 0 .. b (diagonal last). The reference's
// factorisation subtracts, for every entry (i, j), the products L_ik L_jk in ascending k, each product rounded
// before the subtraction, then divides by L_jj (or takes the square root on the diagonal); its solves subtract
// in ascending k (forward) and descending i (backward). Any schedule that keeps that order per entry gives the
// same bits, so the factorisation here is blocked by panels of nb columns:
//
//   A  panel factorisation: column by column inside the panel (scale, update of the panel's later columns,
//      pivot), the panel's entries held in registers (each thread some rows of one column), two barriers per
//      column;
//   B  trailing update of the rows below the panel by the whole panel: 4 x 4 register tiles, each entry's nb
//      products subtracted in ascending k (one shared-memory load per two multiplies);
//   C  the forward substitution of the panel's rows and its update of the b rows below, by one warp, while the
//      other warps run B;
//   D  the panel's rows are final: written back to global memory, and their window slots refilled (cp.async)
//      with rows W further on, which a panel two steps later first needs.
//
// The backward substitution then walks the rows in blocks of nb from the bottom: one warp solves the block's
// triangle, all threads update the b rows above it (products in descending i), the block's slots are refilled
// with rows W lower. Rows live in a circular window of W = 2 nb + b rows in shared memory (row i in slot i mod
// W); a band too wide for that window is factorised in place in global memory by the same code.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <type_traits>

namespace ifea {
namespace band {

constexpr int kThreads = 512;
constexpr int kMaxSmem = 200 * 1024;
constexpr int kOwn = 10;          // panel entries a thread keeps in registers
constexpr int kStageRows = 256;   // panel rows the register path takes

struct Plan {
    int nb = 32, W = 0;
    bool smem = true;
    size_t bytes = 0;  // dynamic shared memory of the launch
};

// Panel width and window for an n x n band of half-bandwidth b. Window W = 2 nb + b rows of b + 1 doubles and their
// right-hand-side entries; widest panel that fits, else the band stays in global memory (window = the band).
inline Plan plan(int n, int b)
{
    Plan p;
    size_t w = (size_t)b + 1;
    for (int nb : {32, 16, 8}) {
        int W = (int)std::min<int64_t>((int64_t)n, 2 * (int64_t)nb + b);
        size_t bytes = (size_t)W * (w + 1) * sizeof(double) + (size_t)(2 * nb + b) * sizeof(int64_t);
        if (bytes <= (size_t)kMaxSmem) {
            p.nb = nb;
            p.W = W;
            p.bytes = bytes;
            p.smem = true;
            return p;
        }
    }
    p.nb = 32;
    p.W = n;
    p.smem = false;
    p.bytes = (size_t)(2 * 32 + b) * sizeof(int64_t);  // the row-offset table only
    return p;
}

__device__ __forceinline__ void cp8(double *dst, const double *src)
{
    unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(src) : "memory");
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
__device__ __forceinline__ void cp_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// err_row[0] = -1 on success, else the first row whose pivot was not positive; pivot[0] that pivot.
template <bool SMEM>
__global__ void __launch_bounds__(kThreads) k_band_chol(int n, int b, int nb, int W, double *__restrict__ a,
                                                        double *__restrict__ rhs, int32_t *err_row, double *pivot)
{
    using Off = typename std::conditional<SMEM, int, int64_t>::type;
    extern __shared__ __align__(16) unsigned char band_smem[];
    __shared__ int s_bad;
    __shared__ double xs[32];
    __shared__ double lcol[kStageRows], stage[kStageRows];  // the scaled column kk; the updated column kk + 1
    const int w = b + 1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned FULL = 0xffffffffu;
    // layout: row-offset table (2 nb + b entries) | window rows (W x w) | window right-hand side (W)
    int64_t *rowoff_base = (int64_t *)band_smem;
    double *win, *rv;
    if constexpr (SMEM) {
        win = (double *)(band_smem + (size_t)(2 * nb + b) * sizeof(int64_t));
        rv = win + (size_t)W * w;
    } else {
        win = a;
        rv = rhs;
    }
    auto slot = [&](int i) -> Off { return SMEM ? (Off)(i % W) : (Off)i; };
    // entry (i, j) of a resident row, j in [i - b, i]
    auto E = [&](int i, int j) -> double & { return win[slot(i) * (Off)w + (j - i + b)]; };
    auto RV = [&](int i) -> double & { return rv[slot(i)]; };
    // rows [r0, r1) of the band (and of the right-hand side) into their window slots, asynchronously
    auto fetch = [&](int r0, int r1) {
        if constexpr (SMEM) {
            r0 = max(r0, 0);
            r1 = min(r1, n);
            if (r1 <= r0) return;
            int64_t cnt = (int64_t)(r1 - r0) * w;
            for (int64_t t = tid; t < cnt; t += kThreads) {
                int i = r0 + (int)(t / w), c = (int)(t % w);
                cp8(win + (size_t)(i % W) * w + c, a + (size_t)i * w + c);
            }
            if (rhs)
                for (int i = r0 + tid; i < r1; i += kThreads) cp8(rv + (i % W), rhs + i);
            cp_commit();
        }
    };
    // rows [r0, r1) are final: back to global memory
    auto retire = [&](int r0, int r1, bool rows) {
        if constexpr (SMEM) {
            if (rows) {
                int64_t cnt = (int64_t)(r1 - r0) * w;
                for (int64_t t = tid; t < cnt; t += kThreads) {
                    int i = r0 + (int)(t / w), c = (int)(t % w);
                    a[(size_t)i * w + c] = win[(size_t)(i % W) * w + c];
                }
            }
            if (rhs)
                for (int i = r0 + tid; i < r1; i += kThreads) rhs[i] = rv[i % W];
        }
    };
    auto do_pivot = [&](int k) {
        double s = E(k, k);
        if (!(s > 0) || isnan(s)) {
            s_bad = k;
            *pivot = s;
        } else {
            E(k, k) = sqrt(s);
        }
    };

    if (tid == 0) {
        s_bad = -1;
        *pivot = 0.0;
    }
    if constexpr (SMEM) {
        int r1 = min(n, W);
        for (int64_t t = tid; t < (int64_t)r1 * w; t += kThreads) win[t] = a[t];
        if (rhs)
            for (int i = tid; i < r1; i += kThreads) rv[i] = rhs[i];
    }
    __syncthreads();

    Off *rowoff = (Off *)rowoff_base;  // rowoff[t]: offset of E(k0 + t, 0) in win (may be negative)
    for (int k0 = 0; k0 < n; k0 += nb) {
        const int k1 = min(n, k0 + nb);
        const int last = min(n - 1, k1 - 1 + b);  // last row the panel's columns reach
        for (int t = tid; t <= last - k0; t += kThreads) {
            int i = k0 + t;
            rowoff[t] = slot(i) * (Off)w - i + b;
        }
        if (tid == 0) do_pivot(k0);
        __syncthreads();
        if (s_bad >= 0) break;
        auto P = [&](int i, int j) -> double & { return win[rowoff[i - k0] + j]; };

        // A: the panel's columns. Rows r = 0 .. R - 1 of the panel (relative to k0); with the window in shared
        // memory and at most kOwn rows per thread, every thread keeps the entries of one panel column (ct) in
        // registers, rows rt, rt + step, ..., and a column step is: scale column kk (one row per thread, into
        // the window and lcol), barrier, each thread subtracts column kk's products from its entries (the owners
        // of column kk + 1 then hand it to stage[] and its pivot is taken), barrier.
        const int np = k1 - k0, R = last - k0 + 1;
        const int lg = nb == 32 ? 5 : nb == 16 ? 4 : 3, step = kThreads >> lg;
        if (SMEM && R <= kStageRows && (R + step - 1) / step <= kOwn && (1 << lg) == nb) {
            const int ct = tid & (nb - 1), rt = tid >> lg;
            double v[kOwn];
#pragma unroll
            for (int u = 0; u < kOwn; u++) {
                int r = rt + u * step;
                v[u] = (r < R && ct < np && r >= ct && r - ct <= b) ? P(k0 + r, k0 + ct) : 0.0;
            }
            for (int kk = 0; kk < np; kk++) {
                const int k = k0 + kk;
                const double lkk = P(k, k);
                for (int r = tid; r < R; r += kThreads)
                    if (r > kk && r - kk <= b) {
                        double l = (kk == 0 ? P(k0 + r, k) : stage[r]) / lkk;
                        lcol[r] = l;
                        P(k0 + r, k) = l;
                    }
                __syncthreads();
                if (ct > kk && ct < np) {
                    const double ljk = lcol[ct];
#pragma unroll
                    for (int u = 0; u < kOwn; u++) {
                        int r = rt + u * step;
                        if (r < R && r >= ct && r <= kk + b) v[u] = v[u] - lcol[r] * ljk;
                    }
                    if (ct == kk + 1) {
#pragma unroll
                        for (int u = 0; u < kOwn; u++) {
                            int r = rt + u * step;
                            if (r < R && r >= ct && r - ct <= b) {
                                if (r == ct) {
                                    P(k0 + r, k0 + r) = v[u];
                                    do_pivot(k0 + r);  // (kk + 1, kk + 1) is final now
                                } else {
                                    stage[r] = v[u];
                                }
                            }
                        }
                    }
                }
                __syncthreads();
                if (s_bad >= 0) break;
            }
        } else {
            // column by column with every entry in the window (bands too wide for the register path)
            for (int k = k0; k < k1; k++) {
                const double lkk = P(k, k);
                const int r = min(n - 1, k + b);
                for (int i = k + 1 + tid; i <= r; i += kThreads) P(i, k) = P(i, k) / lkk;
                __syncthreads();
                const int c = k1 - 1 - k, rows = r - k;
                for (int idx = tid; idx < c * rows; idx += kThreads) {
                    int di = idx / c, dj = idx - di * c;
                    int i = k + 1 + di, j = k + 1 + dj;
                    if (j <= i) {
                        double &e = P(i, j);
                        e = e - P(i, k) * P(j, k);
                        if (idx == 0) do_pivot(k + 1);  // (k + 1, k + 1) is final now
                    }
                }
                __syncthreads();
                if (s_bad >= 0) break;
            }
        }
        if (s_bad >= 0) break;

        // B on all warps but the last, C on the last warp (when there is a right-hand side)
        const int nbw = rhs ? kThreads - 32 : kThreads;
        if (tid < nbw) {
            const int m = last - k1 + 1;  // rows below the panel
            const int T = (m + 3) >> 2;
            const int pairs = ((T + 1) >> 1) * (T + 1);
            for (int idx = tid; idx < pairs; idx += nbw) {
                int q = idx / (T + 1), cc = idx - q * (T + 1);
                int ti, tj;
                if (cc <= q) {
                    ti = q;
                    tj = cc;
                } else {
                    ti = T - 1 - q;
                    tj = cc - q - 1;
                    if (ti == q) continue;  // the middle tile row of an odd count is covered by the first branch
                }
                const int ib = k1 + 4 * ti, jb = k1 + 4 * tj;
                Off pi[4], pj[4];
                int kf[4];
                bool iv[4], jv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    int i = ib + u, j = jb + u;
                    iv[u] = i <= last;
                    jv[u] = j <= last;
                    pi[u] = iv[u] ? rowoff[i - k0] : 0;
                    pj[u] = jv[u] ? rowoff[j - k0] : 0;
                    kf[u] = max(k0, i - b);
                }
                double s[4][4];
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++) s[u][v] = (iv[u] && jb + v <= ib + u) ? win[pi[u] + jb + v] : 0.0;
                for (int k = kf[0]; k < k1; k++) {
                    double li[4], lj[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        li[u] = (iv[u] && k >= kf[u]) ? win[pi[u] + k] : 0.0;
                        lj[u] = (jv[u] && k >= jb + u - b) ? win[pj[u] + k] : 0.0;
                    }
#pragma unroll
                    for (int u = 0; u < 4; u++)
#pragma unroll
                        for (int v = 0; v < 4; v++)
                            if (k >= kf[u]) s[u][v] = s[u][v] - li[u] * lj[v];
                }
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++)
                        if (iv[u] && jb + v <= ib + u) win[pi[u] + jb + v] = s[u][v];
            }
        } else {
            // C: forward substitution of rows [k0, k1), then their products out of the rows below
            const int np = k1 - k0;
            double y = lane < np ? RV(k0 + lane) : 0.0;
            for (int kk = 0; kk < np; kk++) {
                if (lane == kk) y = y / P(k0 + kk, k0 + kk);
                double xk = __shfl_sync(FULL, y, kk);
                if (lane > kk && lane < np && lane - kk <= b) y = y - P(k0 + lane, k0 + kk) * xk;
            }
            if (lane < np) {
                RV(k0 + lane) = y;
                xs[lane] = y;
            }
            __syncwarp();
            for (int i = k1 + lane; i <= last; i += 32) {
                double rr = RV(i);
                for (int k = max(k0, i - b); k < k1; k++) rr = rr - P(i, k) * xs[k - k0];
                RV(i) = rr;
            }
        }
        __syncthreads();
        // D: rows [k0, k1) are final
        retire(k0, k1, true);
        if constexpr (SMEM) cp_wait_all();
        __syncthreads();
        fetch(k0 + W, k1 + W);
    }
    if constexpr (SMEM) cp_wait_all();
    __syncthreads();
    if (s_bad >= 0) {
        if (tid == 0) *err_row = s_bad;
        return;
    }
    if (tid == 0) *err_row = -1;
    if (!rhs) return;

    // backward substitution, blocks of nb rows from the bottom; rows [n - W, n) are still resident
    for (int i1 = n; i1 > 0;) {
        const int i0 = max(0, i1 - nb);
        const int np = i1 - i0;
        if (warp == 0) {
            double y = lane < np ? RV(i0 + lane) : 0.0;
            for (int kk = np - 1; kk >= 0; kk--) {
                const int i = i0 + kk;
                if (lane == kk) y = y / E(i, i);
                double xi = __shfl_sync(FULL, y, kk);
                if (lane < kk && kk - lane <= b) y = y - E(i, i0 + lane) * xi;
            }
            if (lane < np) {
                RV(i0 + lane) = y;
                xs[lane] = y;
            }
        }
        __syncthreads();
        for (int k = max(0, i0 - b) + tid; k < i0; k += kThreads) {
            double rr = RV(k);
            for (int i = min(i1 - 1, k + b); i >= i0; i--) rr = rr - E(i, k) * xs[i - i0];
            RV(k) = rr;
        }
        __syncthreads();
        retire(i0, i1, false);
        if constexpr (SMEM) cp_wait_all();
        __syncthreads();
        fetch(i0 - W, i1 - W);
        i1 = i0;
    }
    if constexpr (SMEM) cp_wait_all();
}

// Launch on `st` with the plan for (n, b); the caller has raised the kernel's shared-memory limit to plan.bytes.
inline void launch(const Plan &p, int n, int b, double *a, double *rhs, int32_t *err_row, double *pivot,
                   cudaStream_t st)
{
    if (p.smem)
        k_band_chol<true><<<1, kThreads, p.bytes, st>>>(n, b, p.nb, p.W, a, rhs, err_row, pivot);
    else
        k_band_chol<false><<<1, kThreads, p.bytes, st>>>(n, b, p.nb, p.W, a, rhs, err_row, pivot);
}

inline const void *kernel_of(const Plan &p)
{
    return p.smem ? (const void *)k_band_chol<true> : (const void *)k_band_chol<false>;
}

}  // namespace band
}  // namespace ifea
