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
constexpr int kBlkRows = 4;       // rows of 32 per lane in the eight-column block factorisation
constexpr int kStageRows = 256;   // panel rows the register path takes

struct Plan {
    int nb = 32, W = 0;
    bool smem = true;
    size_t bytes = 0;  // dynamic shared memory of the launch
};

// Panel width and window for an n x n band of half-bandwidth b. Window W = 2 nb + b rows of b + 1 doubles (padded
// to an odd count) and their right-hand-side entries; widest panel that fits, else the band stays in global
// memory (window = the band).
inline Plan plan(int n, int b)
{
    Plan p;
    size_t w = (size_t)b + 1;
    for (int nb : {32, 16, 8}) {
        int W = (int)std::min<int64_t>((int64_t)n, 2 * (int64_t)nb + b);
        size_t bytes = (size_t)W * ((w | 1) + 1) * sizeof(double) + (size_t)(2 * nb + b) * sizeof(int64_t);
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
    __shared__ typename std::conditional<SMEM, int, int64_t>::type brow[32];  // row offsets of a backward block
    const int w = b + 1;
    // window rows are an odd number of doubles apart, so that a warp reading one column of consecutive rows
    // touches distinct banks (the band in global memory keeps its stride w)
    const int ws = SMEM ? (w | 1) : w;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const unsigned FULL = 0xffffffffu;
    // layout: row-offset table (2 nb + b entries) | window rows (W x w) | window right-hand side (W)
    int64_t *rowoff_base = (int64_t *)band_smem;
    double *win, *rv;
    if constexpr (SMEM) {
        win = (double *)(band_smem + (size_t)(2 * nb + b) * sizeof(int64_t));
        rv = win + (size_t)W * ws;
    } else {
        win = a;
        rv = rhs;
    }
    auto slot = [&](int i) -> Off { return SMEM ? (Off)(i % W) : (Off)i; };
    // entry (i, j) of a resident row, j in [i - b, i]
    auto E = [&](int i, int j) -> double & { return win[slot(i) * (Off)ws + (j - i + b)]; };
    auto RV = [&](int i) -> double & { return rv[slot(i)]; };
    // rows [r0, r1) of the band (and of the right-hand side) into their window slots, asynchronously
    auto fetch = [&](int r0, int r1) {
        if constexpr (SMEM) {
            r0 = max(r0, 0);
            r1 = min(r1, n);
            if (r1 <= r0) return;
            // a warp per row, a lane per entry
            for (int i = r0 + warp; i < r1; i += kThreads / 32) {
                double *d = win + (size_t)(i % W) * ws;
                const double *g = a + (size_t)i * w;
                for (int c = lane; c < w; c += 32) cp8(d + c, g + c);
            }
            if (rhs)
                for (int i = r0 + tid; i < r1; i += kThreads) cp8(rv + (i % W), rhs + i);
            cp_commit();
        }
    };
    // rows [r0, r1) are final: back to global memory
    auto retire = [&](int r0, int r1, bool rows) {
        if constexpr (SMEM) {
            if (rows)
                for (int i = r0 + warp; i < r1; i += kThreads / 32) {
                    const double *d = win + (size_t)(i % W) * ws;
                    double *g = a + (size_t)i * w;
                    for (int c = lane; c < w; c += 32) g[c] = d[c];
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
        for (int i = warp; i < r1; i += kThreads / 32)
            for (int c = lane; c < w; c += 32) win[(size_t)i * ws + c] = a[(size_t)i * w + c];
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
            rowoff[t] = slot(i) * (Off)ws - i + b;
        }
        const int np = k1 - k0, R = last - k0 + 1;  // panel columns; panel rows (relative to k0)
        const bool blocked = SMEM && R <= 32 * kBlkRows;
        if (!blocked && tid == 0) do_pivot(k0);
        __syncthreads();
        if (s_bad >= 0) break;
        auto P = [&](int i, int j) -> double & { return win[rowoff[i - k0] + j]; };

        // A: the panel's columns, in blocks of eight when the panel has at most 32 kBlkRows rows: warp 0 factors
        // a block in registers (lane l holds rows J + l + 32 q of its eight columns; pivots and column entries
        // travel by shuffles), barrier, every warp subtracts the block's products from the panel's later columns
        // (one column per lane, rows split over the warps), barrier.
        const int lg = nb == 32 ? 5 : nb == 16 ? 4 : 3, step = kThreads >> lg;
        if (blocked) {
            for (int J = 0; J < np; J += 8) {
                const int nc = min(8, np - J);
                if (warp == 0) {
                    double v[kBlkRows][8];
#pragma unroll
                    for (int q = 0; q < kBlkRows; q++)
#pragma unroll
                        for (int cc = 0; cc < 8; cc++) {
                            int r = J + lane + 32 * q, c = J + cc;
                            v[q][cc] = (cc < nc && r < R && r >= c && r - c <= b) ? P(k0 + r, k0 + c) : 0.0;
                        }
                    bool bad = false;
#pragma unroll
                    for (int cc = 0; cc < 8; cc++) {
                        if (bad || cc >= nc) continue;  // warp-uniform
                        const int c = J + cc;
                        const double piv = __shfl_sync(FULL, v[0][cc], cc);  // row c sits on lane cc
                        if (!(piv > 0) || isnan(piv)) {
                            if (lane == 0) {
                                s_bad = k0 + c;
                                *pivot = piv;
                            }
                            bad = true;
                            continue;
                        }
                        const double lkk = sqrt(piv);
                        if (lane == cc) v[0][cc] = lkk;
                        // the quotients for every lane and row (no branch around the divisions, which would
                        // serialise them), kept where the row belongs to column c's band
#pragma unroll
                        for (int q = 0; q < kBlkRows; q++) {
                            int r = J + lane + 32 * q;
                            const double qv = v[q][cc] / lkk;
                            if (r > c && r < R && r - c <= b) v[q][cc] = qv;
                        }
#pragma unroll
                        for (int c2 = 0; c2 < 8; c2++) {
                            if (c2 <= cc || c2 >= nc) continue;
                            const double l2 = __shfl_sync(FULL, v[0][cc], c2);  // L(J + c2, c)
#pragma unroll
                            for (int q = 0; q < kBlkRows; q++) {
                                int r = J + lane + 32 * q;
                                if (r >= J + c2 && r < R && r <= c + b) v[q][c2] = v[q][c2] - v[q][cc] * l2;
                            }
                        }
                    }
#pragma unroll
                    for (int q = 0; q < kBlkRows; q++)
#pragma unroll
                        for (int cc = 0; cc < 8; cc++) {
                            int r = J + lane + 32 * q, c = J + cc;
                            if (cc < nc && r < R && r >= c && r - c <= b) P(k0 + r, k0 + c) = v[q][cc];
                        }
                }
                __syncthreads();
                if (s_bad >= 0) break;
                if (J + 8 < np) {
                    const int c = J + 8 + lane;  // one later panel column per lane, rows over the warps
                    if (c < np) {
                        double lc[8];
#pragma unroll
                        for (int cc = 0; cc < 8; cc++) lc[cc] = (cc < nc && c - (J + cc) <= b) ? P(k0 + c, k0 + J + cc) : 0.0;
                        for (int r = c + warp; r < R && r <= c + b; r += kThreads / 32) {
                            double e = P(k0 + r, k0 + c);
#pragma unroll
                            for (int cc = 0; cc < 8; cc++)
                                if (cc < nc && r - (J + cc) <= b) e = e - P(k0 + r, k0 + J + cc) * lc[cc];
                            P(k0 + r, k0 + c) = e;
                        }
                    }
                    __syncthreads();
                }
            }
        } else if (SMEM && R <= kStageRows && (R + step - 1) / step <= kOwn && (1 << lg) == nb) {
            // every thread keeps the entries of one panel column (ct) in registers, rows rt, rt + step, ...; a
            // column step is: scale column kk (one row per thread, into the window and lcol), barrier, each
            // thread subtracts column kk's products from its entries (the owners of column kk + 1 then hand it
            // to stage[] and its pivot is taken), barrier
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
                // rows past the panel's reach borrow row ib's (or jb's) entries: computed, never stored
                Off pi[4], pj[4];
                int kf[4];
                bool iv[4];
#pragma unroll
                for (int u = 0; u < 4; u++) {
                    int i = ib + u, j = jb + u;
                    iv[u] = i <= last;
                    pi[u] = rowoff[(iv[u] ? i : ib) - k0];
                    pj[u] = rowoff[(j <= last ? j : jb) - k0];
                    kf[u] = max(k0, i - b);
                }
                double s[4][4];
#pragma unroll
                for (int u = 0; u < 4; u++)
#pragma unroll
                    for (int v = 0; v < 4; v++) s[u][v] = (iv[u] && jb + v <= ib + u) ? win[pi[u] + jb + v] : 0.0;
                // the first rows' earliest columns lie outside the later rows' band: those few steps are masked
                const int kfull = min(k1, kf[3]);
                for (int k = kf[0]; k < kfull; k++) {
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        if (k < kf[u]) continue;
                        double li = win[pi[u] + k];
#pragma unroll
                        for (int v = 0; v < 4; v++)
                            if (jb + v <= ib + u) s[u][v] = s[u][v] - li * win[pj[v] + k];
                    }
                }
                // every entry of the tile takes every remaining step: loads one step ahead
                if (kfull < k1) {
                    double li[4], lj[4];
#pragma unroll
                    for (int u = 0; u < 4; u++) {
                        li[u] = win[pi[u] + kfull];
                        lj[u] = win[pj[u] + kfull];
                    }
                    for (int k = kfull; k < k1; k++) {
                        double ni[4], nj[4];
                        const int kn = min(k + 1, k1 - 1);
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            ni[u] = win[pi[u] + kn];
                            nj[u] = win[pj[u] + kn];
                        }
#pragma unroll
                        for (int u = 0; u < 4; u++)
#pragma unroll
                            for (int v = 0; v < 4; v++) s[u][v] = s[u][v] - li[u] * lj[v];
#pragma unroll
                        for (int u = 0; u < 4; u++) {
                            li[u] = ni[u];
                            lj[u] = nj[u];
                        }
                    }
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
                const double yd = y / P(k0 + kk, k0 + kk);  // every lane divides; lane kk keeps it
                if (lane == kk) y = yd;
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
            // lane l: row i0 + l; the block's row offsets go to brow[] for the update of the rows above
            Off ro = lane < np ? slot(i0 + lane) * (Off)ws - (i0 + lane) + b : 0;
            brow[lane] = ro;
            double y = lane < np ? RV(i0 + lane) : 0.0, d = lane < np ? win[ro + i0 + lane] : 1.0;
            __syncwarp();
            double e = 0.0;  // L(i, i0 + lane) of the current step's row i, loaded one step ahead
            if (np >= 1 && lane < np - 1 && np - 1 - lane <= b) e = win[brow[np - 1] + i0 + lane];
            for (int kk = np - 1; kk >= 0; kk--) {
                double en = 0.0;
                if (kk >= 1 && lane < kk - 1 && kk - 1 - lane <= b) en = win[brow[kk - 1] + i0 + lane];
                const double yd = y / d;  // every lane divides; lane kk keeps it
                if (lane == kk) y = yd;
                const double xi = __shfl_sync(FULL, y, kk);
                if (lane < kk && kk - lane <= b) y = y - e * xi;
                e = en;
            }
            if (lane < np) {
                RV(i0 + lane) = y;
                xs[lane] = y;
            }
        }
        __syncthreads();
        for (int k = max(0, i0 - b) + tid; k < i0; k += kThreads) {
            double rr = RV(k);
            for (int i = min(i1 - 1, k + b); i >= i0; i--) rr = rr - win[brow[i - i0] + k] * xs[i - i0];
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
