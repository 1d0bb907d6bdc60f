// kernels3d.cuh — sm_100a kernels of the 3D rigid-viscoplastic Newton iteration (ThreeD/Forging3DSolver.cs).
//
// Layout in HBM: node data SoA-of-xyz (x, vg, v: 3 doubles per node; nodal frames: 9 doubles per node),
// element data 12 doubles of shape-function gradients per tet, the system in the reference's full symmetric CSC
// with 3x3 node blocks, so node j's three columns are one contiguous chunk of 9*|nbr(j)| values.
//
// Determinism: every sum that the reference forms serially is formed here by one thread or one warp in the
// reference's order (element order for the scatter, ascending ring node for K_vol), never by atomics. Global
// reductions use a fixed grid and a fixed tree, so repeated runs are bit-identical.
#pragma once
#include "common.cuh"
#include "runtime.cuh"

namespace ifea {

enum AsmMode { ASM_MATRIX = 0, ASM_RESIDUAL = 1, ASM_ENERGY = 2 };

// Reduction slots (partials[slot * kReduceBlocks + block]).
enum Slot {
    S_E_VOL = 0, S_E_ELEM, S_E_FRIC, S_P_ELEM, S_P_FRIC, S_MAXDIAG, S_RNORM2, S_DOT, S_NORM_A, S_NORM_B,
    S_REACTION, S_MAX_B, S_MAX_T, S_KEPT_B, S_KEPT_T, S_MAXPEN, S_MINQ, S_VOLUME, S_MAXEDGE, S_THIN,
    S_RZ, S_RZNEW, S_PQ, S_RR, S_BB, S_FILL, S_BOX0, S_BOX1, S_BOX2, S_BOX3, S_BOX4, S_BOX5,
    S_COUNT
};

struct View3 {
    int nn, ne, ndof, nbf;
    // topology
    const int32_t *tets, *nts, *ntl, *qk, *gslot, *bface, *bowner, *nfs, *nfl;
    const int8_t *ntl_local;
    const uint8_t *bsym, *is_surface, *on_x0, *on_y0;
    const int32_t *nbr_start, *nbr, *diag_slot, *g_start, *g_node;
    const int32_t *kv_start, *kv_n, *kv_pj, *kv_kstart, *kv_k;
    const double *h_local;
    // state
    double *x, *vg, *vg_prev, *ax, *fixed_val, *k_fric, *a_fric, *grad, *vol, *v_node, *g_coef, *c_local;
    double *kvol, *val, *eps, *dmg, *el_sig, *el_rate, *el_dev, *el_mean;
    double *v, *r, *b, *dv, *v_trial;
    double *e_r, *e_g, *e_w, *e_energy, *e_power;
    int32_t *n_fix, *die_axis;
    uint8_t *fixed, *contact, *release;
    double *partials, *scalars;
    int32_t *err;
    HField die[2];
    double C, N, M, eps0, friction, ram, rate_cut, k_pen, u0, newton_blend, gap;
};

__device__ __forceinline__ d3 axis_of(const View3 &V, int n, int k) { return ld3(V.ax + 9 * n, k); }
__device__ __forceinline__ d3 to_local(const View3 &V, int n, d3 g)
{
    return mk3(dot3(g, axis_of(V, n, 0)), dot3(g, axis_of(V, n, 1)), dot3(g, axis_of(V, n, 2)));
}
__device__ __forceinline__ d3 to_global(const View3 &V, int n, double l0, double l1, double l2)
{
    return add3(add3(scl3(l0, axis_of(V, n, 0)), scl3(l1, axis_of(V, n, 1))), scl3(l2, axis_of(V, n, 2)));
}
__device__ __forceinline__ d3 die_velocity(int c, double ram) { return c == IFEA_TOP_DIE ? mk3(0, 0, -ram) : mk3(0, 0, 0); }
__device__ __forceinline__ double offset_of(int c, double gap) { return c == IFEA_TOP_DIE ? gap : 0.0; }
__device__ __forceinline__ const HField &surface(const View3 &V, int c) { return c == IFEA_TOP_DIE ? V.die[1] : V.die[0]; }
__device__ __forceinline__ d3 sym_p(const View3 &V, d3 p, int n) { return mk3(V.on_x0[n] ? 0 : p.x, V.on_y0[n] ? 0 : p.y, p.z); }
__device__ __forceinline__ double quality_of(const View3 &V, const double *x, int e)
{
    const int32_t *t = V.tets + 4 * e;
    return tet_quality(ld3(x, t[0]), ld3(x, t[1]), ld3(x, t[2]), ld3(x, t[3]));
}

#define GRID_STRIDE(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

// Writes the block's K partial sums to partials[slot_k][blockIdx.x].
template <int K>
__device__ __forceinline__ void emit_sum(const View3 &V, double (&acc)[K], const int (&slots)[K])
{
    __shared__ double sh[32 * K];
    block_sum<K>(acc, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < K; k++) V.partials[slots[k] * kReduceBlocks + blockIdx.x] = acc[k];
}
template <int K>
__device__ __forceinline__ void emit_max(const View3 &V, double (&acc)[K], const int (&slots)[K])
{
    __shared__ double sh[32 * K];
    block_max<K>(acc, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < K; k++) V.partials[slots[k] * kReduceBlocks + blockIdx.x] = acc[k];
}

// Which slots to reduce: code = slot | (is_max << 16).
struct SlotList {
    int n;
    int code[12];
};

// Sums (or maxes) the partials of the listed slots into scalars[slot]; one block per slot, fixed order.
__global__ void k_finalize(double *partials, double *scalars, SlotList list)
{
    int s = blockIdx.x;
    if (s >= list.n) return;
    int code = list.code[s];
    int slot = code & 0xffff;
    bool is_max = (code >> 16) != 0;
    double acc[1] = {is_max ? -INFINITY : 0.0};
    for (int i = threadIdx.x; i < kReduceBlocks; i += blockDim.x) {
        double p = partials[slot * kReduceBlocks + i];
        acc[0] = is_max ? fmax(acc[0], p) : acc[0] + p;
    }
    __shared__ double sh[32];
    if (is_max) block_max<1>(acc, sh); else block_sum<1>(acc, sh);
    if (threadIdx.x == 0) scalars[slot] = acc[0];
}

// ------------------------------------------------------------------ PrepareStep (Forging3DSolver.cs:660-758)

// Nodal frames by Gram–Schmidt of the symmetry-plane and die normals; fixed DOFs and their values.
__global__ void k_frames(View3 V)
{
    GRID_STRIDE(n, V.nn)
    {
        d3 dirs[3], e[3];
        double vals[3], ev[3] = {0, 0, 0};
        e[0] = e[1] = e[2] = mk3(0, 0, 0);
        int k = 0, die_axis = -1, die_idx = -1;
        if (V.on_x0[n]) { dirs[k] = mk3(1, 0, 0); vals[k] = 0; k++; }
        if (V.on_y0[n]) { dirs[k] = mk3(0, 1, 0); vals[k] = 0; k++; }
        int c = V.contact[n];
        if (c != IFEA_FREE) {
            d3 nrm;
            hf_project(surface(V, c), ld3(V.x, n), offset_of(c, V.gap), &nrm);
            dirs[k] = nrm;
            vals[k] = dot3(die_velocity(c, V.ram), nrm);
            die_idx = k;
            k++;
        }
        int m = 0;
        for (int q = 0; q < k; q++) {
            d3 d = dirs[q];
            double val = vals[q];
            for (int s = 0; s < m; s++) {
                double proj = dot3(d, e[s]);
                d = sub3(d, scl3(proj, e[s]));
                val -= proj * ev[s];
            }
            double len = len3(d);
            if (len < 0.2) continue;
            e[m] = scl3(1 / len, d);
            ev[m] = val / len;
            if (q == die_idx) die_axis = m;
            m++;
        }
        if (m == 0) { e[0] = mk3(1, 0, 0); e[1] = mk3(0, 1, 0); e[2] = mk3(0, 0, 1); }
        else if (m == 1) {
            d3 helper = fabs(e[0].x) < 0.8 ? mk3(1, 0, 0) : mk3(0, 1, 0);
            e[1] = nrm3(cross3(e[0], helper));
            e[2] = cross3(e[0], e[1]);
        } else if (m == 2) {
            e[2] = nrm3(cross3(e[0], e[1]));
        }
        for (int a = 0; a < 3; a++) st3(V.ax + 9 * n, a, e[a]);
        V.n_fix[n] = m;
        V.die_axis[n] = die_axis;
        for (int q = 0; q < 3; q++) {
            V.fixed[3 * n + q] = q < m;
            V.fixed_val[3 * n + q] = q < m ? ev[q] : 0.0;
        }
        V.release[n] = 0;
    }
}

// Shape-function gradients and volumes; the lowest inverted tet index goes to err[0].
__global__ void k_grad(View3 V)
{
    GRID_STRIDE(el, V.ne)
    {
        const int32_t *t = V.tets + 4 * el;
        d3 p0 = ld3(V.x, t[0]);
        d3 a = sub3(ld3(V.x, t[1]), p0), b = sub3(ld3(V.x, t[2]), p0), c = sub3(ld3(V.x, t[3]), p0);
        double det = dot3(a, cross3(b, c));
        if (!(det > 0)) atomicMin(&V.err[0], el);
        d3 g1 = scl3(1 / det, cross3(b, c)), g2 = scl3(1 / det, cross3(c, a)), g3 = scl3(1 / det, cross3(a, b));
        d3 g0 = neg3(add3(add3(g1, g2), g3));
        double *g = V.grad + 12 * el;
        st3(g, 0, g0); st3(g, 1, g1); st3(g, 2, g2); st3(g, 3, g3);
        V.vol[el] = det / 6;
    }
}

// Nodal volumes and the averaged-nodal gradient operator g_n (BuildAnp :764-795), one node per thread in the
// reference's accumulation order.
__global__ void k_anp_coef(View3 V)
{
    GRID_STRIDE(n, V.nn)
    {
        double vn = 0;
        for (int32_t q = V.nts[n]; q < V.nts[n + 1]; q++) vn += V.vol[V.ntl[q]] / 4;
        V.v_node[n] = vn;
        for (int32_t p = V.g_start[n]; p < V.g_start[n + 1]; p++) st3(V.g_coef, p, mk3(0, 0, 0));
        for (int32_t q = V.nts[n]; q < V.nts[n + 1]; q++) {
            int e = V.ntl[q];
            double w = V.vol[e] / 4 / vn;
            for (int a = 0; a < 4; a++) {
                int p = V.gslot[4 * q + a];
                d3 gc = scl3(w, ld3(V.grad + 12 * e, a));
                st3(V.g_coef, p, add3(ld3(V.g_coef, p), gc));
            }
        }
    }
}

// c_local[p] = ToLocal(gNode[p], gCoef[p])
__global__ void k_clocal(View3 V, int total)
{
    GRID_STRIDE(p, total) { st3(V.c_local, p, to_local(V, V.g_node[p], ld3(V.g_coef, p))); }
}

// K_vol = sum_n kPen V_n (R g)(R g)^T (BuildAnp :801-822), gathered per column node: one warp per node, the
// column chunk in shared memory, ring nodes n in ascending order so each slot sums in the reference's order.
__global__ void k_kvol(View3 V, int max_nbr)
{
    extern __shared__ double smem[];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    double *col = smem + (size_t)warp * 9 * max_nbr;
    for (int j = blockIdx.x * wpb + warp; j < V.nn; j += gridDim.x * wpb) {
        int nb = V.nbr_start[j + 1] - V.nbr_start[j];
        for (int s = lane; s < 9 * nb; s += 32) col[s] = 0.0;
        __syncwarp();
        for (int32_t pr = V.kv_start[j]; pr < V.kv_start[j + 1]; pr++) {
            int n = V.kv_n[pr];
            double kv = V.k_pen * V.v_node[n];
            d3 cj = ld3(V.c_local, V.kv_pj[pr]);
            int g0 = V.g_start[n], cnt = V.g_start[n + 1] - g0, ks = V.kv_kstart[pr];
            for (int t = lane; t < cnt; t += 32) {
                d3 ci = ld3(V.c_local, g0 + t);
                int k = V.kv_k[ks + t];
                for (int cjx = 0; cjx < 3; cjx++)
                    for (int cix = 0; cix < 3; cix++)
                        col[cjx * 3 * nb + 3 * k + cix] += kv * (get3(ci, cix) * get3(cj, cjx));
            }
            __syncwarp();
        }
        double *dst = V.kvol + 9 * (size_t)V.nbr_start[j];
        for (int s = lane; s < 9 * nb; s += 32) dst[s] = col[s];
        __syncwarp();
    }
}

// Friction areas and lagged shear yield stress (BuildFriction :829-850), gathered in face order per node.
__global__ void k_friction_prep(View3 V)
{
    GRID_STRIDE(n, V.nn)
    {
        double af = 0, ks = 0;
        int kc = 0;
        for (int32_t q = V.nfs[n]; q < V.nfs[n + 1]; q++) {
            int k = V.nfl[q];
            int a = V.bface[3 * k], b = V.bface[3 * k + 1], c = V.bface[3 * k + 2];
            double area = 0.5 * len3(cross3(sub3(ld3(V.x, b), ld3(V.x, a)), sub3(ld3(V.x, c), ld3(V.x, a))));
            double kk = V.el_sig[V.bowner[k]] / sqrt(3.0);
            af += area / 3;
            ks += kk;
            kc++;
        }
        V.a_fric[n] = af;
        V.k_fric[n] = kc > 0 ? ks / kc : 0;
    }
}

// LoadVelocityGuess (:854-869)
__global__ void k_guess(View3 V, int trend)
{
    GRID_STRIDE(n, V.nn)
    {
        d3 g = ld3(V.vg, n);
        if (trend) g = sub3(scl3(2, g), ld3(V.vg_prev, n));
        d3 l = to_local(V, n, g);
        for (int c = 0; c < 3; c++) {
            int d = 3 * n + c;
            V.v[d] = V.fixed[d] ? V.fixed_val[d] : get3(l, c);
        }
    }
}

// ------------------------------------------------------------------ Assemble (:1115-1217)

// Column p of B (6 engineering strain-rate rows) for node gradient g, component c (Kernel :1317-1327).
__device__ __forceinline__ void b_column(const double *g, int c, double (&B)[6])
{
    double bx = g[0], by = g[1], bz = g[2];
    B[0] = c == 0 ? bx : 0; B[1] = c == 1 ? by : 0; B[2] = c == 2 ? bz : 0;
    B[3] = c == 0 ? by : (c == 1 ? bx : 0);
    B[4] = c == 1 ? bz : (c == 2 ? by : 0);
    B[5] = c == 0 ? bz : (c == 2 ? bx : 0);
}
__device__ __forceinline__ void mb_column(const double (&B)[6], double (&MB)[6])
{
    double tr = (B[0] + B[1] + B[2]) / 3;
    MB[0] = 2.0 / 3.0 * (B[0] - tr);
    MB[1] = 2.0 / 3.0 * (B[1] - tr);
    MB[2] = 2.0 / 3.0 * (B[2] - tr);
    MB[3] = B[3] / 3;
    MB[4] = B[4] / 3;
    MB[5] = B[5] / 3;
}

// One element per thread: strain rate, flow stress, residual in local frames, energy/power, element fields;
// for the matrix also G = B^T M eps-dot and the scalars vol*mu, vol*coefN*NewtonBlend (Kernel :1312-1400).
template <int MODE>
__global__ void __launch_bounds__(256) k_element(View3 V, const double *__restrict__ v, int newton)
{
    double acc[2] = {0, 0};
    GRID_STRIDE(e, V.ne)
    {
        const int32_t *t = V.tets + 4 * e;
        int nd[4] = {t[0], t[1], t[2], t[3]};
        double g[12];
        for (int k = 0; k < 12; k++) g[k] = V.grad[12 * e + k];
        double ve[12];
        for (int a = 0; a < 4; a++) {
            d3 gv = to_global(V, nd[a], v[3 * nd[a]], v[3 * nd[a] + 1], v[3 * nd[a] + 2]);
            ve[3 * a] = gv.x; ve[3 * a + 1] = gv.y; ve[3 * a + 2] = gv.z;
        }
        // eps = B ve, summed over the 12 columns in order (zero columns contribute +-0)
        double eps[6] = {0, 0, 0, 0, 0, 0};
        for (int k = 0; k < 12; k++) {
            double B[6];
            b_column(g + 3 * (k / 3), k % 3, B);
            for (int i = 0; i < 6; i++) eps[i] += B[i] * ve[k];
        }
        double ev3 = (eps[0] + eps[1] + eps[2]) / 3;
        double d0 = eps[0] - ev3, d1 = eps[1] - ev3, d2 = eps[2] - ev3;
        double rate = sqrt(rmax(2.0 / 3.0 * (d0 * d0 + d1 * d1 + d2 * d2) + (eps[3] * eps[3] + eps[4] * eps[4] + eps[5] * eps[5]) / 3.0, 0));
        double me[6] = {2.0 / 3.0 * d0, 2.0 / 3.0 * d1, 2.0 / 3.0 * d2, eps[3] / 3, eps[4] / 3, eps[5] / 3};
        double vol = V.vol[e];
        double strain = V.eps[e];
        double sigCut = flow_stress(V.C, V.N, V.M, V.eps0, strain, V.rate_cut);
        double mu0 = sigCut / V.rate_cut, mExp = V.M;
        double mu, sig, wDens, coefN;
        if (rate > V.rate_cut) {
            sig = flow_stress(V.C, V.N, V.M, V.eps0, strain, rate);
            mu = sig / rate;
            wDens = 0.5 * sigCut * V.rate_cut + (sig * rate - sigCut * V.rate_cut) / (mExp + 1);
            coefN = (mExp - 1) * mu / (rate * rate);
        } else {
            mu = mu0;
            sig = mu0 * rate;
            wDens = 0.5 * mu0 * rate * rate;
            coefN = 0;
        }
        double energy = vol * wDens, power = vol * sig * rate;
        acc[0] += energy;
        acc[1] += power;
        if (MODE == ASM_ENERGY) continue;
        V.e_energy[e] = energy;
        V.e_power[e] = power;
        V.el_sig[e] = sig;
        V.el_rate[e] = rate;
        for (int i = 0; i < 6; i++) V.el_dev[6 * e + i] = mu * me[i];
        double G[12];
        for (int k = 0; k < 12; k++) {
            double B[6];
            b_column(g + 3 * (k / 3), k % 3, B);
            double s = 0;
            for (int i = 0; i < 6; i++) s += B[i] * me[i];
            G[k] = s;
        }
        for (int a = 0; a < 4; a++) {
            d3 rl = to_local(V, nd[a], mk3(vol * mu * G[3 * a], vol * mu * G[3 * a + 1], vol * mu * G[3 * a + 2]));
            V.e_r[12 * e + 3 * a] = rl.x;
            V.e_r[12 * e + 3 * a + 1] = rl.y;
            V.e_r[12 * e + 3 * a + 2] = rl.z;
        }
        if (MODE != ASM_MATRIX) continue;
        for (int k = 0; k < 12; k++) V.e_g[12 * e + k] = G[k];
        V.e_w[2 * e] = vol * mu;
        V.e_w[2 * e + 1] = newton ? vol * coefN * V.newton_blend : 0;
    }
    const int slots[2] = {S_E_ELEM, S_P_ELEM};
    emit_sum<2>(V, acc, slots);
}

// Rotated element block R_i K_ab R_j^T (ElementWork :1287-1309) for rows of node a, columns of node b.
__device__ __forceinline__ void element_block(const View3 &V, int e, int a, int b, int i, int j, double (&out)[9])
{
    const double *g = V.grad + 12 * e;
    const double *G = V.e_g + 12 * e;
    double wm = V.e_w[2 * e], wn = V.e_w[2 * e + 1];
    double ke[3][3];
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            int p = 3 * a + r, q = 3 * b + c;
            int lo = p < q ? p : q, hi = p < q ? q : p;
            double Bl[6], Bh[6], MBh[6];
            b_column(g + 3 * (lo / 3), lo % 3, Bl);
            b_column(g + 3 * (hi / 3), hi % 3, Bh);
            mb_column(Bh, MBh);
            double s = 0;
            for (int k = 0; k < 6; k++) s += Bl[k] * MBh[k];
            ke[r][c] = wm * s + wn * G[lo] * G[hi];
        }
    double blk[3][3];
    for (int r = 0; r < 3; r++) {
        d3 ar = axis_of(V, i, r);
        for (int c = 0; c < 3; c++) blk[r][c] = ar.x * ke[0][c] + ar.y * ke[1][c] + ar.z * ke[2][c];
    }
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            d3 bc = axis_of(V, j, c);
            out[3 * r + c] = blk[r][0] * bc.x + blk[r][1] * bc.y + blk[r][2] * bc.z;
        }
}

// Vector shear friction on the free axes of a contact node (Assemble :1175-1214): residual, energy, power and,
// for the matrix, the 3x3 diagonal block kq[q][p].
__device__ __forceinline__ bool friction_node(const View3 &V, int n, const double *v, bool newton, double (&fr)[3],
                                              double &energy, double &power, double (&kq)[3][3])
{
    if (V.contact[n] == IFEA_FREE || V.n_fix[n] >= 3) return false;
    double c = V.friction * V.k_fric[n] * V.a_fric[n] * (2 / M_PI);
    if (c <= 0) return false;
    d3 vd = to_local(V, n, die_velocity(V.contact[n], V.ram));
    int k0 = V.n_fix[n];
    double s[3] = {0, 0, 0}, s2 = 0;
    for (int q = k0; q < 3; q++) {
        s[q] = v[3 * n + q] - get3(vd, q);
        s2 += s[q] * s[q];
    }
    double sl = sqrt(s2), z = sl / V.u0, at = atan(z);
    energy = c * (sl * at - 0.5 * V.u0 * log(1 + z * z));
    power = c * at * sl;
    double gs = sl > 1e-12 * V.u0 ? at / sl : 1 / V.u0;
    for (int q = 0; q < 3; q++) fr[q] = q >= k0 ? c * gs * s[q] : 0.0;
    double tang = c / (V.u0 * (1 + z * z));
    for (int q = 0; q < 3; q++)
        for (int p = 0; p < 3; p++) {
            double kqp = 0;
            if (q >= k0 && p >= k0) {
                if (newton && sl > 1e-12 * V.u0)
                    kqp = c * gs * ((q == p ? 1 : 0) - s[q] * s[p] / s2) + tang * s[q] * s[p] / s2;
                else
                    kqp = q == p ? c * gs : 0;
            }
            kq[q][p] = kqp;
        }
    return true;
}

// Column-node assembly, one warp per node j:
//   R_j = (K_vol v)_j + sum over tets of j in ascending order of the rotated element residual + friction;
//   MATRIX: the node's value chunk = K_vol chunk + element blocks (a, b_j) added in element order + friction,
//   then (BC) fixed rows/columns to identity and the free-diagonal maximum; b = -R with fixed entries zero.
template <int MODE, bool BC>
__global__ void __launch_bounds__(256) k_columns(View3 V, const double *__restrict__ v, int newton, int max_nbr)
{
    extern __shared__ double smem[];
    int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, wpb = blockDim.x >> 5;
    double *col = smem + (size_t)warp * 9 * max_nbr;
    double acc[5] = {0, 0, 0, 0, 0};  // E_VOL, E_FRIC, P_FRIC, RNORM2, (max diag separately)
    double maxdiag[1] = {0.0};
    for (int j = blockIdx.x * wpb + warp; j < V.nn; j += gridDim.x * wpb) {
        int nb = V.nbr_start[j + 1] - V.nbr_start[j];
        const int32_t *nbr = V.nbr + V.nbr_start[j];
        const double *kchunk = V.kvol + 9 * (size_t)V.nbr_start[j];
        // (K_vol v)_j: three rows, contiguous slices of the chunk (K_vol is exactly symmetric)
        double rv[3] = {0, 0, 0};
        for (int t = lane; t < 3 * nb; t += 32) {
            int k = t / 3, c = t % 3;
            double vv = v[3 * nbr[k] + c];
            for (int ci = 0; ci < 3; ci++) rv[ci] += kchunk[ci * 3 * nb + t] * vv;
        }
        for (int ci = 0; ci < 3; ci++)
            for (int o = 16; o > 0; o >>= 1) rv[ci] += __shfl_xor_sync(0xffffffffu, rv[ci], o);
        if (lane == 0) acc[0] += 0.5 * v[3 * j] * rv[0] + 0.5 * v[3 * j + 1] * rv[1] + 0.5 * v[3 * j + 2] * rv[2];
        double fr[3] = {0, 0, 0}, kq[3][3], fe = 0, fp = 0;
        bool has_fric = V.friction > 0 && friction_node(V, j, v, newton, fr, fe, fp, kq);
        if (lane == 0) { acc[1] += fe; acc[2] += fp; }
        if (MODE == ASM_ENERGY) continue;
        // residual: element contributions in ascending element order, then friction
        if (lane < 3) {
            double s = rv[lane];
            for (int32_t q = V.nts[j]; q < V.nts[j + 1]; q++) s += V.e_r[12 * V.ntl[q] + 3 * V.ntl_local[q] + lane];
            s += fr[lane];
            V.r[3 * j + lane] = s;
            bool fx = V.fixed[3 * j + lane];
            double bval = fx ? 0.0 : -s;
            V.b[3 * j + lane] = bval;
            acc[3] += bval * bval;
        }
        if (MODE != ASM_MATRIX) continue;
        for (int s = lane; s < 9 * nb; s += 32) col[s] = kchunk[s];
        __syncwarp();
        // element blocks, 8 tets per pass (4 lanes each); adds applied tet by tet in ascending order
        int q0 = V.nts[j], q1 = V.nts[j + 1];
        for (int qb = q0; qb < q1; qb += 8) {
            int q = qb + (lane >> 2), a = lane & 3;
            double blk[9];
            int k = -1;
            if (q < q1) {
                int e = V.ntl[q], b = V.ntl_local[q];
                int i = V.tets[4 * e + a];
                k = V.qk[4 * q + a];
                element_block(V, e, a, b, i, j, blk);
            }
            for (int t = 0; t < 8; t++) {
                if ((lane >> 2) == t && k >= 0)
                    for (int r = 0; r < 3; r++)
                        for (int c = 0; c < 3; c++) col[c * 3 * nb + 3 * k + r] += blk[3 * r + c];
                __syncwarp();
            }
        }
        // friction block on the diagonal (Pos(n,q,n,p) = column p, row component q)
        if (has_fric && lane == 0) {
            int kself = (V.diag_slot[3 * j] - 9 * V.nbr_start[j]) / 3;
            for (int qq = 0; qq < 3; qq++)
                for (int p = 0; p < 3; p++) col[p * 3 * nb + 3 * kself + qq] += kq[qq][p];
        }
        __syncwarp();
        double *dst = V.val + 9 * (size_t)V.nbr_start[j];
        for (int s = lane; s < 9 * nb; s += 32) {
            double val = col[s];
            if (BC) {
                int cj = s / (3 * nb), rem = s % (3 * nb), k = rem / 3, ci = rem % 3;
                int row = 3 * nbr[k] + ci, cdof = 3 * j + cj;
                if (V.fixed[row] || V.fixed[cdof]) val = row == cdof ? 1.0 : 0.0;
                else if (row == cdof) maxdiag[0] = rmax(maxdiag[0], val);
            }
            dst[s] = val;
        }
        __syncwarp();
    }
    const int slots[4] = {S_E_VOL, S_E_FRIC, S_P_FRIC, S_RNORM2};
    double a4[4] = {acc[0], acc[1], acc[2], acc[3]};
    emit_sum<4>(V, a4, slots);
    const int mslots[1] = {S_MAXDIAG};
    emit_max<1>(V, maxdiag, mslots);
}

// Separate BC pass (used when the assembly ran without it) (SolveVelocity :892-901).
__global__ void k_apply_bc(View3 V)
{
    double maxdiag[1] = {0.0};
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = warp; j < V.nn; j += nw) {
        int nb = V.nbr_start[j + 1] - V.nbr_start[j];
        const int32_t *nbr = V.nbr + V.nbr_start[j];
        double *chunk = V.val + 9 * (size_t)V.nbr_start[j];
        for (int s = lane; s < 9 * nb; s += 32) {
            int cj = s / (3 * nb), rem = s % (3 * nb), k = rem / 3, ci = rem % 3;
            int row = 3 * nbr[k] + ci, cdof = 3 * j + cj;
            if (V.fixed[row] || V.fixed[cdof]) chunk[s] = row == cdof ? 1.0 : 0.0;
            else if (row == cdof) maxdiag[0] = rmax(maxdiag[0], chunk[s]);
        }
        if (lane < 3) {
            bool fx = V.fixed[3 * j + lane];
            if (fx) V.r[3 * j + lane] = 0.0;
            V.b[3 * j + lane] = fx ? 0.0 : -V.r[3 * j + lane];
        }
    }
    const int mslots[1] = {S_MAXDIAG};
    emit_max<1>(V, maxdiag, mslots);
}

// Regularisation of the free diagonals by 1e-10 * max diagonal (SolveVelocity :903-908).
__global__ void k_regularise(View3 V)
{
    double reg = 1e-10 * V.scalars[S_MAXDIAG];
    GRID_STRIDE(d, V.ndof)
    {
        if (!V.fixed[d]) V.val[V.diag_slot[d]] += reg;
    }
}

// y = A x with A the assembled values in 3x3 node blocks, row form: one warp per node.
__global__ void k_spmv(View3 V, const double *__restrict__ x, double *__restrict__ y)
{
    int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
    int nw = (gridDim.x * blockDim.x) >> 5;
    for (int j = warp; j < V.nn; j += nw) {
        int nb = V.nbr_start[j + 1] - V.nbr_start[j];
        const int32_t *nbr = V.nbr + V.nbr_start[j];
        const double *chunk = V.val + 9 * (size_t)V.nbr_start[j];
        double s[3] = {0, 0, 0};
        for (int t = lane; t < 3 * nb; t += 32) {
            double xv = x[3 * nbr[t / 3] + t % 3];
            for (int ci = 0; ci < 3; ci++) s[ci] += chunk[ci * 3 * nb + t] * xv;
        }
        for (int ci = 0; ci < 3; ci++)
            for (int o = 16; o > 0; o >>= 1) s[ci] += __shfl_xor_sync(0xffffffffu, s[ci], o);
        if (lane < 3) y[3 * j + lane] = s[lane];
    }
}

// partials: slot A = sum a.b, slot B = sum a.a (optional)
__global__ void k_dot2(View3 V, const double *a, const double *b, int slot_ab, const double *c, int slot_cc)
{
    double acc[2] = {0, 0};
    GRID_STRIDE(i, V.ndof)
    {
        acc[0] += a[i] * b[i];
        if (c) acc[1] += c[i] * c[i];
    }
    __shared__ double sh[64];
    block_sum<2>(acc, sh);
    if (threadIdx.x == 0) {
        V.partials[slot_ab * kReduceBlocks + blockIdx.x] = acc[0];
        if (c) V.partials[slot_cc * kReduceBlocks + blockIdx.x] = acc[1];
    }
}

__global__ void k_axpy(int n, double *y, const double *x, const double *a, double alpha)
{
    GRID_STRIDE(i, n) { y[i] = x[i] + alpha * a[i]; }
}

// ------------------------------------------------------------------ FinalEvaluation (:1402-1451)

__global__ void k_final_nodes(View3 V)
{
    double acc[1] = {0};
    double mx[2] = {0, 0};
    GRID_STRIDE(n, V.nn)
    {
        st3(V.vg_prev, n, ld3(V.vg, n));
        st3(V.vg, n, to_global(V, n, V.v[3 * n], V.v[3 * n + 1], V.v[3 * n + 2]));
        int c = V.contact[n];
        if (c == IFEA_FREE) continue;
        d3 rg = to_global(V, n, V.r[3 * n], V.r[3 * n + 1], V.r[3 * n + 2]);
        if (c == IFEA_TOP_DIE) acc[0] -= rg.z;
        int da = V.die_axis[n];
        if (da < 0) continue;
        double comp = V.r[3 * n + da];
        if (c == IFEA_TOP_DIE) mx[1] = rmax(mx[1], comp); else mx[0] = rmax(mx[0], comp);
    }
    const int s1[1] = {S_REACTION};
    emit_sum<1>(V, acc, s1);
    const int s2[2] = {S_MAX_B, S_MAX_T};
    emit_max<2>(V, mx, s2);
}

__global__ void k_release(View3 V)
{
    double kept[2] = {0, 0};
    double maxB = rmax(0.0, V.scalars[S_MAX_B]), maxT = rmax(0.0, V.scalars[S_MAX_T]);
    GRID_STRIDE(n, V.nn)
    {
        int c = V.contact[n];
        if (c == IFEA_FREE || V.die_axis[n] < 0) continue;
        double comp = V.r[3 * n + V.die_axis[n]];
        double thr = 0.02 * (c == IFEA_TOP_DIE ? maxT : maxB);
        if (comp < -thr) V.release[n] = 1;
        else if (c == IFEA_TOP_DIE) kept[1] += 1;
        else kept[0] += 1;
    }
    const int s[2] = {S_KEPT_B, S_KEPT_T};
    emit_sum<2>(V, kept, s);
}

__global__ void k_release_keep(View3 V)
{
    bool keptB = V.scalars[S_KEPT_B] > 0, keptT = V.scalars[S_KEPT_T] > 0;
    if (keptB && keptT) return;
    GRID_STRIDE(n, V.nn)
    {
        int c = V.contact[n];
        if ((!keptT && c == IFEA_TOP_DIE) || (!keptB && c == IFEA_BOTTOM_DIE)) V.release[n] = 0;
    }
}

// Element mean stress from the nodal ANP volumetric strain rates (:1439-1449).
__global__ void k_nodal_mean(View3 V, double *nodal)
{
    GRID_STRIDE(n, V.nn)
    {
        double ev = 0;
        for (int32_t p = V.g_start[n]; p < V.g_start[n + 1]; p++) ev += dot3(ld3(V.g_coef, p), ld3(V.vg, V.g_node[p]));
        nodal[n] = V.k_pen * ev;
    }
}
__global__ void k_el_mean(View3 V, const double *nodal)
{
    GRID_STRIDE(e, V.ne)
    {
        const int32_t *t = V.tets + 4 * e;
        V.el_mean[e] = 0.25 * (nodal[t[0]] + nodal[t[1]] + nodal[t[2]] + nodal[t[3]]);
    }
}

// ------------------------------------------------------------------ TryUpdate (:1455-1537)

// Area-weighted outward normals of the surface nodes (SurfaceNormals :1540-1562), gathered in face order.
__global__ void k_surface_normals(View3 V, const double *x, double *nrm)
{
    GRID_STRIDE(n, V.nn)
    {
        d3 s = mk3(0, 0, 0);
        for (int32_t q = V.nfs[n]; q < V.nfs[n + 1]; q++) {
            int k = V.nfl[q];
            int a = V.bface[3 * k], b = V.bface[3 * k + 1], c = V.bface[3 * k + 2];
            s = add3(s, cross3(sub3(ld3(x, b), ld3(x, a)), sub3(ld3(x, c), ld3(x, a))));
        }
        if (V.on_x0[n]) s.x = 0;
        if (V.on_y0[n]) s.y = 0;
        if (len23(s) > 0) s = nrm3(s);
        st3(nrm, n, s);
    }
}

// Predicted positions, contact release / capture and projection (:1464-1496).
__global__ void k_predict(View3 V, double dt, double gapT, double tol_h, int lenient, double *xT, double *pred,
                          uint8_t *cT)
{
    double mx[1] = {0};
    GRID_STRIDE(n, V.nn)
    {
        double hl = lenient ? tol_h : V.h_local[n];
        d3 p = sym_p(V, add3(ld3(V.x, n), scl3(dt, ld3(V.vg, n))), n);
        st3(pred, n, p);
        int c = V.contact[n];
        uint8_t ct = IFEA_FREE;
        d3 tmp;
        if (c != IFEA_FREE && !V.release[n]) {
            const HField &sf = surface(V, c);
            double off = offset_of(c, gapT);
            if (hf_clearance(sf, p, off) > 0.05 * hl) ct = IFEA_FREE;
            else {
                p = sym_p(V, hf_project(sf, p, off, &tmp), n);
                ct = (uint8_t)c;
            }
        } else if (V.is_surface[n]) {
            double cb = hf_clearance(V.die[0], p, 0), ctp = hf_clearance(V.die[1], p, gapT);
            if (cb < 0 || ctp < 0) {
                int hit = cb <= ctp ? IFEA_BOTTOM_DIE : IFEA_TOP_DIE;
                d3 q = sym_p(V, hf_project(surface(V, hit), p, offset_of(hit, gapT), &tmp), n);
                double pen = len3(sub3(q, p));
                mx[0] = rmax(mx[0], pen / hl);
                p = q;
                ct = (uint8_t)hit;
            }
        }
        cT[n] = ct;
        st3(xT, n, p);
    }
    const int s[1] = {S_MAXPEN};
    emit_max<1>(V, mx, s);
}

// min quality (as a max of -q) and the lowest element index with q <= thr (err[1])
__global__ void k_quality_check(View3 V, const double *x, double thr)
{
    double mx[1] = {-INFINITY};
    GRID_STRIDE(e, V.ne)
    {
        double q = quality_of(V, x, e);
        mx[0] = fmax(mx[0], -q);
        if (q <= thr) atomicMin(&V.err[1], e);
    }
    const int s[1] = {S_MINQ};
    emit_max<1>(V, mx, s);
}

// Worst quality of the tets around node n (WorstAround :1683-1689), warp-parallel min.
__device__ double worst_around_warp(const View3 &V, const double *x, int n)
{
    int lane = threadIdx.x & 31;
    double q = DBL_MAX;
    for (int32_t k = V.nts[n] + lane; k < V.nts[n + 1]; k += 32) q = rmin(q, quality_of(V, x, V.ntl[k]));
    for (int o = 16; o > 0; o >>= 1) {
        double other = __shfl_xor_sync(0xffffffffu, q, o);
        q = (q != q || other != other) ? NAN : (other < q ? other : q);
    }
    return q;
}

// PushOut (:1570-1589)
__device__ d3 push_out(const HField &die, double offset, d3 p, d3 outward, double h)
{
    d3 tmp;
    if (len23(outward) == 0 || hf_clearance(die, p, offset) >= 0) return hf_project(die, p, offset, &tmp);
    d3 d = neg3(outward);
    double step = 0.1 * h, lo = 0, hi = -1;
    for (double t = step; t <= 2 * h + 1e-12; t += step) {
        if (hf_clearance(die, add3(p, scl3(t, d)), offset) >= 0) { hi = t; break; }
        lo = t;
    }
    if (hi < 0) return hf_project(die, p, offset, &tmp);
    for (int i = 0; i < 25; i++) {
        double mid = 0.5 * (lo + hi);
        if (hf_clearance(die, add3(p, scl3(mid, d)), offset) >= 0) hi = mid; else lo = mid;
    }
    return add3(p, scl3(hi, d));
}

// ImprovePlacement (:1625-1679) with the reference's sequential semantics: a single warp scans the tets in
// order, 32 at a time, and handles the first one below qmin before rescanning from the next tet (earlier
// moves change later qualities). counters[0] = moves, counters[1] = corner penetrations.
__global__ void k_improve_placement(View3 V, double *x, uint8_t *contact, const double *pred, const double *nrm,
                                    double gap, double qmin, double h, int lenient, double corner_frac, int *counters)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    int lane = threadIdx.x;
    int total = 0;
    for (int sweep = 0; sweep < 4; sweep++) {
        int count = 0;
        int e0 = 0;
        while (e0 < V.ne) {
            int e = e0 + lane;
            bool bad = e < V.ne && quality_of(V, x, e) < qmin;
            unsigned m = __ballot_sync(0xffffffffu, bad);
            if (!m) { e0 += 32; continue; }
            int eb = e0 + __ffs(m) - 1;
            for (int a = 0; a < 4; a++) {
                int n = V.tets[4 * eb + a];
                int c = contact[n];
                if (c == IFEA_FREE) continue;
                const HField &die = surface(V, c);
                double off = offset_of(c, gap);
                double hl = V.h_local[n];
                double tl = lenient ? h : hl;
                double allow = lenient ? 0.3 * h : corner_frac * hl;
                d3 cand[8];
                int k = 0;
                d3 tmp;
                d3 pn = ld3(pred, n);
                d3 closest = sym_p(V, hf_project(die, pn, off, &tmp), n);
                cand[k++] = closest;
                d3 push = sym_p(V, push_out(die, off, pn, ld3(nrm, n), h), n);
                if (len3(sub3(push, pn)) <= 0.5 * tl) cand[k++] = push;
                double pen = -hf_clearance(die, pn, off);
                const double fs[4] = {0.0, 0.25, 0.5, 0.75};
                for (int q = 0; q < 4; q++)
                    if (pen * (1 - fs[q]) <= allow) cand[k++] = lerp3(pn, closest, fs[q]);
                d3 old = ld3(x, n);
                double best = worst_around_warp(V, x, n);
                int pick = -1;
                for (int ci = 0; ci < k; ci++) {
                    if (eq3(cand[ci], old)) continue;
                    __syncwarp();
                    if (lane == 0) st3(x, n, cand[ci]);
                    __syncwarp();
                    double q = worst_around_warp(V, x, n);
                    if (q > best + 1e-6) { best = q; pick = ci; }
                }
                __syncwarp();
                if (lane == 0) st3(x, n, pick >= 0 ? cand[pick] : old);
                __syncwarp();
                if (pick < 0) continue;
                if (lane == 0) {
                    if (eq3(cand[pick], pn) && pen < 0) contact[n] = IFEA_FREE;
                    if (hf_clearance(die, cand[pick], off) < -1e-9) counters[1]++;
                }
                __syncwarp();
                count++;
            }
            e0 = eb + 1;
        }
        total += count;
        if (count == 0) break;
    }
    if (lane == 0) counters[0] += total;
}

// SmoothInterior (:1776-1838): bad nodes fixed per sweep, then processed strictly in node order by one warp.
__global__ void k_smooth_interior(View3 V, double *x, double qtarget, int sweeps, uint8_t *bad, int *moves_out)
{
    if (blockIdx.x != 0 || threadIdx.x >= 32) return;
    int lane = threadIdx.x;
    int moves = 0;
    for (int s = 0; s < sweeps; s++) {
        for (int n = lane; n < V.nn; n += 32) bad[n] = 0;
        __syncwarp();
        bool any = false;
        for (int e = lane; e < V.ne; e += 32) {
            if (quality_of(V, x, e) >= qtarget) continue;
            for (int a = 0; a < 4; a++) bad[V.tets[4 * e + a]] = 1;
            any = true;
        }
        __syncwarp();
        if (!__any_sync(0xffffffffu, any)) break;
        int sweep_moves = 0;
        for (int n0 = 0; n0 < V.nn; n0 += 32) {
            int nl = n0 + lane;
            bool todo = nl < V.nn && bad[nl] && !V.is_surface[nl];
            unsigned m = __ballot_sync(0xffffffffu, todo);
            while (m) {
                int n = n0 + __ffs(m) - 1;
                m &= m - 1;
                // centroid of the neighbours over the node's tets (sum in tet order, lane 0) and worst quality
                d3 sum = mk3(0, 0, 0);
                int cnt = 0;
                if (lane == 0) {
                    for (int32_t k = V.nts[n]; k < V.nts[n + 1]; k++) {
                        int e = V.ntl[k];
                        for (int a = 0; a < 4; a++) {
                            int mm = V.tets[4 * e + a];
                            if (mm == n) continue;
                            sum = add3(sum, ld3(x, mm));
                            cnt++;
                        }
                    }
                }
                cnt = __shfl_sync(0xffffffffu, cnt, 0);
                sum.x = __shfl_sync(0xffffffffu, sum.x, 0);
                sum.y = __shfl_sync(0xffffffffu, sum.y, 0);
                sum.z = __shfl_sync(0xffffffffu, sum.z, 0);
                double worst = worst_around_warp(V, x, n);
                if (cnt == 0) continue;
                d3 old = ld3(x, n);
                d3 c = scl3(1.0 / cnt, sum);
                const double lambdas[3] = {1.0, 0.5, 0.25};
                for (int l = 0; l < 3; l++) {
                    d3 p = add3(old, scl3(lambdas[l], sub3(c, old)));
                    __syncwarp();
                    if (lane == 0) st3(x, n, mk3(V.on_x0[n] ? 0 : p.x, V.on_y0[n] ? 0 : p.y, p.z));
                    __syncwarp();
                    double q = worst_around_warp(V, x, n);
                    if (q > worst + 1e-6) { sweep_moves++; break; }
                    __syncwarp();
                    if (lane == 0) st3(x, n, old);
                    __syncwarp();
                }
            }
        }
        moves += sweep_moves;
        if (sweep_moves == 0) break;
    }
    if (lane == 0) *moves_out += moves;
}

// ------------------------------------------------------------------ step bookkeeping and telemetry

// eps += rate dt and Cockcroft–Latham damage (Step :626-627, AccumulateDamage :1844-1855)
__global__ void k_strain_damage(View3 V, double dt)
{
    GRID_STRIDE(e, V.ne)
    {
        V.eps[e] += V.el_rate[e] * dt;
        double sig = V.el_sig[e];
        if (!(sig > 0) || V.el_rate[e] <= V.rate_cut) continue;
        const double *d = V.el_dev + 6 * e;
        double m = V.el_mean[e];
        double s1 = principal_max3(d[0] + m, d[1] + m, d[2] + m, d[3], d[4], d[5]);
        if (s1 > 0) V.dmg[e] += s1 / sig * V.el_rate[e] * dt;
    }
}

__global__ void k_volume(View3 V)
{
    double acc[1] = {0};
    GRID_STRIDE(e, V.ne)
    {
        const int32_t *t = V.tets + 4 * e;
        acc[0] += tet_volume(ld3(V.x, t[0]), ld3(V.x, t[1]), ld3(V.x, t[2]), ld3(V.x, t[3]));
    }
    const int s[1] = {S_VOLUME};
    emit_sum<1>(V, acc, s);
}

// Longest surface edge (RemeshTrigger :1875-1882) and thinnest die-held layer (LayerLimitedIncrement :236-249)
__global__ void k_edges_layers(View3 V)
{
    double mx[2] = {0, -INFINITY};
    GRID_STRIDE(k, V.nbf)
    {
        const int32_t *f = V.bface + 3 * k;
        d3 a = ld3(V.x, f[0]), b = ld3(V.x, f[1]), c = ld3(V.x, f[2]);
        mx[0] = rmax(mx[0], rmax(len3(sub3(b, a)), rmax(len3(sub3(c, b)), len3(sub3(a, c)))));
    }
    GRID_STRIDE(n, V.nn)
    {
        if (V.contact[n] != IFEA_TOP_DIE) continue;
        d3 p = ld3(V.x, n);
        double zb = hf_height(V.die[0], p.x, p.y), zt = hf_height(V.die[1], p.x, p.y) + V.gap;
        if (isfinite(zb) && isfinite(zt) && zt > zb) mx[1] = fmax(mx[1], -(zt - zb));
    }
    const int s[2] = {S_MAXEDGE, S_THIN};
    emit_max<2>(V, mx, s);
}

// ------------------------------------------------------------------ constructor tail (:156-184)

__global__ void k_initial_contact(View3 V, double tol, double *clr_b, double *clr_t)
{
    GRID_STRIDE(n, V.nn)
    {
        V.contact[n] = IFEA_FREE;
        clr_b[n] = INFINITY;
        clr_t[n] = INFINITY;
        if (!V.is_surface[n]) continue;
        d3 p = ld3(V.x, n);
        double cb = hf_clearance(V.die[0], p, 0), ct = hf_clearance(V.die[1], p, V.gap);
        clr_b[n] = cb;
        clr_t[n] = ct;
        if (cb < tol) V.contact[n] = IFEA_BOTTOM_DIE;
        else if (ct < tol) V.contact[n] = IFEA_TOP_DIE;
    }
}

__global__ void k_place_and_velocity(View3 V, double rate_ref, double cx, double cy, double min_z)
{
    GRID_STRIDE(n, V.nn)
    {
        int c = V.contact[n];
        if (c != IFEA_FREE) {
            d3 tmp;
            st3(V.x, n, sym_p(V, hf_project(surface(V, c), ld3(V.x, n), offset_of(c, V.gap), &tmp), n));
        }
    }
}
__global__ void k_initial_velocity(View3 V, double rate_ref, double cx, double cy, double min_z)
{
    GRID_STRIDE(n, V.nn)
    {
        d3 p = ld3(V.x, n);
        st3(V.vg, n, mk3(0.5 * rate_ref * (p.x - cx), 0.5 * rate_ref * (p.y - cy), -rate_ref * (p.z - min_z)));
    }
}

}  // namespace ifea

namespace ifea {
// PCG pieces with the step scalars kept on the device (Pcg, Forging3DSolver.cs:1051-1087).
__global__ void k_pcg_residual(int n, const double *b, const double *q, double *r)
{
    GRID_STRIDE(i, n) { r[i] = b[i] - q[i]; }
}
__global__ void k_pcg_xr(int n, const double *scalars, double *x, double *r, const double *p, const double *q)
{
    double alpha = scalars[S_RZ] / scalars[S_PQ];
    GRID_STRIDE(i, n)
    {
        x[i] += alpha * p[i];
        r[i] -= alpha * q[i];
    }
}
__global__ void k_pcg_p(int n, const double *scalars, double *p, const double *z)
{
    double beta = scalars[S_RZNEW] / scalars[S_RZ];
    GRID_STRIDE(i, n) { p[i] = z[i] + beta * p[i]; }
}
__global__ void k_pcg_roll(double *scalars) { scalars[S_RZ] = scalars[S_RZNEW]; }
}  // namespace ifea
