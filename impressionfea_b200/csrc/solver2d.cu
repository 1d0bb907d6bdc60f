// solver2d.cu — the 2D axisymmetric / plane-strain forging increment (Solver/ForgingSolver.cs) on the GPU and
// its C ABI (ifea2d_*, ifea_band_factor_solve).
//
// Per Newton iteration: one thread per quad computes the element stiffness and residual (2x2 Gauss deviatoric
// power + 1-point volumetric penalty, nodal (t, n) rotation); band cells and residual entries are then gathered in
// element order (the reference's serial scatter order); fixed DOFs, friction and the band Cholesky follow. The
// band Cholesky (band.cuh) runs in one CTA, blocked by panels over a circular window of rows in shared memory;
// every entry's products are subtracted in the same order as the reference's row-oriented loop, so the factor and
// the solution are bit-identical to SymmetricBandMatrix.Factorize / Solve.
#include <climits>
#include <cmath>
#include <cstdarg>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "band.cuh"
#include "common.cuh"
#include "mesh2d.h"
#include "runtime.cuh"

namespace ifea {

namespace {

std::string fmt2(const char *f, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, f);
    vsnprintf(buf, sizeof buf, f, ap);
    va_end(ap);
    return buf;
}

struct d2 {
    double x, y;
};
IFEA_HD d2 mk2(double x, double y) { d2 r; r.x = x; r.y = y; return r; }
IFEA_HD d2 add2(d2 a, d2 b) { return mk2(a.x + b.x, a.y + b.y); }
IFEA_HD d2 sub2(d2 a, d2 b) { return mk2(a.x - b.x, a.y - b.y); }
IFEA_HD d2 scl2(double s, d2 a) { return mk2(s * a.x, s * a.y); }
IFEA_HD double dot2(d2 a, d2 b) { return a.x * b.x + a.y * b.y; }
IFEA_HD double cross2(d2 a, d2 b) { return a.x * b.y - a.y * b.x; }
IFEA_HD double len2(d2 a) { return sqrt(a.x * a.x + a.y * a.y); }
IFEA_HD d2 nrm2(d2 a) { double l = len2(a); return l > 0 ? mk2(a.x / l, a.y / l) : a; }
IFEA_HD d2 ld2(const double *p, int n) { return mk2(p[2 * n], p[2 * n + 1]); }
IFEA_HD void st2(double *p, int n, d2 v) { p[2 * n] = v.x; p[2 * n + 1] = v.y; }

// Piecewise-linear die profile (Geometry/DieSurface.cs), points in device memory.
struct Profile {
    int side, n;
    const double *p;  // 2 per point
};

// HeightAt (:85-98)
IFEA_HD double prof_height(const Profile &d, double x)
{
    if (x <= d.p[0]) return d.p[1];
    if (x >= d.p[2 * (d.n - 1)]) return d.p[2 * (d.n - 1) + 1];
    int lo = 0, hi = d.n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (d.p[2 * mid] <= x) lo = mid; else hi = mid;
    }
    double t = (x - d.p[2 * lo]) / (d.p[2 * hi] - d.p[2 * lo]);
    return d.p[2 * lo + 1] + t * (d.p[2 * hi + 1] - d.p[2 * lo + 1]);
}
// Clearance (:116-120)
IFEA_HD double prof_clearance(const Profile &d, d2 q, double offset)
{
    double h = prof_height(d, q.x) + offset;
    return d.side == 0 ? q.y - h : h - q.y;
}
// SegmentNormal (:123-127)
IFEA_HD d2 prof_seg_normal(const Profile &d, int k)
{
    d2 dd = nrm2(sub2(ld2(d.p, k + 1), ld2(d.p, k)));
    return d.side == 0 ? mk2(-dd.y, dd.x) : mk2(dd.y, -dd.x);
}
// Project (:130-160)
IFEA_HD d2 prof_project(const Profile &d, d2 q, double offset, d2 *normal)
{
    d2 shift = mk2(0, offset);
    double best = DBL_MAX, bestT = 0;
    int bestK = 0;
    d2 bestQ = mk2(0, 0);
    for (int k = 0; k < d.n - 1; k++) {
        d2 a = add2(ld2(d.p, k), shift);
        d2 ab = sub2(ld2(d.p, k + 1), ld2(d.p, k));
        double t = rclamp(dot2(sub2(q, a), ab) / dot2(ab, ab), 0.0, 1.0);
        d2 c = add2(a, scl2(t, ab));
        double dd = dot2(sub2(q, c), sub2(q, c));
        if (dd < best) { best = dd; bestK = k; bestT = t; bestQ = c; }
    }
    d2 n = prof_seg_normal(d, bestK);
    if (bestT < 1e-9 && bestK > 0) n = nrm2(add2(n, prof_seg_normal(d, bestK - 1)));
    else if (bestT > 1 - 1e-9 && bestK < d.n - 2) n = nrm2(add2(n, prof_seg_normal(d, bestK + 1)));
    if (normal) *normal = n;
    return bestQ;
}

enum Slot2 { T_ENERGY = 0, T_POWER, T_RNORM2, T_DOT, T_NDV, T_NV, T_REACT, T_MAXB, T_MAXT, T_KEPTB, T_KEPTT, T_MAXPEN,
             T_MINQ, T_AREA, T_MOMENT, T_MAXEDGE, T_EFRIC, T_PFRIC, T_COUNT };

struct View2 {
    int nn, ne, ndof, hb, nloop, axi;
    const int32_t *conn, *eq, *loop, *loop_owner, *cell_ptr, *cell_idx, *cell_src, *dof_ptr, *dof_src, *node_edge;
    int ncell;
    const uint8_t *is_axis;
    double *x, *vg, *v, *v_trial, *r, *dv, *band, *ke, *re, *eps, *dmg, *el_dev, *el_sig, *el_rate, *el_mean;
    double *tan, *nrm, *fixed_val, *k_fric, *a_fric;
    uint8_t *contact, *rotated, *fixed, *release;
    double *partials, *scalars;
    int32_t *err;
    Profile die[2];
    double C, N, M, eps0, friction, ram, rate_cut, k_pen, u0, gap, length;
};

#define GS2(i, n) for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < (n); i += gridDim.x * blockDim.x)

template <int K>
__device__ __forceinline__ void emit2(const View2 &V, double (&acc)[K], const int (&slots)[K], bool is_max)
{
    __shared__ double sh[32 * K];
    if (is_max) block_max<K>(acc, sh); else block_sum<K>(acc, sh);
    if (threadIdx.x == 0)
        for (int k = 0; k < K; k++) V.partials[slots[k] * kReduceBlocks + blockIdx.x] = acc[k];
}

struct SlotList2 {
    int n;
    int code[10];
};
__global__ void k2_finalize(double *partials, double *scalars, SlotList2 l)
{
    int s = blockIdx.x;
    if (s >= l.n) return;
    int slot = l.code[s] & 0xffff;
    bool is_max = (l.code[s] >> 16) != 0;
    double acc[1] = {is_max ? -INFINITY : 0.0};
    for (int i = threadIdx.x; i < kReduceBlocks; i += blockDim.x) {
        double p = partials[slot * kReduceBlocks + i];
        acc[0] = is_max ? fmax(acc[0], p) : acc[0] + p;
    }
    __shared__ double sh[32];
    if (is_max) block_max<1>(acc, sh); else block_sum<1>(acc, sh);
    if (threadIdx.x == 0) scalars[slot] = acc[0];
}

__device__ __forceinline__ int dof2(const View2 &V, int n, int c) { return 2 * V.eq[n] + c; }
__device__ __forceinline__ d2 die_vel2(int c, double ram) { return c == IFEA_TOP_DIE ? mk2(0, -ram) : mk2(0, 0); }
__device__ __forceinline__ double off2(int c, double gap) { return c == IFEA_TOP_DIE ? gap : 0.0; }
__device__ __forceinline__ const Profile &surf2(const View2 &V, int c) { return c == IFEA_TOP_DIE ? V.die[1] : V.die[0]; }
__device__ __forceinline__ double weight2(const View2 &V, double x) { return V.axi ? 2 * M_PI * x : 2 * V.length; }
__device__ __forceinline__ d2 gvel2(const View2 &V, const double *v, int n)
{
    double a = v[dof2(V, n, 0)], b = v[dof2(V, n, 1)];
    return V.rotated[n] ? add2(scl2(a, ld2(V.tan, n)), scl2(b, ld2(V.nrm, n))) : mk2(a, b);
}

// Shape (:563-590)
__device__ __forceinline__ double shape2(double xi, double eta, const double *ex, const double *ey, double *sn, double *dnx,
                                         double *dny)
{
    double dxi[4] = {-(1 - eta) / 4, (1 - eta) / 4, (1 + eta) / 4, -(1 + eta) / 4};
    double deta[4] = {-(1 - xi) / 4, -(1 + xi) / 4, (1 + xi) / 4, (1 - xi) / 4};
    sn[0] = (1 - xi) * (1 - eta) / 4;
    sn[1] = (1 + xi) * (1 - eta) / 4;
    sn[2] = (1 + xi) * (1 + eta) / 4;
    sn[3] = (1 - xi) * (1 + eta) / 4;
    double j11 = 0, j12 = 0, j21 = 0, j22 = 0;
    for (int a = 0; a < 4; a++) {
        j11 += dxi[a] * ex[a];
        j12 += dxi[a] * ey[a];
        j21 += deta[a] * ex[a];
        j22 += deta[a] * ey[a];
    }
    double det = j11 * j22 - j12 * j21;
    if (!(det > 0)) return det;
    for (int a = 0; a < 4; a++) {
        dnx[a] = (j22 * dxi[a] - j12 * deta[a]) / det;
        dny[a] = (-j21 * dxi[a] + j11 * deta[a]) / det;
    }
    return det;
}

// ElementKernel (:592-721) + RotateElementBlock (:541-561); one quad per thread.
template <int MATRIX>
__global__ void __launch_bounds__(128) k2_element(View2 V, const double *__restrict__ v, int newton, int write_fields)
{
    const double G = 0.57735026918962576;
    const double GXi[4] = {-G, G, G, -G}, GEta[4] = {-G, -G, G, G};
    double acc[2] = {0, 0};
    GS2(e, V.ne)
    {
        double ex[4], ey[4], ve[8], sn[4], dnx[4], dny[4], ke[64], re[8];
        int nd[4];
        for (int a = 0; a < 4; a++) {
            int n = V.conn[4 * e + a];
            nd[a] = n;
            ex[a] = V.x[2 * n];
            ey[a] = V.x[2 * n + 1];
            d2 g = gvel2(V, v, n);
            ve[2 * a] = g.x;
            ve[2 * a + 1] = g.y;
        }
        if (MATRIX)
            for (int k = 0; k < 64; k++) ke[k] = 0;
        for (int k = 0; k < 8; k++) re[k] = 0;
        double eps = V.eps[e];
        double sigCut = flow_stress(V.C, V.N, V.M, V.eps0, eps, V.rate_cut);
        double mu0 = sigCut / V.rate_cut, mExp = V.M;
        double sigSum = 0, rateSum = 0, s0Sum = 0, s1Sum = 0, s2Sum = 0, tSum = 0, energy = 0, power = 0;
        bool bad = false;
        for (int g = 0; g < 4; g++) {
            double det = shape2(GXi[g], GEta[g], ex, ey, sn, dnx, dny);
            if (!(det > 0)) { bad = true; break; }
            double r = 0;
            for (int a = 0; a < 4; a++) r += sn[a] * ex[a];
            double w = det * weight2(V, r);
            double b0[8], b1[8], b2[8], b3[8];
            for (int a = 0; a < 4; a++) {
                b0[2 * a] = dnx[a]; b0[2 * a + 1] = 0;
                b1[2 * a] = 0; b1[2 * a + 1] = dny[a];
                b2[2 * a] = V.axi ? sn[a] / r : 0; b2[2 * a + 1] = 0;
                b3[2 * a] = dny[a]; b3[2 * a + 1] = dnx[a];
            }
            double e0 = 0, e1 = 0, e2 = 0, e3 = 0;
            for (int k = 0; k < 8; k++) {
                e0 += b0[k] * ve[k];
                e1 += b1[k] * ve[k];
                e2 += b2[k] * ve[k];
                e3 += b3[k] * ve[k];
            }
            double ev3 = (e0 + e1 + e2) / 3;
            double d0 = e0 - ev3, d1 = e1 - ev3, dd2 = e2 - ev3;
            double rate = sqrt(rmax(2.0 / 3.0 * (d0 * d0 + d1 * d1 + dd2 * dd2) + e3 * e3 / 3.0, 0));
            double m0 = 2.0 / 3.0 * d0, m1 = 2.0 / 3.0 * d1, m2 = 2.0 / 3.0 * dd2, m3 = e3 / 3.0;
            double g8[8];
            for (int k = 0; k < 8; k++) g8[k] = b0[k] * m0 + b1[k] * m1 + b2[k] * m2 + b3[k] * m3;
            double mu, sig, wDens, coefN;
            if (rate > V.rate_cut) {
                sig = flow_stress(V.C, V.N, V.M, V.eps0, eps, rate);
                mu = sig / rate;
                wDens = 0.5 * sigCut * V.rate_cut + (sig * rate - sigCut * V.rate_cut) / (mExp + 1);
                coefN = (mExp - 1) * mu / (rate * rate);
            } else {
                mu = mu0;
                sig = mu0 * rate;
                wDens = 0.5 * mu0 * rate * rate;
                coefN = 0;
            }
            energy += w * wDens;
            power += w * sig * rate;
            sigSum += sig;
            rateSum += rate;
            s0Sum += mu * m0;
            s1Sum += mu * m1;
            s2Sum += mu * m2;
            tSum += mu * m3;
            double wm = w * mu;
            for (int k = 0; k < 8; k++) re[k] += wm * g8[k];
            if (!MATRIX) continue;
            double mb[4][8];
            for (int k = 0; k < 8; k++) {
                double tr = (b0[k] + b1[k] + b2[k]) / 3;
                mb[0][k] = 2.0 / 3.0 * (b0[k] - tr);
                mb[1][k] = 2.0 / 3.0 * (b1[k] - tr);
                mb[2][k] = 2.0 / 3.0 * (b2[k] - tr);
                mb[3][k] = b3[k] / 3.0;
            }
            double wn = newton ? w * coefN : 0;
            for (int p = 0; p < 8; p++)
                for (int q = 0; q <= p; q++) {
                    double s = b0[p] * mb[0][q] + b1[p] * mb[1][q] + b2[p] * mb[2][q] + b3[p] * mb[3][q];
                    ke[8 * p + q] += wm * s + wn * g8[p] * g8[q];
                }
        }
        if (!bad) {
            double det0 = shape2(0, 0, ex, ey, sn, dnx, dny);
            if (!(det0 > 0)) bad = true;
            else {
                double rc = 0;
                for (int a = 0; a < 4; a++) rc += sn[a] * ex[a];
                double w0 = 4 * det0 * weight2(V, rc);
                double c8[8], evol = 0;
                for (int a = 0; a < 4; a++) {
                    c8[2 * a] = dnx[a] + (V.axi ? sn[a] / rc : 0);
                    c8[2 * a + 1] = dny[a];
                }
                for (int k = 0; k < 8; k++) evol += c8[k] * ve[k];
                double kw = V.k_pen * w0;
                for (int k = 0; k < 8; k++) re[k] += kw * evol * c8[k];
                energy += 0.5 * kw * evol * evol;
                power += kw * evol * evol;
                if (MATRIX) {
                    for (int p = 0; p < 8; p++)
                        for (int q = 0; q <= p; q++) ke[8 * p + q] += kw * c8[p] * c8[q];
                    for (int p = 0; p < 8; p++)
                        for (int q = p + 1; q < 8; q++) ke[8 * p + q] = ke[8 * q + p];
                }
                if (write_fields) {
                    V.el_sig[e] = sigSum / 4;
                    V.el_rate[e] = rateSum / 4;
                    V.el_dev[4 * e] = s0Sum / 4;
                    V.el_dev[4 * e + 1] = s1Sum / 4;
                    V.el_dev[4 * e + 2] = s2Sum / 4;
                    V.el_dev[4 * e + 3] = tSum / 4;
                    V.el_mean[e] = V.k_pen * evol;
                }
            }
        }
        if (bad) {
            atomicMin(&V.err[0], e);
            continue;
        }
        acc[0] += energy;
        acc[1] += power;
        // rotation of rotated nodes' rows and columns into their (t, n) frames
        for (int a = 0; a < 4; a++) {
            int n = nd[a];
            if (!V.rotated[n]) continue;
            d2 t = ld2(V.tan, n), nn = ld2(V.nrm, n);
            int r0 = 2 * a, r1 = r0 + 1;
            double f0 = re[r0], f1 = re[r1];
            re[r0] = t.x * f0 + t.y * f1;
            re[r1] = nn.x * f0 + nn.y * f1;
            if (!MATRIX) continue;
            for (int c = 0; c < 8; c++) {
                double k0 = ke[8 * r0 + c], k1 = ke[8 * r1 + c];
                ke[8 * r0 + c] = t.x * k0 + t.y * k1;
                ke[8 * r1 + c] = nn.x * k0 + nn.y * k1;
            }
            for (int rr = 0; rr < 8; rr++) {
                double k0 = ke[8 * rr + r0], k1 = ke[8 * rr + r1];
                ke[8 * rr + r0] = t.x * k0 + t.y * k1;
                ke[8 * rr + r1] = nn.x * k0 + nn.y * k1;
            }
        }
        for (int k = 0; k < 8; k++) V.re[8 * e + k] = re[k];
        if (MATRIX)
            for (int k = 0; k < 64; k++) V.ke[64 * e + k] = ke[k];
    }
    const int slots[2] = {T_ENERGY, T_POWER};
    emit2<2>(V, acc, slots, false);
}

// Friction at a rotated contact node (Assemble :513-535): residual, energy, power, tangent.
__device__ __forceinline__ bool fric2(const View2 &V, const double *v, int n, int newton, double &f, double &en,
                                      double &pw, double &kt)
{
    if (!V.rotated[n]) return false;
    double c = V.friction * V.k_fric[n] * V.a_fric[n] * (2 / M_PI);
    if (c <= 0) return false;
    int d = dof2(V, n, 0);
    double s = v[d] - dot2(die_vel2(V.contact[n], V.ram), ld2(V.tan, n));
    double z = s / V.u0;
    f = c * atan(z);
    en = c * (s * atan(z) - 0.5 * V.u0 * log(1 + z * z));
    pw = f * s;
    kt = newton ? c / (V.u0 * (1 + z * z)) : (fabs(z) > 1e-9 ? f / s : c / V.u0);
    return true;
}

// Band cells gathered in element order; zero contributions skipped (Assemble :505-509).
__global__ void k2_band(View2 V)
{
    GS2(c, V.ncell)
    {
        double s = 0;
        for (int32_t k = V.cell_ptr[c]; k < V.cell_ptr[c + 1]; k++) {
            double kv = V.ke[V.cell_src[k]];
            if (kv != 0) s += kv;
        }
        V.band[V.cell_idx[c]] = s;
    }
}

// Residual per DOF in element order, then friction (energy/power partials), then fixed rows/columns of the band
// (ConstrainDof) and r[fixed] = 0.
__global__ void k2_residual_friction(View2 V, const double *__restrict__ v, int newton, int matrix, int bc)
{
    double acc[3] = {0, 0, 0};
    GS2(n, V.nn)
    {
        for (int c = 0; c < 2; c++) {
            int d = dof2(V, n, c);
            double s = 0;
            for (int32_t k = V.dof_ptr[d]; k < V.dof_ptr[d + 1]; k++) s += V.re[V.dof_src[k]];
            V.r[d] = s;
        }
        double f = 0, en = 0, pw = 0, kt = 0;
        if (V.friction > 0 && fric2(V, v, n, newton, f, en, pw, kt)) {
            int d = dof2(V, n, 0);
            V.r[d] += f;
            acc[0] += en;
            acc[1] += pw;
            if (matrix) V.band[(int64_t)d * (V.hb + 1) + V.hb] += kt;
        }
        if (bc)
            for (int c = 0; c < 2; c++) {
                int d = dof2(V, n, c);
                if (V.fixed[d]) V.r[d] = 0;
                acc[2] += V.r[d] * V.r[d];
            }
    }
    const int s2[3] = {T_EFRIC, T_PFRIC, T_RNORM2};
    emit2<3>(V, acc, s2, false);
}

// ConstrainDof (SymmetricBandMatrix.cs:50-57) for every fixed DOF, cell-wise.
__global__ void k2_constrain(View2 V)
{
    int64_t total = (int64_t)V.ndof * (V.hb + 1);
    for (int64_t c = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; c < total; c += (int64_t)gridDim.x * blockDim.x) {
        int i = (int)(c / (V.hb + 1));
        int j = i - V.hb + (int)(c % (V.hb + 1));
        if (j < 0) continue;
        if (V.fixed[i] || V.fixed[j]) V.band[c] = i == j ? 1.0 : 0.0;
    }
}

__global__ void k2_frames(View2 V)
{
    GS2(n, V.nn)
    {
        V.rotated[n] = 0;
        st2(V.tan, n, mk2(1, 0));
        st2(V.nrm, n, mk2(0, 1));
        V.release[n] = 0;
        int d0 = dof2(V, n, 0), d1 = dof2(V, n, 1);
        V.fixed[d0] = V.fixed[d1] = 0;
        V.fixed_val[d0] = V.fixed_val[d1] = 0;
        bool axis = V.is_axis[n];
        int c = V.contact[n];
        if (c != IFEA_FREE) {
            d2 dv = die_vel2(c, V.ram);
            if (axis) {
                V.fixed[d0] = 1; V.fixed_val[d0] = 0;
                V.fixed[d1] = 1; V.fixed_val[d1] = dv.y;
            } else {
                d2 nrm;
                prof_project(surf2(V, c), ld2(V.x, n), off2(c, V.gap), &nrm);
                st2(V.nrm, n, nrm);
                st2(V.tan, n, mk2(nrm.y, -nrm.x));
                V.rotated[n] = 1;
                V.fixed[d1] = 1;
                V.fixed_val[d1] = dot2(dv, nrm);
            }
        } else if (axis) {
            V.fixed[d0] = 1;
            V.fixed_val[d0] = 0;
        }
        // tributary friction area and lagged k from the (at most two) boundary edges at the node, in loop order
        double af = 0, ks = 0;
        int kc = 0;
        for (int q = 0; q < 2; q++) {
            int k = V.node_edge[2 * n + q];
            if (k < 0) continue;
            int a = V.loop[k], bnode = V.loop[(k + 1) % V.nloop];
            double len = len2(sub2(ld2(V.x, bnode), ld2(V.x, a)));
            double area = len * weight2(V, 0.5 * (V.x[2 * a] + V.x[2 * bnode]));
            af += 0.5 * area;
            ks += V.el_sig[V.loop_owner[k]] / sqrt(3.0);
            kc++;
        }
        V.a_fric[n] = af;
        V.k_fric[n] = kc > 0 ? ks / kc : 0;
    }
}

__global__ void k2_guess(View2 V)
{
    GS2(n, V.nn)
    {
        d2 g = ld2(V.vg, n);
        int d0 = dof2(V, n, 0), d1 = dof2(V, n, 1);
        double v0 = g.x, v1 = g.y;
        if (V.rotated[n]) {
            v0 = dot2(g, ld2(V.tan, n));
            v1 = dot2(g, ld2(V.nrm, n));
        }
        V.v[d0] = V.fixed[d0] ? V.fixed_val[d0] : v0;
        V.v[d1] = V.fixed[d1] ? V.fixed_val[d1] : v1;
    }
}

__global__ void k2_dots(View2 V, const double *a, const double *b, const double *c)
{
    double acc[2] = {0, 0};
    GS2(i, V.ndof)
    {
        acc[0] += a[i] * b[i];
        if (c) acc[1] += c[i] * c[i];
    }
    const int s[2] = {T_DOT, T_NDV};
    emit2<2>(V, acc, s, false);
}

__global__ void k2_axpy(int n, double *y, const double *x, const double *d, double beta)
{
    GS2(i, n) { y[i] = x[i] + beta * d[i]; }
}
__global__ void k2_neg(int n, double *y, const double *x)
{
    GS2(i, n) { y[i] = -x[i]; }
}

// FinalEvaluation (:737-784)
__global__ void k2_final(View2 V)
{
    double acc[1] = {0}, mx[2] = {0, 0};
    GS2(n, V.nn)
    {
        st2(V.vg, n, gvel2(V, V.v, n));
        int c = V.contact[n];
        if (c == IFEA_FREE) continue;
        double r0 = V.r[dof2(V, n, 0)], r1 = V.r[dof2(V, n, 1)];
        d2 rg = V.rotated[n] ? add2(scl2(r0, ld2(V.tan, n)), scl2(r1, ld2(V.nrm, n))) : mk2(r0, r1);
        if (c == IFEA_TOP_DIE) acc[0] -= rg.y;
        if (!V.rotated[n]) continue;
        if (c == IFEA_TOP_DIE) mx[1] = rmax(mx[1], r1); else mx[0] = rmax(mx[0], r1);
    }
    const int s1[1] = {T_REACT};
    emit2<1>(V, acc, s1, false);
    const int s2[2] = {T_MAXB, T_MAXT};
    emit2<2>(V, mx, s2, true);
}
__global__ void k2_release(View2 V)
{
    double kept[2] = {0, 0};
    double maxB = rmax(0.0, V.scalars[T_MAXB]), maxT = rmax(0.0, V.scalars[T_MAXT]);
    GS2(n, V.nn)
    {
        int c = V.contact[n];
        if (c == IFEA_FREE) continue;
        if (!V.rotated[n]) {
            kept[c == IFEA_TOP_DIE ? 1 : 0] += 1;
            continue;
        }
        double comp = V.r[dof2(V, n, 1)];
        double thr = 0.02 * (c == IFEA_TOP_DIE ? maxT : maxB);
        if (comp < -thr) V.release[n] = 1;
        else kept[c == IFEA_TOP_DIE ? 1 : 0] += 1;
    }
    const int s[2] = {T_KEPTB, T_KEPTT};
    emit2<2>(V, kept, s, false);
}
__global__ void k2_release_keep(View2 V)
{
    bool kb = V.scalars[T_KEPTB] > 0, kt = V.scalars[T_KEPTT] > 0;
    if (kb && kt) return;
    GS2(n, V.nn)
    {
        int c = V.contact[n];
        if ((!kt && c == IFEA_TOP_DIE) || (!kb && c == IFEA_BOTTOM_DIE)) V.release[n] = 0;
    }
}

// Quality (:900-914)
__device__ double quality2(const View2 &V, const double *x, int e)
{
    double q = DBL_MAX;
    for (int a = 0; a < 4; a++) {
        d2 p = ld2(x, V.conn[4 * e + a]);
        d2 nx = sub2(ld2(x, V.conn[4 * e + (a + 1) % 4]), p);
        d2 pv = sub2(ld2(x, V.conn[4 * e + (a + 3) % 4]), p);
        double l = len2(nx) * len2(pv);
        q = rmin(q, l > 0 ? cross2(nx, pv) / l : -1);
    }
    return q;
}

// TryUpdate (:789-864), allowFold = false: predicted positions and contact
__global__ void k2_predict(View2 V, double dt, double gapT, double tol_sep, double *xT, uint8_t *cT)
{
    double mx[1] = {0};
    GS2(n, V.nn)
    {
        bool axis = V.is_axis[n];
        d2 p = add2(ld2(V.x, n), scl2(dt, ld2(V.vg, n)));
        if (axis) p = mk2(0, p.y);
        int c = V.contact[n];
        uint8_t ct = IFEA_FREE;
        if (c != IFEA_FREE && !V.release[n]) {
            const Profile &sf = surf2(V, c);
            double off = off2(c, gapT);
            if (prof_clearance(sf, p, off) > tol_sep) ct = IFEA_FREE;
            else {
                p = axis ? mk2(0, prof_height(sf, 0) + off) : prof_project(sf, p, off, nullptr);
                ct = (uint8_t)c;
            }
        } else {
            double cb = prof_clearance(V.die[0], p, 0), ctp = prof_clearance(V.die[1], p, gapT);
            if (cb < 0 || ctp < 0) {
                int hit = cb <= ctp ? IFEA_BOTTOM_DIE : IFEA_TOP_DIE;
                const Profile &sf = surf2(V, hit);
                double off = off2(hit, gapT);
                d2 q = axis ? mk2(0, prof_height(sf, 0) + off) : prof_project(sf, p, off, nullptr);
                mx[0] = rmax(mx[0], len2(sub2(q, p)));
                p = q;
                ct = (uint8_t)hit;
            }
        }
        st2(xT, n, p);
        cT[n] = ct;
    }
    const int s[1] = {T_MAXPEN};
    emit2<1>(V, mx, s, true);
}

__global__ void k2_quality(View2 V, const double *x, double thr)
{
    double mx[1] = {-INFINITY};
    GS2(e, V.ne)
    {
        double q = quality2(V, x, e);
        mx[0] = fmax(mx[0], -q);
        if (q <= thr) atomicMin(&V.err[1], e);
    }
    const int s[1] = {T_MINQ};
    emit2<1>(V, mx, s, true);
}

// eps += rate dt; Cockcroft–Latham damage with Principal.Max2D (AccumulateDamage :724-734)
__global__ void k2_strain_damage(View2 V, double dt)
{
    GS2(e, V.ne)
    {
        V.eps[e] += V.el_rate[e] * dt;
        double sig = V.el_sig[e];
        if (!(sig > 0) || V.el_rate[e] <= V.rate_cut) continue;
        double m = V.el_mean[e];
        double xx = V.el_dev[4 * e] + m, yy = V.el_dev[4 * e + 1] + m, xy = V.el_dev[4 * e + 3], zz = V.el_dev[4 * e + 2] + m;
        double c = 0.5 * (xx + yy), r = sqrt(0.25 * (xx - yy) * (xx - yy) + xy * xy);
        double s1 = rmax(c + r, zz);
        if (s1 > 0) V.dmg[e] += s1 / sig * V.el_rate[e] * dt;
    }
}

// Volume (:1399-1413) and the longest boundary edge (RemeshTrigger :971-974) over the loop
__global__ void k2_loop_metrics(View2 V)
{
    double acc[2] = {0, 0}, mx[1] = {0};
    GS2(k, V.nloop)
    {
        d2 a = ld2(V.x, V.loop[k]), b = ld2(V.x, V.loop[(k + 1) % V.nloop]);
        double cr = a.x * b.y - b.x * a.y;
        acc[0] += 0.5 * cr;
        acc[1] += (a.x + b.x) * cr / 6.0;
        mx[0] = rmax(mx[0], len2(sub2(b, a)));
    }
    const int s[2] = {T_AREA, T_MOMENT};
    emit2<2>(V, acc, s, false);
    const int s2[1] = {T_MAXEDGE};
    emit2<1>(V, mx, s2, true);
}

// CaptureFoldOver (:927-962): sequential over the boundary loop, one thread.
__global__ void k2_capture(View2 V, double h, double sin_limit, int *captured)
{
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    int m = V.nloop, cnt = 0;
    bool changed = true;
    for (int pass = 0; pass < 4 && changed; pass++) {
        changed = false;
        for (int k = 0; k < m; k++) {
            int n = V.loop[k];
            int c = V.contact[n];
            if (c == IFEA_FREE) continue;
            int fs[2] = {V.loop[(k + m - 1) % m], V.loop[(k + 1) % m]};
            for (int q = 0; q < 2; q++) {
                int f = fs[q];
                if (V.contact[f] != IFEA_FREE || V.is_axis[f]) continue;
                const Profile &sf = surf2(V, c);
                double off = off2(c, V.gap);
                d2 nrm;
                prof_project(sf, ld2(V.x, n), off, &nrm);
                d2 u = sub2(ld2(V.x, f), ld2(V.x, n));
                double len = len2(u);
                if (len <= 0 || dot2(u, nrm) / len > sin_limit) continue;
                d2 qq = prof_project(sf, ld2(V.x, f), off, nullptr);
                if (len2(sub2(qq, ld2(V.x, f))) > 0.5 * h) continue;
                st2(V.x, f, qq);
                V.contact[f] = (uint8_t)c;
                cnt++;
                changed = true;
            }
        }
    }
    *captured = cnt;
}

__global__ void k2_init_contact(View2 V, double tol)
{
    GS2(k, V.nloop)
    {
        int n = V.loop[k];
        if (prof_clearance(V.die[0], ld2(V.x, n), 0) < tol) V.contact[n] = IFEA_BOTTOM_DIE;
        else if (prof_clearance(V.die[1], ld2(V.x, n), V.gap) < tol) V.contact[n] = IFEA_TOP_DIE;
    }
}

}  // namespace

struct Forging2D {
    ifea2d_params P;
    cudaStream_t st = nullptr;
    std::string err;
    QuadTopology topo;
    std::vector<double> bottom, top;
    bool axi;
    double ram, rate_ref, rate_cut, sig_ref, k_pen, u0, h, gap0, gap, time = 0, vol0 = 0, last_rel = INFINITY, seat;
    double load = 0, reaction = 0, power = 0;
    int step_index = 0, iterations = 0, remesh_requests = 0, captured = 0, n_factor = 0;
    DBuf<int32_t> d_conn, d_eq, d_loop, d_owner, d_cptr, d_cidx, d_csrc, d_dptr, d_dsrc, d_nedge, d_err, d_cnt;
    DBuf<uint8_t> d_axis, d_contact, d_rot, d_fixed, d_release, d_cT;
    DBuf<double> d_x, d_xT, d_vg, d_v[2], d_r, d_dv, d_band, d_ke, d_re, d_eps, d_dmg, d_eldev, d_elsig, d_elrate,
        d_elmean, d_tan, d_nrm, d_fixedval, d_kfric, d_afric, d_partials, d_scalars, d_prof[2], d_piv;
    int vcur = 0;
    HostPinned<double> hs;
    HostPinned<int32_t> hi;
    band::Plan bplan;

    Forging2D(const ifea2d_params &p, int nb, const double *bxy, int ntp, const double *txy) : P(p)
    {
        cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        axi = P.axisymmetric != 0;
        auto prof = [](int n, const double *xy, std::vector<double> &out) {
            if (n < 2) throw Failure(IFEA_INPUT_INVALID, "A die profile needs at least two points.");
            for (int i = 1; i < n; i++)
                if (!(xy[2 * i] > xy[2 * i - 2]))
                    throw Failure(IFEA_INPUT_INVALID, "Die profile x-coordinates must be strictly increasing. Use a draft angle on walls.");
            out.assign(xy, xy + 2 * n);
            if (xy[2 * n - 2] < 1000.0) { out.push_back(1000.0); out.push_back(xy[2 * n - 1]); }
        };
        prof(nb, bxy, bottom);
        prof(ntp, txy, top);
        auto range = [](const std::vector<double> &pp, double x0, double x1, double *mn, double *mx) {
            int n = (int)pp.size() / 2;
            auto H = [&](double x) {
                if (x <= pp[0]) return pp[1];
                if (x >= pp[2 * (n - 1)]) return pp[2 * (n - 1) + 1];
                int lo = 0, hi = n - 1;
                while (hi - lo > 1) {
                    int mid = (lo + hi) >> 1;
                    if (pp[2 * mid] <= x) lo = mid; else hi = mid;
                }
                double t = (x - pp[2 * lo]) / (pp[2 * hi] - pp[2 * lo]);
                return pp[2 * lo + 1] + t * (pp[2 * hi + 1] - pp[2 * lo + 1]);
            };
            double a = H(x0), b = H(x1);
            double lo = rmin(a, b), hi = rmax(a, b);
            for (int i = 0; i < n; i++) {
                if (pp[2 * i] <= x0 || pp[2 * i] >= x1) continue;
                lo = rmin(lo, pp[2 * i + 1]);
                hi = rmax(hi, pp[2 * i + 1]);
            }
            *mn = lo; *mx = hi;
        };
        double r0 = P.radius, h0 = P.height, mn, mx;
        range(bottom, 0, r0, &mn, &mx);
        seat = mx;
        std::vector<double> x;
        std::string e = topo.build_structured(P.nx, P.nz, r0, seat, h0, x);
        if (!e.empty()) throw Failure(IFEA_INPUT_INVALID, e);
        h = rmin(r0 / P.nx, h0 / P.nz);
        double tmin, tmax;
        range(top, 0, r0, &tmin, &tmax);
        gap0 = gap = seat + h0 - tmin;
        ram = P.ram;
        rate_ref = ram / h0;
        rate_cut = 1e-3 * rate_ref;
        sig_ref = flow_stress(P.C, P.N, P.M, P.eps0, 0, rate_ref);
        k_pen = 1e5 * sig_ref / rate_ref;
        u0 = 5e-3 * ram;
        int nn = topo.nn, ne = topo.ne, nd = topo.ndof;
        d_conn.upload(topo.conn, st); d_eq.upload(topo.eq, st); d_loop.upload(topo.loop, st);
        d_owner.upload(topo.loop_owner, st); d_cptr.upload(topo.cell_ptr, st); d_cidx.upload(topo.cell_idx, st);
        d_csrc.upload(topo.cell_src, st); d_dptr.upload(topo.dof_ptr, st); d_dsrc.upload(topo.dof_src, st);
        d_nedge.upload(topo.node_edge, st); d_axis.upload(topo.is_axis, st);
        d_x.upload(x, st);
        d_prof[0].upload(bottom, st);
        d_prof[1].upload(top, st);
        d_xT.resize(2 * (size_t)nn); d_vg.resize(2 * (size_t)nn); d_v[0].resize(nd); d_v[1].resize(nd); d_r.resize(nd);
        d_dv.resize(nd); d_band.resize(topo.band_size()); d_ke.resize(64 * (size_t)ne); d_re.resize(8 * (size_t)ne);
        d_eps.resize(ne); d_dmg.resize(ne); d_eldev.resize(4 * (size_t)ne); d_elsig.resize(ne); d_elrate.resize(ne);
        d_elmean.resize(ne); d_tan.resize(2 * (size_t)nn); d_nrm.resize(2 * (size_t)nn); d_fixedval.resize(nd);
        d_kfric.resize(nn); d_afric.resize(nn); d_contact.resize(nn); d_rot.resize(nn); d_fixed.resize(nd);
        d_release.resize(nn); d_cT.resize(nn); d_partials.resize((size_t)T_COUNT * kReduceBlocks);
        d_scalars.resize(T_COUNT); d_err.resize(4); d_cnt.resize(4); d_piv.resize(2);
        for (auto *b : {&d_eps, &d_dmg, &d_eldev, &d_elrate, &d_elmean, &d_v[0], &d_v[1], &d_r, &d_dv}) b->zero(st);
        d_contact.zero(st); d_release.zero(st); d_rot.zero(st);
        std::vector<double> sig(ne, sig_ref);
        d_elsig.upload(sig, st);
        hs.resize(T_COUNT + 4);
        hi.resize(8);
        bplan = band::plan(nd, topo.half_band);
        ensure_dynamic_smem(band::kernel_of(bplan), bplan.bytes);
        // initial contact on the boundary loop (tol 1e-3 h) and velocity field (:130-139)
        View2 V = view();
        k2_init_contact<<<grid(topo.nloop), 128, 0, st>>>(V, 1e-3 * h);
        double sx = axi ? 0.5 : 1.0;
        std::vector<double> vg(2 * (size_t)nn);
        for (int n = 0; n < nn; n++) {
            vg[2 * n] = sx * rate_ref * x[2 * n];
            vg[2 * n + 1] = -rate_ref * (x[2 * n + 1] - seat);
        }
        d_vg.upload(vg, st);
        vol0 = volume();
    }
    ~Forging2D()
    {
        if (st) {
            cudaStreamSynchronize(st);
            cudaStreamDestroy(st);
        }
    }

    int grid(int n) const { return std::max(1, std::min((n + 127) / 128, 4 * 148)); }

    View2 view()
    {
        View2 V;
        memset(&V, 0, sizeof V);
        V.nn = topo.nn; V.ne = topo.ne; V.ndof = topo.ndof; V.hb = topo.half_band; V.nloop = topo.nloop; V.axi = axi;
        V.conn = d_conn; V.eq = d_eq; V.loop = d_loop; V.loop_owner = d_owner; V.cell_ptr = d_cptr; V.cell_idx = d_cidx;
        V.cell_src = d_csrc; V.dof_ptr = d_dptr; V.dof_src = d_dsrc; V.node_edge = d_nedge;
        V.ncell = (int)topo.cell_idx.size(); V.is_axis = d_axis;
        V.x = d_x; V.vg = d_vg; V.v = d_v[vcur]; V.v_trial = d_v[1 - vcur]; V.r = d_r; V.dv = d_dv; V.band = d_band;
        V.ke = d_ke; V.re = d_re; V.eps = d_eps; V.dmg = d_dmg; V.el_dev = d_eldev; V.el_sig = d_elsig;
        V.el_rate = d_elrate; V.el_mean = d_elmean; V.tan = d_tan; V.nrm = d_nrm; V.fixed_val = d_fixedval;
        V.k_fric = d_kfric; V.a_fric = d_afric; V.contact = d_contact; V.rotated = d_rot; V.fixed = d_fixed;
        V.release = d_release; V.partials = d_partials; V.scalars = d_scalars; V.err = d_err;
        V.die[0] = Profile{0, (int)bottom.size() / 2, d_prof[0].p};
        V.die[1] = Profile{1, (int)top.size() / 2, d_prof[1].p};
        V.C = P.C; V.N = P.N; V.M = P.M; V.eps0 = P.eps0; V.friction = P.friction; V.ram = ram;
        V.rate_cut = rate_cut; V.k_pen = k_pen; V.u0 = u0; V.gap = gap; V.length = P.length;
        return V;
    }
    void finalize(std::initializer_list<int> codes)
    {
        SlotList2 l;
        l.n = 0;
        for (int c : codes) l.code[l.n++] = c;
        k2_finalize<<<l.n, 256, 0, st>>>(d_partials, d_scalars, l);
    }
    static int MX(int s) { return s | (1 << 16); }
    const double *read()
    {
        cuda_check(cudaMemcpyAsync(hs.p, d_scalars.p, T_COUNT * sizeof(double), cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaStreamSynchronize(st), "cudaStreamSynchronize");
        return hs.p;
    }
    void reset_err()
    {
        int32_t v[4] = {INT_MAX, INT_MAX, 0, 0};
        cuda_check(cudaMemcpyAsync(d_err.p, v, sizeof v, cudaMemcpyHostToDevice, st), "H2D");
        cuda_check(cudaStreamSynchronize(st), "sync");
    }
    void read_err(int32_t *o)
    {
        cuda_check(cudaMemcpyAsync(hi.p, d_err.p, 4 * sizeof(int32_t), cudaMemcpyDeviceToHost, st), "D2H");
        cuda_check(cudaStreamSynchronize(st), "sync");
        memcpy(o, hi.p, 16);
    }

    double volume()
    {
        View2 V = view();
        k2_loop_metrics<<<kReduceBlocks, 128, 0, st>>>(V);
        finalize({T_AREA, T_MOMENT, MX(T_MAXEDGE)});
        const double *s = read();
        return axi ? 2 * M_PI * s[T_MOMENT] : 2 * P.length * s[T_AREA];
    }

    void prepare()
    {
        View2 V = view();
        k2_frames<<<grid(topo.nn), 128, 0, st>>>(V);
        k2_guess<<<grid(topo.nn), 128, 0, st>>>(V);
        cuda_check(cudaGetLastError(), "prepare launch");
    }

    // Assemble (:471-538); matrix: band + constraints (bc) as SolveVelocity does before factorising.
    double assemble(bool matrix, int newton, const double *v, bool bc, double *pw)
    {
        View2 V = view();
        reset_err();
        if (matrix) k2_element<1><<<kReduceBlocks, 128, 0, st>>>(V, v, newton, 1);
        else k2_element<0><<<kReduceBlocks, 128, 0, st>>>(V, v, newton, 1);
        if (matrix) {
            d_band.zero(st);
            k2_band<<<grid(V.ncell), 128, 0, st>>>(V);
        }
        k2_residual_friction<<<kReduceBlocks, 128, 0, st>>>(V, v, newton, matrix, bc);
        if (matrix && bc) k2_constrain<<<grid((int)std::min<int64_t>(topo.band_size(), INT_MAX)), 128, 0, st>>>(V);
        finalize({T_ENERGY, T_POWER, T_EFRIC, T_PFRIC, T_RNORM2});
        const double *s = read();
        int32_t e4[4];
        read_err(e4);
        if (e4[0] != INT_MAX)
            throw Failure(IFEA_MESH_DISTORTED, fmt2("Element %d has a non-positive Jacobian at step %d.", e4[0], step_index));
        if (pw) *pw = s[T_POWER] + s[T_PFRIC];
        return s[T_ENERGY] + s[T_EFRIC];
    }

    void factor_solve(double *rhs)
    {
        cuda_check(cudaMemsetAsync(d_err.p + 2, 0xff, sizeof(int32_t), st), "memset");
        band::launch(bplan, topo.ndof, topo.half_band, d_band, rhs, d_err.p + 2, d_piv, st);
        cuda_check(cudaGetLastError(), "band factor launch");
        int32_t e4[4];
        read_err(e4);
        n_factor++;
        if (e4[2] >= 0) {
            double piv = 0;
            d_piv.download(&piv, 1, st);
            cuda_check(cudaStreamSynchronize(st), "sync");
            throw Failure(IFEA_NOT_SPD, fmt2("Stiffness matrix not positive definite at equation %d (pivot %.3E). The billet is probably unrestrained.", e4[2], piv));
        }
    }

    // SolveVelocity (:403-461)
    int solve_velocity(bool picard_fallback, bool *converged, const volatile int32_t *cancel)
    {
        *converged = false;
        last_rel = INFINITY;
        int it, damped = 0, picard_until = 2, n = topo.ndof;
        for (it = 1; it <= P.max_iter; it++) {
            if (cancel && *cancel) throw Failure(IFEA_CANCELLED, "The operation was canceled.");
            int newton = it > picard_until;
            double e0 = assemble(true, newton, d_v[vcur], true, nullptr);
            k2_neg<<<grid(n), 128, 0, st>>>(n, d_dv, d_r);
            factor_solve(d_dv);
            View2 V = view();
            k2_dots<<<kReduceBlocks, 128, 0, st>>>(V, d_r, d_dv, d_dv);
            finalize({T_DOT, T_NDV});
            const double *s = read();
            double slope = s[T_DOT], ndv = sqrt(s[T_NDV]);
            double beta = 1.0;
            for (int ls = 0; ls < 8; ls++) {
                k2_axpy<<<grid(n), 128, 0, st>>>(n, d_v[1 - vcur], d_v[vcur], d_dv, beta);
                double e1 = assemble(false, 0, d_v[1 - vcur], false, nullptr);
                if (e1 <= e0 + 1e-4 * beta * slope + 1e-11 * fabs(e0)) break;
                beta *= 0.5;
            }
            vcur = 1 - vcur;
            V = view();
            k2_dots<<<kReduceBlocks, 128, 0, st>>>(V, d_v[vcur], d_v[vcur], nullptr);
            finalize({T_DOT});
            double nv = sqrt(read()[T_DOT]);
            double rel = beta * ndv / rmax(nv, 1e-30);
            last_rel = rel;
            if (std::isnan(rel)) throw Failure(IFEA_DIVERGED, fmt2("Velocity solution became NaN at step %d.", step_index));
            if (rel < P.tol) {
                *converged = true;
                return it;
            }
            damped = newton && beta < 0.5 ? damped + 1 : 0;
            if (picard_fallback && damped >= 3) {
                picard_until = it + 4;
                damped = 0;
            }
        }
        return it - 1;
    }

    double final_evaluation(double *reaction_out)
    {
        double pw = 0;
        assemble(false, 0, d_v[vcur], false, &pw);
        View2 V = view();
        k2_final<<<kReduceBlocks, 128, 0, st>>>(V);
        finalize({T_REACT, MX(T_MAXB), MX(T_MAXT)});
        k2_release<<<kReduceBlocks, 128, 0, st>>>(V);
        finalize({T_KEPTB, T_KEPTT});
        k2_release_keep<<<grid(topo.nn), 128, 0, st>>>(V);
        reaction = read()[T_REACT];
        if (reaction_out) *reaction_out = reaction;
        return pw;
    }

    double min_quality(const double *x)
    {
        View2 V = view();
        k2_quality<<<kReduceBlocks, 128, 0, st>>>(V, x, -INFINITY);
        finalize({MX(T_MINQ)});
        return -read()[T_MINQ];
    }

    bool try_update(double dt, std::string &why)
    {
        double gapT = rmax(0, gap - ram * dt);
        if (gapT < 1e-9) gapT = 0;
        View2 V = view();
        k2_predict<<<kReduceBlocks, 128, 0, st>>>(V, dt, gapT, 0.05 * h, d_xT, d_cT);
        finalize({MX(T_MAXPEN)});
        double maxPen = read()[T_MAXPEN];
        if (maxPen > 0.5 * h) {
            why = fmt2("die penetration %.3f mm exceeds h/2", maxPen);
            return false;
        }
        reset_err();
        k2_quality<<<kReduceBlocks, 128, 0, st>>>(V, d_xT, 0.002);
        int32_t e4[4];
        read_err(e4);
        if (e4[1] != INT_MAX) {
            why = fmt2("element %d folded", e4[1]);
            return false;
        }
        swap_buf(d_x, d_xT);
        swap_buf(d_contact, d_cT);
        gap = gapT;
        time += dt;
        return true;
    }

    // Advance (:215-290) with remeshing unavailable
    void step(ifea_step_info *info, const volatile int32_t *cancel)
    {
        if (gap <= 1e-9) throw Failure(IFEA_BAD_STATE, "Simulation already reached the closed-die position.");
        step_index++;
        if (min_quality(d_x) < 0.15) remesh_requests++;
        else {
            volume();
            if (hs.p[T_MAXEDGE] > 2.5 * h) remesh_requests++;
        }
        int its = 0;
        bool ok = false;
        double dt = 0;
        std::string why;
        for (int pass = 0; pass < 2 && !ok; pass++) {
            prepare();
            bool conv = false;
            its = solve_velocity(false, &conv, cancel);
            if (!conv && last_rel >= 1e-3) {
                View2 V = view();
                k2_guess<<<grid(topo.nn), 128, 0, st>>>(V);
                its += solve_velocity(true, &conv, cancel);
            }
            if (!conv && !(last_rel < 1e-3))
                throw Failure(IFEA_DIVERGED, fmt2("Newton-Raphson diverged at step %d (stroke %.3f mm): |dv|/|v| = %.2E after %d iterations.",
                                                  step_index, gap0 - gap, last_rel, its));
            double pw = final_evaluation(&reaction);
            power = pw;
            load = pw / ram;
            dt = rmin(P.ds, gap) / ram;
            if (gap - ram * dt < 0.05 * P.ds) dt = gap / ram;
            for (int attempt = 0; attempt < 4 && !ok; attempt++) {
                double dta = dt / (1 << attempt);
                ok = try_update(dta, why);
                if (ok) dt = dta;
            }
            if (!ok) {
                remesh_requests++;
                break;
            }
        }
        if (!ok)
            throw Failure(IFEA_MESH_DISTORTED, fmt2("Mesh distortion at step %d (stroke %.3f mm): %s. Results up to the previous increment are kept; refine h or reduce ds.",
                                                    step_index, gap0 - gap, why.c_str()));
        View2 V = view();
        k2_strain_damage<<<grid(topo.ne), 128, 0, st>>>(V, dt);
        // CaptureFoldOver with the remesh rejected: the capture is undone when it leaves a poor element (:279-285)
        cuda_check(cudaMemcpyAsync(d_xT.p, d_x.p, 2 * topo.nn * sizeof(double), cudaMemcpyDeviceToDevice, st), "D2D");
        cuda_check(cudaMemcpyAsync(d_cT.p, d_contact.p, topo.nn, cudaMemcpyDeviceToDevice, st), "D2D");
        d_cnt.zero(st);
        k2_capture<<<1, 1, 0, st>>>(V, h, sin(25 * M_PI / 180), d_cnt);
        int32_t c4[4];
        d_cnt.download(c4, 4, st);
        cuda_check(cudaStreamSynchronize(st), "sync");
        if (c4[0] > 0) {
            remesh_requests++;
            if (min_quality(d_x) <= 0.05) {
                swap_buf(d_x, d_xT);
                swap_buf(d_contact, d_cT);
            } else {
                captured += c4[0];
            }
        }
        iterations = its;
        double vol = volume();
        if (info) {
            info->step = step_index;
            info->iterations = its;
            info->load = load;
            info->reaction = reaction;
            info->stroke = gap0 - gap;
            info->gap = gap;
            info->time = time;
            info->dt = dt;
            info->volume_change_pct = 100.0 * (vol - vol0) / vol0;
            info->last_rel = last_rel;
            info->n_factor = n_factor;
            info->n_pcg = 0;
            info->remesh_requests = remesh_requests;
            info->cutbacks = 0;
        }
    }

    struct Ref {
        void *p;
        size_t count;
        int bytes;
    };
    Ref array(const std::string &nm)
    {
        size_t nn = topo.nn, ne = topo.ne, nd = topo.ndof;
#define A(name, buf, cnt) if (nm == name) return Ref{(void *)(buf).p, (size_t)(cnt), (int)sizeof(*(buf).p)};
        A("x", d_x, 2 * nn) A("vg", d_vg, 2 * nn) A("v", d_v[vcur], nd) A("r", d_r, nd) A("dv", d_dv, nd)
        A("eps", d_eps, ne) A("dmg", d_dmg, ne) A("el_sig", d_elsig, ne) A("el_rate", d_elrate, ne)
        A("el_mean", d_elmean, ne) A("el_dev", d_eldev, 4 * ne) A("contact", d_contact, nn) A("release", d_release, nn)
        A("rotated", d_rot, nn) A("fixed", d_fixed, nd) A("fixed_val", d_fixedval, nd) A("tan", d_tan, 2 * nn)
        A("nrm", d_nrm, 2 * nn) A("k_fric", d_kfric, nn) A("a_fric", d_afric, nn) A("band", d_band, topo.band_size())
#undef A
        if (nm == "eq") return Ref{(void *)topo.eq.data(), topo.eq.size(), -4};
        if (nm == "loop") return Ref{(void *)topo.loop.data(), topo.loop.size(), -4};
        if (nm == "loop_owner") return Ref{(void *)topo.loop_owner.data(), topo.loop_owner.size(), -4};
        if (nm == "conn") return Ref{(void *)topo.conn.data(), topo.conn.size(), -4};
        throw Failure(IFEA_INPUT_INVALID, "unknown array name '" + nm + "'");
    }
    double scalar(const std::string &nm)
    {
#define S(name, v) if (nm == name) return (double)(v);
        S("gap", gap) S("gap0", gap0) S("time", time) S("load", load) S("reaction", reaction) S("power", power)
        S("iterations", iterations) S("last_rel", last_rel) S("vol0", vol0) S("step_index", step_index)
        S("half_band", topo.half_band) S("rate_ref", rate_ref) S("k_pen", k_pen) S("h", h) S("nn", topo.nn)
        S("ne", topo.ne) S("ndof", topo.ndof) S("remesh_requests", remesh_requests) S("n_factor", n_factor)
        S("captured", captured) S("nloop", topo.nloop)
#undef S
        if (nm == "volume") return volume();
        if (nm == "min_quality") return min_quality(d_x);
        throw Failure(IFEA_INPUT_INVALID, "unknown scalar name '" + nm + "'");
    }
};

}  // namespace ifea

using ifea::Failure;
using ifea::Forging2D;

struct ifea2d {
    Forging2D *s = nullptr;
    std::string err;
};

template <typename F>
static ifea_status guard2(ifea2d *c, F &&f)
{
    if (!c || !c->s) return IFEA_INPUT_INVALID;
    try {
        f(*c->s);
        c->err.clear();
        return IFEA_OK;
    } catch (Failure &e) {
        c->err = e.what();
        return e.status;
    } catch (std::exception &e) {
        c->err = e.what();
        return IFEA_CUDA_ERROR;
    }
}

extern "C" {

ifea_status ifea2d_create(const ifea2d_params *params, int32_t n_bottom, const double *bottom_xy, int32_t n_top,
                          const double *top_xy, ifea2d **out)
{
    if (!params || !bottom_xy || !top_xy || !out) return IFEA_INPUT_INVALID;
    *out = nullptr;
    if (!(params->radius > 0) || !(params->height > 0) || !(params->ram > 0) || !(params->ds > 0) || params->nx < 1 ||
        params->nz < 1 || params->max_iter < 1)
        return IFEA_INPUT_INVALID;
    ifea2d *c = new ifea2d;
    try {
        c->s = new Forging2D(*params, n_bottom, bottom_xy, n_top, top_xy);
    } catch (Failure &e) {
        delete c;
        return e.status;
    } catch (...) {
        delete c;
        return IFEA_CUDA_ERROR;
    }
    *out = c;
    return IFEA_OK;
}

void ifea2d_destroy(ifea2d *ctx)
{
    if (!ctx) return;
    delete ctx->s;
    delete ctx;
}

const char *ifea2d_last_error(const ifea2d *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

ifea_status ifea2d_step(ifea2d *ctx, ifea_step_info *info, const volatile int32_t *cancel)
{
    return guard2(ctx, [&](Forging2D &s) { s.step(info, cancel); });
}

ifea_status ifea2d_prepare(ifea2d *ctx)
{
    return guard2(ctx, [&](Forging2D &s) { s.prepare(); });
}

ifea_status ifea2d_assemble(ifea2d *ctx, int32_t matrix, int32_t newton, const double *v_host, double *energy, double *power)
{
    return guard2(ctx, [&](Forging2D &s) {
        const double *v = s.d_v[s.vcur];
        if (v_host) {
            s.d_v[1 - s.vcur].upload(v_host, s.topo.ndof, s.st);
            v = s.d_v[1 - s.vcur];
        }
        double e = s.assemble(matrix != 0, newton, v, false, power);
        if (energy) *energy = e;
    });
}

ifea_status ifea2d_solve_velocity(ifea2d *ctx, int32_t picard_fallback, int32_t *iterations, int32_t *converged)
{
    return guard2(ctx, [&](Forging2D &s) {
        bool conv = false;
        int it = s.solve_velocity(picard_fallback != 0, &conv, nullptr);
        if (iterations) *iterations = it;
        if (converged) *converged = conv;
    });
}

ifea_status ifea2d_array_size(ifea2d *ctx, const char *name, int64_t *count, int32_t *elem_bytes)
{
    if (!name) return IFEA_INPUT_INVALID;
    return guard2(ctx, [&](Forging2D &s) {
        auto a = s.array(name);
        if (count) *count = (int64_t)a.count;
        if (elem_bytes) *elem_bytes = a.bytes < 0 ? -a.bytes : a.bytes;
    });
}

ifea_status ifea2d_get_array(ifea2d *ctx, const char *name, void *dst, int64_t count)
{
    if (!name || !dst) return IFEA_INPUT_INVALID;
    return guard2(ctx, [&](Forging2D &s) {
        auto a = s.array(name);
        if ((size_t)count != a.count) throw Failure(IFEA_INPUT_INVALID, "array size mismatch");
        if (a.bytes < 0) {
            memcpy(dst, a.p, a.count * (size_t)(-a.bytes));
            return;
        }
        ifea::cuda_check(cudaMemcpyAsync(dst, a.p, a.count * (size_t)a.bytes, cudaMemcpyDeviceToHost, s.st), "D2H");
        ifea::cuda_check(cudaStreamSynchronize(s.st), "sync");
    });
}

ifea_status ifea2d_get_scalar(ifea2d *ctx, const char *name, double *value)
{
    if (!name || !value) return IFEA_INPUT_INVALID;
    return guard2(ctx, [&](Forging2D &s) { *value = s.scalar(name); });
}

// SymmetricBandMatrix.Factorize + Solve on the GPU with host buffers (band overwritten by L, rhs by x).
ifea_status ifea_band_factor_solve(int32_t n, int32_t half_bandwidth, double *band, double *rhs, int32_t *bad_row,
                                   double *pivot)
{
    if (n <= 0 || half_bandwidth < 0 || !band) return IFEA_INPUT_INVALID;
    int b = std::min(half_bandwidth, n - 1);
    cudaStream_t st = nullptr;
    try {
        ifea::cuda_check(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking), "cudaStreamCreate");
        ifea::DBuf<double> a, x, piv;
        ifea::DBuf<int32_t> err;
        a.upload(band, (size_t)n * (b + 1), st);
        if (rhs) x.upload(rhs, n, st);
        piv.resize(1);
        err.resize(1);
        ifea::band::Plan plan = ifea::band::plan(n, b);
        ifea::ensure_dynamic_smem(ifea::band::kernel_of(plan), plan.bytes);
        ifea::band::launch(plan, n, b, a, rhs ? x.p : nullptr, err, piv, st);
        ifea::cuda_check(cudaGetLastError(), "band launch");
        int32_t e = -1;
        double pv = 0;
        err.download(&e, 1, st);
        piv.download(&pv, 1, st);
        a.download(band, (size_t)n * (b + 1), st);
        if (rhs) x.download(rhs, n, st);
        ifea::cuda_check(cudaStreamSynchronize(st), "sync");
        cudaStreamDestroy(st);
        if (bad_row) *bad_row = e;
        if (pivot) *pivot = pv;
        return e >= 0 ? IFEA_NOT_SPD : IFEA_OK;
    } catch (Failure &f) {
        if (st) cudaStreamDestroy(st);
        return f.status;
    }
}

}  // extern "C"
