/*
 * o_common.c — shared pieces of the CPU oracle: geometry helpers, height-field die, principal stress,
 * and the band Cholesky (the sparse SPD factorisation is in o_spd.c).
 * TEST INFRASTRUCTURE ONLY (see ifea_oracle.h).
 */
#include "o_internal.h"
#include <float.h>
#include <stdio.h>

/* ThreeD/Vec3.cs:35-56 (Ericson, Real-Time Collision Detection 5.1.5). */
v3 o_closest_on_triangle(v3 p, v3 a, v3 b, v3 c)
{
    v3 ab = vsub(b, a), ac = vsub(c, a), ap = vsub(p, a);
    double d1 = vdot(ab, ap), d2 = vdot(ac, ap);
    if (d1 <= 0 && d2 <= 0) return a;
    v3 bp = vsub(p, b);
    double d3 = vdot(ab, bp), d4 = vdot(ac, bp);
    if (d3 >= 0 && d4 <= d3) return b;
    double vc = d1 * d4 - d3 * d2;
    if (vc <= 0 && d1 >= 0 && d3 <= 0) return vadd(a, vscale(d1 / (d1 - d3), ab));
    v3 cp = vsub(p, c);
    double d5 = vdot(ab, cp), d6 = vdot(ac, cp);
    if (d6 >= 0 && d5 <= d6) return c;
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return vadd(a, vscale(d2 / (d2 - d6), ac));
    double va = d3 * d6 - d5 * d4;
    if (va <= 0 && d4 - d3 >= 0 && d5 - d6 >= 0) return vadd(b, vscale((d4 - d3) / (d4 - d3 + (d5 - d6)), vsub(c, b)));
    double denom = 1 / (va + vb + vc);
    return vadd(vadd(a, vscale(vb * denom, ab)), vscale(vc * denom, ac));
}

/* ThreeD/TetMesh.cs:104 */
double o_tet_volume(v3 a, v3 b, v3 c, v3 d) { return vdot(vsub(b, a), vcross(vsub(c, a), vsub(d, a))) / 6.0; }

/* ThreeD/TetMesh.cs:107-112 */
double o_tet_quality4(v3 a, v3 b, v3 c, v3 d)
{
    double l2 = (vlen2(vsub(b, a)) + vlen2(vsub(c, a)) + vlen2(vsub(d, a)) + vlen2(vsub(c, b)) + vlen2(vsub(d, b)) +
                 vlen2(vsub(d, c))) / 6.0;
    return l2 > 0 ? 6 * sqrt(2.0) * o_tet_volume(a, b, c, d) / pow(l2, 1.5) : -1;
}

double o3d_tet_quality(const double *a, const double *b, const double *c, const double *d)
{
    return o_tet_quality4(V3(a[0], a[1], a[2]), V3(b[0], b[1], b[2]), V3(c[0], c[1], c[2]), V3(d[0], d[1], d[2]));
}

double o_flow_stress(double C, double N, double M, double eps0, double strain, double rate)
{
    return law_stress(C, N, M, eps0, strain, rate);
}

/* Solver/Principal.cs:7-19 */
double o_principal_max3(double xx, double yy, double zz, double xy, double yz, double zx)
{
    double p1 = xy * xy + yz * yz + zx * zx;
    double q = (xx + yy + zz) / 3;
    if (p1 < 1e-30 * (xx * xx + yy * yy + zz * zz + 1e-300)) return dmax(xx, dmax(yy, zz));
    double p2 = (xx - q) * (xx - q) + (yy - q) * (yy - q) + (zz - q) * (zz - q) + 2 * p1;
    double p = sqrt(p2 / 6);
    double bxx = (xx - q) / p, byy = (yy - q) / p, bzz = (zz - q) / p, bxy = xy / p, byz = yz / p, bzx = zx / p;
    double detB = bxx * (byy * bzz - byz * byz) - bxy * (bxy * bzz - byz * bzx) + bzx * (bxy * byz - byy * bzx);
    double r = dclamp(detB / 2, -1, 1);
    double phi = acos(r) / 3;
    return q + 2 * p * cos(phi);
}

/* ------------------------------------------------------------------ height-field die */

/* ThreeD/HeightFieldDie.cs:100-107 */
double hf_height(const o_hfdie *d, double x, double y)
{
    double fx = dclamp((x - d->x0) / d->dx, 0, d->nx), fy = dclamp((y - d->y0) / d->dx, 0, d->ny);
    int i = imin((int)fx, d->nx - 1), j = imin((int)fy, d->ny - 1);
    double u = fx - i, v = fy - j;
    int w = d->nx + 1;
    return (1 - u) * (1 - v) * d->h[j * w + i] + u * (1 - v) * d->h[j * w + i + 1] + (1 - u) * v * d->h[(j + 1) * w + i] +
           u * v * d->h[(j + 1) * w + i + 1];
}

/* ThreeD/HeightFieldDie.cs:130-134 */
double hf_clearance(const o_hfdie *d, v3 p, double offset)
{
    double h = hf_height(d, p.x, p.y) + offset;
    return d->side == 0 ? p.z - h : h - p.z;
}

static v3 hf_vertex(const o_hfdie *d, int i, int j, double offset)
{
    return V3(d->x0 + i * d->dx, d->y0 + j * d->dx, d->h[j * (d->nx + 1) + i] + offset);
}

/* ThreeD/HeightFieldDie.cs:157-191 */
v3 hf_project(const o_hfdie *d, v3 p, double offset, v3 *normal)
{
    double reach = fabs(hf_clearance(d, p, offset)) + 1.5 * d->dx;
    int i0 = iclamp((int)floor((p.x - reach - d->x0) / d->dx), 0, d->nx - 1);
    int i1 = iclamp((int)floor((p.x + reach - d->x0) / d->dx), 0, d->nx - 1);
    int j0 = iclamp((int)floor((p.y - reach - d->y0) / d->dx), 0, d->ny - 1);
    int j1 = iclamp((int)floor((p.y + reach - d->y0) / d->dx), 0, d->ny - 1);
    double best = DBL_MAX;
    v3 bestQ = p;
    v3 bestN = d->side == 0 ? V3(0, 0, 1) : vneg(V3(0, 0, 1));
    for (int j = j0; j <= j1; j++) {
        for (int i = i0; i <= i1; i++) {
            v3 a = hf_vertex(d, i, j, offset), b = hf_vertex(d, i + 1, j, offset);
            v3 c = hf_vertex(d, i + 1, j + 1, offset), dd = hf_vertex(d, i, j + 1, offset);
            v3 tri[2][3] = {{a, b, c}, {a, c, dd}};
            for (int t = 0; t < 2; t++) {
                v3 q = o_closest_on_triangle(p, tri[t][0], tri[t][1], tri[t][2]);
                double d2 = vlen2(vsub(q, p));
                if (d2 >= best) continue;
                best = d2;
                bestQ = q;
                v3 n = vnormalized(vcross(vsub(tri[t][1], tri[t][0]), vsub(tri[t][2], tri[t][0])));
                bestN = d->side == 0 ? n : vneg(n);
            }
        }
    }
    *normal = bestN;
    return bestQ;
}

/* ------------------------------------------------------------------ band Cholesky (Solver/SymmetricBandMatrix.cs) */
struct oband {
    int n, b, w;
    double *a;
    int factored;
};

oband *oband_create(int n, int half_bandwidth)
{
    if (n <= 0) return NULL;
    oband *m = (oband *)calloc(1, sizeof(oband));
    m->n = n;
    m->b = imin(half_bandwidth, n - 1);
    m->w = m->b + 1;
    m->a = (double *)calloc((size_t)n * m->w, sizeof(double));
    return m;
}

void oband_destroy(oband *m)
{
    if (!m) return;
    free(m->a);
    free(m);
}

int oband_bandwidth(const oband *m) { return m->b; }
static inline int64_t bidx(const oband *m, int i, int j) { return (int64_t)i * m->w + (j - i + m->b); }

/* SymmetricBandMatrix.cs:36-41 */
int oband_add(oband *m, int i, int j, double v)
{
    if (j > i) { int t = i; i = j; j = t; }
    if (i - j > m->b) return -1;
    m->a[bidx(m, i, j)] += v;
    return 0;
}

double oband_get(const oband *m, int i, int j)
{
    if (j > i) { int t = i; i = j; j = t; }
    return i - j > m->b ? 0.0 : m->a[bidx(m, i, j)];
}

void oband_clear(oband *m)
{
    memset(m->a, 0, sizeof(double) * (size_t)m->n * m->w);
    m->factored = 0;
}

/* SymmetricBandMatrix.cs:50-57 */
void oband_constrain(oband *m, int i)
{
    int j0 = imax(0, i - m->b);
    for (int j = j0; j < i; j++) m->a[bidx(m, i, j)] = 0;
    int k1 = imin(m->n - 1, i + m->b);
    for (int k = i + 1; k <= k1; k++) m->a[bidx(m, k, i)] = 0;
    m->a[bidx(m, i, i)] = 1.0;
}

/* SymmetricBandMatrix.cs:60-88 */
int oband_factorize(oband *m, double *pivot)
{
    int b = m->b;
    double *a = m->a;
    for (int i = 0; i < m->n; i++) {
        int j0 = imax(0, i - b);
        int64_t rowI = (int64_t)i * m->w - i + b;
        for (int j = j0; j <= i; j++) {
            int64_t rowJ = (int64_t)j * m->w - j + b;
            int k0 = imax(j0, j - b);
            double s = a[rowI + j];
            for (int k = k0; k < j; k++) s -= a[rowI + k] * a[rowJ + k];
            if (j == i) {
                if (!(s > 0) || isnan(s)) {
                    if (pivot) *pivot = s;
                    return i;
                }
                a[rowI + i] = sqrt(s);
            } else {
                a[rowI + j] = s / a[rowJ + j];
            }
        }
    }
    m->factored = 1;
    return -1;
}

/* SymmetricBandMatrix.cs:91-111 */
int oband_solve(oband *m, double *rhs)
{
    if (!m->factored) return -1;
    int b = m->b;
    for (int i = 0; i < m->n; i++) {
        int64_t row = (int64_t)i * m->w - i + b;
        double s = rhs[i];
        for (int k = imax(0, i - b); k < i; k++) s -= m->a[row + k] * rhs[k];
        rhs[i] = s / m->a[row + i];
    }
    for (int i = m->n - 1; i >= 0; i--) {
        int64_t row = (int64_t)i * m->w - i + b;
        double xi = rhs[i] / m->a[row + i];
        rhs[i] = xi;
        for (int k = imax(0, i - b); k < i; k++) rhs[k] -= m->a[row + k] * xi;
    }
    return 0;
}

double *oband_data(oband *m, int64_t *count)
{
    if (count) *count = (int64_t)m->n * m->w;
    return m->a;
}
