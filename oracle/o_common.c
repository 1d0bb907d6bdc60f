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
/* ---- TriMeshSolid (ThreeD/TriMeshSolid.cs:17-82): bucket grids, each cell's triangles in ascending order ---- */
void o_trimesh_free(o_trimesh *m)
{
    free(m->v); free(m->t); free(m->xy_start); free(m->xy_items); free(m->g3_start); free(m->g3_items);
    memset(m, 0, sizeof *m);
}

static int tm_cx2(const o_trimesh *m, double x) { return iclamp((int)((x - m->mn[0]) / m->c2), 0, m->nx2 - 1); }
static int tm_cy2(const o_trimesh *m, double y) { return iclamp((int)((y - m->mn[1]) / m->c2), 0, m->ny2 - 1); }
static int tm_c3(const o_trimesh *m, double v, double lo, int n) { return iclamp((int)((v - lo) / m->c3), 0, n - 1); }

int o_trimesh_build(o_trimesh *m, int nv, const double *v, int nt, const int *tri)
{
    o_trimesh_free(m);
    if (nv < 3 || nt < 1) return -1;
    for (int k = 0; k < 3 * nt; k++)
        if (tri[k] < 0 || tri[k] >= nv) return -1;
    m->nv = nv; m->nt = nt;
    m->v = (double *)malloc(sizeof(double) * 3 * (size_t)nv);
    m->t = (int *)malloc(sizeof(int) * 3 * (size_t)nt);
    memcpy(m->v, v, sizeof(double) * 3 * (size_t)nv);
    memcpy(m->t, tri, sizeof(int) * 3 * (size_t)nt);
    for (int a = 0; a < 3; a++) m->mn[a] = DBL_MAX, m->mx[a] = -DBL_MAX;
    for (int i = 0; i < nv; i++)
        for (int a = 0; a < 3; a++) {
            m->mn[a] = fmin(m->mn[a], v[3 * i + a]);
            m->mx[a] = fmax(m->mx[a], v[3 * i + a]);
        }
    double ex = m->mx[0] - m->mn[0], ey = m->mx[1] - m->mn[1], ez = m->mx[2] - m->mn[2];
    double ext = fmax(ex, fmax(ey, ez));
    m->c2 = fmax(ext / 200, sqrt((ex + 1e-9) * (ey + 1e-9) / imax(nt, 1)) * 2);
    m->nx2 = imax(1, (int)ceil(ex / m->c2) + 1);
    m->ny2 = imax(1, (int)ceil(ey / m->c2) + 1);
    m->c3 = fmax(ext / 120, cbrt((ex + 1e-9) * (ey + 1e-9) * (ez + 1e-9) / imax(nt, 1)) * 2);
    m->gx = imax(1, (int)ceil(ex / m->c3) + 1);
    m->gy = imax(1, (int)ceil(ey / m->c3) + 1);
    m->gz = imax(1, (int)ceil(ez / m->c3) + 1);
    size_t n2 = (size_t)m->nx2 * m->ny2, n3 = (size_t)m->gx * m->gy * m->gz;
    m->xy_start = (int *)calloc(n2 + 1, sizeof(int));
    m->g3_start = (int *)calloc(n3 + 1, sizeof(int));
    int *f2 = NULL, *f3 = NULL;
    for (int pass = 0; pass < 2; pass++) {
        if (pass == 1) {
            for (size_t c = 0; c < n2; c++) m->xy_start[c + 1] += m->xy_start[c];
            for (size_t c = 0; c < n3; c++) m->g3_start[c + 1] += m->g3_start[c];
            m->xy_items = (int *)malloc(sizeof(int) * (size_t)(m->xy_start[n2] + 1));
            m->g3_items = (int *)malloc(sizeof(int) * (size_t)(m->g3_start[n3] + 1));
            f2 = (int *)malloc(sizeof(int) * n2);
            f3 = (int *)malloc(sizeof(int) * n3);
            memcpy(f2, m->xy_start, sizeof(int) * n2);
            memcpy(f3, m->g3_start, sizeof(int) * n3);
        }
        for (int k = 0; k < nt; k++) {
            const double *a = m->v + 3 * m->t[3 * k], *b = m->v + 3 * m->t[3 * k + 1], *c = m->v + 3 * m->t[3 * k + 2];
            double lx = fmin(a[0], fmin(b[0], c[0])), hx = fmax(a[0], fmax(b[0], c[0]));
            double ly = fmin(a[1], fmin(b[1], c[1])), hy = fmax(a[1], fmax(b[1], c[1]));
            double lz = fmin(a[2], fmin(b[2], c[2])), hz = fmax(a[2], fmax(b[2], c[2]));
            for (int j = tm_cy2(m, ly); j <= tm_cy2(m, hy); j++)
                for (int i = tm_cx2(m, lx); i <= tm_cx2(m, hx); i++) {
                    size_t cell = (size_t)j * m->nx2 + i;
                    if (pass == 0) m->xy_start[cell + 1]++;
                    else m->xy_items[f2[cell]++] = k;
                }
            for (int kk = tm_c3(m, lz, m->mn[2], m->gz); kk <= tm_c3(m, hz, m->mn[2], m->gz); kk++)
                for (int j = tm_c3(m, ly, m->mn[1], m->gy); j <= tm_c3(m, hy, m->mn[1], m->gy); j++)
                    for (int i = tm_c3(m, lx, m->mn[0], m->gx); i <= tm_c3(m, hx, m->mn[0], m->gx); i++) {
                        size_t cell = ((size_t)kk * m->gy + j) * m->gx + i;
                        if (pass == 0) m->g3_start[cell + 1]++;
                        else m->g3_items[f3[cell]++] = k;
                    }
        }
    }
    free(f2);
    free(f3);
    return 0;
}

static v3 tm_vertex(const o_trimesh *m, int i) { return V3(m->v[3 * i], m->v[3 * i + 1], m->v[3 * i + 2]); }

/* VerticalHits (:96-121) folded into its two uses: mode 0 counts the hits above zq (Contains), mode 1 keeps the
   highest (side 0) or lowest hit in *zext (SurfaceZ); returns the number of hits */
static int tm_hits(const o_trimesh *m, double x, double y, int mode, double zq, int side, double *zext)
{
    int n = 0, above = 0;
    if (x < m->mn[0] || x > m->mx[0] || y < m->mn[1] || y > m->mx[1]) return 0;
    x += 1.2345e-7;
    y += 2.3456e-7;
    int cell = tm_cy2(m, y) * m->nx2 + tm_cx2(m, x);
    for (int q = m->xy_start[cell]; q < m->xy_start[cell + 1]; q++) {
        int t = m->xy_items[q];
        v3 a = tm_vertex(m, m->t[3 * t]), b = tm_vertex(m, m->t[3 * t + 1]), c = tm_vertex(m, m->t[3 * t + 2]);
        double d = (b.x - a.x) * (c.y - a.y) - (c.x - a.x) * (b.y - a.y);
        if (fabs(d) < 1e-300) continue;
        double u = ((x - a.x) * (c.y - a.y) - (c.x - a.x) * (y - a.y)) / d;
        double v = ((b.x - a.x) * (y - a.y) - (x - a.x) * (b.y - a.y)) / d;
        if (u < 0 || v < 0 || u + v > 1) continue;
        double z = a.z + u * (b.z - a.z) + v * (c.z - a.z);
        if (mode == 0) above += z > zq;
        else *zext = n == 0 ? z : (side == 0 ? fmax(*zext, z) : fmin(*zext, z));
        n++;
    }
    return mode == 0 ? above : n;
}

/* Contains (:125-137) */
static int tm_contains(const o_trimesh *m, v3 p)
{
    if (p.x < m->mn[0] || p.x > m->mx[0] || p.y < m->mn[1] || p.y > m->mx[1] || p.z < m->mn[2] || p.z > m->mx[2]) return 0;
    return (tm_hits(m, p.x, p.y, 0, p.z, 0, NULL) & 1) == 1;
}

/* Closest (:139-178) */
static int tm_closest(const o_trimesh *m, v3 p, double maxd, v3 *point, v3 *normal, double *dist)
{
    *point = p;
    *normal = V3(0, 0, 1);
    int ci = (int)floor((p.x - m->mn[0]) / m->c3), cj = (int)floor((p.y - m->mn[1]) / m->c3), ck = (int)floor((p.z - m->mn[2]) / m->c3);
    int max_ring = (int)ceil(maxd / m->c3) + 1;
    double best = maxd * maxd;
    for (int ring = 0; ring <= max_ring; ring++) {
        for (int k = ck - ring; k <= ck + ring; k++) {
            if (k < 0 || k >= m->gz) continue;
            for (int j = cj - ring; j <= cj + ring; j++) {
                if (j < 0 || j >= m->gy) continue;
                int shell_row = abs(j - cj) == ring || abs(k - ck) == ring;
                int istep = shell_row || ring == 0 ? 1 : 2 * ring;
                for (int i = ci - ring; i <= ci + ring; i += istep) {
                    if (i < 0 || i >= m->gx) continue;
                    int cell = (k * m->gy + j) * m->gx + i;
                    for (int q = m->g3_start[cell]; q < m->g3_start[cell + 1]; q++) {
                        int t = m->g3_items[q];
                        v3 a = tm_vertex(m, m->t[3 * t]), b = tm_vertex(m, m->t[3 * t + 1]), c = tm_vertex(m, m->t[3 * t + 2]);
                        v3 cq = o_closest_on_triangle(p, a, b, c);
                        double dd = vlen2(vsub(cq, p));
                        if (dd >= best) continue;
                        best = dd;
                        *point = cq;
                        *normal = vnormalized(vcross(vsub(b, a), vsub(c, a)));
                    }
                }
            }
        }
        if (sqrt(best) <= ring * m->c3) break;
    }
    *dist = sqrt(best);
    return *dist < maxd;
}

/* TriMeshDie.Clearance / Project / SurfaceZ (:267-296), Reach = 6 */
static double tm_clearance(const o_trimesh *m, v3 p, double offset)
{
    const double reach = 6;
    v3 q = V3(p.x, p.y, p.z - offset);
    if (q.x < m->mn[0] - reach || q.x > m->mx[0] + reach || q.y < m->mn[1] - reach || q.y > m->mx[1] + reach ||
        q.z < m->mn[2] - reach || q.z > m->mx[2] + reach)
        return reach;
    int inside = tm_contains(m, q);
    v3 c, n;
    double dist;
    double d = tm_closest(m, q, reach, &c, &n, &dist) ? dist : reach;
    return inside ? -d : d;
}
static v3 tm_project(const o_trimesh *m, int side, v3 p, double offset, v3 *normal)
{
    const double reach = 6;
    v3 q = V3(p.x, p.y, p.z - offset), c, n;
    double dist;
    if (!tm_closest(m, q, 4 * reach, &c, &n, &dist)) n = side == 0 ? V3(0, 0, 1) : V3(0, 0, -1);
    *normal = n;
    return V3(c.x, c.y, c.z + offset);
}
static double tm_surface_z(const o_trimesh *m, int side, double x, double y)
{
    double z = 0;
    return tm_hits(m, x, y, 1, 0, side, &z) ? z : NAN;
}

double hf_height(const o_hfdie *d, double x, double y)
{
    if (d->kind == 1) return tm_surface_z(&d->tm, d->side, x, y);
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
    if (d->kind == 1) return tm_clearance(&d->tm, p, offset);
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
    if (d->kind == 1) return tm_project(&d->tm, d->side, p, offset, normal);
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
