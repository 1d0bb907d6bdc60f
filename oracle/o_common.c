/*
 * o_common.c — shared pieces of the CPU oracle: geometry helpers, height-field die, principal stress,
 * the oracle's sparse SPD factorisation (ISpdSolver stand-in) and the band Cholesky.
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

/* ------------------------------------------------------------------ sparse SPD (oracle ISpdSolver backend)
 *
 * The reference's managed backend is CSparse.NET 4.4.1 (ManagedSpdSolver.cs:28-34): an up-looking Cholesky
 * with an approximate-minimum-degree ordering. CSparse is not available here; this restates the up-looking
 * algorithm (Davis, "Direct Methods for Sparse Linear Systems", cs_chol / cs_ereach / cs_etree) with a
 * nested-dissection order from recursive BFS level-set bisection. Any symmetric order gives the same factor
 * up to rounding, which is all the PCG / factorisation logic above it depends on.
 */

typedef struct {
    int n;
    const int32_t *ap, *ai;
} o_graph;

/* BFS over nodes with part[] == tag; returns the number of levels, fills level[] and order[] */
static int bfs_levels(const o_graph *g, int root, const int *part, int tag, int *level, int *order, int *count)
{
    int head = 0, tail = 0;
    order[tail++] = root;
    level[root] = 0;
    int maxl = 0;
    while (head < tail) {
        int u = order[head++];
        for (int32_t p = g->ap[u]; p < g->ap[u + 1]; p++) {
            int w = g->ai[p];
            if (w == u || part[w] != tag || level[w] >= 0) continue;
            level[w] = level[u] + 1;
            if (level[w] > maxl) maxl = level[w];
            order[tail++] = w;
        }
    }
    *count = tail;
    return maxl + 1;
}

typedef struct { int *nodes; int cnt; } o_range;

static void nd_order(const o_graph *g, int *part, int *level, int *order, int *perm, int *nperm, int *nodes, int cnt,
                     int tag, int *next_tag)
{
    /* nodes[] holds exactly the nodes with part == tag */
    if (cnt <= 0) return;
    if (cnt <= 48) {
        for (int k = 0; k < cnt; k++) perm[(*nperm)++] = nodes[k];
        return;
    }
    for (int k = 0; k < cnt; k++) level[nodes[k]] = -1;
    /* pseudo-peripheral start inside the first component */
    int root = nodes[0], reach = 0, nl = 0;
    for (int pass = 0; pass < 3; pass++) {
        for (int k = 0; k < cnt; k++) level[nodes[k]] = -1;
        nl = bfs_levels(g, root, part, tag, level, order, &reach);
        int last = order[reach - 1];
        if (pass < 2) root = last;
    }
    if (reach < cnt) {
        /* disconnected: the component of root first, then the rest */
        int ta = (*next_tag)++, tb = (*next_tag)++;
        int *a = (int *)malloc(sizeof(int) * reach), *b = (int *)malloc(sizeof(int) * (cnt - reach));
        int na = 0, nb = 0;
        for (int k = 0; k < cnt; k++) {
            int u = nodes[k];
            if (level[u] >= 0) { part[u] = ta; a[na++] = u; }
            else { part[u] = tb; b[nb++] = u; }
        }
        nd_order(g, part, level, order, perm, nperm, a, na, ta, next_tag);
        nd_order(g, part, level, order, perm, nperm, b, nb, tb, next_tag);
        free(a);
        free(b);
        return;
    }
    if (nl < 3) {
        for (int k = 0; k < cnt; k++) perm[(*nperm)++] = nodes[k];
        return;
    }
    /* separator = the level where the cumulative count crosses half */
    int *lc = (int *)calloc((size_t)nl, sizeof(int));
    for (int k = 0; k < cnt; k++) lc[level[nodes[k]]]++;
    int acc = 0, sep = nl / 2;
    for (int l = 0; l < nl; l++) {
        acc += lc[l];
        if (2 * acc >= cnt) { sep = l; break; }
    }
    if (sep == 0) sep = 1;
    if (sep == nl - 1) sep = nl - 2;
    free(lc);
    int ta = (*next_tag)++, tb = (*next_tag)++, ts = (*next_tag)++;
    int *a = (int *)malloc(sizeof(int) * cnt), *b = (int *)malloc(sizeof(int) * cnt), *s = (int *)malloc(sizeof(int) * cnt);
    int na = 0, nb = 0, ns = 0;
    for (int k = 0; k < cnt; k++) {
        int u = nodes[k];
        int l = level[u];
        if (l < sep) { part[u] = ta; a[na++] = u; }
        else if (l > sep) { part[u] = tb; b[nb++] = u; }
        else { part[u] = ts; s[ns++] = u; }
    }
    nd_order(g, part, level, order, perm, nperm, a, na, ta, next_tag);
    nd_order(g, part, level, order, perm, nperm, b, nb, tb, next_tag);
    for (int k = 0; k < ns; k++) perm[(*nperm)++] = s[k];
    free(a);
    free(b);
    free(s);
}

ospd *ospd_create(void) { return (ospd *)calloc(1, sizeof(ospd)); }

static void ospd_release(ospd *f)
{
    free(f->ap); free(f->ai); free(f->perm); free(f->pinv); free(f->cp); free(f->ci); free(f->cmap);
    free(f->parent); free(f->lp); free(f->li); free(f->lx); free(f->work); free(f->stack); free(f->mark);
    memset(f, 0, sizeof(*f));
}

void ospd_destroy(ospd *f)
{
    if (!f) return;
    ospd_release(f);
    free(f);
}

/* cs_ereach: pattern of row k of L (nonzeros of L(k, 0:k-1)) in topological order in s[top..n-1] */
static int ereach(const ospd *f, int k, int *s, int *w)
{
    int n = f->n, top = n;
    w[k] = k + 1; /* mark k with a stamp unique to this row */
    for (int32_t p = f->cp[k]; p < f->cp[k + 1]; p++) {
        int i = f->ci[p];
        if (i > k) continue;
        int len = 0;
        while (w[i] != k + 1) {
            s[len++] = i;
            w[i] = k + 1;
            i = f->parent[i];
            if (i < 0) break;
        }
        while (len > 0) s[--top] = s[--len];
    }
    return top;
}

int ospd_analyze(ospd *f, int n, const int32_t *col_ptr, const int32_t *row_idx)
{
    ospd_release(f);
    f->n = n;
    int nnz = col_ptr[n];
    f->nnz_full = nnz;
    f->ap = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
    f->ai = (int32_t *)malloc(sizeof(int32_t) * (nnz > 0 ? nnz : 1));
    memcpy(f->ap, col_ptr, sizeof(int32_t) * (n + 1));
    memcpy(f->ai, row_idx, sizeof(int32_t) * nnz);
    /* ordering */
    o_graph g = {n, f->ap, f->ai};
    int *part = (int *)calloc((size_t)n, sizeof(int)), *level = (int *)malloc(sizeof(int) * n);
    int *order = (int *)malloc(sizeof(int) * n), *nodes = (int *)malloc(sizeof(int) * n);
    f->perm = (int *)malloc(sizeof(int) * n);
    f->pinv = (int *)malloc(sizeof(int) * n);
    for (int k = 0; k < n; k++) nodes[k] = k;
    int nperm = 0, next_tag = 1;
    nd_order(&g, part, level, order, f->perm, &nperm, nodes, n, 0, &next_tag);
    free(part); free(level); free(order); free(nodes);
    for (int k = 0; k < n; k++) f->pinv[f->perm[k]] = k;
    /* upper triangle of C = P A P' in CSC, with a map back to the full value array */
    f->cp = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
    for (int j = 0; j < n; j++)
        for (int32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
            int i2 = f->pinv[row_idx[p]], j2 = f->pinv[j];
            if (i2 <= j2) f->cp[j2 + 1]++;
        }
    for (int j = 0; j < n; j++) f->cp[j + 1] += f->cp[j];
    int unnz = f->cp[n];
    f->ci = (int32_t *)malloc(sizeof(int32_t) * (unnz > 0 ? unnz : 1));
    f->cmap = (int *)malloc(sizeof(int) * (unnz > 0 ? unnz : 1));
    int *fill = (int *)malloc(sizeof(int) * (n + 1));
    memcpy(fill, f->cp, sizeof(int) * (n + 1));
    for (int j = 0; j < n; j++)
        for (int32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
            int i2 = f->pinv[row_idx[p]], j2 = f->pinv[j];
            if (i2 <= j2) {
                f->ci[fill[j2]] = i2;
                f->cmap[fill[j2]] = (int)p;
                fill[j2]++;
            }
        }
    free(fill);
    /* elimination tree (cs_etree, ata = 0) */
    f->parent = (int *)malloc(sizeof(int) * n);
    int *anc = (int *)malloc(sizeof(int) * n);
    for (int k = 0; k < n; k++) {
        f->parent[k] = -1;
        anc[k] = -1;
        for (int32_t p = f->cp[k]; p < f->cp[k + 1]; p++) {
            int i = f->ci[p];
            while (i != -1 && i < k) {
                int inext = anc[i];
                anc[i] = k;
                if (inext == -1) f->parent[i] = k;
                i = inext;
            }
        }
    }
    free(anc);
    /* column counts by running the row reaches once */
    f->stack = (int *)malloc(sizeof(int) * n);
    f->mark = (int *)malloc(sizeof(int) * n);
    f->work = (double *)malloc(sizeof(double) * n);
    int64_t *cnt = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    for (int k = 0; k < n; k++) f->mark[k] = 0;
    for (int k = 0; k < n; k++) {
        int top = ereach(f, k, f->stack, f->mark);
        for (int t = top; t < n; t++) cnt[f->stack[t]]++;
        cnt[k]++;
    }
    f->lp = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    f->lp[0] = 0;
    for (int k = 0; k < n; k++) f->lp[k + 1] = f->lp[k] + cnt[k];
    free(cnt);
    f->lnz = f->lp[n];
    f->li = (int *)malloc(sizeof(int) * (f->lnz > 0 ? f->lnz : 1));
    f->lx = (double *)malloc(sizeof(double) * (f->lnz > 0 ? f->lnz : 1));
    f->factored = 0;
    return 0;
}

/* cs_chol: up-looking numeric factorisation, values in the order of the full CSC pattern */
int ospd_factorize(ospd *f, const double *values)
{
    int n = f->n;
    int64_t *c = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
    memcpy(c, f->lp, sizeof(int64_t) * (n + 1));
    double *x = f->work;
    for (int k = 0; k < n; k++) { x[k] = 0; f->mark[k] = 0; }
    f->factored = 0;
    f->bad_pivot = -1;
    for (int k = 0; k < n; k++) {
        int top = ereach(f, k, f->stack, f->mark);
        x[k] = 0;
        for (int32_t p = f->cp[k]; p < f->cp[k + 1]; p++) x[f->ci[p]] += values[f->cmap[p]];
        double d = x[k];
        x[k] = 0;
        for (; top < n; top++) {
            int i = f->stack[top];
            double lki = x[i] / f->lx[f->lp[i]];
            x[i] = 0;
            for (int64_t p = f->lp[i] + 1; p < c[i]; p++) x[f->li[p]] -= f->lx[p] * lki;
            d -= lki * lki;
            int64_t p = c[i]++;
            f->li[p] = k;
            f->lx[p] = lki;
        }
        if (!(d > 0)) {
            f->bad_pivot = f->perm[k];
            free(c);
            return -1;
        }
        int64_t p = c[k]++;
        f->li[p] = k;
        f->lx[p] = sqrt(d);
    }
    free(c);
    f->factored = 1;
    return 0;
}

int ospd_solve(ospd *f, const double *b, double *xout)
{
    if (!f->factored) return -1;
    int n = f->n;
    double *x = f->work;
    for (int k = 0; k < n; k++) x[k] = b[f->perm[k]];
    for (int j = 0; j < n; j++) {
        x[j] /= f->lx[f->lp[j]];
        for (int64_t p = f->lp[j] + 1; p < f->lp[j + 1]; p++) x[f->li[p]] -= f->lx[p] * x[j];
    }
    for (int j = n - 1; j >= 0; j--) {
        for (int64_t p = f->lp[j] + 1; p < f->lp[j + 1]; p++) x[j] -= f->lx[p] * x[f->li[p]];
        x[j] /= f->lx[f->lp[j]];
    }
    for (int k = 0; k < n; k++) xout[f->perm[k]] = x[k];
    for (int k = 0; k < n; k++)
        if (!isfinite(xout[k])) return -2;
    return 0;
}

int64_t ospd_factor_nonzeros(const ospd *f) { return f->lnz; }
int ospd_bad_pivot(const ospd *f) { return f->bad_pivot; }

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
