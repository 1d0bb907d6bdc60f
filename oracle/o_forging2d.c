/*
 * o_forging2d.c — CPU FP64 restatement of Solver/ForgingSolver.cs (2D axisymmetric / plane-strain Q4 path),
 * Mesh/QuadMesh.cs (structured mesh, reverse Cuthill–McKee numbering, boundary loop) and
 * Geometry/DieSurface.cs. TEST INFRASTRUCTURE ONLY (see ifea_oracle.h). Remeshing is out of scope: it is
 * treated as rejected, as ForgingSolver does when RemeshCore fails.
 */
#include "o_internal.h"
#include <float.h>
#include <stdio.h>

enum { FREE = 0, BOTTOM = 1, TOP = 2 };
enum { E_OK = 0, E_INPUT = 1, E_DIVERGED = 2, E_DISTORTED = 3, E_NOT_SPD = 4, E_STATE = 5 };

typedef struct { double x, y; } v2;
static inline v2 V2(double x, double y) { v2 r = {x, y}; return r; }
static inline v2 w_add(v2 a, v2 b) { return V2(a.x + b.x, a.y + b.y); }
static inline v2 w_sub(v2 a, v2 b) { return V2(a.x - b.x, a.y - b.y); }
static inline v2 w_scale(double s, v2 a) { return V2(s * a.x, s * a.y); }
static inline double w_dot(v2 a, v2 b) { return a.x * b.x + a.y * b.y; }
static inline double w_cross(v2 a, v2 b) { return a.x * b.y - a.y * b.x; }
static inline double w_len(v2 a) { return sqrt(a.x * a.x + a.y * a.y); }
static inline v2 w_norm(v2 a) { double l = w_len(a); return l > 0 ? V2(a.x / l, a.y / l) : a; }

typedef struct { int side; int n; v2 *p; } o_die2;

/* DieSurface ctor (Geometry/DieSurface.cs:18-36) */
static int die2_init(o_die2 *d, int side, int n, const double *xy)
{
    if (n < 2) return -1;
    for (int i = 1; i < n; i++)
        if (!(xy[2 * i] > xy[2 * i - 2])) return -1;
    int extra = xy[2 * n - 2] < 1000.0;
    d->side = side;
    d->n = n + extra;
    d->p = (v2 *)malloc(sizeof(v2) * d->n);
    for (int i = 0; i < n; i++) d->p[i] = V2(xy[2 * i], xy[2 * i + 1]);
    if (extra) d->p[n] = V2(1000.0, xy[2 * n - 1]);
    return 0;
}

/* DieSurface.HeightAt (:85-98) */
static double die2_height(const o_die2 *d, double x)
{
    const v2 *p = d->p;
    if (x <= p[0].x) return p[0].y;
    if (x >= p[d->n - 1].x) return p[d->n - 1].y;
    int lo = 0, hi = d->n - 1;
    while (hi - lo > 1) {
        int mid = (lo + hi) >> 1;
        if (p[mid].x <= x) lo = mid; else hi = mid;
    }
    double t = (x - p[lo].x) / (p[hi].x - p[lo].x);
    return p[lo].y + t * (p[hi].y - p[lo].y);
}

/* HeightRange (:101-113) */
static void die2_range(const o_die2 *d, double x0, double x1, double *mn, double *mx)
{
    double a = die2_height(d, x0), b = die2_height(d, x1);
    double lo = dmin(a, b), hi = dmax(a, b);
    for (int i = 0; i < d->n; i++) {
        if (d->p[i].x <= x0 || d->p[i].x >= x1) continue;
        lo = dmin(lo, d->p[i].y);
        hi = dmax(hi, d->p[i].y);
    }
    *mn = lo; *mx = hi;
}

/* Clearance (:116-120) */
static double die2_clearance(const o_die2 *d, v2 p, double offset)
{
    double h = die2_height(d, p.x) + offset;
    return d->side == 0 ? p.y - h : h - p.y;
}

/* SegmentNormal (:123-127) */
static v2 die2_seg_normal(const o_die2 *d, int k)
{
    v2 dd = w_norm(w_sub(d->p[k + 1], d->p[k]));
    return d->side == 0 ? V2(-dd.y, dd.x) : V2(dd.y, -dd.x);
}

/* Project (:130-160) */
static v2 die2_project(const o_die2 *d, v2 p, double offset, v2 *normal, double *distance)
{
    v2 shift = V2(0, offset);
    double best = DBL_MAX, bestT = 0;
    int bestK = 0;
    v2 bestQ = V2(0, 0);
    for (int k = 0; k < d->n - 1; k++) {
        v2 a = w_add(d->p[k], shift);
        v2 ab = w_sub(d->p[k + 1], d->p[k]);
        double t = dclamp(w_dot(w_sub(p, a), ab) / w_dot(ab, ab), 0.0, 1.0);
        v2 q = w_add(a, w_scale(t, ab));
        double dd = w_dot(w_sub(p, q), w_sub(p, q));
        if (dd < best) { best = dd; bestK = k; bestT = t; bestQ = q; }
    }
    v2 n = die2_seg_normal(d, bestK);
    if (bestT < 1e-9 && bestK > 0) n = w_norm(w_add(n, die2_seg_normal(d, bestK - 1)));
    else if (bestT > 1 - 1e-9 && bestK < d->n - 2) n = w_norm(w_add(n, die2_seg_normal(d, bestK + 1)));
    if (normal) *normal = n;
    if (distance) *distance = sqrt(best);
    return bestQ;
}

double o2d_die_project(const double *pts, int npts, int side, double px, double py, double offset, double *qx, double *qy,
                       double *nx, double *ny)
{
    o_die2 d;
    if (die2_init(&d, side, npts, pts) != 0) return NAN;
    v2 n;
    double dist;
    v2 q = die2_project(&d, V2(px, py), offset, &n, &dist);
    *qx = q.x; *qy = q.y; *nx = n.x; *ny = n.y;
    free(d.p);
    return dist;
}

double o2d_die_height(const double *pts, int npts, double x)
{
    o_die2 d;
    if (die2_init(&d, 0, npts, pts) != 0) return NAN;
    double h = die2_height(&d, x);
    free(d.p);
    return h;
}

struct o2d {
    o2d_params p;
    o_die2 bottom, top;
    int axi;
    int nn, ne, ndof, half_band, nloop;
    int32_t *conn, *eq, *loop, *loop_owner;
    uint8_t *is_axis;
    double *x, *vg, *v, *r, *dv, *v_trial;
    double *eps, *dmg, *el_dev, *el_sig, *el_rate, *el_mean;
    uint8_t *contact, *rotated, *fixed, *release;
    double *tan, *nrm, *fixed_val, *k_fric, *a_fric;
    oband *k;
    double ram, rate_ref, rate_cut, sig_ref, k_pen, u0, h, gap0, gap, time, vol0, last_rel, seat;
    int step_index, iterations, remesh_requests, captured_total;
    double load, reaction, power;
    char err[512];
};

static int fail2(o2d *s, int code, const char *msg)
{
    snprintf(s->err, sizeof(s->err), "%s", msg);
    return code;
}
const char *o2d_error(const o2d *s) { return s->err; }

static inline v2 XX(const o2d *s, int n) { return V2(s->x[2 * n], s->x[2 * n + 1]); }
static inline v2 g2(const double *a, int n) { return V2(a[2 * n], a[2 * n + 1]); }
static inline void s2(double *a, int n, v2 v) { a[2 * n] = v.x; a[2 * n + 1] = v.y; }
static inline int dof(const o2d *s, int n, int c) { return 2 * s->eq[n] + c; }
static inline v2 die_vel2(int c, double ram) { return c == TOP ? V2(0, -ram) : V2(0, 0); }
static inline const o_die2 *surf2(const o2d *s, int c) { return c == TOP ? &s->top : &s->bottom; }
static inline double off2(int c, double gap) { return c == TOP ? gap : 0.0; }
static inline double weight(const o2d *s, double x) { return s->axi ? 2 * M_PI * x : 2 * s->p.length; }

/* QuadMesh.NumberEquations (Mesh/QuadMesh.cs:82-141) with HashSet insertion order and a stable OrderBy */
typedef struct { int32_t *start, *list; int32_t *deg; } adjacency;

static int peripheral(int start, const adjacency *adj, int nn, int32_t *depth, int32_t *queue)
{
    int node = start, bestDepth = -1;
    for (int pass = 0; pass < 4; pass++) {
        for (int i = 0; i < nn; i++) depth[i] = -1;
        int head = 0, tail = 0;
        depth[node] = 0;
        queue[tail++] = node;
        int last = node;
        while (head < tail) {
            int n = queue[head++];
            last = n;
            for (int32_t q = adj->start[n]; q < adj->start[n] + adj->deg[n]; q++) {
                int m = adj->list[q];
                if (depth[m] >= 0) continue;
                depth[m] = depth[n] + 1;
                queue[tail++] = m;
            }
        }
        if (depth[last] <= bestDepth) break;
        bestDepth = depth[last];
        node = last;
    }
    return node;
}

static int number_equations(o2d *s)
{
    int nn = s->nn, ne = s->ne;
    adjacency adj;
    adj.start = (int32_t *)calloc((size_t)nn + 1, sizeof(int32_t));
    adj.deg = (int32_t *)calloc((size_t)nn, sizeof(int32_t));
    int32_t *cnt = (int32_t *)calloc((size_t)nn, sizeof(int32_t));
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++) cnt[s->conn[4 * e + a]] += 3;
    for (int i = 0; i < nn; i++) adj.start[i + 1] = adj.start[i] + cnt[i];
    adj.list = (int32_t *)malloc(sizeof(int32_t) * (adj.start[nn] + 1));
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                if (a == b) continue;
                int n = s->conn[4 * e + a], m = s->conn[4 * e + b], found = 0;
                for (int32_t q = adj.start[n]; q < adj.start[n] + adj.deg[n]; q++)
                    if (adj.list[q] == m) { found = 1; break; }
                if (!found) adj.list[adj.start[n] + adj.deg[n]++] = m;
            }
    int32_t *order = (int32_t *)malloc(sizeof(int32_t) * nn), *depth = (int32_t *)malloc(sizeof(int32_t) * nn);
    int32_t *queue = (int32_t *)malloc(sizeof(int32_t) * nn), *cand = (int32_t *)malloc(sizeof(int32_t) * (nn + 1));
    uint8_t *seen = (uint8_t *)calloc((size_t)nn, 1);
    int norder = 0;
    while (norder < nn) {
        int start = -1;
        for (int n = 0; n < nn; n++)
            if (!seen[n] && (start < 0 || adj.deg[n] < adj.deg[start])) start = n;
        start = peripheral(start, &adj, nn, depth, queue);
        int head = 0, tail = 0;
        queue[tail++] = start;
        seen[start] = 1;
        while (head < tail) {
            int n = queue[head++];
            order[norder++] = n;
            int nc = 0;
            for (int32_t q = adj.start[n]; q < adj.start[n] + adj.deg[n]; q++)
                if (!seen[adj.list[q]]) cand[nc++] = adj.list[q];
            /* stable insertion sort by degree (Enumerable.OrderBy is stable) */
            for (int i = 1; i < nc; i++) {
                int key = cand[i], j = i - 1;
                while (j >= 0 && adj.deg[cand[j]] > adj.deg[key]) { cand[j + 1] = cand[j]; j--; }
                cand[j + 1] = key;
            }
            for (int i = 0; i < nc; i++) { seen[cand[i]] = 1; queue[tail++] = cand[i]; }
        }
    }
    for (int k = 0; k < nn; k++) s->eq[order[nn - 1 - k]] = k;
    int band = 1;
    for (int e = 0; e < ne; e++) {
        int lo = 0x7fffffff, hi = -0x7fffffff - 1;
        for (int a = 0; a < 4; a++) {
            int q = s->eq[s->conn[4 * e + a]];
            lo = imin(lo, q); hi = imax(hi, q);
        }
        band = imax(band, 2 * (hi - lo) + 1);
    }
    s->half_band = band;
    free(adj.start); free(adj.deg); free(adj.list); free(cnt); free(order); free(depth); free(queue); free(cand); free(seen);
    return 0;
}

/* QuadMesh.TraceBoundary (:173-221) */
static int trace_boundary(o2d *s)
{
    int nn = s->nn, ne = s->ne;
    /* undirected edge counts */
    int64_t m = 4 * (int64_t)ne;
    int64_t *keys = (int64_t *)malloc(sizeof(int64_t) * m);
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++) {
            int p = s->conn[4 * e + a], q = s->conn[4 * e + (a + 1) % 4];
            int lo = imin(p, q), hi = imax(p, q);
            keys[4 * e + a] = (int64_t)lo * nn + hi;
        }
    int64_t *sorted = (int64_t *)malloc(sizeof(int64_t) * m);
    memcpy(sorted, keys, sizeof(int64_t) * m);
    /* simple sort */
    int cmp64(const void *a, const void *b);
    qsort(sorted, (size_t)m, sizeof(int64_t), cmp64);
    int32_t *next_to = (int32_t *)malloc(sizeof(int32_t) * nn), *next_el = (int32_t *)malloc(sizeof(int32_t) * nn);
    int32_t *key_order = (int32_t *)malloc(sizeof(int32_t) * nn);
    for (int i = 0; i < nn; i++) next_to[i] = -1;
    int nkeys = 0;
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++) {
            int64_t k = keys[4 * e + a];
            /* count via binary search range */
            int64_t lo = 0, hi = m;
            while (lo < hi) { int64_t mid = (lo + hi) / 2; if (sorted[mid] < k) lo = mid + 1; else hi = mid; }
            int c = 0;
            for (int64_t t = lo; t < m && sorted[t] == k; t++) c++;
            if (c != 1) continue;
            int p = s->conn[4 * e + a], q = s->conn[4 * e + (a + 1) % 4];
            if (next_to[p] >= 0) {
                free(keys); free(sorted); free(next_to); free(next_el); free(key_order);
                return fail2(s, E_INPUT, "Mesh boundary is not a simple closed loop (pinched node).");
            }
            next_to[p] = q; next_el[p] = e;
            key_order[nkeys++] = p;
        }
    free(keys); free(sorted);
    if (nkeys == 0) { free(next_to); free(next_el); free(key_order); return fail2(s, E_INPUT, "Mesh has no boundary."); }
    int start = key_order[0];
    for (int k = 0; k < nkeys; k++) {
        int n = key_order[k];
        if (s->is_axis[n] && (!s->is_axis[start] || n < start)) start = n;
    }
    s->loop = (int32_t *)malloc(sizeof(int32_t) * nkeys);
    s->loop_owner = (int32_t *)malloc(sizeof(int32_t) * nkeys);
    int cnt = 0, cur = start;
    do {
        s->loop[cnt] = cur;
        s->loop_owner[cnt] = next_el[cur];
        cnt++;
        cur = next_to[cur];
        if (cnt > nkeys || cur < 0) { free(next_to); free(next_el); free(key_order); return fail2(s, E_INPUT, "Mesh boundary consists of several loops."); }
    } while (cur != start);
    free(next_to); free(next_el); free(key_order);
    if (cnt != nkeys) return fail2(s, E_INPUT, "Mesh boundary consists of several loops.");
    s->nloop = cnt;
    return 0;
}

int cmp64(const void *a, const void *b)
{
    int64_t x = *(const int64_t *)a, y = *(const int64_t *)b;
    return (x > y) - (x < y);
}

static double volume2(const o2d *s, const double *x)
{
    double area = 0, moment = 0;
    for (int k = 0; k < s->nloop; k++) {
        v2 a = g2(x, s->loop[k]), b = g2(x, s->loop[(k + 1) % s->nloop]);
        double cr = a.x * b.y - b.x * a.y;
        area += 0.5 * cr;
        moment += (a.x + b.x) * cr / 6.0;
    }
    return s->axi ? 2 * M_PI * moment : 2 * s->p.length * area;
}

/* ForgingSolver ctor (:104-145) */
o2d *o2d_create(const o2d_params *p, int n_bottom, const double *bottom_xy, int n_top, const double *top_xy)
{
    o2d *s = (o2d *)calloc(1, sizeof(o2d));
    s->p = *p;
    s->axi = p->axisymmetric;
    if (die2_init(&s->bottom, 0, n_bottom, bottom_xy) || die2_init(&s->top, 1, n_top, top_xy)) {
        fail2(s, E_INPUT, "invalid die profile");
        return s;
    }
    double r0 = p->radius, h0 = p->height;
    double mn, mx;
    die2_range(&s->bottom, 0, r0, &mn, &mx);
    double seat = mx;
    s->seat = seat;
    int nx = p->nx, ny = p->nz;
    s->nn = (nx + 1) * (ny + 1);
    s->ne = nx * ny;
    s->ndof = 2 * s->nn;
    s->x = (double *)calloc((size_t)2 * s->nn, sizeof(double));
    s->is_axis = (uint8_t *)calloc((size_t)s->nn, 1);
    for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
            int n = j * (nx + 1) + i;
            s->x[2 * n] = r0 * i / nx;
            s->x[2 * n + 1] = seat + h0 * j / ny;
            s->is_axis[n] = i == 0;
        }
    s->conn = (int32_t *)malloc(sizeof(int32_t) * 4 * s->ne);
    int e = 0;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            s->conn[e++] = j * (nx + 1) + i;
            s->conn[e++] = j * (nx + 1) + i + 1;
            s->conn[e++] = (j + 1) * (nx + 1) + i + 1;
            s->conn[e++] = (j + 1) * (nx + 1) + i;
        }
    s->eq = (int32_t *)malloc(sizeof(int32_t) * s->nn);
    number_equations(s);
    if (trace_boundary(s)) return s;
    s->h = dmin(r0 / nx, h0 / ny);
    double tmin, tmax;
    die2_range(&s->top, 0, r0, &tmin, &tmax);
    s->gap0 = s->gap = seat + h0 - tmin;
    s->ram = p->ram;
    s->rate_ref = s->ram / h0;
    s->rate_cut = 1e-3 * s->rate_ref;
    s->sig_ref = law_stress(p->C, p->N, p->M, p->eps0, 0, s->rate_ref);
    s->k_pen = 1e5 * s->sig_ref / s->rate_ref;
    s->u0 = 5e-3 * s->ram;
    int nn = s->nn, ne = s->ne;
    s->vg = (double *)calloc((size_t)2 * nn, sizeof(double));
    s->v = (double *)calloc((size_t)s->ndof, sizeof(double));
    s->r = (double *)calloc((size_t)s->ndof, sizeof(double));
    s->dv = (double *)calloc((size_t)s->ndof, sizeof(double));
    s->v_trial = (double *)calloc((size_t)s->ndof, sizeof(double));
    s->eps = (double *)calloc((size_t)ne, sizeof(double));
    s->dmg = (double *)calloc((size_t)ne, sizeof(double));
    s->el_dev = (double *)calloc((size_t)4 * ne, sizeof(double));
    s->el_sig = (double *)calloc((size_t)ne, sizeof(double));
    s->el_rate = (double *)calloc((size_t)ne, sizeof(double));
    s->el_mean = (double *)calloc((size_t)ne, sizeof(double));
    s->contact = (uint8_t *)calloc((size_t)nn, 1);
    s->rotated = (uint8_t *)calloc((size_t)nn, 1);
    s->fixed = (uint8_t *)calloc((size_t)s->ndof, 1);
    s->release = (uint8_t *)calloc((size_t)nn, 1);
    s->tan = (double *)calloc((size_t)2 * nn, sizeof(double));
    s->nrm = (double *)calloc((size_t)2 * nn, sizeof(double));
    s->fixed_val = (double *)calloc((size_t)s->ndof, sizeof(double));
    s->k_fric = (double *)calloc((size_t)nn, sizeof(double));
    s->a_fric = (double *)calloc((size_t)nn, sizeof(double));
    s->k = oband_create(s->ndof, s->half_band);
    for (int q = 0; q < ne; q++) s->el_sig[q] = s->sig_ref;
    double tol = 1e-3 * s->h;
    for (int k = 0; k < s->nloop; k++) {
        int n = s->loop[k];
        if (die2_clearance(&s->bottom, XX(s, n), 0) < tol) s->contact[n] = BOTTOM;
        else if (die2_clearance(&s->top, XX(s, n), s->gap) < tol) s->contact[n] = TOP;
    }
    double sx = s->axi ? 0.5 : 1.0;
    for (int n = 0; n < nn; n++) s2(s->vg, n, V2(sx * s->rate_ref * s->x[2 * n], -s->rate_ref * (s->x[2 * n + 1] - seat)));
    s->vol0 = volume2(s, s->x);
    return s;
}

void o2d_destroy(o2d *s)
{
    if (!s) return;
    void *ptrs[] = {s->bottom.p, s->top.p, s->conn, s->eq, s->loop, s->loop_owner, s->is_axis, s->x, s->vg, s->v, s->r, s->dv,
                    s->v_trial, s->eps, s->dmg, s->el_dev, s->el_sig, s->el_rate, s->el_mean, s->contact, s->rotated, s->fixed,
                    s->release, s->tan, s->nrm, s->fixed_val, s->k_fric, s->a_fric};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); k++) free(ptrs[k]);
    oband_destroy(s->k);
    free(s);
}

static void fix(o2d *s, int d, double value) { s->fixed[d] = 1; s->fixed_val[d] = value; }

/* PrepareConstraints (:304-358) */
static void prepare_constraints(o2d *s)
{
    memset(s->fixed, 0, s->ndof);
    memset(s->fixed_val, 0, sizeof(double) * s->ndof);
    memset(s->a_fric, 0, sizeof(double) * s->nn);
    memset(s->release, 0, s->nn);
    for (int n = 0; n < s->nn; n++) {
        s->rotated[n] = 0;
        s2(s->tan, n, V2(1, 0));
        s2(s->nrm, n, V2(0, 1));
        int axis = s->is_axis[n];
        int c = s->contact[n];
        if (c != FREE) {
            v2 dvl = die_vel2(c, s->ram);
            if (axis) {
                fix(s, dof(s, n, 0), 0);
                fix(s, dof(s, n, 1), dvl.y);
            } else {
                v2 nrm;
                die2_project(surf2(s, c), XX(s, n), off2(c, s->gap), &nrm, NULL);
                s2(s->nrm, n, nrm);
                s2(s->tan, n, V2(nrm.y, -nrm.x));
                s->rotated[n] = 1;
                fix(s, dof(s, n, 1), w_dot(dvl, nrm));
            }
        } else if (axis) {
            fix(s, dof(s, n, 0), 0);
        }
    }
    double *ksum = (double *)calloc((size_t)s->nn, sizeof(double));
    int32_t *kcnt = (int32_t *)calloc((size_t)s->nn, sizeof(int32_t));
    for (int k = 0; k < s->nloop; k++) {
        int a = s->loop[k], b = s->loop[(k + 1) % s->nloop];
        double len = w_len(w_sub(XX(s, b), XX(s, a)));
        double area = len * weight(s, 0.5 * (s->x[2 * a] + s->x[2 * b]));
        s->a_fric[a] += 0.5 * area;
        s->a_fric[b] += 0.5 * area;
        double kk = s->el_sig[s->loop_owner[k]] / sqrt(3.0);
        ksum[a] += kk; kcnt[a]++;
        ksum[b] += kk; kcnt[b]++;
    }
    for (int n = 0; n < s->nn; n++) s->k_fric[n] = kcnt[n] > 0 ? ksum[n] / kcnt[n] : 0;
    free(ksum); free(kcnt);
}

/* LoadVelocityGuess (:366-388) */
static void load_velocity_guess2(o2d *s)
{
    for (int n = 0; n < s->nn; n++) {
        v2 g = g2(s->vg, n);
        int d0 = dof(s, n, 0), d1 = dof(s, n, 1);
        if (s->rotated[n]) {
            s->v[d0] = w_dot(g, g2(s->tan, n));
            s->v[d1] = w_dot(g, g2(s->nrm, n));
        } else {
            s->v[d0] = g.x;
            s->v[d1] = g.y;
        }
    }
    for (int d = 0; d < s->ndof; d++)
        if (s->fixed[d]) s->v[d] = s->fixed_val[d];
}

int o2d_prepare(o2d *s)
{
    prepare_constraints(s);
    load_velocity_guess2(s);
    return 0;
}

static v2 global_velocity2(const o2d *s, const double *v, int n)
{
    double a = v[dof(s, n, 0)], b = v[dof(s, n, 1)];
    return s->rotated[n] ? w_add(w_scale(a, g2(s->tan, n)), w_scale(b, g2(s->nrm, n))) : V2(a, b);
}

static const double GP = 0.57735026918962576;

typedef struct {
    double ex[4], ey[4], ve[8], sn[4], dnx[4], dny[4], dxi[4], deta[4];
    double ke[64], re[8];
    int edof[8];
} escratch;

/* Shape (:563-590); returns det (<= 0 means distorted) */
static double shape(escratch *w, double xi, double eta)
{
    w->dxi[0] = -(1 - eta) / 4; w->dxi[1] = (1 - eta) / 4; w->dxi[2] = (1 + eta) / 4; w->dxi[3] = -(1 + eta) / 4;
    w->deta[0] = -(1 - xi) / 4; w->deta[1] = -(1 + xi) / 4; w->deta[2] = (1 + xi) / 4; w->deta[3] = (1 - xi) / 4;
    w->sn[0] = (1 - xi) * (1 - eta) / 4;
    w->sn[1] = (1 + xi) * (1 - eta) / 4;
    w->sn[2] = (1 + xi) * (1 + eta) / 4;
    w->sn[3] = (1 - xi) * (1 + eta) / 4;
    double j11 = 0, j12 = 0, j21 = 0, j22 = 0;
    for (int a = 0; a < 4; a++) {
        j11 += w->dxi[a] * w->ex[a];
        j12 += w->dxi[a] * w->ey[a];
        j21 += w->deta[a] * w->ex[a];
        j22 += w->deta[a] * w->ey[a];
    }
    double det = j11 * j22 - j12 * j21;
    if (!(det > 0)) return det;
    for (int a = 0; a < 4; a++) {
        w->dnx[a] = (j22 * w->dxi[a] - j12 * w->deta[a]) / det;
        w->dny[a] = (-j21 * w->dxi[a] + j11 * w->deta[a]) / det;
    }
    return det;
}

/* ElementKernel (:592-721); returns 0 or the failing element's code */
static int element_kernel(o2d *s, int e, int matrix, int newton, escratch *w, double *energy, double *power)
{
    static const double GXi[4] = {-0.57735026918962576, 0.57735026918962576, 0.57735026918962576, -0.57735026918962576};
    static const double GEta[4] = {-0.57735026918962576, -0.57735026918962576, 0.57735026918962576, 0.57735026918962576};
    (void)GP;
    if (matrix) memset(w->ke, 0, sizeof w->ke);
    memset(w->re, 0, sizeof w->re);
    double eps = s->eps[e];
    double sigCut = law_stress(s->p.C, s->p.N, s->p.M, s->p.eps0, eps, s->rate_cut);
    double mu0 = sigCut / s->rate_cut;
    double mExp = s->p.M;
    double sigSum = 0, rateSum = 0, s0Sum = 0, s1Sum = 0, s2Sum = 0, tSum = 0;
    double b0[8], b1[8], b2[8], b3[8], mb[4][8], g8[8], c8[8];
    for (int g = 0; g < 4; g++) {
        double det = shape(w, GXi[g], GEta[g]);
        if (!(det > 0)) return 1;
        double r = 0;
        for (int a = 0; a < 4; a++) r += w->sn[a] * w->ex[a];
        double wt = det * weight(s, r);
        for (int a = 0; a < 4; a++) {
            b0[2 * a] = w->dnx[a]; b0[2 * a + 1] = 0;
            b1[2 * a] = 0; b1[2 * a + 1] = w->dny[a];
            b2[2 * a] = s->axi ? w->sn[a] / r : 0; b2[2 * a + 1] = 0;
            b3[2 * a] = w->dny[a]; b3[2 * a + 1] = w->dnx[a];
        }
        double e0 = 0, e1 = 0, e2 = 0, e3 = 0;
        for (int k = 0; k < 8; k++) {
            e0 += b0[k] * w->ve[k];
            e1 += b1[k] * w->ve[k];
            e2 += b2[k] * w->ve[k];
            e3 += b3[k] * w->ve[k];
        }
        double ev3 = (e0 + e1 + e2) / 3;
        double d0 = e0 - ev3, d1 = e1 - ev3, d2 = e2 - ev3;
        double rate = sqrt(dmax(2.0 / 3.0 * (d0 * d0 + d1 * d1 + d2 * d2) + e3 * e3 / 3.0, 0));
        double m0 = 2.0 / 3.0 * d0, m1 = 2.0 / 3.0 * d1, m2 = 2.0 / 3.0 * d2, m3 = e3 / 3.0;
        for (int k = 0; k < 8; k++) g8[k] = b0[k] * m0 + b1[k] * m1 + b2[k] * m2 + b3[k] * m3;
        double mu, sig, wDens, coefN;
        if (rate > s->rate_cut) {
            sig = law_stress(s->p.C, s->p.N, s->p.M, s->p.eps0, eps, rate);
            mu = sig / rate;
            wDens = 0.5 * sigCut * s->rate_cut + (sig * rate - sigCut * s->rate_cut) / (mExp + 1);
            coefN = (mExp - 1) * mu / (rate * rate);
        } else {
            mu = mu0;
            sig = mu0 * rate;
            wDens = 0.5 * mu0 * rate * rate;
            coefN = 0;
        }
        *energy += wt * wDens;
        *power += wt * sig * rate;
        sigSum += sig;
        rateSum += rate;
        s0Sum += mu * m0;
        s1Sum += mu * m1;
        s2Sum += mu * m2;
        tSum += mu * m3;
        double wm = wt * mu;
        for (int k = 0; k < 8; k++) w->re[k] += wm * g8[k];
        if (!matrix) continue;
        for (int k = 0; k < 8; k++) {
            double tr = (b0[k] + b1[k] + b2[k]) / 3;
            mb[0][k] = 2.0 / 3.0 * (b0[k] - tr);
            mb[1][k] = 2.0 / 3.0 * (b1[k] - tr);
            mb[2][k] = 2.0 / 3.0 * (b2[k] - tr);
            mb[3][k] = b3[k] / 3.0;
        }
        double wn = newton ? wt * coefN : 0;
        for (int p = 0; p < 8; p++)
            for (int q = 0; q <= p; q++) {
                double sv = b0[p] * mb[0][q] + b1[p] * mb[1][q] + b2[p] * mb[2][q] + b3[p] * mb[3][q];
                w->ke[8 * p + q] += wm * sv + wn * g8[p] * g8[q];
            }
    }
    double det0 = shape(w, 0, 0);
    if (!(det0 > 0)) return 1;
    double rc = 0;
    for (int a = 0; a < 4; a++) rc += w->sn[a] * w->ex[a];
    double w0 = 4 * det0 * weight(s, rc);
    double evol = 0;
    for (int a = 0; a < 4; a++) {
        c8[2 * a] = w->dnx[a] + (s->axi ? w->sn[a] / rc : 0);
        c8[2 * a + 1] = w->dny[a];
    }
    for (int k = 0; k < 8; k++) evol += c8[k] * w->ve[k];
    double kw = s->k_pen * w0;
    for (int k = 0; k < 8; k++) w->re[k] += kw * evol * c8[k];
    *energy += 0.5 * kw * evol * evol;
    *power += kw * evol * evol;
    if (matrix) {
        for (int p = 0; p < 8; p++)
            for (int q = 0; q <= p; q++) w->ke[8 * p + q] += kw * c8[p] * c8[q];
        for (int p = 0; p < 8; p++)
            for (int q = p + 1; q < 8; q++) w->ke[8 * p + q] = w->ke[8 * q + p];
    }
    s->el_sig[e] = sigSum / 4;
    s->el_rate[e] = rateSum / 4;
    s->el_dev[4 * e] = s0Sum / 4;
    s->el_dev[4 * e + 1] = s1Sum / 4;
    s->el_dev[4 * e + 2] = s2Sum / 4;
    s->el_dev[4 * e + 3] = tSum / 4;
    s->el_mean[e] = s->k_pen * evol;
    return 0;
}

/* RotateElementBlock (:541-561) */
static void rotate_block(escratch *w, int a, v2 t, v2 n, int matrix)
{
    int r0 = 2 * a, r1 = r0 + 1;
    double f0 = w->re[r0], f1 = w->re[r1];
    w->re[r0] = t.x * f0 + t.y * f1;
    w->re[r1] = n.x * f0 + n.y * f1;
    if (!matrix) return;
    for (int c = 0; c < 8; c++) {
        double k0 = w->ke[8 * r0 + c], k1 = w->ke[8 * r1 + c];
        w->ke[8 * r0 + c] = t.x * k0 + t.y * k1;
        w->ke[8 * r1 + c] = n.x * k0 + n.y * k1;
    }
    for (int r = 0; r < 8; r++) {
        double k0 = w->ke[8 * r + r0], k1 = w->ke[8 * r + r1];
        w->ke[8 * r + r0] = t.x * k0 + t.y * k1;
        w->ke[8 * r + r1] = n.x * k0 + n.y * k1;
    }
}

static int distorted_elem = -1;

/* Assemble (:471-538) */
double o2d_assemble(o2d *s, int matrix, int newton, const double *v, double *power_out)
{
    if (matrix) oband_clear(s->k);
    memset(s->r, 0, sizeof(double) * s->ndof);
    double energy = 0, power = 0;
    escratch w;
    distorted_elem = -1;
    for (int e = 0; e < s->ne; e++) {
        for (int a = 0; a < 4; a++) {
            int n = s->conn[4 * e + a];
            w.ex[a] = s->x[2 * n];
            w.ey[a] = s->x[2 * n + 1];
            v2 g = global_velocity2(s, v, n);
            w.ve[2 * a] = g.x;
            w.ve[2 * a + 1] = g.y;
            w.edof[2 * a] = dof(s, n, 0);
            w.edof[2 * a + 1] = dof(s, n, 1);
        }
        if (element_kernel(s, e, matrix, newton, &w, &energy, &power)) {
            distorted_elem = e;
            if (power_out) *power_out = NAN;
            return NAN;
        }
        for (int a = 0; a < 4; a++) {
            int n = s->conn[4 * e + a];
            if (s->rotated[n]) rotate_block(&w, a, g2(s->tan, n), g2(s->nrm, n), matrix);
        }
        for (int p = 0; p < 8; p++) {
            s->r[w.edof[p]] += w.re[p];
            if (!matrix) continue;
            for (int q = 0; q <= p; q++) {
                double kv = w.ke[8 * p + q];
                if (kv != 0) oband_add(s->k, w.edof[p], w.edof[q], kv);
            }
        }
    }
    double m = s->p.friction;
    if (m > 0) {
        for (int n = 0; n < s->nn; n++) {
            if (!s->rotated[n]) continue;
            double c = m * s->k_fric[n] * s->a_fric[n] * (2 / M_PI);
            if (c <= 0) continue;
            int d = dof(s, n, 0);
            double sv = v[d] - w_dot(die_vel2(s->contact[n], s->ram), g2(s->tan, n));
            double z = sv / s->u0;
            double f = c * atan(z);
            s->r[d] += f;
            energy += c * (sv * atan(z) - 0.5 * s->u0 * log(1 + z * z));
            power += f * sv;
            if (matrix) {
                double kt = newton ? c / (s->u0 * (1 + z * z)) : (fabs(z) > 1e-9 ? f / sv : c / s->u0);
                oband_add(s->k, d, d, kt);
            }
        }
    }
    if (power_out) *power_out = power;
    return energy;
}

static double norm2v(const double *a, int n)
{
    double sum = 0;
    for (int k = 0; k < n; k++) sum += a[k] * a[k];
    return sqrt(sum);
}

/* SolveVelocity (:403-461); returns iterations or -error */
int o2d_solve_velocity(o2d *s, int picard_fallback, int *converged)
{
    *converged = 0;
    s->last_rel = INFINITY;
    int it, damped = 0, picard_until = 2;
    for (it = 1; it <= s->p.max_iter; it++) {
        int newton = it > picard_until;
        double e0 = o2d_assemble(s, 1, newton, s->v, NULL);
        if (distorted_elem >= 0) {
            char msg[160];
            snprintf(msg, sizeof msg, "Element %d has a non-positive Jacobian at step %d.", distorted_elem, s->step_index);
            return -fail2(s, E_DISTORTED, msg);
        }
        for (int d = 0; d < s->ndof; d++) {
            if (!s->fixed[d]) continue;
            oband_constrain(s->k, d);
            s->r[d] = 0;
        }
        double pivot = 0;
        int bad = oband_factorize(s->k, &pivot);
        if (bad >= 0) {
            char msg[200];
            snprintf(msg, sizeof msg, "Stiffness matrix not positive definite at equation %d (pivot %.3E). The billet is probably unrestrained.", bad, pivot);
            return -fail2(s, E_NOT_SPD, msg);
        }
        for (int d = 0; d < s->ndof; d++) s->dv[d] = -s->r[d];
        oband_solve(s->k, s->dv);
        double slope = 0;
        for (int d = 0; d < s->ndof; d++) slope += s->r[d] * s->dv[d];
        double beta = 1.0;
        for (int ls = 0; ls < 8; ls++) {
            for (int d = 0; d < s->ndof; d++) s->v_trial[d] = s->v[d] + beta * s->dv[d];
            double e1 = o2d_assemble(s, 0, 0, s->v_trial, NULL);
            if (e1 <= e0 + 1e-4 * beta * slope + 1e-11 * fabs(e0)) break;
            beta *= 0.5;
        }
        memcpy(s->v, s->v_trial, sizeof(double) * s->ndof);
        double rel = beta * norm2v(s->dv, s->ndof) / dmax(norm2v(s->v, s->ndof), 1e-30);
        s->last_rel = rel;
        if (isnan(rel)) {
            char msg[120];
            snprintf(msg, sizeof msg, "Velocity solution became NaN at step %d.", s->step_index);
            return -fail2(s, E_DIVERGED, msg);
        }
        if (rel < s->p.tol) { *converged = 1; return it; }
        damped = newton && beta < 0.5 ? damped + 1 : 0;
        if (picard_fallback && damped >= 3) { picard_until = it + 4; damped = 0; }
    }
    return it - 1;
}

/* FinalEvaluation (:737-784) */
double o2d_final_evaluation(o2d *s, double *reaction_out)
{
    double power;
    o2d_assemble(s, 0, 0, s->v, &power);
    double reaction = 0, maxB = 0, maxT = 0;
    for (int n = 0; n < s->nn; n++) {
        s2(s->vg, n, global_velocity2(s, s->v, n));
        if (s->contact[n] == FREE) continue;
        double r0 = s->r[dof(s, n, 0)], r1 = s->r[dof(s, n, 1)];
        v2 rg = s->rotated[n] ? w_add(w_scale(r0, g2(s->tan, n)), w_scale(r1, g2(s->nrm, n))) : V2(r0, r1);
        if (s->contact[n] == TOP) reaction -= rg.y;
        if (!s->rotated[n]) continue;
        double comp = r1;
        if (s->contact[n] == TOP) maxT = dmax(maxT, comp); else maxB = dmax(maxB, comp);
    }
    int keptB = 0, keptT = 0;
    for (int n = 0; n < s->nn; n++) {
        if (s->contact[n] == FREE) continue;
        if (!s->rotated[n]) {
            if (s->contact[n] == TOP) keptT++; else keptB++;
            continue;
        }
        double comp = s->r[dof(s, n, 1)];
        double thr = 0.02 * (s->contact[n] == TOP ? maxT : maxB);
        if (comp < -thr) s->release[n] = 1;
        else if (s->contact[n] == TOP) keptT++;
        else keptB++;
    }
    if (keptT == 0 || keptB == 0)
        for (int n = 0; n < s->nn; n++)
            if ((keptT == 0 && s->contact[n] == TOP) || (keptB == 0 && s->contact[n] == BOTTOM)) s->release[n] = 0;
    if (reaction_out) *reaction_out = reaction;
    return power;
}

/* Quality (:900-914) */
static double quality2(const o2d *s, const double *x, int e)
{
    double q = DBL_MAX;
    for (int a = 0; a < 4; a++) {
        v2 p = g2(x, s->conn[4 * e + a]);
        v2 nx = w_sub(g2(x, s->conn[4 * e + (a + 1) % 4]), p);
        v2 pv = w_sub(g2(x, s->conn[4 * e + (a + 3) % 4]), p);
        double l = w_len(nx) * w_len(pv);
        q = dmin(q, l > 0 ? w_cross(nx, pv) / l : -1);
    }
    return q;
}

static double min_quality2(const o2d *s, const double *x)
{
    double q = DBL_MAX;
    for (int e = 0; e < s->ne; e++) q = dmin(q, quality2(s, x, e));
    return q;
}

/* TryUpdate (:789-864), allowFold = false */
static int try_update2(o2d *s, double dt, char *why, size_t whylen)
{
    double gapT = dmax(0, s->gap - s->ram * dt);
    if (gapT < 1e-9) gapT = 0;
    double *xT = (double *)malloc(sizeof(double) * 2 * s->nn);
    uint8_t *cT = (uint8_t *)calloc((size_t)s->nn, 1);
    double tolSep = 0.05 * s->h, maxPen = 0;
    for (int n = 0; n < s->nn; n++) {
        int axis = s->is_axis[n];
        v2 p = w_add(XX(s, n), w_scale(dt, g2(s->vg, n)));
        if (axis) p = V2(0, p.y);
        int c = s->contact[n];
        if (c != FREE && !s->release[n]) {
            const o_die2 *sf = surf2(s, c);
            double off = off2(c, gapT);
            if (die2_clearance(sf, p, off) > tolSep) cT[n] = FREE;
            else {
                p = axis ? V2(0, die2_height(sf, 0) + off) : die2_project(sf, p, off, NULL, NULL);
                cT[n] = (uint8_t)c;
            }
        } else {
            double cb = die2_clearance(&s->bottom, p, 0);
            double ctp = die2_clearance(&s->top, p, gapT);
            if (cb < 0 || ctp < 0) {
                int hit = cb <= ctp ? BOTTOM : TOP;
                const o_die2 *sf = surf2(s, hit);
                double off = off2(hit, gapT);
                v2 q = axis ? V2(0, die2_height(sf, 0) + off) : die2_project(sf, p, off, NULL, NULL);
                maxPen = dmax(maxPen, w_len(w_sub(q, p)));
                p = q;
                cT[n] = (uint8_t)hit;
            }
        }
        s2(xT, n, p);
    }
    if (maxPen > 0.5 * s->h) {
        snprintf(why, whylen, "die penetration %.3f mm exceeds h/2", maxPen);
        free(xT); free(cT);
        return 0;
    }
    for (int e = 0; e < s->ne; e++)
        if (quality2(s, xT, e) <= 0.002) {
            snprintf(why, whylen, "element %d folded", e);
            free(xT); free(cT);
            return 0;
        }
    memcpy(s->x, xT, sizeof(double) * 2 * s->nn);
    memcpy(s->contact, cT, s->nn);
    s->gap = gapT;
    s->time += dt;
    free(xT); free(cT);
    why[0] = 0;
    return 1;
}

/* CaptureFoldOver (:927-962) */
static int capture_fold_over(o2d *s)
{
    int m = s->nloop;
    double sinLimit = sin(25 * M_PI / 180);
    int captured = 0, changed = 1;
    for (int pass = 0; pass < 4 && changed; pass++) {
        changed = 0;
        for (int k = 0; k < m; k++) {
            int n = s->loop[k];
            int c = s->contact[n];
            if (c == FREE) continue;
            int fs[2] = {s->loop[(k + m - 1) % m], s->loop[(k + 1) % m]};
            for (int q = 0; q < 2; q++) {
                int f = fs[q];
                if (s->contact[f] != FREE || s->is_axis[f]) continue;
                const o_die2 *sf = surf2(s, c);
                double off = off2(c, s->gap);
                v2 nrm;
                die2_project(sf, XX(s, n), off, &nrm, NULL);
                v2 u = w_sub(XX(s, f), XX(s, n));
                double len = w_len(u);
                if (len <= 0 || w_dot(u, nrm) / len > sinLimit) continue;
                v2 qq = die2_project(sf, XX(s, f), off, NULL, NULL);
                if (w_len(w_sub(qq, XX(s, f))) > 0.5 * s->h) continue;
                s2(s->x, f, qq);
                s->contact[f] = (uint8_t)c;
                captured++;
                changed = 1;
            }
        }
    }
    return captured;
}

/* Principal.Max2D (Solver/Principal.cs:22-26) */
static double max2d(double xx, double yy, double xy, double zz)
{
    double c = 0.5 * (xx + yy), r = sqrt(0.25 * (xx - yy) * (xx - yy) + xy * xy);
    return dmax(c + r, zz);
}

/* AccumulateDamage (:724-734) */
static void accumulate_damage2(o2d *s, double dt)
{
    for (int e = 0; e < s->ne; e++) {
        double sig = s->el_sig[e];
        if (!(sig > 0) || s->el_rate[e] <= s->rate_cut) continue;
        double m = s->el_mean[e];
        double s1 = max2d(s->el_dev[4 * e] + m, s->el_dev[4 * e + 1] + m, s->el_dev[4 * e + 3], s->el_dev[4 * e + 2] + m);
        if (s1 > 0) s->dmg[e] += s1 / sig * s->el_rate[e] * dt;
    }
}

/* Advance (:215-290) with remeshing unavailable */
int o2d_step(o2d *s)
{
    if (s->gap <= 1e-9) return fail2(s, E_STATE, "Simulation already reached the closed-die position.");
    s->step_index++;
    /* RemeshTrigger (:966-976): counted only */
    if (min_quality2(s, s->x) < 0.15) s->remesh_requests++;
    else {
        double maxEdge = 0;
        for (int k = 0; k < s->nloop; k++) maxEdge = dmax(maxEdge, w_len(w_sub(XX(s, s->loop[(k + 1) % s->nloop]), XX(s, s->loop[k]))));
        if (maxEdge > 2.5 * s->h) s->remesh_requests++;
    }
    int iterations = 0, ok = 0;
    double load = 0, reaction = 0, dt = 0;
    char why[160] = "";
    for (int pass = 0; pass < 2 && !ok; pass++) {
        o2d_prepare(s);
        int converged;
        iterations = o2d_solve_velocity(s, 0, &converged);
        if (iterations < 0) return -iterations;
        if (!converged && s->last_rel >= 1e-3) {
            load_velocity_guess2(s);
            int more = o2d_solve_velocity(s, 1, &converged);
            if (more < 0) return -more;
            iterations += more;
        }
        if (!converged) {
            if (!(s->last_rel < 1e-3)) {
                char msg[200];
                snprintf(msg, sizeof msg, "Newton-Raphson diverged at step %d (stroke %.3f mm): |dv|/|v| = %.2E after %d iterations.",
                         s->step_index, s->gap0 - s->gap, s->last_rel, iterations);
                return fail2(s, E_DIVERGED, msg);
            }
        }
        double power = o2d_final_evaluation(s, &reaction);
        s->power = power;
        load = power / s->ram;
        dt = dmin(s->p.ds, s->gap) / s->ram;
        if (s->gap - s->ram * dt < 0.05 * s->p.ds) dt = s->gap / s->ram;
        for (int attempt = 0; attempt < 4 && !ok; attempt++) {
            double dta = dt / (1 << attempt);
            ok = try_update2(s, dta, why, sizeof why);
            if (ok) dt = dta;
        }
        if (!ok) { s->remesh_requests++; break; } /* Remesh("fold during update") unavailable */
    }
    if (!ok) {
        char msg[300];
        snprintf(msg, sizeof msg, "Mesh distortion at step %d (stroke %.3f mm): %s.", s->step_index, s->gap0 - s->gap, why);
        return fail2(s, E_DISTORTED, msg);
    }
    for (int e = 0; e < s->ne; e++) s->eps[e] += s->el_rate[e] * dt;
    accumulate_damage2(s, dt);
    double *savedX = (double *)malloc(sizeof(double) * 2 * s->nn);
    uint8_t *savedC = (uint8_t *)malloc((size_t)s->nn);
    memcpy(savedX, s->x, sizeof(double) * 2 * s->nn);
    memcpy(savedC, s->contact, s->nn);
    int captured = capture_fold_over(s);
    if (captured > 0) {
        s->remesh_requests++; /* Remesh("fold-over ...") unavailable: the capture is undone when it leaves a poor element */
        if (min_quality2(s, s->x) <= 0.05) {
            memcpy(s->x, savedX, sizeof(double) * 2 * s->nn);
            memcpy(s->contact, savedC, s->nn);
        } else {
            s->captured_total += captured;
        }
    }
    free(savedX); free(savedC);
    s->iterations = iterations;
    s->load = load;
    s->reaction = reaction;
    s->err[0] = 0;
    return E_OK;
}

void *o2d_array(o2d *s, const char *name, int64_t *count)
{
#define ARR(nm, ptr, cnt) if (!strcmp(name, nm)) { *count = (cnt); return (void *)(ptr); }
    ARR("x", s->x, 2 * (int64_t)s->nn)
    ARR("vg", s->vg, 2 * (int64_t)s->nn)
    ARR("v", s->v, s->ndof)
    ARR("r", s->r, s->ndof)
    ARR("dv", s->dv, s->ndof)
    ARR("eps", s->eps, s->ne)
    ARR("dmg", s->dmg, s->ne)
    ARR("el_sig", s->el_sig, s->ne)
    ARR("el_rate", s->el_rate, s->ne)
    ARR("el_mean", s->el_mean, s->ne)
    ARR("el_dev", s->el_dev, 4 * (int64_t)s->ne)
    ARR("contact", s->contact, s->nn)
    ARR("release", s->release, s->nn)
    ARR("rotated", s->rotated, s->nn)
    ARR("fixed", s->fixed, s->ndof)
    ARR("fixed_val", s->fixed_val, s->ndof)
    ARR("tan", s->tan, 2 * (int64_t)s->nn)
    ARR("nrm", s->nrm, 2 * (int64_t)s->nn)
    ARR("k_fric", s->k_fric, s->nn)
    ARR("a_fric", s->a_fric, s->nn)
    ARR("conn", s->conn, 4 * (int64_t)s->ne)
    ARR("eq", s->eq, s->nn)
    ARR("is_axis", s->is_axis, s->nn)
    ARR("loop", s->loop, s->nloop)
    ARR("loop_owner", s->loop_owner, s->nloop)
    if (!strcmp(name, "band")) return oband_data(s->k, count);
#undef ARR
    *count = 0;
    return NULL;
}

double o2d_scalar(o2d *s, const char *name)
{
#define SC(nm, v) if (!strcmp(name, nm)) return (double)(v);
    SC("gap", s->gap) SC("gap0", s->gap0) SC("time", s->time) SC("load", s->load) SC("reaction", s->reaction)
    SC("power", s->power) SC("iterations", s->iterations) SC("last_rel", s->last_rel) SC("vol0", s->vol0)
    SC("volume", volume2(s, s->x)) SC("step_index", s->step_index) SC("half_band", s->half_band)
    SC("bandwidth", oband_bandwidth(s->k)) SC("rate_ref", s->rate_ref) SC("rate_cut", s->rate_cut) SC("sig_ref", s->sig_ref)
    SC("k_pen", s->k_pen) SC("u0", s->u0) SC("h", s->h) SC("seat", s->seat) SC("remesh_requests", s->remesh_requests)
    SC("nn", s->nn) SC("ne", s->ne) SC("ndof", s->ndof) SC("nloop", s->nloop) SC("min_quality", min_quality2(s, s->x))
    SC("captured", s->captured_total)
#undef SC
    return NAN;
}
