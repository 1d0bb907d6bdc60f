/*
 * o_forging3d.c — CPU FP64 restatement of ThreeD/Forging3DSolver.cs (the 3D per-Newton-iteration path and the
 * stepping around it, remeshing excluded). TEST INFRASTRUCTURE ONLY (see ifea_oracle.h).
 *
 * Remeshing is out of scope: where the reference would remesh (RemeshTrigger, recovery ladder) the oracle
 * counts the request and behaves as if the remesh had been rejected, which is what Forging3DSolver does when
 * RemeshCore returns false.
 */
#include "o_internal.h"
#include <float.h>
#include <stdio.h>

enum { FREE = 0, BOTTOM = 1, TOP = 2 };
enum { E_OK = 0, E_INPUT = 1, E_DIVERGED = 2, E_DISTORTED = 3, E_NOT_SPD = 4, E_STATE = 5 };

struct o3d {
    o3d_params p;
    double rate_ref, rate_cut, sig_ref, k_pen, u0, h;
    double gap0, gap, ds_cur, time, last_rel, vol0;
    int step_index, warm, recovery_pass, have_dies;
    o_hfdie die[2];
    /* mesh */
    int nn, ne, ndof, nbf;
    int32_t *tets;
    uint8_t *on_x0, *on_y0, *is_surface;
    int32_t *nts, *ntl;            /* node -> tet CSR (TetMesh.NodeTetStart/List) */
    int32_t *bface, *bowner;       /* boundary faces (outward), owner tet */
    uint8_t *bsym;
    int32_t *nbr_start, *nbr;      /* sorted two-ring neighbours */
    int32_t *col_ptr, *row_idx;
    int64_t nnz;
    int32_t *e_nbr;
    double *h_local;
    /* state */
    double *x, *vg, *vg_prev;      /* nn x 3 */
    int have_vg_prev;
    double *eps, *dmg, *el_dev, *el_sig, *el_rate, *el_mean;
    uint8_t *contact, *release, *fixed;
    double *ax;                    /* nn x 9: ax0, ax1, ax2 */
    int32_t *n_fix, *die_axis;
    double *fixed_val, *k_fric, *a_fric;
    double *grad, *vol;
    double *v, *r, *dv, *v_trial, *rvol, *v_node;
    int32_t *g_start, *g_node;
    double *g_coef;                /* 3 per entry */
    int64_t g_len;
    double *kvol, *val;
    double *e_r, *e_k, *e_energy, *e_power;
    /* linear solver */
    ospd *lin;
    int need_analyze, have_factor, pcg_failures, pcg_skip;
    double *pr, *pz, *pp, *pq;
    /* statistics */
    int iterations, n_pcg, n_fact, n_newton, n_assemble, remesh_requests, projection_reverts, corner_penetrations;
    int lin_its_total;
    double load, reaction, power, rnorm_last, beta_last, max_diag_last;
    char err[512];
    /* remeshing: the host's remesher, called where Step remeshes (ThreeD/Forging3DSolver.cs:544-611) */
    o3d_remesh_fn remesh_cb;
    void *remesh_user;
    int remesh_count, refinement_levels, max_nodes, nhot, have_fail_at;
    double fail_at[3];
    double hot[4 * 64];            /* places where increments failed: x, y, z, refinement level */
};

static int fail(o3d *s, int code, const char *msg)
{
    snprintf(s->err, sizeof(s->err), "%s", msg);
    return code;
}

const char *o3d_error(const o3d *s) { return s->err; }

o3d *o3d_create(const o3d_params *p)
{
    o3d *s = (o3d *)calloc(1, sizeof(o3d));
    s->p = *p;
    s->h = p->h;
    s->ds_cur = p->ds;
    /* Forging3DSolver.cs:146-150 */
    s->rate_ref = p->ram / p->size;
    s->rate_cut = 1e-3 * s->rate_ref;
    s->sig_ref = law_stress(p->C, p->N, p->M, p->eps0, 0, s->rate_ref);
    s->k_pen = p->penalty_factor * s->sig_ref / s->rate_ref;
    s->u0 = 5e-3 * p->ram;
    s->refinement_levels = 1;
    s->max_nodes = 1 << 30;
    s->lin = ospd_create();
    s->need_analyze = 1;
    return s;
}

static void free_mesh(o3d *s)
{
    /* every pointer is cleared too: a mesh replaced by a remesh must not leave one behind to be freed twice */
    void **ptrs[] = {(void **)&s->tets, (void **)&s->on_x0, (void **)&s->on_y0, (void **)&s->is_surface,
                     (void **)&s->nts, (void **)&s->ntl, (void **)&s->bface, (void **)&s->bowner, (void **)&s->bsym,
                     (void **)&s->nbr_start, (void **)&s->nbr, (void **)&s->col_ptr, (void **)&s->row_idx,
                     (void **)&s->e_nbr, (void **)&s->h_local, (void **)&s->x, (void **)&s->vg, (void **)&s->vg_prev,
                     (void **)&s->eps, (void **)&s->dmg, (void **)&s->el_dev, (void **)&s->el_sig,
                     (void **)&s->el_rate, (void **)&s->el_mean, (void **)&s->contact, (void **)&s->release,
                     (void **)&s->fixed, (void **)&s->ax, (void **)&s->n_fix, (void **)&s->die_axis,
                     (void **)&s->fixed_val, (void **)&s->k_fric, (void **)&s->a_fric, (void **)&s->grad,
                     (void **)&s->vol, (void **)&s->v, (void **)&s->r, (void **)&s->dv, (void **)&s->v_trial,
                     (void **)&s->rvol, (void **)&s->v_node, (void **)&s->g_start, (void **)&s->g_node,
                     (void **)&s->g_coef, (void **)&s->kvol, (void **)&s->val, (void **)&s->e_r, (void **)&s->e_k,
                     (void **)&s->e_energy, (void **)&s->e_power, (void **)&s->pr, (void **)&s->pz, (void **)&s->pp,
                     (void **)&s->pq};
    for (size_t k = 0; k < sizeof(ptrs) / sizeof(ptrs[0]); k++) {
        free(*ptrs[k]);
        *ptrs[k] = NULL;
    }
    s->g_len = 0;
}

void o3d_destroy(o3d *s)
{
    if (!s) return;
    free_mesh(s);
    free(s->die[0].h);
    free(s->die[1].h);
    o_trimesh_free(&s->die[0].tm);
    o_trimesh_free(&s->die[1].tm);
    ospd_destroy(s->lin);
    free(s);
}

#define NEW(T, n) ((T *)calloc((size_t)((n) > 0 ? (n) : 1), sizeof(T)))

static inline v3 X(const o3d *s, int n) { return V3(s->x[3 * n], s->x[3 * n + 1], s->x[3 * n + 2]); }
static inline v3 AX(const o3d *s, int n, int k) { const double *a = s->ax + 9 * n + 3 * k; return V3(a[0], a[1], a[2]); }
static inline v3 xget(const double *a, int n) { return V3(a[3 * n], a[3 * n + 1], a[3 * n + 2]); }
static inline void xset(double *a, int n, v3 v) { a[3 * n] = v.x; a[3 * n + 1] = v.y; a[3 * n + 2] = v.z; }

/* Forging3DSolver.cs:825, :827, :871 */
static inline v3 to_local(const o3d *s, int n, v3 g) { return V3(vdot(g, AX(s, n, 0)), vdot(g, AX(s, n, 1)), vdot(g, AX(s, n, 2))); }
static inline v3 to_global(const o3d *s, int n, double l0, double l1, double l2)
{
    return vadd(vadd(vscale(l0, AX(s, n, 0)), vscale(l1, AX(s, n, 1))), vscale(l2, AX(s, n, 2)));
}
static inline v3 global_velocity(const o3d *s, const double *v, int n) { return to_global(s, n, v[3 * n], v[3 * n + 1], v[3 * n + 2]); }
static inline v3 die_velocity(int c, double ram) { return c == TOP ? V3(0, 0, -ram) : V3(0, 0, 0); }
static inline double offset_of(int c, double gap) { return c == TOP ? gap : 0.0; }
static inline const o_hfdie *surface(const o3d *s, int c) { return c == TOP ? &s->die[1] : &s->die[0]; }
static inline v3 sym(const o3d *s, v3 p, int n) { return V3(s->on_x0[n] ? 0 : p.x, s->on_y0[n] ? 0 : p.y, p.z); }
static inline double tet_quality_x(const o3d *s, const double *x, int e)
{
    const int32_t *t = s->tets + 4 * e;
    return o_tet_quality4(xget(x, t[0]), xget(x, t[1]), xget(x, t[2]), xget(x, t[3]));
}

static int bsearch_i32(const int32_t *a, int n, int key)
{
    int lo = 0, hi = n - 1;
    while (lo <= hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] == key) return mid;
        if (a[mid] < key) lo = mid + 1; else hi = mid - 1;
    }
    return -1;
}

/* Pos (Forging3DSolver.cs:524) */
static inline int64_t pos(const o3d *s, int i, int ci, int j, int cj)
{
    return s->col_ptr[3 * j + cj] + 3 * bsearch_i32(s->nbr + s->nbr_start[j], s->nbr_start[j + 1] - s->nbr_start[j], i) + ci;
}

typedef struct { int32_t k[3]; int32_t ins; int32_t a, b, c, owner; } face_rec;
static int face_cmp(const void *pa, const void *pb)
{
    const face_rec *a = (const face_rec *)pa, *b = (const face_rec *)pb;
    for (int q = 0; q < 3; q++)
        if (a->k[q] != b->k[q]) return a->k[q] < b->k[q] ? -1 : 1;
    return a->ins < b->ins ? -1 : (a->ins > b->ins);
}
static int ins_cmp(const void *pa, const void *pb)
{
    const face_rec *a = (const face_rec *)pa, *b = (const face_rec *)pb;
    return a->ins < b->ins ? -1 : (a->ins > b->ins);
}
static int i32_cmp(const void *a, const void *b) { int x = *(const int32_t *)a, y = *(const int32_t *)b; return (x > y) - (x < y); }

/* TetMesh ctor (ThreeD/TetMesh.cs:9-65) + Allocate/BuildPattern/LocalLengths (Forging3DSolver.cs:403-521) */
int o3d_set_mesh(o3d *s, int nn, int ne, const double *x, const int32_t *tets, const uint8_t *on_x0, const uint8_t *on_y0)
{
    free_mesh(s);
    s->nn = nn; s->ne = ne; s->ndof = 3 * nn;
    s->tets = NEW(int32_t, 4 * ne); memcpy(s->tets, tets, sizeof(int32_t) * 4 * ne);
    s->on_x0 = NEW(uint8_t, nn); memcpy(s->on_x0, on_x0, nn);
    s->on_y0 = NEW(uint8_t, nn); memcpy(s->on_y0, on_y0, nn);
    for (int k = 0; k < 4 * ne; k++)
        if (tets[k] < 0 || tets[k] >= nn) return fail(s, E_INPUT, "tet references a node outside the mesh");
    /* node -> tet CSR */
    s->nts = NEW(int32_t, nn + 1);
    for (int k = 0; k < 4 * ne; k++) s->nts[tets[k] + 1]++;
    for (int i = 0; i < nn; i++) s->nts[i + 1] += s->nts[i];
    s->ntl = NEW(int32_t, 4 * ne);
    int32_t *fill = NEW(int32_t, nn + 1);
    memcpy(fill, s->nts, sizeof(int32_t) * (nn + 1));
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++) s->ntl[fill[tets[4 * e + a]]++] = e;
    free(fill);
    /* boundary faces, in Dictionary insertion order */
    face_rec *fr = NEW(face_rec, 4 * ne);
    for (int e = 0; e < ne; e++) {
        int a = tets[4 * e], b = tets[4 * e + 1], c = tets[4 * e + 2], d = tets[4 * e + 3];
        int f3[4][3] = {{a, c, b}, {a, b, d}, {a, d, c}, {b, c, d}};
        for (int f = 0; f < 4; f++) {
            face_rec *r = &fr[4 * e + f];
            int p = f3[f][0], q = f3[f][1], w = f3[f][2];
            r->a = p; r->b = q; r->c = w; r->owner = e; r->ins = 4 * e + f;
            int k0 = p, k1 = q, k2 = w, t;
            if (k0 > k1) { t = k0; k0 = k1; k1 = t; }
            if (k1 > k2) { t = k1; k1 = k2; k2 = t; }
            if (k0 > k1) { t = k0; k0 = k1; k1 = t; }
            r->k[0] = k0; r->k[1] = k1; r->k[2] = k2;
        }
    }
    qsort(fr, (size_t)4 * ne, sizeof(face_rec), face_cmp);
    face_rec *bf = NEW(face_rec, 4 * ne);
    int nbf = 0;
    for (int i = 0; i < 4 * ne;) {
        int j = i + 1;
        while (j < 4 * ne && memcmp(fr[j].k, fr[i].k, sizeof(fr[i].k)) == 0) j++;
        if (j - i > 2) { free(fr); free(bf); return fail(s, E_INPUT, "Tetrahedral mesh is not manifold (face shared by more than two tets)."); }
        if (j - i == 1) bf[nbf++] = fr[i];
        i = j;
    }
    free(fr);
    qsort(bf, (size_t)nbf, sizeof(face_rec), ins_cmp);
    s->nbf = nbf;
    s->bface = NEW(int32_t, 3 * nbf); s->bowner = NEW(int32_t, nbf); s->bsym = NEW(uint8_t, nbf);
    s->is_surface = NEW(uint8_t, nn);
    for (int k = 0; k < nbf; k++) {
        s->bface[3 * k] = bf[k].a; s->bface[3 * k + 1] = bf[k].b; s->bface[3 * k + 2] = bf[k].c;
        s->bowner[k] = bf[k].owner;
        s->bsym[k] = (on_x0[bf[k].a] && on_x0[bf[k].b] && on_x0[bf[k].c]) || (on_y0[bf[k].a] && on_y0[bf[k].b] && on_y0[bf[k].c]);
        if (!s->bsym[k])
            for (int a = 0; a < 3; a++) s->is_surface[s->bface[3 * k + a]] = 1;
    }
    free(bf);
    /* two-ring pattern (BuildPattern :469-521) */
    s->nbr_start = NEW(int32_t, nn + 1);
    int32_t *buf = NEW(int32_t, 1024);
    int cap = 1024;
    int64_t total = 0, tcap = (int64_t)nn * 64;
    int32_t *all = NEW(int32_t, tcap);
    int32_t *ring = NEW(int32_t, 256);
    int rcap = 256;
    for (int i = 0; i < nn; i++) {
        /* one ring of i (its patch) */
        int rn = 0;
        for (int32_t q = s->nts[i]; q < s->nts[i + 1]; q++) {
            int e = s->ntl[q];
            for (int a = 0; a < 4; a++) {
                if (rn == rcap) { rcap *= 2; ring = (int32_t *)realloc(ring, sizeof(int32_t) * rcap); }
                ring[rn++] = tets[4 * e + a];
            }
        }
        qsort(ring, (size_t)rn, sizeof(int32_t), i32_cmp);
        int u = 0;
        for (int k = 0; k < rn; k++) if (k == 0 || ring[k] != ring[k - 1]) ring[u++] = ring[k];
        rn = u;
        int bn = 0;
        for (int k = 0; k < rn; k++) {
            int n = ring[k];
            for (int32_t q = s->nts[n]; q < s->nts[n + 1]; q++) {
                int e = s->ntl[q];
                for (int a = 0; a < 4; a++) {
                    if (bn == cap) { cap *= 2; buf = (int32_t *)realloc(buf, sizeof(int32_t) * cap); }
                    buf[bn++] = tets[4 * e + a];
                }
            }
        }
        qsort(buf, (size_t)bn, sizeof(int32_t), i32_cmp);
        int m = 0;
        for (int k = 0; k < bn; k++) if (k == 0 || buf[k] != buf[k - 1]) buf[m++] = buf[k];
        if (total + m > tcap) { while (total + m > tcap) tcap *= 2; all = (int32_t *)realloc(all, sizeof(int32_t) * tcap); }
        memcpy(all + total, buf, sizeof(int32_t) * m);
        total += m;
        s->nbr_start[i + 1] = (int32_t)total;
    }
    free(buf); free(ring);
    s->nbr = all;
    s->col_ptr = NEW(int32_t, s->ndof + 1);
    for (int j = 0; j < nn; j++)
        for (int c = 0; c < 3; c++) s->col_ptr[3 * j + c + 1] = s->col_ptr[3 * j + c] + 3 * (s->nbr_start[j + 1] - s->nbr_start[j]);
    s->nnz = s->col_ptr[s->ndof];
    s->row_idx = NEW(int32_t, s->nnz);
    for (int j = 0; j < nn; j++)
        for (int c = 0; c < 3; c++) {
            int64_t p = s->col_ptr[3 * j + c];
            for (int32_t k = s->nbr_start[j]; k < s->nbr_start[j + 1]; k++) {
                int i = s->nbr[k];
                s->row_idx[p++] = 3 * i; s->row_idx[p++] = 3 * i + 1; s->row_idx[p++] = 3 * i + 2;
            }
        }
    /* EnsureElementBuffers slot map (:1248-1261) */
    s->e_nbr = NEW(int32_t, 16 * ne);
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                int j = tets[4 * e + b];
                s->e_nbr[16 * e + 4 * a + b] = bsearch_i32(s->nbr + s->nbr_start[j], s->nbr_start[j + 1] - s->nbr_start[j], tets[4 * e + a]);
            }
    /* state arrays */
    s->x = NEW(double, 3 * nn); memcpy(s->x, x, sizeof(double) * 3 * nn);
    s->vg = NEW(double, 3 * nn); s->vg_prev = NEW(double, 3 * nn); s->have_vg_prev = 0;
    s->eps = NEW(double, ne); s->dmg = NEW(double, ne); s->el_dev = NEW(double, 6 * ne);
    s->el_sig = NEW(double, ne); s->el_rate = NEW(double, ne); s->el_mean = NEW(double, ne);
    s->contact = NEW(uint8_t, nn); s->release = NEW(uint8_t, nn); s->fixed = NEW(uint8_t, s->ndof);
    s->ax = NEW(double, 9 * nn); s->n_fix = NEW(int32_t, nn); s->die_axis = NEW(int32_t, nn);
    s->fixed_val = NEW(double, s->ndof); s->k_fric = NEW(double, nn); s->a_fric = NEW(double, nn);
    s->grad = NEW(double, 12 * ne); s->vol = NEW(double, ne);
    s->v = NEW(double, s->ndof); s->r = NEW(double, s->ndof); s->dv = NEW(double, s->ndof);
    s->v_trial = NEW(double, s->ndof); s->rvol = NEW(double, s->ndof); s->v_node = NEW(double, nn);
    s->g_start = NEW(int32_t, nn + 1);
    s->kvol = NEW(double, s->nnz); s->val = NEW(double, s->nnz);
    s->e_r = NEW(double, 12 * ne); s->e_k = NEW(double, 144 * ne); s->e_energy = NEW(double, ne); s->e_power = NEW(double, ne);
    s->pr = NEW(double, s->ndof); s->pz = NEW(double, s->ndof); s->pp = NEW(double, s->ndof); s->pq = NEW(double, s->ndof);
    for (int e = 0; e < ne; e++) s->el_sig[e] = s->sig_ref;
    /* LocalLengths (:443-466) */
    s->h_local = NEW(double, nn);
    int32_t *cnt = NEW(int32_t, nn);
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++)
            for (int b = a + 1; b < 4; b++) {
                int i = tets[4 * e + a], j = tets[4 * e + b];
                double l = vlen(vsub(xget(x, i), xget(x, j)));
                s->h_local[i] += l; s->h_local[j] += l; cnt[i]++; cnt[j]++;
            }
    for (int n = 0; n < nn; n++) s->h_local[n] = cnt[n] > 0 ? dmin(s->h_local[n] / cnt[n], s->h) : s->h;
    free(cnt);
    s->need_analyze = 1;
    s->have_factor = 0;
    return E_OK;
}

int o3d_set_die(o3d *s, int side, int nx, int ny, double x0, double y0, double dx, const double *h)
{
    if (side < 0 || side > 1 || nx < 1 || ny < 1 || !(dx > 0)) return fail(s, E_INPUT, "invalid die");
    o_hfdie *d = &s->die[side];
    free(d->h);
    o_trimesh_free(&d->tm);
    d->kind = 0;
    d->side = side; d->nx = nx; d->ny = ny; d->x0 = x0; d->y0 = y0; d->dx = dx;
    d->h = NEW(double, (nx + 1) * (ny + 1));
    memcpy(d->h, h, sizeof(double) * (nx + 1) * (ny + 1));
    s->have_dies |= 1 << side;
    return E_OK;
}

/* TriMeshDie (ThreeD/TriMeshSolid.cs:248-297) in place of a height field */
int o3d_set_trimesh_die(o3d *s, int side, int nv, const double *v, int nt, const int *tri)
{
    if (side < 0 || side > 1) return fail(s, E_INPUT, "invalid die");
    o_hfdie *d = &s->die[side];
    free(d->h);
    d->h = NULL;
    if (o_trimesh_build(&d->tm, nv, v, nt, tri) != 0) return fail(s, E_INPUT, "invalid triangulated die");
    d->kind = 1;
    d->side = side;
    d->nx = d->ny = 1;
    d->x0 = d->tm.mn[0]; d->y0 = d->tm.mn[1]; d->dx = d->tm.c2;
    s->have_dies |= 1 << side;
    return E_OK;
}

double o3d_die_height(o3d *s, int side, double x, double y) { return hf_height(&s->die[side], x, y); }

double o3d_die_project(o3d *s, int side, const double *p, double offset, double *q, double *nrm)
{
    v3 n;
    v3 r = hf_project(&s->die[side], V3(p[0], p[1], p[2]), offset, &n);
    q[0] = r.x; q[1] = r.y; q[2] = r.z; nrm[0] = n.x; nrm[1] = n.y; nrm[2] = n.z;
    return vlen(vsub(r, V3(p[0], p[1], p[2])));
}

double o3d_die_clearance(o3d *s, int side, const double *p, double offset)
{
    return hf_clearance(&s->die[side], V3(p[0], p[1], p[2]), offset);
}

static double volume(const o3d *s)
{
    double v = 0;
    for (int e = 0; e < s->ne; e++) {
        const int32_t *t = s->tets + 4 * e;
        v += o_tet_volume(X(s, t[0]), X(s, t[1]), X(s, t[2]), X(s, t[3]));
    }
    return v * s->p.sym_factor;
}

/* ForceContact (:366-378) */
static void force_contact(o3d *s, int side)
{
    int best = -1;
    double bestC = DBL_MAX;
    for (int n = 0; n < s->nn; n++) {
        if (!s->is_surface[n]) continue;
        double c = side == BOTTOM ? hf_clearance(&s->die[0], X(s, n), 0) : hf_clearance(&s->die[1], X(s, n), s->gap);
        if (c < bestC) { bestC = c; best = n; }
    }
    if (best >= 0) s->contact[best] = (uint8_t)side;
}

/* Constructor tail (Forging3DSolver.cs:141-184) */
int o3d_init(o3d *s, double gap0, double min_x, double min_y, double min_z, double max_x, double max_y)
{
    if (s->have_dies != 3 || s->nn == 0) return fail(s, E_INPUT, "mesh and both dies must be set first");
    s->gap0 = s->gap = gap0;
    double tol = 0.05 * s->h;
    int nb = 0, nt = 0;
    for (int n = 0; n < s->nn; n++) {
        if (!s->is_surface[n]) continue;
        if (hf_clearance(&s->die[0], X(s, n), 0) < tol) { s->contact[n] = BOTTOM; nb++; }
        else if (hf_clearance(&s->die[1], X(s, n), s->gap) < tol) { s->contact[n] = TOP; nt++; }
    }
    if (nb == 0) force_contact(s, BOTTOM);
    if (nt == 0) force_contact(s, TOP);
    for (int n = 0; n < s->nn; n++) {
        if (s->contact[n] == FREE) continue;
        v3 nrm;
        v3 p = hf_project(surface(s, s->contact[n]), X(s, n), offset_of(s->contact[n], s->gap), &nrm);
        xset(s->x, n, sym(s, p, n));
    }
    for (int n = 0; n < s->nn; n++) {
        v3 p = X(s, n);
        double cx = 0.5 * (min_x + max_x), cy = 0.5 * (min_y + max_y);
        xset(s->vg, n, V3(0.5 * s->rate_ref * (p.x - cx), 0.5 * s->rate_ref * (p.y - cy), -s->rate_ref * (p.z - min_z)));
    }
    s->vol0 = volume(s);
    return E_OK;
}

/* BuildAnp (:761-823) */
static void build_anp(o3d *s)
{
    const int32_t *t = s->tets;
    memset(s->v_node, 0, sizeof(double) * s->nn);
    for (int e = 0; e < s->ne; e++)
        for (int a = 0; a < 4; a++) s->v_node[t[4 * e + a]] += s->vol[e] / 4;
    /* first pass: size */
    int64_t total = 0;
    int maxdeg = 0;
    for (int n = 0; n < s->nn; n++) maxdeg = imax(maxdeg, s->nts[n + 1] - s->nts[n]);
    int32_t *mapn = NEW(int32_t, 4 * maxdeg + 4);
    for (int n = 0; n < s->nn; n++) {
        int cnt = 0;
        for (int32_t q = s->nts[n]; q < s->nts[n + 1]; q++) {
            int e = s->ntl[q];
            for (int a = 0; a < 4; a++) {
                int m = t[4 * e + a], found = 0;
                for (int k = 0; k < cnt; k++) if (mapn[k] == m) { found = 1; break; }
                if (!found) mapn[cnt++] = m;
            }
        }
        total += cnt;
    }
    free(s->g_node); free(s->g_coef);
    s->g_node = NEW(int32_t, total);
    s->g_coef = NEW(double, 3 * total);
    s->g_len = total;
    int64_t pcount = 0;
    for (int n = 0; n < s->nn; n++) {
        int64_t base = pcount;
        for (int32_t q = s->nts[n]; q < s->nts[n + 1]; q++) {
            int e = s->ntl[q];
            double w = s->vol[e] / 4 / s->v_node[n];
            for (int a = 0; a < 4; a++) {
                int m = t[4 * e + a];
                v3 gc = vscale(w, V3(s->grad[12 * e + 3 * a], s->grad[12 * e + 3 * a + 1], s->grad[12 * e + 3 * a + 2]));
                int64_t idx = -1;
                for (int64_t k = base; k < pcount; k++) if (s->g_node[k] == m) { idx = k; break; }
                if (idx >= 0) {
                    v3 c = vadd(xget(s->g_coef, (int)idx), gc);
                    xset(s->g_coef, (int)idx, c);
                } else {
                    s->g_node[pcount] = m;
                    xset(s->g_coef, (int)pcount, gc);
                    pcount++;
                }
            }
        }
        s->g_start[n + 1] = (int32_t)pcount;
    }
    free(mapn);
    memset(s->kvol, 0, sizeof(double) * s->nnz);
    for (int n = 0; n < s->nn; n++) {
        double kv = s->k_pen * s->v_node[n];
        for (int32_t p = s->g_start[n]; p < s->g_start[n + 1]; p++) {
            int i = s->g_node[p];
            v3 ci = to_local(s, i, xget(s->g_coef, p));
            for (int32_t q = s->g_start[n]; q < s->g_start[n + 1]; q++) {
                int j = s->g_node[q];
                v3 cj = to_local(s, j, xget(s->g_coef, q));
                double block[9];
                for (int r = 0; r < 3; r++)
                    for (int c = 0; c < 3; c++) block[3 * r + c] = vget(ci, r) * vget(cj, c);
                /* AddBlock (:526-534) */
                int k = bsearch_i32(s->nbr + s->nbr_start[j], s->nbr_start[j + 1] - s->nbr_start[j], i);
                for (int cj2 = 0; cj2 < 3; cj2++) {
                    int64_t pp = s->col_ptr[3 * j + cj2] + 3 * k;
                    for (int ci2 = 0; ci2 < 3; ci2++) s->kvol[pp + ci2] += kv * block[ci2 * 3 + cj2];
                }
            }
        }
    }
}

/* BuildFriction (:829-850) */
static void build_friction(o3d *s)
{
    memset(s->a_fric, 0, sizeof(double) * s->nn);
    double *ksum = NEW(double, s->nn);
    int32_t *kcnt = NEW(int32_t, s->nn);
    for (int k = 0; k < s->nbf; k++) {
        if (s->bsym[k]) continue;
        int a = s->bface[3 * k], b = s->bface[3 * k + 1], c = s->bface[3 * k + 2];
        double area = 0.5 * vlen(vcross(vsub(X(s, b), X(s, a)), vsub(X(s, c), X(s, a))));
        double kk = s->el_sig[s->bowner[k]] / sqrt(3.0);
        int nodes[3] = {a, b, c};
        for (int q = 0; q < 3; q++) {
            int n = nodes[q];
            s->a_fric[n] += area / 3;
            ksum[n] += kk;
            kcnt[n]++;
        }
    }
    for (int n = 0; n < s->nn; n++) s->k_fric[n] = kcnt[n] > 0 ? ksum[n] / kcnt[n] : 0;
    free(ksum); free(kcnt);
}

/* LoadVelocityGuess (:854-869) */
static void load_velocity_guess(o3d *s)
{
    int trend = s->p.extrapolate_start && s->warm && s->have_vg_prev;
    for (int n = 0; n < s->nn; n++) {
        v3 g = xget(s->vg, n);
        if (trend) g = vsub(vscale(2, g), xget(s->vg_prev, n));
        v3 l = to_local(s, n, g);
        s->v[3 * n] = l.x; s->v[3 * n + 1] = l.y; s->v[3 * n + 2] = l.z;
    }
    for (int d = 0; d < s->ndof; d++)
        if (s->fixed[d]) s->v[d] = s->fixed_val[d];
}

/* PrepareStep (:660-758) */
int o3d_prepare_step(o3d *s)
{
    memset(s->fixed, 0, s->ndof);
    memset(s->fixed_val, 0, sizeof(double) * s->ndof);
    memset(s->release, 0, s->nn);
    v3 dirs[3], e[3];
    double vals[3], ev[3];
    e[0] = e[1] = e[2] = V3(0, 0, 0);
    ev[0] = ev[1] = ev[2] = 0;
    for (int n = 0; n < s->nn; n++) {
        int k = 0;
        s->die_axis[n] = -1;
        if (s->on_x0[n]) { dirs[k] = V3(1, 0, 0); vals[k] = 0; k++; }
        if (s->on_y0[n]) { dirs[k] = V3(0, 1, 0); vals[k] = 0; k++; }
        int die_idx = -1;
        if (s->contact[n] != FREE) {
            v3 nrm;
            hf_project(surface(s, s->contact[n]), X(s, n), offset_of(s->contact[n], s->gap), &nrm);
            dirs[k] = nrm;
            vals[k] = vdot(die_velocity(s->contact[n], s->p.ram), nrm);
            die_idx = k;
            k++;
        }
        int m = 0;
        for (int q = 0; q < k; q++) {
            v3 d = dirs[q];
            double val = vals[q];
            for (int sidx = 0; sidx < m; sidx++) {
                double proj = vdot(d, e[sidx]);
                d = vsub(d, vscale(proj, e[sidx]));
                val -= proj * ev[sidx];
            }
            double len = vlen(d);
            if (len < 0.2) continue;
            e[m] = vscale(1 / len, d);
            ev[m] = val / len;
            if (q == die_idx) s->die_axis[n] = m;
            m++;
        }
        if (m == 0) { e[0] = V3(1, 0, 0); e[1] = V3(0, 1, 0); e[2] = V3(0, 0, 1); }
        else if (m == 1) {
            v3 helper = fabs(e[0].x) < 0.8 ? V3(1, 0, 0) : V3(0, 1, 0);
            e[1] = vnormalized(vcross(e[0], helper));
            e[2] = vcross(e[0], e[1]);
        } else if (m == 2) {
            e[2] = vnormalized(vcross(e[0], e[1]));
        }
        for (int a = 0; a < 3; a++) { s->ax[9 * n + 3 * a] = e[a].x; s->ax[9 * n + 3 * a + 1] = e[a].y; s->ax[9 * n + 3 * a + 2] = e[a].z; }
        s->n_fix[n] = m;
        for (int q = 0; q < m; q++) { s->fixed[3 * n + q] = 1; s->fixed_val[3 * n + q] = ev[q]; }
    }
    const int32_t *t = s->tets;
    for (int el = 0; el < s->ne; el++) {
        v3 p0 = X(s, t[4 * el]);
        v3 a = vsub(X(s, t[4 * el + 1]), p0), b = vsub(X(s, t[4 * el + 2]), p0), c = vsub(X(s, t[4 * el + 3]), p0);
        double det = vdot(a, vcross(b, c));
        if (!(det > 0)) {
            char msg[160];
            snprintf(msg, sizeof msg, "Tetrahedron %d is inverted at step %d.", el, s->step_index);
            return fail(s, E_DISTORTED, msg);
        }
        v3 g1 = vscale(1 / det, vcross(b, c)), g2 = vscale(1 / det, vcross(c, a)), g3 = vscale(1 / det, vcross(a, b));
        v3 g0 = vneg(vadd(vadd(g1, g2), g3));
        v3 g[4] = {g0, g1, g2, g3};
        for (int q = 0; q < 4; q++) {
            s->grad[12 * el + 3 * q] = g[q].x; s->grad[12 * el + 3 * q + 1] = g[q].y; s->grad[12 * el + 3 * q + 2] = g[q].z;
        }
        s->vol[el] = det / 6;
    }
    build_anp(s);
    build_friction(s);
    load_velocity_guess(s);
    return E_OK;
}

/* Kernel (:1312-1400) */
static void kernel(o3d *s, int e, int matrix, int newton, const double *ve, double *re, double *ke, double *energy, double *power)
{
    double vol = s->vol[e];
    int o = 12 * e;
    double B[72], MB[72], G[12];
    memset(B, 0, sizeof B);
    for (int a = 0; a < 4; a++) {
        double bx = s->grad[o + 3 * a], by = s->grad[o + 3 * a + 1], bz = s->grad[o + 3 * a + 2];
        int c = 3 * a;
        B[0 * 12 + c] = bx;
        B[1 * 12 + c + 1] = by;
        B[2 * 12 + c + 2] = bz;
        B[3 * 12 + c] = by; B[3 * 12 + c + 1] = bx;
        B[4 * 12 + c + 1] = bz; B[4 * 12 + c + 2] = by;
        B[5 * 12 + c] = bz; B[5 * 12 + c + 2] = bx;
    }
    double eps[6];
    for (int i = 0; i < 6; i++) {
        double sum = 0;
        for (int k = 0; k < 12; k++) sum += B[i * 12 + k] * ve[k];
        eps[i] = sum;
    }
    double ev3 = (eps[0] + eps[1] + eps[2]) / 3;
    double d0 = eps[0] - ev3, d1 = eps[1] - ev3, d2 = eps[2] - ev3;
    double rate = sqrt(dmax(2.0 / 3.0 * (d0 * d0 + d1 * d1 + d2 * d2) + (eps[3] * eps[3] + eps[4] * eps[4] + eps[5] * eps[5]) / 3.0, 0));
    double me[6];
    me[0] = 2.0 / 3.0 * d0; me[1] = 2.0 / 3.0 * d1; me[2] = 2.0 / 3.0 * d2;
    me[3] = eps[3] / 3; me[4] = eps[4] / 3; me[5] = eps[5] / 3;
    for (int k = 0; k < 12; k++) {
        double sum = 0;
        for (int i = 0; i < 6; i++) sum += B[i * 12 + k] * me[i];
        G[k] = sum;
    }
    double strain = s->eps[e];
    double sigCut = law_stress(s->p.C, s->p.N, s->p.M, s->p.eps0, strain, s->rate_cut);
    double mu0 = sigCut / s->rate_cut, mExp = s->p.M;
    double mu, sig, wDens, coefN;
    if (rate > s->rate_cut) {
        sig = law_stress(s->p.C, s->p.N, s->p.M, s->p.eps0, strain, rate);
        mu = sig / rate;
        wDens = 0.5 * sigCut * s->rate_cut + (sig * rate - sigCut * s->rate_cut) / (mExp + 1);
        coefN = (mExp - 1) * mu / (rate * rate);
    } else {
        mu = mu0;
        sig = mu0 * rate;
        wDens = 0.5 * mu0 * rate * rate;
        coefN = 0;
    }
    *energy = vol * wDens;
    *power = vol * sig * rate;
    for (int k = 0; k < 12; k++) re[k] = vol * mu * G[k];
    s->el_sig[e] = sig;
    s->el_rate[e] = rate;
    for (int i = 0; i < 6; i++) s->el_dev[6 * e + i] = mu * me[i];
    if (!matrix) return;
    for (int k = 0; k < 12; k++) {
        double tr = (B[k] + B[12 + k] + B[24 + k]) / 3;
        MB[k] = 2.0 / 3.0 * (B[k] - tr);
        MB[12 + k] = 2.0 / 3.0 * (B[12 + k] - tr);
        MB[24 + k] = 2.0 / 3.0 * (B[24 + k] - tr);
        MB[36 + k] = B[36 + k] / 3;
        MB[48 + k] = B[48 + k] / 3;
        MB[60 + k] = B[60 + k] / 3;
    }
    double wm = vol * mu, wn = newton ? vol * coefN * s->p.newton_blend : 0;
    for (int p = 0; p < 12; p++)
        for (int q = p; q < 12; q++) {
            double sum = 0;
            for (int i = 0; i < 6; i++) sum += B[i * 12 + p] * MB[i * 12 + q];
            double val = wm * sum + wn * G[p] * G[q];
            ke[p * 12 + q] = val;
            ke[q * 12 + p] = val;
        }
}

/* ElementWork (:1265-1310) */
static void element_work(o3d *s, int e, int matrix, int newton, const double *v)
{
    const int32_t *t = s->tets;
    double ve[12], re[12], ke[144];
    for (int a = 0; a < 4; a++) {
        v3 g = global_velocity(s, v, t[4 * e + a]);
        ve[3 * a] = g.x; ve[3 * a + 1] = g.y; ve[3 * a + 2] = g.z;
    }
    kernel(s, e, matrix, newton, ve, re, ke, &s->e_energy[e], &s->e_power[e]);
    for (int a = 0; a < 4; a++) {
        v3 rl = to_local(s, t[4 * e + a], V3(re[3 * a], re[3 * a + 1], re[3 * a + 2]));
        s->e_r[12 * e + 3 * a] = rl.x; s->e_r[12 * e + 3 * a + 1] = rl.y; s->e_r[12 * e + 3 * a + 2] = rl.z;
    }
    if (!matrix) return;
    double blk[9];
    for (int a = 0; a < 4; a++) {
        int i = t[4 * e + a];
        for (int b = 0; b < 4; b++) {
            int j = t[4 * e + b];
            int64_t o = 144 * (int64_t)e + 9 * (4 * a + b);
            for (int r = 0; r < 3; r++) {
                v3 ar = AX(s, i, r);
                for (int c = 0; c < 3; c++)
                    blk[3 * r + c] = ar.x * ke[(3 * a) * 12 + 3 * b + c] + ar.y * ke[(3 * a + 1) * 12 + 3 * b + c] + ar.z * ke[(3 * a + 2) * 12 + 3 * b + c];
            }
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) {
                    v3 bc = AX(s, j, c);
                    s->e_k[o + 3 * r + c] = blk[3 * r] * bc.x + blk[3 * r + 1] * bc.y + blk[3 * r + 2] * bc.z;
                }
        }
    }
}

/* Assemble (:1115-1217) */
double o3d_assemble(o3d *s, int matrix, int newton, const double *v, double *power_out)
{
    s->n_assemble++;
    memset(s->rvol, 0, sizeof(double) * s->ndof);
    for (int j = 0; j < s->ndof; j++) {
        double vj = v[j];
        if (vj == 0) continue;
        for (int32_t p = s->col_ptr[j]; p < s->col_ptr[j + 1]; p++) s->rvol[s->row_idx[p]] += s->kvol[p] * vj;
    }
    double energy = 0;
    for (int d = 0; d < s->ndof; d++) energy += 0.5 * v[d] * s->rvol[d];
    double power = 2 * energy;
    memcpy(s->r, s->rvol, sizeof(double) * s->ndof);
    if (matrix) memcpy(s->val, s->kvol, sizeof(double) * s->nnz);
    const int32_t *t = s->tets;
#pragma omp parallel for schedule(static)
    for (int e = 0; e < s->ne; e++) element_work(s, e, matrix, newton, v);
    for (int e = 0; e < s->ne; e++) {
        energy += s->e_energy[e];
        power += s->e_power[e];
        for (int a = 0; a < 4; a++) {
            int n = t[4 * e + a];
            s->r[3 * n] += s->e_r[12 * e + 3 * a];
            s->r[3 * n + 1] += s->e_r[12 * e + 3 * a + 1];
            s->r[3 * n + 2] += s->e_r[12 * e + 3 * a + 2];
        }
        if (!matrix) continue;
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                int j = t[4 * e + b], k = s->e_nbr[16 * e + 4 * a + b];
                int64_t o = 144 * (int64_t)e + 9 * (4 * a + b);
                for (int cj = 0; cj < 3; cj++) {
                    int64_t p = s->col_ptr[3 * j + cj] + 3 * k;
                    for (int ci = 0; ci < 3; ci++) s->val[p + ci] += s->e_k[o + 3 * ci + cj];
                }
            }
    }
    double m = s->p.friction;
    if (m > 0) {
        for (int n = 0; n < s->nn; n++) {
            if (s->contact[n] == FREE || s->n_fix[n] >= 3) continue;
            double c = m * s->k_fric[n] * s->a_fric[n] * (2 / M_PI);
            if (c <= 0) continue;
            v3 vd = to_local(s, n, die_velocity(s->contact[n], s->p.ram));
            int k0 = s->n_fix[n];
            double sv[3] = {0, 0, 0}, s2 = 0;
            for (int q = k0; q < 3; q++) {
                sv[q] = v[3 * n + q] - vget(vd, q);
                s2 += sv[q] * sv[q];
            }
            double sl = sqrt(s2), z = sl / s->u0, at = atan(z);
            energy += c * (sl * at - 0.5 * s->u0 * log(1 + z * z));
            power += c * at * sl;
            double gs = sl > 1e-12 * s->u0 ? at / sl : 1 / s->u0;
            for (int q = k0; q < 3; q++) s->r[3 * n + q] += c * gs * sv[q];
            if (!matrix) continue;
            double tang = c / (s->u0 * (1 + z * z));
            for (int q = k0; q < 3; q++)
                for (int p = k0; p < 3; p++) {
                    double kqp;
                    if (newton && sl > 1e-12 * s->u0)
                        kqp = c * gs * ((q == p ? 1 : 0) - sv[q] * sv[p] / s2) + tang * sv[q] * sv[p] / s2;
                    else
                        kqp = q == p ? c * gs : 0;
                    s->val[pos(s, n, q, n, p)] += kqp;
                }
        }
    }
    if (power_out) *power_out = power;
    return energy;
}

static double norm(const double *a, int n)
{
    double sum = 0;
    for (int k = 0; k < n; k++) sum += a[k] * a[k];
    return sqrt(sum);
}
static double dot(const double *a, const double *b, int n)
{
    double sum = 0;
    for (int k = 0; k < n; k++) sum += a[k] * b[k];
    return sum;
}

/* MatVec (:1089-1098) */
static void matvec(const o3d *s, const double *v, double *y)
{
    memset(y, 0, sizeof(double) * s->ndof);
    for (int j = 0; j < s->ndof; j++) {
        double vj = v[j];
        if (vj == 0) continue;
        for (int32_t p = s->col_ptr[j]; p < s->col_ptr[j + 1]; p++) y[s->row_idx[p]] += s->val[p] * vj;
    }
}

/* Pcg (:1051-1087) */
static int pcg(o3d *s, const double *b, double *x, double tol, int max_it)
{
    int n = s->ndof;
    double bnorm = norm(b, n);
    if (bnorm == 0) { memset(x, 0, sizeof(double) * n); return 0; }
    ospd_solve(s->lin, b, x);
    matvec(s, x, s->pq);
    for (int i = 0; i < n; i++) s->pr[i] = b[i] - s->pq[i];
    ospd_solve(s->lin, s->pr, s->pz);
    memcpy(s->pp, s->pz, sizeof(double) * n);
    double rz = dot(s->pr, s->pz, n);
    for (int it = 0; it < max_it; it++) {
        if (norm(s->pr, n) <= tol * bnorm) return it;
        matvec(s, s->pp, s->pq);
        double alpha = rz / dot(s->pp, s->pq, n);
        for (int i = 0; i < n; i++) {
            x[i] += alpha * s->pp[i];
            s->pr[i] -= alpha * s->pq[i];
        }
        ospd_solve(s->lin, s->pr, s->pz);
        double rzNew = dot(s->pr, s->pz, n);
        double beta = rzNew / rz;
        rz = rzNew;
        for (int i = 0; i < n; i++) s->pp[i] = s->pz[i] + beta * s->pp[i];
    }
    return norm(s->pr, n) <= tol * bnorm ? max_it : -1;
}

/* SolveLinear (:965-1019); returns 0 (pcg) / 1 (factorised) / <0 error */
static int solve_linear(o3d *s, const double *b, double *x)
{
    if (s->have_factor && s->pcg_skip > 0) {
        s->pcg_skip--;
    } else if (s->have_factor) {
        int its = pcg(s, b, x, 1e-7, s->p.pcg_budget);
        if (its >= 0) {
            s->pcg_failures = 0;
            s->n_pcg++;
            s->lin_its_total += its;
            return 0;
        }
        if (++s->pcg_failures >= 2) s->pcg_skip = imin(64, 1 << (s->pcg_failures - 1));
    }
    if (s->need_analyze) {
        ospd_set_geometry(s->lin, s->nn, s->x);
        ospd_analyze(s->lin, s->ndof, s->col_ptr, s->row_idx);
        s->need_analyze = 0;
    }
    if (ospd_factorize(s->lin, s->val) != 0) {
        s->have_factor = 0;
        char msg[200];
        snprintf(msg, sizeof msg, "Sparse factorisation failed at step %d (oracle multifrontal Cholesky): not positive definite at equation %d.",
                 s->step_index, ospd_bad_pivot(s->lin));
        return -fail(s, E_DIVERGED, msg);
    }
    if (ospd_solve(s->lin, b, x) != 0) {
        s->have_factor = 0;
        return -fail(s, E_DIVERGED, "Sparse factorisation failed: non-finite solution.");
    }
    s->have_factor = 1;
    s->n_fact++;
    return 1;
}

/* BC zeroing and regularisation (:892-913) */
int o3d_apply_bc(o3d *s, double *max_diag_out)
{
    double maxDiag = 0;
    for (int j = 0; j < s->ndof; j++)
        for (int32_t p = s->col_ptr[j]; p < s->col_ptr[j + 1]; p++) {
            int i = s->row_idx[p];
            if (s->fixed[i] || s->fixed[j]) s->val[p] = i == j ? 1 : 0;
            else if (i == j) maxDiag = dmax(maxDiag, s->val[p]);
        }
    double reg = 1e-10 * maxDiag;
    for (int j = 0; j < s->ndof; j++)
        if (!s->fixed[j]) s->val[pos(s, j / 3, j % 3, j / 3, j % 3)] += reg;
    for (int d = 0; d < s->ndof; d++)
        if (s->fixed[d]) s->r[d] = 0;
    if (max_diag_out) *max_diag_out = maxDiag;
    s->max_diag_last = maxDiag;
    return E_OK;
}

/* SolveVelocity (:875-948); returns iterations or -error */
int o3d_solve_velocity(o3d *s, int *converged)
{
    *converged = 0;
    s->last_rel = INFINITY;
    int it, halved = 0, secant_only = 0;
    const int newton_limit = 20;
    for (it = 1; it <= s->p.max_iter; it++) {
        if (s->p.sticky_secant && halved >= 2) secant_only = 1;
        int newton = (s->warm || it > 2) && it <= newton_limit && !secant_only && !(s->p.adaptive_newton && halved >= 2);
        if (newton) s->n_newton++;
        double e0 = o3d_assemble(s, 1, newton, s->v, NULL);
        o3d_apply_bc(s, NULL);
        s->rnorm_last = norm(s->r, s->ndof);
        for (int d = 0; d < s->ndof; d++) s->r[d] = -s->r[d];
        int how = solve_linear(s, s->r, s->dv);
        if (how < 0) return how;
        double slope = 0;
        for (int d = 0; d < s->ndof; d++) slope -= s->r[d] * s->dv[d];
        double beta = 1;
        for (int ls = 0; ls < 8; ls++) {
            for (int d = 0; d < s->ndof; d++) s->v_trial[d] = s->v[d] + beta * s->dv[d];
            double e1 = o3d_assemble(s, 0, 0, s->v_trial, NULL);
            if (e1 <= e0 + 1e-4 * beta * slope + 1e-11 * fabs(e0)) break;
            double curv = (e1 - e0 - slope * beta) / (beta * beta);
            beta = s->p.quadratic_ls && curv > 0 ? dclamp(-slope / (2 * curv), 0.1 * beta, 0.7 * beta) : 0.5 * beta;
        }
        memcpy(s->v, s->v_trial, sizeof(double) * s->ndof);
        halved = newton && beta < 1 ? halved + 1 : 0;
        double rel = beta * norm(s->dv, s->ndof) / dmax(norm(s->v, s->ndof), 1e-30);
        s->last_rel = rel;
        s->beta_last = beta;
        if (isnan(rel)) {
            char msg[120];
            snprintf(msg, sizeof msg, "Velocity solution became NaN at step %d.", s->step_index);
            return -fail(s, E_DIVERGED, msg);
        }
        if (rel < s->p.tol) { *converged = 1; return it; }
    }
    return it - 1;
}

/* FinalEvaluation (:1402-1451) */
double o3d_final_evaluation(o3d *s, double *reaction_out)
{
    double power;
    o3d_assemble(s, 0, 0, s->v, &power);
    memcpy(s->vg_prev, s->vg, sizeof(double) * 3 * s->nn);
    s->have_vg_prev = 1;
    double reaction = 0, maxB = 0, maxT = 0;
    for (int n = 0; n < s->nn; n++) {
        xset(s->vg, n, global_velocity(s, s->v, n));
        if (s->contact[n] == FREE) continue;
        v3 rg = to_global(s, n, s->r[3 * n], s->r[3 * n + 1], s->r[3 * n + 2]);
        if (s->contact[n] == TOP) reaction -= rg.z;
        if (s->die_axis[n] < 0) continue;
        double comp = s->r[3 * n + s->die_axis[n]];
        if (s->contact[n] == TOP) maxT = dmax(maxT, comp); else maxB = dmax(maxB, comp);
    }
    int keptB = 0, keptT = 0;
    for (int n = 0; n < s->nn; n++) {
        if (s->contact[n] == FREE || s->die_axis[n] < 0) continue;
        double comp = s->r[3 * n + s->die_axis[n]];
        double thr = 0.02 * (s->contact[n] == TOP ? maxT : maxB);
        if (comp < -thr) s->release[n] = 1;
        else if (s->contact[n] == TOP) keptT++;
        else keptB++;
    }
    if (keptB == 0 || keptT == 0)
        for (int n = 0; n < s->nn; n++)
            if ((keptT == 0 && s->contact[n] == TOP) || (keptB == 0 && s->contact[n] == BOTTOM)) s->release[n] = 0;
    double *nodal = NEW(double, s->nn);
    for (int n = 0; n < s->nn; n++) {
        double ev = 0;
        for (int32_t p = s->g_start[n]; p < s->g_start[n + 1]; p++) ev += vdot(xget(s->g_coef, p), xget(s->vg, s->g_node[p]));
        nodal[n] = s->k_pen * ev;
    }
    const int32_t *t = s->tets;
    for (int e = 0; e < s->ne; e++)
        s->el_mean[e] = 0.25 * (nodal[t[4 * e]] + nodal[t[4 * e + 1]] + nodal[t[4 * e + 2]] + nodal[t[4 * e + 3]]);
    free(nodal);
    s->reaction = reaction;
    if (reaction_out) *reaction_out = reaction;
    return power;
}

/* SurfaceNormals (:1540-1562) */
static void surface_normals(const o3d *s, const double *x, double *nrm)
{
    memset(nrm, 0, sizeof(double) * 3 * s->nn);
    for (int k = 0; k < s->nbf; k++) {
        if (s->bsym[k]) continue;
        int a = s->bface[3 * k], b = s->bface[3 * k + 1], c = s->bface[3 * k + 2];
        v3 an = vcross(vsub(xget(x, b), xget(x, a)), vsub(xget(x, c), xget(x, a)));
        xset(nrm, a, vadd(xget(nrm, a), an));
        xset(nrm, b, vadd(xget(nrm, b), an));
        xset(nrm, c, vadd(xget(nrm, c), an));
    }
    for (int i = 0; i < s->nn; i++) {
        v3 n = xget(nrm, i);
        if (s->on_x0[i]) n.x = 0;
        if (s->on_y0[i]) n.y = 0;
        if (vlen2(n) > 0) n = vnormalized(n);
        xset(nrm, i, n);
    }
}

static double tol_len(const o3d *s, double local) { return s->recovery_pass >= 2 ? s->h : local; }
static double corner_allowance(const o3d *s, double local)
{
    static const double ladder[2] = {0.05, 0.1};
    return s->recovery_pass >= 2 ? 0.3 * s->h : ladder[iclamp(s->recovery_pass, 0, 1)] * local;
}

/* PushOut (:1570-1589) */
static v3 push_out(const o3d *s, const o_hfdie *die, double offset, v3 p, v3 outward)
{
    v3 nrm;
    if (vlen2(outward) == 0 || hf_clearance(die, p, offset) >= 0) return hf_project(die, p, offset, &nrm);
    v3 d = vneg(outward);
    double step = 0.1 * s->h, lo = 0, hi = -1;
    for (double t = step; t <= 2 * s->h + 1e-12; t += step) {
        if (hf_clearance(die, vadd(p, vscale(t, d)), offset) >= 0) { hi = t; break; }
        lo = t;
    }
    if (hi < 0) return hf_project(die, p, offset, &nrm);
    for (int i = 0; i < 25; i++) {
        double mid = 0.5 * (lo + hi);
        if (hf_clearance(die, vadd(p, vscale(mid, d)), offset) >= 0) hi = mid; else lo = mid;
    }
    return vadd(p, vscale(hi, d));
}

static double worst_around(const o3d *s, const double *x, int n)
{
    double q = DBL_MAX;
    for (int32_t k = s->nts[n]; k < s->nts[n + 1]; k++) q = dmin(q, tet_quality_x(s, x, s->ntl[k]));
    return q;
}

/* ImprovePlacement (:1625-1679) */
static int improve_placement(o3d *s, double *x, uint8_t *contact, const double *pred, const double *nrm, double gap, double qmin)
{
    int total = 0;
    v3 cand[8];
    for (int sweep = 0; sweep < 4; sweep++) {
        int count = 0;
        for (int e = 0; e < s->ne; e++) {
            if (tet_quality_x(s, x, e) >= qmin) continue;
            for (int a = 0; a < 4; a++) {
                int n = s->tets[4 * e + a];
                if (contact[n] == FREE) continue;
                const o_hfdie *die = surface(s, contact[n]);
                double off = offset_of(contact[n], gap);
                int k = 0;
                v3 tmp;
                v3 pn = xget(pred, n);
                v3 closest = sym(s, hf_project(die, pn, off, &tmp), n);
                cand[k++] = closest;
                v3 push = sym(s, push_out(s, die, off, pn, xget(nrm, n)), n);
                if (vlen(vsub(push, pn)) <= 0.5 * tol_len(s, s->h_local[n])) cand[k++] = push;
                double pen = -hf_clearance(die, pn, off);
                static const double fs[4] = {0.0, 0.25, 0.5, 0.75};
                for (int q = 0; q < 4; q++)
                    if (pen * (1 - fs[q]) <= corner_allowance(s, s->h_local[n])) cand[k++] = vlerp(pn, closest, fs[q]);
                v3 old = xget(x, n);
                double best = worst_around(s, x, n);
                int pick = -1;
                for (int c = 0; c < k; c++) {
                    if (veq(cand[c], old)) continue;
                    xset(x, n, cand[c]);
                    double q = worst_around(s, x, n);
                    if (q > best + 1e-6) { best = q; pick = c; }
                }
                xset(x, n, pick >= 0 ? cand[pick] : old);
                if (pick < 0) continue;
                if (veq(cand[pick], pn) && pen < 0) contact[n] = FREE;
                if (hf_clearance(die, cand[pick], off) < -1e-9) s->corner_penetrations++;
                count++;
            }
        }
        total += count;
        if (count == 0) break;
    }
    return total;
}

/* SmoothInterior (:1776-1838) */
static int smooth_interior(const o3d *s, double *x, double qtarget, int sweeps)
{
    int moves = 0;
    uint8_t *bad = NEW(uint8_t, s->nn);
    for (int sw = 0; sw < sweeps; sw++) {
        memset(bad, 0, s->nn);
        int any = 0;
        for (int e = 0; e < s->ne; e++) {
            if (tet_quality_x(s, x, e) >= qtarget) continue;
            for (int a = 0; a < 4; a++) bad[s->tets[4 * e + a]] = 1;
            any = 1;
        }
        if (!any) break;
        int sweep_moves = 0;
        for (int n = 0; n < s->nn; n++) {
            if (!bad[n] || s->is_surface[n]) continue;
            v3 sum = V3(0, 0, 0);
            int cnt = 0;
            double worst = DBL_MAX;
            for (int32_t k = s->nts[n]; k < s->nts[n + 1]; k++) {
                int e = s->ntl[k];
                for (int a = 0; a < 4; a++) {
                    int m = s->tets[4 * e + a];
                    if (m == n) continue;
                    sum = vadd(sum, xget(x, m));
                    cnt++;
                }
                worst = dmin(worst, tet_quality_x(s, x, e));
            }
            if (cnt == 0) continue;
            v3 old = xget(x, n);
            v3 c = vscale(1.0 / cnt, sum);
            static const double lambdas[3] = {1.0, 0.5, 0.25};
            for (int l = 0; l < 3; l++) {
                v3 p = vadd(old, vscale(lambdas[l], vsub(c, old)));
                xset(x, n, V3(s->on_x0[n] ? 0 : p.x, s->on_y0[n] ? 0 : p.y, p.z));
                double q = DBL_MAX;
                for (int32_t k = s->nts[n]; k < s->nts[n + 1]; k++) q = dmin(q, tet_quality_x(s, x, s->ntl[k]));
                if (q > worst + 1e-6) { sweep_moves++; break; }
                xset(x, n, old);
            }
        }
        moves += sweep_moves;
        if (sweep_moves == 0) break;
    }
    free(bad);
    return moves;
}

/* TryUpdate (:1455-1537) */
int o3d_try_update(o3d *s, double dt, int *ok)
{
    double gapT = dmax(0, s->gap - s->p.ram * dt);
    if (gapT < 1e-9) gapT = 0;
    int nn = s->nn;
    double *xT = NEW(double, 3 * nn), *pred = NEW(double, 3 * nn), *nrm = NEW(double, 3 * nn);
    uint8_t *cT = NEW(uint8_t, nn);
    surface_normals(s, s->x, nrm);
    double maxPenRel = 0;
    for (int n = 0; n < nn; n++) {
        v3 p = sym(s, vadd(X(s, n), vscale(dt, xget(s->vg, n))), n);
        xset(pred, n, p);
        int c = s->contact[n];
        v3 tmp;
        if (c != FREE && !s->release[n]) {
            const o_hfdie *surf = surface(s, c);
            double off = offset_of(c, gapT);
            if (hf_clearance(surf, p, off) > 0.05 * tol_len(s, s->h_local[n])) cT[n] = FREE;
            else {
                p = sym(s, hf_project(surf, p, off, &tmp), n);
                cT[n] = (uint8_t)c;
            }
        } else if (s->is_surface[n]) {
            double cb = hf_clearance(&s->die[0], p, 0), ctp = hf_clearance(&s->die[1], p, gapT);
            if (cb < 0 || ctp < 0) {
                int hit = cb <= ctp ? BOTTOM : TOP;
                v3 q = sym(s, hf_project(surface(s, hit), p, offset_of(hit, gapT), &tmp), n);
                double pen = vlen(vsub(q, p));
                maxPenRel = dmax(maxPenRel, pen / tol_len(s, s->h_local[n]));
                p = q;
                cT[n] = (uint8_t)hit;
            }
        }
        xset(xT, n, p);
    }
    *ok = 0;
    if (maxPenRel > 0.5) {
        free(xT); free(pred); free(nrm); free(cT);
        return fail(s, E_OK, "die penetration exceeds half the local element size");
    }
    int reverted = improve_placement(s, xT, cT, pred, nrm, gapT, 0.05);
    if (reverted > 0) s->projection_reverts += reverted;
    smooth_interior(s, xT, 0.05, 6);
    for (int e = 0; e < s->ne; e++) {
        if (tet_quality_x(s, xT, e) <= 0.005) {
            /* the failure point for local refinement at the next remesh (_failAt, :1517) */
            for (int c = 0; c < 3; c++)
                s->fail_at[c] = 0.25 * (xT[3 * s->tets[4 * e] + c] + xT[3 * s->tets[4 * e + 1] + c] +
                                        xT[3 * s->tets[4 * e + 2] + c] + xT[3 * s->tets[4 * e + 3] + c]);
            s->have_fail_at = 1;
            char msg[120];
            snprintf(msg, sizeof msg, "tetrahedron %d collapsed", e);
            free(xT); free(pred); free(nrm); free(cT);
            return fail(s, E_OK, msg);
        }
    }
    memcpy(s->x, xT, sizeof(double) * 3 * nn);
    memcpy(s->contact, cT, nn);
    s->gap = gapT;
    s->time += dt;
    *ok = 1;
    free(xT); free(pred); free(nrm); free(cT);
    return E_OK;
}

static double min_quality(const o3d *s)
{
    double q = DBL_MAX;
    for (int e = 0; e < s->ne; e++) q = dmin(q, tet_quality_x(s, s->x, e));
    return q;
}

/* RemeshTrigger (:1867-1883): first-aid smoothing, then whether a remesh is due (counted as a request) */
static int remesh_trigger(o3d *s)
{
    if (min_quality(s) < s->p.remesh_quality) smooth_interior(s, s->x, s->p.remesh_quality, 6);
    if (min_quality(s) < s->p.remesh_quality) { s->remesh_requests++; return 1; }
    double maxEdge = 0;
    for (int k = 0; k < 3 * s->nbf; k += 3) {
        const int32_t *f = s->bface;
        maxEdge = dmax(maxEdge, dmax(vlen(vsub(X(s, f[k + 1]), X(s, f[k]))),
                                     dmax(vlen(vsub(X(s, f[k + 2]), X(s, f[k + 1]))), vlen(vsub(X(s, f[k]), X(s, f[k + 2]))))));
    }
    if (maxEdge > 2.8 * s->h) { s->remesh_requests++; return 1; }
    return 0;
}

/* Remesh (:1945-1956): the host's remesher replaces the mesh and state (o3d_replace_mesh) and returns 1, or
 * rejects the new mesh and returns 0; without a remesher the request stays only counted */
static int remesh(o3d *s)
{
    if (!s->remesh_cb) return 0;
    int ok = s->remesh_cb(s->remesh_user, s);
    if (ok) s->remesh_count++;
    return ok;
}

void o3d_set_remesher(o3d *s, o3d_remesh_fn fn, void *user)
{
    s->remesh_cb = fn;
    s->remesh_user = user;
}

/* the new mesh and the state remapped onto it (RemeshCore's Allocate and field hand-over, :2042-2057); the
 * increment state (gap, time, step, counters) stays, the next increment starts cold (_warm = false) */
int o3d_replace_mesh(o3d *s, int nn, int ne, const double *x, const int32_t *tets, const uint8_t *on_x0,
                     const uint8_t *on_y0, const uint8_t *contact, const double *vg, const double *eps,
                     const double *dmg, const double *sig, const double *rate, const double *mean)
{
    int rc = o3d_set_mesh(s, nn, ne, x, tets, on_x0, on_y0);
    if (rc != E_OK) return rc;
    memcpy(s->contact, contact, nn);
    memcpy(s->vg, vg, sizeof(double) * 3 * nn);
    memcpy(s->eps, eps, sizeof(double) * ne);
    memcpy(s->dmg, dmg, sizeof(double) * ne);
    memcpy(s->el_sig, sig, sizeof(double) * ne);
    memcpy(s->el_rate, rate, sizeof(double) * ne);
    memcpy(s->el_mean, mean, sizeof(double) * ne);
    s->have_vg_prev = 0;
    s->warm = 0;
    s->pcg_failures = 0;
    s->pcg_skip = 0;
    return E_OK;
}

/* LayerLimitedIncrement (:236-249) */
static double layer_limited_increment(const o3d *s, double step_cap)
{
    double thinnest = INFINITY;
    for (int n = 0; n < s->nn; n++) {
        if (s->contact[n] != TOP) continue;
        v3 p = X(s, n);
        double zb = hf_height(&s->die[0], p.x, p.y), zt = hf_height(&s->die[1], p.x, p.y) + s->gap;
        if (isfinite(zb) && isfinite(zt) && zt > zb) thinnest = dmin(thinnest, zt - zb);
    }
    return isfinite(thinnest) ? dmax(0.1 * thinnest, step_cap / (1 << s->p.max_cutbacks)) : INFINITY;
}

/* AccumulateDamage (:1844-1855) */
static void accumulate_damage(o3d *s, double dt)
{
    for (int e = 0; e < s->ne; e++) {
        double sig = s->el_sig[e];
        if (!(sig > 0) || s->el_rate[e] <= s->rate_cut) continue;
        int o = 6 * e;
        double m = s->el_mean[e];
        double s1 = o_principal_max3(s->el_dev[o] + m, s->el_dev[o + 1] + m, s->el_dev[o + 2] + m, s->el_dev[o + 3], s->el_dev[o + 4], s->el_dev[o + 5]);
        if (s1 > 0) s->dmg[e] += s1 / sig * s->el_rate[e] * dt;
    }
}

/* Step (:540-638) with remeshing unavailable */
int o3d_step(o3d *s)
{
    if (s->gap <= 1e-9) return fail(s, E_STATE, "Simulation already reached the closed-die position.");
    s->step_index++;
    if (remesh_trigger(s)) remesh(s);
    double step_cap = s->p.ds * s->h / s->p.h;
    int iterations = 0, ok = 0, used_cutback = 0, rc;
    double load = 0, reaction = 0, dt = 0;
    const int passes = 4;
    for (int pass = 0; pass < passes && !ok; pass++) {
        s->recovery_pass = pass;
        if ((rc = o3d_prepare_step(s)) != E_OK) return rc;
        int converged;
        iterations = o3d_solve_velocity(s, &converged);
        if (iterations < 0) return -iterations;
        if (!converged) {
            if (s->last_rel < 1e-2) {
                /* warning: not fully converged; continuing */
            } else {
                if (pass < passes - 1) {
                    s->remesh_requests++;
                    if (remesh(s)) continue; /* Remesh("stalled velocity solution") */
                }
                char msg[200];
                snprintf(msg, sizeof msg, "Velocity solution did not converge at step %d (stroke %.3f mm): |dv|/|v| = %.2e.",
                         s->step_index, s->gap0 - s->gap, s->last_rel);
                return fail(s, E_DIVERGED, msg);
            }
        }
        double power = o3d_final_evaluation(s, &reaction);
        s->power = power;
        load = power / s->p.ram * s->p.sym_factor;
        reaction *= s->p.sym_factor;
        double ds = dmin(s->p.auto_step ? dmin(s->ds_cur, step_cap) : step_cap, layer_limited_increment(s, step_cap));
        dt = dmin(ds, s->gap) / s->p.ram;
        if (s->gap - s->p.ram * dt < 0.05 * ds) dt = s->gap / s->p.ram;
        for (int attempt = 0; attempt <= s->p.max_cutbacks && !ok; attempt++) {
            double dta = dt / (1 << attempt);
            o3d_try_update(s, dta, &ok);
            if (ok) { dt = dta; used_cutback = attempt; }
        }
        if (ok || pass == passes - 1) break;
        if (pass >= 1 && s->refinement_levels > 0 && s->have_fail_at) {
            if (s->nhot == 64) {
                memmove(s->hot, s->hot + 4, sizeof(double) * 4 * 63);
                s->nhot--;
            }
            double *hs = s->hot + 4 * s->nhot++;
            hs[0] = s->fail_at[0]; hs[1] = s->fail_at[1]; hs[2] = s->fail_at[2];
            hs[3] = imin(pass, s->refinement_levels);
        }
        s->remesh_requests++;
        remesh(s); /* a rejected remesh does not end the ladder */
    }
    s->recovery_pass = 0;
    if (!ok) {
        char msg[200];
        snprintf(msg, sizeof msg, "Mesh distortion at step %d (stroke %.3f mm): %s.", s->step_index, s->gap0 - s->gap, s->err);
        return fail(s, E_DISTORTED, msg);
    }
    if (s->p.auto_step) {
        double used = s->p.ram * dt;
        s->ds_cur = used_cutback > 0 ? dmax(used, step_cap / (1 << s->p.max_cutbacks)) : dmin(step_cap, 1.5 * s->ds_cur);
    }
    for (int e = 0; e < s->ne; e++) s->eps[e] += s->el_rate[e] * dt;
    accumulate_damage(s, dt);
    s->warm = 1;
    s->iterations = iterations;
    s->load = load;
    s->reaction = reaction;
    s->err[0] = 0;
    return E_OK;
}

void o3d_set_warm(o3d *s, int warm) { s->warm = warm; }

void *o3d_array(o3d *s, const char *name, int64_t *count)
{
#define ARR(nm, ptr, cnt) if (!strcmp(name, nm)) { *count = (cnt); return (void *)(ptr); }
    ARR("x", s->x, 3 * (int64_t)s->nn)
    ARR("hot", s->hot, 4 * (int64_t)s->nhot)
    ARR("vg", s->vg, 3 * (int64_t)s->nn)
    ARR("eps", s->eps, s->ne)
    ARR("dmg", s->dmg, s->ne)
    ARR("el_sig", s->el_sig, s->ne)
    ARR("el_rate", s->el_rate, s->ne)
    ARR("el_mean", s->el_mean, s->ne)
    ARR("el_dev", s->el_dev, 6 * (int64_t)s->ne)
    ARR("contact", s->contact, s->nn)
    ARR("release", s->release, s->nn)
    ARR("fixed", s->fixed, s->ndof)
    ARR("fixed_val", s->fixed_val, s->ndof)
    ARR("ax", s->ax, 9 * (int64_t)s->nn)
    ARR("n_fix", s->n_fix, s->nn)
    ARR("die_axis", s->die_axis, s->nn)
    ARR("k_fric", s->k_fric, s->nn)
    ARR("a_fric", s->a_fric, s->nn)
    ARR("grad", s->grad, 12 * (int64_t)s->ne)
    ARR("vol", s->vol, s->ne)
    ARR("v", s->v, s->ndof)
    ARR("r", s->r, s->ndof)
    ARR("dv", s->dv, s->ndof)
    ARR("v_node", s->v_node, s->nn)
    ARR("g_start", s->g_start, s->nn + 1)
    ARR("g_node", s->g_node, s->g_len)
    ARR("g_coef", s->g_coef, 3 * s->g_len)
    ARR("kvol", s->kvol, s->nnz)
    ARR("val", s->val, s->nnz)
    ARR("col_ptr", s->col_ptr, s->ndof + 1)
    ARR("row_idx", s->row_idx, s->nnz)
    ARR("nbr_start", s->nbr_start, s->nn + 1)
    ARR("nbr", s->nbr, s->nbr_start ? s->nbr_start[s->nn] : 0)
    ARR("e_nbr", s->e_nbr, 16 * (int64_t)s->ne)
    ARR("h_local", s->h_local, s->nn)
    ARR("bface", s->bface, 3 * (int64_t)s->nbf)
    ARR("bowner", s->bowner, s->nbf)
    ARR("bsym", s->bsym, s->nbf)
    ARR("is_surface", s->is_surface, s->nn)
    ARR("e_r", s->e_r, 12 * (int64_t)s->ne)
    ARR("e_energy", s->e_energy, s->ne)
    ARR("e_power", s->e_power, s->ne)
    ARR("tets", s->tets, 4 * (int64_t)s->ne)
#undef ARR
    *count = 0;
    return NULL;
}

double o3d_scalar(o3d *s, const char *name)
{
#define SC(nm, v) if (!strcmp(name, nm)) return (double)(v);
    SC("gap", s->gap) SC("gap0", s->gap0) SC("time", s->time) SC("load", s->load) SC("reaction", s->reaction)
    SC("power", s->power) SC("iterations", s->iterations) SC("last_rel", s->last_rel) SC("vol0", s->vol0)
    SC("volume", volume(s)) SC("step_index", s->step_index) SC("n_pcg", s->n_pcg) SC("n_fact", s->n_fact)
    SC("n_newton", s->n_newton) SC("n_assemble", s->n_assemble) SC("remesh_requests", s->remesh_requests)
    SC("projection_reverts", s->projection_reverts) SC("corner_penetrations", s->corner_penetrations)
    SC("rate_ref", s->rate_ref) SC("rate_cut", s->rate_cut) SC("sig_ref", s->sig_ref) SC("k_pen", s->k_pen)
    SC("u0", s->u0) SC("nnz", s->nnz) SC("ds_cur", s->ds_cur) SC("warm", s->warm) SC("rnorm", s->rnorm_last)
    SC("beta", s->beta_last) SC("max_diag", s->max_diag_last) SC("have_factor", s->have_factor)
    SC("pcg_skip", s->pcg_skip) SC("pcg_failures", s->pcg_failures) SC("lin_its", s->lin_its_total)
    SC("nbf", s->nbf) SC("min_quality", min_quality(s)) SC("recovery_pass", s->recovery_pass)
    SC("factor_nnz", ospd_factor_nonzeros(s->lin))
    SC("remesh_count", s->remesh_count) SC("refinement_levels", s->refinement_levels) SC("max_nodes", s->max_nodes)
    SC("h", s->h) SC("nn", s->nn) SC("ne", s->ne)
#undef SC
    return NAN;
}

int o3d_set_scalar(o3d *s, const char *name, double v)
{
    if (!strcmp(name, "gap")) { s->gap = v; return 0; }
    if (!strcmp(name, "recovery_pass")) { s->recovery_pass = (int)v; return 0; }
    if (!strcmp(name, "ds_cur")) { s->ds_cur = v; return 0; }
    if (!strcmp(name, "warm")) { s->warm = (int)v; return 0; }
    if (!strcmp(name, "refinement_levels")) { s->refinement_levels = (int)v; return 0; }
    if (!strcmp(name, "max_nodes")) { s->max_nodes = (int)v; return 0; }
    return -1;
}
