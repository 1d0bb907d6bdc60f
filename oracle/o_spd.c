/*
 * o_spd.c — the oracle's sparse SPD factorisation (its ISpdSolver backend). TEST INFRASTRUCTURE ONLY
 * (see ifea_oracle.h): the checker the GPU factorisation is compared against and the CPU baseline's solver.
 *
 * The reference's CPU backends are Intel MKL PARDISO 2026.1.0.226 (a threaded supernodal solver,
 * Solver/Linear/MklPardisoSolver.cs:41-43, :88-99) and CSparse.NET 4.4.1 (an up-looking Cholesky,
 * Solver/Linear/ManagedSpdSolver.cs:28-34). Neither is available here. This restates the published supernodal
 * multifrontal Cholesky (Duff and Reid 1983; Liu, "The multifrontal method for sparse matrix solution: theory
 * and practice", SIAM Review 1992):
 *   - a nested-dissection order: recursive coordinate bisection of the node graph when node coordinates are
 *     given (ospd_set_geometry), else recursive BFS level-set bisection of the matrix graph;
 *   - the elimination tree and the column counts by row subtrees (Davis 2006, cs_etree / cs_ereach);
 *   - fundamental supernodes, merged into their parents while the merged front stays mostly nonzero
 *     (relaxed amalgamation);
 *   - per supernode, in an order where children come first: the dense frontal matrix (A's entries of its
 *     columns, then its children's update matrices added in child order), a tiled right-looking dense
 *     Cholesky of its pivot columns, and the Schur complement handed to the parent as its update matrix.
 * Independent supernodes of one tree level run on OpenMP threads; the few large fronts near the root run their
 * tile operations on all threads. Every entry's operations happen in a fixed order whatever the thread count,
 * so the factor is reproducible. Any symmetric order gives the same factor up to rounding, which is all the
 * PCG / refactorisation logic above it depends on.
 *
 * This file is compiled with FMA contraction allowed (-ffp-contract=fast): the factorisation has no
 * counterpart whose rounding the reference fixes.
 */
#include <float.h>
#include <math.h>
#include <omp.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "ifea_oracle.h"

struct ospd {
    int n;
    int *perm, *pinv;          /* new k = pinv[old] */
    int32_t *ucp, *uci;        /* upper triangle of P A P' (CSC): etree and column counts */
    int64_t *lcp;              /* lower triangle of P A P' (CSC) ... */
    int32_t *lci;
    int64_t *lmap;             /* ... entry -> index into the full value array */
    int *parent;               /* elimination tree */
    int ns;                    /* supernodes */
    int *sn_first;             /* columns [sn_first[s], sn_first[s + 1]) */
    int *sn_parent;
    int64_t *sn_rptr;          /* rows of front s: sn_rows[sn_rptr[s] .. sn_rptr[s + 1]), ascending */
    int *sn_rows;
    int *ch_ptr, *ch_list;     /* children of each supernode, ascending */
    int nlvl;
    int *lvl_ptr, *lvl_sn;     /* supernodes by height above the leaves */
    int64_t *sn_lptr;          /* factor block of s: m x k column-major at lx + sn_lptr[s] */
    double *lx;
    int64_t lnz;               /* factor entries (lower trapezoids of the blocks, explicit zeros included) */
    double flops;
    double *work;
    int factored;
    int bad_pivot;
    int geo_nodes;             /* node coordinates for the ordering (optional) */
    double *geo_xyz;
};

/* ------------------------------------------------------------------ ordering: recursive BFS level-set bisection */

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

/* ------------------------------------------------------------------ ordering: coordinate nested dissection
 *
 * When the caller gives node coordinates (3 equations per node, DOF = 3 node + c), the order is a recursive
 * coordinate bisection of the node graph (George 1973, nested dissection of grids; its geometric form as in
 * Miller, Teng, Thurston and Vavasis 1998): the nodes are split at the median along the longest extent of their
 * bounding box; the separator, numbered after both halves, is a minimum vertex cover of the edges between the
 * halves (for more than 256 nodes) or the smaller of the two one-sided boundary sets; a node's three equations
 * stay consecutive. */

typedef struct {
    const double *xyz;
    int axis;
} o_axis_key;
static __thread o_axis_key g_key;

static int cmp_axis(const void *a, const void *b)
{
    int u = *(const int *)a, v = *(const int *)b;
    double xu = g_key.xyz[3 * u + g_key.axis], xv = g_key.xyz[3 * v + g_key.axis];
    if (xu < xv) return -1;
    if (xu > xv) return 1;
    return (u > v) - (u < v);
}

/* Minimum vertex cover of the bipartite cut graph between the boundary sets of two halves (König's theorem
 * on a maximum matching from Hopcroft and Karp 1973). ua[] / ub[] are the boundary nodes of either half;
 * adjacency from ua to ub in (ap, aj) over local indices. On return in_cover_a[i] / in_cover_b[j] mark the cover. */
static void min_vertex_cover(int na, int nb, const int *ap, const int *aj, char *in_cover_a, char *in_cover_b)
{
    int *mate_a = (int *)malloc(sizeof(int) * (na > 0 ? na : 1)), *mate_b = (int *)malloc(sizeof(int) * (nb > 0 ? nb : 1));
    int *dist = (int *)malloc(sizeof(int) * (na > 0 ? na : 1)), *queue = (int *)malloc(sizeof(int) * (na > 0 ? na : 1));
    int *stk = (int *)malloc(sizeof(int) * (na > 0 ? na : 1)), *it = (int *)malloc(sizeof(int) * (na > 0 ? na : 1));
    for (int i = 0; i < na; i++) mate_a[i] = -1;
    for (int j = 0; j < nb; j++) mate_b[j] = -1;
    for (;;) {
        /* BFS layers from the free vertices of side a */
        int head = 0, tail = 0, found = 0;
        for (int i = 0; i < na; i++) {
            if (mate_a[i] < 0) { dist[i] = 0; queue[tail++] = i; }
            else dist[i] = -1;
        }
        while (head < tail) {
            int i = queue[head++];
            for (int p = ap[i]; p < ap[i + 1]; p++) {
                int j = aj[p], i2 = mate_b[j];
                if (i2 < 0) found = 1;
                else if (dist[i2] < 0) { dist[i2] = dist[i] + 1; queue[tail++] = i2; }
            }
        }
        if (!found) break;
        /* DFS along the layers (iterative), one augmenting path per free vertex */
        int augmented = 0;
        for (int r = 0; r < na; r++) {
            if (mate_a[r] >= 0 || dist[r] != 0) continue;
            int top = 0;
            stk[top++] = r;
            it[r] = ap[r];
            int end_j = -1;
            while (top > 0 && end_j < 0) {
                int i = stk[top - 1];
                if (it[i] >= ap[i + 1]) { dist[i] = -1; top--; continue; }
                int j = aj[it[i]++], i2 = mate_b[j];
                if (i2 < 0) { end_j = j; break; }
                if (dist[i2] == dist[i] + 1) { it[i2] = ap[i2]; stk[top++] = i2; }
            }
            if (end_j < 0) continue;
            /* flip the path: stk[0..top-1] are side-a vertices, each matched to the b vertex it stepped through */
            int j = end_j;
            for (int q = top - 1; q >= 0; q--) {
                int i = stk[q];
                int prev = mate_a[i];
                mate_a[i] = j;
                mate_b[j] = i;
                j = prev;
            }
            augmented++;
        }
        if (!augmented) break;
    }
    /* König: Z = vertices reachable from free side-a vertices by alternating paths */
    char *za = (char *)calloc((size_t)(na > 0 ? na : 1), 1), *zb = (char *)calloc((size_t)(nb > 0 ? nb : 1), 1);
    int head = 0, tail = 0;
    for (int i = 0; i < na; i++)
        if (mate_a[i] < 0) { za[i] = 1; queue[tail++] = i; }
    while (head < tail) {
        int i = queue[head++];
        for (int p = ap[i]; p < ap[i + 1]; p++) {
            int j = aj[p];
            if (zb[j]) continue;
            zb[j] = 1;
            int i2 = mate_b[j];
            if (i2 >= 0 && !za[i2]) { za[i2] = 1; queue[tail++] = i2; }
        }
    }
    for (int i = 0; i < na; i++) in_cover_a[i] = !za[i];
    for (int j = 0; j < nb; j++) in_cover_b[j] = zb[j];
    free(za); free(zb); free(mate_a); free(mate_b); free(dist); free(queue); free(stk); free(it);
}

static void coord_nd(const int *np, const int *nj, const double *xyz, int *side, int *loc, int *nodes, int cnt,
                     int *out, int *nout)
{
    if (cnt <= 64) {
        for (int k = 0; k < cnt; k++) out[(*nout)++] = nodes[k];
        return;
    }
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int k = 0; k < cnt; k++)
        for (int c = 0; c < 3; c++) {
            double v = xyz[3 * nodes[k] + c];
            if (v < lo[c]) lo[c] = v;
            if (v > hi[c]) hi[c] = v;
        }
    int axis = 0;
    for (int c = 1; c < 3; c++)
        if (hi[c] - lo[c] > hi[axis] - lo[axis]) axis = c;
    g_key.xyz = xyz;
    g_key.axis = axis;
    qsort(nodes, (size_t)cnt, sizeof(int), cmp_axis);
    int half = cnt / 2;
    /* side: 1 = first half, 2 = second half, 0 = outside this range */
    for (int k = 0; k < cnt; k++) side[nodes[k]] = k < half ? 1 : 2;
    int na_b = 0, nb_b = 0;  /* boundary sizes of either half */
    for (int k = 0; k < cnt; k++) {
        int u = nodes[k], su = side[u], touch = 0;
        for (int p = np[u]; p < np[u + 1] && !touch; p++) {
            int w = nj[p];
            if (side[w] != 0 && side[w] != su) touch = 1;
        }
        if (touch) {
            if (su == 1) na_b++;
            else nb_b++;
        }
    }
    int *a = (int *)malloc(sizeof(int) * cnt), *b = (int *)malloc(sizeof(int) * cnt), *s = (int *)malloc(sizeof(int) * cnt);
    int na = 0, nb = 0, ns = 0;
    if (cnt > 256) {
        /* separator = a minimum vertex cover of the cut edges */
        int *ua = (int *)malloc(sizeof(int) * (na_b > 0 ? na_b : 1)), *ub = (int *)malloc(sizeof(int) * (nb_b > 0 ? nb_b : 1));
        int ka = 0, kb = 0;
        for (int k = 0; k < cnt; k++) {
            int u = nodes[k], su = side[u], touch = 0;
            for (int p = np[u]; p < np[u + 1] && !touch; p++) {
                int w = nj[p];
                if (side[w] != 0 && side[w] != su) touch = 1;
            }
            if (!touch) continue;
            if (su == 1) { loc[u] = ka; ua[ka++] = u; }
            else { loc[u] = kb; ub[kb++] = u; }
        }
        int *ap = (int *)malloc(sizeof(int) * (ka + 1));
        ap[0] = 0;
        for (int i = 0; i < ka; i++) {
            int c = 0;
            for (int p = np[ua[i]]; p < np[ua[i] + 1]; p++) c += side[nj[p]] == 2;
            ap[i + 1] = ap[i] + c;
        }
        int *aj = (int *)malloc(sizeof(int) * (ap[ka] > 0 ? ap[ka] : 1));
        for (int i = 0, q = 0; i < ka; i++)
            for (int p = np[ua[i]]; p < np[ua[i] + 1]; p++)
                if (side[nj[p]] == 2) aj[q++] = loc[nj[p]];
        char *ca = (char *)malloc((size_t)(ka > 0 ? ka : 1)), *cb = (char *)malloc((size_t)(kb > 0 ? kb : 1));
        min_vertex_cover(ka, kb, ap, aj, ca, cb);
        for (int i = 0; i < ka; i++) if (ca[i]) side[ua[i]] = 3;
        for (int j = 0; j < kb; j++) if (cb[j]) side[ub[j]] = 3;
        free(ua); free(ub); free(ap); free(aj); free(ca); free(cb);
        for (int k = 0; k < cnt; k++) {
            int u = nodes[k];
            if (side[u] == 3) s[ns++] = u;
            else if (side[u] == 1) a[na++] = u;
            else b[nb++] = u;
        }
    } else {
        /* separator = the smaller one-sided boundary */
        int sep_side = na_b <= nb_b ? 1 : 2;
        for (int k = 0; k < cnt; k++) {
            int u = nodes[k], su = side[u], touch = 0;
            if (su == sep_side)
                for (int p = np[u]; p < np[u + 1] && !touch; p++) {
                    int w = nj[p];
                    if (side[w] != 0 && side[w] != su) touch = 1;
                }
            if (touch) s[ns++] = u;
            else if (su == 1) a[na++] = u;
            else b[nb++] = u;
        }
    }
    for (int k = 0; k < cnt; k++) side[nodes[k]] = 0;
    coord_nd(np, nj, xyz, side, loc, a, na, out, nout);
    coord_nd(np, nj, xyz, side, loc, b, nb, out, nout);
    for (int k = 0; k < ns; k++) out[(*nout)++] = s[k];
    free(a);
    free(b);
    free(s);
}

/* Node order of a 3-DOF-per-node pattern by coord_nd, expanded to equations; returns 0 if the pattern is not
 * in 3 x 3 node blocks (the caller falls back to the graph bisection). */
static int coord_order(int n, const int32_t *col_ptr, const int32_t *row_idx, int nnodes, const double *xyz, int *perm)
{
    if (n != 3 * nnodes) return 0;
    int *np = (int *)malloc(sizeof(int) * (nnodes + 1));
    np[0] = 0;
    for (int u = 0; u < nnodes; u++) {
        int cntu = 0;
        for (int32_t p = col_ptr[3 * u]; p < col_ptr[3 * u + 1]; p++)
            if (row_idx[p] % 3 == 0 && row_idx[p] / 3 != u) cntu++;
        np[u + 1] = np[u] + cntu;
    }
    int *nj = (int *)malloc(sizeof(int) * (np[nnodes] > 0 ? np[nnodes] : 1));
    for (int u = 0; u < nnodes; u++) {
        int q = np[u];
        for (int32_t p = col_ptr[3 * u]; p < col_ptr[3 * u + 1]; p++)
            if (row_idx[p] % 3 == 0 && row_idx[p] / 3 != u) nj[q++] = row_idx[p] / 3;
    }
    int *side = (int *)calloc((size_t)nnodes, sizeof(int)), *nodes = (int *)malloc(sizeof(int) * nnodes);
    int *out = (int *)malloc(sizeof(int) * nnodes), *loc = (int *)malloc(sizeof(int) * nnodes);
    for (int u = 0; u < nnodes; u++) nodes[u] = u;
    int nout = 0;
    coord_nd(np, nj, xyz, side, loc, nodes, nnodes, out, &nout);
    free(loc);
    for (int k = 0; k < nnodes; k++)
        for (int c = 0; c < 3; c++) perm[3 * k + c] = 3 * out[k] + c;
    free(np); free(nj); free(side); free(nodes); free(out);
    return 1;
}

/* ------------------------------------------------------------------ dense kernels (column-major) */

enum { MR = 8, NR = 6, TILE = 256 };
typedef double v8d __attribute__((vector_size(64)));

/* C[0:mr, 0:nr] (ld ldc) -= Ap * Bp^T over kc steps; Ap packed [p][MR], Bp packed [p][NR]. Compiled once per
 * instruction set and chosen at run time by the CPU's features. */
#define MICRO_KERNEL_BODY                                                                                       \
    v8d acc[NR];                                                                                                \
    for (int c = 0; c < NR; c++) acc[c] = (v8d){0, 0, 0, 0, 0, 0, 0, 0};                                        \
    for (int p = 0; p < kc; p++) {                                                                              \
        v8d a;                                                                                                  \
        memcpy(&a, Ap + (int64_t)p * MR, sizeof a);                                                             \
        const double *b = Bp + (int64_t)p * NR;                                                                 \
        for (int c = 0; c < NR; c++) acc[c] += a * b[c];                                                        \
    }                                                                                                           \
    for (int c = 0; c < nr; c++) {                                                                              \
        double *cc = C + (int64_t)c * ldc;                                                                      \
        for (int r = 0; r < mr; r++) cc[r] -= acc[c][r];                                                        \
    }
typedef void (*micro_fn)(int, const double *, const double *, double *, int64_t, int, int);
__attribute__((target("avx512f"))) static void micro_avx512(int kc, const double *restrict Ap,
                                                            const double *restrict Bp, double *restrict C,
                                                            int64_t ldc, int mr, int nr) { MICRO_KERNEL_BODY }
__attribute__((target("avx2,fma"))) static void micro_avx2(int kc, const double *restrict Ap,
                                                           const double *restrict Bp, double *restrict C, int64_t ldc,
                                                           int mr, int nr) { MICRO_KERNEL_BODY }
static void micro_generic(int kc, const double *restrict Ap, const double *restrict Bp, double *restrict C,
                          int64_t ldc, int mr, int nr) { MICRO_KERNEL_BODY }
static micro_fn micro_kernel = NULL;

static void select_micro_kernel(void)
{
    if (micro_kernel) return;
    __builtin_cpu_init();
    if (__builtin_cpu_supports("avx512f")) micro_kernel = micro_avx512;
    else if (__builtin_cpu_supports("avx2") && __builtin_cpu_supports("fma")) micro_kernel = micro_avx2;
    else micro_kernel = micro_generic;
}

/* Pack an mb x kb block (ld) as MR-row panels [panel][p][MR] / NR-row panels [panel][p][NR], zero padded. */
static void pack_a(int mb, int kb, const double *src, int64_t ld, double *dst)
{
    int np = (mb + MR - 1) / MR;
    for (int ip = 0; ip < np; ip++) {
        int rows = mb - ip * MR < MR ? mb - ip * MR : MR;
        double *d = dst + (size_t)ip * MR * kb;
        for (int p = 0; p < kb; p++) {
            const double *s = src + ip * MR + (int64_t)p * ld;
            for (int r = 0; r < rows; r++) d[p * MR + r] = s[r];
            for (int r = rows; r < MR; r++) d[p * MR + r] = 0.0;
        }
    }
}

static void pack_b(int nb, int kb, const double *src, int64_t ld, double *dst)
{
    int np = (nb + NR - 1) / NR;
    for (int jp = 0; jp < np; jp++) {
        int cols = nb - jp * NR < NR ? nb - jp * NR : NR;
        double *d = dst + (size_t)jp * NR * kb;
        for (int p = 0; p < kb; p++) {
            const double *s = src + jp * NR + (int64_t)p * ld;
            for (int c = 0; c < cols; c++) d[p * NR + c] = s[c];
            for (int c = cols; c < NR; c++) d[p * NR + c] = 0.0;
        }
    }
}

static size_t packed_a_size(int mb, int kb) { return (size_t)((mb + MR - 1) / MR) * MR * kb; }
static size_t packed_b_size(int nb, int kb) { return (size_t)((nb + NR - 1) / NR) * NR * kb; }

/* C (mb x nb, ld ldc) -= A B^T from packed panels over kb; lower != 0 skips micro-tiles above the diagonal. */
static void gemm_packed(int mb, int nb, int kb, const double *Ap, const double *Bp, double *C, int64_t ldc, int lower)
{
    int mp = (mb + MR - 1) / MR, np = (nb + NR - 1) / NR;
    for (int jp = 0; jp < np; jp++) {
        int j0 = jp * NR, nr = nb - j0 < NR ? nb - j0 : NR;
        for (int ip = 0; ip < mp; ip++) {
            int i0 = ip * MR, mr = mb - i0 < MR ? mb - i0 : MR;
            if (lower && i0 + mr - 1 < j0) continue;
            micro_kernel(kb, Ap + (size_t)ip * MR * kb, Bp + (size_t)jp * NR * kb, C + i0 + (int64_t)j0 * ldc, ldc, mr, nr);
        }
    }
}

/* Unblocked Cholesky of the nb x nb diagonal tile A (ld lda), lower; returns the failing column or -1. */
static int potrf_tile(int nb, double *A, int64_t lda)
{
    for (int c = 0; c < nb; c++) {
        double *ac = A + (int64_t)c * lda;
        double d = ac[c];
        if (!(d > 0) || isnan(d)) return c;
        d = sqrt(d);
        ac[c] = d;
        double inv = 1.0 / d;
        for (int r = c + 1; r < nb; r++) ac[r] *= inv;
        for (int c2 = c + 1; c2 < nb; c2++) {
            double l = ac[c2];
            double *a2 = A + (int64_t)c2 * lda;
            for (int r = c2; r < nb; r++) a2[r] -= ac[r] * l;
        }
    }
    return -1;
}

/* X (nb x nb, ld nb) = -L^-1 for the factored lower tile L (ld ldl): forward substitution on the identity. */
static void neg_tri_inverse(int nb, const double *L, int64_t ldl, double *X)
{
    memset(X, 0, sizeof(double) * (size_t)nb * nb);
    for (int j = 0; j < nb; j++) {
        double *x = X + (int64_t)j * nb;  /* column j of L^-1 */
        x[j] = 1.0 / L[j + (int64_t)j * ldl];
        for (int c = j; c < nb; c++) {
            double xc = x[c];
            if (c > j) {
                xc /= L[c + (int64_t)c * ldl];
                x[c] = xc;
            }
            const double *lc = L + (int64_t)c * ldl;
            for (int r = c + 1; r < nb; r++) x[r] -= lc[r] * xc;
        }
    }
    for (size_t t = 0; t < (size_t)nb * nb; t++) X[t] = -X[t];
}

/* Partial Cholesky of the m x m front F (ld m, lower): the first k columns are eliminated, the trailing
 * (m - k) x (m - k) block becomes the Schur complement. Tiled right-looking; tile boundaries at multiples of
 * TILE inside [0, k) and inside [k, m). Per pivot tile: Cholesky of the diagonal tile, the tiles below times
 * L^-T (through the tile's inverse), each packed once, then every trailing tile (i, j) minus L_i L_j^T.
 * Returns the failing column or -1. */
static int front_factor(int m, int k, double *F, int par)
{
    int nt0 = (k + TILE - 1) / TILE, nt1 = (m - k + TILE - 1) / TILE, nt = nt0 + nt1;
    int *tb = (int *)malloc(sizeof(int) * (nt + 1));
    for (int t = 0; t < nt0; t++) tb[t] = t * TILE;
    for (int t = 0; t < nt1; t++) tb[nt0 + t] = k + t * TILE;
    tb[nt] = m;
    double **pa = (double **)calloc((size_t)nt, sizeof(double *)), **pb = (double **)calloc((size_t)nt, sizeof(double *));
    double *inv = (double *)malloc(sizeof(double) * TILE * TILE);
    double *pinv = (double *)malloc(sizeof(double) * packed_b_size(TILE, TILE));
    int bad = -1;
    int64_t ld = m;
    for (int kk = 0; kk < nt0 && bad < 0; kk++) {
        int c0 = tb[kk], nb = tb[kk + 1] - c0;
        double *Dkk = F + c0 + (int64_t)c0 * ld;
        int f = potrf_tile(nb, Dkk, ld);
        if (f >= 0) {
            bad = c0 + f;
            break;
        }
        int nrow = nt - kk - 1;
        if (nrow == 0) break;
        neg_tri_inverse(nb, Dkk, ld, inv);
        pack_b(nb, nb, inv, nb, pinv);  /* B(c, p) = -Linv(c, p): tile Linv^T = tile0 - tile0 (-Linv)^T */
#pragma omp parallel for schedule(dynamic, 1) if (par && nrow > 1)
        for (int i = kk + 1; i < nt; i++) {
            int r0 = tb[i], mb = tb[i + 1] - r0;
            double *T = F + r0 + (int64_t)c0 * ld;
            double *tmp = (double *)malloc(sizeof(double) * packed_a_size(mb, nb));
            pack_a(mb, nb, T, ld, tmp);
            for (int c = 0; c < nb; c++) memset(T + (int64_t)c * ld, 0, sizeof(double) * mb);
            gemm_packed(mb, nb, nb, tmp, pinv, T, ld, 0);
            free(tmp);
            pa[i] = (double *)malloc(sizeof(double) * packed_a_size(mb, nb));
            pb[i] = (double *)malloc(sizeof(double) * packed_b_size(mb, nb));
            pack_a(mb, nb, T, ld, pa[i]);
            pack_b(mb, nb, T, ld, pb[i]);
        }
        /* trailing update of tiles (i, j), kk < j <= i */
        int npairs = nrow * (nrow + 1) / 2;
#pragma omp parallel for schedule(dynamic, 1) if (par && npairs > 1)
        for (int q = 0; q < npairs; q++) {
            int di = (int)((sqrt(8.0 * q + 1.0) - 1.0) * 0.5);
            while ((di + 1) * (di + 2) / 2 <= q) di++;
            while (di * (di + 1) / 2 > q) di--;
            int dj = q - di * (di + 1) / 2;
            int i = kk + 1 + di, j = kk + 1 + dj;
            int r0 = tb[i], mb = tb[i + 1] - r0, j0 = tb[j], nbj = tb[j + 1] - j0;
            gemm_packed(mb, nbj, nb, pa[i], pb[j], F + r0 + (int64_t)j0 * ld, ld, i == j);
        }
        for (int i = kk + 1; i < nt; i++) {
            free(pa[i]);
            free(pb[i]);
            pa[i] = pb[i] = NULL;
        }
    }
    free(pa);
    free(pb);
    free(inv);
    free(pinv);
    free(tb);
    return bad;
}

/* ------------------------------------------------------------------ analysis */

ospd *ospd_create(void) { return (ospd *)calloc(1, sizeof(ospd)); }

static void ospd_release(ospd *f)
{
    free(f->perm); free(f->pinv); free(f->ucp); free(f->uci); free(f->lcp); free(f->lci); free(f->lmap);
    free(f->parent); free(f->sn_first); free(f->sn_parent); free(f->sn_rptr); free(f->sn_rows); free(f->ch_ptr);
    free(f->ch_list); free(f->lvl_ptr); free(f->lvl_sn); free(f->sn_lptr); free(f->lx); free(f->work);
    int gn = f->geo_nodes;
    double *gx = f->geo_xyz;
    memset(f, 0, sizeof(*f));
    f->geo_nodes = gn;
    f->geo_xyz = gx;
}

void ospd_set_geometry(ospd *f, int nnodes, const double *xyz)
{
    free(f->geo_xyz);
    f->geo_xyz = NULL;
    f->geo_nodes = 0;
    if (nnodes <= 0 || !xyz) return;
    f->geo_xyz = (double *)malloc(sizeof(double) * 3 * (size_t)nnodes);
    memcpy(f->geo_xyz, xyz, sizeof(double) * 3 * (size_t)nnodes);
    f->geo_nodes = nnodes;
}

void ospd_destroy(ospd *f)
{
    if (!f) return;
    ospd_release(f);
    free(f->geo_xyz);
    free(f);
}

/* cs_ereach: pattern of row k of L (nonzeros of L(k, 0:k-1)) in s[top..n-1] */
static int ereach(const ospd *f, int k, int *s, int *w)
{
    int n = f->n, top = n;
    w[k] = k + 1;
    for (int32_t p = f->ucp[k]; p < f->ucp[k + 1]; p++) {
        int i = f->uci[p];
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

static int cmp_int(const void *a, const void *b)
{
    int x = *(const int *)a, y = *(const int *)b;
    return (x > y) - (x < y);
}

int ospd_analyze(ospd *f, int n, const int32_t *col_ptr, const int32_t *row_idx)
{
    select_micro_kernel();
    ospd_release(f);
    f->n = n;
    /* ordering */
    o_graph g = {n, col_ptr, row_idx};
    int *part = (int *)calloc((size_t)n, sizeof(int)), *level = (int *)malloc(sizeof(int) * n);
    int *order = (int *)malloc(sizeof(int) * n), *nodes = (int *)malloc(sizeof(int) * n);
    f->perm = (int *)malloc(sizeof(int) * n);
    f->pinv = (int *)malloc(sizeof(int) * n);
    for (int k = 0; k < n; k++) nodes[k] = k;
    int nperm = 0, next_tag = 1;
    if (!(f->geo_nodes > 0 && coord_order(n, col_ptr, row_idx, f->geo_nodes, f->geo_xyz, f->perm)))
        nd_order(&g, part, level, order, f->perm, &nperm, nodes, n, 0, &next_tag);
    free(part); free(level); free(order); free(nodes);
    for (int k = 0; k < n; k++) f->pinv[f->perm[k]] = k;
    /* upper and lower triangles of C = P A P' */
    f->ucp = (int32_t *)calloc((size_t)n + 1, sizeof(int32_t));
    f->lcp = (int64_t *)calloc((size_t)n + 1, sizeof(int64_t));
    for (int j = 0; j < n; j++)
        for (int32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
            int i2 = f->pinv[row_idx[p]], j2 = f->pinv[j];
            if (i2 <= j2) f->ucp[j2 + 1]++;
            if (i2 >= j2) f->lcp[j2 + 1]++;
        }
    for (int j = 0; j < n; j++) {
        f->ucp[j + 1] += f->ucp[j];
        f->lcp[j + 1] += f->lcp[j];
    }
    f->uci = (int32_t *)malloc(sizeof(int32_t) * (f->ucp[n] > 0 ? f->ucp[n] : 1));
    f->lci = (int32_t *)malloc(sizeof(int32_t) * (f->lcp[n] > 0 ? f->lcp[n] : 1));
    f->lmap = (int64_t *)malloc(sizeof(int64_t) * (f->lcp[n] > 0 ? f->lcp[n] : 1));
    {
        int32_t *uf = (int32_t *)malloc(sizeof(int32_t) * (n + 1));
        int64_t *lf = (int64_t *)malloc(sizeof(int64_t) * (n + 1));
        memcpy(uf, f->ucp, sizeof(int32_t) * (n + 1));
        memcpy(lf, f->lcp, sizeof(int64_t) * (n + 1));
        for (int j = 0; j < n; j++)
            for (int32_t p = col_ptr[j]; p < col_ptr[j + 1]; p++) {
                int i2 = f->pinv[row_idx[p]], j2 = f->pinv[j];
                if (i2 <= j2) f->uci[uf[j2]++] = i2;
                if (i2 >= j2) {
                    f->lci[lf[j2]] = i2;
                    f->lmap[lf[j2]++] = p;
                }
            }
        free(uf);
        free(lf);
    }
    /* elimination tree (cs_etree) */
    f->parent = (int *)malloc(sizeof(int) * n);
    {
        int *anc = (int *)malloc(sizeof(int) * n);
        for (int k = 0; k < n; k++) {
            f->parent[k] = -1;
            anc[k] = -1;
            for (int32_t p = f->ucp[k]; p < f->ucp[k + 1]; p++) {
                int i = f->uci[p];
                while (i != -1 && i < k) {
                    int inext = anc[i];
                    anc[i] = k;
                    if (inext == -1) f->parent[i] = k;
                    i = inext;
                }
            }
        }
        free(anc);
    }
    /* column counts of L by the row subtrees */
    int64_t *cnt = (int64_t *)calloc((size_t)n, sizeof(int64_t));
    {
        int *stk = (int *)malloc(sizeof(int) * n), *mark = (int *)calloc((size_t)n, sizeof(int));
        for (int k = 0; k < n; k++) {
            int top = ereach(f, k, stk, mark);
            for (int t = top; t < n; t++) cnt[stk[t]]++;
            cnt[k]++;
        }
        free(stk);
        free(mark);
    }
    /* fundamental supernodes */
    int *nchild = (int *)calloc((size_t)n, sizeof(int));
    for (int j = 0; j < n; j++)
        if (f->parent[j] >= 0) nchild[f->parent[j]]++;
    int *first = (int *)malloc(sizeof(int) * (n + 1));
    int ns = 0;
    for (int j = 0; j < n; j++) {
        int cont = j > 0 && f->parent[j - 1] == j && cnt[j - 1] == cnt[j] + 1 && nchild[j] == 1;
        if (!cont) first[ns++] = j;
    }
    first[ns] = n;
    free(nchild);
    /* relaxed amalgamation: merge supernode s into its parent p when p starts right after s, the merged front
     * (s's columns on top of p's front) keeps at most 10 % explicit zeros, or the merged supernode stays narrow */
    {
        int *sn_of = (int *)malloc(sizeof(int) * n);
        for (int s = 0; s < ns; s++)
            for (int j = first[s]; j < first[s + 1]; j++) sn_of[j] = s;
        int *alive_first = (int *)malloc(sizeof(int) * ns), *alive_end = (int *)malloc(sizeof(int) * ns);
        int64_t *front_m = (int64_t *)malloc(sizeof(int64_t) * ns);
        double *zeros = (double *)calloc((size_t)ns, sizeof(double)), *dense = (double *)malloc(sizeof(double) * ns);
        int *rep = (int *)malloc(sizeof(int) * ns);
        for (int s = 0; s < ns; s++) {
            alive_first[s] = first[s];
            alive_end[s] = first[s + 1];
            front_m[s] = cnt[first[s]];
            int64_t k = first[s + 1] - first[s];
            dense[s] = (double)(k * front_m[s] - k * (k - 1) / 2);
            rep[s] = s;
        }
        for (int s = 0; s < ns; s++) {
            int last = alive_end[s] - 1;
            int pc = f->parent[last];
            if (pc < 0) continue;
            int p = sn_of[pc];
            while (rep[p] != p) p = rep[p];
            if (alive_first[p] != alive_end[s]) continue;  /* not contiguous */
            int64_t ks = alive_end[s] - alive_first[s], kp = alive_end[p] - alive_first[p];
            int64_t mnew = ks + front_m[p], knew = ks + kp;
            double dnew = (double)(knew * mnew - knew * (knew - 1) / 2);
            double truth = 0;
            for (int j = alive_first[s]; j < alive_end[s]; j++) truth += (double)cnt[j];
            truth += dense[p] - zeros[p];
            double znew = dnew - truth;
            if (knew <= 16 || znew <= 0.1 * dnew) {
                rep[s] = p;
                alive_first[p] = alive_first[s];
                front_m[p] = mnew;
                dense[p] = dnew;
                zeros[p] = znew;
            }
        }
        int ns2 = 0;
        for (int s = 0; s < ns; s++)
            if (rep[s] == s) first[ns2++] = alive_first[s];
        first[ns2] = n;
        ns = ns2;
        free(sn_of); free(alive_first); free(alive_end); free(front_m); free(zeros); free(dense); free(rep);
    }
    free(cnt);
    f->ns = ns;
    f->sn_first = (int *)realloc(first, sizeof(int) * (ns + 1));
    /* supernodal tree */
    int *sn_of = (int *)malloc(sizeof(int) * n);
    for (int s = 0; s < ns; s++)
        for (int j = f->sn_first[s]; j < f->sn_first[s + 1]; j++) sn_of[j] = s;
    f->sn_parent = (int *)malloc(sizeof(int) * ns);
    for (int s = 0; s < ns; s++) {
        int pc = f->parent[f->sn_first[s + 1] - 1];
        f->sn_parent[s] = pc >= 0 ? sn_of[pc] : -1;
    }
    f->ch_ptr = (int *)calloc((size_t)ns + 1, sizeof(int));
    for (int s = 0; s < ns; s++)
        if (f->sn_parent[s] >= 0) f->ch_ptr[f->sn_parent[s] + 1]++;
    for (int s = 0; s < ns; s++) f->ch_ptr[s + 1] += f->ch_ptr[s];
    f->ch_list = (int *)malloc(sizeof(int) * (f->ch_ptr[ns] > 0 ? f->ch_ptr[ns] : 1));
    {
        int *fill = (int *)malloc(sizeof(int) * (ns + 1));
        memcpy(fill, f->ch_ptr, sizeof(int) * (ns + 1));
        for (int s = 0; s < ns; s++)
            if (f->sn_parent[s] >= 0) f->ch_list[fill[f->sn_parent[s]]++] = s;
        free(fill);
    }
    /* row structures: own columns, then rows below from A's columns and the children's update rows */
    f->sn_rptr = (int64_t *)malloc(sizeof(int64_t) * (ns + 1));
    int64_t cap = (int64_t)n * 8, used = 0;
    f->sn_rows = (int *)malloc(sizeof(int) * cap);
    int *mark = (int *)malloc(sizeof(int) * n);
    for (int j = 0; j < n; j++) mark[j] = -1;
    int *below = (int *)malloc(sizeof(int) * n);
    for (int s = 0; s < ns; s++) {
        int c0 = f->sn_first[s], c1 = f->sn_first[s + 1];
        int nb = 0;
        f->sn_rptr[s] = used;  /* also the end of supernode s - 1, read below when it is a child */
        for (int j = c0; j < c1; j++)
            for (int64_t p = f->lcp[j]; p < f->lcp[j + 1]; p++) {
                int i = f->lci[p];
                if (i >= c1 && mark[i] != s) { mark[i] = s; below[nb++] = i; }
            }
        for (int q = f->ch_ptr[s]; q < f->ch_ptr[s + 1]; q++) {
            int c = f->ch_list[q];
            int kc = f->sn_first[c + 1] - f->sn_first[c];
            for (int64_t p = f->sn_rptr[c] + kc; p < f->sn_rptr[c + 1]; p++) {
                int i = f->sn_rows[p];
                if (i >= c1 && mark[i] != s) { mark[i] = s; below[nb++] = i; }
            }
        }
        qsort(below, (size_t)nb, sizeof(int), cmp_int);
        int64_t m = (c1 - c0) + nb;
        while (used + m > cap) {
            cap *= 2;
            f->sn_rows = (int *)realloc(f->sn_rows, sizeof(int) * cap);
        }
        for (int j = c0; j < c1; j++) f->sn_rows[used++] = j;
        for (int q = 0; q < nb; q++) f->sn_rows[used++] = below[q];
    }
    f->sn_rptr[ns] = used;
    free(mark);
    free(below);
    free(sn_of);
    /* factor storage and work estimate */
    f->sn_lptr = (int64_t *)malloc(sizeof(int64_t) * (ns + 1));
    int64_t off = 0;
    double lnz = 0, flops = 0;
    for (int s = 0; s < ns; s++) {
        int64_t k = f->sn_first[s + 1] - f->sn_first[s], m = f->sn_rptr[s + 1] - f->sn_rptr[s];
        f->sn_lptr[s] = off;
        off += m * k;
        lnz += (double)(m * k - k * (k - 1) / 2);
        for (int64_t c = 0; c < k; c++) flops += (double)(m - c) * (double)(m - c);
    }
    f->sn_lptr[ns] = off;
    f->lnz = (int64_t)lnz;
    f->flops = flops;
    f->lx = (double *)malloc(sizeof(double) * (off > 0 ? off : 1));
    /* tree levels: height above the leaves */
    int *lev = (int *)calloc((size_t)ns, sizeof(int));
    int nlvl = 0;
    for (int s = 0; s < ns; s++) {
        if (lev[s] + 1 > nlvl) nlvl = lev[s] + 1;
        int p = f->sn_parent[s];
        if (p >= 0 && lev[p] < lev[s] + 1) lev[p] = lev[s] + 1;
    }
    f->nlvl = nlvl;
    f->lvl_ptr = (int *)calloc((size_t)nlvl + 1, sizeof(int));
    for (int s = 0; s < ns; s++) f->lvl_ptr[lev[s] + 1]++;
    for (int l = 0; l < nlvl; l++) f->lvl_ptr[l + 1] += f->lvl_ptr[l];
    f->lvl_sn = (int *)malloc(sizeof(int) * (ns > 0 ? ns : 1));
    {
        int *fill = (int *)malloc(sizeof(int) * (nlvl + 1));
        memcpy(fill, f->lvl_ptr, sizeof(int) * (nlvl + 1));
        for (int s = 0; s < ns; s++) f->lvl_sn[fill[lev[s]]++] = s;
        free(fill);
    }
    free(lev);
    f->work = (double *)malloc(sizeof(double) * (n > 0 ? n : 1));
    f->factored = 0;
    f->bad_pivot = -1;
    return 0;
}

/* ------------------------------------------------------------------ numeric factorisation */

/* One front: assemble, factor its pivot columns, keep the Schur complement in fronts[s] for the parent. */
static int process_front(ospd *f, int s, const double *values, double **fronts, int *pos, int par)
{
    int c0 = f->sn_first[s];
    int k = f->sn_first[s + 1] - c0;
    int m = (int)(f->sn_rptr[s + 1] - f->sn_rptr[s]);
    const int *rows = f->sn_rows + f->sn_rptr[s];
    double *F = (double *)calloc((size_t)m * m, sizeof(double));
    for (int a = 0; a < m; a++) pos[rows[a]] = a;
#pragma omp parallel for schedule(static) if (par && k > 64)
    for (int c = 0; c < k; c++) {
        int j = c0 + c;
        double *fc = F + (int64_t)c * m;
        for (int64_t p = f->lcp[j]; p < f->lcp[j + 1]; p++) fc[pos[f->lci[p]]] = values[f->lmap[p]];
    }
    for (int q = f->ch_ptr[s]; q < f->ch_ptr[s + 1]; q++) {
        int ch = f->ch_list[q];
        int kc = f->sn_first[ch + 1] - f->sn_first[ch];
        int mc = (int)(f->sn_rptr[ch + 1] - f->sn_rptr[ch]);
        int u = mc - kc;
        const int *rc = f->sn_rows + f->sn_rptr[ch] + kc;
        const double *U = fronts[ch] + (int64_t)kc * mc + kc;
#pragma omp parallel for schedule(static) if (par && u > 256)
        for (int b = 0; b < u; b++) {
            double *fb = F + (int64_t)pos[rc[b]] * m;
            const double *ub = U + (int64_t)b * mc;
            for (int a = b; a < u; a++) fb[pos[rc[a]]] += ub[a];
        }
        free(fronts[ch]);
        fronts[ch] = NULL;
    }
    int bad = front_factor(m, k, F, par);
    if (bad >= 0) {
        free(F);
        return c0 + bad;
    }
    double *L = f->lx + f->sn_lptr[s];
    for (int c = 0; c < k; c++) memcpy(L + (int64_t)c * m, F + (int64_t)c * m, sizeof(double) * m);
    if (f->sn_parent[s] >= 0 && m > k) fronts[s] = F;
    else free(F);
    return -1;
}

int ospd_factorize(ospd *f, const double *values)
{
    int n = f->n, ns = f->ns;
    f->factored = 0;
    f->bad_pivot = -1;
    double **fronts = (double **)calloc((size_t)(ns > 0 ? ns : 1), sizeof(double *));
    int nthreads = omp_get_max_threads();
    int **pos = (int **)malloc(sizeof(int *) * nthreads);
    for (int t = 0; t < nthreads; t++) pos[t] = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
    int bad = -1;
    for (int l = 0; l < f->nlvl && bad < 0; l++) {
        int a = f->lvl_ptr[l], b = f->lvl_ptr[l + 1];
        if (b - a >= 2 * nthreads) {
#pragma omp parallel for schedule(dynamic, 1)
            for (int q = a; q < b; q++) {
                int r = process_front(f, f->lvl_sn[q], values, fronts, pos[omp_get_thread_num()], 0);
                if (r >= 0) {
#pragma omp critical
                    if (bad < 0 || r < bad) bad = r;
                }
            }
        } else {
            for (int q = a; q < b && bad < 0; q++) {
                int r = process_front(f, f->lvl_sn[q], values, fronts, pos[0], 1);
                if (r >= 0) bad = r;
            }
        }
    }
    for (int s = 0; s < ns; s++) free(fronts[s]);
    free(fronts);
    for (int t = 0; t < nthreads; t++) free(pos[t]);
    free(pos);
    if (bad >= 0) {
        f->bad_pivot = f->perm[bad];
        return -1;
    }
    f->factored = 1;
    return 0;
}

/* ------------------------------------------------------------------ solves */

int ospd_solve(ospd *f, const double *b, double *xout)
{
    if (!f->factored) return -1;
    int n = f->n, ns = f->ns;
    double *x = f->work;
    for (int k = 0; k < n; k++) x[k] = b[f->perm[k]];
    /* L y = b */
    for (int s = 0; s < ns; s++) {
        int c0 = f->sn_first[s], k = f->sn_first[s + 1] - c0;
        int m = (int)(f->sn_rptr[s + 1] - f->sn_rptr[s]);
        const int *rows = f->sn_rows + f->sn_rptr[s];
        const double *L = f->lx + f->sn_lptr[s];
        double *xs = x + c0;
        for (int c = 0; c < k; c++) {
            const double *lc = L + (int64_t)c * m;
            double xc = xs[c] / lc[c];
            xs[c] = xc;
            for (int r = c + 1; r < k; r++) xs[r] -= lc[r] * xc;
            for (int r = k; r < m; r++) x[rows[r]] -= lc[r] * xc;
        }
    }
    /* L^T x = y */
    for (int s = ns - 1; s >= 0; s--) {
        int c0 = f->sn_first[s], k = f->sn_first[s + 1] - c0;
        int m = (int)(f->sn_rptr[s + 1] - f->sn_rptr[s]);
        const int *rows = f->sn_rows + f->sn_rptr[s];
        const double *L = f->lx + f->sn_lptr[s];
        double *xs = x + c0;
        for (int c = k - 1; c >= 0; c--) {
            const double *lc = L + (int64_t)c * m;
            double acc = xs[c];
            for (int r = c + 1; r < k; r++) acc -= lc[r] * xs[r];
            for (int r = k; r < m; r++) acc -= lc[r] * x[rows[r]];
            xs[c] = acc / lc[c];
        }
    }
    for (int k = 0; k < n; k++) xout[f->perm[k]] = x[k];
    for (int k = 0; k < n; k++)
        if (!isfinite(xout[k])) return -2;
    return 0;
}

int64_t ospd_factor_nonzeros(const ospd *f) { return f->lnz; }
int ospd_bad_pivot(const ospd *f) { return f->bad_pivot; }
double ospd_factor_flops(const ospd *f) { return f->flops; }
int ospd_supernodes(const ospd *f) { return f->ns; }
