// remesh.cu — host-side remeshing of the 3D workpiece (see remesh.h).
//
// Follows the reference's RemeshCore (ThreeD/Forging3DSolver.cs:1958-2101) step by step, because the new mesh and
// the state carried over decide every later increment: the old mesh's point locator is the inside test of an
// isosurface stuffing at h; the stuffed mesh is refined where increments failed before; surface nodes close to a
// die are put on it; the free surface is shifted along its normals to restore the part's volume; contact nodes of
// poor tets are placed to favour quality; nodes of flattened tets go back to their stuffed positions; interior
// smoothing and surface untangling repair what is left; the result is kept when it is sound (or clearly better
// than the mesh in use); element history comes from the old element at each new centroid and nodal velocities by
// linear interpolation in the old mesh.
#include "remesh.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <thread>
#include <unordered_map>
#include <utility>

#include "../../include/ifea_gpu.h"
#include "host_par.h"

namespace ifea {

namespace {

// f(i) for i in [0, n) on the host's threads (contiguous chunks); serial for small n
template <class F>
void parallel_for(int n, F &&f, bool parallel = true)
{
    int nt = parallel && n >= 4096 ? (int)std::min(32u, std::max(1u, std::thread::hardware_concurrency())) : 1;
    if (nt == 1) {
        for (int i = 0; i < n; i++) f(i);
        return;
    }
    int chunk = (n + nt - 1) / nt;
    std::vector<std::thread> th;
    for (int t = 0; t < nt; t++)
        th.emplace_back([&, t] {
            int a = t * chunk, b = std::min(n, a + chunk);
            for (int i = a; i < b; i++) f(i);
        });
    for (auto &x : th) x.join();
}

inline uint64_t edge_key(int a, int b)
{
    return a < b ? ((uint64_t)(uint32_t)a << 32) | (uint32_t)b : ((uint64_t)(uint32_t)b << 32) | (uint32_t)a;
}

inline d3 centroid4(const std::vector<d3> &x, const int32_t *t)
{
    return scl3(0.25, add3(add3(add3(x[t[0]], x[t[1]]), x[t[2]]), x[t[3]]));
}

double min_quality(const std::vector<d3> &x, const std::vector<int32_t> &t)
{
    double q = DBL_MAX;
    for (size_t e = 0; e < t.size() / 4; e++)
        q = rmin(q, tet_quality(x[t[4 * e]], x[t[4 * e + 1]], x[t[4 * e + 2]], x[t[4 * e + 3]]));
    return q;
}

// The parts of TetMesh (ThreeD/TetMesh.cs:9-64) the placement steps read: node -> tets, outward boundary faces
// in first-encounter order with their symmetry flag, surface nodes. False if a face has more than two tets.
struct LightMesh {
    int nn = 0, ne = 0;
    std::vector<int32_t> nts, ntl, bface;
    std::vector<uint8_t> bsym, surf, onx, ony;
    bool build(int nn_, const std::vector<int32_t> &t, const std::vector<d3> &x, bool sym_x, bool sym_y)
    {
        nn = nn_;
        ne = (int)(t.size() / 4);
        onx.assign(nn, 0);
        ony.assign(nn, 0);
        for (int n = 0; n < nn; n++) {
            onx[n] = sym_x && x[n].x == 0;
            ony[n] = sym_y && x[n].y == 0;
        }
        nts.assign(nn + 1, 0);
        for (int v : t) nts[v + 1]++;
        for (int n = 0; n < nn; n++) nts[n + 1] += nts[n];
        ntl.assign(t.size(), 0);
        std::vector<int32_t> fill(nts.begin(), nts.end() - 1);
        for (int e = 0; e < ne; e++)
            for (int a = 0; a < 4; a++) ntl[fill[t[4 * e + a]]++] = e;
        struct F {
            int32_t k0, k1, k2, p, q, r, seq;
        };
        // faces bucketed by their smallest node (in creation order within a bucket), each bucket sorted by its
        // other two nodes and creation order on the host's threads; a face met once is a boundary face
        std::vector<int32_t> fstart(nn + 1, 0);
        std::vector<F> faces(4 * (size_t)ne);
        for (int e = 0; e < ne; e++) {
            int a = t[4 * e], b = t[4 * e + 1], c = t[4 * e + 2], d = t[4 * e + 3];
            const int tri[4][3] = {{a, c, b}, {a, b, d}, {a, d, c}, {b, c, d}};
            for (int f = 0; f < 4; f++) {
                int s[3] = {tri[f][0], tri[f][1], tri[f][2]};
                std::sort(s, s + 3);
                faces[4 * (size_t)e + f] = {s[0], s[1], s[2], tri[f][0], tri[f][1], tri[f][2], 4 * e + f};
                fstart[s[0] + 1]++;
            }
        }
        for (int n = 0; n < nn; n++) fstart[n + 1] += fstart[n];
        std::vector<F> byk(faces.size());
        {
            std::vector<int32_t> at(fstart.begin(), fstart.end() - 1);
            for (const F &f : faces) byk[at[f.k0]++] = f;
        }
        std::vector<std::vector<F>> part(par_chunk_count(nn));
        std::atomic<bool> bad{false};
        par_chunks(nn, [&](int ti, int n0, int n1) {
            for (int n = n0; n < n1; n++) {
                F *b = byk.data() + fstart[n], *e = byk.data() + fstart[n + 1];
                std::sort(b, e, [](const F &u, const F &v) {
                    if (u.k1 != v.k1) return u.k1 < v.k1;
                    if (u.k2 != v.k2) return u.k2 < v.k2;
                    return u.seq < v.seq;
                });
                for (F *i = b; i < e;) {
                    F *j = i + 1;
                    while (j < e && j->k1 == i->k1 && j->k2 == i->k2) j++;
                    if (j - i > 2) bad = true;
                    else if (j - i == 1) part[ti].push_back(*i);
                    i = j;
                }
            }
        });
        if (bad) return false;
        std::vector<F> boundary;
        for (auto &v : part) boundary.insert(boundary.end(), v.begin(), v.end());
        std::sort(boundary.begin(), boundary.end(), [](const F &u, const F &v) { return u.seq < v.seq; });
        bface.clear();
        bsym.clear();
        surf.assign(nn, 0);
        for (const F &f : boundary) {
            bface.push_back(f.p);
            bface.push_back(f.q);
            bface.push_back(f.r);
            bool s = (onx[f.p] && onx[f.q] && onx[f.r]) || (ony[f.p] && ony[f.q] && ony[f.r]);
            bsym.push_back(s);
            if (!s) surf[f.p] = surf[f.q] = surf[f.r] = 1;
        }
        return true;
    }
};

}  // namespace

// ------------------------------------------------------------------ TetLocator (ThreeD/TetMesh.cs:116-263)

TetLocator::TetLocator(const std::vector<d3> &x, const std::vector<int32_t> &tets, double cell) : x_(x), t_(tets), cell_(cell)
{
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (const d3 &p : x) {
        lo[0] = rmin(lo[0], p.x); hi[0] = rmax(hi[0], p.x);
        lo[1] = rmin(lo[1], p.y); hi[1] = rmax(hi[1], p.y);
        lo[2] = rmin(lo[2], p.z); hi[2] = rmax(hi[2], p.z);
    }
    min_ = mk3(lo[0] - cell, lo[1] - cell, lo[2] - cell);
    nx_ = (int)((hi[0] - min_.x) / cell) + 2;
    ny_ = (int)((hi[1] - min_.y) / cell) + 2;
    nz_ = (int)((hi[2] - min_.z) / cell) + 2;
    size_t ncell = (size_t)nx_ * ny_ * nz_;
    start_.assign(ncell + 1, 0);
    int ne = (int)(tets.size() / 4);
    auto each = [&](int e, auto &&act) {
        d3 l = x[tets[4 * e]], h = l;
        for (int a = 1; a < 4; a++) {
            d3 p = x[tets[4 * e + a]];
            l = mk3(rmin(l.x, p.x), rmin(l.y, p.y), rmin(l.z, p.z));
            h = mk3(rmax(h.x, p.x), rmax(h.y, p.y), rmax(h.z, p.z));
        }
        int i0 = iclamp((int)((l.x - min_.x) / cell_), 0, nx_ - 1), i1 = iclamp((int)((h.x - min_.x) / cell_), 0, nx_ - 1);
        int j0 = iclamp((int)((l.y - min_.y) / cell_), 0, ny_ - 1), j1 = iclamp((int)((h.y - min_.y) / cell_), 0, ny_ - 1);
        int k0 = iclamp((int)((l.z - min_.z) / cell_), 0, nz_ - 1), k1 = iclamp((int)((h.z - min_.z) / cell_), 0, nz_ - 1);
        for (int k = k0; k <= k1; k++)
            for (int j = j0; j <= j1; j++)
                for (int i = i0; i <= i1; i++) act(((size_t)k * ny_ + j) * nx_ + i);
    };
    for (int e = 0; e < ne; e++) each(e, [&](size_t c) { start_[c + 1]++; });
    // bounding boxes for find(): a point whose barycentric weights are all >= -1e-9 lies within 3e-9 x the tet's
    // extent of its box; the margin, 1e-4 of a cell, leaves room for the weights' rounding too
    bb_margin_ = 1e-4 * cell_;
    bb_.resize(6 * (size_t)ne);
    parallel_for(ne, [&](int e) {
        d3 l = x[tets[4 * e]], h = l;
        for (int a = 1; a < 4; a++) {
            d3 p = x[tets[4 * e + a]];
            l = mk3(rmin(l.x, p.x), rmin(l.y, p.y), rmin(l.z, p.z));
            h = mk3(rmax(h.x, p.x), rmax(h.y, p.y), rmax(h.z, p.z));
        }
        double *b = &bb_[6 * (size_t)e];
        b[0] = l.x - bb_margin_; b[1] = l.y - bb_margin_; b[2] = l.z - bb_margin_;
        b[3] = h.x + bb_margin_; b[4] = h.y + bb_margin_; b[5] = h.z + bb_margin_;
    });
    for (size_t c = 0; c < ncell; c++) start_[c + 1] += start_[c];
    items_.assign(start_[ncell], 0);
    std::vector<int32_t> fill(start_.begin(), start_.end() - 1);
    for (int e = 0; e < ne; e++) each(e, [&](size_t c) { items_[fill[c]++] = e; });
    nstart_.assign(ncell + 1, 0);
    std::vector<int32_t> ncell_of(x.size());
    for (size_t n = 0; n < x.size(); n++) {
        ncell_of[n] = cell_of(x[n]);
        nstart_[ncell_of[n] + 1]++;
    }
    for (size_t c = 0; c < ncell; c++) nstart_[c + 1] += nstart_[c];
    nitems_.assign(x.size(), 0);
    std::vector<int32_t> nfill(nstart_.begin(), nstart_.end() - 1);
    for (size_t n = 0; n < x.size(); n++) nitems_[nfill[ncell_of[n]]++] = (int32_t)n;
}

int TetLocator::cell_of(d3 p) const
{
    int i = iclamp((int)((p.x - min_.x) / cell_), 0, nx_ - 1), j = iclamp((int)((p.y - min_.y) / cell_), 0, ny_ - 1),
        k = iclamp((int)((p.z - min_.z) / cell_), 0, nz_ - 1);
    return (int)(((size_t)k * ny_ + j) * nx_ + i);
}

int TetLocator::find(d3 p, double w[4]) const
{
    w[0] = w[1] = w[2] = w[3] = 0;
    int c = cell_of(p);
    for (int32_t k = start_[c]; k < start_[c + 1]; k++) {
        int e = items_[k];
        const double *bb = &bb_[6 * (size_t)e];
        if (p.x < bb[0] || p.y < bb[1] || p.z < bb[2] || p.x > bb[3] || p.y > bb[4] || p.z > bb[5]) continue;
        d3 a = x_[t_[4 * e]], b = x_[t_[4 * e + 1]], cc = x_[t_[4 * e + 2]], d = x_[t_[4 * e + 3]];
        double v = tet_volume(a, b, cc, d);
        if (v <= 0) continue;
        double b0 = tet_volume(p, b, cc, d) / v, b1 = tet_volume(a, p, cc, d) / v, b2 = tet_volume(a, b, p, d) / v;
        double b3 = 1 - b0 - b1 - b2;
        const double tol = -1e-9;
        if (b0 >= tol && b1 >= tol && b2 >= tol && b3 >= tol) {
            w[0] = b0; w[1] = b1; w[2] = b2; w[3] = b3;
            return e;
        }
    }
    return -1;
}

d3 TetLocator::interpolate(d3 p, const double *field) const
{
    double w[4];
    int e = find(p, w);
    if (e >= 0) {
        d3 r = scl3(w[0], ld3(field, t_[4 * e]));
        for (int a = 1; a < 4; a++) r = add3(r, scl3(w[a], ld3(field, t_[4 * e + a])));
        return r;
    }
    return ld3(field, nearest_node(p));
}

// the nearest node (the lowest index among equally near ones), searched ring by ring over a grid of nodes; any
// node outside the rings searched so far is at least r cells away
int TetLocator::nearest_node(d3 p) const
{
    int ci = iclamp((int)((p.x - min_.x) / cell_), 0, nx_ - 1), cj = iclamp((int)((p.y - min_.y) / cell_), 0, ny_ - 1),
        ck = iclamp((int)((p.z - min_.z) / cell_), 0, nz_ - 1);
    double dmin = DBL_MAX;
    int best = 0;
    int rmax = std::max(nx_, std::max(ny_, nz_));
    for (int r = 0; r <= rmax; r++) {
        for (int k = ck - r; k <= ck + r; k++)
            for (int j = cj - r; j <= cj + r; j++)
                for (int i = ci - r; i <= ci + r; i++) {
                    if (i < 0 || j < 0 || k < 0 || i >= nx_ || j >= ny_ || k >= nz_) continue;
                    if (std::max(std::abs(i - ci), std::max(std::abs(j - cj), std::abs(k - ck))) != r) continue;
                    size_t c = ((size_t)k * ny_ + j) * nx_ + i;
                    for (int32_t q = nstart_[c]; q < nstart_[c + 1]; q++) {
                        int n = nitems_[q];
                        double dd = len23(sub3(x_[n], p));
                        if (dd < dmin || (dd == dmin && n < best)) {
                            dmin = dd;
                            best = n;
                        }
                    }
                }
        // a point outside the grid box is farther still from everything beyond ring r, so this stop is safe
        if (dmin < DBL_MAX && sqrt(dmin) <= r * cell_) break;
    }
    return best;
}

int TetLocator::find_nearest(d3 p) const
{
    double w[4];
    int e = find(p, w);
    if (e >= 0) return e;
    int c = cell_of(p), best_e = -1;
    double best = DBL_MAX;
    for (int32_t k = start_[c]; k < start_[c + 1]; k++) {
        int ee = items_[k];
        double dd = len23(sub3(centroid4(x_, t_.data() + 4 * (size_t)ee), p));
        if (dd < best) {
            best = dd;
            best_e = ee;
        }
    }
    if (best_e >= 0) return best_e;
    for (int ee = 0; ee < (int)(t_.size() / 4); ee++) {
        double dd = len23(sub3(centroid4(x_, t_.data() + 4 * (size_t)ee), p));
        if (dd < best) {
            best = dd;
            best_e = ee;
        }
    }
    return best_e;
}

// ------------------------------------------------------------------ isosurface stuffing (ThreeD/IsosurfaceStuffing.cs)

void stuff_uniform(const std::function<bool(d3)> &inside, d3 lo, d3 hi, double h, bool sym_x, bool sym_y,
                   std::vector<d3> &out_pts, std::vector<int32_t> &out_tets, bool parallel)
{
    const double alpha_long = 0.24999, alpha_short = 0.41189;  // the published warp thresholds
    const double eps = 1e-7 * h;
    auto In = [&](d3 p) {
        if ((sym_x && p.x < 0) || (sym_y && p.y < 0)) return false;
        return inside(mk3(sym_x ? rmax(p.x, eps) : p.x, sym_y ? rmax(p.y, eps) : p.y, p.z));
    };
    // lattice offset: no lattice vertex on a symmetry plane, which keeps the plane / surface creases filled
    const d3 off = mk3(0.31 * h, 0.37 * h, 0.17 * h);
    int i0 = (int)floor(lo.x / h) - 1, i1 = (int)ceil(hi.x / h) + 1;
    int j0 = (int)floor(lo.y / h) - 1, j1 = (int)ceil(hi.y / h) + 1;
    int k0 = (int)floor(lo.z / h) - 1, k1 = (int)ceil(hi.z / h) + 1;
    int ni = i1 - i0, nj = j1 - j0, nk = k1 - k0;
    int64_t n_corner = (int64_t)(ni + 1) * (nj + 1) * (nk + 1), n_center = (int64_t)ni * nj * nk;
    auto corner = [&](int i, int j, int k) { return (int)(((int64_t)(k - k0) * (nj + 1) + (j - j0)) * (ni + 1) + (i - i0)); };
    auto center = [&](int i, int j, int k) { return (int)(n_corner + ((int64_t)(k - k0) * nj + (j - j0)) * ni + (i - i0)); };
    std::vector<d3> pos;
    pos.reserve((size_t)(n_corner + n_center));
    for (int k = k0; k <= k1; k++)
        for (int j = j0; j <= j1; j++)
            for (int i = i0; i <= i1; i++) pos.push_back(add3(mk3(i * h, j * h, k * h), off));
    for (int k = k0; k < k1; k++)
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++) pos.push_back(add3(mk3((i + 0.5) * h, (j + 0.5) * h, (k + 0.5) * h), off));
    // BCC tets: two face-adjacent cube centres and one edge of their shared face
    std::vector<int32_t> lat;
    auto add_pair = [&](int c1, int c2, int a, int b, int c, int d) {
        const int q[4][4] = {{c1, c2, a, b}, {c1, c2, b, c}, {c1, c2, c, d}, {c1, c2, d, a}};
        for (auto &r : q) lat.insert(lat.end(), r, r + 4);
    };
    for (int k = k0; k < k1; k++)
        for (int j = j0; j < j1; j++)
            for (int i = i0; i < i1; i++) {
                int c = center(i, j, k);
                if (i + 1 < i1)
                    add_pair(c, center(i + 1, j, k), corner(i + 1, j, k), corner(i + 1, j + 1, k), corner(i + 1, j + 1, k + 1), corner(i + 1, j, k + 1));
                if (j + 1 < j1)
                    add_pair(c, center(i, j + 1, k), corner(i, j + 1, k), corner(i + 1, j + 1, k), corner(i + 1, j + 1, k + 1), corner(i, j + 1, k + 1));
                if (k + 1 < k1)
                    add_pair(c, center(i, j, k + 1), corner(i, j, k + 1), corner(i + 1, j, k + 1), corner(i + 1, j + 1, k + 1), corner(i, j + 1, k + 1));
            }
    auto is_corner = [&](int v) { return v < n_corner; };
    std::vector<int8_t> sign(pos.size());
    parallel_for((int)pos.size(), [&](int v) { sign[v] = In(pos[v]) ? -1 : 1; }, parallel);
    auto crosses = [&](int u, int w) { return (sign[u] < 0 && sign[w] > 0) || (sign[u] > 0 && sign[w] < 0); };
    const int ea[6] = {0, 0, 0, 1, 1, 2}, eb[6] = {1, 2, 3, 2, 3, 3};
    // cut points on the edges between an inside and an outside vertex, in creation order, each bisected on the
    // inside test (independently of the others)
    std::unordered_map<uint64_t, int> cut_index;
    std::vector<std::pair<uint64_t, d3>> cuts;
    for (size_t t = 0; t < lat.size(); t += 4)
        for (int q = 0; q < 6; q++) {
            int u = lat[t + ea[q]], w = lat[t + eb[q]];
            if (!crosses(u, w)) continue;
            uint64_t key = edge_key(u, w);
            if (cut_index.count(key)) continue;
            cut_index[key] = (int)cuts.size();
            cuts.push_back({key, mk3(0, 0, 0)});
        }
    parallel_for((int)cuts.size(), [&](int ci) {
        int u = (int)(cuts[ci].first >> 32), w = (int)(cuts[ci].first & 0xffffffffu);
        d3 pin = sign[u] < 0 ? pos[u] : pos[w], pout = sign[u] < 0 ? pos[w] : pos[u];
        for (int it = 0; it < 16; it++) {
            d3 m = scl3(0.5, add3(pin, pout));
            if (In(m)) pin = m;
            else pout = m;
        }
        d3 cp = scl3(0.5, add3(pin, pout));
        if (sym_x && fabs(cp.x) < 1e-4 * h) cp.x = 0;
        if (sym_y && fabs(cp.y) < 1e-4 * h) cp.y = 0;
        cuts[ci].second = cp;
    }, parallel);
    // warp lattice vertices too close to a cut point onto it (the nearest cut; the first on ties)
    std::vector<int> warp_to(pos.size(), -1);
    std::vector<double> warp_d(pos.size(), DBL_MAX);
    for (size_t ci = 0; ci < cuts.size(); ci++) {
        int u = (int)(cuts[ci].first >> 32), w = (int)(cuts[ci].first & 0xffffffffu);
        d3 c = cuts[ci].second;
        double len = len3(sub3(pos[w], pos[u]));
        double alpha = is_corner(u) == is_corner(w) ? alpha_long : alpha_short;
        for (int v : {u, w}) {
            double d = len3(sub3(c, pos[v]));
            if (d >= alpha * len) continue;
            if (d < warp_d[v]) {
                warp_d[v] = d;
                warp_to[v] = (int)ci;
            }
        }
    }
    for (size_t v = 0; v < pos.size(); v++)
        if (warp_to[v] >= 0) {
            pos[v] = cuts[warp_to[v]].second;
            sign[v] = 0;
        }
    // clip and tetrahedralise every lattice tet that reaches into the body; clipped polyhedra are coned from their
    // smallest vertex id, face diagonals by the same rule, so neighbouring tets agree on shared faces
    std::unordered_map<uint64_t, int> cut_vertex;
    auto cut_v = [&](int u, int w) {
        uint64_t key = edge_key(u, w);
        auto it = cut_vertex.find(key);
        if (it != cut_vertex.end()) return it->second;
        pos.push_back(cuts[cut_index.at(key)].second);
        sign.push_back(0);
        int id = (int)pos.size() - 1;
        cut_vertex[key] = id;
        return id;
    };
    const double min_vol = 1e-6 * h * h * h;
    std::vector<int32_t> tets;
    auto emit = [&](int a, int b, int c, int d) {
        double v = tet_volume(pos[a], pos[b], pos[c], pos[d]);
        if (fabs(v) < min_vol) return;
        if (v < 0) std::swap(c, d);
        tets.push_back(a); tets.push_back(b); tets.push_back(c); tets.push_back(d);
    };
    auto cone = [&](const std::vector<int> &f, int apex) {
        if (f.size() < 3 || std::find(f.begin(), f.end(), apex) != f.end()) return;
        int s = (int)(std::min_element(f.begin(), f.end()) - f.begin()), n = (int)f.size();
        for (int q = 1; q < n - 1; q++) emit(apex, f[s], f[(s + q) % n], f[(s + q + 1) % n]);
    };
    auto order_planar = [&](std::vector<int> &f, const std::vector<int> &all) {
        d3 c = mk3(0, 0, 0);
        for (int v : f) c = add3(c, pos[v]);
        c = scl3(1.0 / f.size(), c);
        d3 inner = mk3(0, 0, 0);
        int cnt = 0;
        for (int v : all)
            if (sign[v] < 0) {
                inner = add3(inner, pos[v]);
                cnt++;
            }
        d3 nrm = nrm3(sub3(c, scl3(1.0 / std::max(cnt, 1), inner)));
        d3 ax = fabs(nrm.x) < 0.9 ? mk3(1, 0, 0) : mk3(0, 1, 0);
        d3 u = nrm3(cross3(ax, nrm)), w = cross3(nrm, u);
        std::vector<std::pair<double, int>> keyed;
        for (int v : f) keyed.push_back({atan2(dot3(sub3(pos[v], c), w), dot3(sub3(pos[v], c), u)), v});
        std::stable_sort(keyed.begin(), keyed.end(),
                         [](const std::pair<double, int> &a, const std::pair<double, int> &b) { return a.first < b.first; });
        for (size_t i = 0; i < f.size(); i++) f[i] = keyed[i].second;
    };
    const int faces[4][3] = {{0, 1, 2}, {0, 1, 3}, {0, 2, 3}, {1, 2, 3}};
    std::vector<int> poly, face, iface;
    for (size_t t = 0; t < lat.size(); t += 4) {
        int v[4] = {lat[t], lat[t + 1], lat[t + 2], lat[t + 3]};
        int neg = 0, pc = 0;
        for (int q = 0; q < 4; q++) {
            if (sign[v[q]] < 0) neg++;
            else if (sign[v[q]] > 0) pc++;
        }
        if (neg == 0) continue;
        if (pc == 0) {
            emit(v[0], v[1], v[2], v[3]);
            continue;
        }
        poly.clear();
        iface.clear();
        for (int q = 0; q < 4; q++) {
            if (sign[v[q]] <= 0) poly.push_back(v[q]);
            if (sign[v[q]] == 0) iface.push_back(v[q]);
        }
        for (int q = 0; q < 6; q++) {
            int u = v[ea[q]], w = v[eb[q]];
            if (crosses(u, w)) {
                int c = cut_v(u, w);
                poly.push_back(c);
                iface.push_back(c);
            }
        }
        int apex = *std::min_element(poly.begin(), poly.end());
        for (auto &f : faces) {
            face.clear();
            for (int q = 0; q < 3; q++) {
                int a = v[f[q]], b = v[f[(q + 1) % 3]];
                if (sign[a] <= 0) face.push_back(a);
                if (crosses(a, b)) face.push_back(cut_v(a, b));
            }
            cone(face, apex);
        }
        if (iface.size() >= 3) {
            order_planar(iface, poly);
            cone(iface, apex);
        }
    }
    // compact: points in order of first use
    std::vector<int> map(pos.size(), -1);
    out_pts.clear();
    out_tets.assign(tets.size(), 0);
    for (size_t q = 0; q < tets.size(); q++) {
        int old = tets[q];
        if (map[old] < 0) {
            map[old] = (int)out_pts.size();
            out_pts.push_back(pos[old]);
        }
        out_tets[q] = map[old];
    }
}

// ------------------------------------------------------------------ local refinement (ThreeD/TetRefiner.cs)

namespace {
struct EdgeHash {
    size_t operator()(uint64_t k) const
    {
        k ^= k >> 33;
        k *= 0xff51afd7ed558ccdULL;
        k ^= k >> 33;
        return (size_t)k;
    }
};
}  // namespace

int refine_tets(std::vector<d3> &pts, std::vector<int32_t> &tl, const std::function<double(d3)> &target, int max_nodes)
{
    std::unordered_map<uint64_t, std::vector<int>, EdgeHash> edges;
    edges.reserve(tl.size() * 2);
    auto add_edges = [&](int e) {
        for (int i = 0; i < 4; i++)
            for (int j = i + 1; j < 4; j++) edges[edge_key(tl[4 * (size_t)e + i], tl[4 * (size_t)e + j])].push_back(e);
    };
    auto remove_edges = [&](int e) {
        for (int i = 0; i < 4; i++)
            for (int j = i + 1; j < 4; j++) {
                auto it = edges.find(edge_key(tl[4 * (size_t)e + i], tl[4 * (size_t)e + j]));
                if (it == edges.end()) continue;
                auto &l = it->second;
                auto p = std::find(l.begin(), l.end(), e);
                if (p != l.end()) l.erase(p);
            }
    };
    auto longest = [&](int e, int &ba, int &bb) {
        double best = -1;
        ba = bb = 0;
        for (int i = 0; i < 4; i++)
            for (int j = i + 1; j < 4; j++) {
                int a = tl[4 * (size_t)e + i], b = tl[4 * (size_t)e + j];
                double l = len23(sub3(pts[a], pts[b]));
                // deterministic tie-break on node ids: neighbouring tets choose the same edge
                if (l > best * (1 + 1e-12) || (fabs(l - best) <= best * 1e-12 && edge_key(a, b) < edge_key(ba, bb))) {
                    best = l;
                    ba = a;
                    bb = b;
                }
            }
        return sqrt(best);
    };
    auto split = [&](int a, int b) {
        int m = (int)pts.size();
        pts.push_back(scl3(0.5, add3(pts[a], pts[b])));
        std::vector<int> around = edges[edge_key(a, b)];
        for (int e : around) {
            remove_edges(e);
            size_t nt = tl.size() / 4;
            for (int i = 0; i < 4; i++) tl.push_back(tl[4 * (size_t)e + i]);
            // b becomes the midpoint in the original, a in the copy: both keep the orientation
            for (int i = 0; i < 4; i++) {
                if (tl[4 * (size_t)e + i] == b) tl[4 * (size_t)e + i] = m;
                if (tl[4 * nt + i] == a) tl[4 * nt + i] = m;
            }
            add_edges(e);
            add_edges((int)nt);
        }
        edges.erase(edge_key(a, b));
    };
    // Rivara's longest-edge propagation: bisect an edge only once it is the longest of every tet around it
    auto refine_edge = [&](int a0, int b0) {
        std::vector<std::pair<int, int>> stack{{a0, b0}};
        int count = 0;
        while (!stack.empty() && (int)pts.size() < max_nodes && stack.size() < 64) {
            auto [a, b] = stack.back();
            auto it = edges.find(edge_key(a, b));
            if (it == edges.end() || it->second.empty()) {
                stack.pop_back();
                continue;
            }
            bool deferred = false;
            for (int f : it->second) {
                int fa, fb;
                longest(f, fa, fb);
                if (edge_key(fa, fb) == edge_key(a, b)) continue;
                stack.push_back({fa, fb});
                deferred = true;
                break;
            }
            if (deferred) continue;
            stack.pop_back();
            split(a, b);
            count++;
        }
        return count;
    };
    // the edge map is built only when some tet needs refining
    bool any = false;
    for (int e = 0; e < (int)(tl.size() / 4) && !any; e++) {
        int a, b;
        double len = longest(e, a, b);
        any = len > 1.05 * target(centroid4(pts, tl.data() + 4 * (size_t)e));
    }
    if (!any) return 0;
    for (int e = 0; e < (int)(tl.size() / 4); e++) add_edges(e);
    int splits = 0;
    for (int pass = 0; pass < 12 && (int)pts.size() < max_nodes; pass++) {
        struct Todo {
            double len;
            int a, b;
        };
        std::vector<Todo> todo;
        for (int e = 0; e < (int)(tl.size() / 4); e++) {
            int a, b;
            double len = longest(e, a, b);
            if (len > 1.05 * target(centroid4(pts, tl.data() + 4 * (size_t)e))) todo.push_back({len, a, b});
        }
        if (todo.empty()) break;
        std::stable_sort(todo.begin(), todo.end(), [](const Todo &x, const Todo &y) { return x.len > y.len; });
        int done = 0;
        for (const Todo &t : todo) {
            if ((int)pts.size() >= max_nodes) break;
            auto it = edges.find(edge_key(t.a, t.b));
            if (it == edges.end() || it->second.empty()) continue;  // already split
            done += refine_edge(t.a, t.b);
        }
        splits += done;
        if (done == 0) break;
    }
    return splits;
}

// ------------------------------------------------------------------ RemeshCore (ThreeD/Forging3DSolver.cs:1958-2101)

namespace {

struct Placer {
    const RemeshInput &in;
    const LightMesh &M;
    const std::vector<int32_t> &t;
    const std::vector<double> &hloc;
    bool lenient() const { return in.recovery_pass >= 2; }
    double tol(double local) const { return lenient() ? in.h : local; }  // Tol (:1605)
    double corner_allowance(double local) const                           // CornerAllowance (:1608-1609)
    {
        static const double ladder[2] = {0.05, 0.1};
        return lenient() ? 0.3 * in.h : ladder[iclamp(in.recovery_pass, 0, 1)] * local;
    }
    const HField &surface(int c) const { return c == IFEA_TOP_DIE ? in.die[1] : in.die[0]; }
    double offset(int c) const { return c == IFEA_TOP_DIE ? in.gap : 0.0; }
    d3 sym_on(d3 p, int n) const { return mk3(M.onx[n] ? 0 : p.x, M.ony[n] ? 0 : p.y, p.z); }
    double quality(const std::vector<d3> &x, int e) const
    {
        return tet_quality(x[t[4 * (size_t)e]], x[t[4 * (size_t)e + 1]], x[t[4 * (size_t)e + 2]], x[t[4 * (size_t)e + 3]]);
    }
    // nodes of the tets below qtarget (the tets' qualities on the host's threads); false if there are none
    bool mark_bad(const std::vector<d3> &x, double qtarget, std::vector<uint8_t> &bad) const
    {
        std::vector<uint8_t> low(M.ne);
        parallel_for(M.ne, [&](int e) { low[e] = quality(x, e) < qtarget; });
        std::fill(bad.begin(), bad.end(), 0);
        bool any = false;
        for (int e = 0; e < M.ne; e++) {
            if (!low[e]) continue;
            for (int a = 0; a < 4; a++) bad[t[4 * (size_t)e + a]] = 1;
            any = true;
        }
        return any;
    }
    double worst_around(const std::vector<d3> &x, int n) const
    {
        double q = DBL_MAX;
        for (int32_t k = M.nts[n]; k < M.nts[n + 1]; k++) q = rmin(q, quality(x, M.ntl[k]));
        return q;
    }
    // PushOut (:1570-1593): exit along the inward normal, else the closest die point
    d3 push_out(const HField &die, double off, d3 p, d3 outward) const
    {
        if (len23(outward) == 0 || hf_clearance(die, p, off) >= 0) return hf_project(die, p, off, nullptr);
        d3 d = neg3(outward);
        double step = 0.1 * in.h, lo = 0, hi = -1;
        for (double s = step; s <= 2 * in.h + 1e-12; s += step) {
            if (hf_clearance(die, add3(p, scl3(s, d)), off) >= 0) {
                hi = s;
                break;
            }
            lo = s;
        }
        if (hi < 0) return hf_project(die, p, off, nullptr);
        for (int i = 0; i < 25; i++) {
            double mid = 0.5 * (lo + hi);
            if (hf_clearance(die, add3(p, scl3(mid, d)), off) >= 0) hi = mid;
            else lo = mid;
        }
        return add3(p, scl3(hi, d));
    }
    // ImprovePlacement (:1625-1679)
    int improve_placement(std::vector<d3> &x, std::vector<uint8_t> &contact, const std::vector<d3> &pred,
                          const std::vector<d3> &nrm, double qmin) const
    {
        int total = 0;
        for (int sweep = 0; sweep < 4; sweep++) {
            int count = 0;
            for (int e = 0; e < M.ne; e++) {
                if (quality(x, e) >= qmin) continue;
                for (int a = 0; a < 4; a++) {
                    int n = t[4 * (size_t)e + a];
                    if (contact[n] == IFEA_FREE) continue;
                    const HField &die = surface(contact[n]);
                    double off = offset(contact[n]);
                    d3 cand[8];
                    int k = 0;
                    d3 closest = sym_on(hf_project(die, pred[n], off, nullptr), n);
                    cand[k++] = closest;
                    d3 push = sym_on(push_out(die, off, pred[n], nrm[n]), n);
                    if (len3(sub3(push, pred[n])) <= 0.5 * tol(hloc[n])) cand[k++] = push;
                    double pen = -hf_clearance(die, pred[n], off);
                    const double fr[4] = {0.0, 0.25, 0.5, 0.75};
                    for (double f : fr)
                        if (pen * (1 - f) <= corner_allowance(hloc[n])) cand[k++] = lerp3(pred[n], closest, f);
                    d3 old = x[n];
                    double best = worst_around(x, n);
                    int pick = -1;
                    for (int c = 0; c < k; c++) {
                        if (eq3(cand[c], old)) continue;
                        x[n] = cand[c];
                        double q = worst_around(x, n);
                        if (q > best + 1e-6) {
                            best = q;
                            pick = c;
                        }
                    }
                    x[n] = pick >= 0 ? cand[pick] : old;
                    if (pick < 0) continue;
                    if (eq3(cand[pick], pred[n]) && pen < 0) contact[n] = IFEA_FREE;
                    count++;
                }
            }
            total += count;
            if (count == 0) break;
        }
        return total;
    }
    // SmoothInterior (:1776-1838)
    int smooth_interior(std::vector<d3> &x, double qtarget, int sweeps) const
    {
        int moves = 0;
        std::vector<uint8_t> bad(M.nn);
        for (int s = 0; s < sweeps; s++) {
            bool any = mark_bad(x, qtarget, bad);
            if (!any) break;
            int sm = 0;
            for (int n = 0; n < M.nn; n++) {
                if (!bad[n] || M.surf[n]) continue;
                d3 sum = mk3(0, 0, 0);
                int cnt = 0;
                double worst = DBL_MAX;
                for (int32_t k = M.nts[n]; k < M.nts[n + 1]; k++) {
                    int e = M.ntl[k];
                    for (int a = 0; a < 4; a++) {
                        int m = t[4 * (size_t)e + a];
                        if (m == n) continue;
                        sum = add3(sum, x[m]);
                        cnt++;
                    }
                    worst = rmin(worst, quality(x, e));
                }
                if (cnt == 0) continue;
                d3 old = x[n], c = scl3(1.0 / cnt, sum);
                const double lam[3] = {1.0, 0.5, 0.25};
                for (double l : lam) {
                    d3 p = add3(old, scl3(l, sub3(c, old)));
                    x[n] = mk3(M.onx[n] ? 0 : p.x, M.ony[n] ? 0 : p.y, p.z);
                    double q = DBL_MAX;
                    for (int32_t k = M.nts[n]; k < M.nts[n + 1]; k++) q = rmin(q, quality(x, M.ntl[k]));
                    if (q > worst + 1e-6) {
                        sm++;
                        break;
                    }
                    x[n] = old;
                }
            }
            moves += sm;
            if (sm == 0) break;
        }
        return moves;
    }
    // UntangleSurface (:1698-1767)
    int untangle_surface(std::vector<d3> &x, std::vector<uint8_t> &contact, const std::vector<d3> &stuffed,
                         double qtarget, int sweeps) const
    {
        int moves = 0;
        std::vector<uint8_t> bad(M.nn);
        for (int s = 0; s < sweeps; s++) {
            bool any = mark_bad(x, qtarget, bad);
            if (!any) break;
            int sm = 0;
            for (int n = 0; n < M.nn; n++) {
                if (!bad[n] || !M.surf[n]) continue;
                d3 sum = mk3(0, 0, 0);
                int cnt = 0;
                for (int32_t k = M.nts[n]; k < M.nts[n + 1]; k++) {
                    int e = M.ntl[k];
                    for (int a = 0; a < 4; a++) {
                        int m = t[4 * (size_t)e + a];
                        if (m == n) continue;
                        sum = add3(sum, x[m]);
                        cnt++;
                    }
                }
                if (cnt == 0) continue;
                d3 old = x[n];
                double worst = worst_around(x, n);
                d3 centroid = scl3(1.0 / cnt, sum), best = old;
                double best_q = worst;
                const d3 targets[2] = {stuffed[n], centroid};
                const double lam[3] = {1.0, 0.5, 0.25};
                for (const d3 &tg : targets)
                    for (double l : lam) {
                        d3 p = sym_on(add3(old, scl3(l, sub3(tg, old))), n);
                        if (rmin(hf_clearance(in.die[0], p, 0), hf_clearance(in.die[1], p, in.gap)) < 0) continue;
                        x[n] = p;
                        double q = worst_around(x, n);
                        if (q > best_q + 1e-6) {
                            best = p;
                            best_q = q;
                        }
                    }
                x[n] = best;
                if (!eq3(best, old)) {
                    contact[n] = IFEA_FREE;
                    sm++;
                }
            }
            moves += sm;
            if (sm == 0) break;
        }
        return moves;
    }
};

// SurfaceNormals (:1540-1568): area-weighted outward unit normals at surface nodes
std::vector<d3> surface_normals(const LightMesh &M, const std::vector<d3> &x)
{
    std::vector<d3> n(M.nn, mk3(0, 0, 0));
    for (size_t k = 0; k < M.bsym.size(); k++) {
        if (M.bsym[k]) continue;
        int a = M.bface[3 * k], b = M.bface[3 * k + 1], c = M.bface[3 * k + 2];
        d3 an = cross3(sub3(x[b], x[a]), sub3(x[c], x[a]));
        n[a] = add3(n[a], an);
        n[b] = add3(n[b], an);
        n[c] = add3(n[c], an);
    }
    for (int i = 0; i < M.nn; i++) {
        if (M.onx[i]) n[i].x = 0;
        if (M.ony[i]) n[i].y = 0;
        if (len23(n[i]) > 0) n[i] = nrm3(n[i]);
    }
    return n;
}

// LocalLengths (:443-466): mean length of the node's edges (over its tets), capped at h
std::vector<double> local_lengths_of(const LightMesh &M, const std::vector<int32_t> &t, const std::vector<d3> &x, double h)
{
    std::vector<double> sum(M.nn, 0.0);
    std::vector<int> count(M.nn, 0);
    for (int e = 0; e < M.ne; e++)
        for (int a = 0; a < 4; a++)
            for (int b = a + 1; b < 4; b++) {
                int i = t[4 * (size_t)e + a], j = t[4 * (size_t)e + b];
                double l = len3(sub3(x[i], x[j]));
                sum[i] += l;
                sum[j] += l;
                count[i]++;
                count[j]++;
            }
    for (int n = 0; n < M.nn; n++) sum[n] = count[n] > 0 ? rmin(sum[n] / count[n], h) : h;
    return sum;
}

// CompensateVolume (:2108-2147): shift the free surface along its normals to restore the modelled volume
void compensate_volume(const RemeshInput &in, const LightMesh &M, const std::vector<int32_t> &t, std::vector<d3> &x,
                       const std::vector<uint8_t> &contact)
{
    const double max_compensation = 1.0;  // Forging3DSolver.MaxCompensation, x h per remesh
    double vol = 0;
    for (int e = 0; e < M.ne; e++)
        vol += tet_volume(x[t[4 * (size_t)e]], x[t[4 * (size_t)e + 1]], x[t[4 * (size_t)e + 2]], x[t[4 * (size_t)e + 3]]);
    double deficit = in.vol_target - vol;
    std::vector<d3> normals(M.nn, mk3(0, 0, 0));
    for (size_t k = 0; k < M.bsym.size(); k++) {
        if (M.bsym[k]) continue;
        int a = M.bface[3 * k], b = M.bface[3 * k + 1], c = M.bface[3 * k + 2];
        d3 an = scl3(0.5, cross3(sub3(x[b], x[a]), sub3(x[c], x[a])));
        normals[a] = add3(normals[a], an);
        normals[b] = add3(normals[b], an);
        normals[c] = add3(normals[c], an);
    }
    double rate = 0;
    std::vector<uint8_t> moving(M.nn, 0);
    for (int n = 0; n < M.nn; n++) {
        if (!M.surf[n] || contact[n] != IFEA_FREE) continue;
        d3 nv = normals[n];
        if (M.onx[n]) nv.x = 0;
        if (M.ony[n]) nv.y = 0;
        rate += len3(nv) / 3;
        normals[n] = nrm3(nv);
        moving[n] = !(normals[n].x == 0 && normals[n].y == 0 && normals[n].z == 0);
    }
    if (rate <= 0) return;
    double shift = rclamp(deficit / rate, -max_compensation * in.h, max_compensation * in.h);
    for (int n = 0; n < M.nn; n++) {
        if (!moving[n]) continue;
        d3 moved = add3(x[n], scl3(shift, normals[n]));
        if (hf_clearance(in.die[0], moved, 0) > 0 && hf_clearance(in.die[1], moved, in.gap) > 0) x[n] = moved;
    }
}

}  // namespace

namespace {
double seconds_since(std::chrono::steady_clock::time_point t0)
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}
}  // namespace

bool remesh_workpiece(const RemeshInput &in, RemeshOutput &out)
{
    auto t0 = std::chrono::steady_clock::now();
    std::vector<d3> ox(in.nn);
    for (int n = 0; n < in.nn; n++) ox[n] = ld3(in.x, n);
    std::vector<int32_t> ot(in.tets, in.tets + 4 * (size_t)in.ne);
    out.q_old = min_quality(ox, ot);
    TetLocator locator(ox, ot, 2 * in.h);
    d3 lo = ox[0], hi = ox[0];
    for (const d3 &p : ox) {
        lo = mk3(rmin(lo.x, p.x), rmin(lo.y, p.y), rmin(lo.z, p.z));
        hi = mk3(rmax(hi.x, p.x), rmax(hi.y, p.y), rmax(hi.z, p.z));
    }
    std::vector<d3> x;
    std::vector<int32_t> t;
    stuff_uniform([&](d3 p) { return locator.contains(p); }, lo, hi, in.h, in.sym_x, in.sym_y, x, t, true);
    if (t.empty()) {
        out.why = "isosurface stuffing produced no tetrahedra";
        return false;
    }
    out.t_stuff = seconds_since(t0);
    t0 = std::chrono::steady_clock::now();
    if (in.refinement_levels > 0) {
        // TargetSize (:287-305) with the reference defaults (no graded mesh, thin-flash or die-edge refinement): h,
        // and h / 2^level within 2 h of the places where earlier increments failed
        double hmin = in.h / (1 << in.refinement_levels);
        auto target = [&](d3 p) {
            double s = in.h;
            for (const HotSpot &hs : in.hot)
                if (len23(sub3(p, hs.at)) < 4 * in.h * in.h) s = rmin(s, rmax(in.h / (1 << hs.level), hmin));
            return s;
        };
        out.splits = refine_tets(x, t, target, in.max_nodes);
    }
    out.t_refine = seconds_since(t0);
    t0 = std::chrono::steady_clock::now();
    int nn = (int)x.size();
    if (in.on_topology) {
        // the caller's work on the final tets (the stepper's topology and analysis) starts here, beside the
        // surface extraction and placement below; the symmetry-plane flags are LightMesh's
        std::vector<uint8_t> onx(nn), ony(nn);
        for (int n = 0; n < nn; n++) {
            onx[n] = in.sym_x && x[n].x == 0;
            ony[n] = in.sym_y && x[n].y == 0;
        }
        in.on_topology(x, t, onx, ony);
    }
    LightMesh M;
    if (!M.build(nn, t, x, in.sym_x, in.sym_y)) {
        out.why = "Tetrahedral mesh is not manifold (face shared by more than two tets)";
        return false;
    }
    std::vector<d3> stuffed = x;
    std::vector<uint8_t> contact(nn, IFEA_FREE);
    std::vector<d3> nrm = surface_normals(M, x);
    std::vector<double> hloc = local_lengths_of(M, t, x, in.h);
    Placer pl{in, M, t, hloc};
    for (int n = 0; n < nn; n++) {
        if (!M.surf[n]) continue;
        double cb = hf_clearance(in.die[0], x[n], 0), ctp = hf_clearance(in.die[1], x[n], in.gap), tolc = 0.12 * pl.tol(hloc[n]);
        if (cb < tolc && cb <= ctp) contact[n] = IFEA_BOTTOM_DIE;
        else if (ctp < tolc) contact[n] = IFEA_TOP_DIE;
        if (contact[n] != IFEA_FREE) {
            d3 q = hf_project(pl.surface(contact[n]), x[n], pl.offset(contact[n]), nullptr);
            x[n] = mk3(M.onx[n] ? 0 : q.x, M.ony[n] ? 0 : q.y, q.z);
        }
    }
    compensate_volume(in, M, t, x, contact);
    pl.improve_placement(x, contact, stuffed, nrm, 0.1);
    // thin sections one tet thick can be flattened by projection onto both dies: nodes of such tets go back to
    // their stuffed positions (never into a die) and are released
    for (int sweep = 0; sweep < 4; sweep++) {
        int reverted = 0;
        for (int e = 0; e < M.ne; e++) {
            if (pl.quality(x, e) >= 0.03) continue;
            for (int a = 0; a < 4; a++) {
                int n = t[4 * (size_t)e + a];
                if (eq3(x[n], stuffed[n])) continue;
                if (rmin(hf_clearance(in.die[0], stuffed[n], 0), hf_clearance(in.die[1], stuffed[n], in.gap)) < -0.05 * pl.tol(hloc[n]))
                    continue;
                x[n] = stuffed[n];
                contact[n] = IFEA_FREE;
                reverted++;
            }
        }
        if (reverted == 0) break;
    }
    pl.smooth_interior(x, 0.2, 10);
    pl.untangle_surface(x, contact, stuffed, 0.03, 6);
    pl.smooth_interior(x, 0.2, 4);
    out.q_new = min_quality(x, t);
    // a sound mesh, or one clearly better than the mesh in use (near closure the old one is worse still)
    if (out.q_new < 0.02 && !(out.q_new > 0.002 && out.q_new > out.q_old + 0.002)) {
        char buf[96];
        snprintf(buf, sizeof buf, "new mesh quality %.3f", out.q_new);
        out.why = buf;
        return false;
    }
    out.t_place = seconds_since(t0);
    t0 = std::chrono::steady_clock::now();
    int ne = M.ne;
    out.eps.assign(ne, 0); out.dmg.assign(ne, 0); out.sig.assign(ne, in.sig_ref); out.rate.assign(ne, 0); out.mean.assign(ne, 0);
    parallel_for(ne, [&](int e) {
        int f = locator.find_nearest(centroid4(x, t.data() + 4 * (size_t)e));
        if (f < 0) return;
        out.eps[e] = in.eps[f];
        out.dmg[e] = in.dmg[f];
        out.sig[e] = in.sig[f];
        out.rate[e] = in.rate[f];
        out.mean[e] = in.mean[f];
    });
    out.vg.assign(3 * (size_t)nn, 0);
    parallel_for(nn, [&](int n) { st3(out.vg.data(), n, locator.interpolate(x[n], in.vg)); });
    out.x.assign(3 * (size_t)nn, 0);
    for (int n = 0; n < nn; n++) st3(out.x.data(), n, x[n]);
    out.tets = std::move(t);
    out.on_x0 = M.onx;
    out.on_y0 = M.ony;
    out.contact = std::move(contact);
    out.t_remap = seconds_since(t0);
    return true;
}

}  // namespace ifea

// ------------------------------------------------------------------ C ABI (IsosurfaceStuffing.Stuff, TetRefiner.Refine)

struct ifea_tetmesh {
    std::vector<d3> x;
    std::vector<int32_t> t;
};

extern "C" {

ifea_status ifea_tetmesh_stuff(ifea_inside_fn inside, void *user, const double *lo3, const double *hi3, double h,
                               int32_t sym_x, int32_t sym_y, ifea_tetmesh **out)
{
    if (!inside || !lo3 || !hi3 || !out || !(h > 0)) return IFEA_INPUT_INVALID;
    *out = nullptr;
    try {
        auto *m = new ifea_tetmesh;
        ifea::stuff_uniform([&](d3 p) { return inside(p.x, p.y, p.z, user) != 0; }, mk3(lo3[0], lo3[1], lo3[2]),
                            mk3(hi3[0], hi3[1], hi3[2]), h, sym_x != 0, sym_y != 0, m->x, m->t, false);
        *out = m;
        return IFEA_OK;
    } catch (...) {
        return IFEA_CUDA_ERROR;
    }
}

ifea_status ifea_tetmesh_refine(ifea_tetmesh *m, ifea_size_fn size, void *user, int32_t max_nodes, int32_t *splits)
{
    if (!m || !size) return IFEA_INPUT_INVALID;
    try {
        int s = ifea::refine_tets(m->x, m->t, [&](d3 p) { return size(p.x, p.y, p.z, user); }, max_nodes);
        if (splits) *splits = s;
        return IFEA_OK;
    } catch (...) {
        return IFEA_CUDA_ERROR;
    }
}

int32_t ifea_tetmesh_node_count(const ifea_tetmesh *m) { return m ? (int32_t)m->x.size() : 0; }
int32_t ifea_tetmesh_tet_count(const ifea_tetmesh *m) { return m ? (int32_t)(m->t.size() / 4) : 0; }

ifea_status ifea_tetmesh_get(const ifea_tetmesh *m, double *x, int32_t *tets)
{
    if (!m || !x || !tets) return IFEA_INPUT_INVALID;
    for (size_t n = 0; n < m->x.size(); n++) st3(x, (int)n, m->x[n]);
    std::copy(m->t.begin(), m->t.end(), tets);
    return IFEA_OK;
}

void ifea_tetmesh_destroy(ifea_tetmesh *m) { delete m; }

}  // extern "C"

// ------------------------------------------------------------------ C ABI (RemeshCore on host arrays)

struct ifea_remesh_result {
    ifea::RemeshOutput out;
};

extern "C" {

ifea_status ifea_remesh_workpiece(const ifea_remesh_args *a, ifea_remesh_result **out)
{
    if (!a || !out || a->nn <= 0 || a->ne <= 0 || !a->x || !a->tets || !a->vg || !a->eps || !a->dmg || !a->sig ||
        !a->rate || !a->mean || !a->bottom.h || !a->top.h || (a->n_hot > 0 && !a->hot))
        return IFEA_INPUT_INVALID;
    *out = nullptr;
    try {
        ifea::RemeshInput in;
        in.nn = a->nn; in.ne = a->ne; in.x = a->x; in.tets = a->tets; in.vg = a->vg;
        in.eps = a->eps; in.dmg = a->dmg; in.sig = a->sig; in.rate = a->rate; in.mean = a->mean;
        const ifea_die_grid *g[2] = {&a->bottom, &a->top};
        for (int k = 0; k < 2; k++) {
            in.die[k].side = k; in.die[k].nx = g[k]->nx; in.die[k].ny = g[k]->ny;
            in.die[k].x0 = g[k]->x0; in.die[k].y0 = g[k]->y0; in.die[k].dx = g[k]->dx; in.die[k].h = g[k]->h;
        }
        in.gap = a->gap; in.h = a->h; in.vol_target = a->vol_target; in.sym_x = a->sym_x != 0; in.sym_y = a->sym_y != 0;
        in.recovery_pass = a->recovery_pass; in.refinement_levels = a->refinement_levels; in.max_nodes = a->max_nodes;
        in.sig_ref = a->sig_ref;
        for (int k = 0; k < a->n_hot; k++)
            in.hot.push_back({mk3(a->hot[4 * k], a->hot[4 * k + 1], a->hot[4 * k + 2]), (int)a->hot[4 * k + 3]});
        auto *r = new ifea_remesh_result;
        bool ok = ifea::remesh_workpiece(in, r->out);
        *out = r;
        return ok ? IFEA_OK : IFEA_MESH_DISTORTED;
    } catch (...) {
        return IFEA_CUDA_ERROR;
    }
}

int32_t ifea_remesh_node_count(const ifea_remesh_result *r) { return r ? (int32_t)(r->out.x.size() / 3) : 0; }
int32_t ifea_remesh_tet_count(const ifea_remesh_result *r) { return r ? (int32_t)(r->out.tets.size() / 4) : 0; }
const char *ifea_remesh_why(const ifea_remesh_result *r) { return r ? r->out.why.c_str() : ""; }

ifea_status ifea_remesh_get(const ifea_remesh_result *r, double *x, int32_t *tets, uint8_t *on_x0, uint8_t *on_y0,
                            uint8_t *contact, double *vg, double *eps, double *dmg, double *sig, double *rate,
                            double *mean)
{
    if (!r || r->out.tets.empty()) return IFEA_BAD_STATE;
    const ifea::RemeshOutput &o = r->out;
    auto cp = [](auto *dst, const auto &v) {
        if (dst) std::copy(v.begin(), v.end(), dst);
    };
    cp(x, o.x); cp(tets, o.tets); cp(on_x0, o.on_x0); cp(on_y0, o.on_y0); cp(contact, o.contact); cp(vg, o.vg);
    cp(eps, o.eps); cp(dmg, o.dmg); cp(sig, o.sig); cp(rate, o.rate); cp(mean, o.mean);
    return IFEA_OK;
}

void ifea_remesh_destroy(ifea_remesh_result *r) { delete r; }

}  // extern "C"
