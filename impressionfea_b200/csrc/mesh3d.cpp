// mesh3d.cpp — host-side tetrahedral topology and index maps (see mesh3d.h).
#include "mesh3d.h"

#include "host_par.h"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <numeric>

namespace ifea {

namespace {
struct FaceKey {
    int32_t k0, k1, k2, ins;  // sorted node triple, insertion index 4 e + f
};

// the four faces of a tet, in the reference's order
inline void tet_face(const int32_t *tv, int f, int32_t &a, int32_t &b, int32_t &c)
{
    static const int8_t F[4][3] = {{0, 2, 1}, {0, 1, 3}, {0, 3, 2}, {1, 2, 3}};
    a = tv[F[f][0]], b = tv[F[f][1]], c = tv[F[f][2]];
}
}  // namespace

std::string TetTopology::build(int nn_, int ne_, const double *x, const int32_t *t, const uint8_t *ox,
                               const uint8_t *oy)
{
    (void)x;
    nn = nn_;
    ne = ne_;
    ndof = 3 * nn;
    if (nn <= 0 || ne <= 0) return "The workpiece produced an empty mesh; reduce the element size h.";
    tets.assign(t, t + 4 * (size_t)ne);
    on_x0.assign(ox, ox + nn);
    on_y0.assign(oy, oy + nn);
    for (int32_t v : tets)
        if (v < 0 || v >= nn) return "A tetrahedron references a node outside the mesh.";

    // node -> tet CSR (TetMesh.cs:18-29)
    nts.assign(nn + 1, 0);
    for (int32_t v : tets) nts[v + 1]++;
    for (int i = 0; i < nn; i++) nts[i + 1] += nts[i];
    ntl.assign(4 * (size_t)ne, 0);
    ntl_local.assign(4 * (size_t)ne, 0);
    {
        std::vector<int32_t> fill(nts.begin(), nts.end() - 1);
        for (int e = 0; e < ne; e++)
            for (int a = 0; a < 4; a++) {
                int32_t q = fill[tets[4 * e + a]]++;
                ntl[q] = e;
                ntl_local[q] = (int8_t)a;
            }
    }

    // boundary faces in the Dictionary's insertion order (TetMesh.cs:31-64)
    // a face is on the boundary when no other face has its node set; kept in insertion order. Faces are bucketed
    // by their smallest node; within a bucket, equal (second, third) node pairs form the groups.
    std::vector<int32_t> bf;
    {
        std::vector<int32_t> fstart(nn + 1, 0);
        std::vector<FaceKey> fr(4 * (size_t)ne);
        for (int e = 0; e < ne; e++)
            for (int f = 0; f < 4; f++) {
                int32_t a, b, c;
                tet_face(&tets[4 * (size_t)e], f, a, b, c);
                if (a > b) std::swap(a, b);
                if (b > c) std::swap(b, c);
                if (a > b) std::swap(a, b);
                fr[4 * (size_t)e + f] = {a, b, c, 4 * e + f};
                fstart[a + 1]++;
            }
        for (int i = 0; i < nn; i++) fstart[i + 1] += fstart[i];
        std::vector<FaceKey> byk(fr.size());
        {
            std::vector<int32_t> fill(fstart.begin(), fstart.end() - 1);
            for (const FaceKey &k : fr) byk[fill[k.k0]++] = k;
        }
        std::vector<std::vector<int32_t>> part(par_chunk_count(nn));
        std::atomic<bool> bad{false};
        par_chunks(nn, [&](int t, int a0, int a1) {
            std::vector<FaceKey> g;
            for (int a = a0; a < a1; a++) {
                g.assign(byk.begin() + fstart[a], byk.begin() + fstart[a + 1]);
                std::sort(g.begin(), g.end(), [](const FaceKey &p, const FaceKey &q) {
                    return p.k1 != q.k1 ? p.k1 < q.k1 : p.k2 < q.k2;
                });
                for (size_t i = 0; i < g.size();) {
                    size_t j = i + 1;
                    while (j < g.size() && g[j].k1 == g[i].k1 && g[j].k2 == g[i].k2) j++;
                    if (j - i == 1) part[t].push_back(g[i].ins);
                    else if (j - i > 2) bad = true;
                    i = j;
                }
            }
        });
        if (bad) return "Tetrahedral mesh is not manifold (face shared by more than two tets).";
        for (auto &v : part) bf.insert(bf.end(), v.begin(), v.end());
    }
    std::sort(bf.begin(), bf.end());
    int nbf = (int)bf.size();
    bface.resize(3 * (size_t)nbf);
    bowner.resize(nbf);
    bsym.resize(nbf);
    is_surface.assign(nn, 0);
    for (int k = 0; k < nbf; k++) {
        int32_t a, b, c;
        tet_face(&tets[4 * (size_t)(bf[k] / 4)], bf[k] % 4, a, b, c);
        bface[3 * k] = a;
        bface[3 * k + 1] = b;
        bface[3 * k + 2] = c;
        bowner[k] = bf[k] / 4;
        bsym[k] = (ox[a] && ox[b] && ox[c]) || (oy[a] && oy[b] && oy[c]);
        if (!bsym[k])
            for (int q = 0; q < 3; q++) is_surface[bface[3 * k + q]] = 1;
    }
    // node -> non-symmetry faces in face order
    nfs.assign(nn + 1, 0);
    for (int k = 0; k < nbf; k++)
        if (!bsym[k])
            for (int q = 0; q < 3; q++) nfs[bface[3 * k + q] + 1]++;
    for (int i = 0; i < nn; i++) nfs[i + 1] += nfs[i];
    nfl.assign(nfs[nn], 0);
    {
        std::vector<int32_t> fill(nfs.begin(), nfs.end() - 1);
        for (int k = 0; k < nbf; k++)
            if (!bsym[k])
                for (int q = 0; q < 3; q++) nfl[fill[bface[3 * k + q]]++] = k;
    }

    // patches (one ring, sorted) and the two-ring pattern, per chunk of nodes, joined in node order
    const int ncx = par_chunk_count(nn);
    std::vector<int32_t> ring_start(nn + 1, 0), ring_list;
    {
        std::vector<std::vector<int32_t>> part(ncx);
        par_chunks(nn, [&](int t, int n0, int n1) {
            std::vector<int32_t> mark(nn, -1);
            auto &out = part[t];
            for (int n = n0; n < n1; n++) {
                size_t b = out.size();
                for (int32_t q = nts[n]; q < nts[n + 1]; q++)
                    for (int a = 0; a < 4; a++) {
                        int32_t v = tets[4 * ntl[q] + a];
                        if (mark[v] != n) {
                            mark[v] = n;
                            out.push_back(v);
                        }
                    }
                std::sort(out.begin() + b, out.end());
                ring_start[n + 1] = (int32_t)(out.size() - b);
            }
        });
        for (int i = 0; i < nn; i++) ring_start[i + 1] += ring_start[i];
        ring_list.reserve(ring_start[nn]);
        for (auto &v : part) ring_list.insert(ring_list.end(), v.begin(), v.end());
    }
    struct Span {
        const int32_t *b, *e;
        const int32_t *begin() const { return b; }
        const int32_t *end() const { return e; }
        size_t size() const { return (size_t)(e - b); }
    };
    auto ring = [&](int i) { return Span{ring_list.data() + ring_start[i], ring_list.data() + ring_start[i + 1]}; };
    nbr_start.assign(nn + 1, 0);
    nbr.clear();
    {
        std::vector<std::vector<int32_t>> part(ncx);
        std::vector<int32_t> part_max(ncx, 0);
        par_chunks(nn, [&](int t, int i0, int i1) {
            std::vector<int32_t> mark(nn, -1), buf;
            std::vector<uint64_t> bits;  // ascending order of a node set through a bitmap over its index window
            auto &out = part[t];
            for (int i = i0; i < i1; i++) {
                buf.clear();
                int32_t lo = nn, hi = -1;
                for (int32_t n : ring(i))
                    for (int32_t q : ring(n))
                        if (mark[q] != i) {
                            mark[q] = i;
                            buf.push_back(q);
                            lo = std::min(lo, q);
                            hi = std::max(hi, q);
                        }
                if (hi - lo < (1 << 16)) {
                    size_t nw = (size_t)(hi - lo) / 64 + 1;
                    if (bits.size() < nw) bits.resize(nw, 0);
                    for (int32_t q : buf) bits[(q - lo) >> 6] |= 1ull << ((q - lo) & 63);
                    size_t k = 0;
                    for (size_t w = 0; w < nw; w++)
                        for (uint64_t v = bits[w]; v; v &= v - 1) buf[k++] = lo + (int32_t)(64 * w) + __builtin_ctzll(v);
                    std::fill(bits.begin(), bits.begin() + nw, 0);
                } else {
                    std::sort(buf.begin(), buf.end());
                }
                out.insert(out.end(), buf.begin(), buf.end());
                nbr_start[i + 1] = (int32_t)buf.size();
                part_max[t] = std::max<int32_t>(part_max[t], (int32_t)buf.size());
            }
        });
        size_t total = 0;
        for (auto &v : part) total += v.size();
        if (total * 9 > (size_t)INT32_MAX) return "Sparse pattern exceeds 32-bit indexing.";
        for (int i = 0; i < nn; i++) nbr_start[i + 1] += nbr_start[i];
        nbr.reserve(total);
        for (auto &v : part) nbr.insert(nbr.end(), v.begin(), v.end());
        max_nbr = *std::max_element(part_max.begin(), part_max.end());
    }
    col_ptr.assign(ndof + 1, 0);
    for (int j = 0; j < nn; j++)
        for (int c = 0; c < 3; c++) col_ptr[3 * j + c + 1] = col_ptr[3 * j + c] + 3 * (nbr_start[j + 1] - nbr_start[j]);
    nnz = col_ptr[ndof];
    if ((int64_t)nbr.size() * 9 > INT32_MAX) return "Sparse pattern exceeds 32-bit indexing.";
    row_idx.resize(nnz);
    par_chunks(nn, [&](int, int j0, int j1) {
        for (int j = j0; j < j1; j++)
            for (int c = 0; c < 3; c++) {
                int64_t p = col_ptr[3 * j + c];
                for (int32_t k = nbr_start[j]; k < nbr_start[j + 1]; k++) {
                    int i = nbr[k];
                    row_idx[p++] = 3 * i;
                    row_idx[p++] = 3 * i + 1;
                    row_idx[p++] = 3 * i + 2;
                }
            }
    });
    auto slot = [&](int j, int i) {
        const int32_t *b = nbr.data() + nbr_start[j], *e = nbr.data() + nbr_start[j + 1];
        const int32_t *it = std::lower_bound(b, e, i);
        return (it != e && *it == i) ? (int32_t)(it - b) : -1;
    };
    // slot of node i in nbr[j] by a position map of nbr[j] (-1 when absent), column node by column node; node j
    // is corner b of each of its tets e exactly once, so the chunks write disjoint entries
    auto fill_pos = [&](std::vector<int32_t> &pos, int j, bool on) {
        for (int32_t k = nbr_start[j]; k < nbr_start[j + 1]; k++) pos[nbr[k]] = on ? k - nbr_start[j] : -1;
    };
    e_nbr.assign(16 * (size_t)ne, 0);
    par_chunks(nn, [&](int, int j0, int j1) {
        std::vector<int32_t> pos(nn, -1);
        for (int j = j0; j < j1; j++) {
            fill_pos(pos, j, true);
            for (int32_t q = nts[j]; q < nts[j + 1]; q++) {
                int e = ntl[q], b = ntl_local[q];
                for (int a = 0; a < 4; a++) e_nbr[16 * (size_t)e + 4 * a + b] = pos[tets[4 * e + a]];
            }
            fill_pos(pos, j, false);
        }
    });
    qk.assign(16 * (size_t)ne, 0);
    diag_slot.assign(ndof, 0);
    par_chunks(nn, [&](int, int j0, int j1) {
        for (int j = j0; j < j1; j++) {
            for (int32_t q = nts[j]; q < nts[j + 1]; q++) {
                int e = ntl[q], b = ntl_local[q];
                for (int a = 0; a < 4; a++) qk[4 * (size_t)q + a] = e_nbr[16 * e + 4 * a + b];
            }
            int k = slot(j, j);
            for (int c = 0; c < 3; c++) diag_slot[3 * j + c] = col_ptr[3 * j + c] + 3 * k + c;
        }
    });

    // ANP patches in first-encounter order (BuildAnp :774-795), per chunk of nodes: positions local to the
    // chunk, shifted by the chunk's offset once the chunks' sizes are known
    g_start.assign(nn + 1, 0);
    g_node.clear();
    gslot.assign(16 * (size_t)ne, 0);
    {
        std::vector<std::vector<int32_t>> part(ncx);
        par_chunks(nn, [&](int t, int n0, int n1) {
            std::vector<int32_t> mark(nn, -1), at(nn);
            auto &out = part[t];
            for (int n = n0; n < n1; n++) {
                for (int32_t q = nts[n]; q < nts[n + 1]; q++) {
                    int e = ntl[q];
                    for (int a = 0; a < 4; a++) {
                        int m = tets[4 * e + a];
                        if (mark[m] != n) {
                            mark[m] = n;
                            at[m] = (int32_t)out.size();
                            out.push_back(m);
                        }
                        gslot[4 * (size_t)q + a] = at[m];
                    }
                }
                g_start[n + 1] = (int32_t)out.size();
            }
        });
        std::vector<int32_t> off(ncx, 0);
        for (int t = 1; t < ncx; t++) off[t] = off[t - 1] + (int32_t)part[t - 1].size();
        par_chunks(nn, [&](int t, int n0, int n1) {
            for (int n = n0; n < n1; n++) {
                g_start[n + 1] += off[t];
                for (int64_t q = 4 * (int64_t)nts[n]; q < 4 * (int64_t)nts[n + 1]; q++) gslot[q] += off[t];
            }
        });
        for (auto &v : part) g_node.insert(g_node.end(), v.begin(), v.end());
    }
    // K_vol gather lists
    kv_start.assign(nn + 1, 0);
    for (int j = 0; j < nn; j++) kv_start[j + 1] = kv_start[j] + (int32_t)ring(j).size();
    kv_n.resize(kv_start[nn]);
    kv_pj.resize(kv_start[nn]);
    kv_kstart.resize(kv_start[nn]);
    std::vector<int32_t> kstart(nn + 1, 0);
    par_chunks(nn, [&](int, int j0, int j1) {
        for (int j = j0; j < j1; j++) {
            int32_t c = 0;
            for (int32_t n : ring(j)) c += g_start[n + 1] - g_start[n];
            kstart[j + 1] = c;
        }
    });
    for (int j = 0; j < nn; j++) kstart[j + 1] += kstart[j];
    kv_k.resize(kstart[nn]);
    std::atomic<bool> lost{false};
    par_chunks(nn, [&](int, int j0, int j1) {
        std::vector<int32_t> pos(nn, -1);
        for (int j = j0; j < j1; j++) {
            fill_pos(pos, j, true);
            int32_t r = kv_start[j], kk = kstart[j];
            for (int32_t n : ring(j)) {
                int32_t pj = -1;
                for (int32_t p = g_start[n]; p < g_start[n + 1]; p++)
                    if (g_node[p] == j) { pj = p; break; }
                if (pj < 0) lost = true;
                kv_n[r] = n;
                kv_pj[r] = pj;
                kv_kstart[r++] = kk;
                for (int32_t p = g_start[n]; p < g_start[n + 1]; p++) kv_k[kk++] = pos[g_node[p]];
            }
            fill_pos(pos, j, false);
        }
    });
    if (lost) return "internal error: patch does not contain its ring node";
    return "";
}

std::vector<double> local_lengths(const TetTopology &t, const double *x, double h)
{
    std::vector<double> sum(t.nn, 0.0);
    std::vector<int> cnt(t.nn, 0);
    for (int e = 0; e < t.ne; e++)
        for (int a = 0; a < 4; a++)
            for (int b = a + 1; b < 4; b++) {
                int i = t.tets[4 * e + a], j = t.tets[4 * e + b];
                double dx = x[3 * i] - x[3 * j], dy = x[3 * i + 1] - x[3 * j + 1], dz = x[3 * i + 2] - x[3 * j + 2];
                double l = std::sqrt(dx * dx + dy * dy + dz * dz);
                sum[i] += l;
                sum[j] += l;
                cnt[i]++;
                cnt[j]++;
            }
    for (int n = 0; n < t.nn; n++) {
        if (cnt[n] > 0) {
            double m = sum[n] / cnt[n];
            sum[n] = (m != m) ? m : (m < h ? m : h);
        } else {
            sum[n] = h;
        }
    }
    return sum;
}

}  // namespace ifea
