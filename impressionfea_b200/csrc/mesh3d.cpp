// mesh3d.cpp — host-side tetrahedral topology and index maps (see mesh3d.h).
#include "mesh3d.h"

#include <algorithm>
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
    // a face is on the boundary when no other face has its node set; kept in insertion order
    std::vector<FaceKey> fr(4 * (size_t)ne);
    for (int e = 0; e < ne; e++)
        for (int f = 0; f < 4; f++) {
            int32_t a, b, c;
            tet_face(&tets[4 * (size_t)e], f, a, b, c);
            if (a > b) std::swap(a, b);
            if (b > c) std::swap(b, c);
            if (a > b) std::swap(a, b);
            fr[4 * (size_t)e + f] = {a, b, c, 4 * e + f};
        }
    // only the size of each group of equal node sets matters: one (boundary), two (interior) or more (error)
    std::vector<int32_t> bf;
    auto group = [&](size_t i, size_t j) {
        if (j - i == 1) bf.push_back(fr[i].ins);
        return j - i <= 2;
    };
    if (nn < (1 << 21)) {  // node triples packed into one key of 3 x bits(nn) bits, LSD radix sort by 11 bits
        int nbits = 1;
        while ((1 << nbits) < nn) nbits++;
        std::vector<uint64_t> key(fr.size()), key2(fr.size());
        std::vector<int32_t> ord(fr.size()), ord2(fr.size());
        for (size_t i = 0; i < fr.size(); i++) {
            key[i] = ((uint64_t)fr[i].k0 << (2 * nbits)) | ((uint64_t)fr[i].k1 << nbits) | (uint64_t)fr[i].k2;
            ord[i] = (int32_t)i;
        }
        for (int sh = 0; sh < 3 * nbits; sh += 11) {
            size_t cnt[2049] = {0};
            for (uint64_t k : key) cnt[((k >> sh) & 2047) + 1]++;
            for (int b = 0; b < 2048; b++) cnt[b + 1] += cnt[b];
            for (size_t i = 0; i < key.size(); i++) {
                size_t d = cnt[(key[i] >> sh) & 2047]++;
                key2[d] = key[i];
                ord2[d] = ord[i];
            }
            key.swap(key2);
            ord.swap(ord2);
        }
        std::vector<FaceKey> sorted(fr.size());
        for (size_t i = 0; i < fr.size(); i++) sorted[i] = fr[ord[i]];
        fr.swap(sorted);
    } else {
        std::sort(fr.begin(), fr.end(), [](const FaceKey &p, const FaceKey &q) {
            if (p.k0 != q.k0) return p.k0 < q.k0;
            if (p.k1 != q.k1) return p.k1 < q.k1;
            return p.k2 < q.k2;
        });
    }
    for (size_t i = 0; i < fr.size();) {
        size_t j = i + 1;
        while (j < fr.size() && fr[j].k0 == fr[i].k0 && fr[j].k1 == fr[i].k1 && fr[j].k2 == fr[i].k2) j++;
        if (!group(i, j)) return "Tetrahedral mesh is not manifold (face shared by more than two tets).";
        i = j;
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

    // patches (one ring, sorted) and the two-ring pattern
    std::vector<int32_t> ring_start(nn + 1, 0), ring_list, mark(nn, -1);
    ring_list.reserve(16 * (size_t)nn);
    for (int n = 0; n < nn; n++) {
        for (int32_t q = nts[n]; q < nts[n + 1]; q++)
            for (int a = 0; a < 4; a++) {
                int32_t v = tets[4 * ntl[q] + a];
                if (mark[v] != n) {
                    mark[v] = n;
                    ring_list.push_back(v);
                }
            }
        std::sort(ring_list.begin() + ring_start[n], ring_list.end());
        ring_start[n + 1] = (int32_t)ring_list.size();
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
    std::vector<int32_t> buf;
    std::fill(mark.begin(), mark.end(), -1);
    std::vector<uint64_t> bits;  // ascending order of a node set through a bitmap over its index window
    max_nbr = 0;
    for (int i = 0; i < nn; i++) {
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
        nbr.insert(nbr.end(), buf.begin(), buf.end());
        nbr_start[i + 1] = (int32_t)nbr.size();
        max_nbr = std::max<int32_t>(max_nbr, (int32_t)buf.size());
    }
    col_ptr.assign(ndof + 1, 0);
    for (int j = 0; j < nn; j++)
        for (int c = 0; c < 3; c++) col_ptr[3 * j + c + 1] = col_ptr[3 * j + c] + 3 * (nbr_start[j + 1] - nbr_start[j]);
    nnz = col_ptr[ndof];
    if ((int64_t)nbr.size() * 9 > INT32_MAX) return "Sparse pattern exceeds 32-bit indexing.";
    row_idx.assign(nnz, 0);
    for (int j = 0; j < nn; j++)
        for (int c = 0; c < 3; c++) {
            int64_t p = col_ptr[3 * j + c];
            for (int32_t k = nbr_start[j]; k < nbr_start[j + 1]; k++) {
                int i = nbr[k];
                row_idx[p++] = 3 * i;
                row_idx[p++] = 3 * i + 1;
                row_idx[p++] = 3 * i + 2;
            }
        }
    auto slot = [&](int j, int i) {
        const int32_t *b = nbr.data() + nbr_start[j], *e = nbr.data() + nbr_start[j + 1];
        const int32_t *it = std::lower_bound(b, e, i);
        return (it != e && *it == i) ? (int32_t)(it - b) : -1;
    };
    // slot of node i in nbr[j] by a position map of nbr[j] (-1 when absent), column node by column node
    std::vector<int32_t> pos(nn, -1);
    auto fill_pos = [&](int j, bool on) {
        for (int32_t k = nbr_start[j]; k < nbr_start[j + 1]; k++) pos[nbr[k]] = on ? k - nbr_start[j] : -1;
    };
    e_nbr.assign(16 * (size_t)ne, 0);
    for (int j = 0; j < nn; j++) {
        fill_pos(j, true);
        for (int32_t q = nts[j]; q < nts[j + 1]; q++) {
            int e = ntl[q], b = ntl_local[q];
            for (int a = 0; a < 4; a++) e_nbr[16 * (size_t)e + 4 * a + b] = pos[tets[4 * e + a]];
        }
        fill_pos(j, false);
    }
    qk.assign(16 * (size_t)ne, 0);
    for (int j = 0; j < nn; j++)
        for (int32_t q = nts[j]; q < nts[j + 1]; q++) {
            int e = ntl[q], b = ntl_local[q];
            for (int a = 0; a < 4; a++) qk[4 * (size_t)q + a] = e_nbr[16 * e + 4 * a + b];
        }
    diag_slot.assign(ndof, 0);
    for (int n = 0; n < nn; n++) {
        int k = slot(n, n);
        for (int c = 0; c < 3; c++) diag_slot[3 * n + c] = col_ptr[3 * n + c] + 3 * k + c;
    }

    // ANP patches in first-encounter order (BuildAnp :774-795)
    g_start.assign(nn + 1, 0);
    g_node.clear();
    gslot.assign(16 * (size_t)ne, 0);
    std::fill(mark.begin(), mark.end(), -1);
    std::vector<int32_t> at(nn);  // position of a node in the patch being built (valid where mark == n)
    for (int n = 0; n < nn; n++) {
        for (int32_t q = nts[n]; q < nts[n + 1]; q++) {
            int e = ntl[q];
            for (int a = 0; a < 4; a++) {
                int m = tets[4 * e + a];
                if (mark[m] != n) {
                    mark[m] = n;
                    at[m] = (int32_t)g_node.size();
                    g_node.push_back(m);
                }
                gslot[4 * (size_t)q + a] = at[m];
            }
        }
        g_start[n + 1] = (int32_t)g_node.size();
    }
    // K_vol gather lists
    kv_start.assign(nn + 1, 0);
    for (int j = 0; j < nn; j++) kv_start[j + 1] = kv_start[j] + (int32_t)ring(j).size();
    kv_n.resize(kv_start[nn]);
    kv_pj.resize(kv_start[nn]);
    kv_kstart.resize(kv_start[nn]);
    {
        size_t nk = 0;
        for (int j = 0; j < nn; j++)
            for (int32_t n : ring(j)) nk += g_start[n + 1] - g_start[n];
        kv_k.resize(nk);
    }
    int32_t kk = 0;
    for (int j = 0; j < nn; j++) {
        fill_pos(j, true);
        int32_t r = kv_start[j];
        for (int32_t n : ring(j)) {
            int32_t pj = -1;
            for (int32_t p = g_start[n]; p < g_start[n + 1]; p++)
                if (g_node[p] == j) { pj = p; break; }
            if (pj < 0) return "internal error: patch does not contain its ring node";
            kv_n[r] = n;
            kv_pj[r] = pj;
            kv_kstart[r++] = kk;
            for (int32_t p = g_start[n]; p < g_start[n + 1]; p++) kv_k[kk++] = pos[g_node[p]];
        }
        fill_pos(j, false);
    }
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
