// mesh3d.cpp — host-side tetrahedral topology and index maps (see mesh3d.h).
#include "mesh3d.h"

#include <algorithm>
#include <array>
#include <cmath>
#include <numeric>

namespace ifea {

namespace {
struct FaceRec {
    std::array<int32_t, 3> key;
    int32_t ins, a, b, c, owner;
};
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
    std::vector<FaceRec> fr(4 * (size_t)ne);
    for (int e = 0; e < ne; e++) {
        int a = tets[4 * e], b = tets[4 * e + 1], c = tets[4 * e + 2], d = tets[4 * e + 3];
        int f3[4][3] = {{a, c, b}, {a, b, d}, {a, d, c}, {b, c, d}};
        for (int f = 0; f < 4; f++) {
            FaceRec &r = fr[4 * e + f];
            r.a = f3[f][0];
            r.b = f3[f][1];
            r.c = f3[f][2];
            r.owner = e;
            r.ins = 4 * e + f;
            r.key = {r.a, r.b, r.c};
            std::sort(r.key.begin(), r.key.end());
        }
    }
    std::sort(fr.begin(), fr.end(), [](const FaceRec &p, const FaceRec &q) {
        return p.key != q.key ? p.key < q.key : p.ins < q.ins;
    });
    std::vector<FaceRec> bf;
    for (size_t i = 0; i < fr.size();) {
        size_t j = i + 1;
        while (j < fr.size() && fr[j].key == fr[i].key) j++;
        if (j - i > 2) return "Tetrahedral mesh is not manifold (face shared by more than two tets).";
        if (j - i == 1) bf.push_back(fr[i]);
        i = j;
    }
    std::sort(bf.begin(), bf.end(), [](const FaceRec &p, const FaceRec &q) { return p.ins < q.ins; });
    int nbf = (int)bf.size();
    bface.resize(3 * (size_t)nbf);
    bowner.resize(nbf);
    bsym.resize(nbf);
    is_surface.assign(nn, 0);
    for (int k = 0; k < nbf; k++) {
        bface[3 * k] = bf[k].a;
        bface[3 * k + 1] = bf[k].b;
        bface[3 * k + 2] = bf[k].c;
        bowner[k] = bf[k].owner;
        bsym[k] = (ox[bf[k].a] && ox[bf[k].b] && ox[bf[k].c]) || (oy[bf[k].a] && oy[bf[k].b] && oy[bf[k].c]);
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
    std::vector<std::vector<int32_t>> ring(nn);
    for (int n = 0; n < nn; n++) {
        auto &r = ring[n];
        for (int32_t q = nts[n]; q < nts[n + 1]; q++)
            for (int a = 0; a < 4; a++) r.push_back(tets[4 * ntl[q] + a]);
        std::sort(r.begin(), r.end());
        r.erase(std::unique(r.begin(), r.end()), r.end());
    }
    nbr_start.assign(nn + 1, 0);
    nbr.clear();
    std::vector<int32_t> buf;
    max_nbr = 0;
    for (int i = 0; i < nn; i++) {
        buf.clear();
        for (int32_t n : ring[i]) buf.insert(buf.end(), ring[n].begin(), ring[n].end());
        std::sort(buf.begin(), buf.end());
        buf.erase(std::unique(buf.begin(), buf.end()), buf.end());
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
    e_nbr.assign(16 * (size_t)ne, 0);
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) e_nbr[16 * e + 4 * a + b] = slot(tets[4 * e + b], tets[4 * e + a]);
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
    for (int n = 0; n < nn; n++) {
        int32_t base = (int32_t)g_node.size();
        for (int32_t q = nts[n]; q < nts[n + 1]; q++) {
            int e = ntl[q];
            for (int a = 0; a < 4; a++) {
                int m = tets[4 * e + a];
                int32_t idx = -1;
                for (int32_t p = base; p < (int32_t)g_node.size(); p++)
                    if (g_node[p] == m) { idx = p; break; }
                if (idx < 0) {
                    idx = (int32_t)g_node.size();
                    g_node.push_back(m);
                }
                gslot[4 * (size_t)q + a] = idx;
            }
        }
        g_start[n + 1] = (int32_t)g_node.size();
    }
    // K_vol gather lists
    kv_start.assign(nn + 1, 0);
    kv_n.clear();
    kv_pj.clear();
    kv_kstart.clear();
    kv_k.clear();
    for (int j = 0; j < nn; j++) {
        for (int32_t n : ring[j]) {
            int32_t pj = -1;
            for (int32_t p = g_start[n]; p < g_start[n + 1]; p++)
                if (g_node[p] == j) { pj = p; break; }
            if (pj < 0) return "internal error: patch does not contain its ring node";
            kv_n.push_back(n);
            kv_pj.push_back(pj);
            kv_kstart.push_back((int32_t)kv_k.size());
            for (int32_t p = g_start[n]; p < g_start[n + 1]; p++) kv_k.push_back(slot(j, g_node[p]));
        }
        kv_start[j + 1] = (int32_t)kv_n.size();
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
