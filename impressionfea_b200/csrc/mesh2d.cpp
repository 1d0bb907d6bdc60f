// mesh2d.cpp — 2D quad topology: structured mesh, RCM equation numbering with the reference's tie-breaking
// (HashSet insertion order, stable OrderBy), boundary loop, and the band gather maps.
#include "mesh2d.h"

#include <algorithm>
#include <map>
#include <queue>

namespace ifea {

namespace {

// Peripheral (QuadMesh.cs:143-171): repeated BFS to the last-dequeued node while the depth grows (<= 4 passes).
int peripheral(int start, const std::vector<std::vector<int32_t>> &adj)
{
    int node = start, best_depth = -1;
    std::vector<int> depth(adj.size());
    for (int pass = 0; pass < 4; pass++) {
        std::fill(depth.begin(), depth.end(), -1);
        std::queue<int> q;
        q.push(node);
        depth[node] = 0;
        int last = node;
        while (!q.empty()) {
            int n = q.front();
            q.pop();
            last = n;
            for (int m : adj[n]) {
                if (depth[m] >= 0) continue;
                depth[m] = depth[n] + 1;
                q.push(m);
            }
        }
        if (depth[last] <= best_depth) break;
        best_depth = depth[last];
        node = last;
    }
    return node;
}

}  // namespace

std::string QuadTopology::build_structured(int nx, int ny, double r, double y0, double h, std::vector<double> &x)
{
    if (nx < 1 || ny < 1) return "invalid structured mesh size";
    nn = (nx + 1) * (ny + 1);
    ne = nx * ny;
    ndof = 2 * nn;
    x.assign(2 * (size_t)nn, 0.0);
    is_axis.assign(nn, 0);
    for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
            int n = j * (nx + 1) + i;
            x[2 * n] = r * i / nx;
            x[2 * n + 1] = y0 + h * j / ny;
            is_axis[n] = i == 0;
        }
    conn.clear();
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            conn.push_back(j * (nx + 1) + i);
            conn.push_back(j * (nx + 1) + i + 1);
            conn.push_back((j + 1) * (nx + 1) + i + 1);
            conn.push_back((j + 1) * (nx + 1) + i);
        }
    // adjacency in HashSet insertion order
    std::vector<std::vector<int32_t>> adj(nn);
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++)
            for (int b = 0; b < 4; b++) {
                if (a == b) continue;
                auto &l = adj[conn[4 * e + a]];
                int m = conn[4 * e + b];
                if (std::find(l.begin(), l.end(), m) == l.end()) l.push_back(m);
            }
    std::vector<int32_t> order;
    order.reserve(nn);
    std::vector<uint8_t> seen(nn, 0);
    while ((int)order.size() < nn) {
        int start = -1;
        for (int n = 0; n < nn; n++)
            if (!seen[n] && (start < 0 || adj[n].size() < adj[start].size())) start = n;
        start = peripheral(start, adj);
        std::queue<int> q;
        q.push(start);
        seen[start] = 1;
        while (!q.empty()) {
            int n = q.front();
            q.pop();
            order.push_back(n);
            std::vector<int32_t> cand;
            for (int m : adj[n])
                if (!seen[m]) cand.push_back(m);
            std::stable_sort(cand.begin(), cand.end(), [&](int a, int b) { return adj[a].size() < adj[b].size(); });
            for (int m : cand) {
                seen[m] = 1;
                q.push(m);
            }
        }
    }
    eq.assign(nn, 0);
    for (int k = 0; k < nn; k++) eq[order[nn - 1 - k]] = k;
    int band = 1;
    for (int e = 0; e < ne; e++) {
        int lo = INT32_MAX, hi = INT32_MIN;
        for (int a = 0; a < 4; a++) {
            lo = std::min(lo, eq[conn[4 * e + a]]);
            hi = std::max(hi, eq[conn[4 * e + a]]);
        }
        band = std::max(band, 2 * (hi - lo) + 1);
    }
    half_band = std::min(band, ndof - 1);  // SymmetricBandMatrix clamps to n - 1

    // boundary loop (TraceBoundary)
    std::map<std::pair<int, int>, int> cnt;
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++) {
            int p = conn[4 * e + a], q = conn[4 * e + (a + 1) % 4];
            cnt[{std::min(p, q), std::max(p, q)}]++;
        }
    std::vector<int32_t> next_to(nn, -1), next_el(nn, -1), keys;
    for (int e = 0; e < ne; e++)
        for (int a = 0; a < 4; a++) {
            int p = conn[4 * e + a], q = conn[4 * e + (a + 1) % 4];
            if (cnt[{std::min(p, q), std::max(p, q)}] != 1) continue;
            if (next_to[p] >= 0) return "Mesh boundary is not a simple closed loop (pinched node).";
            next_to[p] = q;
            next_el[p] = e;
            keys.push_back(p);
        }
    if (keys.empty()) return "Mesh has no boundary.";
    int start = keys[0];
    for (int n : keys)
        if (is_axis[n] && (!is_axis[start] || n < start)) start = n;
    loop.clear();
    loop_owner.clear();
    int cur = start;
    do {
        loop.push_back(cur);
        loop_owner.push_back(next_el[cur]);
        cur = next_to[cur];
        if (loop.size() > keys.size() || cur < 0) return "Mesh boundary consists of several loops.";
    } while (cur != start);
    if (loop.size() != keys.size()) return "Mesh boundary consists of several loops.";
    nloop = (int)loop.size();
    node_edge.assign(2 * (size_t)nn, -1);
    for (int k = 0; k < nloop; k++) {
        int a = loop[k], b = loop[(k + 1) % nloop];
        for (int n : {a, b}) {
            int32_t *slot = &node_edge[2 * (size_t)n];
            if (slot[0] < 0) slot[0] = k;
            else slot[1] = k;
        }
    }

    // band gather maps in element order
    struct C { int64_t cell; int32_t src; };
    std::vector<C> cc;
    cc.reserve(36 * (size_t)ne);
    std::vector<std::pair<int32_t, int32_t>> dd;
    dd.reserve(8 * (size_t)ne);
    for (int e = 0; e < ne; e++) {
        int edof[8];
        for (int a = 0; a < 4; a++) {
            edof[2 * a] = 2 * eq[conn[4 * e + a]];
            edof[2 * a + 1] = edof[2 * a] + 1;
        }
        for (int p = 0; p < 8; p++) {
            dd.push_back({edof[p], 8 * e + p});
            for (int q = 0; q <= p; q++) {
                int i = edof[p], j = edof[q];
                if (j > i) std::swap(i, j);
                if (i - j > half_band) return "Element entry lies outside the band.";
                cc.push_back({band_index(i, j), 64 * e + 8 * p + q});
            }
        }
    }
    std::stable_sort(cc.begin(), cc.end(), [](const C &a, const C &b) { return a.cell < b.cell; });
    cell_ptr.assign(1, 0);
    cell_idx.clear();
    cell_src.clear();
    for (size_t k = 0; k < cc.size(); k++) {
        if (k == 0 || cc[k].cell != cc[k - 1].cell) {
            if (k) cell_ptr.push_back((int32_t)cell_src.size());
            cell_idx.push_back((int32_t)cc[k].cell);
        }
        cell_src.push_back(cc[k].src);
    }
    cell_ptr.push_back((int32_t)cell_src.size());
    std::stable_sort(dd.begin(), dd.end(), [](const auto &a, const auto &b) { return a.first < b.first; });
    dof_ptr.assign(ndof + 1, 0);
    dof_src.clear();
    for (auto &p : dd) {
        dof_ptr[p.first + 1]++;
        dof_src.push_back(p.second);
    }
    for (int d = 0; d < ndof; d++) dof_ptr[d + 1] += dof_ptr[d];
    return "";
}

}  // namespace ifea
