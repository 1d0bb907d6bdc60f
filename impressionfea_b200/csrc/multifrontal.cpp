// multifrontal.cpp — symbolic analysis of the GPU multifrontal Cholesky (see multifrontal.h).
#include "multifrontal.h"

#include "host_par.h"

#include <cusolverSp.h>
#include <cusparse.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <chrono>
#include <climits>
#include <functional>
#include <memory>
#include <numeric>
#include <thread>

namespace ifea {

namespace {
// Nested dissection by coordinate cuts. A set of more than kLeaf nodes is cut by a plane normal to one axis at
// 40-60 % of its nodes; among the three axes and five positions the cut whose smaller one-sided boundary (the
// nodes of one side with a neighbour on the other) is smallest, with a penalty for imbalance, wins, and that
// boundary is the separator. On the kCoverDepth top levels the separator is then reduced to a minimum vertex
// cover of the edges across the cut (maximum bipartite matching and König's theorem) when that is smaller. The
// separator is numbered after both halves, which recurse; leaves keep their order. A node can only neighbour the
// other side from within reach[ax] of the plane (its longest edge along that axis), so the boundary scans cover a
// slab of the sorted set, not all of it.
// The two halves of a cut share no node, so from depth 1 to kParDepth - 1 one of them recurses on a new host
// thread; every subtree writes its own fragment of the reverse order and the fragments are joined in the
// sequential order, so the result does not depend on the threads. Set stamps come from one atomic counter, so
// that no two sets (of any thread) share a stamp.
// A set mark read by one thread while another writes it (a neighbour in the other half): relaxed atomic access.
struct SetMark {
    std::atomic<int32_t> v{0};
    operator int32_t() const { return v.load(std::memory_order_relaxed); }
    SetMark &operator=(int32_t x)
    {
        v.store(x, std::memory_order_relaxed);
        return *this;
    }
};

struct CoordNd {
    static constexpr int kLeaf = 32, kCoverDepth = 2, kParDepth = 4;
    int nb;
    const int *gp, *gi;
    const double *x;
    std::unique_ptr<SetMark[]> mark;
    std::vector<int32_t> loc;  // position of a node in the V side of the cover being built (-1 elsewhere)
    std::vector<double> reach[3];
    std::atomic<int> stamp{0};

    double X(int v, int ax) const { return x[3 * (size_t)v + ax]; }
    bool less(int a, int b, int ax) const { return X(a, ax) < X(b, ax) || (X(a, ax) == X(b, ax) && a < b); }

    void run(int32_t *pnode)
    {
        mark.reset(new SetMark[nb]);
        loc.assign(nb, -1);
        for (int ax = 0; ax < 3; ax++) reach[ax].assign(nb, 0.0);
        par_chunks(nb, [&](int, int v0, int v1) {
            for (int ax = 0; ax < 3; ax++)
                for (int v = v0; v < v1; v++)
                    for (int p = gp[v]; p < gp[v + 1]; p++)
                        reach[ax][v] = std::max(reach[ax][v], std::fabs(X(v, ax) - X(gi[p], ax)));
        });
        std::vector<int> all(nb);
        std::iota(all.begin(), all.end(), 0);
        std::vector<int32_t> perm_rev;  // nodes in reverse elimination order
        perm_rev.reserve(nb);
        split(all, 0, perm_rev);
        for (int k = 0; k < nb; k++) pnode[k] = perm_rev[nb - 1 - k];
    }

    // one-sided boundary of the cut arr[0, mid) | arr[mid, n), in arr order; stops once it holds `limit` nodes
    void boundary(const std::vector<int> &arr, int mid, int ax, double mr, bool left, int in_set, std::vector<int> &out,
                  size_t limit)
    {
        out.clear();
        int n = (int)arr.size(), piv = arr[mid], last = arr[mid - 1];
        if (left) {
            double lo = X(piv, ax) - mr;
            int i0 = (int)(std::lower_bound(arr.begin(), arr.begin() + mid, lo, [&](int v, double c) { return X(v, ax) < c; }) -
                           arr.begin());
            for (int i = i0; i < mid && out.size() < limit; i++) {
                int v = arr[i];
                for (int p = gp[v]; p < gp[v + 1]; p++)
                    if (mark[gi[p]] == in_set && !less(gi[p], piv, ax)) {
                        out.push_back(v);
                        break;
                    }
            }
        } else {
            double hi = X(last, ax) + mr;
            for (int i = mid; i < n && X(arr[i], ax) <= hi && out.size() < limit; i++) {
                int v = arr[i];
                for (int p = gp[v]; p < gp[v + 1]; p++)
                    if (mark[gi[p]] == in_set && less(gi[p], piv, ax)) {
                        out.push_back(v);
                        break;
                    }
            }
        }
    }

    // Minimum vertex cover of the edges between side L and side R, with the separator S counted on side sside
    // (0 left, 1 right): U = left nodes with a right neighbour, V = right nodes with a left neighbour; a maximum
    // matching (greedy, then augmenting paths searched depth first, an explicit stack in place of recursion) and
    // König's theorem give the cover (U minus Z) + (V in Z), Z the nodes reachable from unmatched U by
    // alternating paths.
    std::vector<int> cover(const std::vector<int> &L, const std::vector<int> &R, const std::vector<int> &S, int sL, int sR,
                           int sside)
    {
        auto isL = [&](int v) { return mark[v] == sL || (mark[v] == -7 && sside == 0); };
        auto isR = [&](int v) { return mark[v] == sR || (mark[v] == -7 && sside == 1); };
        for (int v : S) mark[v] = -7;
        std::vector<int> U, V;
        auto classify = [&](const std::vector<int> &vs) {
            for (int v : vs) {
                bool l = isL(v);
                for (int p = gp[v]; p < gp[v + 1]; p++) {
                    int w = gi[p];
                    if ((l && isR(w)) || (!l && isL(w))) {
                        (l ? U : V).push_back(v);
                        break;
                    }
                }
            }
        };
        classify(L), classify(R), classify(S);
        for (int i = 0; i < (int)V.size(); i++) loc[V[i]] = i;
        std::vector<std::vector<int>> adj(U.size());
        for (int i = 0; i < (int)U.size(); i++)
            for (int p = gp[U[i]]; p < gp[U[i] + 1]; p++) {
                int w = gi[p];
                if (isR(w) && loc[w] >= 0) adj[i].push_back(loc[w]);
            }
        std::vector<int> mu(U.size(), -1), mv(V.size(), -1);
        std::vector<int32_t> vis(V.size(), -1);  // per call: the two halves of a split cover concurrently
        for (int u = 0; u < (int)U.size(); u++)
            for (int v : adj[u])
                if (mv[v] < 0) {
                    mu[u] = v, mv[v] = u;
                    break;
                }
        std::vector<std::pair<int, int>> st;  // (u, next edge)
        for (int u0 = 0; u0 < (int)U.size(); u0++) {
            if (mu[u0] >= 0) continue;
            st.assign(1, {u0, 0});
            while (!st.empty()) {
                auto &top = st.back();
                int u = top.first;
                if (top.second == (int)adj[u].size()) {
                    st.pop_back();
                    continue;
                }
                int v = adj[u][top.second++];
                if (vis[v] == u0) continue;
                vis[v] = u0;
                if (mv[v] < 0) {  // augmenting path found: every frame takes the edge it last followed
                    for (auto &f : st) {
                        int vf = adj[f.first][f.second - 1];
                        mu[f.first] = vf, mv[vf] = f.first;
                    }
                    break;
                }
                st.push_back({mv[v], 0});
            }
        }
        std::vector<char> zu(U.size(), 0), zv(V.size(), 0);
        std::vector<int> q;
        for (int u = 0; u < (int)U.size(); u++)
            if (mu[u] < 0) zu[u] = 1, q.push_back(u);
        while (!q.empty()) {
            int u = q.back();
            q.pop_back();
            for (int v : adj[u])
                if (!zv[v]) {
                    zv[v] = 1;
                    int u2 = mv[v];
                    if (u2 >= 0 && !zu[u2]) zu[u2] = 1, q.push_back(u2);
                }
        }
        std::vector<int> C;
        for (int u = 0; u < (int)U.size(); u++)
            if (!zu[u]) C.push_back(U[u]);
        for (int v = 0; v < (int)V.size(); v++)
            if (zv[v]) C.push_back(V[v]);
        for (int v : V) loc[v] = -1;
        for (int v : S) mark[v] = sside == 0 ? sL : sR;
        return C;
    }

    void split(std::vector<int> &set, int depth, std::vector<int32_t> &perm_rev)
    {
        int n = (int)set.size();
        if (n <= kLeaf) {
            for (int i = n - 1; i >= 0; i--) perm_rev.push_back(set[i]);
            return;
        }
        int in_set = ++stamp;
        for (int v : set) mark[v] = in_set;
        double best = 1e300;
        int best_ax = -1, best_mid = 0;
        std::vector<int> arr[3], SL, SR, S;
        bool s_left = true;
        for (int ax = 0; ax < 3; ax++) {
            arr[ax] = set;
            std::sort(arr[ax].begin(), arr[ax].end(), [&](int a, int b) { return less(a, b, ax); });
            double mr = 0;
            for (int v : set) mr = std::max(mr, reach[ax][v]);
            for (int f = 40; f <= 60; f += 5) {
                int mid = (int)((int64_t)n * f / 100);
                if (mid < 1 || mid >= n) continue;
                // a boundary of `limit` nodes or more cannot beat the best cut so far (the penalty is >= 1)
                size_t limit = best < 1e300 ? (size_t)best + 1 : SIZE_MAX;
                boundary(arr[ax], mid, ax, mr, true, in_set, SL, limit);
                boundary(arr[ax], mid, ax, mr, false, in_set, SR, limit);
                bool useL = SL.size() <= SR.size();
                const std::vector<int> &B = useL ? SL : SR;
                double nl = mid - (useL ? (double)B.size() : 0), nr = (n - mid) - (useL ? 0 : (double)B.size());
                double cost = B.size() * (1.0 + 2.0 * std::max(0.0, std::max(nl, nr) / n - 0.5));
                if (cost < best) best = cost, best_ax = ax, best_mid = mid, s_left = useL, S = B;
            }
        }
        int in_sep = ++stamp;
        for (int v : S) mark[v] = in_sep;
        std::vector<int> L, R;
        const std::vector<int> &a = arr[best_ax];
        for (int i = 0; i < n; i++)
            if (mark[a[i]] != in_sep) (i < best_mid ? L : R).push_back(a[i]);
        if (depth < kCoverDepth) {
            int sL = ++stamp, sR = ++stamp;
            for (int v : L) mark[v] = sL;
            for (int v : R) mark[v] = sR;
            std::vector<int> C0 = cover(L, R, S, sL, sR, 0), C1 = cover(L, R, S, sL, sR, 1);
            int sside = C0.size() <= C1.size() ? 0 : 1;
            std::vector<int> &C = sside == 0 ? C0 : C1;
            if (C.size() < S.size()) {
                int in_c = ++stamp;
                for (int v : C) mark[v] = in_c;
                std::vector<int> L2, R2;
                for (int v : L)
                    if (mark[v] != in_c) L2.push_back(v);
                for (int v : R)
                    if (mark[v] != in_c) R2.push_back(v);
                for (int v : S)
                    if (mark[v] != in_c) (sside == 0 ? L2 : R2).push_back(v);
                S.swap(C), L.swap(L2), R.swap(R2);
            }
        }
        (void)s_left;
        for (int i = (int)S.size() - 1; i >= 0; i--) perm_rev.push_back(S[i]);
        for (auto &v : arr) std::vector<int>().swap(v);
        std::vector<int>().swap(set);
        // the halves on two threads: they touch disjoint nodes' marks and cover slots (their neighbours outside
        // are the separator's, which neither changes), and the right half's order goes first either way
        if (depth < kParDepth && (int)(L.size() + R.size()) > 4096) {
            std::vector<int32_t> pr, pl;
            std::thread t([&] { split(R, depth + 1, pr); });
            split(L, depth + 1, pl);
            t.join();
            perm_rev.insert(perm_rev.end(), pr.begin(), pr.end());
            perm_rev.insert(perm_rev.end(), pl.begin(), pl.end());
        } else {
            split(R, depth + 1, perm_rev);
            split(L, depth + 1, perm_rev);
        }
    }
};
}  // namespace

std::string MfSymbolic::analyze(int n_, const int32_t *cp, const int32_t *ri, int block, void *hsp, void *descr,
                                const double *node_xyz, const int32_t *node_start, const int32_t *node_list)
{
    n = n_;
    if (n <= 0) return "empty system";
    if (block < 1 || n % block) block = 1;
    const int nb = n / block;

    // 1. nested dissection of the block graph (no self loops); per chunk of nodes, joined in node order
    std::vector<int> gp(nb + 1, 0), gi;
    const bool given = block > 1 && node_start && node_list;  // the node graph from the caller's node lists
    if (given) {
        gi.reserve((size_t)node_start[nb]);
        for (int b = 0; b < nb; b++) {
            for (int32_t k = node_start[b]; k < node_start[b + 1]; k++)
                if (node_list[k] != b) gi.push_back(node_list[k]);
            gp[b + 1] = (int)gi.size();
        }
    } else {
        std::vector<std::vector<int>> part(par_chunk_count(nb));
        par_chunks(nb, [&](int t, int b0, int b1) {
            std::vector<int> mark(nb, -1);
            part[t].reserve((size_t)(cp[(size_t)b1 * block] - cp[(size_t)b0 * block]) / (block * block));
            for (int b = b0; b < b1; b++) {
                int d = b * block, c = 0;
                for (int32_t p = cp[d]; p < cp[d + 1]; p++) {
                    int o = block == 3 ? ri[p] / 3 : ri[p] / block;  // a constant divisor for the 3D case
                    if (o == b || mark[o] == b) continue;
                    mark[o] = b;
                    part[t].push_back(o);
                    c++;
                }
                gp[b + 1] = c;
            }
        });
        for (int b = 0; b < nb; b++) gp[b + 1] += gp[b];
        gi.reserve(gp[nb]);
        for (auto &v : part) gi.insert(gi.end(), v.begin(), v.end());
    }
    std::vector<int> pnode(nb);
    if (!gi.empty() && node_xyz) {
        auto t0 = std::chrono::steady_clock::now();
        CoordNd nd{nb, gp.data(), gi.data(), node_xyz};
        nd.run(pnode.data());
        order_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    } else if (gi.empty() || !hsp) {
        std::iota(pnode.begin(), pnode.end(), 0);
    } else {
        auto t0 = std::chrono::steady_clock::now();
        cusolverStatus_t st = cusolverSpXcsrmetisndHost((cusolverSpHandle_t)hsp, nb, (int)gi.size(), (cusparseMatDescr_t)descr,
                                                        gp.data(), gi.data(), nullptr, pnode.data());
        order_s = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
        if (st != CUSOLVER_STATUS_SUCCESS) return "METIS ordering failed (cuSOLVER status " + std::to_string((int)st) + ")";
    }
    // 1b. Steps 2-6 are structural. When every nonzero of the matrix belongs to a full block x block node block
    //     (the diagonal blocks included), they run on the node graph and are expanded afterwards: a node's
    //     columns form a chain in the elimination tree (3k -> 3k + 1 -> 3k + 2 for block 3), the postorder keeps
    //     them together, column counts are cc(block k + c) = block cc_node(k) - c, and the supernode test and the
    //     row structures carry over node by node. Otherwise they run on the matrix itself.
    bool nodal = block > 1, sorted_rows = true;
    if (nodal && !given) {
        std::atomic<bool> all_nodal{true}, all_sorted{true};
        par_chunks(nb, [&](int, int b0, int b1) {
            bool nodal = true, sorted_rows = true;
            std::vector<int> rmark(n, -1), dmark(n, -1);
            for (int b = b0; b < b1 && nodal && all_nodal; b++) {
                // rows of node b's blocks: its own and its neighbours'
                for (int c = 0; c < block; c++) rmark[b * block + c] = b;
                for (int p = gp[b]; p < gp[b + 1]; p++)
                    for (int c = 0; c < block; c++) rmark[gi[p] * block + c] = b;
                int64_t want = (int64_t)block * (gp[b + 1] - gp[b] + 1);
                for (int c = 0; c < block && nodal; c++) {
                    int d = b * block + c;
                    if (cp[d + 1] - cp[d] != want) {
                        nodal = false;
                        break;
                    }
                    // rows in range, in the node's blocks and all distinct (strictly increasing rows need no marks)
                    bool inc = true;
                    for (int32_t p = cp[d]; p < cp[d + 1]; p++) {
                        int r = ri[p];
                        if ((unsigned)r >= (unsigned)n || rmark[r] != b) {
                            nodal = false;
                            break;
                        }
                        if (p > cp[d] && r <= ri[p - 1]) inc = false;
                    }
                    sorted_rows = sorted_rows && inc;
                    if (nodal && !inc)
                        for (int32_t p = cp[d]; p < cp[d + 1]; p++) {
                            if (dmark[ri[p]] == d) {
                                nodal = false;
                                break;
                            }
                            dmark[ri[p]] = d;
                        }
                }
            }
            if (!nodal) all_nodal = false;
            if (!sorted_rows) all_sorted = false;
        });
        nodal = all_nodal;
        sorted_rows = all_sorted;
    }
    const int B = nodal ? block : 1, ns = n / B;  // structural granularity and column count
    const int32_t *scp = cp, *sri = ri;
    std::vector<int32_t> perm0(ns), pinv0(ns);
    if (nodal) {
        scp = gp.data();
        sri = gi.data();
        for (int k = 0; k < nb; k++) perm0[k] = pnode[k];
    } else {
        for (int k = 0; k < nb; k++)
            for (int c = 0; c < block; c++) perm0[k * block + c] = pnode[k] * block + c;
    }
    for (int k = 0; k < ns; k++) pinv0[perm0[k]] = k;

    // 2. elimination tree of P A P' (Liu's algorithm with path compression)
    std::vector<int32_t> par(ns, -1), anc(ns, -1);
    for (int k = 0; k < ns; k++) {
        int d = perm0[k];
        for (int32_t p = scp[d]; p < scp[d + 1]; p++) {
            int i = pinv0[sri[p]];
            while (i != -1 && i < k) {
                int inext = anc[i];
                anc[i] = k;
                if (inext == -1) par[i] = k;
                i = inext;
            }
        }
    }
    // 3. postorder (children in ascending order)
    std::vector<int32_t> head(ns, -1), next(ns, -1), post(ns);
    for (int j = ns - 1; j >= 0; j--)
        if (par[j] != -1) {
            next[j] = head[par[j]];
            head[par[j]] = j;
        }
    {
        std::vector<int32_t> stack;
        int k = 0;
        for (int j = 0; j < ns; j++) {
            if (par[j] != -1) continue;
            stack.push_back(j);
            while (!stack.empty()) {
                int p = stack.back();
                int i = head[p];
                if (i == -1) {
                    stack.pop_back();
                    post[k++] = p;
                } else {
                    head[p] = next[i];
                    stack.push_back(i);
                }
            }
        }
        if (k != ns) return "internal error: elimination tree postorder incomplete";
    }
    perm.resize(ns);
    pinv.resize(ns);
    std::vector<int32_t> postinv(ns);
    for (int k = 0; k < ns; k++) postinv[post[k]] = k;
    for (int k = 0; k < ns; k++) perm[k] = perm0[post[k]];
    for (int k = 0; k < ns; k++) pinv[perm[k]] = k;
    std::vector<int32_t> parent_c(ns);
    for (int k = 0; k < ns; k++) parent_c[k] = par[post[k]] < 0 ? -1 : postinv[par[post[k]]];

    // 4. column counts of L (diagonal included) from the skeleton of the row subtrees (Gilbert, Ng and Peyton,
    //    1994), in O(|A| alpha) instead of one step per factor entry. The numbering is a postorder, so every
    //    subtree is a contiguous range [first[j], j]. Walking the columns in order, an entry a_ij (i > j) counts
    //    for column j when j starts a new leaf of row i's subtree (first[j] > the largest first seen for row i);
    //    the least common ancestor of j and row i's previous leaf counts one less. Column counts are the subtree
    //    sums of these differences.
    std::vector<int64_t> cc(ns, 0);
    {
        std::vector<int32_t> first(ns, -1), maxfirst(ns, -1), prevleaf(ns, -1), anc(ns);
        for (int k = 0; k < ns; k++) {
            cc[k] = first[k] == -1 ? 1 : 0;  // a leaf of the elimination tree
            for (int j = k; j != -1 && first[j] == -1; j = parent_c[j]) first[j] = k;
            anc[k] = k;
        }
        for (int j = 0; j < ns; j++) {
            if (parent_c[j] != -1) cc[parent_c[j]]--;
            int d = perm[j];
            for (int32_t p = scp[d]; p < scp[d + 1]; p++) {
                int i = pinv[sri[p]];
                if (i <= j || first[j] <= maxfirst[i]) continue;
                maxfirst[i] = first[j];
                int jprev = prevleaf[i];
                prevleaf[i] = j;
                cc[j]++;
                if (jprev == -1) continue;
                int q = jprev;  // least common ancestor of jprev and j, with path compression
                while (q != anc[q]) q = anc[q];
                for (int t = jprev; t != q;) {
                    int tp = anc[t];
                    anc[t] = q;
                    t = tp;
                }
                cc[q]--;
            }
            if (parent_c[j] != -1) anc[j] = parent_c[j];
        }
        for (int j = 0; j < ns; j++)
            if (parent_c[j] != -1) cc[parent_c[j]] += cc[j];
    }
    // 5. supernodes: k joins k-1's supernode when struct(L_{k-1}) = {k-1} u struct(L_k)
    std::vector<int32_t> sn_of(ns);
    c0.clear();
    for (int k = 0; k < ns; k++) {
        bool join = k > 0 && parent_c[k - 1] == k && cc[k - 1] == cc[k] + 1;
        if (!join) c0.push_back(k);
        sn_of[k] = (int)c0.size() - 1;
    }
    nsuper = (int)c0.size();
    ncol.resize(nsuper);
    for (int s = 0; s < nsuper; s++) ncol[s] = (s + 1 < nsuper ? c0[s + 1] : ns) - c0[s];
    parent.assign(nsuper, -1);
    for (int s = 0; s < nsuper; s++) {
        int last = c0[s] + ncol[s] - 1;
        if (parent_c[last] >= 0) parent[s] = sn_of[parent_c[last]];
    }
    // 6. row structures (children precede parents in postorder). The subtrees hanging at depth kRowDepth below the
    //    roots are disjoint postorder ranges and are built on host threads; the supernodes above them follow in
    //    order. Each supernode's structure is its own and its children's rows, so the result does not depend on the
    //    split.
    std::vector<std::vector<int32_t>> strc(nsuper);
    std::vector<std::vector<int32_t>> kids(nsuper);
    for (int s = 0; s < nsuper; s++)
        if (parent[s] >= 0) kids[parent[s]].push_back(s);
    {
        std::atomic<bool> bad_counts{false};
        auto build_range = [&](const std::vector<int32_t> &order, std::vector<int32_t> &mark, std::vector<uint64_t> &bits) {
            for (int s : order) {
                int first = c0[s], end = c0[s] + ncol[s];
                auto &v = strc[s];
                int lo = ns, hi = -1;
                auto add = [&](int i) {
                    if (i >= end && mark[i] != s) {
                        mark[i] = s;
                        v.push_back(i);
                        lo = std::min(lo, i);
                        hi = std::max(hi, i);
                    }
                };
                for (int j = first; j < end; j++) {
                    int d = perm[j];
                    for (int32_t p = scp[d]; p < scp[d + 1]; p++) add(pinv[sri[p]]);
                }
                for (int c : kids[s])
                    for (int i : strc[c]) add(i);
                if (v.size() < 64 || (size_t)(hi - lo) > 64 * v.size()) {
                    std::sort(v.begin(), v.end());
                } else {
                    for (int i : v) bits[(size_t)(i - lo) >> 6] |= 1ull << ((i - lo) & 63);
                    size_t k = 0, nw = (size_t)(hi - lo) / 64 + 1;
                    for (size_t w = 0; w < nw; w++) {
                        for (uint64_t b = bits[w]; b; b &= b - 1) v[k++] = lo + (int)(64 * w) + __builtin_ctzll(b);
                        bits[w] = 0;
                    }
                }
                if ((int64_t)v.size() + ncol[s] != cc[first]) bad_counts = true;
            }
        };
        // depth below the roots; the subtree of s is the postorder range [first_sn[s], s]
        constexpr int kRowDepth = 3;
        std::vector<int32_t> depth(nsuper, 0), first_sn(nsuper);
        for (int s = nsuper - 1; s >= 0; s--) depth[s] = parent[s] >= 0 ? depth[parent[s]] + 1 : 0;
        for (int s = 0; s < nsuper; s++) first_sn[s] = s;
        for (int s = 0; s < nsuper; s++)
            if (parent[s] >= 0) first_sn[parent[s]] = std::min(first_sn[parent[s]], first_sn[s]);
        std::vector<std::vector<int32_t>> ranges;
        std::vector<uint8_t> in_range(nsuper, 0);
        if (nsuper >= 256)
            for (int s = 0; s < nsuper; s++)
                if (depth[s] == kRowDepth) {
                    ranges.emplace_back();
                    for (int q = first_sn[s]; q <= s; q++) ranges.back().push_back(q), in_range[q] = 1;
                }
        std::vector<int32_t> top;
        for (int s = 0; s < nsuper; s++)
            if (!in_range[s]) top.push_back(s);
        if (!ranges.empty()) {
            std::vector<std::thread> th;
            std::atomic<int> next{0};
            int nth = (int)std::min<size_t>(ranges.size(), std::max(1u, std::thread::hardware_concurrency()));
            for (int t = 0; t < nth; t++)
                th.emplace_back([&] {
                    std::vector<int32_t> mark(ns, -1);
                    std::vector<uint64_t> bits((size_t)ns / 64 + 1, 0);
                    for (int r; (r = next.fetch_add(1)) < (int)ranges.size();) build_range(ranges[r], mark, bits);
                });
            for (auto &t : th) t.join();
        }
        {
            std::vector<int32_t> mark(ns, -1);
            std::vector<uint64_t> bits((size_t)ns / 64 + 1, 0);
            build_range(top, mark, bits);
        }
        if (bad_counts) return "internal error: supernode structure does not match the column counts";
    }
    if (B > 1) {  // node numbering -> equation numbering
        std::vector<int32_t> pn(perm);
        perm.resize(n);
        pinv.resize(n);
        for (int k = 0; k < ns; k++)
            for (int c = 0; c < B; c++) perm[k * B + c] = pn[k] * B + c;
        for (int k = 0; k < n; k++) pinv[perm[k]] = k;
        auto expand = [&](int s) {
            c0[s] *= B;
            ncol[s] *= B;
            std::vector<int32_t> v(strc[s].size() * B);
            for (size_t k = 0; k < strc[s].size(); k++)
                for (int c = 0; c < B; c++) v[k * B + c] = strc[s][k] * B + c;
            strc[s] = std::move(v);
        };
        int nth = nsuper < 256 ? 1 : (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency()));
        std::atomic<int> next{0};
        auto worker = [&] {
            for (int s; (s = next.fetch_add(1)) < nsuper;) expand(s);
        };
        std::vector<std::thread> th;
        for (int t = 1; t < nth; t++) th.emplace_back(worker);
        worker();
        for (auto &t : th) t.join();
    }
    // 6b. relaxed amalgamation: merge a supernode into its parent when it is the parent's contiguous (last) child
    //     and the explicit zeros this adds stay small; chains inside a separator collapse into one front.
    {
        std::vector<int32_t> mc0(c0.begin(), c0.end()), mnc(ncol.begin(), ncol.end()), mpar(parent.begin(), parent.end());
        std::vector<int64_t> zeros(nsuper, 0);
        std::vector<uint8_t> alive(nsuper, 1);
        std::vector<int32_t> rep(nsuper);  // representative (merged node) of each original supernode
        for (int q = 0; q < nsuper; q++) rep[q] = q;
        auto find = [&](int q) {
            while (q >= 0 && !alive[q]) q = rep[q];
            return q;
        };
        for (int p = 0; p < nsuper; p++) {
            int c = p - 1;  // only the immediately preceding supernode can be contiguous
            if (c < 0 || !alive[c] || find(mpar[c]) != p || mc0[c] + mnc[c] != mc0[p]) continue;
            int64_t mp = mnc[p] + (int64_t)strc[p].size();
            int64_t nrc = (int64_t)strc[c].size();
            int64_t add = (int64_t)mnc[c] * (mp - nrc);                    // zeros in c's columns
            int64_t ncm = mnc[c] + mnc[p];
            int64_t total = ncm * (ncm + 1) / 2 + ncm * (int64_t)strc[p].size();
            bool small = ncm <= 16;
            if (!(small || (zeros[c] + zeros[p] + add) * 5 <= total)) continue;  // at most 20 % explicit zeros
            // merge c into p: p keeps its parent and structure, gains c's columns and children
            mc0[p] = mc0[c];
            mnc[p] = (int32_t)ncm;
            zeros[p] += zeros[c] + add;
            alive[c] = 0;
            rep[c] = p;
        }
        // compact
        std::vector<int32_t> newid(nsuper, -1);
        int ns = 0;
        for (int q = 0; q < nsuper; q++)
            if (alive[q]) newid[q] = ns++;
        std::vector<int32_t> c0n, ncn, parn;
        std::vector<std::vector<int32_t>> strn;
        for (int q = 0; q < nsuper; q++) {
            if (!alive[q]) continue;
            c0n.push_back(mc0[q]);
            ncn.push_back(mnc[q]);
            int pp = find(mpar[q]);
            parn.push_back(pp < 0 ? -1 : newid[pp]);
            strn.push_back(std::move(strc[q]));
        }
        nsuper = ns;
        c0 = c0n;
        ncol = ncn;
        parent = parn;
        strc = std::move(strn);
        kids.assign(nsuper, {});
        for (int q = 0; q < nsuper; q++)
            if (parent[q] >= 0) kids[parent[q]].push_back(q);
    }
    // 7. fronts, levels, maps
    m.resize(nsuper);
    level.assign(nsuper, 0);
    max_m = max_ncol = 0;
    factor_nnz = 0;
    for (int s = 0; s < nsuper; s++) {
        m[s] = ncol[s] + (int)strc[s].size();
        for (int c : kids[s]) level[s] = std::max(level[s], level[c] + 1);
        max_m = std::max(max_m, m[s]);
        max_ncol = std::max(max_ncol, ncol[s]);
        factor_nnz += (int64_t)ncol[s] * (ncol[s] + 1) / 2 + (int64_t)ncol[s] * (int64_t)strc[s].size();
    }
    nlevels = 0;
    for (int s = 0; s < nsuper; s++) nlevels = std::max(nlevels, level[s] + 1);
    level_start.assign(nlevels + 1, 0);
    for (int s = 0; s < nsuper; s++) level_start[level[s] + 1]++;
    for (int l = 0; l < nlevels; l++) level_start[l + 1] += level_start[l];
    level_list.assign(nsuper, 0);
    {
        std::vector<int32_t> fill(level_start.begin(), level_start.end() - 1);
        for (int s = 0; s < nsuper; s++) level_list[fill[level[s]]++] = s;
    }
    front_off.assign(nsuper, 0);
    level_pool_start.assign(nlevels + 1, 0);
    pool = 0;
    for (int l = 0; l < nlevels; l++) {
        level_pool_start[l] = pool;
        for (int32_t q = level_start[l]; q < level_start[l + 1]; q++) {
            int s = level_list[q];
            front_off[s] = pool;
            pool += (int64_t)m[s] * m[s];
        }
    }
    level_pool_start[nlevels] = pool;
    idx_start.assign(nsuper + 1, 0);
    for (int s = 0; s < nsuper; s++) idx_start[s + 1] = idx_start[s] + m[s];
    idx.resize(idx_start[nsuper]);
    for (int s = 0; s < nsuper; s++) {
        int o = idx_start[s];
        for (int k = 0; k < ncol[s]; k++) idx[o + k] = c0[s] + k;
        for (size_t k = 0; k < strc[s].size(); k++) idx[o + ncol[s] + k] = strc[s][k];
    }
    relmap_start.assign(nsuper + 1, 0);
    uvec_start.assign(nsuper + 1, 0);
    for (int s = 0; s < nsuper; s++) {
        relmap_start[s + 1] = relmap_start[s] + (int)strc[s].size();
        uvec_start[s + 1] = uvec_start[s] + (int)strc[s].size();
    }
    uvec_pool = uvec_start[nsuper];
    relmap.assign(relmap_start[nsuper], 0);
    std::vector<int32_t> pos(n, -1);  // row -> position in the front at hand (reset after each front)
    for (int p = 0; p < nsuper; p++) {
        if (parent[p] < 0 && !strc[p].empty()) return "internal error: a root supernode has off-diagonal rows";
        if (kids[p].empty()) continue;
        const int32_t *pb = idx.data() + idx_start[p];
        for (int k = 0; k < m[p]; k++) pos[pb[k]] = k;
        for (int s : kids[p])
            for (size_t k = 0; k < strc[s].size(); k++) {
                int32_t q = pos[strc[s][k]];
                if (q < 0) return "internal error: child row missing from the parent front";
                relmap[relmap_start[s] + k] = q;
            }
        for (int k = 0; k < m[p]; k++) pos[pb[k]] = -1;
    }
    // original values -> fronts, grouped by level. The entries of one front form one range: a count pass sizes
    // the ranges, a fill pass writes them; both hand the fronts out to host threads one at a time.
    std::atomic<int> bad{0};
    auto walk = [&](int q, std::vector<int32_t> &pos, int64_t *dst, int32_t *src) {
        int s = level_list[q];
        const int32_t *ib = idx.data() + idx_start[s];
        for (int k = 0; k < m[s]; k++) pos[ib[k]] = k;
        int64_t cnt = 0;
        for (int j = c0[s]; j < c0[s] + ncol[s]; j++) {
            int d = perm[j];
            int64_t base = front_off[s] + (int64_t)(j - c0[s]) * m[s];
            if (nodal && sorted_rows) {
                // rows come in whole node blocks, consecutive in the new numbering and in the front
                for (int32_t p = cp[d]; p < cp[d + 1]; p += B) {
                    int i0 = pinv[ri[p]];
                    if (i0 + B - 1 < j) continue;
                    if (pos[i0] < 0) {
                        bad = 1;
                        continue;
                    }
                    for (int r = std::max(0, j - i0); r < B; r++, cnt++)
                        if (dst) dst[cnt] = base + pos[i0] + r, src[cnt] = p + r;
                }
                continue;
            }
            for (int32_t p = cp[d]; p < cp[d + 1]; p++) {
                int i = pinv[ri[p]];
                if (i < j) continue;
                if (pos[i] < 0) {
                    bad = 1;
                    continue;
                }
                if (dst) dst[cnt] = base + pos[i], src[cnt] = p;
                cnt++;
            }
        }
        for (int k = 0; k < m[s]; k++) pos[ib[k]] = -1;
        return cnt;
    };
    int nth = cp[n] < (1 << 18) ? 1 : (int)std::min<unsigned>(16, std::max(1u, std::thread::hardware_concurrency()));
    nth = std::max(1, std::min(nth, nsuper));
    std::vector<std::vector<int32_t>> tpos(nth, std::vector<int32_t>(n, -1));
    auto each_front = [&](const std::function<void(int, std::vector<int32_t> &)> &body) {
        std::atomic<int> next{0};
        auto work = [&](int t) {
            for (int q; (q = next++) < nsuper;) body(q, tpos[t]);
        };
        std::vector<std::thread> th;
        for (int t = 1; t < nth; t++) th.emplace_back(work, t);
        work(0);
        for (auto &x : th) x.join();
    };
    std::vector<int64_t> fstart(nsuper + 1, 0);  // entry range of the q-th front in level order
    each_front([&](int q, std::vector<int32_t> &ps) { fstart[q + 1] = walk(q, ps, nullptr, nullptr); });
    if (bad) return "internal error: matrix entry outside its front";
    for (int q = 0; q < nsuper; q++) fstart[q + 1] += fstart[q];
    if (fstart[nsuper] > INT32_MAX) return "Factor scatter map exceeds 32-bit indexing.";
    a_dst.resize(fstart[nsuper]);
    a_src.resize(fstart[nsuper]);
    each_front([&](int q, std::vector<int32_t> &ps) { walk(q, ps, a_dst.data() + fstart[q], a_src.data() + fstart[q]); });
    a_level_start.assign(nlevels + 1, 0);
    for (int l = 0; l <= nlevels; l++) a_level_start[l] = (int32_t)fstart[level_start[l]];
    // extend-add schedule: r-th child (ascending) of every parent of a level
    max_rank = 1;
    for (int s = 0; s < nsuper; s++) max_rank = std::max<int>(max_rank, (int)kids[s].size());
    ext_start.assign((size_t)nlevels * max_rank + 1, 0);
    std::vector<std::vector<int32_t>> buckets((size_t)nlevels * max_rank);
    for (int l = 0; l < nlevels; l++)
        for (int32_t q = level_start[l]; q < level_start[l + 1]; q++) {
            int p = level_list[q];
            for (size_t r = 0; r < kids[p].size(); r++) buckets[(size_t)l * max_rank + r].push_back(kids[p][r]);
        }
    ext_child.clear();
    for (size_t b = 0; b < buckets.size(); b++) {
        ext_start[b] = (int32_t)ext_child.size();
        ext_child.insert(ext_child.end(), buckets[b].begin(), buckets[b].end());
    }
    ext_start[buckets.size()] = (int32_t)ext_child.size();
    return "";
}

}  // namespace ifea
