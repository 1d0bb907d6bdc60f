// trimesh.h — host construction of a triangulated die's bucket grids (TriMeshSolid's constructor,
// ThreeD/TriMeshSolid.cs:17-82): the bounding box, an xy grid of cell c2 and a 3D grid of cell c3, each cell listing
// the triangles whose bounding box overlaps it, in triangle order. The device queries are in common.cuh (TriGrid).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <string>
#include <vector>

#include "common.cuh"

namespace ifea {

struct TriMeshHost {
    std::vector<double> v;
    std::vector<int32_t> t, xy_start, xy_items, g3_start, g3_items;
    TriGrid grid;  // host pointers into the vectors above

    std::string build(int nv, const double *vert, int nt, const int32_t *tri)
    {
        if (nv < 3 || nt < 1 || !vert || !tri) return "a triangulated die needs vertices and triangles";
        for (int k = 0; k < 3 * nt; k++)
            if (tri[k] < 0 || tri[k] >= nv) return "triangle vertex index out of range";
        v.assign(vert, vert + 3 * (size_t)nv);
        t.assign(tri, tri + 3 * (size_t)nt);
        TriGrid &g = grid;
        double mn[3] = {1.7976931348623157e308, 1.7976931348623157e308, 1.7976931348623157e308};
        double mx[3] = {-1.7976931348623157e308, -1.7976931348623157e308, -1.7976931348623157e308};
        for (int i = 0; i < nv; i++)
            for (int a = 0; a < 3; a++) {
                mn[a] = std::min(mn[a], v[3 * (size_t)i + a]);
                mx[a] = std::max(mx[a], v[3 * (size_t)i + a]);
            }
        for (int a = 0; a < 3; a++) g.mn[a] = mn[a], g.mx[a] = mx[a];
        double ex = mx[0] - mn[0], ey = mx[1] - mn[1], ez = mx[2] - mn[2];
        double ext = std::max(ex, std::max(ey, ez));
        g.c2 = std::max(ext / 200, std::sqrt((ex + 1e-9) * (ey + 1e-9) / std::max(nt, 1)) * 2);
        g.nx2 = std::max(1, (int)std::ceil(ex / g.c2) + 1);
        g.ny2 = std::max(1, (int)std::ceil(ey / g.c2) + 1);
        g.c3 = std::max(ext / 120, std::cbrt((ex + 1e-9) * (ey + 1e-9) * (ez + 1e-9) / std::max(nt, 1)) * 2);
        g.gx = std::max(1, (int)std::ceil(ex / g.c3) + 1);
        g.gy = std::max(1, (int)std::ceil(ey / g.c3) + 1);
        g.gz = std::max(1, (int)std::ceil(ez / g.c3) + 1);
        auto cx2 = [&](double x) { return std::clamp((int)((x - mn[0]) / g.c2), 0, g.nx2 - 1); };
        auto cy2 = [&](double y) { return std::clamp((int)((y - mn[1]) / g.c2), 0, g.ny2 - 1); };
        auto c3 = [&](double val, double lo, int n) { return std::clamp((int)((val - lo) / g.c3), 0, n - 1); };
        size_t n2 = (size_t)g.nx2 * g.ny2, n3 = (size_t)g.gx * g.gy * g.gz;
        xy_start.assign(n2 + 1, 0);
        g3_start.assign(n3 + 1, 0);
        // two passes (count, fill) over the triangles in order, so each cell lists them ascending
        for (int pass = 0; pass < 2; pass++) {
            std::vector<int32_t> f2, f3;
            if (pass == 1) {
                for (size_t c = 0; c < n2; c++) xy_start[c + 1] += xy_start[c];
                for (size_t c = 0; c < n3; c++) g3_start[c + 1] += g3_start[c];
                xy_items.assign(xy_start[n2], 0);
                g3_items.assign(g3_start[n3], 0);
                f2.assign(xy_start.begin(), xy_start.end() - 1);
                f3.assign(g3_start.begin(), g3_start.end() - 1);
            }
            for (int k = 0; k < nt; k++) {
                const double *a = &v[3 * (size_t)t[3 * k]], *b = &v[3 * (size_t)t[3 * k + 1]], *c = &v[3 * (size_t)t[3 * k + 2]];
                double lx = std::min(a[0], std::min(b[0], c[0])), hx = std::max(a[0], std::max(b[0], c[0]));
                double ly = std::min(a[1], std::min(b[1], c[1])), hy = std::max(a[1], std::max(b[1], c[1]));
                double lz = std::min(a[2], std::min(b[2], c[2])), hz = std::max(a[2], std::max(b[2], c[2]));
                for (int j = cy2(ly); j <= cy2(hy); j++)
                    for (int i = cx2(lx); i <= cx2(hx); i++) {
                        size_t cell = (size_t)j * g.nx2 + i;
                        if (pass == 0) xy_start[cell + 1]++;
                        else xy_items[f2[cell]++] = k;
                    }
                for (int kk = c3(lz, mn[2], g.gz); kk <= c3(hz, mn[2], g.gz); kk++)
                    for (int j = c3(ly, mn[1], g.gy); j <= c3(hy, mn[1], g.gy); j++)
                        for (int i = c3(lx, mn[0], g.gx); i <= c3(hx, mn[0], g.gx); i++) {
                            size_t cell = ((size_t)kk * g.gy + j) * g.gx + i;
                            if (pass == 0) g3_start[cell + 1]++;
                            else g3_items[f3[cell]++] = k;
                        }
            }
        }
        g.nt = nt;
        point_at_host();
        return "";
    }

    void point_at_host()
    {
        grid.v = v.data();
        grid.t = t.data();
        grid.xy_start = xy_start.data();
        grid.xy_items = xy_items.data();
        grid.g3_start = g3_start.data();
        grid.g3_items = g3_items.data();
    }
};

}  // namespace ifea
