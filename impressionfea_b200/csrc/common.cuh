// common.cuh — device/host helpers shared by the forging kernels.
//
// Arithmetic is written in the reference's evaluation order (left to right, no contraction; the library is
// built with --fmad=false) so per-element and per-node results can be compared with the FP64 restatement
// to the last bit wherever no transcendental function is involved.
#pragma once
#include <cuda_runtime.h>
#include <float.h>
#include <math.h>
#include <stdint.h>

#define IFEA_HD __host__ __device__ __forceinline__

struct d3 {
    double x, y, z;
};
IFEA_HD d3 mk3(double x, double y, double z) { d3 r; r.x = x; r.y = y; r.z = z; return r; }
IFEA_HD d3 add3(d3 a, d3 b) { return mk3(a.x + b.x, a.y + b.y, a.z + b.z); }
IFEA_HD d3 sub3(d3 a, d3 b) { return mk3(a.x - b.x, a.y - b.y, a.z - b.z); }
IFEA_HD d3 neg3(d3 a) { return mk3(-a.x, -a.y, -a.z); }
IFEA_HD d3 scl3(double s, d3 a) { return mk3(s * a.x, s * a.y, s * a.z); }
IFEA_HD double dot3(d3 a, d3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
IFEA_HD d3 cross3(d3 a, d3 b) { return mk3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
IFEA_HD double len3(d3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
IFEA_HD double len23(d3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
IFEA_HD d3 nrm3(d3 a) { double l = len3(a); return l > 0 ? mk3(a.x / l, a.y / l, a.z / l) : a; }
IFEA_HD double get3(d3 a, int i) { return i == 0 ? a.x : (i == 1 ? a.y : a.z); }
IFEA_HD d3 lerp3(d3 a, d3 b, double t) { return add3(a, scl3(t, sub3(b, a))); }
IFEA_HD bool eq3(d3 a, d3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }
IFEA_HD d3 ld3(const double *p, int n) { return mk3(p[3 * n], p[3 * n + 1], p[3 * n + 2]); }
IFEA_HD void st3(double *p, int n, d3 v) { p[3 * n] = v.x; p[3 * n + 1] = v.y; p[3 * n + 2] = v.z; }

// Math.Max / Math.Min / Math.Clamp semantics for doubles (NaN propagates through Max/Min).
IFEA_HD double rmax(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }
IFEA_HD double rmin(double a, double b) { return (a != a || b != b) ? NAN : (a < b ? a : b); }
IFEA_HD double rclamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }
IFEA_HD int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }

// sigma = C (eps0 + max(eps,0))^n * max(rate,1e-12)^m  (Materials/FlowStressLaw.cs:8-9)
IFEA_HD double flow_stress(double C, double N, double M, double eps0, double strain, double rate)
{
    return C * pow(eps0 + rmax(strain, 0), N) * pow(rmax(rate, 1e-12), M);
}

// Closest point on a triangle (ThreeD/Vec3.cs:35-56; Ericson 5.1.5).
IFEA_HD d3 closest_on_triangle(d3 p, d3 a, d3 b, d3 c)
{
    d3 ab = sub3(b, a), ac = sub3(c, a), ap = sub3(p, a);
    double d1 = dot3(ab, ap), d2 = dot3(ac, ap);
    if (d1 <= 0 && d2 <= 0) return a;
    d3 bp = sub3(p, b);
    double d3v = dot3(ab, bp), d4 = dot3(ac, bp);
    if (d3v >= 0 && d4 <= d3v) return b;
    double vc = d1 * d4 - d3v * d2;
    if (vc <= 0 && d1 >= 0 && d3v <= 0) return add3(a, scl3(d1 / (d1 - d3v), ab));
    d3 cp = sub3(p, c);
    double d5 = dot3(ab, cp), d6 = dot3(ac, cp);
    if (d6 >= 0 && d5 <= d6) return c;
    double vb = d5 * d2 - d1 * d6;
    if (vb <= 0 && d2 >= 0 && d6 <= 0) return add3(a, scl3(d2 / (d2 - d6), ac));
    double va = d3v * d6 - d5 * d4;
    if (va <= 0 && d4 - d3v >= 0 && d5 - d6 >= 0) return add3(b, scl3((d4 - d3v) / (d4 - d3v + (d5 - d6)), sub3(c, b)));
    double denom = 1 / (va + vb + vc);
    return add3(add3(a, scl3(vb * denom, ab)), scl3(vc * denom, ac));
}

// TetMesh.Volume / Quality (ThreeD/TetMesh.cs:104-112): 6*sqrt(2)*V / L_rms^3.
IFEA_HD double tet_volume(d3 a, d3 b, d3 c, d3 d) { return dot3(sub3(b, a), cross3(sub3(c, a), sub3(d, a))) / 6.0; }
IFEA_HD double tet_quality(d3 a, d3 b, d3 c, d3 d)
{
    double l2 = (len23(sub3(b, a)) + len23(sub3(c, a)) + len23(sub3(d, a)) + len23(sub3(c, b)) + len23(sub3(d, b)) +
                 len23(sub3(d, c))) / 6.0;
    return l2 > 0 ? 6 * sqrt(2.0) * tet_volume(a, b, c, d) / pow(l2, 1.5) : -1;
}

// Rigid die z = h(x, y) on a regular grid (ThreeD/HeightFieldDie.cs). Pointer h lives in device memory.
// A die given as a closed triangulated solid (TriMeshDie over TriMeshSolid, ThreeD/TriMeshSolid.cs:5-180, :248-297):
// vertices, triangles, bounding box, and the solid's two bucket grids in its own layout (an xy grid of cell c2 for
// vertical hits, a 3D grid of cell c3 for closest points; each cell lists its triangles in ascending order).
struct TriGrid {
    const double *v = nullptr;   // 3 per vertex
    const int32_t *t = nullptr;  // 3 per triangle
    int nt = 0;
    double mn[3] = {0, 0, 0}, mx[3] = {0, 0, 0};
    double c2 = 1;
    int nx2 = 1, ny2 = 1;
    const int32_t *xy_start = nullptr, *xy_items = nullptr;
    double c3 = 1;
    int gx = 1, gy = 1, gz = 1;
    const int32_t *g3_start = nullptr, *g3_items = nullptr;
};

struct HField {
    int side;  // 0 bottom, 1 top
    int nx, ny;
    double x0, y0, dx;
    const double *h;
    int kind = 0;  // 0 height field (the fields above), 1 triangulated solid (tm)
    TriGrid tm;
};

IFEA_HD d3 tm_vertex(const TriGrid &g, int i) { return mk3(g.v[3 * i], g.v[3 * i + 1], g.v[3 * i + 2]); }

// VerticalHits (TriMeshSolid.cs:96-121): every triangle of the point's xy cell that the vertical line through the
// (jittered) point crosses, as its z; visit(z) for each.
template <typename F>
IFEA_HD void tm_vertical_hits(const TriGrid &g, double x, double y, F &&visit)
{
    if (x < g.mn[0] || x > g.mx[0] || y < g.mn[1] || y > g.mx[1]) return;
    x += 1.2345e-7;
    y += 2.3456e-7;
    int cx = iclamp((int)((x - g.mn[0]) / g.c2), 0, g.nx2 - 1), cy = iclamp((int)((y - g.mn[1]) / g.c2), 0, g.ny2 - 1);
    int cell = cy * g.nx2 + cx;
    for (int q = g.xy_start[cell]; q < g.xy_start[cell + 1]; q++) {
        int t = g.xy_items[q];
        d3 a = tm_vertex(g, g.t[3 * t]), b = tm_vertex(g, g.t[3 * t + 1]), c = tm_vertex(g, g.t[3 * t + 2]);
        double d = (b.x - a.x) * (c.y - a.y) - (c.x - a.x) * (b.y - a.y);
        if (fabs(d) < 1e-300) continue;
        double u = ((x - a.x) * (c.y - a.y) - (c.x - a.x) * (y - a.y)) / d;
        double v = ((b.x - a.x) * (y - a.y) - (x - a.x) * (b.y - a.y)) / d;
        if (u < 0 || v < 0 || u + v > 1) continue;
        visit(a.z + u * (b.z - a.z) + v * (c.z - a.z));
    }
}

// Contains (:125-137): inside when an odd number of hits lies above the point
IFEA_HD bool tm_contains(const TriGrid &g, d3 p)
{
    if (p.x < g.mn[0] || p.x > g.mx[0] || p.y < g.mn[1] || p.y > g.mx[1] || p.z < g.mn[2] || p.z > g.mx[2]) return false;
    int above = 0;
    tm_vertical_hits(g, p.x, p.y, [&](double z) { above += z > p.z; });
    return (above & 1) == 1;
}

// Closest (:139-178): rings of 3D cells around the point's cell until the best distance is within the ring
IFEA_HD bool tm_closest(const TriGrid &g, d3 p, double maxd, d3 *point, d3 *normal, double *dist)
{
    d3 bp = p, bn = mk3(0, 0, 1);
    int ci = (int)floor((p.x - g.mn[0]) / g.c3), cj = (int)floor((p.y - g.mn[1]) / g.c3), ck = (int)floor((p.z - g.mn[2]) / g.c3);
    int max_ring = (int)ceil(maxd / g.c3) + 1;
    double best = maxd * maxd;
    for (int ring = 0; ring <= max_ring; ring++) {
        for (int k = ck - ring; k <= ck + ring; k++) {
            if (k < 0 || k >= g.gz) continue;
            for (int j = cj - ring; j <= cj + ring; j++) {
                if (j < 0 || j >= g.gy) continue;
                bool shell_row = abs(j - cj) == ring || abs(k - ck) == ring;
                int istep = shell_row || ring == 0 ? 1 : 2 * ring;
                for (int i = ci - ring; i <= ci + ring; i += istep) {
                    if (i < 0 || i >= g.gx) continue;
                    int cell = (k * g.gy + j) * g.gx + i;
                    for (int q = g.g3_start[cell]; q < g.g3_start[cell + 1]; q++) {
                        int t = g.g3_items[q];
                        d3 a = tm_vertex(g, g.t[3 * t]), b = tm_vertex(g, g.t[3 * t + 1]), c = tm_vertex(g, g.t[3 * t + 2]);
                        d3 cq = closest_on_triangle(p, a, b, c);
                        double dd = len23(sub3(cq, p));
                        if (dd >= best) continue;
                        best = dd;
                        bp = cq;
                        bn = nrm3(cross3(sub3(b, a), sub3(c, a)));
                    }
                }
            }
        }
        if (sqrt(best) <= ring * g.c3) break;
    }
    *point = bp;
    *normal = bn;
    *dist = sqrt(best);
    return *dist < maxd;
}

// TriMeshDie.Clearance / Project / SurfaceZ (:267-296): the die moved by `offset` along z; Reach = 6 mm
IFEA_HD double tm_clearance(const TriGrid &g, d3 p, double offset)
{
    const double reach = 6;
    d3 q = mk3(p.x, p.y, p.z - offset);
    if (q.x < g.mn[0] - reach || q.x > g.mx[0] + reach || q.y < g.mn[1] - reach || q.y > g.mx[1] + reach ||
        q.z < g.mn[2] - reach || q.z > g.mx[2] + reach)
        return reach;
    bool inside = tm_contains(g, q);
    d3 c, n;
    double dist;
    double d = tm_closest(g, q, reach, &c, &n, &dist) ? dist : reach;
    return inside ? -d : d;
}
IFEA_HD d3 tm_project(const TriGrid &g, int side, d3 p, double offset, d3 *normal)
{
    const double reach = 6;
    d3 q = mk3(p.x, p.y, p.z - offset), c, n;
    double dist;
    if (!tm_closest(g, q, 4 * reach, &c, &n, &dist)) n = side == 0 ? mk3(0, 0, 1) : mk3(0, 0, -1);
    if (normal) *normal = n;
    return mk3(c.x, c.y, c.z + offset);
}
IFEA_HD double tm_surface_z(const TriGrid &g, int side, double x, double y)
{
    bool any = false;
    double z = 0;
    tm_vertical_hits(g, x, y, [&](double h) {
        z = !any ? h : (side == 0 ? rmax(z, h) : rmin(z, h));
        any = true;
    });
    return any ? z : NAN;
}

// HeightAt (:100-107); a triangulated die's SurfaceZ
IFEA_HD double hf_height(const HField &d, double x, double y)
{
    if (d.kind == 1) return tm_surface_z(d.tm, d.side, x, y);
    double fx = rclamp((x - d.x0) / d.dx, 0, d.nx), fy = rclamp((y - d.y0) / d.dx, 0, d.ny);
    int i = min((int)fx, d.nx - 1), j = min((int)fy, d.ny - 1);
    double u = fx - i, v = fy - j;
    int w = d.nx + 1;
    return (1 - u) * (1 - v) * d.h[j * w + i] + u * (1 - v) * d.h[j * w + i + 1] + (1 - u) * v * d.h[(j + 1) * w + i] +
           u * v * d.h[(j + 1) * w + i + 1];
}

// Clearance (:130-134): > 0 in the open cavity, < 0 penetrating.
IFEA_HD double hf_clearance(const HField &d, d3 p, double offset)
{
    if (d.kind == 1) return tm_clearance(d.tm, p, offset);
    double h = hf_height(d, p.x, p.y) + offset;
    return d.side == 0 ? p.z - h : h - p.z;
}

IFEA_HD d3 hf_vertex(const HField &d, int i, int j, double offset)
{
    return mk3(d.x0 + i * d.dx, d.y0 + j * d.dx, d.h[j * (d.nx + 1) + i] + offset);
}

// Project (:157-191): closest point over the two triangles of each cell within reach; normal out of the die.
IFEA_HD d3 hf_project(const HField &d, d3 p, double offset, d3 *normal)
{
    if (d.kind == 1) return tm_project(d.tm, d.side, p, offset, normal);
    double reach = fabs(hf_clearance(d, p, offset)) + 1.5 * d.dx;
    int i0 = iclamp((int)floor((p.x - reach - d.x0) / d.dx), 0, d.nx - 1);
    int i1 = iclamp((int)floor((p.x + reach - d.x0) / d.dx), 0, d.nx - 1);
    int j0 = iclamp((int)floor((p.y - reach - d.y0) / d.dx), 0, d.ny - 1);
    int j1 = iclamp((int)floor((p.y + reach - d.y0) / d.dx), 0, d.ny - 1);
    double best = DBL_MAX;
    d3 bestQ = p;
    d3 bestN = d.side == 0 ? mk3(0, 0, 1) : neg3(mk3(0, 0, 1));
    for (int j = j0; j <= j1; j++) {
        for (int i = i0; i <= i1; i++) {
            d3 a = hf_vertex(d, i, j, offset), b = hf_vertex(d, i + 1, j, offset);
            d3 c = hf_vertex(d, i + 1, j + 1, offset), e = hf_vertex(d, i, j + 1, offset);
            for (int t = 0; t < 2; t++) {
                d3 tb = t == 0 ? b : c, tc = t == 0 ? c : e;
                d3 q = closest_on_triangle(p, a, tb, tc);
                double dd = len23(sub3(q, p));
                if (dd >= best) continue;
                best = dd;
                bestQ = q;
                d3 n = nrm3(cross3(sub3(tb, a), sub3(tc, a)));
                bestN = d.side == 0 ? n : neg3(n);
            }
        }
    }
    if (normal) *normal = bestN;
    return bestQ;
}

// Principal.Max3 (Solver/Principal.cs:7-19)
IFEA_HD double principal_max3(double xx, double yy, double zz, double xy, double yz, double zx)
{
    double p1 = xy * xy + yz * yz + zx * zx;
    double q = (xx + yy + zz) / 3;
    if (p1 < 1e-30 * (xx * xx + yy * yy + zz * zz + 1e-300)) return rmax(xx, rmax(yy, zz));
    double p2 = (xx - q) * (xx - q) + (yy - q) * (yy - q) + (zz - q) * (zz - q) + 2 * p1;
    double p = sqrt(p2 / 6);
    double bxx = (xx - q) / p, byy = (yy - q) / p, bzz = (zz - q) / p, bxy = xy / p, byz = yz / p, bzx = zx / p;
    double detB = bxx * (byy * bzz - byz * byz) - bxy * (bxy * bzz - byz * bzx) + bzx * (bxy * byz - byy * bzx);
    double r = rclamp(detB / 2, -1, 1);
    double phi = acos(r) / 3;
    return q + 2 * p * cos(phi);
}

#define IFEA_CUDA_CHECK(call)                                                                                   \
    do {                                                                                                        \
        cudaError_t _e = (call);                                                                                \
        if (_e != cudaSuccess) throw ifea::CudaFailure(#call, _e);                                              \
    } while (0)
