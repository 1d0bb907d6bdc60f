/* Internal helpers of the CPU oracle (test infrastructure only; see ifea_oracle.h). */
#ifndef O_INTERNAL_H
#define O_INTERNAL_H
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "ifea_oracle.h"

/* Vec3 (ThreeD/Vec3.cs:4-57): every operator evaluates left to right like the record struct. */
typedef struct { double x, y, z; } v3;
static inline v3 V3(double x, double y, double z) { v3 r = {x, y, z}; return r; }
static inline v3 vadd(v3 a, v3 b) { return V3(a.x + b.x, a.y + b.y, a.z + b.z); }
static inline v3 vsub(v3 a, v3 b) { return V3(a.x - b.x, a.y - b.y, a.z - b.z); }
static inline v3 vneg(v3 a) { return V3(-a.x, -a.y, -a.z); }
static inline v3 vscale(double s, v3 a) { return V3(s * a.x, s * a.y, s * a.z); }
static inline double vdot(v3 a, v3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
static inline v3 vcross(v3 a, v3 b) { return V3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
static inline double vlen(v3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
static inline double vlen2(v3 a) { return a.x * a.x + a.y * a.y + a.z * a.z; }
static inline v3 vnormalized(v3 a) { double l = vlen(a); return l > 0 ? V3(a.x / l, a.y / l, a.z / l) : a; }
static inline double vget(v3 a, int i) { return i == 0 ? a.x : i == 1 ? a.y : a.z; }
static inline v3 vlerp(v3 a, v3 b, double t) { return vadd(a, vscale(t, vsub(b, a))); }
static inline int veq(v3 a, v3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

static inline double dmax(double a, double b) { return (a != a || b != b) ? NAN : (a > b ? a : b); }
static inline double dmin(double a, double b) { return (a != a || b != b) ? NAN : (a < b ? a : b); }
static inline double dclamp(double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int iclamp(int v, int lo, int hi) { return v < lo ? lo : (v > hi ? hi : v); }
static inline int imin(int a, int b) { return a < b ? a : b; }
static inline int imax(int a, int b) { return a > b ? a : b; }

/* FlowStressLaw.Stress (Materials/FlowStressLaw.cs:8-9). */
static inline double law_stress(double C, double N, double M, double eps0, double strain, double rate)
{
    return C * pow(eps0 + dmax(strain, 0), N) * pow(dmax(rate, 1e-12), M);
}

/* Vec3.ClosestOnTriangle (ThreeD/Vec3.cs:35-56). */
v3 o_closest_on_triangle(v3 p, v3 a, v3 b, v3 c);
/* TetMesh.Volume / Quality (ThreeD/TetMesh.cs:104-112). */
double o_tet_volume(v3 a, v3 b, v3 c, v3 d);
double o_tet_quality4(v3 a, v3 b, v3 c, v3 d);

/* Triangulated solid (ThreeD/TriMeshSolid.cs:5-180): vertices, triangles, bounding box and its two bucket grids. */
typedef struct {
    int nv, nt;
    double *v;
    int *t;
    double mn[3], mx[3];
    double c2;
    int nx2, ny2;
    int *xy_start, *xy_items;
    double c3;
    int gx, gy, gz;
    int *g3_start, *g3_items;
} o_trimesh;
int o_trimesh_build(o_trimesh *m, int nv, const double *v, int nt, const int *tri);
void o_trimesh_free(o_trimesh *m);

/* Die (ThreeD/HeightFieldDie.cs; kind 1: TriMeshDie, ThreeD/TriMeshSolid.cs:248-297). */
typedef struct { int side; double x0, y0, dx; int nx, ny; double *h; int kind; o_trimesh tm; } o_hfdie;
double hf_height(const o_hfdie *d, double x, double y);
double hf_clearance(const o_hfdie *d, v3 p, double offset);
v3 hf_project(const o_hfdie *d, v3 p, double offset, v3 *normal);

#endif
