// remesh.h — host-side remeshing of the 3D workpiece and the remap of its state (Forging3DSolver.RemeshCore,
// ThreeD/Forging3DSolver.cs:1958-2145): isosurface stuffing of the deformed body, local refinement, contact
// placement on the dies, volume compensation, quality repair, then element and nodal fields carried over from the
// old mesh through a point locator.
#pragma once
#include <functional>
#include <string>
#include <vector>

#include "common.cuh"

namespace ifea {

// Bucket grid over the tets of a mesh for point location (TetLocator, ThreeD/TetMesh.cs:116-263).
class TetLocator {
  public:
    TetLocator(const std::vector<d3> &x, const std::vector<int32_t> &tets, double cell);
    // containing tet and barycentric weights, or -1
    int find(d3 p, double w[4]) const;
    bool contains(d3 p) const
    {
        double w[4];
        return find(p, w) >= 0;
    }
    // linear interpolation of a nodal field (3 per node); the nearest node's value outside the mesh
    d3 interpolate(d3 p, const double *field) const;
    // containing tet, else the tet whose centroid is nearest (first in the point's cell, else over all)
    int find_nearest(d3 p) const;

    // the nearest node (the lowest index among equally near ones)
    int nearest_node(d3 p) const;

  private:
    int cell_of(d3 p) const;
    const std::vector<d3> &x_;
    const std::vector<int32_t> &t_;
    double cell_;
    d3 min_;
    int nx_, ny_, nz_;
    std::vector<int32_t> start_, items_, nstart_, nitems_;
    // each tet's bounding box (min xyz, max xyz), widened by bb_margin_: a point outside it fails the containment
    // test, so find() skips such candidates before the volume arithmetic and returns the same tet
    std::vector<double> bb_;
    double bb_margin_ = 0;
};

// Isosurface stuffing on the body-centred-cubic lattice of spacing h (IsosurfaceStuffing.Stuff,
// ThreeD/IsosurfaceStuffing.cs:19-277; Labelle and Shewchuk 2007). Positively oriented tets.
// With parallel, inside() is called from several host threads at once.
void stuff_uniform(const std::function<bool(d3)> &inside, d3 lo, d3 hi, double h, bool sym_x, bool sym_y,
                   std::vector<d3> &pts, std::vector<int32_t> &tets, bool parallel);

// Longest-edge bisection until every tet's longest edge is at most 1.05 target(centroid), within max_nodes
// (TetRefiner.Refine, ThreeD/TetRefiner.cs:14-158). Returns the number of edge splits.
int refine_tets(std::vector<d3> &pts, std::vector<int32_t> &tets, const std::function<double(d3)> &target,
                int max_nodes);

struct HotSpot {
    d3 at;
    int level;
};

struct RemeshInput {
    int nn = 0, ne = 0;
    const double *x = nullptr;       // 3 per node
    const int32_t *tets = nullptr;   // 4 per tet
    const double *vg = nullptr;      // global velocity, 3 per node
    const double *eps = nullptr, *dmg = nullptr, *sig = nullptr, *rate = nullptr, *mean = nullptr;  // per tet
    HField die[2];                   // bottom, top (closed position); h on the host
    double gap = 0, h = 0, vol_target = 0;  // vol_target: the initial volume of the modelled part
    bool sym_x = true, sym_y = true;
    int recovery_pass = 0, refinement_levels = 1, max_nodes = 1 << 30;
    double sig_ref = 0;
    std::vector<HotSpot> hot;
    // called once the new mesh's connectivity is final (after refinement, before the surface is extracted and
    // contact placement moves its nodes): node positions so far, tets, symmetry-plane flags. A caller can start
    // work that needs only the connectivity (topology, symbolic analysis) while the remesher places and remaps;
    // the mesh may still be rejected after the call (not manifold, too poor).
    std::function<void(const std::vector<d3> &, const std::vector<int32_t> &, const std::vector<uint8_t> &,
                       const std::vector<uint8_t> &)>
        on_topology;
};

struct RemeshOutput {
    std::vector<double> x, vg, eps, dmg, sig, rate, mean;
    std::vector<int32_t> tets;
    std::vector<uint8_t> on_x0, on_y0, contact;
    double q_old = 0, q_new = 0;
    int splits = 0;
    std::string why;  // the reason a remesh was rejected
    double t_stuff = 0, t_refine = 0, t_place = 0, t_remap = 0;  // host seconds of the phases
};

// true: accepted (out holds the new mesh and state); false: rejected, out.why says why
bool remesh_workpiece(const RemeshInput &in, RemeshOutput &out);

}  // namespace ifea
