// mesh2d.h — host-side topology of the 2D quad mesh (Mesh/QuadMesh.cs) and the band-assembly maps.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace ifea {

struct QuadTopology {
    int nn = 0, ne = 0, ndof = 0, half_band = 0, nloop = 0;
    std::vector<int32_t> conn;        // 4 per element, counter-clockwise
    std::vector<uint8_t> is_axis;
    std::vector<int32_t> eq;          // equation block of each node (reverse Cuthill–McKee, QuadMesh.cs:82-141)
    std::vector<int32_t> loop, loop_owner;  // boundary loop (QuadMesh.cs:173-221)
    // band assembly gather maps (element order): cells that receive element entries, and their contributions
    // as e*64 + 8p + q; residual contributions per DOF as e*8 + p
    std::vector<int32_t> cell_ptr, cell_idx, cell_src;
    std::vector<int32_t> dof_ptr, dof_src;
    // for each node, the (at most two) boundary-loop edges that touch it, in loop order
    std::vector<int32_t> node_edge;   // 2 per node, -1 when absent

    // Structured nx x ny grid over [0, r] x [y0, y0 + h] (QuadMesh.Structured, :51-80); coordinates to x.
    std::string build_structured(int nx, int ny, double r, double y0, double h, std::vector<double> &x);
    int64_t band_size() const { return (int64_t)ndof * (half_band + 1); }
    int64_t band_index(int i, int j) const { return (int64_t)i * (half_band + 1) + (j - i + half_band); }
};

}  // namespace ifea
