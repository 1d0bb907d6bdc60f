// mesh3d.h — host-side topology of a tetrahedral workpiece and the index maps the device kernels use.
//
// Everything here is integer work done once per mesh (the reference does it in the TetMesh constructor,
// Forging3DSolver.Allocate/BuildPattern and EnsureElementBuffers); it must match the reference bit for bit.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace ifea {

struct TetTopology {
    int nn = 0, ne = 0, ndof = 0;
    std::vector<int32_t> tets;                 // 4 per element
    std::vector<uint8_t> on_x0, on_y0;
    // node -> tet CSR in ascending element order (TetMesh.NodeTetStart/List, ThreeD/TetMesh.cs:18-29)
    std::vector<int32_t> nts, ntl;
    std::vector<int8_t> ntl_local;             // position of the node inside each listed tet
    // boundary faces in Dictionary insertion order (ThreeD/TetMesh.cs:31-64)
    std::vector<int32_t> bface, bowner;
    std::vector<uint8_t> bsym, is_surface;
    // node -> non-symmetry boundary faces, in face order (for friction areas and surface normals)
    std::vector<int32_t> nfs, nfl;
    // sorted two-ring neighbours (BuildPattern, Forging3DSolver.cs:469-494)
    std::vector<int32_t> nbr_start, nbr;
    // full symmetric CSC in 3x3 node blocks (Forging3DSolver.cs:496-515)
    std::vector<int32_t> col_ptr, row_idx;
    int64_t nnz = 0;
    int32_t max_nbr = 0;
    // eNbr slot map (Forging3DSolver.cs:1248-1261) and, per node-tet entry q, the slot of each of the tet's
    // four nodes in the column node's neighbour list: qk[4*q + a] = eNbr[16*e + 4*a + b]
    std::vector<int32_t> e_nbr, qk;
    std::vector<int32_t> diag_slot;            // value index of each diagonal entry (Pos(n,c,n,c))
    // averaged-nodal-pressure patches (BuildAnp, Forging3DSolver.cs:774-795): per node n, its patch nodes in
    // first-encounter order, and for each node-tet entry the patch slot of every node of that tet
    std::vector<int32_t> g_start, g_node, gslot;
    // K_vol gather lists: for column node j, the ring nodes n (ascending), the slot of j in n's patch, and for
    // every patch entry of n the position of that node in nbr[j]
    std::vector<int32_t> kv_start, kv_n, kv_pj, kv_kstart, kv_k;

    std::string build(int nn, int ne, const double *x, const int32_t *tets, const uint8_t *on_x0,
                      const uint8_t *on_y0);
};

// LocalLengths (Forging3DSolver.cs:443-466): mean edge length at each node, capped at h.
std::vector<double> local_lengths(const TetTopology &t, const double *x, double h);

}  // namespace ifea
