// Host-side analysis driver for the CPU tests: builds the library's tetrahedral topology (mesh3d.cpp) and the
// multifrontal symbolic analysis (multifrontal.cpp) from a mesh file and writes every array they produce.
//
// usage: host_analysis_driver <mesh.bin> <out.bin> <block> [xyz]
//   mesh.bin: int32 nn, ne; float64 x[3 nn]; int32 tets[4 ne]; uint8 on_x0[nn], on_y0[nn]
//   out.bin:  records (char name[24], int32 element bytes, int64 count, data)
// The symbolic analysis runs without a cuSOLVER handle, i.e. in the identity node order, or with "xyz" in the
// coordinate nested-dissection order.
//        host_analysis_driver quad <nx> <ny> <out.bin>
//   the structured quad mesh of the 2D path (mesh2d.cpp): numbering, boundary loop and band gather maps.
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "mesh2d.h"
#include "mesh3d.h"
#include "multifrontal.h"

namespace {
FILE *out = nullptr;

template <class V>
void put(const char *name, const V &v)
{
    char nm[24] = {0};
    std::strncpy(nm, name, sizeof nm - 1);
    int32_t eb = (int32_t)sizeof(typename V::value_type);
    int64_t n = (int64_t)v.size();
    std::fwrite(nm, 1, sizeof nm, out);
    std::fwrite(&eb, 4, 1, out);
    std::fwrite(&n, 8, 1, out);
    if (n) std::fwrite(v.data(), eb, v.size(), out);
}

template <class T>
bool get(FILE *f, std::vector<T> &v, size_t n)
{
    v.resize(n);
    return std::fread(v.data(), sizeof(T), n, f) == n;
}
}  // namespace

int quad(int nx, int ny, const char *path)
{
    ifea::QuadTopology q;
    std::vector<double> x;
    std::string e = q.build_structured(nx, ny, 1.0, 0.0, 1.0, x);
    if (!e.empty()) {
        std::fprintf(stderr, "quad: %s\n", e.c_str());
        return 5;
    }
    out = std::fopen(path, "wb");
    if (!out) return 7;
    std::vector<int64_t> sc = {q.nn, q.ne, q.ndof, q.half_band, q.nloop};
    put("quad_scalars", sc), put("conn", q.conn), put("is_axis", q.is_axis), put("eq", q.eq), put("loop", q.loop);
    put("loop_owner", q.loop_owner), put("cell_ptr", q.cell_ptr), put("cell_idx", q.cell_idx);
    put("cell_src", q.cell_src), put("dof_ptr", q.dof_ptr), put("dof_src", q.dof_src), put("node_edge", q.node_edge);
    std::fclose(out);
    return 0;
}

int main(int argc, char **argv)
{
    if (argc == 5 && std::strcmp(argv[1], "quad") == 0) return quad(std::atoi(argv[2]), std::atoi(argv[3]), argv[4]);
    if (argc != 4 && argc != 5) return 2;
    // optional 4th argument: "xyz" (coordinate dissection), "lists" (coordinate dissection, the node graph passed
    // as the topology's node lists)
    bool lists = argc == 5 && std::strcmp(argv[4], "lists") == 0;
    bool xyz = lists || (argc == 5 && std::strcmp(argv[4], "xyz") == 0);
    FILE *f = std::fopen(argv[1], "rb");
    if (!f) return 3;
    int32_t hdr[2];
    std::vector<double> x;
    std::vector<int32_t> t;
    std::vector<uint8_t> ox, oy;
    bool ok = std::fread(hdr, 4, 2, f) == 2 && get(f, x, 3 * (size_t)hdr[0]) && get(f, t, 4 * (size_t)hdr[1]) &&
              get(f, ox, hdr[0]) && get(f, oy, hdr[0]);
    std::fclose(f);
    if (!ok) return 4;

    ifea::TetTopology topo;
    std::string e = topo.build(hdr[0], hdr[1], x.data(), t.data(), ox.data(), oy.data());
    if (!e.empty()) {
        std::fprintf(stderr, "topology: %s\n", e.c_str());
        return 5;
    }
    ifea::MfSymbolic S;
    e = S.analyze(topo.ndof, topo.col_ptr.data(), topo.row_idx.data(), std::atoi(argv[3]), nullptr, nullptr,
                  xyz ? x.data() : nullptr, lists ? topo.nbr_start.data() : nullptr, lists ? topo.nbr.data() : nullptr);
    if (!e.empty()) {
        std::fprintf(stderr, "symbolic: %s\n", e.c_str());
        return 6;
    }
    out = std::fopen(argv[2], "wb");
    if (!out) return 7;
    put("nts", topo.nts), put("ntl", topo.ntl), put("bface", topo.bface), put("bowner", topo.bowner);
    put("bsym", topo.bsym), put("is_surface", topo.is_surface), put("nfs", topo.nfs), put("nfl", topo.nfl);
    put("nbr_start", topo.nbr_start), put("nbr", topo.nbr), put("col_ptr", topo.col_ptr);
    put("row_idx", topo.row_idx), put("e_nbr", topo.e_nbr), put("qk", topo.qk), put("diag_slot", topo.diag_slot);
    put("g_start", topo.g_start), put("g_node", topo.g_node), put("gslot", topo.gslot);
    put("kv_start", topo.kv_start), put("kv_n", topo.kv_n), put("kv_pj", topo.kv_pj);
    put("kv_kstart", topo.kv_kstart), put("kv_k", topo.kv_k);
    std::vector<int64_t> sc = {S.n, S.nsuper, S.nlevels, S.pool, S.uvec_pool, S.max_rank, S.factor_nnz, S.max_m,
                               S.max_ncol};
    put("sym_scalars", sc);
    put("perm", S.perm), put("pinv", S.pinv), put("c0", S.c0), put("ncol", S.ncol), put("m", S.m);
    put("parent", S.parent), put("level", S.level), put("front_off", S.front_off), put("idx_start", S.idx_start);
    put("idx", S.idx), put("relmap_start", S.relmap_start), put("relmap", S.relmap), put("uvec_start", S.uvec_start);
    put("a_dst", S.a_dst), put("a_src", S.a_src), put("a_level_start", S.a_level_start);
    put("level_start", S.level_start), put("level_list", S.level_list), put("level_pool_start", S.level_pool_start);
    put("ext_start", S.ext_start), put("ext_child", S.ext_child);
    std::fclose(out);
    return 0;
}
