// multifrontal.h — symbolic analysis of the GPU multifrontal sparse Cholesky (host side).
//
// Pipeline (once per sparsity pattern): nested-dissection order of the node graph (METIS through cuSOLVER's host
// helper), elimination tree and its postorder, column counts, supernodes (columns whose factor structure nests),
// the row structure of every supernode, the frontal-matrix layout, the child->parent index maps of the
// extend-add, and the level schedule (a supernode's level = 1 + the highest level of its children).
#pragma once
#include <cstdint>
#include <memory>
#include <string>
#include <utility>
#include <vector>

namespace ifea {

// Allocator whose resize() leaves new elements uninitialised (for arrays that are written in full right after).
template <class T>
struct UninitAlloc : std::allocator<T> {
    template <class U>
    struct rebind {
        using other = UninitAlloc<U>;
    };
    UninitAlloc() = default;
    template <class U>
    UninitAlloc(const UninitAlloc<U> &) noexcept {}
    template <class U>
    void construct(U *p) noexcept
    {
        ::new ((void *)p) U;
    }
    template <class U, class... A>
    void construct(U *p, A &&...a)
    {
        ::new ((void *)p) U(std::forward<A>(a)...);
    }
};

struct MfSymbolic {
    int n = 0, nsuper = 0, nlevels = 0;
    std::vector<int32_t> perm, pinv;              // new -> old, old -> new
    // supernodes (columns [c0, c1) in the new numbering)
    std::vector<int32_t> c0, ncol, m, parent, level;
    std::vector<int64_t> front_off;               // offset of the m x m column-major front in the pool
    int64_t pool = 0;                              // total doubles of all fronts
    std::vector<int32_t> idx_start, idx;          // global (new) row index of each front row
    std::vector<int32_t> relmap_start, relmap;    // struct rows of s -> row position in parent's front
    std::vector<int32_t> uvec_start;              // offset of s's update vector (nrow) in the solve pool
    int64_t uvec_pool = 0;
    // original-value scatter: dst offset in the pool <- src index into the full CSC value array
    std::vector<int64_t, UninitAlloc<int64_t>> a_dst;
    std::vector<int32_t, UninitAlloc<int32_t>> a_src;
    std::vector<int32_t> a_level_start;           // a_dst/a_src ranges per level (fronts are stored by level)
    // level schedule
    std::vector<int32_t> level_start, level_list;  // supernodes of each level (ascending index)
    std::vector<int64_t> level_pool_start;         // pool range of each level's fronts (contiguous)
    // extend-add: per (level, child rank r) the children c whose parent lies in that level
    std::vector<int32_t> ext_start, ext_child;     // index = level * max_rank + r
    int max_rank = 0;
    int64_t factor_nnz = 0;
    int max_m = 0, max_ncol = 0;
    double order_s = 0;  // host seconds spent in the nested-dissection ordering (METIS) of the last analysis

    // Full symmetric CSC pattern (both triangles) of an n x n matrix; block = 3 orders 3x3 node blocks together.
    // The node order is METIS nested dissection through cuSOLVER's host helper, or, when node_xyz (3 coordinates
    // per node) is given, this file's coordinate nested dissection (coordinate_nd).
    // node_start / node_list (block > 1): each node's neighbours, itself included, ascending, for a caller that built
    // col_ptr / row_idx as the full block x block pattern of exactly these lists with ascending rows (the stepper's
    // TetTopology): the node graph is read from them and the pattern's node structure is not verified again.
    std::string analyze(int n, const int32_t *col_ptr, const int32_t *row_idx, int block, void *cusolver_sp_handle,
                        void *mat_descr, const double *node_xyz = nullptr, const int32_t *node_start = nullptr,
                        const int32_t *node_list = nullptr);
};

}  // namespace ifea
