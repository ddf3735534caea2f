// fmm_tree.hpp -- the reference octree as flat arrays.
//
// The tree, its leaves and its interaction lists are those of FastMultipoleSolver::build
// (cpp/fmm/fmm_solver.cpp:48-98): same geometry, same leaf set (collect_leaves skips
// massless subtrees, :210-226), same near and far lists in the same order
// (build_leaf_interactions, :254-277).  Layout, shared by the host builder below and the
// device builder (fmm_build.cu):
//   * every node the reference creates, numbered breadth-first: each level is a contiguous
//     range and the 8 children of a split node are consecutive, in octant order;
//   * a node owns the bodies perm[beg .. end) (perm = bodies in depth-first tree order,
//     ascending index within a leaf);
//   * leaves with mass > 0 in depth-first order as CSR arrays, with their near leaves
//     (leaf ordinals) and far nodes (node ids) in walk order.
#pragma once

#include <cstdint>
#include <vector>

namespace gx {

struct FmmTree {
    // all nodes, breadth-first
    std::vector<int32_t> node_beg, node_end;
    std::vector<int32_t> node_child;  // first of 8 children, -1 for a leaf
    std::vector<double> node_cx, node_cy, node_cz, node_hw;
    std::vector<int32_t> level_off;  // nodes of level d: [level_off[d], level_off[d + 1])
    std::vector<int32_t> perm;       // n bodies in tree order
    // leaves with mass > 0, depth-first
    std::vector<int32_t> leaf_off;   // n_leaves + 1
    std::vector<int32_t> leaf_part;  // body indices, ascending within a leaf
    std::vector<int32_t> leaf_node;  // node id of each leaf
    std::vector<int32_t> near_off;   // n_leaves + 1
    std::vector<int32_t> near_leaf;  // leaf ordinals, walk order
    std::vector<int32_t> far_off;    // n_leaves + 1
    std::vector<int32_t> far_node;   // node ids, walk order
    int64_t n_far = 0;    // far-list entries
    int64_t n_pairs = 0;  // P2P target-source pairs, self pairs included
    int32_t n_leaves() const { return (int32_t)leaf_off.size() - 1; }
    int32_t n_nodes() const { return (int32_t)node_child.size(); }
    int32_t n_levels() const { return (int32_t)level_off.size() - 1; }
};

// Builds the tree on the host; when want_far is false the far lists are counted but not
// stored.  Returns a GX_* status (the message is recorded for gx_last_error).
int build_fmm_tree(int64_t n, const double* x, const double* y, const double* z, const double* m,
                   double softening, double theta, int64_t leaf_capacity, int max_depth, bool want_far,
                   FmmTree* out);

}  // namespace gx
