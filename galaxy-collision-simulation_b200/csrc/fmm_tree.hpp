// fmm_tree.hpp -- the reference octree as flat arrays (host side).
//
// The tree, its leaves and its interaction lists are those of FastMultipoleSolver::build
// (cpp/fmm/fmm_solver.cpp:48-98): same geometry, same leaf set (collect_leaves skips
// massless subtrees, :210-226), same near and far lists in the same order
// (build_leaf_interactions, :254-277).  Only nodes with mass > 0 are numbered; they are
// numbered breadth-first so the massive children of a node are consecutive and every
// level is a contiguous range (the device's upward pass walks levels bottom-up).
#pragma once

#include <cstdint>
#include <vector>

namespace gx {

struct FmmTree {
    // leaves (mass > 0) in the depth-first order of collect_leaves
    std::vector<int32_t> leaf_off;   // n_leaves + 1
    std::vector<int32_t> leaf_part;  // body indices, ascending within a leaf
    std::vector<int32_t> near_off;   // n_leaves + 1
    std::vector<int32_t> near_leaf;  // leaf ordinals, walk order
    std::vector<int32_t> leaf_node;  // node id of each leaf
    // nodes (mass > 0), breadth-first
    std::vector<int32_t> node_child;   // first massive child, -1 for a leaf
    std::vector<int32_t> node_nchild;  // number of massive children
    std::vector<int32_t> level_off;    // internal nodes of each level: level_node[level_off[d] ..]
    std::vector<int32_t> level_node;
    std::vector<int32_t> far_off;   // n_leaves + 1
    std::vector<int32_t> far_node;  // node ids, walk order
    int64_t all_nodes = 0;  // every node the reference creates, massless ones included
    int64_t n_far = 0;      // far-list entries
    int64_t n_pairs = 0;    // P2P target-source pairs, self pairs included
    int32_t n_leaves() const { return (int32_t)leaf_off.size() - 1; }
    int32_t n_nodes() const { return (int32_t)node_child.size(); }
};

// Builds the tree; when want_far is false the far lists are counted but not stored.
// Returns a GX_* status (the message is recorded for gx_last_error).
int build_fmm_tree(int64_t n, const double* x, const double* y, const double* z, const double* m,
                   double softening, double theta, int64_t leaf_capacity, int max_depth, bool want_far,
                   FmmTree* out);

}  // namespace gx
