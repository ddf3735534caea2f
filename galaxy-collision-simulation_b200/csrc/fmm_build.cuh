// fmm_build.cuh -- the reference octree and its interaction lists built on the device.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gx {

constexpr int kKeyLevels = 21;  // octant levels a 63-bit path key resolves
constexpr int kBboxBlocks = 296;

// Tree topology from the bodies (layout of fmm_tree.hpp).  Capacity is the number of node
// slots allocated; hdr receives {n_nodes, n_levels, overflow} where overflow is 1 when a
// node below kKeyLevels still has to split (the host builder takes such trees) and 2 when
// the node slots ran out.
struct TreeBuildArgs {
    int32_t n;
    const double* x;
    const double* y;
    const double* z;
    double softening;
    int64_t cap;
    int max_depth;
    int32_t capacity;
    double* part;     // bbox partials, 6 * kBboxBlocks
    double* root;     // cx, cy, cz, hw
    uint64_t* keys;   // n, then sorted in place through keys_alt
    uint64_t* keys_alt;
    int32_t* idx;     // n
    int32_t* perm;    // n: bodies in tree order
    int32_t* beg;     // capacity each
    int32_t* end;
    int32_t* child;
    double* cx;
    double* cy;
    double* cz;
    double* hw;
    int32_t* level_off;  // kKeyLevels + 3
    int32_t* hdr;        // 3
    // Levels of the key that the sort orders (0: all kKeyLevels).  Fewer levels take fewer
    // radix passes; a tree that would split a node at that depth sets hdr[2] bit 2 instead
    // (the caller rebuilds with more levels).
    int key_levels;
};
size_t tree_build_temp_bytes(int32_t n, int64_t cap);
cudaError_t launch_tree_build(const TreeBuildArgs& t, void* temp, size_t temp_bytes, cudaStream_t st);
// After a successful build: bodies of every leaf in ascending index order in t.perm
// (uses t.idx as scratch).
cudaError_t launch_tree_leaf_order(const TreeBuildArgs& t, int32_t n_nodes, void* temp, size_t temp_bytes,
                                   cudaStream_t st);

// What the list walk reads of a node, packed (56 B); mask has bit c set when child c has
// mass > 0.
struct WalkNode {
    double cx, cy, cz, hw;
    double mass;
    int32_t child;
    int32_t beg, end;
    int32_t mask;
};

// Leaves with mass > 0 (depth-first) and their near / far lists, after the node moments.
struct TreeListArgs {
    int32_t n;
    int32_t n_nodes;
    const int32_t* beg;
    const int32_t* end;
    const int32_t* child;
    const int32_t* perm;
    const double* cx;
    const double* cy;
    const double* cz;
    const double* hw;
    const double* rec;  // node records (mass at slot 3)
    // Optional (capacity mode): the bodies' masses and, filled by launch_tree_massive, the
    // number of bodies with mass > 0 before each tree position (n + 1).  With all masses
    // finite and >= 0 a node's mass is > 0 exactly when its range holds such a body, so the
    // lists then need no node records and can be built while the moments are computed.
    const double* m;
    int32_t* mprefix;
    WalkNode* wn;       // n_nodes, filled before the walk
    double theta;
    int64_t t_begin, t_end;
    // body-position scratch, n + 1 each
    int32_t* start_flag;
    int32_t* start_ord;
    int32_t* keep;
    int32_t* newpos;
    // leaves, n_nodes + 1 each
    int32_t* leaf_off;
    int32_t* leaf_part;  // n
    int32_t* leaf_node;
    int32_t* node_leaf;  // n_nodes
    // per-leaf counts and their exclusive sums, n_nodes + 1 each
    int32_t* far_cnt;
    int32_t* near_cnt;
    int32_t* item_cnt;
    int32_t* slot_cnt;
    int32_t* far_off;
    int32_t* near_off;
    int32_t* item_off;
    int32_t* slot_off;
    unsigned long long* totals;  // 6: far, near, items, slots (overflow check), far and near body pairs
    // fill pass: the near lists unsorted (leaf ordinals), then sorted into near_leaf
    uint64_t* near_key;
    int32_t* long_leaf;   // leaves whose near lists are sorted by a separate kernel
    int32_t* long_count;
    int32_t* far_node;
    int32_t* near_leaf;
    void* items;  // M2PItem
    // Capacity mode (nullable cnt_nodes / overflow): n_nodes is the capacity of the node
    // arrays and the count is read on the device (cnt_nodes = the topology build's header
    // {nodes, levels, flags}; a flag leaves no nodes); far/near/item/slot pools were reserved
    // by capacity, pool_check marks an overflow when a total exceeds its pool (and records the
    // largest totals seen in need[5], with a sticky copy of the flag), and the fill pass and
    // everything after it are skipped.
    const int32_t* cnt_nodes;
    int* overflow;
    int* overflow_sticky;
    unsigned long long* need;  // {nodes, far, near, items, slots}
    int64_t far_cap, near_cap, item_cap, slot_cap;
};
size_t tree_list_temp_bytes(int32_t n, int32_t n_nodes);
// Leaf compaction, the count walk and the offsets (sizes become known on the host after it).
cudaError_t launch_tree_lists_count(const TreeListArgs& a, void* temp, size_t temp_bytes, cudaStream_t st);
// Capacity mode: after the count pass, the overflow check of the pools (and of the topology
// build's header tree_hdr).
// mprefix from the masses (a.m, a.perm); a mass < 0 or NaN marks an overflow with bit 1 of
// the sticky word (the caller then evaluates through the host-read path).  temp: scan scratch
// for n + 1 ints.
cudaError_t launch_tree_massive(const TreeListArgs& a, void* temp, size_t temp_bytes, cudaStream_t st);
cudaError_t launch_pool_check(const TreeListArgs& a, const int32_t* tree_hdr, cudaStream_t st);
// The fill walk (each leaf's lists sorted into depth-first order) and the far-field work items.
cudaError_t launch_tree_lists_fill(const TreeListArgs& a, int32_t n_leaves, cudaStream_t st);
// The far-field items reordered by decreasing cost (targets x nodes) into out.
struct M2PItem;
size_t item_order_temp_bytes(int32_t n_items);
// n_items is the length of the arrays; n_real (nullable: all) the items on the device.
cudaError_t launch_item_order(const M2PItem* items, const int32_t* leaf_off, int32_t n_items,
                              const unsigned long long* n_real, const int* overflow, uint32_t* cost,
                              uint32_t* cost_alt, int32_t* idx, int32_t* idx_alt, void* temp, size_t temp_bytes,
                              M2PItem* out, cudaStream_t st);

}  // namespace gx
