// leaf_lists.cpp -- host construction of the reference octree's leaf lists as CSR arrays.
//
// FastMultipoleSolver::build (cpp/fmm/fmm_solver.cpp:48-98) inserts bodies one at a time;
// a leaf splits into 8 children when it would hold more than leaf_capacity bodies and its
// depth is below max_depth (:133-155).  That produces the same tree as the recursive
// 8-way partition below (every node with more than leaf_capacity bodies above max_depth is
// split), and every leaf lists its bodies in ascending index order.  The geometry is
// computed with the reference's operations in the reference's order, so a body lands in
// the same octant (child_index_for, :104-109) and the same well-separated test
// (:228-241) gives the same near lists (build_leaf_interactions, :254-277).  Leaves are
// numbered in the depth-first child order of collect_leaves (:210-226), which skips
// massless subtrees.  The tree must be identical, not merely similar: the P2P sum of the
// drop-in runs over exactly these lists.
#include "gx.h"
#include "fmm_tree.hpp"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <limits>
#include <new>
#include <string>
#include <vector>

extern "C" int gxi_fail(int code, const char* msg);
extern "C" int gxi_leaf_lists_from_device(int64_t n, const double* x, const double* y, const double* z,
                                          const double* m, double softening, double theta, int64_t leaf_capacity,
                                          int max_depth, void* stream, gx::FmmTree* T, int* on_device);

struct gx_leaf_lists {
    gx::FmmTree t;
};

namespace {

struct Node {
    double c[3];
    double hw;
    double mass;
    int child0;  // first of 8 consecutive children, -1 for a leaf
    int64_t beg, end;
    int leaf_id;
    int id;  // breadth-first number
};

struct Builder {
    const double *x, *y, *z, *m;
    int64_t cap;
    int max_depth;
    double theta;
    std::vector<Node> nodes;
    std::vector<int64_t> perm, tmp;

    int octant(const Node& nd, int64_t p) const {
        return (x[p] >= nd.c[0] ? 1 : 0) + 2 * (y[p] >= nd.c[1] ? 1 : 0) + 4 * (z[p] >= nd.c[2] ? 1 : 0);
    }

    void build(int node, int depth) {
        const int64_t beg = nodes[node].beg, end = nodes[node].end;
        if (end - beg <= cap || depth >= max_depth) {
            double mass = 0.0;
            for (int64_t k = beg; k < end; ++k) mass += m[perm[k]];
            nodes[node].mass = mass;
            return;
        }
        const double chw = nodes[node].hw * 0.5;
        const double pc[3] = {nodes[node].c[0], nodes[node].c[1], nodes[node].c[2]};
        const int first = (int)nodes.size();
        for (int c = 0; c < 8; ++c) {
            Node ch{};
            const double sx = (c & 1) ? 1.0 : -1.0, sy = (c & 2) ? 1.0 : -1.0, sz = (c & 4) ? 1.0 : -1.0;
            ch.c[0] = pc[0] + sx * chw;
            ch.c[1] = pc[1] + sy * chw;
            ch.c[2] = pc[2] + sz * chw;
            ch.hw = chw;
            ch.child0 = -1;
            ch.leaf_id = -1;
            nodes.push_back(ch);
        }
        nodes[node].child0 = first;
        int64_t cnt[8] = {0};
        for (int64_t k = beg; k < end; ++k) cnt[octant(nodes[node], perm[k])]++;
        int64_t off[8], run = beg;
        for (int c = 0; c < 8; ++c) {
            off[c] = run;
            run += cnt[c];
        }
        for (int64_t k = beg; k < end; ++k) {
            const int64_t p = perm[k];
            tmp[off[octant(nodes[node], p)]++] = p;
        }
        std::copy(tmp.begin() + beg, tmp.begin() + end, perm.begin() + beg);
        run = beg;
        double mass = 0.0;
        for (int c = 0; c < 8; ++c) {
            nodes[first + c].beg = run;
            nodes[first + c].end = run + cnt[c];
            run += cnt[c];
            build(first + c, depth + 1);
            mass += nodes[first + c].mass;
        }
        nodes[node].mass = mass;
    }

    void collect(int node, std::vector<int>& leaves) {
        Node& nd = nodes[node];
        if (nd.mass <= 0.0) return;
        if (nd.child0 < 0) {
            nd.leaf_id = (int)leaves.size();
            leaves.push_back(node);
            return;
        }
        for (int c = 0; c < 8; ++c) collect(nd.child0 + c, leaves);
    }

    bool well_separated(const Node& t, const Node& s) const {
        if (s.mass <= 0.0) return false;
        const double dx = s.c[0] - t.c[0], dy = s.c[1] - t.c[1], dz = s.c[2] - t.c[2];
        const double dist = std::sqrt(dx * dx + dy * dy + dz * dz);
        if (dist == 0.0) return false;
        const double comb = 2.0 * (t.hw + s.hw);
        return comb / dist < theta;
    }

    void walk(int target, int source, std::vector<int32_t>& near, std::vector<int32_t>* far, int64_t& n_far) const {
        const Node& s = nodes[source];
        if (s.mass <= 0.0) return;
        if (source != target && well_separated(nodes[target], s)) {
            ++n_far;
            if (far) far->push_back(s.id);
            return;
        }
        if (s.child0 < 0) {
            near.push_back(s.leaf_id);
            return;
        }
        for (int c = 0; c < 8; ++c) walk(target, s.child0 + c, near, far, n_far);
    }
};

}  // namespace

namespace gx {

int build_fmm_tree(int64_t n, const double* x, const double* y, const double* z, const double* m,
                   double softening, double theta, int64_t leaf_capacity, int max_depth, bool want_far,
                   FmmTree* out) {
    if (n <= 0 || !x || !y || !z || !m || !out)
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "octree: need n > 0 and x, y, z, m");
    if (n > (int64_t)std::numeric_limits<int32_t>::max())
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "octree: n exceeds the int32 index range");
    try {
        Builder b;
        b.x = x;
        b.y = y;
        b.z = z;
        b.m = m;
        // FastMultipoleSolver constructor clamps (fmm_solver.cpp:12-18)
        b.cap = std::max<int64_t>(1, leaf_capacity);
        b.max_depth = std::max(1, max_depth);
        b.theta = std::max(1.0e-6, theta);
        b.perm.resize((size_t)n);
        b.tmp.resize((size_t)n);
        double mn[3] = {std::numeric_limits<double>::infinity(), std::numeric_limits<double>::infinity(),
                        std::numeric_limits<double>::infinity()};
        double mx[3] = {-mn[0], -mn[1], -mn[2]};
        for (int64_t i = 0; i < n; ++i) {
            b.perm[(size_t)i] = i;
            mn[0] = std::min(mn[0], x[i]);
            mn[1] = std::min(mn[1], y[i]);
            mn[2] = std::min(mn[2], z[i]);
            mx[0] = std::max(mx[0], x[i]);
            mx[1] = std::max(mx[1], y[i]);
            mx[2] = std::max(mx[2], z[i]);
        }
        // root cell (fmm_solver.cpp:77-85)
        Node root{};
        for (int c = 0; c < 3; ++c) root.c[c] = (mn[c] + mx[c]) * 0.5;
        root.hw = 0.5 * std::max({mx[0] - mn[0], mx[1] - mn[1], mx[2] - mn[2]});
        root.hw = std::max(root.hw, softening + 1.0e-6);
        root.hw *= 1.0001;
        root.child0 = -1;
        root.leaf_id = -1;
        root.beg = 0;
        root.end = n;
        b.nodes.reserve((size_t)(n / std::max<int64_t>(1, b.cap)) * 3 + 64);
        b.nodes.push_back(root);
        b.build(0, 0);
        std::vector<int> leaves;
        b.collect(0, leaves);

        FmmTree& T = *out;
        T = FmmTree();
        // breadth-first numbering of every node; the 8 children of a node stay consecutive
        std::vector<int> bfs, depth;
        bfs.reserve(b.nodes.size());
        depth.reserve(b.nodes.size());
        bfs.push_back(0);
        depth.push_back(0);
        b.nodes[0].id = 0;
        for (size_t k = 0; k < bfs.size(); ++k) {
            const Node& nd = b.nodes[bfs[k]];
            if (nd.child0 < 0) continue;
            for (int c = 0; c < 8; ++c) {
                b.nodes[nd.child0 + c].id = (int)bfs.size();
                bfs.push_back(nd.child0 + c);
                depth.push_back(depth[k] + 1);
            }
        }
        const size_t nn = bfs.size();
        T.node_beg.resize(nn);
        T.node_end.resize(nn);
        T.node_child.resize(nn);
        T.node_cx.resize(nn);
        T.node_cy.resize(nn);
        T.node_cz.resize(nn);
        T.node_hw.resize(nn);
        for (size_t k = 0; k < nn; ++k) {
            const Node& nd = b.nodes[bfs[k]];
            T.node_beg[k] = (int32_t)nd.beg;
            T.node_end[k] = (int32_t)nd.end;
            T.node_child[k] = nd.child0 < 0 ? -1 : b.nodes[nd.child0].id;
            T.node_cx[k] = nd.c[0];
            T.node_cy[k] = nd.c[1];
            T.node_cz[k] = nd.c[2];
            T.node_hw[k] = nd.hw;
        }
        T.level_off.assign(depth.back() + 2, 0);
        for (size_t k = 0; k < nn; ++k) T.level_off[depth[k] + 1] = (int32_t)(k + 1);
        T.perm.resize((size_t)n);
        for (int64_t k = 0; k < n; ++k) T.perm[(size_t)k] = (int32_t)b.perm[(size_t)k];

        const size_t nl = leaves.size();
        T.leaf_off.resize(nl + 1);
        T.near_off.resize(nl + 1);
        T.far_off.resize(nl + 1);
        T.leaf_node.resize(nl);
        T.leaf_part.reserve((size_t)n);
        for (size_t l = 0; l < nl; ++l) {
            const Node& nd = b.nodes[leaves[l]];
            T.leaf_node[l] = nd.id;
            T.leaf_off[l] = (int32_t)T.leaf_part.size();
            for (int64_t k = nd.beg; k < nd.end; ++k) T.leaf_part.push_back((int32_t)b.perm[(size_t)k]);
        }
        T.leaf_off[nl] = (int32_t)T.leaf_part.size();
        std::vector<int32_t> near;
        for (size_t l = 0; l < nl; ++l) {
            T.near_off[l] = (int32_t)T.near_leaf.size();
            T.far_off[l] = (int32_t)T.far_node.size();
            near.clear();
            b.walk(leaves[l], 0, near, want_far ? &T.far_node : nullptr, T.n_far);
            const int64_t nt = T.leaf_off[l + 1] - T.leaf_off[l];
            for (int32_t s : near) {
                T.near_leaf.push_back(s);
                T.n_pairs += nt * (int64_t)(T.leaf_off[s + 1] - T.leaf_off[s]);
            }
            if (T.near_leaf.size() > (size_t)std::numeric_limits<int32_t>::max() ||
                T.far_node.size() > (size_t)std::numeric_limits<int32_t>::max())
                return gxi_fail(GX_ERR_INVALID_ARGUMENT, "octree: interaction lists exceed the int32 range");
        }
        T.near_off[nl] = (int32_t)T.near_leaf.size();
        T.far_off[nl] = (int32_t)T.far_node.size();
        return GX_OK;
    } catch (const std::bad_alloc&) {
        return gxi_fail(GX_ERR_OUT_OF_MEMORY, "octree: host allocation failed");
    }
}

}  // namespace gx

extern "C" int gx_leaf_lists_build(int64_t n, const double* x, const double* y, const double* z,
                                   const double* m, double softening, double theta,
                                   int64_t leaf_capacity, int max_depth, gx_leaf_lists** out) {
    if (!out) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_leaf_lists_build: out is null");
    *out = nullptr;
    if (n <= 0 || !x || !y || !z || !m)
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_leaf_lists_build: need n > 0 and x, y, z, m");
    if (n > (int64_t)std::numeric_limits<int32_t>::max())
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_leaf_lists_build: n exceeds the int32 index range");
    gx_leaf_lists* L = new (std::nothrow) gx_leaf_lists();
    if (!L) return gxi_fail(GX_ERR_OUT_OF_MEMORY, "gx_leaf_lists_build: host allocation failed");
    const int rc = gx::build_fmm_tree(n, x, y, z, m, softening, theta, leaf_capacity, max_depth, false, &L->t);
    if (rc != GX_OK) {
        delete L;
        return rc;
    }
    *out = L;
    return GX_OK;
}

extern "C" int gx_leaf_lists_build_device(int64_t n, const double* x, const double* y, const double* z,
                                          const double* m, double softening, double theta, int64_t leaf_capacity,
                                          int max_depth, void* stream, gx_leaf_lists** out, int* built_on_device) {
    if (!out) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_leaf_lists_build_device: out is null");
    *out = nullptr;
    if (n <= 0 || !x || !y || !z || !m)
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_leaf_lists_build_device: need n > 0 and x, y, z, m");
    gx_leaf_lists* L = new (std::nothrow) gx_leaf_lists();
    if (!L) return gxi_fail(GX_ERR_OUT_OF_MEMORY, "gx_leaf_lists_build_device: host allocation failed");
    int dev = 0;
    const int rc = gxi_leaf_lists_from_device(n, x, y, z, m, softening, theta, leaf_capacity, max_depth, stream, &L->t,
                                              &dev);
    if (rc != GX_OK) {
        delete L;
        return rc;
    }
    if (built_on_device) *built_on_device = dev;
    *out = L;
    return GX_OK;
}

extern "C" int gx_leaf_lists_info(const gx_leaf_lists* l, int32_t* n_leaves, int64_t* n_leaf_particles,
                                  int64_t* n_near, int64_t* n_far, int64_t* n_p2p_pairs) {
    if (!l) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_leaf_lists_info: null handle");
    if (n_leaves) *n_leaves = l->t.n_leaves();
    if (n_leaf_particles) *n_leaf_particles = (int64_t)l->t.leaf_part.size();
    if (n_near) *n_near = (int64_t)l->t.near_leaf.size();
    if (n_far) *n_far = l->t.n_far;
    if (n_p2p_pairs) *n_p2p_pairs = l->t.n_pairs;
    return GX_OK;
}

extern "C" int gx_leaf_lists_export(const gx_leaf_lists* l, int32_t* leaf_offsets, int32_t* leaf_particles,
                                    int32_t* near_offsets, int32_t* near_leaves) {
    if (!l) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_leaf_lists_export: null handle");
    if (leaf_offsets) std::copy(l->t.leaf_off.begin(), l->t.leaf_off.end(), leaf_offsets);
    if (leaf_particles) std::copy(l->t.leaf_part.begin(), l->t.leaf_part.end(), leaf_particles);
    if (near_offsets) std::copy(l->t.near_off.begin(), l->t.near_off.end(), near_offsets);
    if (near_leaves) std::copy(l->t.near_leaf.begin(), l->t.near_leaf.end(), near_leaves);
    return GX_OK;
}

extern "C" int gx_leaf_lists_free(gx_leaf_lists* l) {
    delete l;
    return GX_OK;
}
