// fmm.cuh -- launchers of the FMM far field: leaf moments (P2M), the upward pass (M2M)
// and the multipole evaluation at the targets (M2P).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gx {

// One node record, 48 doubles (384 B):
//   [0..2]   centre of mass        [3]      mass
//   [4..34]  raw moments sum m u^a, u = body - centre of mass, for the 31 multi-indices a
//            of degree 2..4 in the reference's exponent order (multipole.cpp:16-26),
//            so record[k] is the reference's moment values[k]
//   [35]     trace of the degree-2 moments            sum m |u|^2
//   [36..38] traces of the degree-3 moments           sum m |u|^2 u_i
//   [39..44] traces of the degree-4 moments (xx xy xz yy yz zz)  sum m |u|^2 u_i u_j
//   [45]     double trace                             sum m |u|^4
constexpr int kFmmRec = 48;
constexpr int kRecMass = 3, kRecMom = 4, kRecTrQ = 35, kRecW = 36, kRecT2 = 39, kRecTr2 = 45;

// The record of the mixed-precision far field, 52 floats (208 B): the centre of mass as
// three doubles in floats [0..5] (offsets to the targets are taken in FP64), then slots
// 3..45 of the FP64 record rounded to FP32 in floats [6..48], zero padding to [51].
constexpr int kRec32 = 52;

// Far-field work item: one target leaf and a chunk of its far list.
struct M2PItem {
    int32_t leaf;
    int32_t fb, fe;   // far_node[fb .. fe)
    int32_t chunk;    // index of this chunk among the leaf's chunks
    int32_t nchunks;
    int32_t pad;
    int64_t scratch;  // first partial-sum slot of the leaf (targets), when nchunks > 1
};

struct FmmArgs {
    const double* x;
    const double* y;
    const double* z;
    const double* m;
    // every node, breadth-first (each level contiguous, the 8 children of a node consecutive)
    int32_t n_nodes;
    const int32_t* node_beg;  // bodies perm[beg .. end)
    const int32_t* node_end;
    const int32_t* node_child;  // first child, -1 for a leaf
    const double* node_cx;
    const double* node_cy;
    const double* node_cz;
    const int32_t* perm;
    // leaves with mass > 0, depth-first
    int32_t n_leaves;
    const int32_t* leaf_off;
    const int32_t* leaf_part;
    const int32_t* far_node;
    double* rec;   // n_nodes * kFmmRec
    float* rec32;  // n_nodes * kRec32, mixed-precision far field only
    const M2PItem* items;
    int32_t n_items;
    double* scratch;  // partial sums of split leaves: 3 doubles per (chunk, target)
    int* done;        // chunks finished per leaf (zeroed before the launch)
    double* ax;       // accumulated into
    double* ay;
    double* az;
    int64_t t_begin, t_end;  // only bodies in [t_begin, t_end) are written
    double G;
    double eps2;
    float eps2f;
    int order;  // effective expansion order: 0, 2 or 4
    // Counts on the device, when the host did not read them back (nullable): n_nodes,
    // n_leaves and n_items above are then capacities, and kernels use min(count, capacity).
    // cnt_nodes points at the topology build's header {nodes, levels, flags}: with a flag
    // set (node slots exhausted, or a tree too deep for the device build) there are no nodes.
    // overflow (nullable) set: a pool was too small, the evaluation is skipped.
    const int32_t* cnt_nodes;
    const int32_t* cnt_leaves;
    const unsigned long long* cnt_items;
    const int* overflow;
};

__device__ __forceinline__ int fmm_nodes(const FmmArgs& a) {
    if (!a.cnt_nodes) return a.n_nodes;
    return a.cnt_nodes[2] ? 0 : min(a.cnt_nodes[0], a.n_nodes);
}
__device__ __forceinline__ int fmm_items(const FmmArgs& a) {
    return a.cnt_items ? (int)min(*a.cnt_items, (unsigned long long)a.n_items) : a.n_items;
}

constexpr int kMaxLevels = 22;  // levels an octree of 63-bit path keys can have

// Effective expansion order of multipole_acceleration (multipole.cpp:261-265).
int fmm_effective_order(int expansion_order);
constexpr int kM2PChunk = 512;  // far nodes per work item

// Stream-ordered: leaf moments, then one launch per level (deepest first), then M2P.
cudaError_t launch_fmm_moments(const FmmArgs& a, const int32_t* level_off_host, int n_levels, cudaStream_t st);
// The same with every internal node in one launch (blocks wait on their children's flags):
// ticket (1 int) and ready (n_nodes ints) are scratch; a wait that times out sets bit 0 of
// err[0] and err[1].
cudaError_t launch_fmm_moments_tree(const FmmArgs& a, int* ticket, int* ready, int* err, int sms, cudaStream_t st);
// ax += nx etc. for i < n (the near field added to the far field).
cudaError_t launch_fmm_add_near(int64_t n, double* ax, double* ay, double* az, const double* nx, const double* ny,
                                const double* nz, int sms, cudaStream_t st);
// mixed: FP32 multipole arithmetic on FP64 offsets (fills a.rec32 from a.rec first); else FP64.
cudaError_t launch_fmm_m2p(const FmmArgs& a, bool mixed, cudaStream_t st);


}  // namespace gx
