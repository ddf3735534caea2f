// p2p.cuh -- launcher of the FMM near-field leaf kernel.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gx {

struct P2PArgs {
    const double* x;
    const double* y;
    const double* z;
    const double* m;
    const int32_t* leaf_off;   // n_leaves + 1
    const int32_t* leaf_part;  // body indices grouped by leaf
    const int32_t* near_off;   // n_leaves + 1
    const int32_t* near_leaf;  // leaf ids
    int32_t n_leaves;
    double* ax;  // accumulated into
    double* ay;
    double* az;
    int64_t t_begin, t_end;  // only bodies in [t_begin, t_end) are written
    double G;
    double eps2;
    float eps2f;
    // work plan and partial sums, carved from the scratch passed to launch_p2p
    int64_t* plan_src;      // sources per leaf
    int64_t* plan_need;     // partial sums a split leaf needs (chunks x targets), n_leaves + 1
    int64_t* plan_scratch;  // per-leaf offset of its partial sums (exclusive scan of plan_need)
    int* plan_chunks;       // source chunks per leaf
    int* plan_groups;       // target groups per leaf
    int* plan_cnt;          // items per leaf (groups x chunks), n_leaves + 1
    int* plan_item_off;     // exclusive scan of plan_cnt
    int* plan_done;         // items finished per leaf
    int* plan_n_items;      // = plan_item_off + n_leaves
    int* plan_item_leaf;    // leaf of each item (the first plan_item_cap items)
    int plan_item_cap;
    uint32_t* plan_key;     // cost of one item of each leaf (0: no items), n_leaves + 1
    int* plan_ord;          // leaves by decreasing item cost, n_leaves + 1
    int* plan_cnt_sorted;   // plan_cnt in that order
    int* plan_off_sorted;   // its exclusive scan: item offsets in that order
    int* ticket;
    // (x, y, z, m) of leaf_part[k] at slot k, gathered once per launch when the leaf slots
    // fit the buffer (src_ok); sources are then read by slot, without the leaf_part hop
    double4* src;
    int* src_ok;
    double* scratch;
    int64_t split_max_slots;  // leaves are split only if their slots number at most this
    // Capacity mode (nullable): the leaf count on the device (n_leaves is then the capacity
    // of the leaf arrays), an overflow flag that turns the launch into a no-op, and the
    // expected leaf count for the choice of block size.
    const int32_t* cnt_leaves;
    const int* overflow;
    int32_t leaves_hint;
};

__device__ __forceinline__ int p2p_leaves_now(const P2PArgs& a) {
    if (a.overflow && *a.overflow) return 0;
    return a.cnt_leaves ? min(*a.cnt_leaves, a.n_leaves) : a.n_leaves;
}

// Targets per thread of the fast forms: 2 or 4 forces that many, 0 restores the choice by
// mean leaf size (for measurements).
void p2p_set_targets_per_thread(int tpt);
// Device scratch launch_p2p needs for n bodies and n_leaves leaves.
size_t p2p_scratch_bytes(int64_t n, int32_t n_leaves);
// Stream-ordered: plan on the device, then the persistent leaf kernel (sms x occupancy CTAs).
cudaError_t launch_p2p(P2PArgs a, int64_t n_bodies, int precision, void* scratch, int sms, cudaStream_t st);

}  // namespace gx
