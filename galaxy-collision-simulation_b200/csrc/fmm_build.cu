// fmm_build.cu -- the reference octree (FastMultipoleSolver::build,
// cpp/fmm/fmm_solver.cpp:48-98) and its interaction lists (:228-277) built on the device.
//
// The reference inserts bodies one at a time; a leaf splits when it would hold more than
// leaf_capacity bodies below max_depth (:133-155).  The resulting tree is the recursive
// 8-way partition in which exactly the nodes with more than leaf_capacity bodies above
// max_depth are split.  A body's octant at every level depends only on its position and on
// the cell centres along its path, which follow the reference's recurrence
// (child centre = centre +- half_width * 0.5, :111-131; octant by >=, :104-109).  So:
//   1. root cell from the bounding box (:62-85);
//   2. every body's path as a 63-bit key, 3 bits per level, level 0 in the top bits;
//   3. a stable radix sort of (key, body): depth-first tree order;
//   4. one CTA walks the levels: a node with more than leaf_capacity bodies splits into 8
//      children whose body ranges are found by binary search on the sorted keys;
//   5. a second stable sort on (leaf rank, body) puts the bodies of every leaf in
//      ascending index order, the order the reference's sums run in.
// Nodes are numbered breadth-first.  Trees that need a split below level 21 (more than
// leaf_capacity nearly coincident bodies) are reported back for the host builder.
//
// Lists: a leaf with mass > 0 walks the tree depth-first from the root with the
// reference's tests (mass > 0, well_separated, leaf) in the reference's child order.
// One thread per leaf; a count pass, exclusive sums, a fill pass.
#include "fmm_build.cuh"
#include "fmm.cuh"
#include "gx_device.cuh"

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cfloat>

namespace gx {
namespace {

constexpr int kBboxThreads = 256;
constexpr int kBuildThreads = 1024;
constexpr int kWalkThreads = 128;
constexpr int kStack = 7 * (kKeyLevels + 1) + 8;

__global__ void __launch_bounds__(kBboxThreads) bbox_partial_kernel(const TreeBuildArgs t) {
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int i = blockIdx.x * kBboxThreads + threadIdx.x; i < t.n; i += gridDim.x * kBboxThreads) {
        const double v[3] = {t.x[i], t.y[i], t.z[i]};
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            lo[c] = fmin(lo[c], v[c]);
            hi[c] = fmax(hi[c], v[c]);
        }
    }
    __shared__ double s[6][kBboxThreads / 32];
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        lo[c] = warp_min(lo[c]);
        hi[c] = warp_max(hi[c]);
    }
    const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
        for (int c = 0; c < 3; ++c) {
            s[c][w] = lo[c];
            s[3 + c][w] = hi[c];
        }
    __syncthreads();
    if (threadIdx.x < 6) {
        double v = s[threadIdx.x][0];
        for (int k = 1; k < kBboxThreads / 32; ++k) v = threadIdx.x < 3 ? fmin(v, s[threadIdx.x][k]) : fmax(v, s[threadIdx.x][k]);
        t.part[blockIdx.x * 6 + threadIdx.x] = v;
    }
}

// Root cell (fmm_solver.cpp:62-85), one thread.
__global__ void bbox_final_kernel(const TreeBuildArgs t, int blocks) {
    double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
    for (int b = 0; b < blocks; ++b)
        for (int c = 0; c < 3; ++c) {
            lo[c] = fmin(lo[c], t.part[b * 6 + c]);
            hi[c] = fmax(hi[c], t.part[b * 6 + 3 + c]);
        }
    for (int c = 0; c < 3; ++c) t.root[c] = dmul(dadd(lo[c], hi[c]), 0.5);
    double hw = dmul(0.5, fmax(fmax(dsub(hi[0], lo[0]), dsub(hi[1], lo[1])), dsub(hi[2], lo[2])));
    hw = fmax(hw, dadd(t.softening, 1.0e-6));
    t.root[3] = dmul(hw, 1.0001);
}

__device__ __forceinline__ int octant_of(double x, double y, double z, double cx, double cy, double cz) {
    return (x >= cx ? 1 : 0) + (y >= cy ? 2 : 0) + (z >= cz ? 4 : 0);
}

// Child centre (subdivide, fmm_solver.cpp:111-131): centre + sign * (half_width * 0.5).
__device__ __forceinline__ double child_centre(double c, double chw, bool up) { return dadd(c, up ? chw : -chw); }

__global__ void __launch_bounds__(256) keys_kernel(const TreeBuildArgs t) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= t.n) return;
    const double x = t.x[i], y = t.y[i], z = t.z[i];
    double cx = t.root[0], cy = t.root[1], cz = t.root[2], hw = t.root[3];
    uint64_t key = 0;
    for (int l = 0; l < kKeyLevels; ++l) {
        const int o = octant_of(x, y, z, cx, cy, cz);
        key |= (uint64_t)o << (3 * (kKeyLevels - 1 - l));
        const double chw = dmul(hw, 0.5);
        cx = child_centre(cx, chw, o & 1);
        cy = child_centre(cy, chw, o & 2);
        cz = child_centre(cz, chw, o & 4);
        hw = chw;
    }
    t.keys[i] = key;
    t.idx[i] = i;
}

// First position p in [b, e) whose octant at shift sh is >= o (octants are non-decreasing
// in a cell's sorted range).
__device__ __forceinline__ int lower_octant(const uint64_t* keys, int b, int e, int sh, int o) {
    while (b < e) {
        const int mid = (b + e) >> 1;
        if ((int)((keys[mid] >> sh) & 7) < o) b = mid + 1;
        else e = mid;
    }
    return b;
}

// One CTA builds the whole topology level by level.
__global__ void __launch_bounds__(kBuildThreads) tree_build_kernel(const TreeBuildArgs t, const uint64_t* keys) {
    __shared__ int s_warp[kBuildThreads / 32];
    __shared__ int s_over;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    if (tid == 0) {
        t.beg[0] = 0;
        t.end[0] = t.n;
        t.cx[0] = t.root[0];
        t.cy[0] = t.root[1];
        t.cz[0] = t.root[2];
        t.hw[0] = t.root[3];
        t.level_off[0] = 0;
        t.level_off[1] = 1;
        s_over = 0;
    }
    __syncthreads();
    int lb = 0, le = 1, L = 0;
    while (lb < le) {
        int next = le;
        for (int k0 = lb; k0 < le; k0 += kBuildThreads) {
            const int k = k0 + tid;
            int split = 0;
            if (k < le && t.end[k] - t.beg[k] > t.cap && L < t.max_depth) {
                if (L >= kKeyLevels) atomicOr(&s_over, 1);
                else split = 1;
            }
            // block-wide exclusive scan of the split flags
            int v = split;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const int u = __shfl_up_sync(0xffffffffu, v, o);
                if (lane >= o) v += u;
            }
            if (lane == 31) s_warp[wid] = v;
            __syncthreads();
            if (wid == 0) {
                int w = s_warp[lane];
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int u = __shfl_up_sync(0xffffffffu, w, o);
                    if (lane >= o) w += u;
                }
                s_warp[lane] = w;
            }
            __syncthreads();
            const int rank = v - split + (wid > 0 ? s_warp[wid - 1] : 0);
            const int total = s_warp[kBuildThreads / 32 - 1];
            const bool room = (int64_t)next + 8 * (int64_t)total <= (int64_t)t.capacity;
            if (!room && tid == 0) atomicOr(&s_over, 2);
            if (k < le) {
                if (split && room) {
                    const int c0 = next + 8 * rank;
                    t.child[k] = c0;
                    const int b = t.beg[k], e = t.end[k];
                    const int sh = 3 * (kKeyLevels - 1 - L);
                    const double chw = dmul(t.hw[k], 0.5);
                    const double pcx = t.cx[k], pcy = t.cy[k], pcz = t.cz[k];
                    int lo = b;
                    for (int c = 0; c < 8; ++c) {
                        const int hi = c == 7 ? e : lower_octant(keys, lo, e, sh, c + 1);
                        t.beg[c0 + c] = lo;
                        t.end[c0 + c] = hi;
                        t.child[c0 + c] = -1;
                        t.cx[c0 + c] = child_centre(pcx, chw, c & 1);
                        t.cy[c0 + c] = child_centre(pcy, chw, c & 2);
                        t.cz[c0 + c] = child_centre(pcz, chw, c & 4);
                        t.hw[c0 + c] = chw;
                        lo = hi;
                    }
                } else {
                    t.child[k] = -1;
                }
            }
            next += 8 * total;
            __syncthreads();
            if (s_over) break;
        }
        if (s_over) break;
        lb = le;
        le = next;
        ++L;
        if (tid == 0) t.level_off[L + 1] = le;
    }
    if (tid == 0) {
        t.hdr[0] = le;
        t.hdr[1] = L;
        t.hdr[2] = s_over;
    }
}

__global__ void __launch_bounds__(256) gather_perm_kernel(const int32_t* idx_sorted, int32_t* perm, int n) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i < n) perm[i] = idx_sorted[i];
}

// Leaf order: the first body position of every non-empty leaf.
__global__ void __launch_bounds__(256) leaf_start_kernel(const TreeBuildArgs t, int n_nodes, int32_t* flag) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k < n_nodes && t.child[k] < 0 && t.end[k] > t.beg[k]) flag[t.beg[k]] = 1;
}

// (rank of the body's leaf, body index): sorting these puts each leaf's bodies in
// ascending index order (the reference's particle_indices order) and moves nothing
// across leaves.
__global__ void __launch_bounds__(256) leaf_key_kernel(const TreeBuildArgs t, const int32_t* rank) {
    const int p = blockIdx.x * 256 + threadIdx.x;
    if (p < t.n) t.keys[p] = ((uint64_t)(rank[p] - 1) << 31) | (uint64_t)t.perm[p];
}

__global__ void __launch_bounds__(256) leaf_unpack_kernel(const uint64_t* keys, int32_t* perm, int n) {
    const int p = blockIdx.x * 256 + threadIdx.x;
    if (p < n) perm[p] = (int32_t)(keys[p] & 0x7fffffffull);
}

__device__ __forceinline__ double node_mass(const double* rec, int k) { return rec[(size_t)k * kFmmRec + kRecMass]; }

// Marks the first body position of every leaf with mass > 0 and the bodies it keeps.
__global__ void __launch_bounds__(256) leaf_mark_kernel(const TreeListArgs a) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= a.n_nodes || a.child[k] >= 0 || !(node_mass(a.rec, k) > 0.0)) return;
    const int b = a.beg[k], e = a.end[k];
    a.start_flag[b] = 1;
    for (int p = b; p < e; ++p) a.keep[p] = 1;
}

__global__ void __launch_bounds__(256) leaf_emit_kernel(const TreeListArgs a) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k >= a.n_nodes || a.child[k] >= 0 || !(node_mass(a.rec, k) > 0.0)) return;
    const int b = a.beg[k], e = a.end[k];
    const int o = a.start_ord[b];
    a.leaf_node[o] = k;
    a.node_leaf[k] = o;
    a.leaf_off[o] = a.newpos[b];
    a.leaf_off[o + 1] = a.newpos[e];
    for (int p = b; p < e; ++p) a.leaf_part[a.newpos[p]] = a.perm[p];
}

// well_separated (fmm_solver.cpp:228-241) for a source with mass > 0.
__device__ __forceinline__ bool well_separated(const TreeListArgs& a, int t, int s) {
    const double dx = dsub(a.cx[s], a.cx[t]), dy = dsub(a.cy[s], a.cy[t]), dz = dsub(a.cz[s], a.cz[t]);
    const double dist = __dsqrt_rn(dadd(dadd(dmul(dx, dx), dmul(dy, dy)), dmul(dz, dz)));
    if (dist == 0.0) return false;
    const double comb = dmul(2.0, dadd(a.hw[t], a.hw[s]));
    return __ddiv_rn(comb, dist) < a.theta;
}

// build_leaf_interactions (fmm_solver.cpp:254-277) for every leaf with mass > 0.
template <bool FILL>
__global__ void __launch_bounds__(kWalkThreads) walk_kernel(const TreeListArgs a) {
    const int l = blockIdx.x * kWalkThreads + threadIdx.x;
    const int n_leaves = a.start_ord[a.n];
    if (l >= n_leaves) return;
    const int t = a.leaf_node[l];
    int stack[kStack];
    int sp = 0;
    stack[sp++] = 0;
    int nf = 0, nn = 0;
    const int fo = FILL ? a.far_off[l] : 0, no = FILL ? a.near_off[l] : 0;
    while (sp > 0) {
        const int s = stack[--sp];
        if (!(node_mass(a.rec, s) > 0.0)) continue;
        if (s != t && well_separated(a, t, s)) {
            if (FILL) a.far_node[fo + nf] = s;
            ++nf;
            continue;
        }
        const int c0 = a.child[s];
        if (c0 < 0) {
            if (FILL) a.near_leaf[no + nn] = a.node_leaf[s];
            ++nn;
            continue;
        }
        for (int c = 7; c >= 0; --c) stack[sp++] = c0 + c;
    }
    if (FILL) return;
    a.far_cnt[l] = nf;
    a.near_cnt[l] = nn;
    // far-field work items: only leaves with a target in range
    const int tb = a.leaf_off[l], te = a.leaf_off[l + 1];
    bool any = false;
    for (int k = tb; k < te && !any; ++k) any = a.leaf_part[k] >= a.t_begin && a.leaf_part[k] < a.t_end;
    const int nch = (any && nf > 0) ? (nf + kM2PChunk - 1) / kM2PChunk : 0;
    const int slots = nch > 1 ? nch * (te - tb) : 0;
    a.item_cnt[l] = nch;
    a.slot_cnt[l] = slots;
    atomicAdd(&a.totals[0], (unsigned long long)nf);
    atomicAdd(&a.totals[1], (unsigned long long)nn);
    atomicAdd(&a.totals[2], (unsigned long long)nch);
    atomicAdd(&a.totals[3], (unsigned long long)slots);
}

__global__ void __launch_bounds__(256) items_kernel(const TreeListArgs a, int n_leaves) {
    const int l = blockIdx.x * 256 + threadIdx.x;
    if (l >= n_leaves) return;
    const int nch = a.item_cnt[l];
    const int fb = a.far_off[l], fe = a.far_off[l + 1];
    M2PItem* items = (M2PItem*)a.items;
    for (int c = 0; c < nch; ++c) {
        M2PItem it;
        it.leaf = l;
        it.fb = fb + c * kM2PChunk;
        it.fe = min(fe, it.fb + kM2PChunk);
        it.chunk = c;
        it.nchunks = nch;
        it.pad = 0;
        it.scratch = nch > 1 ? a.slot_off[l] : 0;
        items[a.item_off[l] + c] = it;
    }
}

size_t scan_bytes(int count) {
    size_t b = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b, (const int32_t*)nullptr, (int32_t*)nullptr, count);
    return b;
}

}  // namespace

int leaf_key_bits(int32_t n) {
    int b = 1;
    while (b < 31 && (1ll << b) <= (long long)n) ++b;
    return 31 + b;
}

size_t tree_build_temp_bytes(int32_t n) {
    size_t b = 0, c = 0, d = 0;
    cub::DoubleBuffer<uint64_t> k(nullptr, nullptr);
    cub::DoubleBuffer<int32_t> v(nullptr, nullptr);
    cub::DeviceRadixSort::SortPairs(nullptr, b, k, v, n, 0, 3 * kKeyLevels);
    cub::DeviceRadixSort::SortKeys(nullptr, c, k, n, 0, leaf_key_bits(n));
    cub::DeviceScan::InclusiveSum(nullptr, d, (const int32_t*)nullptr, (int32_t*)nullptr, n);
    return std::max(b, std::max(c, d));
}

cudaError_t launch_tree_build(const TreeBuildArgs& t, void* temp, size_t temp_bytes, cudaStream_t st) {
    bbox_partial_kernel<<<kBboxBlocks, kBboxThreads, 0, st>>>(t);
    bbox_final_kernel<<<1, 1, 0, st>>>(t, kBboxBlocks);
    keys_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(t);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cub::DoubleBuffer<uint64_t> k(t.keys, t.keys_alt);
    cub::DoubleBuffer<int32_t> v(t.idx, t.perm);
    e = cub::DeviceRadixSort::SortPairs(temp, temp_bytes, k, v, t.n, 0, 3 * kKeyLevels, st);
    if (e != cudaSuccess) return e;
    if (v.Current() != t.perm) gather_perm_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(v.Current(), t.perm, t.n);
    tree_build_kernel<<<1, kBuildThreads, 0, st>>>(t, k.Current());
    return cudaGetLastError();
}

cudaError_t launch_tree_leaf_order(const TreeBuildArgs& t, int32_t n_nodes, void* temp, size_t temp_bytes,
                                   cudaStream_t st) {
    cudaError_t e;
    // t.idx is free after the first sort: leaf-start flags, then their inclusive sum in place
    if ((e = cudaMemsetAsync(t.idx, 0, (size_t)t.n * sizeof(int32_t), st)) != cudaSuccess) return e;
    leaf_start_kernel<<<(n_nodes + 255) / 256, 256, 0, st>>>(t, n_nodes, t.idx);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t tb = temp_bytes;
    if ((e = cub::DeviceScan::InclusiveSum(temp, tb, t.idx, t.idx, t.n, st)) != cudaSuccess) return e;
    leaf_key_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(t, t.idx);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cub::DoubleBuffer<uint64_t> k(t.keys, t.keys_alt);
    tb = temp_bytes;
    if ((e = cub::DeviceRadixSort::SortKeys(temp, tb, k, t.n, 0, leaf_key_bits(t.n), st)) != cudaSuccess) return e;
    leaf_unpack_kernel<<<(t.n + 255) / 256, 256, 0, st>>>(k.Current(), t.perm, t.n);
    return cudaGetLastError();
}

size_t tree_list_temp_bytes(int32_t n, int32_t n_nodes) {
    return std::max(scan_bytes(n + 1), scan_bytes(n_nodes + 1));
}

cudaError_t launch_tree_lists_count(const TreeListArgs& a, void* temp, size_t temp_bytes, cudaStream_t st) {
    cudaError_t e;
    const size_t nb = (size_t)(a.n + 1) * sizeof(int32_t), lb = (size_t)(a.n_nodes + 1) * sizeof(int32_t);
    if ((e = cudaMemsetAsync(a.start_flag, 0, nb, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.keep, 0, nb, st)) != cudaSuccess) return e;
    for (int32_t* p : {a.far_cnt, a.near_cnt, a.item_cnt, a.slot_cnt})
        if ((e = cudaMemsetAsync(p, 0, lb, st)) != cudaSuccess) return e;
    if ((e = cudaMemsetAsync(a.totals, 0, 4 * sizeof(unsigned long long), st)) != cudaSuccess) return e;
    const int gn = (a.n_nodes + 255) / 256;
    leaf_mark_kernel<<<gn, 256, 0, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    size_t tb = temp_bytes;
    if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, a.start_flag, a.start_ord, a.n + 1, st)) != cudaSuccess) return e;
    tb = temp_bytes;
    if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, a.keep, a.newpos, a.n + 1, st)) != cudaSuccess) return e;
    leaf_emit_kernel<<<gn, 256, 0, st>>>(a);
    walk_kernel<false><<<(a.n_nodes + kWalkThreads - 1) / kWalkThreads, kWalkThreads, 0, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const int32_t* cnt[4] = {a.far_cnt, a.near_cnt, a.item_cnt, a.slot_cnt};
    int32_t* off[4] = {a.far_off, a.near_off, a.item_off, a.slot_off};
    for (int k = 0; k < 4; ++k) {
        tb = temp_bytes;
        if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, cnt[k], off[k], a.n_nodes + 1, st)) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

cudaError_t launch_tree_lists_fill(const TreeListArgs& a, int32_t n_leaves, cudaStream_t st) {
    if (n_leaves == 0) return cudaSuccess;
    walk_kernel<true><<<(n_leaves + kWalkThreads - 1) / kWalkThreads, kWalkThreads, 0, st>>>(a);
    items_kernel<<<(n_leaves + 255) / 256, 256, 0, st>>>(a, n_leaves);
    return cudaGetLastError();
}

}  // namespace gx
