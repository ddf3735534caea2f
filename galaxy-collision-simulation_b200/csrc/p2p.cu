// p2p.cu -- FMM near-field (P2P) leaf kernel.
//
// Replaces the near loop of FastMultipoleSolver::evaluate_particle
// (cpp/fmm/fmm_solver.cpp:295-310): for every body i of a target leaf, the pair terms of
// all bodies j != i of the leaf's near leaves, in near-list order and leaf body order.
//
// Work decomposition.  The bodies of a target leaf's near leaves form one source sequence
// (near-list order, then leaf order).  Leaf costs are very uneven (in the N = 65,536
// two-disk tree the heaviest leaf has 13x the mean number of sources), so a leaf is cut into
// target groups x source chunks (at most kMaxChunks chunks of at least kMinChunk sources),
// items of bounded cost.  A plan computed on the device (p2p_count_kernel, then one block's
// counting sort of the leaves by item cost and its scans, or a CUB sort and scans for large
// leaf tables) numbers the items, the leaves with the costliest items first;
// a persistent grid takes them from a ticket counter, so that the last items handed out are
// the cheapest and the blocks finish together.  Items of an
// unsplit leaf add their sums to the accelerations directly (target groups are disjoint).
// A leaf split into chunks writes per-chunk partial sums to scratch; the block that finishes
// the leaf's last item (a per-leaf counter, after a memory fence) adds the partials in chunk
// order -- no block ever waits for another, and the order of summation does not depend on
// scheduling.
//
// Inside an item: a warp scan of the near leaves' sizes lets every thread find its own
// slots of the chunk and stage them into shared memory 4 x block at a time, from a copy of
// (x, y, z, m) in leaf-slot order gathered once per launch.  In the fast forms every thread
// serves two targets (halving the shared-memory reads per interaction): a group's targets
// form H rows of two, each row gets L = block / H threads that split the staged sources (any
// L, so a 22-body leaf keeps 121 of 128 threads busy), and a row's L partial sums are added
// in lane order.  Blocks are one warp when the mean leaf is small (independent items hide the
// gathers' latency) and four warps otherwise.
// The exact form uses one chunk and one group per leaf and one lane per target, and walks
// the sources in the reference's order starting from the incoming acceleration (the far
// field), which makes it bit-identical to the reference's evaluate_particle.
#include <algorithm>
#include <atomic>

#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_scan.cuh>

#include "gx_device.cuh"
#include "p2p.cuh"

namespace gx {
namespace {

constexpr int kNearBatch = 256;  // near leaves whose (start, length) sit in shared memory at once
constexpr int kMaxChunks = 8;    // a leaf's source sequence is split into at most this many items
constexpr int kMinChunk = 256;   // ... of at least this many sources
constexpr int kMinGroup = 8;     // targets of a group, when a leaf's targets are split
constexpr int kStageCost = 8;    // staging one source costs about this many interactions
constexpr int kWarpBlockMaxMean = 12;  // mean bodies per leaf up to which blocks are one warp
std::atomic<int> g_p2p_tpt{0};          // 0: the default shape; 2 or 4: forced (measurement)

// Per leaf (one warp each): number of sources, and the split of the leaf into target groups
// x source chunks of cost at most about item_cost each, where an item of g targets and s
// sources costs s x (g + kStageCost).  Target groups need no partial sums, so a heavy leaf
// is cut into groups first when kMaxChunks chunks would still leave items above item_cost.
// A split leaf needs chunks partial sums per target; chunks <= kMaxChunks keeps the total
// within kMaxChunks x (leaf slots), and leaves are not split at all when the slots exceed
// split_max_slots (a CSR that repeats bodies).  Entry n_leaves of the counts is zero, so
// that the exclusive scans end with the totals.
__global__ void __launch_bounds__(256) p2p_count_kernel(const P2PArgs a, int exact, int64_t item_cost) {
    const int l = (int)((blockIdx.x * 256u + threadIdx.x) >> 5), lane = threadIdx.x & 31;
    if (l > a.n_leaves) return;
    const int nl = p2p_leaves_now(a);
    if (l >= nl) {  // past the last leaf (up to the capacity): no work, so the scans end with the totals
        if (lane == 0) {
            a.plan_cnt[l] = 0;
            a.plan_need[l] = 0;
            a.plan_key[l] = 0;
            a.plan_ord[l] = l;
        }
        return;
    }
    int64_t src = 0;
    for (int q = a.near_off[l] + lane; q < a.near_off[l + 1]; q += 32) {
        const int s = a.near_leaf[q];
        src += a.leaf_off[s + 1] - a.leaf_off[s];
    }
    for (int o = 16; o > 0; o >>= 1) src += __shfl_xor_sync(0xffffffffu, src, o);
    if (lane != 0) return;
    const int nt = a.leaf_off[l + 1] - a.leaf_off[l];
    int chunks = 0, groups = 1;
    if (nt > 0 && src > 0) {
        chunks = 1;
        if (!exact) {
            const int64_t cap = kMaxChunks * item_cost;
            int64_t g = nt;
            if (src * (g + kStageCost) > cap) g = max((int64_t)kMinGroup, cap / src - kStageCost);
            g = min(g, (int64_t)nt);
            groups = (int)((nt + g - 1) / g);
            g = (nt + groups - 1) / groups;  // equal groups
            const int64_t c_cost = (src * (g + kStageCost) + item_cost - 1) / item_cost;
            const int64_t c_src = (src + kMinChunk - 1) / kMinChunk;
            chunks = (int)max((int64_t)1, min((int64_t)kMaxChunks, min(c_cost, c_src)));
            if (a.leaf_off[nl] > a.split_max_slots) chunks = 1;
        }
    }
    a.plan_src[l] = src;
    a.plan_chunks[l] = chunks;
    a.plan_groups[l] = groups;
    a.plan_cnt[l] = chunks * groups;
    a.plan_need[l] = chunks > 1 ? (int64_t)chunks * nt : 0;
    // Sort key: the cost of one item, cs sources x (g targets + the staging cost), on a
    // log scale with four steps per octave (7 bits; 0: no items).
    uint32_t key = 0;
    if (chunks > 0) {
        const int64_t g = (nt + groups - 1) / groups, cs = (src + chunks - 1) / chunks;
        const uint32_t cost = (uint32_t)min((int64_t)0x7fffffffLL, max((int64_t)4, cs * (g + kStageCost)));
        const int msb = 31 - __clz(cost);
        key = (uint32_t)(msb * 4 + ((cost >> (msb - 2)) & 3));
    }
    a.plan_key[l] = key;
    a.plan_ord[l] = l;
}

// The item counts in decreasing-cost order, and back: each leaf's first item number.
__global__ void __launch_bounds__(256) p2p_cnt_sorted_kernel(const P2PArgs a, const int* ord, int nl) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k < nl) a.plan_cnt_sorted[k] = a.plan_cnt[ord[k]];
}
__global__ void __launch_bounds__(256) p2p_off_scatter_kernel(const P2PArgs a, const int* ord, int nl) {
    const int k = blockIdx.x * 256 + threadIdx.x;
    if (k < nl) a.plan_item_off[ord[k]] = a.plan_off_sorted[k];
}

// The whole plan order in one block when the leaf table is small (at most kSmallPlan entries):
// leaves by decreasing item-cost key (a counting sort on the 7-bit keys; leaves with equal keys
// land in no fixed order, which changes only the order in which items are handed out, never a
// sum), the item counts in that order, their exclusive scan (plan_off_sorted and each leaf's
// first item), and the exclusive scan of the partial-sum needs in leaf order.  It replaces a
// radix sort, two scans and two scatter kernels -- about nine launches -- with one.
constexpr int kSmallPlan = 16384;
constexpr int kSmallPlanThreads = 1024;

// Exclusive scan of v over the block (kSmallPlanThreads threads); *carry holds the running
// total of the earlier chunks and is advanced.  Ends with a barrier.
template <typename T>
__device__ __forceinline__ T block_exclusive_scan(T v, T* s_warp, T* carry) {
    const int t = threadIdx.x, lane = t & 31, w = t >> 5;
    T x = v;
    for (int o = 1; o < 32; o <<= 1) {
        const T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        T z = s_warp[lane];
        for (int o = 1; o < 32; o <<= 1) {
            const T y = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += y;
        }
        s_warp[lane] = z;
    }
    __syncthreads();
    const T incl = x + (w > 0 ? s_warp[w - 1] : T(0)) + *carry;
    __syncthreads();
    if (t == kSmallPlanThreads - 1) *carry = incl;
    __syncthreads();
    return incl - v;
}

__global__ void __launch_bounds__(kSmallPlanThreads) p2p_small_plan_kernel(const P2PArgs a, int* ord_sorted, int nl) {
    __shared__ int s_bin[128];
    __shared__ int s_wi[32];
    __shared__ long long s_wl[32];
    __shared__ int s_ci;
    __shared__ long long s_cl;
    const int t = threadIdx.x;
    if (t < 128) s_bin[t] = 0;
    if (t == 0) {
        s_ci = 0;
        s_cl = 0;
    }
    __syncthreads();
    for (int k = t; k < nl; k += kSmallPlanThreads) atomicAdd(&s_bin[a.plan_key[k] & 127], 1);
    __syncthreads();
    if (t == 0) {  // bin starts, largest key first
        int run = 0;
        for (int b = 127; b >= 0; --b) {
            const int c = s_bin[b];
            s_bin[b] = run;
            run += c;
        }
    }
    __syncthreads();
    for (int k = t; k < nl; k += kSmallPlanThreads) {  // plan_ord is the identity here
        const int pos = atomicAdd(&s_bin[a.plan_key[k] & 127], 1);
        ord_sorted[pos] = k;
        a.plan_cnt_sorted[pos] = a.plan_cnt[k];
    }
    __syncthreads();
    for (int c0 = 0; c0 < nl; c0 += kSmallPlanThreads) {
        const int k = c0 + t;
        const int v = k < nl ? a.plan_cnt_sorted[k] : 0;
        const int ex = block_exclusive_scan<int>(v, s_wi, &s_ci);
        if (k < nl) {
            a.plan_off_sorted[k] = ex;
            a.plan_item_off[ord_sorted[k]] = ex;
        }
    }
    for (int c0 = 0; c0 < nl; c0 += kSmallPlanThreads) {
        const int k = c0 + t;
        const long long v = k < nl ? (long long)a.plan_need[k] : 0;
        const long long ex = block_exclusive_scan<long long>(v, s_wl, &s_cl);
        if (k < nl) a.plan_scratch[k] = (int64_t)ex;
    }
}

// The leaf of every item: item plan_item_off[l] + k belongs to leaf l (k < plan_cnt[l]).  One
// thread per leaf writes its own items, so the table costs one pass; the leaf kernel then
// finds an item's leaf with one load instead of a binary search of dependent loads over the
// item offsets, which dominated items of small leaves.
__global__ void __launch_bounds__(256) p2p_item_leaf_kernel(const P2PArgs a) {
    const int l = blockIdx.x * 256 + threadIdx.x;
    if (l >= p2p_leaves_now(a)) return;
    const int b = a.plan_item_off[l], c = a.plan_cnt[l];
    for (int k = 0; k < c && b + k < a.plan_item_cap; ++k) a.plan_item_leaf[b + k] = l;
}

// Slot-ordered copy of the sources: src[k] = (x, y, z, m) of body leaf_part[k], for every
// leaf slot k, when the slots fit the buffer (cap of them; a CSR that lists a body in
// several leaves can have more, and the leaf kernel then reads through leaf_part).
__global__ void __launch_bounds__(256) p2p_gather_kernel(const P2PArgs a, int64_t cap) {
    const int nl = p2p_leaves_now(a);
    const int64_t np = nl > 0 ? a.leaf_off[nl] : 0;
    const bool ok = np <= cap;
    if (blockIdx.x == 0 && threadIdx.x == 0) *a.src_ok = ok ? 1 : 0;
    if (!ok) return;
    for (int64_t k = (int64_t)blockIdx.x * 256 + threadIdx.x; k < np; k += (int64_t)gridDim.x * 256) {
        const int j = a.leaf_part[k];
        a.src[k] = make_double4(a.x[j], a.y[j], a.z[j], a.m[j]);
    }
}

// Asynchronous global -> shared copies (cp.async): the staging of the next pass of sources is
// in flight while the current pass is computed, without holding the data in registers.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_group 0;" ::: "memory"); }

// Resident threads per SM the launch bounds ask for: 640 (20 warps) with two targets per
// thread; with four, 512 in the mixed form and 384 in FP64 (four FP64 chains per thread in
// place of warps).
constexpr int p2p_threads_per_sm(int mode, int tpt) { return tpt == 2 ? 640 : mode == kMixed ? 512 : 384; }

// BS threads per block (a multiple of 32), 4 x BS sources staged per pass, TPT targets per
// thread in the fast forms (2 or 4).
template <int MODE, bool EPS0, int BS, int TPT>
__global__ void __launch_bounds__(BS, p2p_threads_per_sm(MODE, TPT) / BS) p2p_kernel(const P2PArgs a) {
    constexpr int kP2PBlock = BS;
    constexpr int kP2PJT = 4 * BS;  // sources staged per shared-memory pass
    static_assert(TPT == 2 || TPT == 4, "two or four targets per thread");
    // Sources of a pass arrive as (x, y), (z, m) double pairs by cp.async.  FP64 forms read
    // them there, from two buffers: pass k + 1 is copied into one while pass k is read from
    // the other.  The mixed form copies into one raw buffer and each thread converts its own
    // slots into FP32 offsets, stored by source PAIR -- (x0, x1, y0, y1), (z0, z1, m0, m1) -- in
    // two packed buffers: one 16-byte load gives every coordinate of two sources as packed
    // pairs, so each target (held duplicated) takes two interactions per f32x2 instruction.
    // A thread stages kStageU consecutive slots; the raw buffers hold slot c of thread
    // t = c / kStageU, u = c mod kStageU at raw_at(c) = u x block + (t + 2u) mod block: the
    // lanes of a warp copy to (and convert from) consecutive 16-byte words, and the runs of
    // consecutive slots that the FP64 forms read together spread over the 8 groups of 4
    // banks (11 consecutive slots: at most 2 in a group, as in a linear layout).
    constexpr int kRawBufs = MODE == kMixed ? 1 : 2;
    constexpr int kPairs = kP2PJT / 2;
    constexpr int kStageU = kP2PJT / kP2PBlock;  // slots a thread stages per pass
    __shared__ __align__(16) double2 sraw[kRawBufs][2][kP2PJT];
    __shared__ __align__(16) float4 spk[MODE == kMixed ? 2 : 1][MODE == kMixed ? 2 * kPairs : 1];
    // source body indices: raw order (FP64 forms: one per raw buffer; mixed: the third), and
    // in the mixed form pair order (the first two, one per packed buffer)
    __shared__ __align__(8) int sidx[MODE == kMixed ? 3 : 2][kP2PJT];
    __shared__ int s_beg[kNearBatch];
    __shared__ int s_pre[kNearBatch + 1];
    __shared__ int s_item, s_last;
    // row partial sums of the fast forms, in the raw buffer (free once a sweep has ended)
    static_assert(sizeof(sraw) >= 3 * TPT * kP2PBlock * sizeof(double), "row sums fit the raw buffer");
    double* const s_red = reinterpret_cast<double*>(&sraw[0][0][0]);
    auto raw_at = [](int c) { return (c % kStageU) * kP2PBlock + (c / kStageU + 2 * (c % kStageU)) % kP2PBlock; };

    // body indices of the staged sources are needed only to skip the target itself where a
    // zero distance does not already give a zero term
    constexpr bool kNeedIdx = MODE == kF64Exact || EPS0;
    const int tid = threadIdx.x;
    const int n_items = *a.plan_n_items;
    const bool by_slot = *a.src_ok != 0;
    for (;;) {
        if (tid == 0) s_item = atomicAdd(a.ticket, 1);
        __syncthreads();
        const int item = s_item;
        __syncthreads();
        if (item >= n_items) return;
        // leaf owning the item: one load from the table p2p_item_leaf_kernel filled; items past
        // the table (possible only with device CSR arrays that repeat bodies) search the offsets
        int leaf;
        if (item < a.plan_item_cap) {
            leaf = a.plan_item_leaf[item];
        } else {
            int lo = 0, hi = a.n_leaves;  // largest k with plan_off_sorted[k] <= item
            while (hi - lo > 1) {
                const int mid = (lo + hi) >> 1;
                if (a.plan_off_sorted[mid] <= item) lo = mid;
                else hi = mid;
            }
            leaf = a.plan_ord[lo];
        }
        const int chunks = a.plan_chunks[leaf], groups = a.plan_groups[leaf];
        const int local = item - a.plan_item_off[leaf];
        const int chunk = local % chunks, group = local / chunks;
        const int64_t src = a.plan_src[leaf];
        const int64_t per = (src + chunks - 1) / chunks;
        const int64_t c_lo = (int64_t)chunk * per;
        const int64_t c_hi = min(src, c_lo + per);

        const int tb = a.leaf_off[leaf];
        const int nt = a.leaf_off[leaf + 1] - tb;
        // this item's targets: group `group` of `groups` equal groups of the leaf's bodies
        const int gsz = (nt + groups - 1) / groups;
        const int g_lo = group * gsz, g_hi = min(nt, g_lo + gsz);
        const int nb = a.near_off[leaf], ne = a.near_off[leaf + 1];
        // Origin of the mixed form: the leaf's first body (near sources are close to it).
        const int first = a.leaf_part[tb];
        const double ox = a.x[first], oy = a.y[first], oz = a.z[first];

        // cp.async of this thread's slots of a pass: kStageU consecutive slots from
        // c0 + kStageU * tid of the current near batch (s_pre / s_beg) into raw buffer rb and
        // index buffer ib.  One binary search finds the near leaf of the first slot; the
        // others are in the same leaf or a few leaves further.
        auto issue = [&](int c0, int take, int rb, int ib, int cnt) {
            const int cb = tid * kStageU;
            if (cb < take) {
                int l2 = 0, h2 = cnt;  // s_pre[l2] <= c0 + cb < s_pre[h2]
                while (h2 - l2 > 1) {
                    const int mid = (l2 + h2) >> 1;
                    if (s_pre[mid] <= c0 + cb) l2 = mid;
                    else h2 = mid;
                }
#pragma unroll
                for (int u = 0; u < kStageU; ++u) {
                    const int c = cb + u;
                    if (c >= take) break;
                    const int sl = c0 + c;
                    while (s_pre[l2 + 1] <= sl) ++l2;  // sl < s_pre[cnt]: ends by l2 = cnt - 1
                    const int pos = s_beg[l2] + (sl - s_pre[l2]);
                    const int r = raw_at(c);
                    double* dxy = reinterpret_cast<double*>(&sraw[rb][0][r]);
                    double* dzm = reinterpret_cast<double*>(&sraw[rb][1][r]);
                    if (by_slot) {
                        const double* g = reinterpret_cast<const double*>(a.src + pos);
                        cp_async16(dxy, g);
                        cp_async16(dzm, g + 2);
                        if (kNeedIdx) cp_async4(&sidx[ib][r], a.leaf_part + pos);
                    } else {
                        const int j = a.leaf_part[pos];
                        cp_async8(dxy, a.x + j);
                        cp_async8(dxy + 1, a.y + j);
                        cp_async8(dzm, a.z + j);
                        cp_async8(dzm + 1, a.m + j);
                        if (kNeedIdx) sidx[ib][r] = j;
                    }
                }
            }
            cp_async_commit();
        };
        // Mixed form: this thread's slots of the pass, raw -> FP32 offsets in packed buffer pb,
        // one 16-byte store per pair and array; an odd count is padded with a massless source
        // far away (its term is exactly zero).
        auto convert = [&](int take, int pb) {
            static_assert(kStageU % 2 == 0, "a thread converts whole pairs");
#pragma unroll
            for (int k = 0; k < kStageU / 2; ++k) {
                const int c = tid * kStageU + 2 * k;
                if (c >= take) break;
                const double2 a0 = sraw[0][0][raw_at(c)], b0 = sraw[0][1][raw_at(c)];
                double2 a1 = make_double2(ox + 1e18, oy), b1 = make_double2(oz, 0.0);
                if (c + 1 < take) {
                    a1 = sraw[0][0][raw_at(c + 1)];
                    b1 = sraw[0][1][raw_at(c + 1)];
                }
                if (kNeedIdx) {
                    sidx[pb][c] = sidx[2][raw_at(c)];
                    sidx[pb][c + 1] = c + 1 < take ? sidx[2][raw_at(c + 1)] : -1;
                }
                const float x0 = __double2float_rn(a0.x - ox), x1 = __double2float_rn(a1.x - ox);
                const float y0 = __double2float_rn(a0.y - oy), y1 = __double2float_rn(a1.y - oy);
                const float z0 = __double2float_rn(b0.x - oz), z1 = __double2float_rn(b1.x - oz);
                spk[pb][c >> 1] = make_float4(x0, x1, y0, y1);
                spk[pb][kPairs + (c >> 1)] = make_float4(z0, z1, __double2float_rn(b0.y), __double2float_rn(b1.y));
            }
        };
        // Every source slot [c_lo, c_hi) of this item, kP2PJT per pass, compute(take, buf)
        // on each: the near list is walked in batches, a warp scan of the near leaves' sizes
        // lets every thread find its own slots.  One barrier per pass: after it the pass's
        // buffer is complete and every thread has finished the previous pass, whose buffer
        // then takes the copies of the next.
        // Near leaves qb .. qb + cnt - 1 of the list: s_beg[q] = first slot of leaf q, s_pre[q] =
        // sources before it in the batch (a warp scan of the sizes).  Ends with a barrier.
        auto load_batch = [&](int qb, int cnt) {
            for (int q = tid; q < cnt; q += kP2PBlock) {
                const int s = a.near_leaf[qb + q];
                const int b = a.leaf_off[s];
                s_beg[q] = b;
                s_pre[q + 1] = a.leaf_off[s + 1] - b;
            }
            if (tid == 0) s_pre[0] = 0;
            __syncthreads();
            if (tid < 32) {  // inclusive scan of the lengths s_pre[1..cnt] by warp 0
                int carry = 0;
                for (int k0 = 1; k0 <= cnt; k0 += 32) {
                    const int k = k0 + tid;
                    int v = k <= cnt ? s_pre[k] : 0;
                    for (int o = 1; o < 32; o <<= 1) {
                        const int u = __shfl_up_sync(0xffffffffu, v, o);
                        if (tid >= o) v += u;
                    }
                    if (k <= cnt) s_pre[k] = v + carry;
                    carry += __shfl_sync(0xffffffffu, v, 31);
                }
            }
            __syncthreads();
        };
        auto sweep = [&](auto&& compute) {
            int64_t base = 0;  // slots before the current near batch
            for (int qb = nb; qb < ne && base < c_hi; qb += kNearBatch) {
                const int cnt = min(kNearBatch, ne - qb);
                load_batch(qb, cnt);
                const int total = s_pre[cnt];
                // this batch covers slots [base, base + total) of the sequence; keep [c_lo, c_hi)
                const int b_lo = (int)max((int64_t)0, c_lo - base);
                const int b_hi = (int)min((int64_t)total, c_hi - base);
                int buf = 0;
                if (b_lo < b_hi) issue(b_lo, min(kP2PJT, b_hi - b_lo), 0, MODE == kMixed ? 2 : 0, cnt);
                for (int c0 = b_lo; c0 < b_hi; c0 += kP2PJT, buf ^= 1) {
                    const int take = min(kP2PJT, b_hi - c0);
                    cp_async_wait_all();
                    if (MODE == kMixed) convert(take, buf);
                    __syncthreads();
                    const int c1 = c0 + kP2PJT;
                    if (c1 < b_hi) issue(c1, min(kP2PJT, b_hi - c1), kRawBufs == 2 ? buf ^ 1 : 0, MODE == kMixed ? 2 : buf ^ 1, cnt);
                    compute(take, buf);
                }
                base += total;
                __syncthreads();  // s_beg / s_pre and the buffers are rewritten by the next batch
            }
        };

        if constexpr (MODE == kF64Exact) {
            // One target per thread, sources in the reference's order, starting from the
            // incoming acceleration (the far field).
            for (int t0 = 0; t0 < nt; t0 += kP2PBlock) {
                const int t = t0 + tid;
                const int i = t < nt ? a.leaf_part[tb + t] : first;
                const bool ok = t < nt && i >= a.t_begin && i < a.t_end;
                const double xi = a.x[i], yi = a.y[i], zi = a.z[i];
                double fx = 0.0, fy = 0.0, fz = 0.0;
                if (ok) {
                    fx = a.ax[i];
                    fy = a.ay[i];
                    fz = a.az[i];
                }
                sweep([&](int cnt, int buf) {
                    const int* I = sidx[buf];
                    for (int jj = 0; jj < cnt; ++jj) {
                        const int r = raw_at(jj);
                        if (I[r] == i) continue;
                        const double2 xy = sraw[buf][0][r], zm = sraw[buf][1][r];
                        const double4 q = make_double4(xy.x, xy.y, zm.x, zm.y);
                        const double rx = dsub(q.x, xi), ry = dsub(q.y, yi), rz = dsub(q.z, zi);
                        const double s2 = dadd(dadd(dadd(dmul(rx, rx), dmul(ry, ry)), dmul(rz, rz)), a.eps2);
                        if (s2 == 0.0) {
                            fx = dadd(fx, 0.0);
                            fy = dadd(fy, 0.0);
                            fz = dadd(fz, 0.0);
                            continue;
                        }
                        const double inv = __ddiv_rn(1.0, __dsqrt_rn(s2));
                        const double inv3 = dmul(dmul(inv, inv), inv);
                        const double scale = dmul(dmul(a.G, q.w), inv3);
                        fx = dadd(fx, dmul(rx, scale));
                        fy = dadd(fy, dmul(ry, scale));
                        fz = dadd(fz, dmul(rz, scale));
                    }
                });
                if (ok) {
                    a.ax[i] = fx;
                    a.ay[i] = fy;
                    a.az[i] = fz;
                }
            }
            continue;
        } else {
            // TPT targets per thread: the leaf's targets (up to TPT x kP2PBlock per pass) form
            // H rows of TPT (row r holds targets r, r + H, r + 2H, ...); every row gets
            // L = block / H lanes that split the staged sources, and a row's L partial sums
            // are added in lane order in shared memory.
            for (int t0 = g_lo; t0 < g_hi; t0 += TPT * kP2PBlock) {
                const int ntp = min(TPT * kP2PBlock, g_hi - t0);
                const int H = (ntp + TPT - 1) / TPT;
                const int L = max(1, kP2PBlock / H);
                const bool act = tid < H * L;
                const int row = act ? tid / L : 0, lane = act ? tid - row * L : 0;
                int ti[TPT];
                bool has[TPT];
                double xt[TPT], yt[TPT], zt[TPT];
#pragma unroll
                for (int h = 0; h < TPT; ++h) {
                    has[h] = act && row + h * H < ntp;
                    ti[h] = a.leaf_part[tb + t0 + row + (has[h] ? h * H : 0)];
                    xt[h] = a.x[ti[h]];
                    yt[h] = a.y[ti[h]];
                    zt[h] = a.z[ti[h]];
                }
                double f[3 * TPT];
#pragma unroll
                for (int k = 0; k < 3 * TPT; ++k) f[k] = 0.0;
                if constexpr (MODE == kF64) {
                    sweep([&](int cnt, int buf) {
                        if (!act) return;
                        const int* I = sidx[buf];
                        auto source = [&](const int r) {
                            const double2 xy = sraw[buf][0][r], zm = sraw[buf][1][r];
#pragma unroll
                            for (int h = 0; h < TPT; ++h) {
                                const double dx = xy.x - xt[h], dy = xy.y - yt[h], dz = zm.x - zt[h];
                                const double r2 = fma(dz, dz, fma(dy, dy, fma(dx, dx, a.eps2)));
                                double y = rsqrt_f64(r2);
                                if (EPS0) y = (r2 == 0.0 || I[r] == ti[h]) ? 0.0 : y;
                                const double w = zm.y * (y * y * y);
                                f[3 * h] = fma(dx, w, f[3 * h]);
                                f[3 * h + 1] = fma(dy, w, f[3 * h + 1]);
                                f[3 * h + 2] = fma(dz, w, f[3 * h + 2]);
                            }
                        };
                        // the order of the sources does not matter here: a full pass is read
                        // in buffer order, a partial one through raw_at
                        if (cnt == kP2PJT) {
#pragma unroll 2
                            for (int r = lane; r < kP2PJT; r += L) source(r);
                        } else {
#pragma unroll 2
                            for (int jj = lane; jj < cnt; jj += L) source(raw_at(jj));
                        }
                    });
                } else {
                    // every target duplicated into both halves of its packed registers
                    f2 XI[TPT], YI[TPT], ZI[TPT];
#pragma unroll
                    for (int h = 0; h < TPT; ++h) {
                        const float fx = __double2float_rn(xt[h] - ox), fy = __double2float_rn(yt[h] - oy);
                        const float fz = __double2float_rn(zt[h] - oz);
                        XI[h] = pk2(fx, fx);
                        YI[h] = pk2(fy, fy);
                        ZI[h] = pk2(fz, fz);
                    }
                    const f2 E2 = pk2(a.eps2f, a.eps2f);
                    sweep([&](int cnt, int buf) {
                        if (!act) return;
                        const float4* PA = &spk[buf][0];
                        const float4* PB = &spk[buf][kPairs];
                        const int2* I2 = reinterpret_cast<const int2*>(sidx[buf]);
                        f2 PX[TPT], PY[TPT], PZ[TPT];
#pragma unroll
                        for (int h = 0; h < TPT; ++h) PX[h] = PY[h] = PZ[h] = pk2(0.f, 0.f);
                        const int np = (cnt + 1) >> 1;
#pragma unroll 4
                        for (int pp = lane; pp < np; pp += L) {
                            f2 X, Y, Z, M;
                            lds_v2b64(reinterpret_cast<const float*>(&PA[pp]), X, Y);
                            lds_v2b64(reinterpret_cast<const float*>(&PB[pp]), Z, M);
                            int2 jj2 = make_int2(-1, -1);
                            if (EPS0) jj2 = I2[pp];
#pragma unroll
                            for (int h = 0; h < TPT; ++h) {
                                const f2 dX = sub2(X, XI[h]);
                                const f2 dY = sub2(Y, YI[h]);
                                const f2 dZ = sub2(Z, ZI[h]);
                                f2 R = fma2(dX, dX, E2);
                                R = fma2(dY, dY, R);
                                R = fma2(dZ, dZ, R);
                                float r0, r1;
                                upk2(R, r0, r1);
                                float i0 = rsqrt_f32(r0), i1 = rsqrt_f32(r1);
                                if (EPS0) {
                                    i0 = (r0 == 0.f || jj2.x == ti[h]) ? 0.f : i0;
                                    i1 = (r1 == 0.f || jj2.y == ti[h]) ? 0.f : i1;
                                }
                                const f2 I = pk2(i0, i1);
                                f2 T = mul2(I, I);
                                T = mul2(T, I);
                                const f2 W = mul2(M, T);
                                PX[h] = fma2(dX, W, PX[h]);
                                PY[h] = fma2(dY, W, PY[h]);
                                PZ[h] = fma2(dZ, W, PZ[h]);
                            }
                        }
#pragma unroll
                        for (int h = 0; h < TPT; ++h) {  // the pass's two halves, added into FP64 sums
                            float p0, p1;
                            upk2(PX[h], p0, p1);
                            f[3 * h] += (double)(p0 + p1);
                            upk2(PY[h], p0, p1);
                            f[3 * h + 1] += (double)(p0 + p1);
                            upk2(PZ[h], p0, p1);
                            f[3 * h + 2] += (double)(p0 + p1);
                        }
                    });
                }
                if (act)
#pragma unroll
                    for (int k = 0; k < 3 * TPT; ++k) s_red[k * kP2PBlock + tid] = f[k];
                __syncthreads();
                if (act && lane == 0) {
                    double S[3 * TPT];
#pragma unroll
                    for (int k = 0; k < 3 * TPT; ++k) S[k] = 0.0;
                    for (int q = 0; q < L; ++q)
#pragma unroll
                        for (int k = 0; k < 3 * TPT; ++k) S[k] += s_red[k * kP2PBlock + tid + q];
#pragma unroll
                    for (int h = 0; h < TPT; ++h) {
                        if (!has[h]) continue;
                        const int t = t0 + row + h * H;
                        const int i = ti[h];
                        if (i < a.t_begin || i >= a.t_end) continue;
                        if (chunks == 1) {
                            a.ax[i] = a.ax[i] + a.G * S[3 * h];
                            a.ay[i] = a.ay[i] + a.G * S[3 * h + 1];
                            a.az[i] = a.az[i] + a.G * S[3 * h + 2];
                        } else {
                            const size_t k = (size_t)(a.plan_scratch[leaf] + (int64_t)chunk * nt + t) * 3;
                            a.scratch[k] = S[3 * h];
                            a.scratch[k + 1] = S[3 * h + 1];
                            a.scratch[k + 2] = S[3 * h + 2];
                        }
                    }
                }
                __syncthreads();
            }
        }
        if (chunks == 1) continue;
        // Split leaf: the CTA that completes its last chunk adds the partials in chunk order.
        __threadfence();
        __syncthreads();
        if (tid == 0) s_last = (atomicAdd(&a.plan_done[leaf], 1) == chunks * groups - 1);
        __syncthreads();
        if (!s_last) continue;
        __threadfence();
        for (int t = tid; t < nt; t += kP2PBlock) {
            const int i = a.leaf_part[tb + t];
            if (i < a.t_begin || i >= a.t_end) continue;
            double sx = 0.0, sy = 0.0, sz = 0.0;
            for (int c = 0; c < chunks; ++c) {
                const size_t k = (size_t)(a.plan_scratch[leaf] + (int64_t)c * nt + t) * 3;
                sx += __ldcg(&a.scratch[k]);
                sy += __ldcg(&a.scratch[k + 1]);
                sz += __ldcg(&a.scratch[k + 2]);
            }
            a.ax[i] = a.ax[i] + a.G * sx;
            a.ay[i] = a.ay[i] + a.G * sy;
            a.az[i] = a.az[i] + a.G * sz;
        }
    }
}

template <int MODE, bool EPS0, int BS, int TPT>
int p2p_occupancy() {
    static int occ = 0;
    if (occ == 0) {
        int nb = 0;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, p2p_kernel<MODE, EPS0, BS, TPT>, BS, 0) != cudaSuccess ||
            nb < 1)
            nb = 1;
        occ = nb;
    }
    return occ;
}

template <int MODE, bool EPS0, int BS, int TPT>
cudaError_t launch_main(const P2PArgs& a, int sms, cudaStream_t st) {
    const int grid = sms * p2p_occupancy<MODE, EPS0, BS, TPT>();
    p2p_kernel<MODE, EPS0, BS, TPT><<<grid, BS, 0, st>>>(a);
    return cudaGetLastError();
}

template <int MODE, bool EPS0>
cudaError_t launch_bs(const P2PArgs& a, int bs, int tpt, int sms, cudaStream_t st) {
    if (MODE == kF64Exact || tpt == 2)
        return bs == 32 ? launch_main<MODE, EPS0, 32, 2>(a, sms, st) : launch_main<MODE, EPS0, 128, 2>(a, sms, st);
    return bs == 32 ? launch_main<MODE, EPS0, 32, 4>(a, sms, st) : launch_main<MODE, EPS0, 128, 4>(a, sms, st);
}

}  // namespace

namespace {

// Items of a plan: a leaf of nt targets has at most kMaxChunks chunks x ceil(nt / kMinGroup)
// groups, so the total is at most kMaxChunks (n / kMinGroup + n_leaves) <= n + 8 n_leaves.
size_t item_leaf_bytes(int64_t n, int32_t n_leaves) {
    return ((size_t)kMaxChunks * ((size_t)n / kMinGroup + (size_t)n_leaves + 1) * sizeof(int) + 255) & ~(size_t)255;
}

size_t plan_scan_temp_bytes(int32_t n_leaves) {
    size_t b1 = 0, b2 = 0, b3 = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, b1, (const int*)nullptr, (int*)nullptr, n_leaves + 1);
    cub::DeviceScan::ExclusiveSum(nullptr, b2, (const int64_t*)nullptr, (int64_t*)nullptr, n_leaves + 1);
    cub::DeviceRadixSort::SortPairsDescending(nullptr, b3, (const uint32_t*)nullptr, (uint32_t*)nullptr,
                                              (const int*)nullptr, (int*)nullptr, n_leaves + 1);
    return (std::max({b1, b2, b3}) + 255) & ~(size_t)255;
}

}  // namespace

void p2p_set_targets_per_thread(int tpt) { g_p2p_tpt.store(tpt == 2 || tpt == 4 ? tpt : 0); }

size_t p2p_scratch_bytes(int64_t n, int32_t n_leaves) {
    // plan arrays (src, need and scratch offsets int64; chunks, groups, counts, item offsets,
    // done counters int; item-cost keys and leaf order, each with the sort's second buffer,
    // counts and offsets in that order), the item -> leaf table, the scan's and sort's
    // temporary storage, src_ok + ticket, the partial sums (at most kMaxChunks per leaf slot,
    // leaf slots <= n when leaves are split), and the slot-ordered sources (32 bytes per
    // body); 256 bytes of alignment per piece.
    const size_t nl = (size_t)n_leaves + 1;
    return nl * (3 * 8 + 11 * 4) + item_leaf_bytes(n, n_leaves) + plan_scan_temp_bytes(n_leaves) + 6 * 256 +
           (size_t)kMaxChunks * 3 * sizeof(double) * (size_t)n + (size_t)n * sizeof(double4);
}

cudaError_t launch_p2p(P2PArgs a, int64_t n_bodies, int precision, void* scratch, int sms, cudaStream_t st) {
    if (a.n_leaves <= 0) return cudaSuccess;
    const bool eps0 = precision == kMixed ? (a.eps2f < 1e-24f) : (a.eps2 < 1e-200);
    const size_t nl = (size_t)a.n_leaves + 1;
    char* p = (char*)scratch;
    auto carve = [&](size_t bytes) {
        char* q = p;
        p += bytes;
        return q;
    };
    auto align = [&] { p = (char*)(((uintptr_t)p + 255) & ~(uintptr_t)255); };
    a.plan_src = (int64_t*)carve(nl * 8);
    a.plan_need = (int64_t*)carve(nl * 8);
    a.plan_scratch = (int64_t*)carve(nl * 8);
    a.plan_chunks = (int*)carve(nl * 4);
    a.plan_groups = (int*)carve(nl * 4);
    a.plan_cnt = (int*)carve(nl * 4);
    a.plan_item_off = (int*)carve(nl * 4);
    a.plan_done = (int*)carve(nl * 4);
    a.plan_n_items = a.plan_item_off + a.n_leaves;
    a.plan_key = (uint32_t*)carve(nl * 4);
    uint32_t* key_sorted = (uint32_t*)carve(nl * 4);
    a.plan_ord = (int*)carve(nl * 4);
    int* ord_sorted = (int*)carve(nl * 4);
    a.plan_cnt_sorted = (int*)carve(nl * 4);
    a.plan_off_sorted = (int*)carve(nl * 4);
    align();
    a.plan_item_leaf = (int*)carve(item_leaf_bytes(n_bodies, a.n_leaves));
    a.plan_item_cap = (int)std::min<size_t>(item_leaf_bytes(n_bodies, a.n_leaves) / sizeof(int), 0x7fffffff);
    align();
    size_t temp_bytes = plan_scan_temp_bytes(a.n_leaves);
    void* temp = carve(temp_bytes);
    align();
    a.ticket = (int*)carve(256);
    a.src_ok = a.ticket + 1;
    a.scratch = (double*)carve((size_t)kMaxChunks * 3 * sizeof(double) * (size_t)n_bodies);
    align();
    a.src = (double4*)carve((size_t)n_bodies * sizeof(double4));
    a.split_max_slots = n_bodies;
    // Block size: with few bodies per leaf a leaf's item is small, and one-warp blocks (20
    // independent warps per SM, no block-wide barriers) hide the latency of its gathers;
    // larger leaves keep 4-warp blocks that share each staged source among more threads.
    const int leaves_est = a.leaves_hint > 0 ? a.leaves_hint : a.n_leaves;
    const int bs = n_bodies <= (int64_t)kWarpBlockMaxMean * leaves_est ? 32 : 128;
    // Targets per thread: two.  Four (two packed pairs per staged source in the mixed form,
    // four FP64 chains per thread) measured 2-40% slower at every size and leaf capacity
    // tried (N = 65,536 and 2^20, leaf 16 and 64); the shape stays selectable for measurement.
    const int forced = g_p2p_tpt.load();
    const int tpt = forced ? forced : 2;
    const int64_t item_cost = (int64_t)1024 * bs;
    cudaError_t e = cudaMemsetAsync(a.plan_done, 0, nl * 4, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(a.ticket, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    p2p_gather_kernel<<<sms * 8, 256, 0, st>>>(a, n_bodies);
    p2p_count_kernel<<<(a.n_leaves + 8) / 8, 256, 0, st>>>(a, precision == kF64Exact ? 1 : 0, item_cost);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    // With few items per block, the leaves by decreasing item cost and the items numbered in
    // that order: without it the last items handed out can be the largest, and at
    // N = 65,536 leaf 64 (3011 leaves, 740 blocks) the SMs sat idle for 18% of the P2P kernel.
    // With many items per block the tail is small and the sort (four launches) is skipped,
    // except in the exact form, whose leaves are never split (N = 2^20 leaf 16: 17 ms sorted,
    // 28 ms in leaf order).
    size_t tb = temp_bytes;
    const bool sorted = precision == kF64Exact || leaves_est <= 16 * 4 * sms;
    if (sorted && nl <= (size_t)kSmallPlan) {
        p2p_small_plan_kernel<<<1, kSmallPlanThreads, 0, st>>>(a, ord_sorted, (int)nl);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        a.plan_ord = ord_sorted;
    } else if (sorted) {
        if ((e = cub::DeviceRadixSort::SortPairsDescending(temp, tb, a.plan_key, key_sorted, a.plan_ord,
                                                           ord_sorted, (int)nl, 0, 7, st)) != cudaSuccess)
            return e;
        const unsigned gl = (unsigned)((nl + 255) / 256);
        p2p_cnt_sorted_kernel<<<gl, 256, 0, st>>>(a, ord_sorted, (int)nl);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        tb = temp_bytes;
        if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, a.plan_cnt_sorted, a.plan_off_sorted, (int)nl, st)) !=
            cudaSuccess)
            return e;
        p2p_off_scatter_kernel<<<gl, 256, 0, st>>>(a, ord_sorted, (int)nl);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
        a.plan_ord = ord_sorted;  // the leaf kernel's fallback search walks the sorted order
    } else {
        // leaf order: plan_ord is the identity the count kernel wrote
        if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, a.plan_cnt, a.plan_item_off, (int)nl, st)) != cudaSuccess)
            return e;
        a.plan_off_sorted = a.plan_item_off;
    }
    if (!(sorted && nl <= (size_t)kSmallPlan)) {  // the small plan kernel scanned the needs already
        tb = temp_bytes;
        if ((e = cub::DeviceScan::ExclusiveSum(temp, tb, a.plan_need, a.plan_scratch, (int)nl, st)) != cudaSuccess)
            return e;
    }
    p2p_item_leaf_kernel<<<(a.n_leaves + 255) / 256, 256, 0, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if (precision == kF64Exact) return launch_bs<kF64Exact, false>(a, bs, 2, sms, st);
    if (precision == kF64)
        return eps0 ? launch_bs<kF64, true>(a, bs, tpt, sms, st) : launch_bs<kF64, false>(a, bs, tpt, sms, st);
    return eps0 ? launch_bs<kMixed, true>(a, bs, tpt, sms, st) : launch_bs<kMixed, false>(a, bs, tpt, sms, st);
}

}  // namespace gx
