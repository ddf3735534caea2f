// force.cuh -- host-visible description of the direct-force kernels (force.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "precision.cuh"

namespace gx {

// One launch of the tiled direct sum: targets (a range or an index list) against the
// sources [0, n_src) of one SoA system.  The grid is one-dimensional, chunk-minor: CTA b
// works on target tile b / nsplit and source chunk b % nsplit (the j-split), so the
// nsplit CTAs of one tile start together.  With more than one chunk every CTA writes FP64
// partial sums; with `tile_count` set, the CTA that finishes a tile last (an atomic
// ticket per tile) adds the tile's partials in chunk order and writes the result, so the
// partials are consumed while they are still in L2 and no second kernel runs; without it,
// force_reduce_kernel adds them in a second launch.  Either way the sum is taken in chunk
// order, so results do not depend on scheduling.
struct ForceArgs {
    const double* x;
    const double* y;
    const double* z;
    const double* m;
    int64_t n_src;
    const int64_t* tgt_idx;  // nullable: targets are t_begin + t.  Entries outside
                             // [0, n_src) are not read through: their results are NaN
    int64_t t_begin;
    int64_t n_tgt;
    int64_t j_chunk;  // sources per chunk (a multiple of the kernel's j tile)
    int nsplit;       // number of chunks
    double* ax;       // results, indexed by target ordinal t
    double* ay;
    double* az;
    double* part;     // nsplit * 3 * n_tgt partial sums when nsplit > 1
    unsigned* tile_count;  // nullable: one zeroed ticket per target tile (fused reduction);
                           // the last CTA of a tile resets its ticket to 0
    double* vx;       // optional closing kick v[body] += a * kick_dt (nullable)
    double* vy;
    double* vz;
    double kick_dt;
    double G;
    double eps2;      // softening^2 in FP64
    float eps2f;      // softening^2 rounded to FP32 (mixed precision)
};

struct ForceVariant {
    int precision;
    int block;
    int ipt;   // targets per thread
    int jt;    // j tile (sources staged per shared-memory pass)
    int packed;  // 0 scalar FP32, 1 two sources per f32x2, 2 two targets per f32x2
    int eps0;  // guards s == 0 pairs (softening 0)
    const void* fn;
};

// All compiled variants; eps0 variants are separate entries.
const ForceVariant* force_variants(int* count);
// Variants usable for (precision, eps0) in the order of gx_variant_* ids.
int force_variant_ids(int precision, int eps0, int* ids, int max_ids);

// Launches variant `v` over args (ceil(n_tgt / (block*ipt)) * nsplit CTAs) and, when
// nsplit > 1 without tile tickets, the ordered partial-sum reduction with the epilogue.
cudaError_t force_launch(const ForceVariant& v, const ForceArgs& args, cudaStream_t stream);

// Target tiles of one launch of `v` (the number of tickets a fused reduction needs).
int64_t force_tiles(const ForceVariant& v, int64_t n_tgt);

// Resident CTAs per SM for a variant (occupancy query, cached).
int force_occupancy(const ForceVariant& v);

}  // namespace gx
