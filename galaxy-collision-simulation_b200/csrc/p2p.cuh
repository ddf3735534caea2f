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
    double G;
    double eps2;
    float eps2f;
};

cudaError_t launch_p2p(const P2PArgs& a, int precision, cudaStream_t st);

}  // namespace gx
