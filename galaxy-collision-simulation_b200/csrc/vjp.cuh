// vjp.cuh -- launcher of the adjoint (vector-Jacobian product) kernel.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gx {

struct VjpArgs {
    const double* x;
    const double* y;
    const double* z;
    const double* m;
    const double* lx;  // cotangent on the accelerations
    const double* ly;
    const double* lz;
    int64_t n;
    int64_t j_chunk;  // multiple of vjp_jt(precision)
    int nsplit;
    double* gx;
    double* gy;
    double* gz;
    double* gm;    // nullable
    double* part;  // nsplit * 4 * n when nsplit > 1
    double G;
    double eps2;
    float eps2f;
};

int vjp_tile(int precision);  // targets per CTA
int vjp_jt(int precision);    // sources per shared-memory pass

struct VjpShape {
    int block, ipt, jt, occupancy;
};
VjpShape vjp_shape(int precision);  // launch shape and resident CTAs per SM
cudaError_t launch_vjp(const VjpArgs& a, int precision, cudaStream_t st);

}  // namespace gx
