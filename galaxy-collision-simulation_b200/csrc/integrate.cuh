// integrate.cuh -- launchers for the kick/drift kernels and the FP64 diagnostics.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace gx {

cudaError_t launch_kick(int64_t n, double* vx, double* vy, double* vz, const double* ax,
                        const double* ay, const double* az, double dt, cudaStream_t st);
cudaError_t launch_drift(int64_t n, double* x, double* y, double* z, const double* vx,
                         const double* vy, const double* vz, double dt, cudaStream_t st);
cudaError_t launch_kick_drift(int64_t n, double* x, double* y, double* z, double* vx,
                              double* vy, double* vz, const double* ax, const double* ay,
                              const double* az, double kdt, double ddt, cudaStream_t st);

// Device scratch (bytes) the diagnostics of n bodies need; out13 is a device pointer.
size_t diagnostics_scratch_bytes(int64_t n);
cudaError_t launch_diagnostics(int64_t n, const double* x, const double* y, const double* z,
                               const double* vx, const double* vy, const double* vz,
                               const double* m, double G, double eps2, double* scratch,
                               double* out13, cudaStream_t st);

}  // namespace gx
