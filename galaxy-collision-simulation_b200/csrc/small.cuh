// small.cuh -- the kick-drift-kick loop of a small system (n <= kSmallMaxBodies) in one
// cooperative launch (small.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gx {

constexpr int kSmallMaxBodies = 4096;

struct SmallArgs {
    int n;
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az;  // state: read at the start, written at the end
    const double* m;
    double* buf;       // two position buffers, buf[(p * 3 + c) * n + i]
    unsigned* bar;     // grid barrier: [0] arrivals, [1] generation
    int* status;       // 0, or 1 when a barrier wait gave up (the launch then stops early)
    double G, eps2, dt;
    int64_t steps;
    unsigned long long timeout_ns;  // longest wait at one barrier
    int64_t stall_step;             // test hook: CTA 0 leaves before this step's barrier (-1: never)
};

// Targets per warp: 1, 2 or 4 forces that many, 0 restores the choice from n (measurements).
void small_set_targets_per_warp(int tpw);
// Warps per target of the FP64 form: 1 or 2 forces that many, 0 restores the choice (measurements).
void small_set_warps_per_target(int wpt);
// Device bytes of the scratch a launch needs (position buffers, barrier, status); the barrier
// and status words sit at the start and must be zero before each launch.
size_t small_scratch_bytes(int n);
// Lays out the scratch for `a` (a.buf, a.bar, a.status from `scratch`).
void small_bind_scratch(SmallArgs& a, void* scratch);
// Runs a.steps KDK steps (kick dt/2, drift dt, force, kick dt/2) of a.n bodies: FP64 with the
// refined rsqrt (precision kF64) or the reference's exact operation order (kF64Exact).
// Clears the barrier words on `st` first.  cudaErrorNotSupported for other precisions, n out
// of range or a device without cooperative launch.
cudaError_t small_steps_launch(const SmallArgs& a, int precision, bool eps0, int device, cudaStream_t st);

}  // namespace gx
