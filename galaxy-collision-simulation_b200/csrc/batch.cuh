// batch.cuh -- persistent batched-ensemble kernels (batch.cu).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace gx {

struct BatchArgs {
    const double* x;
    const double* y;
    const double* z;
    const double* m;
    const int64_t* offsets;  // n_instances + 1 (device)
    const int2* items;       // (instance, tile) work items, in execution order (device)
    int n_items;
    int* counter;            // ticket counter, zeroed before every launch (device)
    double* ax;
    double* ay;
    double* az;
    double* vx;  // optional closing kick (nullable)
    double* vy;
    double* vz;
    double kick_dt;
    double G;
    double eps2;
    float eps2f;
};

struct BatchVariant {
    int precision;
    int block;
    int ipt;
    int jt;
    int eps0;
    const void* fn;
};

const BatchVariant* batch_variants(int* count);
int batch_variant_ids(int precision, int eps0, int* ids, int max_ids);
int batch_occupancy(const BatchVariant& v);
// Zeroes the ticket counter and launches `grid` persistent CTAs.
cudaError_t batch_force_launch(const BatchVariant& v, const BatchArgs& args, int grid,
                               cudaStream_t st);

// Diagnostics per instance.  pot_args.items lists (instance, tile) items of
// batch_potential_tile() targets; item_first/item_count give each instance's items.
int batch_potential_tile();
cudaError_t batch_diagnostics_launch(const BatchArgs& pot_args, int n_pot_items,
                                     int n_instances, const double* vx, const double* vy,
                                     const double* vz, const int* item_first,
                                     const int* item_count, double* pot_part, double* out,
                                     cudaStream_t st);

}  // namespace gx
