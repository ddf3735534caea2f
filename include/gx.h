/*
 * gx.h -- C ABI of the B200 softened-gravity engine (direct O(N^2) forces, fused
 * kick-drift-kick integration, FMM P2P near-field leaves, FP64 diagnostics, batched
 * ensembles and the adjoint of the direct force).
 *
 * Plain C: pointers, sizes and status codes only; no exceptions cross this boundary.
 * Every function returns a gx_status; gx_last_error() gives the message of the last
 * failure on the calling thread.  There is no CPU fallback: without a CUDA device
 * every compute call returns GX_ERR_NO_DEVICE.
 *
 * Array arguments are structure-of-arrays FP64 (x, y, z, m, ...).  Unless a function
 * says otherwise, all arrays of one call must be either all device memory (then the
 * call is stream-ordered on `stream` and returns without synchronising) or all host
 * memory (then the call copies in, computes and copies out, and returns after the
 * stream has finished).  `stream` is a cudaStream_t; NULL means the legacy default
 * stream.
 *
 * Reference interfaces replaced (ryan-charette/galaxy-collision-simulation):
 *   cpp/cuda/cuda_solver.hpp:10-12        cuda_solver_available, compute_cuda_direct_accelerations,
 *                                          cuda_direct_leapfrog_step
 *   cpp/direct/direct_solver.hpp:22-28    compute_direct_accelerations[_for_targets]
 *   cpp/core/integrator.hpp:11-21         kick, drift, leapfrog_step
 *   cpp/core/diagnostics.hpp:11-21        Diagnostics, compute_diagnostics
 *   cpp/fmm/fmm_solver.cpp:295-310        the P2P near-field loop of evaluate_particle
 *   cpp/fmm/fmm_solver.hpp:37-47,71-83    the leaf lists (particle_indices, near_leaves)
 */
#ifndef GX_H
#define GX_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

#define GX_ABI_VERSION 1

typedef enum gx_status {
    GX_OK = 0,
    GX_ERR_INVALID_ARGUMENT = 1, /* bad size, null pointer, mixed host/device pointers ... */
    GX_ERR_NO_DEVICE = 2,        /* no usable CUDA device (the reference fell back to the CPU) */
    GX_ERR_CUDA = 3,             /* a CUDA runtime error; the message names the call */
    GX_ERR_TIMEOUT = 4,          /* a bounded wait gave up (gx_session_synchronize_timeout) */
    GX_ERR_OUT_OF_MEMORY = 5,    /* device or host allocation failed */
    GX_ERR_UNSUPPORTED = 6       /* valid request this build does not implement */
} gx_status;

typedef enum gx_precision {
    /* FP64 pair arithmetic, tiled; FMA contraction and a refined hardware rsqrt.
     * Relative error vs the reference ~1e-15. */
    GX_PRECISION_F64 = 0,
    /* FP32 pair arithmetic on offsets from a per-tile FP64 origin, per-tile compensated
     * (two-sum) accumulation, FP64 results.  Median relative error ~1e-7. */
    GX_PRECISION_MIXED = 1,
    /* FP64 with the reference's exact operation order, IEEE sqrt and division and no FMA
     * contraction: bit-identical to compute_direct_accelerations_for_targets
     * (cpp/direct/direct_solver.cpp:59-83) and, for P2P, to evaluate_particle. */
    GX_PRECISION_F64_EXACT = 2
} gx_precision;

/* PhysicsParams (cpp/core/simulation_params.hpp:5-8). */
typedef struct gx_physics {
    double G;         /* gravitational_constant */
    double softening; /* Plummer epsilon; eps^2 is added to |r|^2 */
} gx_physics;

/* Diagnostics (cpp/core/diagnostics.hpp:11-19), fields in diagnostics.csv column order. */
typedef struct gx_diagnostics {
    double total_mass;
    double kinetic_energy;
    double potential_energy;
    double total_energy;
    double momentum[3];
    double center_of_mass[3];
    double angular_momentum[3];
} gx_diagnostics;

/* ---- library -------------------------------------------------------------------- */
const char* gx_last_error(void);
int gx_abi_version(void);
/* cuda_solver_available (cpp/cuda/cuda_solver.cu:185-189): *available = 1 when a CUDA
 * device of compute capability 10.0 can be used. */
int gx_device_available(int* available);

/* ---- stateless direct sum --------------------------------------------------------- */
/* compute_cuda_direct_accelerations (cpp/cuda/cuda_solver.cu:191-210) and
 * compute_direct_accelerations (cpp/direct/direct_solver.cpp:38-57): a_i for every body. */
int gx_direct_accel(int64_t n, const double* x, const double* y, const double* z,
                    const double* m, gx_physics phys, int precision, double* ax, double* ay,
                    double* az, void* stream);

/* compute_direct_accelerations_for_targets (cpp/direct/direct_solver.cpp:59-83): targets
 * [begin, end) against all n sources; results at ax[i - begin].  With `targets` non-null,
 * targets[k] for k < n_targets instead of a range (begin/end ignored; n_targets used).
 * Host index arrays are checked (an entry outside [0, n) returns GX_ERR_INVALID_ARGUMENT);
 * device index arrays are not read back: an entry outside [0, n) is never used as an
 * address, and its row of ax, ay, az is NaN. */
int gx_direct_accel_targets(int64_t n, const double* x, const double* y, const double* z,
                            const double* m, int64_t begin, int64_t end, const int64_t* targets,
                            int64_t n_targets, gx_physics phys, int precision, double* ax,
                            double* ay, double* az, void* stream);

/* cuda_direct_leapfrog_step (cpp/cuda/cuda_solver.cu:212-246) / leapfrog_step
 * (cpp/core/integrator.cpp:33-42): one KDK step in place, reusing the caller's a as the
 * first kick's acceleration; x, v and a are updated. */
int gx_leapfrog_step(int64_t n, double* x, double* y, double* z, double* vx, double* vy,
                     double* vz, double* ax, double* ay, double* az, const double* m,
                     double dt, gx_physics phys, int precision, void* stream);

/* kick (cpp/core/integrator.cpp:7-11): v += a*dt.  drift (:13-17): x += v*dt.
 * kick_drift: v += a*kick_dt then x += v*drift_dt.  Device pointers only. */
int gx_kick(int64_t n, double* vx, double* vy, double* vz, const double* ax,
            const double* ay, const double* az, double dt, void* stream);
int gx_drift(int64_t n, double* x, double* y, double* z, const double* vx, const double* vy,
             const double* vz, double dt, void* stream);
int gx_kick_drift(int64_t n, double* x, double* y, double* z, double* vx, double* vy,
                  double* vz, const double* ax, const double* ay, const double* az,
                  double kick_dt, double drift_dt, void* stream);

/* compute_diagnostics (cpp/core/diagnostics.cpp:7-37) in FP64 on the device. */
int gx_diagnostics_compute(int64_t n, const double* x, const double* y, const double* z,
                           const double* vx, const double* vy, const double* vz,
                           const double* m, gx_physics phys, gx_diagnostics* out,
                           void* stream);

/* ---- resident session (the step loop of cpp/core/main.cpp:172-184) ------------------ */
/* The session owns device copies of the state; steps run as CUDA-graph launches with no
 * host synchronisation; host copies happen only in set_state / get_state. */
typedef struct gx_session gx_session;

int gx_session_create(int64_t n, gx_physics phys, int device, gx_session** out);
int gx_session_destroy(gx_session* s);
/* Stream the session's work is ordered on (default: a stream the session creates). */
int gx_session_set_stream(gx_session* s, void* stream);
int gx_session_get_stream(gx_session* s, void** stream);
/* Host or device arrays; a (ax..az) may be null (then accelerations are zeroed and the
 * caller computes them with gx_session_compute_accelerations). */
int gx_session_set_state(gx_session* s, const double* x, const double* y, const double* z,
                         const double* vx, const double* vy, const double* vz,
                         const double* m, const double* ax, const double* ay,
                         const double* az);
int gx_session_get_state(gx_session* s, double* x, double* y, double* z, double* vx,
                         double* vy, double* vz, double* ax, double* ay, double* az);
/* Device pointers of the resident arrays, in the order x,y,z,vx,vy,vz,ax,ay,az,m. */
int gx_session_device_arrays(gx_session* s, double** ptrs10);
int gx_session_compute_accelerations(gx_session* s, int precision);
/* n_steps KDK steps (kick dt/2, drift dt, force, kick dt/2 per step).  Systems of at most
 * 4096 bodies in GX_PRECISION_F64 or _F64_EXACT run all n_steps in one cooperative launch
 * (each step: kick-drift, one grid barrier, force, kick; the exact form stays bit-identical
 * to the reference); larger systems and the mixed form replay CUDA graphs of 32 steps.  A
 * grid barrier that cannot complete within 4 s stops the launch, leaves the state of the
 * previous call, and the next synchronising call returns GX_ERR_TIMEOUT. */
int gx_session_step(gx_session* s, int64_t n_steps, double dt, int precision);
/* Whether small systems use the single-launch step loop (default 1); 0 replays graphs of
 * separate kick-drift and force launches instead.  No reference counterpart. */
int gx_session_set_persistent(gx_session* s, int enable);
/* The session's force: the reference FMM with `opt` (the options and semantics of
 * gx_fmm_accel, declared below), or the direct sum again with opt == NULL (the default).
 * With the FMM, gx_session_step runs chunks of up to 32 KDK steps, each replayed as one CUDA
 * graph with no host synchronisation inside: the octree, lists, moments, far and near field
 * of every step run in device pools sized by a first evaluation with headroom.  After each
 * chunk the session reads one overflow word; when a pool was too small it restores the
 * chunk's starting state (copied on the device), regrows the pools and redoes the chunk, and
 * a tree that needs the host builder (more than leaf_capacity nearly coincident bodies) is
 * stepped one evaluation at a time through gx_fmm_accel's path.  Results equal gx_fmm_accel
 * between kick-drift and kick launches step by step (bit for bit in the exact form).  Owned
 * target ranges (gx_session_set_targets) are not supported with the FMM.  No reference
 * counterpart: the reference's FMM step loop is cpp/core/main.cpp:172-184 with
 * compute_fmm_accelerations (cpp/fmm/fmm_solver.cpp:315-322). */
struct gx_fmm_options;
int gx_session_set_fmm(gx_session* s, const struct gx_fmm_options* opt);
/* The bodies this session owns: [begin, begin + count) (default: all n).  Steps, the two
 * half steps below and compute_accelerations kick, drift and evaluate forces for the owned
 * bodies only, with all n bodies as sources -- the ownership range of the reference's MPI
 * step (cpp/mpi/distributed_solver.cpp:68-79, cpp/core/main.cpp:240-253).  A multi-process
 * caller exchanges the owned positions between the two halves of each step. */
int gx_session_set_targets(gx_session* s, int64_t begin, int64_t count);
/* Opening half of a KDK step for the owned bodies: v += a * kick_dt, then x += v * drift_dt
 * (kick and drift, cpp/core/integrator.cpp:7-17). */
int gx_session_kick_drift(gx_session* s, double kick_dt, double drift_dt);
/* Closing half: accelerations of the owned bodies from all n, then v += a * kick_dt. */
int gx_session_force_kick(gx_session* s, double kick_dt, int precision);
int gx_session_diagnostics(gx_session* s, gx_diagnostics* out);
/* gx_snapshot_write of the session's state on the session's stream (declared below). */
struct gx_snapshot_writer;
int gx_session_snapshot(gx_session* s, struct gx_snapshot_writer* w, int step, double time);
int gx_session_synchronize(gx_session* s);
/* Bounded host wait: GX_ERR_TIMEOUT if the stream is still busy after timeout_ms. */
int gx_session_synchronize_timeout(gx_session* s, double timeout_ms);
/* Force-kernel timing: when enabled, every force launch of the session is bracketed by
 * CUDA events on the session stream (graphs are bypassed while enabled). */
int gx_session_enable_timing(gx_session* s, int enable);
int gx_session_force_timing(gx_session* s, double* total_ms, int64_t* launches);
/* Kernel configuration used for `precision` (variant id, j-split count). */
int gx_session_get_config(gx_session* s, int precision, int* variant, int* jsplit);
int gx_session_set_config(gx_session* s, int precision, int variant, int jsplit);
/* Times the candidate configurations on the session's own state and keeps the fastest;
 * returns its time per force evaluation. */
int gx_session_autotune(gx_session* s, int precision, double* best_ms);

/* ---- FMM P2P near field (cpp/fmm/fmm_solver.cpp:295-310) --------------------------- */
/* For every body i of leaf l (leaf_particles[leaf_offsets[l] .. leaf_offsets[l+1]]),
 * adds sum over near leaves s of leaf l (near_leaves[near_offsets[l] .. [l+1]]) and their
 * bodies j != i of the pair term to (ax[i], ay[i], az[i]).  Leaf ids are row numbers of
 * leaf_offsets.  Pass the far field in a to get the reference's full FMM result.  Each body
 * sits in at most one leaf slot, as in the reference's octree: host CSR arrays that list a
 * body twice are rejected (GX_ERR_INVALID_ARGUMENT); device CSR arrays are trusted, and a
 * body listed twice there gets an unspecified sum (the kernel stays within its buffers). */
int gx_p2p_leaves(int64_t n, const double* x, const double* y, const double* z,
                  const double* m, int32_t n_leaves, const int32_t* leaf_offsets,
                  const int32_t* leaf_particles, const int32_t* near_offsets,
                  const int32_t* near_leaves, gx_physics phys, int precision, double* ax,
                  double* ay, double* az, void* stream);

/* ---- initial conditions (cpp/core/initial_conditions.cpp:37-114) ------------------ */
/* GalaxyConfig (cpp/core/initial_conditions.hpp:14-24). */
typedef struct gx_galaxy {
    int64_t n_particles;
    double mass;
    double radius;
    double position[3];
    double velocity[3];
    double orientation;
    uint32_t group_id;
    uint32_t reserved;
    double thickness;
    double inclination;
} gx_galaxy;
/* Bodies generate_galaxies makes for the list: galaxies with n_particles == 0, mass <= 0 or
 * radius <= 0 make none (initial_conditions.cpp:46-48). */
int64_t gx_galaxies_body_count(int32_t n_galaxies, const gx_galaxy* galaxies);
/* generate_galaxies (initial_conditions.cpp:92-114) on the device: the reference's disk
 * model, bodies concatenated in galaxy order, written to host or device arrays of
 * gx_galaxies_body_count entries (group_id may be NULL).  The random numbers come from a
 * counter-based generator (Philox4x32-10 keyed by the seed, counter = galaxy, body, block),
 * not from the reference's mt19937_64 stream: same distributions, different draws; a
 * galaxy's bodies do not depend on the other galaxies. */
int gx_generate_galaxies(int32_t n_galaxies, const gx_galaxy* galaxies, gx_physics phys,
                         uint64_t seed, double* x, double* y, double* z, double* vx, double* vy,
                         double* vz, double* m, uint32_t* group_id, void* stream);

/* ---- snapshot output (cpp/io/snapshot_writer.cpp:38-128) ------------------------- */
/* SnapshotWriter with output that does not stall the stepping stream.  CSV files are the
 * reference's byte for byte (snapshot_%06d.csv, diagnostics.csv); the binary form
 * snapshot_%06d.bin holds the same state as SoA doubles ("GXSNAP01", int64 n, int32 step,
 * int32 fields = 10, double time, x y z vx vy vz ax ay az m, uint32 group ids). */
#define GX_SNAPSHOT_CSV 1
#define GX_SNAPSHOT_BINARY 2
typedef struct gx_snapshot_writer gx_snapshot_writer;
/* SnapshotWriter constructor (snapshot_writer.cpp:38-57): creates `directory` and, with
 * GX_SNAPSHOT_CSV, starts diagnostics.csv with the reference's header.  n and the group ids
 * (NULL: all 0) are fixed for the writer's life; `slots` snapshots may be in flight. */
int gx_snapshot_writer_create(const char* directory, int64_t n, const uint32_t* group_id,
                              int formats, int slots, gx_snapshot_writer** out);
/* Waits until every snapshot handed over so far is written; the first write error. */
int gx_snapshot_writer_flush(gx_snapshot_writer* w);
/* Flushes, then frees the writer; returns the flush status. */
int gx_snapshot_writer_destroy(gx_snapshot_writer* w);
/* write_snapshot (snapshot_writer.cpp:72-96) of arrays x..az, m -- all host or all device
 * memory.  Device arrays are copied device-to-device on `stream` (later work on `stream`
 * may overwrite them at once), then to pinned host memory on the writer's own stream; a
 * writer thread formats and writes.  Host arrays are copied during the call.  Blocks only
 * while all slots are in flight. */
int gx_snapshot_write(gx_snapshot_writer* w, int step, double time, const double* x,
                      const double* y, const double* z, const double* vx, const double* vy,
                      const double* vz, const double* ax, const double* ay, const double* az,
                      const double* m, void* stream);
/* write_diagnostics (snapshot_writer.cpp:99-128): one row of diagnostics.csv. */
int gx_snapshot_write_diagnostics(gx_snapshot_writer* w, int step, double time,
                                  const gx_diagnostics* d);

/* The run description that SnapshotWriter::write_metadata takes from SimulationConfig
 * (cpp/core/config.hpp:20-35) and the particle count. */
typedef struct gx_run_metadata {
    const char* name;
    const char* solver;
    int64_t particle_count;
    int32_t steps;
    int32_t snapshot_every;
    int32_t dim;
    int32_t fmm_expansion_order;
    double dt;
    double gravitational_constant;
    double softening;
    double tree_theta;
    int64_t tree_leaf_capacity;
} gx_run_metadata;
/* write_metadata (snapshot_writer.cpp:49-69): metadata.json in the writer's directory, byte
 * for byte the reference's (strings with '"' and '\' escaped; doubles as the default
 * ostream format prints them, six significant digits). */
int gx_snapshot_write_metadata(gx_snapshot_writer* w, const gx_run_metadata* md);

/* ---- FMM (cpp/fmm/fmm_solver.hpp:15-20, fmm_solver.cpp:315-333) --------------------- */
/* FmmOptions with the reference's defaults: theta 0.6, leaf_capacity 16, max_depth 32,
 * expansion_order 4. */
typedef struct gx_fmm_options {
    double theta;
    int64_t leaf_capacity;
    int32_t max_depth;
    int32_t expansion_order;
} gx_fmm_options;

/* FmmStats (fmm_solver.hpp:22-27), then three counts of this engine: far_pairs = sum over
 * leaves of (bodies x far nodes), near_pairs = sum over leaves of (bodies x bodies of
 * its near leaves, itself included), tree_levels = depth of the octree + 1. */
typedef struct gx_fmm_stats {
    int64_t node_count;
    int64_t leaf_count;
    int64_t far_interactions;
    int64_t near_interactions;
    int64_t far_pairs;
    int64_t near_pairs;
    int64_t tree_levels;
} gx_fmm_stats;

/* compute_fmm_accelerations_for_targets (fmm_solver.cpp:324-333); begin = 0, end = n is
 * compute_fmm_accelerations (:315-322).  The reference octree, its interaction lists,
 * the node moments (bit-identical to the reference's), the multipole far field and the
 * P2P near field all run on the device; trees deeper than 21 levels are built on the host.
 * GX_PRECISION_F64 and _F64_EXACT evaluate the far field in FP64 (the exact form also makes
 * the near field bit-identical to the reference's loop); GX_PRECISION_MIXED evaluates both
 * fields in FP32 arithmetic on offsets taken in FP64.  Only bodies in [begin, min(end, n)) are written; bodies
 * of massless leaves get zero, as in the reference.  Masses must be >= 0 (host arrays are
 * checked).  Host or device arrays; `stats` may be NULL. */
int gx_fmm_accel(int64_t n, const double* x, const double* y, const double* z, const double* m,
                 gx_physics phys, gx_fmm_options opt, int precision, int64_t begin, int64_t end,
                 double* ax, double* ay, double* az, gx_fmm_stats* stats, void* stream);

/* gx_fmm_accel that also reports where the device time went: phase_ms[GX_FMM_PHASES]
 * receives, from CUDA events on `stream`, the octree build (host clock when the host
 * builder ran), the node moments, the interaction lists, the far field and the near
 * field, in milliseconds.  Synchronizes the stream.  No reference counterpart. */
#define GX_FMM_PHASES 5
int gx_fmm_accel_timed(int64_t n, const double* x, const double* y, const double* z,
                       const double* m, gx_physics phys, gx_fmm_options opt, int precision,
                       int64_t begin, int64_t end, double* ax, double* ay, double* az,
                       gx_fmm_stats* stats, void* stream, double* phase_ms);

/* Node data of the reference octree (p2m_m2m / compute_multipole_moments,
 * fmm_solver.cpp:157-208), computed on the device: for every node with mass > 0, numbered
 * breadth-first from the root with children in octant order, 35 doubles: centre of mass
 * (3), mass, and moment values[4..34] in the reference's exponent order.  Bit-identical
 * to the reference's.  Host arrays only; records == NULL returns the node count. */
int gx_fmm_moments(int64_t n, const double* x, const double* y, const double* z, const double* m,
                   gx_physics phys, gx_fmm_options opt, int64_t capacity, double* records,
                   int64_t* n_nodes);

/* Leaf lists of the reference octree (FastMultipoleSolver::build, fmm_solver.cpp:48-98,
 * 210-277) built on the host as CSR arrays for gx_p2p_leaves. Host arrays only. */
typedef struct gx_leaf_lists gx_leaf_lists;
int gx_leaf_lists_build(int64_t n, const double* x, const double* y, const double* z,
                        const double* m, double softening, double theta,
                        int64_t leaf_capacity, int max_depth, gx_leaf_lists** out);
/* The same lists built on the device (host arrays in, host lists out): the octree from a
 * stable sort of per-body 63-bit cell paths, the lists by a per-leaf walk.  A tree that
 * needs a split below depth 21 (more than leaf_capacity nearly coincident bodies) is built
 * by the host builder instead; *built_on_device (nullable) reports which ran. */
int gx_leaf_lists_build_device(int64_t n, const double* x, const double* y, const double* z,
                               const double* m, double softening, double theta,
                               int64_t leaf_capacity, int max_depth, void* stream,
                               gx_leaf_lists** out, int* built_on_device);
int gx_leaf_lists_info(const gx_leaf_lists* l, int32_t* n_leaves, int64_t* n_leaf_particles,
                       int64_t* n_near, int64_t* n_far, int64_t* n_p2p_pairs);
int gx_leaf_lists_export(const gx_leaf_lists* l, int32_t* leaf_offsets,
                         int32_t* leaf_particles, int32_t* near_offsets,
                         int32_t* near_leaves);
int gx_leaf_lists_free(gx_leaf_lists* l);

/* ---- batched ensembles (no reference counterpart) ---------------------------------- */
/* n_instances independent systems concatenated in one SoA; instance b owns bodies
 * offsets[b] .. offsets[b+1].  Forces never cross instances. */
int gx_batch_accel(int32_t n_instances, const int64_t* offsets, const double* x,
                   const double* y, const double* z, const double* m, gx_physics phys,
                   int precision, double* ax, double* ay, double* az, void* stream);

typedef struct gx_batch gx_batch;
int gx_batch_create(int32_t n_instances, const int64_t* offsets, gx_physics phys, int device,
                    gx_batch** out);
int gx_batch_destroy(gx_batch* b);
int gx_batch_set_stream(gx_batch* b, void* stream);
int gx_batch_set_state(gx_batch* b, const double* x, const double* y, const double* z,
                       const double* vx, const double* vy, const double* vz, const double* m);
int gx_batch_get_state(gx_batch* b, double* x, double* y, double* z, double* vx, double* vy,
                       double* vz, double* ax, double* ay, double* az);
int gx_batch_device_arrays(gx_batch* b, double** ptrs10);
int gx_batch_compute_accelerations(gx_batch* b, int precision);
/* n_steps KDK steps of every instance; captured once as one CUDA graph and replayed. */
int gx_batch_step(gx_batch* b, int64_t n_steps, double dt, int precision);
/* Per-instance diagnostics, out[n_instances]. */
int gx_batch_diagnostics(gx_batch* b, gx_diagnostics* out);
int gx_batch_synchronize(gx_batch* b);
int gx_batch_get_config(gx_batch* b, int precision, int* variant);
int gx_batch_set_config(gx_batch* b, int precision, int variant);
int gx_batch_autotune(gx_batch* b, int precision, double* best_ms);
int gx_batch_enable_timing(gx_batch* b, int enable);
int gx_batch_force_timing(gx_batch* b, double* total_ms, int64_t* launches);

/* ---- adjoint of the direct force (no reference counterpart) ------------------------ */
/* For cotangent l on the accelerations a(x, m):
 *   gx_k = dL/dx_k = G sum_j [ s^-3/2 (m_k l_j - m_j l_k) - 3 s^-5/2 (m_k l_j.d - m_j l_k.d) d ]
 *   gm_k = dL/dm_k = -G sum_j s^-3/2 l_j.d,      d = x_j - x_k, s = |d|^2 + eps^2.
 * gm may be null.  Device or host arrays (all of one kind). */
int gx_direct_vjp(int64_t n, const double* x, const double* y, const double* z,
                  const double* m, const double* lx, const double* ly, const double* lz,
                  gx_physics phys, int precision, double* gx, double* gy, double* gz,
                  double* gm, void* stream);

/* ---- direct sum without allocation (no counterpart in the reference) ---------------- */
/* For callers that cannot allocate device memory at call time (memory reserved up front by
 * another allocator, real-time loops that must stay out of the allocator, code running under
 * a stream capture that forbids allocation).  Same result as gx_direct_accel on DEVICE arrays,
 * but the partial sums of the source split live in one fixed 12 MiB device array that is part
 * of the library (held by every GPU that loads it until exit) -- nothing is allocated or freed.
 * Limits: n <= 65536 (larger n returns GX_ERR_INVALID_ARGUMENT); device pointers only.  The
 * first call on a device looks up the array's device address; make that first call before any
 * stream capture.  Every call shares the array and it keeps the last call's contents (each
 * call overwrites every element it reads, so nothing needs clearing); calls that overlap on
 * the GPU -- on different streams, or different host threads -- race on it. */
int gx_direct_accel_noalloc(int64_t n, const double* x, const double* y, const double* z,
                            const double* m, gx_physics phys, int precision, double* ax,
                            double* ay, double* az, void* stream);

/* ---- kernel variants ---------------------------------------------------------------- */
/* Number of direct-force variants for a precision and a printable description. */
int gx_variant_count(int precision, int* count);
int gx_variant_describe(int precision, int variant, char* buf, int buflen);

/* ---- fault injection for tests (no GPU fault: failures are made on the host or by a
 * participant that leaves a bounded wait) ----------------------------------------------- */
/* The next `count` device allocations made by the library fail with GX_ERR_OUT_OF_MEMORY. */
int gx_debug_fail_allocations(int count);
/* The next single-launch session step loop (gx_session_step on a small system) loses one
 * participant: its first CTA leaves before the barrier of step `step` instead of arriving,
 * and the barrier waits are cut to 0.2 s, so the other CTAs give up, the launch ends early
 * and the next synchronising session call returns GX_ERR_TIMEOUT.  Nothing faults. */
int gx_debug_stall_barrier(int64_t step);
/* Targets per thread of the FP64 and mixed P2P kernels: 2 or 4 forces that shape, 0 restores
 * the default (2).  For measurements; results agree within the forms' tolerances either way. */
int gx_debug_p2p_targets_per_thread(int tpt);
/* Targets per warp of the single-launch step loop: 1, 2 or 4 forces that shape, 0 (default)
 * picks it from n.  For measurements; results agree within the forms' tolerances (the exact
 * form stays bit-identical) either way. */
int gx_debug_small_targets_per_warp(int tpw);
/* Warps per target of the FP64 single-launch step loop: 1 or 2 forces that shape, 0 (default)
 * picks it.  For measurements; results agree within the FP64 tolerance either way. */
int gx_debug_small_warps_per_target(int wpt);
/* Sessions that set up their FMM pools after this call size them with no headroom (1) or
 * with the default half again plus a margin (0), so that tests can make a pool overflow and
 * check that the step is redone with regrown pools.  With 1 the tree sort also starts with
 * one level of the path keys, so the first tree deeper than that is redone with all levels. */
int gx_debug_fmm_tight_pools(int enable);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* GX_H */
