/*
 * gx_oracle.c -- TEST INFRASTRUCTURE ONLY (the parity checker, never the product).
 *
 * A plain-C, single-precision-free (FP64 throughout) restatement of the reference
 * softened-gravity path of ryan-charette/galaxy-collision-simulation.  Only
 * tests/, __graft_entry__.smoke() and bench.py's cpu_baseline / reference leg may
 * load this library, and only as the checker or the timed CPU baseline.  The
 * product (the CUDA engine behind include/gx.h) never links, loads or calls it.
 *
 * Every function reproduces the reference's operation order so that results are
 * bit-identical to the reference C++ on the same inputs when both are built with
 * -ffp-contract=off (the reference builds with -std=c++17, i.e. without FMA
 * contraction on x86-64):
 *   pair term            cpp/direct/direct_solver.cpp:8-23   (softened_acceleration)
 *   symmetric all-pairs  cpp/direct/direct_solver.cpp:38-57  (compute_direct_accelerations)
 *   per-target gather    cpp/direct/direct_solver.cpp:59-83  (..._for_targets)
 *   kick / drift / KDK   cpp/core/integrator.cpp:7-42
 *   diagnostics          cpp/core/diagnostics.cpp:7-37
 *   octree leaf lists    cpp/fmm/fmm_solver.cpp:48-98,104-155,157-182,210-277
 *   P2P near-field loop  cpp/fmm/fmm_solver.cpp:295-310
 *   ownership ranges     cpp/mpi/distributed_solver.cpp:68-79
 *
 * The oracle is pinned against the reference's golden snapshots and its smoke-test
 * known-answer case (tests/golden/, tests/test_oracle_golden.py).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORACLE_API __attribute__((visibility("default")))

/* ---- a1: one pair term (direct_solver.cpp:8-23) ---------------------------------- */
static inline void pair_term(double tx, double ty, double tz, double sx, double sy, double sz,
                             double m, double G, double eps, double out[3]) {
    const double rx = sx - tx, ry = sy - ty, rz = sz - tz;
    const double eps2 = eps * eps;
    const double s2 = (rx * rx + ry * ry + rz * rz) + eps2; /* norm_squared(r) + eps2 */
    if (s2 == 0.0) {
        out[0] = 0.0; out[1] = 0.0; out[2] = 0.0;
        return;
    }
    const double inv_r = 1.0 / sqrt(s2);
    const double inv_r3 = inv_r * inv_r * inv_r;
    const double scale = G * m * inv_r3;
    out[0] = rx * scale; out[1] = ry * scale; out[2] = rz * scale;
}

ORACLE_API void oracle_pair(double tx, double ty, double tz, double sx, double sy, double sz,
                            double m, double G, double eps, double* out3) {
    pair_term(tx, ty, tz, sx, sy, sz, m, G, eps, out3);
}

/* ---- a3: per-target gather over all j ascending, skip i==j (direct_solver.cpp:59-83) - */
ORACLE_API void oracle_direct_targets(int64_t n, const double* x, const double* y, const double* z,
                                      const double* m, double G, double eps, int64_t begin,
                                      int64_t end, double* ax, double* ay, double* az) {
    if (end > n) end = n;
    for (int64_t i = begin; i < end; ++i) {
        double acc[3] = {0.0, 0.0, 0.0}, t[3];
        for (int64_t j = 0; j < n; ++j) {
            if (i == j) continue;
            pair_term(x[i], y[i], z[i], x[j], y[j], z[j], m[j], G, eps, t);
            acc[0] += t[0]; acc[1] += t[1]; acc[2] += t[2];
        }
        ax[i] = acc[0]; ay[i] = acc[1]; az[i] = acc[2];
    }
}

/* Same gather for an explicit target list; results land at out[k] for targets[k]. */
ORACLE_API void oracle_direct_indexed(int64_t n, const double* x, const double* y, const double* z,
                                      const double* m, double G, double eps, int64_t n_targets,
                                      const int64_t* targets, double* ax, double* ay, double* az) {
    for (int64_t k = 0; k < n_targets; ++k) {
        const int64_t i = targets[k];
        double acc[3] = {0.0, 0.0, 0.0}, t[3];
        for (int64_t j = 0; j < n; ++j) {
            if (i == j) continue;
            pair_term(x[i], y[i], z[i], x[j], y[j], z[j], m[j], G, eps, t);
            acc[0] += t[0]; acc[1] += t[1]; acc[2] += t[2];
        }
        ax[k] = acc[0]; ay[k] = acc[1]; az[k] = acc[2];
    }
}

/* ---- ownership ranges (distributed_solver.cpp:68-79) ------------------------------- */
ORACLE_API void oracle_ownership(int64_t count, int rank, int size, int64_t* begin, int64_t* end) {
    if (size <= 1) { *begin = 0; *end = count; return; }
    const int64_t base = count / size, rem = count % size;
    const int64_t b = (int64_t)rank * base + ((int64_t)rank < rem ? (int64_t)rank : rem);
    *begin = b;
    *end = b + base + ((int64_t)rank < rem ? 1 : 0);
}

/* Threaded a3 over ownership ranges of an explicit target list (CPU baseline timing). */
typedef struct {
    int64_t n; const double *x, *y, *z, *m; double G, eps;
    int64_t n_targets; const int64_t* targets; double *ax, *ay, *az; int rank, size;
} mt_job;

static void* mt_worker(void* arg) {
    mt_job* j = (mt_job*)arg;
    int64_t b, e;
    oracle_ownership(j->n_targets, j->rank, j->size, &b, &e);
    oracle_direct_indexed(j->n, j->x, j->y, j->z, j->m, j->G, j->eps, e - b, j->targets + b,
                          j->ax + b, j->ay + b, j->az + b);
    return NULL;
}

ORACLE_API int oracle_direct_indexed_mt(int64_t n, const double* x, const double* y, const double* z,
                                        const double* m, double G, double eps, int64_t n_targets,
                                        const int64_t* targets, double* ax, double* ay, double* az,
                                        int threads) {
    if (threads < 1) threads = 1;
    pthread_t* tid = (pthread_t*)calloc((size_t)threads, sizeof(pthread_t));
    mt_job* jobs = (mt_job*)calloc((size_t)threads, sizeof(mt_job));
    if (!tid || !jobs) { free(tid); free(jobs); return -1; }
    for (int r = 0; r < threads; ++r) {
        mt_job jb = {n, x, y, z, m, G, eps, n_targets, targets, ax, ay, az, r, threads};
        jobs[r] = jb;
        pthread_create(&tid[r], NULL, mt_worker, &jobs[r]);
    }
    for (int r = 0; r < threads; ++r) pthread_join(tid[r], NULL);
    free(tid); free(jobs);
    return 0;
}

/* ---- a2: symmetric all-pairs with Newton-3 update (direct_solver.cpp:38-57) ---------- */
ORACLE_API void oracle_direct_symmetric(int64_t n, const double* x, const double* y, const double* z,
                                        const double* m, double G, double eps, double* ax,
                                        double* ay, double* az) {
    for (int64_t i = 0; i < n; ++i) { ax[i] = 0.0; ay[i] = 0.0; az[i] = 0.0; }
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = i + 1; j < n; ++j) {
            const double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
            const double eps2 = eps * eps;
            const double s2 = (dx * dx + dy * dy + dz * dz) + eps2;
            if (s2 == 0.0) continue;
            const double inv_r = 1.0 / sqrt(s2);
            const double inv_r3 = inv_r * inv_r * inv_r;
            const double scale = G * inv_r3;
            const double si = scale * m[j], sj = scale * m[i];
            ax[i] += dx * si; ay[i] += dy * si; az[i] += dz * si;
            ax[j] -= dx * sj; ay[j] -= dy * sj; az[j] -= dz * sj;
        }
    }
}

/* ---- a7: kick, drift, KDK leapfrog (integrator.cpp:7-42) ---------------------------- */
ORACLE_API void oracle_kick(int64_t n, double* vx, double* vy, double* vz, const double* ax,
                            const double* ay, const double* az, double dt) {
    for (int64_t i = 0; i < n; ++i) { vx[i] += ax[i] * dt; vy[i] += ay[i] * dt; vz[i] += az[i] * dt; }
}

ORACLE_API void oracle_drift(int64_t n, double* x, double* y, double* z, const double* vx,
                             const double* vy, const double* vz, double dt) {
    for (int64_t i = 0; i < n; ++i) { x[i] += vx[i] * dt; y[i] += vy[i] * dt; z[i] += vz[i] * dt; }
}

/* solver: 0 = symmetric a2 (the CLI's "direct"), 1 = per-target a3 (CUDA-kernel order) */
ORACLE_API void oracle_leapfrog(int64_t n, double* x, double* y, double* z, double* vx, double* vy,
                                double* vz, double* ax, double* ay, double* az, const double* m,
                                double G, double eps, double dt, int steps, int solver) {
    for (int s = 0; s < steps; ++s) {
        oracle_kick(n, vx, vy, vz, ax, ay, az, 0.5 * dt);
        oracle_drift(n, x, y, z, vx, vy, vz, dt);
        if (solver == 0)
            oracle_direct_symmetric(n, x, y, z, m, G, eps, ax, ay, az);
        else
            oracle_direct_targets(n, x, y, z, m, G, eps, 0, n, ax, ay, az);
        oracle_kick(n, vx, vy, vz, ax, ay, az, 0.5 * dt);
    }
}

/* ---- a9: diagnostics (diagnostics.cpp:7-37) ----------------------------------------
 * out[13] = total_mass, kinetic, potential, total, momentum xyz, centre of mass xyz,
 * angular momentum xyz -- the column order of the reference's diagnostics.csv. */
ORACLE_API void oracle_diagnostics(int64_t n, const double* x, const double* y, const double* z,
                                   const double* vx, const double* vy, const double* vz,
                                   const double* m, double G, double eps, double* out) {
    double M = 0.0, KE = 0.0, PE = 0.0, P[3] = {0, 0, 0}, C[3] = {0, 0, 0}, L[3] = {0, 0, 0};
    for (int64_t i = 0; i < n; ++i) {
        M += m[i];
        KE += 0.5 * m[i] * (vx[i] * vx[i] + vy[i] * vy[i] + vz[i] * vz[i]);
        P[0] += vx[i] * m[i]; P[1] += vy[i] * m[i]; P[2] += vz[i] * m[i];
        C[0] += x[i] * m[i]; C[1] += y[i] * m[i]; C[2] += z[i] * m[i];
        const double cx = y[i] * vz[i] - z[i] * vy[i];
        const double cy = z[i] * vx[i] - x[i] * vz[i];
        const double cz = x[i] * vy[i] - y[i] * vx[i];
        L[0] += cx * m[i]; L[1] += cy * m[i]; L[2] += cz * m[i];
    }
    if (M > 0.0) { C[0] /= M; C[1] /= M; C[2] /= M; }
    const double eps2 = eps * eps;
    for (int64_t i = 0; i < n; ++i) {
        for (int64_t j = i + 1; j < n; ++j) {
            const double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
            const double d = sqrt((dx * dx + dy * dy + dz * dz) + eps2);
            if (d == 0.0) continue;
            PE -= G * m[i] * m[j] / d;
        }
    }
    out[0] = M; out[1] = KE; out[2] = PE; out[3] = KE + PE;
    out[4] = P[0]; out[5] = P[1]; out[6] = P[2];
    out[7] = C[0]; out[8] = C[1]; out[9] = C[2];
    out[10] = L[0]; out[11] = L[1]; out[12] = L[2];
}

/* ---- a8: octree leaf lists (fmm_solver.cpp:48-98,104-155,157-182,210-277) ------------
 * The reference inserts bodies one at a time; a node splits when it would hold more
 * than leaf_capacity bodies and its depth is below max_depth.  The resulting tree is the
 * recursive 8-way partition below, with each leaf's bodies in ascending index order.
 * Leaves are numbered in depth-first child order 0..7 (collect_leaves); near lists are
 * in the depth-first order of build_leaf_interactions. */
typedef struct {
    double c[3], hw, mass;
    int child0;           /* index of child 0 (children are consecutive) or -1 for a leaf */
    int64_t pbeg, pend;   /* range into the permutation array (leaves only) */
    int leaf_id;          /* ordinal among collected leaves, -1 if not collected */
} onode;

typedef struct {
    onode* nodes; int n_nodes, cap_nodes;
    int64_t* perm;        /* body indices grouped by leaf */
    int64_t* tmp;
    const double *x, *y, *z, *m;
    int64_t leaf_capacity; int max_depth;
} otree;

static int push_node(otree* t) {
    if (t->n_nodes == t->cap_nodes) {
        int nc = t->cap_nodes ? 2 * t->cap_nodes : 1024;
        onode* nn = (onode*)realloc(t->nodes, (size_t)nc * sizeof(onode));
        if (!nn) return -1;
        t->nodes = nn; t->cap_nodes = nc;
    }
    return t->n_nodes++;
}

static int build_node(otree* t, int node, int64_t beg, int64_t end, int depth) {
    onode* nd = &t->nodes[node];
    nd->child0 = -1; nd->pbeg = beg; nd->pend = end; nd->leaf_id = -1;
    if ((end - beg) <= t->leaf_capacity || depth >= t->max_depth) {
        double mass = 0.0;
        for (int64_t k = beg; k < end; ++k) mass += t->m[t->perm[k]];
        t->nodes[node].mass = mass;
        return 0;
    }
    /* subdivide (fmm_solver.cpp:111-131): children centred at c +/- hw/2 per octant bit */
    const double chw = nd->hw * 0.5;
    const double pc[3] = {nd->c[0], nd->c[1], nd->c[2]};
    int first = -1;
    for (int c = 0; c < 8; ++c) {
        int id = push_node(t);
        if (id < 0) return -1;
        if (c == 0) first = id;
        onode* ch = &t->nodes[id];
        const double sx = (c & 1) ? 1.0 : -1.0, sy = (c & 2) ? 1.0 : -1.0, sz = (c & 4) ? 1.0 : -1.0;
        ch->c[0] = pc[0] + sx * chw; ch->c[1] = pc[1] + sy * chw; ch->c[2] = pc[2] + sz * chw;
        ch->hw = chw;
    }
    t->nodes[node].child0 = first;
    /* stable partition by child_index_for (fmm_solver.cpp:104-109) */
    int64_t counts[8] = {0};
    for (int64_t k = beg; k < end; ++k) {
        const int64_t p = t->perm[k];
        const int oct = (t->x[p] >= pc[0] ? 1 : 0) + 2 * (t->y[p] >= pc[1] ? 1 : 0) + 4 * (t->z[p] >= pc[2] ? 1 : 0);
        counts[oct]++;
    }
    int64_t off[8], run = beg;
    for (int c = 0; c < 8; ++c) { off[c] = run; run += counts[c]; }
    for (int64_t k = beg; k < end; ++k) {
        const int64_t p = t->perm[k];
        const int oct = (t->x[p] >= pc[0] ? 1 : 0) + 2 * (t->y[p] >= pc[1] ? 1 : 0) + 4 * (t->z[p] >= pc[2] ? 1 : 0);
        t->tmp[off[oct]++] = p;
    }
    memcpy(t->perm + beg, t->tmp + beg, (size_t)(end - beg) * sizeof(int64_t));
    run = beg;
    double mass = 0.0;
    for (int c = 0; c < 8; ++c) {
        if (build_node(t, first + c, run, run + counts[c], depth + 1) != 0) return -1;
        run += counts[c];
        mass += t->nodes[first + c].mass; /* p2m_m2m: parent mass = sum of child masses */
    }
    t->nodes[node].mass = mass;
    return 0;
}

static void collect(otree* t, int node, int* leaves, int* nl) {
    onode* nd = &t->nodes[node];
    if (nd->mass <= 0.0) return;
    if (nd->child0 < 0) { nd->leaf_id = *nl; leaves[(*nl)++] = node; return; }
    for (int c = 0; c < 8; ++c) collect(t, nd->child0 + c, leaves, nl);
}

static int well_separated(const onode* T, const onode* S, double theta) {
    if (S->mass <= 0.0) return 0;
    const double dx = S->c[0] - T->c[0], dy = S->c[1] - T->c[1], dz = S->c[2] - T->c[2];
    const double dist = sqrt(dx * dx + dy * dy + dz * dz);
    if (dist == 0.0) return 0;
    const double comb = 2.0 * (T->hw + S->hw);
    return comb / dist < theta;
}

typedef struct { int32_t* v; int64_t n, cap; } ivec;
static int ivec_push(ivec* a, int32_t x) {
    if (a->n == a->cap) {
        int64_t nc = a->cap ? 2 * a->cap : 4096;
        int32_t* nv = (int32_t*)realloc(a->v, (size_t)nc * sizeof(int32_t));
        if (!nv) return -1;
        a->v = nv; a->cap = nc;
    }
    a->v[a->n++] = x;
    return 0;
}

static int walk(otree* t, int target, int source, double theta, ivec* near, int64_t* n_far) {
    const onode* S = &t->nodes[source];
    if (S->mass <= 0.0) return 0;
    if (source != target && well_separated(&t->nodes[target], S, theta)) { (*n_far)++; return 0; }
    if (S->child0 < 0) return ivec_push(near, (int32_t)S->leaf_id);
    for (int c = 0; c < 8; ++c)
        if (walk(t, target, S->child0 + c, theta, near, n_far) != 0) return -1;
    return 0;
}

/* Builds the reference's leaf lists as CSR.  Returns 0 on success.  Caller frees the
 * four output arrays with oracle_free.  leaf ids index leaf_offsets / near_offsets. */
ORACLE_API int oracle_leaf_lists(int64_t n, const double* x, const double* y, const double* z,
                                 const double* m, double eps, double theta, int64_t leaf_capacity,
                                 int max_depth, int32_t* n_leaves_out, int32_t** leaf_offsets,
                                 int32_t** leaf_particles, int32_t** near_offsets,
                                 int32_t** near_leaves, int64_t* n_near_out, int64_t* n_far_out) {
    otree t;
    memset(&t, 0, sizeof(t));
    if (n <= 0) return -1;
    t.x = x; t.y = y; t.z = z; t.m = m;
    /* FastMultipoleSolver ctor clamps (fmm_solver.cpp:12-18) */
    t.leaf_capacity = leaf_capacity < 1 ? 1 : leaf_capacity;
    t.max_depth = max_depth < 1 ? 1 : max_depth;
    if (theta < 1.0e-6) theta = 1.0e-6;
    t.perm = (int64_t*)malloc((size_t)n * sizeof(int64_t));
    t.tmp = (int64_t*)malloc((size_t)n * sizeof(int64_t));
    if (!t.perm || !t.tmp) return -1;
    double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
    for (int64_t i = 0; i < n; ++i) {
        t.perm[i] = i;
        mn[0] = fmin(mn[0], x[i]); mn[1] = fmin(mn[1], y[i]); mn[2] = fmin(mn[2], z[i]);
        mx[0] = fmax(mx[0], x[i]); mx[1] = fmax(mx[1], y[i]); mx[2] = fmax(mx[2], z[i]);
    }
    int root = push_node(&t);
    if (root < 0) return -1;
    onode* r = &t.nodes[root];
    r->c[0] = (mn[0] + mx[0]) * 0.5; r->c[1] = (mn[1] + mx[1]) * 0.5; r->c[2] = (mn[2] + mx[2]) * 0.5;
    double ext = mx[0] - mn[0];
    if (mx[1] - mn[1] > ext) ext = mx[1] - mn[1];
    if (mx[2] - mn[2] > ext) ext = mx[2] - mn[2];
    double hw = 0.5 * ext;
    if (hw < eps + 1.0e-6) hw = eps + 1.0e-6;
    r->hw = hw * 1.0001;
    if (build_node(&t, root, 0, n, 0) != 0) return -1;

    int* leaves = (int*)malloc((size_t)t.n_nodes * sizeof(int));
    int nl = 0;
    collect(&t, root, leaves, &nl);
    int32_t* lo = (int32_t*)malloc((size_t)(nl + 1) * sizeof(int32_t));
    int32_t* lp = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    int32_t* no = (int32_t*)malloc((size_t)(nl + 1) * sizeof(int32_t));
    ivec near = {0, 0, 0};
    int64_t n_far = 0, run = 0;
    for (int l = 0; l < nl; ++l) {
        const onode* L = &t.nodes[leaves[l]];
        lo[l] = (int32_t)run;
        for (int64_t k = L->pbeg; k < L->pend; ++k) lp[run++] = (int32_t)t.perm[k];
        no[l] = (int32_t)near.n;
        if (walk(&t, leaves[l], root, theta, &near, &n_far) != 0) return -1;
    }
    lo[nl] = (int32_t)run; no[nl] = (int32_t)near.n;
    *n_leaves_out = nl; *leaf_offsets = lo; *leaf_particles = lp; *near_offsets = no;
    *near_leaves = near.v; *n_near_out = near.n; *n_far_out = n_far;
    free(leaves); free(t.nodes); free(t.perm); free(t.tmp);
    return 0;
}

ORACLE_API void oracle_free(void* p) { free(p); }

/* ---- a8: P2P near field (fmm_solver.cpp:295-310) ------------------------------------
 * For every body of every leaf, adds the near-leaf pair terms (source order: near list
 * order, then leaf body order; self skipped by index) to acc, starting from the value
 * already in ax/ay/az -- exactly how evaluate_particle continues after its far field. */
ORACLE_API void oracle_p2p_near(int64_t n, const double* x, const double* y, const double* z,
                                const double* m, double G, double eps, int32_t n_leaves,
                                const int32_t* leaf_offsets, const int32_t* leaf_particles,
                                const int32_t* near_offsets, const int32_t* near_leaves,
                                double* ax, double* ay, double* az) {
    (void)n;
    for (int32_t l = 0; l < n_leaves; ++l) {
        for (int32_t a = leaf_offsets[l]; a < leaf_offsets[l + 1]; ++a) {
            const int32_t i = leaf_particles[a];
            double acc[3] = {ax[i], ay[i], az[i]}, t[3];
            for (int32_t q = near_offsets[l]; q < near_offsets[l + 1]; ++q) {
                const int32_t s = near_leaves[q];
                for (int32_t b = leaf_offsets[s]; b < leaf_offsets[s + 1]; ++b) {
                    const int32_t j = leaf_particles[b];
                    if (j == i) continue;
                    pair_term(x[i], y[i], z[i], x[j], y[j], z[j], m[j], G, eps, t);
                    acc[0] += t[0]; acc[1] += t[1]; acc[2] += t[2];
                }
            }
            ax[i] = acc[0]; ay[i] = acc[1]; az[i] = acc[2];
        }
    }
}

/* ---- adjoint: vector-Jacobian product of the direct accelerations ---------------------
 * No reference counterpart (the reference has no gradients).  For a = G sum_j m_j d s^-3/2
 * with d = x_j - x_i, s = |d|^2 + eps^2 and a cotangent lambda on a:
 *   dL/dx_k = G sum_j [ s^-3/2 (m_k l_j - m_j l_k) - 3 s^-5/2 (m_k l_j.d - m_j l_k.d) d ],
 *   dL/dm_k = -G sum_j s^-3/2 l_j.d,            d = x_j - x_k.
 * Straight double loops; pairs with s == 0 are skipped like the forward. */
ORACLE_API void oracle_direct_vjp(int64_t n, const double* x, const double* y, const double* z,
                                  const double* m, const double* lx, const double* ly,
                                  const double* lz, double G, double eps, double* gx, double* gy,
                                  double* gz, double* gm) {
    const double eps2 = eps * eps;
    for (int64_t k = 0; k < n; ++k) {
        double g[3] = {0, 0, 0}, h = 0.0;
        for (int64_t j = 0; j < n; ++j) {
            if (j == k) continue;
            const double d[3] = {x[j] - x[k], y[j] - y[k], z[j] - z[k]};
            const double s = d[0] * d[0] + d[1] * d[1] + d[2] * d[2] + eps2;
            if (s == 0.0) continue;
            const double i3 = 1.0 / (s * sqrt(s)), i5 = i3 / s;
            const double lj[3] = {lx[j], ly[j], lz[j]}, lk[3] = {lx[k], ly[k], lz[k]};
            const double ljd = lj[0] * d[0] + lj[1] * d[1] + lj[2] * d[2];
            const double lkd = lk[0] * d[0] + lk[1] * d[1] + lk[2] * d[2];
            const double c = 3.0 * i5 * (m[k] * ljd - m[j] * lkd);
            for (int q = 0; q < 3; ++q) g[q] += i3 * (m[k] * lj[q] - m[j] * lk[q]) - c * d[q];
            h -= i3 * ljd;
        }
        gx[k] = G * g[0]; gy[k] = G * g[1]; gz[k] = G * g[2];
        if (gm) gm[k] = G * h;
    }
}

/* ---- disk initial conditions ------------------------------------------------------------
 * generate_disk_galaxy (cpp/core/initial_conditions.cpp:37-89) with the draws of the engine's
 * counter-based generator: Philox4x32-10 (Salmon et al., SC'11) keyed by the seed, counter
 * (body, body >> 32, galaxy index, block), two 53-bit uniforms per block, Box-Muller normals.
 * One galaxy; `gal_index` is its position in the caller's galaxy list. */
static void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0], p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0, n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        c[0] = n0;
        c[1] = (uint32_t)p1;
        c[2] = n2;
        c[3] = (uint32_t)p0;
        k0 += 0x9E3779B9u;
        k1 += 0xBB67AE85u;
    }
}

static double u53(uint32_t hi, uint32_t lo) {
    return (double)((((uint64_t)hi << 32) | lo) >> 11) * (1.0 / 9007199254740992.0);
}

ORACLE_API void oracle_generate_disk(int64_t n, double mass, double radius, double thickness, double orientation,
                                     double inclination, const double* pos, const double* vel, uint32_t gal_index,
                                     double G, double eps, uint64_t seed, double* x, double* y, double* z,
                                     double* vx, double* vy, double* vz, double* m) {
    const double pi = 3.141592653589793238462643383279502884;
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const double pm = mass / (double)n;
    const double disp = 0.025 * sqrt(G * mass / radius);
    const double scale = radius / 3.0;
    const double max_cdf = 1.0 - exp(-radius / scale);
    for (int64_t i = 0; i < n; ++i) {
        uint32_t c[3][4];
        for (uint32_t b = 0; b < 3; ++b) {
            c[b][0] = (uint32_t)i;
            c[b][1] = (uint32_t)((uint64_t)i >> 32);
            c[b][2] = gal_index;
            c[b][3] = b;
            philox4x32_10(c[b], k0, k1);
        }
        const double u_r = u53(c[0][0], c[0][1]), u_t = u53(c[0][2], c[0][3]);
        const double b1 = sqrt(-2.0 * log(1.0 - u53(c[1][0], c[1][1]))), a1 = 2.0 * pi * u53(c[1][2], c[1][3]);
        const double b2 = sqrt(-2.0 * log(1.0 - u53(c[2][0], c[2][1]))), a2 = 2.0 * pi * u53(c[2][2], c[2][3]);
        const double nz = b1 * cos(a1), nvx = b1 * sin(a1), nvy = b2 * cos(a2), nvz = b2 * sin(a2);
        double u = u_r < 1.0e-12 ? 1.0e-12 : u_r;
        if (u > 1.0 - 1.0e-12) u = 1.0 - 1.0e-12;
        const double r = -scale * log(1.0 - u * max_cdf);            /* :28-33 */
        const double th = 2.0 * pi * u_t;
        const double lp[3] = {r * cos(th), r * sin(th), thickness > 0.0 ? thickness * nz : 0.0};
        double frac = (r * r) / (radius * radius);
        if (frac > 1.0) frac = 1.0;
        const double menc = mass * frac > pm ? mass * frac : pm;       /* :66-67 */
        const double sr2 = r * r + eps * eps;
        const double vc = sqrt(G * menc * r * r / pow(sr2, 1.5));      /* :68-72 */
        const double lv[3] = {-sin(th) * vc + disp * nvx, cos(th) * vc + disp * nvy, 0.25 * disp * nvz};
        const double ci = cos(inclination), si = sin(inclination), co = cos(orientation), so = sin(orientation);
        double* outp[3] = {x, y, z};
        double* outv[3] = {vx, vy, vz};
        for (int w = 0; w < 2; ++w) {                                   /* rotate_x, then rotate_z (:11-26) */
            const double* v = w ? lv : lp;
            const double y1 = ci * v[1] - si * v[2], z1 = si * v[1] + ci * v[2];
            const double o[3] = {co * v[0] - so * y1, so * v[0] + co * y1, z1};
            for (int a = 0; a < 3; ++a) (w ? outv : outp)[a][i] = (w ? vel : pos)[a] + o[a];
        }
        m[i] = pm;
    }
}
