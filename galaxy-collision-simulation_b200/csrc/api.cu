// api.cu -- the C ABI of include/gx.h: argument checking, host/device pointer handling,
// kernel-variant choice (with the j-split sized by a wave-quantisation model), the
// resident session with CUDA-graph stepping, batched ensembles, the adjoint and the
// autotuner.  No exception crosses the ABI; every entry point returns a gx_status and
// records a message for gx_last_error() on the calling thread.
#include "gx.h"

#include "batch.cuh"
#include "fmm.cuh"
#include "fmm_build.cuh"
#include "fmm_tree.hpp"
#include "force.cuh"
#include "integrate.cuh"
#include "p2p.cuh"
#include "small.cuh"
#include "vjp.cuh"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <initializer_list>
#include <limits>
#include <map>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

using namespace gx;

// ======================================================================================
// errors
// ======================================================================================
namespace {
thread_local std::string g_err;
std::atomic<int> g_fail_allocs{0};
std::atomic<int64_t> g_stall_step{-1};  // gx_debug_stall_barrier
std::atomic<int> g_fmm_tight_pools{0};  // gx_debug_fmm_tight_pools: no headroom (tests of the regrowth)

int fail(int code, const char* fmt, ...) {
    char buf[1024];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_err = buf;
    return code;
}

int fail_cuda(cudaError_t e, const char* what) {
    cudaGetLastError();  // clear a non-sticky error so the context stays usable
    return fail(e == cudaErrorMemoryAllocation ? GX_ERR_OUT_OF_MEMORY : GX_ERR_CUDA, "%s: %s (%s)",
                what, cudaGetErrorString(e), cudaGetErrorName(e));
}

#define GX_CUDA(call)                                        \
    do {                                                     \
        cudaError_t e_ = (call);                             \
        if (e_ != cudaSuccess) return fail_cuda(e_, #call);  \
    } while (0)

#define GX_TRY(call)                    \
    do {                                \
        int s_ = (call);                \
        if (s_ != GX_OK) return s_;     \
    } while (0)

#define GX_GUARD_BEGIN try {
#define GX_GUARD_END                                                                 \
    }                                                                                \
    catch (const std::bad_alloc&) {                                                  \
        return fail(GX_ERR_OUT_OF_MEMORY, "host allocation failed");                 \
    }                                                                                \
    catch (...) {                                                                    \
        return fail(GX_ERR_CUDA, "unexpected C++ exception inside the gx library");  \
    }

cudaError_t dev_alloc(void** p, size_t bytes) {
    int left = g_fail_allocs.load();
    while (left > 0) {
        if (g_fail_allocs.compare_exchange_weak(left, left - 1)) return cudaErrorMemoryAllocation;
    }
    return cudaMalloc(p, bytes ? bytes : 16);
}

cudaMemPool_t library_pool(int dev);

// Stream-ordered scratch from the library's own memory pool (library_pool), never from the
// device's default pool that the host application may be using.
cudaError_t dev_alloc_async(void** p, size_t bytes, cudaStream_t st) {
    int left = g_fail_allocs.load();
    while (left > 0) {
        if (g_fail_allocs.compare_exchange_weak(left, left - 1)) return cudaErrorMemoryAllocation;
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    cudaMemPool_t pool = library_pool(dev);
    if (!pool) return cudaErrorMemoryAllocation;
    return cudaMallocFromPoolAsync(p, bytes ? bytes : 16, pool, st);
}

// ======================================================================================
// devices, pointers
// ======================================================================================
int g_dev_status = -1;  // -1 unknown, else GX_OK / GX_ERR_NO_DEVICE
std::string g_dev_msg;
std::once_flag g_dev_once;

int require_device() {
    std::call_once(g_dev_once, [] {
        int count = 0;
        cudaError_t e = cudaGetDeviceCount(&count);
        if (e != cudaSuccess || count <= 0) {
            cudaGetLastError();
            g_dev_status = GX_ERR_NO_DEVICE;
            g_dev_msg = std::string("no CUDA device: ") + (e != cudaSuccess ? cudaGetErrorString(e) : "count is 0");
            return;
        }
        for (int d = 0; d < count; ++d) {
            cudaDeviceProp p;
            if (cudaGetDeviceProperties(&p, d) == cudaSuccess && p.major == 10 && p.minor == 0) {
                g_dev_status = GX_OK;
                return;
            }
        }
        g_dev_status = GX_ERR_NO_DEVICE;
        g_dev_msg = "no device of compute capability 10.0 (this build targets sm_100a only)";
    });
    if (g_dev_status != GX_OK) return fail(GX_ERR_NO_DEVICE, "%s", g_dev_msg.c_str());
    return GX_OK;
}

int sm_count(int dev) {
    static std::mutex mu;
    static std::map<int, int> cache;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    int v = 148;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
        cudaGetLastError();
        v = 148;
    }
    cache[dev] = v;
    return v;
}

// Stream-ordered scratch comes from a memory pool the library creates for each device (its
// release threshold is unlimited, so repeated calls on host arrays reuse the same memory
// instead of remapping it).  The device's default pool, which the host application or torch
// may use, is left as it is.  The pool lives until the process exits.
cudaMemPool_t library_pool(int dev) {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    std::lock_guard<std::mutex> lock(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props;
    std::memset(&props, 0, sizeof(props));
    props.allocType = cudaMemAllocationTypePinned;
    props.handleTypes = cudaMemHandleTypeNone;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if (cudaMemPoolCreate(&pool, &props) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    uint64_t thr = UINT64_MAX;
    if (cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr) != cudaSuccess) cudaGetLastError();
    pools[dev] = pool;
    return pool;
}

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (dev >= 0 && cudaGetDevice(&prev) == cudaSuccess && prev != dev) cudaSetDevice(dev);
        else prev = -1;
    }
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

// All non-null pointers must be of one kind: *device = true for device/managed memory.
int classify(std::initializer_list<const void*> ptrs, bool* device, int* dev_id, const char* fn) {
    int kind = 0;  // 0 unknown, 1 host, 2 device
    *dev_id = -1;
    for (const void* p : ptrs) {
        if (!p) continue;
        cudaPointerAttributes at;
        int k = 1;
        if (cudaPointerGetAttributes(&at, p) == cudaSuccess) {
            if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) {
                k = 2;
                *dev_id = at.device;
            }
        } else {
            cudaGetLastError();
        }
        if (kind == 0) kind = k;
        else if (kind != k)
            return fail(GX_ERR_INVALID_ARGUMENT, "%s: arrays mix host and device memory", fn);
    }
    *device = kind == 2;
    if (!*device) cudaGetDevice(dev_id);
    return GX_OK;
}

bool valid_precision(int p) { return p == kF64 || p == kMixed || p == kF64Exact; }

int check_phys(const gx_physics& ph, const char* fn) {
    if (!std::isfinite(ph.G) || !std::isfinite(ph.softening) || ph.softening < 0.0)
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: G must be finite and softening finite and >= 0", fn);
    return GX_OK;
}

bool eps0_of(int precision, const gx_physics& ph) {
    const double e2 = ph.softening * ph.softening;
    if (precision == kMixed) return (float)e2 < 1e-24f;
    return e2 < 1e-200;
}

// Device scratch obtained from the stream-ordered pool and returned (stream-ordered) at
// scope exit.  Move-only: a copy would free the allocation twice.
struct AsyncBuf {
    void* p = nullptr;
    cudaStream_t st = nullptr;
    AsyncBuf() = default;
    AsyncBuf(const AsyncBuf&) = delete;
    AsyncBuf& operator=(const AsyncBuf&) = delete;
    AsyncBuf(AsyncBuf&& o) noexcept : p(o.p), st(o.st) { o.p = nullptr; }
    AsyncBuf& operator=(AsyncBuf&&) = delete;
    ~AsyncBuf() {
        if (p && cudaFreeAsync(p, st) != cudaSuccess) cudaGetLastError();  // nothing to report to
    }
    int alloc(size_t bytes, cudaStream_t s) {
        st = s;
        cudaError_t e = dev_alloc_async(&p, bytes, s);
        if (e != cudaSuccess) {
            p = nullptr;
            return fail_cuda(e, "cudaMallocAsync (scratch)");
        }
        return GX_OK;
    }
    double* d() const { return (double*)p; }
};

// ======================================================================================
// variant choice
// ======================================================================================
struct Choice {
    int variant = -1;
    int nsplit = 1;
};

// Source chunking: j_chunk a multiple of jt, nsplit = number of chunks actually used.
void split_layout(int64_t n_src, int jt, int want, int64_t* chunk, int* nsplit) {
    if (want < 1) want = 1;
    int64_t c = (n_src + want - 1) / want;
    c = ((c + jt - 1) / jt) * jt;
    if (c < jt) c = jt;
    *chunk = c;
    *nsplit = (int)std::max<int64_t>(1, (n_src + c - 1) / c);
}

// Predicted time of (variant, nsplit) in units of "one SM running one source against one
// target at full rate".  The CTAs are spread evenly over the SMs (L per SM); an SM runs
// them in rounds of `occupancy` concurrent CTAs, and a round with fewer CTAs than needed to
// cover latency (about 12 warps) runs at a proportionally lower rate.
double rounds_cost(int block, int ipt, int jt, int occ, int64_t n_tgt, int64_t n_src, int ns, int sms) {
    const int64_t tile = (int64_t)block * ipt;
    const int64_t T = (n_tgt + tile - 1) / tile;
    int64_t chunk;
    int nse;
    split_layout(n_src, jt, ns, &chunk, &nse);
    const int64_t L = (T * nse + sms - 1) / sms;
    const double W = (double)tile * (double)(chunk + jt);
    const double warps = block / 32.0;
    auto eff = [&](int64_t c) { return std::min(1.0, (double)c * warps / 12.0); };
    const int64_t full = L / occ, rem = L % occ;
    double t = (double)full * (double)occ * W / eff(occ);
    if (rem) t += (double)rem * W / eff(rem);
    // the ordered reduction pass reads nse partials per target
    if (nse > 1) t += 0.05 * (double)nse * (double)n_tgt * 64.0 / sms;
    return t;
}

double split_cost(const ForceVariant& v, int64_t n_tgt, int64_t n_src, int ns, int sms) {
    return rounds_cost(v.block, v.ipt, v.jt, force_occupancy(v), n_tgt, n_src, ns, sms);
}

int best_split(const ForceVariant& v, int64_t n_tgt, int64_t n_src, int sms) {
    if (v.precision == kF64Exact) return 1;
    int best = 1;
    double bc = split_cost(v, n_tgt, n_src, 1, sms);
    for (int ns = 2; ns <= 64; ++ns) {
        int64_t chunk;
        int nse;
        split_layout(n_src, v.jt, ns, &chunk, &nse);
        if (nse != ns) continue;
        const double c = split_cost(v, n_tgt, n_src, ns, sms);
        if (c < bc * 0.995) {
            bc = c;
            best = ns;
        }
    }
    return best;
}

std::mutex g_tune_mu;
std::map<std::tuple<int, int, int, int64_t>, Choice> g_tuned;  // (device, precision, eps0, n)

// Time per interaction of a variant relative to the fastest of its precision, measured on B200
// at N = 2^20 (the wave model cannot see instruction-level differences between variants).
double variant_rate_penalty(const ForceVariant& v) {
    if (v.precision == kMixed) {
        if (v.packed == 2) return v.block * v.ipt >= 1024 ? 1.0 : 1.02;  // targets packed
        if (v.packed == 1) return v.block * v.ipt >= 1024 ? 1.04 : 1.10;  // sources packed
        return 1.25;                                                      // scalar FP32
    }
    if (v.precision == kF64) return v.block * v.ipt >= 512 ? 1.0 : 1.05;
    return 1.0;
}

// Untuned choice: the wave model over all variants of the precision, weighted by each
// variant's measured per-interaction rate.
Choice heuristic_choice(int dev, int precision, bool eps0, int64_t n_tgt, int64_t n_src) {
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        auto it = g_tuned.find(std::make_tuple(dev, precision, (int)eps0, n_src));
        if (it != g_tuned.end() && n_tgt == n_src) return it->second;
    }
    int ids[32];
    const int c = std::min(32, force_variant_ids(precision, eps0 ? 1 : 0, ids, 32));
    int cnt;
    const ForceVariant* all = force_variants(&cnt);
    const int sms = sm_count(dev);
    Choice best;
    double bc = 1e300;
    for (int k = 0; k < c; ++k) {
        const ForceVariant& v = all[ids[k]];
        if (precision == kMixed && !v.packed) continue;  // the scalar form is kept for measurement only
        const int ns = best_split(v, n_tgt, n_src, sms);
        const double cost = split_cost(v, n_tgt, n_src, ns, sms) * variant_rate_penalty(v);
        if (cost < bc) {
            bc = cost;
            best.variant = ids[k];
            best.nsplit = ns;
        }
    }
    return best;
}

// ======================================================================================
// force evaluation on device pointers
// ======================================================================================
struct ForceJob {
    const double *x, *y, *z, *m;
    int64_t n_src;
    const int64_t* tgt_idx;
    int64_t t_begin, n_tgt;
    double *ax, *ay, *az;
    double *vx, *vy, *vz;
    double kick_dt;
};

ForceArgs make_args(const ForceJob& j, const gx_physics& ph, const ForceVariant& v, int nsplit,
                    double* part) {
    ForceArgs a;
    a.x = j.x;
    a.y = j.y;
    a.z = j.z;
    a.m = j.m;
    a.n_src = j.n_src;
    a.tgt_idx = j.tgt_idx;
    a.t_begin = j.t_begin;
    a.n_tgt = j.n_tgt;
    int ns = nsplit;
    split_layout(j.n_src, v.jt, nsplit, &a.j_chunk, &ns);
    a.nsplit = ns;
    a.ax = j.ax;
    a.ay = j.ay;
    a.az = j.az;
    a.part = part;
    a.tile_count = nullptr;
    a.vx = j.vx;
    a.vy = j.vy;
    a.vz = j.vz;
    a.kick_dt = j.kick_dt;
    a.G = ph.G;
    a.eps2 = ph.softening * ph.softening;
    a.eps2f = (float)a.eps2;
    return a;
}

// Scratch of a split force evaluation: the tile tickets of the fused reduction first (zeroed
// when the scratch is allocated and left zeroed by every launch), then the
// nsplit * 3 * n_tgt partial sums.  The ticket area depends only on max(n_src, n_tgt) and
// is sized for the smallest tile of any variant (64 targets), so a session's later
// launches -- another variant, another split, fewer targets -- find the same zeroed
// tickets and never write partial sums over them.
size_t ticket_bytes(int64_t n) { return (((size_t)(n / 64 + 1) * sizeof(unsigned)) + 255) / 256 * 256; }

size_t part_bytes(const ForceVariant& v, int64_t n_src, int64_t n_tgt, int nsplit) {
    int64_t chunk;
    int ns;
    split_layout(n_src, v.jt, nsplit, &chunk, &ns);
    return ns > 1 ? ticket_bytes(std::max(n_src, n_tgt)) + (size_t)ns * 3 * (size_t)n_tgt * sizeof(double) : 0;
}

// Runs one force evaluation with scratch from `part` (whose tickets are zero), or from a
// stream-ordered allocation whose tickets are cleared here.  Split evaluations reduce in
// the kernel (fused, tile tickets).
int run_force(const ForceJob& j, const gx_physics& ph, int precision, Choice ch, int dev,
              cudaStream_t st, double* part, size_t part_cap) {
    int cnt;
    const ForceVariant* all = force_variants(&cnt);
    const bool eps0 = eps0_of(precision, ph);
    if (ch.variant < 0) ch = heuristic_choice(dev, precision, eps0, j.n_tgt, j.n_src);
    const ForceVariant& v = all[ch.variant];
    const size_t need = part_bytes(v, j.n_src, j.n_tgt, ch.nsplit);
    const size_t tb = ticket_bytes(std::max(j.n_src, j.n_tgt));
    AsyncBuf tmp;
    if (need > part_cap) {
        GX_TRY(tmp.alloc(need, st));
        part = tmp.d();
        GX_CUDA(cudaMemsetAsync(part, 0, tb, st));
    }
    ForceArgs a = make_args(j, ph, v, ch.nsplit, part);
    if (a.nsplit > 1) {
        if (force_tiles(v, j.n_tgt) * (int64_t)sizeof(unsigned) > (int64_t)tb)
            return fail(GX_ERR_UNSUPPORTED, "force variant tile smaller than 64 targets");
        a.tile_count = (unsigned*)part;
        a.part = (double*)((char*)part + tb);
    }
    (void)cudaGetLastError();  // drop a stale non-sticky error of unrelated earlier work; sticky ones resurface below
    GX_CUDA(force_launch(v, a, st));
    return GX_OK;
}

// ======================================================================================
// host staging helpers
// ======================================================================================
struct HostStage {
    cudaStream_t st;
    std::deque<AsyncBuf> bufs;  // stable addresses; released in reverse order at scope exit
    explicit HostStage(cudaStream_t s) : st(s) {}
    // Device copy of a host array (nullptr stays nullptr).
    int in(const double* h, int64_t n, double** d) {
        if (!h) {
            *d = nullptr;
            return GX_OK;
        }
        bufs.emplace_back();
        GX_TRY(bufs.back().alloc((size_t)std::max<int64_t>(n, 1) * sizeof(double), st));
        *d = bufs.back().d();
        if (n > 0) GX_CUDA(cudaMemcpyAsync(*d, h, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, st));
        return GX_OK;
    }
    int out(double** d, int64_t n) {
        bufs.emplace_back();
        GX_TRY(bufs.back().alloc((size_t)std::max<int64_t>(n, 1) * sizeof(double), st));
        *d = bufs.back().d();
        return GX_OK;
    }
    template <typename T>
    int in_any(const T* h, int64_t n, T** d) {
        if (!h) {
            *d = nullptr;
            return GX_OK;
        }
        bufs.emplace_back();
        GX_TRY(bufs.back().alloc((size_t)std::max<int64_t>(n, 1) * sizeof(T), st));
        *d = (T*)bufs.back().p;
        if (n > 0) GX_CUDA(cudaMemcpyAsync(*d, h, (size_t)n * sizeof(T), cudaMemcpyHostToDevice, st));
        return GX_OK;
    }
};

int copy_back(double* h, const double* d, int64_t n, cudaStream_t st) {
    if (h && n > 0) GX_CUDA(cudaMemcpyAsync(h, d, (size_t)n * sizeof(double), cudaMemcpyDeviceToHost, st));
    return GX_OK;
}

}  // namespace

// ======================================================================================
// library
// ======================================================================================
extern "C" int gxi_fail(int code, const char* msg) { return fail(code, "%s", msg); }

extern "C" const char* gx_last_error(void) { return g_err.c_str(); }

extern "C" int gx_abi_version(void) { return GX_ABI_VERSION; }

extern "C" int gx_device_available(int* available) {
    if (!available) return fail(GX_ERR_INVALID_ARGUMENT, "gx_device_available: null pointer");
    *available = require_device() == GX_OK ? 1 : 0;
    return GX_OK;
}

extern "C" int gx_debug_fail_allocations(int count) {
    g_fail_allocs.store(count < 0 ? 0 : count);
    return GX_OK;
}

extern "C" int gx_debug_p2p_targets_per_thread(int tpt) {
    if (tpt != 0 && tpt != 2 && tpt != 4)
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_debug_p2p_targets_per_thread: 0, 2 or 4");
    p2p_set_targets_per_thread(tpt);
    return GX_OK;
}

extern "C" int gx_debug_small_targets_per_warp(int tpw) {
    if (tpw != 0 && tpw != 1 && tpw != 2 && tpw != 4)
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_debug_small_targets_per_warp: 0, 1, 2 or 4");
    small_set_targets_per_warp(tpw);
    return GX_OK;
}

extern "C" int gx_debug_small_warps_per_target(int wpt) {
    if (wpt != 0 && wpt != 1 && wpt != 2)
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_debug_small_warps_per_target: 0, 1 or 2");
    small_set_warps_per_target(wpt);
    return GX_OK;
}

extern "C" int gx_debug_fmm_tight_pools(int enable) {
    g_fmm_tight_pools.store(enable ? 1 : 0);
    return GX_OK;
}

extern "C" int gx_debug_stall_barrier(int64_t step) {
    g_stall_step.store(step < 0 ? -1 : step);
    return GX_OK;
}

extern "C" int gx_variant_count(int precision, int* count) {
    if (!count || !valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "gx_variant_count: bad arguments");
    int ids[64];
    *count = force_variant_ids(precision, 0, ids, 64);
    if (precision != kF64Exact) *count += force_variant_ids(precision, 1, ids, 64);
    return GX_OK;
}

extern "C" int gx_variant_describe(int precision, int variant, char* buf, int buflen) {
    int cnt;
    const ForceVariant* all = force_variants(&cnt);
    if (!buf || buflen <= 0 || variant < 0 || variant >= cnt || all[variant].precision != precision)
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_variant_describe: bad arguments");
    const ForceVariant& v = all[variant];
    const char* p = v.precision == kMixed ? "mixed" : v.precision == kF64 ? "f64" : "f64-exact";
    snprintf(buf, (size_t)buflen, "%s block=%d ipt=%d jt=%d%s%s", p, v.block, v.ipt, v.jt,
             v.packed == 1 ? " f32x2" : v.packed == 2 ? " f32x2-targets" : "",
             v.eps0 && v.precision != kF64Exact ? " eps0" : "");
    return GX_OK;
}

// ======================================================================================
// stateless direct sum
// ======================================================================================
static int direct_common(int64_t n, const double* x, const double* y, const double* z, const double* m,
                         int64_t begin, int64_t end, const int64_t* targets, int64_t n_targets,
                         gx_physics phys, int precision, double* ax, double* ay, double* az, void* stream,
                         const char* fn) {
    if (n < 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: n < 0", fn);
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: unknown precision %d", fn, precision);
    GX_TRY(check_phys(phys, fn));
    const int64_t nt = targets ? n_targets : end - begin;
    if (!targets && (begin < 0 || end < begin || end > n))
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: need 0 <= begin <= end <= n", fn);
    if (targets && n_targets < 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: n_targets < 0", fn);
    if (nt > 0 && (!x || !y || !z || !m || !ax || !ay || !az))
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    GX_TRY(require_device());
    if (nt == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, m, ax, ay, az, targets}, &device, &dev, fn));
    DeviceGuard guard(dev);
    cudaStream_t st = (cudaStream_t)stream;
    if (device) {
        ForceJob j{x, y, z, m, n, targets, targets ? 0 : begin, nt, ax, ay, az, nullptr, nullptr, nullptr, 0.0};
        return run_force(j, phys, precision, Choice(), dev, st, nullptr, 0);
    }
    if (targets) {
        for (int64_t k = 0; k < n_targets; ++k)
            if (targets[k] < 0 || targets[k] >= n) return fail(GX_ERR_INVALID_ARGUMENT, "%s: target index out of range", fn);
    }
    HostStage hs(st);
    double *dx, *dy, *dz, *dm, *dax, *day, *daz;
    int64_t* dt = nullptr;
    GX_TRY(hs.in(x, n, &dx));
    GX_TRY(hs.in(y, n, &dy));
    GX_TRY(hs.in(z, n, &dz));
    GX_TRY(hs.in(m, n, &dm));
    GX_TRY(hs.in_any(targets, n_targets, &dt));
    GX_TRY(hs.out(&dax, nt));
    GX_TRY(hs.out(&day, nt));
    GX_TRY(hs.out(&daz, nt));
    ForceJob j{dx, dy, dz, dm, n, dt, targets ? 0 : begin, nt, dax, day, daz, nullptr, nullptr, nullptr, 0.0};
    GX_TRY(run_force(j, phys, precision, Choice(), dev, st, nullptr, 0));
    GX_TRY(copy_back(ax, dax, nt, st));
    GX_TRY(copy_back(ay, day, nt, st));
    GX_TRY(copy_back(az, daz, nt, st));
    GX_CUDA(cudaStreamSynchronize(st));
    return GX_OK;
}

extern "C" int gx_direct_accel(int64_t n, const double* x, const double* y, const double* z, const double* m,
                               gx_physics phys, int precision, double* ax, double* ay, double* az,
                               void* stream) {
    GX_GUARD_BEGIN
    return direct_common(n, x, y, z, m, 0, n, nullptr, 0, phys, precision, ax, ay, az, stream, "gx_direct_accel");
    GX_GUARD_END
}

extern "C" int gx_direct_accel_targets(int64_t n, const double* x, const double* y, const double* z,
                                       const double* m, int64_t begin, int64_t end, const int64_t* targets,
                                       int64_t n_targets, gx_physics phys, int precision, double* ax,
                                       double* ay, double* az, void* stream) {
    GX_GUARD_BEGIN
    return direct_common(n, x, y, z, m, begin, end, targets, n_targets, phys, precision, ax, ay, az, stream,
                         "gx_direct_accel_targets");
    GX_GUARD_END
}

// ======================================================================================
// integration
// ======================================================================================
extern "C" int gx_kick(int64_t n, double* vx, double* vy, double* vz, const double* ax, const double* ay,
                       const double* az, double dt, void* stream) {
    GX_GUARD_BEGIN
    if (n < 0 || (n > 0 && (!vx || !vy || !vz || !ax || !ay || !az)))
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_kick: bad arguments");
    GX_TRY(require_device());
    if (n == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({vx, vy, vz, ax, ay, az}, &device, &dev, "gx_kick"));
    if (!device) return fail(GX_ERR_INVALID_ARGUMENT, "gx_kick: device arrays only");
    DeviceGuard g(dev);
    GX_CUDA(launch_kick(n, vx, vy, vz, ax, ay, az, dt, (cudaStream_t)stream));
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_drift(int64_t n, double* x, double* y, double* z, const double* vx, const double* vy,
                        const double* vz, double dt, void* stream) {
    GX_GUARD_BEGIN
    if (n < 0 || (n > 0 && (!x || !y || !z || !vx || !vy || !vz)))
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_drift: bad arguments");
    GX_TRY(require_device());
    if (n == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, vx, vy, vz}, &device, &dev, "gx_drift"));
    if (!device) return fail(GX_ERR_INVALID_ARGUMENT, "gx_drift: device arrays only");
    DeviceGuard g(dev);
    GX_CUDA(launch_drift(n, x, y, z, vx, vy, vz, dt, (cudaStream_t)stream));
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_kick_drift(int64_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                             const double* ax, const double* ay, const double* az, double kick_dt,
                             double drift_dt, void* stream) {
    GX_GUARD_BEGIN
    if (n < 0 || (n > 0 && (!x || !y || !z || !vx || !vy || !vz || !ax || !ay || !az)))
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_kick_drift: bad arguments");
    GX_TRY(require_device());
    if (n == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, vx, vy, vz, ax, ay, az}, &device, &dev, "gx_kick_drift"));
    if (!device) return fail(GX_ERR_INVALID_ARGUMENT, "gx_kick_drift: device arrays only");
    DeviceGuard g(dev);
    GX_CUDA(launch_kick_drift(n, x, y, z, vx, vy, vz, ax, ay, az, kick_dt, drift_dt, (cudaStream_t)stream));
    return GX_OK;
    GX_GUARD_END
}

// One KDK step on device arrays: kick(dt/2) + drift(dt), force with the closing kick fused.
static int kdk_device(int64_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz, double* ax,
                      double* ay, double* az, const double* m, double dt, const gx_physics& phys, int precision,
                      Choice ch, int dev, cudaStream_t st, double* part, size_t part_cap) {
    const double half = 0.5 * dt;
    GX_CUDA(launch_kick_drift(n, x, y, z, vx, vy, vz, ax, ay, az, half, dt, st));
    ForceJob j{x, y, z, m, n, nullptr, 0, n, ax, ay, az, vx, vy, vz, half};
    return run_force(j, phys, precision, ch, dev, st, part, part_cap);
}

extern "C" int gx_leapfrog_step(int64_t n, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                                double* ax, double* ay, double* az, const double* m, double dt, gx_physics phys,
                                int precision, void* stream) {
    GX_GUARD_BEGIN
    const char* fn = "gx_leapfrog_step";
    if (n < 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: n < 0", fn);
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: unknown precision", fn);
    if (!std::isfinite(dt)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: dt must be finite", fn);
    GX_TRY(check_phys(phys, fn));
    if (n > 0 && (!x || !y || !z || !vx || !vy || !vz || !ax || !ay || !az || !m))
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    GX_TRY(require_device());
    if (n == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, vx, vy, vz, ax, ay, az, m}, &device, &dev, fn));
    DeviceGuard g(dev);
    cudaStream_t st = (cudaStream_t)stream;
    if (device) return kdk_device(n, x, y, z, vx, vy, vz, ax, ay, az, m, dt, phys, precision, Choice(), dev, st, nullptr, 0);
    HostStage hs(st);
    double* d[10];
    const double* h[10] = {x, y, z, vx, vy, vz, ax, ay, az, m};
    for (int k = 0; k < 10; ++k) GX_TRY(hs.in(h[k], n, &d[k]));
    GX_TRY(kdk_device(n, d[0], d[1], d[2], d[3], d[4], d[5], d[6], d[7], d[8], d[9], dt, phys, precision, Choice(),
                      dev, st, nullptr, 0));
    double* o[9] = {x, y, z, vx, vy, vz, ax, ay, az};
    for (int k = 0; k < 9; ++k) GX_TRY(copy_back(o[k], d[k], n, st));
    GX_CUDA(cudaStreamSynchronize(st));
    return GX_OK;
    GX_GUARD_END
}

static void fill_diag(const double* v, gx_diagnostics* out) {
    out->total_mass = v[0];
    out->kinetic_energy = v[1];
    out->potential_energy = v[2];
    out->total_energy = v[3];
    for (int c = 0; c < 3; ++c) {
        out->momentum[c] = v[4 + c];
        out->center_of_mass[c] = v[7 + c];
        out->angular_momentum[c] = v[10 + c];
    }
}

extern "C" int gx_diagnostics_compute(int64_t n, const double* x, const double* y, const double* z,
                                      const double* vx, const double* vy, const double* vz, const double* m,
                                      gx_physics phys, gx_diagnostics* out, void* stream) {
    GX_GUARD_BEGIN
    const char* fn = "gx_diagnostics_compute";
    if (n < 0 || !out) return fail(GX_ERR_INVALID_ARGUMENT, "%s: bad arguments", fn);
    GX_TRY(check_phys(phys, fn));
    if (n > 0 && (!x || !y || !z || !vx || !vy || !vz || !m)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    GX_TRY(require_device());
    std::memset(out, 0, sizeof(*out));
    if (n == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, vx, vy, vz, m}, &device, &dev, fn));
    DeviceGuard g(dev);
    cudaStream_t st = (cudaStream_t)stream;
    HostStage hs(st);
    const double* d[7] = {x, y, z, vx, vy, vz, m};
    if (!device) {
        for (int k = 0; k < 7; ++k) {
            double* p;
            GX_TRY(hs.in(d[k], n, &p));
            d[k] = p;
        }
    }
    AsyncBuf scratch;
    GX_TRY(scratch.alloc(diagnostics_scratch_bytes(n) + 16 * sizeof(double), st));
    double* res = scratch.d();
    double* work = res + 16;
    GX_CUDA(launch_diagnostics(n, d[0], d[1], d[2], d[3], d[4], d[5], d[6], phys.G,
                               phys.softening * phys.softening, work, res, st));
    double h[13];
    GX_CUDA(cudaMemcpyAsync(h, res, sizeof(h), cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaStreamSynchronize(st));
    fill_diag(h, out);
    return GX_OK;
    GX_GUARD_END
}

// ======================================================================================
// resident session
// ======================================================================================
namespace {
struct FmmWork;
void fmm_work_release(FmmWork* w);
}  // namespace

struct gx_session {
    int device = 0;
    int64_t n = 0;
    gx_physics phys{1.0, 0.02};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double* buf = nullptr;  // 10 * n doubles
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *m;
    double* part = nullptr;
    size_t part_cap = 0;
    double* diag = nullptr;  // device: 16 result slots + diagnostics scratch
    size_t diag_cap = 0;
    double* host_diag = nullptr;  // pinned, 16 doubles
    Choice cfg[3];
    std::map<std::tuple<int64_t, uint64_t, int, int, int>, cudaGraphExec_t> graphs;
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    double timed_ms = 0.0;
    int64_t timed_launches = 0;
    int64_t t_begin = 0;        // owned targets [t_begin, t_begin + t_count): kicked, drifted and
    int64_t t_count = 0;        // given forces by the session (all bodies unless set_targets)
    bool persistent = true;     // small systems step in one cooperative launch (small.cu)
    void* small = nullptr;      // its scratch: barrier words, status, two position buffers
    bool small_pending = false; // a launch ran since the status word was last read
    // FMM force (gx_session_set_fmm): the options, the capacity-mode workspace (sized by a
    // first evaluation, regrown on overflow), a copy of the state a chunk of steps starts
    // from, and pinned words for the chunk's overflow flag
    bool fmm_on = false;
    bool fmm_host_only = false;  // the tree needs the host builder: evaluations read sizes back
    gx_fmm_options fmm_opt{0.6, 16, 32, 4};
    FmmWork* fmm = nullptr;
    double* backup = nullptr;
    int* host_flag = nullptr;

    void clear_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }
};

namespace {

int session_choice(gx_session* s, int precision, Choice* out) {
    if (s->cfg[precision].variant < 0) {
        s->cfg[precision] = heuristic_choice(s->device, precision, eps0_of(precision, s->phys), s->t_count, s->n);
    }
    *out = s->cfg[precision];
    return GX_OK;
}

int session_ensure_part(gx_session* s, const Choice& ch) {
    int cnt;
    const ForceVariant* all = force_variants(&cnt);
    const size_t need = part_bytes(all[ch.variant], s->n, s->n, ch.nsplit);
    if (need <= s->part_cap) return GX_OK;
    if (s->part) {
        cudaStreamSynchronize(s->stream);
        cudaFree(s->part);
        s->part = nullptr;
        s->part_cap = 0;
    }
    void* p;
    cudaError_t e = dev_alloc(&p, need);
    if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc (session j-split scratch)");
    s->part = (double*)p;
    s->part_cap = need;
    GX_CUDA(cudaMemsetAsync(p, 0, ticket_bytes(s->n), s->stream));  // tile tickets of the fused reduction
    return GX_OK;
}

int flush_events(gx_session* s) {
    if (s->events.empty()) return GX_OK;
    GX_CUDA(cudaStreamSynchronize(s->stream));
    for (auto& ev : s->events) {
        float ms = 0.f;
        GX_CUDA(cudaEventElapsedTime(&ms, ev.first, ev.second));
        s->timed_ms += ms;
        s->timed_launches += 1;
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    s->events.clear();
    return GX_OK;
}

// Force evaluation of the session (closing kick when kick_dt != 0), timed on request.
int session_fmm_force(gx_session* s, int precision, double kick_dt);
int session_fmm_compute(gx_session* s, int precision);
int session_fmm_steps(gx_session* s, int64_t n_steps, double dt, int precision);

int session_force(gx_session* s, int precision, double kick_dt) {
    if (s->fmm_on) return session_fmm_force(s, precision, kick_dt);
    Choice ch;
    GX_TRY(session_choice(s, precision, &ch));
    GX_TRY(session_ensure_part(s, ch));
    ForceJob j{s->x, s->y, s->z, s->m, s->n, nullptr, s->t_begin, s->t_count, s->ax + s->t_begin,
               s->ay + s->t_begin, s->az + s->t_begin,
               kick_dt != 0.0 ? s->vx : nullptr, kick_dt != 0.0 ? s->vy : nullptr,
               kick_dt != 0.0 ? s->vz : nullptr, kick_dt};
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (s->timing) {
        GX_CUDA(cudaEventCreate(&e0));
        GX_CUDA(cudaEventCreate(&e1));
        GX_CUDA(cudaEventRecord(e0, s->stream));
    }
    const int r = run_force(j, s->phys, precision, ch, s->device, s->stream, s->part, s->part_cap);
    if (s->timing) {
        GX_CUDA(cudaEventRecord(e1, s->stream));
        s->events.emplace_back(e0, e1);
    }
    return r;
}

// Opening half of a step for the owned bodies: kick(kick_dt) then drift(drift_dt).
int session_kick_drift(gx_session* s, double kick_dt, double drift_dt) {
    const int64_t b = s->t_begin;
    GX_CUDA(launch_kick_drift(s->t_count, s->x + b, s->y + b, s->z + b, s->vx + b, s->vy + b, s->vz + b, s->ax + b,
                              s->ay + b, s->az + b, kick_dt, drift_dt, s->stream));
    return GX_OK;
}

int session_enqueue_steps(gx_session* s, int64_t k, double dt, int precision) {
    const double half = 0.5 * dt;
    for (int64_t i = 0; i < k; ++i) {
        GX_TRY(session_kick_drift(s, half, dt));
        GX_TRY(session_force(s, precision, half));
    }
    return GX_OK;
}

int session_graph(gx_session* s, int64_t k, double dt, int precision, cudaGraphExec_t* out) {
    Choice ch;
    if (s->fmm_on) {
        ch.variant = -2;  // the FMM force; graphs are dropped when its workspace changes
        ch.nsplit = 0;
    } else {
        GX_TRY(session_choice(s, precision, &ch));
        GX_TRY(session_ensure_part(s, ch));
    }
    uint64_t dtb;
    std::memcpy(&dtb, &dt, sizeof(dtb));
    const auto key = std::make_tuple(k, dtb, precision, ch.variant, ch.nsplit);
    auto it = s->graphs.find(key);
    if (it != s->graphs.end()) {
        *out = it->second;
        return GX_OK;
    }
    GX_CUDA(cudaStreamBeginCapture(s->stream, cudaStreamCaptureModeThreadLocal));
    int r = session_enqueue_steps(s, k, dt, precision);
    cudaGraph_t graph = nullptr;
    cudaError_t e = cudaStreamEndCapture(s->stream, &graph);
    if (r != GX_OK) {
        if (graph) cudaGraphDestroy(graph);
        return r;
    }
    if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture (session steps)");
    cudaGraphExec_t exec = nullptr;
    e = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGraphInstantiate (session steps)");
    if (s->graphs.size() > 32) s->clear_graphs();
    s->graphs[key] = exec;
    *out = exec;
    return GX_OK;
}

int check_session(gx_session* s, const char* fn) {
    if (!s) return fail(GX_ERR_INVALID_ARGUMENT, "%s: null session", fn);
    return GX_OK;
}

// Steps that run as one cooperative launch: small systems in FP64 or the exact form, unless
// the caller turned it off or is timing force launches one by one.
bool session_small_eligible(const gx_session* s, int precision) {
    return s->persistent && !s->timing && !s->fmm_on && s->n <= kSmallMaxBodies && s->t_begin == 0 &&
           s->t_count == s->n && (precision == kF64 || precision == kF64Exact);
}

int session_small_steps(gx_session* s, int64_t k, double dt, int precision) {
    if (!s->small) {
        void* p = nullptr;
        cudaError_t e = dev_alloc(&p, small_scratch_bytes((int)s->n));
        if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc (session small-system scratch)");
        s->small = p;
    }
    SmallArgs a;
    a.n = (int)s->n;
    a.x = s->x; a.y = s->y; a.z = s->z;
    a.vx = s->vx; a.vy = s->vy; a.vz = s->vz;
    a.ax = s->ax; a.ay = s->ay; a.az = s->az;
    a.m = s->m;
    a.G = s->phys.G;
    a.eps2 = s->phys.softening * s->phys.softening;
    a.dt = dt;
    a.steps = k;
    a.timeout_ns = 4000000000ull;
    a.stall_step = g_stall_step.exchange(-1);
    if (a.stall_step >= 0) a.timeout_ns = 200000000ull;
    small_bind_scratch(a, s->small);
    (void)cudaGetLastError();
    const cudaError_t e = small_steps_launch(a, precision, eps0_of(precision, s->phys), s->device, s->stream);
    if (e == cudaErrorNotSupported) return GX_ERR_UNSUPPORTED;
    if (e != cudaSuccess) return fail_cuda(e, "small-system step launch");
    s->small_pending = true;
    return GX_OK;
}

// After the stream has been synchronized: GX_ERR_TIMEOUT when a cooperative step launch gave
// up on a barrier since the last check.
int session_small_status(gx_session* s) {
    if (!s->small_pending) return GX_OK;
    s->small_pending = false;
    int st = 0;
    GX_CUDA(cudaMemcpy(&st, (char*)s->small + 2 * sizeof(unsigned), sizeof(int), cudaMemcpyDeviceToHost));
    if (st != 0)
        return fail(GX_ERR_TIMEOUT, "session step: a grid barrier of the single-launch step loop timed out; "
                                    "the state is that of the last completed gx_session_step call");
    return GX_OK;
}

}  // namespace

extern "C" int gx_session_create(int64_t n, gx_physics phys, int device, gx_session** out) {
    GX_GUARD_BEGIN
    const char* fn = "gx_session_create";
    if (!out) return fail(GX_ERR_INVALID_ARGUMENT, "%s: out is null", fn);
    *out = nullptr;
    if (n < 1) return fail(GX_ERR_INVALID_ARGUMENT, "%s: n must be >= 1", fn);
    GX_TRY(check_phys(phys, fn));
    GX_TRY(require_device());
    int count = 0;
    GX_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(GX_ERR_INVALID_ARGUMENT, "%s: device %d out of range", fn, device);
    DeviceGuard g(device);
    gx_session* s = new gx_session();
    s->device = device;
    s->n = n;
    s->t_count = n;
    s->phys = phys;
    void* p = nullptr;
    cudaError_t e = dev_alloc(&p, (size_t)n * 10 * sizeof(double));
    if (e != cudaSuccess) {
        delete s;
        return fail_cuda(e, "cudaMalloc (session state)");
    }
    s->buf = (double*)p;
    double** arr[10] = {&s->x, &s->y, &s->z, &s->vx, &s->vy, &s->vz, &s->ax, &s->ay, &s->az, &s->m};
    for (int k = 0; k < 10; ++k) *arr[k] = s->buf + (size_t)k * (size_t)n;
    s->diag_cap = diagnostics_scratch_bytes(n) + 16 * sizeof(double);
    e = dev_alloc(&p, s->diag_cap);
    if (e == cudaSuccess) s->diag = (double*)p;
    if (e == cudaSuccess) e = cudaMallocHost((void**)&s->host_diag, 16 * sizeof(double));
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->buf, 0, (size_t)n * 10 * sizeof(double), s->stream);
    if (e != cudaSuccess) {
        const int r = fail_cuda(e, "gx_session_create");
        if (s->diag) cudaFree(s->diag);
        if (s->host_diag) cudaFreeHost(s->host_diag);
        cudaFree(s->buf);
        delete s;
        return r;
    }
    s->own_stream = true;
    *out = s;
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_session_destroy(gx_session* s) {
    GX_GUARD_BEGIN
    if (!s) return GX_OK;
    DeviceGuard g(s->device);
    cudaStreamSynchronize(s->stream);
    for (auto& ev : s->events) {
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    s->clear_graphs();
    fmm_work_release(s->fmm);
    if (s->backup) cudaFree(s->backup);
    if (s->host_flag) cudaFreeHost(s->host_flag);
    if (s->small) cudaFree(s->small);
    if (s->part) cudaFree(s->part);
    if (s->diag) cudaFree(s->diag);
    if (s->host_diag) cudaFreeHost(s->host_diag);
    if (s->buf) cudaFree(s->buf);
    if (s->own_stream) cudaStreamDestroy(s->stream);
    delete s;
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_session_set_stream(gx_session* s, void* stream) {
    GX_TRY(check_session(s, "gx_session_set_stream"));
    DeviceGuard g(s->device);
    cudaStreamSynchronize(s->stream);
    if (s->own_stream) cudaStreamDestroy(s->stream);
    s->own_stream = false;
    s->stream = (cudaStream_t)stream;
    return GX_OK;
}

extern "C" int gx_session_get_stream(gx_session* s, void** stream) {
    GX_TRY(check_session(s, "gx_session_get_stream"));
    if (!stream) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_get_stream: null");
    *stream = (void*)s->stream;
    return GX_OK;
}

extern "C" int gx_session_set_state(gx_session* s, const double* x, const double* y, const double* z,
                                    const double* vx, const double* vy, const double* vz, const double* m,
                                    const double* ax, const double* ay, const double* az) {
    GX_GUARD_BEGIN
    const char* fn = "gx_session_set_state";
    GX_TRY(check_session(s, fn));
    if (!x || !y || !z || !vx || !vy || !vz || !m) return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    if ((ax || ay || az) && !(ax && ay && az)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: give all of ax, ay, az or none", fn);
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, vx, vy, vz, m, ax, ay, az}, &device, &dev, fn));
    DeviceGuard g(s->device);
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const double* src[10] = {x, y, z, vx, vy, vz, ax, ay, az, m};
    double* dst[10] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az, s->m};
    const size_t bytes = (size_t)s->n * sizeof(double);
    for (int k = 0; k < 10; ++k) {
        if (src[k]) GX_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, kind, s->stream));
        else GX_CUDA(cudaMemsetAsync(dst[k], 0, bytes, s->stream));
    }
    if (!device) GX_CUDA(cudaStreamSynchronize(s->stream));
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_session_get_state(gx_session* s, double* x, double* y, double* z, double* vx, double* vy,
                                    double* vz, double* ax, double* ay, double* az) {
    GX_GUARD_BEGIN
    const char* fn = "gx_session_get_state";
    GX_TRY(check_session(s, fn));
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, vx, vy, vz, ax, ay, az}, &device, &dev, fn));
    DeviceGuard g(s->device);
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    double* dst[9] = {x, y, z, vx, vy, vz, ax, ay, az};
    const double* src[9] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az};
    const size_t bytes = (size_t)s->n * sizeof(double);
    for (int k = 0; k < 9; ++k)
        if (dst[k]) GX_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, kind, s->stream));
    GX_CUDA(cudaStreamSynchronize(s->stream));
    return session_small_status(s);
    GX_GUARD_END
}

extern "C" int gx_session_snapshot(gx_session* s, gx_snapshot_writer* w, int step, double time) {
    GX_GUARD_BEGIN
    GX_TRY(check_session(s, "gx_session_snapshot"));
    DeviceGuard g(s->device);
    return gx_snapshot_write(w, step, time, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az, s->m,
                             s->stream);
    GX_GUARD_END
}

extern "C" int gx_session_device_arrays(gx_session* s, double** p) {
    GX_TRY(check_session(s, "gx_session_device_arrays"));
    if (!p) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_device_arrays: null");
    double* a[10] = {s->x, s->y, s->z, s->vx, s->vy, s->vz, s->ax, s->ay, s->az, s->m};
    for (int k = 0; k < 10; ++k) p[k] = a[k];
    return GX_OK;
}

extern "C" int gx_session_compute_accelerations(gx_session* s, int precision) {
    GX_GUARD_BEGIN
    GX_TRY(check_session(s, "gx_session_compute_accelerations"));
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_compute_accelerations: precision");
    DeviceGuard g(s->device);
    if (s->fmm_on) return session_fmm_compute(s, precision);
    return session_force(s, precision, 0.0);
    GX_GUARD_END
}

extern "C" int gx_session_step(gx_session* s, int64_t n_steps, double dt, int precision) {
    GX_GUARD_BEGIN
    const char* fn = "gx_session_step";
    GX_TRY(check_session(s, fn));
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: unknown precision", fn);
    if (n_steps < 0 || !std::isfinite(dt)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: need n_steps >= 0, finite dt", fn);
    if (n_steps == 0) return GX_OK;
    DeviceGuard g(s->device);
    if (s->fmm_on) return session_fmm_steps(s, n_steps, dt, precision);
    if (session_small_eligible(s, precision)) {
        const int r = session_small_steps(s, n_steps, dt, precision);
        if (r != GX_ERR_UNSUPPORTED) return r;
    }
    if (s->timing || s->stream == nullptr) return session_enqueue_steps(s, n_steps, dt, precision);
    const int64_t chunk = std::min<int64_t>(n_steps, 32);
    cudaGraphExec_t ge;
    GX_TRY(session_graph(s, chunk, dt, precision, &ge));
    const int64_t full = n_steps / chunk, rem = n_steps % chunk;
    for (int64_t i = 0; i < full; ++i) GX_CUDA(cudaGraphLaunch(ge, s->stream));
    if (rem) {
        GX_TRY(session_graph(s, rem, dt, precision, &ge));
        GX_CUDA(cudaGraphLaunch(ge, s->stream));
    }
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_session_diagnostics(gx_session* s, gx_diagnostics* out) {
    GX_GUARD_BEGIN
    GX_TRY(check_session(s, "gx_session_diagnostics"));
    if (!out) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_diagnostics: null");
    DeviceGuard g(s->device);
    GX_CUDA(launch_diagnostics(s->n, s->x, s->y, s->z, s->vx, s->vy, s->vz, s->m, s->phys.G,
                               s->phys.softening * s->phys.softening, s->diag + 16, s->diag, s->stream));
    GX_CUDA(cudaMemcpyAsync(s->host_diag, s->diag, 13 * sizeof(double), cudaMemcpyDeviceToHost, s->stream));
    GX_CUDA(cudaStreamSynchronize(s->stream));
    fill_diag(s->host_diag, out);
    return session_small_status(s);
    GX_GUARD_END
}

extern "C" int gx_session_synchronize(gx_session* s) {
    GX_TRY(check_session(s, "gx_session_synchronize"));
    DeviceGuard g(s->device);
    GX_CUDA(cudaStreamSynchronize(s->stream));
    return session_small_status(s);
}

extern "C" int gx_session_set_persistent(gx_session* s, int enable) {
    GX_TRY(check_session(s, "gx_session_set_persistent"));
    s->persistent = enable != 0;
    return GX_OK;
}

extern "C" int gx_session_set_fmm(gx_session* s, const gx_fmm_options* opt) {
    GX_GUARD_BEGIN
    GX_TRY(check_session(s, "gx_session_set_fmm"));
    if (opt && !(opt->theta == opt->theta)) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_set_fmm: theta is NaN");
    DeviceGuard g(s->device);
    GX_CUDA(cudaStreamSynchronize(s->stream));
    fmm_work_release(s->fmm);
    s->fmm = nullptr;
    s->fmm_host_only = false;
    s->fmm_on = opt != nullptr;
    if (opt) s->fmm_opt = *opt;
    s->clear_graphs();
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_session_set_targets(gx_session* s, int64_t begin, int64_t count) {
    GX_TRY(check_session(s, "gx_session_set_targets"));
    if (begin < 0 || count < 0 || begin + count > s->n)
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_set_targets: need 0 <= begin, 0 <= count, begin + count <= n");
    DeviceGuard g(s->device);
    GX_CUDA(cudaStreamSynchronize(s->stream));
    s->t_begin = begin;
    s->t_count = count;
    for (auto& c : s->cfg) c = Choice();
    s->clear_graphs();
    return GX_OK;
}

extern "C" int gx_session_kick_drift(gx_session* s, double kick_dt, double drift_dt) {
    GX_GUARD_BEGIN
    GX_TRY(check_session(s, "gx_session_kick_drift"));
    if (!std::isfinite(kick_dt) || !std::isfinite(drift_dt))
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_kick_drift: time steps must be finite");
    DeviceGuard g(s->device);
    if (s->t_count == 0) return GX_OK;
    return session_kick_drift(s, kick_dt, drift_dt);
    GX_GUARD_END
}

extern "C" int gx_session_force_kick(gx_session* s, double kick_dt, int precision) {
    GX_GUARD_BEGIN
    GX_TRY(check_session(s, "gx_session_force_kick"));
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_force_kick: precision");
    if (!std::isfinite(kick_dt)) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_force_kick: kick_dt must be finite");
    DeviceGuard g(s->device);
    if (s->t_count == 0) return GX_OK;
    return session_force(s, precision, kick_dt);
    GX_GUARD_END
}

extern "C" int gx_session_synchronize_timeout(gx_session* s, double timeout_ms) {
    GX_TRY(check_session(s, "gx_session_synchronize_timeout"));
    DeviceGuard g(s->device);
    cudaEvent_t ev;
    GX_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaError_t e = cudaEventRecord(ev, s->stream);
    if (e != cudaSuccess) {
        cudaEventDestroy(ev);
        return fail_cuda(e, "cudaEventRecord");
    }
    const auto t0 = std::chrono::steady_clock::now();
    for (;;) {
        e = cudaEventQuery(ev);
        if (e != cudaErrorNotReady) break;
        const double el = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        if (el > timeout_ms) {
            cudaEventDestroy(ev);
            return fail(GX_ERR_TIMEOUT, "gx_session_synchronize_timeout: stream still busy after %.1f ms", timeout_ms);
        }
        std::this_thread::sleep_for(std::chrono::microseconds(200));
    }
    cudaEventDestroy(ev);
    if (e != cudaSuccess) return fail_cuda(e, "cudaEventQuery");
    return session_small_status(s);
}

extern "C" int gx_session_enable_timing(gx_session* s, int enable) {
    GX_TRY(check_session(s, "gx_session_enable_timing"));
    DeviceGuard g(s->device);
    GX_TRY(flush_events(s));
    s->timing = enable != 0;
    s->timed_ms = 0.0;
    s->timed_launches = 0;
    return GX_OK;
}

extern "C" int gx_session_force_timing(gx_session* s, double* total_ms, int64_t* launches) {
    GX_TRY(check_session(s, "gx_session_force_timing"));
    DeviceGuard g(s->device);
    GX_TRY(flush_events(s));
    if (total_ms) *total_ms = s->timed_ms;
    if (launches) *launches = s->timed_launches;
    return GX_OK;
}

extern "C" int gx_session_get_config(gx_session* s, int precision, int* variant, int* jsplit) {
    GX_TRY(check_session(s, "gx_session_get_config"));
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_get_config: precision");
    DeviceGuard g(s->device);
    Choice ch;
    GX_TRY(session_choice(s, precision, &ch));
    if (variant) *variant = ch.variant;
    if (jsplit) {
        int cnt;
        const ForceVariant* all = force_variants(&cnt);
        int64_t chunk;
        int ns;
        split_layout(s->n, all[ch.variant].jt, ch.nsplit, &chunk, &ns);
        *jsplit = ns;
    }
    return GX_OK;
}

extern "C" int gx_session_set_config(gx_session* s, int precision, int variant, int jsplit) {
    GX_TRY(check_session(s, "gx_session_set_config"));
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_set_config: precision");
    int cnt;
    const ForceVariant* all = force_variants(&cnt);
    const bool eps0 = eps0_of(precision, s->phys);
    if (variant < 0 || variant >= cnt || all[variant].precision != precision ||
        (precision != kF64Exact && (bool)all[variant].eps0 != eps0))
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_set_config: variant %d does not fit precision %d, softening %g",
                    variant, precision, s->phys.softening);
    if (jsplit < 1 || jsplit > 4096 || (precision == kF64Exact && jsplit != 1))
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_session_set_config: jsplit out of range");
    s->cfg[precision].variant = variant;
    s->cfg[precision].nsplit = jsplit;
    return GX_OK;
}

// ---- autotuner ---------------------------------------------------------------------
namespace {

// Times `reps` force evaluations of targets [0, n_tgt) with a given choice on the
// session's state (results go to the session's acceleration array).
int time_choice(gx_session* s, int precision, Choice ch, int64_t n_tgt, int reps, double* ms_out) {
    GX_TRY(session_ensure_part(s, ch));
    ForceJob j{s->x, s->y, s->z, s->m, s->n, nullptr, s->t_begin, n_tgt, s->ax + s->t_begin, s->ay + s->t_begin,
               s->az + s->t_begin, nullptr, nullptr, nullptr, 0.0};
    GX_TRY(run_force(j, s->phys, precision, ch, s->device, s->stream, s->part, s->part_cap));  // warm-up
    cudaEvent_t e0, e1;
    GX_CUDA(cudaEventCreate(&e0));
    GX_CUDA(cudaEventCreate(&e1));
    double best = 1e300;
    for (int r = 0; r < reps; ++r) {
        GX_CUDA(cudaEventRecord(e0, s->stream));
        GX_TRY(run_force(j, s->phys, precision, ch, s->device, s->stream, s->part, s->part_cap));
        GX_CUDA(cudaEventRecord(e1, s->stream));
        GX_CUDA(cudaEventSynchronize(e1));
        float ms;
        GX_CUDA(cudaEventElapsedTime(&ms, e0, e1));
        best = std::min(best, (double)ms);
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    *ms_out = best;
    return GX_OK;
}

}  // namespace

extern "C" int gx_session_autotune(gx_session* s, int precision, double* best_ms) {
    GX_GUARD_BEGIN
    const char* fn = "gx_session_autotune";
    GX_TRY(check_session(s, fn));
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: precision", fn);
    DeviceGuard g(s->device);
    int cnt;
    const ForceVariant* all = force_variants(&cnt);
    const bool eps0 = eps0_of(precision, s->phys);
    int ids[32];
    const int c = std::min(32, force_variant_ids(precision, eps0 ? 1 : 0, ids, 32));
    const int sms = sm_count(s->device);
    // Save the accelerations: timing runs overwrite them.
    void* save = nullptr;
    GX_CUDA(dev_alloc(&save, (size_t)s->n * 3 * sizeof(double)));
    GX_CUDA(cudaMemcpyAsync(save, s->ax, (size_t)s->n * 3 * sizeof(double), cudaMemcpyDeviceToDevice, s->stream));
    Choice best;
    double bms = 1e300;
    int status = GX_OK;
    const bool large = (double)s->t_count * (double)s->n > 4.0e10;
    // Phase 1: every variant at the split the wave model prefers for it (small systems also try
    // a few fixed splits).  Phase 2 (large systems): other splits for the three best variants.
    std::vector<std::pair<double, Choice>> ranked;
    for (int k = 0; k < c && status == GX_OK; ++k) {
        const ForceVariant& v = all[ids[k]];
        std::vector<int> splits = {best_split(v, s->t_count, s->n, sms)};
        if (!large) {
            for (int ns : {1, 2, 4, 8})
                if (std::find(splits.begin(), splits.end(), ns) == splits.end() && (int64_t)ns * v.jt <= s->n)
                    splits.push_back(ns);
        }
        for (int ns : splits) {
            const Choice ch{ids[k], ns};
            double ms;
            status = time_choice(s, precision, ch, s->t_count, large ? 1 : 3, &ms);
            if (status != GX_OK) break;
            ranked.emplace_back(ms, ch);
        }
    }
    if (status == GX_OK && large && !ranked.empty()) {
        std::sort(ranked.begin(), ranked.end(), [](const auto& a, const auto& b) { return a.first < b.first; });
        const size_t top = std::min<size_t>(3, ranked.size());
        std::vector<std::pair<double, Choice>> extra;
        for (size_t r = 0; r < top && status == GX_OK; ++r) {
            const ForceVariant& v = all[ranked[r].second.variant];
            for (int ns : {1, 2, 4, 8}) {
                if (ns == ranked[r].second.nsplit || (int64_t)ns * v.jt > s->n) continue;
                const Choice ch{ranked[r].second.variant, ns};
                double ms;
                status = time_choice(s, precision, ch, s->t_count, 1, &ms);
                if (status != GX_OK) break;
                extra.emplace_back(ms, ch);
            }
        }
        ranked.insert(ranked.end(), extra.begin(), extra.end());
    }
    for (const auto& r : ranked)
        if (r.first < bms) {
            bms = r.first;
            best = r.second;
        }
    // the caller's accelerations back, whatever the timing runs did to them
    cudaError_t restore = cudaMemcpyAsync(s->ax, save, (size_t)s->n * 3 * sizeof(double), cudaMemcpyDeviceToDevice,
                                          s->stream);
    if (restore == cudaSuccess) restore = cudaStreamSynchronize(s->stream);
    cudaFree(save);
    if (status != GX_OK) return status;
    if (restore != cudaSuccess) return fail_cuda(restore, "cudaMemcpyAsync (autotune: restoring the accelerations)");
    if (best.variant < 0) return fail(GX_ERR_UNSUPPORTED, "%s: no candidate variant", fn);
    s->cfg[precision] = best;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        if (s->t_count == s->n) g_tuned[std::make_tuple(s->device, precision, (int)eps0, s->n)] = best;
    }
    s->clear_graphs();
    if (best_ms) *best_ms = bms;
    return GX_OK;
    GX_GUARD_END
}

// ======================================================================================
// P2P
// ======================================================================================
extern "C" int gx_p2p_leaves(int64_t n, const double* x, const double* y, const double* z, const double* m,
                             int32_t n_leaves, const int32_t* leaf_offsets, const int32_t* leaf_particles,
                             const int32_t* near_offsets, const int32_t* near_leaves, gx_physics phys,
                             int precision, double* ax, double* ay, double* az, void* stream) {
    GX_GUARD_BEGIN
    const char* fn = "gx_p2p_leaves";
    if (n < 0 || n_leaves < 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: negative size", fn);
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: unknown precision", fn);
    GX_TRY(check_phys(phys, fn));
    if (n_leaves > 0 && (!x || !y || !z || !m || !leaf_offsets || !leaf_particles || !near_offsets || !ax || !ay || !az))
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    GX_TRY(require_device());
    if (n_leaves == 0 || n == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, m, leaf_offsets, leaf_particles, near_offsets, near_leaves, ax, ay, az}, &device, &dev, fn));
    DeviceGuard g(dev);
    cudaStream_t st = (cudaStream_t)stream;
    P2PArgs a{};
    a.n_leaves = n_leaves;
    a.t_begin = 0;
    a.t_end = n;
    a.G = phys.G;
    a.eps2 = phys.softening * phys.softening;
    a.eps2f = (float)a.eps2;
    AsyncBuf scratch;
    GX_TRY(scratch.alloc(p2p_scratch_bytes(n, n_leaves), st));
    if (device) {
        a.x = x; a.y = y; a.z = z; a.m = m;
        a.leaf_off = leaf_offsets; a.leaf_part = leaf_particles; a.near_off = near_offsets; a.near_leaf = near_leaves;
        a.ax = ax; a.ay = ay; a.az = az;
        GX_CUDA(launch_p2p(a, n, precision, scratch.p, sm_count(dev), st));
        return GX_OK;
    }
    // Host arrays: validate the CSR (the kernel trusts it), then stage.
    const int32_t n_lp = leaf_offsets[n_leaves];
    const int32_t n_nl = near_offsets[n_leaves];
    if (leaf_offsets[0] != 0 || near_offsets[0] != 0 || n_lp < 0 || n_nl < 0)
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: CSR offsets must start at 0", fn);
    for (int32_t l = 0; l < n_leaves; ++l)
        if (leaf_offsets[l + 1] < leaf_offsets[l] || near_offsets[l + 1] < near_offsets[l])
            return fail(GX_ERR_INVALID_ARGUMENT, "%s: CSR offsets must be non-decreasing", fn);
    {
        std::vector<unsigned char> seen((size_t)n, 0);
        for (int32_t k = 0; k < n_lp; ++k) {
            const int32_t i = leaf_particles[k];
            if (i < 0 || i >= n) return fail(GX_ERR_INVALID_ARGUMENT, "%s: body index out of range", fn);
            if (seen[(size_t)i]++) return fail(GX_ERR_INVALID_ARGUMENT, "%s: body %d listed in two leaf slots", fn, (int)i);
        }
    }
    for (int32_t k = 0; k < n_nl; ++k)
        if (near_leaves[k] < 0 || near_leaves[k] >= n_leaves) return fail(GX_ERR_INVALID_ARGUMENT, "%s: leaf id out of range", fn);
    HostStage hs(st);
    double *dx, *dy, *dz, *dm, *dax, *day, *daz;
    int32_t *dlo, *dlp, *dno, *dnl;
    GX_TRY(hs.in(x, n, &dx));
    GX_TRY(hs.in(y, n, &dy));
    GX_TRY(hs.in(z, n, &dz));
    GX_TRY(hs.in(m, n, &dm));
    GX_TRY(hs.in(ax, n, &dax));
    GX_TRY(hs.in(ay, n, &day));
    GX_TRY(hs.in(az, n, &daz));
    GX_TRY(hs.in_any(leaf_offsets, (int64_t)n_leaves + 1, &dlo));
    GX_TRY(hs.in_any(leaf_particles, (int64_t)n_lp, &dlp));
    GX_TRY(hs.in_any(near_offsets, (int64_t)n_leaves + 1, &dno));
    GX_TRY(hs.in_any(near_leaves ? near_leaves : leaf_offsets, (int64_t)std::max<int32_t>(n_nl, 1), &dnl));
    a.x = dx; a.y = dy; a.z = dz; a.m = dm;
    a.leaf_off = dlo; a.leaf_part = dlp; a.near_off = dno; a.near_leaf = dnl;
    a.ax = dax; a.ay = day; a.az = daz;
    GX_CUDA(launch_p2p(a, n, precision, scratch.p, sm_count(dev), st));
    GX_TRY(copy_back(ax, dax, n, st));
    GX_TRY(copy_back(ay, day, n, st));
    GX_TRY(copy_back(az, daz, n, st));
    GX_CUDA(cudaStreamSynchronize(st));
    return GX_OK;
    GX_GUARD_END
}

// ======================================================================================
// FMM: the reference octree, its moments, far field and near field
// ======================================================================================
namespace {

// Optional phase timing of one FMM evaluation: events on the caller's stream at the phase
// boundaries (tree, moments, lists, far field, near field).
struct FmmTimer {
    cudaEvent_t ev[6] = {};
    double host_tree_ms = -1.0;  // the host builder's own time, when it ran
    int create() {
        for (auto& e : ev) GX_CUDA(cudaEventCreate(&e));
        return GX_OK;
    }
    ~FmmTimer() {
        for (auto& e : ev)
            if (e) cudaEventDestroy(e);
    }
};

int mark(FmmTimer* tm, int k, cudaStream_t st) {
    if (tm) GX_CUDA(cudaEventRecord(tm->ev[k], st));
    return GX_OK;
}

// Device arrays and sizes of one FMM evaluation's tree, built on the device or the host.
struct FmmPlan {
    HostStage hs;
    explicit FmmPlan(cudaStream_t s) : hs(s) {}
    bool on_device = false;
    int32_t n_nodes = 0, n_leaves = 0;
    std::vector<int32_t> level_off;
    int64_t n_far = 0, n_near = 0, n_slots = 0;
    int64_t far_pairs = 0, near_pairs = 0;
    FmmArgs fa{};
    const int32_t* near_off = nullptr;
    const int32_t* near_leaf = nullptr;
};

template <typename T>
int dev_array(HostStage& hs, int64_t count, T** p) {
    hs.bufs.emplace_back();
    GX_TRY(hs.bufs.back().alloc((size_t)std::max<int64_t>(count, 1) * sizeof(T), hs.st));
    *p = (T*)hs.bufs.back().p;
    return GX_OK;
}

template <typename T>
int dev_copy(HostStage& hs, const std::vector<T>& v, const T** p) {
    T* d;
    GX_TRY(hs.in_any(v.data(), (int64_t)v.size(), &d));
    *p = d;
    return GX_OK;
}

void fmm_common_args(FmmArgs& fa, const double* dx, const double* dy, const double* dz, const double* dm,
                     gx_physics phys, gx_fmm_options opt, int64_t begin, int64_t end) {
    fa.x = dx;
    fa.y = dy;
    fa.z = dz;
    fa.m = dm;
    fa.t_begin = begin;
    fa.t_end = end;
    fa.G = phys.G;
    fa.eps2 = phys.softening * phys.softening;
    fa.order = fmm_effective_order(std::min(4, std::max(0, opt.expansion_order)));
}

// Host builder: the octree and lists on the host, moments on the device.
int fmm_plan_host(FmmPlan& P, int64_t n, const double* hx, const double* hy, const double* hz, const double* hm,
                  const double* dx, const double* dy, const double* dz, const double* dm, gx_physics phys,
                  gx_fmm_options opt, int64_t begin, int64_t end, FmmTimer* tm) {
    HostStage& hs = P.hs;
    FmmTree T;
    const auto h0 = std::chrono::steady_clock::now();
    GX_TRY(build_fmm_tree(n, hx, hy, hz, hm, phys.softening, opt.theta, opt.leaf_capacity, opt.max_depth, true, &T));
    if (tm) tm->host_tree_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - h0).count();
    GX_TRY(mark(tm, 0, hs.st));
    P.near_pairs = T.n_pairs;
    for (int32_t l = 0; l < T.n_leaves(); ++l)
        P.far_pairs += (int64_t)(T.far_off[l + 1] - T.far_off[l]) * (T.leaf_off[l + 1] - T.leaf_off[l]);
    FmmArgs& fa = P.fa;
    fmm_common_args(fa, dx, dy, dz, dm, phys, opt, begin, end);
    P.n_nodes = fa.n_nodes = T.n_nodes();
    P.n_leaves = fa.n_leaves = T.n_leaves();
    P.level_off = T.level_off;
    P.n_far = T.n_far;
    P.n_near = (int64_t)T.near_leaf.size();
    GX_TRY(dev_copy(hs, T.node_beg, &fa.node_beg));
    GX_TRY(dev_copy(hs, T.node_end, &fa.node_end));
    GX_TRY(dev_copy(hs, T.node_child, &fa.node_child));
    GX_TRY(dev_copy(hs, T.node_cx, &fa.node_cx));
    GX_TRY(dev_copy(hs, T.node_cy, &fa.node_cy));
    GX_TRY(dev_copy(hs, T.node_cz, &fa.node_cz));
    GX_TRY(dev_copy(hs, T.perm, &fa.perm));
    GX_TRY(dev_copy(hs, T.leaf_off, &fa.leaf_off));
    GX_TRY(dev_copy(hs, T.leaf_part, &fa.leaf_part));
    GX_TRY(dev_copy(hs, T.far_node, &fa.far_node));
    GX_TRY(dev_copy(hs, T.near_off, &P.near_off));
    GX_TRY(dev_copy(hs, T.near_leaf, &P.near_leaf));
    GX_TRY(mark(tm, 1, hs.st));
    GX_TRY(dev_array(hs, (int64_t)P.n_nodes * kFmmRec, &fa.rec));
    GX_CUDA(launch_fmm_moments(fa, P.level_off.data(), T.n_levels(), hs.st));
    GX_TRY(mark(tm, 2, hs.st));
    // far-field work items for the leaves that hold a target in [begin, end)
    std::vector<M2PItem> items;
    int64_t slots = 0;
    for (int32_t l = 0; l < P.n_leaves; ++l) {
        const int32_t fb = T.far_off[l], fe = T.far_off[l + 1];
        if (fe == fb) continue;
        bool any = false;
        for (int32_t k = T.leaf_off[l]; k < T.leaf_off[l + 1] && !any; ++k)
            any = T.leaf_part[k] >= begin && T.leaf_part[k] < end;
        if (!any) continue;
        const int32_t nch = (fe - fb + kM2PChunk - 1) / kM2PChunk;
        const int64_t base = nch > 1 ? slots : 0;
        if (nch > 1) slots += (int64_t)nch * (T.leaf_off[l + 1] - T.leaf_off[l]);
        for (int32_t c = 0; c < nch; ++c) {
            M2PItem it;
            it.leaf = l;
            it.fb = fb + c * kM2PChunk;
            it.fe = std::min(fe, it.fb + kM2PChunk);
            it.chunk = c;
            it.nchunks = nch;
            it.pad = 0;
            it.scratch = base;
            items.push_back(it);
        }
    }
    if (items.size() > (size_t)std::numeric_limits<int32_t>::max())
        return fail(GX_ERR_UNSUPPORTED, "FMM: too many far-field work items");
    // largest items first (targets x nodes), as the device builder orders them
    std::stable_sort(items.begin(), items.end(), [&](const M2PItem& u, const M2PItem& v) {
        const int64_t cu = (int64_t)(T.leaf_off[u.leaf + 1] - T.leaf_off[u.leaf]) * (u.fe - u.fb);
        const int64_t cv = (int64_t)(T.leaf_off[v.leaf + 1] - T.leaf_off[v.leaf]) * (v.fe - v.fb);
        return cu > cv;
    });
    fa.n_items = (int32_t)items.size();
    P.n_slots = slots;
    if (!items.empty()) GX_TRY(dev_copy(hs, items, &fa.items));
    GX_TRY(mark(tm, 3, hs.st));
    return GX_OK;
}

// Device builder; *deep is set (and nothing else is valid) when the tree needs a split
// below the key depth, which the host builder handles.
int fmm_plan_device(FmmPlan& P, int64_t n, const double* dx, const double* dy, const double* dz, const double* dm,
                    gx_physics phys, gx_fmm_options opt, int64_t begin, int64_t end, bool* deep, FmmTimer* tm) {
    HostStage& hs = P.hs;
    cudaStream_t st = hs.st;
    GX_TRY(mark(tm, 0, st));
    *deep = false;
    P.on_device = true;
    const int64_t cap = std::max<int64_t>(1, opt.leaf_capacity);
    TreeBuildArgs t{};
    t.n = (int32_t)n;
    t.x = dx;
    t.y = dy;
    t.z = dz;
    t.softening = phys.softening;
    t.cap = cap;
    t.max_depth = std::max(1, opt.max_depth);
    GX_TRY(dev_array(hs, 6 * kBboxBlocks, &t.part));
    GX_TRY(dev_array(hs, 4, &t.root));
    GX_TRY(dev_array(hs, n, &t.keys));
    GX_TRY(dev_array(hs, n, &t.keys_alt));
    GX_TRY(dev_array(hs, n, &t.idx));
    GX_TRY(dev_array(hs, n, &t.perm));
    GX_TRY(dev_array(hs, kKeyLevels + 3, &t.level_off));
    GX_TRY(dev_array(hs, 3, &t.hdr));
    const size_t sort_bytes = tree_build_temp_bytes(t.n, cap);
    void* sort_temp;
    GX_TRY(dev_array(hs, (int64_t)sort_bytes, (char**)&sort_temp));
    // node slots: 1 + 8 per split node; at most n / (cap + 1) nodes split per level
    const int64_t per_level = n / (cap + 1) + 1;
    int32_t hdr[3] = {0, 0, 0};
    std::vector<int32_t> loff(kKeyLevels + 3);
    for (int attempt = 0; attempt < 2; ++attempt) {
        const int64_t splits = attempt == 0 ? std::min<int64_t>(3 * per_level + 64, kKeyLevels * per_level)
                                            : kKeyLevels * per_level;
        const int64_t capacity = 1 + 8 * splits;
        if (capacity > std::numeric_limits<int32_t>::max()) return fail(GX_ERR_UNSUPPORTED, "FMM: tree too large");
        t.capacity = (int32_t)capacity;
        GX_TRY(dev_array(hs, capacity, &t.beg));
        GX_TRY(dev_array(hs, capacity, &t.end));
        GX_TRY(dev_array(hs, capacity, &t.child));
        GX_TRY(dev_array(hs, capacity, &t.cx));
        GX_TRY(dev_array(hs, capacity, &t.cy));
        GX_TRY(dev_array(hs, capacity, &t.cz));
        GX_TRY(dev_array(hs, capacity, &t.hw));
        GX_CUDA(launch_tree_build(t, sort_temp, sort_bytes, st));
        GX_CUDA(cudaMemcpyAsync(hdr, t.hdr, sizeof(hdr), cudaMemcpyDeviceToHost, st));
        GX_CUDA(cudaMemcpyAsync(loff.data(), t.level_off, loff.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
        GX_CUDA(cudaStreamSynchronize(st));
        if (hdr[2] & 1) {
            *deep = true;
            return GX_OK;
        }
        if (!(hdr[2] & 2)) break;
        if (attempt == 1) return fail(GX_ERR_UNSUPPORTED, "FMM: node slots exhausted");
    }
    GX_CUDA(launch_tree_leaf_order(t, hdr[0], sort_temp, sort_bytes, st));
    GX_TRY(mark(tm, 1, st));
    FmmArgs& fa = P.fa;
    fmm_common_args(fa, dx, dy, dz, dm, phys, opt, begin, end);
    P.n_nodes = fa.n_nodes = hdr[0];
    P.level_off.assign(loff.begin(), loff.begin() + hdr[1] + 1);
    fa.node_beg = t.beg;
    fa.node_end = t.end;
    fa.node_child = t.child;
    fa.node_cx = t.cx;
    fa.node_cy = t.cy;
    fa.node_cz = t.cz;
    fa.perm = t.perm;
    GX_TRY(dev_array(hs, (int64_t)P.n_nodes * kFmmRec, &fa.rec));
    GX_CUDA(launch_fmm_moments(fa, P.level_off.data(), hdr[1], st));
    GX_TRY(mark(tm, 2, st));

    TreeListArgs la{};
    la.n = t.n;
    la.n_nodes = P.n_nodes;
    la.beg = t.beg;
    la.end = t.end;
    la.child = t.child;
    la.perm = t.perm;
    la.cx = t.cx;
    la.cy = t.cy;
    la.cz = t.cz;
    la.hw = t.hw;
    la.rec = fa.rec;
    la.theta = std::max(1.0e-6, opt.theta);  // FastMultipoleSolver constructor (fmm_solver.cpp:16)
    la.t_begin = begin;
    la.t_end = end;
    const int64_t nb = n + 1, lb = (int64_t)P.n_nodes + 1;
    GX_TRY(dev_array(hs, nb, &la.start_flag));
    GX_TRY(dev_array(hs, nb, &la.start_ord));
    GX_TRY(dev_array(hs, nb, &la.keep));
    GX_TRY(dev_array(hs, nb, &la.newpos));
    GX_TRY(dev_array(hs, lb, &la.leaf_off));
    GX_TRY(dev_array(hs, n, &la.leaf_part));
    GX_TRY(dev_array(hs, lb, &la.leaf_node));
    GX_TRY(dev_array(hs, lb, &la.node_leaf));
    for (int32_t** p : {&la.far_cnt, &la.near_cnt, &la.item_cnt, &la.slot_cnt, &la.far_off, &la.near_off, &la.item_off,
                        &la.slot_off})
        GX_TRY(dev_array(hs, lb, p));
    GX_TRY(dev_array(hs, 6, &la.totals));
    GX_TRY(dev_array(hs, (int64_t)P.n_nodes, &la.wn));
    const size_t list_bytes = tree_list_temp_bytes(la.n, la.n_nodes);
    void* list_temp;
    GX_TRY(dev_array(hs, (int64_t)list_bytes, (char**)&list_temp));
    GX_CUDA(launch_tree_lists_count(la, list_temp, list_bytes, st));
    int32_t nl = 0;
    unsigned long long tot[6];
    GX_CUDA(cudaMemcpyAsync(&nl, la.start_ord + n, sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaMemcpyAsync(tot, la.totals, sizeof(tot), cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaStreamSynchronize(st));
    for (int k = 0; k < 4; ++k)
        if (tot[k] > (unsigned long long)std::numeric_limits<int32_t>::max())
            return fail(GX_ERR_UNSUPPORTED, "FMM: interaction lists exceed the int32 range");
    P.far_pairs = (int64_t)tot[4];
    P.near_pairs = (int64_t)tot[5];
    P.n_leaves = fa.n_leaves = nl;
    P.n_far = (int64_t)tot[0];
    P.n_near = (int64_t)tot[1];
    fa.n_items = (int32_t)tot[2];
    P.n_slots = (int64_t)tot[3];
    GX_TRY(dev_array(hs, P.n_far, &la.far_node));
    GX_TRY(dev_array(hs, P.n_near, &la.near_key));
    GX_TRY(dev_array(hs, (int64_t)nl, &la.long_leaf));
    GX_TRY(dev_array(hs, 1, &la.long_count));
    GX_TRY(dev_array(hs, P.n_near, &la.near_leaf));
    M2PItem* items;
    GX_TRY(dev_array(hs, fa.n_items, &items));
    la.items = items;
    GX_CUDA(launch_tree_lists_fill(la, nl, st));
    // far-field items, largest first
    M2PItem* sorted_items;
    uint32_t *cost, *cost_alt;
    int32_t *idx, *idx_alt;
    GX_TRY(dev_array(hs, fa.n_items, &sorted_items));
    GX_TRY(dev_array(hs, fa.n_items, &cost));
    GX_TRY(dev_array(hs, fa.n_items, &cost_alt));
    GX_TRY(dev_array(hs, fa.n_items, &idx));
    GX_TRY(dev_array(hs, fa.n_items, &idx_alt));
    const size_t order_bytes = item_order_temp_bytes(fa.n_items);
    void* order_temp;
    GX_TRY(dev_array(hs, (int64_t)order_bytes, (char**)&order_temp));
    GX_CUDA(launch_item_order(items, la.leaf_off, fa.n_items, nullptr, nullptr, cost, cost_alt, idx, idx_alt, order_temp, order_bytes,
                              sorted_items, st));
    items = sorted_items;
    GX_TRY(mark(tm, 3, st));
    fa.leaf_off = la.leaf_off;
    fa.leaf_part = la.leaf_part;
    fa.far_node = la.far_node;
    fa.items = items;
    P.near_off = la.near_off;
    P.near_leaf = la.near_leaf;
    return GX_OK;
}

// Either builder for device-resident inputs; host copies of the inputs (hx..hm, may be
// null) spare a download when the host builder has to take over.
int fmm_plan(std::unique_ptr<FmmPlan>& P, cudaStream_t st, int64_t n, const double* hx, const double* hy,
             const double* hz, const double* hm, const double* dx, const double* dy, const double* dz, const double* dm,
             gx_physics phys, gx_fmm_options opt, int64_t begin, int64_t end, FmmTimer* tm = nullptr) {
    P.reset(new FmmPlan(st));
    bool deep = false;
    GX_TRY(fmm_plan_device(*P, n, dx, dy, dz, dm, phys, opt, begin, end, &deep, tm));
    if (!deep) return GX_OK;
    std::vector<double> hbuf;
    if (!hx) {
        hbuf.resize((size_t)n * 4);
        const double* src[4] = {dx, dy, dz, dm};
        for (int k = 0; k < 4; ++k)
            GX_CUDA(cudaMemcpyAsync(hbuf.data() + (size_t)k * n, src[k], (size_t)n * sizeof(double),
                                    cudaMemcpyDeviceToHost, st));
        GX_CUDA(cudaStreamSynchronize(st));
        hx = hbuf.data();
        hy = hx + n;
        hz = hy + n;
        hm = hz + n;
    }
    P.reset(new FmmPlan(st));
    return fmm_plan_host(*P, n, hx, hy, hz, hm, dx, dy, dz, dm, phys, opt, begin, end, tm);
}

int check_fmm_inputs(int64_t n, const double* m, bool device, const char* fn) {
    if (n > (int64_t)std::numeric_limits<int32_t>::max() / 2)
        return fail(GX_ERR_UNSUPPORTED, "%s: n exceeds the int32 index range", fn);
    if (!device)
        for (int64_t i = 0; i < n; ++i)
            if (m[i] < 0.0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: masses must be >= 0", fn);
    return GX_OK;
}


int fmm_accel(const char* fn, int64_t n, const double* x, const double* y, const double* z, const double* m,
              gx_physics phys, gx_fmm_options opt, int precision, int64_t begin, int64_t end, double* ax, double* ay,
              double* az, gx_fmm_stats* stats, void* stream, double* phase_ms) {
    if (stats) *stats = gx_fmm_stats{0, 0, 0, 0, 0, 0, 0};
    if (phase_ms)
        for (int k = 0; k < GX_FMM_PHASES; ++k) phase_ms[k] = 0.0;
    if (n < 0 || begin < 0 || end < 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: negative size or range", fn);
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: unknown precision", fn);
    GX_TRY(check_phys(phys, fn));
    if (!(opt.theta == opt.theta)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: theta is NaN", fn);
    end = std::min(end, n);  // compute_targets (fmm_solver.cpp:24-33)
    if (n == 0 || begin >= end) return GX_OK;
    if (!x || !y || !z || !m || !ax || !ay || !az) return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    GX_TRY(require_device());
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, m, ax, ay, az}, &device, &dev, fn));
    GX_TRY(check_fmm_inputs(n, m, device, fn));
    DeviceGuard g(dev);
    cudaStream_t st = (cudaStream_t)stream;

    HostStage hs(st);
    const double *dx = x, *dy = y, *dz = z, *dm = m;
    double *dax = ax, *day = ay, *daz = az;
    if (!device) {
        double *tx, *ty, *tz, *tm;
        GX_TRY(hs.in(x, n, &tx));
        GX_TRY(hs.in(y, n, &ty));
        GX_TRY(hs.in(z, n, &tz));
        GX_TRY(hs.in(m, n, &tm));
        dx = tx; dy = ty; dz = tz; dm = tm;
        GX_TRY(hs.out(&dax, n));
        GX_TRY(hs.out(&day, n));
        GX_TRY(hs.out(&daz, n));
    }
    std::unique_ptr<FmmTimer> tm;
    if (phase_ms) {
        tm.reset(new FmmTimer());
        GX_TRY(tm->create());
    }
    std::unique_ptr<FmmPlan> P;
    GX_TRY(fmm_plan(P, st, n, device ? nullptr : x, device ? nullptr : y, device ? nullptr : z, device ? nullptr : m,
                    dx, dy, dz, dm, phys, opt, begin, end, tm.get()));
    if (stats) {
        // node_count counts every node the reference creates, massless ones included
        stats->node_count = P->n_nodes;
        stats->leaf_count = P->n_leaves;
        stats->far_interactions = P->n_far;
        stats->near_interactions = P->n_near;
        stats->far_pairs = P->far_pairs;
        stats->near_pairs = P->near_pairs;
        stats->tree_levels = (int64_t)P->level_off.size() - 1;
    }
    // reset_accelerations over the target range (fmm_solver.cpp:31); the far and near
    // fields are then added
    for (double* p : {dax, day, daz}) GX_CUDA(cudaMemsetAsync(p + begin, 0, (size_t)(end - begin) * sizeof(double), st));
    if (P->n_leaves > 0) {
        FmmArgs& fa = P->fa;
        fa.ax = dax;
        fa.ay = day;
        fa.az = daz;
        AsyncBuf part, done, p2p_scratch;
        GX_TRY(part.alloc((size_t)std::max<int64_t>(P->n_slots, 1) * 3 * sizeof(double), st));
        GX_TRY(done.alloc((size_t)P->n_leaves * sizeof(int), st));
        GX_CUDA(cudaMemsetAsync(done.p, 0, (size_t)P->n_leaves * sizeof(int), st));
        fa.scratch = part.d();
        fa.done = (int*)done.p;
        // the mixed form evaluates the far field in FP32 on FP64 offsets, from FP32 copies
        // of the node records
        AsyncBuf rec32;
        const bool mixed = precision == kMixed;
        fa.rec32 = nullptr;
        fa.eps2f = (float)fa.eps2;
        if (mixed) {
            GX_TRY(rec32.alloc((size_t)std::max<int32_t>(fa.n_nodes, 1) * kRec32 * sizeof(float), st));
            fa.rec32 = (float*)rec32.p;
        }
        GX_CUDA(launch_fmm_m2p(fa, mixed, st));
        GX_TRY(mark(tm.get(), 4, st));

        P2PArgs pa{};
        pa.x = dx; pa.y = dy; pa.z = dz; pa.m = dm;
        pa.leaf_off = fa.leaf_off; pa.leaf_part = fa.leaf_part; pa.near_off = P->near_off; pa.near_leaf = P->near_leaf;
        pa.n_leaves = P->n_leaves;
        pa.ax = dax; pa.ay = day; pa.az = daz;
        pa.t_begin = begin;
        pa.t_end = end;
        pa.G = phys.G;
        pa.eps2 = phys.softening * phys.softening;
        pa.eps2f = (float)pa.eps2;
        GX_TRY(p2p_scratch.alloc(p2p_scratch_bytes(n, P->n_leaves), st));
        GX_CUDA(launch_p2p(pa, n, precision, p2p_scratch.p, sm_count(dev), st));
    } else {
        GX_TRY(mark(tm.get(), 4, st));
    }
    GX_TRY(mark(tm.get(), 5, st));
    if (!device) {
        GX_TRY(copy_back(ax + begin, dax + begin, end - begin, st));
        GX_TRY(copy_back(ay + begin, day + begin, end - begin, st));
        GX_TRY(copy_back(az + begin, daz + begin, end - begin, st));
        GX_CUDA(cudaStreamSynchronize(st));
    }
    if (phase_ms) {
        GX_CUDA(cudaEventSynchronize(tm->ev[5]));
        for (int k = 0; k < GX_FMM_PHASES; ++k) {
            float ms = 0.0f;
            GX_CUDA(cudaEventElapsedTime(&ms, tm->ev[k], tm->ev[k + 1]));
            phase_ms[k] = ms;
        }
        if (tm->host_tree_ms >= 0.0) phase_ms[0] = tm->host_tree_ms;
    }
    return GX_OK;
}

// ---- FMM evaluation without host reads (capacity mode) ---------------------------------
// gx_fmm_accel reads two sizes back per evaluation (node and level counts after the tree,
// list totals after the count walk) and sizes everything after them exactly.  FmmWork holds
// the same device arrays sized by capacities instead -- node slots and list, item and slot
// pools from a sizing evaluation with headroom -- so that an evaluation is a fixed sequence of
// launches with no host synchronisation (and can be captured in a CUDA graph): every kernel
// reads its counts on the device, pool_check marks an overflow when this evaluation needs more
// than a pool holds (or the tree needs the host builder), and everything after it is skipped;
// the caller checks the sticky flag and redoes the work with larger pools.
struct FmmWork {
    int64_t n = 0;
    gx_physics phys{};
    gx_fmm_options opt{};
    int32_t node_cap = 0;
    int64_t far_cap = 0, near_cap = 0, item_cap = 0, slot_cap = 0;
    int32_t leaves_hint = 0;
    std::vector<void*> owned;
    TreeBuildArgs t{};
    void* tree_temp = nullptr;
    size_t tree_bytes = 0;
    FmmArgs fa{};
    TreeListArgs la{};
    void* list_temp = nullptr;
    size_t list_bytes = 0;
    M2PItem *items = nullptr, *sorted = nullptr;
    uint32_t *cost = nullptr, *cost_alt = nullptr;
    int32_t *idx = nullptr, *idx_alt = nullptr;
    void* order_temp = nullptr;
    size_t order_bytes = 0;
    void* p2p_scratch = nullptr;
    int* flags = nullptr;                // device: [0] per-evaluation overflow, [1] sticky (bit 1: too deep)
    int* m2m_ready = nullptr;            // device: per-node flags and a ticket of the one-launch M2M
    int* m2m_ticket = nullptr;
    // Second stream of the evaluation (moments, far field) and the events that fork and join
    // it; the near field of the FP64 and mixed forms goes to near[0..3n) and is added after.
    cudaStream_t aux = nullptr;
    cudaEvent_t fork0 = nullptr, fork = nullptr, join = nullptr;
    double* near = nullptr;
    unsigned long long* need = nullptr;  // device: largest {nodes, far, near, items, slots, tree levels} seen
    int key_levels = 0;                  // levels of the path keys the tree sort orders
    ~FmmWork() {
        if (aux) {
            cudaStreamSynchronize(aux);
            cudaStreamDestroy(aux);
        }
        if (fork0) cudaEventDestroy(fork0);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        for (void* p : owned) cudaFree(p);
    }
    template <typename T>
    int grab(int64_t count, T** p) {
        void* q = nullptr;
        cudaError_t e = dev_alloc(&q, (size_t)std::max<int64_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc (FMM workspace)");
        owned.push_back(q);
        *p = (T*)q;
        return GX_OK;
    }
};

int64_t with_headroom(int64_t v) { return g_fmm_tight_pools.load() ? std::max<int64_t>(v, 1) : v + v / 2 + 4096; }

// Capacities from a sizing evaluation's counts (or from the largest counts an overflowing
// evaluation needed), with half again as much headroom; node slots never above the most a
// tree of n bodies can have.
// The tree sort orders key_levels levels of the path keys: two more than the sizing tree had,
// so a tree two levels deeper still builds; a deeper one sets the overflow flag and the
// chunk is redone with all levels.
int fmm_work_create(std::unique_ptr<FmmWork>& W, int64_t n, gx_physics phys, gx_fmm_options opt, int64_t nodes,
                    int64_t leaves, int64_t far, int64_t near, int64_t items, int64_t slots, int key_levels,
                    cudaStream_t st) {
    W.reset(new FmmWork());
    FmmWork& w = *W;
    w.key_levels = std::max(1, std::min(key_levels, (int)kKeyLevels));
    w.n = n;
    w.phys = phys;
    w.opt = opt;
    const int64_t cap = std::max<int64_t>(1, opt.leaf_capacity);
    const int64_t node_bound = 1 + 8 * (int64_t)kKeyLevels * (n / (cap + 1) + 1);
    w.node_cap = (int32_t)std::min<int64_t>({with_headroom(nodes), node_bound, (int64_t)0x7fff0000});
    w.far_cap = with_headroom(far);
    w.near_cap = with_headroom(near);
    w.item_cap = std::min<int64_t>(with_headroom(items), 0x7fff0000);
    w.slot_cap = with_headroom(slots);
    w.leaves_hint = (int32_t)std::max<int64_t>(1, leaves);
    const int32_t NC = w.node_cap;
    TreeBuildArgs& t = w.t;
    t.n = (int32_t)n;
    t.softening = phys.softening;
    t.cap = cap;
    t.max_depth = std::max(1, opt.max_depth);
    t.capacity = NC;
    t.key_levels = w.key_levels;
    GX_TRY(w.grab(6 * kBboxBlocks, &t.part));
    GX_TRY(w.grab(4, &t.root));
    GX_TRY(w.grab(n, &t.keys));
    GX_TRY(w.grab(n, &t.keys_alt));
    GX_TRY(w.grab(n, &t.idx));
    GX_TRY(w.grab(n, &t.perm));
    GX_TRY(w.grab(kKeyLevels + 3, &t.level_off));
    GX_TRY(w.grab(3, &t.hdr));
    for (int32_t** q : {&t.beg, &t.end, &t.child}) GX_TRY(w.grab(NC, q));
    for (double** q : {&t.cx, &t.cy, &t.cz, &t.hw}) GX_TRY(w.grab(NC, q));
    w.tree_bytes = tree_build_temp_bytes(t.n, cap);
    GX_TRY(w.grab((int64_t)w.tree_bytes, (char**)&w.tree_temp));
    GX_TRY(w.grab(2, &w.flags));
    GX_TRY(w.grab(6, &w.need));
    GX_TRY(w.grab(NC, &w.m2m_ready));
    GX_TRY(w.grab(1, &w.m2m_ticket));
    GX_TRY(w.grab(3 * n, &w.near));
    GX_CUDA(cudaStreamCreateWithFlags(&w.aux, cudaStreamNonBlocking));
    GX_CUDA(cudaEventCreateWithFlags(&w.fork0, cudaEventDisableTiming));
    GX_CUDA(cudaEventCreateWithFlags(&w.fork, cudaEventDisableTiming));
    GX_CUDA(cudaEventCreateWithFlags(&w.join, cudaEventDisableTiming));

    FmmArgs& fa = w.fa;
    fmm_common_args(fa, nullptr, nullptr, nullptr, nullptr, phys, opt, 0, n);
    fa.n_nodes = NC;
    fa.node_beg = t.beg;
    fa.node_end = t.end;
    fa.node_child = t.child;
    fa.node_cx = t.cx;
    fa.node_cy = t.cy;
    fa.node_cz = t.cz;
    fa.perm = t.perm;
    fa.cnt_nodes = t.hdr;
    GX_TRY(w.grab((int64_t)NC * kFmmRec, &fa.rec));
    GX_TRY(w.grab((int64_t)NC * kRec32, &fa.rec32));

    TreeListArgs& la = w.la;
    la.n = t.n;
    la.n_nodes = NC;
    la.beg = t.beg;
    la.end = t.end;
    la.child = t.child;
    la.perm = t.perm;
    la.cx = t.cx;
    la.cy = t.cy;
    la.cz = t.cz;
    la.hw = t.hw;
    la.rec = fa.rec;
    la.theta = std::max(1.0e-6, opt.theta);
    la.t_begin = 0;
    la.t_end = n;
    la.cnt_nodes = t.hdr;
    la.overflow = w.flags;
    la.overflow_sticky = w.flags + 1;
    la.need = w.need;
    la.far_cap = w.far_cap;
    la.near_cap = w.near_cap;
    GX_TRY(w.grab(n + 1, &la.mprefix));
    la.item_cap = w.item_cap;
    la.slot_cap = w.slot_cap;
    for (int32_t** q : {&la.start_flag, &la.start_ord, &la.keep, &la.newpos}) GX_TRY(w.grab(n + 1, q));
    GX_TRY(w.grab((int64_t)NC + 1, &la.leaf_off));
    GX_TRY(w.grab(n, &la.leaf_part));
    GX_TRY(w.grab((int64_t)NC + 1, &la.leaf_node));
    GX_TRY(w.grab((int64_t)NC + 1, &la.node_leaf));
    for (int32_t** q : {&la.far_cnt, &la.near_cnt, &la.item_cnt, &la.slot_cnt, &la.far_off, &la.near_off,
                        &la.item_off, &la.slot_off})
        GX_TRY(w.grab((int64_t)NC + 1, q));
    GX_TRY(w.grab(6, &la.totals));
    GX_TRY(w.grab(NC, &la.wn));
    w.list_bytes = tree_list_temp_bytes(la.n, NC);
    GX_TRY(w.grab((int64_t)w.list_bytes, (char**)&w.list_temp));
    GX_TRY(w.grab(w.far_cap, &la.far_node));
    GX_TRY(w.grab(w.near_cap, &la.near_key));
    GX_TRY(w.grab(w.near_cap, &la.near_leaf));
    GX_TRY(w.grab((int64_t)NC, &la.long_leaf));
    GX_TRY(w.grab(1, &la.long_count));
    GX_TRY(w.grab(w.item_cap, &w.items));
    la.items = w.items;
    GX_TRY(w.grab(w.item_cap, &w.sorted));
    GX_TRY(w.grab(w.item_cap, &w.cost));
    GX_TRY(w.grab(w.item_cap, &w.cost_alt));
    GX_TRY(w.grab(w.item_cap, &w.idx));
    GX_TRY(w.grab(w.item_cap, &w.idx_alt));
    w.order_bytes = item_order_temp_bytes((int32_t)w.item_cap);
    GX_TRY(w.grab((int64_t)w.order_bytes, (char**)&w.order_temp));

    fa.n_leaves = NC;
    fa.cnt_leaves = la.start_ord + n;
    fa.leaf_off = la.leaf_off;
    fa.leaf_part = la.leaf_part;
    fa.far_node = la.far_node;
    fa.items = w.sorted;
    fa.n_items = (int32_t)w.item_cap;
    fa.cnt_items = la.totals + 2;
    fa.overflow = w.flags;
    GX_TRY(w.grab(w.slot_cap * 3, &fa.scratch));
    GX_TRY(w.grab(NC, &fa.done));
    GX_TRY(w.grab((int64_t)p2p_scratch_bytes(n, NC), (char**)&w.p2p_scratch));
    GX_CUDA(cudaMemsetAsync(w.flags, 0, 2 * sizeof(int), st));
    GX_CUDA(cudaMemsetAsync(w.need, 0, 6 * sizeof(unsigned long long), st));
    return GX_OK;
}

// One FMM evaluation of the bodies (device arrays of w.n) into ax, ay, az, stream-ordered,
// with no host synchronisation.  A pool overflow leaves ax, ay, az zeroed and sets flags[1].
int fmm_work_enqueue(FmmWork& w, const double* x, const double* y, const double* z, const double* m,
                     int precision, double* ax, double* ay, double* az, int dev, cudaStream_t st) {
    const int64_t n = w.n;
    TreeBuildArgs& t = w.t;
    t.x = x;
    t.y = y;
    t.z = z;
    GX_CUDA(cudaMemsetAsync(w.flags, 0, sizeof(int), st));
    GX_CUDA(launch_tree_build(t, w.tree_temp, w.tree_bytes, st));
    GX_CUDA(launch_tree_leaf_order(t, w.node_cap, w.tree_temp, w.tree_bytes, st));
    FmmArgs& fa = w.fa;
    fa.x = x;
    fa.y = y;
    fa.z = z;
    fa.m = m;
    // Two streams after the tree: the moments and then the far field on aux; the lists (which
    // need only whether a node has mass, from counts of massive bodies) and the near field on
    // the caller's stream.  The far field waits for the lists.  The exact form's near field
    // continues the far field's sums in the reference's order, so it waits for the far field;
    // the other forms write the near field apart and add it once both are done.
    const bool side = precision != kF64Exact;
    GX_CUDA(cudaEventRecord(w.fork0, st));
    GX_CUDA(cudaStreamWaitEvent(w.aux, w.fork0, 0));
    GX_CUDA(launch_fmm_moments_tree(fa, w.m2m_ticket, w.m2m_ready, w.flags, sm_count(dev), w.aux));
    TreeListArgs& la = w.la;
    la.m = m;
    GX_CUDA(launch_tree_massive(la, w.list_temp, w.list_bytes, st));
    GX_CUDA(launch_tree_lists_count(la, w.list_temp, w.list_bytes, st));
    GX_CUDA(launch_pool_check(la, t.hdr, st));
    GX_CUDA(launch_tree_lists_fill(la, w.node_cap, st));
    GX_CUDA(launch_item_order(w.items, la.leaf_off, (int32_t)w.item_cap, la.totals + 2, w.flags, w.cost, w.cost_alt,
                              w.idx, w.idx_alt, w.order_temp, w.order_bytes, w.sorted, st));
    GX_CUDA(cudaEventRecord(w.fork, st));
    GX_CUDA(cudaStreamWaitEvent(w.aux, w.fork, 0));
    for (double* p : {ax, ay, az}) GX_CUDA(cudaMemsetAsync(p, 0, (size_t)n * sizeof(double), w.aux));
    fa.ax = ax;
    fa.ay = ay;
    fa.az = az;
    fa.eps2f = (float)fa.eps2;
    GX_CUDA(cudaMemsetAsync(fa.done, 0, (size_t)w.node_cap * sizeof(int), w.aux));
    GX_CUDA(launch_fmm_m2p(fa, precision == kMixed, w.aux));
    GX_CUDA(cudaEventRecord(w.join, w.aux));
    if (side) GX_CUDA(cudaMemsetAsync(w.near, 0, (size_t)(3 * n) * sizeof(double), st));
    else GX_CUDA(cudaStreamWaitEvent(st, w.join, 0));
    double* nx = side ? w.near : ax;
    double* ny = side ? w.near + n : ay;
    double* nz = side ? w.near + 2 * n : az;
    P2PArgs pa{};
    pa.x = x; pa.y = y; pa.z = z; pa.m = m;
    pa.leaf_off = la.leaf_off; pa.leaf_part = la.leaf_part; pa.near_off = la.near_off; pa.near_leaf = la.near_leaf;
    pa.n_leaves = w.node_cap;
    pa.cnt_leaves = la.start_ord + n;
    pa.overflow = w.flags;
    pa.leaves_hint = w.leaves_hint;
    pa.ax = nx; pa.ay = ny; pa.az = nz;
    pa.t_begin = 0;
    pa.t_end = n;
    pa.G = w.phys.G;
    pa.eps2 = w.phys.softening * w.phys.softening;
    pa.eps2f = (float)pa.eps2;
    GX_CUDA(launch_p2p(pa, n, precision, w.p2p_scratch, sm_count(dev), st));
    if (side) {
        GX_CUDA(cudaStreamWaitEvent(st, w.join, 0));
        GX_CUDA(launch_fmm_add_near(n, ax, ay, az, nx, ny, nz, sm_count(dev), st));
    }
    return GX_OK;
}

void fmm_work_release(FmmWork* w) { delete w; }

// Sizes the session's FMM workspace from one evaluation that reads its sizes back (the
// accelerations of that evaluation are not kept); *device_ok is false when the tree needs
// the host builder.
int session_fmm_size(gx_session* s, bool* device_ok) {
    std::unique_ptr<FmmPlan> P(new FmmPlan(s->stream));
    bool deep = false;
    GX_TRY(fmm_plan_device(*P, s->n, s->x, s->y, s->z, s->m, s->phys, s->fmm_opt, 0, s->n, &deep, nullptr));
    *device_ok = !deep;
    if (deep) return GX_OK;
    std::unique_ptr<FmmWork> W;
    GX_TRY(fmm_work_create(W, s->n, s->phys, s->fmm_opt, P->n_nodes, P->n_leaves, P->n_far, P->n_near,
                           P->fa.n_items, P->n_slots,
                           g_fmm_tight_pools.load() ? 1 : (int)P->level_off.size() - 1 + 2, s->stream));
    fmm_work_release(s->fmm);
    s->fmm = W.release();
    s->clear_graphs();
    return GX_OK;
}

// After an overflow: pools at least as large as the largest an evaluation needed, and half
// again larger than before.
int session_fmm_regrow(gx_session* s) {
    FmmWork& w = *s->fmm;
    unsigned long long need[6];
    GX_CUDA(cudaMemcpyAsync(need, w.need, sizeof(need), cudaMemcpyDeviceToHost, s->stream));
    GX_CUDA(cudaStreamSynchronize(s->stream));
    std::unique_ptr<FmmWork> W;
    GX_TRY(fmm_work_create(W, s->n, s->phys, s->fmm_opt, std::max<int64_t>((int64_t)need[0], w.node_cap),
                           w.leaves_hint, std::max<int64_t>((int64_t)need[1], w.far_cap),
                           std::max<int64_t>((int64_t)need[2], w.near_cap), std::max<int64_t>((int64_t)need[3], w.item_cap),
                           std::max<int64_t>((int64_t)need[4], w.slot_cap),
                           std::max(w.key_levels, (int)std::min<unsigned long long>(need[5], kKeyLevels) + 2), s->stream));
    fmm_work_release(s->fmm);
    s->fmm = W.release();
    s->clear_graphs();
    return GX_OK;
}

// An evaluation that reads its sizes back (and builds deep trees on the host).
int session_fmm_eval_sync(gx_session* s, int precision) {
    return fmm_accel("gx_session_step", s->n, s->x, s->y, s->z, s->m, s->phys, s->fmm_opt, precision, 0, s->n, s->ax,
                     s->ay, s->az, nullptr, s->stream, nullptr);
}

int session_fmm_force(gx_session* s, int precision, double kick_dt) {
    if (!s->fmm) return fail(GX_ERR_CUDA, "session FMM force: workspace missing");
    GX_TRY(fmm_work_enqueue(*s->fmm, s->x, s->y, s->z, s->m, precision, s->ax, s->ay, s->az, s->device, s->stream));
    if (kick_dt != 0.0) GX_CUDA(launch_kick(s->n, s->vx, s->vy, s->vz, s->ax, s->ay, s->az, kick_dt, s->stream));
    return GX_OK;
}

int session_fmm_prepare(gx_session* s) {
    if (s->t_begin != 0 || s->t_count != s->n)
        return fail(GX_ERR_UNSUPPORTED, "session FMM: owned target ranges are not supported with the FMM force");
    if (s->fmm || s->fmm_host_only) return GX_OK;
    bool ok = true;
    GX_TRY(session_fmm_size(s, &ok));
    if (!ok) s->fmm_host_only = true;
    return GX_OK;
}

// Reads the chunk's sticky overflow word (synchronises the stream): 0, 1 (a pool overflowed)
// or 3 (the tree needs the host builder).
int session_fmm_flag(gx_session* s, int* flag) {
    if (!s->host_flag) GX_CUDA(cudaMallocHost((void**)&s->host_flag, sizeof(int)));
    GX_CUDA(cudaMemcpyAsync(s->host_flag, s->fmm->flags + 1, sizeof(int), cudaMemcpyDeviceToHost, s->stream));
    GX_CUDA(cudaStreamSynchronize(s->stream));
    *flag = *s->host_flag;
    return GX_OK;
}

int session_fmm_compute(gx_session* s, int precision) {
    GX_TRY(session_fmm_prepare(s));
    for (int attempt = 0; attempt < 3 && !s->fmm_host_only; ++attempt) {
        GX_CUDA(cudaMemsetAsync(s->fmm->flags + 1, 0, sizeof(int), s->stream));
        GX_TRY(session_fmm_force(s, precision, 0.0));
        int flag = 0;
        GX_TRY(session_fmm_flag(s, &flag));
        if (flag == 0) return GX_OK;
        if (flag & 2) {
            s->fmm_host_only = true;
            break;
        }
        GX_TRY(session_fmm_regrow(s));
    }
    return session_fmm_eval_sync(s, precision);
}

// KDK steps with the FMM force: chunks of up to 32 steps, each replayed as one CUDA graph (no
// host synchronisation inside it) from a copy of the state taken on the device; after a chunk
// one read of its overflow word.  An overflow restores the copy, regrows the pools and redoes
// the chunk; a tree that needs the host builder, or a third overflow, takes the chunk one
// evaluation at a time through the path that reads its sizes back.
int session_fmm_steps(gx_session* s, int64_t n_steps, double dt, int precision) {
    GX_TRY(session_fmm_prepare(s));
    const double half = 0.5 * dt;
    auto eager = [&](int64_t k) -> int {
        for (int64_t i = 0; i < k; ++i) {
            GX_TRY(session_kick_drift(s, half, dt));
            GX_TRY(session_fmm_eval_sync(s, precision));
            GX_CUDA(launch_kick(s->n, s->vx, s->vy, s->vz, s->ax, s->ay, s->az, half, s->stream));
        }
        return GX_OK;
    };
    const size_t state_bytes = (size_t)9 * (size_t)s->n * sizeof(double);  // x .. az, contiguous
    for (int64_t done = 0; done < n_steps;) {
        const int64_t k = std::min<int64_t>(n_steps - done, 32);
        bool ok = false;
        for (int attempt = 0; attempt < 3 && !s->fmm_host_only; ++attempt) {
            if (!s->backup) {
                void* p = nullptr;
                cudaError_t e = dev_alloc(&p, state_bytes);
                if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc (session FMM state copy)");
                s->backup = (double*)p;
            }
            GX_CUDA(cudaMemcpyAsync(s->backup, s->buf, state_bytes, cudaMemcpyDeviceToDevice, s->stream));
            GX_CUDA(cudaMemsetAsync(s->fmm->flags + 1, 0, sizeof(int), s->stream));
            if (s->timing || s->stream == nullptr) {
                GX_TRY(session_enqueue_steps(s, k, dt, precision));
            } else {
                cudaGraphExec_t ge;
                GX_TRY(session_graph(s, k, dt, precision, &ge));
                GX_CUDA(cudaGraphLaunch(ge, s->stream));
            }
            int flag = 0;
            GX_TRY(session_fmm_flag(s, &flag));
            if (flag == 0) {
                ok = true;
                break;
            }
            GX_CUDA(cudaMemcpyAsync(s->buf, s->backup, state_bytes, cudaMemcpyDeviceToDevice, s->stream));
            if (flag & 2) {
                s->fmm_host_only = true;
                break;
            }
            GX_TRY(session_fmm_regrow(s));
        }
        if (!ok) GX_TRY(eager(k));
        done += k;
    }
    return GX_OK;
}

}  // namespace

extern "C" int gx_fmm_accel(int64_t n, const double* x, const double* y, const double* z, const double* m,
                            gx_physics phys, gx_fmm_options opt, int precision, int64_t begin, int64_t end,
                            double* ax, double* ay, double* az, gx_fmm_stats* stats, void* stream) {
    GX_GUARD_BEGIN
    return fmm_accel("gx_fmm_accel", n, x, y, z, m, phys, opt, precision, begin, end, ax, ay, az, stats, stream,
                     nullptr);
    GX_GUARD_END
}

extern "C" int gx_fmm_accel_timed(int64_t n, const double* x, const double* y, const double* z, const double* m,
                                  gx_physics phys, gx_fmm_options opt, int precision, int64_t begin, int64_t end,
                                  double* ax, double* ay, double* az, gx_fmm_stats* stats, void* stream,
                                  double* phase_ms) {
    GX_GUARD_BEGIN
    if (!phase_ms) return fail(GX_ERR_INVALID_ARGUMENT, "gx_fmm_accel_timed: phase_ms is null");
    return fmm_accel("gx_fmm_accel_timed", n, x, y, z, m, phys, opt, precision, begin, end, ax, ay, az, stats, stream,
                     phase_ms);
    GX_GUARD_END
}

extern "C" int gx_fmm_moments(int64_t n, const double* x, const double* y, const double* z, const double* m,
                              gx_physics phys, gx_fmm_options opt, int64_t capacity, double* records,
                              int64_t* n_nodes) {
    GX_GUARD_BEGIN
    const char* fn = "gx_fmm_moments";
    if (!n_nodes) return fail(GX_ERR_INVALID_ARGUMENT, "%s: n_nodes is null", fn);
    *n_nodes = 0;
    if (n < 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: n < 0", fn);
    GX_TRY(check_phys(phys, fn));
    if (n == 0) return GX_OK;
    if (!x || !y || !z || !m) return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    bool device;
    int dev;
    GX_TRY(require_device());
    GX_TRY(classify({x, y, z, m, records}, &device, &dev, fn));
    if (device) return fail(GX_ERR_INVALID_ARGUMENT, "%s: host arrays only", fn);
    GX_TRY(check_fmm_inputs(n, m, false, fn));
    DeviceGuard g(dev);
    cudaStream_t st = nullptr;
    HostStage hs(st);
    double *dx, *dy, *dz, *dm;
    GX_TRY(hs.in(x, n, &dx));
    GX_TRY(hs.in(y, n, &dy));
    GX_TRY(hs.in(z, n, &dz));
    GX_TRY(hs.in(m, n, &dm));
    std::unique_ptr<FmmPlan> P;
    GX_TRY(fmm_plan(P, st, n, x, y, z, m, dx, dy, dz, dm, phys, opt, 0, n));
    const int32_t nn = P->n_nodes;
    std::vector<double> h((size_t)nn * kFmmRec);
    std::vector<int32_t> child((size_t)nn);
    GX_CUDA(cudaMemcpyAsync(h.data(), P->fa.rec, h.size() * sizeof(double), cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaMemcpyAsync(child.data(), P->fa.node_child, child.size() * sizeof(int32_t), cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaStreamSynchronize(st));
    // nodes with mass > 0, breadth-first from the root, children in octant order
    std::vector<int32_t> bfs;
    if (nn > 0 && h[kRecMass] > 0.0) bfs.push_back(0);
    for (size_t k = 0; k < bfs.size(); ++k) {
        const int32_t c0 = child[bfs[k]];
        if (c0 < 0) continue;
        for (int c = 0; c < 8; ++c)
            if (h[(size_t)(c0 + c) * kFmmRec + kRecMass] > 0.0) bfs.push_back(c0 + c);
    }
    *n_nodes = (int64_t)bfs.size();
    if (!records) return GX_OK;
    if (capacity < (int64_t)bfs.size())
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: records hold %lld nodes, the tree has %zu", fn, (long long)capacity,
                    bfs.size());
    for (size_t k = 0; k < bfs.size(); ++k)
        std::copy(&h[(size_t)bfs[k] * kFmmRec], &h[(size_t)bfs[k] * kFmmRec] + 35, records + k * 35);
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gxi_leaf_lists_from_device(int64_t n, const double* x, const double* y, const double* z,
                                          const double* m, double softening, double theta, int64_t leaf_capacity,
                                          int max_depth, void* stream, gx::FmmTree* T, int* on_device) {
    GX_GUARD_BEGIN
    const char* fn = "gx_leaf_lists_build_device";
    GX_TRY(require_device());
    GX_TRY(check_fmm_inputs(n, m, false, fn));
    cudaStream_t st = (cudaStream_t)stream;
    HostStage hs(st);
    double *dx, *dy, *dz, *dm;
    GX_TRY(hs.in(x, n, &dx));
    GX_TRY(hs.in(y, n, &dy));
    GX_TRY(hs.in(z, n, &dz));
    GX_TRY(hs.in(m, n, &dm));
    gx_physics phys{1.0, softening};
    gx_fmm_options opt{theta, leaf_capacity, max_depth, 4};
    std::unique_ptr<FmmPlan> P;
    GX_TRY(fmm_plan(P, st, n, x, y, z, m, dx, dy, dz, dm, phys, opt, 0, n));
    *on_device = P->on_device ? 1 : 0;
    const int32_t nl = P->n_leaves;
    T->leaf_off.resize((size_t)nl + 1);
    T->near_off.resize((size_t)nl + 1);
    GX_CUDA(cudaMemcpyAsync(T->leaf_off.data(), P->fa.leaf_off, T->leaf_off.size() * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaMemcpyAsync(T->near_off.data(), P->near_off, T->near_off.size() * sizeof(int32_t),
                            cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaStreamSynchronize(st));
    T->leaf_part.resize((size_t)T->leaf_off[nl]);
    T->near_leaf.resize((size_t)P->n_near);
    if (!T->leaf_part.empty())
        GX_CUDA(cudaMemcpyAsync(T->leaf_part.data(), P->fa.leaf_part, T->leaf_part.size() * sizeof(int32_t),
                                cudaMemcpyDeviceToHost, st));
    if (!T->near_leaf.empty())
        GX_CUDA(cudaMemcpyAsync(T->near_leaf.data(), P->near_leaf, T->near_leaf.size() * sizeof(int32_t),
                                cudaMemcpyDeviceToHost, st));
    GX_CUDA(cudaStreamSynchronize(st));
    T->n_far = P->n_far;
    T->n_pairs = 0;
    for (int32_t l = 0; l < nl; ++l)
        for (int32_t k = T->near_off[l]; k < T->near_off[l + 1]; ++k)
            T->n_pairs += (int64_t)(T->leaf_off[l + 1] - T->leaf_off[l]) *
                          (T->leaf_off[T->near_leaf[k] + 1] - T->leaf_off[T->near_leaf[k]]);
    return GX_OK;
    GX_GUARD_END
}

// ======================================================================================
// adjoint
// ======================================================================================
extern "C" int gx_direct_vjp(int64_t n, const double* x, const double* y, const double* z, const double* m,
                             const double* lx, const double* ly, const double* lz, gx_physics phys, int precision,
                             double* gxo, double* gyo, double* gzo, double* gmo, void* stream) {
    GX_GUARD_BEGIN
    const char* fn = "gx_direct_vjp";
    if (n < 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: n < 0", fn);
    if (precision != kF64 && precision != kMixed)
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: precision must be F64 or MIXED", fn);
    GX_TRY(check_phys(phys, fn));
    if (n > 0 && (!x || !y || !z || !m || !lx || !ly || !lz || !gxo || !gyo || !gzo))
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    GX_TRY(require_device());
    if (n == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, m, lx, ly, lz, gxo, gyo, gzo, gmo}, &device, &dev, fn));
    DeviceGuard g(dev);
    cudaStream_t st = (cudaStream_t)stream;
    HostStage hs(st);
    const double* in[7] = {x, y, z, m, lx, ly, lz};
    double* out[4] = {gxo, gyo, gzo, gmo};
    if (!device) {
        for (int k = 0; k < 7; ++k) {
            double* p;
            GX_TRY(hs.in(in[k], n, &p));
            in[k] = p;
        }
        for (int k = 0; k < 4; ++k) {
            if (!out[k]) continue;
            double* p;
            GX_TRY(hs.out(&p, n));
            out[k] = p;
        }
    }
    VjpArgs a;
    a.x = in[0]; a.y = in[1]; a.z = in[2]; a.m = in[3]; a.lx = in[4]; a.ly = in[5]; a.lz = in[6];
    a.n = n;
    a.gx = out[0]; a.gy = out[1]; a.gz = out[2]; a.gm = out[3];
    a.G = phys.G;
    a.eps2 = phys.softening * phys.softening;
    a.eps2f = (float)a.eps2;
    // source split chosen by the same per-SM-rounds model as the forward kernels
    const int sms = sm_count(dev);
    int want = 1;
    {
        const VjpShape sh = vjp_shape(precision);
        double best = rounds_cost(sh.block, sh.ipt, sh.jt, sh.occupancy, n, n, 1, sms);
        for (int ns = 2; ns <= 64; ++ns) {
            int64_t chunk;
            int nse;
            split_layout(n, sh.jt, ns, &chunk, &nse);
            if (nse != ns) continue;
            const double c = rounds_cost(sh.block, sh.ipt, sh.jt, sh.occupancy, n, n, ns, sms);
            if (c < best * 0.995) {
                best = c;
                want = ns;
            }
        }
    }
    split_layout(n, vjp_jt(precision), want, &a.j_chunk, &a.nsplit);
    AsyncBuf part;
    a.part = nullptr;
    if (a.nsplit > 1) {
        GX_TRY(part.alloc((size_t)a.nsplit * 4 * (size_t)n * sizeof(double), st));
        a.part = part.d();
    }
    GX_CUDA(launch_vjp(a, precision, st));
    if (!device) {
        for (int k = 0; k < 4; ++k)
            if (out[k]) GX_TRY(copy_back(k == 0 ? gxo : k == 1 ? gyo : k == 2 ? gzo : gmo, out[k], n, st));
        GX_CUDA(cudaStreamSynchronize(st));
    }
    return GX_OK;
    GX_GUARD_END
}

// ======================================================================================
// batched ensembles
// ======================================================================================
struct gx_batch {
    int device = 0;
    int32_t ni = 0;
    std::vector<int64_t> off_h;
    int64_t n = 0;
    gx_physics phys{1.0, 0.05};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double* buf = nullptr;
    double *x, *y, *z, *vx, *vy, *vz, *ax, *ay, *az, *m;
    int64_t* off_d = nullptr;
    int2* items_d = nullptr;
    int n_items = 0;
    int items_tile = 0;
    int* counter = nullptr;
    int cfg[3] = {-1, -1, -1};
    int2* pot_items_d = nullptr;
    int n_pot_items = 0;
    int* pot_first_d = nullptr;
    int* pot_count_d = nullptr;
    double* pot_part = nullptr;
    double* diag_out = nullptr;
    std::map<std::tuple<int64_t, uint64_t, int, int>, cudaGraphExec_t> graphs;
    bool timing = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> events;
    double timed_ms = 0.0;
    int64_t timed_launches = 0;

    void clear_graphs() {
        for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
        graphs.clear();
    }
};

namespace {

int batch_default_variant(gx_batch* b, int precision) {
    if (b->cfg[precision] >= 0) return b->cfg[precision];
    int ids[16];
    const int c = batch_variant_ids(precision, eps0_of(precision, b->phys) ? 1 : 0, ids, 16);
    if (c <= 0) return -1;
    b->cfg[precision] = ids[0];
    return ids[0];
}

// (instance, tile) items for tiles of `tile` targets, largest instances first.
int batch_build_items(gx_batch* b, int tile) {
    if (b->items_tile == tile && b->items_d) return GX_OK;
    std::vector<int> order((size_t)b->ni);
    for (int i = 0; i < b->ni; ++i) order[(size_t)i] = i;
    std::stable_sort(order.begin(), order.end(), [&](int p, int q) {
        return b->off_h[p + 1] - b->off_h[p] > b->off_h[q + 1] - b->off_h[q];
    });
    std::vector<int2> items;
    for (int inst : order) {
        const int64_t nb = b->off_h[inst + 1] - b->off_h[inst];
        const int64_t tiles = (nb + tile - 1) / tile;
        for (int64_t t = 0; t < tiles; ++t) items.push_back(make_int2(inst, (int)t));
    }
    if (items.size() > (size_t)INT32_MAX) return fail(GX_ERR_INVALID_ARGUMENT, "batch: too many work items");
    if (b->items_d) {
        cudaStreamSynchronize(b->stream);
        cudaFree(b->items_d);
        b->items_d = nullptr;
    }
    void* p;
    cudaError_t e = dev_alloc(&p, std::max<size_t>(1, items.size()) * sizeof(int2));
    if (e != cudaSuccess) return fail_cuda(e, "cudaMalloc (batch items)");
    b->items_d = (int2*)p;
    if (!items.empty())
        GX_CUDA(cudaMemcpyAsync(b->items_d, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    GX_CUDA(cudaStreamSynchronize(b->stream));
    b->n_items = (int)items.size();
    b->items_tile = tile;
    b->clear_graphs();
    return GX_OK;
}

BatchArgs batch_args(gx_batch* b, double kick_dt) {
    BatchArgs a;
    a.x = b->x; a.y = b->y; a.z = b->z; a.m = b->m;
    a.offsets = b->off_d;
    a.items = b->items_d;
    a.n_items = b->n_items;
    a.counter = b->counter;
    a.ax = b->ax; a.ay = b->ay; a.az = b->az;
    a.vx = kick_dt != 0.0 ? b->vx : nullptr;
    a.vy = kick_dt != 0.0 ? b->vy : nullptr;
    a.vz = kick_dt != 0.0 ? b->vz : nullptr;
    a.kick_dt = kick_dt;
    a.G = b->phys.G;
    a.eps2 = b->phys.softening * b->phys.softening;
    a.eps2f = (float)a.eps2;
    return a;
}

int batch_force(gx_batch* b, int precision, double kick_dt) {
    const int vid = batch_default_variant(b, precision);
    if (vid < 0) return fail(GX_ERR_UNSUPPORTED, "batch: precision %d has no batched variant", precision);
    int cnt;
    const BatchVariant& v = batch_variants(&cnt)[vid];
    GX_TRY(batch_build_items(b, v.block * v.ipt));
    if (b->n_items == 0) return GX_OK;
    const int grid = std::max(1, std::min(b->n_items, sm_count(b->device) * batch_occupancy(v)));
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (b->timing) {
        GX_CUDA(cudaEventCreate(&e0));
        GX_CUDA(cudaEventCreate(&e1));
        GX_CUDA(cudaEventRecord(e0, b->stream));
    }
    GX_CUDA(batch_force_launch(v, batch_args(b, kick_dt), grid, b->stream));
    if (b->timing) {
        GX_CUDA(cudaEventRecord(e1, b->stream));
        b->events.emplace_back(e0, e1);
    }
    return GX_OK;
}

int batch_enqueue_steps(gx_batch* b, int64_t k, double dt, int precision) {
    const double half = 0.5 * dt;
    for (int64_t i = 0; i < k; ++i) {
        GX_CUDA(launch_kick_drift(b->n, b->x, b->y, b->z, b->vx, b->vy, b->vz, b->ax, b->ay, b->az, half, dt, b->stream));
        GX_TRY(batch_force(b, precision, half));
    }
    return GX_OK;
}

int batch_flush_events(gx_batch* b) {
    if (b->events.empty()) return GX_OK;
    GX_CUDA(cudaStreamSynchronize(b->stream));
    for (auto& ev : b->events) {
        float ms = 0.f;
        GX_CUDA(cudaEventElapsedTime(&ms, ev.first, ev.second));
        b->timed_ms += ms;
        b->timed_launches += 1;
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    b->events.clear();
    return GX_OK;
}

int check_batch(gx_batch* b, const char* fn) {
    if (!b) return fail(GX_ERR_INVALID_ARGUMENT, "%s: null batch", fn);
    return GX_OK;
}

void batch_release(gx_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    for (auto& ev : b->events) {
        cudaEventDestroy(ev.first);
        cudaEventDestroy(ev.second);
    }
    b->clear_graphs();
    void* ptrs[] = {b->buf, b->off_d, b->items_d, b->counter, b->pot_items_d, b->pot_first_d,
                    b->pot_count_d, b->pot_part, b->diag_out};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (b->own_stream && b->stream) cudaStreamDestroy(b->stream);
    delete b;
}

}  // namespace

extern "C" int gx_batch_create(int32_t n_instances, const int64_t* offsets, gx_physics phys, int device,
                               gx_batch** out) {
    GX_GUARD_BEGIN
    const char* fn = "gx_batch_create";
    if (!out) return fail(GX_ERR_INVALID_ARGUMENT, "%s: out is null", fn);
    *out = nullptr;
    if (n_instances < 1 || !offsets) return fail(GX_ERR_INVALID_ARGUMENT, "%s: need n_instances >= 1 and offsets", fn);
    if (offsets[0] != 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: offsets[0] must be 0", fn);
    for (int32_t i = 0; i < n_instances; ++i)
        if (offsets[i + 1] < offsets[i]) return fail(GX_ERR_INVALID_ARGUMENT, "%s: offsets must be non-decreasing", fn);
    if (offsets[n_instances] < 1) return fail(GX_ERR_INVALID_ARGUMENT, "%s: no bodies", fn);
    GX_TRY(check_phys(phys, fn));
    GX_TRY(require_device());
    int count = 0;
    GX_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count) return fail(GX_ERR_INVALID_ARGUMENT, "%s: device %d out of range", fn, device);
    DeviceGuard g(device);
    gx_batch* b = new gx_batch();
    b->device = device;
    b->ni = n_instances;
    b->off_h.assign(offsets, offsets + n_instances + 1);
    b->n = offsets[n_instances];
    b->phys = phys;
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        delete b;
        return fail_cuda(e, "cudaStreamCreate (batch)");
    }
    b->own_stream = true;
    void* p = nullptr;
    e = dev_alloc(&p, (size_t)b->n * 10 * sizeof(double));
    if (e == cudaSuccess) {
        b->buf = (double*)p;
        double** arr[10] = {&b->x, &b->y, &b->z, &b->vx, &b->vy, &b->vz, &b->ax, &b->ay, &b->az, &b->m};
        for (int k = 0; k < 10; ++k) *arr[k] = b->buf + (size_t)k * (size_t)b->n;
        e = dev_alloc(&p, (size_t)(n_instances + 1) * sizeof(int64_t));
    }
    if (e == cudaSuccess) {
        b->off_d = (int64_t*)p;
        e = dev_alloc(&p, 16);
    }
    if (e == cudaSuccess) {
        b->counter = (int*)p;
        // diagnostics work lists: tiles of batch_potential_tile() targets, instance order
        const int pt = batch_potential_tile();
        std::vector<int2> pitems;
        std::vector<int> first((size_t)n_instances), cnt((size_t)n_instances);
        for (int32_t i = 0; i < n_instances; ++i) {
            const int64_t nb = offsets[i + 1] - offsets[i];
            first[(size_t)i] = (int)pitems.size();
            const int64_t tiles = (nb + pt - 1) / pt;
            for (int64_t t = 0; t < tiles; ++t) pitems.push_back(make_int2(i, (int)t));
            cnt[(size_t)i] = (int)tiles;
        }
        b->n_pot_items = (int)pitems.size();
        e = dev_alloc(&p, std::max<size_t>(1, pitems.size()) * sizeof(int2));
        if (e == cudaSuccess) {
            b->pot_items_d = (int2*)p;
            e = dev_alloc(&p, (size_t)n_instances * sizeof(int));
        }
        if (e == cudaSuccess) {
            b->pot_first_d = (int*)p;
            e = dev_alloc(&p, (size_t)n_instances * sizeof(int));
        }
        if (e == cudaSuccess) {
            b->pot_count_d = (int*)p;
            e = dev_alloc(&p, std::max<size_t>(1, pitems.size()) * sizeof(double));
        }
        if (e == cudaSuccess) {
            b->pot_part = (double*)p;
            e = dev_alloc(&p, (size_t)n_instances * 13 * sizeof(double));
        }
        if (e == cudaSuccess) {
            b->diag_out = (double*)p;
            if (!pitems.empty())
                e = cudaMemcpyAsync(b->pot_items_d, pitems.data(), pitems.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream);
        }
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->pot_first_d, first.data(), first.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->pot_count_d, cnt.data(), cnt.size() * sizeof(int), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->off_d, offsets, (size_t)(n_instances + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, b->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(b->buf, 0, (size_t)b->n * 10 * sizeof(double), b->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    }
    if (e != cudaSuccess) {
        const int r = fail_cuda(e, "gx_batch_create");
        batch_release(b);
        return r;
    }
    *out = b;
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_batch_destroy(gx_batch* b) {
    GX_GUARD_BEGIN
    if (!b) return GX_OK;
    DeviceGuard g(b->device);
    batch_release(b);
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_batch_set_stream(gx_batch* b, void* stream) {
    GX_TRY(check_batch(b, "gx_batch_set_stream"));
    DeviceGuard g(b->device);
    cudaStreamSynchronize(b->stream);
    if (b->own_stream) cudaStreamDestroy(b->stream);
    b->own_stream = false;
    b->stream = (cudaStream_t)stream;
    b->clear_graphs();
    return GX_OK;
}

extern "C" int gx_batch_set_state(gx_batch* b, const double* x, const double* y, const double* z, const double* vx,
                                  const double* vy, const double* vz, const double* m) {
    GX_GUARD_BEGIN
    const char* fn = "gx_batch_set_state";
    GX_TRY(check_batch(b, fn));
    if (!x || !y || !z || !vx || !vy || !vz || !m) return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, vx, vy, vz, m}, &device, &dev, fn));
    DeviceGuard g(b->device);
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    const double* src[7] = {x, y, z, vx, vy, vz, m};
    double* dst[7] = {b->x, b->y, b->z, b->vx, b->vy, b->vz, b->m};
    const size_t bytes = (size_t)b->n * sizeof(double);
    for (int k = 0; k < 7; ++k) GX_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, kind, b->stream));
    GX_CUDA(cudaMemsetAsync(b->ax, 0, 3 * bytes, b->stream));
    GX_CUDA(cudaStreamSynchronize(b->stream));
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_batch_get_state(gx_batch* b, double* x, double* y, double* z, double* vx, double* vy, double* vz,
                                  double* ax, double* ay, double* az) {
    GX_GUARD_BEGIN
    const char* fn = "gx_batch_get_state";
    GX_TRY(check_batch(b, fn));
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, vx, vy, vz, ax, ay, az}, &device, &dev, fn));
    DeviceGuard g(b->device);
    const cudaMemcpyKind kind = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    double* dst[9] = {x, y, z, vx, vy, vz, ax, ay, az};
    const double* src[9] = {b->x, b->y, b->z, b->vx, b->vy, b->vz, b->ax, b->ay, b->az};
    const size_t bytes = (size_t)b->n * sizeof(double);
    for (int k = 0; k < 9; ++k)
        if (dst[k]) GX_CUDA(cudaMemcpyAsync(dst[k], src[k], bytes, kind, b->stream));
    GX_CUDA(cudaStreamSynchronize(b->stream));
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_batch_device_arrays(gx_batch* b, double** p) {
    GX_TRY(check_batch(b, "gx_batch_device_arrays"));
    if (!p) return fail(GX_ERR_INVALID_ARGUMENT, "gx_batch_device_arrays: null");
    double* a[10] = {b->x, b->y, b->z, b->vx, b->vy, b->vz, b->ax, b->ay, b->az, b->m};
    for (int k = 0; k < 10; ++k) p[k] = a[k];
    return GX_OK;
}

extern "C" int gx_batch_compute_accelerations(gx_batch* b, int precision) {
    GX_GUARD_BEGIN
    GX_TRY(check_batch(b, "gx_batch_compute_accelerations"));
    if (precision != kF64 && precision != kMixed)
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_batch_compute_accelerations: precision must be F64 or MIXED");
    DeviceGuard g(b->device);
    return batch_force(b, precision, 0.0);
    GX_GUARD_END
}

extern "C" int gx_batch_step(gx_batch* b, int64_t n_steps, double dt, int precision) {
    GX_GUARD_BEGIN
    const char* fn = "gx_batch_step";
    GX_TRY(check_batch(b, fn));
    if (precision != kF64 && precision != kMixed) return fail(GX_ERR_INVALID_ARGUMENT, "%s: precision must be F64 or MIXED", fn);
    if (n_steps < 0 || !std::isfinite(dt)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: need n_steps >= 0, finite dt", fn);
    if (n_steps == 0) return GX_OK;
    DeviceGuard g(b->device);
    if (b->timing || b->stream == nullptr) return batch_enqueue_steps(b, n_steps, dt, precision);
    const int vid = batch_default_variant(b, precision);
    if (vid < 0) return fail(GX_ERR_UNSUPPORTED, "%s: no batched variant", fn);
    int cnt;
    const BatchVariant& v = batch_variants(&cnt)[vid];
    GX_TRY(batch_build_items(b, v.block * v.ipt));
    uint64_t dtb;
    std::memcpy(&dtb, &dt, sizeof(dtb));
    // The whole multi-step run is one graph (capped at 1024 steps per graph).
    const int64_t chunk = std::min<int64_t>(n_steps, 1024);
    auto get = [&](int64_t k, cudaGraphExec_t* ge) -> int {
        const auto key = std::make_tuple(k, dtb, precision, vid);
        auto it = b->graphs.find(key);
        if (it != b->graphs.end()) {
            *ge = it->second;
            return GX_OK;
        }
        GX_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        const int r = batch_enqueue_steps(b, k, dt, precision);
        cudaGraph_t graph = nullptr;
        cudaError_t e = cudaStreamEndCapture(b->stream, &graph);
        if (r != GX_OK) {
            if (graph) cudaGraphDestroy(graph);
            return r;
        }
        if (e != cudaSuccess) return fail_cuda(e, "cudaStreamEndCapture (batch)");
        cudaGraphExec_t exec;
        e = cudaGraphInstantiate(&exec, graph, 0);
        cudaGraphDestroy(graph);
        if (e != cudaSuccess) return fail_cuda(e, "cudaGraphInstantiate (batch)");
        if (b->graphs.size() > 16) b->clear_graphs();
        b->graphs[key] = exec;
        *ge = exec;
        return GX_OK;
    };
    cudaGraphExec_t ge;
    GX_TRY(get(chunk, &ge));
    for (int64_t i = 0; i < n_steps / chunk; ++i) GX_CUDA(cudaGraphLaunch(ge, b->stream));
    if (n_steps % chunk) {
        GX_TRY(get(n_steps % chunk, &ge));
        GX_CUDA(cudaGraphLaunch(ge, b->stream));
    }
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_batch_diagnostics(gx_batch* b, gx_diagnostics* out) {
    GX_GUARD_BEGIN
    GX_TRY(check_batch(b, "gx_batch_diagnostics"));
    if (!out) return fail(GX_ERR_INVALID_ARGUMENT, "gx_batch_diagnostics: null");
    DeviceGuard g(b->device);
    BatchArgs a = batch_args(b, 0.0);
    a.items = b->pot_items_d;
    a.n_items = b->n_pot_items;
    GX_CUDA(batch_diagnostics_launch(a, b->n_pot_items, b->ni, b->vx, b->vy, b->vz, b->pot_first_d, b->pot_count_d,
                                     b->pot_part, b->diag_out, b->stream));
    std::vector<double> h((size_t)b->ni * 13);
    GX_CUDA(cudaMemcpyAsync(h.data(), b->diag_out, h.size() * sizeof(double), cudaMemcpyDeviceToHost, b->stream));
    GX_CUDA(cudaStreamSynchronize(b->stream));
    for (int32_t i = 0; i < b->ni; ++i) fill_diag(h.data() + (size_t)i * 13, out + i);
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_batch_synchronize(gx_batch* b) {
    GX_TRY(check_batch(b, "gx_batch_synchronize"));
    DeviceGuard g(b->device);
    GX_CUDA(cudaStreamSynchronize(b->stream));
    return GX_OK;
}

extern "C" int gx_batch_get_config(gx_batch* b, int precision, int* variant) {
    GX_TRY(check_batch(b, "gx_batch_get_config"));
    if ((precision != kF64 && precision != kMixed) || !variant)
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_batch_get_config: bad arguments");
    *variant = batch_default_variant(b, precision);
    return GX_OK;
}

extern "C" int gx_batch_set_config(gx_batch* b, int precision, int variant) {
    GX_TRY(check_batch(b, "gx_batch_set_config"));
    int cnt;
    const BatchVariant* all = batch_variants(&cnt);
    if ((precision != kF64 && precision != kMixed) || variant < 0 || variant >= cnt ||
        all[variant].precision != precision || (bool)all[variant].eps0 != eps0_of(precision, b->phys))
        return fail(GX_ERR_INVALID_ARGUMENT, "gx_batch_set_config: variant does not fit");
    b->cfg[precision] = variant;
    b->clear_graphs();
    return GX_OK;
}

extern "C" int gx_batch_autotune(gx_batch* b, int precision, double* best_ms) {
    GX_GUARD_BEGIN
    const char* fn = "gx_batch_autotune";
    GX_TRY(check_batch(b, fn));
    if (precision != kF64 && precision != kMixed) return fail(GX_ERR_INVALID_ARGUMENT, "%s: precision", fn);
    DeviceGuard g(b->device);
    int ids[16];
    const int c = std::min(16, batch_variant_ids(precision, eps0_of(precision, b->phys) ? 1 : 0, ids, 16));
    const bool was_timing = b->timing;
    b->timing = false;
    cudaEvent_t e0, e1;
    GX_CUDA(cudaEventCreate(&e0));
    GX_CUDA(cudaEventCreate(&e1));
    int best = -1;
    double bms = 1e300;
    int status = GX_OK;
    for (int k = 0; k < c && status == GX_OK; ++k) {
        b->cfg[precision] = ids[k];
        status = batch_force(b, precision, 0.0);  // warm-up (and item rebuild)
        double t = 1e300;
        for (int r = 0; r < 2 && status == GX_OK; ++r) {
            cudaEventRecord(e0, b->stream);
            status = batch_force(b, precision, 0.0);
            cudaEventRecord(e1, b->stream);
            float ms = 0.f;
            const cudaError_t te = cudaEventSynchronize(e1);
            if (te == cudaSuccess && cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess) t = std::min(t, (double)ms);
            else if (status == GX_OK) status = fail_cuda(te != cudaSuccess ? te : cudaGetLastError(), "batch autotune timing");
        }
        if (status == GX_OK && t < bms) {
            bms = t;
            best = ids[k];
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->timing = was_timing;
    if (status != GX_OK) return status;
    b->cfg[precision] = best;
    b->clear_graphs();
    // accelerations must describe the state again
    GX_TRY(batch_force(b, precision, 0.0));
    if (best_ms) *best_ms = bms;
    return GX_OK;
    GX_GUARD_END
}

extern "C" int gx_batch_enable_timing(gx_batch* b, int enable) {
    GX_TRY(check_batch(b, "gx_batch_enable_timing"));
    DeviceGuard g(b->device);
    GX_TRY(batch_flush_events(b));
    b->timing = enable != 0;
    b->timed_ms = 0.0;
    b->timed_launches = 0;
    return GX_OK;
}

extern "C" int gx_batch_force_timing(gx_batch* b, double* total_ms, int64_t* launches) {
    GX_TRY(check_batch(b, "gx_batch_force_timing"));
    DeviceGuard g(b->device);
    GX_TRY(batch_flush_events(b));
    if (total_ms) *total_ms = b->timed_ms;
    if (launches) *launches = b->timed_launches;
    return GX_OK;
}

extern "C" int gx_batch_accel(int32_t n_instances, const int64_t* offsets, const double* x, const double* y,
                              const double* z, const double* m, gx_physics phys, int precision, double* ax,
                              double* ay, double* az, void* stream) {
    GX_GUARD_BEGIN
    const char* fn = "gx_batch_accel";
    if (n_instances < 1 || !offsets || !x || !y || !z || !m || !ax || !ay || !az)
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: bad arguments", fn);
    if (precision != kF64 && precision != kMixed) return fail(GX_ERR_INVALID_ARGUMENT, "%s: precision must be F64 or MIXED", fn);
    GX_TRY(require_device());
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, m, ax, ay, az}, &device, &dev, fn));
    int cur = 0;
    cudaGetDevice(&cur);
    gx_batch* b = nullptr;
    GX_TRY(gx_batch_create(n_instances, offsets, phys, device ? dev : cur, &b));
    int r = GX_OK;
    {
        DeviceGuard g(b->device);
        const int64_t n = b->n;
        const cudaMemcpyKind kin = device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
        const cudaMemcpyKind kout = device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
        cudaStream_t st = (cudaStream_t)stream;
        // Order the batch's own stream after the caller's stream.
        cudaEvent_t ev;
        cudaError_t e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventRecord(ev, st);
        if (e == cudaSuccess) e = cudaStreamWaitEvent(b->stream, ev, 0);
        const double* src[4] = {x, y, z, m};
        double* dst[4] = {b->x, b->y, b->z, b->m};
        for (int k = 0; k < 4 && e == cudaSuccess; ++k)
            e = cudaMemcpyAsync(dst[k], src[k], (size_t)n * sizeof(double), kin, b->stream);
        if (e != cudaSuccess) r = fail_cuda(e, fn);
        if (r == GX_OK) r = batch_force(b, precision, 0.0);
        double* out[3] = {ax, ay, az};
        const double* res[3] = {b->ax, b->ay, b->az};
        for (int k = 0; k < 3 && r == GX_OK; ++k) {
            e = cudaMemcpyAsync(out[k], res[k], (size_t)n * sizeof(double), kout, b->stream);
            if (e != cudaSuccess) r = fail_cuda(e, fn);
        }
        if (r == GX_OK) {
            e = cudaStreamSynchronize(b->stream);
            if (e != cudaSuccess) r = fail_cuda(e, fn);
        }
        cudaEventDestroy(ev);
    }
    gx_batch_destroy(b);
    return r;
    GX_GUARD_END
}

// ======================================================================================
// direct sum that allocates nothing
// ======================================================================================
// Some callers cannot allocate device memory when they call in: a process whose GPU memory
// is entirely reserved up front by another framework's caching allocator, a real-time step
// loop that must never enter the allocator, or code that runs while a stream is being
// captured with allocation forbidden.  gx_direct_accel_noalloc serves them: it runs the same
// tiled, source-split direct sum as gx_direct_accel on the caller's device arrays, but keeps
// the split's partial sums in one fixed file-scope device array instead of allocating
// scratch.  The array is part of the library's device image, so every GPU that loads the
// library holds it (12 MiB) until the process exits.
namespace {

constexpr int64_t kNoAllocMaxBodies = 65536;  // largest n this entry point accepts
constexpr int kNoAllocMaxSplit = 8;           // source chunks whose partials the array holds
constexpr size_t kNoAllocScratchDoubles = (size_t)kNoAllocMaxSplit * 3 * (size_t)kNoAllocMaxBodies;

static __device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];

std::mutex g_noalloc_mu;
std::map<int, double*> g_noalloc_addr;  // device ordinal -> device address of the array

// The array's name is only a host-side stand-in in host code; its device address is looked
// up once per device, with that device current, and reused.
int noalloc_scratch(int dev, double** out) {
    std::lock_guard<std::mutex> lock(g_noalloc_mu);
    auto it = g_noalloc_addr.find(dev);
    if (it != g_noalloc_addr.end()) {
        *out = it->second;
        return GX_OK;
    }
    void* p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return fail_cuda(e, "cudaGetSymbolAddress (gx_direct_accel_noalloc scratch)");
    g_noalloc_addr[dev] = (double*)p;
    *out = (double*)p;
    return GX_OK;
}

}  // namespace

extern "C" int gx_direct_accel_noalloc(int64_t n, const double* x, const double* y, const double* z,
                                       const double* m, gx_physics phys, int precision, double* ax, double* ay,
                                       double* az, void* stream) {
    GX_GUARD_BEGIN
    const char* fn = "gx_direct_accel_noalloc";
    if (n < 0) return fail(GX_ERR_INVALID_ARGUMENT, "%s: n < 0", fn);
    if (n > kNoAllocMaxBodies)
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: n = %lld exceeds the fixed scratch limit of %lld bodies",
                    fn, (long long)n, (long long)kNoAllocMaxBodies);
    if (!valid_precision(precision)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: unknown precision %d", fn, precision);
    GX_TRY(check_phys(phys, fn));
    if (n > 0 && (!x || !y || !z || !m || !ax || !ay || !az)) return fail(GX_ERR_INVALID_ARGUMENT, "%s: null array", fn);
    GX_TRY(require_device());
    if (n == 0) return GX_OK;
    bool device;
    int dev;
    GX_TRY(classify({x, y, z, m, ax, ay, az}, &device, &dev, fn));
    if (!device)
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: device arrays only (host arrays would need staging buffers)", fn);
    DeviceGuard guard(dev);
    double* scratch = nullptr;
    GX_TRY(noalloc_scratch(dev, &scratch));
    int cnt;
    const ForceVariant* all = force_variants(&cnt);
    Choice ch = heuristic_choice(dev, precision, eps0_of(precision, phys), n, n);
    ch.nsplit = std::min(ch.nsplit, kNoAllocMaxSplit);
    const ForceVariant& v = all[ch.variant];
    ForceJob j{x, y, z, m, n, nullptr, 0, n, ax, ay, az, nullptr, nullptr, nullptr, 0.0};
    const ForceArgs a = make_args(j, phys, v, ch.nsplit, scratch);
    if ((size_t)a.nsplit * 3 * (size_t)n > kNoAllocScratchDoubles)
        return fail(GX_ERR_INVALID_ARGUMENT, "%s: partial sums exceed the fixed scratch array", fn);
    (void)cudaGetLastError();
    GX_CUDA(force_launch(v, a, (cudaStream_t)stream));
    return GX_OK;
    GX_GUARD_END
}
