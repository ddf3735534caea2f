// snapshot.cu -- snapshot and diagnostics output of the reference's SnapshotWriter
// (cpp/io/snapshot_writer.cpp:38-128), taken asynchronously from device-resident state.
//
// CSV text is the reference's byte for byte: `std::setprecision(17)` on a default-format
// stream prints a double as printf's "%.17g" (libstdc++ formats through vsnprintf with
// "%.*g"), integers as decimal; rows "id,group_id,mass,x,y,z,vx,vy,vz,ax,ay,az" after a
// "# time=" line; file names snapshot_%06d.csv; diagnostics.csv starts with the reference's
// header and gains one row per gx_snapshot_write_diagnostics call.  The binary form is this
// engine's own: snapshot_%06d.bin = 8-byte magic "GXSNAP01", int64 n, int32 step, int32
// field count (10), double time, then x, y, z, vx, vy, vz, ax, ay, az, m (n doubles each,
// little-endian) and the group ids (n uint32).
//
// A device snapshot costs the caller's stream one device-to-device copy of the state into a
// slot (80 B/body, ~30 us at N = 2^20); the slot then goes to pinned host memory on the
// writer's own stream, and a writer thread formats and writes it while the caller's stream
// keeps stepping.  Calls block only when every slot is still in flight.
#include "gx.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <filesystem>
#include <mutex>
#include <new>
#include <string>
#include <thread>
#include <vector>

extern "C" int gxi_fail(int code, const char* msg);

namespace {

constexpr int kFields = 10;  // x, y, z, vx, vy, vz, ax, ay, az, m

struct Slot {
    std::vector<double> host;  // host-array snapshots
    double* pinned = nullptr;  // device snapshots: kFields * n doubles
    double* dev = nullptr;
    cudaEvent_t landed = nullptr;
    bool from_device = false;
    int step = 0;
    double time = 0.0;
    const double* data() const { return from_device ? pinned : host.data(); }
};

bool is_device_pointer(const void* p, int* dev) {
    if (!p) return false;
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();  // no device or unknown pointer: host memory
        return false;
    }
    if (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged) {
        *dev = at.device;
        return true;
    }
    return false;
}

size_t format_row(char* p, size_t cap, size_t i, uint32_t g, const double* const* f, int64_t k) {
    const int w = std::snprintf(p, cap, "%zu,%u,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g\n", i, g,
                                f[9][k], f[0][k], f[1][k], f[2][k], f[3][k], f[4][k], f[5][k], f[6][k], f[7][k],
                                f[8][k]);
    return w > 0 ? (size_t)w : 0;
}

}  // namespace

struct gx_snapshot_writer {
    std::filesystem::path dir;
    int64_t n = 0;
    std::vector<uint32_t> group;
    int formats = 0;
    int device = -1;
    cudaStream_t side = nullptr;
    std::vector<Slot> slots;
    std::deque<int> free_slots, queue;
    std::mutex mu;
    std::condition_variable cv;
    std::thread worker;
    bool stop = false;
    int busy = 0;  // slots handed to the worker and not yet written
    int error = GX_OK;
    std::string error_msg;
    std::mutex diag_mu;
    FILE* diag = nullptr;

    void fail_write(const std::string& msg) {
        std::lock_guard<std::mutex> l(mu);
        if (error == GX_OK) {
            error = GX_ERR_INVALID_ARGUMENT;
            error_msg = msg;
        }
    }

    void write_csv(const Slot& s) {
        char name[64];
        std::snprintf(name, sizeof name, "snapshot_%06d.csv", s.step);
        const std::string path = (dir / name).string();
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) return fail_write("could not write " + path);
        std::fprintf(f, "# time=%.17g\nid,group_id,mass,x,y,z,vx,vy,vz,ax,ay,az\n", s.time);
        const double* base = s.data();
        const double* fld[kFields];
        for (int k = 0; k < kFields; ++k) fld[k] = base + (size_t)k * n;
        // rows formatted in parallel chunks, written in order
        const int nt = (int)std::max<int64_t>(1, std::min<int64_t>({16, (int64_t)std::thread::hardware_concurrency(),
                                                                    (n + 4095) / 4096}));
        std::vector<std::string> out((size_t)nt);
        auto work = [&](int t) {
            const int64_t b = n * t / nt, e = n * (t + 1) / nt;
            std::string& o = out[(size_t)t];
            o.resize((size_t)(e - b) * 280);
            size_t at = 0;
            char row[320];
            for (int64_t k = b; k < e; ++k) {
                const size_t w = format_row(row, sizeof row, (size_t)k, group.empty() ? 0u : group[(size_t)k], fld, k);
                if (at + w > o.size()) o.resize(o.size() * 2 + w);
                std::memcpy(&o[at], row, w);
                at += w;
            }
            o.resize(at);
        };
        std::vector<std::thread> pool;
        for (int t = 1; t < nt; ++t) pool.emplace_back(work, t);
        work(0);
        for (auto& th : pool) th.join();
        bool ok = true;
        for (const auto& o : out) ok = ok && std::fwrite(o.data(), 1, o.size(), f) == o.size();
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) fail_write("short write to " + path);
    }

    void write_binary(const Slot& s) {
        char name[64];
        std::snprintf(name, sizeof name, "snapshot_%06d.bin", s.step);
        const std::string path = (dir / name).string();
        FILE* f = std::fopen(path.c_str(), "wb");
        if (!f) return fail_write("could not write " + path);
        const char magic[8] = {'G', 'X', 'S', 'N', 'A', 'P', '0', '1'};
        const int64_t nn = n;
        const int32_t step = s.step, fields = kFields;
        bool ok = std::fwrite(magic, 1, 8, f) == 8 && std::fwrite(&nn, 8, 1, f) == 1 && std::fwrite(&step, 4, 1, f) == 1 &&
                  std::fwrite(&fields, 4, 1, f) == 1 && std::fwrite(&s.time, 8, 1, f) == 1;
        ok = ok && std::fwrite(s.data(), sizeof(double), (size_t)kFields * n, f) == (size_t)kFields * n;
        std::vector<uint32_t> g0;
        const uint32_t* g = group.data();
        if (group.empty()) {
            g0.assign((size_t)n, 0u);
            g = g0.data();
        }
        ok = ok && std::fwrite(g, 4, (size_t)n, f) == (size_t)n;
        ok = (std::fclose(f) == 0) && ok;
        if (!ok) fail_write("short write to " + path);
    }

    void run() {
        if (device >= 0) cudaSetDevice(device);
        for (;;) {
            int k;
            {
                std::unique_lock<std::mutex> l(mu);
                cv.wait(l, [&] { return stop || !queue.empty(); });
                if (queue.empty()) return;
                k = queue.front();
                queue.pop_front();
            }
            Slot& s = slots[(size_t)k];
            bool ok = true;
            if (s.from_device && cudaEventSynchronize(s.landed) != cudaSuccess) {
                cudaGetLastError();
                fail_write("snapshot copy from the device failed");
                ok = false;
            }
            if (ok && (formats & GX_SNAPSHOT_CSV)) write_csv(s);
            if (ok && (formats & GX_SNAPSHOT_BINARY)) write_binary(s);
            {
                std::lock_guard<std::mutex> l(mu);
                free_slots.push_back(k);
                --busy;
            }
            cv.notify_all();
        }
    }

    int acquire() {
        std::unique_lock<std::mutex> l(mu);
        cv.wait(l, [&] { return !free_slots.empty(); });
        const int k = free_slots.front();
        free_slots.pop_front();
        return k;
    }

    void hand_over(int k) {
        {
            std::lock_guard<std::mutex> l(mu);
            queue.push_back(k);
            ++busy;
        }
        cv.notify_all();
    }

    int release_unused(int k, int rc) {
        {
            std::lock_guard<std::mutex> l(mu);
            free_slots.push_front(k);
        }
        cv.notify_all();
        return rc;
    }
};

extern "C" int gx_snapshot_writer_create(const char* directory, int64_t n, const uint32_t* group_id, int formats,
                                         int slots, gx_snapshot_writer** out) {
    if (!out) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_writer_create: out is null");
    *out = nullptr;
    if (!directory || n < 0 || slots < 1 || (formats & ~(GX_SNAPSHOT_CSV | GX_SNAPSHOT_BINARY)) || !formats)
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_writer_create: bad arguments");
    gx_snapshot_writer* w = new (std::nothrow) gx_snapshot_writer();
    if (!w) return gxi_fail(GX_ERR_OUT_OF_MEMORY, "gx_snapshot_writer_create: host allocation failed");
    try {
        w->dir = directory;
        w->n = n;
        w->formats = formats;
        if (group_id) w->group.assign(group_id, group_id + n);
        std::error_code ec;
        std::filesystem::create_directories(w->dir, ec);
        if (ec) {
            delete w;
            return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_writer_create: could not create the directory");
        }
        if (formats & GX_SNAPSHOT_CSV) {
            // SnapshotWriter constructor (snapshot_writer.cpp:38-57)
            w->diag = std::fopen((w->dir / "diagnostics.csv").string().c_str(), "wb");
            if (!w->diag) {
                delete w;
                return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_writer_create: could not open diagnostics.csv");
            }
            std::fputs("step,time,n,total_mass,kinetic_energy,potential_energy,total_energy,"
                       "momentum_x,momentum_y,momentum_z,"
                       "center_of_mass_x,center_of_mass_y,center_of_mass_z,"
                       "angular_momentum_x,angular_momentum_y,angular_momentum_z\n",
                       w->diag);
            std::fflush(w->diag);
        }
        w->slots.resize((size_t)slots);
        for (int k = 0; k < slots; ++k) w->free_slots.push_back(k);
        w->worker = std::thread([w] { w->run(); });
    } catch (const std::exception&) {
        delete w;
        return gxi_fail(GX_ERR_OUT_OF_MEMORY, "gx_snapshot_writer_create: host allocation failed");
    }
    *out = w;
    return GX_OK;
}

extern "C" int gx_snapshot_writer_flush(gx_snapshot_writer* w) {
    if (!w) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_writer_flush: null writer");
    std::string msg;
    int rc;
    {
        std::unique_lock<std::mutex> l(w->mu);
        w->cv.wait(l, [&] { return w->busy == 0; });
        rc = w->error;
        msg = w->error_msg;
    }
    if (w->diag) {
        std::lock_guard<std::mutex> l(w->diag_mu);
        std::fflush(w->diag);
    }
    return rc == GX_OK ? GX_OK : gxi_fail(rc, ("snapshot output: " + msg).c_str());
}

extern "C" int gx_snapshot_writer_destroy(gx_snapshot_writer* w) {
    if (!w) return GX_OK;
    const int rc = gx_snapshot_writer_flush(w);
    {
        std::lock_guard<std::mutex> l(w->mu);
        w->stop = true;
    }
    w->cv.notify_all();
    if (w->worker.joinable()) w->worker.join();
    if (w->device >= 0) cudaSetDevice(w->device);
    for (Slot& s : w->slots) {
        if (s.pinned) cudaFreeHost(s.pinned);
        if (s.dev) cudaFree(s.dev);
        if (s.landed) cudaEventDestroy(s.landed);
    }
    if (w->side) cudaStreamDestroy(w->side);
    if (w->diag) std::fclose(w->diag);
    cudaGetLastError();
    delete w;
    return rc;
}

extern "C" int gx_snapshot_write(gx_snapshot_writer* w, int step, double time, const double* x, const double* y,
                                 const double* z, const double* vx, const double* vy, const double* vz,
                                 const double* ax, const double* ay, const double* az, const double* m,
                                 void* stream) {
    if (!w) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write: null writer");
    const double* src[kFields] = {x, y, z, vx, vy, vz, ax, ay, az, m};
    for (const double* p : src)
        if (!p && w->n > 0) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write: null array");
    int dev = -1, kinds = 0;
    for (const double* p : src) {
        int d = -1;
        if (is_device_pointer(p, &d)) {
            if (dev >= 0 && d != dev)
                return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write: arrays on different devices");
            dev = d;
            ++kinds;
        }
    }
    if (kinds != 0 && kinds != kFields)
        return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write: mix of host and device arrays");
    const size_t bytes = (size_t)w->n * sizeof(double);
    const int k = w->acquire();
    Slot& s = w->slots[(size_t)k];
    s.step = step;
    s.time = time;
    if (kinds == 0) {
        s.from_device = false;
        try {
            s.host.resize((size_t)kFields * w->n);
        } catch (const std::exception&) {
            return w->release_unused(k, gxi_fail(GX_ERR_OUT_OF_MEMORY, "gx_snapshot_write: host allocation failed"));
        }
        for (int f = 0; f < kFields; ++f)
            if (bytes) std::memcpy(s.host.data() + (size_t)f * w->n, src[f], bytes);
        w->hand_over(k);
        return GX_OK;
    }
    if (w->device >= 0 && w->device != dev)
        return w->release_unused(k, gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write: writer bound to another device"));
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(dev);
    auto cuda_fail = [&](cudaError_t e, const char* what) {
        cudaGetLastError();
        cudaSetDevice(prev);
        return w->release_unused(k, gxi_fail(GX_ERR_CUDA, (std::string(what) + ": " + cudaGetErrorString(e)).c_str()));
    };
    cudaError_t e;
    if (w->device < 0) {
        if ((e = cudaStreamCreateWithFlags(&w->side, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(e, "gx_snapshot_write: stream");
        w->device = dev;
    }
    // each resource of the slot is made on its own, so a failed attempt leaves the slot
    // usable: the next write that gets it retries what is still missing
    if (!s.dev) {
        if ((e = cudaMalloc(&s.dev, (size_t)kFields * bytes + 16)) != cudaSuccess) {
            s.dev = nullptr;
            return cuda_fail(e, "gx_snapshot_write");
        }
    }
    if (!s.pinned) {
        if ((e = cudaMallocHost(&s.pinned, (size_t)kFields * bytes + 16)) != cudaSuccess) {
            s.pinned = nullptr;
            return cuda_fail(e, "gx_snapshot_write");
        }
    }
    if (!s.landed) {
        if ((e = cudaEventCreateWithFlags(&s.landed, cudaEventDisableTiming)) != cudaSuccess) {
            s.landed = nullptr;
            return cuda_fail(e, "gx_snapshot_write");
        }
    }
    s.from_device = true;
    cudaStream_t st = (cudaStream_t)stream;
    for (int f = 0; f < kFields; ++f)
        if (bytes && (e = cudaMemcpyAsync(s.dev + (size_t)f * w->n, src[f], bytes, cudaMemcpyDeviceToDevice, st)) != cudaSuccess)
            return cuda_fail(e, "gx_snapshot_write: device copy");
    // the writer's stream takes the copy to the host once the caller's stream has made it
    if ((e = cudaEventRecord(s.landed, st)) != cudaSuccess) return cuda_fail(e, "gx_snapshot_write");
    if ((e = cudaStreamWaitEvent(w->side, s.landed, 0)) != cudaSuccess) return cuda_fail(e, "gx_snapshot_write");
    if (bytes && (e = cudaMemcpyAsync(s.pinned, s.dev, (size_t)kFields * bytes, cudaMemcpyDeviceToHost, w->side)) != cudaSuccess)
        return cuda_fail(e, "gx_snapshot_write: host copy");
    if ((e = cudaEventRecord(s.landed, w->side)) != cudaSuccess) return cuda_fail(e, "gx_snapshot_write");
    cudaSetDevice(prev);
    w->hand_over(k);
    return GX_OK;
}

extern "C" int gx_snapshot_write_diagnostics(gx_snapshot_writer* w, int step, double time, const gx_diagnostics* d) {
    if (!w || !d) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write_diagnostics: null argument");
    if (!w->diag) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write_diagnostics: the writer has no CSV output");
    std::lock_guard<std::mutex> l(w->diag_mu);
    // write_diagnostics (snapshot_writer.cpp:99-128)
    const int r = std::fprintf(w->diag,
                               "%d,%.17g,%lld,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,%.17g,"
                               "%.17g,%.17g\n",
                               step, time, (long long)w->n, d->total_mass, d->kinetic_energy, d->potential_energy,
                               d->total_energy, d->momentum[0], d->momentum[1], d->momentum[2], d->center_of_mass[0],
                               d->center_of_mass[1], d->center_of_mass[2], d->angular_momentum[0],
                               d->angular_momentum[1], d->angular_momentum[2]);
    return r > 0 ? GX_OK : gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write_diagnostics: write failed");
}

// write_metadata (snapshot_writer.cpp:49-69).  The reference streams doubles with the
// ostream defaults (no precision set on that stream): "%g", six significant digits.
extern "C" int gx_snapshot_write_metadata(gx_snapshot_writer* w, const gx_run_metadata* md) {
    if (!w || !md) return gxi_fail(GX_ERR_INVALID_ARGUMENT, "gx_snapshot_write_metadata: null argument");
    auto esc = [](const char* s) {
        std::string e;
        for (const char* p = s ? s : ""; *p; ++p) {
            if (*p == '"' || *p == '\\') e.push_back('\\');
            e.push_back(*p);
        }
        return e;
    };
    const std::filesystem::path path = w->dir / "metadata.json";
    FILE* f = std::fopen(path.string().c_str(), "w");
    if (!f) return gxi_fail(GX_ERR_INVALID_ARGUMENT, ("could not write " + path.string()).c_str());
    const int r = std::fprintf(f,
                               "{\n"
                               "  \"name\": \"%s\",\n"
                               "  \"solver\": \"%s\",\n"
                               "  \"particle_count\": %lld,\n"
                               "  \"steps\": %d,\n"
                               "  \"dt\": %g,\n"
                               "  \"snapshot_every\": %d,\n"
                               "  \"dim\": %d,\n"
                               "  \"gravitational_constant\": %g,\n"
                               "  \"softening\": %g,\n"
                               "  \"tree_theta\": %g,\n"
                               "  \"tree_leaf_capacity\": %lld,\n"
                               "  \"fmm_expansion_order\": %d\n"
                               "}\n",
                               esc(md->name).c_str(), esc(md->solver).c_str(), (long long)md->particle_count,
                               (int)md->steps, md->dt, (int)md->snapshot_every, (int)md->dim,
                               md->gravitational_constant, md->softening, md->tree_theta,
                               (long long)md->tree_leaf_capacity, (int)md->fmm_expansion_order);
    const bool ok = r > 0 && std::fclose(f) == 0;
    return ok ? GX_OK : gxi_fail(GX_ERR_INVALID_ARGUMENT, ("write failed: " + path.string()).c_str());
}
