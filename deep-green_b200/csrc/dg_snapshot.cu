// dg_snapshot.cu -- snapshots of a context's state: the groups save_to_disk
// writes (deep-green src/rs/src/io.rs:5-196) for the primitive and conserved
// fields, captured on the device and written to a self-describing binary file
// (HDF5 is not available to this library).
//
// Capture: the requested fields are packed on the device into the snapshot's
// own dense buffer (the primitives converted from the state at the start of
// the last step, the conserved state copied), in order on the context's
// stream; a copy stream then moves the buffer to pinned host memory.  The
// context may keep stepping at once: nothing the capture reads is touched by
// the next step, and the transfer reads only the snapshot's buffer.
//
// File: "DGSNAP01", a little-endian u64 header length, a JSON header, then the
// datasets, each starting on a 4096-byte boundary, raw C-order values.
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dg_ctx.h"

using namespace dg;

namespace {

thread_local std::string g_snap_err;   // the calling thread's last failure

int sfail(int code, const std::string &msg) {
    g_snap_err = msg;
    return code;
}

constexpr size_t kAlign = 4096;
constexpr const char *kPrimNames[5] = {"rho", "vx", "vy", "vz", "pressure"};
constexpr const char *kConsNames[5] = {"mass", "momentum_x", "momentum_y", "momentum_z", "energy"};

size_t round_up(size_t v) { return (v + kAlign - 1) / kAlign * kAlign; }

// JSON string literal of s (quotes and backslashes escaped).
std::string jstr(const char *s) {
    std::string o = "\"";
    for (const char *p = s; *p; ++p) {
        if (*p == '"' || *p == '\\') o += '\\';
        o += *p;
    }
    return o + "\"";
}

int write_file(const char *path, int dtype, const int32_t shape[3], int nfields, const char *const names[],
               const void *const data[], uint64_t steps, const char *attrs) {
    if (!path || !shape || !names || !data || nfields <= 0) return sfail(DG_ERR_INVALID, "null or empty argument");
    if (dtype != DG_F32 && dtype != DG_F64) return sfail(DG_ERR_INVALID, "dtype must be DG_F32 or DG_F64");
    for (int i = 0; i < 3; ++i)
        if (shape[i] <= 0) return sfail(DG_ERR_INVALID, "shape must be positive");
    const size_t elem = dtype == DG_F64 ? 8 : 4;
    const size_t bytes = (size_t)shape[0] * shape[1] * shape[2] * elem;
    // the header's length decides the first offset: size it with the widest
    // offsets, then pad it with spaces up to the data start
    auto header = [&](size_t first) {
        std::string h = "{\"format\": \"deep-green snapshot\", \"version\": 1, \"dtype\": ";
        h += dtype == DG_F64 ? "\"float64\"" : "\"float32\"";
        h += ", \"shape\": [" + std::to_string(shape[0]) + ", " + std::to_string(shape[1]) + ", " +
             std::to_string(shape[2]) + "], \"steps\": " + std::to_string(steps);
        if (attrs && *attrs) h += std::string(", \"attrs\": ") + attrs;
        h += ", \"datasets\": [";
        for (int i = 0; i < nfields; ++i) {
            if (!names[i] || !data[i]) return std::string();
            h += std::string(i ? ", " : "") + "{\"name\": " + jstr(names[i]) +
                 ", \"offset\": " + std::to_string(first + i * round_up(bytes)) +
                 ", \"nbytes\": " + std::to_string(bytes) + "}";
        }
        return h + "]}";
    };
    std::string h = header(1ull << 40);
    if (h.empty()) return sfail(DG_ERR_INVALID, "null dataset name or data");
    const size_t first = round_up(16 + h.size());
    h = header(first);
    h.resize(first - 16, ' ');
    FILE *f = std::fopen(path, "wb");
    if (!f) return sfail(DG_ERR_INVALID, std::string("cannot open ") + path);
    const uint64_t hl = h.size();
    bool ok = std::fwrite("DGSNAP01", 1, 8, f) == 8 && std::fwrite(&hl, 8, 1, f) == 1 &&
              std::fwrite(h.data(), 1, h.size(), f) == h.size();
    std::vector<char> pad(round_up(bytes) - bytes, 0);
    for (int i = 0; ok && i < nfields; ++i) {
        ok = std::fwrite(data[i], 1, bytes, f) == bytes;
        if (ok && i + 1 < nfields && !pad.empty()) ok = std::fwrite(pad.data(), 1, pad.size(), f) == pad.size();
    }
    ok = (std::fclose(f) == 0) && ok;
    if (!ok) return sfail(DG_ERR_INVALID, std::string("write failed: ") + path);
    return DG_OK;
}

}  // namespace

struct dg_snapshot {
    dg_ctx *ctx = nullptr;
    int device = 0;
    uint32_t groups = 0;
    int nfields = 0;
    size_t field_bytes = 0;
    void *dev = nullptr;              // dense fields, in file order
    void *host = nullptr;             // pinned copy
    cudaStream_t copy = nullptr;
    cudaEvent_t packed = nullptr, landed = nullptr;
    bool pending = false;
    uint64_t steps = 0;
    std::string attrs;
};

extern "C" {

int32_t dg_snapshot_write_host(const char *path, int32_t dtype, const int32_t shape[3], int32_t nfields,
                               const char *const names[], const void *const data[], uint64_t steps,
                               const char *attrs) {
    return write_file(path, dtype, shape, nfields, names, data, steps, attrs);
}

int32_t dg_snapshot_create(dg_ctx *c, uint32_t groups, dg_snapshot **out) {
    if (!c || !out) return sfail(DG_ERR_INVALID, "null argument");
    *out = nullptr;
    if (groups == 0 || (groups & ~(DG_SNAP_PRIMITIVES | DG_SNAP_CONSERVED)))
        return sfail(DG_ERR_INVALID, "groups must be a non-empty set of DG_SNAP_* bits");
    if (cudaSetDevice(c->info.device) != cudaSuccess) return sfail(DG_ERR_NO_DEVICE, "cannot select device");
    dg_snapshot *s = new dg_snapshot();
    s->ctx = c;
    s->device = c->info.device;
    s->groups = groups;
    s->nfields = 5 * (((groups & DG_SNAP_PRIMITIVES) ? 1 : 0) + ((groups & DG_SNAP_CONSERVED) ? 1 : 0));
    s->field_bytes = (size_t)c->nx * c->ny * c->nz * c->elem;
    const size_t total = s->field_bytes * s->nfields;
    cudaError_t e = cudaMalloc(&s->dev, total);
    if (e == cudaSuccess) e = cudaMallocHost(&s->host, total);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->packed, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->landed, cudaEventDisableTiming);
    if (e != cudaSuccess) {
        dg_snapshot_destroy(s);
        return sfail(DG_ERR_CUDA, std::string("snapshot allocation: ") + cudaGetErrorString(e));
    }
    char a[512];
    std::snprintf(a, sizeof a,
                  "{\"nghosts\": 2, \"ds\": %.17g, \"gamma\": %.17g, \"cfl\": %.17g, \"g\": %.17g, "
                  "\"bcs\": [%d, %d, %d, %d, %d, %d], \"limiter\": %d, \"gravity\": %d}",
                  c->info.ds, c->info.gamma, c->info.cfl, c->info.g, c->info.bcs[0], c->info.bcs[1], c->info.bcs[2],
                  c->info.bcs[3], c->info.bcs[4], c->info.bcs[5], c->info.limiter, c->info.gravity);
    s->attrs = a;
    *out = s;
    return DG_OK;
}

int32_t dg_snapshot_destroy(dg_snapshot *s) {
    if (!s) return DG_OK;
    cudaSetDevice(s->device);
    if (s->copy) cudaStreamSynchronize(s->copy);
    if (s->packed) cudaEventDestroy(s->packed);
    if (s->landed) cudaEventDestroy(s->landed);
    if (s->copy) cudaStreamDestroy(s->copy);
    cudaFree(s->dev);
    cudaFreeHost(s->host);
    delete s;
    return DG_OK;
}

int32_t dg_snapshot_begin(dg_snapshot *s) {
    if (!s) return sfail(DG_ERR_INVALID, "null argument");
    dg_ctx *c = s->ctx;
    if (!c->has_state) return sfail(DG_ERR_NO_STATE, "no state set");
    if (cudaSetDevice(c->info.device) != cudaSuccess) return sfail(DG_ERR_NO_DEVICE, "cannot select device");
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r, const char *where) {
        if (r != cudaSuccess && e == cudaSuccess) {
            e = r;
            g_snap_err = std::string(where) + ": " + cudaGetErrorString(r);
        }
        return r == cudaSuccess;
    };
    // the previous capture's transfer must have left the buffer
    if (!ok(cudaStreamWaitEvent(c->stream, s->landed, 0), "wait for the previous copy")) return DG_ERR_CUDA;
    char *dst = static_cast<char *>(s->dev);
    const long long dfs = (long long)c->nx * c->ny * c->nz;
    if (s->groups & DG_SNAP_PRIMITIVES) {
        // the state at the start of the last step, as dg_get_primitives
        const void *src = c->steps > 0 ? c->buf[1 - c->cur] : c->buf[c->cur];
        cudaError_t r;
        if (c->elem == 8) {
            r = launch_cons_to_prim_policy<double, true>(grid_args<double>(c, src, nullptr),
                                                         static_cast<const double *>(src),
                                                         reinterpret_cast<double *>(dst), dfs, c->nz, c->stream);
        } else {
            auto a = grid_args<float>(c, src, nullptr);
            r = c->exact ? launch_cons_to_prim_policy<float, true>(a, static_cast<const float *>(src),
                                                                   reinterpret_cast<float *>(dst), dfs, c->nz,
                                                                   c->stream)
                         : launch_cons_to_prim_policy<float, false>(a, static_cast<const float *>(src),
                                                                    reinterpret_cast<float *>(dst), dfs, c->nz,
                                                                    c->stream);
        }
        if (!ok(r, "snapshot primitives")) return DG_ERR_CUDA;
        dst += 5 * s->field_bytes;
    }
    if (s->groups & DG_SNAP_CONSERVED) {
        const size_t row = (size_t)c->nz * c->elem;
        for (int f = 0; f < 5; ++f) {
            const char *src = static_cast<const char *>(c->buf[c->cur]) + (size_t)f * c->fstride * c->elem;
            if (!ok(cudaMemcpy2DAsync(dst + f * s->field_bytes, row, src, (size_t)c->pitch * c->elem, row,
                                      (size_t)c->nx * c->ny, cudaMemcpyDeviceToDevice, c->stream),
                    "snapshot conserved"))
                return DG_ERR_CUDA;
        }
    }
    if (!ok(cudaEventRecord(s->packed, c->stream), "record") ||
        !ok(cudaStreamWaitEvent(s->copy, s->packed, 0), "copy stream wait") ||
        !ok(cudaMemcpyAsync(s->host, s->dev, s->field_bytes * s->nfields, cudaMemcpyDeviceToHost, s->copy),
            "device to host copy") ||
        !ok(cudaEventRecord(s->landed, s->copy), "record"))
        return DG_ERR_CUDA;
    s->steps = c->steps;
    s->pending = true;
    return DG_OK;
}

int32_t dg_snapshot_wait(dg_snapshot *s, const void **host) {
    if (!s) return sfail(DG_ERR_INVALID, "null argument");
    if (!s->pending) return sfail(DG_ERR_NO_STATE, "no snapshot begun");
    if (cudaSetDevice(s->device) != cudaSuccess) return sfail(DG_ERR_NO_DEVICE, "cannot select device");
    const cudaError_t e = cudaEventSynchronize(s->landed);
    if (e != cudaSuccess) return sfail(DG_ERR_CUDA, std::string("snapshot copy: ") + cudaGetErrorString(e));
    if (host) *host = s->host;
    return DG_OK;
}

int32_t dg_snapshot_write(dg_snapshot *s, const char *path) {
    if (!s || !path) return sfail(DG_ERR_INVALID, "null argument");
    int r = dg_snapshot_wait(s, nullptr);
    if (r != DG_OK) return r;
    std::string full[10];
    const char *names[10];
    const void *data[10];
    int n = 0;
    const char *base = static_cast<const char *>(s->host);
    if (s->groups & DG_SNAP_PRIMITIVES)
        for (int f = 0; f < 5; ++f, ++n) {
            full[n] = std::string("primitives/") + kPrimNames[f];
            names[n] = full[n].c_str();
            data[n] = base + n * s->field_bytes;
        }
    if (s->groups & DG_SNAP_CONSERVED)
        for (int f = 0; f < 5; ++f, ++n) {
            full[n] = std::string("conserved/") + kConsNames[f];
            names[n] = full[n].c_str();
            data[n] = base + n * s->field_bytes;
        }
    const dg_ctx *c = s->ctx;
    const int32_t shape[3] = {c->nx, c->ny, c->nz};
    return write_file(path, c->elem == 8 ? DG_F64 : DG_F32, shape, n, names, data, s->steps, s->attrs.c_str());
}

// Message of the last failed snapshot call (all snapshots share it).
const char *dg_snapshot_last_error(const dg_snapshot *) { return g_snap_err.c_str(); }

}  // extern "C"
