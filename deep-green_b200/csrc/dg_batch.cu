// dg_batch.cu -- many independent grids advanced together: one persistent
// launch per step (work items of every grid from one queue), per-grid CFL
// dt, steps replayed from a captured CUDA graph, and an autotuner that picks
// the tile shape (rows per tile) and x-planes per work item by timing the
// live batch.
//
// The reference advances one grid per compute_step call
// (src/rs/src/physics.rs:595-681); a batch is N such grids whose steps are
// independent (nothing is exchanged between grids).
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "../../include/deepgreen.h"
#include "dg_host.h"
#include "dg_kernels.cuh"
#include "dg_sweep_impl.cuh"

using namespace dg;
using sweep::BatchItem;

namespace {

constexpr int kTY = kSweepRowsF32;   // tile rows of the batched sweep
constexpr int kRing = sizeof(sweep::Smem<float, kTY, 5>) + 1024 <= 232448 ? 5 : 4;
constexpr int kTZs = sweep::kTileZ;  // tile columns
constexpr int kCombos = 4;           // (limiter, gravity) pairs; one launch each

int combo_of(const dg_sim_info &f) { return (f.limiter ? 1 : 0) + (f.gravity ? 2 : 0); }

struct GridSlot {
    dg_sim_info info;        // as stored: sizes and boundaries along the stored axes
    int perm[3];             // stored axis d is the caller's axis perm[d]
    int cn[3];               // the caller's ghosted sizes (x, y, z)
    int nx, ny, nz, pitch;
    long long fstride;
    size_t state_bytes;
    void *buf[2];
    int nitems, item_off;
};

}  // namespace

struct dg_batch {
    int n = 0;
    int device = 0;
    std::vector<GridSlot> g;
    void *arena = nullptr;           // all state buffers
    DevCtl *ctl = nullptr;           // one control block per grid
    Partial *part = nullptr;         // per work item (and set-up reductions)
    size_t part_cap = 0;
    GridArgs<float> *d_args[2] = {nullptr, nullptr};   // [parity]: src = buf[parity]
    CUtensorMap *d_maps[2] = {nullptr, nullptr};
    BatchItem *d_items = nullptr;
    size_t items_cap = 0;
    int nitems = 0;
    int combo_off[kCombos + 1] = {0, 0, 0, 0, 0};   // items of each (limiter, gravity) pair
    unsigned *d_queue = nullptr;     // one counter per pair
    int tile_rows = kTY;
    int chunk = 0;                   // x-planes per work item (0 = automatic)
    int chunk_used = 0;
    unsigned long long steps = 0;    // steps since the states were set
    cudaStream_t stream = nullptr;
    cudaGraphExec_t graph = nullptr;
    bool dirty = true;               // items / descriptors must be rebuilt
    std::string err;
};

namespace {

int bfail(dg_batch *b, int code, const std::string &m) {
    if (b) b->err = m;
    else set_global_error(m);
    return code;
}

#define B_CUDA(b, expr)                                                                         \
    do {                                                                                        \
        cudaError_t e_ = (expr);                                                                \
        if (e_ != cudaSuccess) return bfail((b), DG_ERR_CUDA, std::string(#expr) + ": " + cudaGetErrorString(e_)); \
    } while (0)

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

GridArgs<float> args_of(const dg_batch *b, int i, int parity) {
    const GridSlot &s = b->g[i];
    GridArgs<float> a;
    std::memset(&a, 0, sizeof(a));
    a.src = static_cast<const float *>(s.buf[parity]);
    a.dst = static_cast<float *>(s.buf[1 - parity]);
    a.nx = s.nx;
    a.ny = s.ny;
    a.nz = s.nz;
    a.pitch = s.pitch;
    a.fstride = s.fstride;
    set_boundaries(a, s.info.bcs);
    a.gravity = s.info.gravity;
    a.limiter = s.info.limiter;
    a.nparts = s.nitems;
    const float ds = (float)s.info.ds;
    a.k.ds = ds;
    a.k.vol = ds * ds * ds;
    a.k.inv_vol = 1.0f / a.k.vol;
    a.k.gamma = (float)s.info.gamma;
    a.k.gm1 = a.k.gamma - 1.0f;
    a.k.inv_gm1 = 1.0f / a.k.gm1;
    a.k.half_ds = ds / 2.0f;
    a.k.two_ds = 2.0f * ds;
    a.k.inv_ds = 1.0f / ds;
    a.k.inv_2ds = 1.0f / (2.0f * ds);
    a.k.cfl = (float)s.info.cfl;
    a.k.g = (float)s.info.g;
    a.ctl = b->ctl + i;
    a.part = b->part + s.item_off;
    return a;
}

// Work items, per-grid arguments and TMA descriptors for the current tiling.
int rebuild(dg_batch *b) {
    auto fn = encode_fn();
    if (!fn) return bfail(b, DG_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
    const int ty = b->tile_rows;
    // x-planes per item: as for one grid, sized on the batch's total tiles
    long long tiles_total = 0;
    int min_nx = 1 << 30;
    for (auto &s : b->g) {
        tiles_total += (long long)((s.ny - 4 + ty - 1) / ty) * ((s.nz - 4 + kTZs - 1) / kTZs);
        min_nx = std::min(min_nx, s.nx - 4);
    }
    int chunk = b->chunk;
    if (chunk <= 0) {
        long long cells = 0;
        for (auto &s : b->g) cells += (long long)(s.nx - 4) * (s.ny - 4) * (s.nz - 4);
        // ~8 waves of one block per SM worth of items, at least 16 planes
        const long long items_target = (long long)kSms * 8;
        const long long tile_cells = (long long)ty * kTZs;
        long long c = cells / std::max<long long>(1, items_target * tile_cells);
        chunk = (int)std::max<long long>(16, c);
    }
    b->chunk_used = chunk;
    // items: grouped by (limiter, gravity), largest grids first, each grid's
    // items contiguous
    std::vector<int> order(b->n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int x, int y) {
        const int cx = combo_of(b->g[x].info), cy = combo_of(b->g[y].info);
        if (cx != cy) return cx < cy;
        auto sz = [&](int i) { return (long long)b->g[i].nx * b->g[i].ny * b->g[i].nz; };
        return sz(x) > sz(y);
    });
    std::vector<BatchItem> items;
    int off = 0;
    for (int c = 0; c <= kCombos; ++c) b->combo_off[c] = 0;
    for (int i : order) {
        GridSlot &s = b->g[i];
        const int tz_n = (s.nz - 4 + kTZs - 1) / kTZs, ty_n = (s.ny - 4 + ty - 1) / ty;
        const int cx_n = (s.nx - 4 + chunk - 1) / chunk;
        s.item_off = off;
        s.nitems = tz_n * ty_n * cx_n;
        int local = 0;
        for (int cx = 0; cx < cx_n; ++cx)
            for (int yy = 0; yy < ty_n; ++yy)
                for (int zz = 0; zz < tz_n; ++zz) items.push_back(BatchItem{i, local++, zz, yy, cx});
        off += s.nitems;
        b->combo_off[combo_of(s.info) + 1] = off;
    }
    for (int c = 1; c <= kCombos; ++c) b->combo_off[c] = std::max(b->combo_off[c], b->combo_off[c - 1]);
    b->nitems = (int)items.size();
    if ((size_t)b->nitems > b->items_cap) {
        if (b->d_items) cudaFree(b->d_items);
        b->items_cap = (size_t)b->nitems;
        B_CUDA(b, cudaMalloc(&b->d_items, b->items_cap * sizeof(BatchItem)));
    }
    if ((size_t)std::max(b->nitems, kReduceBlocks) > b->part_cap) {
        if (b->part) cudaFree(b->part);
        b->part_cap = (size_t)std::max(b->nitems, kReduceBlocks);
        B_CUDA(b, cudaMalloc(&b->part, b->part_cap * sizeof(Partial)));
    }
    B_CUDA(b, cudaMemcpyAsync(b->d_items, items.data(), items.size() * sizeof(BatchItem), cudaMemcpyHostToDevice,
                              b->stream));
    for (int p = 0; p < 2; ++p) {
        std::vector<GridArgs<float>> args(b->n);
        std::vector<CUtensorMap> maps(b->n);
        for (int i = 0; i < b->n; ++i) {
            args[i] = args_of(b, i, p);
            const GridSlot &s = b->g[i];
            cuuint64_t dims[4] = {(cuuint64_t)s.nz, (cuuint64_t)s.ny, (cuuint64_t)s.nx, 5};
            cuuint64_t strides[3] = {(cuuint64_t)s.pitch * 4, (cuuint64_t)s.pitch * s.ny * 4,
                                     (cuuint64_t)s.fstride * 4};
            cuuint32_t box[4] = {(cuuint32_t)(kTZs + 4), (cuuint32_t)(ty + 4), 1, 5};
            cuuint32_t estr[4] = {1, 1, 1, 1};
            if (fn(&maps[i], CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, s.buf[p], dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
                return bfail(b, DG_ERR_CUDA, "cuTensorMapEncodeTiled failed for grid " + std::to_string(i));
        }
        B_CUDA(b, cudaMemcpyAsync(b->d_args[p], args.data(), b->n * sizeof(GridArgs<float>), cudaMemcpyHostToDevice,
                                  b->stream));
        B_CUDA(b, cudaMemcpyAsync(b->d_maps[p], maps.data(), b->n * sizeof(CUtensorMap), cudaMemcpyHostToDevice,
                                  b->stream));
    }
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    if (b->graph) {
        cudaGraphExecDestroy(b->graph);
        b->graph = nullptr;
    }
    b->dirty = false;
    return DG_OK;
}

constexpr int kSmem = sweep::smem_bytes<float, kTY, kRing>();

template <int LIM, bool GRAV> cudaError_t prepare_kernel() {
    static std::atomic<unsigned long long> done{0};
    return ensure_dynamic_smem(sweep::sweep_batch_kernel<kTY, kRing, LIM, GRAV>, kSmem, done);
}

template <int LIM, bool GRAV> void launch_combo(dg_batch *b, int parity, int c) {
    const int n = b->combo_off[c + 1] - b->combo_off[c];
    sweep::sweep_batch_kernel<kTY, kRing, LIM, GRAV><<<std::min(n, kSms), 32 * (kTY + 2), kSmem, b->stream>>>(
        b->d_args[parity], b->d_maps[parity], b->d_items + b->combo_off[c], n, b->d_queue + c, b->chunk_used);
}

// one step of every grid (no synchronisation): one persistent launch per
// (limiter, gravity) pair present in the batch
int launch_one(dg_batch *b, int parity) {
    B_CUDA(b, cudaMemsetAsync(b->d_queue, 0, kCombos * sizeof(unsigned), b->stream));
    for (int c = 0; c < kCombos; ++c) {
        if (b->combo_off[c + 1] == b->combo_off[c]) continue;
        switch (c) {
            case 0: launch_combo<0, false>(b, parity, c); break;
            case 1: launch_combo<1, false>(b, parity, c); break;
            case 2: launch_combo<0, true>(b, parity, c); break;
            default: launch_combo<1, true>(b, parity, c); break;
        }
        B_CUDA(b, cudaGetLastError());
    }
    return DG_OK;
}

int enqueue(dg_batch *b, int nsteps) {
    int r;
    if (b->dirty && (r = rebuild(b)) != DG_OK) return r;
    int done = 0;
    if (nsteps > 0 && (b->steps & 1)) {   // graph below starts from parity 0
        if ((r = launch_one(b, 1)) != DG_OK) return r;
        ++b->steps;
        ++done;
    }
    if (nsteps - done >= 2 && !b->graph) {
        cudaGraph_t g;
        B_CUDA(b, cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
        int r0 = launch_one(b, 0);
        int r1 = r0 == DG_OK ? launch_one(b, 1) : r0;
        const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
        if (r0 != DG_OK || r1 != DG_OK) return r0 != DG_OK ? r0 : r1;
        B_CUDA(b, ce);
        const cudaError_t ie = cudaGraphInstantiate(&b->graph, g, 0);
        cudaGraphDestroy(g);
        B_CUDA(b, ie);
    }
    while (nsteps - done >= 2) {
        B_CUDA(b, cudaGraphLaunch(b->graph, b->stream));
        b->steps += 2;
        done += 2;
    }
    if (done < nsteps) {
        if ((r = launch_one(b, (int)(b->steps & 1))) != DG_OK) return r;
        ++b->steps;
    }
    return DG_OK;
}

int check_timeouts(dg_batch *b) {
    for (int i = 0; i < b->n; ++i) {
        unsigned f = 0;
        B_CUDA(b, cudaMemcpyAsync(&f, &b->ctl[i].flags, sizeof(f), cudaMemcpyDeviceToHost, b->stream));
        B_CUDA(b, cudaStreamSynchronize(b->stream));
        if (f & kStatusTimeout) return bfail(b, DG_ERR_TIMEOUT, "a device-side wait timed out in grid " + std::to_string(i));
    }
    return DG_OK;
}

}  // namespace

namespace {

// Orientation of a grid stored with DG_BATCH_REORIENT: the axis order
// (stored x, y, z = caller axes perm[0..2]) with the fewest padded cells --
// z widths round up to the tile's 64 columns, y to its rows, x not at all
// (charging short x axes for the planes a work item re-stages measured
// slower on the batch64 workload) -- z kept in place for a grid with
// gravity (it acts along z).  Ties keep the caller's order.
void choose_orientation(const dg_sim_info &f, bool reorient, int perm[3]) {
    perm[0] = 0; perm[1] = 1; perm[2] = 2;
    if (!reorient) return;
    const long long n[3] = {f.nx, f.ny, f.nz};
    auto cost = [&](const int p[3]) {
        const long long y = (n[p[1]] + kTY - 1) / kTY * kTY, z = (n[p[2]] + kTZs - 1) / kTZs * kTZs;
        return n[p[0]] * y * z;
    };
    static const int perms[6][3] = {{0, 1, 2}, {1, 0, 2}, {0, 2, 1}, {2, 0, 1}, {1, 2, 0}, {2, 1, 0}};
    long long best = cost(perm);
    for (const auto &p : perms) {
        if (f.gravity && p[2] != 2) continue;
        const long long c = cost(p);
        if (c < best) { best = c; perm[0] = p[0]; perm[1] = p[1]; perm[2] = p[2]; }
    }
}

// Copies 5 fields between the caller's layout (dense, ghosted sizes cn,
// velocity / momentum components along the caller's axes) and the stored
// one (pitched, axes permuted by perm, components likewise).  TO_STORED:
// caller -> stored; else stored -> caller.  One thread per destination cell.
template <bool TO_STORED>
__global__ void permute_fields(const float *src, float *dst, int cn0, int cn1, int cn2, int p0, int p1, int p2,
                               int pitch, long long fstride) {
    const int cn[3] = {cn0, cn1, cn2}, p[3] = {p0, p1, p2};
    const long long ncaller = (long long)cn0 * cn1 * cn2;
    const int sn0 = cn[p0], sn1 = cn[p1], sn2 = cn[p2];
    const long long nstored = (long long)sn0 * sn1 * sn2;
    const long long total = TO_STORED ? nstored : ncaller;
    for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < 5 * total;
         t += (long long)gridDim.x * blockDim.x) {
        const int f = (int)(t / total);
        const long long c = t % total;
        int s[3], q[3];   // stored and caller coordinates
        if (TO_STORED) {
            s[2] = (int)(c % sn2);
            s[1] = (int)(c / sn2 % sn1);
            s[0] = (int)(c / ((long long)sn2 * sn1));
            for (int d = 0; d < 3; ++d) q[p[d]] = s[d];
        } else {
            q[2] = (int)(c % cn2);
            q[1] = (int)(c / cn2 % cn1);
            q[0] = (int)(c / ((long long)cn2 * cn1));
            for (int d = 0; d < 3; ++d) s[d] = q[p[d]];
        }
        // stored component 1 + d is the caller's component 1 + p[d]
        const int fs = f, fc = (f >= 1 && f <= 3) ? 1 + p[f - 1] : f;
        const long long ci = ((long long)q[0] * cn1 + q[1]) * cn2 + q[2];
        const long long si = ((long long)s[0] * sn1 + s[1]) * pitch + s[2];
        if (TO_STORED) dst[fs * fstride + si] = src[fc * ncaller + ci];
        else dst[fc * ncaller + ci] = src[fs * fstride + si];
    }
}

int launch_permute(dg_batch *b, const GridSlot &s, bool to_stored, const float *src, float *dst) {
    const long long cells = 5LL * s.cn[0] * s.cn[1] * s.cn[2];
    const int threads = 256;
    const int blocks = (int)std::min<long long>((cells + threads - 1) / threads, 148LL * 16);
    if (to_stored)
        permute_fields<true><<<blocks, threads, 0, b->stream>>>(src, dst, s.cn[0], s.cn[1], s.cn[2], s.perm[0],
                                                                s.perm[1], s.perm[2], s.pitch, s.fstride);
    else
        permute_fields<false><<<blocks, threads, 0, b->stream>>>(src, dst, s.cn[0], s.cn[1], s.cn[2], s.perm[0],
                                                                 s.perm[1], s.perm[2], s.pitch, s.fstride);
    B_CUDA(b, cudaGetLastError());
    return DG_OK;
}

bool identity(const GridSlot &s) { return s.perm[0] == 0 && s.perm[1] == 1 && s.perm[2] == 2; }

}  // namespace

extern "C" {

int32_t dg_batch_create(int32_t n, const dg_sim_info *infos, dg_batch **out) {
    return dg_batch_create_ex(n, infos, 0, out);
}

int32_t dg_batch_create_ex(int32_t n, const dg_sim_info *infos, uint32_t flags, dg_batch **out) {
    if (!out) return bfail(nullptr, DG_ERR_INVALID, "null out");
    if (flags & ~(uint32_t)DG_BATCH_REORIENT) return bfail(nullptr, DG_ERR_INVALID, "unknown batch flags");
    *out = nullptr;
    if (n < 1 || !infos) return bfail(nullptr, DG_ERR_INVALID, "need at least one grid");
    for (int i = 0; i < n; ++i) {
        const dg_sim_info &f = infos[i];
        if (f.nghosts != 2 || f.nx < 2 || f.ny < 2 || f.nz < 2 || !(f.ds > 0) || !(f.gamma > 1) || !(f.cfl > 0))
            return bfail(nullptr, DG_ERR_INVALID, "grid " + std::to_string(i) + ": bad sizes or constants");
        if (f.precision != DG_F32 || f.rounding != DG_ROUNDING_DEFAULT)
            return bfail(nullptr, DG_ERR_INVALID, "batches run the FP32 fast kernel (precision DG_F32, default rounding)");
        if (f.device != infos[0].device) return bfail(nullptr, DG_ERR_INVALID, "all grids of a batch share one device");
        if (f.limiter != DG_LIMITER_NONE && f.limiter != DG_LIMITER_MINMOD)
            return bfail(nullptr, DG_ERR_INVALID, "bad limiter");
        for (int a = 0; a < 3; ++a) {
            const int lo = f.bcs[2 * a], hi = f.bcs[2 * a + 1];
            if (!valid_bc_pair(lo, hi))
                return bfail(nullptr, DG_ERR_INVALID, "grid " + std::to_string(i) + ": bad boundary types");
        }
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, infos[0].device) != cudaSuccess || prop.major != 10)
        return bfail(nullptr, DG_ERR_NO_DEVICE, "the kernels are built for sm_100a (B200)");
    dg_batch *b = new dg_batch();
    b->n = n;
    b->device = infos[0].device;
    b->g.resize(n);
    size_t total = 0;
    for (int i = 0; i < n; ++i) {
        GridSlot &s = b->g[i];
        const dg_sim_info &f = infos[i];
        choose_orientation(f, (flags & DG_BATCH_REORIENT) != 0, s.perm);
        const int cn[3] = {f.nx, f.ny, f.nz};
        s.info = f;
        s.info.nx = cn[s.perm[0]];
        s.info.ny = cn[s.perm[1]];
        s.info.nz = cn[s.perm[2]];
        for (int d = 0; d < 3; ++d) {
            s.info.bcs[2 * d] = f.bcs[2 * s.perm[d]];
            s.info.bcs[2 * d + 1] = f.bcs[2 * s.perm[d] + 1];
            s.cn[d] = cn[d] + 4;
        }
        s.nx = s.info.nx + 4;
        s.ny = s.info.ny + 4;
        s.nz = s.info.nz + 4;
        s.pitch = (s.nz + 31) / 32 * 32;
        s.fstride = (long long)s.nx * s.ny * s.pitch;
        s.state_bytes = ((size_t)5 * s.fstride * 4 + 255) / 256 * 256;
        total += 2 * s.state_bytes;
    }
    auto bail = [&](int code) {
        set_global_error(b->err);
        dg_batch_destroy(b);
        return code;
    };
    if (cudaSetDevice(b->device) != cudaSuccess) { b->err = "cudaSetDevice failed"; return bail(DG_ERR_CUDA); }
    cudaError_t e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc(&b->arena, total);
    if (e == cudaSuccess) e = cudaMalloc(&b->ctl, n * sizeof(DevCtl));
    for (int p = 0; p < 2 && e == cudaSuccess; ++p) {
        e = cudaMalloc(&b->d_args[p], n * sizeof(GridArgs<float>));
        if (e == cudaSuccess) e = cudaMalloc(&b->d_maps[p], n * sizeof(CUtensorMap));
    }
    if (e == cudaSuccess) e = cudaMalloc(&b->d_queue, kCombos * sizeof(unsigned));
    if (e == cudaSuccess) e = cudaMemsetAsync(b->arena, 0, total, b->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(b->ctl, 0, n * sizeof(DevCtl), b->stream);
    if (e == cudaSuccess) e = prepare_kernel<0, false>();
    if (e == cudaSuccess) e = prepare_kernel<1, false>();
    if (e == cudaSuccess) e = prepare_kernel<0, true>();
    if (e == cudaSuccess) e = prepare_kernel<1, true>();
    if (e == cudaSuccess) e = cudaStreamSynchronize(b->stream);
    if (e != cudaSuccess) { b->err = std::string("batch set-up: ") + cudaGetErrorString(e); return bail(DG_ERR_CUDA); }
    char *p = static_cast<char *>(b->arena);
    for (auto &s : b->g) {
        s.buf[0] = p;
        s.buf[1] = p + s.state_bytes;
        p += 2 * s.state_bytes;
    }
    if (rebuild(b) != DG_OK) return bail(DG_ERR_CUDA);
    *out = b;
    return DG_OK;
}

int32_t dg_batch_destroy(dg_batch *b) {
    if (!b) return DG_OK;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->graph) cudaGraphExecDestroy(b->graph);
    if (b->arena) cudaFree(b->arena);
    if (b->ctl) cudaFree(b->ctl);
    if (b->part) cudaFree(b->part);
    for (int p = 0; p < 2; ++p) {
        if (b->d_args[p]) cudaFree(b->d_args[p]);
        if (b->d_maps[p]) cudaFree(b->d_maps[p]);
    }
    if (b->d_items) cudaFree(b->d_items);
    if (b->d_queue) cudaFree(b->d_queue);
    if (b->stream) cudaStreamDestroy(b->stream);
    delete b;
    return DG_OK;
}

// Set grid i's state from host primitives (calc_conserved on the device).
// The grid joins the batch at its current step count.
int32_t dg_batch_set_primitives(dg_batch *b, int32_t i, const void *const prim[5]) {
    if (!b || !prim || i < 0 || i >= b->n) return bfail(b, DG_ERR_INVALID, "bad argument");
    B_CUDA(b, cudaSetDevice(b->device));
    GridSlot &s = b->g[i];
    const int cur = (int)(b->steps & 1);
    void *stage = s.buf[1 - cur];
    for (int f = 0; f < 5; ++f)
        if (!prim[f]) return bfail(b, DG_ERR_INVALID, "null field");
    if (identity(s)) {
        const size_t row = (size_t)s.nz * 4;
        for (int f = 0; f < 5; ++f)
            B_CUDA(b, cudaMemcpy2DAsync(static_cast<char *>(stage) + (size_t)f * s.fstride * 4, (size_t)s.pitch * 4,
                                        prim[f], row, row, (size_t)s.nx * s.ny, cudaMemcpyHostToDevice, b->stream));
    } else {
        // the caller's fields, dense, into the other buffer, then permuted
        // into the stored layout
        const size_t cells = (size_t)s.cn[0] * s.cn[1] * s.cn[2];
        float *raw = static_cast<float *>(s.buf[cur]);
        for (int f = 0; f < 5; ++f)
            B_CUDA(b, cudaMemcpyAsync(raw + f * cells, prim[f], cells * 4, cudaMemcpyHostToDevice, b->stream));
        const int r = launch_permute(b, s, true, raw, static_cast<float *>(stage));
        if (r != DG_OK) return r;
    }
    GridArgs<float> a = args_of(b, i, cur);
    a.part = b->part;
    B_CUDA(b, cudaMemsetAsync(a.ctl, 0, sizeof(DevCtl), b->stream));
    // the grid's step counter must match the batch's parity: the kernels
    // read dt[step & 1]
    const unsigned long long st = b->steps;
    B_CUDA(b, cudaMemcpyAsync(&a.ctl->step, &st, sizeof(st), cudaMemcpyHostToDevice, b->stream));
    B_CUDA(b, launch_prim_to_cons<float>(a, static_cast<const float *>(stage), s.fstride, s.pitch,
                                         static_cast<float *>(s.buf[cur]), b->stream));
    B_CUDA(b, launch_fill_ghosts<float>(a, static_cast<float *>(s.buf[cur]), b->stream));
    B_CUDA(b, (launch_reduce_policy<float, false>(a, 1, b->stream)));
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    return DG_OK;
}

int32_t dg_batch_step(dg_batch *b, int32_t nsteps) {
    if (!b || nsteps < 0) return bfail(b, DG_ERR_INVALID, "bad argument");
    B_CUDA(b, cudaSetDevice(b->device));
    int r = enqueue(b, nsteps);
    if (r != DG_OK) return r;
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    return check_timeouts(b);
}

int32_t dg_batch_enqueue(dg_batch *b, int32_t nsteps) {
    if (!b || nsteps < 0) return bfail(b, DG_ERR_INVALID, "bad argument");
    B_CUDA(b, cudaSetDevice(b->device));
    return enqueue(b, nsteps);
}

// dt of the last nsteps steps of grid i (nsteps <= 4096).
int32_t dg_batch_get_dts(dg_batch *b, int32_t i, int32_t nsteps, double *dts) {
    if (!b || !dts || i < 0 || i >= b->n || nsteps < 0 || nsteps > kHist || (unsigned long long)nsteps > b->steps)
        return bfail(b, DG_ERR_INVALID, "bad argument");
    B_CUDA(b, cudaSetDevice(b->device));
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    std::vector<double> hist(kHist);
    B_CUDA(b, cudaMemcpy(hist.data(), b->ctl[i].hist, kHist * sizeof(double), cudaMemcpyDeviceToHost));
    const unsigned long long first = b->steps - nsteps;
    for (int s = 0; s < nsteps; ++s) dts[s] = hist[(first + s) % kHist];
    return DG_OK;
}

int32_t dg_batch_get_conserved(dg_batch *b, int32_t i, void *const cons[5]) {
    if (!b || !cons || i < 0 || i >= b->n) return bfail(b, DG_ERR_INVALID, "bad argument");
    B_CUDA(b, cudaSetDevice(b->device));
    const GridSlot &s = b->g[i];
    const char *src = static_cast<const char *>(s.buf[b->steps & 1]);
    for (int f = 0; f < 5; ++f)
        if (!cons[f]) return bfail(b, DG_ERR_INVALID, "null field");
    if (identity(s)) {
        const size_t row = (size_t)s.nz * 4;
        for (int f = 0; f < 5; ++f)
            B_CUDA(b, cudaMemcpy2DAsync(cons[f], row, src + (size_t)f * s.fstride * 4, (size_t)s.pitch * 4, row,
                                        (size_t)s.nx * s.ny, cudaMemcpyDeviceToHost, b->stream));
    } else {
        // permuted back into the caller's layout in the other buffer (which
        // the next step overwrites), then copied out dense
        const size_t cells = (size_t)s.cn[0] * s.cn[1] * s.cn[2];
        float *raw = static_cast<float *>(s.buf[1 - (b->steps & 1)]);
        const int r = launch_permute(b, s, false, reinterpret_cast<const float *>(src), raw);
        if (r != DG_OK) return r;
        for (int f = 0; f < 5; ++f)
            B_CUDA(b, cudaMemcpyAsync(cons[f], raw + f * cells, cells * 4, cudaMemcpyDeviceToHost, b->stream));
    }
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    return DG_OK;
}

// Tile rows (the sweep kernel's tile rows, as dg_batch_get_tiling reports
// them) and x-planes per work item (0 = automatic).
int32_t dg_batch_set_tiling(dg_batch *b, int32_t tile_rows, int32_t chunk) {
    if (!b || tile_rows != kTY || chunk < 0)
        return bfail(b, DG_ERR_INVALID, "bad tiling (tile rows must be " + std::to_string(kTY) + ")");
    b->tile_rows = tile_rows;
    b->chunk = chunk;
    b->dirty = true;
    return DG_OK;
}

int32_t dg_batch_get_tiling(dg_batch *b, int32_t *tile_rows, int32_t *chunk, int32_t *items) {
    if (!b) return DG_ERR_INVALID;
    if (b->dirty) {
        int r = rebuild(b);
        if (r != DG_OK) return r;
    }
    if (tile_rows) *tile_rows = b->tile_rows;
    if (chunk) *chunk = b->chunk_used;
    if (items) *items = b->nitems;
    return DG_OK;
}

// Autotuner: times `steps` steps (after one warm-up step) of every
// candidate tiling on the live batch, keeps the fastest, and restores the
// states, dt and step counters so that tuning leaves no trace.  Writes the
// choice and its time per step.
int32_t dg_batch_autotune(dg_batch *b, int32_t steps, int32_t *tile_rows, int32_t *chunk, double *ms_per_step) {
    if (!b || steps < 1) return bfail(b, DG_ERR_INVALID, "bad argument");
    B_CUDA(b, cudaSetDevice(b->device));
    int r;
    if (b->dirty && (r = rebuild(b)) != DG_OK) return r;
    // save: current states (both buffers, so the parity is irrelevant) and control blocks
    size_t total = 0;
    for (auto &s : b->g) total += 2 * s.state_bytes;
    void *save = nullptr;
    DevCtl *save_ctl = nullptr;
    B_CUDA(b, cudaMalloc(&save, total));
    B_CUDA(b, cudaMalloc(&save_ctl, b->n * sizeof(DevCtl)));
    B_CUDA(b, cudaMemcpyAsync(save, b->arena, total, cudaMemcpyDeviceToDevice, b->stream));
    B_CUDA(b, cudaMemcpyAsync(save_ctl, b->ctl, b->n * sizeof(DevCtl), cudaMemcpyDeviceToDevice, b->stream));
    const unsigned long long steps0 = b->steps;
    const int rows_cand[1] = {kTY};
    const int chunk_cand[6] = {16, 24, 32, 64, 128, 256};
    double best = 1e30;
    int best_rows = b->tile_rows, best_chunk = b->chunk;
    cudaEvent_t e0, e1;
    B_CUDA(b, cudaEventCreate(&e0));
    B_CUDA(b, cudaEventCreate(&e1));
    for (int rr : rows_cand)
        for (int cc : chunk_cand) {
            b->tile_rows = rr;
            b->chunk = cc;
            b->dirty = true;
            if ((r = enqueue(b, 1)) != DG_OK) return r;   // warm-up (and graph capture below)
            B_CUDA(b, cudaEventRecord(e0, b->stream));
            if ((r = enqueue(b, steps)) != DG_OK) return r;
            B_CUDA(b, cudaEventRecord(e1, b->stream));
            B_CUDA(b, cudaEventSynchronize(e1));
            float ms = 0;
            B_CUDA(b, cudaEventElapsedTime(&ms, e0, e1));
            if (ms / steps < best) {
                best = ms / steps;
                best_rows = rr;
                best_chunk = cc;
            }
            // restore
            B_CUDA(b, cudaMemcpyAsync(b->arena, save, total, cudaMemcpyDeviceToDevice, b->stream));
            B_CUDA(b, cudaMemcpyAsync(b->ctl, save_ctl, b->n * sizeof(DevCtl), cudaMemcpyDeviceToDevice, b->stream));
            b->steps = steps0;
        }
    B_CUDA(b, cudaStreamSynchronize(b->stream));
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(save);
    cudaFree(save_ctl);
    b->tile_rows = best_rows;
    b->chunk = best_chunk;
    b->dirty = true;
    if (tile_rows) *tile_rows = best_rows;
    if (chunk) *chunk = best_chunk;
    if (ms_per_step) *ms_per_step = best;
    return check_timeouts(b);
}

int32_t dg_batch_get_orientation(dg_batch *b, int32_t i, int32_t axes[3]) {
    if (!b || !axes || i < 0 || i >= b->n) return bfail(b, DG_ERR_INVALID, "bad argument");
    for (int d = 0; d < 3; ++d) axes[d] = b->g[i].perm[d];
    return DG_OK;
}

int32_t dg_batch_get_stream(dg_batch *b, void **stream) {
    if (!b || !stream) return bfail(b, DG_ERR_INVALID, "null argument");
    *stream = (void *)b->stream;
    return DG_OK;
}

const char *dg_batch_last_error(const dg_batch *b) { return b ? b->err.c_str() : dg_last_error(nullptr); }

}  // extern "C"
