// dg_capi.cu -- the C ABI declared in include/deepgreen.h.
//
// A context owns two device copies of the ghosted state (the step reads one
// and writes the other), the step control block (dt, sums, history) and
// the per-block partials buffer, plus one TMA descriptor per state buffer.
#include <cudaTypedefs.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>

#include "../../include/deepgreen.h"
#include "dg_ctx.h"

using namespace dg;


namespace {

// message of the calling thread's last failure outside a context
thread_local std::string g_create_err = "no error";

PFN_cuTensorMapEncodeTiled_v12000 get_encode_fn() {
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

int auto_chunk(const dg_ctx *c) {
    return c->chunk > 0 ? c->chunk : choose_chunk(c->nx, c->ny, c->nz, c->kind);
}

int encode_map(dg_ctx *c, int i) {
    auto fn = get_encode_fn();
    if (!fn) return fail(c, DG_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
    const int ty = step_tile_rows(c->kind);
    cuuint64_t dims[4] = {(cuuint64_t)c->nz, (cuuint64_t)c->ny, (cuuint64_t)c->nx, 5};
    cuuint64_t strides[3] = {(cuuint64_t)c->pitch * c->elem, (cuuint64_t)c->pitch * c->ny * c->elem,
                             (cuuint64_t)c->fstride * c->elem};
    cuuint32_t box[4] = {(cuuint32_t)step_box_cols(c->kind), (cuuint32_t)(ty + 4), 1, 5};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    CUresult r = fn(&c->tmap[i], c->elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                    4, c->buf[i], dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                    CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                    CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return fail(c, DG_ERR_CUDA, "cuTensorMapEncodeTiled failed: " + std::to_string((int)r));
    return DG_OK;
}

int use_device(dg_ctx *c) {
    DG_CUDA(c, cudaSetDevice(c->info.device));
    return DG_OK;
}

// Fill ghosts of the current state, then the dt / sums reduction.
int finish_state(dg_ctx *c) {
    cudaError_t e;
    if (c->elem == 8) {
        auto a = grid_args<double>(c, c->buf[c->cur], c->buf[c->cur]);
        e = launch_fill_ghosts<double>(a, static_cast<double *>(c->buf[c->cur]), c->stream);
        if (e == cudaSuccess) e = launch_reduce_policy<double, true>(a, 1, c->stream);
    } else {
        auto a = grid_args<float>(c, c->buf[c->cur], c->buf[c->cur]);
        e = launch_fill_ghosts<float>(a, static_cast<float *>(c->buf[c->cur]), c->stream);
        if (e == cudaSuccess)
            e = c->exact ? launch_reduce_policy<float, true>(a, 1, c->stream)
                         : launch_reduce_policy<float, false>(a, 1, c->stream);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "state set-up kernels");
    c->has_state = true;
    c->steps = 0;
    return DG_OK;
}

int reset_ctl(dg_ctx *c) {
    DG_CUDA(c, cudaMemsetAsync(c->ctl, 0, sizeof(DevCtl), c->stream));
    return DG_OK;
}

// Copy 5 dense host/device fields (n^3 each) into the pitched buffer dst.
int copy_in(dg_ctx *c, void *dst, const void *const src[5], cudaMemcpyKind kind) {
    const size_t row = (size_t)c->nz * c->elem;
    for (int f = 0; f < 5; ++f) {
        if (!src[f]) return fail(c, DG_ERR_INVALID, "null field pointer");
        char *d = static_cast<char *>(dst) + (size_t)f * c->fstride * c->elem;
        DG_CUDA(c, cudaMemcpy2DAsync(d, (size_t)c->pitch * c->elem, src[f], row, row, (size_t)c->nx * c->ny, kind,
                                     c->stream));
    }
    return DG_OK;
}

// Host transfers move each field as one contiguous copy (the copy engines'
// fast case; row-by-row copies of the pitched layout from host memory run
// at about half the rate) through a dense device copy of the fields; the
// re-pitch between the dense and the pitched layout is a device-to-device
// copy.
size_t dense_field_bytes(const dg_ctx *c) { return (size_t)c->nx * c->ny * c->nz * c->elem; }

int upload_dense(dg_ctx *c, void *dense, const void *const src[5]) {
    const size_t fb = dense_field_bytes(c);
    for (int f = 0; f < 5; ++f) {
        if (!src[f]) return fail(c, DG_ERR_INVALID, "null field pointer");
        DG_CUDA(c, cudaMemcpyAsync(static_cast<char *>(dense) + f * fb, src[f], fb, cudaMemcpyHostToDevice,
                                   c->stream));
    }
    return DG_OK;
}

int download_dense(dg_ctx *c, void *const dst[5], const void *dense) {
    const size_t fb = dense_field_bytes(c);
    for (int f = 0; f < 5; ++f) {
        if (!dst[f]) return fail(c, DG_ERR_INVALID, "null field pointer");
        DG_CUDA(c, cudaMemcpyAsync(dst[f], static_cast<const char *>(dense) + f * fb, fb, cudaMemcpyDeviceToHost,
                                   c->stream));
    }
    return DG_OK;
}

// dense <-> pitched, on the device
int repitch(dg_ctx *c, void *dst, const void *src, bool to_pitched) {
    const size_t row = (size_t)c->nz * c->elem, fb = dense_field_bytes(c);
    const size_t pitched = (size_t)c->pitch * c->elem;
    for (int f = 0; f < 5; ++f) {
        const size_t po = (size_t)f * c->fstride * c->elem;
        if (to_pitched)
            DG_CUDA(c, cudaMemcpy2DAsync(static_cast<char *>(dst) + po, pitched, static_cast<const char *>(src) + f * fb,
                                         row, row, (size_t)c->nx * c->ny, cudaMemcpyDeviceToDevice, c->stream));
        else
            DG_CUDA(c, cudaMemcpy2DAsync(static_cast<char *>(dst) + f * fb, row, static_cast<const char *>(src) + po,
                                         pitched, row, (size_t)c->nx * c->ny, cudaMemcpyDeviceToDevice, c->stream));
    }
    return DG_OK;
}

int copy_out(dg_ctx *c, void *const dst[5], const void *src, cudaMemcpyKind kind) {
    const size_t row = (size_t)c->nz * c->elem;
    for (int f = 0; f < 5; ++f) {
        if (!dst[f]) return fail(c, DG_ERR_INVALID, "null field pointer");
        const char *s = static_cast<const char *>(src) + (size_t)f * c->fstride * c->elem;
        DG_CUDA(c, cudaMemcpy2DAsync(dst[f], row, s, (size_t)c->pitch * c->elem, row, (size_t)c->nx * c->ny, kind,
                                     c->stream));
    }
    return DG_OK;
}

int check_flags(dg_ctx *c) {
    unsigned flags = 0;
    DG_CUDA(c, cudaMemcpyAsync(&flags, &c->ctl->flags, sizeof(flags), cudaMemcpyDeviceToHost, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    if (flags & kStatusTimeout) {
        c->has_state = false;
        return fail(c, DG_ERR_TIMEOUT, "a device-side wait timed out; state invalid, set a new state");
    }
    return DG_OK;
}

int enqueue(dg_ctx *c, int nsteps) {
    const int chunk = auto_chunk(c);
    for (int s = 0; s < nsteps; ++s) {
        const int src = c->cur, dst = 1 - c->cur;
        cudaError_t e;
        if (c->elem == 8) {
            auto a = grid_args<double>(c, c->buf[src], c->buf[dst]);
            e = c->kind == kFastF64 ? launch_sweep(a, &c->tmap[src], chunk, c->stream)
                                    : launch_step_policy<double, true>(a, &c->tmap[src], c->info.limiter, chunk,
                                                                       c->stream);
        } else {
            auto a = grid_args<float>(c, c->buf[src], c->buf[dst]);
            e = c->exact ? launch_step_policy<float, true>(a, &c->tmap[src], c->info.limiter, chunk, c->stream)
                         : launch_sweep(a, &c->tmap[src], chunk, c->stream);
        }
        if (e != cudaSuccess) return cuda_fail(c, e, "step kernel launch");
        c->cur = dst;
        ++c->steps;
    }
    return DG_OK;
}

int read_dts(dg_ctx *c, int nsteps, double *dts) {
    // dt of steps [steps - nsteps, steps) sit in the history ring
    if (nsteps > kHist) return fail(c, DG_ERR_INVALID, "at most 4096 dt values per read");
    if ((unsigned long long)nsteps > c->steps) return fail(c, DG_ERR_INVALID, "fewer steps taken than requested");
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    const unsigned long long first = c->steps - nsteps;
    int done = 0;
    while (done < nsteps) {
        const int pos = (int)((first + done) % kHist);
        const int n = std::min(nsteps - done, kHist - pos);
        DG_CUDA(c, cudaMemcpy(dts + done, &c->ctl->hist[pos], n * sizeof(double), cudaMemcpyDeviceToHost));
        done += n;
    }
    return DG_OK;
}

}  // namespace

// Entry points for the other C-ABI sources of the library (dg_ctx.h).
int dg::ctx_enqueue(dg_ctx *c, int nsteps) { return enqueue(c, nsteps); }

int dg::ctx_begin_state(dg_ctx *c) {
    int r = use_device(c);
    return r != DG_OK ? r : reset_ctl(c);
}

int dg::ctx_finish_state(dg_ctx *c) { return finish_state(c); }

int dg::ctx_check_flags(dg_ctx *c) { return check_flags(c); }

namespace {
// dt of the coming step := dt (the step counter lives on the device)
__global__ void set_next_dt_kernel(DevCtl *ctl, double dt) { ctl->dt[ctl->step & 1] = dt; }
}  // namespace

void dg::set_global_error(const std::string &msg) { g_create_err = msg; }

extern "C" {

int32_t dg_abi_version(void) { return DG_ABI_VERSION; }

int32_t dg_create(const dg_sim_info *info, dg_ctx **out) {
    auto set_err = [](const std::string &m) { g_create_err = m; };
    if (!out) return DG_ERR_INVALID;
    *out = nullptr;
    if (!info) { set_err("null info"); return DG_ERR_INVALID; }
    if (info->nghosts != 2) { set_err("nghosts must be 2"); return DG_ERR_INVALID; }
    if (info->nx < 2 || info->ny < 2 || info->nz < 2) { set_err("each axis needs >= 2 interior cells"); return DG_ERR_INVALID; }
    if (!(info->ds > 0) || !(info->gamma > 1) || !(info->cfl > 0)) { set_err("ds > 0, gamma > 1, cfl > 0 required"); return DG_ERR_INVALID; }
    if (info->precision != DG_F32 && info->precision != DG_F64) { set_err("precision must be DG_F32 or DG_F64"); return DG_ERR_INVALID; }
    if (info->limiter != DG_LIMITER_NONE && info->limiter != DG_LIMITER_MINMOD) { set_err("unknown limiter"); return DG_ERR_INVALID; }
    if (info->rounding != DG_ROUNDING_DEFAULT && info->rounding != DG_ROUNDING_REFERENCE &&
        info->rounding != DG_ROUNDING_FAST) { set_err("unknown rounding policy"); return DG_ERR_INVALID; }
    for (int a = 0; a < 3; ++a) {
        const int lo = info->bcs[2 * a], hi = info->bcs[2 * a + 1];
        if (lo < 0 || lo > DG_BC_CONDUCTING_WALL || hi < 0 || hi > DG_BC_CONDUCTING_WALL) { set_err("unknown boundary type"); return DG_ERR_INVALID; }
        // Simulation::new (grid.rs:55-63) pairs periodic faces
        if (!valid_bc_pair(lo, hi)) { set_err("periodic faces must come in pairs"); return DG_ERR_INVALID; }
    }
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || info->device < 0 || info->device >= ndev) {
        set_err("no CUDA device with that ordinal");
        return DG_ERR_NO_DEVICE;
    }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, info->device) != cudaSuccess || prop.major != 10) {
        set_err("the kernels are built for sm_100a (B200)");
        return DG_ERR_NO_DEVICE;
    }
    dg_ctx *c = new (std::nothrow) dg_ctx();
    if (!c) { set_err("out of host memory"); return DG_ERR_INVALID; }
    c->info = *info;
    c->elem = info->precision == DG_F64 ? 8 : 4;
    c->exact = info->rounding == DG_ROUNDING_REFERENCE || (c->elem == 8 && info->rounding == DG_ROUNDING_DEFAULT);
    c->kind = c->elem == 8 ? (c->exact ? kRefF64 : kFastF64) : (c->exact ? kRefF32 : kFastF32);
    c->nx = info->nx + 4;
    c->ny = info->ny + 4;
    c->nz = info->nz + 4;
    c->pitch = (c->nz + 31) / 32 * 32;
    // Test hook: a context created while DG_DEBUG_WAIT_BUDGET is set gives
    // its step kernels' waits for staged planes that many SM clocks (0 or
    // less: every such wait gives up at once, without waiting) instead of
    // ~2 s, so that a test can make the waits run out and check that the
    // step reports DG_ERR_TIMEOUT and the device stays usable.
    if (const char *wb = std::getenv("DG_DEBUG_WAIT_BUDGET")) {
        const long long v = std::atoll(wb);
        c->wait_budget = v > 0 ? v : -1;
    }
    c->fstride = (long long)c->nx * c->ny * c->pitch;
    c->state_bytes = (size_t)5 * c->fstride * c->elem;
    auto bail = [&](int code) {
        set_err(c->err);
        dg_destroy(c);
        return code;
    };
    if (cudaSetDevice(info->device) != cudaSuccess) { c->err = "cudaSetDevice failed"; return bail(DG_ERR_CUDA); }
    cudaError_t e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking);
    for (int i = 0; i < 2 && e == cudaSuccess; ++i) e = cudaMalloc(&c->buf[i], c->state_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&c->ctl, sizeof(DevCtl));
    if (e == cudaSuccess) {
        const int ty = step_tile_rows(c->kind), tzc = step_tile_cols(c->kind);
        long long tiles = (long long)((c->ny - 4 + ty - 1) / ty) * ((c->nz - 4 + tzc - 1) / tzc);
        long long cap = tiles * (c->nx - 4);   // chunk >= 1
        if (cap < kReduceBlocks) cap = kReduceBlocks;
        c->part_cap = (int)cap;
        e = cudaMalloc(&c->part, (size_t)cap * sizeof(Partial));
    }
    if (e != cudaSuccess) { c->err = std::string("device allocation: ") + cudaGetErrorString(e); return bail(DG_ERR_CUDA); }
    for (int i = 0; i < 2; ++i)
        if (encode_map(c, i) != DG_OK) return bail(DG_ERR_CUDA);
    if (reset_ctl(c) != DG_OK) return bail(DG_ERR_CUDA);
    if (cudaMemsetAsync(c->buf[0], 0, c->state_bytes, c->stream) != cudaSuccess ||
        cudaMemsetAsync(c->buf[1], 0, c->state_bytes, c->stream) != cudaSuccess ||
        cudaStreamSynchronize(c->stream) != cudaSuccess) {
        c->err = "initial memset failed";
        return bail(DG_ERR_CUDA);
    }
    *out = c;
    return DG_OK;
}

int32_t dg_destroy(dg_ctx *c) {
    if (!c) return DG_OK;
    cudaSetDevice(c->info.device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    for (int i = 0; i < 2; ++i)
        if (c->buf[i]) cudaFree(c->buf[i]);
    if (c->ctl) cudaFree(c->ctl);
    if (c->part) cudaFree(c->part);
    if (c->prim_scratch) cudaFree(c->prim_scratch);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
    return DG_OK;
}

int32_t dg_set_conserved(dg_ctx *c, const void *const cons[5]) {
    if (!c || !cons) return fail(c, DG_ERR_INVALID, "null argument");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    if ((r = reset_ctl(c)) != DG_OK) return r;
    // the other state buffer holds the dense upload
    if ((r = upload_dense(c, c->buf[1 - c->cur], cons)) != DG_OK) return r;
    if ((r = repitch(c, c->buf[c->cur], c->buf[1 - c->cur], true)) != DG_OK) return r;
    if ((r = finish_state(c)) != DG_OK) return r;
    return check_flags(c);
}

int32_t dg_set_conserved_device(dg_ctx *c, const void *const cons[5]) {
    if (!c || !cons) return fail(c, DG_ERR_INVALID, "null argument");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    if ((r = reset_ctl(c)) != DG_OK) return r;
    if ((r = copy_in(c, c->buf[c->cur], cons, cudaMemcpyDeviceToDevice)) != DG_OK) return r;
    if ((r = finish_state(c)) != DG_OK) return r;
    return check_flags(c);
}

int32_t dg_set_primitives(dg_ctx *c, const void *const prim[5]) {
    if (!c || !prim) return fail(c, DG_ERR_INVALID, "null argument");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    if ((r = reset_ctl(c)) != DG_OK) return r;
    // stage the primitives densely in the other state buffer, convert into the current one
    void *stage = c->buf[1 - c->cur];
    if ((r = upload_dense(c, stage, prim)) != DG_OK) return r;
    const long long dfs = (long long)c->nx * c->ny * c->nz;
    cudaError_t e;
    if (c->elem == 8) {
        auto a = grid_args<double>(c, stage, c->buf[c->cur]);
        e = launch_prim_to_cons<double>(a, static_cast<const double *>(stage), dfs, c->nz,
                                        static_cast<double *>(c->buf[c->cur]), c->stream);
    } else {
        auto a = grid_args<float>(c, stage, c->buf[c->cur]);
        e = launch_prim_to_cons<float>(a, static_cast<const float *>(stage), dfs, c->nz,
                                       static_cast<float *>(c->buf[c->cur]), c->stream);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "prim_to_cons");
    if ((r = finish_state(c)) != DG_OK) return r;
    return check_flags(c);
}

int32_t dg_enqueue_steps(dg_ctx *c, int32_t nsteps) {
    if (!c || nsteps < 0) return fail(c, DG_ERR_INVALID, "bad argument");
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    return enqueue(c, nsteps);
}

int32_t dg_get_dts(dg_ctx *c, int32_t nsteps, double *dts) {
    if (!c || !dts || nsteps < 0) return fail(c, DG_ERR_INVALID, "bad argument");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    if ((r = read_dts(c, nsteps, dts)) != DG_OK) return r;
    return check_flags(c);
}

int32_t dg_synchronize(dg_ctx *c) {
    if (!c) return DG_ERR_INVALID;
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_flags(c);
}

int32_t dg_compute_step(dg_ctx *c, int32_t nsteps, double *dts) {
    if (!c || nsteps < 0) return fail(c, DG_ERR_INVALID, "bad argument");
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    int done = 0;
    while (done < nsteps) {
        const int n = std::min(nsteps - done, kHist);
        if ((r = enqueue(c, n)) != DG_OK) return r;
        if (dts) {
            if ((r = read_dts(c, n, dts + done)) != DG_OK) return r;
        }
        done += n;
    }
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_flags(c);
}

int32_t dg_next_dt(dg_ctx *c, double *dt) {
    if (!c || !dt) return fail(c, DG_ERR_INVALID, "null argument");
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    DG_CUDA(c, cudaMemcpyAsync(dt, &c->ctl->dt[c->steps & 1], sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_flags(c);
}

int32_t dg_compute_step_dt(dg_ctx *c, double dt) {
    if (!c) return fail(c, DG_ERR_INVALID, "null argument");
    if (!(dt > 0.0) || !std::isfinite(dt)) return fail(c, DG_ERR_INVALID, "dt must be positive and finite");
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    set_next_dt_kernel<<<1, 1, 0, c->stream>>>(c->ctl, dt);
    DG_CUDA(c, cudaGetLastError());
    if ((r = enqueue(c, 1)) != DG_OK) return r;
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return check_flags(c);
}

int32_t dg_get_conserved(dg_ctx *c, void *const cons[5]) {
    if (!c || !cons) return fail(c, DG_ERR_INVALID, "null argument");
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    if (!c->prim_scratch) DG_CUDA(c, cudaMalloc(&c->prim_scratch, c->state_bytes));
    if ((r = repitch(c, c->prim_scratch, c->buf[c->cur], false)) != DG_OK) return r;
    if ((r = download_dense(c, cons, c->prim_scratch)) != DG_OK) return r;
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

int32_t dg_get_conserved_device(dg_ctx *c, void *const cons[5]) {
    if (!c || !cons) return fail(c, DG_ERR_INVALID, "null argument");
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    if ((r = copy_out(c, cons, c->buf[c->cur], cudaMemcpyDeviceToDevice)) != DG_OK) return r;
    // the destination belongs to the caller's streams: return after the copies
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

int32_t dg_get_primitives(dg_ctx *c, void *const prim[5]) {
    if (!c || !prim) return fail(c, DG_ERR_INVALID, "null argument");
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    if (!c->prim_scratch) DG_CUDA(c, cudaMalloc(&c->prim_scratch, c->state_bytes));
    // the state at the start of the last step is the other buffer; the
    // primitives are written densely for contiguous host copies
    const void *src = c->steps > 0 ? c->buf[1 - c->cur] : c->buf[c->cur];
    const long long dfs = (long long)c->nx * c->ny * c->nz;
    cudaError_t e;
    if (c->elem == 8) {
        auto a = grid_args<double>(c, src, nullptr);
        e = launch_cons_to_prim_policy<double, true>(a, static_cast<const double *>(src),
                                                     static_cast<double *>(c->prim_scratch), dfs, c->nz, c->stream);
    } else {
        auto a = grid_args<float>(c, src, nullptr);
        auto *dstp = static_cast<float *>(c->prim_scratch);
        e = c->exact ? launch_cons_to_prim_policy<float, true>(a, static_cast<const float *>(src), dstp, dfs, c->nz,
                                                               c->stream)
                     : launch_cons_to_prim_policy<float, false>(a, static_cast<const float *>(src), dstp, dfs, c->nz,
                                                                c->stream);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "cons_to_prim");
    if ((r = download_dense(c, prim, c->prim_scratch)) != DG_OK) return r;
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

int32_t dg_conservation_sums(dg_ctx *c, double out[5]) {
    if (!c || !out) return fail(c, DG_ERR_INVALID, "null argument");
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    // FP64 sums of the current state, reduced on the device in a fixed order
    cudaError_t e;
    if (c->elem == 8) {
        e = launch_reduce_policy<double, true>(grid_args<double>(c, c->buf[c->cur], nullptr), 0, c->stream);
    } else {
        auto a = grid_args<float>(c, c->buf[c->cur], nullptr);
        e = c->exact ? launch_reduce_policy<float, true>(a, 0, c->stream)
                     : launch_reduce_policy<float, false>(a, 0, c->stream);
    }
    if (e != cudaSuccess) return cuda_fail(c, e, "sum reduction");
    DG_CUDA(c, cudaMemcpyAsync(out, c->ctl->sums, 5 * sizeof(double), cudaMemcpyDeviceToHost, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    return DG_OK;
}

int32_t dg_get_stream(dg_ctx *c, void **stream) {
    if (!c || !stream) return fail(c, DG_ERR_INVALID, "null argument");
    *stream = (void *)c->stream;
    return DG_OK;
}

int32_t dg_step_launch_shape(dg_ctx *c, int32_t *blocks, int32_t *threads, int32_t *chunk) {
    if (!c) return DG_ERR_INVALID;
    const int ch = auto_chunk(c);
    const int b = step_grid_blocks(c->nx, c->ny, c->nz, c->kind, ch);
    if (blocks) *blocks = b;
    if (threads) *threads = step_threads(c->kind);
    if (chunk) *chunk = ch;
    return DG_OK;
}

int32_t dg_set_chunk(dg_ctx *c, int32_t chunk) {
    if (!c || chunk < 0) return fail(c, DG_ERR_INVALID, "bad argument");
    c->chunk = chunk;
    return DG_OK;
}

int32_t dg_status(dg_ctx *c, uint32_t *flags) {
    if (!c || !flags) return fail(c, DG_ERR_INVALID, "null argument");
    int r;
    if ((r = use_device(c)) != DG_OK) return r;
    unsigned f = 0;
    DG_CUDA(c, cudaMemcpyAsync(&f, &c->ctl->flags, sizeof(f), cudaMemcpyDeviceToHost, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    *flags = f;
    return DG_OK;
}

const char *dg_last_error(const dg_ctx *c) {
    return c ? c->err.c_str() : g_create_err.c_str();
}

}  // extern "C"
