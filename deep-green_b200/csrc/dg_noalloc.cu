// dg_noalloc.cu -- dg_compute_step_noalloc: one Euler step on memory the
// caller owns, with no device allocation by this library.
//
// Why it exists: some programs cannot let a library call cudaMalloc.  A host
// application that hands all device memory to its own pool allocator (and
// sizes that pool at start-up) cannot have a second allocator take memory
// behind its back, and a plug-in running inside such a program has no say
// over allocation at all.  The context API (dg_create) allocates its state
// buffers and its scratch; this entry point allocates nothing: the caller
// passes the input and output states, and the step's scratch memory (the
// step control block and the per-block partial results of the dt / sum
// reductions) lives in a fixed-size array in the library's own device image.
//
// Limits and rules:
//   * the scratch array holds the control block plus kMaxBlocks per-block
//     partials (1 MiB in total); grids that need more blocks are rejected
//     with DG_ERR_INVALID;
//   * every GPU that loads the library holds this 1 MiB until the process
//     exits;
//   * all calls share the one array (per device): calls that overlap on the
//     GPU, from different host threads or on different streams, race and
//     give wrong results;
//   * the first call on a device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.
#include <cudaTypedefs.h>

#include <cstddef>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/deepgreen.h"
#include "dg_kernels.cuh"

namespace dg {
namespace {

constexpr size_t kNoAllocScratchBytes = 1u << 20;
constexpr size_t kPartialOffset = (sizeof(DevCtl) + 255) / 256 * 256;
constexpr int kMaxBlocks = (int)((kNoAllocScratchBytes - kPartialOffset) / sizeof(Partial));

// The scratch.  In host code this name is only a stand-in for the device
// symbol: its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[64];   // device address of g_noalloc_scratch, per device

// errors are reported through dg_last_error(NULL)
int fail(int code, const std::string &m) {
    set_global_error(m);
    return code;
}

// Set-up, once per device, with that device current.
int scratch_address(int dev, void **out) {
    if (dev < 0 || dev >= 64) return fail(DG_ERR_INVALID, "device ordinal out of range");
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return fail(DG_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return DG_OK;
}

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

template <class T>
GridArgs<T> args_for(const dg_sim_info *info, const void *src, void *dst, void *scratch) {
    GridArgs<T> a;
    a.src = static_cast<const T *>(src);
    a.dst = static_cast<T *>(dst);
    a.nx = info->nx + 4;
    a.ny = info->ny + 4;
    a.nz = info->nz + 4;
    a.pitch = a.nz;
    a.fstride = (long long)a.nx * a.ny * a.nz;
    set_boundaries(a, info->bcs);
    a.gravity = info->gravity;
    a.limiter = info->limiter;
    a.nparts = 0;
    a.wait_budget = 0;
    const T ds = (T)info->ds;
    a.k.ds = ds;
    a.k.vol = ds * ds * ds;
    a.k.inv_vol = T(1) / a.k.vol;
    a.k.gamma = (T)info->gamma;
    a.k.gm1 = a.k.gamma - T(1);
    a.k.inv_gm1 = T(1) / a.k.gm1;
    a.k.half_ds = ds / T(2);
    a.k.two_ds = T(2) * ds;
    a.k.inv_ds = T(1) / ds;
    a.k.inv_2ds = T(1) / (T(2) * ds);
    a.k.cfl = (T)info->cfl;
    a.k.g = (T)info->g;
    a.ctl = static_cast<DevCtl *>(scratch);
    a.part = reinterpret_cast<Partial *>(static_cast<unsigned char *>(scratch) + kPartialOffset);
    return a;
}

template <class T>
int run(const dg_sim_info *info, int kind, void *cons_in, void *cons_out, double *dt_used, cudaStream_t st,
        void *scratch) {
    const int elem = (int)sizeof(T);
    GridArgs<T> a = args_for<T>(info, cons_in, cons_out, scratch);
    const int chunk = choose_chunk(a.nx, a.ny, a.nz, kind);
    const int blocks = step_grid_blocks(a.nx, a.ny, a.nz, kind, chunk);
    if (blocks > kMaxBlocks || kReduceBlocks > kMaxBlocks)
        return fail(DG_ERR_INVALID, "grid too large for the no-allocation scratch (" + std::to_string(blocks) +
                                        " blocks > " + std::to_string(kMaxBlocks) + ")");
    auto fn = encode_fn();
    if (!fn) return fail(DG_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
    CUtensorMap map;
    const int ty = step_tile_rows(kind);
    cuuint64_t dims[4] = {(cuuint64_t)a.nz, (cuuint64_t)a.ny, (cuuint64_t)a.nx, 5};
    cuuint64_t strides[3] = {(cuuint64_t)a.pitch * elem, (cuuint64_t)a.pitch * a.ny * elem,
                             (cuuint64_t)a.fstride * elem};
    cuuint32_t box[4] = {(cuuint32_t)step_box_cols(kind), (cuuint32_t)(ty + 4), 1, 5};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    if (fn(&map, elem == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, cons_in, dims,
           strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
           CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) != CUDA_SUCCESS)
        return fail(DG_ERR_INVALID, "cuTensorMapEncodeTiled rejected the state layout");

    // the control fields of the scratch must start at zero on every call
    cudaError_t e = cudaMemsetAsync(scratch, 0, offsetof(DevCtl, hist), st);
    if (e == cudaSuccess) e = launch_fill_ghosts<T>(a, static_cast<T *>(cons_in), st);
    if constexpr (sizeof(T) == 4) {
        if (kind == kFastF32) {
            if (e == cudaSuccess) e = launch_reduce_policy<float, false>(a, 1, st);
            if (e == cudaSuccess) e = launch_sweep(a, &map, chunk, st);
        } else {
            if (e == cudaSuccess) e = launch_reduce_policy<float, true>(a, 1, st);
            if (e == cudaSuccess) e = launch_step_policy<float, true>(a, &map, info->limiter, chunk, st);
        }
    } else {
        if (e == cudaSuccess) e = launch_reduce_policy<double, true>(a, 1, st);
        if (e == cudaSuccess)
            e = kind == kFastF64 ? launch_sweep(a, &map, chunk, st)
                                 : launch_step_policy<double, true>(a, &map, info->limiter, chunk, st);
    }
    if (e != cudaSuccess) return fail(DG_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
    if (dt_used) {
        // dt of the step = history entry 0 (step counter started at zero)
        e = cudaMemcpyAsync(dt_used, static_cast<unsigned char *>(scratch) + offsetof(DevCtl, hist), sizeof(double),
                            cudaMemcpyDeviceToHost, st);
        unsigned flags = 0;
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&flags, static_cast<unsigned char *>(scratch) + offsetof(DevCtl, flags),
                                sizeof(flags), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail(DG_ERR_CUDA, std::string("read-back: ") + cudaGetErrorString(e));
        if (flags & kStatusTimeout) return fail(DG_ERR_TIMEOUT, "a device-side wait timed out; output invalid");
    }
    return DG_OK;
}

}  // namespace
}  // namespace dg

// Restores the calling thread's current device on every return path: the
// callers of this entry point manage their own devices.
struct DeviceGuard {
    int prev = -1;
    ~DeviceGuard() {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

extern "C" int32_t dg_compute_step_noalloc(const dg_sim_info *info, void *cons_in, void *cons_out,
                                           double *dt_used, void *stream) {
    using namespace dg;
    if (!info || !cons_in || !cons_out) return fail(DG_ERR_INVALID, "null argument");
    if (info->nghosts != 2 || info->nx < 2 || info->ny < 2 || info->nz < 2)
        return fail(DG_ERR_INVALID, "need nghosts == 2 and >= 2 interior cells per axis");
    if (!(info->ds > 0) || !(info->gamma > 1) || !(info->cfl > 0))
        return fail(DG_ERR_INVALID, "ds > 0, gamma > 1, cfl > 0 required");
    if (info->precision != DG_F32 && info->precision != DG_F64) return fail(DG_ERR_INVALID, "bad precision");
    if (info->limiter != DG_LIMITER_NONE && info->limiter != DG_LIMITER_MINMOD) return fail(DG_ERR_INVALID, "bad limiter");
    if (info->rounding != DG_ROUNDING_DEFAULT && info->rounding != DG_ROUNDING_REFERENCE &&
        info->rounding != DG_ROUNDING_FAST)
        return fail(DG_ERR_INVALID, "bad rounding policy");
    for (int ax = 0; ax < 3; ++ax) {
        const int lo = info->bcs[2 * ax], hi = info->bcs[2 * ax + 1];
        if (!valid_bc_pair(lo, hi)) return fail(DG_ERR_INVALID, "bad boundary types (periodic faces come in pairs)");
    }
    const int elem = info->precision == DG_F64 ? 8 : 4;
    if (((size_t)(info->nz + 4) * elem) % 16 != 0)
        return fail(DG_ERR_INVALID, "(nz + 4) * element size must be a multiple of 16 bytes for the TMA copies");
    if ((reinterpret_cast<uintptr_t>(cons_in) | reinterpret_cast<uintptr_t>(cons_out)) & 15)
        return fail(DG_ERR_INVALID, "state pointers must be 16-byte aligned");
    if (cons_in == cons_out) return fail(DG_ERR_INVALID, "input and output states must differ");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(DG_ERR_NO_DEVICE, "no current CUDA device");
    DeviceGuard guard;
    if (dev != info->device) {
        if (cudaSetDevice(info->device) != cudaSuccess) return fail(DG_ERR_NO_DEVICE, "cannot select the requested device");
        guard.prev = dev;
    }
    void *scratch = nullptr;
    int r = scratch_address(info->device, &scratch);
    if (r != DG_OK) return r;
    const bool exact = info->rounding == DG_ROUNDING_REFERENCE || (elem == 8 && info->rounding == DG_ROUNDING_DEFAULT);
    const int kind = elem == 8 ? (exact ? kRefF64 : kFastF64) : (exact ? kRefF32 : kFastF32);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    return elem == 8 ? run<double>(info, kind, cons_in, cons_out, dt_used, st, scratch)
                     : run<float>(info, kind, cons_in, cons_out, dt_used, st, scratch);
}

// Status flags left in the shared scratch by the last no-allocation step on
// `device` (the flags word of its control block; the next call clears it).
extern "C" int32_t dg_noalloc_status(int32_t device, uint32_t *flags) {
    using namespace dg;
    if (!flags) return fail(DG_ERR_INVALID, "null argument");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || device < 0 || device >= ndev)
        return fail(DG_ERR_NO_DEVICE, "no CUDA device with that ordinal");
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return fail(DG_ERR_NO_DEVICE, "no current CUDA device");
    DeviceGuard guard;
    if (dev != device) {
        if (cudaSetDevice(device) != cudaSuccess) return fail(DG_ERR_NO_DEVICE, "cannot select the requested device");
        guard.prev = dev;
    }
    void *scratch = nullptr;
    int r = scratch_address(device, &scratch);
    if (r != DG_OK) return r;
    unsigned f = 0;
    const cudaError_t e = cudaMemcpy(&f, static_cast<unsigned char *>(scratch) + offsetof(DevCtl, flags), sizeof(f),
                                     cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail(DG_ERR_CUDA, std::string("read-back: ") + cudaGetErrorString(e));
    *flags = f;
    return DG_OK;
}
