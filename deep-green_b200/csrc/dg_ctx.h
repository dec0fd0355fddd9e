// dg_ctx.h -- the context behind the opaque dg_ctx handle of deepgreen.h and
// the small helpers that the C-ABI sources share (internal header).
#pragma once
#include <string>

#include "../../include/deepgreen.h"
#include "dg_kernels.cuh"

struct dg_ctx {
    dg_sim_info info;
    int elem;                  // 4 or 8
    int nx, ny, nz;            // ghosted extents
    int pitch;                 // z-row pitch in elements
    long long fstride;         // elements per field
    size_t state_bytes;
    void *buf[2];
    int cur;                   // buffer holding the current state
    bool has_state;
    unsigned long long steps;  // steps since the state was set
    dg::DevCtl *ctl;
    dg::Partial *part;
    int part_cap;
    void *prim_scratch;        // lazily allocated: dense primitives for dg_get_primitives
    CUtensorMap tmap[2];
    cudaStream_t stream;
    int chunk;                 // 0 = automatic
    bool exact;                // reference-rounding policy
    int kind;                  // KernelKind of the step kernel
    long long wait_budget;     // 0: default; from DG_DEBUG_WAIT_BUDGET (tests of the timeout path)
    std::string err;
};

namespace dg {

inline int fail(dg_ctx *c, int code, const std::string &msg) {
    if (c) c->err = msg;
    return code;
}

inline int cuda_fail(dg_ctx *c, cudaError_t e, const char *where) {
    return fail(c, DG_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

#define DG_CUDA(c, expr)                                         \
    do {                                                         \
        cudaError_t e_ = (expr);                                 \
        if (e_ != cudaSuccess) return cuda_fail((c), e_, #expr); \
    } while (0)

template <class T> inline GridArgs<T> grid_args(const dg_ctx *c, const void *src, void *dst) {
    GridArgs<T> a;
    a.src = static_cast<const T *>(src);
    a.dst = static_cast<T *>(dst);
    a.nx = c->nx;
    a.ny = c->ny;
    a.nz = c->nz;
    a.pitch = c->pitch;
    a.fstride = c->fstride;
    set_boundaries(a, c->info.bcs);
    a.gravity = c->info.gravity;
    a.limiter = c->info.limiter;
    a.nparts = 0;
    a.wait_budget = c->wait_budget;
    const T ds = (T)c->info.ds;
    a.k.ds = ds;
    a.k.vol = ds * ds * ds;
    a.k.inv_vol = T(1) / a.k.vol;
    a.k.gamma = (T)c->info.gamma;
    a.k.gm1 = a.k.gamma - T(1);
    a.k.inv_gm1 = T(1) / a.k.gm1;
    a.k.half_ds = ds / T(2);
    a.k.two_ds = T(2) * ds;
    a.k.inv_ds = T(1) / ds;
    a.k.inv_2ds = T(1) / (T(2) * ds);
    a.k.cfl = (T)c->info.cfl;
    a.k.g = (T)c->info.g;
    a.ctl = c->ctl;
    a.part = c->part;
    return a;
}

// Implemented in dg_capi.cu.
int ctx_enqueue(dg_ctx *c, int nsteps);     // n plain steps, asynchronous
int ctx_begin_state(dg_ctx *c);             // select the device, reset the step control block
int ctx_finish_state(dg_ctx *c);            // ghosts + dt of the current buffer; state valid, 0 steps
int ctx_check_flags(dg_ctx *c);             // synchronise and report a device-side timeout

}  // namespace dg
