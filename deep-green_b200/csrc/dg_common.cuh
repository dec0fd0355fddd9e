// dg_common.cuh -- pieces shared by the step kernels: PTX wrappers for
// mbarrier and TMA, the ghost-image rules of the reference's boundary
// conditions, and the fixed-order reduction of per-block partials.
#pragma once
#include <cstdio>

#include "dg_kernels.cuh"

namespace dg {

// ---------------------------------------------------------------------------
// PTX helpers (mbarrier, TMA)
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint32_t smem_u32(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_inval(uint64_t *bar) {
    asm volatile("mbarrier.inval.shared::cta.b64 [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ void fence_mbar_init() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void fence_proxy_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

// Bounded wait on an mbarrier phase: false after ~`budget` SM clocks; a
// negative budget gives up without waiting (the timeout test hook).
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity, long long budget) {
    if (budget < 0) return false;
    const uint32_t addr = smem_u32(bar);
    auto try_wait = [&]() {
        uint32_t ok;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
            "selp.u32 %0, 1, 0, p;\n\t}"
            : "=r"(ok)
            : "r"(addr), "r"(parity)
            : "memory");
        return ok != 0;
    };
    if (try_wait()) return true;   // the usual case: no clock reads
    const long long t0 = clock64();
    while (true) {
        if (try_wait()) return true;
        if (clock64() - t0 > budget) return false;
    }
}

// 4-D tiled TMA load (z, y, x, field) into shared memory, completing on bar.
__device__ __forceinline__ void tma_load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2,
                                            int c3, uint64_t *bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
        "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
        : "memory");
}

constexpr long long kWaitBudget = 4000000000LL;  // ~2 s of SM clock

// The budget a step kernel gives its waits for staged planes: the grid's own
// (a context created with DG_DEBUG_WAIT_BUDGET set; negative: give up at
// once) or the default (0).  Waits that let copies in flight land before a
// block exits keep kWaitBudget.
template <class A> __device__ __forceinline__ long long wait_budget_of(const A &a) {
    return a.wait_budget != 0 ? a.wait_budget : kWaitBudget;
}

// ---------------------------------------------------------------------------
// Ghost images: the set of cells (interior cell itself plus ghosts) that
// hold a copy of interior coordinate c along one axis of extent n
// (boundaries.rs / handle_walls source rules, inverted).  flip[i] = 1 when
// the copy is a wall mirror (normal momentum negated).
// ---------------------------------------------------------------------------
__host__ __device__ __forceinline__ int axis_images(int c, int n, int lo, int hi, int out[4], int flip[4]) {
    int m = 0;
    out[m] = c; flip[m++] = 0;
    if (lo == kPeriodic) {
        if (c == n - 4) { out[m] = 0; flip[m++] = 0; }
        if (c == n - 3) { out[m] = 1; flip[m++] = 0; }
    } else if (lo == kOutflow) {
        if (c == 2) { out[m] = 0; flip[m++] = 0; out[m] = 1; flip[m++] = 0; }
    } else {
        if (c == 2) { out[m] = 1; flip[m++] = 1; }
        if (c == 3) { out[m] = 0; flip[m++] = 1; }
    }
    if (hi == kPeriodic) {
        if (c == 2 && m < 4) { out[m] = n - 2; flip[m++] = 0; }
        if (c == 3 && m < 4) { out[m] = n - 1; flip[m++] = 0; }
    } else if (hi == kOutflow) {
        if (c == n - 3 && m < 3) { out[m] = n - 2; flip[m++] = 0; out[m] = n - 1; flip[m++] = 0; }
    } else {
        if (c == n - 3 && m < 4) { out[m] = n - 2; flip[m++] = 1; }
        if (c == n - 4 && m < 4) { out[m] = n - 1; flip[m++] = 1; }
    }
    return m;
}

// Source interior coordinate of ghosted coordinate g along one axis, and
// whether the copy is a wall mirror.
__host__ __device__ __forceinline__ int axis_source(int g, int n, int lo, int hi, int *flip) {
    *flip = 0;
    if (g >= 2 && g <= n - 3) return g;
    if (g < 2) {
        if (lo == kPeriodic) return g == 0 ? n - 4 : n - 3;
        if (lo == kOutflow) return 2;
        *flip = 1;
        return g == 1 ? 2 : 3;
    }
    if (hi == kPeriodic) return g == n - 2 ? 2 : 3;
    if (hi == kOutflow) return n - 3;
    *flip = 1;
    return g == n - 2 ? n - 3 : n - 4;
}

// Modes of final_reduce.
enum ReduceMode { kSumsOnly = 0, kSetDt = 1, kAdvance = 2 };

template <class T>
__device__ void final_reduce(const GridArgs<T> &a, int tid, int nt, double *red, int mode, int nb);

// Block-level reduction of (sums, min wave time, NaN flag) into
// a.part[idx] in a fixed order.  Returns true, in every thread, in the last
// of the nb blocks (work items) of this grid to finish.
template <class T>
__device__ bool block_partial(const GridArgs<T> &a, double sum[5], double wm, unsigned nanf, int tid, int nt,
                              double *red, int *is_last, int idx, int nb) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int f = 0; f < 5; ++f) sum[f] += __shfl_xor_sync(0xffffffffu, sum[f], o);
        wm = fmin(wm, __shfl_xor_sync(0xffffffffu, wm, o));
        nanf |= __shfl_xor_sync(0xffffffffu, nanf, o);
    }
    const int warp = tid >> 5, lane = tid & 31;
    if (lane == 0) {
        for (int f = 0; f < 5; ++f) red[warp * 7 + f] = sum[f];
        red[warp * 7 + 5] = wm;
        red[warp * 7 + 6] = (double)nanf;
    }
    __syncthreads();
    if (tid == 0) {
        Partial p;
        for (int f = 0; f < 5; ++f) p.sums[f] = 0;
        p.wmin = INFINITY;
        p.nan = 0;
        for (int w = 0; w < nt / 32; ++w) {
            for (int f = 0; f < 5; ++f) p.sums[f] += red[w * 7 + f];
            p.wmin = fmin(p.wmin, red[w * 7 + 5]);
            p.nan |= red[w * 7 + 6] != 0.0;
        }
        p.pad = 0;
        a.part[idx] = p;
        __threadfence();
        const unsigned ticket = atomicAdd(&a.ctl->counter, 1u);
        *is_last = ticket == (unsigned)nb - 1;
    }
    __syncthreads();
    return *is_last != 0;
}

// Fixed-order reduction of a launch's partials by its last block.
// kAdvance: a step finished -> record its dt, set the next dt, step += 1;
// kSetDt: a state was just set -> dt of the coming step; kSumsOnly: sums.
template <class T>
__device__ void final_reduce(const GridArgs<T> &a, int tid, int nt, double *red, int mode, int nb) {
    double acc[5] = {0, 0, 0, 0, 0};
    double wm = INFINITY;
    unsigned nanf = 0;
    for (int b = tid; b < nb; b += nt) {
        const volatile Partial *p = a.part + b;
        for (int f = 0; f < 5; ++f) acc[f] += p->sums[f];
        wm = fmin(wm, p->wmin);
        nanf |= p->nan;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
        for (int f = 0; f < 5; ++f) acc[f] += __shfl_xor_sync(0xffffffffu, acc[f], o);
        wm = fmin(wm, __shfl_xor_sync(0xffffffffu, wm, o));
        nanf |= __shfl_xor_sync(0xffffffffu, nanf, o);
    }
    const int warp = tid >> 5, lane = tid & 31, nw = nt >> 5;
    __syncthreads();
    if (lane == 0) {
        for (int f = 0; f < 5; ++f) red[warp * 7 + f] = acc[f];
        red[warp * 7 + 5] = wm;
        red[warp * 7 + 6] = (double)nanf;
    }
    __syncthreads();
    if (tid == 0) {
        double tot[5] = {0, 0, 0, 0, 0};
        double w = INFINITY;
        unsigned nn = 0;
        for (int i = 0; i < nw; ++i) {
            for (int f = 0; f < 5; ++f) tot[f] += red[i * 7 + f];
            w = fmin(w, red[i * 7 + 5]);
            nn |= red[i * 7 + 6] != 0.0;
        }
        DevCtl *c = a.ctl;
        const unsigned long long st = c->step;
        // calc_timestep: CFL * min, or CFL * 1.0 when a NaN was seen
        // (physics.rs:191-195), evaluated in the step's precision.
        const T dtn = nn ? (T)a.k.cfl * T(1.0) : (T)a.k.cfl * (T)w;
        for (int f = 0; f < 5; ++f) c->sums[f] = tot[f];
        if (mode != kSumsOnly && nn) c->flags |= kStatusNonFinite;
        if (mode == kAdvance) {
            c->hist[st % kHist] = c->dt[st & 1];
            c->dt[(st + 1) & 1] = (double)dtn;
            c->step = st + 1;
        } else if (mode == kSetDt) {
            c->dt[st & 1] = (double)dtn;
        }
        c->counter = 0;
        __threadfence();
    }
}

}  // namespace dg
