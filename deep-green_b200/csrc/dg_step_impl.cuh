// dg_step_impl.cuh -- the fused Euler step for sm_100a and its helper
// kernels, templated on precision and arithmetic policy (dg_physics.cuh).
// Instantiated by dg_step_fast.cu (fused multiply-add allowed) and
// dg_step_ref.cu (compiled with --fmad=false: reference rounding).
//
// One launch = one compute_step of the reference (deep-green
// src/rs/src/physics.rs:595-681).  The reference runs ten passes over 45
// full arrays (primitives, ghost fills, gradients, predictor, three flux
// sweeps, flux ghosts, update).  Here each CTA owns a 32 (z) x TY (y)
// column of cells and marches along x.  Per x-plane:
//   (a) one TMA copy brings the 5 conserved fields of a (TY+4) x 36 region
//       (2-cell halo) into a shared-memory ring; converted to primitives in
//       place;
//   (b) slopes (central or minmod) and the half-step predictor for the
//       plane's cells plus a 1-cell cross-shaped halo;
//   (c) the x-face flux of the column (kept in registers from plane to
//       plane), (d) y- and z-face fluxes of the plane, each face once;
//   (e) conservative update of the previous plane, written straight to the
//       output state together with its ghost-cell images;
//   (f) the epilogue folds ds/(c_s+|v|) of the new state (next dt) and FP64
//       conservation sums into per-block partials; the last block reduces
//       them in a fixed order.
// Boundary semantics of the reference's ghost updates for the derived
// arrays (boundaries.rs:5-195, handle_walls 197-407) are reproduced on the
// fly:
//   PERIODIC  ghost gradients/predictions/fluxes are computed from the
//             ghost primitives (identical to the reference's copies);
//   OUTFLOW   the ghost cell takes the gradient and prediction of the first
//             interior cell; at the lower face the face flux equals the
//             next face's (the reference copies flux[2] into flux[1], so
//             cell 2 sees no divergence along that axis);
//   WALL      ghost gradients are computed from the mirrored primitives,
//             the ghost prediction is the mirror of the interior one.
// Ghost layers of the state itself are kept up to date in memory (every
// updated cell also writes its periodic/outflow/wall images), so the TMA
// boxes need no fix-up.
#pragma once
#include <cstdio>

#include "dg_common.cuh"
#include "dg_host.h"

namespace dg {

// ---------------------------------------------------------------------------
// Shared-memory layout of the step kernel
// ---------------------------------------------------------------------------
template <class T, int TY, int R> struct StepSmem {
    static constexpr int RY = TY + 4;                       // staged rows
    static constexpr int kFieldElems = RY * kRZ;            // one field of one plane
    static constexpr int kBoxBytes = 5 * kFieldElems * (int)sizeof(T);
    static constexpr int kSlotElems = ((kBoxBytes + 127) / 128) * 128 / (int)sizeof(T);
    static constexpr int SY = TY + 2, SZ = kTZ + 2;         // predicted-state rectangle
    static constexpr int kRect = SY * SZ;

    T ring[R * kSlotElems];      // TMA destinations; primitives after conversion
    T xt[5 * kRect];             // predicted primitives
    T gy[5 * kRect];             // y-slopes
    T gz[5 * kRect];             // z-slopes
    T fy[2][5 * (TY + 1) * kTZ]; // y-face fluxes, double-buffered by plane parity
    T fz[2][5 * TY * (kTZ + 1)]; // z-face fluxes, double-buffered by plane parity
    uint64_t bar[R];
    double red[(TY * kTZ / 32) * 7];
    int abort_flag;
    int is_last;
};

template <class T, int TY, int LIM, int R, bool EXACT>
struct StepKernel {
    using S = StepSmem<T, TY, R>;
    using Ph = Phys<T, EXACT>;
    static constexpr int NT = TY * kTZ;

    // primitive f of region cell (ry, rz) in ring slot `slot`
    static __device__ __forceinline__ T &P(S &s, int slot, int f, int ry, int rz) {
        return s.ring[slot * S::kSlotElems + f * S::kFieldElems + ry * kRZ + rz];
    }
    static __device__ __forceinline__ int ridx(int sy, int sz) { return sy * S::SZ + sz; }

    // Slopes along x, y, z of the 5 primitives of region cell (ry, rz) of
    // the plane in slot s0 (neighbour planes in sm, sp).
    static __device__ __forceinline__ void slopes(S &s, int sm, int s0, int sp, int ry, int rz,
                                                  const Consts<T> &k, T w[5], T gx[5], T gy[5], T gz[5]) {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            const T c = P(s, s0, f, ry, rz);
            w[f] = c;
            gx[f] = Ph::template slope<LIM>(P(s, sm, f, ry, rz), c, P(s, sp, f, ry, rz), k);
            gy[f] = Ph::template slope<LIM>(P(s, s0, f, ry - 1, rz), c, P(s, s0, f, ry + 1, rz), k);
            gz[f] = Ph::template slope<LIM>(P(s, s0, f, ry, rz - 1), c, P(s, s0, f, ry, rz + 1), k);
        }
    }

    // Gradients and predicted state stored for region cell (ry, rz), with
    // the ghost-layer-1 rules of the y and z boundaries.  Returns the
    // x-slopes and prediction of the stored cell in gx_out / xt_out.
    static __device__ __forceinline__ void cell_state(S &s, const GridArgs<T> &a, int sm, int s0, int sp,
                                                      int ry, int rz, int gyc, int gzc, T dt, T gx_out[5],
                                                      T xt_out[5]) {
        const Consts<T> &k = a.k;
        T w[5], gx[5], gy[5], gz[5];
        // Which boundary rule applies (at most one axis for cells used).
        int rule = kPeriodic, axis = 0, nry = ry, nrz = rz;
        if (gyc == 1) { rule = a.bc[2]; axis = 2; nry = ry + 1; }
        else if (gyc == a.ny - 2) { rule = a.bc[3]; axis = 2; nry = ry - 1; }
        else if (gzc == 1) { rule = a.bc[4]; axis = 3; nrz = rz + 1; }
        else if (gzc == a.nz - 2) { rule = a.bc[5]; axis = 3; nrz = rz - 1; }

        if (rule == kOutflow) {
            // ghost takes slopes and prediction of the interior neighbour
            slopes(s, sm, s0, sp, nry, nrz, k, w, gx, gy, gz);
            Ph::predict(w, gx, gy, gz, dt, k, xt_out);
        } else {
            slopes(s, sm, s0, sp, ry, rz, k, w, gx, gy, gz);
            if (rule == kWall) {
                // slopes from the mirrored ghost primitives; prediction =
                // mirror of the interior neighbour's (normal velocity negated)
                T w2[5], gx2[5], gy2[5], gz2[5];
                slopes(s, sm, s0, sp, nry, nrz, k, w2, gx2, gy2, gz2);
                Ph::predict(w2, gx2, gy2, gz2, dt, k, xt_out);
                xt_out[axis] = -xt_out[axis];
            } else {
                Ph::predict(w, gx, gy, gz, dt, k, xt_out);
            }
        }
        const int r = ridx(ry - 1, rz - 1);
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            s.xt[f * S::kRect + r] = xt_out[f];
            s.gy[f * S::kRect + r] = gy[f];
            s.gz[f * S::kRect + r] = gz[f];
            gx_out[f] = gx[f];
        }
    }

    // y-face flux between rectangle cells (sy-1, sz) [lower] and (sy, sz);
    // heat: the face of a lower conducting wall.
    static __device__ __forceinline__ void yface(S &s, int sy, int sz, const Consts<T> &k, T F[5], bool heat) {
        T xl[5], gl[5], xu[5], gu[5];
        const int rl = ridx(sy - 1, sz), ru = ridx(sy, sz);
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            xl[f] = s.xt[f * S::kRect + rl];
            gl[f] = s.gy[f * S::kRect + rl];
            xu[f] = s.xt[f * S::kRect + ru];
            gu[f] = s.gy[f * S::kRect + ru];
        }
        Ph::face(xl, gl, xu, gu, 2, 0, 0, 0, k, F, heat);
    }

    // z-face flux between rectangle cells (sy, sz-1) and (sy, sz); klow is
    // the ghosted z index of the lower cell (gravity height).
    static __device__ __forceinline__ void zface(S &s, int sy, int sz, const GridArgs<T> &a, int klow, T F[5]) {
        T xl[5], gl[5], xu[5], gu[5];
        const int rl = ridx(sy, sz - 1), ru = ridx(sy, sz);
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            xl[f] = s.xt[f * S::kRect + rl];
            gl[f] = s.gz[f * S::kRect + rl];
            xu[f] = s.xt[f * S::kRect + ru];
            gu[f] = s.gz[f * S::kRect + ru];
        }
        Ph::face(xl, gl, xu, gu, 3, a.gravity, grav_klow(klow, a.nz, a.bc[4]), a.nz, a.k, F, klow == 1 && (a.heat & 4));
    }

    static __device__ void run(const GridArgs<T> &a, const CUtensorMap *tmap, int chunk, unsigned char *raw) {
        S &s = *reinterpret_cast<S *>(raw);
        const Consts<T> &k = a.k;
        const int lz = threadIdx.x, ly = threadIdx.y;
        const int tid = ly * kTZ + lz;

        const int tiles_z = (a.nz - 4 + kTZ - 1) / kTZ;
        const int tiles_y = (a.ny - 4 + TY - 1) / TY;
        int b = blockIdx.x;
        const int tz = b % tiles_z; b /= tiles_z;
        const int ty = b % tiles_y; b /= tiles_y;
        const int cx = b;
        const int y0 = 2 + ty * TY, z0 = 2 + tz * kTZ;     // first interior cell of the tile
        const int xs = 2 + cx * chunk;
        const int xe = min(xs + chunk, a.nx - 2);          // planes [xs, xe) are updated
        const int np = xe - xs + 4;                        // planes xs-2 .. xe+1 are staged
        const int gyo = y0 + ly, gzo = z0 + lz;            // own cell (ghosted coordinates)
        const bool own_valid = gyo <= a.ny - 3 && gzo <= a.nz - 3;

        const unsigned step = (unsigned)a.ctl->step;
        const T dt = (T)a.ctl->dt[step & 1];

        // a previous launch timed out: the state is invalid, do nothing (the
        // flag is read once, so that every thread takes the same branch)
        if (tid == 0) {
            s.abort_flag = (*(volatile unsigned *)&a.ctl->flags & kStatusTimeout) ? 2 : 0;
            if (!s.abort_flag) {
                for (int i = 0; i < R; ++i) mbar_init(&s.bar[i], 1);
                fence_mbar_init();
            }
        }
        __syncthreads();
        if (s.abort_flag) return;
        if (tid == 0) {
            for (int l = 0; l < R && l < np; ++l) {
                mbar_expect_tx(&s.bar[l], S::kBoxBytes);
                tma_load_4d(&s.ring[l * S::kSlotElems], tmap, z0 - 2, y0 - 2, xs - 2 + l, 0, &s.bar[l]);
            }
        }

        // ghost images of the own column along y and z (fixed per thread)
        int yimg[4], yflp[4], zimg[4], zflp[4];
        const int nyi = own_valid ? axis_images(gyo, a.ny, a.bc[2], a.bc[3], yimg, yflp) : 0;
        const int nzi = own_valid ? axis_images(gzo, a.nz, a.bc[4], a.bc[5], zimg, zflp) : 0;

        T cA[5], cB[5], cC[5];
        T xt_prev[5], gx_prev[5], fx_lo[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) { cA[f] = cB[f] = cC[f] = xt_prev[f] = gx_prev[f] = fx_lo[f] = T(0); }
        double sum[5] = {0, 0, 0, 0, 0};
        T wmin = T(INFINITY);
        unsigned nanf = 0;

        constexpr int HR = (TY + 4) * kRZ - TY * kTZ;   // halo cells of the staged region
        constexpr int HC = 2 * kTZ + 2 * TY;            // halo cells of the predicted rectangle

        // (a) wait for staged plane l and convert it to primitives in place;
        // the own cell's conserved values go to `keep`.
        auto convert = [&](int l, T keep[5]) -> bool {
            const int slot = l % R;
            if (!mbar_wait(&s.bar[slot], (l / R) & 1, wait_budget_of(a))) return false;
            {
                const int ry = ly + 2, rz = lz + 2;
                T u[5], w[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) u[f] = P(s, slot, f, ry, rz);
                Ph::prim(u, w, k);
#pragma unroll
                for (int f = 0; f < 5; ++f) { P(s, slot, f, ry, rz) = w[f]; keep[f] = u[f]; }
            }
            for (int h = tid; h < HR; h += NT) {
                int ry, rz;
                if (h < 4 * kRZ) {
                    const int r4 = h / kRZ;
                    rz = h % kRZ;
                    ry = r4 < 2 ? r4 : TY + r4;
                } else {
                    const int j = h - 4 * kRZ, c4 = j & 3;
                    ry = 2 + (j >> 2);
                    rz = c4 < 2 ? c4 : kTZ + c4;
                }
                T u[5], w[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) u[f] = P(s, slot, f, ry, rz);
                Ph::prim(u, w, k);
#pragma unroll
                for (int f = 0; f < 5; ++f) P(s, slot, f, ry, rz) = w[f];
            }
            return true;
        };

        bool ok = convert(0, cA);
        if (ok) ok = convert(1, cB);
        if (!ok) s.abort_flag = 1;

        int issued = (np < R) ? np : R;   // planes whose TMA has been issued
        for (int m = xs - 1; m <= xe; ++m) {
            const int l = m - xs + 3;      // staged index of plane m+1
            if (!convert(l, cC)) s.abort_flag = 1;
            // generic writes to the slot precede the TMA that later refills it
            fence_proxy_async();
            __syncthreads();               // S1: primitives of planes m-1..m+1 ready
            if (s.abort_flag) break;

            const int sm = (l - 2) % R, s0 = (l - 1) % R, sp = l % R;
            const bool plane_upd = m >= xs && m < xe;

            // (b) own cell: slopes + prediction
            T xt_cur[5], gx_cur[5];
            cell_state(s, a, sm, s0, sp, ly + 2, lz + 2, gyo, gzo, dt, gx_cur, xt_cur);
            if (plane_upd) {
                for (int h = tid; h < HC; h += NT) {
                    int yl, zl;
                    if (h < kTZ) { yl = -1; zl = h; }
                    else if (h < 2 * kTZ) { yl = TY; zl = h - kTZ; }
                    else if (h < 2 * kTZ + TY) { yl = h - 2 * kTZ; zl = -1; }
                    else { yl = h - 2 * kTZ - TY; zl = kTZ; }
                    T gxh[5], xth[5];
                    cell_state(s, a, sm, s0, sp, yl + 2, zl + 2, y0 + yl, z0 + zl, dt, gxh, xth);
                }
            }

            // (c) x-face flux between planes m-1 and m (own column)
            T fx_hi[5] = {T(0), T(0), T(0), T(0), T(0)};
            if (m >= xs) {
                if (m == 2 && a.bc[0] == kWall) {
#pragma unroll
                    for (int f = 0; f < 5; ++f) xt_prev[f] = xt_cur[f];
                    xt_prev[1] = -xt_prev[1];
                }
                if (m == a.nx - 2) {
                    if (a.bc[1] == kOutflow) {
#pragma unroll
                        for (int f = 0; f < 5; ++f) { xt_cur[f] = xt_prev[f]; gx_cur[f] = gx_prev[f]; }
                    } else if (a.bc[1] == kWall) {
#pragma unroll
                        for (int f = 0; f < 5; ++f) xt_cur[f] = xt_prev[f];
                        xt_cur[1] = -xt_cur[1];
                    }
                }
                Ph::face(xt_prev, gx_prev, xt_cur, gx_cur, 1, 0, 0, 0, k, fx_hi, m == 2 && (a.heat & 1));
            }
            __syncthreads();               // S2: predicted rectangle ready; slot of plane m-1 free

            if (tid == 0 && issued < np) {
                const int slot = (l - 2) % R;   // plane m-1's slot
                mbar_expect_tx(&s.bar[slot], S::kBoxBytes);
                tma_load_4d(&s.ring[slot * S::kSlotElems], tmap, z0 - 2, y0 - 2, xs - 2 + issued, 0,
                            &s.bar[slot]);
                ++issued;
            } else if (issued < np) {
                ++issued;
            }

            // (d) y- and z-face fluxes of plane m, into buffer m & 1
            if (plane_upd) {
                T *fyb = s.fy[m & 1], *fzb = s.fz[m & 1];
                T F[5];
                yface(s, ly + 1, lz + 1, k, F, y0 + ly == 2 && (a.heat & 2));
#pragma unroll
                for (int f = 0; f < 5; ++f) fyb[(f * (TY + 1) + ly) * kTZ + lz] = F[f];
                zface(s, ly + 1, lz + 1, a, gzo - 1, F);
#pragma unroll
                for (int f = 0; f < 5; ++f) fzb[(f * TY + ly) * (kTZ + 1) + lz] = F[f];
                if (ly == 0) {
                    yface(s, TY + 1, lz + 1, k, F, false);
#pragma unroll
                    for (int f = 0; f < 5; ++f) fyb[(f * (TY + 1) + TY) * kTZ + lz] = F[f];
                } else if (ly == 1 && lz < TY) {
                    zface(s, lz + 1, kTZ + 1, a, z0 + kTZ - 1, F);
#pragma unroll
                    for (int f = 0; f < 5; ++f) fzb[(f * TY + lz) * (kTZ + 1) + kTZ] = F[f];
                }
            }
            __syncthreads();               // S3: face fluxes of plane m ready

            // (e) update plane m-1 with its y/z fluxes (buffer (m-1) & 1)
            const int xu = m - 1;
            if (xu >= xs && xu < xe && own_valid) {
                const T *fyb = s.fy[xu & 1], *fzb = s.fz[xu & 1];
                const bool x_out = xu == 2 && a.bc[0] == kOutflow;
                const bool y_out = gyo == 2 && a.bc[2] == kOutflow;
                const bool z_out = gzo == 2 && a.bc[4] == kOutflow;
                T u[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    // lower outflow faces repeat the next face's flux
                    // (boundaries.rs:107-111 applied to the fluxes)
                    const T fyh = fyb[(f * (TY + 1) + ly + 1) * kTZ + lz];
                    const T fyl = y_out ? fyh : fyb[(f * (TY + 1) + ly) * kTZ + lz];
                    const T fzh = fzb[(f * TY + ly) * (kTZ + 1) + lz + 1];
                    const T fzl = z_out ? fzh : fzb[(f * TY + ly) * (kTZ + 1) + lz];
                    const T fxl = x_out ? fx_hi[f] : fx_lo[f];
                    u[f] = Ph::update(cA[f], fx_hi[f], fxl, fyh, fyl, fzh, fzl, dt, k);
                }
                // (f) epilogue: next-dt wave speed and FP64 sums of the new state
                {
                    T w[5];
                    Ph::prim(u, w, k);
                    const T wd = Ph::wave_dt(w, k);
                    if (wd != wd) nanf = 1;
                    else wmin = fmin(wmin, wd);
#pragma unroll
                    for (int f = 0; f < 5; ++f) sum[f] += (double)u[f];
                }
                int ximg[4], xflp[4];
                const int nxi = axis_images(xu, a.nx, a.bc[0], a.bc[1], ximg, xflp);
                for (int ix = 0; ix < nxi; ++ix)
                    for (int iy = 0; iy < nyi; ++iy)
                        for (int iz = 0; iz < nzi; ++iz) {
                            const long long o = ((long long)ximg[ix] * a.ny + yimg[iy]) * a.pitch + zimg[iz];
                            a.dst[o] = u[0];
                            a.dst[a.fstride + o] = xflp[ix] ? -u[1] : u[1];
                            a.dst[2 * a.fstride + o] = yflp[iy] ? -u[2] : u[2];
                            a.dst[3 * a.fstride + o] = zflp[iz] ? -u[3] : u[3];
                            a.dst[4 * a.fstride + o] = u[4];
                        }
            }

            // rotate the column pipeline
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                if (m >= xs) fx_lo[f] = fx_hi[f];
                xt_prev[f] = xt_cur[f];
                gx_prev[f] = gx_cur[f];
                cA[f] = cB[f];
                cB[f] = cC[f];
            }
        }

        if (s.abort_flag) {
            // drain the copies still in flight before the CTA's shared
            // memory is released, then report the timeout
            // (the latest copy of every slot is among the last R issued; a
            // completed phase returns at once)
            if (tid == 0) {
                for (int l2 = issued > R ? issued - R : 0; l2 < issued; ++l2)
                    mbar_wait(&s.bar[l2 % R], (l2 / R) & 1, kWaitBudget);
                atomicOr(&a.ctl->flags, kStatusTimeout);
            }
            return;
        }
        block_finish(s, a, sum, wmin, nanf, tid);
    }

    // Per-block reduction and, in the launch's last block, the fixed-order
    // reduction of all partials: next dt, conservation sums, step counter.
    static __device__ void block_finish(S &s, const GridArgs<T> &a, double sum[5], T wmin, unsigned nanf,
                                        int tid) {
        double wm = (double)wmin;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
#pragma unroll
            for (int f = 0; f < 5; ++f) sum[f] += __shfl_xor_sync(0xffffffffu, sum[f], o);
            wm = fmin(wm, __shfl_xor_sync(0xffffffffu, wm, o));
            nanf |= __shfl_xor_sync(0xffffffffu, nanf, o);
        }
        const int warp = tid >> 5, lane = tid & 31;
        constexpr int NW = NT / 32;
        if (lane == 0) {
            for (int f = 0; f < 5; ++f) s.red[warp * 7 + f] = sum[f];
            s.red[warp * 7 + 5] = wm;
            s.red[warp * 7 + 6] = (double)nanf;
        }
        __syncthreads();
        if (tid == 0) {
            Partial p;
            for (int f = 0; f < 5; ++f) p.sums[f] = 0;
            p.wmin = INFINITY;
            p.nan = 0;
            for (int w = 0; w < NW; ++w) {
                for (int f = 0; f < 5; ++f) p.sums[f] += s.red[w * 7 + f];
                p.wmin = fmin(p.wmin, s.red[w * 7 + 5]);
                p.nan |= s.red[w * 7 + 6] != 0.0;
            }
            p.pad = 0;
            a.part[blockIdx.x] = p;
            __threadfence();
            const unsigned ticket = atomicAdd(&a.ctl->counter, 1u);
            s.is_last = ticket == gridDim.x - 1;
        }
        __syncthreads();
        if (!s.is_last) return;
        __threadfence();
        final_reduce<T>(a, tid, NT, s.red, kAdvance, gridDim.x);
    }
};

template <class T, int TY, int LIM, int R, bool EXACT>
__global__ void __launch_bounds__(TY * kTZ)
    step_kernel(const GridArgs<T> a, const __grid_constant__ CUtensorMap tmap, int chunk) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    StepKernel<T, TY, LIM, R, EXACT>::run(a, &tmap, chunk, smem_raw);
}

// ---------------------------------------------------------------------------
// Helper kernels (set-up and read-back; not on the per-step path)
// ---------------------------------------------------------------------------

// Reduction of the current state (dt of the first step, conservation sums).
template <class T, bool EXACT>
__global__ void __launch_bounds__(256) reduce_kernel(const GridArgs<T> a, int set_dt) {
    __shared__ double red[8 * 7];
    __shared__ int is_last;
    const int tid = threadIdx.x;
    const long long nyi = a.ny - 4, nzi = a.nz - 4;
    const long long total = (long long)(a.nx - 4) * nyi * nzi;
    double sum[5] = {0, 0, 0, 0, 0};
    double wm = INFINITY;
    unsigned nanf = 0;
    float smax = 0.0f;   // fast policy: max wave speed (NaN-propagating)
    // the cells c = blockIdx.x * 256 + tid + k * stride, with (x, y, z)
    // advanced by the stride's own decomposition (no division per cell)
    const long long stride = (long long)gridDim.x * 256;
    long long c = blockIdx.x * 256LL + tid;
    int x = (int)(c / (nyi * nzi)), y = (int)((c / nzi) % nyi), z = (int)(c % nzi);
    const int sx = (int)(stride / (nyi * nzi)), sy = (int)((stride / nzi) % nyi), sz = (int)(stride % nzi);
    for (; c < total; c += stride) {
        const long long o = ((long long)(x + 2) * a.ny + (y + 2)) * a.pitch + (z + 2);
        z += sz;
        if (z >= nzi) { z -= (int)nzi; ++y; }
        y += sy;
        if (y >= nyi) { y -= (int)nyi; ++x; }
        x += sx;
        T u[5], w[5];
        for (int f = 0; f < 5; ++f) u[f] = a.src[f * a.fstride + o];
        Phys<T, EXACT>::prim(u, w, a.k);
        if constexpr (EXACT) {
            const T wd = Phys<T, EXACT>::wave_dt(w, a.k);
            if (wd != wd) nanf = 1;
            else wm = fmin(wm, (double)wd);
        } else {
            smax = max_nan(smax, fast_speed(w[0], w[1], w[2], w[3], w[4], a.k.gamma));
        }
        for (int f = 0; f < 5; ++f) sum[f] += (double)u[f];
    }
    if constexpr (!EXACT) {
        if (smax != smax) nanf = 1;
        else wm = (double)__fdiv_rn(a.k.ds, smax);
    }
    for (int o = 16; o > 0; o >>= 1) {
        for (int f = 0; f < 5; ++f) sum[f] += __shfl_xor_sync(0xffffffffu, sum[f], o);
        wm = fmin(wm, __shfl_xor_sync(0xffffffffu, wm, o));
        nanf |= __shfl_xor_sync(0xffffffffu, nanf, o);
    }
    if ((tid & 31) == 0) {
        for (int f = 0; f < 5; ++f) red[(tid >> 5) * 7 + f] = sum[f];
        red[(tid >> 5) * 7 + 5] = wm;
        red[(tid >> 5) * 7 + 6] = (double)nanf;
    }
    __syncthreads();
    if (tid == 0) {
        Partial p;
        for (int f = 0; f < 5; ++f) p.sums[f] = 0;
        p.wmin = INFINITY;
        p.nan = 0;
        for (int w = 0; w < 8; ++w) {
            for (int f = 0; f < 5; ++f) p.sums[f] += red[w * 7 + f];
            p.wmin = fmin(p.wmin, red[w * 7 + 5]);
            p.nan |= red[w * 7 + 6] != 0.0;
        }
        p.pad = 0;
        a.part[blockIdx.x] = p;
        __threadfence();
        is_last = atomicAdd(&a.ctl->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    final_reduce<T>(a, tid, 256, red, set_dt ? kSetDt : kSumsOnly, gridDim.x);
}

// Copy every ghost cell of buf from its interior source (boundary rules).
// Ghost cell e (0 .. ghost_cells - 1) as ghosted coordinates: the two
// layers of each x face (4 ny nz cells), then those of each y face over the
// interior x (4 (nx-4) nz), then those of each z face over the interior x, y
// (4 (nx-4)(ny-4)).
__device__ __forceinline__ void ghost_cell(long long e, int nx, int ny, int nz, int &x, int &y, int &z) {
    const long long fx = 4LL * ny * nz, fy = 4LL * (nx - 4) * nz;
    if (e < fx) {
        const int s = (int)(e / ((long long)ny * nz));
        const long long r = e - (long long)s * ny * nz;
        x = s < 2 ? s : nx - 4 + s;
        y = (int)(r / nz);
        z = (int)(r - (long long)y * nz);
    } else if (e < fx + fy) {
        e -= fx;
        const int xi = (int)(e / (4LL * nz));
        const int r = (int)(e - (long long)xi * 4 * nz);
        const int s = r / nz;
        x = xi + 2;
        y = s < 2 ? s : ny - 4 + s;
        z = r - s * nz;
    } else {
        e -= fx + fy;
        const long long row = e >> 2;
        const int s = (int)(e & 3);
        x = (int)(row / (ny - 4)) + 2;
        y = (int)(row - (long long)(x - 2) * (ny - 4)) + 2;
        z = s < 2 ? s : nz - 4 + s;
    }
}

template <class T> __global__ void fill_ghosts_kernel(const GridArgs<T> a, T *buf) {
    const long long total = (long long)a.nx * a.ny * a.nz - (long long)(a.nx - 4) * (a.ny - 4) * (a.nz - 4);
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        int x, y, z;
        ghost_cell(c, a.nx, a.ny, a.nz, x, y, z);
        int fx, fy, fz;
        const int sx = axis_source(x, a.nx, a.bc[0], a.bc[1], &fx);
        const int sy = axis_source(y, a.ny, a.bc[2], a.bc[3], &fy);
        const int sz = axis_source(z, a.nz, a.bc[4], a.bc[5], &fz);
        const long long o = ((long long)x * a.ny + y) * a.pitch + z;
        const long long so = ((long long)sx * a.ny + sy) * a.pitch + sz;
        buf[o] = buf[so];
        buf[a.fstride + o] = fx ? -buf[a.fstride + so] : buf[a.fstride + so];
        buf[2 * a.fstride + o] = fy ? -buf[2 * a.fstride + so] : buf[2 * a.fstride + so];
        buf[3 * a.fstride + o] = fz ? -buf[3 * a.fstride + so] : buf[3 * a.fstride + so];
        buf[4 * a.fstride + o] = buf[4 * a.fstride + so];
    }
}

// calc_conserved over the interior (physics.rs:143-175); prim is dense
// with its own pitch/field stride.
template <class T>
__global__ void prim_to_cons_kernel(const GridArgs<T> a, const T *prim, long long pfs, int ppitch, T *cons) {
    const long long total = (long long)a.nx * a.ny * a.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        const long long xy = c / a.nz;
        const int z = (int)(c % a.nz);
        const long long po = xy * ppitch + z, co = xy * a.pitch + z;
        T w[5], u[5];
        for (int f = 0; f < 5; ++f) w[f] = prim[f * pfs + po];
        prim_to_cons(w, u, a.k.vol, a.k.gm1);
        for (int f = 0; f < 5; ++f) cons[f * a.fstride + co] = u[f];
    }
}

// calc_primitives over every cell (ghosts included).
template <class T, bool EXACT>
__global__ void cons_to_prim_kernel(const GridArgs<T> a, const T *cons, T *prim, long long pfs, int ppitch) {
    const long long total = (long long)a.nx * a.ny * a.nz;
    for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < total;
         c += (long long)gridDim.x * blockDim.x) {
        const long long xy = c / a.nz;
        const int z = (int)(c % a.nz);
        const long long po = xy * ppitch + z, co = xy * a.pitch + z;
        T u[5], w[5];
        for (int f = 0; f < 5; ++f) u[f] = cons[f * a.fstride + co];
        Phys<T, EXACT>::prim(u, w, a.k);
        for (int f = 0; f < 5; ++f) prim[f * pfs + po] = w[f];
    }
}

// ---------------------------------------------------------------------------
// Launch wrappers (instantiated per policy by the two translation units)
// ---------------------------------------------------------------------------
template <class T> constexpr int tile_rows() { return sizeof(T) == 8 ? 4 : 8; }   // == step_tile_rows(kRef*)
constexpr int kRing = 4;

template <class T, bool EXACT, int LIM>
static cudaError_t launch_step_t(const GridArgs<T> &a, const CUtensorMap *tmap, int chunk, cudaStream_t st) {
    constexpr int TY = tile_rows<T>();
    using S = StepSmem<T, TY, kRing>;
    auto kern = step_kernel<T, TY, LIM, kRing, EXACT>;
    const int smem = (int)sizeof(S) + 1024;
    static std::atomic<unsigned long long> attr_set{0};   // per instantiation
    const cudaError_t e = ensure_dynamic_smem(kern, smem, attr_set);
    if (e != cudaSuccess) return e;
    const int blocks = step_grid_blocks(a, chunk);
    kern<<<blocks, dim3(kTZ, TY), smem, st>>>(a, *tmap, chunk);
    return cudaGetLastError();
}

template <class T, bool EXACT>
cudaError_t launch_step_policy(const GridArgs<T> &a, const CUtensorMap *tmap, int limiter, int chunk,
                               cudaStream_t st) {
    return limiter ? launch_step_t<T, EXACT, 1>(a, tmap, chunk, st) : launch_step_t<T, EXACT, 0>(a, tmap, chunk, st);
}

template <class T, bool EXACT> cudaError_t launch_reduce_policy(const GridArgs<T> &a, int set_dt, cudaStream_t st) {
    const long long total = (long long)(a.nx - 4) * (a.ny - 4) * (a.nz - 4);
    long long blocks = (total + 255) / 256;
    if (blocks > kReduceBlocks) blocks = kReduceBlocks;
    reduce_kernel<T, EXACT><<<(int)blocks, 256, 0, st>>>(a, set_dt);
    return cudaGetLastError();
}

inline int flat_blocks(long long total) {
    long long b = (total + 255) / 256;
    if (b > kSms * 16) b = kSms * 16;
    if (b < 1) b = 1;
    return (int)b;
}

template <class T, bool EXACT>
cudaError_t launch_cons_to_prim_policy(const GridArgs<T> &a, const T *cons, T *prim, long long pfs, int ppitch,
                                       cudaStream_t st) {
    cons_to_prim_kernel<T, EXACT><<<flat_blocks((long long)a.nx * a.ny * a.nz), 256, 0, st>>>(a, cons, prim, pfs,
                                                                                             ppitch);
    return cudaGetLastError();
}

}  // namespace dg
