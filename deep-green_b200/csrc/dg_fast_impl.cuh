// dg_fast_impl.cuh -- FP32 production step for sm_100a: one launch per
// compute_step (deep-green src/rs/src/physics.rs:595-681), fast arithmetic.
//
// Same march and boundary semantics as the reference-rounding kernel
// (dg_step_impl.cuh), organised to cut issued instructions and shared-memory
// traffic:
//   * a thread owns a PAIR of cells stacked in y (rows y, y+1) at one z;
//     every per-cell quantity is a float2 and the arithmetic runs on
//     Blackwell's packed FP32 pipe (__ffma2_rn / __fadd2_rn / __fmul2_rn):
//     one instruction updates both cells;
//   * each face flux is computed once: the x-face from registers carried
//     along the march, the two y-faces of a pair (its lower face and the
//     one between its rows) and the lower z-face, all packed two at a time;
//   * z-neighbours exchange face states and fluxes by warp shuffles, the
//     y-neighbour pair above/below through small shared arrays; only the
//     tile's halo ring (one row above/below, one column left/right) is
//     computed separately, and its face states/fluxes go through shared
//     memory;
//   * slopes are kept in cell units (slope * ds): the face offsets become
//     +-s/2 and the predictor uses dt/(2 ds), so no per-slope scaling;
//     minmod is the clamp min(max(b, min(a,0)), max(a,0)); the sound speed
//     is g*rsqrt(g*rho) with g = gamma*p (one MUFU instead of two).
// Results match the FP64 oracle to the FP32 tolerance (1e-5 relative L1 on
// smooth problems), not bit for bit.
#pragma once
#include "dg_common.cuh"

namespace dg {
namespace fastk {

using f2 = float2;

// ---- scalar / packed arithmetic with one interface ---------------------------
__device__ __forceinline__ float vadd(float a, float b) { return a + b; }
__device__ __forceinline__ float vsub(float a, float b) { return a - b; }
__device__ __forceinline__ float vmul(float a, float b) { return a * b; }
__device__ __forceinline__ float vfma(float a, float b, float c) { return fmaf(a, b, c); }
__device__ __forceinline__ float vspl(float s, float) { return s; }
__device__ __forceinline__ float vrcp(float a) { return __fdividef(1.0f, a); }
__device__ __forceinline__ float vrsq(float a) { return rsqrtf(a); }
__device__ __forceinline__ float vsqrt(float a) { return __fsqrt_rn(a); }
__device__ __forceinline__ float vmax(float a, float b) { return fmaxf(a, b); }
__device__ __forceinline__ float vabs(float a) { return fabsf(a); }
__device__ __forceinline__ float mm1(float a, float b) { return fminf(fmaxf(b, fminf(a, 0.0f)), fmaxf(a, 0.0f)); }
__device__ __forceinline__ float vminmod(float a, float b) { return mm1(a, b); }

__device__ __forceinline__ f2 vadd(f2 a, f2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ f2 vsub(f2 a, f2 b) { return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a); }
__device__ __forceinline__ f2 vmul(f2 a, f2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ f2 vfma(f2 a, f2 b, f2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ f2 vspl(float s, f2) { return make_float2(s, s); }
__device__ __forceinline__ f2 vrcp(f2 a) { return make_float2(__fdividef(1.0f, a.x), __fdividef(1.0f, a.y)); }
__device__ __forceinline__ f2 vrsq(f2 a) { return make_float2(rsqrtf(a.x), rsqrtf(a.y)); }
__device__ __forceinline__ f2 vsqrt(f2 a) { return make_float2(__fsqrt_rn(a.x), __fsqrt_rn(a.y)); }
__device__ __forceinline__ f2 vmax(f2 a, f2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ f2 vabs(f2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ f2 vminmod(f2 a, f2 b) { return make_float2(mm1(a.x, b.x), mm1(a.y, b.y)); }

template <class V> __device__ __forceinline__ V S(float s) { return vspl(s, V()); }

// Constants of the fast policy.
struct FK {
    float inv_vol, gamma, gm1, inv_gm1;
    float scale;   // dt * ds * ds (update of totals with fluxes lacking their *ds)
    float ds;
    int lim;       // 0 central slopes, 1 minmod
};

// Conserved totals -> primitives (calc_primitives, physics.rs:112-140).
template <class V> __device__ __forceinline__ void prim(const V u[5], V w[5], const FK &k) {
    const V ir = vrcp(u[0]);
    const V rho = vmul(u[0], S<V>(k.inv_vol));
    const V vx = vmul(u[1], ir), vy = vmul(u[2], ir), vz = vmul(u[3], ir);
    const V v2 = vfma(vz, vz, vfma(vy, vy, vmul(vx, vx)));
    w[0] = rho;
    w[1] = vx;
    w[2] = vy;
    w[3] = vz;
    // (E/V - rho v^2 / 2) (gamma - 1)
    w[4] = vmul(vfma(vmul(S<V>(-0.5f), rho), v2, vmul(u[4], S<V>(k.inv_vol))), S<V>(k.gm1));
}

// Slope in cell units (slope * ds): central (q+ - q-)/2 or minmod of the
// one-sided differences (calc_gradients, physics.rs:206-208, times ds).
template <class V> __device__ __forceinline__ V slope(V qm, V q0, V qp, int lim) {
    if (lim == 0) return vmul(vsub(qp, qm), S<V>(0.5f));
    return vminmod(vsub(q0, qm), vsub(qp, q0));
}

// Half-step predictor (extrapolate_primitives_t, physics.rs:251-278) with
// cell-unit slopes sx, sy, sz; hd = dt / (2 ds).
template <class V>
__device__ __forceinline__ void predict(const V w[5], const V sx[5], const V sy[5], const V sz[5], float hd,
                                        const FK &k, V out[5]) {
    const V rho = w[0], vx = w[1], vy = w[2], vz = w[3], p = w[4];
    const V nh = S<V>(-hd);
    const V ir = vrcp(rho);
    const V div = vadd(vadd(sx[1], sy[2]), sz[3]);
    out[0] = vfma(nh, vfma(rho, div, vfma(vz, sz[0], vfma(vy, sy[0], vmul(vx, sx[0])))), rho);
    out[1] = vfma(nh, vfma(ir, sx[4], vfma(vz, sz[1], vfma(vy, sy[1], vmul(vx, sx[1])))), vx);
    out[2] = vfma(nh, vfma(ir, sy[4], vfma(vz, sz[2], vfma(vy, sy[2], vmul(vx, sx[2])))), vy);
    out[3] = vfma(nh, vfma(ir, sz[4], vfma(vz, sz[3], vfma(vy, sy[3], vmul(vx, sx[3])))), vz);
    const V gp = vmul(S<V>(k.gamma), p);
    out[4] = vfma(nh, vfma(vz, sz[4], vfma(vy, sy[4], vfma(vx, sx[4], vmul(gp, div)))), p);
}

// Rusanov flux (calc_flux_reconstruction, physics.rs:338-400) without the
// final *ds.  a: state on the lower side of the face, b: upper side, both
// (rho, vx, vy, vz, p); N: index of the normal velocity.  gh = G*h of the
// gravity term when grav.
template <int N, class V>
__device__ __forceinline__ void face(const V a[5], const V b[5], bool grav, V gh, const FK &k, V F[5]) {
    constexpr int T1 = N == 1 ? 2 : 1, T2 = N == 3 ? 2 : 3;
    const V ra = a[0], ua = a[N], va = a[T1], wa = a[T2], pa = a[4];
    const V rb = b[0], ub = b[N], vb = b[T1], wb = b[T2], pb = b[4];
    const V h = S<V>(0.5f);
    const V ea = vfma(vmul(h, ra), vfma(wa, wa, vfma(va, va, vmul(ua, ua))), vmul(pa, S<V>(k.inv_gm1)));
    const V eb = vfma(vmul(h, rb), vfma(wb, wb, vfma(vb, vb, vmul(ub, ub))), vmul(pb, S<V>(k.inv_gm1)));
    const V mua = vmul(ra, ua), mva = vmul(ra, va), mwa = vmul(ra, wa);
    const V mub = vmul(rb, ub), mvb = vmul(rb, vb), mwb = vmul(rb, wb);
    const V rs = vmul(vadd(ra, rb), h);
    const V mu = vmul(vadd(mua, mub), h), mv = vmul(vadd(mva, mvb), h), mw = vmul(vadd(mwa, mwb), h);
    const V es = vmul(vadd(ea, eb), h);
    const V irs = vrcp(rs);
    const V us = vmul(mu, irs);
    const V ps = vmul(vfma(vmul(vfma(mw, mw, vfma(mv, mv, vmul(mu, mu))), S<V>(-0.5f)), irs, es), S<V>(k.gm1));
    const V ga = vmul(S<V>(k.gamma), pa), gb = vmul(S<V>(k.gamma), pb);
    const V ca = vadd(vmul(ga, vrsq(vmul(ga, ra))), vabs(ua));
    const V cb = vadd(vmul(gb, vrsq(vmul(gb, rb))), vabs(ub));
    const V nhc = vmul(vmax(ca, cb), S<V>(-0.5f));
    V fu = vfma(mu, us, ps);
    V fe = vmul(vadd(es, ps), us);
    if (grav) {
        fu = vfma(rs, gh, fu);
        fe = vfma(vmul(vmul(h, rs), vadd(ua, ub)), gh, fe);
    }
    F[0] = vfma(nhc, vsub(rb, ra), mu);
    F[N] = vfma(nhc, vsub(mub, mua), fu);
    F[T1] = vfma(nhc, vsub(mvb, mva), vmul(mv, us));
    F[T2] = vfma(nhc, vsub(mwb, mwa), vmul(mw, us));
    F[4] = vfma(nhc, vsub(eb, ea), fe);
}

__device__ __forceinline__ float comp(f2 v, int i) { return i ? v.y : v.x; }
__device__ __forceinline__ void setc(f2 &v, int i, float s) {
    if (i) v.y = s;
    else v.x = s;
}

// W warps, each owning 32 columns x 2 rows (a y-pair per thread): the tile
// is TY = 2W rows x 32 columns.  The tile's halo ring (rows y0-1 and y0+TY,
// columns z0-1 and z0+32) is computed two cells per thread with the same
// packed code by the first 32+TY threads, and the tile's edge faces by the
// first 16+TY/2.
template <int W, int R> struct Smem {
    static constexpr int TY = 2 * W;
    static constexpr int NT = 32 * W;
    static constexpr int NOWN = NT;
    static constexpr int RY = TY + 4;
    static constexpr int kFieldElems = RY * kRZ;
    static constexpr int kBoxBytes = 5 * kFieldElems * 4;
    static constexpr int kSlotElems = ((kBoxBytes + 127) / 128) * 128 / 4;

    float ring[R * kSlotElems];   // TMA destinations; primitives after conversion
    f2 own_cons[3][5][NOWN];      // each own thread's conserved pair, 3 planes
    float ypl[W + 1][5][32];      // y+ states: [0] halo row y0-1, [w+1] upper row of pair w
    float ymn_top[5][32];         // y- state of halo row y0+TY
    float zpl_left[5][TY];        // z+ state of halo column z0-1
    float zmn_right[5][TY];       // z- state of halo column z0+32
    float zpl_edge[5][TY];        // z+ state of own column z0+31
    // fluxes exchanged between threads, double-buffered by plane parity: a
    // plane's divergence is completed after the next plane's first barrier
    float fy_pub[2][W][5][32];    // y-flux of the lower face of pair w
    float fy_edge[2][5][32];      // y-flux of face (y0+TY-1 | y0+TY)
    float fz_edge[2][5][TY];      // z-flux of face (z0+31 | z0+32)
    float fz_last[2][5][TY];      // lower z-flux of own column z0+31 (lane 31)
    uint64_t bar[R];
    double red[W * 7];
    int abort_flag;
    int is_last;
};

// LIM: the slope limiter as a compile-time constant, or -1 to read it from
// the grid's arguments.
// SKIP_PAD: leave the states of cells past the first ghost layer (the
// padding of ragged tiles, common in batches of small grids) uncomputed; the
// single-grid kernel keeps the smaller code.
template <int W, int R, bool SKIP_PAD = false, int LIM = -1> struct Kernel {
    using Sm = Smem<W, R>;
    static constexpr int TY = Sm::TY, NT = Sm::NT, NOWN = Sm::NOWN;

    // slope with the limiter fixed at compile time (LIM >= 0) or read at
    // run time (LIM < 0: grids of a batch may differ)
    template <class V> static __device__ __forceinline__ V slp(V qm, V q0, V qp, int lim) {
        if constexpr (LIM >= 0) return slope(qm, q0, qp, LIM);
        else return slope(qm, q0, qp, lim);
    }

    static __device__ __forceinline__ float &P(Sm &s, int slot, int f, int ry, int rz) {
        return s.ring[slot * Sm::kSlotElems + f * Sm::kFieldElems + ry * kRZ + rz];
    }

    // Predicted state and cell-unit slopes of ONE cell at region (ry, rz)
    // of the plane in slot s0, applying the y/z ghost-layer-1 rules of the
    // reference's derived-array ghost copies (see dg_step_impl.cuh).
    static __device__ void cell_scalar(Sm &s, const GridArgs<float> &a, const FK &k, float hd, int sm, int s0,
                                       int sp, int ry, int rz, int gyc, int gzc, float xt[5], float sx[5],
                                       float sy[5], float sz[5]) {
        int rule = kPeriodic, axis = 0, nry = ry, nrz = rz;
        if (gyc == 1) { rule = a.bc[2]; axis = 2; nry = ry + 1; }
        else if (gyc == a.ny - 2) { rule = a.bc[3]; axis = 2; nry = ry - 1; }
        else if (gzc == 1) { rule = a.bc[4]; axis = 3; nrz = rz + 1; }
        else if (gzc == a.nz - 2) { rule = a.bc[5]; axis = 3; nrz = rz - 1; }
        auto slopes_at = [&](int y, int z, float w[5], float gx[5], float gy[5], float gz[5]) {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const float c = P(s, s0, f, y, z);
                w[f] = c;
                gx[f] = slp(P(s, sm, f, y, z), c, P(s, sp, f, y, z), k.lim);
                gy[f] = slp(P(s, s0, f, y - 1, z), c, P(s, s0, f, y + 1, z), k.lim);
                gz[f] = slp(P(s, s0, f, y, z - 1), c, P(s, s0, f, y, z + 1), k.lim);
            }
        };
        float w[5];
        if (rule == kOutflow) {
            slopes_at(nry, nrz, w, sx, sy, sz);
            predict(w, sx, sy, sz, hd, k, xt);
        } else {
            slopes_at(ry, rz, w, sx, sy, sz);
            if (rule == kWall) {
                float w2[5], gx2[5], gy2[5], gz2[5];
                slopes_at(nry, nrz, w2, gx2, gy2, gz2);
                predict(w2, gx2, gy2, gz2, hd, k, xt);
                xt[axis] = -xt[axis];
            } else {
                predict(w, sx, sy, sz, hd, k, xt);
            }
        }
    }

    static __device__ __forceinline__ float grav_h(const GridArgs<float> &a, int klow) {
        return a.k.g * (float(a.nz - 4) * a.k.ds - float(klow - 2) * a.k.ds);
    }

    // New state of the pair: its wave speed (next dt) and the store with its
    // ghost-cell images.  (Conservation sums are computed on demand by the
    // state reduction, not every step.)
    static __device__ __forceinline__ void epilogue(const GridArgs<float> &a, const FK &k, int xu, const f2 u[5],
                                                    bool val1, int gy0, int gzo, int nyi0, int nyi1, int nzi,
                                                    const int *yimg0, const int *yflp0, const int *yimg1,
                                                    const int *yflp1, const int *zimg, const int *zflp,
                                                    bool col_img, float &smax) {
        f2 q[5];
        prim(u, q, k);
        smax = max_nan(smax, fast_speed(q[0].x, q[1].x, q[2].x, q[3].x, q[4].x, k.gamma));
        if (val1) smax = max_nan(smax, fast_speed(q[0].y, q[1].y, q[2].y, q[3].y, q[4].y, k.gamma));
        // ghost images exist only next to the x faces or on boundary columns
        const bool x_edge = xu <= 3 || xu >= a.nx - 4;
        if (!x_edge && !col_img) {
            const long long o0 = ((long long)xu * a.ny + gy0) * a.pitch + gzo;
            const long long o1 = o0 + a.pitch;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                a.dst[f * a.fstride + o0] = u[f].x;
                if (val1) a.dst[f * a.fstride + o1] = u[f].y;
            }
            return;
        }
        int ximg[4], xflp[4];
        const int nxi = axis_images(xu, a.nx, a.bc[0], a.bc[1], ximg, xflp);
        if (nxi == 1 && !col_img) {
            const long long o0 = ((long long)xu * a.ny + gy0) * a.pitch + gzo;
            const long long o1 = o0 + a.pitch;
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                a.dst[f * a.fstride + o0] = u[f].x;
                if (val1) a.dst[f * a.fstride + o1] = u[f].y;
            }
            return;
        }
        for (int r = 0; r < 2; ++r) {
            if (r == 1 && !val1) break;
            const int nyi = r ? nyi1 : nyi0;
            for (int ix = 0; ix < nxi; ++ix)
                for (int iy = 0; iy < nyi; ++iy)
                    for (int iz = 0; iz < nzi; ++iz) {
                        const int yy = r ? yimg1[iy] : yimg0[iy];
                        const int fyl = r ? yflp1[iy] : yflp0[iy];
                        const long long o = ((long long)ximg[ix] * a.ny + yy) * a.pitch + zimg[iz];
                        const float u0 = comp(u[0], r), u1 = comp(u[1], r), u2 = comp(u[2], r);
                        const float u3 = comp(u[3], r), u4 = comp(u[4], r);
                        a.dst[o] = u0;
                        a.dst[a.fstride + o] = xflp[ix] ? -u1 : u1;
                        a.dst[2 * a.fstride + o] = fyl ? -u2 : u2;
                        a.dst[3 * a.fstride + o] = zflp[iz] ? -u3 : u3;
                        a.dst[4 * a.fstride + o] = u4;
                    }
        }
    }

    // Predicted state and slopes of two arbitrary cells A, B (region
    // coordinates) as one packed computation, or cell by cell with the
    // boundary rules when either is outside the interior.
    static __device__ __forceinline__ void pair_state(Sm &s, const GridArgs<float> &a, const FK &k, float hd, int sm,
                                                      int s0, int sp, int ryA, int rzA, int ryB, int rzB, int y0, int z0,
                                                      f2 xt[5], f2 sx[5], f2 sy[5], f2 sz[5]) {
        const int gyA = y0 - 2 + ryA, gzA = z0 - 2 + rzA, gyB = y0 - 2 + ryB, gzB = z0 - 2 + rzB;
        const bool regA = gyA >= 2 && gyA <= a.ny - 3 && gzA >= 2 && gzA <= a.nz - 3;
        const bool regB = gyB >= 2 && gyB <= a.ny - 3 && gzB >= 2 && gzB <= a.nz - 3;
        if (regA && regB) {
            f2 c[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                c[f] = make_float2(P(s, s0, f, ryA, rzA), P(s, s0, f, ryB, rzB));
                const f2 xm = make_float2(P(s, sm, f, ryA, rzA), P(s, sm, f, ryB, rzB));
                const f2 xp = make_float2(P(s, sp, f, ryA, rzA), P(s, sp, f, ryB, rzB));
                const f2 ym = make_float2(P(s, s0, f, ryA - 1, rzA), P(s, s0, f, ryB - 1, rzB));
                const f2 yp = make_float2(P(s, s0, f, ryA + 1, rzA), P(s, s0, f, ryB + 1, rzB));
                const f2 zm = make_float2(P(s, s0, f, ryA, rzA - 1), P(s, s0, f, ryB, rzB - 1));
                const f2 zp = make_float2(P(s, s0, f, ryA, rzA + 1), P(s, s0, f, ryB, rzB + 1));
                sx[f] = slp(xm, c[f], xp, k.lim);
                sy[f] = slp(ym, c[f], yp, k.lim);
                sz[f] = slp(zm, c[f], zp, k.lim);
            }
            predict(c, sx, sy, sz, hd, k, xt);
        } else {
            // cells past the first ghost layer (the padding of a ragged tile)
            // feed no face of an interior cell: their states may be left zero
            const bool needA = !SKIP_PAD || (gyA <= a.ny - 2 && gzA <= a.nz - 2);
            const bool needB = !SKIP_PAD || (gyB <= a.ny - 2 && gzB <= a.nz - 2);
#pragma unroll
            for (int r = 0; r < 2; ++r) {
                float t[5], gx[5], gy[5], gz[5];
                if (r ? needB : needA) {
                    cell_scalar(s, a, k, hd, sm, s0, sp, r ? ryB : ryA, r ? rzB : rzA, r ? gyB : gyA, r ? gzB : gzA, t,
                                gx, gy, gz);
                } else {
#pragma unroll
                    for (int f = 0; f < 5; ++f) t[f] = gx[f] = gy[f] = gz[f] = 0.0f;
                }
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    setc(xt[f], r, t[f]);
                    setc(sx[f], r, gx[f]);
                    setc(sy[f], r, gy[f]);
                    setc(sz[f], r, gz[f]);
                }
            }
        }
    }

    // One work item: tile (ty, tz) of grid `a`, x-planes of chunk cx.  Its
    // partial result goes to a.part[part_idx]; the last of the grid's nparts
    // items reduces them (next dt).  Returns false after a device-side wait
    // timed out (status flag set).
    static __device__ bool run_tile(const GridArgs<float> &a, const CUtensorMap *tmap, int tz, int ty, int cx, int chunk,
                                    int part_idx, int nparts, unsigned char *raw) {
        Sm &s = *reinterpret_cast<Sm *>(raw);
        const int lane = threadIdx.x, w = threadIdx.y;
        const int tid = w * 32 + lane;
        constexpr bool own = true;

        const int y0 = 2 + ty * TY, z0 = 2 + tz * kTZ;
        const int xs = 2 + cx * chunk;
        const int xe = min(xs + chunk, a.nx - 2);
        const int np = xe - xs + 4;
        // own pair (own warps): rows y0+2w, y0+2w+1 at column z0+lane
        const int gy0 = y0 + 2 * w, gy1 = gy0 + 1, gzo = z0 + lane;
        const int ry0 = 2 + 2 * w, ry1 = ry0 + 1, rzo = lane + 2;
        const bool zval = own && gzo <= a.nz - 3;
        const bool val0 = zval && gy0 <= a.ny - 3, val1 = zval && gy1 <= a.ny - 3;
        const bool regular = val1;

        if (*(volatile unsigned *)&a.ctl->flags & kStatusTimeout) return false;
        const unsigned step = (unsigned)a.ctl->step;
        const float dt = (float)a.ctl->dt[step & 1];
        FK k;
        k.inv_vol = a.k.inv_vol;
        k.gamma = a.k.gamma;
        k.gm1 = a.k.gm1;
        k.inv_gm1 = a.k.inv_gm1;
        k.ds = a.k.ds;
        const float hd = 0.5f * dt * a.k.inv_ds;   // dt / (2 ds)
        k.scale = dt * a.k.ds * a.k.ds;
        const int lim = a.limiter;
        k.lim = lim;
        const bool grav = a.gravity != 0;

        if (tid == 0) {
            s.abort_flag = 0;
            for (int i = 0; i < R; ++i) mbar_init(&s.bar[i], 1);
            fence_mbar_init();
        }
        __syncthreads();
        if (tid == 0) {
            for (int l = 0; l < R && l < np; ++l) {
                mbar_expect_tx(&s.bar[l], Sm::kBoxBytes);
                tma_load_4d(&s.ring[l * Sm::kSlotElems], tmap, z0 - 2, y0 - 2, xs - 2 + l, 0, &s.bar[l]);
            }
        }

        // ghost images of the own column along y (per row) and z
        int yimg0[4], yflp0[4], yimg1[4], yflp1[4], zimg[4], zflp[4];
        const int nyi0 = val0 ? axis_images(gy0, a.ny, a.bc[2], a.bc[3], yimg0, yflp0) : 0;
        const int nyi1 = val1 ? axis_images(gy1, a.ny, a.bc[2], a.bc[3], yimg1, yflp1) : 0;
        const int nzi = zval ? axis_images(gzo, a.nz, a.bc[4], a.bc[5], zimg, zflp) : 0;
        const bool col_img = nzi > 1 || nyi0 > 1 || nyi1 > 1;

        // carried along the march: prediction and x-slope of the previous
        // plane, and acc = (y/z flux divergence of the previous plane) minus
        // (its lower x-face flux), so the update is cons - scale*(fx + acc)
        f2 xt_prev[5], sx_prev[5], acc[5];
        float fyy[5];   // upper row's lower y-flux, kept until the face above it is known
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            xt_prev[f] = sx_prev[f] = acc[f] = make_float2(0.f, 0.f);
            fyy[f] = 0.f;
        }
        float smax = 0.0f;   // max wave speed of the updated cells (NaN-propagating)

        constexpr int HR = 4 * kRZ + 4 * TY;   // staged halo cells (rows 0,1,TY+2,TY+3; cols 0,1,34,35)

        // (a) wait for staged plane l, convert to primitives in place: own
        // warps their pairs (keeping the conserved values), halo warps the
        // staged halo cells
        auto convert = [&](int l) -> bool {
            const int slot = l % R;
            if (!mbar_wait(&s.bar[slot], (l / R) & 1, kWaitBudget)) return false;
            {
                f2 u[5], q[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) u[f] = make_float2(P(s, slot, f, ry0, rzo), P(s, slot, f, ry1, rzo));
                prim(u, q, k);
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    P(s, slot, f, ry0, rzo) = q[f].x;
                    P(s, slot, f, ry1, rzo) = q[f].y;
                    s.own_cons[l % 3][f][tid] = u[f];
                }
            }
            {
                for (int h = tid; h < HR; h += NT) {
                    int ry, rz;
                    if (h < 4 * kRZ) {
                        const int r4 = h / kRZ;
                        rz = h - r4 * kRZ;
                        ry = r4 < 2 ? r4 : TY + r4;
                    } else {
                        const int j = h - 4 * kRZ, c4 = j & 3;
                        ry = 2 + (j >> 2);
                        rz = c4 < 2 ? c4 : kTZ + c4;
                    }
                    float u[5], q[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) u[f] = P(s, slot, f, ry, rz);
                    prim(u, q, k);
#pragma unroll
                    for (int f = 0; f < 5; ++f) P(s, slot, f, ry, rz) = q[f];
                }
            }
            return true;
        };

        bool ok = convert(0);
        if (ok) ok = convert(1);
        if (!ok) s.abort_flag = 1;

        int issued = (np < R) ? np : R;
        for (int m = xs - 1; m <= xe; ++m) {
            const int l = m - xs + 3;   // staged index of plane m+1
            if (!convert(l)) s.abort_flag = 1;
            fence_proxy_async();
            __syncthreads();   // S1: primitives of planes m-1..m+1 and plane m-1's fluxes ready
            if (s.abort_flag) break;
            const int sm = (l - 2) % R, s0 = (l - 1) % R, sp = l % R;
            const bool plane_upd = m >= xs && m < xe;

            // ---- (e1) complete the divergence of plane m-1 with the fluxes
            // other threads published: the upper row's upper y-face and, on
            // lane 31, the tile's edge z-face
            if (m - 1 >= xs && m - 1 < xe) {
                const int pb = (m - 1) & 1;
                const bool z_out = gzo == 2 && a.bc[4] == kOutflow;
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    // each deferred term enters as a difference of the two
                    // faces, as the other terms did
                    const float top = (w + 1 < W) ? s.fy_pub[pb][w + 1][f][lane] : s.fy_edge[pb][f][lane];
                    acc[f].y += top - fyy[f];
                    if (lane == 31 && !z_out) {
                        acc[f].x += s.fz_edge[pb][f][2 * w] - s.fz_last[pb][f][2 * w];
                        acc[f].y += s.fz_edge[pb][f][2 * w + 1] - s.fz_last[pb][f][2 * w + 1];
                    }
                }
            }

            // ---- (b') tile halo ring: rows y0-1 / y0+TY of each column, columns
            // z0-1 / z0+32 of each row, one pair per thread
            if (plane_upd && tid < 32 + TY) {
                const bool rows = tid < 32;
                const int hyA = rows ? 1 : tid - 32 + 2, hzA = rows ? tid + 2 : 1;
                const int hyB = rows ? TY + 2 : tid - 32 + 2, hzB = rows ? tid + 2 : kTZ + 2;
                f2 hxt[5], hsx[5], hsy[5], hsz[5];
                pair_state(s, a, k, hd, sm, s0, sp, hyA, hzA, hyB, hzB, y0, z0, hxt, hsx, hsy, hsz);
                if (rows) {
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        s.ypl[0][f][tid] = fmaf(hsy[f].x, 0.5f, hxt[f].x);
                        s.ymn_top[f][tid] = fmaf(hsy[f].y, -0.5f, hxt[f].y);
                    }
                } else {
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        s.zpl_left[f][tid - 32] = fmaf(hsz[f].x, 0.5f, hxt[f].x);
                        s.zmn_right[f][tid - 32] = fmaf(hsz[f].y, -0.5f, hxt[f].y);
                    }
                }
            }
            f2 xt[5], sx[5], sy[5], sz[5], fx[5];
            if (own) {
                // ---- (b) own pair: slopes and prediction --------------------
                if (regular) {
                    f2 c[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        c[f] = make_float2(P(s, s0, f, ry0, rzo), P(s, s0, f, ry1, rzo));
                        const f2 xm = make_float2(P(s, sm, f, ry0, rzo), P(s, sm, f, ry1, rzo));
                        const f2 xp = make_float2(P(s, sp, f, ry0, rzo), P(s, sp, f, ry1, rzo));
                        const f2 ym = make_float2(P(s, s0, f, ry0 - 1, rzo), c[f].x);
                        const f2 yp = make_float2(c[f].y, P(s, s0, f, ry1 + 1, rzo));
                        const f2 zm = make_float2(P(s, s0, f, ry0, rzo - 1), P(s, s0, f, ry1, rzo - 1));
                        const f2 zp = make_float2(P(s, s0, f, ry0, rzo + 1), P(s, s0, f, ry1, rzo + 1));
                        sx[f] = slp(xm, c[f], xp, lim);
                        sy[f] = slp(ym, c[f], yp, lim);
                        sz[f] = slp(zm, c[f], zp, lim);
                    }
                    predict(c, sx, sy, sz, hd, k, xt);
                } else {
                    pair_state(s, a, k, hd, sm, s0, sp, ry0, rzo, ry1, rzo, y0, z0, xt, sx, sy, sz);
                }
                // publish the face states other threads need: the upper row's
                // y+ state (pair above) and, from lane 31, the z+ states (edge)
                if (plane_upd) {
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        s.ypl[w + 1][f][lane] = fmaf(sy[f].y, 0.5f, xt[f].y);
                        if (lane == 31) {
                            s.zpl_edge[f][2 * w] = fmaf(sz[f].x, 0.5f, xt[f].x);
                            s.zpl_edge[f][2 * w + 1] = fmaf(sz[f].y, 0.5f, xt[f].y);
                        }
                    }
                }
                // ---- (c) x-face between planes m-1 and m ---------------------
                if (m >= xs) {
                    if (m == 2 && a.bc[0] == kWall) {
#pragma unroll
                        for (int f = 0; f < 5; ++f) xt_prev[f] = xt[f];
                        xt_prev[1] = vmul(xt_prev[1], S<f2>(-1.0f));
                    }
                    if (m == a.nx - 2) {
                        if (a.bc[1] == kOutflow) {
#pragma unroll
                            for (int f = 0; f < 5; ++f) { xt[f] = xt_prev[f]; sx[f] = sx_prev[f]; }
                        } else if (a.bc[1] == kWall) {
#pragma unroll
                            for (int f = 0; f < 5; ++f) xt[f] = xt_prev[f];
                            xt[1] = vmul(xt[1], S<f2>(-1.0f));
                        }
                    }
                    f2 lo[5], up[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        lo[f] = vfma(sx_prev[f], S<f2>(0.5f), xt_prev[f]);
                        up[f] = vfma(sx[f], S<f2>(-0.5f), xt[f]);
                    }
                    face<1>(lo, up, false, S<f2>(0.f), k, fx);
                } else {
#pragma unroll
                    for (int f = 0; f < 5; ++f) fx[f] = make_float2(0.f, 0.f);
                }
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    xt_prev[f] = xt[f];
                    sx_prev[f] = sx[f];
                }
                // ---- (e2) update plane m-1: cons - scale * (fx_hi + acc) ------
                const int xu = m - 1;
                if (xu >= xs && xu < xe && val0) {
                    const bool x_out = xu == 2 && a.bc[0] == kOutflow;   // acc holds no x-flux then
                    const int cs = (xu - xs + 2) % 3;
                    f2 u[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const f2 cA = s.own_cons[cs][f][tid];
                        const f2 t = x_out ? acc[f] : vadd(fx[f], acc[f]);
                        u[f] = vfma(S<f2>(-k.scale), t, cA);
                    }
                    epilogue(a, k, xu, u, val1, gy0, gzo, nyi0, nyi1, nzi, yimg0, yflp0, yimg1, yflp1, zimg, zflp,
                             col_img, smax);
                }
            }
            __syncthreads();   // S2: halo states and pair publications ready; slot of m-1 free

            if (tid == 0 && issued < np) {
                const int slot = (l - 2) % R;
                mbar_expect_tx(&s.bar[slot], Sm::kBoxBytes);
                tma_load_4d(&s.ring[slot * Sm::kSlotElems], tmap, z0 - 2, y0 - 2, xs - 2 + issued, 0, &s.bar[slot]);
            }
            if (issued < np) ++issued;

            // ---- (d) y- and z-faces of plane m --------------------------------
            f2 fy[5], fz[5];
            if (plane_upd && own) {
                {   // y: faces (y0+2w-1 | y0+2w) and (y0+2w | y0+2w+1)
                    f2 lo[5], up[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        lo[f] = make_float2(s.ypl[w][f][lane], fmaf(sy[f].x, 0.5f, xt[f].x));
                        up[f] = vfma(sy[f], S<f2>(-0.5f), xt[f]);
                    }
                    face<2>(lo, up, false, S<f2>(0.f), k, fy);
#pragma unroll
                    for (int f = 0; f < 5; ++f) s.fy_pub[m & 1][w][f][lane] = fy[f].x;
                }
                {   // z: lower face of each cell, left state from lane-1
                    f2 lo[5], up[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const f2 zpl = vfma(sz[f], S<f2>(0.5f), xt[f]);
                        f2 v;
                        v.x = __shfl_up_sync(0xffffffffu, zpl.x, 1);
                        v.y = __shfl_up_sync(0xffffffffu, zpl.y, 1);
                        if (lane == 0) v = make_float2(s.zpl_left[f][2 * w], s.zpl_left[f][2 * w + 1]);
                        lo[f] = v;
                        up[f] = vfma(sz[f], S<f2>(-0.5f), xt[f]);
                    }
                    const float ghs = grav ? grav_h(a, gzo - 1) : 0.f;
                    face<3>(lo, up, grav, make_float2(ghs, ghs), k, fz);
                }
            }
            if (plane_upd && tid < 16 + TY / 2) {
                // tile edge faces: y (y0+TY-1 | y0+TY) x 32 and z (z0+31 | z0+32) x TY
                if (tid < 16) {
                    const int h = tid;
                    f2 lo[5], up[5], F[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        lo[f] = make_float2(s.ypl[W][f][h], s.ypl[W][f][h + 16]);
                        up[f] = make_float2(s.ymn_top[f][h], s.ymn_top[f][h + 16]);
                    }
                    face<2>(lo, up, false, S<f2>(0.f), k, F);
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        s.fy_edge[m & 1][f][h] = F[f].x;
                        s.fy_edge[m & 1][f][h + 16] = F[f].y;
                    }
                } else {
                    const int r = tid - 16;
                    f2 lo[5], up[5], F[5];
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        lo[f] = make_float2(s.zpl_edge[f][r], s.zpl_edge[f][r + TY / 2]);
                        up[f] = make_float2(s.zmn_right[f][r], s.zmn_right[f][r + TY / 2]);
                    }
                    const float ghs = grav ? grav_h(a, z0 + kTZ - 1) : 0.f;
                    face<3>(lo, up, grav, make_float2(ghs, ghs), k, F);
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        s.fz_edge[m & 1][f][r] = F[f].x;
                        s.fz_edge[m & 1][f][r + TY / 2] = F[f].y;
                    }
                }
            }

            if (plane_upd) {
                // ---- (e0) this plane's divergence, minus its lower x-face flux,
                // from what this thread holds; completed at the next plane
                // lower x-outflow face repeats the next face's flux: plane 2
                // gets no x-divergence (boundaries.rs:107-111 on the fluxes)
                const bool x_out = m == 2 && a.bc[0] == kOutflow;
                const bool y_out = gy0 == 2 && a.bc[2] == kOutflow;
                const bool z_out = gzo == 2 && a.bc[4] == kOutflow;
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    f2 dy;
                    // lower outflow face repeats the next face's flux (cell 2 sees none)
                    dy.x = y_out ? 0.f : fy[f].y - fy[f].x;
                    dy.y = 0.f;
                    fyy[f] = fy[f].y;
                    f2 zh;
                    zh.x = __shfl_down_sync(0xffffffffu, fz[f].x, 1);
                    zh.y = __shfl_down_sync(0xffffffffu, fz[f].y, 1);
                    f2 dz = z_out ? make_float2(0.f, 0.f) : vsub(zh, fz[f]);
                    if (lane == 31) {
                        s.fz_last[m & 1][f][2 * w] = fz[f].x;
                        s.fz_last[m & 1][f][2 * w + 1] = fz[f].y;
                        dz = make_float2(0.f, 0.f);
                    }
                    const f2 d = vadd(dy, dz);
                    acc[f] = x_out ? d : vsub(d, fx[f]);
                }
            }
        }

        if (s.abort_flag) {
            if (tid == 0) {
                for (int l2 = issued > R ? issued - R : 0; l2 < issued; ++l2)
                    mbar_wait(&s.bar[l2 % R], (l2 / R) & 1, kWaitBudget);
                atomicOr(&a.ctl->flags, kStatusTimeout);
            }
            return false;
        }
        // every staged plane was consumed: the barriers can be re-initialised
        // by the next work item of a persistent launch
        if (tid == 0)
            for (int i = 0; i < R; ++i) mbar_inval(&s.bar[i]);
        // min over cells of ds/speed = ds / max speed
        const unsigned nanf = smax != smax;
        const double wmin = nanf ? INFINITY : (double)__fdiv_rn(k.ds, smax);
        double sum[5] = {0, 0, 0, 0, 0};
        if (block_partial(a, sum, wmin, nanf, tid, NT, s.red, &s.is_last, part_idx, nparts)) {
            __threadfence();
            final_reduce<float>(a, tid, NT, s.red, kAdvance, nparts);
        }
        return true;
    }
};

template <int W, int R, int LIM>
__global__ void __launch_bounds__(32 * W, 2) fast_step_kernel(const GridArgs<float> a,
                                                                   const __grid_constant__ CUtensorMap tmap,
                                                                   int chunk) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    constexpr int TY = Smem<W, R>::TY;
    const int tiles_z = (a.nz - 4 + kTZ - 1) / kTZ;
    const int tiles_y = (a.ny - 4 + TY - 1) / TY;
    int b = blockIdx.x;
    const int tz = b % tiles_z;
    b /= tiles_z;
    const int ty = b % tiles_y;
    Kernel<W, R, false, LIM>::run_tile(a, &tmap, tz, ty, b / tiles_y, chunk, blockIdx.x, gridDim.x, smem_raw);
}

// Batched step: one persistent launch advances many independent grids by
// one step each.  Work items (grid, tile, x-chunk) are taken from an atomic
// queue; each grid keeps its own control block, so its dt is its own CFL
// dt.  Grid arguments are copied to shared memory per item; the grid's TMA
// descriptor is read from global memory (written by the host before launch).
struct BatchItem {
    int g, local, tz, ty, cx;
};

template <int W, int R>
__global__ void __launch_bounds__(32 * W, 2) batch_step_kernel(const GridArgs<float> *__restrict__ args,
                                                              const CUtensorMap *__restrict__ maps,
                                                              const BatchItem *__restrict__ items, int nitems,
                                                              unsigned *queue, int chunk) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ int s_item;
    __shared__ __align__(16) GridArgs<float> s_args;
    const int tid = threadIdx.y * 32 + threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) return;
        const BatchItem bi = items[it];
        constexpr int kWords = (int)(sizeof(GridArgs<float>) / 4);
        for (int i = tid; i < kWords; i += 32 * W)
            reinterpret_cast<int *>(&s_args)[i] = reinterpret_cast<const int *>(&args[bi.g])[i];
        __syncthreads();
        // a register copy: the tile code reads the arguments all through the
        // march, and shared-memory loads of them cost ~10 % of the step
        const GridArgs<float> ga = s_args;
        const bool ok = Kernel<W, R, true>::run_tile(ga, &maps[bi.g], bi.tz, bi.ty, bi.cx, chunk, bi.local, ga.nparts,
                                               smem_raw);
        __syncthreads();
        if (!ok) return;
    }
}

}  // namespace fastk
}  // namespace dg
