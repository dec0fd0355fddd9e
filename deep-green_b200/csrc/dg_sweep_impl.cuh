// dg_sweep_impl.cuh -- the production step kernel of compute_step
// (deep-green src/rs/src/physics.rs:595-681) with fused arithmetic (the
// "fast" policy), in FP32 on packed pairs or in FP64: one launch per step,
// or two (interior tiles, frame) on grids with interior tiles.
//
// Decomposition.  A block owns a tile of TY rows (y) x 64 columns (z) of
// cells and marches along x through a chunk of planes.  Each plane arrives by
// one 4-D TMA copy (68 columns x (TY + 4) rows x 5 fields: the tile and its
// 2-cell halo, no multicast) in a ring of R slots, and stays there as
// conserved totals until its cells are updated.
//   * Owned warps (TY): warp r owns row y0 + r; lane l owns the two adjacent
//     cells (z, z + 1), z = z0 + 2l, as one pair.  Every per-cell formula is
//     written on pairs, and in FP32 a pair is one packed register, so the
//     arithmetic runs on Blackwell's packed instructions (add/sub/mul/fma
//     .f32x2: two cells per instruction).  The x-neighbours of a cell are
//     carried in registers along the march; the y-neighbours come from the
//     other warps' rows through shared memory; the z-neighbours from shared
//     memory (primitives) and warp shuffles (face states, fluxes).
//   * Halo warp A: the row below the tile and the halo columns left/right of
//     it; halo warp B: the row above the tile, the face between it and the
//     tile's top row, and the faces on the tile's right edge.  They produce
//     the predicted face states (or, on a domain face, what the reference's
//     ghost-layer rules leave there) and the fluxes no owned lane computes,
//     so the owned warps run no halo code: their only boundary handling is
//     per-plane / per-row / per-lane switches.
// One block barrier per plane.  Before it: convert plane m + 1 to
// primitives, slopes and predicted state of plane m, the x-face flux between
// planes m - 1 and m, publish face states.  After it: the y- and z-face
// fluxes of plane m and the update of plane m - 1.
//
// Ghost-layer rules of the reference's derived arrays (gradients, predicted
// states, fluxes; boundaries.rs:5-195 and handle_walls :197-407 applied to
// them in compute_step, physics.rs:595-681), as composed rules:
//   periodic: ghosts are computed like interior cells from the ghost
//             primitives (the ghost layers hold the wrapped copies); the
//             lower z boundary face carries the top face's gravity height
//             (the reference copies that face's flux, grav_klow);
//   outflow:  a ghost takes the adjacent interior cell's slopes and
//             prediction, and the lower face repeats the next face's flux,
//             so the first interior cell sees no divergence along that axis;
//   wall:     a ghost's slopes come from its own (mirrored) primitives and
//             its prediction is the mirrored prediction of the interior cell.
//
// Flux convention: face() returns 2F for mass and momenta and 4F for energy
// (F the reference's flux without its final *ds); the update scales undo it.
#pragma once
#include "dg_common.cuh"

namespace dg {
namespace sweep {

constexpr int kTileZ = 64;            // tile columns: 32 lanes x 2 cells
constexpr int kBoxZ = kTileZ + 4;     // staged columns: 2-cell halo each side

// ---------------------------------------------------------------------------
// Pair arithmetic.  float2: packed FP32 instructions; double2: two scalar
// operations.  Scalars of the pair's element type have the same interface.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 vadd(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 vmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 vfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }
__device__ __forceinline__ float2 vsub(float2 a, float2 b) {
    float2 r;
    asm("{\n\t.reg .b64 ra, rb, rd;\n\t"
        "mov.b64 ra, {%2, %3};\n\t"
        "mov.b64 rb, {%4, %5};\n\t"
        "sub.rn.f32x2 rd, ra, rb;\n\t"
        "mov.b64 {%0, %1}, rd;\n\t}"
        : "=f"(r.x), "=f"(r.y)
        : "f"(a.x), "f"(a.y), "f"(b.x), "f"(b.y));
    return r;
}
__device__ __forceinline__ double2 vadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 vsub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 vmul(double2 a, double2 b) { return make_double2(a.x * b.x, a.y * b.y); }
__device__ __forceinline__ double2 vfma(double2 a, double2 b, double2 c) {
    return make_double2(fma(a.x, b.x, c.x), fma(a.y, b.y, c.y));
}

template <class T> struct PairT;
template <> struct PairT<float> { using type = float2; };
template <> struct PairT<double> { using type = double2; };

template <class V> __device__ __forceinline__ V spl(double s);
template <> __device__ __forceinline__ float2 spl<float2>(double s) { return make_float2((float)s, (float)s); }
template <> __device__ __forceinline__ double2 spl<double2>(double s) { return make_double2(s, s); }
__device__ __forceinline__ float2 mk(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ double2 mk(double a, double b) { return make_double2(a, b); }

// 1/x of both cells: the fast policy's reciprocal (Phys<T, false>::prim).
__device__ __forceinline__ float2 vrcp(float2 a) { return make_float2(rcp_approx(a.x), rcp_approx(a.y)); }
__device__ __forceinline__ double2 vrcp(double2 a) { return make_double2(1.0 / a.x, 1.0 / a.y); }
__device__ __forceinline__ float2 vrsq(float2 a) { return make_float2(rsqrt_approx(a.x), rsqrt_approx(a.y)); }
__device__ __forceinline__ double2 vrsq(double2 a) { return make_double2(rsqrt(a.x), rsqrt(a.y)); }
__device__ __forceinline__ float2 vmax(float2 a, float2 b) { return make_float2(fmaxf(a.x, b.x), fmaxf(a.y, b.y)); }
__device__ __forceinline__ double2 vmax(double2 a, double2 b) { return make_double2(fmax(a.x, b.x), fmax(a.y, b.y)); }
__device__ __forceinline__ float2 vabs(float2 a) { return make_float2(fabsf(a.x), fabsf(a.y)); }
__device__ __forceinline__ double2 vabs(double2 a) { return make_double2(fabs(a.x), fabs(a.y)); }

// minmod(a, b): 0 when the signs differ or either is zero, else the one of
// smaller magnitude.  FP32: min(|a|, |b|) carrying the product of the signs
// (min.xorsign.abs), clamped at zero, given a's sign; equal to the clamp
// form min(max(b, min(a, 0)), max(a, 0)) except for the sign of a zero.
__device__ __forceinline__ float mm(float a, float b) {
    float r;
    asm("min.xorsign.abs.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    r = fmaxf(r, 0.0f);
    return __int_as_float(__float_as_int(r) | (__float_as_int(a) & (int)0x80000000));
}
__device__ __forceinline__ double mm(double a, double b) { return fmin(fmax(b, fmin(a, 0.0)), fmax(a, 0.0)); }
__device__ __forceinline__ float2 mm(float2 a, float2 b) { return make_float2(mm(a.x, b.x), mm(a.y, b.y)); }
__device__ __forceinline__ double2 mm(double2 a, double2 b) { return make_double2(mm(a.x, b.x), mm(a.y, b.y)); }

// Slope in cell units (slope * ds) from the backward and forward
// differences: minmod (LIM 1) or the reference's central difference
// (LIM 0, physics.rs:206-208, times ds).
template <int LIM, class V> __device__ __forceinline__ V slope(V dm, V dp) {
    if constexpr (LIM == 0) return vmul(vadd(dm, dp), spl<V>(0.5));
    else return mm(dm, dp);
}
template <int LIM, class S> __device__ __forceinline__ S slope1(S dm, S dp) {
    if constexpr (LIM == 0) return (dm + dp) * S(0.5);
    else return mm(dm, dp);
}

// Per-grid constants of the kernel in the pair type.
template <class T> struct K {
    T inv_vol, gamma, gm1, kp, c1, sg;
    T iv_h;    // inv_vol / 2
    T nh4;     // -4 hd, hd = dt / (2 ds): the predictor's factor on products of halves
    T sc[5];   // update scale per field: -dt ds^2 / 2 (mass, momenta), / 4 (energy)
    T hq4;     // conducting wall: 4 Q/V per kelvin of (273 - t_in), the energy flux's scale
};

// Conducting-wall heat of one cell in the energy flux's scale (4 Q/V,
// wall_heat's formula with its constant factor folded into k.hq4); xr, xp:
// rho/2 and p/2 of the face's lower cell, whose quotient is t_in * RS.
template <class T> __device__ __forceinline__ T heat4(T xr, T xp, const K<T> &k) {
    return (T(273.0f) - xp / (T(287.0f) * xr)) * k.hq4;
}

// Conserved totals -> primitives (calc_primitives, physics.rs:112-140), the
// fast policy's operation sequence (the same as Phys<T, false>::prim, so the
// dt of the updated state agrees bit for bit with the state reduction).
template <class V, class T> __device__ __forceinline__ void prim(const V u[5], V w[5], const K<T> &k) {
    const V ir = vrcp(u[0]);
    const V rho = vmul(u[0], spl<V>(k.inv_vol));
    const V vx = vmul(u[1], ir), vy = vmul(u[2], ir), vz = vmul(u[3], ir);
    const V v2 = vfma(vz, vz, vfma(vy, vy, vmul(vx, vx)));
    w[0] = rho;
    w[1] = vx;
    w[2] = vy;
    w[3] = vz;
    w[4] = vmul(vfma(vmul(spl<V>(-0.5), rho), v2, vmul(u[4], spl<V>(k.inv_vol))), spl<V>(k.gm1));
}

// Half primitives: the march works on q/2 (and hence on half slopes s/2 from
// their differences), so that the face states xt -+ s/2 are plain sums.
// Every quantity is the full one scaled by a power of two, and the
// predictor below scales back exactly: results equal those of the full-size
// formulas bit for bit.  prim_half is prim's operation sequence on halves:
// 1/(2M), rho/2, v/2, |v|^2/4 and p/2 = (E/(2V) - 2 (rho/2)|v|^2/4)(gamma-1).
template <class V, class T> __device__ __forceinline__ void prim_half(const V u[5], V w[5], const K<T> &k) {
    const V irh = vrcp(vadd(u[0], u[0]));
    const V rho = vmul(u[0], spl<V>(k.iv_h));
    const V vx = vmul(u[1], irh), vy = vmul(u[2], irh), vz = vmul(u[3], irh);
    const V v2 = vfma(vz, vz, vfma(vy, vy, vmul(vx, vx)));
    w[0] = rho;
    w[1] = vx;
    w[2] = vy;
    w[3] = vz;
    const V t = vfma(vadd(rho, rho), v2, vmul(u[4], spl<V>(-(double)k.iv_h)));
    w[4] = vmul(t, spl<V>(-(double)k.gm1));
}

// Half-step predictor (extrapolate_primitives_t, physics.rs:251-278) on half
// primitives qh and half slopes (cell units): returns the full predicted
// state.  Every product of two halves is a quarter of the full product, so
// the sums are quarters and the factor is -4 hd (hd = dt / (2 ds)).
template <class V, class T>
__device__ __forceinline__ void predict(const V qh[5], const V sx[5], const V sy[5], const V sz[5], const K<T> &k,
                                        V out[5]) {
    const V rho = vadd(qh[0], qh[0]), vx = vadd(qh[1], qh[1]), vy = vadd(qh[2], qh[2]);
    const V vz = vadd(qh[3], qh[3]), p = vadd(qh[4], qh[4]);
    const V nh = spl<V>(k.nh4);
    const V ir = vrcp(vadd(rho, rho));   // 1 / (4 rho_h)
    const V div = vadd(vadd(sx[1], sy[2]), sz[3]);
    out[0] = vfma(nh, vfma(qh[0], div, vfma(qh[3], sz[0], vfma(qh[2], sy[0], vmul(qh[1], sx[0])))), rho);
    out[1] = vfma(nh, vfma(ir, sx[4], vfma(qh[3], sz[1], vfma(qh[2], sy[1], vmul(qh[1], sx[1])))), vx);
    out[2] = vfma(nh, vfma(ir, sy[4], vfma(qh[3], sz[2], vfma(qh[2], sy[2], vmul(qh[1], sx[2])))), vy);
    out[3] = vfma(nh, vfma(ir, sz[4], vfma(qh[3], sz[3], vfma(qh[2], sy[3], vmul(qh[1], sx[3])))), vz);
    const V gp = vmul(spl<V>(k.gamma), qh[4]);
    out[4] = vfma(nh, vfma(qh[3], sz[4], vfma(qh[2], sy[4], vfma(qh[1], sx[4], vmul(gp, div)))), p);
}

// Rusanov face flux (calc_flux_reconstruction, physics.rs:338-400): a is the
// state on the lower side of the face, b on the upper side, both (rho, vx,
// vy, vz, p); N is the index of the normal velocity.  Star state = mean of
// the two conserved states; flux = physical flux of the star state minus
// c/2 (U_b - U_a), c the larger of the two sides' c_s + |v_n|.  Returns
// 2F (mass, momenta) and 4F (energy), F without its *ds; with GRAV the
// gravity source term of the z faces (physics.rs:366-372), gh = G h.
template <int N, bool GRAV, class V, class T>
__device__ __forceinline__ void face(const V a[5], const V b[5], V gh, const K<T> &k, V F[5]) {
    constexpr int T1 = N == 1 ? 2 : 1, T2 = N == 3 ? 2 : 3;
    const V ra = a[0], ua = a[N], va = a[T1], wa = a[T2], pa = a[4];
    const V rb = b[0], ub = b[N], vb = b[T1], wb = b[T2], pb = b[4];
    const V mua = vmul(ra, ua), mva = vmul(ra, va), mwa = vmul(ra, wa);
    const V mub = vmul(rb, ub), mvb = vmul(rb, vb), mwb = vmul(rb, wb);
    // twice the total energy of each side: rho |v|^2 + 2 p / (gamma - 1)
    const V ea = vfma(mwa, wa, vfma(mva, va, vfma(mua, ua, vmul(spl<V>(k.kp), pa))));
    const V eb = vfma(mwb, wb, vfma(mvb, vb, vfma(mub, ub, vmul(spl<V>(k.kp), pb))));
    const V sr = vadd(ra, rb), smu = vadd(mua, mub), smv = vadd(mva, mvb), smw = vadd(mwa, mwb);
    const V se = vadd(ea, eb);
    const V irs = vrcp(sr);
    const V us = vmul(smu, irs);                                                 // star normal velocity
    const V kk = vfma(smu, us, vmul(vfma(smw, smw, vmul(smv, smv)), irs));       // |S_m|^2 / S_rho
    const V p2 = vfma(kk, spl<V>(-(double)k.c1), vmul(se, spl<V>(k.c1)));        // 2 p*
    const V ca = vfma(vmul(pa, vrsq(vmul(pa, ra))), spl<V>(k.sg), vabs(ua));   // c_s + |v_n|, side a
    const V cb = vfma(vmul(pb, vrsq(vmul(pb, rb))), spl<V>(k.sg), vabs(ub));
    const V c = vmax(ca, cb);
    V fu = vfma(smu, us, p2);
    V fe = vmul(vadd(vadd(p2, p2), se), us);
    if constexpr (GRAV) {
        fu = vfma(sr, gh, fu);
        fe = vfma(vmul(sr, vadd(ua, ub)), gh, fe);
    }
    // dissipation c (U_a - U_b) with the factors of the convention above
    F[0] = vfma(c, vsub(ra, rb), smu);
    F[N] = vfma(c, vsub(mua, mub), fu);
    F[T1] = vfma(c, vsub(mva, mvb), vmul(smv, us));
    F[T2] = vfma(c, vsub(mwa, mwb), vmul(smw, us));
    F[4] = vfma(c, vsub(ea, eb), fe);
}

// xt + s/2 (sign > 0) or xt - s/2: with half slopes hs = s/2, a sum
template <class V> __device__ __forceinline__ void half_step(const V xt[5], const V hs[5], double sign, V out[5]) {
#pragma unroll
    for (int f = 0; f < 5; ++f) out[f] = sign > 0 ? vadd(xt[f], hs[f]) : vsub(xt[f], hs[f]);
}

// Boundary modes of a tile side.
enum Mode : int { kNormal = 0, kOut = 1, kWallM = 2 };

__device__ __forceinline__ int side_mode(bool on_face, int bc) {
    if (!on_face || bc == kPeriodic) return kNormal;
    return bc == kOutflow ? kOut : kWallM;
}

template <class T, int TY, int R> struct Smem {
    static constexpr int kRows = TY + 4;                  // staged rows y0-2 .. y0+TY+1
    static constexpr int kFieldElems = kRows * kBoxZ;
    static constexpr int kBoxBytes = 5 * kFieldElems * (int)sizeof(T);
    static constexpr int kSlotElems = ((kBoxBytes + 127) / 128) * 128 / (int)sizeof(T);
    static constexpr int kPbRows = TY + 2;                // primitive rows y0-1 .. y0+TY
    T ring[R * kSlotElems];                               // conserved totals as staged
    T pb[2][5][kPbRows][kBoxZ];                           // primitives, by plane parity
    T ypl[2][TY + 1][5][kTileZ];                          // upper y state, rows y0-1 .. y0+TY-1
    T fy[2][TY + 1][5][kTileZ];                           // flux of the lower y face, rows y0 .. y0+TY
    T ytop[2][5][kTileZ];                                 // top row's xt (wall) or lower state (outflow)
    T zl[2][TY][5];                                       // left halo column: upper z state (wall: +sz/2)
    T zr[2][TY][5];                                       // right halo column: lower z state (wall: -sz/2)
    T zeu[2][TY][5];                                      // last column's upper z state (even width)
    T zex[2][TY][5];                                      // last column's xt (wall) or lower state (outflow)
    T fz[2][TY][5];                                       // flux of the right edge face (even width)
    uint64_t bar[R];
    double red[(TY + 2) * 7];
    // set when a wait gave up, read after the next barrier; two slots by
    // plane parity, so a warp already working on plane m + 1 cannot flag a
    // warp that is still between the barriers of plane m
    int abort_flag[2];
    int skip;
    int is_last;
};

template <class T, int TY, int R, int LIM, bool GRAV> struct Sweep {
    using V = typename PairT<T>::type;
    using Sm = Smem<T, TY, R>;
    static constexpr int W = TY + 2;      // warps: TY owned rows, A, B
    static constexpr int NT = 32 * W;
    static constexpr int WA = TY, WB = TY + 1;

    static __device__ __forceinline__ T *slot(Sm &s, int l) { return s.ring + (l % R) * Sm::kSlotElems; }
    // staged conserved value: field f, staged row ry (0 = y0-2), column cz (0 = z0-2)
    static __device__ __forceinline__ T &C(T *sl, int f, int ry, int cz) {
        return sl[(f * Sm::kRows + ry) * kBoxZ + cz];
    }
    static __device__ __forceinline__ V ldv(const T *p) { return *reinterpret_cast<const V *>(p); }
    static __device__ __forceinline__ void stv(T *p, V v) { *reinterpret_cast<V *>(p) = v; }

    static __device__ __forceinline__ V mirror(V v, bool on) { return on ? vmul(v, spl<V>(-1.0)) : v; }

    // Gravity height term of a z face whose lower cell has ghosted index klow.
    static __device__ __forceinline__ T grav_h(const GridArgs<T> &a, int klow) {
        return a.k.g * (T(a.nz - 4) * a.k.ds - T(klow - 2) * a.k.ds);
    }

    // NaN-propagating maximum of wave speeds.
    static __device__ __forceinline__ float smax_of(float m, float v) { return max_nan(m, v); }
    static __device__ __forceinline__ double smax_of(double m, double v) {
        return (m != m || v != v) ? (m + v) : fmax(m, v);
    }

    // Wave speeds c_s + |v| of the pair's cells in the updated state (the
    // quantity whose maximum sets the next dt, physics.rs:186-190).  FP32:
    // the state reduction's own scalar function (fast_speed), so that dt
    // agrees bit for bit with it; the packed form of the same operations
    // did not (one unit in the last place on some cells).  FP64: IEEE
    // square roots.
    static __device__ __forceinline__ V speed_pair(const V q[5], const K<T> &k) {
        if constexpr (sizeof(T) == 4) {
            return mk(fast_speed(q[0].x, q[1].x, q[2].x, q[3].x, q[4].x, k.gamma),
                      fast_speed(q[0].y, q[1].y, q[2].y, q[3].y, q[4].y, k.gamma));
        } else {
            auto one = [&](T r, T vx, T vy, T vz, T p) {
                return sqrt(k.gamma * p / r) + sqrt(vx * vx + vy * vy + vz * vz);
            };
            return mk(one(q[0].x, q[1].x, q[2].x, q[3].x, q[4].x), one(q[0].y, q[1].y, q[2].y, q[3].y, q[4].y));
        }
    }

    // The ghost-cell images of one updated cell (all but the cell itself):
    // the copies the reference's ghost fill makes of a cell next to a domain
    // face (axis_images: periodic wrap, outflow copy, wall mirror with the
    // normal momentum negated).  Rare: only cells within two of a face of a
    // grid of odd width.  Inlined like xy_images (a call in the march costs
    // more than the larger code).
    static __device__ __forceinline__ void images(const GridArgs<T> &a, int x, int y, int z, T u0, T u1, T u2, T u3,
                                               T u4) {
        int ximg[4], xflp[4], yimg[4], yflp[4], zimg[4], zflp[4];
        const int nxi = axis_images(x, a.nx, a.bc[0], a.bc[1], ximg, xflp);
        const int nyi = axis_images(y, a.ny, a.bc[2], a.bc[3], yimg, yflp);
        const int nzi = axis_images(z, a.nz, a.bc[4], a.bc[5], zimg, zflp);
        for (int ix = 0; ix < nxi; ++ix)
            for (int iy = 0; iy < nyi; ++iy)
                for (int iz = 0; iz < nzi; ++iz) {
                    if (ix == 0 && iy == 0 && iz == 0) continue;   // the cell itself
                    const long long o = ((long long)ximg[ix] * a.ny + yimg[iy]) * a.pitch + zimg[iz];
                    a.dst[o] = u0;
                    a.dst[a.fstride + o] = xflp[ix] ? -u1 : u1;
                    a.dst[2 * a.fstride + o] = yflp[iy] ? -u2 : u2;
                    a.dst[3 * a.fstride + o] = zflp[iz] ? -u3 : u3;
                    a.dst[4 * a.fstride + o] = u4;
                }
    }

    // An updated pair (or its first cell) at (xq, yq, z), and for a lane at
    // a z face of an even-width grid its z-image pair at zt (cells zc0, zc1
    // of the pair; field 3 negated for a wall); fields 1 / 2 negated for a
    // mirror along x / y.
    static __device__ __forceinline__ void put(const GridArgs<T> &a, int xq, int yq, int z, const V u[5], bool s0,
                                               bool s1, bool fx, bool fy, int zt, int zc0, int zc1, bool zflip) {
        const long long o = ((long long)xq * a.ny + yq) * a.pitch + z;
        if (s1) {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const bool neg = (f == 1 && fx) || (f == 2 && fy);
                stv(a.dst + f * a.fstride + o, neg ? vmul(u[f], spl<V>(-1.0)) : u[f]);
            }
            if (zt >= 0) {
                const long long oz = ((long long)xq * a.ny + yq) * a.pitch + zt;
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    V v = mk(zc0 ? u[f].y : u[f].x, zc1 ? u[f].y : u[f].x);
                    if ((f == 1 && fx) || (f == 2 && fy) || (f == 3 && zflip)) v = vmul(v, spl<V>(-1.0));
                    stv(a.dst + f * a.fstride + oz, v);
                }
            }
        } else if (s0) {
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const bool neg = (f == 1 && fx) || (f == 2 && fy);
                a.dst[f * a.fstride + o] = neg ? -u[f].x : u[f].x;
            }
        }
    }

    // The x / y ghost images of an updated pair next to an x or y face
    // (boundary planes and rows only): the pair again at every image plane
    // and row, with its z images (put).  Inlined: a call in the march
    // constrains the register allocation of the whole loop.
    static __device__ __forceinline__ void xy_images(const GridArgs<T> &a, int xu, int y, int z, V u0, V u1, V u2, V u3,
                                                  V u4, bool s0, bool s1, int zt, int zc0, int zc1, bool zflip) {
        const V u[5] = {u0, u1, u2, u3, u4};
        int ximg[4], xflp[4], yimg[4], yflp[4];
        const int nxi = axis_images(xu, a.nx, a.bc[0], a.bc[1], ximg, xflp);
        const int nyi = axis_images(y, a.ny, a.bc[2], a.bc[3], yimg, yflp);
        for (int ix = 0; ix < nxi; ++ix)
            for (int iy = 0; iy < nyi; ++iy)
                if (ix || iy) put(a, ximg[ix], yimg[iy], z, u, s0, s1, xflp[ix] != 0, yflp[iy] != 0, zt, zc0, zc1, zflip);
    }

    // Load a pair of staged conserved values and convert it.
    static __device__ __forceinline__ void load_prim_pair(T *sl, int ry, int cz, const K<T> &k, V q[5]) {
        V u[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) u[f] = ldv(&C(sl, f, ry, cz));
        prim_half(u, q, k);
    }
    // Two staged cells that are not adjacent (columns c0, c1 of row ry).
    static __device__ __forceinline__ void load_prim_split(T *sl, int ry, int c0, int c1, const K<T> &k, V q[5]) {
        V u[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) u[f] = mk(C(sl, f, ry, c0), C(sl, f, ry, c1));
        prim_half(u, q, k);
    }
    static __device__ __forceinline__ void store_pb(Sm &s, int par, int row, int col, const V q[5]) {
#pragma unroll
        for (int f = 0; f < 5; ++f) stv(&s.pb[par][f][row][col], q[f]);
    }

    // Slopes and prediction of the pair of adjacent cells at primitive-buffer
    // row `row`, columns (col, col + 1): x from the carried difference dq and
    // the new one dn, y from rows row -+ 1 (or the values ym / yp when given),
    // z from columns col - 1 and col + 2.
    static __device__ __forceinline__ void slopes_adj(Sm &s, int par, int row, int col, const V q[5], const V dq[5],
                                                      const V dn[5], const V *ym, const V *yp, V sx[5], V sy[5],
                                                      V sz[5]) {
#pragma unroll
        for (int f = 0; f < 5; ++f) {
            sx[f] = slope<LIM>(dq[f], dn[f]);
            const V m = ym ? ym[f] : ldv(&s.pb[par][f][row - 1][col]);
            const V p = yp ? yp[f] : ldv(&s.pb[par][f][row + 1][col]);
            sy[f] = slope<LIM>(vsub(q[f], m), vsub(p, q[f]));
            const T zl = s.pb[par][f][row][col - 1], zr = s.pb[par][f][row][col + 2];
            const T dmid = q[f].y - q[f].x;
            sz[f] = mk(slope1<LIM>(q[f].x - zl, dmid), slope1<LIM>(dmid, zr - q[f].y));
        }
    }

    // Block-wide barrier reached from the three roles' own code (bar.sync
    // counts arrivals, not call sites; every role takes the same sequence).
    static __device__ __forceinline__ void barrier() { asm volatile("bar.sync 0;" ::: "memory"); }

    // Plane nx-3 with a non-periodic upper x face: the owned warps stash the
    // ghost rule's operands in the y-state slot of parity (nx-2) & 1, which
    // the row above reads until the end of plane nx-4's second phase.  Every
    // role takes one more barrier at the start of that plane.
    static __device__ __forceinline__ bool upper_stash(const GridArgs<T> &a, int m) {
        return m == a.nx - 3 && a.bc[1] != kPeriodic;
    }

    // Geometry and constants of one work item, shared by the three roles.
    struct Tile {
        long long budget;   // SM clocks a wait for a staged plane may take
        int y0, z0, xs, xe, np, vy, vz, e;
        bool odd;
        int ylo, yhi, zlo, zhi;
        K<T> k;
        V gh, ghe;   // gravity terms: the lane's two lower z faces, the right edge face
    };

    static __device__ __forceinline__ bool wait_plane(Sm &s, int l, long long budget) {
        return mbar_wait(&s.bar[l % R], (l / R) & 1, budget);
    }

    // ---------------------------------------------------------------------
    // Owned warp: row y0 + r, lane pair at buffer columns (col, col + 1).
    //
    // Plane m's iteration, before the barrier: convert plane m+1; update
    // plane m-2 (its last fluxes arrived with the barrier of plane m-1) and
    // compute its wave speeds; slopes, prediction and the x-face flux
    // between planes m-1 and m; publish the face states other warps need;
    // store plane m-2.  After the barrier: the y- and z-face fluxes of plane
    // m.  The update comes first and its stores last, so that one straight
    // run of code interleaves its long dependency chain (loads, reciprocal,
    // square roots) with the slopes and the prediction of plane m.
    // ---------------------------------------------------------------------
    //
    // IN: the tile is interior (InteriorTiles): every row and column is
    // valid and no y or z face, ghost image or halo rule touches it, so the
    // boundary switches below are compile-time constants.
    template <bool IN>
    static __device__ void run_owned(Sm &s, const GridArgs<T> &a, const Tile &t, int r, int lane, T &smax) {
        const unsigned full = 0xffffffffu;
        const K<T> &k = t.k;
        const int col = 2 + 2 * lane;
        const bool active = IN || r < t.vy;
        const int y = t.y0 + r, z = t.z0 + 2 * lane;
        const bool val0 = IN || 2 * lane < t.vz, val1 = IN || 2 * lane + 1 < t.vz;
        const bool edge = IN ? lane == kTileZ / 2 - 1 : lane == t.e;
        const bool edge_even = edge && (IN || !t.odd);
        const bool yout = !IN && r == 0 && t.ylo == kOut;
        const bool zout = !IN && lane == 0 && t.zlo == kOut;
        const bool zheat = !IN && lane == 0 && t.zlo == kWallM && (a.heat & 4);
        const bool img_y = !IN && (y <= 3 || y >= a.ny - 4);
        const bool img_z = !IN && (z <= 3 || z + 1 >= a.nz - 4);
        // carried along the march: lox, the lower state of the x face ahead
        // (xt + s/2 of the previous plane); nacc, the previous plane's flux
        // balance so far, negated (its lower faces' fluxes enter with a plus
        // sign, so no flux is negated on its own; negation being exact, the
        // sums round as the balance itself would); tu, the update term of the
        // plane before it.  The own cell's primitives of the current and the
        // previous plane are read back from the primitive buffer.
        V lox[5], nacc[5], tu[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) lox[f] = nacc[f] = tu[f] = spl<V>(0.0);

        // Update of plane xu (staged index sl_idx) with the term tu: the new
        // state and its wave speeds (stores are left to the caller).
        auto update = [&](int xu, int sl_idx, V u[5], V &sp) {
            const int pp = xu & 1;
            T *sl = slot(s, sl_idx);
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                V tt = tu[f];
                // its upper y flux (row above) and right edge flux (warp B)
                if (!yout) tt = vadd(tt, ldv(&s.fy[pp][r + 1][f][2 * lane]));
                const T fe = s.fz[pp][r][f];
                tt.y += edge_even ? fe : T(0);
                u[f] = vfma(spl<V>(k.sc[f]), tt, ldv(&C(sl, f, r + 2, col)));
            }
            V w[5];
            prim(u, w, k);
            sp = speed_pair(w, k);
        };
        // Ghost images along z of the lane's pair.  With an even interior
        // width every pair is aligned with the faces, and the images of a
        // pair at a z face are one pair at zt: (u[c0], u[c1]), the z
        // momentum negated for a wall (axis_images' rules: periodic wrap,
        // outflow copy of the first/last cell, wall mirror).  Odd widths and
        // width 2 take the per-cell path (images()).
        const bool even_z = ((a.nz - 4) & 1) == 0 && a.nz - 4 >= 4;   // (width 2: both faces on one pair)
        int zt = -1, zc0 = 0, zc1 = 1;
        bool zflip = false;
        if (!IN && even_z && val1) {
            if (z == 2) {
                if (a.bc[4] == kPeriodic) { zt = a.nz - 2; }
                else if (a.bc[4] == kOutflow) { zt = 0; zc1 = 0; }
                else { zt = 0; zc0 = 1; zc1 = 0; zflip = true; }
            } else if (z + 1 == a.nz - 3) {
                if (a.bc[5] == kPeriodic) { zt = 0; }
                else if (a.bc[5] == kOutflow) { zt = a.nz - 2; zc0 = 1; }
                else { zt = a.nz - 2; zc0 = 1; zc1 = 0; zflip = true; }
            }
        }
        const bool zslow = !even_z && img_z;
        auto store = [&](int xu, const V u[5], const V &sp, bool on) {
            const bool s0 = on && val0, s1 = on && val1;
            if (s0) smax = smax_of(smax, sp.x);
            if (s1) smax = smax_of(smax, sp.y);
            put(a, xu, y, z, u, s0, s1, false, false, zt, zc0, zc1, zflip);
            const bool img_x = xu <= 3 || xu >= a.nx - 4;
            if (on && (img_x || img_y)) xy_images(a, xu, y, z, u[0], u[1], u[2], u[3], u[4], s0, s1, zt, zc0, zc1, zflip);
            if (on && zslow) {
                if (s0) images(a, xu, y, z, u[0].x, u[1].x, u[2].x, u[3].x, u[4].x);
                if (s1) images(a, xu, y, z + 1, u[0].y, u[1].y, u[2].y, u[3].y, u[4].y);
            }
        };

        // prologue: planes xs-2, xs-1 (the own row of both into the buffer)
        bool ok = wait_plane(s, 0, t.budget);
        if (ok && active) {
            V q0[5];
            load_prim_pair(slot(s, 0), r + 2, col, k, q0);
            store_pb(s, t.xs & 1, r + 1, col, q0);
        }
        ok = ok && wait_plane(s, 1, t.budget);
        if (ok && active) {
            V q1[5];
            load_prim_pair(slot(s, 1), r + 2, col, k, q1);
            store_pb(s, (t.xs - 1) & 1, r + 1, col, q1);
        }
        if (!ok) s.abort_flag[t.xs & 1] = 1;
        fence_proxy_async();
        barrier();
        if (s.abort_flag[t.xs & 1]) return;
        bool aborted = false;
        for (int m = t.xs - 1; m <= t.xe; ++m) {
            const int l = m - t.xs + 3;
            const int pm = m & 1;
            const bool upd = m >= t.xs && m < t.xe;
            V sy[5], sz[5], xtc[5];
            if (upper_stash(a, m)) barrier();
            if (!wait_plane(s, l, t.budget)) s.abort_flag[m & 1] = 1;
            if (active) {
                V q[5], dq[5], qn[5], dn[5], sx[5], xt[5], u[5], sp;
                // the own cell at planes m and m-1 (this thread's entries), read
                // before the conversion of plane m+1 replaces plane m-1's
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    q[f] = ldv(&s.pb[pm][f][r + 1][col]);
                    dq[f] = vsub(q[f], ldv(&s.pb[pm ^ 1][f][r + 1][col]));
                }
                load_prim_pair(slot(s, l), r + 2, col, k, qn);
                store_pb(s, pm ^ 1, r + 1, col, qn);
                // update of plane m-2 (from plane xs on; earlier iterations
                // compute on a valid slot and store nothing)
                const bool do_upd = m - 2 >= t.xs;
                update(m - 2, do_upd ? l - 3 : 0, u, sp);
#pragma unroll
                for (int f = 0; f < 5; ++f) dn[f] = vsub(qn[f], q[f]);
                slopes_adj(s, pm, r + 1, col, q, dq, dn, nullptr, nullptr, sx, sy, sz);
                predict(q, sx, sy, sz, k, xt);
                // ghost rules of the x faces (rare planes): a wall's ghost
                // plane 1 takes the mirrored prediction of plane 2 with its
                // own slope; the upper ghost plane takes the last plane's state
                // and slope (outflow) or its mirrored prediction with its own
                // slope (wall).  The operands wait one plane in the own row's
                // slot of the y-state buffer of the parity no plane publishes
                // meanwhile: ypl[0] before plane 2 publishes, ypl[(nx-2) & 1]
                // after plane nx-4 was read (upper_stash's barrier) and with
                // no upper ghost publish.
                // planes next to an x face (ghost rules, their stash, the
                // lower outflow face, heat) take the full path; the others
                // one test
                if (m > 3 && m < a.nx - 3) {
                    if (m >= t.xs) {
                        V up[5], fx[5];
                        half_step(xt, sx, -1.0, up);
                        face<1, false>(lox, up, spl<V>(0.0), k, fx);
#pragma unroll
                        for (int f = 0; f < 5; ++f) {
                            tu[f] = vsub(fx[f], nacc[f]);
                            nacc[f] = fx[f];
                        }
                    }
                } else {
                    const bool wall_lo = a.bc[0] == kWall, hi_rule = a.bc[1] != kPeriodic;
                    T *stash = &s.ypl[m == 1 ? 0 : (a.nx - 2) & 1][r + 1][0][2 * lane];
                    if ((m == 1 && wall_lo) || (m == a.nx - 3 && hi_rule)) {
    #pragma unroll
                        for (int f = 0; f < 5; ++f) {
                            // lower wall: plane 1's slope; upper outflow: xt - s/2;
                            // upper wall: the mirrored xt
                            const V v = m == 1 ? sx[f]
                                               : (a.bc[1] == kOutflow ? vsub(xt[f], sx[f]) : mirror(xt[f], f == 1));
                            stv(stash + f * kTileZ, v);
                        }
                    }
                    if (m >= t.xs) {
                        V lo[5], up[5], fx[5];
                        half_step(xt, sx, -1.0, up);
    #pragma unroll
                        for (int f = 0; f < 5; ++f) lo[f] = lox[f];
                        if (m == 2 && wall_lo) {
                            const T *st0 = &s.ypl[0][r + 1][0][2 * lane];
    #pragma unroll
                            for (int f = 0; f < 5; ++f) lo[f] = vadd(mirror(xt[f], f == 1), ldv(st0 + f * kTileZ));
                        }
                        if (m == a.nx - 2 && hi_rule) {
                            const T *st1 = &s.ypl[(a.nx - 2) & 1][r + 1][0][2 * lane];
    #pragma unroll
                            for (int f = 0; f < 5; ++f) {
                                const V v = ldv(st1 + f * kTileZ);
                                up[f] = a.bc[1] == kOutflow ? v : vsub(v, sx[f]);
                            }
                        }
                        face<1, false>(lo, up, spl<V>(0.0), k, fx);
                        // plane m-1 is complete but for its upper y flux and its
                        // right edge flux (added at its update, two planes on); on
                        // a lower outflow x face plane 2 sees no x divergence
                        const bool xo_prev = m - 1 == 2 && a.bc[0] == kOutflow;
                        const bool xo = m == 2 && a.bc[0] == kOutflow;
    #pragma unroll
                        for (int f = 0; f < 5; ++f) {
                            tu[f] = xo_prev ? vmul(nacc[f], spl<V>(-1.0)) : vsub(fx[f], nacc[f]);
                            nacc[f] = xo ? spl<V>(0.0) : fx[f];
                        }
                        if (m == 2 && (a.heat & 1)) {
                            // conducting lower x face: its heat enters plane 2
                            // (the ghost plane's state mirrors plane 2's)
                            nacc[4].x += heat4(xt[0].x, xt[4].x, k);
                            nacc[4].y += heat4(xt[0].y, xt[4].y, k);
                        }
                    }
                }
                half_step(xt, sx, 1.0, lox);
#pragma unroll
                for (int f = 0; f < 5; ++f) xtc[f] = xt[f];
                if (upd) {
                    V st[5];
                    half_step(xt, sy, 1.0, st);
#pragma unroll
                    for (int f = 0; f < 5; ++f) stv(&s.ypl[pm][r + 1][f][2 * lane], st[f]);
                    if (!IN && r == t.vy - 1 && t.yhi != kNormal) {
                        // for the face above the top row (computed by warp B)
                        if (t.yhi == kOut) half_step(xt, sy, -1.0, st);
#pragma unroll
                        for (int f = 0; f < 5; ++f) stv(&s.ytop[pm][f][2 * lane], t.yhi == kOut ? st[f] : xt[f]);
                    }
                    if (edge_even) {
                        // the right edge face (warp B) needs the last column's states
#pragma unroll
                        for (int f = 0; f < 5; ++f) {
                            s.zeu[pm][r][f] = xt[f].y + sz[f].y;
                            s.zex[pm][r][f] = (!IN && t.zhi == kOut) ? xt[f].y - sz[f].y : xt[f].y;
                        }
                    }
                }
                store(m - 2, u, sp, do_upd);
            }
            fence_proxy_async();
            barrier();
            if (s.abort_flag[m & 1]) { aborted = true; break; }
            if (!active || !upd) continue;
            // ================= after the barrier: y and z faces of plane m
            const V *xt = xtc;
            V ndy[5];   // the lower y face's flux (plus the heat of a conducting face)
            if (!yout) {
                V lo[5], up[5], fyv[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) lo[f] = ldv(&s.ypl[pm][r][f][2 * lane]);
                if (!IN && r == 0 && t.ylo == kWallM) {
                    // wall ghost row: mirrored prediction of this row + its own half slope
#pragma unroll
                    for (int f = 0; f < 5; ++f) lo[f] = vadd(lo[f], mirror(xt[f], f == 2));
                }
                half_step(xt, sy, -1.0, up);
                face<2, false>(lo, up, spl<V>(0.0), k, fyv);
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    stv(&s.fy[pm][r][f][2 * lane], fyv[f]);
                    ndy[f] = fyv[f];
                }
                if (!IN && r == 0 && t.ylo == kWallM && (a.heat & 2)) {
                    // conducting lower y face (the ghost row mirrors row 2)
                    ndy[4].x += heat4(xt[0].x, xt[4].x, k);
                    ndy[4].y += heat4(xt[0].y, xt[4].y, k);
                }
            } else {
#pragma unroll
                for (int f = 0; f < 5; ++f) ndy[f] = spl<V>(0.0);
            }
            V lo[5], up[5], fzv[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                const V U = vadd(xt[f], sz[f]);
                const V L = vsub(xt[f], sz[f]);
                // the halo columns' states (broadcast loads, used by lane 0
                // and, for an odd width, by the edge lane)
                const T mx = f == 3 ? -xt[f].x : xt[f].x;   // wall mirror of the pair's first cell
                T zlv = s.zl[pm][r][f];
                if (!IN && t.zlo == kWallM) zlv += mx;
                T zrv = s.zr[pm][r][f];
                if (!IN && t.zhi == kWallM) zrv += mx;
                if (!IN && t.zhi == kOut) zrv = L.x;
                const T left = __shfl_up_sync(full, U.y, 1);
                lo[f] = mk(lane == 0 ? zlv : left, U.x);
                // odd width: the edge lane's second cell is the right ghost column
                up[f] = mk(L.x, !IN && edge && t.odd ? zrv : L.y);
            }
            face<3, GRAV>(lo, up, t.gh, k, fzv);
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                T hi = __shfl_down_sync(full, fzv[f].x, 1);
                if (edge_even) hi = T(0);   // right edge face: added at the update
                V dz = vsub(mk(fzv[f].y, hi), fzv[f]);
                if (zout) dz.x = T(0);
                // conducting lower z face: the heat of the first column
                if (f == 4 && zheat) dz.x -= heat4(xt[0].x, xt[4].x, k);
                nacc[f] = vadd(nacc[f], vsub(ndy[f], dz));
            }
        }
        // the last plane of the chunk: its fluxes arrived with the last barrier
        if (!aborted && active && t.xe - 1 >= t.xs) {
            V u[5], sp;
            update(t.xe - 1, t.xe - t.xs + 1, u, sp);
            store(t.xe - 1, u, sp, true);
        }
    }

    // ---------------------------------------------------------------------
    // Halo warp A: the row below the tile (y0 - 1, lanes as pairs), the
    // halo columns z0 - 1 and z0 + vz of rows y0 .. y0 + vy - 1 (lane l: row
    // y0 + l, the two columns as one pair), the primitives of the staged
    // columns outside the lanes' pairs, and the TMA copies.  Returns the
    // number of planes it requested.
    // ---------------------------------------------------------------------
    static __device__ int run_a(Sm &s, const GridArgs<T> &a, const CUtensorMap *tmap, const Tile &t, int lane) {
        const K<T> &k = t.k;
        const int col = 2 + 2 * lane;
        const bool tl = lane < t.vy;
        const bool cl = lane < 2 * (TY + 2);
        const int crow = lane >> 1, ccol = (lane & 1) ? kTileZ + 2 : 0;
        const int rc = t.vz + 2;   // buffer column of the right halo column
        int issued = t.np < R ? t.np : R;
        V q[5], dq[5], q2[5], qt[5], dqt[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) q[f] = dq[f] = q2[f] = qt[f] = dqt[f] = spl<V>(0.0);
        auto convert = [&](int l, V qn[5], V q2n[5], V qtn[5], bool store) {
            T *sl = slot(s, l);
            const int par = (t.xs - 2 + l) & 1;
            load_prim_pair(sl, 0, col, k, q2n);
            load_prim_pair(sl, 1, col, k, qn);
            if (tl) load_prim_split(sl, lane + 2, 1, rc, k, qtn);
            if (store) {
                store_pb(s, par, 0, col, qn);
                if (cl) {
                    V c[5];
                    load_prim_pair(sl, crow + 1, ccol, k, c);
                    store_pb(s, par, crow, ccol, c);
                }
            }
        };
        bool ok = wait_plane(s, 0, t.budget);
        if (ok) convert(0, q, q2, qt, false);
        ok = ok && wait_plane(s, 1, t.budget);
        if (ok) {
            V qn[5], q2n[5], qtn[5];
            convert(1, qn, q2n, qtn, true);
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                dq[f] = vsub(qn[f], q[f]);
                q[f] = qn[f];
                q2[f] = q2n[f];
                dqt[f] = vsub(qtn[f], qt[f]);
                qt[f] = qtn[f];
            }
        }
        if (!ok) s.abort_flag[t.xs & 1] = 1;
        fence_proxy_async();
        barrier();
        if (s.abort_flag[t.xs & 1]) return issued;
        for (int m = t.xs - 1; m <= t.xe; ++m) {
            const int l = m - t.xs + 3;
            const int pm = m & 1;
            const bool upd = m >= t.xs && m < t.xe;
            if (upper_stash(a, m)) barrier();
            if (!wait_plane(s, l, t.budget)) s.abort_flag[m & 1] = 1;
            V qn[5], q2n[5], qtn[5], dn[5], dtn[5];
#pragma unroll
            for (int f = 0; f < 5; ++f) qtn[f] = spl<V>(0.0);
            convert(l, qn, q2n, qtn, true);
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                dn[f] = vsub(qn[f], q[f]);
                dtn[f] = vsub(qtn[f], qt[f]);
            }
            if (upd) {
                V sx[5], sy[5], sz[5], xt[5], st[5];
                if (t.ylo != kOut) {
                    // row y0 - 1: its upper face state (wall ghost: its own half slope)
                    slopes_adj(s, pm, 0, col, q, dq, dn, q2, nullptr, sx, sy, sz);
                    if (t.ylo == kNormal) {
                        predict(q, sx, sy, sz, k, xt);
                        half_step(xt, sy, 1.0, st);
                    } else {
#pragma unroll
                        for (int f = 0; f < 5; ++f) st[f] = sy[f];
                    }
#pragma unroll
                    for (int f = 0; f < 5; ++f) stv(&s.ypl[pm][0][f][2 * lane], st[f]);
                }
                if (tl && !(t.zlo == kOut && t.zhi == kOut)) {
                    // halo columns of row y0 + lane: left (x) and right (y) of the pair
                    const int row = lane + 1;
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        sx[f] = slope<LIM>(dqt[f], dtn[f]);
                        const V ym = mk(s.pb[pm][f][row - 1][1], s.pb[pm][f][row - 1][rc]);
                        const V yp = mk(s.pb[pm][f][row + 1][1], s.pb[pm][f][row + 1][rc]);
                        sy[f] = slope<LIM>(vsub(qt[f], ym), vsub(yp, qt[f]));
                        const V zm = mk(s.pb[pm][f][row][0], s.pb[pm][f][row][rc - 1]);
                        const V zp = mk(s.pb[pm][f][row][2], s.pb[pm][f][row][rc + 1]);
                        sz[f] = slope<LIM>(vsub(qt[f], zm), vsub(zp, qt[f]));
                    }
                    predict(qt, sx, sy, sz, k, xt);
#pragma unroll
                    for (int f = 0; f < 5; ++f) {
                        const T hz0 = sz[f].x, hz1 = sz[f].y;   // half slopes
                        s.zl[pm][lane][f] = t.zlo == kWallM ? hz0 : xt[f].x + hz0;
                        s.zr[pm][lane][f] = t.zhi == kWallM ? -hz1 : xt[f].y - hz1;
                    }
                }
            }
#pragma unroll
            for (int f = 0; f < 5; ++f) {
                q[f] = qn[f];
                dq[f] = dn[f];
                q2[f] = q2n[f];
                qt[f] = qtn[f];
                dqt[f] = dtn[f];
            }
            fence_proxy_async();
            barrier();
            if (s.abort_flag[m & 1]) break;
            // from plane xs on, the barrier frees the slot of plane m-2
            // (staged index m - xs): stage plane m-2+R there (the first R
            // planes were staged before the march)
            const int nl = m - t.xs + R;
            if (m >= t.xs && nl < t.np) {
                if (lane == 0) {
                    mbar_expect_tx(&s.bar[nl % R], Sm::kBoxBytes);
                    tma_load_4d(slot(s, nl), tmap, t.z0 - 2, t.y0 - 2, t.xs - 2 + nl, 0, &s.bar[nl % R]);
                }
                issued = nl + 1;
            }
        }
        return issued;
    }

    // ---------------------------------------------------------------------
    // Halo warp B: the row above the tile (y0 + vy, lanes as pairs), the
    // face between it and the tile's top row, and (even tile width) the
    // faces on the tile's right edge, two rows per lane.
    // ---------------------------------------------------------------------
    static __device__ void run_b(Sm &s, const GridArgs<T> &a, const Tile &t, int lane) {
        const K<T> &k = t.k;
        const int col = 2 + 2 * lane;
        const int br = t.vy + 1;   // buffer row of y0 + vy
        V q[5], dq[5], q2[5], lb[5];
#pragma unroll
        for (int f = 0; f < 5; ++f) q[f] = dq[f] = q2[f] = lb[f] = spl<V>(0.0);
        bool ok = wait_plane(s, 0, t.budget);
        if (ok) {
            load_prim_pair(slot(s, 0), br + 1, col, k, q);
            load_prim_pair(slot(s, 0), br + 2, col, k, q2);
        }
        ok = ok && wait_plane(s, 1, t.budget);
        if (ok) {
            V qn[5];
            load_prim_pair(slot(s, 1), br + 1, col, k, qn);
            load_prim_pair(slot(s, 1), br + 2, col, k, q2);
            store_pb(s, (t.xs - 1) & 1, br, col, qn);
#pragma unroll
            for (int f = 0; f < 5; ++f) { dq[f] = vsub(qn[f], q[f]); q[f] = qn[f]; }
        }
        if (!ok) s.abort_flag[t.xs & 1] = 1;
        fence_proxy_async();
        barrier();
        if (s.abort_flag[t.xs & 1]) return;
        for (int m = t.xs - 1; m <= t.xe; ++m) {
            const int l = m - t.xs + 3;
            const int pm = m & 1;
            const bool upd = m >= t.xs && m < t.xe;
            if (upper_stash(a, m)) barrier();
            if (!wait_plane(s, l, t.budget)) s.abort_flag[m & 1] = 1;
            V qn[5], q2n[5], dn[5];
            load_prim_pair(slot(s, l), br + 1, col, k, qn);
            load_prim_pair(slot(s, l), br + 2, col, k, q2n);
            store_pb(s, (m + 1) & 1, br, col, qn);
#pragma unroll
            for (int f = 0; f < 5; ++f) dn[f] = vsub(qn[f], q[f]);
            if (upd && t.yhi != kOut) {
                V sx[5], sy[5], sz[5], xt[5];
                slopes_adj(s, pm, br, col, q, dq, dn, nullptr, q2, sx, sy, sz);
                if (t.yhi == kNormal) {
                    predict(q, sx, sy, sz, k, xt);
                    half_step(xt, sy, -1.0, lb);
                } else {
#pragma unroll
                    for (int f = 0; f < 5; ++f) lb[f] = vmul(sy[f], spl<V>(-1.0));
                }
            }
#pragma unroll
            for (int f = 0; f < 5; ++f) { q[f] = qn[f]; dq[f] = dn[f]; q2[f] = q2n[f]; }
            fence_proxy_async();
            barrier();
            if (s.abort_flag[m & 1]) break;
            if (!upd) continue;
            {   // face (y0+vy-1 | y0+vy)
                V lo[5], up[5], F[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    lo[f] = ldv(&s.ypl[pm][t.vy][f][2 * lane]);
                    if (t.yhi == kNormal) up[f] = lb[f];
                    else {
                        const V x = ldv(&s.ytop[pm][f][2 * lane]);
                        up[f] = t.yhi == kOut ? x : vadd(lb[f], mirror(x, f == 2));
                    }
                }
                face<2, false>(lo, up, spl<V>(0.0), k, F);
#pragma unroll
                for (int f = 0; f < 5; ++f) stv(&s.fy[pm][t.vy][f][2 * lane], F[f]);
            }
            if (!t.odd && lane < TY / 2) {
                // right edge faces of rows lane and lane + TY/2
                const int ra = lane, rb = lane + TY / 2;
                V lo[5], up[5], F[5];
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    lo[f] = mk(s.zeu[pm][ra][f], s.zeu[pm][rb][f]);
                    const V zr = mk(s.zr[pm][ra][f], s.zr[pm][rb][f]);
                    const V zx = mk(s.zex[pm][ra][f], s.zex[pm][rb][f]);
                    up[f] = t.zhi == kNormal ? zr : (t.zhi == kOut ? zx : vadd(zr, mirror(zx, f == 3)));
                }
                face<3, GRAV>(lo, up, t.ghe, k, F);
#pragma unroll
                for (int f = 0; f < 5; ++f) {
                    s.fz[pm][ra][f] = F[f].x;
                    s.fz[pm][rb][f] = F[f].y;
                }
            }
        }
    }

    // One work item: tile (ty, tz) of grid `a`, x-planes of chunk cx.  Its
    // partial result goes to a.part[part_idx]; the last of the grid's
    // nparts items reduces them (next dt).  Returns false after a
    // device-side wait timed out (status flag set).
    template <bool IN>
    static __device__ bool run_tile(const GridArgs<T> &a, const CUtensorMap *tmap, int tz, int ty, int cx, int chunk,
                                    int part_idx, int nparts, unsigned char *raw) {
        Sm &s = *reinterpret_cast<Sm *>(raw);
        const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
        Tile t;
        t.budget = wait_budget_of(a);
        t.y0 = 2 + ty * TY;
        t.z0 = 2 + tz * kTileZ;
        t.xs = 2 + cx * chunk;
        t.xe = min(t.xs + chunk, a.nx - 2);
        t.np = t.xe - t.xs + 4;
        t.vy = min(TY, a.ny - 2 - t.y0);
        t.vz = min(kTileZ, a.nz - 2 - t.z0);
        t.e = (t.vz - 1) >> 1;
        t.odd = (t.vz & 1) != 0;
        t.ylo = side_mode(t.y0 == 2, a.bc[2]);
        t.yhi = side_mode(t.y0 + t.vy == a.ny - 2, a.bc[3]);
        t.zlo = side_mode(t.z0 == 2, a.bc[4]);
        t.zhi = side_mode(t.z0 + t.vz == a.nz - 2, a.bc[5]);

        const unsigned step = (unsigned)a.ctl->step;
        const T dt = (T)a.ctl->dt[step & 1];
        t.k.inv_vol = a.k.inv_vol;
        t.k.gamma = a.k.gamma;
        t.k.gm1 = a.k.gm1;
        t.k.kp = T(2) * a.k.inv_gm1;
        t.k.c1 = T(0.5) * a.k.gm1;
        t.k.sg = (T)sqrt((double)a.k.gamma);
        t.k.iv_h = T(0.5) * a.k.inv_vol;
        t.k.nh4 = T(-2) * dt * a.k.inv_ds;   // -4 dt / (2 ds)
        {
            const T scale = dt * a.k.ds * a.k.ds;
            t.k.sc[0] = t.k.sc[1] = t.k.sc[2] = t.k.sc[3] = T(-0.5) * scale;
            t.k.sc[4] = T(-0.25) * scale;
            // wall_heat's factor S / (d/kappa + 1/hc_out) / V, times 4
            const T ds = a.k.ds;
            t.k.hq4 = T(4) * ((ds * ds) / ((T(0.008f) / T(0.2f)) + (T(1.0f) / T(10.0f)))) / (ds * ds * ds);
        }
        t.gh = t.ghe = spl<V>(0.0);
        if constexpr (GRAV) {
            t.gh = mk(grav_h(a, grav_klow(t.z0 + 2 * lane - 1, a.nz, a.bc[4])), grav_h(a, t.z0 + 2 * lane));
            const T g1 = grav_h(a, t.z0 + t.vz - 1);
            t.ghe = mk(g1, g1);
        }

        // an earlier step's wait gave up: leave the state alone (read once,
        // so every thread of the block takes the same branch)
        if (tid == 0) {
            s.skip = (*(volatile unsigned *)&a.ctl->flags & kStatusTimeout) != 0;
            s.abort_flag[0] = s.abort_flag[1] = 0;
            if (!s.skip) {
                for (int i = 0; i < R; ++i) mbar_init(&s.bar[i], 1);
                fence_mbar_init();
            }
        }
        __syncthreads();
        if (s.skip) return false;
        if (warp == WA && lane == 0) {
            for (int l = 0; l < R && l < t.np; ++l) {
                mbar_expect_tx(&s.bar[l], Sm::kBoxBytes);
                tma_load_4d(slot(s, l), tmap, t.z0 - 2, t.y0 - 2, t.xs - 2 + l, 0, &s.bar[l]);
            }
        }
        T smax = T(0);
        int issued = 0;
        if (warp < TY) run_owned<IN>(s, a, t, warp, lane, smax);
        else if (warp == WA) issued = run_a(s, a, tmap, t, lane);
        else run_b(s, a, t, lane);
        __syncthreads();
        if (s.abort_flag[0] | s.abort_flag[1]) {
            if (warp == WA && lane == 0) {
                // let the copies in flight land before the block exits
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
        double wmin;
        if constexpr (sizeof(T) == 4) wmin = nanf ? INFINITY : (double)__fdiv_rn(a.k.ds, smax);
        else wmin = nanf ? INFINITY : a.k.ds / smax;
        double sum[5] = {0, 0, 0, 0, 0};
        if (block_partial(a, sum, wmin, nanf, tid, NT, s.red, &s.is_last, part_idx, nparts)) {
            __threadfence();
            final_reduce<T>(a, tid, NT, s.red, kAdvance, nparts);
        }
        return true;
    }
};

// Shared memory of one block (bytes), with room to align the base to 1 KB.
template <class T, int TY, int R> constexpr int smem_bytes() {
    static_assert(sizeof(Smem<T, TY, R>) + 1024 <= 232448, "sweep tile exceeds the 227 KB of shared memory per block");
    return (int)sizeof(Smem<T, TY, R>) + 1024;
}

// Registers per thread: a block's warps are spread over the SM's four
// sub-partitions, each with 16384 registers, so the busiest one (ceil(W/4)
// warps) bounds them; in the allocation granule of 8, at most 255.
template <int TY> constexpr int sweep_max_regs() {
    constexpr int per_sub = (TY + 2 + 3) / 4;
    constexpr int r = 16384 / (32 * per_sub) / 8 * 8;
    return r > 255 ? 255 : r;
}

// One step's interior launch (IN; blocks: interior tiles x chunks, whole
// columns when they fill the SMs: interior_chunk) or frame launch (blocks:
// frame tiles x chunks), InteriorTiles.
// The two touch disjoint tiles of the output and read only the input state,
// so the frame launch may run beside the interior one (programmatic
// dependent launch, launch_sweep).  They share one reduction: the interior
// blocks hold partials [0, n_in), the frame blocks the rest, and whichever
// block of either takes the last ticket advances dt (every block has read
// the step's dt by then).  Without interior tiles the frame launch is the
// whole step (n_in = 0).
template <class T, int TY, int R, int LIM, bool GRAV, bool IN>
__global__ void __maxnreg__(sweep_max_regs<TY>()) sweep_step_kernel(const GridArgs<T> a,
                                                                      const __grid_constant__ CUtensorMap tmap,
                                                                      int chunk, int n_in, int nparts) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // the frame launch reads nothing this launch writes: let it start on the
    // SMs this launch leaves free
    if constexpr (IN) asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
    const InteriorTiles it(a.ny, a.nz, TY, kTileZ);
    int b = blockIdx.x, ty, tz;
    if constexpr (IN) {
        tz = 1 + b % it.nz;
        b /= it.nz;
        ty = 1 + b % it.ny;
        b /= it.ny;
    } else {
        const int nf = it.frame();
        it.frame_tile(b % nf, ty, tz);
        b /= nf;
    }
    const int part = IN ? (int)blockIdx.x : n_in + (int)blockIdx.x;
    Sweep<T, TY, R, LIM, GRAV>::template run_tile<IN>(a, &tmap, tz, ty, b, chunk, part, nparts, smem_raw);
}

// Batched step: one persistent launch advances many independent grids by
// one step each.  Work items (grid, tile, x-chunk) are taken from an atomic
// queue; each grid keeps its own control block, so its dt is its own CFL dt.
// Grid arguments are copied to shared memory per item and then to
// registers; the grid's TMA descriptor is read from global memory (written
// by the host before launch).  All grids of one launch share the limiter and
// the gravity switch (the host launches one kernel per combination).
struct BatchItem {
    int g, local, tz, ty, cx;
};

template <int TY, int R, int LIM, bool GRAV>
__global__ void __maxnreg__(sweep_max_regs<TY>()) sweep_batch_kernel(const GridArgs<float> *__restrict__ args,
                                                                     const CUtensorMap *__restrict__ maps,
                                                                     const BatchItem *__restrict__ items,
                                                                     int nitems, unsigned *queue, int chunk) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    __shared__ int s_item;
    __shared__ __align__(16) GridArgs<float> s_args;
    const int tid = threadIdx.x;
    for (;;) {
        if (tid == 0) s_item = (int)atomicAdd(queue, 1u);
        __syncthreads();
        const int it = s_item;
        if (it >= nitems) return;
        const BatchItem bi = items[it];
        constexpr int kWords = (int)(sizeof(GridArgs<float>) / 4);
        for (int i = tid; i < kWords; i += blockDim.x)
            reinterpret_cast<int *>(&s_args)[i] = reinterpret_cast<const int *>(&args[bi.g])[i];
        __syncthreads();
        const GridArgs<float> ga = s_args;
        const bool ok = Sweep<float, TY, R, LIM, GRAV>::template run_tile<false>(ga, &maps[bi.g], bi.tz, bi.ty, bi.cx, chunk,
                                                                 bi.local, ga.nparts, smem_raw);
        __syncthreads();
        if (!ok) return;
    }
}

}  // namespace sweep
}  // namespace dg
