// dg_physics.cuh -- per-cell and per-face arithmetic of deep-green's Euler
// step, shared by every kernel of this library.
//
// Two arithmetic policies implement the same formulas (deep-green
// src/rs/src/physics.rs; each function cites the lines it follows):
//
//   Phys<T, true>   "reference rounding": the reference's operation order and
//                   association, IEEE division and square root.  Compiled
//                   without fused multiply-add contraction (--fmad=false) it
//                   rounds exactly like the reference's scalar code, so the
//                   GPU result equals the CPU restatement bit for bit.  Used
//                   for FP64 and, on request, for FP32.
//   Phys<T, false>  "fast": the conversion of a state to primitives with one
//                   reciprocal and fused multiply-adds, as the fused-arithmetic
//                   sweep kernel (dg_sweep_impl.cuh) computes it; used by the
//                   reductions and conversions that must agree with it.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace dg {

// Boundary types in the kernels (DG_BC_*): a conducting wall (DG_BC_CONDUCTING_WALL)
// reaches them as kWall plus a heat-source flag (GridArgs::heat).
enum Bc : int { kPeriodic = 0, kOutflow = 1, kWall = 2 };

// Lower-cell index whose gravity height a z face's flux carries.  The
// reference copies the flux of face nz-3 into face 1 on a periodic z axis
// (apply_boundary_conditions4 on the fluxes, boundaries.rs:113-118): the
// first interior cell's lower face carries the top face's gravity term.
__host__ __device__ __forceinline__ int grav_klow(int klow, int nz, int bc_zlo) {
    return klow == 1 && bc_zlo == kPeriodic ? nz - 3 : klow;
}

// Conducting-wall heat per unit volume, Q / V, of the reference's CUDA flux
// kernel (src/cu/include/kernels.h:561-575) in its operation order, with its
// constants (constants.h:63-66: RS = 287, T_OUT_KELVIN = 273, VOUT_MS = 0;
// wall thickness d = 0.008 and conductivity kappa = 0.2 as float literals)
// and t_in = p / (RS rho) of the face's lower cell (its extrapolated state).
template <class T> __host__ __device__ __forceinline__ T wall_heat(T rho, T p, T ds) {
    const T rs = T(287.0f), t_out = T(273.0f), vout = T(0.0f);
    const T t_in = p / (rs * rho);
    const T hc_out = T(10.0f) - vout + T(10.0f) * sqrt(vout);
    const T S = ds * ds;
    const T V = ds * ds * ds;
    const T d = T(0.008f), kappa = T(0.2f);
    const T Q = (t_out - t_in) * (S / ((d / kappa) + (T(1.0f) / hc_out)));
    return Q / V;
}

// Runtime constants of one grid, derived once on the host in precision T.
template <class T> struct Consts {
    T ds;        // cell size
    T vol;       // ds*ds*ds (physics.rs:110, powi(3))
    T inv_vol;   // 1 / vol
    T gamma;     // ratio of specific heats (globals.rs:3)
    T gm1;       // gamma - 1
    T inv_gm1;   // 1 / (gamma - 1)
    T half_ds;   // ds / 2 : face reconstruction offset (physics.rs:313-336)
    T two_ds;    // 2 * ds : central-difference denominator (physics.rs:206)
    T inv_ds;    // 1 / ds
    T inv_2ds;   // 1 / (2 ds)
    T cfl;       // globals.rs:4
    T g;         // gravity acceleration (globals.rs:7)
};

// The fast policy's FP32 reciprocal and reciprocal square root: the
// hardware approximations without the subnormal range handling (the states
// never reach subnormal densities or pressures), one instruction each.
__device__ __forceinline__ float rcp_approx(float x) {
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}
__device__ __forceinline__ float rsqrt_approx(float x) {
    float r;
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(x));
    return r;
}

template <class T> __device__ __forceinline__ T fast_rcp(T x);
template <> __device__ __forceinline__ float fast_rcp<float>(float x) { return rcp_approx(x); }
template <> __device__ __forceinline__ double fast_rcp<double>(double x) { return 1.0 / x; }

// minmod slope limiter (an addition of this library; the reference uses
// unlimited central slopes): zero when the one-sided slopes differ in sign
// or one is zero, else the one of smaller magnitude.
template <class T> __device__ __forceinline__ T minmod(T a, T b) {
    if (!(a * b > T(0))) return T(0);
    return fabs(a) < fabs(b) ? a : b;
}

template <class T, bool EXACT> struct Phys;

// NaN-propagating maximum (PTX max.NaN): a NaN wave speed anywhere must
// reach the reduction, as it does in the reference (physics.rs:191-195).
__device__ __forceinline__ float max_nan(float a, float b) {
    float r;
    asm("max.NaN.f32 %0, %1, %2;" : "=f"(r) : "f"(a), "f"(b));
    return r;
}

// Fast-policy wave speed c_s + |v| of one primitive state (the quantity
// whose maximum sets dt, physics.rs:186-190): sqrt(gamma p / rho) as
// g*rsqrt(g*rho) with g = gamma p, |v| as v2*rsqrt(v2) (rsqrt_approx).  The fast kernels
// take dt = CFL * ds / max(speed), the same minimum as CFL * min(ds/speed)
// without a divide per cell.  Explicit _rn operations: every kernel that
// calls this rounds the same way.
__device__ __forceinline__ float fast_speed(float rho, float vx, float vy, float vz, float p, float gamma) {
    const float g = __fmul_rn(gamma, p);
    const float cs = __fmul_rn(g, rsqrt_approx(__fmul_rn(g, rho)));
    const float v2 = __fmaf_rn(vz, vz, __fmaf_rn(vy, vy, __fmul_rn(vx, vx)));
    const float vm = __fmul_rn(v2, rsqrt_approx(fmaxf(v2, 1e-30f)));
    return __fadd_rn(cs, vm);
}

// ---------------------------------------------------------------------------
// Reference rounding
// ---------------------------------------------------------------------------
template <class T> struct Phys<T, true> {
    // calc_primitives, physics.rs:112-140
    static __device__ __forceinline__ void prim(const T u[5], T w[5], const Consts<T> &k) {
        const T r = u[0] / k.vol;
        const T vx = u[1] / (r * k.vol);
        const T vy = u[2] / (r * k.vol);
        const T vz = u[3] / (r * k.vol);
        w[0] = r;
        w[1] = vx;
        w[2] = vy;
        w[3] = vz;
        w[4] = (u[4] / k.vol - T(0.5) * r * (vx * vx + vy * vy + vz * vz)) * k.gm1;
    }

    // calc_timestep body, physics.rs:187-189
    static __device__ __forceinline__ T wave_dt(const T w[5], const Consts<T> &k) {
        return k.ds / (sqrt(k.gamma * w[4] / w[0]) + sqrt(w[1] * w[1] + w[2] * w[2] + w[3] * w[3]));
    }

    // calc_gradients, physics.rs:206-208 (LIM 0); minmod of the one-sided
    // differences (LIM 1)
    template <int LIM> static __device__ __forceinline__ T slope(T qm, T q0, T qp, const Consts<T> &k) {
        if (LIM == 0) return (qp - qm) / k.two_ds;
        return minmod((q0 - qm) / k.ds, (qp - q0) / k.ds);
    }

    // extrapolate_primitives_t, physics.rs:251-278; gx/gy/gz are d/dx, d/dy,
    // d/dz of (rho, vx, vy, vz, p)
    static __device__ __forceinline__ void predict(const T w[5], const T gx[5], const T gy[5], const T gz[5], T dt,
                                                   const Consts<T> &k, T out[5]) {
        const T rho = w[0], vx = w[1], vy = w[2], vz = w[3], p = w[4];
        const T h = T(0.5) * dt;
        out[0] = rho - h * (vx * gx[0] + rho * gx[1] + vy * gy[0] + rho * gy[2] + vz * gz[0] + rho * gz[3]);
        out[1] = vx - h * (vx * gx[1] + vy * gy[1] + vz * gz[1] + (T(1.0) / rho) * gx[4]);
        out[2] = vy - h * (vx * gx[2] + vy * gy[2] + vz * gz[2] + (T(1.0) / rho) * gy[4]);
        out[3] = vz - h * (vx * gx[3] + vy * gy[3] + vz * gz[3] + (T(1.0) / rho) * gz[4]);
        out[4] = p - h * (k.gamma * p * (gx[1] + gy[2] + gz[3]) + vx * gx[4] + vy * gy[4] + vz * gz[4]);
    }

    // calc_flux_reconstruction, physics.rs:313-405, for the face between the
    // lower cell (xl, gl = predicted state, slope along the face normal) and
    // the upper cell (xu, gu).  n = 1, 2, 3: index of the normal velocity.
    // The result includes the final *ds (physics.rs:401-405).  klow: z index
    // of the lower cell, for the gravity term (z faces only, grav != 0).
    // heat: the face is the first face of a lower conducting wall; its
    // energy flux takes Q / V after the advective part (kernels.h:561-575).
    static __device__ __forceinline__ void face(const T xl[5], const T gl[5], const T xu[5], const T gu[5], int n,
                                                int grav, int klow, int nz, const Consts<T> &k, T F[5],
                                                bool heat = false) {
        const int t1 = n == 1 ? 2 : 1, t2 = n == 3 ? 2 : 3;
        const T half = k.half_ds;
        const T rl = xu[0] - gu[0] * half;
        const T rr = xl[0] + gl[0] * half;
        const T vxl = xu[n] - gu[n] * half;
        const T vxr = xl[n] + gl[n] * half;
        const T vyl = xu[t1] - gu[t1] * half;
        const T vyr = xl[t1] + gl[t1] * half;
        const T vzl = xu[t2] - gu[t2] * half;
        const T vzr = xl[t2] + gl[t2] * half;
        const T pl = xu[4] - gu[4] * half;
        const T pr = xl[4] + gl[4] * half;
        const T en_left = T(0.5) * (rl * (vxl * vxl + vyl * vyl + vzl * vzl)) + (pl / k.gm1);
        const T en_right = T(0.5) * (rr * (vxr * vxr + vyr * vyr + vzr * vzr)) + (pr / k.gm1);
        const T rho_star = (rl + rr) / T(2.0);
        const T mx = (rl * vxl + rr * vxr) / T(2.0);
        const T my = (rl * vyl + rr * vyr) / T(2.0);
        const T mz = (rl * vzl + rr * vzr) / T(2.0);
        const T en_star = T(0.5) * (en_left + en_right);
        const T p_star = k.gm1 * (en_star - T(0.5) * (mx * mx + my * my + mz * mz) / rho_star);
        T f0 = mx;
        T f1 = (mx * mx / rho_star) + p_star;
        T f2 = mx * my / rho_star;
        T f3 = mx * mz / rho_star;
        T f4 = (en_star + p_star) * (mx / rho_star);
        if (heat) f4 += wall_heat(xl[0], xl[4], k.ds);
        if (grav) {
            const T h = (T(nz) - T(2.0) * T(2)) * k.ds - (T(klow) - T(2.0)) * k.ds;
            f1 += T(1.0) * rho_star * k.g * h;
            f4 += T(0.5) * rho_star * (vxl + vxr) * k.g * h;
        }
        const T c_l = sqrt(k.gamma * pl / rl) + fabs(vxl);
        const T c_r = sqrt(k.gamma * pr / rr) + fabs(vxr);
        const T c_star = fmax(c_l, c_r);
        f0 = mx - T(0.5) * c_star * (rl - rr);
        f1 -= c_star * (rl * vxl - rr * vxr) / T(2.0);
        f2 -= c_star * (rl * vyl - rr * vyr) / T(2.0);
        f3 -= c_star * (rl * vzl - rr * vzr) / T(2.0);
        f4 -= c_star * (en_left - en_right) / T(2.0);
        F[0] = f0 * k.ds;
        F[n] = f1 * k.ds;
        F[t1] = f2 * k.ds;
        F[t2] = f3 * k.ds;
        F[4] = f4 * k.ds;
    }

    // add_fluxes, physics.rs:548-554, same summation order
    static __device__ __forceinline__ T update(T u, T fxh, T fxl, T fyh, T fyl, T fzh, T fzl, T dt,
                                               const Consts<T> &k) {
        return u - dt * k.ds * (fxh - fxl + fyh - fyl + fzh - fzl);
    }
};

// ---------------------------------------------------------------------------
// Fast
// ---------------------------------------------------------------------------
template <class T> struct Phys<T, false> {
    // Same operation sequence as the sweep kernel's conversion of the
    // updated state (dg_sweep_impl.cuh prim), so dt agrees bit for bit
    // between the state reduction and the step's fused reduction.
    static __device__ __forceinline__ void prim(const T u[5], T w[5], const Consts<T> &k) {
        const T ir = fast_rcp(u[0]);   // 1 / (rho V)
        const T rho = u[0] * k.inv_vol;
        const T vx = u[1] * ir, vy = u[2] * ir, vz = u[3] * ir;
        const T v2 = fma(vz, vz, fma(vy, vy, vx * vx));
        w[0] = rho;
        w[1] = vx;
        w[2] = vy;
        w[3] = vz;
        w[4] = fma(T(-0.5) * rho, v2, u[4] * k.inv_vol) * k.gm1;
    }
};

// Primitives -> conserved totals (calc_conserved, physics.rs:146-174);
// reference order.
template <class T>
__host__ __device__ __forceinline__ void prim_to_cons(const T w[5], T u[5], T vol, T gm1) {
    const T rho = w[0], vx = w[1], vy = w[2], vz = w[3], p = w[4];
    u[0] = rho * vol;
    u[1] = vx * rho * vol;
    u[2] = vy * rho * vol;
    u[3] = vz * rho * vol;
    u[4] = vol * (rho * (vx * vx + vy * vy + vz * vz) / T(2.0) + p / gm1);
}

}  // namespace dg
