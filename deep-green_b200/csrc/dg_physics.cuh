// dg_physics.cuh -- per-cell and per-face arithmetic of deep-green's Euler
// step, shared by every kernel of this library.
//
// The formulas are those of the reference's Rust path (deep-green
// src/rs/src/physics.rs); each function cites the lines it follows.  The
// operation order is re-associated where that saves instructions (one
// reciprocal per state instead of several divides; the ds and dt factors of
// the update folded into one scale): results differ from the reference's
// rounding at the level of the unit roundoff of T, which is what the
// tolerances of the parity tests (1e-12 relative for double, 1e-5 for float
// against the double oracle) allow.
#pragma once

#include <cuda_runtime.h>
#include <math.h>

namespace dg {

enum Bc : int { kPeriodic = 0, kOutflow = 1, kWall = 2 };

template <class T> struct Num;

template <> struct Num<float> {
    // Reciprocal to ~1 ulp: MUFU.RCP refined by one Newton step would be
    // exact-ish; the hardware approximation alone is within 2^-22.
    static __device__ __forceinline__ float rcp(float x) { return __fdividef(1.0f, x); }
    static __device__ __forceinline__ float sqrt_(float x) { return sqrtf(x); }
};

template <> struct Num<double> {
    static __device__ __forceinline__ double rcp(double x) { return 1.0 / x; }
    static __device__ __forceinline__ double sqrt_(double x) { return sqrt(x); }
};

// Runtime constants of one grid, derived once on the host.
template <class T> struct Consts {
    T ds;        // cell size
    T inv_vol;   // 1 / ds^3
    T vol;       // ds^3
    T gamma;     // ratio of specific heats
    T gm1;       // gamma - 1
    T inv_gm1;   // 1 / (gamma - 1)
    T half_ds;   // ds / 2 : face reconstruction offset (physics.rs:313-336)
    T inv_ds;    // 1 / ds
    T inv_2ds;   // 1 / (2 ds) : central gradient (physics.rs:206-208)
    T cfl;
    T g;         // gravity acceleration (globals.rs:7)
};

// minmod slope limiter (an addition of this library; the reference uses
// unlimited central slopes).  Zero when the one-sided slopes differ in sign
// or one of them is zero, else the one of smaller magnitude.
template <class T> __device__ __forceinline__ T minmod(T a, T b) {
    const T pick = fabs(a) < fabs(b) ? a : b;
    return (a * b > T(0)) ? pick : T(0);
}

// Slope of q at a cell from its two neighbours along one axis: the
// reference's central difference (physics.rs:206-208) or minmod.
template <class T, int LIM>
__device__ __forceinline__ T slope(T qm, T q0, T qp, const Consts<T> &k) {
    if (LIM == 0) return (qp - qm) * k.inv_2ds;
    return minmod((q0 - qm) * k.inv_ds, (qp - q0) * k.inv_ds);
}

// Conserved totals -> primitives (calc_primitives, physics.rs:109-141).
template <class T>
__device__ __forceinline__ void cons_to_prim(const T u[5], T w[5], const Consts<T> &k) {
    const T rho = u[0] * k.inv_vol;
    const T ir = Num<T>::rcp(u[0]);  // 1 / (rho * V)
    const T vx = u[1] * ir, vy = u[2] * ir, vz = u[3] * ir;
    w[0] = rho;
    w[1] = vx;
    w[2] = vy;
    w[3] = vz;
    w[4] = (u[4] * k.inv_vol - T(0.5) * rho * (vx * vx + vy * vy + vz * vz)) * k.gm1;
}

// Primitives -> conserved totals (calc_conserved, physics.rs:143-175).
template <class T>
__host__ __device__ __forceinline__ void prim_to_cons(const T w[5], T u[5], T vol, T gm1) {
    const T rho = w[0], vx = w[1], vy = w[2], vz = w[3], p = w[4];
    u[0] = rho * vol;
    u[1] = vx * rho * vol;
    u[2] = vy * rho * vol;
    u[3] = vz * rho * vol;
    u[4] = vol * (rho * (vx * vx + vy * vy + vz * vz) / T(2) + p / gm1);
}

// ds / (c_s + |v|) of one cell (the quantity minimised by calc_timestep,
// physics.rs:186-190).  NaN propagates so the caller can flag it.
template <class T>
__device__ __forceinline__ T wave_dt(const T w[5], const Consts<T> &k) {
    const T cs = Num<T>::sqrt_(k.gamma * w[4] * Num<T>::rcp(w[0]));
    const T vm = Num<T>::sqrt_(w[1] * w[1] + w[2] * w[2] + w[3] * w[3]);
    return k.ds * Num<T>::rcp(cs + vm);
}

// Half-step predictor (extrapolate_primitives_t, physics.rs:251-278).
// gx/gy/gz hold d/dx, d/dy, d/dz of (rho, vx, vy, vz, p); hdt = dt / 2.
template <class T>
__device__ __forceinline__ void predict(const T w[5], const T gx[5], const T gy[5], const T gz[5],
                                        T hdt, const Consts<T> &k, T out[5]) {
    const T rho = w[0], vx = w[1], vy = w[2], vz = w[3], p = w[4];
    const T ir = Num<T>::rcp(rho);
    const T div = gx[1] + gy[2] + gz[3];
    out[0] = rho - hdt * (vx * gx[0] + vy * gy[0] + vz * gz[0] + rho * div);
    out[1] = vx - hdt * (vx * gx[1] + vy * gy[1] + vz * gz[1] + ir * gx[4]);
    out[2] = vy - hdt * (vx * gx[2] + vy * gy[2] + vz * gz[2] + ir * gy[4]);
    out[3] = vz - hdt * (vx * gx[3] + vy * gy[3] + vz * gz[3] + ir * gz[4]);
    out[4] = p - hdt * (k.gamma * p * div + vx * gx[4] + vy * gy[4] + vz * gz[4]);
}

// Rusanov / local Lax-Friedrichs flux through one face
// (calc_flux_reconstruction, physics.rs:338-405) WITHOUT the final *ds
// (the caller folds it into the update scale).
//   a: reconstructed primitive state on the lower side of the face
//      (the reference's "r" values: lower cell + slope*ds/2),
//   b: the upper side (the reference's "l" values: upper cell - slope*ds/2),
//   n: index 1..3 of the velocity component normal to the face.
// grav_h: G*h of the gravity term (physics.rs:366-372) or 0.
template <class T>
__device__ __forceinline__ void face_flux(const T a[5], const T b[5], int n, T grav_h,
                                          const Consts<T> &k, T F[5]) {
    const int t1 = n == 1 ? 2 : 1;
    const int t2 = n == 3 ? 2 : 3;
    const T ra = a[0], ua = a[n], va = a[t1], wa = a[t2], pa = a[4];
    const T rb = b[0], ub = b[n], vb = b[t1], wb = b[t2], pb = b[4];
    const T ea = T(0.5) * ra * (ua * ua + va * va + wa * wa) + pa * k.inv_gm1;
    const T eb = T(0.5) * rb * (ub * ub + vb * vb + wb * wb) + pb * k.inv_gm1;
    const T mua = ra * ua, mva = ra * va, mwa = ra * wa;
    const T mub = rb * ub, mvb = rb * vb, mwb = rb * wb;
    const T rs = T(0.5) * (ra + rb);
    const T mu = T(0.5) * (mua + mub), mv = T(0.5) * (mva + mvb), mw = T(0.5) * (mwa + mwb);
    const T es = T(0.5) * (ea + eb);
    const T irs = Num<T>::rcp(rs);
    const T us = mu * irs;
    const T ps = k.gm1 * (es - T(0.5) * (mu * mu + mv * mv + mw * mw) * irs);
    const T ca = Num<T>::sqrt_(k.gamma * pa * Num<T>::rcp(ra)) + fabs(ua);
    const T cb = Num<T>::sqrt_(k.gamma * pb * Num<T>::rcp(rb)) + fabs(ub);
    const T c = fmax(ca, cb);
    const T hc = T(0.5) * c;
    T fr = mu, fu = mu * us + ps, fv = mv * us, fw = mw * us, fe = (es + ps) * us;
    if (grav_h != T(0)) {
        fu += rs * grav_h;
        fe += T(0.5) * rs * (ua + ub) * grav_h;
    }
    // F -= c/2 (U_upper - U_lower)
    F[0] = fr - hc * (rb - ra);
    F[n] = fu - hc * (mub - mua);
    F[t1] = fv - hc * (mvb - mva);
    F[t2] = fw - hc * (mwb - mwa);
    F[4] = fe - hc * (eb - ea);
}

}  // namespace dg
