// dg_learned.cu -- the learned coarse step: coarsening, network inputs and
// training targets, and the corrector (plain step + network correction with
// positivity mask, mean removal, conservation check and fallback).
//
// All kernels here are element-wise passes over FP32 SoA states; the
// network's convolutions are the tensor-core kernels of dg_conv.cuh.
#include <cuda_bf16.h>

#include <algorithm>
#include <cmath>
#include <string>

#include "../../include/deepgreen_net.h"
#include "dg_common.cuh"
#include "dg_ctx.h"
#include "dg_net_impl.h"

using namespace dg;

namespace {

constexpr int kLearnBlocks = kSms * 4;
constexpr int kLearnThreads = 256;

// A conserved FP32 state: 5 fields of ghosted rows, interior cube of n.
struct View {
    const float *p;
    int pitch;            // elements per z-row
    int nyg;              // rows per x-plane (ghosted y extent)
    long long fstride;    // elements per field
    int n;                // interior cells per axis
};

struct NormDev {
    float in_mean[16], in_inv_std[16], out_std[16];
};

__device__ __forceinline__ int wrapi(int i, int n) {
    i %= n;
    return i < 0 ? i + n : i;
}

// element offset of interior cell (x, y, z), coordinates already in 0..n-1
__device__ __forceinline__ long long vidx(const View &v, int x, int y, int z) {
    return ((long long)(x + 2) * v.nyg + (y + 2)) * v.pitch + (z + 2);
}

View dense_view(const float *p, int n) {
    View v;
    v.p = p;
    v.pitch = n + 4;
    v.nyg = n + 4;
    v.fstride = (long long)(n + 4) * (n + 4) * (n + 4);
    v.n = n;
    return v;
}

View ctx_view(const dg_ctx *c, const void *buf) {
    View v;
    v.p = static_cast<const float *>(buf);
    v.pitch = c->pitch;
    v.nyg = c->ny;
    v.fstride = c->fstride;
    v.n = c->info.nx;
    return v;
}

// raw input channels 0..13 of one cell (densities before b, after a)
__device__ __forceinline__ void raw_features(const View &b, const View &a, long long i, float inv_vol, float gm1,
                                             float f[16]) {
    float u1[5], u0[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        u1[c] = a.p[i + c * a.fstride] * inv_vol;
        u0[c] = b.p[i + c * b.fstride] * inv_vol;
    }
#pragma unroll
    for (int c = 0; c < 5; ++c) {
        f[c] = u1[c];
        f[5 + c] = u1[c] - u0[c];
    }
    const float ir = 1.0f / u1[0];
    f[10] = u1[1] * ir;
    f[11] = u1[2] * ir;
    f[12] = u1[3] * ir;
    f[13] = gm1 * (u1[4] - 0.5f * (u1[1] * u1[1] + u1[2] * u1[2] + u1[3] * u1[3]) * ir);
    f[14] = 0.0f;
    f[15] = 0.0f;
}

__global__ void features_kernel(View b, View a, NormDev nm, float inv_vol, float gm1, int ox, int oy, int oz, int ext,
                                __nv_bfloat16 *__restrict__ out) {
    const long long total = (long long)ext * ext * ext;
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < (unsigned)total; v += gridDim.x * blockDim.x) {
        const unsigned row = v / (unsigned)ext;
        const int cz = (int)(v - row * (unsigned)ext), cy = (int)(row % (unsigned)ext), cx = (int)(row / (unsigned)ext);
        const int x = wrapi(ox + cx, a.n), y = wrapi(oy + cy, a.n), z = wrapi(oz + cz, a.n);
        float f[16];
        raw_features(b, a, vidx(a, x, y, z), inv_vol, gm1, f);
        uint4 w[2];
        uint32_t *u = reinterpret_cast<uint32_t *>(w);
#pragma unroll
        for (int c = 0; c < 16; c += 2) {
            __nv_bfloat162 h = __floats2bfloat162_rn((f[c] - nm.in_mean[c]) * nm.in_inv_std[c],
                                                     (f[c + 1] - nm.in_mean[c + 1]) * nm.in_inv_std[c + 1]);
            u[c >> 1] = *reinterpret_cast<uint32_t *>(&h);
        }
        uint4 *dst = reinterpret_cast<uint4 *>(out + (size_t)v * 16);
        dst[0] = w[0];
        dst[1] = w[1];
    }
}

__global__ void targets_kernel(View a, View t, NormDev nm, float inv_vol, int ox, int oy, int oz, int ext,
                               float *__restrict__ out) {
    const long long total = (long long)ext * ext * ext;
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < (unsigned)total; v += gridDim.x * blockDim.x) {
        const unsigned row = v / (unsigned)ext;
        const int cz = (int)(v - row * (unsigned)ext), cy = (int)(row % (unsigned)ext), cx = (int)(row / (unsigned)ext);
        const int x = wrapi(ox + cx, a.n), y = wrapi(oy + cy, a.n), z = wrapi(oz + cz, a.n);
        const long long ia = vidx(a, x, y, z), it = vidx(t, x, y, z);
        float4 *dst = reinterpret_cast<float4 *>(out + (size_t)v * 16);
        float o[8];
#pragma unroll
        for (int c = 0; c < 5; ++c)
            o[c] = (t.p[it + c * t.fstride] - a.p[ia + c * a.fstride]) * inv_vol / nm.out_std[c];
        o[5] = o[6] = o[7] = 0.0f;
        dst[0] = make_float4(o[0], o[1], o[2], o[3]);
        dst[1] = make_float4(o[4], o[5], o[6], o[7]);
        dst[2] = make_float4(0.f, 0.f, 0.f, 0.f);
        dst[3] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
}

// coarse interior cell = sum of its 8 fine cells, per field
__global__ void coarsen_kernel(View f, float *__restrict__ dst, int pitch, int nyg, long long fstride, int n) {
    const long long total = (long long)n * n * n;
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < (unsigned)total; v += gridDim.x * blockDim.x) {
        const unsigned row = v / (unsigned)n;
        const int z = (int)(v - row * (unsigned)n), y = (int)(row % (unsigned)n), x = (int)(row / (unsigned)n);
        const long long o = ((long long)(x + 2) * nyg + (y + 2)) * pitch + (z + 2);
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            float s = 0.0f;
#pragma unroll
            for (int a = 0; a < 2; ++a)
#pragma unroll
                for (int b = 0; b < 2; ++b) {
                    const long long i = vidx(f, 2 * x + a, 2 * y + b, 2 * z) + c * f.fstride;
                    s += f.p[i] + f.p[i + 1];
                }
            dst[o + c * fstride] = s;
        }
    }
}

// ---------------------------------------------------------------------------
// Corrector kernels
// ---------------------------------------------------------------------------
struct CorrCtl {
    unsigned counter;                 // last-block ticket of the running launch
    unsigned fallback;                // the current step keeps the plain state
    unsigned long long masked;        // masked cells of the current step
    double mean[5];                   // mean correction over unmasked cells (totals)
    // totals since creation
    unsigned long long steps, fallbacks, masked_total, violations;
    double max_drift;
    double last_drift;                // of the latest step, kept or not
    double last_field_drift[5];
};

constexpr int kCorrVals = 6;   // per-block partials of the correction pass

__device__ __forceinline__ bool positive(const float u[5], float gm1, float inv_vol) {
    const float r = u[0] * inv_vol;
    const float e = u[4] * inv_vol;
    const float m2 = (u[1] * u[1] + u[2] * u[2] + u[3] * u[3]) * inv_vol * inv_vol;
    const float p = gm1 * (e - 0.5f * m2 / r);
    return r > 0.0f && p > 0.0f && isfinite(r) && isfinite(p);
}

// Sum K doubles over the block into part[blockIdx.x][K]; true in every thread
// of the last block to finish.
template <int K>
__device__ bool block_sum(double v[K], double *part, unsigned *counter) {
    __shared__ double red[kLearnThreads / 32][K];
    __shared__ int last;
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) v[k] += __shfl_xor_sync(0xffffffffu, v[k], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) red[warp][k] = v[k];
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int k = 0; k < K; ++k) {
            double s = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) s += red[w][k];
            part[(size_t)blockIdx.x * K + k] = s;
        }
        __threadfence();
        last = atomicAdd(counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    return last != 0;
}

// In every thread of the last block: the fixed-order sum of all blocks'
// partials (the first K of each block's KP values), thread t taking blocks
// t, t + blockDim.x, ..., then a shuffle tree and the warps in order; the
// result is valid in thread 0.
template <int K, int KP>
__device__ void final_sum_strided(const double *part, double s[K]) {
    __shared__ double red[kLearnThreads / 32][K];
#pragma unroll
    for (int k = 0; k < K; ++k) s[k] = 0.0;
    const volatile double *vp = part;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x)
#pragma unroll
        for (int k = 0; k < K; ++k) s[k] += vp[(size_t)b * KP + k];
#pragma unroll
    for (int k = 0; k < K; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s[k] += __shfl_xor_sync(0xffffffffu, s[k], o);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0)
#pragma unroll
        for (int k = 0; k < K; ++k) red[warp][k] = s[k];
    __syncthreads();
    if (threadIdx.x == 0)
        for (int k = 0; k < K; ++k) {
            double t = 0.0;
            for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += red[w][k];
            s[k] = t;
        }
}

// pass 1: raw correction (totals) = divergence of the network's face fluxes,
// positivity mask, sums for the mean
__global__ void __launch_bounds__(kLearnThreads) correct_kernel(View u1, const float *__restrict__ out, NormDev nm,
                                                                float vol, float inv_vol, float gm1,
                                                                float *__restrict__ delta, uint8_t *__restrict__ mask,
                                                                double *part, CorrCtl *ctl) {
    const int n = u1.n;
    const long long total = (long long)n * n * n;
    double acc[kCorrVals] = {0, 0, 0, 0, 0, 0};
    for (unsigned v = blockIdx.x * blockDim.x + threadIdx.x; v < (unsigned)total; v += gridDim.x * blockDim.x) {
        const unsigned row = v / (unsigned)n;
        const int z = (int)(v - row * (unsigned)n), y = (int)(row % (unsigned)n), x = (int)(row / (unsigned)n);
        const long long i = vidx(u1, x, y, z);
        // divergence of the face fluxes (channel 5 d + c), periodic; rows of
        // 16 floats read as float4 / float2 pieces
        const unsigned nn = (unsigned)n * n;
        const unsigned lx = (unsigned)(x == 0 ? n - 1 : x - 1) * nn + (unsigned)y * n + z;
        const unsigned ly = (unsigned)x * nn + (unsigned)(y == 0 ? n - 1 : y - 1) * n + z;
        const unsigned lz = (unsigned)x * nn + (unsigned)y * n + (z == 0 ? n - 1 : z - 1);
        const float4 *own = reinterpret_cast<const float4 *>(out) + (size_t)v * 4;
        const float4 f0 = own[0], f1 = own[1], f2 = own[2], f3 = own[3];
        const float hi[15] = {f0.x, f0.y, f0.z, f0.w, f1.x, f1.y, f1.z, f1.w,
                              f2.x, f2.y, f2.z, f2.w, f3.x, f3.y, f3.z};
        const float4 ax = reinterpret_cast<const float4 *>(out)[(size_t)lx * 4];
        const float ax4 = out[(size_t)lx * 16 + 4];
        const float4 ay = reinterpret_cast<const float4 *>(out)[(size_t)ly * 4 + 1];
        const float2 ay8 = reinterpret_cast<const float2 *>(out)[(size_t)ly * 8 + 4];
        const float2 az10 = reinterpret_cast<const float2 *>(out)[(size_t)lz * 8 + 5];
        const float4 az12 = reinterpret_cast<const float4 *>(out)[(size_t)lz * 4 + 3];
        const float lo_x[5] = {ax.x, ax.y, ax.z, ax.w, ax4};
        const float lo_y[5] = {ay.y, ay.z, ay.w, ay8.x, ay8.y};
        const float lo_z[5] = {az10.x, az10.y, az12.x, az12.y, az12.z};
        float o[5];
#pragma unroll
        for (int c = 0; c < 5; ++c)
            o[c] = ((hi[c] - lo_x[c]) + (hi[5 + c] - lo_y[c])) + (hi[10 + c] - lo_z[c]);
        float d[5], u[5];
        bool ok = true;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            d[c] = o[c] * nm.out_std[c] * vol;
            u[c] = u1.p[i + c * u1.fstride] + d[c];
            ok &= isfinite(d[c]);
        }
        ok = ok && positive(u, gm1, inv_vol);
        mask[v] = ok ? 0 : 1;
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            const float dc = ok ? d[c] : 0.0f;
            delta[c * total + v] = dc;
            acc[c] += dc;
        }
        acc[5] += ok ? 0.0 : 1.0;
    }
    if (!block_sum<kCorrVals>(acc, part, &ctl->counter)) return;
    double s[kCorrVals];
    final_sum_strided<kCorrVals, kCorrVals>(part, s);
    if (threadIdx.x == 0) {
        const double kept = (double)total - s[5];
        for (int c = 0; c < 5; ++c) ctl->mean[c] = kept > 0 ? s[c] / kept : 0.0;
        ctl->masked = (unsigned long long)s[5];
        ctl->counter = 0;
        __threadfence();
    }
}

// 64 random bits per (step, cell): SplitMix64 finaliser of a counter
// (Steele, Lea & Flood 2014); field c takes bits 12c .. 12c+11 as its dither,
// uniform on 4096 centred levels in (-1/2, 1/2).
__device__ __forceinline__ unsigned long long cell_bits(unsigned long long step, unsigned long long cell) {
    unsigned long long z = step * 0x9E3779B97F4A7C15ull + cell;
    z += 0x9E3779B97F4A7C15ull;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// (k + 1/2) / 4096 - 1/2 for the 12-bit k of the field, built without an
// integer conversion: 1 + k/4096 is the double with exponent 0 and k in the
// top mantissa bits, and subtracting 3/2 - 1/8192 is exact.
__device__ __forceinline__ double dither(unsigned long long bits, int field) {
    const unsigned k = (unsigned)(bits >> (12 * field)) & 4095u;
    return __hiloint2double((int)(0x3FF00000u | (k << 8)), 0) - (1.5 - 0.5 / 4096.0);
}

// x rounded to FP32 with a dither of one unit in the last place (stochastic
// rounding: the expected result is x).  Round-to-nearest would be biased
// here: the network's FP32 output puts the correction on a grid only a few
// bits finer than the state's, and the mean removal shifts that grid by a
// constant, so nearest rounding errs the same way in most cells and moves
// the totals by ~1e-9 of their L1 norm; dithered, the errors cancel to
// ~1e-7 / sqrt(cells).
__device__ __forceinline__ float round_dithered(double x, double h) {
    const float r = (float)x;
    const float a = fabsf(r);
    if (!isfinite(a)) return r;
    // the spacing above a: exact in FP32 (adjacent values)
    const float ulp = __uint_as_float(__float_as_uint(a) + 1u) - a;
    return (float)(x + h * (double)ulp);
}

constexpr int kApplyVals = 11;  // per-block partials of the apply pass (+ the wave-speed maximum)

// Ghosted coordinate of the periodic image of interior coordinate c
// (0..n-1), or -1: cells 0, 1 reappear as ghosts n+2, n+3 and cells n-2,
// n-1 as ghosts 0, 1 (the copies fill_ghosts makes on a periodic axis).
__device__ __forceinline__ int periodic_image(int c, int n) {
    return c < 2 ? c + 2 + n : (c >= n - 2 ? c + 2 - n : -1);
}

// Stores of one corrected z-quad (4 cells, z0 % 4 == 0) of field c at
// interior row (x, y), with the periodic ghost images of cells next to a face.
__device__ __forceinline__ void store_quad(float *dst, const View &v, int x, int y, int z0, int c, float q0,
                                           float q1, float q2, float q3) {
    const int n = v.n;
    float *f = dst + c * v.fstride;
    const int xi = periodic_image(x, n), yi = periodic_image(y, n);
    const bool zlo = z0 == 0, zhi = z0 == n - 4;
    if (xi < 0 && yi < 0 && !zlo && !zhi) {
        float *row = f + ((long long)(x + 2) * v.nyg + (y + 2)) * v.pitch;
        *reinterpret_cast<float2 *>(row + z0 + 2) = make_float2(q0, q1);
        *reinterpret_cast<float2 *>(row + z0 + 4) = make_float2(q2, q3);
        return;
    }
    for (int a = 0; a < 2; ++a) {
        const int gx = a ? xi : x + 2;
        if (gx < 0) continue;
        for (int b = 0; b < 2; ++b) {
            const int gy = b ? yi : y + 2;
            if (gy < 0) continue;
            float *row = f + ((long long)gx * v.nyg + gy) * v.pitch;
            *reinterpret_cast<float2 *>(row + z0 + 2) = make_float2(q0, q1);
            *reinterpret_cast<float2 *>(row + z0 + 4) = make_float2(q2, q3);
            if (zlo) {
                row[n + 2] = q0;
                row[n + 3] = q1;
            }
            if (zhi) {
                row[0] = q2;
                row[1] = q3;
            }
        }
    }
}

// pass 2: the corrected state into dst (interior and periodic ghosts),
// conservation and positivity check, and the corrected state's dt (the
// fast policy's CFL * ds / max(c_s + |v|), as the plain step's own
// reduction computes it).  One thread per z-quad; n % 4 == 0.
__global__ void __launch_bounds__(kLearnThreads) apply_kernel(View u1, float *__restrict__ dst,
                                                              const float *__restrict__ delta,
                                                              const uint8_t *__restrict__ mask, GridArgs<float> g,
                                                              double tol, double *part, CorrCtl *ctl) {
    const int n = u1.n;
    const unsigned nq = (unsigned)n / 4, total = (unsigned)n * n * n, quads = total / 4;
    double mean[5];
#pragma unroll
    for (int c = 0; c < 5; ++c) mean[c] = ctl->mean[c];
    const unsigned long long step = ctl->steps;
    // acc: 0-4 sum of u - old, 5-9 sum |old|, 10 positivity violations
    double acc[kApplyVals];
#pragma unroll
    for (int k = 0; k < kApplyVals; ++k) acc[k] = 0.0;
    float smax = 0.0f;
    for (unsigned qd = blockIdx.x * blockDim.x + threadIdx.x; qd < quads; qd += gridDim.x * blockDim.x) {
        const unsigned row = qd / nq;
        const int z0 = (int)(qd - row * nq) * 4, y = (int)(row % (unsigned)n), x = (int)(row / (unsigned)n);
        const unsigned v = row * (unsigned)n + (unsigned)z0;
        const long long i = vidx(u1, x, y, z0);
        const uchar4 mk = *reinterpret_cast<const uchar4 *>(mask + v);
        const bool keep[4] = {mk.x != 0, mk.y != 0, mk.z != 0, mk.w != 0};
        float old[5][4], d[5][4], u[5][4];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            const float2 a0 = *reinterpret_cast<const float2 *>(u1.p + i + c * u1.fstride);
            const float2 a1 = *reinterpret_cast<const float2 *>(u1.p + i + c * u1.fstride + 2);
            const float4 dd = *reinterpret_cast<const float4 *>(delta + (size_t)c * total + v);
            old[c][0] = a0.x; old[c][1] = a0.y; old[c][2] = a1.x; old[c][3] = a1.y;
            d[c][0] = dd.x; d[c][1] = dd.y; d[c][2] = dd.z; d[c][3] = dd.w;
        }
#pragma unroll
        for (int j = 0; j < 4; ++j) {
            const unsigned long long bits = cell_bits(step, v + j);
            float w[5], cu[5];
#pragma unroll
            for (int c = 0; c < 5; ++c) {
                const double o = (double)old[c][j];
                u[c][j] = keep[j] ? old[c][j] : round_dithered(o + ((double)d[c][j] - mean[c]), dither(bits, c));
                cu[c] = u[c][j];
                acc[c] += (double)u[c][j] - o;
                acc[5 + c] += fabs(o);
            }
            acc[10] += (keep[j] || positive(cu, g.k.gm1, g.k.inv_vol)) ? 0.0 : 1.0;
            Phys<float, false>::prim(cu, w, g.k);
            smax = max_nan(smax, fast_speed(w[0], w[1], w[2], w[3], w[4], g.k.gamma));
        }
#pragma unroll
        for (int c = 0; c < 5; ++c) store_quad(dst, u1, x, y, z0, c, u[c][0], u[c][1], u[c][2], u[c][3]);
    }
    // block partials: the sums, then the wave-speed maximum (NaN-propagating)
    __shared__ double red[kLearnThreads / 32][kApplyVals + 1];
    __shared__ int last;
#pragma unroll
    for (int k = 0; k < kApplyVals; ++k)
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) smax = max_nan(smax, __shfl_xor_sync(0xffffffffu, smax, o));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (lane == 0) {
#pragma unroll
        for (int k = 0; k < kApplyVals; ++k) red[warp][k] = acc[k];
        red[warp][kApplyVals] = (double)smax;
    }
    __syncthreads();
    constexpr int KP = kApplyVals + 1;
    if (threadIdx.x == 0) {
        for (int k = 0; k < KP; ++k) {
            double t = k < kApplyVals ? 0.0 : red[0][k];
            for (int w = k < kApplyVals ? 0 : 1; w < (int)(blockDim.x >> 5); ++w)
                t = k < kApplyVals ? t + red[w][k] : (double)max_nan((float)t, (float)red[w][k]);
            part[(size_t)blockIdx.x * KP + k] = t;
        }
        __threadfence();
        last = atomicAdd(&ctl->counter, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    double s[kApplyVals];
    final_sum_strided<kApplyVals, KP>(part, s);
    __shared__ float smw[kLearnThreads / 32];
    const volatile double *vp = part;
    float sm = 0.0f;
    for (unsigned b = threadIdx.x; b < gridDim.x; b += blockDim.x) sm = max_nan(sm, (float)vp[(size_t)b * KP + kApplyVals]);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) sm = max_nan(sm, __shfl_xor_sync(0xffffffffu, sm, o));
    if (lane == 0) smw[warp] = sm;
    __syncthreads();
    if (threadIdx.x != 0) return;
    for (int w = 1; w < (int)(blockDim.x >> 5); ++w) sm = max_nan(sm, smw[w]);
    double drift = 0.0;
    for (int c = 0; c < 5; ++c) {
        const double dr = s[5 + c] > 0 ? fabs(s[c]) / s[5 + c] : fabs(s[c]);
        ctl->last_field_drift[c] = dr;
        drift = fmax(drift, dr);
    }
    ctl->last_drift = drift;
    ctl->violations += (unsigned long long)s[10];
    const bool fb = s[10] > 0.0 || !(drift <= tol);
    ctl->fallback = fb ? 1u : 0u;
    ctl->steps += 1;
    if (fb) {
        ctl->fallbacks += 1;     // the plain step's dt stays
    } else {
        ctl->masked_total += ctl->masked;
        ctl->max_drift = fmax(ctl->max_drift, drift);
        // dt of the coming step from the kept state (kSetDt of the state reduction)
        DevCtl *dc = g.ctl;
        const bool nn = sm != sm;
        const float w = __fdiv_rn(g.k.ds, sm);
        dc->dt[dc->step & 1] = (double)(nn ? g.k.cfl * 1.0f : g.k.cfl * w);
        if (nn) dc->flags |= kStatusNonFinite;
    }
    ctl->counter = 0;
    __threadfence();
}

// pass 3 (only when the step falls back): dst := the plain state, ghosts included
__global__ void fallback_kernel(const float *__restrict__ src, float *__restrict__ dst, long long count,
                                const CorrCtl *ctl) {
    if (ctl->fallback == 0) return;
    for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < count;
         e += (long long)gridDim.x * blockDim.x)
        dst[e] = src[e];
}

NormDev to_dev(const dg_learned_norm *n) {
    NormDev d;
    for (int c = 0; c < 16; ++c) {
        d.in_mean[c] = n->in_mean[c];
        d.in_inv_std[c] = c < DG_LEARNED_INPUTS ? n->in_inv_std[c] : 0.0f;
        d.out_std[c] = n->out_std[c];
    }
    return d;
}

thread_local std::string g_learn_err;   // the calling thread's last failure

int lfail(int code, const std::string &m) {
    g_learn_err = m;
    set_global_error(m);
    return code;
}

bool periodic_cube(const dg_ctx *c) {
    for (int i = 0; i < 6; ++i)
        if (c->info.bcs[i] != DG_BC_PERIODIC) return false;
    return c->info.nx == c->info.ny && c->info.ny == c->info.nz;
}

}  // namespace

struct dg_corrector {
    dg_ctx *ctx = nullptr;            // not owned; must outlive the corrector's steps
    int device = 0;
    dg_net *net = nullptr;
    NormDev norm;
    int n = 0;
    double tol = 1e-10;
    __nv_bfloat16 *feat = nullptr;
    float *out = nullptr;
    float *delta = nullptr;
    uint8_t *mask = nullptr;
    double *part = nullptr;
    CorrCtl *ctl = nullptr;
    std::string err;
};

extern "C" {

int32_t dg_coarsen(dg_ctx *fine, dg_ctx *coarse) {
    if (!fine || !coarse) return lfail(DG_ERR_INVALID, "null argument");
    if (fine->elem != 4 || coarse->elem != 4) return fail(coarse, DG_ERR_INVALID, "FP32 grids only");
    if (!fine->has_state) return fail(coarse, DG_ERR_NO_STATE, "the fine grid has no state");
    if (fine->info.nx != 2 * coarse->info.nx || fine->info.ny != 2 * coarse->info.ny ||
        fine->info.nz != 2 * coarse->info.nz || coarse->info.nx != coarse->info.ny ||
        coarse->info.ny != coarse->info.nz)
        return fail(coarse, DG_ERR_INVALID, "fine interior must be twice the (cubic) coarse interior");
    if (fine->info.device != coarse->info.device) return fail(coarse, DG_ERR_INVALID, "grids on different devices");
    int r;
    if ((r = ctx_begin_state(coarse)) != DG_OK) return r;
    // the coarse stream must see the fine grid's completed steps
    DG_CUDA(coarse, cudaStreamSynchronize(fine->stream));
    View f = ctx_view(fine, fine->buf[fine->cur]);
    coarsen_kernel<<<kLearnBlocks, kLearnThreads, 0, coarse->stream>>>(
        f, static_cast<float *>(coarse->buf[coarse->cur]), coarse->pitch, coarse->ny, coarse->fstride, coarse->info.nx);
    DG_CUDA(coarse, cudaGetLastError());
    if ((r = ctx_finish_state(coarse)) != DG_OK) return r;
    return ctx_check_flags(coarse);
}

int32_t dg_learned_features(const dg_learned_norm *norm, const float *before, const float *after, int32_t n, double ds,
                            double gamma, int32_t ox, int32_t oy, int32_t oz, int32_t ext, void *feat, void *stream) {
    if (!norm || !before || !after || !feat) return lfail(DG_ERR_INVALID, "null argument");
    if (n < 1 || ext < 1 || !(ds > 0) || !(gamma > 1)) return lfail(DG_ERR_INVALID, "bad extents or constants");
    if (ext > 1600 || n > 1600) return lfail(DG_ERR_INVALID, "extents above 1600 cells per axis");
    if (reinterpret_cast<uintptr_t>(feat) & 15) return lfail(DG_ERR_INVALID, "feat must be 16-byte aligned");
    const float vol = (float)(ds * ds * ds);
    features_kernel<<<kLearnBlocks, kLearnThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        dense_view(before, n), dense_view(after, n), to_dev(norm), 1.0f / vol, (float)(gamma - 1.0), ox, oy, oz, ext,
        static_cast<__nv_bfloat16 *>(feat));
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DG_OK : lfail(DG_ERR_CUDA, std::string("features: ") + cudaGetErrorString(e));
}

int32_t dg_learned_targets(const dg_learned_norm *norm, const float *after, const float *truth, int32_t n, double ds,
                           int32_t ox, int32_t oy, int32_t oz, int32_t ext, float *out, void *stream) {
    if (!norm || !after || !truth || !out) return lfail(DG_ERR_INVALID, "null argument");
    if (n < 1 || ext < 1 || !(ds > 0)) return lfail(DG_ERR_INVALID, "bad extents or constants");
    if (ext > 1600 || n > 1600) return lfail(DG_ERR_INVALID, "extents above 1600 cells per axis");
    if (reinterpret_cast<uintptr_t>(out) & 15) return lfail(DG_ERR_INVALID, "out must be 16-byte aligned");
    for (int c = 0; c < DG_LEARNED_OUTPUTS; ++c)
        if (!(norm->out_std[c] > 0)) return lfail(DG_ERR_INVALID, "out_std must be positive");
    const float vol = (float)(ds * ds * ds);
    targets_kernel<<<kLearnBlocks, kLearnThreads, 0, static_cast<cudaStream_t>(stream)>>>(
        dense_view(after, n), dense_view(truth, n), to_dev(norm), 1.0f / vol, ox, oy, oz, ext, out);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DG_OK : lfail(DG_ERR_CUDA, std::string("targets: ") + cudaGetErrorString(e));
}

int32_t dg_corrector_create(dg_ctx *coarse, dg_net *net, const dg_learned_norm *norm, dg_corrector **out) {
    if (!coarse || !net || !norm || !out) return lfail(DG_ERR_INVALID, "null argument");
    *out = nullptr;
    if (coarse->elem != 4 || coarse->exact) return lfail(DG_ERR_INVALID, "the corrector needs the FP32 fast step");
    if (!periodic_cube(coarse)) return lfail(DG_ERR_INVALID, "the corrector needs a cubic, periodic grid");
    if (coarse->info.nx > 1024) return lfail(DG_ERR_INVALID, "the corrector takes grids of at most 1024^3 cells");
    if (coarse->info.nx % 4 != 0) return lfail(DG_ERR_INVALID, "the corrector needs n divisible by 4");
    if (net_inputs(net) != DG_LEARNED_INPUTS || net_outputs(net) != DG_LEARNED_OUTPUTS)
        return lfail(DG_ERR_INVALID, "the network must have 14 inputs and 15 (flux) outputs");
    if (net_device(net) != coarse->info.device) return lfail(DG_ERR_INVALID, "network and grid on different devices");
    for (int c = 0; c < DG_LEARNED_OUTPUTS; ++c)
        if (!(norm->out_std[c] > 0)) return lfail(DG_ERR_INVALID, "out_std must be positive");
    if (cudaSetDevice(coarse->info.device) != cudaSuccess) return lfail(DG_ERR_NO_DEVICE, "cannot select device");
    dg_corrector *k = new dg_corrector();
    k->ctx = coarse;
    k->device = coarse->info.device;
    k->net = net;
    k->norm = to_dev(norm);
    k->n = coarse->info.nx;
    const long long n = k->n, nf = n + 8, cells = n * n * n;
    cudaError_t e = cudaMalloc(&k->feat, (size_t)nf * nf * nf * 16 * 2);
    if (e == cudaSuccess) e = cudaMalloc(&k->out, (size_t)cells * 16 * 4);
    if (e == cudaSuccess) e = cudaMalloc(&k->delta, (size_t)cells * 5 * 4);
    if (e == cudaSuccess) e = cudaMalloc(&k->mask, (size_t)cells);
    if (e == cudaSuccess) e = cudaMalloc(&k->part, (size_t)kLearnBlocks * (kApplyVals + 1) * sizeof(double));
    if (e == cudaSuccess) e = cudaMalloc(&k->ctl, sizeof(CorrCtl));
    if (e == cudaSuccess) e = cudaMemset(k->ctl, 0, sizeof(CorrCtl));
    if (e != cudaSuccess) {
        dg_corrector_destroy(k);
        return lfail(DG_ERR_CUDA, std::string("corrector allocation: ") + cudaGetErrorString(e));
    }
    *out = k;
    return DG_OK;
}

int32_t dg_corrector_destroy(dg_corrector *k) {
    if (!k) return DG_OK;
    // the context may already be gone: touch only the corrector's own state
    cudaSetDevice(k->device);
    cudaDeviceSynchronize();
    cudaFree(k->feat);
    cudaFree(k->out);
    cudaFree(k->delta);
    cudaFree(k->mask);
    cudaFree(k->part);
    cudaFree(k->ctl);
    delete k;
    return DG_OK;
}

int32_t dg_corrector_set_tolerance(dg_corrector *k, double tol) {
    if (!k || !(tol >= 0)) return lfail(DG_ERR_INVALID, "bad argument");
    k->tol = tol;
    return DG_OK;
}

int32_t dg_corrector_step(dg_corrector *k, int32_t nsteps) {
    if (!k || nsteps < 0) return lfail(DG_ERR_INVALID, "bad argument");
    dg_ctx *c = k->ctx;
    if (!c->has_state) return fail(c, DG_ERR_NO_STATE, "no state set");
    DG_CUDA(c, cudaSetDevice(c->info.device));
    const float vol = (float)(c->info.ds * c->info.ds * c->info.ds);
    const float gm1 = (float)(c->info.gamma - 1.0);
    for (int s = 0; s < nsteps; ++s) {
        int r;
        if ((r = ctx_enqueue(c, 1)) != DG_OK) return r;
        const int cur = c->cur, other = 1 - cur;
        View u1 = ctx_view(c, c->buf[cur]);
        View u0 = ctx_view(c, c->buf[other]);
        features_kernel<<<kLearnBlocks, kLearnThreads, 0, c->stream>>>(u0, u1, k->norm, 1.0f / vol, gm1, -4, -4, -4,
                                                                        k->n + 8, k->feat);
        DG_CUDA(c, cudaGetLastError());
        if ((r = net_forward_stream(k->net, k->feat, 1, k->n + 8, k->n + 8, k->n + 8, k->out, c->stream)) != DG_OK)
            return fail(c, r, std::string("network: ") + net_error(k->net));
        correct_kernel<<<kLearnBlocks, kLearnThreads, 0, c->stream>>>(u1, k->out, k->norm, vol, 1.0f / vol, gm1,
                                                                       k->delta, k->mask, k->part, k->ctl);
        float *dst = static_cast<float *>(c->buf[other]);
        apply_kernel<<<kLearnBlocks, kLearnThreads, 0, c->stream>>>(u1, dst, k->delta, k->mask,
                                                                     grid_args<float>(c, dst, dst), k->tol, k->part,
                                                                     k->ctl);
        fallback_kernel<<<kLearnBlocks, kLearnThreads, 0, c->stream>>>(static_cast<const float *>(c->buf[cur]), dst,
                                                                        5 * c->fstride, k->ctl);
        DG_CUDA(c, cudaGetLastError());
        c->cur = other;
    }
    return DG_OK;
}

int32_t dg_corrector_stats(dg_corrector *k, dg_learned_stats *out) {
    if (!k || !out) return lfail(DG_ERR_INVALID, "null argument");
    dg_ctx *c = k->ctx;
    DG_CUDA(c, cudaSetDevice(c->info.device));
    CorrCtl h;
    DG_CUDA(c, cudaMemcpyAsync(&h, k->ctl, sizeof(h), cudaMemcpyDeviceToHost, c->stream));
    DG_CUDA(c, cudaStreamSynchronize(c->stream));
    unsigned st = 0;
    DG_CUDA(c, cudaMemcpy(&st, net_status(k->net), sizeof(st), cudaMemcpyDeviceToHost));
    if (st) return fail(c, DG_ERR_TIMEOUT, "a network kernel's wait timed out; results invalid");
    out->steps = h.steps;
    out->fallback_steps = h.fallbacks;
    out->masked_cells = h.masked_total;
    out->cells = h.steps * (unsigned long long)k->n * k->n * k->n;
    out->max_drift = h.max_drift;
    out->last_drift = h.last_drift;
    out->violations = h.violations;
    return ctx_check_flags(c);
}

const char *dg_corrector_last_error(const dg_corrector *k) {
    if (k && k->ctx) return k->ctx->err.c_str();
    return g_learn_err.c_str();
}

}  // extern "C"
