// dg_conv.cuh -- BF16 3x3x3 convolution kernels of the correction network on
// the 5th-generation tensor cores (tcgen05, FP32 accumulation in TMEM).
//
// Activations are channels-last, [n][x][y][z][C] BF16, z fastest.  Every
// convolution is "valid": an input of extents (X, Y, Z) gives an output of
// (X-2, Y-2, Z-2), out[v] = sum_t W_t in[v + t], t = (dx, dy, dz) in 0..2,
// weights W[co][ci][dx][dy][dz] (the layout of torch.nn.Conv3d on tensors
// ordered (n, C, x, y, z)).
//
// Forward / input-gradient kernel (implicit GEMM, D[M=128 positions,
// N=COUT] = sum over 27 taps x CIN channels):
//   * positions are enumerated along the flattened (y, z) index of the INPUT,
//     p = y * Zin + z, within one (n, x) plane; tap (dx, dy, dz) is then the
//     plane x+dx shifted by dy*Zin + dz, so one tile of 128 consecutive p
//     needs, per channel group of 8 and per dy, one window of 136 positions
//     in each of the 3 planes x..x+2 -- one 4-D TMA box (8 ch, 136 p, 3 x, 1)
//     that lands as [dx][p][8 ch], i.e. 8 positions x 16 bytes = one K-major
//     core matrix; every tap's A operand is the same window at a different
//     start address.  Positions with z >= Zin-2 wrap into the next row and
//     are dropped by the epilogue (2 of every Zin positions).
//   * all 27 x CIN x COUT weights stay in shared memory (K-major, packed on
//     the host as [tap][ci/8][co][8]).
//   * warp 0 issues TMA copies into a 2-stage ring, warp 1 owns TMEM and
//     issues the MMAs (one thread), warps 2-5 drain the double-buffered
//     accumulators (bias, GELU / GELU', BF16 or FP32 stores).
//   The input-gradient of a layer is the same kernel run on the output
//   gradient zero-padded by 2 with the taps flipped and W transposed.
//
// Weight-gradient kernel: dW_t[co][ci] = sum_v dZ[v][co] X[v+t][ci] over
// all output positions v.  D[M=128, N=COUT] per (dy, dz) pair, 9 TMEM
// accumulators; the M rows are (dx in 0..3, ci) -- dx = 3 is a block of
// ones, which turns its rows into the bias gradient sum_v dZ[v][co].  Both
// operands are MN-major: K is the position along z, 16 bytes apart.
//
// Every wait is bounded (~2 s); a timeout sets a status bit and the block
// drains its copies and MMAs and frees its TMEM before returning.
#pragma once
#include <cuda.h>
#include <cuda_bf16.h>
#include <stdint.h>

#include "dg_tc.cuh"

namespace dg {
namespace net {

constexpr int kM = 128;                    // positions per tile (MMA M)
constexpr int kWz = 136;                   // window positions per row (>= kM + 2; 128-byte boxes)
constexpr int kBox = 3 * kWz * 16;         // one TMA box: 3 rows of kWz positions x 8 channels (6528 B)
constexpr int kStages = 2;
constexpr int kConvThreads = 192;          // 6 warps: TMA, MMA, 4 x epilogue
constexpr unsigned kNetTimeout = 0x2u;     // status bit: a wait ran out

enum Epilogue : int { kEpiGelu = 0, kEpiLinear = 1, kEpiDGelu = 2 };

struct ConvArgs {
    int nb, xi, yi, zi;             // input extents
    int xo, yo, zo;                 // output extents (input - 2)
    int tpp;                        // tiles per (n, x) plane: ceil(yo * zi / kM)
    int ntiles;                     // nb * xo * tpp
    int ox, oy, oz, off;            // extents of the output buffer and offset of the output region in it
    const float *bias;              // [COUT] (kEpiGelu, kEpiLinear)
    __nv_bfloat16 *out_a;           // BF16 output: activation (kEpiGelu) or gradient (kEpiDGelu)
    __nv_bfloat16 *out_z;           // BF16 pre-activation, dense [nb][xo][yo][zo][COUT] (kEpiGelu, may be null)
    float *out_f;                   // FP32 output (kEpiLinear)
    const __nv_bfloat16 *zsrc;      // pre-activation below, dense [nb][xo][yo][zo][COUT] (kEpiDGelu)
    unsigned *status;
};

struct WgradArgs {
    int nb, xo, yo, zo;             // extents of the output-gradient region
    int nseg;                       // z segments of kM positions per row
    int ntiles;                     // nb * xo * yo * nseg
    float *part;                    // per block: [COUT][CIN][27] weight partials then [COUT] bias partials
    unsigned *status;
};

__device__ __forceinline__ unsigned char *align128(unsigned char *p) {
    const uint32_t s = smem_u32(p);
    return p + ((128u - (s & 127u)) & 127u);
}

__device__ __forceinline__ float gelu(float x) { return 0.5f * x * (1.0f + erff(x * 0.70710678118654752f)); }

__device__ __forceinline__ float gelu_grad(float x) {
    return 0.5f * (1.0f + erff(x * 0.70710678118654752f)) + x * 0.39894228040143268f * expf(-0.5f * x * x);
}

// All lanes of the warp agree on a wait's outcome.
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity) {
    const bool ok = mbar_wait(bar, parity, kWaitBudget);
    return __all_sync(0xffffffffu, ok);
}

__device__ __forceinline__ void store_bf16(__nv_bfloat16 *dst, const float *v, int n) {
    for (int c = 0; c < n; c += 8) {
        uint4 w;
        __nv_bfloat162 h0 = __floats2bfloat162_rn(v[c + 0], v[c + 1]);
        __nv_bfloat162 h1 = __floats2bfloat162_rn(v[c + 2], v[c + 3]);
        __nv_bfloat162 h2 = __floats2bfloat162_rn(v[c + 4], v[c + 5]);
        __nv_bfloat162 h3 = __floats2bfloat162_rn(v[c + 6], v[c + 7]);
        w.x = *reinterpret_cast<uint32_t *>(&h0);
        w.y = *reinterpret_cast<uint32_t *>(&h1);
        w.z = *reinterpret_cast<uint32_t *>(&h2);
        w.w = *reinterpret_cast<uint32_t *>(&h3);
        *reinterpret_cast<uint4 *>(dst + c) = w;
    }
}

__device__ __forceinline__ void load_bf16(const __nv_bfloat16 *src, float *v, int n) {
    for (int c = 0; c < n; c += 8) {
        const uint4 w = *reinterpret_cast<const uint4 *>(src + c);
        const uint32_t u[4] = {w.x, w.y, w.z, w.w};
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            v[c + 2 * i] = __uint_as_float(u[i] << 16);
            v[c + 2 * i + 1] = __uint_as_float(u[i] & 0xFFFF0000u);
        }
    }
}

template <int CIN, int COUT>
struct ConvSmem {
    static constexpr int CG = CIN / 8;
    static constexpr int WB = 27 * CG * COUT * 16;           // weights
    static constexpr int STAGE = CG * 3 * kBox;              // one input window
    static constexpr int BYTES = WB + kStages * STAGE + 128 /*barriers*/ + 128 /*alignment*/;
};

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kConvThreads, 1)
    conv_fwd_kernel(const __grid_constant__ CUtensorMap in_map, const __nv_bfloat16 *__restrict__ wpack, ConvArgs a) {
    static_assert(CIN % 16 == 0 && (COUT == 16 || COUT == 32), "unsupported channel counts");
    using L = ConvSmem<CIN, COUT>;
    constexpr int CG = L::CG, KC = CIN / 16;
    constexpr uint32_t TCOLS = 2 * COUT < 32 ? 32 : 2 * COUT;
    constexpr uint32_t IDESC = tc::idesc_bf16(kM, COUT, 0, 0);

    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = align128(smem_raw);
    unsigned char *wsm = smem;
    unsigned char *stg = smem + L::WB;
    uint64_t *bars = reinterpret_cast<uint64_t *>(stg + kStages * L::STAGE);
    uint64_t *full = bars, *empty = bars + 2, *tfull = bars + 4, *tempty = bars + 6, *wbar = bars + 8,
             *drain = bars + 9;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 10);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(full + i, 1);
            mbar_init(empty + i, 1);
            mbar_init(tfull + i, 1);
            mbar_init(tempty + i, 4);
        }
        mbar_init(wbar, 1);
        mbar_init(drain, 1);
        fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(tslot, TCOLS);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tbase = *tslot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            mbar_expect_tx(wbar, L::WB);
            tc::bulk_load(wsm, wpack, L::WB, wbar);
            int it = 0;
            for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++it) {
                const int s = it & 1, u = it >> 1;
                if (u > 0 && !mbar_wait(empty + s, (u - 1) & 1, kWaitBudget)) {
                    ok = false;
                    break;
                }
                const int pt = tile % a.tpp, bx = tile / a.tpp;
                const int x = bx % a.xo, b = bx / a.xo;
                const int p0 = pt * kM;
                mbar_expect_tx(full + s, L::STAGE);
                unsigned char *dst = stg + s * L::STAGE;
                for (int cg = 0; cg < CG; ++cg)
                    for (int dy = 0; dy < 3; ++dy)
                        tma_load_4d(dst + (cg * 3 + dy) * kBox, &in_map, cg * 8, p0 + dy * a.zi, x, b, full + s);
            }
            // copies still in flight must land before the block exits
            for (int j = it - 2 < 0 ? 0 : it - 2; j < it; ++j) ok &= mbar_wait(full + (j & 1), (j >> 1) & 1, kWaitBudget);
            ok &= mbar_wait(wbar, 0, kWaitBudget);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            ok = mbar_wait(wbar, 0, kWaitBudget);
            int it = 0;
            const uint32_t b0 = smem_u32(wsm);
            for (int tile = blockIdx.x; ok && tile < a.ntiles; tile += gridDim.x, ++it) {
                const int s = it & 1, u = it >> 1;
                if (!mbar_wait(full + s, u & 1, kWaitBudget)) {
                    ok = false;
                    break;
                }
                if (u > 0 && !mbar_wait(tempty + s, (u - 1) & 1, kWaitBudget)) {
                    ok = false;
                    break;
                }
                tc::fence_after();
                const uint32_t d = tbase + (uint32_t)(s * COUT);
                const uint32_t a0 = smem_u32(stg + s * L::STAGE);
#pragma unroll 1
                for (int t = 0; t < 27; ++t) {
                    const int dx = t / 9, dy = (t / 3) % 3, dz = t % 3;
#pragma unroll
                    for (int kc = 0; kc < KC; ++kc) {
                        const uint32_t aa = a0 + (uint32_t)((2 * kc * 3 + dy) * kBox + (dx * kWz + dz) * 16);
                        const uint32_t ba = b0 + (uint32_t)((t * CG + 2 * kc) * COUT * 16);
                        tc::mma_bf16(d, tc::sdesc(aa, 3 * kBox, 128), tc::sdesc(ba, COUT * 16, 128), IDESC,
                                     (t | kc) != 0);
                    }
                }
                tc::commit(empty + s);
                tc::commit(tfull + s);
            }
            tc::commit(drain);
            ok &= mbar_wait(drain, 0, kWaitBudget);
        }
    } else {
        const int q = warp & 3;
        int it = 0;
        for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++it) {
            const int s = it & 1, u = it >> 1;
            if (!warp_wait(tfull + s, u & 1)) {
                ok = false;
                break;
            }
            tc::fence_after();
            float acc[COUT];
#pragma unroll
            for (int c = 0; c < COUT; c += 16)
                tc::tmem_ld16(tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)(s * COUT + c), acc + c);
            tc::tmem_wait_ld();
            tc::fence_before();
            __syncwarp();
            if (lane == 0) tc::mbar_arrive(tempty + s);

            const int pt = tile % a.tpp, bx = tile / a.tpp;
            const int x = bx % a.xo, b = bx / a.xo;
            const int p = pt * kM + 32 * q + lane;
            const int y = p / a.zi, z = p - y * a.zi;
            if (y >= a.yo || z >= a.zo) continue;
            const long long o =
                ((((long long)b * a.ox + x + a.off) * a.oy + y + a.off) * a.oz + z + a.off) * COUT;
            const long long dn = ((((long long)b * a.xo + x) * a.yo + y) * a.zo + z) * COUT;
            if constexpr (EPI == kEpiGelu) {
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] += __ldg(a.bias + c);
                if (a.out_z) store_bf16(a.out_z + dn, acc, COUT);
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] = gelu(acc[c]);
                store_bf16(a.out_a + o, acc, COUT);
            } else if constexpr (EPI == kEpiLinear) {
#pragma unroll
                for (int c = 0; c < COUT; c += 4) {
                    float4 v = make_float4(acc[c] + __ldg(a.bias + c), acc[c + 1] + __ldg(a.bias + c + 1),
                                           acc[c + 2] + __ldg(a.bias + c + 2), acc[c + 3] + __ldg(a.bias + c + 3));
                    *reinterpret_cast<float4 *>(a.out_f + o + c) = v;
                }
            } else {
                float zv[COUT];
                load_bf16(a.zsrc + dn, zv, COUT);
#pragma unroll
                for (int c = 0; c < COUT; ++c) acc[c] *= gelu_grad(zv[c]);
                store_bf16(a.out_a + o, acc, COUT);
            }
        }
    }
    if (!ok) atomicOr(a.status, kNetTimeout);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 1) tc::tmem_dealloc(tbase, TCOLS);
}

template <int CIN, int COUT>
struct WgradSmem {
    static constexpr int XSTAGE = 16 * kBox;                 // 16 row groups (dx, cg) of [dy][kWz][8]
    static constexpr int GSTAGE = (COUT / 8) * kM * 16;      // output gradient [co/8][kM][8]
    static constexpr int BYTES = kStages * (XSTAGE + GSTAGE) + 128 + 128;
};

template <int CIN, int COUT>
__global__ void __launch_bounds__(kConvThreads, 1)
    conv_wgrad_kernel(const __grid_constant__ CUtensorMap x_map, const __grid_constant__ CUtensorMap g_map,
                      WgradArgs a) {
    static_assert((CIN == 16 || CIN == 32) && (COUT == 16 || COUT == 32), "unsupported channel counts");
    using L = WgradSmem<CIN, COUT>;
    constexpr int CG = CIN / 8, GG = COUT / 8;
    constexpr uint32_t NACC = 9 * COUT;
    constexpr uint32_t TCOLS = NACC <= 256 ? 256 : 512;
    constexpr uint32_t IDESC = tc::idesc_bf16(kM, COUT, 1, 1);
    constexpr uint32_t TX = 3 * CG * kBox + GG * kM * 16;    // bytes landing per tile

    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = align128(smem_raw);
    unsigned char *xs = smem;                                  // kStages x XSTAGE
    unsigned char *gs = smem + kStages * L::XSTAGE;            // kStages x GSTAGE
    uint64_t *bars = reinterpret_cast<uint64_t *>(gs + kStages * L::GSTAGE);
    uint64_t *full = bars, *empty = bars + 2, *done = bars + 4;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 6);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // rows dx = 3 of both stages hold ones (bias gradient)
    {
        const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
        for (int s = 0; s < kStages; ++s) {
            uint4 *p = reinterpret_cast<uint4 *>(xs + s * L::XSTAGE + 3 * CG * kBox);
            for (int i = threadIdx.x; i < CG * kBox / 16; i += blockDim.x) p[i] = ones;
        }
        fence_proxy_async();
    }
    if (threadIdx.x == 0) {
        for (int i = 0; i < 2; ++i) {
            mbar_init(full + i, 1);
            mbar_init(empty + i, 1);
        }
        mbar_init(done, 1);
        fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(tslot, TCOLS);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tbase = *tslot;
    bool ok = true;
    const int mytiles = blockIdx.x < a.ntiles ? (a.ntiles - 1 - blockIdx.x) / gridDim.x + 1 : 0;

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;
            for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++it) {
                const int s = it & 1, u = it >> 1;
                if (u > 0 && !mbar_wait(empty + s, (u - 1) & 1, kWaitBudget)) {
                    ok = false;
                    break;
                }
                int r = tile;
                const int seg = r % a.nseg; r /= a.nseg;
                const int y = r % a.yo; r /= a.yo;
                const int x = r % a.xo, b = r / a.xo;
                const int z0 = seg * kM;
                mbar_expect_tx(full + s, TX);
                unsigned char *xd = xs + s * L::XSTAGE;
                for (int dx = 0; dx < 3; ++dx)
                    for (int cg = 0; cg < CG; ++cg)
                        tc::tma_load_5d(xd + (dx * CG + cg) * kBox, &x_map, cg * 8, z0, y, x + dx, b, full + s);
                unsigned char *gd = gs + s * L::GSTAGE;
                for (int g = 0; g < GG; ++g)
                    tc::tma_load_5d(gd + g * kM * 16, &g_map, g * 8, z0 + 2, y + 2, x + 2, b, full + s);
            }
            for (int j = it - 2 < 0 ? 0 : it - 2; j < it; ++j) ok &= mbar_wait(full + (j & 1), (j >> 1) & 1, kWaitBudget);
        }
    } else if (warp == 1) {
        if (lane == 0) {
            int it = 0;
            for (int tile = blockIdx.x; tile < a.ntiles; tile += gridDim.x, ++it) {
                const int s = it & 1, u = it >> 1;
                if (!mbar_wait(full + s, u & 1, kWaitBudget)) {
                    ok = false;
                    break;
                }
                tc::fence_after();
                const int seg = tile % a.nseg;
                const int len = min(kM, a.zo - seg * kM);
                const int nk = (len + 15) >> 4;
                const uint32_t xa = smem_u32(xs + s * L::XSTAGE);
                const uint32_t ga = smem_u32(gs + s * L::GSTAGE);
#pragma unroll 1
                for (int ks = 0; ks < nk; ++ks) {
                    const uint64_t bd = tc::sdesc(ga + (uint32_t)(ks * 256), 128, kM * 16);
#pragma unroll
                    for (int j = 0; j < 9; ++j) {
                        const int dy = j / 3, dz = j % 3;
                        const uint32_t aa = xa + (uint32_t)((dy * kWz + dz + 16 * ks) * 16);
                        tc::mma_bf16(tbase + (uint32_t)(j * COUT), tc::sdesc(aa, 128, kBox), bd, IDESC,
                                     (it | ks) != 0);
                    }
                }
                tc::commit(empty + s);
            }
            tc::commit(done);
        }
    } else {
        const int q = warp & 3;
        const int m = 32 * q + lane;            // TMEM lane = row of D
        const int jgrp = m >> 3, ci_lo = m & 7;
        const int dx = jgrp / CG, cg = jgrp % CG;
        const bool have = mytiles > 0;
        if (have && !warp_wait(done, 0)) ok = false;
        tc::fence_after();
        float *wpart = a.part + (size_t)blockIdx.x * (COUT * CIN * 27 + COUT);
#pragma unroll 1
        for (int j = 0; j < 9; ++j) {
            float v[COUT];
#pragma unroll
            for (int c = 0; c < COUT; c += 16) tc::tmem_ld16(tbase + ((uint32_t)(32 * q) << 16) + j * COUT + c, v + c);
            tc::tmem_wait_ld();
            if (!have || !ok) {
#pragma unroll
                for (int c = 0; c < COUT; ++c) v[c] = 0.0f;
            }
            if (dx < 3) {
                const int ci = cg * 8 + ci_lo;
                const int t = dx * 9 + j;
#pragma unroll
                for (int co = 0; co < COUT; ++co) wpart[((size_t)co * CIN + ci) * 27 + t] = v[co];
            } else if (dx == 3 && cg == 0 && ci_lo == 0 && j == 0) {
#pragma unroll
                for (int co = 0; co < COUT; ++co) wpart[COUT * CIN * 27 + co] = v[co];
            }
        }
    }
    if (warp == 1 && lane == 0) ok &= mbar_wait(done, 0, kWaitBudget);
    if (!ok) atomicOr(a.status, kNetTimeout);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    if (warp == 1) tc::tmem_dealloc(tbase, TCOLS);
}

}  // namespace net
}  // namespace dg
