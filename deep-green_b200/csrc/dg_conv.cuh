// dg_conv.cuh -- BF16 3x3x3 convolution kernels of the correction network on
// the 5th-generation tensor cores (tcgen05, FP32 accumulation in TMEM).
//
// Activations are BF16 channels-last, [n][x][y][z][C], z fastest.  Every
// convolution is "valid": an input of extents (X, Y, Z) gives an output of
// (X-2, Y-2, Z-2), out[v] = sum_t W_t in[v + t], t = (dx, dy, dz) in 0..2,
// weights W[co][ci][dx][dy][dz] (the layout of torch.nn.Conv3d on tensors
// ordered (n, C, x, y, z)).
//
// Forward / input-gradient kernel (implicit GEMM, D[M=128 positions,
// N=COUT] = sum over 27 taps x CIN channels):
//   * positions are enumerated along the flattened (y, z) index of the INPUT,
//     p = y * Zin + z, within one (n, x) plane; tap (dx, dy, dz) is then the
//     plane x+dx shifted by dy*Zin + dz.  A tile of 128 consecutive p needs,
//     per dy, a window of 136 positions of an input plane: one TMA box of
//     rows of CIN channels (64 or 32 bytes), written with the hardware's 64-
//     or 32-byte swizzle, which is the canonical swizzled K-major operand
//     layout of the tensor cores; each (dy, dz) is that window at a start
//     address dz rows further.  Positions with z >= Zin-2 wrap into the next
//     row and are dropped by the epilogue (2 of every Zin positions).
//   * a block walks along x through a column of tiles (fixed n and p range,
//     x in a chunk).  Input plane P serves output planes P, P-1 and P-2 (taps
//     dx = 0, 1, 2), so each (dy, dz, 16 channels) is ONE MMA with N = 3 COUT
//     against the weights [W(dx=2) | W(dx=1) | W(dx=0)]: its three column
//     blocks land in the TMEM accumulators of output planes P-2, P-1, P,
//     which sit in a ring of 8 consecutive slots (an MMA that would wrap the
//     ring is split in two).  Output plane P-2 is then complete; the epilogue
//     drains its slot and zeroes it for reuse, so every MMA accumulates.
//     Each input plane is read from shared memory once, by 9 x CIN/16 MMAs.
//   * input planes arrive by TMA into a ring of shared-memory slots (3
//     windows each); planes at the start of a chunk produce two partial
//     outputs that are drained and discarded.
//   * all weights stay in shared memory, packed on the host as
//     [dy, dz][dx' = 2-dx][co][ci] rows, swizzled like the windows.
//   * warp 0 issues the TMA copies; warps 1 and 2 each issue half of every
//     plane's MMAs (one thread each, descriptors advanced by constant
//     offsets) into their own ring of accumulators -- a single thread's
//     dependent issue loop, not the tensor core, would otherwise set the
//     pace; warps 3-10 drain both rings (two warps per TMEM sub-partition,
//     each half of the columns: sum, bias, GELU / GELU', BF16 or FP32
//     stores) in a fixed order, so results do not depend on timing.
//   The input-gradient of a layer is the same kernel run on the output
//   gradient zero-padded by 2 with the taps flipped and W transposed.
//
// Weight-gradient kernel: dW_t[co][ci] = sum_v dZ[v][co] X[v+t][ci] over
// all output positions v.  D[M=128, N=COUT] per (dy, dz) pair, 9 TMEM
// accumulators; the M rows are (dx in 0..3, ci) -- dx = 3 is a block of
// ones, which turns its rows into the bias gradient sum_v dZ[v][co].  Both
// operands are MN-major: K is the position along z, 16 bytes apart.  A block
// walks a column of output rows along y (one tile = one row segment of kM
// positions): the input rows y, y+1, y+2 that tile y reads sit in a ring of
// 4 rows per (dx, channel group), so each tile brings one new input row.
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
constexpr int kConvThreads = 192;          // weight gradient: 6 warps (TMA, MMA, 4 x epilogue)
constexpr int kIssuers = 2;                // forward: MMA-issuing warps, each with its own accumulators
constexpr int kFwdThreads = 32 * (1 + kIssuers + 8);   // forward: TMA, issuers, 8 x epilogue
// Forward kernel: TMEM accumulator slots (output planes) of one issuer's ring;
// the rings of all issuers fill the 512 TMEM columns.
template <int COUT> constexpr int fwd_ring() { return 512 / (kIssuers * COUT); }
constexpr int kSlots = 4;                  // input-plane slots of the forward kernel's shared-memory ring
constexpr unsigned kNetTimeout = 0x2u;     // status bit: a wait ran out

enum Epilogue : int { kEpiGelu = 0, kEpiLinear = 1, kEpiDGelu = 2 };

struct ConvArgs {
    int nb, xi, yi, zi;             // input extents
    int xo, yo, zo;                 // output extents (input - 2)
    int tpp;                        // tiles per (n, x) plane: ceil(yo * zi / kM)
    int xchunk;                     // planes of x per work unit
    int nxc;                        // x chunks: ceil(xo / xchunk)
    int nunits;                     // work units nb * tpp * nxc: (n, p range, x chunk)
    int ox, oy, oz, off;            // extents of the output buffer and offset of the output region in it
    const float *bias;              // [COUT] (kEpiGelu, kEpiLinear)
    __nv_bfloat16 *out_a;           // BF16 output: activation (kEpiGelu) or gradient (kEpiDGelu)
    __nv_bfloat16 *out_z;           // BF16 pre-activation, extents (xo, yo, zo), no offset (kEpiGelu, may be null)
    float *out_f;                   // FP32 output (kEpiLinear)
    const __nv_bfloat16 *zsrc;      // pre-activation below, extents (xo, yo, zo), no offset (kEpiDGelu)
    unsigned *status;
};

struct WgradArgs {
    int nb, xo, yo, zo;             // extents of the output-gradient region
    int nseg;                       // z segments of kM positions per row
    int ych, nyc;                   // rows per work unit, units per column: ceil(yo / ych)
    int nunits;                     // work units (n, x, z segment, y chunk): nb * xo * nseg * nyc
    float *part;                    // per block: [COUT][CIN][27] weight partials then [COUT] bias partials
    unsigned *status;
};

__device__ __forceinline__ unsigned char *align128(unsigned char *p) {
    const uint32_t s = smem_u32(p);
    return p + ((128u - (s & 127u)) & 127u);
}

__device__ __forceinline__ unsigned char *align1024(unsigned char *p) {
    const uint32_t s = smem_u32(p);
    return p + ((1024u - (s & 1023u)) & 1023u);
}

// GELU in its tanh form, x/2 (1 + tanh(sqrt(2/pi) (x + 0.044715 x^3)))
// (Hendrycks & Gimpel 2016), on the hardware tanh approximation
// (tanh.approx.f32, relative error ~2^-11, far below BF16 rounding).
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float kGeluC0 = 0.79788456080286536f;   // sqrt(2 / pi)
constexpr float kGeluC1 = 0.044715f;

__device__ __forceinline__ float gelu(float x) {
    const float t = tanh_approx(kGeluC0 * (x + kGeluC1 * x * x * x));
    return 0.5f * x * (1.0f + t);
}

__device__ __forceinline__ float gelu_grad(float x) {
    const float t = tanh_approx(kGeluC0 * (x + kGeluC1 * x * x * x));
    return 0.5f * (1.0f + t) + 0.5f * x * (1.0f - t * t) * kGeluC0 * (1.0f + 3.0f * kGeluC1 * x * x);
}

// All lanes of the warp agree on a wait's outcome.
__device__ __forceinline__ bool warp_wait(uint64_t *bar, uint32_t parity) {
    const bool ok = tc::mbar_sleep_wait(bar, parity, kWaitBudget);
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

// 16 values as BF16 with one 32-byte store (dst 32-byte aligned).
__device__ __forceinline__ void store16_bf16(__nv_bfloat16 *dst, const float *v) {
    uint32_t w[8];
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        __nv_bfloat162 h = __floats2bfloat162_rn(v[2 * i], v[2 * i + 1]);
        w[i] = *reinterpret_cast<uint32_t *>(&h);
    }
    asm volatile("st.global.v8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(dst), "r"(w[0]), "r"(w[1]),
                 "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7])
                 : "memory");
}

// 8 FP32 values with one 32-byte store (dst 32-byte aligned).
__device__ __forceinline__ void store8_f32(float *dst, const float *v) {
    asm volatile("st.global.v8.f32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"l"(dst), "f"(v[0]), "f"(v[1]),
                 "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7])
                 : "memory");
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
    static constexpr int ROW = CIN * 2;                       // bytes of one position (swizzle width)
    static constexpr int WB = 27 * COUT * ROW;                // weights
    static constexpr int WIN = (kWz * ROW + 1023) / 1024 * 1024;   // one window, 1024-byte aligned
    static constexpr int SLOT = 3 * WIN;                      // the dy windows of one x-plane
    static constexpr int BYTES = WB + kSlots * SLOT + 1024 /*barriers*/ + 1024 /*alignment*/;
};

template <int CIN, int COUT, int EPI>
__global__ void __launch_bounds__(kFwdThreads, 1)
    conv_fwd_kernel(const __grid_constant__ CUtensorMap in_map, const __nv_bfloat16 *__restrict__ wpack, ConvArgs a) {
    static_assert((CIN == 16 || CIN == 32) && (COUT == 16 || COUT == 32), "unsupported channel counts");
    static_assert(kIssuers == 1 || kIssuers == 2, "one or two issuing warps");
    using L = ConvSmem<CIN, COUT>;
    constexpr int KC = CIN / 16;
    constexpr int ROW = L::ROW;
    constexpr int NC = COUT / 2;                 // columns per epilogue warp
    constexpr int NB = 3 * COUT;                 // rows of the weight operand (three dx blocks)
    constexpr int R = fwd_ring<COUT>();          // slots of one issuer's ring
    constexpr int RING = R * COUT;               // TMEM columns of one issuer's ring
    constexpr uint32_t TCOLS = kIssuers * RING;  // 512
    static_assert(TCOLS == 512 && R >= 8, "ring layout");
    constexpr uint32_t ID3 = tc::idesc_bf16(kM, 3 * COUT, 0, 0);
    constexpr uint32_t ID2 = tc::idesc_bf16(kM, 2 * COUT, 0, 0);
    constexpr uint32_t ID1 = tc::idesc_bf16(kM, COUT, 0, 0);
    constexpr int EPI0 = 1 + kIssuers;           // first epilogue warp

    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = align1024(smem_raw);   // swizzle patterns follow address bits
    unsigned char *wsm = smem;
    unsigned char *ring = smem + L::WB;
    uint64_t *bars = reinterpret_cast<uint64_t *>(ring + kSlots * L::SLOT);
    uint64_t *full = bars, *empty = bars + kSlots, *tfull = bars + 2 * kSlots, *tempty = tfull + R,
             *wbar = tempty + R, *drain = wbar + 1;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(drain + kIssuers);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int i = 0; i < kSlots; ++i) {
            mbar_init(full + i, 1);
            mbar_init(empty + i, kIssuers);
        }
        for (int i = 0; i < R; ++i) {
            mbar_init(tfull + i, kIssuers);
            mbar_init(tempty + i, 8);
        }
        mbar_init(wbar, 1);
        for (int i = 0; i < kIssuers; ++i) mbar_init(drain + i, 1);
        fence_mbar_init();
    }
    if (warp == 1) tc::tmem_alloc(tslot, TCOLS);
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    const uint32_t tbase = *tslot;
    const int q = warp & 3;                      // epilogue: TMEM sub-partition (lanes 32q..32q+31)
    const int c0 = ((warp - EPI0) >> 2) * NC;    // epilogue: first column of this warp's half
    if (warp >= EPI0) {
        // every accumulator starts at zero: all MMAs accumulate
        float zero[NC];
#pragma unroll
        for (int c = 0; c < NC; ++c) zero[c] = 0.0f;
        for (int sl = 0; sl < kIssuers * R; ++sl) {
            const uint32_t ta = tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)(sl * COUT + c0);
            if constexpr (NC == 16) tc::tmem_st16(ta, zero);
            else tc::tmem_st8(ta, zero);
        }
        tc::tmem_wait_st();
    }
    tc::fence_before();
    __syncthreads();
    tc::fence_after();
    bool ok = true;
    float bias[NC];                              // epilogue: this warp's bias columns
#pragma unroll
    for (int c = 0; c < NC; ++c) bias[c] = (EPI != kEpiDGelu && warp >= EPI0) ? __ldg(a.bias + c0 + c) : 0.0f;

    if (warp == 0) {
        if (lane == 0) {
            mbar_expect_tx(wbar, L::WB);
            tc::bulk_load(wsm, wpack, L::WB, wbar);
            long long g = 0;                      // planes issued by this block
            for (int unit = blockIdx.x; ok && unit < a.nunits; unit += gridDim.x) {
                const int xc = unit % a.nxc, r = unit / a.nxc;
                const int pt = r % a.tpp, b = r / a.tpp;
                const int x0 = xc * a.xchunk, len = min(a.xchunk, a.xo - x0);
                const int p0 = pt * kM;
                for (int k = 0; k < len + 2; ++k, ++g) {
                    const int slot = (int)(g % kSlots);
                    const long long use = g / kSlots;
                    if (use > 0 && !tc::mbar_sleep_wait(empty + slot, (uint32_t)((use - 1) & 1), kWaitBudget)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(full + slot, 3 * kWz * ROW);
                    unsigned char *dst = ring + slot * L::SLOT;
                    for (int dy = 0; dy < 3; ++dy)
                        tma_load_4d(dst + dy * L::WIN, &in_map, 0, p0 + dy * a.zi, x0 + k, b, full + slot);
                }
            }
            // copies still in flight must land before the block exits
            for (long long j = g - kSlots < 0 ? 0 : g - kSlots; j < g; ++j)
                ok &= tc::mbar_sleep_wait(full + (int)(j % kSlots), (uint32_t)((j / kSlots) & 1), kWaitBudget);
            ok &= tc::mbar_sleep_wait(wbar, 0, kWaitBudget);
        }
    } else if (warp <= kIssuers) {
        // The whole warp runs the issue loop and one elected lane issues each
        // plane's MMAs and commits (see elect_one).
        const int me = warp - 1;              // issuer index: its half of the MMAs, its ring
        ok = warp_wait(wbar, 0);
        long long g = 0;                      // input planes consumed = output slots completed
        const uint64_t b0 = tc::sdesc_sw(smem_u32(wsm), ROW);
        const uint32_t rbase = tbase + (uint32_t)(me * RING);
        for (int unit = blockIdx.x; ok && unit < a.nunits; unit += gridDim.x) {
            const int xc = unit % a.nxc;
            const int len = min(a.xchunk, a.xo - xc * a.xchunk);
            for (int k = 0; k < len + 2; ++k, ++g) {
                const int ps = (int)(g % kSlots);
                bool got = tc::mbar_sleep_wait(full + ps, (uint32_t)((g / kSlots) & 1), kWaitBudget);
                // the third block writes output slot g+2 first: its previous
                // occupant must have been drained and zeroed
                const long long w2 = g + 2;
                if (got && w2 >= R)
                    got = tc::mbar_sleep_wait(tempty + (int)(w2 % R), (uint32_t)((w2 / R - 1) & 1), kWaitBudget);
                if (!__all_sync(0xffffffffu, got)) {
                    ok = false;
                    break;
                }
                tc::fence_after();
                const int s0 = (int)(g % R);
                const uint32_t d0 = rbase + (uint32_t)(s0 * COUT);
                // descriptors advance by (byte offset >> 4) in their 14-bit address field;
                // every address stays below 256 KB, so no carry leaves the field
                const uint64_t a0 = tc::sdesc_sw(smem_u32(ring + ps * L::SLOT), ROW);
                // this issuer's MMAs: every (tap, channel half) with one issuer; with
                // two, channel half kc = me (CIN 32) or taps 0-4 / 5-8 (CIN 16)
                constexpr int NT = kIssuers == 1 ? 9 * KC : (KC == 2 ? 9 : 5);
                const int t9lo = (kIssuers == 2 && KC == 1) ? me * 5 : 0;
                const int t9hi = (kIssuers == 2 && KC == 1) ? (me ? 9 : 5) : 9;
                const int kc0 = (kIssuers == 2 && KC == 2) ? me : 0;
                if (tc::elect_one()) {
                    if (s0 <= R - 3) {
#pragma unroll
                        for (int j = 0; j < NT; ++j) {
                            const int t9 = t9lo + j % 9, kc = kc0 + j / 9;
                            if (t9 >= t9hi) break;
                            const int dy = t9 / 3, dz = t9 % 3;
                            const uint64_t ad = a0 + (uint32_t)((dy * L::WIN + dz * ROW + kc * 32) >> 4);
                            const uint64_t bd = b0 + (uint32_t)((t9 * NB * ROW + kc * 32) >> 4);
                            tc::mma_bf16(d0, ad, bd, ID3, 1u);
                        }
                    } else {
                        // the three blocks would wrap the ring: two MMAs each
                        const int n1 = R - s0;
                        const uint32_t i1 = n1 == 2 ? ID2 : ID1, i2 = n1 == 2 ? ID1 : ID2;
                        const uint32_t bo2 = (uint32_t)((n1 * COUT * ROW) >> 4);
#pragma unroll
                        for (int j = 0; j < NT; ++j) {
                            const int t9 = t9lo + j % 9, kc = kc0 + j / 9;
                            if (t9 >= t9hi) break;
                            const int dy = t9 / 3, dz = t9 % 3;
                            const uint64_t ad = a0 + (uint32_t)((dy * L::WIN + dz * ROW + kc * 32) >> 4);
                            const uint64_t bd = b0 + (uint32_t)((t9 * NB * ROW + kc * 32) >> 4);
                            tc::mma_bf16(d0, ad, bd, i1, 1u);
                            tc::mma_bf16(rbase, ad, bd + bo2, i2, 1u);
                        }
                    }
                    tc::commit(empty + ps);           // input plane g is not needed again
                    tc::commit(tfull + s0);           // output slot g is complete
                }
                __syncwarp();
            }
        }
        if (tc::elect_one()) tc::commit(drain + me);
        __syncwarp();
        ok &= warp_wait(drain + me, 0);
    } else {
        long long g = 0;
        for (int unit = blockIdx.x; ok && unit < a.nunits; unit += gridDim.x) {
            const int xc = unit % a.nxc, r = unit / a.nxc;
            const int pt = r % a.tpp, b = r / a.tpp;
            const int x0 = xc * a.xchunk, len = min(a.xchunk, a.xo - x0);
            const int p = pt * kM + 32 * q + lane;
            const int y = p / a.zi, z = p - y * a.zi;
            const bool valid = y < a.yo && z < a.zo;
            for (int k = 0; k < len + 2; ++k, ++g) {
                const int sl = (int)(g % R);
                if (!warp_wait(tfull + sl, (uint32_t)((g / R) & 1))) {
                    ok = false;
                    break;
                }
                tc::fence_after();
                float v[NC], v2[NC], zero[NC];
#pragma unroll
                for (int c = 0; c < NC; ++c) zero[c] = 0.0f;
                const uint32_t ta = tbase + ((uint32_t)(32 * q) << 16) + (uint32_t)(sl * COUT + c0);
                if constexpr (NC == 16) {
                    tc::tmem_ld16(ta, v);
                    if constexpr (kIssuers == 2) tc::tmem_ld16(ta + RING, v2);
                    tc::tmem_wait_ld();
                    tc::tmem_st16(ta, zero);
                    if constexpr (kIssuers == 2) tc::tmem_st16(ta + RING, zero);
                } else {
                    tc::tmem_ld8(ta, v);
                    if constexpr (kIssuers == 2) tc::tmem_ld8(ta + RING, v2);
                    tc::tmem_wait_ld();
                    tc::tmem_st8(ta, zero);
                    if constexpr (kIssuers == 2) tc::tmem_st8(ta + RING, zero);
                }
                tc::tmem_wait_st();
                tc::fence_before();
                __syncwarp();
                if (lane == 0) tc::mbar_arrive(tempty + sl);
                // slot g holds output plane x0 + k - 2 of this chunk when k >= 2;
                // the first two slots of a chunk mix planes of two chunks
                if (k < 2 || !valid) continue;
                if constexpr (kIssuers == 2)
#pragma unroll
                    for (int c = 0; c < NC; ++c) v[c] += v2[c];

                const int x = x0 + k - 2;
                const long long o =
                    ((((long long)b * a.ox + x + a.off) * a.oy + y + a.off) * a.oz + z + a.off) * COUT + c0;
                const long long dn = ((((long long)b * a.xo + x) * a.yo + y) * a.zo + z) * COUT + c0;
                // one 32-byte store per lane and tensor where the columns allow
                // (COUT 32: 16 BF16 columns; COUT 16: 8 FP32 columns)
                if constexpr (EPI == kEpiGelu) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) v[c] += bias[c];
                    if (a.out_z) {
                        if constexpr (NC == 16) store16_bf16(a.out_z + dn, v);
                        else store_bf16(a.out_z + dn, v, NC);
                    }
#pragma unroll
                    for (int c = 0; c < NC; ++c) v[c] = gelu(v[c]);
                    if constexpr (NC == 16) store16_bf16(a.out_a + o, v);
                    else store_bf16(a.out_a + o, v, NC);
                } else if constexpr (EPI == kEpiLinear) {
#pragma unroll
                    for (int c = 0; c < NC; ++c) v[c] += bias[c];
                    if constexpr (NC == 8) {
                        store8_f32(a.out_f + o, v);
                    } else {
#pragma unroll
                        for (int c = 0; c < NC; c += 4)
                            *reinterpret_cast<float4 *>(a.out_f + o + c) = make_float4(v[c], v[c + 1], v[c + 2], v[c + 3]);
                    }
                } else {
                    float zv[NC];
                    load_bf16(a.zsrc + dn, zv, NC);
#pragma unroll
                    for (int c = 0; c < NC; ++c) v[c] *= gelu_grad(zv[c]);
                    if constexpr (NC == 16) store16_bf16(a.out_a + o, v);
                    else store_bf16(a.out_a + o, v, NC);
                }
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
    static constexpr int ROWB = kWz * 16;                    // one input row of one group: [kWz][8 ch]
    static constexpr int GROUP = 4 * ROWB;                   // a ring of 4 rows per group (the SBO of A)
    static constexpr int XRING = 16 * GROUP;                 // 16 groups (dx, cg); dx = 3 holds ones
    static constexpr int GSTAGE = (COUT / 8) * kM * 16;      // output gradient [co/8][kM][8]
    static constexpr int BYTES = XRING + kStages * GSTAGE + 128 + 128;
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
    constexpr uint32_t ROWTX = 3 * CG * L::ROWB;             // one new input row of every data group
    constexpr uint32_t GTX = GG * kM * 16;                   // one tile's output-gradient segment

    extern __shared__ unsigned char smem_raw[];
    unsigned char *smem = align128(smem_raw);
    unsigned char *xr = smem;                                  // input-row rings [16 groups][4 rows]
    unsigned char *gs = smem + L::XRING;                       // kStages x GSTAGE
    uint64_t *bars = reinterpret_cast<uint64_t *>(gs + kStages * L::GSTAGE);
    uint64_t *full = bars, *empty = bars + 2, *done = bars + 4;
    uint32_t *tslot = reinterpret_cast<uint32_t *>(bars + 6);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    // the dx = 3 groups hold ones in every ring row (bias gradient)
    {
        const uint4 ones = make_uint4(0x3F803F80u, 0x3F803F80u, 0x3F803F80u, 0x3F803F80u);
        uint4 *p = reinterpret_cast<uint4 *>(xr + 3 * CG * L::GROUP);
        for (int i = threadIdx.x; i < CG * L::GROUP / 16; i += blockDim.x) p[i] = ones;
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

    if (warp == 0) {
        if (lane == 0) {
            int it = 0;                                          // tiles of this block so far
            for (int unit = blockIdx.x; ok && unit < a.nunits; unit += gridDim.x) {
                int r = unit;
                const int yc = r % a.nyc; r /= a.nyc;
                const int seg = r % a.nseg; r /= a.nseg;
                const int x = r % a.xo, b = r / a.xo;
                const int y0 = yc * a.ych, ylen = min(a.ych, a.yo - y0);
                const int z0 = seg * kM;
                for (int j = 0; j < ylen; ++j, ++it) {
                    const int s = it & 1, u = it >> 1;
                    // tile it-2 done: its gradient stage and the ring row that
                    // this tile's new row replaces are free
                    if (u > 0 && !mbar_wait(empty + s, (u - 1) & 1, kWaitBudget)) {
                        ok = false;
                        break;
                    }
                    // a new column loads rows y0, y0+1 too, over the rows
                    // that tile it-1 still reads
                    if (j == 0 && it > 0 && !mbar_wait(empty + ((it - 1) & 1), ((it - 1) >> 1) & 1, kWaitBudget)) {
                        ok = false;
                        break;
                    }
                    const int first = j == 0 ? 0 : 2;            // new rows: j+first .. j+2
                    mbar_expect_tx(full + s, (3 - first) * ROWTX + GTX);
                    for (int dr = first; dr < 3; ++dr) {
                        const int slot = (it + dr) & 3;
                        for (int dx = 0; dx < 3; ++dx)
                            for (int cg = 0; cg < CG; ++cg)
                                tma_load_4d(xr + (dx * CG + cg) * L::GROUP + slot * L::ROWB, &x_map, cg * 8, z0,
                                            y0 + j + dr, b * (a.xo + 2) + x + dx, full + s);
                    }
                    unsigned char *gd = gs + s * L::GSTAGE;
                    for (int g = 0; g < GG; ++g)
                        tma_load_4d(gd + g * kM * 16, &g_map, g * 8, z0 + 2, y0 + j + 2, b * (a.xo + 4) + x + 2,
                                    full + s);
                }
            }
            for (int j = it - 2 < 0 ? 0 : it - 2; j < it; ++j) ok &= mbar_wait(full + (j & 1), (j >> 1) & 1, kWaitBudget);
        }
    } else if (warp == 1) {
        // the whole warp runs the issue loop; the elected lane issues each
        // tile's MMAs and its commit (see elect_one)
        int it = 0;
        for (int unit = blockIdx.x; ok && unit < a.nunits; unit += gridDim.x) {
            int r = unit;
            const int yc = r % a.nyc; r /= a.nyc;
            const int seg = r % a.nseg;
            const int ylen = min(a.ych, a.yo - yc * a.ych);
            const int len = min(kM, a.zo - seg * kM);
            const int nk = (len + 15) >> 4;
            for (int j = 0; j < ylen; ++j, ++it) {
                const int s = it & 1, u = it >> 1;
                if (!warp_wait(full + s, u & 1)) {
                    ok = false;
                    break;
                }
                tc::fence_after();
                const uint32_t xa = smem_u32(xr);
                const uint32_t ga = smem_u32(gs + s * L::GSTAGE);
                if (tc::elect_one()) {
#pragma unroll 1
                    for (int ks = 0; ks < nk; ++ks) {
                        const uint64_t bd = tc::sdesc(ga + (uint32_t)(ks * 256), 128, kM * 16);
                        const uint32_t acc = (it | ks) != 0;
#pragma unroll
                        for (int t9 = 0; t9 < 9; ++t9) {
                            const int dy = t9 / 3, dz = t9 % 3;
                            const uint32_t aa =
                                xa + (uint32_t)(((it + dy) & 3) * L::ROWB) + (uint32_t)((dz + 16 * ks) * 16);
                            tc::mma_bf16(tbase + (uint32_t)(t9 * COUT), tc::sdesc(aa, 128, L::GROUP), bd, IDESC,
                                         acc);
                        }
                    }
                    tc::commit(empty + s);
                }
                __syncwarp();
            }
        }
        if (tc::elect_one()) tc::commit(done);
        __syncwarp();
    } else {
        const int q = warp & 3;
        const int m = 32 * q + lane;            // TMEM lane = row of D
        const int jgrp = m >> 3, ci_lo = m & 7;
        const int dx = jgrp / CG, cg = jgrp % CG;
        const bool have = blockIdx.x < a.nunits;
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
