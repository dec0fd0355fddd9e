// dg_net.cu -- the correction network: parameters, Adam, workspace and the
// C ABI of deepgreen_net.h.  The convolutions are the tcgen05 kernels of
// dg_conv.cuh; everything else here is small element-wise kernels.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/deepgreen_net.h"
#include "dg_conv.cuh"
#include "dg_host.h"
#include "dg_net_impl.h"

using namespace dg;
using namespace dg::net;

namespace {

constexpr int kIO = DG_NET_IO_CHANNELS;
constexpr int kH = DG_NET_HIDDEN;
constexpr int kCin[4] = {kIO, kH, kH, kH};
constexpr int kCout[4] = {kH, kH, kH, kIO};

struct Workspace {
    int n = 0, x = 0, y = 0, z = 0;   // input extents it was sized for
    bool train = false;
    __nv_bfloat16 *act[3] = {};        // A1..A3 dense
    __nv_bfloat16 *pre[3] = {};        // Z1..Z3 dense (training)
    float *out = nullptr;              // network output (training)
    __nv_bfloat16 *dz[4] = {};         // gradients w.r.t. Z1..Z3 and the output, padded by 2
    size_t act_bytes[3] = {}, dz_bytes[4] = {}, out_bytes = 0;
    float *gbuf = nullptr;             // flux-form loss: gradient w.r.t. the corrections
    long long gbuf_elems = 0;
    float *wsample = nullptr;          // flux-form loss: per-entry weights (after gbuf)
};

}  // namespace

struct dg_net {
    int device = 0;
    int inputs = 0, outputs = 0;
    cudaStream_t stream = nullptr;
    float *w[4] = {}, *b[4] = {};
    float *gw[4] = {}, *gb[4] = {};
    float *mw[4] = {}, *vw[4] = {}, *mb[4] = {}, *vb[4] = {};
    __nv_bfloat16 *wf[4] = {};         // forward packing
    __nv_bfloat16 *wd[4] = {};         // input-gradient packing (layers 1..3)
    unsigned *status = nullptr;
    float *wpart = nullptr;            // weight-gradient partials, one row per block
    double *loss_part = nullptr;
    double *pow_part = nullptr;        // flux-form loss: target power partials [64 entries][kPowBlocks]
    int nsm = 148;
    long long adam_t = 0;
    Workspace ws;
    std::string err;
};

namespace {

// message of the calling thread's last failure outside a network
thread_local std::string g_net_err;

int fail(dg_net *n, int code, const std::string &m) {
    if (n) n->err = m;
    else g_net_err = m;
    return code;
}

#define NET_CUDA(net, call)                                                                  \
    do {                                                                                     \
        cudaError_t e_ = (call);                                                             \
        if (e_ != cudaSuccess) return fail(net, DG_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    });
    return fn;
}

// Channels-last BF16 tensors [n][x][y][z][c] seen by TMA.
// Forward / input-gradient operand: 4-D view (c, y*z, x, n), box (c, kWz,
// 1, 1) -- one window of one x-plane -- written with the 64-byte (c = 32)
// or 32-byte (c = 16) swizzle the tensor cores read.
bool map_conv_input(CUtensorMap *m, const void *base, int c, int n, int x, int y, int z) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t e = 2;
    cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)y * z, (cuuint64_t)x, (cuuint64_t)n};
    cuuint64_t strides[3] = {c * e, (cuuint64_t)y * z * c * e, (cuuint64_t)x * y * z * c * e};
    cuuint32_t box[4] = {(cuuint32_t)c, (cuuint32_t)kWz, 1, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, c == 32 ? CU_TENSOR_MAP_SWIZZLE_64B : CU_TENSOR_MAP_SWIZZLE_32B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// Weight-gradient operands: 4-D view (c, z, y, x + n * x_extent), box (8,
// bz, by, 1): 8 channels of each position, no swizzle.
bool map_wgrad(CUtensorMap *m, const void *base, int c, int n, int x, int y, int z, int bz, int by) {
    auto fn = encode_fn();
    if (!fn) return false;
    const cuuint64_t e = 2;
    cuuint64_t dims[4] = {(cuuint64_t)c, (cuuint64_t)z, (cuuint64_t)y, (cuuint64_t)x * n};
    cuuint64_t strides[3] = {c * e, (cuuint64_t)z * c * e, (cuuint64_t)y * z * c * e};
    cuuint32_t box[4] = {8, (cuuint32_t)bz, (cuuint32_t)by, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void *>(base), dims, strides, box, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// ---------------------------------------------------------------------------
// Element-wise kernels
// ---------------------------------------------------------------------------

// Weight operand of the forward kernel: rows r = ((dy, dz), dx' = 2 - dx, co)
// of kin channels (2 kin bytes), in the tensor cores' swizzled K-major layout:
// the 16-byte chunk c of row r is stored at chunk c ^ ((r * row >> 7) &
// (row/16 - 1)) (the shared-memory copy starts 1024-byte aligned).  `flip`
// packs the input-gradient convolution instead, with cin' = cout, cout' =
// cin and W'_t[co'][ci'] = W_{26-t}[ci'][co'] (taps flipped, channels
// transposed).
__global__ void pack_kernel(const float *__restrict__ w, __nv_bfloat16 *__restrict__ out, int cin, int cout,
                            int flip) {
    const int kin = flip ? cout : cin, kout = flip ? cin : cout;   // channels of the packed convolution
    const int row = 2 * kin;
    const int total = 27 * kin * kout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const int r = i / kin, pos = i % kin;
        const int mask = ((r * row) >> 7) & (row / 16 - 1);
        const int ci = (((pos >> 3) ^ mask) << 3) | (pos & 7);     // logical channel stored here
        const int n = r % (3 * kout), t9 = r / (3 * kout);
        const int dx = 2 - n / kout, co = n % kout;
        const int t = dx * 9 + t9;
        const float v = flip ? w[((size_t)ci * cin + co) * 27 + (26 - t)] : w[((size_t)co * cin + ci) * 27 + t];
        out[i] = __float2bfloat16_rn(v);
    }
}

// Fixed-order sum of the per-block weight-gradient partials.
__global__ void wgrad_reduce_kernel(const float *__restrict__ part, int nblocks, int cin, int cout, float *gw,
                                    float *gb) {
    const int nw = cout * cin * 27, row = nw + cout;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < row; i += gridDim.x * blockDim.x) {
        float s = 0.0f;
        for (int k = 0; k < nblocks; ++k) s += part[(size_t)k * row + i];
        if (i < nw) gw[i] = s;
        else gb[i - nw] = s;
    }
}

// Loss and its gradient w.r.t. the network output: L = mean (out - t)^2 over
// positions and the first `nout` channels.  The gradient (BF16) goes to the
// interior of a buffer padded by 2 on each side; per-block partial sums of
// the squared error go to part[blockIdx.x].
__global__ void loss_kernel(const float *__restrict__ out, const float *__restrict__ tgt, int n, int x, int y, int z,
                            int nout, float scale, __nv_bfloat16 *__restrict__ dz, double *part) {
    __shared__ double red[32];
    const long long total = (long long)n * x * y * z;
    double acc = 0.0;
    for (long long v = blockIdx.x * (long long)blockDim.x + threadIdx.x; v < total;
         v += (long long)gridDim.x * blockDim.x) {
        long long r = v;
        const int iz = r % z; r /= z;
        const int iy = r % y; r /= y;
        const int ix = r % x;
        const int b = (int)(r / x);
        float g[kIO];
#pragma unroll
        for (int c = 0; c < kIO; ++c) {
            const float d = c < nout ? out[v * kIO + c] - tgt[(size_t)v * kIO + c] : 0.0f;
            acc += (double)d * d;
            g[c] = scale * d;
        }
        const long long o = ((((long long)b * (x + 4) + ix + 2) * (y + 4) + iy + 2) * (z + 4) + iz + 2) * kIO;
        store_bf16(dz + o, g, kIO);
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) s += red[i];
        part[blockIdx.x] = s;
    }
}

// Flux-form loss, pass 1: the correction of target cell t is the divergence
// of the network's face fluxes, dU_c(t) = sum_d F_{d,c}(t+1) - F_{d,c}(t+1-e_d)
// (output channel 5 d + c, output cell t+1 in an output one cell larger than
// the target on each axis); residual r = dU - target, squared-error partials
// per block, and g = scale * r into gbuf [n][s^3][5].
// Target power of each batch entry: block (x, b) sums the squares of the 5
// target channels over its share of entry b's cells (rows of 16 floats read
// as one float4 and one float) into part[b][x].
constexpr int kPowBlocks = 64;
__global__ void __launch_bounds__(256) sample_power_kernel(const float *__restrict__ tgt, int s,
                                                           double *__restrict__ part) {
    __shared__ double red[8];
    const int b = blockIdx.y;
    const long long per = (long long)s * s * s;
    const float *t = tgt + (long long)b * per * 16;
    double acc = 0.0;
    for (long long v = blockIdx.x * 256LL + threadIdx.x; v < per; v += kPowBlocks * 256LL) {
        const float4 a = *reinterpret_cast<const float4 *>(t + v * 16);
        const float e = t[v * 16 + 4];
        acc += (double)a.x * a.x + (double)a.y * a.y + (double)a.z * a.z + (double)a.w * a.w + (double)e * e;
    }
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int i = 0; i < 8; ++i) sum += red[i];
        part[b * kPowBlocks + blockIdx.x] = sum;
    }
}

// Per batch entry b: w[b] = 1 when not balancing, else mean power of all
// targets / (power of entry b's target + floor * mean power), so that every
// crop counts alike whatever the size of its corrections.  One block of 64
// threads; thread b sums entry b's partials in order.
__global__ void sample_weight_kernel(const double *__restrict__ part, int n, int s, int balance, float floor_frac,
                                     float *__restrict__ w) {
    __shared__ double pw[64];
    const long long per = (long long)s * s * s;
    const int b = threadIdx.x;
    if (b < n) {
        double sum = 0.0;
        for (int x = 0; x < kPowBlocks; ++x) sum += part[b * kPowBlocks + x];
        pw[b] = sum / (per * 5.0);
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double mean = 0.0;
        for (int i = 0; i < n; ++i) mean += pw[i];
        mean /= n;
        for (int i = 0; i < n; ++i)
            w[i] = balance && mean > 0.0 ? (float)(mean / (pw[i] + floor_frac * mean)) : 1.0f;
    }
}

// I: the index type, 32-bit whenever the batch's cells fit (divisions by
// the crop extent are then 32-bit).
template <class I>
__global__ void flux_residual_kernel(const float *__restrict__ out, const float *__restrict__ tgt, int n, int s,
                                     float scale, const float *__restrict__ wsample, float *__restrict__ gbuf,
                                     double *part) {
    __shared__ double red[32];
    const I total = (I)n * s * s * s;
    const int o = s + 1;
    double acc = 0.0;
    for (I v = blockIdx.x * (I)blockDim.x + threadIdx.x; v < total; v += (I)gridDim.x * blockDim.x) {
        I r = v;
        const int iz = r % s; r /= s;
        const int iy = r % s; r /= s;
        const int ix = r % s;
        const int b = (int)(r / s);
        const long long c0 = ((((long long)b * o + ix + 1) * o + iy + 1) * o + iz + 1) * kIO;
        const long long lo[3] = {c0 - (long long)o * o * kIO, c0 - (long long)o * kIO, c0 - kIO};
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            float du = 0.0f;
#pragma unroll
            for (int d = 0; d < 3; ++d) du += out[c0 + 5 * d + c] - out[lo[d] + 5 * d + c];
            const float res = du - tgt[(size_t)v * kIO + c];
            const float wb = wsample[b];
            acc += (double)wb * res * res;
            gbuf[(size_t)v * 5 + c] = scale * wb * res;
        }
    }
#pragma unroll
    for (int sh = 16; sh > 0; sh >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, sh);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double sum = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i) sum += red[i];
        part[blockIdx.x] = sum;
    }
}

// Flux-form loss, pass 2: dL/dF_{d,c}(q) = g_c(q-1) - g_c(q-1+e_d) (terms whose
// target cell lies outside the target are absent), as BF16 into the interior
// of the output-gradient buffer padded by 2; channel 15 is zero.
template <class I>
__global__ void flux_grad_kernel(const float *__restrict__ gbuf, int n, int s, __nv_bfloat16 *__restrict__ dz) {
    const int o = s + 1;
    const I total = (I)n * o * o * o;
    for (I v = blockIdx.x * (I)blockDim.x + threadIdx.x; v < total; v += (I)gridDim.x * blockDim.x) {
        I r = v;
        const int qz = r % o; r /= o;
        const int qy = r % o; r /= o;
        const int qx = r % o;
        const int b = (int)(r / o);
        auto gat = [&](int tx, int ty, int tz, int c) -> float {
            if (tx < 0 || ty < 0 || tz < 0 || tx >= s || ty >= s || tz >= s) return 0.0f;
            return gbuf[((((long long)b * s + tx) * s + ty) * s + tz) * 5 + c];
        };
        float g[kIO];
#pragma unroll
        for (int c = 0; c < 5; ++c) {
            const float self = gat(qx - 1, qy - 1, qz - 1, c);
            g[c] = self - gat(qx, qy - 1, qz - 1, c);
            g[5 + c] = self - gat(qx - 1, qy, qz - 1, c);
            g[10 + c] = self - gat(qx - 1, qy - 1, qz, c);
        }
        g[15] = 0.0f;
        const long long d = ((((long long)b * (o + 4) + qx + 2) * (o + 4) + qy + 2) * (o + 4) + qz + 2) * kIO;
        store_bf16(dz + d, g, kIO);
    }
}

__global__ void adam_kernel(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                            float *__restrict__ v, int count, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < count; i += gridDim.x * blockDim.x) {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.0f - b1) * gi;
        const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
        m[i] = mi;
        v[i] = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
    }
}

// Unpadded copy of the interior of a BF16 tensor padded by 2 (test access).
__global__ void unpad_kernel(const __nv_bfloat16 *__restrict__ src, __nv_bfloat16 *__restrict__ dst, int n, int x,
                             int y, int z, int c) {
    const long long total = (long long)n * x * y * z * c;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < total;
         i += (long long)gridDim.x * blockDim.x) {
        long long r = i;
        const int ic = r % c; r /= c;
        const int iz = r % z; r /= z;
        const int iy = r % y; r /= y;
        const int ix = r % x;
        const int b = (int)(r / x);
        dst[i] = src[((((long long)b * (x + 4) + ix + 2) * (y + 4) + iy + 2) * (z + 4) + iz + 2) * c + ic];
    }
}

// ---------------------------------------------------------------------------
// Launch helpers
// ---------------------------------------------------------------------------
template <int CIN, int COUT, int EPI>
cudaError_t launch_conv(dg_net *net, const void *in, int nb, int xi, int yi, int zi, const __nv_bfloat16 *w,
                        ConvArgs a, cudaStream_t st) {
    using L = ConvSmem<CIN, COUT>;
    auto kern = conv_fwd_kernel<CIN, COUT, EPI>;
    static std::atomic<unsigned long long> attr_set{0};
    const cudaError_t attr_err = ensure_dynamic_smem(kern, L::BYTES, attr_set);
    if (attr_err != cudaSuccess) return attr_err;
    CUtensorMap m;
    if (!map_conv_input(&m, in, CIN, nb, xi, yi, zi)) return cudaErrorInvalidValue;
    a.nb = nb;
    a.xi = xi; a.yi = yi; a.zi = zi;
    a.xo = xi - 2; a.yo = yi - 2; a.zo = zi - 2;
    a.tpp = (a.yo * zi + kM - 1) / kM;
    // blocks holding all 512 TMEM columns cannot share an SM
    const int per_sm = 1;
    const int slots = per_sm * net->nsm;
    // longest x chunk (fewest re-loaded planes) that still gives every block
    // a few work units
    a.xchunk = 8;
    for (int len : {64, 32, 16}) {
        const long long units = (long long)nb * a.tpp * ((a.xo + len - 1) / len);
        if (units >= 4LL * slots) {
            a.xchunk = len;
            break;
        }
    }
    a.nxc = (a.xo + a.xchunk - 1) / a.xchunk;
    a.nunits = nb * a.tpp * a.nxc;
    a.status = net->status;
    const int grid = std::max(1, std::min(a.nunits, slots));
    kern<<<grid, kFwdThreads, L::BYTES, st>>>(m, w, a);
    return cudaGetLastError();
}

template <int CIN, int COUT>
cudaError_t launch_wgrad(dg_net *net, const void *x_in, const void *g_pad, int nb, int xo, int yo, int zo, float *gw,
                         float *gb) {
    using L = WgradSmem<CIN, COUT>;
    auto kern = conv_wgrad_kernel<CIN, COUT>;
    static std::atomic<unsigned long long> attr_set{0};
    const cudaError_t attr_err = ensure_dynamic_smem(kern, L::BYTES, attr_set);
    if (attr_err != cudaSuccess) return attr_err;
    CUtensorMap mx, mg;
    if (!map_wgrad(&mx, x_in, CIN, nb, xo + 2, yo + 2, zo + 2, kWz, 1)) return cudaErrorInvalidValue;
    if (!map_wgrad(&mg, g_pad, COUT, nb, xo + 4, yo + 4, zo + 4, kM, 1)) return cudaErrorInvalidValue;
    WgradArgs a;
    a.nb = nb; a.xo = xo; a.yo = yo; a.zo = zo;
    a.nseg = (zo + kM - 1) / kM;
    // columns along y split into chunks so that every block gets ~6 units
    const long long cols = (long long)nb * xo * a.nseg;
    const long long want = 6LL * net->nsm;
    int nyc = (int)std::min<long long>(yo, std::max<long long>(1, (want + cols - 1) / cols));
    a.ych = (yo + nyc - 1) / nyc;
    a.nyc = (yo + a.ych - 1) / a.ych;
    a.nunits = (int)(cols * a.nyc);
    a.part = net->wpart;
    a.status = net->status;
    const int grid = std::max(1, std::min(a.nunits, net->nsm));
    kern<<<grid, kConvThreads, L::BYTES, net->stream>>>(mx, mg, a);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    wgrad_reduce_kernel<<<64, 256, 0, net->stream>>>(net->wpart, grid, CIN, COUT, gw, gb);
    return cudaGetLastError();
}

int repack(dg_net *net) {
    for (int l = 0; l < 4; ++l) {
        pack_kernel<<<64, 256, 0, net->stream>>>(net->w[l], net->wf[l], kCin[l], kCout[l], 0);
        if (l > 0) pack_kernel<<<64, 256, 0, net->stream>>>(net->w[l], net->wd[l], kCin[l], kCout[l], 1);
    }
    NET_CUDA(net, cudaGetLastError());
    return DG_OK;
}

void free_ws(Workspace &ws) {
    for (int i = 0; i < 3; ++i) {
        cudaFree(ws.act[i]);
        cudaFree(ws.pre[i]);
        ws.act[i] = ws.pre[i] = nullptr;
    }
    for (int i = 0; i < 4; ++i) {
        cudaFree(ws.dz[i]);
        ws.dz[i] = nullptr;
    }
    cudaFree(ws.out);
    ws.out = nullptr;
    cudaFree(ws.gbuf);
    ws.gbuf = nullptr;
    ws.gbuf_elems = 0;
    ws.n = 0;
}

int ensure_ws(dg_net *net, int n, int x, int y, int z, bool train) {
    Workspace &ws = net->ws;
    if (ws.n == n && ws.x == x && ws.y == y && ws.z == z && (ws.train || !train)) return DG_OK;
    // the workspace may be in use on any stream (the corrector runs the
    // network on its grid's stream)
    NET_CUDA(net, cudaDeviceSynchronize());
    free_ws(ws);
    for (int l = 0; l < 3; ++l) {
        const size_t e = (size_t)n * (x - 2 * (l + 1)) * (y - 2 * (l + 1)) * (z - 2 * (l + 1));
        ws.act_bytes[l] = e * kH * 2;
        NET_CUDA(net, cudaMalloc(&ws.act[l], ws.act_bytes[l]));
        if (train) NET_CUDA(net, cudaMalloc(&ws.pre[l], ws.act_bytes[l]));
    }
    if (train) {
        const size_t eo = (size_t)n * (x - 8) * (y - 8) * (z - 8);
        ws.out_bytes = eo * kIO * 4;
        NET_CUDA(net, cudaMalloc(&ws.out, ws.out_bytes));
        for (int l = 0; l < 4; ++l) {
            // gradient w.r.t. the output of layer l (extent x - 2(l+1)), padded by 2
            const int k = 2 * (l + 1);
            const size_t e = (size_t)n * (x - k + 4) * (y - k + 4) * (z - k + 4);
            ws.dz_bytes[l] = e * kCout[l] * 2;
            NET_CUDA(net, cudaMalloc(&ws.dz[l], ws.dz_bytes[l]));
            NET_CUDA(net, cudaMemsetAsync(ws.dz[l], 0, ws.dz_bytes[l], net->stream));
        }
    }
    ws.n = n; ws.x = x; ws.y = y; ws.z = z;
    ws.train = train;
    return DG_OK;
}

int check_status(dg_net *net) {
    unsigned st = 0;
    NET_CUDA(net, cudaMemcpyAsync(&st, net->status, sizeof(st), cudaMemcpyDeviceToHost, net->stream));
    NET_CUDA(net, cudaStreamSynchronize(net->stream));
    if (st & kNetTimeout) return fail(net, DG_ERR_TIMEOUT, "a device-side wait timed out; results invalid");
    return DG_OK;
}

uint64_t splitmix(uint64_t &s) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

int check_extents(dg_net *net, int n, int x, int y, int z) {
    if (n < 1 || x < 9 || y < 9 || z < 9)
        return fail(net, DG_ERR_INVALID, "input extents must be at least 9 per axis and n >= 1");
    if ((long long)(y - 2) * z >= (1LL << 31) / 2 || (long long)n * x * y * z >= (1LL << 40))
        return fail(net, DG_ERR_INVALID, "input too large");
    return DG_OK;
}

// Forward pass on stream st; stores pre-activations when train is set.
int forward(dg_net *net, const void *feat, int n, int x, int y, int z, float *out, bool train, cudaStream_t st) {
    Workspace &ws = net->ws;
    cudaError_t e;
    const void *in = feat;
    int xi = x, yi = y, zi = z;
    for (int l = 0; l < 3; ++l) {
        ConvArgs a{};
        a.ox = xi - 2; a.oy = yi - 2; a.oz = zi - 2; a.off = 0;
        a.bias = net->b[l];
        a.out_a = ws.act[l];
        a.out_z = train ? ws.pre[l] : nullptr;
        if (l == 0) e = launch_conv<kIO, kH, kEpiGelu>(net, in, n, xi, yi, zi, net->wf[l], a, st);
        else e = launch_conv<kH, kH, kEpiGelu>(net, in, n, xi, yi, zi, net->wf[l], a, st);
        if (e != cudaSuccess) return fail(net, DG_ERR_CUDA, std::string("conv launch: ") + cudaGetErrorString(e));
        in = ws.act[l];
        xi -= 2; yi -= 2; zi -= 2;
    }
    ConvArgs a{};
    a.ox = xi - 2; a.oy = yi - 2; a.oz = zi - 2; a.off = 0;
    a.bias = net->b[3];
    a.out_f = out;
    e = launch_conv<kH, kIO, kEpiLinear>(net, in, n, xi, yi, zi, net->wf[3], a, st);
    if (e != cudaSuccess) return fail(net, DG_ERR_CUDA, std::string("conv launch: ") + cudaGetErrorString(e));
    return DG_OK;
}

// Backward pass from the output gradient in ws.dz[3] down to the weights of
// layer 0 (weight gradients of every layer, input gradients of layers 1-3).
int backward(dg_net *net, const void *feat, int n, int x, int y, int z) {
    Workspace &ws = net->ws;
    cudaError_t e;
    for (int l = 3; l >= 0; --l) {
        const int k = 2 * (l + 1);
        const int ex = x - k, ey = y - k, ez = z - k;        // extents of layer l's output
        const void *xin = l == 0 ? feat : ws.act[l - 1];
        if (l == 3) e = launch_wgrad<kH, kIO>(net, xin, ws.dz[l], n, ex, ey, ez, net->gw[l], net->gb[l]);
        else if (l == 0) e = launch_wgrad<kIO, kH>(net, xin, ws.dz[l], n, ex, ey, ez, net->gw[l], net->gb[l]);
        else e = launch_wgrad<kH, kH>(net, xin, ws.dz[l], n, ex, ey, ez, net->gw[l], net->gb[l]);
        if (e != cudaSuccess) return fail(net, DG_ERR_CUDA, std::string("wgrad launch: ") + cudaGetErrorString(e));
        if (l == 0) break;
        // gradient w.r.t. the pre-activation of layer l-1 (extent ex+2), into its padded buffer
        ConvArgs a{};
        a.ox = ex + 2 + 4; a.oy = ey + 2 + 4; a.oz = ez + 2 + 4; a.off = 2;
        a.out_a = ws.dz[l - 1];
        a.zsrc = ws.pre[l - 1];
        if (l == 3) e = launch_conv<kIO, kH, kEpiDGelu>(net, ws.dz[l], n, ex + 4, ey + 4, ez + 4, net->wd[l], a,
                                                        net->stream);
        else e = launch_conv<kH, kH, kEpiDGelu>(net, ws.dz[l], n, ex + 4, ey + 4, ez + 4, net->wd[l], a,
                                                net->stream);
        if (e != cudaSuccess) return fail(net, DG_ERR_CUDA, std::string("dgrad launch: ") + cudaGetErrorString(e));
    }
    return DG_OK;
}

}  // namespace

// Entry points for the other sources of the library (dg_net_impl.h).
int dg::net_forward_stream(dg_net *net, const void *feat, int n, int x, int y, int z, float *out, cudaStream_t st) {
    if (int r = check_extents(net, n, x, y, z)) return r;
    if (int r = ensure_ws(net, n, x, y, z, false)) return r;
    return forward(net, feat, n, x, y, z, out, false, st);
}

int dg::net_inputs(const dg_net *net) { return net->inputs; }
int dg::net_device(const dg_net *net) { return net->device; }
int dg::net_outputs(const dg_net *net) { return net->outputs; }
unsigned *dg::net_status(dg_net *net) { return net->status; }
const char *dg::net_error(const dg_net *net) { return net->err.c_str(); }

extern "C" {

int32_t dg_net_create(const dg_net_info *info, dg_net **out) {
    if (!info || !out) return fail(nullptr, DG_ERR_INVALID, "null argument");
    *out = nullptr;
    if (info->inputs < 1 || info->inputs > kIO || info->outputs < 1 || info->outputs > kIO)
        return fail(nullptr, DG_ERR_INVALID, "inputs and outputs must be in 1..16");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(nullptr, DG_ERR_NO_DEVICE, "no CUDA device");
    if (info->device < 0 || info->device >= ndev) return fail(nullptr, DG_ERR_INVALID, "bad device ordinal");
    if (cudaSetDevice(info->device) != cudaSuccess) return fail(nullptr, DG_ERR_NO_DEVICE, "cannot select device");
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, info->device) != cudaSuccess || prop.major != 10)
        return fail(nullptr, DG_ERR_NO_DEVICE, "the network kernels need an sm_100 GPU");
    dg_net *net = new dg_net();
    net->device = info->device;
    net->inputs = info->inputs;
    net->outputs = info->outputs;
    net->nsm = prop.multiProcessorCount;
    auto bail = [&](int code) {
        dg_net_destroy(net);
        return code;
    };
    auto cu = [&](cudaError_t e, const char *what) {
        if (e != cudaSuccess) {
            fail(nullptr, DG_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
            return false;
        }
        return true;
    };
    if (!cu(cudaStreamCreateWithFlags(&net->stream, cudaStreamNonBlocking), "stream")) return bail(DG_ERR_CUDA);
    size_t maxrow = 0;
    for (int l = 0; l < 4; ++l) {
        const size_t nw = (size_t)27 * kCin[l] * kCout[l], nb = kCout[l];
        maxrow = std::max(maxrow, nw + nb);
        float **fl[] = {&net->w[l], &net->gw[l], &net->mw[l], &net->vw[l]};
        for (auto p : fl)
            if (!cu(cudaMalloc(p, nw * 4), "cudaMalloc") || !cu(cudaMemset(*p, 0, nw * 4), "memset"))
                return bail(DG_ERR_CUDA);
        float **fb[] = {&net->b[l], &net->gb[l], &net->mb[l], &net->vb[l]};
        for (auto p : fb)
            if (!cu(cudaMalloc(p, nb * 4), "cudaMalloc") || !cu(cudaMemset(*p, 0, nb * 4), "memset"))
                return bail(DG_ERR_CUDA);
        if (!cu(cudaMalloc(&net->wf[l], nw * 2), "cudaMalloc")) return bail(DG_ERR_CUDA);
        if (l > 0 && !cu(cudaMalloc(&net->wd[l], nw * 2), "cudaMalloc")) return bail(DG_ERR_CUDA);
    }
    if (!cu(cudaMalloc(&net->wpart, maxrow * net->nsm * 4), "cudaMalloc")) return bail(DG_ERR_CUDA);
    if (!cu(cudaMalloc(&net->loss_part, 4096 * sizeof(double)), "cudaMalloc")) return bail(DG_ERR_CUDA);
    if (!cu(cudaMalloc(&net->pow_part, 64 * kPowBlocks * sizeof(double)), "cudaMalloc")) return bail(DG_ERR_CUDA);
    if (!cu(cudaMalloc(&net->status, sizeof(unsigned)), "cudaMalloc") ||
        !cu(cudaMemset(net->status, 0, sizeof(unsigned)), "memset"))
        return bail(DG_ERR_CUDA);
    // Seeded initialisation: uniform with the variance of He initialisation
    // (GELU layers), the last layer scaled by out_scale; biases zero.
    uint64_t s = info->seed;
    for (int l = 0; l < 4; ++l) {
        const int ci_real = l == 0 ? info->inputs : kH, co_real = l == 3 ? info->outputs : kH;
        std::vector<float> w((size_t)27 * kCin[l] * kCout[l], 0.0f);
        const double bound = std::sqrt(6.0 / (27.0 * ci_real)) * (l == 3 ? info->out_scale : 1.0);
        for (int co = 0; co < co_real; ++co)
            for (int ci = 0; ci < ci_real; ++ci)
                for (int t = 0; t < 27; ++t) {
                    const double u = (double)(splitmix(s) >> 11) * (1.0 / 9007199254740992.0);
                    w[((size_t)co * kCin[l] + ci) * 27 + t] = (float)((2.0 * u - 1.0) * bound);
                }
        if (!cu(cudaMemcpy(net->w[l], w.data(), w.size() * 4, cudaMemcpyHostToDevice), "upload"))
            return bail(DG_ERR_CUDA);
    }
    if (repack(net) != DG_OK || !cu(cudaStreamSynchronize(net->stream), "init")) return bail(DG_ERR_CUDA);
    *out = net;
    return DG_OK;
}

int32_t dg_net_destroy(dg_net *net) {
    if (!net) return DG_OK;
    cudaSetDevice(net->device);
    if (net->stream) cudaStreamSynchronize(net->stream);
    free_ws(net->ws);
    for (int l = 0; l < 4; ++l) {
        float *ps[] = {net->w[l], net->b[l], net->gw[l], net->gb[l], net->mw[l], net->vw[l], net->mb[l], net->vb[l]};
        for (auto p : ps) cudaFree(p);
        cudaFree(net->wf[l]);
        cudaFree(net->wd[l]);
    }
    cudaFree(net->wpart);
    cudaFree(net->loss_part);
    cudaFree(net->pow_part);
    cudaFree(net->status);
    if (net->stream) cudaStreamDestroy(net->stream);
    delete net;
    return DG_OK;
}

static int layer_dims(dg_net *net, int layer, int *ci_real, int *co_real) {
    if (layer < 0 || layer > 3) return fail(net, DG_ERR_INVALID, "layer must be 0..3");
    *ci_real = layer == 0 ? net->inputs : kH;
    *co_real = layer == 3 ? net->outputs : kH;
    return DG_OK;
}

int32_t dg_net_set_layer(dg_net *net, int32_t layer, const float *w, const float *b) {
    if (!net || !w || !b) return fail(net, DG_ERR_INVALID, "null argument");
    int cr, orl;
    if (int r = layer_dims(net, layer, &cr, &orl)) return r;
    NET_CUDA(net, cudaSetDevice(net->device));
    std::vector<float> wp((size_t)27 * kCin[layer] * kCout[layer], 0.0f), bp(kCout[layer], 0.0f);
    for (int co = 0; co < orl; ++co) {
        bp[co] = b[co];
        for (int ci = 0; ci < cr; ++ci)
            for (int t = 0; t < 27; ++t) wp[((size_t)co * kCin[layer] + ci) * 27 + t] = w[((size_t)co * cr + ci) * 27 + t];
    }
    NET_CUDA(net, cudaStreamSynchronize(net->stream));
    NET_CUDA(net, cudaMemcpy(net->w[layer], wp.data(), wp.size() * 4, cudaMemcpyHostToDevice));
    NET_CUDA(net, cudaMemcpy(net->b[layer], bp.data(), bp.size() * 4, cudaMemcpyHostToDevice));
    if (int r = repack(net)) return r;
    NET_CUDA(net, cudaStreamSynchronize(net->stream));
    return DG_OK;
}

static int get_pair(dg_net *net, int layer, const float *dw, const float *db, float *w, float *b) {
    int cr, orl;
    if (int r = layer_dims(net, layer, &cr, &orl)) return r;
    NET_CUDA(net, cudaSetDevice(net->device));
    NET_CUDA(net, cudaStreamSynchronize(net->stream));
    std::vector<float> wp((size_t)27 * kCin[layer] * kCout[layer]), bp(kCout[layer]);
    NET_CUDA(net, cudaMemcpy(wp.data(), dw, wp.size() * 4, cudaMemcpyDeviceToHost));
    NET_CUDA(net, cudaMemcpy(bp.data(), db, bp.size() * 4, cudaMemcpyDeviceToHost));
    for (int co = 0; co < orl; ++co) {
        if (b) b[co] = bp[co];
        if (w)
            for (int ci = 0; ci < cr; ++ci)
                for (int t = 0; t < 27; ++t) w[((size_t)co * cr + ci) * 27 + t] = wp[((size_t)co * kCin[layer] + ci) * 27 + t];
    }
    return DG_OK;
}

int32_t dg_net_get_layer(dg_net *net, int32_t layer, float *w, float *b) {
    if (!net) return fail(net, DG_ERR_INVALID, "null argument");
    if (layer < 0 || layer > 3) return fail(net, DG_ERR_INVALID, "layer must be 0..3");
    return get_pair(net, layer, net->w[layer], net->b[layer], w, b);
}

int32_t dg_net_get_grad(dg_net *net, int32_t layer, float *gw, float *gb) {
    if (!net) return fail(net, DG_ERR_INVALID, "null argument");
    if (layer < 0 || layer > 3) return fail(net, DG_ERR_INVALID, "layer must be 0..3");
    return get_pair(net, layer, net->gw[layer], net->gb[layer], gw, gb);
}

int32_t dg_net_forward(dg_net *net, const void *feat, int32_t n, int32_t x, int32_t y, int32_t z, float *out) {
    if (!net || !feat || !out) return fail(net, DG_ERR_INVALID, "null argument");
    if (int r = check_extents(net, n, x, y, z)) return r;
    // the output is written with 32-byte stores
    if ((reinterpret_cast<uintptr_t>(feat) & 15) || (reinterpret_cast<uintptr_t>(out) & 31))
        return fail(net, DG_ERR_INVALID, "feat must be 16-byte and out 32-byte aligned");
    NET_CUDA(net, cudaSetDevice(net->device));
    if (int r = ensure_ws(net, n, x, y, z, false)) return r;
    return forward(net, feat, n, x, y, z, out, false, net->stream);
}

int32_t dg_net_forward_backward(dg_net *net, const void *feat, const float *target, int32_t n, int32_t x, int32_t y,
                                int32_t z, double *loss) {
    if (!net || !feat || !target) return fail(net, DG_ERR_INVALID, "null argument");
    if (int r = check_extents(net, n, x, y, z)) return r;
    if ((reinterpret_cast<uintptr_t>(feat) | reinterpret_cast<uintptr_t>(target)) & 15)
        return fail(net, DG_ERR_INVALID, "device pointers must be 16-byte aligned");
    NET_CUDA(net, cudaSetDevice(net->device));
    if (int r = ensure_ws(net, n, x, y, z, true)) return r;
    Workspace &ws = net->ws;
    if (int r = forward(net, feat, n, x, y, z, ws.out, true, net->stream)) return r;
    const int xo = x - 8, yo = y - 8, zo = z - 8;
    const long long nvox = (long long)n * xo * yo * zo;
    const float scale = (float)(2.0 / ((double)nvox * net->outputs));
    const int lblocks = (int)std::min<long long>(4096, (nvox + 255) / 256);
    loss_kernel<<<lblocks, 256, 0, net->stream>>>(ws.out, target, n, xo, yo, zo, net->outputs, scale, ws.dz[3],
                                                  net->loss_part);
    NET_CUDA(net, cudaGetLastError());
    if (int r = backward(net, feat, n, x, y, z)) return r;
    if (int r = check_status(net)) return r;
    if (loss) {
        std::vector<double> part(lblocks);
        NET_CUDA(net, cudaMemcpy(part.data(), net->loss_part, lblocks * sizeof(double), cudaMemcpyDeviceToHost));
        double s = 0.0;
        for (double v : part) s += v;
        *loss = s / ((double)nvox * net->outputs);
    }
    return DG_OK;
}

int32_t dg_net_forward_backward_flux(dg_net *net, const void *feat, const float *target, int32_t n, int32_t x,
                                     int32_t y, int32_t z, int32_t balance, double *loss) {
    if (!net || !feat || !target) return fail(net, DG_ERR_INVALID, "null argument");
    if (n > 64) return fail(net, DG_ERR_INVALID, "at most 64 batch entries");
    if (net->outputs != 15) return fail(net, DG_ERR_INVALID, "the flux form needs a network with 15 outputs");
    if (x != y || y != z) return fail(net, DG_ERR_INVALID, "the flux form takes cubic crops");
    if (int r = check_extents(net, n, x, y, z)) return r;
    if (x < 10) return fail(net, DG_ERR_INVALID, "the flux form needs extents of at least 10");
    if ((reinterpret_cast<uintptr_t>(feat) | reinterpret_cast<uintptr_t>(target)) & 15)
        return fail(net, DG_ERR_INVALID, "device pointers must be 16-byte aligned");
    NET_CUDA(net, cudaSetDevice(net->device));
    if (int r = ensure_ws(net, n, x, y, z, true)) return r;
    Workspace &ws = net->ws;
    const int s = x - 9;                                   // target extent
    const long long ntgt = (long long)n * s * s * s;
    if (ws.gbuf_elems < ntgt * 5) {
        NET_CUDA(net, cudaStreamSynchronize(net->stream));
        cudaFree(ws.gbuf);
        ws.gbuf = nullptr;
        ws.gbuf_elems = 0;
        NET_CUDA(net, cudaMalloc(&ws.gbuf, ntgt * 5 * sizeof(float) + 64 * sizeof(float)));
        ws.gbuf_elems = ntgt * 5;
    }
    ws.wsample = ws.gbuf + ws.gbuf_elems;
    if (int r = forward(net, feat, n, x, y, z, ws.out, true, net->stream)) return r;
    const float scale = (float)(2.0 / ((double)ntgt * 5));
    const int lblocks = (int)std::min<long long>(4096, (ntgt + 255) / 256);
    sample_power_kernel<<<dim3(kPowBlocks, n), 256, 0, net->stream>>>(target, s, net->pow_part);
    sample_weight_kernel<<<1, 64, 0, net->stream>>>(net->pow_part, n, s, balance, 0.01f, ws.wsample);
    if ((long long)n * (s + 1) * (s + 1) * (s + 1) < (1LL << 32)) {
        flux_residual_kernel<unsigned><<<lblocks, 256, 0, net->stream>>>(ws.out, target, n, s, scale, ws.wsample,
                                                                        ws.gbuf, net->loss_part);
        flux_grad_kernel<unsigned><<<1024, 256, 0, net->stream>>>(ws.gbuf, n, s, ws.dz[3]);
    } else {
        flux_residual_kernel<unsigned long long><<<lblocks, 256, 0, net->stream>>>(ws.out, target, n, s, scale,
                                                                                  ws.wsample, ws.gbuf, net->loss_part);
        flux_grad_kernel<unsigned long long><<<1024, 256, 0, net->stream>>>(ws.gbuf, n, s, ws.dz[3]);
    }
    NET_CUDA(net, cudaGetLastError());
    if (int r = backward(net, feat, n, x, y, z)) return r;
    if (int r = check_status(net)) return r;
    if (loss) {
        std::vector<double> part(lblocks);
        NET_CUDA(net, cudaMemcpy(part.data(), net->loss_part, lblocks * sizeof(double), cudaMemcpyDeviceToHost));
        double sum = 0.0;
        for (double v : part) sum += v;
        *loss = sum / ((double)ntgt * 5);
    }
    return DG_OK;
}

int32_t dg_net_adam_step(dg_net *net, float lr, float beta1, float beta2, float eps) {
    if (!net) return fail(net, DG_ERR_INVALID, "null argument");
    NET_CUDA(net, cudaSetDevice(net->device));
    net->adam_t += 1;
    const float c1 = (float)(1.0 - std::pow((double)beta1, (double)net->adam_t));
    const float c2 = (float)(1.0 - std::pow((double)beta2, (double)net->adam_t));
    for (int l = 0; l < 4; ++l) {
        const int nw = 27 * kCin[l] * kCout[l];
        adam_kernel<<<64, 256, 0, net->stream>>>(net->w[l], net->gw[l], net->mw[l], net->vw[l], nw, lr, beta1, beta2,
                                                 eps, c1, c2);
        adam_kernel<<<1, 64, 0, net->stream>>>(net->b[l], net->gb[l], net->mb[l], net->vb[l], kCout[l], lr, beta1,
                                               beta2, eps, c1, c2);
    }
    NET_CUDA(net, cudaGetLastError());
    return repack(net);
}

int32_t dg_net_get_tensor(dg_net *net, int32_t layer, int32_t which, void *host, uint64_t bytes) {
    if (!net || !host) return fail(net, DG_ERR_INVALID, "null argument");
    Workspace &ws = net->ws;
    if (!ws.train || ws.n == 0) return fail(net, DG_ERR_NO_STATE, "no forward_backward has run");
    if (layer < 0 || layer > 3 || which < 0 || which > 3) return fail(net, DG_ERR_INVALID, "bad layer or tensor");
    NET_CUDA(net, cudaSetDevice(net->device));
    NET_CUDA(net, cudaStreamSynchronize(net->stream));
    const int k = 2 * (layer + 1);
    const int ex = ws.x - k, ey = ws.y - k, ez = ws.z - k;
    const size_t count = (size_t)ws.n * ex * ey * ez * kCout[layer];
    if (which == 0 || which == 1) {
        if (layer == 3) return fail(net, DG_ERR_INVALID, "layer 3 has no activation; use which = 2");
        if (bytes < count * 2) return fail(net, DG_ERR_INVALID, "host buffer too small");
        NET_CUDA(net, cudaMemcpy(host, which == 0 ? ws.act[layer] : ws.pre[layer], count * 2, cudaMemcpyDeviceToHost));
    } else if (which == 2) {
        if (layer != 3) return fail(net, DG_ERR_INVALID, "the output belongs to layer 3");
        if (bytes < count * 4) return fail(net, DG_ERR_INVALID, "host buffer too small");
        NET_CUDA(net, cudaMemcpy(host, ws.out, count * 4, cudaMemcpyDeviceToHost));
    } else {
        if (bytes < count * 2) return fail(net, DG_ERR_INVALID, "host buffer too small");
        __nv_bfloat16 *tmp = nullptr;
        NET_CUDA(net, cudaMalloc(&tmp, count * 2));
        unpad_kernel<<<256, 256, 0, net->stream>>>(ws.dz[layer], tmp, ws.n, ex, ey, ez, kCout[layer]);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaMemcpyAsync(host, tmp, count * 2, cudaMemcpyDeviceToHost, net->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(net->stream);
        cudaFree(tmp);
        if (e != cudaSuccess) return fail(net, DG_ERR_CUDA, std::string("get_tensor: ") + cudaGetErrorString(e));
    }
    return DG_OK;
}

int32_t dg_net_synchronize(dg_net *net) {
    if (!net) return fail(net, DG_ERR_INVALID, "null argument");
    NET_CUDA(net, cudaStreamSynchronize(net->stream));
    return check_status(net);
}

void *dg_net_get_stream(dg_net *net) { return net ? net->stream : nullptr; }

const char *dg_net_last_error(const dg_net *net) {
    return net ? net->err.c_str() : g_net_err.c_str();
}

}  // extern "C"
