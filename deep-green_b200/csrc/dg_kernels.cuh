// dg_kernels.cuh -- device-side data structures shared by the kernels and
// the C-ABI layer.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "dg_physics.cuh"

namespace dg {

constexpr int kTZ = 32;          // tile width along z (one warp)
constexpr int kRZ = kTZ + 4;     // staged region width along z (2-cell halo)
constexpr int kHist = 4096;      // dt history ring on the device
constexpr unsigned kStatusNonFinite = 0x1u;
constexpr unsigned kStatusTimeout = 0x2u;

// Step control block, one per grid, in device memory.  The step kernel of
// step s reads dt[s & 1] (computed from the state at the start of step s)
// and its last block writes dt[(s + 1) & 1] from the updated state, so dt
// never travels through the host.
struct DevCtl {
    unsigned long long step;   // steps completed since the state was set
    unsigned int counter;      // blocks of the running launch that finished
    unsigned int flags;        // sticky status bits (kStatus*)
    double dt[2];
    double sums[5];            // FP64 interior sums of the current state
    double hist[kHist];        // dt used by step s at hist[s % kHist]
};

// Per-block partial results of a launch, reduced in a fixed order by the
// launch's last block (deterministic sums).
struct Partial {
    double sums[5];
    double wmin;               // min over the block's cells of ds/(c_s+|v|)
    unsigned int nan;
    unsigned int pad;
};

// Geometry and physics of one grid as the kernels see it.
template <class T> struct GridArgs {
    const T *src;              // state read by the step (5 fields)
    T *dst;                    // state written by the step
    int nx, ny, nz;            // ghosted extents (interior + 4)
    int pitch;                 // elements between consecutive z-rows
    long long fstride;         // elements between fields
    int bc[6];
    int gravity;
    int limiter;               // 0 central slopes, 1 minmod
    int nparts;                // work items of this grid in a batched launch
    Consts<T> k;
    DevCtl *ctl;
    Partial *part;
};

// SMs of a B200 (2 dies x 74); grid sizes below are multiples of it
constexpr int kSms = 148;
constexpr int kReduceBlocks = kSms * 8;   // grid of the state-reduction kernel

// The three step kernels: reference rounding in double and in float
// (dg_step_impl.cuh) and the fast float kernel (dg_fast_impl.cuh).
enum KernelKind : int { kRefF64 = 0, kRefF32 = 1, kFastF32 = 2 };

// Warps of the fast kernel; each owns 2 rows of the tile.
constexpr int kFastOwnWarps = 8;

// Tile rows (y) of each kernel; every tile is 32 cells wide in z.
inline int step_tile_rows(int kind) {
    return kind == kRefF64 ? 4 : (kind == kRefF32 ? 8 : 2 * kFastOwnWarps);
}
inline int step_threads(int kind) { return kind == kFastF32 ? 32 * kFastOwnWarps : 32 * step_tile_rows(kind); }

// Blocks of one step launch: (y tiles) x (z tiles) x (x chunks of `chunk`
// planes).
inline int step_grid_blocks(int nx, int ny, int nz, int kind, int chunk) {
    const int ty = step_tile_rows(kind);
    const int tiles_z = (nz - 4 + kTZ - 1) / kTZ;
    const int tiles_y = (ny - 4 + ty - 1) / ty;
    const int chunks = (nx - 4 + chunk - 1) / chunk;
    return tiles_z * tiles_y * chunks;
}
// Default x-planes per block: enough blocks for ~14 waves of resident CTAs
// (2 per SM), at least 20 planes per block (each block re-stages
// 4 planes at its ends).  Measured: flat within 1 % from 43 to 74 planes on
// 512^3; best at 22 planes on 256^3 (5 % faster than 32).
inline int choose_chunk(int nx, int ny, int nz, int kind) {
    const int ty = step_tile_rows(kind);
    const long long tiles = (long long)((ny - 4 + ty - 1) / ty) * ((nz - 4 + kTZ - 1) / kTZ);
    const int nxi = nx - 4;
    const long long target = 2LL * kSms * 14;
    long long chunks = (target + tiles - 1) / tiles;
    const long long maxc = nxi / 20 > 0 ? nxi / 20 : 1;
    if (chunks > maxc) chunks = maxc;
    if (chunks < 1) chunks = 1;
    return (int)((nxi + chunks - 1) / chunks);
}

template <class T> int step_grid_blocks(const GridArgs<T> &a, int chunk) {
    return step_grid_blocks(a.nx, a.ny, a.nz, sizeof(T) == 8 ? kRefF64 : kRefF32, chunk);
}

// Launch helpers.  EXACT selects the reference-rounding policy
// (dg_step_ref.cu, built with --fmad=false) or the fast one
// (dg_step_fast.cu); float/fast, float/exact and double/exact exist.
template <class T, bool EXACT>
cudaError_t launch_step_policy(const GridArgs<T> &a, const CUtensorMap *tmap_src, int limiter, int chunk,
                               cudaStream_t st);
template <class T, bool EXACT> cudaError_t launch_reduce_policy(const GridArgs<T> &a, int set_dt, cudaStream_t st);
template <class T, bool EXACT>
cudaError_t launch_cons_to_prim_policy(const GridArgs<T> &a, const T *cons, T *prim, long long prim_fstride,
                                       int prim_pitch, cudaStream_t st);
// Message returned by dg_last_error(NULL) (errors not tied to a context).
void set_global_error(const std::string &msg);

cudaError_t launch_fast_step(const GridArgs<float> &a, const CUtensorMap *tmap_src, int chunk, cudaStream_t st);
template <class T> cudaError_t launch_fill_ghosts(const GridArgs<T> &a, T *buf, cudaStream_t st);
template <class T>
cudaError_t launch_prim_to_cons(const GridArgs<T> &a, const T *prim, long long prim_fstride, int prim_pitch, T *cons,
                                cudaStream_t st);

}  // namespace dg
