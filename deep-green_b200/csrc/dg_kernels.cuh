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
    int bc[6];                 // Bc per face (x-, x+, y-, y+, z-, z+)
    int heat;                  // bit a: the lower face of axis a is a conducting wall
    int gravity;
    int limiter;               // 0 central slopes, 1 minmod
    int nparts;                // work items of this grid in a batched launch
    long long wait_budget;     // SM clocks a wait for a staged plane may take (kWaitBudget)
    Consts<T> k;
    DevCtl *ctl;
    Partial *part;
};

// Boundary types of dg_sim_info (DG_BC_*) into the kernels' form.  A
// conducting wall (DG_BC_CONDUCTING_WALL = 3, the reference CUDA variant's
// BC::CONDUCTING_WALL) follows the wall rule for every ghost (kernels.h:327)
// and adds a heat source to the energy flux of its face.  The reference adds
// it at the flux of lower-cell index 1 for a lower face and n - 2 for an
// upper face (kernels.h:561-661): only the lower face's reaches an interior
// cell, so only lower faces set a heat bit.
constexpr int kBcConductingWall = 3;
inline bool valid_bc_pair(int lo, int hi) {
    return lo >= 0 && lo <= kBcConductingWall && hi >= 0 && hi <= kBcConductingWall &&
           (lo == kPeriodic) == (hi == kPeriodic);
}
template <class T> inline void set_boundaries(GridArgs<T> &a, const int32_t bcs[6]) {
    a.heat = 0;
    for (int f = 0; f < 6; ++f) {
        const bool cond = bcs[f] == kBcConductingWall;
        a.bc[f] = cond ? (int)kWall : (int)bcs[f];
        if (cond && (f & 1) == 0) a.heat |= 1 << (f / 2);
    }
}

// SMs of a B200 (2 dies x 74); grid sizes below are multiples of it
constexpr int kSms = 148;
constexpr int kReduceBlocks = kSms * 8;   // grid of the state-reduction kernel

// The step kernels: reference rounding in double and in float
// (dg_step_impl.cuh) and the fused-arithmetic sweep in float and in double
// (dg_sweep_impl.cuh).
enum KernelKind : int { kRefF64 = 0, kRefF32 = 1, kFastF32 = 2, kFastF64 = 3 };

inline bool is_sweep(int kind) { return kind == kFastF32 || kind == kFastF64; }

// Owned tile rows (y) of each kernel.  A sweep block also runs two halo warps.
#ifndef DG_SWEEP_ROWS_F32
#define DG_SWEEP_ROWS_F32 14
#endif
constexpr int kSweepRowsF32 = DG_SWEEP_ROWS_F32;
constexpr int kSweepRowsF64 = 4;
inline int step_tile_rows(int kind) {
    switch (kind) {
        case kRefF64: return 4;
        case kRefF32: return 8;
        case kFastF32: return kSweepRowsF32;
        default: return kSweepRowsF64;
    }
}
// Tile columns (z) and the staged box width (2-cell halo each side).
inline int step_tile_cols(int kind) { return is_sweep(kind) ? 64 : kTZ; }
inline int step_box_cols(int kind) { return step_tile_cols(kind) + 4; }
inline int step_threads(int kind) {
    return is_sweep(kind) ? 32 * (step_tile_rows(kind) + 2) : 32 * step_tile_rows(kind);
}

// Tiles of a sweep step.  Interior tiles are full tiles (rows x cols) at
// least two cells clear of every y and z face, so that no row or column of
// them is on a face or writes a ghost image: they form the rectangle of tile
// rows [1, 1 + ny) x tile columns [1, 1 + nz) (tile row t starts at cell
// 2 + t * rows and needs 2 + (t + 1) * rows <= interior cells); ny = nz = 0
// when either side has none.  The other tiles are the frame.  A step with
// interior tiles is two launches: the interior tiles, one block per tile
// marching all of x, built without the owned warps' boundary switches, and
// the frame in x-chunks (launch_sweep).
struct InteriorTiles {
    int tiles_y, tiles_z, ny, nz;
    __host__ __device__ InteriorTiles(int ghosted_ny, int ghosted_nz, int rows, int cols) {
        const int iy = ghosted_ny - 4, iz = ghosted_nz - 4;
        tiles_y = (iy + rows - 1) / rows;
        tiles_z = (iz + cols - 1) / cols;
        ny = iy >= 2 ? (iy - 2) / rows - 1 : 0;
        nz = iz >= 2 ? (iz - 2) / cols - 1 : 0;
        if (ny <= 0 || nz <= 0) ny = nz = 0;
    }
    __host__ __device__ int interior() const { return ny * nz; }
    __host__ __device__ int frame() const { return tiles_y * tiles_z - ny * nz; }
    // tile of frame index f: the rows outside the rectangle whole, then the
    // rectangle's rows left and right of it
    __host__ __device__ void frame_tile(int f, int &ty, int &tz) const {
        const int full = (tiles_y - ny) * tiles_z;
        if (f < full) {
            const int r = f / tiles_z;
            tz = f % tiles_z;
            ty = r < 1 ? r : r + ny;
        } else {
            const int g = f - full, w = tiles_z - nz;
            ty = 1 + g / w;
            const int c = g % w;
            tz = c < 1 ? c : c + nz;
        }
    }
};

// x-planes per block of a sweep step's interior launch: whole columns when
// the interior tiles alone fill the SMs at least once (the frame's shorter
// blocks then fill the interior launch's last wave), else the frame's chunk
// (a few long blocks would leave most SMs idle).
inline int interior_chunk(int nx, const InteriorTiles &it, int chunk) {
    return it.interior() >= kSms ? nx - 4 : chunk;
}

// Blocks of one step: (y tiles) x (z tiles) x (x chunks of `chunk` planes);
// for a sweep step with interior tiles, the interior tiles x their chunks
// (interior_chunk) plus the frame tiles x chunks (both launches together).
inline int step_grid_blocks(int nx, int ny, int nz, int kind, int chunk) {
    const int ty = step_tile_rows(kind), tzc = step_tile_cols(kind);
    const int chunks = (nx - 4 + chunk - 1) / chunk;
    if (is_sweep(kind)) {
        const InteriorTiles it(ny, nz, ty, tzc);
        const int ci = interior_chunk(nx, it, chunk);
        return it.interior() * ((nx - 4 + ci - 1) / ci) + it.frame() * chunks;
    }
    const int tiles_z = (nz - 4 + tzc - 1) / tzc;
    const int tiles_y = (ny - 4 + ty - 1) / ty;
    return tiles_z * tiles_y * chunks;
}
// Default x-planes per block.  Reference-rounding kernels: enough blocks for
// ~14 waves of resident CTAs (2 per SM), at least 20 planes per block (each
// block re-stages 4 planes at its ends); measured flat within 1 % from 43
// to 74 planes on 512^3.  Sweep kernels (one block per SM): with interior
// tiles, the frame launch's chunk (the interior launch marches whole
// columns); without, the split of x into chunks that minimises waves x
// (planes per block + 3 re-staged), with at least 24 planes per block.
inline int choose_chunk(int nx, int ny, int nz, int kind) {
    const int ty = step_tile_rows(kind), tzc = step_tile_cols(kind);
    // sweep steps whose interior tiles fill the SMs (interior_chunk): the
    // frame's blocks fill the interior launch's last wave, in short chunks
    // (32-64 planes measured 38.2-38.6 GCUPS on 512^3 Sod, whole columns
    // 34.1-34.4)
    if (is_sweep(kind) && InteriorTiles(ny, nz, ty, tzc).interior() >= kSms) return nx - 4 < 64 ? nx - 4 : 64;
    const long long tiles = (long long)((ny - 4 + ty - 1) / ty) * ((nz - 4 + tzc - 1) / tzc);
    const int nxi = nx - 4;
    if (is_sweep(kind)) {
        const int maxc = nxi / 24 > 0 ? nxi / 24 : 1;
        long long best = -1;
        int bestc = 1;
        for (int c = 1; c <= maxc && c <= 64; ++c) {
            const long long per = (nxi + c - 1) / c;
            const long long waves = (tiles * c + kSms - 1) / kSms;
            const long long cost = waves * (per + 3);
            if (best < 0 || cost < best) { best = cost; bestc = c; }
        }
        return (nxi + bestc - 1) / bestc;
    }
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

// The sweep kernel (kFastF32 / kFastF64 contexts); the tensor map's box is
// step_box_cols x (step_tile_rows + 4) x 1 x 5.
cudaError_t launch_sweep(const GridArgs<float> &a, const CUtensorMap *tmap_src, int chunk, cudaStream_t st);
cudaError_t launch_sweep(const GridArgs<double> &a, const CUtensorMap *tmap_src, int chunk, cudaStream_t st);
template <class T> cudaError_t launch_fill_ghosts(const GridArgs<T> &a, T *buf, cudaStream_t st);
template <class T>
cudaError_t launch_prim_to_cons(const GridArgs<T> &a, const T *prim, long long prim_fstride, int prim_pitch, T *cons,
                                cudaStream_t st);

}  // namespace dg
