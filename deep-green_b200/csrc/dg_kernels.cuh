// dg_kernels.cuh -- device-side data structures shared by the kernels and
// the C-ABI layer.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>
#include <stdint.h>

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
    Consts<T> k;
    DevCtl *ctl;
    Partial *part;
};

// Launch helpers implemented in dg_step.cu.
template <class T>
cudaError_t launch_step(const GridArgs<T> &a, const CUtensorMap *tmap_src, int limiter, int chunk,
                        cudaStream_t st);
template <class T>
cudaError_t launch_reduce(const GridArgs<T> &a, int set_dt, cudaStream_t st);
template <class T> cudaError_t launch_fill_ghosts(const GridArgs<T> &a, T *buf, cudaStream_t st);
template <class T>
cudaError_t launch_prim_to_cons(const GridArgs<T> &a, const T *prim, long long prim_fstride,
                                int prim_pitch, T *cons, cudaStream_t st);
template <class T>
cudaError_t launch_cons_to_prim(const GridArgs<T> &a, const T *cons, T *prim, long long prim_fstride,
                                int prim_pitch, cudaStream_t st);
template <class T> int step_grid_blocks(const GridArgs<T> &a, int chunk);
int step_tile_rows(bool is_double);

}  // namespace dg
