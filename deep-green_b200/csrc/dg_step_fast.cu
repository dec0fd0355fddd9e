// dg_step_fast.cu -- the fused-arithmetic step (fast policy; multiply-add
// contraction allowed): the sweep kernel in FP32 and FP64, and the fast
// policy's state reduction.  Kernels: dg_sweep_impl.cuh, dg_step_impl.cuh.
#include "dg_host.h"
#include "dg_step_impl.cuh"
#include "dg_sweep_impl.cuh"

namespace dg {

namespace {
template <class T> struct SweepCfg;
template <> struct SweepCfg<float> {
    // five staged planes when they fit in shared memory, else four
    static constexpr int TY = kSweepRowsF32;
    static constexpr int R = sizeof(sweep::Smem<float, TY, 5>) + 1024 <= 232448 ? 5 : 4;
};
template <> struct SweepCfg<double> {
    static constexpr int TY = kSweepRowsF64, R = 4;
};

// One step: with interior tiles (InteriorTiles) two launches sharing one
// reduction -- the interior tiles, with the owned warps' boundary switches
// compiled out (419 instead of 594 instructions per cell), in whole columns
// when they fill the SMs and else in `chunk`-plane blocks
// (interior_chunk), then the frame in `chunk`-plane blocks, launched as a
// programmatic dependent so that it fills the SMs the interior launch's last
// wave leaves free.  Without interior tiles, one launch of the general
// kernel over all tiles.  (One kernel body holding both variants of the
// loop ran slower than either alone.)
template <class T, int LIM, bool GRAV>
cudaError_t launch_sweep_t(const GridArgs<T> &a, const CUtensorMap *tmap, int chunk, cudaStream_t st) {
    constexpr int TY = SweepCfg<T>::TY, R = SweepCfg<T>::R;
    auto k_in = sweep::sweep_step_kernel<T, TY, R, LIM, GRAV, true>;
    auto k_frame = sweep::sweep_step_kernel<T, TY, R, LIM, GRAV, false>;
    constexpr int smem = sweep::smem_bytes<T, TY, R>();
    static std::atomic<unsigned long long> attr_in{0}, attr_frame{0};
    cudaError_t e = ensure_dynamic_smem(k_in, smem, attr_in);
    if (e == cudaSuccess) e = ensure_dynamic_smem(k_frame, smem, attr_frame);
    if (e != cudaSuccess) return e;
    const InteriorTiles it(a.ny, a.nz, TY, sweep::kTileZ);
    const int chunk_in = interior_chunk(a.nx, it, chunk);
    const int n_in = it.interior() * ((a.nx - 4 + chunk_in - 1) / chunk_in);
    const int n_fr = it.frame() * ((a.nx - 4 + chunk - 1) / chunk);
    const int nparts = n_in + n_fr;   // = step_grid_blocks(): the partials' bound
    if (n_in == 0) {
        k_frame<<<n_fr, 32 * (TY + 2), smem, st>>>(a, *tmap, chunk, 0, nparts);
        return cudaGetLastError();
    }
    k_in<<<n_in, 32 * (TY + 2), smem, st>>>(a, *tmap, chunk_in, n_in, nparts);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3((unsigned)n_fr);
    cfg.blockDim = dim3(32 * (TY + 2));
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, k_frame, a, *tmap, chunk, n_in, nparts);
}

// One kernel per (limiter, gravity): the slope and flux code of the march
// is fixed at compile time.
template <class T>
cudaError_t launch_sweep_any(const GridArgs<T> &a, const CUtensorMap *tmap, int chunk, cudaStream_t st) {
    if (a.gravity) {
        return a.limiter == 0 ? launch_sweep_t<T, 0, true>(a, tmap, chunk, st)
                              : launch_sweep_t<T, 1, true>(a, tmap, chunk, st);
    }
    return a.limiter == 0 ? launch_sweep_t<T, 0, false>(a, tmap, chunk, st)
                          : launch_sweep_t<T, 1, false>(a, tmap, chunk, st);
}
}  // namespace

cudaError_t launch_sweep(const GridArgs<float> &a, const CUtensorMap *tmap, int chunk, cudaStream_t st) {
    return launch_sweep_any(a, tmap, chunk, st);
}
cudaError_t launch_sweep(const GridArgs<double> &a, const CUtensorMap *tmap, int chunk, cudaStream_t st) {
    return launch_sweep_any(a, tmap, chunk, st);
}

template cudaError_t launch_reduce_policy<float, false>(const GridArgs<float> &, int, cudaStream_t);
template cudaError_t launch_cons_to_prim_policy<float, false>(const GridArgs<float> &, const float *, float *,
                                                              long long, int, cudaStream_t);
}  // namespace dg
