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

template <class T, int LIM, bool GRAV>
cudaError_t launch_sweep_t(const GridArgs<T> &a, const CUtensorMap *tmap, int chunk, cudaStream_t st) {
    constexpr int TY = SweepCfg<T>::TY, R = SweepCfg<T>::R;
    auto kern = sweep::sweep_step_kernel<T, TY, R, LIM, GRAV>;
    constexpr int smem = sweep::smem_bytes<T, TY, R>();
    static std::atomic<unsigned long long> attr_set{0};
    const cudaError_t e = ensure_dynamic_smem(kern, smem, attr_set);
    if (e != cudaSuccess) return e;
    const int blocks = step_grid_blocks(a.nx, a.ny, a.nz, sizeof(T) == 4 ? kFastF32 : kFastF64, chunk);
    kern<<<blocks, 32 * (TY + 2), smem, st>>>(a, *tmap, chunk);
    return cudaGetLastError();
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
