// dg_step_fast.cu -- FP32 step with the fast arithmetic policy (fused
// multiply-add contraction allowed).  Kernels: dg_step_impl.cuh.
#include "dg_fast_impl.cuh"
#include "dg_host.h"
#include "dg_step_impl.cuh"

namespace dg {

namespace {
template <int LIM>
cudaError_t launch_fast_step_t(const GridArgs<float> &a, const CUtensorMap *tmap, int chunk, cudaStream_t st) {
    constexpr int W = kFastOwnWarps, R = 4;
    using Sm = fastk::Smem<W, R>;
    auto kern = fastk::fast_step_kernel<W, R, LIM>;
    const int smem = (int)sizeof(Sm) + 1024;
    static std::atomic<unsigned long long> attr_set{0};
    const cudaError_t e = ensure_dynamic_smem(kern, smem, attr_set);
    if (e != cudaSuccess) return e;
    const int blocks = step_grid_blocks(a.nx, a.ny, a.nz, kFastF32, chunk);
    kern<<<blocks, dim3(32, W), smem, st>>>(a, *tmap, chunk);
    return cudaGetLastError();
}
}  // namespace

// One kernel per limiter: the slope code of the hot loop is fixed at compile
// time.
cudaError_t launch_fast_step(const GridArgs<float> &a, const CUtensorMap *tmap, int chunk, cudaStream_t st) {
    return a.limiter == 0 ? launch_fast_step_t<0>(a, tmap, chunk, st) : launch_fast_step_t<1>(a, tmap, chunk, st);
}
template cudaError_t launch_reduce_policy<float, false>(const GridArgs<float> &, int, cudaStream_t);
template cudaError_t launch_cons_to_prim_policy<float, false>(const GridArgs<float> &, const float *, float *,
                                                              long long, int, cudaStream_t);
}  // namespace dg
