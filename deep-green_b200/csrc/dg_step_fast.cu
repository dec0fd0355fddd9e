// dg_step_fast.cu -- FP32 step with the fast arithmetic policy (fused
// multiply-add contraction allowed).  Kernels: dg_step_impl.cuh.
#include "dg_step_impl.cuh"

namespace dg {
template cudaError_t launch_step_policy<float, false>(const GridArgs<float> &, const CUtensorMap *, int, int,
                                                      cudaStream_t);
template cudaError_t launch_reduce_policy<float, false>(const GridArgs<float> &, int, cudaStream_t);
template cudaError_t launch_cons_to_prim_policy<float, false>(const GridArgs<float> &, const float *, float *,
                                                              long long, int, cudaStream_t);
}  // namespace dg
