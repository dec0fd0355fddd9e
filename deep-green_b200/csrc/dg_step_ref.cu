// dg_step_ref.cu -- the reference-rounding policy (FP64, and FP32 on
// request).  This file is compiled with --fmad=false so that no multiply-add
// is fused and every operation rounds as in the reference's scalar code.
// Also holds the set-up kernels that must round like the reference
// (calc_conserved) and the ghost fill.  Kernels: dg_step_impl.cuh.
#include "dg_step_impl.cuh"

namespace dg {

template <class T> cudaError_t launch_fill_ghosts(const GridArgs<T> &a, T *buf, cudaStream_t st) {
    const long long ghosts = (long long)a.nx * a.ny * a.nz - (long long)(a.nx - 4) * (a.ny - 4) * (a.nz - 4);
    fill_ghosts_kernel<T><<<flat_blocks(ghosts), 256, 0, st>>>(a, buf);
    return cudaGetLastError();
}

template <class T>
cudaError_t launch_prim_to_cons(const GridArgs<T> &a, const T *prim, long long pfs, int ppitch, T *cons,
                                cudaStream_t st) {
    prim_to_cons_kernel<T><<<flat_blocks((long long)a.nx * a.ny * a.nz), 256, 0, st>>>(a, prim, pfs, ppitch, cons);
    return cudaGetLastError();
}

#define DG_REF_INSTANTIATE(T)                                                                                      \
    template cudaError_t launch_step_policy<T, true>(const GridArgs<T> &, const CUtensorMap *, int, int,            \
                                                     cudaStream_t);                                                \
    template cudaError_t launch_reduce_policy<T, true>(const GridArgs<T> &, int, cudaStream_t);                     \
    template cudaError_t launch_cons_to_prim_policy<T, true>(const GridArgs<T> &, const T *, T *, long long, int,   \
                                                             cudaStream_t);                                        \
    template cudaError_t launch_fill_ghosts<T>(const GridArgs<T> &, T *, cudaStream_t);                            \
    template cudaError_t launch_prim_to_cons<T>(const GridArgs<T> &, const T *, long long, int, T *, cudaStream_t);

DG_REF_INSTANTIATE(float)
DG_REF_INSTANTIATE(double)

}  // namespace dg
