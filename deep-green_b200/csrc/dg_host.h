// dg_host.h -- host-side helpers shared by the kernel launchers.
#pragma once

#include <cuda_runtime.h>

#include <atomic>

namespace dg {

// cudaFuncSetAttribute acts on the current device, so a kernel's dynamic
// shared-memory limit is raised once per device.  `done` is the caller's
// record for that one kernel: a bit per device ordinal (ordinals past 63 set
// the attribute on every call).  Safe to call from several threads.
template <class Kernel>
inline cudaError_t ensure_dynamic_smem(Kernel kern, int bytes, std::atomic<unsigned long long> &done) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    const unsigned long long bit = dev < 64 ? 1ull << dev : 0ull;
    if (bit && (done.load(std::memory_order_acquire) & bit)) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
    if (e == cudaSuccess) done.fetch_or(bit, std::memory_order_release);
    return e;
}

}  // namespace dg
