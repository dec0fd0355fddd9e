// cuda_runtime.h (host shim) -- TEST INFRASTRUCTURE ONLY.
//
// Lets g++ compile the reference's CUDA solver headers (deep-green
// src/cu/include/kernels.h, grid.hpp, matrix3d.hpp) for the host, so that
// its kernels run on the CPU as the checker's pin.  Device memory is host
// memory; a kernel launch is a loop over the launch's threads
// (refcu_host.cpp).  Only what those headers use is declared.
#pragma once
#include <cassert>
#include <cstddef>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <memory>
#include <cstdint>
#include <vector>
#include <ucontext.h>

#define __global__
#define __device__
#define __host__
// One block runs at a time (launch_concurrent), so block-shared arrays are
// function statics.
#define __shared__ static

struct dim3 {
    unsigned int x = 1, y = 1, z = 1;
};

// Launch coordinates of the thread being emulated.
namespace refcu {
inline thread_local dim3 thread_idx, block_idx;
inline dim3 block_dim, grid_dim;
}  // namespace refcu
#define threadIdx (::refcu::thread_idx)
#define blockIdx (::refcu::block_idx)
#define blockDim (::refcu::block_dim)
#define gridDim (::refcu::grid_dim)

// Kernels with block barriers or warp shuffles (reduce_min_kernel) need
// every thread of a block alive at once.  A block's threads run here as
// fibers on one host thread, each switched out at every barrier and shuffle
// and resumed in turn; all other kernels run their threads one after another
// (refcu_host.cpp).
namespace refcu {
struct Fiber {
    ucontext_t ctx;
    std::vector<char> stack;
    bool done = false;
};
struct BlockSync {
    ucontext_t sched;
    std::vector<Fiber> fibers;
    unsigned int current = 0;
    // Barrier generations: a thread waits until the generation it arrived in
    // is over.  Index 0: the block; 1 + w: warp w.
    std::vector<unsigned int> arrived, generation, members;
    std::vector<double> lanes;  // one exchange slot per thread (values widened)
    bool stalled = false;
};
inline BlockSync *sync_state = nullptr;

inline void yield_to_scheduler() {
    BlockSync &s = *sync_state;
    swapcontext(&s.fibers[s.current].ctx, &s.sched);
}

inline void barrier_wait(unsigned int b) {
    BlockSync &s = *sync_state;
    const unsigned int gen = s.generation[b];
    if (++s.arrived[b] == s.members[b]) {
        s.arrived[b] = 0;
        ++s.generation[b];
    }
    while (s.generation[b] == gen) yield_to_scheduler();
}

inline void syncthreads() { barrier_wait(0); }

template <class T> T shfl_down(T v, unsigned int offset) {
    BlockSync &s = *sync_state;
    const unsigned int t = thread_idx.x, lane = t % 32, w = t / 32;
    s.lanes[t] = static_cast<double>(v);
    barrier_wait(1 + w);
    T r = lane + offset < 32 ? static_cast<T>(s.lanes[t + offset]) : v;
    barrier_wait(1 + w);
    return r;
}

template <class F> struct FiberArg {
    F *fn;
    unsigned int t;
};
template <class F> void fiber_entry(unsigned int lo, unsigned int hi) {
    auto *a = reinterpret_cast<FiberArg<F> *>((static_cast<std::uintptr_t>(hi) << 32) | lo);
    thread_idx = dim3{a->t, 0, 0};
    (*a->fn)();
    sync_state->fibers[a->t].done = true;
}

// Runs fn() once per thread of a <<<nb, nt>>> launch, block after block,
// with all threads of a block concurrent as fibers.  A block whose live
// threads all wait at a barrier that the others left without reaching (a
// thread that returned early) is reported instead of waiting for ever.
template <class F> bool launch_concurrent(std::size_t nb, std::size_t nt, F fn) {
    assert(nt % 32 == 0);
    BlockSync s;
    s.fibers.resize(nt);
    s.lanes.assign(nt, 0.0);
    const unsigned int nbar = 1 + static_cast<unsigned int>(nt / 32);
    s.arrived.assign(nbar, 0);
    s.generation.assign(nbar, 0);
    s.members.assign(nbar, 32);
    s.members[0] = static_cast<unsigned int>(nt);
    sync_state = &s;
    block_dim = dim3{static_cast<unsigned int>(nt), 1, 1};
    grid_dim = dim3{static_cast<unsigned int>(nb), 1, 1};
    std::vector<FiberArg<F>> args(nt);
    for (std::size_t b = 0; b < nb && !s.stalled; ++b) {
        block_idx = dim3{static_cast<unsigned int>(b), 0, 0};
        for (std::size_t t = 0; t < nt; ++t) {
            Fiber &f = s.fibers[t];
            f.done = false;
            f.stack.resize(256 * 1024);
            getcontext(&f.ctx);
            f.ctx.uc_stack.ss_sp = f.stack.data();
            f.ctx.uc_stack.ss_size = f.stack.size();
            f.ctx.uc_link = &s.sched;
            args[t] = FiberArg<F>{&fn, static_cast<unsigned int>(t)};
            const auto ptr = reinterpret_cast<std::uintptr_t>(&args[t]);
            makecontext(&f.ctx, reinterpret_cast<void (*)()>(&fiber_entry<F>), 2,
                        static_cast<unsigned int>(ptr & 0xffffffffu), static_cast<unsigned int>(ptr >> 32));
        }
        for (;;) {
            std::size_t live = 0, finished = 0;
            const auto gens = s.generation;
            const auto arr = s.arrived;
            for (std::size_t t = 0; t < nt; ++t) {
                if (s.fibers[t].done) continue;
                ++live;
                s.current = static_cast<unsigned int>(t);
                thread_idx = dim3{static_cast<unsigned int>(t), 0, 0};
                swapcontext(&s.sched, &s.fibers[t].ctx);
                finished += s.fibers[t].done;
            }
            if (live == finished) break;
            if (finished == 0 && gens == s.generation && arr == s.arrived) {
                s.stalled = true;  // no thread advanced in a whole round
                break;
            }
        }
    }
    sync_state = nullptr;
    return !s.stalled;
}

// The form a <<<nb, nt>>> launch takes after the build step's rewrite of
// the launch syntax: launcher{nb, nt}.run(fn, args...).
struct launcher {
    std::size_t nb, nt;
    template <class F, class... A> void run(F fn, A... args) {
        auto body = [&] { fn(args...); };
        if (!launch_concurrent(nb, nt, body)) {
            std::fprintf(stderr, "refcu: a block's threads stopped at a barrier that not all reach\n");
            std::exit(7);
        }
    }
};
}  // namespace refcu
using refcu_launcher = refcu::launcher;

inline void __syncthreads() { refcu::syncthreads(); }
template <class T> T __shfl_down_sync(unsigned int, T v, unsigned int offset) {
    return refcu::shfl_down(v, offset);
}

enum cudaMemcpyKind {
    cudaMemcpyHostToHost = 0,
    cudaMemcpyHostToDevice = 1,
    cudaMemcpyDeviceToHost = 2,
    cudaMemcpyDeviceToDevice = 3
};
typedef int cudaError_t;
typedef void *cudaStream_t;
template <class T> cudaError_t cudaMalloc(T **p, std::size_t n) {
    *p = static_cast<T *>(std::malloc(n));
    return *p ? 0 : 2;
}
inline cudaError_t cudaFree(void *p) { std::free(p); return 0; }
inline cudaError_t cudaMemcpy(void *d, const void *s, std::size_t n, cudaMemcpyKind) {
    std::memcpy(d, s, n);
    return 0;
}
inline cudaError_t cudaMemset(void *d, int v, std::size_t n) { std::memset(d, v, n); return 0; }
inline cudaError_t cudaDeviceSynchronize() { return 0; }
