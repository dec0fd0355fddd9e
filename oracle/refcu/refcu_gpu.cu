// refcu_gpu.cu -- the reference's CUDA solver, run and timed on the GPU.
//
// TEST AND MEASUREMENT INFRASTRUCTURE ONLY: the same-box comparator for the
// library's step (bench.py --case refcuda); nothing in the library links it.
//
// Compiles deep-green's src/cu/include/physics.hpp (with kernels.h,
// grid.hpp, matrix3d.hpp and one configuration header, all unchanged,
// read where they lie) with nvcc; only spdlog, HighFive and NVTX, which the
// reference takes from a developer's install, are the no-op stubs of
// stubs/.  The step is the reference's own EULERCFD::compute_step
// (physics.hpp:336-490), the set-up its own init function for the
// configuration's RUN_SETUP (physics.hpp init_khi / init_trb / init_sod /
// init_greenhouse, chosen as eulernv.cu:46-60 chooses), in float as
// eulernv.cu:63 runs it, followed by the initial calc_conserved of
// compute() (physics.hpp:533-537).
//
// calc_timestep's reduce_min_kernel returns early for threads past the
// array before its __syncthreads (kernels.h:88-104); main() refuses a grid
// whose cell count is not a whole number of its 256-thread blocks, so no
// thread of any block does.
//
// Usage: refcu_gpu <warmup> <steps> [state.bin]
//   Prints one JSON line: configuration, interior cells, ms per step (CUDA
//   events around the timed compute_step calls, which synchronise
//   internally), GCUPS over interior cells, every dt.  With state.bin,
//   writes the initial primitives (5 x NX*NY*NZ floats, rho vx vy vz p) and
//   the conserved state after the first step (5 x NX*NY*NZ floats) with
//   that step's dt (one double) first, so a caller can repeat the first step
//   from the same state and compare.
#include "physics.hpp"

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <vector>

using namespace EULERCFD;
using namespace EULERCFD::CONSTS;

namespace {

using T = float;
constexpr GridInfo<T> kInfo{NX, NY, NZ, NGHOSTS, LX, LY, LZ};
using DeviceGrid = Grid<T, kInfo, BACKEND::DEVICE>;

void init(DeviceGrid &g) {
    if constexpr (RUN_SETUP == SETUP::KHI) init_khi<T>(g);
    else if constexpr (RUN_SETUP == SETUP::TRB) init_trb<T>(g);
    else if constexpr (RUN_SETUP == SETUP::GREENHOUSE) init_greenhouse<T>(g);
    else init_sod<T>(g);
}

const char *setup_name() {
    switch (RUN_SETUP) {
        case SETUP::KHI: return "KHI";
        case SETUP::TRB: return "TRB";
        case SETUP::SOD: return "SOD";
        default: return "GREENHOUSE";
    }
}

bool write_fields(FILE *f, std::array<T *, 5> fields, std::size_t n) {
    std::vector<T> host(n);
    for (T *d : fields) {
        if (cudaMemcpy(host.data(), d, n * sizeof(T), cudaMemcpyDeviceToHost) != cudaSuccess) return false;
        if (std::fwrite(host.data(), sizeof(T), n, f) != n) return false;
    }
    return true;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <warmup> <steps> [state.bin]\n", argv[0]);
        return 1;
    }
    const int warmup = std::atoi(argv[1]), steps = std::atoi(argv[2]);
    if (warmup < 1 || steps < 1) return 1;
    constexpr auto lp = launch_params(kInfo.size());
    if (kInfo.size() % lp[1] != 0) {
        std::fprintf(stderr, "grid of %zu cells is not a whole number of %zu-thread blocks\n",
                     kInfo.size(), lp[1]);
        return 2;
    }
    auto g = std::make_unique<DeviceGrid>();
    const std::size_t n = g->size();
    init(*g);
    FILE *state = nullptr;
    if (argc > 3) {
        state = std::fopen(argv[3], "wb");
        if (!state || !write_fields(state, g->get_primitive_pointers(), n)) return 3;
    }
    kernel_calc_conserved<T, kInfo.dv()>
        <<<lp[0], lp[1]>>>(g->get_primitive_pointers(), g->get_conserved_pointers(), g->size());
    if (cudaDeviceSynchronize() != cudaSuccess) return 4;

    T dt = 0.5;  // compute() starts from 0.5; compute_step replaces it
    std::vector<double> dts;
    for (int s = 0; s < warmup; ++s) {
        dt = compute_step<T, kInfo>(*g, dt)[0];
        dts.push_back(dt);
        if (s == 0 && state) {
            const double d0 = dt;
            if (std::fwrite(&d0, sizeof(double), 1, state) != 1) return 3;
            if (!write_fields(state, g->get_conserved_pointers(), n)) return 3;
            std::fclose(state);
            state = nullptr;
        }
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    for (int s = 0; s < steps; ++s) {
        dt = compute_step<T, kInfo>(*g, dt)[0];
        dts.push_back(dt);
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    const cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        std::fprintf(stderr, "CUDA error %s\n", cudaGetErrorString(err));
        return 5;
    }
    const double interior = double(NX - 2 * NGHOSTS) * double(NY - 2 * NGHOSTS) * double(NZ - 2 * NGHOSTS);
    const double ms_step = ms / steps;
    std::printf("{\"setup\": \"%s\", \"NX\": %zu, \"NY\": %zu, \"NZ\": %zu, \"interior_cells\": %.0f, "
                "\"warmup\": %d, \"steps\": %d, \"ms_per_step\": %.6f, \"gcups\": %.6f, \"dts\": [",
                setup_name(), NX, NY, NZ, interior, warmup, steps, ms_step, interior / (ms_step * 1e6));
    for (std::size_t i = 0; i < dts.size(); ++i) std::printf("%s%.9g", i ? ", " : "", dts[i]);
    std::printf("]}\n");
    return 0;
}
