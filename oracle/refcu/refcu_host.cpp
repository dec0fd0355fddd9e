// refcu_host.cpp -- the reference's CUDA solver kernels, run on the host.
//
// TEST INFRASTRUCTURE ONLY: this program produces golden vectors from the
// reference's own code to pin the oracle against; nothing in the library
// links or runs it.
//
// It compiles deep-green's src/cu/include/kernels.h (with grid.hpp,
// matrix3d.hpp and a configuration header: the reference's constants.h or
// one of its ini_files/*.h, all read where they lie) against the host shim
// in shim/ (device memory = host memory, a launch = a loop over its
// threads).  The only change to the reference's text is the one launch in
// kernels.h's calc_timestep, rewritten by the build from <<<nb, nt>>> syntax
// into a call of refcu_launcher, which runs that reduction with every thread
// of a block alive (barrier, shuffles).  Grid sizes, boundaries, gamma, CFL,
// ds and gravity are the configuration header's compile-time constants.
//
// main() below restates the host-side orchestration that physics.hpp (which
// g++ cannot parse because of its launch syntax) performs:
//   compute():       kernel_calc_conserved once (physics.hpp:525-538)
//   compute_step():  physics.hpp:336-490 -- calc_primitives, apply_boundaries
//                    (the six ghost kernels, physics.hpp:313-332), calc_timestep,
//                    calc_gradients, calc_xtr, calc_fluxes x 3 (with the
//                    argument permutations of physics.hpp:431-455),
//                    calc_addfluxes -- in that order, with the same template
//                    arguments and launch shapes.
//
// Usage:  refcu_host info
//           prints the configuration as JSON
//         refcu_host run <4|8> <nsteps> <in.bin> <out.bin>
//           in.bin:  5 x NX*NY*NZ values (rho, vx, vy, vz, p; ghosts
//                    included, index (i*NY + j)*NZ + k) of the precision;
//           out.bin: nsteps doubles (each step's dt), then 5 x NX*NY*NZ
//                    conserved values (mass, momx, momy, momz, e) after the
//                    last step, in the precision.
#include "kernels.h"

#include <cinttypes>
#include <cstdio>
#include <string>

namespace {

using namespace EULERCFD;
using namespace EULERCFD::CONSTS;

// A <<<nb, nt>>> launch of a kernel without block barriers: every thread
// runs to completion in turn.
template <class F> void launch_each(std::size_t nb, std::size_t nt, F fn) {
    refcu::block_dim = dim3{static_cast<unsigned int>(nt), 1, 1};
    refcu::grid_dim = dim3{static_cast<unsigned int>(nb), 1, 1};
    for (std::size_t b = 0; b < nb; ++b) {
        refcu::block_idx = dim3{static_cast<unsigned int>(b), 0, 0};
        for (std::size_t t = 0; t < nt; ++t) {
            refcu::thread_idx = dim3{static_cast<unsigned int>(t), 0, 0};
            fn();
        }
    }
}

template <class T> using HostGrid =
    Grid<T, GridInfo<T>{NX, NY, NZ, NGHOSTS, LX, LY, LZ}, BACKEND::DEVICE>;

template <class T> void apply_boundaries_host(std::array<T *, 5> src, std::size_t len,
                                              std::array<std::size_t, 2> lp) {
    launch_each(lp[0], lp[1], [&] { kernel_update_ghosts<T, 0, bcs[0], NGHOSTS>(src, len); });
    launch_each(lp[0], lp[1], [&] { kernel_update_ghosts<T, 1, bcs[1], NGHOSTS>(src, len); });
    launch_each(lp[0], lp[1], [&] { kernel_update_ghosts<T, 2, bcs[2], NGHOSTS>(src, len); });
    launch_each(lp[0], lp[1], [&] { kernel_update_ghosts<T, 3, bcs[3], NGHOSTS>(src, len); });
    launch_each(lp[0], lp[1], [&] { kernel_update_ghosts<T, 4, bcs[4], NGHOSTS>(src, len); });
    launch_each(lp[0], lp[1], [&] { kernel_update_ghosts<T, 5, bcs[5], NGHOSTS>(src, len); });
}

template <class T> T step(HostGrid<T> &g) {
    constexpr GridInfo<T> G{NX, NY, NZ, NGHOSTS, LX, LY, LZ};
    constexpr auto lp = launch_params(G.size());
    const std::size_t n = g.size();
    launch_each(lp[0], lp[1], [&] {
        kernel_calc_primitives<T, G.dv()>(g.get_conserved_pointers(), g.get_primitive_pointers(), n);
    });
    apply_boundaries_host<T>(g.get_primitive_pointers(), n, lp);
    const T dt = calc_timestep<T>(g.get_primitive_pointers(), n, lp);
    launch_each(lp[0], lp[1], [&] {
        kernel_calc_gradients<T, G.dsx()>(g.get_primitive_pointers(), g.get_gradients_pointers(), n);
    });
    launch_each(lp[0], lp[1], [&] {
        kernel_calc_xtr<T, G.dsx()>(g.get_primitive_pointers(), g.get_primitive_xtr_pointers(),
                                    g.get_gradients_pointers(), n, dt);
    });
    launch_each(lp[0], lp[1], [&] {
        kernel_calc_fluxes<T, G.dsx()>(g.fmass_x.data(), g.fmomx_x.data(), g.fmomy_x.data(),
                                       g.fmomz_x.data(), g.fe_x.data(), g.drho_x.data(),
                                       g.dvx_x.data(), g.dvy_x.data(), g.dvz_x.data(),
                                       g.dp_x.data(), g.rho_xtr.data(), g.vx_xtr.data(),
                                       g.vy_xtr.data(), g.vz_xtr.data(), g.p_xtr.data(), n,
                                       std::array<std::size_t, 3>{1, 0, 0}, 0);
    });
    launch_each(lp[0], lp[1], [&] {
        kernel_calc_fluxes<T, G.dsx()>(g.fmass_y.data(), g.fmomy_y.data(), g.fmomx_y.data(),
                                       g.fmomz_y.data(), g.fe_y.data(), g.drho_y.data(),
                                       g.dvy_y.data(), g.dvx_y.data(), g.dvz_y.data(),
                                       g.dp_y.data(), g.rho_xtr.data(), g.vy_xtr.data(),
                                       g.vx_xtr.data(), g.vz_xtr.data(), g.p_xtr.data(), n,
                                       std::array<std::size_t, 3>{0, 1, 0}, 1);
    });
    launch_each(lp[0], lp[1], [&] {
        kernel_calc_fluxes<T, G.dsx()>(g.fmass_z.data(), g.fmomz_z.data(), g.fmomx_z.data(),
                                       g.fmomy_z.data(), g.fe_z.data(), g.drho_z.data(),
                                       g.dvz_z.data(), g.dvx_z.data(), g.dvy_z.data(),
                                       g.dp_z.data(), g.rho_xtr.data(), g.vz_xtr.data(),
                                       g.vx_xtr.data(), g.vy_xtr.data(), g.p_xtr.data(), n,
                                       std::array<std::size_t, 3>{0, 0, 1}, 2);
    });
    launch_each(lp[0], lp[1], [&] {
        kernel_calc_addfluxes<T, G.dsx()>(g.get_fluxes_pointers(), g.get_conserved_pointers(), n, dt);
    });
    return dt;
}

template <class T> int run(int nsteps, const char *in_path, const char *out_path) {
    constexpr GridInfo<T> G{NX, NY, NZ, NGHOSTS, LX, LY, LZ};
    constexpr auto lp = launch_params(G.size());
    // calc_timestep's reduction returns early for threads past the array
    // before its block barrier; with the array an exact number of blocks
    // no thread does.
    if (G.size() % lp[1] != 0) {
        std::fprintf(stderr, "grid of %zu cells is not a whole number of %zu-thread blocks\n",
                     G.size(), lp[1]);
        return 2;
    }
    auto g = std::make_unique<HostGrid<T>>();
    const std::size_t n = g->size();
    FILE *in = std::fopen(in_path, "rb");
    if (!in) return 3;
    for (T *p : g->get_primitive_pointers())
        if (std::fread(p, sizeof(T), n, in) != n) { std::fclose(in); return 4; }
    std::fclose(in);
    launch_each(lp[0], lp[1], [&] {
        kernel_calc_conserved<T, G.dv()>(g->get_primitive_pointers(), g->get_conserved_pointers(), n);
    });
    std::vector<double> dts;
    for (int s = 0; s < nsteps; ++s) dts.push_back(static_cast<double>(step<T>(*g)));
    FILE *out = std::fopen(out_path, "wb");
    if (!out) return 5;
    std::fwrite(dts.data(), sizeof(double), dts.size(), out);
    for (T *p : g->get_conserved_pointers()) std::fwrite(p, sizeof(T), n, out);
    std::fclose(out);
    return 0;
}

void print_info() {
    std::printf("{\"NX\": %zu, \"NY\": %zu, \"NZ\": %zu, \"NGHOSTS\": %zu, "
                "\"DELTA\": %.17g, \"GAMMA\": %.17g, \"CFL\": %.17g, \"G\": %.17g, "
                "\"GRAVITY\": %d, \"bcs\": [%d, %d, %d, %d, %d, %d], "
                "\"bc_names\": [\"PERIODIC\", \"WALL\", \"CONDUCTING_WALL\", \"OUTFLOW\"]}\n",
                NX, NY, NZ, NGHOSTS, static_cast<double>(DELTA), static_cast<double>(GAMMA),
                static_cast<double>(CFL), static_cast<double>(EULERCFD::CONSTS::G), GRAVITY ? 1 : 0,
                static_cast<int>(bcs[0]), static_cast<int>(bcs[1]), static_cast<int>(bcs[2]),
                static_cast<int>(bcs[3]), static_cast<int>(bcs[4]), static_cast<int>(bcs[5]));
}

}  // namespace

int main(int argc, char **argv) {
    if (argc >= 2 && std::string(argv[1]) == "info") {
        print_info();
        return 0;
    }
    if (argc != 6 || std::string(argv[1]) != "run") {
        std::fprintf(stderr, "usage: %s info | run <4|8> <nsteps> <in.bin> <out.bin>\n", argv[0]);
        return 1;
    }
    const int prec = std::atoi(argv[2]), nsteps = std::atoi(argv[3]);
    if (nsteps < 0) return 1;
    if (prec == 4) return run<float>(nsteps, argv[4], argv[5]);
    if (prec == 8) return run<double>(nsteps, argv[4], argv[5]);
    return 1;
}
