// Drives the C++ mirror of the reference API (include/deepgreen.hpp) the way
// deep-green's main.rs drives the Rust one: Simulation::new,
// SimulationGrid::new, filling the primitives, calc_conserved, compute_step.
//
//   grid_api validate
//       checks that need no GPU (argument checks, errors as exceptions)
//   grid_api run NX NY NZ DS LIMITER STEPS B0 B1 B2 B3 B4 B5 IN OUT
//       reads the 5 ghosted FP64 primitive fields from IN, runs calc_conserved
//       and STEPS compute_step calls (gamma 1.4, CFL 0.4), writes the STEPS
//       dts and the 5 conserved fields (FP64, C order) to OUT
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "deepgreen.hpp"

using namespace deepgreen;

namespace {

int fail(const char *what) {
    std::fprintf(stderr, "grid_api: %s\n", what);
    return 1;
}

template <class F> bool throws(int32_t code, const char *needle, F f) {
    try {
        f();
    } catch (const Error &e) {
        return e.code == code && std::strstr(e.what(), needle) != nullptr;
    }
    return false;
}

int validate() {
    const std::array<BoundaryType, 6> outflow{BoundaryType::OUTFLOW, BoundaryType::OUTFLOW, BoundaryType::OUTFLOW,
                                              BoundaryType::OUTFLOW, BoundaryType::OUTFLOW, BoundaryType::OUTFLOW};
    // grid.rs:55-63: a periodic axis needs periodic faces
    if (!throws(DG_ERR_INVALID, "periodic", [&] { Simulation::new_(4, 4, 4, 0.1, outflow, {true, false, false}, 2, false); }))
        return fail("periodic axis with outflow faces accepted");
    const Simulation s = Simulation::new_(4, 3, 2, 0.1, outflow, {false, false, false}, 2, false);
    if (s.nx != 8 || s.ny != 7 || s.nz != 6) return fail("ghosts not added to the sizes");
    if (s.gamma != GAMMA || s.cfl != CFL || s.g != G) return fail("globals.rs defaults not applied");
    // physics.rs:14 asserts nghosts == 2; the library refuses it before any device work
    const Simulation s3 = Simulation::new_(4, 4, 4, 0.1, outflow, {false, false, false}, 3, false);
    if (!throws(DG_ERR_INVALID, "nghosts", [&] { SimulationGrid<double> g(s3); }))
        return fail("nghosts 3 accepted");
    Simulation sp = s;
    sp.bcs[0] = BoundaryType::PERIODIC;   // one periodic face only
    if (!throws(DG_ERR_INVALID, "periodic", [&] { SimulationGrid<float> g(sp); }))
        return fail("unpaired periodic face accepted");
    std::printf("validate ok\n");
    return 0;
}

int run(int argc, char **argv) {
    if (argc != 16) return fail("run needs 14 arguments");
    const std::size_t nx = std::strtoul(argv[2], nullptr, 10), ny = std::strtoul(argv[3], nullptr, 10),
                      nz = std::strtoul(argv[4], nullptr, 10);
    const double ds = std::strtod(argv[5], nullptr);
    const int limiter = std::atoi(argv[6]), steps = std::atoi(argv[7]);
    std::array<BoundaryType, 6> bcs{};
    for (int i = 0; i < 6; ++i) bcs[i] = (BoundaryType)std::atoi(argv[8 + i]);
    std::array<bool, 3> per{};
    for (int a = 0; a < 3; ++a) per[a] = bcs[2 * a] == BoundaryType::PERIODIC;
    Simulation sim = Simulation::new_(nx, ny, nz, ds, bcs, per, 2, false);
    sim.gamma = 1.4;
    sim.cfl = 0.4;
    sim.limiter = limiter;

    SimulationGrid<double> grid = SimulationGrid<double>::new_(sim);
    FILE *in = std::fopen(argv[14], "rb");
    if (!in) return fail("cannot open input");
    for (auto *f : grid.primitives().fields())
        if (std::fread(f->data(), sizeof(double), f->v.size(), in) != f->v.size()) return fail("short input");
    std::fclose(in);

    calc_conserved(grid);
    std::vector<double> dts;
    for (int s = 0; s < steps; ++s) {
        double dt = 0.0;
        compute_step(sim, grid, dt);
        dts.push_back(dt);
    }
    FILE *out = std::fopen(argv[15], "wb");
    if (!out) return fail("cannot open output");
    bool ok = std::fwrite(dts.data(), sizeof(double), dts.size(), out) == dts.size();
    for (auto *f : grid.conserved().fields())
        ok = ok && std::fwrite(f->data(), sizeof(double), f->v.size(), out) == f->v.size();
    ok = (std::fclose(out) == 0) && ok;
    return ok ? 0 : fail("write failed");
}

}  // namespace

int main(int argc, char **argv) {
    try {
        if (argc >= 2 && std::string(argv[1]) == "validate") return validate();
        if (argc >= 2 && std::string(argv[1]) == "run") return run(argc, argv);
    } catch (const Error &e) {
        std::fprintf(stderr, "grid_api: error %d: %s\n", e.code, e.what());
        return 2;
    }
    return fail("usage: grid_api validate | run ...");
}
