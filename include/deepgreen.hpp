/*
 * deepgreen.hpp -- C++ mirror of deep-green's Rust grid/state/step API over
 * the C ABI of deepgreen.h (header only, C++17).
 *
 *   reference (src/rs/src/...)               this header
 *   ---------------------------------------  ----------------------------------
 *   BoundaryType            grid.rs:23-28     deepgreen::BoundaryType
 *   Simulation / new        grid.rs:30-76     deepgreen::Simulation / new_
 *   Primitives, Conserved   grid.rs:87-101    deepgreen::Primitives<T>, Conserved<T>
 *   SimulationGrid / new    grid.rs:111-221   deepgreen::SimulationGrid<T> / new_
 *   calc_conserved          physics.rs:143    deepgreen::calc_conserved
 *   compute_step            physics.rs:595    deepgreen::compute_step
 *   globals                 globals.rs:3-8    GAMMA, CFL, G (defaults of Simulation)
 *
 * Same names and argument meaning; two differences.  The state lives in GPU
 * memory: the host arrays of a grid are refreshed from the device when they
 * are read after a step (primitives() holds the state at the start of the
 * last step and conserved() the state after it, as the reference leaves
 * them).  And where the reference panics (assert!, unwrap) this header
 * throws deepgreen::Error carrying the library's status code and message.
 * T is float (the reference's f32) or double (the FP64 build).
 */
#ifndef DEEPGREEN_HPP
#define DEEPGREEN_HPP

#include <array>
#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <utility>
#include <vector>

#include "deepgreen.h"

namespace deepgreen {

struct Error : std::runtime_error {
    int32_t code;
    Error(int32_t c, const std::string &msg) : std::runtime_error(msg), code(c) {}
};

// CONDUCTING_WALL: the reference's CUDA variant only (src/cu/include/constants.h:44)
enum class BoundaryType : int32_t {
    PERIODIC = DG_BC_PERIODIC,
    OUTFLOW = DG_BC_OUTFLOW,
    WALL = DG_BC_WALL,
    CONDUCTING_WALL = DG_BC_CONDUCTING_WALL
};

// globals.rs:3-8 (f32 in the reference)
inline constexpr double GAMMA = 5.0 / 3.0;
inline constexpr double CFL = 0.2;
inline constexpr double G = -0.1;

// grid.rs:30-41.  nx, ny, nz include the ghost layers, as Simulation::new
// stores them.  The reference's statics and the limiter are run-time fields.
struct Simulation {
    std::size_t nx = 0, ny = 0, nz = 0;
    double ds = 0.0;
    std::array<BoundaryType, 6> bcs{};
    std::array<bool, 3> periodicity{};
    std::size_t nghosts = 2;
    bool gravity = false;
    double gamma = GAMMA, cfl = CFL, g = G;
    int32_t limiter = DG_LIMITER_NONE;
    int32_t device = 0;

    // grid.rs:44-76: a periodic axis must have periodic faces on both sides
    static Simulation new_(std::size_t nx, std::size_t ny, std::size_t nz, double ds,
                           const std::array<BoundaryType, 6> &bcs, const std::array<bool, 3> &periodicity,
                           std::size_t nghosts, bool gravity) {
        for (int a = 0; a < 3; ++a)
            if (periodicity[a] && (bcs[2 * a] != BoundaryType::PERIODIC || bcs[2 * a + 1] != BoundaryType::PERIODIC))
                throw Error(DG_ERR_INVALID, "periodic axis " + std::to_string(a) + " needs periodic faces");
        Simulation s;
        s.nx = nx + 2 * nghosts;
        s.ny = ny + 2 * nghosts;
        s.nz = nz + 2 * nghosts;
        s.ds = ds;
        s.bcs = bcs;
        s.periodicity = periodicity;
        s.nghosts = nghosts;
        s.gravity = gravity;
        return s;
    }
};

// A C-order (x slowest, z fastest) 3-D array, the layout of the reference's
// Array3 and of the C ABI's host arrays.
template <class T> struct Array3 {
    std::size_t nx = 0, ny = 0, nz = 0;
    std::vector<T> v;
    Array3() = default;
    Array3(std::size_t x, std::size_t y, std::size_t z) : nx(x), ny(y), nz(z), v(x * y * z, T(0)) {}
    T &operator()(std::size_t i, std::size_t j, std::size_t k) { return v[(i * ny + j) * nz + k]; }
    const T &operator()(std::size_t i, std::size_t j, std::size_t k) const { return v[(i * ny + j) * nz + k]; }
    T *data() { return v.data(); }
    const T *data() const { return v.data(); }
};

template <class T> struct Primitives {
    Array3<T> rho, vx, vy, vz, p;
    std::array<Array3<T> *, 5> fields() { return {&rho, &vx, &vy, &vz, &p}; }
};

template <class T> struct Conserved {
    Array3<T> mass, momentum_x, momentum_y, momentum_z, energy;
    std::array<Array3<T> *, 5> fields() { return {&mass, &momentum_x, &momentum_y, &momentum_z, &energy}; }
};

namespace detail {
inline void check(int32_t rc, const dg_ctx *ctx) {
    if (rc != DG_OK) throw Error(rc, dg_last_error(ctx));
}
template <class F> std::array<void *, 5> ptrs(F &state) {
    std::array<void *, 5> p{};
    auto f = state.fields();
    for (int i = 0; i < 5; ++i) p[i] = f[i]->data();
    return p;
}
}  // namespace detail

template <class T> class SimulationGrid;
template <class T> void calc_conserved(SimulationGrid<T> &grid);
template <class T> void compute_step(const Simulation &info, SimulationGrid<T> &grid, T &dt);

// grid.rs:111-221 with the state on the GPU.  primitives() starts as zeroed
// host arrays (as SimulationGrid::new allocates them) for the caller to fill
// before calc_conserved.
template <class T> class SimulationGrid {
    static_assert(std::is_same_v<T, float> || std::is_same_v<T, double>, "float or double");

  public:
    Simulation info;

    explicit SimulationGrid(const Simulation &sim) : info(sim) {
        for (auto *f : prim_.fields()) *f = Array3<T>(sim.nx, sim.ny, sim.nz);
        for (auto *f : cons_.fields()) *f = Array3<T>(sim.nx, sim.ny, sim.nz);
        dg_sim_info d{};
        const std::size_t g2 = 2 * sim.nghosts;
        if (sim.nx <= g2 || sim.ny <= g2 || sim.nz <= g2) throw Error(DG_ERR_INVALID, "no interior cells");
        d.nx = (int32_t)(sim.nx - g2);
        d.ny = (int32_t)(sim.ny - g2);
        d.nz = (int32_t)(sim.nz - g2);
        d.nghosts = (int32_t)sim.nghosts;
        d.ds = sim.ds;
        d.gamma = sim.gamma;
        d.cfl = sim.cfl;
        d.g = sim.g;
        for (int i = 0; i < 6; ++i) d.bcs[i] = (int32_t)sim.bcs[i];
        d.gravity = sim.gravity ? 1 : 0;
        d.limiter = sim.limiter;
        d.precision = std::is_same_v<T, double> ? DG_F64 : DG_F32;
        d.device = sim.device;
        d.rounding = DG_ROUNDING_DEFAULT;
        detail::check(dg_create(&d, &ctx_), nullptr);
    }
    static SimulationGrid new_(const Simulation &sim) { return SimulationGrid(sim); }

    SimulationGrid(const SimulationGrid &) = delete;
    SimulationGrid &operator=(const SimulationGrid &) = delete;
    SimulationGrid(SimulationGrid &&o) noexcept
        : info(o.info), ctx_(std::exchange(o.ctx_, nullptr)), prim_(std::move(o.prim_)), cons_(std::move(o.cons_)),
          has_state_(o.has_state_), prim_stale_(o.prim_stale_), cons_stale_(o.cons_stale_) {}
    SimulationGrid &operator=(SimulationGrid &&o) noexcept {
        if (this != &o) {
            if (ctx_) dg_destroy(ctx_);
            info = o.info;
            ctx_ = std::exchange(o.ctx_, nullptr);
            prim_ = std::move(o.prim_);
            cons_ = std::move(o.cons_);
            has_state_ = o.has_state_;
            prim_stale_ = o.prim_stale_;
            cons_stale_ = o.cons_stale_;
        }
        return *this;
    }
    ~SimulationGrid() {
        if (ctx_) dg_destroy(ctx_);
    }

    Primitives<T> &primitives() {
        if (prim_stale_) {
            auto p = detail::ptrs(prim_);
            detail::check(dg_get_primitives(ctx_, p.data()), ctx_);
            prim_stale_ = false;
        }
        return prim_;
    }
    Conserved<T> &conserved() {
        if (cons_stale_) {
            auto p = detail::ptrs(cons_);
            detail::check(dg_get_conserved(ctx_, p.data()), ctx_);
            cons_stale_ = false;
        }
        return cons_;
    }
    dg_ctx *context() const { return ctx_; }

  private:
    dg_ctx *ctx_ = nullptr;
    Primitives<T> prim_;
    Conserved<T> cons_;
    bool has_state_ = false;
    bool prim_stale_ = false, cons_stale_ = false;

    friend void calc_conserved<T>(SimulationGrid<T> &grid);
    friend void compute_step<T>(const Simulation &info, SimulationGrid<T> &grid, T &dt);
};

// physics.rs:143-175: the conserved state from the grid's primitives (the
// host arrays); from here on the state lives on the device.
template <class T> void calc_conserved(SimulationGrid<T> &grid) {
    std::array<const void *, 5> p{};
    auto f = grid.prim_.fields();
    for (int i = 0; i < 5; ++i) p[i] = f[i]->data();
    detail::check(dg_set_primitives(grid.ctx_, p.data()), grid.ctx_);
    grid.has_state_ = true;
    grid.cons_stale_ = true;
}

// physics.rs:595-681: one step; dt receives the step's CFL dt, computed from
// the state at its start.
template <class T> void compute_step(const Simulation &info, SimulationGrid<T> &grid, T &dt) {
    (void)info;
    if (!grid.has_state_) throw Error(DG_ERR_NO_STATE, "calc_conserved must run before compute_step");
    double d = 0.0;
    detail::check(dg_compute_step(grid.ctx_, 1, &d), grid.ctx_);
    dt = (T)d;
    grid.prim_stale_ = grid.cons_stale_ = true;
}

}  // namespace deepgreen

#endif  // DEEPGREEN_HPP
