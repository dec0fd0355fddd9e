/*
 * dg_oracle.h -- CPU oracle for the deep-green Euler finite-volume step.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA
 * implementation: only the test-suite, the smoke check and the CPU-baseline
 * leg of the benchmark may load it.  The product path never links it.
 *
 * It restates, array by array and in the same operation order, the Rust
 * reference path of deep-green:
 *   src/rs/src/physics.rs   calc_primitives (109-141), calc_conserved (143-175),
 *                           calc_timestep (177-196), calc_gradients (198-215),
 *                           extrapolate_primitives_t (217-282),
 *                           calc_flux_reconstruction (284-409), add_fluxes
 *                           (539-593), compute_step (595-681)
 *   src/rs/src/boundaries.rs apply_boundary_conditions (5-99),
 *                           apply_boundary_conditions4 (101-195),
 *                           handle_walls (197-407)
 *   src/rs/src/grid.rs      Simulation::new (44-76), ghost-update methods
 *                           (121-167), SimulationGrid::new (169-221)
 * It keeps all 45 ghosted arrays of SimulationGrid (5 primitives, 5
 * extrapolated primitives, 5 conserved, 5 gradients x 3, 5 fluxes x 3) and
 * fills ghosts with whole-slice copies exactly as the reference does.
 *
 * Parameters that the reference hard-codes as statics (globals.rs:3-8:
 * GAMMA, CFL, G) are runtime fields here.  One addition that the reference
 * does not have is switchable and off by default: a minmod slope limiter
 * (limiter = 1).  Gravity follows physics.rs:366-372.  The conducting wall
 * (DGO_CONDUCTING_WALL) exists only in the reference's CUDA variant
 * (src/cu/include/kernels.h:559-661); it is restated onto this path as
 * that code applies it (see flux_sweep).
 *
 * PARITY PINNED against the reference's own code where it can run here.
 * The Rust path cannot be built (no Rust toolchain or crates), and the
 * reference ships no tests or stored outputs.  Its CUDA variant's kernels
 * (src/cu/include/kernels.h) do run here, compiled for the host by
 * oracle/refcu on the reference's own configuration headers; their outputs
 * are the golden vectors tests/golden/refcu_cases.npz.  Given the same dt,
 * this oracle is bit for bit equal to them in FP64 on the KHI configuration
 * (periodic, 5 steps) and the TRB configuration (walls, gravity), within
 * 2e-15 on the Sod configuration (whose ds is not a power of two: the CUDA
 * gradient multiplies by 1/(2 ds) where the Rust one divides), and in FP32
 * bit for bit except one last-place unit of mass (a double literal in the
 * CUDA mass flux); its own dt is within one last-place unit of theirs.
 * Two parts of the Rust path have no counterpart there and stay pinned only
 * by the independent NumPy restatement (oracle/numpy_twin.py) and by
 * physics checks: the ghost rules of the derived arrays (gradients,
 * predicted states, fluxes; boundaries.rs applied in compute_step), which
 * the CUDA variant does not apply, so the first interior layer at a wall
 * or outflow face differs between the two variants by design; and the
 * minmod limiter, this project's addition.
 *
 * Build: make -C oracle   (gcc, -O2 -fopenmp -ffp-contract=off)
 */
#ifndef DG_ORACLE_H
#define DG_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* BoundaryType, grid.rs:23-28 (same order), plus the CUDA variant's
 * conducting wall (src/cu/include/constants.h:44 BC::CONDUCTING_WALL): a
 * wall whose ghosts follow the wall rule (src/cu/include/kernels.h:327) and
 * whose flux gets a heat source (kernels.h:559-661; see flux_sweep). */
enum { DGO_PERIODIC = 0, DGO_OUTFLOW = 1, DGO_WALL = 2, DGO_CONDUCTING_WALL = 3 };

/* Array groups of SimulationGrid, grid.rs:111-118. */
enum { DGO_PRIM = 0, DGO_XTR = 1, DGO_CONS = 2, DGO_GRAD = 3, DGO_FLUX = 4 };

/* Threading of the restatement: serial; parallel only where the Rust code
 * uses rayon Zip::par_for_each (calc_primitives, calc_conserved,
 * calc_timestep, calc_gradients); or every phase parallel. */
enum { DGO_SERIAL = 0, DGO_RUST_LIKE = 1, DGO_ALL_PARALLEL = 2 };

typedef struct dgo_info {
    int32_t nx, ny, nz;  /* interior cells; arrays are (n+4)^3 with 2 ghosts */
    int32_t bcs[6];      /* x-, x+, y-, y+, z-, z+ */
    int32_t gravity;     /* Simulation::gravity */
    int32_t limiter;     /* 0: central slopes (reference); 1: minmod */
    double ds, gamma, cfl, g;
} dgo_info;

typedef struct dgo_ctx dgo_ctx;

/* precision: 8 (double) or 4 (float).  Returns NULL on bad arguments. */
dgo_ctx *dgo_create(const dgo_info *info, int32_t precision);
void dgo_destroy(dgo_ctx *ctx);
void dgo_set_threads(dgo_ctx *ctx, int32_t mode);
/* Pointer to an internal array: group DGO_PRIM/XTR/CONS: (n_x,n_y,n_z);
 * DGO_GRAD/FLUX: (n_x,n_y,n_z,3).  field: 0 rho/mass, 1 vx/mom_x,
 * 2 vy/mom_y, 3 vz/mom_z, 4 p/energy. */
void *dgo_field(dgo_ctx *ctx, int32_t group, int32_t field);
/* physics.rs:143 */
void dgo_calc_conserved(dgo_ctx *ctx);
/* physics.rs:109 */
void dgo_calc_primitives(dgo_ctx *ctx);
/* grid.rs:121 */
void dgo_update_primitive_ghost_cells(dgo_ctx *ctx);
/* physics.rs:177; returns dt in double. */
double dgo_calc_timestep(dgo_ctx *ctx);
/* physics.rs:595; runs nsteps steps, dt of each step written to dts[]
 * (may be NULL).  Returns 0. */
int32_t dgo_compute_step(dgo_ctx *ctx, int32_t nsteps, double *dts);
/* compute_step with each step's dt taken from dts[] (converted to the
 * context's precision) instead of calc_timestep: compares the rest of the
 * step with an implementation whose dt rounds differently (the reference's
 * CUDA variant, whose CFL * DELTA is a float product).  -1 if dts is NULL. */
int32_t dgo_compute_step_given_dts(dgo_ctx *ctx, int32_t nsteps, const double *dts);

#ifdef __cplusplus
}
#endif
#endif
