/*
 * deepgreen.h -- C ABI of the B200 implementation of deep-green's 3D
 * compressible Euler finite-volume step.
 *
 * The reference exposes its step as Rust free functions over a host-side
 * grid (deep-green src/rs/src/physics.rs and grid.rs).  This header is the
 * boundary a Rust `-sys` crate (or ctypes, cgo, ...) binds instead:
 *
 *   reference (src/rs/src/...)                     this ABI
 *   ---------------------------------------------  -----------------------------
 *   Simulation::new            grid.rs:44-76        dg_sim_info + dg_create
 *   SimulationGrid::new        grid.rs:169-221      dg_create (device buffers)
 *   calc_conserved             physics.rs:143-175   dg_set_primitives
 *   grid.conserved.* (write)   grid.rs:87-93        dg_set_conserved
 *   update_primitive_ghost_cells grid.rs:121-135    applied inside every call
 *   compute_step               physics.rs:595-681   dg_compute_step
 *   grid.conserved.* (read)    grid.rs:87-93        dg_get_conserved
 *   grid.primitives.* (read)   grid.rs:95-101       dg_get_primitives
 *
 * Conventions (all functions):
 *   - return int32_t: DG_OK (0) or a negative DG_ERR_* code; nothing throws
 *     across the ABI; dg_last_error() gives a message for the last failure.
 *   - host arrays are C-order (x slowest, z fastest) with the reference's
 *     two ghost layers: (nx+4) x (ny+4) x (nz+4) elements, float or double
 *     as dg_sim_info.precision says.  Conserved fields hold per-cell totals
 *     (mass = rho * ds^3, ...), as the reference's Conserved does.
 *   - one context = one device + one CUDA stream; do not call one context
 *     from two host threads at once (the reference's SimulationGrid is not
 *     shared either).  State stays on the device between calls.
 *   - Every kernel runs on the GPU; there is no CPU path.  A call made
 *     where the device or the kernels are unavailable returns an error.
 */
#ifndef DEEPGREEN_H
#define DEEPGREEN_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define DG_ABI_VERSION 1

/* status codes */
#define DG_OK 0
#define DG_ERR_INVALID (-1)   /* bad argument or unsupported configuration */
#define DG_ERR_CUDA (-2)      /* CUDA runtime/driver error */
#define DG_ERR_NO_STATE (-3)  /* step or read before any state was set */
#define DG_ERR_TIMEOUT (-4)   /* a bounded device-side wait gave up */
#define DG_ERR_NO_DEVICE (-5) /* no usable sm_100 device */

/* BoundaryType, grid.rs:23-28 (same order). Faces: x-, x+, y-, y+, z-, z+. */
#define DG_BC_PERIODIC 0
#define DG_BC_OUTFLOW 1
#define DG_BC_WALL 2
/* Opt-in, from the reference's CUDA variant (src/cu/include/constants.h:44
 * BC::CONDUCTING_WALL, the source term of src/cu/include/kernels.h:559-661):
 * a wall whose ghosts follow DG_BC_WALL's rule and whose face conducts heat
 * between the gas and an outside at 273 K through a wall of thickness 0.008
 * and conductivity 0.2 (outside film coefficient 10, gas constant 287, the
 * reference's constants).  The energy flux through the face gets
 * Q / V = (273 - p/(287 rho)) * (ds^2 / (0.008/0.2 + 1/10)) / ds^3 before
 * the dissipation term, p and rho of the ghost cell's extrapolated state.
 * As in the reference, which adds the term at the flux of lower-cell index
 * 1 on a lower face and n - 2 on an upper face, only a LOWER face's heat
 * reaches the interior: an upper conducting face acts as a plain wall. */
#define DG_BC_CONDUCTING_WALL 3

/* slope limiter: NONE = the reference's central slopes (physics.rs:198-215);
 * MINMOD is an addition of this library */
#define DG_LIMITER_NONE 0
#define DG_LIMITER_MINMOD 1

#define DG_F32 0
#define DG_F64 1

/* arithmetic policy: DEFAULT = fast fused arithmetic for DG_F32 and the
 * reference's rounding for DG_F64; REFERENCE = the reference's operation
 * order without fused multiply-add, IEEE divide/sqrt (bitwise reproducible
 * against a scalar restatement of the Rust code) for either precision;
 * FAST = the fused-arithmetic production kernel in either precision (in
 * DG_F64 it is that kernel's double build, within 1e-12 of the reference's
 * arithmetic rather than bit for bit) */
#define DG_ROUNDING_DEFAULT 0
#define DG_ROUNDING_REFERENCE 1
#define DG_ROUNDING_FAST 2

/* status flags (dg_status) */
#define DG_STATUS_NONFINITE 0x1u  /* a NaN wave speed was seen; dt fell back to cfl*1.0
                                     as calc_timestep does (physics.rs:191-195) */
#define DG_STATUS_TIMEOUT 0x2u    /* a device-side wait ran out; results invalid */

/* Runtime form of Simulation (grid.rs:30-41) plus the constants the
 * reference keeps as statics (globals.rs:3-8). */
typedef struct dg_sim_info {
    int32_t nx, ny, nz;  /* interior cells per axis (>= 2), the arguments of
                            Simulation::new before it adds the ghosts */
    int32_t nghosts;     /* must be 2 (physics.rs:14) */
    double ds;           /* uniform cell size */
    double gamma;        /* globals::GAMMA */
    double cfl;          /* globals::CFL */
    double g;            /* globals::G, used when gravity != 0 */
    int32_t bcs[6];      /* DG_BC_*, Simulation::bcs; periodic faces come in pairs */
    int32_t gravity;     /* Simulation::gravity: z-sweep source, physics.rs:366-372 */
    int32_t limiter;     /* DG_LIMITER_* */
    int32_t precision;   /* DG_F32 or DG_F64 */
    int32_t device;      /* CUDA device ordinal */
    int32_t rounding;    /* DG_ROUNDING_* */
} dg_sim_info;

typedef struct dg_ctx dg_ctx;

/* ABI version of the loaded library (DG_ABI_VERSION). */
int32_t dg_abi_version(void);

/* Simulation::new + SimulationGrid::new: validates info and allocates the
 * device state.  *out is NULL on failure. */
int32_t dg_create(const dg_sim_info *info, dg_ctx **out);
int32_t dg_destroy(dg_ctx *ctx);

/* Primitive fields (rho, vx, vy, vz, p) in; computes the conserved state on
 * the device exactly as calc_conserved (physics.rs:143-175).  Ghost values
 * of the input are ignored: ghosts are refilled by the boundary rules. */
int32_t dg_set_primitives(dg_ctx *ctx, const void *const prim[5]);
/* Conserved fields (mass, mom_x, mom_y, mom_z, energy) in. */
int32_t dg_set_conserved(dg_ctx *ctx, const void *const cons[5]);

/* compute_step (physics.rs:595-681) repeated nsteps times on the device.
 * dt of every step (computed from the state at the start of that step, as
 * calc_timestep does) is written to dts[0..nsteps-1] when dts is non-NULL.
 * Blocks until the steps are done. */
int32_t dg_compute_step(dg_ctx *ctx, int32_t nsteps, double *dts);

/* Conserved state after the last step, ghosts filled by the boundary rules. */
int32_t dg_get_conserved(dg_ctx *ctx, void *const cons[5]);
/* Primitive fields as SimulationGrid::primitives holds them after
 * compute_step returns: the state at the START of the last step (the
 * reference converts before it updates), ghosts filled.  Before any step:
 * the primitives of the current state. */
int32_t dg_get_primitives(dg_ctx *ctx, void *const prim[5]);

/* FP64 sums over interior cells of the five conserved fields of the current
 * state (global mass, momentum and energy). */
int32_t dg_conservation_sums(dg_ctx *ctx, double out[5]);

/* Device-pointer variants of dg_set_conserved / dg_get_conserved for
 * callers that keep the fields in their own CUDA allocations (same layout
 * as the host arrays).  The copies run on the context's stream, a
 * non-blocking stream that does not order against the caller's streams:
 * work that writes the source fields must be complete when
 * dg_set_conserved_device is called.  Both calls return after their copies
 * finished. */
int32_t dg_set_conserved_device(dg_ctx *ctx, const void *const cons[5]);
int32_t dg_get_conserved_device(dg_ctx *ctx, void *const cons[5]);

/* Asynchronous stepping: enqueue nsteps steps on the context's stream and
 * return at once.  dg_get_dts then reads the dt of the last nsteps steps
 * (nsteps <= 4096) after synchronizing. */
int32_t dg_enqueue_steps(dg_ctx *ctx, int32_t nsteps);
int32_t dg_get_dts(dg_ctx *ctx, int32_t nsteps, double *dts);
int32_t dg_synchronize(dg_ctx *ctx);
/* The cudaStream_t the context launches on, as void*. */
int32_t dg_get_stream(dg_ctx *ctx, void **stream);
/* The step's blocks (all launches of one step together), threads per
 * block and x-planes per block.  The production kernel steps a grid that
 * has interior tiles (full tiles two cells clear of every y and z face) in
 * two launches: one block per interior tile marching all of x, then the
 * other tiles in blocks of `chunk` x-planes; otherwise one launch of
 * `chunk`-plane blocks.  Any pointer may be NULL. */
int32_t dg_step_launch_shape(dg_ctx *ctx, int32_t *blocks, int32_t *threads, int32_t *chunk);
/* Override the x-planes per block of the step kernel (0 = automatic; for
 * the production kernel on a grid with interior tiles, of the blocks along
 * the faces). */
int32_t dg_set_chunk(dg_ctx *ctx, int32_t chunk);

/* The dt the next compute_step will take (calc_timestep, physics.rs:177, of
 * the current state).  No counterpart in the reference, where dt is only
 * known after the step; a solve that must end on a given time reads it to
 * shorten its last step.  Synchronises. */
int32_t dg_next_dt(dg_ctx *ctx, double *dt);

/* One step with a caller-chosen dt instead of the CFL dt of calc_timestep
 * (physics.rs:177).  No counterpart in the reference: it advances a coarse
 * grid over exactly the time of two fine-grid steps when the solver
 * generates training pairs for the learned correction, and lets a solve end
 * on a given time.  The next dt is computed from the new state as usual.
 * Synchronises. */
int32_t dg_compute_step_dt(dg_ctx *ctx, double dt);

/* One compute_step on caller-owned device memory; the library allocates
 * nothing.  No counterpart in the reference: it is for callers that must
 * not let a library call cudaMalloc, such as a host program whose device
 * memory is owned by its own pool allocator sized at start-up.
 *   cons_in   device pointer, 5 consecutive fields (mass, mom_x, mom_y,
 *             mom_z, energy), each (nx+4)(ny+4)(nz+4) elements, C order,
 *             float or double per info->precision; (nz+4)*element size
 *             must be a multiple of 16 bytes and the pointer 16-byte
 *             aligned.  Its ghost cells are rewritten in place by the
 *             boundary rules before the step.
 *   cons_out  same layout, distinct from cons_in: the state after the
 *             step, ghosts filled.
 *   dt_used   host pointer or NULL: the dt of the step (from cons_in, as
 *             calc_timestep computes it); when given, the call waits for
 *             the stream and reports a device-side wait that gave up as
 *             DG_ERR_TIMEOUT.  Without it the call returns at once and
 *             cannot see the device's status: read it with
 *             dg_noalloc_status after synchronizing the stream.
 *   stream    cudaStream_t or NULL.
 * The step's scratch (control block and per-block partials) is a 1 MiB
 * array in the library's device image, held by every GPU that loads the
 * library until exit; grids needing more than it holds are rejected with
 * DG_ERR_INVALID.  All calls share that array: calls that overlap on the
 * GPU race.  The first call on a device looks up the array's address with
 * that device current; make it before any stream capture.  The calling
 * thread's current device is the same after the call as before it.
 * Errors: dg_last_error(NULL). */
int32_t dg_compute_step_noalloc(const dg_sim_info *info, void *cons_in, void *cons_out, double *dt_used,
                                void *stream);
/* DG_STATUS_* flags the last dg_compute_step_noalloc call on `device` left
 * in the shared scratch (DG_STATUS_TIMEOUT: that step's output is invalid).
 * Call it after the stream of that step has been synchronized; the next
 * no-allocation step on the device clears them.  Allocates nothing. */
int32_t dg_noalloc_status(int32_t device, uint32_t *flags);

/* ---- Snapshots (save_to_disk, io.rs:5-196) -------------------------------
 * The groups save_to_disk writes for the state: "primitives" (rho, vx, vy,
 * vz, pressure: the state at the start of the last step, as
 * dg_get_primitives) and "conserved" (mass, momentum_x, momentum_y,
 * momentum_z, energy: the current state), each field the full ghosted
 * (nx+4, ny+4, nz+4) C-order array in the context's precision.  (The
 * "gradients" and "fluxes" groups are step intermediates that the fused step
 * never stores; they are not written.)  HDF5 is not available, so the file is
 * "DGSNAP01", a little-endian uint64 header length, a JSON header (dtype,
 * shape, steps, the context's constants as "attrs", and per dataset its
 * "group/name", byte offset and size), then the datasets, each starting on
 * a 4096-byte boundary.  deepgreen.snapshot.read (Python) reads it. */
#define DG_SNAP_PRIMITIVES 0x1u
#define DG_SNAP_CONSERVED 0x2u
typedef struct dg_snapshot dg_snapshot;
/* Device and pinned host buffers for the chosen groups of ctx's state;
 * reusable for every output of a run.  ctx must outlive the snapshot. */
int32_t dg_snapshot_create(dg_ctx *ctx, uint32_t groups, dg_snapshot **out);
int32_t dg_snapshot_destroy(dg_snapshot *snap);
/* Capture the current state: the fields are packed on the device in order
 * on ctx's stream, then copied to pinned host memory on a copy stream.
 * Returns at once; ctx may keep stepping (the capture does not wait for the
 * steps and the steps do not disturb the capture). */
int32_t dg_snapshot_begin(dg_snapshot *snap);
/* Wait for the last capture's copy; *host (if non-NULL) receives the pinned
 * buffer: the fields, dense, in file order. */
int32_t dg_snapshot_wait(dg_snapshot *snap, const void **host);
/* Wait for the last capture and write it to path. */
int32_t dg_snapshot_write(dg_snapshot *snap, const char *path);
/* The file writer on host arrays (no device needed): nfields datasets
 * "group/name" of shape[0]*shape[1]*shape[2] values of dtype (DG_F32 or
 * DG_F64); attrs is a JSON object or NULL. */
int32_t dg_snapshot_write_host(const char *path, int32_t dtype, const int32_t shape[3], int32_t nfields,
                               const char *const names[], const void *const data[], uint64_t steps,
                               const char *attrs);
/* Message of the calling thread's last failed snapshot call. */
const char *dg_snapshot_last_error(const dg_snapshot *snap);

/* ---- Batches: many independent grids, one persistent launch per step ----
 * No counterpart in the reference, which steps one grid per compute_step
 * call (physics.rs:595-681); a batch is N such grids advanced together.
 * Each grid keeps its own state, boundary types, constants and CFL dt.
 * Steps are replayed from a captured CUDA graph.  Batches run the FP32 fast
 * kernel (precision DG_F32, rounding DEFAULT); all grids on one device. */
typedef struct dg_batch dg_batch;
int32_t dg_batch_create(int32_t n, const dg_sim_info *infos, dg_batch **out);
/* Creation flags of dg_batch_create_ex. */
enum {
    /* Each grid may be stored with its axes permuted: the order with the
     * fewest padded cells (z rounds up to the kernel's 64-column tiles, y to
     * its rows, x not at all); z stays z for a grid with gravity.  Inputs
     * and outputs keep the caller's layout (permuted on the device).  A
     * permuted grid's step equals the caller-order step up to rounding (its
     * flux balance adds the axes in another order), not bit for bit. */
    DG_BATCH_REORIENT = 1
};
/* dg_batch_create with flags (0: dg_batch_create). */
int32_t dg_batch_create_ex(int32_t n, const dg_sim_info *infos, uint32_t flags, dg_batch **out);
/* Stored axis d of grid i is the caller's axis axes[d] (0 x, 1 y, 2 z). */
int32_t dg_batch_get_orientation(dg_batch *b, int32_t i, int32_t axes[3]);
int32_t dg_batch_destroy(dg_batch *b);
/* grid i's state from host primitives, as dg_set_primitives */
int32_t dg_batch_set_primitives(dg_batch *b, int32_t i, const void *const prim[5]);
/* nsteps steps of every grid; blocks until done */
int32_t dg_batch_step(dg_batch *b, int32_t nsteps);
/* same, returning at once (ordered on dg_batch_get_stream's stream) */
int32_t dg_batch_enqueue(dg_batch *b, int32_t nsteps);
/* dt of grid i over the last nsteps steps (nsteps <= 4096) */
int32_t dg_batch_get_dts(dg_batch *b, int32_t i, int32_t nsteps, double *dts);
/* grid i's conserved state, ghosts filled, as dg_get_conserved */
int32_t dg_batch_get_conserved(dg_batch *b, int32_t i, void *const cons[5]);
/* tile rows (the production kernel's tile rows, as dg_batch_get_tiling
 * reports them) and x-planes per work item (0 = automatic) */
int32_t dg_batch_set_tiling(dg_batch *b, int32_t tile_rows, int32_t chunk);
int32_t dg_batch_get_tiling(dg_batch *b, int32_t *tile_rows, int32_t *chunk, int32_t *items);
/* times `steps` steps of each candidate tiling on the live batch, keeps the
 * fastest and restores the state it started from */
int32_t dg_batch_autotune(dg_batch *b, int32_t steps, int32_t *tile_rows, int32_t *chunk, double *ms_per_step);
int32_t dg_batch_get_stream(dg_batch *b, void **stream);
/* message of the last failure on b (NULL: as dg_last_error(NULL)) */
const char *dg_batch_last_error(const dg_batch *b);

/* Sticky DG_STATUS_* flags raised by the device since the state was last
 * set (dg_set_*). */
int32_t dg_status(dg_ctx *ctx, uint32_t *flags);

/* Message of the last failed call on ctx (or, when ctx is NULL, of the
 * calling thread's last failed dg_create).  Never NULL. */
const char *dg_last_error(const dg_ctx *ctx);

#ifdef __cplusplus
}
#endif
#endif
