/*
 * dg_oracle_impl.h -- precision-generic body of the CPU oracle (test
 * infrastructure; see dg_oracle.h).  Included twice by dg_oracle.c with
 * REAL = double / float and SFX = _f64 / _f32.
 *
 * Every function names the reference lines it restates.  Floating-point
 * expressions keep the reference's association order and the file is
 * compiled with -ffp-contract=off, so the float instantiation rounds the
 * way the Rust f32 code does (Rust never contracts a*b+c into an fma).
 */

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)
#define FN(name) CAT(name, SFX)

typedef struct FN(state) {
    dgo_info info;
    int nx, ny, nz;        /* ghosted sizes, Simulation::new grid.rs:65-67 */
    size_t ncell;
    int mode;
    REAL *prim[5], *xtr[5], *cons[5], *grad[5], *flux[5];
} FN(state);

#define I3(s, i, j, k) ((((size_t)(i) * (size_t)(s)->ny + (size_t)(j)) * (size_t)(s)->nz) + (size_t)(k))

static FN(state) *FN(st_create)(const dgo_info *info) {
    FN(state) *s = (FN(state) *)calloc(1, sizeof(FN(state)));
    if (!s) return NULL;
    s->info = *info;
    s->nx = info->nx + 4;
    s->ny = info->ny + 4;
    s->nz = info->nz + 4;
    s->ncell = (size_t)s->nx * s->ny * s->nz;
    s->mode = DGO_RUST_LIKE;
    for (int f = 0; f < 5; ++f) {
        /* SimulationGrid::new zero-initialises all arrays (grid.rs:174-212). */
        s->prim[f] = (REAL *)calloc(s->ncell, sizeof(REAL));
        s->xtr[f] = (REAL *)calloc(s->ncell, sizeof(REAL));
        s->cons[f] = (REAL *)calloc(s->ncell, sizeof(REAL));
        s->grad[f] = (REAL *)calloc(s->ncell * 3, sizeof(REAL));
        s->flux[f] = (REAL *)calloc(s->ncell * 3, sizeof(REAL));
        if (!s->prim[f] || !s->xtr[f] || !s->cons[f] || !s->grad[f] || !s->flux[f]) return NULL;
    }
    return s;
}

static void FN(st_destroy)(FN(state) *s) {
    if (!s) return;
    for (int f = 0; f < 5; ++f) {
        free(s->prim[f]); free(s->xtr[f]); free(s->cons[f]);
        free(s->grad[f]); free(s->flux[f]);
    }
    free(s);
}

/* One whole-slice assignment `mesh.slice_mut(s![.., dst, ..]).assign(&src)`
 * along `axis`, for a field with `comp` trailing components (1 for Array3,
 * 3 for Array4).  `neg` negates the copied values (the mapv_inplace(-1.0*x)
 * of handle_walls, boundaries.rs:218). */
static void FN(copy_slice)(const FN(state) *s, REAL *a, int comp, int axis, int dst, int src,
                           int neg) {
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const int par = s->mode == DGO_ALL_PARALLEL;
    if (axis == 0) {
#pragma omp parallel for if (par)
        for (int j = 0; j < ny; ++j)
            for (int k = 0; k < nz; ++k)
                for (int c = 0; c < comp; ++c) {
                    REAL v = a[I3(s, src, j, k) * comp + c];
                    a[I3(s, dst, j, k) * comp + c] = neg ? (REAL)-1.0 * v : v;
                }
    } else if (axis == 1) {
#pragma omp parallel for if (par)
        for (int i = 0; i < nx; ++i)
            for (int k = 0; k < nz; ++k)
                for (int c = 0; c < comp; ++c) {
                    REAL v = a[I3(s, i, src, k) * comp + c];
                    a[I3(s, i, dst, k) * comp + c] = neg ? (REAL)-1.0 * v : v;
                }
    } else {
#pragma omp parallel for if (par)
        for (int i = 0; i < nx; ++i)
            for (int j = 0; j < ny; ++j)
                for (int c = 0; c < comp; ++c) {
                    REAL v = a[I3(s, i, j, src) * comp + c];
                    a[I3(s, i, j, dst) * comp + c] = neg ? (REAL)-1.0 * v : v;
                }
    }
}

/* apply_boundary_conditions (Array3, comp 1) and apply_boundary_conditions4
 * (Array4, comp 3), boundaries.rs:5-99 and 101-195: for each face in the
 * order x-, x+, y-, y+, z-, z+: OUTFLOW copies the first/last interior
 * slice into both ghosts, PERIODIC copies the opposite interior slices,
 * WALL does nothing. */
static void FN(apply_bc)(const FN(state) *s, REAL *a, int comp) {
    const int n[3] = {s->nx, s->ny, s->nz};
    for (int face = 0; face < 6; ++face) {
        const int axis = face / 2, upper = face & 1, m = n[axis];
        switch (s->info.bcs[face]) {
        case DGO_OUTFLOW:
            if (!upper) {
                FN(copy_slice)(s, a, comp, axis, 0, 2, 0);
                FN(copy_slice)(s, a, comp, axis, 1, 2, 0);
            } else {
                FN(copy_slice)(s, a, comp, axis, m - 2, m - 3, 0);
                FN(copy_slice)(s, a, comp, axis, m - 1, m - 3, 0);
            }
            break;
        case DGO_PERIODIC:
            if (!upper) {
                FN(copy_slice)(s, a, comp, axis, 0, m - 4, 0);
                FN(copy_slice)(s, a, comp, axis, 1, m - 3, 0);
            } else {
                FN(copy_slice)(s, a, comp, axis, m - 2, 2, 0);
                FN(copy_slice)(s, a, comp, axis, m - 1, 3, 0);
            }
            break;
        default: /* WALL, CONDUCTING_WALL */
            break;
        }
    }
}

/* handle_walls, boundaries.rs:197-407: for each WALL face (order x-, x+,
 * y-, y+, z-, z+) mirror the two interior slices into the ghosts, with the
 * normal velocity negated.  Lower: 1 <- 2, 0 <- 3; upper: n-2 <- n-3,
 * n-1 <- n-4. */
static void FN(handle_walls)(const FN(state) *s, REAL *q[5]) {
    const int n[3] = {s->nx, s->ny, s->nz};
    for (int face = 0; face < 6; ++face) {
        /* the CUDA variant fills a conducting wall's ghosts by the wall
         * rule (src/cu/include/kernels.h:327) */
        if (s->info.bcs[face] != DGO_WALL && s->info.bcs[face] != DGO_CONDUCTING_WALL) continue;
        const int axis = face / 2, upper = face & 1, m = n[axis];
        const int d0 = upper ? m - 2 : 1, s0 = upper ? m - 3 : 2;
        const int d1 = upper ? m - 1 : 0, s1 = upper ? m - 4 : 3;
        for (int f = 0; f < 5; ++f) FN(copy_slice)(s, q[f], 1, axis, d0, s0, f == 1 + axis);
        for (int f = 0; f < 5; ++f) FN(copy_slice)(s, q[f], 1, axis, d1, s1, f == 1 + axis);
    }
}

/* grid.rs:121-135 / 137-151 */
static void FN(update_prim_ghosts)(const FN(state) *s, REAL *q[5]) {
    FN(handle_walls)(s, q);
    for (int f = 0; f < 5; ++f) FN(apply_bc)(s, q[f], 1);
}

/* physics.rs:109-141 */
static void FN(calc_primitives)(FN(state) *s) {
    const REAL ds = (REAL)s->info.ds;
    const REAL V = ds * ds * ds;
    const REAL gm1 = (REAL)s->info.gamma - (REAL)1.0;
    const int par = s->mode != DGO_SERIAL;
    REAL *r = s->prim[0], *vx = s->prim[1], *vy = s->prim[2], *vz = s->prim[3], *p = s->prim[4];
    const REAL *M = s->cons[0], *Mx = s->cons[1], *My = s->cons[2], *Mz = s->cons[3], *E = s->cons[4];
#pragma omp parallel for if (par)
    for (size_t c = 0; c < s->ncell; ++c) {
        r[c] = M[c] / V;
        vx[c] = Mx[c] / (r[c] * V);
        vy[c] = My[c] / (r[c] * V);
        vz[c] = Mz[c] / (r[c] * V);
        p[c] = (E[c] / V - (REAL)0.5 * r[c] * (vx[c] * vx[c] + vy[c] * vy[c] + vz[c] * vz[c])) * gm1;
    }
}

/* physics.rs:143-175 */
static void FN(calc_conserved)(FN(state) *s) {
    const REAL ds = (REAL)s->info.ds;
    const REAL V = ds * ds * ds;
    const REAL gm1 = (REAL)s->info.gamma - (REAL)1.0;
    const int par = s->mode != DGO_SERIAL;
    const REAL *r = s->prim[0], *vx = s->prim[1], *vy = s->prim[2], *vz = s->prim[3], *p = s->prim[4];
    REAL *M = s->cons[0], *Mx = s->cons[1], *My = s->cons[2], *Mz = s->cons[3], *E = s->cons[4];
#pragma omp parallel for if (par)
    for (size_t c = 0; c < s->ncell; ++c) {
        M[c] = r[c] * V;
        Mx[c] = vx[c] * r[c] * V;
        My[c] = vy[c] * r[c] * V;
        Mz[c] = vz[c] * r[c] * V;
        E[c] = V * (r[c] * (vx[c] * vx[c] + vy[c] * vy[c] + vz[c] * vz[c]) / (REAL)2.0 + p[c] / gm1);
    }
}

/* physics.rs:177-196.  ndarray-stats QuantileExt::min returns Err on any
 * NaN (partial_cmp is None), and the reference then uses 1.0. */
static REAL FN(calc_timestep)(FN(state) *s) {
    const REAL ds = (REAL)s->info.ds;
    const REAL gam = (REAL)s->info.gamma;
    const REAL *r = s->prim[0], *vx = s->prim[1], *vy = s->prim[2], *vz = s->prim[3], *p = s->prim[4];
    const int par = s->mode != DGO_SERIAL;
    REAL vmin = (REAL)INFINITY;
    int nan = 0;
#pragma omp parallel for if (par) reduction(min : vmin) reduction(| : nan)
    for (size_t c = 0; c < s->ncell; ++c) {
        REAL v = ds / (SQRT(gam * p[c] / r[c]) + SQRT(vx[c] * vx[c] + vy[c] * vy[c] + vz[c] * vz[c]));
        if (v != v) nan = 1;
        else if (v < vmin) vmin = v;
    }
    const REAL minv = nan ? (REAL)1.0 : vmin;
    return (REAL)s->info.cfl * minv;
}

/* Slope limiter added by this project (the reference computes unlimited
 * central slopes everywhere).  minmod(a, b): 0 when a, b differ in sign or
 * one is zero, else the one of smaller magnitude. */
static inline REAL FN(minmod)(REAL a, REAL b) {
    if (!(a * b > (REAL)0.0)) return (REAL)0.0;
    return FABS(a) < FABS(b) ? a : b;
}

/* physics.rs:198-215: central differences on i, j, k in 1..n-2, all three
 * directions; other entries keep their previous value. */
static void FN(calc_gradients)(FN(state) *s, const REAL *q, REAL *g) {
    const REAL ds = (REAL)s->info.ds;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const int par = s->mode != DGO_SERIAL;
    const int lim = s->info.limiter;
    const size_t sx = (size_t)ny * nz, sy = (size_t)nz, sz = 1;
    const size_t st[3] = {sx, sy, sz};
#pragma omp parallel for if (par)
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 1; k < nz - 1; ++k) {
                const size_t c = I3(s, i, j, k);
                for (int d = 0; d < 3; ++d) {
                    REAL val;
                    if (!lim) {
                        val = (q[c + st[d]] - q[c - st[d]]) / ((REAL)2.0 * ds);
                    } else {
                        val = FN(minmod)((q[c] - q[c - st[d]]) / ds, (q[c + st[d]] - q[c]) / ds);
                    }
                    g[c * 3 + d] = val;
                }
            }
}

/* physics.rs:217-282, over every cell including ghosts. */
static void FN(extrapolate)(FN(state) *s, REAL dt) {
    const REAL gam = (REAL)s->info.gamma;
    const int par = s->mode == DGO_ALL_PARALLEL;
    REAL *const *P = s->prim, *const *G = s->grad, *const *X = s->xtr;
#pragma omp parallel for if (par)
    for (size_t c = 0; c < s->ncell; ++c) {
        const REAL rho = P[0][c], vx = P[1][c], vy = P[2][c], vz = P[3][c], p = P[4][c];
        const REAL drho_dx = G[0][3 * c], dvx_dx = G[1][3 * c], dvy_dx = G[2][3 * c], dvz_dx = G[3][3 * c];
        const REAL drho_dy = G[0][3 * c + 1], dvx_dy = G[1][3 * c + 1], dvy_dy = G[2][3 * c + 1],
                   dvz_dy = G[3][3 * c + 1];
        const REAL drho_dz = G[0][3 * c + 2], dvx_dz = G[1][3 * c + 2], dvy_dz = G[2][3 * c + 2],
                   dvz_dz = G[3][3 * c + 2];
        const REAL dp_dx = G[4][3 * c], dp_dy = G[4][3 * c + 1], dp_dz = G[4][3 * c + 2];
        const REAL h = (REAL)0.5 * dt;
        X[0][c] = rho - h * (vx * drho_dx + rho * dvx_dx + vy * drho_dy + rho * dvy_dy + vz * drho_dz +
                             rho * dvz_dz);
        X[1][c] = vx - h * (vx * dvx_dx + vy * dvx_dy + vz * dvx_dz + ((REAL)1.0 / rho) * dp_dx);
        X[2][c] = vy - h * (vx * dvy_dx + vy * dvy_dy + vz * dvy_dz + ((REAL)1.0 / rho) * dp_dy);
        X[3][c] = vz - h * (vx * dvz_dx + vy * dvz_dy + vz * dvz_dz + ((REAL)1.0 / rho) * dp_dz);
        X[4][c] = p - h * (gam * p * (dvx_dx + dvy_dy + dvz_dz) + vx * dp_dx + vy * dp_dy + vz * dp_dz);
    }
}

/* Heat conducted through a conducting wall, per unit volume: Q / V of the
 * CUDA variant's flux kernel (src/cu/include/kernels.h:561-575), with its
 * constants (constants.h:63-66: RS = 287, T_OUT_KELVIN = 273, VOUT_MS = 0;
 * wall thickness d = 0.008, conductivity kappa = 0.2 as float literals) and
 * t_in = p / (RS rho) of the face's lower cell. */
static REAL FN(wall_heat)(REAL rho, REAL p, REAL ds) {
    const REAL rs = (REAL)287.0f, t_out = (REAL)273.0f, vout = (REAL)0.0f;
    const REAL t_in = p / (rs * rho);
    const REAL hc_out = (REAL)10.0f - vout + (REAL)10.0f * SQRT(vout);
    const REAL S = ds * ds;
    const REAL V = ds * ds * ds;
    const REAL d = (REAL)0.008f, kappa = (REAL)0.2f;
    const REAL Q = (t_out - t_in) * (S / ((d / kappa) + ((REAL)1.0f / hc_out)));
    return Q / V;
}

/* physics.rs:284-409 for sweep direction `dim`.  The caller passes the
 * arrays permuted so that slot 1 holds the normal component
 * (compute_step, physics.rs:616-677); `fo` are the output flux arrays in
 * the same permuted order.  Conducting walls: the CUDA variant adds Q / V
 * to the energy flux of every face whose lower-cell index is 1 on the axis
 * of a lower conducting face, or n - 2 on the axis of an upper one, in each
 * of the three sweeps, after the advective flux and before gravity and the
 * dissipation (kernels.h:561-661; its bcs order is x-, y-, z-, x+, y+, z+,
 * mapped here onto this path's x-, x+, y-, y+, z-, z+).  Only the normal
 * flux at a lower wall's first face reaches an interior cell; the others
 * touch ghost cells only. */
static void FN(flux_sweep)(FN(state) *s, int dim, REAL *fo[5], REAL *const gi[5], REAL *const xi[5]) {
    const REAL ds = (REAL)s->info.ds;
    const REAL gam = (REAL)s->info.gamma;
    const REAL G = (REAL)s->info.g;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const int par = s->mode == DGO_ALL_PARALLEL;
    const int grav = s->info.gravity && dim == 2;
    int heat = 0;
    for (int f = 0; f < 6; ++f) heat |= s->info.bcs[f] == DGO_CONDUCTING_WALL;
    const size_t off = dim == 0 ? (size_t)ny * nz : (dim == 1 ? (size_t)nz : 1);
    const REAL *rho = xi[0], *vx = xi[1], *vy = xi[2], *vz = xi[3], *p = xi[4];
    const REAL *drho = gi[0], *dvx = gi[1], *dvy = gi[2], *dvz = gi[3], *dp = gi[4];
#pragma omp parallel for if (par)
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 1; k < nz - 1; ++k) {
                const size_t c = I3(s, i, j, k), u = c + off;
                const REAL half = ds / (REAL)2.;
                const REAL rl = rho[u] - (drho[3 * u + dim]) * half;
                const REAL rr = rho[c] + (drho[3 * c + dim]) * half;
                const REAL vxl = vx[u] - (dvx[3 * u + dim]) * half;
                const REAL vxr = vx[c] + (dvx[3 * c + dim]) * half;
                const REAL vyl = vy[u] - (dvy[3 * u + dim]) * half;
                const REAL vyr = vy[c] + (dvy[3 * c + dim]) * half;
                const REAL vzl = vz[u] - (dvz[3 * u + dim]) * half;
                const REAL vzr = vz[c] + (dvz[3 * c + dim]) * half;
                const REAL pl = p[u] - (dp[3 * u + dim]) * half;
                const REAL pr = p[c] + (dp[3 * c + dim]) * half;

                const REAL en_left = (REAL)0.5 * (rl * (vxl * vxl + vyl * vyl + vzl * vzl)) + (pl / (gam - (REAL)1.0));
                const REAL en_right = (REAL)0.5 * (rr * (vxr * vxr + vyr * vyr + vzr * vzr)) + (pr / (gam - (REAL)1.0));
                const REAL rho_star = (rl + rr) / (REAL)2.0;
                const REAL mx = (rl * vxl + rr * vxr) / (REAL)2.0;
                const REAL my = (rl * vyl + rr * vyr) / (REAL)2.0;
                const REAL mz = (rl * vzl + rr * vzr) / (REAL)2.0;
                const REAL en_star = (REAL)0.5 * (en_left + en_right);
                const REAL p_star = (gam - (REAL)1.0) * (en_star - (REAL)0.5 * (mx * mx + my * my + mz * mz) / rho_star);

                const size_t o = 3 * c + dim;
                fo[0][o] = mx;
                fo[1][o] = (mx * mx / rho_star) + p_star;
                fo[2][o] = mx * my / rho_star;
                fo[3][o] = mx * mz / rho_star;
                fo[4][o] = (en_star + p_star) * (mx / rho_star);
                if (heat) {
                    const int idx[3] = {i, j, k}, nn[3] = {nx, ny, nz};
                    for (int a = 0; a < 3; ++a)   /* lower faces x, y, z */
                        if (s->info.bcs[2 * a] == DGO_CONDUCTING_WALL && idx[a] == 1)
                            fo[4][o] += FN(wall_heat)(rho[c], p[c], ds);
                    for (int a = 0; a < 3; ++a)   /* upper faces */
                        if (s->info.bcs[2 * a + 1] == DGO_CONDUCTING_WALL && idx[a] == nn[a] - 2)
                            fo[4][o] += FN(wall_heat)(rho[c], p[c], ds);
                }
                if (grav) {
                    const REAL h = ((REAL)nz - (REAL)2.0 * (REAL)2) * ds - ((REAL)k - (REAL)2.0) * ds;
                    fo[1][o] += (REAL)1.0 * rho_star * G * h;
                    fo[4][o] += (REAL)0.5 * rho_star * (vxl + vxr) * G * h;
                }
                const REAL c_l = SQRT(gam * pl / rl) + FABS(vxl);
                const REAL c_r = SQRT(gam * pr / rr) + FABS(vxr);
                const REAL c_star = FMAX(c_l, c_r);
                fo[0][o] = mx - (REAL)0.5 * c_star * (rl - rr);
                fo[1][o] -= c_star * (rl * vxl - rr * vxr) / (REAL)2.0;
                fo[2][o] -= c_star * (rl * vyl - rr * vyr) / (REAL)2.0;
                fo[3][o] -= c_star * (rl * vzl - rr * vzr) / (REAL)2.0;
                fo[4][o] -= c_star * (en_left - en_right) / (REAL)2.0;
                fo[0][o] *= ds;
                fo[1][o] *= ds;
                fo[2][o] *= ds;
                fo[3][o] *= ds;
                fo[4][o] *= ds;
            }
}

/* physics.rs:539-593, cells 1..n-2 on every axis. */
static void FN(add_fluxes)(FN(state) *s, REAL dt) {
    const REAL ds = (REAL)s->info.ds;
    const int nx = s->nx, ny = s->ny, nz = s->nz;
    const int par = s->mode == DGO_ALL_PARALLEL;
    const size_t sx = (size_t)ny * nz, sy = (size_t)nz;
#pragma omp parallel for if (par)
    for (int i = 1; i < nx - 1; ++i)
        for (int j = 1; j < ny - 1; ++j)
            for (int k = 1; k < nz - 1; ++k) {
                const size_t c = I3(s, i, j, k);
                for (int f = 0; f < 5; ++f) {
                    const REAL *F = s->flux[f];
                    s->cons[f][c] -= dt * ds *
                                     (F[3 * c + 0] - F[3 * (c - sx) + 0] + F[3 * c + 1] - F[3 * (c - sy) + 1] +
                                      F[3 * c + 2] - F[3 * (c - 1) + 2]);
                }
            }
}

/* physics.rs:595-681.  dt_given: NULL, or the step's dt to use in place
 * of calc_timestep's (dgo_compute_step_given_dts). */
static REAL FN(compute_step)(FN(state) *s, const double *dt_given) {
    FN(calc_primitives)(s);
    FN(update_prim_ghosts)(s, s->prim);
    const REAL dt = dt_given ? (REAL)*dt_given : FN(calc_timestep)(s);
    for (int f = 0; f < 5; ++f) FN(calc_gradients)(s, s->prim[f], s->grad[f]);
    for (int f = 0; f < 5; ++f) FN(apply_bc)(s, s->grad[f], 3);
    FN(extrapolate)(s, dt);
    FN(update_prim_ghosts)(s, s->xtr);
    {
        REAL *fo[5] = {s->flux[0], s->flux[1], s->flux[2], s->flux[3], s->flux[4]};
        REAL *gi[5] = {s->grad[0], s->grad[1], s->grad[2], s->grad[3], s->grad[4]};
        REAL *xi[5] = {s->xtr[0], s->xtr[1], s->xtr[2], s->xtr[3], s->xtr[4]};
        FN(flux_sweep)(s, 0, fo, gi, xi);
    }
    {
        REAL *fo[5] = {s->flux[0], s->flux[2], s->flux[1], s->flux[3], s->flux[4]};
        REAL *gi[5] = {s->grad[0], s->grad[2], s->grad[1], s->grad[3], s->grad[4]};
        REAL *xi[5] = {s->xtr[0], s->xtr[2], s->xtr[1], s->xtr[3], s->xtr[4]};
        FN(flux_sweep)(s, 1, fo, gi, xi);
    }
    {
        REAL *fo[5] = {s->flux[0], s->flux[3], s->flux[1], s->flux[2], s->flux[4]};
        REAL *gi[5] = {s->grad[0], s->grad[3], s->grad[1], s->grad[2], s->grad[4]};
        REAL *xi[5] = {s->xtr[0], s->xtr[3], s->xtr[1], s->xtr[2], s->xtr[4]};
        FN(flux_sweep)(s, 2, fo, gi, xi);
    }
    for (int f = 0; f < 5; ++f) FN(apply_bc)(s, s->flux[f], 3);
    FN(add_fluxes)(s, dt);
    return dt;
}

#undef I3
#undef FN
