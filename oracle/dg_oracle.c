/*
 * dg_oracle.c -- CPU oracle (test infrastructure; see dg_oracle.h).
 * Instantiates the precision-generic body for double and float and exposes
 * a small C API used through ctypes by the tests and the CPU baseline.
 */
#include "dg_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define REAL double
#define SFX _f64
#define SQRT sqrt
#define FABS fabs
#define FMAX fmax
#include "dg_oracle_impl.h"
#undef REAL
#undef SFX
#undef SQRT
#undef FABS
#undef FMAX

#define REAL float
#define SFX _f32
#define SQRT sqrtf
#define FABS fabsf
#define FMAX fmaxf
#include "dg_oracle_impl.h"
#undef REAL
#undef SFX
#undef SQRT
#undef FABS
#undef FMAX

struct dgo_ctx {
    int precision;
    state_f64 *d;
    state_f32 *f;
};

dgo_ctx *dgo_create(const dgo_info *info, int32_t precision) {
    if (!info || info->nx < 2 || info->ny < 2 || info->nz < 2) return NULL;
    if (precision != 4 && precision != 8) return NULL;
    for (int a = 0; a < 3; ++a) {
        /* Simulation::new asserts periodic pairs (grid.rs:55-63). */
        const int lo = info->bcs[2 * a], hi = info->bcs[2 * a + 1];
        if (lo < 0 || lo > 3 || hi < 0 || hi > 3) return NULL;
        if ((lo == DGO_PERIODIC) != (hi == DGO_PERIODIC)) return NULL;
    }
    dgo_ctx *c = (dgo_ctx *)calloc(1, sizeof(dgo_ctx));
    if (!c) return NULL;
    c->precision = precision;
    if (precision == 8) c->d = st_create_f64(info);
    else c->f = st_create_f32(info);
    if (!c->d && !c->f) {
        free(c);
        return NULL;
    }
    return c;
}

void dgo_destroy(dgo_ctx *c) {
    if (!c) return;
    if (c->d) st_destroy_f64(c->d);
    if (c->f) st_destroy_f32(c->f);
    free(c);
}

void dgo_set_threads(dgo_ctx *c, int32_t mode) {
    if (c->d) c->d->mode = mode;
    if (c->f) c->f->mode = mode;
}

void *dgo_field(dgo_ctx *c, int32_t group, int32_t field) {
    if (field < 0 || field > 4) return NULL;
    if (c->d) {
        state_f64 *s = c->d;
        switch (group) {
        case DGO_PRIM: return s->prim[field];
        case DGO_XTR: return s->xtr[field];
        case DGO_CONS: return s->cons[field];
        case DGO_GRAD: return s->grad[field];
        case DGO_FLUX: return s->flux[field];
        }
    } else {
        state_f32 *s = c->f;
        switch (group) {
        case DGO_PRIM: return s->prim[field];
        case DGO_XTR: return s->xtr[field];
        case DGO_CONS: return s->cons[field];
        case DGO_GRAD: return s->grad[field];
        case DGO_FLUX: return s->flux[field];
        }
    }
    return NULL;
}

void dgo_calc_conserved(dgo_ctx *c) {
    if (c->d) calc_conserved_f64(c->d);
    else calc_conserved_f32(c->f);
}

void dgo_calc_primitives(dgo_ctx *c) {
    if (c->d) calc_primitives_f64(c->d);
    else calc_primitives_f32(c->f);
}

void dgo_update_primitive_ghost_cells(dgo_ctx *c) {
    if (c->d) update_prim_ghosts_f64(c->d, c->d->prim);
    else update_prim_ghosts_f32(c->f, c->f->prim);
}

double dgo_calc_timestep(dgo_ctx *c) {
    if (c->d) return calc_timestep_f64(c->d);
    return (double)calc_timestep_f32(c->f);
}

int32_t dgo_compute_step(dgo_ctx *c, int32_t nsteps, double *dts) {
    for (int32_t s = 0; s < nsteps; ++s) {
        double dt = c->d ? compute_step_f64(c->d, NULL) : (double)compute_step_f32(c->f, NULL);
        if (dts) dts[s] = dt;
    }
    return 0;
}

int32_t dgo_compute_step_given_dts(dgo_ctx *c, int32_t nsteps, const double *dts) {
    if (!dts) return -1;
    for (int32_t s = 0; s < nsteps; ++s) {
        if (c->d) compute_step_f64(c->d, &dts[s]);
        else compute_step_f32(c->f, &dts[s]);
    }
    return 0;
}
