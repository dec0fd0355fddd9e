"""Independent NumPy restatement of deep-green's Rust Euler step.

TEST INFRASTRUCTURE ONLY (checker, never the product path).

Written separately from the C oracle (``dg_oracle_impl.h``) and in a
different style: whole-array slicing instead of index loops.  The two
readings of the Rust source are compared with each other in the tests.
The C oracle is further pinned against the reference's CUDA kernels run on
the host (dg_oracle.h); this reading is what pins the parts those kernels
lack (the ghost rules of the derived arrays).

Reference lines restated (paths within deep-green):
  src/rs/src/physics.rs: calc_primitives 109-141, calc_conserved 143-175,
      calc_timestep 177-196, calc_gradients 198-215,
      extrapolate_primitives_t 217-282, calc_flux_reconstruction 284-409,
      add_fluxes 539-593, compute_step 595-681
  src/rs/src/boundaries.rs: apply_boundary_conditions 5-99,
      apply_boundary_conditions4 101-195, handle_walls 197-407
  src/rs/src/grid.rs: update_*_ghost_cells 121-167
"""
from __future__ import annotations

import numpy as np

PERIODIC, OUTFLOW, WALL, CONDUCTING_WALL = 0, 1, 2, 3


def _sl(axis: int, idx):
    s = [slice(None)] * 3
    s[axis] = idx
    return tuple(s)


class TwinState:
    """Ghosted arrays of SimulationGrid (grid.rs:111-118).

    prim/xtr/cons: list of 5 arrays (n, n, n); grad/flux: 5 arrays
    (n, n, n, 3).  ``bcs`` follows Simulation::bcs (x-, x+, y-, y+, z-, z+).
    """

    def __init__(self, shape, ds, bcs, gamma, cfl, dtype=np.float64, limiter=0,
                 gravity=False, g=-0.1):
        n = tuple(int(s) + 4 for s in shape)
        self.n = n
        self.dtype = np.dtype(dtype)
        T = self.dtype.type
        self.ds, self.gamma, self.cfl, self.g = T(ds), T(gamma), T(cfl), T(g)
        self.bcs = list(bcs)
        self.limiter = limiter
        self.gravity = gravity
        z3 = lambda: np.zeros(n, dtype=self.dtype)
        z4 = lambda: np.zeros(n + (3,), dtype=self.dtype)
        self.prim = [z3() for _ in range(5)]
        self.xtr = [z3() for _ in range(5)]
        self.cons = [z3() for _ in range(5)]
        self.grad = [z4() for _ in range(5)]
        self.flux = [z4() for _ in range(5)]

    # ---- boundaries.rs ------------------------------------------------
    def _bc_scalar_like(self, a):
        """apply_boundary_conditions / apply_boundary_conditions4 on one array."""
        for face, bc in enumerate(self.bcs):
            ax, up = divmod(face, 2)
            m = self.n[ax]
            if bc == OUTFLOW:
                src = a[_sl(ax, m - 3 if up else 2)].copy()
                for g in ((m - 2, m - 1) if up else (0, 1)):
                    a[_sl(ax, g)] = src
            elif bc == PERIODIC:
                pairs = ((m - 2, 2), (m - 1, 3)) if up else ((0, m - 4), (1, m - 3))
                for dst, src in pairs:
                    a[_sl(ax, dst)] = a[_sl(ax, src)].copy()

    def _walls(self, q):
        """handle_walls: mirror two interior slices, negate normal velocity."""
        for face, bc in enumerate(self.bcs):
            if bc not in (WALL, CONDUCTING_WALL):
                continue
            ax, up = divmod(face, 2)
            m = self.n[ax]
            pairs = ((m - 2, m - 3), (m - 1, m - 4)) if up else ((1, 2), (0, 3))
            for dst, src in pairs:
                for f in range(5):
                    v = q[f][_sl(ax, src)].copy()
                    if f == 1 + ax:
                        v = -v
                    q[f][_sl(ax, dst)] = v

    def _prim_ghosts(self, q):
        self._walls(q)
        for f in range(5):
            self._bc_scalar_like(q[f])

    # ---- physics.rs -----------------------------------------------------
    def calc_conserved(self):
        T = self.dtype.type
        V = self.ds * self.ds * self.ds
        r, vx, vy, vz, p = self.prim
        self.cons[0][...] = r * V
        self.cons[1][...] = vx * r * V
        self.cons[2][...] = vy * r * V
        self.cons[3][...] = vz * r * V
        self.cons[4][...] = V * (r * (vx * vx + vy * vy + vz * vz) / T(2.0) + p / (self.gamma - T(1.0)))

    def calc_primitives(self):
        T = self.dtype.type
        V = self.ds * self.ds * self.ds
        M, Mx, My, Mz, E = self.cons
        with np.errstate(all="ignore"):
            r = M / V
            vx = Mx / (r * V)
            vy = My / (r * V)
            vz = Mz / (r * V)
            p = (E / V - T(0.5) * r * (vx * vx + vy * vy + vz * vz)) * (self.gamma - T(1.0))
        for dst, src in zip(self.prim, (r, vx, vy, vz, p)):
            dst[...] = src

    def calc_timestep(self):
        r, vx, vy, vz, p = self.prim
        with np.errstate(all="ignore"):
            w = self.ds / (np.sqrt(self.gamma * p / r) + np.sqrt(vx * vx + vy * vy + vz * vz))
        if np.isnan(w).any():
            return self.cfl * self.dtype.type(1.0)
        return self.cfl * w.min()

    def _gradient(self, q, out):
        T = self.dtype.type
        inner = (slice(1, -1),) * 3
        for d in range(3):
            lo = [slice(1, -1)] * 3
            hi = [slice(1, -1)] * 3
            lo[d] = slice(0, -2)
            hi[d] = slice(2, None)
            if self.limiter == 0:
                out[inner + (d,)] = (q[tuple(hi)] - q[tuple(lo)]) / (T(2.0) * self.ds)
            else:
                c = q[inner]
                a = (c - q[tuple(lo)]) / self.ds
                b = (q[tuple(hi)] - c) / self.ds
                pick = np.where(np.abs(a) < np.abs(b), a, b)
                out[inner + (d,)] = np.where(a * b > 0, pick, T(0.0))

    def _extrapolate(self, dt):
        T = self.dtype.type
        rho, vx, vy, vz, p = self.prim
        g = [[self.grad[f][..., d] for d in range(3)] for f in range(5)]
        (drx, dry, drz), (dxx, dxy, dxz), (dyx, dyy, dyz), (dzx, dzy, dzz), (dpx, dpy, dpz) = g
        h = T(0.5) * dt
        with np.errstate(all="ignore"):
            inv = T(1.0) / rho
            self.xtr[0][...] = rho - h * (vx * drx + rho * dxx + vy * dry + rho * dyy + vz * drz + rho * dzz)
            self.xtr[1][...] = vx - h * (vx * dxx + vy * dxy + vz * dxz + inv * dpx)
            self.xtr[2][...] = vy - h * (vx * dyx + vy * dyy + vz * dyz + inv * dpy)
            self.xtr[3][...] = vz - h * (vx * dzx + vy * dzy + vz * dzz + inv * dpz)
            self.xtr[4][...] = p - h * (self.gamma * p * (dxx + dyy + dzz) + vx * dpx + vy * dpy + vz * dpz)

    def _flux(self, dim, perm):
        """One calc_flux_reconstruction sweep; ``perm`` puts the normal
        velocity/momentum in slot 1 (physics.rs:616-677)."""
        T = self.dtype.type
        ds, gam = self.ds, self.gamma
        gm1 = gam - T(1.0)
        c_sl = (slice(1, -1),) * 3
        u_sl = [slice(1, -1)] * 3
        u_sl[dim] = slice(2, None)
        u_sl = tuple(u_sl)
        X = [self.xtr[i] for i in perm]
        G = [self.grad[i][..., dim] for i in perm]
        half = ds / T(2.0)
        with np.errstate(all="ignore"):
            L = [X[f][u_sl] - G[f][u_sl] * half for f in range(5)]   # reference "l": upper cell
            R = [X[f][c_sl] + G[f][c_sl] * half for f in range(5)]   # reference "r": lower cell
            rl, vxl, vyl, vzl, pl = L
            rr, vxr, vyr, vzr, pr = R
            en_l = T(0.5) * (rl * (vxl * vxl + vyl * vyl + vzl * vzl)) + (pl / gm1)
            en_r = T(0.5) * (rr * (vxr * vxr + vyr * vyr + vzr * vzr)) + (pr / gm1)
            rs = (rl + rr) / T(2.0)
            mx = (rl * vxl + rr * vxr) / T(2.0)
            my = (rl * vyl + rr * vyr) / T(2.0)
            mz = (rl * vzl + rr * vzr) / T(2.0)
            es = T(0.5) * (en_l + en_r)
            ps = gm1 * (es - T(0.5) * (mx * mx + my * my + mz * mz) / rs)
            f1 = (mx * mx / rs) + ps
            f2 = mx * my / rs
            f3 = mx * mz / rs
            f4 = (es + ps) * (mx / rs)
            if CONDUCTING_WALL in self.bcs:
                f4 = self._wall_heat(f4, X[0][c_sl], X[4][c_sl])
            if self.gravity and dim == 2:
                nz = self.n[2]
                k = np.arange(1, nz - 1, dtype=self.dtype)[None, None, :]
                h = (T(nz) - T(2.0) * T(2)) * ds - (k - T(2.0)) * ds
                f1 = f1 + T(1.0) * rs * self.g * h
                f4 = f4 + T(0.5) * rs * (vxl + vxr) * self.g * h
            cl = np.sqrt(gam * pl / rl) + np.abs(vxl)
            cr = np.sqrt(gam * pr / rr) + np.abs(vxr)
            cs = np.fmax(cl, cr)
            out = [
                mx - T(0.5) * cs * (rl - rr),
                f1 - cs * (rl * vxl - rr * vxr) / T(2.0),
                f2 - cs * (rl * vyl - rr * vyr) / T(2.0),
                f3 - cs * (rl * vzl - rr * vzr) / T(2.0),
                f4 - cs * (en_l - en_r) / T(2.0),
            ]
        for slot, src in enumerate(perm):
            self.flux[src][c_sl + (dim,)] = out[slot] * ds

    def _wall_heat(self, f4, rho, p):
        """Conducting walls (src/cu/include/kernels.h:561-661): Q / V added to
        the energy flux of the faces whose lower cell has index 1 on a lower
        conducting face's axis, or n - 2 on an upper one's, lower faces first;
        t_in = p / (RS rho) of that lower cell."""
        T = self.dtype.type
        ds = self.ds
        t_in = p / (T(np.float32(287.0)) * rho)
        hc = T(np.float32(10.0)) - T(0.0) + T(np.float32(10.0)) * np.sqrt(T(0.0))
        S = ds * ds
        V = ds * ds * ds
        d, kappa = T(np.float32(0.008)), T(np.float32(0.2))
        Q = (T(np.float32(273.0)) - t_in) * (S / ((d / kappa) + (T(np.float32(1.0)) / hc)))
        q = Q / V
        for up in (0, 1):
            for ax in range(3):
                if self.bcs[2 * ax + up] != CONDUCTING_WALL:
                    continue
                pos = f4.shape[ax] - 1 if up else 0   # cell index n - 2 or 1
                sl = _sl(ax, pos)
                f4[sl] = f4[sl] + q[sl]
        return f4

    def _add_fluxes(self, dt):
        c = (slice(1, -1),) * 3
        xm = (slice(0, -2), slice(1, -1), slice(1, -1))
        ym = (slice(1, -1), slice(0, -2), slice(1, -1))
        zm = (slice(1, -1), slice(1, -1), slice(0, -2))
        for f in range(5):
            F = self.flux[f]
            self.cons[f][c] -= dt * self.ds * (F[c + (0,)] - F[xm + (0,)] + F[c + (1,)] - F[ym + (1,)]
                                               + F[c + (2,)] - F[zm + (2,)])

    def compute_step(self):
        self.calc_primitives()
        self._prim_ghosts(self.prim)
        dt = self.calc_timestep()
        for f in range(5):
            self._gradient(self.prim[f], self.grad[f])
        for f in range(5):
            self._bc_scalar_like(self.grad[f])
        self._extrapolate(dt)
        self._prim_ghosts(self.xtr)
        self._flux(0, (0, 1, 2, 3, 4))
        self._flux(1, (0, 2, 1, 3, 4))
        self._flux(2, (0, 3, 1, 2, 4))
        for f in range(5):
            self._bc_scalar_like(self.flux[f])
        self._add_fluxes(dt)
        return dt
