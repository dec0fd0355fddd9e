"""NumPy model of the fused kernel's boundary algorithm (test helper).

The CUDA step does not store gradients, predicted states or fluxes, so it
cannot copy their ghost layers the way the reference does
(src/rs/src/boundaries.rs:5-195, grid.rs:153-167).  It keeps only the
ghosted conserved state, fills its ghosts by composing the per-axis source
rules, and reproduces the effect of the reference's derived-array ghost
copies with three local rules:
  PERIODIC  layer-1 ghost slopes/predictions computed from ghost primitives;
  OUTFLOW   layer-1 ghost takes slopes and prediction of the first interior
            cell, and the lower face's flux equals the next face's;
  WALL      layer-1 ghost slopes computed from ghost primitives, prediction
            = mirror of the first interior cell's.
This model applies the same rules with the oracle's arithmetic so the tests
can show, on the CPU and bit for bit, that the rules are equivalent to the
reference's array copies.
"""
from __future__ import annotations

import numpy as np

PERIODIC, OUTFLOW, WALL = 0, 1, 2


def axis_source(g, n, lo, hi):
    """Interior source index of ghosted index g and whether it is a mirror."""
    if 2 <= g <= n - 3:
        return g, False
    if g < 2:
        if lo == PERIODIC:
            return (n - 4 if g == 0 else n - 3), False
        if lo == OUTFLOW:
            return 2, False
        return (2 if g == 1 else 3), True
    if hi == PERIODIC:
        return (2 if g == n - 2 else 3), False
    if hi == OUTFLOW:
        return n - 3, False
    return (n - 3 if g == n - 2 else n - 4), True


def fill_ghosts(u, bcs):
    """Ghost fill of a 5-field state by the composed source rule."""
    n = u[0].shape
    src = []
    for a in range(3):
        idx = np.empty(n[a], dtype=np.int64)
        flip = np.zeros(n[a], dtype=bool)
        for g in range(n[a]):
            idx[g], flip[g] = axis_source(g, n[a], bcs[2 * a], bcs[2 * a + 1])
        src.append((idx, flip))
    (ix, fx), (iy, fy), (iz, fz) = src
    out = [f[np.ix_(ix, iy, iz)].copy() for f in u]
    for a, fl in enumerate((fx, fy, fz)):
        shape = [1, 1, 1]
        shape[a] = -1
        sign = np.where(fl, -1.0, 1.0).reshape(shape).astype(u[0].dtype)
        out[1 + a] = out[1 + a] * sign
    return out


class FusedModel:
    def __init__(self, shape, ds, bcs, gamma, cfl, dtype=np.float64, limiter=0):
        self.shape = tuple(shape)
        self.n = tuple(s + 4 for s in shape)
        self.dtype = np.dtype(dtype)
        T = self.dtype.type
        self.ds, self.gamma, self.cfl = T(ds), T(gamma), T(cfl)
        self.bcs = tuple(bcs)
        self.limiter = limiter
        self.cons = None

    def set_conserved(self, cons):
        self.cons = fill_ghosts([np.asarray(c, dtype=self.dtype) for c in cons], self.bcs)

    def _prims(self, u):
        T = self.dtype.type
        V = self.ds * self.ds * self.ds
        M, Mx, My, Mz, E = u
        with np.errstate(all="ignore"):
            r = M / V
            vx = Mx / (r * V)
            vy = My / (r * V)
            vz = Mz / (r * V)
            p = (E / V - T(0.5) * r * (vx * vx + vy * vy + vz * vz)) * (self.gamma - T(1.0))
        return [r, vx, vy, vz, p]

    def _slopes(self, q, i, j, k):
        """Slopes (3 axes) of one field at cell (i, j, k) as the oracle does."""
        T = self.dtype.type
        out = []
        for d, (di, dj, dk) in enumerate(((1, 0, 0), (0, 1, 0), (0, 0, 1))):
            qm, q0, qp = q[i - di, j - dj, k - dk], q[i, j, k], q[i + di, j + dj, k + dk]
            if self.limiter == 0:
                out.append((qp - qm) / (T(2.0) * self.ds))
            else:
                a = (q0 - qm) / self.ds
                b = (qp - q0) / self.ds
                out.append((a if abs(a) < abs(b) else b) if a * b > 0 else T(0.0))
        return out

    def _cell(self, P, c):
        """Slopes and prediction computed at cell c from the primitives."""
        T = self.dtype.type
        g = [self._slopes(P[f], *c) for f in range(5)]
        rho, vx, vy, vz, p = (P[f][c] for f in range(5))
        (drx, dry, drz), (dxx, dxy, dxz), (dyx, dyy, dyz), (dzx, dzy, dzz), (dpx, dpy, dpz) = g
        h = T(0.5) * self.dt
        with np.errstate(all="ignore"):
            x = [rho - h * (vx * drx + rho * dxx + vy * dry + rho * dyy + vz * drz + rho * dzz),
                 vx - h * (vx * dxx + vy * dxy + vz * dxz + (T(1.0) / rho) * dpx),
                 vy - h * (vx * dyx + vy * dyy + vz * dyz + (T(1.0) / rho) * dpy),
                 vz - h * (vx * dzx + vy * dzy + vz * dzz + (T(1.0) / rho) * dpz),
                 p - h * (self.gamma * p * (dxx + dyy + dzz) + vx * dpx + vy * dpy + vz * dpz)]
        return g, x

    def _state(self, P, c):
        """Slopes and prediction the fused kernel uses for cell c (interior or
        layer-1 ghost on one axis), by the boundary rules above."""
        n = self.n
        for a in range(3):
            if c[a] in (1, n[a] - 2):
                upper = c[a] == n[a] - 2
                bc = self.bcs[2 * a + upper]
                nb = list(c)
                nb[a] = n[a] - 3 if upper else 2
                nb = tuple(nb)
                if bc == OUTFLOW:
                    return self._cell(P, nb)
                if bc == WALL:
                    g, _ = self._cell(P, c)
                    _, x = self._cell(P, nb)
                    x = list(x)
                    x[1 + a] = -x[1 + a]
                    return g, x
                return self._cell(P, c)
        return self._cell(P, c)

    def _flux(self, lo, hi, dim):
        """Face flux with the oracle's arithmetic (lo: lower cell (g, x))."""
        T = self.dtype.type
        ds, gam = self.ds, self.gamma
        perm = {0: (0, 1, 2, 3, 4), 1: (0, 2, 1, 3, 4), 2: (0, 3, 1, 2, 4)}[dim]
        half = ds / T(2.0)
        gl, xl = lo
        gu, xu = hi
        L = [xu[perm[s]] - gu[perm[s]][dim] * half for s in range(5)]
        R = [xl[perm[s]] + gl[perm[s]][dim] * half for s in range(5)]
        rl, vxl, vyl, vzl, pl = L
        rr, vxr, vyr, vzr, pr = R
        gm1 = gam - T(1.0)
        with np.errstate(all="ignore"):
            en_l = T(0.5) * (rl * (vxl * vxl + vyl * vyl + vzl * vzl)) + (pl / gm1)
            en_r = T(0.5) * (rr * (vxr * vxr + vyr * vyr + vzr * vzr)) + (pr / gm1)
            rs = (rl + rr) / T(2.0)
            mx = (rl * vxl + rr * vxr) / T(2.0)
            my = (rl * vyl + rr * vyr) / T(2.0)
            mz = (rl * vzl + rr * vzr) / T(2.0)
            es = T(0.5) * (en_l + en_r)
            ps = gm1 * (es - T(0.5) * (mx * mx + my * my + mz * mz) / rs)
            cs = max(np.sqrt(gam * pl / rl) + abs(vxl), np.sqrt(gam * pr / rr) + abs(vxr))
            out = [mx - T(0.5) * cs * (rl - rr),
                   ((mx * mx / rs) + ps) - cs * (rl * vxl - rr * vxr) / T(2.0),
                   (mx * my / rs) - cs * (rl * vyl - rr * vyr) / T(2.0),
                   (mx * mz / rs) - cs * (rl * vzl - rr * vzr) / T(2.0),
                   ((es + ps) * (mx / rs)) - cs * (en_l - en_r) / T(2.0)]
        F = [None] * 5
        for s in range(5):
            F[perm[s]] = out[s] * ds
        return F

    def step(self):
        T = self.dtype.type
        P = self._prims(self.cons)
        n = self.n
        inner = (slice(2, -2),) * 3
        with np.errstate(all="ignore"):
            w = self.ds / (np.sqrt(self.gamma * P[4][inner] / P[0][inner])
                           + np.sqrt(P[1][inner] ** 2 + P[2][inner] ** 2 + P[3][inner] ** 2))
        self.dt = self.cfl * (T(1.0) if np.isnan(w).any() else w.min())
        cache = {}

        def st(c):
            if c not in cache:
                cache[c] = self._state(P, c)
            return cache[c]

        new = [u.copy() for u in self.cons]
        for i in range(2, n[0] - 2):
            for j in range(2, n[1] - 2):
                for k in range(2, n[2] - 2):
                    c = (i, j, k)
                    div = [T(0.0)] * 5
                    terms = []
                    for d in range(3):
                        e = [0, 0, 0]
                        e[d] = 1
                        up = (i + e[0], j + e[1], k + e[2])
                        dn = (i - e[0], j - e[1], k - e[2])
                        Fh = self._flux(st(c), st(up), d)
                        if c[d] == 2 and self.bcs[2 * d] == OUTFLOW:
                            Fl = Fh
                        else:
                            Fl = self._flux(st(dn), st(c), d)
                        terms.append((Fh, Fl))
                    for f in range(5):
                        (h0, l0), (h1, l1), (h2, l2) = terms
                        div[f] = h0[f] - l0[f] + h1[f] - l1[f] + h2[f] - l2[f]
                        new[f][c] = self.cons[f][c] - self.dt * self.ds * div[f]
        self.cons = fill_ghosts(new, self.bcs)
        return self.dt
