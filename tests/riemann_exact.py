"""Exact solution of the 1-D Riemann problem for the Euler equations of an
ideal gas (test infrastructure: the physics check of the oracle on the Sod
shock tube).

The published method (E. F. Toro, "Riemann Solvers and Numerical Methods for
Fluid Dynamics", ch. 4): the star-region pressure is the root of
f_L(p) + f_R(p) + (u_R - u_L) = 0, where f_K is the shock (Rankine-Hugoniot)
branch for p > p_K and the rarefaction (isentropic) branch otherwise; the
star velocity follows, and the solution at x/t is sampled from the wave
pattern (shocks, rarefaction fans, contact).
"""
from __future__ import annotations

import math

import numpy as np


def _f(p, rho, pk, ck, g):
    """Velocity jump across the wave of one side and its derivative in p."""
    if p > pk:
        a = 2.0 / ((g + 1.0) * rho)
        b = (g - 1.0) / (g + 1.0) * pk
        s = math.sqrt(a / (p + b))
        return (p - pk) * s, s * (1.0 - 0.5 * (p - pk) / (b + p))
    r = p / pk
    e = (g - 1.0) / (2.0 * g)
    return 2.0 * ck / (g - 1.0) * (r ** e - 1.0), 1.0 / (rho * ck) * r ** (-(g + 1.0) / (2.0 * g))


def star_state(left, right, g):
    """(p*, u*) of the Riemann problem left=(rho, u, p), right=(rho, u, p)."""
    rl, ul, pl = left
    rr, ur, pr = right
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    if 2.0 * (cl + cr) / (g - 1.0) <= ur - ul:
        raise ValueError("the data create a vacuum")
    p = max(1e-8, 0.5 * (pl + pr))
    for _ in range(100):
        fl, dl = _f(p, rl, pl, cl, g)
        fr, dr = _f(p, rr, pr, cr, g)
        step = (fl + fr + ur - ul) / (dl + dr)
        pn = max(1e-8, p - step)
        if abs(pn - p) <= 1e-14 * (pn + p):
            p = pn
            break
        p = pn
    fl, _ = _f(p, rl, pl, cl, g)
    fr, _ = _f(p, rr, pr, cr, g)
    return p, 0.5 * (ul + ur) + 0.5 * (fr - fl)


def sample(left, right, g, xi):
    """(rho, u, p) at the similarity coordinates xi = (x - x0) / t."""
    rl, ul, pl = left
    rr, ur, pr = right
    ps, us = star_state(left, right, g)
    cl, cr = math.sqrt(g * pl / rl), math.sqrt(g * pr / rr)
    gm = (g - 1.0) / (g + 1.0)
    out = np.empty((3, len(xi)))
    for i, s in enumerate(np.asarray(xi, dtype=float)):
        if s <= us:   # left of the contact
            if ps > pl:   # left shock
                sl = ul - cl * math.sqrt((g + 1.0) / (2.0 * g) * ps / pl + (g - 1.0) / (2.0 * g))
                st = (rl * ((ps / pl + gm) / (gm * ps / pl + 1.0)), us, ps)
                out[:, i] = (rl, ul, pl) if s <= sl else st
            else:         # left rarefaction
                csl = cl * (ps / pl) ** ((g - 1.0) / (2.0 * g))
                if s <= ul - cl:
                    out[:, i] = (rl, ul, pl)
                elif s >= us - csl:
                    out[:, i] = (rl * (ps / pl) ** (1.0 / g), us, ps)
                else:
                    u = 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * ul + s)
                    c = 2.0 / (g + 1.0) * (cl + 0.5 * (g - 1.0) * (ul - s))
                    rho = rl * (c / cl) ** (2.0 / (g - 1.0))
                    out[:, i] = (rho, u, pl * (c / cl) ** (2.0 * g / (g - 1.0)))
        else:         # right of the contact
            if ps > pr:   # right shock
                sr = ur + cr * math.sqrt((g + 1.0) / (2.0 * g) * ps / pr + (g - 1.0) / (2.0 * g))
                st = (rr * ((ps / pr + gm) / (gm * ps / pr + 1.0)), us, ps)
                out[:, i] = (rr, ur, pr) if s >= sr else st
            else:         # right rarefaction
                csr = cr * (ps / pr) ** ((g - 1.0) / (2.0 * g))
                if s >= ur + cr:
                    out[:, i] = (rr, ur, pr)
                elif s <= us + csr:
                    out[:, i] = (rr * (ps / pr) ** (1.0 / g), us, ps)
                else:
                    u = 2.0 / (g + 1.0) * (-cr + 0.5 * (g - 1.0) * ur + s)
                    c = 2.0 / (g + 1.0) * (cr - 0.5 * (g - 1.0) * (ur - s))
                    rho = rr * (c / cr) ** (2.0 / (g - 1.0))
                    out[:, i] = (rho, u, pr * (c / cr) ** (2.0 * g / (g - 1.0)))
    return out
