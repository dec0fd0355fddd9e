"""Physics checks of the oracle (the restated reference step), beside the
parity tests: the reference pins nothing, so its restatement is held to the
mathematics as well.  The GPU kernels match the oracle (test_parity_gpu), so
they inherit these properties.

- Sod shock tube against the exact Riemann solution: the L1 density error
  falls under refinement.
- Isentropic vortex (periodic, advected by (1, 1)): after one period the
  state returns to the initial one, with an error that falls under
  refinement.
"""
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
sys.path.insert(0, str(ROOT / "oracle"))
sys.path.insert(0, str(Path(__file__).resolve().parent))

import pyoracle  # noqa: E402
import riemann_exact as rx  # noqa: E402
from deepgreen import setups  # noqa: E402

GAMMA = 1.4
SOD_L, SOD_R = (1.0, 0.0, 1.0), (0.125, 0.0, 0.1)


def test_exact_solver_known_answer():
    # Sod's problem (gamma 1.4): star pressure 0.30313, star velocity 0.92745
    # (the published values of the exact solution)
    p, u = rx.star_state(SOD_L, SOD_R, GAMMA)
    assert p == pytest.approx(0.30313, abs=5e-6) and u == pytest.approx(0.92745, abs=5e-6)
    rho, vel, pres = rx.sample(SOD_L, SOD_R, GAMMA, np.array([-10.0, 10.0, u - 1e-9, u + 1e-9]))
    assert rho[0] == 1.0 and rho[1] == 0.125 and pres[2] == pres[3] == pytest.approx(p)
    assert vel[2] == vel[3] == pytest.approx(u) and rho[2] > rho[3]   # density jumps at the contact


def _run_to(o, t_end):
    t = 0.0
    while t < t_end:
        t += float(o.step(1)[0])
    return t


def test_sod_converges_to_the_exact_solution():
    errs = []
    for n in (64, 128, 256):
        prim, ds, bcs = setups.sod(n, ny=2, nz=2)
        o = pyoracle.Oracle((n, 2, 2), ds, bcs, gamma=GAMMA, cfl=0.4, limiter=1, threads=pyoracle.SERIAL)
        o.set_primitives(prim)
        t = _run_to(o, 0.15)
        cons = o.conserved()
        o.close()
        rho = cons[0][2:-2, 2:-2, 2:-2] / ds ** 3
        assert np.ptp(rho, axis=(1, 2)).max() == 0.0     # stays one-dimensional
        x = (np.arange(n) + 0.5) * ds
        exact = rx.sample(SOD_L, SOD_R, GAMMA, (x - 0.5) / t)
        errs.append(np.mean(np.abs(rho[:, 0, 0] - exact[0])))
    # measured: 0.0128, 0.0067, 0.0039
    assert errs[0] < 0.02 and errs[1] < 0.6 * errs[0] and errs[2] < 0.7 * errs[1], errs


def test_vortex_returns_after_one_period_with_falling_error():
    errs = []
    for n in (32, 64, 128):
        prim, ds, bcs = setups.isentropic_vortex(n, gamma=GAMMA, nz=2)
        o = pyoracle.Oracle((n, n, 2), ds, bcs, gamma=GAMMA, cfl=0.4, limiter=1,
                            threads=pyoracle.ALL_PARALLEL)
        o.set_primitives(prim)
        rho0 = o.conserved()[0][2:-2, 2:-2, 2] / ds ** 3
        _run_to(o, 10.0)   # the box is 10 wide, the flow (1, 1): one period
        rho = o.conserved()[0][2:-2, 2:-2, 2] / ds ** 3
        o.close()
        errs.append(np.mean(np.abs(rho - rho0)))
    # measured: 0.0202, 0.0101, 0.0031
    assert errs[0] < 0.03 and errs[1] < 0.6 * errs[0] and errs[2] < 0.5 * errs[1], errs
