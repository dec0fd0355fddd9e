"""GPU parity through the C++ mirror of the reference API
(include/deepgreen.hpp, driven by tests/cpp/grid_api.cpp the way main.rs
drives the Rust one): the FP64 step after calc_conserved and six
compute_step calls matches the FP64 oracle to 1e-12 relative L1 per
conserved field, dt to 1e-13."""
import subprocess

import numpy as np
import pytest

import cpp_api
import pyoracle
from conftest import random_primitives, rel_l1

pytestmark = pytest.mark.gpu

P, O, W = 0, 1, 2


@pytest.mark.parametrize("bcs,limiter", [((W, W, P, P, O, O), 1), ((O,) * 6, 0)])
def test_cpp_mirror_matches_the_oracle(tmp_path, bcs, limiter):
    shape, ds, steps = (13, 11, 45), 0.05, 6
    prim = random_primitives(shape, 7 + limiter)
    inp, out = tmp_path / "prim.bin", tmp_path / "out.bin"
    np.concatenate([np.ascontiguousarray(a, dtype=np.float64).ravel() for a in prim]).tofile(inp)
    exe = cpp_api.build(tmp_path)
    args = [str(exe), "run", *map(str, shape), repr(ds), str(limiter), str(steps), *map(str, bcs), str(inp),
            str(out)]
    r = subprocess.run(args, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stderr
    n = tuple(s + 4 for s in shape)
    raw = np.fromfile(out, dtype=np.float64)
    assert raw.size == steps + 5 * int(np.prod(n))
    dts, cons = raw[:steps], raw[steps:].reshape((5,) + n)

    o = pyoracle.Oracle(shape, ds, bcs, gamma=1.4, cfl=0.4, limiter=limiter, threads=pyoracle.ALL_PARALLEL)
    o.set_primitives(prim)
    ref_dts = o.step(steps)
    ref = o.conserved()
    o.close()
    np.testing.assert_allclose(dts, ref_dts, rtol=1e-13)
    errs = [rel_l1(cons[f], ref[f]) for f in range(5)]
    assert max(errs) <= 1e-12, errs
