"""The boundary rules the fused CUDA kernel applies on the fly (it keeps no
gradient, prediction or flux arrays) give bit-for-bit the reference's
results with its array-copy ghost updates (CPU check of the derivation)."""
import numpy as np
import pytest

import pyoracle
from conftest import INTERIOR, random_primitives
from fused_model import FusedModel

P, O, W = 0, 1, 2


@pytest.mark.parametrize("bcs", [(P,) * 6, (O,) * 6, (W,) * 6, (W, W, P, P, O, O), (P, P, W, W, O, O),
                                 (O, W, W, O, P, P), (W, O, O, W, W, W)])
@pytest.mark.parametrize("limiter", [0, 1])
@pytest.mark.parametrize("shape", [(4, 5, 3), (2, 3, 2)])
def test_fused_boundary_rules_equal_reference_ghost_copies(bcs, limiter, shape):
    o = pyoracle.Oracle(shape, 0.1, bcs, gamma=1.4, cfl=0.4, limiter=limiter)
    o.set_primitives(random_primitives(shape, 5))
    m = FusedModel(shape, 0.1, bcs, 1.4, 0.4, limiter=limiter)
    m.set_conserved(o.conserved())
    for _ in range(3):
        assert o.step(1)[0] == m.step()
        c = o.conserved()
        for f in range(5):
            np.testing.assert_array_equal(m.cons[f][INTERIOR], c[f][INTERIOR])
