"""GPU parity: the CUDA step (through the C ABI) against the CPU oracle.

Tolerances (per conserved field, relative L1 = sum|a-b| / sum|b| over the
interior, against the FP64 oracle):
    FP64 kernel <= 1e-12,   FP32 kernel <= 1e-5.
The reference-rounding policy (FP64, or FP32 on request) is further checked
to be bit-identical to the oracle of the same precision.  On the 200-step
Kelvin-Helmholtz run the transverse momenta are noise-level fields that the
instability amplifies; there the FP32 bound is: mass and energy <= 1e-5, and
every field within 2x of the error of the reference's own f32 arithmetic
(the oracle's float instantiation).
"""
from pathlib import Path

import numpy as np
import pytest

import pyoracle
from conftest import INTERIOR, random_primitives, rel_l1
from deepgreen import capi, setups

pytestmark = pytest.mark.gpu

P, O, W = 0, 1, 2
TOL = {capi.F64: 1e-12, capi.F32: 1e-5}
DT_TOL = {capi.F64: 1e-13, capi.F32: 1e-6}
BC_SETS = [(P,) * 6, (O,) * 6, (W,) * 6, (W, W, P, P, O, O), (P, P, W, W, O, O), (O, W, W, O, P, P)]
GOLD = Path(__file__).parent / "golden" / "oracle_cases.npz"


def gpu_run(shape, ds, bcs, prim, steps, precision, limiter=1, gamma=1.4, cfl=0.4, gravity=False, chunk=0,
            rounding=capi.ROUNDING_DEFAULT):
    ctx = capi.Context(shape, ds, bcs, gamma=gamma, cfl=cfl, limiter=limiter, precision=precision,
                       gravity=gravity, rounding=rounding)
    if chunk:
        ctx.set_chunk(chunk)
    ctx.set_primitives([np.asarray(a, dtype=ctx.dtype) for a in prim])
    dts = ctx.compute_step(steps)
    cons = ctx.get_conserved()
    return ctx, dts, cons


def oracle_run(shape, ds, bcs, prim, steps, limiter=1, gamma=1.4, cfl=0.4, gravity=False, dtype=np.float64):
    o = pyoracle.Oracle(shape, ds, bcs, gamma=gamma, cfl=cfl, limiter=limiter, gravity=gravity,
                        threads=pyoracle.ALL_PARALLEL, dtype=dtype)
    o.set_primitives([np.asarray(a, dtype=dtype) for a in prim])
    dts = o.step(steps)
    return o, dts, o.conserved()


def assert_parity(cons, ref, dts, ref_dts, precision, label=""):
    errs = [rel_l1(cons[f], ref[f]) for f in range(5)]
    assert max(errs) <= TOL[precision], f"{label} rel-L1 per field {errs}"
    np.testing.assert_allclose(dts, ref_dts, rtol=DT_TOL[precision], err_msg=label)
    return errs


@pytest.mark.parametrize("precision", [capi.F64, capi.F32])
def test_golden_cases(precision):
    import sys
    sys.path.insert(0, str(GOLD.parent))
    import make_golden
    gold = np.load(GOLD)
    for name, shape, bcs, lim, grav, steps, seed in make_golden.CASES:
        prim = random_primitives(shape, seed)
        _, dts, cons = gpu_run(shape, 0.1, bcs, prim, steps, precision, limiter=lim, gravity=bool(grav))
        ref = [np.pad(gold[f"{name}/cons"][f], 2) for f in range(5)]
        assert_parity(cons, ref, dts, gold[f"{name}/dts"], precision, name)


@pytest.mark.parametrize("bcs", BC_SETS)
@pytest.mark.parametrize("limiter", [0, 1])
@pytest.mark.parametrize("precision", [capi.F64, capi.F32])
def test_bc_matrix_ragged_tiles(bcs, limiter, precision):
    # y not a multiple of the tile rows, z spans two ragged warp tiles,
    # several x-chunks per column
    shape = (13, 11, 45)
    prim = random_primitives(shape, 100 + limiter)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 6, limiter=limiter)
    _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 6, precision, limiter=limiter, chunk=4)
    assert_parity(cons, ref, dts, ref_dts, precision, str(bcs))


def test_kelvin_helmholtz_64_200_steps_fp64():
    """The CPU-runnable workload: 64^3 periodic KH, gamma 1.4, minmod,
    CFL 0.4, 200 steps, FP64 against the FP64 oracle."""
    prim, ds, bcs = setups.kelvin_helmholtz(64, seed=1)
    _, ref_dts, ref = oracle_run((64,) * 3, ds, bcs, prim, 200)
    _, dts, cons = gpu_run((64,) * 3, ds, bcs, prim, 200, capi.F64)
    errs = assert_parity(cons, ref, dts, ref_dts, capi.F64, "kh64")
    print("kh64 fp64 rel-L1 per field", errs)


def test_kelvin_helmholtz_64_200_steps_fp32():
    prim, ds, bcs = setups.kelvin_helmholtz(64, seed=1)
    _, ref_dts, ref = oracle_run((64,) * 3, ds, bcs, prim, 200)
    _, ref32_dts, ref32 = oracle_run((64,) * 3, ds, bcs, prim, 200, dtype=np.float32)
    _, dts, cons = gpu_run((64,) * 3, ds, bcs, prim, 200, capi.F32)
    errs = [rel_l1(cons[f], ref[f]) for f in range(5)]
    ref32_errs = [rel_l1(ref32[f], ref[f]) for f in range(5)]
    print("kh64 fp32 rel-L1 per field", errs, "reference f32 arithmetic", ref32_errs)
    assert errs[0] <= 1e-5 and errs[4] <= 1e-5, errs
    for f in range(5):
        assert errs[f] <= 2.0 * ref32_errs[f] + 1e-7, (f, errs, ref32_errs)
    # dt follows the fastest cell, which the amplified noise moves: bound
    # its drift by the reference f32 arithmetic's own drift
    drift = np.max(np.abs(dts / ref_dts - 1))
    ref_drift = np.max(np.abs(ref32_dts / ref_dts - 1))
    assert drift <= 2.0 * ref_drift + 1e-6, (drift, ref_drift)


@pytest.mark.parametrize("case", ["sod", "vortex"])
@pytest.mark.parametrize("precision", [capi.F64, capi.F32])
def test_sod_and_vortex_48(case, precision):
    if case == "sod":
        prim, ds, bcs = setups.sod(48)
    else:
        prim, ds, bcs = setups.isentropic_vortex(48)
    _, ref_dts, ref = oracle_run((48,) * 3, ds, bcs, prim, 40)
    _, dts, cons = gpu_run((48,) * 3, ds, bcs, prim, 40, precision)
    assert_parity(cons, ref, dts, ref_dts, precision, case)


def test_gravity_wall_case():
    shape = (9, 10, 40)
    prim = random_primitives(shape, 33)
    bcs = (P, P, O, O, W, W)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 8, limiter=0, gravity=True)
    _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 8, capi.F64, limiter=0, gravity=True)
    assert_parity(cons, ref, dts, ref_dts, capi.F64, "gravity")


def test_tiling_does_not_change_results():
    """Every cell is computed by the same arithmetic whatever the tiling:
    results are bitwise identical across x-chunk sizes."""
    shape = (24, 17, 40)
    prim = random_primitives(shape, 44)
    outs = []
    for chunk in (0, 1, 5, 24):
        _, dts, cons = gpu_run(shape, 0.05, BC_SETS[3], prim, 5, capi.F32, chunk=chunk)
        outs.append((dts, cons))
    for dts, cons in outs[1:]:
        np.testing.assert_array_equal(dts, outs[0][0])
        for f in range(5):
            np.testing.assert_array_equal(cons[f][INTERIOR], outs[0][1][f][INTERIOR])


def test_deterministic_sums_and_state():
    shape = (20, 20, 20)
    prim = random_primitives(shape, 55)
    a = gpu_run(shape, 0.05, BC_SETS[0], prim, 4, capi.F64)
    b = gpu_run(shape, 0.05, BC_SETS[0], prim, 4, capi.F64)
    np.testing.assert_array_equal(a[0].conservation_sums(), b[0].conservation_sums())
    for f in range(5):
        np.testing.assert_array_equal(a[2][f], b[2][f])


def test_conservation_sums_and_periodic_conservation():
    prim, ds, bcs = setups.kelvin_helmholtz(32, seed=4)
    ctx = capi.Context((32,) * 3, ds, bcs, gamma=1.4, cfl=0.4, limiter=1, precision=capi.F64)
    ctx.set_primitives(prim)
    s0 = ctx.conservation_sums()
    c0 = ctx.get_conserved()
    np.testing.assert_allclose(s0, [c[INTERIOR].sum() for c in c0], rtol=1e-13)
    ctx.compute_step(50)
    s1 = ctx.conservation_sums()
    c1 = ctx.get_conserved()
    np.testing.assert_allclose(s1, [c[INTERIOR].sum() for c in c1], rtol=1e-12, atol=1e-16)
    for f in (0, 1, 4):
        assert abs(s1[f] - s0[f]) <= 1e-12 * abs(s0[f])


def test_ghost_cells_follow_boundary_rules():
    """Downloaded ghosts are the images the reference's ghost fill makes."""
    from fused_model import fill_ghosts
    shape = (10, 9, 11)
    prim = random_primitives(shape, 66)
    for bcs in BC_SETS:
        _, _, cons = gpu_run(shape, 0.05, bcs, prim, 2, capi.F64)
        ref = fill_ghosts(cons, bcs)
        for f in range(5):
            np.testing.assert_array_equal(cons[f], ref[f])


def test_primitives_are_pre_step_state_like_reference():
    """After compute_step the reference's grid.primitives hold the state the
    step started from, ghosts filled (physics.rs:597-598)."""
    shape = (8, 9, 10)
    prim = random_primitives(shape, 77)
    bcs = BC_SETS[5]
    o, _, _ = oracle_run(shape, 0.05, bcs, prim, 3)
    ctx, _, _ = gpu_run(shape, 0.05, bcs, prim, 3, capi.F64)
    got = ctx.get_primitives()
    want = o.primitives()
    for f in range(5):
        np.testing.assert_allclose(got[f], want[f], rtol=1e-12, atol=1e-13)


def test_nonfinite_state_flags_and_cfl_fallback():
    shape = (8, 8, 8)
    prim = random_primitives(shape, 88)
    prim[4][5, 5, 5] = -1.0
    ctx, dts, _ = gpu_run(shape, 0.1, BC_SETS[0], prim, 1, capi.F64, cfl=0.4)
    assert dts[0] == pytest.approx(0.4)
    assert ctx.status() & capi.STATUS_NONFINITE


def test_reference_shaped_api():
    """Simulation / SimulationGrid / calc_conserved / compute_step used the
    way the reference's main.rs uses them."""
    from deepgreen import BoundaryType as BT, Simulation, SimulationGrid, calc_conserved, compute_step
    sim = Simulation.new(16, 12, 20, 1.0 / 16, (BT.OUTFLOW,) * 6, gamma=1.4, cfl=0.4, limiter=1,
                         precision=capi.F64)
    grid = SimulationGrid.new(sim)
    prim, ds, _ = setups.sod(16, ny=12, nz=20)
    for dst, src in zip(grid.primitives.fields(), prim):
        dst[...] = src
    calc_conserved(grid)
    dt = compute_step(sim, grid)
    o, ref_dts, ref = oracle_run((16, 12, 20), ds, (O,) * 6, prim, 1)
    assert dt == pytest.approx(ref_dts[0], rel=1e-13)
    got = grid.conserved.fields()
    for f in range(5):
        assert rel_l1(got[f], ref[f]) <= 1e-12


# ---------------------------------------------------------------------------
# Reference rounding: bit-identical to the oracle of the same precision
# ---------------------------------------------------------------------------
@pytest.mark.parametrize("precision,dtype", [(capi.F64, np.float64), (capi.F32, np.float32)])
def test_reference_rounding_bitwise_golden_and_matrix(precision, dtype):
    import sys
    sys.path.insert(0, str(GOLD.parent))
    import make_golden
    cases = [(name, shape, bcs, lim, grav, steps, random_primitives(shape, seed), 0.1)
             for name, shape, bcs, lim, grav, steps, seed in make_golden.CASES]
    for i, bcs in enumerate(BC_SETS):
        shape = (13, 11, 45)
        cases.append((f"matrix{i}", shape, bcs, i % 2, 0, 5, random_primitives(shape, 200 + i), 0.05))
    for name, shape, bcs, lim, grav, steps, prim, ds in cases:
        _, ref_dts, ref = oracle_run(shape, ds, bcs, prim, steps, limiter=lim, gravity=bool(grav), dtype=dtype)
        _, dts, cons = gpu_run(shape, ds, bcs, prim, steps, precision, limiter=lim, gravity=bool(grav),
                               rounding=capi.ROUNDING_REFERENCE, chunk=3)
        np.testing.assert_array_equal(dts, ref_dts, err_msg=name)
        for f in range(5):
            np.testing.assert_array_equal(cons[f][INTERIOR], ref[f][INTERIOR], err_msg=f"{name} field {f}")


def test_reference_rounding_bitwise_kh64_fp64():
    prim, ds, bcs = setups.kelvin_helmholtz(64, seed=1)
    _, ref_dts, ref = oracle_run((64,) * 3, ds, bcs, prim, 200)
    _, dts, cons = gpu_run((64,) * 3, ds, bcs, prim, 200, capi.F64)
    np.testing.assert_array_equal(dts, ref_dts)
    for f in range(5):
        np.testing.assert_array_equal(cons[f][INTERIOR], ref[f][INTERIOR])


# ---------------------------------------------------------------------------
# The production (sweep) kernel's FP64 build: the same code as the FP32
# production kernel (tiles, halo warps, boundary switches), in double
# precision with fused arithmetic, against the FP64 oracle at 1e-12
# ---------------------------------------------------------------------------
def test_sweep_fp64_golden_cases():
    import sys
    sys.path.insert(0, str(GOLD.parent))
    import make_golden
    gold = np.load(GOLD)
    for name, shape, bcs, lim, grav, steps, seed in make_golden.CASES:
        prim = random_primitives(shape, seed)
        _, dts, cons = gpu_run(shape, 0.1, bcs, prim, steps, capi.F64, limiter=lim, gravity=bool(grav),
                               rounding=capi.ROUNDING_FAST)
        ref = [np.pad(gold[f"{name}/cons"][f], 2) for f in range(5)]
        assert_parity(cons, ref, dts, gold[f"{name}/dts"], capi.F64, name)


# shapes that exercise the sweep tiles: several y tiles (12 rows) with a
# ragged last one, two z tiles (64 columns) with an even and an odd ragged
# remainder, several x chunks
SWEEP_SHAPES = [(13, 11, 45), (9, 30, 100), (7, 13, 77)]


@pytest.mark.parametrize("shape", SWEEP_SHAPES)
@pytest.mark.parametrize("bcs", BC_SETS)
@pytest.mark.parametrize("limiter", [0, 1])
@pytest.mark.parametrize("precision", [capi.F64, capi.F32])
def test_sweep_bc_matrix_tiles(shape, bcs, limiter, precision):
    prim = random_primitives(shape, 300 + limiter)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 5, limiter=limiter)
    _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 5, precision, limiter=limiter, chunk=4,
                           rounding=capi.ROUNDING_FAST)
    assert_parity(cons, ref, dts, ref_dts, precision, f"{shape} {bcs}")


def test_sweep_fp64_gravity_and_kh64():
    shape = (9, 10, 40)
    prim = random_primitives(shape, 33)
    bcs = (P, P, O, O, W, W)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 8, limiter=0, gravity=True)
    _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 8, capi.F64, limiter=0, gravity=True,
                           rounding=capi.ROUNDING_FAST)
    assert_parity(cons, ref, dts, ref_dts, capi.F64, "gravity")
    # the 64^3 KH workload, 200 steps: mass, x-momentum and energy within
    # 1e-12; the transverse momenta are the noise-level fields the instability
    # amplifies (v_z is the seeded +-1e-3 noise alone), where unit-roundoff
    # differences of the fused arithmetic grow to a few 1e-12 (measured:
    # 6.4e-13 y, 2.5e-12 z); they are bounded by 1e-11
    prim, ds, bcs = setups.kelvin_helmholtz(64, seed=1)
    _, ref_dts, ref = oracle_run((64,) * 3, ds, bcs, prim, 200)
    _, dts, cons = gpu_run((64,) * 3, ds, bcs, prim, 200, capi.F64, rounding=capi.ROUNDING_FAST)
    errs = [rel_l1(cons[f], ref[f]) for f in range(5)]
    print("kh64 sweep fp64 rel-L1 per field", errs)
    assert max(errs[0], errs[1], errs[4]) <= 1e-12, errs
    assert max(errs[2], errs[3]) <= 1e-11, errs
    np.testing.assert_allclose(dts, ref_dts, rtol=1e-12)   # dt follows the amplified noise as well


# ---------------------------------------------------------------------------
# Conducting walls (DG_BC_CONDUCTING_WALL, the reference CUDA variant's heat
# source, src/cu/include/kernels.h:559-661) on every kernel: the reference
# rounding bit for bit against the oracle of the same precision, the sweep
# at the FP32 / FP64 tolerances.  A hot gas (t_in ~ 1200 K against the
# wall's 273 K) makes the heat term visible: the oracle with plain walls
# differs from the one with conducting walls far beyond the tolerances.
# ---------------------------------------------------------------------------
C = capi.CONDUCTING_WALL
COND_BCS = [(C, W, C, O, C, C), (W, C, P, P, C, O), (C, C, C, C, C, C)]


def _hot_gas(shape, seed):
    prim = random_primitives(shape, seed)
    return [prim[0] * 1.2, prim[1] * 50.0, prim[2] * 50.0, prim[3] * 50.0, prim[4] * 4e5]


@pytest.mark.parametrize("bcs", COND_BCS)
@pytest.mark.parametrize("precision,dtype", [(capi.F64, np.float64), (capi.F32, np.float32)])
def test_conducting_wall_reference_rounding_bitwise(bcs, precision, dtype):
    shape = (13, 11, 45)
    prim = _hot_gas(shape, 41)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 5, dtype=dtype)
    _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 5, precision, rounding=capi.ROUNDING_REFERENCE, chunk=3)
    np.testing.assert_array_equal(dts, ref_dts)
    for f in range(5):
        np.testing.assert_array_equal(cons[f][INTERIOR], ref[f][INTERIOR], err_msg=f"field {f}")


@pytest.mark.parametrize("shape", [(13, 11, 45), (9, 30, 100)])
@pytest.mark.parametrize("bcs", COND_BCS)
@pytest.mark.parametrize("precision", [capi.F64, capi.F32])
def test_conducting_wall_sweep(shape, bcs, precision):
    prim = _hot_gas(shape, 43)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 5)
    _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 5, precision, chunk=4, rounding=capi.ROUNDING_FAST)
    assert_parity(cons, ref, dts, ref_dts, precision, f"{shape} {bcs}")
    # the heat term itself, on the first layer of each lower conducting
    # face: the kernel's energy change against plain walls is the oracle's
    # (the term is ~1e-3 of the layer's energy over these steps, far above
    # either precision's error)
    plain = tuple(W if b == C else b for b in bcs)
    _, _, ref_plain = oracle_run(shape, 0.05, plain, prim, 5)
    for ax in range(3):
        if bcs[2 * ax] != C:
            continue
        layer = tuple(slice(2, 3) if a == ax else slice(2, -2) for a in range(3))
        d_ref = ref[4][layer] - ref_plain[4][layer]
        d_gpu = cons[4][layer] - ref_plain[4][layer]
        assert np.abs(d_ref).sum() > 1e-4 * np.abs(ref[4][layer]).sum()
        assert np.abs(d_gpu - d_ref).sum() <= 1e-2 * np.abs(d_ref).sum(), f"axis {ax}"


# ---------------------------------------------------------------------------
# Seeded random configurations: shapes from 2 to 90 cells per axis (ragged
# tiles in y and z, odd and even widths, several x chunks), every boundary
# combination the reference allows (periodic faces in pairs, conducting
# walls included), both limiters, gravity on or off; the FP64 sweep build at
# 1e-12 and the FP32 build at 1e-5 against the FP64 oracle
# ---------------------------------------------------------------------------
def _random_config(rng):
    shape = tuple(int(v) for v in rng.integers(2, 91, 3))
    bcs = []
    for _ in range(3):
        if rng.random() < 0.3:
            bcs += [P, P]
        else:
            bcs += [int(rng.choice([O, W, C])), int(rng.choice([O, W, C]))]
    return shape, tuple(bcs), int(rng.integers(0, 2)), bool(rng.random() < 0.3), int(rng.integers(1, 6))


@pytest.mark.parametrize("bcs,lim,grav", [((P,) * 6, 1, False), ((W, O, P, P, O, W), 0, True),
                                          ((O, W, W, O, W, O), 1, True), ((P, P, O, W, P, P), 1, False)])
def test_sweep_interior_tiles(bcs, lim, grav):
    """Grids wide enough to hold interior tiles (full tiles two cells clear
    of every y and z face, three or more tiles per axis) beside boundary and
    ragged tiles, as the random configurations (at most 90 cells per axis)
    do not: the FP64 build (4-row tiles) within 1e-12 and FP32 (14-row
    tiles) within 1e-5 of the oracle."""
    shape = (11, 47, 198)
    prim = random_primitives(shape, 777 + lim + 2 * grav)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 4, limiter=lim, gravity=grav)
    for precision in (capi.F64, capi.F32):
        _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 4, precision, limiter=lim, gravity=grav, chunk=5,
                               rounding=capi.ROUNDING_FAST)
        assert_parity(cons, ref, dts, ref_dts, precision, f"{bcs} lim {lim} grav {grav}")


@pytest.mark.parametrize("case", range(12))
def test_sweep_random_configurations(case):
    rng = np.random.default_rng(9000 + case)
    shape, bcs, lim, grav, chunk = _random_config(rng)
    prim = random_primitives(shape, 9100 + case)
    if C in bcs:
        prim = _hot_gas(shape, 9100 + case)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 4, limiter=lim, gravity=grav)
    for precision in (capi.F64, capi.F32):
        _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 4, precision, limiter=lim, gravity=grav, chunk=chunk,
                               rounding=capi.ROUNDING_FAST)
        assert_parity(cons, ref, dts, ref_dts, precision, f"{shape} {bcs} lim {lim} grav {grav} chunk {chunk}")


@pytest.mark.parametrize("case", range(12))
def test_reference_rounding_random_configurations(case):
    """The same configurations on the reference-rounding kernel: bit for bit
    against the FP64 oracle."""
    rng = np.random.default_rng(9000 + case)
    shape, bcs, lim, grav, chunk = _random_config(rng)
    prim = _hot_gas(shape, 9100 + case) if C in bcs else random_primitives(shape, 9100 + case)
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 4, limiter=lim, gravity=grav)
    _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 4, capi.F64, limiter=lim, gravity=grav, chunk=chunk,
                           rounding=capi.ROUNDING_REFERENCE)
    np.testing.assert_array_equal(dts, ref_dts)
    for f in range(5):
        np.testing.assert_array_equal(cons[f][INTERIOR], ref[f][INTERIOR], err_msg=f"field {f}")


def test_gravity_with_periodic_z():
    """Gravity on a periodic z axis: the reference copies the flux of the top
    face (nz-3) into the first cell's lower face, gravity term included."""
    shape = (9, 10, 6)
    prim = random_primitives(shape, 77)
    bcs = (P,) * 6
    _, ref_dts, ref = oracle_run(shape, 0.05, bcs, prim, 5, gravity=True)
    for precision, rounding in ((capi.F64, capi.ROUNDING_REFERENCE), (capi.F64, capi.ROUNDING_FAST),
                                (capi.F32, capi.ROUNDING_DEFAULT)):
        _, dts, cons = gpu_run(shape, 0.05, bcs, prim, 5, precision, gravity=True, rounding=rounding)
        if rounding == capi.ROUNDING_REFERENCE:
            for f in range(5):
                np.testing.assert_array_equal(cons[f][INTERIOR], ref[f][INTERIOR])
        else:
            assert_parity(cons, ref, dts, ref_dts, precision, f"rounding {rounding}")

