"""Pin the CPU oracle (oracle/gf_oracle.c) to the gpuFoam reference.

Two independent pins:
* the golden fixtures of tests/golden/, produced by the reference's own code
  (tests/golden/make_golden.py), and
* the reference compiled in place (oracle/_ref/libgf_ref.so), run live on
  further seeded inputs when that library is present.

The restatement follows the reference's operation order and both are built
with -ffp-contract=off against the same libm, so the comparisons are bit for
bit (NaN == NaN).
"""
import os

import numpy as np
import pytest

from gpufoam_b200 import mechanism as M
from oracle.oracle import REF_LIB, Oracle, lu, ode_inputs

GOLDEN = os.path.join(os.path.dirname(__file__), "golden")
CASES = ["h2size", "coverage", "grisize", "foam_h2", "foam_gri", "foam_yao"]


def load(name):
    return dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))


class _Raw:
    """RawMechanism stand-in rebuilt from the flat arrays stored in a fixture."""

    def __init__(self, g):
        from gpufoam_b200.mechanism import RawMechanism, RawReaction
        nS = int(g["mech_nS"])
        nR = int(g["mech_nR"])
        rxs = []
        for r in range(nR):
            ri, rd = g["mech_rint"][r], g["mech_rdbl"][r]
            nl, nr = int(ri[2]), int(ri[3])
            rxs.append(RawReaction(
                int(ri[0]), bool(ri[1]),
                [(int(ri[4 + i]), float(rd[i]), float(rd[10 + i])) for i in range(nl)],
                [(int(ri[14 + i]), float(rd[20 + i]), float(rd[30 + i])) for i in range(nr)],
                *[float(x) for x in rd[40:46]], troe=tuple(float(x) for x in rd[46:50]),
                efficiencies=(g["mech_eff"][r].copy() if ri[0] != 0 else None)))
        self.mech = RawMechanism("fixture", [f"S{i}" for i in range(nS)], g["mech_W"], g["mech_Tlow"],
                                 g["mech_Thigh"], g["mech_Tcommon"], g["mech_high"], g["mech_low"], rxs,
                                 float(g["mech_rxnTlow"]), float(g["mech_rxnThigh"]))


def fixture_mech(g):
    return _Raw(g).mech


def eq(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


@pytest.mark.parametrize("name", CASES)
def test_tables_and_pointwise_vs_golden(name):
    g = load(name)
    o = Oracle(fixture_mech(g), "port")
    sp, rx, ie = o.tables()
    assert eq(sp, g["species_tables"])
    assert eq(rx, g["reaction_tables"])
    assert eq(ie, g["int_exponents"])
    assert eq(o.constants(), g["constants"])
    assert eq(o.thermo_eval(101325.0, 700.0), g["thermo_700"])
    assert eq(o.thermo_eval(101325.0, 1500.0), g["thermo_1500"])
    for k in range(2):
        assert eq(o.reaction_eval(g["states"][k]), g["reaction_eval"][k])
    assert eq(o.derivatives(g["states"]), g["dydx"])
    dfdx, J = o.jacobian(g["states"])
    assert eq(dfdx, g["dfdx"])
    assert eq(J, g["J"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("solver", [12, 23, 34])
def test_attempt_vs_golden(name, solver):
    g = load(name)
    o = Oracle(fixture_mech(g), "port")
    y, err = o.attempt(ode_inputs(solver), g["states"], g["dydx"], g["attempt_dx"])
    assert eq(y, g[f"attempt{solver}_y"])
    assert eq(err, g[f"attempt{solver}_err"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("solver", [12, 23, 34])
def test_cells_vs_golden(name, solver):
    g = load(name)
    o = Oracle(fixture_mech(g), "port")
    Y, dtc, counts, status = o.cells(ode_inputs(solver), g["cells"], float(g["deltaT"]), float(g["deltaTChem0"]))
    assert eq(Y, g[f"cells{solver}_Y"])
    assert eq(dtc, g[f"cells{solver}_dtc"])
    assert eq(counts, g[f"cells{solver}_counts"])
    assert (status == 0).all()


@pytest.mark.parametrize("name", CASES)
def test_treact_gate_and_compute_rr_vs_golden(name):
    g = load(name)
    o = Oracle(fixture_mech(g), "port")
    Y, dtc, counts, status = o.cells(ode_inputs(34), g["cells"], float(g["deltaT"]), float(g["deltaTChem0"]),
                                     Treact=float(g["treact"]))
    assert eq(Y, g["cells34_treact_Y"])
    assert eq(dtc, g["cells34_treact_dtc"])
    skipped = g["cells"][:, -2] <= float(g["treact"])
    assert (status[skipped] == 4).all() and (counts[skipped] == 0).all()
    RR, dtc_new, mn = o.compute_rr_host(float(g["deltaT"]), float(g["rr_dtcmax"]), g["rr_rho"], g["cells"],
                                        g["cells34_Y"], g["cells34_dtc"])
    assert eq(RR, g["rr_RR"])
    assert eq(dtc_new, g["rr_dtc"])
    assert mn == float(g["rr_min"])


def test_lu_vs_golden():
    g = load("lu")
    for m in g["sizes"]:
        LU, piv, x = lu("port", g[f"A{m}"], np.ones((1, m)))
        assert eq(LU, g[f"LU{m}"]) and eq(piv, g[f"piv{m}"]) and eq(x, g[f"x{m}"])


needs_ref = pytest.mark.skipif(not os.path.exists(REF_LIB), reason="reference oracle not built")


@needs_ref
@pytest.mark.parametrize("factory,seed", [(M.h2_size, 3), (M.coverage, 4), (M.gri_size, 5), (M.large, 1)])
def test_port_vs_reference_live(factory, seed):
    mech = factory(seed)
    a, b = Oracle(mech, "port"), Oracle(mech, "reference")
    for x, y in zip(a.tables(), b.tables()):
        assert eq(x, y)
    states = M.make_cells(mech, 6, seed=seed + 100, T_range=(600.0, 2600.0))
    assert eq(a.derivatives(states), b.derivatives(states))
    for x, y in zip(a.jacobian(states), b.jacobian(states)):
        assert eq(x, y)
    dydx = a.derivatives(states)
    for s in (12, 23, 34):
        for x, y in zip(a.attempt(ode_inputs(s), states, dydx, 3e-9), b.attempt(ode_inputs(s), states, dydx, 3e-9)):
            assert eq(x, y)
    if mech.n_species <= 60:
        cells = M.make_cells(mech, 8, seed=seed + 200)
        dT = 1e-6
        ra = a.cells(ode_inputs(34), cells, dT, 1e-7)
        rb = b.cells(ode_inputs(34), cells, dT, 1e-7)
        for x, y in zip(ra[:3], rb[:3]):
            assert eq(x, y)


@needs_ref
@pytest.mark.parametrize("name", CASES)
def test_side_paths_port_vs_reference(name):
    """calculate / tc / reactionRR / specieReactionRR / Qdot (gpuChemistryModel.C:145-450):
    the C restatement against the reference's own reaction objects, bit for bit,
    including a state with all concentrations zero (tc = vGreat)."""
    g = load(name)
    mech = fixture_mech(g)
    a, b = Oracle(mech, "port"), Oracle(mech, "reference")
    y = np.vstack([g["states"], M.make_cells(mech, 4, seed=7, T_range=(250.0, 3500.0))])
    rho = np.linspace(0.05, 3.0, y.shape[0])
    rho[-1] = 0.0
    RRa, tca = a.cell_fields(rho, y)
    RRb, tcb = b.cell_fields(rho, y)
    assert eq(RRa, RRb) and eq(tca, tcb)
    assert tca[-1] == np.finfo(np.float64).max / 10
    assert eq(a.qdot(RRa), b.qdot(RRb))
    for r in range(0, mech.n_reactions, max(1, mech.n_reactions // 17)):
        for x, z in zip(a.reaction_fields(r, rho, y), b.reaction_fields(r, rho, y)):
            assert eq(x, z)


@needs_ref
@pytest.mark.parametrize("name", ["foam_h2", "foam_gri", "foam_yao"])
def test_reference_test_configuration(name):
    """The reference's own unit-test configuration: its real mechanisms at its test
    condition (testHelpers/mechanisms.H:36-107, state 0 of the fixtures) with its
    ODE inputs (absTol 1e-12, relTol 1e-1, create_gpu_inputs.C:59-71), every
    Rosenbrock solver, over 1e-7 and 1e-5 s: the restatement equals the
    reference bit for bit, step counts included."""
    g = load(name)
    mech = fixture_mech(g)
    a, b = Oracle(mech, "port"), Oracle(mech, "reference")
    cells = np.vstack([g["states"][:1], g["cells"][1:3]])
    for s in (12, 23, 34):
        inp = ode_inputs(s, absTol=1e-12, relTol=1e-1)
        for dT in (1e-7, 1e-5):
            ra = a.cells(inp, cells, dT, 1e-7)
            rb = b.cells(inp, cells, dT, 1e-7)
            for x, y in zip(ra[:3], rb[:3]):
                assert eq(x, y)


@needs_ref
def test_reference_counted_wrapper_matches_reference_functor():
    """The counting wrapper used for step counts gives the same states as the
    reference's own singleCellSolver functor."""
    mech = M.h2_size(7)
    b = Oracle(mech, "reference")
    cells = M.make_cells(mech, 16, seed=9)
    Y1, d1, _, _ = b.cells(ode_inputs(23), cells, 1e-5, 1e-7, Treact=1500.0)
    Y2, d2 = b.cells_uncounted(ode_inputs(23), cells, 1e-5, 1e-7, Treact=1500.0)
    assert eq(Y1, Y2) and eq(d1, d2)


def test_max_steps_and_nonfinite_status():
    """Failure reporting of the oracle: maxSteps exhausted leaves deltaTChem at
    its input (odeSolve returns without writing dxTry, gpuODESolverBase.H:80-111)
    and flags MAX_STEPS; a NaN mass fraction is integrated (the mixture clips it
    with fmax) and flagged NONFINITE; a NaN temperature fails the T > Treact
    gate of singleCellSolver.H:31 and is skipped, as in the reference."""
    mech = M.h2_size(0)
    o = Oracle(mech, "port")
    cells = M.make_cells(mech, 4, seed=1)
    Y, dtc, counts, status = o.cells(ode_inputs(34, maxSteps=2), cells, 1e-5, 1e-7)
    assert (status == 2).all() and (counts[:, 0] == 2).all() and (dtc == 1e-7).all()
    bad = cells.copy()
    bad[1, 0] = np.nan
    bad[2, -2] = np.nan
    Y, dtc, counts, status = o.cells(ode_inputs(34), bad, 1e-5, 1e-7)
    assert status[1] == 3 and status[2] == 4 and dtc[2] == 1e-5
    assert status[0] == 0 and status[3] == 0
