"""Generate the golden fixtures of tests/golden/ from the gpuFoam reference.

Run where the reference tree exists (GPUFOAM_REFERENCE, else a directory
named reference beside this repository; its FP64 headers are compiled in
place by oracle/Makefile into oracle/_ref/libgf_ref.so):

    python tests/golden/make_golden.py

Every expected value in the .npz files below comes from the reference's own
code (gpuThermo, gpuReaction, gpuODESystem, LUDecompose/LUBacksubstitute,
gpuRosenbrock12/23/34, odeSolve, singleCellSolver), evaluated on seeded
synthetic mechanisms and cell states, and on the three real mechanisms of the
reference's unit tests (foam_*.npz, read from their OpenFOAM dictionaries by
gpufoam_b200.foam_dict). The raw mechanism is stored with the results so that
the fixtures do not depend on the generator or the reference tree.

    python tests/golden/make_golden.py [case ...]   # default: all cases
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gpufoam_b200 import mechanism as M  # noqa: E402
from oracle.oracle import REFERENCE_ROOT, Oracle, flatten, lu, ode_inputs  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))

CASES = [
    # name, mechanism factory, n states, n cells per solver, deltaT
    ("h2size", M.h2_size, 8, 32, 1e-5),
    ("coverage", M.coverage, 8, 32, 1e-5),
    ("grisize", M.gri_size, 6, 12, 1e-6),
]

# The real mechanisms of the reference's unit tests (OpenFOAM dictionaries
# embedded as C++ raw strings in gpu_chemistry/unittest/testHelpers/), read by
# gpufoam_b200.foam_dict, with the reference's own test condition
# (testHelpers/mechanisms.H:36-107: T = 1000 K, the mechanism's p and three
# non-zero mass fractions) as state 0.
HELPERS = os.path.join(REFERENCE_ROOT, "gpu_chemistry", "unittest", "testHelpers")
FOAM = [
    # name, file stem, (species index, Y) of the test condition, p, n states, n cells, deltaT
    ("foam_h2", "h2", [(0, 0.2), (2, 0.2), (9, 0.6)], 202650.0, 8, 32, 1e-5),
    ("foam_gri", "gri", [(0, 0.2), (4, 0.5), (47, 0.3)], 1.36789e6, 6, 12, 1e-6),
    ("foam_yao", "yao", [(44, 0.2), (8, 0.2), (53, 0.6)], 1.36789e6, 6, 12, 1e-6),
]


def foam_factory(stem):
    from gpufoam_b200 import foam_dict

    def make(_seed):
        return foam_dict.read_mechanism_files(os.path.join(HELPERS, f"{stem}_thermos.h"),
                                              os.path.join(HELPERS, f"{stem}_reactions.h"), stem)
    return make


def test_condition(mech, fractions, p):
    y = np.zeros(mech.n_eqns)
    for i, v in fractions:
        y[i] = v
    y[-2], y[-1] = 1000.0, p
    return y


def make_case(name, factory, n_states, n_cells, deltaT, first_state=None):
    mech = factory(0)
    ref = Oracle(mech, "reference")
    fl = flatten(mech)
    out = {f"mech_{k}": np.asarray(v) for k, v in fl.items()}
    sp, rx, ie = ref.tables()
    out.update(species_tables=sp, reaction_tables=rx, int_exponents=ie, constants=ref.constants())
    out["thermo_700"] = ref.thermo_eval(101325.0, 700.0)
    out["thermo_1500"] = ref.thermo_eval(101325.0, 1500.0)
    states = M.make_cells(mech, n_states, seed=11)
    if first_state is not None:
        states = np.vstack([first_state[None, :], states[1:]])
    out["states"] = states
    out["reaction_eval"] = np.stack([ref.reaction_eval(s) for s in states[:2]])
    out["dydx"] = ref.derivatives(states)
    dfdx, J = ref.jacobian(states)
    out["dfdx"], out["J"] = dfdx, J
    rng = np.random.default_rng(5)
    dxs = 10.0 ** rng.uniform(-10, -7, size=n_states)
    out["attempt_dx"] = dxs
    for s in (12, 23, 34):
        y, err = ref.attempt(ode_inputs(s), states, out["dydx"], dxs)
        out[f"attempt{s}_y"], out[f"attempt{s}_err"] = y, err
    cells = M.make_cells(mech, n_cells, seed=12)
    if first_state is not None:
        cells = np.vstack([first_state[None, :], cells[1:]])
    out["cells"] = cells
    out["deltaT"] = np.array(deltaT)
    out["deltaTChem0"] = np.array(1e-7)
    for s in (12, 23, 34):
        Y, dtc, counts, _ = ref.cells(ode_inputs(s), cells, deltaT, 1e-7)
        out[f"cells{s}_Y"], out[f"cells{s}_dtc"], out[f"cells{s}_counts"] = Y, dtc, counts
    # the Treact gate: half of the cells below the threshold
    Treact = float(np.median(cells[:, -2]))
    Y, dtc, counts, _ = ref.cells(ode_inputs(34), cells, deltaT, 1e-7, Treact=Treact)
    out["treact"] = np.array(Treact)
    out["cells34_treact_Y"], out["cells34_treact_dtc"] = Y, dtc
    # host computeRR arithmetic on the R34 result
    rho = np.linspace(0.2, 1.3, n_cells)
    RR, dtc_new, mn = ref.compute_rr_host(deltaT, 5e-8, rho, cells, out["cells34_Y"], out["cells34_dtc"])
    out.update(rr_rho=rho, rr_RR=RR, rr_dtc=dtc_new, rr_min=np.array(mn), rr_dtcmax=np.array(5e-8))
    np.savez_compressed(os.path.join(OUT, f"{name}.npz"), **out)
    print(name, "written", {k: v.shape for k, v in out.items() if hasattr(v, "shape") and v.size > 50})


def make_lu():
    rng = np.random.default_rng(3)
    out = {}
    out["sizes"] = np.array([3, 4, 5, 7, 10, 12, 16, 24, 33, 49, 54])
    for m in out["sizes"]:
        A = rng.uniform(size=(1, m, m))
        b = np.ones((1, m))
        LU, piv, x = lu("reference", A, b)
        out[f"A{m}"], out[f"LU{m}"], out[f"piv{m}"], out[f"x{m}"] = A, LU, piv, x
    np.savez_compressed(os.path.join(OUT, "lu.npz"), **out)
    print("lu written")


def make_lu_forms():
    """LUDecompose + LUBacksubstitute of the reference at the sizes the solve
    kernels' forms switch at (m <= 64 register panel, larger blocked; the
    10-, 53- and 100-species mechanisms give m = 11, 54, 101), on four kinds of
    matrices: uniform entries, small integers (exact ties of vv |a|, the "last
    max wins" rule, and zero pivots), a zero column (the gpuSmall pivot), and
    the Rosenbrock matrices I / (gamma dx) - J of real Jacobians."""
    rng = np.random.default_rng(17)
    out = {"sizes": np.array([11, 12, 33, 54, 55, 64, 65, 101])}
    jac = {}
    for factory in (M.h2_size, M.gri_size, M.large):
        mech = factory(0)
        states = M.make_cells(mech, 2, seed=23)
        _, J = Oracle(mech, "reference").jacobian(states)
        m = mech.n_species + 1
        jac[m] = J[:, :m, :m]
    kinds = []
    for m in out["sizes"]:
        mats = {"uniform": rng.uniform(size=(1, m, m)),
                "ties": rng.integers(-3, 4, size=(1, m, m)).astype(np.float64)}
        z = rng.uniform(-1.0, 1.0, size=(1, m, m))
        z[:, :, m // 3] = 0.0
        mats["zerocol"] = z
        if m in jac:
            dx = np.array([1e-9, 1e-6])
            mats["rosenbrock"] = -jac[m] + np.eye(m)[None] / (0.5 * dx[:, None, None])
        for kind, A in mats.items():
            b = np.stack([np.ones((A.shape[0], m)), rng.standard_normal((A.shape[0], m))], axis=1)
            xs = []
            for r in range(2):
                LU, piv, x = lu("reference", A, b[:, r])
                xs.append(x)
            key = f"{kind}_{m}"
            kinds.append(key)
            out[f"A_{key}"], out[f"b_{key}"] = A, b
            out[f"LU_{key}"], out[f"piv_{key}"], out[f"x_{key}"] = LU, piv, np.stack(xs, axis=1)
    out["cases"] = np.array(kinds)
    np.savez_compressed(os.path.join(OUT, "lu_forms.npz"), **out)
    print("lu_forms written", len(kinds), "cases")


if __name__ == "__main__":
    only = sys.argv[1:]
    if not only or "lu" in only:
        make_lu()
    if not only or "lu_forms" in only:
        make_lu_forms()
    for case in CASES:
        if not only or case[0] in only:
            make_case(*case)
    for name, stem, fractions, p, n_states, n_cells, deltaT in FOAM:
        if only and name not in only:
            continue
        factory = foam_factory(stem)
        make_case(name, factory, n_states, n_cells, deltaT, first_state=test_condition(factory(0), fractions, p))
