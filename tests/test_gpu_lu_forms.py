"""The solve kernels' LU factorisation and solves against the reference's
LUDecompose / LUBacksubstitute (gpuOde/ludecompose.H:9-130).

tests/golden/lu_forms.npz holds the reference's factors, pivots and solutions
(tests/golden/make_golden.py) at m = 11, 12, 33, 54, 55, 64, 65 and 101, on
uniform, small-integer (exact ties of the pivot criterion, "last max wins"),
zero-column (the gpuSmall pivot) and Rosenbrock (I / (gamma dx) - J of the
10-, 53- and 100-species mechanisms) matrices.

gf_lu_factor_solve runs lu_factor / lu_solve_any, the code of the solve
kernels, with 1 to 256 threads per matrix: the register-panel factorisation
(32 or more threads, m <= 64) and the blocked one (otherwise).

* exact rounding (each update a - l u rounded twice, as the reference's CPU
  build computes it): factors and pivots bit for bit equal to the reference
  in every form;
* the production rounding (FMA): every form gives the same factors bit for
  bit; pivots equal to the reference's and factors within 1e-12 of the
  largest entry of their row wherever the reference has no exact tie (an FMA
  rounds a tie differently);
* solutions within 1e-9 of max |x| (reciprocal pivots and a descending
  backward sum are ulp-level reorderings), except behind a gpuSmall pivot
  (x ~ 1e16, no digits to compare).
"""
import os

import numpy as np
import pytest

from gpufoam_b200 import evaluator as E

pytestmark = pytest.mark.gpu

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "lu_forms.npz")
FORMS = [1, 4, 8, 16, 32, 64, 96, 128, 256]


@pytest.fixture(scope="module")
def golden():
    import torch
    from gpufoam_b200 import build
    build.build()
    assert torch.cuda.is_available()
    return np.load(GOLDEN)


def cases(g):
    return [str(c) for c in g["cases"]]


def run(g, case, G, exact):
    LU, piv, x = E.lu_factor_solve(g[f"A_{case}"], g[f"b_{case}"], G, exact)
    return LU.cpu().numpy(), piv.cpu().numpy(), x.cpu().numpy()


def check_solution(g, case, x):
    if case.startswith("zerocol"):
        return
    xr = g[f"x_{case}"]
    scale = np.abs(xr).max(axis=2, keepdims=True)
    assert (np.abs(x - xr) <= 1e-9 * scale).all(), f"{case}: worst {np.max(np.abs(x - xr) / scale):.3g}"


@pytest.mark.parametrize("G", FORMS)
def test_exact_rounding_bit_for_bit(golden, G):
    for case in cases(golden):
        LU, piv, x = run(golden, case, G, exact=True)
        assert np.array_equal(piv, golden[f"piv_{case}"]), f"{case} G={G}: pivots"
        assert np.array_equal(LU, golden[f"LU_{case}"]), (
            f"{case} G={G}: {np.sum(LU != golden[f'LU_{case}'])} factor entries differ")
        check_solution(golden, case, x)


def test_production_rounding(golden):
    for case in cases(golden):
        first = None
        for G in FORMS:
            LU, piv, x = run(golden, case, G, exact=False)
            if first is None:
                first = (LU, piv)
            else:
                assert np.array_equal(piv, first[1]) and np.array_equal(LU, first[0]), (
                    f"{case}: G={G} differs from G={FORMS[0]}")
            if case.startswith("ties"):
                continue
            assert np.array_equal(piv, golden[f"piv_{case}"]), f"{case} G={G}: pivots"
            LUr = golden[f"LU_{case}"]
            row = np.abs(LUr).max(axis=2, keepdims=True)
            assert (np.abs(LU - LUr) <= 1e-12 * row).all(), f"{case} G={G}"
            check_solution(golden, case, x)
