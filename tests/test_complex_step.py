"""The tangent-linear reference (oracle/complex_step.py) and the frozen-step
replay (orc_replay), pinned on the CPU before they check the GPU adjoint.

* The complex-step map's real part equals the oracle's Rosenbrock attempt
  (pinned bit for bit to the reference) to rounding, on the golden states of
  three mechanisms and all three solvers.
* Its derivatives (Im / eps) agree with central differences of the C oracle
  along random directions of the initial state and of the per-reaction
  (ln|A|, beta, Ta), on mechanisms with every rate type, irreversible reactions
  and non-integer exponents.
* orc_replay equals the same steps taken one by one through orc_attempt.
"""
import numpy as np
import pytest

from gpufoam_b200 import adjoint as AD
from gpufoam_b200 import mechanism as M
from oracle.complex_step import ComplexStepMap
from oracle.oracle import Oracle, ode_inputs
from tests.test_oracle import fixture_mech, load


def replay_by_attempts(orc, inp, y0, steps, nS):
    y = np.array(y0, dtype=np.float64)
    for h in steps:
        y = orc.attempt(inp, y[None], orc.derivatives(y[None]), h)[0][0]
    y[:nS] = np.maximum(y[:nS], 0.0)
    return y


@pytest.mark.parametrize("name", ["h2size", "coverage", "grisize"])
@pytest.mark.parametrize("solver", [12, 23, 34])
def test_real_part_is_the_oracle_attempt(name, solver):
    g = load(name)
    raw = fixture_mech(g)
    cs = ComplexStepMap(raw, solver)
    orc = Oracle(raw, "port")
    th = AD.parameters_of(raw)
    for y0, dx in zip(g["states"], g["attempt_dx"]):
        with np.errstate(all="ignore"):
            y = np.real(cs.step(y0.astype(complex), float(dx), th.astype(complex)))
        ref = orc.attempt(ode_inputs(solver), y0[None], orc.derivatives(y0[None]), dx)[0][0]
        assert (np.abs(y - ref) <= 1e-12 * (np.abs(ref) + np.abs(ref).max() * 1e-12)).all()


@pytest.mark.parametrize("factory", [M.h2_size, M.coverage])
def test_derivatives_match_central_differences(factory):
    raw = factory(0)
    nS = raw.n_species
    cs = ComplexStepMap(raw, 34)
    orc = Oracle(raw, "port")
    inp = ode_inputs(34)
    y0 = M.make_cells(raw, 1, seed=4)[0]
    steps = [1e-7, 3e-7, 1e-6]
    th = AD.parameters_of(raw)
    rng = np.random.default_rng(0)
    d = rng.standard_normal(y0.shape) * (np.abs(y0) + 1e-6)
    d[nS + 1] = 0.0
    tl = cs.directional(y0, steps, th, dy=d)
    eps = 1e-6
    fd = (orc.replay(inp, y0 + eps * d, steps) - orc.replay(inp, y0 - eps * d, steps)) / (2 * eps)
    assert np.max(np.abs(tl - fd)) <= 1e-7 * np.abs(fd).max()
    dth = rng.standard_normal(th.shape) * np.array([1.0, 0.1, 100.0])
    tl = cs.directional(y0, steps, th, dtheta=dth)
    h = 1e-5

    def at(t):
        return Oracle(AD.with_parameters(raw, t), "port").replay(inp, y0, steps)
    fd = (at(th + h * dth) - at(th - h * dth)) / (2 * h)
    assert np.max(np.abs(tl - fd)) <= 1e-7 * np.abs(fd).max()


def test_replay_equals_the_attempts():
    raw = M.gri_size(0)
    orc = Oracle(raw, "port")
    inp = ode_inputs(34)
    y0 = M.make_cells(raw, 1, seed=9)[0]
    steps = [1e-8, 5e-8, 2e-7, 7e-7]
    assert np.array_equal(orc.replay(inp, y0, steps), replay_by_attempts(orc, inp, y0, steps, raw.n_species))
