"""Discrete adjoint (gf_solve_record / gf_adjoint) against the oracle.

The oracle (oracle/gf_oracle.c, pinned to the reference) replays the recorded
accepted steps with the step sequence frozen: y_{k+1} = Rosenbrock attempt(y_k,
f(y_k), h_k), then the final max(0, Y) clip of singleCellSolver (orc_replay).
Checks:

* initial state: central differences with a relative step of 1e-6 of that map
  along a random direction (all species, T, every cell), to 1e-5 relative;
* per-reaction (ln|A|, beta, Ta) on random parameters: central differences with
  relative steps 1e-4 and 2e-4, Richardson-extrapolated (a 1e-6 step is below
  the loss's rounding noise for the small parameter gradients), to 1e-5
  relative, or 1e-5 of the largest parameter gradient for the tiny ones;
* a tangent-linear reference on the CPU (oracle/complex_step.py): the frozen
  map restated in complex arithmetic, whose imaginary part at x + i eps d
  carries the derivative of every operation along d (the complex-step method,
  exact to rounding), along a random direction of all initial states and a
  random direction of all rate parameters, against the adjoint's gradient
  along the same directions, to 1e-5 relative.
"""
import concurrent.futures

import numpy as np
import pytest

from gpufoam_b200 import adjoint as AD
from gpufoam_b200 import evaluator as E
from gpufoam_b200 import mechanism as M
from oracle.complex_step import ComplexStepMap
from oracle.oracle import Oracle, ode_inputs


def test_parameters_roundtrip():
    raw = M.h2_size(0)
    th = AD.parameters_of(raw)
    raw2 = AD.with_parameters(raw, th + 0.0)
    for a, b in zip(raw.reactions, raw2.reactions):
        assert a.A == pytest.approx(b.A, rel=1e-14) and a.beta == b.beta and a.Ta == b.Ta


class Case:
    """One recorded integration on the GPU, its adjoint, and the oracle's
    frozen-step replay."""

    def __init__(self, raw, n_cells, deltaT, solver, seed, T_range=(1000.0, 2500.0)):
        import torch
        self.raw, self.nS, self.n = raw, raw.n_species, n_cells
        self.cells = M.make_cells(raw, n_cells, seed=seed, T_range=T_range)
        sol = AD.AdjointSolver(raw, E.OdeInputs(f"Rosenbrock{solver}", absTol=1e-8, relTol=1e-4), traj_cap=2048)
        Y0 = torch.as_tensor(self.cells, device="cuda")
        dtc = torch.full((n_cells,), 1e-7, dtype=torch.float64, device="cuda")
        Y1, status, counters = sol.forward(Y0, deltaT, dtc)
        torch.cuda.synchronize()
        assert (status.cpu().numpy() == 0).all()
        rng = np.random.default_rng(seed + 1)
        self.rng = rng
        self.w = rng.standard_normal((n_cells, self.nS + 2))
        self.w[:, self.nS] *= 1e-3  # T in K against mass fractions
        self.w[:, self.nS + 1] = 0.0
        Y0bar, thb, st = sol.backward(torch.as_tensor(self.w, device="cuda"))
        torch.cuda.synchronize()
        assert (st.cpu().numpy() == 0).all()
        self.Y0bar, self.thb = Y0bar.cpu().numpy(), thb.cpu().numpy()
        traj = sol._rec["traj"].cpu().numpy()
        cnt = counters.cpu().numpy()
        self.steps = [traj[c, :cnt[c, 0], self.nS + 1] for c in range(n_cells)]
        self.Y1 = Y1.cpu().numpy()
        self.solver = solver
        self.inp = ode_inputs(solver)
        self.orc = Oracle(raw, "port")

    def loss(self, orc, cells):
        return sum(float(np.dot(self.w[c], orc.replay(self.inp, cells[c], self.steps[c]))) for c in range(self.n))

    def theta_loss(self, theta):
        return self.loss(Oracle(AD.with_parameters(self.raw, theta), "port"), self.cells)


def check_case(case, n_params, replay_rtol=1e-10):
    nS, cells = case.nS, case.cells
    # the replay reproduces the GPU integration
    for c in range(case.n):
        yf = case.orc.replay(case.inp, cells[c], case.steps[c])
        np.testing.assert_allclose(yf, case.Y1[c], rtol=replay_rtol, atol=1e-14)
    # initial state, random direction, central FD (relative step 1e-6)
    d = case.rng.standard_normal(cells.shape)
    d[:, nS + 1] = 0.0
    scale = np.abs(cells) + 1e-6
    eps = 1e-6
    fd = (case.loss(case.orc, cells + eps * scale * d) - case.loss(case.orc, cells - eps * scale * d)) / (2 * eps)
    ad = float(np.sum(case.Y0bar * scale * d))
    assert abs(ad - fd) <= 1e-5 * abs(fd), ("initial state", ad, fd)
    # tangent-linear (complex step) along the same direction, and along a
    # random direction of all rate parameters
    cs = ComplexStepMap(case.raw, case.solver)
    th0 = AD.parameters_of(case.raw)
    tl = sum(float(np.dot(case.w[c], cs.directional(cells[c], case.steps[c], th0, dy=scale[c] * d[c])))
             for c in range(case.n))
    assert abs(ad - tl) <= 1e-5 * abs(tl), ("tangent-linear, initial state", ad, tl)
    dth = case.rng.standard_normal(th0.shape) * np.maximum(np.abs(th0), 1.0)
    tl = sum(float(np.dot(case.w[c], cs.directional(cells[c], case.steps[c], th0, dtheta=dth)))
             for c in range(case.n))
    ad = float(np.sum(case.thb * dth))
    assert abs(ad - tl) <= 1e-5 * abs(tl), ("tangent-linear, parameters", ad, tl)
    # parameters: Richardson-extrapolated central differences (the losses in parallel)
    picks = sorted({(int(case.rng.integers(case.raw.n_reactions)), int(case.rng.integers(3)))
                    for _ in range(n_params)})
    gmax = np.abs(case.thb).max()

    def fd_param(rk):
        r, k = rk

        def fd_at(hr):
            step = hr * max(abs(th0[r, k]), 1.0)
            tp, tm = th0.copy(), th0.copy()
            tp[r, k] += step
            tm[r, k] -= step
            return (case.theta_loss(tp) - case.theta_loss(tm)) / (2 * step)
        return (4.0 * fd_at(1e-4) - fd_at(2e-4)) / 3.0

    with concurrent.futures.ThreadPoolExecutor() as ex:
        fds = list(ex.map(fd_param, picks))
    for (r, k), fd in zip(picks, fds):
        ad = float(case.thb[r, k])
        assert abs(ad - fd) <= 1e-5 * max(abs(fd), gmax), (r, k, ad, fd, gmax)


@pytest.mark.gpu
@pytest.mark.parametrize("solver", [34, 23, 12])
def test_adjoint_h2size(solver):
    check_case(Case(M.h2_size(0), 3, 1e-5, solver, seed=11 + solver), n_params=64)


@pytest.mark.gpu
def test_adjoint_coverage_mechanism():
    """Every rate type (Arrhenius, third body, Lindemann and Troe fall-off),
    irreversible reactions and non-integer exponents."""
    check_case(Case(M.coverage(0), 3, 1e-5, 34, seed=7), n_params=64)


@pytest.mark.gpu
def test_adjoint_grisize():
    check_case(Case(M.gri_size(0), 2, 1e-6, 34, seed=12), n_params=24)


@pytest.mark.gpu
def test_adjoint_differentiation_workload():
    """The differentiation workload's configuration: the GRI-size mechanism,
    T ~ U[1100, 1600] K, deltaT = 1e-4 s (through ignition, ~170 accepted
    steps per cell), Rosenbrock34; 4 cells, 64 random parameters."""
    case = Case(M.gri_size(0), 4, 1e-4, 34, seed=4096, T_range=(1100.0, 1600.0))
    assert min(len(s) for s in case.steps) >= 50
    check_case(case, n_params=64, replay_rtol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("name, deltaT", [("foam_h2", 1e-5), ("foam_gri", 1e-6)])
def test_adjoint_real_mechanism(name, deltaT):
    """The reference's real H2 and GRI-Mech 3.0 test mechanisms (read from their
    OpenFOAM dictionaries, stored in the golden fixtures)."""
    from tests.test_oracle import fixture_mech, load
    check_case(Case(fixture_mech(load(name)), 2, deltaT, 34, seed=21), n_params=24)


@pytest.mark.gpu
def test_autograd_function():
    """ChemistryStep through torch.autograd: loss.backward() fills Y0.grad and
    theta.grad with the adjoint's gradients."""
    import torch
    raw = M.h2_size(0)
    sol = AD.AdjointSolver(raw, E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4), traj_cap=1024)
    cells = M.make_cells(raw, 4, seed=3)
    Y0 = torch.tensor(cells, device="cuda", requires_grad=True)
    theta = torch.tensor(sol.parameters(), requires_grad=True)
    wts = torch.as_tensor(np.random.default_rng(2).standard_normal(cells.shape), device="cuda")
    Y1 = AD.ChemistryStep.apply(Y0, theta, sol, 1e-5, 1e-7)
    (wts * Y1).sum().backward()
    assert Y0.grad is not None and theta.grad is not None
    assert torch.isfinite(Y0.grad).all() and torch.isfinite(theta.grad).all()
    # the same numbers as the solver's own backward
    Yb, thb, st = sol.backward(wts)
    assert torch.equal(Y0.grad, Yb) and np.array_equal(theta.grad.numpy(), thb.cpu().numpy())
    # a perturbed theta changes the forward (the parameters are live inputs)
    th2 = theta.detach().clone()
    th2[0, 0] += 0.5
    Y2 = AD.ChemistryStep.apply(Y0.detach(), th2, sol, 1e-5, 1e-7)
    assert not torch.equal(Y1.detach(), Y2)
