"""GPU parity of the CUDA path against the reference.

Every test calls the CUDA kernels through the C ABI (libgpufoam_b200.so) and
compares with (a) golden vectors generated by the reference's own code and
(b) the CPU oracle (oracle/gf_oracle.c, pinned bit for bit to the reference by
tests/test_oracle.py) on further seeded inputs.
"""
import os

import numpy as np
import pytest

from gpufoam_b200 import evaluator as E
from gpufoam_b200 import mechanism as M
from oracle.oracle import Oracle, ode_inputs
from tests.parity import (assert_jacobian_close, assert_rates_close, assert_states_close, jacobian_scale,
                          rate_scale, step_count_agreement)
from tests.test_oracle import fixture_mech, load

pytestmark = pytest.mark.gpu

CASES = ["h2size", "coverage", "grisize", "foam_h2", "foam_gri", "foam_yao"]
LAUNCHES = {
    "plain": dict(kind=0),
    "persist-g1-hbm": dict(kind=1, threads_per_cell=1, scratch_in_shared=0),
    "persist-g8-smem": dict(kind=1, threads_per_cell=8, scratch_in_shared=1),
    "persist-g32-smem": dict(kind=1, threads_per_cell=32, scratch_in_shared=1),
    "persist-g32-hbm": dict(kind=1, threads_per_cell=32, scratch_in_shared=0),
    "persist-g4-hbm": dict(kind=1, threads_per_cell=4, scratch_in_shared=0),
    "persist-g64-smem": dict(kind=1, threads_per_cell=64, scratch_in_shared=1),
    "persist-g96-smem-slim": dict(kind=1, threads_per_cell=96, scratch_in_shared=1, register_budget=1),
    "persist-g128-smem-slim": dict(kind=1, threads_per_cell=128, scratch_in_shared=1, register_budget=1),
    "persist-g256-smem": dict(kind=1, threads_per_cell=256, scratch_in_shared=1),
    "persist-g128-hbm": dict(kind=1, threads_per_cell=128, scratch_in_shared=0),
}


@pytest.fixture(scope="module")
def torch():
    import torch
    from gpufoam_b200 import build
    build.build()
    assert torch.cuda.is_available()
    return torch


_mechs = {}


def gpu_mech(name):
    if name not in _mechs:
        g = load(name)
        _mechs[name] = (g, fixture_mech(g), E.Mechanism(fixture_mech(g)))
    return _mechs[name]


@pytest.mark.parametrize("name", CASES)
def test_rates_vs_reference(torch, name):
    g, raw, mech = gpu_mech(name)
    got = E.rates(mech, g["states"]).cpu().numpy()
    assert_rates_close(got, g["dydx"], rate_scale(raw, g["states"]))
    assert (got[:, -1] == 0).all()


@pytest.mark.parametrize("name", CASES)
def test_jacobian_vs_reference(torch, name):
    g, raw, mech = gpu_mech(name)
    dfdx, J = E.jacobian(mech, g["states"])
    assert_rates_close(dfdx.cpu().numpy(), g["dfdx"], rate_scale(raw, g["states"]))
    assert_jacobian_close(J.cpu().numpy(), g["J"], jacobian_scale(raw, g["states"]))


def test_lu_vs_reference(torch):
    g = load("lu")
    for m in g["sizes"]:
        LU, piv = E.lu_decompose(g[f"A{m}"])
        assert np.array_equal(piv.cpu().numpy(), g[f"piv{m}"])
        np.testing.assert_allclose(LU.cpu().numpy(), g[f"LU{m}"], rtol=1e-12, atol=1e-14)
        x = E.lu_backsubstitute(LU, piv, np.ones((1, m)))
        np.testing.assert_allclose(x.cpu().numpy(), g[f"x{m}"], rtol=1e-11, atol=1e-13)


def run_cells(torch, mech, cells, deltaT, dtc0, solver, launch, Treact=0.0, relTol=1e-4, absTol=1e-8, **kw):
    s = E.Solver([mech], E.OdeInputs(name=f"Rosenbrock{solver}", absTol=absTol, relTol=relTol, **kw), Treact)
    s.set_launch(**launch)
    Y0 = torch.as_tensor(cells, dtype=torch.float64, device="cuda").contiguous()
    dtc = torch.full((cells.shape[0],), dtc0, dtype=torch.float64, device="cuda")
    out = s.solve(Y0, deltaT, dtc)
    torch.cuda.synchronize()
    return (out["Ynew"].cpu().numpy(), out["deltaTChem"].cpu().numpy(), out["counters"].cpu().numpy(),
            out["status"].cpu().numpy(), out["stats"])


@pytest.mark.parametrize("name", CASES)
@pytest.mark.parametrize("solver", [12, 23, 34])
def test_cells_vs_golden(torch, name, solver):
    """Full singleCellSolver integration vs the reference's golden outputs."""
    g, raw, mech = gpu_mech(name)
    Y, dtc, cnt, st, stats = run_cells(torch, mech, g["cells"], float(g["deltaT"]), float(g["deltaTChem0"]),
                                       solver, LAUNCHES["persist-g32-smem"], absTol=1e-8, relTol=1e-4)
    assert (st == 0).all()
    assert_states_close(Y, g[f"cells{solver}_Y"], raw.n_species, 1e-4, f"{name} R{solver}")
    # step counts: >= 99% equal; on these small samples every cell
    agree = step_count_agreement(cnt, g[f"cells{solver}_counts"])
    assert agree >= 0.99, agree
    np.testing.assert_allclose(dtc, g[f"cells{solver}_dtc"], rtol=1e-6)


@pytest.mark.parametrize("launch", list(LAUNCHES))
def test_launch_forms_agree_with_oracle(torch, launch):
    """Every launch form (plain, persistent G=1..256, shared / HBM scratch)
    against the oracle on 192 H2-size cells, R34."""
    raw = M.h2_size(0)
    mech = E.Mechanism(raw)
    cells = M.make_cells(raw, 192, seed=21)
    ref = Oracle(raw, "port").cells(ode_inputs(34), cells, 1e-5, 1e-7)
    Y, dtc, cnt, st, stats = run_cells(torch, mech, cells, 1e-5, 1e-7, 34, LAUNCHES[launch])
    assert (st == 0).all()
    assert_states_close(Y, ref[0], raw.n_species, 1e-4, launch)
    assert step_count_agreement(cnt, ref[2]) >= 0.99
    assert stats["accepted"] == int(cnt[:, 0].sum()) and stats["attempts"] == int(cnt[:, 1].sum())
    assert stats["min_delta_t"] == float(dtc.min())


def test_grisize_cells_vs_oracle(torch):
    raw = M.gri_size(0)
    mech = E.Mechanism(raw)
    cells = M.make_cells(raw, 48, seed=31)
    ref = Oracle(raw, "port").cells(ode_inputs(23), cells, 1e-6, 1e-7)
    for launch in ("persist-g32-smem", "persist-g128-smem-slim", "plain"):
        Y, dtc, cnt, st, _ = run_cells(torch, mech, cells, 1e-6, 1e-7, 23, LAUNCHES[launch])
        assert (st == 0).all()
        assert_states_close(Y, ref[0], raw.n_species, 1e-4, launch)
        assert step_count_agreement(cnt, ref[2]) >= 0.99


def test_compute_rr_mirror(torch):
    """GpuKernelEvaluator.computeRR / computeYNew (host arrays) against the
    reference's host arithmetic on oracle-integrated states."""
    g, raw, mech = gpu_mech("h2size")
    cells = g["cells"]
    n = cells.shape[0]
    ev = E.GpuKernelEvaluator(n, raw.n_eqns, raw.n_species, mech,
                              E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4))
    dt0 = np.full(n, float(g["deltaTChem0"]))
    RR, dtn, mn = ev.computeRR(float(g["deltaT"]), float(g["rr_dtcmax"]), g["rr_rho"], dt0, cells)
    Ynew, dtn2 = ev.computeYNew(float(g["deltaT"]), float(g["rr_dtcmax"]), dt0, cells)
    assert_states_close(Ynew.reshape(n, -1), g["cells34_Y"], raw.n_species, 1e-4)
    # computeYNew does not clamp; computeRR does, and returns the min before clamping
    np.testing.assert_allclose(dtn2, g["cells34_dtc"], rtol=1e-6)
    np.testing.assert_allclose(mn, g["rr_min"], rtol=1e-6)
    assert (dtn <= float(g["rr_dtcmax"])).all()
    np.testing.assert_allclose(dtn, g["rr_dtc"], rtol=1e-6)
    # RR = rho (Ynew - Y0) / deltaT inherits the state tolerance
    ref_RR = g["rr_RR"]
    tolY = 1e-9 + 10 * 1e-4 * np.abs(g["cells34_Y"][:, :raw.n_species])
    tol = g["rr_rho"][:, None] * tolY / float(g["deltaT"])
    assert (np.abs(RR.reshape(n, -1) - ref_RR) <= tol).all()


def test_compute_rr_local_time_step(torch):
    """computeRR with a flow step per cell (gf_compute_rr_lts, host arrays) against
    gf_solve with deltaT_cell on device memory: the same kernel, bit for bit, and
    RR = rho (Ynew - Y0) / deltaT_i with each cell's own step."""
    g, raw, mech = gpu_mech("h2size")
    cells = g["cells"]
    n = cells.shape[0]
    rng = np.random.default_rng(4)
    dts = M.log_uniform(rng, 1e-7, 1e-5, n)
    rho = np.linspace(0.3, 1.2, n)
    dt0 = np.full(n, 1e-7)
    ev = E.GpuKernelEvaluator(n, raw.n_eqns, raw.n_species, mech,
                              E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4))
    RR, dtn, mn = ev.computeRRLocal(dts, 5e-8, rho, dt0, cells)
    s = E.Solver([mech], E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4))
    s.set_launch(**ev.solver.get_launch())
    Yd = torch.as_tensor(cells, device="cuda")
    dtc = torch.as_tensor(dt0, device="cuda").clone()
    out = s.solve(Yd, 0.0, dtc, deltaTChemMax=5e-8, rho=torch.as_tensor(rho, device="cuda"),
                  deltaT_cell=torch.as_tensor(dts, device="cuda"),
                  RR=torch.zeros((n, raw.n_species), dtype=torch.float64, device="cuda"))
    torch.cuda.synchronize()
    assert np.array_equal(RR.reshape(n, -1), out["RR"].cpu().numpy())
    assert np.array_equal(dtn, dtc.cpu().numpy()) and mn == out["stats"]["min_delta_t"]
    Yn = out["Ynew"].cpu().numpy()
    ref = rho[:, None] * (Yn[:, :raw.n_species] - cells[:, :raw.n_species]) / dts[:, None]
    assert np.array_equal(RR.reshape(n, -1), ref)
    with pytest.raises(ValueError):
        ev.computeRRLocal(dts[:-1], 5e-8, rho, dt0, cells)


def test_treact_gate(torch):
    g, raw, mech = gpu_mech("h2size")
    Treact = float(g["treact"])
    Y, dtc, cnt, st, _ = run_cells(torch, mech, g["cells"], float(g["deltaT"]), 1e-7, 34,
                                   LAUNCHES["persist-g32-smem"], Treact=Treact)
    skipped = g["cells"][:, -2] <= Treact
    assert (st[skipped] == 4).all() and (st[~skipped] == 0).all()
    assert np.array_equal(Y[skipped], g["cells"][skipped])
    assert (dtc[skipped] == float(g["deltaT"])).all()
    assert_states_close(Y, g["cells34_treact_Y"], raw.n_species, 1e-4)


def test_max_steps_and_nonfinite_status(torch):
    raw = M.h2_size(0)
    mech = E.Mechanism(raw)
    cells = M.make_cells(raw, 4, seed=1)
    Y, dtc, cnt, st, stats = run_cells(torch, mech, cells, 1e-5, 1e-7, 34, LAUNCHES["persist-g32-smem"], maxSteps=2)
    assert (st == 2).all() and (cnt[:, 0] == 2).all() and (dtc == 1e-7).all()
    assert stats["failed"] == 4
    bad = cells.copy()
    bad[1, 0] = np.nan
    bad[2, -2] = np.nan
    for launch in ("plain", "persist-g32-smem"):
        Y, dtc, cnt, st, _ = run_cells(torch, mech, bad, 1e-5, 1e-7, 34, LAUNCHES[launch])
        assert st[1] == 3 and st[2] == 4 and st[0] == 0 and st[3] == 0


def test_determinism(torch):
    raw = M.coverage(0)
    mech = E.Mechanism(raw)
    cells = M.make_cells(raw, 96, seed=5)
    first = run_cells(torch, mech, cells, 1e-5, 1e-7, 34, LAUNCHES["persist-g32-smem"])
    for _ in range(3):
        again = run_cells(torch, mech, cells, 1e-5, 1e-7, 34, LAUNCHES["persist-g32-smem"])
        assert np.array_equal(first[0], again[0]) and np.array_equal(first[2], again[2])


@pytest.mark.parametrize("launch", ["plain", "persist-g64-smem", "persist-g8-smem"])
def test_all_cells_equal(torch, launch):
    """The reference's single-cell-solver test shape (every cell the same state,
    gpu_test_kernels.cu:659-749): every cell's result and step counts equal,
    bit for bit, whichever slot or group integrated it."""
    g, raw, mech = gpu_mech("foam_gri")
    cells = np.repeat(g["states"][:1], 300, axis=0)
    Y, dtc, cnt, st, _ = run_cells(torch, mech, cells, 1e-6, 1e-7, 34, LAUNCHES[launch])
    assert (st == 0).all()
    assert (Y == Y[0]).all() and (dtc == dtc[0]).all() and (cnt == cnt[0]).all()
    ref = Oracle(raw, "port").cells(ode_inputs(34), cells[:1], 1e-6, 1e-7)
    assert_states_close(Y[:1], ref[0], raw.n_species, 1e-4, launch)


def test_mixed_mechanisms_per_cell_dt(torch):
    """One launch over cells of two mechanisms with per-cell deltaT and p."""
    raws = [M.h2_size(0), M.coverage(0)]
    mechs = [E.Mechanism(r) for r in raws]
    rng = np.random.default_rng(3)
    n_each = 48
    ld = max(r.n_eqns for r in raws)
    Y = np.zeros((2 * n_each, ld))
    mid = np.repeat([0, 1], n_each).astype(np.int32)
    dts = M.log_uniform(rng, 1e-7, 1e-5, 2 * n_each)
    parts = []
    for k, r in enumerate(raws):
        c = M.make_cells(r, n_each, seed=40 + k, p_range=(0.5 * 101325, 40 * 101325))
        Y[k * n_each:(k + 1) * n_each, :r.n_eqns] = c
        parts.append(c)
    perm = rng.permutation(2 * n_each)
    Y, mid, dts = Y[perm], mid[perm], dts[perm]
    s = E.Solver(mechs, E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4))
    s.set_launch(kind=1, threads_per_cell=32, scratch_in_shared=1)
    Yd = torch.as_tensor(Y, device="cuda")
    dtc = torch.full((2 * n_each,), 1e-7, dtype=torch.float64, device="cuda")
    out = s.solve(Yd, 0.0, dtc, deltaT_cell=torch.as_tensor(dts, device="cuda"),
                  mech_id=torch.as_tensor(mid, device="cuda"))
    Yg = out["Ynew"].cpu().numpy()
    cnt = out["counters"].cpu().numpy()
    for k, r in enumerate(raws):
        sel = mid == k
        ref = Oracle(r, "port").cells(ode_inputs(34), Y[sel, :r.n_eqns], 0.0, 1e-7, deltaT_cell=dts[sel])
        assert_states_close(Yg[sel, :r.n_eqns], ref[0], r.n_species, 1e-4, f"mech {k}")
        assert step_count_agreement(cnt[sel], ref[2]) >= 0.99


def test_graph_replay_matches_solve(torch):
    """The captured solve (gf_solve_graph_*) against gf_solve: bit-identical
    states, steps and totals on every replay; a new flow step through
    set_delta_t; the graph unaffected by a later change of the solver's launch."""
    raws = [M.h2_size(0), M.coverage(0)]
    mechs = [E.Mechanism(r) for r in raws]
    rng = np.random.default_rng(8)
    n = 160
    ld = max(r.n_eqns for r in raws)
    Y = np.zeros((n, ld))
    mid = rng.integers(0, 2, n).astype(np.int32)
    for k, r in enumerate(raws):
        sel = mid == k
        Y[sel, :r.n_eqns] = M.make_cells(r, int(sel.sum()), seed=60 + k)
    s = E.Solver(mechs, E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4))
    s.set_launch(kind=1, threads_per_cell=32, scratch_in_shared=1)
    Yd = torch.as_tensor(Y, device="cuda")
    md = torch.as_tensor(mid, device="cuda")
    rho = torch.as_tensor(np.linspace(0.3, 1.1, n), device="cuda")

    def direct(dT):
        dtc = torch.full((n,), 1e-7, dtype=torch.float64, device="cuda")
        # zero-filled outputs: the columns past a cell's own nEqns / nSpecie are not written
        out = s.solve(Yd, dT, dtc, rho=rho, mech_id=md, Ynew=torch.zeros_like(Yd), RR=torch.zeros_like(Yd))
        torch.cuda.synchronize()
        return (out["Ynew"].cpu().numpy(), out["RR"].cpu().numpy(), dtc.cpu().numpy(),
                out["status"].cpu().numpy(), out["counters"].cpu().numpy(), out["stats"])

    ref = direct(1e-5)
    dtc = torch.empty(n, dtype=torch.float64, device="cuda")
    status = torch.empty(n, dtype=torch.int32, device="cuda")
    counters = torch.empty((n, 2), dtype=torch.int32, device="cuda")
    g = s.capture(Yd, 1e-5, dtc, rho=rho, mech_id=md, status=status, counters=counters,
                  Ynew=torch.zeros_like(Yd), RR=torch.zeros_like(Yd))
    stream = torch.cuda.Stream()
    s.set_launch(kind=0)  # the graph keeps the launch form it was captured with
    for _ in range(3):
        dtc.fill_(1e-7)
        g.launch(stream)
        stream.synchronize()
        got = (g["Ynew"].cpu().numpy(), g["RR"].cpu().numpy(), dtc.cpu().numpy(), status.cpu().numpy(),
               counters.cpu().numpy())
        for a, b in zip(got, ref[:5]):
            assert np.array_equal(a, b)
        assert g.stats() == ref[5]
    s.set_launch(kind=1, threads_per_cell=32, scratch_in_shared=1)
    ref2 = direct(3e-6)
    g.set_delta_t(3e-6)
    dtc.fill_(1e-7)
    g.launch(stream)
    stream.synchronize()
    assert np.array_equal(g["Ynew"].cpu().numpy(), ref2[0])
    assert np.array_equal(counters.cpu().numpy(), ref2[4])
    assert g.stats() == ref2[5]
    g.close()
