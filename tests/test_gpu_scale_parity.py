"""GPU parity on the batches and launch forms that bench.py measures.

The cells come from the benchmark's own batches (bench.make_batch, the same
seeds): a stratified sample of each, integrated on the GPU in the launch form
the benchmark times and in the plain one-thread-per-cell form, and compared
with the CPU oracle (oracle/gf_oracle.c, pinned bit for bit to the reference)
cell by cell:

* |dY| <= 1e-9 + 10 relTol |Y|, |dT| <= 1e-3 K, p unchanged;
* accepted-step counts equal in >= 99% of the cells;
* per-cell statuses equal (the 100-species mechanism has cells that end
  non-finite in the reference itself: a Rosenbrock stage point leaves the
  physical range and the error norm's fmax ignores the NaN, so the step is
  accepted; the kernels keep that rule).
"""
import numpy as np
import pytest

import bench
from gpufoam_b200 import evaluator as E
from oracle.oracle import Oracle, ode_inputs
from tests.parity import assert_states_close, step_count_agreement

pytestmark = pytest.mark.gpu

# the forms the autotuner picks between on the GRI-size batches (the fastest
# first: 128 threads, 4-column LU panels, the kernel compiled for m = 54)
BENCH_FORMS = {
    "g128-slim-panel4-m54": dict(kind=1, threads_per_cell=128, scratch_in_shared=1, register_budget=1, lu_panel=4,
                                 specialize=1),
    "g96-slim-panel4-m54": dict(kind=1, threads_per_cell=96, scratch_in_shared=1, register_budget=1, lu_panel=4,
                                specialize=1),
    "g64-panel4-m54": dict(kind=1, threads_per_cell=64, scratch_in_shared=1, lu_panel=4, specialize=1),
    "g64-panel4": dict(kind=1, threads_per_cell=64, scratch_in_shared=1, lu_panel=4),
    "g64": dict(kind=1, threads_per_cell=64, scratch_in_shared=1, register_budget=0),
}
PLAIN = dict(kind=0)


@pytest.fixture(scope="module")
def torch():
    import torch
    from gpufoam_b200 import build
    build.build()
    assert torch.cuda.is_available()
    return torch


def stratified(values, edges, per_bin, seed):
    """Indices of per_bin cells drawn from each [edges[k], edges[k+1]) bin of values."""
    rng = np.random.default_rng(seed)
    out = []
    for lo, hi in zip(edges[:-1], edges[1:]):
        idx = np.nonzero((values >= lo) & (values < hi))[0]
        out.append(rng.choice(idx, size=min(per_bin, idx.size), replace=False))
    return np.sort(np.concatenate(out))


def solve(torch, mechs, ode, cells, deltaT, launch, mech_id=None, dT_cell=None):
    s = E.Solver(mechs, ode)
    s.set_launch(**launch)
    Y0 = torch.as_tensor(cells, device="cuda")
    dtc = torch.full((cells.shape[0],), bench.DTC0, dtype=torch.float64, device="cuda")
    out = s.solve(Y0, deltaT, dtc, mech_id=None if mech_id is None else torch.as_tensor(mech_id, device="cuda"),
                  deltaT_cell=None if dT_cell is None else torch.as_tensor(dT_cell, device="cuda"))
    torch.cuda.synchronize()
    return (out["Ynew"].cpu().numpy(), dtc.cpu().numpy(), out["counters"].cpu().numpy(),
            out["status"].cpu().numpy())


def compare(got, ref, raw, what):
    Y, dtc, cnt, st = got
    rY, rdtc, rcnt, rst = ref
    assert np.array_equal(st, rst), f"{what}: statuses differ in {(st != rst).sum()} cells"
    ok = rst == 0
    assert_states_close(Y[ok, :raw.n_eqns], rY[ok], raw.n_species, 1e-4, what)
    agree = step_count_agreement(cnt, rcnt)
    assert agree >= 0.99, f"{what}: accepted-step counts equal in {agree:.4f} of the cells"
    same = ok & (cnt[:, 0] == rcnt[:, 0])
    np.testing.assert_allclose(dtc[same], rdtc[same], rtol=1e-5, err_msg=what)
    return agree


@pytest.mark.parametrize("workload, edges", [
    ("gri-100k", [1000.0, 1375.0, 1750.0, 2125.0, 2500.1]),
    # the cold (near-inert) and the igniting modes of the bimodal batch
    ("gri-bimodal-1M", [300.0, 700.1, 1100.0, 2400.1]),
])
def test_bench_batch_sample(torch, workload, edges):
    """A stratified 2048-cell sample of the benchmark batch (seed 1000, as the
    single-GPU bench) in the forms the benchmark's autotuner picks between and
    the plain form."""
    wl = bench.WORKLOADS[workload]
    batch = bench.make_batch(wl, seed=1000)
    raw = batch.raws[0]
    T = batch.cells[:, raw.n_species]
    per_bin = 2048 // (len(edges) - 1)
    idx = stratified(T, np.array(edges), per_bin, seed=3)
    if workload == "gri-bimodal-1M":
        # 1024 cold and 1024 igniting cells
        cold = stratified(T, np.array(edges[:2]), 1024, seed=3)
        hot = stratified(T, np.array(edges[2:]), 1024, seed=4)
        idx = np.sort(np.concatenate([cold, hot]))
    cells = np.ascontiguousarray(batch.cells[idx])
    ref = Oracle(raw, "port").cells(ode_inputs(34), cells, wl["dT"], bench.DTC0)
    mech = E.Mechanism(raw)
    ode = E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4)
    for name, form in list(BENCH_FORMS.items()) + [("plain", PLAIN)]:
        got = solve(torch, [mech], ode, cells, wl["dT"], form)
        compare(got, ref, raw, f"{workload} {name}")


MIXED_FORMS = {
    "g256-smem": dict(kind=1, threads_per_cell=256, scratch_in_shared=1),
    "g32-smem": dict(kind=1, threads_per_cell=32, scratch_in_shared=1),
    "g64-hbm": dict(kind=1, threads_per_cell=64, scratch_in_shared=0),
    "plain": PLAIN,
}


@pytest.fixture(scope="module")
def mixed_case(torch):
    """A sample of the mixed batch (10-, 53- and 100-species mechanisms, per-cell
    deltaT ~ log-U[1e-7, 1e-4] s, p ~ U[0.5, 40] atm) and the oracle's results
    for each mechanism's cells."""
    wl = bench.WORKLOADS["mixed-750k"]
    batch = bench.make_batch(wl, seed=1000)
    rng = np.random.default_rng(9)
    take = {0: 512, 1: 384, 2: 192}
    idx = np.sort(np.concatenate([rng.choice(np.nonzero(batch.mech_id == k)[0], size=v, replace=False)
                                  for k, v in take.items()]))
    cells = np.ascontiguousarray(batch.cells[idx])
    mid = batch.mech_id[idx].copy()
    dts = batch.dT_cell[idx].copy()
    refs = {}
    for k, raw in enumerate(batch.raws):
        sel = mid == k
        refs[k] = Oracle(raw, "port").cells(ode_inputs(34), cells[sel, :raw.n_eqns], 0.0, bench.DTC0,
                                            deltaT_cell=dts[sel])
    mechs = [E.Mechanism(r) for r in batch.raws]
    return batch.raws, mechs, cells, mid, dts, refs


@pytest.mark.parametrize("form", list(MIXED_FORMS))
def test_mixed_batch_sample(torch, mixed_case, form):
    """One launch over cells of three mechanisms (m = 11, 54 and 101: the
    register-panel LU and the blocked LU for the 100-species cells) with a
    flow step and a pressure per cell."""
    raws, mechs, cells, mid, dts, refs = mixed_case
    ode = E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4)
    Y, dtc, cnt, st = solve(torch, mechs, ode, cells, 0.0, MIXED_FORMS[form], mech_id=mid, dT_cell=dts)
    for k, raw in enumerate(raws):
        sel = mid == k
        compare((Y[sel], dtc[sel], cnt[sel], st[sel]), refs[k], raw, f"mixed {form}, {raw.n_species} species")


@pytest.mark.parametrize("form", ["plain", "g8-smem", "g32-smem", "g64-smem", "g256-hbm"])
def test_bad_mechanism_id(torch, form):
    """Cells whose mechanism id is outside the solver's mechanisms: status
    GF_CELL_BAD_MECHANISM, the input row copied to Ynew, RR and counters zero,
    deltaTChem unchanged, counted as failed; every other cell as the oracle."""
    from gpufoam_b200 import mechanism as M
    raws = [M.h2_size(0), M.coverage(0)]
    mechs = [E.Mechanism(r) for r in raws]
    launch = PLAIN if form == "plain" else dict(kind=1, threads_per_cell=int(form.split("-")[0][1:]),
                                                 scratch_in_shared=int(form.endswith("smem")))
    n = 96
    ld = max(r.n_eqns for r in raws)
    rng = np.random.default_rng(12)
    mid = rng.integers(0, 2, n).astype(np.int32)
    bad = np.zeros(n, dtype=bool)
    bad[[3, 17, 40, 41, 95]] = True
    mid[bad] = np.array([2, -1, 7, 1 << 30, -(1 << 30)], dtype=np.int32)
    Y = np.zeros((n, ld))
    for k, r in enumerate(raws):
        sel = mid == k
        Y[sel, :r.n_eqns] = M.make_cells(r, int(sel.sum()), seed=30 + k)
    Y[bad] = rng.uniform(0.0, 1.0, size=(bad.sum(), ld))
    s = E.Solver(mechs, E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4))
    s.set_launch(**launch)
    Yd = torch.as_tensor(Y, device="cuda")
    dtc0 = np.full(n, 3e-8)
    dtc = torch.as_tensor(dtc0, device="cuda").clone()
    rho = torch.as_tensor(np.linspace(0.3, 1.1, n), device="cuda")
    out = s.solve(Yd, 1e-5, dtc, rho=rho, mech_id=torch.as_tensor(mid, device="cuda"),
                  Ynew=torch.full_like(Yd, np.nan), RR=torch.full_like(Yd, np.nan))
    torch.cuda.synchronize()
    st = out["status"].cpu().numpy()
    Yn = out["Ynew"].cpu().numpy()
    RR = out["RR"].cpu().numpy()
    cnt = out["counters"].cpu().numpy()
    dtn = dtc.cpu().numpy()
    assert (st[bad] == 5).all() and (st[~bad] == 0).all()
    assert np.array_equal(Yn[bad], Y[bad]) and (RR[bad] == 0).all() and (cnt[bad] == 0).all()
    assert np.array_equal(dtn[bad], dtc0[bad])
    assert out["stats"]["failed"] == int(bad.sum())
    assert out["stats"]["min_delta_t"] == float(dtn[~bad].min())
    for k, r in enumerate(raws):
        sel = mid == k
        ref = Oracle(r, "port").cells(ode_inputs(34), Y[sel, :r.n_eqns], 1e-5, 3e-8)
        assert_states_close(Yn[sel, :r.n_eqns], ref[0], r.n_species, 1e-4, f"{form} mech {k}")
        assert step_count_agreement(cnt[sel], ref[2]) >= 0.99
