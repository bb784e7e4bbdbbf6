"""The launch-form autotuner on a B200: tune() times the candidate forms on a
sample of cells, applies the fastest, and that form passes parity against the
oracle on other cells of the same mechanism."""
import numpy as np
import pytest

from gpufoam_b200 import autotune
from gpufoam_b200 import evaluator as E
from gpufoam_b200 import mechanism as M
from oracle.oracle import Oracle, ode_inputs
from tests.parity import assert_states_close, step_count_agreement

pytestmark = pytest.mark.gpu


def test_tuned_form_passes_parity():
    import torch
    from gpufoam_b200 import build
    build.build()
    raw = M.gri_size(0)
    mech = E.Mechanism(raw)
    ode = E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4)
    s = E.Solver([mech], ode)
    sample = M.make_cells(raw, 2048, seed=71)
    cands = [c for c in autotune.candidates(s.workspace_doubles())
             if c["kind"] == 0 or c["threads_per_cell"] in (16, 32, 64, 96, 128)]
    res = autotune.tune(s, sample, 1e-6, configs=cands, use_cache=False)
    best = res["best"]
    assert s.get_launch() == best
    assert len(res["table"]) >= 4
    assert min(ms for _, ms in res["table"]) == [ms for c, ms in res["table"] if c == best][0]
    cells = M.make_cells(raw, 256, seed=72)
    ref = Oracle(raw, "port").cells(ode_inputs(34), cells, 1e-6, 1e-7)
    dtc = torch.full((256,), 1e-7, dtype=torch.float64, device="cuda")
    out = s.solve(torch.as_tensor(cells, device="cuda"), 1e-6, dtc)
    torch.cuda.synchronize()
    assert (out["status"].cpu().numpy() == 0).all()
    assert_states_close(out["Ynew"].cpu().numpy(), ref[0], raw.n_species, 1e-4, f"tuned form {best}")
    assert step_count_agreement(out["counters"].cpu().numpy(), ref[2]) >= 0.99


@pytest.mark.parametrize("factory", [M.h2_size, M.gri_size, M.large])
def test_tuned_variants_parity(factory):
    """Every tile and specialisation variant the autotuner can pick (LU panels
    of 4 and 16 columns; the kernel compiled for the mechanism's matrix size,
    m = 11, 54, 101) against the oracle, for 32, 64 and 128 threads per cell."""
    import torch
    from gpufoam_b200 import _native as N
    raw = factory(0)
    mech = E.Mechanism(raw)
    ode = E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4)
    n = 64
    cells = M.make_cells(raw, n, seed=73)
    dT = 1e-5 if raw.n_species <= 10 else 1e-6
    ref = Oracle(raw, "port").cells(ode_inputs(34), cells, dT, 1e-7)
    ws = E.Solver([mech], ode).workspace_doubles() * 8
    for G in (32, 64, 96, 128):
        regs = 1 if G in (96, 128) else 0
        forms = [dict(specialize=1, scratch_in_shared=0)]
        if raw.n_species == 53:
            forms += [dict(specialize=1, lu_panel=4, scratch_in_shared=0)]
        if ws <= 227 * 1024:
            forms += [dict(specialize=1, scratch_in_shared=1), dict(lu_panel=4, scratch_in_shared=1),
                      dict(lu_panel=16, scratch_in_shared=1)]
            if raw.n_species == 53:
                forms += [dict(specialize=1, lu_panel=4, scratch_in_shared=1)]
        for f in forms:
            s = E.Solver([mech], ode)
            s.set_launch(kind=1, threads_per_cell=G, register_budget=regs, **f)
            dtc = torch.full((n,), 1e-7, dtype=torch.float64, device="cuda")
            out = s.solve(torch.as_tensor(cells, device="cuda"), dT, dtc)
            torch.cuda.synchronize()
            st = out["status"].cpu().numpy()
            assert np.array_equal(st, ref[3]), (G, f)
            ok = st == 0
            assert_states_close(out["Ynew"].cpu().numpy()[ok], ref[0][ok], raw.n_species, 1e-4, f"G={G} {f}")
            assert step_count_agreement(out["counters"].cpu().numpy(), ref[2]) >= 0.99
    # forms that are not compiled are refused
    s = E.Solver([mech], ode)
    for bad in (dict(threads_per_cell=16, specialize=1), dict(threads_per_cell=64, register_budget=1, lu_panel=4),
                dict(threads_per_cell=64, lu_panel=4, scratch_in_shared=0),
                dict(threads_per_cell=64, lu_panel=16, specialize=1), dict(threads_per_cell=256, lu_panel=4)):
        with pytest.raises(N.GfError, match="UNSUPPORTED"):
            s.set_launch(kind=1, **bad)
    cov = E.Mechanism(M.coverage(0))   # 12 species: no kernel compiled for m = 13
    with pytest.raises(N.GfError, match="UNSUPPORTED"):
        E.Solver([cov], ode).set_launch(kind=1, threads_per_cell=64, specialize=1)
