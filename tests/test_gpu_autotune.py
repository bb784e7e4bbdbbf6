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
             if c["kind"] == 0 or c["threads_per_cell"] in (16, 32, 64, 128)]
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
