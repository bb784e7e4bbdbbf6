"""gf_solve_noalloc: the solve for callers that cannot allocate device memory
(a host code whose device memory belongs to another allocator, or a loop that
forbids allocation once it has started). Its scratch is a static device array
inside the library instead of memory from cudaMalloc.

Compared through the C ABI with gf_solve on the same cells, for two calls in a
row (the second call must not see state the first left in the shared array).
This file is named to run last; it builds everything it needs, so it also
passes alone in a fresh process."""
import numpy as np
import pytest

from gpufoam_b200 import evaluator as E
from gpufoam_b200 import mechanism as M
from tests.parity import assert_states_close, step_count_agreement

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("factory,n,deltaT", [(M.gri_size, 300, 1e-6), (M.h2_size, 2000, 1e-5)])
def test_noalloc_matches_gf_solve(factory, n, deltaT):
    import torch
    from gpufoam_b200 import build
    build.build()
    raw = factory(0)
    mech = E.Mechanism(raw)
    ode = E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4)
    cells = M.make_cells(raw, n, seed=77)
    Y0 = torch.as_tensor(cells, device="cuda")
    rho = torch.linspace(0.2, 1.2, n, dtype=torch.float64, device="cuda")

    solver = E.Solver([mech], ode)
    solver.set_launch(kind=1, threads_per_cell=32, scratch_in_shared=0, register_budget=1)
    dtc_ref = torch.full((n,), 1e-7, dtype=torch.float64, device="cuda")
    ref = solver.solve(Y0, deltaT, dtc_ref, rho=rho)
    torch.cuda.synchronize()
    Y_ref = ref["Ynew"].cpu().numpy()
    RR_ref = ref["RR"][:, :raw.n_species].cpu().numpy()
    cnt_ref = ref["counters"].cpu().numpy()

    for call in range(2):
        dtc = torch.full((n,), 1e-7, dtype=torch.float64, device="cuda")
        Ynew = torch.empty_like(Y0)
        RR = torch.empty((n, raw.n_species), dtype=torch.float64, device="cuda")
        status = torch.empty(n, dtype=torch.int32, device="cuda")
        counters = torch.empty((n, 2), dtype=torch.int32, device="cuda")
        stats = E.solve_noalloc(mech, ode, Y0, deltaT, dtc, Ynew, rho=rho, RR=RR, status=status, counters=counters)
        torch.cuda.synchronize()
        Y = Ynew.cpu().numpy()
        assert (status.cpu().numpy() == 0).all(), f"call {call}"
        assert_states_close(Y, Y_ref, raw.n_species, 1e-4, f"noalloc call {call}")
        cnt = counters.cpu().numpy()
        assert step_count_agreement(cnt, cnt_ref) >= 0.99
        np.testing.assert_allclose(dtc.cpu().numpy(), dtc_ref.cpu().numpy(), rtol=1e-6)
        tol = rho.cpu().numpy()[:, None] * (1e-9 + 10 * 1e-4 * np.abs(Y_ref[:, :raw.n_species])) / deltaT
        assert (np.abs(RR.cpu().numpy() - RR_ref) <= tol).all()
        assert stats["accepted"] == int(cnt[:, 0].sum()) and stats["attempts"] == int(cnt[:, 1].sum())
        assert stats["min_delta_t"] == float(dtc.min())
