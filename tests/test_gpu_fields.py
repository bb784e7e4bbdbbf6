"""GPU parity of the plugin's per-cell side paths (gf_cell_rates, gf_reaction_rates,
gf_qdot; the reference computes them on the CPU, gpuChemistryModel.C:145-450)
against the reference's own code compiled for the CPU (oracle/_ref), on the six
fixture mechanisms, the reference's three real ones among them.

Tolerances: the rates follow the project's parity contract (1e-12 of the
gross-rate scale W_i sum_r |nu_ir| (|kf Cf| + |kr Cr|), since omega = kf Cf -
kr Cr cancels); tc 1e-12 relative; Qdot bit-exact on the same RR (the
reference's sequential sum)."""
import ctypes as C

import numpy as np
import pytest

from gpufoam_b200 import _native as N
from gpufoam_b200 import evaluator as E
from oracle.oracle import Oracle
from tests.test_gpu_parity import CASES, gpu_mech

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def torch():
    import torch
    from gpufoam_b200 import build
    build.build()
    assert torch.cuda.is_available()
    return torch


def species_scale(raw, parts):
    """W_i sum_r |nu_ir| (|kf Cf| + |kr Cr|) per cell and species."""
    n = parts.shape[0]
    sc = np.zeros((n, raw.n_species))
    gross = np.abs(parts).sum(axis=2)  # [n][nR]
    for r, rx in enumerate(raw.reactions):
        for i, st, _ in rx.lhs + rx.rhs:
            sc[:, i] += abs(st) * gross[:, r]
    return sc * raw.W


def states_of(g, raw, n_random, seed):
    from gpufoam_b200 import mechanism as M
    y = g["states"]
    if n_random:
        y = np.vstack([y, M.make_cells(raw, n_random, seed=seed)])
    rho = np.random.default_rng(seed).uniform(0.05, 2.0, y.shape[0])
    return rho, y


@pytest.mark.parametrize("name", CASES)
def test_calculate_and_tc(torch, name):
    g, raw, mech = gpu_mech(name)
    rho, y = states_of(g, raw, 0, 3)
    ref_RR, ref_tc = Oracle(raw, "reference").cell_fields(rho, y)
    RR, tc = E.cell_rates(mech, rho, y)
    RR, tc = RR.cpu().numpy(), tc.cpu().numpy()
    sc = species_scale(raw, Oracle(raw, "port").rate_parts(rho, y))
    assert (np.abs(RR - ref_RR) <= 1e-12 * sc + 1e-300).all()
    assert np.allclose(tc, ref_tc, rtol=1e-12, atol=0)
    # either output alone
    RR2, none = E.cell_rates(mech, rho, y, want_tc=False)
    assert none is None and np.array_equal(RR2.cpu().numpy(), RR)
    none, tc2 = E.cell_rates(mech, rho, y, want_RR=False)
    assert none is None and np.array_equal(tc2.cpu().numpy(), tc)


@pytest.mark.parametrize("name", ["grisize", "foam_gri", "foam_yao"])
def test_calculate_many_cells(torch, name):
    """Thousands of cells (every warp takes several, grid-stride) against the port."""
    g, raw, mech = gpu_mech(name)
    rho, y = states_of(g, raw, 6000, 8)
    o = Oracle(raw, "port")
    ref_RR, ref_tc = o.cell_fields(rho, y)
    RR, tc = E.cell_rates(mech, rho, y)
    sc = species_scale(raw, o.rate_parts(rho, y))
    assert (np.abs(RR.cpu().numpy() - ref_RR) <= 1e-12 * sc + 1e-300).all()
    assert np.allclose(tc.cpu().numpy(), ref_tc, rtol=1e-12, atol=0)


def test_tc_without_reactions_running(torch):
    """All concentrations zero: no reaction runs, tc = vGreat (the reference's branch)."""
    g, raw, mech = gpu_mech("foam_h2")
    y = g["states"][:4]
    _, tc = E.cell_rates(mech, np.zeros(4), y, want_RR=False)
    ref = Oracle(raw, "reference").cell_fields(np.zeros(4), y)[1]
    assert np.array_equal(tc.cpu().numpy(), ref)
    assert (ref == np.finfo(np.float64).max / 10).all()


@pytest.mark.parametrize("name", CASES)
def test_reaction_rr(torch, name):
    g, raw, mech = gpu_mech(name)
    rho, y = states_of(g, raw, 24, 4)
    ref = Oracle(raw, "reference")
    parts = Oracle(raw, "port").rate_parts(rho, y)
    # the first reaction of every rate type, the irreversible ones, and a few more
    pick = set()
    for t in range(4):
        pick.update([r for r, rx in enumerate(raw.reactions) if rx.rate_type == t][:2])
    pick.update([r for r, rx in enumerate(raw.reactions) if rx.irreversible][:2])
    pick.update(np.random.default_rng(1).choice(raw.n_reactions, size=min(6, raw.n_reactions), replace=False))
    for r in sorted(int(x) for x in pick):
        om, RR = E.reaction_rates(mech, r, rho, y)
        ref_om, ref_RR = ref.reaction_fields(r, rho, y)
        gross = np.abs(parts[:, r]).sum(axis=1)
        assert (np.abs(om.cpu().numpy() - ref_om) <= 1e-12 * gross + 1e-300).all(), r
        sc = np.zeros((y.shape[0], raw.n_species))
        for i, st, _ in raw.reactions[r].lhs + raw.reactions[r].rhs:
            sc[:, i] += abs(st) * gross * raw.W[i]
        assert (np.abs(RR.cpu().numpy() - ref_RR) <= 1e-12 * sc + 1e-300).all(), r


@pytest.mark.parametrize("name", CASES)
def test_qdot_bit_exact(torch, name):
    g, raw, mech = gpu_mech(name)
    rng = np.random.default_rng(5)
    RR = rng.standard_normal((5000, raw.n_species)) * 10.0 ** rng.uniform(-3, 3, (5000, 1))
    ref = Oracle(raw, "reference").qdot(RR)
    assert np.array_equal(E.qdot(mech, RR).cpu().numpy(), ref)
    assert np.array_equal(Oracle(raw, "port").qdot(RR), ref)


def test_side_path_argument_checks(torch):
    g, raw, mech = gpu_mech("h2size")
    lib = N.load()
    y = torch.zeros((2, raw.n_eqns), dtype=torch.float64, device="cuda")
    rho = torch.ones(2, dtype=torch.float64, device="cuda")
    out = torch.zeros((2, raw.n_species), dtype=torch.float64, device="cuda")
    p = lambda t: C.c_void_p(t.data_ptr())
    assert lib.gf_cell_rates(mech.handle, 2, p(rho), p(y), raw.n_eqns - 1, p(out), raw.n_species, None, None) == 1
    assert lib.gf_cell_rates(mech.handle, 2, p(rho), p(y), raw.n_eqns, p(out), raw.n_species - 1, None, None) == 1
    assert lib.gf_reaction_rates(mech.handle, 2, raw.n_reactions, p(rho), p(y), raw.n_eqns, None, p(out),
                                 raw.n_species, None) == 1
    assert lib.gf_reaction_rates(mech.handle, 2, -1, p(rho), p(y), raw.n_eqns, None, p(out), raw.n_species,
                                 None) == 1
    assert lib.gf_qdot(mech.handle, 2, p(out), raw.n_species - 1, p(rho), None) == 1
    assert lib.gf_cell_rates(mech.handle, 0, None, None, raw.n_eqns, None, raw.n_species, None, None) == 0
