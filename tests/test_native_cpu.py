"""CPU checks of the C-ABI library: it loads, exports every declared symbol, and
its host-side loader arithmetic (makeGpuThermo x R scaling, set_reaction_thermo
ΔThermo, integer-exponent detection) reproduces the reference's processed
tables bit for bit. No compute call needs a GPU here."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from gpufoam_b200 import _native as N
from gpufoam_b200 import build as B
from gpufoam_b200 import evaluator as E
from gpufoam_b200 import mechanism as M

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
GOLDEN = os.path.join(ROOT, "tests", "golden")


@pytest.fixture(scope="module")
def lib():
    B.build()
    return N.load()


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "gpufoam_b200.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gf_[a-z_0-9]+)\s*\(", txt)))


def test_exports_every_declared_symbol(lib):
    syms = header_symbols()
    assert len(syms) >= 19
    for s in syms:
        assert hasattr(lib, s), s
    assert set(syms) == set(N.EXPORTS)
    assert lib.gf_abi_version() == 1


def test_strerror(lib):
    assert lib.gf_strerror(0) == b"ok"
    assert lib.gf_strerror(2) == b"Invalid ODE Solver type"


@pytest.mark.parametrize("name", ["h2size", "coverage", "grisize", "foam_h2", "foam_gri", "foam_yao"])
def test_loader_arithmetic_matches_reference_tables(lib, name):
    from tests.test_oracle import fixture_mech
    g = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    mech = fixture_mech(g)
    th = E.make_gpu_thermos(mech)
    rx, _keep = E.make_gpu_reactions(mech, th)
    assert np.array_equal(E.thermo_table(th, mech.n_species), g["species_tables"])
    assert np.array_equal(E.thermo_table(rx, mech.n_reactions), g["reaction_tables"])
    ie = g["int_exponents"]
    for r in range(mech.n_reactions):
        for k in range(rx[r].n_lhs):
            assert rx[r].lhs[k].integer_exponent == ie[r, k]
        for k in range(rx[r].n_rhs):
            assert rx[r].rhs[k].integer_exponent == ie[r, 10 + k]


def test_mass_imbalance_rejected(lib):
    mech = M.h2_size(0)
    th = E.make_gpu_thermos(mech)
    lhs = (N.GfSpecieCoeff * 10)()
    rhs = (N.GfSpecieCoeff * 10)()
    lhs[0] = N.GfSpecieCoeff(0, 1, 1.0, 1.0)   # H
    rhs[0] = N.GfSpecieCoeff(4, 1, 1.0, 1.0)   # O2: not balanced
    out = N.GfThermo()
    assert lib.gf_reaction_thermo(th, mech.n_species, 1, lhs, 1, rhs, C.byref(out)) == 4


def test_unknown_solver_rejected(lib):
    assert lib.gf_solver_create(None, 1, None, 0.0, None) == 1
    fake = (C.c_void_p * 1)(C.c_void_p(0x1000).value)
    ode = N.GfOdeInputs(99, 1e-8, 1e-4, 10000, 0.9, 0.2, 0.25, 0.2, 10.0)
    h = C.c_void_p()
    assert lib.gf_solver_create(fake, 1, C.byref(ode), 0.0, C.byref(h)) == 2
    with pytest.raises(ValueError, match="Invalid ODE Solver type"):
        E.OdeInputs(name="seulex").to_c()


def test_ode_input_defaults():
    o = E.read_gpuODESolverInputs({"solver": "Rosenbrock23"})
    assert (o.absTol, o.relTol, o.maxSteps, o.safeScale, o.alphaInc, o.alphaDec, o.minScale, o.maxScale) == (
        np.finfo(float).eps, 1e-4, 10000, 0.9, 0.2, 0.25, 0.2, 10.0)


def test_is_integer_rule():
    # isInteger truncates toward zero and only rejects a positive remainder
    assert E.is_integer(2.0) and E.is_integer(-0.5) and not E.is_integer(1.5)


def test_null_handles_rejected_without_a_device(lib):
    """Entry points added around the solve reject missing handles before any
    CUDA call (no GPU needed)."""
    st = N.GfStats()
    out = C.c_void_p()
    assert lib.gf_solve_graph_create(None, 4, 1e-6, None, 1.0, None, None, None, 12, None, None, None, 0, None,
                                     None, C.byref(out)) == 1
    assert lib.gf_solve_graph_launch(None, None) == 1
    assert lib.gf_solve_graph_set_delta_t(None, 1e-6) == 1
    assert lib.gf_solve_graph_stats(None, C.byref(st)) == 1
    lib.gf_solve_graph_destroy(None)
    assert lib.gf_cell_rates(None, 4, None, None, 12, None, 10, None, None) == 1
    assert lib.gf_reaction_rates(None, 4, 0, None, None, 12, None, None, 10, None) == 1
    assert lib.gf_qdot(None, 4, None, 10, None, None) == 1


def test_solve_tensor_checks():
    """The solve wrappers refuse, before any pointer reaches the C ABI, a tensor
    the kernels would read or write past its end, one of the wrong type, and one
    that is not on Y0's CUDA device (on this machine every tensor is on the
    CPU, so a tensor that passes the type and size checks fails the device one)."""
    import torch
    f64, i32 = torch.float64, torch.int32
    n, ne, ns = 4, 12, 10
    Y0 = torch.zeros((n, ne), dtype=f64)

    def refused(match, **kw):
        with pytest.raises(ValueError, match=match):
            E.check_solve_tensors(n, ne, ns, kw.pop("Y0", Y0), **kw)

    # type and size failures, each caught before the device check
    refused("Y0 must be float64", Y0=Y0.float())
    refused("Y0 must be a row-contiguous", Y0=torch.zeros((n, ne - 1), dtype=f64))
    refused("Y0 must be a row-contiguous", Y0=torch.zeros((ne, n), dtype=f64).t())
    refused("Ynew must be a row-contiguous", Ynew=torch.zeros((n, ne - 1), dtype=f64))
    refused("Ynew must have Y0's shape", Ynew=torch.zeros((n, ne + 2), dtype=f64))
    refused("RR must be a row-contiguous", RR=torch.zeros((n - 1, ns), dtype=f64))
    refused("RR must be a row-contiguous", RR=torch.zeros((n, ns - 1), dtype=f64))
    refused("RR must be float64", RR=torch.zeros((n, ns), dtype=torch.float32))
    refused("deltaTChem must be torch.float64", deltaTChem=torch.zeros(n, dtype=torch.float32))
    refused("deltaTChem must be a contiguous tensor of at least 4", deltaTChem=torch.zeros(n - 1, dtype=f64))
    refused("rho must be a contiguous tensor", rho=torch.zeros(2 * n, dtype=f64)[::2])
    refused("deltaT_cell must be a contiguous tensor", deltaT_cell=torch.zeros(1, dtype=f64))
    refused("mech_id must be torch.int32", mech_id=torch.zeros(n, dtype=torch.int64))
    refused("status must be a contiguous tensor", status=torch.zeros(n - 1, dtype=i32))
    refused("counters must be a contiguous tensor of at least 8", counters=torch.zeros((n, 1), dtype=i32))
    refused("must be a torch tensor", deltaTChem=np.zeros(n))
    # right types and sizes: only the device is wrong here
    refused("must be on Y0's CUDA device", Ynew=torch.zeros_like(Y0), RR=torch.zeros((n, ns), dtype=f64),
            deltaTChem=torch.zeros(n, dtype=f64), rho=torch.zeros(n, dtype=f64),
            mech_id=torch.zeros(n, dtype=i32), status=torch.zeros(n, dtype=i32),
            counters=torch.zeros((n, 2), dtype=i32))


def test_host_array_checks():
    """computeRR / computeYNew refuse host arrays whose sizes do not match nCells."""
    n, ne = 5, 12
    E.check_host_arrays(n, ne, np.zeros(n * ne), np.zeros(n), np.zeros(n), np.zeros(n))
    with pytest.raises(ValueError, match="nCells"):
        E.check_host_arrays(n, ne, np.zeros(n * ne - 1), np.zeros(n))
    with pytest.raises(ValueError, match="rho"):
        E.check_host_arrays(n, ne, np.zeros(n * ne), np.zeros(n), np.zeros(n + 1))
    with pytest.raises(ValueError, match="deltaT "):
        E.check_host_arrays(n, ne, np.zeros(n * ne), np.zeros(n), np.zeros(n), np.zeros(n - 1))


@pytest.mark.parametrize("name", ["h2size", "coverage", "grisize", "foam_h2", "foam_gri", "foam_yao"])
def test_device_tables_pass_the_bounds_check(lib, name):
    """gf_mech_create checks every index the kernels follow (gather-stream
    positions and slots, staging slots, third-body rows, species entries) before
    it allocates: on a machine without a GPU a valid mechanism gets as far as the
    allocation (GF_ERR_NO_DEVICE), a bad table would stop at GF_ERR_UNSUPPORTED."""
    import torch
    from tests.test_oracle import fixture_mech
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the allocation succeeds")
    raw = fixture_mech(dict(np.load(os.path.join(GOLDEN, f"{name}.npz"))))
    with pytest.raises(N.GfError, match="GF_ERR_NO_DEVICE"):
        E.Mechanism(raw)


def test_autotune_cache_key_follows_the_build(monkeypatch):
    """A cached launch pick is keyed on the library build: a different build
    digest gives a different key (no GPU needed: the device name is faked)."""
    import torch
    from gpufoam_b200 import autotune

    class FakeMech:
        n_species, n_reactions = 53, 325

        class raw:
            name = "gri_size"

    monkeypatch.setattr(torch.cuda, "get_device_name", lambda *a: "B200")
    ode = E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4)
    monkeypatch.setattr(autotune, "_BUILD_HASH", "aaaa")
    k1 = autotune._key([FakeMech()], ode)
    monkeypatch.setattr(autotune, "_BUILD_HASH", "bbbb")
    assert autotune._key([FakeMech()], ode) != k1
    monkeypatch.setattr(autotune, "_BUILD_HASH", None)
    assert len(autotune.build_hash()) == 16
