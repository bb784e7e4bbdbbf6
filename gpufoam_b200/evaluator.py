"""Host-side mirror of gpuFoam's chemistry evaluator, over the C ABI.

Reference interfaces mirrored (paths relative to gpu_chemistry/src/):
  * ``read_gpuODESolverInputs`` — gpuOde/readGpuOdeInputs.H:8-26 (defaults);
  * ``make_gpu_thermos`` / ``make_gpu_reactions`` — gpuThermo/makeGpuThermo.H:16-66
    and gpuReaction/makeGpuReactions.H:18-142 (x R scaling, reaction ΔThermo,
    integer-exponent detection) on a RawMechanism instead of OpenFOAM dictionaries;
  * ``GpuKernelEvaluator`` — gpuKernelEvaluator/gpuKernelEvaluator.H:18-85:
    ``computeYNew`` and ``computeRR`` with the same arguments, results and error
    behaviour (an unknown solver name raises, as make_gpuODESolver throws).

Device memory and streams come from PyTorch; the computation is the CUDA path
of libgpufoam_b200.so. There is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
from typing import Optional, Sequence

import numpy as np

from . import _native as N
from .mechanism import RATE_ARRHENIUS, RawMechanism

_SOLVERS = {"Rosenbrock12": 12, "Rosenbrock23": 23, "Rosenbrock34": 34}
_DBL_EPS = np.finfo(np.float64).eps


@dataclasses.dataclass
class OdeInputs:
    """gpuODESolverInputs (gpuOde/gpuODESolverInputs.H:9-23)."""
    name: str = "Rosenbrock34"
    absTol: float = _DBL_EPS
    relTol: float = 1e-4
    maxSteps: int = 10000
    safeScale: float = 0.9
    alphaInc: float = 0.2
    alphaDec: float = 0.25
    minScale: float = 0.2
    maxScale: float = 10.0

    def to_c(self) -> N.GfOdeInputs:
        if self.name not in _SOLVERS:
            # make_gpuODESolver throws std::logic_error (makeGpuOdeSolver.H:28)
            raise ValueError("Invalid ODE Solver type")
        return N.GfOdeInputs(_SOLVERS[self.name], self.absTol, self.relTol, int(self.maxSteps), self.safeScale,
                             self.alphaInc, self.alphaDec, self.minScale, self.maxScale)


def read_gpuODESolverInputs(d: dict) -> OdeInputs:
    """odeCoeffs dictionary -> OdeInputs, with the reference's defaults."""
    return OdeInputs(name=d["solver"], absTol=d.get("absTol", _DBL_EPS), relTol=d.get("relTol", 1e-4),
                     maxSteps=int(d.get("maxSteps", 10000)), safeScale=d.get("safeScale", 0.9),
                     alphaInc=d.get("alphaIncrease", 0.2), alphaDec=d.get("alphaDecrease", 0.25),
                     minScale=d.get("minScale", 0.2), maxScale=d.get("maxScale", 10.0))


def is_integer(x: float) -> bool:
    """isInteger (gpuReaction/gpuSpecieExponent.H:7-19): truncate, integer unless positive remainder."""
    X = int(x)
    return not (x - X > 0)


def make_gpu_thermos(mech: RawMechanism):
    lib = N.load()
    arr = (N.GfThermo * mech.n_species)()
    for i in range(mech.n_species):
        hi = (C.c_double * 7)(*mech.high_raw[i])
        lo = (C.c_double * 7)(*mech.low_raw[i])
        N.check(lib.gf_thermo_from_nasa(1.0, float(mech.W[i]), float(mech.Tlow[i]), float(mech.Thigh[i]),
                                        float(mech.Tcommon[i]), hi, lo, C.byref(arr[i])), "gf_thermo_from_nasa")
    return arr


def _coeffs(side):
    out = (N.GfSpecieCoeff * N.GF_MAX_REACTION_WIDTH)()
    if len(side) > N.GF_MAX_REACTION_WIDTH:
        raise ValueError("Too long reaction")
    for k, (idx, st, ex) in enumerate(side):
        integer = is_integer(ex)
        out[k] = N.GfSpecieCoeff(int(idx), int(integer), float(st), float(int(ex)) if integer else float(ex))
    return out


def make_gpu_reactions(mech: RawMechanism, thermos):
    lib = N.load()
    arr = (N.GfReaction * max(mech.n_reactions, 1))()
    keep = []
    for r, rx in enumerate(mech.reactions):
        g = arr[r]
        g.n_lhs, g.n_rhs = len(rx.lhs), len(rx.rhs)
        g.lhs = _coeffs(rx.lhs)
        g.rhs = _coeffs(rx.rhs)
        N.check(lib.gf_reaction_thermo(thermos, mech.n_species, g.n_lhs, g.lhs, g.n_rhs, g.rhs, C.byref(g.thermo)),
                "gf_reaction_thermo")
        g.rate_type = rx.rate_type
        g.irreversible = int(rx.irreversible)
        g.A, g.beta, g.Ta = rx.A, rx.beta, rx.Ta
        g.Ainf, g.betainf, g.Tainf = rx.Ainf, rx.betainf, rx.Tainf
        g.troe_alpha, g.troe_Tsss, g.troe_Ts, g.troe_Tss = rx.troe
        if rx.rate_type != RATE_ARRHENIUS:
            e = np.ascontiguousarray(rx.efficiencies, dtype=np.float64)
            keep.append(e)
            g.efficiencies = e.ctypes.data_as(C.POINTER(C.c_double))
        g.Tlow, g.Thigh = mech.rxn_Tlow, mech.rxn_Thigh
    return arr, keep


def thermo_table(arr, n) -> np.ndarray:
    """[n][19] = Y, W, Tlow, Thigh, Tcommon, high[7], low[7] (the oracle's table layout)."""
    out = np.zeros((n, 19))
    for i in range(n):
        t = arr[i]
        if isinstance(t, N.GfReaction):
            t = t.thermo
        out[i, :5] = (t.Y, t.W, t.Tlow, t.Thigh, t.Tcommon)
        out[i, 5:12] = list(t.high)
        out[i, 12:19] = list(t.low)
    return out


class Mechanism:
    """Device-resident mechanism tables (gf_mech)."""

    def __init__(self, raw: RawMechanism):
        import torch  # noqa: F401  (initialises the CUDA context torch shares)
        self.raw = raw
        self.lib = N.load()
        self.thermos = make_gpu_thermos(raw)
        self.reactions, self._keep = make_gpu_reactions(raw, self.thermos)
        desc = N.GfMechDesc(raw.n_species, raw.n_reactions, self.thermos, self.reactions)
        h = C.c_void_p()
        N.check(self.lib.gf_mech_create(C.byref(desc), C.byref(h)), "gf_mech_create")
        self.handle = h
        self.n_species = raw.n_species
        self.n_reactions = raw.n_reactions
        self.n_eqns = raw.n_species + 2

    def tables(self):
        return thermo_table(self.thermos, self.n_species), thermo_table(self.reactions, self.n_reactions)

    def device_bytes(self) -> int:
        b = C.c_longlong()
        N.check(self.lib.gf_mech_info(self.handle, None, None, C.byref(b)), "gf_mech_info")
        return b.value

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gf_mech_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def _stream_ptr(stream=None):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return C.c_void_p(s.cuda_stream)


def _dev(x, dtype=None):
    import torch
    t = torch.as_tensor(x)
    if dtype is not None:
        t = t.to(dtype)
    return t.to("cuda").contiguous()


def _ptr(t):
    return C.c_void_p(t.data_ptr()) if t is not None else None


def check_solve_tensors(n, n_eqns, n_species, Y0, Ynew=None, RR=None, deltaTChem=None, rho=None,
                        deltaT_cell=None, mech_id=None, status=None, counters=None):
    """Every tensor a solve reads or writes, checked before the C ABI sees a
    pointer (the kernels index them by cell with no size information):
    float64 (int32 for mech_id, status, counters), the sizes the solve touches
    (Y0/Ynew rows of at least n_eqns, RR rows of at least n_species, one value
    per cell, counters [n][2]), contiguous rows, and all on Y0's CUDA device.
    Raises ValueError."""
    import torch
    f64, i32 = torch.float64, torch.int32

    def tensor(name, t):
        if not isinstance(t, torch.Tensor):
            raise ValueError(f"{name} must be a torch tensor")
        return t

    Y0 = tensor("Y0", Y0)
    if Y0.dtype != f64:
        raise ValueError("Y0 must be float64")
    if Y0.dim() != 2 or Y0.shape[0] != n or Y0.shape[1] < n_eqns or Y0.stride(1) != 1:
        raise ValueError(f"Y0 must be a row-contiguous [{n}][>= {n_eqns}] tensor")
    rows = [("Ynew", Ynew, n_eqns), ("RR", RR, n_species)]
    for name, t, width in rows:
        if t is None:
            continue
        tensor(name, t)
        if t.dtype != f64:
            raise ValueError(f"{name} must be float64")
        if t.dim() != 2 or t.shape[0] != n or t.shape[1] < width or t.stride(1) != 1:
            raise ValueError(f"{name} must be a row-contiguous [{n}][>= {width}] tensor")
    if Ynew is not None and (Ynew.shape[1] != Y0.shape[1] or Ynew.stride(0) != Y0.stride(0)):
        raise ValueError("Ynew must have Y0's shape and row stride")
    per_cell = [("deltaTChem", deltaTChem, f64, 1), ("rho", rho, f64, 1), ("deltaT_cell", deltaT_cell, f64, 1),
                ("mech_id", mech_id, i32, 1), ("status", status, i32, 1), ("counters", counters, i32, 2)]
    for name, t, dtype, k in per_cell:
        if t is None:
            continue
        tensor(name, t)
        if t.dtype != dtype:
            raise ValueError(f"{name} must be {dtype}")
        if t.numel() < k * n or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous tensor of at least {k * n} values")
    for name, t in [("Y0", Y0)] + [(nm, t) for nm, t, _ in rows] + [(nm, t) for nm, t, _, _ in per_cell]:
        if t is not None and (not t.is_cuda or t.device != Y0.device):
            raise ValueError(f"{name} must be on Y0's CUDA device")


def check_host_arrays(n, n_eqns, Y, deltaTChem, rho=None, deltaT=None):
    """Host arrays of computeRR / computeYNew: Y of n * n_eqns values, one
    deltaTChem (and rho, deltaT) per cell. Raises ValueError."""
    if Y.size != n * n_eqns:
        raise ValueError(f"Y must hold nCells * nEqns = {n * n_eqns} values, not {Y.size}")
    for name, a in (("deltaTChem", deltaTChem), ("rho", rho), ("deltaT", deltaT)):
        if a is not None and a.shape != (n,):
            raise ValueError(f"{name} must hold one value per cell ({n})")


class Solver:
    """gf_solver: one or more mechanisms + ODE inputs + Treact + launch form."""

    def __init__(self, mechs: Sequence[Mechanism], ode: OdeInputs, Treact: float = 0.0):
        self.lib = N.load()
        self.mechs = list(mechs)
        arr = (C.c_void_p * len(self.mechs))(*[m.handle.value for m in self.mechs])
        h = C.c_void_p()
        N.check(self.lib.gf_solver_create(arr, len(self.mechs), C.byref(ode.to_c()), float(Treact), C.byref(h)),
                "gf_solver_create")
        self.handle = h
        self.ode = ode
        self.Treact = Treact
        self.max_neq = max(m.n_eqns for m in self.mechs)
        self.max_species = max(m.n_species for m in self.mechs)

    def set_launch(self, kind=1, threads_per_cell=32, scratch_in_shared=1, cells_per_block=0, blocks_per_sm=0,
                   register_budget=0, lu_panel=0, specialize=0):
        cfg = N.GfLaunchConfig(kind, threads_per_cell, scratch_in_shared, cells_per_block, blocks_per_sm,
                               register_budget, lu_panel, specialize)
        N.check(self.lib.gf_solver_set_launch(self.handle, C.byref(cfg)), "gf_solver_set_launch")

    def workspace_doubles(self) -> int:
        """Per-cell workspace of the solve kernels, in doubles (gf_solver_info)."""
        ws = C.c_int()
        N.check(self.lib.gf_solver_info(self.handle, C.byref(ws), None, None), "gf_solver_info")
        return ws.value

    def get_launch(self) -> dict:
        cfg = N.GfLaunchConfig()
        N.check(self.lib.gf_solver_get_launch(self.handle, C.byref(cfg)), "gf_solver_get_launch")
        return cfg.as_dict()

    def solve(self, Y0, deltaT: float, deltaTChem, deltaTChemMax: float = np.inf, rho=None, deltaT_cell=None,
              mech_id=None, Ynew=None, RR=None, want_status=True, want_counters=True, want_stats=True,
              stream=None):
        """Device-tensor solve (gf_solve). Y0 [n][ld] float64 cuda; deltaTChem [n] is updated in place.
        Returns dict(Ynew, RR, deltaTChem, status, counters, stats)."""
        import torch
        n = int(Y0.shape[0])
        ld = int(Y0.stride(0))
        if Ynew is None:
            Ynew = torch.empty_like(Y0)
        if rho is not None and RR is None:
            RR = torch.empty((n, ld), dtype=torch.float64, device=Y0.device)
        status = torch.empty(n, dtype=torch.int32, device=Y0.device) if want_status else None
        counters = torch.empty((n, 2), dtype=torch.int32, device=Y0.device) if want_counters else None
        check_solve_tensors(n, self.max_neq, self.max_species, Y0, Ynew, RR, deltaTChem, rho, deltaT_cell, mech_id,
                            status, counters)
        st = N.GfStats()
        N.check(self.lib.gf_solve(self.handle, n, float(deltaT), _ptr(deltaT_cell), float(deltaTChemMax),
                                  _ptr(mech_id), _ptr(rho), _ptr(Y0), ld, _ptr(Ynew), _ptr(deltaTChem), _ptr(RR),
                                  int(RR.stride(0)) if RR is not None else 0, _ptr(status), _ptr(counters),
                                  C.byref(st) if want_stats else None, _stream_ptr(stream)), "gf_solve")
        return dict(Ynew=Ynew, RR=RR, deltaTChem=deltaTChem, status=status, counters=counters,
                    stats=dict(accepted=st.accepted_steps, attempts=st.attempts, failed=st.failed_cells,
                               min_delta_t=st.min_delta_t) if want_stats else None)

    def capture(self, Y0, deltaT: float, deltaTChem, deltaTChemMax: float = np.inf, rho=None, deltaT_cell=None,
                mech_id=None, Ynew=None, RR=None, status=None, counters=None) -> "SolveGraph":
        """The solve with these tensors captured as a CUDA graph (gf_solve_graph_create):
        every launch re-reads Y0 / deltaTChem and rewrites Ynew, RR, status, counters in place."""
        import torch
        n = int(Y0.shape[0])
        ld = int(Y0.stride(0))
        if Ynew is None:
            Ynew = torch.empty_like(Y0)
        if rho is not None and RR is None:
            RR = torch.empty((n, ld), dtype=torch.float64, device=Y0.device)
        check_solve_tensors(n, self.max_neq, self.max_species, Y0, Ynew, RR, deltaTChem, rho, deltaT_cell, mech_id,
                            status, counters)
        h = C.c_void_p()
        N.check(self.lib.gf_solve_graph_create(self.handle, n, float(deltaT), _ptr(deltaT_cell), float(deltaTChemMax),
                                               _ptr(mech_id), _ptr(rho), _ptr(Y0), ld, _ptr(Ynew), _ptr(deltaTChem),
                                               _ptr(RR), int(RR.stride(0)) if RR is not None else 0, _ptr(status),
                                               _ptr(counters), C.byref(h)), "gf_solve_graph_create")
        return SolveGraph(self, h, dict(Y0=Y0, deltaTChem=deltaTChem, rho=rho, deltaT_cell=deltaT_cell,
                                        mech_id=mech_id, Ynew=Ynew, RR=RR, status=status, counters=counters))

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gf_solver_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class SolveGraph:
    """A captured solve (gf_solve_graph): launch() enqueues it on a stream; the
    tensors it was captured with stay referenced here for its lifetime."""

    def __init__(self, solver: Solver, handle, tensors):
        self.solver = solver
        self.lib = solver.lib
        self.handle = handle
        self.tensors = tensors

    def __getitem__(self, name):
        return self.tensors[name]

    def launch(self, stream=None):
        N.check(self.lib.gf_solve_graph_launch(self.handle, _stream_ptr(stream)), "gf_solve_graph_launch")

    def set_delta_t(self, deltaT: float):
        N.check(self.lib.gf_solve_graph_set_delta_t(self.handle, float(deltaT)), "gf_solve_graph_set_delta_t")

    def stats(self) -> dict:
        """Totals of the last launch (after its stream has synchronized)."""
        st = N.GfStats()
        N.check(self.lib.gf_solve_graph_stats(self.handle, C.byref(st)), "gf_solve_graph_stats")
        return dict(accepted=st.accepted_steps, attempts=st.attempts, failed=st.failed_cells,
                    min_delta_t=st.min_delta_t)

    def close(self):
        if getattr(self, "handle", None):
            self.lib.gf_solve_graph_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class GpuKernelEvaluator:
    """Mirror of FoamGpu::GpuKernelEvaluator (gpuKernelEvaluator.H:18-85).

    GpuKernelEvaluator(nCells, nEqns, nSpecie, mechanism, odeInputs, Treact=0)
    where ``mechanism`` replaces the reference's (thermos, reactions) vectors.
    Inputs and outputs are host arrays, as in the reference."""

    def __init__(self, nCells: int, nEqns: int, nSpecie: int, mechanism, odeInputs: OdeInputs,
                 Treact: float = 0.0):
        if isinstance(mechanism, RawMechanism):
            mechanism = Mechanism(mechanism)
        if nEqns != nSpecie + 2 or mechanism.n_species != nSpecie:
            raise ValueError("nEqns must be nSpecie + 2 and match the mechanism")
        self.nCells, self.nEqns, self.nSpecie = nCells, nEqns, nSpecie
        self.mechanism = mechanism
        self.solver = Solver([mechanism], odeInputs, Treact)
        self.lib = self.solver.lib

    def computeYNew(self, deltaT: float, deltaTChemMax: float, deltaTChem, Y):
        """-> (Ynew [nCells*nEqns], deltaTChemNew [nCells]) (gpuKernelEvaluator.cu:35-63)."""
        dtc = np.ascontiguousarray(deltaTChem, dtype=np.float64)
        Yh = np.ascontiguousarray(Y, dtype=np.float64).reshape(-1)
        n = dtc.shape[0]
        check_host_arrays(n, self.nEqns, Yh, dtc)
        Ynew = np.empty(n * self.nEqns)
        dtn = np.empty(n)
        N.check(self.lib.gf_compute_ynew(self.solver.handle, n, float(deltaT), float(deltaTChemMax),
                                         dtc.ctypes.data, Yh.ctypes.data, Ynew.ctypes.data, dtn.ctypes.data),
                "gf_compute_ynew")
        return Ynew, dtn

    def computeRR(self, deltaT: float, deltaTChemMax: float, rho, deltaTChem, Y):
        """-> (RR [nCells*nSpecie], deltaTChemNew [nCells] clamped, minDeltaT)
        (gpuKernelEvaluator.cu:65-97)."""
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        dtc = np.ascontiguousarray(deltaTChem, dtype=np.float64)
        Yh = np.ascontiguousarray(Y, dtype=np.float64).reshape(-1)
        n = rho.shape[0]
        check_host_arrays(n, self.nEqns, Yh, dtc, rho)
        RR = np.empty(n * self.nSpecie)
        dtn = np.empty(n)
        mn = C.c_double()
        N.check(self.lib.gf_compute_rr(self.solver.handle, n, float(deltaT), float(deltaTChemMax), rho.ctypes.data,
                                       dtc.ctypes.data, Yh.ctypes.data, RR.ctypes.data, dtn.ctypes.data,
                                       C.byref(mn)), "gf_compute_rr")
        return RR, dtn, mn.value

    def computeRRLocal(self, deltaT, deltaTChemMax: float, rho, deltaTChem, Y):
        """computeRR with a flow time step per cell, deltaT [nCells] (local time
        stepping; the reference's solve(const scalarField&) throws,
        gpuChemistryModel.C:328-333) -> (RR, deltaTChemNew clamped, minDeltaT)."""
        dT = np.ascontiguousarray(deltaT, dtype=np.float64)
        rho = np.ascontiguousarray(rho, dtype=np.float64)
        dtc = np.ascontiguousarray(deltaTChem, dtype=np.float64)
        Yh = np.ascontiguousarray(Y, dtype=np.float64).reshape(-1)
        n = rho.shape[0]
        check_host_arrays(n, self.nEqns, Yh, dtc, rho, dT)
        RR = np.empty(n * self.nSpecie)
        dtn = np.empty(n)
        mn = C.c_double()
        N.check(self.lib.gf_compute_rr_lts(self.solver.handle, n, dT.ctypes.data, float(deltaTChemMax),
                                           rho.ctypes.data, dtc.ctypes.data, Yh.ctypes.data, RR.ctypes.data,
                                           dtn.ctypes.data, C.byref(mn)), "gf_compute_rr_lts")
        return RR, dtn, mn.value


def solve_noalloc(mech: Mechanism, ode: OdeInputs, Y0, deltaT: float, deltaTChem, Ynew, Treact: float = 0.0,
                  deltaTChemMax: float = np.inf, rho=None, RR=None, status=None, counters=None, stats=True,
                  stream=None):
    """gf_solve_noalloc: the solve for callers that cannot allocate device
    memory. Every array is the caller's (cuda tensors); deltaTChem is updated
    in place and Ynew/RR/status/counters are written. The library's static
    device scratch is shared by all calls, so calls must not overlap on a GPU.
    Returns the statistics dict when stats=True (this waits for the stream,
    and is refused on a stream that is being captured)."""
    lib = N.load()
    n = int(Y0.shape[0])
    check_solve_tensors(n, mech.n_eqns, mech.n_species, Y0, Ynew, RR, deltaTChem, rho, None, None, status, counters)
    st = N.GfStats()
    N.check(lib.gf_solve_noalloc(mech.handle, C.byref(ode.to_c()), float(Treact), n, float(deltaT), None,
                                 float(deltaTChemMax), _ptr(rho), _ptr(Y0), int(Y0.stride(0)), _ptr(Ynew),
                                 _ptr(deltaTChem), _ptr(RR), int(RR.stride(0)) if RR is not None else 0,
                                 _ptr(status), _ptr(counters), C.byref(st) if stats else None, _stream_ptr(stream)),
            "gf_solve_noalloc")
    if stats:
        return dict(accepted=st.accepted_steps, attempts=st.attempts, failed=st.failed_cells,
                    min_delta_t=st.min_delta_t)
    return None


# ---- parity entry points ----------------------------------------------------

def rates(mech: Mechanism, y):
    """derivatives(y) for states y [n][nEqns] (host or device) -> cuda tensor."""
    import torch
    yd = _dev(y, torch.float64)
    out = torch.empty_like(yd)
    N.check(mech.lib.gf_rates(mech.handle, yd.shape[0], _ptr(yd), _ptr(out), _stream_ptr()), "gf_rates")
    return out


def jacobian(mech: Mechanism, y):
    import torch
    yd = _dev(y, torch.float64)
    n = yd.shape[1]
    dfdx = torch.empty_like(yd)
    J = torch.empty((yd.shape[0], n, n), dtype=torch.float64, device="cuda")
    N.check(mech.lib.gf_jacobian(mech.handle, yd.shape[0], _ptr(yd), _ptr(dfdx), _ptr(J), _stream_ptr()),
            "gf_jacobian")
    return dfdx, J


def lu_decompose(A):
    import torch
    lib = N.load()
    Ad = _dev(A, torch.float64).clone()
    k, m, _ = Ad.shape
    piv = torch.empty((k, m), dtype=torch.int32, device="cuda")
    N.check(lib.gf_lu_decompose(k, m, _ptr(Ad), _ptr(piv), _stream_ptr()), "gf_lu_decompose")
    return Ad, piv


def lu_backsubstitute(LU, piv, b):
    import torch
    lib = N.load()
    bd = _dev(b, torch.float64).clone()
    k, m = bd.shape
    N.check(lib.gf_lu_backsubstitute(k, m, _ptr(_dev(LU, torch.float64)), _ptr(_dev(piv, torch.int32)), _ptr(bd),
                                     _stream_ptr()), "gf_lu_backsubstitute")
    return bd


def lu_factor_solve(A, b, threads_per_matrix: int, exact: bool = False):
    """LUDecompose + LUBacksubstitute as the solve kernels run them with
    threads_per_matrix threads per matrix (gf_lu_factor_solve): A [k][m][m],
    b [k][n_rhs][m] (host or device) -> (factors, pivots, solutions), cuda tensors.
    exact=True rounds each elimination update twice (no FMA contraction)."""
    import torch
    lib = N.load()
    Ad = _dev(A, torch.float64).clone()
    bd = _dev(b, torch.float64).clone()
    k, m, _ = Ad.shape
    if bd.dim() != 3 or bd.shape[0] != k or bd.shape[2] != m:
        raise ValueError("b must be [n_mats][n_rhs][m]")
    piv = torch.empty((k, m), dtype=torch.int32, device="cuda")
    N.check(lib.gf_lu_factor_solve(k, m, _ptr(Ad), _ptr(piv), _ptr(bd), int(bd.shape[1]), int(threads_per_matrix),
                                   int(bool(exact)), _stream_ptr()), "gf_lu_factor_solve")
    return Ad, piv, bd


# ---- the plugin's per-cell side paths (gpuChemistryModel.C:145-450), on the GPU

def cell_rates(mech: Mechanism, rho, y, want_RR: bool = True, want_tc: bool = True):
    """calculate() and tc() at c = rho Y / W: (RR [n][nS] or None, tc [n] or None), cuda tensors."""
    import torch
    yd = _dev(y, torch.float64)
    rd = _dev(rho, torch.float64)
    n = yd.shape[0]
    RR = torch.empty((n, mech.n_species), dtype=torch.float64, device="cuda") if want_RR else None
    tc = torch.empty(n, dtype=torch.float64, device="cuda") if want_tc else None
    N.check(mech.lib.gf_cell_rates(mech.handle, n, _ptr(rd), _ptr(yd), yd.shape[1], _ptr(RR), mech.n_species,
                                   _ptr(tc), _stream_ptr()), "gf_cell_rates")
    return RR, tc


def reaction_rates(mech: Mechanism, reaction: int, rho, y):
    """reactionRR(r) and specieReactionRR(r): (omega [n], RR [n][nS]), cuda tensors."""
    import torch
    yd = _dev(y, torch.float64)
    rd = _dev(rho, torch.float64)
    n = yd.shape[0]
    om = torch.empty(n, dtype=torch.float64, device="cuda")
    RR = torch.empty((n, mech.n_species), dtype=torch.float64, device="cuda")
    N.check(mech.lib.gf_reaction_rates(mech.handle, n, int(reaction), _ptr(rd), _ptr(yd), yd.shape[1], _ptr(om),
                                       _ptr(RR), mech.n_species, _stream_ptr()), "gf_reaction_rates")
    return om, RR


def qdot(mech: Mechanism, RR):
    """Qdot() from species mass rates RR [n][nS] (host or device) -> cuda tensor [n]."""
    import torch
    rd = _dev(RR, torch.float64)
    out = torch.empty(rd.shape[0], dtype=torch.float64, device="cuda")
    N.check(mech.lib.gf_qdot(mech.handle, rd.shape[0], _ptr(rd), rd.shape[1], _ptr(out), _stream_ptr()), "gf_qdot")
    return out


# ---- the plugin's field gather and rate scatter (gpuChemistryModel.C:33-53, :351-356), on the GPU

def gather_states(Y_fields, T, p, ld: Optional[int] = None):
    """Per-species fields (a sequence of nS cuda tensors of n cells) plus T and p ->
    the cell-major states [n][ld] (ld >= nS + 2) that gf_solve takes."""
    import torch
    nS = len(Y_fields)
    n = int(T.shape[0])
    ld = ld or nS + 2
    for f in list(Y_fields) + [T, p]:
        if f.dtype != torch.float64 or not f.is_cuda or not f.is_contiguous() or f.numel() < n:
            raise ValueError("fields must be contiguous float64 cuda tensors of at least n cells")
    y = torch.zeros((n, ld), dtype=torch.float64, device="cuda")
    ptrs = (C.c_void_p * max(nS, 1))(*[f.data_ptr() for f in Y_fields])
    lib = N.load()
    N.check(lib.gf_gather_states(n, nS, ptrs, _ptr(T), _ptr(p), _ptr(y), ld, _stream_ptr()), "gf_gather_states")
    return y


def scatter_rates(RR, RR_fields):
    """Cell-major rates RR [n][>= nS] -> the per-species fields RR_fields (nS cuda tensors of n)."""
    import torch
    nS = len(RR_fields)
    n = int(RR.shape[0])
    if RR.dim() != 2 or RR.stride(1) != 1 or RR.shape[1] < nS or RR.dtype != torch.float64 or not RR.is_cuda:
        raise ValueError("RR must be a row-contiguous float64 cuda tensor [n][>= nS]")
    for f in RR_fields:
        if f.dtype != torch.float64 or not f.is_cuda or not f.is_contiguous() or f.numel() < n:
            raise ValueError("RR fields must be contiguous float64 cuda tensors of at least n cells")
    ptrs = (C.c_void_p * max(nS, 1))(*[f.data_ptr() for f in RR_fields])
    lib = N.load()
    N.check(lib.gf_scatter_rates(n, nS, _ptr(RR), int(RR.stride(0)), ptrs, _stream_ptr()), "gf_scatter_rates")
