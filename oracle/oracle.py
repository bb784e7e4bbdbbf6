"""TEST INFRASTRUCTURE ONLY — ctypes access to the two CPU oracles.

* ``Oracle("port")``: this project's plain-C restatement (oracle/gf_oracle.c,
  built into oracle/liboracle.so).
* ``Oracle("reference")``: the gpuFoam reference's own FP64 code compiled in
  place (oracle/ref_driver.cpp, built into oracle/_ref/libgf_ref.so).

Both take the same flat raw mechanism (see oracle/gf_oracle.h) and expose the
same functions, so a test can run one against the other. Only tests/,
__graft_entry__.smoke() and bench.py's CPU-baseline legs may import this
module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# the gpuFoam source tree: GPUFOAM_REFERENCE, else a directory named reference
# beside this repository (the same rule as oracle/Makefile)
REFERENCE_ROOT = os.environ.get("GPUFOAM_REFERENCE",
                                os.path.normpath(os.path.join(HERE, "..", "..", "reference")))
PORT_LIB = os.path.join(HERE, "liboracle.so")
REF_LIB = os.path.join(HERE, "_ref", "libgf_ref.so")

_dp = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")
_ip = np.ctypeslib.ndpointer(dtype=np.int32, flags="C_CONTIGUOUS")


class OdeInputs(C.Structure):
    """Same layout as gf_ode_inputs / orc_ode_inputs."""
    _fields_ = [("solver", C.c_int), ("absTol", C.c_double), ("relTol", C.c_double),
                ("maxSteps", C.c_int), ("safeScale", C.c_double), ("alphaInc", C.c_double),
                ("alphaDec", C.c_double), ("minScale", C.c_double), ("maxScale", C.c_double)]


def ode_inputs(solver=34, absTol=1e-8, relTol=1e-4, maxSteps=10000, safeScale=0.9,
               alphaInc=0.2, alphaDec=0.25, minScale=0.2, maxScale=10.0) -> OdeInputs:
    """Defaults of read_gpuODESolverInputs (readGpuOdeInputs.H:8-26) except the
    tolerances, which default to the benchmark's absTol 1e-8, relTol 1e-4."""
    return OdeInputs(int(solver), absTol, relTol, int(maxSteps), safeScale, alphaInc, alphaDec,
                     minScale, maxScale)


def build(force: bool = False) -> None:
    """Build the oracles (make -C oracle)."""
    if force or not os.path.exists(PORT_LIB) or (
            os.path.isdir(os.path.join(REFERENCE_ROOT, "gpu_chemistry")) and not os.path.exists(REF_LIB)):
        subprocess.run(["make", "-s", "-C", HERE], check=True)


def flatten(mech):
    """Flat raw arrays of a gpufoam_b200.mechanism.RawMechanism."""
    nS, nR = mech.n_species, mech.n_reactions
    rint = np.zeros((max(nR, 1), 24), dtype=np.int32)
    rdbl = np.zeros((max(nR, 1), 50), dtype=np.float64)
    eff = np.zeros((max(nR, 1), nS), dtype=np.float64)
    for r, rx in enumerate(mech.reactions):
        rint[r, 0] = rx.rate_type
        rint[r, 1] = int(rx.irreversible)
        rint[r, 2] = len(rx.lhs)
        rint[r, 3] = len(rx.rhs)
        for i, (idx, st, ex) in enumerate(rx.lhs):
            rint[r, 4 + i] = idx
            rdbl[r, i] = st
            rdbl[r, 10 + i] = ex
        for i, (idx, st, ex) in enumerate(rx.rhs):
            rint[r, 14 + i] = idx
            rdbl[r, 20 + i] = st
            rdbl[r, 30 + i] = ex
        rdbl[r, 40:43] = (rx.A, rx.beta, rx.Ta)
        rdbl[r, 43:46] = (rx.Ainf, rx.betainf, rx.Tainf)
        rdbl[r, 46:50] = rx.troe
        if rx.efficiencies is not None:
            eff[r] = rx.efficiencies
    return dict(nS=nS, W=np.ascontiguousarray(mech.W, dtype=np.float64),
                Tlow=np.ascontiguousarray(mech.Tlow, dtype=np.float64),
                Thigh=np.ascontiguousarray(mech.Thigh, dtype=np.float64),
                Tcommon=np.ascontiguousarray(mech.Tcommon, dtype=np.float64),
                high=np.ascontiguousarray(mech.high_raw, dtype=np.float64),
                low=np.ascontiguousarray(mech.low_raw, dtype=np.float64),
                nR=nR, rint=rint, rdbl=rdbl, eff=eff,
                rxnTlow=float(mech.rxn_Tlow), rxnThigh=float(mech.rxn_Thigh))


class Oracle:
    """One CPU oracle bound to one mechanism."""

    def __init__(self, mech, kind: str = "port"):
        build()
        path = PORT_LIB if kind == "port" else REF_LIB
        if not os.path.exists(path):
            raise FileNotFoundError(f"oracle library missing: {path}")
        self.kind = kind
        self.lib = C.CDLL(path)
        p = "orc_" if kind == "port" else "ref_"
        self._p = p
        L = self.lib
        f = getattr(L, p + "mech_create")
        f.restype = C.c_void_p
        f.argtypes = [C.c_int, _dp, _dp, _dp, _dp, _dp, _dp, C.c_int, _ip, _dp, _dp, C.c_double, C.c_double]
        getattr(L, p + "mech_destroy").argtypes = [C.c_void_p]
        getattr(L, p + "mech_tables").argtypes = [C.c_void_p, _dp, _dp, _ip]
        getattr(L, p + "thermo_eval").argtypes = [C.c_void_p, C.c_double, C.c_double, _dp]
        getattr(L, p + "reaction_eval").argtypes = [C.c_void_p, _dp, _dp]
        getattr(L, p + "derivatives").argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        getattr(L, p + "jacobian").argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
        getattr(L, p + "lu").argtypes = [C.c_int, C.c_int, _dp, _ip, _dp]
        getattr(L, p + "attempt").argtypes = [C.c_void_p, C.POINTER(OdeInputs), C.c_int, _dp, _dp, _dp, _dp, _dp]
        if kind == "port":
            L.orc_cells.argtypes = [C.c_void_p, C.POINTER(OdeInputs), C.c_double, C.c_int, C.c_double,
                                    C.c_void_p, _dp, _dp, _ip, _ip, C.c_int]
        else:
            L.ref_cells_counted.argtypes = [C.c_void_p, C.POINTER(OdeInputs), C.c_double, C.c_int,
                                            C.c_double, C.c_void_p, _dp, _dp, _ip, C.c_int]
            L.ref_cells.argtypes = [C.c_void_p, C.POINTER(OdeInputs), C.c_double, C.c_int, C.c_double,
                                    _dp, _dp, C.c_int]
        f = getattr(L, p + "compute_rr_host")
        f.restype = C.c_double
        f.argtypes = [C.c_int, C.c_int, C.c_double, C.c_double, _dp, _dp, _dp, _dp, _dp]
        getattr(L, p + "constants").argtypes = [_dp]
        getattr(L, p + "cell_fields").argtypes = [C.c_void_p, C.c_int, _dp, _dp, C.c_void_p, C.c_void_p]
        getattr(L, p + "reaction_fields").argtypes = [C.c_void_p, C.c_int, C.c_int, _dp, _dp, C.c_void_p,
                                                      C.c_void_p]
        getattr(L, p + "qdot").argtypes = [C.c_void_p, C.c_int, _dp, _dp]
        if kind == "port":
            L.orc_rate_parts.argtypes = [C.c_void_p, C.c_int, _dp, _dp, _dp]
            L.orc_replay.argtypes = [C.c_void_p, C.POINTER(OdeInputs), C.c_int, _dp, _dp]
        self.mech = mech
        fl = flatten(mech)
        self._flat = fl
        self.nS = fl["nS"]
        self.nR = fl["nR"]
        self.h = f = getattr(L, p + "mech_create")(
            fl["nS"], fl["W"], fl["Tlow"], fl["Thigh"], fl["Tcommon"], fl["high"], fl["low"],
            fl["nR"], fl["rint"], fl["rdbl"], fl["eff"], fl["rxnTlow"], fl["rxnThigh"])
        if not self.h:
            raise ValueError("oracle rejected the mechanism (mass imbalance)")

    def close(self):
        if getattr(self, "h", None):
            getattr(self.lib, self._p + "mech_destroy")(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- tables and pointwise functions
    def tables(self):
        sp = np.zeros((self.nS, 19))
        rx = np.zeros((max(self.nR, 1), 19))
        ie = np.zeros((max(self.nR, 1), 20), dtype=np.int32)
        getattr(self.lib, self._p + "mech_tables")(self.h, sp, rx, ie)
        return sp, rx[: self.nR], ie[: self.nR]

    def thermo_eval(self, p: float, T: float):
        out = np.zeros((self.nS, 8))
        getattr(self.lib, self._p + "thermo_eval")(self.h, p, T, out)
        return out

    def reaction_eval(self, y):
        out = np.zeros((max(self.nR, 1), 6))
        getattr(self.lib, self._p + "reaction_eval")(self.h, np.ascontiguousarray(y, dtype=np.float64), out)
        return out[: self.nR]

    def derivatives(self, y):
        y = np.ascontiguousarray(np.atleast_2d(y), dtype=np.float64)
        out = np.zeros_like(y)
        getattr(self.lib, self._p + "derivatives")(self.h, y.shape[0], y, out)
        return out

    def jacobian(self, y):
        y = np.ascontiguousarray(np.atleast_2d(y), dtype=np.float64)
        n = y.shape[1]
        dfdx = np.zeros_like(y)
        J = np.zeros((y.shape[0], n, n))
        getattr(self.lib, self._p + "jacobian")(self.h, y.shape[0], y, dfdx, J)
        return dfdx, J

    def attempt(self, inputs: OdeInputs, y0, dydx0, dx):
        y0 = np.ascontiguousarray(np.atleast_2d(y0), dtype=np.float64)
        dydx0 = np.ascontiguousarray(np.atleast_2d(dydx0), dtype=np.float64)
        dx = np.ascontiguousarray(np.broadcast_to(np.asarray(dx, dtype=np.float64), (y0.shape[0],)))
        y = np.zeros_like(y0)
        err = np.zeros(y0.shape[0])
        getattr(self.lib, self._p + "attempt")(self.h, C.byref(inputs), y0.shape[0], y0, dydx0, dx, y, err)
        return y, err

    def cells(self, inputs: OdeInputs, Y, deltaT, deltaTChem, Treact: float = 0.0,
              deltaT_cell: Optional[np.ndarray] = None, nthreads: int = 0):
        """singleCellSolver over cells. Returns (Ynew, deltaTChemNew, counts[n,2], status or None)."""
        Y = np.array(Y, dtype=np.float64, order="C", copy=True)
        n = Y.shape[0]
        dtc = np.array(np.broadcast_to(np.asarray(deltaTChem, dtype=np.float64), (n,)), order="C", copy=True)
        counts = np.zeros((n, 2), dtype=np.int32)
        dtp = None
        if deltaT_cell is not None:
            dtcell = np.ascontiguousarray(deltaT_cell, dtype=np.float64)
            dtp = dtcell.ctypes.data_as(C.c_void_p)
        if self.kind == "port":
            status = np.zeros(n, dtype=np.int32)
            self.lib.orc_cells(self.h, C.byref(inputs), Treact, n, float(deltaT), dtp, Y, dtc, counts,
                               status, nthreads)
            return Y, dtc, counts, status
        self.lib.ref_cells_counted(self.h, C.byref(inputs), Treact, n, float(deltaT), dtp, Y, dtc, counts,
                                   nthreads)
        return Y, dtc, counts, None

    def cells_uncounted(self, inputs: OdeInputs, Y, deltaT, deltaTChem, Treact=0.0, nthreads: int = 0):
        """The reference's own singleCellSolver functor (reference oracle only)."""
        assert self.kind == "reference"
        Y = np.array(Y, dtype=np.float64, order="C", copy=True)
        n = Y.shape[0]
        dtc = np.array(np.broadcast_to(np.asarray(deltaTChem, dtype=np.float64), (n,)), order="C", copy=True)
        self.lib.ref_cells(self.h, C.byref(inputs), Treact, n, float(deltaT), Y, dtc, nthreads)
        return Y, dtc

    def replay(self, inputs: OdeInputs, y0, steps):
        """The frozen-step map (port only): the recorded step sizes replayed from
        y0, one attempt each, then max(0, Y)."""
        y = np.array(y0, dtype=np.float64, order="C", copy=True)
        st = np.ascontiguousarray(steps, dtype=np.float64)
        self.lib.orc_replay(self.h, C.byref(inputs), int(st.size), st, y)
        return y

    def compute_rr_host(self, deltaT, deltaTChemMax, rho, Y0, Ynew, deltaTChemNew):
        n = Y0.shape[0]
        RR = np.zeros((n, self.nS))
        dtc = np.array(deltaTChemNew, dtype=np.float64, copy=True)
        mn = getattr(self.lib, self._p + "compute_rr_host")(
            n, self.nS, deltaT, deltaTChemMax, np.ascontiguousarray(rho, dtype=np.float64),
            np.ascontiguousarray(Y0), np.ascontiguousarray(Ynew), dtc, RR)
        return RR, dtc, mn

    # ---- the plugin's per-cell side paths (gpuChemistryModel.C:145-450)
    def cell_fields(self, rho, y):
        """calculate() and tc(): (RR [n][nS], tc [n]) at c = rho Y / W."""
        y = np.ascontiguousarray(np.atleast_2d(y), dtype=np.float64)
        n = y.shape[0]
        RR = np.zeros((n, self.nS))
        tc = np.zeros(n)
        getattr(self.lib, self._p + "cell_fields")(self.h, n, np.ascontiguousarray(rho, dtype=np.float64), y,
                                                   RR.ctypes.data_as(C.c_void_p), tc.ctypes.data_as(C.c_void_p))
        return RR, tc

    def reaction_fields(self, reaction, rho, y):
        """reactionRR(r) and specieReactionRR(r): (omega [n], RR [n][nS])."""
        y = np.ascontiguousarray(np.atleast_2d(y), dtype=np.float64)
        n = y.shape[0]
        om = np.zeros(n)
        RR = np.zeros((n, self.nS))
        getattr(self.lib, self._p + "reaction_fields")(self.h, n, int(reaction),
                                                       np.ascontiguousarray(rho, dtype=np.float64), y,
                                                       om.ctypes.data_as(C.c_void_p), RR.ctypes.data_as(C.c_void_p))
        return om, RR

    def rate_parts(self, rho, y):
        """(kf Cf, kr Cr) [n][nR][2] at c = rho Y / W (port only; tolerance scales)."""
        y = np.ascontiguousarray(np.atleast_2d(y), dtype=np.float64)
        out = np.zeros((y.shape[0], max(self.nR, 1), 2))
        self.lib.orc_rate_parts(self.h, y.shape[0], np.ascontiguousarray(rho, dtype=np.float64), y, out)
        return out[:, : self.nR]

    def qdot(self, RR):
        """Qdot() from species mass rates RR [n][nS]."""
        RR = np.ascontiguousarray(np.atleast_2d(RR), dtype=np.float64)
        out = np.zeros(RR.shape[0])
        getattr(self.lib, self._p + "qdot")(self.h, RR.shape[0], RR, out)
        return out

    def constants(self):
        out = np.zeros(9)
        getattr(self.lib, self._p + "constants")(out)
        return out


def lu(kind: str, A, b):
    """LUDecompose + LUBacksubstitute of matrices A [k][m][m] and b [k][m]."""
    build()
    lib = C.CDLL(PORT_LIB if kind == "port" else REF_LIB)
    f = lib.orc_lu if kind == "port" else lib.ref_lu
    f.argtypes = [C.c_int, C.c_int, _dp, _ip, _dp]
    A = np.array(A, dtype=np.float64, order="C", copy=True)
    b = np.array(b, dtype=np.float64, order="C", copy=True)
    k, m = b.shape
    piv = np.zeros((k, m), dtype=np.int32)
    f(m, k, A, piv, b)
    return A, piv, b
