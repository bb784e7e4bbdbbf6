"""Discrete adjoint of the chemistry integration, as a torch.autograd.Function.

The forward pass integrates every cell over one flow step with the CUDA path
(gf_solve_record) and records its accepted steps; the backward pass is the
hand-written reverse sweep gf_adjoint: every recorded step is recomputed from
its start state and differentiated exactly as the Rosenbrock method computes
it (step sizes frozen). Gradients come out w.r.t. the initial states (Y, T)
and, per reaction, w.r.t. (ln|A|, beta, Ta) of its rate constant k (k0 for
fall-off reactions), Ta = Ea / R.

    sol = AdjointSolver(raw_mechanism, OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4))
    theta = sol.parameters()                       # [nR, 3] float64 (ln|A|, beta, Ta)
    Y1 = ChemistryStep.apply(Y0, theta, sol, 1e-4, 1e-7)
    loss = (w * Y1).sum(); loss.backward()         # Y0.grad, theta.grad

There is no counterpart in the reference (gpuFoam integrates forward only).
"""
from __future__ import annotations

import ctypes as C
import copy
import math
from typing import Optional

import numpy as np
import torch

from . import _native as N
from . import evaluator as E
from .mechanism import RATE_ARRHENIUS, RawMechanism

R_UNIVERSAL = 8.314462618  # J/mol/K: dL/dEa [J/mol] = dL/dTa / R_UNIVERSAL


def parameters_of(raw: RawMechanism) -> np.ndarray:
    """[nR, 3] (ln|A|, beta, Ta) of each reaction's k (k0 for fall-off)."""
    out = np.zeros((raw.n_reactions, 3))
    for r, x in enumerate(raw.reactions):
        out[r] = (math.log(abs(x.A)) if x.A != 0 else 0.0, x.beta, x.Ta)
    return out


def with_parameters(raw: RawMechanism, theta: np.ndarray) -> RawMechanism:
    """A copy of the mechanism whose k (k0) Arrhenius parameters are theta
    (the sign of each A is kept)."""
    out = copy.deepcopy(raw)
    for r, x in enumerate(out.reactions):
        sign = -1.0 if x.A < 0 else 1.0
        x.A = sign * math.exp(float(theta[r, 0]))
        x.beta = float(theta[r, 1])
        x.Ta = float(theta[r, 2])
    return out


class AdjointSolver:
    """Forward with a recorded trajectory, then the adjoint sweep (gf_solve_record
    / gf_adjoint). One mechanism; traj_cap bounds the accepted steps per cell."""

    def __init__(self, raw: RawMechanism, ode: E.OdeInputs, traj_cap: int = 4096, launch: Optional[dict] = None):
        self.raw = raw
        self.ode = ode
        self.traj_cap = int(traj_cap)
        self.launch = launch
        self._theta_key = None
        self._set_mechanism(raw)

    def _set_mechanism(self, raw: RawMechanism):
        self.mech = E.Mechanism(raw)
        self.solver = E.Solver([self.mech], self.ode)
        if self.launch:
            self.solver.set_launch(**self.launch)

    def parameters(self) -> np.ndarray:
        return parameters_of(self.raw)

    def set_parameters(self, theta: np.ndarray):
        key = np.asarray(theta, dtype=np.float64).tobytes()
        if key != self._theta_key:
            self._set_mechanism(with_parameters(self.raw, np.asarray(theta)))
            self._theta_key = key

    def forward(self, Y0, deltaT: float, deltaTChem):
        """Y0 [n][nS+2] float64 cuda; deltaTChem [n] (updated in place).
        Returns Ynew and keeps the recording for backward()."""
        import torch
        n, ld = Y0.shape
        if deltaTChem.numel() != n or deltaTChem.dtype != torch.float64 or not deltaTChem.is_contiguous():
            raise ValueError("deltaTChem must be a contiguous float64 tensor of one value per cell")
        lib = N.load()
        Y0 = Y0.contiguous()
        Ynew = torch.empty_like(Y0)
        status = torch.zeros(n, dtype=torch.int32, device=Y0.device)
        counters = torch.zeros((n, 2), dtype=torch.int32, device=Y0.device)
        m = self.raw.n_species + 1
        traj = torch.empty((n, self.traj_cap, m + 1), dtype=torch.float64, device=Y0.device)
        stream = torch.cuda.current_stream().cuda_stream
        N.check(lib.gf_solve_record(self.solver.handle, n, float(deltaT), Y0.data_ptr(), ld, Ynew.data_ptr(),
                                    deltaTChem.data_ptr(), status.data_ptr(), counters.data_ptr(), traj.data_ptr(),
                                    self.traj_cap, stream), "gf_solve_record")
        self._rec = dict(Y0=Y0, Ynew=Ynew, status=status, counters=counters, traj=traj, ld=ld)
        return Ynew, status, counters

    def backward(self, Ybar):
        """Gradients w.r.t. Y0 [n][ld] and, summed over cells, theta [nR, 3];
        also the per-cell status of the sweep."""
        import torch
        rec = self._rec
        n, ld = rec["Y0"].shape
        lib = N.load()
        if tuple(Ybar.shape) != (n, ld):
            raise ValueError("Ybar must have the shape of the recorded states")
        Ybar = Ybar.contiguous().to(torch.float64)
        Y0bar = torch.zeros_like(rec["Y0"])
        thb = torch.zeros((n, self.raw.n_reactions * 3), dtype=torch.float64, device=Ybar.device)
        status = torch.zeros(n, dtype=torch.int32, device=Ybar.device)
        stream = torch.cuda.current_stream().cuda_stream
        N.check(lib.gf_adjoint(self.solver.handle, n, rec["traj"].data_ptr(), self.traj_cap,
                               rec["counters"].data_ptr(), rec["status"].data_ptr(), rec["Y0"].data_ptr(),
                               rec["Ynew"].data_ptr(), Ybar.data_ptr(), ld, Y0bar.data_ptr(), thb.data_ptr(),
                               status.data_ptr(), stream), "gf_adjoint")
        return Y0bar, thb.sum(dim=0).reshape(self.raw.n_reactions, 3), status


class ChemistryStep(torch.autograd.Function):
    """Y1 = integrate(Y0; theta) over deltaT, differentiable w.r.t. Y0 (species
    and T; p has no gradient) and theta [nR, 3] (ln|A|, beta, Ta)."""

    @staticmethod
    def forward(ctx, Y0, theta, solver: AdjointSolver, deltaT: float, deltaTChem0: float):
        solver.set_parameters(theta.detach().cpu().numpy())
        dtc = torch.full((Y0.shape[0],), float(deltaTChem0), dtype=torch.float64, device=Y0.device)
        Y1, status, counters = solver.forward(Y0.detach(), deltaT, dtc)
        ctx.solver = solver
        ctx.theta_device = theta.device
        return Y1

    @staticmethod
    def backward(ctx, Ybar):
        Y0bar, thb, status = ctx.solver.backward(Ybar)
        return Y0bar, thb.to(ctx.theta_device), None, None, None
