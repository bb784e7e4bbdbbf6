"""Algorithmic FLOP count of the per-cell chemistry integration.

This is the figure the roofline's `achieved` uses; it is a fixed model of the
work the algorithm requires, not a count of what the kernel executes. Per cell
and flow step, with n = nEqns = nS + 2, A = attempted Rosenbrock steps
(accepted + rejected) and S = accepted steps (both counted by the kernel):

    FLOP   = A * F_att(s, d) + S * F_rhs
    F_att  = F_jac + n^2 + F_LU + s * F_bs + d * F_rhs + 10 n
    F_LU   = 2 n^3 / 3
    F_bs   = 2 n^2
    F_rhs  = 30 nS + sum_r c_rhs(r)
    c_rhs  = 20 t_r + 4 (nl + nr) + [2 nS if third-body or fall-off]
    F_jac  = 40 nS + sum_r [c_rhs(r) + 2 (nl + nr)^2 + (4 (nl + nr) nS if third-body/fall-off)]
             + 15 nS^2 + 2 nS^2

t_r counts the transcendental calls (exp/log/log10/pow) on the reaction's path,
20 FLOP each: 2 per Arrhenius evaluation (pow, exp; a fall-off rate has two:
k0 and kInf), +3 for Kc when reversible, +6 for the Troe F. (s, d) = stages
with a linear solve and extra RHS evaluations: (2, 1) Rosenbrock12,
(3, 1) Rosenbrock23, (4, 2) Rosenbrock34 (gpuRosenbrock12/23/34.H).
"""
from __future__ import annotations

from .mechanism import RATE_ARRHENIUS, RATE_LINDEMANN, RATE_THIRD_BODY, RATE_TROE, RawMechanism

STAGES = {12: (2, 1), 23: (3, 1), 34: (4, 2)}


def per_reaction_rhs(mech: RawMechanism):
    nS = mech.n_species
    out = []
    for r in mech.reactions:
        t = 4 if r.rate_type in (RATE_LINDEMANN, RATE_TROE) else 2
        if not r.irreversible:
            t += 3
        if r.rate_type == RATE_TROE:
            t += 6
        w = len(r.lhs) + len(r.rhs)
        tb = r.rate_type != RATE_ARRHENIUS
        out.append((20 * t + 4 * w + (2 * nS if tb else 0), w, tb))
    return out


def model(mech: RawMechanism, solver: int):
    """(F_att, F_rhs) in FLOP for the mechanism and Rosenbrock variant."""
    nS = mech.n_species
    n = nS + 2
    s, d = STAGES[solver]
    rx = per_reaction_rhs(mech)
    F_rhs = 30 * nS + sum(c for c, _, _ in rx)
    F_jac = 40 * nS + sum(c + 2 * w * w + (4 * w * nS if tb else 0) for c, w, tb in rx) + 15 * nS * nS + 2 * nS * nS
    F_LU = 2.0 * n ** 3 / 3.0
    F_bs = 2.0 * n * n
    F_att = F_jac + n * n + F_LU + s * F_bs + d * F_rhs + 10 * n
    return float(F_att), float(F_rhs)


def total(mech: RawMechanism, solver: int, attempts: int, accepted: int) -> float:
    F_att, F_rhs = model(mech, solver)
    return attempts * F_att + accepted * F_rhs


def bytes_per_cell(mech: RawMechanism, per_cell_dt: bool = False) -> int:
    """Algorithmic HBM bytes per cell and flow step: read (n + 1) doubles
    (Y, T, p, deltaTChem) and write (n + 1) (Ynew, deltaTChemNew); local time
    stepping adds deltaT, and mixed batches a mechanism id (+24 B)."""
    n = mech.n_species + 2
    return 16 * (n + 1) + (24 if per_cell_dt else 0)
