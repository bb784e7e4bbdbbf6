"""Seeded synthetic reaction mechanisms and cell batches.

No public benchmark data is involved in this project's workloads: every
mechanism and every batch of cell states is drawn here from a seed, with the
shapes and parameter distributions of the gpuFoam chemistry configurations:

* reactions: reversible Arrhenius with log10 A ~ U[8, 14], beta ~ U[-1.5, 2],
  Ea ~ U[0, 200] kJ/mol (Ta = Ea / R_u), third-body Arrhenius with
  efficiencies ~ U[0.5, 12], Troe fall-off with alpha ~ U[0.4, 0.8] and
  T***, T*, T** ~ log-U[1e1, 1e4] K;
* species: NASA-7 (JANAF) polynomials per species, continuous in Cp, H and S
  at Tcommon = 1000 K, positive Cp over 200-5000 K;
* cells: T ~ U[Tmin, Tmax], p fixed (or drawn), Y ~ Dirichlet(0.5).

Element balance: species are small molecules over four pseudo-elements with the
masses of H, O, C and N, and every reaction conserves atoms, so the mass
balance check of the reference loader (makeGpuReactions.H:48-54, |lhs - rhs|
<= 0.1 kg/kmol) always passes. One species is an inert N2 that only acts as a
third body.

The raw form mirrors what the OpenFOAM dictionaries hold (thermo coefficients
before the x R scaling of makeGpuThermo.H:41-44, reactions as
(index, stoich, exponent) lists as in makeGpuReactions.H:61-88).
"""
from __future__ import annotations

import dataclasses
import itertools
import math
from typing import List, Optional, Tuple

import numpy as np

R_U = 8.314462618  # J/mol/K, Ta = Ea / R_U

RATE_ARRHENIUS = 0
RATE_THIRD_BODY = 1
RATE_LINDEMANN = 2
RATE_TROE = 3

# pseudo-elements (masses of H, O, C, N)
_ELEMENT_MASS = np.array([1.00794, 15.9994, 12.0107, 14.0067])

DBL_MAX_OVER_10 = np.finfo(np.float64).max / 10.0


@dataclasses.dataclass
class RawReaction:
    rate_type: int
    irreversible: bool
    lhs: List[Tuple[int, float, float]]  # (species index, stoich coeff, exponent)
    rhs: List[Tuple[int, float, float]]
    A: float = 0.0
    beta: float = 0.0
    Ta: float = 0.0
    Ainf: float = 0.0
    betainf: float = 0.0
    Tainf: float = 0.0
    troe: Tuple[float, float, float, float] = (0.0, 1.0, 1.0, 1.0)  # alpha, Tsss, Ts, Tss
    efficiencies: Optional[np.ndarray] = None


@dataclasses.dataclass
class RawMechanism:
    name: str
    species: List[str]
    W: np.ndarray          # [nS] kg/kmol
    Tlow: np.ndarray       # [nS]
    Thigh: np.ndarray      # [nS]
    Tcommon: np.ndarray    # [nS]
    high_raw: np.ndarray   # [nS, 7] NASA-7 (Cp/R units)
    low_raw: np.ndarray    # [nS, 7]
    reactions: List[RawReaction]
    rxn_Tlow: float = 0.0
    rxn_Thigh: float = DBL_MAX_OVER_10

    @property
    def n_species(self) -> int:
        return len(self.species)

    @property
    def n_reactions(self) -> int:
        return len(self.reactions)

    @property
    def n_eqns(self) -> int:
        return self.n_species + 2

    def type_counts(self):
        counts = {}
        for r in self.reactions:
            counts[r.rate_type] = counts.get(r.rate_type, 0) + 1
        return counts


# --------------------------------------------------------------------------
# species

def _composition_pool(max_atoms: int):
    """All compositions over (H, O, C) with 1..max_atoms atoms (N only in N2)."""
    pool = []
    for h in range(0, max_atoms + 1):
        for o in range(0, max_atoms + 1 - h):
            for c in range(0, max_atoms + 1 - h - o):
                if h + o + c == 0:
                    continue
                pool.append((h, o, c, 0))
    # small molecules first so that small mechanisms look like H2/O2 chemistry
    pool.sort(key=lambda t: (sum(t), t[2], -t[0]))
    return pool


def _pick_species(n_species: int, rng: np.random.Generator):
    n_reactive = n_species - 1
    pool = _composition_pool(8)
    # always keep the smallest H/O molecules, then draw the rest with a bias
    # towards small molecules (weight ~ 1/atoms^2)
    core = [t for t in pool if t[2] == 0 and sum(t) <= 4][: min(n_reactive, 9)]
    rest = [t for t in pool if t not in core]
    w = np.array([1.0 / (sum(t) ** 2) for t in rest])
    w /= w.sum()
    n_more = n_reactive - len(core)
    picked = list(core)
    if n_more > 0:
        idx = rng.choice(len(rest), size=n_more, replace=False, p=w)
        picked += [rest[i] for i in sorted(idx)]
    picked.append((0, 0, 0, 2))  # inert N2
    return picked


def _name(comp):
    parts = []
    for sym, k in zip("HOCN", comp):
        if k:
            parts.append(sym + (str(k) if k > 1 else ""))
    return "".join(parts)


# standard enthalpies of formation of the gaseous atoms H, O, C, N [J/mol]
_ATOM_HF = np.array([218.0e3, 249.2e3, 716.7e3, 472.7e3])


def _nasa7(comp, rng: np.random.Generator, inert=False):
    """Random NASA-7 low/high coefficient sets (Cp/R, H/R, S/R units).

    Cp/R is a quartic in t = T/1000 on each range; the high range continues the
    low one at t = 1 in value, and the a5/a6 constants make H and S continuous
    at Tcommon = 1000 K. The enthalpy of formation is the atoms' minus a bond
    energy of U[300, 450] kJ/mol per bond (atoms - 1 bonds), so that bond
    forming releases heat as in real chemistry; S298/R grows with the atom count.
    """
    n_atoms = int(sum(comp))
    base = 2.5 if n_atoms == 1 else 3.5 + 0.5 * (n_atoms - 2)
    top = 2.5 if n_atoms == 1 else max(4.5, 3.0 * n_atoms - 2.0)
    while True:
        b = np.array([
            base + rng.uniform(-0.3, 0.5),
            rng.uniform(0.0, 1.0) * (top - base) * 0.8,
            rng.uniform(-0.5, 0.5),
            rng.uniform(-0.3, 0.3),
            rng.uniform(-0.05, 0.05),
        ])
        t = np.linspace(0.2, 1.0, 81)
        cp = np.polyval(b[::-1], t)
        if cp.min() >= 2.0 and cp.max() <= top + 3.0:
            break
    c1 = np.polyval(b[::-1], 1.0)
    while True:
        s = rng.uniform(0.0, 0.8) * max(top - c1, 0.2)
        q = rng.uniform(-0.15, 0.0) * max(top - c1, 0.2) * 0.25
        r3 = rng.uniform(-0.01, 0.01)
        w4 = rng.uniform(-0.001, 0.001)
        # Cp_high(t) = c1 + s u + q u^2 + r3 u^3 + w4 u^4, u = t - 1, expanded in t
        cu = [c1, s, q, r3, w4]
        bh = np.zeros(5)
        for k, ck in enumerate(cu):
            for j in range(k + 1):
                bh[j] += ck * math.comb(k, j) * (-1.0) ** (k - j)
        t = np.linspace(1.0, 5.0, 161)
        cp = np.polyval(bh[::-1], t)
        if cp.min() >= 2.0:
            break
    scale = np.array([1.0, 1e-3, 1e-6, 1e-9, 1e-12])
    low = np.zeros(7)
    high = np.zeros(7)
    low[:5] = b * scale
    high[:5] = bh * scale

    def h_over_r(a, T):
        return (((((a[4] / 5.0 * T + a[3] / 4.0) * T + a[2] / 3.0) * T + a[1] / 2.0) * T + a[0]) * T)

    def s_over_r(a, T):
        return ((((a[4] / 4.0 * T + a[3] / 3.0) * T + a[2] / 2.0) * T + a[1]) * T + a[0] * math.log(T))

    if inert:
        hf = 0.0
    else:
        bonds = rng.uniform(300e3, 450e3, size=max(n_atoms - 1, 0)).sum()
        hf = (float(np.dot(comp, _ATOM_HF)) - bonds) / R_U  # Hf/R at 298.15 K [K]
    s298 = 10.0 + 5.5 * n_atoms + rng.uniform(-2.0, 2.0)
    low[5] = hf - h_over_r(low, 298.15)
    low[6] = s298 - s_over_r(low, 298.15)
    high[5] = h_over_r(low, 1000.0) + low[5] - h_over_r(high, 1000.0)
    high[6] = s_over_r(low, 1000.0) + low[6] - s_over_r(high, 1000.0)
    return high, low


# --------------------------------------------------------------------------
# reactions

def _arrhenius(rng, order: int):
    """(A, beta, Ta) in the OpenFOAM form k = A T^beta exp(-Ta/T) [kmol, m^3, s].

    log10 A ~ U[8, 14] is read in CHEMKIN units (cm^3/mol)^(order-1)/s — the
    units of the reference's mechanism sources (tutorials/*/chemkin/chem.inp) —
    and as the prefactor at T_ref = 1000 K, so the stored OpenFOAM prefactor is
    A * 1e-3^(order-1) * T_ref^-beta. Independent draws of A and beta would
    otherwise reach 1e14 * 2500^2 (seven orders above the collision limit).
    """
    logA = rng.uniform(8.0, 14.0)
    beta = rng.uniform(-1.5, 2.0)
    Ea = rng.uniform(0.0, 200e3)  # J/mol
    A = 10.0 ** logA * (1e-3 ** (order - 1)) * 1000.0 ** (-beta)
    return A, beta, Ea / R_U


def _troe(rng):
    alpha = rng.uniform(0.4, 0.8)
    tsss, ts, tss = (10.0 ** rng.uniform(1.0, 4.0) for _ in range(3))
    return (alpha, tsss, ts, tss)


def _side(indices, frac_exponent=None):
    """(index, stoich, exponent) entries; repeated species merge into one entry."""
    out = []
    for i in sorted(set(indices), key=indices.index):
        k = indices.count(i)
        e = float(k) if frac_exponent is None else frac_exponent
        out.append((i, float(k), e))
    return out


def make_mechanism(n_species: int, n_arrhenius: int, n_third_body: int, n_troe: int,
                   seed: int = 0, n_lindemann: int = 0, n_irreversible: int = 0,
                   n_fractional: int = 0, name: Optional[str] = None,
                   rxn_Tlow: float = 0.0, rxn_Thigh: float = DBL_MAX_OVER_10) -> RawMechanism:
    """Draw a mechanism. `n_irreversible` of the Arrhenius reactions are made
    irreversible and `n_fractional` get a non-integer reactant exponent (both 0
    in the benchmark configurations; the feature-coverage test mechanism uses
    them)."""
    rng = np.random.default_rng(seed)
    comps = _pick_species(n_species, rng)
    species = [_name(c) for c in comps]
    # disambiguate duplicate names (isomers)
    seen = {}
    for i, s in enumerate(species):
        if s in seen:
            seen[s] += 1
            species[i] = f"{s}_{seen[s]}"
        else:
            seen[s] = 0
    W = np.array([float(np.dot(c, _ELEMENT_MASS)) for c in comps])
    nS = n_species
    high = np.zeros((nS, 7))
    low = np.zeros((nS, 7))
    for i, c in enumerate(comps):
        h, l = _nasa7(c, rng, inert=(i == nS - 1))
        high[i], low[i] = h, l

    reactive = list(range(nS - 1))
    by_comp = {}
    for i in reactive:
        by_comp.setdefault(comps[i], []).append(i)

    def add(a, b):
        return tuple(x + y for x, y in zip(a, b))

    def sub(a, b):
        return tuple(x - y for x, y in zip(a, b))

    exchanges, associations = [], []
    for a, b in itertools.combinations_with_replacement(reactive, 2):
        tot = add(comps[a], comps[b])
        for c in by_comp.get(tot, []):
            associations.append(((a, b), (c,)))
        for c in reactive:
            rem = sub(tot, comps[c])
            if min(rem) < 0:
                continue
            for d in by_comp.get(rem, []):
                if d < c:
                    continue
                if sorted((a, b)) == sorted((c, d)):
                    continue
                exchanges.append(((a, b), (c, d)))
    # canonical, de-duplicated (a reaction and its reverse are the same reaction)
    def canon(rx):
        l, r = tuple(sorted(rx[0])), tuple(sorted(rx[1]))
        return min((l, r), (r, l))
    exchanges = sorted({canon(x) for x in exchanges})
    associations = sorted({canon(x) for x in associations})
    if len(exchanges) < n_arrhenius or len(associations) < n_third_body + n_troe + n_lindemann:
        raise ValueError("species set too small for the requested reaction counts")

    # molar Gibbs energy G/(R T) of every species at 1500 K (high-range polynomial)
    def g_rt(i, T=1500.0):
        a = high[i]
        h = (((((a[4] / 5.0 * T + a[3] / 4.0) * T + a[2] / 3.0) * T + a[1] / 2.0) * T + a[0]) * T + a[5])
        s_ = ((((a[4] / 4.0 * T + a[3] / 3.0) * T + a[2] / 2.0) * T + a[1]) * T + a[0] * math.log(T) + a[6])
        return h / T - s_
    G1500 = np.array([g_rt(i) for i in range(nS)])

    def exothermic(l, r):
        # orient every reaction so that its forward direction is the
        # thermodynamically favoured one (K >= 1 at 1500 K): the drawn rate
        # then belongs to the downhill direction and the reverse rate kf/Kc
        # stays bounded
        dG = sum(G1500[i] for i in r) - sum(G1500[i] for i in l)
        return (l, r) if dG <= 0.0 else (r, l)

    ex_idx = rng.choice(len(exchanges), size=n_arrhenius, replace=False)
    n_assoc = n_third_body + n_troe + n_lindemann
    as_idx = rng.choice(len(associations), size=n_assoc, replace=False)

    reactions: List[RawReaction] = []
    for k in ex_idx:
        l, r = exothermic(*exchanges[k])
        A, beta, Ta = _arrhenius(rng, order=len(l))
        reactions.append(RawReaction(RATE_ARRHENIUS, False, _side(list(l)), _side(list(r)), A, beta, Ta))
    kinds = [RATE_THIRD_BODY] * n_third_body + [RATE_TROE] * n_troe + [RATE_LINDEMANN] * n_lindemann
    for kind, k in zip(kinds, as_idx):
        l, r = exothermic(*associations[k])  # A + B (+M) = AB or its reverse
        eff = rng.uniform(0.5, 12.0, size=nS)
        # third-body and low-pressure (k0) rates carry the extra order of M
        A, beta, Ta = _arrhenius(rng, order=len(l) + 1)
        rx = RawReaction(kind, False, _side(list(l)), _side(list(r)), A, beta, Ta, efficiencies=eff)
        if kind in (RATE_TROE, RATE_LINDEMANN):
            rx.Ainf, rx.betainf, rx.Tainf = _arrhenius(rng, order=len(l))
            if kind == RATE_TROE:
                rx.troe = _troe(rng)
        reactions.append(rx)
    # interleave the kinds the way real mechanisms do (not grouped by type)
    order = rng.permutation(len(reactions))
    reactions = [reactions[i] for i in order]
    # optional feature coverage
    arr = [i for i, r in enumerate(reactions) if r.rate_type == RATE_ARRHENIUS]
    for i in arr[:n_irreversible]:
        reactions[i].irreversible = True
    for i in arr[n_irreversible:n_irreversible + n_fractional]:
        r = reactions[i]
        idx, st, _ = r.lhs[0]
        r.lhs[0] = (idx, st, st + 0.5)
    return RawMechanism(name or f"synthetic-{nS}sp-{len(reactions)}rx-seed{seed}", species, W,
                        np.full(nS, 200.0), np.full(nS, 5000.0), np.full(nS, 1000.0),
                        high, low, reactions, rxn_Tlow, rxn_Thigh)


# --------------------------------------------------------------------------
# the mechanisms of the benchmark configurations

def h2_size(seed: int = 0) -> RawMechanism:
    """10 species (incl. inert N2), 27 reversible reactions: 20 Arrhenius,
    5 third-body, 2 Troe."""
    return make_mechanism(10, 20, 5, 2, seed=seed, name=f"synthetic-H2size-seed{seed}")


def gri_size(seed: int = 0) -> RawMechanism:
    """53 species, 325 reversible reactions: 250 Arrhenius, 45 third-body, 30 Troe."""
    return make_mechanism(53, 250, 45, 30, seed=seed, name=f"synthetic-GRIsize-seed{seed}")


def large(seed: int = 0) -> RawMechanism:
    """100 species, 600 reversible reactions: 460 Arrhenius, 85 third-body, 55 Troe."""
    return make_mechanism(100, 460, 85, 55, seed=seed, name=f"synthetic-100sp-seed{seed}")


def coverage(seed: int = 0) -> RawMechanism:
    """Small mechanism exercising every rate path of the reference: irreversible
    Arrhenius, non-integer exponents, Lindemann and Troe fall-off, third body."""
    return make_mechanism(12, 14, 3, 2, seed=seed, n_lindemann=2, n_irreversible=3,
                          n_fractional=2, name=f"synthetic-coverage-seed{seed}")


# --------------------------------------------------------------------------
# cell batches

def make_cells(mech: RawMechanism, n_cells: int, seed: int = 0, T_range=(1000.0, 2500.0),
               p: float = 101325.0, bimodal: Optional[Tuple[float, Tuple[float, float], Tuple[float, float]]] = None,
               p_range: Optional[Tuple[float, float]] = None, dirichlet_alpha: float = 0.5,
               cold_reactive_fraction: Optional[float] = None) -> np.ndarray:
    """[n_cells, nS + 2] cell states (Y..., T, p), cell-major.

    bimodal = (fraction_cold, (Tlo, Thi)_cold, (Tlo, Thi)_hot): cells drawn cold
    or hot, then shuffled by the seed. cold_reactive_fraction (bimodal only):
    the cold cells are near-inert, their Dirichlet composition scaled to this
    total mass fraction and the rest given to the inert species (the last
    one); None leaves every cell's Dirichlet composition as drawn.
    """
    rng = np.random.default_rng(seed)
    nS = mech.n_species
    Y = rng.dirichlet(np.full(nS, dirichlet_alpha), size=n_cells)
    Y /= Y.sum(axis=1, keepdims=True)
    if bimodal is None:
        T = rng.uniform(T_range[0], T_range[1], size=n_cells)
    else:
        frac, cold, hot = bimodal
        n_cold = int(round(frac * n_cells))
        T = np.concatenate([rng.uniform(cold[0], cold[1], size=n_cold),
                            rng.uniform(hot[0], hot[1], size=n_cells - n_cold)])
        is_cold = np.arange(n_cells) < n_cold
        order = rng.permutation(n_cells)
        T, is_cold = T[order], is_cold[order]
        if cold_reactive_fraction is not None:
            eps = float(cold_reactive_fraction)
            Y[is_cold] *= eps
            Y[is_cold, nS - 1] += 1.0 - eps
    if p_range is None:
        P = np.full(n_cells, p)
    else:
        P = rng.uniform(p_range[0], p_range[1], size=n_cells)
    out = np.empty((n_cells, nS + 2))
    out[:, :nS] = Y
    out[:, nS] = T
    out[:, nS + 1] = P
    return out


def log_uniform(rng: np.random.Generator, lo: float, hi: float, size: int) -> np.ndarray:
    return np.exp(rng.uniform(math.log(lo), math.log(hi), size=size))
