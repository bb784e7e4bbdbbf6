"""Shared tolerance helpers of the parity tests.

Tolerances (from the project's parity contract):
  * rates / Jacobian: 1e-12 relative on identical states, with a per-entry
    floor of 1e-12 x the entry's absolute-rate scale (sum of |kf Cf| + |kr Cr|
    over the contributing reactions) because omega = kf Cf - kr Cr cancels
    near equilibrium;
  * integrated states: |dY| <= 1e-9 + 10 relTol |Y| and |dT| <= 1e-3 K;
  * accepted-step counts equal in >= 99% of cells.
"""
import numpy as np

RR = 6.02214e+26 * 1.38065e-23


def rate_scale(mech, y):
    """Absolute-rate scale of dY_i/dt and dT/dt at the states y [n][nS+2]:
    W_i/rhoM * sum_r |nu_ir| (|kf Cf| + |kr Cr|) and sum_i |scale_i Ha_i| / CpM,
    evaluated with numpy from the raw mechanism (reference formulas)."""
    from oracle.oracle import Oracle
    o = Oracle(mech, "port")
    nS = mech.n_species
    y = np.atleast_2d(y)
    out = np.zeros_like(y)
    for k, s in enumerate(y):
        T, p = s[nS], s[nS + 1]
        Yc = np.maximum(s[:nS], 0.0)
        Rsp = RR / mech.W
        rho = p / (Rsp * T)
        rhoM = 1.0 / np.sum(Yc / rho)
        c = rhoM * Yc / mech.W
        ev = o.reaction_eval(s)
        th = o.thermo_eval(p, T)
        CpM = np.sum(Yc * th[:, 0])
        sc = np.zeros(nS)
        for r, rx in enumerate(mech.reactions):
            Cf = np.prod([c[i] ** e for i, _, e in rx.lhs])
            Cr = np.prod([c[i] ** e for i, _, e in rx.rhs])
            a = abs(ev[r, 0] * Cf) + abs(ev[r, 1] * Cr)
            for i, st, _ in rx.lhs:
                sc[i] += abs(st) * a
            for i, st, _ in rx.rhs:
                sc[i] += abs(st) * a
        sc *= mech.W / rhoM
        out[k, :nS] = sc
        out[k, nS] = np.sum(np.abs(sc * th[:, 1])) / CpM
    return out


def jacobian_scale(mech, y):
    """Absolute-contribution scale of every Jacobian entry at the states y:
    the reference's J with each reaction term (dCf kf, dCr kr, dwdT, third-body
    dk/dc, gpuReaction.H:547-702) and each conversion term (gpuODESystem.H:65-146)
    taken in absolute value. The rounding error of an entry is bounded by a
    small multiple of eps times this scale, however much the terms cancel."""
    from oracle.oracle import Oracle
    o = Oracle(mech, "port")
    nS = mech.n_species
    n = nS + 2
    y = np.atleast_2d(y)
    out = np.zeros((y.shape[0], n, n))
    for k, s in enumerate(y):
        T, p = s[nS], s[nS + 1]
        Yc = np.maximum(s[:nS], 0.0)
        rho = p / ((RR / mech.W) * T)
        rhoM = 1.0 / np.sum(Yc / rho)
        c = rhoM * Yc / mech.W
        ev = o.reaction_eval(s)
        th = o.thermo_eval(p, T)
        Cp, Ha = th[:, 0], th[:, 1]
        CpM = np.sum(Yc * Cp)
        dCpMdT = np.sum(Yc * th[:, 5])
        alphav = np.sum(Yc / rho / T) * rhoM
        dydx = o.derivatives(s)[0]
        raw = np.zeros((nS, nS + 1))

        def dC(side, j):
            v = 1.0
            for i, (idx, st, e) in enumerate(side):
                v *= e * c[idx] ** (e - 1) if i == j else c[idx] ** e
            return v

        for r, rx in enumerate(mech.reactions):
            kf, kr, dwdT = ev[r, 0], ev[r, 1], ev[r, 5]
            both = rx.lhs + rx.rhs
            for j, (jdx, _, _) in enumerate(rx.lhs):
                v = abs(dC(rx.lhs, j) * kf)
                for idx, st, _ in both:
                    raw[idx, jdx] += abs(st) * v
            if not rx.irreversible:
                for j, (jdx, _, _) in enumerate(rx.rhs):
                    v = abs(dC(rx.rhs, j) * kr)
                    for idx, st, _ in both:
                        raw[idx, jdx] += abs(st) * v
            for idx, st, _ in both:
                raw[idx, nS] += abs(st) * abs(dwdT)
            if rx.rate_type == 1:
                Mc = np.dot(rx.efficiencies, c)
                Ak = abs(kf / Mc) if Mc else 0.0
                Cf = np.prod([c[i] ** e for i, _, e in rx.lhs])
                Cr = np.prod([c[i] ** e for i, _, e in rx.rhs])
                tmp = abs(Cf) + abs(Cr / ev[r, 3])
                for idx, st, _ in both:
                    raw[idx, :nS] += abs(st) * np.abs(rx.efficiencies) * Ak * tmp
        WbyR = mech.W / rhoM
        S = np.zeros((n, n))
        S[:nS, :nS] = WbyR[:, None] * raw[:, :nS] * (rhoM / mech.W)[None, :] + \
            np.abs(rhoM / rho[None, :] * dydx[:nS, None])
        S[:nS, nS] = WbyR * (raw[:, nS] + alphav * np.sum(raw[:, :nS] * c[None, :], axis=1)) + \
            np.abs(alphav * dydx[:nS])
        S[nS, :nS] = (np.sum(S[:nS, :nS] * np.abs(Ha)[:, None], axis=0) + np.abs(Cp * dydx[nS])) / CpM
        S[nS, nS] = (np.sum(np.abs(dydx[:nS] * Cp) + S[:nS, nS] * np.abs(Ha)) + abs(dydx[nS] * dCpMdT)) / CpM
        out[k] = S
    return out


def assert_rates_close(got, ref, scale, rtol=1e-12):
    got, ref = np.asarray(got), np.asarray(ref)
    bound = rtol * (np.abs(ref) + scale)
    err = np.abs(got - ref)
    bad = err > bound
    assert not bad.any(), f"{bad.sum()} entries beyond 1e-12: worst {np.max(err / np.maximum(bound, 1e-300)):.3g}x bound"


def assert_jacobian_close(got, ref, scale, rtol=1e-12):
    """1e-12 relative per entry with the per-entry floor 1e-12 x the entry's
    absolute-contribution scale (jacobian_scale), the Jacobian analogue of the
    rate tolerance."""
    got, ref = np.asarray(got), np.asarray(ref)
    bound = rtol * (np.abs(ref) + scale)
    err = np.abs(got - ref)
    bad = err > bound
    assert not bad.any(), (f"{bad.sum()} of {bad.size} entries beyond tolerance; worst ratio "
                           f"{np.max(err / np.maximum(bound, 1e-300)):.3g}")


def assert_states_close(got, ref, nS, relTol, what=""):
    got, ref = np.asarray(got), np.asarray(ref)
    dY = np.abs(got[:, :nS] - ref[:, :nS])
    tolY = 1e-9 + 10 * relTol * np.abs(ref[:, :nS])
    badY = dY > tolY
    dT = np.abs(got[:, nS] - ref[:, nS])
    badT = dT > 1e-3
    assert not badY.any() and not badT.any(), (
        f"{what}: {badY.any(axis=1).sum()} cells with |dY| out of tolerance (worst {np.max(dY - tolY):.3g}), "
        f"{badT.sum()} with |dT| > 1e-3 K (worst {dT.max():.3g})")
    assert np.array_equal(got[:, nS + 1], ref[:, nS + 1]), "pressure must be carried unchanged"


def step_count_agreement(got_counts, ref_counts):
    got_counts, ref_counts = np.asarray(got_counts), np.asarray(ref_counts)
    return float(np.mean(got_counts[:, 0] == ref_counts[:, 0]))
