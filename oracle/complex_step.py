"""TEST INFRASTRUCTURE ONLY — tangent-linear reference of the frozen-step
Rosenbrock map by the complex-step method.

The map is the one the adjoint differentiates: the accepted steps of a
recorded integration replayed with their sizes frozen,
y_{k+1} = attempt(y_k, f(y_k), h_k) (gpuRosenbrock12/23/34.H solve with the
Jacobian of gpuODESystem.H:198-281 and the LU of ludecompose.H:9-130), then
singleCellSolver's final clip max(0, Y) (singleCellSolver.H:41-45). This
module restates that map in numpy with every quantity complex: evaluated at
x + i eps d (eps = 1e-30), Im(map) / eps is the derivative of the map along d,
exact to rounding (the complex-step method: each operation propagates its
own linearisation, as forward-mode differentiation does, with no difference
quotient). Branches (coefficient sets, the pivot search, the K cap, the
clips) follow the real parts; |x| and max are taken as their analytic
continuations (x or -x by the sign of the real part). Directions may move the
initial states and the per-reaction (ln|A|, beta, Ta) of k (k0 for fall-off
reactions).

The restatement follows oracle/gf_oracle.c (pinned bit for bit to the
reference) function by function; the thermodynamic tables (species
coefficients x R, the reactions' ΔThermo) are taken from that oracle. Its real
part agrees with the oracle's attempt to rounding (tests/test_complex_step.py).
"""
from __future__ import annotations

import math

import numpy as np

RR = 6.02214e+26 * 1.38065e-23
PSTD = 1e5
VSMALL = np.finfo(np.float64).tiny
SMALL = np.finfo(np.float64).eps
VGREAT = np.finfo(np.float64).max / 10.0
LN10 = math.log(10.0)

# gpuRosenbrock12.H:14-31, gpuRosenbrock23.H:13-37, gpuRosenbrock34.H:13-46
_G12 = 1.0 + 1.0 / 1.414213562373095
ROS = {
    12: dict(gamma=_G12, a=[[], [1.0 / _G12]], c=[[], [-2.0 / _G12]], b=[(3.0 / 2.0) / _G12, (1.0 / 2.0) / _G12],
             d=[_G12, -_G12], new_f=[False, True]),
    23: dict(gamma=0.43586652150845899941601945119356, a=[[], [1.0], [1.0, 0.0]],
             c=[[], [-1.0156171083877702091975600115545],
                [4.0759956452537699824805835358067, 9.2076794298330791242156818474003]],
             b=[1.0, 6.1697947043828245592553615689730, -0.4277225654321857332623837380651],
             d=[0.43586652150845899941601945119356, 0.24291996454816804366592249683314,
                2.1851380027664058511513169485832], new_f=[False, True, False]),
    34: dict(gamma=0.5, a=[[], [2.0], [48.0 / 25.0, 6.0 / 25.0], []],
             c=[[], [-8.0], [372.0 / 25.0, 12.0 / 5.0], [-112.0 / 125.0, -54.0 / 125.0, -2.0 / 5.0]],
             b=[19.0 / 9.0, 1.0 / 2.0, 25.0 / 108.0, 125.0 / 108.0],
             d=[1.0 / 2.0, -3.0 / 2.0, 605.0 / 250.0, 29.0 / 250.0], new_f=[False, True, True, False]),
}


def cabs(x):
    """|x| continued analytically: x or -x by the sign of the real part."""
    return np.where(np.real(x) < 0, -x, x)


def cmax(a, b):
    """fmax by the real parts, keeping the chosen operand."""
    return np.where(np.real(a) >= np.real(b), a, b)


def cmin(a, b):
    return np.where(np.real(a) <= np.real(b), a, b)


class ComplexStepMap:
    """The frozen-step map of one mechanism (a gpufoam_b200.mechanism.RawMechanism)."""

    def __init__(self, raw, solver: int = 34):
        from oracle.oracle import Oracle
        sp, rx, _ = Oracle(raw, "port").tables()
        self.raw = raw
        self.nS = nS = raw.n_species
        self.nR = nR = raw.n_reactions
        self.n = nS + 2
        self.solver = solver
        # species: W, Tcommon, coefficients x R [7] (low, high)
        self.W = sp[:, 1].copy()
        self.Tcommon = sp[:, 4].copy()
        self.sp_high = sp[:, 5:12].copy()
        self.sp_low = sp[:, 12:19].copy()
        # reactions: ΔThermo Y, W, Tcommon, coefficients
        self.rY, self.rW, self.rTc = rx[:, 0].copy(), rx[:, 1].copy(), rx[:, 4].copy()
        self.r_high, self.r_low = rx[:, 5:12].copy(), rx[:, 12:19].copy()
        self.nm = self.rY / self.rW
        self.nm_small = np.abs(self.nm - SMALL) < VSMALL
        self.type = np.array([r.rate_type for r in raw.reactions])
        self.irr = np.array([bool(r.irreversible) for r in raw.reactions])
        self.sign = np.array([-1.0 if r.A < 0 else 1.0 for r in raw.reactions])
        self.Ainf = np.array([r.Ainf for r in raw.reactions])
        self.betainf = np.array([r.betainf for r in raw.reactions])
        self.Tainf = np.array([r.Tainf for r in raw.reactions])
        self.troe = np.array([r.troe for r in raw.reactions]).reshape(nR, 4)
        self.eff = np.zeros((nR, nS))
        for q, r in enumerate(raw.reactions):
            if r.efficiencies is not None:
                self.eff[q] = r.efficiencies
        self.Tlow, self.Thigh = float(raw.rxn_Tlow), float(raw.rxn_Thigh)
        # padded sides [nR][w]: species, stoichiometry, exponent, integer exponent (or None)
        w = max(max(len(r.lhs) for r in raw.reactions), max(len(r.rhs) for r in raw.reactions))
        self.w = w

        def side(name):
            idx = np.zeros((nR, w), dtype=np.int64)
            st = np.zeros((nR, w))
            ex = np.zeros((nR, w))
            isint = np.zeros((nR, w), dtype=bool)
            valid = np.zeros((nR, w), dtype=bool)
            for q, r in enumerate(raw.reactions):
                for e, (i, s, x) in enumerate(getattr(r, name)):
                    idx[q, e], st[q, e], valid[q, e] = i, s, True
                    X = int(x)
                    integer = not (x - X > 0)       # isInteger, gpuSpecieExponent.H:7-19
                    isint[q, e] = integer
                    ex[q, e] = float(X) if integer else x
            return idx, st, ex, isint, valid

        self.L = side("lhs")
        self.Rs = side("rhs")
        # raw-Jacobian scatter (gpuReaction.H:547-648): flat index into J[n][n] and signed stoichiometry
        self._build_scatter()

    # ---------------------------------------------------------------- thermo
    def _species_coeffs(self, T):
        low = np.real(T) < self.Tcommon
        return np.where(low[:, None], self.sp_low, self.sp_high)

    def _reaction_coeffs(self, T):
        low = np.real(T) < self.rTc
        return np.where(low[:, None], self.r_low, self.r_high)

    @staticmethod
    def _Cp(a, T):
        return (((a[:, 4] * T + a[:, 3]) * T + a[:, 2]) * T + a[:, 1]) * T + a[:, 0]

    @staticmethod
    def _Ha(a, T):
        return ((((a[:, 4] / 5.0 * T + a[:, 3] / 4.0) * T + a[:, 2] / 3.0) * T + a[:, 1] / 2.0) * T + a[:, 0]) * T + \
            a[:, 5]

    @staticmethod
    def _dCpdT(a, T):
        return ((4.0 * a[:, 4] * T + 3.0 * a[:, 3]) * T + 2.0 * a[:, 2]) * T + a[:, 1]

    @staticmethod
    def _Gstd(a, T, logT):
        return (a[:, 0] * (1.0 - logT) - (((a[:, 4] / 20.0 * T + a[:, 3] / 12.0) * T + a[:, 2] / 6.0) * T +
                                          a[:, 1] / 2.0) * T - a[:, 6]) * T + a[:, 5]

    @staticmethod
    def _S_pstd(a, T, logT):
        return (((a[:, 4] / 4.0 * T + a[:, 3] / 3.0) * T + a[:, 2] / 2.0) * T + a[:, 1]) * T + a[:, 0] * logT + \
            a[:, 6]

    def _Kc(self, T, with_dT=False):
        """Kc and dKc/dT / Kc of every reaction (gpuThermo.H:80-169)."""
        a = self._reaction_coeffs(T)
        logT = np.log(T)
        G = self._Gstd(a, T, logT)
        RRT = RR * T
        arg = -self.rY * G / RRT
        K = np.where(np.real(arg) < 600, np.exp(np.where(np.real(arg) < 600, arg, 0.0)), math.sqrt(VGREAT))
        Kc = np.where(self.nm_small, K, K * np.power(PSTD / RRT, self.nm))
        if not with_dT:
            return Kc
        S = self._S_pstd(a, T, logT)
        ret = (S + G / T) * self.rY / RRT
        ret = np.where(self.nm_small, ret, ret - self.nm / T)
        return Kc, ret

    # ------------------------------------------------------------- reactions
    def _arrhenius(self, A, beta, Ta, T):
        """gpuArrheniusReactionRate.H:16-26; a factor the reference skips for a
        zero beta or Ta (its value is 1) is kept when the direction moves it."""
        ak = A + 0.0 * T
        beta = np.asarray(beta)
        Ta = np.asarray(Ta)
        use_b = (np.abs(np.real(beta)) > VSMALL) | (np.imag(beta) != 0)
        use_t = (np.abs(np.real(Ta)) > VSMALL) | (np.imag(Ta) != 0)
        ak = np.where(use_b, ak * np.power(T + 0j, beta), ak)
        ak = np.where(use_t, ak * np.exp(-Ta / T), ak)
        return ak

    def _troe_F(self, T, Pr):
        alpha, Tsss, Ts, Tss = (self.troe[:, k] for k in range(4))
        logPr = np.log(cmax(Pr, SMALL + 0j)) / LN10
        Fcent = (1.0 - alpha) * np.exp(-T / Tsss) + alpha * np.exp(-T / Ts) + np.exp(-Tss / T)
        logFcent = np.log(cmax(Fcent, SMALL + 0j)) / LN10
        c = -0.4 - 0.67 * logFcent
        nn = 0.75 - 1.27 * logFcent
        x1 = nn - 0.14 * (logPr + c)
        x2 = (logPr + c) / x1
        x3 = 1.0 + x2 * x2
        x4 = logFcent / x3
        return np.exp(x4 * LN10)

    def _rates(self, T, c, theta, everything=False):
        """kf of every reaction (gpuReactionRate.H:164-173) at T and concentrations
        c; with everything, also dkf/dT and the third-body Ak
        (gpuArrheniusReactionRate.H:97-107, gpuThirdBodyArrheniusReactionRate.H:105-121,
        gpuFallOffReactionRate.H:127-158)."""
        A = self.sign * np.exp(theta[:, 0])
        beta, Ta = theta[:, 1], theta[:, 2]
        Ak = self._arrhenius(A, beta, Ta, T)
        M = self.eff @ c
        kInf = self._arrhenius(self.Ainf, self.betainf, self.Tainf, T)
        falloff = self.type >= 2
        kInf_s = np.where(falloff, kInf, 1.0)
        Pr = Ak / kInf_s * M
        F = np.where(self.type == 3, self._troe_F(T, np.where(falloff, Pr, 1.0)), 1.0)
        k = np.where(self.type == 0, Ak, np.where(self.type == 1, M * Ak, kInf * (Pr / (1.0 + Pr)) * F))
        if not everything:
            return k
        dArr = Ak * (beta + Ta / T) / T
        dInf = kInf * (self.betainf + self.Tainf / T) / T
        dT = np.where(self.type == 0, dArr, np.where(self.type == 1, M * dArr, dInf * ((Pr / (1.0 + Pr)) * F)))
        return k, dT, Ak

    def _side_pows(self, side, c):
        idx, st, ex, isint, valid = side
        x = c[idx]
        p = np.where(valid, np.power(x, ex), 1.0)
        pm1 = np.where(valid, np.where(isint & (ex == 1.0), 1.0 + 0j, np.power(x, ex - 1.0)), 1.0)
        return p, pm1

    def _mixture(self, y, p, jac):
        nS = self.nS
        T = y[nS]
        yi = cmax(y[:nS], 0.0 + 0j)
        a = self._species_coeffs(T)
        rhoi = p / ((RR / self.W) * T)
        rhoM = 1.0 / np.sum(yi / rhoi)
        Cp = self._Cp(a, T)
        Ha = self._Ha(a, T)
        CpM = np.sum(yi * Cp)
        c = rhoM * (yi / self.W)
        out = dict(T=T, rhoM=rhoM, Cp=Cp, Ha=Ha, CpM=CpM, c=c, rhoi=rhoi)
        if jac:
            out["dCpMdT"] = np.sum(yi * self._dCpdT(a, T))
            out["alphav"] = np.sum(yi / rhoi * (1.0 / T)) * rhoM
        return out

    # ----------------------------------------------------------- ODE system
    def derivatives(self, y, theta):
        """gpuODESystem::derivatives (gpuODESystem.H:164-196)."""
        nS, n = self.nS, self.n
        p = y[nS + 1]
        mx = self._mixture(y, p, False)
        T, c = mx["T"], mx["c"]
        Tc = cmin(cmax(T, self.Tlow + 0j), self.Thigh + 0j)
        kf = self._rates(Tc, c, theta)
        kr = np.where(self.irr, 0.0, kf / self._Kc(Tc))
        pl, _ = self._side_pows(self.L, c)
        pr, _ = self._side_pows(self.Rs, c)
        omega = kf * np.prod(pl, axis=1) - kr * np.prod(pr, axis=1)
        dN = np.zeros(nS, dtype=complex)
        for side, sgn in ((self.L, -1.0), (self.Rs, 1.0)):
            idx, st, _, _, valid = side
            np.add.at(dN, idx[valid], (sgn * st * omega[:, None])[valid])
        out = np.zeros(n, dtype=complex)
        out[:nS] = dN * self.W / mx["rhoM"]
        out[nS] = -np.sum(out[:nS] * mx["Ha"]) / mx["CpM"]
        return out

    def _build_scatter(self):
        nS, n = self.nS, self.n
        Li, Lst, _, _, Lv = self.L
        Ri, Rst, _, _, Rv = self.Rs
        rows, cols, coef, src = [], [], [], []
        # (kind, reaction, entry) sources: dCf[r][j] (kind 0), dCr[r][j] (kind 1), dwdT[r] (kind 2)
        for q in range(self.nR):
            both = [(Li[q, e], -Lst[q, e]) for e in range(self.w) if Lv[q, e]] + \
                   [(Ri[q, e], Rst[q, e]) for e in range(self.w) if Rv[q, e]]
            for j in range(self.w):
                if Lv[q, j]:
                    for row, s in both:
                        rows.append(row); cols.append(Li[q, j]); coef.append(s); src.append((0, q, j))
            for j in range(self.w):
                if Rv[q, j]:
                    for row, s in both:
                        rows.append(row); cols.append(Ri[q, j]); coef.append(-s); src.append((1, q, j))
            for row, s in both:
                rows.append(row); cols.append(nS); coef.append(s); src.append((2, q, 0))
        self._sc_flat = np.array(rows) * n + np.array(cols)
        self._sc_coef = np.array(coef)
        self._sc_src = np.array(src)
        # third-body rows: J[row, :nS] += s * ddc_r (kind 3)
        tb_rows, tb_coef, tb_r = [], [], []
        for q in range(self.nR):
            if self.type[q] == 1:
                for e in range(self.w):
                    if Lv[q, e]:
                        tb_rows.append(Li[q, e]); tb_coef.append(-Lst[q, e]); tb_r.append(q)
                for e in range(self.w):
                    if Rv[q, e]:
                        tb_rows.append(Ri[q, e]); tb_coef.append(Rst[q, e]); tb_r.append(q)
        self._tb_rows, self._tb_coef, self._tb_r = np.array(tb_rows, dtype=np.int64), np.array(tb_coef), \
            np.array(tb_r, dtype=np.int64)

    def jacobian(self, y, theta):
        """gpuODESystem::jacobian (gpuODESystem.H:198-281): (dfdx, J [n][n])."""
        nS, n = self.nS, self.n
        p = y[nS + 1]
        mx = self._mixture(y, p, True)
        T, c, rhoM = mx["T"], mx["c"], mx["rhoM"]
        kf, dkdT, Ak = self._rates(T, c, theta, everything=True)
        Kc, dKc = self._Kc(T, with_dT=True)
        kr = np.where(self.irr, 0.0, kf / Kc)
        pl, pml = self._side_pows(self.L, c)
        pr, pmr = self._side_pows(self.Rs, c)
        Cf = np.prod(pl, axis=1)
        Cr = np.where(self.irr, 0.0, np.prod(pr, axis=1))
        w = self.w

        def dC(pw, pm, ex):
            out = np.empty_like(pw)
            for j in range(w):
                d = np.ones(pw.shape[0], dtype=complex)
                for i in range(w):
                    d = d * (ex[:, j] * pm[:, j] if i == j else pw[:, i])
                out[:, j] = d
            return out

        dCf = dC(pl, pml, self.L[2]) * kf[:, None]
        dCr = np.where(self.irr[:, None], 0.0, dC(pr, pmr, self.Rs[2]) * kr[:, None])
        omega = Cf * kf - Cr * kr
        dkrdT = dkdT / Kc - kr * dKc
        dwdT = Cf * dkdT - np.where(self.irr, 0.0, Cr * dkrdT)
        # dfdx = f(y) at the unclipped T (gpuODESystem.H:226-243)
        dN = np.zeros(nS, dtype=complex)
        for side, sgn in ((self.L, -1.0), (self.Rs, 1.0)):
            idx, st, _, _, valid = side
            np.add.at(dN, idx[valid], (sgn * st * omega[:, None])[valid])
        dfdx = np.zeros(n, dtype=complex)
        dfdx[:nS] = dN * self.W / rhoM
        dfdx[nS] = -np.sum(dfdx[:nS] * mx["Ha"]) / mx["CpM"]
        # raw dN/dc and dN/dT
        kind, q, j = self._sc_src[:, 0], self._sc_src[:, 1], self._sc_src[:, 2]
        val = np.where(kind == 0, dCf[q, j], np.where(kind == 1, dCr[q, j], dwdT[q]))
        Jr = np.zeros(n * n, dtype=complex)
        np.add.at(Jr, self._sc_flat, self._sc_coef * val)
        Jr = Jr.reshape(n, n)
        if self._tb_r.size:
            tmp = Cf - np.where(self.irr, 0.0, Cr / Kc)
            ddc = self.eff[self._tb_r] * (Ak[self._tb_r] * tmp[self._tb_r])[:, None]
            np.add.at(Jr, (np.repeat(self._tb_rows, nS), np.tile(np.arange(nS), self._tb_rows.size)),
                      (self._tb_coef[:, None] * ddc).reshape(-1))
        # ddY_dcdY, ddT_dtdY, ddT_dtdT (gpuODESystem.H:65-146)
        J = np.zeros((n, n), dtype=complex)
        WbyR = self.W / rhoM
        vj = 1.0 / mx["rhoi"]
        J[:nS, :nS] = WbyR[:, None] * Jr[:nS, :nS] * (rhoM / self.W)[None, :] + rhoM * vj[None, :] * dfdx[:nS, None]
        alphav = mx["alphav"]
        J[:nS, nS] = WbyR * (Jr[:nS, nS] - np.sum(Jr[:nS, :nS] * c[None, :] * alphav, axis=1)) + alphav * dfdx[:nS]
        J[nS, :nS] = (-np.sum(J[:nS, :nS] * mx["Ha"][:, None], axis=0) - mx["Cp"] * dfdx[nS]) / mx["CpM"]
        J[nS, nS] = (-np.sum(dfdx[:nS] * mx["Cp"] + J[:nS, nS] * mx["Ha"]) - dfdx[nS] * mx["dCpMdT"]) / mx["CpM"]
        return dfdx, J

    # ------------------------------------------------------------------- LU
    @staticmethod
    def lu_decompose(A):
        """LUDecompose (ludecompose.H:9-92) in right-looking order; pivots by the
        real parts of vv |a| (last max wins), a zero pivot becomes gpuSmall."""
        A = A.copy()
        m = A.shape[0]
        vv = np.empty(m, dtype=complex)
        for i in range(m):
            k = int(np.argmax(np.abs(np.real(A[i]))))
            vv[i] = 1.0 / cabs(A[i, k])
        piv = np.zeros(m, dtype=np.int64)
        for k in range(m):
            cand = np.real(vv[k:] * cabs(A[k:, k]))
            best = np.max(cand)
            iMax = k + int(np.nonzero(cand == best)[0][-1])
            piv[k] = iMax
            if iMax != k:
                A[[k, iMax]] = A[[iMax, k]]
                vv[iMax] = vv[k]
            if A[k, k] == 0:
                A[k, k] = SMALL
            if k != m - 1:
                A[k + 1:, k] *= 1.0 / A[k, k]
                A[k + 1:, k + 1:] -= np.outer(A[k + 1:, k], A[k, k + 1:])
        return A, piv

    @staticmethod
    def lu_solve(LU, piv, b):
        """LUBacksubstitute (ludecompose.H:94-130)."""
        x = b.copy()
        m = LU.shape[0]
        for i in range(m):
            ip = piv[i]
            if ip != i:
                x[i], x[ip] = x[ip], x[i]
        for i in range(1, m):
            x[i] -= np.dot(LU[i, :i], x[:i])
        for i in range(m - 1, -1, -1):
            x[i] = (x[i] - np.dot(LU[i, i + 1:], x[i + 1:])) / LU[i, i]
        return x

    # ----------------------------------------------------------- Rosenbrock
    def step(self, y0, h, theta):
        """One attempt of the solver from y0 with step h and dydx0 = f(y0): the new state."""
        C = ROS[self.solver]
        s = len(C["b"])
        n = self.n
        dydx0 = self.derivatives(y0, theta)
        dfdx, J = self.jacobian(y0, theta)
        W = -J + np.eye(n) / (C["gamma"] * h)
        LU, piv = self.lu_decompose(W)
        k = []
        f = dydx0
        for st in range(s):
            if st > 0 and C["new_f"][st]:
                yt = y0 + sum(C["a"][st][j] * k[j] for j in range(st))
                f = self.derivatives(yt, theta)
            rhs = f + h * C["d"][st] * dfdx
            if st > 0:
                rhs = rhs + sum(C["c"][st][j] * k[j] for j in range(st)) / h
            k.append(self.lu_solve(LU, piv, rhs))
        return y0 + sum(C["b"][st] * k[st] for st in range(s))

    def frozen_map(self, y0, steps, theta):
        """The recorded steps replayed from y0, then max(0, Y)."""
        y = np.asarray(y0, dtype=complex).copy()
        with np.errstate(all="ignore"):  # the unused branches of np.where (other rate types)
            for h in steps:
                y = self.step(y, float(h), theta)
        y[:self.nS] = cmax(y[:self.nS], 0.0 + 0j)
        return y

    def directional(self, y0, steps, theta, dy=None, dtheta=None, eps=1e-30):
        """d map / d(y0, theta) along (dy, dtheta) by the complex step."""
        y = np.asarray(y0, dtype=complex) + (0 if dy is None else 1j * eps * np.asarray(dy))
        th = np.asarray(theta, dtype=complex) + (0 if dtheta is None else 1j * eps * np.asarray(dtheta))
        return np.imag(self.frozen_map(y, steps, th)) / eps
