// Differentiation helpers of the discrete adjoint (gf_adjoint.cu): forward-mode
// dual numbers, the rate and thermo expressions for a generic scalar, and the
// per-reaction vector-Jacobian product, following the same formulas, in the
// same order, as the double-precision device code in gf_device.cuh (gpuReaction.H,
// gpuThermo.H, gpuArrheniusReactionRate.H, gpuThirdBodyArrheniusReactionRate.H,
// gpuFallOffReactionRate.H, gpuTroeFallOffFunction.H of the reference).
#pragma once

#include "gf_device.cuh"

namespace gf {

// ------------------------------------------------------------ dual numbers

template <int K>
struct Dual {
    double v;
    double d[K];
};

template <int K>
__device__ __forceinline__ Dual<K> dconst(double v) {
    Dual<K> r;
    r.v = v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = 0.0;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> dseed(double v, int k0) {
    Dual<K> r = dconst<K>(v);
#pragma unroll
    for (int k = 0; k < K; ++k)
        if (k == k0) r.d[k] = 1.0;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] + b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] - b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(const Dual<K>& a) {
    Dual<K> r;
    r.v = -a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -a.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b.v + a.v * b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a.v / b.v;
    const double ib = 1.0 / b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = (a.d[k] - r.v * b.d[k]) * ib;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator+(const Dual<K>& a, double b) {
    Dual<K> r = a;
    r.v = a.v + b;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator+(double a, const Dual<K>& b) {
    return b + a;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(const Dual<K>& a, double b) {
    Dual<K> r = a;
    r.v = a.v - b;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator-(double a, const Dual<K>& b) {
    Dual<K> r;
    r.v = a - b.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = -b.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator*(const Dual<K>& a, double b) {
    Dual<K> r;
    r.v = a.v * b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * b;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator*(double a, const Dual<K>& b) {
    return b * a;
}
template <int K>
__device__ __forceinline__ Dual<K> operator/(const Dual<K>& a, double b) {
    Dual<K> r;
    r.v = a.v / b;
    const double ib = 1.0 / b;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * ib;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> operator/(double a, const Dual<K>& b) {
    return dconst<K>(a) / b;
}
template <int K>
__device__ __forceinline__ Dual<K> exp(const Dual<K>& a) {
    Dual<K> r;
    r.v = ::exp(a.v);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = r.v * a.d[k];
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> log(const Dual<K>& a) {
    Dual<K> r;
    r.v = ::log(a.v);
    const double ia = 1.0 / a.v;
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = a.d[k] * ia;
    return r;
}
template <int K>
__device__ __forceinline__ Dual<K> pow(const Dual<K>& a, double e) {
    Dual<K> r;
    r.v = ::pow(a.v, e);
    const double dv = e * ::pow(a.v, e - 1.0);
#pragma unroll
    for (int k = 0; k < K; ++k) r.d[k] = dv * a.d[k];
    return r;
}
__device__ __forceinline__ double val(double a) { return a; }
template <int K>
__device__ __forceinline__ double val(const Dual<K>& a) {
    return a.v;
}

// ---------------------------------------------- per-reaction quantities (S)

// gpuSpecieExponent.H:21-36 / 103-110 for a generic scalar
template <class S>
__device__ __forceinline__ S integer_pow_s(const S& x, int e) {
    if (e == 0) return x * 0.0 + 1.0;
    if (e == 1) return x;
    if (e == 2) return x * x;
    S xx = e > 0 ? x : 1.0 / x;
    S y = x * 0.0 + 1.0;
    for (int i = e; i != 0; i /= 2) {
        if (i % 2) y = y * xx;
        xx = xx * xx;
    }
    return y;
}
template <class S>
__device__ __forceinline__ S specie_pow_s(const S& x, int iexp, double sexp) {
    return iexp != kNoIntExp ? integer_pow_s(x, iexp) : pow(x, sexp);
}
template <class S>
__device__ __forceinline__ S specie_pow_m1_s(const S& x, int iexp, double sexp) {
    return iexp != kNoIntExp ? integer_pow_s(x, iexp - 1) : pow(x, sexp + (-1.0));
}

// th_Gstd / th_S_pstd of gf_device.cuh with T a generic scalar
template <class S>
__device__ __forceinline__ S th_Gstd_s(const Poly7& a, const S& T, const S& logT) {
    return ((a.a0 * (1.0 - logT) - (((a.a4 / 20.0 * T + a.a3 / 12.0) * T + a.a2 / 6.0) * T + a.a1 / 2.0) * T - a.a6) *
                T +
            a.a5);
}
template <class S>
__device__ __forceinline__ S th_S_pstd_s(const Poly7& a, const S& T, const S& logT) {
    return ((((a.a4 / 4.0 * T + a.a3 / 3.0) * T + a.a2 / 2.0) * T + a.a1) * T + a.a0 * logT + a.a6);
}

// Troe F of gf_device.cuh (gpuTroeFallOffFunction.H:27-47) for a generic scalar
template <class S>
__device__ __forceinline__ S troe_F_s(const DevMech& M, int q, const S& T, const S& invT, const S& Pr) {
    const double* tp = M.troe + 4 * q;
    const double alpha = ldg(tp), iTsss = ldg(tp + 1), iTs = ldg(tp + 2), Tss = ldg(tp + 3);
    constexpr double kInvLn10 = 0.43429448190325182765;
    constexpr double kLn10 = 2.30258509299404568402;
    const S logPr = (val(Pr) > kSmall ? log(Pr) : Pr * 0.0 + ::log(kSmall)) * kInvLn10;
    const S Fcent = (1.0 - alpha) * exp(-T * iTsss) + alpha * exp(-T * iTs) + exp(-Tss * invT);
    const S logFcent = (val(Fcent) > kSmall ? log(Fcent) : Fcent * 0.0 + ::log(kSmall)) * kInvLn10;
    const S c = -0.4 - 0.67 * logFcent;
    const S n = 0.75 - 1.27 * logFcent;
    const S x1 = n - 0.14 * (logPr + c);
    const S x2 = (logPr + c) / x1;
    const S x3 = 1.0 + x2 * x2;
    const S x4 = logFcent / x3;
    return exp(x4 * kLn10);
}

// The per-reaction vector-Jacobian product of the sweep. The quantities of
// reaction q that enter the right-hand side and the Jacobian, as
// stage_omega / stage_jacobian_params compute them, are omega; D[e] = kf dCf_e
// (lhs entry e < kSideInline) and kr dCr_e (rhs entry kSideInline + e), dC_e
// = e_e c_e^(e_e - 1) prod_{i != e} c_i^e_i in the reference's product order;
// dwdT; P = Ak (Cf - Cr/Kc) (third body). With the caller's weights (ob for
// omega, gD[e] for D[e], gT for dwdT, gE for P) this writes the gradient of
//   h = ob omega + sum_e gD[e] D[e] + gT dwdT + gE P
// w.r.t. the reaction's inputs to gr[]: the species entries (lhs 0 ..
// kSideInline-1, rhs kSideInline ..), then M, T, ln|A|, beta, Ta.
//   * M, T and the Arrhenius parameters enter through the rate constants and
//     the equilibrium constant: one forward-mode pass with those 5 directions
//     and the concentration products held as plain values; h collapses to
//     ob omega + wf kf + wr kr + gT dwdT + gE P with wf = sum_j gD[j] dCf_j
//     and wr = sum_j gD[kSideInline + j] dCr_j, so only a few dual values are
//     live at once.
//   * The concentrations enter only through the products C and dC_j: their
//     derivatives in closed form, with the second derivatives e (e - 1) c^(e - 2).
constexpr int kVjpK = 5;  // M, T, ln|A|, beta, Ta
__device__ __forceinline__ void rxn_vjp(const DevMech& M, int q, const Rxn& R, const double* c, double Mc_v,
                                        double T_v, double ob, const double* gD, double gT, double gE,
                                        double* gr) {
    using D = Dual<kVjpK>;
    const D Mc = dseed<kVjpK>(Mc_v, 0);
    const D T = dseed<kVjpK>(T_v, 1);
    const D lnA0 = dseed<kVjpK>(R.lnA0, 2), beta0 = dseed<kVjpK>(R.beta0, 3), Ta0 = dseed<kVjpK>(R.Ta0, 4);
    // concentration products: p = c^e, q1 = e c^(e-1) (as specie_pow_m1), q2 = e (e-1) c^(e-2)
    double p[2][kSideInline], q1[2][kSideInline], q2[2][kSideInline], Cs[2] = {1.0, 1.0};
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const int n = side ? R.nr : R.nl;
#pragma unroll
        for (int e = 0; e < kSideInline; ++e) {
            p[side][e] = 1.0;
            q1[side][e] = 1.0;
            q2[side][e] = 0.0;
            if (e < n) {
                const double x = c[side * kSideInline + e];
                const int ie = R.iexp[side][e];
                const double se = R.sexp[side][e];
                p[side][e] = specie_pow(x, ie, se);
                q1[side][e] = se * specie_pow_m1(x, ie, se);
                if (ie != kNoIntExp)
                    q2[side][e] = ie == 1 ? 0.0 : se * (se - 1.0) * integer_pow(x, ie - 2);
                else
                    q2[side][e] = se * (se - 1.0) * real_pow(x, se - 2.0);
                Cs[side] *= p[side][e];
            }
        }
    }
    double dC[2][kSideInline];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const int n = side ? R.nr : R.nl;
#pragma unroll
        for (int j = 0; j < kSideInline; ++j) {
            double d = 0.0;
            if (j < n) {
                d = 1.0;
#pragma unroll
                for (int i = 0; i < kSideInline; ++i)
                    if (i < n) d *= (i == j) ? q1[side][i] : p[side][i];
            }
            dC[side][j] = d;
        }
    }
    double wsum[2] = {0.0, 0.0};
#pragma unroll
    for (int side = 0; side < 2; ++side)
#pragma unroll
        for (int j = 0; j < kSideInline; ++j) wsum[side] += gD[side * kSideInline + j] * dC[side][j];
    // rate constants and the equilibrium constant over T, M and the parameters
    const D invT = 1.0 / T;
    const D logT = log(T);
    const D l0 = beta0 * logT + lnA0 - Ta0 * invT;
    D kf, ddT, Ak = dconst<kVjpK>(0.0);
    if (R.type == GF_RATE_ARRHENIUS) {
        Ak = R.sA0 * exp(l0);
        kf = Ak;
        ddT = Ak * ((beta0 + Ta0 * invT) * invT);
    } else if (R.type == GF_RATE_THIRD_BODY_ARRHENIUS) {
        Ak = R.sA0 * exp(l0);
        kf = Mc * Ak;
        ddT = Mc * (Ak * ((beta0 + Ta0 * invT) * invT));
    } else {
        const double b1 = ldg(M.beta1 + q), T1 = ldg(M.Ta1 + q), lA1 = ldg(M.lnA1 + q), s1 = ldg(M.sA1 + q);
        const D l1 = b1 * logT + lA1 - T1 * invT;
        const D kInf = s1 * exp(l1);
        const D Pr = ((R.sA0 * s1) * exp(l0 - l1)) * Mc;
        const D F = R.type == GF_RATE_TROE_FALLOFF ? troe_F_s(M, q, T, invT, Pr) : dconst<kVjpK>(1.0);
        const D temp = (Pr / (1.0 + Pr)) * F;
        kf = kInf * temp;
        ddT = (kInf * ((b1 + T1 * invT) * invT)) * temp;
    }
    const double Cf = Cs[0];
    const bool tb = R.type == GF_RATE_THIRD_BODY_ARRHENIUS;
    D h = (ob * Cf + wsum[0]) * kf + (gT * Cf) * ddT;
    double kr_v = 0.0, invKc_v = 1.0, dkrdT_v = 0.0;
    if (!R.irr) {
        const double Cr = Cs[1];
        const Poly7 a = reaction_coeffs_at(M, q, T_v, R.Tcommon);
        const D Gstd = th_Gstd_s(a, T, logT);
        const D arg = -R.Y * Gstd * invT * (1.0 / kRR);
        D lnK = arg.v < 600 ? arg : dconst<kVjpK>(0.5 * ::log(kVGreat));
        if (!R.nm_small) lnK = lnK + R.nm * log(kPstd / (kRR * T));
        const D invKc = exp(-lnK);
        D dK = (th_S_pstd_s(a, T, logT) + Gstd * invT) * R.Y * invT * (1.0 / kRR);
        if (!R.nm_small) dK = dK - R.nm * invT;
        const D kr = kf * invKc;
        const D dkrdT = ddT * invKc - kr * dK;
        // omega -= Cr kr, dwdT -= Cr dkrdT, D[rhs] = kr dCr
        h = h + (wsum[1] - ob * Cr) * kr - (gT * Cr) * dkrdT;
        if (tb) h = h + gE * (Ak * (Cf - Cr * invKc));
        kr_v = kr.v;
        invKc_v = invKc.v;
        dkrdT_v = dkrdT.v;
    } else if (tb) {
        h = h + gE * (Ak * Cf);
    }
#pragma unroll
    for (int k = 0; k < kVjpK; ++k) gr[2 * kSideInline + k] = h.d[k];
    // the species entries, closed form
    const double kf_v = kf.v, ddT_v = ddT.v, Ak_v = Ak.v;
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const int n = side ? R.nr : R.nl;
        const bool on = !(side && R.irr);
        const double ks = side ? kr_v : kf_v;
        // d(ob omega + gT dwdT + gE P) per unit dC_k of this side
        const double wk = side ? -(ob * kr_v + gT * dkrdT_v + (tb ? gE * Ak_v * invKc_v : 0.0))
                               : ob * kf_v + gT * ddT_v + (tb ? gE * Ak_v : 0.0);
#pragma unroll
        for (int k = 0; k < kSideInline; ++k) {
            double g = 0.0;
            if (k < n && on) {
                // sum_j gD[j] d(dC_j)/dc_k
                double s2 = 0.0;
#pragma unroll
                for (int j = 0; j < kSideInline; ++j) {
                    if (j < n) {
                        double d = 1.0;
#pragma unroll
                        for (int i = 0; i < kSideInline; ++i) {
                            if (i < n) {
                                if (i == j && i == k)
                                    d *= q2[side][i];
                                else if (i == j || i == k)
                                    d *= q1[side][i];
                                else
                                    d *= p[side][i];
                            }
                        }
                        s2 += gD[side * kSideInline + j] * d;
                    }
                }
                g = wk * dC[side][k] + ks * s2;
            }
            gr[side * kSideInline + k] = g;
        }
    }
}

}  // namespace gf
