// Differentiation helpers of the discrete adjoint (gf_adjoint.cu): forward-mode
// dual numbers and the per-reaction quantities of the chemistry written once
// for a generic scalar, following the same formulas, in the same order, as the
// double-precision device code in gf_device.cuh (gpuReaction.H,
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

// The quantities of reaction q that enter the right-hand side and the
// Jacobian, as stage_omega / stage_jacobian_params compute them:
//   omega; D[e]: dCf/dc * kf of lhs entry e (e < kSideInline) and dCr/dc * kr of
//   rhs entry e (kSideInline + e); dwdT; P = Ak (Cf - Cr/Kc) (third body).
// Inputs: the concentrations of the reaction's species entries c[e], the
// third-body concentration Mc, T, and the k (or k0) Arrhenius parameters.
template <class S>
struct RxnVals {
    S omega, dwdT, P;
    S D[2 * kSideInline];
};

template <class S>
__device__ __forceinline__ void rxn_eval(const DevMech& M, int q, const Rxn& R, const S* c, const S& Mc, const S& T,
                                         const S& lnA0, const S& beta0, const S& Ta0, RxnVals<S>& out) {
    const S invT = 1.0 / T;
    const S logT = log(T);
    const S lx = log(kPstd / (kRR * T));
    const S l0 = beta0 * logT + lnA0 - Ta0 * invT;
    S kf, ddT, Ak = T * 0.0;
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
        const S l1 = b1 * logT + lA1 - T1 * invT;
        const S kInf = s1 * exp(l1);
        const S Pr = ((R.sA0 * s1) * exp(l0 - l1)) * Mc;
        const S F = R.type == GF_RATE_TROE_FALLOFF ? troe_F_s(M, q, T, invT, Pr) : T * 0.0 + 1.0;
        const S temp = (Pr / (1.0 + Pr)) * F;
        kf = kInf * temp;
        ddT = (kInf * ((b1 + T1 * invT) * invT)) * temp;
    }
    // sides
    S Cf = T * 0.0 + 1.0, Cr = T * 0.0 + 1.0;
    S pw[2][kSideInline], dm[2][kSideInline];
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const int n = side ? R.nr : R.nl;
#pragma unroll
        for (int e = 0; e < kSideInline; ++e) {
            pw[side][e] = T * 0.0 + 1.0;
            dm[side][e] = T * 0.0 + 1.0;
            if (e < n) {
                const S& x = c[side * kSideInline + e];
                pw[side][e] = specie_pow_s(x, R.iexp[side][e], R.sexp[side][e]);
                dm[side][e] = R.sexp[side][e] * specie_pow_m1_s(x, R.iexp[side][e], R.sexp[side][e]);
            }
        }
    }
#pragma unroll
    for (int e = 0; e < kSideInline; ++e)
        if (e < R.nl) Cf = Cf * pw[0][e];
    S omega = Cf * kf;
    S dwdT = Cf * ddT;
    S invKc = T * 0.0 + 1.0, kr = T * 0.0;
    if (!R.irr) {
        const Poly7 a = reaction_coeffs_at(M, q, val(T), R.Tcommon);
        const S Gstd = th_Gstd_s(a, T, logT);
        const S arg = -R.Y * Gstd * invT * (1.0 / kRR);
        S lnK = val(arg) < 600 ? arg : T * 0.0 + 0.5 * ::log(kVGreat);
        if (!R.nm_small) lnK = lnK + R.nm * lx;
        invKc = exp(-lnK);
        S dK = (th_S_pstd_s(a, T, logT) + Gstd * invT) * R.Y * invT * (1.0 / kRR);
        if (!R.nm_small) dK = dK - R.nm * invT;
        kr = kf * invKc;
#pragma unroll
        for (int e = 0; e < kSideInline; ++e)
            if (e < R.nr) Cr = Cr * pw[1][e];
        const S dkrdT = ddT * invKc - kr * dK;
        dwdT = dwdT - Cr * dkrdT;
        omega = omega - Cr * kr;
    } else {
        Cr = T * 0.0;
    }
#pragma unroll
    for (int side = 0; side < 2; ++side) {
        const int n = side ? R.nr : R.nl;
#pragma unroll
        for (int j = 0; j < kSideInline; ++j) {
            S d = T * 0.0 + 1.0;
            if (j < n) {
#pragma unroll
                for (int i = 0; i < kSideInline; ++i)
                    if (i < n) d = d * ((i == j) ? dm[side][i] : pw[side][i]);
                d = d * (side ? kr : kf);
            } else {
                d = T * 0.0;
            }
            out.D[side * kSideInline + j] = d;
        }
    }
    if (R.irr) {
#pragma unroll
        for (int j = 0; j < kSideInline; ++j) out.D[kSideInline + j] = T * 0.0;
    }
    out.omega = omega;
    out.dwdT = dwdT;
    out.P = R.type == GF_RATE_THIRD_BODY_ARRHENIUS ? Ak * (Cf - Cr * invKc) : T * 0.0;
}

}  // namespace gf
