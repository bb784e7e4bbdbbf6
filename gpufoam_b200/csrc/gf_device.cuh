// Device code of the per-cell chemistry path (sm_100a, FP64 on CUDA cores).
//
// One templated code path serves every launch form: a "group" of G threads
// (G = 1, 2, 4, 8, 16, 32, aligned inside a warp) integrates one cell. G = 1 is
// the reference's one-thread-per-cell model; G = 32 is a warp per cell with the
// cell's Jacobian/LU held in shared memory. Loops over species, reactions,
// rows and columns are strided over the group's lanes; everything that decides
// control flow (error norm, step size, status) is group-uniform.
//
// The arithmetic follows gpuFoam's device code (paths below are relative to
// gpu_chemistry/src/ of the reference): gpuThermo/gpuThermo.H,
// gpuReaction/*.H, gpuOde/gpuODESystem.H, ludecompose.H, gpuRosenbrock*.H,
// gpuAdaptiveSolver.H, gpuODESolverBase.H and
// gpuKernelEvaluator/singleCellSolver.H. Where the order of a floating-point
// reduction is changed for parallelism it is noted; those change results at
// the ulp level only.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "gf_internal.h"

namespace gf {

// gpu_utils/common/gpu_constants.H:13-82
constexpr double kRR = 6.02214e+26 * 1.38065e-23;
constexpr double kPstd = 1e5;
constexpr double kVSmall = 2.2250738585072014e-308;  // numeric_limits<double>::min()
constexpr double kSmall = 2.220446049250313e-16;     // numeric_limits<double>::epsilon()
constexpr double kVGreat = 1.7976931348623157e+308 / 10.0;
constexpr int kMaxRejects = 100000;  // rejected attempts within one substep

// ------------------------------------------------------- phase timers
// Built only with -DGF_PHASE_TIMERS (a profiling variant of the library):
// lane 0 of each group accumulates clock64() cycles per phase of the solve.
#ifdef GF_PHASE_TIMERS
__device__ unsigned long long g_phase_cycles[16];
#define GF_PH_BEGIN(g) \
    (g).sync();        \
    const long long _gf_ph0 = clock64();
#define GF_PH_END(g, k) \
    (g).sync();         \
    if ((g).lane == 0) atomicAdd(&g_phase_cycles[k], (unsigned long long)(clock64() - _gf_ph0));
#else
#define GF_PH_BEGIN(g)
#define GF_PH_END(g, k)
#endif
enum { PH_MIX = 0, PH_NMPOW, PH_OMEGA, PH_GATHER_RHS, PH_JPARAMS, PH_JROWS, PH_TROW, PH_SHIFT, PH_LU, PH_SOLVE,
       PH_VEC, PH_ATTEMPT, PH_CELL };

// ---------------------------------------------------------------- groups

template <int G>
struct Grp {
    int lane;
    unsigned mask;
    __device__ __forceinline__ Grp() {
        const int wl = threadIdx.x & 31;
        lane = wl & (G - 1);
        mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << (wl & ~(G - 1)));
    }
    __device__ __forceinline__ void sync() const {
        if (G > 1) __syncwarp(mask);
    }
    __device__ __forceinline__ double bcast(double v, int src) const {
        if (G == 1) return v;
        return __shfl_sync(mask, v, src, G);
    }
    __device__ __forceinline__ long long bcast_ll(long long v, int src) const {
        if (G == 1) return v;
        return __shfl_sync(mask, v, src, G);
    }
    __device__ __forceinline__ double sum(double v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, G);
        return v;
    }
    // max with fmax semantics: a NaN operand is ignored (normaliseError.H:22)
    __device__ __forceinline__ double fmax_(double v) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o, G));
        return v;
    }
    __device__ __forceinline__ int any(int p) const {
        if (G == 1) return p;
        return (__ballot_sync(mask, p) & mask) != 0;
    }
};

// ------------------------------------------------------------- workspace

// Contiguous per-cell workspace (shared memory, or a per-cell block in HBM).
struct WsC {
    double* p;
    __device__ __forceinline__ double& operator[](int i) const { return p[i]; }
    __device__ __forceinline__ int& ip(int i) const { return *reinterpret_cast<int*>(p + i); }
};
// Interleaved workspace: element i of a cell at p[i * s] (p already offset by
// the cell's slot), so that consecutive threads touch consecutive addresses.
struct WsS {
    double* p;
    long long s;
    __device__ __forceinline__ double& operator[](int i) const { return p[(long long)i * s]; }
    __device__ __forceinline__ int& ip(int i) const { return *reinterpret_cast<int*>(p + (long long)i * s); }
};

template <class T>
__device__ __forceinline__ T ldg(const T* p) {
    return __ldg(p);
}

// ------------------------------------------------------------ thermo

// JANAF coefficient set of species i at T (gpuThermo.H:29-32)
__device__ __forceinline__ int coef_branch(double T, double Tcommon) { return T < Tcommon ? 0 : 1; }

struct Poly7 {
    double a0, a1, a2, a3, a4, a5, a6;
};

__device__ __forceinline__ Poly7 species_coeffs(const DevMech& M, int i, double T) {
    const int b = coef_branch(T, ldg(M.Tcommon + i));
    const double* c = M.coef + (size_t)b * 7 * M.nS + i;
    Poly7 a;
    a.a0 = ldg(c);
    a.a1 = ldg(c + M.nS);
    a.a2 = ldg(c + 2 * M.nS);
    a.a3 = ldg(c + 3 * M.nS);
    a.a4 = ldg(c + 4 * M.nS);
    a.a5 = ldg(c + 5 * M.nS);
    a.a6 = ldg(c + 6 * M.nS);
    return a;
}

__device__ __forceinline__ Poly7 reaction_coeffs(const DevMech& M, int r, double T) {
    const int b = coef_branch(T, ldg(M.rTcommon + r));
    const double* c = M.rcoef + (size_t)b * 7 * M.nR + r;
    Poly7 a;
    a.a0 = ldg(c);
    a.a1 = ldg(c + M.nR);
    a.a2 = ldg(c + 2 * M.nR);
    a.a3 = ldg(c + 3 * M.nR);
    a.a4 = ldg(c + 4 * M.nR);
    a.a5 = ldg(c + 5 * M.nR);
    a.a6 = ldg(c + 6 * M.nR);
    return a;
}

// gpuThermo.H:177-184 (the perfect-gas Cp term is 0)
__device__ __forceinline__ double th_Cp(const Poly7& a, double T) {
    return ((((a.a4 * T + a.a3) * T + a.a2) * T + a.a1) * T + a.a0);
}
// gpuThermo.H:210-221
__device__ __forceinline__ double th_Ha(const Poly7& a, double T) {
    return (((((a.a4 / 5.0 * T + a.a3 / 4.0) * T + a.a2 / 3.0) * T + a.a1 / 2.0) * T + a.a0) * T + a.a5);
}
// gpuThermo.H:333-338
__device__ __forceinline__ double th_dCpdT(const Poly7& a, double T) {
    return (((4.0 * a.a4 * T + 3.0 * a.a3) * T + 2.0 * a.a2) * T + a.a1);
}
// gpuThermo.H:287-299
__device__ __forceinline__ double th_Gstd(const Poly7& a, double T, double logT) {
    return ((a.a0 * (1.0 - logT) - (((a.a4 / 20.0 * T + a.a3 / 12.0) * T + a.a2 / 6.0) * T + a.a1 / 2.0) * T - a.a6) *
                T +
            a.a5);
}
// gpuThermo.H:261-271 at p = pStd (the -R ln(p/pStd) term is zero there)
__device__ __forceinline__ double th_S_pstd(const Poly7& a, double T, double logT) {
    return ((((a.a4 / 4.0 * T + a.a3 / 3.0) * T + a.a2 / 2.0) * T + a.a1) * T + a.a0 * logT + a.a6);
}

// ------------------------------------------------------------ reactions
//
// Rate constants are evaluated in log space: k = sign(A) exp(ln|A| + beta ln T
// - Ta / T) (gpuArrheniusReactionRate.H:16-26 computes A * pow(T, beta) *
// exp(-Ta / T)), Kc = exp(lnK + nm ln(pStd / (RR T))) (gpuThermo.H:80-113,
// 139-169 compute exp and pow), the Troe function with exp/log instead of
// pow(10, .)/log10. The results differ from the reference at the level of a
// few ulp of the exponent argument (a relative 1e-14 for |arg| ~ 50), far
// inside the 1e-12 rate tolerance, and save the double-precision pow calls
// and divisions that dominate the reaction loops.

// temperature-dependent per-call quantities
struct TCache {
    double T, invT, logT, lx;  // lx = ln(pStd / (RR T))
};

__device__ __forceinline__ TCache make_tcache(double T) {
    TCache t;
    t.T = T;
    t.invT = 1.0 / T;
    t.logT = log(T);
    t.lx = log(kPstd / (kRR * T));
    return t;
}

// ln of the K part of Kc, capped as K() caps it (gpuThermo.H:84-85)
__device__ __forceinline__ double reaction_lnKc(const DevMech& M, int q, const TCache& tc, double* Gstd_out,
                                                Poly7* a_out) {
    const Poly7 a = reaction_coeffs(M, q, tc.T);
    const double Y = ldg(M.rY + q);
    const double Gstd = th_Gstd(a, tc.T, tc.logT);
    const double arg = -Y * Gstd * tc.invT * (1.0 / kRR);
    double lnK = arg < 600 ? arg : 0.5 * log(kVGreat);
    if (!ldg(M.rnm_small + q)) lnK += ldg(M.rnm + q) * tc.lx;
    if (Gstd_out) *Gstd_out = Gstd;
    if (a_out) *a_out = a;
    return lnK;
}

// dKc/dT / Kc (gpuThermo.H:160-166)
__device__ __forceinline__ double reaction_dKcdTbyKc(const DevMech& M, int q, const TCache& tc, double Gstd,
                                                     const Poly7& a) {
    const double S = th_S_pstd(a, tc.T, tc.logT);
    double ret = (S + Gstd * tc.invT) * ldg(M.rY + q) * tc.invT * (1.0 / kRR);
    if (!ldg(M.rnm_small + q)) ret = ret - ldg(M.rnm + q) * tc.invT;
    return ret;
}

// gpuSpecieExponent.H:21-36
__device__ __forceinline__ double integer_pow(double x, int e) {
    if (e == 0) return 1;
    if (e == 1) return x;
    if (e == 2) return x * x;
    double xx = e > 0 ? x : 1 / x;
    double y = 1;
    for (int i = e; i != 0; i /= 2) {
        if (i % 2) y *= xx;
        xx *= xx;
    }
    return y;
}
// gpuSpecieExponent.H:103-110
__device__ __forceinline__ double specie_pow(double x, int iexp, double sexp) {
    return iexp != kNoIntExp ? integer_pow(x, iexp) : pow(x, sexp);
}
// speciePow(c, e - 1) (gpuReaction.H:418-420 with gpuSpecieExponent::operator-)
__device__ __forceinline__ double specie_pow_m1(double x, int iexp, double sexp) {
    return iexp != kNoIntExp ? integer_pow(x, iexp - 1) : pow(x, sexp + (-1.0));
}

// ln|k| of Arrhenius factor f (0: k / k0, 1: kInf) and its sign
__device__ __forceinline__ double arr_ln(const DevMech& M, int q, int f, const TCache& tc) {
    const double lnA = ldg((f ? M.lnA1 : M.lnA0) + q);
    const double beta = ldg((f ? M.beta1 : M.beta0) + q);
    const double Ta = ldg((f ? M.Ta1 : M.Ta0) + q);
    return fma(beta, tc.logT, lnA) - Ta * tc.invT;
}
__device__ __forceinline__ double arr_dlnkdT(const DevMech& M, int q, int f, const TCache& tc) {
    const double beta = ldg((f ? M.beta1 : M.beta0) + q);
    const double Ta = ldg((f ? M.Ta1 : M.Ta0) + q);
    return (beta + Ta * tc.invT) * tc.invT;  // (beta + Ta/T)/T
}

// third-body concentration M = sum eff_i c_i (gpuThirdBodyEfficiencies.H:28-35)
// (species-major table: the lanes of a warp, each on its own reaction, read
// consecutive addresses; two partial sums for latency)
template <class W>
__device__ __forceinline__ double third_body_M(const DevMech& M, int q, const W& w, int c_off) {
    const double* e = M.eff_t + ldg(M.tb_row + q);
    const int st = M.n_tb;
    double s0 = 0, s1 = 0;
    int i = 0;
    for (; i + 1 < M.nS; i += 2) {
        s0 += ldg(e + (size_t)i * st) * w[c_off + i];
        s1 += ldg(e + (size_t)(i + 1) * st) * w[c_off + i + 1];
    }
    if (i < M.nS) s0 += ldg(e + (size_t)i * st) * w[c_off + i];
    return s0 + s1;
}

// Troe F (gpuTroeFallOffFunction.H:27-47); troe[] holds alpha, 1/T***, 1/T*, T**
__device__ __forceinline__ double troe_F(const DevMech& M, int q, const TCache& tc, double Pr) {
    const double* tp = M.troe + 4 * q;
    const double alpha = ldg(tp), iTsss = ldg(tp + 1), iTs = ldg(tp + 2), Tss = ldg(tp + 3);
    constexpr double kInvLn10 = 0.43429448190325182765;
    constexpr double kLn10 = 2.30258509299404568402;
    const double logPr = log(fmax(Pr, kSmall)) * kInvLn10;
    const double Fcent = (1.0 - alpha) * exp(-tc.T * iTsss) + alpha * exp(-tc.T * iTs) + exp(-Tss * tc.invT);
    const double logFcent = log(fmax(Fcent, kSmall)) * kInvLn10;
    const double c = -0.4 - 0.67 * logFcent;
    const double n = 0.75 - 1.27 * logFcent;
    const double x1 = n - 0.14 * (logPr + c);
    const double x2 = (logPr + c) / x1;
    const double x3 = 1.0 + x2 * x2;
    const double x4 = logFcent / x3;
    return exp(x4 * kLn10);
}

// Forward rate constant kf (operator(), gpuReactionRate.H:164-173); with
// want_dT also dkf/dT and, for third-body rates, the pure Arrhenius part Ak
// ("everything", gpuArrheniusReactionRate.H:97-107,
// gpuThirdBodyArrheniusReactionRate.H:105-121, gpuFallOffReactionRate.H:127-158).
template <class W>
__device__ __forceinline__ double rate_k(const DevMech& M, int q, int type, const TCache& tc, const W& w, int c_off,
                                         bool want_dT, double* dT_out, double* Ak_out) {
    if (type == GF_RATE_ARRHENIUS) {
        const double Ak = ldg(M.sA0 + q) * exp(arr_ln(M, q, 0, tc));
        if (want_dT) *dT_out = Ak * arr_dlnkdT(M, q, 0, tc);
        return Ak;
    }
    if (type == GF_RATE_THIRD_BODY_ARRHENIUS) {
        const double Ak = ldg(M.sA0 + q) * exp(arr_ln(M, q, 0, tc));
        const double Mc = third_body_M(M, q, w, c_off);
        if (want_dT) *dT_out = Mc * (Ak * arr_dlnkdT(M, q, 0, tc));
        *Ak_out = Ak;
        return Mc * Ak;
    }
    // fall-off: Pr = k0 / kInf * M, k = kInf Pr / (1 + Pr) F
    const double l0 = arr_ln(M, q, 0, tc), l1 = arr_ln(M, q, 1, tc);
    const double s0 = ldg(M.sA0 + q), s1 = ldg(M.sA1 + q);
    const double kInf = s1 * exp(l1);
    const double Mc = third_body_M(M, q, w, c_off);
    const double Pr = (s0 * s1) * exp(l0 - l1) * Mc;
    const double F = type == GF_RATE_TROE_FALLOFF ? troe_F(M, q, tc, Pr) : 1.0;
    const double temp = (Pr / (1.0 + Pr)) * F;
    if (want_dT) *dT_out = (kInf * arr_dlnkdT(M, q, 1, tc)) * temp;
    return kInf * temp;
}

// ------------------------------------------------------------- layout

__host__ __device__ inline WsLayout make_layout(int nS, int nR, int n_slots) {
    WsLayout L;
    const int m = nS + 1;
    L.ld = m | 1;
    int o = 0;
    L.J = o;
    o += m * L.ld;
    L.y0 = o; o += m;
    L.yt = o; o += m;
    L.dydx0 = o; o += m;
    L.dydx = o; o += m;
    L.dfdx = o; o += m;
    L.k1 = o; o += m;
    L.k2 = o; o += m;
    L.k3 = o; o += m;
    L.k4 = o; o += m;
    L.vv = o; o += m;
    L.piv = o; o += m;
    L.perm = o; o += m;
    L.c = o; o += nS;
    L.Cp = o; o += nS;
    L.Ha = o; o += nS;
    L.rhoMbyW = o; o += nS;
    L.vj = o; o += nS;
    L.kcache = o; o += 3 * (nR > 0 ? nR : 1);
    L.stage = o; o += (n_slots > 0 ? n_slots : 1);
    L.scal = o; o += 8;
    L.size = o;
    return L;
}

// per-call scalars kept in the workspace scal[] block
enum { S_KCACHE_T = 0 };

// ------------------------------------------------------------ ODE system

// Mixture properties + concentrations (gpuMixture.H:33-121). The sums over
// species run lane-strided and are combined by a fixed shuffle tree
// (deterministic; the reference sums sequentially).
template <int G, class W>
__device__ __forceinline__ void mixture(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L, int y_off,
                                        double p, bool jac, double* rhoM_o, double* CpM_o, double* dCpMdT_o,
                                        double* alphav_o) {
    const int nS = M.nS;
    const double T = w[y_off + nS];
    const double invT = 1.0 / T;
    double s_rho = 0, s_cp = 0, s_dcp = 0, s_av = 0;
    for (int i = g.lane; i < nS; i += G) {
        const double yi = fmax(w[y_off + i], 0.0);
        const double rhoi = p / (ldg(M.Rsp + i) * T);
        const Poly7 a = species_coeffs(M, i, T);
        const double Cpi = th_Cp(a, T);
        const double Hai = th_Ha(a, T);
        s_rho += yi / rhoi;
        s_cp += yi * Cpi;
        w[L.Ha + i] = Hai;
        w[L.c + i] = yi / ldg(M.W + i);
        if (jac) {
            const double vi = 1.0 / rhoi;
            s_dcp += yi * th_dCpdT(a, T);
            s_av += yi * vi * invT;
            w[L.Cp + i] = Cpi;
            w[L.vj + i] = vi;
        }
    }
    const double rhoM = 1.0 / g.sum(s_rho);
    *rhoM_o = rhoM;
    *CpM_o = g.sum(s_cp);
    if (jac) {
        *dCpMdT_o = g.sum(s_dcp);
        *alphav_o = g.sum(s_av) * rhoM;
    }
    for (int i = g.lane; i < nS; i += G) {
        w[L.c + i] *= rhoM;
        if (jac) w[L.rhoMbyW + i] = rhoM / ldg(M.W + i);
    }
    g.sync();
}

// Net rate omega of every reaction at the clipped temperature (gpuReaction.H:472-488)
// With write_cache, kf, 1/Kc and the third-body Ak of every reaction are kept
// in kcache[] for the Jacobian at the same state (same T and concentrations,
// hence the same values: the reference evaluates them twice).
template <int G, class W>
__device__ __forceinline__ void stage_omega(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L,
                                            const TCache& tc, bool write_cache) {
    for (int q = g.lane; q < M.nR; q += G) {
        const int type = ldg(M.rtype + q);
        double dummy, Ak = 0.0;
        const double kf = rate_k(M, q, type, tc, w, L.c, false, &dummy, &Ak);
        double kr = 0.0, invKc = 1.0;
        if (!ldg(M.rirr + q)) {
            invKc = exp(-reaction_lnKc(M, q, tc, nullptr, nullptr));
            kr = kf * invKc;
        }
        if (write_cache) {
            w[L.kcache + 3 * q] = kf;
            w[L.kcache + 3 * q + 1] = invKc;
            w[L.kcache + 3 * q + 2] = Ak;
        }
        const int sp = ldg(M.sp_off + q);
        const int nl = ldg(M.nl + q), nr = ldg(M.nr + q);
        double Cf = 1.0, Cr = 1.0;
        for (int e = 0; e < nl; ++e)
            Cf *= specie_pow(w[L.c + ldg(M.sidx + sp + e)], ldg(M.siexp + sp + e), ldg(M.sexp + sp + e));
        for (int e = nl; e < nl + nr; ++e)
            Cr *= specie_pow(w[L.c + ldg(M.sidx + sp + e)], ldg(M.siexp + sp + e), ldg(M.sexp + sp + e));
        w[L.stage + ldg(M.slot + q)] = kf * Cf - kr * Cr;
    }
    g.sync();
}

// dN_s/dt gathered in the reference's order, scaled to dY/dt (gpuODESystem.H:40-48,
// 184-189), then dT/dt (:53-63). Writes out[0..m).
template <int G, class W>
__device__ __forceinline__ void gather_rhs(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L,
                                           int out_off, double rhoM, double CpM) {
    const int nS = M.nS;
    double s_h = 0;
    for (int s = g.lane; s < nS; s += G) {
        double acc = 0;
        const int e1 = ldg(M.dn_ptr + s + 1);
        for (int k = ldg(M.dn_ptr + s); k < e1; ++k) acc += ldg(M.dn_coef + k) * w[L.stage + ldg(M.dn_slot + k)];
        acc *= ldg(M.W + s) / rhoM;
        w[out_off + s] = acc;
        s_h += acc * w[L.Ha + s];
    }
    const double sh = g.sum(s_h);
    if (g.lane == 0) w[out_off + nS] = (-sh) / CpM;
    g.sync();
}

// gpuODESystem::derivatives (gpuODESystem.H:164-196): out = f(y), entries 0..nS
template <int G, class W>
__device__ __forceinline__ void derivatives(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L,
                                            int y_off, double p, int out_off, bool write_cache = false) {
    double rhoM, CpM, d0, d1;
    g.sync();
    {
        GF_PH_BEGIN(g)
        mixture(g, M, w, L, y_off, p, false, &rhoM, &CpM, &d0, &d1);
        GF_PH_END(g, PH_MIX)
    }
    const double T = w[y_off + M.nS];
    const double Tc = fmin(fmax(T, M.Tlow), M.Thigh);
    const TCache tc = make_tcache(Tc);
    // the Jacobian evaluates at the unclipped T: the cache serves it only when
    // the clip left T unchanged
    const bool cache_requested = write_cache;
    write_cache = write_cache && (Tc == T);
    {
        GF_PH_BEGIN(g)
        stage_omega(g, M, w, L, tc, write_cache);
        GF_PH_END(g, PH_OMEGA)
    }
    if (cache_requested && g.lane == 0) w[L.scal + S_KCACHE_T] = write_cache ? T : -1.0;
    {
        GF_PH_BEGIN(g)
        gather_rhs(g, M, w, L, out_off, rhoM, CpM);
        GF_PH_END(g, PH_GATHER_RHS)
    }
}

// Per-reaction Jacobian parameters (computeReactionParameters, gpuReaction.H:650-702)
template <int G, class W>
__device__ __forceinline__ void stage_jacobian_params(const Grp<G>& g, const DevMech& M, const W& w,
                                                      const WsLayout& L, const TCache& tc, bool use_cache) {
    for (int q = g.lane; q < M.nR; q += G) {
        const int type = ldg(M.rtype + q);
        const int sp = ldg(M.sp_off + q);
        const int nl = ldg(M.nl + q), nr = ldg(M.nr + q);
        const int so = ldg(M.slot + q);
        double ddT = 0.0, Ak = 0.0, kf;
        double cachedInvKc = 0.0;
        if (use_cache) {
            // dk/dT = k dln(k)/dT with the kInf factor for fall-off rates
            // (gpuFallOffReactionRate.H:140-141)
            kf = w[L.kcache + 3 * q];
            cachedInvKc = w[L.kcache + 3 * q + 1];
            Ak = w[L.kcache + 3 * q + 2];
            const int f = (type == GF_RATE_LINDEMANN_FALLOFF || type == GF_RATE_TROE_FALLOFF) ? 1 : 0;
            ddT = kf * arr_dlnkdT(M, q, f, tc);
        } else {
            kf = rate_k(M, q, type, tc, w, L.c, true, &ddT, &Ak);
        }
        double lp[kMaxW];
        double Cf = 1.0;
        for (int e = 0; e < nl; ++e) {
            lp[e] = specie_pow(w[L.c + ldg(M.sidx + sp + e)], ldg(M.siexp + sp + e), ldg(M.sexp + sp + e));
            Cf *= lp[e];
        }
        for (int j = 0; j < nl; ++j) {
            double d = 1;
            for (int i = 0; i < nl; ++i) {
                if (i == j) {
                    d *= ldg(M.sexp + sp + i) *
                         specie_pow_m1(w[L.c + ldg(M.sidx + sp + i)], ldg(M.siexp + sp + i), ldg(M.sexp + sp + i));
                } else {
                    d *= lp[i];
                }
            }
            w[L.stage + so + 2 + j] = d * kf;
        }
        double dwdT = Cf * ddT;
        double omega = Cf * kf;
        double Cr = 0.0, invKc = 1.0;
        if (!ldg(M.rirr + q)) {
            double Gstd;
            Poly7 a;
            if (use_cache) {
                a = reaction_coeffs(M, q, tc.T);
                Gstd = th_Gstd(a, tc.T, tc.logT);
                invKc = cachedInvKc;
            } else {
                invKc = exp(-reaction_lnKc(M, q, tc, &Gstd, &a));
            }
            const double dKcdTbyKc = reaction_dKcdTbyKc(M, q, tc, Gstd, a);
            const double kr = kf * invKc;
            double rp[kMaxW];
            Cr = 1.0;
            for (int e = 0; e < nr; ++e) {
                rp[e] = specie_pow(w[L.c + ldg(M.sidx + sp + nl + e)], ldg(M.siexp + sp + nl + e),
                                   ldg(M.sexp + sp + nl + e));
                Cr *= rp[e];
            }
            const double dkrdT = ddT * invKc - kr * dKcdTbyKc;
            dwdT -= Cr * dkrdT;
            omega -= Cr * kr;
            for (int j = 0; j < nr; ++j) {
                double d = 1;
                for (int i = 0; i < nr; ++i) {
                    if (i == j) {
                        const int b = sp + nl + i;
                        d *= ldg(M.sexp + b) * specie_pow_m1(w[L.c + ldg(M.sidx + b)], ldg(M.siexp + b), ldg(M.sexp + b));
                    } else {
                        d *= rp[i];
                    }
                }
                w[L.stage + so + 2 + nl + j] = d * kr;
            }
        }
        w[L.stage + so] = omega;
        w[L.stage + so + 1] = dwdT;
        if (type == GF_RATE_THIRD_BODY_ARRHENIUS) {
            w[L.stage + so + 2 + nl + nr] = Ak;
            w[L.stage + so + 3 + nl + nr] = Cf - Cr * invKc;
        }
    }
    g.sync();
}

// gpuODESystem::jacobian (gpuODESystem.H:198-281): dfdx (entries 0..nS) and J
// (m x m, Y and T rows/columns; the p row/column are zero).
//   phase 1 (lanes over rows): raw dN/dc and T-column pair contributions;
//   phase 2 (lanes over columns): third-body dk/dc rows, reaction by reaction;
//   phase 3 (lanes over rows): ddY_dcdY (gpuODESystem.H:65-103);
//   then the T row (ddT_dtdY, ddT_dtdT, :108-146).
// Within an entry the pair terms keep the reference's order; third-body terms
// follow all pair terms of the entry (the reference interleaves them by
// reaction), an ulp-level reordering.
template <int G, class W>
__device__ __forceinline__ void jacobian(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L,
                                         int y_off, double p, bool allow_cache = false) {
    const int nS = M.nS;
    const int ld = L.ld;
    double rhoM, CpM, dCpMdT, alphav;
    g.sync();
    {
        GF_PH_BEGIN(g)
        mixture(g, M, w, L, y_off, p, true, &rhoM, &CpM, &dCpMdT, &alphav);
        GF_PH_END(g, PH_MIX)
    }
    const TCache tc = make_tcache(w[y_off + nS]);
    const bool use_cache = allow_cache && w[L.scal + S_KCACHE_T] == tc.T;
    {
        GF_PH_BEGIN(g)
        stage_jacobian_params(g, M, w, L, tc, use_cache);
        GF_PH_END(g, PH_JPARAMS)
    }
    {
        GF_PH_BEGIN(g)
        gather_rhs(g, M, w, L, L.dfdx, rhoM, CpM);
        GF_PH_END(g, PH_GATHER_RHS)
    }
    {
    GF_PH_BEGIN(g)
    // phase 1
    for (int s = g.lane; s < nS; s += G) {
        const int row = L.J + s * ld;
        for (int c = 0; c <= nS; ++c) w[row + c] = 0.0;
        const int e1 = ldg(M.jr_ptr + s + 1);
        for (int k = ldg(M.jr_ptr + s); k < e1; ++k) {
            const JrRec rec = M.jr[k];
            w[row + rec.col] += rec.coef * w[L.stage + rec.slot];
        }
    }
    g.sync();
    // phase 2
    for (int t = 0; t < M.n_tbt; ++t) {
        const int q = ldg(M.tbt_q + t);
        const int s = ldg(M.tbt_s + t);
        const double cf = ldg(M.tbt_coef + t);
        const int so = ldg(M.slot + q) + 2 + ldg(M.nl + q) + ldg(M.nr + q);
        const double Ak = w[L.stage + so], tmp = w[L.stage + so + 1];
        const double* e = M.eff + (size_t)ldg(M.tb_row + q) * nS;
        for (int c = g.lane; c < nS; c += G) w[L.J + s * ld + c] += cf * ((ldg(e + c) * Ak) * tmp);
        g.sync();
    }
    // phase 3
    for (int s = g.lane; s < nS; s += G) {
        const double WiByrhoM = ldg(M.W + s) / rhoM;
        const double dfs = w[L.dfdx + s];
        const int row = L.J + s * ld;
        double ddN = w[row + nS];
        for (int c = 0; c < nS; ++c) {
            const double raw = w[row + c];
            ddN -= raw * w[L.c + c] * alphav;
            w[row + c] = WiByrhoM * raw * w[L.rhoMbyW + c] + rhoM * w[L.vj + c] * dfs;
        }
        w[row + nS] = WiByrhoM * ddN + alphav * dfs;
    }
    g.sync();
    GF_PH_END(g, PH_JROWS)
    }
    GF_PH_BEGIN(g)
    // T row: ddT_dtdY (gpuODESystem.H:108-126)
    const double dTdt = w[L.dfdx + nS];
    for (int i = g.lane; i < nS; i += G) {
        double acc = 0.0;
        for (int j = 0; j < nS; ++j) acc -= w[L.J + j * ld + i] * w[L.Ha + j];
        acc -= w[L.Cp + i] * dTdt;
        w[L.J + nS * ld + i] = acc / CpM;
    }
    // ddT_dtdT (gpuODESystem.H:129-146)
    double s_tt = 0.0;
    for (int i = g.lane; i < nS; i += G) s_tt += w[L.dfdx + i] * w[L.Cp + i] + w[L.J + i * ld + nS] * w[L.Ha + i];
    const double stt = g.sum(s_tt);
    if (g.lane == 0) w[L.J + nS * ld + nS] = ((-stt) - dTdt * dCpMdT) / CpM;
    g.sync();
    GF_PH_END(g, PH_TROW)
}

// ------------------------------------------------------------------ LU

// a = -J + I/(gamma dx) (gpuAdaptiveSolver.H:51-73) and the implicit row
// scaling vv = 1/max|a_ij| of LUDecompose (ludecompose.H:9-21).
template <int G, class W>
__device__ __forceinline__ void shift_and_scale(const Grp<G>& g, const W& w, int A, int ld, int vv, int m,
                                                double diag) {
    for (int i = g.lane; i < m; i += G) {
        double mx = 0.0;
        for (int j = 0; j < m; ++j) {
            double v = -w[A + i * ld + j];
            if (j == i) v += diag;
            w[A + i * ld + j] = v;
            const double t = fabs(v);
            if (t > mx) mx = t;
        }
        w[vv + i] = 1.0 / mx;
    }
    g.sync();
}

template <int G, class W>
__device__ __forceinline__ void row_scale(const Grp<G>& g, const W& w, int A, int ld, int vv, int m) {
    for (int i = g.lane; i < m; i += G) {
        double mx = 0.0;
        for (int j = 0; j < m; ++j) {
            const double t = fabs(w[A + i * ld + j]);
            if (t > mx) mx = t;
        }
        w[vv + i] = 1.0 / mx;
    }
    g.sync();
}

// LUDecompose (ludecompose.H:9-92) in right-looking form: at step k the pivot
// column holds exactly the Crout sums of the reference, the pivot is the last
// row with the largest vv*|a| (">=", :62), full rows are swapped, a zero pivot
// becomes gpuSmall and the column below is scaled by 1/pivot. Every entry
// receives its updates in the same k order as the reference's Crout loops.
template <int G, class W>
__device__ __forceinline__ void lu_decompose(const Grp<G>& g, const W& w, int A, int ld, int piv, int vv, int m) {
    for (int k = 0; k < m; ++k) {
        // pivot search
        double best = -1.0;
        int bi = -1;
        for (int i = k + g.lane; i < m; i += G) {
            const double t = w[vv + i] * fabs(w[A + i * ld + k]);
            if (t >= best) {
                best = t;
                bi = i;
            }
        }
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) {
            const double ob = __shfl_xor_sync(g.mask, best, o, G);
            const int oi = __shfl_xor_sync(g.mask, bi, o, G);
            if (ob > best || (ob == best && oi > bi)) {
                best = ob;
                bi = oi;
            }
        }
        const int iMax = bi < 0 ? 0 : bi;
        if (iMax != k) {
            for (int j = g.lane; j < m; j += G) {
                const double t = w[A + k * ld + j];
                w[A + k * ld + j] = w[A + iMax * ld + j];
                w[A + iMax * ld + j] = t;
            }
        }
        g.sync();
        if (g.lane == 0) {
            w.ip(piv + k) = iMax;
            if (iMax != k) w[vv + iMax] = w[vv + k];
            if (w[A + k * ld + k] == 0.0) w[A + k * ld + k] = kSmall;
        }
        g.sync();
        if (k != m - 1) {
            const double rDiag = 1.0 / w[A + k * ld + k];
            for (int i = k + 1 + g.lane; i < m; i += G) w[A + i * ld + k] *= rDiag;
            g.sync();
            for (int j = k + 1 + g.lane; j < m; j += G) {
                const double ukj = w[A + k * ld + j];
                for (int i = k + 1; i < m; ++i) w[A + i * ld + j] -= w[A + i * ld + k] * ukj;
            }
            g.sync();
        }
    }
}

// Blocked form of lu_decompose (panels of NB columns). For every entry the
// sequence of updates is the same as in the unblocked loop (all steps k in
// ascending order; row exchanges move rows that have received the same
// updates), so the factors are identical; the trailing matrix receives NB
// updates per load/store instead of one.
template <int G, int NB, class W>
__device__ __forceinline__ void lu_decompose_blocked(const Grp<G>& g, const W& w, int A, int ld, int piv, int vv,
                                                     int m) {
    for (int k0 = 0; k0 < m; k0 += NB) {
        const int kb = min(NB, m - k0);
        const int k1 = k0 + kb;
        // 1. panel: columns [k0, k1), rows [k0, m)
        for (int k = k0; k < k1; ++k) {
            double best = -1.0;
            int bi = -1;
            for (int i = k + g.lane; i < m; i += G) {
                const double t = w[vv + i] * fabs(w[A + i * ld + k]);
                if (t >= best) {
                    best = t;
                    bi = i;
                }
            }
#pragma unroll
            for (int o = G / 2; o > 0; o >>= 1) {
                const double ob = __shfl_xor_sync(g.mask, best, o, G);
                const int oi = __shfl_xor_sync(g.mask, bi, o, G);
                if (ob > best || (ob == best && oi > bi)) {
                    best = ob;
                    bi = oi;
                }
            }
            const int iMax = bi < 0 ? 0 : bi;
            if (iMax != k) {
                for (int j = g.lane; j < m; j += G) {
                    const double t = w[A + k * ld + j];
                    w[A + k * ld + j] = w[A + iMax * ld + j];
                    w[A + iMax * ld + j] = t;
                }
            }
            g.sync();
            if (g.lane == 0) {
                w.ip(piv + k) = iMax;
                if (iMax != k) w[vv + iMax] = w[vv + k];
                if (w[A + k * ld + k] == 0.0) w[A + k * ld + k] = kSmall;
            }
            g.sync();
            if (k != m - 1) {
                const double rDiag = 1.0 / w[A + k * ld + k];
                for (int i = k + 1 + g.lane; i < m; i += G) {
                    const double lik = w[A + i * ld + k] * rDiag;
                    w[A + i * ld + k] = lik;
                    for (int j = k + 1; j < k1; ++j) w[A + i * ld + j] -= lik * w[A + k * ld + j];
                }
                g.sync();
            }
        }
        if (k1 >= m) break;
        // 2. U12: rows [k0, k1), columns [k1, m)
        for (int j = k1 + g.lane; j < m; j += G) {
            double u[NB];
#pragma unroll
            for (int t = 0; t < NB; ++t) {
                if (t < kb) {
                    double v = w[A + (k0 + t) * ld + j];
                    for (int t2 = 0; t2 < t; ++t2) v -= w[A + (k0 + t) * ld + k0 + t2] * u[t2];
                    u[t] = v;
                    w[A + (k0 + t) * ld + j] = v;
                }
            }
            // 3. trailing update of this column: rows [k1, m)
            for (int i = k1; i < m; ++i) {
                double a = w[A + i * ld + j];
#pragma unroll
                for (int t = 0; t < NB; ++t)
                    if (t < kb) a -= w[A + i * ld + k0 + t] * u[t];
                w[A + i * ld + j] = a;
            }
        }
        g.sync();
    }
}

// LUBacksubstitute (ludecompose.H:94-130): the row exchanges first (equivalent
// to the reference's on-the-fly exchange, which only moves untouched values),
// then column-oriented forward and backward substitution. Forward: same
// subtraction order as the reference; backward: descending column order
// (the reference sums ascending), an ulp-level difference.
template <int G, class W>
__device__ __forceinline__ void lu_solve(const Grp<G>& g, const W& w, int A, int ld, int piv, int m, int b) {
    GF_PH_BEGIN(g)
    g.sync();
    if (g.lane == 0) {
        for (int i = 0; i < m; ++i) {
            const int ip = w.ip(piv + i);
            if (ip != i) {
                const double t = w[b + ip];
                w[b + ip] = w[b + i];
                w[b + i] = t;
            }
        }
    }
    g.sync();
    for (int j = 0; j < m - 1; ++j) {
        const double bj = w[b + j];
        for (int i = j + 1 + g.lane; i < m; i += G) w[b + i] -= w[A + i * ld + j] * bj;
        g.sync();
    }
    for (int j = m - 1; j >= 0; --j) {
        const double xj = w[b + j] / w[A + j * ld + j];
        g.sync();
        if (g.lane == 0) w[b + j] = xj;
        for (int i = g.lane; i < j; i += G) w[b + i] -= w[A + i * ld + j] * xj;
        g.sync();
    }
    GF_PH_END(g, PH_SOLVE)
}

// The row permutation LUBacksubstitute applies to a right-hand side (its
// sequence of exchanges b[i] <-> b[piv[i]]) as one gather: rhs'[i] = b[perm[i]].
template <int G, class W>
__device__ __forceinline__ void lu_perm(const Grp<G>& g, const W& w, int piv, int perm, int m) {
    g.sync();
    if (g.lane == 0) {
        for (int i = 0; i < m; ++i) w.ip(perm + i) = i;
        for (int i = 0; i < m; ++i) {
            const int ip = w.ip(piv + i);
            if (ip != i) {
                const int t = w.ip(perm + i);
                w.ip(perm + i) = w.ip(perm + ip);
                w.ip(perm + ip) = t;
            }
        }
    }
    g.sync();
}

// LUBacksubstitute with the right-hand side in registers: lane l holds rows
// l, l + G, ...; the pivot value of each step is broadcast by a shuffle, so
// the substitution chain runs without shared-memory round trips or barriers.
// Same subtraction order as lu_solve.
constexpr int kRegRows = 160;
template <int G, class W>
__device__ __forceinline__ void lu_solve_reg(const Grp<G>& g, const W& w, int A, int ld, int perm, int m, int b) {
    constexpr int R = kRegRows / G;
    GF_PH_BEGIN(g)
    double x[R];
    g.sync();
#pragma unroll
    for (int t = 0; t < R; ++t) {
        const int i = t * G + g.lane;
        x[t] = i < m ? w[b + w.ip(perm + i)] : 0.0;
    }
    g.sync();
#pragma unroll
    for (int t = 0; t < R; ++t) {
        if (t * G < m - 1) {
            const int lmax = min(G, m - 1 - t * G);
            for (int l = 0; l < lmax; ++l) {
                const int j = t * G + l;
                const double bj = __shfl_sync(g.mask, x[t], l, G);
#pragma unroll
                for (int u = t; u < R; ++u) {
                    const int i = u * G + g.lane;
                    if (i > j && i < m) x[u] -= w[A + i * ld + j] * bj;
                }
            }
        }
    }
#pragma unroll
    for (int t = R - 1; t >= 0; --t) {
        if (t * G < m) {
            const int lmax = min(G, m - t * G);
            for (int l = lmax - 1; l >= 0; --l) {
                const int j = t * G + l;
                const double xj = __shfl_sync(g.mask, x[t], l, G) / w[A + j * ld + j];
                if (g.lane == l) x[t] = xj;
#pragma unroll
                for (int u = 0; u <= t; ++u) {
                    const int i = u * G + g.lane;
                    if (i < j) x[u] -= w[A + i * ld + j] * xj;
                }
            }
        }
    }
#pragma unroll
    for (int t = 0; t < R; ++t) {
        const int i = t * G + g.lane;
        if (i < m) w[b + i] = x[t];
    }
    g.sync();
    GF_PH_END(g, PH_SOLVE)
}

template <int G, class W>
__device__ __forceinline__ void lu_solve_any(const Grp<G>& g, const W& w, int A, int ld, int piv, int perm, int m,
                                             int b) {
    if constexpr (G >= 16) {
        if (m <= kRegRows) {
            lu_solve_reg(g, w, A, ld, perm, m, b);
            return;
        }
    }
    lu_solve(g, w, A, ld, piv, m, b);
}

// ------------------------------------------------------------- Rosenbrock

struct RosCoeffs {
    int s;  // stages with a linear solve
    double gamma, a21, a31, a32, c21, c31, c32, c41, c42, c43, b1, b2, b3, b4, e1, e2, e3, e4, d1, d2, d3, d4;
};

// gpuRosenbrock12.H:14-31, gpuRosenbrock23.H:13-37, gpuRosenbrock34.H:13-46
__device__ __forceinline__ RosCoeffs ros_coeffs(int solver) {
    RosCoeffs c = {};
    if (solver == GF_ROSENBROCK12) {
        const double gamma = 1.0 + 1.0 / 1.414213562373095;
        c.s = 2;
        c.gamma = gamma;
        c.a21 = 1.0 / gamma;
        c.c21 = -2.0 / gamma;
        c.b1 = (3.0 / 2.0) / gamma;
        c.b2 = (1.0 / 2.0) / gamma;
        c.e1 = c.b1 - 1.0 / gamma;
        c.e2 = c.b2;
        c.d1 = gamma;
        c.d2 = -gamma;
    } else if (solver == GF_ROSENBROCK23) {
        c.s = 3;
        c.a21 = 1;
        c.a31 = 1;
        c.a32 = 0;
        c.c21 = -1.0156171083877702091975600115545;
        c.c31 = 4.0759956452537699824805835358067;
        c.c32 = 9.2076794298330791242156818474003;
        c.b1 = 1;
        c.b2 = 6.1697947043828245592553615689730;
        c.b3 = -0.4277225654321857332623837380651;
        c.e1 = 0.5;
        c.e2 = -2.9079558716805469821718236208017;
        c.e3 = 0.2235406989781156962736090927619;
        c.gamma = 0.43586652150845899941601945119356;
        c.d1 = 0.43586652150845899941601945119356;
        c.d2 = 0.24291996454816804366592249683314;
        c.d3 = 2.1851380027664058511513169485832;
    } else {
        c.s = 4;
        c.a21 = 2.0;
        c.a31 = 48.0 / 25.0;
        c.a32 = 6.0 / 25.0;
        c.c21 = -8.0;
        c.c31 = 372.0 / 25.0;
        c.c32 = 12.0 / 5.0;
        c.c41 = -112.0 / 125.0;
        c.c42 = -54.0 / 125.0;
        c.c43 = -2.0 / 5.0;
        c.b1 = 19.0 / 9.0;
        c.b2 = 1.0 / 2.0;
        c.b3 = 25.0 / 108.0;
        c.b4 = 125.0 / 108.0;
        c.e1 = 34.0 / 108.0;
        c.e2 = 7.0 / 36.0;
        c.e3 = 0.0;
        c.e4 = 125.0 / 108.0;
        c.gamma = 1.0 / 2.0;
        c.d1 = 1.0 / 2.0;
        c.d2 = -3.0 / 2.0;
        c.d3 = 605.0 / 250.0;
        c.d4 = 29.0 / 250.0;
    }
    return c;
}

// One attempt solve(y0, dydx0, dx, y) of gpuRosenbrock12/23/34 (their
// solve(y0, dydx0, dx, y, buffer)); returns the normalised error
// (normaliseError.H:6-29; the p entry contributes 0). y0 is at y0_off, the
// candidate is written to yt_off.
template <int G, class W>
__device__ double ros_attempt(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L, const RosCoeffs& C,
                              const OdeParams& o, int y0_off, int yt_off, double p, double dx) {
    const int m = M.m;
    const int ld = L.ld;
    jacobian(g, M, w, L, y0_off, p, true);
    {
        GF_PH_BEGIN(g)
        shift_and_scale(g, w, L.J, ld, L.vv, m, 1.0 / (C.gamma * dx));
        GF_PH_END(g, PH_SHIFT)
    }
    {
        GF_PH_BEGIN(g)
        lu_decompose_blocked<G, 8>(g, w, L.J, ld, L.piv, L.vv, m);
        GF_PH_END(g, PH_LU)
    }
    if (G >= 16) lu_perm(g, w, L.piv, L.perm, m);
    for (int i = g.lane; i < m; i += G) w[L.k1 + i] = w[L.dydx0 + i] + dx * C.d1 * w[L.dfdx + i];
    lu_solve_any(g, w, L.J, ld, L.piv, L.perm, m, L.k1);
    for (int i = g.lane; i < m; i += G) w[yt_off + i] = w[y0_off + i] + C.a21 * w[L.k1 + i];
    derivatives(g, M, w, L, yt_off, p, L.dydx);
    for (int i = g.lane; i < m; i += G)
        w[L.k2 + i] = w[L.dydx + i] + dx * C.d2 * w[L.dfdx + i] + C.c21 * w[L.k1 + i] / dx;
    lu_solve_any(g, w, L.J, ld, L.piv, L.perm, m, L.k2);
    if (C.s >= 3) {
        if (C.s == 4) {
            for (int i = g.lane; i < m; i += G)
                w[yt_off + i] = w[y0_off + i] + C.a31 * w[L.k1 + i] + C.a32 * w[L.k2 + i];
            derivatives(g, M, w, L, yt_off, p, L.dydx);
        }
        for (int i = g.lane; i < m; i += G)
            w[L.k3 + i] = w[L.dydx + i] + dx * C.d3 * w[L.dfdx + i] + (C.c31 * w[L.k1 + i] + C.c32 * w[L.k2 + i]) / dx;
        lu_solve_any(g, w, L.J, ld, L.piv, L.perm, m, L.k3);
    }
    if (C.s == 4) {
        for (int i = g.lane; i < m; i += G)
            w[L.k4 + i] = w[L.dydx + i] + dx * C.d4 * w[L.dfdx + i] +
                          (C.c41 * w[L.k1 + i] + C.c42 * w[L.k2 + i] + C.c43 * w[L.k3 + i]) / dx;
        lu_solve_any(g, w, L.J, ld, L.piv, L.perm, m, L.k4);
    }
    double emax = 0.0;
    for (int i = g.lane; i < m; i += G) {
        const double y0i = w[y0_off + i];
        double yi, ei;
        if (C.s == 2) {
            yi = y0i + C.b1 * w[L.k1 + i] + C.b2 * w[L.k2 + i];
            ei = C.e1 * w[L.k1 + i] + C.e2 * w[L.k2 + i];
        } else if (C.s == 3) {
            yi = y0i + C.b1 * w[L.k1 + i] + C.b2 * w[L.k2 + i] + C.b3 * w[L.k3 + i];
            ei = C.e1 * w[L.k1 + i] + C.e2 * w[L.k2 + i] + C.e3 * w[L.k3 + i];
        } else {
            yi = y0i + C.b1 * w[L.k1 + i] + C.b2 * w[L.k2 + i] + C.b3 * w[L.k3 + i] + C.b4 * w[L.k4 + i];
            ei = C.e1 * w[L.k1 + i] + C.e2 * w[L.k2 + i] + C.e4 * w[L.k4 + i];
        }
        w[yt_off + i] = yi;
        const double tol = o.absTol + o.relTol * fmax(fabs(y0i), fabs(yi));
        emax = fmax(emax, fabs(ei) / tol);
    }
    const double err = g.fmax_(emax);
    g.sync();
    return err;
}

// ------------------------------------------------------------ cell driver

struct CellResult {
    int status;
    int accepted;
    int attempts;
    double dxTry;
};

// odeSolve (gpuODESolverBase.H:67-111) + adaptiveSolve (gpuAdaptiveSolver.H:83-134).
// The state lives at *y_off (swapped with *yt_off on acceptance). Returns a
// gf_cell_status. maxSteps exhausted: dxTry is left unchanged (the reference
// returns without writing it).
template <int G, class W>
__device__ int ode_solve(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L, const OdeParams& o,
                         const RosCoeffs& C, double xStart, double xEnd, int* y_off, int* yt_off, double p,
                         double* dxTry, int* accepted, int* attempts) {
    double step_dxTry = *dxTry;
    bool last = false;
    double x = xStart;
    const double inc_threshold = pow(o.maxScale / o.safeScale, -1.0 / o.alphaInc);
    for (int nStep = 0; nStep < o.maxSteps; nStep++) {
        const double dxTry0 = step_dxTry;
        if ((x + step_dxTry - xEnd) * (x + step_dxTry - xStart) > 0) {
            last = true;
            step_dxTry = xEnd - x;
        }
        double dx = step_dxTry;
        double err = 0.0;
        int rejects = 0;
        derivatives(g, M, w, L, *y_off, p, L.dydx0, true);
        do {
            GF_PH_BEGIN(g)
            err = ros_attempt(g, M, w, L, C, o, *y_off, *yt_off, p, dx);
            GF_PH_END(g, PH_ATTEMPT)
            ++*attempts;
            if (err > 1) {
                const double scale = fmax(o.safeScale * pow(err, -o.alphaDec), o.minScale);
                dx *= scale;
                // the reference traps here (gpuAdaptiveSolver.H:111-114); the cap
                // also ends the loop for step controls that never shrink dx
                if (dx < kVSmall || ++rejects > kMaxRejects) return GF_CELL_STEP_UNDERFLOW;
            }
        } while (err > 1.0);
        x += dx;
        const int t = *y_off;
        *y_off = *yt_off;
        *yt_off = t;
        if (err > inc_threshold) {
            step_dxTry = fmin(fmax(o.safeScale * pow(err, -o.alphaInc), o.minScale), o.maxScale) * dx;
        } else {
            step_dxTry = o.safeScale * o.maxScale * dx;
        }
        ++*accepted;
        if ((x - xEnd) * (xEnd - xStart) >= 0) {
            if (nStep > 0 && last) step_dxTry = dxTry0;
            *dxTry = step_dxTry;
            return GF_CELL_OK;
        }
    }
    return GF_CELL_MAX_STEPS;
}

// order-preserving key of a double for atomicMin
__device__ __forceinline__ unsigned long long dbl_key(double v) {
    const unsigned long long b = (unsigned long long)__double_as_longlong(v);
    return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}

// singleCellSolver::operator() (singleCellSolver.H:27-51) with the
// computeYNew / computeRR epilogue (gpuKernelEvaluator.cu:84-96) fused:
// RR, the min of deltaTChemNew before clamping, and the clamp.
template <int G, class W>
__device__ void process_cell(const Grp<G>& g, const DevMech& M, const W& w, const LaunchArgs& a, int cell) {
    const WsLayout L = make_layout(M.nS, M.nR, M.n_slots);
    const int nS = M.nS, m = M.m;
    const double* yin = a.Y0 + (size_t)cell * a.ld_y;
    int y_off = L.y0, yt_off = L.yt;
    for (int i = g.lane; i < m; i += G) w[y_off + i] = yin[i];
    const double p = yin[nS + 1];
    const double T0 = yin[nS];
    const double dT = a.deltaT_cell ? a.deltaT_cell[cell] : a.deltaT;
    double dxTry = a.deltaTChem[cell];
    int status = GF_CELL_OK, accepted = 0, attempts = 0;
    if (g.lane == 0) w[L.scal + S_KCACHE_T] = -1.0;
    g.sync();
    if (T0 > a.Treact) {
        const RosCoeffs C = ros_coeffs(a.ode.solver);
        double timeLeft = dT;
        while (timeLeft > kSmall) {
            const double dt = timeLeft;
            const int st = ode_solve(g, M, w, L, a.ode, C, 0.0, dt, &y_off, &yt_off, p, &dxTry, &accepted, &attempts);
            if (st != GF_CELL_OK && status == GF_CELL_OK) status = st;
            if (st == GF_CELL_STEP_UNDERFLOW) break;
            int bad = 0;
            for (int i = g.lane; i < m; i += G) {
                const double v = w[y_off + i];
                if (!isfinite(v)) bad = 1;
                if (i < nS) w[y_off + i] = fmax(0.0, v);
            }
            if (g.any(bad) && status == GF_CELL_OK) status = GF_CELL_NONFINITE;
            g.sync();
            timeLeft -= dt;
        }
    } else {
        dxTry = dT;
        status = GF_CELL_SKIPPED;
    }
    // outputs
    if (a.Ynew) {
        double* yo = a.Ynew + (size_t)cell * a.ld_y;
        for (int i = g.lane; i < m; i += G) yo[i] = w[y_off + i];
        if (g.lane == 0) yo[nS + 1] = p;
    }
    if (a.RR) {
        const double rho = a.rho[cell];
        double* rr = a.RR + (size_t)cell * a.ld_rr;
        for (int i = g.lane; i < nS; i += G) rr[i] = rho * (w[y_off + i] - yin[i]) / dT;
    }
    if (g.lane == 0) {
        a.deltaTChem[cell] = fmin(dxTry, a.deltaTChemMax);
        if (a.status) a.status[cell] = status;
        if (a.counters) {
            a.counters[2 * cell] = accepted;
            a.counters[2 * cell + 1] = attempts;
        }
    }
    // per-cell aggregates: min over cells before clamping, counters (queue[1..4])
    if (g.lane == 0) {
        atomicMin(a.queue + 1, dbl_key(dxTry));
        atomicAdd(a.queue + 2, (unsigned long long)accepted);
        atomicAdd(a.queue + 3, (unsigned long long)attempts);
        if (status != GF_CELL_OK && status != GF_CELL_SKIPPED) atomicAdd(a.queue + 4, 1ull);
    }
    g.sync();
}

}  // namespace gf
