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
// one accumulator per translation unit (each has its own device module)
static __device__ unsigned long long g_phase_cycles[20];
// adds this translation unit's accumulators to out[20], optionally clearing them
static inline int phase_cycles_local(unsigned long long* out, int reset) {
    unsigned long long v[20];
    cudaMemcpyFromSymbol(v, g_phase_cycles, sizeof(v));
    for (int i = 0; i < 20; ++i) out[i] += v[i];
    if (reset) {
        unsigned long long z[20] = {};
        cudaMemcpyToSymbol(g_phase_cycles, z, sizeof(z));
    }
    return (int)cudaGetLastError();
}
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
       PH_ADJ_RXN, PH_ATTEMPT, PH_ADJ_RECOMPUTE, PH_ADJ_TSOLVE, PH_ADJ_VJP, PH_ADJ_JTERM, PH_LU_PANEL, PH_LU_U12,
       PH_LU_TRAIL, PH_LU_PERM };

// Unroll depths of two latency-bound loops: third-body rows whose loads are in
// flight together (third_body_all) and gather-stream records per batch
// (stream_gather). 4 each: measured faster on the B200 than 8 (more loads in
// flight, but more code to fetch inside the solve kernel) and than 2.
#ifndef GF_TB_ROWS
#define GF_TB_ROWS 4
#endif
#ifndef GF_GATHER_BATCH
#define GF_GATHER_BATCH 4
#endif

// ---------------------------------------------------------------- groups

// Cross-warp reduction buffer of a multi-warp group (one group per CTA).
__device__ __forceinline__ double* grp_red_buf() {
    __shared__ double buf[8];
    return buf;
}

// G <= 32: G aligned lanes of one warp, several groups per warp/CTA.
// G = 64, 96, 128, 256: the whole CTA (one cell per CTA); barriers are
// __syncthreads and reductions go through a small shared buffer, in a fixed
// warp order (deterministic).
template <int G>
struct Grp {
    static constexpr int W = G > 32 ? G / 32 : 1;  // warps in the group
    int lane;
    unsigned mask;
    __device__ __forceinline__ int warp() const { return G > 32 ? lane >> 5 : 0; }  // warp in the group
    __device__ __forceinline__ Grp() {
        const int wl = threadIdx.x & 31;
        if constexpr (G >= 32) {
            lane = G > 32 ? (int)threadIdx.x : wl;
            mask = 0xffffffffu;
        } else {
            lane = wl & (G - 1);
            mask = ((1u << G) - 1u) << (wl & ~(G - 1));
        }
    }
    __device__ __forceinline__ void sync() const {
        if (G > 32)
            __syncthreads();
        else if (G > 1)
            __syncwarp(mask);
    }
    __device__ __forceinline__ long long bcast_ll(long long v, int src) const {
        if (G == 1) return v;
        if (G > 32) {
            long long* b = reinterpret_cast<long long*>(grp_red_buf());
            __syncthreads();
            if (lane == src) b[0] = v;
            __syncthreads();
            v = b[0];
            __syncthreads();
            return v;
        }
        return __shfl_sync(mask, v, src, G);
    }
    __device__ __forceinline__ double sum(double v) const {
        constexpr int L = G > 32 ? 32 : G;
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(mask, v, o, L);
        if (G > 32) {
            double* b = grp_red_buf();
            if ((threadIdx.x & 31) == 0) b[lane >> 5] = v;
            __syncthreads();
            v = b[0];
#pragma unroll
            for (int k = 1; k < W; ++k) v += b[k];
            __syncthreads();
        }
        return v;
    }
    // max with fmax semantics: a NaN operand is ignored (normaliseError.H:22)
    __device__ __forceinline__ double fmax_(double v) const {
        constexpr int L = G > 32 ? 32 : G;
#pragma unroll
        for (int o = L / 2; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(mask, v, o, L));
        if (G > 32) {
            double* b = grp_red_buf();
            if ((threadIdx.x & 31) == 0) b[lane >> 5] = v;
            __syncthreads();
            v = b[0];
#pragma unroll
            for (int k = 1; k < W; ++k) v = fmax(v, b[k]);
            __syncthreads();
        }
        return v;
    }
    __device__ __forceinline__ int any(int p) const {
        if (G == 1) return p;
        if (G > 32) return __syncthreads_or(p) != 0;
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

// A reaction's packed data (RxnHead) and the species entries of both sides,
// requested with independent 16-byte loads before any of them is used.
struct Rxn {
    int type, irr, slot, tb_row, nl, nr, sp_off, nm_small;
    double lnA0, beta0, Ta0, sA0, Tcommon, Y, nm;
    int idx[2][kSideInline], iexp[2][kSideInline];
    double sexp[2][kSideInline];
};

__device__ __forceinline__ void load_rxn(const DevMech& M, int q, Rxn& R) {
    const int4* h = reinterpret_cast<const int4*>(M.rxh + q);
    const int4 h0 = __ldg(h), h1 = __ldg(h + 1);
    const double2* hd = reinterpret_cast<const double2*>(M.rxh + q) + 2;
    const double2 d0 = __ldg(hd), d1 = __ldg(hd + 1);
    const int4* sp = reinterpret_cast<const int4*>(M.rxs + (size_t)q * 2 * kSideInline);
    int4 v[2 * kSideInline];
#pragma unroll
    for (int e = 0; e < 2 * kSideInline; ++e) v[e] = __ldg(sp + e);
    R.type = h0.x;
    R.irr = h0.y;
    R.slot = h0.z;
    R.tb_row = h0.w;
    R.nl = h1.x;
    R.nr = h1.y;
    R.sp_off = h1.z;
    R.nm_small = h1.w;
    R.lnA0 = d0.x;
    R.beta0 = d0.y;
    R.Ta0 = d1.x;
    R.sA0 = d1.y;
    const double2 d2 = __ldg(hd + 2);
    R.Tcommon = d2.x;
    R.Y = d2.y;
    R.nm = __ldg(reinterpret_cast<const double*>(hd + 3));
#pragma unroll
    for (int e = 0; e < 2 * kSideInline; ++e) {
        R.idx[e / kSideInline][e % kSideInline] = v[e].x;
        R.iexp[e / kSideInline][e % kSideInline] = v[e].y;
        R.sexp[e / kSideInline][e % kSideInline] = __hiloint2double(v[e].w, v[e].z);
    }
}

__device__ __forceinline__ Poly7 reaction_coeffs_at(const DevMech& M, int r, double T, double Tcommon) {
    const int b = coef_branch(T, Tcommon);
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
__device__ __forceinline__ double reaction_lnKc(const DevMech& M, int q, const Rxn& R, const TCache& tc,
                                                double* Gstd_out, Poly7* a_out) {
    const Poly7 a = reaction_coeffs_at(M, q, tc.T, R.Tcommon);
    const double Gstd = th_Gstd(a, tc.T, tc.logT);
    const double arg = -R.Y * Gstd * tc.invT * (1.0 / kRR);
    double lnK = arg < 600 ? arg : 0.5 * log(kVGreat);
    if (!R.nm_small) lnK += R.nm * tc.lx;
    if (Gstd_out) *Gstd_out = Gstd;
    if (a_out) *a_out = a;
    return lnK;
}

// dKc/dT / Kc (gpuThermo.H:160-166)
__device__ __forceinline__ double reaction_dKcdTbyKc(const Rxn& R, const TCache& tc, double Gstd, const Poly7& a) {
    const double S = th_S_pstd(a, tc.T, tc.logT);
    double ret = (S + Gstd * tc.invT) * R.Y * tc.invT * (1.0 / kRR);
    if (!R.nm_small) ret = ret - R.nm * tc.invT;
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
// x^e for a non-integer exponent (rare: most mechanisms have integer
// exponents only), out of line: the many call sites share one copy of the
// math library's pow, which keeps the solve's instruction footprint smaller.
static __device__ __noinline__ double real_pow(double x, double e) { return pow(x, e); }
// gpuSpecieExponent.H:103-110
__device__ __forceinline__ double specie_pow(double x, int iexp, double sexp) {
    return iexp != kNoIntExp ? integer_pow(x, iexp) : real_pow(x, sexp);
}
// speciePow(c, e - 1) (gpuReaction.H:418-420 with gpuSpecieExponent::operator-)
__device__ __forceinline__ double specie_pow_m1(double x, int iexp, double sexp) {
    return iexp != kNoIntExp ? integer_pow(x, iexp - 1) : real_pow(x, sexp + (-1.0));
}

// ln|k| of an Arrhenius factor: k (or the fall-off k0) from the reaction's
// head, kInf from the fall-off tables; and dln(k)/dT = (beta + Ta/T)/T
__device__ __forceinline__ double arr_ln0(const Rxn& R, const TCache& tc) {
    return fma(R.beta0, tc.logT, R.lnA0) - R.Ta0 * tc.invT;
}
__device__ __forceinline__ double arr_ln1(const DevMech& M, int q, const TCache& tc) {
    return fma(ldg(M.beta1 + q), tc.logT, ldg(M.lnA1 + q)) - ldg(M.Ta1 + q) * tc.invT;
}
__device__ __forceinline__ double arr_dlnkdT0(const Rxn& R, const TCache& tc) {
    return (R.beta0 + R.Ta0 * tc.invT) * tc.invT;
}
__device__ __forceinline__ double arr_dlnkdT1(const DevMech& M, int q, const TCache& tc) {
    return (ldg(M.beta1 + q) + ldg(M.Ta1 + q) * tc.invT) * tc.invT;
}

// Third-body concentrations M_t = sum_i eff_ti c_i of every third-body and
// fall-off reaction (gpuThirdBodyEfficiencies.H:28-35), written to Mtb[t]:
// lanes over species (coalesced rows of eff), warps over reactions, rows in
// batches of GF_TB_ROWS so that their loads are in flight together; each sum is
// lane-strided and combined by a fixed shuffle tree (deterministic; the
// reference sums sequentially, an ulp-level reordering).
template <int G, class W>
__device__ __forceinline__ void third_body_all(const Grp<G>& g, const DevMech& M, const W& w, int c_off, int m_off) {
    constexpr int LW = G > 32 ? 32 : G;
    constexpr int NW = G > 32 ? G / 32 : 1;
    constexpr int RB = GF_TB_ROWS;
    constexpr int SPL = 3;  // species per lane held at once: nS <= SPL * LW, else looped
    const int rg = G > 32 ? (g.lane >> 5) : 0;
    const int rl = G > 32 ? (g.lane & 31) : g.lane;
    const unsigned mask = G > 32 ? 0xffffffffu : g.mask;
    const int nS = M.nS;
    for (int t0 = rg * RB; t0 < M.n_tb; t0 += NW * RB) {
        double sum[RB];
        if (nS <= SPL * LW) {
            double cv[SPL];
#pragma unroll
            for (int k = 0; k < SPL; ++k) {
                const int i = rl + k * LW;
                cv[k] = i < nS ? w[c_off + i] : 0.0;
            }
            double e[RB][SPL];
#pragma unroll
            for (int b = 0; b < RB; ++b)
#pragma unroll
                for (int k = 0; k < SPL; ++k) {
                    const int i = rl + k * LW;
                    e[b][k] = (t0 + b < M.n_tb && i < nS) ? ldg(M.eff + (size_t)(t0 + b) * nS + i) : 0.0;
                }
#pragma unroll
            for (int b = 0; b < RB; ++b) {
                double acc = 0.0;
#pragma unroll
                for (int k = 0; k < SPL; ++k) acc += e[b][k] * cv[k];
                sum[b] = acc;
            }
        } else {
#pragma unroll
            for (int b = 0; b < RB; ++b) {
                double acc = 0.0;
                if (t0 + b < M.n_tb)
                    for (int i = rl; i < nS; i += LW) acc += ldg(M.eff + (size_t)(t0 + b) * nS + i) * w[c_off + i];
                sum[b] = acc;
            }
        }
#pragma unroll
        for (int b = 0; b < RB; ++b) {
#pragma unroll
            for (int o = LW / 2; o > 0; o >>= 1) sum[b] += __shfl_xor_sync(mask, sum[b], o, LW);
            if (rl == 0 && t0 + b < M.n_tb) w[m_off + t0 + b] = sum[b];
        }
    }
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
// Mc: the reaction's third-body concentration (third_body_all), unused for
// plain Arrhenius rates.
__device__ __forceinline__ double rate_k(const DevMech& M, int q, const Rxn& R, const TCache& tc, double Mc,
                                         bool want_dT, double* dT_out, double* Ak_out) {
    const int type = R.type;
    if (type == GF_RATE_ARRHENIUS) {
        const double Ak = R.sA0 * exp(arr_ln0(R, tc));
        if (want_dT) *dT_out = Ak * arr_dlnkdT0(R, tc);
        return Ak;
    }
    if (type == GF_RATE_THIRD_BODY_ARRHENIUS) {
        const double Ak = R.sA0 * exp(arr_ln0(R, tc));
        if (want_dT) *dT_out = Mc * (Ak * arr_dlnkdT0(R, tc));
        *Ak_out = Ak;
        return Mc * Ak;
    }
    // fall-off: Pr = k0 / kInf * M, k = kInf Pr / (1 + Pr) F
    const double l0 = arr_ln0(R, tc), l1 = arr_ln1(M, q, tc);
    const double s0 = R.sA0, s1 = ldg(M.sA1 + q);
    const double kInf = s1 * exp(l1);
    const double Pr = (s0 * s1) * exp(l0 - l1) * Mc;
    const double F = type == GF_RATE_TROE_FALLOFF ? troe_F(M, q, tc, Pr) : 1.0;
    const double temp = (Pr / (1.0 + Pr)) * F;
    if (want_dT) *dT_out = (kInf * arr_dlnkdT1(M, q, tc)) * temp;
    return kInf * temp;
}

// ------------------------------------------------------------- layout

// Per-cell workspace layout. The solve kernels (sweep = false) keep Cp, v and
// rhoM/W, which only the Jacobian reads, in k2..k4 (the stage vectors, not yet
// written while the Jacobian is built), and have one pivot region: the solves
// follow either the pivots or their permutation (solve_layout places the other
// in k1, free until the first stage). The adjoint's sweep (sweep = true) needs
// both after the stages and gets separate regions.
__host__ __device__ inline WsLayout make_layout(int nS, int nR, int n_slots, int n_tb, bool sweep = false) {
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
    if (sweep) {
        L.perm = o; o += m;
    } else {
        L.perm = L.piv;
    }
    L.c = o; o += nS;
    L.Ha = o; o += nS;
    if (sweep) {
        L.Cp = o; o += nS;
        L.rhoMbyW = o; o += nS;
        L.vj = o; o += nS;
    } else {
        L.Cp = L.k2;
        L.vj = L.k3;
        L.rhoMbyW = L.k4;
    }
    L.stage = o; o += (n_slots > 0 ? n_slots : 1);
    L.Mtb = o; o += (n_tb > 0 ? n_tb : 1);
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
// for the Jacobian at the same state (same T and concentrations, hence the
// same values: the reference evaluates them twice), in the reaction's own
// staging slots 1..3 (every reaction has at least four: omega, dwdT and one
// term per side); only the Jacobian's parameters overwrite them, after reading.
template <int G, class W>
__device__ __forceinline__ void stage_omega(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L,
                                            const TCache& tc, bool write_cache) {
    for (int q = g.lane; q < M.nR; q += G) {
        Rxn R;
        load_rxn(M, q, R);
        const int so = R.slot;
        const double Mc = R.tb_row >= 0 ? w[L.Mtb + R.tb_row] : 0.0;
        double dummy, Ak = 0.0;
        const double kf = rate_k(M, q, R, tc, Mc, false, &dummy, &Ak);
        double kr = 0.0, invKc = 1.0;
        if (!R.irr) {
            invKc = exp(-reaction_lnKc(M, q, R, tc, nullptr, nullptr));
            kr = kf * invKc;
        }
        if (write_cache) {
            w[L.stage + so + 1] = kf;
            w[L.stage + so + 2] = invKc;
            w[L.stage + so + 3] = Ak;
        }
        const double Cf = side_C(M, w, L.c, R, 0);
        const double Cr = side_C(M, w, L.c, R, 1);
        w[L.stage + so] = kf * Cf - kr * Cr;
    }
    g.sync();
}

__host__ __device__ constexpr int log2_group(int G) { return G <= 1 ? 0 : 1 + log2_group(G / 2); }
// The index of a group size's gather streams in DevMech (group_size_of).
__host__ __device__ constexpr int stream_index(int G) { return G == 96 ? 9 : log2_group(G); }

// Runs this thread's share of a gather stream (gf_internal.h, Stream):
// dst[pos] = sum of coef * src[slot] over each entry's records, in order.
// Every record load is independent of the sums (coalesced 16-byte loads), so
// they pipeline; one thread owns each output entry (no barriers inside).
template <int G, class W>
__device__ __forceinline__ void stream_gather(const Grp<G>& g, const Stream& st, const W& w, int src, int dst) {
    constexpr int U = GF_GATHER_BATCH;  // records in flight per thread
    const int4* r = reinterpret_cast<const int4*>(st.rec) + g.lane;
    const int len = st.len;
    double acc = 0.0;
    for (int k0 = 0; k0 < len; k0 += U) {
        int4 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = (k0 + u < len) ? __ldg(r + (size_t)(k0 + u) * G) : make_int4(-1, -1, 0, 0);
        // the sources of the batch are read before any of its results is
        // stored (the source and destination regions are disjoint)
        double x[U];
#pragma unroll
        for (int u = 0; u < U; ++u) x[u] = v[u].y >= 0 ? w[src + v[u].y] : 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (v[u].y >= 0) acc += __hiloint2double(v[u].w, v[u].z) * x[u];
            if (v[u].x >= 0) {
                w[dst + v[u].x] = acc;
                acc = 0.0;
            }
        }
    }
}

// dN_s/dt gathered in the reference's order, scaled to dY/dt (gpuODESystem.H:40-48,
// 184-189), then dT/dt (:53-63). Writes out[0..m).
template <int G, class W>
__device__ __forceinline__ void gather_rhs(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L,
                                           int out_off, double rhoM, double CpM) {
    const int nS = M.nS;
    stream_gather(g, M.dst[stream_index(G)], w, L.stage, out_off);
    g.sync();
    double s_h = 0;
    for (int s = g.lane; s < nS; s += G) {
        const double acc = w[out_off + s] * (ldg(M.W + s) / rhoM);
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
        if (M.n_tb > 0) {
            third_body_all(g, M, w, L.c, L.Mtb);
            g.sync();
        }
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

// Product C = prod c^e of one side of a reaction (side 0: lhs, 1: rhs), in
// the reference's order (calcCf / calcCr, gpuReaction.H:372-386).
template <class W>
__device__ __forceinline__ double side_C(const DevMech& M, const W& w, int c_off, const Rxn& R, int side) {
    const int n = side ? R.nr : R.nl;
    double C = 1.0;
    if (n <= kSideInline) {
#pragma unroll
        for (int e = 0; e < kSideInline; ++e)
            if (e < n) C *= specie_pow(w[c_off + R.idx[side][e]], R.iexp[side][e], R.sexp[side][e]);
        return C;
    }
    const int b = R.sp_off + (side ? R.nl : 0);
    for (int e = 0; e < n; ++e)
        C *= specie_pow(w[c_off + ldg(M.sidx + b + e)], ldg(M.siexp + b + e), ldg(M.sexp + b + e));
    return C;
}

// One side of a reaction: returns C = prod c^e and writes kmul * dC/dc_j to
// out + j, each the product over i of e_i c_i^(e_i - 1) (i == j) or c_i^e_i
// (i != j) in the reference's order (calcdCfdcj / calcdCrdcj, :388-470). Up to
// kSideInline species the powers stay in registers; wider sides recompute
// them (the same values).
template <class W>
__device__ __forceinline__ double side_products(const DevMech& M, const W& w, int c_off, const Rxn& R, int side,
                                                double kmul, int out) {
    const int n = side ? R.nr : R.nl;
    if (n <= kSideInline) {
        double pw[kSideInline], dm[kSideInline];
#pragma unroll
        for (int e = 0; e < kSideInline; ++e) {
            pw[e] = 1.0;
            dm[e] = 1.0;
            if (e < n) {
                const double x = w[c_off + R.idx[side][e]];
                pw[e] = specie_pow(x, R.iexp[side][e], R.sexp[side][e]);
                dm[e] = R.sexp[side][e] * specie_pow_m1(x, R.iexp[side][e], R.sexp[side][e]);
            }
        }
        double C = 1.0;
#pragma unroll
        for (int e = 0; e < kSideInline; ++e)
            if (e < n) C *= pw[e];
#pragma unroll
        for (int j = 0; j < kSideInline; ++j) {
            if (j < n) {
                double d = 1;
#pragma unroll
                for (int i = 0; i < kSideInline; ++i)
                    if (i < n) d *= (i == j) ? dm[i] : pw[i];
                w[out + j] = d * kmul;
            }
        }
        return C;
    }
    const int b = R.sp_off + (side ? R.nl : 0);
    double C = 1.0;
    for (int e = 0; e < n; ++e)
        C *= specie_pow(w[c_off + ldg(M.sidx + b + e)], ldg(M.siexp + b + e), ldg(M.sexp + b + e));
    for (int j = 0; j < n; ++j) {
        double d = 1;
        for (int i = 0; i < n; ++i) {
            const double x = w[c_off + ldg(M.sidx + b + i)];
            const int ie = ldg(M.siexp + b + i);
            const double se = ldg(M.sexp + b + i);
            d *= (i == j) ? se * specie_pow_m1(x, ie, se) : specie_pow(x, ie, se);
        }
        w[out + j] = d * kmul;
    }
    return C;
}

// Per-reaction Jacobian parameters (computeReactionParameters, gpuReaction.H:650-702)
template <int G, class W>
__device__ __forceinline__ void stage_jacobian_params(const Grp<G>& g, const DevMech& M, const W& w,
                                                      const WsLayout& L, const TCache& tc, bool use_cache) {
    for (int q = g.lane; q < M.nR; q += G) {
        Rxn R;
        load_rxn(M, q, R);
        const int type = R.type;
        const int nl = R.nl;
        const int so = R.slot;
        double ddT = 0.0, Ak = 0.0, kf;
        double cachedInvKc = 0.0;
        if (use_cache) {
            // dk/dT = k dln(k)/dT with the kInf factor for fall-off rates
            // (gpuFallOffReactionRate.H:140-141)
            kf = w[L.stage + so + 1];
            cachedInvKc = w[L.stage + so + 2];
            Ak = w[L.stage + so + 3];
            const bool falloff = type == GF_RATE_LINDEMANN_FALLOFF || type == GF_RATE_TROE_FALLOFF;
            ddT = kf * (falloff ? arr_dlnkdT1(M, q, tc) : arr_dlnkdT0(R, tc));
        } else {
            kf = rate_k(M, q, R, tc, R.tb_row >= 0 ? w[L.Mtb + R.tb_row] : 0.0, true, &ddT, &Ak);
        }
        const double Cf = side_products(M, w, L.c, R, 0, kf, L.stage + so + 2);
        double dwdT = Cf * ddT;
        double omega = Cf * kf;
        double Cr = 0.0, invKc = 1.0;
        if (!R.irr) {
            double Gstd;
            Poly7 a;
            if (use_cache) {
                a = reaction_coeffs_at(M, q, tc.T, R.Tcommon);
                Gstd = th_Gstd(a, tc.T, tc.logT);
                invKc = cachedInvKc;
            } else {
                invKc = exp(-reaction_lnKc(M, q, R, tc, &Gstd, &a));
            }
            const double dKcdTbyKc = reaction_dKcdTbyKc(R, tc, Gstd, a);
            const double kr = kf * invKc;
            Cr = side_products(M, w, L.c, R, 1, kr, L.stage + so + 2 + nl);
            const double dkrdT = ddT * invKc - kr * dKcdTbyKc;
            dwdT -= Cr * dkrdT;
            omega -= Cr * kr;
        }
        w[L.stage + so] = omega;
        w[L.stage + so + 1] = dwdT;
        if (type == GF_RATE_THIRD_BODY_ARRHENIUS) w[L.stage + so + 2 + nl + R.nr] = Ak * (Cf - Cr * invKc);
    }
    g.sync();
}

// gpuODESystem::jacobian (gpuODESystem.H:198-281): dfdx (entries 0..nS) and J
// (m x m, Y and T rows/columns; the p row/column are zero).
//   raw entries (gather stream, one thread per entry): dN/dc, T-column and
//     third-body terms in the reference's order per entry;
//   phase 3 (lanes over rows): ddY_dcdY (gpuODESystem.H:65-103);
//   then the T row (ddT_dtdY, ddT_dtdT, :108-146).
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
        if (!use_cache && M.n_tb > 0) {
            third_body_all(g, M, w, L.c, L.Mtb);
            g.sync();
        }
        stage_jacobian_params(g, M, w, L, tc, use_cache);
        GF_PH_END(g, PH_JPARAMS)
    }
    // the staging slots that held the cache now hold the Jacobian terms
    if (allow_cache && g.lane == 0) w[L.scal + S_KCACHE_T] = -1.0;
    {
        GF_PH_BEGIN(g)
        gather_rhs(g, M, w, L, L.dfdx, rhoM, CpM);
        GF_PH_END(g, PH_GATHER_RHS)
    }
    {
    GF_PH_BEGIN(g)
    // raw dN/dc, T-column and third-body terms of every entry (species rows x
    // species and T columns), one thread per entry, in the reference's order
    stream_gather(g, M.jst[stream_index(G)], w, L.stage, L.J);
    g.sync();
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

// One elimination update a - l * u. The solve kernels contract it to one FMA
// (EXACT = false); EXACT = true rounds the product and the difference
// separately, as the reference's CPU build (no contraction) computes the Crout
// sums of ludecompose.H:36-55, so that parity kernels can compare factors bit
// for bit.
template <bool EXACT>
__device__ __forceinline__ double msub(double a, double l, double u) {
    if constexpr (EXACT)
        return __dsub_rn(a, __dmul_rn(l, u));
    else
        return fma(-l, u, a);
}

// LUDecompose (ludecompose.H:9-92) in right-looking form: at step k the pivot
// column holds exactly the Crout sums of the reference, the pivot is the last
// row with the largest vv*|a| (">=", :62), full rows are swapped, a zero pivot
// becomes gpuSmall and the column below is scaled by 1/pivot. Every entry
// receives its updates in the same k order as the reference's Crout loops.
template <int G, bool EXACT = false, class W>
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
                for (int i = k + 1; i < m; ++i) w[A + i * ld + j] = msub<EXACT>(w[A + i * ld + j], w[A + i * ld + k], ukj);
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
// Panel steps k0 .. k1-1 of the blocked LU (a group of at most one warp):
// pivot search, row exchange, zero-pivot fix, column scaling and the update of
// the panel's remaining columns.
template <int G, bool EXACT = false, class W>
__device__ __forceinline__ void lu_panel(const Grp<G>& g, const W& w, int A, int ld, int piv, int vv, int m, int k0,
                                         int k1) {
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
                for (int j = k + 1; j < k1; ++j) w[A + i * ld + j] = msub<EXACT>(w[A + i * ld + j], lik, w[A + k * ld + j]);
            }
            g.sync();
        }
    }
}

// Panel steps k0 .. k1-1 with the panel held in registers (one full warp):
// register slot (lane l, r) holds a panel row (initially row k0 + l + 32 r)
// with its row scaling, and a label: the row position it has in the
// reference's matrix after the exchanges so far. An exchange of rows k and
// iMax swaps the two slots' labels instead of moving data; the pivot search,
// its tie-break ("last max wins" by position), the update condition and the
// write-back all go by label. The row scaling stays with its data, which is
// the reference's vv[iMax] = vv[k] (ludecompose.H:71-78); the scaling left at
// position k is never read again. The pivot search reduces across lanes with
// three integer warp reductions on order-preserving keys of the non-negative
// candidates (high word, low word, then the largest position). Same
// operations, in the same order per entry, as lu_panel. The pivots go to
// piv[]; the exchanges of the columns outside the panel are left to
// lu_apply_swaps. Difference: when every candidate of a column is NaN, the
// reference exchanges row k with row 0 (its iMax starts at 0); here none is.
template <int RP, int NB, bool EXACT = false, class W>
__device__ __forceinline__ void lu_panel_reg(const Grp<32>& g, const W& w, int A, int ld, int piv, int vv, int m,
                                             int k0, int k1) {
    const int l = g.lane;
    const int kb = k1 - k0;
    double a[RP][NB];
    double sv[RP];
    int lab[RP];
#pragma unroll
    for (int r = 0; r < RP; ++r) {
        const int p = k0 + l + 32 * r;
        lab[r] = p < m ? p : m;  // slots past the last row never qualify
#pragma unroll
        for (int t = 0; t < NB; ++t) a[r][t] = (p < m && t < kb) ? w[A + p * ld + k0 + t] : 0.0;
        sv[r] = p < m ? w[vv + p] : 0.0;
    }
#pragma unroll
    for (int kk = 0; kk < NB; ++kk) {
        if (kk >= kb) break;
        const int k = k0 + kk;
        // pivot search: the last position with the largest vv * |a| (ludecompose.H:57-63)
        double best = -1.0;
        int bi = -1;
#pragma unroll
        for (int r = 0; r < RP; ++r) {
            if (lab[r] >= k && lab[r] < m) {
                const double t = sv[r] * fabs(a[r][kk]);
                if (t > best || (t == best && lab[r] > bi)) {
                    best = t;
                    bi = lab[r];
                }
            }
        }
        const bool has = bi >= 0;
        const unsigned hi = has ? (unsigned)__double2hiint(best) : 0u;
        const unsigned lo = has ? (unsigned)__double2loint(best) : 0u;
        const unsigned mh = __reduce_max_sync(0xffffffffu, hi);
        const unsigned ml = __reduce_max_sync(0xffffffffu, hi == mh ? lo : 0u);
        const int mr =
            (int)__reduce_max_sync(0xffffffffu, (has && hi == mh && lo == ml) ? (unsigned)(bi + 1) : 0u) - 1;
        const int iMax = mr < 0 ? k : mr;
        // the slot that holds position iMax becomes position k, and the slot
        // that held position k becomes iMax
        int ri = -1;
#pragma unroll
        for (int r = 0; r < RP; ++r)
            if (lab[r] == iMax) ri = r;
        const unsigned own = __ballot_sync(0xffffffffu, ri >= 0);
        const int li = __ffs(own) - 1;
        ri = __shfl_sync(0xffffffffu, ri, li);
        if (iMax != k) {
#pragma unroll
            for (int r = 0; r < RP; ++r) {
                if (lab[r] == k)
                    lab[r] = iMax;
                else if (lab[r] == iMax)
                    lab[r] = k;
            }
        }
        if (l == 0) w.ip(piv + k) = iMax;
        // pivot row (now position k), broadcast; a zero pivot becomes gpuSmall (:81)
        double urow[NB];
#pragma unroll
        for (int t = 0; t < NB; ++t) {
            double x = a[0][t];
#pragma unroll
            for (int r = 1; r < RP; ++r)
                if (r == ri) x = a[r][t];
            urow[t] = (t >= kk && t < kb) ? __shfl_sync(0xffffffffu, x, li) : 0.0;
        }
        if (urow[kk] == 0.0) {
            urow[kk] = kSmall;
#pragma unroll
            for (int r = 0; r < RP; ++r)
                if (l == li && r == ri) a[r][kk] = kSmall;
        }
        if (k != m - 1) {
            const double rDiag = 1.0 / urow[kk];
#pragma unroll
            for (int r = 0; r < RP; ++r) {
                if (lab[r] > k && lab[r] < m) {
                    const double lik = a[r][kk] * rDiag;
                    a[r][kk] = lik;
#pragma unroll
                    for (int t = kk + 1; t < NB; ++t)
                        if (t < kb) a[r][t] = msub<EXACT>(a[r][t], lik, urow[t]);
                }
            }
        }
    }
#pragma unroll
    for (int r = 0; r < RP; ++r) {
        if (lab[r] < m) {
#pragma unroll
            for (int t = 0; t < NB; ++t)
                if (t < kb) w[A + lab[r] * ld + k0 + t] = a[r][t];
            w[vv + lab[r]] = sv[r];
        }
    }
}

// The row exchanges of panel steps k0 .. k1-1 (pivots in piv[]) applied in
// order to one column j outside the panel.
template <class W>
__device__ __forceinline__ void lu_apply_swaps(const W& w, int A, int ld, int piv, int k0, int k1, int j) {
    for (int k = k0; k < k1; ++k) {
        const int iMax = w.ip(piv + k);
        if (iMax != k) {
            const double t = w[A + k * ld + j];
            w[A + k * ld + j] = w[A + iMax * ld + j];
            w[A + iMax * ld + j] = t;
        }
    }
}

// Register-panel form of the blocked LU for a full warp or a multi-warp group
// (m <= 32 RP, RP panel rows per lane): warp 0 factors each panel in registers; every column outside the
// panel takes the panel's row exchanges, then (columns right of the panel) its
// U12 rows; then the trailing matrix is updated (lanes over columns, warps over
// rows). Every entry receives its updates in k order, as in lu_decompose.
template <int G, int NB, bool EXACT = false, int RP = 2, class W>
__device__ __forceinline__ void lu_decompose_regpanel(const Grp<G>& g, const W& w, int A, int ld, int piv, int vv,
                                                      int m) {
    constexpr int NWp = G > 32 ? G / 32 : 1;
    const int wid = g.warp();
    const int l = G > 32 ? (int)(threadIdx.x & 31) : g.lane;
    for (int k0 = 0; k0 < m; ) {
        const int kb = min(NB, m - k0);
        const int k1 = k0 + kb;
        {
            GF_PH_BEGIN(g)
            if (wid == 0) {
                Grp<32> g32;
                lu_panel_reg<RP, NB, EXACT>(g32, w, A, ld, piv, vv, m, k0, k1);
            }
            g.sync();
            GF_PH_END(g, PH_LU_PANEL)
        }
        {
            GF_PH_BEGIN(g)
            // row exchanges outside the panel, and U12 of the columns right of it
            for (int j = g.lane; j < m - kb; j += G) {
                const int jj = j < k0 ? j : j + kb;
                lu_apply_swaps(w, A, ld, piv, k0, k1, jj);
                if (jj >= k1) {
                    double u[NB];
#pragma unroll
                    for (int t = 0; t < NB; ++t) u[t] = t < kb ? w[A + (k0 + t) * ld + jj] : 0.0;
#pragma unroll
                    for (int t = 1; t < NB; ++t) {
                        if (t < kb) {
                            double v = u[t];
#pragma unroll
                            for (int t2 = 0; t2 < t; ++t2) v = msub<EXACT>(v, w[A + (k0 + t) * ld + k0 + t2], u[t2]);
                            u[t] = v;
                            w[A + (k0 + t) * ld + jj] = v;
                        }
                    }
                }
            }
            g.sync();
            GF_PH_END(g, PH_LU_U12)
        }
        if (k1 >= m) break;
        {
            GF_PH_BEGIN(g)
            for (int j = k1 + l; j < m; j += 32) {
                double u[NB];
#pragma unroll
                for (int t = 0; t < NB; ++t) u[t] = t < kb ? w[A + (k0 + t) * ld + j] : 0.0;
                for (int i = k1 + wid; i < m; i += NWp) {
                    double a = w[A + i * ld + j];
#pragma unroll
                    for (int t = 0; t < NB; ++t)
                        if (t < kb) a = msub<EXACT>(a, w[A + i * ld + k0 + t], u[t]);
                    w[A + i * ld + j] = a;
                }
            }
            g.sync();
            GF_PH_END(g, PH_LU_TRAIL)
        }
        k0 = k1;
    }
}

template <int G, int NB, bool EXACT = false, class W>
__device__ __forceinline__ void lu_decompose_blocked(const Grp<G>& g, const W& w, int A, int ld, int piv, int vv,
                                                     int m) {
    if constexpr (G > 32) {
        // multi-warp group: warp 0 factors each panel; the U12 rows and the
        // trailing matrix are updated by all warps (lanes over columns, warps
        // over rows), each entry still receiving its updates in k order
        constexpr int NWp = G / 32;
        const int wid = g.warp(), l = threadIdx.x & 31;
        for (int k0 = 0; k0 < m; k0 += NB) {
            const int kb = min(NB, m - k0);
            const int k1 = k0 + kb;
            if (wid == 0) {
                Grp<32> g32;
                lu_panel<32, EXACT>(g32, w, A, ld, piv, vv, m, k0, k1);
            }
            __syncthreads();
            if (k1 >= m) break;
            for (int j = k1 + g.lane; j < m; j += G) {
                for (int t = 1; t < kb; ++t) {
                    double v = w[A + (k0 + t) * ld + j];
                    for (int t2 = 0; t2 < t; ++t2)
                        v = msub<EXACT>(v, w[A + (k0 + t) * ld + k0 + t2], w[A + (k0 + t2) * ld + j]);
                    w[A + (k0 + t) * ld + j] = v;
                }
            }
            __syncthreads();
            for (int j = k1 + l; j < m; j += 32) {
                double u[NB];
#pragma unroll
                for (int t = 0; t < NB; ++t) u[t] = t < kb ? w[A + (k0 + t) * ld + j] : 0.0;
                for (int i = k1 + wid; i < m; i += NWp) {
                    double a = w[A + i * ld + j];
#pragma unroll
                    for (int t = 0; t < NB; ++t)
                        if (t < kb) a = msub<EXACT>(a, w[A + i * ld + k0 + t], u[t]);
                    w[A + i * ld + j] = a;
                }
            }
            __syncthreads();
        }
    } else {
    for (int k0 = 0; k0 < m; k0 += NB) {
        const int kb = min(NB, m - k0);
        const int k1 = k0 + kb;
        // 1. panel: columns [k0, k1), rows [k0, m)
        lu_panel<G, EXACT>(g, w, A, ld, piv, vv, m, k0, k1);
        if (k1 >= m) break;
        // 2. U12: rows [k0, k1), columns [k1, m)
        for (int j = k1 + g.lane; j < m; j += G) {
            double u[NB];
#pragma unroll
            for (int t = 0; t < NB; ++t) {
                if (t < kb) {
                    double v = w[A + (k0 + t) * ld + j];
                    for (int t2 = 0; t2 < t; ++t2) v = msub<EXACT>(v, w[A + (k0 + t) * ld + k0 + t2], u[t2]);
                    u[t] = v;
                    w[A + (k0 + t) * ld + j] = v;
                }
            }
            // 3. trailing update of this column: rows [k1, m)
            for (int i = k1; i < m; ++i) {
                double a = w[A + i * ld + j];
#pragma unroll
                for (int t = 0; t < NB; ++t)
                    if (t < kb) a = msub<EXACT>(a, w[A + i * ld + k0 + t], u[t]);
                w[A + i * ld + j] = a;
            }
        }
        g.sync();
    }
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
// A group of 32 or more threads computes each position's source in parallel
// (the exchanges undone in reverse order: the row at position p came from
// piv-exchange k applied to the source so far, k = m-1 .. 0); smaller groups
// run the exchanges in order on one thread. Both give the same permutation.
template <int G, class W>
__device__ __forceinline__ void lu_perm(const Grp<G>& g, const W& w, int piv, int perm, int m) {
    g.sync();
    if constexpr (G >= 32) {
        for (int p = g.lane; p < m; p += G) {
            int s = p;
            for (int k = m - 1; k >= 0; --k) {
                const int q = w.ip(piv + k);
                s = s == k ? q : (s == q ? k : s);
            }
            w.ip(perm + p) = s;
        }
    } else if (g.lane == 0) {
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
// Same subtraction order as lu_solve; the backward step multiplies by the
// reciprocal of the diagonal, rdiag[j] = 1 / U[j][j] (computed once per LU),
// instead of dividing (ulp-level).
constexpr int kRegRows = 160;

// Whether the solves of a group of G threads (lu_solve_any) take the row
// permutation as a gather list (perm) or follow the pivots step by step (piv).
template <int G>
__host__ __device__ constexpr bool solve_uses_perm(int m) {
    return (G >= 32 && m <= 64) || (G > 32 && m <= 128) || (G >= 16 && G <= 32 && m <= kRegRows);
}

// The solve kernels' layout for a group of G threads: the pivot array the
// solves do not read (written by the factorisation or by lu_perm, consumed
// before the first stage) goes to k1.
template <int G>
__host__ __device__ inline WsLayout solve_layout(int nS, int nR, int n_slots, int n_tb) {
    WsLayout L = make_layout(nS, nR, n_slots, n_tb);
    if (solve_uses_perm<G>(nS + 1))
        L.piv = L.k1;
    else
        L.perm = L.k1;
    return L;
}
template <int G, class W>
__device__ __forceinline__ void lu_solve_reg(const Grp<G>& g, const W& w, int A, int ld, int perm, int rdiag, int m,
                                             int b) {
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
                const double xj = __shfl_sync(g.mask, x[t], l, G) * w[rdiag + j];
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

// Register form for one full warp with R rows per lane (m <= 32 R): lane l
// holds rows l + 32 u. The steps run in tiles of 32, the step loop unrolled by
// kSolveUnroll (4: measured faster than 8, 16 and full unrolling, whose code
// costs more in instruction fetch inside the solve kernel than it saves), so
// the loads of later steps can be issued early (the loop stores nothing).
// Same operations and order as lu_solve_reg.
#ifndef GF_SOLVE_UNROLL
#define GF_SOLVE_UNROLL 4
#endif
constexpr int kSolveUnroll = GF_SOLVE_UNROLL;  // substitution steps unrolled together
template <int R, class W>
__device__ __forceinline__ void lu_solve_warp(const W& w, int A, int ld, int perm, int rdiag, int m, int b) {
    const int lane = threadIdx.x & 31;
    double x[R];
    bool in[R];
    __syncwarp();
#pragma unroll
    for (int u = 0; u < R; ++u) {
        const int i = u * 32 + lane;
        in[u] = i < m;
        x[u] = in[u] ? w[b + w.ip(perm + i)] : 0.0;
    }
    // forward substitution with the unit lower factor, column by column
#pragma unroll
    for (int t = 0; t < R; ++t) {
        if (32 * t >= m - 1) break;
#pragma unroll kSolveUnroll
        for (int l = 0; l < 32; ++l) {
            const int j = 32 * t + l;
            if (j >= m - 1) break;
            const double bj = __shfl_sync(0xffffffffu, x[t], l);
            if (lane > l && in[t]) x[t] -= w[A + (32 * t + lane) * ld + j] * bj;
#pragma unroll
            for (int u = t + 1; u < R; ++u)
                if (in[u]) x[u] -= w[A + (32 * u + lane) * ld + j] * bj;
        }
    }
    // backward substitution, descending columns, x_j = (...) * (1 / U[j][j])
#pragma unroll
    for (int t = R - 1; t >= 0; --t) {
        if (32 * t >= m) continue;
#pragma unroll kSolveUnroll
        for (int l = 31; l >= 0; --l) {
            const int j = 32 * t + l;
            if (j >= m) continue;
            const double xj = __shfl_sync(0xffffffffu, x[t], l) * w[rdiag + j];
            if (lane == l) x[t] = xj;
            if (lane < l) x[t] -= w[A + (32 * t + lane) * ld + j] * xj;
#pragma unroll
            for (int u = 0; u < t; ++u) x[u] -= w[A + (32 * u + lane) * ld + j] * xj;
        }
    }
#pragma unroll
    for (int u = 0; u < R; ++u)
        if (in[u]) w[b + 32 * u + lane] = x[u];
    __syncwarp();
}

// rdiag: 1 / diagonal of U, used by the register form (G >= 16).
template <int G, class W>
__device__ __forceinline__ void lu_solve_any(const Grp<G>& g, const W& w, int A, int ld, int piv, int perm, int rdiag,
                                             int m, int b) {
    if constexpr (G >= 32) {
        // the substitution chain is sequential: one warp (the cell's warp, or
        // warp 0 of a multi-warp group) runs it in registers
        if (m <= 64) {
            g.sync();
            GF_PH_BEGIN(g)
            if (G == 32 || g.lane < 32) lu_solve_warp<2>(w, A, ld, perm, rdiag, m, b);
            g.sync();
            GF_PH_END(g, PH_SOLVE)
            return;
        }
        if constexpr (G > 32) {
            // 64 < m <= 128 (the 100-species mechanism): four rows per lane,
            // instead of the shared-memory form with a barrier per step
            if (m <= 128) {
                g.sync();
                if (g.lane < 32) lu_solve_warp<4>(w, A, ld, perm, rdiag, m, b);
                g.sync();
                return;
            }
        }
    }
    if constexpr (G >= 16 && G <= 32) {
        if (m <= kRegRows) {
            lu_solve_reg(g, w, A, ld, perm, rdiag, m, b);
            return;
        }
    }
    lu_solve(g, w, A, ld, piv, m, b);
}

// The factorisation as the solve kernels run it, after the row scaling vv:
// the register-panel form for a full warp or a multi-warp group (m <= 64),
// the blocked form otherwise, both with panels of NB columns; then, for groups of 16 or more threads, the
// reciprocal pivots 1 / U[i][i] (written over vv, which is no longer needed)
// and the row permutation of the solves (lu_solve_any).
template <int G, bool EXACT = false, int NB = 8, class W>
__device__ __forceinline__ void lu_factor(const Grp<G>& g, const W& w, int A, int ld, int piv, int vv, int perm,
                                          int m) {
    {
        GF_PH_BEGIN(g)
        bool done = false;
        if constexpr (G >= 32) {
            if (m <= 64) {
                lu_decompose_regpanel<G, NB, EXACT>(g, w, A, ld, piv, vv, m);
                done = true;
            }
        }
        if (!done) lu_decompose_blocked<G, NB, EXACT>(g, w, A, ld, piv, vv, m);
        GF_PH_END(g, PH_LU)
    }
    if (G >= 16) {
        GF_PH_BEGIN(g)
        for (int i = g.lane; i < m; i += G) w[vv + i] = 1.0 / w[A + i * ld + i];
        lu_perm(g, w, piv, perm, m);
        GF_PH_END(g, PH_LU_PERM)
    }
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

// Stage coefficients by (uniform) stage index: a_ij of the derivative points
// (stages 1 and 2), c_ij of the right-hand sides and d_i.
__device__ __forceinline__ double ros_a(const RosCoeffs& C, int i, int j) {
    return i == 1 ? C.a21 : (j == 0 ? C.a31 : C.a32);
}
__device__ __forceinline__ double ros_c(const RosCoeffs& C, int i, int j) {
    if (i == 1) return C.c21;
    if (i == 2) return j == 0 ? C.c31 : C.c32;
    return j == 0 ? C.c41 : (j == 1 ? C.c42 : C.c43);
}
__device__ __forceinline__ double ros_d(const RosCoeffs& C, int i) {
    return i == 0 ? C.d1 : (i == 1 ? C.d2 : (i == 2 ? C.d3 : C.d4));
}

// I/(gamma dx) - J of the Jacobian in L.J, and its LU (gpuAdaptiveSolver.H:51-73).
template <int G, class W, int NB = 8>
__device__ __forceinline__ void shift_and_factor(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L,
                                                 const RosCoeffs& C, double dx) {
    const int m = M.m;
    const int ld = L.ld;
    {
        GF_PH_BEGIN(g)
        shift_and_scale(g, w, L.J, ld, L.vv, m, 1.0 / (C.gamma * dx));
        GF_PH_END(g, PH_SHIFT)
    }
    lu_factor<G, false, NB>(g, w, L.J, ld, L.piv, L.vv, L.perm, m);
}

// The Jacobian at y0, then shift_and_factor.
template <int G, class W, int NB = 8>
__device__ __forceinline__ void factor_step(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L,
                                            const RosCoeffs& C, int y0_off, double p, double dx) {
    jacobian(g, M, w, L, y0_off, p, true);
    shift_and_factor<G, W, NB>(g, M, w, L, C, dx);
}

// One attempt solve(y0, dydx0, dx, y) of gpuRosenbrock12/23/34 (their
// solve(y0, dydx0, dx, y, buffer)); returns the normalised error
// (normaliseError.H:6-29; the p entry contributes 0). y0 is at y0_off, the
// candidate is written to yt_off.
// SAVE (the adjoint sweep): the caller has factored the step (L.J holds the
// LU); the stage points are kept at save_y2 / save_y3 and f at them at
// save_f2 / save_f3.
// F0 (the solve kernel): the attempt also evaluates the step's f(y0) into
// dydx0 when first_deriv is set (the first attempt of a step), through the
// stage loop's derivative call: one call site, a smaller instruction
// footprint. Otherwise the caller provides dydx0.
template <int G, class W, bool SAVE = false, bool F0 = false, int NB = 8>
__device__ __forceinline__ double ros_attempt(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L, const RosCoeffs& C,
                              const OdeParams& o, int y0_off, int yt_off, double p, double dx, int save_y2 = -1,
                              int save_y3 = -1, bool first_deriv = false, int save_f2 = -1, int save_f3 = -1) {
    const int m = M.m;
    const int ld = L.ld;
    if constexpr (!F0 && !SAVE) factor_step<G, W, NB>(g, M, w, L, C, y0_off, p, dx);
    // stages: k_i solves (I/(gamma dx) - J) k_i = f_i + dx d_i dfdx + sum_j c_ij k_j / dx,
    // f_0 = f(y0), f_i = f(y0 + sum_j a_ij k_j) where the method takes a new
    // derivative (stage 1; stage 2 of Rosenbrock34), else the previous one.
    // One loop, so the solve and the derivative each have a single call site;
    // with F0, pass st = -1 evaluates f(y0) (first_deriv) and factors the step.
#pragma unroll 1
    for (int st = F0 ? -1 : 0; st < C.s; ++st) {
        const bool new_f = st < 0 ? first_deriv : (st == 1 || (st == 2 && C.s == 4));
        int at = y0_off, out = L.dydx0;
        if (st > 0 && new_f) {
            // the stage point (kept at save_y2 / save_y3 when asked: the adjoint sweep)
            const int pt = !SAVE ? yt_off : (st == 1 ? save_y2 : (st == 2 ? save_y3 : yt_off));
            for (int i = g.lane; i < m; i += G) {
                double v = w[y0_off + i];
                for (int j = 0; j < st; ++j) v += ros_a(C, st, j) * w[L.k1 + j * m + i];
                w[pt + i] = v;
            }
            at = pt;
            out = L.dydx;
        }
        if (new_f) derivatives(g, M, w, L, at, p, out, st < 0);
        if constexpr (SAVE) {
            if (st > 0 && new_f) {
                const int fs = st == 1 ? save_f2 : save_f3;
                for (int i = g.lane; i < m; i += G) w[fs + i] = w[L.dydx + i];
            }
        }
        if constexpr (F0) {
            if (st < 0) {
                factor_step<G, W, NB>(g, M, w, L, C, y0_off, p, dx);
                continue;
            }
        }
        const int ki = L.k1 + st * m;
        const int src = st == 0 ? L.dydx0 : L.dydx;
        const double dd = dx * ros_d(C, st);
        for (int i = g.lane; i < m; i += G) {
            double v = w[src + i] + dd * w[L.dfdx + i];
            if (st > 0) {
                double cs = ros_c(C, st, 0) * w[L.k1 + i];
                for (int j = 1; j < st; ++j) cs += ros_c(C, st, j) * w[L.k1 + j * m + i];
                v += cs / dx;
            }
            w[ki + i] = v;
        }
        lu_solve_any(g, w, L.J, ld, L.piv, L.perm, L.vv, m, ki);
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
// REC (the adjoint's forward pass): each accepted step's start state and
// size are recorded at rec (rec_cap steps at most, rec_ld doubles each).
template <int G, class W, bool REC = false, int NB = 8>
__device__ __forceinline__ int ode_solve(const Grp<G>& g, const DevMech& M, const W& w, const WsLayout& L, const OdeParams& o,
                         const RosCoeffs& C, double xStart, double xEnd, int* y_off, int* yt_off, double p,
                         double* dxTry, int* accepted, int* attempts, double* rec = nullptr, int rec_cap = 0,
                         int rec_ld = 0) {
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
        // adaptiveSolve's derivatives call before its retry loop
        // (gpuAdaptiveSolver.H:96): in the solve kernel, inside the first attempt
        if constexpr (REC) derivatives(g, M, w, L, *y_off, p, L.dydx0, true);
        do {
            GF_PH_BEGIN(g)
            err = ros_attempt<G, W, false, !REC, NB>(g, M, w, L, C, o, *y_off, *yt_off, p, dx, -1, -1, rejects == 0);
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
        if constexpr (REC) {
            // the accepted step's start state and size, for the adjoint sweep
            if (*accepted >= rec_cap) return GF_CELL_MAX_STEPS;
            double* r = rec + (size_t)(*accepted) * rec_ld;
            for (int i = g.lane; i < M.m; i += G) r[i] = w[*y_off + i];
            if (g.lane == 0) r[M.m] = dx;
        }
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
template <int G, class W, bool REC = false, int NB = 8>
__device__ __forceinline__ void process_cell_body(const Grp<G>& g, const DevMech& M, const W& w, const LaunchArgs& a,
                                                  int cell) {
    const WsLayout L = solve_layout<G>(M.nS, M.nR, M.n_slots, M.n_tb);
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
            double* rec = REC ? a.traj + (size_t)cell * a.traj_cap * a.traj_ld : nullptr;
            const int st = ode_solve<G, W, REC, NB>(g, M, w, L, a.ode, C, 0.0, dt, &y_off, &yt_off, p, &dxTry, &accepted,
                                                &attempts, rec, a.traj_cap, a.traj_ld);
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

// process_cell_body with the LU panel width NB and, for MS > 0, the matrix
// size m = MS (nS = MS - 1) fixed at compile time: the caller launches such a
// kernel only for mechanisms of that size, and the compiler then resolves the
// workspace offsets, loop bounds and tile predicates that depend on it.
template <int G, class W, bool REC = false, int NB = 8, int MS = 0>
__device__ __forceinline__ void process_cell(const Grp<G>& g, const DevMech& M, const W& w, const LaunchArgs& a,
                                             int cell) {
    if constexpr (MS == 0) {
        process_cell_body<G, W, REC, NB>(g, M, w, a, cell);
    } else {
        DevMech Ms = M;
        Ms.m = MS;
        Ms.nS = MS - 1;
        process_cell_body<G, W, REC, NB>(g, Ms, w, a, cell);
    }
}

}  // namespace gf
