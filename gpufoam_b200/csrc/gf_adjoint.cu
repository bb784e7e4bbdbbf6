// Discrete adjoint of the Rosenbrock integration (sm_100a, FP64).
//
// Forward: gf_solve_record runs the solve and records, per cell, the state at
// the start of every accepted step and its size (the step sequence is then
// frozen). Reverse: gf_adjoint sweeps the recorded steps backwards; each step
// is recomputed from its start state (Jacobian, LU, stages: recomputation
// instead of storing the stages) and its Rosenbrock map y1 = y0 + sum b_i k_i,
// (I/(gamma h) - J(y0)) k_i = f_i + h d_i dfdx + sum_j c_ij k_j / h, is
// differentiated exactly as computed (gpuRosenbrock12/23/34.H):
//   * stages in reverse: rbar_i = W^-T kbar_i with the same LU factors,
//     fbar_i += rbar_i, dfdx_bar += h d_i rbar_i, kbar_j += c_ij / h rbar_i, and
//     at a derivative point y_i = y0 + sum a_ij k_j the vector-Jacobian product
//     of f (ybar0 += (df/dy)^T fbar_i, kbar_j += a_ij (df/dy)^T fbar_i);
//   * Jbar = sum_i rbar_i k_i^T, pulled back through the T row, the dc/dY
//     conversion (gpuODESystem.H:65-146) and the raw per-reaction terms of the
//     Jacobian as the reference computes them (so the reference's
//     approximations of the Jacobian, e.g. fall-off rates without their
//     concentration dependence, are differentiated as they stand);
//   * dfdx = f(y0) (the reference fills dfdx with the derivatives,
//     gpuODESystem.H:198-281), so its adjoint joins f's at y0.
// Per-reaction derivatives w.r.t. the reaction's inputs (its species'
// concentrations, the third-body concentration, T and the k (or k0) Arrhenius
// parameters ln|A|, beta, Ta): closed forms for the omega-only products of
// Arrhenius and third-body reactions, otherwise rxn_vjp (the concentrations in
// closed form, T, M and the parameters by 5-direction dual numbers); the
// mixture, conversion and T-row parts are reversed by hand.
// The loss gradient w.r.t. the final states comes in as Ybar; out come the
// gradients w.r.t. the initial states (Y, T) and, summed over the sweep, per
// reaction w.r.t. (ln|A|, beta, Ta) of its k (k0 for fall-off) rate.
// Assumptions: T stays inside the reactions' temperature limits (the rates
// are not clipped), sides have at most kSideInline species, and one
// odeSolve call covers the flow step (no maxSteps exhaustion).
#include <cuda_runtime.h>

#include <algorithm>

#include "gf_adjoint.cuh"
#include "gf_internal.h"

namespace gf {

constexpr int kAdjK = 2 * kSideInline + 5;  // reaction inputs: species entries, M, T, ln|A|, beta, Ta
constexpr int kSeedM = 2 * kSideInline, kSeedT = kSeedM + 1, kSeedLnA = kSeedM + 2, kSeedBeta = kSeedM + 3,
              kSeedTa = kSeedM + 4;

// workspace of the sweep, after the forward workspace of make_layout
struct AdjLayout {
    int y2, y3, rb, kb, yb, fb0, fb2, fb3, fs, f2, f3, Jb, raw, Jc, dfc, cb, Mb, gq, ms, vb, dn, ab, dd, size;
};
enum { MS_RHO = 0, MS_CPM, MS_DCPM, MS_AV, MS_RHOB, MS_CPMB, MS_DCPMB, MS_AVB, MS_TB, MS_SH, MS_N = 16 };

// y2, y3, fs, f2 and f3 live in the forward workspace (shared memory), after
// its make_layout part (fwd_size doubles in all); every other array is in the
// per-CTA adjoint region in global memory, offsets from 0.
__host__ __device__ inline AdjLayout make_adj_layout(const WsLayout& L, int nS, int nR, int n_tb, int* fwd_size) {
    const int m = nS + 1;
    AdjLayout A;
    A.y2 = L.size;
    A.y3 = L.size + m;
    A.fs = L.size + 2 * m;            // f at the point being reversed
    A.f2 = L.size + 3 * m;            // f at the stage points, from the recompute
    A.f3 = L.size + 4 * m;
    *fwd_size = L.size + 5 * m;
    int o = 0;
    A.rb = o; o += 4 * m;
    A.kb = o; o += 4 * m;
    A.yb = o; o += m;
    A.fb0 = o; o += m;
    A.fb2 = o; o += m;
    A.fb3 = o; o += m;
    A.Jb = o; o += m * L.ld;
    A.raw = o; o += m * L.ld;
    A.Jc = o; o += m * L.ld;          // the converted Jacobian at y0 (before the shift)
    A.dfc = o; o += m;                // its dfdx
    A.cb = o; o += nS;
    A.Mb = o; o += (n_tb > 0 ? n_tb : 1);
    A.gq = o; o += 2 * kSideInline * (nR > 0 ? nR : 1);
    A.ms = o; o += MS_N;
    A.vb = o; o += 4 * nS;           // Cp, Ha, rhoM/W, v adjoints
    A.dn = o; o += nS;               // dN/dt adjoints
    A.ab = o; o += m;                // T-row scratch
    A.dd = o; o += m;                // ddN adjoints of the rows
    A.size = o;
    return A;
}

struct AdjArgs {
    int n_cells;
    const double* traj;
    int traj_cap, traj_ld;
    const int* counters;  // [n][2] accepted, attempts of the recording solve
    const int* fstatus;   // recording solve's per-cell status
    const double* Y0;     // initial states (p taken from here)
    const double* Ynew;   // final (clipped) states
    const double* Ybar;   // loss gradient w.r.t. Ynew
    int ld_y;
    double* Y0bar;        // out: gradient w.r.t. Y0
    double* theta_bar;    // out: [n][3 nR] per reaction (mechanism order): d/d ln|A|, d/d beta, d/d Ta
    int* status;          // out: per-cell status (0 ok)
    double Treact;
    OdeParams ode;
    double* ws;
    long long ws_per_cell;
    unsigned long long* queue;
};

// ------------------------------------------------------------------ pieces

// W^T x = b with the factors of W (rows permuted: P W = L U): U^T z = b
// (forward substitution), L^T v = z (backward, unit diagonal), x[perm[i]] =
// v[i]. One warp, R rows per lane (lane l holds rows l + 32 u), column by
// column with the pivot value broadcast by a shuffle; the entries used at
// step j are row j of the factors (contiguous). m <= 32 R.
template <int R, class W>
__device__ void lu_solve_transposed_warp(const W& w, const WsC& wa, int A, int ld, int perm, int m, int b, int x) {
    const int lane = threadIdx.x & 31;
    double z[R];
#pragma unroll
    for (int u = 0; u < R; ++u) {
        const int i = 32 * u + lane;
        z[u] = i < m ? wa[b + i] : 0.0;
    }
    // U^T z = b: z_j = b_j / U[j][j], then b_i -= U[j][i] z_j for i > j
    for (int j = 0; j < m; ++j) {
        const int t = j >> 5, l = j & 31;
        double zt = z[0];
#pragma unroll
        for (int u = 1; u < R; ++u)
            if (u == t) zt = z[u];
        const double zj = __shfl_sync(0xffffffffu, zt, l) / w[A + j * ld + j];
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const int i = 32 * u + lane;
            if (i == j) z[u] = zj;
            if (i > j && i < m) z[u] -= w[A + j * ld + i] * zj;
        }
    }
    // L^T v = z: v_j final, then z_i -= L[j][i] v_j for i < j (descending j)
    for (int j = m - 1; j >= 0; --j) {
        const int t = j >> 5, l = j & 31;
        double zt = z[0];
#pragma unroll
        for (int u = 1; u < R; ++u)
            if (u == t) zt = z[u];
        const double vj = __shfl_sync(0xffffffffu, zt, l);
#pragma unroll
        for (int u = 0; u < R; ++u) {
            const int i = 32 * u + lane;
            if (i < j) z[u] -= w[A + j * ld + i] * vj;
        }
    }
#pragma unroll
    for (int u = 0; u < R; ++u) {
        const int i = 32 * u + lane;
        if (i < m) wa[x + w.ip(perm + i)] = z[u];
    }
}

template <int G, class W>
__device__ void lu_solve_transposed(const Grp<G>& g, const W& w, const WsC& wa, int A, int ld, int perm, int m, int b,
                                    int x) {
    g.sync();
    if (threadIdx.x < 32) {
        if (m <= 64)
            lu_solve_transposed_warp<2>(w, wa, A, ld, perm, m, b, x);
        else if (m <= 128)
            lu_solve_transposed_warp<4>(w, wa, A, ld, perm, m, b, x);
        else
            lu_solve_transposed_warp<10>(w, wa, A, ld, perm, m, b, x);
    }
    g.sync();
}

// stream_gather with the sources in one workspace and the results in another
template <int G, class WS, class WD>
__device__ __forceinline__ void stream_gather2(const Grp<G>& g, const Stream& st, const WS& ws, int src, const WD& wd,
                                               int dst) {
    constexpr int U = GF_GATHER_BATCH;
    const int4* r = reinterpret_cast<const int4*>(st.rec) + g.lane;
    const int len = st.len;
    double acc = 0.0;
    for (int k0 = 0; k0 < len; k0 += U) {
        int4 v[U];
#pragma unroll
        for (int u = 0; u < U; ++u) v[u] = (k0 + u < len) ? __ldg(r + (size_t)(k0 + u) * G) : make_int4(-1, -1, 0, 0);
        double x[U];
#pragma unroll
        for (int u = 0; u < U; ++u) x[u] = v[u].y >= 0 ? ws[src + v[u].y] : 0.0;
#pragma unroll
        for (int u = 0; u < U; ++u) {
            if (v[u].y >= 0) acc += __hiloint2double(v[u].w, v[u].z) * x[u];
            if (v[u].x >= 0) {
                wd[dst + v[u].x] = acc;
                acc = 0.0;
            }
        }
    }
}

// Mixture of the state at y (gpuMixture.H:33-121), as mixture() computes it,
// with its scalars kept in ms[]: rhoM, CpM, dCpMdT, alphav.
template <int G, class W>
__device__ void adj_mixture(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const WsLayout& L, const AdjLayout& A,
                            int y_off, double p) {
    double rhoM, CpM, dCpMdT, alphav;
    mixture(g, M, w, L, y_off, p, true, &rhoM, &CpM, &dCpMdT, &alphav);
    if (g.lane == 0) {
        wa[A.ms + MS_RHO] = rhoM;
        wa[A.ms + MS_CPM] = CpM;
        wa[A.ms + MS_DCPM] = dCpMdT;
        wa[A.ms + MS_AV] = alphav;
    }
    g.sync();
}

// Reverse of mixture(): given the adjoints of c (cb), Cp, Ha, rhoM/W, v (vb)
// and of the scalars (ms), adds the gradient w.r.t. the state y to ybar.
template <int G, class W>
__device__ void adj_mixture_reverse(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const WsLayout& L,
                                    const AdjLayout& A, int y_off, double p, int ybar) {
    const int nS = M.nS;
    const double T = w[y_off + nS];
    const double invT = 1.0 / T;
    const double rhoM = wa[A.ms + MS_RHO];
    // sums of the forward that the reverse needs
    double s_av = 0.0;
    for (int i = g.lane; i < nS; i += G) {
        const double yi = fmax(w[y_off + i], 0.0);
        const double rhoi = p / (ldg(M.Rsp + i) * T);
        s_av += yi * (1.0 / rhoi) * invT;
    }
    s_av = g.sum(s_av);
    double rhoMb_l = 0.0;
    for (int i = g.lane; i < nS; i += G) {
        const double yi = fmax(w[y_off + i], 0.0);
        rhoMb_l += wa[A.vb + 2 * nS + i] / ldg(M.W + i) + wa[A.cb + i] * (yi / ldg(M.W + i));
    }
    const double rhoMb = wa[A.ms + MS_RHOB] + g.sum(rhoMb_l) + wa[A.ms + MS_AVB] * s_av;
    const double s_avb = wa[A.ms + MS_AVB] * rhoM;
    const double s_rhob = -rhoMb * rhoM * rhoM;
    const double CpMb = wa[A.ms + MS_CPMB], dCpMb = wa[A.ms + MS_DCPMB];
    double Tb = 0.0, invTb = 0.0;
    for (int i = g.lane; i < nS; i += G) {
        const double Yi = w[y_off + i];
        const double yi = fmax(Yi, 0.0);
        const double rhoi = p / (ldg(M.Rsp + i) * T);
        const double vi = 1.0 / rhoi;
        const Poly7 a = species_coeffs(M, i, T);
        const double Cpi = th_Cp(a, T);
        const double dCpi = th_dCpdT(a, T);
        const double d2Cpi = (12.0 * a.a4 * T + 6.0 * a.a3) * T + 2.0 * a.a2;
        const double yb = s_rhob / rhoi + CpMb * Cpi + wa[A.cb + i] * rhoM / ldg(M.W + i) + dCpMb * dCpi +
                          s_avb * vi * invT;
        double rhoib = -s_rhob * yi / (rhoi * rhoi);
        const double vb = wa[A.vb + 3 * nS + i] + s_avb * yi * invT;
        rhoib += -vb / (rhoi * rhoi);
        Tb += rhoib * (-rhoi / T);
        Tb += (wa[A.vb + i] + CpMb * yi) * dCpi;  // Cp_i(T)
        Tb += wa[A.vb + nS + i] * Cpi;             // Ha_i(T): dHa/dT = Cp
        Tb += dCpMb * yi * d2Cpi;                 // dCp_i/dT(T)
        invTb += s_avb * yi * vi;
        wa[ybar + i] += Yi > 0.0 ? yb : 0.0;
    }
    Tb = g.sum(Tb);
    invTb = g.sum(invTb);
    if (g.lane == 0) wa[ybar + nS] += Tb - invTb * invT * invT + wa[A.ms + MS_TB];
    g.sync();
}

// Per-reaction reverse: omega_bar from dN/dt adjoints (dn) and, when the
// Jacobian's raw adjoint (rawb, m x ld) is given, the pullback of its terms;
// the derivatives w.r.t. the reaction's inputs (closed form or rxn_vjp);
// concentration adjoints to the
// per-entry slots (gq), third-body ones to Mb, T to ms[MS_TB] (summed by the
// caller), parameters to theta_bar (accumulated).
template <int G, class W>
__device__ void adj_reactions(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const WsLayout& L, const AdjLayout& A,
                              int y_off, int rawb, double* theta_bar) {
    const int nS = M.nS;
    const double T = w[y_off + nS];
    double Tb = 0.0;
    for (int q = g.lane; q < M.nR; q += G) {
        Rxn R;
        load_rxn(M, q, R);
        // omega_bar = sum over the reaction's species of nu * dN/dt_bar
        double ob = 0.0;
        for (int e = 0; e < R.nl; ++e) ob -= ldg(M.sst + R.sp_off + e) * wa[A.dn + R.idx[0][e]];
        for (int e = 0; e < R.nr; ++e) ob += ldg(M.sst + R.sp_off + R.nl + e) * wa[A.dn + R.idx[1][e]];
        // the Jacobian terms' weights: ghat[col] = sum over rows s of the
        // reaction of nu_s * rawbar[s][col]
        double gD[2 * kSideInline], gT = 0.0, gE = 0.0;
#pragma unroll
        for (int e = 0; e < 2 * kSideInline; ++e) gD[e] = 0.0;
        if (rawb >= 0) {
            const int ld = L.ld;
            for (int side = 0; side < 2; ++side) {
                const int n = side ? R.nr : R.nl;
                for (int r = 0; r < n; ++r) {
                    const double nu = side ? ldg(M.sst + R.sp_off + R.nl + r) : -ldg(M.sst + R.sp_off + r);
                    const int s = R.idx[side][r];
                    const int row = rawb + s * ld;
#pragma unroll
                    for (int e = 0; e < 2 * kSideInline; ++e) {
                        const int sd = e / kSideInline, ee = e % kSideInline;
                        if (ee < (sd ? R.nr : R.nl)) gD[e] += nu * w[row + R.idx[sd][ee]];
                    }
                    gT += nu * w[row + nS];
                    if (R.type == GF_RATE_THIRD_BODY_ARRHENIUS) {
                        const double* eff = M.eff + (size_t)R.tb_row * nS;
                        double acc = 0.0;
                        for (int c = 0; c < nS; ++c) acc += ldg(eff + c) * w[row + c];
                        gE += nu * acc;
                    }
                }
            }
            // rhs terms enter the raw Jacobian with the opposite sign (-dCr/dc kr)
#pragma unroll
            for (int e = kSideInline; e < 2 * kSideInline; ++e) gD[e] = -gD[e];
        }
        if (rawb < 0 && (R.type == GF_RATE_ARRHENIUS || R.type == GF_RATE_THIRD_BODY_ARRHENIUS)) {
            // omega only, closed form: with phi = Cf - Cr/Kc, d omega / d kf = phi,
            // d omega / d c (lhs) = kf dCf/dc, (rhs) = -kr dCr/dc,
            // d omega / dT = phi dkf/dT + kr Cr dln(Kc)/dT (the ln K cap of
            // gpuThermo.H:84-85 taken as computed), d kf / d(ln|A|, beta, Ta) =
            // kf (1, ln T, -1/T), d omega / dM = Ak phi (third body)
            const double invT = 1.0 / T, logT = ::log(T);
            const double Ak = R.sA0 * ::exp(fma(R.beta0, logT, R.lnA0) - R.Ta0 * invT);
            const double Mc = R.tb_row >= 0 ? w[L.Mtb + R.tb_row] : 0.0;
            const double kf = R.type == GF_RATE_THIRD_BODY_ARRHENIUS ? Mc * Ak : Ak;
            const double dkfdT = kf * ((R.beta0 + R.Ta0 * invT) * invT);
            double pw[2][kSideInline], dm[2][kSideInline], C2[2] = {1.0, 1.0};
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const int n = side ? R.nr : R.nl;
#pragma unroll
                for (int e = 0; e < kSideInline; ++e) {
                    pw[side][e] = 1.0;
                    dm[side][e] = 1.0;
                    if (e < n) {
                        const double x = w[L.c + R.idx[side][e]];
                        pw[side][e] = specie_pow(x, R.iexp[side][e], R.sexp[side][e]);
                        dm[side][e] = R.sexp[side][e] * specie_pow_m1(x, R.iexp[side][e], R.sexp[side][e]);
                        C2[side] *= pw[side][e];
                    }
                }
            }
            double invKc = 1.0, kr = 0.0, dlnK = 0.0, Cr = 0.0;
            if (!R.irr) {
                const TCache tc = make_tcache(T);
                const Poly7 a = reaction_coeffs_at(M, q, T, R.Tcommon);
                const double Gstd = th_Gstd(a, T, logT);
                const double arg = -R.Y * Gstd * invT * (1.0 / kRR);
                double lnK = arg < 600 ? arg : 0.5 * ::log(kVGreat);
                if (!R.nm_small) lnK += R.nm * tc.lx;
                invKc = ::exp(-lnK);
                kr = kf * invKc;
                Cr = C2[1];
                if (arg < 600) dlnK = (th_S_pstd(a, T, logT) + Gstd * invT) * R.Y * invT * (1.0 / kRR);
                if (!R.nm_small) dlnK -= R.nm * invT;
            }
            const double phi = C2[0] - Cr * invKc;
            double gr[2 * kSideInline];
#pragma unroll
            for (int side = 0; side < 2; ++side) {
                const int n = side ? R.nr : R.nl;
#pragma unroll
                for (int j = 0; j < kSideInline; ++j) {
                    double d = 0.0;
                    if (j < n && !(side && R.irr)) {
                        d = 1.0;
#pragma unroll
                        for (int i = 0; i < kSideInline; ++i)
                            if (i < n) d *= (i == j) ? dm[side][i] : pw[side][i];
                        d *= side ? -kr : kf;
                    }
                    gr[side * kSideInline + j] = ob * d;
                }
            }
#pragma unroll
            for (int e = 0; e < 2 * kSideInline; ++e) wa[A.gq + q * 2 * kSideInline + e] = gr[e];
            if (R.tb_row >= 0) wa[A.Mb + R.tb_row] = ob * Ak * phi;
            Tb += ob * (phi * dkfdT + kr * Cr * dlnK);
            const int r = ldg(M.r_of_q + q);
            const double gk = ob * phi * kf;
            theta_bar[3 * r] += gk;
            theta_bar[3 * r + 1] += gk * logT;
            theta_bar[3 * r + 2] += -gk * invT;
            continue;
        }
        // the vector-Jacobian product of the reaction's quantities (rxn_vjp)
        double c[2 * kSideInline];
#pragma unroll
        for (int e = 0; e < 2 * kSideInline; ++e) {
            const int sd = e / kSideInline, ee = e % kSideInline;
            const bool on = ee < (sd ? R.nr : R.nl);
            c[e] = on ? w[L.c + R.idx[sd][ee]] : 1.0;
        }
        double gr[kAdjK];
        rxn_vjp(M, q, R, c, R.tb_row >= 0 ? w[L.Mtb + R.tb_row] : 0.0, T, ob, gD, gT, gE, gr);
#pragma unroll
        for (int e = 0; e < 2 * kSideInline; ++e) wa[A.gq + q * 2 * kSideInline + e] = gr[e];
        if (R.tb_row >= 0) wa[A.Mb + R.tb_row] = gr[kSeedM];
        Tb += gr[kSeedT];
        const int r = ldg(M.r_of_q + q);
        theta_bar[3 * r] += gr[kSeedLnA];
        theta_bar[3 * r + 1] += gr[kSeedBeta];
        theta_bar[3 * r + 2] += gr[kSeedTa];
    }
    Tb = g.sum(Tb);
    if (g.lane == 0) wa[A.ms + MS_TB] += Tb;
    g.sync();
}

// Concentration adjoints: the per-entry slots gathered per species (stream),
// plus the third-body terms c_bar[i] += sum_t Mbar[t] eff[t][i].
template <int G, class W>
__device__ void adj_gather_c(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const AdjLayout& A) {
    stream_gather(g, M.cst[stream_index(G)], wa, A.gq, A.dd);
    g.sync();
    for (int i = g.lane; i < M.nS; i += G) {
        double acc = wa[A.cb + i] + wa[A.dd + i];
        for (int t = 0; t < M.n_tb; ++t) acc += wa[A.Mb + t] * ldg(M.eff + (size_t)t * M.nS + i);
        wa[A.cb + i] = acc;
    }
    g.sync();
}

// Reverse of the derivatives' assembly (gpuODESystem.H:164-196) given fbar
// (m) at the point whose f is in fs: dN/dt adjoints to dn, and the adjoints
// of Ha, CpM, rhoM added to vb / ms.
template <int G, class W>
__device__ void adj_rhs_assembly(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const WsLayout& L,
                                 const AdjLayout& A, int fbar) {
    const int nS = M.nS;
    const double rhoM = wa[A.ms + MS_RHO], CpM = wa[A.ms + MS_CPM];
    const double dTdt = w[A.fs + nS];
    const double dTb = wa[fbar + nS];
    const double shb = -dTb / CpM;
    double rhoMb = 0.0;
    for (int s = g.lane; s < nS; s += G) {
        const double dYdt = w[A.fs + s];
        const double Wr = ldg(M.W + s) / rhoM;
        const double dYb = wa[fbar + s] + shb * w[L.Ha + s];
        wa[A.vb + nS + s] += shb * dYdt;
        wa[A.dn + s] = dYb * Wr;
        rhoMb += dYb * (dYdt / Wr) * (-ldg(M.W + s) / (rhoM * rhoM));
    }
    rhoMb = g.sum(rhoMb);
    if (g.lane == 0) {
        // dT/dt = -sh / CpM, sh = sum dY/dt Ha  ->  d/dCpM = -dT/dt / CpM
        wa[A.ms + MS_CPMB] += dTb * (-dTdt / CpM);
        wa[A.ms + MS_RHOB] += rhoMb;
    }
    g.sync();
}

template <int G, class W>
__device__ void adj_clear_point(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const AdjLayout& A) {
    for (int i = g.lane; i < 4 * M.nS; i += G) wa[A.vb + i] = 0.0;
    for (int i = g.lane; i < M.nS; i += G) wa[A.cb + i] = 0.0;
    for (int i = g.lane; i < MS_N; i += G)
        if (i >= MS_RHOB) wa[A.ms + i] = 0.0;
    g.sync();
}

// ybar += (df/dy)^T fbar at the point y (no Jacobian term)
template <int G, class W>
__device__ void adj_vjp_f(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const WsLayout& L, const AdjLayout& A,
                          int y_off, double p, int f_off, int fbar, int ybar, double* theta_bar) {
    // f at y: the recompute's value (f_off; the same state and code)
    for (int i = g.lane; i < M.m; i += G) w[A.fs + i] = w[f_off + i];
    adj_mixture(g, M, w, wa, L, A, y_off, p);     // c, Ha, Cp, v, rhoM/W and the scalars at y
    if (M.n_tb > 0) {
        third_body_all(g, M, w, L.c, L.Mtb);          // the third-body concentrations at y
        g.sync();
    }
    adj_clear_point(g, M, w, wa, A);
    adj_rhs_assembly(g, M, w, wa, L, A, fbar);
    {
        GF_PH_BEGIN(g)
        adj_reactions(g, M, w, wa, L, A, y_off, -1, theta_bar);
        GF_PH_END(g, PH_ADJ_RXN)
    }
    adj_gather_c(g, M, w, wa, A);
    adj_mixture_reverse(g, M, w, wa, L, A, y_off, p, ybar);
}

// Jacobian term at y0 together with the VJP of f at y0: Jbar (A.Jb) pulled
// back through the T row and the conversion to the raw entries (into L.J),
// the adjoints of the mixture quantities, and dfdx_bar added to fbar.
template <int G, class W>
__device__ void adj_jacobian_term(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const WsLayout& L,
                                  const AdjLayout& A, int y_off, double p, int fbar, int ybar, double* theta_bar) {
    const int nS = M.nS, ld = L.ld;
    // forward at y0, all from the recompute (the same state and code): f
    // (L.dydx0), the converted J and dfdx (A.Jc, A.dfc), the raw entries
    // (A.raw); the mixture and the third-body concentrations are evaluated again
    for (int i = g.lane; i < M.m; i += G) {
        w[A.fs + i] = w[L.dydx0 + i];
        w[L.dfdx + i] = wa[A.dfc + i];
    }
    for (int e = g.lane; e < M.m * ld; e += G) w[L.J + e] = wa[A.Jc + e];
    adj_mixture(g, M, w, wa, L, A, y_off, p);
    if (M.n_tb > 0) {
        third_body_all(g, M, w, L.c, L.Mtb);
        g.sync();
    }
    adj_clear_point(g, M, w, wa, A);
    const double CpM = wa[A.ms + MS_CPM], rhoM = wa[A.ms + MS_RHO], alphav = wa[A.ms + MS_AV],
                 dCpMdT = wa[A.ms + MS_DCPM];
    const double dTdt = w[L.dfdx + nS];
    // (a) T row: J[nS][i] = (-sum_j J[j][i] Ha_j - Cp_i dTdt) / CpM (i < nS) and
    //     J[nS][nS] = (-sum_i (dfdx_i Cp_i + J[i][nS] Ha_i) - dTdt dCpMdT) / CpM
    double CpMb = 0.0, dTdtb = 0.0;
    for (int i = g.lane; i < nS; i += G) {
        const double Jb = wa[A.Jb + nS * ld + i];
        const double ab = Jb / CpM;
        wa[A.ab + i] = ab;
        CpMb += -Jb * w[L.J + nS * ld + i] / CpM;
        wa[A.vb + i] += -ab * dTdt;  // Cp_i
        dTdtb += -ab * w[L.Cp + i];
        for (int j = 0; j < nS; ++j) wa[A.Jb + j * ld + i] += -ab * w[L.Ha + j];
    }
    CpMb = g.sum(CpMb);
    dTdtb = g.sum(dTdtb);
    const double JbTT = wa[A.Jb + nS * ld + nS];
    const double bb = JbTT / CpM;
    if (g.lane == 0) {
        wa[A.ms + MS_CPMB] += CpMb - JbTT * w[L.J + nS * ld + nS] / CpM;
        wa[A.ms + MS_DCPMB] += -bb * dTdt;
        wa[fbar + nS] += dTdtb - bb * dCpMdT;
    }
    g.sync();
    // Ha_j adjoint: sum_i -ab_i J[j][i] - bb J[j][nS]; Cp_i, dfdx_i from the TT entry
    for (int j = g.lane; j < nS; j += G) {
        double acc = 0.0;
        for (int i = 0; i < nS; ++i) acc += -wa[A.ab + i] * w[L.J + j * ld + i];
        acc += -bb * w[L.J + j * ld + nS];
        wa[A.vb + nS + j] += acc;
        wa[A.vb + j] += -bb * w[L.dfdx + j];
        wa[fbar + j] += -bb * w[L.Cp + j];
        wa[A.Jb + j * ld + nS] += -bb * w[L.Ha + j];
    }
    g.sync();
    // (b) conversion rows: J[s][c] = Wr_s raw[s][c] rW_c + rhoM v_c dfdx_s,
    //     ddN_s = raw[s][nS] - sum_c raw[s][c] c_c alphav, J[s][nS] = Wr_s ddN_s + alphav dfdx_s
    double avb = 0.0, rhoMb = 0.0;
    for (int s = g.lane; s < nS; s += G) {
        const double Wr = ldg(M.W + s) / rhoM;
        const double dfs = w[L.dfdx + s];
        const int row = A.raw + s * ld, brow = A.Jb + s * ld;
        double ddN = wa[row + nS];
        for (int c = 0; c < nS; ++c) ddN -= wa[row + c] * w[L.c + c] * alphav;
        const double JbT = wa[brow + nS];
        const double ddNb = JbT * Wr;
        double Wrb = JbT * ddN;
        avb += JbT * dfs;
        double dfsb = JbT * alphav;
        for (int c = 0; c < nS; ++c) {
            const double Jb = wa[brow + c];
            const double raw = wa[row + c];
            Wrb += Jb * raw * w[L.rhoMbyW + c];
            rhoMb += Jb * w[L.vj + c] * dfs;
            dfsb += Jb * rhoM * w[L.vj + c];
            avb += -ddNb * raw * w[L.c + c];
            w[L.J + s * ld + c] = Jb * Wr * w[L.rhoMbyW + c] - ddNb * w[L.c + c] * alphav;  // raw_bar
        }
        w[L.J + s * ld + nS] = ddNb;
        wa[A.dd + s] = ddNb;
        rhoMb += -Wrb * ldg(M.W + s) / (rhoM * rhoM);
        wa[fbar + s] += dfsb;
    }
    avb = g.sum(avb);
    rhoMb = g.sum(rhoMb);
    if (g.lane == 0) {
        wa[A.ms + MS_AVB] += avb;
        wa[A.ms + MS_RHOB] += rhoMb;
    }
    g.sync();
    // (c) columns: rhoM/W_c, v_c and c_c adjoints
    for (int c = g.lane; c < nS; c += G) {
        double rWb = 0.0, vb = 0.0, cb = 0.0;
        for (int s = 0; s < nS; ++s) {
            const double Jb = wa[A.Jb + s * ld + c];
            const double raw = wa[A.raw + s * ld + c];
            rWb += Jb * (ldg(M.W + s) / rhoM) * raw;
            vb += Jb * rhoM * w[L.dfdx + s];
            cb += -wa[A.dd + s] * raw * alphav;
        }
        wa[A.vb + 2 * nS + c] += rWb;
        wa[A.vb + 3 * nS + c] += vb;
        wa[A.cb + c] += cb;
    }
    g.sync();
    // the VJP of f at y0 with the completed fbar, the raw terms' pullback, and
    // the mixture reverse for all of it
    adj_rhs_assembly(g, M, w, wa, L, A, fbar);
    {
        GF_PH_BEGIN(g)
        adj_reactions(g, M, w, wa, L, A, y_off, L.J, theta_bar);
        GF_PH_END(g, PH_ADJ_RXN)
    }
    // third-body concentrations: the stage pass left Mtb from the Jacobian's
    // mixture, the same state
    adj_gather_c(g, M, w, wa, A);
    adj_mixture_reverse(g, M, w, wa, L, A, y_off, p, ybar);
}

// One recorded step in reverse: ybar (A.yb) holds the adjoint of the step's
// end state on entry and of its start state (L.y0) on exit.
template <int G, class W>
__device__ void adj_step(const Grp<G>& g, const DevMech& M, const W& w, const WsC& wa, const WsLayout& L, const AdjLayout& A,
                         const RosCoeffs& C, const OdeParams& o, double p, double h, double* theta_bar) {
    const int m = M.m, ld = L.ld;
    // recompute the attempt (stages kept: k_i, y2, y3; LU factors in L.J)
    if (g.lane == 0) w[L.scal + S_KCACHE_T] = -1.0;
    g.sync();
    {
        GF_PH_BEGIN(g)
        // f(y0) keeps its rate constants for the Jacobian at the same state
        derivatives(g, M, w, L, L.y0, p, L.dydx0, true);
        jacobian(g, M, w, L, L.y0, p, true);
        // kept for the Jacobian term: the raw entries (from the Jacobian terms
        // in the staging slots), the converted Jacobian and dfdx
        stream_gather2(g, M.jst[stream_index(G)], w, L.stage, wa, A.raw);
        for (int e = g.lane; e < m * ld; e += G) wa[A.Jc + e] = w[L.J + e];
        for (int i = g.lane; i < m; i += G) wa[A.dfc + i] = w[L.dfdx + i];
        g.sync();
        shift_and_factor(g, M, w, L, C, h);
        ros_attempt<G, W, true>(g, M, w, L, C, o, L.y0, L.yt, p, h, A.y2, A.y3, false, A.f2, A.f3);
        GF_PH_END(g, PH_ADJ_RECOMPUTE)
    }
    // kbar_i = b_i ybar; the ybar of y1 = y0 + sum b_i k_i flows to y0 unchanged
    const double bc[4] = {C.b1, C.b2, C.b3, C.b4};
    for (int i = g.lane; i < m; i += G) {
        for (int st = 0; st < C.s; ++st) wa[A.kb + st * m + i] = bc[st] * wa[A.yb + i];
        wa[A.fb0 + i] = 0.0;
        wa[A.fb2 + i] = 0.0;
        wa[A.fb3 + i] = 0.0;
    }
    g.sync();
    for (int st = C.s - 1; st >= 0; --st) {
        const int rb = A.rb + st * m;
        {
            GF_PH_BEGIN(g)
            lu_solve_transposed(g, w, wa, L.J, ld, L.perm, m, A.kb + st * m, rb);
            GF_PH_END(g, PH_ADJ_TSOLVE)
        }
        const int fsrc = st == 0 ? A.fb0 : (st == 1 || C.s == 3 ? A.fb2 : A.fb3);
        const double hd = h * ros_d(C, st);
        for (int i = g.lane; i < m; i += G) {
            const double r = wa[rb + i];
            wa[fsrc + i] += r;
            wa[A.fb0 + i] += hd * r;  // dfdx = f(y0)
            for (int j = 0; j < st; ++j) wa[A.kb + j * m + i] += (ros_c(C, st, j) / h) * r;
        }
        g.sync();
        if (st == 1 || (st == 2 && C.s == 4)) {
            const int pt = st == 1 ? A.y2 : A.y3;
            const int fb = st == 1 ? A.fb2 : A.fb3;
            // ybar of the stage point: into fs-free scratch (A.ab), then to y0 and k_j
            for (int i = g.lane; i < m; i += G) wa[A.ab + i] = 0.0;
            g.sync();
            {
                GF_PH_BEGIN(g)
                adj_vjp_f(g, M, w, wa, L, A, pt, p, st == 1 ? A.f2 : A.f3, fb, A.ab, theta_bar);
                GF_PH_END(g, PH_ADJ_VJP)
            }
            for (int i = g.lane; i < m; i += G) {
                const double yb = wa[A.ab + i];
                wa[A.yb + i] += yb;
                for (int j = 0; j < st; ++j) wa[A.kb + j * m + i] += ros_a(C, st, j) * yb;
            }
            g.sync();
        }
    }
    // Jbar = sum_i rbar_i k_i^T  (W = I/(gamma h) - J, k_i = W^-1 r_i)
    for (int e = g.lane; e < m * m; e += G) {
        const int a = e / m, b = e % m;
        double acc = 0.0;
        for (int st = 0; st < C.s; ++st) acc += wa[A.rb + st * m + a] * w[L.k1 + st * m + b];
        wa[A.Jb + a * ld + b] = acc;
    }
    g.sync();
    {
        GF_PH_BEGIN(g)
        adj_jacobian_term(g, M, w, wa, L, A, L.y0, p, A.fb0, A.yb, theta_bar);
        GF_PH_END(g, PH_ADJ_JTERM)
    }
}

__global__ void __launch_bounds__(64) adjoint_kernel(const DevMech M, const AdjArgs a) {
    extern __shared__ double smem[];
    Grp<64> g;
    const WsLayout L = make_layout(M.nS, M.nR, M.n_slots, M.n_tb, true);
    int fwd = 0;
    const AdjLayout A = make_adj_layout(L, M.nS, M.nR, M.n_tb, &fwd);
    WsC w{smem};
    WsC wa{a.ws + (size_t)blockIdx.x * a.ws_per_cell};
    const RosCoeffs C = ros_coeffs(a.ode.solver);
    const int nS = M.nS, m = M.m;
    for (;;) {
        long long cell = 0;
        if (g.lane == 0) cell = (long long)atomicAdd(a.queue, 1ull);
        cell = g.bcast_ll(cell, 0);
        if (cell >= a.n_cells) break;
        double* thb = a.theta_bar + (size_t)cell * 3 * M.nR;
        for (int i = g.lane; i < 3 * M.nR; i += 64) thb[i] = 0.0;
        const double* yin = a.Y0 + (size_t)cell * a.ld_y;
        const double* yfin = a.Ynew + (size_t)cell * a.ld_y;
        const double* ybr = a.Ybar + (size_t)cell * a.ld_y;
        const double p = yin[nS + 1];
        const int fst = a.fstatus[cell];
        const int N = a.counters[2 * cell];
        // the final clip max(0, Y) (singleCellSolver.H:42-45): gradient passes where Y > 0
        for (int i = g.lane; i < m; i += 64)
            wa[A.yb + i] = (fst == GF_CELL_SKIPPED || i == nS || yfin[i] > 0.0) ? ybr[i] : 0.0;
        int status = fst == GF_CELL_SKIPPED ? GF_CELL_OK : fst;
        if (fst == GF_CELL_OK) {
            for (int k = N - 1; k >= 0; --k) {
                const double* rec = a.traj + ((size_t)cell * a.traj_cap + k) * a.traj_ld;
                for (int i = g.lane; i < m; i += 64) w[L.y0 + i] = rec[i];
                const double h = rec[m];
                __syncthreads();
                adj_step(g, M, w, wa, L, A, C, a.ode, p, h, thb);
            }
        }
        double* yo = a.Y0bar + (size_t)cell * a.ld_y;
        for (int i = g.lane; i < m; i += 64) yo[i] = status == GF_CELL_OK ? wa[A.yb + i] : 0.0;
        if (g.lane == 0) {
            yo[nS + 1] = 0.0;
            a.status[cell] = status;
        }
        __syncthreads();
    }
}

// The recording solve (gf_solve_record): the persistent form with one cell
// per 128-thread CTA, workspace in shared memory, at most 128 registers, and
// each accepted step recorded for the sweep.
__global__ void __launch_bounds__(128, 4) record_kernel(const DevMech M, const LaunchArgs a) {
    extern __shared__ double smem[];
    Grp<128> g;
    for (;;) {
        long long cell = 0;
        if (g.lane == 0) cell = (long long)atomicAdd(a.queue, 1ull);
        cell = g.bcast_ll(cell, 0);
        if (cell >= a.n_cells) break;
        process_cell<128, WsC, true>(g, M, WsC{smem}, a, (int)cell);
    }
}

__global__ void adj_reset(unsigned long long* q) { q[0] = 0; }

int launch_record(const DevMech& M, const LaunchArgs& a, void* stream) {
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const int smem = make_layout(M.nS, M.nR, M.n_slots, M.n_tb).size * (int)sizeof(double);
    if (smem > 227 * 1024) return (int)cudaErrorInvalidValue;
    cudaFuncSetAttribute(record_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, record_kernel, 128, smem);
    if (e != cudaSuccess) return (int)e;
    if (per_sm < 1) return (int)cudaErrorInvalidConfiguration;
    launch_epilogue_reset(a.queue, stream);
    if (a.n_cells > 0) record_kernel<<<per_sm * device_sm_count(), 128, smem, s>>>(M, a);
    return (int)cudaGetLastError();
}

int adjoint_ws_doubles(const DevMech& M) {
    const WsLayout L = make_layout(M.nS, M.nR, M.n_slots, M.n_tb, true);
    int fwd = 0;
    return make_adj_layout(L, M.nS, M.nR, M.n_tb, &fwd).size;
}

static int adjoint_smem_bytes(const DevMech& M) {
    const WsLayout L = make_layout(M.nS, M.nR, M.n_slots, M.n_tb, true);
    int fwd = 0;
    make_adj_layout(L, M.nS, M.nR, M.n_tb, &fwd);
    return fwd * (int)sizeof(double);
}

int adjoint_blocks_per_sm(const DevMech& M) {
    const int smem = adjoint_smem_bytes(M);
    if (smem > 227 * 1024) return 0;
    cudaFuncSetAttribute(adjoint_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, adjoint_kernel, 64, smem) != cudaSuccess) return 0;
    return per_sm;
}

int launch_adjoint_cells(const DevMech& M, int n_cells, const double* traj, int traj_cap, const int* counters,
                         const int* fwd_status, const double* Y0, const double* Ynew, const double* Ybar, int ld_y,
                         double* Y0bar, double* theta_bar, int* status, const OdeParams& ode, double* ws,
                         long long ws_per_cell, int n_blocks, unsigned long long* queue, void* stream) {
    AdjArgs a;
    a.n_cells = n_cells;
    a.traj = traj;
    a.traj_cap = traj_cap;
    a.traj_ld = M.m + 1;
    a.counters = counters;
    a.fstatus = fwd_status;
    a.Y0 = Y0;
    a.Ynew = Ynew;
    a.Ybar = Ybar;
    a.ld_y = ld_y;
    a.Y0bar = Y0bar;
    a.theta_bar = theta_bar;
    a.status = status;
    a.Treact = 0.0;
    a.ode = ode;
    a.ws = ws;
    a.ws_per_cell = ws_per_cell;
    a.queue = queue;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    adj_reset<<<1, 1, 0, s>>>(queue);
    if (n_cells > 0) adjoint_kernel<<<n_blocks, 64, adjoint_smem_bytes(M), s>>>(M, a);
    return (int)cudaGetLastError();
}

#ifdef GF_PHASE_TIMERS
int phase_cycles_adj(unsigned long long* out, int reset) { return phase_cycles_local(out, reset); }
#endif

}  // namespace gf
