// TEST INFRASTRUCTURE ONLY — never part of the product path.
//
// C driver around the gpuFoam reference's own FP64 chemistry code, compiled
// for the host CPU from the reference headers where they lie (see
// oracle/Makefile; nothing is copied into this repository). The reference's
// device code is plain __host__ __device__ C++ that g++ compiles unchanged
// (gpu_utils/common/cuda_host_dev.H:3-28), i.e. exactly the reference's own
// "CPU" test path (gpu_chemistry/unittest/cpuTestKernels/cpu_test_kernels.C).
//
// What the driver adds, because the reference's versions need OpenFOAM:
//  * mechanism construction by constructor from a flat raw description,
//    restating makeGpuThermo (makeGpuThermo.H:16-48: coefficients x R) and
//    set_reaction_thermo (makeGpuReactions.H:18-59) with the reference's own
//    gpuThermo operators (*, +=, ==);
//  * a counting wrapper around the reference Rosenbrock solvers so that the
//    accepted/attempted substeps of odeSolve can be compared per cell;
//  * the host-side computeRR arithmetic (gpuKernelEvaluator.cu:65-97);
//  * an OpenMP loop over cells (schedule(dynamic,1): one cell per chunk) for the timed CPU
//    baseline.
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>
#include <omp.h>

#include "cpuMemoryResource.H"
#include "gpuODESolver.H"
#include "gpuODESystem.H"
#include "gpuReaction.H"
#include "gpuThermo.H"
#include "makeGpuOdeSolver.H"
#include "singleCellSolver.H"

using namespace FoamGpu;

namespace {

constexpr int RINT = 24;   // rate_type, irreversible, n_lhs, n_rhs, lhs idx[10], rhs idx[10]
constexpr int RDBL = 50;   // lhs stoich[10], lhs exp[10], rhs stoich[10], rhs exp[10],
                           // A, beta, Ta, Ainf, betainf, Tainf, alpha, Tsss, Ts, Tss

struct RefMech {
    int nS = 0, nR = 0;
    std::vector<gpuThermo> thermos;
    std::vector<gpuReaction> reactions;
};

struct OdeIn {  // layout of gf_ode_inputs (include/gpufoam_b200.h)
    int solver;
    double absTol, relTol;
    int maxSteps;
    double safeScale, alphaInc, alphaDec, minScale, maxScale;
};

gpuODESolverInputs to_inputs(const OdeIn& o) {
    gpuODESolverInputs i;
    i.name = o.solver == 12 ? "Rosenbrock12" : (o.solver == 23 ? "Rosenbrock23" : "Rosenbrock34");
    i.absTol = o.absTol;
    i.relTol = o.relTol;
    i.maxSteps = o.maxSteps;
    i.safeScale = o.safeScale;
    i.alphaInc = o.alphaInc;
    i.alphaDec = o.alphaDec;
    i.minScale = o.minScale;
    i.maxScale = o.maxScale;
    return i;
}

gpuReaction::specieCoeffArray side(int n, const int* idx, const double* st, const double* ex) {
    gpuReaction::specieCoeffArray ret{};
    for (int i = 0; i < n; ++i) {
        ret[i].index = idx[i];
        ret[i].stoichCoeff = st[i];
        const double e = ex[i];
        // make_specie_coeffs (makeGpuReactions.H:61-88)
        if (isInteger(e)) {
            ret[i].exponent = gpuSpecieExponent(gLabel(e));
        } else {
            ret[i].exponent = gpuSpecieExponent(gScalar(e));
        }
    }
    return ret;
}

gpuThirdBodyEfficiencies tbe(int nS, const double* eff) {
    gpuThirdBodyEfficiencies::effArray a{};
    for (int i = 0; i < nS; ++i) a[i] = eff[i];
    return gpuThirdBodyEfficiencies(nS, a);
}

// Counting wrapper: the reference's odeSolve/adaptiveSolve templates run on
// this type; it forwards the single-attempt solve to the reference solver.
template <class Base> struct CountingOde : public Base {
    mutable long accepted = 0;
    mutable long attempts = 0;
    explicit CountingOde(const Base& b) : Base(b) {}

    void solve(gScalar& x, mdspan<gScalar, 1> y, stepState& step, gpuBuffer& buffer) const {
        const gScalar x0 = x;
        adaptiveSolve(*this, x, y, step.dxTry, buffer);
        step.dxDid = x - x0;
        ++accepted;
    }
    gScalar solve(const mdspan<const gScalar, 1> y0, const mdspan<const gScalar, 1> dydx0,
                  const gScalar dx, mdspan<gScalar, 1> y, gpuBuffer& buffer) const {
        ++attempts;
        return Base::solve(y0, dydx0, dx, y, buffer);
    }
};

template <class F> void with_solver(const RefMech& m, const OdeIn& o, F&& f) {
    gpuODESystem sys(m.nS + 2, m.nR, m.thermos.data(), m.reactions.data());
    const auto in = to_inputs(o);
    if (o.solver == 12) {
        f(CountingOde<gpuRosenbrock12<gpuODESystem>>(gpuRosenbrock12<gpuODESystem>(sys, in)));
    } else if (o.solver == 23) {
        f(CountingOde<gpuRosenbrock23<gpuODESystem>>(gpuRosenbrock23<gpuODESystem>(sys, in)));
    } else {
        f(CountingOde<gpuRosenbrock34<gpuODESystem>>(gpuRosenbrock34<gpuODESystem>(sys, in)));
    }
}

struct Buf {
    cpuMemoryResource mem;
    std::vector<gpuBuffer> b;
    explicit Buf(int nS) : mem(1, nS), b(splitToBuffers(mem)) {}
};

}  // namespace

extern "C" {

void* ref_mech_create(int nS, const double* W, const double* Tlow, const double* Thigh,
                      const double* Tcommon, const double* high_raw, const double* low_raw,
                      int nR, const int* rint, const double* rdbl, const double* eff,
                      double rxnTlow, double rxnThigh) {
    auto* m = new RefMech;
    m->nS = nS;
    m->nR = nR;
    // makeGpuThermo: coefficients scaled by the specie gas constant R = RR/W
    for (int i = 0; i < nS; ++i) {
        const gpuPerfectGas eos(1.0, W[i]);
        gpuThermo::coeffArray hi{}, lo{};
        for (int k = 0; k < 7; ++k) {
            hi[k] = eos.R() * high_raw[7 * i + k];
            lo[k] = eos.R() * low_raw[7 * i + k];
        }
        m->thermos.push_back(gpuThermo(1.0, W[i], Tlow[i], Thigh[i], Tcommon[i], hi, lo));
    }
    for (int r = 0; r < nR; ++r) {
        const int* ri = rint + RINT * r;
        const double* rd = rdbl + RDBL * r;
        const int type = ri[0];
        const bool irr = ri[1] != 0;
        const int nl = ri[2], nr = ri[3];
        const auto lhs = side(nl, ri + 4, rd + 0, rd + 10);
        const auto rhs = side(nr, ri + 14, rd + 20, rd + 30);
        gpu::Arrhenius k(rd[40], rd[41], rd[42]);
        gpuReactionRate rate;
        if (type == 0) {
            rate = gpuReactionRate(k, irr);
        } else if (type == 1) {
            rate = gpuReactionRate(gpu::ThirdBodyArrhenius(k, tbe(nS, eff + nS * r)), irr);
        } else if (type == 2) {
            gpu::Arrhenius kinf(rd[43], rd[44], rd[45]);
            rate = gpuReactionRate(gpu::ArrheniusLindemannFallOff(k, kinf, gpuLindemannFallOffFunction(),
                                                                  tbe(nS, eff + nS * r)), irr);
        } else {
            gpu::Arrhenius kinf(rd[43], rd[44], rd[45]);
            gpuTroeFallOffFunction F(rd[46], rd[47], rd[48], rd[49]);
            rate = gpuReactionRate(gpu::ArrheniusTroeFallOff(k, kinf, F, tbe(nS, eff + nS * r)), irr);
        }
        gpuReaction reaction(m->thermos[0], lhs, rhs, nl, nr, rate, rxnTlow, rxnThigh);
        // set_reaction_thermo (makeGpuReactions.H:18-59) with the reference operators
        const auto& rr = reaction.rhs();
        const auto& ll = reaction.lhs();
        gpuThermo rhsThermo(rr[0].stoichCoeff * m->thermos[rr[0].index].W() * m->thermos[rr[0].index]);
        for (gLabel i = 1; i < gLabel(rr.size()); ++i) {
            rhsThermo += rr[i].stoichCoeff * m->thermos[rr[i].index].W() * m->thermos[rr[i].index];
        }
        gpuThermo lhsThermo(ll[0].stoichCoeff * m->thermos[ll[0].index].W() * m->thermos[ll[0].index]);
        for (gLabel i = 1; i < gLabel(ll.size()); ++i) {
            lhsThermo += ll[i].stoichCoeff * m->thermos[ll[i].index].W() * m->thermos[ll[i].index];
        }
        if (std::abs(lhsThermo.Y() - rhsThermo.Y()) > 0.1) {
            delete m;
            return nullptr;
        }
        reaction.get_thermo() = (lhsThermo == rhsThermo);
        m->reactions.push_back(reaction);
    }
    return m;
}

void ref_mech_destroy(void* h) { delete static_cast<RefMech*>(h); }

static void dump_thermo(const gpuThermo& t, double* o) {
    o[0] = t.Y();
    o[1] = t.W();
    o[2] = t.Tlow_;
    o[3] = t.Thigh_;
    o[4] = t.Tcommon_;
    for (int k = 0; k < 7; ++k) o[5 + k] = t.highCpCoeffs_[k];
    for (int k = 0; k < 7; ++k) o[12 + k] = t.lowCpCoeffs_[k];
}

// Processed tables: species thermo [nS][19] and reaction ΔThermo [nR][19]
// (Y, W, Tlow, Thigh, Tcommon, high[7], low[7]) plus per-reaction integer
// exponent flags [nR][20] (lhs then rhs; -1 beyond the side's length).
void ref_mech_tables(void* h, double* species_out, double* reaction_out, int* int_exp_out) {
    auto* m = static_cast<RefMech*>(h);
    for (int i = 0; i < m->nS; ++i) dump_thermo(m->thermos[i], species_out + 19 * i);
    for (int r = 0; r < m->nR; ++r) {
        const gpuReaction& R = m->reactions[r];
        dump_thermo(static_cast<const gpuThermo&>(R), reaction_out + 19 * r);
        for (int i = 0; i < 10; ++i) {
            int_exp_out[20 * r + i] = i < R.lhs_size_ ? int(R.lhs_[i].exponent.hasIntegerExponent()) : -1;
            int_exp_out[20 * r + 10 + i] = i < R.rhs_size_ ? int(R.rhs_[i].exponent.hasIntegerExponent()) : -1;
        }
    }
}

// Thermo functions of every species at (p, T): [nS][8] = Cp, Ha, Hs, S, Gstd, dCpdT, K, Kc
void ref_thermo_eval(void* h, double p, double T, double* out) {
    auto* m = static_cast<RefMech*>(h);
    for (int i = 0; i < m->nS; ++i) {
        const gpuThermo& t = m->thermos[i];
        double* o = out + 8 * i;
        o[0] = t.Cp(p, T);
        o[1] = t.Ha(p, T);
        o[2] = t.Hs(p, T);
        o[3] = t.S(p, T);
        o[4] = t.Gstd(T);
        o[5] = t.dCpdT(p, T);
        o[6] = t.K(p, T);
        o[7] = t.Kc(p, T);
    }
}

// Per-reaction quantities at a state y: [nR][6] = kf, kr, omega (derivatives
// path), Kc, dKcdTbyKc, dwdT (jacobian path).
void ref_reaction_eval(void* h, const double* y, double* out) {
    auto* m = static_cast<RefMech*>(h);
    const int nS = m->nS;
    Buf buf(nS);
    gpuMixture mix(m->thermos.data());
    std::vector<double> Ha(nS + 2), c(nS), ddc(nS);
    auto ys = mdspan<const gScalar, 1>(y, extents<1>{nS + 2});
    auto Has = mdspan<gScalar, 1>(Ha.data(), extents<1>{nS + 2});
    auto cs = mdspan<gScalar, 1>(c.data(), extents<1>{nS});
    mix.computeDerivativeRequired(ys, Has, cs);
    const double T = y[nS], p = y[nS + 1];
    auto cc = mdspan<const gScalar, 1>(c.data(), extents<1>{nS});
    for (int r = 0; r < m->nR; ++r) {
        const gpuReaction& R = m->reactions[r];
        double* o = out + 6 * r;
        o[0] = R.kf(p, T, cc);
        o[1] = R.kr(p, T, cc);
        o[2] = R.omega(p, T, cc);
        const auto kk = R.KcAnddKcTbyKc(p, T);
        o[3] = kk[0];
        o[4] = kk[1];
        auto ds = mdspan<gScalar, 1>(ddc.data(), extents<1>{nS});
        const auto prm = computeReactionParameters(R, cc, p, T, ds);
        o[5] = prm.dwdT;
    }
}

void ref_derivatives(void* h, int n, const double* y, double* dydx) {
    auto* m = static_cast<RefMech*>(h);
    const int ne = m->nS + 2;
    gpuODESystem sys(ne, m->nR, m->thermos.data(), m->reactions.data());
    Buf buf(m->nS);
    for (int c = 0; c < n; ++c) {
        auto ys = mdspan<const gScalar, 1>(y + ne * c, extents<1>{ne});
        auto ds = mdspan<gScalar, 1>(dydx + ne * c, extents<1>{ne});
        sys.derivatives(ys, ds, buf.b[0]);
    }
}

void ref_jacobian(void* h, int n, const double* y, double* dfdx, double* J) {
    auto* m = static_cast<RefMech*>(h);
    const int ne = m->nS + 2;
    gpuODESystem sys(ne, m->nR, m->thermos.data(), m->reactions.data());
    Buf buf(m->nS);
    for (int c = 0; c < n; ++c) {
        auto ys = mdspan<const gScalar, 1>(y + ne * c, extents<1>{ne});
        auto ds = mdspan<gScalar, 1>(dfdx + ne * c, extents<1>{ne});
        auto Js = mdspan<gScalar, 2>(J + ne * ne * c, extents<2>{ne, ne});
        sys.jacobian(ys, ds, Js, buf.b[0]);
    }
}

// LUDecompose + LUBacksubstitute on n_mats [m][m] matrices (in place) and
// right-hand sides b [n_mats][m] (in place).
void ref_lu(int m, int n_mats, double* A, int* piv, double* b) {
    std::vector<double> vv(m);
    for (int k = 0; k < n_mats; ++k) {
        auto As = mdspan<gScalar, 2>(A + m * m * k, extents<2>{m, m});
        auto ps = mdspan<gLabel, 1>(piv + m * k, extents<1>{m});
        auto vs = mdspan<gScalar, 1>(vv.data(), extents<1>{m});
        LUDecompose(As, ps, vs);
        auto Ac = mdspan<const gScalar, 2>(A + m * m * k, extents<2>{m, m});
        auto pc = mdspan<const gLabel, 1>(piv + m * k, extents<1>{m});
        auto bs = mdspan<gScalar, 1>(b + m * k, extents<1>{m});
        LUBacksubstitute(Ac, pc, bs);
    }
}

// One Rosenbrock attempt solve(y0, dydx0, dx, y) per state; returns err per state.
void ref_attempt(void* h, const OdeIn* o, int n, const double* y0, const double* dydx0,
                 const double* dx, double* y, double* err) {
    auto* m = static_cast<RefMech*>(h);
    const int ne = m->nS + 2;
    with_solver(*m, *o, [&](auto ode) {
        Buf buf(m->nS);
        for (int c = 0; c < n; ++c) {
            auto y0s = mdspan<const gScalar, 1>(y0 + ne * c, extents<1>{ne});
            auto d0s = mdspan<const gScalar, 1>(dydx0 + ne * c, extents<1>{ne});
            auto ys = mdspan<gScalar, 1>(y + ne * c, extents<1>{ne});
            err[c] = ode.solve(y0s, d0s, dx[c], ys, buf.b[0]);
        }
    });
}

// singleCellSolver semantics (singleCellSolver.H:27-51) per cell, with the
// counting wrapper: Y [n][ne] and deltaTChem [n] in/out, counts [n][2] =
// (accepted, attempts). deltaT_cell may be NULL (uniform deltaT).
void ref_cells_counted(void* h, const OdeIn* o, double Treact, int n, double deltaT,
                       const double* deltaT_cell, double* Y, double* deltaTChem, int* counts,
                       int nthreads) {
    auto* m = static_cast<RefMech*>(h);
    const int nS = m->nS, ne = nS + 2;
    with_solver(*m, *o, [&](auto ode_proto) {
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : omp_get_max_threads())
        {
            Buf buf(nS);
            auto ode = ode_proto;
#pragma omp for schedule(dynamic, 1)
            for (int c = 0; c < n; ++c) {
                ode.accepted = 0;
                ode.attempts = 0;
                const double dT = deltaT_cell ? deltaT_cell[c] : deltaT;
                auto Ys = mdspan<gScalar, 1>(Y + ne * c, extents<1>{ne});
                if (Ys[nS] > Treact) {
                    gScalar timeLeft = dT;
                    while (timeLeft > gpuSmall) {
                        gScalar dt = timeLeft;
                        odeSolve(ode, 0, dt, Ys, deltaTChem[c], buf.b[0]);
                        for (int i = 0; i < nS; ++i) Ys[i] = fmax(0.0, Ys[i]);
                        timeLeft -= dt;
                    }
                } else {
                    deltaTChem[c] = dT;
                }
                counts[2 * c] = int(ode.accepted);
                counts[2 * c + 1] = int(ode.attempts);
            }
        }
    });
}

// The reference's own singleCellSolver functor over cells (no counting) —
// the unmodified per-cell path, used as the timed CPU baseline.
void ref_cells(void* h, const OdeIn* o, double Treact, int n, double deltaT, double* Y,
               double* deltaTChem, int nthreads) {
    auto* m = static_cast<RefMech*>(h);
    const int nS = m->nS, ne = nS + 2;
    gpuODESystem sys(ne, m->nR, m->thermos.data(), m->reactions.data());
    const gpuODESolver solver = make_gpuODESolver(sys, to_inputs(*o));
#pragma omp parallel num_threads(nthreads > 0 ? nthreads : omp_get_max_threads())
    {
        Buf buf(nS);
#pragma omp for schedule(dynamic, 1)
        for (int c = 0; c < n; ++c) {
            // one-cell views so that each thread uses its own scratch buffer
            auto Ys = mdspan<gScalar, 2>(Y + ne * c, extents<2>{1, ne});
            auto dts = mdspan<gScalar, 1>(deltaTChem + c, extents<1>{1});
            auto bs = mdspan<gpuBuffer, 1>(buf.b.data(), extents<1>{1});
            singleCellSolver op(deltaT, nS, dts, Ys, bs, solver, Treact);
            op(0);
        }
    }
}

// Host arithmetic of GpuKernelEvaluator::computeRR after the kernel
// (gpuKernelEvaluator.cu:84-96): RR, min before clamping, clamp.
double ref_compute_rr_host(int n, int nS, double deltaT, double deltaTChemMax, const double* rho,
                           const double* Y0, const double* Ynew, double* deltaTChemNew, double* RR) {
    const int ne = nS + 2;
    for (int j = 0; j < n; ++j) {
        for (int i = 0; i < nS; ++i) {
            RR[j * nS + i] = rho[j] * (Ynew[j * ne + i] - Y0[j * ne + i]) / deltaT;
        }
    }
    double mn = deltaTChemNew[0];
    for (int j = 1; j < n; ++j) mn = std::min(mn, deltaTChemNew[j]);
    for (int j = 0; j < n; ++j) deltaTChemNew[j] = std::min(deltaTChemNew[j], deltaTChemMax);
    return mn;
}

// The plugin's per-cell side paths (gpuChemistryModel.C) on the reference's
// own reactions: c_i = rho Y_i / W_i (:163-166); calculate() :145-186 (RR,
// dNdtByV in mechanism order times W), tc() :366-427 with omegaf = kf Cf and
// omegar = kr Cr split as gpuReaction::omega computes them (gpuReaction.H:472-488).
void ref_cell_fields(void* h, int n, const double* rho, const double* y, double* RR, double* tc) {
    auto* m = static_cast<RefMech*>(h);
    const int nS = m->nS, ne = nS + 2;
    std::vector<double> c(nS), dN(nS);
    auto cc = mdspan<const gScalar, 1>(c.data(), extents<1>{nS});
    for (int j = 0; j < n; ++j) {
        const double* yj = y + (size_t)j * ne;
        const double T = yj[nS], p = yj[nS + 1];
        for (int i = 0; i < nS; ++i) c[i] = rho[j] * yj[i] / m->thermos[i].W();
        if (RR) {
            std::fill(dN.begin(), dN.end(), 0.0);
            auto ds = mdspan<gScalar, 1>(dN.data(), extents<1>{nS});
            for (int r = 0; r < m->nR; ++r) m->reactions[r].dNdtByV(p, T, cc, ds);
            for (int i = 0; i < nS; ++i) RR[(size_t)j * nS + i] = dN[i] * m->thermos[i].W();
        }
        if (tc) {
            double sumW = 0, sumWRateByCTot = 0;
            for (int r = 0; r < m->nR; ++r) {
                const gpuReaction& R = m->reactions[r];
                const gScalar clippedT = fmin(fmax(T, R.Tlow()), R.Thigh());
                const gScalar kf = R.kf(p, clippedT, cc);
                const gScalar kr = R.kr(kf, p, clippedT, R.Kc(p, clippedT), cc);
                const gScalar omegaf = kf * R.calcCf(R.lhsPowers(cc));
                const gScalar omegar = kr * R.calcCr(R.rhsPowers(cc));
                double wf = 0;
                for (size_t s = 0; s < R.rhs().size(); ++s) wf += R.rhs()[s].stoichCoeff * omegaf;
                sumW += wf;
                sumWRateByCTot += wf * wf;
                double wr = 0;
                for (size_t s = 0; s < R.lhs().size(); ++s) wr += R.lhs()[s].stoichCoeff * omegar;
                sumW += wr;
                sumWRateByCTot += wr * wr;
            }
            double ctot = 0;
            for (int i = 0; i < nS; ++i) ctot += c[i];
            tc[j] = sumWRateByCTot == 0 ? gpuVGreat : sumW / sumWRateByCTot * ctot;
        }
    }
}

// reactionRR(r) :188-229 and specieReactionRR(r) :231-298.
void ref_reaction_fields(void* h, int n, int r, const double* rho, const double* y, double* omega, double* RR) {
    auto* m = static_cast<RefMech*>(h);
    const int nS = m->nS, ne = nS + 2;
    const gpuReaction& R = m->reactions[r];
    std::vector<double> c(nS);
    auto cc = mdspan<const gScalar, 1>(c.data(), extents<1>{nS});
    for (int j = 0; j < n; ++j) {
        const double* yj = y + (size_t)j * ne;
        for (int i = 0; i < nS; ++i) c[i] = rho[j] * yj[i] / m->thermos[i].W();
        const double om = R.omega(yj[nS + 1], yj[nS], cc);
        if (omega) omega[j] = om;
        if (RR) {
            double* o = RR + (size_t)j * nS;
            std::fill(o, o + nS, 0.0);
            R.dNdtByV(om, mdspan<gScalar, 1>(o, extents<1>{nS}));
            for (int i = 0; i < nS; ++i) o[i] = o[i] * m->thermos[i].W();
        }
    }
}

// Qdot() :429-450 with gpuThermo::Hf (gpuThermo.H:243-254) for hf.
void ref_qdot(void* h, int n, const double* RR, double* qdot) {
    auto* m = static_cast<RefMech*>(h);
    for (int j = 0; j < n; ++j) {
        double q = 0;
        for (int i = 0; i < m->nS; ++i) q -= m->thermos[i].Hf() * RR[(size_t)j * m->nS + i];
        qdot[j] = q;
    }
}

// Reference constants (gpu_constants.H): RR, pStd, Tstd, NNA, k, vGreat, vSmall, small, great
void ref_constants(double* out) {
    out[0] = gpuRR;
    out[1] = gpupStd;
    out[2] = gpuTstd;
    out[3] = gpuNNA;
    out[4] = gpuk;
    out[5] = gpuVGreat;
    out[6] = gpuVSmall;
    out[7] = gpuSmall;
    out[8] = gpuGreat;
}

}  // extern "C"
