// Header-only C++ drop-in for FoamGpu::GpuKernelEvaluator over the C ABI of
// gpufoam_b200.h. Same class name, constructor role and member signatures as
// the reference (gpu_chemistry/src/gpuKernelEvaluator/gpuKernelEvaluator/
// gpuKernelEvaluator.H:18-85): computeYNew (gpuKernelEvaluator.cu:35-63) and
// computeRR (gpuKernelEvaluator.cu:65-97) on host vectors; the mechanism comes
// in as the C ABI's flat structs (gf_thermo with coefficients x R,
// gf_reaction with its reaction thermo), which the plugin's loaders fill. The
// ODE inputs come in as the reference's own gpuODESolverInputs
// (gpuOde/gpuODESolverInputs.H:9-23, the struct read_gpuODESolverInputs
// returns: any struct with its members name, absTol, ... is accepted) or as a
// gf_ode_inputs. Errors become std::runtime_error with the library's message;
// an unknown solver name throws as make_gpuODESolver does (makeGpuOdeSolver.H:28).
#ifndef GPUFOAM_B200_HPP
#define GPUFOAM_B200_HPP

#include <stdexcept>
#include <string>
#include <tuple>
#include <utility>
#include <vector>

#include "gpufoam_b200.h"

namespace FoamGpu {

// gpuODESolverInputs (gpuOde/gpuODESolverInputs.H:9-23) with the reference's
// defaults (gpuOde/readGpuOdeInputs.H:8-26) and the solver by name.
inline gf_ode_inputs make_gf_ode_inputs(const std::string& name, double absTol, double relTol,
                                        int maxSteps = 10000, double safeScale = 0.9, double alphaInc = 0.2,
                                        double alphaDec = 0.25, double minScale = 0.2, double maxScale = 10.0) {
    gf_ode_inputs in{};
    if (name == "Rosenbrock12") {
        in.solver = GF_ROSENBROCK12;
    } else if (name == "Rosenbrock23") {
        in.solver = GF_ROSENBROCK23;
    } else if (name == "Rosenbrock34") {
        in.solver = GF_ROSENBROCK34;
    } else {
        throw std::logic_error("Invalid ODE Solver type: " + name);
    }
    in.absTol = absTol;
    in.relTol = relTol;
    in.maxSteps = maxSteps;
    in.safeScale = safeScale;
    in.alphaInc = alphaInc;
    in.alphaDec = alphaDec;
    in.minScale = minScale;
    in.maxScale = maxScale;
    return in;
}

class GpuKernelEvaluator {
public:
    GpuKernelEvaluator() = default;

    // The reference's constructor with its gpuODESolverInputs (solver by name).
    template <class OdeInputs, class = decltype(std::declval<const OdeInputs&>().name.c_str(),
                                                std::declval<const OdeInputs&>().maxScale)>
    GpuKernelEvaluator(int nCells, int nEqns, int nSpecie, const std::vector<gf_thermo>& thermos,
                       const std::vector<gf_reaction>& reactions, const OdeInputs& odeInputs, double Treact = 0.0)
        : GpuKernelEvaluator(nCells, nEqns, nSpecie, thermos, reactions,
                             make_gf_ode_inputs(odeInputs.name, odeInputs.absTol, odeInputs.relTol,
                                                int(odeInputs.maxSteps), odeInputs.safeScale, odeInputs.alphaInc,
                                                odeInputs.alphaDec, odeInputs.minScale, odeInputs.maxScale),
                             Treact) {}

    GpuKernelEvaluator(int nCells, int nEqns, int nSpecie, const std::vector<gf_thermo>& thermos,
                       const std::vector<gf_reaction>& reactions, const gf_ode_inputs& odeInputs,
                       double Treact = 0.0)
        : nCells_(nCells), nEqns_(nEqns), nSpecie_(nSpecie) {
        if (nEqns != nSpecie + 2 || int(thermos.size()) != nSpecie)
            throw std::invalid_argument("GpuKernelEvaluator: nEqns must be nSpecie + 2, one thermo per specie");
        const gf_mech_desc d{nSpecie, int(reactions.size()), thermos.data(), reactions.data()};
        check(gf_mech_create(&d, &mech_));
        const gf_mech* m = mech_;
        const int s = gf_solver_create(&m, 1, &odeInputs, Treact, &solver_);
        if (s != GF_OK) {
            gf_mech_destroy(mech_);
            mech_ = nullptr;
            check(s);
        }
    }
    GpuKernelEvaluator(const GpuKernelEvaluator&) = delete;
    GpuKernelEvaluator& operator=(const GpuKernelEvaluator&) = delete;
    ~GpuKernelEvaluator() {
        gf_solver_destroy(solver_);
        gf_mech_destroy(mech_);
    }

    // (Ynew [nCells * nEqns], deltaTChemNew [nCells]), deltaTChemNew not clamped
    std::pair<std::vector<double>, std::vector<double>> computeYNew(double deltaT, double deltaTChemMax,
                                                                     const std::vector<double>& deltaTChem,
                                                                     const std::vector<double>& Y) {
        const int n = int(deltaTChem.size());
        if (Y.size() != size_t(n) * nEqns_) throw std::invalid_argument("computeYNew: Y size");
        std::vector<double> Ynew(Y.size()), dtc(n);
        check(gf_compute_ynew(solver_, n, deltaT, deltaTChemMax, deltaTChem.data(), Y.data(), Ynew.data(),
                              dtc.data()));
        return {std::move(Ynew), std::move(dtc)};
    }

    // (RR [nCells * nSpecie], deltaTChemNew [nCells] clamped, minDeltaT before clamping)
    std::tuple<std::vector<double>, std::vector<double>, double> computeRR(double deltaT, double deltaTChemMax,
                                                                           const std::vector<double>& rho,
                                                                           const std::vector<double>& deltaTChem,
                                                                           const std::vector<double>& Y) {
        const int n = int(rho.size());
        if (deltaTChem.size() != size_t(n) || Y.size() != size_t(n) * nEqns_)
            throw std::invalid_argument("computeRR: array sizes");
        std::vector<double> RR(size_t(n) * nSpecie_), dtc(n);
        double minDeltaT = 0.0;
        check(gf_compute_rr(solver_, n, deltaT, deltaTChemMax, rho.data(), deltaTChem.data(), Y.data(), RR.data(),
                            dtc.data(), &minDeltaT));
        return std::make_tuple(std::move(RR), std::move(dtc), minDeltaT);
    }

    // computeRR with a flow time step per cell (local time stepping; the
    // reference's solve(const scalarField&) throws, gpuChemistryModel.C:328-333)
    std::tuple<std::vector<double>, std::vector<double>, double> computeRR(const std::vector<double>& deltaT,
                                                                           double deltaTChemMax,
                                                                           const std::vector<double>& rho,
                                                                           const std::vector<double>& deltaTChem,
                                                                           const std::vector<double>& Y) {
        const int n = int(rho.size());
        if (deltaT.size() != size_t(n) || deltaTChem.size() != size_t(n) || Y.size() != size_t(n) * nEqns_)
            throw std::invalid_argument("computeRR: array sizes");
        std::vector<double> RR(size_t(n) * nSpecie_), dtc(n);
        double minDeltaT = 0.0;
        check(gf_compute_rr_lts(solver_, n, deltaT.data(), deltaTChemMax, rho.data(), deltaTChem.data(), Y.data(),
                                RR.data(), dtc.data(), &minDeltaT));
        return std::make_tuple(std::move(RR), std::move(dtc), minDeltaT);
    }

    int nCells() const { return nCells_; }
    gf_solver* solver() { return solver_; }
    gf_mech* mechanism() { return mech_; }

private:
    static void check(int s) {
        if (s != GF_OK) {
            std::string msg = gf_strerror(s);
            if (s == GF_ERR_CUDA) msg += std::string(": ") + gf_last_cuda_error();
            throw std::runtime_error("gpufoam_b200: " + msg);
        }
    }
    int nCells_ = 0, nEqns_ = 0, nSpecie_ = 0;
    gf_mech* mech_ = nullptr;
    gf_solver* solver_ = nullptr;
};

}  // namespace FoamGpu

#endif
