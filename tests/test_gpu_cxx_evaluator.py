"""The C++ seam on a B200: a C++17 program compiled against
include/gpufoam_b200.hpp builds FoamGpu::GpuKernelEvaluator the way the
plugin's makeEvaluator does (gpuChemistryModel.C:55-81: nCells, nEqns, nSpecie,
the thermos, the reactions, the ODE inputs as the reference's
gpuODESolverInputs struct with the solver by name, Treact) and runs computeRR
and computeYNew on the golden cells of the 10-species mechanism. The results
are compared with the reference's own integration and host arithmetic
(gpuKernelEvaluator.cu:65-97: RR = rho (Ynew - Y0) / deltaT, deltaTChemNew
clamped, minDeltaT before clamping) stored in tests/golden/h2size.npz.
"""
import ctypes as C
import os
import shutil
import subprocess

import numpy as np
import pytest

from gpufoam_b200 import _native as N
from gpufoam_b200 import evaluator as E
from tests.parity import assert_states_close
from tests.test_oracle import fixture_mech, load

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "gpufoam_b200")

PROGRAM = r"""
#include <cstdio>
#include <fstream>
#include <string>
#include <vector>
#include "gpufoam_b200.hpp"

// the reference's gpuODESolverInputs (gpuOde/gpuODESolverInputs.H:9-23), as
// read_gpuODESolverInputs returns it
namespace FoamGpu {
struct gpuODESolverInputs {
    std::string name;
    double absTol, relTol;
    int maxSteps;
    double safeScale, alphaInc, alphaDec, minScale, maxScale;
};
}  // namespace FoamGpu

template <class T>
std::vector<T> load(const std::string& path, size_t n) {
    std::vector<T> v(n);
    std::ifstream f(path, std::ios::binary);
    f.read(reinterpret_cast<char*>(v.data()), std::streamsize(n * sizeof(T)));
    if (!f) throw std::runtime_error("short file " + path);
    return v;
}

template <class T>
void save(const std::string& path, const std::vector<T>& v) {
    std::ofstream f(path, std::ios::binary);
    f.write(reinterpret_cast<const char*>(v.data()), std::streamsize(v.size() * sizeof(T)));
}

int main(int argc, char** argv) {
    if (argc != 7) return 2;
    const std::string dir = argv[1];
    const int nS = std::stoi(argv[2]), nR = std::stoi(argv[3]), n = std::stoi(argv[4]);
    const double deltaT = std::stod(argv[5]), deltaTChemMax = std::stod(argv[6]);
    const int ne = nS + 2;
    auto thermos = load<gf_thermo>(dir + "/thermos.bin", nS);
    auto reactions = load<gf_reaction>(dir + "/reactions.bin", nR);
    auto eff = load<double>(dir + "/eff.bin", size_t(nR) * nS);
    for (int r = 0; r < nR; ++r)
        reactions[r].efficiencies = reactions[r].rate_type == GF_RATE_ARRHENIUS ? nullptr : &eff[size_t(r) * nS];
    auto Y = load<double>(dir + "/Y.bin", size_t(n) * ne);
    auto rho = load<double>(dir + "/rho.bin", n);
    auto dtc = load<double>(dir + "/dtc.bin", n);
    const FoamGpu::gpuODESolverInputs in{"Rosenbrock34", 1e-8, 1e-4, 10000, 0.9, 0.2, 0.25, 0.2, 10.0};
    FoamGpu::GpuKernelEvaluator evaluator(n, ne, nS, thermos, reactions, in, 0.0);
    auto rr = evaluator.computeRR(deltaT, deltaTChemMax, rho, dtc, Y);
    auto yn = evaluator.computeYNew(deltaT, deltaTChemMax, dtc, Y);
    save(dir + "/RR.bin", std::get<0>(rr));
    save(dir + "/dtc_rr.bin", std::get<1>(rr));
    save(dir + "/min.bin", std::vector<double>{std::get<2>(rr)});
    save(dir + "/Ynew.bin", yn.first);
    save(dir + "/dtc_ynew.bin", yn.second);
    try {
        FoamGpu::gpuODESolverInputs bad = in;
        bad.name = "Euler";
        FoamGpu::GpuKernelEvaluator e2(n, ne, nS, thermos, reactions, bad);
        return 3;
    } catch (const std::logic_error&) {
    }
    std::printf("ok\n");
    return 0;
}
"""


def test_cxx_evaluator_compute_rr(tmp_path):
    from gpufoam_b200 import build
    build.build()
    if not shutil.which("g++"):
        pytest.skip("no host C++ compiler")
    g = load("h2size")
    raw = fixture_mech(g)
    nS, nR = raw.n_species, raw.n_reactions
    thermos = E.make_gpu_thermos(raw)
    reactions, _ = E.make_gpu_reactions(raw, thermos)
    d = str(tmp_path)
    with open(os.path.join(d, "thermos.bin"), "wb") as f:
        f.write(bytes(thermos))
    with open(os.path.join(d, "reactions.bin"), "wb") as f:
        f.write(bytes(reactions)[:nR * C.sizeof(N.GfReaction)])
    eff = np.zeros((nR, nS))
    for r, rx in enumerate(raw.reactions):
        if rx.efficiencies is not None:
            eff[r] = rx.efficiencies
    eff.tofile(os.path.join(d, "eff.bin"))
    cells = np.ascontiguousarray(g["cells"])
    n = cells.shape[0]
    cells.tofile(os.path.join(d, "Y.bin"))
    np.ascontiguousarray(g["rr_rho"]).tofile(os.path.join(d, "rho.bin"))
    np.full(n, float(g["deltaTChem0"])).tofile(os.path.join(d, "dtc.bin"))
    src = os.path.join(d, "evaluator.cpp")
    exe = os.path.join(d, "evaluator")
    with open(src, "w") as f:
        f.write(PROGRAM)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Wextra", "-Werror", "-O2", "-I", INC, "-o", exe, src,
                    "-L", LIBDIR, "-lgpufoam_b200", f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True)
    deltaT, dtcmax = float(g["deltaT"]), float(g["rr_dtcmax"])
    out = subprocess.run([exe, d, str(nS), str(nR), str(n), repr(deltaT), repr(dtcmax)], capture_output=True,
                         text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", (out.returncode, out.stdout, out.stderr)
    RR = np.fromfile(os.path.join(d, "RR.bin")).reshape(n, nS)
    dtn = np.fromfile(os.path.join(d, "dtc_rr.bin"))
    mn = float(np.fromfile(os.path.join(d, "min.bin"))[0])
    Ynew = np.fromfile(os.path.join(d, "Ynew.bin")).reshape(n, nS + 2)
    dtn2 = np.fromfile(os.path.join(d, "dtc_ynew.bin"))
    # computeYNew: the integrated states and unclamped chemistry steps of the reference
    assert_states_close(Ynew, g["cells34_Y"], nS, 1e-4, "C++ computeYNew")
    np.testing.assert_allclose(dtn2, g["cells34_dtc"], rtol=1e-6)
    # computeRR: RR inherits the state tolerance; clamped steps and the min before clamping
    tolY = 1e-9 + 10 * 1e-4 * np.abs(g["cells34_Y"][:, :nS])
    tol = g["rr_rho"][:, None] * tolY / deltaT
    assert (np.abs(RR - g["rr_RR"]) <= tol).all()
    assert (dtn <= dtcmax).all()
    np.testing.assert_allclose(dtn, g["rr_dtc"], rtol=1e-6)
    np.testing.assert_allclose(mn, float(g["rr_min"]), rtol=1e-6)
