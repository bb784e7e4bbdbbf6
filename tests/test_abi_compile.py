"""The boundary as a C or C++ caller sees it, on CPU: a C99 program and a C++17
program compile against include/gpufoam_b200.h / gpufoam_b200.hpp with
warnings as errors, link libgpufoam_b200.so and run the entry points that need
no device (the loader arithmetic, status strings, argument errors)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from gpufoam_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INC = os.path.join(ROOT, "include")
LIBDIR = os.path.join(ROOT, "gpufoam_b200")

C_SRC = r"""
#include <stdio.h>
#include "gpufoam_b200.h"
int main(void) {
    double hi[7] = {3, 0, 0, 0, 0, -900, -2}, lo[7] = {2.3, 0.008, -1.9e-05, 2e-08, -7e-12, -917, 0.68};
    gf_thermo t;
    gf_mech* m = 0;
    int s = gf_thermo_from_nasa(1.0, 2.016, 200, 5000, 1000, hi, lo, &t);
    int e = gf_mech_create(0, &m);
    printf("%d %d %d %s|%.17g %.17g\n", gf_abi_version(), s, e, gf_strerror(2), t.high[0], t.low[5]);
    return 0;
}
"""

CXX_SRC = r"""
#include <cstdio>
#include <stdexcept>
#include "gpufoam_b200.hpp"
// both computeRR overloads compile (the per-cell one: local time stepping)
double use_overloads(FoamGpu::GpuKernelEvaluator& ev) {
    std::vector<double> rho{1.0}, dtc{1e-7}, Y(4, 0.0), dT{1e-6};
    auto a = ev.computeRR(1e-6, 1.0, rho, dtc, Y);
    auto b = ev.computeRR(dT, 1.0, rho, dtc, Y);
    return std::get<2>(a) + std::get<2>(b);
}
int main() {
    int fails = 0;
    gf_ode_inputs in = FoamGpu::make_gf_ode_inputs("Rosenbrock23", 1e-8, 1e-4);
    if (in.solver != GF_ROSENBROCK23 || in.maxSteps != 10000 || in.maxScale != 10.0) ++fails;
    try { FoamGpu::make_gf_ode_inputs("Euler", 1e-8, 1e-4); ++fails; } catch (const std::logic_error&) {}
    try {
        std::vector<gf_thermo> th(2);
        std::vector<gf_reaction> rx;
        FoamGpu::GpuKernelEvaluator ev(4, 5, 2, th, rx, in);  // nEqns != nSpecie + 2
        ++fails;
    } catch (const std::invalid_argument&) {}
    std::printf("%d\n", fails);
    return fails;
}
"""


def _compile_and_run(tmp_path, compiler, std, src, name):
    exe = os.path.join(tmp_path, name)
    srcf = exe + (".c" if compiler == "gcc" else ".cpp")
    with open(srcf, "w") as f:
        f.write(src)
    subprocess.run([compiler, f"-std={std}", "-Wall", "-Wextra", "-Werror", "-I", INC, "-o", exe, srcf, "-L", LIBDIR,
                    "-lgpufoam_b200", f"-Wl,-rpath,{LIBDIR}"], check=True, capture_output=True, text=True)
    return subprocess.run([exe], check=True, capture_output=True, text=True, timeout=60).stdout


@pytest.fixture(scope="module")
def built():
    from gpufoam_b200 import build as B
    B.build()
    if not shutil.which("gcc") or not shutil.which("g++"):
        pytest.skip("no host compiler")


def test_c_program(built, tmp_path):
    out = _compile_and_run(str(tmp_path), "gcc", "c99", C_SRC, "c_abi").strip()
    head, vals = out.split("|")
    ver, s, e, msg = head.split(" ", 3)
    assert (int(ver), int(s), int(e), msg) == (1, N.GF_OK, 1, "Invalid ODE Solver type")
    # the same x R scaling as the Python loader (makeGpuThermo.H:41-44)
    R = 6.02214e+26 * 1.38065e-23 / 2.016
    assert np.array_equal(np.array([float(v) for v in vals.split()]), np.array([R * 3.0, R * -917.0]))


def test_cxx_evaluator_header(built, tmp_path):
    assert _compile_and_run(str(tmp_path), "g++", "c++17", CXX_SRC, "cxx_abi").strip() == "0"
