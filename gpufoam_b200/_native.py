"""ctypes binding of the C ABI in include/gpufoam_b200.h.

The shared library libgpufoam_b200.so is built in-tree (gpufoam_b200/build.py).
There is no fallback: if the library is missing or fails to load, every entry
point raises.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("GPUFOAM_LIB", os.path.join(HERE, "libgpufoam_b200.so"))

GF_MAX_REACTION_WIDTH = 10
GF_MAX_SPECIES = 300

GF_OK = 0
STATUS_NAMES = {
    0: "GF_OK", 1: "GF_ERR_INVALID_ARGUMENT", 2: "GF_ERR_UNKNOWN_SOLVER", 3: "GF_ERR_UNSUPPORTED",
    4: "GF_ERR_MASS_IMBALANCE", 5: "GF_ERR_CUDA", 6: "GF_ERR_NO_DEVICE", 7: "GF_ERR_OUT_OF_MEMORY",
    8: "GF_ERR_CELL_FAILURE",
}
CELL_OK, CELL_STEP_UNDERFLOW, CELL_MAX_STEPS, CELL_NONFINITE, CELL_SKIPPED, CELL_BAD_MECHANISM = range(6)

# every symbol the header declares
EXPORTS = [
    "gf_thermo_from_nasa", "gf_reaction_thermo", "gf_mech_create", "gf_mech_destroy", "gf_mech_info",
    "gf_solver_create", "gf_solver_destroy", "gf_solver_set_launch", "gf_solver_get_launch", "gf_solve",
    "gf_compute_rr", "gf_compute_ynew", "gf_rates", "gf_jacobian", "gf_lu_decompose", "gf_lu_backsubstitute",
    "gf_strerror", "gf_abi_version", "gf_last_cuda_error", "gf_measure_fp64_peak", "gf_solve_noalloc",
    "gf_solve_record", "gf_adjoint", "gf_solve_graph_create", "gf_solve_graph_set_delta_t",
    "gf_solve_graph_launch", "gf_solve_graph_stats", "gf_solve_graph_destroy", "gf_cell_rates",
    "gf_reaction_rates", "gf_qdot", "gf_gather_states", "gf_scatter_rates", "gf_compute_rr_lts",
    "gf_lu_factor_solve", "gf_solver_info",
]


class GfThermo(C.Structure):
    _fields_ = [("Y", C.c_double), ("W", C.c_double), ("Tlow", C.c_double), ("Thigh", C.c_double),
                ("Tcommon", C.c_double), ("high", C.c_double * 7), ("low", C.c_double * 7)]


class GfSpecieCoeff(C.Structure):
    _fields_ = [("index", C.c_int), ("integer_exponent", C.c_int), ("stoich", C.c_double),
                ("exponent", C.c_double)]


class GfReaction(C.Structure):
    _fields_ = [("thermo", GfThermo), ("n_lhs", C.c_int), ("n_rhs", C.c_int),
                ("lhs", GfSpecieCoeff * GF_MAX_REACTION_WIDTH), ("rhs", GfSpecieCoeff * GF_MAX_REACTION_WIDTH),
                ("rate_type", C.c_int), ("irreversible", C.c_int),
                ("A", C.c_double), ("beta", C.c_double), ("Ta", C.c_double),
                ("Ainf", C.c_double), ("betainf", C.c_double), ("Tainf", C.c_double),
                ("troe_alpha", C.c_double), ("troe_Tsss", C.c_double), ("troe_Ts", C.c_double),
                ("troe_Tss", C.c_double), ("efficiencies", C.POINTER(C.c_double)),
                ("Tlow", C.c_double), ("Thigh", C.c_double)]


class GfMechDesc(C.Structure):
    _fields_ = [("n_species", C.c_int), ("n_reactions", C.c_int), ("thermos", C.POINTER(GfThermo)),
                ("reactions", C.POINTER(GfReaction))]


class GfOdeInputs(C.Structure):
    _fields_ = [("solver", C.c_int), ("absTol", C.c_double), ("relTol", C.c_double), ("maxSteps", C.c_int),
                ("safeScale", C.c_double), ("alphaInc", C.c_double), ("alphaDec", C.c_double),
                ("minScale", C.c_double), ("maxScale", C.c_double)]


class GfLaunchConfig(C.Structure):
    _fields_ = [("kind", C.c_int), ("threads_per_cell", C.c_int), ("scratch_in_shared", C.c_int),
                ("cells_per_block", C.c_int), ("blocks_per_sm", C.c_int), ("register_budget", C.c_int),
                ("lu_panel", C.c_int), ("specialize", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class GfStats(C.Structure):
    _fields_ = [("accepted_steps", C.c_longlong), ("attempts", C.c_longlong), ("failed_cells", C.c_longlong),
                ("min_delta_t", C.c_double)]


class GfError(RuntimeError):
    def __init__(self, status: int, where: str, lib=None):
        msg = f"{where}: {STATUS_NAMES.get(status, status)}"
        if lib is not None:
            try:
                msg += f" ({lib.gf_strerror(status).decode()})"
                if status == 5:
                    msg += f": {lib.gf_last_cuda_error().decode()}"
            except Exception:
                pass
        super().__init__(msg)
        self.status = status


_lib = None


def load() -> C.CDLL:
    """Load the native library (raises if it is missing)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"gpufoam_b200 native library not built: {LIB_PATH} "
                          "(run python -m gpufoam_b200.build)")
    lib = C.CDLL(LIB_PATH)
    vp, ip, dp = C.c_void_p, C.c_int, C.c_double
    P = C.POINTER
    lib.gf_thermo_from_nasa.argtypes = [dp, dp, dp, dp, dp, P(dp), P(dp), P(GfThermo)]
    lib.gf_reaction_thermo.argtypes = [P(GfThermo), ip, ip, P(GfSpecieCoeff), ip, P(GfSpecieCoeff), P(GfThermo)]
    lib.gf_mech_create.argtypes = [P(GfMechDesc), P(vp)]
    lib.gf_mech_destroy.argtypes = [vp]
    lib.gf_mech_destroy.restype = None
    lib.gf_mech_info.argtypes = [vp, P(ip), P(ip), P(C.c_longlong)]
    lib.gf_solver_create.argtypes = [P(vp), ip, P(GfOdeInputs), dp, P(vp)]
    lib.gf_solver_destroy.argtypes = [vp]
    lib.gf_solver_destroy.restype = None
    lib.gf_solver_set_launch.argtypes = [vp, P(GfLaunchConfig)]
    lib.gf_solver_get_launch.argtypes = [vp, P(GfLaunchConfig)]
    lib.gf_solver_info.argtypes = [vp, P(ip), P(ip), P(ip)]
    lib.gf_solve.argtypes = [vp, ip, dp, vp, dp, vp, vp, vp, ip, vp, vp, vp, ip, vp, vp, P(GfStats), vp]
    lib.gf_compute_rr.argtypes = [vp, ip, dp, dp, vp, vp, vp, vp, vp, P(dp)]
    lib.gf_compute_ynew.argtypes = [vp, ip, dp, dp, vp, vp, vp, vp]
    lib.gf_compute_rr_lts.argtypes = [vp, ip, vp, dp, vp, vp, vp, vp, vp, P(dp)]
    lib.gf_rates.argtypes = [vp, ip, vp, vp, vp]
    lib.gf_jacobian.argtypes = [vp, ip, vp, vp, vp, vp]
    lib.gf_lu_decompose.argtypes = [ip, ip, vp, vp, vp]
    lib.gf_lu_backsubstitute.argtypes = [ip, ip, vp, vp, vp, vp]
    lib.gf_lu_factor_solve.argtypes = [ip, ip, vp, vp, vp, ip, ip, ip, vp]
    lib.gf_measure_fp64_peak.argtypes = [dp, P(dp)]
    lib.gf_solve_noalloc.argtypes = [vp, P(GfOdeInputs), dp, ip, dp, vp, dp, vp, vp, ip, vp, vp, vp, ip, vp, vp,
                                     P(GfStats), vp]
    lib.gf_solve_record.argtypes = [vp, ip, dp, vp, ip, vp, vp, vp, vp, vp, ip, vp]
    lib.gf_adjoint.argtypes = [vp, ip, vp, ip, vp, vp, vp, vp, vp, ip, vp, vp, vp, vp]
    lib.gf_solve_graph_create.argtypes = [vp, ip, dp, vp, dp, vp, vp, vp, ip, vp, vp, vp, ip, vp, vp, P(vp)]
    lib.gf_solve_graph_set_delta_t.argtypes = [vp, dp]
    lib.gf_solve_graph_launch.argtypes = [vp, vp]
    lib.gf_solve_graph_stats.argtypes = [vp, P(GfStats)]
    lib.gf_solve_graph_destroy.argtypes = [vp]
    lib.gf_solve_graph_destroy.restype = None
    lib.gf_cell_rates.argtypes = [vp, ip, vp, vp, ip, vp, ip, vp, vp]
    lib.gf_reaction_rates.argtypes = [vp, ip, ip, vp, vp, ip, vp, vp, ip, vp]
    lib.gf_qdot.argtypes = [vp, ip, vp, ip, vp, vp]
    lib.gf_gather_states.argtypes = [ip, ip, P(vp), vp, vp, vp, ip, vp]
    lib.gf_scatter_rates.argtypes = [ip, ip, vp, ip, P(vp), vp]
    lib.gf_strerror.argtypes = [ip]
    lib.gf_strerror.restype = C.c_char_p
    lib.gf_abi_version.restype = ip
    lib.gf_last_cuda_error.restype = C.c_char_p
    _lib = lib
    return lib


def check(status: int, where: str) -> None:
    if status != GF_OK:
        raise GfError(status, where, _lib)
