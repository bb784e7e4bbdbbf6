"""Build the in-tree native library gpufoam_b200/libgpufoam_b200.so for sm_100a.

    python -m gpufoam_b200.build [--force] [-v]

nvcc cross-compiles without a GPU; the library links the CUDA runtime only.
Each source compiles to its own object in parallel (the persistent kernel is
instantiated in one file per group size), then one nvcc call links them.
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "libgpufoam_b200.so")
OBJ = os.path.join(os.path.dirname(HERE), "_build", "obj")
GROUPS = [1, 2, 4, 8, 16, 32, 64, 96, 128, 256]
SOURCES = (["gf_host.cpp", "gf_kernels.cu", "gf_peak.cu", "gf_noalloc.cu", "gf_adjoint.cu", "gf_fields.cu", "gf_fieldio.cu"] +
           [f"gf_persist_g{g}.cu" for g in GROUPS] + [f"gf_persist_g{g}_tuned.cu" for g in (32, 64, 96, 128)])
HEADERS = ["gf_internal.h", "gf_device.cuh", "gf_persist.cuh", "gf_adjoint.cuh", os.path.join("..", "..", "include", "gpufoam_b200.h")]

NVCC_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC",
]


def _mtime(f: str) -> float:
    return os.path.getmtime(os.path.join(CSRC, f))


def _stale(src: str, obj: str) -> bool:
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(_mtime(f) > t for f in [src] + HEADERS)


def build(force: bool = False, verbose: bool = False, extra_flags=None, out: str = OUT) -> str:
    """Compile the sources that changed (all with force) and link `out`."""
    if not force and os.path.exists(out):
        t = os.path.getmtime(out)
        if all(_mtime(f) <= t for f in SOURCES + HEADERS):
            return out  # up to date (object files need not be present)
    nvcc = os.environ.get("NVCC", "nvcc")
    flags = NVCC_FLAGS + list(extra_flags or [])
    tag = "" if not extra_flags else "_" + hashlib.sha1(" ".join(extra_flags).encode()).hexdigest()[:8]
    objdir = OBJ + tag
    os.makedirs(objdir, exist_ok=True)
    objs = [os.path.join(objdir, os.path.splitext(s)[0] + ".o") for s in SOURCES]
    todo = [(s, o) for s, o in zip(SOURCES, objs) if force or _stale(s, o)]

    def compile_one(so):
        src, obj = so
        cmd = [nvcc, *flags, "-c", "-o", obj, os.path.join(CSRC, src)]
        if verbose:
            cmd[1:1] = ["-Xptxas", "-v"]
        subprocess.run(cmd, check=True)

    if todo:
        with ThreadPoolExecutor(max_workers=max(1, min(len(todo), os.cpu_count() or 1))) as ex:
            list(ex.map(compile_one, todo))
    if todo or not os.path.exists(out) or any(os.path.getmtime(o) > os.path.getmtime(out) for o in objs):
        subprocess.run([nvcc, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", out, *objs],
                       check=True)
    return out


if __name__ == "__main__":
    build(force="--force" in sys.argv, verbose="-v" in sys.argv)
    print(OUT)
