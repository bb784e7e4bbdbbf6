"""Launch-form autotuner of the chemistry kernels.

For a mechanism and ODE settings it times every launch form the library
offers on a sample of the caller's cells and keeps the fastest:

  * plain: one thread per cell, HBM scratch (the reference's launch model);
  * persistent work queue with G = 1, 4, 8, 16, 32 threads per cell (groups
    inside a warp) or 64, 96, 128, 256 (one cell per CTA), the per-cell workspace in
    shared memory (when it fits) or in HBM, and two register budgets;
  * for 32, 64, 96 and 128 threads per cell, the tile and specialisation variants:
    LU panels of 4 or 16 columns instead of 8, and the kernel compiled for the
    mechanism's matrix size (10-, 53- and 100-species mechanisms), which fixes
    the workspace offsets, loop bounds and the unrolled tiles' predicates.

Results are cached per (device, library build, mechanism shape, solver) in
memory and in a JSON file (GPUFOAM_AUTOTUNE_CACHE, default
~/.cache/gpufoam_b200/autotune.json); a rebuilt library tunes afresh.
"""
from __future__ import annotations

import hashlib
import json
import os
from typing import Dict, List, Optional

import numpy as np

from . import evaluator as E

_CACHE: Dict[str, dict] = {}


def _cache_path() -> str:
    return os.environ.get("GPUFOAM_AUTOTUNE_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "gpufoam_b200", "autotune.json"))


_BUILD_HASH: Optional[str] = None


def build_hash() -> str:
    """Digest of the loaded library file: a cached pick is only reused with the
    kernels it was timed on."""
    global _BUILD_HASH
    if _BUILD_HASH is None:
        from . import _native as N
        h = hashlib.sha1()
        with open(N.LIB_PATH, "rb") as f:
            for block in iter(lambda: f.read(1 << 20), b""):
                h.update(block)
        _BUILD_HASH = h.hexdigest()[:16]
    return _BUILD_HASH


def _key(mechs, ode: E.OdeInputs) -> str:
    import torch
    h = hashlib.sha1()
    h.update(torch.cuda.get_device_name().encode())
    h.update(build_hash().encode())
    for m in mechs:
        h.update(f"{m.n_species}/{m.n_reactions}/{m.raw.name}".encode())
    h.update(f"{ode.name}/{ode.relTol}/{ode.absTol}".encode())
    return h.hexdigest()[:16]


def candidates(max_ws_doubles: int) -> List[dict]:
    """Launch forms worth timing for a workspace of max_ws_doubles per cell:
    the plain kernel, and persistent forms with the workspace in shared memory
    when a CTA's groups fit (else in HBM), both register budgets."""
    ws = max_ws_doubles * 8
    out = [dict(kind=0, threads_per_cell=1, scratch_in_shared=0, cells_per_block=0, blocks_per_sm=0,
                register_budget=0, lu_panel=0, specialize=0)]
    for G in (1, 4, 8, 16, 32, 64, 96, 128, 256):
        groups_per_cta = max(1, 128 // G) if G <= 32 else 1
        shared_ok = ws * (1 if G <= 32 else groups_per_cta) <= 227 * 1024
        for shared in ((1, 0) if shared_ok else (0,)):
            for regs in (0, 1):
                out.append(dict(kind=1, threads_per_cell=G, scratch_in_shared=shared, cells_per_block=0,
                                blocks_per_sm=0, register_budget=regs, lu_panel=0, specialize=0))
            if G in (32, 64, 96, 128):
                # the tuned variants (gf_solver_set_launch refuses those that do
                # not apply to the solver's mechanisms; tune() skips them)
                regs = 1 if G in (96, 128) else 0
                for nb in (0, 4):
                    out.append(dict(kind=1, threads_per_cell=G, scratch_in_shared=shared, cells_per_block=0,
                                    blocks_per_sm=0, register_budget=regs, lu_panel=nb, specialize=1))
                if shared:
                    for nb in (4, 16):
                        out.append(dict(kind=1, threads_per_cell=G, scratch_in_shared=1, cells_per_block=0,
                                        blocks_per_sm=0, register_budget=regs, lu_panel=nb, specialize=0))
    return out


def time_config(solver: E.Solver, cfg: dict, Y0, dtc0, deltaT: float, reps: int = 2, deltaT_cell=None,
                mech_id=None, give_up_ms: float = float("inf")) -> float:
    """Mean ms of one solve over the sample with launch form cfg (the first,
    untimed-for-the-mean run is returned as is when it exceeds give_up_ms)."""
    import torch
    solver.set_launch(**cfg)
    dtc = dtc0.clone()
    Ynew = torch.empty_like(Y0)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    solver.solve(Y0, deltaT, dtc, Ynew=Ynew, deltaT_cell=deltaT_cell, mech_id=mech_id, want_status=False,
                 want_counters=False, want_stats=False)
    e1.record()
    torch.cuda.synchronize()
    first = e0.elapsed_time(e1)
    if first > give_up_ms:
        return first
    ms = []
    for _ in range(reps):
        dtc.copy_(dtc0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        solver.solve(Y0, deltaT, dtc, Ynew=Ynew, deltaT_cell=deltaT_cell, mech_id=mech_id, want_status=False,
                     want_counters=False, want_stats=False)
        e1.record()
        torch.cuda.synchronize()
        ms.append(e0.elapsed_time(e1))
    return float(np.mean(ms))


def tune(solver: E.Solver, Y_sample, deltaT: float, dtc0: float = 1e-7, deltaT_cell=None, mech_id=None,
         configs: Optional[List[dict]] = None, use_cache: bool = True, verbose: bool = False) -> dict:
    """Pick the fastest launch form for `solver` on a sample of cells and apply
    it. Returns dict(best=cfg, table=[(cfg, ms)])."""
    import torch
    key = _key(solver.mechs, solver.ode)
    if use_cache and key in _CACHE:
        solver.set_launch(**_CACHE[key]["best"])
        return _CACHE[key]
    if use_cache and key not in _CACHE and os.path.exists(_cache_path()):
        try:
            disk = json.load(open(_cache_path()))
            if key in disk:
                _CACHE[key] = disk[key]
                solver.set_launch(**disk[key]["best"])
                return disk[key]
        except Exception:
            pass
    Y0 = torch.as_tensor(Y_sample, dtype=torch.float64, device="cuda").contiguous()
    d0 = torch.full((Y0.shape[0],), dtc0, dtype=torch.float64, device="cuda")
    ws = solver.workspace_doubles()
    table = []
    cands = configs or candidates(ws)
    # the usual winners first, so that slow forms are cut off early
    cands = sorted(cands, key=lambda c: (c["kind"] == 0, abs(c["threads_per_cell"] - 96), -c["scratch_in_shared"]))
    best_ms = float("inf")
    for cfg in cands:
        try:
            ms = time_config(solver, cfg, Y0, d0, deltaT, deltaT_cell=deltaT_cell, mech_id=mech_id,
                             give_up_ms=3.0 * best_ms)
            best_ms = min(best_ms, ms)
        except Exception as e:  # a form the device cannot launch
            if verbose:
                print("skip", cfg, e)
            continue
        table.append((cfg, ms))
        if verbose:
            print(json.dumps(cfg), f"{ms:.2f} ms")
    best = min(table, key=lambda t: t[1])[0]
    solver.set_launch(**best)
    res = dict(best=best, table=table)
    _CACHE[key] = res
    if use_cache:
        try:
            os.makedirs(os.path.dirname(_cache_path()), exist_ok=True)
            disk = json.load(open(_cache_path())) if os.path.exists(_cache_path()) else {}
            disk[key] = res
            json.dump(disk, open(_cache_path(), "w"))
        except Exception:
            pass
    return res
