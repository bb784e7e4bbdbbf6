#!/usr/bin/env python
"""Benchmark: cells/s per flow step (ΔT) of the per-cell chemistry solve.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload gri-bimodal-1M|gri-100k|h2-1k|mixed-750k|...] [--solver 34]
                    [--no-plain] [--no-e2e] [--no-cpu]

A step is one gf_solve over the whole batch: every cell integrated over one
flow time step ΔT with adaptive Rosenbrock substeps, relTol 1e-4, absTol 1e-8,
starting each step from the same states and deltaTChem = 1e-7 s (the
reference tutorials' initialChemicalTimeStep). Inputs are seeded synthetic
batches; L2 (126 MB) is flushed before every timed step by writing a 256 MB
buffer (outside the timed region).

The default workload is the 1M-cell batch of the 53-species mechanism with
bimodal temperatures (40 % near-inert cells at 300-700 K, 60 % igniting cells
at 1100-2400 K, shuffled): the batch the persistent-vs-plain comparison is
stated on. Both arms print the same `metric` string.

`value`     persistent work-queue kernel, captured once as a CUDA graph and
            replayed every step; inputs resident in HBM, CUDA events
`plain`     the one-thread-per-cell kernel on the same batch (the reference's
            launch model, also replayed from a graph), for the
            persistent-vs-plain ratio; one untimed warm-up solve on a 64k-cell
            part of the batch, then --plain-steps timed steps over all of it
`substeps_per_cell` the spread of accepted substeps per cell over the batch
`e2e`       GpuKernelEvaluator.computeRR through the C ABI from pinned host
            arrays: H2D of Y/ΔTChem/rho, the solve, D2H of RR/ΔTChem
`roofline`  FP64 pipe: algorithmic FLOP (gpufoam_b200/flops.py) per launch ÷
            launch time, against the DFMA peak measured live on this GPU
`cpu_baseline` the reference's own FP64 code (compiled in place, OpenMP over
            cells, one cell per scheduling chunk, on all host cores) on a
            bounded sample of the same batch

Multi-GPU (torchrun): every rank integrates its own batch of the workload's
size (weak scaling, cells are independent); the one exchange per step is the
min over ranks of the new chemistry time step (NCCL all-reduce).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # name: mechanism, cells, deltaT, T sampling
    "h2-1k": dict(mech="h2", n=1024, dT=1e-5, T=(1000.0, 2500.0)),
    "gri-100k": dict(mech="gri", n=100_000, dT=1e-6, T=(1000.0, 2500.0)),
    # bimodal: 40 % near-inert cells (reactive mass fraction 1e-4, the rest the
    # inert species) at 300-700 K and 60 % igniting cells at 1100-2400 K
    "gri-bimodal-1M": dict(mech="gri", n=1_000_000, dT=1e-6, bimodal=(0.4, (300.0, 700.0), (1100.0, 2400.0)),
                           cold_reactive=1e-4),
    # one launch over three mechanisms (10, 53 and 100 species), per-cell
    # deltaT ~ log-U[1e-7, 1e-4] s and p ~ U[0.5, 40] atm, cells shuffled
    "mixed-750k": dict(mixed=((("h2", 200_000), ("gri", 500_000), ("large", 50_000))), dT=0.0,
                       dT_cell=(1e-7, 1e-4), p=(0.5 * 101325.0, 40 * 101325.0)),
    # the same proportions at a tenth of the size (a bounded measurement)
    "mixed-75k": dict(mixed=((("h2", 20_000), ("gri", 50_000), ("large", 5_000))), dT=0.0,
                      dT_cell=(1e-7, 1e-4), p=(0.5 * 101325.0, 40 * 101325.0)),
    # small cases of the same kernels, for ncu captures and launch sweeps
    "gri-4k": dict(mech="gri", n=4096, dT=1e-6, T=(1000.0, 2500.0)),
    "gri-16k": dict(mech="gri", n=16384, dT=1e-6, T=(1000.0, 2500.0)),
    "gri-bimodal-64k": dict(mech="gri", n=65536, dT=1e-6, bimodal=(0.4, (300.0, 700.0), (1100.0, 2400.0)),
                            cold_reactive=1e-4),
    # the real GRI-Mech 3.0 of the reference's unit tests (53 species, 325
    # reactions, read from its OpenFOAM dictionaries into tests/golden/foam_gri.npz)
    "gri30-100k": dict(mech="gri30", n=100_000, dT=1e-6, T=(1000.0, 2500.0)),
}
DTC0 = 1e-7


def metric_name(workload, solver):
    """The metric string both arms print (the driver pairs the lines by it)."""
    return f"cells/s per ΔT at relTol 1e-4 ({workload}, R{solver})"


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per cell of the
# persistent kernel on the GRI-size mechanism, from one ncu capture of 4 096
# cells in the launch form below (profiles/persistent_kernel_g128_gri4k.md):
# 2 877 952 B read, 97 536 B written. Scaled by the cell count for the same
# kernel on the larger GRI-size batches (the per-cell inputs and outputs are
# moved once, the tables stay in L2).
NCU_DRAM_BYTES_PER_CELL_GRI = (2877952 + 97536) / 4096
NCU_PROFILED_FORM = dict(threads_per_cell=128, register_budget=1, lu_panel=4, specialize=1)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="gri-bimodal-1M", choices=list(WORKLOADS))
    ap.add_argument("--solver", type=int, default=34, choices=[12, 23, 34])
    ap.add_argument("--launch", default="auto", choices=["fixed", "auto", "sweep"],
                    help="fixed: --threads-per-cell/--shared; auto: autotuner on a sample; "
                         "sweep: print every launch form's time to stderr, then use the best")
    ap.add_argument("--threads-per-cell", type=int, default=64)
    ap.add_argument("--shared", type=int, default=1)
    ap.add_argument("--register-budget", type=int, default=0, choices=[0, 1],
                    help="persistent kernel: 0 = up to 255 registers per thread, 1 = at most 128")
    ap.add_argument("--lu-panel", type=int, default=0, choices=[0, 4, 8, 16],
                    help="persistent kernel, fixed launch: columns per LU panel (0 = 8)")
    ap.add_argument("--specialize", type=int, default=0, choices=[0, 1],
                    help="persistent kernel, fixed launch: the kernel compiled for the mechanism's matrix size")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--plain-steps", type=int, default=1,
                    help="timed steps of the plain-kernel leg over the whole batch (at most --steps), after "
                         "one untimed warm-up solve on a 64k-cell part of it; the plain kernel runs several "
                         "times longer than the persistent one on the bimodal and mixed batches")
    ap.add_argument("--plain-cells", type=int, default=100_000,
                    help="mixed batches: cells of the random part the plain kernel is timed on")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--no-adjoint", action="store_true",
                    help="skip the adjoint measurement (4096 GRI-size cells, deltaT 1e-4 s)")
    ap.add_argument("--adjoint-only", action="store_true",
                    help="print only the adjoint measurement (one JSON line) and exit")
    ap.add_argument("--adjoint-cells", type=int, default=4096)
    return ap.parse_args()


class Batch:
    """A workload's cells: mechanisms, states [n][ld], per-cell mechanism ids
    and time steps (None for a single mechanism / one deltaT)."""

    def __init__(self, raws, cells, mech_id=None, dT_cell=None):
        self.raws, self.cells, self.mech_id, self.dT_cell = raws, cells, mech_id, dT_cell


def _mech(name):
    from gpufoam_b200 import mechanism as M
    if name == "gri30":
        from tests.test_oracle import fixture_mech, load
        return fixture_mech(load("foam_gri"))
    return {"h2": M.h2_size, "gri": M.gri_size, "large": M.large}[name](0)


def make_batch(wl, seed) -> Batch:
    from gpufoam_b200 import mechanism as M
    if "mixed" in wl:
        rng = np.random.default_rng(seed)
        raws = [_mech(name) for name, _ in wl["mixed"]]
        ld = max(r.n_eqns for r in raws)
        n = sum(k for _, k in wl["mixed"])
        cells = np.zeros((n, ld))
        mid = np.empty(n, dtype=np.int32)
        o = 0
        for k, ((_, cnt), r) in enumerate(zip(wl["mixed"], raws)):
            cells[o:o + cnt, :r.n_eqns] = M.make_cells(r, cnt, seed=seed + 17 * k, p_range=wl["p"])
            mid[o:o + cnt] = k
            o += cnt
        perm = rng.permutation(n)
        dts = M.log_uniform(rng, wl["dT_cell"][0], wl["dT_cell"][1], n)
        return Batch(raws, np.ascontiguousarray(cells[perm]), mid[perm], dts)
    raw = _mech(wl["mech"])
    if "bimodal" in wl:
        cells = M.make_cells(raw, wl["n"], seed=seed, bimodal=wl["bimodal"],
                             cold_reactive_fraction=wl.get("cold_reactive"))
    else:
        cells = M.make_cells(raw, wl["n"], seed=seed, T_range=wl["T"])
    return Batch([raw], cells)


class Clocks:
    """nvidia-smi samples during the timed region."""

    def __init__(self, device_index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={q}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(device_index)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _cpu_rate_one(raw, cells, solver, dT, dT_cell, seconds, nthreads):
    """cells/s of the CPU path on one mechanism: a short call sizes the sample,
    then one call over about `seconds` of cells (at least 32 per thread), each
    cell its own OpenMP scheduling chunk so every thread stays busy to the end.
    Returns (cells/s of the sized call, cells in it, kind, its seconds)."""
    from oracle.oracle import REF_LIB, Oracle, ode_inputs
    kind = "reference" if os.path.exists(REF_LIB) else "port"
    o = Oracle(raw, kind)
    inp = ode_inputs(solver)

    def run(lo, hi):
        chunk = np.ascontiguousarray(cells[lo:hi, :raw.n_eqns])
        t0 = time.perf_counter()
        if kind == "reference" and dT_cell is None:
            o.cells_uncounted(inp, chunk, dT, DTC0, nthreads=nthreads)
        else:
            o.cells(inp, chunk, dT, DTC0, deltaT_cell=None if dT_cell is None else dT_cell[lo:hi],
                    nthreads=nthreads)
        return time.perf_counter() - t0

    n_all = cells.shape[0]
    probe = min(n_all, 4 * nthreads)
    rate = probe / max(run(0, probe), 1e-9)
    size = int(min(n_all - probe, max(32 * nthreads, rate * seconds)))
    if size <= 0:
        return rate, probe, kind, probe / rate
    t = run(probe, probe + size)
    return size / t, size, kind, t


def cpu_reference_rate(batch, solver, dT, seconds, nthreads, offset=0):
    """The reference's own singleCellSolver (oracle/_ref, or the port) over a
    bounded sample of the batch (from `offset`; the batches are shuffled) with
    all host threads. Several mechanisms: each is timed on its own cells for a
    share of the time, and the batch rate is n / sum_k(n_k / rate_k).
    Returns (cells/s, sample size, kind, seconds)."""
    if batch.mech_id is None:
        return _cpu_rate_one(batch.raws[0], batch.cells[offset:], solver, dT, None, seconds, nthreads)
    n = batch.cells.shape[0]
    t_inv, done_all, t_all, kind = 0.0, 0, 0.0, None
    for k, raw in enumerate(batch.raws):
        sel = np.nonzero(batch.mech_id == k)[0]
        share = max(seconds * len(sel) / n, seconds / (2 * len(batch.raws)))
        r, done, kind, t = _cpu_rate_one(raw, batch.cells[sel], solver, dT, batch.dT_cell[sel], share, nthreads)
        t_inv += len(sel) / r
        done_all += done
        t_all += t
    return n / t_inv, done_all, kind, t_all


ADJOINT = dict(mech="gri", n=4096, dT=1e-4, T=(1100.0, 1600.0))


def adjoint_measure(solver_launch, steps, n_cells=4096):
    """Forward (plain solve and recording solve) and adjoint sweep times on the
    differentiation workload: 4096 GRI-size cells, T ~ U[1100, 1600] K, deltaT
    1e-4 s (through ignition), Rosenbrock34; loss = seeded weights . final (Y, T).
    Gradients w.r.t. the initial states and all (ln|A|, beta, Ta) per reaction."""
    import torch
    from gpufoam_b200 import adjoint as AD
    from gpufoam_b200 import evaluator as E
    from gpufoam_b200 import mechanism as M
    raw = M.gri_size(0)
    cells = M.make_cells(raw, n_cells, seed=4096, T_range=ADJOINT["T"])
    ode = E.OdeInputs("Rosenbrock34", absTol=1e-8, relTol=1e-4)
    sol = AD.AdjointSolver(raw, ode, traj_cap=4096, launch=solver_launch)
    Y0 = torch.as_tensor(cells, device="cuda")
    w = torch.as_tensor(np.random.default_rng(5).standard_normal(cells.shape), device="cuda")
    w[:, raw.n_species + 1] = 0.0
    ev = lambda: (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
    flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device="cuda")  # 256 MB > L2, before each timing
    fw, rec, adj = [], [], []
    for k in range(steps + 1):
        dtc = torch.full((n_cells,), DTC0, dtype=torch.float64, device="cuda")
        flush.zero_()
        a0, a1 = ev()
        a0.record()
        sol.solver.solve(Y0, ADJOINT["dT"], dtc, want_status=False, want_counters=False, want_stats=False)
        a1.record()
        dtc = torch.full((n_cells,), DTC0, dtype=torch.float64, device="cuda")
        flush.zero_()
        b0, b1 = ev()
        b0.record()
        Y1, status, counters = sol.forward(Y0, ADJOINT["dT"], dtc)
        b1.record()
        flush.zero_()
        c0, c1 = ev()
        c0.record()
        Y0bar, thb, st = sol.backward(w)
        c1.record()
        torch.cuda.synchronize()
        if k > 0:
            fw.append(a0.elapsed_time(a1))
            rec.append(b0.elapsed_time(b1))
            adj.append(c0.elapsed_time(c1))
    cnt = counters.cpu().numpy()
    ok = int(((status.cpu().numpy() == 0) & (st.cpu().numpy() == 0)).sum())
    f, r, a = float(np.mean(fw)), float(np.mean(rec)), float(np.mean(adj))
    return {"workload": f"{n_cells} GRI-size cells, T~U[1100,1600] K, deltaT 1e-4 s, Rosenbrock34",
            "forward_ms": f, "forward_recording_ms": r, "adjoint_ms": a, "adjoint_over_forward": a / f,
            "gradient_over_forward": (r + a) / f,
            "accepted_steps_per_cell": {"mean": float(cnt[:, 0].mean()), "max": int(cnt[:, 0].max())},
            "cells_ok": ok, "parameters": f"{raw.n_reactions} x (ln|A|, beta, Ta)"}


def main():
    args = parse()
    wl = WORKLOADS[args.workload]
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    nthreads = os.cpu_count() or 1
    cfg_desc = {"workload": args.workload, "solver": f"Rosenbrock{args.solver}", "relTol": 1e-4, "absTol": 1e-8,
                "deltaT": wl["dT"] if "dT_cell" not in wl else f"per cell, log-U{list(wl['dT_cell'])} s"}

    if args.adjoint_only:
        import torch
        torch.cuda.set_device(local)
        print(json.dumps({"adjoint": adjoint_measure(dict(kind=1, threads_per_cell=args.threads_per_cell,
                                                          scratch_in_shared=1, register_budget=args.register_budget),
                                                     max(1, args.steps), args.adjoint_cells)}))
        return

    if args.impl == "reference":
        if rank != 0:
            return
        batch = make_batch(wl, seed=1000)
        times, rates, sample = [], [], None
        n_all = batch.cells.shape[0]
        for k in range(args.warmup + args.steps):
            r, done, kind, t = cpu_reference_rate(batch, args.solver, wl["dT"], max(2.0, args.cpu_seconds / 4),
                                                  nthreads, offset=(k * 7919 * nthreads) % max(1, n_all // 2))
            if k >= args.warmup:
                rates.append(r)
                times.append(t)
                sample = done
        value = float(np.mean(rates))
        line = {"impl": "reference", "metric": metric_name(args.workload, args.solver),
                "value": value, "unit": "cells/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
                "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic",
                "config": dict(cfg_desc, cells=int(batch.cells.shape[0])),
                "cpu_baseline": {"value": value, "unit": "cells/s", "cores": nthreads, "kind": kind,
                                 "sample": f"{sample} cells of the {args.workload} batch per step (a new "
                                           f"part of the shuffled batch each step), the reference's "
                                           f"singleCellSolver per cell, OpenMP schedule(dynamic,1) over cells"},
                "e2e": {"value": value, "unit": "cells/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return

    import torch
    import torch.distributed as dist

    from gpufoam_b200 import _native as N
    from gpufoam_b200 import evaluator as E
    from gpufoam_b200 import flops as F
    from gpufoam_b200 import sharding

    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    batch = make_batch(wl, seed=1000 + rank)
    cells = batch.cells
    n = cells.shape[0]
    mechs = [E.Mechanism(r) for r in batch.raws]
    ode = E.OdeInputs(f"Rosenbrock{args.solver}", absTol=1e-8, relTol=1e-4)
    Y0 = torch.as_tensor(cells, device="cuda")
    mid = None if batch.mech_id is None else torch.as_tensor(batch.mech_id, device="cuda")
    dtcell = None if batch.dT_cell is None else torch.as_tensor(batch.dT_cell, device="cuda")
    dtc0 = torch.full((n,), DTC0, dtype=torch.float64, device="cuda")
    dtc = dtc0.clone()
    Ynew = torch.empty_like(Y0)
    lib = N.load()

    # written before every timed step so that no input or table is left in L2
    l2_flush = torch.empty(32 * 1024 * 1024, dtype=torch.float64, device="cuda")

    def timed(solver, steps, warmup, part=None):
        """W + K replays of the solve captured as a CUDA graph (queue reset +
        solve kernel), each timed with CUDA events on the launching stream;
        part: indices of the cells to solve (default all)."""
        stream = torch.cuda.current_stream()
        if part is None:
            Y0p, dtcp, dtc0p, Ynewp, dtcellp, midp = Y0, dtc, dtc0, Ynew, dtcell, mid
        else:
            ix = torch.as_tensor(part, device="cuda")
            Y0p, dtc0p = Y0[ix].contiguous(), dtc0[ix].contiguous()
            dtcp, Ynewp = dtc0p.clone(), torch.empty_like(Y0p)
            dtcellp = None if dtcell is None else dtcell[ix].contiguous()
            midp = None if mid is None else mid[ix].contiguous()
        counters = torch.empty((Y0p.shape[0], 2), dtype=torch.int32, device="cuda")
        graph = solver.capture(Y0p, wl["dT"], dtcp, Ynew=Ynewp, deltaT_cell=dtcellp, mech_id=midp,
                               counters=counters)
        for _ in range(warmup):
            dtcp.copy_(dtc0p)
            graph.launch(stream)
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        ms = []
        launches = 0
        for _ in range(steps):
            dtcp.copy_(dtc0p)
            l2_flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            graph.launch(stream)
            e1.record(stream)
            launches += 2  # queue reset + the solve kernel
            if world > 1:
                # the exchange of the step: min over ranks of the new chemistry time step
                sharding.global_min_delta_t(float(dtcp.min()), device="cuda")
            torch.cuda.synchronize()
            ms.append(e0.elapsed_time(e1))
        torch.cuda.synchronize()
        if world > 1:
            dist.barrier()
        cnt = counters.cpu().numpy()
        graph.close()
        return ms, cnt, launches

    def flop_of(cnt):
        if batch.mech_id is None:
            return F.total(batch.raws[0], args.solver, int(cnt[:, 1].sum()), int(cnt[:, 0].sum()))
        return sum(F.total(r, args.solver, int(cnt[batch.mech_id == k, 1].sum()), int(cnt[batch.mech_id == k, 0].sum()))
                   for k, r in enumerate(batch.raws))

    # FP64 roofline denominator, measured on this GPU
    import ctypes
    peak = ctypes.c_double()
    N.check(lib.gf_measure_fp64_peak(200.0, ctypes.byref(peak)), "gf_measure_fp64_peak")

    solver = E.Solver(mechs, ode)
    solver.set_launch(kind=1, threads_per_cell=args.threads_per_cell, scratch_in_shared=args.shared,
                      register_budget=args.register_budget, lu_panel=args.lu_panel, specialize=args.specialize)
    tuned = None
    if args.launch != "fixed":
        from gpufoam_b200 import autotune
        rng = np.random.default_rng(7)
        pick = rng.choice(n, size=min(n, 8192), replace=False)
        tuned = autotune.tune(solver, cells[pick], wl["dT"], DTC0, use_cache=(args.launch == "auto"),
                              deltaT_cell=None if dtcell is None else dtcell[torch.as_tensor(pick, device="cuda")],
                              mech_id=None if mid is None else mid[torch.as_tensor(pick, device="cuda")],
                              verbose=False)
        if args.launch == "sweep" and rank == 0:
            for cfg, ms in tuned["table"]:
                print(json.dumps({"sweep": cfg, "ms": ms, "cells": int(len(pick))}), file=sys.stderr)
    clocks = Clocks(torch.cuda.current_device()) if rank == 0 else None
    ms, cnt, launches = timed(solver, args.steps, args.warmup)
    clk = clocks.stop() if clocks else None
    ms_step = float(np.mean(ms))
    t_max = ms_step
    if world > 1:
        t = torch.tensor([ms_step], dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        t_max = float(t.item())
    value = world * n / (t_max * 1e-3)
    attempts, accepted = int(cnt[:, 1].sum()), int(cnt[:, 0].sum())
    flop = flop_of(cnt)
    achieved = flop / (ms_step * 1e-3) / 1e12

    plain = None
    if not args.no_plain:
        ps = E.Solver(mechs, ode)
        ps.set_launch(kind=0)
        # warm-up: one untimed solve over a part of the batch (a plain step over
        # the whole bimodal or mixed batch takes minutes)
        k = min(n, 65536)
        ps.solve(Y0[:k], wl["dT"], dtc0[:k].clone(), deltaT_cell=None if dtcell is None else dtcell[:k],
                 mech_id=None if mid is None else mid[:k], want_status=False, want_counters=False,
                 want_stats=False)
        torch.cuda.synchronize()
        # mixed batches: the plain kernel is timed on a random part of the batch
        # (its cells/s; a plain step over the whole 750k-cell batch takes ~15 min)
        part = None
        if batch.mech_id is not None and n > args.plain_cells:
            part = np.sort(np.random.default_rng(11).choice(n, size=args.plain_cells, replace=False))
        n_plain = n if part is None else len(part)
        pms, pcnt, _ = timed(ps, max(1, min(args.steps, args.plain_steps)), 0, part=part)
        pm = float(np.mean(pms))
        if world > 1:
            t = torch.tensor([pm], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            pm = float(t.item())
        plain = {"value": world * n_plain / (pm * 1e-3), "ms_per_step": pm, "unit": "cells/s",
                 "steps": len(pms), "launch": "one thread per cell, HBM scratch (the reference's launch model)",
                 "warmup": f"one untimed solve over {k} cells of the batch",
                 "cells": n_plain if part is None else f"{n_plain} of the {n} cells, drawn at random (seed 11)"}
        del ps

    e2e = None
    if not args.no_e2e and batch.mech_id is None:
        raw = batch.raws[0]
        ev = E.GpuKernelEvaluator(n, raw.n_eqns, raw.n_species, mechs[0], ode)
        ev.solver.set_launch(**solver.get_launch())
        hY = torch.empty((n, raw.n_eqns), dtype=torch.float64, pin_memory=True)
        hY.copy_(torch.as_tensor(cells))
        hrho = torch.empty(n, dtype=torch.float64, pin_memory=True)
        hrho.copy_(torch.as_tensor(np.linspace(0.2, 1.2, n)))
        hdtc = torch.full((n,), DTC0, dtype=torch.float64).pin_memory()
        ev.computeRR(wl["dT"], 1.0, hrho.numpy(), hdtc.numpy(), hY.numpy())
        em = []
        for _ in range(max(1, min(args.steps, 2))):
            torch.cuda.synchronize()
            l2_flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            RR, dtn, mn = ev.computeRR(wl["dT"], 1.0, hrho.numpy(), hdtc.numpy(), hY.numpy())
            e1.record()
            torch.cuda.synchronize()
            em.append(e0.elapsed_time(e1))
        et = float(np.mean(em))
        if world > 1:
            t = torch.tensor([et], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            et = float(t.item())
        e2e = {"value": world * n / (et * 1e-3), "unit": "cells/s",
               "h2d_bytes_per_step": int(n * (raw.n_eqns + 2) * 8),
               "d2h_bytes_per_step": int(n * (raw.n_species + 1) * 8),
               "api": "GpuKernelEvaluator.computeRR -> gf_compute_rr (pinned host arrays)"}
        del ev
    elif not args.no_e2e:
        # several mechanisms: the device-memory entry point from pinned host arrays
        hY = torch.empty(cells.shape, dtype=torch.float64, pin_memory=True)
        hY.copy_(torch.as_tensor(cells))
        hm = torch.as_tensor(batch.mech_id).pin_memory()
        hdt = torch.as_tensor(batch.dT_cell).pin_memory()
        hdtc = torch.full((n,), DTC0, dtype=torch.float64).pin_memory()
        hout = torch.empty(cells.shape, dtype=torch.float64, pin_memory=True)
        hdtn = torch.empty(n, dtype=torch.float64, pin_memory=True)
        em = []
        for _ in range(max(1, min(args.steps, 2))):
            torch.cuda.synchronize()
            l2_flush.zero_()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dY, dm, ddt, dd = (hY.to("cuda", non_blocking=True), hm.to("cuda", non_blocking=True),
                               hdt.to("cuda", non_blocking=True), hdtc.to("cuda", non_blocking=True))
            solver.solve(dY, 0.0, dd, Ynew=dY, deltaT_cell=ddt, mech_id=dm, want_status=False,
                         want_counters=False, want_stats=False)
            hout.copy_(dY, non_blocking=True)
            hdtn.copy_(dd, non_blocking=True)
            e1.record()
            torch.cuda.synchronize()
            em.append(e0.elapsed_time(e1))
        et = float(np.mean(em))
        if world > 1:
            t = torch.tensor([et], dtype=torch.float64, device="cuda")
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            et = float(t.item())
        e2e = {"value": world * n / (et * 1e-3), "unit": "cells/s",
               "h2d_bytes_per_step": int(n * (cells.shape[1] * 8 + 4 + 8 + 8)),
               "d2h_bytes_per_step": int(n * (cells.shape[1] + 1) * 8),
               "api": "Solver.solve -> gf_solve with per-cell deltaT and mechanism id (pinned host arrays)"}

    adjoint = None
    if rank == 0 and world == 1 and not args.no_adjoint and batch.mech_id is None:
        adjoint = adjoint_measure(solver.get_launch(), 1)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        r, done, kind, t = cpu_reference_rate(batch, args.solver, wl["dT"], args.cpu_seconds, nthreads)
        cpu = {"value": r, "unit": "cells/s", "cores": nthreads, "kind": kind,
               "sample": f"{done} cells of the {args.workload} batch ({t:.1f} s), the reference's "
                         f"singleCellSolver per cell, OpenMP schedule(dynamic,1)"}

    acc = cnt[:, 0]
    if batch.mech_id is not None:
        acc = acc[acc > 0] if (acc > 0).any() else acc
    spread = {"min": int(acc.min()), "p1": float(np.percentile(acc, 1)), "p50": float(np.percentile(acc, 50)),
              "p99": float(np.percentile(acc, 99)), "max": int(acc.max()),
              "max_over_min": float(acc.max() / max(acc.min(), 1)),
              "p99_over_p1": float(np.percentile(acc, 99) / max(np.percentile(acc, 1), 1.0))}

    if rank == 0:
        line = {
            "metric": metric_name(args.workload, args.solver),
            "value": value, "unit": "cells/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": t_max, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": dict(cfg_desc, cells_per_gpu=n,
                           mechanisms=[f"{r.n_species} species / {r.n_reactions} reactions" for r in batch.raws],
                           deltaTChem0=DTC0, kernel="persistent work queue, CUDA-graph replay",
                           launch=solver.get_launch(), l2="flushed before each timed step (256 MB write)",
                           parallelism=f"cells sharded over {world} GPU(s)"),
            "roofline": {"bound": "fp64", "achieved": achieved, "peak": peak.value, "unit": "TFLOP/s",
                         "frac": achieved / peak.value,
                         "traffic": (NCU_DRAM_BYTES_PER_CELL_GRI * n
                                     if wl.get("mech") == "gri" and all(solver.get_launch()[k] == v
                                                                        for k, v in NCU_PROFILED_FORM.items())
                                     else None),
                         "traffic_source": "ncu dram bytes of 4096 GRI-size cells, scaled per cell",
                         "algorithmic_bytes_per_launch": int(n * 2 * cells.shape[1] * 8),
                         "peak_source": "measured DFMA microbenchmark on this GPU (gf_measure_fp64_peak)",
                         "algorithmic_flop_per_launch": flop, "attempts": attempts, "accepted": accepted},
            "plain": plain,
            "persistent_vs_plain": (value / plain["value"]) if plain else None,
            "substeps_per_cell": spread,
            "e2e": e2e, "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk,
            "adjoint": adjoint,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
