#!/usr/bin/env python
"""Throughput of the IMEX_SfloW2D time step on one B200 (or N independent
replicas), printed as one JSON line.

Workload: the 4096^2 synthetic fractal-DEM run (10 m cells, Hurst 0.8, 800 m
relief + 15 degree slope, seeded; three solid classes 1e-5/1e-4/1e-3 m with
settling and erosion; radial inlet 1e7 kg/s at 1000 K; Voellmy-Salm
friction), with a 2 m resting current covering the DEM so that every cell
carries the whole step (mask, MUSCL + KT fluxes, explicit terms, Newton
relaxation, erosion/deposition).  A step = one pass of the driver loop
(check_solve, timestep, dt clipping, imex_RK_solver,
update_erosion_deposition_cell) on the device.

  value     cell-updates/s with the state resident in HBM (CUDA events on
            the stream the library runs on), summed over ranks
  e2e       the same metric through the public API with host buffers: each
            step uploads q from pinned host memory, advances, and reads q back
  roofline  dominant kernel: algorithmic bytes per launch / its mean event time
  cpu_baseline  the CPU oracle (a line-by-line C++ port of the reference,
            OpenMP) on the same 4096^2 workload with all host threads (a
            512^2 instance of the generator with one thread)

`--impl reference` times that CPU port alone (the reference itself is
Fortran and cannot be built here: no Fortran compiler in the image).
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "FP64 cell-updates/s (4096² grid); Newton iters/cell, learned vs plain"
UNIT = "cell-updates/s"
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
FALLBACK_HBM_GBS = 6650.0
BUILD_MODE = "exact"   # the headline build; fast mode is measured beside it


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=4096, help="grid side")
    ap.add_argument("--layer", type=float, default=2.0, help="initial current thickness (m)")
    ap.add_argument("--cpu-n", type=int, default=0,
                    help="grid side of the all-thread CPU baseline (0 = the --n grid)")
    ap.add_argument("--cpu1-n", type=int, default=512,
                    help="grid side of the one-thread CPU sample")
    ap.add_argument("--parity-n", type=int, default=512,
                    help="grid side of the GPU-vs-oracle record")
    ap.add_argument("--ref-budget", type=float, default=150.0,
                    help="seconds of timed steps in --impl reference (at least one step)")
    ap.add_argument("--cpu-steps", type=int, default=0, help="0 = choose ~10-20 s of work")
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--ens-members", type=int, default=256)
    ap.add_argument("--ens-steps", type=int, default=1000)
    ap.add_argument("--no-ensemble", action="store_true")
    ap.add_argument("--ens-compare", action="store_true",
                    help="also time the ensemble through per-member graphs over streams")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-setup", action="store_true")
    ap.add_argument("--output-n", type=int, default=1024,
                    help="grid side of the output measurement (0 = skip)")
    ap.add_argument("--learned-pairs", type=int, default=10_000_000)
    ap.add_argument("--learned-n", type=int, default=1024, help="side of the comparison grid")
    ap.add_argument("--parity-steps", type=int, default=10,
                    help="steps of the GPU-vs-oracle check on the CPU sample (0 = skip)")
    ap.add_argument("--no-config-rates", action="store_true")
    ap.add_argument("--no-fast", action="store_true", help="skip the fast-mode measurement")
    return ap.parse_args()


def workload_name(n):
    return ("fractal-dem inlet %dx%d, 10 m cells, 3 solid classes, settling+erosion, Voellmy, "
            "2 m initial layer" % (n, n))


def workload(n, layer):
    from imex_sflow2d_v2_b200 import configs
    return configs.fractal_inlet(n=n, initial_layer=layer)


def bytes_per_cell(ns, erosion, listed=(1.0, 0.0, 0.0)):
    """Algorithmic bytes per grid cell and step of each timed kernel group
    (8-byte values, 1-byte masks, 4-byte list entries).  `listed` is the
    fraction of cells that run Newton iteration 2, 3 and 4.. (each such pass
    reads and writes the cell's Newton state)."""
    nv = 4 + ns
    out = {
        "mask": 8 + 1,                                  # q1 read, mask byte written
        "flux": 8 * nv + 1 + 16 + 8 * nv,               # q, mask, B'x, B'y read; X written
        # q, X, mask, B' read; q_si, Rj, iterate, residual, |r|^2, status, list written
        "stage2_first": 16 * nv + 17 + 32 * nv + 8 + 1 + 4,
        # per pass and listed cell: q, Rj, q_si, iterate, residual, |r|^2, B', list
        # read; iterate, residual, |r|^2, list written
        "stage2_iter": sum(listed) * (40 * nv + 8 + 16 + 4 + 16 * nv + 8 + 4),
        "stage2_post": 8 * nv + 1 + 16 + 1 + 8 * nv,    # iterate, status, q_si(2), mask; q
    }
    if erosion:                                         # q, mask, B' read; q written;
        out["erosion"] = 8 * nv + 1 + 16 + 8 * nv + 2 * 3 * 8 * ns  # 3 planes per class r+w
    return out


def fp64_counts():
    """FP64 instructions (DADD+DMUL+DFMA, per thread) per cell of each kernel
    group and build ("exact", "fast"), from the ncu captures summarised in
    profiles/fp64_inst_per_cell.json."""
    try:
        return json.load(open(os.path.join(ROOT, "profiles", "fp64_inst_per_cell.json")))
    except Exception:
        return {}


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.gpu = gpu_index
        self.proc = None
        self.lines = []
        self.thread = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
            return
        self.thread = threading.Thread(target=self._read, daemon=True)
        self.thread.start()

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self.thread:
            self.thread.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax = float(parts[2])
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def cpu_info():
    """Host CPU model, logical CPUs and the vector flags the timing build uses."""
    model, flags = "unknown", set()
    try:
        with open("/proc/cpuinfo") as f:
            for line in f:
                if line.startswith("model name") and model == "unknown":
                    model = line.split(":", 1)[1].strip()
                elif line.startswith("flags") and not flags:
                    flags = set(line.split(":", 1)[1].split())
    except OSError:
        pass
    keep = [x for x in ("avx2", "fma", "avx512f", "amx_tile") if x in flags]
    return {"model": model, "logical_cpus": os.cpu_count(), "flags": keep}


def _time_oracle(args, p, st, q, threads, timing, budget_s, warmup=1, max_steps=50):
    """Cell-updates/s of the oracle on (p, st, q): `warmup` untimed steps
    (at least one: page-in, thread start-up), then enough steps for about
    `budget_s` seconds, at least one and at most `max_steps`."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    o = orc.Oracle(p, st, threads=threads, timing=timing)
    o.set_state(q, 0.0)
    o.set_clock(0.0, 1e-2)
    t0 = time.perf_counter()
    o.advance(max(1, warmup))
    one = (time.perf_counter() - t0) / max(1, warmup)
    steps = args.cpu_steps if args.cpu_steps > 0 else \
        max(1, min(max_steps, int(budget_s / max(one, 1e-3))))
    t0 = time.perf_counter()
    o.advance(steps)
    el = time.perf_counter() - t0
    return p.nx * p.ny * steps / el, steps, el


def cpu_baseline(args, single_thread=True, warmup=1, budget_s=15.0, max_steps=50):
    """The oracle's timing build (-O3, x86-64-v3, contraction on, stale-read
    instrument off; the checker build if this CPU lacks AVX2/FMA) on the
    benchmark workload itself (--cpu-n 0: the --n grid, same generator, seed
    and physics) with all host threads, and on a --cpu1-n instance of the
    same generator with one thread (a full-size step would take minutes
    there).  Its OpenMP loops are the reference's (assembly,
    erosion/deposition, reconstruction, fluxes, Newton)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    timing = orc.timing_build_usable()
    orc.build(target=orc.TIMING if timing else orc.CHECKER)
    n_all = args.cpu_n if args.cpu_n > 0 else args.n
    p, st, q = workload(n_all, args.layer)
    cores = len(os.sched_getaffinity(0))
    v_all, s_all, el_all = _time_oracle(args, p, st, q, cores, timing, budget_s, warmup,
                                        max_steps)
    del p, st, q
    out = {"value": v_all, "unit": UNIT, "cores": int(cores), "kind": "port",
           "build": ("oracle timing build: g++ -O3 -march=x86-64-v3 -ffp-contract=fast, "
                     "instrument off" if timing else "oracle checker build: g++ -O2 "
                     "-ffp-contract=off (no AVX2/FMA on this CPU)"),
           "same_config": n_all == args.n,
           "sample": "%dx%d grid of the benchmark generator (seed, physics, 2 m layer), "
                     "%d steps after %d untimed, %.1f s, OpenMP %d threads"
                     % (n_all, n_all, s_all, max(1, warmup), el_all, cores),
           "threads_all": {"threads": int(cores), "grid": [n_all, n_all], "value": v_all,
                           "steps": s_all, "seconds": el_all},
           "cpu": cpu_info()}
    if single_thread:
        p1, st1, q1 = workload(args.cpu1_n, args.layer)
        v1, n1, el1 = _time_oracle(args, p1, st1, q1, 1, timing, 12.0)
        out["threads_1"] = {"threads": 1, "grid": [args.cpu1_n, args.cpu1_n], "value": v1,
                            "steps": n1, "seconds": el1}
    return out


def cpu_parity(args, device):
    """The GPU path against the oracle's checker build on the CPU baseline's
    sample (same instance, same steps through advance): masks, t and every
    conserved variable after the steps."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    from imex_sflow2d_v2_b200.solver import ImexSolver
    p, st, q = workload(args.parity_n, args.layer)
    steps = args.parity_steps
    o = orc.Oracle(p, st, threads=orc.lib().oracle_max_threads())
    g = ImexSolver(p, st, device=device)
    for x in (o, g):
        x.set_state(q, 0.0)
        x.set_clock(0.0, 1e-2)
    _, to = o.advance(steps)
    _, tg = g.advance(steps)
    qo, qg = o.get_state(), g.get_state()
    masks = all(np.array_equal(a, b) for a, b in zip(o.get_masks(), g.get_masks()))
    den = float(np.abs(qo).sum())
    rl1 = float(np.abs(qo - qg).sum()) / den if den > 0 else float(np.abs(qo - qg).sum())
    ex = all(np.array_equal(a, b) for a, b in zip(o.get_exchange(), g.get_exchange()))
    so, sg = o.stats(), g.stats()
    g.close()
    return {"workload": "%dx%d instance of the benchmark generator" % (args.parity_n, args.parity_n),
            "steps": steps, "masks_equal": bool(masks), "q_equal": bool(np.array_equal(qo, qg)),
            "exchange_equal": bool(ex), "rel_l1": rl1, "t_equal": bool(to == tg),
            "newton_iters_equal": bool(so.newton_iters == sg.newton_iters),
            "stale_wet_reads": int(o.stale_wet_reads()), "tolerance_rel_l1": 1e-10}


CHUNK = 50


def _oracle_config_rate(p, st, q, steps, budget_s):
    """The oracle's timing build (all host threads) on a workload from its
    initial state, advanced in chunks of CHUNK steps until `steps` are done
    or `budget_s` seconds have passed: (steps done, seconds, threads)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as orc
    timing = orc.timing_build_usable()
    orc.build(target=orc.TIMING if timing else orc.CHECKER)
    # every host thread this process may run on (OpenMP's current maximum
    # is whatever the last Oracle set, 1 after the one-thread baseline)
    threads = len(os.sched_getaffinity(0))
    o = orc.Oracle(p, st, threads=threads, timing=timing)
    o.set_state(q, 0.0)
    o.set_clock(0.0, 1e-2)
    done, el = 0, 0.0
    while done < steps and el < budget_s:
        n_ = min(CHUNK, steps - done)
        t0 = time.perf_counter()
        o.advance(n_)
        el += time.perf_counter() - t0
        done += n_
    return done, el, int(threads)


def config_rates(args, device, cpu=True):
    """Cell-updates/s of the first two workloads at their stated sizes and
    step counts, each run from its initial state through advance() replayed
    from a CUDA graph (device time by CUDA events on the library's stream,
    one event per chunk of CHUNK steps).  With `cpu`, the oracle's timing
    build runs the same workload from the same initial state on all host
    threads for the stated steps or a time budget, whichever ends first, and
    the GPU's time over those same first steps sits beside it."""
    import torch
    from imex_sflow2d_v2_b200 import configs
    from imex_sflow2d_v2_b200.solver import ImexSolver
    out = {}
    for name, (p, st, q), steps, budget in (
            ("dambreak_200", configs.dambreak(), 500, 30.0),
            ("radial_current_1024", configs.radial_current(), 2000, 25.0)):
        g = ImexSolver(p, st, device=device)
        stream = torch.cuda.current_stream()
        g.set_stream(stream.cuda_stream)
        g.set_state(q, 0.0)
        g.set_clock(0.0, 1e-2)
        g.sync()
        evs = [torch.cuda.Event(enable_timing=True)]
        evs[0].record(stream)
        for chunk in range(0, steps, CHUNK):
            g.advance(min(CHUNK, steps - chunk), use_graph=True)
            evs.append(torch.cuda.Event(enable_timing=True))
            evs[-1].record(stream)
        torch.cuda.synchronize()
        ms = evs[0].elapsed_time(evs[-1])
        s_ = g.stats()
        out[name] = {"grid": [p.nx, p.ny], "steps": steps,
                     "value": p.nx * p.ny * steps / (ms * 1e-3), "unit": UNIT,
                     "ms_per_step": ms / steps, "solve_cells_last_step": int(s_.solve_cells),
                     "t_end": s_.t, "errors": int(s_.error_mask)}
        g.close()
        if cpu:
            done, el, threads = _oracle_config_rate(p, st, q, steps, budget)
            gms = evs[0].elapsed_time(evs[(done + CHUNK - 1) // CHUNK])
            cv = p.nx * p.ny * done / el
            gv = p.nx * p.ny * done / (gms * 1e-3)
            out[name]["cpu_oracle"] = {
                "steps": done, "seconds": el, "threads": threads, "value": cv, "unit": UNIT,
                "kind": "port", "gpu_value_same_steps": gv, "gpu_over_cpu": gv / cv,
                "sample": "steps 1..%d of the same run from its initial state" % done}
    return out


def run_ensemble_streams(args):
    """The ensemble workload through per-member graphs over streams (the
    mode the batched one replaces), for comparison; same timing rule."""
    from imex_sflow2d_v2_b200 import configs
    from imex_sflow2d_v2_b200.solver import ImexEnsemble
    mem = configs.ensemble_members(n_members=args.ens_members)
    ens = ImexEnsemble([(p, st) for p, st, q, s in mem])
    ens.set_mode(per_member_graphs=True)
    for m, (p, st, q, s) in enumerate(mem):
        ens.member(m).set_state(q, 0.0)
        ens.member(m).set_clock(0.0, 1e-2)
    n_tune = 6      # stream counts 1, 2, 4, 8, 16, 32
    ens.advance(n_tune)
    t0 = time.perf_counter()
    ens.advance(args.ens_steps - n_tune)
    el = time.perf_counter() - t0
    per_run = el * args.ens_steps / (args.ens_steps - n_tune)
    k, tried = ens.tuning()
    ens.close()
    return {"seconds": per_run, "members_per_hour": args.ens_members * 3600.0 / per_run,
            "k_streams": k, "tuning_ms_per_step": tried}


def run_ensemble(args):
    """Batched ensemble (fourth workload): members/hour for `ens_steps` steps
    of every member.  The first six steps (the tuner's trials of the tile
    shapes; real steps of the run) are taken before the timed region; the
    rate is scaled to all `ens_steps` steps."""
    import math
    from imex_sflow2d_v2_b200 import configs
    from imex_sflow2d_v2_b200.solver import ImexEnsemble
    mem = configs.ensemble_members(n_members=args.ens_members)
    ens = ImexEnsemble([(p, st) for p, st, q, s in mem])
    for m, (p, st, q, s) in enumerate(mem):
        ens.member(m).set_state(q, 0.0)
        ens.member(m).set_clock(0.0, 1e-2)
    cells = sum(p.nx * p.ny for p, *_ in mem)
    n_tune = 6
    t0 = time.perf_counter()
    ens.advance(n_tune)
    tune_s = time.perf_counter() - t0
    t0 = time.perf_counter()
    rc, bad = ens.advance(args.ens_steps - n_tune)
    el = time.perf_counter() - t0
    per_run = el * args.ens_steps / (args.ens_steps - n_tune)
    shape, tried = ens.tile_shape()
    k, tried_k = ens.tuning()
    flagged, finite, solve = [], 0, 0
    for m in range(len(mem)):
        st_ = ens.member(m).stats()
        solve += int(st_.solve_cells)
        if st_.error_mask:
            flagged.append({"member": m, "error_mask": int(st_.error_mask)})
        q = ens.member(m).get_state()
        finite += int(bool(math.isfinite(float(q.sum()))))
    ens.close()
    return {"members": args.ens_members, "steps_per_member": args.ens_steps,
            "cells_total": cells, "seconds": per_run,
            "members_per_hour": args.ens_members * 3600.0 / per_run,
            "cell_updates_per_s": cells * args.ens_steps / per_run,
            "mode": "batched" if shape != (0, 0) else "per-member graphs over streams",
            "tile_shape": list(shape), "tile_shape_trials_ms": [[list(s_), ms] for s_, ms in tried],
            "k_streams": k, "tuning_ms_per_step": tried_k,
            "tuning_steps": n_tune, "tuning_seconds": tune_s,
            "timing": "host clock around the synchronous advance of steps %d..%d (the tuner's "
                      "%d trial steps before it), scaled to %d steps"
                      % (n_tune + 1, args.ens_steps, n_tune, args.ens_steps),
            "solve_cells_last_step": solve,
            "members_finite_at_end": finite,
            "members_with_reference_checks": flagged[:16],
            "n_members_with_reference_checks": len(flagged),
            "data": "synthetic (seeded sampler: side U{256..1024}, bump height U[5,50] m, "
                    "sigma U[50,300] m, mfr logU[1e6,1e8] kg/s, T U[600,1200] K, "
                    "d logU[1e-5,1e-3] m; zero-gradient boundaries)"}


def run_setup(args):
    """Set-up on the device (DEM sampling, cell fractions, restart regridding):
    kernel and end-to-end times at the benchmark's grid size against the CPU
    oracle on bounded samples of the same routines."""
    import numpy as np
    from imex_sflow2d_v2_b200 import configs
    from imex_sflow2d_v2_b200 import grid_setup as GS
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n, cs = args.n, 10.0
    out = {}
    # DEM of n+2 nodes at the grid's spacing, nodes half a cell west/south of
    # the cell centres (the reference's node-centred rasters)
    z = configs.fractal_dem(n + 2, cs, 0.8, 800.0, 15.0, 20261203)
    dem = GS.Raster(n + 2, n + 2, -cs, -cs, cs, -9999.0, z)
    GS.init_grid_topography(dem, 64, 64, 0.0, 0.0, cs, check=False)      # warm-up
    t = {}
    t0 = time.perf_counter()
    GS.init_grid_topography(dem, n, n, 0.0, 0.0, cs, check=False, timing=t)
    e2e = time.perf_counter() - t0
    m = min(n, 1024)
    t0 = time.perf_counter()
    O.setup_dem(z[:m + 2, :m + 2], -cs, -cs, cs, -9999.0, m, m, 0.0, 0.0, cs)
    cpu = time.perf_counter() - t0
    out["dem"] = {"cells": n * n, "kernel_ms": t["kernel_ms"], "e2e_ms": e2e * 1e3,
                  "cells_per_s": n * n / (t["kernel_ms"] * 1e-3),
                  "e2e_cells_per_s": n * n / e2e,
                  "cpu_cells_per_s": m * m / cpu, "cpu_sample": "%dx%d grid, 1 thread" % (m, m)}
    # a collapse of radius n/8 cells at the domain centre
    r = cs * n / 8
    c0 = cs * n / 2
    t = {}
    t0 = time.perf_counter()
    f = GS.compute_cell_fract(n, n, 0.0, 0.0, cs, c0, c0, r, 0.7 * r, 30.0, timing=t)
    e2e = time.perf_counter() - t0
    cand = int(np.count_nonzero(f)) or 1
    rc_ = cs * 16
    t0 = time.perf_counter()
    fc = O.cell_fract(64, 64, 0.0, 0.0, cs, 320.0, 320.0, rc_, 0.7 * rc_, 30.0)
    cpu = time.perf_counter() - t0
    cand_cpu = int(np.count_nonzero(fc)) or 1
    out["cell_fract"] = {"grid": [n, n], "radius_m": r, "cells_inside": cand,
                         "kernel_ms": t["kernel_ms"], "e2e_ms": e2e * 1e3,
                         "subgrid_points_per_s": cand * 40000 / (t["kernel_ms"] * 1e-3),
                         "cpu_subgrid_points_per_s": cand_cpu * 40000 / cpu,
                         "cpu_sample": "radius 160 m on a 64x64 grid, OpenMP %d threads"
                                       % (os.cpu_count() or 1)}
    # restart raster at 2.5x the grid's resolution over the whole domain
    nr = int(n * 1.25)
    fin = np.asfortranarray(np.abs(z[:min(nr, n + 2), :min(nr, n + 2)]) * 1e-3)
    ras = GS.Raster(fin.shape[0], fin.shape[1], 0.0, 0.0, cs * 0.8, -9999.0, fin)
    t = {}
    t0 = time.perf_counter()
    GS.regrid_scalar(ras, n, n, 0.0, 0.0, cs, timing=t)
    e2e = time.perf_counter() - t0
    m = min(n, 512)
    t0 = time.perf_counter()
    O.regrid(fin[:int(m * 1.25) + 2, :int(m * 1.25) + 2], 0.0, 0.0, cs * 0.8, -9999.0, m, m,
             0.0, 0.0, cs)
    cpu = time.perf_counter() - t0
    out["regrid"] = {"cells": n * n, "raster": list(fin.shape), "kernel_ms": t["kernel_ms"],
                     "e2e_ms": e2e * 1e3, "cells_per_s": n * n / (t["kernel_ms"] * 1e-3),
                     "cpu_cells_per_s": m * m / cpu, "cpu_sample": "%dx%d grid, 1 thread" % (m, m)}
    return out


def run_output(args, g, p, steps):
    """output_solution from the device at the benchmark's size: the
    .q_2d/.p_2d/ESRI files of one output written by the library's host
    thread while `steps` further steps run, against the same steps without
    output (the cost the output adds to the run)."""
    import tempfile
    import torch
    out = {}
    with tempfile.TemporaryDirectory() as d:
        run = os.path.join(d, "bench")
        g.sync()
        t0 = time.perf_counter()
        g.advance(steps)
        g.sync()
        base = time.perf_counter() - t0
        t0 = time.perf_counter()
        g.output(run, 1, cons=True, phys=True, esri=True)
        t_enq = time.perf_counter() - t0
        g.advance(steps)
        g.sync()
        t_steps = time.perf_counter() - t0
        g.output_wait()
        t_all = time.perf_counter() - t0
        size = sum(os.path.getsize(os.path.join(d, f)) for f in os.listdir(d))
        nfiles = len(os.listdir(d))
    out = {"files": nfiles, "bytes": size, "enqueue_ms": t_enq * 1e3,
           "steps_after_output": steps, "steps_ms_without_output": base * 1e3,
           "steps_ms_with_output": t_steps * 1e3, "output_done_ms": t_all * 1e3,
           "text_MB_per_s": size / 1e6 / t_all, "threads": os.cpu_count(),
           "timing": "host clock; the files are formatted while the steps run"}
    return out


def run_learned(args, g, p):
    """Learned vs plain Newton start (fifth workload): pairs harvested from the
    benchmark's own 4096^2 fractal run (third workload), the network trained
    on them by the library's kernels, then the radial-current workload (1024^2,
    two solid classes, Voellmy) stepped from one state with the plain start
    and with the learned one."""
    import numpy as np
    from imex_sflow2d_v2_b200 import configs, warmstart
    from imex_sflow2d_v2_b200.solver import ImexMLP, ImexSolver
    cells = p.nx * p.ny
    stride = max(1, int(cells // max(1, args.learned_pairs // 5)))
    g.harvest_start(capacity=args.learned_pairs, stride=stride)
    hsteps = 0
    while g.harvest_data()[2] < args.learned_pairs and hsteps < 40:
        g.advance(1)
        hsteps += 1
    g.harvest_stop()
    net = ImexMLP(seed=20261203)
    t0 = time.perf_counter()
    n_pairs, losses = warmstart.train(net, g, epochs=3, batch=8192, lr=2e-3)
    train_s = time.perf_counter() - t0
    # comparison workload: develop the current, then the same steps both ways
    pr, str_, qr = configs.radial_current(nx=args.learned_n, ny=args.learned_n)
    d = ImexSolver(pr, str_)
    d.set_state(qr, 0.0)
    d.set_clock(0.0, 1e-2)
    d.advance(300)
    q_dev, t_dev = d.get_state(), d.stats().t
    d.close()
    out = {}
    states = {}
    for mode in ("plain", "learned"):
        r = ImexSolver(pr, str_)
        r.set_state(q_dev, t_dev)
        r.set_clock(t_dev, 1e-2)
        if mode == "learned":
            r.set_warmstart(net)
        r.profile(True)
        its = cellsn = fb = 0
        steps = 20
        for _ in range(steps):
            r.advance(1)
            st_ = r.stats()
            its += st_.newton_iters
            cellsn += st_.newton_cells
            fb += st_.warm_fallback_cells
        kt = r.kernel_times()
        s2 = sum(kt[k][0] for k in ("stage2_first", "stage2_iter", "stage2_post")) / steps
        states[mode] = r.get_state()
        out[mode] = {"newton_iters_per_cell": its / max(1, cellsn), "newton_cells": cellsn,
                     "stage2_ms_per_step": s2, "fallback_cells": fb}
        r.close()
    a, b = states["plain"], states["learned"]
    diff = float(np.abs(a - b).sum() / max(np.abs(a).sum(), 1e-300))
    net.close()
    return {"train_pairs": n_pairs, "harvest_steps": hsteps, "harvest_stride": stride,
            "train_epochs": len(losses), "train_loss_per_epoch": [float(x) for x in losses],
            "train_seconds": train_s, "compare_workload": "radial current %d^2, 2 solid classes, "
            "Voellmy; 300 plain steps, then 20 steps each way" % args.learned_n,
            "plain": out["plain"], "learned": out["learned"],
            "rel_l1_learned_vs_plain_after_20_steps": diff}


def run_fast(args, p, st, q0, device, cells, g_exact):
    """Fast mode (contracted multiply-adds) on the headline workload: its
    device-timed rate over the same warm-up and timed steps, and its state,
    masks and clock after those steps against the exact mode's (`g_exact`,
    which ran the same steps from the same state)."""
    import numpy as np
    import torch
    from imex_sflow2d_v2_b200.solver import ImexSolver
    gf = ImexSolver(p, st, device=device, fast=True)
    stream = torch.cuda.current_stream()
    gf.set_stream(stream.cuda_stream)
    gf.set_state(q0, 0.0)
    gf.set_clock(0.0, 1e-2)
    for _ in range(args.warmup):
        gf.advance(1)
    gf.sync()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        gf.advance(1)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    qf, qe = gf.get_state(), g_exact.get_state()
    masks = all(np.array_equal(a, b) for a, b in zip(gf.get_masks(), g_exact.get_masks()))
    den = float(np.abs(qe).sum())
    rl1 = float(np.abs(qf - qe).sum()) / den if den > 0 else 0.0
    tf, te = gf.stats().t, g_exact.stats().t
    info = gf.lib.imex_gpu_build_info().decode()
    gf.close()
    return {"value": cells * args.steps / (ms * 1e-3), "unit": UNIT,
            "ms_per_step": ms / args.steps, "build": info,
            "compared_after_steps": args.warmup + args.steps,
            "masks_equal": bool(masks), "rel_l1_vs_exact": rl1,
            "t_rel_diff": abs(tf - te) / max(abs(te), 1e-300),
            "tolerance_rel_l1": 1e-10}


def run_reference(args, rank, world):
    if rank != 0:
        return
    # W untimed steps of the benchmark workload, then up to K timed steps
    # within --ref-budget seconds (at least one)
    cb = cpu_baseline(args, single_thread=False, warmup=args.warmup, budget_s=args.ref_budget,
                      max_steps=args.steps)
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(args.n), "grid": [args.n, args.n],
                       "cells": args.n * args.n, "parallelism": "host threads (OpenMP)",
                       "sample": cb["sample"], "steps_timed": cb["threads_all"]["steps"]},
            "cpu_baseline": cb,
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0},
            "note": "the reference is Fortran; no Fortran compiler in this image, so its "
                    "C++ restatement (the oracle, timing build, the reference's OpenMP "
                    "loops) is timed"}
    print(json.dumps(line), flush=True)


def roofline_line(dom, fp64, achieved, peak, peak_src, traffic, alg_bytes, avg_s, timed,
                  steps_timed, fp64_peak, hbm_frac_s8d, s8d_bytes):
    """The dominant kernel group's roofline.  Flux, Newton and erosion are
    bound by dependent FP64 arithmetic, so their headline fraction is the
    FP64-pipe one; the HBM figures stay beside it: `achieved`/`frac_hbm` from
    the split design's algorithmic bytes, `traffic` (ncu DRAM bytes per
    launch, whose ratio to `alg_bytes_per_launch` measures re-reads and
    spills) and `hbm_frac_s8d` (the whole step against the fused minimum of
    `s8d_bytes_per_cell`)."""
    fp64_bound = fp64 is not None and dom in ("flux", "stage2_first", "stage2_iter", "erosion")
    line = {"kernel": dom,
            "bound": "fp64" if fp64_bound else "hbm",
            "achieved": fp64["achieved_inst_per_s"] / 1e12 if fp64_bound else achieved,
            "peak": fp64["peak_inst_per_s"] / 1e12 if fp64_bound else peak,
            "unit": "T FP64 inst/s" if fp64_bound else "GB/s",
            "frac": fp64["frac"] if fp64_bound else achieved / peak,
            "peak_source": ("measured FP64 FMA chain (k_fp64_probe)" if fp64_bound
                            else peak_src),
            "achieved_hbm_gbs": achieved, "peak_hbm_gbs": peak, "peak_hbm_source": peak_src,
            "frac_hbm": achieved / peak,
            "traffic": traffic, "alg_bytes_per_launch": alg_bytes,
            "traffic_over_alg": (traffic / alg_bytes) if traffic else None,
            "avg_launch_ms": avg_s * 1e3,
            "kernel_ms_per_step": {k: v[0] / steps_timed for k, v in timed.items()},
            "fp64_pipe": fp64, "fp64_fma_peak_gflops": fp64_peak,
            "hbm_frac_s8d": hbm_frac_s8d, "s8d_bytes_per_cell": s8d_bytes}
    return line


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    import numpy as np
    import torch
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=300))
    from imex_sflow2d_v2_b200 import build as b
    from imex_sflow2d_v2_b200.solver import ImexSolver, measure_fp64_peak
    b.build()
    p, st, q0 = workload(args.n, args.layer)
    n = args.n
    cells = n * n
    g = ImexSolver(p, st, device=local)
    stream = torch.cuda.current_stream()
    g.set_stream(stream.cuda_stream)
    g.set_state(q0, 0.0)
    g.set_clock(0.0, 1e-2)
    for _ in range(args.warmup):
        g.advance(1)
    g.sync()
    s0 = g.stats(reset_errors=True)
    g.profile(True)
    sampler = ClockSampler(local)
    sampler.start()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        g.advance(1)
    ev1.record(stream)
    torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    clocks = sampler.stop()
    kt = g.kernel_times()
    g.profile(False)
    s1 = g.stats()
    from imex_sflow2d_v2_b200.replicas import job_rate
    value, sec = job_rate(ms * 1e-3, cells * args.steps, dist, "cuda")
    ms = sec * 1e3
    if dist:
        dist.barrier()
    launches = int(s1.kernel_launches - s0.kernel_launches)
    newton_per_cell = s1.newton_iters / max(1, s1.newton_cells)

    # roofline of the dominant kernel (event times from the timed region)
    erosion = bool(p.erosion_coeff != 0.0 or p.settling_flag)
    hist = list(s1.newton_hist)
    ncells_newton = max(1, s1.newton_cells)
    listed = (sum(hist[1:]) / cells, sum(hist[2:]) / cells, sum(hist[3:]) / cells)
    bpc = bytes_per_cell(p.n_solid, erosion, listed)
    timed = {k: v for k, v in kt.items() if v[1] > 0}
    dom = max(timed, key=lambda k: timed[k][0])
    steps_timed = args.steps
    dom_ms = timed[dom][0] / steps_timed            # per step (a group may be several launches)
    avg_s = dom_ms * 1e-3
    alg_bytes = bpc[dom] * cells
    peak = None
    peak_src = "fallback"
    try:
        peak = float(json.load(open(PEAKS_FILE))["hbm_gbs"])
        peak_src = "measured"
    except Exception:
        peak = FALLBACK_HBM_GBS
    achieved = alg_bytes / avg_s / 1e9
    traffic = None
    try:
        tr = json.load(open(os.path.join(ROOT, "profiles", "traffic.json")))
        traffic = tr.get(dom)
    except Exception:
        pass
    fp64_peak = None
    try:
        fp64_peak = measure_fp64_peak(local)
    except Exception:
        pass
    # FP64 pipe: instructions per cell (ncu) x cells / live kernel time, against
    # the measured FMA-chain peak (one FP64 instruction per lane per FMA)
    fpc = fp64_counts().get(BUILD_MODE, {})
    fp64 = None
    fp64_all = {}
    if fp64_peak:
        peak_inst_s = fp64_peak * 1e9 / 2.0
        for k_, (tot_ms, _) in timed.items():
            if fpc.get(k_):
                fp64_all[k_] = fpc[k_] * cells / (tot_ms / steps_timed * 1e-3) / peak_inst_s
        if dom in fpc:
            inst_s = fpc[dom] * cells / avg_s
            fp64 = {"kernel": dom, "inst_per_cell": fpc[dom], "achieved_inst_per_s": inst_s,
                    "peak_inst_per_s": peak_inst_s, "frac": inst_s / peak_inst_s,
                    "peak_source": "measured FP64 FMA chain (k_fp64_probe)",
                    "frac_per_kernel": fp64_all}
    # the whole step against the HBM roofline of the fused minimum traffic:
    # 8*(3*n_v + 2) + 1 bytes per cell plus 8*(3*n_s*2) for the erosion planes
    nv_ = 4 + p.n_solid
    s8d_bytes = 8 * (3 * nv_ + 2) + 1 + (8 * 3 * p.n_solid * 2 if erosion else 0)
    hbm_frac_s8d = s8d_bytes * cells / (ms / args.steps * 1e-3) / 1e9 / peak

    # end to end through the public API with pinned host buffers
    e2e = None
    if not args.no_e2e:
        nv = 4 + p.n_solid
        hq = torch.empty(nv * cells, dtype=torch.float64, pin_memory=True).numpy()
        hq[:] = np.asarray(q0).ravel(order="F")
        g.set_clock(0.0, 1e-2)
        g.sync()
        if dist:
            dist.barrier()
        # one untimed call: the first one on a context creates its transfer
        # stream and events and loads the band kernels
        g.advance_host(hq, 0.0, out=hq)
        hq[:] = np.asarray(q0).ravel(order="F")
        g.set_clock(0.0, 1e-2)
        g.sync()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            g.advance_host(hq, 0.0, out=hq)
        g.sync()
        el = time.perf_counter() - t0
        e2e_rate, el = job_rate(el, cells * args.e2e_steps, dist, "cuda")
        # the same steps as three calls (state up, step, state down), whose
        # transfers cannot overlap the step
        hq[:] = np.asarray(q0).ravel(order="F")
        g.set_clock(0.0, 1e-2)
        g.sync()
        if dist:
            dist.barrier()
        t0 = time.perf_counter()
        for _ in range(args.e2e_steps):
            g.set_state(hq, 0.0)
            g.advance(1)
            g.get_state(out=hq)
        g.sync()
        el3 = time.perf_counter() - t0
        calls_rate, _ = job_rate(el3, cells * args.e2e_steps, dist, "cuda")
        e2e = {"value": e2e_rate, "unit": UNIT,
               "h2d_bytes_per_step": nv * cells * 8, "d2h_bytes_per_step": nv * cells * 8,
               "steps": args.e2e_steps,
               "api": "imex_gpu_advance_host (pinned host q in and out, transfers in row "
                      "bands overlapped with the step)",
               "three_calls": {"value": calls_rate, "unit": UNIT,
                               "api": "imex_gpu_set_state + imex_gpu_advance(1) + "
                                      "imex_gpu_get_state"}}

    fast = None
    if rank == 0 and world == 1 and not args.no_fast:
        # the exact context ran warm-up + timed steps from q0; the e2e leg
        # re-ran it from q0, so bring it to the same step count again
        if not args.no_e2e:
            g.set_state(q0, 0.0)
            g.set_clock(0.0, 1e-2)
            g.advance(args.warmup + args.steps)
        fast = run_fast(args, p, st, q0, local, cells, g)
    learned = None
    if rank == 0 and world == 1 and not args.no_learned:
        learned = run_learned(args, g, p)
    g.close()
    ensemble = None
    if rank == 0 and world == 1 and not args.no_ensemble:
        ensemble = run_ensemble(args)
        if args.ens_compare:
            ensemble["per_member_graphs"] = run_ensemble_streams(args)
    setup = None
    if rank == 0 and world == 1 and not args.no_setup:
        setup = run_setup(args)
    output = None
    if rank == 0 and world == 1 and args.output_n > 0:
        po, sto, qo = workload(args.output_n, args.layer)
        go = ImexSolver(po, sto, device=local)
        go.set_state(qo, 0.0)
        go.set_clock(0.0, 1e-2)
        go.advance(3)
        output = run_output(args, go, po, 20)
        output["grid"] = [args.output_n, args.output_n]
        go.close()
    cb = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_baseline(args)
    parity = None
    if rank == 0 and world == 1 and args.parity_steps > 0:
        parity = cpu_parity(args, local)
    rates = None
    if rank == 0 and world == 1 and not args.no_config_rates:
        rates = config_rates(args, local, cpu=not args.no_cpu_baseline)
        rates["fractal_inlet_%d" % n] = {"grid": [n, n], "steps": args.steps, "value": value,
                                         "unit": UNIT, "ms_per_step": ms / args.steps,
                                         "note": "the headline value (2 m initial layer)"}
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_name(n),
                       "grid": [n, n], "cells": cells, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "inputs larger than L2 (state %.2f GB)" % (8 * (4 + p.n_solid) * cells / 1e9),
                       "solve_cells_per_step": int(s1.solve_cells)},
            "newton_iters_per_cell": newton_per_cell,
            "newton_cells_per_step": s1.newton_cells,
            "newton_hist": hist[:6],
            "lnsrch_trials_per_cell": s1.lnsrch_trials / ncells_newton,
            "gpu_launches": launches,
            "clocks": clocks,
            "roofline": roofline_line(dom, fp64, achieved, peak, peak_src, traffic, alg_bytes,
                                      avg_s, timed, steps_timed, fp64_peak, hbm_frac_s8d,
                                      s8d_bytes),
            "e2e": e2e,
            "cpu_baseline": cb,
            "errors": int(s1.error_mask),
            "build": BUILD_MODE,
            "parity": parity,
            "config_rates": rates,
            "fast_mode": fast,
            "ensemble": ensemble,
            "learned_vs_plain": learned,
            "setup": setup,
            "output": output,
        }
        print(json.dumps(line), flush=True)
    g.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
