#!/usr/bin/env python
"""Throughput of the CloverLeaf hydro step on B200: cell-steps/s and the
fraction of the HBM roofline, FP64 plain form and FP32 form in the same run.

Workload: the reference benchmark problem (InputDecks/clover_bm*.in physics:
background rho=0.2 e=1.0, rectangle [0,5]x[0,2] rho=1.0 e=2.5 on [0,10]^2,
gamma 1.4, reflective) on a 7680x7680 mesh.  One "step" is one hydro
timestep of the reference driver (timestep, PdV predictor, accelerate, PdV
corrector, flux_calc, advection, reset_field, and field_summary every 10
steps).  The headline runs the timed steps as one device-resident CUDA graph
through the C ABI's cb_run with fuse = 1 (dt on the device; ideal_gas,
viscosity and calc_dt in one pass; the PdV predictor, accelerate, the PdV
corrector and flux_calc in one pass; reset_field inside the second sweeps:
FP64 results identical to the bit to the phase-by-phase calls).  The same
steps enqueued phase by phase in the driver's call order, with the driver's
per-step dt read-back, are timed too (host_loop), with CUDA events at every
phase boundary; the roofline's kernel, the fused Lagrangian pass, is timed
the same way in a host loop with the chunk's call fusion on (the graph's
fused passes launched one by one, an event pair around each).  Every field array is 472 MB, far above
the 126 MB L2, so no flush is needed between steps.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference]

Besides the headline FP64 line, the same JSON line carries: the FP32 form on
the same deck and dt sequence (speed-up and errors against FP64), FP64 at
15360^2, the batched ensemble of 512 seeded decks in one persistent launch
(FP64 and FP32, autotuned, against the same decks run one after the other),
the adjoint at 480^2 x 200 steps (timings, dot-product test, finite
differences), the reference's own CUDA model on the same deck and GPU, the
end-to-end figure through the C ABI with host buffers, and the reference
OpenMP build on the host cores (cpu_baseline).

N > 1 runs under torchrun: the path does not shard (one mesh per GPU, no
decomposition), so each rank advances its own replica
and value is the sum over ranks (weak scaling).  --impl reference times the
reference's own OpenMP build (oracle/_ref/omp) on the host cores instead.
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "oracle"))

METRIC = "cell-steps/s and % HBM roofline: FP64 plain vs FP32 form at stated error"
UNIT = "cell-steps/s"
# Array touches per cell of each driver-level phase (the algorithmic byte count:
# one read of each distinct full-grid input, one write of each output).
PHASE_ARRAYS = {"ideal_gas": 4, "viscosity": 5, "calc_dt": 8, "pdv_predict": 11 + 4 + 4, "accelerate": 10,
                "pdv_correct": 13, "flux_calc": 8, "advec_cell_s1": 8, "advec_mom_s1": 8, "advec_cell_s2": 7,
                "advec_mom_s2": 7, "reset_field": 8, "field_summary": 10}
# the Lagrangian pass's own distinct arrays: reads xvel0, yvel0, density0, energy0,
# pressure, viscosity; writes pressure, soundspeed, xvel1, yvel1, density1,
# energy1, vol_flux_x, vol_flux_y (the four phases it replaces count 50)
LAGRANGIAN_ARRAYS = 14
LAGRANGIAN_REPLACES = ("pdv_predict", "accelerate", "pdv_correct", "flux_calc")
STEP_ARRAYS = 105  # the step's phases, ideal_gas .. reset_field
LARGE_STEPS = 50  # the 15360^2 deck runs 50 steps
# The advection passes of the fused step and their own distinct arrays: the x
# sweep as one pass reads density1, energy1, vol_flux_x, vol_flux_y, xvel1,
# yvel1 and writes density1, energy1, mass_flux_x, xvel1, yvel1 (as the
# second sweep: level 0 in place of level 1, no vol_flux_y read, density1
# kept: 11 as well); the y sweep as the first sweep: advec_cell 4 + 3,
# advec_mom 5 + 2; as the second sweep with reset_field's copy: advec_cell
# density1, energy1, vol_flux_y read, density1, density0, energy0,
# mass_flux_y written, advec_mom xvel1, yvel1, density1, mass_flux_y read,
# xvel0, yvel0 written
SWEEP_ARRAYS = {"x_sweep": 11, "y_sweep_first": 14, "y_sweep_second": 13}
SWEEP_MARKS = ("advec_cell_s1", "advec_mom_s1", "advec_cell_s2", "advec_mom_s2", "reset_field")


def max_over_ranks(ms, device):
    """The slowest rank's time (ms) for the whole-job figure: one all_reduce(MAX)
    of the device-timed elapsed time, the only collective of a replicas run."""
    import torch
    t = torch.tensor([float(ms)], dtype=torch.float64, device=device)
    torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
    return float(t.item())


def replicas_value(cells, steps, world, ms_max):
    """Whole-job cell-steps/s of `world` replicas that each advanced `cells`
    cells for `steps` steps, timed by the slowest."""
    return cells * steps * world / (ms_max / 1e3)


def _plain(o):
    """numpy scalars in the JSON line as plain numbers."""
    if hasattr(o, "item"):
        return o.item()
    raise TypeError(f"not JSON serialisable: {type(o).__name__}")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
         "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
         "clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.p = None
        self.path = None

    def __enter__(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "100"],
                                      stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        if self.p is None or not self.path or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            w = [x.strip() for x in line.split(",")]
            if len(w) < 9:
                continue
            try:
                sm.append(float(w[1]))
                mx = float(w[2])
            except ValueError:
                continue
            for n, v in zip(names, w[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def bench_deck(cells, gamma=1.4):
    from cloverleaf_b200 import benchmark_deck, nudged
    d = benchmark_deck(cells, end_step=10 ** 9, end_time=1.0e30)
    d.gamma = gamma
    return nudged(d)


class PhaseTimer:
    """CUDA events on the chunk's own stream at every phase boundary.  With
    `run`, the advection marks carry the step's first direction ("@x" when
    the x sweep goes first, "@y" otherwise)."""

    def __init__(self, chunk, run=None):
        import torch
        self.torch = torch
        self.stream = torch.cuda.ExternalStream(chunk.stream())
        self.marks = []
        self.run = run

    def __call__(self, name):
        e = self.torch.cuda.Event(enable_timing=True)
        e.record(self.stream)
        if self.run is not None and name in SWEEP_MARKS:
            name += "@x" if self.run.advect_x else "@y"
        self.marks.append((name, e))

    def totals(self):
        tot, cnt = {}, {}
        for (n, a), (_, b) in zip(self.marks, self.marks[1:]):
            if n == "end":
                continue
            tot[n] = tot.get(n, 0.0) + a.elapsed_time(b)
            cnt[n] = cnt.get(n, 0) + 1
        return tot, cnt


def run_form(precision, cells, warmup, steps, forced_dt=None, with_phases=False, rank=0, world=1, fuse_calls=False,
             tag_sweeps=False):
    """Sets up a chunk, runs warmup steps, then times `steps` steps; returns
    (ms, run, chunk, phase totals, launches in the timed region).  With
    `fuse_calls` the chunk runs the driver's calls as the fused passes (one
    launch each): the calc_dt mark times the ideal_gas + viscosity + calc_dt
    pass (and the dt read-back), flux_calc the Lagrangian pass, reset_field
    the two second sweeps."""
    import torch
    from cloverleaf_b200 import Chunk, HydroRun
    dk = bench_deck(cells)
    dev = torch.cuda.current_device()
    c = Chunk(cells, cells, precision=precision, device=dev)
    run = HydroRun(c, dk, forced_dt=forced_dt, fuse_calls=fuse_calls)
    run.start()
    for _ in range(warmup):
        run.hydro_step()
    ext = torch.cuda.ExternalStream(c.stream())
    timer = PhaseTimer(c, run if tag_sweeps else None) if with_phases else None
    run.probe = timer
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    n0 = c.launch_count()
    t0.record(ext)
    for _ in range(steps):
        run.hydro_step()
    t1.record(ext)
    c.synchronize()
    torch.cuda.synchronize()
    n1 = c.launch_count()
    if world > 1:
        torch.distributed.barrier()
    run.probe = None
    ms = t0.elapsed_time(t1)
    phases = timer.totals() if timer else None
    return ms, run, c, phases, n1 - n0


def resident_form(precision, cells, warmup, steps, rank=0, world=1, fuse=True):
    """Sets up a chunk, runs `warmup` steps as one device-resident graph
    (cb_run), then times `steps` steps as another cb_run call, which launches
    again the graph the warm-up call captured and instantiated (the chunk keeps
    it); returns (ms, run, chunk, launches in the timed region)."""
    import torch
    from cloverleaf_b200 import Chunk, HydroRun
    dk = bench_deck(cells)
    c = Chunk(cells, cells, precision=precision, device=torch.cuda.current_device())
    run = HydroRun(c, dk)
    run.start()
    run.run_steps_on_device(max_steps=run.step + warmup, fuse=fuse)
    ext = torch.cuda.ExternalStream(c.stream())
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c.synchronize()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    n0 = c.launch_count()
    t0.record(ext)
    run.run_steps_on_device(max_steps=run.step + steps, fuse=fuse)
    t1.record(ext)
    c.synchronize()
    torch.cuda.synchronize()
    n1 = c.launch_count()
    if world > 1:
        torch.distributed.barrier()
    return t0.elapsed_time(t1), run, c, n1 - n0


# fields the fused graph must leave bit-identical to the phase-by-phase loop
CHECKED_FIELDS = ("density0", "energy0", "xvel0", "yvel0", "pressure", "soundspeed", "viscosity")


def fused_identity(fused_final, fused_dt, fused_summaries, chunk, run):
    """Compares the fused graph's final state, dt sequence and summaries
    with the phase-by-phase loop's after the same steps of the same deck:
    every value must agree to the bit (the fused kernels evaluate the same
    expressions in the same order)."""
    import numpy as np
    bad = []
    for n in CHECKED_FIELDS:
        a, b = fused_final[n], chunk.read(n)
        if not np.array_equal(a.view(np.int64), b.view(np.int64)):
            bad.append(f"{n}: {int((a.view(np.int64) != b.view(np.int64)).sum())} values differ")
    if fused_dt != list(run.dt_trace):
        bad.append("dt sequence differs")
    if [tuple(vars(x).values()) for x in fused_summaries] != [tuple(vars(x).values()) for x in run.summaries]:
        bad.append("summaries differ")
    return {"bit_identical": not bad, "fields": list(CHECKED_FIELDS), "steps": len(fused_dt),
            "also": "dt of every step, every summary record", "mismatches": bad}


def rel_errors(a64, a32):
    import numpy as np
    d = np.abs(a32 - a64)
    den = np.abs(a64)
    floor = 1e-12 * den.max() if den.max() > 0 else 1e-300
    return float(d.sum() / den.sum()) if den.sum() > 0 else float(d.sum()), float((d / np.maximum(den, floor)).max())


def e2e_run(cells, warmup, steps):
    """The same metric through the public C ABI with host buffers: the timed
    region uploads the step-0 state (density0, energy0, xvel0, yvel0) from
    pinned host memory, advances `steps` steps as the headline does (cb_run,
    fused; its dt trace and summaries come back to the host) and reads the
    final state back to pinned host memory."""
    import numpy as np
    import torch
    from cloverleaf_b200 import Chunk, HydroRun
    dk = bench_deck(cells)
    c = Chunk(cells, cells, device=torch.cuda.current_device())
    run = HydroRun(c, dk)
    run.start()
    names = ["density0", "energy0", "xvel0", "yvel0"]
    host = {n: torch.empty(tuple(reversed(c.extent(n))), dtype=torch.float64, pin_memory=True).numpy() for n in names}
    for n in names:
        host[n][...] = c.read(n)
    run.run_steps_on_device(max_steps=warmup, fuse=True)
    run2 = HydroRun(c, dk)
    run2.summaries = []
    ext = torch.cuda.ExternalStream(c.stream())
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    c.synchronize()
    torch.cuda.synchronize()
    t0.record(ext)
    for n in names:
        c.write(n, host[n])
    run2.run_steps_on_device(max_steps=steps, fuse=True)
    for n in names:
        c.read_into(n, host[n])
    t1.record(ext)
    torch.cuda.synchronize()
    ms = t0.elapsed_time(t1)
    h2d = sum(host[n].nbytes for n in names)
    d2h = sum(host[n].nbytes for n in names) + 8 * steps + 40 * len(run2.summaries)
    c.close()
    return ms, h2d, d2h


def resident_leg(sizes=((960, 87), (7680, 100)), warmup=3):
    """The whole hydro loop as one device-resident CUDA graph (cb_run, without
    and with fused passes) against the host-driven loop (dt read back every
    step: the reference driver's path) -- phase by phase, with call fusion,
    and with call fusion and the Lagrangian pass run ahead from calc_dt --
    FP64, same deck, same steps; ms per step from CUDA events on the chunk's
    stream around the whole loop (the graph's capture and instantiation
    included)."""
    import torch
    from cloverleaf_b200 import Chunk, HydroRun
    out = []
    for cells, steps in sizes:
        row = {"cells": f"{cells}x{cells}", "steps": steps}
        for mode in ("host_loop", "host_loop_fused_calls", "host_loop_fused_ahead", "device_graph", "device_graph_fused"):
            c = Chunk(cells, cells, device=torch.cuda.current_device())
            r = HydroRun(c, bench_deck(cells), fuse_calls=mode.startswith("host_loop_fused"), dt_ahead=mode == "host_loop_fused_ahead")
            r.start()
            for _ in range(warmup):
                r.hydro_step()
            ext = torch.cuda.ExternalStream(c.stream())
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            c.synchronize()
            torch.cuda.synchronize()
            t0.record(ext)
            if mode.startswith("device_graph"):
                r.run_steps_on_device(max_steps=r.step + steps, fuse=mode == "device_graph_fused")
            else:
                for _ in range(steps):
                    r.hydro_step()
            t1.record(ext)
            torch.cuda.synchronize()
            ms = t0.elapsed_time(t1)
            row[mode] = {"ms_per_step": ms / steps, "value": cells * cells * steps / (ms / 1e3), "unit": UNIT}
            c.close()
        row["speedup"] = row["host_loop"]["ms_per_step"] / row["device_graph"]["ms_per_step"]
        row["speedup_fused"] = row["host_loop"]["ms_per_step"] / row["device_graph_fused"]["ms_per_step"]
        out.append(row)
    return out


def sweep_rooflines(ftag, ctag, cells, peak):
    """The fused step's advection passes from the call-fused host loop's
    direction-tagged groups: the x sweep as one pass with its edge strip
    (advec_mom_s1 when x goes first, reset_field when y goes first), the y
    sweep as the first sweep (advec_cell_s1 + advec_mom_s1 when y goes first)
    and as the second (reset_field when x goes first); ms per launch and the
    fraction of the peak its own arrays reach."""
    def per(keys, n_key):
        n = ctag.get(n_key, 0)
        return sum(ftag.get(k, 0.0) for k in keys) / n if n else None
    xs = [v for v in (per(["advec_mom_s1@x"], "advec_mom_s1@x"), per(["reset_field@y"], "reset_field@y")) if v]
    ms = {"x_sweep": sum(xs) / len(xs) if xs else None,
          "y_sweep_first": per(["advec_cell_s1@y", "advec_mom_s1@y"], "advec_mom_s1@y"),
          "y_sweep_second": per(["reset_field@x"], "reset_field@x")}
    out = {}
    for k, t in ms.items():
        if t:
            gbs = SWEEP_ARRAYS[k] * 8 * cells * cells / (t / 1e3) / 1e9
            out[k] = {"ms_per_launch": t, "arrays": SWEEP_ARRAYS[k], "achieved": gbs, "frac": gbs / peak}
    return out


def traffic_per_launch(kernel, cells):
    """DRAM bytes per launch from the committed ncu summary, scaled to `cells`."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as f:
            t = json.load(f)
        e = t[kernel]
        return e["dram_bytes_per_cell"] * cells * cells
    except Exception:
        return None


def batch_leg(n_decks, seq_sample):
    """The batched ensemble: n_decks seeded decks of uneven size, each with its
    own gamma and dt, run to t = 0.5 by one persistent launch (FP64 and FP32),
    after the autotuner has picked the schedule; against the same decks run
    one after the other through the C ABI (cb_run per deck: each deck's whole
    run as one device-resident graph with fused passes) on a seeded sample."""
    import numpy as np
    from cloverleaf_b200 import FP32, FP64, Batch, Chunk, HydroRun, ensemble_decks
    from cloverleaf_b200 import batch as B
    decks = ensemble_decks(n_decks)
    out = {"decks": n_decks, "seed": "0xC10E, numpy PCG64", "sides": list(B.ENSEMBLE_SIDES), "end_time": 0.5,
           "cells": int(sum(d.x_cells * d.y_cells for d in decks))}
    finals = {}
    for prec, name in ((FP64, "fp64"), (FP32, "fp32")):
        b = Batch(decks, prec)
        best, trials = b.autotune(repeats=1)
        ms = []
        for _ in range(3):
            b.run()
            ms.append(b.synchronize())
        res = [b.result(k) for k in range(n_decks)]
        cs = sum(d.x_cells * d.y_cells * r.steps for d, r in zip(decks, res))
        t = statistics.median(ms)
        sched, lanes, ctas = b.schedule()
        out[name] = {"value": cs / (t / 1e3), "unit": UNIT, "ms": t, "cell_steps": cs,
                     "done": sum(r.status == B.DECK_DONE for r in res), "steps_min": min(r.steps for r in res),
                     "steps_max": max(r.steps for r in res), "schedule": best, "lanes": lanes, "ctas": ctas,
                     "launches_per_run": 1, "trials": trials}
        finals[name] = [b.read(k, "density0")[2:-2, 2:-2] for k in range(0, n_decks, max(1, n_decks // 64))]
        b.close()
    l1 = [float(np.abs(a - c).sum() / np.abs(a).sum()) for a, c in zip(finals["fp64"], finals["fp32"])]
    out["fp32"]["density_l1_rel_vs_fp64"] = {"max": max(l1), "mean": statistics.mean(l1), "decks_checked": len(l1)}
    sample = decks[::max(1, n_decks // seq_sample)][:seq_sample]
    for prec, name in ((FP64, "sequential_fp64"), (FP32, "sequential_fp32")):
        cs, tsum = 0, 0.0
        for dk in sample:
            c = Chunk(dk.x_cells, dk.y_cells, precision=prec, gamma=dk.gamma)
            r = HydroRun(c, dk)
            r.start()
            c.synchronize()
            t0 = time.perf_counter()
            r.run_steps_on_device(fuse=True)
            c.synchronize()
            tsum += time.perf_counter() - t0
            cs += dk.x_cells * dk.y_cells * r.step
            c.close()
        out[name] = {"value": cs / tsum, "unit": UNIT, "sample": f"{len(sample)} of the {n_decks} decks (every "
                     f"{max(1, n_decks // seq_sample)}th), one after the other, each run to its end as one device-resident "
                     f"graph with fused passes (cb_run, fuse = 1); wall clock incl. the graph's capture"}
    out["speedup_fp64_vs_sequential"] = out["fp64"]["value"] / out["sequential_fp64"]["value"]
    out["speedup_fp32_vs_sequential"] = out["fp32"]["value"] / out["sequential_fp32"]["value"]
    return out


def ke_exact(adj, dk):
    """The final kinetic energy of an Adjoint's primal chunk as an exactly
    rounded sum (math.fsum) of the per-cell terms of field_summary
    (src/serial/field_summary.cpp:70-90), so that finite differences of it
    carry no summation-order noise."""
    import math
    import numpy as np
    nx, ny = dk.x_cells, dk.y_cells
    d = adj.read_field("density0")[2:ny + 2, 2:nx + 2]
    u = adj.read_field("xvel0")
    v = adj.read_field("yvel0")
    vsq = np.zeros((ny, nx))
    for kv in (0, 1):
        for jv in (0, 1):
            uu, vv = u[2 + kv:ny + 2 + kv, 2 + jv:nx + 2 + jv], v[2 + kv:ny + 2 + kv, 2 + jv:nx + 2 + jv]
            vsq = vsq + 0.25 * (uu * uu + vv * vv)
    vol = ((dk.xmax - dk.xmin) / nx) * ((dk.ymax - dk.ymin) / ny)
    return math.fsum(((vol * d) * 0.5 * vsq).ravel())


def adjoint_leg(n=480, steps=200, fd_cells=64, hs=(1e-6, 1e-4)):
    """The adjoint run: the benchmark layout at n x n with a seeded +-5%
    uniform perturbation of every cell's initial density and energy, `steps`
    steps; the gradient of the final kinetic energy by the reverse sweep,
    checked against the tangent-linear run (dot-product test, two seeded
    directions) and against central finite differences of the exactly summed
    kinetic energy at `fd_cells` seeded cells (and gamma), with the forward
    run's dt sequence held fixed, at step h = 1e-6 and, for comparison, 1e-4."""
    import numpy as np
    import torch
    from cloverleaf_b200 import Adjoint, benchmark_deck, nudged
    dk = nudged(benchmark_deck(n, end_step=steps))
    adj = Adjoint(dk, device=torch.cuda.current_device())
    rng = np.random.default_rng(0xAD7)
    rho = adj.read_field("density0")[2:-2, 2:-2] * (1.0 + rng.uniform(-0.05, 0.05, (n, n)))
    e = adj.read_field("energy0")[2:-2, 2:-2] * (1.0 + rng.uniform(-0.05, 0.05, (n, n)))
    adj.set_initial(rho, e, 1.4)
    t0 = time.perf_counter()
    ke = adj.forward(steps)
    t_fwd = time.perf_counter() - t0
    dts = adj.dt()
    t0 = time.perf_counter()
    gr, ge, gg = adj.gradient()
    t_rev = time.perf_counter() - t0
    st = adj.stats()
    dots = []
    t_tan = 0.0
    for k in range(2):
        dr, de, dg = rng.standard_normal((n, n)), rng.standard_normal((n, n)), float(rng.standard_normal())
        t0 = time.perf_counter()
        _, dke = adj.tangent(dr, de, dg)
        t_tan = time.perf_counter() - t0
        lhs = float((gr * dr).sum() + (ge * de).sum() + gg * dg)
        scale = float(np.abs(gr * dr).sum() + np.abs(ge * de).sum() + abs(gg * dg))
        dots.append(abs(lhs - dke) / scale)
    cells = [(int(rng.integers(n)), int(rng.integers(n))) for _ in range(fd_cells)]
    gmax = max(float(np.abs(gr).max()), float(np.abs(ge).max()))
    adj.set_initial(rho, e, 1.4)
    adj.forward(steps, dts)
    j0 = ke_exact(adj, dk)
    fd = {}
    t0 = time.perf_counter()
    for h in hs:
        smooth, kinks = [], 0
        for (j, i) in cells:
            for which, g in (("rho", gr), ("e", ge)):
                vals = []
                for s in (1.0, -1.0):
                    r2, e2 = rho.copy(), e.copy()
                    (r2 if which == "rho" else e2)[j, i] += s * h
                    adj.set_initial(r2, e2, 1.4)
                    adj.forward(steps, dts)
                    vals.append(ke_exact(adj, dk))
                d = (vals[0] - vals[1]) / (2 * h)
                dp, dm = (vals[0] - j0) / h, (j0 - vals[1]) / h
                # a branch of the scheme (limiter, upwind switch) flipping inside
                # [x - h, x + h] shows as one-sided differences that disagree
                if abs(dp - dm) > 0.01 * max(abs(dp), abs(dm), 1e-6 * gmax):
                    kinks += 1
                    continue
                smooth.append(abs(d - g[j, i]) / max(abs(g[j, i]), 1e-6 * gmax))
        vals = []
        for s in (1.0, -1.0):
            adj.set_initial(rho, e, 1.4 + s * h)
            adj.forward(steps, dts)
            vals.append(ke_exact(adj, dk))
        dg_fd = (vals[0] - vals[1]) / (2 * h)
        smooth = sorted(smooth) or [float("nan")]
        fd[f"h={h:g}"] = {"kink_hits": kinks, "smooth_cells": len(smooth), "rel_err_median": smooth[len(smooth) // 2],
                          "rel_err_max": smooth[-1], "over_1e-4": int(sum(x > 1e-4 for x in smooth)),
                          "gamma_fd": dg_fd, "gamma_rel_err": abs(dg_fd - gg) / abs(gg)}
    t_fd = time.perf_counter() - t0
    adj.close()
    # pass rule: the dot-product test against the tangent-linear run is the exact
    # check; the finite differences at h = 1e-6 must agree on the smooth cells
    # (no branch flip within +-h) to a median of 1e-4 relative, and for gamma
    # to 1e-4 (single small derivatives carry the differences' own rounding)
    f6 = fd.get("h=1e-06")
    fd_pass = bool(f6 and f6["smooth_cells"] > 0 and f6["rel_err_median"] <= 1e-4 and f6["gamma_rel_err"] <= 1e-4)
    checks = {"dot_test_pass": max(dots) <= 1e-10, "fd_pass": fd_pass,
              "rule": "dot test <= 1e-10; at h = 1e-6: median rel err over the smooth cells <= 1e-4, gamma rel err <= 1e-4"}
    return {"mesh": f"{n}x{n}", "steps": steps, "perturbation": "+-5% uniform per cell, seed 0xAD7", "ke": ke,
            "forward_s": t_fwd, "gradient_s": t_rev, "tangent_s": t_tan, "fd_s": t_fd,
            "cell_steps_per_s_forward": n * n * steps / t_fwd,
            "checkpoint_interval": st["checkpoint_interval"], "checkpoints": st["checkpoints"],
            "recomputed_steps": st["recomputed_steps"], "device_mb": st["device_bytes"] / 2 ** 20,
            "dot_test_rel": max(dots), "gamma_adjoint": gg, "grad_max_abs": gmax, "checks": checks,
            "fd": {"cells": fd_cells, "objective": "final kinetic energy summed exactly (math.fsum of the per-cell terms)",
                   "rel_err": "|fd - adjoint| / max(|adjoint|, 1e-6 max|grad|), over the smooth cells",
                   "kink_hit": "one-sided differences disagreeing by more than 1%: a branch flips within +-h", **fd}}


def reference_exe():
    return os.path.join(ROOT, "oracle", "_ref", "omp")


def run_reference_omp(cells, steps, threads, timeout=900):
    """Runs the reference OpenMP build on the benchmark deck for `steps` steps;
    returns the per-step "Step time per cell" values the driver prints
    (driver/hydro.cpp:209-220)."""
    from cloverleaf_b200 import benchmark_deck, format_deck
    exe = reference_exe()
    with tempfile.TemporaryDirectory() as tmp:
        deck = os.path.join(tmp, "clover.in")
        with open(deck, "w") as f:
            f.write(format_deck(benchmark_deck(cells, end_step=steps, end_time=1.0e30)))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads), OMP_PROC_BIND="true", OMP_PLACES="cores")
        p = subprocess.run([exe, "--file", deck, "--out", os.path.join(tmp, "clover.out")], cwd=tmp, env=env,
                           capture_output=True, text=True, timeout=timeout)
        if p.returncode != 0:
            raise RuntimeError(f"reference OpenMP build exited {p.returncode}: {p.stdout[-500:]}")
        return [float(x) for x in re.findall(r"Step time per cell\s+([0-9.eE+-]+)", p.stdout)]


def reference_cuda_leg(cells, steps=10, warm=2, timeout=900):
    """The reference's own CUDA model (oracle/_ref/cuda: the unmodified driver
    and src/cuda built for sm_100a with the model's nvcc flags) on the same
    deck and the same B200, for comparison: cell-steps/s from the driver's
    per-step "Step time per cell" lines (driver/hydro.cpp:209-220) after
    `warm` steps, and its final kinetic energy."""
    from cloverleaf_b200 import benchmark_deck, format_deck
    exe = os.path.join(ROOT, "oracle", "_ref", "cuda")
    if not os.path.exists(exe):
        return {"unavailable": "oracle/_ref/cuda was not built (needs the reference sources)"}
    with tempfile.TemporaryDirectory() as tmp:
        deck = os.path.join(tmp, "clover.in")
        with open(deck, "w") as f:
            f.write(format_deck(benchmark_deck(cells, end_step=warm + steps, end_time=1.0e30)))
        p = subprocess.run([exe, "--file", deck, "--out", os.path.join(tmp, "clover.out")], cwd=tmp, capture_output=True, text=True,
                           timeout=timeout)
        if p.returncode != 0:
            return {"error": f"exited {p.returncode}: {p.stdout[-300:]}"}
        per_cell = [float(x) for x in re.findall(r"Step time per cell\s+([0-9.eE+-]+)", p.stdout)][warm:]
        return {"value": 1.0 / statistics.mean(per_cell), "unit": UNIT, "steps": len(per_cell),
                "sample": f"reference CUDA model (src/cuda, nvcc -O3 -extended-lambda -use_fast_math -restrict, sm_100a), "
                          f"{cells}x{cells} benchmark deck, steps {warm + 1}-{warm + len(per_cell)}, driver's per-step timer"}


def cpu_cores():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_baseline(cells):
    """The reference OpenMP build on all host cores, bounded: 3 steps of the
    same deck (the first step is dropped).  Falls back to the C oracle port
    (one core, a 960^2 sample) if the reference build is absent."""
    cores = cpu_cores()
    if os.path.exists(reference_exe()):
        per_cell = run_reference_omp(cells, 4, cores)  # step times of steps 1-3 (the last step prints none)
        v = 1.0 / statistics.mean(per_cell[1:3])
        return {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": f"reference OpenMP build (oracle/_ref/omp, g++ -O3), {cells}x{cells} benchmark deck, "
                          f"steps 2-3 of a 4-step run, OMP_NUM_THREADS={cores}"}
    import oracle
    from cloverleaf_b200 import benchmark_deck, nudged
    dk = nudged(benchmark_deck(960, end_step=3))
    o = oracle.OracleChunk(960, 960)
    t = time.time()
    o.run(dk)
    dt = time.time() - t
    return {"value": 960 * 960 * 3 / dt, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "C oracle port, one core, 960x960 benchmark deck, 3 steps incl. setup"}


def main_reference(args, rank, world):
    if rank != 0:
        return
    cores = cpu_cores()
    if not os.path.exists(reference_exe()):
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/omp was not built (needs the reference sources)"}))
        return
    steps, warm = args.steps, args.warmup
    # the driver prints a step's time after every step but the last: a run of
    # warm + steps + 1 steps gives the `steps` timed values after `warm`
    per_cell = run_reference_omp(args.size, warm + steps + 1, cores, timeout=3600)
    timed = per_cell[warm:warm + steps]
    if len(timed) != steps:
        raise SystemExit(f"bench.py: the reference run printed {len(per_cell)} step times, expected {warm + steps}")
    v = 1.0 / statistics.mean(timed)
    ms = statistics.mean(timed) * args.size * args.size * 1e3
    line = {"metric": METRIC, "value": v, "unit": UNIT, "impl": "reference", "n_gpus": world, "steps": len(timed),
            "warmup": warm, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic: the reference benchmark deck generated in-process",
            "config": {"workload": f"clover_bm FP64 {args.size}x{args.size}, hydro steps", "cells": args.size * args.size,
                       "l2": "inputs larger than L2 (host run)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": f"reference OpenMP build, {args.size}^2, steps {warm + 1}-{warm + len(timed)} of "
                                       f"{warm + steps}, OMP_NUM_THREADS={cores}"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=100)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--size", type=int, default=7680)
    ap.add_argument("--large", type=int, default=15360, help="second FP64 size timed (0 to skip)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--batch", type=int, default=512, help="decks of the batched-ensemble leg (0 to skip)")
    ap.add_argument("--adjoint", type=int, default=480, help="mesh side of the adjoint leg (0 to skip)")
    ap.add_argument("--adjoint-steps", type=int, default=200)
    ap.add_argument("--no-ref-cuda", action="store_true", help="skip timing the reference's CUDA model")
    ap.add_argument("--no-resident", action="store_true", help="skip the device-resident loop leg")
    args = ap.parse_args()

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        return main_reference(args, rank, world)
    if args.warmup < 3:
        raise SystemExit("bench.py: --warmup must be at least 3")

    import torch
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                             device_id=torch.device("cuda", local))
    from cloverleaf_b200 import FP32, FP64

    S = args.size
    peak, peak_kind = peaks()
    # headline: the steps as one device-resident graph (cb_run, fused passes)
    with ClockSampler(local) as clk:
        ms64, run64r, c64r, launches = resident_form(FP64, S, args.warmup, args.steps, rank=rank, world=world)
    clocks = clk.summary()
    if world > 1:
        ms64 = max_over_ranks(ms64, "cuda")
    value = replicas_value(S * S, args.steps, world, ms64)
    ms32r, run32r, c32r, _ = resident_form(FP32, S, args.warmup, args.steps, rank=rank, world=world)
    if world > 1:
        ms32r = max_over_ranks(ms32r, "cuda")
    value32 = replicas_value(S * S, args.steps, world, ms32r)

    def field_errors(ca, cb):
        errs = {}
        for name in ("density0", "energy0", "pressure", "xvel0", "yvel0"):
            l1, mx = rel_errors(ca.read(name)[2:-2, 2:-2], cb.read(name)[2:-2, 2:-2])
            errs[name] = {"l1_rel": l1, "max_rel": mx}
        return errs

    errs_resident = field_errors(c64r, c32r)
    # the fused graph's final state, kept on the host for the bit-identity
    # check against the phase-by-phase loop below (same deck, same steps)
    fused_final = {n: c64r.read(n) for n in CHECKED_FIELDS}
    fused_dt = list(run64r.dt_trace)
    fused_summaries = list(run64r.summaries)
    c64r.close()
    c32r.close()

    # the same steps phase by phase (host loop): per-phase CUDA events for the kernel roofline
    ms64h, run64, c64, phases, _ = run_form(FP64, S, args.warmup, args.steps, with_phases=True, rank=rank, world=world)
    if world > 1:
        ms64h = max_over_ranks(ms64h, "cuda")
    fused_check = fused_identity(fused_final, fused_dt, fused_summaries, c64, run64)
    del fused_final
    # FP32 form phase by phase, replaying the FP64 run's dt sequence: errors against FP64 at the same time
    dts = list(run64.dt_trace)
    ms32, run32, c32, ph32, _ = run_form(FP32, S, args.warmup, args.steps, forced_dt=dts, with_phases=True, world=world)
    if world > 1:
        ms32 = max_over_ranks(ms32, "cuda")
    errs = field_errors(c64, c32)

    def drift(run):
        s0, s1 = run.summaries[0], run.summaries[-1]
        return {"mass": (s1.mass - s0.mass) / s0.mass,
                "total_energy": ((s1.ie + s1.ke) - (s0.ie + s0.ke)) / (s0.ie + s0.ke)}

    fp32 = {"value": value32, "unit": UNIT, "ms_per_step": ms32r / args.steps, "speedup_vs_fp64": value32 / value,
            "path": "cb_run fused, its own dt sequence",
            "errors_vs_fp64": errs, "errors_dt_sequence": "FP32 phase by phase replaying the FP64 run's dt sequence",
            "errors_vs_fp64_resident": errs_resident,
            "errors_resident_dt_sequence": "each form's own dt, compared after the same number of steps",
            "drift_fp64": drift(run64), "drift_fp32": drift(run32),
            "host_loop": {"value": replicas_value(S * S, args.steps, world, ms32), "ms_per_step": ms32 / args.steps},
            "phase_ms_per_step": {k: ph32[0][k] / args.steps for k in sorted(ph32[0])}}
    host_loop = {"value": replicas_value(S * S, args.steps, world, ms64h), "unit": UNIT, "ms_per_step": ms64h / args.steps,
                 "path": "phase-by-phase C ABI calls in the driver's order, dt read back every step"}
    c64.close()
    c32.close()

    large = None
    if args.large:
        try:
            msl, _, cl, _ = resident_form(FP64, args.large, 3, LARGE_STEPS, world=world)
            cl.close()
            if world > 1:
                msl = max_over_ranks(msl, "cuda")
            large = {"cells": f"{args.large}x{args.large}", "steps": LARGE_STEPS,
                     "value": replicas_value(args.large ** 2, LARGE_STEPS, world, msl), "unit": UNIT,
                     "ms_per_step": msl / LARGE_STEPS, "path": "cb_run fused, 3 warm-up steps"}
        except Exception as e:  # memory or other failure is reported, not hidden
            large = {"error": str(e)}

    ms_e2e, h2d, d2h = e2e_run(S, args.warmup, args.steps)
    if world > 1:
        ms_e2e = max_over_ranks(ms_e2e, "cuda")
    e2e = {"value": replicas_value(S * S, args.steps, world, ms_e2e), "unit": UNIT,
           "h2d_bytes_per_step": h2d / args.steps, "d2h_bytes_per_step": d2h / args.steps}

    # roofline of kt_lagrange (the fused Lagrangian pass; the largest share of
    # the step's launch list), with the advection passes beside it: the fused
    # passes in a host loop (call fusion), a CUDA event pair around each group
    # of calls on the chunk's stream; the flux_calc group is the Lagrangian
    # pass (with the pressure's outer-ring copy, a few microseconds)
    lag_steps = min(args.steps, 20)
    msf, _, cf, phf, _ = run_form(FP64, S, args.warmup, lag_steps, with_phases=True, rank=rank, world=world, fuse_calls=True,
                                  tag_sweeps=True)
    cf.close()
    ftag, ctag = phf
    ftot, fcnt = {}, {}
    for k in ftag:  # the groups over both step directions
        g = k.split("@")[0]
        ftot[g] = ftot.get(g, 0.0) + ftag[k]
        fcnt[g] = fcnt.get(g, 0) + ctag[k]
    dom = "flux_calc"
    avg_ms = ftot[dom] / fcnt[dom]
    alg = LAGRANGIAN_ARRAYS * 8 * S * S
    achieved = alg / (avg_ms / 1e3) / 1e9
    traffic = traffic_per_launch("lagrangian", S)  # kt_lagrange's DRAM bytes per cell (profiles/traffic.json)
    tot, cnt = phases
    replaced_ms = sum(tot[k] / cnt[k] for k in LAGRANGIAN_REPLACES)
    roof = {"kernel": "kt_lagrange<double, 8>", "timed_in": f"host loop with call fusion, {lag_steps} steps (flux_calc group)",
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
            "traffic_frac": (traffic / (avg_ms / 1e3) / 1e9 / peak) if traffic else None,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
            else "fallback 6.65 TB/s", "traffic": traffic, "alg_bytes_per_launch": alg, "ms_per_launch": avg_ms,
            "replaced_phases_ms": replaced_ms,
            "replaced_phases_alg_bytes": sum(PHASE_ARRAYS[k] for k in LAGRANGIAN_REPLACES) * 8 * S * S,
            "step_frac": value / world * STEP_ARRAYS * 8 / 1e9 / peak,
            "fused_calls_ms_per_step": msf / lag_steps,
            "fused_calls_phase_ms_per_step": {k: ftot[k] / lag_steps for k in sorted(ftot)},
            "fused_calls_kernels": {"calc_dt": "kt_ig_visc_dt + 8-byte dt read-back", "flux_calc": "kt_lagrange + ring copy",
                                    "advec_cell_s1": "kt_advec_cell (y first; held back when x goes first)",
                                    "advec_mom_s1": "kt_advec_sweep_x + edge strip (x first) / kt_advec_mom (y first)",
                                    "reset_field": "both second sweeps (with reset_field's copy)",
                                    "field_summary": "k_field_summary + 40-byte read-back"},
            "phase_ms_per_step": {k: tot[k] / args.steps for k in sorted(tot)},
            "sweeps": sweep_rooflines(ftag, ctag, S, peak)}

    batch = None
    if args.batch:
        try:
            batch = batch_leg(args.batch, 32)
        except Exception as e:
            batch = {"error": str(e)}

    adjoint = None
    if args.adjoint:
        try:
            adjoint = adjoint_leg(args.adjoint, args.adjoint_steps)
        except Exception as e:
            adjoint = {"error": str(e)}

    resident = None
    if not args.no_resident:
        try:
            resident = resident_leg(((960, 87), (S, 100)))
        except Exception as e:
            resident = {"error": str(e)}

    ref_cuda = None
    if rank == 0 and world == 1 and not args.no_ref_cuda:
        try:
            ref_cuda = reference_cuda_leg(S)
            if "value" in ref_cuda:
                ref_cuda["b200_speedup"] = value / ref_cuda["value"]
        except Exception as e:
            ref_cuda = {"error": str(e)}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            cpu = cpu_baseline(S)
        except Exception as e:
            cpu = {"error": str(e)}

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms64 / args.steps,
                # compact figures first: the fused graph's parity with the phase-by-phase loop, the FP32 form,
                # the phase-by-phase path, the 15360^2 deck, the dominant kernel
                "fused_bit_identical": fused_check["bit_identical"],
                "fp32_value": value32, "fp32_speedup": value32 / value,
                "fp32_density_l1": errs_resident["density0"]["l1_rel"],
                "host_loop_value": host_loop["value"],
                "large_value": large.get("value") if large else None,
                "roofline_frac": roof["frac"],
                "higher_is_better": True, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic: the reference benchmark deck generated in-process",
                "config": {"workload": f"clover_bm FP64 {S}x{S} hydro steps (InputDecks/clover_bm64_300.in physics)",
                           "cells": S * S, "l2": "no flush: every field array (472 MB) exceeds the 126 MB L2",
                           "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
                           "path": "cb_run: the timed steps as one device-resident CUDA graph, fused passes",
                           "halo": "folded into producers"},
                "roofline": roof, "fused_check": fused_check, "host_loop": host_loop, "fp32": fp32, "large": large, "batch": batch, "adjoint": adjoint, "resident_loop": resident, "reference_cuda": ref_cuda, "e2e": e2e, "gpu_launches": launches,
                "clocks": clocks, "cpu_baseline": cpu}
        print(json.dumps(line, default=_plain))
    if world > 1:
        torch.distributed.destroy_process_group()
    if not fused_check["bit_identical"]:
        raise SystemExit(f"bench.py: the fused graph's results differ from the phase-by-phase loop: {fused_check['mismatches']}")


if __name__ == "__main__":
    main()
