"""Run a clover.in deck (or the benchmark problem at any size) on a B200
through the C ABI, in the reference driver's call order, and print the
field summaries.

  python -m cloverleaf_b200.run --deck clover.in
  python -m cloverleaf_b200.run --bm 4608 --steps 2 [--precision fp32] [--no-fold] [--lagrangian |
                                                      --fuse-calls [--dt-ahead] | --resident [--fuse]]
  python -m cloverleaf_b200.run --ensemble 512 [--precision fp32] [--runs 3]
"""
from __future__ import annotations

import argparse
import sys
import time

from . import FP32, FP64, Chunk, HydroRun
from .deck import benchmark_deck, nudged, read_deck


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__, formatter_class=argparse.RawDescriptionHelpFormatter)
    g = ap.add_mutually_exclusive_group(required=True)
    g.add_argument("--deck", help="clover.in deck file")
    g.add_argument("--bm", type=int, help="benchmark problem on an N x N mesh")
    g.add_argument("--ensemble", type=int, help="the seeded batched ensemble of N decks, one persistent launch per run")
    ap.add_argument("--steps", type=int, default=None, help="stop after this many steps (default: the deck's end)")
    ap.add_argument("--precision", choices=["fp64", "fp32"], default="fp64")
    ap.add_argument("--no-fold", action="store_true", help="run every update_halo as its own pass")
    ap.add_argument("--resident", action="store_true", help="run the steps as one device-resident CUDA graph (cb_run)")
    ap.add_argument("--fuse", action="store_true", help="with --resident: fused passes (cb_run fuse = 1)")
    ap.add_argument("--lagrangian", action="store_true",
                    help="host loop with one cb_lagrangian call in place of PdV, accelerate, PdV and flux_calc")
    ap.add_argument("--fuse-calls", action="store_true",
                    help="host loop with the chunk's call fusion on (the fused passes, one launch each)")
    ap.add_argument("--dt-ahead", action="store_true",
                    help="with --fuse-calls: the Lagrangian pass run ahead from calc_dt (cb_set_dt_ahead)")
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--runs", type=int, default=1, help="ensemble runs after one warm-up run")
    ap.add_argument("--cells-per-cta", type=int, default=0, help="ensemble schedule: cells per CTA (0: the default schedule)")
    ap.add_argument("--variant", type=int, default=0, help="ensemble schedule: tile variant (with --cells-per-cta)")
    args = ap.parse_args(argv)
    if args.ensemble:
        return ensemble(args)

    dk = read_deck(args.deck) if args.deck else nudged(benchmark_deck(args.bm, end_step=args.steps or 87))
    c = Chunk(dk.x_cells, dk.y_cells, precision=FP32 if args.precision == "fp32" else FP64, device=args.device)
    run = HydroRun(c, dk, fold=not args.no_fold, lagrangian=args.lagrangian, fuse_calls=args.fuse_calls,
                   dt_ahead=args.fuse_calls and args.dt_ahead)
    t = time.time()
    if args.resident:
        run.start()
        run.run_steps_on_device(max_steps=args.steps, fuse=args.fuse)
    else:
        run.run(max_steps=args.steps)
    c.synchronize()
    wall = time.time() - t
    for s in run.summaries:
        print(f" step {s.step:6d} time {s.time:.6e} vol {s.vol:.15e} mass {s.mass:.15e} ie {s.ie:.15e} "
              f"ke {s.ke:.15e} press {s.press:.15e}")
    print(f" {run.step} steps of {dk.x_cells}x{dk.y_cells} in {wall:.3f} s "
          f"({dk.x_cells * dk.y_cells * run.step / wall:.4e} cell-steps/s incl. setup); {c.launch_count()} kernel launches")
    if dk.test_problem == 2 and run.step == 87:
        qa = abs(100.0 * (run.summaries[-1].ke / 1.19316898756307) - 100.0)
        print(f" Test problem 2 is within {qa}% of the expected solution: {'PASSED' if qa < 0.001 else 'NOT PASSED'}")
    c.close()
    return 0


def ensemble(args):
    from .batch import Batch, ensemble_decks
    decks = ensemble_decks(args.ensemble)
    b = Batch(decks, precision=FP32 if args.precision == "fp32" else FP64, device=args.device)
    if args.cells_per_cta > 0:
        b.set_schedule(cells_per_cta=args.cells_per_cta, variant=args.variant)
    sched, lanes, ctas = b.schedule()
    for k in range(args.runs + 1):
        b.run()
        ms = b.synchronize()
        res = [b.result(q) for q in range(len(decks))]
        cs = sum(d.x_cells * d.y_cells * r.steps for d, r in zip(decks, res))
        print(f" {'warm-up' if k == 0 else 'run'}: {len(decks)} decks, {cs} cell-steps in {ms:.2f} ms "
              f"({cs / ms * 1e3:.4e} cell-steps/s); {sum(r.status == 1 for r in res)} done; schedule {sched}, {lanes} lanes, "
              f"{ctas} CTAs")
    b.close()
    return 0


if __name__ == "__main__":
    sys.exit(main())
