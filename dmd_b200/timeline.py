"""Per-kernel device timeline of a few MD steps (CUPTI through torch.profiler).

Shows what runs where inside the step graph: start and end of every kernel of
a step relative to the step's first kernel, so overlap between the main stream
(list rebuild, pair kernel) and the bonded/PME stream is visible, plus the
mean step period and per-kernel totals.

    python -m dmd_b200.timeline [--steps 30] [--precision mixed] [--show 3]
                                [--workload water30k|water750k|argon4k|batch256]

Runs on the headline workload (water 30k NVT, PHYS profile) by default.  A
diagnostic: numbers printed under a profiler are not benchmark values.
"""
from __future__ import annotations

import argparse
import os
import sys


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--show", type=int, default=3, help="steps printed kernel by kernel")
    ap.add_argument("--workload", default="water30k",
                    choices=["water30k", "water750k", "argon4k", "batch256"])
    ap.add_argument("--plain", action="store_true",
                    help="run the steps without the profiler (a target for ncu)")
    ap.add_argument("--timed", action="store_true",
                    help="profile the timed path (step_timed: events around every step, pair "
                         "kernel and PME chain, L2 flushed between steps) instead of run_n")
    ap.add_argument("--flush-mb", type=int, default=512, help="L2 flush buffer of --timed")
    args = ap.parse_args()
    import torch
    from torch.profiler import ProfilerActivity, profile

    sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    from dmd_b200.core import Engine
    from dmd_b200 import workloads as W

    if args.workload == "batch256":
        from dmd_b200.batch import Batch
        eng = Batch(precision=args.precision, profile="phys")
        for w in W.batch_256():
            eng.admit(w.config(), args.warmup + args.steps)
        eng.step(args.warmup)
        if args.plain:
            eng.step(args.steps)
            return
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            eng.step(args.steps)
    else:
        if args.workload == "water30k":
            w = W.water_box(n_mol=10_000, box=6.69, seed=7, spacing=0.1045, thermostat="nose-hoover",
                            dt=0.0005)
        elif args.workload == "water750k":
            w = W.water_box(n_mol=250_000, box=19.56, seed=7, spacing=0.1019, thermostat="berendsen",
                            barostat="berendsen", dt=0.0005)
        else:
            w = W.argon_fcc(n_cells=10, a=0.575, T=120.0, seed=2024, dt=0.002)
        eng = Engine(w.config(), precision=args.precision, profile="phys")
        eng.run_n(args.warmup)
        eng.positions
        if args.plain:
            eng.run_n(args.steps)
            eng.positions
            return
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            if args.timed:
                eng.step_timed(args.steps, args.flush_mb << 20)
            else:
                eng.run_n(args.steps)
            eng.positions
    ev = [e for e in prof.events() if e.device_type.name == "CUDA" and "Memcpy" not in e.name
          and "Memset" not in e.name]
    ev.sort(key=lambda e: e.time_range.start)

    def short(name):
        return name.replace("void ", "").replace("dmd::(anonymous namespace)::", "").replace("dmd::", "")[:44]

    starts = [e.time_range.start for e in ev if "k_kick_drift" in e.name]
    if len(starts) > 1:
        print(f"steps {len(starts)}  mean step period {(starts[-1] - starts[0]) / (len(starts) - 1):.1f} us")
    for si in range(min(args.show, max(len(starts) - 1, 0))):
        t0, t1 = starts[si], starts[si + 1]
        print(f"--- step {si}: {t1 - t0:.1f} us")
        for e in ev:
            if t0 <= e.time_range.start < t1:
                print(f"{short(e.name):44s} start {e.time_range.start - t0:7.1f}  end "
                      f"{e.time_range.end - t0:7.1f}  dur {e.time_range.end - e.time_range.start:6.1f}")
    agg = {}
    for e in ev:
        a = agg.setdefault(short(e.name), [0, 0.0])
        a[0] += 1
        a[1] += e.time_range.end - e.time_range.start
    print(f"--- totals over {args.steps} steps")
    for k, (n, t) in sorted(agg.items(), key=lambda x: -x[1][1]):
        print(f"{k:44s} {n:6d} launches {t:10.1f} us  {t / n:7.2f} us avg")


if __name__ == "__main__":
    main()
