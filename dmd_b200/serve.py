"""Served MD job stream: continuous batching of jobs over one device batch.

Jobs arrive (Poisson arrivals at a stated rate, or at given times), wait in a
FIFO queue, and are admitted into the running ``Batch`` as soon as the HBM
budget allows — also while other jobs are mid-run.  The loop advances every
running job by ``chunk`` steps per device call, collects the jobs that reached
their step count, releases their memory and admits more.  State stays on the
device from admission to completion.

Reported: per-step latency (device call time / steps advanced) and job
completion latency (completion - arrival), p50 and p99, and aggregate
atom-steps/s over the whole stream.

    python -m dmd_b200.serve --jobs 24 --rate 2.0 --precision mixed

The job mix is the served-stream configuration: 70% LJ argon with N
log-uniform in [1k, 50k], 30% flexible 3-site water with N in [3k, 96k]
(multiples of 3) and PME mesh spacing <= 0.11 nm, steps uniform in
[1000, 20000], one seed per job (``--scale`` shrinks N and steps for tests).
"""
from __future__ import annotations

import argparse
import dataclasses
import json
import math
import time

import numpy as np

from . import workloads as W
from .batch import Batch, BudgetExceeded


@dataclasses.dataclass
class Job:
    jid: int
    cfg: object
    n_steps: int
    arrival: float                 # seconds after the start (or steps in virtual time)
    n_atoms: int = 0
    slot: int = -1
    admitted: float = math.nan
    done: float = math.nan
    result: dict = dataclasses.field(default_factory=dict)
    steps_done: int = 0
    packed: bool = False           # in the device table (admitted before the last device call)
    repacks: list = dataclasses.field(default_factory=list)  # own step counts at table rebuilds


def job_mix(n_jobs: int, rate: float, seed: int = 2025, scale: float = 1.0):
    """Seeded served-stream jobs with Poisson arrival times (rate jobs/s)."""
    rng = np.random.default_rng(seed)
    t = 0.0
    jobs = []
    for k in range(n_jobs):
        t += rng.exponential(1.0 / rate) if rate > 0 else 0.0
        steps = max(10, int(rng.integers(1000, 20001) * scale))
        if rng.uniform() < 0.7:
            n = int(round(math.exp(rng.uniform(math.log(1000), math.log(50000))) * scale))
            n = max(64, n)
            w = W.lj_fluid(n, float(rng.uniform(0.60, 0.85)), float(rng.uniform(0.8, 1.5)), seed + k)
        else:
            n_mol = max(100, int(rng.integers(1000, 32001) * scale))
            box = (n_mol / 33.43) ** (1 / 3)
            K = max(8, math.ceil(box / 0.11))
            w = W.water_box(n_mol=n_mol, box=box, seed=seed + k, spacing=box / K)
        cfg = w.config()
        jobs.append(Job(k, cfg, steps, t, n_atoms=len(cfg.masses)))
    return jobs


def _pcts(v):
    if not v:
        return None
    return {"p50": 1e3 * float(np.percentile(v, 50)), "p99": 1e3 * float(np.percentile(v, 99)), "calls": len(v)}


def serve(jobs, budget_bytes=150 * 10**9, precision="mixed", profile="phys", chunk=100,
          virtual=False):
    """Run the job stream through one continuously batched device batch.

    virtual=True measures arrivals in executed steps instead of seconds (a
    deterministic schedule, for tests)."""
    b = Batch(budget_bytes=budget_bytes, precision=precision, profile=profile)
    queue = sorted(jobs, key=lambda j: j.arrival)
    running: dict[int, Job] = {}
    step_lat = []              # seconds per step of each device call
    rebuilt = []               # whether that call rebuilt the device table first
    configs: dict = {}         # launch configurations the rebuilt tables ran with -> calls
    t0 = time.perf_counter()
    clock_steps = 0
    atom_steps = 0
    dirty = False              # a slot was admitted or released since the last device call

    def now():
        return float(clock_steps) if virtual else time.perf_counter() - t0

    while queue or running:
        # admit arrived jobs in FIFO order while the budget allows
        while queue and queue[0].arrival <= now():
            j = queue[0]
            try:
                j.slot = b.admit(j.cfg, j.n_steps)
            except BudgetExceeded:
                if not running:
                    raise
                break
            j.admitted = now()
            running[j.slot] = j
            queue.pop(0)
            dirty = True
        if not running:
            if virtual:
                clock_steps = int(math.ceil(queue[0].arrival))
            else:
                time.sleep(max(0.0, queue[0].arrival - now()))
            continue
        live = sum(j.n_atoms for j in running.values())
        rebuilt.append(dirty)
        if dirty:
            # the device table is rebuilt at this call: running jobs carry their
            # state over and rebuild their pair lists (Engine.repack alone)
            for j in running.values():
                if j.packed:
                    j.repacks.append(j.steps_done)
            dirty = False
        t = time.perf_counter()
        b.step(chunk)
        dt = time.perf_counter() - t
        if rebuilt[-1]:
            li = b.launch_info()
            key = (li["nb_form"], li["nb_blocks_per_sm"], li["tuned"], li["min_image_kernel"])
            configs[key] = configs.get(key, 0) + 1
        step_lat.append(dt / chunk)
        clock_steps += chunk
        atom_steps += live * chunk
        for j in running.values():
            j.packed = True
            j.steps_done = min(j.n_steps, j.steps_done + chunk)
        for slot in b.poll():
            j = running.pop(slot)
            j.done = now()
            s = b.scalars(slot)
            j.result = {"positions": b.positions(slot), "velocities": b.velocities(slot),
                        "potential_energy": s.potential_energy, "step": int(s.step)}
            b.release(slot)
            dirty = True
    wall = time.perf_counter() - t0
    done = [j.done - j.arrival for j in jobs]
    done_steps = sum(j.n_atoms * j.n_steps for j in jobs)
    return {
        "jobs": len(jobs),
        "atom_steps_per_s": done_steps / wall if not virtual else None,
        "wall_s": wall,
        "step_latency_ms": {"p50": 1e3 * float(np.percentile(step_lat, 50)),
                            "p99": 1e3 * float(np.percentile(step_lat, 99))},
        # the same split by calls that rebuilt the table first (an admission or
        # release) and calls that did not: the spread of the steady calls is
        # the job mix (how many atoms run at once), the difference between the
        # two the cost of the rebuilds
        "step_latency_ms_steady": _pcts([t for t, r in zip(step_lat, rebuilt) if not r]),
        "step_latency_ms_rebuild": _pcts([t for t, r in zip(step_lat, rebuilt) if r]),
        "job_latency": {"p50": float(np.percentile(done, 50)), "p99": float(np.percentile(done, 99)),
                        "unit": "steps" if virtual else "s"},
        "launch_configs": [{"nb_form": k[0], "nb_blocks_per_sm": k[1], "tuned": k[2],
                            "min_image_kernel": k[3], "tables": v} for k, v in sorted(configs.items())],
        "work_atom_steps": done_steps,
        "padded_atom_steps": atom_steps,
    }


def run_alone(job: Job, precision="mixed", profile="phys", device=None):
    """The same job in an engine of its own: positions, velocities, potential
    energy.  Fixed-point force sums, per-replica reductions and pair lists
    rebuilt in their own frame at table rebuilds make this equal to the job's
    result in the mix, bit for bit."""
    from .core import Engine
    e = Engine(job.cfg, precision=precision, profile=profile, device=device)
    e.run_n(job.n_steps)
    out = e.positions, e.velocities, e.potential_energy
    e.close()
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=24)
    ap.add_argument("--rate", type=float, default=2.0, help="Poisson arrival rate (jobs/s)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--budget-gb", type=float, default=150.0)
    ap.add_argument("--chunk", type=int, default=100)
    ap.add_argument("--scale", type=float, default=1.0)
    ap.add_argument("--seed", type=int, default=2025)
    args = ap.parse_args()
    jobs = job_mix(args.jobs, args.rate, args.seed, args.scale)
    out = serve(jobs, int(args.budget_gb * 1e9), args.precision, "phys", args.chunk)
    out.update({"rate_jobs_per_s": args.rate, "precision": args.precision,
                "budget_gb": args.budget_gb, "chunk": args.chunk, "scale": args.scale})
    print(json.dumps(out))


if __name__ == "__main__":
    main()
