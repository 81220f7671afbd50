#!/usr/bin/env python
"""Headline benchmark: MD throughput (atom-steps/s) of the force-and-integrate path.

Workload (the configuration the metric is quoted on): flexible 3-site water,
10,000 molecules (30,000 atoms) in a 6.69 nm cubic box, SPME 64^3 (order 4,
beta 3.12 nm^-1, cutoff 1.0 nm), Nose-Hoover NVT at 300 K, dt 0.5 fs; seeded
synthetic jittered-lattice start (no dataset).  Physically consistent profile
(gradient-consistent forces; the reference's own flexible-water forces are
unstable), mixed precision (FP32 pair / mesh / bonded arithmetic, int64
fixed-point forces, FP64 integration).  The all-FP64 GPU path is timed on the
same system for the mixed-vs-FP64 comparison, and both are checked against the
FP64 CPU oracle at the starting configuration.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Defaults: K = 2000 timed steps (long enough for ~30 clock samples), W = 20.
The CPU baseline (and the whole reference arm) is the reference's own C++ path
compiled by oracle/Makefile, one core, a bounded 10-step sample.

N > 1 runs one independent replica per GPU (one process per GPU, weak
scaling, no collective on the data path); the step time is the max over ranks.
One JSON line is printed by rank 0.
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

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L2_FLUSH_BYTES = 256 << 20          # > 126 MB L2: each timed step starts with a cold L2
MEASURED_PEAK_HBM_GBS = 6538.9      # fallback when MEASURED_PEAKS.json is absent: measured copy BW
SM_COUNT, FP32_LANES = 148, 128
# Algorithmic work of the pair kernel per atom and evaluation (water, rc 1.0 nm,
# 210 half-neighbours): tile-stream bytes and FLOPs (70 FLOP per LJ + erfc pair).
PAIR_BYTES_PER_ATOM = 650.0
PAIR_FLOP_PER_ATOM = 14690.0
# DRAM bytes (read + write) of one pair-kernel launch on this workload, from the
# ncu capture summarised in profiles/k_nb_f32_water30k.md (7.05 MB read, 0 written:
# the 30k-atom working set stays in the 126 MB L2 apart from the first touch).
PAIR_DRAM_BYTES = 7.05e6


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.f.name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def _peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d.get("hbm_gbs", MEASURED_PEAK_HBM_GBS)), "measured"
    return 6650.0, "fallback"


def workload(rank: int):
    from dmd_b200 import workloads
    return workloads.water_box(n_mol=10_000, box=6.69, seed=7 + rank, spacing=0.1045,
                               thermostat="nose-hoover", dt=0.0005)


def rel_rms(a, b):
    import numpy as np
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def run_ours(args):
    import numpy as np
    import torch
    ws, rank, local = _dist()
    torch.cuda.set_device(local)
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    from dmd_b200.core import Engine

    w = workload(rank)
    cfg = w.config()
    n_atoms = w.n_atoms
    dt = cfg.dt

    def barrier():
        if ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max_over_ranks(v: float) -> float:
        if ws == 1:
            return v
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64, device=f"cuda:{local}")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def timed(precision):
        eng = Engine(cfg, precision=precision, profile="phys", device=local)
        eng.run_n(args.warmup)
        eng.positions  # sync
        barrier()
        sampler = ClockSampler(local)
        sampler.start()
        t = eng.step_timed(args.steps, L2_FLUSH_BYTES)
        clocks = sampler.stop()
        barrier()
        step_ms = max_over_ranks(t["step_ms"])
        nb_ms = max_over_ranks(t["nonbonded_ms"] / max(t["nonbonded_launches"], 1))
        return eng, t, step_ms, nb_ms, clocks

    eng, t_mixed, step_ms, nb_ms, clocks = timed("mixed")
    value = ws * n_atoms * args.steps / (step_ms / 1e3)
    s = eng.scalars()
    _, t64, step_ms64, _, _ = timed("fp64")
    value64 = ws * n_atoms * args.steps / (step_ms64 / 1e3)

    # end to end through the public API: one run_n(1) call per MD step plus the
    # potential-energy read, host buffers, wall clock
    eng_e = Engine(cfg, precision="mixed", profile="phys", device=local)
    eng_e.run_n(args.warmup)
    _ = eng_e.potential_energy
    barrier()
    t0 = time.perf_counter()
    pe = 0.0
    for _ in range(args.steps):
        eng_e.run_n(1)
        pe = eng_e.potential_energy
    e2e_s = max_over_ranks(time.perf_counter() - t0)
    e2e_value = ws * n_atoms * args.steps / e2e_s

    out = None
    if rank == 0:
        # accuracy at the starting configuration against the FP64 CPU oracle
        from oracle.oracle import Oracle
        F_o, e_o = Oracle().forces(cfg, "phys")
        acc = {}
        for prec in ("mixed", "fp64"):
            e0 = Engine(cfg, precision=prec, profile="phys", device=local)
            F, e = e0.compute_forces()
            acc[prec] = {"rel_rms_force_err": rel_rms(F, F_o),
                         "rel_energy_err": abs(sum(e.values()) - e_o["total"]) / abs(e_o["total"])}
            e0.close()
        # CPU baseline: the reference algorithm (REF profile, O(N^2) list every 5
        # steps, FP64) on one host core, bounded sample
        cpu = None
        if not args.skip_cpu and ws == 1:
            cpu = cpu_reference(cfg, n_atoms, args.cpu_steps)
        hbm_peak, peak_kind = _peaks()
        t_nb = nb_ms / 1e3
        b_alg = PAIR_BYTES_PER_ATOM * n_atoms
        f_alg = PAIR_FLOP_PER_ATOM * n_atoms
        f_sm = (clocks.get("sm_mhz") or 1965.0) * 1e6
        p32 = SM_COUNT * FP32_LANES * 2 * f_sm / 1e12
        achieved = b_alg / t_nb / 1e9
        tflops = f_alg / t_nb / 1e12
        roof = {
            "kernel": "k_nb_f32 (LJ + real-space Ewald pair kernel)",
            "bound": "hbm", "achieved": round(achieved, 2), "peak": hbm_peak, "unit": "GB/s",
            "frac": round(achieved / hbm_peak, 4),
            "traffic": PAIR_DRAM_BYTES,
            "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
            "launch_ms": round(nb_ms, 5),
            "launch_note": "average over the timed steps, measured while the bonded + PME chain "
                           "runs beside it on a second stream",
            "algorithmic_bytes_per_launch": b_alg, "algorithmic_flop_per_launch": f_alg,
            "fp32": {"achieved_tflops": round(tflops, 3), "peak_tflops": round(p32, 2),
                     "frac": round(tflops / p32, 4),
                     "peak_note": "148 SMs x 128 FP32 lanes x 2 x median SM clock of the run"},
            "binding_roof": "fp32 (arithmetic intensity 22.6 FLOP/B > ridge)",
        }
        out = {
            "metric": "atom-steps/s", "value": round(value, 1), "unit": "atom-steps/s",
            "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": round(step_ms / args.steps, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "precision": "mixed: FP32 pair/mesh/bonded math, int64 fixed-point forces, FP64 integration",
            "data": "synthetic (seeded jittered-lattice water, random orientations)",
            "config": {"workload": "water_30k_nvt_pme64", "n_atoms": n_atoms, "box_nm": cfg.box_size,
                       "pme_mesh": 64, "cutoff_nm": 1.0, "skin_nm": 0.1, "dt_ps": dt,
                       "thermostat": "nose-hoover 300 K", "profile": "phys",
                       "l2": "flushed between timed steps (256 MiB overwrite outside the step events)",
                       "parallelism": f"replicas x{ws} (one independent system per GPU)"},
            "ns_per_day": round(dt * 1e-3 * args.steps / (step_ms / 1e3) * 86400, 2),
            "fp64_path": {"value": round(value64, 1), "ms_per_step": round(step_ms64 / args.steps, 5),
                          "mixed_over_fp64": round(value / value64, 3)},
            "accuracy_vs_fp64_cpu_oracle": acc,
            "e2e": {"value": round(e2e_value, 1), "unit": "atom-steps/s",
                    "h2d_bytes_per_step": 8, "d2h_bytes_per_step": 8 + 2 * 232,
                    "how": "Engine.run_n(1) + Engine.potential_energy per MD step (C ABI, host "
                           "buffers, host wall clock); inputs are the step target, result the "
                           "energy scalars"},
            "roofline": roof,
            "cpu_baseline": cpu,
            "gpu_launches": int(t_mixed["kernel_launches"]),
            "clocks": clocks,
            "list_builds": int(s.list_builds),
        }
    if ws > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    return out


def cpu_reference(cfg, n_atoms, steps):
    """The reference's CPU path on one host core (the reference has no threading
    on this path), timed on a bounded sample from the start of the run.

    Preferred: the reference's own C++ (src/ compiled unmodified by oracle/Makefile;
    CoulombPME against the FFTW-API shim, since FFTW3 is not installed), stepped
    in SimulationEngine::step order: its O(N^2) LennardJones list rebuilt every
    10 force evaluations, two evaluations per step, FP64.  If that build is not
    present, the oracle's restatement of the same algorithm (REF profile)."""
    from oracle.oracle import Oracle, Ref, ref_available
    if ref_available():
        eng, kind = Ref().engine(cfg), "reference"
        what = "reference C++ (src/, unmodified; PME via the FFTW-API shim)"
    else:
        eng, kind = Oracle().engine(cfg, "ref", brute_list=True), "port"
        what = "oracle restatement of the reference algorithm (REF profile)"
    t0 = time.perf_counter()
    eng.step(steps)
    dt = time.perf_counter() - t0
    return {"value": round(n_atoms * steps / dt, 1), "unit": "atom-steps/s", "cores": 1,
            "kind": kind,
            "sample": f"{steps} MD steps of the same 30,000-atom water box from the start "
                      f"({what}; includes {(steps + 4) // 5} O(N^2) list rebuilds), {dt:.1f} s"}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return None
    w = workload(0)
    cfg = w.config()
    steps = min(args.steps, args.cpu_steps)
    cpu = cpu_reference(cfg, w.n_atoms, steps)
    v = cpu["value"]
    return {"impl": "reference", "metric": "atom-steps/s", "value": v, "unit": "atom-steps/s",
            "n_gpus": ws, "steps": steps, "warmup": 0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "water_30k_nvt_pme64", "n_atoms": w.n_atoms, "profile": "ref",
                       "implementation": cpu["sample"].split("(")[1].split(";")[0],
                       "sample_steps": steps},
            "cpu_baseline": cpu,
            "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--skip-cpu", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
