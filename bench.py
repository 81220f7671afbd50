#!/usr/bin/env python
"""MD throughput (atom-steps/s) of the force-and-integrate path on one B200.

Default workload (the configuration the headline metric is quoted on):
flexible 3-site water, 10,000 molecules (30,000 atoms) in a 6.69 nm cubic box,
SPME 64^3 (order 4, beta 3.12 nm^-1, cutoff 1.0 nm), Nose-Hoover NVT at 300 K,
dt 0.5 fs; seeded synthetic jittered-lattice start (no dataset).  Physically
consistent profile (gradient-consistent forces; the reference's own
flexible-water forces are unstable), mixed precision (FP32 pair / mesh /
bonded arithmetic, int64 fixed-point forces, FP64 integration).  The all-FP64
GPU path is timed on the same system for the mixed-vs-FP64 comparison, and
both are checked against the FP64 CPU oracle at the starting configuration.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload water30k|argon4k|water750k|batch256|serve]

Other workloads (same JSON line, their own config):
  argon4k    LJ argon NVE, 4,000 atoms (10x10x10 FCC, 5.75 nm box), dt 2 fs
  water750k  the water model at 250,000 molecules (19.56 nm box), SPME 192^3,
             Berendsen thermostat + Berendsen barostat (NPT), dt 0.5 fs
  batch256   256 independent replicas in one device batch (192 LJ fluids of
             500-20,000 atoms, 64 united-atom decane melts of 50-400 chains),
             against the FP64 batch and the same replicas run one per launch
  serve      a Poisson stream of MD jobs (70% LJ argon 1k-50k atoms, 30% water
             with SPME 3k-96k atoms, 1,000-20,000 steps each) continuously
             batched under a 150 GB HBM budget; p50/p99 step and job latency

The CPU baseline (and the whole reference arm) is the reference's own C++ path
compiled by oracle/Makefile, one core, a bounded sample.

N > 1 runs one independent replica per GPU (one process per GPU, weak
scaling, no collective on the data path); the step time is the max over ranks.
One JSON line is printed by rank 0.
"""
from __future__ import annotations

import argparse
import json
import math
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
WORKLOADS = ("water30k", "argon4k", "water750k", "batch256", "serve")
CPU_MAX_ATOMS = 100_000             # above this the reference's O(N^2) list build takes hours

# Algorithmic work of the pair kernel per atom and evaluation, as a tile-streaming
# pair kernel must do it: bytes = (half j-tiles per i-tile) x (32 x 16 B j payload
# + 8 B list entry) / 32 + 40 B (own float4 read + three int64 force writes);
# FLOPs = half-pairs within the cutoff x 38 (LJ) or 70 (LJ + erfc Ewald).
# Water (rc 1.0 nm, 100.2 atoms/nm^3, 210 half-neighbours): 650 B, 14,690 FLOP.
# Argon (rc 1.0 nm, 21.0 atoms/nm^3, 44 half-neighbours): 241 B, 1,675 FLOP.
PAIR_WORK = {"water": (650.0, 14690.0), "argon": (241.0, 1675.0)}
# DRAM bytes (read + write) of one pair-kernel launch, from the ncu captures in
# profiles/ (water 30k: 7.62 MB read, 0 written -- the working set stays in L2;
# water 750k: 190.0 + 13.9 MB; the 256-replica batch: 217.3 + 34.0 MB).
PAIR_DRAM_BYTES = {"water30k": 7.62e6, "water750k": 203.9e6, "batch256": 251.3e6}


def lj_pair_work(n: int, box: float, rc: float, flop_per_pair: float = 38.0):
    """Per-atom algorithmic (bytes, FLOP) of the pair kernel for a homogeneous
    system of n atoms in a cubic box (the same model as PAIR_WORK): half j-tiles
    per i-tile = atoms within rc + one tile edge of a tile, halved, / 32."""
    rho = n / box ** 3
    edge = (32.0 / rho) ** (1.0 / 3.0)
    vol = 4.0 / 3.0 * math.pi
    tiles = min(0.5 * rho * vol * (rc + edge) ** 3, n) / 32.0
    half_pairs = min(0.5 * rho * vol * rc ** 3, 0.5 * n)
    return tiles * (32 * 16 + 8) / 32.0 + 40.0, half_pairs * flop_per_pair


def _dist():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 50 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def _lines(self) -> int:
        try:
            with open(self.f.name) as fh:
                return sum(1 for _ in fh)
        except OSError:
            return 0

    def start(self):
        """Start sampling and return once the first sample is written (nvidia-smi
        takes a moment to start, longer than a short timed region)."""
        try:
            self.p = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "50"],
                stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None
            return
        t0 = time.time()
        while self._lines() < 1 and time.time() - t0 < 5.0 and self.p.poll() is None:
            time.sleep(0.02)
        self.n0 = self._lines()

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        # at least one sample taken after the timed region started
        t0 = time.time()
        while self._lines() < getattr(self, "n0", 0) + 2 and time.time() - t0 < 1.0:
            time.sleep(0.02)
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        lines = self.f.readlines()
        skip = max(getattr(self, "n0", 0) - 1, 0)  # samples taken before the timed region
        for line in lines[skip:] if len(lines) > skip else lines:
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


# ---------------------------------------------------------------------------
# workloads

def water30k(rank: int):
    from dmd_b200 import workloads
    return workloads.water_box(n_mol=10_000, box=6.69, seed=7 + rank, spacing=0.1045,
                               thermostat="nose-hoover", dt=0.0005)


def argon4k(rank: int):
    from dmd_b200 import workloads
    return workloads.argon_fcc(n_cells=10, a=0.575, T=120.0, seed=2024 + rank, dt=0.002)


def water750k(rank: int):
    from dmd_b200 import workloads
    return workloads.water_box(n_mol=250_000, box=19.56, seed=7 + rank, spacing=0.1019,
                               thermostat="berendsen", barostat="berendsen", dt=0.0005)


SINGLE = {
    "water30k": dict(make=water30k, kind="water", pme=64, ensemble="nose-hoover NVT 300 K",
                     desc="seeded jittered-lattice water, random orientations"),
    "argon4k": dict(make=argon4k, kind="argon", pme=None, ensemble="NVE (velocities at 120 K)",
                    desc="FCC argon lattice, Maxwell-Boltzmann velocities from a seed",
                    skin=0.1),  # the configuration states a 0.1 nm skin
    "water750k": dict(make=water750k, kind="water", pme=192,
                      ensemble="Berendsen T 300 K + Berendsen P 1 bar (NPT)",
                      desc="seeded jittered-lattice water, random orientations"),
}


def rel_rms(a, b):
    import numpy as np
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


class Ranks:
    """Process-group plumbing: barrier and max over ranks (no-ops at N = 1).

    One process per GPU over NCCL; without a GPU (host-side tests) the same
    calls run over gloo with CPU tensors.
    """

    def __init__(self, local: int):
        import torch
        self.ws, self.rank, self.local = _dist()
        self.cuda = torch.cuda.is_available()
        if self.cuda:
            torch.cuda.set_device(local)
        if self.ws > 1:
            import datetime
            import torch.distributed as dist
            dist.init_process_group("nccl" if self.cuda else "gloo",
                                    timeout=datetime.timedelta(seconds=120))

    def barrier(self):
        if self.ws > 1:
            import torch.distributed as dist
            dist.barrier()

    def max(self, v: float) -> float:
        if self.ws == 1:
            return v
        import torch
        import torch.distributed as dist
        t = torch.tensor([v], dtype=torch.float64,
                         device=f"cuda:{self.local}" if self.cuda else "cpu")
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.ws > 1:
            import torch.distributed as dist
            dist.barrier()
            dist.destroy_process_group()


def roofline(kind_bytes: float, kind_flop: float, nb_ms: float, clocks: dict, traffic,
             kernel: str, fp32_binding: bool, launch_note: str) -> dict:
    """The pair kernel against its binding roof (top-level fields) with the other
    roof as a sub-field.  FP32 binds where the arithmetic intensity of the
    algorithmic work is above the ridge (water: LJ + Ewald), HBM below it (LJ)."""
    hbm_peak, peak_kind = _peaks()
    t_nb = nb_ms / 1e3
    gbs = kind_bytes / t_nb / 1e9
    tflops = kind_flop / t_nb / 1e12
    f_mhz = clocks.get("sm_mhz")
    f_sm = (f_mhz or 1965.0) * 1e6
    p32 = SM_COUNT * FP32_LANES * 2 * f_sm / 1e12
    hbm = {"bound": "hbm", "achieved": round(gbs, 2), "peak": hbm_peak, "unit": "GB/s",
           "frac": round(gbs / hbm_peak, 4),
           "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"}
    fp32 = {"bound": "fp32", "achieved": round(tflops, 3), "peak": round(p32, 2), "unit": "TFLOP/s",
            "frac": round(tflops / p32, 4),
            "peak_source": "148 SMs x 128 FP32 lanes x 2 FLOP x " +
                           (f"the run's median SM clock ({f_mhz:.0f} MHz)" if f_mhz else
                            "1,965 MHz (clocks.max.sm; no clock sample in the timed region)")}
    top, other = (fp32, hbm) if fp32_binding else (hbm, fp32)
    out = {"kernel": kernel}
    out.update(top)
    out.update({
        "traffic": traffic,
        "launch_ms": round(nb_ms, 5),
        "launch_note": launch_note,
        "algorithmic_bytes_per_launch": kind_bytes, "algorithmic_flop_per_launch": kind_flop,
        "binding_roof": ("fp32 (arithmetic intensity above the ridge)" if fp32_binding
                         else "hbm (arithmetic intensity below the ridge)"),
        "other_roof": other,
    })
    return out


def run_single(args, R: Ranks):
    """One system per GPU: water30k, argon4k or water750k."""
    from dmd_b200.core import Engine, default_skin
    spec = SINGLE[args.workload]
    w = spec["make"](R.rank)
    cfg = w.config()
    n_atoms = w.n_atoms
    dt = cfg.dt

    skin = spec.get("skin")  # None: the library's default

    def timed(precision):
        eng = Engine(cfg, precision=precision, profile="phys", device=R.local, skin=skin)
        eng.run_n(args.warmup)
        eng.positions  # sync
        R.barrier()
        sampler = ClockSampler(R.local)
        sampler.start()
        t = eng.step_timed(args.steps, L2_FLUSH_BYTES)
        clocks = sampler.stop()
        R.barrier()
        step_ms = R.max(t["step_ms"])
        nb_ms = R.max(t["nonbonded_ms"] / max(t["nonbonded_launches"], 1))
        return eng, t, step_ms, nb_ms, clocks

    eng, t_mixed, step_ms, nb_ms, clocks = timed("mixed")
    value = R.ws * n_atoms * args.steps / (step_ms / 1e3)
    launch = eng.launch_info()
    s = eng.scalars()
    evals_per_step = t_mixed["nonbonded_launches"] / max(t_mixed["sampled_steps"], 1)
    # accuracy is checked at the starting configuration, except on a perfect
    # lattice (argon FCC: every force vanishes by symmetry), where it is checked
    # at the configuration the timed run reached
    acc_pos = eng.positions if spec["kind"] == "argon" else None
    eng.close()
    _, t64, step_ms64, _, _ = timed("fp64")
    value64 = R.ws * n_atoms * args.steps / (step_ms64 / 1e3)

    # end to end through the public API: one run_n(1) call per MD step plus the
    # potential-energy read, host buffers, wall clock
    eng_e = Engine(cfg, precision="mixed", profile="phys", device=R.local, skin=skin)
    eng_e.run_n(args.warmup)
    _ = eng_e.potential_energy
    R.barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        eng_e.run_n(1)
        _ = eng_e.potential_energy
    e2e_s = R.max(time.perf_counter() - t0)
    e2e_value = R.ws * n_atoms * args.steps / e2e_s
    eng_e.close()

    if R.rank != 0:
        return None
    drift = nve_drift(cfg, R.local, args.drift_steps, skin) if spec["kind"] == "argon" else None
    # accuracy at the starting configuration against the FP64 CPU oracle
    from oracle.oracle import Oracle
    F_o, e_o = Oracle().forces(cfg, "phys", pos=acc_pos)
    acc = {"configuration": "start" if acc_pos is None else
           f"after the {args.warmup + args.steps}-step timed run"}
    for prec in ("mixed", "fp64"):
        e0 = Engine(cfg, precision=prec, profile="phys", device=R.local, skin=skin)
        if acc_pos is not None:
            e0.set_positions(acc_pos)
        F, e = e0.compute_forces()
        acc[prec] = {"rel_rms_force_err": rel_rms(F, F_o),
                     "rel_energy_err": abs(sum(e.values()) - e_o["total"]) / abs(e_o["total"])}
        e0.close()
    cpu = None
    if not args.skip_cpu and R.ws == 1 and n_atoms > CPU_MAX_ATOMS:
        cpu = cpu_reference_extrapolated(n_atoms, water30k(0).config(), args.cpu_steps)
    elif not args.skip_cpu and R.ws == 1:
        cpu = cpu_reference([cfg], args.cpu_steps, f"the same {n_atoms:,}-atom system")
    b_atom, f_atom = PAIR_WORK[spec["kind"]]
    roof = roofline(b_atom * n_atoms, f_atom * n_atoms, nb_ms, clocks,
                    PAIR_DRAM_BYTES.get(args.workload),
                    "k_nb_f32 (LJ + real-space Ewald pair kernel)" if spec["kind"] == "water"
                    else "k_nb_f32 (LJ pair kernel)",
                    spec["kind"] == "water",
                    "average over the timed steps" + (
                        ", measured while the bonded + PME chain runs beside it on a second stream"
                        if spec["pme"] else ""))
    config = {"workload": f"{args.workload}", "n_atoms": n_atoms, "box_nm": cfg.box_size,
              "cutoff_nm": cfg.lj_cutoff, "skin_nm": skin if skin is not None else default_skin(),
              "dt_ps": dt,
              "ensemble": spec["ensemble"], "profile": "phys",
              "force_evaluations_per_step": round(evals_per_step, 3),
              "l2": "flushed between timed steps (256 MiB overwrite outside the step events)",
              "parallelism": f"replicas x{R.ws} (one independent system per GPU)"}
    if spec["pme"]:
        config.update({"pme_mesh": spec["pme"], "pme_order": 4, "ewald_beta": 3.12})
    return {
        "metric": "atom-steps/s", "value": round(value, 1), "unit": "atom-steps/s",
        "n_gpus": R.ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(step_ms / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "precision": "mixed: FP32 pair/mesh/bonded math, int64 fixed-point forces, FP64 integration",
        "data": f"synthetic ({spec['desc']})",
        "config": config,
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
        "launch": launch,
        "clocks": clocks,
        "list_builds": int(s.list_builds),
        "energies_in_timed_steps": "the device-timed value evaluates the energies and the virial "
                                   "only on the last timed step (the ensemble needs none inside a "
                                   "step); e2e reads them after every step",
        **({"nve_drift": drift} if drift else {}),
    }


def nve_drift(cfg, device: int, steps: int, skin=None) -> dict:
    """NVE energy drift max_t |E(t) - E(0)| / |E(0)| over `steps` steps
    (tests/integration/test_argon_nve.cpp:150-171 of the reference), E = the
    potential energy plus sum(m v^2)/2 read after every step: the GPU paths
    (one run_n(1) per step through the C ABI) and the reference's own engine
    (src/ compiled unmodified, REF profile) on the same inputs."""
    import numpy as np
    from dmd_b200.core import Engine
    from oracle.oracle import Ref, ref_available
    m = np.asarray(cfg.masses)

    def run(step, vel, pe):
        e = []
        for _ in range(steps):
            step()
            v = vel()
            e.append(0.5 * float(np.sum(m[:, None] * v * v)) + pe())
        e = np.asarray(e)
        return float(np.max(np.abs(e - e[0])) / abs(e[0]))

    out = {"steps": steps, "dt_ps": cfg.dt,
           "metric": "max over steps of |E(t) - E(t1)| / |E(t1)|, E = potential + kinetic read "
                     "after every step, t1 the first step (both engines evaluate their initial "
                     "forces inside it); the criterion of the reference's "
                     "tests/integration/test_argon_nve.cpp"}
    for prec, prof in (("mixed", "phys"), ("fp64", "phys"), ("mixed", "ref")):
        eng = Engine(cfg, precision=prec, profile=prof, device=device, skin=skin)
        out[f"gpu_{prec}_{prof}"] = run(lambda: eng.run_n(1), lambda: eng.velocities,
                                        lambda: eng.potential_energy)
        eng.close()
    if ref_available():
        re_ = Ref().engine(cfg)
        t0 = time.perf_counter()
        out["reference_cpu_ref"] = run(lambda: re_.step(1), lambda: re_.get(1),
                                       lambda: re_.scalars()["pe"])
        out["reference_seconds"] = round(time.perf_counter() - t0, 1)
    else:
        out["reference_cpu_ref"] = None
    return out


# CPU sample of the batch: 8 replicas in the batch's 3:1 LJ : decane proportion,
# one per host core at once
BATCH_CPU_SAMPLE = (0, 1, 2, 3, 4, 5, 192, 193)
BATCH_CPU_WHAT = "replicas 0-5 (LJ fluids) and 192-193 (decane melts) of the 256-replica batch"


def run_batch(args, R: Ranks):
    """256 independent replicas advanced together in one device batch."""
    from dmd_b200 import workloads as W
    from dmd_b200.batch import Batch
    from dmd_b200.core import Engine
    ws_ = W.batch_256(seed=1234 + 1000 * R.rank)
    cfgs = [w.config() for w in ws_]
    n_atoms = sum(w.n_atoms for w in ws_)
    target = args.warmup + args.steps + 1

    def timed(precision):
        b = Batch(precision=precision, profile="phys", device=R.local)
        slots = [b.admit(c, target) for c in cfgs]
        b.step(args.warmup)
        R.barrier()
        sampler = ClockSampler(R.local)
        sampler.start()
        t = b.step_timed(args.steps, L2_FLUSH_BYTES)
        clocks = sampler.stop()
        R.barrier()
        return b, slots, t, clocks

    b, slots, t_mixed, clocks = timed("mixed")
    launch = b.launch_info()
    step_ms = R.max(t_mixed["step_ms"])
    nb_ms = R.max(t_mixed["nonbonded_ms"] / max(t_mixed["nonbonded_launches"], 1))
    value = R.ws * n_atoms * args.steps / (step_ms / 1e3)
    list_builds = sum(int(b.scalars(s).list_builds) for s in slots)
    used = b.used_bytes

    # end to end through the public API: Batch.step(1) per MD step (each call
    # returns after the device finished and the per-replica status records were
    # read back), then every replica's potential energy
    n_e2e = min(args.steps, 50)
    b_e = Batch(precision="mixed", profile="phys", device=R.local)
    for c in cfgs:
        b_e.admit(c, args.warmup + n_e2e)
    b_e.step(args.warmup)
    R.barrier()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        b_e.step(1)
    pe = [b_e.scalars(s).potential_energy for s in b_e.slots]
    e2e_s = R.max(time.perf_counter() - t0)
    e2e_value = R.ws * n_atoms * n_e2e / e2e_s
    b_e.close()
    b.close()

    b64, _, t64, _ = timed("fp64")
    step_ms64 = R.max(t64["step_ms"])
    value64 = R.ws * n_atoms * args.steps / (step_ms64 / 1e3)
    b64.close()

    # the same replicas one per launch: each replica alone in its own engine,
    # stepped with the same kernels; device time summed over replicas
    solo_steps = max(3, min(args.steps, 20))
    solo_ms = 0.0
    for c in cfgs:
        e = Engine(c, precision="mixed", profile="phys", device=R.local)
        e.run_n(args.warmup)
        solo_ms += e.step_timed(solo_steps)["step_ms"]
        e.close()
    solo_ms = R.max(solo_ms)
    value_solo = R.ws * n_atoms * solo_steps / (solo_ms / 1e3)

    if R.rank != 0:
        return None
    from oracle.oracle import Oracle
    o = Oracle()
    sample = [0, 1, 2, 192, 193]
    acc = {}
    for prec in ("mixed", "fp64"):
        errs, eerrs = [], []
        for k in sample:
            F_o, e_o = o.forces(cfgs[k], "phys")
            e0 = Engine(cfgs[k], precision=prec, profile="phys", device=R.local)
            F, e = e0.compute_forces()
            e0.close()
            errs.append(rel_rms(F, F_o))
            eerrs.append(abs(sum(e.values()) - e_o["total"]) / abs(e_o["total"]))
        acc[prec] = {"rel_rms_force_err_max": max(errs), "rel_energy_err_max": max(eerrs),
                     "replicas": sample}
    cpu = None
    if not args.skip_cpu and R.ws == 1:
        cpu = cpu_reference_concurrent([cfgs[k] for k in BATCH_CPU_SAMPLE], args.cpu_steps,
                                       BATCH_CPU_WHAT)
    # pair-kernel algorithmic work, summed over the replicas
    b_alg = f_alg = 0.0
    for w, c in zip(ws_, cfgs):
        ba, fa = lj_pair_work(w.n_atoms, c.box_size, c.lj_cutoff)
        b_alg += ba * w.n_atoms
        f_alg += fa * w.n_atoms
    roof = roofline(b_alg, f_alg, nb_ms, clocks, PAIR_DRAM_BYTES["batch256"],
                    "k_nb_f32 (LJ pair kernel over all 256 replicas in one launch)", False,
                    "average over the timed steps, one launch covers every replica")
    n_lj = sum(1 for w in ws_ if w.name.startswith("lj_"))
    return {
        "metric": "atom-steps/s", "value": round(value, 1), "unit": "atom-steps/s",
        "n_gpus": R.ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": round(step_ms / args.steps, 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "precision": "mixed: FP32 pair/mesh/bonded math, int64 fixed-point forces, FP64 integration",
        "data": "synthetic (seeded LJ fluids on jittered lattices, decane melts grown as "
                "self-avoiding random walks; one seed per replica)",
        "config": {"workload": "batch256", "replicas": len(cfgs), "lj_fluids": n_lj,
                   "decane_melts": len(cfgs) - n_lj, "n_atoms_total": n_atoms,
                   "atoms_min": min(w.n_atoms for w in ws_),
                   "atoms_max": max(w.n_atoms for w in ws_), "dt_ps": 0.002, "ensemble": "NVE",
                   "profile": "phys", "device_bytes": used,
                   "l2": "flushed between timed steps (256 MiB overwrite outside the step events)",
                   "parallelism": f"replicas x{R.ws} (one 256-replica batch per GPU)"},
        "fp64_path": {"value": round(value64, 1), "ms_per_step": round(step_ms64 / args.steps, 5),
                      "mixed_over_fp64": round(value / value64, 3)},
        "one_per_launch": {"value": round(value_solo, 1), "steps": solo_steps,
                           "batched_over_one_per_launch": round(value / value_solo, 3),
                           "how": "each replica alone in its own engine (same kernels, one CUDA "
                                  "graph per step), device step times summed over the replicas"},
        "accuracy_vs_fp64_cpu_oracle": acc,
        "e2e": {"value": round(e2e_value, 1), "unit": "atom-steps/s", "steps": n_e2e,
                "h2d_bytes_per_step": 4, "d2h_bytes_per_step": 240 * len(cfgs),
                "how": "Batch.step(1) per MD step through the C ABI (returns after the device "
                       "finished; reads back each replica's 240-byte status record), potential "
                       "energies of all replicas read at the end; host wall clock"},
        "roofline": roof,
        "cpu_baseline": cpu,
        "gpu_launches": int(t_mixed["kernel_launches"]),
        "launch": launch,
        "clocks": clocks,
        "list_builds": list_builds,
        "potential_energy_finite": bool(all(math.isfinite(x) for x in pe)),
    }


def run_serve(args, R: Ranks):
    """A Poisson stream of MD jobs, continuously batched under an HBM budget."""
    from dmd_b200.core import Engine
    from dmd_b200.serve import job_mix, serve
    out = {}
    for prec in ("mixed", "fp64"):
        jobs = job_mix(args.jobs, args.rate, seed=2025 + R.rank, scale=args.scale)
        R.barrier()
        sampler = ClockSampler(R.local)
        sampler.start()
        res = serve(jobs, budget_bytes=150 * 10**9, precision=prec, profile="phys",
                    chunk=args.chunk)
        clocks = sampler.stop()
        res["atom_steps_per_s"] = R.ws * res["work_atom_steps"] / R.max(res["wall_s"])
        out[prec] = (res, clocks, jobs)
    if R.rank != 0:
        return None
    res, clocks, jobs = out["mixed"]
    res64 = out["fp64"][0]
    from oracle.oracle import Oracle
    o = Oracle()
    acc = {}
    sample = [j for j in jobs if j.n_atoms <= 20000][:3]
    for prec in ("mixed", "fp64"):
        errs = []
        for j in sample:
            F_o, _ = o.forces(j.cfg, "phys")
            e0 = Engine(j.cfg, precision=prec, profile="phys", device=R.local)
            F, _ = e0.compute_forces()
            e0.close()
            errs.append(rel_rms(F, F_o))
        acc[prec] = {"rel_rms_force_err_max": max(errs), "jobs": [j.jid for j in sample]}
    cpu = None
    if not args.skip_cpu and R.ws == 1:
        cpu = cpu_reference([j.cfg for j in sample[:2]], args.cpu_steps,
                            f"jobs {sample[0].jid} and {sample[1].jid} of the same stream")
    steps_total = sum(j.n_steps for j in jobs)
    return {
        "metric": "atom-steps/s", "value": round(res["atom_steps_per_s"], 1),
        "unit": "atom-steps/s", "n_gpus": R.ws, "steps": steps_total, "warmup": 0,
        "ms_per_step": round(res["step_latency_ms"]["p50"], 5), "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "precision": "mixed: FP32 pair/mesh/bonded math, int64 fixed-point forces, FP64 integration",
        "data": "synthetic (seeded job stream: LJ argon and SPME water, one seed per job)",
        "config": {"workload": "serve", "jobs": len(jobs), "rate_jobs_per_s": args.rate,
                   "scale": args.scale, "chunk_steps": args.chunk, "budget_gb": 150,
                   "atoms_min": min(j.n_atoms for j in jobs),
                   "atoms_max": max(j.n_atoms for j in jobs), "profile": "phys",
                   "l2": "not flushed (jobs' state stays resident, far above L2 in total)",
                   "parallelism": f"replicas x{R.ws} (one job stream per GPU)"},
        "latency": {"step_ms": res["step_latency_ms"], "job_s": res["job_latency"],
                    "step_ms_steady": res["step_latency_ms_steady"],
                    "step_ms_rebuild": res["step_latency_ms_rebuild"]},
        "wall_s": round(res["wall_s"], 3),
        "fp64_path": {"value": round(res64["atom_steps_per_s"], 1),
                      "latency": {"step_ms": res64["step_latency_ms"], "job_s": res64["job_latency"]},
                      "mixed_over_fp64": round(res["atom_steps_per_s"] / res64["atom_steps_per_s"], 3)},
        "accuracy_vs_fp64_cpu_oracle": acc,
        "e2e": {"value": round(res["atom_steps_per_s"], 1), "unit": "atom-steps/s",
                "h2d_bytes_per_step": None, "d2h_bytes_per_step": None,
                "how": "the whole stream through dmd_b200.serve (C ABI batch API, host wall clock "
                       "from the first arrival to the last completion; job inputs uploaded at "
                       "admission, final positions read at completion)"},
        "roofline": None,
        "cpu_baseline": cpu,
        "gpu_launches": None,
        "launch": res["launch_configs"],
        "clocks": clocks,
    }


def _ref_worker(args):
    """One replica on one host core (spawned process): the reference's engine
    stepped `steps` times; returns (atom-steps, seconds, kind)."""
    cfg, steps = args
    sys.path.insert(0, ROOT)
    from oracle.oracle import Oracle, Ref, ref_available
    if ref_available():
        eng, kind = Ref().engine(cfg), "reference"
    else:
        eng, kind = Oracle().engine(cfg, "ref", brute_list=True), "port"
    t0 = time.perf_counter()
    eng.step(steps)
    return len(cfg.masses) * steps, time.perf_counter() - t0, kind


def cpu_reference_concurrent(cfgs, steps, what_sample):
    """Independent replicas on the host cores at once, one process per replica
    and core (the reference's engine is single-threaded): aggregate atom-steps/s
    = all replicas' atom-steps / the slowest replica's time.  Processes are
    spawned, never forked, so no CUDA state is inherited."""
    import multiprocessing as mp
    cores = min(len(cfgs), os.cpu_count() or 1)
    with mp.get_context("spawn").Pool(cores) as pool:
        res = pool.map(_ref_worker, [(c, steps) for c in cfgs])
    atom_steps = sum(r[0] for r in res)
    secs = max(r[1] for r in res)
    kind = res[0][2]
    return {"value": round(atom_steps / secs, 1), "unit": "atom-steps/s", "cores": cores,
            "kind": kind,
            "sample": f"{steps} MD steps from the start of each of {what_sample}, {len(cfgs)} "
                      f"processes on {cores} host cores at once (the reference's C++, src/ "
                      f"unmodified, one replica per core); slowest replica {secs:.1f} s"}


def cpu_reference_extrapolated(n_atoms, small_cfg, steps):
    """The reference's rate for a system too large to time directly (its first
    step alone builds an O(N^2) pair list), from the same water model at a
    timed size: per step = (list rebuild, O(N^2) pair tests, every 5 steps) +
    (everything else, linear in N), each part timed on the smaller box and
    scaled by its own law."""
    from oracle.oracle import Ref, ref_available
    if not ref_available():
        return None
    n1 = len(small_cfg.masses)
    ref = Ref()
    t0 = time.perf_counter()
    ref.lj(small_cfg)  # a fresh LennardJones: one O(N^2) rebuild + one pair pass
    t_rb = time.perf_counter() - t0
    eng = ref.engine(small_cfg)
    t0 = time.perf_counter()
    eng.step(steps)
    t_steps = time.perf_counter() - t0
    rebuilds = (2 * steps + 9) // 10  # every 10 force evaluations, 2 per step
    t_other = max(t_steps - rebuilds * t_rb, 0.0) / steps
    scale = n_atoms / n1
    t_step = t_rb * scale * scale / 5.0 + t_other * scale
    return {"value": round(n_atoms / t_step, 1), "unit": "atom-steps/s", "cores": 1,
            "kind": "reference",
            "sample": f"extrapolated: the reference's C++ (src/, unmodified) timed on the "
                      f"{n1:,}-atom box of the same water model -- one O(N^2) list rebuild "
                      f"({t_rb:.2f} s) and {steps} MD steps ({t_steps:.1f} s) -- then the "
                      f"rebuild (every 5 steps) scaled by (N/{n1:,})^2 and the rest of the step "
                      f"by N/{n1:,}; predicted {t_step:.0f} s per step at {n_atoms:,} atoms"}


def cpu_reference(cfgs, steps, what_sample):
    """The reference's CPU path on one host core (the reference has no threading
    on this path), timed on a bounded sample from the start of each run.

    Preferred: the reference's own C++ (src/ compiled unmodified by oracle/Makefile;
    CoulombPME against the FFTW-API shim, since FFTW3 is not installed), stepped
    in SimulationEngine::step order: its O(N^2) LennardJones list rebuilt every
    10 force evaluations, two evaluations per step, FP64.  If that build is not
    present, the oracle's restatement of the same algorithm (REF profile)."""
    from oracle.oracle import Oracle, Ref, ref_available
    if ref_available():
        make, kind = (lambda c: Ref().engine(c)), "reference"
        what = "reference C++ (src/, unmodified; PME via the FFTW-API shim)"
    else:
        make, kind = (lambda c: Oracle().engine(c, "ref", brute_list=True)), "port"
        what = "oracle restatement of the reference algorithm (REF profile)"
    atom_steps, secs = 0, 0.0
    for cfg in cfgs:
        eng = make(cfg)
        t0 = time.perf_counter()
        eng.step(steps)
        secs += time.perf_counter() - t0
        atom_steps += len(cfg.masses) * steps
    return {"value": round(atom_steps / secs, 1), "unit": "atom-steps/s", "cores": 1,
            "kind": kind,
            "sample": f"{steps} MD steps from the start of {what_sample} ({what}; includes "
                      f"{(steps + 4) // 5} O(N^2) list rebuilds per system), {secs:.1f} s"}


def run_reference(args):
    ws, rank, _ = _dist()
    if rank != 0:
        return None
    steps = min(args.steps, args.cpu_steps)
    if args.workload in SINGLE:
        w = SINGLE[args.workload]["make"](0)
        cfgs = [w.config()]
        what = f"the same {w.n_atoms:,}-atom system"
        if w.n_atoms > CPU_MAX_ATOMS:
            cpu = cpu_reference_extrapolated(w.n_atoms, water30k(0).config(), steps)
        else:
            cpu = cpu_reference(cfgs, steps, what)
    elif args.workload == "batch256":
        from dmd_b200 import workloads as W
        ws_ = W.batch_256(seed=1234)
        cfgs = [ws_[k].config() for k in BATCH_CPU_SAMPLE]
        cpu = cpu_reference_concurrent(cfgs, steps, BATCH_CPU_WHAT)
    else:
        from dmd_b200.serve import job_mix
        jobs = [j for j in job_mix(args.jobs, args.rate, seed=2025, scale=args.scale)
                if j.n_atoms <= 20000][:2]
        cfgs = [j.cfg for j in jobs]
        cpu = cpu_reference(cfgs, steps, "two jobs of the served stream")
    if cpu is None:
        return {"impl": "reference", "metric": "atom-steps/s", "value": None,
                "unit": "atom-steps/s", "n_gpus": ws,
                "unavailable": "the reference build (oracle/_ref) is not present"}
    v = cpu["value"]
    return {"impl": "reference", "metric": "atom-steps/s", "value": v, "unit": "atom-steps/s",
            "n_gpus": ws, "steps": steps, "warmup": 0, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "n_atoms": sum(len(c.masses) for c in cfgs),
                       "profile": "ref",
                       "implementation": ("the reference's C++ (src/, unmodified; PME via the "
                                          "FFTW-API shim)" if cpu["kind"] == "reference" else
                                          "the oracle's restatement of the reference algorithm"),
                       "sample_steps": steps},
            "cpu_baseline": cpu,
            "e2e": {"value": v, "unit": "atom-steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


def run_ours(args):
    ws, rank, local = _dist()
    R = Ranks(local)
    try:
        if args.workload in SINGLE:
            return run_single(args, R)
        if args.workload == "batch256":
            return run_batch(args, R)
        return run_serve(args, R)
    finally:
        R.close()


DEFAULT_STEPS = {"water30k": 2000, "argon4k": 2000, "water750k": 200, "batch256": 200, "serve": 10}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", choices=WORKLOADS, default="water30k")
    ap.add_argument("--cpu-steps", type=int, default=10)
    ap.add_argument("--drift-steps", type=int, default=1000, help="argon4k: NVE drift run length")
    ap.add_argument("--skip-cpu", action="store_true")
    # served stream
    ap.add_argument("--jobs", type=int, default=24)
    ap.add_argument("--rate", type=float, default=2.0, help="Poisson arrivals (jobs/s)")
    ap.add_argument("--scale", type=float, default=1.0, help="shrinks job sizes and steps")
    ap.add_argument("--chunk", type=int, default=100, help="steps per device call")
    args = ap.parse_args()
    if args.steps is None:
        args.steps = DEFAULT_STEPS[args.workload]
    if args.warmup < 3:
        args.warmup = 3
    out = run_reference(args) if args.impl == "reference" else run_ours(args)
    if out is not None:
        print(json.dumps(out), flush=True)


if __name__ == "__main__":
    main()
