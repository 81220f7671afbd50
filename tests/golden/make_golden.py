"""Golden fixtures produced by the reference's own code.

Runs the reference's C++ classes compiled unmodified from their sources
(oracle/_ref/libdmdref.so, built by oracle/Makefile; CoulombPME against the
FFTW-API shim) on small seeded systems and writes, per case,

    tests/golden/<case>/system.json, config.json   (the reference's input format)
    tests/golden/<case>/expected.npz               (forces, energies, pair lists,
                                                    trajectory end states)

Only this script needs the reference tree; the fixtures it writes are what the
tests read.  Regenerate with:  python tests/golden/make_golden.py
"""
from __future__ import annotations

import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from dmd_b200 import workloads as W  # noqa: E402
from dmd_b200.inputs import load_inputs  # noqa: E402
from oracle.oracle import Ref, build  # noqa: E402


def _jitter(w, sigma, seed):
    rng = np.random.default_rng(seed)
    w.pos = w.pos + rng.normal(0.0, sigma, w.pos.shape)
    return w


def cases():
    """(name, workload, kind) with kind 'components' or ('trajectory', steps)."""
    argon = _jitter(W.argon_fcc(n_cells=4, a=0.575, T=120.0, seed=5), 0.01, 1)
    water = _jitter(W.water_box(n_mol=100, box=1.45, seed=3, spacing=0.1, thermostat="nose-hoover",
                                dt=0.0005), 0.005, 2)
    decane = _jitter(W.decane_melt(12, 7), 0.002, 3)
    argon_t = W.argon_fcc(n_cells=3, a=0.575, T=120.0, seed=11, rc=0.8)
    argon_t.thermostat = W._thermo("nose-hoover", T=100.0)
    water_t = W.water_box(n_mol=60, box=1.24, seed=4, spacing=0.11, thermostat="nose-hoover",
                          dt=0.0005)
    return [("argon_components", argon, "components"),
            ("water_pme_components", water, "components"),
            ("decane_components", decane, "components"),
            ("argon_nh_trajectory", argon_t, ("trajectory", 25)),
            ("water_pme_trajectory", water_t, ("trajectory", 6))]


def main():
    build(ref=True)
    ref = Ref()
    for name, w, kind in cases():
        system, config = w.to_json()
        cfg = load_inputs(system, config)
        out = {}
        if kind == "components":
            f, e, (pi, pj) = ref.lj(cfg)
            out.update(lj_f=f, lj_e=e, lj_pi=pi, lj_pj=pj)
            if len(cfg.bond_i):
                out["bond_f"], out["bond_e"] = ref.bond(cfg)
            if len(cfg.angle_i):
                out["angle_f"], out["angle_e"] = ref.angle(cfg)
            if len(cfg.dihedral_i):
                out["dihedral_f"], out["dihedral_e"] = ref.dihedral(cfg)
            if len(cfg.excl_i):
                out["exclusion_f"], out["exclusion_e"] = ref.exclusion(cfg)
            if cfg.coulomb_type == "pme":
                out["pme_f"], out["pme_e"] = ref.pme(cfg)
        else:
            eng = ref.engine(cfg)
            eng.step(kind[1])
            s = eng.scalars()
            out.update(pos=eng.get(0), vel=eng.get(1), forces=eng.get(2), pe=s["pe"],
                       steps=kind[1], lj_counter=s["lj_counter"], zeta=s["zeta"])
        d = os.path.join(HERE, name)
        os.makedirs(d, exist_ok=True)
        with open(os.path.join(d, "system.json"), "w") as fh:
            json.dump(system, fh)
        with open(os.path.join(d, "config.json"), "w") as fh:
            json.dump(config, fh, indent=1)
        np.savez_compressed(os.path.join(d, "expected.npz"), **{k: np.asarray(v) for k, v in out.items()})
        print(name, cfg.pos_x.shape[0], "atoms:", ", ".join(sorted(out)))


if __name__ == "__main__":
    main()
