"""Input files -> SimulationConfig: this package's reader of the reference's
``system.json`` / ``config.json`` formats.

The formats are the reference's (python/dmd/system.py:18-114 reads system.json,
python/dmd/config.py:13-58 defines the strict config.json schema); the reader
is table driven:

* ``CONFIG_KEYS`` lists every config.json key once, with its JSON type and the
  SimulationConfig attribute it sets.  One pass over that table both checks a
  document (every key present, no others, types as declared) and applies it.
* ``TERMS`` lists each force-field term list of system.json with its index and
  parameter columns.  A parameter column is read when the list's first term
  carries it (later terms missing it take 0), as the reference does.

Atom type names are numbered in sorted order and every listed LJ pair fills
both (i, j) and (j, i) of an n_types x n_types table that starts at sigma 1,
epsilon 0 (python/dmd/system.py:36-55): the C++ side has no combining rule.

Backend options (precision, semantic profile, skin) are not config keys; they
are Engine / Batch keyword arguments.
"""
from __future__ import annotations

import json
from typing import Any

import numpy as np

from .core import SimulationConfig

# (section, key, JSON type, SimulationConfig attribute; "a.b" = nested)
CONFIG_KEYS = (
    ("run", "dt", float, "dt"),
    ("run", "n_steps", int, "n_steps"),
    ("run", "init_temperature", float, "init_temperature"),
    ("run", "gen_vel", bool, "gen_vel"),
    ("run", "seed", int, "seed"),
    ("output", "trajectory_path", str, "trajectory_path"),
    ("output", "nstxout", int, "nstxout"),
    ("output", "nstvout", int, "nstvout"),
    ("output", "nstenergy", int, "nstenergy"),
    ("output", "energy_path", str, "energy_path"),
    ("output", "checkpoint_interval", int, "checkpoint_interval"),
    ("output", "checkpoint_path", str, "checkpoint_path"),
    ("lj", "cutoff", float, "lj_cutoff"),
    ("electrostatics", "coulomb_type", str, "coulomb_type"),
    ("electrostatics", "cutoff", float, "coulomb_cutoff"),
    ("electrostatics", "pme_order", int, "pme_order"),
    ("electrostatics", "pme_grid_spacing", float, "pme_grid_spacing"),
    ("electrostatics", "ewald_coeff", float, "ewald_coeff"),
    ("thermostat", "type", str, "thermostat.type"),
    ("thermostat", "temperature", float, "thermostat.temperature"),
    ("thermostat", "tau", float, "thermostat.tau"),
    ("thermostat", "frequency", float, "thermostat.frequency"),
    ("barostat", "type", str, "barostat.type"),
    ("barostat", "pressure", float, "barostat.pressure"),
    ("barostat", "tau", float, "barostat.tau"),
    ("barostat", "compressibility", float, "barostat.compressibility"),
    ("constraints", "type", str, "constraint_type"),
    ("constraints", "tolerance", float, "constraint_tolerance"),
)

# term list -> (index columns, parameter columns): (JSON key, attribute, dtype)
TERMS = {
    "bonds": ((("i", "bond_i"), ("j", "bond_j")),
              (("k", "bond_k", float), ("r0", "bond_r0", float))),
    "angles": ((("i", "angle_i"), ("j", "angle_j"), ("k", "angle_k")),
               (("k_theta", "angle_k_theta", float), ("theta0", "angle_theta0", float))),
    "dihedrals": ((("i", "dihedral_i"), ("j", "dihedral_j"), ("k", "dihedral_k"), ("l", "dihedral_l")),
                  (("k_phi", "dihedral_k_phi", float), ("periodicity", "dihedral_periodicity", int),
                   ("phi0", "dihedral_phi0", float))),
    "impropers": ((("i", "improper_i"), ("j", "improper_j"), ("k", "improper_k"), ("l", "improper_l")),
                  (("k_phi", "improper_k_phi", float), ("phi0", "improper_phi0", float))),
}


class InputError(ValueError):
    """A config.json / system.json document that does not fit the format."""


def _json_type_ok(value: Any, kind: type) -> bool:
    # JSON has one number type: an integer literal is a valid float field (and,
    # as in the reference's isinstance check, a bool passes as an int)
    if kind is float:
        return isinstance(value, (int, float)) and not isinstance(value, bool)
    return isinstance(value, kind)


def check_config(doc: dict) -> None:
    """Raise InputError unless `doc` has exactly the keys of CONFIG_KEYS with
    the declared JSON types."""
    if not isinstance(doc, dict):
        raise InputError("config.json: the document must be an object")
    expected: dict[str, dict[str, type]] = {}
    for sec, key, kind, _ in CONFIG_KEYS:
        expected.setdefault(sec, {})[key] = kind
    for sec in doc:
        if sec not in expected:
            raise InputError(f"config.json: unknown section '{sec}'")
    for sec, keys in expected.items():
        if sec not in doc:
            raise InputError(f"config.json: missing section '{sec}'")
        body = doc[sec]
        for key in body:
            if key not in keys:
                raise InputError(f"config.json: unknown key '{sec}.{key}'")
        for key, kind in keys.items():
            if key not in body:
                raise InputError(f"config.json: missing key '{sec}.{key}'")
            if not _json_type_ok(body[key], kind):
                raise InputError(f"config.json: '{sec}.{key}' must be a {kind.__name__}, "
                                 f"not {type(body[key]).__name__}")


def _set(cfg: SimulationConfig, path: str, value: Any) -> None:
    obj = cfg
    *head, last = path.split(".")
    for part in head:
        obj = getattr(obj, part)
    setattr(obj, last, value)


def apply_config(cfg: SimulationConfig, doc: dict) -> SimulationConfig:
    """Check a config.json document and copy it onto `cfg`.  LJ is switched on
    (the reference's apply_config does the same, python/dmd/config.py:104); a
    SHAKE request without constraint pairs in the system is an error."""
    check_config(doc)
    for sec, key, kind, attr in CONFIG_KEYS:
        v = doc[sec][key]
        _set(cfg, attr, float(v) if kind is float else v)
    cfg.use_lj = True
    if cfg.constraint_type == "shake" and len(cfg.constraint_i) == 0:
        raise InputError("config.json: constraints.type is 'shake' but system.json lists no constraints")
    return cfg


def _column(terms: list, key: str, dtype) -> np.ndarray:
    return np.array([t.get(key, 0) for t in terms], dtype=dtype)


def read_system(doc: dict, cfg: SimulationConfig | None = None) -> SimulationConfig:
    """Fill a SimulationConfig from a system.json document."""
    cfg = SimulationConfig() if cfg is None else cfg
    cell, atoms = doc["cell"], doc["atoms"]
    pos = np.asarray(cell["positions"], dtype=np.float64).reshape(-1, 3)
    n = len(pos)
    cfg.box_size = float(cell.get("box_size", 3.0))
    cfg.pos_x, cfg.pos_y, cfg.pos_z = pos[:, 0].copy(), pos[:, 1].copy(), pos[:, 2].copy()
    cfg.masses = np.asarray(atoms["mass"], dtype=np.float64)
    cfg.charges = np.asarray(atoms["charge"], dtype=np.float64) if "charge" in atoms else np.zeros(n)
    names = list(atoms.get("type", []))
    index = {nm: k for k, nm in enumerate(sorted(set(names)))}
    cfg.atom_types = np.array([index[nm] for nm in names], dtype=np.int32)

    ff = doc.get("force_field", {})
    lj = ff.get("lennard_jones")
    if lj:
        nt = len(index)
        sigma, eps = np.ones((nt, nt)), np.zeros((nt, nt))
        for p in lj.get("pairs", []):
            a, b = index[p["type_i"]], index[p["type_j"]]
            sigma[a, b] = sigma[b, a] = p.get("sigma", 1.0)
            eps[a, b] = eps[b, a] = p.get("epsilon", 0.0)
        cfg.use_lj = True
        cfg.lj_cutoff = float(lj.get("cutoff", 2.5))
        cfg.lj_sigma, cfg.lj_epsilon = sigma.ravel(), eps.ravel()
    for name, (idx_cols, par_cols) in TERMS.items():
        terms = ff.get(name, [])
        if not terms:
            continue
        for key, attr in idx_cols:
            setattr(cfg, attr, _column(terms, key, np.int32))
        for key, attr, dtype in par_cols:
            if key in terms[0]:
                setattr(cfg, attr, _column(terms, key, np.int32 if dtype is int else np.float64))
    cons = ff.get("constraints", [])
    if cons:
        cfg.constraint_i = [c["i"] for c in cons]
        cfg.constraint_j = [c["j"] for c in cons]
        cfg.constraint_dist = [c["distance"] for c in cons]
    excl = doc.get("exclusions", [])
    cfg.excl_i = [int(e[0]) for e in excl]
    cfg.excl_j = [int(e[1]) for e in excl]
    return cfg


def _document(src) -> dict:
    if isinstance(src, dict):
        return src
    text = str(src)
    if text.lstrip().startswith("{"):
        return json.loads(text)
    with open(text) as fh:
        return json.load(fh)


def load_inputs(system, config) -> SimulationConfig:
    """SimulationConfig from a system.json and a config.json (each a dict, a
    JSON string or a file path)."""
    return apply_config(read_system(_document(system)), _document(config))
