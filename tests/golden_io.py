"""Golden fixtures for the D3Q19 TRT step, generated by
tests/golden/make_golden.py from LBM-Bench's own kernels (oracle/_ref) and
committed. Each case records its inputs (geometry, seed, parameters) and the
SHA-256 of the final state over fluid cells, plus a few totals; tiny cases
also keep the full final state.
"""
from __future__ import annotations

import hashlib
import json
import os

import numpy as np

import oracle as O

GOLDEN_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES_JSON = os.path.join(GOLDEN_DIR, "golden_cases.json")
ARRAYS_NPZ = os.path.join(GOLDEN_DIR, "golden_arrays.npz")


def state_digest(f: np.ndarray, flags: np.ndarray) -> str:
    """SHA-256 of f[:, fluid cells] as little-endian float64, C order."""
    m = O.fluid_mask(flags)
    a = np.ascontiguousarray(f[:, m], dtype="<f8")
    return hashlib.sha256(a.tobytes()).hexdigest()


def build_flags(case: dict, arrays) -> np.ndarray:
    """Flags of a case: a reference geometry (rebuilt with our own
    generator-independent rules via the oracle module's callers) or stored."""
    if "flags_key" in case:
        return np.asarray(arrays[case["flags_key"]], dtype=np.int32)
    return reference_geometry(case["geometry"], case["dims"], case["periodic_in"])


def reference_geometry(kind: str, dims, periodic_in):
    """Restates the reference's geometryCreate (src/lbm.c:52-187) in numpy
    so fixtures can be rebuilt without the reference tree."""
    nx, ny, nz = dims
    per = list(periodic_in)
    k = kind.lower()
    nb = 8
    if k.startswith("channel"):
        kind_id = "channel"
    elif k.startswith("box"):
        kind_id = "box"
    elif k.startswith("pipe"):
        kind_id = "pipe"
    elif k.startswith("blocks"):
        kind_id = "blocks"
        if len(kind) > 7:
            nb = int(kind[7:]) if kind[7:].lstrip("-").isdigit() and int(kind[7:]) > 0 else 8
    elif k.startswith("fluid"):
        kind_id = "fluid"
    else:
        raise ValueError(kind)
    if kind_id in ("channel", "pipe", "blocks"):
        per[0] = 1
    elif kind_id == "fluid":
        per = [1, 1, 1]
    flags = np.ones((nz, ny, nx), dtype=np.int32)
    if not per[0]:
        flags[:, :, 0] = 0
        flags[:, :, nx - 1] = 0
    if not per[1]:
        flags[:, 0, :] = 0
        flags[:, ny - 1, :] = 0
    if not per[2]:
        flags[0, :, :] = 0
        flags[nz - 1, :, :] = 0
    if kind_id == "pipe":
        cy, cz = ny / 2.0 - 0.5, nz / 2.0 - 0.5
        r = min(ny, nz) / 2 - 1
        z, y = np.meshgrid(np.arange(nz), np.arange(ny), indexing="ij")
        out = (z - cz) ** 2 + (y - cy) ** 2 >= r * r
        flags[out, :] = 0
    elif kind_id == "blocks":
        z = np.arange(nz)[:, None, None]
        y = np.arange(ny)[None, :, None]
        x = np.arange(nx)[None, None, :]
        solid = ((z % (2 * nb)) >= nb) & ((y % (2 * nb)) >= nb) & ((x % (2 * nb)) >= nb)
        flags[solid] = 0
    return flags


def effective_periodic(case: dict):
    return tuple(case["periodic"])


def initial_state(case: dict, flags: np.ndarray) -> np.ndarray:
    """The case's seeded perturbed equilibrium: the counter-based generator
    of the benchmark (init "counter", the product's lbm_perturbed_equilibrium
    restated) or numpy's default generator (every other case)."""
    if case.get("init") == "counter":
        return O.counter_equilibrium(flags, case["seed"], case.get("amp", 1e-4))
    return O.perturbed_state(flags, case["seed"], amp=case.get("amp", 1e-4))


def load():
    with open(CASES_JSON) as fh:
        cases = json.load(fh)
    arrays = np.load(ARRAYS_NPZ)
    return cases, arrays
