"""Generates the golden fixtures (golden_cases.json, golden_arrays.npz) from
LBM-Bench's own kernels, compiled unmodified from the reference tree into
oracle/_ref (run `make -C oracle` first; needs the reference sources, so it
runs where they are mounted, not on the GPU host).

For every case the script
  * builds the geometry with the reference's geometryCreate (or a stored
    porous flag field),
  * injects a seeded perturbed equilibrium through kd->SetNode,
  * runs the reference's pull-soa, push-soa and aa-soa kernels (plus the AoS
    and blocked variants for the first cases) and checks they agree bit for
    bit,
  * records the SHA-256 of the final state over fluid cells and some totals.
It also records the reference's Poiseuille verification (-V) result, two
pressure-driven channels run with the reference's Zou-He boundary pass
after every pull and push step, and the stated config-0 case at full size:
a 64^3 channel, omega 1.25, Lambda 3/16, F 1e-6, the counter-based seeded
+-1e-4 equilibrium of the benchmark, 1000 steps (several minutes of CPU).

Usage: python tests/golden/make_golden.py [--only NAME ...]
  --only regenerates the named cases and keeps every other stored case.
"""
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle as O  # noqa: E402
import golden_io  # noqa: E402

CASES = [
    # name, geometry, dims, periodic_in, omega, lambda, xforce, force, steps, seed, variant
    ("channel_l12", "channel", (12, 10, 14), (0, 0, 0), 1.25, 1 / 12, 1e-6, 1, 20, 7, "verify"),
    ("channel_l316", "channel", (12, 10, 14), (0, 0, 0), 1.25, 3 / 16, 1e-6, 1, 20, 7,
     "verify_l316"),
    ("box_xy", "box", (10, 9, 8), (1, 1, 0), 1.0, 1 / 12, 1e-5, 1, 10, 11, "verify"),
    ("blocks2_l316", "blocks-2", (12, 12, 12), (0, 0, 0), 0.7, 3 / 16, 1e-6, 1, 8, 3,
     "verify_l316"),
    ("pipe", "pipe", (9, 12, 11), (0, 0, 0), 1.6, 1 / 12, 1e-6, 1, 6, 5, "verify"),
    ("fluid_all_periodic", "fluid", (6, 7, 5), (0, 0, 0), 1.9, 3 / 16, 2e-6, 1, 12, 9,
     "verify_l316"),
    ("box_z_walls_noforce", "box", (8, 9, 10), (1, 1, 0), 1.1, 1 / 12, 0.0, 0, 14, 21, "plain"),
    ("channel_noforce", "channel", (16, 12, 10), (0, 0, 0), 1.25, 1 / 12, 0.0, 0, 10, 4, "plain"),
    ("tiny_box_xyz_walls", "box", (6, 5, 4), (0, 0, 0), 1.2, 1 / 12, 1e-6, 1, 4, 2, "verify"),
    ("tiny_channel", "channel", (5, 6, 5), (0, 0, 0), 1.25, 3 / 16, 1e-6, 1, 6, 8, "verify_l316"),
]
FULL_STATE = {"tiny_box_xyz_walls", "tiny_channel"}
ALL_KERNELS = {"channel_l12", "box_xy", "blocks2_l316"}


def porous_flags(dims, fraction, rmin, rmax, seed):
    """A small porous channel for the fixtures: channel walls plus random
    spheres (numpy generator, stored in the fixture, so the product's own
    generator is not involved)."""
    nx, ny, nz = dims
    flags = golden_io.reference_geometry("channel", dims, (0, 0, 0))
    rng = np.random.default_rng(seed)
    z, y, x = np.meshgrid(np.arange(nz), np.arange(ny), np.arange(nx), indexing="ij")
    while (flags == 0).mean() < fraction:
        c = rng.uniform(0, 1, 3) * np.array([nx, ny, nz])
        r = rng.uniform(rmin, rmax)
        dx = np.minimum(np.abs(x - c[0]), nx - np.abs(x - c[0]))
        inside = dx ** 2 + (y - c[1]) ** 2 + (z - c[2]) ** 2 <= r * r
        flags[inside] = 0
    return flags


# The 64^3 channel of the first benchmark configuration, at its stated size.
CONFIG0 = ("config0_channel64", "channel", (64, 64, 64), (0, 0, 0), 1.25, 3 / 16, 1e-6, 1, 1000,
           7, "verify_l316")


def run_case(name, geo, dims, pin, omega, lam, xforce, force, steps, seed, variant, arrays,
             flags=None, init="rng"):
    ref = O.Reference(variant)
    if flags is None:
        flags, per, counts = ref.geometry(geo, dims, pin)
        mine = golden_io.reference_geometry(geo, dims, pin)
        assert np.array_equal(mine, flags), f"{name}: numpy geometry restatement differs"
    else:
        per = (1, 0, 0)
    f0 = O.counter_equilibrium(flags, seed) if init == "counter" else \
        O.perturbed_state(flags, seed)
    kernels = ["pull-soa", "push-soa", "aa-soa"]
    if name in ALL_KERNELS:
        kernels = ref.kernels()
    outs = {}
    for k in kernels:
        out, dur, it, nbb = ref.run(k, flags, per, f0, steps, omega, xforce)
        outs[k] = (out, it, nbb)
    m = O.fluid_mask(flags)
    base = outs["pull-soa"][0]
    for k, (out, it, nbb) in outs.items():
        assert np.array_equal(out[:, m], base[:, m]), f"{name}: {k} differs from pull-soa"
    rho, ux, uy, uz = O.moments(base, flags)
    case = {
        "name": name, "geometry": geo, "dims": list(dims), "periodic_in": list(pin),
        "periodic": list(per), "omega": omega, "lambda": lam, "xforce": xforce,
        "force_on": force, "steps": steps, "seed": seed, "amp": 1e-4, "reference_build": variant,
        "kernels_agreeing": kernels, "n_fluid": int(m.sum()),
        "n_bounce_back_pull": int(outs["pull-soa"][2]),
        "aa_final_iteration": int(outs["aa-soa"][1]),
        "sha256": golden_io.state_digest(base, flags),
        "mass": float(rho[m].sum()), "momentum": [float(ux[m].sum()), float(uy[m].sum()),
                                                  float(uz[m].sum())],
    }
    if init == "counter":
        case["init"] = "counter"
        vel = [a[m] / rho[m] for a in (ux, uy, uz)]
        case["norms"] = {"rho_l2": float(np.linalg.norm(rho[m])),
                         "u_l2": float(np.sqrt(sum(float((v * v).sum()) for v in vel)))}
    if name in FULL_STATE:
        arrays[f"{name}_f"] = base
        case["state_key"] = f"{name}_f"
    return case, flags


def inlet_outlet_flags(dims, solid, seed):
    """Channel (walls on the y and z faces) with inlet cells (2) on x = 0
    and outlet cells (4) on x = nx-1, plus random solid cells inside."""
    nx, ny, nz = dims
    rng = np.random.default_rng(seed)
    flags = np.ones((nz, ny, nx), dtype=np.int32)
    flags[rng.uniform(size=flags.shape) < solid] = 0
    flags[:, :, 0] = 2
    flags[:, :, -1] = 4
    flags[:, [0, -1], :] = 0
    flags[[0, -1], :, :] = 0
    return flags


PRESSURE_CASES = [
    # name, dims, solid, seed, omega, lambda, xforce, force, steps, rho_in, rho_out, variant
    ("pressure_channel", (12, 9, 8), 0.0, 31, 1.25, 3 / 16, 0.0, 0, 30, 1.005, 0.995,
     "verify_l316"),
    ("pressure_porous", (16, 10, 10), 0.15, 32, 1.1, 1 / 12, 1e-6, 1, 12, 1.002, 0.999,
     "verify"),
]


def run_pressure_case(name, dims, solid, seed, omega, lam, xforce, force, steps, rho_in,
                      rho_out, variant, arrays):
    """The reference's pull and push kernels, one step per kd->Kernel call,
    each followed by its Zou-He pass kernelComputeBoundaryConditions
    (src/lbm.c:676-785); they must agree bit for bit."""
    ref = O.Reference(variant)
    flags = inlet_outlet_flags(dims, solid, seed)
    f0 = O.perturbed_state(flags, seed)
    per = (0, 0, 0)
    outs = {k: ref.run_pressure(k, flags, per, f0, steps, omega, xforce, rho_in, rho_out)
            for k in ("pull-soa", "push-soa")}
    m = O.fluid_mask(flags)
    assert np.array_equal(outs["pull-soa"][:, m], outs["push-soa"][:, m]), name
    base = outs["pull-soa"]
    rho, ux, uy, uz = O.moments(base, flags)
    arrays[f"{name}_flags"] = flags.astype(np.int8)
    return {
        "name": name, "geometry": "stored", "dims": list(dims), "periodic_in": [0, 0, 0],
        "periodic": list(per), "omega": omega, "lambda": lam, "xforce": xforce,
        "force_on": force, "steps": steps, "seed": seed, "amp": 1e-4, "reference_build": variant,
        "kernels_agreeing": ["pull-soa", "push-soa"], "n_fluid": int(m.sum()),
        "flags_key": f"{name}_flags", "pressure": {"rho_in": rho_in, "rho_out": rho_out},
        "sha256": golden_io.state_digest(base, flags),
        "mass": float(rho[m].sum()), "momentum": [float(ux[m].sum()), float(uy[m].sum()),
                                                  float(uz[m].sum())],
    }


def main():
    import argparse
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", nargs="*", default=None)
    only = ap.parse_args().only
    O.build()
    if only:
        cases, stored = golden_io.load()
        arrays = {k: stored[k] for k in stored.files}
        for name in only:
            if name != CONFIG0[0]:
                raise SystemExit(f"--only supports {CONFIG0[0]}")
            case, _ = run_case(*CONFIG0, arrays=arrays, init="counter")
            cases = [c for c in cases if c["name"] != name] + [case]
            print(case["name"], case["sha256"][:16], case["n_fluid"])
        with open(golden_io.CASES_JSON, "w") as fh:
            json.dump(cases, fh, indent=1)
        np.savez_compressed(golden_io.ARRAYS_NPZ, **arrays)
        return
    arrays = {}
    cases = []
    for row in CASES:
        case, _ = run_case(*row, arrays=arrays)
        cases.append(case)
        print(case["name"], case["sha256"][:16], case["n_fluid"])
    # porous case with stored flags
    flags = porous_flags((24, 20, 20), 0.2, 2.0, 4.0, seed=12)
    arrays["porous_flags"] = flags.astype(np.int8)
    case, _ = run_case("porous_l316", "stored", (24, 20, 20), (0, 0, 0), 1.25, 3 / 16, 1e-6, 1,
                       16, 13, "verify_l316", arrays, flags=flags)
    case["flags_key"] = "porous_flags"
    case["solid_fraction"] = float((flags == 0).mean())
    cases.append(case)
    print(case["name"], case["sha256"][:16], case["n_fluid"])

    for row in PRESSURE_CASES:
        case = run_pressure_case(*row, arrays=arrays)
        cases.append(case)
        print(case["name"], case["sha256"][:16], case["n_fluid"])

    # the reference's own -V run: 16^3 box, x/y periodic, omega 1, F 1e-5,
    # 1000 steps from its (omega-scaled) equilibrium init, src/cli.c:84-99
    ref = O.Reference("verify")
    flags, per, _ = ref.geometry("box", (16, 16, 16), (1, 1, 0))
    verify = {}
    for k in ("pull-soa", "push-soa", "aa-soa"):
        f0 = ref.initial_state(k, flags, per, 1.0)
        out, _, _, _ = ref.run(k, flags, per, f0, 1000, 1.0, 1e-5)
        verify[k] = {"error_norm": ref.verify(flags, per, out, 1.0, 1e-5),
                     "sha256": golden_io.state_digest(out, flags)}
    f_init = ref.initial_state("aa-soa", flags, per, 1.0)
    arrays["verify_initial_f"] = f_init
    cases.append({"name": "poiseuille_V", "geometry": "box", "dims": [16, 16, 16],
                  "periodic_in": [1, 1, 0], "periodic": list(per), "omega": 1.0,
                  "lambda": 1 / 12, "xforce": 1e-5, "force_on": 1, "steps": 1000,
                  "initial_key": "verify_initial_f", "reference_build": "verify",
                  "verify": verify, "sha256": verify["pull-soa"]["sha256"]})
    print("poiseuille", verify)

    case, _ = run_case(*CONFIG0, arrays=arrays, init="counter")
    cases.append(case)
    print(case["name"], case["sha256"][:16], case["n_fluid"])

    with open(golden_io.CASES_JSON, "w") as fh:
        json.dump(cases, fh, indent=1)
    np.savez_compressed(golden_io.ARRAYS_NPZ, **arrays)


if __name__ == "__main__":
    main()
