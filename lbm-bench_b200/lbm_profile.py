"""Runs a few steps of the step kernels on a porous channel, for profilers.

    python lbm-bench_b200/lbm_profile.py --size 192 --pattern aa --precision fp64,fp16 --steps 2

Builds the n^3 porous channel of the benchmark (20% solid spheres, r 4-8,
seed 42), and for each precision in turn uploads the seeded initial state,
runs `--steps` steps of the chosen pattern and checks the state is finite.
Launch order per precision: mask_kernel, 19 pack_plane_kernel launches, then
the step kernels (AA alternates even, odd, ...).
"""
import argparse
import os
import sys

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))

import lbmb200 as L  # noqa: E402


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=192)
    ap.add_argument("--pattern", choices=list(L.PATTERNS), default="aa")
    ap.add_argument("--precision", default="fp64",
                    help="comma-separated list of " + ", ".join(L.PRECISIONS))
    ap.add_argument("--steps", type=int, default=6)
    a = ap.parse_args()
    n = a.size
    flags, frac, _ = L.porous_channel((n, n, n), 0.2, 4.0, 8.0, seed=42)
    f0 = L.perturbed_equilibrium(flags, seed=7, amplitude=1e-4)
    for prec in a.precision.split(","):
        with L.Solver(flags, (1, 0, 0), a.pattern, L.PRECISIONS[prec]) as s:
            s.set_params(1.25, 3 / 16, 1e-6, True)
            s.set_state(f0)
            ms = s.run_timed(a.steps)
            _, bad = s.mass_momentum()
            print(f"{n}^3 {a.pattern} {prec}: {s.fluid_cells} fluid cells, {a.steps} steps "
                  f"in {ms:.3f} ms ({s.fluid_cells * a.steps / ms / 1e3:.1f} MLUPS), "
                  f"{s.bytes_per_update:.0f} B/update, nonfinite {bad}")
            if bad:
                raise SystemExit("non-finite populations")


if __name__ == "__main__":
    main()
