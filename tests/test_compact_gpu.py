"""The compact (fluid-only) layout, lbm_create_compact, on a B200.

FP64 must stay bit-identical to the reference: the golden fixtures made
from LBM-Bench's own kernels (including the 64^3 x 1000-step config-0 case
and the Zou-He pressure cases), the oracle on seeded random geometries with
every combination of periodic axes (a periodic z axis takes the kernel's
wrapped-neighbour path), and the dense layout at full size. FP32/FP16
storage must agree with the dense layout's reduced-precision kernels to
within their own rounding, and the reductions and transfers must give the
same numbers in both layouts.
"""
import numpy as np
import pytest

import golden_io
import lbmb200 as L
import oracle as O

pytestmark = pytest.mark.gpu

CASES, _ = golden_io.load()
STEP_CASES = [c for c in CASES if "verify" not in c and "pressure" not in c]
PRESSURE_CASES = [c for c in CASES if "pressure" in c]
PATTERNS = ["pull", "push", "aa"]


def run(flags, periodic, f0, steps, omega, lam, xforce, force_on, pattern, precision=L.F64,
        compact=True):
    with L.Solver(flags, periodic, pattern, precision, compact=compact) as s:
        assert s.compact == compact
        s.set_params(omega, lam, xforce, force_on)
        s.set_state(f0)
        s.run(steps)
        s.synchronize()
        return s.get_state()


@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("case", STEP_CASES, ids=[c["name"] for c in STEP_CASES])
def test_compact_fp64_bit_identical_to_reference_fixtures(golden, case, pattern):
    _, arrays = golden
    flags = golden_io.build_flags(case, arrays)
    f0 = golden_io.initial_state(case, flags)
    out = run(flags, case["periodic"], f0, case["steps"], case["omega"], case["lambda"],
              case["xforce"], bool(case["force_on"]), pattern)
    assert golden_io.state_digest(out, flags) == case["sha256"]


@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("case", PRESSURE_CASES, ids=[c["name"] for c in PRESSURE_CASES])
def test_compact_pressure_boundary_matches_reference(golden, case, pattern):
    _, arrays = golden
    flags = golden_io.build_flags(case, arrays)
    f0 = golden_io.initial_state(case, flags)
    p = case["pressure"]
    with L.Solver(flags, case["periodic"], pattern, L.F64, compact=True) as s:
        s.set_params(case["omega"], case["lambda"], case["xforce"], bool(case["force_on"]))
        s.set_pressure_bc(p["rho_in"], p["rho_out"])
        s.set_state(f0)
        s.run(case["steps"])
        out = s.get_state()
    assert golden_io.state_digest(out, flags) == case["sha256"]


@pytest.mark.parametrize("seed", range(10))
def test_compact_fp64_bit_identical_to_oracle_random_geometries(oracle, seed):
    """Random obstacles, random periodic axes (all eight combinations over
    the seeds), nz not a multiple of 32 and larger than 32, odd and even step
    counts, force on and off."""
    rng = np.random.default_rng(700 + seed)
    per = ((seed >> 0) & 1, (seed >> 1) & 1, (seed >> 2) & 1) if seed < 8 else (1, 1, 1)
    dims = (int(rng.integers(3, 12)), int(rng.integers(3, 12)), int(rng.integers(5, 70)))
    nx, ny, nz = dims
    flags = (rng.uniform(size=(nz, ny, nx)) > 0.3).astype(np.int32)
    if not per[0]:
        flags[:, :, [0, -1]] = 0
    if not per[1]:
        flags[:, [0, -1], :] = 0
    if not per[2]:
        flags[[0, -1], :, :] = 0
    f0 = O.perturbed_state(flags, seed + 300, amp=5e-3)
    omega = float(rng.uniform(0.6, 1.9))
    steps = int(rng.integers(1, 10))
    force_on = seed % 2 == 0
    ref = oracle.run(flags, per, f0, steps, omega, 3 / 16, 3e-6, force_on)
    m = O.fluid_mask(flags)
    for pattern in PATTERNS:
        out = run(flags, per, f0, steps, omega, 3 / 16, 3e-6, force_on, pattern)
        assert np.array_equal(out[:, m], ref[:, m]), (pattern, per, dims, steps)
        assert np.all(out[:, ~m] == 0.0)


def test_compact_fluid_on_non_periodic_faces(oracle):
    """Fluid on non-periodic faces: the box gets a solid frame, the outside
    acts as a wall, as in the dense layout and the oracle."""
    rng = np.random.default_rng(91)
    flags = (rng.uniform(size=(13, 9, 7)) > 0.2).astype(np.int32)
    per = (0, 1, 0)
    f0 = O.perturbed_state(flags, 4, amp=3e-3)
    ref = oracle.run(flags, per, f0, 5, 1.15, 3 / 16, 2e-6, True)
    m = O.fluid_mask(flags)
    for pattern in PATTERNS:
        out = run(flags, per, f0, 5, 1.15, 3 / 16, 2e-6, True, pattern)
        assert np.array_equal(out[:, m], ref[:, m]), pattern


@pytest.mark.parametrize("precision", [L.F32, L.F16])
@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("dims", [(40, 36, 64), (23, 17, 45)])
def test_compact_reduced_precision_bit_identical_to_dense(pattern, precision, dims):
    """FP32/FP16 storage: the compact layout's pair kernels apply to every
    cell the operations of the dense layout's pair kernels, so the states are
    bit-identical; both stay close to FP64. nz = 45 is odd (a pair with a
    padding cell at the row end) and not a multiple of 32."""
    flags, _, _ = L.porous_channel(dims, 0.2, 3.0, 5.0, seed=8)
    f0 = L.perturbed_equilibrium(flags, seed=3, amplitude=1e-4)
    steps = 24
    c = run(flags, (1, 0, 0), f0, steps, 1.25, 3 / 16, 1e-6, True, pattern, precision)
    d = run(flags, (1, 0, 0), f0, steps, 1.25, 3 / 16, 1e-6, True, pattern, precision,
            compact=False)
    r = run(flags, (1, 0, 0), f0, steps, 1.25, 3 / 16, 1e-6, True, pattern, L.F64)
    m = O.fluid_mask(flags)
    assert np.array_equal(c[:, m], d[:, m])
    tol = 1e-6 if precision == L.F32 else 2e-4
    assert np.abs(c[:, m] - r[:, m]).max() < tol


@pytest.mark.parametrize("precision", [L.F64, L.F32, L.F16])
@pytest.mark.parametrize("per", [(1, 0, 0), (1, 1, 1)])
def test_compact_reduced_precision_random_geometries(oracle, precision, per):
    """Random obstacles with periodic y and z too (the pair kernels'
    wrapped-neighbour path): compact equals dense bit for bit."""
    rng = np.random.default_rng(41 + sum(per))
    nx, ny, nz = 9, 11, 37
    flags = (rng.uniform(size=(nz, ny, nx)) > 0.3).astype(np.int32)
    if not per[1]:
        flags[:, [0, -1], :] = 0
    if not per[2]:
        flags[[0, -1], :, :] = 0
    f0 = O.perturbed_state(flags, 5, amp=2e-3)
    m = O.fluid_mask(flags)
    for pattern in PATTERNS:
        c = run(flags, per, f0, 7, 1.3, 3 / 16, 2e-6, True, pattern, precision)
        d = run(flags, per, f0, 7, 1.3, 3 / 16, 2e-6, True, pattern, precision, compact=False)
        assert np.array_equal(c[:, m], d[:, m]), pattern


@pytest.mark.parametrize("precision", [L.F64, L.F32, L.F16])
def test_compact_split_steps_equal_whole_steps(precision):
    """Steps launched as several x-plane ranges (lbm_step_begin / _planes /
    _end) cover storage ranges that start and end anywhere: the local AA
    even kernel's partial groups at both ends must give the whole step's
    state."""
    flags, _, _ = L.porous_channel((17, 13, 30), 0.25, 2.0, 4.0, seed=6)
    f0 = L.perturbed_equilibrium(flags, seed=2, amplitude=1e-3)
    cuts = [0, 3, 4, 9, 10, 16, 17]
    states = []
    for split in (False, True):
        with L.Solver(flags, (1, 0, 0), "aa", precision, compact=True) as s:
            s.set_params(1.2, 3 / 16, 1e-6, True)
            s.set_state(f0)
            for _ in range(6):
                if split:
                    s.step_begin()
                    for a, b in zip(cuts[:-1], cuts[1:]):
                        s.step_planes(a, b, side=(a % 2 == 1))
                    s.step_end()
                else:
                    s.run(1)
            states.append(s.get_state())
    m = O.fluid_mask(flags)
    assert np.array_equal(states[0][:, m], states[1][:, m])


@pytest.mark.parametrize("split", [False, True], ids=["whole", "split"])
def test_compact_fp16_large_ranges_equal_dense(split):
    """FP16 AA on 1.3 M stored cells, as whole steps and as split steps whose
    plane ranges (one plane, 49, 76) start and end anywhere in the storage
    order and run on two streams: the local even kernel's whole and partial
    groups and the two-cell odd kernel must give the dense layout's state
    bit for bit."""
    flags, _, _ = L.porous_channel((128, 96, 136), 0.2, 3.0, 6.0, seed=12)
    f0 = L.perturbed_equilibrium(flags, seed=4, amplitude=1e-4)
    steps = 8
    d = run(flags, (1, 0, 0), f0, steps, 1.25, 3 / 16, 1e-6, True, "aa", L.F16, compact=False)
    cuts = [0, 1, 50, 51, 127, 128]
    with L.Solver(flags, (1, 0, 0), "aa", L.F16, compact=True) as s:
        assert s.fluid_cells > 1_000_000
        s.set_params(1.25, 3 / 16, 1e-6, True)
        s.set_state(f0)
        for _ in range(steps):
            if split:
                s.step_begin()
                for a, b in zip(cuts[:-1], cuts[1:]):
                    s.step_planes(a, b, side=(b - a > 1))
                s.step_end()
            else:
                s.run(1)
        s.synchronize()
        c = s.get_state()
    m = O.fluid_mask(flags)
    assert np.array_equal(c[:, m], d[:, m])


def test_compact_reductions_and_transfers_equal_dense():
    flags, _, _ = L.porous_channel((48, 40, 72), 0.25, 3.0, 6.0, seed=5)
    f0 = L.perturbed_equilibrium(flags, seed=9, amplitude=1e-3)
    out = {}
    for compact in (False, True):
        with L.Solver(flags, (1, 0, 0), "aa", L.F64, compact=compact) as s:
            s.set_params(1.3, 3 / 16, 1e-6, True)
            s.set_state(f0)
            s.run(7)
            tot, bad = s.mass_momentum()
            mom = s.moments()
            obj = s.objective()
            # the same FP16 run compared against the FP64 state held in each layout
            with L.Solver(flags, (1, 0, 0), "aa", L.F16) as b:
                b.set_params(1.3, 3 / 16, 1e-6, True)
                b.set_state(f0)
                b.run(7)
                cmp = b.compare(s)
            out[compact] = (tot, bad, mom, obj, cmp, s.get_state(), s.device_bytes)
            if compact:
                with L.Solver(flags, (1, 0, 0), "aa", L.F64) as d:
                    d.set_params(1.3, 3 / 16, 1e-6, True)
                    d.set_state(f0)
                    d.run(7)
                    zero = s.compare(d)
    dense, comp = out[False], out[True]
    assert np.array_equal(dense[0], comp[0]) and dense[1] == comp[1] == 0
    for a, b in zip(dense[2], comp[2]):
        assert np.array_equal(a, b)
    assert dense[3] == comp[3]
    assert np.allclose(dense[4], comp[4], rtol=1e-12, atol=0)
    assert zero[0] == 0.0 and zero[2] == 0.0 and zero[4] == 0.0
    assert np.array_equal(dense[5], comp[5])
    assert comp[6] < dense[6]  # no storage for solid cells


@pytest.mark.parametrize("pattern", PATTERNS)
def test_compact_device_initial_state_equals_dense(pattern):
    flags, _, _ = L.porous_channel((20, 18, 40), 0.2, 2.0, 3.0, seed=4)
    states = []
    for compact in (False, True):
        with L.Solver(flags, (1, 0, 0), pattern, L.F64, compact=compact) as s:
            s.init_equilibrium(seed=5, amplitude=1e-4)
            states.append(s.get_state())
    assert np.array_equal(states[0], states[1])


def test_compact_rejects_brinkman_term():
    flags, _, _ = L.geometry("channel", (8, 8, 8))
    with L.Solver(flags, (1, 0, 0), "aa", L.F64, compact=True) as s:
        with pytest.raises(L.LbmError) as e:
            s.set_porosity(np.ones((8, 8, 8), dtype=np.float32), 0.1)
        assert "compact" in str(e.value)


@pytest.mark.slow
def test_compact_full_size_equals_dense_bitwise():
    """The 256^3 porous benchmark workload, 20 steps: compact pull, push and
    AA give the dense layout's FP64 state bit for bit."""
    flags, _, _ = L.porous_channel((256, 256, 256), 0.2, 4.0, 8.0, seed=42)
    f0 = L.perturbed_equilibrium(flags, seed=7, amplitude=1e-4)
    m = O.fluid_mask(flags)
    dense = run(flags, (1, 0, 0), f0, 20, 1.25, 3 / 16, 1e-6, True, "aa", compact=False)
    for pattern in PATTERNS:
        c = run(flags, (1, 0, 0), f0, 20, 1.25, 3 / 16, 1e-6, True, pattern)
        assert np.array_equal(c[:, m], dense[:, m]), pattern
        del c


@pytest.mark.parametrize("precision", [L.F64, L.F32, L.F16])
@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("compact", [False, True], ids=["dense", "compact"])
def test_checkpoint_resume_is_bit_identical(tmp_path, pattern, precision, compact):
    """lbm_save_state after 7 steps (AA: an odd count, so the state is in the
    even-step orientation), then 6 more steps; a fresh solver that loads the
    file and runs the same 6 steps ends in the same state, bit for bit, in
    either layout (the file does not depend on it)."""
    flags, _, _ = L.porous_channel((20, 18, 36), 0.2, 2.0, 4.0, seed=12)
    f0 = L.perturbed_equilibrium(flags, seed=3, amplitude=1e-3)
    path = str(tmp_path / "state.lbm")
    with L.Solver(flags, (1, 0, 0), pattern, precision, compact=compact) as s:
        s.set_params(1.2, 3 / 16, 1e-6, True)
        s.set_state(f0)
        s.run(7)
        s.save_state(path)
        s.run(6)
        want = s.get_state()
    with L.Solver(flags, (1, 0, 0), pattern, precision, compact=not compact) as r:
        r.set_params(1.2, 3 / 16, 1e-6, True)
        r.load_state(path)
        assert r.steps_done == 7
        r.run(6)
        got = r.get_state()
    assert np.array_equal(got, want)


def test_checkpoint_rejects_other_geometry(tmp_path):
    flags, _, _ = L.porous_channel((16, 24, 28), 0.25, 2.0, 3.0, seed=1)
    other, _, _ = L.porous_channel((16, 24, 28), 0.25, 2.0, 3.0, seed=2)
    assert (flags != 0).sum() != (other != 0).sum()
    path = str(tmp_path / "a.lbm")
    with L.Solver(flags, (1, 0, 0), "aa", L.F64) as s:
        s.init_equilibrium(seed=1)
        s.save_state(path)
    with L.Solver(other, (1, 0, 0), "aa", L.F64) as r:
        with pytest.raises(L.LbmError, match="fluid cells"):
            r.load_state(path)
    with L.Solver(flags, (1, 0, 0), "pull", L.F64) as r:
        with pytest.raises(L.LbmError, match="pattern"):
            r.load_state(path)
    bad = tmp_path / "bad.lbm"
    bad.write_bytes(b"not a state file")
    with L.Solver(flags, (1, 0, 0), "aa", L.F64) as r:
        with pytest.raises(L.LbmError, match="not a liblbmb200 state file"):
            r.load_state(str(bad))
