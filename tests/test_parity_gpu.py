"""Parity of the CUDA kernels (liblbmb200) with the reference, on a B200.

FP64 results must be bit-identical: to the golden fixtures made from
LBM-Bench's own pull/push/AA kernels, and to the oracle restatement on
seeded random cases. At full size (256^3 porous channel) parity is checked
through properties that do not need the CPU: the three propagation patterns
agree bit for bit, mass is conserved, and the body force adds exactly
F * n_fluid of x momentum per step in a periodic box.
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


def gpu_run(flags, periodic, f0, steps, omega, lam, xforce, force_on, pattern,
            precision=L.F64):
    with L.Solver(flags, periodic, pattern, precision) as s:
        s.set_params(omega, lam, xforce, force_on)
        s.set_state(f0)
        s.run(steps)
        s.synchronize()
        return s.get_state()


@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("case", STEP_CASES, ids=[c["name"] for c in STEP_CASES])
def test_fp64_bit_identical_to_reference_fixtures(golden, case, pattern):
    _, arrays = golden
    flags = golden_io.build_flags(case, arrays)
    f0 = golden_io.initial_state(case, flags)
    out = gpu_run(flags, case["periodic"], f0, case["steps"], case["omega"], case["lambda"],
                  case["xforce"], bool(case["force_on"]), pattern)
    assert golden_io.state_digest(out, flags) == case["sha256"]


@pytest.mark.parametrize("pattern", PATTERNS)
def test_poiseuille_verification_run_matches_reference(golden, pattern):
    cases, arrays = golden
    case = next(c for c in cases if c["name"] == "poiseuille_V")
    flags = golden_io.reference_geometry("box", case["dims"], case["periodic_in"])
    f0 = arrays[case["initial_key"]]
    out = gpu_run(flags, case["periodic"], f0, case["steps"], 1.0, 1 / 12, 1e-5, True, pattern)
    assert golden_io.state_digest(out, flags) == case["sha256"]


def _random_case(seed):
    rng = np.random.default_rng(seed)
    dims = tuple(int(v) for v in rng.integers(5, 23, size=3))
    per = tuple(int(v) for v in rng.integers(0, 2, size=3))
    nx, ny, nz = dims
    flags = (rng.uniform(size=(nz, ny, nx)) > 0.25).astype(np.int32)
    # non-periodic faces are obstacle cells, as in every reference geometry
    if not per[0]:
        flags[:, :, [0, -1]] = 0
    if not per[1]:
        flags[:, [0, -1], :] = 0
    if not per[2]:
        flags[[0, -1], :, :] = 0
    return flags, per, rng


@pytest.mark.parametrize("seed", range(8))
def test_fp64_bit_identical_to_oracle_random_geometries(oracle, seed):
    flags, per, rng = _random_case(seed)
    f0 = O.perturbed_state(flags, seed + 100, amp=5e-3)
    omega = float(rng.uniform(0.6, 1.9))
    lam = [1 / 12, 3 / 16, 0.25][seed % 3]
    steps = int(rng.integers(1, 12))
    force_on = bool(seed % 2 == 0)
    ref = oracle.run(flags, per, f0, steps, omega, lam, 3e-6, force_on)
    m = O.fluid_mask(flags)
    for pattern in PATTERNS:
        out = gpu_run(flags, per, f0, steps, omega, lam, 3e-6, force_on, pattern)
        assert np.array_equal(out[:, m], ref[:, m]), pattern
        assert np.all(out[:, ~m] == 0.0)


@pytest.mark.parametrize("seed", range(4))
def test_fluid_on_non_periodic_faces_bounces_off_the_box(oracle, seed):
    """Flags with fluid on non-periodic faces (which the reference's own
    geometries never produce): the outside acts as a wall, as in the oracle."""
    rng = np.random.default_rng(50 + seed)
    dims = tuple(int(v) for v in rng.integers(4, 15, size=3))
    per = tuple(int(v) for v in rng.integers(0, 2, size=3))
    nx, ny, nz = dims
    flags = (rng.uniform(size=(nz, ny, nx)) > 0.2).astype(np.int32)
    f0 = O.perturbed_state(flags, seed, amp=3e-3)
    ref = oracle.run(flags, per, f0, 6, 1.15, 3 / 16, 2e-6, True)
    m = O.fluid_mask(flags)
    for pattern in PATTERNS:
        out = gpu_run(flags, per, f0, 6, 1.15, 3 / 16, 2e-6, True, pattern)
        assert np.array_equal(out[:, m], ref[:, m]), pattern
        lp = gpu_run(flags, per, f0, 6, 1.15, 3 / 16, 2e-6, True, pattern, L.F32)
        assert np.abs(lp[:, m] - ref[:, m]).max() < 1e-6, pattern


def test_unaligned_z_extent_and_single_cell_rows(oracle):
    # nz = 3 (well below one sector of pitch) and nx = 1 periodic
    for dims, per in (((9, 7, 3), (1, 0, 1)), ((1, 6, 33), (1, 0, 0)), ((5, 1, 40), (0, 1, 0))):
        nx, ny, nz = dims
        flags = np.ones((nz, ny, nx), dtype=np.int32)
        if not per[1]:
            flags[:, [0, -1], :] = 0
        if not per[2]:
            flags[[0, -1], :, :] = 0
        if not per[0]:
            flags[:, :, [0, -1]] = 0
        f0 = O.perturbed_state(flags, 3, amp=1e-3)
        ref = oracle.run(flags, per, f0, 5, 1.3, 3 / 16, 1e-6, True)
        m = O.fluid_mask(flags)
        for pattern in PATTERNS:
            out = gpu_run(flags, per, f0, 5, 1.3, 3 / 16, 1e-6, True, pattern)
            assert np.array_equal(out[:, m], ref[:, m]), (dims, pattern)


@pytest.mark.parametrize("pattern", PATTERNS)
def test_state_round_trip_is_exact(pattern):
    flags, per, _ = L.geometry("blocks-3", (20, 17, 15))
    f0 = L.perturbed_equilibrium(flags, seed=2, amplitude=1e-3)
    with L.Solver(flags, per, pattern) as s:
        s.set_state(f0)
        assert np.array_equal(s.get_state(), f0)
        s.set_params(1.2, 3 / 16, 1e-6, True)
        s.run(3)  # AA: odd count leaves the even-step orientation
        a = s.get_state()
        s.set_state(a)
        assert np.array_equal(s.get_state(), a)


def test_moments_match_state():
    flags, per, _ = L.geometry("pipe", (12, 14, 13))
    f0 = L.perturbed_equilibrium(flags, seed=9, amplitude=2e-3)
    with L.Solver(flags, per, "aa") as s:
        s.set_params(1.1, 1 / 12, 1e-6, True)
        s.set_state(f0)
        s.run(7)
        f = s.get_state()
        rho, ux, uy, uz = s.moments()
        tot, bad = s.mass_momentum()
    r2, x2, y2, z2 = O.moments(f, flags)
    for a, b in ((rho, r2), (ux, x2), (uy, y2), (uz, z2)):
        assert np.allclose(a, b, rtol=0, atol=1e-15)
    assert bad == 0
    m = O.fluid_mask(flags)
    assert tot[0] == pytest.approx(r2[m].sum(), rel=1e-14)
    assert tot[1] == pytest.approx(x2[m].sum(), rel=1e-9, abs=1e-18)


@pytest.fixture(scope="module")
def porous256():
    flags, frac, n = L.porous_channel((256, 256, 256), 0.2, 4.0, 8.0, seed=42)
    f0 = L.perturbed_equilibrium(flags, seed=7, amplitude=1e-4)
    return flags, f0


@pytest.mark.slow
def test_full_size_patterns_agree_bitwise(porous256):
    """256^3 porous channel (20% solid, r 4-8): pull, push and AA give the
    same FP64 state after 20 steps, and the state is finite."""
    flags, f0 = porous256
    outs = {}
    for pattern in PATTERNS:
        with L.Solver(flags, (1, 0, 0), pattern) as s:
            s.set_params(1.25, 3 / 16, 1e-6, True)
            s.set_state(f0)
            s.run(20)
            tot, bad = s.mass_momentum()
            assert bad == 0
            outs[pattern] = s.get_state()
    m = O.fluid_mask(flags)
    assert np.array_equal(outs["pull"][:, m], outs["push"][:, m])
    assert np.array_equal(outs["pull"][:, m], outs["aa"][:, m])


@pytest.mark.slow
@pytest.mark.parametrize("pattern", PATTERNS)
def test_full_size_conservation_in_periodic_box(pattern):
    """256^3 fully periodic fluid, no walls: each step conserves mass and the
    Luo force adds exactly F of x momentum per cell (sum_d 3 w_d c_dx^2 = 1)."""
    n = 256
    flags, per, _ = L.geometry("fluid", (n, n, n))
    f0 = L.perturbed_equilibrium(flags, seed=1, amplitude=1e-3)
    F, steps = 1e-6, 40
    with L.Solver(flags, per, pattern) as s:
        s.set_params(1.3, 3 / 16, F, True)
        s.set_state(f0)
        t0, _ = s.mass_momentum()
        s.run(steps)
        t1, bad = s.mass_momentum()
    cells = n ** 3
    assert bad == 0
    assert abs(t1[0] - t0[0]) <= 1e-12 * t0[0]
    assert t1[1] - t0[1] == pytest.approx(F * cells * steps, rel=1e-9)
    assert abs(t1[2] - t0[2]) < 1e-9 and abs(t1[3] - t0[3]) < 1e-9


@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("precision", [L.F64, L.F16])
def test_device_initial_state_equals_host_generator(pattern, precision):
    flags, frac, _ = L.porous_channel((20, 18, 16), 0.2, 2.0, 3.0, seed=4)
    f0 = L.perturbed_equilibrium(flags, seed=77, amplitude=1e-3)
    with L.Solver(flags, (1, 0, 0), pattern, precision) as a, \
            L.Solver(flags, (1, 0, 0), pattern, precision) as b:
        a.set_state(f0)
        b.init_equilibrium(seed=77, amplitude=1e-3)
        assert np.array_equal(a.get_state(), b.get_state())


@pytest.mark.parametrize("shape", [(None, None, "2"), ("1", "2", "1"), ("3", "6", "3"),
                                   ("2", "8", "2"), ("1", "4", "2")])
@pytest.mark.parametrize("seed", [1, 4, 6])
def test_pipelined_and_plain_fp64_kernels_agree(oracle, monkeypatch, seed, shape):
    """The bulk-copy pipelined FP64 kernels (LBM_B200_TMA=1) and the plain
    ones give the oracle's state bit for bit, for any tile height, pipeline
    depth and number of consumer groups."""
    flags, per, rng = _random_case(seed)
    f0 = O.perturbed_state(flags, seed, amp=4e-3)
    ref = oracle.run(flags, per, f0, 7, 1.3, 3 / 16, 2e-6, True)
    m = O.fluid_mask(flags)
    if shape[0]:
        monkeypatch.setenv("LBM_B200_TMA_T", shape[0])
        monkeypatch.setenv("LBM_B200_TMA_STAGES", shape[1])
    monkeypatch.setenv("LBM_B200_TMA_GROUPS", shape[2])
    for tma in ("1", "0"):
        monkeypatch.setenv("LBM_B200_TMA", tma)
        for pattern in PATTERNS:
            out = gpu_run(flags, per, f0, 7, 1.3, 3 / 16, 2e-6, True, pattern)
            assert np.array_equal(out[:, m], ref[:, m]), (tma, pattern)


@pytest.mark.parametrize("groups", ["1", "2", "3"])
@pytest.mark.parametrize("pattern", PATTERNS)
def test_pipelined_kernels_full_size(porous256, monkeypatch, pattern, groups):
    """256^3 porous channel, hundreds of tiles per CTA: the pipelined FP64
    kernels give the plain kernels' state bit for bit after 10 steps, with
    1, 2 and 3 consumer groups."""
    flags, f0 = porous256
    outs = {}
    monkeypatch.setenv("LBM_B200_TMA_GROUPS", groups)
    for tma in ("0", "1"):
        monkeypatch.setenv("LBM_B200_TMA", tma)
        with L.Solver(flags, (1, 0, 0), pattern) as s:
            s.set_params(1.25, 3 / 16, 1e-6, True)
            s.set_state(f0)
            s.run(10)
            s.synchronize()
            outs[tma] = s.get_state()
    m = O.fluid_mask(flags)
    assert np.array_equal(outs["0"][:, m], outs["1"][:, m])


# ---------------------------------------------------------------------------
# Zou-He pressure boundary (src/lbm.c:676-785)
# ---------------------------------------------------------------------------

def _inlet_outlet(dims, solid, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    flags = np.ones((nz, ny, nx), dtype=np.int32)
    flags[rng.uniform(size=flags.shape) < solid] = 0
    flags[:, :, 0] = 2
    flags[:, :, -1] = 4
    flags[:, [0, -1], :] = 0
    flags[[0, -1], :, :] = 0
    return flags


def _pressure_run(flags, f0, steps, omega, lam, xforce, force_on, rho_in, rho_out, pattern,
                  precision=L.F64):
    with L.Solver(flags, (0, 0, 0), pattern, precision) as s:
        s.set_params(omega, lam, xforce, force_on)
        s.set_pressure_bc(rho_in, rho_out)
        s.set_state(f0)
        s.run(steps)
        s.synchronize()
        return s.get_state(), s.mass_momentum()[0]


@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("case", PRESSURE_CASES, ids=[c["name"] for c in PRESSURE_CASES])
def test_pressure_boundary_bit_identical_to_reference_fixtures(golden, case, pattern):
    """The reference's pull and push kernels each followed by its Zou-He
    pass give the golden digest; every pattern here must reproduce it (AA
    too: the boundary follows each of its steps)."""
    _, arrays = golden
    flags = golden_io.build_flags(case, arrays)
    f0 = golden_io.initial_state(case, flags)
    p = case["pressure"]
    out, _ = _pressure_run(flags, f0, case["steps"], case["omega"], case["lambda"],
                           case["xforce"], bool(case["force_on"]), p["rho_in"], p["rho_out"],
                           pattern)
    assert golden_io.state_digest(out, flags) == case["sha256"]


@pytest.mark.parametrize("seed", range(4))
def test_pressure_boundary_bit_identical_to_oracle(oracle, seed):
    rng = np.random.default_rng(200 + seed)
    dims = tuple(int(v) for v in rng.integers(5, 16, size=3))
    flags = _inlet_outlet(dims, 0.2, seed)
    f0 = O.perturbed_state(flags, seed, amp=2e-3)
    steps = int(rng.integers(1, 12))
    rho_in, rho_out = 1.0 + 0.01 * rng.uniform(), 1.0 - 0.01 * rng.uniform()
    ref = oracle.run_pressure(flags, (0, 0, 0), f0, steps, 1.3, 3 / 16, 1e-6, True, rho_in,
                              rho_out)
    m = O.fluid_mask(flags)
    for pattern in PATTERNS:
        out, _ = _pressure_run(flags, f0, steps, 1.3, 3 / 16, 1e-6, True, rho_in, rho_out,
                               pattern)
        assert np.array_equal(out[:, m], ref[:, m]), pattern


@pytest.mark.parametrize("precision,tol", [(L.F32, 1e-5), (L.F16, 2e-3)])
def test_pressure_boundary_reduced_precision(precision, tol):
    """A pressure-driven channel (64 cells long, rho 1.01 -> 0.99) with the
    boundary in FP32/FP16 storage tracks FP64, and the flow goes from the
    high-pressure inlet to the outlet."""
    flags = _inlet_outlet((64, 18, 20), 0.0, 1)
    f0 = L.perturbed_equilibrium(flags, seed=3, amplitude=1e-4)
    a, ta = _pressure_run(flags, f0, 400, 1.25, 3 / 16, 0.0, False, 1.01, 0.99, "aa")
    b, tb = _pressure_run(flags, f0, 400, 1.25, 3 / 16, 0.0, False, 1.01, 0.99, "aa", precision)
    r2, x2, _, _ = O.moments(a, flags)
    r3, x3, _, _ = O.moments(b, flags)
    m = O.fluid_mask(flags)
    assert ta[1] > 0.0  # x momentum from inlet to outlet
    assert np.linalg.norm(x3[m] - x2[m]) <= tol * np.linalg.norm(x2[m])
    # density drops from inlet to outlet
    assert r2[1][m[1]].mean() > r2[-2][m[-2]].mean()


def test_pressure_boundary_argument_errors():
    flags, per, _ = L.geometry("channel", (10, 8, 8))
    with L.Solver(flags, per, "aa") as s:
        with pytest.raises(L.LbmError):
            s.set_pressure_bc(1.01, 0.99)  # no inlet/outlet cells
        s.set_pressure_bc(1.0, 1.0, on=False)
    flags = _inlet_outlet((10, 8, 8), 0.0, 2)
    with L.Solver(flags, (0, 0, 0), "aa") as s:
        with pytest.raises(L.LbmError):
            s.set_pressure_bc(-1.0, 0.99)
        s.set_pressure_bc(1.01, 0.99)
        s.run(2)
        s.synchronize()
