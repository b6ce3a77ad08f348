"""The CPU oracle (our C restatement, oracle/lbm_oracle.c) pinned against the
reference: the committed golden fixtures made from LBM-Bench's own kernels,
and, where oracle/_ref was built, the live reference kernels."""
import numpy as np
import pytest

import golden_io
import oracle as O

CASES, _ = golden_io.load()
STEP_CASES = [c for c in CASES if "verify" not in c and "pressure" not in c]
PRESSURE_CASES = [c for c in CASES if "pressure" in c]


def test_velocity_set_tables():
    # inverse map is an involution with c_inv(d) = -c_d, and the weights
    # give the isotropy sums of D3Q19
    for d in range(19):
        e = O.INV[d]
        assert O.INV[e] == d
        assert (O.CX[e], O.CY[e], O.CZ[e]) == (-O.CX[d], -O.CY[d], -O.CZ[d])
    assert abs(O.W.sum() - 1.0) < 1e-15
    assert abs((O.W * O.CX * O.CX).sum() - 1 / 3) < 1e-15
    assert abs((O.W * O.CX).sum()) < 1e-15


@pytest.mark.parametrize("case", STEP_CASES, ids=[c["name"] for c in STEP_CASES])
def test_oracle_matches_golden(oracle, golden, case):
    _, arrays = golden
    flags = golden_io.build_flags(case, arrays)
    f0 = golden_io.initial_state(case, flags)
    out = oracle.run(flags, case["periodic"], f0, case["steps"], case["omega"], case["lambda"],
                     case["xforce"], force_on=bool(case["force_on"]))
    assert golden_io.state_digest(out, flags) == case["sha256"]
    if "state_key" in case:
        ref = arrays[case["state_key"]]
        m = O.fluid_mask(flags)
        assert np.array_equal(out[:, m], ref[:, m])


def test_oracle_poiseuille_golden(oracle, golden):
    cases, arrays = golden
    case = next(c for c in cases if c["name"] == "poiseuille_V")
    flags = golden_io.reference_geometry("box", case["dims"], case["periodic_in"])
    f0 = arrays[case["initial_key"]]
    out = oracle.run(flags, case["periodic"], f0, case["steps"], case["omega"], case["lambda"],
                     case["xforce"], force_on=True)
    assert golden_io.state_digest(out, flags) == case["sha256"]


@pytest.mark.skipif(not O.ref_available("verify"), reason="oracle/_ref not built here")
@pytest.mark.parametrize("steps", [1, 3, 5])
@pytest.mark.parametrize("kernel", ["pull-soa", "push-soa", "pull-aos", "blk-push-soa"])
def test_oracle_vs_live_reference_odd_steps(oracle, kernel, steps):
    ref = O.Reference("verify")
    flags, per, _ = ref.geometry("blocks-3", (13, 11, 9), (0, 0, 0))
    f0 = O.perturbed_state(flags, 99, amp=3e-3)
    out, _, _, _ = ref.run(kernel, flags, per, f0, steps, 1.37, 2e-6)
    mine = oracle.run(flags, per, f0, steps, 1.37, 1 / 12, 2e-6)
    m = O.fluid_mask(flags)
    assert np.array_equal(out[:, m], mine[:, m])


@pytest.mark.skipif(not O.ref_available("plain"), reason="oracle/_ref not built here")
def test_oracle_vs_live_reference_benchmark_build(oracle):
    # the benchmark build (no -DVERIFICATION) applies no body force
    ref = O.Reference("plain")
    flags, per, _ = ref.geometry("pipe", (10, 13, 12), (0, 0, 0))
    f0 = O.perturbed_state(flags, 5, amp=2e-3)
    out, _, it, _ = ref.run("aa-soa", flags, per, f0, 8, 0.9, 1e-5)
    mine = oracle.run(flags, per, f0, 8, 0.9, 1 / 12, 1e-5, force_on=False)
    m = O.fluid_mask(flags)
    assert it == 7
    assert np.array_equal(out[:, m], mine[:, m])


def test_oracle_adjoint_matches_central_differences(oracle):
    flags = golden_io.reference_geometry("channel", (8, 7, 6), (0, 0, 0))
    per = (1, 0, 0)
    f0 = O.perturbed_state(flags, 3, amp=1e-3)
    rng = np.random.default_rng(5)
    por = rng.uniform(0, 1, size=(8, 7, 6)).astype(np.float32)
    steps, om, lam, F, alpha = 25, 1.25, 3 / 16, 1e-5, 0.2
    J, g = oracle.adjoint(flags, per, f0, steps, om, lam, F, alpha, por)
    assert J == pytest.approx(oracle.objective(
        flags, oracle.run_brinkman(flags, per, f0, steps, om, lam, F, alpha, por)), rel=1e-14)
    m = O.fluid_mask(flags)
    assert np.all(g[~m] == 0.0)
    cells = np.argwhere(m)[::7][:6]
    for c in map(tuple, cells):
        a, b = por.copy(), por.copy()
        a[c] += np.float32(1e-3)
        b[c] -= np.float32(1e-3)
        ja = oracle.objective(flags, oracle.run_brinkman(flags, per, f0, steps, om, lam, F,
                                                         alpha, a))
        jb = oracle.objective(flags, oracle.run_brinkman(flags, per, f0, steps, om, lam, F,
                                                         alpha, b))
        fd = (ja - jb) / (float(a[c]) - float(b[c]))
        assert abs(g[c] - fd) <= 1e-5 * abs(fd), (c, g[c], fd)


def test_oracle_brinkman_zero_alpha_is_plain_step(oracle):
    flags = golden_io.reference_geometry("channel", (7, 6, 6), (0, 0, 0))
    f0 = O.perturbed_state(flags, 1)
    por = np.full((7, 6, 6), 0.5, dtype=np.float32)
    a = oracle.run_brinkman(flags, (1, 0, 0), f0, 5, 1.1, 1 / 12, 1e-6, 0.0, por)
    b = oracle.run(flags, (1, 0, 0), f0, 5, 1.1, 1 / 12, 1e-6)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("case", PRESSURE_CASES, ids=[c["name"] for c in PRESSURE_CASES])
def test_oracle_pressure_boundary_matches_golden(oracle, golden, case):
    """Zou-He pressure boundary after every step (src/lbm.c:676-785): the
    oracle gives the reference's pull/push state (golden digest)."""
    _, arrays = golden
    flags = golden_io.build_flags(case, arrays)
    f0 = golden_io.initial_state(case, flags)
    p = case["pressure"]
    out = oracle.run_pressure(flags, case["periodic"], f0, case["steps"], case["omega"],
                              case["lambda"], case["xforce"], bool(case["force_on"]),
                              p["rho_in"], p["rho_out"])
    assert golden_io.state_digest(out, flags) == case["sha256"]


@pytest.mark.skipif(not O.ref_available("verify"), reason="oracle/_ref not built here")
@pytest.mark.parametrize("seed", [1, 2, 3])
@pytest.mark.parametrize("kernel", ["pull-soa", "push-soa"])
def test_oracle_pressure_boundary_vs_live_reference(oracle, kernel, seed):
    rng = np.random.default_rng(seed)
    nx, ny, nz = (int(v) for v in rng.integers(5, 13, size=3))
    flags = np.ones((nz, ny, nx), dtype=np.int32)
    flags[rng.uniform(size=flags.shape) < 0.2] = 0
    flags[:, :, 0] = 2
    flags[:, :, -1] = 4
    flags[:, [0, -1], :] = 0
    flags[[0, -1], :, :] = 0
    f0 = O.perturbed_state(flags, seed, amp=2e-3)
    steps = int(rng.integers(1, 9))
    rho_in, rho_out = 1.0 + 0.01 * rng.uniform(), 1.0 - 0.01 * rng.uniform()
    ref = O.Reference("verify")
    out = ref.run_pressure(kernel, flags, (0, 0, 0), f0, steps, 1.2, 1e-6, rho_in, rho_out)
    mine = oracle.run_pressure(flags, (0, 0, 0), f0, steps, 1.2, 1 / 12, 1e-6, True, rho_in,
                               rho_out)
    m = O.fluid_mask(flags)
    assert np.array_equal(out[:, m], mine[:, m])
