"""The first two benchmark configurations at their stated sizes, against
LBM-Bench's own kernels.

Config 0: a 64^3 channel (x periodic, obstacle walls on the y and z faces),
omega 1.25, Lambda 3/16, body force F_x = 1e-6, the seeded +-1e-4
equilibrium of the benchmark, 1000 steps, FP64. The committed fixture
`config0_channel64` holds the SHA-256 of the final state on which the
reference's pull-soa, push-soa and aa-soa agree bit for bit (LBM-Bench's
sources built with Lambda 3/16, tests/golden/make_golden.py). The GPU's
pull, push and AA must reproduce that digest. Where the reference build
travels with the repository (oracle/_ref), its pull-soa also runs here on
the host cores and the normwise relative density and velocity errors of
every GPU pattern are computed and checked against the stated 1e-12 bound
(they are 0).

Config 1: the 256^3 porous channel of the benchmark (20% solid spheres,
r 4-8, seed 42). The reference's strict pull-soa runs 10 steps on the host
(about 10 GB of host memory); the GPU's FP64 AA, pull and push states after
10 steps must equal it bit for bit.
"""
import numpy as np
import pytest

import golden_io
import lbmb200 as L
import oracle as O

pytestmark = pytest.mark.gpu

PATTERNS = ["aa", "pull", "push"]
BOUND = 1e-12  # normwise relative rho and u error allowed against the reference


def _case(name):
    cases, _ = golden_io.load()
    return next(c for c in cases if c["name"] == name)


def _gpu_state(flags, periodic, f0, steps, pattern, omega=1.25, lam=3 / 16, xforce=1e-6):
    with L.Solver(flags, periodic, pattern, L.F64) as s:
        s.set_params(omega, lam, xforce, True)
        s.set_state(f0)
        s.run(steps)
        s.synchronize()
        out = s.get_state()
        _, bad = s.mass_momentum(check=False)
    assert bad == 0
    return out


@pytest.fixture(scope="module")
def config0():
    case = _case("config0_channel64")
    flags = golden_io.build_flags(case, None)
    f0 = golden_io.initial_state(case, flags)
    # the product's own generator gives the same initial state
    assert np.array_equal(f0, L.perturbed_equilibrium(flags, seed=case["seed"],
                                                      amplitude=case["amp"]))
    outs = {p: _gpu_state(flags, case["periodic"], f0, case["steps"], p) for p in PATTERNS}
    return case, flags, f0, outs


def test_config0_case_is_the_stated_one(config0):
    case, flags, _, _ = config0
    assert case["dims"] == [64, 64, 64] and case["steps"] == 1000
    assert (case["omega"], case["lambda"], case["xforce"]) == (1.25, 3 / 16, 1e-6)
    assert case["init"] == "counter" and case["amp"] == 1e-4
    assert set(case["kernels_agreeing"]) == {"pull-soa", "push-soa", "aa-soa"}
    assert case["n_fluid"] == 64 * 62 * 62 == int((flags != 0).sum())


@pytest.mark.parametrize("pattern", PATTERNS)
def test_config0_bit_identical_to_reference_digest(config0, pattern):
    case, flags, _, outs = config0
    assert golden_io.state_digest(outs[pattern], flags) == case["sha256"]
    rho, ux, uy, uz = O.moments(outs[pattern], flags)
    m = O.fluid_mask(flags)
    vel = [a[m] / rho[m] for a in (ux, uy, uz)]
    # the norms the fixture records (summation order may differ between BLAS builds)
    assert float(np.linalg.norm(rho[m])) == pytest.approx(case["norms"]["rho_l2"], rel=1e-13)
    assert float(np.sqrt(sum(float((v * v).sum()) for v in vel))) == \
        pytest.approx(case["norms"]["u_l2"], rel=1e-13)


@pytest.mark.slow
@pytest.mark.skipif(not O.ref_available("verify_l316"),
                    reason="the reference build (oracle/_ref) is not present")
def test_config0_normwise_error_against_live_reference(config0):
    case, flags, f0, outs = config0
    ref = O.Reference("verify_l316")
    r, _, _, _ = ref.run("pull-soa", flags, case["periodic"], f0, case["steps"], case["omega"],
                         case["xforce"])
    assert golden_io.state_digest(r, flags) == case["sha256"]
    for pattern in PATTERNS:
        e_rho, e_u = O.normwise_errors(outs[pattern], r, flags)
        assert e_rho <= BOUND and e_u <= BOUND, (pattern, e_rho, e_u)
        assert e_rho == 0.0 and e_u == 0.0, (pattern, e_rho, e_u)


@pytest.mark.slow
@pytest.mark.skipif(not O.ref_available("verify_l316"),
                    reason="the reference build (oracle/_ref) is not present")
def test_config1_porous256_against_live_reference():
    flags, frac, nsph = L.porous_channel((256, 256, 256), 0.2, 4.0, 8.0, seed=42)
    assert 0.2 <= frac < 0.201
    f0 = L.perturbed_equilibrium(flags, seed=7, amplitude=1e-4)
    steps = 10
    ref = O.Reference("verify_l316")
    r, _, _, _ = ref.run("pull-soa", flags, (1, 0, 0), f0, steps, 1.25, 1e-6)
    m = O.fluid_mask(flags)
    for pattern in PATTERNS:
        g = _gpu_state(flags, (1, 0, 0), f0, steps, pattern)
        e_rho, e_u = O.normwise_errors(g, r, flags)
        assert e_rho <= BOUND and e_u <= BOUND, (pattern, e_rho, e_u)
        assert np.array_equal(g[:, m], r[:, m]), pattern
        del g
