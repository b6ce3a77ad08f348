"""Reduced-precision paths (FP32 arithmetic on shifted populations f - w,
stored as FP32 or scaled FP16) against the FP64 path of the same seed, on
a B200. Tolerances are written per test; the headline target is an L2
relative velocity error <= 1e-3 for FP16 storage."""
import numpy as np
import pytest

import lbmb200 as L

pytestmark = pytest.mark.gpu


def errors(a: L.Solver, b: L.Solver):
    """(L2 relative error of u, L2 relative error of rho, max abs u error)."""
    d = a.compare(b)
    return np.sqrt(d[0] / d[1]), np.sqrt(d[2] / d[3]), d[4]


@pytest.fixture(scope="module")
def porous64():
    flags, frac, _ = L.porous_channel((64, 64, 64), 0.2, 4.0, 8.0, seed=5)
    f0 = L.perturbed_equilibrium(flags, seed=6, amplitude=1e-4)
    return flags, f0


@pytest.mark.parametrize("pattern", ["aa", "pull", "push"])
@pytest.mark.parametrize("precision,tol_u,tol_rho", [(L.F32, 1e-5, 1e-7), (L.F16, 1e-3, 1e-5)])
def test_reduced_precision_error_vs_fp64(porous64, pattern, precision, tol_u, tol_rho):
    flags, f0 = porous64
    with L.Solver(flags, (1, 0, 0), pattern, L.F64) as ref, \
            L.Solver(flags, (1, 0, 0), pattern, precision) as lp:
        for s in (ref, lp):
            s.set_params(1.25, 3 / 16, 1e-6, True)
            s.set_state(f0)
            s.run(300)
        eu, erho, _ = errors(lp, ref)
        _, bad = lp.mass_momentum()
    assert bad == 0
    assert eu <= tol_u, eu
    assert erho <= tol_rho, erho


def test_fp16_state_round_trip_bound():
    flags, per, _ = L.geometry("channel", (16, 16, 16))
    f0 = L.perturbed_equilibrium(flags, seed=3, amplitude=1e-2)
    w = np.array([1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4
                 + [1 / 3])
    with L.Solver(flags, per, "aa", L.F16) as s:
        s.set_state(f0)
        back = s.get_state()
    m = np.transpose(flags, (2, 1, 0)) != 0
    g = f0[:, m] - w[:, None]
    err = np.abs(back[:, m] - f0[:, m])
    # round-to-nearest FP16 of the scaled deviation: relative 2^-11 (normal
    # range) or half a subnormal step (2^-25 / scale) absolute
    bound = np.maximum(np.abs(g) * 2.0 ** -11, 2.0 ** -25 / 16384) * (1 + 1e-3)
    assert np.all(err <= bound)


def test_fp32_bytes_and_steps_per_launch():
    flags, per, _ = L.geometry("channel", (8, 8, 8))
    for prec, size in ((L.F64, 8), (L.F32, 4), (L.F16, 2)):
        with L.Solver(flags, per, "aa", prec) as s:
            assert s.bytes_per_update == 2 * 19 * size
            s.run(5)
            s.synchronize()
            assert s.launch_count == 5 and s.steps_done == 5
