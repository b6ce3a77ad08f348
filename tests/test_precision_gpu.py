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


def _random_walls(rng, dims, per, solid=0.25):
    nx, ny, nz = dims
    flags = (rng.uniform(size=(nz, ny, nx)) > solid).astype(np.int32)
    if not per[0]:
        flags[:, :, [0, -1]] = 0
    if not per[1]:
        flags[:, [0, -1], :] = 0
    if not per[2]:
        flags[[0, -1], :, :] = 0
    return flags


@pytest.mark.parametrize("precision", [L.F32, L.F16])
@pytest.mark.parametrize("per", [(1, 0, 0), (1, 1, 1), (0, 1, 1)])
def test_shuffle_aligned_kernels_equal_generic_pair_kernels(precision, per):
    """For nz a multiple of 64 the shifted patterns run the shuffle-aligned
    two-cell kernels; they move data differently but do the same arithmetic
    as the generic two-cell kernels, so the states must agree bit for bit
    (periodic and walled z, odd and even step counts)."""
    import os
    rng = np.random.default_rng(7)
    dims = (9, 11, 128)
    flags = _random_walls(rng, dims, per)
    f0 = L.perturbed_equilibrium(flags, seed=4, amplitude=2e-3)
    for pattern in ("aa", "pull", "push"):
        outs = []
        for no_shuffle in ("0", "1"):
            os.environ["LBM_B200_NO_SHUFFLE"] = no_shuffle
            try:
                with L.Solver(flags, per, pattern, precision) as s:
                    s.set_params(1.3, 3 / 16, 1e-5, True)
                    s.set_state(f0)
                    s.run(5)
                    outs.append(s.get_state())
            finally:
                os.environ.pop("LBM_B200_NO_SHUFFLE", None)
        assert np.array_equal(outs[0], outs[1]), pattern


@pytest.mark.parametrize("dims", [(9, 11, 128), (7, 6, 13), (5, 8, 30)])
@pytest.mark.parametrize("per", [(1, 0, 0), (1, 1, 1), (0, 1, 1)])
def test_fp16_four_cell_even_kernel_equals_pair_kernel(monkeypatch, dims, per):
    """FP16 AA even steps run the four-cells-per-thread kernel; it collides
    the two pairs with the pair kernel's arithmetic, so the states agree bit
    for bit with LBM_B200_NO_QUAD=1 (ragged nz, walls, force, odd and even
    step counts)."""
    rng = np.random.default_rng(sum(dims))
    flags = _random_walls(rng, dims, per)
    f0 = L.perturbed_equilibrium(flags, seed=5, amplitude=2e-3)
    for steps in (1, 4, 7):
        outs = []
        for no_quad in ("0", "1"):
            monkeypatch.setenv("LBM_B200_NO_QUAD", no_quad)
            with L.Solver(flags, per, "aa", L.F16) as s:
                s.set_params(1.3, 3 / 16, 1e-5, True)
                s.set_state(f0)
                s.run(steps)
                outs.append(s.get_state())
        assert np.array_equal(outs[0], outs[1]), steps


@pytest.mark.parametrize("dims", [(9, 11, 128), (6, 5, 256)])
@pytest.mark.parametrize("per", [(1, 0, 0), (1, 1, 1), (0, 1, 1)])
def test_fp16_four_cell_shifted_kernels_equal_pair_kernels(monkeypatch, dims, per):
    """For nz a multiple of 128 the FP16 pull, push and AA odd steps run the
    four-cells-per-thread shuffle kernel; it collides the two pairs with the
    pair kernels' arithmetic, so the states agree bit for bit with
    LBM_B200_NO_QUAD=1 (the two-cell shuffle kernel): walled and periodic z,
    force, odd and even step counts."""
    rng = np.random.default_rng(sum(dims) + sum(per))
    flags = _random_walls(rng, dims, per, solid=0.3)
    f0 = L.perturbed_equilibrium(flags, seed=6, amplitude=2e-3)
    for pattern in ("aa", "pull", "push"):
        for steps in (1, 4, 7):
            outs = []
            for no_quad in ("0", "1"):
                monkeypatch.setenv("LBM_B200_NO_QUAD", no_quad)
                with L.Solver(flags, per, pattern, L.F16) as s:
                    s.set_params(1.3, 3 / 16, 1e-5, steps != 4)
                    s.set_state(f0)
                    s.run(steps)
                    outs.append(s.get_state())
            assert np.array_equal(outs[0], outs[1]), (pattern, steps)


@pytest.mark.parametrize("per", [(1, 0, 0), (1, 1, 1)])
def test_shuffle_aligned_kernels_track_the_oracle(oracle, per):
    import oracle as O
    rng = np.random.default_rng(11)
    dims = (8, 10, 64)
    flags = _random_walls(rng, dims, per)
    f0 = O.perturbed_state(flags, 3, amp=2e-3)
    ref = oracle.run(flags, per, f0, 7, 1.2, 1 / 12, 1e-5, True)
    m = O.fluid_mask(flags)
    for pattern in ("aa", "pull", "push"):
        with L.Solver(flags, per, pattern, L.F32) as s:
            s.set_params(1.2, 1 / 12, 1e-5, True)
            s.set_state(f0)
            s.run(7)
            out = s.get_state()
        assert np.abs(out[:, m] - ref[:, m]).max() < 1e-6, pattern
