"""Failure detection without faulting the GPU: allocation failure is an
error status (the request is refused by cudaMalloc, nothing is launched),
a NaN injected into the host state is caught by the FP64 reduction, and bad
arguments are rejected on the host."""
import numpy as np
import pytest

import lbmb200 as L

pytestmark = pytest.mark.gpu


def test_oversized_lattice_is_an_allocation_error_and_device_stays_usable():
    # 900^3 pull FP64 needs 2 x 19 x 900^3 x 8 B = 222 GB > 180 GB of HBM
    n = 900
    flags = np.ones((n, n, n), dtype=np.int32)
    with pytest.raises(L.LbmError) as e:
        L.Solver(flags, (1, 1, 1), "pull", L.F64)
    assert e.value.code == -3
    del flags
    small, per, _ = L.geometry("channel", (8, 8, 8))
    with L.Solver(small, per, "aa") as s:
        s.run(2)
        s.synchronize()


def test_nan_in_state_is_reported():
    flags, per, _ = L.geometry("channel", (12, 10, 10))
    f0 = L.perturbed_equilibrium(flags, seed=1)
    f0[3, 5, 4, 4] = np.nan
    with L.Solver(flags, per, "aa") as s:
        s.set_state(f0)
        s.run(4)
        with pytest.raises(L.LbmError) as e:
            s.mass_momentum()
        assert e.value.code == -4
        _, bad = s.mass_momentum(check=False)
        assert bad > 0


def test_bad_arguments_are_rejected():
    flags, per, _ = L.geometry("channel", (8, 8, 8))
    with pytest.raises(L.LbmError):
        L.Solver(flags, per, pattern=7)
    with L.Solver(flags, per, "aa") as s:
        with pytest.raises(L.LbmError):
            s.set_params(omega=2.5)
        with pytest.raises(L.LbmError):
            s.run(-1)
        with pytest.raises(L.LbmError):
            s.set_fp16_scale(1024.0)  # not an FP16 solver
    with L.Solver(flags, per, "aa", L.F16) as s:
        with pytest.raises(L.LbmError):
            s.set_fp16_scale(1000.0)  # not a power of two
