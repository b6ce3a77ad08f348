"""lbm_mass_momentum_noalloc: the allocation-free variant of the FP64
mass/momentum reduction, called through the C ABI with buffers the caller
owns (here allocated by torch, standing in for a host application whose
allocator owns the device memory). Its totals must equal the solver's own
lbm_mass_momentum on the same state, on two calls in a row - the second on
a smaller box, so rows left in the shared scratch by the first call would
show if they leaked - and a box larger than the scratch holds must be
rejected with a clear error.

This file is named to be collected last, so a run that stops at the first
failure has already run every other test."""
import ctypes

import numpy as np
import pytest

import lbmb200 as L

pytestmark = pytest.mark.gpu

# same tolerances as the solver's own moment test (test_moments_match_state)
MASS_REL = 1e-14
MOMENTUM_REL, MOMENTUM_ABS = 1e-9, 1e-18


def _state(kind, dims, steps, seed):
    if kind == "porous":
        flags, _, _ = L.porous_channel(dims, 0.2, 3.0, 5.0, seed=seed)
        per = (1, 0, 0)
    else:
        flags, per, _ = L.geometry(kind, dims)
    f0 = L.perturbed_equilibrium(flags, seed=seed, amplitude=1e-3)
    with L.Solver(flags, per, "aa", L.F64) as s:
        s.set_params(1.25, 3 / 16, 1e-6, True)
        s.set_state(f0)
        s.run(steps)
        f = s.get_state()
        totals, bad = s.mass_momentum()
    return flags, f, totals, bad


def _noalloc(f_dev, flags_dev, dims, stream=None):
    nx, ny, nz = dims
    out = np.zeros(4)
    bad = ctypes.c_longlong(-1)
    handle = ctypes.c_void_p(stream.cuda_stream) if stream is not None else None
    rc = L.lib().lbm_mass_momentum_noalloc(
        ctypes.c_void_p(f_dev.data_ptr()), ctypes.c_void_p(flags_dev.data_ptr()), nx, ny, nz,
        out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)), ctypes.byref(bad), handle)
    return rc, out, bad.value


def _check(out, ref, kind):
    assert out[0] == pytest.approx(ref[0], rel=MASS_REL)
    for k in (1, 2, 3):
        assert out[k] == pytest.approx(ref[k], rel=MOMENTUM_REL, abs=MOMENTUM_ABS), (kind, k)


def test_noalloc_reduction_matches_solver_on_two_calls_in_a_row():
    torch = pytest.importorskip("torch")
    assert torch.cuda.is_available()
    cases = [("porous", (48, 40, 36), 7, 3), ("pipe", (20, 22, 18), 3, 4)]
    for kind, dims, steps, seed in cases:
        flags, f, ref, ref_bad = _state(kind, dims, steps, seed)
        f_dev = torch.from_numpy(np.ascontiguousarray(f)).to("cuda")
        flags_dev = torch.from_numpy(np.ascontiguousarray(flags)).to("cuda")
        rc, out, bad = _noalloc(f_dev, flags_dev, dims)
        assert rc == 0, L.lib().lbm_last_error()
        assert bad == 0 and ref_bad == 0
        _check(out, ref, kind)


def test_noalloc_on_caller_stream_and_nonfinite_count():
    """A caller-owned stream, queued behind the caller's own work on it;
    then two fluid cells poisoned with NaN and Inf: the call fills the
    totals, counts both cells and returns LBM_ERR_NONFINITE (-4)."""
    torch = pytest.importorskip("torch")
    dims = (40, 24, 28)
    flags, f, ref, _ = _state("porous", dims, 5, 9)
    stream = torch.cuda.Stream()
    with torch.cuda.stream(stream):
        f_dev = torch.from_numpy(np.ascontiguousarray(f)).to("cuda", non_blocking=False)
        flags_dev = torch.from_numpy(np.ascontiguousarray(flags)).to("cuda")
        scaled = f_dev * 1.0  # work queued on the caller's stream before the call
    rc, out, bad = _noalloc(scaled, flags_dev, dims, stream)
    assert rc == 0, L.lib().lbm_last_error()
    assert bad == 0
    _check(out, ref, "stream")
    fluid = np.argwhere(np.transpose(flags, (2, 1, 0)) != 0)
    (x0, y0, z0), (x1, y1, z1) = fluid[0], fluid[len(fluid) // 2]
    poisoned = scaled.clone()
    poisoned[3, x0, y0, z0] = float("nan")
    poisoned[18, x1, y1, z1] = float("inf")
    torch.cuda.synchronize()
    rc, out, bad = _noalloc(poisoned, flags_dev, dims, stream)
    assert rc == -4  # LBM_ERR_NONFINITE
    assert bad == 2
    assert b"2 fluid cells" in L.lib().lbm_last_error()


def test_noalloc_rejects_host_pointer():
    """f must be device memory of the current device."""
    torch = pytest.importorskip("torch")
    dims = (4, 4, 4)
    f_host = torch.zeros((19,) + dims, dtype=torch.float64)
    flags_dev = torch.ones(dims, dtype=torch.int32, device="cuda")
    rc, _, _ = _noalloc(f_host, flags_dev, dims)
    assert rc == -1
    assert b"must be device memory" in L.lib().lbm_last_error() or \
        b"not a device pointer" in L.lib().lbm_last_error()


def test_noalloc_rejects_box_beyond_scratch():
    torch = pytest.importorskip("torch")
    n = 8193  # one plane more than LBM_NOALLOC_MAX_PLANES
    f_dev = torch.zeros((19, n, 1, 1), dtype=torch.float64, device="cuda")
    flags_dev = torch.ones((1, 1, n), dtype=torch.int32, device="cuda")
    rc, _, _ = _noalloc(f_dev, flags_dev, (n, 1, 1))
    assert rc == -1
    assert b"exceeds the maximum of 8192" in L.lib().lbm_last_error()
