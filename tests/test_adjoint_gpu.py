"""Adjoint of the Brinkman step (lbm_adjoint_gradient) on a B200: against
the oracle's adjoint, independent of the checkpoint interval, against central
finite differences of the FP64 forward model, and FP32 against FP64."""
import numpy as np
import pytest

import lbmb200 as L
import oracle as O

pytestmark = pytest.mark.gpu

OMEGA, LAM, F, ALPHA = 1.25, 3 / 16, 1e-5, 0.2


def _case(dims, seed, solid=True):
    if solid:
        flags, _, _ = L.porous_channel(dims, 0.1, 1.5, 2.5, seed=seed)
    else:
        flags, _, _ = L.geometry("channel", dims)
    rng = np.random.default_rng(seed)
    por = rng.uniform(0, 1, size=dims).astype(np.float32)
    f0 = O.perturbed_state(flags, seed, amp=1e-3)
    return flags, (1, 0, 0), por, f0


def _solver(flags, per, por, f0, precision=L.F64):
    s = L.Solver(flags, per, "aa", precision)
    s.set_params(OMEGA, LAM, F, True)
    s.set_porosity(por, ALPHA)
    s.set_state(f0)
    return s


def _objective(flags, per, por, f0, steps):
    with _solver(flags, per, por, f0) as s:
        s.run(steps)
        return s.objective()


def test_adjoint_matches_oracle(oracle):
    flags, per, por, f0 = _case((12, 9, 10), 3)
    steps = 30
    jr, gr = oracle.adjoint(flags, per, f0, steps, OMEGA, LAM, F, ALPHA, por)
    with _solver(flags, per, por, f0) as s:
        j, g, info = s.adjoint_gradient(steps, checkpoint_every=7)
        back = s.get_state()
    assert j == pytest.approx(jr, rel=1e-12)
    scale = np.abs(gr).max()
    assert scale > 0
    assert np.abs(g - gr).max() <= 1e-9 * scale
    # the solver is left at the initial state
    m = O.fluid_mask(flags)
    assert np.array_equal(back[:, m], f0[:, m])
    assert info["checkpoints"] == 5 and info["interval"] == 7


def test_gradient_independent_of_checkpoint_interval():
    flags, per, por, f0 = _case((16, 12, 12), 5)
    grads = []
    infos = []
    for k in (1, 6, 25, 0, L.CKPT_AUTO):
        with _solver(flags, per, por, f0) as s:
            _, g, info = s.adjoint_gradient(25, checkpoint_every=k)
            grads.append(g)
            infos.append(info)
    # the memory-aware schedule has room for every step's momentum here:
    # one segment, saved by the forward sweep, nothing recomputed
    assert infos[-1]["interval"] == 25 and infos[-1]["checkpoints"] == 1
    for g in grads[1:]:
        assert np.array_equal(g, grads[0])


def test_gradient_matches_central_finite_differences():
    """FP64 central differences, eps = 1e-4 in phi, at seeded fluid cells:
    relative agreement <= 1e-4."""
    flags, per, por, f0 = _case((24, 16, 16), 7, solid=False)
    steps = 120
    with _solver(flags, per, por, f0) as s:
        j0, g, _ = s.adjoint_gradient(steps)
    assert j0 == pytest.approx(_objective(flags, per, por, f0, steps), rel=1e-13)
    rng = np.random.default_rng(11)
    m = O.fluid_mask(flags)
    cells = np.argwhere(m)
    # the most sensitive cells plus random ones
    order = np.argsort(-np.abs(g[m]))
    picks = [tuple(cells[i]) for i in order[:3]]
    picks += [tuple(c) for c in cells[rng.choice(len(cells), 3, replace=False)]]
    eps = np.float32(1e-4)
    for c in picks:
        a, b = por.copy(), por.copy()
        a[c] += eps
        b[c] -= eps
        fd = (_objective(flags, per, a, f0, steps) - _objective(flags, per, b, f0, steps)) / (
            float(a[c]) - float(b[c]))
        if abs(fd) < 1e-6 * np.abs(g).max():
            continue  # below the difference quotient's resolution
        assert abs(g[c] - fd) <= 1e-4 * abs(fd), (c, g[c], fd)


def test_fp32_adjoint_tracks_fp64():
    flags, per, por, f0 = _case((32, 24, 24), 9)
    grads = {}
    for prec in (L.F64, L.F32):
        with _solver(flags, per, por, f0, prec) as s:
            _, grads[prec], _ = s.adjoint_gradient(100)
    g64, g32 = grads[L.F64], grads[L.F32]
    rel = np.linalg.norm(g32 - g64) / np.linalg.norm(g64)
    assert rel < 1e-3, rel


def test_adjoint_argument_errors():
    flags, per, por, f0 = _case((8, 8, 8), 1, solid=False)
    with L.Solver(flags, per, "aa", L.F64) as s:
        s.set_state(f0)
        with pytest.raises(L.LbmError):
            s.adjoint_gradient(10)  # no porosity field
    with L.Solver(flags, per, "pull", L.F64) as s:
        s.set_porosity(por, ALPHA)
        with pytest.raises(L.LbmError):
            s.adjoint_gradient(10)  # AA only
