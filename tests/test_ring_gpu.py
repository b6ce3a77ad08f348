"""Native slab ring (lbm_ring_* in include/lbm_b200.h) on a B200.

One slab that is its own neighbour on both sides (an x-periodic domain in a
single slab) is stepped through lbm_ring_run and must reproduce the
undecomposed x-periodic solver bit for bit - with the messages moved by
device copies and by a one-rank NCCL communicator (send and receive to
itself), with and without the overlapped schedule, in every pattern,
precision and layout. Failure detection runs on the host: a two-rank
communicator whose second rank never joins must time out with
LBM_ERR_TIMEOUT, the communicator aborted and the GPU context still usable;
no kernel is in flight while it waits, and it runs in a child process under
a hard time limit."""
import os
import subprocess
import sys

import numpy as np
import pytest

import lbm_slab
import lbmb200 as L
import oracle as O

pytestmark = pytest.mark.gpu

PKG = os.path.dirname(os.path.abspath(L.__file__))


def _domain(dims, seed):
    flags, _, _ = L.porous_channel(dims, 0.2, 1.5, 3.0, seed=seed)
    f0 = L.perturbed_equilibrium(flags, seed=seed, amplitude=1e-3)
    return flags, f0


def _params(s):
    s.set_params(1.25, 3 / 16, 1e-5, True)


def _single(flags, f0, pattern, precision, steps):
    with L.Solver(flags, (1, 0, 0), pattern, precision) as s:
        _params(s)
        s.set_state(f0)
        s.run(steps)
        return s.get_state()


def _slab_of_all(flags, f0, pattern, precision, compact):
    s = L.Solver.slab(lbm_slab.slab_flags(flags, 0, flags.shape[2]), (0, 0), pattern, precision,
                      compact=compact)
    _params(s)
    s.set_state(f0)
    return s


CASES = [(L.F64, False), (L.F32, False), (L.F16, False), (L.F64, True), (L.F16, True)]


@pytest.mark.parametrize("overlap", [False, True], ids=["serial", "overlap"])
@pytest.mark.parametrize("compact", [False, True], ids=["dense", "compact"])
@pytest.mark.parametrize("precision,nccl", CASES,
                         ids=[f"{p}-{'nccl' if n else 'copy'}" for p, n in CASES])
@pytest.mark.parametrize("pattern", ["pull", "push", "aa"])
def test_ring_of_one_equals_undecomposed(pattern, precision, nccl, compact, overlap):
    flags, f0 = _domain((23, 14, 12), 5)
    steps = 9
    ref = _single(flags, f0, pattern, precision, steps)
    s = _slab_of_all(flags, f0, pattern, precision, compact)
    runner = lbm_slab.NativeRunner(s, overlap=overlap, nccl=nccl, timeout_ms=30000)
    assert runner.uses_nccl == nccl
    runner.scatter()
    runner.run(steps)
    runner.gather()
    runner.synchronize()
    assert runner.exchanges >= (steps if pattern != "aa" else 2 * (steps // 2))
    got = s.get_state()
    assert s.steps_done == steps
    runner.close()
    s.close()
    m = O.fluid_mask(flags)
    assert np.array_equal(got[:, m], ref[:, m])


def test_ring_runs_in_windows_across_many_steps():
    """More steps than the run loop keeps queued (two windows of 16): the
    bounded window waits pass and the result stays exact."""
    flags, f0 = _domain((16, 10, 32), 9)
    steps = 70
    ref = _single(flags, f0, "aa", L.F64, steps)
    s = _slab_of_all(flags, f0, "aa", L.F64, True)
    with L.SlabRing(s, 0, 1, L.ring_unique_id(), 30000) as ring:
        ring.scatter()
        for chunk in (33, 37):
            ring.run(chunk, overlap=True)
        ring.gather()
        ring.synchronize()
        got = s.get_state()
    s.close()
    m = O.fluid_mask(flags)
    assert np.array_equal(got[:, m], ref[:, m])


def test_ring_rejects_bad_arguments():
    flags, f0 = _domain((12, 8, 8), 3)
    with L.Solver(flags, (1, 0, 0), "aa", L.F64) as s:
        with pytest.raises(L.LbmError) as e:
            L.SlabRing(s)
        assert e.value.code == -1 and "not a slab" in str(e.value)
    s = _slab_of_all(flags, f0, "aa", L.F64, False)
    with pytest.raises(L.LbmError) as e:
        L.SlabRing(s, 0, 2, None)
    assert e.value.code == -1
    with pytest.raises(L.LbmError) as e:
        L.SlabRing(s, 2, 2, L.ring_unique_id())
    assert e.value.code == -1
    s.close()


_NEVER_JOINS = r"""
import sys, time
sys.path.insert(0, sys.argv[1])
import numpy as np
import lbm_slab
import lbmb200 as L
flags, _, _ = L.porous_channel((12, 8, 8), 0.2, 1.5, 3.0, seed=3)
s = L.Solver.slab(lbm_slab.slab_flags(flags, 0, 12), (0, 0), "aa", L.F64)
s.set_params(1.25, 3 / 16, 1e-5, True)
s.init_equilibrium(seed=1, amplitude=1e-4)
t0 = time.monotonic()
try:
    L.SlabRing(s, 0, 2, L.ring_unique_id(), 3000)
    print("no error")
    sys.exit(1)
except L.LbmError as e:
    waited = time.monotonic() - t0
    print("code", e.code, "waited", round(waited, 2), str(e))
    assert e.code == L.ERR_TIMEOUT and "aborted" in str(e), e
    assert 2.5 < waited < 30, waited
s.run(2)
s.synchronize()
tot, bad = s.mass_momentum()
assert bad == 0
s.close()
print("timeout ok")
"""


def test_ring_creation_times_out_when_a_rank_never_joins():
    """Rank 1 of a two-rank ring never calls lbm_ring_create: rank 0's
    bounded wait runs out after 3 s, the communicator is aborted, the call
    returns LBM_ERR_TIMEOUT, and the solver still steps. No kernel is in
    flight during the wait; the child process has a hard limit."""
    env = dict(os.environ, NCCL_NVLS_ENABLE="0")
    p = subprocess.run([sys.executable, "-c", _NEVER_JOINS, PKG], capture_output=True,
                       text=True, timeout=120, env=env)
    assert p.returncode == 0 and "timeout ok" in p.stdout, (p.stdout[-2000:], p.stderr[-2000:])
