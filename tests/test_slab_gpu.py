"""x-slab decomposition on a B200: slabs made by lbm_create_slab (or
lbm_create_slab_compact) and exchanging halos (lbm_halo_pack /
lbm_halo_unpack) reproduce the undecomposed x-periodic solver bit for bit,
for every propagation pattern, storage precision and layout. The slabs of a ring run in one process on one GPU
(lbm_slab.LocalRing: pack all, synchronise, unpack all), and one slab runs
through lbm_slab.SlabRunner as a ring of one."""
import numpy as np
import pytest

import lbm_slab
import lbmb200 as L
import oracle as O

pytestmark = pytest.mark.gpu

PATTERNS = ["pull", "push", "aa"]


def _domain(dims, seed):
    flags, _, _ = L.porous_channel(dims, 0.2, 1.5, 3.0, seed=seed)
    f0 = L.perturbed_equilibrium(flags, seed=seed, amplitude=1e-3)
    return flags, f0


def _params(s):
    s.set_params(1.25, 3 / 16, 1e-5, True)


def _single(flags, f0, pattern, precision, steps, compact=False):
    with L.Solver(flags, (1, 0, 0), pattern, precision, compact=compact) as s:
        _params(s)
        s.set_state(f0)
        s.run(steps)
        return s.get_state(), s.mass_momentum()[0]


def _slabs(flags, f0, pattern, precision, world, compact=False):
    nx = flags.shape[2]
    out = []
    for r in range(world):
        x0, x1 = lbm_slab.split(nx, world, r)
        s = L.Solver.slab(lbm_slab.slab_flags(flags, x0, x1), (0, 0), pattern, precision,
                          compact=compact)
        _params(s)
        s.set_state(np.ascontiguousarray(f0[:, x0:x1]))
        out.append(s)
    return out


@pytest.mark.parametrize("compact", [False, True], ids=["dense", "compact"])
@pytest.mark.parametrize("precision", [L.F64, L.F32, L.F16])
@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("world", [2, 3])
def test_local_ring_equals_undecomposed(pattern, precision, world, compact):
    flags, f0 = _domain((23, 14, 12), 3 + world)
    steps = 9
    ref, tot_ref = _single(flags, f0, pattern, precision, steps)
    slabs = _slabs(flags, f0, pattern, precision, world, compact)
    ring = lbm_slab.LocalRing(slabs)
    ring.scatter()
    ring.run(steps)
    ring.gather()
    got = np.concatenate([s.get_state() for s in slabs], axis=1)
    tot = np.sum([s.mass_momentum()[0] for s in slabs], axis=0)
    for s in slabs:
        s.close()
    m = O.fluid_mask(flags)
    assert np.array_equal(got[:, m], ref[:, m])
    assert tot[0] == pytest.approx(tot_ref[0], rel=1e-13)


@pytest.mark.parametrize("precision", [L.F64, L.F16])
@pytest.mark.parametrize("pattern", PATTERNS)
def test_shuffle_kernels_on_slabs(pattern, precision):
    """nz = 64: the reduced-precision pull/push/AA-odd steps take the
    shuffle-aligned kernels."""
    flags, f0 = _domain((16, 10, 64), 21)
    ref, _ = _single(flags, f0, pattern, precision, 5)
    slabs = _slabs(flags, f0, pattern, precision, 2)
    ring = lbm_slab.LocalRing(slabs)
    ring.scatter()
    ring.run(5)
    ring.gather()
    got = np.concatenate([s.get_state() for s in slabs], axis=1)
    m = O.fluid_mask(flags)
    assert np.array_equal(got[:, m], ref[:, m])


@pytest.mark.parametrize("pattern", PATTERNS)
def test_slab_runner_ring_of_one_is_periodic(pattern):
    """SlabRunner with no process group: the slab is its own neighbour,
    messages go through CUDA buffers ordered on the solver's stream."""
    flags, f0 = _domain((18, 12, 10), 8)
    ref, _ = _single(flags, f0, pattern, L.F64, 7)
    s = _slabs(flags, f0, pattern, L.F64, 1)[0]
    runner = lbm_slab.SlabRunner(s, lbm_slab.Ring())
    runner.scatter()
    base = runner.exchanges
    runner.run(7)
    ex = runner.exchanges - base
    runner.gather()
    got = s.get_state()
    s.close()
    m = O.fluid_mask(flags)
    assert np.array_equal(got[:, m], ref[:, m])
    expect = {"pull": 7, "push": 7, "aa": 6}[pattern]  # AA: before + after each odd step
    assert ex == expect


@pytest.mark.parametrize("compact", [False, True], ids=["dense", "compact"])
@pytest.mark.parametrize("precision", [L.F64, L.F32, L.F16])
@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("dims", [(18, 12, 10), (9, 6, 128), (2, 8, 64), (1, 9, 7)])
def test_split_steps_ring_of_one_equal_undecomposed(pattern, precision, dims, compact):
    """SlabRunner(overlap=True): each step split into the interior planes on
    the solver's second stream and the boundary planes plus exchanges on its
    own stream (lbm_step_begin / _planes / _end), bit for bit equal to the
    undecomposed solver; FP16 at nz = 128 runs the four-cell kernels, slabs
    of 1 and 2 planes have no interior."""
    flags, f0 = _domain(dims, 31)
    ref, _ = _single(flags, f0, pattern, precision, 7)
    s = _slabs(flags, f0, pattern, precision, 1, compact)[0]
    runner = lbm_slab.SlabRunner(s, lbm_slab.Ring(), overlap=True)
    runner.scatter()
    launches0 = s.launch_count
    runner.run(7)
    runner.gather()
    got = s.get_state()
    split_launches = s.launch_count - launches0
    s.close()
    m = O.fluid_mask(flags)
    assert np.array_equal(got[:, m], ref[:, m])
    assert split_launches == 7 * min(dims[0], 3)


@pytest.mark.parametrize("compact", [False, True], ids=["dense", "compact"])
@pytest.mark.parametrize("pattern", PATTERNS)
def test_split_steps_on_a_ring_of_three(pattern, compact):
    flags, f0 = _domain((23, 14, 12), 17)
    ref, _ = _single(flags, f0, pattern, L.F64, 9)
    slabs = _slabs(flags, f0, pattern, L.F64, 3, compact)
    ring = lbm_slab.LocalRing(slabs, overlap=True)
    ring.scatter()
    ring.run(9)
    ring.gather()
    got = np.concatenate([s.get_state() for s in slabs], axis=1)
    for s in slabs:
        s.close()
    m = O.fluid_mask(flags)
    assert np.array_equal(got[:, m], ref[:, m])


def test_split_step_errors():
    import torch
    flags, f0 = _domain((8, 8, 8), 2)
    buf = torch.empty(1 << 16, dtype=torch.uint8, device="cuda")
    s = L.Solver.slab(lbm_slab.slab_flags(flags, 0, 8), (0, 0), "push")
    with pytest.raises(L.LbmError):
        s.step_planes(0, 8)  # no open step
    with pytest.raises(L.LbmError):
        s.step_end()
    s.step_begin()
    with pytest.raises(L.LbmError):
        s.step_begin()  # already open
    s.step_planes(2, 5, side=True)
    for bad in ((4, 6), (0, 0), (-1, 1), (7, 9)):
        with pytest.raises(L.LbmError):
            s.step_planes(*bad)
    with pytest.raises(L.LbmError):
        s.run(1)
    with pytest.raises(L.LbmError):
        s.get_state()
    with pytest.raises(L.LbmError):
        s.step_end()  # planes 0, 1, 5, 6, 7 missing
    s.step_planes(0, 2)
    s.step_planes(5, 8)
    s.halo_pack(L.HALO_AFTER, buf, buf)  # the open step's messages
    s.step_end()
    s.synchronize()
    assert s.steps_done == 1
    s.close()


@pytest.mark.parametrize("pattern", PATTERNS)
def test_slab_state_round_trip_in_shifted_orientation(pattern):
    """set_state + scatter, then gather + get_state, return the state, at an
    odd step count (the AA state is then shifted too)."""
    flags, f0 = _domain((15, 11, 9), 12)
    slabs = _slabs(flags, f0, pattern, L.F64, 3)
    ring = lbm_slab.LocalRing(slabs)
    ring.scatter()
    ring.run(3)
    for s in slabs:
        assert s.halo_shifted == (pattern != "push")
    f1 = f0 * 1.01
    nx = flags.shape[2]
    for r, s in enumerate(slabs):
        x0, x1 = lbm_slab.split(nx, 3, r)
        s.set_state(np.ascontiguousarray(f1[:, x0:x1]))
    ring.scatter()
    ring.gather()
    got = np.concatenate([s.get_state() for s in slabs], axis=1)
    m = O.fluid_mask(flags)
    assert np.array_equal(got[:, m], f1[:, m])


def test_halo_argument_errors():
    import torch
    flags, f0 = _domain((8, 8, 8), 1)
    buf = torch.empty(1 << 16, dtype=torch.uint8, device="cuda")
    with L.Solver(flags, (1, 0, 0), "aa") as s:
        assert s.halo_bytes == 0 and s.halo_needs == 0
        with pytest.raises(L.LbmError):
            s.halo_pack(L.HALO_BEFORE, buf, buf)
    s = L.Solver.slab(lbm_slab.slab_flags(flags, 0, 8), (0, 0), "aa")
    assert s.halo_bytes == 5 * 8 * 8 * 8
    assert s.halo_needs == 0  # even step: local
    with pytest.raises(L.LbmError):
        s.halo_pack(L.HALO_BEFORE, buf, buf)  # no exchange before an even step
    with pytest.raises(L.LbmError):
        s.halo_pack(3, buf, buf)
    with pytest.raises(L.LbmError):
        s.halo_pack(L.HALO_SCATTER, buf, buf)  # natural orientation: nothing to scatter
    s.run(1)
    assert s.halo_needs == L.HALO_BEFORE | L.HALO_AFTER
    s.halo_pack(L.HALO_BEFORE, buf, buf)
    s.synchronize()
    s.close()
