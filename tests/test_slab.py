"""x-slab decomposition on the CPU: the halo plan (numpy model of the slots,
tests/slab_model.py) and the ring orchestration of lbm_slab over gloo with
2 and 3 processes, bit for bit against the undecomposed x-periodic run."""
import os
import socket
import tempfile

import numpy as np
import pytest

import lbm_slab
import lbmb200 as L
import slab_model as M

PATTERNS = ["pull", "push", "aa"]


def _domain(seed, dims=(12, 6, 5), solid=0.25):
    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    fluid = rng.uniform(size=dims) > solid
    f0 = rng.uniform(0.01, 0.1, size=(M.Q,) + dims) * fluid
    return fluid, f0


def test_split_covers_the_domain():
    for nx, world in ((12, 1), (12, 5), (7, 7), (1000, 8), (257, 4)):
        spans = [lbm_slab.split(nx, world, r) for r in range(world)]
        assert spans[0][0] == 0 and spans[-1][1] == nx
        assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
        sizes = [b - a for a, b in spans]
        assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        lbm_slab.split(3, 4, 0)


def test_slab_flags_wrap_periodically():
    flags = np.arange(2 * 3 * 7).reshape(2, 3, 7)
    s = lbm_slab.slab_flags(flags, 0, 3)
    assert np.array_equal(s[:, :, 0], flags[:, :, 6])
    assert np.array_equal(s[:, :, 1:4], flags[:, :, 0:3])
    assert np.array_equal(s[:, :, 4], flags[:, :, 3])
    s = lbm_slab.slab_flags(flags, 5, 7)
    assert np.array_equal(s[:, :, -1], flags[:, :, 0])


def _model_slabs(fluid, f0, pattern, spans):
    slabs = []
    nx = fluid.shape[0]
    for x0, x1 in spans:
        idx = [(x0 - 1) % nx] + list(range(x0, x1)) + [x1 % nx]
        slabs.append(M.Slab(fluid[idx], pattern, f0[:, x0:x1]))
    return slabs


class _LocalModelRing:
    """Sequential exchange between model slabs of one process."""

    def __init__(self, slabs):
        import torch
        self.slabs = slabs
        self.bufs = [[torch.empty(s.halo_bytes, dtype=torch.uint8) for _ in range(2)]
                     for s in slabs]

    def _exchange(self, when):
        n = len(self.slabs)
        for s, (tl, tr) in zip(self.slabs, self.bufs):
            s.halo_pack(when, tl, tr)
        for i, s in enumerate(self.slabs):
            s.halo_unpack(when, self.bufs[(i - 1) % n][1], self.bufs[(i + 1) % n][0])

    def run(self, steps):
        for _ in range(steps):
            need = self.slabs[0].halo_needs
            if need & M.HALO_BEFORE:
                self._exchange(M.HALO_BEFORE)
            for s in self.slabs:
                s.run(1)
            if need & M.HALO_AFTER:
                self._exchange(M.HALO_AFTER)


@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("world", [1, 2, 3, 4])
def test_halo_plan_reproduces_the_periodic_domain(pattern, world):
    fluid, f0 = _domain(world)
    steps = 7
    ref = M.Periodic(fluid, pattern, f0)
    ref.run(steps)
    spans = [lbm_slab.split(fluid.shape[0], world, r) for r in range(world)]
    slabs = _model_slabs(fluid, f0, pattern, spans)
    _LocalModelRing(slabs).run(steps)
    got = np.concatenate([s.own_state() for s in slabs], axis=1)
    assert np.array_equal(got[:, fluid], ref.own_state()[:, fluid])


def test_after_unpack_needs_the_link_guard():
    """Without the fluid-link guard, a stale ghost slot overwrites a bounced
    population in the push pattern: the guard is load-bearing."""
    fluid, f0 = _domain(5)
    ref = M.Periodic(fluid, "push", f0)
    ref.run(3)
    spans = [lbm_slab.split(fluid.shape[0], 2, r) for r in range(2)]
    slabs = _model_slabs(fluid, f0, "push", spans)

    def unguarded(self, when, from_left, from_right):
        _, _, (ul, sl), (ur, sr) = self._plan(when)
        shp = (5,) + self.state.shape[2:]
        self.state[sl, ul] = from_left.numpy().view(np.float64).reshape(shp)
        self.state[sr, ur] = from_right.numpy().view(np.float64).reshape(shp)

    for s in slabs:
        s.halo_unpack = unguarded.__get__(s)
    _LocalModelRing(slabs).run(3)
    got = np.concatenate([s.own_state() for s in slabs], axis=1)
    assert not np.array_equal(got[:, fluid], ref.own_state()[:, fluid])


# ---------------------------------------------------------------------------
# lbm_slab.SlabRunner over gloo, one process per slab
# ---------------------------------------------------------------------------

def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("dims", [(12, 6, 5), (2, 5, 4), (1, 4, 6)])
def test_split_step_ring_of_one_matches_periodic_run(pattern, dims):
    """SlabRunner(overlap=True) on one slab (its own neighbour): interior
    planes first, then the exchanges and the boundary planes, as the
    overlapped schedule orders them; slabs of 1 and 2 planes included."""
    fluid, f0 = _domain(21, dims)
    ref = M.Periodic(fluid, pattern, f0)
    ref.run(7)
    slab = _model_slabs(fluid, f0, pattern, [(0, dims[0])])[0]
    runner = lbm_slab.SlabRunner(slab, lbm_slab.Ring(), device="cpu", overlap=True)
    runner.run(7)
    assert np.array_equal(slab.own_state()[:, fluid], ref.own_state()[:, fluid])


def _gloo_worker(rank, world, port, pattern, steps, seed, outdir, overlap=False):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        fluid, f0 = _domain(seed)
        x0, x1 = lbm_slab.split(fluid.shape[0], world, rank)
        slab = _model_slabs(fluid, f0, pattern, [(x0, x1)])[0]
        runner = lbm_slab.SlabRunner(slab, lbm_slab.Ring(), device="cpu", overlap=overlap)
        runner.run(steps)
        np.save(os.path.join(outdir, f"rank{rank}.npy"), slab.own_state())
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("overlap", [False, True])
@pytest.mark.parametrize("pattern", PATTERNS)
@pytest.mark.parametrize("world", [2, 3])
def test_slab_runner_over_gloo_matches_periodic_run(pattern, world, overlap):
    import torch.multiprocessing as mp
    seed, steps = 11 + world, 6
    with tempfile.TemporaryDirectory() as outdir:
        mp.start_processes(_gloo_worker,
                           args=(world, _free_port(), pattern, steps, seed, outdir, overlap),
                           nprocs=world, join=True, start_method="spawn")
        got = np.concatenate([np.load(os.path.join(outdir, f"rank{r}.npy"))
                              for r in range(world)], axis=1)
    fluid, f0 = _domain(seed)
    ref = M.Periodic(fluid, pattern, f0)
    ref.run(steps)
    assert np.array_equal(got[:, fluid], ref.own_state()[:, fluid])


# ---------------------------------------------------------------------------
# native ring (lbm_ring_*): the NCCL id reaches every rank; argument checks
# ---------------------------------------------------------------------------

def _id_worker(rank, world, port, outdir):
    import torch.distributed as dist
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank,
                            world_size=world)
    try:
        uid = lbm_slab.share_ring_id()
        with open(os.path.join(outdir, f"id{rank}.bin"), "wb") as f:
            f.write(uid)
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_ring_id_is_shared_by_all_ranks(world):
    """Rank 0 makes the NCCL id (lbm_ring_unique_id, no GPU needed) and the
    process group carries it once; every rank must hold the same bytes."""
    import torch.multiprocessing as mp
    with tempfile.TemporaryDirectory() as outdir:
        mp.start_processes(_id_worker, args=(world, _free_port(), outdir), nprocs=world,
                           join=True, start_method="spawn")
        ids = [open(os.path.join(outdir, f"id{r}.bin"), "rb").read() for r in range(world)]
    assert len(ids[0]) == L.RING_ID_BYTES and any(ids[0])
    assert all(i == ids[0] for i in ids)


def test_ring_id_without_process_group_is_none():
    assert lbm_slab.share_ring_id() is None
    a, b = L.ring_unique_id(), L.ring_unique_id()
    assert len(a) == len(b) == L.RING_ID_BYTES and a != b


def test_ring_create_rejects_bad_arguments_without_gpu():
    import ctypes
    h = ctypes.c_void_p()
    lib = L.lib()
    assert lib.lbm_ring_create(ctypes.byref(h), None, 0, 1, None, 0) == -1
    assert lib.lbm_ring_exchanges(None) == -1 and lib.lbm_ring_uses_nccl(None) == -1
    assert lib.lbm_ring_run(None, 1, 0) == -1
    assert lib.lbm_ring_destroy(None) == 0
