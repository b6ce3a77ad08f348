"""x-slab decomposition of one lattice over a ring of slabs.

The domain is cut along x - the slowest axis of LBM-Bench's SoA index
(src/lbm.h:113-116) and the periodic axis of its channel geometries - into
one slab per rank (one GPU each). A slab is a solver made by lbm_create_slab:
its own planes plus one ghost plane per side holding the neighbour's
boundary cells. Per step only the five populations that cross an x face move
between ring neighbours (lbm_halo_* in include/lbm_b200.h): one message pair
before a pull or AA odd step, one after a push or AA odd step, none around an
AA even step. Results are bit-identical to the undecomposed solver.

The pull state, and the AA state after an odd number of steps, keep part of
a boundary cell's populations in the neighbour's cells: call scatter() after
setting slab states and gather() before reading them.

Transports:
- `NativeRunner`: the ring in C (lbm_ring_* in include/lbm_b200.h, L.SlabRing):
  NCCL send/recv between ring neighbours on the solver's stream and the whole
  step loop issued by the library, so no Python runs per step. torch.distributed
  only carries the NCCL id from rank 0 to the others once.
- `SlabRunner` + `Ring`: the same schedule driven from Python over
  torch.distributed point-to-point (NCCL between GPUs, gloo between CPU
  processes); it also runs the numpy slab model of the tests.
- `LocalRing`: several slabs of one process (on one or several devices) with
  device copies.

LBM-Bench itself has no decomposition (single-node OpenMP, src/main.c).
"""
from __future__ import annotations

import numpy as np

import lbmb200 as L


# ---------------------------------------------------------------------------
# partition
# ---------------------------------------------------------------------------

def split(nx: int, world: int, rank: int):
    """Planes [x0, x1) of slab `rank`: the first nx % world slabs get one
    plane more."""
    if world < 1 or not 0 <= rank < world or nx < world:
        raise ValueError(f"cannot split {nx} planes over {world} slabs (rank {rank})")
    q, r = divmod(nx, world)
    x0 = rank * q + min(rank, r)
    return x0, x0 + q + (1 if rank < r else 0)


def slab_flags(flags: np.ndarray, x0: int, x1: int) -> np.ndarray:
    """Flags (nz, ny, nx) of the whole x-periodic domain -> the slab's flags
    with the neighbours' boundary planes (x0 - 1 and x1, wrapped) around it."""
    nx = flags.shape[2]
    idx = [(x0 - 1) % nx] + list(range(x0, x1)) + [x1 % nx]
    return np.ascontiguousarray(flags[:, :, idx])


# ---------------------------------------------------------------------------
# transports
# ---------------------------------------------------------------------------

class Ring:
    """Point-to-point exchange with the two ring neighbours over a
    torch.distributed process group (all ranks call exchange() together).

    Messages are tagged by direction (1: travelling right, 2: travelling
    left), and every rank posts its operations in the same order - send
    right, send left, receive from left, receive from right - so that with
    two ranks, where both neighbours are the same peer, the i-th send to a
    peer meets that peer's i-th receive from it."""

    def __init__(self, group=None):
        import torch.distributed as dist
        self.dist = dist
        self.group = group
        if dist.is_available() and dist.is_initialized():
            self.rank = dist.get_rank(group)
            self.world = dist.get_world_size(group)
        else:
            self.rank, self.world = 0, 1
        self.left = (self.rank - 1) % self.world
        self.right = (self.rank + 1) % self.world
        if group is not None and self.world > 1:
            self.left = dist.get_global_rank(group, self.left)
            self.right = dist.get_global_rank(group, self.right)

    def exchange(self, send_left, send_right, recv_left, recv_right):
        if self.world == 1:  # both neighbours are this slab: periodic in x
            recv_left.copy_(send_right)
            recv_right.copy_(send_left)
            return
        d = self.dist
        ops = [d.P2POp(d.isend, send_right, self.right, self.group, tag=1),
               d.P2POp(d.isend, send_left, self.left, self.group, tag=2),
               d.P2POp(d.irecv, recv_left, self.left, self.group, tag=1),
               d.P2POp(d.irecv, recv_right, self.right, self.group, tag=2)]
        for w in d.batch_isend_irecv(ops):
            w.wait()


class SlabRunner:
    """Steps one slab of a ring: exchange, step, exchange, as the pattern
    and the step parity need (Solver.halo_needs).

    With overlap=True each step is split (Solver.step_begin / step_planes /
    step_end): the interior planes 1 .. nx-2 run on the solver's second
    stream while its own stream packs, exchanges and unpacks the BEFORE
    messages, updates the boundary planes 0 and nx-1 and exchanges the AFTER
    messages. The exchanged slots and the interior touch disjoint memory, so
    the result is the same bit for bit.

    `solver` is a slab (Solver.slab) or any object with the same halo_*
    methods, run(), the step_* methods (for overlap), shape and stream;
    `device` is where the message buffers live ("cuda" for a GPU slab)."""

    def __init__(self, solver, ring: Ring, device="cuda", overlap=False):
        import torch
        self.torch = torch
        self.s = solver
        self.ring = ring
        self.overlap = overlap
        n = solver.halo_bytes
        if n <= 0:
            raise ValueError("SlabRunner needs a slab solver (lbm_create_slab)")
        self.bufs = [torch.empty(n, dtype=torch.uint8, device=device) for _ in range(4)]
        self.ext = None
        dev = torch.device(device)
        if dev.type == "cuda":
            if dev.index is None:
                dev = torch.device("cuda", torch.cuda.current_device())
            self.ext = torch.cuda.ExternalStream(solver.stream, device=dev)
        self.exchanges = 0

    def _exchange(self, when: int):
        sl, sr, rl, rr = self.bufs
        self.s.halo_pack(when, sl, sr)
        if self.ext is not None:
            with self.torch.cuda.stream(self.ext):
                self.ring.exchange(sl, sr, rl, rr)
        else:
            self.ring.exchange(sl, sr, rl, rr)
        self.s.halo_unpack(when, rl, rr)
        self.exchanges += 1

    def run(self, steps: int):
        for _ in range(steps):
            need = self.s.halo_needs
            if self.overlap:
                self._split_step(need)
                continue
            if need & L.HALO_BEFORE:
                self._exchange(L.HALO_BEFORE)
            self.s.run(1)
            if need & L.HALO_AFTER:
                self._exchange(L.HALO_AFTER)

    def _split_step(self, need: int):
        s = self.s
        nx = s.shape[0]
        s.step_begin()
        if nx > 2:
            s.step_planes(1, nx - 1, side=True)
        if need & L.HALO_BEFORE:
            self._exchange(L.HALO_BEFORE)
        s.step_planes(0, 1)
        if nx > 1:
            s.step_planes(nx - 1, nx)
        if need & L.HALO_AFTER:
            self._exchange(L.HALO_AFTER)
        s.step_end()

    def gather(self):
        """Before reading the state: the neighbours' share of this slab's
        boundary populations into the ghost planes (shifted states only)."""
        if self.s.halo_shifted:
            self._exchange(L.HALO_BEFORE)

    def scatter(self):
        """After setting the state: the boundary populations set_state kept
        in the ghost planes go to the neighbours (shifted states only)."""
        if self.s.halo_shifted:
            self._exchange(L.HALO_SCATTER)


def share_ring_id(group=None):
    """Rank 0 of the process group makes an NCCL id for lbm_ring_create
    (L.ring_unique_id, no GPU needed) and broadcasts it; every rank returns
    the same 128 bytes. None without a process group of two or more ranks."""
    import torch.distributed as dist
    if not (dist.is_available() and dist.is_initialized()) or dist.get_world_size(group) == 1:
        return None
    obj = [L.ring_unique_id() if dist.get_rank(group) == 0 else None]
    src = dist.get_global_rank(group, 0) if group is not None else 0
    dist.broadcast_object_list(obj, src=src, group=group)
    return obj[0]


class NativeRunner:
    """SlabRunner's schedule issued from C (L.SlabRing over lbm_ring_*): the
    halo messages travel over NCCL between ring neighbours, ordered on the
    solver's stream, and no Python runs per step. Ranks are those of the
    process group (ring neighbours rank - 1 and rank + 1); with one rank the
    slab is its own neighbour, by device copies or, with nccl=True, through
    a one-rank NCCL communicator (sends to itself). All ranks construct it
    together (the id broadcast is a collective)."""

    def __init__(self, solver, group=None, overlap=True, timeout_ms=0, nccl=None):
        import torch.distributed as dist
        if dist.is_available() and dist.is_initialized():
            rank, world = dist.get_rank(group), dist.get_world_size(group)
        else:
            rank, world = 0, 1
        uid = share_ring_id(group)
        if uid is None and nccl:
            uid = L.ring_unique_id()
        self.s = solver
        self.overlap = overlap
        self.ring = L.SlabRing(solver, rank, world, uid, timeout_ms)

    @property
    def exchanges(self) -> int:
        return self.ring.exchanges

    @property
    def uses_nccl(self) -> bool:
        return self.ring.uses_nccl

    def run(self, steps: int) -> None:
        self.ring.run(steps, self.overlap)

    def gather(self) -> None:
        self.ring.gather()

    def scatter(self) -> None:
        self.ring.scatter()

    def synchronize(self) -> None:
        self.ring.synchronize()

    def close(self) -> None:
        self.ring.close()


class LocalRing:
    """Several slabs of one ring driven from one process: every slab packs,
    all streams are synchronised, every slab unpacks its neighbours'
    messages. For tests and for domains split over the devices of one
    process; the kernels of different slabs never wait on one another."""

    def __init__(self, solvers, device="cuda", overlap=False):
        import torch
        self.overlap = overlap
        self.solvers = list(solvers)
        self.bufs = []
        for s in self.solvers:
            n = s.halo_bytes
            if n <= 0:
                raise ValueError("LocalRing needs slab solvers (lbm_create_slab)")
            self.bufs.append([torch.empty(n, dtype=torch.uint8, device=device) for _ in range(2)])

    def _exchange(self, when: int):
        n = len(self.solvers)
        for s, (tl, tr) in zip(self.solvers, self.bufs):
            s.halo_pack(when, tl, tr)
        for s in self.solvers:
            s.synchronize()
        for i, s in enumerate(self.solvers):
            left, right = self.bufs[(i - 1) % n], self.bufs[(i + 1) % n]
            s.halo_unpack(when, left[1], right[0])  # left's to_right, right's to_left
        for s in self.solvers:
            s.synchronize()

    def run(self, steps: int):
        for _ in range(steps):
            needs = {s.halo_needs for s in self.solvers}
            if len(needs) != 1:
                raise RuntimeError("slabs of one ring are at different steps")
            need = needs.pop()
            if self.overlap:  # the schedule of SlabRunner(overlap=True)
                for s in self.solvers:
                    s.step_begin()
                    if s.shape[0] > 2:
                        s.step_planes(1, s.shape[0] - 1, side=True)
            if need & L.HALO_BEFORE:
                self._exchange(L.HALO_BEFORE)
            for s in self.solvers:
                if self.overlap:
                    s.step_planes(0, 1)
                    if s.shape[0] > 1:
                        s.step_planes(s.shape[0] - 1, s.shape[0])
                else:
                    s.run(1)
            if need & L.HALO_AFTER:
                self._exchange(L.HALO_AFTER)
            if self.overlap:
                for s in self.solvers:
                    s.step_end()

    def gather(self):
        """Before reading the slabs' states (see SlabRunner.gather)."""
        if self.solvers[0].halo_shifted:
            self._exchange(L.HALO_BEFORE)

    def scatter(self):
        """After setting the slabs' states (see SlabRunner.scatter)."""
        if self.solvers[0].halo_shifted:
            self._exchange(L.HALO_SCATTER)
