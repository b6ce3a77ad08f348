"""Numpy model of the propagation patterns' memory slots, for testing the
x-slab halo plan and the ring orchestration (lbm_slab) without a GPU.

Slots, as the reference's kernels use them (src/kernel_pull_soa.c:98-116,
src/kernel_push_soa.c:131-198, src/kernel_aa_soa.c:42-151 and 168-274):
  pull     the post-collision population d of cell x sits in slot (d, x); a
           step gathers slot d of x - c_d, or slot inv d of x when x - c_d
           is an obstacle (half-way bounce-back)
  push     the population d arriving at x sits in slot (d, x); a step
           scatters to slot d of x + c_d, or to slot inv d of x
  AA even  reads slot d of x, writes slot inv d of x
  AA odd   reads slot inv d of x - c_d (slot d of x across a wall), writes
           slot d of x + c_d (slot inv d of x across a wall)
The collision is an arbitrary local function: the halo plan does not depend
on it. `Periodic` steps the whole x-periodic domain with wrapped indices and
no ghosts - the reference the decomposed runs must equal bit for bit.
`Slab` is one slab with ghost planes and the exchange plan of
lbm_halo_pack / lbm_halo_unpack (lbm_solver.cu), with the Solver.slab
interface that lbm_slab.SlabRunner drives.
"""
import numpy as np

Q = 19
CX = np.array([0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0])
CY = np.array([1, -1, 0, 0, 1, -1, 1, -1, 0, 1, 0, 0, -1, 0, -1, 1, 0, 0, 0])
CZ = np.array([0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, 0])
INV = np.array([[int(np.flatnonzero((CX == -CX[d]) & (CY == -CY[d]) & (CZ == -CZ[d]))[0])
                 for d in range(Q)]]).ravel()
W = np.array([1 / 36 if CX[d] ** 2 + CY[d] ** 2 + CZ[d] ** 2 == 2 else 1 / 18
              for d in range(Q - 1)] + [1 / 3])
PLUS = [d for d in range(Q) if CX[d] == 1]
MINUS = [d for d in range(Q) if CX[d] == -1]
HALO_BEFORE, HALO_AFTER = 1, 2


def collide(f):
    # sums in a fixed order: numpy's reductions round differently with the
    # batch size, which would make slab and whole-domain runs differ
    rho, ux, uy = np.zeros(f.shape[1:]), np.zeros(f.shape[1:]), np.zeros(f.shape[1:])
    for d in range(Q):
        rho = rho + f[d]
        ux = ux + CX[d] * f[d]
        uy = uy + CY[d] * f[d]
    shp = (Q,) + (1,) * (f.ndim - 1)
    return (f - 0.37 * (f - W.reshape(shp) * rho)
            + 0.011 * CX.reshape(shp) * ux + 0.007 * CY.reshape(shp) * uy * ux)


class _Lattice:
    """Shared stepping over cells of x range `own` with neighbour lookup."""

    def __init__(self, fluid, pattern, f0):
        self.fluid = fluid  # bool [nxd, ny, nz] in storage x
        self.pattern = pattern
        nb = 1 if pattern == "aa" else 2
        self.buf = [f0.copy() for _ in range(nb)]
        self.cur = 0
        self.steps_done = 0

    def _xs(self, x, dx):
        raise NotImplementedError

    def step(self):
        self._update(self.own)
        self._advance()

    def _update(self, xs):
        """Updates the cells of storage planes xs for the next step (no
        lattice swap, no step count)."""
        fl = self.fluid
        nxd, ny, nz = fl.shape
        X, Y, Z = np.meshgrid(xs, np.arange(ny), np.arange(nz), indexing="ij")
        live = fl[X, Y, Z]
        X, Y, Z = X[live], Y[live], Z[live]
        nbr = lambda d, s: (self._xs(X, s * CX[d]), (Y + s * CY[d]) % ny, (Z + s * CZ[d]) % nz)
        fin = np.empty((Q, X.size))
        if self.pattern == "aa":
            st = self.buf[0]
            odd = self.steps_done & 1
            for d in range(Q):
                if not odd:
                    fin[d] = st[d, X, Y, Z]
                else:
                    sx, sy, sz = nbr(d, -1)
                    wall = ~fl[sx, sy, sz]
                    fin[d] = np.where(wall, st[d, X, Y, Z], st[INV[d], sx, sy, sz])
            out = collide(fin)
            for d in range(Q):
                if not odd:
                    st[INV[d], X, Y, Z] = out[d]
                else:
                    tx, ty, tz = nbr(d, +1)
                    wall = ~fl[tx, ty, tz]
                    st[INV[d], X[wall], Y[wall], Z[wall]] = out[d][wall]
                    st[d, tx[~wall], ty[~wall], tz[~wall]] = out[d][~wall]
        else:
            src, dst = self.buf[self.cur], self.buf[self.cur ^ 1]
            for d in range(Q):
                if self.pattern == "pull":
                    sx, sy, sz = nbr(d, -1)
                    wall = ~fl[sx, sy, sz]
                    fin[d] = np.where(wall, src[INV[d], X, Y, Z], src[d, sx, sy, sz])
                else:
                    fin[d] = src[d, X, Y, Z]
            out = collide(fin)
            for d in range(Q):
                if self.pattern == "pull":
                    dst[d, X, Y, Z] = out[d]
                else:
                    tx, ty, tz = nbr(d, +1)
                    wall = ~fl[tx, ty, tz]
                    dst[INV[d], X[wall], Y[wall], Z[wall]] = out[d][wall]
                    dst[d, tx[~wall], ty[~wall], tz[~wall]] = out[d][~wall]

    def _advance(self):
        if self.pattern != "aa":
            self.cur ^= 1
        self.steps_done += 1

    def run(self, steps):
        for _ in range(steps):
            self.step()

    @property
    def state(self):
        return self.buf[0] if self.pattern == "aa" else self.buf[self.cur]


class Periodic(_Lattice):
    def __init__(self, fluid, pattern, f0):
        super().__init__(fluid, pattern, f0)
        self.own = np.arange(fluid.shape[0])

    def _xs(self, x, dx):
        return (x + dx) % self.fluid.shape[0]

    def own_state(self):
        return self.state


class Slab(_Lattice):
    """One slab; storage planes 0 and nx + 1 are ghosts."""

    def __init__(self, fluid_with_ghosts, pattern, f0_own):
        nx = fluid_with_ghosts.shape[0] - 2
        f0 = np.zeros((Q,) + fluid_with_ghosts.shape)
        f0[:, 1:nx + 1] = f0_own
        super().__init__(fluid_with_ghosts, pattern, f0)
        self.own = np.arange(1, nx + 1)
        self.nx = nx
        _, ny, nz = fluid_with_ghosts.shape
        self.halo_bytes = 5 * ny * nz * 8
        self.stream = 0

    def _xs(self, x, dx):
        return x + dx

    # the Solver.slab interface
    @property
    def halo_needs(self):
        if self.pattern == "pull":
            return HALO_BEFORE
        if self.pattern == "push":
            return HALO_AFTER
        return HALO_BEFORE | HALO_AFTER if self.steps_done & 1 else 0

    def _plan(self, when):
        first, last, gl, gr = 1, self.nx, 0, self.nx + 1
        if when == HALO_BEFORE:
            rs = PLUS if self.pattern == "pull" else MINUS
            ls = MINUS if self.pattern == "pull" else PLUS
            # (pack plane, set) per side; unpack targets
            return (first, ls), (last, rs), (gl, rs), (gr, ls)
        return (gl, MINUS), (gr, PLUS), (first, PLUS), (last, MINUS)

    def _lattice(self, when):
        # an after-step exchange inside a split step: the lattice being written
        if self.pattern != "aa" and when == HALO_AFTER and getattr(self, "_open", None) is not None:
            return self.buf[self.cur ^ 1]
        return self.state

    def halo_pack(self, when, to_left, to_right):
        (pl, sl), (pr, sr), _, _ = self._plan(when)
        st = self._lattice(when)
        to_left.numpy().view(np.float64)[:] = st[sl, pl].ravel()
        to_right.numpy().view(np.float64)[:] = st[sr, pr].ravel()

    def halo_unpack(self, when, from_left, from_right):
        _, _, (ul, sl), (ur, sr) = self._plan(when)
        st = self._lattice(when)
        shp = (5,) + st.shape[2:]
        for x, sset, msg in ((ul, sl, from_left), (ur, sr, from_right)):
            m = msg.numpy().view(np.float64).reshape(shp)
            for k, d in enumerate(sset):
                if when == HALO_BEFORE:  # ghost planes take everything
                    st[d, x] = m[k]
                    continue
                # own plane: only populations that arrived over a fluid link
                # (across a wall the cell's own step stored the bounce there)
                src = np.roll(np.roll(self.fluid[x - CX[d]], CY[d], 0), CZ[d], 1)
                ok = self.fluid[x] & src
                st[d, x][ok] = m[k][ok]

    def own_state(self):
        return self.state[:, 1:self.nx + 1]

    # split steps: planes update at once, in call order
    def step_begin(self):
        assert getattr(self, "_open", None) is None
        self._open = np.zeros(self.nx, dtype=bool)

    def step_planes(self, x_begin, x_end, side=False):
        assert 0 <= x_begin < x_end <= self.nx and not self._open[x_begin:x_end].any()
        self._open[x_begin:x_end] = True
        self._update(np.arange(x_begin + 1, x_end + 1))

    def step_end(self):
        assert self._open.all()
        self._open = None
        self._advance()

    @property
    def shape(self):
        return (self.nx,) + self.fluid.shape[1:]
