"""Test infrastructure only: ctypes bindings for the CPU oracle libraries.

* ``liboracle.so`` - our C restatement of the D3Q19 TRT step (lbm_oracle.c).
* ``_ref/libref_*.so`` - LBM-Bench's own sources compiled unmodified
  (oracle/Makefile) behind ref_harness.c. Present only where the reference
  tree was available at build time.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg import this module, and only as the checker / the timed CPU baseline.

Array conventions (shared with the product's flat C API):
  flags  int32[nz, ny, nx]   the reference's latticeIndex order, x fastest
                             (src/lbm.h:108-111); 0 = obstacle, 1 = fluid.
  f      float64[19, nx, ny, nz]  z fastest; f[d, x, y, z] is the population
                             of direction d that cell (x,y,z) collides next.
"""
from __future__ import annotations

import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(HERE, "_ref")
Q = 19

# D3Q19 velocity set in the reference's direction order (src/lbm.c:20-29).
CX = np.array([0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0])
CY = np.array([1, -1, 0, 0, 1, -1, 1, -1, 0, 1, 0, 0, -1, 0, -1, 1, 0, 0, 0])
CZ = np.array([0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, 0])
INV = np.array([int(np.flatnonzero((CX == -CX[d]) & (CY == -CY[d]) & (CZ == -CZ[d]))[0])
                for d in range(19)])
W = np.array([1 / 18] * 4 + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4 + [1 / 18] + [1 / 36] * 4
             + [1 / 3])

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)


def build(quiet: bool = True) -> None:
    """Compiles liboracle.so (and oracle/_ref when the reference tree exists)."""
    out = subprocess.run(["make", "-C", HERE, "all"], capture_output=True, text=True)
    if out.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + out.stdout + out.stderr)
    if not quiet:
        print(out.stdout)


def _ptr(a: np.ndarray, kind):
    return a.ctypes.data_as(kind)


class Oracle:
    """Our C restatement (liboracle.so)."""

    def __init__(self, path: str | None = None):
        path = path or os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.orc_run.restype = ctypes.c_int
        L.orc_run.argtypes = [ctypes.c_int] * 3 + [_ip] + [ctypes.c_int] * 3 + \
            [ctypes.c_double] * 3 + [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_run_brinkman.restype = ctypes.c_int
        L.orc_run_brinkman.argtypes = [ctypes.c_int] * 3 + [_ip] + [ctypes.c_int] * 3 + \
            [ctypes.c_double] * 4 + [_fp, ctypes.c_int, _dp, _dp]
        L.orc_run_pressure.restype = ctypes.c_int
        L.orc_run_pressure.argtypes = [ctypes.c_int] * 3 + [_ip] + [ctypes.c_int] * 3 + \
            [ctypes.c_double] * 3 + [ctypes.c_int] + [ctypes.c_double] * 2 + \
            [ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_objective.restype = ctypes.c_double
        L.orc_objective.argtypes = [ctypes.c_int] * 3 + [_ip, _dp]
        L.orc_adjoint_brinkman.restype = ctypes.c_int
        L.orc_adjoint_brinkman.argtypes = [ctypes.c_int] * 3 + [_ip] + [ctypes.c_int] * 3 + \
            [ctypes.c_double] * 4 + [_fp, ctypes.c_int, _dp, _dp, _dp]

    def run(self, flags, periodic, f_in, steps, omega, lam, xforce, force_on=True):
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        f_in = np.ascontiguousarray(f_in, dtype=np.float64)
        out = np.empty_like(f_in)
        rc = self.lib.orc_run(nx, ny, nz, _ptr(flags, _ip), *[int(p) for p in periodic],
                              omega, lam, xforce, int(force_on), steps, _ptr(f_in, _dp),
                              _ptr(out, _dp))
        if rc != 0:
            raise RuntimeError("orc_run failed")
        return out

    def run_brinkman(self, flags, periodic, f_in, steps, omega, lam, xforce, alpha, porosity):
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        f_in = np.ascontiguousarray(f_in, dtype=np.float64)
        por = np.ascontiguousarray(porosity, dtype=np.float32)
        out = np.empty_like(f_in)
        rc = self.lib.orc_run_brinkman(nx, ny, nz, _ptr(flags, _ip), *[int(p) for p in periodic],
                                       omega, lam, xforce, alpha, _ptr(por, _fp), steps,
                                       _ptr(f_in, _dp), _ptr(out, _dp))
        if rc != 0:
            raise RuntimeError("orc_run_brinkman failed")
        return out

    def run_pressure(self, flags, periodic, f_in, steps, omega, lam, xforce, force_on,
                     rho_in, rho_out, bc_every=1):
        """orc_run with the Zou-He pressure boundary after every bc_every-th
        step (inlet flag 2 on x = 0, outlet flag 4 on x = nx-1)."""
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        f_in = np.ascontiguousarray(f_in, dtype=np.float64)
        out = np.empty_like(f_in)
        rc = self.lib.orc_run_pressure(nx, ny, nz, _ptr(flags, _ip), *[int(p) for p in periodic],
                                       omega, lam, xforce, int(force_on), rho_in, rho_out,
                                       bc_every, steps, _ptr(f_in, _dp), _ptr(out, _dp))
        if rc != 0:
            raise RuntimeError("orc_run_pressure failed")
        return out

    def objective(self, flags, f):
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        f = np.ascontiguousarray(f, dtype=np.float64)
        return self.lib.orc_objective(nx, ny, nz, _ptr(flags, _ip), _ptr(f, _dp))

    def adjoint(self, flags, periodic, f_in, steps, omega, lam, xforce, alpha, porosity):
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        f_in = np.ascontiguousarray(f_in, dtype=np.float64)
        por = np.ascontiguousarray(porosity, dtype=np.float32)
        grad = np.zeros((nx, ny, nz), dtype=np.float64)
        j = ctypes.c_double(0.0)
        rc = self.lib.orc_adjoint_brinkman(nx, ny, nz, _ptr(flags, _ip),
                                           *[int(p) for p in periodic], omega, lam, xforce,
                                           alpha, _ptr(por, _fp), steps, _ptr(f_in, _dp),
                                           _ptr(grad, _dp), ctypes.byref(j))
        if rc != 0:
            raise RuntimeError("orc_adjoint_brinkman failed")
        return j.value, grad


def ref_available(variant: str = "verify") -> bool:
    return os.path.exists(os.path.join(REF_DIR, f"libref_{variant}.so"))


class Reference:
    """LBM-Bench's own kernels behind ref_harness.c (oracle/_ref)."""

    def __init__(self, variant: str = "verify"):
        path = os.path.join(REF_DIR, f"libref_{variant}.so")
        if not os.path.exists(path):
            raise FileNotFoundError(path)
        self.lib = ctypes.CDLL(path)
        L = self.lib
        L.ref_n_kernels.restype = ctypes.c_int
        L.ref_kernel_name.restype = ctypes.c_char_p
        L.ref_kernel_name.argtypes = [ctypes.c_int]
        L.ref_max_threads.restype = ctypes.c_int
        L.ref_geometry.restype = ctypes.c_int
        L.ref_geometry.argtypes = [ctypes.c_char_p, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                   _ip, _ip, _ip, _ip]
        L.ref_run.restype = ctypes.c_int
        L.ref_run.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 3 + [_ip] + \
            [ctypes.c_int] * 3 + [ctypes.c_double] * 2 + [ctypes.c_int, ctypes.c_int, _dp, _dp,
                                                          _dp, _ip, _ip]
        L.ref_run_pressure.restype = ctypes.c_int
        L.ref_run_pressure.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 3 + [_ip] + \
            [ctypes.c_int] * 3 + [ctypes.c_double] * 4 + [ctypes.c_int, _dp, _dp]
        L.ref_verify.restype = ctypes.c_int
        L.ref_verify.argtypes = [ctypes.c_int] * 3 + [_ip] + [ctypes.c_int] * 3 + \
            [ctypes.c_double] * 2 + [_dp, _dp]
        L.ref_initial_state.restype = ctypes.c_int
        L.ref_initial_state.argtypes = [ctypes.c_char_p] + [ctypes.c_int] * 3 + [_ip] + \
            [ctypes.c_int] * 3 + [ctypes.c_double, _dp]

    def kernels(self):
        return [self.lib.ref_kernel_name(i).decode() for i in range(self.lib.ref_n_kernels())]

    def max_threads(self) -> int:
        return self.lib.ref_max_threads()

    def geometry(self, kind: str, dims, periodic=(0, 0, 0)):
        nx, ny, nz = dims
        flags = np.zeros((nz, ny, nx), dtype=np.int32)
        pin = np.array(periodic, dtype=np.int32)
        pout = np.zeros(3, dtype=np.int32)
        counts = np.zeros(2, dtype=np.int32)
        self.lib.ref_geometry(kind.encode(), nx, ny, nz, _ptr(pin, _ip), _ptr(flags, _ip),
                              _ptr(pout, _ip), _ptr(counts, _ip))
        return flags, tuple(int(p) for p in pout), (int(counts[0]), int(counts[1]))

    def run(self, kernel, flags, periodic, f_in, steps, omega, xforce, inject=True,
            readback=True):
        """Returns (f_out or None, duration_s, final Iteration, nBounceBackPdfs).
        duration_s is the reference kernel's own timing of its time loop."""
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        if f_in is None:
            f_in = np.zeros((Q, nx, ny, nz))
        f_in = np.ascontiguousarray(f_in, dtype=np.float64)
        out = np.zeros_like(f_in) if readback else None
        dur = ctypes.c_double(0.0)
        it = ctypes.c_int(0)
        nbb = ctypes.c_int(0)
        rc = self.lib.ref_run(kernel.encode(), nx, ny, nz, _ptr(flags, _ip),
                              *[int(p) for p in periodic], omega, xforce, steps, int(inject),
                              _ptr(f_in, _dp), _ptr(out, _dp) if readback else None,
                              ctypes.byref(dur),
                              ctypes.byref(it), ctypes.byref(nbb))
        if rc != 0:
            raise KeyError(kernel)
        return out, dur.value, it.value, nbb.value

    def run_pressure(self, kernel, flags, periodic, f_in, calls, omega, xforce, rho_in,
                     rho_out):
        """`calls` kd->Kernel calls of one iteration (one step for pull and
        push, two for AA), each followed by the reference's
        kernelComputeBoundaryConditions. Returns the final state."""
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        f_in = np.ascontiguousarray(f_in, dtype=np.float64)
        out = np.zeros_like(f_in)
        rc = self.lib.ref_run_pressure(kernel.encode(), nx, ny, nz, _ptr(flags, _ip),
                                       *[int(p) for p in periodic], omega, xforce, rho_in,
                                       rho_out, calls, _ptr(f_in, _dp), _ptr(out, _dp))
        if rc != 0:
            raise KeyError(kernel)
        return out

    def verify(self, flags, periodic, f, omega, xforce) -> float:
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        f = np.ascontiguousarray(f, dtype=np.float64)
        err = ctypes.c_double(0.0)
        self.lib.ref_verify(nx, ny, nz, _ptr(flags, _ip), *[int(p) for p in periodic], omega,
                            xforce, _ptr(f, _dp), ctypes.byref(err))
        return err.value

    def initial_state(self, kernel, flags, periodic, omega):
        nz, ny, nx = flags.shape
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        out = np.zeros((Q, nx, ny, nz))
        self.lib.ref_initial_state(kernel.encode(), nx, ny, nz, _ptr(flags, _ip),
                                   *[int(p) for p in periodic], omega, _ptr(out, _dp))
        return out


# ---------------------------------------------------------------------------
# Seeded inputs shared by tests, fixtures and the CPU baseline
# ---------------------------------------------------------------------------

def equilibrium(rho, ux, uy, uz):
    """Incompressible D3Q19 equilibrium matching the reference's collision
    (src/kernel_pull_soa.c:128-198): w (rho - 1.5 u.u + 3 c.u + 4.5 (c.u)^2).
    Shapes broadcast; returns float64[19, ...]."""
    rho, ux, uy, uz = (np.asarray(a, dtype=np.float64) for a in (rho, ux, uy, uz))
    usq = ux * ux + uy * uy + uz * uz
    out = []
    for d in range(Q):
        cu = CX[d] * ux + CY[d] * uy + CZ[d] * uz
        out.append(W[d] * (rho - 1.5 * usq + 3.0 * cu + 4.5 * cu * cu))
    return np.stack(out)


def perturbed_state(flags, seed, amp=1e-4, rho=1.0):
    """Equilibrium at density rho with a seeded uniform velocity perturbation
    u ~ U(-amp, amp)^3 per fluid cell; obstacle entries are zero."""
    nz, ny, nx = flags.shape
    rng = np.random.default_rng(seed)
    u = rng.uniform(-amp, amp, size=(3, nx, ny, nz))
    f = equilibrium(np.full((nx, ny, nz), rho), u[0], u[1], u[2])
    fluid = np.transpose(flags, (2, 1, 0)) != 0
    f[:, ~fluid] = 0.0
    return f


def fluid_mask(flags):
    """bool[nx, ny, nz] of fluid cells."""
    return np.transpose(flags, (2, 1, 0)) != 0


def moments(f, flags):
    """rho, ux, uy, uz (momentum, as the reference computes it) per cell,
    zero on obstacles; each float64[nx, ny, nz]."""
    rho = f.sum(axis=0)
    ux = np.tensordot(CX.astype(np.float64), f, axes=(0, 0))
    uy = np.tensordot(CY.astype(np.float64), f, axes=(0, 0))
    uz = np.tensordot(CZ.astype(np.float64), f, axes=(0, 0))
    m = fluid_mask(flags)
    return [np.where(m, a, 0.0) for a in (rho, ux, uy, uz)]


# ---------------------------------------------------------------------------
# The benchmark workload, restated without the product library: the seeded
# porous channel and the counter-based perturbed equilibrium. The reference
# has no sphere generator or seeded initial state of its own; these are the
# inputs the benchmark feeds to both arms, so the reference arm builds them
# here and a CPU test checks them bit for bit against the product's C
# generator (lbm_porous_channel / lbm_perturbed_equilibrium).
# ---------------------------------------------------------------------------

_GOLDEN = np.uint64(0x9E3779B97F4A7C15)
_M1 = np.uint64(0xBF58476D1CE4E5B9)
_M2 = np.uint64(0x94D049BB133111EB)


def _mix64(z):
    """splitmix64 finaliser (Steele, Lea, Flood 2014), wrapping uint64."""
    z = (z ^ (z >> np.uint64(30))) * _M1
    z = (z ^ (z >> np.uint64(27))) * _M2
    return z ^ (z >> np.uint64(31))


def _u01(v):
    """Uniform double in [0, 1) from the top 53 bits."""
    return (v >> np.uint64(11)).astype(np.float64) * (1.0 / 9007199254740992.0)


def channel(dims):
    """The reference's `channel` geometry (src/lbm.c:52-187 with x forced
    periodic, src/lbm.c:96-102): obstacle cells at y, z in {0, n-1}.
    Returns int32[nz, ny, nx] flags."""
    nx, ny, nz = dims
    flags = np.ones((nz, ny, nx), dtype=np.int32)
    flags[:, [0, ny - 1], :] = 0
    flags[[0, nz - 1], :, :] = 0
    return flags


def porous_channel(dims, solid_fraction=0.2, rmin=4.0, rmax=8.0, seed=42):
    """Channel plus seeded solid spheres until the solid fraction (walls
    included) reaches `solid_fraction`: per sphere four splitmix64 draws
    (centre x, y, z uniform over the box, radius uniform in [rmin, rmax]);
    a cell is solid when its squared distance to the centre is <= r^2, with
    x wrapped periodically. Returns (flags, fraction, n_spheres)."""
    nx, ny, nz = dims
    flags = channel(dims)
    total = nx * ny * nz
    solid = int((flags == 0).sum())
    state = np.uint64(seed)
    spheres = 0
    with np.errstate(over="ignore"):
        while solid < solid_fraction * total:
            draws = []
            for _ in range(4):
                state = state + _GOLDEN
                draws.append(float(_u01(_mix64(np.array([state], dtype=np.uint64)))[0]))
            cxs, cys, czs = draws[0] * nx, draws[1] * ny, draws[2] * nz
            r = rmin + (rmax - rmin) * draws[3]
            ir = int(np.ceil(r))
            r2 = r * r
            d = np.arange(-ir - 1, ir + 2)
            zs = int(np.floor(czs)) + d
            ys = int(np.floor(cys)) + d
            xs = int(np.floor(cxs)) + d
            zs = zs[(zs >= 0) & (zs < nz)]
            ys = ys[(ys >= 0) & (ys < ny)]
            ez = (zs - czs)[:, None, None]
            ey = (ys - cys)[None, :, None]
            ex = (xs - cxs)[None, None, :]
            inside = (ex * ex + ey * ey) + ez * ez <= r2
            xw = xs % nx
            zi, yi, xi = np.nonzero(inside)
            sel = (zs[zi], ys[yi], xw[xi])
            hit = flags[sel] != 0
            flags[sel] = 0
            # a wrapped x can repeat within one sphere only if 2 ir + 3 > nx
            solid += int(np.unique(np.stack(sel)[:, hit], axis=1).shape[1]) \
                if 2 * ir + 3 > nx else int(hit.sum())
            spheres += 1
    return flags, solid / total, spheres


def counter_equilibrium(flags, seed, amplitude=1e-4, rho=1.0):
    """Equilibrium at density rho with a velocity perturbation drawn per
    fluid cell from a counter-based splitmix64 stream: cell c (f's cell
    order, z fastest) starts from seed ^ mix64(c * golden + 1) and takes
    three draws, u_k = amplitude (2 U - 1). Obstacle entries are 0.
    Returns float64[19, nx, ny, nz]."""
    nz, ny, nx = flags.shape
    n = nx * ny * nz
    c = np.arange(n, dtype=np.uint64)
    with np.errstate(over="ignore"):
        base = np.uint64(seed) ^ _mix64(c * _GOLDEN + np.uint64(1))
        u = []
        for _ in range(3):
            base = base + _GOLDEN
            u.append(amplitude * (2.0 * _u01(_mix64(base)) - 1.0))
    del base, c
    ux, uy, uz = (a.reshape(nx, ny, nz) for a in u)
    usq = ux * ux + uy * uy + uz * uz
    fluid = fluid_mask(flags)
    f = np.empty((Q, nx, ny, nz))
    for d in range(Q):
        cu = float(CX[d]) * ux + float(CY[d]) * uy + float(CZ[d]) * uz
        f[d] = W[d] * (((rho - 1.5 * usq) + 3.0 * cu) + 4.5 * cu * cu)
        f[d][~fluid] = 0.0
    return f


def normwise_errors(f, ref, flags):
    """Normwise relative errors of density and velocity of state f against
    state ref over the fluid cells: ||rho - rho_ref||_2 / ||rho_ref||_2 and
    ||u - u_ref||_2 / ||u_ref||_2 with u = j / rho the velocity vector
    (j the momentum sum_d c_d f_d). Returns (err_rho, err_u)."""
    m = fluid_mask(flags)

    def rho_u(a):
        rho = a[:, m].sum(axis=0)
        j = [np.tensordot(c.astype(np.float64), a[:, m], axes=(0, 0)) for c in (CX, CY, CZ)]
        return rho, [v / rho for v in j]

    r1, u1 = rho_u(f)
    r0, u0 = rho_u(ref)
    e_rho = float(np.linalg.norm(r1 - r0) / np.linalg.norm(r0))
    du = np.sqrt(sum(float(((a - b) ** 2).sum()) for a, b in zip(u1, u0)))
    nu = np.sqrt(sum(float((b * b).sum()) for b in u0))
    return e_rho, float(du / nu)
