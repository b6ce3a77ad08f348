"""Python binding of liblbmb200 (include/lbm_b200.h) over ctypes.

The compute path is the CUDA library; this module only marshals arrays. If
the library is missing, or no CUDA device is visible, solver construction
raises - there is no CPU fallback.

Array conventions (as the C ABI):
  flags  int32[nz, ny, nx]         latticeIndex order of LBM-Bench, x fastest
  f      float64[19, nx, ny, nz]   f[d, x, y, z], z fastest
  cell arrays  [nx, ny, nz]
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.environ.get("LBMB200_LIB") or os.path.join(HERE, "liblbmb200.so")

PUSH, PULL, AA = 0, 1, 2
F64, F32, F16 = 0, 1, 2
CKPT_AUTO = -1  # lbm_adjoint_gradient: least recomputation that fits in device memory
HALO_BEFORE, HALO_AFTER, HALO_SCATTER = 1, 2, 4
RING_ID_BYTES = 128
ERR_COMM, ERR_TIMEOUT = -7, -8
PATTERNS = {"push": PUSH, "pull": PULL, "aa": AA}
PRECISIONS = {"fp64": F64, "fp32": F32, "fp16": F16}
Q = 19

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_fp = ctypes.POINTER(ctypes.c_float)
_llp = ctypes.POINTER(ctypes.c_longlong)
_vp = ctypes.c_void_p


class LbmError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None

# (name, restype, argtypes) of every exported function
_SIGNATURES = [
    ("lbm_create", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  _ip, ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                  ctypes.c_int]),
    ("lbm_create_compact", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("lbm_is_compact", ctypes.c_int, [_vp]),
    ("lbm_compact_index", ctypes.c_int, [_vp, ctypes.c_longlong, ctypes.c_int, ctypes.c_int,
                                         _vp, _vp, ctypes.POINTER(ctypes.c_ulonglong)]),
    ("lbm_create_slab_compact", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int,
                                               ctypes.c_int, ctypes.c_int]),
    ("lbm_create_slab", ctypes.c_int, [ctypes.POINTER(_vp), ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, _ip, ctypes.c_int, ctypes.c_int,
                                       ctypes.c_int, ctypes.c_int]),
    ("lbm_set_pressure_bc", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double,
                                           ctypes.c_int]),
    ("lbm_halo_bytes", ctypes.c_size_t, [_vp]),
    ("lbm_halo_needs", ctypes.c_int, [_vp]),
    ("lbm_halo_shifted", ctypes.c_int, [_vp]),
    ("lbm_halo_pack", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    ("lbm_halo_unpack", ctypes.c_int, [_vp, ctypes.c_int, _vp, _vp]),
    ("lbm_stream", _vp, [_vp]),
    ("lbm_step_begin", ctypes.c_int, [_vp]),
    ("lbm_step_planes", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("lbm_step_end", ctypes.c_int, [_vp]),
    ("lbm_destroy", ctypes.c_int, [_vp]),
    ("lbm_set_params", ctypes.c_int, [_vp, ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                      ctypes.c_int]),
    ("lbm_set_fp16_scale", ctypes.c_int, [_vp, ctypes.c_double]),
    ("lbm_set_porosity", ctypes.c_int, [_vp, _fp, ctypes.c_double]),
    ("lbm_set_state", ctypes.c_int, [_vp, _dp]),
    ("lbm_save_state", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("lbm_load_state", ctypes.c_int, [_vp, ctypes.c_char_p]),
    ("lbm_get_state", ctypes.c_int, [_vp, _dp]),
    ("lbm_run", ctypes.c_int, [_vp, ctypes.c_int]),
    ("lbm_synchronize", ctypes.c_int, [_vp]),
    ("lbm_run_timed", ctypes.c_int, [_vp, ctypes.c_int, _dp]),
    ("lbm_time_launches", ctypes.c_int, [_vp, ctypes.c_int, _dp, _ip, _dp]),
    ("lbm_pin_host", ctypes.c_int, [_vp, ctypes.c_size_t]),
    ("lbm_unpin_host", ctypes.c_int, [_vp]),
    ("lbm_moments", ctypes.c_int, [_vp, _dp, _dp, _dp, _dp]),
    ("lbm_mass_momentum", ctypes.c_int, [_vp, _dp, _llp]),
    ("lbm_compare", ctypes.c_int, [_vp, _vp, _dp]),
    ("lbm_mass_momentum_noalloc", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int,
                                                 ctypes.c_int, _dp, _llp, _vp]),
    ("lbm_objective", ctypes.c_int, [_vp, _dp]),
    ("lbm_init_equilibrium", ctypes.c_int, [_vp, ctypes.c_ulonglong, ctypes.c_double,
                                            ctypes.c_double]),
    ("lbm_device_memory", ctypes.c_int, [ctypes.POINTER(ctypes.c_size_t),
                                         ctypes.POINTER(ctypes.c_size_t)]),
    ("lbm_adjoint_gradient", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int, _dp, _dp, _dp]),
    ("lbm_set_state_padded", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int]),
    ("lbm_get_state_padded", ctypes.c_int, [_vp, _vp, ctypes.c_int, ctypes.c_int]),
    ("lbm_fluid_cells", ctypes.c_longlong, [_vp]),
    ("lbm_steps_done", ctypes.c_longlong, [_vp]),
    ("lbm_device_bytes", ctypes.c_size_t, [_vp]),
    ("lbm_bytes_per_update", ctypes.c_double, [_vp]),
    ("lbm_launch_count", ctypes.c_longlong, [_vp]),
    ("lbm_last_error", ctypes.c_char_p, []),
    ("lbm_device_count", ctypes.c_int, []),
    ("lbm_geometry_create", ctypes.c_int, [ctypes.c_char_p, ctypes.c_int, ctypes.c_int,
                                           ctypes.c_int, _ip, _ip, _llp]),
    ("lbm_porous_channel", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                          ctypes.c_double, ctypes.c_double, ctypes.c_double,
                                          ctypes.c_ulonglong, _ip, _dp, _ip]),
    ("lbm_perturbed_equilibrium", ctypes.c_int, [ctypes.c_int, ctypes.c_int, ctypes.c_int, _ip,
                                                 ctypes.c_ulonglong, ctypes.c_double,
                                                 ctypes.c_double, _dp]),
    ("lbm_ring_unique_id", ctypes.c_int, [_vp]),
    ("lbm_ring_create", ctypes.c_int, [ctypes.POINTER(_vp), _vp, ctypes.c_int, ctypes.c_int, _vp,
                                       ctypes.c_int]),
    ("lbm_ring_run", ctypes.c_int, [_vp, ctypes.c_int, ctypes.c_int]),
    ("lbm_ring_gather", ctypes.c_int, [_vp]),
    ("lbm_ring_scatter", ctypes.c_int, [_vp]),
    ("lbm_ring_synchronize", ctypes.c_int, [_vp]),
    ("lbm_ring_exchanges", ctypes.c_longlong, [_vp]),
    ("lbm_ring_uses_nccl", ctypes.c_int, [_vp]),
    ("lbm_ring_destroy", ctypes.c_int, [_vp]),
]


def lib() -> ctypes.CDLL:
    """Loads liblbmb200.so (built by `make -C lbm-bench_b200`)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise FileNotFoundError(
                f"{LIB_PATH} is missing: build it with `make -C {HERE}` (the CUDA library is "
                "the only implementation; there is no CPU fallback)")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in _SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _lib = L
    return _lib


def _check(rc: int) -> None:
    if rc != 0:
        raise LbmError(rc, lib().lbm_last_error().decode(errors="replace"))


def _p(a: np.ndarray, kind):
    return a.ctypes.data_as(kind)


def device_count() -> int:
    return lib().lbm_device_count()


def device_memory():
    """(free, total) bytes of the current CUDA device."""
    f, t = ctypes.c_size_t(0), ctypes.c_size_t(0)
    _check(lib().lbm_device_memory(ctypes.byref(f), ctypes.byref(t)))
    return f.value, t.value


def _addr(buf) -> int:
    return buf if isinstance(buf, int) else buf.data_ptr()


class Solver:
    """One device lattice (include/lbm_b200.h lbm_create ... lbm_destroy)."""

    def __init__(self, flags, periodic=(1, 0, 0), pattern=AA, precision=F64, compact=False):
        """compact=True: the fluid-only layout (lbm_create_compact)."""
        if isinstance(pattern, str):
            pattern = PATTERNS[pattern]
        if isinstance(precision, str):
            precision = PRECISIONS[precision]
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        nz, ny, nx = flags.shape
        self.shape = (nx, ny, nz)
        self.flags = flags
        self.pattern, self.precision = pattern, precision
        self.periodic = tuple(int(p) for p in periodic)
        h = _vp()
        create = lib().lbm_create_compact if compact else lib().lbm_create
        _check(create(ctypes.byref(h), nx, ny, nz, _p(flags, _ip), *self.periodic, pattern,
                      precision))
        self._h = h

    @property
    def compact(self) -> bool:
        return lib().lbm_is_compact(self._h) == 1

    @classmethod
    def slab(cls, flags, periodic_yz=(0, 0), pattern=AA, precision=F64, compact=False):
        """x-slab of a decomposed domain (lbm_create_slab, or
        lbm_create_slab_compact with compact=True): `flags` has the slab's
        planes plus the neighbours' boundary planes at x = 0 and x = -1
        (shape (nz, ny, nx + 2))."""
        self = cls.__new__(cls)
        if isinstance(pattern, str):
            pattern = PATTERNS[pattern]
        if isinstance(precision, str):
            precision = PRECISIONS[precision]
        flags = np.ascontiguousarray(flags, dtype=np.int32)
        nz, ny, nxg = flags.shape
        nx = nxg - 2
        self.shape = (nx, ny, nz)
        self.flags = flags
        self.pattern, self.precision = pattern, precision
        self.periodic = (0,) + tuple(int(p) for p in periodic_yz)
        h = _vp()
        create = lib().lbm_create_slab_compact if compact else lib().lbm_create_slab
        _check(create(ctypes.byref(h), nx, ny, nz, _p(flags, _ip), *self.periodic[1:], pattern,
                      precision))
        self._h = h
        return self

    # -- halo exchange (slab solvers) --------------------------------------
    @property
    def halo_bytes(self) -> int:
        return lib().lbm_halo_bytes(self._h)

    @property
    def halo_needs(self) -> int:
        """Exchanges the next step takes: HALO_BEFORE | HALO_AFTER bits."""
        return lib().lbm_halo_needs(self._h)

    @property
    def halo_shifted(self) -> bool:
        """The state keeps boundary populations in the ghost planes: exchange
        HALO_BEFORE before reading it, HALO_SCATTER after setting it."""
        return bool(lib().lbm_halo_shifted(self._h))

    def halo_pack(self, when: int, to_left, to_right) -> None:
        """Writes the messages for the left and right neighbours into device
        buffers (integer addresses or objects with data_ptr())."""
        _check(lib().lbm_halo_pack(self._h, when, _addr(to_left), _addr(to_right)))

    def halo_unpack(self, when: int, from_left, from_right) -> None:
        _check(lib().lbm_halo_unpack(self._h, when, _addr(from_left), _addr(from_right)))

    @property
    def stream(self) -> int:
        """The solver's cudaStream_t as an integer."""
        return lib().lbm_stream(self._h) or 0

    # -- split steps (lbm_step_begin / _planes / _end) ----------------------
    def step_begin(self) -> None:
        _check(lib().lbm_step_begin(self._h))

    def step_planes(self, x_begin: int, x_end: int, side: bool = False) -> None:
        """Launches the open step on own planes [x_begin, x_end), on the
        solver's stream or (side=True) on its second stream."""
        _check(lib().lbm_step_planes(self._h, x_begin, x_end, int(side)))

    def step_end(self) -> None:
        _check(lib().lbm_step_end(self._h))

    # -- lifecycle ---------------------------------------------------------
    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().lbm_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # -- configuration -----------------------------------------------------
    def set_params(self, omega=1.0, lam=1.0 / 12.0, xforce=1e-5, force_on=False):
        _check(lib().lbm_set_params(self._h, omega, lam, xforce, int(force_on)))

    def set_pressure_bc(self, rho_in: float, rho_out: float, on: bool = True):
        """Zou-He pressure boundary after every step (lbm_set_pressure_bc):
        inlet cells (flag 2) on x = 0 at rho_in, outlet cells (flag 4) on
        x = nx-1 at rho_out."""
        _check(lib().lbm_set_pressure_bc(self._h, rho_in, rho_out, int(on)))

    def set_fp16_scale(self, scale: float):
        _check(lib().lbm_set_fp16_scale(self._h, scale))

    def set_porosity(self, porosity, alpha: float):
        por = np.ascontiguousarray(porosity, dtype=np.float32)
        _check(lib().lbm_set_porosity(self._h, _p(por, _fp), alpha))

    # -- state -------------------------------------------------------------
    def set_state(self, f):
        f = np.ascontiguousarray(f, dtype=np.float64)
        if f.shape != (Q,) + self.shape:
            raise ValueError(f"state shape {f.shape} != {(Q,) + self.shape}")
        _check(lib().lbm_set_state(self._h, _p(f, _dp)))

    def init_equilibrium(self, seed=1, amplitude=1e-4, rho=1.0):
        """Device-side lbm_perturbed_equilibrium (lbm_init_equilibrium)."""
        _check(lib().lbm_init_equilibrium(self._h, seed, amplitude, rho))

    def get_state(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty((Q,) + self.shape, dtype=np.float64)
        if out.shape != (Q,) + self.shape or out.dtype != np.float64 or \
                not out.flags.c_contiguous:
            raise ValueError("out must be a C-contiguous float64 array of the state's shape")
        _check(lib().lbm_get_state(self._h, _p(out, _dp)))
        return out

    def save_state(self, path: str) -> None:
        """Checkpoint: the state and the step count to a file (lbm_save_state)."""
        _check(lib().lbm_save_state(self._h, os.fsencode(path)))

    def load_state(self, path: str) -> None:
        """Resume from a file written by save_state (lbm_load_state)."""
        _check(lib().lbm_load_state(self._h, os.fsencode(path)))

    # -- stepping ----------------------------------------------------------
    def run(self, steps: int):
        _check(lib().lbm_run(self._h, int(steps)))

    def synchronize(self):
        _check(lib().lbm_synchronize(self._h))

    def run_timed(self, steps: int) -> float:
        ms = ctypes.c_double(0.0)
        _check(lib().lbm_run_timed(self._h, int(steps), ctypes.byref(ms)))
        return ms.value

    def time_launches(self, steps: int):
        """Runs `steps` steps with CUDA events around each launch. Returns
        ({kind: (ms_sum, launches)} for kinds pull, push, aa_even, aa_odd,
        region_ms from the first launch's start to the last one's end)."""
        ms = np.zeros(4)
        cnt = np.zeros(4, dtype=np.int32)
        region = ctypes.c_double(0.0)
        _check(lib().lbm_time_launches(self._h, int(steps), _p(ms, _dp), _p(cnt, _ip),
                                       ctypes.byref(region)))
        names = ("pull", "push", "aa_even", "aa_odd")
        return ({names[k]: (float(ms[k]), int(cnt[k])) for k in range(4) if cnt[k]},
                region.value)

    # -- observables -------------------------------------------------------
    def moments(self):
        q = [np.empty(self.shape) for _ in range(4)]
        _check(lib().lbm_moments(self._h, *[_p(a, _dp) for a in q]))
        return q

    def mass_momentum(self, check=True):
        out = np.zeros(4)
        bad = ctypes.c_longlong(0)
        rc = lib().lbm_mass_momentum(self._h, _p(out, _dp), ctypes.byref(bad))
        if check:
            _check(rc)
        return out, bad.value

    def compare(self, other: "Solver"):
        out = np.zeros(6)
        _check(lib().lbm_compare(self._h, other._h, _p(out, _dp)))
        return out

    def objective(self) -> float:
        j = ctypes.c_double(0.0)
        _check(lib().lbm_objective(self._h, ctypes.byref(j)))
        return j.value

    def adjoint_gradient(self, steps: int, checkpoint_every: int = 0):
        """dJ/dphi after `steps` Brinkman steps from the current state
        (lbm_adjoint_gradient). checkpoint_every: interval, 0 for the sqrt
        schedule, CKPT_AUTO for the least recomputation that fits in device
        memory. Returns (J, grad[nx, ny, nz], info dict)."""
        grad = np.zeros(self.shape)
        j = ctypes.c_double(0.0)
        info = np.zeros(6)
        _check(lib().lbm_adjoint_gradient(self._h, int(steps), int(checkpoint_every),
                                          _p(grad, _dp), ctypes.byref(j), _p(info, _dp)))
        keys = ("forward_ms", "reverse_ms", "interval", "checkpoints", "extra_bytes",
                "peak_bytes")
        return j.value, grad, dict(zip(keys, info.tolist()))

    @property
    def fluid_cells(self) -> int:
        return lib().lbm_fluid_cells(self._h)

    @property
    def steps_done(self) -> int:
        return lib().lbm_steps_done(self._h)

    @property
    def device_bytes(self) -> int:
        return lib().lbm_device_bytes(self._h)

    @property
    def bytes_per_update(self) -> float:
        return lib().lbm_bytes_per_update(self._h)

    @property
    def launch_count(self) -> int:
        return lib().lbm_launch_count(self._h)


def ring_unique_id() -> bytes:
    """The 128-byte NCCL id of a new ring (lbm_ring_unique_id; no GPU
    needed). Rank 0 makes it and every rank passes it to SlabRing."""
    buf = ctypes.create_string_buffer(RING_ID_BYTES)
    _check(lib().lbm_ring_unique_id(buf))
    return buf.raw


class SlabRing:
    """The native ring of one slab solver (lbm_ring_* in
    include/lbm_b200.h): halo messages to the ring neighbours over NCCL
    (rank - 1 and rank + 1, wrapped), the step loop issued from C.

    uid None with nranks 1: the slab is its own neighbour on both sides and
    the messages move by device copies. Every wait on the communicator or
    the stream is bounded by timeout_ms (0: 60 s); when one runs out the
    communicator is aborted and the call raises LbmError(ERR_TIMEOUT)."""

    def __init__(self, solver: Solver, rank: int = 0, nranks: int = 1, uid: bytes | None = None,
                 timeout_ms: int = 0):
        h = _vp()
        idbuf = None
        if uid is not None:
            if len(uid) != RING_ID_BYTES:
                raise ValueError(f"ring id must be {RING_ID_BYTES} bytes, got {len(uid)}")
            idbuf = ctypes.create_string_buffer(bytes(uid), RING_ID_BYTES)
        _check(lib().lbm_ring_create(ctypes.byref(h), solver._h, int(rank), int(nranks), idbuf,
                                     int(timeout_ms)))
        self._h = h
        self.solver = solver
        self.rank, self.nranks = int(rank), int(nranks)

    def run(self, steps: int, overlap: bool = False) -> None:
        """Enqueues `steps` steps with their exchanges (lbm_ring_run)."""
        _check(lib().lbm_ring_run(self._h, int(steps), int(overlap)))

    def gather(self) -> None:
        """Before reading the slab's state (lbm_ring_gather)."""
        _check(lib().lbm_ring_gather(self._h))

    def scatter(self) -> None:
        """After setting the slab's state (lbm_ring_scatter)."""
        _check(lib().lbm_ring_scatter(self._h))

    def synchronize(self) -> None:
        _check(lib().lbm_ring_synchronize(self._h))

    @property
    def exchanges(self) -> int:
        return lib().lbm_ring_exchanges(self._h)

    @property
    def uses_nccl(self) -> bool:
        return lib().lbm_ring_uses_nccl(self._h) == 1

    def close(self) -> None:
        """Destroys the ring (before its solver)."""
        if getattr(self, "_h", None):
            h, self._h = self._h, None
            _check(lib().lbm_ring_destroy(h))

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def pin(a: np.ndarray) -> None:
    """Page-locks a numpy array's buffer (lbm_pin_host)."""
    _check(lib().lbm_pin_host(a.ctypes.data, a.nbytes))


def unpin(a: np.ndarray) -> None:
    _check(lib().lbm_unpin_host(a.ctypes.data))


# ---------------------------------------------------------------------------
# host services
# ---------------------------------------------------------------------------

def geometry(kind: str, dims, periodic=(0, 0, 0)):
    """LBM-Bench geometries; returns (flags, periodic, (fluid, obstacle))."""
    nx, ny, nz = dims
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    per = np.array(periodic, dtype=np.int32)
    counts = np.zeros(2, dtype=np.int64)
    _check(lib().lbm_geometry_create(kind.encode(), nx, ny, nz, _p(per, _ip), _p(flags, _ip),
                                     _p(counts, _llp)))
    return flags, tuple(int(p) for p in per), (int(counts[0]), int(counts[1]))


def porous_channel(dims, solid_fraction=0.2, rmin=4.0, rmax=8.0, seed=42):
    """Channel plus seeded solid spheres; returns (flags, fraction, n_spheres)."""
    nx, ny, nz = dims
    flags = np.zeros((nz, ny, nx), dtype=np.int32)
    frac = ctypes.c_double(0.0)
    n = ctypes.c_int(0)
    _check(lib().lbm_porous_channel(nx, ny, nz, solid_fraction, rmin, rmax, seed,
                                    _p(flags, _ip), ctypes.byref(frac), ctypes.byref(n)))
    return flags, frac.value, n.value


def compact_index(fluid, nz=None):
    """The compact layout's index (lbm_compact_index) of fluid[rows, pitch]
    (bool/uint8, the first nz entries of each row used): returns
    (bits[rows, W], base[rows, W], total) as uint32 arrays and an int."""
    fluid = np.ascontiguousarray(fluid, dtype=np.uint8)
    rows, pitch = fluid.shape
    nz = pitch if nz is None else nz
    W = (nz + 31) // 32
    bits = np.zeros((rows, W), dtype=np.uint32)
    base = np.zeros((rows, W), dtype=np.uint32)
    total = ctypes.c_ulonglong(0)
    _check(lib().lbm_compact_index(fluid.ctypes.data, rows, nz, pitch, bits.ctypes.data,
                                   base.ctypes.data, ctypes.byref(total)))
    return bits, base, int(total.value)


def perturbed_equilibrium(flags, seed=1, amplitude=1e-4, rho=1.0):
    flags = np.ascontiguousarray(flags, dtype=np.int32)
    nz, ny, nx = flags.shape
    f = np.empty((Q, nx, ny, nz))
    _check(lib().lbm_perturbed_equilibrium(nx, ny, nz, _p(flags, _ip), seed, amplitude, rho,
                                           _p(f, _dp)))
    return f



# ---------------------------------------------------------------------------
# drop-in kernels through the reference's own structs (lbm_b200_dropin.h)
# ---------------------------------------------------------------------------

class LatticeDesc(ctypes.Structure):
    """LatticeDescType of the reference (src/lbm.h:54-66)."""
    _fields_ = [("Dims", ctypes.c_int * 3), ("Lattice", ctypes.POINTER(ctypes.c_int)),
                ("nCells", ctypes.c_int), ("nFluid", ctypes.c_int), ("nObst", ctypes.c_int),
                ("nInlet", ctypes.c_int), ("nOutlet", ctypes.c_int), ("PeriodicX", ctypes.c_int),
                ("PeriodicY", ctypes.c_int), ("PeriodicZ", ctypes.c_int),
                ("Name", ctypes.c_char_p)]


def _dropin_types(pdf):
    """ctypes mirrors of CaseDataType, KernelDataType and KernelFunctionsType
    (src/lbm.h:68-106) for PdfType = pdf (c_double, or c_float in a
    PRECISION_SP build)."""

    class CaseData(ctypes.Structure):
        _fields_ = [("Omega", pdf), ("RhoIn", pdf), ("RhoOut", pdf), ("XForce", pdf),
                    ("MaxIterations", ctypes.c_int), ("StatisticsModulus", ctypes.c_int)]

    class KernelData(ctypes.Structure):
        pass

    node_fn = ctypes.CFUNCTYPE(None, ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int,
                               ctypes.c_int, ctypes.POINTER(pdf))
    bcget_fn = ctypes.CFUNCTYPE(None, ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int, ctypes.POINTER(pdf))
    bcset_fn = ctypes.CFUNCTYPE(None, ctypes.POINTER(KernelData), ctypes.c_int, ctypes.c_int,
                                ctypes.c_int, ctypes.c_int, pdf)
    kernel_fn = ctypes.CFUNCTYPE(None, ctypes.POINTER(LatticeDesc), ctypes.POINTER(KernelData),
                                 ctypes.POINTER(CaseData))
    KernelData._fields_ = [
        ("Pdfs", ctypes.POINTER(pdf) * 2), ("PdfsActive", ctypes.POINTER(pdf)),
        ("Dims", ctypes.c_int * 3), ("GlobalDims", ctypes.c_int * 3), ("Offsets", ctypes.c_int * 3),
        ("BounceBackPdfsSrc", ctypes.POINTER(ctypes.c_int)),
        ("BounceBackPdfsDst", ctypes.POINTER(ctypes.c_int)), ("nBounceBackPdfs", ctypes.c_int),
        ("Blk", ctypes.c_int * 3), ("Iteration", ctypes.c_int), ("LoopBalance", ctypes.c_double),
        ("Duration", ctypes.c_double), ("GetNode", node_fn), ("SetNode", node_fn),
        ("BoundaryConditionsGetPdf", bcget_fn), ("BoundaryConditionsSetPdf", bcset_fn),
        ("Kernel", kernel_fn)]
    init_fn = ctypes.CFUNCTYPE(None, ctypes.POINTER(LatticeDesc),
                               ctypes.POINTER(ctypes.POINTER(KernelData)), ctypes.POINTER(CaseData))
    deinit_fn = ctypes.CFUNCTYPE(None, ctypes.POINTER(LatticeDesc),
                                 ctypes.POINTER(ctypes.POINTER(KernelData)))

    class KernelFunctions(ctypes.Structure):
        _fields_ = [("Name", ctypes.c_char_p), ("Init", init_fn), ("Deinit", deinit_fn)]

    return CaseData, KernelData, KernelFunctions


# the reference's default (double) build
CaseData, KernelData, KernelFunctions = _dropin_types(ctypes.c_double)
CaseDataSP, KernelDataSP, KernelFunctionsSP = _dropin_types(ctypes.c_float)
LIB_PATH_SP = os.path.join(HERE, "liblbmb200_sp.so")
_lib_sp = None


def lib_sp():
    """liblbmb200_sp.so: the drop-in kernels for a PRECISION_SP build."""
    global _lib_sp
    if _lib_sp is None:
        if not os.path.exists(LIB_PATH_SP):
            raise OSError(f"{LIB_PATH_SP} not built (make -C lbm-bench_b200)")
        _lib_sp = ctypes.CDLL(LIB_PATH_SP)
    return _lib_sp


def _registry(sp=False):
    L = lib_sp() if sp else lib()
    kf = KernelFunctionsSP if sp else KernelFunctions
    n = ctypes.c_int.in_dll(L, "LBM_B200_N_KERNELS").value
    return (kf * n).in_dll(L, "LbmB200Kernels")


def dropin_kernels(sp=False):
    """Names in the library's registry (LbmB200Kernels)."""
    return [k.Name.decode() for k in _registry(sp)]


class DropIn:
    """One kernel of the drop-in registry driven the way LBM-Bench's driver
    drives a kernel (src/main.c:93-152): look up by name, Init, SetNode,
    Kernel, GetNode, Deinit."""

    def __init__(self, name, flags, periodic, omega=1.0, xforce=1e-5, iterations=10,
                 force_on=None, lam=None, sp=False):
        L = lib_sp() if sp else lib()
        self.sp = sp
        pdf = ctypes.c_float if sp else ctypes.c_double
        case_t = CaseDataSP if sp else CaseData
        self.kf = next((k for k in _registry(sp) if k.Name.decode() == name), None)
        if self.kf is None:
            raise KeyError(name)
        self.aos = "-aos" in name
        L.lbmB200SetBodyForce.argtypes = [ctypes.c_int]
        L.lbmB200SetMagicParameter.argtypes = [ctypes.c_double]
        L.lbmB200SetBodyForce(-1 if force_on is None else int(force_on))
        L.lbmB200SetMagicParameter(1.0 / 12.0 if lam is None else lam)
        self.flags = np.ascontiguousarray(flags, dtype=np.int32)
        nz, ny, nx = self.flags.shape
        self.shape = (nx, ny, nz)
        self.ld = LatticeDesc()
        self.ld.Dims[:] = [nx, ny, nz]
        self.ld.Lattice = self.flags.ctypes.data_as(ctypes.POINTER(ctypes.c_int))
        self.ld.nCells = nx * ny * nz
        self.ld.nFluid = int((self.flags != 0).sum())
        self.ld.nObst = self.ld.nCells - self.ld.nFluid
        self.ld.PeriodicX, self.ld.PeriodicY, self.ld.PeriodicZ = (int(p) for p in periodic)
        self.ld.Name = b"python"
        self.cd = case_t(omega, 1.0, 1.0, xforce, iterations, 100)
        self.kd = ctypes.POINTER(KernelDataSP if sp else KernelData)()
        self.kf.Init(ctypes.byref(self.ld), ctypes.byref(self.kd), ctypes.byref(self.cd))
        self._buf = (pdf * Q)()

    @property
    def data(self) -> KernelData:
        return self.kd.contents

    def pdfs(self, which: int) -> np.ndarray:
        """Zero-copy view of kd->Pdfs[which], shape [19, nx+2, ny+2, nz+2]
        (indexSoA; for the AoS kernels a transposed view of indexAoS)."""
        g = tuple(self.data.GlobalDims)
        n = Q * g[0] * g[1] * g[2]
        a = np.ctypeslib.as_array(self.data.Pdfs[which], shape=(n,))
        if self.aos:
            return np.moveaxis(a.reshape(g + (Q,)), -1, 0)
        return a.reshape((Q,) + g)

    def set_state(self, f):
        """f[19, nx, ny, nz] for fluid cells, written through kd->SetNode."""
        fl = np.transpose(self.flags, (2, 1, 0)) != 0
        for x, y, z in np.argwhere(fl):
            self._buf[:] = f[:, x, y, z]
            self.data.SetNode(self.kd, int(x), int(y), int(z), self._buf)

    def get_state(self):
        """f[19, nx, ny, nz] read through kd->GetNode (0 on obstacles)."""
        out = np.zeros((Q,) + self.shape)
        fl = np.transpose(self.flags, (2, 1, 0)) != 0
        for x, y, z in np.argwhere(fl):
            self.data.GetNode(self.kd, int(x), int(y), int(z), self._buf)
            out[:, x, y, z] = self._buf[:]
        return out

    def run(self, iterations=None):
        """kd->Kernel(ld, kd, cd); returns kd->Duration (s, step loop only)."""
        if iterations is not None:
            self.cd.MaxIterations = int(iterations)
        self.data.Kernel(ctypes.byref(self.ld), self.kd, ctypes.byref(self.cd))
        return self.data.Duration

    def close(self):
        if getattr(self, "kd", None):
            self.kf.Deinit(ctypes.byref(self.ld), ctypes.byref(self.kd))
            self.kd = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()
