"""Host-side logic of liblbmb200 that needs no GPU: geometry generators, the
seeded initial state, the exported C ABI, and the loud failure of the
product path when no CUDA device is present."""
import ctypes
import os
import re

import numpy as np
import pytest

import golden_io
import lbmb200 as L
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
INCLUDE = os.path.join(ROOT, "include")

GEOMS = [("channel", (12, 10, 14), (0, 0, 0)), ("box", (10, 9, 8), (1, 1, 0)),
         ("box", (7, 8, 9), (0, 0, 0)), ("box", (7, 8, 9), (0, 1, 1)),
         ("pipe", (9, 12, 11), (0, 0, 0)), ("pipe", (5, 20, 14), (0, 1, 0)),
         ("blocks", (20, 18, 17), (0, 0, 0)), ("blocks-3", (13, 11, 9), (0, 0, 0)),
         ("blocks-0", (17, 17, 17), (0, 0, 0)), ("fluid", (6, 7, 5), (0, 0, 0)),
         ("CHANNEL", (4, 5, 6), (0, 0, 1))]


@pytest.mark.parametrize("kind,dims,per", GEOMS)
def test_geometry_matches_reference_rules(kind, dims, per):
    flags, per_out, counts = L.geometry(kind, dims, per)
    ref = golden_io.reference_geometry(kind, dims, per)
    assert np.array_equal(flags != 0, ref != 0)
    assert counts == (int((ref != 0).sum()), int((ref == 0).sum()))
    if O.ref_available("verify"):
        rflags, rper, rcounts = O.Reference("verify").geometry(kind, dims, per)
        assert np.array_equal(flags != 0, rflags != 0)
        assert per_out == rper
        assert counts == rcounts


def test_geometry_unknown_type_is_an_error():
    with pytest.raises(L.LbmError):
        L.geometry("sphere", (4, 4, 4))


def test_porous_channel_is_seeded_and_reaches_fraction():
    a, fa, na = L.porous_channel((48, 40, 36), 0.2, 3.0, 5.0, seed=3)
    b, fb, nb = L.porous_channel((48, 40, 36), 0.2, 3.0, 5.0, seed=3)
    c, _, _ = L.porous_channel((48, 40, 36), 0.2, 3.0, 5.0, seed=4)
    assert np.array_equal(a, b) and fa == fb and na == nb
    assert not np.array_equal(a, c)
    assert 0.2 <= fa < 0.2 + 0.05
    assert fa == pytest.approx((a == 0).mean())
    # channel walls are there, x is periodic (no x walls)
    assert np.all(a[:, 0, :] == 0) and np.all(a[:, -1, :] == 0)
    assert np.all(a[0, :, :] == 0) and np.all(a[-1, :, :] == 0)
    assert (a[:, :, 0] != 0).any()


def test_porous_channel_spheres_wrap_in_x():
    flags, _, n = L.porous_channel((16, 40, 40), 0.3, 6.0, 7.0, seed=11)
    # with radius >= 6 on a 16-long periodic axis, some sphere crosses x=0
    interior = flags[1:-1, 1:-1, :] == 0
    assert (interior[:, :, 0] & interior[:, :, -1]).any()


def test_porous_channel_bad_args():
    with pytest.raises(L.LbmError):
        L.porous_channel((8, 8, 8), 0.99, 2, 3)
    with pytest.raises(L.LbmError):
        L.porous_channel((8, 8, 8), 0.2, 3, 2)


def test_perturbed_equilibrium_moments():
    flags, _, _ = L.geometry("channel", (10, 9, 8))
    f = L.perturbed_equilibrium(flags, seed=5, amplitude=1e-3, rho=1.0)
    g = L.perturbed_equilibrium(flags, seed=5, amplitude=1e-3, rho=1.0)
    assert np.array_equal(f, g)
    rho, ux, uy, uz = O.moments(f, flags)
    m = O.fluid_mask(flags)
    assert np.allclose(rho[m], 1.0, atol=1e-15)
    for u in (ux, uy, uz):
        assert np.abs(u[m]).max() <= 1e-3 * (1 + 1e-12)
        assert np.abs(u[m]).max() > 5e-4
    assert np.all(f[:, ~m] == 0.0)
    # equals the oracle module's equilibrium for the same velocities
    assert np.allclose(f[:, m], O.equilibrium(rho[m], ux[m], uy[m], uz[m]), atol=1e-17)


def _declared_functions():
    names = []
    for fn in os.listdir(INCLUDE):
        if not fn.endswith(".h"):
            continue
        src = open(os.path.join(INCLUDE, fn)).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names += re.findall(r"^\s*(?:const\s+)?[A-Za-z_][\w\s\*]*?\b([A-Za-z_]\w*)\s*\(",
                            src, flags=re.M)
    return sorted(set(n for n in names if n not in ("defined",)))


def test_library_exports_every_declared_symbol():
    lib = L.lib()
    names = _declared_functions()
    assert "lbm_create" in names and "lbm_run" in names
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


@pytest.mark.skipif(L.device_count() > 0, reason="a CUDA device is present")
def test_product_path_fails_loudly_without_gpu():
    flags, per, _ = L.geometry("channel", (8, 8, 8))
    with pytest.raises(L.LbmError) as e:
        L.Solver(flags, per)
    assert e.value.code == -6
    assert "no CPU path" in str(e.value)


@pytest.mark.parametrize("dims,frac,rmin,rmax,seed", [
    ((40, 36, 44), 0.2, 4.0, 8.0, 42), ((64, 48, 32), 0.3, 6.0, 12.0, 5),
    ((8, 30, 26), 0.25, 4.0, 8.0, 3),  # 2r + 3 > nx: one sphere wraps onto itself in x
    ((17, 19, 23), 0.0, 4.0, 8.0, 1)])
def test_oracle_workload_equals_product_generator(dims, frac, rmin, rmax, seed):
    """The benchmark's reference arm builds its inputs with the oracle's
    numpy restatement; it must be bit-identical to the product's C
    generator so both arms run the same workload."""
    flags, f_frac, n_sph = L.porous_channel(dims, frac, rmin, rmax, seed=seed)
    oflags, o_frac, o_sph = O.porous_channel(dims, frac, rmin, rmax, seed=seed)
    assert np.array_equal(flags, oflags)
    assert (f_frac, n_sph) == (o_frac, o_sph)
    f = L.perturbed_equilibrium(flags, seed=7, amplitude=1e-4)
    fo = O.counter_equilibrium(oflags, 7, 1e-4)
    assert f.tobytes() == fo.tobytes()


def _rank(fluid):
    """Storage number of every cell in row order (fluid cells only; -1 else)."""
    flat = fluid.reshape(-1).astype(bool)
    num = np.cumsum(flat) - 1
    return np.where(flat, num, -1).reshape(fluid.shape)


@pytest.mark.parametrize("rows,nz,pitch,seed", [(7, 45, 48, 1), (5, 32, 32, 2), (3, 96, 112, 3),
                                                (11, 1, 16, 4), (4, 70, 80, 5)])
def test_compact_index_words_and_bases(rows, nz, pitch, seed):
    """lbm_compact_index: one fluid bit per z, and per 32-cell word the
    number of fluid cells before it in row order; row padding beyond nz is
    ignored."""
    rng = np.random.default_rng(seed)
    fluid = rng.uniform(size=(rows, pitch)) > 0.3
    bits, base, total = L.compact_index(fluid, nz)
    f = fluid[:, :nz]
    assert total == int(f.sum())
    rank = _rank(f)
    for r in range(rows):
        for z in range(nz):
            w, b = divmod(z, 32)
            assert bool((int(bits[r, w]) >> b) & 1) == bool(f[r, z])
            if f[r, z]:
                below = int(bits[r, w]) & ((1 << b) - 1)
                assert int(base[r, w]) + bin(below).count("1") == rank[r, z]


def test_compact_neighbour_identities():
    """The step kernels find a fluid neighbour (row q, z + dz) of a lane at
    z from row q's word at z alone: B_q = base + popc(word & bits below z),
    f_q = bit z; (q, z) -> B_q, (q, z + 1) -> B_q + f_q, (q, z - 1) -> B_q - 1.
    Checked here for every fluid cell and D3Q19 neighbour of a random box,
    x and y periodic (rows wrap), z not (no wrap needed), nz = 70 so the
    z +- 1 neighbours cross word boundaries."""
    rng = np.random.default_rng(9)
    nx, ny, nz = 6, 5, 70
    fluid = rng.uniform(size=(nx, ny, nz)) > 0.35
    bits, base, _ = L.compact_index(fluid.reshape(nx * ny, nz), nz)
    rank = _rank(fluid)
    checked = 0
    for x in range(nx):
        for y in range(ny):
            for z in range(nz):
                if not fluid[x, y, z]:
                    continue
                w, b = divmod(z, 32)
                for d in range(19):
                    xx, yy, zz = (x + O.CX[d]) % nx, (y + O.CY[d]) % ny, z + O.CZ[d]
                    if not (0 <= zz < nz) or not fluid[xx, yy, zz]:
                        continue  # a wall: the mask says so, no index is needed
                    row = xx * ny + yy
                    word = int(bits[row, w])
                    bq = int(base[row, w]) + bin(word & ((1 << b) - 1)).count("1")
                    fq = (word >> b) & 1
                    idx = bq + fq if O.CZ[d] > 0 else bq - 1 if O.CZ[d] < 0 else bq
                    assert idx == rank[xx, yy, zz], (x, y, z, d)
                    checked += 1
    assert checked > 10000


def _prefetch_slices(bits, base, nx, ny, W, nblk, xp):
    """The slices of plane xp that the nblk blocks of one plane ask the L2
    for in the compact AA odd step (cp_plane_prefetch, lbm_step_cp.cuh):
    [s, e) from the base of the plane's first index word to the end of its
    last, split in ceil((e - s) / nblk) cells per block."""
    kb = xp * ny * W
    s = int(base.reshape(-1)[kb])
    ke = kb + ny * W - 1
    e = int(base.reshape(-1)[ke]) + bin(int(bits.reshape(-1)[ke])).count("1")
    chunk = (e - s + nblk - 1) // nblk
    out = []
    for part in range(nblk):
        cb = s + chunk * part
        if cb < e:
            out.append((cb, min(cb + chunk, e)))
    return s, e, out


@pytest.mark.parametrize("dims,nblk", [((24, 20, 70), 20), ((16, 9, 36), 9), ((12, 8, 200), 16),
                                       ((10, 6, 33), 200)])
def test_compact_prefetch_slices_stay_in_bounds(dims, nblk):
    """The L2 prefetch of the compact AA odd step widens each block's slice
    to 16-byte bounds. For every plane the slices must tile exactly the
    plane's stored cells, and the widened byte ranges must stay inside one
    population plane (stride rounded up to 256 bytes) and inside the mask
    array (padded to the same stride), in FP64, FP32 and FP16 storage."""
    nx, ny, nz = dims
    rng = np.random.default_rng(nx * ny + nz)
    fluid = rng.uniform(size=(nx, ny, nz)) > 0.25
    bits, base, total = L.compact_index(fluid.reshape(nx * ny, nz), nz)
    W = bits.shape[1]
    starts = []
    for xp in range(nx):
        s, e, sl = _prefetch_slices(bits, base, nx, ny, W, nblk, xp)
        assert e - s == int(fluid[xp].sum())
        starts.append(s)
        covered = 0
        for cb, ce in sl:
            assert s <= cb < ce <= e
            covered += ce - cb
        assert covered == e - s
        for size in (8, 4, 2):
            plane = (total + 256 // size - 1) // (256 // size) * (256 // size)
            for cb, ce in sl:
                lo, hi = (cb * size) & ~15, (ce * size + 15) & ~15
                assert 0 <= lo < hi <= plane * size
                lo4, hi4 = (cb * 4) & ~15, (ce * 4 + 15) & ~15
                assert 0 <= lo4 < hi4 <= plane * 4
    assert starts == sorted(starts)
