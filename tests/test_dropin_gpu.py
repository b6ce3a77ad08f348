"""The drop-in kernels driven through LBM-Bench's own structs and calling
sequence (Init, SetNode, Kernel, GetNode, Deinit), on a B200: bit-identical
to the reference's kernels on the golden fixtures, and the lbmbench-b200
driver's -V Poiseuille run for every registered kernel."""
import ctypes
import os
import re
import subprocess

import numpy as np
import pytest

import golden_io
import lbmb200 as L
import oracle as O

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CLI = os.path.join(ROOT, "lbm-bench_b200", "lbmbench-b200")
CASES, _ = golden_io.load()
STEP_CASES = [c for c in CASES if "verify" not in c and "pressure" not in c]
PRESSURE_CASES = [c for c in CASES if "pressure" in c]


@pytest.mark.parametrize("kernel", ["cuda-pull-soa", "cuda-push-soa", "cuda-aa-soa"])
@pytest.mark.parametrize("case", STEP_CASES, ids=[c["name"] for c in STEP_CASES])
def test_dropin_bit_identical_to_reference_fixtures(golden, case, kernel):
    _, arrays = golden
    flags = golden_io.build_flags(case, arrays)
    f0 = golden_io.initial_state(case, flags)
    with L.DropIn(kernel, flags, case["periodic"], omega=case["omega"], xforce=case["xforce"],
                  iterations=case["steps"], force_on=bool(case["force_on"]),
                  lam=case["lambda"]) as k:
        k.set_state(f0)
        k.run()
        out = k.get_state()
        data = k.data
        assert data.Duration > 0.0
        if kernel == "cuda-aa-soa":
            assert data.Iteration == case["steps"] - 1
    assert golden_io.state_digest(out, flags) == case["sha256"]


LAYOUT_VARIANTS = ["cuda-pull-aos", "cuda-push-aos", "cuda-blk-push-soa", "cuda-blk-pull-soa"]
SOA_OF = {"cuda-pull-aos": "cuda-pull-soa", "cuda-push-aos": "cuda-push-soa",
          "cuda-blk-push-soa": "cuda-push-soa", "cuda-blk-pull-soa": "cuda-pull-soa"}


@pytest.mark.parametrize("kernel", LAYOUT_VARIANTS)
@pytest.mark.parametrize("case", STEP_CASES[:6], ids=[c["name"] for c in STEP_CASES[:6]])
def test_layout_variants_bit_identical_to_reference_fixtures(golden, case, kernel):
    """The reference's pull-aos / push-aos / blk-*-soa kernels give its SoA
    kernels' results; so do these names."""
    _, arrays = golden
    flags = golden_io.build_flags(case, arrays)
    f0 = golden_io.initial_state(case, flags)
    with L.DropIn(kernel, flags, case["periodic"], omega=case["omega"], xforce=case["xforce"],
                  iterations=case["steps"], force_on=bool(case["force_on"]),
                  lam=case["lambda"]) as k:
        k.set_state(f0)
        k.run()
        out = k.get_state()
        assert tuple(k.data.Blk) == ((8, 8, 8) if "blk" in kernel else tuple(k.data.GlobalDims))
    assert golden_io.state_digest(out, flags) == case["sha256"]


@pytest.mark.parametrize("kernel", ["cuda-pull-aos", "cuda-push-aos"])
@pytest.mark.parametrize("steps", [1, 4])
def test_aos_host_arrays_are_the_soa_arrays_transposed(kernel, steps):
    """After Kernel, every slot of both host lattices (ghost layer and the
    zeros of slots that hold no population included) equals the SoA
    kernel's, in indexAoS order."""
    flags, per, _ = L.geometry("blocks-3", (13, 10, 11))
    f0 = L.perturbed_equilibrium(flags, seed=steps, amplitude=2e-3)
    arrays = {}
    for name in (kernel, SOA_OF[kernel]):
        with L.DropIn(name, flags, per, omega=1.3, iterations=steps, force_on=True) as k:
            k.set_state(f0)
            k.run()
            # DropIn.pdfs reads the AoS kernel's arrays in indexAoS order
            arrays[name] = [k.pdfs(b).copy() for b in (0, 1)]
    for b in (0, 1):
        assert np.array_equal(arrays[kernel][b], arrays[SOA_OF[kernel]][b])


def test_dropin_ends_in_the_buffer_the_reference_ends_in():
    flags, per, _ = L.geometry("channel", (10, 9, 8))
    f0 = L.perturbed_equilibrium(flags, seed=3)
    with L.DropIn("cuda-pull-soa", flags, per, omega=1.2, iterations=3, force_on=True) as k:
        k.set_state(f0)
        k.run()
        # three pointer swaps: the state is in Pdfs[1] (src/kernel_pull_soa.c:211-217)
        addr = lambda p: ctypes.cast(p, ctypes.c_void_p).value  # noqa: E731
        assert addr(k.data.PdfsActive) == addr(k.data.Pdfs[1])
        # the oracle agrees with what GetNode reads
        ref = O.Oracle().run(flags, per, f0, 3, 1.2, 1 / 12, 1e-5, True)
        m = O.fluid_mask(flags)
        assert np.array_equal(k.get_state()[:, m], ref[:, m])


def test_dropin_aa_odd_iteration_count_runs_pairs():
    flags, per, _ = L.geometry("channel", (8, 7, 9))
    f0 = L.perturbed_equilibrium(flags, seed=5)
    with L.DropIn("cuda-aa-soa", flags, per, omega=1.1, iterations=5, force_on=True) as k:
        k.set_state(f0)
        k.run()
        assert k.data.Iteration == 5  # six steps, as src/kernel_aa_soa.c:36 runs them
        ref = O.Oracle().run(flags, per, f0, 6, 1.1, 1 / 12, 1e-5, True)
        m = O.fluid_mask(flags)
        assert np.array_equal(k.get_state()[:, m], ref[:, m])


def test_dropin_reduced_precision_tracks_fp64():
    flags, per, _ = L.geometry("blocks-4", (24, 20, 18))
    f0 = L.perturbed_equilibrium(flags, seed=9, amplitude=1e-3)
    m = O.fluid_mask(flags)
    ref = O.Oracle().run(flags, per, f0, 10, 1.3, 1 / 12, 1e-5, True)
    for name, tol in (("cuda-aa-soa-fp32", 1e-6), ("cuda-pull-soa-fp16", 2e-4)):
        with L.DropIn(name, flags, per, omega=1.3, iterations=10, force_on=True) as k:
            k.set_state(f0)
            k.run()
            out = k.get_state()
        assert np.abs(out[:, m] - ref[:, m]).max() < tol, name


@pytest.mark.parametrize("kernel", ["cuda-pull-soa", "cuda-push-soa", "cuda-aa-soa"])
def test_dropin_single_precision_build(kernel):
    """liblbmb200_sp.so, for a reference built with PRECISION_SP (PdfType
    float, src/lbm.h:48-52): float host lattices and CaseData, FP32 device
    storage, results within FP32 rounding of the FP64 oracle."""
    flags, per, _ = L.geometry("blocks-4", (22, 18, 20))
    f0 = L.perturbed_equilibrium(flags, seed=13, amplitude=1e-3)
    m = O.fluid_mask(flags)
    ref = O.Oracle().run(flags, per, f0, 8, 1.4, 1 / 12, 1e-5, True)
    with L.DropIn(kernel, flags, per, omega=1.4, iterations=8, force_on=True, sp=True) as k:
        assert ctypes.sizeof(k.data.Pdfs[0]._type_) == 4
        assert k.data.LoopBalance == 2 * 19 * 4
        k.set_state(f0)
        k.run()
        # pull / push end in Pdfs[0] after an even number of swaps; AA in its one lattice
        addr = lambda p: ctypes.cast(p, ctypes.c_void_p).value  # noqa: E731
        assert addr(k.data.PdfsActive) == addr(k.data.Pdfs[0])
        out = k.get_state()
        assert out.dtype == np.float64
    err = np.abs(out[:, m] - ref[:, m]).max()
    assert 0 < err < 1e-6


@pytest.mark.parametrize("kernel", L.dropin_kernels() if os.path.exists(L.LIB_PATH) else [])
def test_cli_verification_run_succeeds(kernel):
    """The reference's test.sh runs `lbmbench -V -k K` for every kernel `-l`
    lists and requires exit status 0 (src/test.sh:61-74, 101-103)."""
    r = subprocess.run([CLI, "-V", "-k", kernel], capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stdout + r.stderr
    assert "# VERIFICATION SUCCEEDED." in r.stdout
    err = float(re.search(r"deviation from analytical solution: (\S+)", r.stdout).group(1))
    if not kernel.endswith(("-fp32", "-fp16")):
        # the reference's own -V run on this case gives 4.5614e-02 (golden fixture)
        ref = next(c for c in CASES if c["name"] == "poiseuille_V")["verify"]["aa-soa"]
        assert err == pytest.approx(ref["error_norm"], rel=1e-6)
    else:
        assert err < 0.06


REF_DROPIN = {p: os.path.join(ROOT, "oracle", "_ref", f"lbmbench-dropin-{p}") for p in ("dp", "sp")}


def _kernels_listed(exe):
    out = subprocess.run([exe, "-l"], capture_output=True, text=True, check=True).stdout
    lines = out.splitlines()
    return [ln.split()[0] for ln in lines[lines.index("Available kernels:") + 1:] if ln.strip()]


@pytest.mark.parametrize("prec", ["dp", "sp"])
def test_reference_binary_with_dropin_rows_passes_its_own_verification(prec):
    """The reference's own driver, linked against liblbmb200 with the
    drop-in rows in GKernels[] and nothing else changed (oracle/Makefile):
    what src/test.sh:95-103 does - `-V -k K` for every kernel `-l` lists,
    exit status 0 - for the reference's seven names and the 13 cuda-* rows.
    In the double build the cuda pull/push/AA names (all FP64) give exactly
    the error norm the same binary's own kernels give."""
    exe = REF_DROPIN[prec]
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/lbmbench-dropin-* not built (needs the reference sources)")
    errs = {}
    for k in _kernels_listed(exe):
        r = subprocess.run([exe, "-V", "-k", k], capture_output=True, text=True, timeout=300)
        assert r.returncode == 0, (k, r.stdout[-2000:] + r.stderr[-2000:])
        assert "# VERIFICATION SUCCEEDED." in r.stdout, k
        errs[k] = float(re.search(r"deviation from analytical solution: (\S+)",
                                  r.stdout).group(1))
    assert len(errs) == 20
    if prec == "dp":
        for k in ("cuda-pull-soa", "cuda-push-soa", "cuda-aa-soa", "cuda-pull-aos",
                  "cuda-push-aos", "cuda-blk-push-soa", "cuda-blk-pull-soa"):
            assert errs[k] == errs["aa-soa"], (k, errs[k], errs["aa-soa"])
        assert errs["aa-soa"] == pytest.approx(4.5614e-2, rel=1e-4)
    for k in errs:
        assert errs[k] < 0.06, (k, errs[k])
