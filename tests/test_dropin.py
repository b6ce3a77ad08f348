"""The drop-in boundary without a GPU: the reference-ABI structs of
include/lbm_b200_dropin.h against LBM-Bench's own src/lbm.h, the registry,
the ctypes mirror, and the lbmbench-b200 driver's CLI."""
import ctypes
import os
import subprocess

import pytest

import lbmb200 as L
import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "lbm-bench_b200")
CLI = os.path.join(PKG, "lbmbench-b200")
PROBE = os.path.join(ROOT, "tests", "dropin_layout_probe.c")
# the reference's own src/lbm.h: the unmodified build-time copy that
# oracle/Makefile takes of the reference sources next to its drop-in build
REF_SRC = os.path.join(ROOT, "oracle", "_ref", "dropin_src-dp")


def _probe(tmp_path, *flags):
    exe = tmp_path / ("probe" + "_".join(f.strip("-").replace("/", "") for f in flags))
    cmd = ["gcc", "-std=gnu11", "-I", os.path.join(ROOT, "include"), *flags, PROBE, "-o",
           str(exe), "-L", PKG, "-llbmb200", f"-Wl,-rpath,{PKG}"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    return subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout


def test_dropin_types_compile_and_link_standalone(tmp_path):
    out = _probe(tmp_path)
    assert "rows 3" in out
    assert "sizeof PdfType 8" in out


@pytest.mark.skipif(not os.path.exists(os.path.join(REF_SRC, "lbm.h")),
                    reason="oracle/_ref not built (needs the reference sources)")
@pytest.mark.parametrize("sp", [False, True])
def test_dropin_struct_layout_equals_reference_lbm_h(tmp_path, sp):
    extra = ["-DPRECISION_SP"] if sp else []
    ours = _probe(tmp_path, *extra)
    theirs = _probe(tmp_path, "-DWITH_REFERENCE_HEADER", "-I", REF_SRC, *extra)
    assert ours == theirs


@pytest.mark.parametrize("sp", [False, True])
def test_ctypes_mirror_matches_the_c_layout(tmp_path, sp):
    out = dict(line.rsplit(" ", 1)
               for line in _probe(tmp_path, *(["-DPRECISION_SP"] if sp else [])).splitlines())
    kd, cd = (L.KernelDataSP, L.CaseDataSP) if sp else (L.KernelData, L.CaseData)
    assert int(out["sizeof PdfType"]) == (4 if sp else 8)
    assert int(out["sizeof KernelDataType"]) == ctypes.sizeof(kd)
    assert int(out["sizeof LatticeDescType"]) == ctypes.sizeof(L.LatticeDesc)
    assert int(out["sizeof CaseDataType"]) == ctypes.sizeof(cd)
    assert int(out["KernelDataType.Kernel"]) == kd.Kernel.offset
    assert int(out["KernelDataType.Duration"]) == kd.Duration.offset


def test_single_precision_registry():
    assert L.dropin_kernels(sp=True) == L.dropin_kernels()


# the reference's registry (src/lbm.c:33-41)
REFERENCE_NAMES = ["pull-soa", "pull-aos", "push-soa", "push-aos", "blk-push-soa",
                   "blk-pull-soa", "aa-soa"]


def test_registry_names():
    names = L.dropin_kernels()
    assert names[:7] == ["cuda-" + n for n in REFERENCE_NAMES]
    assert len(names) == 13 and len(set(names)) == 13


@pytest.mark.skipif(not O.ref_available("plain"), reason="oracle/_ref not built here")
def test_registry_covers_the_reference_list():
    assert O.Reference("plain").kernels() == REFERENCE_NAMES


def test_cli_lists_kernels_like_the_reference():
    out = subprocess.run([CLI, "-l"], capture_output=True, text=True, check=True).stdout
    # the reference's test.sh parses -l this way (src/test.sh:95)
    lines = out.splitlines()
    start = lines.index("Available kernels:")
    assert [ln.split()[0] for ln in lines[start + 1:] if ln.strip()] == L.dropin_kernels()


def test_cli_rejects_bad_input():
    r = subprocess.run([CLI, "-d", "8x0x8"], capture_output=True, text=True)
    assert r.returncode != 0 and "ERROR: Y dimension must be > 0." in r.stdout
    r = subprocess.run([CLI, "-d", "8x8x8", "-k", "no-such-kernel"], capture_output=True,
                       text=True)
    assert r.returncode == 1 and 'ERROR: kernel "no-such-kernel" not found.' in r.stdout
    r = subprocess.run([CLI, "-g", "sphere"], capture_output=True, text=True)
    assert r.returncode != 0 and "unknown geometry type" in r.stdout
    r = subprocess.run([CLI, "-h"], capture_output=True, text=True, check=True)
    assert "-V                   Run verification" in r.stdout


@pytest.mark.skipif(L.device_count() > 0, reason="a CUDA device is present")
def test_cli_fails_loudly_without_gpu():
    r = subprocess.run([CLI, "-d", "8x8x8"], capture_output=True, text=True)
    assert r.returncode != 0
    assert "no CPU path" in r.stdout


REF_DROPIN = {p: os.path.join(ROOT, "oracle", "_ref", f"lbmbench-dropin-{p}") for p in ("dp", "sp")}


@pytest.mark.parametrize("prec", ["dp", "sp"])
def test_reference_binary_with_dropin_rows_lists_all_kernels(prec):
    """LBM-Bench's own binary (its main.c/cli.c, oracle/Makefile) with the
    drop-in rows appended to GKernels[]: `-l` lists the reference's seven
    names in its order, then the 13 cuda-* rows, parsed the way
    src/test.sh:95 parses it. No GPU is touched by -l."""
    exe = REF_DROPIN[prec]
    if not os.path.exists(exe):
        pytest.skip("oracle/_ref/lbmbench-dropin-* not built (needs the reference sources)")
    out = subprocess.run([exe, "-l"], capture_output=True, text=True, check=True).stdout
    lines = out.splitlines()
    start = lines.index("Available kernels:")
    names = [ln.split()[0] for ln in lines[start + 1:] if ln.strip()]
    assert names == REFERENCE_NAMES + L.dropin_kernels()
