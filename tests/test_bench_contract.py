"""bench.py's command-line contract without a GPU: the reference arm (LBM-Bench's
own CPU kernels from oracle/_ref) prints one JSON line with the native arm's
metric, unit and direction; ranks other than 0 print nothing; bad flag
combinations are refused."""
import json
import os
import subprocess
import sys

import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BENCH = os.path.join(ROOT, "bench.py")


def _run(*args, env=None, timeout=600):
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        e.pop(k, None)
    e.update(env or {})
    return subprocess.run([sys.executable, BENCH, *args], capture_output=True, text=True,
                          timeout=timeout, env=e, cwd=ROOT)


@pytest.mark.skipif(not (O.ref_available("bench_v3") or O.ref_available("bench_v4")),
                    reason="oracle/_ref not built here")
def test_reference_arm_prints_the_contract_line():
    sys.path.insert(0, ROOT)
    import bench
    r = _run("--impl", "reference", "--steps", "1", "--warmup", "3")
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d["impl"] == "reference"
    assert d["metric"] == bench.METRIC and d["unit"] == "MLUPS"
    assert d["higher_is_better"] is True and d["n_gpus"] == 1
    assert d["value"] > 0 and d["steps"] >= 1 and d["warmup"] == 3
    assert d["config"]["workload"] == bench.WORKLOAD["workload"]
    assert d["cpu_baseline"]["kind"] == "reference" and d["cpu_baseline"]["value"] == d["value"]
    assert d["cpu_baseline"]["cores"] >= 1
    assert d["e2e"] == {"value": d["value"], "unit": "MLUPS", "h2d_bytes_per_step": 0,
                        "d2h_bytes_per_step": 0}


@pytest.mark.skipif(not (O.ref_available("bench_v3") or O.ref_available("bench_v4")),
                    reason="oracle/_ref not built here")
def test_reference_arm_loads_nothing_from_the_product():
    """The reference arm builds its workload with the oracle's generator:
    neither the lbmb200 module nor liblbmb200.so may be loaded in it."""
    code = (
        "import atexit, runpy, sys\n"
        "def check():\n"
        "    maps = open('/proc/self/maps').read()\n"
        "    sys.stderr.write('\\nPRODUCT_LOADED\\n' if ('liblbmb200' in maps or\n"
        "                     'lbmb200' in sys.modules) else '\\nPRODUCT_ABSENT\\n')\n"
        "atexit.register(check)\n"
        f"sys.argv = [{BENCH!r}, '--impl', 'reference', '--steps', '2', '--warmup', '3',\n"
        "            '--size', '40', '--cpu-seconds', '1']\n"
        f"runpy.run_path({BENCH!r}, run_name='__main__')\n")
    e = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        e.pop(k, None)
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                       timeout=300, env=e, cwd=ROOT)
    assert r.returncode == 0, r.stderr[-2000:]
    assert "PRODUCT_ABSENT" in r.stderr and "PRODUCT_LOADED" not in r.stderr
    d = json.loads([ln for ln in r.stdout.splitlines() if ln.strip()][0])
    assert d["impl"] == "reference" and d["value"] > 0
    assert d["config"]["dims"] == [40, 40, 40]
    assert "-march=x86-64-v" in d["cpu_baseline"]["sample"]


def test_reference_arm_runs_on_rank_0_only():
    r = _run("--impl", "reference", "--steps", "1", "--warmup", "3",
             env={"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"}, timeout=120)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


@pytest.mark.parametrize("args", [
    ("--warmup", "2"),                              # fewer than 3 warm-up steps
    ("--config", "2", "--impl", "reference"),       # configs 2-4 are native, one GPU
    ("--config", "4", "--gpus", "2"),
])
def test_bad_flags_are_refused(args):
    r = _run(*args, timeout=120)
    assert r.returncode != 0
    assert "error" in r.stderr
