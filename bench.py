#!/usr/bin/env python
"""Benchmark of the B200 D3Q19 TRT lattice-Boltzmann step (liblbmb200).

Workload (the 256^3 FP64 configuration the headline metric is quoted on):
a 256^3 porous channel - x-periodic, obstacle walls on the y and z faces,
seeded solid spheres with radii uniform in [4, 8] cells until 20% of the
cells are solid - driven by a body force F_x = 1e-6, TRT with omega = 1.25
(tau = 0.8) and Lambda = 3/16, starting from a seeded equilibrium with a
+-1e-4 velocity perturbation. A "step" is one lattice time step over the
whole domain. The state (2.6 GB FP64 for AA) is far larger than the 126 MB
L2, so no flush is needed between steps.

Headline `value`: FP64 AA (in place) MLUPS = fluid cells x steps / device
time, state resident in HBM, timed with CUDA events on the solver's stream
(max over ranks). `e2e`: the same metric through the reference-facing call
with host buffers: upload of the state from pinned host memory, the steps,
and the download of the final state, all inside the timed region.
Variants: FP64 pull and push, FP32 and FP16 storage (FP32 arithmetic) with
their L2 velocity/density error against the FP64 run of the same seed.

`--impl reference` times LBM-Bench's own CPU kernels (compiled from the
reference sources into oracle/_ref) on the host cores on the same workload.

Multi-GPU (`--gpus N` under torchrun): each rank runs an independent replica
of the workload on its own GPU (weak scaling); value = all ranks' updates /
max rank time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "lbm-bench_b200"))

METRIC = ("MLUPS and HBM GB/s (% of roofline) per precision at stated velocity error vs FP64; "
          "adjoint s/step")
WORKLOAD = {"workload": "porous channel 256^3, 20% solid spheres r 4-8, seed 42",
            "dims": [256, 256, 256], "solid_fraction": 0.2, "sphere_radius": [4, 8],
            "omega": 1.25, "lambda": 3 / 16, "xforce": 1e-6, "init": "equilibrium +-1e-4 seed 7",
            "pattern": "AA in place", "l2_flush": "not needed: state 2.6 GB > 126 MB L2"}
FALLBACK_HBM_GBS = 6650.0


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def measured_hbm_peak():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kind: str, precision: str):
    """DRAM bytes per fluid cell update of `kind` from the committed ncu
    summary (profiles/traffic.json), or None."""
    try:
        with open(os.path.join(ROOT, "profiles", "traffic.json")) as fh:
            t = json.load(fh)
        return float(t[precision][kind]["dram_bytes_per_fluid_update"])
    except Exception:
        return None


class ClockSampler:
    """nvidia-smi clock/throttle samples (200 ms) during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu: int):
        self.gpu = gpu
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.gpu), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        time.sleep(0.3)
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc:
            time.sleep(0.25)
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            p = [x.strip() for x in ln.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx.append(float(p[2]))
            except ValueError:
                continue
            for name, v in zip(names, p[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx),
                "reasons": sorted(reasons), "samples": len(sm)}


# ---------------------------------------------------------------------------
# distributed plumbing (one process per GPU)
# ---------------------------------------------------------------------------

class Dist:
    def __init__(self, n: int):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.pg = None
        if self.world > 1:
            import datetime
            import torch
            import torch.distributed as dist
            torch.cuda.set_device(self.local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                    device_id=torch.device("cuda", self.local))
            self.dist, self.torch = dist, torch
            self.pg = True

    def barrier(self):
        if self.pg:
            self.dist.barrier()

    def max(self, v: float) -> float:
        if not self.pg:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device="cuda")
        self.dist.all_reduce(t, op=self.dist.ReduceOp.MAX)
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU baseline: LBM-Bench's own kernels (oracle/_ref)
# ---------------------------------------------------------------------------

def reference_cpu(flags, f0, budget_s: float, max_steps: int, kernels=("push-soa", "pull-soa")):
    """Times the reference's OpenMP kernels on this host on the workload.
    Returns dict(value MLUPS, kernel, steps, cores, variant) or raises."""
    ncores = os.cpu_count() or 1
    os.environ.setdefault("OMP_NUM_THREADS", str(ncores))
    os.environ.setdefault("OMP_PROC_BIND", "close")
    os.environ.setdefault("OMP_PLACES", "cores")
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    variant = "bench_v4" if _has_avx512() and O.ref_available("bench_v4") else "bench_v3"
    if not O.ref_available(variant):
        raise FileNotFoundError(f"oracle/_ref/libref_{variant}.so not built")
    ref = O.Reference(variant)
    threads = ref.max_threads()
    per = (1, 0, 0)
    n_fluid = int((flags != 0).sum())
    best = None
    for k in kernels:  # calibration: 2 steps each
        _, d, _, _ = ref.run(k, flags, per, f0, 2, 1.25, 1e-6, readback=False)
        if best is None or d < best[1]:
            best = (k, d)
    k, d2 = best
    steps = max(2, min(max_steps, int(budget_s / max(d2 / 2, 1e-6))))
    _, dur, _, _ = ref.run(k, flags, per, f0, steps, 1.25, 1e-6, readback=False)
    return {"value": n_fluid * steps / dur / 1e6, "kernel": k, "steps": steps, "cores": threads,
            "variant": variant, "seconds": dur}


def _has_avx512() -> bool:
    try:
        with open("/proc/cpuinfo") as fh:
            return " avx512f" in fh.read()
    except Exception:
        return False


# ---------------------------------------------------------------------------
# workload
# ---------------------------------------------------------------------------

def make_workload(L, n: int):
    flags, frac, nsph = L.porous_channel((n, n, n), 0.2, 4.0, 8.0, seed=42)
    f0 = L.perturbed_equilibrium(flags, seed=7, amplitude=1e-4)
    return flags, f0, frac, nsph


def solver(L, flags, pattern, precision, f0):
    s = L.Solver(flags, (1, 0, 0), pattern, precision)
    s.set_params(1.25, 3 / 16, 1e-6, True)
    s.set_state(f0)
    return s


def run_native(args, dist: Dist):
    import lbmb200 as L
    import numpy as np

    if L.device_count() <= 0:
        raise SystemExit("bench.py: no CUDA device; the native arm has no CPU path")
    n = args.size
    flags, f0, frac, nsph = make_workload(L, n)
    peak, peak_kind = measured_hbm_peak()

    # ---- headline: FP64 AA, device-resident, timed region with per-launch events
    s = solver(L, flags, "aa", L.F64, f0)
    n_fluid = s.fluid_cells
    bpu = s.bytes_per_update
    s.run(args.warmup)
    s.synchronize()
    launches0 = s.launch_count
    dist.barrier()
    s.synchronize()
    with ClockSampler(dist.local) as clk:
        per_kind, region_ms = s.time_launches(args.steps)
        s.synchronize()
    dist.barrier()
    launches = s.launch_count - launches0
    ms = dist.max(region_ms)
    tot, bad = s.mass_momentum(check=False)
    value = dist.world * n_fluid * args.steps / (ms / 1e3) / 1e6
    dom = max(per_kind, key=lambda k: per_kind[k][0])
    dom_ms = per_kind[dom][0] / per_kind[dom][1]
    achieved = n_fluid * bpu / (dom_ms / 1e3) / 1e9
    traffic = ncu_traffic(dom, "fp64")
    roofline = {"bound": "hbm", "kernel": f"step_kernel<StoreF64,{dom}>", "achieved": achieved,
                "peak": peak, "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic * n_fluid if traffic else None,
                "algorithmic_bytes_per_launch": n_fluid * bpu,
                "launch_ms": dom_ms, "per_kind_ms": {k: v[0] / v[1] for k, v in per_kind.items()}}

    # ---- variants (same workload): FP64 pull/push, FP32/FP16 AA with error vs FP64
    variants = {}
    vsteps = max(20, args.steps // 2)
    ref64 = s  # FP64 AA solver; compare after equal step counts
    for pattern in ("pull", "push"):
        v = solver(L, flags, pattern, L.F64, f0)
        v.run(args.warmup)
        t = v.run_timed(vsteps)
        variants[f"fp64_{pattern}"] = {
            "mlups": n_fluid * vsteps / (t / 1e3) / 1e6,
            "gbs": n_fluid * vsteps * v.bytes_per_update / (t / 1e3) / 1e9}
        variants[f"fp64_{pattern}"]["frac"] = variants[f"fp64_{pattern}"]["gbs"] / peak
        v.close()
    for name, prec in (("fp32", L.F32), ("fp16", L.F16)):
        # accuracy: same seed and step count as a fresh FP64 run
        a = solver(L, flags, "aa", L.F64, f0)
        b = solver(L, flags, "aa", prec, f0)
        a.run(args.steps)
        b.run(args.warmup)
        t = b.run_timed(args.steps - args.warmup) if args.steps > args.warmup else None
        d = b.compare(a)
        mlups = n_fluid * (args.steps - args.warmup) / (t / 1e3) / 1e6 if t else None
        variants[f"{name}_aa"] = {
            "mlups": mlups, "gbs": mlups * b.bytes_per_update / 1e3 if mlups else None,
            "l2_rel_err_u": float(np.sqrt(d[0] / d[1])) if d[1] > 0 else None,
            "l2_rel_err_rho": float(np.sqrt(d[2] / d[3])) if d[3] > 0 else None,
            "error_after_steps": args.steps}
        if mlups:
            variants[f"{name}_aa"]["frac"] = variants[f"{name}_aa"]["gbs"] / peak
            variants[f"{name}_aa"]["speedup_vs_fp64_aa"] = mlups / (value / dist.world)
        a.close()
        b.close()

    # ---- e2e: through the reference-facing call with pinned host buffers
    e2e = run_e2e(L, flags, f0, args.steps, dist)

    result = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded porous geometry and initial state)",
        "config": dict(WORKLOAD, solid_fraction_achieved=frac, spheres=nsph,
                       fluid_cells=n_fluid, parallelism=f"replicas x{dist.world}"),
        "gbs": n_fluid * bpu * args.steps / (ms / 1e3) / 1e9,
        "roofline": roofline, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.summary(), "variants": variants,
        "state_check": {"mass": tot[0], "nonfinite_cells": bad},
        "device_bytes": s.device_bytes,
    }
    s.close()
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            cb = reference_cpu(flags, f0, budget_s=args.cpu_seconds, max_steps=args.steps)
            result["cpu_baseline"] = {
                "value": cb["value"], "unit": "MLUPS", "cores": cb["cores"], "kind": "reference",
                "sample": f"{cb['kernel']} (OpenMP, {cb['variant']}) on the same 256^3 porous "
                          f"channel, {cb['steps']} steps, {cb['seconds']:.1f} s"}
        except Exception as exc:  # reported, not fatal
            result["cpu_baseline"] = {"value": None, "unit": "MLUPS", "error": str(exc)}
    return result


def run_e2e(L, flags, f0, steps, dist: Dist):
    """The same metric through the reference-facing call: the drop-in
    kernel's Init (page-locked host arrays in LBM-Bench's padded layout,
    include/lbm_b200_dropin.h), the initial state written into those host
    arrays, then kd->Kernel timed by the host clock - it uploads the state,
    runs the steps and downloads the result. Max over ranks."""
    with L.DropIn("cuda-aa-soa", flags, (1, 0, 0), omega=1.25, xforce=1e-6, iterations=steps,
                  force_on=True, lam=3 / 16) as k:
        host = k.pdfs(0)  # [19, nx+2, ny+2, nz+2]; natural orientation before the first run
        host[:, 1:-1, 1:-1, 1:-1] = f0
        k.run(2)  # first use of the transfer path
        host[:, 1:-1, 1:-1, 1:-1] = f0
        dist.barrier()
        t0 = time.perf_counter()
        k.run(steps)
        t = time.perf_counter() - t0
        n_fluid = int((flags != 0).sum())
        nbytes = host.nbytes
    t = dist.max(t)
    return {"value": dist.world * n_fluid * steps / t / 1e6, "unit": "MLUPS",
            "h2d_bytes_per_step": nbytes / steps, "d2h_bytes_per_step": nbytes / steps,
            "h2d_bytes_per_call": nbytes, "d2h_bytes_per_call": nbytes, "seconds": t,
            "call": "kernelInitCudaAaSoA + kd->Kernel (host arrays in the reference's padded "
                    "layout, page-locked; upload + steps + download inside the timing)"}


def run_reference(args):
    """LBM-Bench's own CPU kernels on this host, same workload and metric."""
    import lbmb200 as L
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    flags, f0, frac, nsph = make_workload(L, args.size)
    try:
        cb = reference_cpu(flags, f0, budget_s=args.cpu_seconds * 3, max_steps=args.steps)
    except FileNotFoundError as exc:
        return {"impl": "reference", "unavailable": f"reference CPU build missing: {exc}"}
    n_fluid = int((flags != 0).sum())
    value = cb["value"]
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "MLUPS",
        "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": cb["steps"],
        "warmup": args.warmup, "ms_per_step": cb["seconds"] * 1e3 / cb["steps"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded porous geometry and initial state)",
        "config": dict(WORKLOAD, solid_fraction_achieved=frac, spheres=nsph,
                       fluid_cells=n_fluid, parallelism="host CPU (OpenMP)"),
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": cb["cores"],
                         "kind": "reference",
                         "sample": f"{cb['kernel']} ({cb['variant']}), {cb['steps']} steps of "
                                   "the 256^3 workload"},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--warmup", type=int, default=10)
    ap.add_argument("--impl", choices=["native", "reference"], default="native")
    ap.add_argument("--size", type=int, default=256, help="cube edge (default 256)")
    ap.add_argument("--cpu-seconds", type=float, default=15.0,
                    help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    if args.impl == "reference":
        res = run_reference(args)
        if res is not None:
            print(json.dumps(res), flush=True)
        return
    dist = Dist(args.gpus)
    try:
        res = run_native(args, dist)
        if dist.rank == 0:
            print(json.dumps(res), flush=True)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
