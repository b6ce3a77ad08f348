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
Variants: FP64 pull and push; FP32 and FP16 storage (FP32 arithmetic) in
the AA and pull patterns, each with its L2 velocity/density error against
the FP64 AA run of the same seed after the same number of steps.

Adjoint (`adjoint` key of the default line): 128^3 Brinkman channel (walls
on the y and z faces, x periodic, FP32 porosity uniform in [0, 1] from a
seed, Brinkman coefficient kappa = 0.1 (1 - phi)), J = mean x velocity on the
outlet plane after 2000 steps, checkpoints every 100 steps; seconds per
step and cost in forward steps, the FP64 gradient against FP64 central
finite differences (eps = 1e-4) at 20 seeded fluid cells, and the FP32
gradient against the FP64 one.

Other workloads, one JSON line each (`--config`):
  2  precision study: 512^3 porous channel (20% solid, r 4-8), 300 steps,
     FP32 and FP16 storage against the FP64 run of the same seed
  3  the adjoint study alone
  4  largest single-GPU sizes: 768^3 porous channel (30% solid, r 6-12),
     FP16 storage, AA, 200 steps; the 384^3 Brinkman adjoint, 1000 steps,
     sqrt checkpoint schedule; peak device memory against the 180 GB HBM

`--impl reference` times LBM-Bench's own CPU kernels (compiled from the
reference sources into oracle/_ref) on the host cores on the same workload.

Multi-GPU (`--gpus N` under torchrun): the porous channel grows to
(N x 256) x 256 x 256 and is cut into one 256^3 x-slab per rank (weak
scaling); each odd AA step exchanges the five x-crossing populations of the
slab faces with the ring neighbours over NCCL (lbm_slab), while a second
stream updates the interior planes; value = all ranks' fluid updates / max
rank device time.
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
        return self._reduce(v, "MAX")

    def sum(self, v: float) -> float:
        return self._reduce(v, "SUM")

    def _reduce(self, v: float, op: str) -> float:
        if not self.pg:
            return v
        t = self.torch.tensor([v], dtype=self.torch.float64, device="cuda")
        self.dist.all_reduce(t, op=getattr(self.dist.ReduceOp, op))
        return float(t.item())

    def close(self):
        if self.pg:
            self.dist.destroy_process_group()


# ---------------------------------------------------------------------------
# CPU baseline: LBM-Bench's own kernels (oracle/_ref)
# ---------------------------------------------------------------------------

MARCH = {"bench_v4": "x86-64-v4", "bench_v3": "x86-64-v3"}


def reference_cpu(flags, f0, budget_s: float, max_steps: int, kernels=("push-soa", "pull-soa")):
    """Times the reference's OpenMP kernels on this host on the workload:
    both OpenMP kernels are calibrated on 2 steps, the faster one is timed
    on as many steps as fit in `budget_s` (at most max_steps). Returns
    dict(value MLUPS, kernel, steps, cores, variant, seconds, sample) or
    raises FileNotFoundError when the reference build is missing."""
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
    nz, ny, nx = flags.shape
    sample = (f"{k}, LBM-Bench's own OpenMP kernel (faster of push-soa/pull-soa on a 2-step "
              f"calibration), built -O3 -ffast-math -fopenmp -march={MARCH[variant]}, "
              f"{threads} threads, {steps} steps of the {nx}x{ny}x{nz} porous channel, "
              f"{dur:.1f} s")
    return {"value": n_fluid * steps / dur / 1e6, "kernel": k, "steps": steps, "cores": threads,
            "variant": variant, "seconds": dur, "sample": sample}


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


def workload_config(n, frac, nsph, n_fluid):
    """The `config` both arms print for the n^3 porous-channel workload."""
    cfg = dict(WORKLOAD, solid_fraction_achieved=frac, spheres=nsph, fluid_cells=n_fluid,
               parallelism="single process")
    if n != 256:
        cfg.update(workload=f"porous channel {n}^3, 20% solid spheres r 4-8, seed 42",
                   dims=[n, n, n])
    return cfg


def solver(L, flags, pattern, precision, f0, compact=False):
    s = L.Solver(flags, (1, 0, 0), pattern, precision, compact=compact)
    s.set_params(1.25, 3 / 16, 1e-6, True)
    s.set_state(f0)
    return s


def run_native(args, dist: Dist):
    import lbmb200 as L
    import numpy as np

    if L.device_count() <= 0:
        raise SystemExit("bench.py: no CUDA device; the native arm has no CPU path")
    if dist.world > 1:
        return run_slabs(args, dist)
    n = args.size
    flags, f0, frac, nsph = make_workload(L, n)
    peak, peak_kind = measured_hbm_peak()

    # ---- headline: FP64 AA, device-resident, timed region with per-launch events
    compact = args.layout == "compact"
    other = "dense" if compact else "compact"
    s = solver(L, flags, "aa", L.F64, f0, compact)
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
    traffic = ncu_traffic(dom, "fp64_compact" if compact else "fp64")
    kname = (("step_kernel_cp_local<StoreF64>" if dom == "aa_even" else
              f"step_kernel_cp<StoreF64,{dom}>") if compact else f"step_kernel<StoreF64,{dom}>")
    roofline = {"bound": "hbm", "kernel": kname, "layout": args.layout, "achieved": achieved,
                "peak": peak, "peak_source": peak_kind, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic * n_fluid if traffic else None,
                "algorithmic_bytes_per_launch": n_fluid * bpu,
                "launch_ms": dom_ms, "per_kind_ms": {k: v[0] / v[1] for k, v in per_kind.items()}}

    # ---- variants (same workload): FP64 pull/push, FP32/FP16 AA with error vs FP64
    variants = {}
    vsteps = max(20, args.steps // 2)
    ref64 = s  # FP64 AA solver; compare after equal step counts
    # FP64 in both layouts (the headline's layout without a suffix)
    for pattern, cp in (("pull", compact), ("push", compact), ("aa", not compact),
                        ("pull", not compact), ("push", not compact)):
        v = solver(L, flags, pattern, L.F64, f0, cp)
        v.run(args.warmup)
        t = v.run_timed(vsteps)
        key = f"fp64_{pattern}" + ("" if cp == compact else f"_{other}")
        variants[key] = {
            "mlups": n_fluid * vsteps / (t / 1e3) / 1e6,
            "gbs": n_fluid * vsteps * v.bytes_per_update / (t / 1e3) / 1e9,
            "layout": "compact" if cp else "dense", "device_bytes": v.device_bytes}
        variants[key]["frac"] = variants[key]["gbs"] / peak
        v.close()
    # FP32 / FP16 storage in both layouts (bit-identical results)
    ref = solver(L, flags, "aa", L.F64, f0, compact)  # accuracy reference: FP64, same seed
    ref.run(args.steps)
    for name, prec in (("fp32", L.F32), ("fp16", L.F16)):
        for pattern, cp in (("aa", False), ("pull", False), ("aa", True), ("pull", True)):
            b = solver(L, flags, pattern, prec, f0, cp)
            b.run(args.warmup)
            t = b.run_timed(args.steps - args.warmup) if args.steps > args.warmup else None
            d = b.compare(ref)
            mlups = n_fluid * (args.steps - args.warmup) / (t / 1e3) / 1e6 if t else None
            key = f"{name}_{pattern}" + ("_compact" if cp else "")
            variants[key] = {
                "mlups": mlups, "gbs": mlups * b.bytes_per_update / 1e3 if mlups else None,
                "l2_rel_err_u": float(np.sqrt(d[0] / d[1])) if d[1] > 0 else None,
                "l2_rel_err_rho": float(np.sqrt(d[2] / d[3])) if d[3] > 0 else None,
                "error_after_steps": args.steps, "layout": "compact" if cp else "dense"}
            if mlups:
                variants[key]["frac"] = variants[key]["gbs"] / peak
                variants[key]["speedup_vs_fp64_aa"] = mlups / (value / dist.world)
            b.close()
    ref.close()

    # ---- e2e: through the reference-facing call with pinned host buffers
    e2e = run_e2e(L, flags, f0, args.steps, dist)

    # ---- adjoint of the Brinkman step (128^3, 2000 steps, checkpoints every 100)
    adjoint = adjoint_study(L, 128, 2000, 100, 20) if not args.no_adjoint else None

    result = {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": dist.world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded porous geometry and initial state)",
        "config": workload_config(n, frac, nsph, n_fluid),
        "gbs": n_fluid * bpu * args.steps / (ms / 1e3) / 1e9,
        "roofline": roofline, "e2e": e2e, "gpu_launches": launches,
        "clocks": clk.summary(), "variants": variants, "adjoint": adjoint,
        "state_check": {"mass": tot[0], "nonfinite_cells": bad},
        "device_bytes": s.device_bytes,
    }
    s.close()
    if not args.no_studies:
        result["ring_1gpu"] = ring_study(L, flags, f0, args.steps, args.warmup, ms / args.steps,
                                         compact)
        result["precision_512"] = precision_study(L, 512, 300, peak)
        result["largest"] = largest_study(L, 768, 200, peak)
    if not args.no_parity:
        result["parity"] = parity_study(L, flags, f0)
    if dist.rank == 0 and dist.world == 1 and not args.no_cpu_baseline:
        try:
            cb = reference_cpu(flags, f0, budget_s=args.cpu_seconds, max_steps=args.steps)
            result["cpu_baseline"] = {
                "value": cb["value"], "unit": "MLUPS", "cores": cb["cores"], "kind": "reference",
                "sample": cb["sample"]}
        except Exception as exc:  # reported, not fatal
            result["cpu_baseline"] = {"value": None, "unit": "MLUPS", "error": str(exc)}
    result["summary"] = summary(result)
    return result


def _r(v, digits=4):
    """v rounded to `digits` significant digits (None stays None)."""
    if v is None:
        return None
    if isinstance(v, bool) or not isinstance(v, (int, float)):
        return v
    return float(f"{v:.{digits}g}")


def summary(r):
    """The headline figures of the default line in one short object, placed
    last so that a reader of only the line's tail still sees them: MLUPS and
    roofline fraction per precision and pattern, errors against FP64, the
    adjoint's cost, and the parity of configs 0 and 1 with the reference."""
    v = r.get("variants", {})
    out = {"fp64_aa": {"mlups": _r(r["value"]), "frac_step": _r(r["gbs"] / r["roofline"]["peak"]),
                       "frac_dominant": _r(r["roofline"]["frac"]),
                       "layout": r["roofline"].get("layout")}}
    for k in ("fp64_pull", "fp64_push", "fp64_aa_dense", "fp64_pull_dense", "fp64_push_dense",
              "fp64_aa_compact", "fp64_pull_compact", "fp64_push_compact"):
        if k in v:
            out[k] = {"mlups": _r(v[k]["mlups"]), "frac": _r(v[k]["frac"])}
    for k in ("fp32_aa", "fp32_pull", "fp16_aa", "fp16_pull", "fp32_aa_compact",
              "fp32_pull_compact", "fp16_aa_compact", "fp16_pull_compact"):
        if k in v and v[k]["mlups"]:
            out[k] = {"mlups": _r(v[k]["mlups"]), "frac": _r(v[k]["frac"]),
                      "x_fp64_aa": _r(v[k]["speedup_vs_fp64_aa"], 3),
                      "err_u": _r(v[k]["l2_rel_err_u"], 2), "err_rho": _r(v[k]["l2_rel_err_rho"], 2)}
    p = r.get("precision_512")
    if p:
        out["p512"] = {"fp64_aa": _r(p["fp64_aa"]["mlups"]),
                       "fp64_aa_dense": _r(p["fp64_aa_dense"]["mlups"])}
        for k in ("fp32_aa", "fp16_aa", "fp32_aa_compact", "fp16_aa_compact"):
            out["p512"][k] = {"mlups": _r(p[k]["mlups"]), "frac": _r(p[k]["frac"]),
                              "x_fp64_aa": _r(p[k]["speedup_vs_fp64_aa"], 3),
                              "err_u": _r(p[k]["l2_rel_err_u"], 2),
                              "err_rho": _r(p[k]["l2_rel_err_rho"], 2)}
    g = r.get("largest")
    if g:
        a = g["adjoint"]["fp32"]
        for k in ("forward_fp16_aa", "forward_fp16_aa_compact"):
            f = g[k]
            out["l768_" + k[8:]] = {"mlups": _r(f["mlups"]), "frac": _r(f["frac"]),
                                     "device_gb": _r(f["device_used_bytes"] / 1e9, 3)}
        out["adj384_fp32"] = {"cost_fwd_steps": _r(a["cost_in_forward_steps"], 3),
                              "s_per_step": _r(a["s_per_step"], 3),
                              "peak_gb": _r(a["peak_device_bytes"] / 1e9, 3)}
    a = r.get("adjoint")
    if a:
        out["adj128"] = {"fp64_cost": _r(a["fp64"]["cost_in_forward_steps"], 3),
                         "fp32_cost": _r(a["fp32"]["cost_in_forward_steps"], 3),
                         "interval": a["fp64"]["checkpoint_interval"]}
        if "fp64_auto_schedule" in a:
            out["adj128"]["fp64_auto_cost"] = _r(a["fp64_auto_schedule"]["cost_in_forward_steps"], 3)
        if "fd_check" in a:
            fd = a["fd_check"]
            out["adj128"]["fd_eps1e-4_max_rel"] = _r(fd["eps_0.0001"]["max_rel_err"], 3)
            out["adj128"]["fd_eps1e-4_within_1e-4"] = fd["eps_0.0001"]["cells_within_1e-4"]
            out["adj128"]["fd_richardson_max_rel"] = _r(fd["richardson_h_0.005"]["max_rel_err"], 3)
        if "fp32_vs_fp64_grad_l2_rel" in a:
            out["adj128"]["fp32_vs_fp64"] = _r(a["fp32_vs_fp64_grad_l2_rel"], 3)
    q = r.get("parity")
    if q and "config0" in q:
        out["parity"] = {c: {"rho": _r(q[c]["max_rel_err_rho"], 3), "u": _r(q[c]["max_rel_err_u"], 3),
                             "bitwise": q[c]["bit_identical"], "steps": q[c]["steps"]}
                         for c in ("config0", "config1")}
    g = r.get("ring_1gpu")
    if g:
        out["ring_1gpu"] = {k: {"ms": _r(g[k]["ms_per_step"]), "overhead": _r(g[k]["overhead"], 3)}
                            for k in ("native_nccl", "native_copy", "python_copy")}
    out["e2e_mlups"] = _r(r["e2e"]["value"])
    if "transfer_gbs" in r["e2e"]:
        out["e2e_transfer_gbs"] = _r(r["e2e"]["transfer_gbs"], 3)
    cb = r.get("cpu_baseline")
    if cb and cb.get("value"):
        out["cpu_ref_mlups"] = _r(cb["value"])
    return out


# ---------------------------------------------------------------------------
# parity at the stated sizes: configs 0 and 1 against LBM-Bench's own kernels
# ---------------------------------------------------------------------------

def parity_study(L, flags256, f0_256, steps256: int = 10):
    """FP64 pull, push and AA on the GPU against the reference's own strict
    pull-soa (oracle/_ref/libref_verify_l316: LBM-Bench's sources with
    -DVERIFICATION, Lambda 3/16, -O2 -ffp-contract=off, OpenMP) run on this
    host's cores, on the same inputs:
      config0  64^3 channel, omega 1.25, F 1e-6, seeded +-1e-4
               equilibrium, 1000 steps;
      config1  the 256^3 porous benchmark workload, `steps256` steps.
    Reports the normwise relative rho and u errors (the stated bound is
    1e-12) and whether the states are bit-identical."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.ref_available("verify_l316"):
        return {"unavailable": "oracle/_ref/libref_verify_l316.so not built"}
    ref = O.Reference("verify_l316")
    threads = ref.max_threads()
    flags64, per64, _ = L.geometry("channel", (64, 64, 64))
    f0_64 = L.perturbed_equilibrium(flags64, seed=7, amplitude=1e-4)
    out = {}
    for name, flags, per, f0, steps in (("config0", flags64, per64, f0_64, 1000),
                                        ("config1", flags256, (1, 0, 0), f0_256, steps256)):
        t0 = time.perf_counter()
        r, _, _, _ = ref.run("pull-soa", flags, per, f0, steps, 1.25, 1e-6)
        ref_s = time.perf_counter() - t0
        m = O.fluid_mask(flags)
        rows = {}
        for pattern in ("aa", "pull", "push"):
            sv = solver(L, flags, pattern, L.F64, f0)
            sv.run(steps)
            g = sv.get_state()
            sv.close()
            e_rho, e_u = O.normwise_errors(g, r, flags)
            rows[pattern] = {"rel_err_rho": e_rho, "rel_err_u": e_u,
                             "bit_identical": bool(np.array_equal(g[:, m], r[:, m]))}
            del g
        nz, ny, nx = flags.shape
        out[name] = {
            "dims": [nx, ny, nz], "steps": steps, "fluid_cells": int(m.sum()),
            "max_rel_err_rho": max(v["rel_err_rho"] for v in rows.values()),
            "max_rel_err_u": max(v["rel_err_u"] for v in rows.values()),
            "bit_identical": all(v["bit_identical"] for v in rows.values()),
            "bound": 1e-12, "patterns": rows,
            "reference": f"LBM-Bench pull-soa, strict FP build (-DVERIFICATION, Lambda 3/16), "
                         f"{threads} OpenMP threads, {ref_s:.1f} s"}
        del r
    return out


# ---------------------------------------------------------------------------
# adjoint of the Brinkman step
# ---------------------------------------------------------------------------

ADJ = {"omega": 1.25, "lambda": 3 / 16, "xforce": 1e-6, "alpha": 0.1, "porosity_seed": 11,
       "init_seed": 7, "amplitude": 1e-4}


def adjoint_solver(L, flags, por, precision):
    s = L.Solver(flags, (1, 0, 0), "aa", precision)
    s.set_params(ADJ["omega"], ADJ["lambda"], ADJ["xforce"], True)
    s.set_porosity(por, ADJ["alpha"])
    s.init_equilibrium(seed=ADJ["init_seed"], amplitude=ADJ["amplitude"])
    return s


def adjoint_study(L, n: int, steps: int, ckpt: int, fd_cells: int, precisions=("fp64", "fp32")):
    """Gradient of J = mean outlet-plane u_x after `steps` Brinkman steps
    with respect to the porosity field: time per step, cost in forward
    steps, FD check (FP64, central, eps 1e-4) and FP32 vs FP64."""
    import numpy as np

    dims = (n, n, n)
    flags, _, _ = L.geometry("channel", dims)
    rng = np.random.default_rng(ADJ["porosity_seed"])
    por = rng.uniform(0.0, 1.0, size=dims).astype(np.float32)
    fluid = np.transpose(flags, (2, 1, 0)) != 0
    prec = {"fp64": L.F64, "fp32": L.F32}
    out = {"workload": f"Brinkman channel {n}^3, porosity U[0,1] seed {ADJ['porosity_seed']}",
           "dims": list(dims), "steps": steps, "checkpoint_every": ckpt,
           "objective": "mean u_x over the fluid cells of the outlet plane x = nx-1",
           **{k: ADJ[k] for k in ("omega", "lambda", "xforce", "alpha")}}
    grads = {}
    for name in precisions:
        s = adjoint_solver(L, flags, por, prec[name])
        n_fluid = s.fluid_cells
        s.run(5)
        fwd_ms = s.run_timed(steps) / steps  # plain Brinkman forward step
        s.init_equilibrium(seed=ADJ["init_seed"], amplitude=ADJ["amplitude"])
        j, g, info = s.adjoint_gradient(steps, ckpt)
        total_ms = info["forward_ms"] + info["reverse_ms"]
        grads[name] = g
        out[name] = {
            "J": j, "s_per_step": total_ms / 1e3 / steps,
            "forward_step_ms": fwd_ms,
            "cost_in_forward_steps": total_ms / steps / fwd_ms,
            "reverse_cost_in_forward_steps": info["reverse_ms"] / steps / fwd_ms,
            "forward_sweep_ms": info["forward_ms"], "reverse_sweep_ms": info["reverse_ms"],
            "checkpoint_interval": int(info["interval"]), "checkpoints": int(info["checkpoints"]),
            "peak_device_bytes": int(info["peak_bytes"]),
            "forward_mlups": n_fluid / fwd_ms / 1e3}
        if name == "fp64" and fd_cells:
            out["fd_check"] = finite_differences(s, por, g, fluid, steps, fd_cells)
        if name == "fp64" and ckpt > 0:
            # the same gradient with the least recomputation that fits in memory
            s.init_equilibrium(seed=ADJ["init_seed"], amplitude=ADJ["amplitude"])
            _, ga, ia = s.adjoint_gradient(steps, L.CKPT_AUTO)
            ta = ia["forward_ms"] + ia["reverse_ms"]
            out["fp64_auto_schedule"] = {
                "s_per_step": ta / 1e3 / steps, "cost_in_forward_steps": ta / steps / fwd_ms,
                "reverse_cost_in_forward_steps": ia["reverse_ms"] / steps / fwd_ms,
                "checkpoint_interval": int(ia["interval"]), "checkpoints": int(ia["checkpoints"]),
                "peak_device_bytes": int(ia["peak_bytes"]),
                "gradient_bitwise_equal_to_interval_run": bool(np.array_equal(ga, g))}
        s.close()
    if "fp64" in grads and "fp32" in grads:
        a, b = grads["fp64"], grads["fp32"]
        out["fp32_vs_fp64_grad_l2_rel"] = float(np.linalg.norm(b - a) / np.linalg.norm(a))
    return out


def finite_differences(s, por, g, fluid, steps, ncells, eps=1e-4, h=5e-3, seed=2024):
    """FP64 central differences of J at `ncells` seeded fluid cells, on the
    solver `s` (its porosity is restored afterwards): with step `eps`, and
    Richardson-extrapolated from steps h and 2h, (4 D(h) - D(2h)) / 3,
    whose truncation error is O(h^4) and whose round-off floor is eps/h
    times lower. The round-off of J (about 1e-18 absolute here, against
    differences 2 eps dJ/dphi of about 4e-15) is what limits the eps = 1e-4
    quotient far from the outlet."""
    import numpy as np

    def j_at(c, delta):
        p = por.copy()
        p[c] = np.float32(p[c] + delta)
        s.set_porosity(p, ADJ["alpha"])
        s.init_equilibrium(seed=ADJ["init_seed"], amplitude=ADJ["amplitude"])
        s.run(steps)
        return float(p[c]), s.objective()

    def quotient(c, step):
        (pa, ja), (pb, jb) = j_at(c, step), j_at(c, -step)
        return (ja - jb) / (pa - pb)

    rng = np.random.default_rng(seed)
    cells = np.argwhere(fluid)
    picks = [tuple(int(v) for v in cells[i])
             for i in rng.choice(len(cells), ncells, replace=False)]
    rows = []
    for c in picks:
        fd = quotient(c, eps)
        rich = (4.0 * quotient(c, h) - quotient(c, 2 * h)) / 3.0
        gc = float(g[c])
        rows.append({"cell": list(c), "adjoint": gc, "fd": fd, "fd_richardson": rich,
                     "rel_err": abs(gc - fd) / abs(fd), "rel_err_richardson":
                     abs(gc - rich) / abs(rich)})
    s.set_porosity(por, ADJ["alpha"])
    gv = np.array([r["adjoint"] for r in rows])
    out = {"cells": ncells, "seed": seed, "per_cell": rows}
    for key, name in (("fd", f"eps_{eps:g}"), ("fd_richardson", f"richardson_h_{h:g}")):
        errs = np.array([r["rel_err" if key == "fd" else "rel_err_richardson"] for r in rows])
        fv = np.array([r[key] for r in rows])
        out[name] = {"max_rel_err": float(errs.max()), "median_rel_err": float(np.median(errs)),
                     "cells_within_1e-4": int((errs <= 1e-4).sum()),
                     "normwise_rel_err": float(np.linalg.norm(gv - fv) / np.linalg.norm(fv))}
    return out


# ---------------------------------------------------------------------------
# other workloads (--config 2, 3, 4)
# ---------------------------------------------------------------------------

def base_line(metric_value, unit, steps, warmup, ms, workload, dtype, extra):
    r = {"metric": METRIC, "value": metric_value, "unit": unit, "n_gpus": 1, "steps": steps,
         "warmup": warmup, "ms_per_step": ms, "higher_is_better": unit != "s/step",
         "scaling": "weak", "vs_baseline": None, "dtype": dtype,
         "data": "synthetic (seeded porous geometry and initial state)", "config": workload}
    r.update(extra)
    return r


def timed_forward(L, flags, pattern, precision, steps, warmup, peak, compact=False):
    s = L.Solver(flags, (1, 0, 0), pattern, precision, compact=compact)
    s.set_params(1.25, 3 / 16, 1e-6, True)
    s.init_equilibrium(seed=7, amplitude=1e-4)
    s.run(warmup)
    with ClockSampler(0) as clk:
        ms = s.run_timed(steps)
    n_fluid = s.fluid_cells
    mlups = n_fluid * steps / (ms / 1e3) / 1e6
    gbs = mlups * s.bytes_per_update / 1e3
    return s, {"mlups": mlups, "gbs": gbs, "frac": gbs / peak, "ms_per_step": ms / steps,
               "fluid_cells": n_fluid, "device_bytes": s.device_bytes,
               "bytes_per_update": s.bytes_per_update, "clocks": clk.summary(),
               "layout": "compact" if compact else "dense"}


def precision_study(L, n: int, steps: int, peak: float):
    """n^3 porous channel (20% solid, r 4-8), `steps` steps: FP64 AA, and
    FP32 and FP16 storage of f - w (FP32 arithmetic) in AA, each with the L2
    relative u and rho errors against the FP64 run of the same seed."""
    import numpy as np

    flags, frac, nsph = L.porous_channel((n, n, n), 0.2, 4.0, 8.0, seed=42)
    d64, r64d = timed_forward(L, flags, "aa", L.F64, steps, 0, peak)
    d64.close()
    ref, r64 = timed_forward(L, flags, "aa", L.F64, steps, 0, peak, compact=True)
    res = {"workload": f"precision study, porous channel {n}^3, 20% solid spheres r 4-8, "
                       "seed 42", "dims": [n] * 3, "steps": steps,
           "solid_fraction_achieved": frac, "spheres": nsph,
           "init": "equilibrium +-1e-4 seed 7 (generated on the device)",
           "error": f"L2 relative error of u and rho over fluid cells vs the FP64 AA run "
                    f"after {steps} steps", "fp64_aa": r64, "fp64_aa_dense": r64d}
    for name, prec in (("fp32", L.F32), ("fp16", L.F16)):
        for cp in (False, True):
            b, r = timed_forward(L, flags, "aa", prec, steps, 0, peak, compact=cp)
            d = b.compare(ref)
            r["l2_rel_err_u"] = float(np.sqrt(d[0] / d[1])) if d[1] > 0 else None
            r["l2_rel_err_rho"] = float(np.sqrt(d[2] / d[3])) if d[3] > 0 else None
            r["speedup_vs_fp64_aa"] = r["mlups"] / r64["mlups"]
            res[f"{name}_aa" + ("_compact" if cp else "")] = r
            b.close()
    _, bad = ref.mass_momentum(check=False)
    res["fp64_nonfinite_cells"] = bad
    ref.close()
    return res


def run_precision_study(args):
    """512^3 porous channel, 300 steps: FP32 and FP16 storage of f - w
    (FP32 arithmetic) against the FP64 run of the same seed."""
    import lbmb200 as L

    n, steps = args.size or 512, args.steps
    peak, peak_kind = measured_hbm_peak()
    res = precision_study(L, n, steps, peak)
    wl = {"workload": res["workload"], "dims": [n] * 3,
          "solid_fraction_achieved": res["solid_fraction_achieved"], "spheres": res["spheres"],
          "steps": steps, "omega": 1.25, "lambda": 3 / 16, "xforce": 1e-6,
          "init": res["init"], "error": res["error"], "hbm_peak_gbs": peak,
          "hbm_peak_source": peak_kind, "l2_flush": "not needed: states of 5-20 GB > 126 MB L2"}
    f16 = res["fp16_aa"]
    return base_line(f16["mlups"], "MLUPS", steps, 0, f16["ms_per_step"], wl, "f32 (f16 storage)",
                     {"variants": res})


def run_adjoint_only(args):
    import lbmb200 as L
    a = adjoint_study(L, args.size or 128, args.steps, 100, 20)
    return base_line(a["fp64"]["s_per_step"], "s/step", args.steps, 5,
                     a["fp64"]["s_per_step"] * 1e3, {"workload": a["workload"]}, "f64",
                     {"adjoint": a})


def largest_study(L, n: int, steps: int, peak: float, na: int = 384, adj_steps: int = 1000):
    """The n^3 FP16 forward (30% solid, r 6-12, AA) and the na^3 FP32
    Brinkman adjoint with the sqrt checkpoint schedule, with device memory
    against the 180 GB HBM."""
    flags, frac, nsph = L.porous_channel((n, n, n), 0.3, 6.0, 12.0, seed=42)
    free0, total = L.device_memory()
    out = {}
    for cp in (False, True):
        s, fwd = timed_forward(L, flags, "aa", L.F16, steps, 3, peak, compact=cp)
        free1, _ = L.device_memory()
        _, bad = s.mass_momentum(check=False)
        fwd.update({"workload": f"FP16 porous channel {n}^3 (30% solid, r 6-12), AA, {steps} "
                                "steps", "nonfinite_cells": bad,
                    "device_used_bytes": total - free1, "device_total_bytes": total,
                    "solid_fraction_achieved": frac, "spheres": nsph})
        s.close()
        out["forward_fp16_aa" + ("_compact" if cp else "")] = fwd
    del flags
    a = adjoint_study(L, na, adj_steps, 0, 0, precisions=("fp32",))
    a["fp32"]["device_total_bytes"] = total
    out["adjoint"] = a
    return out


def run_largest(args):
    """768^3 FP16 forward (30% solid, r 6-12, 200 steps) and the 384^3
    FP32 Brinkman adjoint with the sqrt checkpoint schedule (1000 steps)."""
    import lbmb200 as L

    n = args.size or 768
    peak, peak_kind = measured_hbm_peak()
    res = largest_study(L, n, args.steps, peak)
    fwd = res["forward_fp16_aa"]
    wl = {"workload": f"largest single-GPU sizes: FP16 porous channel {n}^3 (30% solid, r 6-12), "
                      f"{args.steps} steps; FP32 Brinkman adjoint 384^3, 1000 steps, sqrt "
                      "checkpoint schedule",
          "hbm_peak_gbs": peak, "hbm_peak_source": peak_kind, "hbm_capacity_gb": 180}
    return base_line(fwd["mlups"], "MLUPS", args.steps, 3, fwd["ms_per_step"], wl,
                     "f32 (f16 storage)", res)


def ring_study(L, flags, f0, steps: int, warmup: int, plain_ms: float, compact: bool):
    """The halo-exchange data plane on one GPU: the x-periodic channel as one
    x-slab that is its own neighbour, FP64 AA, overlapped schedule. Three
    transports: the native ring through a one-rank NCCL communicator (send
    and receive to itself: the NCCL path of a multi-GPU run without a peer),
    the native ring with device copies, and the Python-driven SlabRunner.
    Device time with CUDA events on the solver's stream; `overhead` is the
    step time against the undecomposed solver's (plain_ms per step)."""
    import lbm_slab
    import torch

    out = {"workload": f"{flags.shape[2]}x{flags.shape[1]}x{flags.shape[0]} channel as one "
                       "x-slab, FP64 AA, ghost planes exchanged every odd step",
           "undecomposed_ms_per_step": plain_ms}
    for name in ("native_nccl", "native_copy", "python_copy"):
        s = L.Solver.slab(lbm_slab.slab_flags(flags, 0, flags.shape[2]), (0, 0), "aa", L.F64,
                          compact=compact)
        s.set_params(1.25, 3 / 16, 1e-6, True)
        s.set_state(f0)
        if name.startswith("native"):
            r = lbm_slab.NativeRunner(s, overlap=True, nccl=name == "native_nccl")
        else:
            r = lbm_slab.SlabRunner(s, lbm_slab.Ring(), overlap=True)
        r.scatter()
        r.run(warmup)
        s.synchronize()
        ext = torch.cuda.ExternalStream(s.stream)
        ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ex0, l0 = r.exchanges, s.launch_count
        t0 = time.perf_counter()
        ev0.record(ext)
        r.run(steps)
        ev1.record(ext)
        issue = time.perf_counter() - t0
        ev1.synchronize()
        ms = ev0.elapsed_time(ev1)
        out[name] = {"ms_per_step": ms / steps, "mlups": s.fluid_cells * steps / (ms / 1e3) / 1e6,
                     "overhead": ms / steps / plain_ms - 1, "exchanges": r.exchanges - ex0,
                     "step_launches": s.launch_count - l0,
                     "host_issue_ms_per_step": issue * 1e3 / steps}
        r.gather()
        tot, bad = s.mass_momentum(check=False)
        out[name]["nonfinite_cells"] = bad
        if hasattr(r, "close"):
            r.close()
        s.close()
    return out


def run_slabs(args, dist: Dist):
    """N GPUs: the porous channel of N x 256 x 256 x 256 cells cut into one
    256^3 x-slab per rank (weak scaling), FP64 AA, halo exchange between
    ring neighbours over NCCL every odd step, overlapped with the update of
    the interior planes. The step loop and the NCCL send/recv are issued by
    the library (lbm_ring_run through lbm_slab.NativeRunner), not by Python
    per step."""
    import lbm_slab
    import lbmb200 as L
    import numpy as np
    import torch

    n, world, rank = args.size, dist.world, dist.rank
    flags, frac, nsph = L.porous_channel((n * world, n, n), 0.2, 4.0, 8.0, seed=42)
    x0, x1 = lbm_slab.split(n * world, world, rank)
    sflags = lbm_slab.slab_flags(flags, x0, x1)
    del flags
    own = np.ascontiguousarray(sflags[:, :, 1:-1])
    f0 = L.perturbed_equilibrium(own, seed=7, amplitude=1e-4)
    peak, peak_kind = measured_hbm_peak()

    s = L.Solver.slab(sflags, (0, 0), "aa", L.F64, compact=args.layout == "compact")
    s.set_params(1.25, 3 / 16, 1e-6, True)
    s.set_state(f0)
    runner = lbm_slab.NativeRunner(s, overlap=True, timeout_ms=120000)
    ext = torch.cuda.ExternalStream(s.stream)
    runner.scatter()
    n_fluid = s.fluid_cells
    bpu = s.bytes_per_update
    runner.run(args.warmup)
    s.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    launches0, ex0 = s.launch_count, runner.exchanges
    dist.barrier()
    s.synchronize()
    with ClockSampler(dist.local) as clk:
        ev0.record(ext)
        runner.run(args.steps)
        ev1.record(ext)
        ev1.synchronize()
    dist.barrier()
    ms = dist.max(ev0.elapsed_time(ev1))
    total_fluid = dist.sum(float(n_fluid))
    # per exchange: the pack kernel, NCCL's grouped send/recv kernel, the unpack kernel
    launches = (s.launch_count - launches0) + 3 * (runner.exchanges - ex0)
    runner.gather()
    tot, bad = s.mass_momentum(check=False)
    mass = dist.sum(tot[0])
    value = total_fluid * args.steps / (ms / 1e3) / 1e6
    achieved = n_fluid * bpu * args.steps / (ms / 1e3) / 1e9

    # e2e: the state up from pinned host memory, the steps with their
    # exchanges, the state back down - host clock, max over ranks
    host = np.empty_like(f0)
    L.pin(f0)
    L.pin(host)
    dist.barrier()
    t0 = time.perf_counter()
    s.set_state(f0)
    runner.scatter()
    runner.run(args.steps)
    runner.gather()
    s.get_state(out=host)
    t = dist.max(time.perf_counter() - t0)
    L.unpin(f0)
    L.unpin(host)
    e2e = {"value": total_fluid * args.steps / t / 1e6, "unit": "MLUPS",
           "h2d_bytes_per_step": f0.nbytes / args.steps,
           "d2h_bytes_per_step": host.nbytes / args.steps, "seconds": t,
           "call": "lbm_set_state (pinned host) + lbm_ring_run (steps + NCCL halo exchange) + "
                   "lbm_get_state, per rank"}
    runner.close()
    s.close()
    return {
        "metric": METRIC, "value": value, "unit": "MLUPS", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded porous geometry and initial state)",
        "config": dict(WORKLOAD, workload=f"porous channel {n * world}x{n}x{n} (one {n}^3 x-slab "
                                          "per GPU), 20% solid spheres r 4-8, seed 42",
                       dims=[n * world, n, n], solid_fraction_achieved=frac, spheres=nsph,
                       fluid_cells=int(total_fluid), parallelism=f"x-slabs x{world}",
                       layout=args.layout,
                       halo="5 populations x 256 x 256 per face, before and after each odd "
                            "AA step, NCCL send/recv between ring neighbours issued from C "
                            "(lbm_ring_run), overlapped with the interior planes' update on a "
                            "second stream"),
        "gbs": achieved * world,
        "roofline": {"bound": "hbm", "kernel": "step_kernel<StoreF64> AA even+odd with halo "
                                               "exchange (whole step, per GPU)",
                     "achieved": achieved, "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": None,
                     "algorithmic_bytes_per_launch": n_fluid * bpu},
        "e2e": e2e, "gpu_launches": launches, "clocks": clk.summary(),
        "state_check": {"mass": mass, "nonfinite_cells_rank0": bad},
    }


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
        device_s = float(k.run(steps))  # kd->Duration: the step loop alone (CUDA events)
        t = time.perf_counter() - t0
        n_fluid = int((flags != 0).sum())
        nbytes = host.nbytes
    t = dist.max(t)
    transfer_s = max(t - device_s, 1e-9)
    return {"value": dist.world * n_fluid * steps / t / 1e6, "unit": "MLUPS",
            "h2d_bytes_per_step": nbytes / steps, "d2h_bytes_per_step": nbytes / steps,
            "h2d_bytes_per_call": nbytes, "d2h_bytes_per_call": nbytes, "seconds": t,
            "step_loop_seconds": device_s, "transfer_seconds": transfer_s,
            "transfer_gbs": 2 * nbytes / transfer_s / 1e9,
            "call": "kernelInitCudaAaSoA + kd->Kernel (host arrays in the reference's padded "
                    "layout, page-locked; upload + steps + download inside the timing)"}


def run_reference(args):
    """LBM-Bench's own CPU kernels on this host, same workload, metric and
    config as the native arm. Nothing of the product is loaded: the inputs
    come from the oracle's restatement of the workload generator (checked
    bit for bit against the product's in tests/test_host.py)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return None
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    n = args.size
    flags, frac, nsph = O.porous_channel((n, n, n), 0.2, 4.0, 8.0, seed=42)
    f0 = O.counter_equilibrium(flags, 7, 1e-4)
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
        "config": workload_config(n, frac, nsph, n_fluid),
        "execution": f"host CPU, {cb['cores']} OpenMP threads",
        "cpu_baseline": {"value": value, "unit": "MLUPS", "cores": cb["cores"],
                         "kind": "reference", "sample": cb["sample"]},
        "e2e": {"value": value, "unit": "MLUPS", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }


def run_profile_case(args):
    """A short run of the step kernels for profilers (ncu): the n^3 porous
    channel of the benchmark, for each precision in turn the seeded initial
    state uploaded (mask_kernel, then 19 pack_plane_kernel launches) and
    `--steps` steps of the pattern (AA alternates even, odd, ...). Prints
    one progress line per precision to standard error, no JSON line."""
    import lbmb200 as L

    pattern, _, precs = args.profile_run.partition(":")
    n = args.size
    flags, _, _ = L.porous_channel((n, n, n), 0.2, 4.0, 8.0, seed=42)
    f0 = L.perturbed_equilibrium(flags, seed=7, amplitude=1e-4)
    for prec in (precs or "fp64").split(","):
        with L.Solver(flags, (1, 0, 0), pattern, L.PRECISIONS[prec],
                      compact=args.layout == "compact") as s:
            s.set_params(1.25, 3 / 16, 1e-6, True)
            s.set_state(f0)
            ms = s.run_timed(args.steps)
            _, bad = s.mass_momentum(check=False)
            log(f"{n}^3 {pattern} {prec}: {s.fluid_cells} fluid cells, {args.steps} steps in "
                f"{ms:.3f} ms, {s.bytes_per_update:.0f} B/update, nonfinite {bad}")
            if bad:
                raise SystemExit("non-finite populations")


def _json_channel():
    """The one JSON line goes to the process's standard output; everything
    else written to file descriptor 1 - the C libraries' progress lines, the
    reference's printf, NCCL - is sent to standard error instead."""
    sys.stdout.flush()
    out = os.fdopen(os.dup(1), "w")
    os.dup2(2, 1)
    return out


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
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-studies", action="store_true",
                    help="skip the 512^3 precision study and the largest sizes")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the comparison with the reference at configs 0 and 1")
    ap.add_argument("--profile-run", metavar="PATTERN:PRECISIONS",
                    help="profiling case, e.g. aa:fp64,fp16 - `--steps` steps of the "
                         "pattern on the --size^3 porous channel, no JSON line")
    ap.add_argument("--layout", choices=["dense", "compact"], default="compact",
                    help="storage layout of the FP64 headline and of --profile-run "
                         "(compact: fluid cells only; default)")
    ap.add_argument("--config", type=int, choices=[1, 2, 3, 4], default=1,
                    help="1: 256^3 patterns (default); 2: 512^3 precision study; "
                         "3: 128^3 adjoint; 4: 768^3 FP16 and 384^3 adjoint")
    args = ap.parse_args()
    if args.profile_run:
        run_profile_case(args)
        return
    if args.warmup < 3:
        ap.error("--warmup must be >= 3")
    out = _json_channel()

    def emit(obj):
        out.write(json.dumps(obj) + "\n")
        out.flush()

    if args.config != 1:
        if args.impl == "reference" or args.gpus != 1:
            ap.error("--config 2-4 run the native arm on one GPU")
        defaults = {2: 300, 3: 2000, 4: 200}
        if "--steps" not in sys.argv:
            args.steps = defaults[args.config]
        if "--size" not in sys.argv:
            args.size = None
        fn = {2: run_precision_study, 3: run_adjoint_only, 4: run_largest}[args.config]
        emit(fn(args))
        return
    if args.impl == "reference":
        res = run_reference(args)
        if res is not None:
            emit(res)
        return
    dist = Dist(args.gpus)
    try:
        res = run_native(args, dist)
        if dist.rank == 0:
            emit(res)
    finally:
        dist.close()


if __name__ == "__main__":
    main()
