#!/usr/bin/env python
"""Benchmark of the fused LBM step (MLUPS and fraction of the HBM roofline).

Default workload: 512x256x256 D3Q27, FP32, regularized third-order Hermite
collision with Vreman LES, inflow/outflow in i, periodic j, no-slip bottom and
free-slip top in k, inflow-turbulence forcing at i=10 (seeded synthetic
fields), no solids.  One "step" is one lattice time step over the whole grid.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank advances its own independent replica (the path has no
exchange step between replicas); rank 0 prints one JSON line.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "MLUPS & % of HBM roofline: FP16-offset store vs plain FP32 at stated L2 error"
L2_NOTE = "inputs larger than L2: the two distribution buffers (7.8 GB) exceed the 126 MB L2, no flush needed"
FALLBACK_HBM_GBS = 6650.0
NOMINAL_HBM_GBS = 8000.0          # B200 HBM3e, the nominal figure the fraction is also quoted against


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=1000)
    ap.add_argument("--warmup", type=int, default=20)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--workload", default="turb_inflow_q27_512x256x256")
    ap.add_argument("--storage", choices=["f32", "f16"], default="f32")
    ap.add_argument("--kernel", choices=["pull", "pair"], default=None,
                    help="steady step kernel (default: the library's choice)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-f16", action="store_true", help="skip the FP16-offset storage comparison")
    ap.add_argument("--no-accuracy", action="store_true",
                    help="skip the FP16 error leg (city workload, 1000 steps, against the FP64 build)")
    ap.add_argument("--no-q19", action="store_true", help="skip the D3Q19 leg of the default workload")
    ap.add_argument("--no-ens", action="store_true", help="skip the batched-ensemble leg of the default run")
    ap.add_argument("--ensemble", action="store_true",
                    help="batched ensemble of 64 uneven D3Q19 members instead of the single-domain run")
    ap.add_argument("--members", type=int, default=64,
                    help="--ensemble: the first N of the 64 members (smaller captures for a profiler)")
    ap.add_argument("--adjoint", action="store_true",
                    help="checkpointed adjoint sweep of a probe-misfit loss (D3Q19 256x128x128 sphere, 100 steps)")
    ap.add_argument("--slabs", action="store_true",
                    help="the default workload as one j slab per rank (tile ny = workload ny) with the halo "
                         "exchange after every step: NCCL between ranks under torchrun, a ring of one tile "
                         "with itself on one GPU")
    ap.add_argument("--adjoint-step", action="store_true",
                    help="time one state-layout reverse step (lbm_state_adjoint_step) of the adjoint workload "
                         "against one fused forward step, on a resident state (about 2.5 GB)")
    ap.add_argument("--accuracy", action="store_true",
                    help="FP16-offset storage error study (city workload) instead of the timing run")
    ap.add_argument("--per-call", action="store_true",
                    help="main.F90's step through the per-call entry points (reference layout) on the workload, "
                         "FP32 and FP64 (the reference's DP build)")
    return ap.parse_args()


def bytes_per_lup(nl, storage):
    return 2 * nl * (2 if storage == "f16" else 4)


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def ncu_traffic(kernel_key, cells):
    """DRAM bytes per launch of the step kernel from the committed ncu summary,
    scaled by cells (traffic of this streaming kernel grows with the cells)."""
    path = os.path.join(ROOT, "profiles", "ncu_traffic.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        e = d[kernel_key]
        return float(e["dram_bytes_per_launch"]) * cells / float(e["cells"])
    except Exception:
        return None


# ---------------------------------------------------------------------------
# clocks during the timed region (NVML, sampled from a thread)
# ---------------------------------------------------------------------------
REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
           0x10: "sync_boost", 0x20: "sw_thermal_slowdown", 0x40: "hw_thermal_slowdown",
           0x80: "hw_power_brake_slowdown", 0x100: "display_clock_setting"}


class ClockSampler:
    def __init__(self, device_index):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._h = None
        try:
            import pynvml
            import torch
            pynvml.nvmlInit()
            props = torch.cuda.get_device_properties(device_index)
            bus = "%08X:%02X:%02X.0" % (props.pci_domain_id, props.pci_bus_id, props.pci_device_id)
            self._h = pynvml.nvmlDeviceGetHandleByPciBusId(bus)
            self._nv = pynvml
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception as e:   # clocks are reported as unavailable, never guessed
            self.error = str(e)

    def _reasons(self):
        nv = self._nv
        fn = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or nv.nvmlDeviceGetCurrentClocksThrottleReasons
        return fn(self._h)

    def _run(self):
        while not self._stop.is_set():
            try:
                self.samples.append(self._nv.nvmlDeviceGetClockInfo(self._h, self._nv.NVML_CLOCK_SM))
                self.reasons |= int(self._reasons())
            except Exception:
                pass
            self._stop.wait(0.02)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        if self._h is not None:
            self._stop.set()
            self._t.join()

    def report(self):
        if self._h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "note": "NVML unavailable"}
        names = [n for b, n in REASONS.items() if self.reasons & b and n != "gpu_idle"]
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": names, "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# CPU baseline: the oracle (restatement of the reference's OpenMP CPU path),
# timed by oracle/cpu_baseline.py in a fresh process that loads neither torch
# nor CUDA; both CPU legs (cpu_baseline and --impl reference) time the same
# 512x256x32 slab of the workload with one oracle run(n) call
# ---------------------------------------------------------------------------
def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def cpu_leg(wl, steps=None, warmup=2, budget_s=15.0):
    import subprocess
    cmd = [sys.executable, "-m", "oracle.cpu_baseline", "--workload", wl.name, "--warmup", str(warmup)]
    cmd += ["--steps", str(steps)] if steps is not None else ["--budget-s", str(budget_s)]
    out = subprocess.run(cmd, cwd=ROOT, capture_output=True, text=True, check=True)
    return json.loads(out.stdout.strip().splitlines()[-1])


def cpu_sample_text(r):
    return ("%dx%dx%d k-slab of the %s workload (%s FP32, same physics), %d steps in one run() call, %.1f s; C++ "
            "restatement of the reference's OpenMP CPU path (the Fortran reference has no compiler in this image), "
            "%d OpenMP threads on %s, fresh process without torch/CUDA"
            % (*r["slab"], r["workload"], r["lattice"], r["steps"], r["seconds"], r["threads"], r["cpu"]))


def cpu_baseline(wl):
    r = cpu_leg(wl)
    return {"value": r["value"], "unit": "MLUPS", "cores": r["threads"], "kind": "port", "sample": cpu_sample_text(r)}


# ---------------------------------------------------------------------------
# reference arm
# ---------------------------------------------------------------------------
def run_reference(a, wl):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    r = cpu_leg(wl, steps=a.steps, warmup=a.warmup)
    mlups = r["value"]
    line = {"impl": "reference", "metric": METRIC, "value": mlups, "unit": "MLUPS", "n_gpus": a.gpus,
            "steps": r["steps"], "warmup": a.warmup, "ms_per_step": round(r["seconds"] / r["steps"] * 1e3, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_of(wl, "f32", a.gpus),
            "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": r["threads"], "kind": "port",
                             "sample": cpu_sample_text(r)},
            "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def config_of(wl, storage, n):
    return {"workload": wl.name, "grid": [wl.nx, wl.ny, wl.nz], "lattice": "D3Q%d" % wl.nl, "storage": storage,
            "collision": "regularized 3rd-order Hermite + Vreman (Cs=0.15), nu=1e-4",
            "boundaries": "i inflow u=%.2f / outflow, j periodic, k no-slip bottom + free-slip top" % wl.uin,
            "forcing": "inflow turbulence at i=10, ampl=%g, nrturb=%d" % (wl.ampl, wl.nrturb) if wl.lturb else "none",
            "l2": L2_NOTE, "parallelism": "replicas x%d" % n if n > 1 else "single GPU"}


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def make_solver(wl, storage, seed, kernel=None):
    import torch
    from lbm_b200 import Params, Solver, workloads as W
    w2 = wl.with_(seed=seed)
    rho, u, v, w = (torch.from_numpy(x).cuda() for x in W.initial_macro(w2))
    uvel = torch.from_numpy(W.inflow_profile(w2)).cuda()
    tb = None
    if w2.lturb:
        uu, vv, ww = (torch.from_numpy(x).cuda() for x in W.turbulence_fields(w2.ny, w2.nz, w2.nrturb, w2.seed))
        tb = (uu, vv, ww, w2.nrturb, w2.ampl)
    p = Params(nx=w2.nx, ny=w2.ny, nz=w2.nz, nl=w2.nl, ibnd=w2.ibnd, jbnd=w2.jbnd, kbnd=w2.kbnd,
               kinevisc=w2.kinevisc, smagorinsky=w2.smagorinsky, iturb_pos=10, storage=storage)
    s = Solver(p, rho, u, v, w, uvel, blanking=None, turbulence=tb)
    if kernel is not None:
        s.lbm.set_kernel(kernel)
    del rho, u, v, w
    torch.cuda.synchronize()
    return s


def timed_steps(s, steps, dist, profile=True):
    """Time exactly `steps` fused steps with CUDA events on the library's stream; max over ranks.
    profile: the library also times every step kernel and the boundary launches
    after it with its own events (the mean kernel duration for the roofline);
    those events stand between consecutive launches and cost the launch
    overlap, so the step rate is taken from a run without them (measure_steps).
    Returns (ms, launches, step-kernel ms summed, step kernels timed, boundary ms summed)."""
    import torch
    from lbm_b200 import replicas
    L = s.lbm
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    L.profile(profile)
    n0 = L.launches
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(L.stream)
    s.step(steps)
    e1.record(L.stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1)
    launched = L.launches - n0
    kms, kn = L.profile_read() if profile else (0.0, 0)
    bms = L.profile_read_boundary()[0] if profile else 0.0
    L.profile(False)
    if dist is not None:
        ms = replicas.max_over_ranks(ms, device="cuda")
        dist.barrier()
    return ms, launched, kms, kn, bms


def measure_steps(s, steps, dist, clk_dev=None):
    """The step rate from `steps` steps timed without per-kernel events (inside the
    clock sampler when clk_dev is given), then the mean step-kernel duration from
    `steps` more steps timed kernel by kernel.  Returns (ms, launches, kernel ms
    summed, kernel launches, boundary ms summed, clock report or None)."""
    clk = None
    if clk_dev is not None:
        with ClockSampler(clk_dev) as sampler:
            ms, launched, _, _, _ = timed_steps(s, steps, dist, profile=False)
        clk = sampler.report()
    else:
        ms, launched, _, _, _ = timed_steps(s, steps, dist, profile=False)
    _, _, kms, kn, bms = timed_steps(s, steps, dist, profile=True)
    return ms, launched, kms, kn, bms, clk


def e2e_steps(s, steps, wl, dist):
    """End to end through the public host-buffer entry point: every step copies the
    inflow profile from pinned host memory and reads the status word back."""
    import torch
    from lbm_b200 import replicas, workloads as W
    uvel_host = torch.from_numpy(W.inflow_profile(wl)).pin_memory()
    if dist is not None:
        dist.barrier()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    bad = 0
    for _ in range(steps):
        bad |= s.lbm.step_host(1, uvel_host)
    torch.cuda.synchronize()
    el = time.perf_counter() - t0
    if dist is not None:
        el = replicas.max_over_ranks(el, device="cuda")
    return el, bad, wl.nz * 4, 4


# ---------------------------------------------------------------------------
# FP16-offset storage accuracy (the city workload, 1000 steps)
# ---------------------------------------------------------------------------
def gpu_run_macro(wl, storage, steps):
    """rho and (u, v, w) interior fields after `steps` fused steps, as float64 torch tensors."""
    import torch
    from lbm_b200 import Params, Solver, workloads as W
    rho, u, v, w = (torch.from_numpy(x).cuda() for x in W.initial_macro(wl))
    uvel = torch.from_numpy(W.inflow_profile(wl)).cuda()
    blank = W.blanking(wl)
    tb = None
    if wl.lturb:
        uu, vv, ww = (torch.from_numpy(x).cuda() for x in W.turbulence_fields(wl.ny, wl.nz, wl.nrturb, wl.seed))
        tb = (uu, vv, ww, wl.nrturb, wl.ampl)
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd,
               kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky, iturb_pos=10, storage=storage)
    s = Solver(p, rho, u, v, w, uvel, blanking=torch.from_numpy(blank).cuda() if blank is not None else None,
               turbulence=tb)
    del rho, u, v, w
    s.step(steps)
    r, uu_, vv_, ww_ = s.macro()
    inner = (slice(1, -1),) * 3
    out = (r[inner].double(), torch.stack([uu_[inner], vv_[inner], ww_[inner]]).double())
    st = s.lbm.status()
    s.close()
    torch.cuda.synchronize()
    return out, st


def dp_run_macro(wl, steps):
    """The same run through the per-call FP64 entry points on the GPU: the
    reference's double-precision build (DP=1), main.F90's init and step order."""
    import torch
    from lbm_b200 import Params, Solver, workloads as W
    rho, u, v, w = (torch.from_numpy(x).cuda().double() for x in W.initial_macro(wl))
    uvel = torch.from_numpy(W.inflow_profile(wl)).cuda().double()
    blank = W.blanking(wl)
    tb = None
    if wl.lturb:
        uu, vv, ww = (torch.from_numpy(x).cuda().double()
                      for x in W.turbulence_fields(wl.ny, wl.nz, wl.nrturb, wl.seed))
        tb = (uu, vv, ww, wl.nrturb, wl.ampl)
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd,
               kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky, iturb_pos=10)
    s = Solver(p, rho, u, v, w, uvel, blanking=torch.from_numpy(blank).cuda() if blank is not None else None,
               turbulence=tb, fused=False)
    del rho, u, v, w
    s.step(steps)
    r, uu_, vv_, ww_ = s.macro()
    inner = (slice(1, -1),) * 3
    out = (r[inner].clone(), torch.stack([uu_[inner], vv_[inner], ww_[inner]]))
    st = s.lbm.status()
    s.close()
    torch.cuda.synchronize()
    return out, st


def rel_l2_pair(a, b):
    """relative L2 of rho, of rho - 1 and of the velocity vector field, a against b."""
    import torch
    ra, ua = (torch.as_tensor(x, device="cuda", dtype=torch.float64) for x in a)
    rb, ub = (torch.as_tensor(x, device="cuda", dtype=torch.float64) for x in b)
    return {"rho": float(torch.linalg.vector_norm(ra - rb) / torch.linalg.vector_norm(rb)),
            "rho_minus_1": float(torch.linalg.vector_norm(ra - rb) / torch.linalg.vector_norm(rb - 1.0)),
            "u": float(torch.linalg.vector_norm(ua - ub) / torch.linalg.vector_norm(ub))}


def accuracy_errors(big, steps):
    """FP16-offset storage and plain FP32 (fused step, the library's default
    kernels) on `big` after `steps` steps, against the same run in FP64 through
    the DP build's per-call entry points on the GPU and against each other."""
    import torch
    t0 = time.perf_counter()
    f32, s32 = gpu_run_macro(big, "f32", steps)
    f16, s16 = gpu_run_macro(big, "f16", steps)
    torch.cuda.empty_cache()
    f64, s64 = dp_run_macro(big, steps)
    torch.cuda.empty_cache()
    e16, e32, e1632 = rel_l2_pair(f16, f64), rel_l2_pair(f32, f64), rel_l2_pair(f16, f32)
    return {"rel_l2_rho_vs_fp64": e16["rho"], "rel_l2_rho_minus_1_vs_fp64": e16["rho_minus_1"],
            "rel_l2_u_vs_fp64": e16["u"], "rel_l2_rho_vs_f32": e1632["rho"], "rel_l2_u_vs_f32": e1632["u"],
            "f32_vs_fp64": {"rel_l2_rho": e32["rho"], "rel_l2_u": e32["u"]},
            "error_bound": "relative L2 <= 1e-3 vs FP64",
            "error_config": {"workload": big.name, "grid": [big.nx, big.ny, big.nz], "steps": steps,
                             "solids": "%d seeded boxes, heights 10-40" % big.city,
                             "fp64": "the DP build's per-call entry points (_f64) on the GPU, main.F90's init and step order",
                             "u": "velocity vector field (u, v, w) over the interior cells"},
            "error_status_flags": [s32, s16, s64], "error_leg_s": round(time.perf_counter() - t0, 1)}


def accuracy_study(steps):
    """FP16-offset storage and plain FP32 (fused step) on the full city workload,
    against each other and against the same run in FP64 through the DP build's
    per-call entry points on the GPU, after `steps` steps each."""
    import torch
    from lbm_b200 import workloads as W
    torch.cuda.set_device(0)
    big = W.CITY_Q27
    t0 = time.perf_counter()
    f32, s32 = gpu_run_macro(big, "f32", steps)
    f16, s16 = gpu_run_macro(big, "f16", steps)
    torch.cuda.empty_cache()
    t1 = time.perf_counter()
    f64, s64 = dp_run_macro(big, steps)
    t2 = time.perf_counter()
    line = {"study": "fp16_offset_storage_accuracy", "steps": steps, "workload": big.name,
            "f16_vs_f64": rel_l2_pair(f16, f64), "f32_vs_f64": rel_l2_pair(f32, f64),
            "f16_vs_f32": rel_l2_pair(f16, f32), "status_flags": [s32, s16, s64],
            "f64": "the per-call FP64 entry points (the reference's DP build) on the GPU, %.1f s" % (t2 - t1),
            "bound": "relative L2 <= 1e-3 vs FP64", "gpu_s": round(t2 - t0, 1)}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# batched ensemble (64 uneven D3Q19 members)
# ---------------------------------------------------------------------------
def ensemble_measure(a, members, dist=None):
    """The batched ensemble of `members` (two launches per step for all members,
    CUDA-graph replay, autotuned launch shape) against the same members run one
    after another through the single-state path; the step kernel timed launch
    by launch (lbm_ensemble_profile) for its roofline fraction."""
    import torch
    from lbm_b200 import replicas
    from lbm_b200 import _lib
    from lbm_b200.ensemble import build_ensemble
    from lbm_b200 import Ensemble
    ens = build_ensemble(members, "f32")
    ens.step(1)
    variant, vms = ens.autotune(5)           # launch shape, then graph replay or direct launches
    _, graph_steps = ens.config()

    def prepare(g):
        # the mode g (graph steps, 0 = direct), a graph captured outside the timed region
        ens.set_graph(g)
        if g:
            if ens.members[0].it % 2:
                ens.step(1)                  # graphs start at parity 0
            ens.step(g)
        ens.step(a.warmup)
    prepare(graph_steps)

    def timed(fn, n):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        fn(n)
        e1.record()
        torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        if dist is not None:
            ms = replicas.max_over_ranks(ms, device="cuda")
        return ms

    with ClockSampler(torch.cuda.current_device()) as clk:
        ms = timed(ens.step, a.steps)
    other = 0 if graph_steps else _lib.LBM_ENS_GRAPH_STEPS
    prepare(other)
    ms_other = timed(ens.step, a.steps)
    prepare(graph_steps)
    k_step, k_bc = ens.profile(a.steps)

    def sequential(n):
        for L in ens.members:
            L.step(n)
    ms_seq = timed(sequential, a.steps)
    st = max(L.status() for L in ens.members)
    ens.close()
    cells = sum(m.cells for m in members)
    hbm, hbm_kind = peaks()
    bl = bytes_per_lup(19, "f32")
    mlups = lambda t: cells * a.steps / (t * 1e-3) / 1e6
    return {"value": round(mlups(ms), 1), "unit": "MLUPS", "ms_per_step": round(ms / a.steps, 4), "cells": cells,
            "members": len(members),
            "batched": {"launches_per_step": 2, "graph_steps": graph_steps,
                        "autotune": {"variant": variant, "shape": Ensemble.variant_shape(variant),
                                     "shapes": [Ensemble.variant_shape(v) for v in range(_lib.LBM_ENS_VARIANTS)],
                                     "shape_ms_per_step": [round(x, 4) for x in vms],
                                     "how": "each (threads per block, min blocks per SM, tiles per block) shape "
                                            "over 5 direct-launch steps, then the fastest replayed from %d-step "
                                            "graphs vs launched directly" % _lib.LBM_ENS_GRAPH_STEPS}},
            ("direct_launches" if graph_steps else "graph_replay"):
                {"value": round(mlups(ms_other), 1), "ms_per_step": round(ms_other / a.steps, 4)},
            "sequential": {"value": round(mlups(ms_seq), 1), "ms_per_step": round(ms_seq / a.steps, 4),
                           "how": "lbm_step on each member's context in turn, %d steps each" % a.steps},
            "speedup_vs_sequential": round(ms_seq / ms, 3),
            "roofline": {"bound": "hbm", "achieved": round(cells * bl / (k_step * 1e-3) / 1e9, 1), "peak": hbm,
                         "unit": "GB/s", "frac": round(cells * bl / (k_step * 1e-3) / 1e9 / hbm, 4),
                         "peak_kind": hbm_kind, "kernel": "k_ens_step<19,float>", "kernel_ms": round(k_step, 4),
                         "traffic": ncu_traffic("k_ens_step<19,float>", cells),
                         "boundary_kernel_ms": round(k_bc, 4),
                         "step_frac": round(cells * bl / (ms / a.steps * 1e-3) / 1e9 / hbm, 4),
                         "note": "frac: the step kernel alone (CUDA events around each launch, %d direct-launch "
                                 "steps); step_frac: the whole graph-replayed step, 152 B per cell update" % a.steps},
            "clocks": clk.report(), "status_flags": st}


def ensemble_bench(a):
    """The batched-ensemble benchmark as its own JSON line.  Under torchrun the
    members are dealt out round-robin to the ranks (independent replicas)."""
    import torch
    from lbm_b200 import replicas, workloads as W
    rank, local, world = replicas.env_rank()
    dist = None
    if world > 1:
        torch.cuda.set_device(local)
        dist = replicas.init("nccl", timeout_s=300, device=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    allm = W.ensemble_members()[:a.members]
    mine = [m for k, m in enumerate(allm) if k % world == rank]
    r = ensemble_measure(a, mine, dist)
    cells = sum(m.cells for m in allm)
    line = {"metric": "aggregate MLUPS of a batched ensemble vs the same members run one after another",
            "value": round(cells / (r["ms_per_step"] * 1e-3) / 1e6, 1),   # every rank's members, max-over-ranks time
            "unit": "MLUPS", "n_gpus": world, "steps": a.steps, "warmup": a.warmup,
            "ms_per_step": r["ms_per_step"], "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f32", "data": "synthetic (seeded member sizes, inflow speeds and inflow-turbulence fields)",
            "config": {"workload": "ensemble_q19_%d_members" % len(allm), "members": len(allm), "cells": cells,
                       "sizes": "nx in [96,192], ny, nz in [48,96], multiples of 8 (seeded)",
                       "physics": "D3Q19 FP32 regularized + Vreman, inflow U[0.03,0.07], turbulence ampl 1e-4 at i=10",
                       "parallelism": "members round-robin over %d GPU(s)" % world if world > 1 else "single GPU",
                       "l2": "inputs larger than L2: %.1f GB of state" % (cells * 19 * 4 * 2 / 1e9)},
            "gpu_launches": 2 * a.steps}
    for k in ("batched", "direct_launches", "graph_replay", "sequential", "speedup_vs_sequential", "roofline",
              "clocks", "status_flags"):
        if k in r:
            line[k] = r[k]
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# adjoint: probe-misfit gradient through 100 steps, checkpoints every 10
# ---------------------------------------------------------------------------
def adjoint_bench(a):
    """Time of the checkpointed reverse sweep against the forward run it
    differentiates (the per-call path, keeping checkpoints), and against the
    fused forward step for the same steps."""
    import torch
    from lbm_b200 import Params, Solver, workloads as W
    from lbm_b200.adjoint import ProbeProblem, initial_state
    torch.cuda.set_device(0)
    wl = W.ADJOINT_Q19
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=10,
               kinevisc=wl.kinevisc)
    blank = torch.from_numpy(W.blanking(wl)).cuda()
    probes = W.probe_cells(wl, 200, 0)
    pb = ProbeProblem(p, probes, wl.steps, blanking=blank, checkpoint=10)
    rho, u, v, w = (torch.from_numpy(x).cuda() for x in W.initial_macro(wl))
    uvel = torch.from_numpy(W.inflow_profile(wl)).cuda()
    f1, f2 = initial_state(pb.lbm, rho, u, v, w, uvel)
    R = pb._macro(f1)
    for _ in range(20):                       # leave the exact initial equilibrium
        f1, f2 = pb._step(f1, f2, R, uvel)
    truth = pb.forward(f1, f2, uvel + torch.from_numpy(W.inflow_perturbation(wl.nz, 0, 5e-3)).cuda(), keep=False)

    def ev():
        return torch.cuda.Event(enable_timing=True)
    pb.forward(f1, f2, uvel)                  # warm-up of every kernel
    pb.backward(torch.zeros(len(probes), 3, device="cuda"))
    torch.cuda.synchronize()
    e0, e1, e2 = ev(), ev(), ev()
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record()
        up = pb.forward(f1, f2, uvel)
        e1.record()
        gf, gu = pb.backward(2.0 * (up - truth))
        e2.record()
        torch.cuda.synchronize()
    t_fwd, t_bwd = e0.elapsed_time(e1), e1.elapsed_time(e2)
    loss = float(((up.double() - truth.double()) ** 2).sum())
    gnorm_f, gnorm_u = float(gf.double().norm()), float(gu.double().norm())
    pb.close()
    torch.cuda.empty_cache()
    # the same gradient with the fused forward and the state-layout reverse sweep
    from lbm_b200.adjoint import FusedProbeProblem
    fb = FusedProbeProblem(p, probes, wl.steps, blanking=blank, checkpoint=10)
    fb.forward(f1, f2, uvel)
    fb.backward(torch.zeros(len(probes), 3, device="cuda"))
    torch.cuda.synchronize()
    s0, s1, s2 = ev(), ev(), ev()
    s0.record()
    us = fb.forward(f1, f2, uvel)
    s1.record()
    sf, su = fb.backward(2.0 * (us - truth))
    s2.record()
    torch.cuda.synchronize()
    ts_fwd, ts_bwd = s0.elapsed_time(s1), s1.elapsed_time(s2)
    agree = float((sf - gf).abs().max() / gf.abs().max())
    # the same reverse sweep with replay and reverse one after the other
    s3, s4 = ev(), ev()
    s3.record()
    tf, tu = fb.backward(2.0 * (us - truth), overlap=False)
    s4.record()
    torch.cuda.synchronize()
    ts_serial = s3.elapsed_time(s4)
    agree_serial = float((tf - gf).abs().max() / gf.abs().max())
    del tf, tu
    fb.close()
    del sf, su
    torch.cuda.empty_cache()
    # the fused forward for the same steps, for scale
    s = Solver(p, rho, u, v, w, uvel, blanking=blank)
    s.step(3)
    torch.cuda.synchronize()
    f0, f9 = ev(), ev()
    f0.record()
    s.step(wl.steps)
    f9.record()
    torch.cuda.synchronize()
    t_fused = f0.elapsed_time(f9)
    s.close()
    cells = wl.cells
    line = {"metric": "adjoint sweep time over forward time (probe-misfit gradient, checkpoint-and-recompute)",
            "value": round(ts_bwd / t_fused, 3), "unit": "x the fused forward (state-layout reverse sweep)",
            "n_gpus": 1, "steps": wl.steps,
            "warmup": 1, "higher_is_better": False, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded initial field, probes and inflow perturbation)",
            "config": {"workload": wl.name, "grid": [wl.nx, wl.ny, wl.nz], "lattice": "D3Q19",
                       "sphere": list(wl.sphere), "probes": len(probes), "checkpoint_every": 10,
                       "controls": "initial f1 (rho, u recomputed from it) and the inflow profile uvel(k)",
                       "target": "same run with uvel + 5e-3 smooth seeded noise"},
            "fused_forward_ms": round(t_fused, 2),
            "state_layout_sweep": {"forward_ms": round(ts_fwd, 2), "reverse_ms": round(ts_bwd, 2),
                                   "reverse_over_forward": round(ts_bwd / ts_fwd, 3),
                                   "reverse_over_fused_forward": round(ts_bwd / t_fused, 3),
                                   "reverse_ms_without_overlap": round(ts_serial, 2),
                                   "gradient_without_overlap_vs_per_call_sweep": agree_serial,
                                   "gradient_vs_per_call_sweep": agree,
                                   "how": "forward by the fused step with a device snapshot every 10 steps "
                                          "(lbm_state_snapshot); reverse restores each segment, replays it "
                                          "into per-step buffers (lbm_step_to) on a second context and stream "
                                          "while the adjoint steps of the segment after it run "
                                          "(lbm_state_adjoint_step)"},
            "per_call_sweep": {"forward_ms": round(t_fwd, 2), "reverse_ms": round(t_bwd, 2),
                               "reverse_over_forward": round(t_bwd / t_fwd, 3),
                               "reverse_over_fused_forward": round(t_bwd / t_fused, 3),
                               "forward_mlups": round(cells * wl.steps / (t_fwd * 1e-3) / 1e6, 1),
                               "how": "forward by the per-call kernels (reference layout) with checkpoints; "
                                      "reverse by lbm_macrovars_drift_adj, lbm_boundarycond_adj and "
                                      "lbm_postcoll_adj"},
            "loss": loss, "grad_norm": {"f1": gnorm_f, "uvel": gnorm_u},
            "gradient_check": "tests/test_gpu_adjoint.py: central FP64 differences, 8 seeded directions, rel <= 1e-4",
            "clocks": clk.report()}
    print(json.dumps(line), flush=True)
    return 0


def adjoint_step_bench(a):
    """One reverse step of the state-layout sweep (D3Q19 256x128x128 sphere):
    lbm_state_adjoint_step pulling from a stepped state, timed over K calls,
    beside one fused forward step.  Algorithmic traffic of the cell kernel:
    the adjoint gathered (Q floats), the pulled state (Q) and the adjoint
    written (Q) per interior cell."""
    import torch
    from lbm_b200 import Params, workloads as W
    from lbm_b200.adjoint import FusedProbeProblem, ProbeProblem, initial_state
    torch.cuda.set_device(0)
    wl = W.ADJOINT_Q19
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=10,
               kinevisc=wl.kinevisc)
    blank = torch.from_numpy(W.blanking(wl)).cuda()
    probes = W.probe_cells(wl, 200, 0)
    fb = FusedProbeProblem(p, probes, 10, blanking=blank)
    L = fb.lbm
    rho, u, v, w = (torch.from_numpy(x).cuda() for x in W.initial_macro(wl))
    fb.uvel = torch.from_numpy(W.inflow_profile(wl)).cuda()
    pp = ProbeProblem(p, probes, 10, blanking=blank)
    f1, f2 = initial_state(pp.lbm, rho, u, v, w, fb.uvel)
    pp.close()
    fb._import(f1, f2)
    del f1, f2
    L.step(3)
    P = L.state_scratch()
    L.state_copy(P)
    Wt, At = L.empty_state(), L.empty_state()
    At.normal_(0.0, 1e-3, generator=torch.Generator(device="cuda").manual_seed(1))
    uh = torch.zeros(wl.nz, dtype=torch.float32, device="cuda")
    steps, warm = max(1, a.steps if a.steps != 1000 else 50), max(3, a.warmup if a.warmup != 20 else 5)

    def ev():
        return torch.cuda.Event(enable_timing=True)
    for _ in range(warm):
        L.state_adjoint_step(Wt, At, P, True, uh)
        Wt, At = At, Wt
        L.step(1)
    torch.cuda.synchronize()
    e0, e1, e2 = ev(), ev(), ev()
    with ClockSampler(torch.cuda.current_device()) as clk:
        e0.record()
        for _ in range(steps):
            L.state_adjoint_step(Wt, At, P, True, uh)
            Wt, At = At, Wt
        e1.record()
        L.step(steps)
        e2.record()
        torch.cuda.synchronize()
    t_rev, t_fwd = e0.elapsed_time(e1) / steps, e1.elapsed_time(e2) / steps
    cells = wl.cells
    hbm, hbm_kind = peaks()
    line = {"metric": "state-layout reverse step time over fused forward step time", "value": round(t_rev / t_fwd, 3),
            "unit": "x", "n_gpus": 1, "steps": steps, "warmup": warm, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded state and adjoint)",
            "config": {"workload": "adjoint_step_" + wl.name, "grid": [wl.nx, wl.ny, wl.nz], "lattice": "D3Q19",
                       "l2": "inputs larger than L2 (3 x 331 MB per step)"},
            "reverse_step_ms": round(t_rev, 4), "fused_step_ms": round(t_fwd, 4),
            "reverse_step_bytes_per_cell": 3 * wl.nl * 4,
            "reverse_step_gbs_of_cell_traffic": round(3 * wl.nl * 4 * cells / (t_rev * 1e-3) / 1e9, 1),
            "hbm_peak_gbs": hbm, "hbm_peak_kind": hbm_kind, "clocks": clk.report()}
    print(json.dumps(line), flush=True)
    fb.close()
    return 0


def per_call_bench(a):
    """MLUPS of main.F90's step (main.F90:283-329) made of the per-call entry
    points on reference-layout arrays: inflow-turbulence forcing, postcoll,
    turbulence apply, boundarycond, drift, macrovars.  This is the path a
    Fortran driver gets by switching its calls one by one; the FP64 arm is the
    DP build's (the _f64 entry points)."""
    import torch
    from lbm_b200 import Lbm, Params, workloads as W
    from lbm_b200.adjoint import initial_state
    torch.cuda.set_device(0)
    wl = W.WORKLOADS[a.workload]
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=10,
               kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky)
    out = {}
    for name, dt in (("f32", torch.float32), ("f64", torch.float64)):
        L = Lbm(p)
        rho, u, v, w = (torch.from_numpy(x).cuda().to(dt) for x in W.initial_macro(wl))
        uvel = torch.from_numpy(W.inflow_profile(wl)).cuda().to(dt)
        f1, f2 = initial_state(L, rho, u, v, w, uvel)
        L.macrovars(rho, u, v, w, f1)
        tau = torch.full(p.sshape, 3.0 * wl.kinevisc + 0.5, dtype=dt, device="cuda")
        turb = [torch.from_numpy(x).cuda().to(dt) for x in W.turbulence_fields(wl.ny, wl.nz, wl.nrturb, wl.seed)]
        df = torch.zeros((wl.nz, wl.ny, wl.nl), dtype=dt, device="cuda")
        it = [0]

        def step():
            it[0] += 1
            if wl.lturb:
                L.inflow_turbulence_forcing(df, rho, u, v, w, *turb, wl.ampl, it[0], wl.nrturb)
            L.postcoll(f1, tau, rho, u, v, w)
            if wl.lturb:
                L.inflow_turbulence_apply(f1, df)
            L.boundarycond(f1, f2, uvel)
            L.drift(f2, f1)
            L.macrovars(rho, u, v, w, f2)

        def swap_step():
            nonlocal f1, f2
            step()
            f1, f2 = f2, f1

        for _ in range(a.warmup):
            swap_step()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        n0 = L.launches
        with ClockSampler(torch.cuda.current_device()) as clk:
            e0.record(L.stream)
            for _ in range(a.steps):
                swap_step()
            e1.record(L.stream)
            torch.cuda.synchronize()
        ms = e0.elapsed_time(e1)
        out[name] = {"value": round(wl.cells * a.steps / (ms * 1e-3) / 1e6, 1), "unit": "MLUPS",
                     "ms_per_step": round(ms / a.steps, 4), "gpu_launches": L.launches - n0,
                     "status": L.status(), "clocks": clk.report()}
        L.close()
        del f1, f2, rho, u, v, w, tau, turb, df
        torch.cuda.empty_cache()
    print(json.dumps({"metric": "MLUPS of the per-call step (reference layout, main.F90:283-329)", "unit": "MLUPS",
                      "value": out["f32"]["value"], "higher_is_better": True, "n_gpus": 1, "steps": a.steps,
                      "warmup": a.warmup, "config": {"workload": wl.name, "grid": [wl.nx, wl.ny, wl.nz],
                                                     "lattice": "D3Q%d" % wl.nl},
                      "data": "synthetic (seeded initial field and turbulence fields)",
                      "f32": out["f32"], "f64_dp_build": out["f64"]}))
    return 0


def slab_bench(a):
    """MLUPS of j slabs: each rank steps one tile of the default workload's size
    (weak scaling: the domain grows in j with the ranks) and exchanges its halo
    planes after every step (lbm_b200.slabs).  Device time with CUDA events,
    max over ranks."""
    import torch
    from lbm_b200 import Params, replicas, slabs, workloads as W
    from lbm_b200.adjoint import initial_state
    rank, local, world = replicas.env_rank()
    torch.cuda.set_device(local)
    if world > 1:
        replicas.init("nccl", timeout_s=120, device=torch.device("cuda", local))
    wl = W.WORKLOADS[a.workload]
    gp = Params(nx=wl.nx, ny=wl.ny * world, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd,
                iturb_pos=min(10, wl.nx), kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky,
                storage=a.storage)
    tile = slabs.SlabTile(gp, rank, world)
    tw = wl.with_(seed=replicas.replica_seed(wl.seed, rank))
    rho, u, v, w = (torch.from_numpy(x).cuda() for x in W.initial_macro(tw))
    uvel = torch.from_numpy(W.inflow_profile(tw)).cuda()
    tile.set_inflow(uvel)
    f1, f2 = initial_state(tile.lbm, rho, u, v, w, uvel)
    R = [tile.lbm.empty_s() for _ in range(4)]
    tile.lbm.macrovars(*R, f1)
    tile.lbm.state_import(f1, f2, *R)
    del f1, f2, R, rho, u, v, w

    def run(n):
        if world > 1:
            tile.step(n)
        else:
            slabs.step_local([tile], n)
    run(max(3, a.warmup))
    torch.cuda.synchronize()
    steps = a.steps if a.steps != 1000 else 200
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        e0.record()
        run(steps)
        e1.record()
        torch.cuda.synchronize()
    ms = replicas.max_over_ranks(e0.elapsed_time(e1), device="cuda" if world > 1 else "cpu")
    cells = wl.nx * wl.ny * wl.nz * world
    plane = tile.lbm.halo_plane_bytes()
    line = {"metric": "MLUPS of j slabs with the halo exchange after every step", "value":
            round(cells * steps / (ms * 1e-3) / 1e6, 1), "unit": "MLUPS", "n_gpus": world, "steps": steps,
            "warmup": max(3, a.warmup), "ms_per_step": round(ms / steps, 4), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": a.storage, "data": "synthetic (seeded per tile)",
            "config": {"workload": "slabs_" + wl.name, "tiles": world, "tile": [wl.nx, wl.ny, wl.nz],
                       "lattice": "D3Q%d" % wl.nl, "exchange": "nccl p2p" if world > 1 else "one tile, a ring to itself",
                       "turbulence": "none (the slab tiles carry no inflow-turbulence slice here)",
                       "l2": "inputs larger than L2"},
            "halo_bytes_per_step_per_tile": 2 * plane, "clocks": clk.report()}
    if rank == 0:
        print(json.dumps(line), flush=True)
    tile.close()
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    return 0


def lattice_leg(a, wl, hbm):
    """The same timed run on another lattice of the workload (FP32 and FP16-offset storage)."""
    import torch
    out = {"workload": wl.name, "lattice": "D3Q%d" % wl.nl}
    for storage in ("f32", "f16"):
        s = make_solver(wl, storage, seed=wl.seed, kernel=a.kernel)
        s.step(a.warmup)
        ms, _, kms, kn, bms, _ = measure_steps(s, a.steps, None)
        st = s.lbm.status()
        s.close()
        del s
        torch.cuda.empty_cache()
        k_ms = kms / max(kn, 1)
        bl = bytes_per_lup(wl.nl, storage)
        r = {"value": round(wl.cells * a.steps / (ms * 1e-3) / 1e6, 1), "unit": "MLUPS",
             "ms_per_step": round(ms / a.steps, 4), "kernel_ms": round(k_ms, 4),
             "boundary_kernel_ms": round(bms / max(kn, 1), 4), "bytes_per_lup": bl,
             "roofline_frac": round(wl.cells * bl / (k_ms * 1e-3) / 1e9 / hbm, 4) if kn else None,
             "status_flags": st}
        if storage == "f32":
            out.update(r)
        else:
            r["speedup_vs_f32"] = round(r["value"] / out["value"], 3)
            out["f16_storage"] = r
    return out


def main():
    a = parse()
    if a.slabs and a.impl == "ours":
        return slab_bench(a)
    if a.per_call and a.impl == "ours":
        return per_call_bench(a)
    if a.adjoint_step and a.impl == "ours":
        return adjoint_step_bench(a)
    if a.adjoint and a.impl == "ours":
        return adjoint_bench(a)
    if a.ensemble and a.impl == "ours":
        return ensemble_bench(a)
    from lbm_b200 import workloads as W
    wl = W.WORKLOADS[a.workload]
    if a.impl == "reference":
        return run_reference(a, wl)
    if a.accuracy:
        return accuracy_study(a.steps)

    import torch
    from lbm_b200 import replicas
    rank, local, world = replicas.env_rank()
    dist = None
    if world > 1:
        torch.cuda.set_device(local)
        dist = replicas.init("nccl", timeout_s=120, device=torch.device("cuda", local))
    else:
        torch.cuda.set_device(0)
    dev = torch.cuda.current_device()

    s = make_solver(wl, a.storage, seed=replicas.replica_seed(wl.seed, rank), kernel=a.kernel)
    s.step(a.warmup)
    torch.cuda.synchronize()
    ms, launched, kms, kn, bms, clocks = measure_steps(s, a.steps, dist, clk_dev=dev)
    st = s.lbm.status()
    cells = wl.cells
    value = world * cells * a.steps / (ms * 1e-3) / 1e6
    hbm, hbm_kind = peaks()
    bl = bytes_per_lup(wl.nl, a.storage)
    k_ms = kms / max(kn, 1)
    achieved = cells * bl / (k_ms * 1e-3) / 1e9 if kn else None
    key = "%s<%d,%s>" % ("k_step_fast" if a.kernel == "pull" else "k_step_pair", wl.nl,
                         "float" if a.storage == "f32" else "__half")
    traffic = ncu_traffic(key, cells)
    line = {"metric": METRIC, "value": round(value, 1), "unit": "MLUPS", "n_gpus": world, "steps": a.steps,
            "warmup": a.warmup, "ms_per_step": round(ms / a.steps, 4), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32" if a.storage == "f32" else "f16-storage/f32-compute",
            "data": "synthetic (seeded initial field, seeded smooth inflow-turbulence fields)",
            "config": config_of(wl, a.storage, world),
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1) if achieved else None, "peak": hbm,
                         "unit": "GB/s", "frac": round(achieved / hbm, 4) if achieved else None,
                         "traffic": traffic, "peak_kind": hbm_kind,
                         "kernel": key, "kernel_ms": round(k_ms, 4), "kernel_launches": kn,
                         "boundary_kernel_ms": round(bms / max(kn, 1), 4),
                         "algorithmic_bytes_per_launch": cells * bl,
                         "frac_of_nominal_8000_gbs": round(achieved / NOMINAL_HBM_GBS, 4) if achieved else None,
                         "note": "frac of %s HBM copy bandwidth; kernel_ms and boundary_kernel_ms: mean "
                                 "durations of the step kernel and of the boundary kernel after it (k_bc_fold), "
                                 "over a second run of the same steps timed launch by launch (value and "
                                 "ms_per_step come from the run without per-launch events); traffic = ncu dram "
                                 "bytes per launch" % hbm_kind},
            "gpu_launches": launched, "clocks": clocks, "status_flags": st}

    if not a.no_e2e:
        el, bad, h2d, d2h = e2e_steps(s, a.steps, wl, dist)
        line["e2e"] = {"value": round(world * cells * a.steps / el / 1e6, 1), "unit": "MLUPS",
                       "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                       "api": "lbm_step_host (uvel host->device, status word device->host, per step)"}
    s.close()
    del s
    torch.cuda.empty_cache()

    if not a.no_f16 and a.storage == "f32" and world == 1:
        s16 = make_solver(wl, "f16", seed=replicas.replica_seed(wl.seed, rank), kernel=a.kernel)
        s16.step(a.warmup)
        ms16, _, kms16, kn16, bms16, _ = measure_steps(s16, a.steps, dist)
        s16.close()
        v16 = world * cells * a.steps / (ms16 * 1e-3) / 1e6
        ach16 = cells * bytes_per_lup(wl.nl, "f16") / (kms16 / max(kn16, 1) * 1e-3) / 1e9 if kn16 else None
        line["f16_storage"] = {"value": round(v16, 1), "unit": "MLUPS", "speedup_vs_f32": round(v16 / value, 3),
                               "roofline_frac": round(ach16 / hbm, 4) if ach16 else None,
                               "kernel_ms": round(kms16 / max(kn16, 1), 4),
                               "traffic": ncu_traffic("k_step_pair<%d,__half>" % wl.nl, cells),
                               "boundary_kernel_ms": round(bms16 / max(kn16, 1), 4),
                               "ms_per_step": round(ms16 / a.steps, 4)}
        torch.cuda.empty_cache()
        if not a.no_accuracy and wl.name == W.CHANNEL_Q27.name:
            # the stated-error half of the metric: the city workload after its 1000 steps
            line["f16_storage"].update(accuracy_errors(W.CITY_Q27, W.CITY_Q27.steps))

    if not a.no_q19 and world == 1 and wl.name == W.CHANNEL_Q27.name:
        line["q19"] = lattice_leg(a, W.CHANNEL_Q19, hbm)
    if not a.no_ens and world == 1 and wl.name == W.CHANNEL_Q27.name:
        line["ensemble"] = dict(workload="ensemble_q19_64_members", **ensemble_measure(a, W.ensemble_members()))
        torch.cuda.empty_cache()

    if rank == 0 and world == 1 and not a.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line), flush=True)
    return 0


if __name__ == "__main__":
    sys.exit(main())
