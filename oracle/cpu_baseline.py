"""Timed CPU baseline of the LBM step: the oracle's time loop (the C++
restatement of the reference's OpenMP CPU path, main.F90:283-329) on a k-slab
of a workload.  TEST AND MEASUREMENT INFRASTRUCTURE ONLY: bench.py runs this
module as a subprocess for its CPU legs (the ``cpu_baseline`` object and the
``--impl reference`` arm); nothing in the product imports it.

It runs in a fresh process that never loads torch or CUDA, so that the only
OpenMP runtime and the only threads in the process are the oracle's, and it
times one ``run(n)`` call over n steps (n given, or the even number of steps
that fits a time budget).  Both CPU legs therefore time the same slab shape
the same way.

    python -m oracle.cpu_baseline --workload turb_inflow_q27_512x256x256 \\
        [--nz 32] [--steps N | --budget-s 15] [--warmup 2] [--threads T]

prints one JSON line: MLUPS, cells, steps, seconds, threads, the CPU model.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import os
import platform
import sys
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

SLAB_NZ = 32     # k-planes of the timed slab: 512x256x32 = 4.2 M cells for the channel workloads


def workloads_module():
    """lbm_b200/workloads.py loaded by path: the package itself imports torch."""
    name = "lbm_workloads_cpu"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "lbm_b200", "workloads.py"))
        m = importlib.util.module_from_spec(spec)
        sys.modules[name] = m
        spec.loader.exec_module(m)
    return sys.modules[name]


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return platform.processor() or "unknown"


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def make_case(wl, nz):
    import numpy as np
    from oracle import oracle as O
    W = workloads_module()
    s = wl.with_(nz=nz)
    cfg = O.Config(s.nx, s.ny, s.nz, s.nl, ibnd=s.ibnd, jbnd=s.jbnd, kbnd=s.kbnd, iturb_pos=10, lturb=s.lturb,
                   nrturb=s.nrturb, ampl=s.ampl, kinevisc=s.kinevisc, smagorinsky=s.smagorinsky)
    o = O.Oracle(cfg, np.float32)
    rho, u, v, w = W.initial_macro(s)
    uvel = W.inflow_profile(s)
    fA, fB = o.zeros_f(), o.zeros_f()
    o.init(fA, fB, rho, u, v, w, uvel)
    tau = np.full(cfg.sshape, 3 * np.float32(s.kinevisc) + 0.5, np.float32)
    kw = {}
    if s.lturb:
        uu, vv, ww = W.turbulence_fields(s.ny, s.nz, s.nrturb, s.seed)
        kw = dict(uu=uu, vv=vv, ww=ww)
    state = {"it": 0}

    def run(n):
        o.run(fA, fB, rho, u, v, w, tau, uvel, n, it0=state["it"], **kw)
        state["it"] += n
    return s, run


def measure(workload, nz=SLAB_NZ, steps=None, budget_s=15.0, warmup=2, threads=None):
    from oracle import oracle as O
    W = workloads_module()
    wl = W.WORKLOADS[workload]
    threads = threads or host_threads()
    O.set_threads(threads)
    s, run = make_case(wl, min(nz, wl.nz))
    t0 = time.perf_counter()
    if warmup:
        run(warmup)
    if steps is None:
        # budget mode: as many steps as fit budget_s, an even number (no final state exchange)
        per_step = (time.perf_counter() - t0) / max(warmup, 1)
        steps = max(2, int(budget_s / max(per_step, 1e-6)))
        steps += steps % 2
    t0 = time.perf_counter()
    run(steps)
    el = time.perf_counter() - t0
    return {"value": round(s.cells * steps / el / 1e6, 3), "unit": "MLUPS", "cells": s.cells, "steps": steps,
            "seconds": round(el, 3), "threads": threads, "omp_num_threads": os.environ.get("OMP_NUM_THREADS"),
            "cpu": cpu_model(), "host_cpus": os.cpu_count(),
            "slab": [s.nx, s.ny, s.nz], "lattice": "D3Q%d" % s.nl, "workload": wl.name}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--workload", required=True)
    ap.add_argument("--nz", type=int, default=SLAB_NZ)
    ap.add_argument("--steps", type=int, default=None)
    ap.add_argument("--budget-s", type=float, default=15.0)
    ap.add_argument("--warmup", type=int, default=2)
    ap.add_argument("--threads", type=int, default=None)
    a = ap.parse_args(argv)
    print(json.dumps(measure(a.workload, a.nz, a.steps, a.budget_s, a.warmup, a.threads)), flush=True)
    assert "torch" not in sys.modules
    return 0


if __name__ == "__main__":
    sys.exit(main())
