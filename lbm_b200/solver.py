"""Time-stepping driver over the library, in the order of main.F90.

:class:`Solver` initialises a run exactly as main.F90:243-247 does
(fequil3 -> fillghosts -> fA = fB -> boundarycond(fB,fA) -> boundarycond(fA,fB))
using the library's per-call kernels, then advances it either with the fused
state API (``step``) or by replaying the reference's per-call sequence
(``step_percall``, main.F90:296-329), which is how Fortran host code that
switches call by call would drive it.
"""
from __future__ import annotations

import torch

from .api import Lbm, Params


class Solver:
    def __init__(self, params: Params, rho, u, v, w, uvel, blanking=None, turbulence=None, it0: int = 0,
                 fused: bool = True):
        """rho,u,v,w: CUDA float32 (nz+2,ny+2,nx+2); uvel: (nz,); blanking: int32 mask or None;
        turbulence: (uu, vv, ww, nrturb, ampl) or None.  With float64 arrays (and
        fused=False) the run goes through the FP64 entry points, the reference's
        DP build."""
        dt = rho.dtype
        if fused and dt != torch.float32:
            raise ValueError("the fused state takes float32 arrays (FP32 or FP16-offset storage); "
                             "a float64 run uses the per-call path (fused=False)")
        self.p = params
        self.lbm = Lbm(params)
        L = self.lbm
        self.rho, self.u, self.v, self.w = (t.contiguous().clone() for t in (rho, u, v, w))
        self.uvel = uvel.contiguous().clone()
        self.blanking = blanking
        self.turbulence = turbulence
        self.fused = fused
        fB = L.empty_f(dt)
        L.fequil3(fB, self.rho, self.u, self.v, self.w)
        L.fillghosts(fB)
        fA = fB.clone()
        L.boundarycond(fB, fA, self.uvel)
        L.boundarycond(fA, fB, self.uvel)
        self.tau = torch.full(params.sshape, 3.0 * params.kinevisc + 0.5, dtype=dt, device="cuda")
        self.it = it0
        if fused:
            L.state_import(fA, fB, self.rho, self.u, self.v, self.w, it=it0)
            L.set_inflow(self.uvel)
            if blanking is not None:
                L.set_solids(blanking)
            if turbulence is not None:
                uu, vv, ww, nrturb, ampl = turbulence
                L.set_turbulence(uu, vv, ww, nrturb, ampl)
            self.f1 = self.f2 = None
        else:
            self.f1, self.f2 = fA, fB
            if turbulence is not None:
                self.df = torch.zeros((params.nz, params.ny, params.nl), dtype=dt, device="cuda")

    # ---- fused path ------------------------------------------------------------
    def step(self, n: int = 1):
        if not self.fused:
            return self.step_percall(n)
        self.lbm.step(n)
        self.it += n

    # ---- per-call path (main.F90:296-329) ---------------------------------------------
    def step_percall(self, n: int = 1):
        L = self.lbm
        for _ in range(n):
            self.it += 1
            if self.turbulence is not None:
                uu, vv, ww, nrturb, ampl = self.turbulence
                L.inflow_turbulence_forcing(self.df, self.rho, self.u, self.v, self.w, uu, vv, ww, ampl, self.it,
                                            nrturb)
            L.postcoll(self.f1, self.tau, self.rho, self.u, self.v, self.w)
            if self.turbulence is not None:
                L.inflow_turbulence_apply(self.f1, self.df)
            if self.blanking is not None:
                L.solids(self.f1, self.blanking)
            L.boundarycond(self.f1, self.f2, self.uvel)
            L.drift(self.f2, self.f1)
            self.f1, self.f2 = self.f2, self.f1
            L.macrovars(self.rho, self.u, self.v, self.w, self.f1)

    # ---- results -----------------------------------------------------------------------
    def macro(self):
        """rho, u, v, w as the reference holds them after the last step."""
        if not self.fused:
            return self.rho, self.u, self.v, self.w
        out = [self.lbm.empty_s() for _ in range(4)]
        self.lbm.get_macro(*out)
        return tuple(out)

    def state(self):
        """(f1, f2) in the reference layout."""
        if not self.fused:
            return self.f1, self.f2
        f1, f2 = self.lbm.empty_f(), self.lbm.empty_f()
        self.lbm.state_export(f1, f2)
        return f1, f2

    def close(self):
        self.lbm.close()
