"""Set-up of a batched ensemble: every member initialised as main.F90:243-262
does (fequil3 -> fillghosts -> fA = fB -> boundarycond twice), then imported
into its own context of one :class:`~lbm_b200.api.Ensemble`."""
from __future__ import annotations

import torch

from .api import Ensemble, Params
from . import workloads as W


def params_of(wl: W.Workload, storage: str = "f32", iturb_pos: int = 10) -> Params:
    return Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd,
                  kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky, iturb_pos=min(iturb_pos, wl.nx), storage=storage)


def init_member(lbm, wl: W.Workload):
    """Initial state of one member in its context (the members' device arrays are
    released after the import)."""
    rho, u, v, w = (torch.from_numpy(x).cuda() for x in W.initial_macro(wl))
    uvel = torch.from_numpy(W.inflow_profile(wl)).cuda()
    fB = lbm.empty_f()
    lbm.fequil3(fB, rho, u, v, w)
    lbm.fillghosts(fB)
    fA = fB.clone()
    lbm.boundarycond(fB, fA, uvel)
    lbm.boundarycond(fA, fB, uvel)
    lbm.state_import(fA, fB, rho, u, v, w)
    lbm.set_inflow(uvel)
    if wl.lturb:
        uu, vv, ww = (torch.from_numpy(x).cuda() for x in W.turbulence_fields(wl.ny, wl.nz, wl.nrturb, wl.seed))
        lbm.set_turbulence(uu, vv, ww, wl.nrturb, wl.ampl)
    blank = W.blanking(wl)
    if blank is not None:
        lbm.set_solids(torch.from_numpy(blank).cuda())


def build_ensemble(members: list, storage: str = "f32") -> Ensemble:
    ens = Ensemble([params_of(wl, storage) for wl in members])
    for lbm, wl in zip(ens.members, members):
        init_member(lbm, wl)
    torch.cuda.synchronize()
    return ens
