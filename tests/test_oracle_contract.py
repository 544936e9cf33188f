"""The oracle built with FMA contraction (-ffp-contract=fast) against the
separately rounded build: the same arithmetic up to FP32 rounding, on a small
case with solids and both lattices.  Contraction moves FP32 results by less
than their distance to FP64, and FP64 results by rounding only."""
import numpy as np
import pytest

from lbm_b200 import workloads as W
from oracle import oracle as O
from tests.conftest import rel_l2


def run(wl, dtype, contract):
    cfg = O.Config(wl.nx, wl.ny, wl.nz, wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=3, lsolids=True,
                   kinevisc=wl.kinevisc, smagorinsky=wl.smagorinsky)
    o = O.Oracle(cfg, dtype, contract=contract)
    rho, u, v, w = (a.astype(dtype) for a in W.initial_macro(wl))
    uvel = W.inflow_profile(wl, dtype)
    fA, fB = o.zeros_f(), o.zeros_f()
    o.init(fA, fB, rho, u, v, w, uvel)
    tau = np.full(cfg.sshape, 3.0 * np.float32(wl.kinevisc) + 0.5, dtype)
    o.run(fA, fB, rho, u, v, w, tau, uvel, wl.steps, blanking=W.blanking(wl))
    return fA, u


@pytest.mark.parametrize("nl", [19, 27])
def test_contracted_oracle_stays_within_the_fp32_floor(nl):
    wl = W.Workload("contract", 20, 12, 10, nl, steps=40, sphere=(8, 6, 5, 3), noise=2e-3)
    f64, u64 = run(wl, np.float64, False)
    f32, u32 = run(wl, np.float32, False)
    f32c, u32c = run(wl, np.float32, True)
    f64c, _ = run(wl, np.float64, True)
    floor = rel_l2(f32, f64)
    shift = rel_l2(f32c, f32)
    assert 0.0 < shift <= floor                       # contraction changes FP32 rounding, not more
    assert rel_l2(f32c, f64) <= 2.0 * floor
    assert rel_l2(f64c, f64) < 1e-12                  # FP64: rounding only
