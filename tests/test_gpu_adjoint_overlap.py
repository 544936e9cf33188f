"""The overlapped reverse sweep (segment replay on a second context and stream
while the adjoint steps of the next segment run) gives the gradient of the
serial sweep bit for bit, also when the backward pass is enqueued right behind
a forward pass that has not finished (the replay stream is ordered after the
forward's snapshots)."""
import numpy as np
import pytest

from lbm_b200 import workloads as W

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def test_overlapped_sweep_equals_serial_sweep():
    from lbm_b200 import Params
    from lbm_b200.adjoint import FusedProbeProblem, ProbeProblem, initial_state
    wl = W.Workload("ovl", 64, 32, 24, 19, steps=30, sphere=(20, 16, 12, 5), noise=1e-3)
    p = Params(nx=wl.nx, ny=wl.ny, nz=wl.nz, nl=wl.nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=4,
               kinevisc=wl.kinevisc)
    blank = torch.from_numpy(W.blanking(wl)).cuda()
    probes = W.probe_cells(wl, 40, 3)
    pp = ProbeProblem(p, probes, wl.steps, blanking=blank)
    rho, u, v, w = (torch.from_numpy(x).cuda() for x in W.initial_macro(wl))
    uvel = torch.from_numpy(W.inflow_profile(wl)).cuda()
    f1, f2 = initial_state(pp.lbm, rho, u, v, w, uvel)
    R = pp._macro(f1)
    for _ in range(10):
        f1, f2 = pp._step(f1, f2, R, uvel)
    pp.close()
    fb = FusedProbeProblem(p, probes, wl.steps, blanking=blank, checkpoint=7)
    uh = torch.from_numpy(np.random.default_rng(3).standard_normal((len(probes), 3)).astype(np.float32)).cuda()
    fb.forward(f1, f2, uvel)
    torch.cuda.synchronize()
    g0, u0 = fb.backward(uh, overlap=False)
    fb.forward(f1, f2, uvel)                  # no synchronisation before the overlapped backward
    g1, u1 = fb.backward(uh, overlap=True)
    torch.cuda.synchronize()
    assert torch.equal(g0, g1)
    assert float((u1 - u0).abs().max()) <= 1e-6 * float(u0.abs().max()) + 1e-12   # atomics reorder uvelhat sums
    fb.close()
