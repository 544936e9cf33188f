"""lbm_step_to: a step written into a caller's buffer gives bit for bit the
state of lbm_step (ghost cells included) although the caller's buffers start
as NaN: the step writes every interior value and carries the ghost shell over
from the buffer it replaces.  The context returns to its own buffers
afterwards."""
import numpy as np
import pytest

from lbm_b200 import workloads as W
from tests.test_gpu_fused import cuda, host, params_of

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


def start(wl, storage, blank=True):
    from lbm_b200 import Solver
    rho, u, v, w = (cuda(a) for a in W.initial_macro(wl))
    uvel = cuda(W.inflow_profile(wl))
    bl = cuda(W.blanking(wl)) if blank and wl.sphere else None
    return Solver(params_of(wl, iturb_pos=3, storage=storage), rho, u, v, w, uvel, blanking=bl, fused=True)


def snapshot(s):
    f1, f2 = s.state()
    return [host(t) for t in (f1, f2, *s.macro())]


CASES = [(1, 0, 12), (11, 22, 12), (0, 0, 0), (1, 11, 22), (0, 12, 0)]


@pytest.mark.parametrize("codes", CASES)
@pytest.mark.parametrize("nl,storage", [(19, "f32"), (27, "f32"), (27, "f16")])
def test_step_to_equals_step(codes, nl, storage):
    ib, jb, kb = codes
    wl = W.Workload("st", 12, 8, 6, nl, steps=6, ibnd=ib, jbnd=jb, kbnd=kb, noise=3e-3, sphere=(6, 4, 3, 2))
    a = start(wl, storage)
    a.step(6)
    ref = snapshot(a)
    a.step(2)
    ref2 = snapshot(a)
    a.close()
    b = start(wl, storage)
    L = b.lbm
    keep = []
    for _ in range(6):
        keep.append(L.state_scratch().fill_(float("nan")))
        L.step_to(keep[-1])
    got = snapshot(b)
    for x, y in zip(got, ref):
        assert np.array_equal(x, y), codes
    # the state copy of the last step is the buffer it was written to
    c = L.state_scratch()
    L.state_copy(c)
    assert torch.equal(c.view(torch.int32), keep[-1].view(torch.int32))   # bytes: padding holds NaN
    b.step(2)                       # back on the context's own buffers
    for x, y in zip(snapshot(b), ref2):
        assert np.array_equal(x, y)
    b.close()


def test_step_to_refuses_bad_buffers():
    from lbm_b200 import LbmError
    wl = W.Workload("st", 12, 8, 6, 19, steps=2)
    s = start(wl, "f32", blank=False)
    L = s.lbm
    d = L.state_scratch()
    with pytest.raises(LbmError, match="aligned"):
        L._call("lbm_step_to", d.data_ptr() + 4)
    s.close()
