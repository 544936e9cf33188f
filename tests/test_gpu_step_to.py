"""Caller-held state buffers.  lbm_step_to: a step written into a caller's
buffer gives bit for bit the state of lbm_step (ghost cells included) although
the caller's buffers start as NaN: the step writes every interior value and
carries the ghost shell over from the buffer it replaces.  The context returns
to its own buffers afterwards.  lbm_state_snapshot / lbm_state_restore: a
context restored from a snapshot exports the same state and steps on bit for
bit like the context the snapshot was taken from."""
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


def exported(s):
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
    ref = exported(a)
    a.step(2)
    ref2 = exported(a)
    a.close()
    b = start(wl, storage)
    L = b.lbm
    keep = []
    for _ in range(6):
        keep.append(L.state_scratch().fill_(float("nan")))
        L.step_to(keep[-1])
    got = exported(b)
    for x, y in zip(got, ref):
        assert np.array_equal(x, y), codes
    # the state copy of the last step is the buffer it was written to
    c = L.state_scratch()
    L.state_copy(c)
    assert torch.equal(c.view(torch.int32), keep[-1].view(torch.int32))   # bytes: padding holds NaN
    b.step(2)                       # back on the context's own buffers
    for x, y in zip(exported(b), ref2):
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


@pytest.mark.parametrize("codes", CASES)
@pytest.mark.parametrize("nl,storage", [(19, "f32"), (27, "f16")])
def test_snapshot_restore_resumes_bit_for_bit(codes, nl, storage):
    ib, jb, kb = codes
    wl = W.Workload("st", 12, 8, 6, nl, steps=6, ibnd=ib, jbnd=jb, kbnd=kb, noise=3e-3, sphere=(6, 4, 3, 2))
    a = start(wl, storage)
    a.step(3)
    snap = a.lbm.snapshot()
    at3 = exported(a)
    a.step(4)
    ref = exported(a)
    a.close()
    b = start(wl, storage)          # another context, another state
    b.step(2)
    b.lbm.restore(snap)
    assert b.lbm.it == 3
    for x, y in zip(exported(b), at3):
        assert np.array_equal(x, y)
    b.step(4)
    for x, y in zip(exported(b), ref):
        assert np.array_equal(x, y)
    # the replay of an adjoint sweep: restore, then steps into caller buffers
    b.lbm.restore(snap)
    keep = []
    for _ in range(4):
        keep.append(b.lbm.state_scratch().fill_(float("nan")))
        b.lbm.step_to(keep[-1])
    for x, y in zip(exported(b), ref):
        assert np.array_equal(x, y)
    b.close()


def test_snapshot_refusals():
    from lbm_b200 import LbmError
    wl = W.Workload("st", 12, 8, 6, 19, steps=2)
    s = start(wl, "f32", blank=False)
    with pytest.raises(LbmError, match="stepped"):
        s.lbm.snapshot()
    s.step(1)
    snap = s.lbm.snapshot()
    o = start(wl.with_(nx=14), "f32", blank=False)
    other = torch.zeros((o.lbm.snapshot_bytes() + 3) // 4, device="cuda")   # o's size, snap's bytes first
    n = min(other.numel(), snap.numel())
    other[:n] = snap[:n]
    with pytest.raises(LbmError, match="parameters"):
        o.lbm.restore(other)
    o.close()
    # same grid, FP16 storage: a snapshot of the FP32 state does not restore there
    h = start(wl, "f16", blank=False)
    other = torch.zeros((h.lbm.snapshot_bytes() + 3) // 4, device="cuda")
    n = min(other.numel(), snap.numel())
    other[:n] = snap[:n]
    with pytest.raises(LbmError, match="parameters"):
        h.lbm.restore(other)
    with pytest.raises(LbmError, match="aligned"):
        s.lbm._call("lbm_state_restore", snap.data_ptr() + 4)
    h.close()
    s.close()
