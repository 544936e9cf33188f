"""Batched ensemble: every member computes exactly what it computes alone."""
import numpy as np
import pytest

from lbm_b200 import workloads as W

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# uneven members: different sizes (rows shorter and longer than a block), inflow speeds and turbulence seeds
MEMBERS = [W.Workload("m0", 16, 8, 6, 19, uin=0.04, lturb=True, ampl=1e-3, nrturb=5, seed=11, noise=2e-3),
           W.Workload("m1", 40, 12, 10, 19, uin=0.06, lturb=True, ampl=1e-3, nrturb=7, seed=12, noise=2e-3),
           W.Workload("m2", 10, 8, 8, 19, uin=0.03, lturb=True, ampl=1e-3, nrturb=3, seed=13, noise=2e-3),
           W.Workload("m3", 300, 9, 7, 19, uin=0.05, lturb=True, ampl=1e-3, nrturb=4, seed=14, noise=2e-3)]


def alone(wl, steps, storage="f32"):
    from lbm_b200 import Lbm
    from lbm_b200.ensemble import init_member, params_of
    L = Lbm(params_of(wl, storage))
    init_member(L, wl)
    L.step(steps)
    f1, f2 = L.empty_f(), L.empty_f()
    L.state_export(f1, f2)
    torch.cuda.synchronize()
    out = (f1.cpu().numpy(), f2.cpu().numpy())
    L.close()
    return out


def exported(ens):
    out = []
    for L in ens.members:
        f1, f2 = L.empty_f(), L.empty_f()
        L.state_export(f1, f2)
        torch.cuda.synchronize()
        out.append((f1.cpu().numpy(), f2.cpu().numpy()))
    return out


@pytest.mark.parametrize("storage", ["f32", "f16"])
@pytest.mark.parametrize("graph", [0, 4])
def test_members_match_single_runs(storage, graph):
    from lbm_b200.ensemble import build_ensemble
    steps = 13                      # first step alone, then graphs of 4 and single steps
    ens = build_ensemble(MEMBERS, storage)
    ens.set_graph(graph)
    ens.step(steps)
    got = exported(ens)
    for m, wl in enumerate(MEMBERS):
        ref = alone(wl, steps, storage)
        for a, b in zip(got[m], ref):
            assert np.array_equal(a, b), (m, float(np.abs(a - b).max()))
        assert ens.members[m].it == steps
        assert ens.members[m].status() == 0
    ens.close()


def test_every_launch_shape_and_autotune():
    from lbm_b200 import Ensemble, _lib
    from lbm_b200.ensemble import build_ensemble
    V, G = _lib.LBM_ENS_VARIANTS, _lib.LBM_ENS_GRAPH_STEPS
    shapes = [Ensemble.variant_shape(v) for v in range(V)]
    assert len(set(shapes)) == V and all(t in (64, 128, 256) and m >= 1 and r >= 1 for t, m, r in shapes)
    ref = [alone(wl, 9) for wl in MEMBERS]
    for v in range(V):
        ens = build_ensemble(MEMBERS)
        ens.set_variant(v)
        ens.step(9)
        for m, got in enumerate(exported(ens)):
            assert all(np.array_equal(a, b) for a, b in zip(got, ref[m])), (v, m)
        ens.close()
    ens = build_ensemble(MEMBERS)
    v, ms = ens.autotune(2)
    assert 0 <= v < V and all(t > 0 for t in ms) and ms[v] == min(ms)
    cv, cg = ens.config()
    assert cv == v and cg in (0, G)
    ens.step(4)
    # the first step (collides in place: the buffer parity stays), V x (warm-up + 2), one step
    # back to parity 0 where needed, graph capture + 2 timed graphs' worth, then 4
    n = V * 3
    assert all(L.it == 1 + n + n % 2 + 3 * G + 4 for L in ens.members)
    ens.close()
    ref = [alone(wl, 8) for wl in MEMBERS]
    ens = build_ensemble(MEMBERS)
    ens.set_graph(4)      # graph replay: same results as direct launches
    ens.step(8)
    for m, got in enumerate(exported(ens)):
        assert all(np.array_equal(a, b) for a, b in zip(got, ref[m])), m
    ens.close()


def test_rejects_unsupported_members():
    from lbm_b200 import Ensemble, LbmError, Params
    with pytest.raises(LbmError, match="same lattice"):
        Ensemble([Params(nx=8, ny=8, nz=8, nl=19, iturb_pos=3), Params(nx=8, ny=8, nz=8, nl=27, iturb_pos=3)])
    with pytest.raises(LbmError, match="periodic j"):
        Ensemble([Params(nx=8, ny=8, nz=8, nl=19, jbnd=11, iturb_pos=3)])
    with pytest.raises(LbmError, match="even nx"):
        Ensemble([Params(nx=9, ny=8, nz=8, nl=19, iturb_pos=3)])
    with pytest.raises(LbmError, match="lbm_create failed"):
        Ensemble([Params(nx=8, ny=8, nz=8, nl=19, iturb_pos=30)])
    ens = Ensemble([Params(nx=8, ny=8, nz=8, nl=19, iturb_pos=3)])
    with pytest.raises(LbmError, match="no state imported"):
        ens.step(1)
    ens.close()


def test_member_stepped_alone_is_caught():
    from lbm_b200.ensemble import build_ensemble
    ens = build_ensemble(MEMBERS[:2])
    ens.step(2)
    ens.members[1].step(1)           # out of phase with member 0
    from lbm_b200 import LbmError
    with pytest.raises(LbmError, match="same step phase"):
        ens.step(1)
    ens.members[0].step(1)           # back in phase
    ens.step(1)
    ens.close()


def test_fp16_d3q27_block_shapes_match_the_ensemble():
    """FP16 D3Q27 runs its single-domain step in blocks of 256 threads where a
    row's pairs fill them (nx = 512 here) and of 128 otherwise (nx = 200); the
    ensemble kernel, with its own launch shapes, must give the same bits."""
    from lbm_b200.ensemble import build_ensemble
    members = [W.Workload("w512", 512, 6, 5, 27, uin=0.05, lturb=True, ampl=1e-3, nrturb=3, seed=21, noise=2e-3),
               W.Workload("w200", 200, 7, 6, 27, uin=0.04, lturb=True, ampl=1e-3, nrturb=4, seed=22, noise=2e-3)]
    steps = 9
    ref = [alone(wl, steps, "f16") for wl in members]
    ens = build_ensemble(members, "f16")
    ens.step(steps)
    for m, got in enumerate(exported(ens)):
        for a, b in zip(got, ref[m]):
            assert np.array_equal(a, b), (members[m].name, float(np.abs(a - b).max()))
    ens.close()
