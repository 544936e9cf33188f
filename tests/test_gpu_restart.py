"""Save a fused state to a reference restart file, resume from it, and compare
the resumed run with the oracle resuming from the same file."""
import numpy as np
import pytest

from lbm_b200 import workloads as W
from oracle import oracle as O
from tests.test_gpu_fused import SMALL, compare_to_floor, cuda, host, params_of

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nl", [19, 27])
def test_resume_matches_the_oracle(nl, tmp_path):
    from lbm_b200 import Lbm, Solver
    from lbm_b200 import restart as R
    wl = SMALL.with_(nl=nl, lturb=False)
    blank = W.blanking(wl)
    rho, u, v, w = (cuda(a) for a in W.initial_macro(wl))
    uvel = cuda(W.inflow_profile(wl))
    s = Solver(params_of(wl, iturb_pos=5), rho, u, v, w, uvel, blanking=cuda(blank))
    s.step(10)
    path = R.restart_name(10, directory=str(tmp_path / "restart"))
    R.save_state(s.lbm, path)
    f_saved = host(s.state()[0])
    s.close()
    *_, f_file = R.read_restart(path, expect=(wl.nx, wl.ny, wl.nz, nl))
    assert np.array_equal(f_file, f_saved)
    # resume in a fresh context
    L = Lbm(params_of(wl, iturb_pos=5))
    R.load_state(L, path, it=10)
    L.set_inflow(uvel)
    L.set_solids(cuda(blank))
    L.step(6)
    g1, g2 = L.empty_f(), L.empty_f()
    L.state_export(g1, g2)
    gm = [L.empty_s() for _ in range(4)]
    L.get_macro(*gm)
    gpu = (host(g1), host(g2), *[host(t) for t in gm])
    assert L.it == 16
    L.close()

    def oracle(dtype):
        cfg = O.Config(wl.nx, wl.ny, wl.nz, nl, ibnd=wl.ibnd, jbnd=wl.jbnd, kbnd=wl.kbnd, iturb_pos=5,
                       lsolids=True, kinevisc=wl.kinevisc)
        o = O.Oracle(cfg, dtype)
        fA = f_file.astype(dtype)
        Rm = [np.zeros(cfg.sshape, dtype) for _ in range(4)]
        o.macrovars(*Rm, fA)                       # main.F90:256-258
        fB = fA.copy()
        tau = np.full(cfg.sshape, 3 * wl.kinevisc + 0.5, dtype)
        o.run(fA, fB, *Rm, tau, W.inflow_profile(wl, dtype), 6, it0=10, blanking=blank)
        return (fA, fB, *Rm)
    compare_to_floor(gpu, oracle(np.float32), oracle(np.float64), "resume")
