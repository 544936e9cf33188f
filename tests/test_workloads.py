"""Synthetic workload generators (no GPU)."""
import numpy as np

from lbm_b200 import workloads as W


def test_ensemble_members_follow_the_stated_distribution():
    ms = W.ensemble_members()
    assert len(ms) == 64
    for m in ms:
        assert 96 <= m.nx <= 192 and 48 <= m.ny <= 96 and 48 <= m.nz <= 96
        assert m.nx % 8 == 0 and m.ny % 8 == 0 and m.nz % 8 == 0
        assert 0.03 <= m.uin <= 0.07 and m.nl == 19 and m.lturb and m.city == 0 and m.sphere is None
    assert len({m.seed for m in ms}) == 64                  # own turbulence seed per member
    assert len({(m.nx, m.ny, m.nz) for m in ms}) > 32       # uneven sizes
    assert 40e6 < sum(m.cells for m in ms) < 56e6
    again = W.ensemble_members()
    assert [(m.nx, m.ny, m.nz, m.uin) for m in ms] == [(m.nx, m.ny, m.nz, m.uin) for m in again]


def test_city_mask_boxes_stand_on_the_floor():
    m = W.blanking(W.CITY_Q27_REDUCED)
    assert m.shape == (66, 66, 130)
    assert m[0].sum() == 0 and m[1].sum() > 0                # k ghost empty, boxes start at k = 1
    assert m[41:].sum() == 0                                 # heights at most 40 cells
    assert set(np.unique(m)) <= {0, 1}


def test_probes_and_inflow_perturbation():
    wl = W.ADJOINT_Q19
    pr = W.probe_cells(wl, 200, 0)
    assert pr.shape == (200, 3) and len({tuple(p) for p in pr}) == 200
    m = W.blanking(wl)
    assert all(m[k, j, i] == 0 for i, j, k in pr)
    assert pr.min() >= 1 and (pr[:, 0] <= wl.nx).all() and (pr[:, 2] <= wl.nz).all()
    d = W.inflow_perturbation(wl.nz, 1, 5e-3)
    assert d.shape == (wl.nz,) and abs(np.abs(d).max() - 5e-3) < 1e-9
    assert np.abs(np.diff(d)).max() < 5e-3 * 0.2          # smooth over k
