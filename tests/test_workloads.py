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
