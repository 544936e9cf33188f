"""The committed fixtures come from the committed generator: rerunning
tests/golden/make_golden.py reproduces every array of golden_small.npz (to FP64
round-off, so a different BLAS or CPU does not matter) and no array is added or
missing."""
import importlib.util
import os

import numpy as np

HERE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def test_generator_reproduces_the_fixtures(tmp_path):
    spec = importlib.util.spec_from_file_location("make_golden", os.path.join(HERE, "make_golden.py"))
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    gen.OUT = str(tmp_path / "golden_small.npz")
    gen.main()
    new = np.load(gen.OUT)
    old = np.load(os.path.join(HERE, "golden_small.npz"))
    assert sorted(new.files) == sorted(old.files)
    for k in old.files:
        a, b = new[k], old[k]
        assert a.shape == b.shape and a.dtype == b.dtype, k
        if np.issubdtype(b.dtype, np.floating):
            np.testing.assert_allclose(a, b, rtol=1e-13, atol=1e-15, err_msg=k)
        else:
            np.testing.assert_array_equal(a, b, err_msg=k)
