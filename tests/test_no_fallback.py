"""Without a CUDA device the product path stops with an error: there is no CPU
or pure-PyTorch fallback for any entry point (these run only where no GPU is
visible)."""
import os
import subprocess
import sys

import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.skipif(torch.cuda.is_available(), reason="checks the behaviour without a CUDA device")

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_contexts_refuse_to_start_without_a_device():
    from lbm_b200 import Ensemble, Lbm, Params
    p = Params(nx=8, ny=4, nz=4, nl=19)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        Lbm(p)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        Ensemble([p])


def test_bench_our_arm_fails_without_a_device():
    r = subprocess.run([sys.executable, "bench.py", "--steps", "1", "--warmup", "0", "--no-cpu-baseline",
                        "--no-e2e", "--no-f16"], cwd=ROOT, capture_output=True, text=True, timeout=600)
    assert r.returncode != 0
    assert not any(ln.startswith("{") for ln in r.stdout.splitlines())


def test_library_load_fails_loudly_when_missing(tmp_path, monkeypatch):
    from lbm_b200 import _lib
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "liblbmb200.so"))
    monkeypatch.setattr(_lib, "_lib", None)
    with pytest.raises(RuntimeError, match="no CPU fallback"):
        _lib.load()
