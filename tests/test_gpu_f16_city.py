"""FP16-offset storage on the city workload at its own size (512x256x256 D3Q27,
16 seeded solid boxes, inflow turbulence at i = 10), 100 of its 1000 steps:
rho and the velocity field within a relative L2 of 1e-3 of the same run in FP64
through the DP build's per-call entry points, and of plain FP32.  The bench's
default run states the errors after all 1000 steps (f16_storage)."""
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

STEPS = 100
BOUND = 1e-3


def test_city_fp16_error_against_fp64_and_fp32():
    import bench
    from lbm_b200 import workloads as W
    wl = W.CITY_Q27
    assert (wl.nx, wl.ny, wl.nz, wl.city, wl.lturb) == (512, 256, 256, 16, True)
    f16, s16 = bench.gpu_run_macro(wl, "f16", STEPS)
    f32, s32 = bench.gpu_run_macro(wl, "f32", STEPS)
    torch.cuda.empty_cache()
    f64, s64 = bench.dp_run_macro(wl, STEPS)
    torch.cuda.empty_cache()
    assert (s16, s32, s64) == (0, 0, 0)
    e16, e32, e1632 = bench.rel_l2_pair(f16, f64), bench.rel_l2_pair(f32, f64), bench.rel_l2_pair(f16, f32)
    print("FP16 vs FP64", e16, "FP32 vs FP64", e32, "FP16 vs FP32", e1632)
    assert e16["rho"] <= BOUND and e16["u"] <= BOUND, e16
    assert e1632["rho"] <= BOUND and e1632["u"] <= BOUND, e1632
    # plain FP32 sits far closer to FP64 than the bound
    assert e32["u"] <= 1e-4 and e32["rho"] <= 1e-5, e32
