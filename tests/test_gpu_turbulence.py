"""GPU inflow-turbulence generator against an independent numpy restatement with
the same counter-based phases, and its statistics."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)


def splitmix64(x):
    with np.errstate(over="ignore"):
        z = (x + np.uint64(0x9E3779B97F4A7C15)) & M64
        z = ((z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)) & M64
        z = ((z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)) & M64
        return z ^ (z >> np.uint64(31))


def reference_fields(ny, nz, nrturb, nf, seed):
    """numpy restatement: spectrum, Hermitian l = 0 and n1/2 columns, inverse real FFT, AR(1) + normalisation."""
    n1, n2 = ny + ny % 2, nz + nz % 2
    h = n1 // 2 + 1
    rx = 10.0 / np.sqrt(3.0)
    deltak = (2 * np.pi) ** 2 / (n1 * n2)
    k2, l2 = (2 * np.pi / n1) ** 2, (2 * np.pi / n2) ** 2
    r = np.sqrt(8.0) / rx
    ll, pp = np.meshgrid(np.arange(-n1 // 2 + 1, n1 // 2 + 1), np.arange(-n2 // 2 + 1, n2 // 2 + 1))
    summ = np.exp(-2.0 * (k2 * ll ** 2 / r ** 2 + l2 * pp ** 2 / r ** 2)).sum() - 1.0
    amp = np.float32(np.sqrt(deltak) * np.sqrt(1.0 / (deltak * summ)))
    ak, al = np.float32(k2 / r ** 2), np.float32(l2 / r ** 2)
    out = []
    for f in range(nf):
        lev = np.zeros((nrturb + 1, nz, ny), np.float64)
        for t in range(nrturb + 1):
            b = f * (nrturb + 1) + t
            X = np.zeros((n2, h), np.complex128)
            for pi in range(n2):
                p0 = pi if pi < n2 // 2 else pi - n2
                for l in range(h):
                    p, sgn, real_only = p0, 1.0, False
                    if l == 0 or l == n1 // 2:
                        if p < 0 and p != -n2 // 2:
                            p, sgn = -p, -1.0
                        real_only = p == 0 or p == -n2 // 2
                    ctr = np.uint64(((b * (n2 + 1) + (p + n2 // 2)) * h + l))
                    u = np.float32(int(splitmix64(np.uint64(seed) ^ splitmix64(ctr)) >> np.uint64(40)) / 16777216.0)
                    phi = np.float32(6.283185307179586) * u
                    ee = amp * np.exp(-(ak * np.float32(l * l) + al * np.float32(p * p)), dtype=np.float32)
                    re, im = ee * np.cos(phi), sgn * ee * np.sin(phi)
                    if real_only:
                        im = 0.0
                    if l == 0 and p == 0:
                        re = 0.0
                    X[pi, l] = re + 1j * im
            y = np.fft.irfft2(X, s=(n2, n1)) * (n1 * n2)
            v = y[:nz, :ny]
            if t > 0:
                v = 0.98 * lev[t - 1] + np.sqrt(1 - 0.98 ** 2) * v
                v = v - v.mean()
                v = v / np.sqrt((v ** 2).sum() / (ny * nz - 1))
            lev[t] = v
        out.append(lev)
    return out


@pytest.mark.parametrize("ny,nz", [(12, 10), (9, 7)])
def test_matches_numpy_restatement(ny, nz):
    from lbm_b200 import Lbm, Params
    nrturb, seed = 4, 1234
    L = Lbm(Params(nx=8, ny=ny, nz=nz, nl=19, iturb_pos=3))
    f = [torch.zeros(nrturb + 1, nz, ny, device="cuda") for _ in range(4)]
    L.inflow_turbulence_compute(f[0], f[1], f[2], nrturb, seed, rr=f[3])
    ref = reference_fields(ny, nz, nrturb, 4, seed)
    for a, b in zip(f, ref):
        a = a.cpu().numpy().astype(np.float64)
        assert np.abs(a - b).max() < 2e-5 * max(1.0, np.abs(b).max()), np.abs(a - b).max()


def test_statistics_of_a_large_plane():
    from lbm_b200 import Lbm, Params
    ny, nz, nrturb = 128, 96, 40
    L = Lbm(Params(nx=8, ny=ny, nz=nz, nl=19, iturb_pos=3))
    f = [torch.zeros(nrturb + 1, nz, ny, device="cuda") for _ in range(3)]
    L.inflow_turbulence_compute(*f, nrturb, seed=7)
    for a in f:
        a = a.double()
        m = a[1:].mean(dim=(1, 2))
        s = a[1:].std(dim=(1, 2))
        assert m.abs().max() < 1e-5 and (s - 1).abs().max() < 1e-5
        corr = [float((a[t] * a[t - 1]).mean()) for t in range(2, nrturb + 1)]
        assert min(corr) > 0.9                                     # AR(1) with 0.98
        # smooth in space: neighbouring cells strongly correlated, distant ones not
        x = a[nrturb]
        assert float((x[:, 1:] * x[:, :-1]).mean()) > 0.8
        assert abs(float((x[:, 40:] * x[:, :-40]).mean())) < 0.3
    # different seeds give different fields, the same seed the same
    g = [torch.zeros(nrturb + 1, nz, ny, device="cuda") for _ in range(3)]
    L.inflow_turbulence_compute(*g, nrturb, seed=7)
    assert torch.equal(f[0], g[0])
    L.inflow_turbulence_compute(*g, nrturb, seed=8)
    assert not torch.equal(f[0], g[0])
