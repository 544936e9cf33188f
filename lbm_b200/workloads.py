"""Seeded synthetic inputs for the LBM step (host side, numpy).

No public dataset is involved: every field below is generated from a seed
with the shapes, sizes and value ranges of the reference's runs.

Array layout is the reference's Fortran layout viewed in C order:
scalars ``(nz+2, ny+2, nx+2)`` for ``(0:nx+1, 0:ny+1, 0:nz+1)``, turbulence
fields ``(nrturb+1, nz, ny)`` for ``uu(ny, nz, 0:nrturb)``.
"""
from __future__ import annotations

import dataclasses

import numpy as np


@dataclasses.dataclass(frozen=True)
class Workload:
    name: str
    nx: int
    ny: int
    nz: int
    nl: int = 27
    steps: int = 200
    uin: float = 0.05          # inflow speed, lattice units
    noise: float = 1.0e-3      # amplitude of the uniform velocity noise
    kinevisc: float = 1.0e-4
    smagorinsky: float = 0.15
    sphere: tuple | None = None  # (ic, jc, kc, radius), 1-based reference indices
    city: int = 0              # number of seeded solid boxes
    lturb: bool = False
    ampl: float = 0.0
    nrturb: int = 100
    ibnd: int = 1
    jbnd: int = 0
    kbnd: int = 12
    seed: int = 0

    @property
    def cells(self) -> int:
        return self.nx * self.ny * self.nz

    def with_(self, **kw) -> "Workload":
        return dataclasses.replace(self, **kw)


# Reference configurations (lattice units, ibgk=3, ihrr=1, ivreman=1, Cs=0.15,
# ibnd=1 inflow/outflow, jbnd=0 periodic, kbnd=12 no-slip bottom / free-slip top).
SPHERE_128 = Workload("sphere_q27_128x64x64", 128, 64, 64, 27, steps=200, sphere=(32, 32, 32, 8))
CHANNEL_Q27 = Workload("turb_inflow_q27_512x256x256", 512, 256, 256, 27, steps=1000, lturb=True, ampl=1.0e-4)
CHANNEL_Q19 = CHANNEL_Q27.with_(name="turb_inflow_q19_512x256x256", nl=19)
# the channel at 84 M cells: a state buffer of 2.4 G elements (64-bit offsets)
CHANNEL_Q27_LARGE = CHANNEL_Q27.with_(name="turb_inflow_q27_512x512x320", ny=512, nz=320)
# one eighth of the channel, for profiler captures that must stay small
CHANNEL_Q27_SMALL = CHANNEL_Q27.with_(name="turb_inflow_q27_256x128x128", nx=256, ny=128, nz=128)
CHANNEL_Q19_SMALL = CHANNEL_Q27_SMALL.with_(name="turb_inflow_q19_256x128x128", nl=19)

# FP16-offset storage study: the channel plus a seeded city of 16 solid boxes on
# the bottom wall (heights 10-40 cells), and the same city physics on a grid
# small enough for 1000 steps of the FP64 oracle on the host
CITY_Q27 = CHANNEL_Q27.with_(name="city_q27_512x256x256", city=16)
CITY_Q27_REDUCED = CITY_Q27.with_(name="city_q27_128x64x64", nx=128, ny=64, nz=64)

# Adjoint workload: D3Q19 channel with a sphere of radius 16; the loss is the
# misfit of u at 200 probes after 100 steps, checkpoints every 10 steps
ADJOINT_Q19 = Workload("adjoint_q19_256x128x128", 256, 128, 128, 19, steps=100, sphere=(64, 64, 64, 16))


def probe_cells(wl: "Workload", n: int, seed: int) -> np.ndarray:
    """n seeded interior fluid cells (i, j, k), 1-based, distinct."""
    rng = np.random.default_rng(seed + 4242)
    blank = blanking(wl)
    seen, out = set(), []
    while len(out) < n:
        c = (int(rng.integers(1, wl.nx + 1)), int(rng.integers(1, wl.ny + 1)), int(rng.integers(1, wl.nz + 1)))
        if c in seen or (blank is not None and blank[c[2], c[1], c[0]] != 0):
            continue
        seen.add(c)
        out.append(c)
    return np.array(out, dtype=np.int64)


def inflow_perturbation(nz: int, seed: int, amp: float, dtype=np.float32) -> np.ndarray:
    """Smooth seeded noise over k = 1..nz with maximum |value| = amp: four sine
    modes of decaying amplitude with seeded phases."""
    rng = np.random.default_rng(seed + 777)
    z = np.arange(nz) / max(nz - 1, 1)
    s = sum(rng.standard_normal() * np.sin((q + 1) * np.pi * z + rng.uniform(0, 2 * np.pi)) / (q + 1) for q in range(4))
    return (amp * s / np.abs(s).max()).astype(dtype)


def ensemble_members(n: int = 64, seed: int = 0, nl: int = 19, storage_steps: int = 500) -> list:
    """Members of the batched-ensemble workload: sizes drawn from the seed with
    nx in [96, 192] and ny, nz in [48, 96], each a multiple of 8; each member has
    its own inflow speed, uniform in [0.03, 0.07], and its own inflow-turbulence
    seed (amplitude 1e-4 at i = 10); physics as the sphere case without solids."""
    rng = np.random.default_rng(seed + 31337)
    out = []
    for m in range(n):
        nx = 8 * int(rng.integers(12, 25))
        ny = 8 * int(rng.integers(6, 13))
        nz = 8 * int(rng.integers(6, 13))
        uin = float(rng.uniform(0.03, 0.07))
        out.append(Workload("ensemble_member_%02d" % m, nx, ny, nz, nl, steps=storage_steps, uin=uin, lturb=True,
                            ampl=1.0e-4, seed=1000 * seed + m + 1))
    return out


WORKLOADS = {w.name: w for w in (SPHERE_128, CHANNEL_Q27, CHANNEL_Q19, CHANNEL_Q27_LARGE, CHANNEL_Q27_SMALL,
                                 CHANNEL_Q19_SMALL, CITY_Q27, CITY_Q27_REDUCED, ADJOINT_Q19)}


def initial_macro(wl: Workload, dtype=np.float32):
    """rho, u, v, w with rho = 1 and u = (uin, 0, 0) + U(-noise, noise) per component.

    The ghost shell is zero, as the reference leaves it after inipert
    (m_inipert.F90:121-130 writes only 1..n)."""
    rng = np.random.default_rng(wl.seed)
    shape = (wl.nz + 2, wl.ny + 2, wl.nx + 2)
    rho = np.zeros(shape, dtype)
    u = np.zeros(shape, dtype)
    v = np.zeros(shape, dtype)
    w = np.zeros(shape, dtype)
    inner = (slice(1, wl.nz + 1), slice(1, wl.ny + 1), slice(1, wl.nx + 1))
    n = (wl.nz, wl.ny, wl.nx)
    rho[inner] = 1.0
    u[inner] = (wl.uin + rng.uniform(-wl.noise, wl.noise, n)).astype(dtype)
    v[inner] = rng.uniform(-wl.noise, wl.noise, n).astype(dtype)
    w[inner] = rng.uniform(-wl.noise, wl.noise, n).astype(dtype)
    return rho, u, v, w


def inflow_profile(wl: Workload, dtype=np.float32):
    """uvel(k) = uini * uvel_shear(k) with uvel_shear = 1 (m_inflow.F90:24-41)."""
    return np.full(wl.nz, wl.uin, dtype)


def sphere_mask(nx, ny, nz, ic, jc, kc, r):
    """lblanking of m_sphere.F90:15-21: (i-ic)^2+(j-jc)^2+(k-kc)^2 < r^2, ghosts included."""
    k, j, i = np.meshgrid(np.arange(nz + 2), np.arange(ny + 2), np.arange(nx + 2), indexing="ij")
    return (((i - ic) ** 2 + (j - jc) ** 2 + (k - kc) ** 2) < r * r).astype(np.int32)


def city_mask(nx, ny, nz, nboxes, seed, hmin=10, hmax=40):
    """Seeded block city: nboxes solid boxes standing on k=1, heights U{hmin..hmax}."""
    rng = np.random.default_rng(seed + 7919)
    m = np.zeros((nz + 2, ny + 2, nx + 2), np.int32)
    for _ in range(nboxes):
        sx = int(rng.integers(8, max(9, nx // 16)))
        sy = int(rng.integers(8, max(9, ny // 8)))
        i0 = int(rng.integers(nx // 8, max(nx // 8 + 1, nx - sx - 8)))
        j0 = int(rng.integers(1, max(2, ny - sy)))
        h = int(rng.integers(hmin, hmax + 1))
        m[1:min(h, nz) + 1, j0:j0 + sy, i0:i0 + sx] = 1
    return m


def blanking(wl: Workload):
    if wl.sphere is not None:
        ic, jc, kc, r = wl.sphere
        return sphere_mask(wl.nx, wl.ny, wl.nz, ic, jc, kc, r)
    if wl.city:
        return city_mask(wl.nx, wl.ny, wl.nz, wl.city, wl.seed)
    return None


def turbulence_fields(ny, nz, nrturb, seed, dtype=np.float32, timecor=0.98, cor=10.0 / np.sqrt(3.0)):
    """Smooth pseudo-random inflow fields uu, vv, ww of shape (nrturb+1, nz, ny).

    Each time level is a 2-D Gaussian random field with a Gaussian spectrum of
    decorrelation length ``cor`` cells (the reference uses 10/sqrt(3),
    m_inflow_turbulence_compute.F90:19-20); levels are chained by the AR(1)
    relation x_t = 0.98 x_{t-1} + sqrt(1-0.98^2) e_t and each level is then
    normalised to zero mean and unit standard deviation (:35-60).  The spectral
    synthesis here is this project's own; the reference's FFTW-based
    generator (m_pseudo2D.F90) is outside the timed path."""
    rng = np.random.default_rng(seed + 104729)
    ky = np.fft.fftfreq(ny)[None, :]
    kz = np.fft.fftfreq(nz)[:, None]
    spec = np.exp(-((2 * np.pi * cor) ** 2) * (ky ** 2 + kz ** 2) / 4.0)

    def field():
        e = rng.standard_normal((nz, ny)) + 1j * rng.standard_normal((nz, ny))
        x = np.real(np.fft.ifft2(e * spec))
        return (x - x.mean()) / (x.std() + 1e-30)

    out = []
    for _ in range(3):
        a = np.zeros((nrturb + 1, nz, ny))
        a[0] = field()
        for t in range(1, nrturb + 1):
            a[t] = timecor * a[t - 1] + np.sqrt(1.0 - timecor ** 2) * field()
            a[t] = a[t] - a[t].mean()
            a[t] = a[t] / np.sqrt((a[t] ** 2).sum() / (ny * nz - 1))
        out.append(a.astype(dtype))
    return tuple(out)
