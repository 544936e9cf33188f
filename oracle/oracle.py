"""ctypes wrapper of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU legs of ``bench.py``
(the CPU baseline and the reference arm, ``--impl reference``) may import this
module; it is the checker, never the product.

Array conventions follow the reference's Fortran layout viewed from numpy in
C order:

* distributions ``f(nl,0:nx+1,0:ny+1,0:nz+1)``  -> ``ndarray[nz+2, ny+2, nx+2, nl]``
* scalars ``rho(0:nx+1,0:ny+1,0:nz+1)``         -> ``ndarray[nz+2, ny+2, nx+2]``
* ``uvel(nz)``, ``ablvisc(nz)``                 -> ``ndarray[nz]``
* ``uu(ny,nz,0:nrturb)``                         -> ``ndarray[nrturb+1, nz, ny]``
* ``turbulence_df(nl,ny,nz)``                    -> ``ndarray[nz, ny, nl]``
* ``lblanking`` logical(4)                       -> ``int32 ndarray[nz+2, ny+2, nx+2]``
"""
from __future__ import annotations

import ctypes
import dataclasses

import numpy as np

from . import build as _build


class OrcParams(ctypes.Structure):
    _fields_ = [
        ("nx", ctypes.c_int32), ("ny", ctypes.c_int32), ("nz", ctypes.c_int32),
        ("nl", ctypes.c_int32), ("ibgk", ctypes.c_int32), ("ihrr", ctypes.c_int32),
        ("ivreman", ctypes.c_int32), ("ibnd", ctypes.c_int32), ("jbnd", ctypes.c_int32),
        ("kbnd", ctypes.c_int32), ("iturb_pos", ctypes.c_int32), ("lsolids", ctypes.c_int32),
        ("lturb", ctypes.c_int32), ("nrturb", ctypes.c_int32),
        ("kinevisc", ctypes.c_double), ("smagorinsky", ctypes.c_double), ("rho0", ctypes.c_double),
        ("udir", ctypes.c_double), ("ampl", ctypes.c_double),
    ]


@dataclasses.dataclass
class Config:
    """Run-time options of the reference (m_readinfile.F90) as plain fields."""
    nx: int
    ny: int
    nz: int
    nl: int = 27
    ibgk: int = 3
    ihrr: int = 1
    ivreman: int = 1
    ibnd: int = 1
    jbnd: int = 0
    kbnd: int = 12
    iturb_pos: int = 10
    lsolids: bool = False
    lturb: bool = False
    nrturb: int = 100
    kinevisc: float = 1.0e-4
    smagorinsky: float = 0.15
    rho0: float = 1.0
    udir: float = 0.0
    ampl: float = 0.0

    def c(self) -> OrcParams:
        return OrcParams(self.nx, self.ny, self.nz, self.nl, self.ibgk, self.ihrr, self.ivreman,
                         self.ibnd, self.jbnd, self.kbnd, self.iturb_pos, int(self.lsolids),
                         int(self.lturb), self.nrturb, self.kinevisc, self.smagorinsky, self.rho0,
                         self.udir, self.ampl)

    # shapes
    @property
    def fshape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2, self.nl)

    @property
    def sshape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2)


_libs = {}
_threads = None


def lib(contract: bool = False):
    """The oracle library: separately rounded (default, as the reference's CPU
    build) or FMA-contracted (contract=True)."""
    if contract not in _libs:
        path = _build.build(contract=contract)
        L = ctypes.CDLL(path)
        L.orc_set_threads.argtypes = [ctypes.c_int]
        if _threads is not None:
            L.orc_set_threads(_threads)
        _libs[contract] = L
    return _libs[contract]


def set_threads(n: int) -> None:
    global _threads
    _threads = int(n)
    lib()
    for L in _libs.values():
        L.orc_set_threads(_threads)


def _ptr(a):
    if a is None:
        return None
    assert a.flags["C_CONTIGUOUS"], "oracle arrays must be C-contiguous"
    return a.ctypes.data_as(ctypes.c_void_p)


class Oracle:
    """Typed front end; ``dtype`` selects the FP32 or FP64 instantiation,
    ``contract`` the FMA-contracted build of the same source."""

    def __init__(self, cfg: Config, dtype=np.float32, contract: bool = False):
        self.cfg = cfg
        self.dtype = np.dtype(dtype)
        self.sfx = "f32" if self.dtype == np.float32 else "f64"
        self._p = cfg.c()
        self._pp = ctypes.byref(self._p)
        self.L = lib(contract)

    def _fn(self, name):
        fn = getattr(self.L, "orc_%s_%s" % (name, self.sfx))
        fn.restype = None
        return fn

    def _chk(self, *arrs):
        for a in arrs:
            if a is not None and a.dtype != self.dtype and a.dtype != np.int32:
                raise TypeError("oracle dtype mismatch: %s vs %s" % (a.dtype, self.dtype))

    # ---- allocation helpers -------------------------------------------------
    def zeros_f(self):
        return np.zeros(self.cfg.fshape, self.dtype)

    def zeros_s(self):
        return np.zeros(self.cfg.sshape, self.dtype)

    # ---- routines (reference subroutine names) ------------------------------
    def fequil3(self, feq, rho, u, v, w):
        self._chk(feq, rho, u, v, w)
        self._fn("fequil3")(self._pp, _ptr(feq), _ptr(rho), _ptr(u), _ptr(v), _ptr(w))

    def postcoll(self, f, tau, rho, u, v, w, ablvisc=None):
        if ablvisc is None:
            ablvisc = np.zeros(self.cfg.nz, self.dtype)
        self._chk(f, tau, rho, u, v, w, ablvisc)
        self._fn("postcoll")(self._pp, _ptr(f), _ptr(tau), _ptr(rho), _ptr(u), _ptr(v), _ptr(w), _ptr(ablvisc))

    def drift(self, f, feq):
        self._chk(f, feq)
        self._fn("drift")(self._pp, _ptr(f), _ptr(feq))

    def macrovars(self, rho, u, v, w, f):
        self._chk(rho, u, v, w, f)
        self._fn("macrovars")(self._pp, _ptr(rho), _ptr(u), _ptr(v), _ptr(w), _ptr(f))

    def regularization(self, f, feq, u, v, w):
        self._chk(f, feq, u, v, w)
        self._fn("regularization")(self._pp, _ptr(f), _ptr(feq), _ptr(u), _ptr(v), _ptr(w))

    def vreman(self, f, tau):
        self._chk(f, tau)
        self._fn("vreman")(self._pp, _ptr(f), _ptr(tau))

    def compute_fneq(self, f, feq):
        self._chk(f, feq)
        self._fn("compute_fneq")(self._pp, _ptr(f), _ptr(feq))

    def compute_f(self, f, feq):
        self._chk(f, feq)
        self._fn("compute_f")(self._pp, _ptr(f), _ptr(feq))

    def boundarycond(self, f1, f2, uvel):
        self._chk(f1, f2, uvel)
        self._fn("boundarycond")(self._pp, _ptr(f1), _ptr(f2), _ptr(uvel))

    def solids(self, f, blanking):
        assert blanking.dtype == np.int32
        self._chk(f)
        self._fn("solids")(self._pp, _ptr(f), _ptr(blanking))

    def turbulence_forcing(self, df, rho, u, v, w, uu, vv, ww, it):
        self._chk(df, rho, u, v, w, uu, vv, ww)
        self._fn("turbulence_forcing")(self._pp, _ptr(df), _ptr(rho), _ptr(u), _ptr(v), _ptr(w),
                                       _ptr(uu), _ptr(vv), _ptr(ww), ctypes.c_int(it))

    def turbulence_apply(self, f, df):
        self._chk(f, df)
        self._fn("turbulence_apply")(self._pp, _ptr(f), _ptr(df))

    def fillghosts(self, f):
        self._chk(f)
        self._fn("fillghosts")(self._pp, _ptr(f))

    def init(self, fA, fB, rho, u, v, w, uvel):
        self._chk(fA, fB, rho, u, v, w, uvel)
        self._fn("init")(self._pp, _ptr(fA), _ptr(fB), _ptr(rho), _ptr(u), _ptr(v), _ptr(w), _ptr(uvel))

    def forcings_apply(self, f, force, rho, u, v, w):
        """force: (nz+2, ny+2, nx+2, 3), the reference's external_forcing(3,0:nx+1,0:ny+1,0:nz+1)."""
        self._chk(f, force, rho, u, v, w)
        self._fn("forcings_apply")(self._pp, _ptr(f), _ptr(force), _ptr(rho), _ptr(u), _ptr(v), _ptr(w))

    def run(self, fA, fB, rho, u, v, w, tau, uvel, nsteps, it0=0, blanking=None, uu=None, vv=None, ww=None,
            ablvisc=None, force=None):
        """Time loop of main.F90:283-329; on return fA is f1 and fB is f2.  force: a fixed
        external_forcing applied every step (main.F90:306), or None."""
        if ablvisc is None:
            ablvisc = np.zeros(self.cfg.nz, self.dtype)
        if self.cfg.lsolids and blanking is None:
            raise ValueError("lsolids needs a blanking mask")
        if self.cfg.lturb and uu is None:
            raise ValueError("lturb needs uu, vv, ww")
        self._chk(fA, fB, rho, u, v, w, tau, uvel, ablvisc, uu, vv, ww, force)
        args = [self._pp, _ptr(fA), _ptr(fB), _ptr(rho), _ptr(u), _ptr(v), _ptr(w), _ptr(tau), _ptr(ablvisc),
                _ptr(blanking), _ptr(uvel), _ptr(uu), _ptr(vv), _ptr(ww), ctypes.c_int(it0), ctypes.c_int(nsteps)]
        if force is None:
            self._fn("run")(*args)
        else:
            self._fn("run_forced")(*args, _ptr(force))


def tables(nl: int, dtype=np.float32):
    """Lattice tables as the oracle builds them (mod_D3Q27setup.F90:28-150)."""
    dt = np.dtype(dtype)
    H2 = np.zeros((nl, 3, 3), dt)      # [l, q, p]  == H2(p,q,l)
    H3 = np.zeros((nl, 3, 3, 3), dt)   # [l, r, q, p] == H3(p,q,r,l)
    w = np.zeros(nl, dt)
    cx = np.zeros(nl, np.int32)
    cy = np.zeros(nl, np.int32)
    cz = np.zeros(nl, np.int32)
    b = np.zeros(nl, np.int32)
    fn = getattr(lib(), "orc_tables_%s" % ("f32" if dt == np.float32 else "f64"))
    rc = fn(ctypes.c_int(nl), _ptr(H2), _ptr(H3), _ptr(w), _ptr(cx), _ptr(cy), _ptr(cz), _ptr(b))
    if rc != 0:
        raise ValueError("nl must be 19 or 27")
    return dict(H2=H2, H3=H3, w=w, cx=cx, cy=cy, cz=cz, bounce=b)
