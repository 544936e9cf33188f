"""Python mirror of the reference's subroutine interfaces over the C ABI.

Each method of :class:`Lbm` is named after the Fortran subroutine it replaces
and takes the same arrays in the same order (geirev/LBM src/*.F90), as CUDA
torch tensors in the reference layout viewed in C order:

* ``f(nl,0:nx+1,0:ny+1,0:nz+1)`` -> ``float32[nz+2, ny+2, nx+2, nl]``
* ``rho(0:nx+1,0:ny+1,0:nz+1)``  -> ``float32[nz+2, ny+2, nx+2]``
* ``uvel(nz)``, ``ablvisc(nz)``  -> ``float32[nz]``
* ``uu(ny,nz,0:nrturb)``          -> ``float32[nrturb+1, nz, ny]``
* ``turbulence_df(nl,ny,nz)``     -> ``float32[nz, ny, nl]``
* ``lblanking`` logical(4)        -> ``int32[nz+2, ny+2, nx+2]``

The per-call methods also take float64 arrays: they then run the ``_f64``
entry points, the reference's DP build (every real in double precision).

torch is used for device memory and streams only; all arithmetic runs in the
library's sm_100a kernels.  Errors raise :class:`LbmError`.
"""
from __future__ import annotations

import ctypes
import dataclasses

import torch

from . import _lib
from ._lib import LbmError, LbmParams


@dataclasses.dataclass
class Params:
    """Run-time options (m_readinfile.F90:3-58, mod_dimensions.F90), lattice units."""
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
    storage: str = "f32"          # fused state storage: "f32" or "f16" (offsets scaled by 2^8)
    kinevisc: float = 1.0e-4
    smagorinsky: float = 0.15
    rho0: float = 1.0
    udir: float = 0.0

    def c(self) -> LbmParams:
        st = {"f32": _lib.LBM_STORE_F32, "f16": _lib.LBM_STORE_F16}[self.storage]
        return LbmParams(self.nx, self.ny, self.nz, self.nl, self.ibgk, self.ihrr, self.ivreman, self.ibnd,
                         self.jbnd, self.kbnd, self.iturb_pos, st, self.kinevisc, self.smagorinsky, self.rho0,
                         self.udir)

    @property
    def fshape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2, self.nl)

    @property
    def sshape(self):
        return (self.nz + 2, self.ny + 2, self.nx + 2)


def _ptr(t):
    return ctypes.c_void_p(t.data_ptr()) if t is not None else None


class Lbm:
    """One context of the C library (``lbm_create``) bound to the current CUDA device."""

    def __init__(self, params: Params, stream: torch.cuda.Stream | None = None, _borrowed=None):
        if not torch.cuda.is_available():
            raise RuntimeError("lbm_b200 needs a CUDA device; there is no CPU fallback")
        self.p = params
        self.L = _lib.load()
        self._cp = params.c()
        self._owned = _borrowed is None
        if _borrowed is not None:      # a member context owned by an Ensemble
            self.h = _borrowed
        else:
            h = ctypes.c_void_p()
            rc = self.L.lbm_create(ctypes.byref(h), ctypes.byref(self._cp))
            if rc != 0:
                raise LbmError(rc, "lbm_create failed for %s" % (params,))
            self.h = h
        self.stream = stream if stream is not None else torch.cuda.current_stream()
        self._call("lbm_set_stream", ctypes.c_void_p(self.stream.cuda_stream))
        self.set_params_f64()      # the float64 calls take the Params values at double precision

    def close(self):
        if getattr(self, "h", None):
            if self._owned:
                self.L.lbm_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    # ---- helpers ---------------------------------------------------------------
    def _call(self, name, *args):
        rc = getattr(self.L, name)(self.h, *args)
        if rc != 0:
            raise LbmError(rc, self.L.lbm_last_error(self.h).decode())
        return rc

    def _chk(self, t, shape, dtype=torch.float32, name="array"):
        if t is None:
            return
        if not t.is_cuda:
            raise LbmError(_lib.LBM_ERR_ARG, "%s must be a CUDA tensor" % name)
        if t.dtype != dtype or tuple(t.shape) != tuple(shape) or not t.is_contiguous():
            raise LbmError(_lib.LBM_ERR_ARG, "%s must be contiguous %s%s, got %s%s" % (
                name, dtype, tuple(shape), t.dtype, tuple(t.shape)))

    def _f(self, *ts, dtype=torch.float32):
        for t in ts:
            self._chk(t, self.p.fshape, dtype, name="f")

    def _s(self, *ts, dtype=torch.float32):
        for t in ts:
            self._chk(t, self.p.sshape, dtype, name="scalar field")

    @staticmethod
    def _real(t):
        """(entry-point suffix, dtype) of a per-call call from its first array:
        float32 runs the reference's default build, float64 its DP build
        (the ``_f64`` entry points); every array of the call has that dtype."""
        if t is not None and t.dtype == torch.float64:
            return "_f64", torch.float64
        return "", torch.float32

    # ---- tensors -----------------------------------------------------------------
    def empty_f(self, dtype=torch.float32):
        return torch.zeros(self.p.fshape, dtype=dtype, device="cuda")

    def empty_s(self, dtype=torch.float32):
        return torch.zeros(self.p.sshape, dtype=dtype, device="cuda")

    # ---- reference subroutines -------------------------------------------------------
    def set_params_f64(self, kinevisc=None, smagorinsky=None, rho0=None, udir=None):
        """kinevisc, smagorinsky, rho0 and udir of the float64 calls at double
        precision (default: the Params values)."""
        p = self.p
        self._call("lbm_set_params_f64", ctypes.c_double(p.kinevisc if kinevisc is None else kinevisc),
                   ctypes.c_double(p.smagorinsky if smagorinsky is None else smagorinsky),
                   ctypes.c_double(p.rho0 if rho0 is None else rho0), ctypes.c_double(p.udir if udir is None else udir))

    def fequil3(self, feq, rho, u, v, w):
        sfx, dt = self._real(feq)
        self._f(feq, dtype=dt)
        self._s(rho, u, v, w, dtype=dt)
        self._call("lbm_fequil3" + sfx, _ptr(feq), _ptr(rho), _ptr(u), _ptr(v), _ptr(w))

    def postcoll(self, f, tau, rho, u, v, w, ablvisc=None):
        sfx, dt = self._real(f)
        self._f(f, dtype=dt)
        self._s(tau, rho, u, v, w, dtype=dt)
        self._chk(ablvisc, (self.p.nz,), dt, name="ablvisc")
        self._call("lbm_postcoll" + sfx, _ptr(f), _ptr(tau), _ptr(rho), _ptr(u), _ptr(v), _ptr(w), _ptr(ablvisc))

    def drift(self, f, feq):
        sfx, dt = self._real(f)
        self._f(f, feq, dtype=dt)
        self._call("lbm_drift" + sfx, _ptr(f), _ptr(feq))

    def macrovars(self, rho, u, v, w, f):
        sfx, dt = self._real(f)
        self._s(rho, u, v, w, dtype=dt)
        self._f(f, dtype=dt)
        self._call("lbm_macrovars" + sfx, _ptr(rho), _ptr(u), _ptr(v), _ptr(w), _ptr(f))

    def regularization(self, f, feq, u, v, w):
        sfx, dt = self._real(f)
        self._f(f, feq, dtype=dt)
        self._s(u, v, w, dtype=dt)
        self._call("lbm_regularization" + sfx, _ptr(f), _ptr(feq), _ptr(u), _ptr(v), _ptr(w))

    def vreman(self, f, tau):
        sfx, dt = self._real(f)
        self._f(f, dtype=dt)
        self._s(tau, dtype=dt)
        self._call("lbm_vreman" + sfx, _ptr(f), _ptr(tau))

    def compute_fneq(self, f, feq):
        sfx, dt = self._real(f)
        self._f(f, feq, dtype=dt)
        self._call("lbm_compute_fneq" + sfx, _ptr(f), _ptr(feq))

    def compute_f(self, f, feq):
        sfx, dt = self._real(f)
        self._f(f, feq, dtype=dt)
        self._call("lbm_compute_f" + sfx, _ptr(f), _ptr(feq))

    def boundarycond(self, f1, f2, uvel):
        sfx, dt = self._real(f1)
        self._f(f1, f2, dtype=dt)
        self._chk(uvel, (self.p.nz,), dt, name="uvel")
        self._call("lbm_boundarycond" + sfx, _ptr(f1), _ptr(f2), _ptr(uvel))

    def solids(self, f, blanking):
        sfx, dt = self._real(f)
        self._f(f, dtype=dt)
        self._chk(blanking, self.p.sshape, torch.int32, name="blanking")
        self._call("lbm_solids" + sfx, _ptr(f), _ptr(blanking))

    def inflow_turbulence_forcing(self, df, rho, u, v, w, uu, vv, ww, ampl, it, nrturb):
        sfx, dt = self._real(df)
        self._chk(df, (self.p.nz, self.p.ny, self.p.nl), dt, name="turbulence_df")
        self._s(rho, u, v, w, dtype=dt)
        for t in (uu, vv, ww):
            self._chk(t, (nrturb + 1, self.p.nz, self.p.ny), dt, name="uu/vv/ww")
        a = ctypes.c_double(ampl) if sfx else ctypes.c_float(ampl)
        self._call("lbm_inflow_turbulence_forcing" + sfx, _ptr(df), _ptr(rho), _ptr(u), _ptr(v), _ptr(w), _ptr(uu),
                   _ptr(vv), _ptr(ww), a, ctypes.c_int32(it), ctypes.c_int32(nrturb))

    def inflow_turbulence_apply(self, f, df):
        sfx, dt = self._real(f)
        self._f(f, dtype=dt)
        self._chk(df, (self.p.nz, self.p.ny, self.p.nl), dt, name="turbulence_df")
        self._call("lbm_inflow_turbulence_apply" + sfx, _ptr(f), _ptr(df))

    def inflow_turbulence_compute(self, uu, vv, ww, nrturb, seed, rr=None):
        """Fill uu, vv, ww (and rr) -- float32 (nrturb+1, nz, ny) -- with the inflow-turbulence levels."""
        for t in (uu, vv, ww, rr):
            self._chk(t, (nrturb + 1, self.p.nz, self.p.ny), name="turbulence field")
        self._call("lbm_inflow_turbulence_compute", _ptr(uu), _ptr(vv), _ptr(ww), _ptr(rr), ctypes.c_int32(nrturb),
                   ctypes.c_uint64(seed))

    # ---- adjoints of the per-call kernels (reverse mode) -------------------------------
    def postcoll_adj(self, fhat, f, rho, u, v, w, rhohat, uhat, vhat, what, tau=None, ablvisc=None, blanking=None):
        """fhat: adjoint of postcoll's output f in, of its input f out; rhohat..what incremented.
        blanking: apply the adjoint of a following solids call first."""
        self._f(fhat, f)
        self._s(rho, u, v, w, rhohat, uhat, vhat, what, tau)
        self._chk(blanking, self.p.sshape, dtype=torch.int32, name="blanking")
        self._call("lbm_postcoll_adj", _ptr(fhat), _ptr(f), _ptr(tau), _ptr(rho), _ptr(u), _ptr(v), _ptr(w),
                   _ptr(ablvisc), _ptr(rhohat), _ptr(uhat), _ptr(vhat), _ptr(what), _ptr(blanking))

    def macrovars_drift_adj(self, fhat_in, fhat_out, rhohat, uhat, vhat, what, rho, u, v, w):
        """macrovars_adj (on the drift output, interior cells) then drift_adj, in one pass."""
        self._f(fhat_in, fhat_out)
        self._s(rhohat, uhat, vhat, what, rho, u, v, w)
        self._call("lbm_macrovars_drift_adj", _ptr(fhat_in), _ptr(fhat_out), _ptr(rhohat), _ptr(uhat), _ptr(vhat),
                   _ptr(what), _ptr(rho), _ptr(u), _ptr(v), _ptr(w))

    def macrovars_adj(self, fhat, rhohat, uhat, vhat, what, f):
        self._f(fhat, f)
        self._s(rhohat, uhat, vhat, what)
        self._call("lbm_macrovars_adj", _ptr(fhat), _ptr(rhohat), _ptr(uhat), _ptr(vhat), _ptr(what), _ptr(f))

    def drift_adj(self, fhat_in, fhat_out):
        self._f(fhat_in, fhat_out)
        self._call("lbm_drift_adj", _ptr(fhat_in), _ptr(fhat_out))

    def boundarycond_adj(self, f1hat, f2hat, uvelhat):
        self._f(f1hat, f2hat)
        self._chk(uvelhat, (self.p.nz,), name="uvelhat")
        self._call("lbm_boundarycond_adj", _ptr(f1hat), _ptr(f2hat), _ptr(uvelhat))

    # ---- reverse sweep in the state layout ------------------------------------------------
    def state_bytes(self) -> int:
        n = ctypes.c_int64()
        self._call("lbm_state_bytes", ctypes.byref(n))
        return n.value

    def empty_state(self):
        """A zeroed FP32 array of one state buffer's size (a state copy or a state-layout adjoint)."""
        return torch.zeros((self.state_bytes() + 3) // 4, dtype=torch.float32, device="cuda")

    def state_scratch(self):
        """An uninitialised FP32 array of one state buffer's size (for lbm_state_copy)."""
        return torch.empty((self.state_bytes() + 3) // 4, dtype=torch.float32, device="cuda")

    def state_copy(self, dst):
        self._call("lbm_state_copy", _ptr(dst))

    def state_adjoint_step(self, W, A, P, pull: bool, uvelhat):
        self._call("lbm_state_adjoint_step", _ptr(W), _ptr(A), _ptr(P), ctypes.c_int32(1 if pull else 0), _ptr(uvelhat))

    def state_adjoint_seed(self, A, P, probes, uhat):
        """probes: int32 CUDA (n, 3) 1-based (i, j, k); uhat: float32 CUDA (n, 3)."""
        self._call("lbm_state_adjoint_seed", _ptr(A), _ptr(P), _ptr(probes.contiguous()), _ptr(uhat.contiguous()),
                   ctypes.c_int32(probes.shape[0]))

    def state_adjoint_export(self, fhat, A):
        self._f(fhat)
        self._call("lbm_state_adjoint_export", _ptr(fhat), _ptr(A))

    def fillghosts(self, f):
        sfx, dt = self._real(f)
        self._f(f, dtype=dt)
        self._call("lbm_fillghosts" + sfx, _ptr(f))

    # ---- fused state ------------------------------------------------------------------
    def state_import(self, f1, f2, rho, u, v, w, it=0):
        self._f(f1, f2)
        self._s(rho, u, v, w)
        self._call("lbm_state_import", _ptr(f1), _ptr(f2), _ptr(rho), _ptr(u), _ptr(v), _ptr(w),
                   ctypes.c_int32(it))

    def state_export(self, f1, f2):
        self._f(f1, f2)
        self._call("lbm_state_export", _ptr(f1), _ptr(f2))

    def get_macro(self, rho, u, v, w):
        self._s(rho, u, v, w)
        self._call("lbm_get_macro", _ptr(rho), _ptr(u), _ptr(v), _ptr(w))

    def set_solids(self, blanking):
        self._chk(blanking, self.p.sshape, torch.int32, name="blanking")
        self._call("lbm_set_solids", _ptr(blanking))

    def set_turbulence(self, uu, vv, ww, nrturb, ampl):
        if uu is None:
            self._call("lbm_set_turbulence", None, None, None, ctypes.c_int32(0), ctypes.c_float(0.0))
            return
        for t in (uu, vv, ww):
            self._chk(t, (nrturb + 1, self.p.nz, self.p.ny), name="uu/vv/ww")
        self._call("lbm_set_turbulence", _ptr(uu), _ptr(vv), _ptr(ww), ctypes.c_int32(nrturb),
                   ctypes.c_float(ampl))

    def forcings_apply(self, f, external_forcing, rho, u, v, w):
        """external_forcing: (nz+2, ny+2, nx+2, 3), the reference's external_forcing(3,0:nx+1,...)."""
        sfx, dt = self._real(f)
        self._f(f, dtype=dt)
        self._chk(external_forcing, self.p.sshape + (3,), dt, name="external_forcing")
        self._s(rho, u, v, w, dtype=dt)
        self._call("lbm_forcings_apply" + sfx, _ptr(f), _ptr(external_forcing), _ptr(rho), _ptr(u), _ptr(v),
                   _ptr(w))

    def set_forcing(self, external_forcing):
        """Fused-step forcing field (read at every step; keep the tensor alive), or None."""
        self._chk(external_forcing, self.p.sshape + (3,), name="external_forcing")
        self._force_ref = external_forcing
        self._call("lbm_set_forcing", _ptr(external_forcing))

    def set_inflow(self, uvel):
        self._chk(uvel, (self.p.nz,), name="uvel")
        self._call("lbm_set_inflow", _ptr(uvel))

    def step(self, nsteps=1):
        self._call("lbm_step", ctypes.c_int32(nsteps))

    # ---- j slabs (one tile of a domain split in j; lbm_b200.slabs drives them) ----
    def set_halo_j(self, on: bool = True):
        self._call("lbm_set_halo_j", ctypes.c_int32(1 if on else 0))

    def halo_plane_bytes(self) -> int:
        n = ctypes.c_int64(0)
        self._call("lbm_halo_plane_bytes", ctypes.byref(n))
        return int(n.value)

    def halo_pack_j(self, to_south, to_north):
        self._call("lbm_halo_pack_j", _ptr(to_south), _ptr(to_north))

    def halo_unpack_j(self, from_south, from_north):
        self._call("lbm_halo_unpack_j", _ptr(from_south), _ptr(from_north))

    def snapshot_bytes(self) -> int:
        n = ctypes.c_int64(0)
        self._call("lbm_state_snapshot_bytes", ctypes.byref(n))
        return int(n.value)

    def snapshot(self, dst=None):
        """Device snapshot of the stepped state (allocated when ``dst`` is None)."""
        if dst is None:
            dst = torch.empty((self.snapshot_bytes() + 3) // 4, dtype=torch.float32, device="cuda")
        self._call("lbm_state_snapshot", _ptr(dst))
        return dst

    def restore(self, src):
        """Resume from a snapshot (same parameters)."""
        self._call("lbm_state_restore", _ptr(src))

    def step_to(self, dst):
        """One step whose state buffer is written to ``dst`` (a :meth:`state_scratch`
        tensor, kept alive by the caller until two more steps or an import)."""
        self._call("lbm_step_to", _ptr(dst))

    def set_kernel(self, which: str):
        """Steady step kernel: "pair" (two cells per thread, default where it applies)
        or "pull" (one cell per thread)."""
        self._call("lbm_set_kernel", ctypes.c_int32({"pull": _lib.LBM_KERNEL_PULL, "pair": _lib.LBM_KERNEL_PAIR}[which]))

    def step_host(self, nsteps, uvel_host=None):
        """Steps with host buffers: uvel_host is a CPU float32 tensor (pinned for async copies)."""
        st = ctypes.c_int32(0)
        if uvel_host is not None:
            if uvel_host.is_cuda or uvel_host.dtype != torch.float32 or tuple(uvel_host.shape) != (self.p.nz,):
                raise LbmError(_lib.LBM_ERR_ARG, "uvel_host must be a CPU float32 tensor of shape (nz,)")
        self._call("lbm_step_host", ctypes.c_int32(nsteps), _ptr(uvel_host), ctypes.byref(st))
        return st.value

    @property
    def it(self):
        v = ctypes.c_int32()
        self._call("lbm_get_step", ctypes.byref(v))
        return v.value

    def status(self):
        v = ctypes.c_int32()
        self._call("lbm_status", ctypes.byref(v))
        return v.value

    def synchronize(self):
        self._call("lbm_synchronize")

    # ---- conservation ----------------------------------------------------------------
    def mass_momentum(self, f, out=None):
        """FP64 (mass, mx, my, mz) of a reference-layout f; returns a CUDA float64 tensor of 4."""
        self._f(f)
        if out is None:
            out = torch.zeros(4, dtype=torch.float64, device="cuda")
        self._chk(out, (4,), torch.float64, name="out")
        self._call("lbm_mass_momentum", _ptr(f), _ptr(out))
        return out

    def conservation(self):
        """FP64 (mass, mx, my, mz) of the fused state's f1."""
        v = (ctypes.c_double * 4)()
        self._call("lbm_conservation", v)
        return tuple(v)

    # ---- instrumentation -------------------------------------------------------------
    @property
    def launches(self):
        v = ctypes.c_int64()
        self._call("lbm_launch_count", ctypes.byref(v))
        return v.value

    def profile(self, enable=True):
        self._call("lbm_profile", ctypes.c_int32(1 if enable else 0))

    def profile_read(self):
        """(summed device ms, launches) of the fused step kernel since profile(True)."""
        ms, n = ctypes.c_double(), ctypes.c_int64()
        self._call("lbm_profile_read", ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value

    def profile_read_boundary(self):
        """(summed device ms, steps) of the boundary launches that followed the
        timed step kernels since profile(True)."""
        ms, n = ctypes.c_double(), ctypes.c_int64()
        self._call("lbm_profile_read_boundary", ctypes.byref(ms), ctypes.byref(n))
        return ms.value, n.value


class Ensemble:
    """Many independent runs advanced together (``lbm_ensemble_*``): two launches
    per step for the whole ensemble, replayed from a CUDA graph.  ``members[m]``
    is an :class:`Lbm` on member m's context, for import, inflow, turbulence,
    export and macro reads."""

    def __init__(self, params: list[Params], stream: torch.cuda.Stream | None = None):
        if not torch.cuda.is_available():
            raise RuntimeError("lbm_b200 needs a CUDA device; there is no CPU fallback")
        self.L = _lib.load()
        arr = (LbmParams * len(params))(*[p.c() for p in params])
        h = ctypes.c_void_p()
        rc = self.L.lbm_ensemble_create(ctypes.byref(h), arr, len(params))
        if rc != 0:
            raise LbmError(rc, self.L.lbm_ensemble_last_error(None).decode())
        self.h = h
        self.members = []
        for m, p in enumerate(params):
            c = ctypes.c_void_p()
            self._call("lbm_ensemble_member", m, ctypes.byref(c))
            self.members.append(Lbm(p, stream=stream, _borrowed=c))

    def _call(self, name, *args):
        rc = getattr(self.L, name)(self.h, *args)
        if rc != 0:
            raise LbmError(rc, self.L.lbm_ensemble_last_error(self.h).decode())
        return rc

    def step(self, nsteps: int = 1):
        self._call("lbm_ensemble_step", int(nsteps))

    def autotune(self, trial_steps: int = 5):
        """Time each launch shape, then graph replay against direct launches for the
        fastest; returns (chosen variant, ms per step of each shape)."""
        v = ctypes.c_int32(0)
        ms = (ctypes.c_float * _lib.LBM_ENS_VARIANTS)()
        self._call("lbm_ensemble_autotune", int(trial_steps), ctypes.byref(v), ms)
        return v.value, list(ms)

    def config(self):
        """(launch shape variant, graph steps: 0 = direct launches) in use."""
        v, g = ctypes.c_int32(0), ctypes.c_int32(0)
        self._call("lbm_ensemble_get_config", ctypes.byref(v), ctypes.byref(g))
        return v.value, g.value

    @staticmethod
    def variant_shape(variant: int):
        """(threads per block, minimum resident blocks per SM, tiles per block) of
        a launch shape."""
        L = _lib.load()
        t, m, r = ctypes.c_int32(0), ctypes.c_int32(0), ctypes.c_int32(0)
        rc = L.lbm_ensemble_variant_shape(int(variant), ctypes.byref(t), ctypes.byref(m), ctypes.byref(r))
        if rc != 0:
            raise LbmError(rc, "variant %d out of range" % variant)
        return t.value, m.value, r.value

    def set_variant(self, v: int):
        self._call("lbm_ensemble_set_variant", int(v))

    def profile(self, nsteps: int):
        """nsteps direct-launch steps timed launch by launch: (step-kernel ms,
        boundary-kernel ms), the means per step."""
        a, b = ctypes.c_float(0.0), ctypes.c_float(0.0)
        self._call("lbm_ensemble_profile", int(nsteps), ctypes.byref(a), ctypes.byref(b))
        return a.value, b.value

    def set_graph(self, steps: int):
        self._call("lbm_ensemble_set_graph", int(steps))

    def close(self):
        if getattr(self, "h", None):
            for mem in self.members:
                mem.h = None
            self.L.lbm_ensemble_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
