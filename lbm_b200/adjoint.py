"""Gradients of a probe-misfit loss through N time steps of the per-call path.

The forward run is main.F90's loop (main.F90:283-329, without the inflow
turbulence): per step postcoll, solids, boundarycond, drift, swap, macrovars,
on the library's per-call kernels.  The state of step n is (f1, f2, rho/u/v/w),
with rho, u, v, w = macrovars(f1); the controls are the initial f1 (its rho, u,
v, w recomputed from it) and the inflow profile uvel(k) that boundarycond uses
in every step.

The reverse sweep chains the library's adjoint kernels in the opposite order
(macrovars and drift in one pass, boundarycond, then solids and postcoll in
one pass).  Memory is bounded by
checkpoint-and-recompute: the forward keeps (f1, f2) every ``checkpoint``
steps; the reverse sweep replays each segment from its checkpoint, keeping the
segment's states, and walks back through it.
"""
from __future__ import annotations

import numpy as np
import torch

from .api import Lbm, Params


class ProbeProblem:
    """u at probe cells after ``nsteps`` steps, and the reverse sweep of its loss.

    probes: int array (P, 3) of 1-based interior (i, j, k) cells.  dtype
    torch.float64 runs the forward through the FP64 entry points (the
    reference's DP build), for finite-difference checks; the reverse sweep
    runs on FP32 states."""

    def __init__(self, params: Params, probes, nsteps: int, blanking=None, checkpoint: int = 10,
                 dtype=torch.float32):
        self.p = params
        self.dtype = dtype
        self.lbm = Lbm(params)
        self.nsteps = int(nsteps)
        self.K = max(1, int(checkpoint))
        self.blanking = blanking
        pr = np.asarray(probes, dtype=np.int64)
        self.probes = pr
        # flat indices into the (nz+2, ny+2, nx+2) scalar fields
        self.pidx = torch.from_numpy((pr[:, 2] * (params.ny + 2) + pr[:, 1]) * (params.nx + 2) + pr[:, 0]).cuda()
        self.tau = torch.full(params.sshape, 3.0 * params.kinevisc + 0.5, dtype=dtype, device="cuda")
        self.ckpt = {}

    # ---- forward ----------------------------------------------------------------------
    def _macro(self, f):
        L = self.lbm
        R = [L.empty_s(self.dtype) for _ in range(4)]
        L.macrovars(*R, f)
        return R

    def _step(self, A, B, R, uvel):
        """one step in place of main.F90's order; returns the new (f1, f2)"""
        L = self.lbm
        L.postcoll(A, self.tau, *R)
        if self.blanking is not None:
            L.solids(A, self.blanking)
        L.boundarycond(A, B, uvel)
        L.drift(B, A)
        A, B = B, A
        L.macrovars(*R, A)
        return A, B

    def probe_u(self, R):
        return torch.stack([R[q].reshape(-1)[self.pidx] for q in (1, 2, 3)], dim=1)

    def forward(self, f1, f2, uvel, keep: bool = True):
        """u, v, w at the probes after nsteps; keeps the checkpoints for backward()."""
        A, B = f1.clone(), f2.clone()
        R = self._macro(A)
        self.ckpt = {}
        self.uvel = uvel.contiguous()
        for n in range(self.nsteps):
            if keep and n % self.K == 0:
                self.ckpt[n] = (A.clone(), B.clone())
            A, B = self._step(A, B, R, self.uvel)
        return self.probe_u(R)

    # ---- reverse ----------------------------------------------------------------------
    def backward(self, uhat_probes):
        """Adjoint of the probe velocities (P, 3) -> (d loss / d f1 initial, d loss / d uvel)."""
        if self.dtype != torch.float32:
            raise ValueError("the reverse sweep runs on FP32 states; this problem's forward is %s" % self.dtype)
        L = self.lbm
        Ah, Bh = L.empty_f(), L.empty_f()
        Rh = [L.empty_s() for _ in range(4)]
        for q in range(3):
            Rh[q + 1].view(-1).index_add_(0, self.pidx, uhat_probes[:, q].contiguous().float())
        uvel_h = torch.zeros(self.p.nz, dtype=torch.float32, device="cuda")
        starts = sorted(self.ckpt)
        for s in reversed(starts):
            e = min(s + self.K, self.nsteps)
            A, B = (t.clone() for t in self.ckpt[s])
            R = self._macro(A)
            states = []                       # (A_n, R_n) of the segment
            for n in range(s, e):
                states.append((A.clone(), [t.clone() for t in R]))
                A, B = self._step(A, B, R, self.uvel)
            R_next = R
            for n in range(e - 1, s - 1, -1):
                A_n, R_n = states[n - s]
                Ah, Bh, Rh = self._reverse_step(Ah, Bh, Rh, A_n, R_n, R_next, uvel_h)
                R_next = R_n
            del states
        A0 = self.ckpt[0][0]
        L.macrovars_adj(Ah, *Rh, A0)          # rho, u, v, w of step 0 are macrovars(f1)
        return Ah, uvel_h

    def _reverse_step(self, Ah, Bh, Rh, A_n, R_n, R_next, uvel_h):
        L = self.lbm
        W = Bh                                # f2 of step n+1 is the post-collision f1 of step n
        # macrovars(f1(n+1)) then drift: interior of f1(n+1) = pull(post-collision f1)
        L.macrovars_drift_adj(W, Ah, *Rh, *R_next)
        for t in Rh:
            t.zero_()
        Bn = Ah                               # f1(n+1)'s ghost cells are f2(n)'s
        L.boundarycond_adj(W, Bn, uvel_h)
        # solids (a swap, its own adjoint) folded into the postcoll adjoint
        L.postcoll_adj(W, A_n, *R_n, *Rh, tau=self.tau, blanking=self.blanking)
        return W, Bn, Rh

    def close(self):
        self.ckpt = {}
        if getattr(self, "_rep", None) is not None:
            self._rep.close()
            self._rep = None
        self.lbm.close()


def initial_state(lbm: Lbm, rho, u, v, w, uvel):
    """(f1, f2) as main.F90:243-247 initialises them: fequil3, fillghosts, f1 = f2,
    boundarycond twice (in the dtype of rho: float32, or float64 for the DP build)."""
    fB = lbm.empty_f(rho.dtype)
    lbm.fequil3(fB, rho, u, v, w)
    lbm.fillghosts(fB)
    fA = fB.clone()
    lbm.boundarycond(fB, fA, uvel)
    lbm.boundarycond(fA, fB, uvel)
    return fA, fB


class FusedProbeProblem:
    """The probe-misfit problem of :class:`ProbeProblem` with the forward run made
    by the fused step (the library's default kernels) and the reverse sweep in
    the state layout (``lbm_state_adjoint_*``).  Checkpoints are device
    snapshots of the fused state (``lbm_state_snapshot``) every ``checkpoint``
    steps, and for the first segment the imported state buffer (the input of
    step 0) with a snapshot after step 0.  Each segment is replayed from its
    snapshot, each step writing its state buffer into an array of its own
    (``lbm_step_to``)."""

    def __init__(self, params: Params, probes, nsteps: int, blanking=None, checkpoint: int = 10):
        if params.storage != "f32":
            raise ValueError("the state-layout reverse sweep needs FP32 state storage")
        self.p = params
        self.lbm = Lbm(params)
        self.nsteps = int(nsteps)
        self.K = max(1, int(checkpoint))
        self.blanking = blanking
        self.probes = np.asarray(probes, dtype=np.int64)
        self.probes_dev = torch.from_numpy(self.probes.astype(np.int32)).cuda()
        self.pidx = torch.from_numpy((self.probes[:, 2] * (params.ny + 2) + self.probes[:, 1]) * (params.nx + 2)
                                     + self.probes[:, 0]).cuda()
        if blanking is not None:
            self.lbm.set_solids(blanking)
        self.ckpt = {}

    def _import(self, f1, f2):
        L = self.lbm
        R = [L.empty_s() for _ in range(4)]
        L.macrovars(*R, f1)
        L.state_import(f1, f2, *R)
        L.set_inflow(self.uvel)

    def forward(self, f1, f2, uvel, keep: bool = True):
        L = self.lbm
        self.uvel = uvel.contiguous()
        self.ckpt = {}
        self._import(f1, f2)
        for n in range(self.nsteps):
            if keep and n % self.K == 0 and n > 0:
                self.ckpt[n] = L.snapshot()
            if keep and n == 0:
                pre = L.state_scratch()
                L.state_copy(pre)            # the imported f1: the input of step 0
            L.step(1)
            if keep and n == 0:
                self.ckpt[0] = (pre, L.snapshot())   # and the state after step 0
        R = [L.empty_s() for _ in range(4)]
        L.get_macro(*R)
        return torch.stack([R[q].reshape(-1)[self.pidx] for q in (1, 2, 3)], dim=1)

    def _replayer(self):
        """The context that replays segments, on a stream of its own with a higher
        priority than the adjoint's, so a replay runs beside the adjoint steps of
        the segment after it (the replay is DRAM-bound, the adjoint cell kernel
        issue-bound)."""
        if getattr(self, "_rep", None) is None:
            stream = torch.cuda.Stream(priority=-1)
            self._rep = Lbm(self.p, stream=stream)
            if self.blanking is not None:
                self._rep.set_solids(self.blanking)
        return self._rep

    def backward(self, uhat_probes, overlap: bool = True):
        """Gradient of the probe loss with respect to the initial f1 and the inflow
        profile.  overlap: replay segment q+1 (on the replay context's stream, into
        the other of two sets of state arrays) while the adjoint steps of segment q
        run; otherwise replay and reverse one segment after the other."""
        L = self.lbm
        W, A = L.empty_state(), L.empty_state()
        uvel_h = torch.zeros(self.p.nz, dtype=torch.float32, device="cuda")
        segs = sorted(self.ckpt, reverse=True)
        R = self._replayer() if overlap else L
        main = L.stream
        rep = R.stream
        rep.wait_stream(main)                # the forward's snapshots and the seed are written on main
        R.set_inflow(self.uvel)
        nsets = 2 if overlap else 1
        sets = [[L.state_scratch() for _ in range(self.K)] for _ in range(nsets)]
        released = [None] * nsets            # event: the adjoint is done with a set

        def replay(q):
            """The states of segment q: P[n - s] after step n, and the input of step s."""
            s, b = segs[q], q % nsets
            e = min(s + self.K, self.nsteps)
            P = list(sets[b][:e - s])
            with torch.cuda.stream(rep):
                if released[b] is not None:
                    rep.wait_event(released[b])
                if s == 0:
                    first, after0 = self.ckpt[0]  # the imported f1 (a step-0 input, not pulled) and the state after step 0
                    P[0] = after0
                    R.restore(after0)
                    start = 1
                else:
                    first = self.ckpt[s]     # the state after step s - 1, which step s pulls from
                    R.restore(first)
                    start = s
                for n in range(start, e):
                    R.step_to(P[n - s])      # the step writes its state into the array
                ready = torch.cuda.Event()
                ready.record(rep)
            return first, P, ready

        # The adjoint steps of segment q are enqueued before the replay of q + 1:
        # restoring a snapshot reads its header on the host, which waits for the
        # replay stream, so the main stream must already hold work by then.
        pending = replay(0)
        for q, s in enumerate(segs):
            b = q % nsets
            e = min(s + self.K, self.nsteps)
            first, P, ready = pending
            main.wait_event(ready)
            with torch.cuda.stream(main):
                if e == self.nsteps:
                    L.state_adjoint_seed(A, P[e - s - 1], self.probes_dev, uhat_probes.float())
                for n in range(e - 1, s - 1, -1):
                    src = P[n - s - 1] if n > s else first
                    L.state_adjoint_step(W, A, src, n > s or s > 0, uvel_h)
                    W, A = A, W               # A: adjoint of f1 before step n, W: of f2
                done = torch.cuda.Event()
                done.record(main)
            released[b] = done
            if q + 1 < len(segs):
                pending = replay(q + 1)
        g = L.empty_f()
        L.state_adjoint_export(g, A)
        main.synchronize()
        del sets
        return g, uvel_h

    def close(self):
        self.ckpt = {}
        if getattr(self, "_rep", None) is not None:
            self._rep.close()
            self._rep = None
        self.lbm.close()
