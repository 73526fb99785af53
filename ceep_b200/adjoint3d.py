"""Checkpointed adjoint of the batched 3D solver and its torch.autograd.Function.

Gradient of a loss on the probe series with respect to the per-cell eps_r,
sigma and Debye delta_eps maps of a ``BatchedFDTD3D``, from the exact discrete
adjoint of its step (``csrc/adjoint3d.cu``) run backwards in time:

* the forward pass keeps the state every ``checkpoint_every`` steps (the last
  segment is run with the E save on, so it is never recomputed);
* the recompute of the next segment overlaps the adjoint of the current one
  on a second stream when a second segment buffer fits in free memory
  (``overlap=None``; True/False force it);
* for each segment, last first, the state is restored, the segment is
  recomputed while the E half-step stores the three E components of every
  step (the recompute skips the CPML shell, which no stored value depends
  on), and the transposed steps run back over it, accumulating d(loss)/d of
  the interior update coefficients (ca, cb, k2) in FP64;
* the chain rule from those coefficients to (eps_r, sigma, delta_eps) runs in
  torch FP64 through the same formulas as the forward
  (src/ceep/solvers/fdtd_3d_batched.py:281-296, src/ceep/materials/dispersive.py:253-261).

Memory per checkpoint is the solver state (E, H, CPML psi, Debye currents);
a segment buffer holds ``checkpoint_every + 1`` copies of the three E
components.  Gradients live on the interior E box [n+1, N-n)^3, the only
cells whose coefficients the probe series depends on.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import torch

from . import physics
from ._lib import check, lib
from .adjoint import coefficient_maps, run_segments_backward
from .distributed import allreduce_gradient
from .solvers import _ptr
from .solvers3d import BatchedFDTD3D


class _AdjDesc3D(C.Structure):
    P = C.c_void_p
    _fields_ = [("mu", P), ("nu", P), ("lj", P), ("grad", P), ("probe_grad", P)]


def save_slot_shape(solver):
    """One slot of a segment buffer: the three E components on the interior
    box [n+1, N-n)^3, the only cells the E half-step updates,
    (3, G, nzi, nyi, nxi, W)."""
    G, nz, ny, nx, W = solver._f["ex"].shape
    n = solver.cpml_thickness
    return (3, G, nz - 2 * n - 1, ny - 2 * n - 1, nx - 2 * n - 1, W)


def interior_e(solver, field):
    """The interior-box view of one (G, nz, ny, nx, W) E component."""
    n = solver.cpml_thickness
    _, nz, ny, nx, _ = field.shape
    return field[:, n + 1:nz - n, n + 1:ny - n, n + 1:nx - n]


class Adjoint3D:
    """Gradient driver for one ``BatchedFDTD3D`` (Debye poles only, CPML >= 2)."""

    def __init__(self, solver: BatchedFDTD3D, checkpoint_every: int = 50, overlap=None, keep_bytes: int = 0,
                 reduce_ranks: bool = False):
        """``reduce_ranks``: as for ``Adjoint2D`` (this rank's transmit events
        only; gradient maps summed over ranks)."""
        if solver._lorentz:
            raise ValueError("the 3D adjoint supports Debye poles only")
        if solver.cpml_thickness < 1:
            raise ValueError("the 3D adjoint needs a CPML (cpml_thickness >= 2)")
        self.s = solver
        self.K = max(1, int(checkpoint_every))
        self.overlap = overlap          # None: when a second segment buffer fits in free memory
        # device bytes the forward pass may spend on keeping trailing segments
        # (each saves its recompute in the backward pass); the last one is
        # always kept
        self.keep_bytes = max(0, int(keep_bytes))
        self.reduce_ranks = bool(reduce_ranks)
        self._kept, self._starts = set(), []
        self._params = None
        self._ckpt = {}
        self._segs = []

    # -- parameters -------------------------------------------------------------
    def set_parameters(self, eps_r, sigma, deps=None, tau=None) -> None:
        """(nx, ny, nz) maps in the reference's axis order; ``deps``/``tau`` are
        the maps of the solver's single Debye pole when it has one."""
        s = self.s
        dev = s.device
        f64 = lambda t: torch.as_tensor(t, dtype=torch.float64).to(dev)
        eps_r, sigma = f64(eps_r), f64(sigma)
        debye = [(f64(deps), f64(tau))] if s._debye else []
        if len(s._debye) > 1:
            raise ValueError("set_parameters takes the maps of one Debye pole")
        self._params = (eps_r, sigma, debye)
        if not s._built:
            s._build()
        coef, ade = physics.coefficient_tensors_3d(eps_r, sigma, s._mu_r, s._sigma_m, s.dt, debye, (), dev)
        s._coef.copy_(coef)
        if ade.shape[0]:
            s._ade_coef.copy_(ade)

    # -- state ---------------------------------------------------------------------
    def _state_tensors(self):
        s = self.s
        ts = list(s._f.values()) + list(s._psi.values())
        if s._j is not None:
            ts.append(s._j)
        return ts

    def _ckpt_views(self):
        """What an interior-only recompute reads: E everywhere (its cells
        outside the interior are read by the H box and may hold a source), H
        on the box [n, N-n)^3 and the currents on the interior [n+1, N-n)^3;
        not the psi arrays nor H in the shell, which it never touches."""
        s = self.s
        n = s.cpml_thickness
        _, nz, ny, nx, _ = s._f["ex"].shape
        box = (slice(None), slice(n, nz - n), slice(n, ny - n), slice(n, nx - n))
        views = [s._f[k] for k in ("ex", "ey", "ez")] + [s._f[k][box] for k in ("hx", "hy", "hz")]
        if s._j is not None:
            views.append(s._j[:, :, :, n + 1:nz - n, n + 1:ny - n, n + 1:nx - n])
        return views

    def _restore(self, a):
        ck = self._ckpt[a]
        if ck is None:                 # step 0: the zero state
            for t in self._state_tensors():
                t.zero_()
        else:
            for t, c in zip(self._ckpt_views(), ck):
                t.copy_(c)

    def _segment_shape(self):
        return (min(self.K, self.s.total_steps) + 1,) + save_slot_shape(self.s)

    def segment_bytes(self):
        """Device bytes of one segment buffer (interior E slots of K + 1 steps)."""
        return 4 * int(np.prod(self._segment_shape()))

    def kept_segments(self, nseg):
        """How many trailing segments the forward pass keeps: the last one
        always, more while their buffers fit in ``keep_bytes``."""
        return max(1, min(nseg, self.keep_bytes // max(1, self.segment_bytes())))

    def _buffers(self, count):
        """`count` segment buffers, allocated once: the save graphs are keyed
        on their addresses."""
        while len(self._segs) < count:
            self._segs.append(torch.empty(self._segment_shape(), dtype=torch.float32, device=self.s.device))
        return self._segs

    def _run_save(self, a, b, buf, interior_only):
        s = self.s
        seg = self._segs[buf]
        stream = torch.cuda.current_stream(s.device)
        for c, k in enumerate(("ex", "ey", "ez")):
            seg[0, c].copy_(interior_e(s, s._f[k]))
        check(lib().ceep3d_plan_run_save(s._plan, a, b - a, C.c_void_p(stream.cuda_stream), int(s.use_graph),
                                         seg.data_ptr(), a, int(interior_only)), "ceep3d_plan_run_save")

    def forward(self) -> torch.Tensor:
        """Run all steps from a zero state, keeping checkpoints; returns the
        probe series (ntx, nprobe, T) float32 on the device."""
        s = self.s
        s.reset()
        T, K = s.total_steps, self.K
        self._ckpt = {}
        starts = list(range(0, T, K))
        M = self.kept_segments(len(starts))
        self._buffers(M)
        stream = torch.cuda.current_stream(s.device)
        self._starts, self._kept = starts, set()
        for j, a in enumerate(starts):
            b = min(a + K, T)
            i = len(starts) - 1 - j                 # index in the backward order
            if i < M:                               # kept: its slots stay in buffer i
                self._run_save(a, b, i, interior_only=False)
                self._kept.add(a)
            else:
                self._ckpt[a] = None if a == 0 else [t.clone() for t in self._ckpt_views()]
                s.advance(a, b - a, stream=stream)
        return s.probe_data[:, :len(s.probe_positions)].clone()

    # -- backward ------------------------------------------------------------------
    def backward(self, grad_probes: torch.Tensor):
        """d(loss)/d(eps_r, sigma[, deps]) as (nx, ny, nz) FP64 maps, given
        d(loss)/d(probe series)."""
        s = self.s
        dev = s.device
        T, K, n = s.total_steps, self.K, s.cpml_thickness
        f32 = dict(dtype=torch.float32, device=dev)
        shape = tuple(s._f["ex"].shape)
        mu = torch.zeros((3,) + shape, **f32)
        nu = torch.zeros((3,) + shape, **f32)
        lj = torch.zeros_like(s._j) if s._j is not None else None
        nd = len(s._debye)
        ks = 2 + nd
        ni = (s.nz - 2 * n - 1, s.ny - 2 * n - 1, s.nx - 2 * n - 1)
        grad = torch.zeros((s._groups, ks) + ni, dtype=torch.float64, device=dev)
        P = len(s.probe_positions)
        gp = torch.zeros((s.batch, max(P, 1), T), **f32)
        if P:
            gp[:, :P] = grad_probes.to(torch.float32)
        d = _AdjDesc3D()
        d.mu, d.nu, d.lj, d.grad, d.probe_grad = mu.data_ptr(), nu.data_ptr(), _ptr(lj), grad.data_ptr(), \
            gp.data_ptr()
        h = C.c_void_p()
        check(lib().ceep3d_adjoint_create(s._plan, C.addressof(d), C.byref(h)), "ceep3d_adjoint_create")
        starts = sorted(self._starts, reverse=True)
        M = len(self._kept)
        overlap = self.overlap
        if overlap is None:
            overlap = len(self._segs) >= 2 or torch.cuda.mem_get_info(dev)[0] > 2 * self.segment_bytes()
        two = bool(overlap) and len(starts) > M
        nbuf = max(M, 2 if two else 1)
        self._buffers(nbuf)

        def recompute(a, buf):
            self._restore(a)
            # the recompute skips the CPML shell, which no saved value depends on
            self._run_save(a, min(a + K, T), buf, interior_only=True)

        def adjoint(a, buf):
            st = torch.cuda.current_stream(dev)
            b = min(a + K, T)
            check(lib().ceep3d_adjoint_run(h, b, b - a, self._segs[buf].data_ptr(), a, C.c_void_p(st.cuda_stream)),
                  "ceep3d_adjoint_run")
        try:
            run_segments_backward(starts, self._kept, recompute, adjoint, dev, two, nbuf)
        finally:
            self._kept = set()
            lib().ceep3d_adjoint_destroy(h)
        full = torch.zeros((ks, s.nz, s.ny, s.nx), dtype=torch.float64, device=dev)
        full[:, n + 1:s.nz - n, n + 1:s.ny - n, n + 1:s.nx - n] = grad.sum(0)
        res = self._chain(full.permute(0, 3, 2, 1))           # (ks, nx, ny, nz)
        return allreduce_gradient(res) if self.reduce_ranks else res

    def _chain(self, grad):
        """Coefficient gradients -> parameter gradients, all (nx, ny, nz)."""
        eps_r, sigma, debye = self._params
        inputs = [eps_r.detach().requires_grad_(True), sigma.detach().requires_grad_(True)]
        deb = [(de.detach().requires_grad_(True), tau.detach()) for de, tau in debye]
        inputs += [de for de, _ in deb]
        with torch.enable_grad():
            ca, cb, _, poles = coefficient_maps(inputs[0], inputs[1], deb, self.s.dt)
            outs = [ca, cb] + [k2 for _, k2, _ in poles]
            grads = torch.autograd.grad(outs, inputs, list(grad[:len(outs)]), allow_unused=True)
        grads = [torch.zeros_like(x) if gr is None else gr for gr, x in zip(grads, inputs)]
        res = {"eps_r": grads[0], "sigma": grads[1]}
        if deb:
            res["deps"] = grads[2]
        return res


class FDTD3DProbes(torch.autograd.Function):
    """probes = FDTD3DProbes.apply(eps_r, sigma, deps, tau, adjoint): the probe
    series of an ``Adjoint3D``'s solver as a differentiable function of the
    (nx, ny, nz) maps (tau is held fixed)."""

    @staticmethod
    def forward(ctx, eps_r, sigma, deps, tau, adjoint: Adjoint3D):
        adjoint.set_parameters(eps_r, sigma, deps, tau)
        ctx.adjoint = adjoint
        ctx.has_deps = deps is not None
        return adjoint.forward()

    @staticmethod
    def backward(ctx, grad_probes):
        g = ctx.adjoint.backward(grad_probes.contiguous())
        return g["eps_r"], g["sigma"], (g.get("deps") if ctx.has_deps else None), None, None


def probes_with_grad_3d(eps_r, sigma, adjoint: Adjoint3D, deps=None, tau=None):
    return FDTD3DProbes.apply(eps_r, sigma, deps, tau, adjoint)
