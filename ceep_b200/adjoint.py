"""Checkpointed adjoint of the batched 2D solver and its torch.autograd.Function.

The reference announces a differentiable solver but implements none
(src/ceep/ai/__init__.py is a docstring).  Here the gradient of a loss on the
probe series with respect to the per-cell eps_r, sigma and Debye delta_eps
maps comes from the exact discrete adjoint of the fused forward step
(``csrc/adjoint2d.cu``), run backwards in time:

* the forward pass stores the full state every ``checkpoint_every`` steps
  and runs its last segment with the save on;
* for each other segment, last first, the state is restored and the segment
  recomputed while the step kernel saves Ez (and, for tau gradients, the
  Debye currents) of every step; the transposed steps run back over each
  segment, accumulating d(loss)/d of the per-cell update coefficients
  (ca, cb, k2, and k1, gamma with ``grad_tau``) in FP64.  The recompute of
  the next segment overlaps the adjoint of the current one on a second
  stream (``overlap``, two segment buffers);
* the chain rule from those coefficients to (eps_r, sigma, delta_eps) runs in
  torch FP64 through the same coefficient formulas as the forward
  (src/ceep/solvers/fdtd_2d_batched.py:151-167, src/ceep/materials/dispersive.py:253-261).

``checkpoint_every=1`` keeps every step (no recompute) when memory allows.
Gradients are defined on the interior E region, where the coefficients act.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import torch

from ._lib import check, lib
from .constants import EPS_0
from .distributed import allreduce_gradient
from .physics import rdiv
from .solvers import BatchedFDTD2D, _ptr


class _AdjDesc(C.Structure):
    P = C.c_void_p
    _fields_ = [("ez", P * 2), ("hx", P * 2), ("hy", P * 2), ("psi_hx", P * 2), ("psi_hy", P * 2),
                ("psi_ezx", P * 2), ("psi_ezy", P * 2), ("j", P * 2), ("jp", P * 2), ("grad", P),
                ("probe_grad", P), ("grad_tau", C.c_int32)]


def grad_width(poles: int) -> int:
    """Per-cell gradient slots of the adjoint: 2 + 3 per pole, rounded up to even."""
    return (2 + 3 * poles + 1) // 2 * 2


def coefficient_maps(eps_r, sigma, debye, dt, lorentz=()):
    """Differentiable (ca, cb, dt/(eps_r eps0), poles) from (nx, ny) FP64 maps;
    poles: Debye (k1, k2, gamma), then Lorentz (k1, k2, k3)
    (dispersive.py:253-261, :278-299)."""
    eps = eps_r * EPS_0
    poles = []
    for de, tau in debye:
        valid = tau > 0
        den = 2.0 * tau + dt
        z = torch.zeros_like(tau)
        k1 = torch.where(valid, (2.0 * tau - dt) / den, z)
        k2 = torch.where(valid, 2.0 * EPS_0 * de * dt / den, z)
        g = torch.where(valid, (1.0 + k1) / 2.0, z)
        eps = eps + k2 / 2.0
        poles.append((k1, k2, g))
    for de, w0, dl in lorentz:
        valid = w0 > 0
        w02, dt2 = w0 * w0, dt * dt
        den = 4.0 + 2.0 * dl * dt + w02 * dt2
        z = torch.zeros_like(w0)
        k1 = torch.where(valid, (8.0 - 2.0 * w02 * dt2) / den, z)
        k3 = torch.where(valid, -(4.0 - 2.0 * dl * dt + w02 * dt2) / den, z)
        k2 = torch.where(valid, 2.0 * EPS_0 * de * w02 * dt2 / den, z)
        eps = eps + k2 / 2.0
        poles.append((k1, k2, k3))
    s = sigma * dt / (2.0 * eps)
    return (1.0 - s) / (1.0 + s), rdiv(dt, eps) / (1.0 + s), rdiv(dt, eps_r * EPS_0), poles


def run_segments_backward(starts, kept, recompute, adjoint, device, overlap, nbuf):
    """Drive the segments of a checkpointed adjoint, last first.

    ``starts`` are the segment starts in descending order; the i-th of them
    uses segment buffer ``i % nbuf``.  ``kept`` is the set of starts whose
    slots the forward pass already left in their buffers (the last segments:
    indices 0 .. len(kept)-1, so ``nbuf >= len(kept)``); every other segment
    is recomputed.  ``recompute(a, buf)`` enqueues, on the current stream, the
    restore of checkpoint ``a`` and the saving recompute of its segment into
    buffer ``buf``; ``adjoint(a, buf)`` enqueues the transposed steps of that
    segment reading buffer ``buf``.  With ``overlap`` (``nbuf >= 2``) the
    recompute of the next segment runs on a second stream while the adjoint
    of the current one runs on a high-priority stream: the two are
    independent (different state, different buffers), and neither saturates
    the GPU alone at these sizes.  Events order each buffer's reuse; the
    caller's stream waits for both at the end."""
    assert nbuf >= max(1, len(kept)) and all(a in kept for a in starts[:len(kept)])
    if not overlap:
        for i, a in enumerate(starts):
            if a not in kept:
                recompute(a, i % nbuf)
            adjoint(a, i % nbuf)
        return
    assert nbuf >= 2
    main = torch.cuda.current_stream(device)
    adj_s = torch.cuda.Stream(device, priority=-1)
    rec_s = torch.cuda.Stream(device)
    adj_s.wait_stream(main)
    rec_s.wait_stream(main)
    freed = [None] * nbuf
    ready = {}

    def issue(i):
        buf = i % nbuf
        if freed[buf] is not None:
            rec_s.wait_event(freed[buf])
        with torch.cuda.stream(rec_s):
            recompute(starts[i], buf)
        ready[i] = rec_s.record_event()

    if starts[0] not in kept:
        issue(0)
    for i, a in enumerate(starts):
        if i + 1 < len(starts) and starts[i + 1] not in kept:
            issue(i + 1)
        if i in ready:
            adj_s.wait_event(ready[i])
        with torch.cuda.stream(adj_s):
            adjoint(a, i % nbuf)
        freed[i % nbuf] = adj_s.record_event()
    main.wait_stream(adj_s)
    main.wait_stream(rec_s)


class Adjoint2D:
    """Gradient driver for one ``BatchedFDTD2D`` with at most one Debye pole
    and any Lorentz poles (two poles in all).

    ``grad_tau`` adds d(loss)/d(tau) for a Debye pole.  Without it tau is held
    fixed: the update coefficients k1 and gamma depend on tau alone, so their
    gradients are never formed and the forward pass does not keep the Debye
    currents of every step (one field less to write and read).  Lorentz poles
    are differentiated in delta_eps; omega_0 and delta are held fixed (k1 and
    k3 depend on them alone)."""

    def __init__(self, solver: BatchedFDTD2D, checkpoint_every: int = 50, grad_tau: bool = False,
                 overlap: bool = True, keep_bytes: int = 0, reduce_ranks: bool = False, rows: int = 0):
        """``reduce_ranks``: the solver holds this rank's transmit events only
        (``distributed.split_sources``) and the loss covers those; the
        gradient maps are summed over ranks (one all_reduce each), so every
        rank returns the gradient of the whole loss."""
        if len(solver._debye) > 1:
            raise ValueError("the adjoint supports one Debye pole (and Lorentz poles)")
        self.s = solver
        self.K = max(1, int(checkpoint_every))
        self.grad_tau = bool(grad_tau)
        self.overlap = bool(overlap)
        self.keep_bytes = max(0, int(keep_bytes))
        self.reduce_ranks = bool(reduce_ranks)
        self.rows = max(0, int(rows))   # tile height of the adjoint launch (0: automatic)
        self._kept = set()
        self.launch_rows = None         # tile rows of the adjoint launch (reported by the library)
        self._params = None
        self._ckpt = {}

    # -- parameters -------------------------------------------------------------
    def set_parameters(self, eps_r: torch.Tensor, sigma: torch.Tensor, deps=None, tau=None,
                       lorentz_deps=()) -> None:
        """(nx, ny) maps in the reference's axis order; ``deps``/``tau`` are the
        Debye maps of the solver's single Debye pole when it has one, and
        ``lorentz_deps`` the delta_eps maps of its Lorentz poles (their
        omega_0 and delta maps are the solver's own)."""
        s = self.s
        dev = s.device
        f64 = lambda t: torch.as_tensor(t, dtype=torch.float64).to(dev)
        eps_r, sigma = f64(eps_r), f64(sigma)
        debye = []
        if s._debye:
            debye = [(f64(deps), f64(tau))]
        if len(lorentz_deps) != len(s._lorentz):
            raise ValueError(f"{len(s._lorentz)} Lorentz delta_eps maps expected")
        lorentz = [(f64(d), f64(w0), f64(dl)) for d, (_, w0, dl) in zip(lorentz_deps, s._lorentz)]
        self._params = (eps_r, sigma, debye, lorentz)
        if not s._built:
            s._build()
        ca, cb, dteps, poles = coefficient_maps(eps_r, sigma, debye, s.dt, lorentz)
        coef = torch.stack([ca, cb, dteps, torch.zeros_like(ca)], -1).transpose(0, 1)   # (ny, nx, 4)
        s._coef.copy_(coef.to(torch.float32))
        if poles:
            ade = torch.stack([torch.stack([a, b, c, torch.zeros_like(a)], -1).transpose(0, 1)
                               for a, b, c in poles])
            s._ade_coef.copy_(ade.to(torch.float32))

    # -- forward with checkpoints ---------------------------------------------------
    def _state(self):
        s = self.s
        cur = s._cur()
        st = {"ez": s._ez[cur], "hx": s._hx[cur], "hy": s._hy[cur], "psi_hy": s._psi_hy[cur],
              "psi_hx": s._psi_hx[cur], "psi_ezx": s._psi_ezx[cur], "psi_ezy": s._psi_ezy[cur]}
        if s._j is not None:
            st["j"] = s._j[cur]
        if s._j_prev is not None:
            st["j_prev"] = s._j_prev[cur]
        return st

    def _seglen(self):
        return self.s.total_steps if self.K == 1 else min(self.K, self.s.total_steps)

    def segment_bytes(self):
        """Device bytes of one segment buffer (the Ez slots, plus the J slots
        when tau gradients are asked for)."""
        s = self.s
        n = (self._seglen() + 1) * s._groups * s.ny * s.nx * s._gwidth
        if s._j is not None and self.grad_tau:
            n += (self._seglen() + 1) * s._j[0].numel()
        return 4 * n

    def kept_segments(self, nseg):
        """How many trailing segments the forward pass keeps: the last one
        always, more while their buffers fit in ``keep_bytes``."""
        return max(1, min(nseg, self.keep_bytes // max(1, self.segment_bytes())))

    def _buffers(self, count):
        """`count` segment buffers (Ez slots, J slots or None), allocated once:
        the saving graphs are keyed on their addresses."""
        s = self.s
        G, W = s._groups, s._gwidth
        slots = self._seglen() + 1
        segs = getattr(self, "_segs", [])
        while len(segs) < count:
            seg_ez = torch.empty((slots, G, s.ny, s.nx, W), dtype=torch.float32, device=s.device)
            seg_j = (torch.zeros((slots,) + tuple(s._j[0].shape), dtype=torch.float32, device=s.device)
                     if s._j is not None and self.grad_tau else None)
            segs.append((seg_ez, seg_j))
        self._segs = segs
        return segs

    def forward(self) -> torch.Tensor:
        """Run all steps from a zero state, keeping checkpoints; returns the probe
        series (ntx, nprobe, T) float32 on the device.  The last segments (the
        last one, and more within ``keep_bytes``) run with the save on into
        their own buffers, so the backward pass never recomputes them; the
        others start from a checkpoint of the full state."""
        s = self.s
        s.reset()
        T, L = s.total_steps, self._seglen()
        self._ckpt = {}
        starts = list(range(0, T, L))
        M = self.kept_segments(len(starts))
        self._buffers(M)
        stream = torch.cuda.current_stream(s.device)
        self._starts, self._kept = starts, set()
        for j, a in enumerate(starts):
            b = min(a + L, T)
            i = len(starts) - 1 - j                 # index in the backward order
            if i < M:
                self._run_save(a, b, i)
                self._kept.add(a)
            else:
                self._ckpt[a] = {k: v.clone() for k, v in self._state().items()}
                s.advance(a, b - a, stream=stream)
        return s.probe_data[:, :len(s.probe_positions)].clone()

    def _restore(self, a):
        s = self.s
        ck = self._ckpt[a]
        s._ez[0].copy_(ck["ez"]); s._hx[0].copy_(ck["hx"]); s._hy[0].copy_(ck["hy"])
        s._psi_hy[0].copy_(ck["psi_hy"]); s._psi_hx[0].copy_(ck["psi_hx"])
        s._psi_ezx[0].copy_(ck["psi_ezx"]); s._psi_ezy[0].copy_(ck["psi_ezy"])
        if "j" in ck:
            s._j[0].copy_(ck["j"])
        if "j_prev" in ck:
            s._j_prev[0].copy_(ck["j_prev"])
        check(lib().ceep2d_plan_set_current_buffer(s._plan, 0), "ceep2d_plan_set_current_buffer")

    def _run_save(self, a, b, buf):
        """Run [a, b) from the current state on the current stream, saving Ez
        (and, for tau gradients, J) of every step into buffer `buf`."""
        s = self.s
        seg_ez, seg_j = self._segs[buf]
        cur = s._cur()
        seg_ez[0].copy_(s._ez[cur])
        if seg_j is not None:
            seg_j[0].copy_(s._j[cur])
        stream = torch.cuda.current_stream(s.device)
        check(lib().ceep2d_plan_run_save(s._plan, a, b - a, C.c_void_p(stream.cuda_stream), int(s.use_graph),
                                         seg_ez.data_ptr(), _ptr(seg_j), a), "ceep2d_plan_run_save")

    # -- backward ------------------------------------------------------------------
    def backward(self, grad_probes: torch.Tensor):
        """d(loss)/d(eps_r, sigma, delta_eps) given d(loss)/d(probe series)."""
        s = self.s
        dev = s.device
        T, L = s.total_steps, self._seglen()
        G, W = s._groups, s._gwidth
        f32 = dict(dtype=torch.float32, device=dev)
        adj = self._adjoint_state()
        nd, nl = len(s._debye), len(s._lorentz)
        kp = grad_width(nd + nl)
        grad = torch.zeros((G, s.ny, s.nx, kp), dtype=torch.float64, device=dev)
        gp = torch.zeros((s.batch, max(len(s.probe_positions), 1), T), **f32)
        gp[:, :grad_probes.shape[1]] = grad_probes.to(torch.float32)
        d = _AdjDesc()
        for name, bufs in adj.items():
            arr = getattr(d, name)
            arr[0], arr[1] = _ptr(bufs[0]), _ptr(bufs[1])
        d.grad, d.probe_grad = grad.data_ptr(), gp.data_ptr()
        d.grad_tau = int(self.grad_tau)
        starts = sorted(self._starts, reverse=True)
        M = len(self._kept)
        two = self.overlap and len(starts) > M
        nbuf = max(M, 2 if two else 1)
        self._buffers(nbuf)
        h = C.c_void_p()
        check(lib().ceep2d_adjoint_create(s._plan, C.addressof(d), C.byref(h)), "ceep2d_adjoint_create")
        if self.rows:
            check(lib().ceep2d_adjoint_set_rows(h, self.rows), "ceep2d_adjoint_set_rows")
        self.launch_rows = lib().ceep2d_adjoint_rows(h)

        def recompute(a, buf):
            self._restore(a)
            self._run_save(a, min(a + L, T), buf)

        def adjoint(a, buf):
            seg_ez, seg_j = self._segs[buf]
            st = torch.cuda.current_stream(dev)
            check(lib().ceep2d_adjoint_run(h, min(a + L, T), min(a + L, T) - a, seg_ez.data_ptr(), _ptr(seg_j), a,
                                           C.c_void_p(st.cuda_stream)), "ceep2d_adjoint_run")
        try:
            run_segments_backward(starts, self._kept, recompute, adjoint, dev, two, nbuf)
        finally:
            self._kept = set()
            lib().ceep2d_adjoint_destroy(h)
        # (G, ny, nx, KP) per TX group -> (2 + 3 poles, ny, nx)
        res = self._chain(grad.sum(0).permute(2, 0, 1)[:2 + 3 * (nd + nl)])
        return allreduce_gradient(res) if self.reduce_ranks else res

    def _adjoint_state(self):
        """The adjoint state, every array a ping-pong pair shaped like the
        forward's: views of one flat buffer kept while the layout stays, zeroed
        with one fill per backward."""
        s = self.s
        specs = [("ez", s._ez[0]), ("hx", s._hx[0]), ("hy", s._hy[0]), ("psi_hx", s._psi_hx[0]),
                 ("psi_hy", s._psi_hy[0]), ("psi_ezx", s._psi_ezx[0]), ("psi_ezy", s._psi_ezy[0]),
                 ("j", s._j[0] if s._j is not None else None),
                 ("jp", s._j_prev[0] if s._j_prev is not None else None)]
        key = tuple((name, None if t is None else (tuple(t.shape), t.dtype)) for name, t in specs)
        if getattr(self, "_adj_key", None) != key:
            total = sum(2 * t.numel() for _, t in specs if t is not None)
            flat = torch.empty(max(total, 1), dtype=torch.float32, device=s.device)
            bufs, off = {}, 0
            for name, t in specs:
                if t is None:
                    bufs[name] = [None, None]
                    continue
                bufs[name] = []
                for _ in range(2):  # every size is a multiple of 4 floats, so every view stays 16-byte aligned
                    bufs[name].append(flat[off:off + t.numel()].view(t.shape))
                    off += t.numel()
            self._adj_flat, self._adj_bufs, self._adj_key = flat, bufs, key
        self._adj_flat.zero_()
        return self._adj_bufs

    def _chain(self, grad):
        """Coefficient gradients (ny, nx) -> parameter gradients (nx, ny)."""
        eps_r, sigma, debye, lorentz = self._params
        inputs = [eps_r.detach().requires_grad_(True), sigma.detach().requires_grad_(True)]
        deb = [(de.detach().requires_grad_(True), tau.detach().requires_grad_(self.grad_tau)) for de, tau in debye]
        lor = [(de.detach().requires_grad_(True), w0, dl) for de, w0, dl in lorentz]
        inputs += [de for de, _ in deb]
        if self.grad_tau:
            inputs += [tau for _, tau in deb]
        inputs += [de for de, _, _ in lor]
        with torch.enable_grad():
            ca, cb, _, poles = coefficient_maps(inputs[0], inputs[1], deb, self.s.dt, lor)
            outs = [ca, cb]
            gouts = [grad[0].t(), grad[1].t()]
            for q, pole in enumerate(poles):
                if q < len(deb):      # Debye: k1, k2, gamma
                    outs += list(pole)
                    gouts += [grad[2 + 3 * q].t(), grad[3 + 3 * q].t(), grad[4 + 3 * q].t()]
                else:                 # Lorentz: only k2 depends on delta_eps
                    outs.append(pole[1])
                    gouts.append(grad[3 + 3 * q].t())
            # without grad_tau, k1 and gamma depend on fixed inputs only
            keep = [i for i, o in enumerate(outs) if o.requires_grad]
            grads = torch.autograd.grad([outs[i] for i in keep], inputs, [gouts[i] for i in keep],
                                        allow_unused=True)
        grads = [torch.zeros_like(x) if gr is None else gr for gr, x in zip(grads, inputs)]
        res = {"eps_r": grads[0], "sigma": grads[1]}
        k = 2
        if deb:
            res["deps"] = grads[2]
            k = 3
            if self.grad_tau:
                res["tau"] = grads[3]
                k = 4
        if lor:
            res["lorentz_deps"] = list(grads[k:k + len(lor)])
        return res


class FDTD2DProbes(torch.autograd.Function):
    """probes = FDTD2DProbes.apply(eps_r, sigma, deps, tau, adjoint, *lorentz_deps):
    the probe series of an ``Adjoint2D``'s solver as a differentiable function
    of the (nx, ny) maps; ``deps``/``tau`` may be None for a solver without a
    Debye pole, and ``lorentz_deps`` are the delta_eps maps of its Lorentz poles."""

    @staticmethod
    def forward(ctx, eps_r, sigma, deps, tau, adjoint: Adjoint2D, *lorentz_deps):
        adjoint.set_parameters(eps_r, sigma, deps, tau, lorentz_deps)
        ctx.adjoint = adjoint
        ctx.has_deps = deps is not None
        ctx.n_lorentz = len(lorentz_deps)
        return adjoint.forward()

    @staticmethod
    def backward(ctx, grad_probes):
        g = ctx.adjoint.backward(grad_probes.contiguous())
        lor = tuple(g.get("lorentz_deps", [None] * ctx.n_lorentz))
        return (g["eps_r"], g["sigma"], g.get("deps") if ctx.has_deps else None,
                g.get("tau") if ctx.has_deps else None, None) + lor


def probes_with_grad(eps_r, sigma, adjoint: Adjoint2D, deps=None, tau=None, lorentz_deps=()):
    return FDTD2DProbes.apply(eps_r, sigma, deps, tau, adjoint, *lorentz_deps)


_LOSS_TWIDDLES = {}  # (frequencies, T, dt, device) -> (F, T) complex128 DFT weights; a few entries


def _loss_twiddles(frequencies, T: int, dt: float, device) -> torch.Tensor:
    import math
    import numpy as np
    f = np.ascontiguousarray(np.asarray(frequencies, np.float64))
    key = (f.tobytes(), int(T), float(dt), str(device))
    tw = _LOSS_TWIDDLES.get(key)
    if tw is None:
        if len(_LOSS_TWIDDLES) >= 8:
            _LOSS_TWIDDLES.pop(next(iter(_LOSS_TWIDDLES)))
        w = 2.0 * math.pi * torch.as_tensor(f, dtype=torch.float64, device=device)
        ph = w[:, None] * (torch.arange(T, dtype=torch.float64, device=device) * dt)[None, :]
        tw = torch.complex(torch.cos(ph) * dt, -torch.sin(ph) * dt)
        _LOSS_TWIDDLES[key] = tw
    return tw


def s_parameter_loss(probes: torch.Tensor, dt: float, frequencies, target: torch.Tensor):
    """L = sum |S - S*|^2 over S[f, rx, tx] = sum_n probe[tx, rx, n] e^{-j w n dt} dt
    (the running DFT of src/ceep/solvers/dft.py:55-90); returns (L, S).  The
    DFT weights are built once per (frequencies, T, dt) and kept."""
    tw = _loss_twiddles(frequencies, probes.shape[-1], dt, probes.device)
    S = torch.einsum("bpt,ft->fpb", probes.to(torch.complex128), tw)
    return (S - target).abs().pow(2).sum(), S
