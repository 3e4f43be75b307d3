"""ε-gradients of plane-DFT objectives by the discrete adjoint of the Yee/CPML step.

The reference solver (r-bridge/opencl-fdtd-solver) has no gradient.  This module adds
one on top of :class:`CUDAFDTD` without changing the forward path:

* ``EpsilonAdjoint.forward(eps_design)`` sets ``εr`` (background outside the design
  box), runs ``n_steps`` from rest with the engine's registered sources, accumulates
  a plane DFT on the objective plane (the same kernel and phase recurrence as
  :class:`CUDAPlaneDFTMonitor`, reference ``monitors.py:571-584``), evaluates
  ``J = fn(D)`` on the patch.  The sweep needs the forward ``E`` over the design's
  edge box at every step (``fdtd_capture_box``).  When all ``n_steps + 1`` boxes
  fit the capture budget (a quarter of the free device memory by default; 5.8 GB
  for a 96×96×16 design over 3000 steps), the forward pass captures them all;
  otherwise it keeps a checkpoint of the full state every ``checkpoint_every``
  steps (fields and ψ stripes: ``CUDAFDTD.save_state``) for replay.
* ``backward()`` runs the adjoint sweep: ``∂J/∂D`` (by torch autograd through ``fn``)
  seeds ``Ē`` on the patch each step (``fdtd_adjoint_seed_add`` / the seed of
  ``fdtd_adjoint_step``) and the transposed step runs backwards in time
  (``fdtd_adjoint_step``), accumulating ``Σ_n Ē^{n+1}·(E^{n+1} − E^n) = ce·∂J/∂ce``
  on the edge box in float64.  With checkpoints, segments are replayed newest
  first with ``E`` captured each step, and the sweep through a segment runs on a
  second stream, concurrently with the replay of the next-older segment (two
  capture buffers, ordered by events).  The host chain rule through
  ``ce = dt/(ε0·ε_edge)`` and the two-cell edge average (reference
  ``materials.py:28-56``) gives ``∂J/∂εr`` per design cell.
* :class:`EpsilonObjective` wraps the pair as a ``torch.autograd.Function``.

The gradient is exact for the discrete scheme (lossless grids: ``set_epsilon``
without σ) and the same bit for bit in both capture modes; its cost is one
forward solve and one adjoint sweep, plus one replayed forward solve in the
checkpoint mode.
"""

from __future__ import annotations

import ctypes

import numpy as np
import torch

from . import _capi as capi
from .engine import CUDAFDTD
from .monitors import CUDAPlaneDFTMonitor

E_NAMES = ("Ex", "Ey", "Ez")


def _default_fn(D):
    return (D.real ** 2 + D.imag ** 2).sum()


class DFTObjective:
    """``J = fn(D)`` of the plane DFT ``D`` over a patch.

    axis, index : the plane (``axis`` 0/1/2 or 'x'/'y'/'z')
    patch       : ``((a0, a1), (b0, b1))`` half-open ranges over the two other axes
                  in x, y, z order
    freqs       : DFT frequencies (Hz)
    components  : E components (``'Ex'``, ``'Ey'``, ``'Ez'``)
    fn          : differentiable torch function of the complex128 tensor
                  ``D[component][freq][a][b]`` returning a real scalar; default
                  ``Σ|D|²``
    """

    def __init__(self, axis, index, patch, freqs, components=("Ex",), fn=None):
        self.axis = {"x": 0, "y": 1, "z": 2}.get(axis, axis)
        if self.axis not in (0, 1, 2):
            raise ValueError(f"axis must be 0, 1, 2 or 'x', 'y', 'z'; got {axis!r}")
        self.index = int(index)
        (a0, a1), (b0, b1) = patch
        self.patch = ((int(a0), int(a1)), (int(b0), int(b1)))
        self.freqs = np.atleast_1d(np.asarray(freqs, dtype=np.float64))
        if not 0 < self.freqs.size <= capi.FDTD_MAX_FREQS:
            raise ValueError(f"1 to {capi.FDTD_MAX_FREQS} frequencies, got {self.freqs.size}")
        comps = (components,) if isinstance(components, str) else tuple(components)
        for c in comps:
            if c not in E_NAMES:
                raise ValueError(f"objective components must be E components, got {c!r}")
        self.components = tuple(c for c in E_NAMES if c in comps)
        self.comp_mask = sum(1 << E_NAMES.index(c) for c in self.components)
        self.fn = _default_fn if fn is None else fn


def _phase_sequence(freqs, dt, n_steps, t_first):
    """E phases of the plane DFT per step (complex128 ``(n_steps, nfreq)``), with the
    recurrence of ``CUDAPlaneDFTMonitor``: ``e^{jωt_first}·dt``, then ``·e^{jωdt}``."""
    omega = 2.0 * np.pi * np.asarray(freqs, np.float64)
    d = np.exp(1j * omega * float(dt))
    out = np.empty((int(n_steps), omega.size), np.complex128)
    p = np.exp(1j * omega * float(t_first)) * float(dt)
    for n in range(int(n_steps)):
        if n > 0:
            p = p * d
        out[n] = p
    return out


def _edge_eps(eps):
    ex = eps.copy()
    ex[:-1] = 0.5 * (eps[:-1] + eps[1:])
    ey = eps.copy()
    ey[:, :-1] = 0.5 * (eps[:, :-1] + eps[:, 1:])
    ez = eps.copy()
    ez[:, :, :-1] = 0.5 * (eps[:, :, :-1] + eps[:, :, 1:])
    return ex, ey, ez


def edge_to_cells(G, eps_full, design, box):
    """``ce·∂J/∂ce`` on the edge box (``G[3][box]``) → ``∂J/∂εr`` per design cell.

    ``ce = dt/(ε0·ε_edge)`` gives ``∂J/∂ε_edge = −G/ε_edge``; ``ε_edge`` is the mean of
    the two cells sharing the edge, the last plane keeping the cell value
    (reference ``materials.py:28-41``), so each cell collects half of its two edges
    along each axis (all of the last-plane edge).
    """
    eps_e = _edge_eps(eps_full)
    shape = eps_full.shape
    bsl = tuple(slice(lo, hi) for lo, hi in box)
    dsl = tuple(slice(lo, hi) for lo, hi in design)
    out = np.zeros(tuple(hi - lo for lo, hi in design), np.float64)
    for c in range(3):
        ge = np.zeros(shape, np.float64)
        ge[bsl] = -G[c] / eps_e[c][bsl]
        n = shape[c]
        cell = np.zeros(shape, np.float64)
        dst = [slice(None)] * 3
        src = [slice(None)] * 3
        dst[c] = slice(0, n - 1)
        cell[tuple(dst)] += 0.5 * ge[tuple(dst)]      # edge i   -> cell i
        dst[c] = slice(1, n)
        src[c] = slice(0, n - 1)
        cell[tuple(dst)] += 0.5 * ge[tuple(src)]      # edge i-1 -> cell i
        dst[c] = slice(n - 1, n)
        cell[tuple(dst)] += ge[tuple(dst)]            # last plane
        out += cell[dsl]
    return out


class EpsilonAdjoint:
    """Objective and discrete-adjoint gradient with respect to ``εr`` in a design box.

    fdtd             : a :class:`CUDAFDTD` with its sources registered (source
                       callbacks must depend only on ``fdtd.t``: segments are replayed)
    design           : ``((i0, i1), (j0, j1), (k0, k1))`` half-open design box
    n_steps          : time steps per solve (from rest at t = 0)
    objective        : :class:`DFTObjective`
    eps_background   : cell-centred ``εr`` outside the design box (default 1)
    checkpoint_every : steps per replayed segment (K) in the checkpoint mode
    capture          : ``"auto"`` (default): keep the forward ``E`` over the edge box
                       for every step when that fits ``capture_budget`` bytes, else
                       checkpoint and replay; ``"all"`` or ``"replay"`` force a mode
    capture_budget   : bytes the ``"auto"`` mode may hold (default: a quarter of the
                       device memory free at the forward call)
    fused_reverse    : True runs each reverse step as the TMA plane march over the
                       CPML-free interior plus CPML-shell kernels, reading one Ē/H̄
                       buffer pair and writing the other; False (default) updates Ē/H̄
                       in place with one thread per cell, measured faster at the
                       shell-heavy 160 x 160 x 96 configuration (143 against 152 µs per
                       reverse step).  Both give the same gradient bit for bit.

    The engine's own monitors are detached while this object steps it.
    """

    def __init__(self, fdtd, design, n_steps, objective, *, eps_background=None,
                 checkpoint_every=100, capture="auto", capture_budget=None,
                 fused_reverse=False):
        if not isinstance(fdtd, CUDAFDTD):
            raise TypeError("EpsilonAdjoint needs a CUDAFDTD engine")
        self.fdtd = fdtd
        shape = (fdtd.Nx, fdtd.Ny, fdtd.Nz)
        self.design = tuple((int(lo), int(hi)) for lo, hi in design)
        if len(self.design) != 3 or any(not (0 <= lo < hi <= n)
                                        for (lo, hi), n in zip(self.design, shape)):
            raise ValueError(f"design box {design} is empty or outside the grid {shape}")
        self.n_steps = int(n_steps)
        if self.n_steps < 1:
            raise ValueError("n_steps must be >= 1")
        self.K = int(checkpoint_every)
        if self.K < 1:
            raise ValueError("checkpoint_every must be >= 1")
        if capture not in ("auto", "all", "replay"):
            raise ValueError(f"capture must be 'auto', 'all' or 'replay', got {capture!r}")
        self.capture = capture
        self.fused_reverse = bool(fused_reverse)
        self.capture_budget = None if capture_budget is None else int(capture_budget)
        if not isinstance(objective, DFTObjective):
            raise TypeError("objective must be a DFTObjective")
        self.objective = objective
        o = objective
        dims = list(shape)
        if not 0 <= o.index < dims[o.axis]:
            raise ValueError(f"objective plane index {o.index} outside [0, {dims[o.axis]})")
        del dims[o.axis]
        (a0, a1), (b0, b1) = o.patch
        if not (0 <= a0 < a1 <= dims[0] and 0 <= b0 < b1 <= dims[1]):
            raise ValueError(f"objective patch {o.patch} is empty or outside the plane {dims}")
        if eps_background is None:
            self.eps_background = np.ones(shape, np.float64)
        else:
            self.eps_background = np.array(eps_background, dtype=np.float64)
            if self.eps_background.shape != shape:
                raise ValueError(f"eps_background shape {self.eps_background.shape} != {shape}")
        # edge box: every edge a design cell's ε reaches
        self.box = tuple((max(0, lo - 1), hi) for lo, hi in self.design)
        self.box_shape = tuple(hi - lo for lo, hi in self.box)
        self._ckpts = None
        self._cap_all = None   # (n_steps + 1, 3, box) forward E, in the capture-all mode
        self._captured = False
        self._seed = None
        self.J = None
        self.D = None

    # ----------------------------------------------------------------- forward
    def _eps_full(self, eps_design):
        eps = np.asarray(eps_design, dtype=np.float64)
        want = tuple(hi - lo for lo, hi in self.design)
        if eps.shape != want:
            raise ValueError(f"eps_design shape {eps.shape} != design box shape {want}")
        full = self.eps_background.copy()
        full[tuple(slice(lo, hi) for lo, hi in self.design)] = eps
        return full

    def forward(self, eps_design):
        """Solve with ``εr = eps_design`` in the design box; return ``J`` (float)."""
        fd = self.fdtd
        o = self.objective
        self._eps = self._eps_full(eps_design)
        fd.set_epsilon(self._eps)
        fd.reset_state()
        capture_all = self._capture_all()
        saved = fd._monitors
        fd._monitors = []
        ckpts = []
        try:
            mon = CUDAPlaneDFTMonitor(fd, o.axis, o.index, o.freqs, o.components)
            self._t_first = fd.t + fd.dt
            if capture_all:
                grid, st = fd._grid, fd.queue.cuda_stream
                lo = (ctypes.c_int32 * 3)(*[b[0] for b in self.box])
                hi = (ctypes.c_int32 * 3)(*[b[1] for b in self.box])
                cap0 = self._cap_all.data_ptr()
                slot = self._cap_all[0].numel() * self._cap_all.element_size()

                eptrs = {}  # E pointer arrays by buffer parity (the step ping-pongs E)

                def grab(m):
                    Ep = eptrs.get(fd._parity)
                    if Ep is None:
                        Ep = eptrs[fd._parity] = (ctypes.c_void_p * 3)(
                            *[t.data_ptr() for t in fd._E])
                    capi.run("fdtd_capture_box", grid, Ep, lo, hi, cap0 + m * slot, st)

                grab(0)
                for n in range(self.n_steps):
                    fd.step()
                    grab(n + 1)
            else:
                for n in range(self.n_steps):
                    if n % self.K == 0:
                        ckpts.append(fd.save_state())
                    fd.step()
        finally:
            fd._monitors = saved
        self._captured = capture_all
        self._ckpts = ckpts
        (a0, a1), (b0, b1) = o.patch
        D = torch.view_as_complex(mon.acc)[:, :, a0:a1, b0:b1].detach().clone()
        Dg = D.clone().requires_grad_(True)
        with torch.enable_grad():
            J = o.fn(Dg)
            (seed,) = torch.autograd.grad(J, Dg)
        self._seed = torch.view_as_real(seed.detach().to(torch.complex128)).contiguous()
        self.D = D
        self.J = float(J.detach())
        return self.J

    def _capture_all(self):
        """Whether this forward keeps E over the edge box for every step; allocates
        (or reuses) the buffer when it does."""
        fd = self.fdtd
        shape = (self.n_steps + 1, 3, *self.box_shape)
        nbytes = int(np.prod(shape)) * np.dtype(fd.dtype).itemsize
        if self.capture == "replay":
            self._cap_all = None
            return False
        if self.capture == "auto" and (self._cap_all is None or
                                       tuple(self._cap_all.shape) != shape):
            budget = self.capture_budget
            if budget is None:
                free, _ = torch.cuda.mem_get_info(fd.device)
                budget = free // 4
            if nbytes > budget:
                self._cap_all = None
                return False
        if self._cap_all is None or tuple(self._cap_all.shape) != shape:
            self._cap_all = None
            with torch.cuda.stream(fd.queue):
                self._cap_all = torch.empty(shape, dtype=fd._tdt, device=fd.device)
        return True

    # ---------------------------------------------------------------- backward
    def _adjoint_buffers(self):
        """Ē, H̄ (two sets when the reverse step is fused: it reads one and writes
        the other) and the two P stripe sets; ``fields[par]`` is the step that
        reads parity ``par``."""
        fd = self.fdtd
        tdt = fd._tdt
        shp = (fd.Nx, fd.Ny, fd.Nz)
        z = lambda s: torch.zeros(s, dtype=tdt, device=fd.device)  # noqa: E731
        nsets = 2 if self.fused_reverse else 1
        Eb = [[z(shp) for _ in range(3)] for _ in range(nsets)]
        Hb = [[z(shp) for _ in range(3)] for _ in range(nsets)]
        stripes = [tuple(p.shape) for p in fd._psi_e]
        PE = [[z(s) for s in stripes] for _ in range(2)]
        PH = [[z(s) for s in stripes] for _ in range(2)]
        fields = []
        for par in range(2):
            f = capi.AdjointFields()
            cur = par % nsets
            for c in range(3):
                f.E[c] = Eb[cur][c].data_ptr()
                f.H[c] = Hb[cur][c].data_ptr()
                f.ce[c] = fd._ce[c].data_ptr()
                if nsets == 2:
                    f.E_next[c] = Eb[cur ^ 1][c].data_ptr()
                    f.H_next[c] = Hb[cur ^ 1][c].data_ptr()
            for q in range(6):
                f.pe[q] = PE[par][q].data_ptr()
                f.pe_next[q] = PE[par ^ 1][q].data_ptr()
                f.ph[q] = PH[par][q].data_ptr()
                f.ph_next[q] = PH[par ^ 1][q].data_ptr()
            fields.append(f)
        return Eb, Hb, PE, PH, fields

    @staticmethod
    def _state_at(Eb, Hb, par):
        """The Ē, H̄ tensors that hold the state read by a step of parity ``par``."""
        k = par % len(Eb)
        return Eb[k], Hb[k]

    def backward(self, grad_output=1.0):
        """``grad_output · ∂J/∂εr`` over the design box (float64 NumPy array)."""
        if self._ckpts is None:
            raise RuntimeError("call forward() before backward()")
        if self._captured:
            return self._backward_captured(grad_output)
        fd = self.fdtd
        o = self.objective
        if fd.lossy:
            raise NotImplementedError("the adjoint gradient needs a lossless grid")
        st = fd.queue.cuda_stream
        N, K = self.n_steps, self.K
        nseg = len(self._ckpts)
        Eb, Hb, PE, PH, fields, ph_dev, G, sd, gb = self._sweep_setup()
        with torch.cuda.stream(fd.queue):
            # two capture buffers: segment s is swept while segment s-1 is replayed
            cap = torch.empty((2, K + 1, 3, *self.box_shape), dtype=fd._tdt, device=fd.device)
        ph_stride = o.freqs.size * 2 * 8
        ph0 = ph_dev.data_ptr()
        lo = (ctypes.c_int32 * 3)(*[b[0] for b in self.box])
        hi = (ctypes.c_int32 * 3)(*[b[1] for b in self.box])
        slot = cap[0, 0].numel() * cap.element_size()
        buf = cap[0].numel() * cap.element_size()
        cap0 = cap.data_ptr()
        grid, cpml = fd._grid, fd._cpml_base
        Ebp = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in Eb[0]])
        # the reverse sweep runs on its own stream, concurrently with the replay
        # of the next-older segment on the engine's stream
        adj = torch.cuda.Stream(device=fd.device)
        ast = adj.cuda_stream
        ready = torch.cuda.Event()
        ready.record(fd.queue)
        adj.wait_event(ready)
        sd.phase = ph0 + (N - 1) * ph_stride
        capi.run("fdtd_adjoint_seed_add", grid, Ebp, sd, ast)

        def replay(seg):
            """Replay segment seg from its checkpoint, capturing E over the edge box;
            yields after each unit of work it enqueued on the engine's stream."""
            base = cap0 + (seg % 2) * buf
            fd.load_state(self._ckpts[seg])
            for m in range(min(N, (seg + 1) * K) - seg * K + 1):
                if m > 0:
                    fd.step()
                Ep = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in fd._E])
                capi.run("fdtd_capture_box", grid, Ep, lo, hi, base + m * slot, st)
                yield

        saved = fd._monitors
        fd._monitors = []
        par = 0
        replayed, swept = {}, {}
        try:
            for _ in replay(nseg - 1):
                pass
            replayed[nseg - 1] = torch.cuda.Event()
            replayed[nseg - 1].record(fd.queue)
            for s in range(nseg - 1, -1, -1):
                adj.wait_event(replayed[s])
                gen = None
                if s >= 1:
                    if s + 1 in swept:  # the buffer segment s-1 fills was swept as s+1
                        fd.queue.wait_event(swept[s + 1])
                    gen = replay(s - 1)
                n0 = s * K
                n1 = min(N, n0 + K)
                base = cap0 + (s % 2) * buf
                for n in range(n1 - 1, n0 - 1, -1):
                    if gen is not None:
                        next(gen, None)
                    gb.e_next = base + (n + 1 - n0) * slot
                    gb.e_prev = base + (n - n0) * slot
                    if n >= 1:
                        sd.phase = ph0 + (n - 1) * ph_stride
                        seed_arg = ctypes.byref(sd)
                    else:
                        seed_arg = None
                    capi.run("fdtd_adjoint_step", grid, fields[par], cpml, gb, seed_arg, ast)
                    par ^= 1
                if gen is not None:
                    for _ in gen:
                        pass
                    replayed[s - 1] = torch.cuda.Event()
                    replayed[s - 1].record(fd.queue)
                swept[s] = torch.cuda.Event()
                swept[s].record(adj)
        finally:
            fd._monitors = saved
            adj.synchronize()
            fd.queue.synchronize()
        self._adjoint_state = self._state_at(Eb, Hb, par)
        g_edges = G.cpu().numpy()
        return float(grad_output) * edge_to_cells(g_edges, self._eps, self.design, self.box)

    def _sweep_setup(self):
        fd = self.fdtd
        o = self.objective
        N = self.n_steps
        with torch.cuda.stream(fd.queue):
            Eb, Hb, PE, PH, fields = self._adjoint_buffers()
            phases = _phase_sequence(o.freqs, fd.dt, N, self._t_first)
            ph_dev = torch.from_numpy(np.ascontiguousarray(
                np.stack([phases.real, phases.imag], -1))).to(fd.device)
            G = torch.zeros((3, *self.box_shape), dtype=torch.float64, device=fd.device)
        (a0, a1), (b0, b1) = o.patch
        sd = capi.AdjointSeed(axis=o.axis, index=o.index, a0=a0, a1=a1, b0=b0, b1=b1,
                              comp_mask=o.comp_mask, nfreq=o.freqs.size,
                              seed=self._seed.data_ptr(), phase=0)
        gb = capi.GradBox()
        for a in range(3):
            gb.lo[a], gb.hi[a] = self.box[a]
        gb.g = G.data_ptr()
        return Eb, Hb, PE, PH, fields, ph_dev, G, sd, gb

    def _backward_captured(self, grad_output):
        """The sweep over E captured by the forward pass: no replay."""
        fd = self.fdtd
        if fd.lossy:
            raise NotImplementedError("the adjoint gradient needs a lossless grid")
        N = self.n_steps
        st = fd.queue.cuda_stream
        Eb, Hb, PE, PH, fields, ph_dev, G, sd, gb = self._sweep_setup()
        ph_stride = self.objective.freqs.size * 2 * 8
        ph0 = ph_dev.data_ptr()
        cap0 = self._cap_all.data_ptr()
        slot = self._cap_all[0].numel() * self._cap_all.element_size()
        grid, cpml = fd._grid, fd._cpml_base
        Ebp = (ctypes.c_void_p * 3)(*[t.data_ptr() for t in Eb[0]])
        sd.phase = ph0 + (N - 1) * ph_stride
        capi.run("fdtd_adjoint_seed_add", grid, Ebp, sd, st)
        par = 0
        for n in range(N - 1, -1, -1):
            gb.e_next = cap0 + (n + 1) * slot
            gb.e_prev = cap0 + n * slot
            if n >= 1:
                sd.phase = ph0 + (n - 1) * ph_stride
                seed_arg = ctypes.byref(sd)
            else:
                seed_arg = None
            capi.run("fdtd_adjoint_step", grid, fields[par], cpml, gb, seed_arg, st)
            par ^= 1
        fd.queue.synchronize()
        self._adjoint_state = self._state_at(Eb, Hb, par)
        g_edges = G.cpu().numpy()
        return float(grad_output) * edge_to_cells(g_edges, self._eps, self.design, self.box)

    def value_and_grad(self, eps_design):
        """``(J, ∂J/∂εr)`` in one forward + adjoint pass."""
        J = self.forward(eps_design)
        return J, self.backward()


class EpsilonObjective(torch.autograd.Function):
    """``J = EpsilonObjective.apply(eps_design, adjoint)``: autograd through the solver."""

    @staticmethod
    def forward(ctx, eps_design, adjoint):
        J = adjoint.forward(eps_design.detach().cpu().numpy())
        ctx.adjoint = adjoint
        ctx.meta = (eps_design.dtype, eps_design.device)
        return torch.tensor(J, dtype=torch.float64, device=eps_design.device)

    @staticmethod
    def backward(ctx, grad_out):
        g = ctx.adjoint.backward(float(grad_out))
        dtype, device = ctx.meta
        return torch.as_tensor(g, device=device).to(dtype), None


def epsilon_objective(eps_design, adjoint):
    """Functional form of :class:`EpsilonObjective`."""
    return EpsilonObjective.apply(eps_design, adjoint)
