"""Step-function API of the uniform-patch solver, on torch tensors.

Two layers:

* `PatchStepper` -- the engine: one device-resident patch (state, bed,
  workspace, run clock) advanced by the fused CUDA step (`dclaw_step` of the
  C ABI), optionally replayed from a captured CUDA graph.
* The step-function API of the reference's differentiable port
  (differentiable_dclaw/dclaw_jax/solver.py:33-41,247-249,277-297,325-388):
  `Grid`, `make_state`, `step`, `cfl_dt`, `rollout`, `rollout_peak`, with the
  same signatures and array shapes (state (5, nx, ny), bed (nx, ny)), but the
  numerics of the reference Fortran step (augmented f-wave Riemann solver,
  MC-limited second order corrections, transverse waves, src2), so results
  are those of D-Claw rather than of the port's HLL/RK2 scheme.

Every compute call goes to the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes
import math
from typing import NamedTuple

import torch

from . import _lib
from .params import CLOCK_DOUBLES, CClock, DClawParams


class Grid(NamedTuple):
    nx: int
    ny: int
    dx: float
    dy: float


class MaterialParams(NamedTuple):
    """Same fields and defaults as the differentiable port's MaterialParams
    (differentiable_dclaw/dclaw_jax/model.py:35-50)."""

    rho_s: float = 2700.0
    rho_f: float = 1000.0
    m_crit: float = 0.64
    mref: float = 0.60
    kref: float = 1.0e-9
    phi_deg: float = 40.0
    delta: float = 0.01
    mu: float = 0.005
    alpha_c: float = 0.01
    sigma_0: float = 1000.0
    c1: float = 1.0
    gz: float = 9.81
    manning_n: float = 0.0


_BC = {"wall": "wall", "open": "extrap", "extrap": "extrap"}


def to_dclaw_params(p, bc_x: str = "wall", bc_y: str = "wall", cfl: float | None = None) -> DClawParams:
    """MaterialParams or DClawParams -> DClawParams with the given boundaries."""
    for bc in (bc_x, bc_y):
        if bc not in _BC:
            raise ValueError(f"unsupported boundary condition {bc!r} (wall, open/extrap)")
    bcs = dict(bc_lower=(_BC[bc_x], _BC[bc_y]), bc_upper=(_BC[bc_x], _BC[bc_y]))
    if isinstance(p, DClawParams):
        d = p.replace(**bcs)
    elif isinstance(p, MaterialParams) or hasattr(p, "phi_deg"):
        d = DClawParams(rho_s=p.rho_s, rho_f=p.rho_f, m_crit=p.m_crit, mref=p.mref, kref=p.kref,
                        phi=p.phi_deg, delta=p.delta, mu=p.mu, alpha_c=p.alpha_c, sigma_0=p.sigma_0,
                        c1=p.c1, grav=p.gz, friction_forcing=p.manning_n > 0.0,
                        manning_coefficient=p.manning_n, **bcs)
    else:
        raise TypeError("params must be DClawParams or MaterialParams")
    if cfl is not None:
        d = d.replace(cfl_desired=float(cfl))
    return d


def make_state(h, hu, hv, hm, pb) -> torch.Tensor:
    return torch.stack([h, hu, hv, hm, pb])


def _require_cuda(t: torch.Tensor, name: str) -> None:
    if not t.is_cuda:
        raise _lib.DClawError(f"{name} must be a CUDA tensor (the solver has no CPU path)")
    if t.dtype != torch.float64:
        raise _lib.DClawError(f"{name} must be float64")


class PatchStepper:
    """One uniform patch on the device, advanced by the fused step.

    q: (5, my, mx) float64 CUDA tensor (x fastest), b: (my, mx). A (7, my,
    mx) state -- the reference's whole q (h, hu, hv, hm, pb, hchi, bdif) --
    runs the full-state step (dclaw_step_full) instead, which also does
    segregation and entrainment; h_e (my, mx) is then the erodible depth
    (required with entrainment).
    """

    def __init__(self, q: torch.Tensor, b: torch.Tensor, params: DClawParams, dx: float, dy: float,
                 branch_log: bool = False, h_e: torch.Tensor | None = None):
        _require_cuda(q, "q")
        _require_cuda(b, "b")
        self.lib = _lib.load()
        self.params = params
        self.cp = params.to_c()
        self.full = q.shape[0] == 7
        if q.shape[0] not in (5, 7):
            raise _lib.DClawError("q must have 5 fields (h, hu, hv, hm, pb) or 7 (+ hchi, bdif)")
        check = self.lib.dclaw_params_check if self.full else self.lib.dclaw_params_check_5
        _lib.check(check(ctypes.byref(self.cp)), "parameter check")
        _, self.my, self.mx = q.shape
        self.dx, self.dy = float(dx), float(dy)
        dev = q.device
        self.qa = q.contiguous().clone()
        self.qb = torch.empty_like(self.qa)
        self.b = b.contiguous()
        self.h_e = None
        if h_e is not None:
            _require_cuda(h_e, "h_e")
            self.h_e = h_e.contiguous()
        if self.full:
            self.work_bytes = self.lib.dclaw_step_full_workspace_bytes(self.mx, self.my)
        else:
            self.work_bytes = self.lib.dclaw_workspace_bytes(self.mx, self.my)
        if self.work_bytes == 0:
            raise _lib.DClawError("invalid patch size")
        self.work = torch.empty(self.work_bytes, dtype=torch.uint8, device=dev)
        self.clock = torch.zeros(CLOCK_DOUBLES, dtype=torch.float64, device=dev)
        nlog = (self.my + 2) * (self.mx + 1) + (self.mx + 2) * (self.my + 1)
        self.brlog = torch.zeros(nlog, dtype=torch.int32, device=dev) if branch_log else None
        self.graph = None
        self.graph_steps = 0

    # ---- clock -------------------------------------------------------------
    def init_clock(self, dt: float, t: float = 0.0, t_final: float = 0.0, fixed_dt: bool = False,
                   t_obs: float = 0.0) -> None:
        """t_obs > 0: with the tick rule every dt is also clipped at the next
        multiple of t_obs, so that t lands on each observation time (the
        port's flume loop)."""
        _lib.check(self.lib.dclaw_clock_init(_lib.ptr(self.clock), float(t), float(dt), float(t_final),
                                             int(fixed_dt), _lib.stream_ptr()), "clock init")
        if t_obs > 0.0:
            _lib.check(self.lib.dclaw_clock_set_obs(_lib.ptr(self.clock), float(t_obs), _lib.stream_ptr()),
                       "clock observation interval")

    def read_clock(self) -> CClock:
        buf = self.clock.cpu().numpy().tobytes()
        return CClock.from_buffer_copy(buf)

    # ---- stepping ----------------------------------------------------------
    def _launch(self, src: torch.Tensor, dst: torch.Tensor) -> None:
        if self.full:
            rc = self.lib.dclaw_step_full(_lib.ptr(src), _lib.ptr(dst), _lib.ptr(self.b), _lib.ptr(self.h_e),
                                          self.mx, self.my, self.dx, self.dy, ctypes.byref(self.cp),
                                          _lib.ptr(self.clock), _lib.ptr(self.work), self.work_bytes,
                                          _lib.ptr(self.brlog), _lib.stream_ptr())
            _lib.check(rc, "dclaw_step_full")
            return
        rc = self.lib.dclaw_step(_lib.ptr(src), _lib.ptr(dst), _lib.ptr(self.b), self.mx, self.my, self.dx,
                                 self.dy, ctypes.byref(self.cp), _lib.ptr(self.clock), _lib.ptr(self.work),
                                 self.work_bytes, _lib.ptr(self.brlog), _lib.stream_ptr())
        _lib.check(rc, "dclaw_step")

    def step(self, nsteps: int = 1, history: torch.Tensor | None = None) -> None:
        """Advance nsteps; history (nsteps, 4) receives the clock's (t, dt_next, cfl, dt_used)
        after each step."""
        for n in range(nsteps):
            self._launch(self.qa, self.qb)
            self.qa, self.qb = self.qb, self.qa
            if history is not None:
                history[n].copy_(self.clock[0:4])

    def capture(self, nsteps: int) -> None:
        """Capture nsteps (even) fused steps into a CUDA graph for replay()."""
        if nsteps % 2:
            raise ValueError("graph length must be even (buffers ping-pong)")
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                for _ in range(nsteps // 2):
                    self._launch(self.qa, self.qb)
                    self._launch(self.qb, self.qa)
        torch.cuda.current_stream().wait_stream(s)
        self.graph = g
        self.graph_steps = nsteps

    def replay(self, times: int = 1) -> None:
        if self.graph is None:
            raise RuntimeError("capture() first")
        for _ in range(times):
            self.graph.replay()

    def state(self) -> torch.Tensor:
        return self.qa

    def status(self) -> int:
        return self.read_clock().status

    # ---- state in host memory ----------------------------------------------
    def step_host(self, q_host: torch.Tensor, out: torch.Tensor | None = None, nbands: int = 0) -> None:
        """One step of a (5, my, mx) float64 state held in host memory:
        q_host -> out (q_host itself, in place, by default), with this
        stepper's bed, parameters and clock. The copies overlap the compute
        band by band when the host tensors are pinned. The stepper's device
        state is not used. Returns once the step is queued on the current
        stream; synchronize it before reading `out`."""
        if self.full:
            raise _lib.DClawError("step_host takes the five-field state")
        out = q_host if out is None else out
        for t, name in ((q_host, "q_host"), (out, "out")):
            if t.is_cuda or t.dtype != torch.float64 or not t.is_contiguous():
                raise _lib.DClawError(f"{name} must be a contiguous float64 host tensor")
            if tuple(t.shape) != (5, self.my, self.mx):
                raise _lib.DClawError(f"{name} must have shape (5, my, mx) = (5, {self.my}, {self.mx})")
        if getattr(self, "host_work", None) is None:
            nbytes = self.lib.dclaw_step_host_workspace_bytes(self.mx, self.my)
            self.host_work = torch.empty(nbytes, dtype=torch.uint8, device=self.qa.device)
        rc = self.lib.dclaw_step_host(_lib.ptr(q_host), _lib.ptr(out), _lib.ptr(self.b), self.mx, self.my,
                                      self.dx, self.dy, ctypes.byref(self.cp), _lib.ptr(self.clock),
                                      _lib.ptr(self.host_work), self.host_work.numel(), int(nbands),
                                      _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_host")


# ---- differentiable-port style API ------------------------------------------
def _to_native(q: torch.Tensor) -> torch.Tensor:
    """(5, nx, ny) (x = axis 1) -> (5, ny, nx) contiguous, x fastest."""
    return q.permute(0, 2, 1).contiguous()


def _from_native(q: torch.Tensor) -> torch.Tensor:
    return q.permute(0, 2, 1).contiguous()


def _bed(b, t: float = 0.0) -> torch.Tensor:
    bb = b(t) if callable(b) else b
    return bb.t().contiguous()


def step(q: torch.Tensor, b, p, grid: Grid, dt: float, bc_x: str = "wall", bc_y: str = "wall") -> torch.Tensor:
    """One D-Claw step of size dt on a (5, nx, ny) state over bed b (nx, ny)."""
    _require_cuda(q, "q")
    st = PatchStepper(_to_native(q), _bed(b), to_dclaw_params(p, bc_x, bc_y), grid.dx, grid.dy)
    st.init_clock(float(dt), fixed_dt=True)
    st.step(1)
    _lib.check(st.status(), "step")
    return _from_native(st.state())


def max_wave_speed(q_native: torch.Tensor, params: DClawParams) -> torch.Tensor:
    """max |u| + sqrt(g h) over wet cells of an (5, ny, nx) state (device scalar)."""
    lib = _lib.load()
    out = torch.zeros(1, dtype=torch.float64, device=q_native.device)
    cp = params.to_c()
    _, my, mx = q_native.shape
    _lib.check(lib.dclaw_max_wave_speed(_lib.ptr(q_native), mx, my, ctypes.byref(cp), _lib.ptr(out),
                                        _lib.stream_ptr()), "max_wave_speed")
    return out[0]


def cfl_dt(q: torch.Tensor, p, grid: Grid, cfl: float) -> torch.Tensor:
    """cfl * min(dx, dy) / max(max wave speed, 1e-6) (solver.py:247-249)."""
    smax = max_wave_speed(_to_native(q), to_dclaw_params(p))
    return cfl * min(grid.dx, grid.dy) / torch.clamp(smax, min=1.0e-6)


def gate_bed(b_base: torch.Tensor, gate_shape: torch.Tensor, gate_t, gate_deg):
    """Moving bed of a headgate release, as the port builds it
    (differentiable_dclaw/dclaw_jax/solver.py:304-322): the closed gate is a
    ridge `gate_shape` on top of `b_base`, lowered to cos(angle(t)) of its
    height as the gate swings open, angle piecewise linear through
    (gate_t, gate_deg) and held at the end values outside them. Returns
    b(t) for `rollout` / `rollout_peak`; t may be a device tensor, so the bed
    is rebuilt on the device without a host round trip."""
    gt = torch.as_tensor(gate_t, dtype=torch.float64, device=b_base.device)
    gd = torch.as_tensor(gate_deg, dtype=torch.float64, device=b_base.device)

    def bed(t):
        t = torch.as_tensor(t, dtype=torch.float64, device=b_base.device).reshape(1)
        k = torch.clamp(torch.searchsorted(gt, t, right=True), 1, len(gt) - 1)
        t0, t1, a0, a1 = gt[k - 1], gt[k], gd[k - 1], gd[k]
        w = torch.clamp((t - t0) / (t1 - t0), 0.0, 1.0)
        angle = torch.where(t <= gt[0], gd[0], torch.where(t >= gt[-1], gd[-1], a0 + w * (a1 - a0)))
        return b_base + torch.cos(angle * (math.pi / 180.0)) * gate_shape

    return bed


def rollout(q0: torch.Tensor, b, p, grid: Grid, t_final: float, cfl: float = 0.4, bc_x: str = "wall",
            bc_y: str = "wall", n_steps: int = 2000, keep_states: bool = True):
    """Advance towards t_final over a fixed number of steps.

    The first dt comes from `cfl_dt`; after that dt follows D-Claw's tick
    rule (dt * cfl / Courant number of the last step, tick.f:490-526) and is
    clipped so that t never passes t_final (dt = 0 afterwards). Returns
    (q_final, t_reached, states, times) like the port; with keep_states=False
    states/times are None. `b` may be a function of t (a moving bed, e.g.
    `gate_bed`): it is evaluated at the start of each step on the device and
    h is left as it is when the bed moves, as GeoClaw does.
    """
    moving = callable(b)
    prm = to_dclaw_params(p, bc_x, bc_y, cfl)
    st = PatchStepper(_to_native(q0), _bed(b, torch.zeros((), dtype=torch.float64, device=q0.device)), prm, grid.dx,
                      grid.dy)
    dt0 = float(cfl_dt(q0, prm, grid, cfl))
    st.init_clock(dt0, t_final=float(t_final))
    states = torch.empty((n_steps,) + tuple(q0.shape), dtype=q0.dtype, device=q0.device) if keep_states else None
    hist = torch.empty((n_steps, 4), dtype=torch.float64, device=q0.device)
    for n in range(n_steps):
        if moving:
            st.b.copy_(b(st.clock[0]).t())
        st.step(1, history=hist[n:n + 1])
        if keep_states:
            states[n].copy_(st.state().permute(0, 2, 1))
    _lib.check(st.status(), "rollout")
    t_reached = hist[-1, 0]
    return _from_native(st.state()), t_reached, states, (hist[:, 0] if keep_states else None)


def rollout_peak(q0: torch.Tensor, b, p, grid: Grid, t_final: float, cfl: float = 0.4, bc_x: str = "wall",
                 bc_y: str = "wall", n_steps: int = 2000, checkpoint_block: int | None = None):
    """Like `rollout` but keeps only the running per-cell peak depth.
    Returns (q_final, t_reached, h_peak)."""
    if checkpoint_block is not None and n_steps % checkpoint_block:
        raise ValueError("n_steps must be a multiple of checkpoint_block")
    moving = callable(b)
    prm = to_dclaw_params(p, bc_x, bc_y, cfl)
    st = PatchStepper(_to_native(q0), _bed(b, torch.zeros((), dtype=torch.float64, device=q0.device)), prm, grid.dx,
                      grid.dy)
    st.init_clock(float(cfl_dt(q0, prm, grid, cfl)), t_final=float(t_final))
    hmax = st.state()[0].clone()
    for _ in range(n_steps):
        if moving:
            st.b.copy_(b(st.clock[0]).t())
        st.step(1)
        torch.maximum(hmax, st.state()[0], out=hmax)
    _lib.check(st.status(), "rollout_peak")
    t = st.read_clock().t
    return _from_native(st.state()), t, hmax.t().contiguous()


__all__ = ["Grid", "MaterialParams", "PatchStepper", "make_state", "step", "cfl_dt", "rollout", "rollout_peak", "gate_bed",
           "to_dclaw_params", "max_wave_speed"]
