"""Reverse-mode gradients of runs of the uniform-patch step.

The reference's differentiable port takes gradients with `jax.grad` through
`rollout_peak(..., checkpoint_block=k)`, whose nested `jax.checkpoint` scans
keep about n/k + k states (differentiable_dclaw/dclaw_jax/solver.py:357-388,
differentiable_dclaw/tests/test_reverse_mode.py:37-49). Here the step is the
reference Fortran's (the fused CUDA step of `solver.PatchStepper`) and its
reverse is hand-written (`dclaw_step_adjoint` of the C ABI, one launch
sequence per step), wrapped in a `torch.autograd.Function` with the same
sqrt(N) time checkpointing:

* forward: run the fused step, record each step's dt on the device, keep the
  state every k steps and the states the caller asked for. Unless k is
  given, it is the smallest block whose checkpoints fit half of the free
  device memory (after the adjoint's two workspaces): every state (k = 1, no
  recompute) when the run fits, as a 512 x 512 run of 500 steps (5 GB)
  does in a B200's 180 GB, and at most ceil(sqrt(n_steps));
* backward: for each block of k steps, last block first, recompute its
  states from its checkpoint with the recorded dts (bit-identical, so every
  branch is the one the forward took), then run the step adjoint backwards
  through the block, adding the caller's output gradients as it passes them.
  Each step adjoint is queued in two parts: the part that does not read
  the output adjoint (the forward recompute, `prepare`) runs on a side
  stream one step ahead, in a second workspace, while the previous step's
  reverse stages run on a high-priority stream.

Time steps are data: the dt of each step (chosen by D-Claw's tick rule from
the previous Courant number, or fixed) is recorded in the forward pass and
not differentiated. Gradients flow to the initial state and to the material
parameters theta = (phi [deg], kref, alpha_c, mu).
"""
from __future__ import annotations

import ctypes
import math
from typing import Sequence

import numpy as np
import torch

from . import _lib
from .params import DClawParams
from .solver import PatchStepper

THETA_NAMES = ("phi", "kref", "alpha_c", "mu")
_DEG = math.pi / 180.0


def theta_of(params: DClawParams, device=None) -> torch.Tensor:
    """(phi [deg], kref, alpha_c, mu) of a parameter set as a float64 tensor."""
    return torch.tensor([params.phi, params.kref, params.alpha_c, params.mu], dtype=torch.float64, device=device)


def with_theta(params: DClawParams, theta) -> DClawParams:
    vals = [float(v) for v in (theta.tolist() if torch.is_tensor(theta) else theta)]
    return params.replace(**dict(zip(THETA_NAMES, vals)))


class StepAdjoint:
    """The adjoint of one step of a fixed patch (bed, parameters, sizes).

    vjp(q_in, dt, lam_out, lam_in, pbar): lam_in = (dS/dq)^T lam_out and
    pbar += (dS/dtheta)^T lam_out with phi in radians; dt is a one-element
    float64 device tensor (the step's dt); all arrays are (5, my, mx).
    """

    def __init__(self, b: torch.Tensor, params: DClawParams, dx: float, dy: float):
        self.lib = _lib.load()
        self.cp = params.to_c()
        _lib.check(self.lib.dclaw_adjoint_supported(ctypes.byref(self.cp)), "adjoint options")
        self.b = b.contiguous()
        self.my, self.mx = self.b.shape
        self.dx, self.dy = float(dx), float(dy)
        self.work_bytes = self.lib.dclaw_adjoint_workspace_bytes(self.mx, self.my)
        if self.work_bytes == 0:
            raise _lib.DClawError("invalid patch size")
        self.work = torch.empty(self.work_bytes, dtype=torch.uint8, device=b.device)
        self.status = torch.zeros(1, dtype=torch.int32, device=b.device)

    def vjp(self, q_in: torch.Tensor, dt: torch.Tensor, lam_out: torch.Tensor, lam_in: torch.Tensor,
            pbar: torch.Tensor, bbar: torch.Tensor | None = None) -> None:
        """bbar ((my, mx), accumulated, optional): += the bed's adjoint."""
        rc = self.lib.dclaw_step_adjoint(_lib.ptr(q_in), _lib.ptr(self.b), self.mx, self.my, self.dx, self.dy,
                                         _lib.ptr(dt), ctypes.byref(self.cp), _lib.ptr(lam_out), _lib.ptr(lam_in),
                                         _lib.ptr(pbar), _lib.ptr(bbar), _lib.ptr(self.work), self.work_bytes,
                                         _lib.ptr(self.status), _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_adjoint")

    def prepare(self, q_in: torch.Tensor, dt: torch.Tensor) -> None:
        """The part of vjp that does not read lam_out (activity blocks and the
        forward recompute into this object's workspace)."""
        rc = self.lib.dclaw_step_adjoint_prepare(_lib.ptr(q_in), _lib.ptr(self.b), self.mx, self.my, self.dx,
                                                 self.dy, _lib.ptr(dt), ctypes.byref(self.cp), _lib.ptr(self.work),
                                                 self.work_bytes, _lib.ptr(self.status), _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_adjoint_prepare")

    def reverse(self, q_in: torch.Tensor, dt: torch.Tensor, lam_out: torch.Tensor, lam_in: torch.Tensor,
                pbar: torch.Tensor, bbar: torch.Tensor | None = None) -> None:
        """The rest of vjp, after prepare with the same q_in and dt."""
        rc = self.lib.dclaw_step_adjoint_reverse(_lib.ptr(q_in), _lib.ptr(self.b), self.mx, self.my, self.dx,
                                                 self.dy, _lib.ptr(dt), ctypes.byref(self.cp), _lib.ptr(lam_out),
                                                 _lib.ptr(lam_in), _lib.ptr(pbar), _lib.ptr(bbar),
                                                 _lib.ptr(self.work), self.work_bytes, _lib.ptr(self.status),
                                                 _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_adjoint_reverse")

    def check_status(self) -> None:
        _lib.check(int(self.status.item()), "adjoint step")


def _pipelined_backward(adjs, n_steps, k, ckpt, segs, recompute, dt_of, lam, lam2, pbar, add_outs, bed_for=None,
                        bbar=None, after_reverse=None):
    """The step adjoints of steps n_steps .. 1, each step's prepare queued on
    a side stream ahead of the previous step's reverse.

    adjs: two adjoint objects (two workspaces), used alternately. ckpt[s] is
    the input of step s k + 1 (block s); with k > 1 the block's other inputs
    are recomputed into segs[s % 2] by recompute(s, seg), queued on the
    reverse stream after the reverses of block s + 1 (so that its kernels,
    persistent ones among them, never hold SMs the reverses wait for; the
    buffer's previous user, block s + 2, is done by then). dt_of(n): step
    n's dt; add_outs(n, lam): adds the output gradients at step count n;
    bed_for(n, adj) (a moving bed): fills adj's bed with step n's, on the
    side stream once adj's workspace is free. bbar (optional): accumulates
    the bed's adjoint over the steps; after_reverse(n) (optional) runs on
    the reverse stream right after step n's reverse (a moving bed's
    parameters take that step's bed adjoint from bbar there).
    The reverses run on a high-priority stream and the prepares (which do
    not read lam) on a normal one, so they fill the SMs the reverses leave
    idle. Returns the final (lam, lam2)."""
    cur = torch.cuda.current_stream()
    rev = torch.cuda.Stream(priority=-8)        # mapped to the device's highest priority
    side = torch.cuda.Stream()
    rev.wait_stream(cur)
    side.wait_stream(cur)
    last_rev = [None, None]               # the last reverse that used each workspace

    def state_of(n):
        s, j = (n - 1) // k, (n - 1) % k
        return ckpt[s] if j == 0 else segs[s % 2][j]

    def prepare(n):
        # on the side stream, after the block's recompute when n is its top step
        s = (n - 1) // k
        if k > 1 and (n == n_steps or n % k == 0):
            with torch.cuda.stream(rev):
                recompute(s, segs[s % 2])
            side.wait_event(rev.record_event())
        if last_rev[n % 2] is not None:
            side.wait_event(last_rev[n % 2])
        if bed_for is not None:
            bed_for(n, adjs[n % 2])
        adjs[n % 2].prepare(state_of(n), dt_of(n))

    with torch.cuda.stream(side):
        prepare(n_steps)
    ev_prep = side.record_event()
    for n in range(n_steps, 0, -1):
        w = n % 2
        with torch.cuda.stream(rev):
            rev.wait_event(ev_prep)
            add_outs(n, lam)
            adjs[w].reverse(state_of(n), dt_of(n), lam, lam2, pbar, bbar)
            if after_reverse is not None:
                after_reverse(n)
            last_rev[w] = rev.record_event()
        if n > 1:
            with torch.cuda.stream(side):
                prepare(n - 1)
            ev_prep = side.record_event()
        lam, lam2 = lam2, lam
    cur.wait_stream(rev)
    cur.wait_stream(side)
    return lam, lam2


# share of the device memory free when a differentiable run starts that its
# checkpoints may take (the step adjoint's two workspaces are set aside first)
CHECKPOINT_MEMORY_FRACTION = 0.5


def checkpoint_block_for(n_steps: int, state_bytes: int, budget_bytes: float) -> int:
    """The smallest block length k whose checkpoints fit the budget: the
    forward pass keeps ceil(n/k) block inputs, the backward pass recomputes
    a block's other k-1 states into a k-state buffer (none when k = 1). The
    backward pass recomputes n - ceil(n/k) steps, so the smallest k that
    fits is the cheapest: k = 1 (every state kept, nothing recomputed)
    whenever the run's states fit, up to k = ceil(sqrt(n)), the memory
    minimum of two-level checkpointing, which is returned when nothing
    smaller fits."""
    n = max(1, int(n_steps))
    kmax = max(1, math.ceil(math.sqrt(n)))
    for k in range(1, kmax):
        nstates = -(-n // k) + (k if k > 1 else 0)
        if nstates * state_bytes <= budget_bytes:
            return k
    return kmax


def _block(n_steps: int, checkpoint_block: int | None, state_bytes: int = 0, reserve_bytes: int = 0,
           device=None) -> int:
    if checkpoint_block is None:
        if state_bytes <= 0 or device is None or device.type != "cuda":
            return max(1, math.ceil(math.sqrt(n_steps)))
        free, _ = torch.cuda.mem_get_info(device)
        budget = CHECKPOINT_MEMORY_FRACTION * max(0, free - reserve_bytes)
        return checkpoint_block_for(n_steps, state_bytes, budget)
    if checkpoint_block < 1:
        raise ValueError("checkpoint_block must be >= 1")
    return int(checkpoint_block)


class _Rollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q0, theta, b, params, dx, dy, n_steps, out_steps, dt0, fixed_dt, t_final, checkpoint_block,
                dt_schedule, select, obs_dt, n_obs, peak, *bed_params):
        prm = with_theta(params, theta.detach().cpu())
        # a moving bed: a function of the simulated time, evaluated before
        # every step (the port's step(q, bed(t), ...) loop)
        bed_fn = b if callable(b) else None
        if bed_fn is not None:
            b = bed_fn(torch.zeros((), dtype=torch.float64, device=q0.device)).contiguous()
        b = b.detach()
        st = PatchStepper(q0.detach(), b, prm, dx, dy)
        if dt_schedule is not None:
            # a replayed schedule keeps the observation interval for the
            # record (a fixed-dt clock is not clipped by it)
            st.init_clock(0.0, fixed_dt=True, t_obs=float(obs_dt) if n_obs else 0.0)
        else:
            st.init_clock(float(dt0), t_final=float(t_final), fixed_dt=bool(fixed_dt), t_obs=float(obs_dt))
        lib = _lib.load()
        k = _block(n_steps, checkpoint_block, q0.numel() * 8,
                   2 * lib.dclaw_adjoint_workspace_bytes(q0.shape[2], q0.shape[1]), q0.device)
        dts = torch.empty(n_steps, dtype=torch.float64, device=q0.device)
        t_start = torch.empty(n_steps if bed_fn is not None else 0, dtype=torch.float64, device=q0.device)
        oshape = tuple(q0.shape) if select is None else tuple(select.shape)
        plane = q0.shape[1] * q0.shape[2]
        if peak:
            # running peak depth from q0's, and the step that set it
            outs = q0.detach()[0].clone()
            argstep = torch.zeros(outs.shape, dtype=torch.int32, device=q0.device)
        elif n_obs:
            # observation slots: filled on the device when the clock lands
            # on an observation time; slots the run does not reach stay 0
            outs = torch.zeros((n_obs,) + oshape, dtype=q0.dtype, device=q0.device)
            obs_step = torch.full((n_obs,), -1, dtype=torch.int32, device=q0.device)
            sel64 = None if select is None else select.reshape(-1).to(torch.int64).contiguous()
            nsel = q0.numel() if select is None else sel64.numel()
        else:
            outs = torch.empty((len(out_steps),) + oshape, dtype=q0.dtype, device=q0.device)
        pick = (lambda t: t) if select is None else (lambda t: t.reshape(-1)[select])
        where = {}
        for idx, n in enumerate(out_steps):
            where.setdefault(n, []).append(idx)
        for idx in where.get(0, []):
            outs[idx].copy_(pick(q0.detach()))
        # every block's first input in one allocation; the step before a
        # block writes straight into its slot, the others ping-pong
        store = torch.empty((max(1, -(-n_steps // k)),) + tuple(q0.shape), dtype=q0.dtype, device=q0.device)
        store[0].copy_(st.qa)
        ckpt = list(store.unbind(0))
        src = ckpt[0]
        for n in range(n_steps):
            nxt = (n + 1) // k
            if (n + 1) % k == 0 and nxt < len(ckpt):
                dst = ckpt[nxt]
            else:
                dst = st.qa if src is not st.qa else st.qb
            if dt_schedule is not None:
                st.clock[1:2].copy_(dt_schedule[n:n + 1])
            if bed_fn is not None:
                t_start[n:n + 1].copy_(st.clock[0:1])
                st.b.copy_(bed_fn(st.clock[0]))
            st._launch(src, dst)
            src = dst
            dts[n:n + 1].copy_(st.clock[3:4])   # dt the step used
            for idx in where.get(n + 1, []):
                outs[idx].copy_(pick(src))
            if peak:
                _lib.check(lib.dclaw_peak_update(_lib.ptr(src), _lib.ptr(outs), _lib.ptr(argstep), plane, n + 1,
                                                 _lib.stream_ptr()), "peak update")
            if n_obs:
                _lib.check(lib.dclaw_obs_record(_lib.ptr(st.clock), 1, None, _lib.ptr(src), _lib.ptr(sel64), nsel,
                                                n_obs, n + 1, _lib.ptr(outs), _lib.ptr(obs_step),
                                                _lib.stream_ptr()), "observation record")
        _lib.check(st.status(), "rollout forward")
        if n_obs:
            # the step each slot was recorded at (-1: not reached) stands in
            # for the output steps of the backward pass
            out_steps = tuple(int(v) for v in obs_step.cpu().tolist())
        # the block inputs are saved tensors: autograd frees them after the
        # backward pass (unless the graph is retained), so a loop of gradient
        # evaluations reuses one allocation instead of holding two
        ctx.save_for_backward(b, dts, store, t_start, *bed_params)
        ctx.bed_fn = bed_fn
        ctx.select = select
        ctx.meta = (prm, float(dx), float(dy), int(n_steps), tuple(out_steps), k)
        ctx.obs_steps = tuple(out_steps) if n_obs else None
        ctx.peak_arg = argstep if peak else None
        return outs

    @staticmethod
    def backward(ctx, g_out):
        b, dts, store, t_start, *bed_params = ctx.saved_tensors
        ckpt = list(store.unbind(0))
        prm, dx, dy, n_steps, out_steps, k = ctx.meta
        bed_fn = ctx.bed_fn
        dev = b.device
        shape = ckpt[0].shape
        where = {}
        for idx, n in enumerate(out_steps):
            where.setdefault(n, []).append(idx)
        # with a moving bed each workspace and the recompute keep their own
        # bed, refilled with the step's bed(t) before they use it
        own = (lambda x: x.clone()) if bed_fn is not None else (lambda x: x)
        adjs = [StepAdjoint(own(b), prm, dx, dy), StepAdjoint(own(b), prm, dx, dy)]
        fw = PatchStepper(ckpt[0], own(b), prm, dx, dy)
        fw.init_clock(0.0, fixed_dt=True)
        lam = torch.zeros(shape, dtype=torch.float64, device=dev)
        lam2 = torch.empty_like(lam)
        pbar = torch.zeros(4, dtype=torch.float64, device=dev)
        seg = torch.empty((k,) + tuple(shape), dtype=torch.float64, device=dev) if k > 1 else None
        g_out = g_out.contiguous() if g_out is not None else None
        sel = ctx.select

        def add_out(idx, target):
            if sel is None:
                target.add_(g_out[idx])
            else:
                target.view(-1).index_add_(0, sel.reshape(-1), g_out[idx].reshape(-1))

        segs = [seg, torch.empty_like(seg)] if k > 1 else None

        def recompute(s, buf):
            # the block's states n0+1 .. n1-1 from its first input, with the recorded dts
            n0, n1 = s * k, min(s * k + k, n_steps)
            src = ckpt[s]
            for n in range(n0 + 1, n1):
                fw.clock[1:2].copy_(dts[n - 1:n])
                if bed_fn is not None:
                    fw.b.copy_(bed_fn(t_start[n - 1]))
                fw._launch(src, buf[n - n0])
                src = buf[n - n0]

        peak_arg = ctx.peak_arg
        lib = _lib.load()

        def add_outs(n, target):
            if g_out is None:
                return
            for idx in where.get(n, []):
                add_out(idx, target)
            if peak_arg is not None:
                _lib.check(lib.dclaw_peak_adjoint(_lib.ptr(g_out), _lib.ptr(peak_arg), peak_arg.numel(), n,
                                                  _lib.ptr(target), _lib.stream_ptr()), "peak adjoint")

        def bed_for(n, adj):
            adj.b.copy_(bed_fn(t_start[n - 1]))

        # the bed's gradient, for a fixed bed that requires one
        bbar = torch.zeros_like(b) if bed_fn is None and ctx.needs_input_grad[2] else None
        # a moving bed's parameters: each step's bed adjoint, through the
        # step's bed b(t_n) = bed_fn(t_n), summed over the steps
        pgrads = [None] * len(bed_params)
        after = None
        want = [i for i, t in enumerate(bed_params) if ctx.needs_input_grad[17 + i]]
        if bed_fn is not None and want:
            bbar = torch.zeros_like(b)
            pgrads = [torch.zeros_like(t) if i in want else None for i, t in enumerate(bed_params)]

            def after(n):
                # retain_graph: bed_fn may close over tensors computed from
                # the parameters outside it (a gate shape amp * ridge), whose
                # graph every step's bed shares
                with torch.enable_grad():
                    bn = bed_fn(t_start[n - 1])
                    gs = torch.autograd.grad(bn, [bed_params[i] for i in want], bbar, allow_unused=True,
                                             retain_graph=True)
                for i, gi in zip(want, gs):
                    if gi is not None:
                        pgrads[i].add_(gi)
                bbar.zero_()

        lam, lam2 = _pipelined_backward(adjs, n_steps, k, ckpt, segs, recompute, lambda n: dts[n - 1:n], lam,
                                        lam2, pbar, add_outs, bed_for if bed_fn is not None else None, bbar, after)
        if bed_fn is not None:
            bbar = None
        add_outs(0, lam)
        _lib.check(fw.status(), "rollout recompute")
        for adj in adjs:
            adj.check_status()
        scale = torch.tensor([_DEG, 1.0, 1.0, 1.0], dtype=torch.float64, device=dev)
        return (lam, pbar * scale, bbar, None, None, None, None, None, None, None, None, None, None, None, None, None,
                None, *pgrads)


def rollout_states(q0: torch.Tensor, theta: torch.Tensor, b, params: DClawParams, dx: float,
                   dy: float, n_steps: int, out_steps: Sequence[int], dt0: float, fixed_dt: bool = False,
                   t_final: float = 0.0, checkpoint_block: int | None = None,
                   dt_schedule: torch.Tensor | None = None, select: torch.Tensor | None = None,
                   obs_dt: float = 0.0, bed_params: Sequence[torch.Tensor] = ()) -> torch.Tensor:
    """Differentiable run of n_steps fused steps on one patch.

    q0: (5, my, mx) float64 CUDA tensor (x fastest), theta: (4,) float64
    tensor (phi [deg], kref, alpha_c, mu) overriding those fields of params,
    b: (my, mx), or a moving bed: a function of the simulated time (a 0-dim
    float64 device tensor) returning the (my, mx) bed, evaluated before every
    step as the port's loops do (e.g. `solver.gate_bed`). A fixed bed that
    requires grad gets its gradient (through calc_taudir's surface slopes
    and the solver's bed step), as the port's rollout_peak is differentiated
    with respect to the whole bed. A moving bed is differentiated with
    respect to bed_params, the tensors the function reads (for `gate_bed`:
    the gate's ridge, its times and its angles, as tensors that require
    grad): each step's bed adjoint goes back through that step's b(t_n).
    Returns the states after each step count in out_steps (0 = q0), shape
    (len(out_steps), 5, my, mx). dt0 is the first dt; with
    fixed_dt every step uses it, otherwise the tick rule picks the next dt
    from the Courant number (clipped at t_final when t_final > 0). Gradients
    reach q0 and theta through the hand-written step adjoint with time
    checkpointing (checkpoint_block steps per block; by default the
    smallest block whose checkpoints fit half of the free device memory,
    `checkpoint_block_for`: 1, every state kept, when the run fits).
    dt_schedule (n_steps,) float64 device tensor: replay these dts instead
    (dt0, fixed_dt and t_final are then ignored) -- e.g. the dts of an
    earlier adaptive run, for finite-difference checks at a fixed schedule.
    select (int64 CUDA tensor of flat indices into the (5, my, mx) state):
    return only these entries at each output step, shape (len(out_steps),
    *select.shape) -- e.g. gauge cells' depths -- instead of whole states.
    obs_dt > 0 (with the tick rule): every dt is also clipped at the next
    multiple of obs_dt, so that the run lands on each observation time, as
    the port's flume loop does (pf_flume/flume_model.py:152-153).
    """
    for n in out_steps:
        if not 0 <= n <= n_steps:
            raise ValueError(f"output step {n} outside 0..{n_steps}")
    if dt_schedule is not None:
        if dt_schedule.shape != (n_steps,) or dt_schedule.dtype != torch.float64 or not dt_schedule.is_cuda:
            raise ValueError("dt_schedule must be a (n_steps,) float64 CUDA tensor")
        dt_schedule = dt_schedule.contiguous()
    return _Rollout.apply(q0, theta, b if callable(b) else b.contiguous(), params, dx, dy, int(n_steps),
                          tuple(int(n) for n in out_steps),
                          float(dt0), bool(fixed_dt), float(t_final), checkpoint_block, dt_schedule, select,
                          float(obs_dt), 0, False, *tuple(bed_params))


def rollout_observations(q0: torch.Tensor, theta: torch.Tensor, b, params: DClawParams, dx: float, dy: float,
                         n_steps: int, obs_dt: float, n_obs: int, dt0: float, t_end: float = 0.0,
                         select: torch.Tensor | None = None, checkpoint_block: int | None = None,
                         dt_schedule: torch.Tensor | None = None,
                         bed_params: Sequence[torch.Tensor] = ()) -> torch.Tensor:
    """Differentiable run that records observations at fixed times, as the
    port's flume loop does (pf_flume/flume_model.py:150-158): every tick-rule
    dt is clipped at the next multiple of obs_dt (and at t_end when
    t_end > 0), and after a step that lands on (k+1) obs_dt with dt > 0,
    slot k receives the state (or its `select` entries). Returns
    (n_obs, 5, my, mx) or (n_obs, *select.shape); slots the n_steps steps
    do not reach stay 0 and take no gradient. `observation_steps(out)`
    gives the step each slot was recorded at. The other arguments are those
    of `rollout_states`; dt_schedule replays recorded dts (the slots then
    follow the replayed times)."""
    if not obs_dt > 0.0 or int(n_obs) < 1:
        raise ValueError("obs_dt must be > 0 and n_obs >= 1")
    if dt_schedule is not None:
        if dt_schedule.shape != (n_steps,) or dt_schedule.dtype != torch.float64 or not dt_schedule.is_cuda:
            raise ValueError("dt_schedule must be a (n_steps,) float64 CUDA tensor")
        dt_schedule = dt_schedule.contiguous()
    return _Rollout.apply(q0, theta, b if callable(b) else b.contiguous(), params, dx, dy, int(n_steps), (),
                          float(dt0), False, float(t_end), checkpoint_block, dt_schedule, select, float(obs_dt),
                          int(n_obs), False, *tuple(bed_params))


def rollout_peak(q0: torch.Tensor, theta: torch.Tensor, b, params: DClawParams, dx: float, dy: float,
                 n_steps: int, dt0: float, t_final: float = 0.0, fixed_dt: bool = False,
                 checkpoint_block: int | None = None, dt_schedule: torch.Tensor | None = None,
                 bed_params: Sequence[torch.Tensor] = ()) -> torch.Tensor:
    """Differentiable running peak depth over n_steps steps, the loss input
    of the port's rollout_peak (differentiable_dclaw/dclaw_jax/solver.py:
    357-388, differentiated by jax.grad): max over q0 and every step's state
    of h, per cell, shape (my, mx). Its gradient reaches q0, theta and a
    fixed bed that requires grad through the step that set each cell's peak
    (ties: the earliest step). The other arguments are those of
    `rollout_states`."""
    if dt_schedule is not None:
        if dt_schedule.shape != (n_steps,) or dt_schedule.dtype != torch.float64 or not dt_schedule.is_cuda:
            raise ValueError("dt_schedule must be a (n_steps,) float64 CUDA tensor")
        dt_schedule = dt_schedule.contiguous()
    return _Rollout.apply(q0, theta, b if callable(b) else b.contiguous(), params, dx, dy, int(n_steps), (),
                          float(dt0), bool(fixed_dt), float(t_final), checkpoint_block, dt_schedule, None, 0.0, 0,
                          True, *tuple(bed_params))


def observation_steps(out: torch.Tensor) -> list:
    """The step count each observation slot of `rollout_observations` or
    `ensemble_rollout_observations` was recorded at (-1: not reached); for
    an ensemble, one list per slot with an entry per member."""
    steps = getattr(out.grad_fn, "obs_steps", None)
    if steps is None:
        raise ValueError("not the output of a differentiable observation run")
    return list(steps)


def checkpoint_block_of(out: torch.Tensor) -> int:
    """The checkpoint block length the differentiable run that produced
    `out` (rollout_states or ensemble_rollout_states) chose."""
    return int(out.grad_fn.meta[-1])


def last_dts(out: torch.Tensor) -> torch.Tensor:
    """The per-step dts recorded by the rollout that produced `out`."""
    fn = out.grad_fn
    if fn is None or not hasattr(fn, "saved_tensors"):
        raise ValueError("not the output of a differentiable rollout")
    return fn.saved_tensors[1]


def initial_state(h0: torch.Tensor, m0: torch.Tensor, params: DClawParams, p_ratio: float = 0.8) -> torch.Tensor:
    """Differentiable (5, my, mx) state at rest from a depth field and a solid
    fraction (scalar or field): hm = h m, pb = p_ratio rho_f g h, then the
    admissibility clip of qfix (digclaw_module.f90:285-345; init_ptype = 3
    style pore pressure, qinit.f90:264-285). Dry cells (h <= dry_tolerance)
    are zero."""
    wet = h0 > params.dry_tolerance
    hs = torch.where(wet, h0, torch.ones_like(h0))
    m = torch.clamp((h0 * m0) / hs, 0.0, 1.0)
    rho = params.rho_s * m + (1.0 - m) * params.rho_f
    pb = torch.minimum(torch.clamp(p_ratio * params.rho_f * params.grav * h0, min=0.0), rho * params.grav * h0)
    z = torch.zeros_like(h0)
    q = torch.stack([h0, z, z, h0 * m, pb])
    return torch.where(wet.unsqueeze(0), q, torch.zeros_like(q))


__all__ = ["StepAdjoint", "rollout_states", "rollout_observations", "observation_steps", "rollout_peak", "theta_of", "with_theta", "initial_state", "last_dts", "THETA_NAMES",
           "EnsembleStepAdjoint", "ensemble_rollout_states", "ensemble_rollout_observations", "ensemble_last_dts"]


# ---- ensembles -----------------------------------------------------------------
class EnsembleStepAdjoint:
    """The adjoint of one ensemble step (every member of an `EnsembleStepper`'s
    layout at once): lam_in = (dS/dq)^T lam_out on the state arenas, and
    pbar[k] += (dS_k/dtheta_k)^T lam_out_k per member (phi in radians).
    dts: (n,) float64 device tensor, member k's dt."""

    def __init__(self, stepper, params_dev: torch.Tensor | None = None):
        from .params import CAdjBatch, CAdjMember

        self.lib = _lib.load()
        st = stepper
        self.n = st.n
        for m in st.members:
            _lib.check(self.lib.dclaw_adjoint_supported(ctypes.byref(m.params.to_c())), "adjoint options")
        q_off = np.array([st.cm[k].q_off for k in range(self.n)], dtype=np.uint64)
        b_off = np.array([st.cm[k].b_off for k in range(self.n)], dtype=np.uint64)
        self.am = (CAdjMember * self.n)()
        self.batch = CAdjBatch()
        _lib.check(self.lib.dclaw_adjoint_batch_layout(self.n, st.mx.ctypes.data, st.my.ctypes.data,
                                                       st.dxs.ctypes.data, st.dys.ctypes.data, q_off.ctypes.data,
                                                       b_off.ctypes.data, self.am, ctypes.byref(self.batch)),
                   "adjoint batch layout")
        dev = st.device
        self.members_dev = torch.frombuffer(bytearray(bytes(self.am)), dtype=torch.uint8).to(dev)
        self.params = st.params if params_dev is None else params_dev
        self.bed = st.bed
        self.work = torch.empty(self.batch.work_bytes, dtype=torch.uint8, device=dev)
        self.status = torch.zeros(self.n, dtype=torch.int32, device=dev)

    def prepare(self, q_in: torch.Tensor, dts: torch.Tensor) -> None:
        rc = self.lib.dclaw_step_adjoint_batched_prepare(ctypes.byref(self.batch), _lib.ptr(self.members_dev),
                                                         _lib.ptr(self.params), _lib.ptr(dts), _lib.ptr(q_in),
                                                         _lib.ptr(self.bed), _lib.ptr(self.work),
                                                         _lib.ptr(self.status), _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_adjoint_batched_prepare")

    def reverse(self, q_in: torch.Tensor, dts: torch.Tensor, lam_out: torch.Tensor, lam_in: torch.Tensor,
                pbar: torch.Tensor, bbar: torch.Tensor | None = None) -> None:
        rc = self.lib.dclaw_step_adjoint_batched_reverse(ctypes.byref(self.batch), _lib.ptr(self.members_dev),
                                                         _lib.ptr(self.params), _lib.ptr(dts), _lib.ptr(q_in),
                                                         _lib.ptr(self.bed), _lib.ptr(lam_out), _lib.ptr(lam_in),
                                                         _lib.ptr(pbar), _lib.ptr(bbar), _lib.ptr(self.work),
                                                         _lib.ptr(self.status), _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_adjoint_batched_reverse")

    def vjp(self, q_in: torch.Tensor, dts: torch.Tensor, lam_out: torch.Tensor, lam_in: torch.Tensor,
            pbar: torch.Tensor, bbar: torch.Tensor | None = None) -> None:
        rc = self.lib.dclaw_step_adjoint_batched(ctypes.byref(self.batch), _lib.ptr(self.members_dev),
                                                 _lib.ptr(self.params), _lib.ptr(dts), _lib.ptr(q_in),
                                                 _lib.ptr(self.bed), _lib.ptr(lam_out), _lib.ptr(lam_in),
                                                 _lib.ptr(pbar), _lib.ptr(bbar), _lib.ptr(self.work),
                                                 _lib.ptr(self.status), _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_adjoint_batched")

    def check_status(self) -> None:
        for k, st in enumerate(self.status.tolist()):
            _lib.check(int(st), f"ensemble adjoint, member {k}")


def _ensemble(members, theta, fixed_dt: bool, bed: torch.Tensor | None = None):
    from .ensemble import EnsembleStepper, Member

    th = theta.detach().cpu().tolist()
    mem = [Member(m.q, m.b, with_theta(m.params, th[k]), m.dx, m.dy, m.dt_initial, m.t_final,
                  getattr(m, "t_obs", 0.0))
           for k, m in enumerate(members)]
    st = EnsembleStepper(mem, theta.device, fixed_dt=fixed_dt)
    if bed is not None:
        if bed.shape != st.bed.shape:
            raise ValueError(f"bed must be the ensemble's bed arena, shape {tuple(st.bed.shape)}")
        st.bed.copy_(bed.detach())
    return st


def _clock_field(st, k: int) -> torch.Tensor:
    from .params import CLOCK_DOUBLES

    return st.clocks.view(st.n, CLOCK_DOUBLES)[:, k]


class _EnsembleRollout(torch.autograd.Function):
    @staticmethod
    def forward(ctx, q0, theta, members, n_steps, out_steps, checkpoint_block, fixed_dt, dt_schedule, select,
                n_obs, bed):
        st = _ensemble(members, theta, fixed_dt or dt_schedule is not None, bed)
        st.qa.copy_(q0.detach())
        lib = _lib.load()
        reserve = 2 * sum(lib.dclaw_adjoint_workspace_bytes(m.q.shape[2], m.q.shape[1]) for m in members)
        k = _block(n_steps, checkpoint_block, st.qa.numel() * 8, reserve, q0.device)
        dts = torch.empty((n_steps, st.n), dtype=torch.float64, device=q0.device)
        oshape = tuple(q0.shape) if select is None else tuple(select.shape)
        if n_obs:
            # observation slots per gauge entry, each filled when its own
            # member's clock lands on an observation time
            sel64 = select.reshape(-1).to(torch.int64).contiguous()
            sel_h = sel64.cpu().numpy()
            offs = np.array([st.cm[k].q_off for k in range(st.n)], dtype=np.int64)
            ends = offs + 5 * st.mx.astype(np.int64) * st.my.astype(np.int64)
            mem_h = np.searchsorted(offs, sel_h, side="right") - 1
            if (mem_h < 0).any() or (sel_h >= ends[np.maximum(mem_h, 0)]).any():
                raise ValueError("select holds arena entries outside every member")
            member = torch.tensor(mem_h, dtype=torch.int32, device=q0.device)
            outs = torch.zeros((n_obs,) + oshape, dtype=q0.dtype, device=q0.device)
            obs_step = torch.full((n_obs, st.n), -1, dtype=torch.int32, device=q0.device)
        else:
            outs = torch.empty((len(out_steps),) + oshape, dtype=q0.dtype, device=q0.device)
        pick = (lambda t: t) if select is None else (lambda t: t[select])
        where = {}
        for idx, n in enumerate(out_steps):
            where.setdefault(n, []).append(idx)
        for idx in where.get(0, []):
            outs[idx].copy_(pick(q0.detach()))
        # as in _Rollout (arenas zeroed: the gaps between members stay zero)
        store = torch.zeros((max(1, -(-n_steps // k)),) + tuple(st.qa.shape), dtype=torch.float64,
                            device=q0.device)
        store[0].copy_(st.qa)
        ckpt = list(store.unbind(0))
        src = ckpt[0]
        for n in range(n_steps):
            nxt = (n + 1) // k
            if (n + 1) % k == 0 and nxt < len(ckpt):
                dst = ckpt[nxt]
            else:
                dst = st.qa if src is not st.qa else st.qb
            if dt_schedule is not None:
                _clock_field(st, 1).copy_(dt_schedule[n])
            st._launch(src, dst)
            src = dst
            dts[n].copy_(_clock_field(st, 3))
            for idx in where.get(n + 1, []):
                outs[idx].copy_(pick(src))
            if n_obs:
                _lib.check(lib.dclaw_obs_record(_lib.ptr(st.clocks), st.n, _lib.ptr(member), _lib.ptr(src),
                                                _lib.ptr(sel64), sel64.numel(), n_obs, n + 1, _lib.ptr(outs),
                                                _lib.ptr(obs_step), _lib.stream_ptr()), "observation record")
        for kk, s in enumerate(st.status()):
            _lib.check(s, f"ensemble rollout, member {kk}")
        # the bed goes through save_for_backward (None when absent) so that an
        # in-place change between forward and backward raises autograd's
        # version error instead of silently changing the recompute
        ctx.save_for_backward(dts, store, bed)
        ctx.select = select
        ctx.meta = (members, theta.detach(), int(n_steps), tuple(out_steps), k)
        ctx.obs_steps = None
        if n_obs:
            steps = obs_step.cpu().numpy()
            ctx.obs_steps = tuple(tuple(int(v) for v in row) for row in steps)
            # backward: at step n, slot k's entries of the members recorded then
            obs_where = {}
            for kk in range(n_obs):
                for n in sorted(set(int(v) for v in steps[kk] if v >= 0)):
                    ents = np.nonzero(steps[kk][mem_h] == n)[0]
                    obs_where.setdefault(n, []).append((kk, torch.tensor(ents, dtype=torch.int64,
                                                                         device=q0.device)))
            ctx.obs_where = obs_where
        return outs

    @staticmethod
    def backward(ctx, g_out):
        dts, store, bed = ctx.saved_tensors
        bed = None if bed is None else bed.detach()
        ckpt = list(store.unbind(0))
        members, theta, n_steps, out_steps, k = ctx.meta
        dev = dts.device
        where = {}
        for idx, n in enumerate(out_steps):
            where.setdefault(n, []).append(idx)
        fw = _ensemble(members, theta, True, bed)
        adjs = [EnsembleStepAdjoint(fw), EnsembleStepAdjoint(fw)]
        # the bed arena's gradient, when the run was given one that requires grad
        bbar = torch.zeros_like(fw.bed) if bed is not None and ctx.needs_input_grad[10] else None
        lam = torch.zeros_like(fw.qa)
        lam2 = torch.zeros_like(lam)   # arena gaps between members stay zero
        pbar = torch.zeros((fw.n, 4), dtype=torch.float64, device=dev)
        seg = torch.zeros((k,) + tuple(fw.qa.shape), dtype=torch.float64, device=dev) if k > 1 else None
        g_out = g_out.contiguous() if g_out is not None else None
        sel = ctx.select

        def add_out(idx, target):
            if sel is None:
                target.add_(g_out[idx])
            else:
                target.index_add_(0, sel.reshape(-1), g_out[idx].reshape(-1))

        obs_where = getattr(ctx, "obs_where", None) if ctx.obs_steps is not None else None
        sel_flat = sel.reshape(-1) if sel is not None else None

        def add_outs(n, target):
            if g_out is None:
                return
            for idx in where.get(n, []):
                add_out(idx, target)
            if obs_where is not None:
                for kk, ents in obs_where.get(n, []):
                    target.index_add_(0, sel_flat[ents], g_out[kk].reshape(-1)[ents])

        segs = [seg, torch.zeros_like(seg)] if k > 1 else None

        def recompute(s, buf):
            n0, n1 = s * k, min(s * k + k, n_steps)
            src = ckpt[s]
            for n in range(n0 + 1, n1):
                _clock_field(fw, 1).copy_(dts[n - 1])
                fw._launch(src, buf[n - n0])
                src = buf[n - n0]

        lam, lam2 = _pipelined_backward(adjs, n_steps, k, ckpt, segs, recompute, lambda n: dts[n - 1], lam, lam2,
                                        pbar, add_outs, None, bbar)
        add_outs(0, lam)
        for kk, st in enumerate(fw.status()):
            _lib.check(st, f"ensemble recompute, member {kk}")
        for adj in adjs:
            adj.check_status()
        scale = torch.tensor([_DEG, 1.0, 1.0, 1.0], dtype=torch.float64, device=dev)
        return lam, pbar * scale, None, None, None, None, None, None, None, None, bbar


def ensemble_rollout_states(q0: torch.Tensor, theta: torch.Tensor, members, n_steps: int, out_steps,
                            checkpoint_block: int | None = None, fixed_dt: bool = False,
                            dt_schedule: torch.Tensor | None = None, select: torch.Tensor | None = None,
                            bed: torch.Tensor | None = None) -> torch.Tensor:
    """Differentiable run of an ensemble (the batched form of `rollout_states`).

    members: list of `ensemble.Member` (bed, parameters, spacing, first dt;
    their q only sets the layout); q0: the state arena of an
    `EnsembleStepper` over them (float64 CUDA tensor, member k at its q_off);
    theta: (n, 4) float64 tensor, row k = (phi [deg], kref, alpha_c, mu) of
    member k. Returns the arenas after each step count in out_steps, shape
    (len(out_steps), arena size). Every member keeps its own dt (tick rule,
    or fixed; dt_schedule (n_steps, n) replays recorded dts). select (int64
    CUDA tensor of arena indices): return only these entries per output
    step (gauges) instead of whole arenas. The backward pass runs the
    batched step adjoint with time checkpointing (block length as in
    `rollout_states`). bed (optional): the bed arena (an `EnsembleStepper`'s
    `bed` layout) to step over instead of the members' beds; when it
    requires grad it gets every member's bed gradient.
    """
    for n in out_steps:
        if not 0 <= n <= n_steps:
            raise ValueError(f"output step {n} outside 0..{n_steps}")
    if dt_schedule is not None and dt_schedule.shape != (n_steps, len(members)):
        raise ValueError("dt_schedule must be (n_steps, n_members)")
    return _EnsembleRollout.apply(q0, theta, list(members), int(n_steps), tuple(int(n) for n in out_steps),
                                  checkpoint_block, bool(fixed_dt), dt_schedule, select, 0, bed)


def ensemble_rollout_observations(q0: torch.Tensor, theta: torch.Tensor, members, n_steps: int, n_obs: int,
                                  select: torch.Tensor, checkpoint_block: int | None = None,
                                  dt_schedule: torch.Tensor | None = None,
                                  bed: torch.Tensor | None = None) -> torch.Tensor:
    """The batched form of `rollout_observations`, the particle filter's
    vmapped flume loop (pf_flume/inference.py:96-108 over
    pf_flume/flume_model.py:150-158): every member steps with its own tick
    rule clipped at the multiples of its `Member.t_obs` (and at its
    t_final), and each gauge entry of `select` (arena indices) is recorded
    into slot k when its own member lands on (k+1) t_obs. Returns
    (n_obs, *select.shape); entries of slots a member does not reach stay 0.
    `observation_steps(out)` gives, per slot, each member's step."""
    if int(n_obs) < 1 or select is None:
        raise ValueError("n_obs >= 1 and a select of gauge entries are required")
    if not any(getattr(m, "t_obs", 0.0) > 0.0 for m in members):
        raise ValueError("no member has an observation interval (Member.t_obs)")
    if dt_schedule is not None and dt_schedule.shape != (n_steps, len(members)):
        raise ValueError("dt_schedule must be (n_steps, n_members)")
    return _EnsembleRollout.apply(q0, theta, list(members), int(n_steps), (), checkpoint_block, False,
                                  dt_schedule, select, int(n_obs), bed)


def ensemble_last_dts(out: torch.Tensor) -> torch.Tensor:
    """The (n_steps, n_members) dts recorded by the ensemble rollout that produced `out`."""
    return out.grad_fn.saved_tensors[0]
