"""The step adjoint on the GPU (dclaw_step_adjoint through the C ABI) and the
differentiable rollout with sqrt(N) checkpointing.

1. One step: the CUDA adjoint against the host build of the same reverse
   routines (tests/adj), which are checked against central finite
   differences on the CPU runner: the state adjoint bit for bit, the
   parameter adjoints (summed in another order) to 1e-12 relative, over wet,
   dry, resting, boundary, order, transverse, limiter and src2 variants.
2. Runs of steps: gradients of a loss over several output states with
   respect to the initial state and the material parameters against
   central finite differences of the CUDA forward run at the same dt
   schedule (fixed, and replayed from an adaptive run), to 1e-6 relative.
3. Checkpointing: every checkpoint block length gives the same bits.
4. The loss at gauge points over output times, with the gradient reaching
   the initial depth field and the solid fraction through the differentiable
   initial state, against finite differences.
"""
import numpy as np
import pytest
import torch

from dclaw_b200 import workloads as W
from dclaw_b200.adjoint import StepAdjoint, last_dts, rollout_states, theta_of
from dclaw_b200.params import DClawParams

from .test_adjoint_cpu import CASES, _case

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def host_adj():
    from ._adj import Adj

    return Adj()


@pytest.mark.parametrize("name", list(CASES))
def test_step_adjoint_matches_host_build(cuda_device, host_adj, name):
    p, q, b = _case(**CASES[name])
    dx, dt = 1.0, 0.02
    rng = np.random.default_rng(100)
    lam = rng.standard_normal(q.shape)
    li_h, pb_h = host_adj.vjp(p, q, b, dx, dx, dt, lam)
    dev = cuda_device
    adj = StepAdjoint(torch.tensor(b, device=dev), p, dx, dx)
    lam_in = torch.empty(q.shape, dtype=torch.float64, device=dev)
    pbar = torch.zeros(4, dtype=torch.float64, device=dev)
    dtt = torch.tensor([dt], dtype=torch.float64, device=dev)
    adj.vjp(torch.tensor(q, device=dev), dtt, torch.tensor(lam, device=dev), lam_in, pbar)
    torch.cuda.synchronize()
    adj.check_status()
    li = lam_in.cpu().numpy()
    assert np.array_equal(li, li_h), f"max |diff| {np.abs(li - li_h).max():.3e}"
    pb = pbar.cpu().numpy()
    assert np.allclose(pb, pb_h, rtol=1e-12, atol=1e-300), (pb, pb_h)
    # the bed's adjoint: bit for bit with the host build, nothing else changed
    _, _, bb_h = host_adj.vjp(p, q, b, dx, dx, dt, lam, bed=True)
    lam_in_b = torch.empty_like(lam_in)
    pbar_b = torch.zeros(4, dtype=torch.float64, device=dev)
    bbar = torch.zeros(b.shape, dtype=torch.float64, device=dev)
    adj.vjp(torch.tensor(q, device=dev), dtt, torch.tensor(lam, device=dev), lam_in_b, pbar_b, bbar)
    assert torch.equal(lam_in_b, lam_in) and torch.equal(pbar_b, pbar)
    assert np.array_equal(bbar.cpu().numpy(), bb_h), f"bed: max |diff| {np.abs(bbar.cpu().numpy() - bb_h).max():.3e}"
    # a second call gives the same bits (no atomics in the sums)
    pbar2 = torch.zeros(4, dtype=torch.float64, device=dev)
    lam_in2 = torch.empty_like(lam_in)
    adj.vjp(torch.tensor(q, device=dev), dtt, torch.tensor(lam, device=dev), lam_in2, pbar2)
    assert torch.equal(lam_in, lam_in2) and torch.equal(pbar, pbar2)


def _small_flow(seed=1, mx=24, my=20, dry_frac=0.25):
    """A moving wet patch with a dry region, on a sloping bed."""
    p, q, b = _case(seed=seed, mx=mx, my=my, dry_frac=0.0)
    X, Y = np.meshgrid(np.arange(mx), np.arange(my))
    dry = (X + 0.7 * Y) > (1.0 - dry_frac) * (mx + 0.7 * my)
    q[:, dry] = 0.0
    return p, q, b


def _loss_weights(q, n_out, seed=5):
    """Random weights scaled by each field's magnitude, so every field's
    terms are O(1) and the loss's rounding stays far below its derivatives."""
    rng = np.random.default_rng(seed)
    w = rng.standard_normal((n_out,) + q.shape)
    sc = np.abs(q).reshape(5, -1).max(1)
    return w / sc[None, :, None, None]


def _fd(f, eps0=1e-6, down=4, up=8):
    """Central difference (f(e) - f(-e)) / 2e and its uncertainty.

    Estimates are taken at e = eps0 * 2^k for k = -down .. up, and the pair
    of neighbouring step sizes (e, 2e) whose estimates agree best is kept:
    returns (estimate at e, |difference of the pair|). Two errors pull the
    step size in opposite ways. A step that straddles a kink of the forward
    map (limiter regimes, the dry tolerance and min/max picks put kinks
    within 1e-6 relative of ordinary states) measures a chord, not the
    derivative the adjoint gives, so smaller steps help; rounding noise
    (every perturbed run rounds its elementary functions afresh, step after
    step) divided by e grows as e shrinks, so larger steps help. Two step
    sizes that agree bound the estimate's error; the caller checks that
    bound against its tolerance rather than widening the tolerance by it."""
    cache = {}

    def cd(e):
        if e not in cache:
            cache[e] = (f(e) - f(-e)) / (2 * e)
        return cache[e]

    es = [eps0 * 2.0**k for k in range(-down, up + 1)]
    best = None
    for k in range(len(es) - 1):
        lo, hi = cd(es[k]), cd(es[k + 1])
        spread = abs(hi - lo)
        rel = spread / max(abs(lo), 1e-300)
        if best is None or rel < best[2]:
            best = (lo, spread, rel)
    return best[0], best[1]


def _close(ad, fd, what, rtol=1e-6):
    """AD against a finite difference to rtol, with the finite difference
    itself settled to a quarter of rtol (two step sizes agreeing to that)."""
    est, spread = fd
    msg = f"{what}: AD {ad:.12e} FD {est:.12e} (FD spread {spread:.2e}, {spread / max(abs(est), 1e-300):.2e} rel)"
    print(msg)
    assert spread <= 0.25 * rtol * abs(est), "finite differences did not settle: " + msg
    assert abs(ad - est) <= rtol * abs(est), msg


def _run_loss(q0, theta, b, p, dx, n, outs, wts, **kw):
    o = rollout_states(q0, theta, b, p, dx, dx, n, outs, **kw)
    return (o * wts).sum(), o


@pytest.mark.parametrize("mode", ["fixed", "adaptive"])
def test_rollout_gradient_matches_finite_differences(cuda_device, mode):
    dev = cuda_device
    p, qn, bn = _small_flow()
    if mode == "adaptive":
        # tick rule at Courant number 0.4: at 0.9 the run's rounding noise,
        # amplified over 16 large steps, leaves the finite differences of
        # the small parameters (kref, mu) uncertain by ~5e-6 relative
        p = p.replace(cfl_desired=0.4)
    dx = 1.0
    n, outs = 16, [4, 9, 16]
    q0 = torch.tensor(qn, device=dev, requires_grad=True)
    b = torch.tensor(bn, device=dev)
    theta = theta_of(p, dev).requires_grad_(True)
    wts = torch.tensor(_loss_weights(qn, len(outs)), device=dev)
    kw = dict(dt0=0.02, fixed_dt=True) if mode == "fixed" else dict(dt0=0.02, fixed_dt=False)
    L, o = _run_loss(q0, theta, b, p, dx, n, outs, wts, **kw)
    sched = last_dts(o).clone()
    L.backward()
    gq, gt = q0.grad.clone(), theta.grad.clone()
    assert torch.isfinite(gq).all() and torch.isfinite(gt).all()

    def Lf(qq, th):
        with torch.no_grad():
            return float(_run_loss(qq, th, b, p, dx, n, outs, wts, dt0=0.0, dt_schedule=sched)[0])

    # initial state: a direction over wet cells only (dry cells stay dry)
    rng = np.random.default_rng(7)
    d = rng.standard_normal(qn.shape) * (np.abs(qn) + 1e-3)
    d[:, qn[0] <= 10 * p.dry_tolerance] = 0.0
    d = torch.tensor(d, device=dev)
    q00, th0 = q0.detach(), theta.detach()
    _close(float((gq * d).sum()), _fd(lambda e: Lf(q00 + e * d, th0)), "state")
    # parameters, one at a time
    for k, scale in enumerate([1.0, p.kref, p.alpha_c, p.mu]):
        e = torch.zeros(4, dtype=torch.float64, device=dev)
        e[k] = scale
        _close(float(gt[k]) * scale, _fd(lambda h: Lf(q00, th0 + h * e), eps0=4e-6), f"theta[{k}]")


def test_rollout_bed_gradient(cuda_device):
    """The gradient with respect to a fixed bed over a checkpointed run
    matches finite differences at the fixed dt, and is the same with every
    state kept and with checkpoint blocks."""
    dev = cuda_device
    p, qn, bn = _small_flow(seed=12)
    n, outs = 16, [8, 16]
    wts = torch.tensor(_loss_weights(qn, len(outs), seed=6), device=dev)
    res = []
    for blk in (1, 4):
        q0 = torch.tensor(qn, device=dev, requires_grad=True)
        theta = theta_of(p, dev)
        b = torch.tensor(bn, device=dev, requires_grad=True)
        L, o = _run_loss(q0, theta, b, p, 1.0, n, outs, wts, dt0=0.02, fixed_dt=True, checkpoint_block=blk)
        L.backward()
        res.append((b.grad.clone(), q0.grad.clone()))
    assert torch.equal(res[0][0], res[1][0]) and torch.equal(res[0][1], res[1][1])
    gb = res[0][0]
    assert gb.abs().max() > 0

    def Lf(bb):
        with torch.no_grad():
            return float(_run_loss(torch.tensor(qn, device=dev), theta_of(p, dev), bb, p, 1.0, n, outs, wts,
                                   dt0=0.02, fixed_dt=True)[0])

    rng = np.random.default_rng(14)
    db = torch.tensor(rng.standard_normal(bn.shape), device=dev)
    b0 = torch.tensor(bn, device=dev)
    _close(float((gb * db).sum()), _fd(lambda e: Lf(b0 + e * db)), "bed")


def test_rollout_gradient_with_a_moving_gate_bed(cuda_device):
    """The port's flume runs step under a moving gate, bed(t) (gate_bed):
    the differentiable run evaluates the bed before every step, its states
    equal stepping with the bed rebuilt each step, and its gradients match
    finite differences at the recorded dt schedule, with every state kept
    and with checkpoint blocks."""
    from dclaw_b200.solver import PatchStepper, gate_bed

    dev = cuda_device
    p, qn, bn = _small_flow(seed=5)
    b0 = torch.tensor(bn, device=dev)
    ridge = torch.zeros_like(b0)
    ridge[:, 10:12] = 0.5                        # a gate across the flow, opening over 0.2 s (10 steps)
    bed = gate_bed(b0, ridge, [0.0, 0.2], [0.0, 90.0])
    n, outs = 16, [8, 16]
    wts = torch.tensor(_loss_weights(qn, len(outs), seed=4), device=dev)
    res = []
    for blk in (1, 4):
        q0 = torch.tensor(qn, device=dev, requires_grad=True)
        theta = theta_of(p, dev).requires_grad_(True)
        L, o = _run_loss(q0, theta, bed, p, 1.0, n, outs, wts, dt0=0.02, fixed_dt=True, checkpoint_block=blk)
        L.backward()
        res.append((o.detach(), q0.grad.clone(), theta.grad.clone()))
    assert all(torch.equal(x, y) for x, y in zip(res[0], res[1])), "checkpoint blocks differ"
    o, gq, gt = res[0]
    # the forward states: the fused step with the bed rebuilt before every step
    st = PatchStepper(torch.tensor(qn, device=dev), bed(torch.zeros((), dtype=torch.float64, device=dev)), p,
                      1.0, 1.0)
    st.init_clock(0.02, fixed_dt=True)
    for k in range(n):
        st.b.copy_(bed(st.clock[0]))
        st.step(1)
        if k + 1 == 8:
            assert torch.equal(st.state(), o[0])
    assert torch.equal(st.state(), o[1])
    # gradients against finite differences
    sched = torch.full((n,), 0.02, dtype=torch.float64, device=dev)

    def Lf(qq, th):
        with torch.no_grad():
            return float(_run_loss(qq, th, bed, p, 1.0, n, outs, wts, dt0=0.0, dt_schedule=sched)[0])

    rng = np.random.default_rng(11)
    d = rng.standard_normal(qn.shape) * (np.abs(qn) + 1e-3)
    d[:, qn[0] <= 10 * p.dry_tolerance] = 0.0
    d = torch.tensor(d, device=dev)
    q00, th0 = torch.tensor(qn, device=dev), theta_of(p, dev)
    _close(float((gq * d).sum()), _fd(lambda e: Lf(q00 + e * d, th0)), "state")
    e0 = torch.zeros(4, dtype=torch.float64, device=dev)
    e0[0] = 1.0
    _close(float(gt[0]), _fd(lambda h: Lf(q00, th0 + h * e0), eps0=4e-6), "phi")


def test_gate_parameter_gradients(cuda_device):
    """The port differentiates its flume runs with respect to the gate
    (gate_bed's ridge, opening times and angles, differentiable_dclaw/
    dclaw_jax/solver.py:304-322). With bed_params the moving bed's step
    adjoints go back through every step's b(t_n): the gradients of the
    ridge height, an opening time and an angle match finite differences at
    the recorded schedule."""
    from dclaw_b200.solver import gate_bed

    dev = cuda_device
    p, qn, bn = _small_flow(seed=5)
    b0 = torch.tensor(bn, device=dev)
    ridge = torch.zeros_like(b0)
    ridge[:, 10:12] = 1.0
    n, outs = 16, [8, 16]
    wts = torch.tensor(_loss_weights(qn, len(outs), seed=4), device=dev)
    sched = torch.full((n,), 0.02, dtype=torch.float64, device=dev)

    def run(amp, gt, gd):
        bed = gate_bed(b0, amp * ridge, gt, gd)
        q0 = torch.tensor(qn, device=dev)
        return _run_loss(q0, theta_of(p, dev), bed, p, 1.0, n, outs, wts, dt0=0.0, dt_schedule=sched,
                         bed_params=(amp, gt, gd))[0]

    amp = torch.tensor(0.5, dtype=torch.float64, device=dev, requires_grad=True)
    gt = torch.tensor([0.013, 0.231], dtype=torch.float64, device=dev, requires_grad=True)
    gd = torch.tensor([0.0, 90.0], dtype=torch.float64, device=dev, requires_grad=True)
    L = run(amp, gt, gd)
    L.backward()
    a0, t0, d0 = amp.detach(), gt.detach(), gd.detach()

    def Lf(a, t, d):
        with torch.no_grad():
            return float(run(a, t, d))

    e1 = torch.tensor([0.0, 1.0], dtype=torch.float64, device=dev)
    _close(float(amp.grad), _fd(lambda e: Lf(a0 + e, t0, d0), eps0=1e-6), "ridge height")
    _close(float(gt.grad[1]), _fd(lambda e: Lf(a0, t0 + e * e1, d0), eps0=1e-6), "opening time")
    _close(float(gd.grad[1]), _fd(lambda e: Lf(a0, t0, d0 + e * e1), eps0=1e-4), "opening angle")


def test_rollout_with_observation_interval(cuda_device):
    """rollout_states(obs_dt=...) steps with the clock clipping dt at every
    observation time: its states equal the fused step's with that clock,
    its dt schedule lands on the observation times, and the recorded
    schedule replays the same run for the gradient."""
    from dclaw_b200.solver import PatchStepper

    dev = cuda_device
    p, qn, bn = _small_flow(seed=3)
    b = torch.tensor(bn, device=dev)
    n, outs, t_obs = 24, [12, 24], 0.03
    wts = torch.tensor(_loss_weights(qn, len(outs), seed=2), device=dev)
    q0 = torch.tensor(qn, device=dev, requires_grad=True)
    theta = theta_of(p, dev).requires_grad_(True)
    L, o = _run_loss(q0, theta, b, p, 1.0, n, outs, wts, dt0=0.02, obs_dt=t_obs)
    sched = last_dts(o).clone()
    L.backward()
    st = PatchStepper(torch.tensor(qn, device=dev), b, p, 1.0, 1.0)
    st.init_clock(0.02, t_obs=t_obs)
    st.step(12)
    assert torch.equal(st.state(), o[0])
    st.step(12)
    assert torch.equal(st.state(), o[1])
    t = st.read_clock().t
    tt = np.cumsum(sched.cpu().numpy())
    assert tt[-1] == t
    assert all(np.abs(tt - m * t_obs).min() < 1e-9 for m in range(1, int(t / t_obs + 1e-9) + 1))
    with torch.no_grad():
        L2, _ = _run_loss(torch.tensor(qn, device=dev), theta_of(p, dev), b, p, 1.0, n, outs, wts, dt0=0.0,
                          dt_schedule=sched)
    assert float(L2) == float(L.detach())
    q1 = torch.tensor(qn, device=dev, requires_grad=True)
    th1 = theta_of(p, dev).requires_grad_(True)
    L3, _ = _run_loss(q1, th1, b, p, 1.0, n, outs, wts, dt0=0.0, dt_schedule=sched)
    L3.backward()
    assert torch.equal(q1.grad, q0.grad) and torch.equal(th1.grad, theta.grad)


def test_rollout_observations(cuda_device):
    """rollout_observations records slot k when t lands on (k+1) obs_dt (the
    port's flume loop): the slots equal the fused step's states at those
    steps, slots past the run stay 0, and the gradient of a loss over the
    slots matches finite differences at the recorded dt schedule (which
    replays the same landings)."""
    from dclaw_b200.adjoint import observation_steps, rollout_observations
    from dclaw_b200.solver import PatchStepper

    dev = cuda_device
    p, qn, bn = _small_flow(seed=6)
    p = p.replace(cfl_desired=0.4)
    b = torch.tensor(bn, device=dev)
    n, obs_dt, n_obs = 30, 0.05, 40
    rng = np.random.default_rng(9)
    sel = torch.tensor(rng.choice(qn.size, 40, replace=False), device=dev)
    wts = torch.tensor(rng.standard_normal((n_obs, 40)), device=dev)
    q0 = torch.tensor(qn, device=dev, requires_grad=True)
    theta = theta_of(p, dev).requires_grad_(True)
    o = rollout_observations(q0, theta, b, p, 1.0, 1.0, n, obs_dt, n_obs, 0.02, select=sel)
    steps = observation_steps(o)
    sched = last_dts(o).clone()
    L = (o * wts).sum()
    L.backward()
    # the slots against stepping one step at a time with the same clock
    st = PatchStepper(torch.tensor(qn, device=dev), b, p, 1.0, 1.0)
    st.init_clock(0.02, t_obs=obs_dt)
    got = {}
    for k in range(n):
        st.step(1)
        c = st.read_clock()
        j = int(np.rint(c.t / obs_dt)) - 1
        if c.dt_last > 0 and 0 <= j < n_obs and abs(c.t - (j + 1) * obs_dt) < 1e-9:
            got[j] = (k + 1, st.state().reshape(-1)[sel].clone())
    assert len(got) >= 4 and any(s < 0 for s in steps)
    for j in range(n_obs):
        if j in got:
            assert steps[j] == got[j][0] and torch.equal(o.detach()[j], got[j][1])
        else:
            assert steps[j] == -1 and not o.detach()[j].any()

    def Lf(qq, th):
        with torch.no_grad():
            oo = rollout_observations(qq, th, b, p, 1.0, 1.0, n, obs_dt, n_obs, 0.0, select=sel, dt_schedule=sched)
            return float((oo * wts).sum())

    assert Lf(q0.detach(), theta.detach()) == float(L.detach())
    d = rng.standard_normal(qn.shape) * (np.abs(qn) + 1e-3)
    d[:, qn[0] <= 10 * p.dry_tolerance] = 0.0
    d = torch.tensor(d, device=dev)
    q00, th0 = q0.detach(), theta.detach()
    _close(float((q0.grad * d).sum()), _fd(lambda e: Lf(q00 + e * d, th0)), "state")
    e0 = torch.zeros(4, dtype=torch.float64, device=dev)
    e0[0] = 1.0
    _close(float(theta.grad[0]), _fd(lambda h: Lf(q00, th0 + h * e0), eps0=4e-6), "phi")


def test_rollout_peak_gradient(cuda_device):
    """adjoint.rollout_peak, the loss input of the port's rollout_peak: the
    running peak depth equals the maximum over stepped states, bit for bit,
    with every state kept and with checkpoint blocks. Its gradient is the
    gradient of the same loss over rollout_states outputs with each cell's
    term taken at the step that set its peak (rollout_states' gradients are
    checked against finite differences above; finite differences of a
    maximum straddle its kinks wherever two steps nearly tie)."""
    from dclaw_b200.adjoint import rollout_peak
    from dclaw_b200.solver import PatchStepper

    dev = cuda_device
    p, qn, bn = _small_flow(seed=8)
    b = torch.tensor(bn, device=dev)
    n = 16
    rng = np.random.default_rng(21)
    w = torch.tensor(rng.standard_normal(qn.shape[1:]), device=dev)
    res = []
    for blk in (1, 4):
        q0 = torch.tensor(qn, device=dev, requires_grad=True)
        theta = theta_of(p, dev).requires_grad_(True)
        hp = rollout_peak(q0, theta, b, p, 1.0, 1.0, n, 0.02, fixed_dt=True, checkpoint_block=blk)
        (hp * w).sum().backward()
        res.append((hp.detach(), q0.grad.clone(), theta.grad.clone()))
    assert all(torch.equal(x, y) for x, y in zip(res[0], res[1])), "checkpoint blocks differ"
    hp, gq, gt = res[0]
    st = PatchStepper(torch.tensor(qn, device=dev), b, p, 1.0, 1.0)
    st.init_clock(0.02, fixed_dt=True)
    ref = torch.tensor(qn[0], device=dev)
    arg = torch.zeros(ref.shape, dtype=torch.int64, device=dev)
    for k in range(n):
        st.step(1)
        h = st.state()[0]
        arg = torch.where(h > ref, torch.full_like(arg, k + 1), arg)
        ref = torch.maximum(ref, h)
    assert torch.equal(hp, ref)
    assert len(torch.unique(arg)) > 3
    # the same loss with each cell's term at the step that set its peak
    q1 = torch.tensor(qn, device=dev, requires_grad=True)
    th1 = theta_of(p, dev).requires_grad_(True)
    o = rollout_states(q1, th1, b, p, 1.0, 1.0, n, list(range(n + 1)), 0.02, fixed_dt=True)
    mask = (arg.unsqueeze(0) == torch.arange(n + 1, device=dev).view(-1, 1, 1)).to(torch.float64)
    (o[:, 0] * mask * w).sum().backward()
    assert torch.allclose(gq, q1.grad, rtol=1e-12, atol=1e-300)
    assert torch.allclose(gt, th1.grad, rtol=1e-12, atol=0.0)


def test_checkpoint_block_gives_identical_gradients(cuda_device):
    dev = cuda_device
    p, qn, bn = _small_flow(seed=2)
    b = torch.tensor(bn, device=dev)
    n, outs = 23, [0, 5, 11, 23]
    wts = torch.tensor(_loss_weights(qn, len(outs), seed=9), device=dev)
    res = []
    for blk in (1, 3, 5, 23, None):
        q0 = torch.tensor(qn, device=dev, requires_grad=True)
        theta = theta_of(p, dev).requires_grad_(True)
        L, _ = _run_loss(q0, theta, b, p, 1.0, n, outs, wts, dt0=0.02, checkpoint_block=blk)
        L.backward()
        res.append((float(L.detach()), q0.grad.clone(), theta.grad.clone()))
    for r in res[1:]:
        assert r[0] == res[0][0]
        assert torch.equal(r[1], res[0][1])
        assert torch.equal(r[2], res[0][2])


def test_gauge_loss_gradient(cuda_device):
    """Loss over gauge cells and output times against a target run at other
    parameters (the shape of the 512 x 512 gradient case); the gradient
    reaches the window's depth field per cell, a solid fraction m0 that sets
    hm = h m0, and theta. The window starts from a flow in motion (40 steps
    after release from rest): from rest, calc_taudir's static-friction
    switch (factor of safety 0 or 1, digclaw_module.f90:500-719) makes the
    loss jump under any perturbation, and no finite difference is defined."""
    from oracle import Oracle

    dev = cuda_device
    n_cells, pre, n = 40, 40, 30
    bn = W.random_terrain(n_cells, 1.0, seed=7)
    p = DClawParams()
    X, Y = np.meshgrid(np.arange(n_cells) + 0.5, np.arange(n_cells) + 0.5)
    h0n = np.maximum(1.5 * (1.0 - ((X - 20) ** 2 + (Y - 20) ** 2) / 10.0**2), 0.0)
    q_rest = W.state_from(h0n, np.full_like(h0n, 0.62), p, 0.8)
    qp = Oracle().run(p, q_rest, bn, 1.0, 1.0, pre, 0.05, libm="portable")["q"]
    b = torch.tensor(bn, device=dev)
    outs = list(range(3, n + 1, 3))
    rng = np.random.default_rng(11)
    gi_t = torch.tensor(rng.integers(10, 30, size=8), device=dev)
    gj_t = torch.tensor(rng.integers(10, 30, size=8), device=dev)
    qpt = torch.tensor(qp, device=dev)
    wet = qpt[0] > p.dry_tolerance

    def start(h, m0):
        return torch.stack([h, qpt[1], qpt[2], torch.where(wet, h * m0, 0.0), qpt[4]])

    def run(h, m0, theta, sched=None):
        kw = dict(dt0=0.0, dt_schedule=sched) if sched is not None else dict(dt0=0.05)
        o = rollout_states(start(h, m0), theta, b, p, 1.0, 1.0, n, outs, **kw)
        return o[:, 0, gj_t, gi_t], o

    with torch.no_grad():
        target, _ = run(qpt[0], torch.tensor(0.6, dtype=torch.float64, device=dev),
                        theta_of(p.replace(phi=30.0, kref=3e-10), dev))
    h = qpt[0].clone().requires_grad_(True)
    m0 = torch.tensor(0.62, dtype=torch.float64, device=dev, requires_grad=True)
    theta = theta_of(p, dev).requires_grad_(True)
    g, o = run(h, m0, theta)
    L = ((g - target) ** 2).sum()
    sched = last_dts(o).clone()
    L.backward()
    assert float(L.detach()) > 0.0

    def Lf(hh, mm, th):
        with torch.no_grad():
            gg, _ = run(hh, mm, th, sched)
            return float(((gg - target) ** 2).sum())

    h00, m00, th0 = h.detach(), m0.detach(), theta.detach()
    d = torch.tensor(np.where(qp[0] > 0.2, rng.standard_normal(qp[0].shape), 0.0), device=dev)
    _close(float((h.grad * d).sum()), _fd(lambda e: Lf(h00 + e * d, m00, th0)), "h")
    _close(float(m0.grad), _fd(lambda e: Lf(h00, m00 + e, th0), eps0=4e-6), "m0")
    # this loss hardly feels the material parameters over 30 steps (relative
    # sensitivities ~1e-3 of the depth's), so their finite differences carry
    # ~1e-4 relative rounding noise; theta is checked at 1e-6 in
    # test_rollout_gradient_matches_finite_differences
    for k, scale in enumerate([1.0, p.kref, p.alpha_c, p.mu]):
        e = torch.zeros(4, dtype=torch.float64, device=dev)
        e[k] = scale
        _close(float(theta.grad[k]) * scale, _fd(lambda hh: Lf(h00, m00, th0 + hh * e), eps0=4e-6), f"theta[{k}]",
               rtol=1e-4)


def test_unsupported_options_are_refused(cuda_device):
    from dclaw_b200 import _lib

    b = torch.zeros((8, 8), dtype=torch.float64, device=cuda_device)
    with pytest.raises(_lib.DClawError):
        StepAdjoint(b, DClawParams(src2method=2, alphamethod=1), 1.0, 1.0)
    with pytest.raises(_lib.DClawError):
        StepAdjoint(b, DClawParams(segregation=1), 1.0, 1.0)
    # Manning friction and the rare-wave corrector have their reverses
    StepAdjoint(b, DClawParams(friction_forcing=True, manning_coefficient=0.03), 1.0, 1.0)
    StepAdjoint(b, DClawParams(rarecorrectortest=True), 1.0, 1.0)


def test_prepare_then_reverse_equals_the_whole_step_adjoint(cuda_device):
    """dclaw_step_adjoint_prepare + _reverse (the two parts the backward
    pass overlaps) give dclaw_step_adjoint's bits, with another step
    prepared in a second workspace in between."""
    p, qn, bn = _small_flow(seed=4)
    dev = cuda_device
    b = torch.tensor(bn, device=dev)
    rng = np.random.default_rng(8)
    q1 = torch.tensor(qn, device=dev)
    q2 = torch.tensor(qn * (1.0 + 0.01 * rng.standard_normal(qn.shape)).clip(min=0.0), device=dev)
    lam = torch.tensor(rng.standard_normal(qn.shape), device=dev)
    dt1 = torch.tensor([0.02], dtype=torch.float64, device=dev)
    dt2 = torch.tensor([0.015], dtype=torch.float64, device=dev)
    ref = StepAdjoint(b, p, 1.0, 1.0)
    li_ref, pb_ref = torch.empty_like(lam), torch.zeros(4, dtype=torch.float64, device=dev)
    ref.vjp(q1, dt1, lam, li_ref, pb_ref)
    a, other = StepAdjoint(b, p, 1.0, 1.0), StepAdjoint(b, p, 1.0, 1.0)
    li, pb = torch.empty_like(lam), torch.zeros(4, dtype=torch.float64, device=dev)
    a.prepare(q1, dt1)
    other.prepare(q2, dt2)
    a.reverse(q1, dt1, lam, li, pb)
    torch.cuda.synchronize()
    for x in (ref, a, other):
        x.check_status()
    assert torch.equal(li, li_ref) and torch.equal(pb, pb_ref)


def test_nan_anywhere_in_the_state_is_reported(cuda_device):
    """A NaN in any field of any cell, near the flow or far from it, sets the
    adjoint's status word (as the forward step's check4nans scan does); a
    clean state leaves it at zero."""
    from dclaw_b200 import _lib

    dev = cuda_device
    p, qn, bn = _small_flow(seed=3)
    b = torch.tensor(bn, device=dev)
    adj = StepAdjoint(b, p, 1.0, 1.0)
    dtt = torch.tensor([0.01], dtype=torch.float64, device=dev)
    lam = torch.ones(qn.shape, dtype=torch.float64, device=dev)
    for where in [None, (3, 0, 0), (4, qn.shape[1] - 1, qn.shape[2] - 1)]:
        q = torch.tensor(qn, device=dev)
        if where is not None:
            q[where] = float("nan")
        adj.status.zero_()
        adj.vjp(q, dtt, lam, torch.empty_like(lam), torch.zeros(4, dtype=torch.float64, device=dev))
        if where is None:
            adj.check_status()
        else:
            with pytest.raises(_lib.DClawError):
                adj.check_status()


def test_select_outputs_give_the_same_gradient(cuda_device):
    """Returning only selected entries (gauges) at the output steps gives the
    gradient of the same loss computed from whole output states."""
    dev = cuda_device
    p, qn, bn = _small_flow(seed=3)
    b = torch.tensor(bn, device=dev)
    n, outs = 12, [4, 8, 12]
    rng = np.random.default_rng(6)
    sel = torch.tensor(rng.choice(qn.size, size=40, replace=False), device=dev)
    res = []
    for use_sel in (False, True):
        q0 = torch.tensor(qn, device=dev, requires_grad=True)
        theta = theta_of(p, dev).requires_grad_(True)
        if use_sel:
            o = rollout_states(q0, theta, b, p, 1.0, 1.0, n, outs, 0.02, select=sel)
        else:
            o = rollout_states(q0, theta, b, p, 1.0, 1.0, n, outs, 0.02).reshape(len(outs), -1)[:, sel]
        L = (o ** 2).sum()
        L.backward()
        res.append((o.detach(), q0.grad.clone(), theta.grad.clone()))
    assert torch.equal(res[0][0], res[1][0])
    assert torch.equal(res[0][1], res[1][1]) and torch.equal(res[0][2], res[1][2])
