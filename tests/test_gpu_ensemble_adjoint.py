"""The batched step adjoint (dclaw_step_adjoint_batched through the C ABI)
and the differentiable ensemble rollout, against the single-patch adjoint
member by member: the batched launches run the same item stages on every
member's own layout, parameters and dt, over the 16 x 16 blocks where the
member is wet (and the blocks beside them), so state adjoints and whole
checkpointed state gradients are bit-identical to dclaw_step_adjoint on each
member alone. The parameter adjoints are block sums grouped by activity
block instead of by 128-item chunk: equal to 1e-12 relative, and the same
bits from call to call. The single-patch adjoint is checked against finite
differences in test_gpu_adjoint.py."""
import numpy as np
import pytest
import torch

from dclaw_b200 import workloads as W
from dclaw_b200.adjoint import (EnsembleStepAdjoint, StepAdjoint, ensemble_rollout_observations,
                                ensemble_rollout_states, observation_steps, rollout_observations, rollout_states,
                                theta_of)
from dclaw_b200.ensemble import EnsembleStepper, Member

pytestmark = pytest.mark.gpu


def _members(seed=5):
    """Uneven members, each with its own parameters and first dt; all in motion
    after a few steps of their release."""
    out = []
    for c in W.flume_ensemble(n=3, seed=seed, width_range=(6, 20), length_range=(40, 90)):
        out.append(Member(c.q, c.b, c.params, c.dx, c.dy, 2.0e-3))
    rf = W.random_field_case(n=40, dx=0.5, seed=seed + 1)
    p = rf.params.replace(bc_lower=("wall", "extrap"), bc_upper=("extrap", "wall"), transverse_waves=1,
                          phi=34.0, kref=2e-10)
    out.append(Member(rf.q, rf.b, p, rf.dx, rf.dy, 0.01))
    rf2 = W.random_field_case(n=32, dx=0.5, seed=seed + 2)
    out.append(Member(rf2.q[:, :21, :].copy(), rf2.b[:21, :].copy(), rf2.params.replace(order=1, limiter=1),
                      0.5, 0.25, 0.005))
    return out


def _advance(members, dev, n=12):
    """The members' states after n steps (moving flows) as new members."""
    ens = EnsembleStepper(members, dev)
    ens.step(n)
    return [Member(ens.state(k).cpu().numpy(), m.b, m.params, m.dx, m.dy, m.dt_initial)
            for k, m in enumerate(members)]


def _close_params(a, b, what):
    assert torch.allclose(a, b, rtol=1e-12, atol=0.0), f"{what}: {a.tolist()} vs {b.tolist()}"


def _mostly_dry(seed=9):
    """Long flumes whose release blocks cover a few of their 16 x 16 blocks,
    so that most blocks are inactive and the list edges matter."""
    out = []
    for c in W.flume_ensemble(n=3, seed=seed, width_range=(40, 70), length_range=(300, 420)):
        out.append(Member(c.q, c.b, c.params, c.dx, c.dy, 2.0e-3))
    return out


@pytest.mark.parametrize("which", ["uneven", "mostly_dry"])
def test_batched_step_adjoint_matches_single_patch(cuda_device, which):
    dev = cuda_device
    members = _advance(_members() if which == "uneven" else _mostly_dry(), dev)
    ens = EnsembleStepper(members, dev)
    adj = EnsembleStepAdjoint(ens)
    rng = np.random.default_rng(3)
    lam = torch.tensor(rng.standard_normal(ens.qa.numel()), device=dev)
    dts = torch.tensor([0.004 + 0.001 * k for k in range(ens.n)], dtype=torch.float64, device=dev)
    lam_in = torch.zeros_like(lam)
    pbar = torch.zeros((ens.n, 4), dtype=torch.float64, device=dev)
    adj.vjp(ens.qa, dts, lam, lam_in, pbar)
    torch.cuda.synchronize()
    adj.check_status()
    # a second call gives the same bits (fixed summation order)
    lam_in2, pbar2 = torch.zeros_like(lam), torch.zeros_like(pbar)
    adj.vjp(ens.qa, dts, lam, lam_in2, pbar2)
    assert torch.equal(lam_in, lam_in2) and torch.equal(pbar, pbar2)
    for k, m in enumerate(members):
        o, c = ens.cm[k].q_off, m.q.size
        sa = StepAdjoint(torch.tensor(m.b, device=dev), m.params, m.dx, m.dy)
        li = torch.empty(m.q.shape, dtype=torch.float64, device=dev)
        pb = torch.zeros(4, dtype=torch.float64, device=dev)
        sa.vjp(ens.qa[o:o + c].view(m.q.shape), dts[k:k + 1], lam[o:o + c].view(m.q.shape).contiguous(), li, pb)
        assert torch.equal(lam_in[o:o + c].view(m.q.shape), li), f"member {k}: state adjoint differs"
        _close_params(pbar[k], pb, f"member {k}: parameter adjoint")


def test_ensemble_gradient_matches_single_patch_gradients(cuda_device):
    """Per-member losses over output times; the batched checkpointed gradient
    equals each member's unbatched rollout_states gradient: states and state
    gradients bit for bit, parameter gradients to 1e-12."""
    dev = cuda_device
    members = _advance(_members(seed=9), dev, n=8)
    ens = EnsembleStepper(members, dev)
    n, outs = 14, [3, 7, 14]
    q0 = ens.qa.clone().requires_grad_(True)
    theta = torch.stack([theta_of(m.params, dev) for m in members]).requires_grad_(True)
    rng = np.random.default_rng(4)
    wts = torch.tensor(rng.standard_normal((len(outs), ens.qa.numel())), device=dev)
    o = ensemble_rollout_states(q0, theta, members, n, outs, checkpoint_block=4)
    L = (o * wts).sum()
    L.backward()
    for k, m in enumerate(members):
        off, c = ens.cm[k].q_off, m.q.size
        qk = torch.tensor(m.q, device=dev, requires_grad=True)
        tk = theta_of(m.params, dev).requires_grad_(True)
        ok = rollout_states(qk, tk, torch.tensor(m.b, device=dev), m.params, m.dx, m.dy, n, outs,
                            m.dt_initial, checkpoint_block=5)
        Lk = (ok * wts[:, off:off + c].view((len(outs),) + m.q.shape)).sum()
        Lk.backward()
        assert torch.equal(o.detach()[:, off:off + c].view(ok.shape), ok.detach()), f"member {k}: states"
        assert torch.equal(q0.grad[off:off + c].view(m.q.shape), qk.grad), f"member {k}: state gradient"
        _close_params(theta.grad[k], tk.grad, f"member {k}: parameter gradient")


def test_ensemble_select_outputs(cuda_device):
    """Selected arena entries at the output steps give the gradient of the same
    loss computed from whole output arenas."""
    dev = cuda_device
    members = _advance(_members(seed=2), dev, n=6)
    ens = EnsembleStepper(members, dev)
    rng = np.random.default_rng(8)
    sel = torch.tensor(np.concatenate([ens.cm[k].q_off + rng.choice(m.q.size, 10, replace=False)
                                       for k, m in enumerate(members)]), device=dev)
    res = []
    for use_sel in (False, True):
        q0 = ens.qa.clone().requires_grad_(True)
        theta = torch.stack([theta_of(m.params, dev) for m in members]).requires_grad_(True)
        if use_sel:
            o = ensemble_rollout_states(q0, theta, members, 9, [3, 9], select=sel)
        else:
            o = ensemble_rollout_states(q0, theta, members, 9, [3, 9])[:, sel]
        (o ** 2).sum().backward()
        res.append((o.detach(), q0.grad.clone(), theta.grad.clone()))
    for a, b in zip(res[0], res[1]):
        assert torch.equal(a, b)


def test_ensemble_observations_match_single_patch(cuda_device):
    """Per-member observation intervals: each member's gauge entries land in
    its own slots at its own steps, bit for bit as rollout_observations on
    the member alone, with the same state gradients and parameter gradients
    to 1e-12."""
    import dataclasses

    dev = cuda_device
    members = [dataclasses.replace(m, t_obs=to) for m, to in
               zip(_advance(_members(seed=4), dev, n=6), [0.01, 0.02, 0.015, 0.03, 0.01])]
    ens = EnsembleStepper(members, dev)
    rng = np.random.default_rng(12)
    n, n_obs, per = 24, 8, 6
    picks = [rng.choice(m.q.size, per, replace=False) for m in members]
    sel = torch.tensor(np.concatenate([ens.cm[k].q_off + picks[k] for k in range(len(members))]), device=dev)
    wts = torch.tensor(rng.standard_normal((n_obs, sel.numel())), device=dev)
    q0 = ens.qa.clone().requires_grad_(True)
    theta = torch.stack([theta_of(m.params, dev) for m in members]).requires_grad_(True)
    o = ensemble_rollout_observations(q0, theta, members, n, n_obs, sel, checkpoint_block=5)
    steps = observation_steps(o)
    (o * wts).sum().backward()
    assert any(s >= 0 for row in steps for s in row)
    for k, m in enumerate(members):
        cols = slice(k * per, (k + 1) * per)
        qk = torch.tensor(m.q, device=dev, requires_grad=True)
        tk = theta_of(m.params, dev).requires_grad_(True)
        sk = torch.tensor(picks[k], device=dev)
        ok = rollout_observations(qk, tk, torch.tensor(m.b, device=dev), m.params, m.dx, m.dy, n, m.t_obs, n_obs,
                                  m.dt_initial, select=sk, checkpoint_block=3)
        assert [row[k] for row in steps] == observation_steps(ok), f"member {k}: steps"
        assert torch.equal(o.detach()[:, cols], ok.detach()), f"member {k}: observations"
        (ok * wts[:, cols]).sum().backward()
        off, c = ens.cm[k].q_off, m.q.size
        assert torch.equal(q0.grad[off:off + c].view(m.q.shape), qk.grad), f"member {k}: state gradient"
        _close_params(theta.grad[k], tk.grad, f"member {k}: parameter gradient")


def test_ensemble_bed_gradient_matches_single_patch(cuda_device):
    """A bed arena that requires grad: each member's bed gradient from the
    batched adjoint equals rollout_states' on the member alone, bit for bit,
    and stepping over the given arena equals stepping over the members'
    own beds."""
    dev = cuda_device
    members = _advance(_members(seed=6), dev, n=6)
    ens = EnsembleStepper(members, dev)
    n, outs = 10, [4, 10]
    rng = np.random.default_rng(5)
    wts = torch.tensor(rng.standard_normal((len(outs), ens.qa.numel())), device=dev)
    q0 = ens.qa.clone().requires_grad_(True)
    theta = torch.stack([theta_of(m.params, dev) for m in members])
    bed = ens.bed.clone().requires_grad_(True)
    o = ensemble_rollout_states(q0, theta, members, n, outs, checkpoint_block=4, bed=bed)
    o_plain = ensemble_rollout_states(ens.qa.clone(), theta, members, n, outs, checkpoint_block=4)
    assert torch.equal(o.detach(), o_plain.detach())
    (o * wts).sum().backward()
    assert bed.grad is not None and bed.grad.abs().max() > 0
    for k, m in enumerate(members):
        off, c = ens.cm[k].q_off, m.q.size
        ob, cb = ens.cm[k].b_off, m.b.size
        qk = torch.tensor(m.q, device=dev, requires_grad=True)
        bk = torch.tensor(m.b, device=dev, requires_grad=True)
        ok = rollout_states(qk, theta_of(m.params, dev), bk, m.params, m.dx, m.dy, n, outs, m.dt_initial,
                            checkpoint_block=3)
        (ok * wts[:, off:off + c].view((len(outs),) + m.q.shape)).sum().backward()
        assert torch.equal(bed.grad[ob:ob + cb].view(m.b.shape), bk.grad), f"member {k}: bed gradient"
        assert torch.equal(q0.grad[off:off + c].view(m.q.shape), qk.grad), f"member {k}: state gradient"
