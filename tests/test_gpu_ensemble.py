"""The batched ensemble step (dclaw_step_batched) against the single-patch
fused step (dclaw_step), bit for bit, member by member: uneven patch sizes,
per-member parameters (friction angle, permeability, m0, alpha, boundary
conditions, order, transverse waves, limiter) and per-member adaptive dt.
The ensemble's tile shapes and persistent grids all give the same bits."""
import numpy as np
import pytest
import torch

from dclaw_b200 import workloads as W
from dclaw_b200.ensemble import EnsembleStepper, Member
from dclaw_b200.solver import PatchStepper

pytestmark = pytest.mark.gpu


def _members(seed=3, t_final=0.0):
    rng = np.random.default_rng(seed)
    out = []
    for c in W.flume_ensemble(n=4, seed=seed, width_range=(5, 40), length_range=(60, 300)):
        out.append(Member(c.q, c.b, c.params, c.dx, c.dy, 2.0e-3, t_final))
    rf = W.random_field_case(n=96, dx=0.5, seed=seed + 1)
    p = rf.params.replace(bc_lower=("wall", "extrap"), bc_upper=("extrap", "wall"), transverse_waves=1)
    out.append(Member(rf.q, rf.b, p, rf.dx, rf.dy, 0.01, t_final))
    rf2 = W.random_field_case(n=64, dx=0.5, seed=seed + 2)
    q = rf2.q[:, :37, :]
    b = rf2.b[:37, :]
    out.append(Member(q, b, rf2.params.replace(order=1, limiter=1), 0.5, 0.25, 0.005, t_final))
    out.append(Member(q[:, :2, :3].copy(), b[:2, :3].copy(), rf2.params, 0.5, 0.5, 0.005, t_final))
    assert len({(m.q.shape[1], m.q.shape[2]) for m in out}) == len(out)
    return out


def _single(members, nsteps, dev):
    res = []
    for m in members:
        ps = PatchStepper(torch.from_numpy(m.q).to(dev), torch.from_numpy(m.b).to(dev), m.params, m.dx, m.dy)
        ps.init_clock(m.dt_initial, t_final=m.t_final, t_obs=m.t_obs)
        ps.step(nsteps)
        c = ps.read_clock()
        res.append((ps.state().cpu().numpy(), (c.t, c.dt, c.cfl, c.nsteps, c.status)))
    return res


def _check(ens, ref):
    clocks = ens.read_clocks()
    for k, (q, clk) in enumerate(ref):
        got = ens.state(k).cpu().numpy()
        assert np.array_equal(got, q), f"member {k}: max |diff| {np.abs(got - q).max()}"
        c = clocks[k]
        assert (c.t, c.dt, c.cfl, c.nsteps, c.status) == clk, f"member {k} clock"


@pytest.mark.parametrize("shape", [0, 1, 2])
def test_batched_matches_single_patch_steps(shape):
    dev = torch.device("cuda:0")
    members = _members()
    ref = _single(members, 25, dev)
    ens = EnsembleStepper(members, dev, tile_shape=shape)
    ens.step(25)
    torch.cuda.synchronize()
    _check(ens, ref)
    assert all(s == 0 for s in ens.status())
    assert any(np.abs(q[1]).max() > 0 for q, _ in ref)  # something moved


def test_batched_one_cta_per_sm_and_t_final():
    dev = torch.device("cuda:0")
    members = _members(seed=5, t_final=0.03)
    ref = _single(members, 12, dev)
    ens = EnsembleStepper(members, dev)
    ens.batch.tile_ctas_per_sm = 1
    ens.step(12)
    torch.cuda.synchronize()
    _check(ens, ref)


def test_batched_observation_intervals():
    """Per-member observation intervals (and t_final) clip each member's dt as
    the single-patch clock does."""
    import dataclasses

    dev = torch.device("cuda:0")
    members = [dataclasses.replace(m, t_obs=to) for m, to in
               zip(_members(seed=9, t_final=0.4), [0.05, 0.0, 0.013, 0.1, 0.02, 0.07, 0.0])]
    ref = _single(members, 30, dev)
    ens = EnsembleStepper(members, dev)
    ens.step(30)
    torch.cuda.synchronize()
    _check(ens, ref)


def test_batched_graph_replay_and_autotune():
    dev = torch.device("cuda:0")
    members = _members(seed=7)
    ref = _single(members, 20, dev)
    ens = EnsembleStepper(members, dev)
    best = ens.autotune(steps=2)
    assert best["tile_shape"] in (0, 1, 2) and len(best["candidates"]) == 6
    ens.step(4)
    ens.capture(8)
    ens.replay(2)
    torch.cuda.synchronize()
    _check(ens, ref)
