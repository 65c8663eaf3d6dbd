"""Parity of the CUDA step (through the C ABI) with the oracle.

Two bars.
1. Against the oracle with the same deterministic elementary functions
   (libm="portable"): everything is bit-identical -- state, the dry/wet
   mask (h == 0), every per-interface branch bit of the last step (dry
   skip, wall problem, sonic, static friction, middle-wave merge side,
   4-cell wet check, limiter regime and upwind side of each wave family,
   transverse splits), and the dt / Courant-number histories -- over the
   full 1000 steps of the slope-runout case.
2. Against the oracle with glibc's libm (what gfortran links on x86-64).
   The step's exp, expm1 and tanh return glibc's bits and its atan and tan
   are correctly rounded, which glibc's are in all but about 0.2 % of
   arguments. So the 200 x 200 slope-runout case is bit-identical to the
   glibc oracle through step 86 (state, masks, branch bits, dt history);
   the first argument where glibc's atan or tan rounds the other way comes
   at step 87. Cases with more wet cells meet such an argument within the
   first steps; there one step agrees to 1e-13 relative and a few steps to
   1e-12 with identical dry/wet masks. Longer runs are not compared: the
   scheme amplifies a one-ulp difference to O(1) within a few hundred steps,
   so only a libm with glibc's own tables could meet a 1e-10 bar there.
"""
import numpy as np
import pytest
import torch

from dclaw_b200 import workloads as W
from dclaw_b200.params import DClawParams

pytestmark = pytest.mark.gpu


def gpu_run(c, n, fixed_dt=False, dt=None, branch_log=True):
    """With the branch log the step runs its full-grid kernels (every
    interface's bits are logged); without it, the kernels over the lists of
    active tiles."""
    from dclaw_b200.solver import PatchStepper

    dev = torch.device("cuda:0")
    st = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), c.params, c.dx, c.dy,
                      branch_log=branch_log)
    st.init_clock(c.dt_initial if dt is None else dt, fixed_dt=fixed_dt)
    hist = torch.zeros((n, 4), dtype=torch.float64, device=dev)
    st.step(n, history=hist)
    torch.cuda.synchronize()
    return dict(q=st.state().cpu().numpy(), hist=hist.cpu().numpy(),
                br=st.brlog.cpu().numpy().view(np.uint32) if branch_log else None, status=st.status())


def rel_err(a, b):
    return max(np.abs(a[m] - b[m]).max() / max(np.abs(b[m]).max(), 1e-300) for m in range(5))


def check(c, n, oracle, fixed_dt=False, glibc_steps=3, glibc_exact=False):
    """Bit-exact against the portable-libm oracle over n steps; against the
    glibc oracle over the first glibc_steps steps, bit for bit (glibc_exact)
    or to 1e-12 with the same dry/wet masks."""
    g = gpu_run(c, n, fixed_dt)
    o = oracle.run(c.params, c.q, c.b, c.dx, c.dy, n, c.dt_initial, fixed_dt=fixed_dt, branch_log=True,
                   libm="portable")
    assert g["status"] == 0 and o["status"] == 0
    assert np.array_equal(g["q"][0] == 0.0, o["q"][0] == 0.0), "dry/wet mask differs"
    br_o = np.concatenate([o["xlog"].ravel(), o["ylog"].ravel()])
    nd = int((g["br"] != br_o).sum())
    assert nd == 0, f"{nd} interfaces took a different branch"
    assert np.array_equal(g["q"], o["q"]), f"state differs (rel {rel_err(g['q'], o['q']):.3e})"
    assert np.array_equal(g["hist"][:, 3], o["dt"]) and np.array_equal(g["hist"][:, 2], o["cfl"])
    # the same steps over the tile lists (no branch log)
    gl = gpu_run(c, n, fixed_dt, branch_log=False)
    assert gl["status"] == 0
    assert np.array_equal(gl["q"], o["q"]), f"tile-list state differs (rel {rel_err(gl['q'], o['q']):.3e})"
    assert np.array_equal(gl["hist"], g["hist"])
    if glibc_steps:
        g3 = gpu_run(c, glibc_steps, fixed_dt)
        o3 = oracle.run(c.params, c.q, c.b, c.dx, c.dy, glibc_steps, c.dt_initial, fixed_dt=fixed_dt,
                        libm="glibc")
        assert np.array_equal(g3["q"][0] == 0.0, o3["q"][0] == 0.0)
        if glibc_exact:
            assert np.array_equal(g3["q"], o3["q"]), f"state differs (rel {rel_err(g3['q'], o3['q']):.3e})"
            assert np.array_equal(g3["hist"][:, 3], o3["dt"]) and np.array_equal(g3["hist"][:, 2], o3["cfl"])
        else:
            assert rel_err(g3["q"], o3["q"]) <= 1e-12
    return g, o


def test_slope_runout_short(cuda_device, oracle):
    check(W.slope_runout(), 20, oracle, glibc_steps=20, glibc_exact=True)


@pytest.mark.parametrize("variant", ["order1", "transverse1", "minmod", "extrap", "src2m1", "swe", "alpha1",
                                     "src2m2", "manning", "speed_limit"])
def test_variants(cuda_device, oracle, variant):
    kw = {"order1": dict(order=1, transverse_waves=0), "transverse1": dict(transverse_waves=1),
          "minmod": dict(limiter=1), "extrap": dict(bc_lower=("extrap", "wall"), bc_upper=("extrap", "extrap")),
          "src2m1": dict(src2method=1), "swe": dict(src2method=-1), "alpha1": dict(alphamethod=1),
          "src2m2": dict(src2method=2, alphamethod=1),
          "manning": dict(friction_forcing=True, manning_coefficient=0.025),
          "speed_limit": dict(speed_limit=2.0)}[variant]
    base = W.slope_runout(n=96)
    c = W.Case(base.name, base.q, base.b, base.dx, base.dy, base.params.replace(**kw), 0, base.dt_initial)
    check(c, 40, oracle)


def test_observation_clamp(cuda_device, oracle):
    """With an observation interval the clock clips every dt at the next
    multiple of it, (floor(t/t_obs + 1e-9) + 1) t_obs - t, as the port's
    flume loop does (pf_flume/flume_model.py:152-153): dt history, Courant
    numbers and state bit for bit with the oracle, and t lands on every
    observation time it passes."""
    from dclaw_b200.solver import PatchStepper

    c = W.slope_runout(n=96)
    n, t_obs = 60, 0.25
    st = PatchStepper(torch.tensor(c.q, device=cuda_device), torch.tensor(c.b, device=cuda_device), c.params,
                      c.dx, c.dy)
    st.init_clock(c.dt_initial, t_obs=t_obs)
    hist = torch.zeros((n, 4), dtype=torch.float64, device=cuda_device)
    st.step(n, history=hist)
    h = hist.cpu().numpy()
    o = oracle.run(c.params, c.q, c.b, c.dx, c.dy, n, c.dt_initial, libm="portable", t_obs=t_obs)
    free = oracle.run(c.params, c.q, c.b, c.dx, c.dy, n, c.dt_initial, libm="portable")
    assert np.array_equal(h[:, 3], o["dt"]) and np.array_equal(h[:, 2], o["cfl"])
    assert np.array_equal(st.state().cpu().numpy(), o["q"])
    assert not np.array_equal(o["dt"], free["dt"])
    t = h[:, 0]
    assert t[-1] == o["t"]
    stops = [m for m in range(1, int(t[-1] / t_obs + 1e-9) + 1)]
    assert len(stops) >= 8
    assert all(np.abs(t - m * t_obs).min() < 1e-9 for m in stops)


def test_random_field_small(cuda_device, oracle):
    check(W.random_field_case(n=256, dx=0.5, seed=5), 30, oracle)


@pytest.mark.parametrize("shape", [(2, 2), (17, 3), (3, 17), (13, 14), (14, 15), (27, 29)])
def test_small_patches(cuda_device, oracle, shape):
    """Patches smaller than, equal to or just over one 14 x 13 tile, and thin
    strips, cut around the wettest cell of a random field: bit for bit
    against the oracle through the full-grid and the tile-list kernels."""
    c = W.random_field_case(n=128, dx=0.5, seed=4)
    my, mx = shape
    j, i = np.unravel_index(np.argmax(c.q[0]), c.q[0].shape)
    j0, i0 = max(0, j - my // 2), max(0, i - mx // 2)
    q = np.ascontiguousarray(c.q[:, j0:j0 + my, i0:i0 + mx])
    b = np.ascontiguousarray(c.b[j0:j0 + my, i0:i0 + mx])
    check(W.Case("small", q, b, c.dx, c.dy, c.params, 10, c.dt_initial), 10, oracle, glibc_steps=0)


def test_dry_tile_fast_path(cuda_device, oracle):
    """Without a branch log the fused step skips tiles whose cells within 3 are
    all dry; the result must not change (mostly dry 384 x 384 random field)."""
    from dclaw_b200.solver import PatchStepper

    c = W.random_field_case(n=384, dx=0.5, seed=9)
    st = PatchStepper(torch.tensor(c.q, device=cuda_device), torch.tensor(c.b, device=cuda_device), c.params,
                      c.dx, c.dy)
    st.init_clock(c.dt_initial)
    st.step(120)
    o = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 120, c.dt_initial, libm="portable")
    assert (c.q[0] == 0).mean() > 0.5
    assert np.array_equal(st.state().cpu().numpy(), o["q"])
    assert st.read_clock().dt_last == o["dt"][-1]


def test_slope_runout_1000_steps(cuda_device, oracle):
    """The 200 x 200 slope-runout case over its full 1000 steps, bit for bit
    with the portable oracle, and through step 86 with the glibc oracle."""
    check(W.slope_runout(), 1000, oracle, glibc_steps=86, glibc_exact=True)


def test_kats_on_gpu(cuda_device):
    # contact wave (tests/eigenstructure_check/check.py:65,80)
    c = W.contact_wave()
    from dclaw_b200.solver import PatchStepper

    dev = cuda_device
    st = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), c.params, c.dx, c.dy)
    st.init_clock(c.dt_initial, t_final=2.0)
    st.step(420)
    q = st.state().cpu().numpy()
    assert abs(st.read_clock().t - 2.0) < 1e-12
    h = q[0]
    u = np.where(h > 1e-6, q[1] / np.where(h > 1e-6, h, 1.0), 0.0)
    assert np.abs(u).max() <= 1e-9 and h.max() - h.min() <= 1e-9
    # lake at rest (differentiable_dclaw/tests/test_lake_at_rest.py:42)
    c = W.lake_at_rest()
    st = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), c.params, c.dx, c.dy)
    st.init_clock(c.dt_initial, t_final=60.0)
    st.step(400)
    q = st.state().cpu().numpy()
    wet = q[0] > 0.01
    assert np.abs(np.where(wet, q[1] / np.maximum(q[0], 1e-9), 0.0)).max() < 1e-8
    assert np.abs(np.where(wet, q[0] + c.b - 5.0, 0.0)).max() < 1e-8
    # dam front bound (check.py:97-118)
    c = W.dam_front()
    st = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), c.params, c.dx, c.dy)
    st.init_clock(c.dt_initial, t_final=1.0)
    st.step(400)
    h = st.state().cpu().numpy()[0][c.my // 2]
    x = (np.arange(c.mx) + 0.5) * c.dx
    assert x[h > 1e-3].max() <= 5.0 + 2.0 * np.sqrt(9.81 * 2.0) * 1.0 + 0.1


def test_patch_calls(cuda_device, oracle):
    """bc2amr, setaux, b4step2, step2 (+fluxes, cflgrid), src2 through the patch API."""
    from dclaw_b200.patch import Patch

    c = W.slope_runout(n=80)
    mx, my = c.mx, c.my
    p = c.params
    dev = cuda_device
    qpad = np.zeros((5, my + 4, mx + 4))
    qpad[:, 2:-2, 2:-2] = c.q
    # evolve a few steps on the oracle to get a moving state
    r = oracle.run(p, c.q, c.b, c.dx, c.dy, 15, c.dt_initial, libm="portable")
    qpad[:, 2:-2, 2:-2] = r["q"]
    P = Patch(p, mx, my)
    qg = torch.tensor(qpad, device=dev)
    P.bc2amr(qg)
    qo = oracle.bc2amr(p, qpad)
    assert np.array_equal(qg.cpu().numpy(), qo)
    auxo = oracle.setaux(p, c.b)
    auxg = torch.zeros((6, my + 4, mx + 4), dtype=torch.float64, device=dev)
    auxg[0, 2:-2, 2:-2] = torch.tensor(c.b, device=dev)
    P.setaux(auxg)
    assert np.array_equal(auxg.cpu().numpy(), auxo)
    P.b4step2(qg, auxg, c.dx, c.dy)
    qg_lib, aux_lib = oracle.b4step2(p, qo, auxo, c.dx, c.dy, libm="glibc")
    qo, auxo = oracle.b4step2(p, qo, auxo, c.dx, c.dy, libm="portable")
    assert np.array_equal(qg.cpu().numpy(), qo) and np.array_equal(auxg.cpu().numpy(), auxo)
    assert np.array_equal(qg_lib, qo)   # b4step2 uses no elementary function on the state
    assert np.abs(aux_lib[3:] - auxo[3:]).max() <= 1e-13
    dt = float(r["dt"][-1])
    fl = torch.zeros((20, my + 4, mx + 4), dtype=torch.float64, device=dev)
    cfl_g = P.step2(qg, auxg, c.dx, c.dy, dt, fluxes=fl)
    so = oracle.step2(p, qo, auxo, c.dx, c.dy, dt, fluxes=True, libm="portable")
    sg = oracle.step2(p, qo, aux_lib, c.dx, c.dy, dt, fluxes=True, libm="glibc")
    assert cfl_g == so["cfl"]
    assert np.array_equal(qg.cpu().numpy(), so["q"])
    assert rel_err(so["q"], sg["q"]) <= 1e-13
    flg = fl.cpu().numpy()
    # the flux entries the update uses
    for k, (di, dj) in enumerate([(1, 0), (0, 0), (0, 1), (0, 0)]):
        for m in range(5):
            a = flg[5 * k + m, 2 + dj:2 + dj + my, 2 + di:2 + di + mx]
            b = so["fluxes"][5 * k + m, 2 + dj:2 + dj + my, 2 + di:2 + di + mx]
            assert np.array_equal(a, b)
    P.src2(qg, auxg, c.dx, c.dy, 0.0, dt)
    qs = oracle.src2(p, so["q"], auxo, dt, libm="portable")
    qsg = oracle.src2(p, so["q"], auxo, dt, libm="glibc")
    assert np.array_equal(qg.cpu().numpy(), qs)
    assert rel_err(qs, qsg) <= 1e-13
    assert P.status() == 0


def test_fortran_layout_adapters(cuda_device, oracle):
    """q(meqn=7, ...) and aux(maux=10, ...) in Fortran cell-major order into
    the patch calls' planes and back: the fields match, the extra fields
    are kept, and a b4step2 + step2 + src2 pass through the adapters gives
    the oracle's state."""
    from dclaw_b200.patch import Patch

    c = W.slope_runout(n=48)
    mx, my = c.mx, c.my
    dev = cuda_device
    rng = np.random.default_rng(3)
    r = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 10, c.dt_initial, libm="portable")
    qpad = np.zeros((5, my + 4, mx + 4))
    qpad[:, 2:-2, 2:-2] = r["q"]
    qf = np.zeros((my + 4, mx + 4, 7))
    qf[..., :5] = np.moveaxis(qpad, 0, -1)
    qf[..., 5:] = rng.standard_normal((my + 4, mx + 4, 2))
    P = Patch(c.params, mx, my)
    qf_d = torch.tensor(qf, device=dev)
    planes = P.from_fortran(qf_d, 5)
    assert torch.equal(planes.cpu(), torch.tensor(qpad))
    auxf = torch.tensor(rng.standard_normal((my + 4, mx + 4, 10)), device=dev)
    aux_planes = P.from_fortran(auxf, 6)
    assert torch.equal(aux_planes, auxf[..., :6].permute(2, 0, 1))
    # a patch step through the adapters against the oracle's patch calls
    aux = torch.zeros((6, my + 4, mx + 4), dtype=torch.float64, device=dev)
    aux[0, 2:-2, 2:-2] = torch.tensor(c.b, device=dev)
    P.setaux(aux)
    P.bc2amr(planes)
    P.b4step2(planes, aux, c.dx, c.dy)
    P.step2(planes, aux, c.dx, c.dy, 0.01)
    P.src2(planes, aux, c.dx, c.dy, 0.0, 0.01)
    P.to_fortran(planes, qf_d)
    back = qf_d.cpu().numpy()
    assert np.array_equal(back[..., 5:], qf[..., 5:])
    assert np.array_equal(np.moveaxis(back[..., :5], -1, 0), planes.cpu().numpy())
    aux_o = oracle.setaux(c.params, c.b)
    qo, aux_o = oracle.b4step2(c.params, oracle.bc2amr(c.params, qpad), aux_o, c.dx, c.dy, libm="portable")
    qo = oracle.step2(c.params, qo, aux_o, c.dx, c.dy, 0.01, libm="portable")["q"]
    qo = oracle.src2(c.params, qo, aux_o, 0.01, libm="portable")
    assert np.array_equal(planes.cpu().numpy()[:, 2:-2, 2:-2], qo[:, 2:-2, 2:-2])


def test_graph_replay_matches_eager(cuda_device):
    from dclaw_b200.solver import PatchStepper

    c = W.random_field_case(n=192, dx=0.5, seed=11)
    dev = cuda_device
    a = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), c.params, c.dx, c.dy)
    a.init_clock(c.dt_initial)
    a.step(12)
    b = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), c.params, c.dx, c.dy)
    b.init_clock(c.dt_initial)
    b.capture(4)
    b.replay(3)
    torch.cuda.synchronize()
    assert torch.equal(a.state(), b.state())
    ca, cb = a.read_clock(), b.read_clock()
    assert ca.t == cb.t and ca.dt == cb.dt and cb.nsteps == 12


def test_full_size_window(cuda_device, oracle):
    """4096 x 4096 run (fixed dt) against the oracle on a window: with a fixed
    dt a cell depends only on cells within 4 per step, so the window's core
    must agree although the oracle sees walls at the window edges."""
    from dclaw_b200.solver import PatchStepper

    c = W.random_field_case(n=4096, dx=0.5, seed=0)
    dev = cuda_device
    n, dt = 8, 0.02
    st = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), c.params, c.dx, c.dy)
    st.init_clock(dt, fixed_dt=True)
    st.step(n)
    assert st.status() == 0
    qg = st.state()
    # the tile-list kernels (no branch log) against the full-grid ones
    full = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), c.params, c.dx, c.dy,
                        branch_log=True)
    full.init_clock(dt, fixed_dt=True)
    full.step(n)
    assert torch.equal(full.state(), qg)
    del full
    # a window around the wettest 256 x 256 block
    h = torch.tensor(c.q[0], device=dev)
    blk = torch.nn.functional.avg_pool2d(h[None, None], 256, 256)[0, 0]
    jb, ib = divmod(int(torch.argmax(blk)), blk.shape[1])
    j0, i0 = jb * 256, ib * 256
    win = slice(j0, j0 + 256), slice(i0, i0 + 256)
    o = oracle.run(c.params, c.q[:, win[0], win[1]], c.b[win[0], win[1]], c.dx, c.dy, n, dt, fixed_dt=True,
                   libm="portable")
    m = 4 * n + 4
    g = qg[:, j0 + m:j0 + 256 - m, i0 + m:i0 + 256 - m].cpu().numpy()
    oo = o["q"][:, m:256 - m, m:256 - m]
    assert (g[0] > 0).sum() > 1000
    assert np.array_equal(g, oo)


def test_nan_reported_as_status(cuda_device):
    from dclaw_b200.solver import PatchStepper

    c = W.slope_runout(n=32)
    q = c.q.copy()
    q[4, 5, 5] = np.nan
    st = PatchStepper(torch.tensor(q, device=cuda_device), torch.tensor(c.b, device=cuda_device), c.params,
                      c.dx, c.dy)
    st.init_clock(c.dt_initial)
    st.step(1)
    assert st.status() == 3


def test_all_dry_stays_dry(cuda_device):
    from dclaw_b200.solver import PatchStepper

    c = W.slope_runout(n=32)
    q = np.zeros_like(c.q)
    st = PatchStepper(torch.tensor(q, device=cuda_device), torch.tensor(c.b, device=cuda_device), c.params,
                      c.dx, c.dy)
    st.init_clock(0.1)
    st.step(3)
    assert torch.count_nonzero(st.state()) == 0 and st.read_clock().cfl == 0.0


def test_step_function_api(cuda_device, oracle):
    """step / cfl_dt / rollout / rollout_peak with the port's (5, nx, ny) shapes."""
    from dclaw_b200 import solver as S

    c = W.slope_runout(n=64)
    dev = cuda_device
    q0 = torch.tensor(c.q, device=dev).permute(0, 2, 1).contiguous()  # (5, nx, ny)
    b = torch.tensor(c.b, device=dev).t().contiguous()
    grid = S.Grid(nx=64, ny=64, dx=c.dx, dy=c.dy)
    p = c.params
    q1 = S.step(q0, b, p, grid, 0.05)
    o = oracle.run(p, c.q, c.b, c.dx, c.dy, 1, 0.05, fixed_dt=True, libm="portable")
    assert np.array_equal(q1.permute(0, 2, 1).cpu().numpy(), o["q"])
    dt = float(S.cfl_dt(q0, p, grid, 0.4))
    h = c.q[0]
    wet = h > 1e-3
    smax = np.max(np.sqrt(9.81 * h[wet]))
    assert abs(dt - 0.4 * c.dx / smax) <= 1e-12 * dt
    qf, t, states, times = S.rollout(q0, b, p, grid, t_final=2.0, cfl=0.9, n_steps=40)
    assert states.shape == (40, 5, 64, 64) and float(t) <= 2.0 + 1e-12
    assert torch.equal(states[-1], qf)
    qp, tp, hmax = S.rollout_peak(q0, b, p, grid, t_final=2.0, cfl=0.9, n_steps=40)
    assert torch.equal(qp, qf) and hmax.shape == (64, 64)
    assert torch.all(hmax >= qf[0]) and torch.all(hmax >= q0[0])


@pytest.mark.parametrize("dt", [0.01, 0.05, 0.5])
def test_src2method2_patch_call(cuda_device, oracle, dt):
    """src2 with mp_update_FE_4quad (src2method 2) through the patch call, on
    states spread over the four (m, p) quadrants: bit for bit against the
    oracle with the same elementary functions, 1e-12 against glibc's."""
    from dclaw_b200.patch import Patch

    from .test_oracle_kats import _quadrant_states

    p = DClawParams(src2method=2, alphamethod=1)
    q = _quadrant_states(p, n=64, seed=33)
    n = q.shape[1] - 4
    aux = np.zeros((6,) + q.shape[1:])
    P = Patch(p, n, n)
    qg = torch.tensor(q, device=cuda_device)
    P.src2(qg, torch.tensor(aux, device=cuda_device), 1.0, 1.0, 0.0, dt)
    got = qg.cpu().numpy()
    want = oracle.src2(p, q, aux, dt, libm="portable")
    assert np.array_equal(got, want), f"max |diff| {np.abs(got - want).max():.3e}"
    ref = oracle.src2(p, q, aux, dt, libm="glibc")
    assert rel_err(ref, got) <= 1e-12
