"""The oracle against the known-answer tests of the reference's own suites.

Pins the CPU restatement (oracle/dclaw_oracle.cpp) to the closed-form
criteria of tests/eigenstructure_check/check.py:65,80,97-118 (contact-wave
preservation, dry dam-break front bound) and
differentiable_dclaw/tests/test_lake_at_rest.py:42 (well-balancing, 1e-8).
"""
import numpy as np
import pytest

from dclaw_b200 import workloads as W


LIBMS = ["glibc", "portable"]


@pytest.mark.parametrize("libm", LIBMS)
def test_contact_wave_kat(oracle, libm):
    c = W.contact_wave()
    r = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 420, c.dt_initial, t_final=2.0, libm=libm)
    assert r["status"] == 0
    assert abs(r["t"] - 2.0) < 1e-12
    q = r["q"]
    h = q[0]
    u = np.where(h > 1e-6, q[1] / np.where(h > 1e-6, h, 1.0), 0.0)
    assert np.abs(u).max() <= 1e-9           # check.py:65
    assert h.max() - h.min() <= 1e-9         # check.py:65
    j = c.my // 2
    x = -5.0 + (np.arange(c.mx) + 0.5) * c.dx
    m0 = c.q[3][j] / c.q[0][j]
    m1 = np.where(h[j] > 1e-6, q[3][j] / h[j], 0.0)
    # the interface: first cell of the m = 0.60 side, before and after
    i0 = np.argmax(m0 > 0.575)
    i1 = np.argmax(m1 > 0.575)
    assert abs(x[i1] - x[i0]) <= 1e-6        # check.py:80


@pytest.mark.parametrize("libm", LIBMS)
def test_dam_front_kat(oracle, libm):
    c = W.dam_front()
    for T in (0.2, 0.5, 1.0):
        r = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 400, c.dt_initial, t_final=T, libm=libm)
        assert r["status"] == 0 and abs(r["t"] - T) < 1e-12
        h = r["q"][0][c.my // 2]
        x = (np.arange(c.mx) + 0.5) * c.dx
        wet = h > 1e-3
        front = x[wet].max() if wet.any() else 5.0
        assert front <= 5.0 + 2.0 * np.sqrt(9.81 * 2.0) * T + 0.1   # check.py:97-118
        assert front > 5.0 + 0.5 * np.sqrt(9.81 * 2.0) * T          # the front does move


@pytest.mark.parametrize("libm", LIBMS)
def test_lake_at_rest_kat(oracle, libm):
    c = W.lake_at_rest()
    r = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 400, c.dt_initial, t_final=60.0, libm=libm)
    q = r["q"]
    wet = q[0] > 0.01
    max_u = np.abs(np.where(wet, q[1] / np.maximum(q[0], 1e-9), 0.0)).max()
    eta_dev = np.abs(np.where(wet, q[0] + c.b - 5.0, 0.0)).max()
    assert max_u < 1e-8 and eta_dev < 1e-8                    # test_lake_at_rest.py:42
    assert np.all(q[0][c.b > 5.01] < 1e-6)                     # the island stays dry


def test_serial_and_parallel_step2_agree(oracle):
    c = W.slope_runout()
    a = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 25, c.dt_initial, parallel=False, branch_log=True)
    b = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 25, c.dt_initial, parallel=True, branch_log=True)
    assert np.array_equal(a["q"], b["q"])
    assert np.array_equal(a["dt"], b["dt"]) and np.array_equal(a["cfl"], b["cfl"])
    assert np.array_equal(a["xlog"], b["xlog"]) and np.array_equal(a["ylog"], b["ylog"])


def test_pointwise_qfix_and_setvars(oracle):
    from dclaw_b200.params import DClawParams

    p = DClawParams()
    s, prim = oracle.qfix(p, [2.0, 1.0, -0.5, 1.3, 5.0e4, 0.0])
    assert s[3] == 2.0 * (1.3 / 2.0) and prim[2] == 1.3 / 2.0
    rho = 2700.0 * prim[2] + (1 - prim[2]) * 1000.0
    assert s[4] == min(max(0.0, 5.0e4), rho * 9.81 * 2.0)
    s, prim = oracle.qfix(p, [5e-4, 1.0, 1.0, 1.0, 1.0, 0.0])
    assert np.all(s == 0) and np.all(prim == 0)
    out = oracle.setvars(p, [1.0, 0.0, 0.0, 0.6, 0.8 * 1000 * 9.81, 0.0])
    rho, kperm, alphainv, m_eq, tanpsi, tau = out
    assert rho == 0.6 * (2700.0 - 1000.0) + 1000.0
    assert m_eq == 0.64 and abs(tanpsi - (0.6 - 0.64)) < 1e-15
    assert kperm == 1e-10 * np.exp(-(0.6 - 0.6) / 0.04)


def test_libm_sensitivity_one_step(oracle):
    """One step with glibc vs the portable elementary functions: the states
    agree to 1e-13, the dry/wet masks exactly."""
    c = W.slope_runout()
    r0 = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 30, c.dt_initial, libm="glibc")
    a = oracle.run(c.params, r0["q"], c.b, c.dx, c.dy, 1, 0.1, fixed_dt=True, libm="glibc")
    b = oracle.run(c.params, r0["q"], c.b, c.dx, c.dy, 1, 0.1, fixed_dt=True, libm="portable")
    assert np.array_equal(a["q"][0] == 0, b["q"][0] == 0)
    for m in range(5):
        assert np.abs(a["q"][m] - b["q"][m]).max() <= 1e-13 * np.abs(a["q"][m]).max()


def _quadrant_states(p, n=48, seed=21):
    """Padded (5, n+4, n+4) states spread over the (m, p) plane of
    mp_update_FE_4quad: m either side of m_crit, pore pressure from 0 to
    above lithostatic, speeds from rest to 6 m/s, depths 5 cm to 2 m."""
    rng = np.random.default_rng(seed)
    h = rng.uniform(0.05, 2.0, (n + 4, n + 4))
    m = rng.uniform(0.40, 0.72, (n + 4, n + 4))
    rho = p.rho_s * m + (1.0 - m) * p.rho_f
    pb = rng.uniform(0.0, 1.1, (n + 4, n + 4)) * rho * p.grav * h
    sp = np.where(rng.random((n + 4, n + 4)) < 0.15, 0.0, rng.uniform(0.0, 6.0, (n + 4, n + 4)))
    ang = rng.uniform(0.0, 2 * np.pi, (n + 4, n + 4))
    return np.stack([h, h * sp * np.cos(ang), h * sp * np.sin(ang), h * m, pb])


@pytest.mark.parametrize("libm", LIBMS)
def test_src2method2_keeps_rho_h(oracle, libm):
    """src2method 2 integrates m and p on the rho h = const manifold
    (mp_update.f90:13-16,30-33): every wet cell's rho h is unchanged by src2
    to rounding, while m and p move."""
    from dclaw_b200.params import DClawParams

    p = DClawParams(src2method=2, alphamethod=1)
    q = _quadrant_states(p)
    aux = np.zeros((6,) + q.shape[1:])
    out = oracle.src2(p, q, aux, 0.05, libm=libm)
    inner = (slice(None), slice(2, -2), slice(2, -2))
    qi, qo = q[inner], out[inner]
    rhoh0 = qi[3] * p.rho_s + (qi[0] - qi[3]) * p.rho_f
    rhoh1 = qo[3] * p.rho_s + (qo[0] - qo[3]) * p.rho_f
    wet = qo[0] > p.dry_tolerance
    assert wet.mean() > 0.95
    assert np.abs(rhoh1 - rhoh0)[wet].max() <= 1e-12 * rhoh0[wet].max()
    assert np.abs(qo[3] / qo[0] - qi[3] / qi[0])[wet].max() > 1e-4     # m moved
    assert np.abs(qo[4] - qi[4])[wet].max() > 1.0                       # p moved


def test_observation_clamp_lands_on_observation_times(oracle):
    """t_obs clips each tick-rule dt at the next multiple of t_obs (the
    port's flume loop, pf_flume/flume_model.py:152-153): t reaches every
    observation time it passes, and no step is longer than the free run's
    rule would make it from the same Courant number."""
    c = W.slope_runout(n=48)
    t_obs = 0.25
    o = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 40, c.dt_initial, libm="portable", t_obs=t_obs)
    assert o["status"] == 0
    t = np.cumsum(o["dt"])
    assert t[-1] == o["t"]
    stops = list(range(1, int(t[-1] / t_obs + 1e-9) + 1))
    assert len(stops) >= 4
    assert all(np.abs(t - m * t_obs).min() < 1e-9 for m in stops)
    rule = np.minimum(o["dt"][:-1] * c.params.cfl_desired / o["cfl"][:-1], c.params.dt_max)
    assert np.all(o["dt"][1:] <= rule) and np.any(o["dt"][1:] < rule)
