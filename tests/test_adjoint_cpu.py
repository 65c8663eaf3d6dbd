"""The hand-written adjoint of the step, on the host build of its device
code (dclaw_b200/csrc/adjoint.cuh), against central finite differences.

Local routines are checked one by one over random inputs (directional
derivatives, two step sizes; samples whose step straddles a kink of the
forward routine are skipped and counted). The whole step's vector-Jacobian
product is checked on small patches with wet, dry and resting cells,
every boundary, order, transverse and limiter option, src2 method, and the
four differentiated parameters (phi, kref, alpha_c, mu). The adjoint
follows the branches the forward step took, so perturbations keep dry
cells dry and resting cells at rest where the forward branch depends on it.
"""
import math

import numpy as np
import pytest

from ._adj import LOCAL_CHECKS, Adj
from dclaw_b200 import workloads as W
from dclaw_b200.params import DClawParams


@pytest.fixture(scope="module")
def adj():
    return Adj()


# bounds: finite differences at steps 1e-6 and 2.5e-7 agree to ~1e-7; the
# wall-problem sample set also holds the rpn2 middle-wave merge, whose side
# is decided by the rounding of a symmetric interface momentum (checked
# through the whole step below, where the merged component vanishes)
@pytest.mark.parametrize("name", [n for n in LOCAL_CHECKS if n != "riemann_dry_side_or_wall"])
def test_local_adjoints_match_finite_differences(adj, name):
    n, err, skipped = adj.local(name, seed=3, n=1500)
    assert n == 1500
    assert skipped <= n // 20
    assert err < 2e-5, f"{name}: max relative error {err:.2e}"


def _case(seed, mx=14, my=11, dry_frac=0.0, moving=True, p=None):
    rng = np.random.default_rng(seed)
    p = p or DClawParams()
    X, Y = np.meshgrid(np.arange(mx), np.arange(my))
    b = 0.3 * np.sin(0.5 * X) + 0.2 * np.cos(0.4 * Y) + 0.05 * X
    h = 1.0 + 0.3 * np.sin(0.7 * X + 0.3) * np.cos(0.5 * Y) + 0.1 * rng.random((my, mx))
    if dry_frac > 0:
        h = np.where(rng.random((my, mx)) < dry_frac, 0.0, h)
    m = 0.55 + 0.05 * rng.random((my, mx))
    hu = (0.5 * np.sin(0.3 * Y) + 0.2 * rng.standard_normal((my, mx))) * h if moving else None
    hv = (0.3 * np.cos(0.2 * X) + 0.2 * rng.standard_normal((my, mx))) * h if moving else None
    return p, W.state_from(h, m, p, 0.7, hu, hv), b


CASES = {
    "wet": dict(seed=1),
    "wet_b": dict(seed=2),
    "dry30": dict(seed=4, dry_frac=0.3),
    "dry50": dict(seed=5, dry_frac=0.5),
    "extrap": dict(seed=6, p=DClawParams(bc_lower=("extrap", "wall"), bc_upper=("wall", "extrap"))),
    "order1": dict(seed=7, p=DClawParams(order=1, transverse_waves=0)),
    "transverse1": dict(seed=8, p=DClawParams(transverse_waves=1)),
    "src2method1": dict(seed=9, p=DClawParams(src2method=1)),
    "src2method-1": dict(seed=10, p=DClawParams(src2method=-1)),
    "minmod": dict(seed=11, p=DClawParams(limiter=1)),
    "superbee": dict(seed=12, p=DClawParams(limiter=2)),
    "alphamethod1": dict(seed=13, p=DClawParams(alphamethod=1)),
    "manning": dict(seed=14, p=DClawParams(friction_forcing=True, manning_coefficient=0.06)),
    "dd_manning": dict(seed=15, p=DClawParams(friction_forcing=True, manning_coefficient=0.04, dd_manning=True,
                                              manning_max=0.1, friction_depth=0.8)),
    "at_rest": dict(seed=3, moving=False),
    # b4step2's speed limit (b4step2.f90:74-100) acting on the faster cells
    "speed_limit": dict(seed=16, p=DClawParams(speed_limit=0.6)),
    # the rare-wave corrector (riemannsolvers_dclaw.f:169-195)
    "rare_corrector": dict(seed=17, p=DClawParams(rarecorrectortest=True)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_step_vjp_matches_finite_differences(adj, name):
    p, q, b = _case(**CASES[name])
    dx, dt = 1.0, 0.02
    rng = np.random.default_rng(100)
    lam = rng.standard_normal(q.shape)
    dq = rng.standard_normal(q.shape) * (np.abs(q) + 1e-3)
    dq[:, q[0] <= p.dry_tolerance] = 0.0
    if name == "at_rest":
        dq[1:3] = 0.0
    li, pb = adj.vjp(p, q, b, dx, dx, dt, lam)

    def L(qq, pp=p):
        return float((lam * adj.step(pp, qq, b, dx, dx, dt)).sum())

    eps = 1e-6
    fd = (L(q + eps * dq) - L(q - eps * dq)) / (2 * eps)
    ad = float((li * dq).sum())
    assert abs(ad - fd) <= 1e-7 * abs(fd), f"state: AD {ad:.12e} FD {fd:.12e}"
    for k, (pname, scale) in enumerate([("phi", 1.0), ("kref", p.kref), ("alpha_c", p.alpha_c), ("mu", p.mu)]):
        def Lp(d):
            if pname == "phi":
                return L(q, p.replace(phi=p.phi + d * 180.0 / math.pi))
            return L(q, p.replace(**{pname: getattr(p, pname) + d}))
        hh = 1e-6 * scale
        fdp = (Lp(hh) - Lp(-hh)) / (2 * hh)
        assert abs(pb[k] - fdp) <= 1e-4 * abs(fdp) + 1e-12, \
            f"{pname}: AD {pb[k]:.10e} FD {fdp:.10e}"


@pytest.mark.parametrize("name", ["wet", "dry30", "dry50", "order1", "transverse1", "at_rest", "manning"])
def test_step_vjp_bed_matches_finite_differences(adj, name):
    """The bed's adjoint (calc_taudir's surface slopes, the solver's bed
    step, ghost beds copied from the nearest cells) against central
    differences of the host step; lam_in and pbar are unchanged by asking
    for it."""
    p, q, b = _case(**CASES[name])
    dx, dt = 1.0, 0.02
    rng = np.random.default_rng(200)
    lam = rng.standard_normal(q.shape)
    li0, pb0 = adj.vjp(p, q, b, dx, dx, dt, lam)
    li, pb, bb = adj.vjp(p, q, b, dx, dx, dt, lam, bed=True)
    assert np.array_equal(li, li0) and np.array_equal(pb, pb0)
    db = rng.standard_normal(b.shape)

    def L(bed):
        return float((lam * adj.step(p, q, bed, dx, dx, dt)).sum())

    eps = 1e-6
    fd = (L(b + eps * db) - L(b - eps * db)) / (2 * eps)
    ad = float((bb * db).sum())
    assert abs(ad - fd) <= 1e-6 * max(abs(fd), 1e-3), f"bed: AD {ad:.12e} FD {fd:.12e}"


def test_checkpoint_block_follows_the_memory_budget():
    """The default checkpoint block: every state kept (k = 1) when the run
    fits the budget, else the smallest k whose ceil(n/k) block inputs plus
    a k-state recompute buffer fit, never above ceil(sqrt(n))."""
    from dclaw_b200.adjoint import checkpoint_block_for

    state = 10_485_760                       # a 512 x 512 state
    assert checkpoint_block_for(500, state, 500 * state) == 1
    assert checkpoint_block_for(500, state, 80e9) == 1
    # 500 states do not fit, 250 + 2 do
    assert checkpoint_block_for(500, state, 300 * state) == 2
    assert checkpoint_block_for(500, state, 252 * state) == 2
    assert checkpoint_block_for(500, state, 251 * state) == 3
    # nothing fits: the two-level minimum ceil(sqrt(n))
    assert checkpoint_block_for(500, state, 0) == math.ceil(math.sqrt(500)) == 23
    for n in [1, 2, 7, 100, 801]:
        for budget in [0, 5 * state, 40 * state, 1e15]:
            k = checkpoint_block_for(n, state, budget)
            assert 1 <= k <= max(1, math.ceil(math.sqrt(n)))
            if k < max(1, math.ceil(math.sqrt(n))):
                assert (-(-n // k) + (k if k > 1 else 0)) * state <= budget
            for j in range(1, k):
                assert (-(-n // j) + (j if j > 1 else 0)) * state > budget
