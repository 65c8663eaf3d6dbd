"""Seeded synthetic inputs for the uniform-patch benchmark cases.

No public benchmark suite is involved: every case is a synthetic terrain and
initial mass built here from a seed. State arrays are (5, my, mx) float64
(h, hu, hv, hm, pb), beds are (my, mx), x fastest; cell centres sit at
(i + 0.5) dx. Initial pore pressure follows init_ptype = 3 style
initialisation, pb = ratio * rho_f * g * h (src/2d/dig/qinit.f90:264-285),
followed by the admissibility clip of qfix.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np

from .params import DClawParams


@dataclasses.dataclass
class Case:
    name: str
    q: np.ndarray          # (5, my, mx)
    b: np.ndarray          # (my, mx)
    dx: float
    dy: float
    params: DClawParams
    nsteps: int
    dt_initial: float

    @property
    def mx(self) -> int:
        return self.q.shape[2]

    @property
    def my(self) -> int:
        return self.q.shape[1]


def _admissible(q: np.ndarray, p: DClawParams) -> np.ndarray:
    """qfix on a whole state (digclaw_module.f90:285-345), numpy form."""
    h, hu, hv, hm, pb = q
    wet = h > p.dry_tolerance
    hs = np.where(wet, h, 1.0)
    m = np.clip(hm / hs, 0.0, 1.0)
    rho = p.rho_s * m + (1.0 - m) * p.rho_f
    pb = np.clip(pb, 0.0, rho * p.grav * h)
    out = np.stack([h, hu, hv, h * m, pb])
    out[:, ~wet] = 0.0
    return out


def state_from(h: np.ndarray, m: np.ndarray, p: DClawParams, p_ratio: float = 0.8,
               hu: np.ndarray | None = None, hv: np.ndarray | None = None) -> np.ndarray:
    z = np.zeros_like(h)
    q = np.stack([h, z if hu is None else hu, z if hv is None else hv, h * m, p_ratio * p.rho_f * p.grav * h])
    return _admissible(q, p)


def slope_runout(n: int = 200, dx: float = 1.0, nsteps: int = 1000, params: DClawParams | None = None) -> Case:
    """200 x 200, dx 1 m: planar 30 deg slope b = tan30 (200 - x) flattening
    to a horizontal runout for x > 150; paraboloid hump h = 2 (1 - r^2/20^2)+
    at (40, 100), at rest, m0 = 0.62, pb = 0.8 rho_f g h; walls."""
    p = params or DClawParams()
    x = (np.arange(n) + 0.5) * dx
    X, Y = np.meshgrid(x, x, indexing="xy")
    L = n * dx
    b = math.tan(math.radians(30.0)) * (L - np.minimum(X, 150.0 * dx / 1.0 if dx == 1.0 else 0.75 * L))
    r2 = (X - 40.0 * (L / 200.0)) ** 2 + (Y - 100.0 * (L / 200.0)) ** 2
    R = 20.0 * (L / 200.0)
    h = np.maximum(2.0 * (1.0 - r2 / R**2), 0.0)
    q = state_from(h, np.full_like(h, 0.62), p, 0.8)
    return Case("slope_runout_200", q, b, dx, dx, p, nsteps, 0.01)


def full_state(q: np.ndarray, params: DClawParams) -> np.ndarray:
    """The reference's whole state (7, my, mx) = (h, hu, hv, hm, pb, hchi,
    bdif) from a five-field one: hchi = chi0 h where segregation is on, as
    qinit sets it (qinit.f90:219-226), else 0; no bed eroded yet (bdif = 0)."""
    z = np.zeros_like(q[0])
    hchi = params.chi0 * q[0] if params.segregation == 1 else z
    return np.concatenate([q, hchi[None], z[None]])


@dataclasses.dataclass
class FullCase:
    """A case on the whole state, with the erodible depth of entrainment."""

    name: str
    q: np.ndarray        # (7, my, mx)
    b: np.ndarray
    h_e: np.ndarray      # (my, mx) erodible depth aux(i_ent)
    dx: float
    dy: float
    params: DClawParams
    nsteps: int
    dt_initial: float


def slope_runout_full(n: int = 200, segregation: int = 1, entrainment: int = 1, beta_seg: float = 0.3,
                      erodible: float = 0.5, params: DClawParams | None = None) -> FullCase:
    """The slope-runout case on the whole state: with segregation a mixture of
    half and half species (chi0 = 0.5) and a species flux coefficient
    beta_seg; with entrainment (method 0, ent_dclaw4) an erodible layer of
    `erodible` m on the slope below the release (x in [60, 150] of 200),
    solid fraction me = 0.65."""
    base = slope_runout(n=n)
    p = (params or base.params).replace(segregation=segregation, beta_seg=beta_seg, entrainment=entrainment,
                                        entrainment_method=0)
    x = (np.arange(n) + 0.5) * base.dx
    X = np.broadcast_to(x[None, :], base.b.shape)
    L = n * base.dx
    h_e = np.where((X >= 0.3 * L) & (X <= 0.75 * L), erodible, 0.0)
    return FullCase(f"slope_runout_full_{n}", full_state(base.q, p), base.b, np.ascontiguousarray(h_e),
                    base.dx, base.dy, p, base.nsteps, base.dt_initial)


def gaussian_random_field(n: int, dx: float, rms: float, slope: float, seed: int) -> np.ndarray:
    """Isotropic Gaussian random field with power spectrum ~ k^slope (slope -3),
    zero mean, scaled to the given RMS."""
    rng = np.random.default_rng(seed)
    white = rng.standard_normal((n, n))
    F = np.fft.rfft2(white)
    kx = np.fft.rfftfreq(n, d=dx)
    ky = np.fft.fftfreq(n, d=dx)
    K = np.sqrt(kx[None, :] ** 2 + ky[:, None] ** 2)
    K[0, 0] = np.inf
    F *= K ** (slope / 2.0)
    f = np.fft.irfft2(F, s=(n, n))
    f -= f.mean()
    f *= rms / f.std()
    return f


def random_terrain(n: int, dx: float, seed: int, tilt_deg: float = 20.0, rms: float = 5.0) -> np.ndarray:
    x = (np.arange(n) + 0.5) * dx
    tilt = math.tan(math.radians(tilt_deg)) * (n * dx - x)[None, :]
    return gaussian_random_field(n, dx, rms, -3.0, seed) + tilt


def paraboloid_sources(n: int, dx: float, seed: int, count: int = 32, wet_fraction: float = 0.30,
                       params: DClawParams | None = None) -> np.ndarray:
    """Sum of `count` seeded paraboloids, peaks U[0.5, 3] m, m0 U[0.55, 0.64]
    per source, radii sized so that about `wet_fraction` of the cells are wet."""
    p = params or DClawParams()
    rng = np.random.default_rng(seed + 1000)
    L = n * dx
    r_mean = math.sqrt(wet_fraction * L * L / (count * math.pi))
    x = (np.arange(n) + 0.5) * dx
    h = np.zeros((n, n))
    hm = np.zeros((n, n))
    for _ in range(count):
        cx, cy = rng.uniform(0.08 * L, 0.92 * L, size=2)
        peak = rng.uniform(0.5, 3.0)
        R = r_mean * rng.uniform(0.85, 1.15)
        m0 = rng.uniform(0.55, 0.64)
        dxs = (x - cx) ** 2
        dys = (x - cy) ** 2
        hk = np.maximum(peak * (1.0 - (dys[:, None] + dxs[None, :]) / R**2), 0.0)
        h += hk
        hm += hk * m0
    m = np.where(h > 0, hm / np.where(h > 0, h, 1.0), 0.0)
    return state_from(h, m, p, 0.8)


def random_field_case(n: int = 4096, dx: float = 0.5, seed: int = 0, nsteps: int = 200,
                      params: DClawParams | None = None) -> Case:
    """4096 x 4096, dx 0.5 m: Gaussian random terrain (spectral slope -3,
    5 m RMS) on a 20 deg tilt, 32 seeded paraboloid sources (~70% dry)."""
    p = params or DClawParams()
    b = random_terrain(n, dx, seed)
    q = paraboloid_sources(n, dx, seed, params=p)
    return Case(f"random_field_{n}", q, b, dx, dx, p, nsteps, 0.01)


# ---- known-answer setups from the reference's own tests -------------------
def contact_wave(params: DClawParams | None = None) -> Case:
    """tests/eigenstructure_check (setinput.py:27-34, setrun.py:65-149):
    m-jump 0.55 / 0.60 at x = 0 in 1 m still water on a flat bed,
    x in [-5, 5], y in [-0.25, 0.25], 0.05 m cells, order 1, no transverse
    waves, MC limiter, walls except an extrapolation boundary at x upper."""
    p = params or DClawParams(rho_f=1000.0, rho_s=2700.0, m_crit=0.64, m0=0.55, mref=0.60, kref=5.0e-9,
                              phi=35.0, delta=0.001, mu=0.005, alpha_c=0.01, c1=1.0, sigma_0=1000.0,
                              order=1, transverse_waves=0, limiter=4, cfl_desired=0.4, cfl_max=0.5,
                              dt_max=0.01, bc_lower=("wall", "wall"), bc_upper=("extrap", "wall"))
    dx = 0.05
    mx, my = 200, 10
    x = -5.0 + (np.arange(mx) + 0.5) * dx
    h = np.ones((my, mx))
    m = np.where(x < 0.0, 0.55, 0.60)[None, :] * np.ones((my, 1))
    q = state_from(h, m, p, 1.0)   # init_ptype = 3 with init_pratio = 1: hydrostatic
    b = np.zeros((my, mx))
    return Case("contact_wave", q, b, dx, dx, p, 0, 1.0e-5)


def dam_front(params: DClawParams | None = None) -> Case:
    """tests/eigenstructure_check damfront: h_L = 2 m for x < 5 on a dry flat
    bed, x in [0, 20], phi = 0, same numerics as the contact test."""
    p = params or contact_wave().params.replace(phi=0.0)
    dx = 0.05
    mx, my = 400, 10
    x = (np.arange(mx) + 0.5) * dx
    h = np.where(x < 5.0, 2.0, 0.0)[None, :] * np.ones((my, 1))
    m = np.full((my, mx), 0.55)
    q = state_from(h, m, p, 1.0)
    b = np.zeros((my, mx))
    return Case("dam_front", q, b, dx, dx, p, 0, 1.0e-5)


def lake_at_rest(params: DClawParams | None = None) -> Case:
    """differentiable_dclaw/tests/test_lake_at_rest.py:22-36: still water at
    eta = 5 m over a bump, a tilt, a pit and a dry island; 60 x 60 cells of
    5 m; phi = 0, c1 = 0; pb = rho_f g h."""
    p = params or DClawParams(phi=0.0, c1=0.0, m_crit=0.64, kref=1.0e-9, mu=0.005)
    n, dx = 60, 5.0
    x = (np.arange(n) + 0.5) * dx
    X, Y = np.meshgrid(x, x, indexing="ij")
    b = (3.0 * np.exp(-((X - 100) ** 2 + (Y - 150) ** 2) / 400.0) + 0.02 * X
         - 1.5 * np.exp(-((X - 200) ** 2 + (Y - 80) ** 2) / 300.0)
         + 6.0 * np.exp(-((X - 220) ** 2 + (Y - 220) ** 2) / 200.0))
    b = b.T  # (my, mx) with x fastest
    h = np.maximum(5.0 - b, 0.0)
    m = np.where(h > 0, 0.5, 0.0)
    z = np.zeros_like(h)
    q = np.stack([h, z, z, h * m, 1000.0 * 9.81 * h])
    q = _admissible(q, p)
    return Case("lake_at_rest", q, b, dx, dx, p, 0, 0.01)


# ---- flume ensembles (batched particle-filter case) -------------------------
def flume_member(width: int, length: int, dx: float, params: DClawParams, slope_deg: float = 31.0,
                 runout_frac: float = 0.25, block_len: float = 3.0, block_h: float = 1.0, p_ratio: float = 0.8):
    """One channel: `length` cells along x at dx, `width` cells across; a
    planar slope of slope_deg down to a horizontal runout over the last
    runout_frac of the length; a rectangular release block block_len m long
    and block_h m high at the head (3 m^2 per metre of width: the cross
    section of a 6 m^3 release in a 2 m wide flume), at rest."""
    x = (np.arange(length) + 0.5) * dx
    L = length * dx
    xb = (1.0 - runout_frac) * L
    b1 = math.tan(math.radians(slope_deg)) * np.maximum(xb - x, 0.0)
    b = np.broadcast_to(b1[None, :], (width, length)).copy()
    h1 = np.where((x >= 0.5) & (x < 0.5 + block_len), block_h, 0.0)
    h = np.broadcast_to(h1[None, :], (width, length)).copy()
    q = state_from(h, np.full_like(h, params.m0), params, p_ratio)
    return q, b


def flume_ensemble(n: int = 256, seed: int = 0, dx: float = 0.05, width_range=(32, 128),
                   length_range=(1024, 4096), nsteps: int = 2000):
    """n flume members of uneven sizes with per-member parameters drawn from
    the priors phi U[28, 40] deg, log10 k0 U[-11, -8], m0 U[0.55, 0.65],
    alpha U[0.005, 0.05]."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        w = int(rng.integers(width_range[0], width_range[1] + 1))
        L = int(rng.integers(length_range[0], length_range[1] + 1))
        p = DClawParams(phi=float(rng.uniform(28.0, 40.0)), kref=float(10.0 ** rng.uniform(-11.0, -8.0)),
                        m0=float(rng.uniform(0.55, 0.65)), alpha_c=float(rng.uniform(0.005, 0.05)))
        q, b = flume_member(w, L, dx, p)
        out.append(Case(f"flume_{w}x{L}", q, b, dx, dx, p, nsteps, 1.0e-3))
    return out


# ---- gradient case -----------------------------------------------------------
@dataclasses.dataclass
class GradientCase:
    """Loss over gauge cells and output times for the gradient benchmark."""

    b: np.ndarray            # (my, mx)
    h0: np.ndarray           # (my, mx) initial depth
    m0: float                # solid fraction of the initial mass
    params: DClawParams      # parameters the gradient is taken at
    true_params: DClawParams  # parameters of the synthetic target run
    gauges: np.ndarray       # (n_gauges, 2) cell indices (j, i)
    out_steps: list          # step counts at which the gauges are read
    nsteps: int
    dx: float
    dt_initial: float


def gradient_case(n: int = 512, dx: float = 1.0, seed: int = 7, nsteps: int = 500, n_gauges: int = 64,
                  n_out: int = 50) -> GradientCase:
    """512 x 512, dx 1 m: the random terrain of the 4096 x 4096 case at this
    seed, paraboloid sources (one uniform solid fraction m0 = 0.62), 64
    seeded gauge cells among the cells the initial mass covers or borders,
    read at 50 evenly spaced output steps over 500 steps. The target comes
    from the same solver at perturbed true parameters (phi 30 deg, kref
    3e-10, alpha_c 0.015). b4step2's speed limit is 30 m/s, the value of the
    reference's own example (examples/gully/setrun.py:519): without it thin
    cells at the flow's edges reach 10-100 m/s and the gradient of a long
    run is dominated by them."""
    p = DClawParams(speed_limit=30.0)
    b = random_terrain(n, dx, seed)
    src = paraboloid_sources(n, dx, seed, params=p)
    h0 = src[0]
    rng = np.random.default_rng(seed + 2000)
    near = np.argwhere(np.maximum.reduce([np.roll(h0, s, a) for a in (0, 1) for s in (-8, 0, 8)]) > 0)
    gauges = near[rng.choice(len(near), size=n_gauges, replace=False)]
    every = max(1, nsteps // n_out)
    out_steps = list(range(every, nsteps + 1, every))[:n_out]
    true = p.replace(phi=30.0, kref=3.0e-10, alpha_c=0.015)
    return GradientCase(b, h0, 0.62, p, true, gauges, out_steps, nsteps, dx, 0.05)


@dataclasses.dataclass
class BatchedGradientCase:
    """Per-member gauge losses over an ensemble of channels."""

    members: list            # Case per member (q at the members' own release block)
    true_params: list        # DClawParams per member for the synthetic targets
    block_masks: list        # (my, mx) 0/1 masks of the release blocks
    block_area: list         # m^2 of each release block
    gauges: list             # (16, 2) cell indices (j, i) per member, along the centreline
    out_steps: list
    nsteps: int


def batched_gradient_case(n: int = 64, seed: int = 11, length: int = 1024, width_range=(128, 256),
                          dx: float = 0.05, n_gauges: int = 16, nsteps: int = 800, n_out: int = 50):
    """n channels of `length` x U[width_range] cells at dx on a 31 deg slope with a
    horizontal runout (the flume members of the ensemble case), each with its
    own parameters from the priors (phi U[28, 40] deg, log10 k0 U[-11, -8],
    m0 U[0.55, 0.65], alpha U[0.005, 0.05]) and a 3 m x 1 m release block;
    16 gauges along each centreline from below the block to the runout, read
    at n_out evenly spaced output steps. Each member's target comes from the
    same solver at its own perturbed parameters (phi + 1.5 deg, kref x 2,
    alpha_c x 1.3)."""
    rng = np.random.default_rng(seed)
    members, true, masks, areas, gauges = [], [], [], [], []
    for _ in range(n):
        w = int(rng.integers(width_range[0], width_range[1] + 1))
        p = DClawParams(phi=float(rng.uniform(28.0, 40.0)), kref=float(10.0 ** rng.uniform(-11.0, -8.0)),
                        m0=float(rng.uniform(0.55, 0.65)), alpha_c=float(rng.uniform(0.005, 0.05)))
        q, b = flume_member(w, length, dx, p)
        mask = (q[0] > 0.0).astype(np.float64)
        members.append(Case(f"channel_{w}x{length}", q, b, dx, dx, p, nsteps, 1.0e-3))
        true.append(p.replace(phi=p.phi + 1.5, kref=2.0 * p.kref, alpha_c=1.3 * p.alpha_c))
        masks.append(mask)
        areas.append(float(mask.sum()) * dx * dx)
        xi = np.linspace(int(4.0 / dx), int(0.9 * length), n_gauges).astype(int)
        gauges.append(np.stack([np.full(n_gauges, w // 2), xi], axis=1))
    every = max(1, nsteps // n_out)
    out_steps = list(range(every, nsteps + 1, every))[:n_out]
    return BatchedGradientCase(members, true, masks, areas, gauges, out_steps, nsteps)
