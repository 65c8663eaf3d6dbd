"""TEST INFRASTRUCTURE: a torch restatement of the reference's differentiable
JAX port (differentiable_dclaw/dclaw_jax/solver.py, model.py), used only to
cross-check the sign and size of gradients of the CUDA step's adjoint.

JAX is not installed here, so the port's own `jax.grad` cannot run; torch
autograd through this restatement stands in for it. The port is a different
discretisation from the Fortran step the CUDA code reproduces (HLL flux on
hydrostatically reconstructed states, SSP-RK2, smooth dry-cell ramp,
implicit pore-pressure relaxation; differentiable_dclaw/README.md:343-371),
so gradients of the two can agree in sign and order of magnitude only.

Map (paths in the youryugi/dclaw tree):
  primitive, qfix        model.py:140-160, 339-355   (EPS_H floor, m clip)
  closures               model.py:55-138             (rho, chi, k, sigma_e, D, m_eq)
  _material_state        model.py:163-192
  friction_step          model.py:301-336
  pb_relaxation_step     model.py:245-298            (6 Newton iterations)
  dilatancy_step         model.py:195-229
  _hll, _tracer_flux     solver.py:93-117
  _hr_fluxes (Audusse)   solver.py:125-191
  _upwind_grad, rhs      solver.py:194-241
  _clip_dry, step        solver.py:252-297
"""
from __future__ import annotations

import math
from typing import NamedTuple

import torch

EPS_H = 1.0e-6
SQRT_EPS = 1.0e-12
DRY_TOLERANCE = 1.0e-3
N_NEWTON_PB = 6
DILATANCY_U_TAPER = 0.05
DILATANCY_H_FLOOR = 0.02


class PortParams(NamedTuple):
    rho_s: float = 2700.0
    rho_f: float = 1000.0
    m_crit: float = 0.64
    mref: float = 0.60
    delta: float = 0.01
    sigma_0: float = 1000.0
    c1: float = 1.0
    gz: float = 9.81


def primitive(q, p):
    h, hu, hv, hm, pb = q
    hs = torch.clamp(h, min=EPS_H)
    m = torch.clamp(hm / hs, 0.0, 1.0)
    return h, hu / hs, hv / hs, m, pb, p.rho_s * m + p.rho_f * (1.0 - m)


def material(q, p, th):
    """Shared closures of the split source stages; th = (phi_deg, kref, alpha_c, mu)."""
    phi_deg, kref, alpha_c, mu = th
    h, u, v, m, pb, rho = primitive(q, p)
    vnorm = torch.sqrt(u * u + v * v + 1.0e-12)
    shear = 2.0 * vnorm / torch.clamp(h, min=EPS_H)
    k = kref * torch.exp(-(m - p.mref) / 0.04)
    sig = torch.clamp(rho * p.gz * h - pb, min=0.0)
    D = -(2.0 * k / (torch.clamp(h, min=p.delta) * mu)) * (pb - p.rho_f * p.gz * h)
    nden = p.rho_s * (shear * p.delta) ** 2 + sig
    nnum = mu * shear
    ratio = torch.sqrt(nden + SQRT_EPS) / (torch.sqrt(nden + SQRT_EPS) + torch.sqrt(torch.clamp(nnum, min=0.0) + SQRT_EPS)
                                           + EPS_H)
    m_eq = torch.where(nnum > 0.0, p.m_crit * ratio, torch.full_like(ratio, p.m_crit))
    tanpsi = p.c1 * (m - m_eq)
    tpp = torch.tan(phi_deg * (math.pi / 180.0) + torch.atan(tanpsi))
    alpha = alpha_c / (torch.clamp(m, min=EPS_H) * (sig + p.sigma_0))
    zeta = 3.0 / (2.0 * alpha * torch.clamp(h, min=EPS_H)) + p.gz * p.rho_f * (rho - p.rho_f) / (4.0 * rho)
    return dict(h=h, u=u, v=v, m=m, pb=pb, rho=rho, vnorm=vnorm, k=k, sig=sig, D=D, tanpsi=tanpsi, tpp=tpp,
                alpha=alpha, zeta=zeta)


def qfix(q, p):
    h = q[0]
    m = torch.clamp(q[3] / torch.clamp(h, min=EPS_H), 0.0, 1.0)
    rho = p.rho_s * m + p.rho_f * (1.0 - m)
    pb = torch.minimum(torch.clamp(q[4], min=0.0), rho * p.gz * torch.clamp(h, min=0.0))
    return torch.stack([q[0], q[1], q[2], h * m, pb])


def friction(q, p, th, dt):
    s = material(q, p, th)
    h, m, rho = s["h"], s["m"], s["rho"]
    hs = torch.clamp(h, min=EPS_H)
    tau = s["sig"] * s["tpp"] * 0.5 * (1.0 + torch.tanh(100.0 * (m - 0.1)))
    hv0 = torch.sqrt(q[1] ** 2 + q[2] ** 2 + 1.0e-24)
    vn = torch.clamp(hv0 / hs - dt * tau / (rho * hs), min=0.0)
    vn = vn * torch.exp(-(1.0 - m) * 2.0 * th[3] * dt / (rho * hs * hs))
    r = hs * vn / hv0
    return torch.stack([q[0], r * q[1], r * q[2], q[3], q[4]])


def pb_relax(q, p, th, dt):
    s = material(q, p, th)
    h, pb, rho = s["h"], s["pb"], s["rho"]
    rate = s["zeta"] * (2.0 * s["k"]) / (torch.clamp(h, min=p.delta) * th[3])
    p_h = p.rho_f * p.gz * h
    lith = rho * p.gz * torch.clamp(h, min=0.0)
    x = rate * dt
    ex = torch.exp(-x)
    base = pb * ex + p_h * (1.0 - ex)
    small = torch.abs(x) < 1.0e-6
    sx = torch.where(small, torch.ones_like(x), x)
    w = dt * torch.where(small, 1.0 - x / 2.0 + x * x / 6.0, (1.0 - torch.exp(-x)) / sx)

    def forcing(pb_):
        st = material(torch.stack([q[0], q[1], q[2], q[3], pb_]), p, th)
        vn = st["vnorm"]
        rr = torch.clamp(vn / DILATANCY_U_TAPER, 0.0, 1.0)
        vn = vn * rr * rr * (3.0 - 2.0 * rr)
        return -(3.0 / (st["alpha"] * torch.clamp(h, min=DILATANCY_H_FLOOR))) * vn * st["tanpsi"]

    def resid(pb_):
        return pb_ - base - w * forcing(pb_)

    pb_new = torch.minimum(torch.clamp(base + w * forcing(pb), min=0.0), lith)
    for _ in range(N_NEWTON_PB):
        x_ = pb_new if pb_new.requires_grad else pb_new.detach().requires_grad_(True)
        r = resid(x_)
        # cells are independent: the gradient of the sum is the Jacobian's diagonal
        (dr,) = torch.autograd.grad(r.sum(), x_, create_graph=True)
        pb_new = torch.minimum(torch.clamp(x_ - r / torch.clamp(dr, min=1.0), min=0.0), lith)
    return pb_new


def dilatancy(q, p, th, dt):
    s = material(q, p, th)
    h, rho, D = s["h"], s["rho"], s["D"]
    rhoh = rho * torch.clamp(h, min=EPS_H)
    fm = torch.exp(-dt * D * p.rho_f / rhoh)
    fh = torch.exp(dt * D * (rho - p.rho_f) / rhoh)
    return torch.stack([q[0] * fh, q[1] * fh, q[2] * fh, q[3] * fm, q[4]])


def _pad(q, axis, bc):
    """one ghost cell each side of spatial axis (0 = x = dim 1 of (5, nx, ny))"""
    a = axis + 1
    lo = q.narrow(a, 0, 1)
    hi = q.narrow(a, q.shape[a] - 1, 1)
    comp = 1 if axis == 0 else 2
    if bc == "wall" and comp < q.shape[0]:   # a one-field pad (pb, h) has no momentum to flip
        sgn = torch.ones(q.shape[0], dtype=q.dtype, device=q.device)
        sgn[comp] = -1.0
        sgn = sgn.view(-1, *([1] * (q.dim() - 1)))
        lo, hi = lo * sgn, hi * sgn
    return torch.cat([lo, q, hi], dim=a)


def _flux(q, p, axis):
    h, u, v, m, pb, rho = primitive(q, p)
    z = torch.zeros_like(h)
    if axis == 0:
        return torch.stack([q[1], q[1] * u + 0.5 * p.gz * h * h, q[1] * v, z, z])
    return torch.stack([q[2], q[2] * u, q[2] * v + 0.5 * p.gz * h * h, z, z])


def _hll(qL, qR, p, axis):
    hL, uL, vL = primitive(qL, p)[:3]
    hR, uR, vR = primitive(qR, p)[:3]
    unL, unR = (uL, uR) if axis == 0 else (vL, vR)
    cL = torch.sqrt(p.gz * torch.clamp(hL, min=0.0) + SQRT_EPS)
    cR = torch.sqrt(p.gz * torch.clamp(hR, min=0.0) + SQRT_EPS)
    sL = torch.clamp(torch.minimum(unL - cL, unR - cR), max=0.0)
    sR = torch.clamp(torch.maximum(unL + cL, unR + cR), min=0.0)
    fL, fR = _flux(qL, p, axis), _flux(qR, p, axis)
    return (sR * fL - sL * fR + sL * sR * (qR - qL)) / torch.clamp(sR - sL, min=SQRT_EPS)


def _hr_fluxes(q, b, axis, bc, p):
    a = axis + 1
    qp = _pad(q, axis, bc)
    bp = _pad(b.expand_as(q), axis, bc)[0]
    n = qp.shape[a]
    qL, qR = qp.narrow(a, 0, n - 1), qp.narrow(a, 1, n - 1)
    bL, bR = bp.narrow(axis, 0, n - 1), bp.narrow(axis, 1, n - 1)
    hL, hR = qL[0], qR[0]
    zf = torch.maximum(bL, bR)
    hLs = torch.clamp(hL + bL - zf, min=0.0)
    hRs = torch.clamp(hR + bR - zf, min=0.0)
    qLs = qL * (hLs / torch.clamp(hL, min=1.0e-12))[None]
    qRs = qR * (hRs / torch.clamp(hR, min=1.0e-12))[None]
    f = _hll(qLs, qRs, p, axis)
    mL, mR = primitive(qL, p)[3], primitive(qR, p)[3]
    f = torch.cat([f[:3], (f[0] * torch.where(f[0] > 0.0, mL, mR))[None], f[4:]])
    mom = 1 + axis
    addL = torch.zeros_like(f)
    addR = torch.zeros_like(f)
    addL[mom] = 0.5 * p.gz * (hL * hL - hLs * hLs)
    addR[mom] = 0.5 * p.gz * (hR * hR - hRs * hRs)
    return f + addL, f + addR


def _upwind(field, vel, axis, d, bc):
    padded = _pad(field[None], axis, bc)[0]
    n = padded.shape[axis]
    fwd = (padded.narrow(axis, 2, n - 2) - padded.narrow(axis, 1, n - 2)) / d
    bwd = (padded.narrow(axis, 1, n - 2) - padded.narrow(axis, 0, n - 2)) / d
    return torch.where(vel >= 0.0, bwd, fwd)


def rhs(q, b, p, dx, dy, bc="wall"):
    h, u, v, m, pb, rho = primitive(q, p)
    fxL, fxR = _hr_fluxes(q, b, 0, bc, p)
    dfx = (fxL[:, 1:, :] - fxR[:, :-1, :]) / dx
    fyL, fyR = _hr_fluxes(q, b, 1, bc, p)
    dfy = (fyL[:, :, 1:] - fyR[:, :, :-1]) / dy
    dh = -dfx[0] - dfy[0]
    dhu = -dfx[1] - dfy[1]
    dhv = -dfx[2] - dfy[2]
    dhm = -dfx[3] - dfy[3]
    dpbx = _upwind(pb, u, 0, dx, bc)
    dpby = _upwind(pb, v, 1, dy, bc)
    hadv = u * _upwind(h, u, 0, dx, bc) + v * _upwind(h, v, 1, dy, bc)
    chi = (p.rho_f + 3.0 * rho) / (4.0 * rho)
    dpb = chi * rho * p.gz * (dh + hadv) - (u * dpbx + v * dpby)
    return torch.stack([dh, dhu, dhv, dhm, dpb])


def clip_dry(q):
    h = torch.clamp(q[0], min=0.0)
    s = torch.clamp((h - DRY_TOLERANCE) / DRY_TOLERANCE, 0.0, 1.0)
    w = s * s * (3.0 - 2.0 * s)
    return torch.cat([h[None], q[1:]]) * w[None]


def step(q, b, p, th, dx, dy, dt, bc="wall"):
    """One step of the port's scheme on a (5, nx, ny) state (x = dim 1)."""
    k1 = rhs(q, b, p, dx, dy, bc)
    q1 = clip_dry(q + dt * k1)
    k2 = rhs(q1, b, p, dx, dy, bc)
    qt = clip_dry(q + 0.5 * dt * (k1 + k2))
    qf = friction(qfix(qt, p), p, th, dt)
    qr = qfix(torch.cat([qf[:4], pb_relax(qf, p, th, dt)[None]]), p)
    return clip_dry(qfix(dilatancy(qr, p, th, dt), p))


def rollout(q0, b, p, th, dx, dy, dt, n_steps, bc="wall"):
    q = q0
    out = []
    for _ in range(n_steps):
        q = step(q, b, p, th, dx, dy, dt, bc)
        out.append(q)
    return out
