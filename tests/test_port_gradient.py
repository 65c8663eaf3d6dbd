"""Gradients of the step's adjoint against the reference's differentiable
port (differentiable_dclaw/dclaw_jax), restated in torch (oracle/jax_port.py)
because JAX is not installed. The port is a different discretisation (HLL
flux with hydrostatic reconstruction and SSP-RK2 instead of the augmented
f-wave solver with MC-limited corrections), so the comparison is the
qualitative one its README allows (differentiable_dclaw/README.md:343-371):
the same sign for every material parameter, magnitudes within a factor of
10, and gradients with respect to the initial depth pointing the same way
(cosine similarity > 0.9) with norms within a factor of 2.

Case: a 1.5 m paraboloid released at 2 m/s down a 30 deg plane (32 x 24
cells of 1 m, phi 28 deg, m0 0.62, pb 0.8 hydrostatic), 20 steps of
0.02 s; the loss is the depth summed over a band 6-14 m downslope of the
release point.
"""
import math

import numpy as np
import pytest
import torch

from dclaw_b200 import workloads as W
from dclaw_b200.params import DClawParams

NX, NY, DX, U0, N, DT = 32, 24, 1.0, 2.0, 20, 0.02
RHO_F, G, P_RATIO = 1000.0, 9.81, 0.8


def _case():
    x = (np.arange(NX) + 0.5) * DX
    y = (np.arange(NY) + 0.5) * DX
    X, Y = np.meshgrid(x, y)
    b = math.tan(math.radians(30.0)) * (NX * DX - X)
    h0 = np.maximum(1.5 * (1 - ((X - 8) ** 2 + (Y - 12) ** 2) / 6.0 ** 2), 0.0)
    band = (X >= 14) & (X <= 22)
    return DClawParams(phi=28.0), b, h0, band


def _port_gradient():
    from oracle import jax_port as JP

    p, b, h0, band = _case()
    th = torch.tensor([p.phi, p.kref, p.alpha_c, p.mu], dtype=torch.float64, requires_grad=True)
    h = torch.tensor(h0.T.copy(), requires_grad=True)   # the port's (nx, ny) layout
    q0 = torch.stack([h, h * U0, torch.zeros_like(h), h * 0.62, P_RATIO * RHO_F * G * h])
    out = JP.rollout(q0, torch.tensor(b.T.copy()), JP.PortParams(), th, DX, DX, DT, N)
    out[-1][0][torch.tensor(band.T)].sum().backward()
    return th.grad.numpy(), h.grad.numpy().T


def _compare(ours_theta, ours_h):
    p, b, h0, band = _case()
    port_theta, port_h = _port_gradient()
    for k, name in enumerate(["phi", "kref", "alpha_c", "mu"]):
        a, c = ours_theta[k], port_theta[k]
        assert a * c > 0.0, f"{name}: opposite signs ({a:.3e} vs {c:.3e})"
        assert 0.1 < a / c < 10.0, f"{name}: magnitudes {a:.3e} vs {c:.3e}"
    mask = h0 > 0.2
    a, c = ours_h[mask], port_h[mask]
    cos = float(a @ c / (np.linalg.norm(a) * np.linalg.norm(c)))
    assert cos > 0.9, f"depth gradients: cosine {cos:.3f}"
    assert 0.5 < np.linalg.norm(a) / np.linalg.norm(c) < 2.0


def test_port_gradient_agrees_with_host_adjoint():
    """The host build of the adjoint (the same source as the CUDA kernels)."""
    from ._adj import Adj

    adj = Adj()
    p, b, h0, band = _case()
    q0 = W.state_from(h0, np.full_like(h0, 0.62), p, P_RATIO, hu=h0 * U0, hv=0 * h0)
    s = [q0]
    for _ in range(N):
        s.append(adj.step(p, s[-1], b, DX, DX, DT))
    lam = np.zeros_like(q0)
    lam[0][band] = 1.0
    pbar = np.zeros(4)
    for k in range(N, 0, -1):
        lam, pk = adj.vjp(p, s[k - 1], b, DX, DX, DT, lam)
        pbar += pk
    theta = np.array([pbar[0] * math.pi / 180.0, pbar[1], pbar[2], pbar[3]])
    # d/dh0 through q0 = (h, U0 h, 0, 0.62 h, 0.8 rho_f g h)
    gh = lam[0] + U0 * lam[1] + 0.62 * lam[3] + P_RATIO * RHO_F * G * lam[4]
    _compare(theta, gh)


@pytest.mark.gpu
def test_port_gradient_agrees_with_cuda_adjoint(cuda_device):
    from dclaw_b200.adjoint import rollout_states, theta_of

    dev = cuda_device
    p, b, h0, band = _case()
    h = torch.tensor(h0, device=dev, requires_grad=True)
    q0 = torch.stack([h, h * U0, torch.zeros_like(h), h * 0.62, P_RATIO * RHO_F * G * h])
    theta = theta_of(p, dev).requires_grad_(True)
    o = rollout_states(q0, theta, torch.tensor(b, device=dev), p, DX, DX, N, [N], DT, fixed_dt=True)
    o[0, 0][torch.tensor(band, device=dev)].sum().backward()
    _compare(theta.grad.cpu().numpy(), h.grad.cpu().numpy())
