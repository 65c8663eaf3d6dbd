"""The full-state step (dclaw_step_full: segregation and entrainment) on the
GPU through the C ABI, against the oracle's seven-field restatement of the
reference (src/2d/dig/*.f90) with the same elementary functions: state,
species field hchi, eroded bed bdif, dt/Courant histories and branch bits
bit for bit; against the glibc oracle to 1e-12 over the first steps."""
import ctypes

import numpy as np
import pytest
import torch

from dclaw_b200 import _lib
from dclaw_b200 import workloads as W
from dclaw_b200.params import CLOCK_DOUBLES
from dclaw_b200.solver import PatchStepper

pytestmark = pytest.mark.gpu


def _run(c, p, n, dev, branch_log=True, h_e=True):
    st = PatchStepper(torch.tensor(c.q, device=dev), torch.tensor(c.b, device=dev), p, c.dx, c.dy,
                      branch_log=branch_log, h_e=torch.tensor(c.h_e, device=dev) if h_e else None)
    st.init_clock(c.dt_initial)
    hist = torch.zeros((n, 4), dtype=torch.float64, device=dev)
    st.step(n, history=hist)
    torch.cuda.synchronize()
    return dict(q=st.state().cpu().numpy(), hist=hist.cpu().numpy(),
                br=st.brlog.cpu().numpy().view(np.uint32) if branch_log else None, status=st.status())


VARIANTS = {
    "segregation_entrainment": dict(),
    "segregation": dict(entrainment=0),
    "entrainment": dict(segregation=0),
    "manning": dict(friction_forcing=True, manning_coefficient=0.03),
    "src2method1": dict(src2method=1),
    "src2method2": dict(src2method=2, alphamethod=1),
    "order1": dict(order=1, transverse_waves=0),
}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_full_state_matches_oracle(cuda_device, oracle, variant):
    c = W.slope_runout_full(n=96)
    p = c.params.replace(**VARIANTS[variant])
    n = 80
    g = _run(c, p, n, cuda_device)
    o = oracle.run_full(p, c.q, c.b, c.dx, c.dy, n, c.dt_initial, h_e=c.h_e, branch_log=True, libm="portable")
    assert g["status"] == 0 and o["status"] == 0
    br = np.concatenate([o["xlog"].ravel(), o["ylog"].ravel()])
    assert int((g["br"] != br).sum()) == 0
    assert np.array_equal(g["q"], o["q"])
    assert np.array_equal(g["hist"][:, 3], o["dt"]) and np.array_equal(g["hist"][:, 2], o["cfl"])
    if p.entrainment:
        assert g["q"][6].max() > 0.0
    if p.segregation:
        wet = g["q"][0] > 0
        chi = g["q"][5][wet] / g["q"][0][wet]
        assert chi.min() < 0.45 and chi.max() > 0.55  # the species have separated


def test_full_state_against_glibc_oracle(cuda_device, oracle):
    c = W.slope_runout_full(n=96)
    g = _run(c, c.params, 3, cuda_device, branch_log=False)
    o = oracle.run_full(c.params, c.q, c.b, c.dx, c.dy, 3, c.dt_initial, h_e=c.h_e, libm="glibc")
    assert np.array_equal(g["q"][0] == 0.0, o["q"][0] == 0.0)
    for m in range(7):
        scale = max(np.abs(o["q"][m]).max(), 1e-300)
        assert np.abs(g["q"][m] - o["q"][m]).max() / scale <= 1e-12, f"field {m}"


def test_full_state_without_extras_equals_the_five_field_step(cuda_device):
    """hchi = bdif = 0, segregation and entrainment off: the full-state step
    returns dclaw_step's bits (the tile-list path) and keeps the extra fields
    zero."""
    base = W.slope_runout(n=128)
    dev = cuda_device
    a = PatchStepper(torch.tensor(base.q, device=dev), torch.tensor(base.b, device=dev), base.params, base.dx,
                     base.dy)
    f = PatchStepper(torch.tensor(W.full_state(base.q, base.params), device=dev), torch.tensor(base.b, device=dev),
                     base.params, base.dx, base.dy)
    for st in (a, f):
        st.init_clock(base.dt_initial)
        st.step(60)
    torch.cuda.synchronize()
    assert torch.equal(a.state(), f.state()[:5])
    assert not torch.any(f.state()[5:])
    assert a.read_clock().dt == f.read_clock().dt


def test_five_field_entry_points_refuse_segregation(cuda_device):
    c = W.slope_runout(n=16)
    b = torch.tensor(c.b, device=cuda_device)
    for kw in (dict(segregation=1), dict(entrainment=1, entrainment_method=0)):
        with pytest.raises(_lib.DClawError):
            PatchStepper(torch.tensor(c.q, device=cuda_device), b, c.params.replace(**kw), c.dx, c.dy)


def test_entrainment_needs_the_erodible_depth(cuda_device):
    c = W.slope_runout_full(n=32)
    lib = _lib.load()
    dev = cuda_device
    q = torch.tensor(c.q, device=dev)
    out = torch.empty_like(q)
    b = torch.tensor(c.b, device=dev)
    work = torch.empty(lib.dclaw_step_full_workspace_bytes(c.q.shape[2], c.q.shape[1]), dtype=torch.uint8,
                       device=dev)
    clk = torch.zeros(CLOCK_DOUBLES, dtype=torch.float64, device=dev)
    cp = c.params.to_c()
    rc = lib.dclaw_step_full(_lib.ptr(q), _lib.ptr(out), _lib.ptr(b), None, c.q.shape[2], c.q.shape[1], c.dx, c.dy,
                             ctypes.byref(cp), _lib.ptr(clk), _lib.ptr(work), work.numel(), None, _lib.stream_ptr())
    assert rc == 1  # DCLAW_ERR_ARG


@pytest.mark.parametrize("case", ["slope_runout", "random_field"])
def test_full_state_skip_matches_full_grid(cuda_device, case):
    """Without a branch log the full-state step skips the cells, fluxes and
    solves that no active tile reads; with one it computes every item. The
    two give the same state, eroded depth and dt history bit for bit over a
    run whose flow front crosses tiles (a slope runout, and a random field
    with about 70 % of its cells dry)."""
    if case == "slope_runout":
        c = W.slope_runout_full(n=96)
        q, b, he, p, dx, dy, dt0, n = c.q, c.b, c.h_e, c.params, c.dx, c.dy, c.dt_initial, 120
    else:
        r = W.random_field_case(n=256, dx=0.5, seed=5)
        p = r.params.replace(segregation=1, beta_seg=0.3, entrainment=1, entrainment_method=0)
        q, b, dx, dy, dt0, n = W.full_state(r.q, p), r.b, r.dx, r.dy, r.dt_initial, 60
        he = np.full(r.b.shape, 0.5)
    c2 = W.FullCase("skip", q, b, np.ascontiguousarray(he), dx, dy, p, n, dt0)
    a = _run(c2, p, n, cuda_device, branch_log=True)
    s = _run(c2, p, n, cuda_device, branch_log=False)
    assert a["status"] == 0 and s["status"] == 0
    assert np.array_equal(a["q"], s["q"])
    assert np.array_equal(a["hist"], s["hist"])
    assert a["q"][6].max() > 0.0
