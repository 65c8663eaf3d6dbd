"""The allocation-free fused step, dclaw_step_noalloc, through the C ABI.

Callers that drive the step from code without a device allocator of their
own (a Fortran time loop bound through iso_c_binding, or a host application
that hands the library only the state it already owns) use this entry point:
its scratch is a fixed device array inside the library instead of a
caller-provided workspace. These checks compare it with dclaw_step (the
workspace entry point) bit for bit -- the tolerance every parity test here
uses -- on two consecutive calls, so the second call also sees the scratch
the first one left behind, and check that oversized patches are refused.
This file sorts last so that a run stopping at its first failure has run
every other test before it.
"""
import ctypes

import numpy as np
import pytest
import torch

from dclaw_b200 import _lib
from dclaw_b200 import workloads as W
from dclaw_b200.params import CLOCK_DOUBLES

pytestmark = pytest.mark.gpu


def _clock(dev, dt):
    lib = _lib.load()
    clk = torch.zeros(CLOCK_DOUBLES, dtype=torch.float64, device=dev)
    _lib.check(lib.dclaw_clock_init(_lib.ptr(clk), 0.0, dt, 0.0, 0, _lib.stream_ptr()), "clock init")
    return clk


# 200 x 200 uses a sixth of the scratch; 508 x 508 fills it exactly
# ((508 + 4)^2 = 2^18 padded cells), where a wrong size check or plane stride
# would first reach past the array
@pytest.mark.parametrize("n", [200, 508])
def test_noalloc_matches_workspace_step_on_two_calls(n):
    assert torch.cuda.is_available()
    lib = _lib.load()
    dev = torch.device("cuda:0")
    c = W.random_field_case(n=n, dx=0.5, seed=21)
    mx, my = c.mx, c.my
    assert (mx + 4) * (my + 4) <= lib.dclaw_step_noalloc_max_cells()
    if n == 508:
        assert (mx + 4) * (my + 4) == lib.dclaw_step_noalloc_max_cells()
    cp = c.params.to_c()
    q0 = torch.tensor(c.q, device=dev)
    b = torch.tensor(c.b, device=dev)
    s = _lib.stream_ptr()

    # reference: the workspace entry point, two steps
    work_bytes = lib.dclaw_workspace_bytes(mx, my)
    work = torch.empty(work_bytes, dtype=torch.uint8, device=dev)
    clk_a = _clock(dev, c.dt_initial)
    qa1, qa2 = torch.empty_like(q0), torch.empty_like(q0)
    _lib.check(lib.dclaw_step(_lib.ptr(q0), _lib.ptr(qa1), _lib.ptr(b), mx, my, c.dx, c.dy, ctypes.byref(cp),
                              _lib.ptr(clk_a), _lib.ptr(work), work_bytes, None, s), "dclaw_step")
    _lib.check(lib.dclaw_step(_lib.ptr(qa1), _lib.ptr(qa2), _lib.ptr(b), mx, my, c.dx, c.dy, ctypes.byref(cp),
                              _lib.ptr(clk_a), _lib.ptr(work), work_bytes, None, s), "dclaw_step")

    # the allocation-free entry point, two calls in a row
    clk_b = _clock(dev, c.dt_initial)
    qb1, qb2 = torch.empty_like(q0), torch.empty_like(q0)
    _lib.check(lib.dclaw_step_noalloc(_lib.ptr(q0), _lib.ptr(qb1), _lib.ptr(b), mx, my, c.dx, c.dy,
                                      ctypes.byref(cp), _lib.ptr(clk_b), s), "dclaw_step_noalloc")
    torch.cuda.synchronize()
    assert torch.equal(qb1, qa1)
    _lib.check(lib.dclaw_step_noalloc(_lib.ptr(qb1), _lib.ptr(qb2), _lib.ptr(b), mx, my, c.dx, c.dy,
                                      ctypes.byref(cp), _lib.ptr(clk_b), s), "dclaw_step_noalloc")
    torch.cuda.synchronize()
    assert torch.equal(qb2, qa2)
    assert torch.equal(clk_a[:4], clk_b[:4])  # t, next dt, Courant number, dt used
    assert int(clk_b.cpu().numpy().view(np.int32)[14]) == 0  # status word
    assert (qb2[0] > 0).sum().item() > 1000
    # the second call also moved the state (not a copy of the first result)
    assert not torch.equal(qb2, qb1)


# far beyond the limit, and one row beyond it (512 x 513 padded cells)
@pytest.mark.parametrize("mx,my", [(600, 600), (508, 509)])
def test_noalloc_rejects_oversized_patch(mx, my):
    lib = _lib.load()
    dev = torch.device("cuda:0")
    cp = W.slope_runout(n=16).params.to_c()
    q = torch.zeros((5, my, mx), dtype=torch.float64, device=dev)
    out = torch.empty_like(q)
    b = torch.zeros((my, mx), dtype=torch.float64, device=dev)
    clk = _clock(dev, 0.01)
    rc = lib.dclaw_step_noalloc(_lib.ptr(q), _lib.ptr(out), _lib.ptr(b), mx, my, 1.0, 1.0, ctypes.byref(cp),
                                _lib.ptr(clk), _lib.stream_ptr())
    assert rc == 6  # DCLAW_ERR_TOO_LARGE
    assert lib.dclaw_error_string(rc) == b"size beyond the fixed limit"
