"""The host-buffer step, dclaw_step_host: a state in host memory stepped with
its copies pipelined band by band against the compute.

The band plan and the argument checks run on the CPU (host-side calls
only). On the GPU the step is compared bit for bit with dclaw_step on the
same state over several steps: square and ragged patches, wet/dry fronts
crossing band edges, band counts from one to one per tile row (and more
than there are, which is capped), in place and out of place, pinned and
pageable host memory.
"""
import ctypes

import numpy as np
import pytest
import torch

from dclaw_b200 import _lib
from dclaw_b200 import workloads as W
from dclaw_b200.params import DClawParams

def _plan(lib, mx, my, nbands):
    first = (ctypes.c_int32 * 66)()
    nb = lib.dclaw_step_host_bands(mx, my, nbands, first, 66)
    return nb, list(first[: nb + 1])


def test_band_plan_covers_every_tile_row():
    lib = _lib.load()
    tile_y = lib.dclaw_rows_granule()      # cells per tile row of the fused step
    for mx, my in [(2, 2), (37, 53), (200, 200), (513, 1000), (4096, 4096), (100, 20000)]:
        nty = -(-my // tile_y)
        for nbands in [0, 1, 2, 3, 7, 64, 1000]:
            nb, first = _plan(lib, mx, my, nbands)
            assert 1 <= nb <= min(64, nty)
            if nbands:
                assert nb == min(nbands, nty, 64)
            assert first[0] == 0 and first[-1] == nty
            assert all(b > a for a, b in zip(first, first[1:]))      # every band holds a tile row
    # the automatic choice: about 28 MB of state per band
    nb, _ = _plan(lib, 4096, 4096, 0)
    assert nb == int(40 * 4096 * 4096 / 28e6) + 1 == 24
    assert _plan(lib, 64, 64, 0)[0] == 1
    assert lib.dclaw_step_host_bands(1, 10, 0, None, 0) == 0


def test_host_step_argument_checks():
    lib = _lib.load()
    assert lib.dclaw_step_host_workspace_bytes(1, 10) == 0
    mx, my = 300, 200
    need = lib.dclaw_step_host_workspace_bytes(mx, my)
    assert need >= lib.dclaw_workspace_bytes(mx, my) * 0 + 2 * 5 * mx * my * 8
    cp = DClawParams().to_c()
    one = ctypes.c_void_p(256)
    # null state, negative band count, too small a workspace: refused before any device work
    assert lib.dclaw_step_host(None, one, one, mx, my, 1.0, 1.0, ctypes.byref(cp), one, one, need, 0, None) == 1
    assert lib.dclaw_step_host(one, one, one, mx, my, 1.0, 1.0, ctypes.byref(cp), one, one, need, -1, None) == 1
    assert lib.dclaw_step_host(one, one, one, mx, my, 0.0, 1.0, ctypes.byref(cp), one, one, need, 0, None) == 1
    assert lib.dclaw_step_host(one, one, one, mx, my, 1.0, 1.0, ctypes.byref(cp), one, one, need - 1, 0,
                               None) == 5
    bad = DClawParams(bed_normal=1).to_c()
    assert lib.dclaw_step_host(one, one, one, mx, my, 1.0, 1.0, ctypes.byref(bad), one, one, need, 0, None) == 2


def _case(n, mx, my, seed):
    c = W.random_field_case(n=n, dx=0.5, seed=seed)
    q = np.ascontiguousarray(c.q[:, :my, :mx])
    b = np.ascontiguousarray(c.b[:my, :mx])
    return c, q, b


@pytest.mark.gpu
@pytest.mark.parametrize("mx,my,nbands,inplace,pinned", [
    (200, 200, 0, True, True),
    (200, 200, 1, False, True),
    (200, 200, 3, True, True),
    (200, 200, 16, False, True),        # one band per tile row (13-row tiles)
    (200, 200, 500, True, False),       # capped at the tile rows; pageable memory
    (173, 131, 4, False, True),         # ragged: last tile row partial (131 = 10 x 13 + 1)
    (96, 190, 5, True, True),
])
def test_host_step_matches_device_step(cuda_device, mx, my, nbands, inplace, pinned):
    from dclaw_b200.solver import PatchStepper

    dev = cuda_device
    c, qn, bn = _case(200, mx, my, 31)
    q0 = torch.tensor(qn, device=dev)
    b = torch.tensor(bn, device=dev)
    ref = PatchStepper(q0, b, c.params, c.dx, c.dy)
    ref.init_clock(c.dt_initial)
    hst = PatchStepper(q0, b, c.params, c.dx, c.dy)
    hst.init_clock(c.dt_initial)
    qh = torch.tensor(qn)
    if pinned:
        qh = qh.pin_memory()
    out = qh if inplace else (torch.empty_like(qh).pin_memory() if pinned else torch.empty_like(qh))
    nsteps = 6
    for _ in range(nsteps):
        ref.step(1)
        hst.step_host(qh, out, nbands=nbands)
        if not inplace:
            qh, out = out, qh
    torch.cuda.synchronize()
    got = qh
    assert torch.equal(got, ref.state().cpu()), "host-buffer step differs from dclaw_step"
    assert torch.equal(hst.clock.cpu(), ref.clock.cpu())
    assert ref.status() == 0 and hst.status() == 0
    # the state moved and has wet and dry cells
    assert not torch.equal(got, torch.tensor(qn))
    assert bool((got[0] > 0).any()) and bool((got[0] == 0).any())


@pytest.mark.gpu
def test_host_step_walls_and_open_boundaries_band_edges(cuda_device):
    """Open (extrapolation) boundaries and a flow front crossing the band
    edges: a dam-break strip along y so that every band is wet."""
    from dclaw_b200.solver import PatchStepper

    dev = cuda_device
    mx, my = 64, 300
    p = DClawParams().replace(bc_lower=(1, 1), bc_upper=(1, 1))
    h = np.zeros((my, mx))
    h[:, : mx // 2] = 1.0
    m = np.full((my, mx), 0.62)
    qn = W.state_from(h, m, p)
    bn = np.zeros((my, mx))
    q0 = torch.tensor(qn, device=dev)
    b = torch.tensor(bn, device=dev)
    ref = PatchStepper(q0, b, p, 0.1, 0.1)
    ref.init_clock(0.002)
    hst = PatchStepper(q0, b, p, 0.1, 0.1)
    hst.init_clock(0.002)
    qh = torch.tensor(qn).pin_memory()
    for _ in range(8):
        ref.step(1)
        hst.step_host(qh, nbands=7)
    torch.cuda.synchronize()
    assert torch.equal(qh, ref.state().cpu())
    assert torch.equal(hst.clock.cpu(), ref.clock.cpu())
