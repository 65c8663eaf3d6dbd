"""Frame output (fort.q / fort.t), gauges and the moving gate bed: host-side
pieces of the step's interface (valout.f90, the flume tools' gauge rule,
the port's gate_bed)."""
import math

import numpy as np
import pytest
import torch

from dclaw_b200.gauges import Gauges
from dclaw_b200.output import fortran_e, read_frame, write_frame
from dclaw_b200.solver import gate_bed


def test_fortran_e_format():
    assert fortran_e(0.0) == "    0.0000000000000000E+00"
    assert fortran_e(1.0) == "    0.1000000000000000E+01"
    assert fortran_e(-2.5e-3) == "   -0.2500000000000000E-02"
    assert fortran_e(123456.789) == "    0.1234567890000000E+06"
    assert fortran_e(1e-120) == "    0.1000000000000000-119"
    assert len(fortran_e(-1.0 / 3.0)) == 26
    assert fortran_e(3.5, 18, 8) == "    0.35000000E+01"


def test_frame_round_trip(tmp_path):
    rng = np.random.default_rng(0)
    my, mx = 7, 9
    q = rng.standard_normal((5, my, mx))
    q[:, 2, 3] = 1e-95                      # below valout's 1e-90 floor: written as zero
    b = rng.standard_normal((my, mx))
    qp, tp = write_frame(str(tmp_path), 12, 3.25, q, b, 0.5, 0.25, xlower=-1.0, ylower=2.0)
    assert qp.endswith("fort.q0012") and tp.endswith("fort.t0012")
    hdr, arr = read_frame(qp)
    assert hdr == {"grid_number": 1, "AMR_level": 1, "mx": mx, "my": my, "xlow": -1.0, "ylow": 2.0, "dx": 0.5,
                   "dy": 0.25}
    want = q.copy()
    want[:, 2, 3] = 0.0
    assert np.allclose(arr[:5], want, rtol=1e-15, atol=0.0)
    assert np.all(arr[5:7] == 0.0)
    assert np.allclose(arr[7], q[0] + b, rtol=1e-15)
    t = open(tp).read().split()
    assert float(t[0]) == 3.25 and t[2] == "8" and t[4] == "1" and t[10] == "2" and t[12] == "ascii"


def test_gauge_rule():
    mx, my, dx = 6, 5, 2.0
    q = torch.zeros((5, my, mx), dtype=torch.float64)
    q[0] = torch.arange(mx * my, dtype=torch.float64).reshape(my, mx) * 0.1 + 1.0   # all wet, linear in i, j
    q[4] = 7.0
    # a gauge between cell centres (i 1..2, j 2..3): bilinear of a linear field is exact
    g = Gauges([1.5 * dx + 0.3], [2.5 * dx + 0.8], mx, my, dx, dx)
    i, j = (1.5 * dx + 0.3) / dx - 0.5, (2.5 * dx + 0.8) / dx - 0.5
    v = g.read(q)
    assert v.shape == (1, 5)
    assert abs(float(v[0, 0]) - (1.0 + 0.1 * (j * mx + i))) < 1e-14 and float(v[0, 4]) == 7.0
    # one of the four cells dry: the nearest cell's value
    q[0, 2, 1] = 0.0
    v = g.read(q)
    jn, inn = round(j), round(i)
    assert float(v[0, 0]) == float(q[0, jn, inn])
    # gradients flow to the selected cells
    qq = q.clone().requires_grad_(True)
    g.read(qq)[0, 0].backward()
    assert float(qq.grad.abs().sum()) == 1.0


def test_gate_bed_matches_the_port_formula():
    b0 = torch.zeros((4, 3), dtype=torch.float64)
    ridge = torch.ones((4, 3), dtype=torch.float64)
    bed = gate_bed(b0, ridge, [0.0, 0.85], [0.0, 90.0])
    for t, ang in [(-1.0, 0.0), (0.0, 0.0), (0.425, 45.0), (0.85, 90.0), (3.0, 90.0)]:
        assert torch.allclose(bed(torch.tensor(t, dtype=torch.float64)), torch.full((4, 3), math.cos(math.radians(ang)), dtype=torch.float64),
                              atol=1e-15)


@pytest.mark.gpu
def test_rollout_with_gate_bed(cuda_device):
    """rollout with a moving bed equals stepping with the bed rebuilt at the
    start of every step."""
    from dclaw_b200 import workloads as W
    from dclaw_b200.solver import Grid, PatchStepper, rollout, to_dclaw_params

    dev = cuda_device
    c = W.flume_member(12, 80, 0.1, W.DClawParams())
    q0n, bn = c
    q0 = torch.tensor(q0n, device=dev).permute(0, 2, 1).contiguous()      # port layout (5, nx, ny)
    b0 = torch.tensor(bn, device=dev).t().contiguous()
    ridge = torch.zeros_like(b0)
    ridge[45:47, :] = 0.8
    bed = gate_bed(b0, ridge, [0.0, 0.3], [0.0, 90.0])
    grid = Grid(80, 12, 0.1, 0.1)
    p = W.DClawParams()
    qf, t, _, _ = rollout(q0, bed, p, grid, t_final=0.6, cfl=0.5, n_steps=40, keep_states=False)
    prm = to_dclaw_params(p, "wall", "wall", 0.5)
    st = PatchStepper(q0.permute(0, 2, 1).contiguous(), bed(torch.zeros((), dtype=torch.float64, device=dev)).t().contiguous(),
                      prm, 0.1, 0.1)
    from dclaw_b200.solver import cfl_dt
    st.init_clock(float(cfl_dt(q0, prm, grid, 0.5)), t_final=0.6)
    for _ in range(40):
        st.b.copy_(bed(st.clock[0]).t())
        st.step(1)
    assert torch.equal(st.state().permute(0, 2, 1), qf)
