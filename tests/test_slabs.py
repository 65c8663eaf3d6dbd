"""One patch over several GPUs as row slabs (dclaw_b200/slabs.py).

CPU: the slab plan (whole tile rows, every row owned once, halos inside the
patch and aligned so that each slab's own rows start a tile row of its
window), and the halo exchange and Courant-number max over two and three
gloo ranks on CPU tensors.
GPU: all slabs of a patch stepped in one process (LocalSlabs: the same
per-slab calls, halos exchanged by copies) equal the whole-patch step bit
for bit, state and clock, over several steps, for 2-4 slabs, walls and
open boundaries, ragged last tile rows.
"""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from dclaw_b200.slabs import Slab, _halo_counts, exchange_halos, slab_plan

G = 14      # a granule for the plan tests (slab_plan takes any)


def test_slab_plan_covers_rows_with_aligned_halos():
    for my in [14, 28, 100, 131, 200, 4096]:
        nty = -(-my // G)
        for world in range(1, min(nty, 9) + 1):
            plan = slab_plan(my, world, G)
            assert len(plan) == world
            assert plan[0].own_first == 1 and plan[-1].own_last == my
            for k, s in enumerate(plan):
                assert (s.own_first - 1) % G == 0
                assert s.own_last == my or s.own_last % G == 0
                assert s.win_first == max(1, s.own_first - G) and s.win_last == min(my, s.own_last + G)
                assert (s.local_first - 1) % G == 0                  # own rows start a tile row of the window
                if k:
                    assert s.own_first == plan[k - 1].own_last + 1
                lo, hi = _halo_counts(plan, k)
                assert lo == (G if k else 0) and hi == (min(G, my - s.own_last) if k < world - 1 else 0)
            counts = [s.own_count for s in plan]
            assert max(counts) - min(counts) <= G + (my % G and G)
    assert slab_plan(100, 2, G, halo=28)[1].win_first == 57 - 28
    with pytest.raises(ValueError):
        slab_plan(100, 2, G, halo=7)           # not a multiple of the tile rows
    with pytest.raises(ValueError):
        slab_plan(28, 3, G)                     # more slabs than tile rows
    with pytest.raises(ValueError):
        slab_plan(100, 3, G, halo=42)          # slabs thinner than the halo


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _worker(rank, world, port, my, mx, out):
    import datetime

    import torch.distributed as dist

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        plan = slab_plan(my, world, G)
        s = plan[rank]
        # the whole patch as row numbers, each rank holding its window with
        # the halo rows blanked
        full = torch.arange(1, my + 1, dtype=torch.float64)[None, :, None].expand(5, my, mx).clone()
        full += torch.arange(5, dtype=torch.float64)[:, None, None] * 1000.0
        q = full[:, s.win_first - 1:s.win_last, :].clone()
        a = s.local_first - 1
        q[:, :a, :] = -1.0
        q[:, a + s.own_count:, :] = -1.0
        exchange_halos(q, plan, rank, dist)
        ok = bool(torch.equal(q, full[:, s.win_first - 1:s.win_last, :]))
        # the Courant numbers combine as the max of their bit patterns
        cfl = torch.tensor([0.25 + 0.5 * rank], dtype=torch.float64)
        bits = cfl.view(torch.int64).clone()
        dist.all_reduce(bits, op=dist.ReduceOp.MAX)
        out[rank] = (ok, float(bits.view(torch.float64)[0]))
        dist.barrier()
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world,my", [(2, 60), (3, 131)])
def test_halo_exchange_gloo_ranks(world, my):
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, my, 7, out)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(120)
        assert p.exitcode == 0
    for r in range(world):
        ok, cfl = out[r]
        assert ok, f"rank {r} halo rows differ from its neighbours' rows"
        assert cfl == 0.25 + 0.5 * (world - 1)


@pytest.mark.gpu
@pytest.mark.parametrize("n,mx,my,nslabs,bc", [
    (200, 200, 200, 2, "wall"),
    (200, 173, 131, 3, "wall"),      # ragged last tile row
    (200, 96, 190, 4, "open"),
])
def test_local_slabs_equal_the_whole_patch_step(cuda_device, n, mx, my, nslabs, bc):
    from dclaw_b200 import workloads as W
    from dclaw_b200.slabs import LocalSlabs
    from dclaw_b200.solver import PatchStepper

    dev = cuda_device
    c = W.random_field_case(n=n, dx=0.5, seed=41)
    p = c.params if bc == "wall" else c.params.replace(bc_lower=(1, 1), bc_upper=(1, 1))
    q0 = torch.tensor(np.ascontiguousarray(c.q[:, :my, :mx]), device=dev)
    b = torch.tensor(np.ascontiguousarray(c.b[:my, :mx]), device=dev)
    ref = PatchStepper(q0, b, p, c.dx, c.dy)
    ref.init_clock(c.dt_initial)
    sl = LocalSlabs(q0, b, p, c.dx, c.dy, nslabs)
    sl.init_clock(c.dt_initial)
    for _ in range(8):
        ref.step(1)
        sl.step(1)
    torch.cuda.synchronize()
    assert torch.equal(sl.state(), ref.state()), "slabs differ from the whole-patch step"
    for s in sl.slabs:
        assert torch.equal(s.st.clock, ref.clock)
    assert not torch.equal(ref.state(), q0)


def test_step_rows_argument_checks():
    """dclaw_step_rows takes whole tile rows only and refuses bad ranges,
    sizes and workspaces on the host, before any device work."""
    import ctypes

    from dclaw_b200 import _lib
    from dclaw_b200.params import DClawParams

    lib = _lib.load()
    g = lib.dclaw_rows_granule()      # cells per tile row of the fused step
    assert 4 <= g <= 50
    mx, my = 50, 100
    need = lib.dclaw_workspace_bytes(mx, my)
    cp = DClawParams().to_c()
    one, two = ctypes.c_void_p(256), ctypes.c_void_p(512)

    def call(first, count, work=need, q_out=two):
        return lib.dclaw_step_rows(one, q_out, one, mx, my, 1.0, 1.0, ctypes.byref(cp), one, one, work, first,
                                   count, None)

    assert call(2, g) == 1            # does not start a tile row
    assert call(1, g - 1) == 1        # does not end on one (and not at the last row)
    assert call(0, g) == 1
    assert call(99, g) == 1           # beyond the patch
    assert call(1, 0) == 1
    assert call(g + 1, 2 * g, q_out=one) == 1   # in place
    assert call(g + 1, 2 * g, work=1024) == 5
    assert lib.dclaw_clock_tick(None, ctypes.byref(cp), None) == 1


@pytest.mark.gpu
def test_dist_slabs_single_rank_equals_the_whole_patch_step(cuda_device):
    """DistSlabs with no process group is one slab holding the whole patch:
    its per-step calls (own rows, Courant bits, tick) equal dclaw_step."""
    from dclaw_b200 import workloads as W
    from dclaw_b200.slabs import DistSlabs
    from dclaw_b200.solver import PatchStepper

    dev = cuda_device
    c = W.random_field_case(n=120, dx=0.5, seed=43)
    q0 = torch.tensor(c.q, device=dev)
    b = torch.tensor(c.b, device=dev)
    ref = PatchStepper(q0, b, c.params, c.dx, c.dy)
    ref.init_clock(c.dt_initial)
    sl = DistSlabs(q0, b, c.params, c.dx, c.dy)
    assert (sl.rank, sl.world) == (0, 1)
    sl.init_clock(c.dt_initial)
    ref.step(6)
    sl.step(6)
    torch.cuda.synchronize()
    assert torch.equal(sl.own(), ref.state())
    assert torch.equal(sl.slab.st.clock, ref.clock)
