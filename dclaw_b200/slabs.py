"""One patch over several GPUs: row slabs with one halo exchange per step.

The reference advances the patches of a level one per OpenMP thread, and
GeoClaw's advanc (called from tick.f:333) takes the largest cflgrid of the
level's patches for the level's next dt. Here one patch too large for one
GPU is split into slabs of whole tile rows, one per GPU, and their Courant
numbers combine the same way:

* every rank holds its own rows and a halo of `halo` rows on each side that
  lies inside the patch (the rows its neighbours own), as a patch of its own
  whose edges at the patch's edges keep the boundary conditions;
* per step: the halo rows are exchanged with the neighbours (NCCL
  send/recv), the rank steps its own rows (`dclaw_step_rows`: the records of
  the rows its tiles read, which the halo covers, its tiles, its cells'
  src2), the Courant numbers are max-reduced over the ranks (the
  order-preserving bit pattern of a non-negative double, an integer max),
  and every rank applies the tick rule (`dclaw_clock_tick`).

One step reads at most 4 rows away (a record reads its neighbours' depths,
a tile reads records 3 rows beyond it), so a halo of one tile row (13
rows) is exact: every rank's rows and dt equal the whole-patch step's, bit
for bit. A slab's halo rows go stale during its step and are refreshed by
the next exchange.

`DistSlabs` runs one slab per process over torch.distributed; `LocalSlabs`
runs all slabs of a patch in one process on one device, exchanging by
copies, with the same per-slab calls (for tests on one GPU: the slabs run
one after another and never wait on each other).
"""
from __future__ import annotations

import ctypes
import dataclasses

import torch

from . import _lib
from .params import DClawParams

CFL_BITS = 5          # int64 index of dclaw_clock.cfl_bits in the clock tensor


@dataclasses.dataclass(frozen=True)
class Slab:
    own_first: int    # 1-based patch rows the slab steps
    own_last: int
    win_first: int    # patch rows it holds (own rows + halo)
    win_last: int

    @property
    def rows(self) -> int:
        return self.win_last - self.win_first + 1

    @property
    def local_first(self) -> int:
        """First own row in the slab's own (window) numbering, 1-based."""
        return self.own_first - self.win_first + 1

    @property
    def own_count(self) -> int:
        return self.own_last - self.own_first + 1


def slab_plan(my: int, world: int, granule: int, halo: int | None = None) -> list[Slab]:
    """Split rows 1..my into `world` slabs of whole tile rows (granule rows
    each, the last possibly partial), balanced by tile rows, with `halo`
    rows (default one tile row; a multiple of the granule, at least 4) on
    each side inside the patch."""
    halo = granule if halo is None else int(halo)
    if halo < 4 or halo % granule:
        raise ValueError(f"halo must be a multiple of {granule} and at least 4")
    nty = -(-my // granule)
    if not 1 <= world <= nty:
        raise ValueError(f"{world} slabs for {nty} tile rows")
    if world > 1 and min((k + 1) * nty // world - k * nty // world for k in range(world)) * granule < halo:
        raise ValueError("a slab thinner than the halo")
    plan = []
    for k in range(world):
        t0, t1 = k * nty // world, (k + 1) * nty // world
        a, b = t0 * granule + 1, min(my, t1 * granule)
        plan.append(Slab(a, b, max(1, a - halo), min(my, b + halo)))
    return plan


def window(global_rows: torch.Tensor, slab: Slab) -> torch.Tensor:
    """The slab's rows of a (..., my, mx) array (a contiguous copy)."""
    return global_rows[..., slab.win_first - 1:slab.win_last, :].contiguous()


class SlabStep:
    """One slab's state, bed, clock and workspace, and its per-step calls.

    q_win: (5, rows, mx) float64 CUDA tensor of the slab's window rows,
    b_win: (rows, mx)."""

    def __init__(self, q_win: torch.Tensor, b_win: torch.Tensor, params: DClawParams, dx: float, dy: float,
                 slab: Slab):
        from .solver import PatchStepper

        self.slab = slab
        self.st = PatchStepper(q_win, b_win, params, dx, dy)
        if self.st.my != slab.rows:
            raise ValueError(f"window of {self.st.my} rows for a slab of {slab.rows}")

    @property
    def q(self) -> torch.Tensor:
        return self.st.qa

    def init_clock(self, dt: float, t: float = 0.0, t_final: float = 0.0, fixed_dt: bool = False) -> None:
        self.st.init_clock(dt, t=t, t_final=t_final, fixed_dt=fixed_dt)

    def cfl_bits(self) -> torch.Tensor:
        return self.st.clock.view(torch.int64)[CFL_BITS:CFL_BITS + 1]

    def compute(self) -> None:
        """Step the own rows (halo rows of the state must be current)."""
        st, s = self.st, self.slab
        rc = st.lib.dclaw_step_rows(_lib.ptr(st.qa), _lib.ptr(st.qb), _lib.ptr(st.b), st.mx, st.my, st.dx, st.dy,
                                    ctypes.byref(st.cp), _lib.ptr(st.clock), _lib.ptr(st.work), st.work_bytes,
                                    s.local_first, s.own_count, _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_rows")

    def finish(self) -> None:
        """After the Courant numbers are combined: tick, and swap buffers."""
        st = self.st
        _lib.check(st.lib.dclaw_clock_tick(_lib.ptr(st.clock), ctypes.byref(st.cp), _lib.stream_ptr()),
                   "dclaw_clock_tick")
        st.qa, st.qb = st.qb, st.qa

    def own(self) -> torch.Tensor:
        """The slab's own rows of the current state, (5, own_count, mx)."""
        a = self.slab.local_first - 1
        return self.st.qa[:, a:a + self.slab.own_count, :]


def _halo_counts(plan: list[Slab], k: int) -> tuple[int, int]:
    """Rows slab k receives from below and from above."""
    s = plan[k]
    return s.own_first - s.win_first, s.win_last - s.own_last


class LocalSlabs:
    """All slabs of one patch in one process on one device (exchange by copies)."""

    def __init__(self, q: torch.Tensor, b: torch.Tensor, params: DClawParams, dx: float, dy: float, nslabs: int,
                 halo: int | None = None):
        lib = _lib.load()
        my = q.shape[1]
        self.plan = slab_plan(my, nslabs, lib.dclaw_rows_granule(), halo)
        self.slabs = [SlabStep(window(q, s), window(b, s), params, dx, dy, s) for s in self.plan]

    def init_clock(self, dt: float, **kw) -> None:
        for s in self.slabs:
            s.init_clock(dt, **kw)

    def exchange(self) -> None:
        for k, sk in enumerate(self.slabs):
            lo, hi = _halo_counts(self.plan, k)
            if lo:
                src = self.slabs[k - 1]
                a = src.slab.local_first + src.slab.own_count - 1 - lo          # src's last lo own rows
                sk.q[:, :lo, :].copy_(src.q[:, a:a + lo, :])
            if hi:
                src = self.slabs[k + 1]
                a = src.slab.local_first - 1                                    # src's first hi own rows
                sk.q[:, sk.slab.rows - hi:, :].copy_(src.q[:, a:a + hi, :])

    def step(self, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            self.exchange()
            for s in self.slabs:
                s.compute()
            bits = torch.stack([s.cfl_bits() for s in self.slabs]).max(dim=0).values
            for s in self.slabs:
                s.cfl_bits().copy_(bits)
                s.finish()

    def state(self) -> torch.Tensor:
        return torch.cat([s.own() for s in self.slabs], dim=1)


class DistSlabs:
    """This rank's slab of one patch, the other slabs on the other ranks of
    the default process group (one process per GPU). q and b are the whole
    patch (every rank passes the same arrays; only its window is kept) or
    already the window (window=True)."""

    def __init__(self, q: torch.Tensor, b: torch.Tensor, params: DClawParams, dx: float, dy: float,
                 halo: int | None = None, my: int | None = None, window_given: bool = False):
        import torch.distributed as dist

        self.dist = dist
        grouped = dist.is_available() and dist.is_initialized()
        self.rank, self.world = (dist.get_rank(), dist.get_world_size()) if grouped else (0, 1)
        lib = _lib.load()
        my = q.shape[1] if my is None else my
        self.plan = slab_plan(my, self.world, lib.dclaw_rows_granule(), halo)
        s = self.plan[self.rank]
        qw, bw = (q, b) if window_given else (window(q, s), window(b, s))
        self.slab = SlabStep(qw, bw, params, dx, dy, s)

    def init_clock(self, dt: float, **kw) -> None:
        self.slab.init_clock(dt, **kw)

    def exchange(self) -> None:
        exchange_halos(self.slab.q, self.plan, self.rank, self.dist)

    def step(self, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            if self.world > 1:
                self.exchange()
            self.slab.compute()
            if self.world > 1:
                self.dist.all_reduce(self.slab.cfl_bits(), op=self.dist.ReduceOp.MAX)
            self.slab.finish()

    def own(self) -> torch.Tensor:
        return self.slab.own()


def exchange_halos(q: torch.Tensor, plan: list[Slab], rank: int, dist) -> None:
    """Fill rank's halo rows of its window q (5, rows, mx) from its
    neighbours' own rows, sending its own edge rows to them (one send and
    one receive per neighbour, issued together)."""
    s = plan[rank]
    lo, hi = _halo_counts(plan, rank)
    ops, recv = [], []
    if rank > 0:
        n_up_prev = _halo_counts(plan, rank - 1)[1]        # rows the slab below takes from this one
        a = s.local_first - 1
        ops.append(dist.P2POp(dist.isend, q[:, a:a + n_up_prev, :].contiguous(), rank - 1))
        buf = torch.empty((q.shape[0], lo, q.shape[2]), dtype=q.dtype, device=q.device)
        ops.append(dist.P2POp(dist.irecv, buf, rank - 1))
        recv.append((0, buf))
    if rank < len(plan) - 1:
        n_lo_next = _halo_counts(plan, rank + 1)[0]        # rows the slab above takes from this one
        a = s.local_first - 1 + s.own_count - n_lo_next
        ops.append(dist.P2POp(dist.isend, q[:, a:a + n_lo_next, :].contiguous(), rank + 1))
        buf = torch.empty((q.shape[0], hi, q.shape[2]), dtype=q.dtype, device=q.device)
        ops.append(dist.P2POp(dist.irecv, buf, rank + 1))
        recv.append((s.rows - hi, buf))
    if ops:
        for w in dist.batch_isend_irecv(ops):
            w.wait()
    for at, buf in recv:
        q[:, at:at + buf.shape[1], :].copy_(buf)
