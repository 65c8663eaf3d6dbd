"""Batched ensembles of uniform patches (the particle-filter use).

The reference's particle filters run one D-Claw-style simulation per
particle, each with its own material parameters, batched with jax.vmap
(gradient_particle_filter/pf_flume/flume_model.py:129-179,
pf_flume/inference.py:96-108). `EnsembleStepper` advances an ensemble of
patches of uneven sizes, each with its own parameters and its own adaptive
dt, with one set of three persistent-kernel launches per ensemble step
(`dclaw_step_batched`), optionally replayed from a captured CUDA graph. The
tile shape and the persistent grid are chosen by `autotune()`, which times
the candidates on the ensemble itself (all candidates give the same bits).
"""
from __future__ import annotations

import ctypes
import dataclasses
import json
import time

import numpy as np
import torch

from . import _lib
from .params import CBatch, CClock, CLOCK_DOUBLES, CMember, CParams, DClawParams


@dataclasses.dataclass
class Member:
    q: np.ndarray        # (5, my, mx) float64
    b: np.ndarray        # (my, mx)
    params: DClawParams
    dx: float
    dy: float
    dt_initial: float
    t_final: float = 0.0
    t_obs: float = 0.0   # observation interval every dt is clipped at (tick rule); 0: off


def clock_array(dts, t_finals, fixed_dt: bool = False, t_obs=None) -> np.ndarray:
    """Host image of n initialised clocks (t = 0) as float64 words. t_obs
    (per member, 0: off): the observation interval every dt is also clipped
    at (with the tick rule), as the device clock's tick does."""
    n = len(dts)
    arr = (CClock * n)()
    for k in range(n):
        dt, tf = float(dts[k]), float(t_finals[k])
        to = float(t_obs[k]) if t_obs is not None else 0.0
        if not fixed_dt and to > 0.0:
            dt = min(dt, (np.floor(0.0 / to + 1.0e-9) + 1.0) * to - 0.0)
        arr[k].t = 0.0
        arr[k].t_final = tf
        arr[k].dt = max(min(dt, tf), 0.0) if tf > 0.0 else dt
        arr[k].fixed_dt = int(fixed_dt)
        arr[k].t_obs = to
    return np.frombuffer(bytes(arr), dtype=np.float64).copy()


class EnsembleStepper:
    """All members on one device, advanced together."""

    def __init__(self, members: list[Member], device="cuda", tile_shape: int = 0, fixed_dt: bool = False):
        self.lib = _lib.load()
        self.members = members
        self.n = len(members)
        self.device = torch.device(device)
        for m in members:
            _lib.check(self.lib.dclaw_params_check_5(ctypes.byref(m.params.to_c())), "member parameters")
        self.mx = np.array([m.q.shape[2] for m in members], dtype=np.int32)
        self.my = np.array([m.q.shape[1] for m in members], dtype=np.int32)
        self.dxs = np.array([m.dx for m in members], dtype=np.float64)
        self.dys = np.array([m.dy for m in members], dtype=np.float64)
        self.fixed_dt = fixed_dt
        self._layout(tile_shape)
        # arenas
        # zeroed: the alignment gaps between members are never written
        self.qa = torch.zeros(self.batch.q_doubles, dtype=torch.float64, device=self.device)
        self.qb = torch.zeros_like(self.qa)
        self.bed = torch.zeros(self.batch.b_doubles, dtype=torch.float64, device=self.device)
        for k, m in enumerate(members):
            o, c = self.cm[k].q_off, int(self.mx[k]) * int(self.my[k])
            self.qa[o:o + 5 * c].copy_(torch.from_numpy(np.ascontiguousarray(m.q, dtype=np.float64).ravel()))
            ob = self.cm[k].b_off
            self.bed[ob:ob + c].copy_(torch.from_numpy(np.ascontiguousarray(m.b, dtype=np.float64).ravel()))
        params = (CParams * self.n)(*[m.params.to_c() for m in members])
        self.params = torch.frombuffer(bytearray(bytes(params)), dtype=torch.uint8).to(self.device)
        self.clocks = torch.tensor(clock_array([m.dt_initial for m in members], [m.t_final for m in members],
                                               fixed_dt, [getattr(m, "t_obs", 0.0) for m in members]),
                                   device=self.device)
        self.graph = None

    def _layout(self, tile_shape: int) -> None:
        self.cm = (CMember * self.n)()
        self.batch = CBatch()
        _lib.check(self.lib.dclaw_batch_layout(self.n, self.mx.ctypes.data, self.my.ctypes.data, self.dxs.ctypes.data,
                                               self.dys.ctypes.data, int(tile_shape), self.cm,
                                               ctypes.byref(self.batch)), "batch layout")
        self.members_dev = torch.frombuffer(bytearray(bytes(self.cm)), dtype=torch.uint8).to(self.device)
        self.work = torch.empty(self.batch.work_bytes, dtype=torch.uint8, device=self.device)
        _lib.check(self.lib.dclaw_batch_reset(ctypes.byref(self.batch), _lib.ptr(self.work), _lib.stream_ptr()),
                   "batch reset")
        self.graph = None

    # ---- stepping ------------------------------------------------------------
    def _launch(self, src, dst) -> None:
        rc = self.lib.dclaw_step_batched(ctypes.byref(self.batch), _lib.ptr(self.members_dev), _lib.ptr(self.params),
                                         _lib.ptr(self.clocks), _lib.ptr(src), _lib.ptr(dst), _lib.ptr(self.bed),
                                         _lib.ptr(self.work), _lib.stream_ptr())
        _lib.check(rc, "dclaw_step_batched")

    def step(self, nsteps: int = 1) -> None:
        for _ in range(nsteps):
            self._launch(self.qa, self.qb)
            self.qa, self.qb = self.qb, self.qa

    def capture(self, nsteps: int) -> None:
        """Capture nsteps (even) ensemble steps into one CUDA graph."""
        if nsteps % 2:
            raise ValueError("graph length must be even (arenas ping-pong)")
        s = torch.cuda.Stream()
        s.wait_stream(torch.cuda.current_stream())
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            with torch.cuda.graph(g, stream=s):
                for _ in range(nsteps // 2):
                    self._launch(self.qa, self.qb)
                    self._launch(self.qb, self.qa)
        torch.cuda.current_stream().wait_stream(s)
        self.graph = g

    def replay(self, times: int = 1) -> None:
        for _ in range(times):
            self.graph.replay()

    # ---- results -------------------------------------------------------------
    def state(self, k: int) -> torch.Tensor:
        o, mx, my = self.cm[k].q_off, int(self.mx[k]), int(self.my[k])
        return self.qa[o:o + 5 * mx * my].view(5, my, mx)

    def read_clocks(self) -> list[CClock]:
        raw = self.clocks.cpu().numpy().tobytes()
        return list((CClock * self.n).from_buffer_copy(raw))

    def status(self) -> list[int]:
        return [c.status for c in self.read_clocks()]

    def cells(self) -> int:
        return int((self.mx.astype(np.int64) * self.my).sum())

    # ---- autotuning ----------------------------------------------------------
    def autotune(self, steps: int = 2, cache: str | None = None) -> dict:
        """Time every compiled tile shape x persistent grid on this ensemble
        (work copies of the current state) and keep the fastest. Results
        are identical for every candidate."""
        key = json.dumps({"gpu": torch.cuda.get_device_name(self.device), "mx": self.mx.tolist(),
                          "my": self.my.tolist()})
        if cache:
            try:
                table = json.load(open(cache))
            except (OSError, ValueError):
                table = {}
            if key in table:
                best = table[key]
                self._layout(best["tile_shape"])
                self.batch.tile_ctas_per_sm = best["tile_ctas_per_sm"]
                return best
        nshape = self.lib.dclaw_batch_tile_shapes(None, None, 16)
        q0, clk0 = self.qa.clone(), self.clocks.clone()
        results = []
        for shape in range(nshape):
            self._layout(shape)
            for cps in (2, 1):
                self.batch.tile_ctas_per_sm = cps
                self.qa.copy_(q0)
                self.clocks.copy_(clk0)
                self.step(1)
                torch.cuda.synchronize()
                e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                e0.record()
                self.step(steps)
                e1.record()
                torch.cuda.synchronize()
                results.append({"tile_shape": shape, "tile_ctas_per_sm": cps, "ms": e0.elapsed_time(e1) / steps})
        best = min(results, key=lambda r: r["ms"])
        self._layout(best["tile_shape"])
        self.batch.tile_ctas_per_sm = best["tile_ctas_per_sm"]
        self.qa.copy_(q0)
        self.clocks.copy_(clk0)
        best = dict(best, candidates=results)
        if cache:
            try:
                table = json.load(open(cache))
            except (OSError, ValueError):
                table = {}
            table[key] = {k: best[k] for k in ("tile_shape", "tile_ctas_per_sm", "ms")}
            json.dump(table, open(cache, "w"))
        return best
