"""step2-style patch calls on torch tensors (padded layout, mbc = 2).

Mirrors the Fortran patch interface that GeoClaw's stepgrid drives:
  bc2amr(q)                                  -- ghost cells (GeoClaw bc2amr)
  setaux(aux)                                -- ghost bed, D-Claw aux defaults (setaux.f90)
  b4step2(q, aux, dx, dy, t, dt)             -- src/2d/dig/b4step2.f90:7
  step2(q, aux, dx, dy, dt) -> cflgrid       -- GeoClaw step2 + stepgrid update
  src2(q, aux, dx, dy, t, dt)                -- src/2d/dig/src2.f90:27
q is (5, my+4, mx+4) (h, hu, hv, hm, pb), aux is (6, my+4, mx+4)
(b, phi, theta, fsphi, taudir_x, taudir_y); both are modified in place like
the Fortran arrays. Argument meaning and order follow the Fortran routines
(t is accepted and unused, as in the reference for these routines).
"""
from __future__ import annotations

import ctypes

import torch

from . import _lib
from .params import CLOCK_DOUBLES, CClock, DClawParams

MBC = 2


class Patch:
    """Holds the parameters, a device clock and the step2 workspace of one patch."""

    def __init__(self, params: DClawParams, mx: int, my: int, device="cuda"):
        self.lib = _lib.load()
        self.params = params
        self.cp = params.to_c()
        _lib.check(self.lib.dclaw_params_check_5(ctypes.byref(self.cp)), "parameter check")
        self.mx, self.my = int(mx), int(my)
        self.work_bytes = self.lib.dclaw_workspace_bytes(self.mx, self.my)
        self.work = torch.empty(self.work_bytes, dtype=torch.uint8, device=device)
        self.clock = torch.zeros(CLOCK_DOUBLES, dtype=torch.float64, device=device)

    def _shape_check(self, t: torch.Tensor, nf: int, name: str) -> None:
        if tuple(t.shape) != (nf, self.my + 2 * MBC, self.mx + 2 * MBC) or not t.is_contiguous():
            raise _lib.DClawError(f"{name} must be a contiguous ({nf}, my+4, mx+4) tensor")
        if not t.is_cuda or t.dtype != torch.float64:
            raise _lib.DClawError(f"{name} must be a float64 CUDA tensor")

    def bc2amr(self, q: torch.Tensor) -> None:
        self._shape_check(q, 5, "q")
        _lib.check(self.lib.dclaw_bc2amr(_lib.ptr(q), self.mx, self.my, MBC, ctypes.byref(self.cp),
                                         _lib.stream_ptr()), "bc2amr")

    def setaux(self, aux: torch.Tensor) -> None:
        self._shape_check(aux, 6, "aux")
        _lib.check(self.lib.dclaw_setaux(_lib.ptr(aux), self.mx, self.my, MBC, ctypes.byref(self.cp),
                                         _lib.stream_ptr()), "setaux")

    def b4step2(self, q: torch.Tensor, aux: torch.Tensor, dx: float, dy: float, t: float = 0.0,
                dt: float = 0.0) -> None:
        self._shape_check(q, 5, "q")
        self._shape_check(aux, 6, "aux")
        _lib.check(self.lib.dclaw_b4step2(_lib.ptr(q), _lib.ptr(aux), self.mx, self.my, MBC, dx, dy, t, dt,
                                          ctypes.byref(self.cp), _lib.ptr(self.clock), _lib.stream_ptr()),
                   "b4step2")

    def step2(self, q: torch.Tensor, aux: torch.Tensor, dx: float, dy: float, dt: float,
              fluxes: torch.Tensor | None = None) -> float:
        """Flux sweeps and the conservative update; returns cflgrid."""
        self._shape_check(q, 5, "q")
        self._shape_check(aux, 6, "aux")
        if fluxes is not None:
            self._shape_check(fluxes, 20, "fluxes")
        _lib.check(self.lib.dclaw_step2(_lib.ptr(q), _lib.ptr(aux), self.mx, self.my, MBC, dx, dy, dt,
                                        ctypes.byref(self.cp), _lib.ptr(self.clock), _lib.ptr(fluxes),
                                        _lib.ptr(self.work), self.work_bytes, _lib.stream_ptr()), "step2")
        return float(self.clock[2].item())

    def src2(self, q: torch.Tensor, aux: torch.Tensor, dx: float, dy: float, t: float, dt: float) -> None:
        self._shape_check(q, 5, "q")
        _lib.check(self.lib.dclaw_src2(_lib.ptr(q), _lib.ptr(aux), self.mx, self.my, MBC, dx, dy, t, dt,
                                       ctypes.byref(self.cp), _lib.stream_ptr()), "src2")

    def from_fortran(self, a: torch.Tensor, nf: int) -> torch.Tensor:
        """The first nf fields of a Fortran patch array a(nf_fortran,
        1-mbc:mx+mbc, 1-mbc:my+mbc) -- here a contiguous float64 CUDA tensor
        of shape (my+4, mx+4, nf_fortran), the same memory -- as the padded
        (nf, my+4, mx+4) planes the patch calls take (q: nf 5 of meqn 7;
        aux: nf 6 of maux)."""
        my, mx = self.my + 2 * MBC, self.mx + 2 * MBC
        if a.dim() != 3 or tuple(a.shape[:2]) != (my, mx) or not a.is_contiguous() or a.dtype != torch.float64:
            raise _lib.DClawError("a must be a contiguous float64 (my+4, mx+4, nf_fortran) tensor")
        out = torch.empty((nf, my, mx), dtype=torch.float64, device=a.device)
        _lib.check(self.lib.dclaw_fields_from_fortran(_lib.ptr(a), int(a.shape[2]), int(nf), self.mx, self.my, MBC,
                                                      _lib.ptr(out), _lib.stream_ptr()), "fields from Fortran layout")
        return out

    def to_fortran(self, planes: torch.Tensor, a: torch.Tensor) -> None:
        """Write the padded planes back into fields 1..nf of the Fortran patch
        array a (shape (my+4, mx+4, nf_fortran)); its other fields are kept."""
        nf = int(planes.shape[0])
        self._shape_check(planes, nf, "planes")
        my, mx = self.my + 2 * MBC, self.mx + 2 * MBC
        if a.dim() != 3 or tuple(a.shape[:2]) != (my, mx) or not a.is_contiguous() or a.dtype != torch.float64:
            raise _lib.DClawError("a must be a contiguous float64 (my+4, mx+4, nf_fortran) tensor")
        _lib.check(self.lib.dclaw_fields_to_fortran(_lib.ptr(planes), nf, int(a.shape[2]), self.mx, self.my, MBC,
                                                    _lib.ptr(a), _lib.stream_ptr()), "fields to Fortran layout")

    def status(self) -> int:
        return CClock.from_buffer_copy(self.clock.cpu().numpy().tobytes()).status
