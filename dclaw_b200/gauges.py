"""Gauges: state values at fixed points of a uniform patch.

The reference's flume tools read a gauge by linear interpolation between
the cell centres around it when those cells are wet (h > 1e-3), and from
the nearer cell otherwise (gradient_particle_filter/flume_solver.py:84-99,
pf_flume/flume_model.py:114-121,144-148, following GeoClaw's gauges
module). On a 2D patch the same rule is bilinear: the four cell centres
around the gauge when all four are wet, else the nearest cell.

`Gauges.select` gives the flat indices of those cells in a (5, my, mx)
state, so a differentiable rollout can return only them
(`rollout_states(..., select=g.select)`); `Gauges.values` turns the
selected entries into gauge values with torch operations, so a loss on
gauge values differentiates back through the rollout.
"""
from __future__ import annotations

import numpy as np
import torch

WET = 1.0e-3


class Gauges:
    def __init__(self, x, y, mx: int, my: int, dx: float, dy: float, xlower: float = 0.0, ylower: float = 0.0,
                 device=None):
        x = np.atleast_1d(np.asarray(x, dtype=np.float64))
        y = np.atleast_1d(np.asarray(y, dtype=np.float64))
        # cell-centre coordinates in cell units: centre of cell i at i + 0.5
        fx = (x - xlower) / dx - 0.5
        fy = (y - ylower) / dy - 0.5
        i0 = np.clip(np.floor(fx).astype(np.int64), 0, mx - 2)
        j0 = np.clip(np.floor(fy).astype(np.int64), 0, my - 2)
        wx = np.clip(fx - i0, 0.0, 1.0)
        wy = np.clip(fy - j0, 0.0, 1.0)
        inear = np.where(wx >= 0.5, i0 + 1, i0)
        jnear = np.where(wy >= 0.5, j0 + 1, j0)
        self.n = len(x)
        self.mx, self.my = mx, my
        plane = mx * my
        # per gauge: 4 corners (j0 i0, j0 i0+1, j0+1 i0, j0+1 i0+1) + nearest, x 5 fields
        cells = np.stack([j0 * mx + i0, j0 * mx + i0 + 1, (j0 + 1) * mx + i0, (j0 + 1) * mx + i0 + 1,
                          jnear * mx + inear], axis=1)                                     # (n, 5)
        sel = cells[:, :, None] + plane * np.arange(5)[None, None, :]                      # (n, 5, 5)
        self.select = torch.tensor(sel.reshape(-1), device=device)
        w = np.stack([(1 - wx) * (1 - wy), wx * (1 - wy), (1 - wx) * wy, wx * wy], axis=1)
        self.w = torch.tensor(w, device=device)

    def values(self, selected: torch.Tensor) -> torch.Tensor:
        """Gauge values (..., n, 5) of (h, hu, hv, hm, pb) from entries picked
        with `select` (trailing dimension n * 25)."""
        v = selected.reshape(selected.shape[:-1] + (self.n, 5, 5))    # (..., gauge, cell, field)
        corners, near = v[..., :4, :], v[..., 4, :]
        wet = (corners[..., 0] > WET).all(dim=-1, keepdim=True)
        interp = (self.w.to(v.dtype)[..., None] * corners).sum(dim=-2)
        return torch.where(wet, interp, near)

    def read(self, q: torch.Tensor) -> torch.Tensor:
        """Gauge values (n, 5) of a (5, my, mx) state."""
        return self.values(q.reshape(-1)[self.select.to(q.device)])
