"""Clawpack ASCII frame output (fort.qXXXX / fort.tXXXX) of a uniform patch.

The reference writes frames with valout (src/2d/dig/valout.f90:10): for
output_format 1 a fort.q file holds, per grid, a header
(valout.f90:74-82) and then, row by row (j outer, i inner), every conserved
field followed by the surface elevation eta = h + b - bdif, in Fortran
E26.16, with a blank line after each row and values below 1e-90 in
magnitude written as zero (valout.f90:177-205). fort.t holds the time and
the counts (valout.f90:83-89,484-485). The fused step keeps 5 of D-Claw's
7 fields; h*chi and the bed change are identically zero for the accepted
options and are written as zeros, so Clawpack's readers see the reference's
layout (meqn 7 + eta).
"""
from __future__ import annotations

import os

import numpy as np

MEQN = 7          # h, hu, hv, hm, pb, hchi, bdif
NGHOST = 2


def fortran_e(v: float, w: int = 26, d: int = 16) -> str:
    """Fortran Ew.d edit descriptor: 0.ddd...E+xx, right-justified to w."""
    v = float(v)
    if v != v or v in (float("inf"), float("-inf")):
        return ("NaN" if v != v else ("Infinity" if v > 0 else "-Infinity")).rjust(w)
    if v == 0.0:
        body = "0." + "0" * d + "E+00"
        return body.rjust(w)
    s = f"{abs(v):.{d - 1}e}"                # d significant digits, d.ddd e+xx
    mant, ex = s.split("e")
    digits = mant.replace(".", "")
    e = int(ex) + 1
    expo = f"E{'+' if e >= 0 else '-'}{abs(e):02d}" if abs(e) < 100 else f"{'+' if e >= 0 else '-'}{abs(e):03d}"
    body = ("-" if v < 0 else "") + "0." + digits + expo
    return body.rjust(w)


def write_frame(outdir: str, frame: int, t: float, q: np.ndarray, b: np.ndarray, dx: float, dy: float,
                xlower: float = 0.0, ylower: float = 0.0, naux: int = 10) -> tuple[str, str]:
    """Write fort.qNNNN and fort.tNNNN for one patch. q: (5, my, mx) state
    (h, hu, hv, hm, pb), b: (my, mx) bed; returns the two paths."""
    q = np.asarray(q, dtype=np.float64)
    b = np.asarray(b, dtype=np.float64)
    _, my, mx = q.shape
    os.makedirs(outdir, exist_ok=True)
    qpath = os.path.join(outdir, f"fort.q{frame:04d}")
    tpath = os.path.join(outdir, f"fort.t{frame:04d}")
    lines = [f"{1:6d}                 grid_number", f"{1:6d}                 AMR_level",
             f"{mx:6d}                 mx", f"{my:6d}                 my",
             f"{fortran_e(xlower)}    xlow", f"{fortran_e(ylower)}    ylow",
             f"{fortran_e(dx)}    dx", f"{fortran_e(dy)}    dy", ""]
    zero = np.zeros((my, mx))
    fields = [q[0], q[1], q[2], q[3], q[4], zero, zero]          # + hchi, bdif
    fields = [np.where(np.abs(f) < 1.0e-90, 0.0, f) for f in fields]
    eta = q[0] + b - 0.0
    eta = np.where(np.abs(eta) < 1.0e-99, 0.0, eta)
    for j in range(my):
        for i in range(mx):
            lines.append("".join(fortran_e(f[j, i]) for f in fields) + fortran_e(eta[j, i]))
        lines.append(" ")
    with open(qpath, "w") as fh:
        fh.write("\n".join(lines) + "\n")
    with open(tpath, "w") as fh:
        fh.write(f"{fortran_e(t, 18, 8)}    time\n{MEQN + 1:6d}                 meqn\n"
                 f"{1:6d}                 ngrids\n{naux:6d}                 naux\n{2:6d}                 ndim\n"
                 f"{NGHOST:6d}                 nghost\n{'ascii':>10s}             format\n\n")
    return qpath, tpath


def read_frame(qpath: str):
    """Parse a single-grid fort.q file back to (header dict, (8, my, mx) array)."""
    with open(qpath) as fh:
        lines = fh.read().splitlines()
    hdr = {}
    keys = ["grid_number", "AMR_level", "mx", "my", "xlow", "ylow", "dx", "dy"]
    for k, line in zip(keys, lines[:8]):
        v = line.split()[0]
        hdr[k] = int(v) if k in ("grid_number", "AMR_level", "mx", "my") else float(v.replace("D", "E"))
    vals = [list(map(float, ln.split())) for ln in lines[9:] if ln.strip()]
    arr = np.array(vals).reshape(hdr["my"], hdr["mx"], -1).transpose(2, 0, 1)
    return hdr, arr
