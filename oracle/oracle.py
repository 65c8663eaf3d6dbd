"""TEST INFRASTRUCTURE: ctypes front end of the C++ oracle (dclaw_oracle.cpp).

The oracle is a line-faithful CPU restatement of the reference Fortran
(src/2d/dig/*.f90, *.f); see the header of dclaw_oracle.cpp for the file:line
map and its parity status (pinned by the reference's closed-form KATs only).
Built with g++ -O2 -ffp-contract=off (no FMA contraction, glibc libm) so the
arithmetic matches gfortran -O on x86-64.
"""
from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

from dclaw_b200.params import CParams, DClawParams

HERE = Path(__file__).resolve().parent
SRC = HERE / "dclaw_oracle.cpp"
_LIB = HERE / "liboracle.so"

_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_uint32)


def lib_path() -> Path:
    return _LIB


def build(force: bool = False) -> Path:
    """Compile the oracle into oracle/liboracle.so (g++, OpenMP)."""
    deps = [SRC, HERE.parent / "dclaw_b200" / "csrc" / "elementary.cuh", HERE.parent / "include" / "dclaw_b200.h"]
    if _LIB.exists() and not force and all(_LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return _LIB
    cmd = ["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fopenmp", "-fPIC",
           "-shared", str(SRC), "-o", str(_LIB) + ".tmp"]
    subprocess.run(cmd, check=True)
    os.replace(str(_LIB) + ".tmp", _LIB)
    return _LIB


def _ptr(a: np.ndarray | None, ty=_dp):
    if a is None:
        return None
    return a.ctypes.data_as(ty)


class Oracle:
    """Thin wrapper; arrays are numpy float64 (C order)."""

    def __init__(self):
        build()
        self.lib = ctypes.CDLL(str(_LIB))
        L = self.lib
        L.oracle_run.restype = ctypes.c_int
        L.oracle_run.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                 ctypes.c_double, _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                                 ctypes.c_int, ctypes.c_int, _dp, _dp, _up, _up, _dp, ctypes.c_double]
        L.oracle_run_full.restype = ctypes.c_int
        L.oracle_run_full.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, _dp, _dp, _dp, ctypes.c_int, ctypes.c_double,
                                      ctypes.c_double, ctypes.c_int, ctypes.c_int, _dp, _dp, _up, _up, _dp]
        L.oracle_threads.restype = ctypes.c_int
        L.oracle_threads.argtypes = [ctypes.c_int]
        for name in ("oracle_bc2amr",):
            getattr(L, name).argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, _dp]
        L.oracle_setaux.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.oracle_b4step2.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                     ctypes.c_double, _dp, _dp]
        L.oracle_step2.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                   ctypes.c_double, ctypes.c_double, _dp, _dp, _dp, _dp, ctypes.c_int, _up, _up]
        L.oracle_src2.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_double, _dp, _dp]
        L.oracle_set_libm.restype = ctypes.c_int
        L.oracle_set_libm.argtypes = [ctypes.c_int]
        L.oracle_elementary.restype = ctypes.c_double
        L.oracle_elementary.argtypes = [ctypes.c_int, ctypes.c_double]
        L.oracle_libm_mismatches.restype = ctypes.c_longlong
        L.oracle_libm_mismatches.argtypes = [ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_longlong,
                                             ctypes.c_ulonglong]
        L.oracle_qfix.argtypes = [ctypes.POINTER(CParams), _dp, _dp]
        L.oracle_setvars.argtypes = [ctypes.POINTER(CParams), _dp, _dp]

    def threads(self, n: int = 0) -> int:
        return self.lib.oracle_threads(n)

    def set_libm(self, libm: str) -> None:
        """'glibc' (default; gfortran on x86-64 Linux links glibc's libm) or
        'portable' (the deterministic elementary functions the CUDA step uses)."""
        if libm not in ("glibc", "portable"):
            raise ValueError(libm)
        self.lib.oracle_set_libm(1 if libm == "portable" else 0)

    ELEMENTARY = ["exp", "atan", "tan", "tanh", "pow73", "log", "expm1"]

    def elementary(self, name: str, x: float) -> float:
        """The portable elementary function `name` (exp, atan, tan, tanh, pow73, log, expm1) at x."""
        return self.lib.oracle_elementary(self.ELEMENTARY.index(name), float(x))

    def libm_mismatches(self, name: str, lo: float, hi: float, n: int, seed: int = 1) -> int:
        """How many of n seeded uniform arguments in [lo, hi) give the portable
        function `name` and glibc's different bits."""
        return self.lib.oracle_libm_mismatches(self.ELEMENTARY.index(name), float(lo), float(hi), int(n), int(seed))

    def run(self, p: DClawParams, q: np.ndarray, b: np.ndarray, dx: float, dy: float, nsteps: int,
            dt_initial: float, t_final: float = 0.0, fixed_dt: bool = False, parallel: bool = True,
            branch_log: bool = False, libm: str = "glibc", t_obs: float = 0.0):
        """Advance q (5, my, mx) by nsteps; returns dict(q, dt, cfl, t, status, xlog, ylog).
        t_obs > 0 clips each dt at the next multiple of t_obs (tick rule only)."""
        self.set_libm(libm)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        b = np.ascontiguousarray(b, dtype=np.float64)
        _, my, mx = q.shape
        dt_hist = np.zeros(max(nsteps, 1))
        cfl_hist = np.zeros(max(nsteps, 1))
        xlog = np.zeros((my + 2, mx + 1), dtype=np.uint32) if branch_log else None
        ylog = np.zeros((mx + 2, my + 1), dtype=np.uint32) if branch_log else None
        t_out = np.zeros(1)
        cp = p.to_c()
        st = self.lib.oracle_run(ctypes.byref(cp), mx, my, dx, dy, _ptr(q), _ptr(b), nsteps, dt_initial,
                                 t_final, int(fixed_dt), int(parallel), _ptr(dt_hist), _ptr(cfl_hist),
                                 _ptr(xlog, _up), _ptr(ylog, _up), _ptr(t_out), float(t_obs))
        return dict(q=q, dt=dt_hist[:nsteps], cfl=cfl_hist[:nsteps], t=float(t_out[0]), status=st,
                    xlog=xlog, ylog=ylog)

    def run_full(self, p: DClawParams, q: np.ndarray, b: np.ndarray, dx: float, dy: float, nsteps: int,
                 dt_initial: float, h_e: np.ndarray | None = None, t_final: float = 0.0, fixed_dt: bool = False,
                 parallel: bool = True, branch_log: bool = False, libm: str = "glibc"):
        """The whole state: q (7, my, mx) = (h, hu, hv, hm, pb, hchi, bdif);
        h_e (my, mx): the erodible depth (entrainment). Same results as run()."""
        self.set_libm(libm)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        b = np.ascontiguousarray(b, dtype=np.float64)
        he = None if h_e is None else np.ascontiguousarray(h_e, dtype=np.float64)
        _, my, mx = q.shape
        dt_hist = np.zeros(max(nsteps, 1))
        cfl_hist = np.zeros(max(nsteps, 1))
        xlog = np.zeros((my + 2, mx + 1), dtype=np.uint32) if branch_log else None
        ylog = np.zeros((mx + 2, my + 1), dtype=np.uint32) if branch_log else None
        t_out = np.zeros(1)
        cp = p.to_c()
        st = self.lib.oracle_run_full(ctypes.byref(cp), mx, my, dx, dy, _ptr(q), _ptr(b), _ptr(he), nsteps,
                                      dt_initial, t_final, int(fixed_dt), int(parallel), _ptr(dt_hist),
                                      _ptr(cfl_hist), _ptr(xlog, _up), _ptr(ylog, _up), _ptr(t_out))
        return dict(q=q, dt=dt_hist[:nsteps], cfl=cfl_hist[:nsteps], t=float(t_out[0]), status=st,
                    xlog=xlog, ylog=ylog)

    # ---- patch calls on the padded SoA layout ------------------------------
    def bc2amr(self, p: DClawParams, q: np.ndarray) -> np.ndarray:
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        my, mx = q.shape[1] - 4, q.shape[2] - 4
        cp = p.to_c()
        self.lib.oracle_bc2amr(ctypes.byref(cp), mx, my, _ptr(q))
        return q

    def setaux(self, p: DClawParams, b: np.ndarray) -> np.ndarray:
        b = np.ascontiguousarray(b, dtype=np.float64)
        my, mx = b.shape
        aux = np.zeros((6, my + 4, mx + 4))
        cp = p.to_c()
        self.lib.oracle_setaux(ctypes.byref(cp), mx, my, _ptr(b), _ptr(aux))
        return aux

    def b4step2(self, p: DClawParams, q: np.ndarray, aux: np.ndarray, dx: float, dy: float, libm: str = "glibc"):
        self.set_libm(libm)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        aux = np.ascontiguousarray(aux, dtype=np.float64).copy()
        my, mx = q.shape[1] - 4, q.shape[2] - 4
        cp = p.to_c()
        self.lib.oracle_b4step2(ctypes.byref(cp), mx, my, dx, dy, _ptr(q), _ptr(aux))
        return q, aux

    def step2(self, p: DClawParams, q: np.ndarray, aux: np.ndarray, dx: float, dy: float, dt: float,
              parallel: bool = False, fluxes: bool = False, branch_log: bool = False, libm: str = "glibc"):
        self.set_libm(libm)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        aux = np.ascontiguousarray(aux, dtype=np.float64)
        my, mx = q.shape[1] - 4, q.shape[2] - 4
        cfl = np.zeros(1)
        fl = np.zeros((20, my + 4, mx + 4)) if fluxes else None
        xlog = np.zeros((my + 2, mx + 1), dtype=np.uint32) if branch_log else None
        ylog = np.zeros((mx + 2, my + 1), dtype=np.uint32) if branch_log else None
        cp = p.to_c()
        self.lib.oracle_step2(ctypes.byref(cp), mx, my, dx, dy, dt, _ptr(q), _ptr(aux), _ptr(cfl), _ptr(fl),
                              int(parallel), _ptr(xlog, _up), _ptr(ylog, _up))
        return dict(q=q, cfl=float(cfl[0]), fluxes=fl, xlog=xlog, ylog=ylog)

    def src2(self, p: DClawParams, q: np.ndarray, aux: np.ndarray, dt: float, libm: str = "glibc") -> np.ndarray:
        self.set_libm(libm)
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        aux = np.ascontiguousarray(aux, dtype=np.float64)
        my, mx = q.shape[1] - 4, q.shape[2] - 4
        cp = p.to_c()
        self.lib.oracle_src2(ctypes.byref(cp), mx, my, dt, _ptr(q), _ptr(aux))
        return q

    def qfix(self, p: DClawParams, state):
        s = np.array(state, dtype=np.float64)
        prim = np.zeros(5)
        cp = p.to_c()
        self.lib.oracle_qfix(ctypes.byref(cp), _ptr(s), _ptr(prim))
        return s, prim

    def setvars(self, p: DClawParams, inp):
        a = np.array(inp, dtype=np.float64)
        out = np.zeros(6)
        cp = p.to_c()
        self.lib.oracle_setvars(ctypes.byref(cp), _ptr(a), _ptr(out))
        return out
