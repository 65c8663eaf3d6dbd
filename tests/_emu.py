"""TEST INFRASTRUCTURE: host build of the CUDA stage functions (tests/emu)."""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

from dclaw_b200.params import CParams

HERE = Path(__file__).resolve().parent / "emu"
SRC = HERE / "emu_step.cpp"
LIB = HERE / "libemu.so"
CSRC = Path(__file__).resolve().parents[1] / "dclaw_b200" / "csrc"

_dp = ctypes.POINTER(ctypes.c_double)
_up = ctypes.POINTER(ctypes.c_uint32)


def build() -> Path:
    deps = [SRC, *CSRC.glob("*.cuh")]
    if LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    str(SRC), "-o", str(LIB)], check=True)
    return LIB


class Emu:
    def __init__(self):
        self.lib = ctypes.CDLL(str(build()))
        for fn in (self.lib.emu_run, self.lib.emu_run_fused):
            fn.restype = ctypes.c_int
            fn.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_double, ctypes.c_double,
                           _dp, _dp, ctypes.c_int, ctypes.c_double, ctypes.c_double, ctypes.c_int, _dp, _dp, _up,
                           _dp]
        self.lib.emu_run_fused.argtypes = self.lib.emu_run_fused.argtypes + [ctypes.c_int] * 3
        self.lib.emu_run_full.restype = ctypes.c_int
        self.lib.emu_run_full.argtypes = [ctypes.POINTER(CParams), ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, _dp, _dp, _dp, ctypes.c_int, ctypes.c_double, _dp, _dp,
                                          _up]

    def run_full(self, p, q, b, dx, dy, nsteps, dt_initial, h_e=None):
        """The full-state stages (7 fields) on the host."""
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        b = np.ascontiguousarray(b, dtype=np.float64)
        he = None if h_e is None else np.ascontiguousarray(h_e, dtype=np.float64)
        _, my, mx = q.shape
        dth = np.zeros(max(nsteps, 1))
        cfh = np.zeros(max(nsteps, 1))
        br = np.zeros((my + 2) * (mx + 1) + (mx + 2) * (my + 1), dtype=np.uint32)
        cp = p.to_c()
        st = self.lib.emu_run_full(ctypes.byref(cp), mx, my, dx, dy, q.ctypes.data_as(_dp), b.ctypes.data_as(_dp),
                                   None if he is None else he.ctypes.data_as(_dp), nsteps, dt_initial,
                                   dth.ctypes.data_as(_dp), cfh.ctypes.data_as(_dp), br.ctypes.data_as(_up))
        return dict(q=q, dt=dth[:nsteps], cfl=cfh[:nsteps], status=st, br=br)

    def run(self, p, q, b, dx, dy, nsteps, dt_initial, t_final=0.0, fixed_dt=False, fused=False, tile=(14, 13),
            src2_in_tile=False):
        q = np.ascontiguousarray(q, dtype=np.float64).copy()
        b = np.ascontiguousarray(b, dtype=np.float64)
        _, my, mx = q.shape
        dth = np.zeros(max(nsteps, 1))
        cfh = np.zeros(max(nsteps, 1))
        br = np.zeros((my + 2) * (mx + 1) + (mx + 2) * (my + 1), dtype=np.uint32)
        t = np.zeros(1)
        cp = p.to_c()
        args = [ctypes.byref(cp), mx, my, dx, dy, q.ctypes.data_as(_dp), b.ctypes.data_as(_dp), nsteps, dt_initial,
                t_final, int(fixed_dt), dth.ctypes.data_as(_dp), cfh.ctypes.data_as(_dp), br.ctypes.data_as(_up),
                t.ctypes.data_as(_dp)]
        st = self.lib.emu_run_fused(*args, *tile, int(src2_in_tile)) if fused else self.lib.emu_run(*args)
        assert st >= 0, "tile size not instantiated in the emulation"
        return dict(q=q, dt=dth[:nsteps], cfl=cfh[:nsteps], status=st, br=br, t=float(t[0]))
