"""TEST INFRASTRUCTURE: host build of the adjoint routines (tests/adj)."""
from __future__ import annotations

import ctypes
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent / "adj"
SRC = HERE / "adj_check.cpp"
LIB = HERE / "libadj.so"
CSRC = Path(__file__).resolve().parents[1] / "dclaw_b200" / "csrc"

_dp = ctypes.POINTER(ctypes.c_double)

LOCAL_CHECKS = ["qfix", "qfix_cmass", "setvars", "setvars_all", "setvars_all_alphamethod1", "riemanntype",
                "riemann_wet", "riemann_dry_side_or_wall", "riemann_at_rest", "riemann_src2method_-1",
                "limiter_minmod", "limiter_superbee", "limiter_vanleer", "limiter_mc", "rpt2", "src2_method0",
                "src2_method1", "src2_method-1", "src2_at_rest", "src2_manning", "src2_dd_manning",
                "riemann_rare_corrector"]


def build() -> Path:
    deps = [SRC, *CSRC.glob("*.cuh")]
    if LIB.exists() and all(d.stat().st_mtime <= LIB.stat().st_mtime for d in deps):
        return LIB
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-shared",
                    str(SRC), "-o", str(LIB)], check=True)
    return LIB


class Adj:
    def __init__(self):
        self.lib = ctypes.CDLL(str(build()))
        self.lib.adj_check_local.restype = ctypes.c_int
        self.lib.adj_check_local.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int, _dp,
                                             ctypes.POINTER(ctypes.c_int)]
        self.lib.adj_step_fwd.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, _dp, _dp, ctypes.c_double, _dp]
        self.lib.adj_step_vjp.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_double,
                                          ctypes.c_double, _dp, _dp, ctypes.c_double, _dp, _dp, _dp, _dp]

    def local(self, name: str, seed: int = 1, n: int = 1000):
        err = ctypes.c_double()
        sk = ctypes.c_int()
        cnt = self.lib.adj_check_local(LOCAL_CHECKS.index(name), seed, n, ctypes.byref(err), ctypes.byref(sk))
        return cnt, err.value, sk.value

    @staticmethod
    def _p(a):
        return np.ascontiguousarray(a, dtype=np.float64).ctypes.data_as(_dp)

    def step(self, p, q, b, dx, dy, dt):
        q = np.ascontiguousarray(q, dtype=np.float64)
        out = np.zeros_like(q)
        cp = p.to_c()
        self.lib.adj_step_fwd(ctypes.byref(cp), q.shape[2], q.shape[1], dx, dy, self._p(q), self._p(b), dt,
                              out.ctypes.data_as(_dp))
        return out

    def vjp(self, p, q, b, dx, dy, dt, lam, bed=False):
        """lam_in, pbar (and the bed's adjoint with bed=True)."""
        q = np.ascontiguousarray(q, dtype=np.float64)
        lam = np.ascontiguousarray(lam, dtype=np.float64)
        li = np.zeros_like(q)
        pb = np.zeros(4)
        bb = np.zeros(q.shape[1:]) if bed else None
        cp = p.to_c()
        rc = self.lib.adj_step_vjp(ctypes.byref(cp), q.shape[2], q.shape[1], dx, dy, self._p(q), self._p(b), dt,
                                   self._p(lam), li.ctypes.data_as(_dp), pb.ctypes.data_as(_dp),
                                   bb.ctypes.data_as(_dp) if bed else None)
        assert rc == 0
        return (li, pb, bb) if bed else (li, pb)
