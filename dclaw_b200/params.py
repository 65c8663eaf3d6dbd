"""Run parameters, mirroring the reference's setrun data classes.

Names and defaults follow src/python/dclaw/data.py:315-351 (DClawInputData),
GeoClaw's geo_data (grav, dry_tolerance, speed_limit, friction_*), and
clawdata (order, transverse_waves, limiter, cfl_*, dt_*, bc_*). As in
set_dig (src/2d/dig/digclaw_module.f90:135-136,150-151) the friction and
slope angles are given in degrees here and handed to the device in radians.

`CParams` is the ctypes image of `dclaw_params` in include/dclaw_b200.h.
"""
from __future__ import annotations

import ctypes
import dataclasses
import math

BC_CODES = {"extrap": 1, "wall": 3}


class CParams(ctypes.Structure):
    _fields_ = [
        ("grav", ctypes.c_double),
        ("dry_tolerance", ctypes.c_double),
        ("speed_limit", ctypes.c_double),
        ("friction_forcing", ctypes.c_int32),
        ("dd_manning", ctypes.c_int32),
        ("manning_coefficient", ctypes.c_double),
        ("friction_depth", ctypes.c_double),
        ("manning_max", ctypes.c_double),
        ("rho_s", ctypes.c_double),
        ("rho_f", ctypes.c_double),
        ("m_crit", ctypes.c_double),
        ("m0", ctypes.c_double),
        ("mref", ctypes.c_double),
        ("kref", ctypes.c_double),
        ("phi", ctypes.c_double),
        ("delta", ctypes.c_double),
        ("mu", ctypes.c_double),
        ("alpha_c", ctypes.c_double),
        ("c1", ctypes.c_double),
        ("sigma_0", ctypes.c_double),
        ("theta_input", ctypes.c_double),
        ("src2method", ctypes.c_int32),
        ("alphamethod", ctypes.c_int32),
        ("rarecorrectortest", ctypes.c_int32),
        ("bed_normal", ctypes.c_int32),
        ("entrainment", ctypes.c_int32),
        ("segregation", ctypes.c_int32),
        ("curvature", ctypes.c_int32),
        ("order", ctypes.c_int32),
        ("transverse_waves", ctypes.c_int32),
        ("limiter", ctypes.c_int32),
        ("bc_lower", ctypes.c_int32 * 2),
        ("bc_upper", ctypes.c_int32 * 2),
        ("cfl_desired", ctypes.c_double),
        ("cfl_max", ctypes.c_double),
        ("dt_max", ctypes.c_double),
        ("beta_seg", ctypes.c_double),
        ("delta_kr_order", ctypes.c_double),
        ("chie", ctypes.c_double),
        ("me", ctypes.c_double),
        ("entrainment_rate", ctypes.c_double),
        ("entrainment_method", ctypes.c_int32),
        ("pad_", ctypes.c_int32),
    ]


class CClock(ctypes.Structure):
    """ctypes image of `dclaw_clock` (device-resident run clock)."""

    _fields_ = [
        ("t", ctypes.c_double),
        ("dt", ctypes.c_double),
        ("cfl", ctypes.c_double),
        ("dt_last", ctypes.c_double),
        ("t_final", ctypes.c_double),
        ("cfl_bits", ctypes.c_uint64),
        ("nsteps", ctypes.c_uint32),
        ("blocks_done", ctypes.c_uint32),
        ("status", ctypes.c_int32),
        ("fixed_dt", ctypes.c_int32),
        ("t_obs", ctypes.c_double),
    ]


CLOCK_DOUBLES = ctypes.sizeof(CClock) // 8  # the clock is kept in a float64 tensor


class CMember(ctypes.Structure):
    """ctypes image of `dclaw_member` (one ensemble member's table entry)."""

    _fields_ = [
        ("mx", ctypes.c_int32), ("my", ctypes.c_int32),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("q_off", ctypes.c_uint64), ("b_off", ctypes.c_uint64),
        ("rec_off", ctypes.c_uint64), ("qs_off", ctypes.c_uint64),
        ("tile0", ctypes.c_uint32), ("ntiles_x", ctypes.c_uint32), ("ntiles", ctypes.c_uint32),
        ("rchunk0", ctypes.c_uint32), ("nrchunks", ctypes.c_uint32),
        ("schunk0", ctypes.c_uint32), ("nschunks", ctypes.c_uint32), ("pad_", ctypes.c_uint32),
    ]


class CBatch(ctypes.Structure):
    """ctypes image of `dclaw_batch` (an ensemble's totals and launch choices)."""

    _fields_ = [
        ("nmembers", ctypes.c_int32), ("tile_shape", ctypes.c_int32),
        ("tile_ctas_per_sm", ctypes.c_int32), ("cell_ctas_per_sm", ctypes.c_int32),
        ("ntiles", ctypes.c_uint32), ("nrchunks", ctypes.c_uint32), ("nschunks", ctypes.c_uint32),
        ("pad_", ctypes.c_uint32),
        ("q_doubles", ctypes.c_uint64), ("b_doubles", ctypes.c_uint64), ("work_bytes", ctypes.c_uint64),
    ]


class CAdjMember(ctypes.Structure):
    """ctypes image of `dclaw_adj_member` (one ensemble member of the adjoint)."""

    _fields_ = [
        ("mx", ctypes.c_int32), ("my", ctypes.c_int32),
        ("dx", ctypes.c_double), ("dy", ctypes.c_double),
        ("q_off", ctypes.c_uint64), ("b_off", ctypes.c_uint64), ("work_off", ctypes.c_uint64),
        ("chunk0", ctypes.c_uint32 * 6), ("nchunk", ctypes.c_uint32 * 6),
    ]


class CAdjBatch(ctypes.Structure):
    """ctypes image of `dclaw_adj_batch`."""

    _fields_ = [
        ("nmembers", ctypes.c_int32), ("chunk_items", ctypes.c_uint32), ("nchunks", ctypes.c_uint32 * 6),
        ("nblocks", ctypes.c_uint32), ("pad_", ctypes.c_uint32), ("work_bytes", ctypes.c_uint64),
    ]


@dataclasses.dataclass
class DClawParams:
    """D-Claw parameters for one run (or one ensemble member).

    Defaults are the reference's DClawInputData defaults except where the
    uniform-patch benchmark cases fix a value (m_crit 0.64, kref 1e-10,
    phi 32 deg, mu 0.005); GeoClaw's speed_limit default is not part of
    the reference tree, so it is set explicitly (1e6 m/s, i.e. inactive).
    """

    # geo_data
    grav: float = 9.81
    dry_tolerance: float = 1.0e-3
    speed_limit: float = 1.0e6
    friction_forcing: bool = False
    manning_coefficient: float = 0.0
    friction_depth: float = 1.0e6
    dd_manning: bool = False
    manning_max: float = 0.06
    # dclaw_data (data.py:315-351)
    rho_s: float = 2700.0
    rho_f: float = 1000.0
    m_crit: float = 0.64
    m0: float = 0.62
    mref: float = 0.60
    kref: float = 1.0e-10
    phi: float = 32.0            # degrees
    delta: float = 0.01
    mu: float = 0.005
    alpha_c: float = 0.01
    c1: float = 1.0
    sigma_0: float = 1.0e3
    src2method: int = 0
    alphamethod: int = 0
    rarecorrectortest: bool = False
    bed_normal: int = 0
    theta_input: float = 0.0     # degrees
    entrainment: int = 0
    segregation: int = 0
    curvature: int = 0
    # segregation and entrainment (data.py:338-347; the full-state step only)
    beta_seg: float = 0.0
    chi0: float = 0.5            # initial species fraction (qinit.f90:219-226); initial states only
    chie: float = 0.5
    delta_kr_order: float = 2.0
    me: float = 0.65
    entrainment_rate: float = 0.2
    entrainment_method: int = 1
    # clawdata
    order: int = 2
    transverse_waves: int = 2
    limiter: int = 4             # MC for every wave family
    bc_lower: tuple = ("wall", "wall")
    bc_upper: tuple = ("wall", "wall")
    cfl_desired: float = 0.9
    cfl_max: float = 1.0
    dt_max: float = 1.0e99

    def replace(self, **kw) -> "DClawParams":
        return dataclasses.replace(self, **kw)

    def to_c(self) -> CParams:
        c = CParams()
        deg = math.pi / 180.0
        for f in CParams._fields_:
            name = f[0]
            if name in ("bc_lower", "bc_upper"):
                vals = getattr(self, name)
                arr = (ctypes.c_int32 * 2)(*[BC_CODES[v] if isinstance(v, str) else int(v) for v in vals])
                setattr(c, name, arr)
            elif name == "phi":
                c.phi = deg * float(self.phi)
            elif name == "theta_input":
                c.theta_input = deg * float(self.theta_input)
            elif name == "pad_":
                continue
            else:
                v = getattr(self, name)
                setattr(c, name, int(v) if isinstance(v, bool) else v)
        return c


def config0_params(**kw) -> DClawParams:
    """Parameters of the 200x200 slope-runout case (rho_s 2700, rho_f 1000,
    phi 32 deg, m_crit 0.64, k0 1e-10, mu 0.005, alpha 0.01, dry_tol 1e-3,
    walls), second order with transverse corrections and the MC limiter."""
    return DClawParams(**kw)
