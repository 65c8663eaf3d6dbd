"""The CUDA step's stage arithmetic (dclaw_b200/csrc/stages.cuh) run on the
host against the oracle: bit-identical state, dt/Courant histories and
branch bits. The oracle runs with the same portable elementary functions as
the device code, so any difference is a logic or operation-order error."""
import numpy as np
import pytest

from dclaw_b200 import workloads as W

from ._emu import Emu


@pytest.fixture(scope="module")
def emu():
    return Emu()


def _cmp(oracle, emu, c, n, fused=False):
    r1 = oracle.run(c.params, c.q, c.b, c.dx, c.dy, n, c.dt_initial, branch_log=True, libm="portable")
    r2 = emu.run(c.params, c.q, c.b, c.dx, c.dy, n, c.dt_initial, fused=fused)
    br1 = np.concatenate([r1["xlog"].ravel(), r1["ylog"].ravel()])
    assert r1["status"] == r2["status"] == 0
    assert np.array_equal(r1["q"], r2["q"])
    assert np.array_equal(r1["dt"], r2["dt"]) and np.array_equal(r1["cfl"], r2["cfl"])
    assert np.array_equal(br1, r2["br"])


@pytest.mark.parametrize("fused", [False, True], ids=["staged", "fused"])
@pytest.mark.parametrize("name", ["slope_runout", "contact_wave", "dam_front", "lake_at_rest"])
def test_cases(oracle, emu, name, fused):
    c = {"slope_runout": W.slope_runout, "contact_wave": W.contact_wave, "dam_front": W.dam_front,
         "lake_at_rest": W.lake_at_rest}[name]()
    _cmp(oracle, emu, c, 40, fused)


VARIANTS = {
    "order1": dict(order=1, transverse_waves=0), "transverse1": dict(transverse_waves=1),
    "minmod": dict(limiter=1), "superbee": dict(limiter=2), "vanleer": dict(limiter=3), "nolimiter": dict(limiter=0),
    "extrap": dict(bc_lower=("extrap", "wall"), bc_upper=("extrap", "extrap")),
    "src2m1": dict(src2method=1), "swe": dict(src2method=-1), "alpha1": dict(alphamethod=1),
    "src2m2": dict(src2method=2, alphamethod=1),
    "rarecorrector": dict(rarecorrectortest=True),
    "manning": dict(friction_forcing=True, manning_coefficient=0.025),
    "dd_manning": dict(friction_forcing=True, manning_coefficient=0.025, dd_manning=True),
    "speed_limit": dict(speed_limit=2.0),
}


@pytest.mark.parametrize("fused", [False, True], ids=["staged", "fused"])
@pytest.mark.parametrize("variant", sorted(VARIANTS))
def test_variants(oracle, emu, variant, fused):
    base = W.slope_runout(n=96)
    c = W.Case(base.name, base.q, base.b, base.dx, base.dy, base.params.replace(**VARIANTS[variant]), 0,
               base.dt_initial)
    _cmp(oracle, emu, c, 60, fused)


@pytest.mark.parametrize("fused", [False, True], ids=["staged", "fused"])
def test_random_field_small(oracle, emu, fused):
    c = W.random_field_case(n=128, dx=0.5, seed=3)
    _cmp(oracle, emu, c, 30, fused)


@pytest.mark.parametrize("src2_in_tile", [False, True])
@pytest.mark.parametrize("tile", [(14, 13), (13, 14), (16, 16), (16, 14), (8, 8)])
def test_fused_tile_shapes_and_partial_tiles(oracle, emu, tile, src2_in_tile):
    """Tile shapes of the fused step on a patch whose sizes are not multiples
    of the tile."""
    c = W.random_field_case(n=128, dx=0.5, seed=4)
    q = c.q[:, :71, :93].copy()
    b = c.b[:71, :93].copy()
    c2 = W.Case("partial", q, b, c.dx, c.dy, c.params, 0, c.dt_initial)
    r1 = oracle.run(c2.params, c2.q, c2.b, c2.dx, c2.dy, 25, c2.dt_initial, branch_log=True, libm="portable")
    r2 = emu.run(c2.params, c2.q, c2.b, c2.dx, c2.dy, 25, c2.dt_initial, fused=True, tile=tile,
                 src2_in_tile=src2_in_tile)
    assert np.array_equal(r1["q"], r2["q"])
    assert np.array_equal(np.concatenate([r1["xlog"].ravel(), r1["ylog"].ravel()]), r2["br"])


@pytest.mark.parametrize("tile", [(14, 13), (16, 14)])
@pytest.mark.parametrize("shape", [(2, 2), (17, 3), (3, 17), (13, 14), (14, 15), (27, 29)])
def test_fused_small_patches(oracle, emu, tile, shape):
    """Patches smaller than, equal to or just over one tile, and thin strips,
    around the wettest cell of a random field: the flux phase with each
    interface limited once (14 x 13) and with each cell limiting both of
    its interfaces (16 x 14) give the oracle's state and branch bits."""
    c = W.random_field_case(n=128, dx=0.5, seed=4)
    my, mx = shape
    j, i = np.unravel_index(np.argmax(c.q[0]), c.q[0].shape)
    j0, i0 = max(0, j - my // 2), max(0, i - mx // 2)
    q = c.q[:, j0:j0 + my, i0:i0 + mx].copy()
    b = c.b[j0:j0 + my, i0:i0 + mx].copy()
    assert q[0].max() > 0.0
    r1 = oracle.run(c.params, q, b, c.dx, c.dy, 10, c.dt_initial, branch_log=True, libm="portable")
    r2 = emu.run(c.params, q, b, c.dx, c.dy, 10, c.dt_initial, fused=True, tile=tile)
    assert np.array_equal(r1["q"], r2["q"])
    assert np.array_equal(np.concatenate([r1["xlog"].ravel(), r1["ylog"].ravel()]), r2["br"])


# ---- the full-state step (segregation, entrainment) --------------------------
FULL_VARIANTS = {
    "extras_zero": dict(segregation=0, entrainment=0),
    "segregation": dict(),
    "segregation_beta0": dict(beta_seg=0.0),
    "entrainment_only": dict(segregation=0),
    "both_manning": dict(friction_forcing=True, manning_coefficient=0.03),
    "both_src2m1": dict(src2method=1),
    "both_swe": dict(src2method=-1),
    "both_src2m2": dict(src2method=2, alphamethod=1),
    "both_order1": dict(order=1, transverse_waves=0),
    "both_extrap": dict(bc_lower=("extrap", "wall"), bc_upper=("extrap", "extrap")),
    "entrainment_method1": dict(entrainment_method=1),
}


@pytest.mark.parametrize("variant", sorted(FULL_VARIANTS))
def test_full_state_stages(oracle, emu, variant):
    """The full-state stages (dclaw_b200/csrc/full_state.cuh) on the host
    against the oracle's seven-field step: state (hchi and bdif included),
    dt/Courant histories and branch bits, bit for bit."""
    kw = dict(FULL_VARIANTS[variant])
    seg = kw.pop("segregation", 1)
    ent = kw.pop("entrainment", 1)
    c = W.slope_runout_full(n=96, segregation=seg, entrainment=ent)
    p = c.params.replace(**kw)
    r1 = oracle.run_full(p, c.q, c.b, c.dx, c.dy, 60, c.dt_initial, h_e=c.h_e, branch_log=True, libm="portable")
    r2 = emu.run_full(p, c.q, c.b, c.dx, c.dy, 60, c.dt_initial, h_e=c.h_e)
    assert r1["status"] == r2["status"] == 0
    assert np.array_equal(r1["q"], r2["q"])
    assert np.array_equal(r1["dt"], r2["dt"]) and np.array_equal(r1["cfl"], r2["cfl"])
    assert np.array_equal(np.concatenate([r1["xlog"].ravel(), r1["ylog"].ravel()]), r2["br"])
    if seg:
        chi = r1["q"][5][r1["q"][0] > 0] / r1["q"][0][r1["q"][0] > 0]
        assert chi.min() >= 0.0 and chi.max() <= 1.0
    if ent and p.entrainment_method == 0:
        assert r1["q"][6].max() > 0.0 and r1["q"][6].max() <= c.h_e.max()
    else:
        assert not r1["q"][6].any()


def test_full_state_without_extras_is_the_five_field_step(oracle):
    """hchi = bdif = 0 with both options off: the oracle's seven-field run
    gives the five-field run's bits and keeps the extra fields zero."""
    c = W.slope_runout(n=96)
    a = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 40, c.dt_initial, libm="portable")
    f = oracle.run_full(c.params, W.full_state(c.q, c.params), c.b, c.dx, c.dy, 40, c.dt_initial, libm="portable")
    assert np.array_equal(a["q"], f["q"][:5]) and not f["q"][5:].any()
