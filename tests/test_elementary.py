"""The portable elementary functions (dclaw_b200/csrc/elementary.cuh), on the
host build the oracle links (the same source the CUDA step compiles).

* exp, expm1, tanh and pow restate the algorithms of glibc's libm (the libm the
  reference's gfortran build calls on x86-64 Linux): bit for bit against
  glibc over the ranges the step produces and the whole domain.
* atan and tan are correctly rounded, checked against 200-bit mpmath; glibc's
  (IBM's accurate tables) differ from correct rounding in about 0.2 % of
  arguments, which is all that is left between the two.
* pow (Manning's h^(7/3)) restates glibc's too: bit for bit.
* log (src2method 2 only) stays within 2 ulp.
"""
import numpy as np
import pytest

from dclaw_b200 import workloads as W


def ulp_err(got, ref):
    ref = np.asarray(ref, dtype=np.longdouble)
    r64 = ref.astype(np.float64)
    u = np.spacing(np.abs(r64)).astype(np.longdouble)
    return np.abs(np.asarray(got, dtype=np.longdouble) - ref) / u


CASES = {
    "exp": (np.exp, [(-700.0, 700.0), (-12.0, 16.0), (-1e-3, 1e-3)], 0.52),
    "expm1": (np.expm1, [(-40.0, 40.0), (-1.0, 1.0), (-1e-3, 1e-3)], 1.0),
    "atan": (np.arctan, [(-1e6, 1e6), (-3.0, 3.0), (-0.2, 0.2)], 0.51),
    "tan": (np.tan, [(-1.5, 1.5), (-0.8, 0.8), (-100.0, 100.0)], 0.51),
    # glibc's tanh is within 2 ulp (its own libm-test-ulps figure); numpy's np.tanh is
    # not glibc's (SIMD code of its own), so the bit-exact check goes through C
    "tanh": (np.tanh, [(-25.0, 25.0), (-0.6, 0.6), (-1e-6, 1e-6), (-60.0, 60.0)], 2.05),
    # h^(7/3) is pow at the double nearest 7/3 (the reference's h**(7.d0/3.d0))
    "pow73": (lambda x: np.power(x, np.longdouble(7.0 / 3.0)), [(1e-3, 10.0), (1e-6, 1e3)], 0.52),
    "log": (np.log, [(1e-300, 1e300), (0.5, 2.0), (0.9, 1.1), (1e-3, 1e3)], 2.0),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_accuracy(oracle, name):
    """Error against numpy's 64-bit-significand long double (itself good to
    about 2^-11 ulp of a double, hence the 0.51 for correct rounding)."""
    fn, ranges, bound = CASES[name]
    rng = np.random.default_rng(7)
    worst = 0.0
    for lo, hi in ranges:
        xs = rng.uniform(lo, hi, 4000)
        if name in ("pow73", "log"):
            xs = np.exp(rng.uniform(np.log(lo), np.log(hi), 4000))
        got = np.array([oracle.elementary(name, x) for x in xs])
        ref = fn(xs.astype(np.longdouble))
        worst = max(worst, float(ulp_err(got, ref).max()))
    assert worst <= bound, f"{name}: {worst:.2f} ulp"


# arguments of the step: exp(-(m - mref)/0.04) and the relaxation factors,
# tanh(100 (m - 0.1)) and the Manning ramp, and the whole domain
GLIBC_RANGES = {
    "exp": [(-10.0, 15.0), (-745.2, 709.8), (-746.0, -700.0), (-1e-8, 1e-8)],
    "expm1": [(-40.0, 40.0), (-1.0, 1.0), (-745.0, 710.0), (-1e-9, 1e-9)],
    "tanh": [(-10.0, 90.0), (-1.0, 1.0), (-22.5, 22.5), (-1e-9, 1e-9)],
    # Manning's h^(7/3) over the depths of a run and far beyond
    "pow73": [(1e-3, 10.0), (0.9, 1.1), (1e-6, 1e3), (1e-300, 1e300)],
}


@pytest.mark.parametrize("name", sorted(GLIBC_RANGES))
def test_bit_exact_with_glibc(oracle, name):
    for k, (lo, hi) in enumerate(GLIBC_RANGES[name]):
        bad = oracle.libm_mismatches(name, lo, hi, 1_000_000, seed=1 + k)
        assert bad == 0, f"{name} on [{lo}, {hi}]: {bad} of 1e6 arguments differ from glibc"


@pytest.mark.parametrize("name", ["atan", "tan"])
def test_correctly_rounded(oracle, name):
    mpmath = pytest.importorskip("mpmath")
    mpmath.mp.prec = 200
    fn = {"atan": mpmath.atan, "tan": mpmath.tan}[name]
    rng = np.random.default_rng(3)
    xs = np.concatenate([rng.uniform(-1.0, 1.0, 1500), rng.uniform(-0.3, 1.5, 1500),
                         rng.uniform(-40.0, 40.0, 500), rng.uniform(-1e-5, 1e-5, 200),
                         np.exp(rng.uniform(-60.0, 60.0 if name == "atan" else 14.0, 300))])
    bad = [x for x in xs if oracle.elementary(name, float(x)) != float(fn(mpmath.mpf(float(x))))]
    assert not bad, f"{name}: {len(bad)} arguments not correctly rounded, e.g. {bad[:3]}"


@pytest.mark.parametrize("name,lo,hi,most", [("atan", -1.0, 1.0, 0.004), ("tan", -0.3, 1.5, 0.004)])
def test_residual_difference_from_glibc(oracle, name, lo, hi, most):
    """What is left between the correctly rounded functions and glibc's."""
    frac = oracle.libm_mismatches(name, lo, hi, 1_000_000) / 1e6
    assert 0.0 < frac <= most


def test_special_values(oracle):
    e = oracle.elementary
    assert e("exp", 0.0) == 1.0 and e("exp", -800.0) == 0.0 and np.isinf(e("exp", 800.0))
    assert np.isnan(e("exp", np.nan)) and np.isnan(e("tanh", np.nan))
    assert e("exp", -np.inf) == 0.0 and np.isinf(e("exp", np.inf))
    assert e("tanh", 30.0) == 1.0 and e("tanh", -30.0) == -1.0 and e("tanh", 1e-20) == 1e-20
    assert e("expm1", -50.0) == -1.0 and e("expm1", 0.0) == 0.0
    assert e("atan", 0.0) == 0.0 and e("atan", 1e300) == np.arctan(1e300) and e("atan", -np.inf) == -np.pi / 2
    assert e("tan", 0.0) == 0.0 and np.isnan(e("tan", np.inf))
    assert e("log", 1.0) == 0.0 and np.isinf(e("log", 0.0)) and e("log", 0.0) < 0 and np.isnan(e("log", -1.0))
    assert e("log", 2.0) == np.log(2.0) and abs(e("log", 5e-324) - np.log(5e-324)) < 1e-12
    # tanh(100 (m - 0.1)) saturates to exactly 1 for debris (m > 0.32) as glibc's does
    for m in (0.33, 0.55, 0.64, 1.0):
        assert e("tanh", 100.0 * (m - 0.1)) == 1.0 == np.tanh(100.0 * (m - 0.1))


def test_slope_runout_glibc_steps(oracle):
    """The step run on these functions against the same step on glibc's libm
    (the oracle both ways): the 200 x 200 slope-runout case (order 2,
    transverse 2, MC) stays bit-identical through step 86, the first
    argument at which glibc's atan or tan is not correctly rounded comes at
    step 87, and the dry/wet masks still agree at step 200."""
    c = W.slope_runout()
    a = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 86, c.dt_initial, libm="glibc")
    b = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 86, c.dt_initial, libm="portable")
    assert np.array_equal(a["q"], b["q"]) and np.array_equal(a["dt"], b["dt"])
    a = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 87, c.dt_initial, libm="glibc")
    b = oracle.run(c.params, c.q, c.b, c.dx, c.dy, 87, c.dt_initial, libm="portable")
    assert not np.array_equal(a["q"], b["q"])
    assert max(np.abs(a["q"][m] - b["q"][m]).max() / np.abs(a["q"][m]).max() for m in range(5)) < 1e-14
