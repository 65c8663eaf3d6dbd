"""The portable elementary functions (dclaw_b200/csrc/elementary.cuh) against
extended-precision references (numpy longdouble, 64-bit significand): the
error stays within 2 ulp of the true value (3 ulp for tan, a quotient of two
series, and for h^(7/3)) on the argument ranges the step produces and well
beyond."""
import numpy as np
import pytest


def ulp_err(got, ref):
    ref = np.asarray(ref, dtype=np.longdouble)
    r64 = ref.astype(np.float64)
    u = np.spacing(np.abs(r64)).astype(np.longdouble)
    return np.abs(np.asarray(got, dtype=np.longdouble) - ref) / u


CASES = {
    "exp": (np.exp, [(-700.0, 700.0), (-12.0, 16.0), (-1e-3, 1e-3)]),
    "atan": (np.arctan, [(-1e6, 1e6), (-3.0, 3.0), (-0.2, 0.2)]),
    "tan": (np.tan, [(-1.5, 1.5), (-0.8, 0.8), (-100.0, 100.0)]),
    "tanh": (np.tanh, [(-25.0, 25.0), (-0.6, 0.6), (-1e-6, 1e-6), (-60.0, 60.0)]),
    "pow73": (lambda x: np.power(x, np.longdouble(7) / 3), [(1e-3, 10.0), (1e-6, 1e3)]),
    "log": (np.log, [(1e-300, 1e300), (0.5, 2.0), (0.9, 1.1), (1e-3, 1e3)]),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_accuracy(oracle, name):
    fn, ranges = CASES[name]
    rng = np.random.default_rng(7)
    worst = 0.0
    for lo, hi in ranges:
        xs = rng.uniform(lo, hi, 4000)
        if name in ("pow73", "log"):
            xs = np.exp(rng.uniform(np.log(lo), np.log(hi), 4000))
        got = np.array([oracle.elementary(name, x) for x in xs])
        ref = fn(xs.astype(np.longdouble))
        worst = max(worst, float(ulp_err(got, ref).max()))
    bound = 3.0 if name in ("tan", "pow73") else 2.0
    assert worst <= bound, f"{name}: {worst:.2f} ulp"


def test_special_values(oracle):
    e = oracle.elementary
    assert e("exp", 0.0) == 1.0 and e("exp", -800.0) == 0.0 and np.isinf(e("exp", 800.0))
    assert np.isnan(e("exp", np.nan)) and np.isnan(e("tanh", np.nan))
    assert e("tanh", 30.0) == 1.0 and e("tanh", -30.0) == -1.0 and e("tanh", 1e-20) == 1e-20
    assert e("atan", 0.0) == 0.0 and abs(e("atan", 1e300) - np.pi / 2) < 1e-16
    assert e("tan", 0.0) == 0.0
    assert e("log", 1.0) == 0.0 and np.isinf(e("log", 0.0)) and e("log", 0.0) < 0 and np.isnan(e("log", -1.0))
    assert e("log", 2.0) == np.log(2.0) and abs(e("log", 5e-324) - np.log(5e-324)) < 1e-12
    # tanh(100 (m - 0.1)) saturates to exactly 1 for debris (m > 0.32) as glibc's does
    for m in (0.33, 0.55, 0.64, 1.0):
        assert e("tanh", 100.0 * (m - 0.1)) == 1.0 == np.tanh(100.0 * (m - 0.1))
