"""The oracle's analytic radial forms, pinned to the reference's own tests of
them (tests/unit/test_analytic_functions.cpp) and to its parameter-Jacobian
bars (tests/unit/test_param_jacobian.cpp:54-100).

- every form's value against the reference formula written out by hand, at
  r = 1.4, 2.05, 2.9 (EveryFormMatchesItsReferenceFormula, :292-425), 1e-12
  relative;
- d/dr against central differences of the value at the reference's points
  (the *_FD tests, :22-233), 1e-6 relative + 1e-10;
- exact zeros past the StiwWeb2 / StiwWeb3 / Tersoff cut-offs and the
  piecewise Tersoff cutoff (TersoffCutoffMatchesThePiecewiseForm, :436-449);
- ∂v/∂θ and ∂²v/∂r∂θ against central differences at the reference's default
  parameters, 1e-5 relative + 1e-8, and ∂²v/∂r², 1e-4 relative + 1e-7.
"""
import math

import numpy as np
import pytest

from forcesmith_b200.abi import FORMS
from oracle import api as O


def val(name, params, r, rmax=6.0):
    return O.form_eval(FORMS[name][0], np.asarray(params, float), r, rmax)[0][0]


def der(name, params, r, rmax=10.0):
    return O.form_eval(FORMS[name][0], np.asarray(params, float), r, rmax)[0][1]


def ref_fc(r, R, S):
    if r <= R:
        return 1.0
    if r >= S:
        return 0.0
    return 0.5 + 0.5 * math.cos(math.pi * (r - R) / (S - R))


def ref_sc(r, r0, h):
    if r >= r0:
        return 0.0
    u = (r - r0) / h
    u4 = (u * u) * (u * u)
    return u4 / (1.0 + u4)


TERSOFF = [1830.8, 471.18, 2.4799, 1.7322, 1.1e-6, 0.78734, 100390.0, 16.217, -0.59825, 2.7, 3.0]
TMOD = TERSOFF + [0.01, -0.02, 0.003, -0.0004, 0.00005]


def reference_values(r):
    """(name, params, value) from the reference's hand-written formulas."""
    sr6 = (1.9 / r) ** 6
    e_m = math.exp(-1.4 * (r - 2.6))
    x_b = (0.3 * 0.3) / (r * r)
    r2 = r * r
    r6 = r2 * r2 * r2
    E0, a, b, c = 1.4, 1.1, 2.3, 0.2
    xg = r / 2.4
    e1, e2 = math.exp(-1.3 * (r - 2.2)), math.exp(-2.1 * (r - 2.9))
    z = r - 1.0
    e_mi = math.exp(-1.3 * z)
    s = r - 1.0
    s2 = s * s
    pair = 1830.8 * math.exp(-2.4799 * r) - 471.18 * math.exp(-1.7322 * r)
    r3, r4 = r2 * r, r2 * r2
    r5 = r4 * r
    corr = 1.0 + 0.01 * r - 0.02 * r2 + 0.003 * r3 - 0.0004 * r4 + 0.00005 * r5
    ks, kt = 0.15 + 0.12, 1.1 + 0.9
    kaw = 1.2 * -0.8 / r + 3.0 * ks * math.exp((kt - r) / ks) - 2.0 * 1.5 / r ** 6.0
    w = r - 2.2
    st = r - 0.2
    eopp = 15.0 / r ** 6.0 + (5.0 / r ** 3.0) * math.cos(2.5 * r + 3.0)
    return [
        ("lj", [0.7, 1.9], 4.0 * 0.7 * (sr6 * sr6 - sr6)),
        ("morse", [0.35, 1.4, 2.6], 0.35 * (1.0 - e_m) * (1.0 - e_m) - 0.35),
        ("buckingham", [500.0, 0.3, 2.0], 500.0 * math.exp(-r / 0.3) - 2.0 * x_b * x_b * x_b),
        ("born", [0.4, 2.1, 3.2, 1.7, 2.4], 0.4 * math.exp((3.2 - r) / 2.1) - 1.7 / r6 + 2.4 / (r6 * r2)),
        ("power_decay", [1.3, 2.4], 1.3 / r ** 2.4),
        ("exp_decay", [4.2, 1.1], 4.2 * math.exp(-1.1 * r)),
        ("mexp_decay", [0.9, 1.2, 2.0], 0.9 * math.exp(-1.2 * (r - 2.0))),
        ("harmonic", [0.6, 2.2], 0.6 * (r - 2.2) * (r - 2.2)),
        ("universal", [E0, a, b, c], E0 * (b / (b - a) * r ** a - a / (b - a) * r ** b) + c * r),
        ("eopp", [15.0, 6.0, 5.0, 3.0, 2.5, 3.0], eopp),
        ("eopp_exp", [12.0, 1.3, 5.0, 3.0, 2.5, 3.0],
         12.0 * math.exp(-1.3 * r) + (5.0 / r ** 3.0) * math.cos(2.5 * r + 3.0)),
        ("meopp", [15.0, 6.0, 5.0, 3.0, 2.5, 3.0, 0.4],
         15.0 / (r - 0.4) ** 6.0 + (5.0 / r ** 3.0) * math.cos(2.5 * r + 3.0)),
        ("gen_lj", [0.8, 12.0, 6.0, 2.4, 0.1], 0.8 / (6.0 - 12.0) * (6.0 * xg ** -12.0 - 12.0 * xg ** -6.0) + 0.1),
        ("double_morse", [0.4, 1.3, 2.2, 0.2, 2.1, 2.9, 0.05],
         0.4 * ((1.0 - e1) * (1.0 - e1) - 1.0) + 0.2 * ((1.0 - e2) * (1.0 - e2) - 1.0) + 0.05),
        ("double_exp", [0.7, 1.9, 2.3, 1.4, 2.0],
         0.7 * math.exp(-1.9 * (r - 2.3) * (r - 2.3)) + math.exp(-1.4 * (r - 2.0))),
        ("mishin", [0.9, 1.6, 0.05, 1.0, 2.0, 1.3], 0.9 * z ** 2.0 * e_mi * (1.0 + 1.6 * e_mi) + 0.05),
        ("sqrt", [0.8, 2.0], 0.8 * math.sqrt(r / 2.0)),
        ("const", [-7.42], -7.42),
        ("parabola", [1.1, -6.0, 10.0], 1.1 * r * r - 6.0 * r + 10.0),
        ("poly5", [0.3, 1.1, -0.4, 0.2, -0.05],
         0.3 + 0.5 * 1.1 * s2 + (-0.4) * s * s2 + 0.2 * s2 * s2 + (-0.05) * s2 * s2 * s),
        ("stiweb_2", [7.0, 0.6, 4.0, 0.0, 1.2, 3.5],
         (7.0 * r ** -4.0 - 0.6 * r ** -0.0) * math.exp(1.2 / (r - 3.5))),
        ("stiweb_3", [1.2, 3.5], math.exp(1.2 / (r - 3.5))),
        ("tersoff", TERSOFF, ref_fc(r, 2.7, 3.0) * pair),
        ("tersoff_mix", [0.9, 1.4], 0.9 * math.exp(-1.4 * r)),
        ("tersoff_mod", TMOD, ref_fc(r, 2.7, 3.0) * pair * corr),
        ("kawamura", [1.2, -0.8, 3.0, 1.1, 0.9, 0.15, 0.12, 2.0, 1.5], kaw),
        ("kawamura_mix", [1.2, -0.8, 3.0, 1.1, 0.9, 0.15, 0.12, 2.0, 1.5, 0.4, 1.3, 2.2],
         kaw + 3.0 * 0.4 * (math.exp(-2.0 * 1.3 * w) - 2.0 * math.exp(-1.3 * w))),
        ("softshell", [1.7, 3.0], (1.7 / r) ** 3.0),
        ("exp_plus", [4.2, 1.1, -0.3], 4.2 * math.exp(-1.1 * r) - 0.3),
        ("strmm", [1.5, -0.5, 0.1, 1.5, 0.2],
         2.0 * 1.5 * math.exp(-(-0.5) / 2.0 * st) - 0.1 * (1.0 + 1.5 * st) * math.exp(-1.5 * st)),
        ("lj_sc", [0.7, 1.9, 1.0], 4.0 * 0.7 * (sr6 * sr6 - sr6) * ref_sc(r, 6.0, 1.0)),
        ("morse_sc", [0.35, 1.4, 2.6, 1.0], (0.35 * (1.0 - e_m) * (1.0 - e_m) - 0.35) * ref_sc(r, 6.0, 1.0)),
        ("exp_decay_sc", [4.2, 1.1, 1.0], 4.2 * math.exp(-1.1 * r) * ref_sc(r, 6.0, 1.0)),
        ("eopp_sc", [15.0, 6.0, 5.0, 3.0, 2.5, 3.0, 1.0], eopp * ref_sc(r, 6.0, 1.0)),
    ]


@pytest.mark.parametrize("r", [1.4, 2.05, 2.9])
def test_every_form_matches_its_reference_formula(r):
    seen = set()
    for name, p, want in reference_values(r):
        got = val(name, p, r, rmax=6.0)
        assert abs(got - want) <= 1e-12 * abs(want) + 1e-300, (name, r, got, want)
        seen.add(name)
    assert seen == set(FORMS), set(FORMS) - seen


# (name, params, rmax, points): the reference's *_FD tests
FD_CASES = [
    ("lj", [1.0, 1.0], 10.0, [1.2, 2.5]),
    ("morse", [1.5, 2.0, 2.0], 10.0, [1.5, 2.5]),
    ("buckingham", [500.0, 0.3, 2.0], 10.0, [1.5, 3.0]),
    ("born", [1000.0, 3.0, 5.0, 2.0, 1.0], 10.0, [1.5, 2.5]),
    ("power_decay", [3.0, 4.0], 10.0, [2.0, 3.0]),
    ("exp_decay", [2.0, 1.5], 10.0, [1.0, 2.5]),
    ("mexp_decay", [1.0, 2.0, 1.5], 10.0, [1.0, 2.5]),
    ("harmonic", [2.0, 2.5], 10.0, [1.5, 3.5]),
    ("universal", [-3.0, 2.0, 1.5, 2.0], 10.0, [1.5, 2.5]),
    ("eopp", [10.0, 6.0, 1.0, 2.0, 2.0, 4.0], 10.0, [1.5, 2.5]),
    ("eopp_exp", [2.0, 1.0, 1.0, 2.0, 0.5, 3.0], 10.0, [1.0, 2.0]),
    ("meopp", [1.0, 1.0, 0.5, 2.0, 1.0, 1.5, 0.3], 10.0, [1.5, 2.5]),
    ("gen_lj", [2.0, 2.5, 12.0, 6.0, 0.0], 10.0, [2.0, 3.0]),
    ("double_morse", [1.0, 2.0, 2.0, 0.5, 1.5, 3.0, 0.1], 10.0, [1.5, 3.0]),
    ("double_exp", [2.0, 1.5, -1.0, 0.8, 0.3], 10.0, [1.0, 3.0]),
    ("mishin", [1.5, -0.5, 2.0, 0.5, 0.3, 1.0], 10.0, [1.0, 2.5]),
    ("sqrt", [2.0, 1.0], 10.0, [1.5, 3.0]),
    ("parabola", [1.0, -2.0, 0.5], 10.0, [1.5, 3.0]),
    ("poly5", [1.0, -0.5, 0.2, -0.1, 0.05], 10.0, [1.5, 2.5]),
    ("stiweb_2", [7.0496, 0.6022, 4.0, 0.0, 1.8, 2.0951], 4.0, [2.3]),
    ("stiweb_3", [2.0951 * 1.2, 3.7712], 4.0, [2.0, 3.0]),
    ("tersoff", TERSOFF, 4.0, [2.4, 2.85]),
    ("tersoff_mix", [1.0, 0.5], 10.0, [1.5, 3.0]),
    ("tersoff_mod", TERSOFF + [0.01, -0.005, 0.002, -0.001, 0.0005], 4.0, [2.4, 2.85]),
    ("kawamura", [1.0, 0.5, 2.0, 0.3, 0.1, 0.05, 0.3, 2.0, 0.01], 10.0, [1.5, 3.0]),
    ("kawamura_mix", [1.0, 0.5, 2.0, 0.3, 0.1, 0.05, 0.3, 2.0, 0.01, 0.5, 0.2, 1.0], 10.0, [1.5, 3.0]),
    ("softshell", [5.0, 8.0], 10.0, [1.5, 2.5]),
    ("exp_plus", [3.0, 2.0, 1.0], 10.0, [1.0, 2.5]),
    ("strmm", [1.5, -0.5, 0.1, 1.5, 0.2], 10.0, [1.0, 2.5]),
    ("lj_sc", [1.0, 1.0, 1.0], 3.0, [1.2, 2.5]),
    ("morse_sc", [1.5, 2.0, 2.0, 1.0], 3.0, [1.5, 2.5]),
    ("exp_decay_sc", [2.0, 1.5, 1.0], 3.0, [1.0, 2.5]),
    ("eopp_sc", [10.0, 6.0, 1.0, 2.0, 2.0, 4.0, 1.0], 3.0, [1.5, 2.5]),
]


@pytest.mark.parametrize("name,p,rmax,points", FD_CASES, ids=[c[0] for c in FD_CASES])
def test_derivative_matches_central_differences(name, p, rmax, points):
    h = 1e-5
    for r in points:
        fd = (val(name, p, r + h, rmax) - val(name, p, r - h, rmax)) / (2 * h)
        an = der(name, p, r, rmax)
        assert abs(an - fd) <= 1e-6 * abs(fd) + 1e-10, (name, r, an, fd)


def test_const_value_and_zero_derivative():
    for r in (1.0, 2.0, 5.0):
        assert val("const", [3.14], r) == 3.14
        assert der("const", [-7.42], r) == 0.0


def test_cutoffs_are_exact_zeros():
    sw = [7.0496, 0.6022, 4.0, 0.0, 1.8, 2.0951]
    assert val("stiweb_2", sw, 4.0) == 0.0 and der("stiweb_2", sw, 4.0) == 0.0
    s3 = [2.0951 * 1.2, 3.7712]
    assert val("stiweb_3", s3, 4.0) == 0.0 and der("stiweb_3", s3, 4.0) == 0.0
    assert val("tersoff", TERSOFF, 3.1) == 0.0 and der("tersoff", TERSOFF, 3.1) == 0.0


def test_tersoff_cutoff_matches_the_piecewise_form():
    def pair(r):
        return 1830.8 * math.exp(-2.4799 * r) - 471.18 * math.exp(-1.7322 * r)
    for r in (1.0, 2.69, 2.7, 2.8, 2.9, 3.0, 3.01, 4.0):
        want = ref_fc(r, 2.7, 3.0) * pair(r)
        assert abs(val("tersoff", TERSOFF, r) - want) <= 1e-12 * abs(want) + 1e-300
    assert val("tersoff", TERSOFF, 3.5) == 0.0 and der("tersoff", TERSOFF, 3.5) == 0.0
    assert val("tersoff", TERSOFF, 2.5) == pair(2.5)


# the reference's ParamDefault values (first entry of each)
DEFAULTS = {
    "lj": [0.1, 2.5], "morse": [0.1, 2.0, 2.5], "buckingham": [1.0, 1.0, 1.0],
    "born": [0.1, 2.0, 3.0, 2.0, 2.5], "power_decay": [1.0, 2.0], "exp_decay": [4.0, 1.0],
    "mexp_decay": [0.1, 0.1, 2.0], "harmonic": [0.1, 2.0], "universal": [1.0, 1.0, 2.0, 0.0],
    "eopp": [15.0, 6.0, 5.0, 3.0, 2.5, 3.0], "eopp_exp": [15.0, 1.0, 5.0, 3.0, 2.5, 3.0],
    "meopp": [15.0, 6.0, 5.0, 3.0, 2.5, 3.0, 0.5], "gen_lj": [0.1, 12.0, 6.0, 2.5, 0.0],
    "double_morse": [0.1, 2.0, 2.5, 0.1, 2.0, 3.0, 0.0], "double_exp": [0.1, 1.0, 2.5, 1.0, 2.5],
    "mishin": [0.1, 1.0, 0.0, 1.0, 2.0, 1.0], "sqrt": [0.1, 2.0], "const": [1.0],
    "parabola": [1.0, 1.0, 1.0], "poly5": [0.0, 0.0, 0.0, 0.0, 0.0],
    "stiweb_2": [1.0, 1.0, 4.0, 0.0, 1.0, 3.0], "stiweb_3": [1.0, 3.0],
    "tersoff": [1000.0, 100.0, 3.0, 1.5, 1e-6, 1.0, 1e5, 20.0, -0.5, 2.7, 3.0],
    "tersoff_mix": [1.0, 1.0],
    "tersoff_mod": [1000.0, 100.0, 3.0, 1.5, 1e-6, 1.0, 1e5, 20.0, -0.5, 2.7, 3.0, 0.0, 0.0, 0.0, 0.0, 0.0],
    "kawamura": [1.0, 1.0, 1.0, 1.0, 1.0, 0.1, 0.1, 1.0, 1.0],
    "kawamura_mix": [1.0, 1.0, 1.0, 1.0, 1.0, 0.1, 0.1, 1.0, 1.0, 0.0, 1.0, 2.5],
    "softshell": [1.0, 2.0], "exp_plus": [4.0, 1.0, 0.0], "strmm": [0.1, 1.0, 0.1, 1.0, 2.5],
    "lj_sc": [0.1, 2.5, 1.0], "morse_sc": [0.1, 2.0, 2.5, 1.0], "exp_decay_sc": [4.0, 1.0, 1.0],
    "eopp_sc": [15.0, 6.0, 5.0, 3.0, 2.5, 3.0, 1.0],
}


def test_defaults_cover_every_form():
    assert set(DEFAULTS) == set(FORMS)
    assert all(len(DEFAULTS[k]) == FORMS[k][1] for k in FORMS)


@pytest.mark.parametrize("name", sorted(DEFAULTS))
@pytest.mark.parametrize("r", [1.7, 2.85])
def test_partials_match_central_differences(name, r):
    """∂v/∂θ, ∂²v/∂r∂θ (1e-5 rel + 1e-8) and ∂²v/∂r² (1e-4 rel + 1e-7) at the
    reference's defaults; the smooth-cutoff forms switch at rmax = 3.2."""
    form = FORMS[name][0]
    p = np.array(DEFAULTS[name], float)
    rmax = 3.2
    out, g, dg = O.form_eval(form, p, r, rmax)
    for i in range(p.size):
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        up, dn = O.form_eval(form, pp, r, rmax)[0], O.form_eval(form, pm, r, rmax)[0]
        fv, fd_ = (up[0] - dn[0]) / (2 * h), (up[1] - dn[1]) / (2 * h)
        assert abs(g[i] - fv) < 1e-5 * abs(fv) + 1e-8, (name, i, g[i], fv)
        assert abs(dg[i] - fd_) < 1e-5 * abs(fd_) + 1e-8, (name, i, dg[i], fd_)
    hh = 1e-5
    fd2 = (O.form_eval(form, p, r + hh, rmax)[0][1] - O.form_eval(form, p, r - hh, rmax)[0][1]) / (2 * hh)
    assert abs(out[2] - fd2) < 1e-4 * abs(fd2) + 1e-7, (name, out[2], fd2)


def test_stiweb_partials_are_zero_past_the_cutoff():
    """Value and derivative are exactly zero past rc; their parameter partials
    are zero as well (the derivative of the zero function)."""
    out, g, dg = O.form_eval(FORMS["stiweb_2"][0], np.array([7.0, 0.6, 4.0, 0.0, 1.2, 3.5]), 3.6)
    assert out[0] == 0.0 and np.all(g == 0.0) and np.all(dg == 0.0)
