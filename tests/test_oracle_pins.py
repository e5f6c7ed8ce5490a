"""Pins the oracle against the reference's own unit-test known answers.

Each test re-expresses a GoogleTest case of the reference (file:line in the
docstring) against the FP64 CPU restatement, so that the oracle the GPU is
checked against is itself anchored on the reference's behaviour.
"""
import math

import numpy as np
import pytest

from forcesmith_b200.abi import Model, Table, FS_FAMILY_EAM, FS_FAMILY_PAIR, FS_FAMILY_SW, FS_FAMILY_ADP
from forcesmith_b200 import synth
from oracle import api as O
from tests.helpers import cluster, concat

# ---------------------------------------------------------------- splines ---


def test_spline_eval_at_knots():
    """test_spline.cpp:13-21"""
    xs = [0.0, 1.5, 3.0, 5.0, 6.0]
    ys = [2.0, 0.5, 3.0, 1.0, 4.0]
    for x, y in zip(xs, ys):
        assert abs(O.spline_eval(xs, ys, x)[0] - y) < 1e-10


def test_spline_linear_function_exact():
    """test_spline.cpp:23-30"""
    a, b = 3.0, -1.5
    xs = [0.0, 1.0, 2.5, 4.0]
    ys = [b, a + b, 2.5 * a + b, 4.0 * a + b]
    for r in (0.5, 1.75, 3.0):
        assert abs(O.spline_eval(xs, ys, r)[0] - (a * r + b)) < 1e-10


def test_spline_linear_deriv_exact():
    """test_spline.cpp:32-39"""
    s = 2.5
    xs = [0.0, 1.0, 3.0, 5.0]
    ys = [0.0, s, 3 * s, 5 * s]
    for r in (0.5, 2.0, 4.0):
        assert abs(O.spline_eval(xs, ys, r)[1] - s) < 1e-10


def test_spline_deriv_consistent_with_eval():
    """test_spline.cpp:42-50"""
    xs = [0.0, 1.0, 2.0, 3.0, 4.0]
    ys = [0.0, 1.0, 4.0, 9.0, 16.0]
    eps = 1e-5
    for r in (0.5, 1.5, 2.5, 3.5):
        fd = (O.spline_eval(xs, ys, r + eps)[0] - O.spline_eval(xs, ys, r - eps)[0]) / (2 * eps)
        assert abs(O.spline_eval(xs, ys, r)[1] - fd) < 1e-5


def test_spline_boundary_extrapolation():
    """test_spline.cpp:54-64"""
    xs, ys = [1.0, 2.0, 3.0], [5.0, 3.0, 1.0]
    v, d = O.spline_eval(xs, ys, 0.0)[:2]
    assert abs(v - 7.0) < 1e-15 and abs(d + 2.0) < 1e-15
    v, d = O.spline_eval(xs, ys, 4.0)[:2]
    assert abs(v + 1.0) < 1e-15 and abs(d + 2.0) < 1e-15


def test_spline_two_knot_and_construct():
    """test_spline.cpp:73-95"""
    v, d = O.spline_eval([0.0, 1.0], [0.0, 1.0], 0.5)[:2]
    assert abs(v - 0.5) < 1e-15 and abs(d - 1.0) < 1e-15
    assert abs(O.spline_eval([1.0, 2.0, 3.0], [2.0, 0.0, 2.0], 2.0)[0]) < 1e-10


def test_spline_monotone_data():
    """test_spline.cpp:79-87"""
    xs = ys = [0.0, 1.0, 2.0, 3.0]
    for k in range(1, 10):
        r = 0.3 * k
        assert O.spline_eval(xs, ys, r + 0.05)[0] > O.spline_eval(xs, ys, r - 0.05)[0]


@pytest.mark.parametrize("r", [-0.3, 0.0, 0.4, 1.0, 2.7, 3.9999, 5.0, 5.6])
def test_spline_site_cache_matches_eval_cubic(r):
    """test_spline.cpp:101-110 (cached basis vs uncached Hermite, 1e-11)"""
    xs = [0.0, 1.0, 2.0, 3.0, 4.0, 5.0]
    ys = [2.0, 0.5, 3.0, 1.0, 4.0, 2.5]
    out = O.spline_eval(xs, ys, r)
    assert abs(out[2] - out[0]) < 1e-11
    assert abs(out[3] - out[1]) < 1e-11


@pytest.mark.parametrize("r", [0.0, 1.5, 2.5, 4.0])
def test_spline_site_cache_matches_eval_linear(r):
    """test_spline.cpp:113-121"""
    out = O.spline_eval([1.0, 2.0, 3.0], [5.0, 3.0, 1.0], r)
    assert abs(out[2] - out[0]) < 1e-12 and abs(out[3] - out[1]) < 1e-12


def test_spline_interval_search_on_knot():
    """locate_interval (spline.cpp:18-30): a distance exactly on knot k is in
    interval k; the last knot stays in interval n-2."""
    xs = [0.0, 1.0, 2.0, 3.0, 4.0, 5.0]
    ys = [2.0, 0.5, 3.0, 1.0, 4.0, 2.5]
    assert O.spline_eval(xs, ys, 2.0)[5] == 2
    assert O.spline_eval(xs, ys, 2.5)[5] == 2
    assert O.spline_eval(xs, ys, 4.9999)[5] == 4


def test_makima_slopes_match_published_formula():
    """The makima slope formula of spline.cpp:43-103 on an interior knot,
    computed independently here."""
    x = np.array([0.0, 1.0, 2.0, 3.0, 4.0, 5.0, 6.0])
    y = np.array([2.0, 0.5, 3.0, 1.0, 4.0, 2.5, 2.7])
    s = O.spline_slopes(x, y)
    m = np.diff(y) / np.diff(x)
    i = 3
    w1 = abs(m[i + 1] - m[i]) + abs(m[i + 1] + m[i]) / 2
    w2 = abs(m[i - 1] - m[i - 2]) + abs(m[i - 1] + m[i - 2]) / 2
    assert abs(s[i] - (w1 * m[i - 1] + w2 * m[i]) / (w1 + w2)) < 1e-15


def test_spline_knot_gradient_matches_central_difference():
    """∂(value, derivative)/∂(knots) of the makima spline against central
    differences with the reference's h = 1e-5 (fd_jacobian.hpp:12)."""
    x = np.linspace(1.0, 5.0, 9)
    y = np.sin(x) * np.exp(-0.3 * x) + 0.1 * x
    for r in (0.8, 1.0, 1.37, 2.5, 3.999, 4.7, 5.0, 5.3):
        gv, gd, _ = O.spline_grad(x, y, r)
        for k in range(x.size):
            yp, ym = y.copy(), y.copy()
            yp[k] += 1e-5
            ym[k] -= 1e-5
            fv = (O.spline_eval(x, yp, r)[0] - O.spline_eval(x, ym, r)[0]) / 2e-5
            fdd = (O.spline_eval(x, yp, r)[1] - O.spline_eval(x, ym, r)[1]) / 2e-5
            assert abs(gv[k] - fv) < 1e-5 * abs(fv) + 1e-8
            assert abs(gd[k] - fdd) < 1e-5 * abs(fdd) + 1e-8


# ---------------------------------------------------- boundary conditions ---


def test_pbc_volume_and_wrap():
    """test_boundary_conditions.cpp:11-47"""
    box = np.diag([10.0, 10.0, 10.0])
    w, vol, _ = O.pbc(box, [12.0, 0.0, 0.0])
    assert abs(vol - 1000.0) < 1e-10 and abs(w[0] - 2.0) < 1e-10
    w, _, _ = O.pbc(box, [-1.0, 0.0, 0.0])
    assert abs(w[0] - 9.0) < 1e-10
    w1, _, _ = O.pbc(box, [12.5, -3.1, 22.7])
    w2, _, _ = O.pbc(box, w1)
    assert np.linalg.norm(w1 - w2) < 1e-10


def test_pbc_triclinic():
    """test_boundary_conditions.cpp:71-96 (comma-initialised, rows)"""
    box = np.array([[10.0, 5.0, 0.0], [0.0, 8.66, 0.0], [0.0, 0.0, 10.0]])
    w1, vol, inv = O.pbc(box, [11.0, 3.0, -1.0])
    assert vol > 0
    w2, _, _ = O.pbc(box, w1)
    assert np.linalg.norm(w1 - w2) < 1e-10
    assert np.allclose(inv @ box, np.eye(3), atol=1e-14)


# ---------------------------------------------------------- neighbour list ---

def _nl_session(ds, rcut):
    # a model whose max cutoff is rcut (one flat spline on [0, rcut])
    o = O.Oracle()
    o.upload(ds)
    o.set_model(Model(FS_FAMILY_PAIR, 1, [Table.spline(0.0, rcut, np.zeros(4))]))
    return o


def test_neighbor_dimer_in_and_out_of_range():
    """test_neighbor_list.cpp:38-66"""
    o = _nl_session(cluster([[0, 0, 0], [2, 0, 0]], 10.0), 3.0)
    assert list(o.neighbor_counts(2)) == [1, 1]
    j, img, d = o.neighbors()
    assert np.allclose(d[0], [2.0, 0, 0], atol=1e-12)
    o = _nl_session(cluster([[0, 0, 0], [5, 0, 0]], 10.0), 3.0)
    assert list(o.neighbor_counts(2)) == [0, 0]


def test_neighbor_self_not_included():
    """test_neighbor_list.cpp:68-76"""
    o = _nl_session(cluster([[0, 0, 0]], 10.0), 5.0)
    assert list(o.neighbor_counts(1)) == [0]


def test_neighbor_minimum_image():
    """test_neighbor_list.cpp:91-101"""
    o = _nl_session(cluster([[0, 0, 0], [9.5, 0, 0]], 10.0), 1.0)
    assert list(o.neighbor_counts(2)) == [1, 1]
    _, img, d = o.neighbors()
    assert abs(d[0, 0] + 0.5) < 1e-10 and list(img[0]) == [-1, 0, 0]


def _fcc(a, m):
    basis = np.array([[0, 0, 0], [0.5, 0.5, 0], [0.5, 0, 0.5], [0, 0.5, 0.5]]) * a
    pos = [np.array([nx, ny, nz]) * a + b for nx in range(m) for ny in range(m) for nz in range(m)
           for b in basis]
    return cluster(np.array(pos), a * m)


def test_neighbor_fcc_counts_and_distances():
    """test_neighbor_list.cpp:165-206"""
    a = 3.615
    o = _nl_session(_fcc(a, 2), 0.75 * a)
    assert np.all(o.neighbor_counts(32) == 12)
    _, _, d = o.neighbors()
    r = np.linalg.norm(d, axis=1)
    assert np.allclose(r, a / math.sqrt(2.0), atol=1e-10)
    assert np.all(r < 0.75 * a)


def test_neighbor_small_box_multiple_images():
    """build_periodic enumerates every image within the cutoff
    (neighbor_list.cpp:65-90): in a box smaller than 2·rc one j appears at
    several images, and the list is symmetric under (i,j,n) ↔ (j,i,−n)."""
    ds = synth.packing(np.array([32], np.int32), seed=5)
    ds = ds.with_types(np.zeros(32, np.int32))
    o = O.Oracle()
    o.upload(ds)
    o.set_model(Model(FS_FAMILY_PAIR, 1, [Table.spline(0.0, 6.0, np.zeros(4))]))
    j, img, d = o.neighbors()
    cnt = o.neighbor_counts(32)
    i = np.repeat(np.arange(32), cnt)
    keys = set(zip(i.tolist(), j.tolist(), map(tuple, img.tolist())))
    assert all((jj, ii, tuple(-np.array(n))) in keys for ii, jj, n in keys)
    assert len(keys) == len(j)
    pairs = set(zip(i.tolist(), j.tolist()))
    assert len(pairs) < len(j)  # some (i, j) appear at more than one image


# ------------------------------------------------------------------- EAM ---

def _eam_stub(A=1.0, beta=1.0, c=1.0):
    """RepulsivePair A/r¹², ExpDensity e^{−βr}, SqrtEmbedding −c√ρ of
    test_eam_force.cpp:12-48 as analytic forms."""
    return Model(FS_FAMILY_EAM, 1, [
        Table.analytic("power_decay", [A, 12.0], 0.1, 20.0),
        Table.analytic("exp_decay", [1.0, beta], 0.1, 20.0),
        Table.analytic("sqrt", [-c, 1.0], 1e-10, 1e6),
    ])


def _eval(model, ds, w_s=0.0):
    o = O.Oracle()
    o.upload(ds)
    o.set_model(model)
    return o.eval(1.0, w_s)


def _dimer(r, box=100.0):
    return cluster([[0, 0, 0], [r, 0, 0]], box)


def test_eam_newton_and_energy_sign():
    """test_eam_force.cpp:74-97"""
    out = _eval(_eam_stub(), _dimer(2.5))
    assert np.linalg.norm(out["forces"].sum(axis=0)) < 1e-12
    assert np.isfinite(out["energy"][0]) and out["energy"][0] < 0


def test_eam_embedding_energy_closed_form():
    """test_eam_force.cpp:99-131 (ρ = e^{−βr}; E = 2·(−c√ρ))"""
    r, beta, c = 2.5, 1.0, 2.0
    out = _eval(_eam_stub(0.0, beta, c), _dimer(r))
    assert abs(out["energy"][0] - 2.0 * (-c * math.sqrt(math.exp(-beta * r)))) < 1e-10


def test_eam_force_is_minus_energy_gradient():
    """test_eam_force.cpp:146-168"""
    r, dr = 2.5, 1e-5
    m = _eam_stub()
    fx = _eval(m, _dimer(r))["forces"][0, 0]

    def e_at(x):
        ds = _dimer(r)
        ds.pos[0, 0] = x
        return _eval(m, ds)["energy"][0]
    fd = -(e_at(dr / 2) - e_at(-dr / 2)) / dr
    assert abs(fx - fd) < 1e-6 * abs(fx)


def test_eam_stress_symmetric():
    """test_eam_force.cpp:170-181"""
    s = _eval(_eam_stub(), _dimer(2.5))["stress"][0].reshape(3, 3)
    assert np.allclose(s, s.T, atol=1e-14)


def test_eam_clamp_penalty():
    """clamp_embedding (kernels.hpp:19-31): ρ beyond the embedding span adds
    1000·Δ² to the limit row and F is taken at the span end."""
    m = _eam_stub(0.0, 1.0, 1.0)
    m.tables[2] = Table.analytic("sqrt", [-1.0, 1.0], 0.5, 1e6)
    r = 2.5
    out = _eval(m, _dimer(r))
    rho = math.exp(-r)
    assert abs(out["limit"][0] - 2 * 1000.0 * (0.5 - rho) ** 2) < 1e-12
    assert abs(out["energy"][0] - 2 * (-math.sqrt(0.5))) < 1e-12


# -------------------------------------------------------------------- SW ---

SI_RCUT = 1.80 * 2.0951


def _sw_calc(lam=None):
    m = synth.sw_model()
    if lam is not None:
        m.tables[1] = Table.lam([lam])
    return m


def test_sw_dimer_energy_closed_form_and_sign():
    """test_stiweb_force.cpp:112-168"""
    r = 2.35
    out = _eval(_sw_calc(), _dimer(r))
    p = _sw_calc().tables[0].values
    A, B, pp, q, delta, a1 = p[:6]
    v2 = (A * r ** -pp - B * r ** -q) * math.exp(delta / (r - a1))
    assert out["energy"][0] < 0
    assert abs(out["energy"][0] - v2) < 1e-10 * abs(v2)
    assert np.linalg.norm(out["forces"].sum(axis=0)) < 1e-11


def test_sw_beyond_cutoff_zero():
    """test_stiweb_force.cpp:170-179"""
    out = _eval(_sw_calc(), _dimer(SI_RCUT + 0.01))
    assert abs(out["energy"][0]) < 1e-14 and np.linalg.norm(out["forces"][0]) < 1e-14


def _triangle(r):
    return cluster([[0, 0, 0], [r, 0, 0], [r * 0.5, r * math.sqrt(3) / 2, 0]], 100.0)


def _tetra(r):
    s = r / (2 * math.sqrt(2))
    return cluster([[s, s, s], [s, -s, -s], [-s, s, -s], [-s, -s, s]], 100.0)


@pytest.mark.parametrize("make,r", [(_triangle, 2.4), (_tetra, 2.35), (_dimer, 2.35)])
def test_sw_newton_and_fd_force(make, r):
    """test_stiweb_force.cpp:125-136,181-269"""
    m = _sw_calc()
    ds = make(r)
    out = _eval(m, ds)
    assert np.linalg.norm(out["forces"].sum(axis=0)) < 1e-10
    dr = 1e-6
    x0 = ds.pos[0, 0]

    def e_at(x):
        d2 = make(r)
        d2.pos[0, 0] = x
        return _eval(m, d2)["energy"][0]
    fd = -(e_at(x0 + dr / 2) - e_at(x0 - dr / 2)) / dr
    assert abs(out["forces"][0, 0] - fd) < 1e-6 * abs(fd) + 1e-10
    s = out["stress"][0].reshape(3, 3)
    assert np.allclose(s, s.T, atol=1e-12)


def test_sw_tetrahedral_angle_is_minimum():
    """test_stiweb_force.cpp:202-224"""
    r = 2.4
    ct = -1.0 / 3.0
    st = math.sqrt(1 - ct * ct)
    m = _sw_calc(lam=1.0)
    tet = cluster([[0, 0, 0], [r, 0, 0], [r * ct, r * st, 0]], 100.0)
    off = cluster([[0, 0, 0], [r, 0, 0], [r * ct, r * st + 0.05, 0]], 100.0)
    assert _eval(m, tet)["energy"][0] < _eval(m, off)["energy"][0]


def test_sw_lambda_per_triplet_indexing():
    """test_stiweb_force.cpp:300-329: λ[i·npair + slot(j,k)], symmetric in (j,k)."""
    # Binary SW: only the (0; 0,1) triplet strength is nonzero.
    sw = synth.sw_model().tables[0]
    lam = np.zeros(6)
    lam[1] = 10.0  # i=0, slot(0,1)
    m = Model(FS_FAMILY_SW, 2, [sw.copy(), sw.copy(), sw.copy(), Table.lam(lam)])
    r = 2.4
    # 120° at atom 0, so atoms 1 and 2 (r·√3 apart) are outside each other's cutoff
    ds = cluster([[0, 0, 0], [r, 0, 0], [-0.5 * r, r * math.sqrt(3) / 2, 0]], 100.0,
                 types=[0, 0, 1])
    e_on = _eval(m, ds)["energy"][0]
    m2 = Model(FS_FAMILY_SW, 2, [sw.copy(), sw.copy(), sw.copy(), Table.lam(np.zeros(6))])
    e_off = _eval(m2, ds)["energy"][0]
    # central atom 0 with neighbours j=1 (type 0), k=2 (type 1): slot(0,1) → λ=10
    c = -0.5
    h = math.exp(sw.values[6] / (r - sw.values[7]))
    assert abs((e_on - e_off) - h * h * 10.0 * (c + 1 / 3) ** 2) < 1e-12


# ------------------------------------------------------------------- ADP ---

def test_adp_zero_moments_reduce_to_eam():
    """test_adp_force.cpp:116-143"""
    eam = _eam_stub()
    zero = Table.analytic("const", [0.0], 0.0, 20.0)
    adp = Model(FS_FAMILY_ADP, 1, [t.copy() for t in eam.tables] + [zero, zero.copy()])
    a, e = _eval(adp, _dimer(2.5)), _eval(eam, _dimer(2.5))
    assert abs(a["energy"][0] - e["energy"][0]) < 1e-12
    assert np.linalg.norm(a["forces"] - e["forces"]) < 1e-12


def test_adp_newton_and_fd_force():
    """test_adp_force.cpp:104-114,205-226 (ExpDipole e^{−r}, ExpQuadrupole e^{−2r})"""
    eam = _eam_stub()
    m = Model(FS_FAMILY_ADP, 1, [t.copy() for t in eam.tables] +
              [Table.analytic("exp_decay", [1.0, 1.0], 0.1, 20.0),
               Table.analytic("exp_decay", [1.0, 2.0], 0.1, 20.0)])
    ds = cluster([[0, 0, 0], [2.5, 0.1, 0], [0.2, 2.3, 0.4]], 100.0)
    out = _eval(m, ds)
    assert np.linalg.norm(out["forces"].sum(axis=0)) < 1e-11
    dr = 1e-5

    def e_at(x):
        d2 = cluster([[x, 0, 0], [2.5, 0.1, 0], [0.2, 2.3, 0.4]], 100.0)
        return _eval(m, d2)["energy"][0]
    fd = -(e_at(dr / 2) - e_at(-dr / 2)) / dr
    assert abs(out["forces"][0, 0] - fd) < 1e-6 * abs(fd) + 1e-9


# ------------------------------------------------- parameter Jacobians ---

FORM_DEFAULTS = {  # analytic_potential.hpp ParamDefault values
    "lj": [0.1, 2.5], "morse": [0.1, 2.0, 2.5], "exp_decay": [4.0, 1.0], "sqrt": [0.1, 2.0],
    "power_decay": [1.0, 2.0], "mexp_decay": [0.1, 0.1, 2.0], "harmonic": [0.1, 2.0],
    "exp_plus": [4.0, 1.0, 0.0], "parabola": [1.0, 1.0, 1.0], "const": [1.0],
    "buckingham": [1.0, 1.0, 1.0], "born": [0.1, 2.0, 3.0, 2.0, 2.5],
}


@pytest.mark.parametrize("name", sorted(FORM_DEFAULTS))
@pytest.mark.parametrize("r", [1.7, 2.9])
def test_form_partials_match_fd(name, r):
    """test_param_jacobian.cpp:54-100: ∂/∂θ and ∂²/∂r∂θ vs central differences
    (1e-5 rel + 1e-8), ∂²/∂r² (1e-4 rel + 1e-7)."""
    from forcesmith_b200.abi import FORMS
    form = FORMS[name][0]
    p = np.array(FORM_DEFAULTS[name])
    out, g, dg = O.form_eval(form, p, r)
    for i in range(p.size):
        h = 1e-6 * max(1.0, abs(p[i]))
        pp, pm = p.copy(), p.copy()
        pp[i] += h
        pm[i] -= h
        up, dn = O.form_eval(form, pp, r)[0], O.form_eval(form, pm, r)[0]
        fv, fd_ = (up[0] - dn[0]) / (2 * h), (up[1] - dn[1]) / (2 * h)
        assert abs(g[i] - fv) < 1e-5 * abs(fv) + 1e-8
        assert abs(dg[i] - fd_) < 1e-5 * abs(fd_) + 1e-8
    hh = 1e-5
    fd2 = (O.form_eval(form, p, r + hh)[0][1] - O.form_eval(form, p, r - hh)[0][1]) / (2 * hh)
    assert abs(out[2] - fd2) < 1e-4 * abs(fd2) + 1e-7


def _jac_pair(oracle_model, ds, w_e, w_s, tol):
    o = O.Oracle()
    o.upload(ds)
    o.set_model(oracle_model)
    Ja = o.jacobian_analytic(w_e, w_s)
    Jf = o.jacobian_fd(w_e, w_s)
    worst = np.max(np.abs(Ja - Jf) / (1.0 + np.abs(Jf)))
    assert worst < tol, worst


C4 = [[0.0, 0.0, 0.0], [2.55, 0.0, 0.0], [0.3, 2.7, 0.1], [2.2, 2.4, 2.9]]


def test_pair_jacobian_matches_fd():
    """test_param_jacobian.cpp:196-225 (Morse pair, forces and stress rows)"""
    m = Model(FS_FAMILY_PAIR, 1, [Table.analytic("morse", [0.35, 1.4, 2.6], 0.5, 6.0)])
    _jac_pair(m, cluster(C4, 14.0), 0.7, 0.0, 1e-6)
    ds = concat(cluster([[0, 0, 0], [2.55, 0.1, 0], [0.3, 2.7, 0.1]], 11.0),
                cluster([[0, 0, 0], [2.9, 0, 0.4], [1.1, 2.5, 0.2], [2.6, 2.2, 2.7]], 12.0))
    _jac_pair(m, ds, 1.0, 0.4, 1e-6)


def test_binary_pair_jacobian_matches_fd():
    """test_param_jacobian.cpp:313-332"""
    m = Model(FS_FAMILY_PAIR, 2, [Table.analytic("morse", [0.35, 1.4, 2.6], 0.5, 6.0),
                                  Table.analytic("morse", [0.22, 1.7, 2.4], 0.5, 6.0),
                                  Table.analytic("exp_decay", [2.1, 1.05], 0.5, 6.0)])
    ds = cluster(C4, 14.0, types=[0, 1, 0, 1])
    _jac_pair(m, ds, 0.7, 0.3, 1e-6)


def _analytic_eam(nt=1):
    if nt == 1:
        return Model(FS_FAMILY_EAM, 1, [Table.analytic("exp_decay", [2.4, 0.9], 0.5, 6.0),
                                        Table.analytic("exp_decay", [1.1, 1.3], 0.5, 6.0),
                                        Table.analytic("sqrt", [-2.0, 1.0], 0.05, 40.0)])
    return Model(FS_FAMILY_EAM, 2, [Table.analytic("exp_decay", [2.4, 0.9], 0.5, 6.0),
                                    Table.analytic("exp_decay", [2.0, 1.1], 0.5, 6.0),
                                    Table.analytic("exp_decay", [1.7, 1.0], 0.5, 6.0),
                                    Table.analytic("exp_decay", [1.1, 1.3], 0.5, 6.0),
                                    Table.analytic("exp_decay", [0.9, 1.15], 0.5, 6.0),
                                    Table.analytic("sqrt", [-2.0, 1.0], 0.05, 40.0),
                                    Table.analytic("sqrt", [-1.6, 1.0], 0.05, 40.0)])


def test_eam_jacobian_matches_fd():
    """test_param_jacobian.cpp:262-290 (B = 1 in the √ embedding: the
    reference's fixture passes B = 0, for which F(ρ) = A√(ρ/0) is infinite)"""
    _jac_pair(_analytic_eam(), cluster(C4, 14.0), 0.7, 0.0, 1e-5)
    ds = concat(cluster([[0, 0, 0], [2.55, 0.1, 0], [0.3, 2.7, 0.1]], 11.0),
                cluster([[0, 0, 0], [2.9, 0, 0.4], [1.1, 2.5, 0.2], [2.6, 2.2, 2.7]], 12.0))
    _jac_pair(_analytic_eam(), ds, 1.0, 0.4, 1e-5)


def test_binary_eam_jacobian_matches_fd():
    """test_param_jacobian.cpp:334-358"""
    ds = cluster(C4 + [[1.2, 0.9, 2.6]], 13.0, types=[0, 1, 0, 1, 1])
    _jac_pair(_analytic_eam(2), ds, 0.8, 0.25, 1e-5)


def test_spline_eam_jacobian_matches_fd():
    """The analytic knot Jacobian (the GPU's method) against the reference's
    own method for splines — central differences over the full residual
    (forcesmith_functor.cpp:279-286) — on a ternary spline EAM."""
    from tests.helpers import small_ternary, ternary_models
    true, start = ternary_models(nknots=10)
    ds = small_ternary(2, 24, seed=3)
    o = O.Oracle()
    o.upload(ds)
    o.set_model(true)
    out = o.eval(1.0, 0.1)
    ds = ds.with_labels(out["forces"], out["energy"], out["stress"])
    _jac_pair(start, ds, 1.0, 0.1, 1e-5)


def test_spline_pair_jacobian_matches_fd():
    from tests.helpers import spline_pair_model, small_ternary
    ds = small_ternary(2, 24, seed=4)
    ds.type[:] = ds.type % 2
    _jac_pair(spline_pair_model(2), ds, 1.0, 0.2, 1e-5)
