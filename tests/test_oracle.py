"""Pin the FP64 oracle against golden fixtures produced by the reference itself
(tests/golden/make_golden.py), plus identities of the restated math."""
import math

import numpy as np
import pytest

from oracle.soap_oracle import OracleSOAP, rel_l2, solid_harmonics, gto_basis, pbc_offsets
from cusoap_b200 import workloads as W

TOL = 1e-10


def _cfg(name, **over):
    P = dict(W.CONFIGS[name])
    P.update(over)
    return OracleSOAP(**P)


def test_basis_matches_reference(golden):
    g = golden("cluster192")
    a, b = gto_basis(5.0, 4, 3)
    assert np.allclose(a, g["alphas"], rtol=1e-14, atol=0)
    assert rel_l2(b, g["betas"]) < 1e-11
    g3 = golden("cells_small")
    a, b = gto_basis(6.0, 8, 6)
    # S has condition ~1e6 at n_max=8: two FP64 eigensolvers agree to ~1e-9
    assert rel_l2(b, g3["betas"]) < 1e-8


@pytest.mark.parametrize("avg", ["off", "inner", "outer", "cc"])
def test_create_cluster192(golden, avg):
    g = golden("cluster192")
    o = _cfg("cluster192", average=avg)
    d = o.create(g["positions"], g["Z"])
    assert d.shape == g[f"create_{avg}"].shape
    assert rel_l2(d, g[f"create_{avg}"]) < TOL


def test_inner_outer_identical_to_off(golden):
    g = golden("cluster192")
    assert np.array_equal(g["create_inner"], g["create_off"])
    assert np.array_equal(g["create_outer"], g["create_off"])


def test_cartesian_centres_and_nocrossover(golden):
    g = golden("cluster192")
    o = _cfg("cluster192")
    cart = [list(map(float, c)) for c in g["cart_centers"]]
    assert rel_l2(o.create(g["positions"], g["Z"], centers=cart), g["create_cart"]) < TOL
    onx = _cfg("cluster192", crossover=False)
    assert rel_l2(onx.create(g["positions"], g["Z"]), g["create_nocross"]) < TOL


def test_feature_bookkeeping(golden):
    g = golden("cluster192")
    o = _cfg("cluster192")
    assert o.n_features() == int(g["n_features_off"])
    for key, pair in (("loc_1_1", (1, 1)), ("loc_1_8", (1, 8)), ("loc_8_8", (8, 8))):
        sl = o.get_location(pair)
        assert [sl.start, sl.stop] == list(g[key])


@pytest.mark.parametrize("avg", ["off", "cc"])
def test_derivatives_cluster192(golden, avg):
    g = golden("cluster192")
    o = _cfg("cluster192", average=avg)
    J, D = o.derivatives(g["positions"], g["Z"], centers=[int(c) for c in g["centers"]],
                         include=[int(i) for i in g["include"]])
    assert rel_l2(J, g[f"deriv_{avg}"]) < TOL
    if avg == "off":
        assert rel_l2(D, g["deriv_off_desc"]) < TOL


def test_derivatives_vs_reference_finite_differences(golden):
    g = golden("cluster192")
    o = _cfg("cluster192")
    J = o.derivatives(g["positions"], g["Z"], centers=[7], include=list(range(12)), return_descriptor=False)
    assert rel_l2(J, g["deriv_fd"]) < 1e-7


def test_periodic_cells(golden):
    g = golden("cells_small")
    for avg in ("off", "inner"):
        o = _cfg("cells512", average=avg)
        for k in range(2):
            d = o.create(g[f"pos{k}"], g[f"Z{k}"], centers=[0, 1, 2], cell=g[f"cell{k}"], pbc=[True] * 3)
            ref = g[f"create{k}"] if avg == "off" else g[f"inner{k}"]
            assert rel_l2(d, ref) < 1e-9


def test_forces_vs_reference_autograd(golden):
    g = golden("waterbox_small")
    o = _cfg("waterbox2001")
    A = g["positions"].shape[0]
    dEdp = np.tile(g["w"], (A, 1))
    F = o.forces(g["positions"], g["Z"], dEdp, cell=g["cell"], pbc=[True] * 3, attach=True)
    assert rel_l2(F, g["forces"]) < 1e-9
    d = o.create(g["positions"], g["Z"], cell=g["cell"], pbc=[True] * 3)
    assert rel_l2(d, g["desc"]) < 1e-10
    # the reference's analytical (autograd, attach=True) Jacobian of two centres
    for k, c in enumerate(g["centers_J"]):
        sel = np.zeros((A, 1))
        sel[int(c)] = 1.0
        Fc = o.forces(g["positions"], g["Z"], sel * g["w"][None], cell=g["cell"], pbc=[True] * 3, attach=True)
        assert rel_l2(-Fc, g["wJ"][k]) < 1e-9


def test_forces_vs_central_differences():
    s = W.water_box(4, 5.0, seed=3, dmin=2.4)
    o = OracleSOAP(species=[1, 8], r_cut=3.0, n_max=3, l_max=3, sigma=0.7, periodic=True)
    rng = np.random.default_rng(1)
    w = rng.standard_normal(o.n_features())
    A = s["positions"].shape[0]
    F = o.forces(s["positions"], s["atomic_numbers"], np.tile(w, (A, 1)), cell=s["cell"], pbc=[True] * 3)
    h = 1e-4
    Ffd = np.zeros_like(F)
    for a in range(A):
        for d in range(3):
            pp = s["positions"].copy(); pp[a, d] += h
            pm = s["positions"].copy(); pm[a, d] -= h
            ep = (o.create(pp, s["atomic_numbers"], cell=s["cell"], pbc=[True] * 3) * w).sum()
            em = (o.create(pm, s["atomic_numbers"], cell=s["cell"], pbc=[True] * 3) * w).sum()
            Ffd[a, d] = -(ep - em) / (2 * h)
    assert rel_l2(F, Ffd) < 1e-6


def test_solid_harmonics_convention():
    """Against scipy's complex harmonics: orthonormal real form, no Condon-Shortley phase."""
    from scipy.special import sph_harm_y
    rng = np.random.default_rng(0)
    xyz = rng.standard_normal((50, 3))
    L = 6
    R = solid_harmonics(xyz, L)
    r = np.linalg.norm(xyz, axis=1)
    th = np.arccos(xyz[:, 2] / r)
    ph = np.arctan2(xyz[:, 1], xyz[:, 0])
    for l in range(L + 1):
        for m in range(-l, l + 1):
            Yc = sph_harm_y(l, abs(m), th, ph)
            cs = (-1) ** abs(m)  # scipy includes the Condon-Shortley phase
            if m == 0:
                v = Yc.real
            elif m > 0:
                v = math.sqrt(2) * cs * Yc.real
            else:
                v = math.sqrt(2) * cs * Yc.imag
            assert np.allclose(R[:, l * l + l + m], v * r ** l, atol=1e-12, rtol=1e-10)
    # l = 1 is (y, z, x) * sqrt(3/4pi)
    assert np.allclose(R[:, 1:4], math.sqrt(3 / (4 * math.pi)) * xyz[:, [1, 2, 0]])


def test_solid_harmonic_gradients_fd():
    rng = np.random.default_rng(2)
    xyz = rng.standard_normal((20, 3))
    R, dR = solid_harmonics(xyz, 7, gradients=True)
    h = 1e-6
    for d in range(3):
        e = np.zeros(3); e[d] = h
        fd = (solid_harmonics(xyz + e, 7) - solid_harmonics(xyz - e, 7)) / (2 * h)
        assert np.allclose(dR[:, d], fd, atol=1e-7, rtol=1e-6)
    # exact at the origin: only l = 1 has a nonzero gradient
    R0, dR0 = solid_harmonics(np.zeros((1, 3)), 4, gradients=True)
    assert R0[0, 0] == pytest.approx(1 / math.sqrt(4 * math.pi))
    assert np.count_nonzero(np.abs(dR0) > 0) == 3


def test_pbc_offsets_cover_cutoff():
    cell = np.eye(3) * 4.3
    off = pbc_offsets(cell, [True, True, True], 7.487)
    assert off.shape == (125, 3)
    off = pbc_offsets(cell, [True, False, True], 7.487)
    assert off.shape == (25, 3)


# ---- polynomial radial basis and weighting functions (golden group G4) ----

POLY_W_CASES = {
    "poly": {"rbf": "polynomial"},
    "w_pow": {"weighting": {"function": "pow", "r0": 2.0, "c": 1.0, "d": 1.0, "m": 1.0, "w0": 0.5}},
    "w_poly": {"weighting": {"function": "poly", "r0": 4.0, "c": 1.0, "m": 2.0}},
    "w_exp": {"weighting": {"function": "exp", "r0": 1.5, "c": 1.0, "d": 0.5}},
    "w_w0": {"weighting": {"w0": 0.0}},
    "poly_w_pow": {"rbf": "polynomial", "weighting": {"function": "pow", "r0": 2.0, "c": 1.0, "d": 1.0, "m": 2.0}},
}


@pytest.mark.parametrize("name", list(POLY_W_CASES))
def test_poly_and_weighting_match_reference(golden, name):
    """create (ps and cc) and the analytical derivatives; with weighting the
    reference differentiates by autograd, the oracle in closed form."""
    g = golden("poly_weighting")
    extra = POLY_W_CASES[name]
    pos, Z = g["positions"], g["Z"]
    o = _cfg("cluster192", **extra)
    assert rel_l2(o.create(pos, Z)[:48], g[f"{name}_create"]) < TOL
    assert rel_l2(_cfg("cluster192", average="cc", **extra).create(pos, Z)[:48], g[f"{name}_cc"]) < TOL
    J = o.derivatives(pos, Z, centers=list(g["centers"]), include=list(g["include"]), return_descriptor=False)
    assert rel_l2(J, g[f"{name}_deriv"]) < TOL


def test_rcut_inferred_from_weighting(golden):
    g = golden("poly_weighting")
    P = {k: v for k, v in W.CONFIGS["cluster192"].items() if k != "r_cut"}
    o = OracleSOAP(**P, r_cut=None,
                   weighting={"function": "pow", "r0": 0.5, "c": 1.0, "d": 1.0, "m": 2.0, "threshold": 1e-2})
    assert abs(o.r_cut - float(g["infer_rcut"])) < 1e-12
    assert rel_l2(o.create(g["positions"], g["Z"])[:48], g["infer_create"]) < TOL


def test_poly_basis_periodic_box(golden):
    g = golden("poly_box")
    o = OracleSOAP(species=[1, 8], r_cut=5.0, n_max=6, l_max=6, sigma=1.0, rbf="polynomial", periodic=True)
    d = o.create(g["positions"], g["Z"], centers=[0, 1, 2, 3], cell=g["cell"], pbc=[True] * 3)
    assert rel_l2(d, g["create"]) < 1e-10


def test_weighting_derivative_is_the_slope():
    """The closed-form dw/dr equals a central difference of w(r)."""
    from oracle.soap_oracle import Weighting
    r = np.linspace(0.3, 6.0, 57)
    for kw in ({"function": "pow", "r0": 2.0, "c": 1.0, "d": 1.0, "m": 1.5},
               {"function": "poly", "r0": 4.5, "c": 2.0, "m": 3.0},
               {"function": "exp", "r0": 1.5, "c": 1.0, "d": 0.5}):
        w = Weighting(**kw)
        _, dw = w.value_and_derivative(r)
        h = 1e-6
        fd = (w.value_and_derivative(r + h)[0] - w.value_and_derivative(r - h)[0]) / (2 * h)
        assert np.allclose(dw, fd, rtol=1e-6, atol=1e-9), kw
