"""GPU parity of the polynomial radial basis and the DScribe weighting
functions against the reference's golden fixtures and the FP64 oracle.
Tolerances as in test_gpu_parity: relative L2 per descriptor row 1e-5, per
centre's Jacobian block and for forces 1e-4."""
import numpy as np
import pytest
import torch

from oracle.soap_oracle import OracleSOAP, rel_l2
from cusoap_b200 import workloads as W

pytestmark = pytest.mark.gpu

DESC_TOL = 1e-5
DERIV_TOL = 1e-4

CASES = {
    "poly": {"rbf": "polynomial"},
    "w_pow": {"weighting": {"function": "pow", "r0": 2.0, "c": 1.0, "d": 1.0, "m": 1.0, "w0": 0.5}},
    "w_poly": {"weighting": {"function": "poly", "r0": 4.0, "c": 1.0, "m": 2.0}},
    "w_exp": {"weighting": {"function": "exp", "r0": 1.5, "c": 1.0, "d": 0.5}},
    "w_w0": {"weighting": {"w0": 0.0}},
    "poly_w_pow": {"rbf": "polynomial", "weighting": {"function": "pow", "r0": 2.0, "c": 1.0, "d": 1.0, "m": 2.0}},
}


def _row_err(a, b):
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    b = np.asarray(b, np.float64).reshape(b.shape[0], -1)
    nb = np.linalg.norm(b, axis=1)
    return float(np.max(np.linalg.norm(a - b, axis=1) / np.where(nb > 0, nb, 1.0)))


def _soap(**over):
    from cusoap_b200 import SOAP
    return SOAP(**{**W.CONFIGS["cluster192"], **over})


@pytest.mark.parametrize("name", list(CASES))
def test_create_and_derivatives_golden(golden, name):
    g = golden("poly_weighting")
    sysd = {"positions": g["positions"], "atomic_numbers": g["Z"]}
    s = _soap(**CASES[name])
    assert max(s.table_error) < 1e-6
    d = s.create(sysd).cpu().numpy()[:48]
    assert _row_err(d, g[f"{name}_create"]) < DESC_TOL
    c = _soap(average="cc", **CASES[name]).create(sysd).cpu().numpy()[:48]
    assert _row_err(c, g[f"{name}_cc"]) < DESC_TOL
    J = s.derivatives(sysd, centers=list(g["centers"]), include=list(g["include"]), return_descriptor=False)
    assert _row_err(J.cpu().numpy(), g[f"{name}_deriv"]) < DERIV_TOL


@pytest.mark.parametrize("name", ["w_pow", "poly", "w_exp"])
def test_forces_vs_oracle(name):
    """Adjoint forces of E = sum w . p through create() with weighting / the
    polynomial basis, against the oracle's closed-form reverse pass."""
    sysd = W.make("cluster192")
    s = _soap(**CASES[name])
    o = OracleSOAP(**{**W.CONFIGS["cluster192"], **CASES[name]})
    rng = np.random.default_rng(3)
    w = rng.standard_normal(s.get_number_of_features())
    pos = torch.tensor(sysd["positions"], device="cuda", requires_grad=True)
    E = (s.create({"positions": pos, "atomic_numbers": sysd["atomic_numbers"]})
         * torch.tensor(w, dtype=torch.float32, device="cuda")).sum()
    E.backward()
    F = -pos.grad.cpu().numpy()
    Fo = o.forces(sysd["positions"], sysd["atomic_numbers"], np.tile(w, (len(sysd["atomic_numbers"]), 1)))
    assert rel_l2(F, Fo) < DERIV_TOL


def test_rcut_inferred_from_weighting(golden):
    from cusoap_b200 import SOAP
    g = golden("poly_weighting")
    P = {k: v for k, v in W.CONFIGS["cluster192"].items() if k != "r_cut"}
    s = SOAP(**P, r_cut=None, weighting={"function": "pow", "r0": 0.5, "c": 1.0, "d": 1.0, "m": 2.0,
                                         "threshold": 1e-2})
    assert abs(s._r_cut - float(g["infer_rcut"])) < 1e-12
    d = s.create({"positions": g["positions"], "atomic_numbers": g["Z"]}).cpu().numpy()[:48]
    assert _row_err(d, g["infer_create"]) < DESC_TOL


def test_poly_box_golden(golden):
    """n_max 6, l_max 6, sigma 1 polynomial basis on a periodic water box:
    high l at short neighbour distances, where the reference's clamped
    Bessel recurrence and the tables' series evaluation differ most."""
    from cusoap_b200 import SOAP
    g = golden("poly_box")
    s = SOAP(species=[1, 8], r_cut=5.0, n_max=6, l_max=6, sigma=1.0, rbf="polynomial", periodic=True)
    d = s.create({"positions": g["positions"], "atomic_numbers": g["Z"], "cell": g["cell"], "pbc": [True] * 3},
                 centers=[0, 1, 2, 3]).cpu().numpy()
    assert _row_err(d, g["create"]) < DESC_TOL


def test_w0_only_changes_the_self_term(golden):
    """weighting={'w0': 0} removes exactly the centre's own Gaussian: the
    difference to the unweighted descriptor is the self term's contribution."""
    g = golden("poly_weighting")
    sysd = {"positions": g["positions"], "atomic_numbers": g["Z"]}
    d0 = _soap(weighting={"w0": 0.0}).create(sysd).cpu().numpy()
    o = OracleSOAP(**{**W.CONFIGS["cluster192"], "weighting": {"w0": 0.0}})
    assert _row_err(d0, o.create(g["positions"], g["Z"])) < DESC_TOL
    d1 = _soap().create(sysd).cpu().numpy()
    assert rel_l2(d0, d1) > 1e-3  # the self term is not negligible
