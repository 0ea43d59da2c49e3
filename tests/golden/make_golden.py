"""Generate the golden fixtures in this folder by running the REFERENCE.

The reference (TACC/cuSOAP ``src/cusoap/soap_generator.py``) is pure Python
and needs the third-party ``sphericart.torch``, which is absent here; the
test-only stand-in under ``oracle/sphericart_shim`` supplies it.  Everything
runs on the CPU in float64.  Run from the repository root:

    python tests/golden/make_golden.py /path/to/reference/src

The fixtures are small ``.npz`` files; the tests never need the reference.
"""
from __future__ import annotations

import os
import sys

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))


POLY_W_CASES = {
    # name: extra constructor arguments on top of the 192-atom cluster's parameters
    "poly": {"rbf": "polynomial"},
    "w_pow": {"weighting": {"function": "pow", "r0": 2.0, "c": 1.0, "d": 1.0, "m": 1.0, "w0": 0.5}},
    "w_poly": {"weighting": {"function": "poly", "r0": 4.0, "c": 1.0, "m": 2.0}},
    "w_exp": {"weighting": {"function": "exp", "r0": 1.5, "c": 1.0, "d": 0.5}},
    "w_w0": {"weighting": {"w0": 0.0}},
    "poly_w_pow": {"rbf": "polynomial", "weighting": {"function": "pow", "r0": 2.0, "c": 1.0, "d": 1.0, "m": 2.0}},
}


def main(ref_src: str, groups=("G1", "G2", "G3", "G4")) -> None:
    sys.path.insert(0, os.path.join(ROOT, "oracle", "sphericart_shim"))
    sys.path.insert(0, ref_src)
    sys.path.insert(1, ROOT)
    from cusoap import SOAP  # the reference package
    from cusoap_b200 import workloads as W

    torch.set_default_dtype(torch.float64)

    def ref(**kw):
        return SOAP(dtype="float64", device="cpu", **kw)

    if "G4" in groups:
        make_poly_weighting(ref, W)
    if "G1" not in groups and "G2" not in groups and "G3" not in groups:
        return

    # --- G1: 192-atom water cluster, the CPU workload's parameters --------
    s = W.make("cluster192")
    P = dict(W.CONFIGS["cluster192"])
    centers = [0, 7, 100]
    include = list(range(40))
    out = {"positions": s["positions"], "Z": s["atomic_numbers"], "centers": np.array(centers),
           "include": np.array(include)}
    soap = ref(**P)
    out["create_off"] = soap.create(s).numpy()
    J, D = soap.derivatives(s, centers=centers, include=include, method="analytical")
    out["deriv_off"], out["deriv_off_desc"] = J.numpy(), D.numpy()
    out["alphas"] = soap._alphas.numpy()
    out["betas"] = soap._betas.numpy()
    out["n_features_off"] = np.array(soap.get_number_of_features())
    out["loc_1_1"] = np.array([soap.get_location((1, 1)).start, soap.get_location((1, 1)).stop])
    out["loc_1_8"] = np.array([soap.get_location((1, 8)).start, soap.get_location((1, 8)).stop])
    out["loc_8_8"] = np.array([soap.get_location((8, 8)).start, soap.get_location((8, 8)).stop])
    for avg in ("inner", "outer"):
        out[f"create_{avg}"] = ref(**{**P, "average": avg}).create(s).numpy()
    soap_cc = ref(**{**P, "average": "cc"})
    out["create_cc"] = soap_cc.create(s).numpy()
    Jc, _ = soap_cc.derivatives(s, centers=centers, include=include, method="analytical")
    out["deriv_cc"] = Jc.numpy()
    # Cartesian centres: one on an atom, one off-atom
    cart = [s["positions"][3].tolist(), [1.0, 2.0, 3.0]]
    out["cart_centers"] = np.array(cart)
    out["create_cart"] = soap.create(s, centers=cart).numpy()
    # crossover=False
    soap_nx = ref(**{**P, "crossover": False})
    out["create_nocross"] = soap_nx.create(s).numpy()
    # numerical derivatives (central differences, h = 1e-4) for one centre
    out["deriv_fd"] = soap.derivatives(s, centers=[7], include=list(range(12)), method="numerical",
                                       return_descriptor=False).numpy()
    np.savez_compressed(os.path.join(HERE, "cluster192.npz"), **out)

    # --- G2: two small periodic cells with the batched workload's parameters
    cells = W.random_cells(2, seed=123, a_min=8, a_max=30)
    P3 = dict(W.CONFIGS["cells512"])
    soap3 = ref(**{**P3, "average": "off"})
    soap3i = ref(**P3)  # average="inner"
    out = {}
    for k, c in enumerate(cells):
        out[f"pos{k}"], out[f"Z{k}"], out[f"cell{k}"] = c["positions"], c["atomic_numbers"], c["cell"]
        out[f"create{k}"] = soap3.create(c, centers=[0, 1, 2]).numpy()
        out[f"inner{k}"] = soap3i.create(c, centers=[0, 1, 2]).numpy()
    out["alphas"], out["betas"] = soap3._alphas.numpy(), soap3._betas.numpy()
    np.savez_compressed(os.path.join(HERE, "cells_small.npz"), **out)

    # --- G3: small periodic water box, differentiation workload parameters
    box = W.water_box(8, 6.21, seed=5, dmin=2.4)
    P4 = dict(W.CONFIGS["waterbox2001"])
    soap4 = ref(**P4)
    F = soap4.get_number_of_features()
    rng = np.random.default_rng(7)
    w = rng.standard_normal(F)
    pos = torch.tensor(box["positions"], requires_grad=True)
    sys_t = {"positions": pos, "atomic_numbers": torch.tensor(box["atomic_numbers"]),
             "cell": torch.tensor(box["cell"]), "pbc": torch.tensor(box["pbc"])}
    desc = soap4._evaluate(sys_t, None, None)  # centres = the (differentiable) positions
    E = (desc * torch.tensor(w)[None, :]).sum()
    E.backward()
    out = {"positions": box["positions"], "Z": box["atomic_numbers"], "cell": box["cell"], "w": w,
           "energy": np.array(float(E)), "forces": -pos.grad.numpy(), "desc": desc.detach().numpy()}
    # the reference's own analytical derivatives (autograd, attach=True) for two centres
    J4 = soap4.derivatives(box, centers=[0, 1], method="analytical", attach=True,
                           return_descriptor=False).numpy()
    out["centers_J"] = np.array([0, 1])
    out["wJ"] = np.einsum("cadf,f->cad", J4, w)
    np.savez_compressed(os.path.join(HERE, "waterbox_small.npz"), **out)
    print("golden fixtures written to", HERE)


def make_poly_weighting(ref, W) -> None:
    """G4: polynomial radial basis and weighting functions on the 192-atom
    cluster: create() (off and cc) and the reference's analytical derivatives
    (its closed form for rbf='polynomial', its autograd path with weighting);
    plus r_cut inferred from a weighting and a heavier polynomial basis
    (n_max 6, l_max 6, sigma 1) on a small periodic water box."""
    s = W.make("cluster192")
    P = dict(W.CONFIGS["cluster192"])
    centers, include = [0, 7, 100], list(range(40))
    out = {"positions": s["positions"], "Z": s["atomic_numbers"], "centers": np.array(centers),
           "include": np.array(include)}
    for name, extra in POLY_W_CASES.items():
        soap = ref(**{**P, **extra})
        out[f"{name}_create"] = soap.create(s).numpy()[:48]  # first 48 centres kept (fixture size)
        out[f"{name}_cc"] = ref(**{**P, **extra, "average": "cc"}).create(s).numpy()[:48]
        J = soap.derivatives(s, centers=centers, include=include, method="analytical", return_descriptor=False)
        out[f"{name}_deriv"] = J.numpy()
    # r_cut from the weighting (pow: r0 (c/threshold - d)^(1/m))
    wt = {"function": "pow", "r0": 0.5, "c": 1.0, "d": 1.0, "m": 2.0, "threshold": 1e-2}
    Pn = {k: v for k, v in P.items() if k != "r_cut"}
    soap = ref(**Pn, r_cut=None, weighting=wt)
    out["infer_rcut"] = np.array(soap._r_cut)
    out["infer_create"] = soap.create(s).numpy()[:48]
    np.savez_compressed(os.path.join(HERE, "poly_weighting.npz"), **out)
    # heavier polynomial basis on a small periodic box
    box = W.water_box(8, 6.21, seed=5, dmin=2.4)
    Pb = {"species": [1, 8], "r_cut": 5.0, "n_max": 6, "l_max": 6, "sigma": 1.0, "rbf": "polynomial",
          "periodic": True}
    soap = ref(**Pb)
    sysb = {"positions": box["positions"], "atomic_numbers": box["atomic_numbers"], "cell": box["cell"],
            "pbc": box["pbc"]}
    outb = {"positions": box["positions"], "Z": box["atomic_numbers"], "cell": box["cell"],
            "create": soap.create(sysb, centers=[0, 1, 2, 3]).numpy()}
    np.savez_compressed(os.path.join(HERE, "poly_box.npz"), **outb)


if __name__ == "__main__":
    main(sys.argv[1] if len(sys.argv) > 1 else "/root/reference/src",
         tuple(sys.argv[2:]) if len(sys.argv) > 2 else ("G1", "G2", "G3", "G4"))
