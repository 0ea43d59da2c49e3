"""The timed CPU port of the reference path (oracle/reference_port.py)
against the reference's own fixtures and the FP64 oracle: it is both the
reference arm of the benchmark and a checker, so it must agree to float64
round-off (1e-10 relative)."""
import numpy as np
import torch

from cusoap_b200 import workloads as W
from oracle.reference_port import ReferencePort
from oracle.soap_oracle import OracleSOAP, rel_l2


def test_port_matches_reference_fixtures(golden):
    g = golden("cluster192")
    port = ReferencePort(**W.CONFIGS["cluster192"], out_dtype=torch.float64)
    d = port.create(g["positions"], g["Z"]).numpy()
    assert rel_l2(d, g["create_off"]) < 1e-10
    cen = [int(c) for c in g["centers"]]
    inc = [int(i) for i in g["include"]]
    J = port.derivatives(g["positions"], g["Z"], cen).numpy()[:, inc]
    assert rel_l2(J, g["deriv_off"]) < 1e-10


def test_port_matches_oracle_on_a_centre_batch():
    s = W.water_cluster(4, 4, 3, seed=7)
    P = dict(W.CONFIGS["cluster3000"])
    port = ReferencePort(**P, out_dtype=torch.float64)
    o = OracleSOAP(**P)
    cen = list(range(10, 30))
    assert rel_l2(port.create(s["positions"], s["atomic_numbers"], cen).numpy(),
                  o.create(s["positions"], s["atomic_numbers"], centers=cen)) < 1e-10
    Jp = port.derivatives(s["positions"], s["atomic_numbers"], cen).numpy()
    Jo = o.derivatives(s["positions"], s["atomic_numbers"], centers=cen, return_descriptor=False)
    assert rel_l2(Jp, Jo) < 1e-10
    # float32 output, as the reference's default dtype
    p32 = ReferencePort(**P)
    assert p32.derivatives(s["positions"], s["atomic_numbers"], cen[:2]).dtype == torch.float32
    assert np.allclose(p32.create(s["positions"], s["atomic_numbers"], cen).numpy(),
                       port.create(s["positions"], s["atomic_numbers"], cen).numpy(), rtol=1e-6, atol=0)
