"""Host-side checks that need no GPU: the C ABI library loads and exports
every symbol the header declares, and the host-only planning function agrees
with the oracle's feature bookkeeping."""
import ctypes
import os
import re

import pytest

from cusoap_b200 import _lib, workloads as W
from oracle.soap_oracle import OracleSOAP

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _header_symbols():
    txt = open(os.path.join(ROOT, "include", "soapb200.h")).read()
    return sorted(set(re.findall(r"^\s*(?:int|int64_t|const char\*)\s+(soapb_\w+)\s*\(", txt, flags=re.M)))


def test_library_exports_every_header_symbol():
    lib = _lib.load()
    syms = _header_symbols()
    assert len(syms) >= 12
    for name in syms:
        assert hasattr(lib, name), name
    assert set(syms) == set(_lib.EXPORTS)
    assert "sm_100a" in _lib.version()


@pytest.mark.parametrize("name", list(W.CONFIGS))
def test_basis_plan_matches_oracle(name):
    P = W.CONFIGS[name]
    lib = _lib.load()
    b = _lib.Basis()
    b.n_max, b.l_max, b.n_species, b.crossover = P["n_max"], P["l_max"], len(P["species"]), 1
    b.r_cut, b.sigma = P["r_cut"], P["sigma"]
    _lib.check(lib.soapb_basis_plan(ctypes.byref(b)))
    o = OracleSOAP(**{k: v for k, v in P.items() if k != "periodic"})
    assert b.n_feat_ps == o.n_power_features()
    assert b.n_feat_cc == len(P["species"]) * P["n_max"] * (P["l_max"] + 1) ** 2
    assert abs(b.cutoff - o.cutoff) < 1e-12
    assert abs(b.eta - o.eta) < 1e-15
    assert b.n_seg * b.seg_width == pytest.approx(b.cutoff)
    assert b.bytes > 0 and b.off_err + 16 <= b.bytes


def test_basis_plan_rejects_bad_sizes():
    lib = _lib.load()
    b = _lib.Basis()
    b.n_max, b.l_max, b.n_species, b.crossover, b.r_cut, b.sigma = 4, 13, 1, 1, 5.0, 0.5
    st = lib.soapb_basis_plan(ctypes.byref(b))
    assert st == _lib.ERR_ARG
    assert "l_max" in lib.soapb_last_error().decode()
    b.l_max, b.n_max = 3, 0
    assert lib.soapb_basis_plan(ctypes.byref(b)) == _lib.ERR_ARG


def test_device_entry_points_validate_before_launch():
    """Null-argument checks run on the host and never touch the device."""
    lib = _lib.load()
    b = _lib.Basis()
    assert lib.soapb_descriptor(ctypes.byref(b), 10, None, None, 0, None, None, None, None) == _lib.ERR_ARG
    assert lib.soapb_forces(ctypes.byref(b), 10, None, None, None, None, 0, None, 1, None, None, 0, None,
                            None) == _lib.ERR_ARG


def test_soap_requires_cuda_device():
    from cusoap_b200 import SOAP
    with pytest.raises(ValueError):
        SOAP(species=[1], r_cut=3.0, n_max=2, l_max=1, device="cpu")


def test_soap_refuses_sizes_beyond_the_kernels_before_device_work():
    """The kernels are built up to n_max 16, l_max 12 (n_max 8 from l_max 10)
    and 16 species; larger requests raise ValueError naming the limit, before
    any CUDA call (this runs without a GPU, and device=None would need one)."""
    from cusoap_b200 import SOAP
    from cusoap_b200.soap import MAX_L_MAX, MAX_N_MAX, MAX_SPECIES
    with pytest.raises(ValueError, match="l_max must be in"):
        SOAP(species=[1, 8], r_cut=5.0, n_max=4, l_max=MAX_L_MAX + 1)
    with pytest.raises(ValueError, match="n_max must be in"):
        SOAP(species=[1, 8], r_cut=5.0, n_max=MAX_N_MAX + 1, l_max=3)
    with pytest.raises(ValueError, match="species"):
        SOAP(species=list(range(1, MAX_SPECIES + 2)), r_cut=5.0, n_max=4, l_max=3)
    with pytest.raises(ValueError, match="l_max >= 10"):
        SOAP(species=[1, 8], r_cut=5.0, n_max=9, l_max=10)
    # the Python limits are the library's
    lib = _lib.load()
    b = _lib.Basis()
    b.n_max, b.l_max, b.n_species, b.crossover, b.r_cut, b.sigma = 8, MAX_L_MAX, MAX_SPECIES, 1, 5.0, 0.5
    assert lib.soapb_basis_plan(ctypes.byref(b)) == _lib.OK
    b.n_max, b.l_max = MAX_N_MAX, 9
    assert lib.soapb_basis_plan(ctypes.byref(b)) == _lib.OK
    b.n_max, b.l_max = 9, 10
    assert lib.soapb_basis_plan(ctypes.byref(b)) == _lib.ERR_ARG
    for field, value in (("n_max", MAX_N_MAX + 1), ("l_max", MAX_L_MAX + 1), ("n_species", MAX_SPECIES + 1)):
        c = _lib.Basis()
        c.n_max, c.l_max, c.n_species, c.crossover, c.r_cut, c.sigma = 4, 3, 2, 1, 5.0, 0.5
        setattr(c, field, value)
        assert lib.soapb_basis_plan(ctypes.byref(c)) == _lib.ERR_ARG, field


def test_read_xyz_plain_and_extended(tmp_path):
    import numpy as np
    from cusoap_b200 import read_xyz
    from cusoap_b200.xyz import atomic_number
    rng = np.random.default_rng(3)
    p1 = rng.uniform(0, 5, size=(3, 3))
    p2 = rng.uniform(0, 9, size=(4, 3))
    text = ["3", "a plain frame"]
    text += [f"{s} {x:.10f} {y:.10f} {z:.10f}" for s, (x, y, z) in zip(["O", "H", "h"], p1)]
    text += ["4", 'Lattice="9.0 0 0 0 9.5 0 0.5 0 10.0" Properties=species:S:1:pos:R:3 pbc="T T F" energy=-1.5']
    text += [f"{s} {x:.10f} {y:.10f} {z:.10f} 0.0" for s, (x, y, z) in zip(["C", "8", "N", "Si"], p2)]
    path = tmp_path / "two.xyz"
    path.write_text("\n".join(text) + "\n")
    frames = read_xyz(str(path))
    assert len(frames) == 2
    a, b = frames
    assert np.allclose(a["positions"], p1) and list(a["atomic_numbers"]) == [8, 1, 1]
    assert "cell" not in a and "pbc" not in a
    assert np.allclose(b["positions"], p2) and list(b["atomic_numbers"]) == [6, 8, 7, 14]
    assert np.allclose(b["cell"], [[9.0, 0, 0], [0, 9.5, 0], [0.5, 0, 10.0]]) and b["pbc"] == [True, True, False]
    last = read_xyz(str(path), index=-1)
    assert list(last["atomic_numbers"]) == [6, 8, 7, 14]
    assert len(read_xyz(str(path), index=slice(0, 1))) == 1
    assert atomic_number("og") == 118 and atomic_number("Fe") == 26
    with pytest.raises(ValueError):
        atomic_number("Xx")
    bad = tmp_path / "bad.xyz"
    bad.write_text("5\ncomment\nH 0 0 0\n")
    with pytest.raises(ValueError):
        read_xyz(str(bad))
