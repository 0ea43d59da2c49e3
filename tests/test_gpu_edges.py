"""Edge cases on the GPU against the FP64 oracle: empty centre lists and
empty structures inside a batch (ragged batches), large l_max (9 with
n_max 10, and 10-12, the largest the library is built for), Cartesian
centres on and off atoms, periodic geometries, and the Jacobian's
max_pairs hint at the C ABI."""
import numpy as np
import pytest
import torch

from oracle.soap_oracle import OracleSOAP, rel_l2
from cusoap_b200 import workloads as W

pytestmark = pytest.mark.gpu

DESC_TOL = 1e-5
DERIV_TOL = 1e-4


def _row_err(a, b):
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    b = np.asarray(b, np.float64).reshape(b.shape[0], -1)
    nb = np.linalg.norm(b, axis=1)
    return float(np.max(np.linalg.norm(a - b, axis=1) / np.where(nb > 0, nb, 1.0)))


def test_empty_centres_and_empty_structure_in_a_batch():
    from cusoap_b200 import SOAP
    P = dict(W.CONFIGS["cluster192"])
    s = SOAP(**P)
    o = OracleSOAP(**P)
    sysd = W.water_cluster(2, 2, 2, seed=1)
    out = s.create(sysd, centers=[])
    assert tuple(out.shape) == (0, s.get_number_of_features())
    empty = {"positions": np.zeros((0, 3)), "atomic_numbers": np.zeros(0, dtype=np.int64)}
    one = {"positions": np.zeros((1, 3)), "atomic_numbers": np.array([8])}
    outs = s.create([sysd, empty, one, sysd])
    assert isinstance(outs, list) and [int(x.shape[0]) for x in outs] == [24, 0, 1, 24]
    ref = o.create(sysd["positions"], sysd["atomic_numbers"])
    assert _row_err(outs[0].cpu().numpy(), ref) < DESC_TOL
    assert torch.equal(outs[0], outs[3])
    assert _row_err(outs[2].cpu().numpy(), o.create(one["positions"], one["atomic_numbers"])) < DESC_TOL


@pytest.mark.parametrize("n_max,l_max,periodic", [(10, 9, False), (8, 10, False), (6, 12, False), (5, 12, True)])
def test_large_l_max_create_derivatives_forces(n_max, l_max, periodic):
    """l_max 9 (the largest of the lanes-grouped-by-l launch shapes with
    n_max up to 16) and l_max 10-12 (one launch shape, n_max <= 8): create,
    the closed-form Jacobian and adjoint forces against the FP64 oracle."""
    from cusoap_b200 import SOAP
    P = dict(species=[1, 8], r_cut=4.0, n_max=n_max, l_max=l_max, sigma=0.5, periodic=periodic)
    s = SOAP(**P)
    o = OracleSOAP(**P)
    sysd = W.water_cluster(2, 2, 2, seed=6)
    if periodic:
        sysd = dict(sysd, cell=np.eye(3) * 7.2, pbc=[True, True, True])
    pos, Z = sysd["positions"], sysd["atomic_numbers"]
    cell, pbc = sysd.get("cell"), sysd.get("pbc")
    assert _row_err(s.create(sysd).cpu().numpy(), o.create(pos, Z, cell=cell, pbc=pbc)) < DESC_TOL
    if not periodic:  # the oracle's closed-form Jacobian is the non-periodic one (SG:2270-2626)
        J = s.derivatives(sysd, centers=[0, 5], include=list(range(10)), return_descriptor=False)
        Jo = o.derivatives(pos, Z, centers=[0, 5], include=list(range(10)), return_descriptor=False)
        assert _row_err(J.cpu().numpy(), Jo) < DERIV_TOL
    w = np.random.default_rng(0).standard_normal(s.get_number_of_features())
    pt = torch.tensor(pos, device="cuda", requires_grad=True)
    (s.create(dict(sysd, positions=pt)) * torch.tensor(w, dtype=torch.float32, device="cuda")).sum().backward()
    Fo = o.forces(pos, Z, np.tile(w, (len(Z), 1)), cell, pbc)
    assert rel_l2(-pt.grad.cpu().numpy(), Fo) < DERIV_TOL


def test_cartesian_centres_on_and_off_atoms_derivatives():
    from cusoap_b200 import SOAP
    P = dict(W.CONFIGS["cluster192"])
    s = SOAP(**P)
    o = OracleSOAP(**P)
    sysd = W.water_cluster(2, 2, 2, seed=2)
    pos, Z = sysd["positions"], sysd["atomic_numbers"]
    cen = [pos[3].tolist(), [0.5, 0.25, 1.0], 7]
    d = s.create(sysd, centers=cen).cpu().numpy()
    assert _row_err(d, o.create(pos, Z, centers=cen)) < DESC_TOL
    J = s.derivatives(sysd, centers=cen, return_descriptor=False).cpu().numpy()
    Jo = o.derivatives(pos, Z, centers=cen, return_descriptor=False)
    assert _row_err(J, Jo) < DERIV_TOL


def _periodic_case(kind, seed=0):
    rng = np.random.default_rng(seed)
    if kind == "triclinic":
        cell = np.array([[9.0, 0.0, 0.0], [3.1, 8.2, 0.0], [-2.4, 1.7, 8.8]])
        pbc = [True, True, True]
    elif kind == "mixed_pbc":
        cell = np.array([[10.0, 0.0, 0.0], [0.0, 11.0, 0.0], [0.0, 0.0, 30.0]])
        pbc = [True, True, False]
    elif kind == "tiny_cell":
        cell = np.array([[3.3, 0.0, 0.0], [0.4, 3.1, 0.0], [0.0, 0.6, 3.5]])
        pbc = [True, True, True]
    elif kind == "rect_x_below":  # x side 4.5 A < 0.75 x the 6.36 A cutoff: the full-window path
        cell = np.diag([4.5, 7.0, 9.0])
        pbc = [True, True, True]
    elif kind == "rect_x_above":  # x side 5.0 A: the sphere-trimmed path with 3 bins on x
        cell = np.diag([5.0, 7.0, 9.0])
        pbc = [True, True, True]
    elif kind == "rect_unwrapped":  # rectangular, atoms spread over several cell images
        cell = np.diag([8.0, 9.5, 11.0])
        pbc = [True, True, True]
    else:  # unwrapped: atoms spread over several cell images
        cell = np.array([[8.5, 0.0, 0.0], [0.0, 9.5, 0.0], [1.0, 0.0, 9.0]])
        pbc = [True, True, True]
    n = 4 if kind == "tiny_cell" else (12 if kind.startswith("rect_x") else 40)
    frac = rng.uniform(0.0, 1.0, size=(n, 3))
    if kind in ("unwrapped", "rect_unwrapped"):
        frac += rng.integers(-2, 3, size=(n, 3))
    if kind == "mixed_pbc":
        frac[:, 2] = rng.uniform(0.3, 0.5, size=n)
    pos = frac @ cell
    Z = rng.choice([1, 8], size=n)
    return {"positions": pos, "atomic_numbers": Z, "cell": cell, "pbc": pbc}


@pytest.mark.parametrize("kind", ["triclinic", "mixed_pbc", "tiny_cell", "unwrapped", "rect_x_below",
                                  "rect_x_above", "rect_unwrapped"])
def test_periodic_geometries_vs_oracle(kind):
    """create and the adjoint forces on periodic geometries the workloads do
    not cover, against the oracle's brute-force image sums.  Rectangular
    cells take the sphere-trimmed neighbour enumeration unless the periodic x
    side is under 0.75 cutoff (then the full window): both sides of that
    threshold are here."""
    from cusoap_b200 import SOAP
    P = dict(species=[1, 8], r_cut=4.5, n_max=4, l_max=3, sigma=0.5, periodic=True)
    s = SOAP(**P)
    o = OracleSOAP(**P)
    sysd = _periodic_case(kind)
    pos, Z, cell, pbc = sysd["positions"], sysd["atomic_numbers"], sysd["cell"], sysd["pbc"]
    d = s.create(sysd).cpu().numpy()
    assert _row_err(d, o.create(pos, Z, cell=cell, pbc=pbc)) < DESC_TOL
    w = np.random.default_rng(1).standard_normal(s.get_number_of_features())
    pt = torch.tensor(pos, device="cuda", requires_grad=True)
    (s.create(dict(sysd, positions=pt)) * torch.tensor(w, dtype=torch.float32, device="cuda")).sum().backward()
    Fo = o.forces(pos, Z, np.tile(w, (len(Z), 1)), cell, pbc)
    assert rel_l2(-pt.grad.cpu().numpy(), Fo) < DERIV_TOL


def test_create_from_extended_xyz(tmp_path):
    """A periodic structure written as extended XYZ and read back with
    read_xyz gives exactly the descriptors of the in-memory structure."""
    from cusoap_b200 import SOAP, read_xyz
    P = dict(species=[1, 8], r_cut=4.5, n_max=4, l_max=3, sigma=0.5, periodic=True)
    s = SOAP(**P)
    sysd = _periodic_case("mixed_pbc", seed=4)
    cell = sysd["cell"]
    lat = " ".join(repr(float(v)) for v in np.asarray(cell).ravel())
    pbc = " ".join("T" if p else "F" for p in sysd["pbc"])
    lines = [str(len(sysd["atomic_numbers"])), f'Lattice="{lat}" pbc="{pbc}"']
    sym = {1: "H", 8: "O"}
    lines += [f"{sym[int(z)]} {x!r} {y!r} {w!r}" for z, (x, y, w) in zip(sysd["atomic_numbers"], sysd["positions"].tolist())]
    path = tmp_path / "cell.xyz"
    path.write_text("\n".join(lines) + "\n")
    frame = read_xyz(str(path), index=0)
    assert torch.equal(s.create(frame), s.create(sysd))


def test_jacobian_max_pairs_hint_at_the_c_abi():
    """soapb_jacobian's max_pairs only sizes the shared-memory sort of a
    centre's entries: with the exact count (what SOAP.derivatives passes) the
    result matches derivatives(); with a hint below the true count the
    crowded centres take the tiled merge path and the result is the same,
    bit for bit (distinct keys sort the same way); the status word stays 0."""
    import ctypes
    from cusoap_b200 import SOAP, _lib
    from cusoap_b200.soap import _Batch, _Pairs, _ptr, _stream
    s = SOAP(**W.CONFIGS["cluster192"])
    sysd = W.water_cluster(3, 3, 3, seed=3)  # 81 atoms; the most crowded centres have 81 pairs
    lib = _lib.load()
    with torch.cuda.device(s.device):
        batch = _Batch(s, [sysd], [None])
        pairs = _Pairs(s, batch, _lib.NL_ALL)
        _, coeff = s._run_descriptor(batch, pairs, _lib.OUT_PS, want_coeff=True)
        n, F = batch.n_atoms, s.get_number_of_features()
        inc_row = torch.arange(n, dtype=torch.int32, device=s.device)
        ws = ctypes.c_int64(0)
        _lib.check(lib.soapb_jacobian_workspace(ctypes.byref(s._basis), batch.n_centres, pairs.total, n, 0,
                                                ctypes.byref(ws)))
        work = torch.empty(max(int(ws.value), 256), dtype=torch.uint8, device=s.device)

        def run(max_pairs):
            out = torch.empty((batch.n_centres, n, 3, F), dtype=torch.float32, device=s.device)
            status = torch.zeros(1, dtype=torch.int32, device=s.device)
            _lib.check(lib.soapb_jacobian(ctypes.byref(s._basis), batch.n_centres, _ptr(pairs.pair_off),
                                          _ptr(pairs.pairs), pairs.total, _ptr(coeff), _ptr(inc_row), n,
                                          _ptr(batch.centre_attach), 0, max_pairs, _lib.OUT_PS, _ptr(out),
                                          _ptr(work), work.numel(), _ptr(status), _stream(s.device)))
            return out, int(status.item())

        exact, flag = run(pairs.max_pairs)
        assert flag == 0
        assert torch.equal(exact, s.derivatives(sysd, return_descriptor=False))
        assert pairs.max_pairs > 64  # the kernel's smallest staging capacity is 64 entries
        small, flag = run(32)
        assert flag == 0
        assert torch.equal(small, exact)
