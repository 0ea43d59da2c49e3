"""GPU checks of the drop-in API beyond the descriptor kernels: numerical
derivatives against the reference's own float64 central differences,
get_location against the reference's slices, sparse output of a list of
systems, the flat batched output, the float64 notice and the adjoint's
status word.  Tolerances (relative L2 per centre block): 1e-4 for
derivatives."""
import warnings

import numpy as np
import pytest
import torch

from cusoap_b200 import workloads as W

pytestmark = pytest.mark.gpu

DERIV_TOL = 1e-4
# Central differences of float32 descriptors carry about 1e-7 |p| / (2 d) of
# rounding noise; at the default step d = 5e-3 A that is up to ~1e-3 of a
# centre's block when the block holds only neighbour atoms (a block with the
# centre's own atom meets DERIV_TOL).
FD32_TOL = 1e-3


def _soap(name, **over):
    from cusoap_b200 import SOAP
    P = dict(W.CONFIGS[name])
    P.update(over)
    return SOAP(**P)


def _block_err(a, b):
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    b = np.asarray(b, np.float64).reshape(b.shape[0], -1)
    nb = np.linalg.norm(b, axis=1)
    return float(np.max(np.linalg.norm(a - b, axis=1) / np.where(nb > 0, nb, 1.0)))


def test_numerical_derivatives_vs_reference_fd(golden):
    """The reference's float64 central differences (d = 1e-4) of centre 7
    w.r.t. atoms 0..11 of the 192-atom cluster, against this float32 path at
    its default step, and against the closed-form Jacobian."""
    g = golden("cluster192")
    s = _soap("cluster192")
    sysd = {"positions": g["positions"], "atomic_numbers": g["Z"]}
    Jn, D = s.derivatives(sysd, centers=[7], include=list(range(12)), method="numerical")
    assert Jn.shape == g["deriv_fd"].shape
    assert _block_err(Jn.cpu().numpy(), g["deriv_fd"]) < DERIV_TOL
    Ja = s.derivatives(sysd, centers=[7], include=list(range(12)), return_descriptor=False)
    assert _block_err(Jn.cpu().numpy(), Ja.cpu().numpy()) < DERIV_TOL
    assert torch.equal(D, s.create(sysd, centers=[7]))


def _oracle_fd(o, cell, centres, inc, attach, d):
    """float64 central differences of the oracle's descriptor with the
    reference's centre conventions (SG:1933-2003): every centre resolved once
    to a point; with attach an index centre rides on its atom."""
    pos = np.asarray(cell["positions"], np.float64)
    base = [pos[c].copy() if isinstance(c, int) else np.asarray(c, np.float64) for c in centres]
    J = np.zeros((len(centres), len(inc), 3, o.n_features()))
    for ai, a in enumerate(inc):
        for k in range(3):
            outs = []
            for sg in (1.0, -1.0):
                p = pos.copy()
                p[a, k] += sg * d
                cen = [list(p[a]) if (attach and c == a) else list(b) for c, b in zip(centres, base)]
                outs.append(o.create(p, cell["atomic_numbers"], centers=cen, cell=cell["cell"], pbc=cell["pbc"]))
            J[:, ai, k] = (outs[0] - outs[1]) / (2.0 * d)
    return J


def test_numerical_derivatives_attach_periodic_and_cartesian():
    """attach=True moves index centres with their atom; a Cartesian centre
    stays fixed; a periodic cell differentiates through its images.  Checked
    against float64 central differences of the oracle at the same step with
    the same conventions (so a neighbour that crosses a centre's cutoff within
    the step, which makes any difference quotient jump, does so in both), and
    against the closed form where no neighbour crosses."""
    from oracle.soap_oracle import OracleSOAP
    s = _soap("cells512")
    o = OracleSOAP(**W.CONFIGS["cells512"])
    cell = W.random_cells(1, seed=11, a_min=40, a_max=40)[0]
    inc = [0, 3, 5]
    pt = [float(x) for x in np.asarray(cell["positions"][2]) + 0.3]
    for centres, attach in (([0, 5], False), ([0, 5], True), ([pt], False)):
        Jn = s.derivatives(cell, centers=centres, include=inc, method="numerical", attach=attach,
                           return_descriptor=False).cpu().numpy()
        Jo = _oracle_fd(o, cell, centres, inc, attach, s.FD_STEP)
        assert _block_err(Jn, Jo) < FD32_TOL, (centres, attach)
    # fixed centres: one atom moves, no neighbour crosses a cutoff here
    Jn = s.derivatives(cell, centers=[0, 5], include=inc, method="numerical", return_descriptor=False)
    Ja = s.derivatives(cell, centers=[0, 5], include=inc, return_descriptor=False)
    assert _block_err(Jn.cpu().numpy(), Ja.cpu().numpy()) < FD32_TOL


def test_numerical_derivatives_arguments():
    s = _soap("cluster192")
    sysd = W.make("cluster192")
    with pytest.raises(ValueError):
        s.derivatives_numerical(sysd, centers=[0], method="analytical")
    with pytest.raises(ValueError):
        s.derivatives_numerical(sysd, centers=[0], d=0.0)
    J = s.derivatives(sysd, centers=[0, 1], include=[], method="numerical", return_descriptor=False)
    assert J.shape == (2, 0, 3, s.get_number_of_features())
    J = s.derivatives(sysd, centers=[0], include=[0, 1, 2], exclude=[1], method="numerical",
                      return_descriptor=False)
    Ja = s.derivatives(sysd, centers=[0], include=[0, 2], return_descriptor=False)
    assert _block_err(J.cpu().numpy(), Ja.cpu().numpy()) < FD32_TOL


def test_get_location_golden(golden):
    g = golden("cluster192")
    s = _soap("cluster192")
    for (z1, z2), key in (((1, 1), "loc_1_1"), ((1, 8), "loc_1_8"), ((8, 1), "loc_1_8"), ((8, 8), "loc_8_8")):
        loc = s.get_location((z1, z2))
        assert (loc.start, loc.stop) == tuple(int(v) for v in g[key]), (z1, z2)
    assert s.get_location(("H", "O")) == s.get_location((1, 8))
    # the slices tile the feature axis
    spans = sorted((s.get_location(p).start, s.get_location(p).stop) for p in ((1, 1), (1, 8), (8, 8)))
    assert spans[0][0] == 0 and spans[-1][1] == s.get_number_of_features()
    assert all(spans[i][1] == spans[i + 1][0] for i in range(len(spans) - 1))
    with pytest.raises(ValueError):
        s.get_location((1, 6))
    with pytest.raises(ValueError):
        _soap("cluster192", average="cc").get_location((1, 8))


def test_sparse_list_and_flat_output():
    cells = W.random_cells(3, seed=4, a_min=10, a_max=30)
    dense = _soap("cells512")
    sp = _soap("cells512", sparse=True)
    want = dense.create(cells)
    got = sp.create(cells)
    parts = list(got) if isinstance(got, list) else [got[i] for i in range(got.shape[0])]
    assert len(parts) == 3
    for p, w in zip(parts, want):
        assert p.is_sparse
        assert torch.equal(p.to_dense(), w)
    same = [cells[0], cells[0]]
    st = sp.create(same)
    assert st.is_sparse and st.shape[0] == 2
    flat, off = dense.create_flat(cells)
    assert flat.is_contiguous() and off.tolist()[0] == 0 and off.tolist()[-1] == flat.shape[0]
    for i, w in enumerate(want):
        assert torch.equal(flat[off[i]:off[i + 1]], w)
    # differentiable like create
    pos = [torch.tensor(c["positions"], device="cuda", requires_grad=True) for c in cells]
    flat, _ = dense.create_flat([dict(c, positions=p) for c, p in zip(cells, pos)])
    flat.sum().backward()
    assert all(p.grad is not None and torch.isfinite(p.grad).all() for p in pos)


def test_float64_notice_and_values(monkeypatch):
    from cusoap_b200 import soap as soap_mod
    monkeypatch.setattr(soap_mod, "_F64_WARNED", False)
    with pytest.warns(UserWarning, match="float32"):
        s64 = _soap("cluster192", dtype="float64")
    with warnings.catch_warnings():
        warnings.simplefilter("error")
        _soap("cluster192", dtype="float64")  # once per process
    sysd = W.make("cluster192")
    d64 = s64.create(sysd, centers=[0, 1])
    assert d64.dtype == torch.float64
    assert torch.equal(d64, _soap("cluster192").create(sysd, centers=[0, 1]).double())


def test_forces_status_word_is_clear_after_an_adjoint():
    s = _soap("waterbox2001")
    box = W.water_box(8, 6.21, seed=5, dmin=2.4)
    pos = torch.tensor(box["positions"], device="cuda", requires_grad=True)
    s.create(dict(box, positions=pos)).sum().backward()
    assert s.forces_status() == 0
    assert torch.isfinite(pos.grad).all()


def test_bounded_wait_gives_up_and_the_context_stays_usable(golden):
    """The bounded wait behind the adjoint's row copies ends on its own: a block
    waits on a barrier that no copy completes, gives up after about a second and
    reports status 1; the same context then still computes the reference's
    descriptors."""
    import ctypes
    import time
    from cusoap_b200 import _lib
    lib = _lib.load()
    status = torch.full((1,), -1, dtype=torch.int32, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    _lib.check(lib.soapb_check_bounded_wait(ctypes.c_void_p(status.data_ptr()),
                                            ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
    torch.cuda.synchronize()
    waited = time.perf_counter() - t0
    assert int(status.item()) == 1
    assert 0.5 < waited < 30.0
    g = golden("cluster192")
    d = _soap("cluster192").create({"positions": g["positions"], "atomic_numbers": g["Z"]})
    assert _block_err(d.cpu().numpy(), g["create_off"]) < 1e-5


def test_jacobian_beyond_one_shared_memory_tile():
    """A centre with more (row, edge) entries than the Jacobian sorts in one
    shared-memory tile (JACOBIAN_TILE_ENTRIES) is sorted in tiles and merged:
    8232 atoms all within the cutoff of centre 0 give 8232 entries (one
    merge), 16462 with attach=True (two merge passes), and a 4-atom include
    list takes the same path with a single tile.  Checked against the
    oracle's fixed-centre Jacobian; with attach the centre atom's row is the
    fixed row minus the sum of all fixed rows (translation invariance)."""
    from cusoap_b200 import SOAP
    from cusoap_b200.soap import JACOBIAN_TILE_ENTRIES
    from oracle.soap_oracle import OracleSOAP
    sysd = W.water_cluster(14, 14, 14, seed=1)  # 8232 atoms
    A = len(sysd["atomic_numbers"])
    assert A > JACOBIAN_TILE_ENTRIES
    P = dict(species=[1, 8], r_cut=100.0, n_max=2, l_max=1, sigma=0.5)
    s, o = SOAP(**P), OracleSOAP(**P)
    Jo = o.derivatives(sysd["positions"], sysd["atomic_numbers"], centers=[0], return_descriptor=False)
    J = s.derivatives(sysd, centers=[0], return_descriptor=False).cpu().numpy()
    assert _block_err(J, Jo) < DERIV_TOL
    Ja = s.derivatives(sysd, centers=[0], attach=True, return_descriptor=False).cpu().numpy()
    Jao = Jo.copy()
    Jao[0, 0] = Jo[0, 0] - Jo[0].sum(axis=0)
    assert _block_err(Ja, Jao) < DERIV_TOL
    few = [0, 1, 2, 100]
    Jf = s.derivatives(sysd, centers=[0], include=few, return_descriptor=False).cpu().numpy()
    assert _block_err(Jf, Jo[:, few]) < DERIV_TOL
