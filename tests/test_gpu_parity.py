"""GPU parity of the CUDA path against the FP64 oracle and the reference's
golden fixtures.  Tolerances (relative L2, per descriptor row / per centre's
Jacobian block, against float64): 1e-5 for descriptors, 1e-4 for
derivatives and forces."""
import numpy as np
import pytest
import torch

from oracle.soap_oracle import OracleSOAP, rel_l2
from cusoap_b200 import workloads as W

pytestmark = pytest.mark.gpu

DESC_TOL = 1e-5
DERIV_TOL = 1e-4


def _soap(name, **over):
    from cusoap_b200 import SOAP
    P = dict(W.CONFIGS[name])
    P.update(over)
    return SOAP(**P)


def _oracle(name, **over):
    P = dict(W.CONFIGS[name])
    P.update(over)
    return OracleSOAP(**P)


def _row_err(a, b):
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    b = np.asarray(b, np.float64).reshape(b.shape[0], -1)
    nb = np.linalg.norm(b, axis=1)
    return float(np.max(np.linalg.norm(a - b, axis=1) / np.where(nb > 0, nb, 1.0)))


def _np(t):
    return t.detach().cpu().numpy()


def test_basis_and_tables():
    s = _soap("cells512")
    o = _oracle("cells512")
    assert rel_l2(s._alphas, o.alphas) < 1e-14
    assert rel_l2(s._betas, o.betas) < 1e-8
    # B and D = d(wB)/dr tables, relative to each function's maximum (the constructor enforces 1e-6)
    assert max(s.table_error) < 5e-7


@pytest.mark.parametrize("avg", ["off", "inner", "outer", "cc"])
def test_create_cluster192_golden(golden, avg):
    g = golden("cluster192")
    s = _soap("cluster192", average=avg)
    d = _np(s.create({"positions": g["positions"], "atomic_numbers": g["Z"]}))
    assert d.shape == g[f"create_{avg}"].shape
    assert _row_err(d, g[f"create_{avg}"]) < DESC_TOL


def test_create_cartesian_centres_and_nocrossover(golden):
    g = golden("cluster192")
    sysd = {"positions": g["positions"], "atomic_numbers": g["Z"]}
    s = _soap("cluster192")
    cart = [list(map(float, c)) for c in g["cart_centers"]]
    assert _row_err(_np(s.create(sysd, centers=cart)), g["create_cart"]) < DESC_TOL
    snx = _soap("cluster192", crossover=False)
    assert _row_err(_np(snx.create(sysd)), g["create_nocross"]) < DESC_TOL
    # index centres given explicitly
    d = _np(s.create(sysd, centers=[5, 0, 17]))
    assert _row_err(d, g["create_off"][[5, 0, 17]]) < DESC_TOL


@pytest.mark.parametrize("avg", ["off", "cc"])
def test_derivatives_cluster192_golden(golden, avg):
    g = golden("cluster192")
    s = _soap("cluster192", average=avg)
    J, D = s.derivatives({"positions": g["positions"], "atomic_numbers": g["Z"]},
                         centers=[int(c) for c in g["centers"]], include=[int(i) for i in g["include"]])
    assert _row_err(_np(J), g[f"deriv_{avg}"]) < DERIV_TOL
    if avg == "off":
        assert _row_err(_np(D), g["deriv_off_desc"]) < DESC_TOL


def test_derivatives_full_cluster192_vs_oracle():
    s = W.make("cluster192")
    gs = _soap("cluster192")
    o = _oracle("cluster192")
    J, D = gs.derivatives(s)
    cen = [0, 1, 50, 191]
    Jo = o.derivatives(s["positions"], s["atomic_numbers"], centers=cen, return_descriptor=False)
    assert _row_err(_np(J[cen]), Jo) < DERIV_TOL
    Do = o.create(s["positions"], s["atomic_numbers"])
    assert _row_err(_np(D), Do) < DESC_TOL
    # attach=True (centre-motion term) on the same variant
    Ja = gs.derivatives(s, centers=[3, 77], attach=True, return_descriptor=False)
    Jf = gs.derivatives(s, centers=[3, 77], attach=False, return_descriptor=False)
    Ja, Jf = _np(Ja).astype(np.float64), _np(Jf).astype(np.float64)
    diff = Ja - Jf
    # attach changes only the centre atom's row: -(sum of every fixed-centre row) ...
    scale = np.abs(Jf[0]).max()
    assert np.abs(np.delete(diff[0], 3, axis=0)).max() <= 1e-6 * scale
    assert np.abs(diff[0, 3] + Jf[0].sum(0)).max() <= 1e-4 * scale
    # ... so with attached centres the rows sum to zero (translation invariance)
    assert np.abs(Ja[1].sum(0)).max() <= 1e-4 * np.abs(Ja[1]).max()


def test_periodic_attach_translation_invariance():
    """Periodic cell, attached centres, every atom included: the Jacobian rows
    of a centre sum to zero (moving every atom moves every centre)."""
    cell = W.random_cells(1, seed=17, a_min=30, a_max=30)[0]
    s = _soap("waterbox2001", species=[1, 6, 7, 8])
    J = _np(s.derivatives(cell, centers=[0, 5, 9], attach=True, return_descriptor=False)).astype(np.float64)
    for k in range(3):
        assert np.abs(J[k].sum(0)).max() <= 1e-4 * np.abs(J[k]).max()


def test_periodic_cells_golden(golden):
    g = golden("cells_small")
    for avg, key in (("off", "create"), ("inner", "inner")):
        s = _soap("cells512", average=avg)
        for k in range(2):
            sysd = {"positions": g[f"pos{k}"], "atomic_numbers": g[f"Z{k}"], "cell": g[f"cell{k}"],
                    "pbc": [True, True, True]}
            d = _np(s.create(sysd, centers=[0, 1, 2]))
            assert _row_err(d, g[f"{key}{k}"]) < DESC_TOL


def test_batched_equals_per_structure():
    cells = W.random_cells(12, seed=3, a_min=8, a_max=60)
    s = _soap("cells512")
    batched = s.create(cells)
    assert isinstance(batched, list)  # uneven sizes -> list, as the reference
    for c, b in zip(cells, batched):
        single = s.create(c)
        assert torch.equal(single, b)
    o = _oracle("cells512")
    for c, b in zip(cells[:4], batched[:4]):
        ref = o.create(c["positions"], c["atomic_numbers"], cell=c["cell"], pbc=c["pbc"])
        assert _row_err(_np(b), ref) < DESC_TOL


def test_forces_autograd_golden(golden):
    g = golden("waterbox_small")
    s = _soap("waterbox2001")
    pos = torch.tensor(g["positions"], dtype=torch.float64, device="cuda", requires_grad=True)
    sysd = {"positions": pos, "atomic_numbers": g["Z"], "cell": g["cell"], "pbc": [True, True, True]}
    d = s.create(sysd)
    assert _row_err(_np(d), g["desc"]) < DESC_TOL
    E = (d.double() * torch.tensor(g["w"], device="cuda")[None, :]).sum()
    E.backward()
    F = -_np(pos.grad)
    assert rel_l2(F, g["forces"]) < DERIV_TOL
    E2, F2 = s.energy_forces(sysd, g["w"])
    assert rel_l2(_np(F2), g["forces"]) < DERIV_TOL
    assert abs(float(E2) - float(g["energy"])) < DESC_TOL * abs(float(g["energy"]))


def test_forces_reference_analytical_two_centres(golden):
    """The reference's own analytical (autograd, attach=True) Jacobian of two
    centres, contracted with w, against the adjoint restricted to them."""
    g = golden("waterbox_small")
    s = _soap("waterbox2001")
    sysd = {"positions": g["positions"], "atomic_numbers": g["Z"], "cell": g["cell"], "pbc": [True, True, True]}
    J = s.derivatives(sysd, centers=[0, 1], attach=True, return_descriptor=False)
    wJ = np.einsum("cadf,f->cad", _np(J).astype(np.float64), g["w"])
    for k in range(2):
        assert rel_l2(wJ[k], g["wJ"][k]) < DERIV_TOL


def test_periodic_derivatives_vs_oracle():
    cell = W.random_cells(1, seed=11, a_min=20, a_max=20)[0]
    s = _soap("cells512")
    o = _oracle("cells512")
    J = s.derivatives(cell, centers=[0, 3], return_descriptor=False)
    # oracle: numerical check through the FP64 forward (fixed centres)
    pos = cell["positions"]
    h = 1e-5
    cen = [pos[0].tolist(), pos[3].tolist()]
    for a in (0, 5):
        for d in range(3):
            pp, pm = pos.copy(), pos.copy()
            pp[a, d] += h
            pm[a, d] -= h
            fd = (o.create(pp, cell["atomic_numbers"], centers=cen, cell=cell["cell"], pbc=cell["pbc"]) -
                  o.create(pm, cell["atomic_numbers"], centers=cen, cell=cell["cell"], pbc=cell["pbc"])) / (2 * h)
            got = _np(J[:, a, d, :])
            # Cartesian centres on an atom keep their self term fixed; a = 0 is the first centre's atom
            assert rel_l2(got, fd) < 1e-4


def test_single_atom_and_dimer():
    from cusoap_b200 import SOAP
    o = OracleSOAP(species=[1, 8], r_cut=4.0, n_max=3, l_max=2, sigma=0.5)
    s = SOAP(species=[1, 8], r_cut=4.0, n_max=3, l_max=2, sigma=0.5)
    one = {"positions": np.zeros((1, 3)), "atomic_numbers": np.array([8])}
    assert _row_err(_np(s.create(one)), o.create(one["positions"], one["atomic_numbers"])) < DESC_TOL
    for r in (0.7, 3.0, o.cutoff - 1e-6, o.cutoff + 1e-6):
        dim = {"positions": np.array([[0.0, 0.0, 0.0], [0.3 * r, 0.4 * r, np.sqrt(0.75) * r]]),
               "atomic_numbers": np.array([1, 8])}
        assert _row_err(_np(s.create(dim)), o.create(dim["positions"], dim["atomic_numbers"])) < DESC_TOL


def test_include_exclude_dtype_sparse():
    from cusoap_b200 import SOAP
    sysd = W.water_cluster(2, 2, 2, seed=4)
    s = SOAP(species=[1, 8], r_cut=4.0, n_max=3, l_max=3, sigma=0.5, dtype="float64", sparse=True)
    d = s.create(sysd)
    assert d.dtype == torch.float64 and d.layout == torch.sparse_coo
    J = s.derivatives(sysd, centers=[0, 2], include=[1, 2, 3, 7], exclude=[2], return_descriptor=False)
    assert J.shape == (2, 3, 3, s.get_number_of_features())
    o = OracleSOAP(species=[1, 8], r_cut=4.0, n_max=3, l_max=3, sigma=0.5)
    Jo = o.derivatives(sysd["positions"], sysd["atomic_numbers"], centers=[0, 2], include=[1, 3, 7],
                       return_descriptor=False)
    assert _row_err(_np(J), Jo) < DERIV_TOL


def test_species_errors():
    from cusoap_b200 import SOAP
    s = SOAP(species=["H", "O"], r_cut=4.0, n_max=2, l_max=1)
    with pytest.raises(ValueError):
        s.create({"positions": np.zeros((1, 3)), "atomic_numbers": np.array([6])})
    with pytest.raises(ValueError):
        SOAP(species=[1], r_cut=4.0, n_max=2, l_max=1, average="bogus")
    with pytest.raises(ValueError):
        SOAP(species=[1], r_cut=4.0, n_max=2, l_max=1, periodic=True).create({"positions": np.zeros((1, 3)),
                                                                              "atomic_numbers": [1]})


@pytest.mark.parametrize("family", [0, 1])
@pytest.mark.parametrize("over", [{}, dict(r_cut=6.0, n_max=8, l_max=4, sigma=1.0),
                                  dict(r_cut=6.0, n_max=8, l_max=6, sigma=0.4)])
def test_deterministic(over, family):
    """Bitwise repeatable descriptors from both kernel families: one lane per
    radial index (family 0, the built-in choice here; its pair streams flush
    in a fixed order) and lanes grouped by l (family 1: the two-pair-stream
    kernel at n_max 4, l_max 3 and n_max 8, l_max 4, the one-stream kernel at
    l_max 6)."""
    s = _soap("cluster192", **over)
    s._basis.tune[3] = family
    sysd = W.make("cluster192")
    a = s.create(sysd)
    b = s.create(sysd)
    assert torch.equal(a, b)


@pytest.mark.parametrize("name", ["cluster192", "cells512", "cluster1M"])
def test_both_descriptor_families_match_the_oracle(name):
    """The radial-index-lane kernel (built-in) and the l-grouped kernel
    (tune[3] = 1) against the FP64 oracle on the same structures, with the
    centres' own atoms (self edges) and Cartesian centres off the atoms."""
    P = dict(W.CONFIGS[name])
    if name == "cluster1M":
        sysd = W.water_cluster(6, 6, 6, seed=2)
    elif name == "cells512":
        sysd = W.random_cells(1, seed=9, a_min=90, a_max=90)[0]
    else:
        sysd = W.make(name)
    o = _oracle(name)
    cen = list(range(0, len(sysd["atomic_numbers"]), 7))
    cart = [list(map(float, np.asarray(sysd["positions"][i]) + 0.37)) for i in (1, 4)]
    want = o.create(sysd["positions"], sysd["atomic_numbers"], centers=cen, cell=sysd.get("cell"),
                    pbc=sysd.get("pbc"))
    want_c = o.create(sysd["positions"], sysd["atomic_numbers"], centers=cart, cell=sysd.get("cell"),
                      pbc=sysd.get("pbc"))
    for family in (0, 1):
        s = _soap(name)
        s._basis.tune[3] = family
        assert _row_err(_np(s.create(sysd, centers=cen)), want) < DESC_TOL, family
        assert _row_err(_np(s.create(sysd, centers=cart)), want_c) < DESC_TOL, family


# ---- full-size workloads: sampled rows against the oracle ----

def test_cluster3000_create_and_derivatives():
    sysd = W.make("cluster3000")
    s = _soap("cluster3000")
    o = _oracle("cluster3000")
    J, D = s.derivatives(sysd)
    assert J.shape == (3000, 3000, 3, 420)
    Do = o.create(sysd["positions"], sysd["atomic_numbers"])
    assert _row_err(_np(D), Do) < DESC_TOL
    assert _row_err(_np(s.create(sysd)), Do) < DESC_TOL
    cen = [0, 1234, 2999]
    Jo = o.derivatives(sysd["positions"], sysd["atomic_numbers"], centers=cen, return_descriptor=False)
    assert _row_err(_np(J[cen]), Jo) < DERIV_TOL
    del J
    torch.cuda.empty_cache()


def test_cells512_batched():
    """The batched create of all 512 cells against the oracle: every centre of 12 cells (the
    smallest, the largest and 10 drawn with a fixed seed); then the batched adjoint forces of
    E = sum w.p over 3 of them (one create_flat launch per stage, one backward)."""
    cells = W.make("cells512")
    s = _soap("cells512")
    out = s.create(cells)
    o = _oracle("cells512")
    sizes = [len(c["atomic_numbers"]) for c in cells]
    rng = np.random.default_rng(7)
    pick = sorted({int(np.argmin(sizes)), int(np.argmax(sizes))} |
                  {int(k) for k in rng.choice(len(cells), 10, replace=False)})
    for k in pick:
        c = cells[k]
        ref = o.create(c["positions"], c["atomic_numbers"], cell=c["cell"], pbc=c["pbc"])
        assert _row_err(_np(out[k]), ref) < DESC_TOL, k
    sub = [cells[k] for k in sorted({pick[len(pick) // 2], int(np.argmin(sizes)), int(np.argmax(sizes))})]
    w = rng.standard_normal(s.get_number_of_features())
    wt = torch.tensor(w, dtype=torch.float32, device="cuda")
    pos = [torch.tensor(c["positions"], device="cuda", requires_grad=True) for c in sub]
    flat, _ = s.create_flat([dict(c, positions=p) for c, p in zip(sub, pos)])
    (flat @ wt).sum().backward()
    for c, p in zip(sub, pos):
        Fo = o.forces(c["positions"], c["atomic_numbers"], np.tile(w, (len(c["atomic_numbers"]), 1)),
                      cell=c["cell"], pbc=c["pbc"])
        assert rel_l2(-_np(p.grad), Fo) < DERIV_TOL


def test_waterbox2001_forces_vs_oracle():
    box = W.make("waterbox2001")
    s = _soap("waterbox2001")
    o = _oracle("waterbox2001")
    rng = np.random.default_rng(0)
    w = rng.standard_normal(s.get_number_of_features())
    E, F = s.energy_forces(box, w)
    Fo = o.forces(box["positions"], box["atomic_numbers"], np.tile(w, (2001, 1)), cell=box["cell"], pbc=box["pbc"])
    assert rel_l2(_np(F), Fo) < DERIV_TOL


def test_cluster1M_sampled():
    sysd = W.make("cluster1M")
    s = _soap("cluster1M")
    out = s.create(sysd)
    assert out.shape == (1_000_002, 680)
    o = _oracle("cluster1M")
    cen = [0, 123_456, 500_000, 1_000_001]
    ref = o.create(sysd["positions"], sysd["atomic_numbers"], centers=cen)
    assert _row_err(_np(out[cen]), ref) < DESC_TOL


def test_forces_many_species_vs_oracle():
    """8 species, n_max 8, l_max 6 (F = 14560): the adjoint's G kernel takes
    its index-table path (the dense W_l matrices would not fit in shared
    memory); forces of E = sum w . p against the oracle."""
    from cusoap_b200 import SOAP
    rng = np.random.default_rng(11)
    n = 60
    pos = rng.uniform(0.0, 9.0, size=(n, 3))
    Z = rng.choice([1, 2, 3, 4, 5, 6, 7, 8], size=n)
    Z[:8] = [1, 2, 3, 4, 5, 6, 7, 8]
    P = dict(species=[1, 2, 3, 4, 5, 6, 7, 8], r_cut=4.0, n_max=8, l_max=6, sigma=0.5)
    s = SOAP(**P)
    o = OracleSOAP(**P)
    w = rng.standard_normal(s.get_number_of_features())
    pt = torch.tensor(pos, device="cuda", requires_grad=True)
    E = (s.create({"positions": pt, "atomic_numbers": Z}) * torch.tensor(w, dtype=torch.float32,
                                                                         device="cuda")).sum()
    E.backward()
    Fo = o.forces(pos, Z, np.tile(w, (n, 1)))
    assert rel_l2(-pt.grad.cpu().numpy(), Fo) < DERIV_TOL


@pytest.mark.parametrize("l_max", [3, 4])
def test_forces_without_crossover_vs_oracle(l_max):
    """crossover=False: the adjoint's W_l has no cross-species entries (they
    stay zero in the G kernel's shared memory); forces of E = sum w . p
    against the oracle, with three species.  l_max 3 (F = 120) takes the TMA
    bulk row loads, l_max 4 (F = 150) the plain ones."""
    from cusoap_b200 import SOAP
    rng = np.random.default_rng(13)
    n = 45
    pos = rng.uniform(0.0, 8.0, size=(n, 3))
    Z = rng.choice([1, 6, 8], size=n)
    P = dict(species=[1, 6, 8], r_cut=4.5, n_max=4, l_max=l_max, sigma=0.5, crossover=False)
    s = SOAP(**P)
    o = OracleSOAP(**P)
    w = rng.standard_normal(s.get_number_of_features())
    pt = torch.tensor(pos, device="cuda", requires_grad=True)
    E = (s.create({"positions": pt, "atomic_numbers": Z}) * torch.tensor(w, dtype=torch.float32,
                                                                         device="cuda")).sum()
    E.backward()
    Fo = o.forces(pos, Z, np.tile(w, (n, 1)))
    assert rel_l2(-pt.grad.cpu().numpy(), Fo) < DERIV_TOL


@pytest.mark.parametrize("n_max,l_max", [(3, 2), (5, 4)])
def test_forces_unaligned_rows_vs_oracle(n_max, l_max):
    """Feature counts F = 63 and 275 and coefficient rows of 54 and 250 floats
    are not multiples of 4: the G kernel loads its rows with plain loads
    instead of TMA bulk copies; forces of E = sum w . p against the oracle."""
    from cusoap_b200 import SOAP
    rng = np.random.default_rng(12)
    n = 40
    pos = rng.uniform(0.0, 7.0, size=(n, 3))
    Z = rng.choice([1, 8], size=n)
    P = dict(species=[1, 8], r_cut=4.0, n_max=n_max, l_max=l_max, sigma=0.5)
    s = SOAP(**P)
    o = OracleSOAP(**P)
    F = s.get_number_of_features()
    assert F % 4 != 0
    w = rng.standard_normal(F)
    pt = torch.tensor(pos, device="cuda", requires_grad=True)
    E = (s.create({"positions": pt, "atomic_numbers": Z}) * torch.tensor(w, dtype=torch.float32,
                                                                         device="cuda")).sum()
    E.backward()
    Fo = o.forces(pos, Z, np.tile(w, (n, 1)))
    assert rel_l2(-pt.grad.cpu().numpy(), Fo) < DERIV_TOL


@pytest.mark.parametrize("name", ["cluster192", "waterbox2001"])
def test_forces_cc_vs_oracle(name):
    """average='cc' is differentiable too: the adjoint runs the cc layout's
    permutation and scale backwards; forces of E = sum w . cc against the
    oracle (periodic box included)."""
    from cusoap_b200 import SOAP
    P = dict(W.CONFIGS[name], average="cc")
    sysd = W.make("cluster192") if name == "cluster192" else W.water_box(8, 6.21, seed=5, dmin=2.4)
    s = SOAP(**P)
    o = OracleSOAP(**P)
    w = np.random.default_rng(8).standard_normal(s.get_number_of_features())
    pt = torch.tensor(sysd["positions"], device="cuda", requires_grad=True)
    d = dict(sysd, positions=pt)
    (s.create(d) * torch.tensor(w, dtype=torch.float32, device="cuda")).sum().backward()
    Fo = o.forces(sysd["positions"], sysd["atomic_numbers"], np.tile(w, (len(sysd["atomic_numbers"]), 1)),
                  sysd.get("cell"), sysd.get("pbc"))
    assert rel_l2(-pt.grad.cpu().numpy(), Fo) < DERIV_TOL
