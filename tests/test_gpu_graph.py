"""The CUDA-graph batch plan (SOAP.batch): replays must give the eager
batched path's results at every new set of positions, the adjoint must give
its forces, and a pair list that outgrows the plan's buffer must be caught
and re-planned (never read past the buffer)."""
import numpy as np
import pytest
import torch

from cusoap_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cells(n, seed=4):
    return W.random_cells(n, seed=seed, a_min=8, a_max=120)


def _with_positions(cells, pos_cat):
    out, o = [], 0
    for c in cells:
        k = len(c["atomic_numbers"])
        out.append(dict(c, positions=pos_cat[o:o + k]))
        o += k
    return out


def test_graph_replays_match_eager_batched():
    from cusoap_b200 import SOAP
    soap = SOAP(**W.CONFIGS["cells512"])
    cells = _cells(24)
    plan = soap.batch(cells)
    pos0 = torch.tensor(np.concatenate([c["positions"] for c in cells]), device="cuda")
    rng = np.random.default_rng(0)
    for step in range(3):
        pos = pos0 + torch.tensor(rng.uniform(-0.05, 0.05, size=pos0.shape), device="cuda") * step
        got = plan.create(pos).clone()
        ref = soap.create(_with_positions(cells, pos))
        ref = torch.cat(ref) if isinstance(ref, list) else ref.reshape(-1, ref.shape[-1])
        assert torch.equal(got, ref), step


def test_graph_adjoint_matches_eager_forces():
    from cusoap_b200 import SOAP
    soap = SOAP(**W.CONFIGS["cells512"])
    cells = _cells(16, seed=9)
    plan = soap.batch(cells)
    w = torch.tensor(np.random.default_rng(1).standard_normal(soap.get_number_of_features()),
                     dtype=torch.float32, device="cuda")
    pos = torch.tensor(np.concatenate([c["positions"] for c in cells]), device="cuda", requires_grad=True)
    (plan.create(pos) * w).sum().backward()
    g_plan = pos.grad.clone()
    pos2 = pos.detach().clone().requires_grad_(True)
    out = soap.create(_with_positions(cells, pos2))
    ((torch.cat(out) if isinstance(out, list) else out.reshape(-1, out.shape[-1])) * w).sum().backward()
    assert torch.allclose(g_plan, pos2.grad, rtol=1e-5, atol=1e-6 * float(pos2.grad.abs().max()))


def test_graph_replans_when_pairs_outgrow_the_buffer():
    """Non-periodic clusters squeezed to 0.7 of their size hold ~2.9x more
    pairs than the plan was built for: the clamp empties the lists, the host
    sees the total, re-plans and replays; the result equals the eager path."""
    from cusoap_b200 import SOAP
    soap = SOAP(**W.CONFIGS["cluster192"])
    systems = [W.water_cluster(3, 3, 3, seed=s) for s in (1, 2, 3)]
    plan = soap.batch(systems, headroom=1.0)
    cap0 = plan.capacity
    squeezed = []
    for sd in systems:
        p = torch.tensor(sd["positions"], device="cuda")
        squeezed.append(p.mean(0, keepdim=True) + 0.7 * (p - p.mean(0, keepdim=True)))
    pos = torch.cat(squeezed)
    got = plan.create(pos).clone()
    assert plan.capacity > cap0
    ref = soap.create(_with_positions(systems, pos))
    ref = torch.cat(ref) if isinstance(ref, list) else ref.reshape(-1, ref.shape[-1])
    assert torch.equal(got, ref)
    # and back at the original positions, the (larger) plan still matches
    pos0 = torch.cat([torch.tensor(sd["positions"], device="cuda") for sd in systems])
    got0 = plan.create(pos0).clone()
    ref0 = soap.create(_with_positions(systems, pos0))
    ref0 = torch.cat(ref0) if isinstance(ref0, list) else ref0.reshape(-1, ref0.shape[-1])
    assert torch.equal(got0, ref0)


def test_graph_plan_cc_and_ase_like_input():
    """The plan with average='cc' (forward and adjoint), on ASE-like objects
    (get_positions / get_atomic_numbers / get_cell / get_pbc)."""
    from cusoap_b200 import SOAP

    class Atoms:
        def __init__(self, d):
            self.d = d

        def get_positions(self):
            return self.d["positions"]

        def get_atomic_numbers(self):
            return self.d["atomic_numbers"]

        def get_cell(self):
            class C:
                array = np.asarray(self.d["cell"])
            return C()

        def get_pbc(self):
            return np.asarray(self.d["pbc"])

    soap = SOAP(**dict(W.CONFIGS["cells512"], average="cc"))
    cells = _cells(6, seed=12)
    atoms = [Atoms(c) for c in cells]
    plan = soap.batch(atoms)
    w = torch.tensor(np.random.default_rng(3).standard_normal(soap.get_number_of_features()),
                     dtype=torch.float32, device="cuda")
    pos = torch.tensor(np.concatenate([c["positions"] for c in cells]), device="cuda", requires_grad=True)
    out = plan.create(pos)
    ref = soap.create(atoms)
    ref = torch.cat(ref) if isinstance(ref, list) else ref.reshape(-1, ref.shape[-1])
    assert torch.equal(out, ref)
    (out @ w).sum().backward()
    pos2 = pos.detach().clone().requires_grad_(True)
    out2 = soap.create(_with_positions(cells, pos2))
    ((torch.cat(out2) if isinstance(out2, list) else out2.reshape(-1, out2.shape[-1])) @ w).sum().backward()
    assert torch.allclose(pos.grad, pos2.grad, rtol=1e-5, atol=1e-6 * float(pos2.grad.abs().max()))
