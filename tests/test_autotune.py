"""The autotuner's candidate sets and cache (CPU), and that a tuned SOAP
object gives the untuned results (GPU)."""
import os

import numpy as np
import pytest

from cusoap_b200 import autotune as AT


def test_min_functions_per_lane_covers_every_function():
    for L in range(10):
        lanes = 32 // (L + 1)
        for N in range(1, 17):
            g = AT.min_functions_per_lane(N, L)
            assert g in (1, 2, 3, 4, 6)
            assert lanes * g >= N
            cands = AT.descriptor_candidates(N, L)
            assert all(w in (1, 2, 4) and gg >= g for w, gg in cands)
            assert len(cands) >= 3


def test_two_pair_streams_rule():
    # n_max 8, l_max 4 (the 1M-atom cluster): one stream keeps 20 of 32 lanes busy
    assert AT.two_pair_streams(8, 4)
    # n_max 7, l_max 3 (28 lanes busy) and every l_max > 4 keep one stream
    assert not AT.two_pair_streams(7, 3)
    assert not AT.two_pair_streams(8, 6)
    for L in range(5):
        for N in range(1, 17):
            if AT.two_pair_streams(N, L):
                lpl = 16 // (L + 1)
                assert lpl * 3 >= N  # at most 3 functions per lane in a half-warp
                assert len(AT.descriptor_candidates(N, L)) == 3


def test_cache_roundtrip(tmp_path):
    path = os.path.join(tmp_path, "tune.json")
    table = {"B200|N8|L6|S4|x1|rbf=gto": {"desc_wpb": 2, "desc_gn": 2, "force_wpb": 4}}
    AT._save(path, table)
    assert AT._load(path) == table
    assert AT._load(os.path.join(tmp_path, "missing.json")) == {}


@pytest.mark.gpu
def test_tuned_results_unchanged(tmp_path):
    import torch
    from cusoap_b200 import SOAP, workloads as W
    soap = SOAP(**W.CONFIGS["cells512"])
    cells = W.random_cells(12, seed=5, a_min=8, a_max=120)
    ref = soap.create(cells)
    ref = torch.cat(ref) if isinstance(ref, list) else ref.reshape(-1, ref.shape[-1])
    choice = soap.autotune(cells, reps=2, cache_path=os.path.join(tmp_path, "t.json"))
    assert choice["desc_wpb"] in (1, 2, 4) and choice["force_wpb"] in (1, 2, 4)
    assert list(soap._basis.tune)[:3] == [choice["desc_wpb"], choice["desc_gn"], choice["force_wpb"]]
    got = soap.create(cells)
    got = torch.cat(got) if isinstance(got, list) else got.reshape(-1, got.shape[-1])
    assert torch.equal(got, ref)
    again = SOAP(**W.CONFIGS["cells512"]).autotune(cells, cache_path=os.path.join(tmp_path, "t.json"))
    assert again["cached"]
