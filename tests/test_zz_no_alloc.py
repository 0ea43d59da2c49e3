"""The no-allocation neighbour-list entry point (soapb_neighbors_noalloc).

It exists for callers that cannot allocate device memory when they need a
neighbour list -- for example a C or Fortran molecular-dynamics driver that
owns a fixed device-memory budget, or a time-step loop where cudaMalloc /
cudaFree would synchronise the device.  Its scratch is a fixed array inside
the library, so these tests check that two calls in a row, through the C
ABI, give exactly the pair list of the regular workspace entry points, and
that the size limit and the capacity flag behave as documented.  This file
is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest
import torch

from cusoap_b200 import workloads as W

pytestmark = pytest.mark.gpu


def _cases():
    yield dict(W.CONFIGS["cluster192"]), [W.make("cluster192")]
    yield dict(W.CONFIGS["cells512"]), W.random_cells(6, seed=21, a_min=8, a_max=120)


def test_noalloc_matches_workspace_path_twice():
    from cusoap_b200 import SOAP, _lib
    from cusoap_b200.soap import _Batch, _Pairs
    lib = _lib.load()
    for params, systems in _cases():
        soap = SOAP(**params)
        batch = _Batch(soap, systems, [None] * len(systems))
        for mode in (_lib.NL_CREATE, _lib.NL_ALL):
            ref = _Pairs(soap, batch, mode)  # regular entry points with a caller workspace
            n_pairs = ref.total
            for call in range(2):
                pair_off = torch.full((batch.n_centres + 1,), -1, dtype=torch.int64, device="cuda")
                pairs = torch.full((n_pairs + 64, 4), float("nan"), dtype=torch.float32, device="cuda")
                status = torch.full((1,), -7, dtype=torch.int32, device="cuda")
                rc = lib.soapb_neighbors_noalloc(ctypes.byref(soap._basis), ctypes.byref(batch.cs),
                                                 ctypes.byref(batch.cc), mode, pair_off.data_ptr(),
                                                 pairs.data_ptr(), pairs.shape[0], status.data_ptr(),
                                                 torch.cuda.current_stream().cuda_stream)
                assert rc == _lib.OK, lib.soapb_last_error()
                torch.cuda.synchronize()
                assert int(status.item()) == 0, (call, int(status.item()))
                assert torch.equal(pair_off, ref.pair_off), call
                assert torch.equal(pairs[:n_pairs], ref.pairs[:n_pairs]), call


def test_noalloc_capacity_flag_and_size_limit():
    from cusoap_b200 import SOAP, _lib
    from cusoap_b200.soap import _Batch
    lib = _lib.load()
    soap = SOAP(**W.CONFIGS["cluster192"])
    batch = _Batch(soap, [W.make("cluster192")], [None])
    st = torch.cuda.current_stream().cuda_stream
    pair_off = torch.empty(batch.n_centres + 1, dtype=torch.int64, device="cuda")
    pairs = torch.empty((16, 4), dtype=torch.float32, device="cuda")
    status = torch.zeros(1, dtype=torch.int32, device="cuda")
    rc = lib.soapb_neighbors_noalloc(ctypes.byref(soap._basis), ctypes.byref(batch.cs), ctypes.byref(batch.cc),
                                     _lib.NL_CREATE, pair_off.data_ptr(), pairs.data_ptr(), 16, status.data_ptr(), st)
    assert rc == _lib.OK
    torch.cuda.synchronize()
    assert int(status.item()) & 4  # capacity too small: flagged, nothing written
    assert int(pair_off[-1].item()) > 16  # the needed size is still reported
    # an input larger than the fixed scratch is refused on the host, before any launch
    big = _lib.Structs(1, 5_000_000, batch.cs.d_atom_off, batch.cs.d_positions, batch.cs.d_species,
                       batch.cs.d_cells, batch.cs.d_pbc)
    rc = lib.soapb_neighbors_noalloc(ctypes.byref(soap._basis), ctypes.byref(big), ctypes.byref(batch.cc),
                                     _lib.NL_CREATE, pair_off.data_ptr(), pairs.data_ptr(), 16, status.data_ptr(), st)
    assert rc == _lib.ERR_ARG
    assert "scratch" in lib.soapb_last_error().decode()
