"""Multi-GPU sharding logic: centre ranges, and the force all-reduce run as
two gloo ranks on CPU with the oracle computing each rank's partial forces
(the reduction, not the kernels, is what runs without a GPU); on a GPU, the
sum of two shards' adjoint forces equals the unsharded adjoint, and the
sharded entry point runs end to end on a one-rank NCCL group."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp

from cusoap_b200.distributed import shard_range


def test_shard_range_partitions():
    for n in (0, 1, 7, 100, 1001):
        for world in (1, 2, 3, 8):
            spans = [shard_range(n, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == n
            assert all(spans[i][1] == spans[i + 1][0] for i in range(world - 1))
            sizes = [hi - lo for lo, hi in spans]
            assert max(sizes) - min(sizes) <= 1
    with pytest.raises(ValueError):
        shard_range(10, 2, 2)


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, q):
    import torch.distributed as dist
    from cusoap_b200 import workloads as W
    from cusoap_b200.distributed import sharded_energy_forces
    from oracle.soap_oracle import OracleSOAP
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        sysd = W.water_cluster(2, 2, 2, seed=3)
        o = OracleSOAP(**W.CONFIGS["cluster192"])
        A = len(sysd["atomic_numbers"])
        w = np.random.default_rng(0).standard_normal(o.n_power_features())

        def compute(lo, hi):
            dEdp = np.zeros((A, len(w)))
            dEdp[lo:hi] = w
            p = o.create(sysd["positions"], sysd["atomic_numbers"])
            E = float((p[lo:hi] * w).sum())
            return torch.tensor(E, dtype=torch.float64), torch.tensor(o.forces(sysd["positions"],
                                                                                sysd["atomic_numbers"], dEdp))

        E, F = sharded_energy_forces(None, sysd, None, compute=compute)
        if rank == 0:
            p = o.create(sysd["positions"], sysd["atomic_numbers"])
            Fref = o.forces(sysd["positions"], sysd["atomic_numbers"], np.tile(w, (A, 1)))
            q.put((E, float((p * w).sum()), float(np.abs(F.numpy() - Fref).max()), float(np.abs(Fref).max())))
    finally:
        dist.destroy_process_group()


def _gather_main(rank, world, port, n_total, q):
    import torch.distributed as dist
    from cusoap_b200.distributed import gather_rows
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world,
                            timeout=__import__("datetime").timedelta(seconds=60))
    try:
        lo, hi = shard_range(n_total, rank, world)
        # stand-in descriptor rows: row i holds (i, i + 0.5, ...), so order and coverage are checkable
        rows = torch.arange(lo, hi, dtype=torch.float32)[:, None] + 0.5 * torch.arange(5, dtype=torch.float32)
        out = gather_rows(rows, n_total)
        q.put((rank, out.numpy()))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("n_total", [7, 8, 1])
def test_gloo_two_ranks_gather_rows(n_total):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_gather_main, args=(r, 2, port, n_total, q)) for r in range(2)]
    for p in procs:
        p.start()
    got = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    want = np.arange(n_total, dtype=np.float32)[:, None] + 0.5 * np.arange(5, dtype=np.float32)
    for r in range(2):
        assert got[r].shape == want.shape
        assert np.array_equal(got[r], want)


def test_gloo_two_ranks_force_allreduce():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=300)
    assert all(p.exitcode == 0 for p in procs), [p.exitcode for p in procs]
    E, Eref, dF, Fmax = q.get(timeout=10)
    assert abs(E - Eref) <= 1e-10 * max(1.0, abs(Eref))
    assert dF <= 1e-10 * Fmax


@pytest.mark.gpu
def test_two_shards_sum_to_the_full_adjoint():
    from cusoap_b200 import SOAP, workloads as W
    from cusoap_b200.distributed import partial_forces
    soap = SOAP(**W.CONFIGS["waterbox2001"])
    box = W.water_box(8, 6.21, seed=5, dmin=2.4)
    A = len(box["atomic_numbers"])
    w = torch.tensor(np.random.default_rng(2).standard_normal(soap.get_number_of_features()),
                     dtype=torch.float32, device="cuda")
    E0, F0 = partial_forces(soap, box, w, 0, A)
    Ea, Fa = partial_forces(soap, box, w, 0, A // 2)
    Eb, Fb = partial_forces(soap, box, w, A // 2, A)
    assert abs(float(Ea + Eb) - float(E0)) <= 1e-5 * abs(float(E0))
    assert torch.allclose(Fa + Fb, F0, rtol=1e-4, atol=1e-5 * float(F0.abs().max()))


@pytest.mark.gpu
def test_sharded_entry_point_one_rank_nccl():
    import torch.distributed as dist
    from cusoap_b200 import SOAP, workloads as W
    from cusoap_b200.distributed import partial_forces, sharded_energy_forces
    os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
    os.environ["MASTER_PORT"] = str(_free_port())
    dist.init_process_group("nccl", rank=0, world_size=1, timeout=__import__("datetime").timedelta(seconds=60))
    try:
        soap = SOAP(**W.CONFIGS["cluster192"])
        sysd = W.make("cluster192")
        w = torch.tensor(np.random.default_rng(4).standard_normal(soap.get_number_of_features()),
                         dtype=torch.float32, device="cuda")
        E, F = sharded_energy_forces(soap, sysd, w)
        E0, F0 = partial_forces(soap, sysd, w, 0, len(sysd["atomic_numbers"]))
        assert abs(E - float(E0)) <= 1e-6 * abs(float(E0))
        assert torch.allclose(F, F0)
    finally:
        dist.destroy_process_group()
