#!/usr/bin/env python
"""Benchmark: atoms/s for SOAP + dP/dr on one B200.

Workload (the single-structure GPU configuration): non-periodic (H2O)_1000
cluster, 3000 atoms on a jittered 10x10x10 lattice (seeded, synthetic);
species H, O; r_cut 10, n_max 7, l_max 3, sigma 0.5, gto, average off.
One step = the descriptor plus the analytical dP/dr of every centre w.r.t.
every atom, (3000, 3000, 3, 420) float32 = 45.4 GB, through the public API
``SOAP.derivatives`` (the same call as the reference's examples).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Prints ONE JSON line.  ``value`` is device-resident throughput (inputs in
HBM, CUDA events around every step, max over ranks); ``e2e`` is the same
call with the positions copied from pinned host memory and both outputs
copied back to pinned host memory inside the timed region; ``roofline`` is
the Jacobian kernel (an HBM write stream) timed with CUDA events during the
timed steps; ``cpu_baseline`` is the reference's algorithm (its timed CPU
port, oracle/reference_port.py) on a bounded sample of its own centre-batch
loop, on every host thread.  Under torchrun each rank runs its own copy of
the workload (weak scaling, no data-path collective).  ``--impl reference``
times that port step by step, every step in full: create + analytical
derivatives of 50 consecutive centres (the reference itself is Python and
does not travel to the benchmark host).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "atoms/s for SOAP + dP/dr, fused batched vs plain, 1 B200, rel err <= 1e-5"
UNIT = "atoms/s"
WORKLOAD = "cluster3000"
CONFIG = {
    "workload": "(H2O)_1000 non-periodic water cluster, 3000 atoms; species H,O; r_cut=10, n_max=7, l_max=3, "
                "sigma=0.5, gto, average=off; create + analytical dP/dr of every centre w.r.t. every atom "
                "(float32 output)",
    "features": 420,
    "l2": "GPU arm: each step writes 45.4 GB (> 126 MB L2) and L2 is also flushed between timed steps",
}
# Centres per step of the reference arm: the reference's own driver loops over
# centre batches, create(centers=range(s, e)) + derivatives(same centres)
# (examples/test_serial.py:53-60).
REF_BATCH = 50


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _traffic_from_profiles():
    """Per-launch DRAM bytes of the Jacobian kernel at this workload, from the
    committed ncu summary (None when absent)."""
    path = os.path.join(ROOT, "profiles", "jacobian_cluster3000.md")
    try:
        for line in open(path):
            if line.strip().startswith("traffic_bytes_per_launch_full:"):
                return float(line.split(":", 1)[1].strip().split()[0])
    except OSError:
        pass
    return None


class Clocks:
    """SM clock and throttle-reason sampler for the timed region.

    Reads NVML (the library behind nvidia-smi) from a background thread every
    5 ms, on the GPU that this process's CUDA device is (matched by UUID, so a
    remapped device list cannot point it at another GPU); falls back to an
    nvidia-smi subprocess.  Only reads; changes no setting."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        import threading
        self.index = index
        self.rows = []
        self.p = None
        self.nv = None
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            h = None
            uuid = str(getattr(torch.cuda.get_device_properties(index), "uuid", "") or "")
            if uuid:
                try:
                    h = nv.nvmlDeviceGetHandleByUUID(uuid if uuid.startswith("GPU-") else "GPU-" + uuid)
                except Exception:
                    h = None
            if h is None:
                h = nv.nvmlDeviceGetHandleByIndex(index)
            self.nv, self.h = nv, h
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            get = getattr(nv, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                nv.nvmlDeviceGetCurrentClocksThrottleReasons
            bits = {"hw_slowdown": "HwSlowdown", "hw_thermal_slowdown": "HwThermalSlowdown",
                    "sw_thermal_slowdown": "SwThermalSlowdown", "sw_power_cap": "SwPowerCap"}
            self.bits = {k: getattr(nv, "nvmlClocksEventReason" + v, None) or getattr(nv, "nvmlClocksThrottleReason" + v)
                         for k, v in bits.items()}
            self.stop_ev = threading.Event()

            def run():
                while not self.stop_ev.is_set():
                    try:
                        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)), int(get(h))))
                    except Exception:
                        pass
                    time.sleep(0.005)
            self.t = threading.Thread(target=run, daemon=True)
            self.t.start()
        except Exception:
            self.nv = None
            self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
            try:
                self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={self.Q}",
                                           "--format=csv,noheader,nounits", "-lms", "20"],
                                          stdout=self.f, stderr=subprocess.DEVNULL)
            except Exception:
                self.p = None

    def wait_first_sample(self, timeout_s: float = 5.0):
        """Block until the first sample exists, so that the timed region that
        follows is covered from its start."""
        t0 = time.time()
        while time.time() - t0 < timeout_s:
            if self.nv is not None and self.rows:
                return
            if self.p is not None and os.path.getsize(self.f.name) > 0:
                return
            if self.nv is None and self.p is None:
                return
            time.sleep(0.002)

    def stop(self):
        if self.nv is not None:
            self.stop_ev.set()
            self.t.join(timeout=2)
            rows = list(self.rows)
            if not rows:
                return {"sm_mhz": None, "sm_max_mhz": self.smax, "reasons": ["no samples"], "source": "nvml"}
            reasons = sorted({k for _, r in rows for k, b in self.bits.items() if r & b})
            return {"sm_mhz": statistics.median(x for x, _ in rows), "sm_max_mhz": self.smax, "reasons": reasons,
                    "samples": len(rows), "source": "nvml"}
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        rows = []
        with open(self.f.name) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        smax = max(float(r[2]) for r in rows if r[2].replace(".", "").isdigit())
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows), "source": "nvidia-smi"}


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def parity_centres(n_centres: int = 24):
    """The sampled centres of the Jacobian parity check."""
    rng = np.random.default_rng(0)
    return [int(c) for c in rng.choice(3000, n_centres, replace=False)]


def _host_threads() -> int:
    return len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)


def _reference_steps(port, sysd, n_steps: int, first: int = 0):
    """n_steps steps of the reference's centre-batch loop on the port:
    create + analytical derivatives of REF_BATCH consecutive centres per
    step.  Step i takes batch (23 i) mod n_batches (a permutation of the
    batches, as 23 is prime to 60), so a few steps sample the whole cluster,
    surface and interior, not only its first lattice rows.  Returns
    per-step seconds and centres."""
    pos, Z = sysd["positions"], sysd["atomic_numbers"]
    n = len(Z)
    n_batches = (n + REF_BATCH - 1) // REF_BATCH
    times, counts = [], []
    for i in range(first, first + n_steps):
        s = ((23 * i) % n_batches) * REF_BATCH
        cen = list(range(s, min(s + REF_BATCH, n)))
        t0 = time.perf_counter()
        port.create(pos, Z, cen)
        port.derivatives(pos, Z, cen)
        times.append(time.perf_counter() - t0)
        counts.append(len(cen))
    return times, counts


def cpu_baseline_sample(n_steps: int = 2):
    """The reference's algorithm (its timed CPU port, float64 inside,
    float32 out, on every host thread) on a bounded sample: n_steps steps of
    its centre-batch loop.  Also returns the float64 checker values of the
    GPU step's parity: every descriptor row, and the Jacobian blocks of the
    parity centres."""
    import torch
    from oracle.reference_port import ReferencePort
    from cusoap_b200 import workloads as W
    threads = _host_threads()
    torch.set_num_threads(threads)
    sysd = W.make(WORKLOAD)
    port = ReferencePort(**W.CONFIGS[WORKLOAD])
    times, counts = _reference_steps(port, sysd, n_steps)
    check = ReferencePort(**W.CONFIGS[WORKLOAD], out_dtype=torch.float64)
    desc = check.create(sysd["positions"], sysd["atomic_numbers"]).numpy()
    jac = check.derivatives(sysd["positions"], sysd["atomic_numbers"], parity_centres()).numpy()
    return {"value": sum(counts) / sum(times), "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n_steps} steps of the reference's centre-batch loop (create + analytical dP/dr of "
                      f"{REF_BATCH} centres per step) on its timed CPU port, {sum(times):.2f} s",
            "seconds": sum(times)}, desc, jac


def _row_err(a, b) -> float:
    """Largest relative L2 error over rows (a row = one centre's descriptor or Jacobian block)."""
    a = np.asarray(a, np.float64).reshape(a.shape[0], -1)
    b = np.asarray(b, np.float64).reshape(b.shape[0], -1)
    nb = np.linalg.norm(b, axis=1)
    return float(np.max(np.linalg.norm(a - b, axis=1) / np.where(nb > 0, nb, 1.0)))


def parity_other_legs(soap_cls, torch):
    """FP64-oracle errors of the batched, scale and differentiation legs'
    computations (the same calls as the timed legs, on samples: 3 cells, 4
    centres of the 1M-atom cluster, all forces of the 2001-atom box)."""
    from oracle.soap_oracle import OracleSOAP, rel_l2
    from cusoap_b200 import workloads as W
    out = {}
    cells = W.make("cells512")[:3]
    s = soap_cls(**W.CONFIGS["cells512"])
    o = OracleSOAP(**W.CONFIGS["cells512"])
    got = s.create(cells)
    out["batched_desc_max_row_rel_l2"] = max(
        _row_err(g.cpu().numpy(), o.create(c["positions"], c["atomic_numbers"], cell=c["cell"], pbc=c["pbc"]))
        for g, c in zip(got, cells))
    big = W.make("cluster1M")
    s = soap_cls(**W.CONFIGS["cluster1M"])
    o = OracleSOAP(**W.CONFIGS["cluster1M"])
    cen = [0, 123_456, 500_000, 1_000_001]
    pos = torch.tensor(big["positions"], dtype=torch.float64, device="cuda")
    got = s.create({"positions": pos, "atomic_numbers": big["atomic_numbers"]})[cen].cpu().numpy()
    out["scale_desc_max_row_rel_l2"] = _row_err(got, o.create(big["positions"], big["atomic_numbers"], centers=cen))
    del pos
    box = W.make("waterbox2001")
    s = soap_cls(**W.CONFIGS["waterbox2001"])
    o = OracleSOAP(**W.CONFIGS["waterbox2001"])
    w = np.random.default_rng(0).standard_normal(s.get_number_of_features())
    p = torch.tensor(box["positions"], dtype=torch.float64, device="cuda", requires_grad=True)
    (s.create(dict(box, positions=p)) @ torch.tensor(w, dtype=torch.float32, device="cuda")).sum().backward()
    Fo = o.forces(box["positions"], box["atomic_numbers"], np.tile(w, (len(box["atomic_numbers"]), 1)),
                  box["cell"], box["pbc"])
    out["diff_forces_rel_l2"] = rel_l2(-p.grad.cpu().numpy(), Fo)
    return out


def run_reference(args):
    """--impl reference: the reference's algorithm on the host CPU, as its
    own driver runs it (examples/test_serial.py:53-60): every step is
    create + analytical derivatives of a batch of REF_BATCH consecutive
    centres, executed in full and timed.  The reference is a Python package
    that does not travel to the benchmark host, so its timed CPU port runs
    (oracle/reference_port.py: the same torch float64 operations, timed
    against the reference itself on the same threads by
    oracle/calibrate_port.py).  Under torchrun only rank 0 runs."""
    import torch
    world, rank, _ = _dist()
    if rank != 0:
        return
    from oracle.reference_port import ReferencePort
    from cusoap_b200 import workloads as W
    threads = _host_threads()
    torch.set_num_threads(threads)
    sysd = W.make(WORKLOAD)
    port = ReferencePort(**W.CONFIGS[WORKLOAD])
    _reference_steps(port, sysd, max(0, args.warmup))
    times, counts = _reference_steps(port, sysd, args.steps, first=max(0, args.warmup))
    t = sum(times)
    value = sum(counts) / t
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)",
            "impl": "reference", "config": dict(CONFIG), "atoms_per_step": REF_BATCH,
            "parallelism": f"{threads} host threads",
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": "port",
                             "sample": f"every step in full: create + analytical dP/dr of {REF_BATCH} consecutive "
                                       f"centres (the reference's centre-batch loop) on its timed CPU port, float64 "
                                       f"inside, float32 out; {args.steps} steps, {t:.2f} s timed"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def plain_cpu_cluster192(soap_cls, torch):
    """The CPU workload of the reference (192-atom (H2O)_64 cluster, n_max 4,
    l_max 3, r_cut 5, sigma 0.5): create + analytical derivatives of every
    centre w.r.t. every atom in float64, on the reference's timed CPU port
    with every host thread; beside it the same call on the GPU path
    (float32 arithmetic)."""
    from oracle.reference_port import ReferencePort
    from cusoap_b200 import workloads as W
    sysd = W.make("cluster192")
    pos, Z = sysd["positions"], sysd["atomic_numbers"]
    threads = _host_threads()
    torch.set_num_threads(threads)
    port = ReferencePort(**W.CONFIGS["cluster192"], out_dtype=torch.float64)
    ts = []
    for _ in range(4):
        t0 = time.perf_counter()
        port.create(pos, Z)
        port.derivatives(pos, Z)
        ts.append(time.perf_counter() - t0)
    t_cpu = statistics.median(ts[1:])
    soap = soap_cls(**W.CONFIGS["cluster192"])
    pos_d = torch.tensor(pos, device="cuda")
    for _ in range(3):
        soap.derivatives({"positions": pos_d, "atomic_numbers": Z})
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(20):
        soap.derivatives({"positions": pos_d, "atomic_numbers": Z})
    e1.record()
    torch.cuda.synchronize()
    t_gpu = e0.elapsed_time(e1) / 20 / 1e3
    n = len(Z)
    return {"workload": "(H2O)_64 non-periodic cluster, 192 atoms; r_cut 5, n_max 4, l_max 3, sigma 0.5; create + "
                        "analytical derivatives of every centre w.r.t. every atom",
            "cpu_port_atoms_per_s": n / t_cpu, "cpu_port_s": t_cpu, "cpu_threads": threads, "cpu_dtype": "f64",
            "gpu_atoms_per_s": n / t_gpu, "gpu_ms": t_gpu * 1e3, "gpu_dtype": "f32",
            "note": "CPU: the reference's algorithm on its timed port, median of 3 after one warm-up; GPU: "
                    "SOAP.derivatives on device-resident positions, 20 calls after 3 warm-ups"}


def batched_vs_plain(soap_cls, torch):
    """The batched workload with forces: 512 periodic cells of 8-400 atoms
    (n_max 8, l_max 6, 4 species), descriptor + adjoint forces of
    E = sum w.p, one batched launch per stage vs a per-structure loop."""
    from cusoap_b200 import workloads as W
    cells = W.make("cells512")
    soap = soap_cls(**W.CONFIGS["cells512"])
    tuned = soap.autotune(cells[:64], reps=2)  # launch shapes for (n_max 8, l_max 6, 4 species); all legs use them
    rng = np.random.default_rng(0)
    w = torch.tensor(rng.standard_normal(soap.get_number_of_features()), dtype=torch.float32, device="cuda")
    dev_cells = [{"positions": torch.tensor(c["positions"], device="cuda"), "atomic_numbers": c["atomic_numbers"],
                  "cell": c["cell"], "pbc": c["pbc"]} for c in cells]
    n_atoms = sum(len(c["atomic_numbers"]) for c in cells)

    def batched():
        sysl = []
        for c in dev_cells:
            d = dict(c)
            d["positions"] = c["positions"].clone().requires_grad_(True)
            sysl.append(d)
        out, _ = soap.create_flat(sysl)  # one (total atoms, F) buffer for the whole batch
        E = (out @ w).sum()
        E.backward()
        return sysl

    def plain():
        for c in dev_cells:
            d = dict(c)
            d["positions"] = c["positions"].clone().requires_grad_(True)
            (soap.create(d) @ w).sum().backward()

    plan = soap.batch(cells)
    pos_all = torch.cat([c["positions"] for c in dev_cells])

    def graph():
        pos = pos_all.clone().requires_grad_(True)
        (plan.create(pos) @ w).sum().backward()
        return pos

    res = {}
    for name, fn, reps in (("batched", batched, 20), ("graph", graph, 20), ("plain", plain, 5)):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        res[name] = n_atoms * reps / (e0.elapsed_time(e1) / 1e3)
    return {"workload": "512 periodic cubic cells, 8-400 atoms (104k atoms), 4 species, r_cut 6, n_max 8, l_max 6, "
                        "sigma 0.4; descriptor + adjoint forces of E = sum w.p per step",
            "batched_atoms_per_s": res["batched"], "plain_atoms_per_s": res["plain"],
            "speedup": res["batched"] / res["plain"],
            "graph_atoms_per_s": res["graph"], "graph_speedup": res["graph"] / res["plain"],
            "graph_note": "SOAP.batch plan: forward and adjoint replayed as two captured CUDA graphs",
            "autotuned": {k: tuned[k] for k in ("desc_wpb", "desc_gn", "force_wpb")}}


def run_batched_only(args):
    """--batched-cells K: the batched path alone (descriptor + adjoint forces
    of E = sum w.p) on the first K cells of the 512-cell workload, one warm-up
    and --steps timed passes, with per-stage CUDA-event times; a profiling
    case for the batched kernels (prints one JSON line, not a bench value)."""
    import torch
    from cusoap_b200 import SOAP, workloads as W
    torch.cuda.set_device(0)
    cells = W.make("cells512")[:args.batched_cells]
    soap = SOAP(**W.CONFIGS["cells512"])
    rng = np.random.default_rng(0)
    w = torch.tensor(rng.standard_normal(soap.get_number_of_features()), dtype=torch.float32, device="cuda")
    dev_cells = [{"positions": torch.tensor(c["positions"], device="cuda"), "atomic_numbers": c["atomic_numbers"],
                  "cell": c["cell"], "pbc": c["pbc"]} for c in cells]

    def one():
        sysl = [dict(c, positions=c["positions"].clone().requires_grad_(True)) for c in dev_cells]
        out, _ = soap.create_flat(sysl)
        E = (out @ w).sum()
        E.backward()

    one()
    torch.cuda.synchronize()
    soap.profile = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(args.steps):
        one()
    e1.record()
    torch.cuda.synchronize()
    st = {k: v / args.steps for k, v in soap.stage_times().items()}
    n_atoms = sum(len(c["atomic_numbers"]) for c in cells)
    print(json.dumps({"workload": f"first {len(cells)} cells of the 512-cell batch ({n_atoms} atoms)",
                      "ms_per_step": e0.elapsed_time(e1) / args.steps, "stage_ms_per_step": st}), flush=True)


def diff_forces(soap_cls, torch, steps: int = 20, warmup: int = 3):
    """The differentiation workload: periodic water box of 2001 atoms
    (667 molecules at 1.0 g/cm^3, 27.1 A cube; n_max 8, l_max 6, sigma 1),
    E = sum_i w . p_i with seeded N(0, 1) weights, forces from create() and
    the adjoint (E.backward()); positions resident on the device."""
    from cusoap_b200 import workloads as W
    box = W.make("waterbox2001")
    soap = soap_cls(**W.CONFIGS["waterbox2001"])
    w = torch.tensor(np.random.default_rng(0).standard_normal(soap.get_number_of_features()),
                     dtype=torch.float32, device="cuda")
    pos0 = torch.tensor(box["positions"], dtype=torch.float64, device="cuda")

    def step():
        pos = pos0.clone().requires_grad_(True)
        (soap.create(dict(box, positions=pos)) @ w).sum().backward()
        return pos.grad

    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        step()
    e1.record()
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    # per-stage times from separate steps (the stage events add host work of their own)
    soap.profile = []
    for _ in range(steps):
        step()
    st = {k: v / steps for k, v in soap.stage_times().items()}
    soap.profile = None
    n = len(box["atomic_numbers"])
    # the same step through the SOAP.batch graph plan (forward and adjoint replayed as graphs)
    plan = soap.batch([box])

    def graph_step():
        pos = pos0.clone().requires_grad_(True)
        (plan.create(pos) @ w).sum().backward()
        return pos.grad

    for _ in range(warmup):
        graph_step()
    torch.cuda.synchronize()
    e0.record()
    for _ in range(steps):
        graph_step()
    e1.record()
    torch.cuda.synchronize()
    ms_g = e0.elapsed_time(e1) / steps
    return {"workload": "periodic water box, 2001 atoms, r_cut 6, n_max 8, l_max 6, sigma 1; E = sum w.p, forces "
                        "by create() + E.backward() (the adjoint)",
            "atoms_per_s": n / (ms / 1e3), "ms_per_step": ms, "stage_ms_per_step": st,
            "graph_atoms_per_s": n / (ms_g / 1e3), "graph_ms_per_step": ms_g,
            "graph_note": "the same step through SOAP.batch([box]): forward and adjoint replayed as captured graphs"}


FP32_PEAK_TFLOPS = 148 * 128 * 2 * 1.965e9 / 1e12  # 148 SMs x 128 FP32 lanes x FMA at the 1965 MHz max clock


def harmonics_flop(L: int) -> int:
    """FLOP of one pair's real solid harmonics up to l_max = L, as the kernels
    compute them: r^2 (5); the Legendre table Q_l^m -- L entries Q_{m+1}^m at 1
    FLOP and (L-1)L/2 three-term entries at 5; the powers (x + i y)^m, 6 per m;
    the (L+1)(L+2)/2 normalisations and the L(L+1) products with cos/sin."""
    return 5 + L + 5 * (L - 1) * L // 2 + 6 * L + (L + 1) * (L + 2) // 2 + L * (L + 1)


def scale_create(soap_cls, torch, steps: int = 3, warmup: int = 2, n_mol: int = 0):
    """The scale workload: create() on the 1,000,002-atom water cluster
    (n_max 8, l_max 4, F = 680, 2.72 GB of output), positions resident on the
    device.  Reports atoms/s and the descriptor kernel against both its HBM
    traffic (pairs read + rows written) and its FP32 work.  n_mol > 0: the
    same lattice cut to n_mol molecules (a smaller profiling case)."""
    from cusoap_b200 import workloads as W
    sysd = W.make("cluster1M") if n_mol <= 0 else W.water_cluster(70, 70, 69, n_mol=n_mol, seed=0)
    soap = soap_cls(**W.CONFIGS["cluster1M"])
    pos = torch.tensor(sysd["positions"], dtype=torch.float64, device="cuda")
    system = {"positions": pos, "atomic_numbers": sysd["atomic_numbers"]}
    for _ in range(warmup):
        out = soap.create(system)
        del out
    torch.cuda.synchronize()
    soap.profile = []
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        out = soap.create(system)
        del out
    e1.record()
    torch.cuda.synchronize()
    st = {k: v / steps for k, v in soap.stage_times().items()}
    soap.profile = None
    n_at, F = len(sysd["atomic_numbers"]), soap.get_number_of_features()
    # pairs: the last create's list length (same every step)
    from cusoap_b200.soap import _Batch, _Pairs
    from cusoap_b200 import _lib
    n_pairs = _Pairs(soap, _Batch(soap, [system], [None]), _lib.NL_CREATE).total
    N, L = W.CONFIGS["cluster1M"]["n_max"], W.CONFIGS["cluster1M"]["l_max"]
    K = (L + 1) ** 2
    # a degree-7 Horner pass is 7 FMAs = 14 FLOP per radial function and pair
    flop = n_pairs * (2 * N * K + N * (L + 1) * 14 + harmonics_flop(L)) + n_at * 2 * F * K / (L + 1)
    byts = n_pairs * 16 + n_at * F * 4
    d_ms = st.get("descriptor", float("nan"))
    peak, _ = _peaks()
    return {"workload": f"(H2O)_{n_at // 3} non-periodic cluster, {n_at:,} atoms; r_cut 6, n_max 8, l_max 4, "
                        "sigma 1; create() only, positions on the device",
            "atoms_per_s": n_at * steps / (e0.elapsed_time(e1) / 1e3), "ms_per_step": e0.elapsed_time(e1) / steps,
            "stage_ms_per_step": st, "pairs": n_pairs,
            "descriptor": {"hbm_bytes": byts, "gbs": byts / d_ms / 1e6, "hbm_frac_of_measured": byts / d_ms / 1e6 / peak,
                           "flop": flop, "tflops": flop / d_ms / 1e9,
                           "fp32_frac_of_nominal": flop / d_ms / 1e9 / FP32_PEAK_TFLOPS,
                           "note": "flop = pairs x (2 N K accumulate + 14 N (l_max+1) radial Horner, 7 FMAs per function + "
                                   f"{harmonics_flop(L)} solid harmonics) + centres x 2 F K/(l_max+1) power spectrum; "
                                   "bytes = 16 B per pair read + F x 4 B per row"}}


def run_ours(args):
    import torch
    world, rank, local = _dist()
    if world > 1:
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=120))
    else:
        torch.cuda.set_device(0)
    device = torch.device("cuda", torch.cuda.current_device())
    from cusoap_b200 import SOAP, _lib, workloads as W
    sysd = W.make(WORKLOAD) if args.nx == 10 else W.water_cluster(args.nx, args.nx, args.nx, seed=0)
    n_at = len(sysd["atomic_numbers"])
    soap = SOAP(**W.CONFIGS[WORKLOAD], device=device)
    pos_d = torch.tensor(sysd["positions"], dtype=torch.float64, device=device)
    Z = sysd["atomic_numbers"]
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)

    def step():
        return soap.derivatives({"positions": pos_d, "atomic_numbers": Z}, return_descriptor=True)

    for _ in range(args.warmup):
        J, D = step()
        del J, D
    torch.cuda.synchronize()

    def barrier():
        if world > 1:
            torch.distributed.barrier()
        torch.cuda.synchronize()

    # ---- device-resident timed region ----
    clocks = Clocks(torch.cuda.current_device() if world == 1 else local)
    clocks.wait_first_sample()
    soap.profile = []
    launches0 = _lib.kernel_launches()
    evs = []
    barrier()
    for i in range(args.steps):
        flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        J, D = step()
        e1.record()
        evs.append((e0, e1))
        if i < args.steps - 1:
            del J, D
    barrier()
    launches = _lib.kernel_launches() - launches0
    clk = clocks.stop()
    # the last timed step's outputs, kept for the parity check against the oracle
    want_parity = rank == 0 and world == 1 and not args.no_cpu and args.nx == 10
    par_J = J[parity_centres()].cpu().numpy() if want_parity else None
    par_D = D.cpu().numpy() if want_parity else None
    del J, D
    stage = soap.stage_times()
    soap.profile = None
    t_ms = sum(a.elapsed_time(b) for a, b in evs)
    if world > 1:
        tt = torch.tensor([t_ms], dtype=torch.float64, device=device)
        torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
        t_ms = float(tt.item())
    ms_per_step = t_ms / args.steps
    value = world * float(n_at) * args.steps / (t_ms / 1e3)

    # ---- roofline of the Jacobian kernel (HBM write stream) ----
    jac_ms = stage.get("jacobian", float("nan")) / args.steps
    jac_bytes = n_at * n_at * 3 * 420 * 4
    peak, peak_kind = _peaks()
    achieved = jac_bytes / (jac_ms / 1e3) / 1e9
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": _traffic_from_profiles() if args.nx == 10 else None, "kernel": "k_jacobian<3>",
                "peak_kind": f"{peak_kind} copy bandwidth (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured"
                else "fallback 6.65 TB/s",
                "algorithmic_bytes_per_launch": jac_bytes, "ms_per_launch": jac_ms,
                "stage_ms_per_step": {k: v / args.steps for k, v in stage.items()}}

    # ---- end to end: pinned host in, pinned host out ----
    e2e = None
    if not args.no_e2e:
        pos_h = torch.tensor(sysd["positions"], dtype=torch.float64).pin_memory()
        D_h = torch.empty((n_at, 420), dtype=torch.float32, pin_memory=True)
        # the Jacobian streams to the host through two 2 GB pinned buffers (every byte
        # crosses PCIe each step; host memory stays bounded with one process per GPU)
        chunk = 1 << 29  # floats
        bufs = [torch.empty(chunk, dtype=torch.float32, pin_memory=True) for _ in range(2)]
        done = [None, None]
        n_e2e = max(1, min(args.steps, args.e2e_steps))
        j_elems = n_at * n_at * 3 * 420

        def e2e_step():
            p = pos_h.to(device, non_blocking=True)
            J, D = soap.derivatives({"positions": p, "atomic_numbers": Z}, return_descriptor=True)
            flat = J.reshape(-1)
            for i, off in enumerate(range(0, flat.numel(), chunk)):
                k = i % 2
                if done[k] is not None:
                    done[k].synchronize()  # the previous copy into this buffer has landed
                n = min(chunk, flat.numel() - off)
                bufs[k][:n].copy_(flat[off:off + n], non_blocking=True)
                done[k] = torch.cuda.Event()
                done[k].record()
            D_h.copy_(D, non_blocking=True)
            del J, D, flat

        e2e_step()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(n_e2e):
            e2e_step()
        e1.record()
        barrier()
        te = e0.elapsed_time(e1)
        if world > 1:
            tt = torch.tensor([te], dtype=torch.float64, device=device)
            torch.distributed.all_reduce(tt, op=torch.distributed.ReduceOp.MAX)
            te = float(tt.item())
        e2e = {"value": world * float(n_at) * n_e2e / (te / 1e3), "unit": UNIT,
               "h2d_bytes_per_step": int(pos_h.numel() * 8 + n_at * 4),
               "d2h_bytes_per_step": int(j_elems * 4 + D_h.numel() * 4), "steps": n_e2e,
               "note": "positions from pinned host; descriptor and the full Jacobian copied back to pinned host "
                       "(the Jacobian through two 2 GB pinned buffers)"}
        del bufs, D_h

    extra = None
    if not args.no_batched and rank == 0:
        try:
            extra = batched_vs_plain(SOAP, torch)
        except Exception as exc:  # reported, never silently dropped
            extra = {"error": repr(exc)}

    scale = None
    diff = None
    if not args.no_batched and rank == 0 and args.nx == 10:
        try:
            scale = scale_create(SOAP, torch)
        except Exception as exc:  # reported, never silently dropped
            scale = {"error": repr(exc)}
        try:
            diff = diff_forces(SOAP, torch)
        except Exception as exc:
            diff = {"error": repr(exc)}

    plain192 = None
    if not args.no_batched and rank == 0 and world == 1 and args.nx == 10 and not args.no_cpu:
        try:
            plain192 = plain_cpu_cluster192(SOAP, torch)
        except Exception as exc:  # reported, never silently dropped
            plain192 = {"error": repr(exc)}

    cpu = None
    parity = None
    if want_parity:
        cpu, o_desc, o_jac = cpu_baseline_sample()
        parity = {"tolerance": {"descriptor": 1e-5, "derivative": 1e-4},
                  "headline_desc_max_row_rel_l2": _row_err(par_D, o_desc),
                  "headline_jacobian_max_centre_rel_l2": _row_err(par_J, o_jac),
                  "note": "relative L2 against float64 (the reference's port with float64 output): every "
                          "descriptor row of the last timed step, and the Jacobian blocks of 24 sampled centres"}
        del o_desc, o_jac
        try:
            parity.update(parity_other_legs(SOAP, torch))
        except Exception as exc:  # reported, never silently dropped
            parity["error"] = repr(exc)

    if world > 1:
        torch.distributed.barrier()
        torch.distributed.destroy_process_group()
    if rank != 0:
        return
    line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded)",
            "config": dict(CONFIG) if args.nx == 10
            else {"workload": f"profiling case: {n_at}-atom water cluster, same parameters"},
            "atoms_per_step": n_at, "parallelism": f"replicas x{world}" if world > 1 else "single GPU",
            "e2e": e2e, "gpu_launches": launches, "roofline": roofline, "clocks": clk, "cpu_baseline": cpu,
            "batched_vs_plain": extra, "scale_create": scale, "diff_forces": diff, "plain_cpu_cluster192": plain192,
            "reference_gpu_kernels": "unavailable on this box: the reference's Triton Jacobian kernels live in its "
                                     "Python package, which does not travel to the benchmark host, and its GPU "
                                     "path needs the sphericart CUDA library, which is not installed there",
            "parity_vs_fp64": parity}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--e2e-steps", type=int, default=3)
    ap.add_argument("--nx", type=int, default=10, help="lattice edge of the water cluster (10 = the workload; "
                                                         "smaller only for profiling captures)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batched-cells", type=int, default=0,
                    help="profiling case: run only the batched path on the first K cells")
    ap.add_argument("--scale-only", action="store_true",
                    help="profiling case: run only the 1,000,002-atom create() leg and print its object")
    ap.add_argument("--scale-mol", type=int, default=0,
                    help="with --scale-only: cut the cluster to this many molecules (smaller profiling case)")
    ap.add_argument("--diff-only", action="store_true",
                    help="profiling case: run only the 2001-atom differentiation leg (forces through the "
                         "adjoint) and print its object")
    args = ap.parse_args()
    if args.diff_only:
        import torch
        from cusoap_b200 import SOAP
        torch.cuda.set_device(0)
        print(json.dumps(diff_forces(SOAP, torch, steps=args.steps, warmup=args.warmup)), flush=True)
    elif args.scale_only:
        import torch
        from cusoap_b200 import SOAP
        torch.cuda.set_device(0)
        print(json.dumps(scale_create(SOAP, torch, steps=args.steps, warmup=args.warmup, n_mol=args.scale_mol)),
              flush=True)
    elif args.batched_cells > 0:
        run_batched_only(args)
    elif args.impl == "reference":
        run_reference(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()
