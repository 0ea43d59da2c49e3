"""Time the reference itself against its timed port (oracle/reference_port.py)
on the same inputs and host threads, and check that they agree.

The reference (TACC/cuSOAP ``src/cusoap/soap_generator.py``) is pure Python
and needs the third-party ``sphericart.torch``, absent here; the test-only
stand-in under ``oracle/sphericart_shim`` supplies it.  Its
``compute_with_gradients`` differentiates with autograd, one backward pass
per harmonic, where sphericart computes gradients in closed form, so the
reference's derivative time is reported both as measured and with the
stand-in's gradient time taken out (timed separately on the same edges).

    python oracle/calibrate_port.py /path/to/reference/src [threads]

Prints one JSON object: per workload, the median of 3 runs of the
reference and of the port, their ratio, and the relative L2 difference of
their outputs.  Run where the reference source exists; the benchmark host
does not have it.
"""
from __future__ import annotations

import json
import os
import sys
import time

import numpy as np
import torch

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _median_time(fn, reps=3):
    ts, out = [], None
    for _ in range(reps):
        t0 = time.perf_counter()
        out = fn()
        ts.append(time.perf_counter() - t0)
    return float(np.median(ts)), out


def _rel(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def main(ref_src: str, threads: int) -> None:
    sys.path.insert(0, os.path.join(HERE, "sphericart_shim"))
    sys.path.insert(0, ref_src)
    sys.path.insert(1, ROOT)
    torch.set_num_threads(threads)
    from cusoap import SOAP  # the reference package
    import sphericart.torch as shim
    from cusoap_b200 import workloads as W
    from oracle.reference_port import ReferencePort

    res = {"threads": threads}
    for name, centres in (("cluster192", None), ("cluster3000", list(range(0, 50)))):
        s = W.make(name)
        P = dict(W.CONFIGS[name])
        ref = SOAP(device="cpu", **P)
        port = ReferencePort(**P)
        pos, Z = s["positions"], s["atomic_numbers"]
        cen = None if centres is None else range(centres[0], centres[-1] + 1)
        t_rc, d_ref = _median_time(lambda: ref.create({"positions": pos, "atomic_numbers": Z}, centers=cen))
        t_rd, j_ref = _median_time(lambda: ref.derivatives({"positions": pos, "atomic_numbers": Z}, centers=cen,
                                                           method="analytical", return_descriptor=False))
        t_pc, d_port = _median_time(lambda: port.create(pos, Z, centres))
        t_pd, j_port = _median_time(lambda: port.derivatives(pos, Z, centres))
        # the stand-in's autograd gradients on the same edge vectors
        cxyz = torch.tensor(pos if centres is None else pos[centres])
        pt = torch.tensor(pos)
        ci, nj = torch.nonzero(torch.cdist(cxyz, pt) ** 2 <= ref._cutoff ** 2, as_tuple=True)
        rvec = pt[nj] - cxyz[ci]
        t_grad, _ = _median_time(lambda: shim.SolidHarmonics(P["l_max"]).compute_with_gradients(rvec))
        ref_step = t_rc + t_rd
        ref_step_sph = ref_step - t_grad
        port_step = t_pc + t_pd
        res[name] = {
            "centres": len(pos) if centres is None else len(centres),
            "reference_s": {"create": t_rc, "derivatives": t_rd, "stand_in_gradients": t_grad,
                            "step": ref_step, "step_without_stand_in_gradients": ref_step_sph},
            "port_s": {"create": t_pc, "derivatives": t_pd, "step": port_step},
            "port_over_reference": port_step / ref_step,
            "port_over_reference_without_stand_in_gradients": port_step / ref_step_sph,
            "rel_diff": {"create": _rel(d_port.numpy(), d_ref.numpy()),
                         "derivatives": _rel(j_port.numpy(), j_ref.numpy())},
        }
        print(name, json.dumps(res[name]), flush=True)
    print(json.dumps(res))


if __name__ == "__main__":
    main(sys.argv[1], int(sys.argv[2]) if len(sys.argv) > 2 else (os.cpu_count() or 1))
