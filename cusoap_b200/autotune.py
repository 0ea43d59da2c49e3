"""Autotuner for the launch shapes of the descriptor and adjoint kernels.

For one basis (n_max, l_max, species, crossover) on one GPU model it times,
with CUDA events on the launch stream, every candidate shape on a sample
system and keeps the fastest:

* descriptor: warps per block (1, 2, 4); for the l-grouped kernel (n_max
  > 8 or l_max > 6) also radial functions per lane (the minimum for n_max
  and l_max, and the next supported size above it: more functions per lane
  means fewer busy lanes but more independent work per lane; with two pair
  streams per warp only the warps per block);
* adjoint edge kernel: warps per block (1, 2, 4).

The choice is written into the basis (``soapb_basis.tune``), so every later
call of that SOAP object uses it; the candidates change only the launch
shape, not the arithmetic of any centre, so results are bitwise unchanged.
Results are cached per key in memory and, when ``CUSOAP_B200_TUNE_CACHE``
names a file (or ``cache_path`` is given), in a JSON file.
"""
from __future__ import annotations

import json
import os
import statistics
from typing import Any, Dict, List, Optional, Tuple

import torch

_GN_SIZES = (1, 2, 3, 4, 6)
_MEMORY: Dict[str, Dict[str, int]] = {}


def min_functions_per_lane(n_max: int, l_max: int) -> int:
    """Smallest supported functions-per-lane for the descriptor's lane map
    (floor(32 / (l_max+1)) lanes share each l)."""
    lanes = 32 // (l_max + 1)
    gn = -(-n_max // lanes)
    return 6 if gn == 5 else gn


def two_pair_streams(n_max: int, l_max: int) -> bool:
    """The descriptor kernel's lane map for (n_max, l_max) -- the rule of
    desc_two_streams in csrc/descriptor.cu: two pair streams per warp (its
    functions per lane fixed) for l_max <= 4 when one stream would leave more
    than a quarter of the lanes without a radial function."""
    if l_max > 4:
        return False
    lpl = 16 // (l_max + 1)
    if -(-n_max // lpl) > 3:
        return False
    gn = min_functions_per_lane(n_max, l_max)
    return (l_max + 1) * -(-n_max // gn) <= 24


def radial_index_lanes(n_max: int, l_max: int) -> bool:
    """The built-in descriptor kernel family for (n_max, l_max) -- the rule
    of DescDispatch in csrc/descriptor.cu: one lane per radial index n (all
    (l, m) accumulators in the lane) for n_max <= 8 and l_max <= 6, lanes
    grouped by l otherwise.  The tuner keeps the family (the two sum in
    different orders) and tunes only launch shapes within it."""
    return n_max <= 8 and l_max <= 6


def descriptor_candidates(n_max: int, l_max: int) -> List[Tuple[int, int]]:
    g0 = min_functions_per_lane(n_max, l_max)
    if radial_index_lanes(n_max, l_max) or two_pair_streams(n_max, l_max):
        # functions per lane are not a choice there
        return [(w, g0) for w in (1, 2, 4)]
    gns = [g for g in _GN_SIZES if g >= g0][:2]
    return [(w, g) for w in (1, 2, 4) for g in gns]


def tune_key(soap) -> str:
    name = torch.cuda.get_device_name(soap.device)
    return (f"{name}|N{soap._n_max}|L{soap._l_max}|S{soap.n_species}|x{int(soap.crossover)}|"
            f"rbf={soap._rbf}")


def _load(path: Optional[str]) -> Dict[str, Dict[str, int]]:
    if not path or not os.path.exists(path):
        return {}
    try:
        with open(path) as f:
            return json.load(f)
    except (OSError, ValueError):
        return {}


def _save(path: Optional[str], table: Dict[str, Dict[str, int]]) -> None:
    if not path:
        return
    tmp = path + ".tmp"
    with open(tmp, "w") as f:
        json.dump(table, f, indent=1, sort_keys=True)
    os.replace(tmp, path)


def apply(soap, choice: Dict[str, int]) -> None:
    soap._basis.tune[0] = int(choice.get("desc_wpb", 0))
    soap._basis.tune[1] = int(choice.get("desc_gn", 0))
    soap._basis.tune[2] = int(choice.get("force_wpb", 0))


def _time_stage(soap, fn, stage: str, reps: int) -> float:
    fn()  # warm-up (kernel attributes, caches)
    times = []
    for _ in range(reps):
        soap.profile = []
        fn()
        t = soap.stage_times().get(stage)
        soap.profile = None
        if t is not None:
            times.append(t)
    return statistics.median(times) if times else float("inf")


def autotune(soap, system: Any, reps: int = 3, cache_path: Optional[str] = None,
             force: bool = False) -> Dict[str, Any]:
    """Pick and apply the fastest launch shapes of ``soap`` on ``system`` (a
    structure or list of structures typical of the intended workload).
    Returns the choice with the measured stage times in ms."""
    cache_path = cache_path or os.environ.get("CUSOAP_B200_TUNE_CACHE")
    key = tune_key(soap)
    table = _load(cache_path)
    table.update(_MEMORY)
    if not force and key in table:
        apply(soap, table[key])
        return dict(table[key], cached=True)

    systems = system if isinstance(system, list) else [system]

    def desc():
        with torch.no_grad():
            soap.create(systems if len(systems) > 1 else systems[0])

    result: Dict[str, Any] = {}
    best = None
    for wpb, gn in descriptor_candidates(soap._n_max, soap._l_max):
        apply(soap, {"desc_wpb": wpb, "desc_gn": gn})
        t = _time_stage(soap, desc, "descriptor", reps)
        result[f"descriptor_ms[wpb={wpb},gn={gn}]"] = t
        if best is None or t < best[0]:
            best = (t, wpb, gn)
    choice = {"desc_wpb": best[1], "desc_gn": best[2], "force_wpb": 0}

    if soap.average != "cc" and all(isinstance(sd, dict) for sd in systems):
        rng = torch.Generator().manual_seed(0)
        w = torch.randn(soap.get_number_of_features(), generator=rng).to(soap.device)

        def adjoint():
            parts = []
            for sd in systems:
                p = torch.as_tensor(sd["positions"], dtype=torch.float64, device=soap.device)
                parts.append(dict(sd, positions=p.clone().requires_grad_(True)))
            out = soap.create(parts if len(parts) > 1 else parts[0])
            out = torch.cat(out) if isinstance(out, list) else out.reshape(-1, out.shape[-1])
            (out * w).sum().backward()

        bestf = None
        for wpb in (1, 2, 4):
            apply(soap, dict(choice, force_wpb=wpb))
            t = _time_stage(soap, adjoint, "forces", reps)
            result[f"forces_ms[wpb={wpb}]"] = t
            if bestf is None or t < bestf[0]:
                bestf = (t, wpb)
        choice["force_wpb"] = bestf[1]

    apply(soap, choice)
    _MEMORY[key] = choice
    table[key] = choice
    _save(cache_path, table)
    return dict(choice, timings_ms=result, cached=False)
