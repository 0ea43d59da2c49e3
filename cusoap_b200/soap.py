"""Drop-in ``SOAP`` class: the reference's public surface over libsoapb200.

Mirrors ``SOAP`` of the reference (TACC/cuSOAP ``src/cusoap/soap_generator.py``,
cited as SG:<line>): the constructor (SG:524-634), ``create``/``generate``
(SG:1691-1757), ``derivatives`` (SG:2628-2699), ``get_number_of_features`` /
``get_location`` (SG:908-962), and the same input adapters (SG:291-332) and
centre handling (SG:966-1003).  All compute runs in the CUDA library; this
module only prepares device buffers (torch tensors) and calls the C ABI.

Differences from the reference, by design:
* the bulk arithmetic is float32 on the GPU (the reference always computes in
  float64, SG:1775-1780); the radial basis is orthonormalised in float64 on
  the GPU and stored as accurate float32 tables, see ``csrc/basis.cu``;
* a list of systems goes through ONE batched launch (the reference loops,
  SG:1716-1733);
* ``create`` is differentiable w.r.t. positions given as a tensor with
  ``requires_grad``: the backward pass is a hand-written adjoint kernel
  (the reference reaches the same gradient only through autograd);
* ``derivatives`` uses the closed-form Jacobian kernel for every case it
  supports (periodic systems, weighting and ``attach=True`` included), where
  the reference falls back to a batched-autograd Jacobian (SG:2677-2698);
* the polynomial basis's radial integrals are evaluated with an accurate
  series / recurrence split of the scaled Bessel functions when the tables
  are built; the reference's clamped upward recurrence differs from it for
  high l at small r (t = 2 eta rx r < l).
"""
from __future__ import annotations

import ctypes
import math
from typing import Any, Dict, List, Optional, Sequence, Tuple, Union

import numpy as np
import torch

from . import _lib
from ._lib import Basis, Centres, Structs, check

from .xyz import ATOMIC_NUMBERS as _SYMBOLS


# Parameter limits of the compiled kernels (csrc/common.cuh kMaxN, kMaxL, kMaxS).
MAX_N_MAX, MAX_L_MAX, MAX_SPECIES = 16, 12, 16
# l_max 10-12 are built for n_max up to 8 (two lanes per l, four radial functions per lane)
MAX_N_MAX_HIGH_L = 8
# Per-centre (row, edge) entries (one per neighbour pair of an included atom,
# two with attach=True) that the Jacobian sorts in shared memory in one tile;
# centres with more are sorted in tiles and merged in the workspace.
JACOBIAN_TILE_ENTRIES = 8192

_F64_WARNED = False


def _warn_float64():
    """dtype='float64' returns float64 tensors, but the descriptor and its
    derivatives are computed in float32 (about 1e-6 relative error against
    float64, within the 1e-5 / 1e-4 tolerances); the reference computes them
    in float64 (SG:1775-1780).  Said once per process."""
    global _F64_WARNED
    if not _F64_WARNED:
        _F64_WARNED = True
        import warnings
        warnings.warn("cusoap_b200: dtype='float64' returns float64 tensors computed in float32 on the GPU "
                      "(about 1e-6 relative error against float64); only the radial basis is built in float64",
                      stacklevel=3)


def _ptr(t: Optional[torch.Tensor]) -> Optional[int]:
    return None if t is None else t.data_ptr()


def _stream(device: torch.device) -> int:
    return torch.cuda.current_stream(device).cuda_stream


def _resolve_z(s) -> int:
    if isinstance(s, str):
        try:
            import ase.data  # optional, as in the reference (SG:555-559)
            return int(ase.data.atomic_numbers[s])
        except Exception:
            if s in _SYMBOLS:
                return _SYMBOLS[s]
            raise ValueError(f"Cannot resolve species symbol '{s}'. Install ASE or use atomic numbers.")
    return int(s)


def _as_positions(x):
    """A torch tensor stays as it is (autograd flows through it); anything
    else becomes a float64 (n, 3) numpy array."""
    if isinstance(x, torch.Tensor):
        return x
    return np.asarray(x, dtype=np.float64).reshape(-1, 3)


def _as_numbers(x) -> np.ndarray:
    """Atomic numbers as a host int64 array."""
    if isinstance(x, torch.Tensor):
        return x.detach().cpu().numpy().astype(np.int64)
    return np.asarray(x, dtype=np.int64).reshape(-1)


class _Weighting:
    """DScribe weighting parameters (SG:403-470); the functions themselves
    are evaluated on the device when the radial tables are built."""

    def __init__(self, function: Optional[str] = None, r0: float = 1.0, c: float = 1.0, d: float = 1.0,
                 m: float = 1.0, w0: float = 1.0):
        if function not in (None, "poly", "pow", "exp"):
            raise ValueError(f"Unknown weighting function: {function}")
        self.function, self.r0, self.c, self.d, self.m, self.w0 = function, float(r0), float(c), float(d), \
            float(m), float(w0)

    def infer_rcut(self, threshold: float = 1e-2) -> float:
        """r_cut where the weight falls to `threshold` (SG:422-438)."""
        if self.function is None:
            raise ValueError("Cannot infer r_cut when weighting.function is None; provide r_cut explicitly.")
        if self.function == "poly":
            return self.r0
        val = self.c / threshold - self.d
        if val <= 0:
            raise ValueError(f"Invalid weighting: c/threshold - d must be >0 for {self.function}.")
        if self.function == "pow":
            return self.r0 * val ** (1.0 / self.m)
        return -self.r0 * math.log(val)


def _poly_grid(r_cut: float, n_max: int, quad_n: int) -> np.ndarray:
    """DScribe polynomial basis on its Gauss-Legendre grid: rx | wr | g_n(rx),
    float64, with g = sqrtm(inv(S)) (r_cut - rx)^(k+2) computed as the
    reference does it (SG:710-752, nodes by Golub-Welsch SG:350-362).  The
    overlap S is so ill-conditioned that only this exact sequence of FP64
    operations reproduces the reference's basis; it runs once per SOAP object
    on the host, like the reference's own set-up."""
    from scipy.linalg import sqrtm
    n, rc = int(n_max), float(r_cut)
    S = np.zeros((n, n))
    for i in range(1, n + 1):
        for j in range(1, n + 1):
            S[i - 1, j - 1] = (2 * rc ** (7 + i + j)) / ((5 + i + j) * (6 + i + j) * (7 + i + j))
    betas = sqrtm(np.linalg.inv(S))
    if np.iscomplexobj(betas):
        raise ValueError("Could not calculate normalization factors for the radial basis in the domain of real "
                         "numbers. Lowering the number of radial basis functions (n_max) or increasing the radial "
                         "cutoff (r_cut) is advised.")
    k = np.arange(1, quad_n, dtype=np.float64)
    beta = k / np.sqrt(4.0 * k * k - 1.0)
    x, V = np.linalg.eigh(np.diag(beta, 1) + np.diag(beta, -1))
    w = 2.0 * V[0, :] ** 2
    rx = rc * 0.5 * (x + 1.0)
    wr = rc * 0.5 * w
    fs = np.stack([(rc - np.clip(rx, 0.0, rc)) ** (kk + 2) for kk in range(1, n + 1)])
    g = np.ascontiguousarray(betas) @ fs
    return np.ascontiguousarray(np.concatenate([rx, wr, g.reshape(-1)]), dtype=np.float64)


class _Batch:
    """Device buffers describing a batch of structures and their centres.
    Host arrays are concatenated first and copied with one transfer each."""

    def __init__(self, soap: "SOAP", systems: List[Any], centers_list: List[Optional[Sequence[Any]]]):
        dev = soap.device
        raw = [soap._system_arrays(s) for s in systems]
        counts_a = [int(r[0].shape[0]) for r in raw]
        atom_off = np.concatenate([[0], np.cumsum(counts_a)]).astype(np.int64)
        self.atom_off_list = atom_off.tolist()
        self.n_atoms = int(atom_off[-1])
        self.pos_tensors = [r[0] for r in raw if isinstance(r[0], torch.Tensor)]
        host_pos = all(isinstance(r[0], np.ndarray) for r in raw)
        Zall = np.concatenate([r[1] for r in raw]) if raw else np.zeros(0, np.int64)
        cells = np.zeros((len(raw), 9))
        pbcs = np.zeros((len(raw), 3), np.uint8)
        if soap.periodic:
            if any(r[2] is None or r[3] is None for r in raw):
                raise ValueError("periodic=True requires cell and pbc.")
            try:  # one conversion for the whole list (numpy / nested-list cells and flags)
                if any(isinstance(r[2], torch.Tensor) or isinstance(r[3], torch.Tensor) for r in raw):
                    raise TypeError
                cells[:] = np.asarray([r[2] for r in raw], dtype=np.float64).reshape(len(raw), 9)
                pbcs[:] = np.asarray([r[3] for r in raw], dtype=bool).reshape(len(raw), 3)
            except (TypeError, ValueError):
                for i, r in enumerate(raw):
                    cells[i] = np.asarray(r[2].detach().cpu() if isinstance(r[2], torch.Tensor) else r[2],
                                          dtype=np.float64).reshape(9)
                    pbcs[i] = np.asarray(r[3].detach().cpu() if isinstance(r[3], torch.Tensor) else r[3],
                                         dtype=bool).reshape(3)
        all_atoms = all(c is None for c in centers_list)
        # Structures evaluated again with new device positions (an MD or relaxation loop) reuse
        # the device copies of their species, offsets, cells, pbc and centre indices: the
        # atomic numbers, cells and flags are compared with the cached ones on the host.
        cached = soap._topology if (all_atoms and not host_pos) else None
        if cached is not None and not (cached["counts"] == counts_a and np.array_equal(cached["Z"], Zall)
                                       and np.array_equal(cached["cells"], cells)
                                       and np.array_equal(cached["pbcs"], pbcs)):
            cached = None
        if cached is not None:
            dev_arrays = cached["dev"]
        else:
            # the small host arrays (and host positions) go to the device in ONE
            # asynchronous copy from a pinned staging buffer
            arrays = [("species", soap._species_lookup(Zall)), ("atom_off", atom_off), ("cells", cells),
                      ("pbc", pbcs)]
            if all_atoms:
                arrays.append(("centre_struct", np.repeat(np.arange(len(raw), dtype=np.int32), counts_a)))
                arrays.append(("centre_atom", np.arange(int(atom_off[-1]), dtype=np.int32)))
            if host_pos:
                host = np.concatenate([r[0] for r in raw]) if raw else np.zeros((0, 3))
                arrays.append(("positions", np.ascontiguousarray(host, dtype=np.float64)))
            dev_arrays = soap._upload(arrays)
            if all_atoms and not host_pos:
                soap._topology = {"counts": list(counts_a), "Z": Zall.copy(), "cells": cells.copy(),
                                  "pbcs": pbcs.copy(), "dev": dev_arrays}
        self.species, self.atom_off = dev_arrays["species"], dev_arrays["atom_off"]
        self.cells, self.pbc = dev_arrays["cells"], dev_arrays["pbc"]
        if host_pos:
            self.positions = dev_arrays["positions"]
            self.pos_tensors = []
        elif all(isinstance(r[0], torch.Tensor) and r[0].device == dev for r in raw):
            # device tensors: one concatenation, one conversion
            self.positions = torch.cat([r[0].detach() for r in raw]).to(torch.float64).contiguous()
        else:
            parts = [r[0].detach().to(dev, torch.float64) if isinstance(r[0], torch.Tensor)
                     else torch.as_tensor(r[0], dtype=torch.float64, device=dev) for r in raw]
            self.positions = torch.cat(parts).contiguous()
        if all_atoms:
            # every atom is a centre, attached to itself (SG:977-979)
            self.counts = counts_a
            self.n_centres = self.n_atoms
            self.centre_xyz = self.positions
            self.centre_atom = dev_arrays["centre_atom"]
            self.centre_attach = self.centre_atom
            self.centre_struct = dev_arrays["centre_struct"]
        else:
            cxyz, cstruct, catom, cattach, self.counts = [], [], [], [], []
            for i, cen in enumerate(centers_list):
                pos_i = self.positions[self.atom_off_list[i]:self.atom_off_list[i + 1]]
                xyz, atom, attach = soap._prepare_centres(pos_i, cen)
                off = self.atom_off_list[i]
                cxyz.append(xyz)
                catom.append(torch.where(atom >= 0, atom + off, atom))
                cattach.append(torch.where(attach >= 0, attach + off, attach))
                cstruct.append(torch.full((xyz.shape[0],), i, dtype=torch.int32, device=dev))
                self.counts.append(int(xyz.shape[0]))
            self.n_centres = sum(self.counts)
            self.centre_xyz = torch.cat([c.detach() for c in cxyz]).contiguous()
            self.centre_struct = torch.cat(cstruct).contiguous()
            self.centre_atom = torch.cat(catom).to(torch.int32).contiguous()
            self.centre_attach = torch.cat(cattach).to(torch.int32).contiguous()
        self._describe(len(raw))

    def _describe(self, n_struct: int):
        self.cs = Structs(n_struct, self.n_atoms, _ptr(self.atom_off), _ptr(self.positions),
                          _ptr(self.species), _ptr(self.cells), _ptr(self.pbc))
        self.cc = Centres(self.n_centres, _ptr(self.centre_xyz), _ptr(self.centre_struct), _ptr(self.centre_atom))

    @classmethod
    def from_device(cls, counts_a: List[int], positions: torch.Tensor, species: torch.Tensor, cells: torch.Tensor,
                    pbc: torch.Tensor, centre_xyz: torch.Tensor, centre_struct: torch.Tensor,
                    centre_atom: torch.Tensor, centre_attach: torch.Tensor, counts: List[int]) -> "_Batch":
        """A batch from arrays already on the device (structures' atoms
        concatenated, counts_a atoms each; centres concatenated, counts per
        structure).  No host-side adapters and no copies."""
        self = cls.__new__(cls)
        dev = positions.device
        atom_off = np.concatenate([[0], np.cumsum(counts_a)]).astype(np.int64)
        self.atom_off_list = atom_off.tolist()
        self.n_atoms = int(atom_off[-1])
        self.pos_tensors = []
        self.atom_off = torch.as_tensor(atom_off).to(dev)
        self.positions = positions.contiguous()
        self.species = species.to(torch.int32).contiguous()
        self.cells = cells.to(torch.float64).reshape(-1, 9).contiguous()
        self.pbc = pbc.to(torch.uint8).reshape(-1, 3).contiguous()
        self.counts = list(counts)
        self.n_centres = int(sum(self.counts))
        self.centre_xyz = centre_xyz.to(torch.float64).contiguous()
        self.centre_struct = centre_struct.to(torch.int32).contiguous()
        self.centre_atom = centre_atom.to(torch.int32).contiguous()
        self.centre_attach = centre_attach.to(torch.int32).contiguous()
        self._describe(len(counts_a))
        return self


class _Pairs:
    """CSR pair list on the device (from soapb_neighbors_count/_fill)."""

    def __init__(self, soap: "SOAP", batch: _Batch, mode: int):
        lib = _lib.load()
        dev = soap.device
        st = _stream(dev)
        ws = ctypes.c_int64(0)
        b = ctypes.byref(soap._basis)
        check(lib.soapb_neighbors_workspace(b, ctypes.byref(batch.cs), ctypes.byref(batch.cc), ctypes.byref(ws)))
        self.work = torch.empty(max(int(ws.value), 256), dtype=torch.uint8, device=dev)
        self.pair_off = torch.empty(batch.n_centres + 1, dtype=torch.int64, device=dev)
        soap._call("neighbors_count", lib.soapb_neighbors_count, b, ctypes.byref(batch.cs), ctypes.byref(batch.cc),
                   mode, _ptr(self.work), self.work.numel(), _ptr(self.pair_off), st)
        # one device->host read: total pairs, largest per-centre count, status flags
        stats = torch.empty(3, dtype=torch.int64, device=dev)
        soap._call("neighbors_stats", lib.soapb_neighbors_stats, b, ctypes.byref(batch.cs), ctypes.byref(batch.cc),
                   _ptr(self.work), _ptr(self.pair_off), _ptr(stats), st)
        self.total, self.max_pairs, status = (int(v) for v in stats.cpu().tolist())
        if status & 1:
            raise ValueError("singular cell in a periodic structure")
        if status & 2:
            raise ValueError("an atom lies more than 511 cells outside its periodic cell")
        if status & 8:
            raise RuntimeError("neighbour enumeration: a window row exceeded its run limit")
        if status:
            raise _lib.SoapbError(_lib.ERR_CAPACITY, f"neighbour list status {status}")
        # the list is allocated to the exact total, so the fill cannot overflow it
        self.pairs = torch.empty((max(self.total, 1), 4), dtype=torch.float32, device=dev)
        soap._call("neighbors_fill", lib.soapb_neighbors_fill, b, ctypes.byref(batch.cs), ctypes.byref(batch.cc),
                   mode, _ptr(self.work), self.work.numel(), _ptr(self.pair_off), _ptr(self.pairs), self.total, st)


class _SOAPFunction(torch.autograd.Function):
    """Descriptor of one batch as a differentiable function of the positions;
    the backward pass is the adjoint kernel (soapb_forces)."""

    @staticmethod
    def forward(ctx, positions, soap, batch, mode):
        pairs = _Pairs(soap, batch, _lib.NL_ALL)
        desc, coeff = soap._run_descriptor(batch, pairs, mode, want_coeff=True)
        ctx.soap, ctx.batch, ctx.pairs, ctx.coeff, ctx.mode = soap, batch, pairs, coeff, mode
        return desc

    @staticmethod
    def backward(ctx, grad_out):
        soap, batch, pairs = ctx.soap, ctx.batch, ctx.pairs
        forces = soap._run_forces(batch, pairs, ctx.coeff, grad_out.contiguous().to(torch.float32), attach=True,
                                  mode=ctx.mode)
        return (-forces).to(torch.float64), None, None, None


class SOAPBatch:
    """A fixed batch of structures (every atom a centre) whose descriptor and
    adjoint run as two captured CUDA graphs, for loops that re-evaluate the
    same structures at new positions (molecular dynamics, relaxations).

    Built by ``SOAP.batch(systems)``.  All buffers are allocated once: the
    pair buffer with ``headroom`` over the first neighbour count.  Per call,
    ``create(positions)`` copies the positions into the batch's position
    buffer and replays the forward graph (neighbour count and fill, a clamp
    that empties the lists if they overflowed the pair buffer, descriptor);
    the one device-to-host read checks the pair total, and an overflow
    rebuilds the plan with a larger buffer and replays.  The backward graph is
    the adjoint: ``create`` is differentiable w.r.t. ``positions``.

    The descriptor returned is the plan's output buffer, overwritten by the
    next replay (clone it to keep it).  Cells, pbc, species and atom counts
    are fixed per plan.
    """

    def __init__(self, soap: "SOAP", systems: List[Any], headroom: float = 1.25):
        self.soap = soap
        self.mode = soap._out_mode()
        self.headroom = float(headroom)
        with torch.cuda.device(soap.device):
            self.b = _Batch(soap, systems, [None] * len(systems))
            self.counts = list(self.b.counts)
            self.n_atoms = self.b.n_atoms
            self._build(capacity=None)

    def _build(self, capacity):
        soap, b, lib, dev = self.soap, self.b, _lib.load(), self.soap.device
        C = b.n_centres
        st = _stream(dev)
        ws = ctypes.c_int64(0)
        check(lib.soapb_neighbors_workspace(ctypes.byref(soap._basis), ctypes.byref(b.cs), ctypes.byref(b.cc),
                                            ctypes.byref(ws)))
        self.work = torch.empty(max(int(ws.value), 256), dtype=torch.uint8, device=dev)
        self.pair_off = torch.empty(C + 1, dtype=torch.int64, device=dev)
        self.total = torch.zeros(1, dtype=torch.int64, device=dev)
        if capacity is None:
            check(lib.soapb_neighbors_count(ctypes.byref(soap._basis), ctypes.byref(b.cs), ctypes.byref(b.cc),
                                            _lib.NL_ALL, _ptr(self.work), self.work.numel(), _ptr(self.pair_off), st))
            capacity = int(int(self.pair_off[-1].item()) * self.headroom) + 1024
        self.capacity = int(capacity)
        self.pairs = torch.empty((self.capacity, 4), dtype=torch.float32, device=dev)
        F, FC = int(soap._basis.n_feat_ps), int(soap._basis.n_feat_cc)
        F = FC if self.mode == _lib.OUT_CC else F
        self.desc = torch.empty((C, F), dtype=torch.float32, device=dev)
        self.coeff = torch.empty((C, FC), dtype=torch.float32, device=dev)
        self.dEdp = torch.empty((C, F), dtype=torch.float32, device=dev)
        self.forces = torch.empty((b.n_atoms, 3), dtype=torch.float32, device=dev)
        wsb = ctypes.c_int64(0)
        check(lib.soapb_forces_workspace(ctypes.byref(soap._basis), C, ctypes.byref(wsb)))
        self.fwork = torch.empty(max(int(wsb.value), 256), dtype=torch.uint8, device=dev)
        self.counter = torch.zeros(1, dtype=torch.int32, device=dev)
        # run once eagerly (sets kernel attributes), then capture both graphs
        self._forward_calls()
        self._backward_calls()
        torch.cuda.synchronize(dev)
        self.g_fwd, self.g_bwd = torch.cuda.CUDAGraph(), torch.cuda.CUDAGraph()
        with torch.cuda.graph(self.g_fwd):
            self._forward_calls()
        with torch.cuda.graph(self.g_bwd):
            self._backward_calls()
        torch.cuda.synchronize(dev)

    def _forward_calls(self):
        soap, b, lib = self.soap, self.b, _lib.load()
        st = _stream(soap.device)
        bb, cs, cc = ctypes.byref(soap._basis), ctypes.byref(b.cs), ctypes.byref(b.cc)
        check(lib.soapb_neighbors_count(bb, cs, cc, _lib.NL_ALL, _ptr(self.work), self.work.numel(),
                                        _ptr(self.pair_off), st))
        check(lib.soapb_neighbors_fill(bb, cs, cc, _lib.NL_ALL, _ptr(self.work), self.work.numel(),
                                       _ptr(self.pair_off), _ptr(self.pairs), self.capacity, st))
        check(lib.soapb_neighbors_clamp(_ptr(self.pair_off), b.n_centres, self.capacity, _ptr(self.total), st))
        check(lib.soapb_descriptor(bb, b.n_centres, _ptr(self.pair_off), _ptr(self.pairs), self.mode,
                                   _ptr(self.desc), _ptr(self.coeff), _ptr(self.counter), st))

    def _backward_calls(self):
        soap, b, lib = self.soap, self.b, _lib.load()
        self.forces.zero_()
        check(lib.soapb_forces(ctypes.byref(soap._basis), b.n_centres, _ptr(self.pair_off), _ptr(self.pairs),
                               _ptr(self.coeff), _ptr(self.dEdp), self.mode, _ptr(b.centre_attach), 1,
                               _ptr(self.forces),
                               _ptr(self.fwork), self.fwork.numel(), _ptr(self.counter), _stream(soap.device)))

    def _replay_forward(self, positions: Optional[torch.Tensor]):
        if positions is not None:
            self.b.positions.copy_(positions.detach().reshape(-1, 3))
        self.g_fwd.replay()
        need = int(self.total.item())
        if need > self.capacity:  # the lists outgrew the pair buffer: re-plan and run again
            self._build(capacity=int(need * self.headroom) + 1024)
            self.g_fwd.replay()
        return self.desc

    def create(self, positions: Optional[torch.Tensor] = None) -> torch.Tensor:
        """(n_atoms, F) descriptors of the whole batch at ``positions``
        ((n_atoms, 3), the structures' atoms concatenated; None: unchanged).
        Differentiable w.r.t. ``positions`` through the adjoint graph."""
        with torch.cuda.device(self.soap.device):
            if positions is not None and torch.is_grad_enabled() and positions.requires_grad:
                return _BatchFunction.apply(positions, self)
            return self._replay_forward(positions)

    def forces_from(self, dEdp: torch.Tensor) -> torch.Tensor:
        """-dE/dx (n_atoms, 3) for a given dE/dp (n_atoms, F), at the
        positions of the last ``create``."""
        with torch.cuda.device(self.soap.device):
            self.dEdp.copy_(dEdp)
            self.g_bwd.replay()
            return self.forces

    def split(self, out: torch.Tensor) -> List[torch.Tensor]:
        """Per-structure views of a batch output."""
        return list(torch.split(out, self.counts))


class _BatchFunction(torch.autograd.Function):
    @staticmethod
    def forward(ctx, positions, plan):
        ctx.plan = plan
        ctx.dtype = positions.dtype
        return plan._replay_forward(positions)

    @staticmethod
    def backward(ctx, grad_out):
        forces = ctx.plan.forces_from(grad_out.contiguous().to(torch.float32))
        return (-forces).to(ctx.dtype), None


class SOAP:
    """DScribe-compatible SOAP on B200 (see the module docstring)."""

    def __init__(
        self,
        r_cut: Optional[float] = None,
        n_max: Optional[int] = None,
        l_max: Optional[int] = None,
        sigma: float = 1.0,
        rbf: str = "gto",
        weighting: Optional[Dict[str, Any]] = None,
        crossover: bool = True,
        average: str = "off",
        species: Optional[Sequence[Union[int, str]]] = None,
        periodic: bool = False,
        sparse: bool = False,
        dtype: str = "float32",
        device: Optional[Union[str, torch.device]] = None,
        quad_n: int = 100,
        max_num_neighbors: Optional[int] = None,
    ):
        # argument checks and messages follow SG:542-602
        if n_max is None or l_max is None:
            raise ValueError("n_max and l_max must be provided.")
        if species is None or len(species) == 0:
            raise ValueError("species must be provided (list of atomic numbers or symbols).")
        if dtype not in ("float32", "float64"):
            raise ValueError("dtype must be 'float32' or 'float64'")
        if dtype == "float64":
            _warn_float64()
        self._dtype_str = dtype
        self.dtype = torch.float32 if dtype == "float32" else torch.float64
        species_Z = [_resolve_z(s) for s in species]
        self._atomic_numbers_list = sorted(set(species_Z))
        self._atomic_number_set = set(self._atomic_numbers_list)
        self._Z_to_species_index = {z: i for i, z in enumerate(self._atomic_numbers_list)}
        self.n_species = len(self._atomic_numbers_list)
        self._n_max = int(n_max)
        self._l_max = int(l_max)
        # limits of the compiled kernels (the reference has none): refused here, before any device work
        if not 1 <= self._n_max <= MAX_N_MAX:
            raise ValueError(f"n_max must be in [1, {MAX_N_MAX}] (the CUDA kernels are built up to n_max "
                             f"{MAX_N_MAX}); got {self._n_max}")
        if not 0 <= self._l_max <= MAX_L_MAX:
            raise ValueError(f"l_max must be in [0, {MAX_L_MAX}] (the CUDA kernels are built up to l_max "
                             f"{MAX_L_MAX}); got {self._l_max}")
        if self._l_max >= 10 and self._n_max > MAX_N_MAX_HIGH_L:
            raise ValueError(f"n_max must be <= {MAX_N_MAX_HIGH_L} for l_max >= 10 (the CUDA kernels are built "
                             f"for that); got n_max {self._n_max}, l_max {self._l_max}")
        if self.n_species > MAX_SPECIES:
            raise ValueError(f"at most {MAX_SPECIES} species are supported (the CUDA kernels are built up to "
                             f"{MAX_SPECIES}); got {self.n_species}")
        self.device = torch.device(device) if device is not None else torch.device("cuda")
        if self.device.type != "cuda":
            raise ValueError("cusoap_b200 runs on CUDA devices only (no CPU fallback)")
        if self.device.index is None:
            self.device = torch.device("cuda", torch.cuda.current_device())
        self._sigma = float(sigma)
        self._eta = 1.0 / (2.0 * self._sigma * self._sigma)
        self._rbf = str(rbf).lower()
        self.crossover = bool(crossover)
        self.average = str(average)
        self.periodic = bool(periodic)
        self.sparse = bool(sparse)
        self.quad_n = int(quad_n)
        self.max_num_neighbors = max_num_neighbors
        if self.average not in ("off", "inner", "outer", "cc"):
            raise ValueError("average must be one of: 'off', 'inner', 'outer', 'cc' (cc = projection coeffs).")
        if self._rbf not in ("gto", "polynomial"):
            raise ValueError("rbf must be 'gto' or 'polynomial'.")
        # weighting dict as DScribe's: may carry 'threshold' for the r_cut inference (SG:584-597)
        self._weighting_dict = dict(weighting) if weighting is not None else None
        self._weighting = None
        thr = 1e-2
        if self._weighting_dict is not None:
            thr = float(self._weighting_dict.get("threshold", 1e-2))
            self._weighting = _Weighting(**{k: v for k, v in self._weighting_dict.items() if k != "threshold"})
        if r_cut is None:
            if self._weighting is None:
                raise ValueError("Either r_cut or weighting must be provided.")
            self._r_cut = float(self._weighting.infer_rcut(thr))
        else:
            self._r_cut = float(r_cut)
        self._cutoff_padding = float(self._sigma * math.sqrt(-2.0 * math.log(1e-3)))  # SG:600-602
        self._cutoff = self._r_cut + self._cutoff_padding
        self._poly_grid = _poly_grid(self._r_cut, self._n_max, self.quad_n) if self._rbf == "polynomial" else None
        self._build_basis()
        self._counter = torch.zeros(1, dtype=torch.int32, device=self.device)
        self._topology = None  # device copies of the last batch's species, offsets, cells (see _Batch)
        self.n_features = int(self.get_number_of_features())
        # When a list, every library call appends (name, start_event, end_event)
        # recorded on the launch stream (per-stage GPU timing).
        self.profile: Optional[list] = None

    def _build_basis(self):
        """Plan and build the basis on the device; tables whose error exceeds
        1e-6 are rebuilt on finer segments (weighting functions with a sharp
        feature need them)."""
        lib = _lib.load()
        w = self._weighting
        seg_hint = 0
        while True:
            b = Basis()
            b.n_max, b.l_max, b.n_species, b.crossover = self._n_max, self._l_max, self.n_species, int(self.crossover)
            b.r_cut, b.sigma = self._r_cut, self._sigma
            b.rbf = _lib.RBF_POLY if self._rbf == "polynomial" else _lib.RBF_GTO
            if w is None:
                b.weighting = _lib.W_NONE
            else:
                b.weighting = {None: _lib.W_W0, "poly": _lib.W_POLY, "pow": _lib.W_POW, "exp": _lib.W_EXP}[w.function]
                b.w_r0, b.w_c, b.w_d, b.w_m, b.w_w0 = w.r0, w.c, w.d, w.m, w.w0
            if self._poly_grid is not None:
                b.quad_n = self.quad_n
                b.h_poly = self._poly_grid.ctypes.data
            b.seg_hint = seg_hint
            check(lib.soapb_basis_plan(ctypes.byref(b)))
            with torch.cuda.device(self.device):
                buf = torch.empty(int(b.bytes), dtype=torch.uint8, device=self.device)
                check(lib.soapb_basis_build(ctypes.byref(b), _ptr(buf), _stream(self.device)))
                L1, N = self._l_max + 1, self._n_max
                alphas, betas, err = np.zeros((L1, N)), np.zeros((L1, N, N)), np.zeros(2)
                check(lib.soapb_basis_download(ctypes.byref(b), alphas.ctypes.data, betas.ctypes.data,
                                               err.ctypes.data, _stream(self.device)))
            self.table_error = (float(err[0]), float(err[1]))
            if max(self.table_error) <= 1e-6:
                break
            if (2 * b.n_seg) * self.n_species > 1024:
                raise _lib.SoapbError(_lib.ERR_ACCURACY, f"radial table error {self.table_error} above 1e-6 "
                                      f"with {b.n_seg} segments (weighting too sharp for the FP32 tables)")
            seg_hint = 2 * b.n_seg
        self._basis, self._basis_buf = b, buf
        self._alphas, self._betas = alphas, betas

    def _call(self, name, fn, *args):
        prof = self.profile
        if prof is None:
            check(fn(*args))
            return
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record()
        rc = fn(*args)
        e1.record()
        prof.append((name, e0, e1))
        check(rc)

    def stage_times(self) -> Dict[str, float]:
        """Milliseconds per library stage recorded in ``self.profile``
        (synchronises)."""
        torch.cuda.synchronize(self.device)
        out: Dict[str, float] = {}
        for name, e0, e1 in self.profile or []:
            out[name] = out.get(name, 0.0) + e0.elapsed_time(e1)
        return out

    # ---- DScribe-like helpers (SG:908-962) ----
    def get_number_of_features(self) -> int:
        if self.average == "cc":
            return int(self._basis.n_feat_cc)
        return int(self._basis.n_feat_ps)

    def get_location(self, species_pair: Tuple[Union[int, str], Union[int, str]]) -> slice:
        if self.average == "cc":
            raise ValueError("get_location is not defined for average='cc' (projection coefficients).")
        if len(species_pair) != 2:
            raise ValueError("species_pair must be length-2.")
        Z1, Z2 = _resolve_z(species_pair[0]), _resolve_z(species_pair[1])
        if Z1 not in self._atomic_number_set or Z2 not in self._atomic_number_set:
            raise ValueError("Species not present in descriptor species list.")
        i, j = self._Z_to_species_index[Z1], self._Z_to_species_index[Z2]
        if i > j:
            i, j = j, i
        symm = (self._n_max * (self._n_max + 1) // 2) * (self._l_max + 1)
        unsymm = (self._n_max * self._n_max) * (self._l_max + 1)
        if self.crossover:
            m_symm = i + int(j > i)
            m_unsymm = j + i * self.n_species - i * (i + 1) / 2 - m_symm
            start = int(m_symm * symm + m_unsymm * unsymm)
            return slice(start, start + (symm if i == j else unsymm))
        if i != j:
            raise ValueError("crossover=False: no cross-species blocks exist.")
        return slice(int(i * symm), int(i * symm) + symm)

    # ---- input adapters (SG:291-332, SG:966-1003) ----
    def _system_arrays(self, system):
        """(positions, Z, cell, pbc) of one system (SG:291-332).  Positions
        stay a torch tensor when given as one (autograd flows through it),
        else become a float64 numpy array; Z is a host int64 array."""
        if type(system) is dict:
            return (_as_positions(system["positions"]), _as_numbers(system["atomic_numbers"]), system.get("cell"),
                    system.get("pbc"))
        if isinstance(system, (tuple, list)):
            if len(system) < 2:
                raise ValueError("Tuple/list system must be (positions, atomic_numbers, [cell], [pbc]).")
            cell = system[2] if len(system) >= 3 else None
            pbc = system[3] if len(system) >= 4 else None
            return _as_positions(system[0]), _as_numbers(system[1]), cell, pbc
        if isinstance(system, dict):
            return (_as_positions(system["positions"]), _as_numbers(system["atomic_numbers"]), system.get("cell"),
                    system.get("pbc"))
        if hasattr(system, "get_positions") and hasattr(system, "get_atomic_numbers"):
            cell = system.get_cell().array if hasattr(system, "get_cell") else None
            pbc = system.get_pbc() if hasattr(system, "get_pbc") else None
            return _as_positions(system.get_positions()), _as_numbers(system.get_atomic_numbers()), cell, pbc
        raise TypeError("Unsupported system type. Provide ASE.Atoms-like, dict, or (positions, Z, cell, pbc).")

    def _species_lookup(self, Z) -> np.ndarray:
        """Host int32 species index of every atom; ValueError for atomic
        numbers outside the species list (SG:1782-1784)."""
        Zc = Z.detach().cpu().numpy() if isinstance(Z, torch.Tensor) else np.asarray(Z, dtype=np.int64)
        bad = set(np.unique(Zc).tolist()) - self._atomic_number_set
        if bad:
            raise ValueError(f"System contains atomic numbers not in species list: {sorted(bad)}")
        lut = np.full(int(Zc.max()) + 1 if Zc.size else 1, -1, dtype=np.int32)
        for z, i in self._Z_to_species_index.items():
            if z < lut.size:
                lut[z] = i
        return lut[Zc] if Zc.size else np.zeros(0, np.int32)

    def _species_index(self, Z) -> torch.Tensor:
        return torch.as_tensor(self._species_lookup(Z)).to(self.device)

    def _upload(self, arrays) -> Dict[str, torch.Tensor]:
        """Copy named host arrays to the device in one asynchronous copy
        through a pinned staging buffer kept by this object; returns typed
        device views.  The staging buffer is reused once its last copy has
        completed."""
        offs, off = [], 0
        for name, a in arrays:
            a = np.ascontiguousarray(a)
            offs.append((name, a, off))
            off = (off + a.nbytes + 255) // 256 * 256
        total = max(off, 256)
        if getattr(self, "_stage", None) is None or self._stage.numel() < total:
            self._stage = torch.empty(max(total, 1 << 16), dtype=torch.uint8, pin_memory=True)
            self._stage_done = None
        if self._stage_done is not None:
            self._stage_done.synchronize()
        host = self._stage.numpy()
        for name, a, o in offs:
            host[o:o + a.nbytes] = a.view(np.uint8).reshape(-1)
        dbuf = torch.empty(total, dtype=torch.uint8, device=self.device)
        dbuf.copy_(self._stage[:total], non_blocking=True)
        self._stage_done = torch.cuda.Event()
        self._stage_done.record(torch.cuda.current_stream(self.device))
        tmap = {np.dtype(np.int32): torch.int32, np.dtype(np.int64): torch.int64,
                np.dtype(np.float64): torch.float64, np.dtype(np.uint8): torch.uint8}
        out = {}
        for name, a, o in offs:
            out[name] = dbuf[o:o + a.nbytes].view(tmap[a.dtype]).reshape(a.shape)
        return out

    def _prepare_centres(self, pos: torch.Tensor, centers):
        """(xyz, self atom, attached atom) per centre.  Index centres are
        attached to their atom; Cartesian centres within 1e-12 of an atom get
        that atom's self term but stay fixed (SG:966-1003)."""
        dev = self.device
        if centers is None:
            idx = torch.arange(pos.shape[0], dtype=torch.int64, device=dev)
            return pos, idx, idx
        xyz, atom, attach = [], [], []
        cart = []
        for c in centers:
            if isinstance(c, (int, np.integer)):
                i = int(c)
                xyz.append(pos[i])
                atom.append(i)
                attach.append(i)
            else:
                cc = torch.as_tensor(np.asarray(c, dtype=np.float64) if not isinstance(c, torch.Tensor) else c,
                                     dtype=torch.float64, device=dev).reshape(3)
                cart.append(len(xyz))
                xyz.append(cc)
                atom.append(-1)
                attach.append(-1)
        if len(xyz) == 0:
            z = torch.zeros(0, dtype=torch.int64, device=dev)
            return torch.zeros((0, 3), dtype=torch.float64, device=dev), z, z
        xyz_t = torch.stack(xyz)
        atom_t = torch.tensor(atom, dtype=torch.int64, device=dev)
        if cart and pos.shape[0] > 0:
            ci = torch.tensor(cart, dtype=torch.int64, device=dev)
            d2 = ((pos.detach()[None, :, :] - xyz_t.detach()[ci][:, None, :]) ** 2).sum(-1)
            dmin, j = d2.min(dim=1)
            atom_t[ci] = torch.where(dmin <= 1e-24, j, torch.full_like(j, -1))
        return xyz_t, atom_t, torch.tensor(attach, dtype=torch.int64, device=dev)

    # ---- kernels ----
    def _run_descriptor(self, batch: _Batch, pairs: _Pairs, mode: int, want_coeff: bool = False):
        lib = _lib.load()
        F = int(self._basis.n_feat_ps if mode == _lib.OUT_PS else self._basis.n_feat_cc)
        out = torch.empty((batch.n_centres, F), dtype=torch.float32, device=self.device)
        coeff = (torch.empty((batch.n_centres, int(self._basis.n_feat_cc)), dtype=torch.float32, device=self.device)
                 if want_coeff else None)
        self._call("descriptor", lib.soapb_descriptor, ctypes.byref(self._basis), batch.n_centres,
                   _ptr(pairs.pair_off), _ptr(pairs.pairs), mode, _ptr(out), _ptr(coeff), _ptr(self._counter),
                   _stream(self.device))
        return out, coeff

    def _run_forces(self, batch, pairs, coeff, dEdp, attach=True, mode=None):
        lib = _lib.load()
        forces = torch.zeros((batch.n_atoms, 3), dtype=torch.float32, device=self.device)
        wsb = ctypes.c_int64(0)
        check(lib.soapb_forces_workspace(ctypes.byref(self._basis), batch.n_centres, ctypes.byref(wsb)))
        work = torch.empty(max(int(wsb.value), 256), dtype=torch.uint8, device=self.device)
        self._call("forces", lib.soapb_forces, ctypes.byref(self._basis), batch.n_centres, _ptr(pairs.pair_off),
                   _ptr(pairs.pairs), _ptr(coeff), _ptr(dEdp), self._out_mode() if mode is None else mode,
                   _ptr(batch.centre_attach), int(bool(attach)), _ptr(forces), _ptr(work), work.numel(),
                   _ptr(self._counter), _stream(self.device))
        self._last_forces_work = (work, batch.n_centres)
        return forces

    def forces_status(self) -> int:
        """Status word of the last adjoint pass (synchronises the stream):
        0 = ok; bit 0 = a row copy of its G stage did not complete within the
        kernel's bounded wait, and the forces of that pass are NaN."""
        last = getattr(self, "_last_forces_work", None)
        if last is None:
            return 0
        work, n_centres = last
        out = ctypes.c_int32(0)
        check(_lib.load().soapb_forces_status(ctypes.byref(self._basis), n_centres, _ptr(work), ctypes.byref(out),
                                              _stream(self.device)))
        return int(out.value)

    def _out_mode(self) -> int:
        return _lib.OUT_CC if self.average == "cc" else _lib.OUT_PS

    # ---- public API ----
    def create(self, system, centers=None, n_jobs: int = 1, only_physical_cores: bool = False,
               verbose: bool = False):
        """Centre-wise descriptors, (n_centres, n_features) per system; a list
        of systems is computed in one batched launch and returned stacked
        when the shapes match, else as a list (SG:1691-1757)."""
        return self.generate(system, centers, n_jobs=n_jobs, only_physical_cores=only_physical_cores,
                             verbose=verbose)

    def generate(self, system, centers=None, n_jobs: int = 1, only_physical_cores: bool = False,
                 verbose: bool = False):
        with torch.cuda.device(self.device):
            if isinstance(system, list):
                systems = system
                if centers is None:
                    centers_list = [None] * len(systems)
                else:
                    if not isinstance(centers, list):
                        raise ValueError("For multiple systems, centers must be a list with one entry per system.")
                    centers_list = centers
                    if len(centers_list) != len(systems):
                        raise ValueError("centers list must match number of systems.")
                if not systems:
                    return []
                out = self._evaluate_batch(systems, centers_list)
                parts = list(torch.split(out, [int(c) for c in self._last_counts]))
                if self.sparse:  # each system's rows in COO, then stacked if possible (SG:1716-1737)
                    parts = [p.to_sparse_coo() for p in parts]
                try:
                    return torch.stack(parts, dim=0)
                except Exception:
                    return parts
            out = self._evaluate_batch([system], [centers])
            return out.to_sparse_coo() if self.sparse else out

    def create_flat(self, systems: List[Any], centers=None) -> Tuple[torch.Tensor, torch.Tensor]:
        """Descriptors of a list of systems as ONE contiguous (total centres,
        F) tensor and the int64 row offsets (n_systems + 1) on the host: rows
        offsets[i]:offsets[i+1] belong to system i.  The same batched launch
        as ``create(list)``, without splitting the output into per-system
        views, so a caller that reduces over all systems needs no
        concatenation.  Differentiable like ``create``; dense output.  No
        counterpart in the reference (its list path returns per-system
        tensors, SG:1716-1733)."""
        systems = list(systems)
        centers_list = [None] * len(systems) if centers is None else list(centers)
        if len(centers_list) != len(systems):
            raise ValueError("centers list must match number of systems.")
        with torch.cuda.device(self.device):
            if not systems:
                return (torch.zeros((0, self.get_number_of_features()), dtype=self.dtype, device=self.device),
                        torch.zeros(1, dtype=torch.int64))
            out = self._evaluate_batch(systems, centers_list)
            offsets = torch.zeros(len(systems) + 1, dtype=torch.int64)
            offsets[1:] = torch.cumsum(torch.tensor(self._last_counts, dtype=torch.int64), 0)
            return out, offsets

    def _evaluate_batch(self, systems, centers_list) -> torch.Tensor:
        batch = _Batch(self, systems, centers_list)
        self._last_counts = batch.counts
        mode = self._out_mode()
        grad = torch.is_grad_enabled() and any(p.requires_grad for p in batch.pos_tensors)
        if grad:
            if len(batch.pos_tensors) != len(systems):
                raise ValueError("differentiable create() needs every structure's positions as a tensor")
            pos = batch.pos_tensors[0] if len(batch.pos_tensors) == 1 else torch.cat(batch.pos_tensors)
            out = _SOAPFunction.apply(pos, self, batch, mode)
        else:
            pairs = _Pairs(self, batch, _lib.NL_CREATE)
            out, _ = self._run_descriptor(batch, pairs, mode)
        return out.to(self.dtype) if self.dtype != torch.float32 else out

    def autotune(self, system, reps: int = 3, cache_path: Optional[str] = None, force: bool = False):
        """Time the candidate launch shapes of the descriptor and adjoint
        kernels on ``system`` and keep the fastest for this object (see
        ``cusoap_b200.autotune``); results are bitwise unchanged."""
        from .autotune import autotune
        return autotune(self, system, reps=reps, cache_path=cache_path, force=force)

    def batch(self, systems: List[Any], headroom: float = 1.25) -> SOAPBatch:
        """A CUDA-graph plan for repeated evaluation of the same structures
        (every atom a centre) at new positions; see ``SOAPBatch``."""
        return SOAPBatch(self, list(systems), headroom)

    def derivatives(self, system, centers=None, include=None, exclude=None, method: str = "auto",
                    return_descriptor: bool = True, attach: bool = False, n_jobs: int = 1,
                    only_physical_cores: bool = False, verbose: bool = False):
        """(n_centres, n_atoms_included, 3, n_features) Jacobian, and the
        descriptor, returned as ``(deriv, desc)`` when return_descriptor
        (SG:2628-2699).  "auto"/"analytical" use the closed-form kernel, for
        any number of neighbours per centre; "numerical" uses central
        differences of create() (step FD_STEP, 5e-3 A)."""
        if method == "numerical":
            return self.derivatives_numerical(system, centers, include, exclude, method="numerical",
                                              return_descriptor=return_descriptor, attach=attach, n_jobs=n_jobs,
                                              only_physical_cores=only_physical_cores, verbose=verbose)
        if method not in ("auto", "analytical"):
            raise ValueError("method must be one of: 'auto', 'analytical', 'numerical'.")
        with torch.cuda.device(self.device):
            batch = _Batch(self, [system], [centers])
            n_atoms = batch.n_atoms
            idx = list(range(n_atoms)) if include is None else [int(i) for i in include]
            if exclude is not None:
                ex = set(int(i) for i in exclude)
                idx = [i for i in idx if i not in ex]
            n_inc = len(idx)
            mode = self._out_mode()
            F = self.get_number_of_features()
            pairs = _Pairs(self, batch, _lib.NL_ALL)
            desc, coeff = self._run_descriptor(batch, pairs, mode, want_coeff=True)
            deriv = torch.empty((batch.n_centres, n_inc, 3, F), dtype=torch.float32, device=self.device)
            if n_inc > 0 and batch.n_centres > 0:
                if include is None and exclude is None:  # every atom, in order: row = atom
                    inc_row = torch.arange(max(n_atoms, 1), dtype=torch.int32, device=self.device)
                else:
                    h = np.full(max(n_atoms, 1), -1, dtype=np.int32)
                    h[np.asarray(idx, dtype=np.int64)] = np.arange(n_inc, dtype=np.int32)
                    inc_row = torch.from_numpy(h).to(self.device)
                status = torch.zeros(1, dtype=torch.int32, device=self.device)
                lib = _lib.load()
                wsb = ctypes.c_int64(0)
                check(lib.soapb_jacobian_workspace(ctypes.byref(self._basis), batch.n_centres, pairs.total, n_inc,
                                                   int(bool(attach)), ctypes.byref(wsb)))
                work = torch.empty(max(int(wsb.value), 256), dtype=torch.uint8, device=self.device)
                self._call("jacobian", lib.soapb_jacobian, ctypes.byref(self._basis), batch.n_centres,
                           _ptr(pairs.pair_off), _ptr(pairs.pairs), pairs.total, _ptr(coeff), _ptr(inc_row), n_inc,
                           _ptr(batch.centre_attach), int(bool(attach)), pairs.max_pairs, mode,
                           _ptr(deriv), _ptr(work), work.numel(), _ptr(status), _stream(self.device))
                # The status word is never set (a centre with more entries than the kernel's
                # shared-memory sort holds is merged in the workspace), so it is not read back:
                # the call returns without waiting for the Jacobian to finish.
            if self.dtype != torch.float32:
                deriv, desc = deriv.to(self.dtype), desc.to(self.dtype)
            return (deriv, desc) if return_descriptor else deriv

    # Default central-difference step (A) of derivatives_numerical.  The
    # reference takes d = 1e-4 with float64 forward passes (SG:1871-1931).
    # These forward passes are float32: a displaced descriptor carries about
    # 1e-7 |p| of rounding, so a difference quotient carries about
    # 1e-7 |p| / (2 d) of noise, against a derivative block that for one
    # neighbour atom is only a small part of |p| per A.  The truncation term
    # grows as (d / sigma)^2 / 6, and an atom within d of a centre's cutoff
    # sees the basis's truncation step (about 1e-3 of its peak), which makes
    # the quotient jump; with attach=True every neighbour of a moving centre
    # can cross, so that happens about d / 1e-4 times as often as with the
    # reference's step.  Measured against the closed form on
    # the workloads (per centre block), 5e-3 A balances them: 6e-5 on the
    # 3000-atom cluster and the periodic cells (sigma 0.4), 8e-4 on the water
    # box, up to 1e-2 for blocks made only of atoms far from the centre;
    # d = 1e-4 gives 2e-3 to 3e-1.
    FD_STEP = 5e-3

    def derivatives_numerical(self, system, centers=None, include=None, exclude=None, method: str = "auto",
                              return_descriptor: bool = True, attach: bool = False, n_jobs: int = 1,
                              only_physical_cores: bool = False, verbose: bool = False,
                              d: Optional[float] = None):
        """Central differences of the descriptor (SG:1871-2003): every
        included atom displaced by +-d along x, y, z, with DScribe's fixed
        centres (attach=False) or index centres moving with their atom
        (attach=True).  Returns (n_centres, n_included, 3, F), and the
        descriptor when return_descriptor.

        All 6 n_included displaced structures go through the batched path,
        one launch per stage for as many structures as fit a fixed memory
        budget.  The displaced descriptors are float32, so the default step
        is ``FD_STEP`` (5e-3 A), not the reference's float64 1e-4, and the
        result is accurate to about 1e-7 |p| / (2 d) absolute: within 1e-4
        relative of float64 differences for a centre's block that includes
        its own atom, up to about 1e-3 to 1e-2 for blocks of distant atoms
        only (see the note at ``FD_STEP``).  The closed-form ``derivatives``
        (about 1e-6) is the accurate path."""
        if method not in ("auto", "numerical"):
            raise ValueError("method must be 'auto' or 'numerical'.")
        d = float(self.FD_STEP if d is None else d)
        if not d > 0.0:
            raise ValueError("d must be positive")
        with torch.cuda.device(self.device):
            desc0 = self.create(system, centers) if return_descriptor else None
            pos, Z, cell, pbc = self._system_arrays(system)
            pos = (pos.detach() if isinstance(pos, torch.Tensor) else torch.as_tensor(pos)).to(self.device,
                                                                                            torch.float64)
            A = int(pos.shape[0])
            idx = list(range(A)) if include is None else [int(i) for i in include]
            if exclude is not None:
                ex = set(int(i) for i in exclude)
                idx = [i for i in idx if i not in ex]
            xyz, atom, att = self._prepare_centres(pos, centers)
            C, F = int(xyz.shape[0]), self.get_number_of_features()
            deriv = torch.zeros((C, len(idx), 3, F), dtype=torch.float32, device=self.device)
            if not idx or C == 0:
                deriv = deriv.to(self.dtype)
                return (deriv, desc0) if return_descriptor else deriv
            xyz = xyz.detach().to(torch.float64)
            atom = atom.to(torch.int64)
            attached = att.to(torch.int64) if attach else torch.full_like(atom, -1)
            species = torch.as_tensor(self._species_lookup(Z)).to(self.device)
            if self.periodic:
                if cell is None or pbc is None:
                    raise ValueError("periodic=True requires cell and pbc.")
                cell_t = torch.as_tensor(np.asarray(cell.detach().cpu() if isinstance(cell, torch.Tensor) else cell,
                                                    dtype=np.float64).reshape(9), device=self.device)
                pbc_t = torch.as_tensor(np.asarray(pbc.detach().cpu() if isinstance(pbc, torch.Tensor) else pbc,
                                                   dtype=bool).reshape(3).astype(np.uint8), device=self.device)
            else:
                cell_t = torch.zeros(9, dtype=torch.float64, device=self.device)
                pbc_t = torch.zeros(3, dtype=torch.uint8, device=self.device)
            # displaced structures: (atom, component) pairs in output order, each as +d then -d
            moves = torch.tensor([(a, k) for a in idx for k in range(3)], dtype=torch.int64, device=self.device)
            # pair-list size of one structure bounds how many structures one launch takes
            base = _Batch.from_device([A], pos, species, cell_t, pbc_t, xyz,
                                      torch.zeros(C, dtype=torch.int32, device=self.device), atom, attached, [C])
            per_struct = max(_Pairs(self, base, _lib.NL_CREATE).total, 1)
            per_move = max(1, min((1 << 26) // (2 * per_struct), (1 << 27) // (2 * C * F), (1 << 22) // (2 * A)))
            for m0 in range(0, moves.shape[0], per_move):
                mv = moves[m0:m0 + per_move]
                n = 2 * mv.shape[0]
                a_s = mv[:, 0].repeat_interleave(2)
                k_s = mv[:, 1].repeat_interleave(2)
                sgn = torch.tensor([d, -d], dtype=torch.float64, device=self.device).repeat(mv.shape[0])
                P = pos.unsqueeze(0).repeat(n, 1, 1)
                rows = torch.arange(n, device=self.device)
                P[rows, a_s, k_s] += sgn
                X = xyz.unsqueeze(0).repeat(n, 1, 1)
                moved = attached.unsqueeze(0) == a_s.unsqueeze(1)  # (n, C): centres riding on the moved atom
                X = torch.where(moved.unsqueeze(-1), P[rows, a_s].unsqueeze(1).expand(n, C, 3), X)
                # a fixed centre stops coinciding with its atom once that atom moves (SG:966-1003)
                lost = (atom.unsqueeze(0) == a_s.unsqueeze(1)) & ~moved
                catom = torch.where(lost, torch.full_like(lost, -1, dtype=torch.int64), atom.unsqueeze(0))
                catom = catom + (rows * A).unsqueeze(1) * (catom >= 0)
                cattach = attached.unsqueeze(0) + (rows * A).unsqueeze(1) * (attached.unsqueeze(0) >= 0)
                batch = _Batch.from_device(
                    [A] * n, P.reshape(-1, 3), species.repeat(n), cell_t.repeat(n, 1), pbc_t.repeat(n, 1),
                    X.reshape(-1, 3), torch.arange(n, dtype=torch.int32, device=self.device).repeat_interleave(C),
                    catom.reshape(-1), cattach.reshape(-1), [C] * n)
                out, _ = self._run_descriptor(batch, _Pairs(self, batch, _lib.NL_CREATE), self._out_mode())
                out = out.view(mv.shape[0], 2, C, F).double()
                diff = ((out[:, 0] - out[:, 1]) / (2.0 * d)).float()  # (moves, C, F)
                # moves run over (included atom, component) in output order
                deriv.view(C, -1, F)[:, m0:m0 + mv.shape[0], :] = diff.permute(1, 0, 2)
            deriv = deriv.to(self.dtype)
            return (deriv, desc0) if return_descriptor else deriv

    def energy_forces(self, system, dEdp) -> Tuple[torch.Tensor, torch.Tensor]:
        """E = sum(dEdp * p) over all atoms as centres, and F = -dE/dx from the
        adjoint kernel (centres attached to their atoms).  dEdp: (F,) weights
        shared by every centre, or (n_atoms, F)."""
        with torch.cuda.device(self.device):
            batch = _Batch(self, [system], [None])
            pairs = _Pairs(self, batch, _lib.NL_ALL)
            desc, coeff = self._run_descriptor(batch, pairs, _lib.OUT_PS, want_coeff=True)
            w = torch.as_tensor(dEdp, dtype=torch.float32, device=self.device)
            if w.dim() == 1:
                w = w.expand(batch.n_centres, -1)
            w = w.contiguous()
            E = (desc.double() * w.double()).sum()
            forces = self._run_forces(batch, pairs, coeff, w, attach=True)
            return E, forces
