"""Timed CPU port of the reference SOAP path -- TEST / BENCHMARK INFRASTRUCTURE ONLY.

``bench.py``'s reference arm and its CPU-baseline leg time this module; the
test suite checks it against the FP64 oracle and the reference's fixtures.
The product package never imports it.

Why a port: the reference (TACC/cuSOAP ``src/cusoap/soap_generator.py``,
cited SG:<line>) is a Python package that is not present where the
benchmark runs.  This file restates, in torch float64 on the CPU, the SAME
sequence of vectorised tensor operations the reference executes on a CPU
device for a non-periodic GTO system, so that its run time is the
reference's algorithm's run time on the same host threads
(``oracle/calibrate_port.py`` measures both):

* ``create`` (SG:1759-1810): chunked GEMM radius search
  ||c||^2 + ||n||^2 - 2 c.n over 1024-centre chunks and ``nonzero``
  (SG:1077-1125, the branch taken without torch_cluster); r <= 1e-12 edges
  dropped (SG:1171-1179); real spherical harmonics of the unit vectors
  (SG:1329); per l the primitive radial factors, their outer product with
  Y_l, an ``index_add_`` over (centre, species) rows and the beta einsum
  (SG:1348-1391); the analytic l = 0 self term of index centres
  (SG:821-850); per l the power-spectrum einsum and the DScribe slices
  (SG:1634-1689).
* ``derivatives`` (SG:2270-2626, the CPU branch after the Triton fast
  paths, taken on a CPU device): the radius edges keeping r = 0; B and Bhat
  from (E, l, k) exponentials and two einsums (SG:2389-2402); solid
  harmonics and their gradients (SG:2412); coefficients from the same edges
  (SG:2419-2429); the dense edge gradient (E, 3, n, K) and its
  ``index_add_`` into (C n_inc S, 3, n, K) (SG:2557-2571); per l the
  product-rule einsum into (C, A, 3, S, n, S, n) and the slice fill
  (SG:2589-2613); cast to the output dtype (SG:2615).

The solid harmonics come from the same Q_l^m recurrence as
``oracle/soap_oracle.py`` (the reference calls the third-party sphericart
library there); gradients are analytic, as sphericart's are.  Only
non-periodic GTO systems without weighting are ported: the workloads this
is timed on.
"""
from __future__ import annotations

import math
from typing import List, Optional, Sequence

import numpy as np
import torch

from .soap_oracle import OracleSOAP, _norms

DT = torch.float64


def _solid(xyz: torch.Tensor, l_max: int, gradients: bool):
    """R_lm = r^l Y_lm (E, K) and optionally dR (E, 3, K), sphericart's
    convention (orthonormal real harmonics, m = -l..l, no Condon-Shortley
    phase), by the Q_l^m recurrence."""
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    E, Lp1 = xyz.shape[0], l_max + 1
    r2 = x * x + y * y + z * z
    zero = torch.zeros_like(x)
    Q = {}
    for m in range(Lp1):
        Q[(m, m)] = torch.full_like(x, float(np.prod(np.arange(2 * m - 1, 0, -2))) if m > 0 else 1.0)
        if m + 1 <= l_max:
            Q[(m + 1, m)] = (2 * m + 1) * z * Q[(m, m)]
        for l in range(m + 2, Lp1):
            Q[(l, m)] = ((2 * l - 1) * z * Q[(l - 1, m)] - (l + m - 1) * r2 * Q[(l - 2, m)]) / (l - m)
    C, S = [torch.ones_like(x)], [zero]
    for m in range(1, Lp1):
        C.append(x * C[m - 1] - y * S[m - 1])
        S.append(x * S[m - 1] + y * C[m - 1])
    nrm = _norms(l_max)
    K = Lp1 * Lp1
    R = torch.empty((E, K), dtype=DT)
    dR = torch.empty((E, 3, K), dtype=DT) if gradients else None
    for l in range(Lp1):
        for m in range(-l, l + 1):
            am, idx = abs(m), l * l + l + m
            q = Q[(l, am)]
            if m == 0:
                phi, px, py = 1.0, zero, zero
            elif m > 0:
                phi, px, py = C[am], am * C[am - 1], -am * S[am - 1]
            else:
                phi, px, py = S[am], am * S[am - 1], am * C[am - 1]
            R[:, idx] = nrm[l, am] * q * phi
            if gradients:
                qp = Q.get((l - 1, am + 1), zero) if l >= 1 else zero
                qz = (l + am) * Q[(l - 1, am)] if l >= 1 and am <= l - 1 else zero
                dR[:, 0, idx] = nrm[l, am] * (-x * qp * phi + q * px)
                dR[:, 1, idx] = nrm[l, am] * (-y * qp * phi + q * py)
                dR[:, 2, idx] = nrm[l, am] * (qz * phi)
    return R, dR


class ReferencePort:
    """The reference's CPU sequence for non-periodic GTO systems (see the
    module docstring); parameters as the reference's SOAP constructor."""

    def __init__(self, species, r_cut, n_max, l_max, sigma=1.0, crossover=True, average="off",
                 out_dtype=torch.float32, **_):
        if average == "cc":
            raise ValueError("the timed port covers the power spectrum only")
        # the reference casts its float64 results to its dtype argument (float32 by default, SG:1809, SG:2615)
        self.out_dtype = out_dtype
        o = OracleSOAP(r_cut=r_cut, n_max=n_max, l_max=l_max, sigma=sigma, species=species, crossover=crossover)
        self.S, self.N, self.L = o.S, o.n_max, o.l_max
        self.K = (self.L + 1) ** 2
        self.eta = o.eta
        self.cutoff = o.cutoff
        self.alphas = torch.tensor(o.alphas, dtype=DT)
        self.betas = torch.tensor(o.betas, dtype=DT)
        self.z2s = o.z2s
        self.self_l0 = torch.tensor(o.self_l0(), dtype=DT)
        self.F = o.n_power_features()
        # DScribe slices (j, jd, l, diag, start, end), SG:1215-1245
        self.slices = []
        f = 0
        for j in range(self.S):
            for jd in range(j, self.S if crossover else j + 1):
                for l in range(self.L + 1):
                    w = self.N * (self.N + 1) // 2 if j == jd else self.N * self.N
                    self.slices.append((j, jd, l, j == jd, f, f + w))
                    f += w
        assert f == self.F
        self.triu = torch.triu_indices(self.N, self.N)
        self.l_of_lm = torch.tensor([l for l in range(self.L + 1) for _ in range(2 * l + 1)])

    def _species(self, Z: torch.Tensor) -> torch.Tensor:
        lut = torch.full((int(Z.max()) + 1,), -1, dtype=torch.long)
        for z, i in self.z2s.items():
            if z < lut.numel():
                lut[z] = i
        return lut[Z]

    def _edges(self, centres: torch.Tensor, pos: torch.Tensor):
        """(centre, neighbour) pairs within the cutoff by the chunked GEMM
        distance and nonzero (SG:1077-1125)."""
        nT = pos.t().contiguous()
        nn = (pos * pos).sum(1)
        c2 = self.cutoff * self.cutoff
        ci, nj = [], []
        for s in range(0, centres.shape[0], 1024):
            c = centres[s:s + 1024]
            d2 = torch.mm(c, nT)
            d2.mul_(-2.0).add_((c * c).sum(1)[:, None]).add_(nn[None, :])
            mask = d2 <= c2
            if mask.any():
                idx = torch.nonzero(mask)
                ci.append(idx[:, 0] + s)
                nj.append(idx[:, 1])
        if not ci:
            e = torch.zeros(0, dtype=torch.long)
            return e, e
        return torch.cat(ci), torch.cat(nj)

    def _power_spectrum(self, coeffs: List[torch.Tensor]) -> torch.Tensor:
        C = coeffs[0].shape[0]
        desc = torch.empty((C, self.F), dtype=DT)
        ti, tj = self.triu[0], self.triu[1]
        for l, cl in enumerate(coeffs):
            P = math.sqrt(8.0 * math.pi ** 2 / (2 * l + 1)) * torch.einsum("cjnm,ckdm->cjknd", cl, cl)
            for j, jd, l2, diag, a, b in self.slices:
                if l2 == l:
                    desc[:, a:b] = P[:, j, j][:, ti, tj] if diag else P[:, j, jd].reshape(C, -1)
        return desc

    def create(self, positions, Z, centers: Optional[Sequence[int]] = None) -> torch.Tensor:
        """(C, F) power spectrum of index centres (all atoms when None)."""
        pos = torch.as_tensor(np.asarray(positions, np.float64))
        Zt = torch.as_tensor(np.asarray(Z, np.int64))
        cidx = torch.arange(pos.shape[0]) if centers is None else torch.as_tensor(list(centers), dtype=torch.long)
        cxyz = pos[cidx]
        ci, nj = self._edges(cxyz, pos)
        rvec = pos[nj] - cxyz[ci]
        r = torch.linalg.norm(rvec, dim=-1)
        keep = r > 1e-12
        ci, nj, rvec, r = ci[keep], nj[keep], rvec[keep], r[keep]
        sp = self._species(Zt)[nj]
        Y, _ = _solid(rvec / r[:, None], self.L, False)
        C = cxyz.shape[0]
        row = ci * self.S + sp
        coeffs = []
        for l in range(self.L + 1):
            a = self.alphas[l][None, :]
            p = a + self.eta
            prim = (math.pi ** 1.5) * (self.eta / p) ** l * p ** -1.5 * (r ** l)[:, None] \
                * torch.exp(-(a * self.eta / p) * (r[:, None] ** 2))
            contrib = (prim[:, :, None] * Y[:, None, l * l:(l + 1) ** 2]).reshape(r.shape[0], -1)
            acc = torch.zeros((C * self.S, contrib.shape[1]), dtype=DT)
            acc.index_add_(0, row, contrib)
            coeffs.append(torch.einsum("ab,csbm->csam", self.betas[l], acc.view(C, self.S, self.N, 2 * l + 1)))
        # the centre's own Gaussian (SG:821-850)
        own = self._species(Zt)[cidx]
        coeffs[0][torch.arange(C), own, :, 0] += self.self_l0[None, :]
        return self._power_spectrum(coeffs).to(self.out_dtype)

    def derivatives(self, positions, Z, centers: Optional[Sequence[int]] = None) -> torch.Tensor:
        """(C, A, 3, F) closed-form Jacobian of the power spectrum w.r.t.
        every atom, fixed centres (SG:2270-2626, CPU branch)."""
        pos = torch.as_tensor(np.asarray(positions, np.float64))
        Zt = torch.as_tensor(np.asarray(Z, np.int64))
        A = pos.shape[0]
        cidx = torch.arange(A) if centers is None else torch.as_tensor(list(centers), dtype=torch.long)
        cxyz = pos[cidx]
        C, S, N, K, Lp1 = cxyz.shape[0], self.S, self.N, self.K, self.L + 1
        ci, nj = self._edges(cxyz, pos)
        E = ci.shape[0]
        rvec = pos[nj] - cxyz[ci]
        r2 = (rvec * rvec).sum(1)
        sp = self._species(Zt)[nj]
        p = self.alphas + self.eta
        gamma = self.alphas * self.eta / p
        pref = (math.pi ** 1.5) * (self.eta / p) ** torch.arange(Lp1, dtype=DT)[:, None] * p ** -1.5
        Qe = pref[None] * torch.exp(-gamma[None] * r2[:, None, None])  # (E, l, k)
        B = torch.einsum("elk,lnk->enl", Qe, self.betas)
        Bh = torch.einsum("elk,lnk->enl", (-2.0 * gamma[None]) * Qe, self.betas)
        Yv, Yg = _solid(rvec, self.L, True)
        cE = B[:, :, self.l_of_lm] * Yv[:, None, :]
        Cacc = torch.zeros((C * S, N * K), dtype=DT)
        Cacc.index_add_(0, ci * S + sp, cE.reshape(E, -1))
        Cc = Cacc.view(C, S, N, K)
        Bl, Bhl = B[:, :, self.l_of_lm], Bh[:, :, self.l_of_lm]
        g = rvec[:, :, None, None] * (Bhl[:, None] * Yv[:, None, None, :]) + Bl[:, None] * Yg[:, :, None, :]
        Dacc = torch.zeros((C * A * S, 3, N, K), dtype=DT)
        Dacc.index_add_(0, (ci * A + nj) * S + sp, g)
        D = Dacc.view(C, A, S, 3, N, K)
        deriv = torch.zeros((C, A, 3, self.F), dtype=DT)
        ti, tj = self.triu[0], self.triu[1]
        for l in range(Lp1):
            s0, s1 = l * l, (l + 1) ** 2
            X = torch.einsum("cajdnm,ckqm->cadjnkq", D[..., s0:s1], Cc[..., s0:s1])
            PD = math.sqrt(8.0 * math.pi ** 2 / (2 * l + 1)) * (X + X.permute(0, 1, 2, 5, 6, 3, 4))
            for j, jd, l2, diag, a, b in self.slices:
                if l2 == l:
                    blk = PD[:, :, :, j, :, jd, :]
                    deriv[..., a:b] = blk[..., ti, tj] if diag else blk.reshape(C, A, 3, -1)
        return deriv.to(self.out_dtype)
