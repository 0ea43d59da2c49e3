"""Test-only stand-in for ``sphericart.torch`` (third-party, pinned by the
reference as ``sphericart>=1.0``; not installed in this container).

Implements the three calls the reference makes (``SphericalHarmonics.compute``,
``SolidHarmonics.compute`` and ``.compute_with_gradients``) from the published
definition of sphericart's real harmonics: orthonormal, m = -l..l, no
Condon-Shortley phase, l=1 = sqrt(3/4pi) (y, z, x).  Written with plain torch
ops so autograd can differentiate through it, which the reference's autograd
derivative path needs.  The recurrence is the one restated in
``oracle/soap_oracle.py::solid_harmonics``.
"""
import math

import torch


def _norm(l, m):
    if m == 0:
        return math.sqrt((2 * l + 1) / (4 * math.pi))
    return math.sqrt((2 * l + 1) / (2 * math.pi) * math.factorial(l - m) / math.factorial(l + m))


def _solid(xyz, l_max):
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    r2 = x * x + y * y + z * z
    Lp1 = l_max + 1
    Q = {}
    for m in range(Lp1):
        dfact = 1.0
        for k in range(2 * m - 1, 0, -2):
            dfact *= k
        Q[(m, m)] = torch.full_like(x, dfact)
        if m + 1 <= l_max:
            Q[(m + 1, m)] = (2 * m + 1) * z * Q[(m, m)]
        for l in range(m + 2, Lp1):
            Q[(l, m)] = ((2 * l - 1) * z * Q[(l - 1, m)] - (l + m - 1) * r2 * Q[(l - 2, m)]) / (l - m)
    C = [torch.ones_like(x)]
    S = [torch.zeros_like(x)]
    for m in range(1, Lp1):
        C.append(x * C[m - 1] - y * S[m - 1])
        S.append(x * S[m - 1] + y * C[m - 1])
    cols = []
    for l in range(Lp1):
        for m in range(-l, l + 1):
            am = abs(m)
            phi = torch.ones_like(x) if m == 0 else (C[am] if m > 0 else S[am])
            cols.append(_norm(l, am) * Q[(l, am)] * phi)
    return torch.stack(cols, dim=-1)


class SolidHarmonics:
    def __init__(self, l_max):
        self.l_max = int(l_max)

    def compute(self, xyz):
        return _solid(xyz, self.l_max)

    def compute_with_gradients(self, xyz):
        with torch.enable_grad():
            p = xyz.detach().clone().requires_grad_(True)
            R = _solid(p, self.l_max)
            grads = []
            for k in range(R.shape[1]):
                g = torch.autograd.grad(R[:, k].sum(), p, retain_graph=True)[0]
                grads.append(g)
            dR = torch.stack(grads, dim=-1)  # (E,3,K)
        return R.detach(), dR.detach()


class SphericalHarmonics:
    def __init__(self, l_max):
        self.l_max = int(l_max)

    def compute(self, xyz):
        r = torch.linalg.norm(xyz, dim=-1, keepdim=True)
        return _solid(xyz / r, self.l_max)
