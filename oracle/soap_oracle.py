"""CPU FP64 restatement of the reference SOAP path -- TEST INFRASTRUCTURE ONLY.

This module is the oracle the CUDA path is checked against. Only the test
suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py``
may import it, and only as the checker / timed CPU baseline; the product
package (``cusoap_b200``) never imports it.

It restates, in vectorised numpy float64, the algorithm of the reference
``src/cusoap/soap_generator.py`` (cited below as ``SG:<line>``):

* GTO basis and Loewdin S^-1/2 ........................ SG:690-708, SG:339-343
* polynomial basis (sqrtm(inv(S)), Gauss-Legendre grid)  SG:350-362, SG:710-752
* polynomial radial integrals (scaled Bessel recurrence)  SG:477-508, SG:1432-1594
* weighting functions (poly / pow / exp, w0, r_cut) .... SG:403-470, SG:584-597
* periodic images (perpendicular widths, offsets) ...... SG:369-396, SG:1015-1021
* radius neighbour list, r~0 edge drop ................. SG:1042-1181
* GTO coefficients c_nlm (primitive radial x Y, beta) .. SG:1294-1391
* analytic self term .................................. SG:765-850
* power spectrum + DScribe feature order ............... SG:1215-1245, SG:1599-1601, SG:1634-1689
* cc projection (l=1 -> (z,x,y), pi^-3/2 for l>=2) .... SG:1603-1632
* closed-form ps / cc Jacobian (fixed centres) ......... SG:2270-2626
* feature counts / get_location ........................ SG:908-962

The real spherical harmonics come from the third-party ``sphericart``
package (pyproject pins ``sphericart>=1.0``; not vendored in the reference,
not installed here).  Its published convention is restated in
``solid_harmonics``: orthonormal real harmonics, m=-l..l, no Condon-Shortley
phase, so the l=1 block is (y, z, x) * sqrt(3/4pi) (the reference relies on
this at SG:1610-1611).  Power-spectrum outputs are invariant under any
orthogonal change of basis within each l, so they do not depend on that
convention; ``average='cc'`` outputs do.

Forces (``forces``) restate what one reverse-mode pass through the
reference's differentiable forward (SG:2007-2113 with grad_outputs = dE/dp,
centres attached to their atoms) computes, in closed form.
"""
from __future__ import annotations

import math
from typing import Optional, Sequence, Tuple

import numpy as np

Y00 = 1.0 / math.sqrt(4.0 * math.pi)


# ---------------------------------------------------------------------------
# basis
# ---------------------------------------------------------------------------

def lowdin_invsqrt(S: np.ndarray, eps: float = 1e-12) -> np.ndarray:
    """S^-1/2 by symmetric eigendecomposition, eigenvalues clamped (SG:339-343)."""
    w, V = np.linalg.eigh(S)
    w = np.clip(w, eps, None)
    return (V * (1.0 / np.sqrt(w))) @ V.T


def gto_basis(r_cut: float, n_max: int, l_max: int) -> Tuple[np.ndarray, np.ndarray]:
    """alpha (l_max+1, n_max) and beta (l_max+1, n_max, n_max) (SG:690-708)."""
    a = np.linspace(1.0, r_cut, n_max)
    alphas, betas = [], []
    for l in range(l_max + 1):
        alpha_l = -np.log(1e-3 / a ** l) / a ** 2
        m = alpha_l[:, None] + alpha_l[None, :]
        S = 0.5 * math.gamma(l + 1.5) * m ** (-(l + 1.5))
        alphas.append(alpha_l)
        betas.append(lowdin_invsqrt(S))
    return np.stack(alphas), np.stack(betas)


def radial_tables(alphas, betas, eta):
    """Per-l constants of the solid-harmonic factorisation (SG:2389-2402):
    gamma_kl = alpha eta / (alpha + eta), pref_kl = pi^1.5 (eta/p)^l p^-1.5."""
    Lp1 = alphas.shape[0]
    p = alphas + eta
    gamma = alphas * eta / p
    lvec = np.arange(Lp1, dtype=np.float64)[:, None]
    pref = math.pi ** 1.5 * (eta / p) ** lvec * p ** (-1.5)
    return gamma, pref


def radial_B_Bhat(r2: np.ndarray, betas, gamma, pref):
    """B[e,n,l] = sum_k beta^l_nk pref_kl exp(-gamma_kl r^2) and
    Bhat[e,n,l] = sum_k beta^l_nk (-2 gamma_kl) pref_kl exp(-gamma_kl r^2)
    (SG:2396-2402)."""
    Q = pref[None] * np.exp(-gamma[None] * r2[:, None, None])  # (E,L,k)
    B = np.einsum("elk,lnk->enl", Q, betas)
    Bhat = np.einsum("elk,lnk->enl", (-2.0 * gamma[None]) * Q, betas)
    return B, Bhat


def gauss_legendre(n: int) -> Tuple[np.ndarray, np.ndarray]:
    """Nodes and weights on [-1, 1] by the Golub-Welsch eigenproblem (SG:350-362)."""
    k = np.arange(1, n, dtype=np.float64)
    beta = k / np.sqrt(4.0 * k * k - 1.0)
    J = np.diag(beta, 1) + np.diag(beta, -1)
    x, V = np.linalg.eigh(J)
    return x, 2.0 * V[0, :] ** 2


def poly_basis(r_cut: float, n_max: int, quad_n: int = 100):
    """DScribe polynomial basis g_n(r) = sum_k beta_nk (r_cut - r)^(k+2) on the
    Gauss-Legendre grid: (rx, wr, gss (n_max, Q)), beta = sqrtm(inv(S)) in
    float64 exactly as the reference computes it (SG:710-752)."""
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
    x, w = gauss_legendre(quad_n)
    rx = rc * 0.5 * (x + 1.0)
    wr = rc * 0.5 * w
    rclip = np.clip(rx, 0.0, rc)
    fs = np.stack([(rc - rclip) ** (k + 2) for k in range(1, n + 1)])
    return rx, wr, np.ascontiguousarray(betas) @ fs


def poly_I_J(r, rx, wr, gss, eta, l_max, want_J):
    """I[e,n,l] = 4 pi int rx^2 g_n e^{-eta (rx-r)^2} ie_l(t) drx and
    J[e,n,l] = 4 pi int rx^3 g_n e^{-eta (rx-r)^2} ie_{l+1}(t) drx, t = 2 eta rx r,
    ie_l = i_l e^{-t} by the upward recurrence with the reference's clamps
    (SG:477-508, SG:1432-1510)."""
    r = np.asarray(r, np.float64)
    Lp1 = l_max + 1
    tt = np.clip(2.0 * eta * rx[None, :] * r[:, None], 1e-12, None)
    e2 = np.exp(-2.0 * tt)
    oOt = 1.0 / tt
    common = 4.0 * math.pi * (rx * rx * wr)[None, :] * np.exp(-eta * (rx[None, :] - r[:, None]) ** 2)
    I = np.empty((len(r), gss.shape[0], Lp1))
    J = np.empty_like(I) if want_J else None
    L_top = Lp1 if want_J else Lp1 - 1
    P_pp = P_p = None
    for l in range(L_top + 1):
        if l == 0:
            P = common * ((1.0 - e2) * (0.5 * oOt))
        elif l == 1:
            P = common * np.clip((1.0 + e2) * (0.5 * oOt) - (1.0 - e2) * (0.5 * oOt * oOt), 0.0, None)
        else:
            P = np.minimum(np.clip(P_pp - (2 * l - 1) * oOt * P_p, 0.0, None), P_p)
        if l < Lp1:
            I[:, :, l] = P @ gss.T
        if want_J and l >= 1:
            J[:, :, l - 1] = (P * rx[None, :]) @ gss.T
        P_pp, P_p = P_p, P
    return I, J


def poly_B_Bhat_r0(rx, wr, gss, eta, l_max):
    """Exact r -> 0 limits of B_nl = I_nl / r^l and Bhat_nl (SG:1512-1543)."""
    common0 = 4.0 * math.pi * rx * rx * wr * np.exp(-eta * rx * rx)
    B0 = np.empty((gss.shape[0], l_max + 1))
    Bh0 = np.empty_like(B0)
    fl = np.ones_like(rx)
    df = 1.0
    for l in range(l_max + 1):
        df_next = df * (2 * l + 3)
        B0[:, l] = (common0 * fl / df) @ gss.T
        Bh0[:, l] = 2.0 * eta * ((common0 * fl * 2.0 * eta * rx * rx / df_next) @ gss.T - B0[:, l])
        fl = fl * 2.0 * eta * rx
        df = df_next
    return B0, Bh0


def poly_B_Bhat(r, rx, wr, gss, eta, l_max):
    """B = I / r^l, Bhat = 2 eta (J - r I) / r^(l+1); edges with r < 1e-4 take
    the exact limits (SG:1545-1594)."""
    r = np.asarray(r, np.float64)
    tiny = r < 1e-4
    rs = np.where(tiny, 1.0, r)
    I, J = poly_I_J(rs, rx, wr, gss, eta, l_max, want_J=True)
    rl = rs[:, None] ** np.arange(l_max + 1)[None, :]
    B = I / rl[:, None, :]
    Bh = 2.0 * eta * (J - rs[:, None, None] * I) / (rl * rs[:, None])[:, None, :]
    if tiny.any():
        B0, Bh0 = poly_B_Bhat_r0(rx, wr, gss, eta, l_max)
        B[tiny] = B0
        Bh[tiny] = Bh0
    return B, Bh


class Weighting:
    """DScribe weighting w(r) (SG:403-470) and its radial derivative, which the
    reference gets from autograd through the same expression."""

    def __init__(self, function=None, r0=1.0, c=1.0, d=1.0, m=1.0, w0=1.0):
        self.function, self.r0, self.c, self.d, self.m, self.w0 = function, float(r0), float(c), float(d), \
            float(m), float(w0)

    def infer_rcut(self, threshold=1e-2) -> float:
        fn = self.function
        if fn is None:
            raise ValueError("Cannot infer r_cut when weighting.function is None; provide r_cut explicitly.")
        if fn == "poly":
            return self.r0
        val = self.c / threshold - self.d
        if val <= 0:
            raise ValueError(f"Invalid weighting: c/threshold - d must be >0 for {fn}.")
        if fn == "pow":
            return self.r0 * val ** (1.0 / self.m)
        if fn == "exp":
            return -self.r0 * math.log(val)
        raise ValueError(f"Unknown weighting function: {fn}")

    def value_and_derivative(self, r):
        """(w, dw/dr) for r >= 0; w0 (and slope 0) on r < 1e-12."""
        r = np.asarray(r, np.float64)
        if self.function is None:
            w, dw = np.ones_like(r), np.zeros_like(r)
        elif self.function == "poly":
            x = r / self.r0
            base = 1.0 + 2.0 * x ** 3 - 3.0 * x ** 2
            inside = (r <= self.r0) & (base > 0)
            bpos = np.where(inside, base, 1.0)
            w = np.where(inside, self.c * bpos ** self.m, 0.0)
            dw = np.where(inside, self.c * self.m * bpos ** (self.m - 1.0) * (6.0 * x * x - 6.0 * x) / self.r0, 0.0)
        elif self.function == "pow":
            x = r / self.r0
            xm = x ** self.m
            w = self.c / (self.d + xm)
            xm1 = np.where(x > 0, x ** (self.m - 1.0), 0.0 if self.m > 1 else (1.0 if self.m == 1 else np.inf))
            dw = -self.c * self.m * xm1 / self.r0 / (self.d + xm) ** 2
        elif self.function == "exp":
            e = np.exp(-r / self.r0)
            w = self.c / (self.d + e)
            dw = self.c * e / self.r0 / (self.d + e) ** 2
        else:
            raise ValueError(f"Unknown weighting function: {self.function}")
        tiny = r < 1e-12
        return np.where(tiny, self.w0, w), np.where(tiny, 0.0, dw)


# ---------------------------------------------------------------------------
# real solid harmonics (sphericart convention)
# ---------------------------------------------------------------------------

def _norms(l_max: int) -> np.ndarray:
    out = np.zeros((l_max + 1, l_max + 1))
    for l in range(l_max + 1):
        out[l, 0] = math.sqrt((2 * l + 1) / (4 * math.pi))
        for m in range(1, l + 1):
            out[l, m] = math.sqrt((2 * l + 1) / (2 * math.pi) * math.factorial(l - m) / math.factorial(l + m))
    return out


def solid_harmonics(xyz: np.ndarray, l_max: int, gradients: bool = False):
    """Real solid harmonics R_lm = r^l Y_lm(rhat), index l*l + l + m, m=-l..l.

    Q_l^m(z, r^2) recurrence: Q_m^m = (2m-1)!!, Q_{m+1}^m = (2m+1) z Q_m^m,
    Q_l^m = ((2l-1) z Q_{l-1}^m - (l+m-1) r^2 Q_{l-2}^m) / (l-m);
    R_l^0 = N_l0 Q_l^0, R_l^{+m} = N_lm Q_l^m Re(x+iy)^m, R_l^{-m} = N_lm Q_l^m Im(x+iy)^m.
    Gradients use dQ_l^m/dx = -x Q_{l-1}^{m+1}, dQ_l^m/dy = -y Q_{l-1}^{m+1},
    dQ_l^m/dz = (l+m) Q_{l-1}^m and d(x+iy)^m = m (x+iy)^{m-1} (dx + i dy).
    Returns R (E,K) and, if requested, dR (E,3,K).
    """
    xyz = np.asarray(xyz, dtype=np.float64)
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    E = xyz.shape[0]
    r2 = x * x + y * y + z * z
    Lp1 = l_max + 1
    Q = np.zeros((Lp1 + 1, Lp1 + 1, E))  # Q[l, m]; padded so Q[l-1, m+1] exists
    for m in range(Lp1):
        Q[m, m] = float(np.prod(np.arange(2 * m - 1, 0, -2))) if m > 0 else 1.0
        if m + 1 <= l_max:
            Q[m + 1, m] = (2 * m + 1) * z * Q[m, m]
        for l in range(m + 2, Lp1):
            Q[l, m] = ((2 * l - 1) * z * Q[l - 1, m] - (l + m - 1) * r2 * Q[l - 2, m]) / (l - m)
    C = np.zeros((Lp1, E))
    Sm = np.zeros((Lp1, E))
    C[0] = 1.0
    for m in range(1, Lp1):
        C[m] = x * C[m - 1] - y * Sm[m - 1]
        Sm[m] = x * Sm[m - 1] + y * C[m - 1]
    Nrm = _norms(l_max)
    K = Lp1 * Lp1
    R = np.zeros((E, K))
    dR = np.zeros((E, 3, K)) if gradients else None
    for l in range(Lp1):
        for m in range(-l, l + 1):
            am = abs(m)
            idx = l * l + l + m
            if m == 0:
                phi, dphx, dphy = 1.0, 0.0, 0.0
            elif m > 0:
                phi = C[am]
                dphx, dphy = am * C[am - 1], -am * Sm[am - 1]
            else:
                phi = Sm[am]
                dphx, dphy = am * Sm[am - 1], am * C[am - 1]
            q = Q[l, am]
            R[:, idx] = Nrm[l, am] * q * phi
            if gradients:
                qp = Q[l - 1, am + 1] if l >= 1 else np.zeros(E)
                qz = (l + am) * Q[l - 1, am] if l >= 1 else np.zeros(E)
                dR[:, 0, idx] = Nrm[l, am] * (-x * qp * phi + q * dphx)
                dR[:, 1, idx] = Nrm[l, am] * (-y * qp * phi + q * dphy)
                dR[:, 2, idx] = Nrm[l, am] * (qz * phi)
    return (R, dR) if gradients else R


# ---------------------------------------------------------------------------
# periodic images
# ---------------------------------------------------------------------------

def perpendicular_lengths(cell: np.ndarray) -> np.ndarray:
    """Perpendicular widths of the cell (SG:369-379)."""
    a, b, c = cell
    bc, ca, ab = np.cross(b, c), np.cross(c, a), np.cross(a, b)
    v = abs(float(np.dot(a, bc)))
    eps = 1e-12
    return np.array([v / (np.linalg.norm(bc) + eps), v / (np.linalg.norm(ca) + eps), v / (np.linalg.norm(ab) + eps)])


def image_repeats(cell: np.ndarray, pbc, cutoff: float) -> np.ndarray:
    """n_rep_i = ceil(cutoff / (perp_i + 1e-12)) on periodic axes, else 0 (SG:382-391)."""
    perps = perpendicular_lengths(cell)
    return np.array([int(math.ceil(cutoff / (perps[i] + 1e-12))) if bool(pbc[i]) else 0 for i in range(3)])


def pbc_offsets(cell: np.ndarray, pbc, cutoff: float) -> np.ndarray:
    """All integer image offsets in [-n_rep, n_rep]^3, ij-indexing (SG:382-396)."""
    n = image_repeats(cell, pbc, cutoff)
    rng = [np.arange(-n[i], n[i] + 1) for i in range(3)]
    ox, oy, oz = np.meshgrid(*rng, indexing="ij")
    return np.stack([ox.ravel(), oy.ravel(), oz.ravel()], axis=-1)


# ---------------------------------------------------------------------------
# the oracle SOAP
# ---------------------------------------------------------------------------

class OracleSOAP:
    """FP64 oracle with the reference constructor semantics (SG:524-634):
    rbf 'gto' or 'polynomial', optional DScribe weighting."""

    def __init__(self, r_cut=None, n_max=None, l_max=None, sigma=1.0, species=(1,), crossover=True,
                 average="off", periodic=False, rbf="gto", weighting=None, quad_n=100):
        self.weighting = None
        thr = 1e-2
        if weighting is not None:
            wd = dict(weighting)
            thr = float(wd.pop("threshold", 1e-2))
            self.weighting = Weighting(**wd)
        if r_cut is None:
            if self.weighting is None:
                raise ValueError("Either r_cut or weighting must be provided.")
            r_cut = self.weighting.infer_rcut(thr)
        self.rbf = str(rbf).lower()
        self.r_cut = float(r_cut)
        self.n_max = int(n_max)
        self.l_max = int(l_max)
        self.sigma = float(sigma)
        self.eta = 1.0 / (2.0 * self.sigma * self.sigma)
        self.species = sorted(set(int(s) for s in species))  # SG:563
        self.S = len(self.species)
        self.z2s = {z: i for i, z in enumerate(self.species)}
        self.crossover = bool(crossover)
        self.average = str(average)
        self.periodic = bool(periodic)
        # cutoff padding for the gaussian tails, threshold 1e-3 (SG:600-602)
        self.cutoff = self.r_cut + self.sigma * math.sqrt(-2.0 * math.log(1e-3))
        if self.rbf == "gto":
            self.alphas, self.betas = gto_basis(self.r_cut, self.n_max, self.l_max)
            self.gamma, self.pref = radial_tables(self.alphas, self.betas, self.eta)
        elif self.rbf == "polynomial":
            self.rx, self.wr, self.gss = poly_basis(self.r_cut, self.n_max, quad_n)
        else:
            raise ValueError("rbf must be 'gto' or 'polynomial'.")
        self.K = (self.l_max + 1) ** 2
        self.l_of_lm = np.array([l for l in range(self.l_max + 1) for _ in range(2 * l + 1)])
        self._build_feature_table()

    # ---- radial factors of one edge: c_nlm = B_nl R_lm, dB/drvec = rvec Bhat ----
    def radial_unweighted(self, r2):
        r2 = np.asarray(r2, np.float64)
        if self.rbf == "gto":
            return radial_B_Bhat(r2, self.betas, self.gamma, self.pref)
        return poly_B_Bhat(np.sqrt(r2), self.rx, self.wr, self.gss, self.eta, self.l_max)

    def radial(self, r2):
        """B[e,n,l], Bhat[e,n,l] including the weighting: w B and
        w Bhat + (dw/dr / r) B; r < 1e-12 edges take w0 (SG:466-469)."""
        B, Bh = self.radial_unweighted(r2)
        if self.weighting is None:
            return B, Bh
        r = np.sqrt(np.asarray(r2, np.float64))
        w, dw = self.weighting.value_and_derivative(r)
        rs = np.where(r < 1e-12, 1.0, r)
        return w[:, None, None] * B, w[:, None, None] * Bh + (dw / rs)[:, None, None] * B

    def self_l0(self):
        """l = 0 value of the centre's own Gaussian, w0 B_n0(0) Y00 (SG:765-797)."""
        B0, _ = self.radial_unweighted(np.zeros(1))
        w0 = self.weighting.w0 if self.weighting is not None else 1.0
        return w0 * B0[0, :, 0] * Y00

    # ---- feature bookkeeping (SG:908-962, SG:1215-1245) ----
    def n_power_features(self) -> int:
        if self.crossover:
            ch = self.S * self.n_max
            return ch * (ch + 1) // 2 * (self.l_max + 1)
        return self.S * (self.l_max + 1) * (self.n_max * (self.n_max + 1) // 2)

    def n_features(self) -> int:
        if self.average == "cc":
            return self.S * self.n_max * self.K
        return self.n_power_features()

    def _build_feature_table(self):
        rows = []
        N = self.n_max
        for j in range(self.S):
            jd_limit = self.S if self.crossover else j + 1
            for jd in range(j, jd_limit):
                for l in range(self.l_max + 1):
                    if j == jd:
                        pairs = [(a, b) for a in range(N) for b in range(a, N)]
                    else:
                        pairs = [(a, b) for a in range(N) for b in range(N)]
                    for a, b in pairs:
                        rows.append((j, jd, a, b, l))
        self.ftab = np.array(rows, dtype=np.int64).reshape(-1, 5)
        assert len(self.ftab) == self.n_power_features()
        self.fpref = np.sqrt(8.0 * math.pi ** 2 / (2 * self.ftab[:, 4] + 1))

    def get_location(self, pair) -> slice:
        i, j = self.z2s[int(pair[0])], self.z2s[int(pair[1])]
        if i > j:
            i, j = j, i
        symm = (self.n_max * (self.n_max + 1) // 2) * (self.l_max + 1)
        unsymm = self.n_max * self.n_max * (self.l_max + 1)
        if self.crossover:
            m_symm = i + int(j > i)
            m_unsymm = j + i * self.S - i * (i + 1) / 2 - m_symm
            start = int(m_symm * symm + m_unsymm * unsymm)
            return slice(start, start + (symm if i == j else unsymm))
        return slice(int(i * symm), int(i * symm) + symm)

    # ---- neighbour list (SG:1042-1181) ----
    def neighbor_list(self, positions, Z, centers_xyz, cell=None, pbc=None, keep_self=False,
                      center_atoms=None):
        """Edges (centre, neighbour atom, rvec) with |rvec| <= cutoff.

        keep_self=False reproduces the create() path: edges with r <= 1e-12 are
        dropped (SG:1174-1179) and the analytic self term is added separately.
        keep_self=True reproduces derivatives_analytical_ps, which keeps them
        (SG:2372-2373)."""
        positions = np.asarray(positions, dtype=np.float64)
        A = positions.shape[0]
        if self.periodic:
            offsets = pbc_offsets(np.asarray(cell, np.float64), pbc, self.cutoff)
            shifts = offsets.astype(np.float64) @ np.asarray(cell, np.float64)
        else:
            shifts = np.zeros((1, 3))
        cutoff2 = self.cutoff * self.cutoff
        ci_l, ai_l, rv_l = [], [], []
        C = centers_xyz.shape[0]
        if A * shifts.shape[0] > 200000:
            from scipy.spatial import cKDTree
            ext = (positions[None] + shifts[:, None]).reshape(-1, 3)
            tree = cKDTree(ext)
            lists = tree.query_ball_point(centers_xyz, self.cutoff)
            for c, lst in enumerate(lists):
                lst = np.asarray(sorted(lst), dtype=np.int64)
                rv = ext[lst] - centers_xyz[c]
                ok = (rv * rv).sum(1) <= cutoff2
                ci_l.append(np.full(int(ok.sum()), c))
                ai_l.append(lst[ok] % A)
                rv_l.append(rv[ok])
        else:
            ext = (positions[None] + shifts[:, None]).reshape(-1, 3)
            chunk = max(1, 2_000_000 // max(1, ext.shape[0]))
            for s in range(0, C, chunk):
                cpos = centers_xyz[s:s + chunk]
                rv = ext[None, :, :] - cpos[:, None, :]
                d2 = (rv * rv).sum(-1)
                cc, ee = np.nonzero(d2 <= cutoff2)
                ci_l.append(cc + s)
                ai_l.append(ee % A)
                rv_l.append(rv[cc, ee])
        ci = np.concatenate(ci_l) if ci_l else np.zeros(0, np.int64)
        ai = np.concatenate(ai_l) if ai_l else np.zeros(0, np.int64)
        rv = np.concatenate(rv_l) if rv_l else np.zeros((0, 3))
        if not keep_self:
            r = np.sqrt((rv * rv).sum(1))
            keep = r > 1e-12
            ci, ai, rv = ci[keep], ai[keep], rv[keep]
        return ci, ai, rv

    def prepare_centers(self, positions, centers):
        """Index or Cartesian centres; Cartesian centres within 1e-12 of an
        atom count as that atom (SG:966-1003)."""
        positions = np.asarray(positions, np.float64)
        if centers is None:
            return positions.copy(), np.arange(positions.shape[0])
        xyz, idx = [], []
        for c in centers:
            if isinstance(c, (int, np.integer)):
                xyz.append(positions[int(c)])
                idx.append(int(c))
            else:
                cc = np.asarray(c, np.float64).reshape(3)
                xyz.append(cc)
                d2 = ((positions - cc) ** 2).sum(1)
                j = int(np.argmin(d2)) if len(d2) else -1
                idx.append(j if j >= 0 and d2[j] <= 1e-24 else -1)
        return np.stack(xyz), np.asarray(idx, np.int64)

    # ---- coefficients (SG:1294-1391) + self term (SG:821-850) ----
    def coefficients(self, positions, Z, centers=None, cell=None, pbc=None, keep_self=False):
        positions = np.asarray(positions, np.float64)
        Z = np.asarray(Z, np.int64)
        cxyz, cidx = self.prepare_centers(positions, centers)
        ci, ai, rv = self.neighbor_list(positions, Z, cxyz, cell, pbc, keep_self=keep_self)
        sp = np.array([self.z2s[int(z)] for z in Z], np.int64)[ai] if len(ai) else np.zeros(0, np.int64)
        C = cxyz.shape[0]
        c = self._accumulate(C, ci, sp, rv)
        if not keep_self:
            # analytic self term (SG:765-785, SG:821-850): B_n0(0) * Y00 on the
            # centre's own species, l=0
            self_l0 = self.self_l0()
            for k in range(C):
                if cidx[k] >= 0:
                    c[k, self.z2s[int(Z[cidx[k]])], :, 0] += self_l0
        return c

    def _accumulate(self, C, ci, sp, rv, chunk=200000):
        N, K, S = self.n_max, self.K, self.S
        out = np.zeros((C * S, N * K))
        for s0 in range(0, len(ci), chunk):
            rvc = rv[s0:s0 + chunk]
            r2 = (rvc * rvc).sum(1)
            B, _ = self.radial(r2)
            R = solid_harmonics(rvc, self.l_max)
            contrib = (B[:, :, self.l_of_lm] * R[:, None, :]).reshape(len(rvc), N * K)
            np.add.at(out, ci[s0:s0 + chunk] * S + sp[s0:s0 + chunk], contrib)
        return out.reshape(C, S, N, K)

    # ---- outputs ----
    def power_spectrum(self, c: np.ndarray) -> np.ndarray:
        """p[c,f] = pref_l sum_m c[j,n,lm] c[j',n',lm] in DScribe order (SG:1634-1689).
        average inner/outer are centre-wise in the reference, identical to off."""
        C = c.shape[0]
        out = np.empty((C, len(self.ftab)))
        for l in range(self.l_max + 1):
            cl = c[..., l * l:(l + 1) * (l + 1)]
            P = np.einsum("cjnm,ckdm->cjknd", cl, cl) * math.sqrt(8 * math.pi ** 2 / (2 * l + 1))
            sel = self.ftab[:, 4] == l
            f = self.ftab[sel]
            out[:, sel] = P[:, f[:, 0], f[:, 1], f[:, 2], f[:, 3]]
        return out

    def cc_perm_scale(self):
        """DScribe cc convention (SG:1603-1622): l=1 stored (z,x,y) = source lm
        (2,3,1); lm >= 4 scaled by pi^-3/2."""
        perm = np.arange(self.K)
        if self.l_max >= 1:
            perm[1:4] = [2, 3, 1]
        scale = np.ones(self.K)
        scale[4:] = math.pi ** -1.5
        return perm, scale

    def projection_cc(self, c: np.ndarray) -> np.ndarray:
        perm, scale = self.cc_perm_scale()
        return (c[..., perm] * scale).reshape(c.shape[0], -1)

    def create(self, positions, Z, centers=None, cell=None, pbc=None) -> np.ndarray:
        """Forward descriptor (SG:1759-1810), float64."""
        c = self.coefficients(positions, Z, centers, cell, pbc, keep_self=False)
        if self.average == "cc":
            return self.projection_cc(c)
        return self.power_spectrum(c)

    # ---- closed-form Jacobian, fixed centres (SG:2270-2626) ----
    def derivatives(self, positions, Z, centers=None, include=None, exclude=None,
                    return_descriptor=True):
        """(C, n_inc, 3, F) Jacobian with DScribe fixed centres; r~0 self
        edges kept (solid harmonics are exact at 0).  Periodic systems are
        supported too (image edges of one atom accumulate)."""
        positions = np.asarray(positions, np.float64)
        Z = np.asarray(Z, np.int64)
        A = positions.shape[0]
        idx = list(range(A)) if include is None else [int(i) for i in include]
        if exclude is not None:
            ex = set(int(i) for i in exclude)
            idx = [i for i in idx if i not in ex]
        n_inc = len(idx)
        inv = np.full(A, -1, np.int64)
        inv[np.asarray(idx, np.int64)] = np.arange(n_inc)
        cxyz, _ = self.prepare_centers(positions, centers)
        C = cxyz.shape[0]
        ci, ai, rv = self.neighbor_list(positions, Z, cxyz, None, None, keep_self=True)
        zs = np.array([self.z2s[int(z)] for z in Z], np.int64)
        sp = zs[ai]
        N, K, S, Lp1 = self.n_max, self.K, self.S, self.l_max + 1
        F = self.n_features()
        r2 = (rv * rv).sum(1)
        B, Bh = self.radial(r2)
        R, dR = solid_harmonics(rv, self.l_max, gradients=True)
        Bl, Bhl = B[:, :, self.l_of_lm], Bh[:, :, self.l_of_lm]
        cE = (Bl * R[:, None, :])
        c = np.zeros((C * S, N * K))
        np.add.at(c, ci * S + sp, cE.reshape(-1, N * K))
        c = c.reshape(C, S, N, K)
        # edge gradient wrt the neighbour position (SG:2563-2567)
        g = rv[:, :, None, None] * (Bhl[:, None] * R[:, None, None, :]) + Bl[:, None] * dR[:, :, None, :]
        op = inv[ai]
        deriv = np.zeros((C, n_inc, 3, F))
        for k in range(C):
            sel = np.nonzero((ci == k) & (op >= 0))[0]
            D = np.zeros((n_inc, S, 3, N, K))
            np.add.at(D, (op[sel], sp[sel]), g[sel])
            if self.average == "cc":
                perm, scale = self.cc_perm_scale()
                deriv[k] = (D[..., perm] * scale).transpose(0, 2, 1, 3, 4).reshape(n_inc, 3, F)
            else:
                deriv[k] = self._ps_jacobian_rows(D, c[k])
        if return_descriptor:
            desc = self.projection_cc(c) if self.average == "cc" else self.power_spectrum(c)
            return deriv, desc
        return deriv

    def _ps_jacobian_rows(self, D, ck):
        """dp_f/dx_{a,d} = pref_l sum_m (D[a,j,d,n,lm] c[j',n',lm] + c[j,n,lm] D[a,j',d,n',lm])
        (product rule, SG:2592-2613)."""
        n_inc = D.shape[0]
        out = np.zeros((n_inc, 3, len(self.ftab)))
        for l in range(self.l_max + 1):
            s0, s1 = l * l, (l + 1) * (l + 1)
            X = np.einsum("ajdnm,kqm->adjnkq", D[..., s0:s1], ck[..., s0:s1])
            PD = math.sqrt(8 * math.pi ** 2 / (2 * l + 1)) * (X + X.transpose(0, 1, 4, 5, 2, 3))
            sel = self.ftab[:, 4] == l
            f = self.ftab[sel]
            out[:, :, sel] = PD[:, :, f[:, 0], f[:, 2], f[:, 1], f[:, 3]]
        return out

    # ---- forces through the descriptor: one reverse pass ----
    def forces(self, positions, Z, dEdp, cell=None, pbc=None, attach=True):
        """F_a = -dE/dx_a for E = sum_{c,f} dEdp[c,f] p[c,f], all atoms as centres.

        Restates one reverse-mode pass of the reference's differentiable forward
        (SG:2064-2098) in closed form: G = dE/dc per centre (product rule of the
        power spectrum), then per edge dE/drvec = sum G (rvec Bhat R + B dR).
        attach=True: centres move with their atoms, so each edge contributes
        -dE/drvec to the neighbour and +dE/drvec to the centre atom (self and
        own-image edges cancel).  attach=False: fixed centres, neighbour term
        only (the r~0 self edge contributes through its l=1 gradient)."""
        positions = np.asarray(positions, np.float64)
        Z = np.asarray(Z, np.int64)
        A = positions.shape[0]
        dEdp = np.asarray(dEdp, np.float64).reshape(A, -1)
        ci, ai, rv = self.neighbor_list(positions, Z, positions.copy(), cell, pbc, keep_self=True)
        zs = np.array([self.z2s[int(z)] for z in Z], np.int64)
        sp = zs[ai]
        N, K, S = self.n_max, self.K, self.S
        r2 = (rv * rv).sum(1)
        B, Bh = self.radial(r2)
        R, dR = solid_harmonics(rv, self.l_max, gradients=True)
        Bl, Bhl = B[:, :, self.l_of_lm], Bh[:, :, self.l_of_lm]
        c = np.zeros((A * S, N * K))
        np.add.at(c, ci * S + sp, (Bl * R[:, None, :]).reshape(-1, N * K))
        c = c.reshape(A, S, N, K)
        G = self.adjoint_G_cc(dEdp) if self.average == "cc" else self.adjoint_G(c, dEdp)
        Ge = G[ci, sp]  # (E, N, K)
        dEdr = (rv * (Ge * Bhl * R[:, None, :]).sum((1, 2))[:, None]
                + np.einsum("enk,edk->ed", Ge * Bl, dR))
        F = np.zeros((A, 3))
        np.add.at(F, ai, -dEdr)
        if attach:
            np.add.at(F, ci, dEdr)
        return F

    def adjoint_G_cc(self, dEdp):
        """G = dE/dc for E = sum dEdp * cc-projection: the cc layout's
        permutation and scale (SG:1603-1622) run backwards."""
        perm, scale = self.cc_perm_scale()
        C = dEdp.shape[0]
        D = np.asarray(dEdp, np.float64).reshape(C, self.S, self.n_max, self.K) * scale
        G = np.zeros_like(D)
        G[..., perm] = D
        return G

    def adjoint_G(self, c, dEdp):
        """G[c,s,n,lm] = dE/dc[c,s,n,lm] for E = sum dEdp * p (power spectrum)."""
        C = c.shape[0]
        N, S = self.n_max, self.S
        G = np.zeros_like(c)
        for l in range(self.l_max + 1):
            sel = np.nonzero(self.ftab[:, 4] == l)[0]
            f = self.ftab[sel]
            a = f[:, 0] * N + f[:, 2]
            b = f[:, 1] * N + f[:, 3]
            W = np.zeros((C, S * N, S * N))
            w = dEdp[:, sel] * self.fpref[sel][None]
            np.add.at(W, (slice(None), a, b), w)
            np.add.at(W, (slice(None), b, a), w)
            cl = c[..., l * l:(l + 1) * (l + 1)].reshape(C, S * N, -1)
            G[..., l * l:(l + 1) * (l + 1)] = np.einsum("cab,cbm->cam", W, cl).reshape(C, S, N, -1)
        return G


def energy(oracle: OracleSOAP, positions, Z, w, cell=None, pbc=None) -> float:
    """E = sum_i w . p_i over all atoms as centres (centres attached)."""
    p = oracle.create(positions, Z, None, cell, pbc)
    return float((p * np.asarray(w)[None, :]).sum())


def rel_l2(a, b) -> float:
    """||a - b|| / ||b||."""
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    nb = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (nb if nb > 0 else 1.0))
