// Radial basis (GTO or polynomial), weighting, FP32 radial tables and the
// feature index tables, built once per basis in FP64 on the device.
//
// Reference: SOAP._init_gto_basis (soap_generator.py:690-708),
// _lowdin_invsqrt (:339-343), _init_poly_basis (:710-752), the polynomial
// radial integrals _poly_I_J / _poly_B_Bhat (:1432-1594) with the scaled
// Bessel functions (:477-508), the Weighting class (:403-470), the self terms
// (:765-819), the cutoff padding (:600-602) and the feature slices
// (:1215-1291).
//
// Every edge's coefficients factor as c_nlm = B(r) R_lm(rvec) with the solid
// harmonic R_lm = r^l Y_lm, so the basis enters the kernels only through two
// radial functions of one variable per (n, l):
//     B(r) = w(r) B_nl(r),   D(r) = d/dr [w(r) B_nl(r)],
//   GTO:  B_nl(r) = sum_k beta^l_nk pref_kl exp(-gamma_kl r^2),
//         (1/r) dB_nl/dr = sum_k beta^l_nk (-2 gamma_kl) pref_kl exp(-gamma_kl r^2);
//   poly: B_nl(r) = 4 pi int rx^2 g_n(rx) exp(-eta (rx^2 + r^2)) (2 eta rx)^l phi_l(2 eta rx r) drx
//         with phi_l(t) = i_l(t) / t^l (modified spherical Bessel), and
//         (1/r) dB_nl/dr = 2 eta (B+_nl - B_nl), B+ the same integral with
//         rx (2 eta rx)^(l+1) phi_(l+1)  (from i_l' = i_(l+1) + (l/t) i_l).
// The Loewdin matrices have entries up to ~1e3 with cancellation (overlap
// condition ~1e6 for GTO at n_max = 8; the polynomial overlap is far worse, so
// its S^-1/2 comes from the caller, computed as the reference does), so the
// functions cannot be evaluated to 1e-6 from FP32 arithmetic.  They are
// sampled here in FP64 and stored as degree-7 polynomials on uniform radial
// segments (Chebyshev interpolation, converted to monomials in the local
// coordinate t in [-1, 1]); the kernels evaluate them with 7 FP32 FMAs.  D is
// stored rather than D / r because D / r is singular at r = 0 for weightings
// with w'(0) != 0 (pow with m = 1, exp); kernels multiply by 1 / r.  phi_l is
// summed from its power series for t <= 40 (positive terms, no cancellation)
// and from the upward recurrence above (stable for t >> l); the reference's
// upward recurrence with clamps loses digits for t < l, i.e. for high l at
// small r.  The build measures the table error against the FP64 functions.
#include <math.h>

#include "common.cuh"

namespace soapb {

struct BasisDev {
  int N, L, S, crossover, nseg, F, rbf, wfn, Q;
  double r_cut, eta, cutoff, h;
  double w_r0, w_c, w_d, w_m, w_w0;
  double* alpha;
  double* beta;
  const double* poly;  // rx[Q] | wr[Q] | g[N][Q]
  float* tab_b;
  float* tab_bh;
  float* tabf;     // function-major [fn][2 nseg][8]: w B on half-width segments
  float* selfv;    // w0 B_nl(0) per function fn = l N + n
  int* ftab;
  int* widx;
  double* err;
};

__device__ void atomic_max_nonneg(double* addr, double v) {
  atomicMax(reinterpret_cast<unsigned long long*>(addr), (unsigned long long)__double_as_longlong(v));
}

// w(r) and dw/dr of the DScribe weighting functions for r > 0 (the r = 0
// value w0 enters through the self values).
__device__ void weight(const BasisDev& a, double r, double& w, double& dw) {
  w = 1.0;
  dw = 0.0;
  if (a.wfn == SOAPB_W_POLY) {
    const double x = r / a.w_r0, base = 1.0 + 2.0 * x * x * x - 3.0 * x * x;
    if (r <= a.w_r0 && base > 0.0) {
      w = a.w_c * pow(base, a.w_m);
      dw = a.w_c * a.w_m * pow(base, a.w_m - 1.0) * (6.0 * x * x - 6.0 * x) / a.w_r0;
    } else {
      w = 0.0;
    }
  } else if (a.wfn == SOAPB_W_POW) {
    const double x = r / a.w_r0, xm = pow(x, a.w_m), den = a.w_d + xm;
    w = a.w_c / den;
    const double xm1 = (a.w_m == 1.0) ? 1.0 : (x > 0.0 ? pow(x, a.w_m - 1.0) : 0.0);
    dw = -a.w_c * a.w_m * xm1 / a.w_r0 / (den * den);
  } else if (a.wfn == SOAPB_W_EXP) {
    const double e = exp(-r / a.w_r0), den = a.w_d + e;
    w = a.w_c / den;
    dw = a.w_c * e / a.w_r0 / (den * den);
  }
}

// phi_l(t) = i_l(t) / t^l and phi_(l+1)(t), both times exp(-s) (s >= t keeps
// the products finite).
__device__ void scaled_phi(int l, double t, double s, double& pl, double& pl1) {
  if (t <= 40.0) {
    // i_l(t) / t^l = sum_k (t^2 / 2)^k / (k! (2l + 2k + 1)!!)
    double df = 1.0;
    for (int k = 3; k <= 2 * l + 1; k += 2) df *= (double)k;
    double term = 1.0 / df, sum = term;
    double term1 = term / (2.0 * l + 3.0), sum1 = term1;
    const double h2 = 0.5 * t * t;
    for (int k = 1; k < 400; ++k) {
      term *= h2 / (k * (2.0 * l + 2.0 * k + 1.0));
      term1 *= h2 / (k * (2.0 * l + 2.0 * k + 3.0));
      sum += term;
      sum1 += term1;
      if (k > t && term < 1e-18 * sum && term1 < 1e-18 * sum1) break;
    }
    const double e = exp(-s);
    pl = sum * e;
    pl1 = sum1 * e;
  } else {
    // ie_k = i_k(t) e^{-t} upward to k = l + 1, then / t^k and * e^{t - s}
    const double e2 = exp(-2.0 * t), ot = 1.0 / t;
    double im = 0.5 * ot * (1.0 - e2);                               // ie_0
    double ic = 0.5 * ot * (1.0 + e2) - 0.5 * ot * ot * (1.0 - e2);  // ie_1
    // ie_(k+1) = ie_(k-1) - (2k+1)/t ie_k with (im, ic) = (ie_(k-1), ie_k);
    // after the loop im = ie_l, ic = ie_(l+1)
    for (int k = 1; k <= l; ++k) {
      const double nxt = im - (2.0 * k + 1.0) * ot * ic;
      im = ic;
      ic = nxt;
    }
    const double tl = pow(t, (double)l);
    const double e = exp(t - s);
    pl = im / tl * e;
    pl1 = ic / (tl * t) * e;
  }
}

// Unweighted B_nl(r) and (1/r) dB_nl/dr (called Bhat) in FP64.
__device__ void exact_radial(const BasisDev& a, const double* s_gamma, const double* s_pref, int fn, double r,
                             double& b, double& bh) {
  const int N = a.N, l = fn / N, n = fn % N;
  b = 0.0;
  bh = 0.0;
  if (a.rbf == SOAPB_RBF_GTO) {
    for (int k = 0; k < N; ++k) {
      const double e = s_pref[l * kMaxN + k] * exp(-s_gamma[l * kMaxN + k] * r * r);
      const double be = a.beta[(l * N + n) * N + k];
      b += be * e;
      bh += be * (-2.0 * s_gamma[l * kMaxN + k]) * e;
    }
    return;
  }
  const int Q = a.Q;
  const double* rx = a.poly;
  const double* wr = a.poly + Q;
  const double* g = a.poly + 2 * Q + (size_t)n * Q;
  const double eta = a.eta;
  double bp = 0.0;
  for (int q = 0; q < Q; ++q) {
    const double x = rx[q], t = 2.0 * eta * x * r;
    // exp(-eta (x - r)^2) exp(-t) = exp(-eta (x^2 + r^2))
    const double s = eta * (x * x + r * r);
    double pl, pl1;
    scaled_phi(l, t, s, pl, pl1);
    const double u = 2.0 * eta * x;
    const double ul = pow(u, (double)l);
    const double common = 4.0 * kPi * wr[q] * x * x * g[q];
    b += common * ul * pl;
    bp += common * x * ul * u * pl1;
  }
  bh = 2.0 * eta * (bp - b);
}

// Table functions B = w B_nl and D = d(w B_nl)/dr.
__device__ void exact_BD(const BasisDev& a, const double* s_gamma, const double* s_pref, int fn, double r, double& B,
                         double& D) {
  double b, bh, w, dw;
  exact_radial(a, s_gamma, s_pref, fn, r, b, bh);
  weight(a, r, w, dw);
  B = w * b;
  D = dw * b + w * r * bh;
}

// Interpolant through the values f_j at the 8 Chebyshev nodes t_j of a
// segment, as float monomial coefficients in the local coordinate t.
__device__ void cheb_to_mono(const double (&f)[kNCoef], float* dst) {
  double cheb[kNCoef];
  for (int i = 0; i < kNCoef; ++i) {
    double s = 0.0;
    for (int j = 0; j < kNCoef; ++j) s += f[j] * cos(i * (2.0 * j + 1.0) * kPi / (2.0 * kNCoef));
    cheb[i] = s * 2.0 / kNCoef;
  }
  cheb[0] *= 0.5;
  // monomial coefficients: sum_i cheb_i T_i(t), T_{i+1} = 2 t T_i - T_{i-1}
  double mono[kNCoef] = {0}, Tprev[kNCoef] = {0}, Tcur[kNCoef] = {0}, Tnext[kNCoef];
  Tcur[0] = 1.0;  // T_0
  for (int i = 0; i < kNCoef; ++i) {
    for (int k = 0; k < kNCoef; ++k) mono[k] += cheb[i] * Tcur[k];
    for (int k = 0; k < kNCoef; ++k)
      Tnext[k] = (i == 0) ? (k == 1 ? 1.0 : 0.0) : (k > 0 ? 2.0 * Tcur[k - 1] : 0.0) - Tprev[k];
    for (int k = 0; k < kNCoef; ++k) { Tprev[k] = Tcur[k]; Tcur[k] = Tnext[k]; }
  }
  for (int k = 0; k < kNCoef; ++k) dst[k] = (float)mono[k];
}

__global__ void __launch_bounds__(512) k_basis_build(BasisDev a) {
  const int N = a.N, L = a.L, NF = N * (L + 1);
  __shared__ double s_gamma[(kMaxL + 1) * kMaxN];
  __shared__ double s_pref[(kMaxL + 1) * kMaxN];
  __shared__ int s_boff[kMaxS * kMaxS * (kMaxL + 1)];
  __shared__ double s_err[4 * (kMaxL + 1) * kMaxN];
  const int tid = threadIdx.x;

  if (a.rbf == SOAPB_RBF_GTO) {
    // alpha_{l,n} = -ln(1e-3 / a_n^l) / a_n^2, a = linspace(1, r_cut, N)
    for (int i = tid; i < NF; i += blockDim.x) {
      const int l = i / N, n = i % N;
      const double an = (N == 1) ? 1.0 : 1.0 + (a.r_cut - 1.0) * (double)n / (double)(N - 1);
      const double al = -log(1e-3 / pow(an, (double)l)) / (an * an);
      a.alpha[l * N + n] = al;
      const double p = al + a.eta;
      s_gamma[l * kMaxN + n] = al * a.eta / p;
      s_pref[l * kMaxN + n] = pow(kPi, 1.5) * pow(a.eta / p, (double)l) * pow(p, -1.5);
    }
    __syncthreads();

    // S_l, Jacobi eigendecomposition, beta_l = V diag(clamp(w, 1e-12)^-1/2) V^T
    if (tid <= L) {
      const int l = tid;
      double S[kMaxN * kMaxN], V[kMaxN * kMaxN];  // one thread per l; local memory
      // Gamma(l + 3/2) = (2l+1)!! sqrt(pi) / 2^(l+1)
      double g = sqrt(kPi);
      for (int k = 1; k <= 2 * l + 1; k += 2) g *= (double)k;
      g /= pow(2.0, (double)(l + 1));
      for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
          const double m = a.alpha[l * N + i] + a.alpha[l * N + j];
          S[i * kMaxN + j] = 0.5 * g * pow(m, -((double)l + 1.5));
          V[i * kMaxN + j] = (i == j) ? 1.0 : 0.0;
        }
      for (int sweep = 0; sweep < 60; ++sweep) {
        double off = 0.0, diag = 0.0;
        for (int i = 0; i < N; ++i) {
          diag += S[i * kMaxN + i] * S[i * kMaxN + i];
          for (int j = i + 1; j < N; ++j) off += S[i * kMaxN + j] * S[i * kMaxN + j];
        }
        if (off <= 1e-34 * diag) break;
        for (int p = 0; p < N; ++p)
          for (int q = p + 1; q < N; ++q) {
            const double apq = S[p * kMaxN + q];
            if (apq == 0.0) continue;
            const double app = S[p * kMaxN + p], aqq = S[q * kMaxN + q];
            const double theta = (aqq - app) / (2.0 * apq);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0), s = t * c;
            for (int k = 0; k < N; ++k) {  // columns p, q
              const double akp = S[k * kMaxN + p], akq = S[k * kMaxN + q];
              S[k * kMaxN + p] = c * akp - s * akq;
              S[k * kMaxN + q] = s * akp + c * akq;
            }
            for (int k = 0; k < N; ++k) {  // rows p, q
              const double apk = S[p * kMaxN + k], aqk = S[q * kMaxN + k];
              S[p * kMaxN + k] = c * apk - s * aqk;
              S[q * kMaxN + k] = s * apk + c * aqk;
            }
            for (int k = 0; k < N; ++k) {
              const double vkp = V[k * kMaxN + p], vkq = V[k * kMaxN + q];
              V[k * kMaxN + p] = c * vkp - s * vkq;
              V[k * kMaxN + q] = s * vkp + c * vkq;
            }
          }
      }
      for (int i = 0; i < N; ++i)
        for (int j = 0; j < N; ++j) {
          double acc = 0.0;
          for (int k = 0; k < N; ++k) {
            const double w = fmax(S[k * kMaxN + k], 1e-12);
            acc += V[i * kMaxN + k] * V[j * kMaxN + k] / sqrt(w);
          }
          a.beta[(l * N + i) * N + j] = acc;
        }
    }
    __syncthreads();
  } else {
    for (int i = tid; i < NF; i += blockDim.x) a.alpha[i] = 0.0;
    for (int i = tid; i < NF * N; i += blockDim.x) a.beta[i] = 0.0;
  }

  // Radial tables: Chebyshev interpolation at 8 nodes per segment, FP64.
  for (int task = tid; task < a.nseg * NF; task += blockDim.x) {
    const int seg = task / NF, fn = task % NF;
    double fb[kNCoef], fh[kNCoef];
    for (int j = 0; j < kNCoef; ++j) {
      const double tj = cos((2.0 * j + 1.0) * kPi / (2.0 * kNCoef));
      const double r = (seg + 0.5 * (tj + 1.0)) * a.h;
      exact_BD(a, s_gamma, s_pref, fn, r, fb[j], fh[j]);
    }
    cheb_to_mono(fb, a.tab_b + ((size_t)seg * NF + fn) * kNCoef);
    cheb_to_mono(fh, a.tab_bh + ((size_t)seg * NF + fn) * kNCoef);
  }
  // Force table: w B alone on segments of half the width, function-major; its
  // polynomial's derivative is D (the derivative of a degree-7 interpolant
  // loses about h per order, halving h wins back 2^7).
  for (int task = tid; task < 2 * a.nseg * NF; task += blockDim.x) {
    const int seg = task % (2 * a.nseg), fn = task / (2 * a.nseg);
    double f[kNCoef];
    for (int j = 0; j < kNCoef; ++j) {
      const double tj = cos((2.0 * j + 1.0) * kPi / (2.0 * kNCoef));
      const double r = (seg + 0.5 * (tj + 1.0)) * (0.5 * a.h);
      double d;
      exact_BD(a, s_gamma, s_pref, fn, r, f[j], d);
    }
    cheb_to_mono(f, a.tabf + ((size_t)fn * force_tab_stride(a.nseg) + seg) * kNCoef);
  }
  // self values: the centre's own Gaussian, w0 B_nl(0) (SG:765-819)
  for (int fn = tid; fn < NF; fn += blockDim.x) {
    double b, bh;
    exact_radial(a, s_gamma, s_pref, fn, 0.0, b, bh);
    a.selfv[fn] = (float)(a.w_w0 * b);
  }
  if (tid == 0) { a.err[0] = 0.0; a.err[1] = 0.0; }
  __syncthreads();

  // Table error: max |table - exact| / max |exact| per function, 17 points per
  // segment over [0, cutoff]; err[0] covers B (both tables), err[1] D (the D
  // table and the force table's derivative).  One task per (function,
  // segment), maxima gathered per function in shared memory.
  for (int fn = tid; fn < NF; fn += blockDim.x) {
    s_err[4 * fn + 0] = 0.0;  // |B error|, |D error|, max |B|, max |D|
    s_err[4 * fn + 1] = 0.0;
    s_err[4 * fn + 2] = 0.0;
    s_err[4 * fn + 3] = 0.0;
  }
  __syncthreads();
  for (int task = tid; task < 3 * a.nseg * NF; task += blockDim.x) {
    const int fn = task % NF, seg = task / NF;  // seg < nseg: B and D tables; above: the force table
    double eb = 0.0, eh = 0.0, mb = 0.0, mh = 0.0;
    if (seg < a.nseg) {
      const float* cb = a.tab_b + ((size_t)seg * NF + fn) * kNCoef;
      const float* ch = a.tab_bh + ((size_t)seg * NF + fn) * kNCoef;
      for (int j = 0; j <= 16; ++j) {
        const double t = -1.0 + j / 8.0;
        const double r = (seg + 0.5 * (t + 1.0)) * a.h;
        if (r > a.cutoff) continue;
        double b, bh;
        exact_BD(a, s_gamma, s_pref, fn, r, b, bh);
        double pb = cb[kDeg], ph = ch[kDeg];
        for (int k = kDeg - 1; k >= 0; --k) { pb = pb * t + cb[k]; ph = ph * t + ch[k]; }
        eb = fmax(eb, fabs(pb - b));
        eh = fmax(eh, fabs(ph - bh));
        mb = fmax(mb, fabs(b));
        mh = fmax(mh, fabs(bh));
      }
    } else {  // the force table: value, and derivative d/dr = (4 / h) d/dt
      const int sf = seg - a.nseg;
      const float* cf = a.tabf + ((size_t)fn * force_tab_stride(a.nseg) + sf) * kNCoef;
      for (int j = 0; j <= 16; ++j) {
        const double t = -1.0 + j / 8.0;
        const double r = (sf + 0.5 * (t + 1.0)) * (0.5 * a.h);
        if (r > a.cutoff) continue;
        double b, bh;
        exact_BD(a, s_gamma, s_pref, fn, r, b, bh);
        double p = cf[kDeg], dp = 0.0;
        for (int k = kDeg - 1; k >= 0; --k) {
          dp = dp * t + p;
          p = p * t + cf[k];
        }
        eb = fmax(eb, fabs(p - b));
        eh = fmax(eh, fabs(dp * 4.0 / a.h - bh));
      }
    }
    atomic_max_nonneg(&s_err[4 * fn + 0], eb);
    atomic_max_nonneg(&s_err[4 * fn + 1], eh);
    atomic_max_nonneg(&s_err[4 * fn + 2], mb);
    atomic_max_nonneg(&s_err[4 * fn + 3], mh);
  }
  __syncthreads();
  for (int fn = tid; fn < NF; fn += blockDim.x) {
    const double eb = s_err[4 * fn], eh = s_err[4 * fn + 1], mb = s_err[4 * fn + 2], mh = s_err[4 * fn + 3];
    atomic_max_nonneg(&a.err[0], mb > 0 ? eb / mb : 0.0);
    atomic_max_nonneg(&a.err[1], mh > 0 ? eh / mh : 0.0);
  }

  // Adjoint index table: widx[(l SN + b) SN + a] = feature of the pair {a, b} at l,
  // a = j N + n, bit 30 set on a == b (d(c_a c_a) = 2 c_a), -1 where no feature exists.
  {
    const int SN = a.S * N;
    for (int i = tid; i < (L + 1) * SN * SN; i += blockDim.x) a.widx[i] = -1;
  }
  // Power-spectrum feature table in DScribe order (SG:1215-1245).
  if (tid == 0) {
    int off = 0, nb = 0;
    const int S = a.S;
    for (int j = 0; j < S; ++j)
      for (int jd = j; jd < (a.crossover ? S : j + 1); ++jd)
        for (int l = 0; l <= L; ++l) {
          s_boff[nb++] = off;
          off += (j == jd) ? N * (N + 1) / 2 : N * N;
        }
  }
  __syncthreads();
  {
    const int S = a.S;
    int b = 0;
    for (int j = 0; j < S; ++j)
      for (int jd = j; jd < (a.crossover ? S : j + 1); ++jd)
        for (int l = 0; l <= L; ++l, ++b) {
          if (b % blockDim.x != tid) continue;
          int f = s_boff[b];
          for (int n = 0; n < N; ++n)
            for (int nd = (j == jd ? n : 0); nd < N; ++nd) {
              // l-major coefficient-pair indices (l S + j) N + n, (l S + j') N + n', and l
              a.ftab[f] = ((l * S + j) * N + n) | (((l * S + jd) * N + nd) << 12) | (l << 24);
              const int SN = S * N, ia = j * N + n, ib = jd * N + nd;
              a.widx[(l * SN + ib) * SN + ia] = f | (ia == ib ? (1 << 30) : 0);
              a.widx[(l * SN + ia) * SN + ib] = f | (ia == ib ? (1 << 30) : 0);
              ++f;
            }
        }
  }
}

}  // namespace soapb

using namespace soapb;

extern "C" int soapb_basis_plan(soapb_basis* b) {
  if (!b) return set_error(SOAPB_ERR_ARG, "null basis");
  if (b->n_max < 1 || b->n_max > kMaxN) return set_error(SOAPB_ERR_ARG, "n_max must be in [1, %d]", kMaxN);
  if (b->l_max < 0 || b->l_max > kMaxL) return set_error(SOAPB_ERR_ARG, "l_max must be in [0, %d]", kMaxL);
  if (b->l_max >= 10 && b->n_max > 8)
    return set_error(SOAPB_ERR_ARG, "l_max >= 10 is built for n_max <= 8 (got n_max %d)", b->n_max);
  if (b->n_species < 1 || b->n_species > kMaxS)
    return set_error(SOAPB_ERR_ARG, "n_species must be in [1, %d]", kMaxS);
  if (!(b->r_cut > 0.0) || !(b->sigma > 0.0)) return set_error(SOAPB_ERR_ARG, "r_cut and sigma must be > 0");
  if (b->rbf != SOAPB_RBF_GTO && b->rbf != SOAPB_RBF_POLY) return set_error(SOAPB_ERR_ARG, "unknown rbf %d", b->rbf);
  if (b->rbf == SOAPB_RBF_POLY && (b->quad_n < 2 || b->quad_n > 4096))
    return set_error(SOAPB_ERR_ARG, "polynomial basis needs quad_n in [2, 4096]");
  if (b->weighting < SOAPB_W_NONE || b->weighting > SOAPB_W_EXP)
    return set_error(SOAPB_ERR_ARG, "unknown weighting %d", b->weighting);
  if (b->weighting >= SOAPB_W_POLY && !(b->w_r0 > 0.0)) return set_error(SOAPB_ERR_ARG, "weighting r0 must be > 0");
  const int N = b->n_max, L = b->l_max, S = b->n_species;
  b->eta = 1.0 / (2.0 * b->sigma * b->sigma);
  b->cutoff = b->r_cut + b->sigma * sqrt(-2.0 * log(1e-3));
  // segment width: the narrowest Gaussian factor sets the scale (0.5 / sqrt(gamma_max))
  double gmax = b->eta;
  if (b->rbf == SOAPB_RBF_GTO) {
    gmax = 0.0;
    for (int l = 0; l <= L; ++l)
      for (int n = 0; n < N; ++n) {
        const double an = (N == 1) ? 1.0 : 1.0 + (b->r_cut - 1.0) * (double)n / (double)(N - 1);
        const double al = -log(1e-3 / pow(an, (double)l)) / (an * an);
        gmax = fmax(gmax, al * b->eta / (al + b->eta));
      }
  }
  double h = 0.5 / sqrt(gmax);
  if (b->weighting >= SOAPB_W_POLY) h = fmin(h, 0.5 * b->w_r0);
  int ns = (int)ceil(b->cutoff / h);
  if (ns < 4) ns = 4;
  if (b->seg_hint > ns) ns = b->seg_hint;
  h = b->cutoff / ns;
  if (b->weighting == SOAPB_W_POLY && b->w_r0 < b->cutoff) {
    // the poly weighting has a kink at r0: put a segment boundary there
    const int k = (int)ceil(b->w_r0 / h - 1e-9);
    h = b->w_r0 / k;
    ns = (int)ceil(b->cutoff / h - 1e-9);
  }
  b->n_seg = ns;
  b->seg_width = h;
  b->n_keys = S * b->n_seg;
  if (b->n_keys > kMaxKeys) return set_error(SOAPB_ERR_ARG, "n_species * n_seg = %d exceeds %d", b->n_keys, kMaxKeys);
  const int ch = S * N;
  b->n_feat_ps = b->crossover ? ch * (ch + 1) / 2 * (L + 1) : S * (L + 1) * (N * (N + 1) / 2);
  b->n_feat_cc = S * N * (L + 1) * (L + 1);
  const int NF = N * (L + 1);
  int64_t off = 0;
  b->off_alpha = off; off = align_up(off + 8 * (int64_t)NF, 256);
  b->off_beta = off; off = align_up(off + 8 * (int64_t)NF * N, 256);
  b->off_tab_b = off; off = align_up(off + 4 * (int64_t)b->n_seg * NF * kNCoef, 256);
  b->off_tab_bh = off; off = align_up(off + 4 * (int64_t)b->n_seg * NF * kNCoef, 256);
  b->off_ftab = off; off = align_up(off + 4 * (int64_t)b->n_feat_ps, 256);
  b->off_widx = off; off = align_up(off + 4 * (int64_t)(L + 1) * (S * N) * (S * N), 256);
  b->off_err = off; off = align_up(off + 16, 256);
  b->off_tabf = off; off = align_up(off + 4 * (int64_t)force_tab_stride(b->n_seg) * NF * kNCoef, 256);
  b->off_self = off; off = align_up(off + 4 * (int64_t)NF, 256);
  b->off_poly = off;
  if (b->rbf == SOAPB_RBF_POLY) off = align_up(off + 8 * (int64_t)(2 + N) * b->quad_n, 256);
  b->bytes = off;
  b->dev = nullptr;
  return SOAPB_OK;
}

extern "C" int soapb_basis_build(soapb_basis* b, void* dev_buf, void* stream) {
  if (!b || !dev_buf) return set_error(SOAPB_ERR_ARG, "null basis or buffer");
  if (b->bytes <= 0) return set_error(SOAPB_ERR_ARG, "call soapb_basis_plan first");
  if (((uintptr_t)dev_buf) % 256) return set_error(SOAPB_ERR_ARG, "basis buffer must be 256-byte aligned");
  if (b->rbf == SOAPB_RBF_POLY && !b->h_poly)
    return set_error(SOAPB_ERR_ARG, "polynomial basis needs h_poly (grid and orthonormal g_n)");
  b->dev = dev_buf;
  char* base = (char*)dev_buf;
  cudaStream_t st = (cudaStream_t)stream;
  BasisDev a;
  a.N = b->n_max; a.L = b->l_max; a.S = b->n_species; a.crossover = b->crossover ? 1 : 0;
  a.nseg = b->n_seg; a.F = b->n_feat_ps;
  a.rbf = b->rbf; a.wfn = b->weighting; a.Q = b->quad_n;
  a.r_cut = b->r_cut; a.eta = b->eta; a.cutoff = b->cutoff; a.h = b->seg_width;
  a.w_r0 = b->w_r0; a.w_c = b->w_c; a.w_d = b->w_d; a.w_m = b->w_m;
  a.w_w0 = (b->weighting == SOAPB_W_NONE) ? 1.0 : b->w_w0;
  a.alpha = (double*)(base + b->off_alpha);
  a.beta = (double*)(base + b->off_beta);
  a.poly = (const double*)(base + b->off_poly);
  a.tab_b = (float*)(base + b->off_tab_b);
  a.tab_bh = (float*)(base + b->off_tab_bh);
  a.tabf = (float*)(base + b->off_tabf);
  a.selfv = (float*)(base + b->off_self);
  a.ftab = (int*)(base + b->off_ftab);
  a.widx = (int*)(base + b->off_widx);
  a.err = (double*)(base + b->off_err);
  if (b->rbf == SOAPB_RBF_POLY) {
    int rc = check_cuda(cudaMemcpyAsync(base + b->off_poly, b->h_poly, 8 * (size_t)(2 + b->n_max) * b->quad_n,
                                        cudaMemcpyHostToDevice, st),
                        "polynomial grid upload");
    if (rc) return rc;
  }
  k_basis_build<<<1, 512, 0, st>>>(a);
  return check_launch("k_basis_build");
}

extern "C" int soapb_basis_download(const soapb_basis* b, double* h_alpha, double* h_beta, double* h_err2,
                                    void* stream) {
  if (!b || !b->dev) return set_error(SOAPB_ERR_ARG, "basis not built");
  const int NF = b->n_max * (b->l_max + 1);
  cudaStream_t st = (cudaStream_t)stream;
  const char* base = (const char*)b->dev;
  int rc;
  if (h_alpha && (rc = check_cuda(cudaMemcpyAsync(h_alpha, base + b->off_alpha, 8 * (size_t)NF,
                                                  cudaMemcpyDeviceToHost, st), "alpha download")))
    return rc;
  if (h_beta && (rc = check_cuda(cudaMemcpyAsync(h_beta, base + b->off_beta, 8 * (size_t)NF * b->n_max,
                                                 cudaMemcpyDeviceToHost, st), "beta download")))
    return rc;
  if (h_err2 && (rc = check_cuda(cudaMemcpyAsync(h_err2, base + b->off_err, 16, cudaMemcpyDeviceToHost, st),
                                 "err download")))
    return rc;
  return check_cuda(cudaStreamSynchronize(st), "basis download sync");
}
