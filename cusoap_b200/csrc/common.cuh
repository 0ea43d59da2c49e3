// Shared device/host helpers of libsoapb200 (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/soapb200.h"

namespace soapb {

constexpr int kDeg = 7;              // radial table: degree-7 polynomial per segment
constexpr int kNCoef = kDeg + 1;
// Function stride of the force table, in half-width segments: 64 when the 2 n_seg half
// segments fit (the edge kernel's table offsets are then compile-time constants), else 2 n_seg.
constexpr int kForceSegStride = 64;
__host__ __device__ inline int force_tab_stride(int nseg) {
  return 2 * nseg <= kForceSegStride ? kForceSegStride : 2 * nseg;
}
constexpr int kMaxL = 12;
constexpr int kMaxN = 16;
constexpr int kMaxS = 16;
constexpr int kMaxKeys = 1024;       // species x radial segments (neighbour sort keys)
constexpr int kAtomBits = 27;        // pair word: atom | species << 27
constexpr int kAtomMask = (1 << kAtomBits) - 1;
constexpr double kPi = 3.14159265358979323846;

// ---- error reporting (capi.cu) ----
int set_error(int status, const char* fmt, ...);
int check_cuda(cudaError_t e, const char* what);
void count_launches(int n);
// Every kernel launch of the library is followed by check_launch(what, n):
// n = number of kernels launched since the previous check.
inline int check_launch(const char* what, int n = 1) {
  count_launches(n);
  return check_cuda(cudaGetLastError(), what);
}

inline int64_t align_up(int64_t x, int64_t a) { return (x + a - 1) / a * a; }

// ---- radial tables ----
// Function index of (n, l) inside a table segment: l-major.
__host__ __device__ inline int fn_index(int n, int l, int N) { return l * N + n; }

// Evaluate the degree-7 segment polynomial with Horner's rule.
__device__ __forceinline__ float horner7(const float (&a)[kNCoef], float t) {
  float p = a[7];
  p = fmaf(p, t, a[6]);
  p = fmaf(p, t, a[5]);
  p = fmaf(p, t, a[4]);
  p = fmaf(p, t, a[3]);
  p = fmaf(p, t, a[2]);
  p = fmaf(p, t, a[1]);
  p = fmaf(p, t, a[0]);
  return p;
}

// Value p and derivative dp/dt of the degree-7 segment polynomial in one pass.
__device__ __forceinline__ void horner7_d(const float (&a)[kNCoef], float t, float& p, float& dp) {
  p = a[7];
  dp = 0.0f;
#pragma unroll
  for (int k = kDeg - 1; k >= 0; --k) {
    dp = fmaf(dp, t, p);
    p = fmaf(p, t, a[k]);
  }
}

__device__ __forceinline__ void load_coef(const float* __restrict__ tab, int seg, int fn, int NF,
                                          float (&a)[kNCoef]) {
  const float4* p = reinterpret_cast<const float4*>(tab + ((size_t)seg * NF + fn) * kNCoef);
  float4 u = __ldg(p), v = __ldg(p + 1);
  a[0] = u.x; a[1] = u.y; a[2] = u.z; a[3] = u.w;
  a[4] = v.x; a[5] = v.y; a[6] = v.z; a[7] = v.w;
}

// Segment index and local coordinate t in [-1, 1] of radius r.
__device__ __forceinline__ void seg_coord(float r, float inv_h, int nseg, int& seg, float& t) {
  float u = r * inv_h;
  seg = min((int)u, nseg - 1);
  t = 2.0f * (u - (float)seg) - 1.0f;
}

// ---- real solid harmonics, sphericart convention ----
// R_lm = r^l Y_lm(rhat), index l*l + l + m, m = -l..l, orthonormal real
// harmonics without the Condon-Shortley phase: l = 1 is sqrt(3/4pi) (y, z, x).
// Q_l^m(z, r^2): Q_m^m = (2m-1)!!, Q_{m+1}^m = (2m+1) z Q_m^m,
// Q_l^m = ((2l-1) z Q_{l-1}^m - (l+m-1) r^2 Q_{l-2}^m) / (l-m);
// R_l^0 = N_l0 Q_l^0, R_l^{+-m} = N_lm Q_l^m {Re, Im}(x + i y)^m.
// Normalisation constants N_lm = sqrt((2l+1)/(4pi) (2 - delta_m0) (l-m)!/(l+m)!)
// are computed at compile time (Newton square root in double) into a
// per-translation-unit constant-memory table, index l*(kMaxL+1)+m.
namespace detail {
constexpr double csqrt(double x) {
  double g = x > 1.0 ? x : 1.0;
  for (int i = 0; i < 200; ++i) g = 0.5 * (g + x / g);
  return g;
}
constexpr double cfact(int n) {
  double f = 1.0;
  for (int i = 2; i <= n; ++i) f *= (double)i;
  return f;
}
struct ShNorm {
  float v[(kMaxL + 1) * (kMaxL + 1)];
};
constexpr ShNorm make_shnorm() {
  ShNorm t{};
  for (int l = 0; l <= kMaxL; ++l)
    for (int m = 0; m <= l; ++m) {
      const double base = (2.0 * l + 1.0) / (4.0 * kPi) * (m == 0 ? 1.0 : 2.0) * cfact(l - m) / cfact(l + m);
      t.v[l * (kMaxL + 1) + m] = (float)csqrt(base);
    }
  return t;
}
}  // namespace detail
static __constant__ detail::ShNorm c_shnorm_tab = detail::make_shnorm();
#define c_shnorm (c_shnorm_tab.v)

__host__ __device__ constexpr int tri(int l, int m) { return l * (l + 1) / 2 + m; }

template <int L>
struct SolidHarmonics {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int NQ = (L + 1) * (L + 2) / 2;

  // Q_l^m for all l <= L, m <= l.
  __device__ __forceinline__ static void legendre(float z, float r2, float (&Q)[NQ]) {
#pragma unroll
    for (int m = 0; m <= L; ++m) {
      float dfact = 1.0f;
#pragma unroll
      for (int k = 2 * m - 1; k > 0; k -= 2) dfact *= (float)k;
      Q[tri(m, m)] = dfact;
      if (m + 1 <= L) Q[tri(m + 1, m)] = (float)(2 * m + 1) * z * dfact;
#pragma unroll
      for (int l = m + 2; l <= L; ++l) {
        const float a = (float)(2 * l - 1) / (float)(l - m);
        const float b = (float)(l + m - 1) / (float)(l - m);
        Q[tri(l, m)] = a * z * Q[tri(l - 1, m)] - b * r2 * Q[tri(l - 2, m)];
      }
    }
  }

  // Values into dst[0..K).
  template <class Store>
  __device__ __forceinline__ static void values(float x, float y, float z, Store&& store) {
    const float r2 = x * x + y * y + z * z;
    float Q[NQ];
    legendre(z, r2, Q);
    float C = 1.0f, S = 0.0f;
#pragma unroll
    for (int m = 0; m <= L; ++m) {
      if (m > 0) {
        const float Cn = x * C - y * S;
        S = x * S + y * C;
        C = Cn;
      }
#pragma unroll
      for (int l = m; l <= L; ++l) {
        const float nq = c_shnorm[l * (kMaxL + 1) + m] * Q[tri(l, m)];
        if (m == 0) {
          store(l * l + l, nq);
        } else {
          store(l * l + l + m, nq * C);
          store(l * l + l - m, nq * S);
        }
      }
    }
  }

  // Values and Cartesian gradients: store(idx, v, dx, dy, dz).
  // dQ_l^m/dx = -x Q_{l-1}^{m+1}, dQ_l^m/dy = -y Q_{l-1}^{m+1},
  // dQ_l^m/dz = (l+m) Q_{l-1}^m; d(x+iy)^m = m (x+iy)^{m-1} (dx + i dy).
  template <class Store>
  __device__ __forceinline__ static void with_gradients(float x, float y, float z, Store&& store) {
    const float r2 = x * x + y * y + z * z;
    float Q[NQ];
    legendre(z, r2, Q);
    float C = 1.0f, S = 0.0f, Cp = 0.0f, Sp = 0.0f;  // (x+iy)^m and ^(m-1)
#pragma unroll
    for (int m = 0; m <= L; ++m) {
      if (m > 0) {
        Cp = C;
        Sp = S;
        const float Cn = x * C - y * S;
        S = x * S + y * C;
        C = Cn;
      }
#pragma unroll
      for (int l = m; l <= L; ++l) {
        const float nrm = c_shnorm[l * (kMaxL + 1) + m];
        const float q = Q[tri(l, m)];
        const float qp = (l >= 1 && m + 1 <= l - 1) ? Q[tri(l - 1, m + 1)] : 0.0f;
        const float qz = (l >= 1 && m <= l - 1) ? (float)(l + m) * Q[tri(l - 1, m)] : 0.0f;
        if (m == 0) {
          store(l * l + l, nrm * q, nrm * (-x * qp), nrm * (-y * qp), nrm * qz);
        } else {
          const float fm = (float)m;
          // +m: Re (x+iy)^m
          store(l * l + l + m, nrm * q * C, nrm * (-x * qp * C + q * fm * Cp), nrm * (-y * qp * C - q * fm * Sp),
                nrm * qz * C);
          // -m: Im (x+iy)^m
          store(l * l + l - m, nrm * q * S, nrm * (-x * qp * S + q * fm * Sp), nrm * (-y * qp * S + q * fm * Cp),
                nrm * qz * S);
        }
      }
    }
  }
};

// Dispatch a functor templated on l_max (0..kMaxL).
template <template <int> class F, class... Args>
inline int dispatch_l(int l, Args&&... args) {
  switch (l) {
    case 0: return F<0>::run(args...);
    case 1: return F<1>::run(args...);
    case 2: return F<2>::run(args...);
    case 3: return F<3>::run(args...);
    case 4: return F<4>::run(args...);
    case 5: return F<5>::run(args...);
    case 6: return F<6>::run(args...);
    case 7: return F<7>::run(args...);
    case 8: return F<8>::run(args...);
    case 9: return F<9>::run(args...);
    case 10: return F<10>::run(args...);
    case 11: return F<11>::run(args...);
    case 12: return F<12>::run(args...);
    default: return set_error(SOAPB_ERR_UNSUPPORTED, "l_max %d > %d not built", l, kMaxL);
  }
}

// Lane -> radial function assignment of the descriptor / adjoint kernels.
// single: lane i owns f = (n = i % N, l = i / N), needs N (L+1) <= 32.
// paired: lane owns (n, l) and (n, L-l) (l < L-l), or two (n, L/2) for even L,
// so every busy lane holds 2L+2 accumulators.
struct LaneFns {
  int n0, l0, n1, l1;  // l1 < 0: no second function; l0 < 0: idle lane
};

__host__ __device__ inline int lanes_needed(int N, int L, bool paired) {
  if (!paired) return N * (L + 1);
  int p1 = ((L + 1) / 2) * N;
  if (L % 2 == 0) p1 += (N + 1) / 2;
  return p1;
}

__host__ __device__ inline LaneFns lane_fns(int lane, int N, int L, bool paired) {
  LaneFns f{-1, -1, -1, -1};
  if (!paired) {
    if (lane < N * (L + 1)) { f.n0 = lane % N; f.l0 = lane / N; }
    return f;
  }
  const int p1 = ((L + 1) / 2) * N;
  if (lane < p1) {
    f.n0 = lane % N; f.l0 = lane / N; f.n1 = f.n0; f.l1 = L - f.l0;
  } else if (L % 2 == 0) {
    const int j = lane - p1;
    if (2 * j < N) {
      f.n0 = 2 * j; f.l0 = L / 2;
      if (2 * j + 1 < N) { f.n1 = 2 * j + 1; f.l1 = L / 2; }
    }
  }
  return f;
}


}  // namespace soapb
