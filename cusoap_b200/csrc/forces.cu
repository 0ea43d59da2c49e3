// Force adjoint: dE/dp (per centre, per power-spectrum feature) -> per-atom
// forces, without materialising the (C, A, 3, F) Jacobian.
//
// Reference: the reference differentiates its forward pass with autograd
// (derivatives_analytical, soap_generator.py:2007-2113; one reverse pass with
// grad_outputs = dE/dp is the feasible form of it).  The same reverse pass in
// closed form:
//   G[c, a, lm] = dE/dc[c, a, lm] = pref_l sum_b W_l[a, b] c[c, b, lm],
//     W_l[a, b] = dE/dp_f for the feature f of the pair {a, b} at l (2x on a = b),
//     a = (species j, radial n);
//   dE/drvec_e = sum_{n,l} ( rvec Bhat_nl u_nl + B_nl v_nl ),
//     u_nl = sum_m G[s_e, n, lm] R_lm(rvec_e), v_nl = sum_m G[s_e, n, lm] grad R_lm(rvec_e);
//   F[neighbour] -= dE/drvec_e, and with attach F[centre atom] += dE/drvec_e
//   (centres move with their atoms; self and own-image edges cancel).
//
// Mapping: one warp per centre (atomic work queue).  G is built in shared
// memory; then, as in the descriptor kernel, lanes own radial functions
// (n, l), pairs come sorted by (species, segment), solid harmonics and their
// gradients are staged 32 edges at a time, and each edge's 3-vector is a
// warp reduction followed by one atomic add per component.
#include "common.cuh"

namespace soapb {

struct ForceArgs {
  const int64_t* pair_off;
  const float4* pairs;
  const float* coeff;
  const float* dEdp;
  const int* centre_atom;
  const float* tab_b;
  const float* tab_bh;
  float* forces;
  int* counter;
  int64_t n_centres;
  int N, S, nseg, F, crossover, attach;
  float inv_h;
};

// Index of the power-spectrum feature of the unordered pair {(j,n), (jd,nd)} at l, or -1.
__device__ __forceinline__ int feature_index(int j, int n, int jd, int nd, int l, int N, int S, int L, int crossover) {
  if (j > jd || (j == jd && n > nd)) {
    int t = j; j = jd; jd = t;
    t = n; n = nd; nd = t;
  }
  const int Nd = N * (N + 1) / 2, No = N * N;
  if (!crossover) {
    if (j != jd) return -1;
    return (j * Nd) * (L + 1) + l * Nd + (n * N - n * (n - 1) / 2 + (nd - n));
  }
  const int bi = j * S - j * (j - 1) / 2 + (jd - j);  // block index of (j, jd), j <= jd
  const int ndiag = j + (jd > j ? 1 : 0);              // diagonal blocks before it
  const int start = (ndiag * Nd + (bi - ndiag) * No) * (L + 1);
  if (j == jd) return start + l * Nd + (n * N - n * (n - 1) / 2 + (nd - n));
  return start + l * No + n * N + nd;
}

template <int L>
struct ForceShape {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int KC = K | 1;
  static constexpr int YS = (4 * K) | 1;  // R and 3 gradient rows per staged edge
  __host__ __device__ static int warp_floats(int S, int N, int F) { return 32 * YS + 128 + 2 * S * N * KC + F; }
};

template <int L, bool PAIRED>
__global__ void __launch_bounds__(128) k_forces(ForceArgs a) {
  using Sh = ForceShape<L>;
  constexpr int K = Sh::K, KC = Sh::KC, YS = Sh::YS;
  constexpr int MT = PAIRED ? 2 * L + 2 : 2 * L + 1;
  extern __shared__ float sm[];
  __shared__ float s_pref[kMaxL + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int N = a.N, S = a.S, NF = N * (L + 1), F = a.F;
  float* Y = sm + (size_t)wid * Sh::warp_floats(S, N, F);  // 32 x (R | dRx | dRy | dRz)
  float* tt = Y + 32 * YS;
  int* sg = (int*)(tt + 32);
  int* spp = sg + 32;
  int* atm = spp + 32;
  float* cb = (float*)(atm + 32);  // S N KC coefficients
  float* G = cb + S * N * KC;      // S N KC adjoint
  float* w = G + S * N * KC;       // F
  if (threadIdx.x <= L) s_pref[threadIdx.x] = sqrtf(8.0f * (float)(kPi * kPi) / (2.0f * threadIdx.x + 1.0f));
  __syncthreads();

  const LaneFns lf = lane_fns(lane, N, L, PAIRED);
  const int m0 = lf.l0 >= 0 ? 2 * lf.l0 + 1 : 0;
  const int mtot = m0 + (lf.l1 >= 0 ? 2 * lf.l1 + 1 : 0);
  const int yoff0 = lf.l0 >= 0 ? lf.l0 * lf.l0 : 0;
  const int yoff1 = lf.l1 >= 0 ? lf.l1 * lf.l1 - m0 : 0;
  const int fn0 = lf.l0 >= 0 ? fn_index(lf.n0, lf.l0, N) : 0;
  const int fn1 = lf.l1 >= 0 ? fn_index(lf.n1, lf.l1, N) : 0;

  for (;;) {
    int c32 = 0;
    if (lane == 0) c32 = atomicAdd(a.counter, 1);
    const int64_t c = __shfl_sync(0xffffffffu, c32, 0);
    if (c >= a.n_centres) break;
    const int catom = a.attach ? a.centre_atom[c] : -1;
    for (int i = lane; i < S * N * K; i += 32) cb[(i / K) * KC + (i % K)] = a.coeff[(size_t)c * S * N * K + i];
    for (int f = lane; f < F; f += 32) w[f] = a.dEdp[(size_t)c * F + f];
    __syncwarp();
    // G = dE/dc: one task per (a = (j, n), l)
    for (int t = lane; t < S * N * (L + 1); t += 32) {
      const int ai = t / (L + 1), l = t % (L + 1);
      const int j = ai / N, n = ai % N;
      float g[2 * L + 1];
#pragma unroll
      for (int m = 0; m < 2 * L + 1; ++m) g[m] = 0.0f;
      for (int bi = 0; bi < S * N; ++bi) {
        const int f = feature_index(j, n, bi / N, bi % N, l, N, S, L, a.crossover);
        if (f < 0) continue;
        const float wt = w[f] * s_pref[l] * (bi == ai ? 2.0f : 1.0f);
        const float* cr = cb + bi * KC + l * l;
#pragma unroll
        for (int m = 0; m < 2 * L + 1; ++m)
          if (m < 2 * l + 1) g[m] = fmaf(wt, cr[m], g[m]);
      }
#pragma unroll
      for (int m = 0; m < 2 * L + 1; ++m)
        if (m < 2 * l + 1) G[ai * KC + l * l + m] = g[m];
    }
    __syncwarp();

    float gr[MT];
    float cf0[kNCoef], cf1[kNCoef], ch0[kNCoef], ch1[kNCoef];
#pragma unroll
    for (int k = 0; k < kNCoef; ++k) { cf0[k] = cf1[k] = ch0[k] = ch1[k] = 0.0f; }
#pragma unroll
    for (int k = 0; k < MT; ++k) gr[k] = 0.0f;
    int cur_sp = -1, cur_seg = -1;
    float fcx = 0.f, fcy = 0.f, fcz = 0.f;  // centre-atom force (lane 0)
    const int64_t p0 = a.pair_off[c], p1 = a.pair_off[c + 1];
    for (int64_t base = p0; base < p1; base += 32) {
      const int nt = (int)min((int64_t)32, p1 - base);
      if (lane < nt) {
        const float4 pr = __ldg(a.pairs + base + lane);
        const int wd = __float_as_int(pr.w);
        const float r = sqrtf(pr.x * pr.x + pr.y * pr.y + pr.z * pr.z);
        int seg;
        float t;
        seg_coord(r, a.inv_h, a.nseg, seg, t);
        tt[lane] = t;
        sg[lane] = seg;
        spp[lane] = (int)((unsigned)wd >> kAtomBits);
        atm[lane] = wd & kAtomMask;
        float* yrow = Y + lane * YS;
        SolidHarmonics<L>::with_gradients(pr.x, pr.y, pr.z, [&](int idx, float v, float dx, float dy, float dz) {
          yrow[idx] = v; yrow[K + idx] = dx; yrow[2 * K + idx] = dy; yrow[3 * K + idx] = dz;
        });
      }
      __syncwarp();
      for (int q = 0; q < nt; ++q) {
        const int sp = spp[q];
        if (sp != cur_sp) {
#pragma unroll
          for (int k = 0; k < MT; ++k) {
            gr[k] = 0.0f;
            if (k < mtot) {
              const bool first = k < m0;
              const int n = first ? lf.n0 : lf.n1, l = first ? lf.l0 : lf.l1, m = first ? k : k - m0;
              gr[k] = G[(sp * N + n) * KC + l * l + m];
            }
          }
          cur_sp = sp;
        }
        const int seg = sg[q];
        if (seg != cur_seg) {
          if (lf.l0 >= 0) { load_coef(a.tab_b, seg, fn0, NF, cf0); load_coef(a.tab_bh, seg, fn0, NF, ch0); }
          if (PAIRED && lf.l1 >= 0) { load_coef(a.tab_b, seg, fn1, NF, cf1); load_coef(a.tab_bh, seg, fn1, NF, ch1); }
          cur_seg = seg;
        }
        const float t = tt[q];
        const float B0 = horner7(cf0, t), H0 = horner7(ch0, t);
        const float B1 = PAIRED ? horner7(cf1, t) : 0.0f, H1 = PAIRED ? horner7(ch1, t) : 0.0f;
        const float* yr = Y + q * YS;
        float u0 = 0.f, u1 = 0.f, vx0 = 0.f, vx1 = 0.f, vy0 = 0.f, vy1 = 0.f, vz0 = 0.f, vz1 = 0.f;
#pragma unroll
        for (int k = 0; k < MT; ++k) {
          if (k < mtot) {
            const bool first = k < m0;
            const int yi = k + (first ? yoff0 : yoff1);
            const float g = gr[k];
            const float ru = g * yr[yi], rx = g * yr[K + yi], ry = g * yr[2 * K + yi], rz = g * yr[3 * K + yi];
            if (first) { u0 += ru; vx0 += rx; vy0 += ry; vz0 += rz; }
            else { u1 += ru; vx1 += rx; vy1 += ry; vz1 += rz; }
          }
        }
        // rvec from the pair (re-read: rows hold R and gradients only)
        const float4 pr = __ldg(a.pairs + base + q);
        const float hu = H0 * u0 + H1 * u1;
        float ex = pr.x * hu + B0 * vx0 + B1 * vx1;
        float ey = pr.y * hu + B0 * vy0 + B1 * vy1;
        float ez = pr.z * hu + B0 * vz0 + B1 * vz1;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          ex += __shfl_xor_sync(0xffffffffu, ex, o);
          ey += __shfl_xor_sync(0xffffffffu, ey, o);
          ez += __shfl_xor_sync(0xffffffffu, ez, o);
        }
        const int atom = atm[q];
        if (lane == 0) {
          if (!(a.attach && atom == catom)) {
            atomicAdd(&a.forces[3 * (size_t)atom + 0], -ex);
            atomicAdd(&a.forces[3 * (size_t)atom + 1], -ey);
            atomicAdd(&a.forces[3 * (size_t)atom + 2], -ez);
            fcx += ex; fcy += ey; fcz += ez;
          }
        }
      }
      __syncwarp();
    }
    if (lane == 0 && catom >= 0) {
      atomicAdd(&a.forces[3 * (size_t)catom + 0], fcx);
      atomicAdd(&a.forces[3 * (size_t)catom + 1], fcy);
      atomicAdd(&a.forces[3 * (size_t)catom + 2], fcz);
    }
    __syncwarp();
  }
}

template <int L, bool PAIRED>
static int launch_forces(const ForceArgs& a, cudaStream_t st) {
  const int per_warp = 4 * ForceShape<L>::warp_floats(a.S, a.N, a.F);
  int wpb = (200 * 1024) / per_warp;
  wpb = wpb > 4 ? 4 : wpb;
  if (wpb < 1) return set_error(SOAPB_ERR_UNSUPPORTED, "forces shared memory %d B per warp too large", per_warp);
  const int smem = wpb * per_warp;
  auto kern = k_forces<L, PAIRED>;
  int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                      "forces smem attribute");
  if (rc) return rc;
  int dev = 0, nsm = 148, occ = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * wpb, smem);
  if (occ < 1) occ = 1;
  int64_t blocks = (int64_t)nsm * occ;
  const int64_t need = (a.n_centres + wpb - 1) / wpb;
  if (blocks > need) blocks = need;
  if (blocks < 1) blocks = 1;
  kern<<<(unsigned)blocks, 32 * wpb, smem, st>>>(a);
  return check_launch("k_forces");
}

template <int L>
struct ForceDispatch {
  static int run(const ForceArgs& a, bool paired, cudaStream_t st) {
    return paired ? launch_forces<L, true>(a, st) : launch_forces<L, false>(a, st);
  }
};

}  // namespace soapb

using namespace soapb;

extern "C" int soapb_forces(const soapb_basis* b, int64_t n_centres, const int64_t* d_pair_off, const void* d_pairs,
                            const float* d_coeff, const float* d_dEdp, const int32_t* d_centre_atom, int32_t attach,
                            float* d_forces, int32_t* d_counter, void* stream) {
  if (!b || !b->dev) return set_error(SOAPB_ERR_ARG, "basis not built");
  if (n_centres < 0 || n_centres >= (int64_t)1 << 31) return set_error(SOAPB_ERR_ARG, "bad n_centres");
  if (n_centres == 0) return SOAPB_OK;
  if (!d_pair_off || !d_coeff || !d_dEdp || !d_forces || !d_counter) return set_error(SOAPB_ERR_ARG, "null argument");
  if (attach && !d_centre_atom) return set_error(SOAPB_ERR_ARG, "attach needs centre atoms");
  const int N = b->n_max, L = b->l_max;
  bool paired;
  if (N * (L + 1) <= 32) paired = false;
  else if (lanes_needed(N, L, true) <= 32) paired = true;
  else return set_error(SOAPB_ERR_UNSUPPORTED, "n_max * (l_max + 1) = %d radial functions exceed one warp", N * (L + 1));
  cudaStream_t st = (cudaStream_t)stream;
  ForceArgs a;
  a.pair_off = d_pair_off;
  a.pairs = (const float4*)d_pairs;
  a.coeff = d_coeff;
  a.dEdp = d_dEdp;
  a.centre_atom = d_centre_atom;
  a.tab_b = (const float*)((const char*)b->dev + b->off_tab_b);
  a.tab_bh = (const float*)((const char*)b->dev + b->off_tab_bh);
  a.forces = d_forces;
  a.counter = d_counter;
  a.n_centres = n_centres;
  a.N = N;
  a.S = b->n_species;
  a.nseg = b->n_seg;
  a.F = b->n_feat_ps;
  a.crossover = b->crossover ? 1 : 0;
  a.attach = attach ? 1 : 0;
  a.inv_h = (float)(1.0 / b->seg_width);
  int rc = check_cuda(cudaMemsetAsync(d_counter, 0, sizeof(int32_t), st), "reset work counter");
  if (rc) return rc;
  return dispatch_l<ForceDispatch>(L, a, paired, st);
}
