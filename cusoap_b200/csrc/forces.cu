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
// Mapping: one warp per centre (atomic work queue), in two phases.
//  1. G in shared memory: lane = a, loop over l and b; the feature of the pair
//     {a, b} at l comes from a per-basis index table (bit 30 marks a = b), and
//     dE/dp is gathered through the read-only cache.
//  2. Edges in chunks of 32: lanes owning radial functions fn evaluate B_fn and
//     Bhat_fn of the chunk's edges into shared memory (coefficients stay in
//     registers while consecutive edges share a table segment, which the
//     (species, segment) pair order makes the common case); then each lane
//     contracts ONE edge: xi_lm = sum_n G[s, n, lm] B_nl, zeta_lm = sum_n
//     G[s, n, lm] Bhat_nl, dE/drvec = sum_lm (rvec zeta_lm R_lm + xi_lm grad R_lm),
//     with the solid harmonics of its own edge evaluated in registers, l by l.
//     Neighbour forces are per-lane float atomics; the centre-atom force is
//     accumulated in registers and reduced once per centre.
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
  const int* widx;
  float* forces;
  int* counter;
  int64_t n_centres;
  int N, S, nseg, F, attach;
  float inv_h;
};

template <int L>
struct ForceShape {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int KC = K | 1;
  static constexpr int RS = 33;  // staging row stride (floats): conflict-free lane and function strides
  // per warp: G (S N KC) | union{ coefficients (S N KC), B and Bhat rows (2 N (L+1) RS) } | t, seg (64)
  __host__ __device__ static int g_floats(int S, int N) { return (S * N * KC + 3) & ~3; }
  __host__ __device__ static int u_floats(int S, int N) {
    const int c = S * N * KC, st = 2 * N * (L + 1) * RS;
    return ((c > st ? c : st) + 3) & ~3;
  }
  __host__ __device__ static int warp_floats(int S, int N) { return g_floats(S, N) + u_floats(S, N) + 64; }
};

// Q_l^m table and the powers (x + i y)^m of one vector, for per-(l, m) solid
// harmonics and gradients (same recurrences and normalisation as SolidHarmonics).
template <int L>
struct EdgeHarmonics {
  static constexpr int NQ = (L + 1) * (L + 2) / 2;
  float Q[NQ], C[L + 1], Sn[L + 1];
  __device__ __forceinline__ EdgeHarmonics(float x, float y, float z) {
    SolidHarmonics<L>::legendre(z, x * x + y * y + z * z, Q);
    C[0] = 1.0f;
    Sn[0] = 0.0f;
#pragma unroll
    for (int m = 1; m <= L; ++m) {
      C[m] = x * C[m - 1] - y * Sn[m - 1];
      Sn[m] = x * Sn[m - 1] + y * C[m - 1];
    }
  }
};

template <int L>
__global__ void __launch_bounds__(128) k_forces(ForceArgs a) {
  using Sh = ForceShape<L>;
  constexpr int K = Sh::K, KC = Sh::KC, RS = Sh::RS;
  extern __shared__ __align__(16) float sm[];
  __shared__ float s_pref[kMaxL + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int N = a.N, S = a.S, NF = N * (L + 1), SN = S * N, F = a.F;
  float* G = sm + (size_t)wid * Sh::warp_floats(S, N);
  float* U = G + Sh::g_floats(S, N);  // coefficients, then B / Bhat staging
  float* Bs = U;
  float* Hs = U + NF * RS;
  float* s_t = U + Sh::u_floats(S, N);
  int* s_seg = reinterpret_cast<int*>(s_t + 32);
  if (threadIdx.x <= L) s_pref[threadIdx.x] = sqrtf(8.0f * (float)(kPi * kPi) / (2.0f * threadIdx.x + 1.0f));
  __syncthreads();

  for (;;) {
    int c32 = 0;
    if (lane == 0) c32 = atomicAdd(a.counter, 1);
    const int64_t c = __shfl_sync(0xffffffffu, c32, 0);
    if (c >= a.n_centres) break;
    const int catom = a.attach ? a.centre_atom[c] : -1;
    const float* crow = a.coeff + (size_t)c * SN * K;
    for (int i = lane; i < SN * K; i += 32) U[(i / K) * KC + (i % K)] = crow[i];
    __syncwarp();

    // ---- G = dE/dc ----
    const float* wrow = a.dEdp + (size_t)c * F;
    for (int a0 = 0; a0 < SN; a0 += 32) {
      const int ai = a0 + lane;
      const bool act = ai < SN;
#pragma unroll
      for (int l = 0; l <= L; ++l) {
        float g[2 * L + 1];
#pragma unroll
        for (int m = 0; m < 2 * L + 1; ++m) g[m] = 0.0f;
        const int* wl = a.widx + (size_t)l * SN * SN;
        for (int bi = 0; bi < SN; ++bi) {
          const int code = act ? __ldg(wl + (size_t)bi * SN + ai) : -1;
          if (code >= 0) {
            float w = __ldg(wrow + (code & 0x3fffffff));
            if (code & (1 << 30)) w *= 2.0f;
            const float* cr = U + bi * KC + l * l;
#pragma unroll
            for (int m = 0; m < 2 * l + 1; ++m) g[m] = fmaf(w, cr[m], g[m]);
          }
        }
        if (act) {
#pragma unroll
          for (int m = 0; m < 2 * l + 1; ++m) G[ai * KC + l * l + m] = s_pref[l] * g[m];
        }
      }
    }
    __syncwarp();

    // ---- edges ----
    float fcx = 0.f, fcy = 0.f, fcz = 0.f;
    const int64_t p0 = a.pair_off[c], p1 = a.pair_off[c + 1];
    for (int64_t base = p0; base < p1; base += 32) {
      const int nt = (int)min((int64_t)32, p1 - base);
      float4 pr = make_float4(0.f, 0.f, 0.f, 0.f);
      if (lane < nt) {
        pr = __ldg(a.pairs + base + lane);
        const float r = sqrtf(pr.x * pr.x + pr.y * pr.y + pr.z * pr.z);
        int seg;
        float t;
        seg_coord(r, a.inv_h, a.nseg, seg, t);
        s_t[lane] = t;
        s_seg[lane] = seg;
      }
      __syncwarp();
      // radial functions of the chunk: lane owns fn, lane + 32, ...
      for (int fn = lane; fn < NF; fn += 32) {
        float cf[kNCoef], ch[kNCoef];
        int cur = -1;
        for (int q = 0; q < nt; ++q) {
          const int sq = s_seg[q];
          if (sq != cur) {
            load_coef(a.tab_b, sq, fn, NF, cf);
            load_coef(a.tab_bh, sq, fn, NF, ch);
            cur = sq;
          }
          const float tq = s_t[q];
          Bs[fn * RS + q] = horner7(cf, tq);
          Hs[fn * RS + q] = horner7(ch, tq);
        }
      }
      __syncwarp();
      if (lane < nt) {
        const int wd = __float_as_int(pr.w);
        const int sp = (int)((unsigned)wd >> kAtomBits), atom = wd & kAtomMask;
        const float x = pr.x, y = pr.y, z = pr.z;
        const EdgeHarmonics<L> eh(x, y, z);
        const float* gs = G + sp * N * KC;
        float ex = 0.f, ey = 0.f, ez = 0.f;
#pragma unroll
        for (int l = 0; l <= L; ++l) {
          float xi[2 * L + 1], ze[2 * L + 1];
#pragma unroll
          for (int m = 0; m < 2 * l + 1; ++m) { xi[m] = 0.0f; ze[m] = 0.0f; }
          for (int n = 0; n < N; ++n) {
            const float b = Bs[(l * N + n) * RS + lane], h = Hs[(l * N + n) * RS + lane];
            const float* gr = gs + n * KC + l * l;
#pragma unroll
            for (int m = 0; m < 2 * l + 1; ++m) {
              const float gv = gr[m];
              xi[m] = fmaf(gv, b, xi[m]);
              ze[m] = fmaf(gv, h, ze[m]);
            }
          }
          // solid harmonics R_l^m and gradients (index l + m within the l block)
#pragma unroll
          for (int m = 0; m <= l; ++m) {
            const float nrm = c_shnorm[l * (kMaxL + 1) + m];
            const float q = eh.Q[tri(l, m)];
            const float qp = (l >= 1 && m + 1 <= l - 1) ? eh.Q[tri(l - 1, m + 1)] : 0.0f;
            const float qz = (l >= 1 && m <= l - 1) ? (float)(l + m) * eh.Q[tri(l - 1, m)] : 0.0f;
            if (m == 0) {
              const float R = nrm * q, dx = nrm * (-x * qp), dy = nrm * (-y * qp), dz = nrm * qz;
              const float zr = ze[l] * R;
              ex += x * zr + xi[l] * dx;
              ey += y * zr + xi[l] * dy;
              ez += z * zr + xi[l] * dz;
            } else {
              const float fm = (float)m;
              const float Cm = eh.C[m], Sm = eh.Sn[m], Cp = eh.C[m - 1], Sp = eh.Sn[m - 1];
              {  // +m
                const float R = nrm * q * Cm;
                const float dx = nrm * (-x * qp * Cm + q * fm * Cp), dy = nrm * (-y * qp * Cm - q * fm * Sp);
                const float dz = nrm * qz * Cm;
                const float zr = ze[l + m] * R;
                ex += x * zr + xi[l + m] * dx;
                ey += y * zr + xi[l + m] * dy;
                ez += z * zr + xi[l + m] * dz;
              }
              {  // -m
                const float R = nrm * q * Sm;
                const float dx = nrm * (-x * qp * Sm + q * fm * Sp), dy = nrm * (-y * qp * Sm + q * fm * Cp);
                const float dz = nrm * qz * Sm;
                const float zr = ze[l - m] * R;
                ex += x * zr + xi[l - m] * dx;
                ey += y * zr + xi[l - m] * dy;
                ez += z * zr + xi[l - m] * dz;
              }
            }
          }
        }
        if (!(a.attach && atom == catom)) {
          atomicAdd(&a.forces[3 * (size_t)atom + 0], -ex);
          atomicAdd(&a.forces[3 * (size_t)atom + 1], -ey);
          atomicAdd(&a.forces[3 * (size_t)atom + 2], -ez);
          fcx += ex;
          fcy += ey;
          fcz += ez;
        }
      }
      __syncwarp();
    }
    if (catom >= 0) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) {
        fcx += __shfl_xor_sync(0xffffffffu, fcx, o);
        fcy += __shfl_xor_sync(0xffffffffu, fcy, o);
        fcz += __shfl_xor_sync(0xffffffffu, fcz, o);
      }
      if (lane == 0) {
        atomicAdd(&a.forces[3 * (size_t)catom + 0], fcx);
        atomicAdd(&a.forces[3 * (size_t)catom + 1], fcy);
        atomicAdd(&a.forces[3 * (size_t)catom + 2], fcz);
      }
    }
    __syncwarp();
  }
}

template <int L>
struct ForceDispatch {
  static int run(const ForceArgs& a, cudaStream_t st) {
    auto kern = k_forces<L>;
    const int per_warp = 4 * ForceShape<L>::warp_floats(a.S, a.N);
    int dev = 0, nsm = 148, smem_sm = 228 * 1024, smem_blk = 227 * 1024;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&smem_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev);
    cudaDeviceGetAttribute(&smem_blk, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // warps per block: the most resident warps per SM (1 KB reserved per block), larger blocks on ties
    int wpb = 0, best = 0;
    for (int w = 4; w >= 1; w >>= 1) {
      const int bytes = w * per_warp;
      if (bytes > smem_blk) continue;
      const int resident = w * (smem_sm / (bytes + 1024));
      if (resident > best) { best = resident; wpb = w; }
    }
    if (wpb == 0) return set_error(SOAPB_ERR_UNSUPPORTED, "forces shared memory %d B per warp too large", per_warp);
    const int smem = wpb * per_warp;
    int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                        "forces smem attribute");
    if (rc) return rc;
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 32 * wpb, smem);
    if (occ < 1) occ = 1;
    int64_t blocks = (int64_t)nsm * occ;
    const int64_t need = (a.n_centres + wpb - 1) / wpb;
    if (blocks > need) blocks = need;
    if (blocks < 1) blocks = 1;
    kern<<<(unsigned)blocks, 32 * wpb, smem, st>>>(a);
    return check_launch("k_forces");
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
  cudaStream_t st = (cudaStream_t)stream;
  ForceArgs a;
  a.pair_off = d_pair_off;
  a.pairs = (const float4*)d_pairs;
  a.coeff = d_coeff;
  a.dEdp = d_dEdp;
  a.centre_atom = d_centre_atom;
  a.tab_b = (const float*)((const char*)b->dev + b->off_tab_b);
  a.tab_bh = (const float*)((const char*)b->dev + b->off_tab_bh);
  a.widx = (const int*)((const char*)b->dev + b->off_widx);
  a.forces = d_forces;
  a.counter = d_counter;
  a.n_centres = n_centres;
  a.N = N;
  a.S = b->n_species;
  a.nseg = b->n_seg;
  a.F = b->n_feat_ps;
  a.attach = attach ? 1 : 0;
  a.inv_h = (float)(1.0 / b->seg_width);
  int rc = check_cuda(cudaMemsetAsync(d_counter, 0, sizeof(int32_t), st), "reset work counter");
  if (rc) return rc;
  return dispatch_l<ForceDispatch>(L, a, st);
}
