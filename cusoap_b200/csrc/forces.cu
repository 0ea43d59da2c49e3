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
// Two kernels:
//  k_adjoint_g  one block per centre: dE/dp row and coefficient row staged in
//               shared memory (coalesced), G[a, lm] computed by thread-tasks
//               (a, l); the pair {a, b} -> feature map is a per-basis index
//               table (bit 30 marks a = b).  G goes to the workspace.
//  k_forces     one warp per centre (atomic work queue), ONE edge per lane:
//               the lane evaluates its edge's radial functions B_nl, Bhat_nl
//               from the function-major copy of the tables (lanes on nearby
//               segments share cache lines), its solid harmonics in registers,
//               and contracts l by l:
//                 xi_lm = sum_n G[s, n, lm] B_nl, zeta_lm = sum_n G[s, n, lm] Bhat_nl,
//                 dE/drvec = sum_lm (rvec zeta_lm R_lm + xi_lm grad R_lm),
//               with G broadcast from shared memory.  Neighbour forces are
//               per-lane float atomics; the centre-atom force is accumulated
//               in registers and reduced once per centre.
#include "common.cuh"

namespace soapb {

struct ForceArgs {
  const int64_t* pair_off;
  const float4* pairs;
  const float* coeff;
  const float* dEdp;
  const int* centre_atom;
  const float* tabt_b;   // [fn][seg][8]
  const float* tabt_bh;  // D = d(w B)/dr; Bhat = D / r
  const float* selfv;    // w0 B_nl(0) for r = 0 edges
  const int* widx;
  const int* ftab;       // l-major pair indices of every feature
  float* G;              // (n_centres, S N K) workspace
  float* forces;
  int* counter;
  int64_t n_centres;
  int N, S, nseg, F, attach, crossover;
  float inv_h;
};

constexpr int kGThreads = 256;

// G = dE/dc for one centre per block iteration.  STAGE_W: the dE/dp row is
// staged in shared memory (else read through the read-only cache, for
// feature counts whose row does not fit).
template <int L, bool STAGE_W>
__global__ void __launch_bounds__(kGThreads) k_adjoint_g(ForceArgs a) {
  constexpr int K = (L + 1) * (L + 1), KC = K | 1;
  extern __shared__ __align__(16) float sm[];
  const int N = a.N, SN = a.S * N, F = a.F;
  float* s_c = sm;                                   // SN x KC
  float* s_w = sm + ((SN * KC + 3) & ~3);            // F (STAGE_W)
  for (int64_t c = blockIdx.x; c < a.n_centres; c += gridDim.x) {
    const float* wrow = a.dEdp + (size_t)c * F;
    const float* crow = a.coeff + (size_t)c * SN * K;
    if (STAGE_W)
      for (int f = threadIdx.x; f < F; f += blockDim.x) s_w[f] = wrow[f];
    for (int i = threadIdx.x; i < SN * K; i += blockDim.x) s_c[(i / K) * KC + (i % K)] = crow[i];
    __syncthreads();
    float* grow = a.G + (size_t)c * SN * K;
    // tasks (a, l), heaviest l first so the last round is light
    for (int t = threadIdx.x; t < SN * (L + 1); t += blockDim.x) {
      const int l = L - t / SN, ai = t % SN;
      const int* wl = a.widx + (size_t)l * SN * SN;
      float g[2 * L + 1];
#pragma unroll
      for (int m = 0; m < 2 * L + 1; ++m) g[m] = 0.0f;
      for (int bi = 0; bi < SN; ++bi) {
        const int code = __ldg(wl + (size_t)bi * SN + ai);
        if (code < 0) continue;
        const int f = code & 0x3fffffff;
        const float w = (STAGE_W ? s_w[f] : __ldg(wrow + f)) * ((code & (1 << 30)) ? 2.0f : 1.0f);
        const float* cr = s_c + bi * KC + l * l;
#pragma unroll
        for (int m = 0; m < 2 * L + 1; ++m)
          if (m < 2 * l + 1) g[m] = fmaf(w, cr[m], g[m]);
      }
      const float pref = sqrtf(8.0f * (float)(kPi * kPi) / (2.0f * l + 1.0f));
#pragma unroll
      for (int m = 0; m < 2 * L + 1; ++m)
        if (m < 2 * l + 1) grow[ai * K + l * l + m] = pref * g[m];
    }
    __syncthreads();
  }
}

// G = dE/dc for one centre per block iteration, W dense in shared memory:
// the dE/dp row is scattered into W_l[a][b] (both triangles, 2x on a = b,
// times pref_l) through the l-major pair table, then G[a, lm] = sum_b
// W_l[a][b] c[b, lm] with lanes over a (W rows padded to SN + 1 floats:
// conflict-free) and c broadcast.  Used while (L+1) SN (SN+1) floats fit.
// One G task (a, l) with l known at compile time: G[a, l^2 .. l^2 + 2l] = sum_b W_l[a][b] c[b, lm].
template <int L, int l>
__device__ __forceinline__ void g_task(const float* Wr, const float* s_c, int SN, float* grow) {
  constexpr int K = (L + 1) * (L + 1), KC = K | 1, M = 2 * l + 1;
  float g[M];
#pragma unroll
  for (int m = 0; m < M; ++m) g[m] = 0.0f;
#pragma unroll 4
  for (int bi = 0; bi < SN; ++bi) {
    const float w = Wr[bi];
    const float* cr = s_c + bi * KC + l * l;
#pragma unroll
    for (int m = 0; m < M; ++m) g[m] = fmaf(w, cr[m], g[m]);
  }
#pragma unroll
  for (int m = 0; m < M; ++m) grow[l * l + m] = g[m];
}

template <int L, int l = 0>
__device__ __forceinline__ void g_task_l(int lr, const float* Wr, const float* s_c, int SN, float* grow) {
  if constexpr (l <= L) {
    if (lr == l) g_task<L, l>(Wr, s_c, SN, grow);
    else g_task_l<L, l + 1>(lr, Wr, s_c, SN, grow);
  }
}

template <int L>
__global__ void __launch_bounds__(kGThreads) k_adjoint_g_dense(ForceArgs a) {
  constexpr int K = (L + 1) * (L + 1), KC = K | 1;
  extern __shared__ __align__(16) float sm[];
  const int N = a.N, S = a.S, SN = S * N, WS = SN + 1, F = a.F;
  float* s_c = sm;                              // SN x KC
  float* s_W = sm + ((SN * KC + 3) & ~3);       // (L+1) x SN x WS
  const int wn = (L + 1) * SN * WS;
  for (int64_t c = blockIdx.x; c < a.n_centres; c += gridDim.x) {
    const float* wrow = a.dEdp + (size_t)c * F;
    const float* crow = a.coeff + (size_t)c * SN * K;
    for (int i = threadIdx.x; i < SN * K; i += blockDim.x) s_c[(i / K) * KC + (i % K)] = crow[i];
    // with crossover every (a, b, l) has a feature and is written below
    if (!a.crossover)
      for (int i = threadIdx.x; i < wn; i += blockDim.x) s_W[i] = 0.0f;
    __syncthreads();
    for (int f = threadIdx.x; f < F; f += blockDim.x) {
      const int code = __ldg(a.ftab + f);
      const int l = code >> 24, base = l * SN;
      const int ia = (code & 0xfff) - base, ib = ((code >> 12) & 0xfff) - base;
      const float w = wrow[f] * sqrtf(8.0f * (float)(kPi * kPi) / (2.0f * l + 1.0f));
      float* Wl = s_W + (size_t)l * SN * WS;
      if (ia == ib) {
        Wl[ia * WS + ia] = 2.0f * w;
      } else {
        Wl[ia * WS + ib] = w;
        Wl[ib * WS + ia] = w;
      }
    }
    __syncthreads();
    float* grow = a.G + (size_t)c * SN * K;
    for (int t = threadIdx.x; t < SN * (L + 1); t += blockDim.x) {
      const int l = L - t / SN, ai = t % SN;
      g_task_l<L>(l, s_W + ((size_t)l * SN + ai) * WS, s_c, SN, grow + ai * K);
    }
    __syncthreads();
  }
}

// G = dE/dc for the cc output (E = sum dEdp . cc-projection): the cc layout's
// l = 1 permutation and pi^-3/2 scale (lm >= 4) run backwards, elementwise.
__global__ void k_adjoint_g_cc(ForceArgs a, int K) {
  const int64_t SNK = (int64_t)a.S * a.N * K;
  const float pi_m15 = (float)(1.0 / (kPi * 1.7724538509055160273));
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < a.n_centres * SNK;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t c = i / SNK, r = i - c * SNK;
    const int lm = (int)(r % K);
    // output position of source lm: l = 1 is stored (z, x, y) = source (2, 3, 1)
    const int dst = (lm == 1) ? 3 : (lm == 2) ? 1 : (lm == 3) ? 2 : lm;
    a.G[i] = a.dEdp[c * SNK + (r - lm) + dst] * (lm >= 4 ? pi_m15 : 1.0f);
  }
}

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
struct ForceShape {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int KC = K | 1;
  __host__ __device__ static int warp_floats(int S, int N) { return (S * N * KC + 3) & ~3; }
};

template <int L>
__global__ void __launch_bounds__(128) k_forces(ForceArgs a) {
  using Sh = ForceShape<L>;
  constexpr int K = Sh::K, KC = Sh::KC;
  extern __shared__ __align__(16) float sm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int N = a.N, SN = a.S * N, nseg = a.nseg;
  float* G = sm + (size_t)wid * Sh::warp_floats(a.S, N);

  for (;;) {
    int c32 = 0;
    if (lane == 0) c32 = atomicAdd(a.counter, 1);
    const int64_t c = __shfl_sync(0xffffffffu, c32, 0);
    if (c >= a.n_centres) break;
    const int catom = a.attach ? a.centre_atom[c] : -1;
    const float* grow = a.G + (size_t)c * SN * K;
    for (int i = lane; i < SN * K; i += 32) G[(i / K) * KC + (i % K)] = grow[i];
    __syncwarp();

    float fcx = 0.f, fcy = 0.f, fcz = 0.f;
    const int64_t p0 = a.pair_off[c], p1 = a.pair_off[c + 1];
    for (int64_t e = p0 + lane; e < p1; e += 32) {
      const float4 pr = __ldg(a.pairs + e);
      const int wd = __float_as_int(pr.w);
      const int sp = (int)((unsigned)wd >> kAtomBits), atom = wd & kAtomMask;
      const float x = pr.x, y = pr.y, z = pr.z;
      int seg;
      float t;
      const float r = sqrtf(x * x + y * y + z * z);
      seg_coord(r, a.inv_h, nseg, seg, t);
      const bool self_edge = !(r > 0.0f);
      const float inv_r = self_edge ? 0.0f : 1.0f / r;
      const EdgeHarmonics<L> eh(x, y, z);
      const float* gs = G + sp * N * KC;
      float ex = 0.f, ey = 0.f, ez = 0.f;
#pragma unroll
      for (int l = 0; l <= L; ++l) {
        float xi[2 * L + 1], ze[2 * L + 1];
#pragma unroll
        for (int m = 0; m < 2 * l + 1; ++m) { xi[m] = 0.0f; ze[m] = 0.0f; }
        for (int n = 0; n < N; ++n) {
          const int fn = l * N + n;
          float cf[kNCoef], ch[kNCoef];
          load_coef(a.tabt_b, fn, seg, nseg, cf);   // function-major: row fn, column seg
          load_coef(a.tabt_bh, fn, seg, nseg, ch);
          const float b = self_edge ? __ldg(a.selfv + fn) : horner7(cf, t), h = horner7(ch, t) * inv_r;
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

static int resident_blocks(const void* kern, int threads, int smem, int* out) {
  int occ = 0;
  int rc = check_cuda(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, threads, smem), "occupancy");
  *out = occ < 1 ? 1 : occ;
  return rc;
}

template <int L>
struct ForceDispatch {
  static int run(const ForceArgs& a, int wpb_tuned, int out_mode, cudaStream_t st) {
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // G = dE/dc
    const int SN = a.S * a.N;
    const int64_t dense_bytes = 4 * (int64_t)(((SN * ((L + 1) * (L + 1) | 1) + 3) & ~3) + (L + 1) * SN * (SN + 1));
    if (out_mode == SOAPB_OUT_CC) {
      const int64_t n = a.n_centres * SN * (L + 1) * (L + 1);
      int64_t blocks = (n + 255) / 256;
      if (blocks > (int64_t)nsm * 32) blocks = (int64_t)nsm * 32;
      k_adjoint_g_cc<<<(unsigned)blocks, 256, 0, st>>>(a, (L + 1) * (L + 1));
      int rc = check_launch("k_adjoint_g_cc");
      if (rc) return rc;
    } else if (dense_bytes <= 100 * 1024) {
      auto kern = k_adjoint_g_dense<L>;
      const int smem = (int)dense_bytes;
      int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                          "adjoint smem attribute");
      if (rc) return rc;
      int occ = 1;
      if ((rc = resident_blocks((const void*)kern, kGThreads, smem, &occ))) return rc;
      int64_t blocks = (int64_t)nsm * occ;
      if (blocks > a.n_centres) blocks = a.n_centres;
      kern<<<(unsigned)blocks, kGThreads, smem, st>>>(a);
      if ((rc = check_launch("k_adjoint_g_dense"))) return rc;
    } else {
      const int cbytes = 4 * ((a.S * a.N * ((L + 1) * (L + 1) | 1) + 3) & ~3);
      const bool stage = cbytes + 4 * (int64_t)a.F <= 100 * 1024;
      auto kern = stage ? k_adjoint_g<L, true> : k_adjoint_g<L, false>;
      const int smem = cbytes + (stage ? 4 * a.F : 0);
      int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                          "adjoint smem attribute");
      if (rc) return rc;
      int occ = 1;
      if ((rc = resident_blocks((const void*)kern, kGThreads, smem, &occ))) return rc;
      int64_t blocks = (int64_t)nsm * occ;
      if (blocks > a.n_centres) blocks = a.n_centres;
      kern<<<(unsigned)blocks, kGThreads, smem, st>>>(a);
      if ((rc = check_launch("k_adjoint_g"))) return rc;
    }
    // edges
    auto kern = k_forces<L>;
    const int per_warp = 4 * ForceShape<L>::warp_floats(a.S, a.N);
    int wpb = (wpb_tuned == 1 || wpb_tuned == 2 || wpb_tuned == 4) ? wpb_tuned : 4;
    while (wpb > 1 && wpb * per_warp > 200 * 1024) wpb >>= 1;
    if (wpb * per_warp > 200 * 1024)
      return set_error(SOAPB_ERR_UNSUPPORTED, "forces: %d B of shared memory per warp is too large", per_warp);
    const int smem = wpb * per_warp;
    int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                        "forces smem attribute");
    if (rc) return rc;
    int occ = 1;
    if ((rc = resident_blocks((const void*)kern, 32 * wpb, smem, &occ))) return rc;
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

static int64_t forces_work_bytes(const soapb_basis* b, int64_t n_centres) {
  const int64_t K = (int64_t)(b->l_max + 1) * (b->l_max + 1);
  return align_up(4 * n_centres * b->n_species * b->n_max * K, 256);
}

extern "C" int soapb_forces_workspace(const soapb_basis* b, int64_t n_centres, int64_t* bytes) {
  if (!b || b->bytes <= 0) return set_error(SOAPB_ERR_ARG, "basis not planned");
  if (n_centres < 0 || !bytes) return set_error(SOAPB_ERR_ARG, "bad n_centres or null bytes");
  *bytes = forces_work_bytes(b, n_centres);
  return SOAPB_OK;
}

extern "C" int soapb_forces(const soapb_basis* b, int64_t n_centres, const int64_t* d_pair_off, const void* d_pairs,
                            const float* d_coeff, const float* d_dEdp, int32_t out_mode, const int32_t* d_centre_atom,
                            int32_t attach, float* d_forces, void* d_work, int64_t work_bytes, int32_t* d_counter,
                            void* stream) {
  if (!b || !b->dev) return set_error(SOAPB_ERR_ARG, "basis not built");
  if (out_mode != SOAPB_OUT_PS && out_mode != SOAPB_OUT_CC)
    return set_error(SOAPB_ERR_ARG, "forces: out_mode must be SOAPB_OUT_PS or SOAPB_OUT_CC");
  if (n_centres < 0 || n_centres >= (int64_t)1 << 31) return set_error(SOAPB_ERR_ARG, "bad n_centres");
  if (n_centres == 0) return SOAPB_OK;
  if (!d_pair_off || !d_coeff || !d_dEdp || !d_forces || !d_counter) return set_error(SOAPB_ERR_ARG, "null argument");
  if (attach && !d_centre_atom) return set_error(SOAPB_ERR_ARG, "attach needs centre atoms");
  if (!d_work || work_bytes < forces_work_bytes(b, n_centres))
    return set_error(SOAPB_ERR_ARG, "forces workspace too small (%lld < %lld)", (long long)work_bytes,
                     (long long)forces_work_bytes(b, n_centres));
  cudaStream_t st = (cudaStream_t)stream;
  ForceArgs a;
  a.pair_off = d_pair_off;
  a.pairs = (const float4*)d_pairs;
  a.coeff = d_coeff;
  a.dEdp = d_dEdp;
  a.centre_atom = d_centre_atom;
  a.tabt_b = (const float*)((const char*)b->dev + b->off_tabt_b);
  a.tabt_bh = (const float*)((const char*)b->dev + b->off_tabt_bh);
  a.selfv = (const float*)((const char*)b->dev + b->off_self);
  a.widx = (const int*)((const char*)b->dev + b->off_widx);
  a.ftab = (const int*)((const char*)b->dev + b->off_ftab);
  a.G = (float*)d_work;
  a.forces = d_forces;
  a.counter = d_counter;
  a.n_centres = n_centres;
  a.N = b->n_max;
  a.S = b->n_species;
  a.nseg = b->n_seg;
  a.F = b->n_feat_ps;
  a.attach = attach ? 1 : 0;
  a.crossover = b->crossover ? 1 : 0;
  a.inv_h = (float)(1.0 / b->seg_width);
  int rc = check_cuda(cudaMemsetAsync(d_counter, 0, sizeof(int32_t), st), "reset work counter");
  if (rc) return rc;
  return dispatch_l<ForceDispatch>(b->l_max, a, b->tune[2], (int)out_mode, st);
}
