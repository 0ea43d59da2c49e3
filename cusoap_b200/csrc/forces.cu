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
// Two stages:
//  k_adjoint_g_pipe  one block per centre iteration: the centre's dE/dp and
//               coefficient rows arrive in shared memory by double-buffered
//               TMA bulk copies, dE/dp is scattered into dense W_l and G[a, lm]
//               is computed by thread-tasks (two rows a, quad of 4 m slots).
//               G goes to the workspace.
//               (k_adjoint_g, with a per-basis pair -> feature index table and
//               no dense W, serves bases whose W does not fit.)
//  k_forces     one warp per centre (atomic work queue), ONE edge per lane:
//               the lane evaluates its edge's radial functions B_nl and
//               Bhat_nl = (dB_nl/dr) / r from one function-major table of
//               w B on half-width segments (value and derivative of the
//               segment polynomial in one Horner pass; lanes on nearby
//               segments share cache lines), its solid harmonics in registers,
//               and contracts l by l:
//                 xi_lm = sum_n G[s, n, lm] B_nl, zeta_lm = sum_n G[s, n, lm] Bhat_nl,
//                 dE/drvec = sum_lm (rvec zeta_lm R_lm + xi_lm grad R_lm),
//               the last sum accumulated as five per-edge scalars, with G
//               broadcast from shared memory.  Neighbour forces are
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
  const float* tabf;     // [fn][nsegf][8]: w B on half-width segments; its derivative is D = d(w B)/dr
  const int* widx;
  const int* ftab;       // l-major pair indices of every feature
  float* G;              // (n_centres, S N K) workspace
  float* forces;
  int* counter;
  int* status;           // bit 0: a TMA row copy of the G stage timed out (G rows NaN)
  int64_t n_centres;
  int N, S, nsegf, F, attach, crossover;
  int fstride;   // function stride of tabf in half-width segments (force_tab_stride)
  float inv_hf;  // 1 / width of a force-table segment
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

// G = dE/dc, one centre per block iteration, W dense in shared memory.
//  - The centre's dE/dp row and coefficient row are brought into shared
//    memory by TMA bulk copies (cp.async.bulk, completion on an mbarrier),
//    double-buffered: the next centre's rows are in flight while this one
//    is computed.  BULK = false (rows not 16-byte aligned) loads them with
//    plain coalesced loads instead.
//  - The dE/dp row is scattered into W_l[a][b] (both triangles, 2x on a = b)
//    through per-block shared-memory indices built once from the l-major
//    pair table; W rows are padded to SN + 1 floats (conflict-free reads by
//    lanes over a).  Entries without a feature stay zero.
//  - The coefficient row is repacked with every l block on a float4
//    boundary, so G[a, lm] = pref_l sum_b W_l[a][b] c[b, lm] runs as equal
//    tasks (rows a and a + SN/2, quad of 4 m slots): each float4 broadcast
//    of c feeds 8 FMAs (a full-warp 128-bit shared read costs 4 wavefronts,
//    broadcast or not, so the rows share it).
//  - G goes through shared memory to coalesced row stores.
// Coefficient row layout of the G kernel: l block l starts at off(l), a multiple of 4.
template <int L>
struct GRow {
  static constexpr int K = (L + 1) * (L + 1);
  __host__ __device__ static constexpr int off(int l) { return l == 0 ? 0 : off(l - 1) + ((2 * l - 1 + 3) & ~3); }
  static constexpr int KP = off(L + 1);
};

// Shared-memory carve-up of k_adjoint_g_pipe in floats (each part a multiple of 4).
struct GLayout {
  int idx, w, craw, cp, W, G, total, fa, snka;
};

// Floats per W_l matrix (SN rows of SN + 1): padded to 16 mod 32, so the two
// half-warps of a G task group, on quads of neighbouring l, read W rows on
// different banks.
__host__ __device__ inline int g_wl(int SN) {
  const int w = SN * (SN + 1);
  return w + (48 - w % 32) % 32;
}

template <int L>
__host__ __device__ inline GLayout g_layout(int F, int SN, int nbuf) {
  constexpr int K = GRow<L>::K, KP = GRow<L>::KP, KG = K | 1;
  GLayout g;
  g.fa = (F + 3) & ~3;
  g.snka = (SN * K + 3) & ~3;
  g.idx = 0;
  g.w = g.idx + g.fa;
  g.craw = g.w + nbuf * g.fa;
  g.cp = g.craw + nbuf * g.snka;
  g.W = g.cp + SN * KP;
  g.G = g.W + (((L + 1) * g_wl(SN) + 3) & ~3);
  g.total = g.G + ((SN * KG + 3) & ~3);
  return g;
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// One TMA bulk copy global -> shared, completing `bytes` on the mbarrier
// (both addresses 16-byte aligned, bytes a multiple of 16).
__device__ __forceinline__ void bulk_g2s(void* s, const void* g, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
                   smem_u32(s)),
               "l"(g), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

// Waits for the phase of the given parity to complete; gives up after about
// one second (global timer) and returns false.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  uint64_t t0, t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    if (done) return true;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > 1000000000ull) return false;
  }
}

template <int L, bool BULK>
__global__ void __launch_bounds__(kGThreads) k_adjoint_g_pipe(ForceArgs a) {
  constexpr int K = GRow<L>::K, KP = GRow<L>::KP, KG = K | 1;
  extern __shared__ __align__(16) float sm[];
  __shared__ __align__(8) uint64_t s_bar[2];
  __shared__ float s_pref[L + 1];
  __shared__ int s_lmoff[K];
  __shared__ int s_quad[KP / 4];  // l | (first m) << 8 of every float4 quad of the padded row
  __shared__ int s_fail;
  const int tid = threadIdx.x, nth = blockDim.x;
  const int N = a.N, SN = a.S * N, WS = SN + 1, WL = g_wl(SN), F = a.F, SNK = SN * K;
  const GLayout ly = g_layout<L>(F, SN, BULK ? 2 : 1);
  int* s_idx = reinterpret_cast<int*>(sm + ly.idx);
  float* s_cp = sm + ly.cp;
  float* s_W = sm + ly.W;
  float* s_G = sm + ly.G;

  // once per block: zero W and the padded row, W indices of every feature
  for (int i = tid; i < ly.total - ly.cp; i += nth) s_cp[i] = 0.0f;  // cp, W and G parts
  for (int f = tid; f < F; f += nth) {
    const int code = __ldg(a.ftab + f);
    const int l = code >> 24, base = l * SN;
    const int ia = (code & 0xfff) - base, ib = ((code >> 12) & 0xfff) - base;
    s_idx[f] = (l * WL + ia * WS + ib) | ((l * WL + ib * WS + ia) << 16);
  }
  if (tid <= L) s_pref[tid] = sqrtf(8.0f * (float)(kPi * kPi) / (2.0f * tid + 1.0f));
  for (int lm = tid; lm < K; lm += nth) {
    int l = 0;
    while ((l + 1) * (l + 1) <= lm) ++l;
    s_lmoff[lm] = GRow<L>::off(l) + lm - l * l;
  }
  for (int q = tid; q < KP / 4; q += nth) {
    int l = 0;
    while (GRow<L>::off(l + 1) <= 4 * q) ++l;
    s_quad[q] = l | ((4 * q - GRow<L>::off(l)) << 8);
  }
  if (tid == 0) {
    s_fail = 0;
    if (BULK) {
      mbar_init(&s_bar[0], 1);
      mbar_init(&s_bar[1], 1);
      asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
    }
  }
  __syncthreads();

  const uint32_t bytes_w = 4u * (uint32_t)F, bytes_c = 4u * (uint32_t)SNK;
  auto issue = [&](int64_t c, int buf) {  // thread 0: both rows of centre c into buffer buf
    mbar_expect_tx(&s_bar[buf], bytes_w + bytes_c);
    bulk_g2s(sm + ly.w + buf * ly.fa, a.dEdp + c * F, bytes_w, &s_bar[buf]);
    bulk_g2s(sm + ly.craw + buf * ly.snka, a.coeff + c * SNK, bytes_c, &s_bar[buf]);
  };
  if (BULK && tid == 0 && (int64_t)blockIdx.x < a.n_centres) issue(blockIdx.x, 0);

  int it = 0;
  for (int64_t c = blockIdx.x; c < a.n_centres; c += gridDim.x, ++it) {
    const int buf = BULK ? (it & 1) : 0;
    const float* w_row = sm + ly.w + buf * ly.fa;
    const float* c_row = sm + ly.craw + buf * ly.snka;
    bool next = false;
    if (BULK) {
      next = c + gridDim.x < a.n_centres;
      if (tid == 0 && next) {
        asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // earlier reads of buf ^ 1 first
        issue(c + gridDim.x, buf ^ 1);
      }
      if (!mbar_wait(&s_bar[buf], (it >> 1) & 1)) s_fail = 1;
    } else {
      float* w_dst = sm + ly.w;
      float* c_dst = sm + ly.craw;
      for (int f = tid; f < F; f += nth) w_dst[f] = a.dEdp[c * F + f];
      for (int i = tid; i < SNK; i += nth) c_dst[i] = a.coeff[c * SNK + i];
    }
    __syncthreads();
    if (s_fail) {
      // A row copy did not complete within the wait: flag it for the host,
      // give this block's copies still in flight (the late one and the
      // prefetch) one more bounded wait so that none lands after the block
      // has exited, and make G of this block's centres NaN.
      if (tid == 0) {
        atomicOr(a.status, 1);
        if (BULK) {
          mbar_wait(&s_bar[buf], (it >> 1) & 1);
          if (next) mbar_wait(&s_bar[buf ^ 1], ((it + 1) >> 1) & 1);
        }
      }
      for (int64_t cc = c; cc < a.n_centres; cc += gridDim.x)
        for (int i = tid; i < SNK; i += nth) a.G[cc * SNK + i] = __int_as_float(0x7fc00000);
      return;
    }
#pragma unroll 4
    for (int f = tid; f < F; f += nth) {
      const int idx = s_idx[f];
      const int ab = idx & 0xffff, ba = idx >> 16;
      const float v = w_row[f] * (ab == ba ? 2.0f : 1.0f);
      s_W[ab] = v;
      s_W[ba] = v;
    }
#pragma unroll 4
    for (int i = tid; i < SNK; i += nth) {
      const int bi = i / K;
      s_cp[bi * KP + s_lmoff[i - bi * K]] = c_row[i];
    }
    __syncthreads();
    // tasks (row pair, quad): G[a, l^2 + m0 .. m0 + 3] = pref_l sum_b W_l[a][b] c[b, quad]
    // for the rows a = ap and ap + SNh; the quad is read as one float4 (lanes over ap share
    // it) and feeds both rows.  Padding slots and a missing second row are not stored.
    const int SNh = (SN + 1) >> 1;
    for (int t = tid; t < SNh * (KP / 4); t += nth) {
      const int qd = t / SNh, a0 = t - qd * SNh, a1 = a0 + SNh;
      const bool two = a1 < SN;
      const int info = s_quad[qd], l = info & 255, m0 = info >> 8;
      const float* W0 = s_W + l * WL + a0 * WS;
      const float* W1 = s_W + l * WL + (two ? a1 : a0) * WS;
      const float4* cq = reinterpret_cast<const float4*>(s_cp) + qd;
      float4 g = make_float4(0.0f, 0.0f, 0.0f, 0.0f), h = g;
#pragma unroll 8
      for (int bi = 0; bi < SN; ++bi) {
        const float w0 = W0[bi], w1 = W1[bi];
        const float4 v = cq[bi * (KP / 4)];
        g.x = fmaf(w0, v.x, g.x);
        g.y = fmaf(w0, v.y, g.y);
        g.z = fmaf(w0, v.z, g.z);
        g.w = fmaf(w0, v.w, g.w);
        h.x = fmaf(w1, v.x, h.x);
        h.y = fmaf(w1, v.y, h.y);
        h.z = fmaf(w1, v.z, h.z);
        h.w = fmaf(w1, v.w, h.w);
      }
      const float p = s_pref[l];
      const int M = 2 * l + 1;
      float* go = s_G + a0 * KG + l * l + m0;
      go[0] = p * g.x;
      if (m0 + 1 < M) go[1] = p * g.y;
      if (m0 + 2 < M) go[2] = p * g.z;
      if (m0 + 3 < M) go[3] = p * g.w;
      if (two) {
        float* g1 = s_G + a1 * KG + l * l + m0;
        g1[0] = p * h.x;
        if (m0 + 1 < M) g1[1] = p * h.y;
        if (m0 + 2 < M) g1[2] = p * h.z;
        if (m0 + 3 < M) g1[3] = p * h.w;
      }
    }
    __syncthreads();
    float* grow = a.G + c * SNK;
#pragma unroll 4
    for (int i = tid; i < SNK; i += nth) {
      const int bi = i / K;
      grow[i] = s_G[bi * KG + i - bi * K];
    }
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

// FAST: n_max 8 and the table stride kForceSegStride at compile time, so the radial loop
// unrolls fully and every G and table offset is an immediate; else both come from the arguments.
template <int L, bool FAST>
__global__ void __launch_bounds__(128) k_forces(ForceArgs a) {
  using Sh = ForceShape<L>;
  constexpr int K = Sh::K, KC = Sh::KC;
  extern __shared__ __align__(16) float sm[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int N = FAST ? 8 : a.N, SN = a.S * N, nsegf = a.nsegf;
  const int fstride = FAST ? kForceSegStride : a.fstride;
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
      seg_coord(r, a.inv_hf, nsegf, seg, t);
      const bool self_edge = !(r > 0.0f);
      const float dt_r = self_edge ? 0.0f : 2.0f * a.inv_hf / r;  // (dt/dr) / r: Bhat = D / r = dP/dt dt_r
      const EdgeHarmonics<L> eh(x, y, z);
      const float* gs = G + sp * N * KC;
      // sum_lm (rvec zeta_lm R_lm + xi_lm grad R_lm), grouped: with u = nrm xi, Phi_m = C_m or S_m,
      //   P1 = sum u Q_{l-1}^{m+1} Phi_m, Pz = sum u (l+m) Q_{l-1}^m Phi_m, Rz = sum zeta R_lm,
      //   Tx, Ty = sum m Q_l^m (d Phi_m / dx, dy) u:  dE/drvec = (x (Rz - P1) + Tx, y (Rz - P1) + Ty, z Rz + Pz)
      float P1 = 0.f, Pz = 0.f, Rz = 0.f, Tx = 0.f, Ty = 0.f;
#pragma unroll
      for (int l = 0; l <= L; ++l) {
        float xi[2 * L + 1], ze[2 * L + 1];
#pragma unroll
        for (int m = 0; m < 2 * l + 1; ++m) { xi[m] = 0.0f; ze[m] = 0.0f; }
        // function-major table: row fn = l N + n, column seg.  The next function's two
        // float4 loads are issued before this one is evaluated, so their latency overlaps
        // the Horner pass and the G contraction.
        float cf[kNCoef];
        load_coef(a.tabf, l * N, seg, fstride, cf);
#pragma unroll (FAST ? 8 : 2)
        for (int n = 0; n < N; ++n) {
          float nx[kNCoef];
          load_coef(a.tabf, l * N + min(n + 1, N - 1), seg, fstride, nx);
          float p, dp;
          horner7_d(cf, t, p, dp);
#pragma unroll
          for (int k = 0; k < kNCoef; ++k) cf[k] = nx[k];
          // xi sums G B, ze sums G dB/dt: the factor (dt/dr) / r of zeta is applied once, to Rz
          const float* gr = gs + n * KC + l * l;
#pragma unroll
          for (int m = 0; m < 2 * l + 1; ++m) {
            const float gv = gr[m];
            xi[m] = fmaf(gv, p, xi[m]);
            ze[m] = fmaf(gv, dp, ze[m]);
          }
        }
        // this l's terms of the grouped sums (xi / ze index l + m within the l block)
#pragma unroll
        for (int m = 0; m <= l; ++m) {
          const float nrm = c_shnorm[l * (kMaxL + 1) + m];
          const float q = eh.Q[tri(l, m)];
          const float qp = (l >= 1 && m + 1 <= l - 1) ? eh.Q[tri(l - 1, m + 1)] : 0.0f;
          const float qz = (l >= 1 && m <= l - 1) ? (float)(l + m) * eh.Q[tri(l - 1, m)] : 0.0f;
          if (m == 0) {
            const float u = nrm * xi[l];
            P1 = fmaf(u, qp, P1);
            Pz = fmaf(u, qz, Pz);
            Rz = fmaf(nrm * q, ze[l], Rz);
          } else {
            const float Cm = eh.C[m], Sm = eh.Sn[m], Cp = eh.C[m - 1], Sp = eh.Sn[m - 1];
            const float u = nrm * xi[l + m], v = nrm * xi[l - m];
            const float U = fmaf(u, Cm, v * Sm);
            P1 = fmaf(U, qp, P1);
            Pz = fmaf(U, qz, Pz);
            const float mq = (float)m * q;
            Tx = fmaf(mq, fmaf(u, Cp, v * Sp), Tx);
            Ty = fmaf(mq, fmaf(v, Cp, -u * Sp), Ty);
            Rz = fmaf(nrm * q, fmaf(ze[l + m], Cm, ze[l - m] * Sm), Rz);
          }
        }
      }
      // an r = 0 edge adds nothing: its l = 0 term has no gradient and B_nl(0) = 0 for l >= 1,
      // so its xi terms are dropped here (and Rz through dt_r = 0)
      const float keep = self_edge ? 0.0f : 1.0f;
      P1 *= keep;
      Pz *= keep;
      Tx *= keep;
      Ty *= keep;
      Rz *= dt_r;
      const float rr = Rz - P1;
      const float ex = fmaf(x, rr, Tx), ey = fmaf(y, rr, Ty), ez = fmaf(z, Rz, Pz);
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
    constexpr int K = (L + 1) * (L + 1);
    // the pipelined dense kernel: W indices must fit 16 bits, shared memory 200 KB
    const bool aligned = ((uintptr_t)a.dEdp % 16 == 0) && ((uintptr_t)a.coeff % 16 == 0) && a.F % 4 == 0 &&
                         (SN * K) % 4 == 0;
    const int64_t pipe_bulk = 4 * (int64_t)g_layout<L>(a.F, SN, 2).total;
    const int64_t pipe_plain = 4 * (int64_t)g_layout<L>(a.F, SN, 1).total;
    const bool pipe_ok = (int64_t)(L + 1) * g_wl(SN) < 65536 && pipe_plain <= 200 * 1024;
    if (out_mode == SOAPB_OUT_CC) {
      const int64_t n = a.n_centres * SN * (L + 1) * (L + 1);
      int64_t blocks = (n + 255) / 256;
      if (blocks > (int64_t)nsm * 32) blocks = (int64_t)nsm * 32;
      k_adjoint_g_cc<<<(unsigned)blocks, 256, 0, st>>>(a, (L + 1) * (L + 1));
      int rc = check_launch("k_adjoint_g_cc");
      if (rc) return rc;
    } else if (pipe_ok) {
      const bool bulk = aligned && pipe_bulk <= 200 * 1024;
      auto kern = bulk ? k_adjoint_g_pipe<L, true> : k_adjoint_g_pipe<L, false>;
      const int smem = (int)(bulk ? pipe_bulk : pipe_plain);
      int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                          "adjoint smem attribute");
      if (rc) return rc;
      int occ = 1;
      if ((rc = resident_blocks((const void*)kern, kGThreads, smem, &occ))) return rc;
      int64_t blocks = (int64_t)nsm * occ;
      if (blocks > a.n_centres) blocks = a.n_centres;
      kern<<<(unsigned)blocks, kGThreads, smem, st>>>(a);
      if ((rc = check_launch("k_adjoint_g_pipe"))) return rc;
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
    auto kern = (a.N == 8 && a.fstride == kForceSegStride) ? k_forces<L, true> : k_forces<L, false>;
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

// Workspace: G (n_centres, S N K) float, then one int32 status word.
static int64_t forces_g_bytes(const soapb_basis* b, int64_t n_centres) {
  const int64_t K = (int64_t)(b->l_max + 1) * (b->l_max + 1);
  return align_up(4 * n_centres * b->n_species * b->n_max * K, 256);
}

static int64_t forces_work_bytes(const soapb_basis* b, int64_t n_centres) {
  return forces_g_bytes(b, n_centres) + 256;
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
  a.tabf = (const float*)((const char*)b->dev + b->off_tabf);
  a.widx = (const int*)((const char*)b->dev + b->off_widx);
  a.ftab = (const int*)((const char*)b->dev + b->off_ftab);
  a.G = (float*)d_work;
  a.forces = d_forces;
  a.counter = d_counter;
  a.status = (int*)((char*)d_work + forces_g_bytes(b, n_centres));
  a.n_centres = n_centres;
  a.N = b->n_max;
  a.S = b->n_species;
  a.nsegf = 2 * b->n_seg;
  a.fstride = force_tab_stride(b->n_seg);
  a.F = b->n_feat_ps;
  a.attach = attach ? 1 : 0;
  a.crossover = b->crossover ? 1 : 0;
  a.inv_hf = (float)(2.0 / b->seg_width);
  int rc = check_cuda(cudaMemsetAsync(d_counter, 0, sizeof(int32_t), st), "reset work counter");
  if (rc) return rc;
  if ((rc = check_cuda(cudaMemsetAsync(a.status, 0, sizeof(int32_t), st), "reset forces status"))) return rc;
  return dispatch_l<ForceDispatch>(b->l_max, a, b->tune[2], (int)out_mode, st);
}

extern "C" int soapb_forces_status(const soapb_basis* b, int64_t n_centres, const void* d_work, int32_t* h_status,
                                   void* stream) {
  if (!b || b->bytes <= 0) return set_error(SOAPB_ERR_ARG, "basis not planned");
  if (n_centres < 0 || !d_work || !h_status) return set_error(SOAPB_ERR_ARG, "bad n_centres, workspace or status");
  if (n_centres == 0) {
    *h_status = 0;
    return SOAPB_OK;
  }
  cudaStream_t st = (cudaStream_t)stream;
  const void* p = (const char*)d_work + forces_g_bytes(b, n_centres);
  int rc = check_cuda(cudaMemcpyAsync(h_status, p, sizeof(int32_t), cudaMemcpyDeviceToHost, st), "forces status");
  if (rc) return rc;
  return check_cuda(cudaStreamSynchronize(st), "forces status sync");
}

namespace soapb {

// Diagnostic of the G stage's bounded wait: one thread arms an mbarrier with a
// transaction count that no copy will fill and waits on it as the G stage
// waits for its row copies.  The wait gives up after about one second and the
// thread writes 1 to *status (0 would mean the phase completed).  No copy is
// in flight, so nothing can land after the block exits.
__global__ void k_check_bounded_wait(int* status) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x != 0) return;
  mbar_init(&bar, 1);
  asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  mbar_expect_tx(&bar, 16);
  *status = mbar_wait(&bar, 0) ? 0 : 1;
}

}  // namespace soapb

extern "C" int soapb_check_bounded_wait(int32_t* d_status, void* stream) {
  if (!d_status) return set_error(SOAPB_ERR_ARG, "null status");
  k_check_bounded_wait<<<1, 32, 0, (cudaStream_t)stream>>>(d_status);
  return check_launch("k_check_bounded_wait");
}
