// Dense descriptor Jacobian d desc[c, f] / d x[a, d], written once per
// element (zeros included) in the DScribe layout (C, n_inc, 3, F).
//
// Reference: derivatives_analytical_ps (soap_generator.py:2270-2626) and its
// Triton kernels _ps_uv_kernel / _ps_jacobian_dense_kernel /
// _cc_jacobian_dense_kernel (:50-220).  Per edge e (centre c -> atom a,
// rvec = x_a - x_c, species s):
//   g[d, n, lm] = r_d Bhat_nl R_lm + B_nl dR_lm/dx_d
//   cc:  d c[s, n, lm] / d x_a,d       = sum_e g
//   ps:  d p[(j n), (j' n'), l] / dx_a,d = pref_l sum_e [ d_{j s} (r_d Bhat_nl U[j'n'l] + B_nl V_d[j'n'l])
//                                                      + d_{j' s} (r_d Bhat_n'l U[jnl] + B_n'l V_d[jnl]) ]
//   with U[k q l] = sum_m R_lm c[k q lm], V_d[k q l] = sum_m dR_lm/dx_d c[k q lm].
// Unlike the reference kernels this accumulates every edge of an atom, so
// periodic images are handled; attach=1 adds the centre-motion term
// (-sum over the centre's edges on the centre atom's row).
//
// The output is ~99% of the traffic (45 GB for 3000 atoms at F=420) and
// mostly zeros, so the kernel is an HBM write stream: one CTA per centre
// writes its contiguous (n_inc, 3, F) block front to back with 16-byte
// streaming stores, computing the few nonzero rows in between from per-edge
// data staged in shared memory.
#include "common.cuh"

namespace soapb {

struct JacArgs {
  const int64_t* pair_off;
  const float4* pairs;
  const float* coeff;
  const int* inc_row;
  const int* centre_atom;
  const float* tab_b;
  const float* tab_bh;
  const int* ftab;
  float* out;
  int* status;
  int64_t n_centres, n_inc;
  int N, S, nseg, F, mode, attach, cap, eb;
  float inv_h;
};

__device__ __forceinline__ void zero_fill(float* __restrict__ p, int64_t n) {
  // head to 16-byte alignment, float4 body, tail
  int64_t head = (int64_t)(((16 - ((uintptr_t)p & 15)) & 15) >> 2);
  if (head > n) head = n;
  for (int64_t i = threadIdx.x; i < head; i += blockDim.x) p[i] = 0.0f;
  float4* q = reinterpret_cast<float4*>(p + head);
  const int64_t n4 = (n - head) >> 2;
  const float4 z = make_float4(0.f, 0.f, 0.f, 0.f);
  for (int64_t i = threadIdx.x; i < n4; i += blockDim.x) __stcs(q + i, z);
  for (int64_t i = head + 4 * n4 + threadIdx.x; i < n; i += blockDim.x) p[i] = 0.0f;
}

template <int L>
struct JacShape {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int KC = K | 1;
  static constexpr int LP = L + 1;
  // floats per staged edge: rvec+species(4) | B, Bhat (2 NF) | R, dR (4K) | U, V (4 S N LP, ps only)
  __host__ __device__ static int edge_floats(int N, int S, int mode) {
    return 4 + 2 * N * LP + 4 * K + (mode == SOAPB_OUT_PS ? 4 * S * N * LP : 0);
  }
};

template <int L>
__global__ void __launch_bounds__(256) k_jacobian(JacArgs a) {
  using Sh = JacShape<L>;
  constexpr int K = Sh::K, KC = Sh::KC, LP = Sh::LP;
  const int N = a.N, S = a.S, NF = N * LP, SNL = S * N * LP;
  const int F = a.F;
  const int tid = threadIdx.x, nth = blockDim.x;
  extern __shared__ float smf[];
  float* cs = smf;                                          // S N KC
  unsigned long long* keys = (unsigned long long*)(smf + ((S * N * KC + 1) & ~1));
  float* ed = (float*)(keys + a.cap);                       // eb * edge_floats
  const int EF = Sh::edge_floats(N, S, a.mode);
  __shared__ float s_pref[kMaxL + 1];
  __shared__ int s_nent;
  if (tid <= L) s_pref[tid] = sqrtf(8.0f * (float)(kPi * kPi) / (2.0f * tid + 1.0f));
  const float pi_m15 = (float)(1.0 / (kPi * 1.7724538509055160273));
  // staged edge slot layout
  auto E_r = [&](int i) { return ed + (size_t)i * EF; };          // rx, ry, rz, species (as float)
  auto E_B = [&](int i) { return ed + (size_t)i * EF + 4; };      // NF
  auto E_Bh = [&](int i) { return ed + (size_t)i * EF + 4 + NF; };
  auto E_R = [&](int i) { return ed + (size_t)i * EF + 4 + 2 * NF; };          // K
  auto E_dR = [&](int i) { return ed + (size_t)i * EF + 4 + 2 * NF + K; };     // 3K
  auto E_U = [&](int i) { return ed + (size_t)i * EF + 4 + 2 * NF + 4 * K; };  // SNL
  auto E_V = [&](int i) { return ed + (size_t)i * EF + 4 + 2 * NF + 4 * K + SNL; };  // 3 SNL

  for (int64_t c = blockIdx.x; c < a.n_centres; c += gridDim.x) {
    const int64_t p0 = a.pair_off[c], p1 = a.pair_off[c + 1];
    const int P = (int)(p1 - p0);
    float* obase = a.out + (size_t)c * a.n_inc * 3 * F;
    const int catom = a.attach ? a.centre_atom[c] : -1;
    const int crow = (catom >= 0) ? a.inc_row[catom] : -1;
    for (int i = tid; i < S * N * K; i += nth) cs[(i / K) * KC + (i % K)] = a.coeff[(size_t)c * S * N * K + i];
    if (tid == 0) s_nent = 0;
    __syncthreads();
    for (int e = tid; e < P; e += nth) {
      const int atom = __float_as_int(a.pairs[p0 + e].w) & kAtomMask;
      if (a.attach && atom == catom) continue;  // centre and neighbour terms cancel
      const int row = a.inc_row[atom];
      if (row >= 0) {
        const int k = atomicAdd(&s_nent, 1);
        if (k < a.cap) keys[k] = ((unsigned long long)row << 32) | (unsigned)e;
      }
      if (crow >= 0) {
        const int k = atomicAdd(&s_nent, 1);
        if (k < a.cap) keys[k] = ((unsigned long long)crow << 32) | (unsigned)e;
      }
    }
    __syncthreads();
    int nent = s_nent;
    if (nent > a.cap) {
      if (tid == 0) atomicOr(a.status, 1);
      nent = a.cap;
    }
    int n2 = 1;
    while (n2 < nent) n2 <<= 1;
    for (int i = nent + tid; i < n2; i += nth) keys[i] = ~0ull;
    __syncthreads();
    for (int k = 2; k <= n2; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = tid; i < n2; i += nth) {
          const int ixj = i ^ j;
          if (ixj > i) {
            const unsigned long long x = keys[i], y = keys[ixj];
            const bool asc = (i & k) == 0;
            if (asc ? (x > y) : (x < y)) { keys[i] = y; keys[ixj] = x; }
          }
        }
        __syncthreads();
      }

    int64_t zero_from = 0;  // first row of this centre's block not yet written
    int last_row = -1;      // row written last (continued rows accumulate)
    for (int b0 = 0; b0 < nent; b0 += a.eb) {
      const int nb = min(a.eb, nent - b0);
      // stage per-edge data
      for (int i = tid; i < nb; i += nth) {
        const int e = (int)(keys[b0 + i] & 0xffffffffu);
        const float4 pr = a.pairs[p0 + e];
        float* er = E_r(i);
        er[0] = pr.x; er[1] = pr.y; er[2] = pr.z;
        er[3] = (float)((unsigned)__float_as_int(pr.w) >> kAtomBits);
        float* R = E_R(i);
        float* dR = E_dR(i);
        SolidHarmonics<L>::with_gradients(pr.x, pr.y, pr.z, [&](int idx, float v, float dx, float dy, float dz) {
          R[idx] = v; dR[idx] = dx; dR[K + idx] = dy; dR[2 * K + idx] = dz;
        });
      }
      __syncthreads();  // rvec of slot i is read by other threads below
      for (int t = tid; t < nb * NF; t += nth) {
        const int i = t / NF, fn = t % NF;
        const float* er = E_r(i);
        const float r = sqrtf(er[0] * er[0] + er[1] * er[1] + er[2] * er[2]);
        int seg;
        float tt;
        seg_coord(r, a.inv_h, a.nseg, seg, tt);
        float cf[kNCoef];
        load_coef(a.tab_b, seg, fn, NF, cf);
        E_B(i)[fn] = horner7(cf, tt);
        load_coef(a.tab_bh, seg, fn, NF, cf);
        E_Bh(i)[fn] = horner7(cf, tt);
      }
      __syncthreads();
      if (a.mode == SOAPB_OUT_PS) {
        for (int t = tid; t < nb * SNL; t += nth) {
          const int i = t / SNL, kq = (t % SNL) / LP, l = t % LP;
          const float* R = E_R(i);
          const float* dR = E_dR(i);
          const float* cr = cs + kq * KC + l * l;
          float u = 0.f, v0 = 0.f, v1 = 0.f, v2 = 0.f;
          for (int m = 0; m < 2 * l + 1; ++m) {
            const float cv = cr[m];
            u = fmaf(R[l * l + m], cv, u);
            v0 = fmaf(dR[l * l + m], cv, v0);
            v1 = fmaf(dR[K + l * l + m], cv, v1);
            v2 = fmaf(dR[2 * K + l * l + m], cv, v2);
          }
          E_U(i)[kq * LP + l] = u;
          float* V = E_V(i);
          V[kq * LP + l] = v0;
          V[SNL + kq * LP + l] = v1;
          V[2 * SNL + kq * LP + l] = v2;
        }
        __syncthreads();
      }
      // rows of this batch, in order
      int g0 = 0;
      while (g0 < nb) {
        const int row = (int)(keys[b0 + g0] >> 32);
        int g1 = g0 + 1;
        while (g1 < nb && (int)(keys[b0 + g1] >> 32) == row) ++g1;
        if ((int64_t)row > zero_from) zero_fill(obase + (size_t)zero_from * 3 * F, ((int64_t)row - zero_from) * 3 * F);
        const bool cont = (row == last_row);
        float* orow = obase + (size_t)row * 3 * F;
        for (int o = tid; o < 3 * F; o += nth) {
          const int d = o / F, f = o - d * F;
          float val = 0.0f;
          if (a.mode == SOAPB_OUT_PS) {
            const int code = __ldg(a.ftab + f);
            const int j = code & 15, jd = (code >> 4) & 15, n = (code >> 8) & 31, nd = (code >> 13) & 31,
                      l = (code >> 18) & 31;
            for (int i = g0; i < g1; ++i) {
              const float* er = E_r(i);
              const int s = (int)er[3];
              const float sign = (a.attach && row == crow) ? -1.0f : 1.0f;
              float tv = 0.0f;
              if (j == s)
                tv += er[d] * E_Bh(i)[l * N + n] * E_U(i)[(jd * N + nd) * LP + l] +
                      E_B(i)[l * N + n] * E_V(i)[d * SNL + (jd * N + nd) * LP + l];
              if (jd == s)
                tv += er[d] * E_Bh(i)[l * N + nd] * E_U(i)[(j * N + n) * LP + l] +
                      E_B(i)[l * N + nd] * E_V(i)[d * SNL + (j * N + n) * LP + l];
              val += sign * tv;
            }
            val *= s_pref[l];
          } else {
            const int sf = f / (N * K), rem = f - sf * N * K, n = rem / K, lo = rem - n * K;
            int src = lo;
            float scale = 1.0f;
            if (lo >= 1 && lo <= 3) src = (lo == 3) ? 1 : lo + 1;
            if (lo >= 4) scale = pi_m15;
            const int l = (int)sqrtf((float)src + 0.5f);
            for (int i = g0; i < g1; ++i) {
              const float* er = E_r(i);
              if ((int)er[3] != sf) continue;
              const float sign = (a.attach && row == crow) ? -1.0f : 1.0f;
              val += sign * (er[d] * E_Bh(i)[l * N + n] * E_R(i)[src] + E_B(i)[l * N + n] * E_dR(i)[d * K + src]);
            }
            val *= scale;
          }
          if (cont) orow[o] += val; else orow[o] = val;
        }
        zero_from = (int64_t)row + 1;
        last_row = row;
        g0 = g1;
        __syncthreads();
      }
    }
    if (zero_from < a.n_inc) zero_fill(obase + (size_t)zero_from * 3 * F, (a.n_inc - zero_from) * 3 * F);
    __syncthreads();
  }
}

template <int L>
struct JacDispatch {
  static int run(JacArgs a, cudaStream_t st) {
    const int EF = JacShape<L>::edge_floats(a.N, a.S, a.mode);
    int eb = (96 * 1024) / (4 * EF);
    eb = eb > 32 ? 32 : eb;
    if (eb < 1) return set_error(SOAPB_ERR_UNSUPPORTED, "jacobian edge data too large");
    a.eb = eb;
    const int cs_floats = (a.S * a.N * JacShape<L>::KC + 1) & ~1;
    const size_t smem = 4 * (size_t)cs_floats + 8 * (size_t)a.cap + 4 * (size_t)eb * EF;
    if (smem > 220 * 1024) return set_error(SOAPB_ERR_UNSUPPORTED, "jacobian shared memory %zu B too large", smem);
    auto kern = k_jacobian<L>;
    int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                        "jacobian smem attribute");
    if (rc) return rc;
    int dev = 0, nsm = 148, occ = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem);
    if (occ < 1) occ = 1;
    int64_t blocks = (int64_t)nsm * occ;
    if (blocks > a.n_centres) blocks = a.n_centres;
    kern<<<(unsigned)blocks, 256, smem, st>>>(a);
    return check_launch("k_jacobian");
  }
};

}  // namespace soapb

using namespace soapb;

extern "C" int soapb_jacobian(const soapb_basis* b, int64_t n_centres, const int64_t* d_pair_off, const void* d_pairs,
                              const float* d_coeff, const int32_t* d_inc_row, int64_t n_inc,
                              const int32_t* d_centre_atom, int32_t attach, int32_t max_pairs, int32_t out_mode,
                              float* d_out, int32_t* d_status, void* stream) {
  if (!b || !b->dev) return set_error(SOAPB_ERR_ARG, "basis not built");
  if (out_mode != SOAPB_OUT_PS && out_mode != SOAPB_OUT_CC) return set_error(SOAPB_ERR_ARG, "bad out_mode");
  if (n_centres <= 0 || n_inc <= 0) return SOAPB_OK;
  if (!d_pair_off || !d_coeff || !d_inc_row || !d_out || !d_status) return set_error(SOAPB_ERR_ARG, "null argument");
  if (attach && !d_centre_atom) return set_error(SOAPB_ERR_ARG, "attach needs centre atoms");
  if (max_pairs < 0) return set_error(SOAPB_ERR_ARG, "bad max_pairs");
  int need = (attach ? 2 : 1) * (max_pairs > 0 ? max_pairs : 1);
  int cap = 1;
  while (cap < need) cap <<= 1;
  if (cap > 8192) return set_error(SOAPB_ERR_UNSUPPORTED, "%d pairs per centre exceed the jacobian kernel's 8192", need);
  JacArgs a;
  a.pair_off = d_pair_off;
  a.pairs = (const float4*)d_pairs;
  a.coeff = d_coeff;
  a.inc_row = d_inc_row;
  a.centre_atom = d_centre_atom;
  a.tab_b = (const float*)((const char*)b->dev + b->off_tab_b);
  a.tab_bh = (const float*)((const char*)b->dev + b->off_tab_bh);
  a.ftab = (const int*)((const char*)b->dev + b->off_ftab);
  a.out = d_out;
  a.status = d_status;
  a.n_centres = n_centres;
  a.n_inc = n_inc;
  a.N = b->n_max;
  a.S = b->n_species;
  a.nseg = b->n_seg;
  a.F = out_mode == SOAPB_OUT_PS ? b->n_feat_ps : b->n_feat_cc;
  a.mode = out_mode;
  a.attach = attach ? 1 : 0;
  a.cap = cap;
  a.eb = 1;
  a.inv_h = (float)(1.0 / b->seg_width);
  return dispatch_l<JacDispatch>(b->l_max, a, (cudaStream_t)stream);
}
