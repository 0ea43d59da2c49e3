// Fused per-centre SOAP descriptor: radial table x real solid harmonics ->
// c_nlm accumulated in registers -> power spectrum / cc / raw epilogue.
//
// Reference: _coefficients_gto (soap_generator.py:1294-1391), the self term
// (:765-850, here the kept r=0 edge of the centre's own atom, whose value is
// exactly B_n0(0) Y00), _power_spectrum (:1634-1689) with the DScribe
// feature order of _build_feature_slices (:1215-1245), and _projection_cc /
// _to_dscribe_cc (:1603-1632).  average 'inner' and 'outer' are centre-wise
// in the reference (coeffs_use = coeffs, :1651-1657), i.e. identical to 'off'.
//
// Mapping: one warp per centre, centres taken from an atomic work queue.
// Each lane owns one radial function (n, l) ("single": N (L+1) <= 32) or two
// with l0 + l1 = L ("paired"), and keeps their 2l+1 m-accumulators in
// registers.  The centre's pairs arrive sorted by (species, radial segment):
// the species switch flushes the accumulators into the warp's coefficient
// buffer, the segment switch (warp-uniform) reloads the lane's table
// coefficients, so the per-pair work is 7 FMAs of Horner per function plus
// one FMA per (n, l, m).  Solid harmonics are computed 32 pairs at a time,
// one pair per lane, into shared memory.
#include "common.cuh"

namespace soapb {

struct DescArgs {
  const int64_t* pair_off;
  const float4* pairs;
  int64_t n_centres;
  const float* tab_b;
  const int* ftab;
  float* out;
  float* coeff_out;  // optional raw c[s][n][lm] rows (S N K floats per centre)
  int* counter;
  int N, S, nseg, F, mode;
  float inv_h;
};

template <int L>
struct DescShape {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int YS = K | 1;  // odd strides: conflict-free shared-memory rows
  static constexpr int KC = K | 1;
  __host__ __device__ static int warp_floats(int S, int N) { return 32 * YS + 96 + S * N * KC; }
};

template <int L, bool PAIRED>
__global__ void __launch_bounds__(128) k_descriptor(DescArgs a) {
  using Sh = DescShape<L>;
  constexpr int K = Sh::K, YS = Sh::YS, KC = Sh::KC;
  constexpr int MT = PAIRED ? 2 * L + 2 : 2 * L + 1;
  extern __shared__ float sm[];
  __shared__ float s_pref[kMaxL + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int N = a.N, S = a.S, NF = N * (L + 1);
  const int cbn = S * N * KC;
  float* Y = sm + (size_t)wid * Sh::warp_floats(S, N);
  float* tt = Y + 32 * YS;
  int* sg = (int*)(tt + 32);
  int* spp = sg + 32;
  float* cbuf = (float*)(spp + 32);
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
    for (int i = lane; i < cbn; i += 32) cbuf[i] = 0.0f;
    float acc[MT];
#pragma unroll
    for (int k = 0; k < MT; ++k) acc[k] = 0.0f;
    float cf0[kNCoef], cf1[kNCoef];
#pragma unroll
    for (int k = 0; k < kNCoef; ++k) { cf0[k] = 0.0f; cf1[k] = 0.0f; }
    int cur_sp = -1, cur_seg = -1;
    const int64_t p0 = a.pair_off[c], p1 = a.pair_off[c + 1];
    __syncwarp();

    auto flush = [&](int sp) {
#pragma unroll
      for (int k = 0; k < MT; ++k) {
        if (k < mtot) {
          const bool first = k < m0;
          const int n = first ? lf.n0 : lf.n1, l = first ? lf.l0 : lf.l1, m = first ? k : k - m0;
          cbuf[(sp * N + n) * KC + l * l + m] += acc[k];
        }
        acc[k] = 0.0f;
      }
    };

    for (int64_t base = p0; base < p1; base += 32) {
      const int nt = (int)min((int64_t)32, p1 - base);
      if (lane < nt) {
        const float4 pr = __ldg(a.pairs + base + lane);
        const int w = __float_as_int(pr.w);
        const float r = sqrtf(pr.x * pr.x + pr.y * pr.y + pr.z * pr.z);
        int seg;
        float t;
        seg_coord(r, a.inv_h, a.nseg, seg, t);
        tt[lane] = t;
        sg[lane] = seg;
        spp[lane] = (int)((unsigned)w >> kAtomBits);
        float* yrow = Y + lane * YS;
        SolidHarmonics<L>::values(pr.x, pr.y, pr.z, [&](int idx, float v) { yrow[idx] = v; });
      }
      __syncwarp();
      for (int q = 0; q < nt; ++q) {
        const int sp = spp[q];
        if (sp != cur_sp) {
          if (cur_sp >= 0) flush(cur_sp);
          cur_sp = sp;
        }
        const int seg = sg[q];
        if (seg != cur_seg) {
          if (lf.l0 >= 0) load_coef(a.tab_b, seg, fn0, NF, cf0);
          if (PAIRED && lf.l1 >= 0) load_coef(a.tab_b, seg, fn1, NF, cf1);
          cur_seg = seg;
        }
        const float t = tt[q];
        const float B0 = horner7(cf0, t);
        const float B1 = PAIRED ? horner7(cf1, t) : 0.0f;
        const float* yr = Y + q * YS;
#pragma unroll
        for (int k = 0; k < MT; ++k) {
          if (k < mtot) {
            const bool first = k < m0;
            acc[k] = fmaf(first ? B0 : B1, yr[k + (first ? yoff0 : yoff1)], acc[k]);
          }
        }
      }
      __syncwarp();
    }
    if (cur_sp >= 0) flush(cur_sp);
    __syncwarp();

    if (a.coeff_out) {
      float* crow = a.coeff_out + (size_t)c * S * N * K;
      for (int f = lane; f < S * N * K; f += 32) {
        const int sn = f / K;
        crow[f] = cbuf[sn * KC + (f - sn * K)];
      }
    }
    float* orow = a.out + (size_t)c * a.F;
    if (a.mode == SOAPB_OUT_PS) {
      for (int f = lane; f < a.F; f += 32) {
        const int code = __ldg(a.ftab + f);
        const int j = code & 15, jd = (code >> 4) & 15, n = (code >> 8) & 31, nd = (code >> 13) & 31,
                  l = (code >> 18) & 31;
        const float* x = cbuf + (j * N + n) * KC + l * l;
        const float* y = cbuf + (jd * N + nd) * KC + l * l;
        float s = 0.0f;
#pragma unroll
        for (int m = 0; m < 2 * L + 1; ++m)
          if (m < 2 * l + 1) s = fmaf(x[m], y[m], s);
        orow[f] = s * s_pref[l];
      }
    } else {
      const bool cc = a.mode == SOAPB_OUT_CC;
      const float pi_m15 = (float)(1.0 / (kPi * 1.7724538509055160273));  // pi^-3/2
      for (int f = lane; f < a.F; f += 32) {
        const int sn = f / K, lm = f - sn * K;
        int src = lm;
        float scale = 1.0f;
        if (cc) {
          // l = 1 stored (z, x, y) = source lm (2, 3, 1); lm >= 4 scaled by pi^-3/2
          if (lm >= 1 && lm <= 3) src = (lm == 3) ? 1 : lm + 1;
          if (lm >= 4) scale = pi_m15;
        }
        orow[f] = cbuf[sn * KC + src] * scale;
      }
    }
    __syncwarp();
  }
}

template <int L, bool PAIRED>
static int launch_descriptor(const DescArgs& a, cudaStream_t st) {
  const int per_warp = 4 * DescShape<L>::warp_floats(a.S, a.N);
  int wpb = (200 * 1024) / per_warp;
  wpb = wpb > 4 ? 4 : wpb;
  if (wpb < 1) return set_error(SOAPB_ERR_UNSUPPORTED, "descriptor shared memory %d B per warp too large", per_warp);
  const int smem = wpb * per_warp;
  auto kern = k_descriptor<L, PAIRED>;
  int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                      "descriptor smem attribute");
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
  return check_launch("k_descriptor");
}

template <int L>
struct DescDispatch {
  static int run(const DescArgs& a, bool paired, cudaStream_t st) {
    return paired ? launch_descriptor<L, true>(a, st) : launch_descriptor<L, false>(a, st);
  }
};

}  // namespace soapb

using namespace soapb;

extern "C" int soapb_descriptor(const soapb_basis* b, int64_t n_centres, const int64_t* d_pair_off,
                                const void* d_pairs, int32_t out_mode, float* d_out, float* d_coeff,
                                int32_t* d_counter, void* stream) {
  if (!b || !b->dev) return set_error(SOAPB_ERR_ARG, "basis not built");
  if (n_centres < 0 || n_centres >= (int64_t)1 << 31) return set_error(SOAPB_ERR_ARG, "bad n_centres");
  if (out_mode != SOAPB_OUT_PS && out_mode != SOAPB_OUT_CC && out_mode != SOAPB_OUT_RAW)
    return set_error(SOAPB_ERR_ARG, "bad out_mode");
  if (n_centres == 0) return SOAPB_OK;
  if (!d_pair_off || !d_out || !d_counter) return set_error(SOAPB_ERR_ARG, "null argument");
  const int N = b->n_max, L = b->l_max;
  bool paired;
  if (N * (L + 1) <= 32) paired = false;
  else if (lanes_needed(N, L, true) <= 32) paired = true;
  else return set_error(SOAPB_ERR_UNSUPPORTED, "n_max * (l_max + 1) = %d radial functions exceed one warp", N * (L + 1));
  cudaStream_t st = (cudaStream_t)stream;
  DescArgs a;
  a.pair_off = d_pair_off;
  a.pairs = (const float4*)d_pairs;
  a.n_centres = n_centres;
  a.tab_b = (const float*)((const char*)b->dev + b->off_tab_b);
  a.ftab = (const int*)((const char*)b->dev + b->off_ftab);
  a.out = d_out;
  a.coeff_out = d_coeff;
  a.counter = d_counter;
  a.N = N;
  a.S = b->n_species;
  a.nseg = b->n_seg;
  a.F = out_mode == SOAPB_OUT_PS ? b->n_feat_ps : b->n_feat_cc;
  a.mode = out_mode;
  a.inv_h = (float)(1.0 / b->seg_width);
  int rc = check_cuda(cudaMemsetAsync(d_counter, 0, sizeof(int32_t), st), "reset work counter");
  if (rc) return rc;
  return dispatch_l<DescDispatch>(L, a, paired, st);
}
