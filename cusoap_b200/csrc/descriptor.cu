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
// Lanes are grouped by l: floor(32 / (L+1)) lanes per l, each owning GN radial
// functions (n, l) of the same l, so one shared-memory read of R_lm feeds GN
// accumulators and the m loop is the same for all of them.  The centre's
// pairs arrive sorted by (species, radial segment): the species switch
// flushes the accumulators into the warp's coefficient buffer, the segment
// switch (warp-uniform) reloads the lane's table coefficients, so the
// per-pair work is 7 FMAs of Horner per function plus one FMA per (n, l, m).
// For l_max <= 4, where one stream leaves lanes idle, each half-warp walks its
// own stream of the pairs (k_descriptor_2s).  Solid harmonics are computed 16
// pairs at a time (32 with two pair streams), one pair per lane, into shared
// memory.  The power-spectrum epilogue walks the DScribe blocks (species pair,
// l) in one non-unrolled l loop; each lane writes consecutive features, so
// the row is stored coalesced.
#include "common.cuh"

namespace soapb {

struct DescArgs {
  const int64_t* pair_off;
  const float4* pairs;
  int64_t n_centres;
  const float* tab_b;
  const float* selfv;  // w0 B_nl(0): value of r = 0 edges (the centre's own Gaussian)
  float* out;
  float* coeff_out;  // optional raw c[s][n][lm] rows (S N K floats per centre)
  int* counter;
  int N, S, nseg, F, mode, crossover;
  float inv_h;
  float self_ratio;  // w0 / w(0): an r = 0 edge's table value times this is its self value
};

// Position of harmonic block l in a pair's Y row: l^2 plus a padding that
// starts every block on a different shared-memory bank (the lane groups of the
// l blocks read the same slot m of their blocks at once: no conflicts).  Plain
// l^2 puts l = 6 on the bank of l = 2 (36 = 4 mod 32), l = 8 on that of l = 0
// and l = 12 on that of l = 4; one float of padding from l = 6, another from
// l = 8 and two more from l = 12 separate them (checked below).
__host__ __device__ constexpr int ybase(int l) { return l * l + (l >= 6) + (l >= 8) + 2 * (l >= 12); }
// Y row position of harmonic index idx = l^2 + l + m (idx >= 36: l >= 6, >= 64: l >= 8, >= 144: l >= 12).
__host__ __device__ constexpr int ypos(int idx) { return idx + (idx >= 36) + (idx >= 64) + 2 * (idx >= 144); }

constexpr bool ybase_banks_distinct() {
  for (int l = 0; l <= kMaxL; ++l) {
    if (l > 0 && ybase(l) < ybase(l - 1) + 2 * l - 1) return false;  // blocks overlap
    for (int k = 0; k < l; ++k)
      if (ybase(k) % 32 == ybase(l) % 32) return false;
    for (int m = 0; m <= 2 * l; ++m)
      if (ypos(l * l + m) != ybase(l) + m) return false;
  }
  return true;
}
static_assert(ybase_banks_distinct(), "Y row blocks must start on distinct banks");

// Extra offset of the Y rows of pairs 16..31 (two pair streams per warp): the
// smallest shift that keeps the l blocks of row q and row q + 16 -- read by
// the two half-warps at once -- on distinct banks.
__host__ __device__ constexpr int half_offset(int L, int YS) {
  for (int h = 0; h < 32; ++h) {
    bool ok = true;
    for (int l = 0; l <= L; ++l)
      for (int k = 0; k <= L; ++k)
        if ((16 * YS + h + ybase(l)) % 32 == ybase(k) % 32) ok = false;
    if (ok) return h;
  }
  return 0;
}

template <int L>
struct DescShape {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int YS = (ybase(L) + 2 * L + 1) | 1;  // odd strides: conflict-free row writes
  static constexpr int HOFF = half_offset(L, YS);
  static constexpr int KC = K | 1;
  __host__ __device__ static int warp_floats(int S, int N) { return 32 * YS + HOFF + 96 + S * N * KC; }
  // one pair stream: 16 staged pairs per batch
  __host__ __device__ static int warp_floats16(int S, int N) { return 16 * YS + 48 + S * N * KC; }
};

// Functions per lane for (N, L): floor(32 / (L+1)) lanes share each l.
inline int desc_group(int N, int L) {
  const int lpl = 32 / (L + 1);
  int gn = (N + lpl - 1) / lpl;
  if (gn == 5) gn = 6;
  return gn;
}

// Two pair streams per warp (each half-warp walks 16 of every 32 pairs, lanes
// grouped by l inside the half, at most 3 functions per lane), for l_max <= 4
// when one stream leaves more than a quarter of the lanes without a function
// (n_max 8, l_max 4: 20 of 32 lanes busy with one stream, 30 with two).
inline bool desc_two_streams(int N, int L) {
  if (L > 4) return false;
  const int lpl = 16 / (L + 1);
  if ((N + lpl - 1) / lpl > 3) return false;
  const int gn = desc_group(N, L);
  return (L + 1) * ((N + gn - 1) / gn) <= 24;
}

constexpr int kMaxBlocks = kMaxS * (kMaxS + 1) / 2;
constexpr int kMaxLNLanes = 6;  // largest l_max of the radial-index-lane kernel (registers)
constexpr int kMaxTri = kMaxN * (kMaxN + 1) / 2;

// Per-block tables of the power-spectrum epilogue: the prefactor
// sqrt(8 pi^2 / (2l+1)) per l, the DScribe species blocks (j | jd << 8, first
// feature) and the (n, n') pairs of the upper-triangle index.
template <int L>
__device__ __forceinline__ void desc_tables(const DescArgs& a, float* s_pref, int* s_blk, unsigned char* s_tri) {
  const int N = a.N, S = a.S;
  if (threadIdx.x <= L) s_pref[threadIdx.x] = sqrtf(8.0f * (float)(kPi * kPi) / (2.0f * threadIdx.x + 1.0f));
  if (threadIdx.x == 0) {
    int nb = 0, f = 0;
    for (int j = 0; j < S; ++j)
      for (int jd = j; jd < (a.crossover ? S : j + 1); ++jd) {
        s_blk[2 * nb] = j | (jd << 8);
        s_blk[2 * nb + 1] = f;
        f += (j == jd ? N * (N + 1) / 2 : N * N) * (L + 1);
        ++nb;
      }
    int p = 0;
    for (int n = 0; n < N; ++n)
      for (int nd = n; nd < N; ++nd, ++p) {
        s_tri[2 * p] = (unsigned char)n;
        s_tri[2 * p + 1] = (unsigned char)nd;
      }
  }
}

// One centre's outputs from its coefficients cbuf[(s N + n) KC + lm]
// (KC = K | 1), written by the whole warp: the raw coefficient row when
// requested, then the power spectrum in DScribe order (each lane writes
// consecutive features of a block, so rows are stored coalesced), or the
// cc / raw projection.
template <int L>
__device__ __forceinline__ void desc_epilogue(const DescArgs& a, int64_t c, const float* cbuf, int lane,
                                              const float* s_pref, const int* s_blk, const unsigned char* s_tri) {
  constexpr int K = (L + 1) * (L + 1), KC = K | 1;
  const int N = a.N, S = a.S;
  if (a.coeff_out) {
    float* crow = a.coeff_out + (size_t)c * S * N * K;
    for (int f = lane; f < S * N * K; f += 32) {
      const int sn = f / K;
      crow[f] = cbuf[sn * KC + (f - sn * K)];
    }
  }
  float* orow = a.out + (size_t)c * a.F;
  if (a.mode == SOAPB_OUT_PS) {
    const int nblk = a.crossover ? S * (S + 1) / 2 : S;
    const int q32 = 32 / N, r32 = 32 % N;  // p -> p + 32 in the off-diagonal (n, n') order
    for (int b = 0; b < nblk; ++b) {
      const int jj = s_blk[2 * b], fb0 = s_blk[2 * b + 1];
      const int j = jj & 255, jd = jj >> 8;
      const bool diag = j == jd;
      const int np = diag ? N * (N + 1) / 2 : N * N;
#pragma unroll 1  // one copy of the l loop: smaller code, fewer instruction-fetch stalls
      for (int l = 0; l <= L; ++l) {
        float* o = orow + fb0 + l * np;
        int n = lane / N, nd = lane - (lane / N) * N;  // off-diagonal (n, n') of p, advanced by 32 per step
        for (int p = lane; p < np; p += 32) {
          if (diag) {
            n = s_tri[2 * p];
            nd = s_tri[2 * p + 1];
          }
          const float* x = cbuf + (j * N + n) * KC + l * l;
          const float* y = cbuf + (jd * N + nd) * KC + l * l;
          float s = 0.0f;
#pragma unroll
          for (int m = 0; m < 2 * l + 1; ++m) s = fmaf(x[m], y[m], s);
          o[p] = s * s_pref[l];
          if (!diag) {
            n += q32;
            nd += r32;
            if (nd >= N) { nd -= N; ++n; }
          }
        }
      }
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
}

// H pair streams per warp (1, or 2 for small l_max): half-warp h takes pairs
// 16 h .. 16 h + 15 of every staged batch of 32.  Each stream keeps its own
// species and segment; the streams flush their species partials into the
// centre's coefficient buffer one after the other, so sums are deterministic.
template <int L, int GN, int H>
__device__ __forceinline__ void descriptor_body(const DescArgs& a) {
  using Sh = DescShape<L>;
  constexpr int YS = Sh::YS, KC = Sh::KC, M = 2 * L + 1;
  constexpr int HL = 32 / H;           // lanes per stream
  constexpr int LPL = HL / (L + 1);    // lanes per l
  constexpr int HOFF = (H == 2) ? Sh::HOFF : 0;
  extern __shared__ float sm[];
  __shared__ float s_pref[kMaxL + 1];
  __shared__ int s_blk[2 * kMaxBlocks];              // (j | jd << 8, first feature) per species block
  __shared__ unsigned char s_tri[2 * kMaxTri];       // (n, n') of the upper-triangle index
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int N = a.N, S = a.S, NF = N * (L + 1);
  const int cbn = S * N * KC;
  // pairs staged per batch: 16 with one stream (half the harmonic rows in shared
  // memory, so more warps fit an SM), 32 with two (16 per stream)
  constexpr int BQ = (H == 2) ? 32 : 16;
  float* Y = sm + (size_t)wid * ((H == 2) ? Sh::warp_floats(S, N) : Sh::warp_floats16(S, N));
  float* tt = Y + BQ * YS + ((H == 2) ? Sh::HOFF : 0);
  int* sg = (int*)(tt + BQ);
  int* spp = sg + BQ;
  float* cbuf = (float*)(spp + BQ);
  desc_tables<L>(a, s_pref, s_blk, s_tri);
  __syncthreads();

  // lane -> stream, l and its functions n = k GN + g
  const int h = (H == 2) ? (lane >> 4) : 0, hl = lane & (HL - 1);
  const int l_me = hl / LPL, k_me = hl % LPL;
  const bool active = l_me <= L && k_me * GN < N;
  const int lme = active ? l_me : 0;
  const int mme = 2 * lme + 1;
  const int ybm = ybase(lme) + h * (16 * YS + HOFF);  // this stream's row block
  float selfb[GN];
#pragma unroll
  for (int g = 0; g < GN; ++g) {
    const int n = k_me * GN + g;
    selfb[g] = (active && n < N) ? __ldg(a.selfv + fn_index(n, lme, N)) : 0.0f;
  }

  for (;;) {
    int c32 = 0;
    if (lane == 0) c32 = atomicAdd(a.counter, 1);
    const int64_t c = __shfl_sync(0xffffffffu, c32, 0);
    if (c >= a.n_centres) break;
    for (int i = lane; i < cbn; i += 32) cbuf[i] = 0.0f;
    float acc[GN][M];
#pragma unroll
    for (int g = 0; g < GN; ++g)
#pragma unroll
      for (int m = 0; m < M; ++m) acc[g][m] = 0.0f;
    float cf[GN][kNCoef];
#pragma unroll
    for (int g = 0; g < GN; ++g)
#pragma unroll
      for (int k = 0; k < kNCoef; ++k) cf[g][k] = 0.0f;
    int cur_sp = -1, cur_seg = -1;
    const int64_t p0 = a.pair_off[c], p1 = a.pair_off[c + 1];
    __syncwarp();

    auto flush = [&](int sp) {
      if (active) {
#pragma unroll
        for (int g = 0; g < GN; ++g) {
          const int n = k_me * GN + g;
          if (n < N) {
            float* dst = cbuf + (sp * N + n) * KC + lme * lme;
#pragma unroll
            for (int m = 0; m < M; ++m)
              if (m < mme) dst[m] += acc[g][m];
          }
        }
      }
#pragma unroll
      for (int g = 0; g < GN; ++g)
#pragma unroll
        for (int m = 0; m < M; ++m) acc[g][m] = 0.0f;
    };

    for (int64_t base = p0; base < p1; base += BQ) {
      const int nt = (int)min((int64_t)BQ, p1 - base);
      if (lane < nt) {
        const float4 pr = __ldg(a.pairs + base + lane);
        const int w = __float_as_int(pr.w);
        const float r = sqrtf(pr.x * pr.x + pr.y * pr.y + pr.z * pr.z);
        int seg;
        float t;
        seg_coord(r, a.inv_h, a.nseg, seg, t);
        tt[lane] = (r > 0.0f) ? t : 3.0f;  // 3: r = 0 edge, takes the self value
        sg[lane] = seg;
        spp[lane] = (int)((unsigned)w >> kAtomBits);
        float* yrow = Y + lane * YS + ((H == 2 && lane >= 16) ? HOFF : 0);
        SolidHarmonics<L>::values(pr.x, pr.y, pr.z, [&](int idx, float v) { yrow[ypos(idx)] = v; });
      }
      __syncwarp();
      const int nq = (H == 2) ? min(nt, 16) : nt;
      for (int j = 0; j < nq; ++j) {
        const int q = h * 16 + j;
        const bool valid = (H == 1) || q < nt;  // the second stream of a short batch idles
        const int sp = valid ? spp[q] : cur_sp;
        if (H == 1) {
          if (sp != cur_sp) {
            if (cur_sp >= 0) flush(cur_sp);
            cur_sp = sp;
          }
        } else if (__any_sync(0xffffffffu, sp != cur_sp)) {
#pragma unroll
          for (int hh = 0; hh < H; ++hh) {  // stream 0 first, then stream 1
            if (h == hh && sp != cur_sp && cur_sp >= 0) flush(cur_sp);
            __syncwarp();
          }
          cur_sp = sp;
        }
        const int seg = valid ? sg[q] : cur_seg;
        if (seg != cur_seg) {
          if (active) {
#pragma unroll
            for (int g = 0; g < GN; ++g) {
              const int n = k_me * GN + g;
              if (n < N) load_coef(a.tab_b, seg, fn_index(n, lme, N), NF, cf[g]);
            }
          }
          cur_seg = seg;
        }
        if (valid) {
          const float t = tt[q];
          float B[GN];
#pragma unroll
          for (int g = 0; g < GN; ++g) B[g] = (t > 2.0f) ? selfb[g] : horner7(cf[g], t);
          // all M slots, without a per-lane test: slots m >= 2l+1 read on along
          // the row (position <= ybase(l) + 2L < YS, in bounds) and collect
          // values that flush() never stores, so no branch is needed per slot
          const float* yr = Y + j * YS + ybm;
#pragma unroll
          for (int m = 0; m < M; ++m) {
            const float yv = yr[m];
#pragma unroll
            for (int g = 0; g < GN; ++g) acc[g][m] = fmaf(B[g], yv, acc[g][m]);
          }
        }
      }
      __syncwarp();
    }
#pragma unroll
    for (int hh = 0; hh < H; ++hh) {
      if (h == hh && cur_sp >= 0) flush(cur_sp);
      __syncwarp();
    }
    desc_epilogue<L>(a, c, cbuf, lane, s_pref, s_blk, s_tri);
    __syncwarp();
  }
}

template <int L, int GN>
__global__ void __launch_bounds__(128) k_descriptor(DescArgs a) {
  descriptor_body<L, GN, 1>(a);
}

// Two pair streams (l_max <= 4): up to 128 registers, 4 blocks of 4 warps per
// SM (1M-atom cluster: 28.7 ms, against 33.6 ms capped at 96 registers for 5 blocks).
template <int L, int GN>
__global__ void __launch_bounds__(128, 4) k_descriptor_2s(DescArgs a) {
  descriptor_body<L, GN, 2>(a);
}

// Epilogue of the radial-index-lane kernel: coefficient rows KR = K4 floats
// apart (16-byte aligned).  For the power spectrum each lane takes one (n, n')
// pair of a species block and walks every l with compile-time m loops,
// reading the two rows as float4; for each l the lanes write consecutive
// features (coalesced).  Same outputs and DScribe order as desc_epilogue.
template <int L, int KR>
__device__ __forceinline__ void desc_epilogue_n(const DescArgs& a, int64_t c, const float* cbuf, int lane,
                                                const float* s_pref, const int* s_blk, const unsigned char* s_tri) {
  constexpr int K = (L + 1) * (L + 1);
  const int N = a.N, S = a.S;
  if (a.coeff_out) {
    float* crow = a.coeff_out + (size_t)c * S * N * K;
    for (int f = lane; f < S * N * K; f += 32) {
      const int sn = f / K;
      crow[f] = cbuf[sn * KR + (f - sn * K)];
    }
  }
  float* orow = a.out + (size_t)c * a.F;
  if (a.mode != SOAPB_OUT_PS) {
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
      orow[f] = cbuf[sn * KR + src] * scale;
    }
    return;
  }
  const int nblk = a.crossover ? S * (S + 1) / 2 : S;
  for (int b = 0; b < nblk; ++b) {
    const int jj = s_blk[2 * b], fb0 = s_blk[2 * b + 1];
    const int j = jj & 255, jd = jj >> 8;
    const bool diag = j == jd;
    const int np = diag ? N * (N + 1) / 2 : N * N;
    for (int p = lane; p < np; p += 32) {
      int n, nd;
      if (diag) {
        n = s_tri[2 * p];
        nd = s_tri[2 * p + 1];
      } else {
        n = p / N;
        nd = p - n * N;
      }
      const float4* x4 = reinterpret_cast<const float4*>(cbuf + (j * N + n) * KR);
      const float4* y4 = reinterpret_cast<const float4*>(cbuf + (jd * N + nd) * KR);
      float* o = orow + fb0 + p;
#pragma unroll
      for (int l = 0; l <= L; ++l) {
        const int q0 = (l * l) / 4, q1 = ((l + 1) * (l + 1) - 1) / 4;  // float4 chunks holding slots l^2..(l+1)^2-1
        float xv[16], yv[16];
#pragma unroll
        for (int q = q0; q <= q1; ++q) {
          const float4 u = x4[q], v = y4[q];
          xv[4 * (q - q0)] = u.x; xv[4 * (q - q0) + 1] = u.y; xv[4 * (q - q0) + 2] = u.z; xv[4 * (q - q0) + 3] = u.w;
          yv[4 * (q - q0)] = v.x; yv[4 * (q - q0) + 1] = v.y; yv[4 * (q - q0) + 2] = v.z; yv[4 * (q - q0) + 3] = v.w;
        }
        float acc = 0.0f;
#pragma unroll
        for (int m = 0; m < 2 * l + 1; ++m) {
          const int i = l * l + m - 4 * q0;
          acc = fmaf(xv[i], yv[i], acc);
        }
        o[l * np] = acc * s_pref[l];
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Radial-index lanes (n_max <= 8, l_max <= 6): lane n of a stream owns the
// radial index n and ALL K = (l_max+1)^2 accumulators c[n][lm] of it, so
// every lane does the same work per pair -- l_max+1 Horner evaluations
// (its functions (n, 0..l_max)) and K FMAs -- with no idle m slots.  NP
// lanes form a stream (NP = 8, or 4 for n_max <= 4); the 32 / NP streams of
// a warp walk contiguous, equal parts of the centre's pair list, so each
// stream sees only its part's species and segment runs and reloads its
// coefficients rarely.  32 pairs (NP per stream) are staged per batch, one
// per lane, as rows of solid harmonics in shared memory; rows have an odd
// stride, so the streams' reads of the same slot k from their rows hit
// different banks and the staging writes are conflict-free.
//
// The r = 0 edge of the centre's own atom needs no test in the pair loop:
// its solid harmonics are (Y00, 0, ..., 0) and its table value is
// w(0) B_n0(0), so staging scales its R_00 by self_ratio = w0 / w(0) and the
// edge adds exactly w0 B_n0(0) Y00.  A stream whose species changes flushes
// its accumulators into the centre's coefficient buffer; streams flush one
// after the other, and in a fixed order at the end, so sums are
// deterministic.
template <int L, int NP>
struct NShape {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int K4 = (K + 3) & ~3;  // row length in floats: float4 reads and writes
  static constexpr int H = 32 / NP;
  // coefficient rows c[s][n][0..K) also K4 floats apart: 16-byte aligned for the epilogue's
  // float4 reads, and the 8 rows n of a species (K4 = 4, 12, 16, 28, 36 or 52) start on 8
  // different groups of four banks
  static constexpr int KC = K4;
  // row q = h NP + j starts at q K4 + 4 h: the H streams' float4 reads of the
  // same slot fall on different groups of four banks whatever K4 is
  static constexpr int YF = 32 * K4 + 4 * H;
  // a multiple of 4 floats, so every warp's rows stay 16-byte aligned for the float4 accesses
  __host__ __device__ static int warp_floats(int S, int N) { return (YF + 4 * 32 + S * N * KC + 3) & ~3; }
};

// One pair's contribution to a radial-index lane: the lane's l_max + 1 radial
// functions at t (Horner), then acc[lm] += B_l R_lm over the pair's harmonic
// row, read as float4.
template <int L, int K4>
__device__ __forceinline__ void accumulate_pair(float (&acc)[(L + 1) * (L + 1)], const float (&cf)[L + 1][kNCoef],
                                                float t, const float* yrow) {
  constexpr int K = (L + 1) * (L + 1);
  float B[L + 1];
#pragma unroll
  for (int l = 0; l <= L; ++l) B[l] = horner7(cf[l], t);
  const float4* yr = reinterpret_cast<const float4*>(yrow);
#pragma unroll
  for (int k4 = 0; k4 < K4 / 4; ++k4) {
    const float4 v = yr[k4];
    const float vv[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int k = 4 * k4 + i;
      if (k < K) {
        int l = 0;
        while ((l + 1) * (l + 1) <= k) ++l;  // compile time: k is unrolled
        acc[k] = fmaf(B[l], vv[i], acc[k]);
      }
    }
  }
}

// Adds a lane's K accumulators to its 16-byte-aligned coefficient row (float4
// read-modify-write; the row's K4 - K padding slots stay zero).
template <int K, int K4>
__device__ __forceinline__ void flush_row(float* row, const float (&acc)[K]) {
  float4* r4 = reinterpret_cast<float4*>(row);
#pragma unroll
  for (int q = 0; q < K4 / 4; ++q) {
    float4 v = r4[q];
    v.x += acc[4 * q];
    if (4 * q + 1 < K) v.y += acc[4 * q + 1];
    if (4 * q + 2 < K) v.z += acc[4 * q + 2];
    if (4 * q + 3 < K) v.w += acc[4 * q + 3];
    r4[q] = v;
  }
}

template <int L, int NP>
__device__ __forceinline__ void descriptor_n_body(const DescArgs& a) {
  using Sh = NShape<L, NP>;
  constexpr int K = Sh::K, K4 = Sh::K4, KC = Sh::KC, H = Sh::H;
  extern __shared__ __align__(16) float sm[];
  __shared__ float s_pref[kMaxL + 1];
  __shared__ int s_blk[2 * kMaxBlocks];
  __shared__ unsigned char s_tri[2 * kMaxTri];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int N = a.N, S = a.S, NF = N * (L + 1);
  float* Y = sm + (size_t)wid * Sh::warp_floats(S, N);
  float* tt = Y + Sh::YF;  // per staged pair: segment coordinate t, segment, species
  int* sg = reinterpret_cast<int*>(tt + 32);
  int* spp = sg + 32;
  float* cbuf = Y + Sh::YF + 4 * 32;
  desc_tables<L>(a, s_pref, s_blk, s_tri);
  __syncthreads();
  const int h = lane / NP, n = lane - h * NP;
  const bool active = n < N;
  const int cbn = S * N * KC;
  float4* myrow = reinterpret_cast<float4*>(Y + lane * K4 + 4 * h);  // the row this lane stages

  for (;;) {
    int c32 = 0;
    if (lane == 0) c32 = atomicAdd(a.counter, 1);
    const int64_t c = __shfl_sync(0xffffffffu, c32, 0);
    if (c >= a.n_centres) break;
    for (int i = lane; i < cbn / 4; i += 32) reinterpret_cast<float4*>(cbuf)[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    // offsets inside the centre's list are 32-bit: 2^31 pairs of one centre would be 34 GB of list
    const int64_t p0 = a.pair_off[c];
    const int P = (int)(a.pair_off[c + 1] - p0);
    const float4* pc = a.pairs + p0;
    const int s0 = (int)(((int64_t)P * h) / H), s1 = (int)(((int64_t)P * (h + 1)) / H);  // this stream's pairs
    const int rounds = (P + H - 1) / H;                                                  // longest stream
    float acc[K];
#pragma unroll
    for (int k = 0; k < K; ++k) acc[k] = 0.0f;
    float cf[L + 1][kNCoef];
#pragma unroll
    for (int l = 0; l <= L; ++l)
#pragma unroll
      for (int k = 0; k < kNCoef; ++k) cf[l][k] = 0.0f;
    // each stream starts on the species of its first pair, so the centre's first batch takes the
    // fast path unless a species changes inside it
    int cur_sp = (s0 < s1) ? (int)((unsigned)__float_as_int(__ldg(&pc[s0].w)) >> kAtomBits) : -1;
    int cur_seg = -1;
    __syncwarp();

    for (int base = 0; base < rounds; base += NP) {
      // stage: lane (h, n) takes pair s0 + base + n of its stream into row `lane`
      const int e = s0 + base + n;
      const bool valid = e < s1;
      const int nvalid = max(0, min(NP, s1 - (s0 + base)));  // this stream's block
      int seg = -1, sp = -1;
      float t = 0.0f;
      {
        // a row past the end of this stream is the harmonics of the origin, (Y00, 0, ..., 0),
        // with R_00 scaled to 0: a zero row that adds nothing
        float yv[K4];
#pragma unroll
        for (int k = K; k < K4; ++k) yv[k] = 0.0f;
        const float4 pr = valid ? __ldg(pc + e) : make_float4(0.0f, 0.0f, 0.0f, 0.0f);
        // the stream's pair of the next batch: into L1 while this batch runs
        if (e + NP < s1) asm volatile("prefetch.global.L1 [%0];" ::"l"(pc + e + NP));
        const float r = sqrtf(pr.x * pr.x + pr.y * pr.y + pr.z * pr.z);
        seg_coord(r, a.inv_h, a.nseg, seg, t);
        sp = (int)((unsigned)__float_as_int(pr.w) >> kAtomBits);
        SolidHarmonics<L>::values(pr.x, pr.y, pr.z, [&](int idx, float v) { yv[idx] = v; });
        // the centre's own Gaussian (r = 0): w0 B_n0(0) Y00
        yv[0] *= valid ? ((r > 0.0f) ? 1.0f : a.self_ratio) : 0.0f;
        if (!valid) {
          seg = -1;
          sp = -1;
          t = 0.0f;
        }
#pragma unroll
        for (int k4 = 0; k4 < K4 / 4; ++k4)
          myrow[k4] = make_float4(yv[4 * k4], yv[4 * k4 + 1], yv[4 * k4 + 2], yv[4 * k4 + 3]);
      }
      // rows past the end repeat the segment and species of the block's last pair (or the
      // stream's current ones), so they change nothing; then one bit per row marks where
      // the segment or the species differs from the stream's previous row
      const int last = h * NP + (nvalid > 0 ? nvalid - 1 : 0);
      const int seg_last = __shfl_sync(0xffffffffu, seg, last), sp_last = __shfl_sync(0xffffffffu, sp, last);
      if (!valid) {
        seg = nvalid > 0 ? seg_last : cur_seg;
        sp = nvalid > 0 ? sp_last : cur_sp;
      }
      int seg_prev = __shfl_up_sync(0xffffffffu, seg, 1), sp_prev = __shfl_up_sync(0xffffffffu, sp, 1);
      if (n == 0) {
        seg_prev = cur_seg;
        sp_prev = cur_sp;
      }
      const unsigned seg_chg = __ballot_sync(0xffffffffu, seg != seg_prev);
      const unsigned sp_chg = __ballot_sync(0xffffffffu, sp != sp_prev);
      tt[lane] = t;
      sg[lane] = seg;
      spp[lane] = sp;
      __syncwarp();
      if (sp_chg == 0) {
        // no species change in any stream: t, a coefficient reload where the segment changes,
        // Horner and the K FMAs per pair
#pragma unroll 2
        for (int j = 0; j < NP; ++j) {
          const int q = h * NP + j;
          if ((seg_chg >> q) & 1u) {
            const int sq = sg[q];
            if (active) {
#pragma unroll
              for (int l = 0; l <= L; ++l) load_coef(a.tab_b, sq, fn_index(n, l, N), NF, cf[l]);
            }
          }
          accumulate_pair<L, K4>(acc, cf, tt[q], Y + q * K4 + 4 * h);
        }
      } else {
#pragma unroll 1
        for (int j = 0; j < NP; ++j) {
          const int q = h * NP + j;
          const int spq = spp[q];
          if (__any_sync(0xffffffffu, spq != cur_sp)) {
#pragma unroll
            for (int hh = 0; hh < H; ++hh) {  // streams flush one after the other
              if (h == hh && spq != cur_sp) {
                if (cur_sp >= 0 && active) {
                  flush_row<K, K4>(cbuf + (cur_sp * N + n) * KC, acc);
                }
#pragma unroll
                for (int k = 0; k < K; ++k) acc[k] = 0.0f;
                cur_sp = spq;
              }
              __syncwarp();
            }
          }
          if ((seg_chg >> q) & 1u) {
            const int sq = sg[q];
            if (active) {
#pragma unroll
              for (int l = 0; l <= L; ++l) load_coef(a.tab_b, sq, fn_index(n, l, N), NF, cf[l]);
            }
          }
          accumulate_pair<L, K4>(acc, cf, tt[q], Y + q * K4 + 4 * h);
        }
      }
      cur_seg = sg[h * NP + NP - 1];
      cur_sp = spp[h * NP + NP - 1];
      __syncwarp();
    }
#pragma unroll
    for (int hh = 0; hh < H; ++hh) {
      if (h == hh && cur_sp >= 0 && active) {
        flush_row<K, K4>(cbuf + (cur_sp * N + n) * KC, acc);
      }
      __syncwarp();
    }
    desc_epilogue_n<L, KC>(a, c, cbuf, lane, s_pref, s_blk, s_tri);
    __syncwarp();
  }
}

// l_max <= 4: 4 blocks of 4 warps per SM at 128 registers; l_max 5: 3 blocks; l_max 6: 2 blocks,
// so its 49 accumulators and 7 x 8 coefficients per lane stay in registers (at 3 blocks they spill)
template <int L, int NP>
__global__ void __launch_bounds__(128, (L <= 4) ? 4 : (L == 5 ? 3 : 2)) k_descriptor_n(DescArgs a) {
  descriptor_n_body<L, NP>(a);
}

template <int L, int NP>
static int launch_descriptor_n(const DescArgs& a, int wpb_tuned, cudaStream_t st) {
  const int per_warp = 4 * NShape<L, NP>::warp_floats(a.S, a.N);
  if (per_warp % 16 != 0) return set_error(SOAPB_ERR_ARG, "descriptor: warp slice of %d B not 16-byte aligned", per_warp);
  int wpb = (200 * 1024) / per_warp;
  wpb = wpb > 4 ? 4 : wpb;
  if ((wpb_tuned == 1 || wpb_tuned == 2 || wpb_tuned == 4) && wpb_tuned <= wpb) wpb = wpb_tuned;
  if (wpb < 1) return set_error(SOAPB_ERR_UNSUPPORTED, "descriptor shared memory %d B per warp too large", per_warp);
  const int smem = wpb * per_warp;
  auto kern = k_descriptor_n<L, NP>;
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
  return check_launch("k_descriptor_n");
}

template <int L, int GN, int H>
static int launch_descriptor(const DescArgs& a, int wpb_tuned, cudaStream_t st) {
  const int per_warp =
      4 * ((H == 2) ? DescShape<L>::warp_floats(a.S, a.N) : DescShape<L>::warp_floats16(a.S, a.N));
  int wpb = (200 * 1024) / per_warp;
  wpb = wpb > 4 ? 4 : wpb;
  if ((wpb_tuned == 1 || wpb_tuned == 2 || wpb_tuned == 4) && wpb_tuned <= wpb) wpb = wpb_tuned;
  if (wpb < 1) return set_error(SOAPB_ERR_UNSUPPORTED, "descriptor shared memory %d B per warp too large", per_warp);
  const int smem = wpb * per_warp;
  auto kern = (H == 2) ? k_descriptor_2s<L, GN> : k_descriptor<L, GN>;
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
  static int run(const DescArgs& a, int gn, int wpb, bool lgroup_only, cudaStream_t st) {
    if constexpr (L <= kMaxLNLanes) {
      if (!lgroup_only && a.N <= 8 && isfinite(a.self_ratio))
        return a.N <= 4 ? launch_descriptor_n<L, 4>(a, wpb, st) : launch_descriptor_n<L, 8>(a, wpb, st);
    }
    if constexpr (L <= 4) {
      if (desc_two_streams(a.N, L)) {  // functions per lane fixed by (N, L): ceil(N / floor(16 / (L+1)))
        const int lpl = 16 / (L + 1), g2 = (a.N + lpl - 1) / lpl;
        switch (g2) {
          case 1: return launch_descriptor<L, 1, 2>(a, wpb, st);
          case 2: return launch_descriptor<L, 2, 2>(a, wpb, st);
          default: return launch_descriptor<L, 3, 2>(a, wpb, st);
        }
      }
    }
    if constexpr (L >= 10) {  // two lanes per l: 4 radial functions per lane cover n_max <= 8
      if (a.N > 8) return set_error(SOAPB_ERR_UNSUPPORTED, "descriptor: l_max %d is built for n_max <= 8", L);
      return launch_descriptor<L, 4, 1>(a, wpb, st);
    } else {
      switch (gn) {
        case 1: return launch_descriptor<L, 1, 1>(a, wpb, st);
        case 2: return launch_descriptor<L, 2, 1>(a, wpb, st);
        case 3: return launch_descriptor<L, 3, 1>(a, wpb, st);
        case 4: return launch_descriptor<L, 4, 1>(a, wpb, st);
        case 6: return launch_descriptor<L, 6, 1>(a, wpb, st);
        default: return set_error(SOAPB_ERR_UNSUPPORTED, "descriptor: %d radial functions per lane not built", gn);
      }
    }
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
  cudaStream_t st = (cudaStream_t)stream;
  DescArgs a;
  a.pair_off = d_pair_off;
  a.pairs = (const float4*)d_pairs;
  a.n_centres = n_centres;
  a.tab_b = (const float*)((const char*)b->dev + b->off_tab_b);
  a.selfv = (const float*)((const char*)b->dev + b->off_self);
  a.out = d_out;
  a.coeff_out = d_coeff;
  a.counter = d_counter;
  a.N = N;
  a.S = b->n_species;
  a.nseg = b->n_seg;
  a.F = out_mode == SOAPB_OUT_PS ? b->n_feat_ps : b->n_feat_cc;
  a.mode = out_mode;
  a.crossover = b->crossover ? 1 : 0;
  a.inv_h = (float)(1.0 / b->seg_width);
  {
    // self_ratio = w0 / w(0) of the weighting (the r = 0 table value is w(0) B_n0(0)); not finite
    // (a weighting singular at r = 0) sends the call to the kernels that use the self table
    const double w0 = b->weighting == SOAPB_W_NONE ? 1.0 : b->w_w0;
    double w_at0 = 1.0;
    if (b->weighting == SOAPB_W_POLY) w_at0 = b->w_c;
    else if (b->weighting == SOAPB_W_POW) w_at0 = b->w_c / (b->w_d + pow(0.0, b->w_m));
    else if (b->weighting == SOAPB_W_EXP) w_at0 = b->w_c / (b->w_d + 1.0);
    a.self_ratio = (float)(w0 / w_at0);
  }
  int rc = check_cuda(cudaMemsetAsync(d_counter, 0, sizeof(int32_t), st), "reset work counter");
  if (rc) return rc;
  int gn = desc_group(N, L);
  const int tg = b->tune[1];
  if (tg > gn && (tg == 2 || tg == 3 || tg == 4 || tg == 6)) gn = tg;
  return dispatch_l<DescDispatch>(L, a, gn, b->tune[0], b->tune[3] == 1, st);
}
