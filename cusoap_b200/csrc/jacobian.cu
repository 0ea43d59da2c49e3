// Dense descriptor Jacobian d desc[c, f] / d x[a, d], written once per
// element (zeros included) in the DScribe layout (C, n_inc, 3, F).
//
// Reference: derivatives_analytical_ps (soap_generator.py:2270-2626) and its
// Triton kernels _ps_uv_kernel / _ps_jacobian_dense_kernel /
// _cc_jacobian_dense_kernel (:50-220).  Per edge e (centre c -> atom a,
// rvec = x_a - x_c, species s):
//   g[d, n, lm] = r_d Bhat_nl R_lm + B_nl dR_lm/dx_d
//   cc:  d c[s, n, lm] / d x_a,d         = sum_e g
//   ps:  d p[(j n), (j' n'), l] / dx_a,d = pref_l sum_e [ d_{j s} (r_d Bhat_nl U[j'n'l] + B_nl V_d[j'n'l])
//                                                        + d_{j' s} (r_d Bhat_n'l U[jnl] + B_n'l V_d[jnl]) ]
//   with U[k q l] = sum_m R_lm c[k q lm], V_d[k q l] = sum_m dR_lm/dx_d c[k q lm].
// Unlike the reference kernels this accumulates every edge of an atom, so
// periodic images are handled; attach=1 adds the centre-motion term
// (-sum over the centre's edges on the centre atom's row).
//
// The output is ~99% of the traffic (45 GB for 3000 atoms at F=420) and
// mostly zeros, so the kernel is an HBM write stream: one CTA per centre
// writes its contiguous (n_inc, 3, F) block front to back, computing the few
// nonzero rows in between.  Each staged edge is pre-contracted into
//   X0[a] = {U, Q, P_x, V_x},  X1[a] = {P_y, V_y, P_z, V_z},  a = (j, n, l),
//   Q = d_{j s} B_nl, P_d = d_{j s} r_d Bhat_nl (times the entry's sign),
// so a nonzero element is pref_l (P_d[a] U[b] + Q[a] V_d[b] + P_d[b] U[a] + Q[b] V_d[a]):
// four FMAs on two pairs of 16-byte shared-memory loads (X is stored l-major,
// a = (l S + j) N + n, so consecutive features read consecutive float4s).
//
// Two launches, sharing a workspace:
//   k_jac_entries  per centre: the (row, edge) entries of its included atoms,
//                  sorted by row, and a bitmap of its nonzero rows;
//   k_jacobian     warp roles inside every block: warp 0 streams the block's
//                  share of the zero rows (64-row chunks in global row order)
//                  with TMA bulk copies of a zero tile in shared memory --
//                  one issuing lane, no load/store-unit traffic -- while warps
//                  1..7 compute the nonzero rows (entries staged in shared
//                  memory, each thread four consecutive features of a row in
//                  the three directions, stored as 16-byte vectors).
// Zero and nonzero rows are disjoint, so every element is written once and the
// two roles never synchronise.
#include "common.cuh"

namespace soapb {

struct JacArgs {
  const int64_t* pair_off;
  const float4* pairs;
  const float* coeff;
  const int* inc_row;
  const int* centre_atom;
  const float* tab_b;
  const float* tab_bh;   // D = d(w B)/dr; Bhat = D / r
  const float* selfv;    // w0 B_nl(0) for r = 0 edges
  const int* ftab;
  float* out;
  int* status;
  int* counter;                  // work queue of the compute kernel
  int* ent_cnt;                  // (n_centres) entries per centre
  unsigned long long* ent;       // sorted entries, centre c at ent_mult * pair_off[c]
  unsigned long long* ent_tmp;   // merge buffer of a centre with more than cap entries, same offsets
  unsigned int* bitmap;          // (n_centres * n_inc) nonzero-row bits
  int64_t n_centres, n_inc;
  int N, S, nseg, F, mode, attach, cap, eb, ent_mult;
  float inv_h;
};

template <int L>
struct JacShape {
  static constexpr int K = (L + 1) * (L + 1);
  static constexpr int KC = K | 1;
  static constexpr int LP = L + 1;
  // staged entry: header(8: rx ry rz species sign) | B, Bhat (NF each) | R (K) | dR (3K) |
  // X0, X1 (4 SNL floats each, ps only, 16-byte aligned); total rounded to 16 bytes
  __host__ __device__ static int xoff(int N) { return (8 + 2 * N * LP + 4 * K + 3) & ~3; }
  __host__ __device__ static int entry_floats(int N, int S, int mode) {
    const int f = xoff(N) + (mode == SOAPB_OUT_PS ? 8 * S * N * LP : 0);
    return (f + 3) & ~3;
  }
  __host__ __device__ static int cs_floats(int N, int S) { return (S * N * KC + 3) & ~3; }
};

// The (row, edge) entries of the centre's included atoms, in any order: each is
// handed to put(k, key) with k = 0, 1, ... from a block counter.  Returns the
// count (all threads of the CTA; ends with a barrier).
template <class Put>
__device__ int gather_entries(const JacArgs& a, int64_t p0, int P, int catom, int crow, int* s_nent, Put put) {
  const int tid = threadIdx.x, nth = blockDim.x;
  if (tid == 0) *s_nent = 0;
  __syncthreads();
  for (int e = tid; e < P; e += nth) {
    const int atom = __float_as_int(a.pairs[p0 + e].w) & kAtomMask;
    if (a.attach && atom == catom) continue;  // centre and neighbour terms cancel
    const int row = a.inc_row[atom];
    if (row >= 0) put(atomicAdd(s_nent, 1), ((unsigned long long)row << 32) | (unsigned)e);
    if (crow >= 0) put(atomicAdd(s_nent, 1), ((unsigned long long)crow << 32) | (unsigned)e);
  }
  __syncthreads();
  return *s_nent;
}

// Ascending bitonic sort of n2 (a power of two) keys in shared memory (all threads of the CTA).
__device__ void block_bitonic(unsigned long long* keys, int n2) {
  const int tid = threadIdx.x, nth = blockDim.x;
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
}

// Sorts n keys (n <= cap) in shared memory, padding to a power of two with ~0.
__device__ void sort_tile(unsigned long long* keys, int n) {
  int n2 = 1;
  while (n2 < n) n2 <<= 1;
  for (int i = n + threadIdx.x; i < n2; i += blockDim.x) keys[i] = ~0ull;
  __syncthreads();
  block_bitonic(keys, n2);
}

// Merges the sorted runs A[0, na) and B[0, nb) (distinct keys) into O: thread t
// writes a contiguous share of the outputs, starting where a binary search of
// the merge path puts its first output (all threads of the CTA).
__device__ void merge_runs(const unsigned long long* A, int na, const unsigned long long* B, int nb,
                           unsigned long long* O) {
  const int total = na + nb, nth = blockDim.x;
  const int per = (total + nth - 1) / nth;
  const int o0 = threadIdx.x * per, o1 = min(o0 + per, total);
  if (o0 >= total) return;
  int lo = max(0, o0 - nb), hi = min(o0, na);
  while (lo < hi) {  // fewest outputs from A such that the next A key follows the last B key taken
    const int i = (lo + hi) >> 1;
    if (A[i] < B[o0 - i - 1]) lo = i + 1;
    else hi = i;
  }
  int i = lo, j = o0 - lo;
  for (int o = o0; o < o1; ++o) O[o] = (j >= nb || (i < na && A[i] < B[j])) ? A[i++] : B[j++];
}

// Per-centre entries sorted by row into dst (global memory).  Centres whose
// entries fit the shared-memory buffer (cap keys) are gathered and sorted
// there.  Larger centres are gathered straight into dst, sorted in tiles of
// cap keys in shared memory, and the sorted runs merged pairwise through tmp
// (the same slot in a second buffer) until one run is left.  Keys are
// distinct, so the order is the same however the gather was interleaved.
__device__ int centre_entries(const JacArgs& a, int64_t p0, int P, int catom, int crow, unsigned long long* skeys,
                              unsigned long long* dst, unsigned long long* tmp, int* s_nent) {
  const int tid = threadIdx.x, nth = blockDim.x;
  if (a.ent_mult * P <= a.cap) {
    const int nent = gather_entries(a, p0, P, catom, crow, s_nent,
                                    [&](int k, unsigned long long key) { skeys[k] = key; });
    sort_tile(skeys, nent);
    for (int i = tid; i < nent; i += nth) dst[i] = skeys[i];
    __syncthreads();
    return nent;
  }
  const int nent = gather_entries(a, p0, P, catom, crow, s_nent,
                                  [&](int k, unsigned long long key) { dst[k] = key; });
  for (int t0 = 0; t0 < nent; t0 += a.cap) {
    const int n = min(a.cap, nent - t0);
    for (int i = tid; i < n; i += nth) skeys[i] = dst[t0 + i];
    sort_tile(skeys, n);
    for (int i = tid; i < n; i += nth) dst[t0 + i] = skeys[i];
    __syncthreads();
  }
  unsigned long long *src = dst, *out = tmp;
  for (int w = a.cap; w < nent; w *= 2) {
    for (int lo = 0; lo < nent; lo += 2 * w) {
      const int mid = min(lo + w, nent), hi = min(lo + 2 * w, nent);
      merge_runs(src + lo, mid - lo, src + mid, hi - mid, out + lo);
    }
    __syncthreads();
    unsigned long long* s = src;
    src = out;
    out = s;
  }
  if (src != dst) {
    for (int i = tid; i < nent; i += nth) dst[i] = src[i];
    __syncthreads();
  }
  return nent;
}

__global__ void __launch_bounds__(256) k_jac_entries(JacArgs a) {
  extern __shared__ __align__(16) unsigned long long skeys[];
  __shared__ int s_nent;
  for (int64_t c = blockIdx.x; c < a.n_centres; c += gridDim.x) {
    const int64_t p0 = a.pair_off[c];
    const int P = (int)(a.pair_off[c + 1] - p0);
    const int catom = a.attach ? a.centre_atom[c] : -1;
    const int crow = (catom >= 0) ? a.inc_row[catom] : -1;
    unsigned long long* dst = a.ent + (size_t)a.ent_mult * p0;
    unsigned long long* tmp = a.ent_tmp + (size_t)a.ent_mult * p0;
    const int nent = centre_entries(a, p0, P, catom, crow, skeys, dst, tmp, &s_nent);
    for (int i = threadIdx.x; i < nent; i += blockDim.x) {
      const int64_t r = (int64_t)c * a.n_inc + (int64_t)(dst[i] >> 32);
      atomicOr(a.bitmap + (r >> 5), 1u << (r & 31));
    }
    if (threadIdx.x == 0) a.ent_cnt[c] = nent;
    __syncthreads();
  }
}

constexpr int kZeroTile = 16384;  // bytes of the shared-memory zero tile
constexpr int kZeroChunkRows = 64;

__device__ __forceinline__ void bulk_s2g(void* g, const void* s, uint32_t bytes) {
  asm volatile("cp.async.bulk.global.shared::cta.bulk_group [%0], [%1], %2;\n" ::"l"(g),
               "r"((uint32_t)__cvta_generic_to_shared(s)), "r"(bytes)
               : "memory");
}

// Zero rows of 64-row chunks (global row order) claimed from a work queue
// (zq), by TMA bulk copies of the zero tile; lane 0 issues, the copies run
// asynchronously and the lane waits for all of them before returning (the
// tile must outlive them).  Every block's zero warp runs this from the start
// and its compute warps join once the centre queue is empty, so the zero
// stream ends together with the compute work.  Rows are 12 F bytes, a
// multiple of 16 (F % 4 == 0).
__device__ void jac_zero_rows_tma(const JacArgs& a, const void* ztile, int* zq) {
  if ((threadIdx.x & 31) != 0) return;
  const int64_t nrows = a.n_centres * a.n_inc;
  const int64_t row_bytes = 12 * (int64_t)a.F;
  const int64_t nchunks = (nrows + kZeroChunkRows - 1) / kZeroChunkRows;
  char* out = reinterpret_cast<char*>(a.out);
  for (;;) {
    const int64_t k = (int64_t)(unsigned)atomicAdd(zq, 1);
    if (k >= nchunks) break;
    const int64_t r0 = k * kZeroChunkRows, r1 = min(r0 + (int64_t)kZeroChunkRows, nrows);
    int64_t run = -1;
    for (int64_t r = r0; r <= r1; ++r) {
      const bool zero = (r < r1) && !((a.bitmap[r >> 5] >> (r & 31)) & 1u);
      if (zero && run < 0) run = r;
      if (!zero && run >= 0) {  // zero rows [run, r)
        char* p = out + run * row_bytes;
        int64_t n = (r - run) * row_bytes;
        while (n > 0) {
          const uint32_t c = (uint32_t)(n < kZeroTile ? n : kZeroTile);
          bulk_s2g(p, ztile, c);
          p += c;
          n -= c;
        }
        run = -1;
      }
    }
    asm volatile("cp.async.bulk.commit_group;\n" ::: "memory");
  }
  asm volatile("cp.async.bulk.wait_group 0;\n" ::: "memory");
}

// Zero rows with 16-byte stores (rows not a multiple of 16 bytes), same chunks.
__device__ void jac_zero_rows_st(const JacArgs& a) {
  const int lane = threadIdx.x & 31;
  const int64_t nrows = a.n_centres * a.n_inc;
  const int64_t rowf = 3 * (int64_t)a.F;
  const int64_t nchunks = (nrows + kZeroChunkRows - 1) / kZeroChunkRows;
  for (int64_t k = blockIdx.x; k < nchunks; k += gridDim.x) {
    const int64_t r0 = k * kZeroChunkRows, r1 = min(r0 + (int64_t)kZeroChunkRows, nrows);
    for (int64_t r = r0; r < r1; ++r) {
      if ((a.bitmap[r >> 5] >> (r & 31)) & 1u) continue;
      float* p = a.out + r * rowf;
      for (int64_t i = lane; i < rowf; i += 32) __stcs(p + i, 0.0f);
    }
  }
}

// Named barrier over the compute warps only (id 1; id 0 is __syncthreads).
__device__ __forceinline__ void compute_bar(int nthreads) {
  asm volatile("bar.sync 1, %0;\n" ::"r"(nthreads) : "memory");
}

// Stage entries [b0, b0 + nb) of the centre into ed (all threads; ends with a barrier).
template <int L>
__device__ void stage_entries(const JacArgs& a, int64_t p0, const unsigned long long* keys, int b0, int nb, int crow,
                              const float* cs, float* ed, int EF, const float* sqrt_pref, int tid, int nth) {
  using Sh = JacShape<L>;
  constexpr int K = Sh::K, KC = Sh::KC, LP = Sh::LP;
  const int N = a.N, S = a.S, NF = N * LP, SNL = S * N * LP, XO = Sh::xoff(N);
  for (int i = tid; i < nb; i += nth) {
    const unsigned long long key = keys[b0 + i];
    const float4 pr = a.pairs[p0 + (int)(key & 0xffffffffu)];
    float* h = ed + (size_t)i * EF;
    h[0] = pr.x; h[1] = pr.y; h[2] = pr.z;
    h[3] = (float)((unsigned)__float_as_int(pr.w) >> kAtomBits);
    h[4] = (a.attach && (int)(key >> 32) == crow) ? -1.0f : 1.0f;
    float* R = h + 8 + 2 * NF;
    float* dR = R + K;
    SolidHarmonics<L>::with_gradients(pr.x, pr.y, pr.z, [&](int idx, float v, float dx, float dy, float dz) {
      R[idx] = v; dR[idx] = dx; dR[K + idx] = dy; dR[2 * K + idx] = dz;
    });
  }
  compute_bar(nth);
  if (tid < (nth / NF) * NF) {  // thread owns radial function fn, entries stepped (division-free loop)
    const int fn = tid % NF, istep = nth / NF;
    for (int i = tid / NF; i < nb; i += istep) {
      float* h = ed + (size_t)i * EF;
      const float r = sqrtf(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
      int seg;
      float tt;
      seg_coord(r, a.inv_h, a.nseg, seg, tt);
      float cf[kNCoef];
      load_coef(a.tab_b, seg, fn, NF, cf);
      h[8 + fn] = (r > 0.0f) ? horner7(cf, tt) : __ldg(a.selfv + fn);
      load_coef(a.tab_bh, seg, fn, NF, cf);
      h[8 + NF + fn] = (r > 0.0f) ? horner7(cf, tt) / r : 0.0f;
    }
  } else if (NF > nth) {  // more radial functions than threads: flat loop
    for (int t = tid; t < nb * NF; t += nth) {
      const int i = t / NF, fn = t % NF;
      float* h = ed + (size_t)i * EF;
      const float r = sqrtf(h[0] * h[0] + h[1] * h[1] + h[2] * h[2]);
      int seg;
      float tt;
      seg_coord(r, a.inv_h, a.nseg, seg, tt);
      float cf[kNCoef];
      load_coef(a.tab_b, seg, fn, NF, cf);
      h[8 + fn] = (r > 0.0f) ? horner7(cf, tt) : __ldg(a.selfv + fn);
      load_coef(a.tab_bh, seg, fn, NF, cf);
      h[8 + NF + fn] = (r > 0.0f) ? horner7(cf, tt) / r : 0.0f;
    }
  }
  compute_bar(nth);
  if (a.mode == SOAPB_OUT_PS) {
    // thread -> coefficient index ai = (l S + j) N + n (decoded once) and first entry;
    // entries stepped by istep (division-free loop)
    const bool small = SNL <= nth;
    const int istep = small ? nth / SNL : 1;
    const int ai0 = small ? tid % SNL : tid;
    const int i0 = small ? (tid < istep * SNL ? tid / SNL : nb) : 0;
    for (int ai = ai0; ai < SNL; ai += (small ? SNL : nth)) {
      const int l = ai / (S * N), jn = ai % (S * N);
      const int j = jn / N, n = jn % N;
      const float* cr = cs + jn * KC + l * l;
      for (int i = i0; i < nb; i += istep) {
        const float* h = ed + (size_t)i * EF;
        const float* R = h + 8 + 2 * NF;
        const float* dR = R + K;
        float u = 0.f, v0 = 0.f, v1 = 0.f, v2 = 0.f;
        for (int m = 0; m < 2 * l + 1; ++m) {
          const float cv = cr[m];
          u = fmaf(R[l * l + m], cv, u);
          v0 = fmaf(dR[l * l + m], cv, v0);
          v1 = fmaf(dR[K + l * l + m], cv, v1);
          v2 = fmaf(dR[2 * K + l * l + m], cv, v2);
        }
        // both factors carry sqrt(pref_l): the value is bilinear in X[a], X[b] of the same l
        const float sp = sqrt_pref[l];
        const bool own = ((int)h[3] == j);
        const float q = own ? sp * h[4] * h[8 + l * N + n] : 0.0f;
        const float bh = own ? sp * h[4] * h[8 + NF + l * N + n] : 0.0f;
        u *= sp; v0 *= sp; v1 *= sp; v2 *= sp;
        float4* X = reinterpret_cast<float4*>(ed + (size_t)i * EF + XO);
        X[ai] = make_float4(u, q, h[0] * bh, v0);
        X[SNL + ai] = make_float4(h[1] * bh, v1, h[2] * bh, v2);
      }
    }
    compute_bar(nth);
  }
}

// Values of the four features 4q .. 4q+3 in the three directions, summed over
// staged entries [g0, g1).  ps: X already carries sqrt(pref_l) on both sides.
template <int L>
__device__ __forceinline__ void quad_values(const JacArgs& a, const float* ed, int EF, int g0, int g1, int q,
                                            float (&v)[3][4]) {
  using Sh = JacShape<L>;
  constexpr int K = Sh::K, LP = Sh::LP;
  const int N = a.N, S = a.S, NF = N * LP, SNL = S * N * LP, XO = Sh::xoff(N), F = a.F;
#pragma unroll
  for (int k = 0; k < 4; ++k) v[0][k] = v[1][k] = v[2][k] = 0.f;
  if (a.mode == SOAPB_OUT_PS) {
    int code[4];
    if ((F & 3) == 0) {
      const int4 c4 = __ldg(reinterpret_cast<const int4*>(a.ftab) + q);  // pre-decoded: ia | ib << 12 | l << 24
      code[0] = c4.x; code[1] = c4.y; code[2] = c4.z; code[3] = c4.w;
    } else {
#pragma unroll
      for (int k = 0; k < 4; ++k) code[k] = (4 * q + k < F) ? __ldg(a.ftab + 4 * q + k) : 0;
    }
    for (int i = g0; i < g1; ++i) {
      const float4* X = reinterpret_cast<const float4*>(ed + (size_t)i * EF + XO);
#pragma unroll
      for (int k = 0; k < 4; ++k) {
        const int ia = code[k] & 4095, ib = (code[k] >> 12) & 4095;
        const float4 pa = X[ia], qa = X[SNL + ia], pb = X[ib], qb = X[SNL + ib];
        v[0][k] += pa.z * pb.x + pa.y * pb.w + pb.z * pa.x + pb.y * pa.w;
        v[1][k] += qa.x * pb.x + pa.y * qb.y + qb.x * pa.x + pb.y * qa.y;
        v[2][k] += qa.z * pb.x + pa.y * qb.w + qb.z * pa.x + pb.y * qa.w;
      }
    }
  } else {
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int f = 4 * q + k;
      if (f >= F) continue;
      const int sf = f / (N * K), rem = f - sf * N * K, n = rem / K, lo = rem - n * K;
      int src = lo;
      float scale = 1.0f;
      // DScribe cc layout: l = 1 stored (z, x, y) = source lm (2, 3, 1); lm >= 4 scaled by pi^-3/2
      if (lo >= 1 && lo <= 3) src = (lo == 3) ? 1 : lo + 1;
      if (lo >= 4) scale = (float)(1.0 / (kPi * 1.7724538509055160273));
      const int l = (int)sqrtf((float)src + 0.5f);
      for (int i = g0; i < g1; ++i) {
        const float* h = ed + (size_t)i * EF;
        if ((int)h[3] != sf) continue;
        const float* R = h + 8 + 2 * NF;
        const float* dR = R + K;
        const float bh = h[4] * h[8 + NF + l * N + n] * R[src], b = h[4] * h[8 + l * N + n];
        v[0][k] += scale * (h[0] * bh + b * dR[src]);
        v[1][k] += scale * (h[1] * bh + b * dR[K + src]);
        v[2][k] += scale * (h[2] * bh + b * dR[2 * K + src]);
      }
    }
  }
}

// Nonzero rows: centres from a work queue, entries staged in batches, each
// task = (row group, four consecutive features) stored as 16-byte vectors.
template <int L>
__global__ void __launch_bounds__(256) k_jacobian(JacArgs a) {
  using Sh = JacShape<L>;
  constexpr int K = Sh::K, KC = Sh::KC;
  constexpr int kCT = 224;  // compute threads (warps 1..7)
  const int N = a.N, S = a.S, F = a.F;
  const int Q = (F + 3) >> 2;
  const bool vec = (F & 3) == 0;
  extern __shared__ __align__(128) float smf[];
  float* ztile = smf;                            // kZeroTile bytes of zeros
  float* cs = ztile + kZeroTile / 4;
  float* ed = cs + Sh::cs_floats(N, S);
  const int EF = Sh::entry_floats(N, S, a.mode);
  __shared__ float s_sqrt_pref[kMaxL + 1];
  __shared__ int s_gstart[33];
  __shared__ int s_ng;
  __shared__ int s_c;
  if (threadIdx.x <= L) s_sqrt_pref[threadIdx.x] = sqrtf(sqrtf(8.0f * (float)(kPi * kPi) / (2.0f * threadIdx.x + 1.0f)));
  for (int i = threadIdx.x; i < kZeroTile / 4; i += blockDim.x) ztile[i] = 0.0f;
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");  // tile visible to the bulk-copy engine
  __syncthreads();
  if (threadIdx.x < 32) {  // zero role
    if (vec) jac_zero_rows_tma(a, ztile, a.counter + 1);
    else jac_zero_rows_st(a);
    return;
  }
  // compute role: warps 1..7, named barrier 1
  const int tid = threadIdx.x - 32;
  // thread -> (quad q0, first group g0t): quads stepped by qstep, groups by gstep (division-free loop)
  const int qstep = Q >= kCT ? kCT : Q, gstep = Q >= kCT ? 1 : kCT / Q;
  const int q0 = Q >= kCT ? tid : tid % Q;
  const int g0t = Q >= kCT ? 0 : (tid < gstep * Q ? tid / Q : 1 << 30);
  for (;;) {
    if (tid == 0) s_c = atomicAdd(a.counter, 1);
    compute_bar(kCT);
    const int64_t c = s_c;
    if (c >= a.n_centres) break;
    const int64_t p0 = a.pair_off[c];
    const int nent = a.ent_cnt[c];
    const unsigned long long* keys = a.ent + (size_t)a.ent_mult * p0;
    const int catom = a.attach ? a.centre_atom[c] : -1;
    const int crow = (catom >= 0) ? a.inc_row[catom] : -1;
    const int SNK = S * N * K;
    for (int i = tid; i < SNK; i += kCT) cs[(i / K) * KC + (i % K)] = a.coeff[(size_t)c * SNK + i];
    compute_bar(kCT);
    float* obase = a.out + (size_t)c * a.n_inc * 3 * F;
    int last_row = -1;
    for (int b0 = 0; b0 < nent; b0 += a.eb) {
      const int nb = min(a.eb, nent - b0);
      stage_entries<L>(a, p0, keys, b0, nb, crow, cs, ed, EF, s_sqrt_pref, tid, kCT);
      if (tid == 0) {  // row groups of this batch
        int ng = 0, prev = -1;
        for (int i = 0; i < nb; ++i) {
          const int row = (int)(keys[b0 + i] >> 32);
          if (row != prev) { s_gstart[ng++] = i; prev = row; }
        }
        s_gstart[ng] = nb;
        s_ng = ng;
      }
      compute_bar(kCT);
      const int ng = s_ng;
      for (int q = q0; q < Q; q += qstep) {
        for (int g = g0t; g < ng; g += gstep) {
          const int g0 = s_gstart[g], g1 = s_gstart[g + 1];
          const int row = (int)(keys[b0 + g0] >> 32);
          const bool cont = (g == 0 && row == last_row);  // continues from the previous batch
          float v[3][4];
          quad_values<L>(a, ed, EF, g0, g1, q, v);
          float* orow = obase + (size_t)row * 3 * F;
#pragma unroll
          for (int d = 0; d < 3; ++d) {
            float* p = orow + d * F + 4 * q;
            if (vec) {
              float4 w = make_float4(v[d][0], v[d][1], v[d][2], v[d][3]);
              if (cont) {
                const float4 o = __ldcg(reinterpret_cast<const float4*>(p));  // written by this CTA last batch
                w.x += o.x; w.y += o.y; w.z += o.z; w.w += o.w;
              }
              __stcs(reinterpret_cast<float4*>(p), w);
            } else {
              for (int k = 0; k < 4 && 4 * q + k < F; ++k) p[k] = cont ? __ldcg(p + k) + v[d][k] : v[d][k];
            }
          }
        }
      }
      last_row = (int)(keys[b0 + nb - 1] >> 32);
      compute_bar(kCT);  // staged entries are rewritten by the next batch
    }
  }
  // centre queue empty: this warp joins the zero-row stream
  if (vec) jac_zero_rows_tma(a, ztile, a.counter + 1);
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct JacLayout {
  int64_t counter, ent_cnt, ent, ent_tmp, bitmap, total;
};

static JacLayout jac_layout(int64_t n_centres, int64_t n_pairs, int64_t n_inc, int attach) {
  JacLayout L{};
  int64_t off = 0;
  auto take = [&](int64_t bytes) { const int64_t o = off; off = align_up(off + bytes, 256); return o; };
  L.counter = take(16);
  L.ent_cnt = take(4 * n_centres);
  L.ent = take(8 * (attach ? 2 : 1) * (n_pairs > 0 ? n_pairs : 1));
  L.ent_tmp = take(8 * (attach ? 2 : 1) * (n_pairs > 0 ? n_pairs : 1));
  L.bitmap = take(4 * ((n_centres * n_inc + 31) / 32));
  L.total = off;
  return L;
}

static int sm_count() {
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  return nsm;
}

template <int L>
struct JacDispatch {
  static int run(JacArgs a, cudaStream_t st) {
    using Sh = JacShape<L>;
    const int nsm = sm_count();
    // 1. entries + bitmap
    {
      const size_t smem = 8 * (size_t)a.cap;
      auto kern = k_jac_entries;
      int rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                          "entries smem attribute");
      if (rc) return rc;
      int occ = 1;
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem);
      int64_t blocks = (int64_t)nsm * (occ < 1 ? 1 : occ);
      if (blocks > a.n_centres) blocks = a.n_centres;
      kern<<<(unsigned)blocks, 256, smem, st>>>(a);
      if ((rc = check_launch("k_jac_entries"))) return rc;
    }
    // 2. one launch: in every block warp 0 streams zero rows, warps 1..7 compute
    int rc;
    const int EF = Sh::entry_floats(a.N, a.S, a.mode);
    const size_t base = kZeroTile + 4 * (size_t)Sh::cs_floats(a.N, a.S);
    const size_t budget = 56 * 1024;  // four CTAs per SM
    int eb = base < budget ? (int)((budget - base) / (4 * (size_t)EF)) : 0;
    eb = eb > 32 ? 32 : eb;
    if (eb < 4) eb = 4;
    a.eb = eb;
    const size_t smem = base + 4 * (size_t)eb * EF;
    if (smem > 220 * 1024) return set_error(SOAPB_ERR_UNSUPPORTED, "jacobian shared memory %zu B too large", smem);
    auto kern = k_jacobian<L>;
    rc = check_cuda(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem),
                    "jacobian smem attribute");
    if (rc) return rc;
    int occ = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kern, 256, smem);
    const int64_t blocks = (int64_t)nsm * (occ < 1 ? 1 : occ);
    kern<<<(unsigned)blocks, 256, smem, st>>>(a);
    return check_launch("k_jacobian");
  }
};

}  // namespace soapb

using namespace soapb;

extern "C" int soapb_jacobian_workspace(const soapb_basis* b, int64_t n_centres, int64_t n_pairs, int64_t n_inc,
                                        int32_t attach, int64_t* bytes) {
  if (!b || !bytes) return set_error(SOAPB_ERR_ARG, "null argument");
  if (n_centres < 0 || n_pairs < 0 || n_inc < 0) return set_error(SOAPB_ERR_ARG, "negative sizes");
  *bytes = jac_layout(n_centres, n_pairs, n_inc, attach).total;
  return SOAPB_OK;
}

extern "C" int soapb_jacobian(const soapb_basis* b, int64_t n_centres, const int64_t* d_pair_off, const void* d_pairs,
                              int64_t n_pairs, const float* d_coeff, const int32_t* d_inc_row, int64_t n_inc,
                              const int32_t* d_centre_atom, int32_t attach, int32_t max_pairs, int32_t out_mode,
                              float* d_out, void* d_work, int64_t work_bytes, int32_t* d_status, void* stream) {
  if (!b || !b->dev) return set_error(SOAPB_ERR_ARG, "basis not built");
  if (out_mode != SOAPB_OUT_PS && out_mode != SOAPB_OUT_CC) return set_error(SOAPB_ERR_ARG, "bad out_mode");
  if (n_centres <= 0 || n_inc <= 0) return SOAPB_OK;
  if (!d_pair_off || !d_coeff || !d_inc_row || !d_out || !d_status || !d_work)
    return set_error(SOAPB_ERR_ARG, "null argument");
  if (attach && !d_centre_atom) return set_error(SOAPB_ERR_ARG, "attach needs centre atoms");
  if (max_pairs < 0 || n_pairs < 0) return set_error(SOAPB_ERR_ARG, "bad pair counts");
  if (((uintptr_t)d_out) % 16) return set_error(SOAPB_ERR_ARG, "output must be 16-byte aligned");
  const JacLayout Lw = jac_layout(n_centres, n_pairs, n_inc, attach);
  if (work_bytes < Lw.total) return set_error(SOAPB_ERR_ARG, "jacobian workspace too small (%lld < %lld)",
                                              (long long)work_bytes, (long long)Lw.total);
  // shared-memory sort buffer of the entries kernel: the largest centre's entries, at most 8192
  // keys (64 KB); each centre with more entries takes the tiled merge in the workspace
  const int64_t need = (int64_t)(attach ? 2 : 1) * (max_pairs > 0 ? max_pairs : 1);
  int cap = 64;
  while (cap < need && cap < 8192) cap <<= 1;
  cudaStream_t st = (cudaStream_t)stream;
  char* w = (char*)d_work;
  JacArgs a;
  a.pair_off = d_pair_off;
  a.pairs = (const float4*)d_pairs;
  a.coeff = d_coeff;
  a.inc_row = d_inc_row;
  a.centre_atom = d_centre_atom;
  a.tab_b = (const float*)((const char*)b->dev + b->off_tab_b);
  a.tab_bh = (const float*)((const char*)b->dev + b->off_tab_bh);
  a.selfv = (const float*)((const char*)b->dev + b->off_self);
  a.ftab = (const int*)((const char*)b->dev + b->off_ftab);
  a.out = d_out;
  a.status = d_status;
  a.counter = (int*)(w + Lw.counter);
  a.ent_cnt = (int*)(w + Lw.ent_cnt);
  a.ent = (unsigned long long*)(w + Lw.ent);
  a.ent_tmp = (unsigned long long*)(w + Lw.ent_tmp);
  a.bitmap = (unsigned int*)(w + Lw.bitmap);
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
  a.ent_mult = attach ? 2 : 1;
  a.inv_h = (float)(1.0 / b->seg_width);
  int rc = check_cuda(cudaMemsetAsync(a.counter, 0, 16, st), "reset work counter");
  if (rc) return rc;
  rc = check_cuda(cudaMemsetAsync(a.bitmap, 0, 4 * ((n_centres * n_inc + 31) / 32), st), "clear row bitmap");
  if (rc) return rc;
  return dispatch_l<JacDispatch>(b->l_max, a, st);
}
