// Cell-list radius neighbour search into a per-centre CSR pair list.
//
// Reference: SOAP._build_neighbor_list (soap_generator.py:1128-1181),
// _radius_edges (:1042-1125), _extend_periodic (:1015-1021), _pbc_offsets
// (:382-396) and _perpendicular_lengths (:369-379).  The reference
// replicates every atom over all (2 n_rep + 1)^3 image offsets and runs an
// all-pairs GEMM distance test; here atoms are binned once per structure
// (counting sort into bins in the cell's fractional frame, periodic axes
// wrapped) and each centre scans only the bins of its window, generating
// images on the fly.  Diagonal frames use bins a quarter of the cutoff wide
// and a window trimmed to the cutoff sphere (visit_fine); other frames use
// bins of perpendicular width >= half the cutoff and a +-2 window (visit).  The image set is
// the reference's: image offset n = T - w_atom + w_centre (T the cell-window
// shift, w the wrap shifts) must satisfy |n_i| <= n_rep_i on periodic axes.
//
// Pairs of a centre are written sorted by (neighbour species, radial table
// segment) -- the order the descriptor kernels consume them in -- and, inside
// a key, in a deterministic candidate order (bins are sorted by atom index).
// Distances are tested and differences taken in FP64; rvec is stored FP32.
#include <math.h>

#include <mutex>

#include "common.cuh"

namespace soapb {

struct GridDesc {
  double H[9];     // rows: lattice a, b, c (identity for non-periodic structures)
  double Hinv[9];  // f_j = sum_i x_i Hinv[i*3+j]
  double fmin[3];  // bin origin in fractional coordinates (non-periodic axes)
  double binw[3];  // fractional bin width
  int nb[3], win[3], nrep[3], per[3];
  int any_per;
  int orth;  // diagonal frame (every non-periodic structure, rectangular cells): sphere-trimmed enumeration
};

struct NLWork {
  GridDesc* grids;
  unsigned long long* fbox;  // (n_struct, 6) ordered-int encodings of fractional min/max
  int* bins_per_struct;      // (n_struct)
  int64_t* bin_off;          // (n_struct + 1)
  int* bin_count;            // (max_bins)
  int64_t* bin_start;        // (max_bins + 1)
  int* bin_cursor;           // (max_bins)
  int* atom_bin;             // (n_atoms)
  int* sorted_atom;          // (n_atoms)
  double4* sorted_pos;       // (n_atoms) {wrapped x, y, z, packed info} (see pack_info)
  double4* cpos;             // (n_centres) wrapped centre positions
  int4* cinfo;               // (n_centres) {bin xyz, struct, wrap, atom}
  int* counts;               // (n_centres)
  int64_t* partials;         // scan partials
  int* status;               // error flags
  int64_t max_bins;
};

// ---------------------------------------------------------------------------
// helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ unsigned long long ord_encode(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b >> 63) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double ord_decode(unsigned long long e) {
  unsigned long long b = (e >> 63) ? (e & 0x7fffffffffffffffull) : ~e;
#ifdef __CUDA_ARCH__
  return __longlong_as_double((long long)b);
#else
  double d;
  memcpy(&d, &b, 8);
  return d;
#endif
}

__device__ __forceinline__ int pack3(int a, int b, int c) { return (a + 512) | ((b + 512) << 10) | ((c + 512) << 20); }
__device__ __forceinline__ void unpack3(int p, int (&v)[3]) {
  v[0] = (p & 1023) - 512;
  v[1] = ((p >> 10) & 1023) - 512;
  v[2] = ((p >> 20) & 1023) - 512;
}
// atom (27 bits) | species (5 bits) | packed wrap shifts (30 bits), carried in
// the fourth double of a sorted-atom record so a candidate is one 32-byte load
// (the bits are only moved, never used as a floating-point value).
__device__ __forceinline__ double pack_info(int atom, int sp, int wrap) {
  const unsigned long long bits = (unsigned long long)(unsigned)atom | ((unsigned long long)(unsigned)sp << kAtomBits) |
                                  ((unsigned long long)(unsigned)wrap << 32);
  return __longlong_as_double((long long)bits);
}
__device__ __forceinline__ void unpack_info(double w, int& atom, int& sp, int& wrap) {
  const unsigned long long bits = (unsigned long long)__double_as_longlong(w);
  atom = (int)(bits & kAtomMask);
  sp = (int)((bits >> kAtomBits) & 31u);
  wrap = (int)(bits >> 32);
}
__device__ __forceinline__ int floordiv(int a, int b) { return (a >= 0) ? a / b : -((-a + b - 1) / b); }

__device__ __forceinline__ int struct_of_atom(const int64_t* atom_off, int n_struct, int64_t a) {
  int lo = 0, hi = n_struct - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (atom_off[mid] <= a) lo = mid; else hi = mid - 1;
  }
  return lo;
}

__device__ __forceinline__ void to_frac(const GridDesc& g, double x, double y, double z, double (&f)[3]) {
#pragma unroll
  for (int j = 0; j < 3; ++j) f[j] = x * g.Hinv[j] + y * g.Hinv[3 + j] + z * g.Hinv[6 + j];
}

// Bin, wrap shift and wrapped position of a point of structure g.
__device__ __forceinline__ bool locate(const GridDesc& g, double x, double y, double z, int (&b)[3], int (&w)[3],
                                       double (&wp)[3]) {
  double f[3];
  to_frac(g, x, y, z, f);
  bool ok = true;
#pragma unroll
  for (int i = 0; i < 3; ++i) {
    if (g.per[i]) {
      const double fl = floor(f[i]);
      w[i] = (int)fl;
      double fr = f[i] - fl;
      int bi = (int)(fr * g.nb[i]);
      b[i] = min(max(bi, 0), g.nb[i] - 1);
      ok &= (w[i] > -512 && w[i] < 511);
    } else {
      w[i] = 0;
      const int bi = (int)floor((f[i] - g.fmin[i]) / g.binw[i]);
      b[i] = min(max(bi, 0), g.nb[i] - 1);
    }
  }
  wp[0] = x - (w[0] * g.H[0] + w[1] * g.H[3] + w[2] * g.H[6]);
  wp[1] = y - (w[0] * g.H[1] + w[1] * g.H[4] + w[2] * g.H[7]);
  wp[2] = z - (w[0] * g.H[2] + w[1] * g.H[5] + w[2] * g.H[8]);
  return ok;
}

// ---------------------------------------------------------------------------
// exclusive scan int32 -> int64 (n + 1 outputs)
// ---------------------------------------------------------------------------

__device__ __forceinline__ int64_t block_incl_scan(int64_t v, int64_t* s_warp) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
  for (int o = 1; o < 32; o <<= 1) {
    const int64_t t = __shfl_up_sync(0xffffffffu, v, o);
    if (lane >= o) v += t;
  }
  if (lane == 31) s_warp[warp] = v;
  __syncthreads();
  if (warp == 0) {
    int64_t w = (lane < (int)(blockDim.x >> 5)) ? s_warp[lane] : 0;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int64_t t = __shfl_up_sync(0xffffffffu, w, o);
      if (lane >= o) w += t;
    }
    s_warp[lane] = w;
  }
  __syncthreads();
  if (warp > 0) v += s_warp[warp - 1];
  return v;
}

__global__ void __launch_bounds__(1024) k_scan_blocks(const int* in, int64_t n, int64_t* out, int64_t* partials) {
  __shared__ int64_t s_warp[32];
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  const int64_t v = (i < n) ? in[i] : 0;
  const int64_t inc = block_incl_scan(v, s_warp);
  if (i < n) out[i] = inc - v;
  if (threadIdx.x == blockDim.x - 1) partials[blockIdx.x] = inc;
}

__global__ void __launch_bounds__(1024) k_scan_partials(int64_t* partials, int64_t nblk, int64_t* total_out) {
  __shared__ int64_t s_warp[32];
  __shared__ int64_t s_carry;
  if (threadIdx.x == 0) s_carry = 0;
  __syncthreads();
  for (int64_t base = 0; base < nblk; base += blockDim.x) {
    const int64_t i = base + threadIdx.x;
    const int64_t v = (i < nblk) ? partials[i] : 0;
    const int64_t inc = block_incl_scan(v, s_warp);
    const int64_t carry = s_carry;
    if (i < nblk) partials[i] = carry + inc - v;
    __syncthreads();
    if (threadIdx.x == blockDim.x - 1) s_carry = carry + inc;
    __syncthreads();
  }
  if (threadIdx.x == 0) *total_out = s_carry;
}

__global__ void k_scan_add(int64_t* out, int64_t n, const int64_t* partials) {
  const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] += partials[i / 1024];
}

static int exclusive_scan(const int* in, int64_t n, int64_t* out, int64_t* partials, cudaStream_t st) {
  const int64_t nblk = (n + 1023) / 1024;
  if (n > 0) {
    k_scan_blocks<<<(unsigned)nblk, 1024, 0, st>>>(in, n, out, partials);
  }
  k_scan_partials<<<1, 1024, 0, st>>>(partials, nblk, out + n);
  if (n > 0) k_scan_add<<<(unsigned)((n + 255) / 256), 256, 0, st>>>(out, n, partials);
  return check_launch("exclusive_scan", n > 0 ? 3 : 1);
}

// ---------------------------------------------------------------------------
// cell lists
// ---------------------------------------------------------------------------

__global__ void k_grid_init(soapb_structs s, NLWork w, double cutoff) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n_struct) return;
  GridDesc g;
  int anyp = 0;
  for (int k = 0; k < 3; ++k) anyp |= s.d_pbc[i * 3 + k] ? 1 : 0;
  for (int k = 0; k < 9; ++k) g.H[k] = anyp ? s.d_cells[i * 9 + k] : ((k % 4 == 0) ? 1.0 : 0.0);
  const double* H = g.H;
  const double det = H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) +
                     H[2] * (H[3] * H[7] - H[4] * H[6]);
  int bad = fabs(det) < 1e-300;
  const double id = bad ? 0.0 : 1.0 / det;
  // inverse of the row-vector matrix: x = f H  =>  f = x H^-1
  g.Hinv[0] = (H[4] * H[8] - H[5] * H[7]) * id;
  g.Hinv[1] = (H[2] * H[7] - H[1] * H[8]) * id;
  g.Hinv[2] = (H[1] * H[5] - H[2] * H[4]) * id;
  g.Hinv[3] = (H[5] * H[6] - H[3] * H[8]) * id;
  g.Hinv[4] = (H[0] * H[8] - H[2] * H[6]) * id;
  g.Hinv[5] = (H[2] * H[3] - H[0] * H[5]) * id;
  g.Hinv[6] = (H[3] * H[7] - H[4] * H[6]) * id;
  g.Hinv[7] = (H[1] * H[6] - H[0] * H[7]) * id;
  g.Hinv[8] = (H[0] * H[4] - H[1] * H[3]) * id;
  for (int k = 0; k < 3; ++k) {
    g.per[k] = anyp ? (s.d_pbc[i * 3 + k] ? 1 : 0) : 0;
    g.fmin[k] = 0.0;
    g.binw[k] = 1.0;
    g.nb[k] = 1;
    g.win[k] = 1;
    g.nrep[k] = 0;
  }
  g.any_per = anyp;
  g.orth = 1;
  for (int k = 0; k < 9; ++k)
    if (k % 4 == 0 ? !(H[k] > 0.0) : H[k] != 0.0) g.orth = 0;
  // perpendicular widths |det| / |cross of the other two rows| (SG:369-379)
  double perp[3];
  for (int k = 0; k < 3; ++k) {
    const double* u = H + 3 * ((k + 1) % 3);
    const double* v = H + 3 * ((k + 2) % 3);
    const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
    perp[k] = fabs(det) / (sqrt(cx * cx + cy * cy + cz * cz) + 1e-12);
    if (g.per[k]) g.nrep[k] = (int)ceil(cutoff / (perp[k] + 1e-12));  // SG:389
  }
  w.grids[i] = g;
  for (int k = 0; k < 3; ++k) {
    w.fbox[i * 6 + k] = ord_encode(INFINITY);
    w.fbox[i * 6 + 3 + k] = ord_encode(-INFINITY);
  }
  if (bad && anyp) atomicOr(w.status, 1);
}

// Fractional bounding box per structure.  Atoms of a structure are
// contiguous, so a warp usually covers one structure: it reduces min / max
// with shuffles and issues one atomic per bound instead of 32.
__global__ void k_frac_bbox(soapb_structs s, NLWork w) {
  const int lane = threadIdx.x & 31;
  const int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t base = (int64_t)blockIdx.x * blockDim.x + (threadIdx.x & ~31); base < s.n_atoms; base += stride) {
    const int64_t a = base + lane;
    const bool valid = a < s.n_atoms;
    int si = 0;
    double f[3] = {0.0, 0.0, 0.0};
    if (valid) {
      si = struct_of_atom(s.d_atom_off, s.n_struct, a);
      to_frac(w.grids[si], s.d_positions[3 * a], s.d_positions[3 * a + 1], s.d_positions[3 * a + 2], f);
    }
    const int si0 = __shfl_sync(0xffffffffu, si, 0);  // lane 0 is always valid here
    if (__all_sync(0xffffffffu, !valid || si == si0)) {
      const GridDesc& g = w.grids[si0];
      for (int k = 0; k < 3; ++k) {
        if (g.per[k]) continue;
        double lo = valid ? f[k] : INFINITY, hi = valid ? f[k] : -INFINITY;
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) {
          lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
          hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
        }
        if (lane == 0) {
          atomicMin(&w.fbox[si0 * 6 + k], ord_encode(lo));
          atomicMax(&w.fbox[si0 * 6 + 3 + k], ord_encode(hi));
        }
      }
    } else if (valid) {
      const GridDesc& g = w.grids[si];
      for (int k = 0; k < 3; ++k) {
        if (g.per[k]) continue;
        atomicMin(&w.fbox[si * 6 + k], ord_encode(f[k]));
        atomicMax(&w.fbox[si * 6 + 3 + k], ord_encode(f[k]));
      }
    }
  }
}

__global__ void k_grid_setup(soapb_structs s, NLWork w, double cutoff) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= s.n_struct) return;
  GridDesc g = w.grids[i];
  const double* H = g.H;
  const double det = fabs(H[0] * (H[4] * H[8] - H[5] * H[7]) - H[1] * (H[3] * H[8] - H[5] * H[6]) +
                          H[2] * (H[3] * H[7] - H[4] * H[6]));
  double perp[3];
  for (int k = 0; k < 3; ++k) {
    const double* u = H + 3 * ((k + 1) % 3);
    const double* v = H + 3 * ((k + 2) % 3);
    const double cx = u[1] * v[2] - u[2] * v[1], cy = u[2] * v[0] - u[0] * v[2], cz = u[0] * v[1] - u[1] * v[0];
    perp[k] = det / (sqrt(cx * cx + cy * cy + cz * cz) + 1e-300);
  }
  const int64_t A = s.d_atom_off[i + 1] - s.d_atom_off[i];
  // Diagonal frames: bins of width >= cutoff / 4, each window row trimmed to
  // the cutoff sphere (visit_fine), unless a periodic x axis would get fewer
  // than 3 bins (a row of the window would wrap into more than 4 runs).
  // Other frames: bins of perpendicular width >= cutoff / 2 and the full
  // +-2 window: 5^3 half-width bins hold 15.6 cutoff^3 of candidates against
  // 27 cutoff^3 for full-width bins.
  if (g.orth && g.per[0] && perp[0] < 0.75 * cutoff) g.orth = 0;
  const double bin_min = (g.orth ? 0.25 : 0.5) * cutoff;
  for (int k = 0; k < 3; ++k) {
    if (g.per[k]) {
      const int nb = (int)floor(perp[k] / bin_min);
      g.nb[k] = min(max(nb, 1), 1023);
      g.fmin[k] = 0.0;
      g.binw[k] = 1.0 / g.nb[k];
    } else {
      double lo = ord_decode(w.fbox[i * 6 + k]), hi = ord_decode(w.fbox[i * 6 + 3 + k]);
      if (!(hi >= lo)) { lo = 0.0; hi = 0.0; }  // no atoms
      const double span = hi - lo;
      const int nb = (int)floor(span * perp[k] / bin_min);
      g.nb[k] = min(max(nb, 1), 1023);
      g.fmin[k] = lo;
      g.binw[k] = span > 0.0 ? span / g.nb[k] : 1.0;
    }
  }
  // cap the bin count of the structure at 2 A + 8
  const int64_t cap = 2 * A + 8;
  while ((int64_t)g.nb[0] * g.nb[1] * g.nb[2] > cap) {
    int k = 0;
    if (g.nb[1] > g.nb[k]) k = 1;
    if (g.nb[2] > g.nb[k]) k = 2;
    const double span = g.binw[k] * g.nb[k];
    g.nb[k] = max(1, g.nb[k] / 2);
    g.binw[k] = span / g.nb[k];
  }
  if (g.orth && g.per[0] && g.nb[0] < 3) g.orth = 0;
  for (int k = 0; k < 3; ++k) {
    const double bw_perp = g.binw[k] * perp[k];  // perpendicular width of one bin
    int win = (int)ceil(cutoff / bw_perp);
    if (!(bw_perp > 0.0)) win = 1;
    if (!g.per[k]) win = min(win, g.nb[k]);
    g.win[k] = max(win, 1);
  }
  w.grids[i] = g;
  w.bins_per_struct[i] = g.nb[0] * g.nb[1] * g.nb[2];
}

__global__ void k_bin_atoms(soapb_structs s, NLWork w) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < s.n_atoms;
       a += (int64_t)gridDim.x * blockDim.x) {
    const int si = struct_of_atom(s.d_atom_off, s.n_struct, a);
    const GridDesc& g = w.grids[si];
    int b[3], wr[3];
    double wp[3];
    if (!locate(g, s.d_positions[3 * a], s.d_positions[3 * a + 1], s.d_positions[3 * a + 2], b, wr, wp))
      atomicOr(w.status, 2);
    const int64_t gb = w.bin_off[si] + ((int64_t)b[2] * g.nb[1] + b[1]) * g.nb[0] + b[0];
    w.atom_bin[a] = (int)gb;
    atomicAdd(&w.bin_count[gb], 1);
  }
}

__global__ void k_scatter_atoms(int64_t n_atoms, NLWork w) {
  for (int64_t a = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; a < n_atoms;
       a += (int64_t)gridDim.x * blockDim.x) {
    const int gb = w.atom_bin[a];
    const int64_t slot = w.bin_start[gb] + atomicAdd(&w.bin_cursor[gb], 1);
    w.sorted_atom[slot] = (int)a;
  }
}

// Sort each bin's atoms by index (warp bitonic sort in shared memory), so
// the candidate order -- and the FP32 accumulation order -- is deterministic.
__global__ void __launch_bounds__(128) k_sort_bins(NLWork w) {
  __shared__ int s_keys[4][1024];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  int* keys = s_keys[wid];
  const int64_t nwarps = (int64_t)gridDim.x * 4;
  for (int64_t b = (int64_t)blockIdx.x * 4 + wid; b < w.max_bins; b += nwarps) {
    const int64_t s0 = w.bin_start[b], s1 = w.bin_start[b + 1];
    const int n = (int)(s1 - s0);
    if (n <= 1) continue;
    if (n > 1024) {  // rare fallback: insertion sort by one lane
      if (lane == 0) {
        int* p = w.sorted_atom + s0;
        for (int i = 1; i < n; ++i) {
          const int v = p[i];
          int j = i - 1;
          while (j >= 0 && p[j] > v) { p[j + 1] = p[j]; --j; }
          p[j + 1] = v;
        }
      }
      __syncwarp();
      continue;
    }
    int n2 = 1;
    while (n2 < n) n2 <<= 1;
    for (int i = lane; i < n2; i += 32) keys[i] = (i < n) ? w.sorted_atom[s0 + i] : 0x7fffffff;
    __syncwarp();
    for (int k = 2; k <= n2; k <<= 1)
      for (int j = k >> 1; j > 0; j >>= 1) {
        for (int i = lane; i < n2; i += 32) {
          const int ixj = i ^ j;
          if (ixj > i) {
            const int a = keys[i], c = keys[ixj];
            const bool asc = (i & k) == 0;
            if (asc ? (a > c) : (a < c)) { keys[i] = c; keys[ixj] = a; }
          }
        }
        __syncwarp();
      }
    for (int i = lane; i < n; i += 32) w.sorted_atom[s0 + i] = keys[i];
    __syncwarp();
  }
}

__global__ void k_gather_atoms(soapb_structs s, NLWork w) {
  for (int64_t slot = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; slot < s.n_atoms;
       slot += (int64_t)gridDim.x * blockDim.x) {
    const int a = w.sorted_atom[slot];
    const int si = struct_of_atom(s.d_atom_off, s.n_struct, a);
    const GridDesc& g = w.grids[si];
    int b[3], wr[3];
    double wp[3];
    locate(g, s.d_positions[3 * (int64_t)a], s.d_positions[3 * (int64_t)a + 1], s.d_positions[3 * (int64_t)a + 2],
           b, wr, wp);
    w.sorted_pos[slot] = make_double4(wp[0], wp[1], wp[2], pack_info((int)a, s.d_species[a], pack3(wr[0], wr[1], wr[2])));
  }
}

__global__ void k_centres(soapb_structs s, soapb_centres c, NLWork w) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < c.n_centres;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int si = c.d_struct[i];
    const GridDesc& g = w.grids[si];
    int b[3], wr[3];
    double wp[3];
    if (!locate(g, c.d_xyz[3 * i], c.d_xyz[3 * i + 1], c.d_xyz[3 * i + 2], b, wr, wp)) atomicOr(w.status, 2);
    w.cpos[i] = make_double4(wp[0], wp[1], wp[2], 0.0);
    w.cinfo[i] = make_int4(b[0] | (b[1] << 10) | (b[2] << 20), si, pack3(wr[0], wr[1], wr[2]), c.d_atom[i]);
  }
}

// ---------------------------------------------------------------------------
// candidate enumeration (warp-synchronous; one warp per centre)
// ---------------------------------------------------------------------------

struct VisitArgs {
  const GridDesc* grids;
  const int64_t* bin_off;
  const int64_t* bin_start;
  const double4* sorted_pos;
  const double4* cpos;
  const int4* cinfo;
  int* status;
  double cutoff, cutoff2;
  int mode;
};

template <class Fn>
__device__ __forceinline__ void visit(const VisitArgs& A, int64_t c, Fn&& fn) {
  const int lane = threadIdx.x & 31;
  const double4 cp = A.cpos[c];
  const int4 ci = A.cinfo[c];
  const GridDesc& g = A.grids[ci.y];
  const int cb[3] = {ci.x & 1023, (ci.x >> 10) & 1023, (ci.x >> 20) & 1023};
  int cw[3];
  unpack3(ci.z, cw);
  const int64_t boff = A.bin_off[ci.y];
  for (int dz = -g.win[2]; dz <= g.win[2]; ++dz) {
    int bz = cb[2] + dz, Tz = 0;
    if (g.per[2]) { Tz = floordiv(bz, g.nb[2]); bz -= Tz * g.nb[2]; }
    else if (bz < 0 || bz >= g.nb[2]) continue;
    for (int dy = -g.win[1]; dy <= g.win[1]; ++dy) {
      int by = cb[1] + dy, Ty = 0;
      if (g.per[1]) { Ty = floordiv(by, g.nb[1]); by -= Ty * g.nb[1]; }
      else if (by < 0 || by >= g.nb[1]) continue;
      // the row's x bins as runs of consecutive bins with one image shift Tx:
      // a run is one contiguous range of bin-sorted atoms
      int dx = -g.win[0];
      while (dx <= g.win[0]) {
        int bx = cb[0] + dx, Tx = 0, run_end;
        if (g.per[0]) {
          Tx = floordiv(bx, g.nb[0]);
          bx -= Tx * g.nb[0];
          run_end = min(g.win[0], dx + (g.nb[0] - 1 - bx));
        } else {
          if (bx < 0) { dx = -cb[0]; continue; }
          if (bx >= g.nb[0]) break;
          run_end = min(g.win[0], g.nb[0] - 1 - cb[0]);
        }
        const int bx1 = bx + (run_end - dx);
        dx = run_end + 1;
        const double sx = Tx * g.H[0] + Ty * g.H[3] + Tz * g.H[6] - cp.x;
        const double sy = Tx * g.H[1] + Ty * g.H[4] + Tz * g.H[7] - cp.y;
        const double sz = Tx * g.H[2] + Ty * g.H[5] + Tz * g.H[8] - cp.z;
        const int T[3] = {Tx, Ty, Tz};
        const int64_t gb = boff + ((int64_t)bz * g.nb[1] + by) * g.nb[0];
        const int64_t s0 = A.bin_start[gb + bx], s1 = A.bin_start[gb + bx1 + 1];
        for (int64_t base = s0; base < s1; base += 32) {
          const int64_t i = base + lane;
          bool ok = false;
          int atom = 0, sp = 0;
          double rx = 0.0, ry = 0.0, rz = 0.0, r2 = 0.0;
          if (i < s1) {
            const double4 p = A.sorted_pos[i];
            int wrap;
            unpack_info(p.w, atom, sp, wrap);
            rx = p.x + sx;
            ry = p.y + sy;
            rz = p.z + sz;
            r2 = rx * rx + ry * ry + rz * rz;
            ok = r2 <= A.cutoff2;
            if (ok && g.any_per) {
              int aw[3];
              unpack3(wrap, aw);
#pragma unroll
              for (int k = 0; k < 3; ++k)
                if (g.per[k]) ok &= abs(T[k] - aw[k] + cw[k]) <= g.nrep[k];
            }
            // create(): drop r <= 1e-12 edges except the centre's own atom (SG:1171-1179)
            if (ok && A.mode == SOAPB_NL_CREATE && r2 <= 1e-24 && atom != ci.w) ok = false;
          }
          fn(ok, atom, sp, rx, ry, rz, r2);
        }
      }
    }
  }
}

// Sphere-trimmed enumeration for diagonal frames (x = f diag(L)): the rows
// (bz, by) of unwrapped bins whose slab comes within the cutoff of the
// centre, each trimmed to the bins x that the sphere's cross-section reaches
// (conservatively: the cutoff plus 1e-8 A).  Up to 32 rows are laid out at a
// time, one per lane; a row's x bins are at most 4 runs of contiguous
// bin-sorted atoms (periodic x axes have >= 3 bins).  The runs of the 32 rows
// form one candidate stream that all lanes walk 32 at a time: a lane finds
// its run from the run starts inside its tile (one OR-reduction and a
// popcount).  Candidate order: z rows, then y, then x, then atom index --
// deterministic, like the full window's.  PIPE: the candidate records of the
// next tile are looked up and loaded while this tile is tested (the fill,
// whose per-candidate work covers the load; the count, which has little work
// per candidate, runs more warps instead).
constexpr int kRunsPerPass = 128;  // 32 rows x at most 4 runs

template <bool PIPE, class Fn>
__device__ __forceinline__ void visit_fine(const VisitArgs& A, int64_t c, int* runs, Fn&& fn) {
  const int lane = threadIdx.x & 31;
  const double4 cp = A.cpos[c];
  const int4 ci = A.cinfo[c];
  const GridDesc& g = A.grids[ci.y];
  int cw[3];
  unpack3(ci.z, cw);
  const int64_t boff = A.bin_off[ci.y];
  const double cm = A.cutoff + 1e-8;
  const double Lv[3] = {g.H[0], g.H[4], g.H[8]};
  const double cv[3] = {cp.x, cp.y, cp.z};
  // bin coordinate u = x / (L binw) - fmin / binw (reciprocals: the 1e-8 A margin covers the rounding)
  const double ib[3] = {1.0 / (Lv[0] * g.binw[0]), 1.0 / (Lv[1] * g.binw[1]), 1.0 / (Lv[2] * g.binw[2])};
  const double ub[3] = {g.fmin[0] / g.binw[0], g.fmin[1] / g.binw[1], g.fmin[2] / g.binw[2]};
  // unwrapped bins of axis k that meet [x0, x1] (clamped to the grid on open axes)
  auto brange = [&](int k, double x0, double x1, int& lo, int& hi) {
    double u0 = fma(x0, ib[k], -ub[k]), u1 = fma(x1, ib[k], -ub[k]);
    if (!g.per[k]) {
      u0 = fmin(fmax(u0, -1.0), (double)g.nb[k]);
      u1 = fmin(fmax(u1, -1.0), (double)g.nb[k]);
    }
    lo = (int)floor(u0);
    hi = (int)floor(u1);
    if (!g.per[k]) {
      lo = max(lo, 0);
      hi = min(hi, g.nb[k] - 1);
    }
  };
  // distance from the centre to the slab of unwrapped bin b on axis k
  auto dmin = [&](int k, int b) {
    const double lo = (g.fmin[k] + b * g.binw[k]) * Lv[k], hi = (g.fmin[k] + (b + 1) * g.binw[k]) * Lv[k];
    return fmax(0.0, fmax(lo - cv[k], cv[k] - hi));
  };
  int bz0, bz1, by0, by1;
  brange(2, cp.z - cm, cp.z + cm, bz0, bz1);
  brange(1, cp.y - cm, cp.y + cm, by0, by1);
  const int ny = by1 - by0 + 1, nz = bz1 - bz0 + 1;
  const int nrows = (ny > 0 && nz > 0) ? ny * nz : 0;
  int* r_start = runs;
  int* r_s0 = runs + kRunsPerPass;
  int* r_T = runs + 2 * kRunsPerPass;
  for (int p0 = 0; p0 < nrows; p0 += 32) {
    // this lane's row and its x runs (slots with len 0 are unused)
    const int row = p0 + lane;
    int rs0[4], rlen[4], rT[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) { rs0[q] = 0; rlen[q] = 0; rT[q] = 0; }
    if (row < nrows) {
      const int bz = bz0 + row / ny, by = by0 + row % ny;
      const double dy = dmin(1, by), dz = dmin(2, bz), d2 = dy * dy + dz * dz;
      if (d2 <= cm * cm) {
        const double ext = sqrt(cm * cm - d2);
        int bx0, bx1;
        brange(0, cp.x - ext, cp.x + ext, bx0, bx1);
        int Ty = 0, byw = by, Tz = 0, bzw = bz;
        if (g.per[1]) { Ty = floordiv(by, g.nb[1]); byw = by - Ty * g.nb[1]; }
        if (g.per[2]) { Tz = floordiv(bz, g.nb[2]); bzw = bz - Tz * g.nb[2]; }
        const int64_t gb = boff + ((int64_t)bzw * g.nb[1] + byw) * g.nb[0];
        int bx = bx0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (bx <= bx1) {
            int Tx = 0, lx = bx, rend = bx1;
            if (g.per[0]) {
              Tx = floordiv(bx, g.nb[0]);
              lx = bx - Tx * g.nb[0];
              rend = min(bx1, bx + (g.nb[0] - 1 - lx));
            }
            const int64_t s0 = A.bin_start[gb + lx], s1 = A.bin_start[gb + lx + (rend - bx) + 1];
            rs0[q] = (int)s0;
            rlen[q] = (int)(s1 - s0);
            rT[q] = pack3(Tx, Ty, Tz);
            bx = rend + 1;
          }
        }
        if (bx <= bx1) atomicOr(A.status, 8);  // more than 4 runs: cannot happen with >= 3 bins on x
      }
    }
    int nr = 0, cnt = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      nr += rlen[q] > 0;
      cnt += rlen[q];
    }
    int nr_inc = nr, cnt_inc = cnt;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int a = __shfl_up_sync(0xffffffffu, nr_inc, o), b = __shfl_up_sync(0xffffffffu, cnt_inc, o);
      if (lane >= o) {
        nr_inc += a;
        cnt_inc += b;
      }
    }
    const int nruns = __shfl_sync(0xffffffffu, nr_inc, 31), total = __shfl_sync(0xffffffffu, cnt_inc, 31);
    {
      int slot = nr_inc - nr, start = cnt_inc - cnt;
#pragma unroll
      for (int q = 0; q < 4; ++q)
        if (rlen[q] > 0) {
          r_start[slot] = start;
          r_s0[slot] = rs0[q];
          r_T[slot] = rT[q];
          start += rlen[q];
          ++slot;
        }
    }
    __syncwarp();
    // the run of each lane's position in the tile at k0, given the run rb of the position
    // before the tile; returns the run of the tile's last position
    auto lookup = [&](int k0, int rb, int& run) {
      const int idx = rb + 1 + lane;
      const int pos = (idx < nruns) ? r_start[idx] - k0 : 32;
      const unsigned mask = __reduce_or_sync(0xffffffffu, (pos >= 0 && pos < 32) ? (1u << pos) : 0u);
      run = rb + __popc(mask & ((2u << lane) - 1u));
      return __shfl_sync(0xffffffffu, run, 31);
    };
    auto load = [&](int k, int run) { return A.sorted_pos[(int64_t)r_s0[run] + (k - r_start[run])]; };
    const double4 zero4 = make_double4(0.0, 0.0, 0.0, 0.0);
    int rb = -1;  // run of the position before the tile
    int run_n = 0;
    double4 rec_n = zero4;
    if constexpr (PIPE) {
      rb = lookup(0, -1, run_n);
      if (lane < total) rec_n = load(lane, run_n);
    }
    for (int k0 = 0; k0 < total; k0 += 32) {
      const int k = k0 + lane;
      int run;
      double4 p = zero4;
      if constexpr (PIPE) {
        run = run_n;
        p = rec_n;
        rec_n = zero4;
        if (k0 + 32 < total) {
          rb = lookup(k0 + 32, rb, run_n);
          if (k + 32 < total) rec_n = load(k + 32, run_n);
        }
      } else {
        rb = lookup(k0, rb, run);
        if (k < total) p = load(k, run);
      }
      bool ok = false;
      int atom = 0, sp = 0;
      double rx = 0.0, ry = 0.0, rz = 0.0, r2 = 0.0;
      if (k < total) {
        int wrap;
        unpack_info(p.w, atom, sp, wrap);
        if (!g.any_per) {  // open structure: no image shifts (warp-uniform)
          rx = p.x - cp.x;
          ry = p.y - cp.y;
          rz = p.z - cp.z;
          r2 = rx * rx + ry * ry + rz * rz;
          ok = r2 <= A.cutoff2;
        } else {
          int T[3];
          unpack3(r_T[run], T);
          rx = p.x + (T[0] * Lv[0] - cp.x);
          ry = p.y + (T[1] * Lv[1] - cp.y);
          rz = p.z + (T[2] * Lv[2] - cp.z);
          r2 = rx * rx + ry * ry + rz * rz;
          ok = r2 <= A.cutoff2;
          if (ok) {
            int aw[3];
            unpack3(wrap, aw);
#pragma unroll
            for (int kk = 0; kk < 3; ++kk)
              if (g.per[kk]) ok &= abs(T[kk] - aw[kk] + cw[kk]) <= g.nrep[kk];
          }
        }
        if (ok && A.mode == SOAPB_NL_CREATE && r2 <= 1e-24 && atom != ci.w) ok = false;
      }
      fn(ok, atom, sp, rx, ry, rz, r2);
    }
    __syncwarp();  // the next pass rewrites the run table
  }
}

// The enumeration for the centre's structure: sphere-trimmed for diagonal
// frames, the full window otherwise (runs: kRunsPerPass * 3 ints of the warp's shared memory).
template <bool PIPE = false, class Fn>
__device__ __forceinline__ void visit_any(const VisitArgs& A, int64_t c, int* runs, Fn&& fn) {
  if (A.grids[A.cinfo[c].y].orth) visit_fine<PIPE>(A, c, runs, fn);
  else visit(A, c, fn);
}

// 8 blocks of 4 warps per SM (64 registers): the count is latency-bound with
// little work per candidate, so more resident warps pay more than pipelining.
__global__ void __launch_bounds__(128, 8) k_count(VisitArgs A, int64_t n_centres, int* counts) {
  __shared__ int s_runs[4][3 * kRunsPerPass];
  const int lane = threadIdx.x & 31;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); c < n_centres; c += nw) {
    int cnt = 0;
    visit_any(A, c, s_runs[threadIdx.x >> 5], [&](bool ok, int, int, double, double, double, double) {
      cnt += __popc(__ballot_sync(0xffffffffu, ok));
    });
    if (lane == 0) counts[c] = cnt;
  }
}

constexpr int kFillStage = 512;  // pairs per centre collected in shared memory

// Fill: one warp per centre.  The centre's accepted candidates are collected
// in shared memory in candidate order (one enumeration), then placed by a
// stable counting sort on the key (species, radial segment) and written to the
// centre's CSR slice.  A centre with more than kFillStage pairs enumerates
// twice instead (histogram, then scatter).  Either way the order is: by key,
// and by candidate order within a key.  The key is recomputed from the FP32
// pair record whenever it is needed (the radius and segment the descriptor
// kernels compute), so no key array takes shared memory.
__global__ void __launch_bounds__(128) k_fill(VisitArgs A, int64_t n_centres, const int64_t* pair_off, float4* pairs,
                                              int64_t capacity, int nseg, float inv_h, int nkeys, int* status) {
  extern __shared__ __align__(16) unsigned char s_raw[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  float4* stage = reinterpret_cast<float4*>(s_raw) + (size_t)wid * kFillStage;
  int* hist = reinterpret_cast<int*>(reinterpret_cast<float4*>(s_raw) + (size_t)(blockDim.x >> 5) * kFillStage) +
              (size_t)wid * nkeys;
  int* runs = reinterpret_cast<int*>(reinterpret_cast<float4*>(s_raw) + (size_t)(blockDim.x >> 5) * kFillStage) +
              (size_t)(blockDim.x >> 5) * nkeys + (size_t)wid * 3 * kRunsPerPass;
  const int64_t nw = (int64_t)gridDim.x * (blockDim.x >> 5);
  if (pair_off[n_centres] > capacity) {
    if (threadIdx.x == 0 && blockIdx.x == 0) atomicOr(status, 4);
    return;
  }
  auto record = [](int atom, int sp, double rx, double ry, double rz) {
    return make_float4((float)rx, (float)ry, (float)rz, __int_as_float(atom | (sp << kAtomBits)));
  };
  auto keyof = [&](const float4& p) {  // species * nseg + segment of the FP32 record
    const float r = sqrtf(p.x * p.x + p.y * p.y + p.z * p.z);
    return (int)((unsigned)__float_as_int(p.w) >> kAtomBits) * nseg + min((int)(r * inv_h), nseg - 1);
  };
  auto scan_hist = [&]() {  // exclusive scan of hist (each lane a contiguous chunk)
    const int per = (nkeys + 31) / 32;
    const int k0 = min(lane * per, nkeys), k1 = min(k0 + per, nkeys);
    int sum = 0;
    for (int k = k0; k < k1; ++k) sum += hist[k];
    int inc = sum;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
      const int t = __shfl_up_sync(0xffffffffu, inc, o);
      if (lane >= o) inc += t;
    }
    int run = inc - sum;
    for (int k = k0; k < k1; ++k) {
      const int v = hist[k];
      hist[k] = run;
      run += v;
    }
    __syncwarp();
  };
  for (int64_t c = (int64_t)blockIdx.x * (blockDim.x >> 5) + wid; c < n_centres; c += nw) {
    for (int k = lane; k < nkeys; k += 32) hist[k] = 0;
    const int64_t base = pair_off[c];
    const int64_t P = pair_off[c + 1] - base;
    __syncwarp();
    if (P <= kFillStage) {
      int n = 0;
      visit_any<true>(A, c, runs, [&](bool ok, int atom, int sp, double rx, double ry, double rz, double) {
        const unsigned bal = __ballot_sync(0xffffffffu, ok);
        if (ok) {
          const int pos = n + __popc(bal & ((1u << lane) - 1u));
          if (pos < kFillStage) {
            const float4 rec = record(atom, sp, rx, ry, rz);
            stage[pos] = rec;
            atomicAdd(&hist[keyof(rec)], 1);
          }
        }
        n += __popc(bal);
      });
      __syncwarp();
      scan_hist();
      const int m = min(n, kFillStage);
      for (int i0 = 0; i0 < m; i0 += 32) {
        const int i = i0 + lane;
        const bool ok = i < m;
        const float4 rec = ok ? stage[i] : make_float4(0.f, 0.f, 0.f, 0.f);
        const int key = ok ? keyof(rec) : -1 - lane;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        const int start = ok ? hist[key] : 0;
        __syncwarp();
        if (ok) {
          pairs[base + start + rank] = rec;
          if (rank == 0) hist[key] = start + __popc(peers);
        }
        __syncwarp();
      }
    } else {
      visit_any<true>(A, c, runs, [&](bool ok, int atom, int sp, double rx, double ry, double rz, double) {
        if (ok) atomicAdd(&hist[keyof(record(atom, sp, rx, ry, rz))], 1);
      });
      __syncwarp();
      scan_hist();
      visit_any<true>(A, c, runs, [&](bool ok, int atom, int sp, double rx, double ry, double rz, double) {
        const float4 rec = record(atom, sp, rx, ry, rz);
        const int key = ok ? keyof(rec) : -1 - lane;
        const unsigned peers = __match_any_sync(0xffffffffu, key);
        const int rank = __popc(peers & ((1u << lane) - 1u));
        const int start = ok ? hist[key] : 0;
        __syncwarp();
        if (ok) {
          pairs[base + start + rank] = rec;
          if (rank == 0) hist[key] = start + __popc(peers);
        }
        __syncwarp();
      });
    }
    __syncwarp();
  }
}

// One block: total pairs, the largest per-centre count and the status flags,
// so the host learns all three from one device-to-host copy.
__global__ void __launch_bounds__(1024) k_stats(const int64_t* pair_off, int64_t n_centres, const int* status,
                                                int64_t* out) {
  __shared__ int64_t s_max[32];
  int64_t m = 0;
  for (int64_t c = threadIdx.x; c < n_centres; c += blockDim.x) {
    const int64_t d = pair_off[c + 1] - pair_off[c];
    m = d > m ? d : m;
  }
  for (int o = 16; o > 0; o >>= 1) {
    const int64_t v = __shfl_xor_sync(0xffffffffu, m, o);
    m = v > m ? v : m;
  }
  if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int i = 1; i < (int)(blockDim.x >> 5); ++i) m = s_max[i] > m ? s_max[i] : m;
    out[0] = pair_off[n_centres];
    out[1] = m;
    out[2] = status[0];
  }
}

// One block: out[0] = the list's total; when it exceeds capacity, every
// offset is set to 0 (all lists empty), so kernels launched after it read
// nothing beyond the pair buffer.  One block: the total is read once before
// any offset is rewritten.
__global__ void __launch_bounds__(1024) k_clamp(int64_t* pair_off, int64_t n_centres, int64_t capacity, int64_t* out) {
  __shared__ int64_t s_total;
  if (threadIdx.x == 0) s_total = pair_off[n_centres];
  __syncthreads();
  const int64_t total = s_total;
  if (threadIdx.x == 0) out[0] = total;
  if (total <= capacity) return;
  for (int64_t i = threadIdx.x; i <= n_centres; i += blockDim.x) pair_off[i] = 0;
}

// ---------------------------------------------------------------------------
// host side
// ---------------------------------------------------------------------------

struct NLLayout {
  int64_t grids, fbox, bps, bin_off, bin_count, bin_start, bin_cursor, atom_bin, sorted_atom, sorted_pos, cpos,
      cinfo, counts, partials, status, total;
  int64_t max_bins;
};

static NLLayout nl_layout(const soapb_structs* s, const soapb_centres* c) {
  NLLayout L{};
  const int64_t ns = s->n_struct, na = s->n_atoms, nc = c->n_centres;
  L.max_bins = 2 * na + 8 * ns + 64;
  const int64_t maxn = (na > nc ? na : nc) + L.max_bins + 2;
  int64_t off = 0;
  auto take = [&](int64_t bytes) { const int64_t o = off; off = align_up(off + bytes, 256); return o; };
  L.grids = take(sizeof(GridDesc) * ns);
  L.fbox = take(8 * 6 * ns);
  L.bps = take(4 * ns);
  L.bin_off = take(8 * (ns + 1));
  L.bin_count = take(4 * L.max_bins);
  L.bin_start = take(8 * (L.max_bins + 1));
  L.bin_cursor = take(4 * L.max_bins);
  L.atom_bin = take(4 * na);
  L.sorted_atom = take(4 * na);
  L.sorted_pos = take(32 * na);
  L.cpos = take(32 * nc);
  L.cinfo = take(16 * nc);
  L.counts = take(4 * nc);
  L.partials = take(8 * ((maxn + 1023) / 1024 + 2));
  L.status = take(16);
  L.total = off;
  return L;
}

static NLWork nl_work(const NLLayout& L, void* base_) {
  char* base = (char*)base_;
  NLWork w;
  w.grids = (GridDesc*)(base + L.grids);
  w.fbox = (unsigned long long*)(base + L.fbox);
  w.bins_per_struct = (int*)(base + L.bps);
  w.bin_off = (int64_t*)(base + L.bin_off);
  w.bin_count = (int*)(base + L.bin_count);
  w.bin_start = (int64_t*)(base + L.bin_start);
  w.bin_cursor = (int*)(base + L.bin_cursor);
  w.atom_bin = (int*)(base + L.atom_bin);
  w.sorted_atom = (int*)(base + L.sorted_atom);
  w.sorted_pos = (double4*)(base + L.sorted_pos);
  w.cpos = (double4*)(base + L.cpos);
  w.cinfo = (int4*)(base + L.cinfo);
  w.counts = (int*)(base + L.counts);
  w.partials = (int64_t*)(base + L.partials);
  w.status = (int*)(base + L.status);
  w.max_bins = L.max_bins;
  return w;
}

static int check_inputs(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c) {
  if (!b || !b->dev) return set_error(SOAPB_ERR_ARG, "basis not built");
  if (!s || !c) return set_error(SOAPB_ERR_ARG, "null structures or centres");
  if (s->n_struct < 1) return set_error(SOAPB_ERR_ARG, "need at least one structure");
  if (s->n_atoms < 0 || c->n_centres < 0) return set_error(SOAPB_ERR_ARG, "negative sizes");
  if (s->n_atoms >= (int64_t)kAtomMask) return set_error(SOAPB_ERR_ARG, "too many atoms (max %d)", kAtomMask);
  if (s->n_atoms > 0 && (!s->d_positions || !s->d_species)) return set_error(SOAPB_ERR_ARG, "null atom arrays");
  if (!s->d_atom_off || !s->d_cells || !s->d_pbc) return set_error(SOAPB_ERR_ARG, "null structure arrays");
  if (c->n_centres > 0 && (!c->d_xyz || !c->d_struct || !c->d_atom)) return set_error(SOAPB_ERR_ARG, "null centre arrays");
  return SOAPB_OK;
}

static VisitArgs visit_args(const soapb_basis* b, const NLWork& w, int mode) {
  VisitArgs A;
  A.grids = w.grids;
  A.bin_off = w.bin_off;
  A.bin_start = w.bin_start;
  A.sorted_pos = w.sorted_pos;
  A.cpos = w.cpos;
  A.cinfo = w.cinfo;
  A.status = w.status;
  A.cutoff = b->cutoff;
  A.cutoff2 = b->cutoff * b->cutoff;
  A.mode = mode;
  return A;
}

static int grid_blocks(int64_t n, int threads) {
  int64_t g = (n + threads - 1) / threads;
  if (g < 1) g = 1;
  if (g > 148 * 64) g = 148 * 64;
  return (int)g;
}

}  // namespace soapb

using namespace soapb;

extern "C" int soapb_neighbors_workspace(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c,
                                         int64_t* bytes) {
  int rc = check_inputs(b, s, c);
  if (rc) return rc;
  if (!bytes) return set_error(SOAPB_ERR_ARG, "null bytes");
  *bytes = nl_layout(s, c).total;
  return SOAPB_OK;
}

extern "C" int soapb_neighbors_count(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c,
                                     int32_t mode, void* d_work, int64_t work_bytes, int64_t* d_pair_off,
                                     void* stream) {
  int rc = check_inputs(b, s, c);
  if (rc) return rc;
  if (mode != SOAPB_NL_CREATE && mode != SOAPB_NL_ALL) return set_error(SOAPB_ERR_ARG, "bad neighbour mode");
  const NLLayout L = nl_layout(s, c);
  if (!d_work || work_bytes < L.total) return set_error(SOAPB_ERR_ARG, "workspace too small (%lld < %lld)",
                                                        (long long)work_bytes, (long long)L.total);
  if (!d_pair_off) return set_error(SOAPB_ERR_ARG, "null pair_off");
  cudaStream_t st = (cudaStream_t)stream;
  NLWork w = nl_work(L, d_work);
  const int ns = s->n_struct;
  if ((rc = check_cuda(cudaMemsetAsync(w.status, 0, 16, st), "memset status"))) return rc;
  if ((rc = check_cuda(cudaMemsetAsync(w.bin_count, 0, 4 * L.max_bins, st), "memset bins"))) return rc;
  if ((rc = check_cuda(cudaMemsetAsync(w.bin_cursor, 0, 4 * L.max_bins, st), "memset cursor"))) return rc;
  const double cutoff = b->cutoff;
  k_grid_init<<<(ns + 127) / 128, 128, 0, st>>>(*s, w, cutoff);
  k_frac_bbox<<<grid_blocks(s->n_atoms, 256), 256, 0, st>>>(*s, w);
  k_grid_setup<<<(ns + 127) / 128, 128, 0, st>>>(*s, w, cutoff);
  if ((rc = check_launch("grid setup", 3))) return rc;
  if ((rc = exclusive_scan(w.bins_per_struct, ns, w.bin_off, w.partials, st))) return rc;
  k_bin_atoms<<<grid_blocks(s->n_atoms, 256), 256, 0, st>>>(*s, w);
  if ((rc = check_launch("k_bin_atoms"))) return rc;
  if ((rc = exclusive_scan(w.bin_count, L.max_bins, w.bin_start, w.partials, st))) return rc;
  k_scatter_atoms<<<grid_blocks(s->n_atoms, 256), 256, 0, st>>>(s->n_atoms, w);
  k_sort_bins<<<grid_blocks(L.max_bins, 4), 128, 0, st>>>(w);
  k_gather_atoms<<<grid_blocks(s->n_atoms, 256), 256, 0, st>>>(*s, w);
  k_centres<<<grid_blocks(c->n_centres, 256), 256, 0, st>>>(*s, *c, w);
  if ((rc = check_launch("cell lists", 5))) return rc;
  const VisitArgs A = visit_args(b, w, mode);
  if (c->n_centres > 0) k_count<<<grid_blocks(c->n_centres, 4), 128, 0, st>>>(A, c->n_centres, w.counts);
  if ((rc = check_launch("k_count", c->n_centres > 0 ? 1 : 0))) return rc;
  return exclusive_scan(w.counts, c->n_centres, d_pair_off, w.partials, st);
}

extern "C" int soapb_neighbors_fill(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c,
                                    int32_t mode, void* d_work, int64_t work_bytes, const int64_t* d_pair_off,
                                    void* d_pairs, int64_t capacity, void* stream) {
  int rc = check_inputs(b, s, c);
  if (rc) return rc;
  const NLLayout L = nl_layout(s, c);
  if (!d_work || work_bytes < L.total) return set_error(SOAPB_ERR_ARG, "workspace too small");
  if (!d_pair_off || (!d_pairs && capacity > 0)) return set_error(SOAPB_ERR_ARG, "null pair arrays");
  if (((uintptr_t)d_pairs) % 16) return set_error(SOAPB_ERR_ARG, "pairs must be 16-byte aligned");
  cudaStream_t st = (cudaStream_t)stream;
  NLWork w = nl_work(L, d_work);
  const VisitArgs A = visit_args(b, w, mode);
  if (c->n_centres > 0) {
    const int smem = 4 * (16 * kFillStage + 4 * b->n_keys + 4 * 3 * kRunsPerPass);
    int rc2 = check_cuda(cudaFuncSetAttribute(k_fill, cudaFuncAttributeMaxDynamicSharedMemorySize, smem),
                         "fill smem attribute");
    if (rc2) return rc2;
    k_fill<<<grid_blocks(c->n_centres, 4), 128, smem, st>>>(A, c->n_centres, d_pair_off, (float4*)d_pairs,
                                                            capacity, b->n_seg, (float)(1.0 / b->seg_width),
                                                            b->n_keys, w.status);
  }
  return check_launch("k_fill", c->n_centres > 0 ? 1 : 0);
}

extern "C" int soapb_neighbors_status(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c,
                                      void* d_work, int32_t* h_status, void* stream) {
  int rc = check_inputs(b, s, c);
  if (rc) return rc;
  const NLLayout L = nl_layout(s, c);
  NLWork w = nl_work(L, d_work);
  cudaStream_t st = (cudaStream_t)stream;
  if ((rc = check_cuda(cudaMemcpyAsync(h_status, w.status, 4, cudaMemcpyDeviceToHost, st), "status download")))
    return rc;
  return check_cuda(cudaStreamSynchronize(st), "status sync");
}

extern "C" int soapb_neighbors_stats(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c,
                                     const void* d_work, const int64_t* d_pair_off, int64_t* d_stats, void* stream) {
  int rc = check_inputs(b, s, c);
  if (rc) return rc;
  if (!d_work || !d_pair_off || !d_stats) return set_error(SOAPB_ERR_ARG, "null workspace, pair_off or stats");
  const NLLayout L = nl_layout(s, c);
  const NLWork w = nl_work(L, const_cast<void*>(d_work));
  k_stats<<<1, 1024, 0, (cudaStream_t)stream>>>(d_pair_off, c->n_centres, w.status, d_stats);
  return check_launch("k_stats");
}

extern "C" int soapb_neighbors_clamp(int64_t* d_pair_off, int64_t n_centres, int64_t capacity, int64_t* d_total,
                                     void* stream) {
  if (!d_pair_off || !d_total || n_centres < 0 || capacity < 0) return set_error(SOAPB_ERR_ARG, "bad clamp arguments");
  k_clamp<<<1, 1024, 0, (cudaStream_t)stream>>>(d_pair_off, n_centres, capacity, d_total);
  return check_launch("k_clamp");
}

// ---------------------------------------------------------------------------
// Neighbour list without any device allocation
// ---------------------------------------------------------------------------
// The regular entry points take a caller-sized workspace.  Some callers have
// no way to provide one at the moment they need a neighbour list: a plain C or
// Fortran molecular-dynamics driver that owns a fixed device-memory budget
// and forbids libraries from allocating after set-up, or a time-step loop
// where cudaMalloc / cudaFree would synchronise the device and stall it.
// soapb_neighbors_noalloc serves them: its scratch is one fixed device array
// that exists from module load to process exit on every GPU that loads the
// library, so the call itself allocates nothing.
namespace soapb {

constexpr int64_t kNoAllocScratchBytes = 8ll << 20;  // 8 MiB per device
static __device__ __align__(256) unsigned char g_nl_scratch[kNoAllocScratchBytes];

static std::mutex g_scratch_mu;
struct ScratchSlot {
  unsigned long long ctx_id;  // id of the CUDA context the address belongs to (0 = unknown)
  void* ptr;
};
static ScratchSlot g_scratch_slot[64] = {};

// Process-unique id of the calling thread's current CUDA context, or 0 when
// the driver cannot report one.  A device reset destroys the context (and
// the module with g_nl_scratch); the next context gets a new id, so a cached
// address is used only inside the context it was looked up in.  The driver
// functions come through the runtime's entry-point query: no link to libcuda.
static unsigned long long current_context_id() {
  typedef int (*GetCurrentFn)(void**);
  typedef int (*GetIdFn)(void*, unsigned long long*);
  static GetCurrentFn get_current = nullptr;
  static GetIdFn get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &f, 4000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (GetCurrentFn)f;
    f = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &f, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (GetIdFn)f;
  });
  if (!get_current || !get_id) return 0;
  void* ctx = nullptr;
  unsigned long long id = 0;
  if (get_current(&ctx) != 0 || !ctx) return 0;
  if (get_id(ctx, &id) != 0) return 0;
  return id;
}

// Device address of g_nl_scratch in the current device's context (the
// host-side symbol is not a device address).  Looked up once per context and
// cached: again after a cudaDeviceReset, and on every call when the context
// id is unavailable.
static int scratch_address(void** out) {
  int dev = 0;
  int rc = check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
  if (rc) return rc;
  if (dev < 0 || dev >= 64) return set_error(SOAPB_ERR_ARG, "device index %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_scratch_mu);
  ScratchSlot& slot = g_scratch_slot[dev];
  const unsigned long long id = current_context_id();
  if (!slot.ptr || id == 0 || slot.ctx_id != id) {
    void* p = nullptr;
    // also creates the device's primary context if this thread has none yet
    rc = check_cuda(cudaGetSymbolAddress(&p, g_nl_scratch), "cudaGetSymbolAddress(g_nl_scratch)");
    if (rc) return rc;
    slot.ptr = p;
    slot.ctx_id = current_context_id();
  }
  *out = slot.ptr;
  return SOAPB_OK;
}

}  // namespace soapb

extern "C" int soapb_neighbors_noalloc(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c,
                                       int32_t mode, int64_t* d_pair_off, void* d_pairs, int64_t capacity,
                                       int32_t* d_status, void* stream) {
  int rc = check_inputs(b, s, c);
  if (rc) return rc;
  if (!d_pair_off || !d_status) return set_error(SOAPB_ERR_ARG, "null pair_off or status");
  const NLLayout L = nl_layout(s, c);
  if (L.total > kNoAllocScratchBytes)
    return set_error(SOAPB_ERR_ARG,
                     "soapb_neighbors_noalloc: this input needs %lld bytes of scratch but the fixed scratch array "
                     "holds %lld bytes (about 67,000 atoms with every atom a centre); use soapb_neighbors_count/_fill with a workspace",
                     (long long)L.total, (long long)kNoAllocScratchBytes);
  void* scratch = nullptr;
  if ((rc = scratch_address(&scratch))) return rc;
  // count clears the scratch words that must start at zero (status, bin counts, bin cursors)
  if ((rc = soapb_neighbors_count(b, s, c, mode, scratch, kNoAllocScratchBytes, d_pair_off, stream))) return rc;
  if ((rc = soapb_neighbors_fill(b, s, c, mode, scratch, kNoAllocScratchBytes, d_pair_off, d_pairs, capacity,
                                 stream)))
    return rc;
  const NLWork w = nl_work(L, scratch);
  return check_cuda(cudaMemcpyAsync(d_status, w.status, sizeof(int32_t), cudaMemcpyDeviceToDevice,
                                    (cudaStream_t)stream),
                    "status copy");
}
