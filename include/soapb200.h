/*
 * soapb200.h -- C ABI of the B200 SOAP descriptor library (libsoapb200.so).
 *
 * The library replaces the compute path of the reference SOAP generator
 * (TACC/cuSOAP, src/cusoap/soap_generator.py, cited as SG:<line>): the
 * radius neighbour search, the GTO coefficient accumulation, the power
 * spectrum / cc projection, the closed-form Jacobian and the force adjoint.
 * The reference exposes these only as private methods of its Python SOAP
 * class; the Python package cusoap_b200 binds the functions below with
 * ctypes and keeps the reference's public SOAP(...) / create() /
 * derivatives() surface.
 *
 * Conventions
 *  - Every pointer named dev_* / d_* is device memory owned by the caller.
 *    The library performs no device allocation of its own; work buffers are
 *    passed in, with their sizes queried beforehand.
 *  - All work is enqueued on the given CUDA stream (cudaStream_t passed as
 *    void*; NULL = legacy default stream); functions return once enqueued.
 *  - Functions return SOAPB_OK (0) or an error status; soapb_last_error()
 *    gives a message for the calling thread.  No C++ exception crosses the
 *    ABI.  A handle (soapb_basis) is not thread-safe; use one per thread or
 *    stream, as the reference's SOAP object is (SG:1921-1922).
 *  - Positions, cells and centre coordinates are float64 (the reference
 *    computes internally in float64, SG:1775-1780); the bulk arithmetic and
 *    all outputs are float32.
 */
#ifndef SOAPB200_H
#define SOAPB200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
  SOAPB_OK = 0,
  SOAPB_ERR_ARG = 1,         /* invalid argument or unsupported size */
  SOAPB_ERR_CUDA = 2,        /* a CUDA runtime call failed */
  SOAPB_ERR_CAPACITY = 3,    /* an output buffer was too small; retry bigger */
  SOAPB_ERR_UNSUPPORTED = 4, /* parameter combination not built */
  SOAPB_ERR_ACCURACY = 5     /* radial tables missed their error bound */
};

/* average / output modes of the descriptor */
enum {
  SOAPB_OUT_PS = 0,  /* power spectrum, DScribe order (average off/inner/outer, SG:1634-1689) */
  SOAPB_OUT_CC = 1,  /* projection coefficients, DScribe cc layout (SG:1603-1632) */
  SOAPB_OUT_RAW = 2  /* c[s][n][lm] per centre, no permutation / scaling */
};

/* radial basis functions (SOAP rbf argument, SG:616-621) */
enum {
  SOAPB_RBF_GTO = 0,  /* Gaussian-type orbitals, Loewdin-orthonormalised (SG:690-708) */
  SOAPB_RBF_POLY = 1  /* DScribe polynomials (r_cut - r)^(k+2), orthonormalised by the caller (SG:710-752) */
};

/* weighting of the neighbour densities (SOAP weighting argument, SG:403-470) */
enum {
  SOAPB_W_NONE = 0,  /* no weighting: w = 1, w0 = 1 */
  SOAPB_W_W0 = 1,    /* function None: w = 1 for r > 0, w0 = w_w0 for the centre's own Gaussian */
  SOAPB_W_POLY = 2,  /* w = c (1 + 2 x^3 - 3 x^2)^m for x = r / r0 <= 1, else 0 */
  SOAPB_W_POW = 3,   /* w = c / (d + x^m) */
  SOAPB_W_EXP = 4    /* w = c / (d + exp(-r / r0)) */
};

/* Radial basis + radial tables.  Fill the input fields, call
 * soapb_basis_plan (host only) to get the sizes, allocate `bytes` of device
 * memory, then soapb_basis_build.  Replaces SOAP.__init__'s basis set-up:
 * _init_gto_basis SG:690-708, _lowdin_invsqrt SG:339-343, _init_poly_basis
 * SG:710-752, the weighting SG:403-470 / SG:584-597, the self terms
 * SG:765-819, the cutoff padding SG:600-602 and the feature tables
 * SG:1215-1291.
 *
 * Radial tables: for every radial function (n, l) and segment, degree-7
 * polynomials in the segment coordinate t in [-1, 1] of
 *   B(r) = w(r) B_nl(r)            (c_nlm of an edge = B(r) R_lm(rvec))
 *   D(r) = d/dr [w(r) B_nl(r)]     (d c_nlm / d rvec = rvec D / r R_lm + B grad R_lm)
 * built in FP64 on the device.  Edges at r = 0 (the centre's own Gaussian)
 * use the per-function self value w0 B_nl(0) instead of the table. */
typedef struct soapb_basis {
  /* inputs */
  int32_t n_max, l_max, n_species, crossover;
  double r_cut, sigma;
  int32_t rbf;          /* SOAPB_RBF_* */
  int32_t weighting;    /* SOAPB_W_* */
  double w_r0, w_c, w_d, w_m, w_w0;  /* weighting parameters (DScribe names) */
  int32_t quad_n;       /* SOAPB_RBF_POLY: Gauss-Legendre points of the caller's grid */
  int32_t seg_hint;     /* 0, or a lower bound on n_seg (finer tables) */
  int32_t tune[4];      /* launch shapes picked by an autotuner, 0 = built-in choice:
                           [0] descriptor warps per block (1, 2, 4), [1] descriptor radial
                           functions per lane of the l-grouped kernel (1, 2, 3, 4, 6; at least
                           the minimum for n_max, l_max), [2] adjoint edge-kernel warps per
                           block (1, 2, 4), [3] descriptor kernel family: 0 = built-in (one
                           lane per radial index n for n_max <= 8, l_max <= 6, else lanes
                           grouped by l), 1 = lanes grouped by l always */
  const double* h_poly; /* SOAPB_RBF_POLY: host rx[quad_n] | wr[quad_n] | g[n_max][quad_n] (g_n on the grid) */
  /* derived by soapb_basis_plan */
  double eta;        /* 1 / (2 sigma^2) */
  double cutoff;     /* r_cut + sigma sqrt(-2 ln 1e-3) */
  double seg_width;  /* radial table segment width (A); n_seg * seg_width >= cutoff */
  int32_t n_seg;     /* radial table segments */
  int32_t n_keys;    /* n_species * n_seg: neighbour sort keys */
  int32_t n_feat_ps; /* SG:913-919 */
  int32_t n_feat_cc; /* SG:909-910 */
  int64_t bytes;     /* device bytes the basis needs */
  int64_t off_alpha, off_beta, off_tab_b, off_tab_bh, off_ftab, off_widx, off_err;  /* byte offsets into dev */
  int64_t off_tabf;  /* function-major table of w B_nl on half-width segments (2 n_seg of them, rows 64
                        half segments apart when they fit, else 2 n_seg): value and derivative */
  int64_t off_self, off_poly;      /* self values (n_max (l_max+1) float); device copy of h_poly */
  void* dev;         /* set by soapb_basis_build */
} soapb_basis;

int soapb_basis_plan(soapb_basis* b);
int soapb_basis_build(soapb_basis* b, void* dev_buf, void* stream);
/* Copy the FP64 alpha (l_max+1, n_max), beta (l_max+1, n_max, n_max) (GTO
 * only) and the two table errors (max |table - exact| / max|exact| per
 * function for B and D) to host memory; synchronises the stream. */
int soapb_basis_download(const soapb_basis* b, double* h_alpha, double* h_beta, double* h_err2, void* stream);

/* A batch of structures.  Atoms of structure i are [atom_off[i], atom_off[i+1]).
 * cells: (n_struct, 3, 3) row vectors (lattice a, b, c); pbc: (n_struct, 3).
 * Structures whose pbc is all zero ignore their cell. */
typedef struct soapb_structs {
  int32_t n_struct;
  int64_t n_atoms;
  const int64_t* d_atom_off;   /* (n_struct + 1) */
  const double* d_positions;   /* (n_atoms, 3) */
  const int32_t* d_species;    /* (n_atoms,) species index in [0, n_species) */
  const double* d_cells;       /* (n_struct, 9) */
  const uint8_t* d_pbc;        /* (n_struct, 3) */
} soapb_structs;

/* Centres: one row per output descriptor row.
 * centre_atom >= 0 marks an index centre (or a Cartesian centre that
 * coincides with that atom, SG:966-1003); its own r=0 edge then carries the
 * analytic self term (SG:765-850). */
typedef struct soapb_centres {
  int64_t n_centres;
  const double* d_xyz;         /* (n_centres, 3) */
  const int32_t* d_struct;     /* (n_centres,) structure of each centre */
  const int32_t* d_atom;       /* (n_centres,) centre atom or -1 */
} soapb_centres;

/* Neighbour pairs, CSR over centres, pairs of a centre sorted by
 * (neighbour species, radial segment).  One pair = float4
 * {rx, ry, rz, bits(atom | species << 27)}, r = neighbour - centre. */
enum {
  SOAPB_NL_CREATE = 0,   /* drop r <= 1e-12 edges except the centre's own (SG:1171-1179) */
  SOAPB_NL_ALL = 1       /* keep every edge within the cutoff (SG:2372-2373) */
};

/* Workspace bytes for soapb_neighbors_count / _fill (cell lists, scan). */
int soapb_neighbors_workspace(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c,
                              int64_t* bytes);
/* Bins the atoms into cell lists (counting sort), counts the pairs of every
 * centre and writes the exclusive scan d_pair_off (n_centres + 1).  The
 * total pair count is d_pair_off[n_centres].  Replaces _radius_edges /
 * _build_neighbor_list / _extend_periodic (SG:1015-1181). */
int soapb_neighbors_count(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c, int32_t mode,
                          void* d_work, int64_t work_bytes, int64_t* d_pair_off, void* stream);
/* Writes the sorted pairs (capacity = allocated pairs).  Must follow
 * soapb_neighbors_count with the same arguments and workspace. */
int soapb_neighbors_fill(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c, int32_t mode,
                         void* d_work, int64_t work_bytes, const int64_t* d_pair_off, void* d_pairs,
                         int64_t capacity, void* stream);
/* Error flags of the last count/fill on this workspace (synchronises the
 * stream): bit 0 singular cell, bit 1 atom more than 511 cells outside its
 * cell, bit 2 pair capacity exceeded, bit 3 internal enumeration limit (a
 * window row of more than 4 runs; not reachable by construction).  0 = no
 * error. */
int soapb_neighbors_status(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c, void* d_work,
                           int32_t* h_status, void* stream);

/* Summary of a neighbour list after soapb_neighbors_count (and, optionally,
 * _fill), for one device-to-host read: d_stats (device int64[3]) receives
 * {total pairs = d_pair_off[n_centres], largest pair count of a centre,
 * status flags as soapb_neighbors_status}.  Stream-ordered, no sync.  No
 * single counterpart in the reference: it replaces the edge-count and
 * max-degree reads around _build_neighbor_list (soap_generator.py:1128-1181). */
int soapb_neighbors_stats(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c, const void* d_work,
                          const int64_t* d_pair_off, int64_t* d_stats, void* stream);

/* For a pair buffer of fixed capacity (a captured CUDA graph replays with
 * the buffers it was captured with): after soapb_neighbors_fill, write the
 * list's total to *d_total (device int64) and, if it exceeds `capacity`,
 * set every offset of d_pair_off to 0 so that the descriptor / Jacobian /
 * adjoint kernels launched after it see empty lists instead of reading past
 * the buffer.  The caller compares *d_total with its capacity and rebuilds
 * with a larger buffer.  Stream-ordered, no sync.  No counterpart in the
 * reference (it allocates per call, SG:1128-1181). */
int soapb_neighbors_clamp(int64_t* d_pair_off, int64_t n_centres, int64_t capacity, int64_t* d_total, void* stream);

/* Neighbour list that allocates nothing, for callers that cannot allocate
 * device memory when they need a list (a C/Fortran MD driver with a fixed
 * device-memory budget, or a time-step loop where cudaMalloc/cudaFree would
 * synchronise the device).  It has no counterpart in the reference.  Same
 * inputs and outputs as soapb_neighbors_count + soapb_neighbors_fill, but
 * the workspace is a fixed 8 MiB device array inside the library (held on
 * every GPU that loads it until the process exits), enough for about
 * 67,000 atoms when every atom is a centre (~124 bytes per atom); larger inputs return SOAPB_ERR_ARG before
 * anything is launched.  Pairs are written only when the total
 * d_pair_off[n_centres] fits `capacity`; *d_status (device int32) receives
 * the error flags of soapb_neighbors_status (bit 2 = capacity too small).
 * The first call in each device's CUDA context looks up the array's device
 * address with cudaGetSymbolAddress and caches it for that context; after a
 * cudaDeviceReset the next call looks it up again.  Make the first call on
 * a device (and the first after a reset) before any stream capture.
 * All calls share the one array and each call clears what must start at
 * zero; calls whose executions overlap on the GPU (other streams, other
 * threads) race on it. */
int soapb_neighbors_noalloc(const soapb_basis* b, const soapb_structs* s, const soapb_centres* c, int32_t mode,
                            int64_t* d_pair_off, void* d_pairs, int64_t capacity, int32_t* d_status,
                            void* stream);

/* Descriptor: fused radial x solid-harmonic accumulation of c_nlm per centre
 * in registers, then the power spectrum / cc / raw epilogue, one warp per
 * centre from a work queue.  d_out: (n_centres, F) float32 with
 * F = n_feat_ps (PS), n_feat_cc (CC, RAW).  d_coeff: optional (may be NULL)
 * second output of the raw c[s][n][lm] rows (n_centres, n_feat_cc), as the
 * derivative and adjoint paths need.  d_counter: one int32 of scratch.
 * Replaces _coefficients_gto SG:1294-1391, _add_self_terms SG:821-850,
 * _power_spectrum SG:1634-1689 and _projection_cc SG:1624-1632. */
int soapb_descriptor(const soapb_basis* b, int64_t n_centres, const int64_t* d_pair_off, const void* d_pairs,
                     int32_t out_mode, float* d_out, float* d_coeff, int32_t* d_counter, void* stream);

/* Workspace bytes of soapb_jacobian (sorted per-centre entries and a merge
 * buffer of the same size, a nonzero-row bitmap, a work counter) for
 * n_pairs = d_pair_off[n_centres] pairs. */
int soapb_jacobian_workspace(const soapb_basis* b, int64_t n_centres, int64_t n_pairs, int64_t n_inc,
                             int32_t attach, int64_t* bytes);
/* Dense Jacobian of the descriptor w.r.t. the included atoms: d_out
 * (n_centres, n_inc, 3, F) float32 (16-byte aligned), every element written
 * once (zeros included).  d_coeff: raw coefficients (soapb_descriptor's
 * d_coeff) on the same SOAPB_NL_ALL pairs.  d_inc_row: (n_atoms,) output row
 * of each atom or -1.  attach = 0: fixed centres (DScribe convention,
 * SG:2297-2301); 1: centres move with their atom (d_centre_atom), adding the
 * centre-motion term.  max_pairs: the largest pair count of any centre (e.g.
 * from soapb_neighbors_stats); it sizes the shared-memory sort of a centre's
 * entries (up to 8192).  A centre with more entries (pairs of included atoms,
 * twice with attach) than that buffer holds is sorted in tiles and merged in
 * the workspace, so there is no limit per centre.  out_mode PS or CC.
 * d_status: int32 word, kept for the ABI and never set.  Every edge of an
 * atom accumulates, so periodic images are handled.  Replaces
 * derivatives_analytical_ps SG:2270-2626 and its Triton kernels SG:50-220. */
int soapb_jacobian(const soapb_basis* b, int64_t n_centres, const int64_t* d_pair_off, const void* d_pairs,
                   int64_t n_pairs, const float* d_coeff, const int32_t* d_inc_row, int64_t n_inc,
                   const int32_t* d_centre_atom, int32_t attach, int32_t max_pairs, int32_t out_mode, float* d_out,
                   void* d_work, int64_t work_bytes, int32_t* d_status, void* stream);

/* Adjoint: given dE/dp (n_centres, F) float32 of the descriptor of out_mode
 * (SOAPB_OUT_PS: F = n_feat_ps; SOAPB_OUT_CC: F = n_feat_cc), accumulate
 * d_forces[a] += -dE/dx_a (float32 (n_atoms, 3); the caller zeroes it) with
 * float atomics.  attach = 1: centres move with their atoms (d_centre_atom);
 * 0: fixed centres.  d_coeff: raw coefficients on SOAPB_NL_ALL pairs.
 * d_work: soapb_forces_workspace bytes (G = dE/dc per centre).  d_counter:
 * one int32 of scratch.  When d_dEdp and d_coeff are 16-byte aligned and
 * their rows are multiples of 16 bytes, the G stage brings each centre's rows
 * in by TMA bulk copies and waits for them at most about one second.  A copy
 * that does not complete in that time sets bit 0 of the workspace's status
 * word (soapb_forces_status), gets one more bounded wait, and turns that
 * block's G rows into NaN (so the forces come out NaN, not silently wrong)
 * instead of hanging the GPU; results computed on that context afterwards
 * should not be trusted.  Replaces one reverse pass of the reference's
 * autograd Jacobian SG:2007-2113 without materialising dp/dr. */
int soapb_forces_workspace(const soapb_basis* b, int64_t n_centres, int64_t* bytes);
int soapb_forces(const soapb_basis* b, int64_t n_centres, const int64_t* d_pair_off, const void* d_pairs,
                 const float* d_coeff, const float* d_dEdp, int32_t out_mode, const int32_t* d_centre_atom,
                 int32_t attach, float* d_forces, void* d_work, int64_t work_bytes, int32_t* d_counter,
                 void* stream);
/* Status word of the last soapb_forces on this workspace (synchronises the
 * stream): 0 = ok, bit 0 = a row copy of the G stage timed out.  No
 * counterpart in the reference (autograd reports no device status). */
int soapb_forces_status(const soapb_basis* b, int64_t n_centres, const void* d_work, int32_t* h_status,
                        void* stream);
/* Diagnostic of the failure path above: one block waits, with the G stage's
 * bounded wait, on a barrier that no copy completes, gives up after about one
 * second and writes 1 to the device int32 *d_status (0 if the wait had ended
 * normally).  Stream-ordered; no copy is in flight, so the context stays
 * usable.  No counterpart in the reference. */
int soapb_check_bounded_wait(int32_t* d_status, void* stream);

/* Message describing the last error on the calling thread ("" if none). */
const char* soapb_last_error(void);
/* Library version string. */
const char* soapb_version(void);
/* Number of kernels this library has launched in the process so far. */
int64_t soapb_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* SOAPB200_H */
