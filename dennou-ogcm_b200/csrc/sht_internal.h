// sht_internal.h -- plan state, device layouts and kernel launchers of the
// B200 spherical-harmonic transform.
//
// Device data layouts (all FP64):
//   grid      xya[b][j][i]        b < nb field-levels, j < J (mu ascending), i < I
//   spectral  wa[b][l]            SPML order l = n(n+1)+m, m in [-n, n]
//   Fourier   F[m][col][j]        complex G^m(mu_j) for m <= N, col < ncol
//                                 (ncol = nb, or 2 nb for two-input operators)
//   internal  S[row][col]         complex coefficient of Pbar_n^m, row = rowoff(m) + n - m,
//                                 n = m..N+1 (one extra degree so that the
//                                 (1-mu^2) d/dmu recurrences close), rowoff(m) =
//                                 sum_{m'<m} (N+2-m').
//   Legendre  P[poff(m) + (n-m) JH + jh]  Pbar_n^m at the northern Gauss rows
//                                 j = JH + jh (JH = J/2), n = m..N+1.
#pragma once

#include <cuda_runtime.h>
#include <cstdint>
#include <cstddef>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/dogcm_sht.h"

namespace sht {

// Row-scale tables used by the longitude transforms (per Gauss row j).
enum RowScale : int {
  RS_FWD_PLAIN = 0,     // analysis: w_j / I
  RS_FWD_INV1MMU2 = 1,  // analysis: w_j / (I (1 - mu_j^2))
  RS_INV_PLAIN = 2,     // synthesis: 1
  RS_INV_INVCOS = 3,    // synthesis: 1 / cos(phi_j)
  RS_INV_INVA1MMU2 = 4, // synthesis: 1 / (a (1 - mu_j^2))
  RS_INV_INVACOS = 5,   // synthesis: 1 / (a cos(phi_j))
  RS_FWD_INVCOS = 6,    // analysis: w_j / (I cos(phi_j)) = w_j cos(phi_j) / (I (1 - mu_j^2))
  RS_COUNT = 7
};

// Spectral-side operators applied between the SPML layout and the internal one.
enum PackOp : int {
  PACK_PLAIN = 0,      // w = c
  PACK_DIVLAMBDA = 1,  // w = i m c
  PACK_DIVMU = 2,      // w = D(c) = -((n+1) eps_n c_{n-1} - n eps_{n+1} c_{n+1})
  PACK_ALPHA = 3,      // w = (i m cA + D(cB)) / a, D = the divmu form    (two column sets)
  PACK_VORDIV = 4,     // vor = (i m cV - D(cU))/a, div = (i m cU + D(cV))/a
};
enum UnpackOp : int {
  UNPACK_PLAIN = 0,      // a
  UNPACK_GRADLAMBDA = 1, // i m a
  UNPACK_GRADMU = 2,     // (k+2) eps_{k+1} a_{k+1} - (k-1) eps_k a_{k-1}
  UNPACK_ALPHA = 3,      // i m aA + GRADMU(aB)                   (two inputs)
  UNPACK_VORDIV2UV = 4,  // psi, chi = -a^2 a/(n(n+1)); U = i m chi - GRADMU(psi), V = i m psi + GRADMU(chi)
  UNPACK_HGRAD = 5,      // i m a and GRADMU(a) from one input    (two column sets)
};

struct Timing {
  bool on = false;
  cudaEvent_t ev[8] = {};
  float ms_fft = 0.f, ms_leg = 0.f, ms_spec = 0.f;
};

// A host-pointer call staged through the plan's page-locked buffer, kept as
// an instantiated CUDA graph (copy in, the operator's kernels, copy out).
// Every pointer in it is a plan buffer, so it replays for any caller arrays
// of the same operator and size until a buffer is reallocated (buf_gen).
struct HostGraph {
  int op = -1, nb = 0, precision = 0, leg_kernel = 0, leg_tile = 0;
  unsigned long long gen = 0;
  cudaGraphExec_t exec = nullptr;  // null after the first call, or when not capturable
  bool failed = false;             // capture was refused: run this call uncaptured
  int launches = 0;                // kernels in the graph
};

}  // namespace sht

struct sht_plan_s {
  uint32_t magic = 0;
  int I = 0, J = 0, N = 0, K = 0, JH = 0, NC = 0, L = 0;
  int fa = 0, fb = 0;           // four-step split NC = 2^fa * 2^fb
  long long R = 0;              // internal rows (N+1)(N+4)/2
  double radius = 1.0;
  int device = 0;
  cudaStream_t stream = nullptr;      // stream used by all work of the plan
  cudaStream_t own_stream = nullptr;  // stream created by sht_init (destroyed by sht_final)
  // host-pointer calls: copy streams and per-chunk events of the pipelined
  // host -> device -> host path (created on first use)
  cudaStream_t copy_in = nullptr, copy_out = nullptr;
  cudaEvent_t chunk_ev[16] = {};
  bool zonal = false;  // im = 1: the axisymmetric (m = 0) transform of wa_zonal_module, lm = nm + 1
  bool direct_dft = false;  // im not a power of two: longitude transform by direct summation
  int M = 0;           // orders transformed: N + 1, or 1 for a zonal plan
  int precision = SHT_PREC_FP64;
  int leg_kernel = 0;  // SHT_OPT_LEGENDRE_KERNEL: 0 auto, 1 per-band, 2 paired persistent, 3 latitude-chunked persistent,
                       // 4 single-kernel small-grid transform (plain analysis and synthesis, im <= 128)
  int leg_tile = 0;    // SHT_OPT_LEGENDRE_TILE: 0 auto; paired kernels: analysis columns per item (8, 16); chunked kernels: latitudes per chunk (16, 32)

  // device tables
  double *d_mu = nullptr, *d_wgt = nullptr, *d_rowscale = nullptr;
  double *d_P = nullptr;
  long long *d_poff = nullptr;
  int *d_rowoff = nullptr;
  double *d_eps = nullptr;  // [m][n], n = 0..N+2
  double2 *d_tw = nullptr;  // exp(-2 pi i k / NC), k < NC
  double2 *d_twI = nullptr; // exp(-2 pi i k / I),  k < NC
  double *d_rn = nullptr;   // -n(n+1) per l
  int2 *d_spec_tiles = nullptr;  // (n, m0) tiles of the spectral conversions
  int n_spec_tiles = 0;          // n = 0..N+1
  int n_pack_tiles = 0;          // n = 0..N (a prefix of the list)
  int2 *d_pairs = nullptr;       // band pairs (m, N-m), (N/2, -1) for even N
  int n_pairs = 0;
  int num_sms = 0;
  int sm_cap = 0;       // at most this many SMs' worth of persistent blocks (0: all); set by a batch that runs plans side by side

  // host copies
  std::vector<double> h_mu, h_wgt;
  std::vector<int> h_rowoff;

  // device workspace (Fourier + internal spectral), grown on demand
  void *d_ws = nullptr;
  size_t ws_bytes = 0;
  // device staging for the host-pointer API, grown on demand
  void *d_io = nullptr;
  size_t io_bytes = 0;
  // page-locked host staging for small host-pointer calls on pageable arrays
  void *h_stage = nullptr;
  size_t h_stage_bytes = 0;

  // split-precision tables (built lazily)
  void *tc_tables = nullptr;
  // device address of the allocation-free entry point's fixed scratch array
  // on this plan's device (looked up on that entry point's first call)
  void *noalloc_scratch = nullptr;

  // graphs of staged host-pointer calls (SHT_OPT_HOST_GRAPHS), the stream
  // they are captured on, and the generation of the buffers they name
  // (bumped whenever d_ws, d_io or h_stage is reallocated)
  bool host_graphs = true;
  std::vector<sht::HostGraph> graphs;
  cudaStream_t cap_stream = nullptr;
  unsigned long long buf_gen = 0;

  std::mutex mtx;
  sht::Timing timing;
};

namespace sht {

constexpr uint32_t kPlanMagic = 0x53485442u;  // "SHTB"

void set_error(const std::string &msg);
int cuda_fail(cudaError_t e, const char *what);
void count_launch(int n = 1);

// Dynamic shared-memory opt-in of a kernel and its resident blocks per SM at
// (smem, threads), on the current device.  The runtime calls behind them
// cost microseconds each, which a per-level call would pay on every launch,
// so the results are cached per device and kernel; the opt-in only grows.
cudaError_t kernel_setup(const void *kern, size_t smem, int threads, int *per_sm = nullptr);

// --- setup kernels (sht_setup.cu)
int build_tables(sht_plan *p);

// --- longitude transforms (sht_fft.cu)
// grid (up to two source arrays: columns [0, nsplit) from g0, the rest from g1;
// or, when gcol is given, column c at gcol[c]) -> F[m][colF0 + col][j],
// scaled per row by rowscale table `rs`.
int launch_fft_fwd(const sht_plan *p, const double *g0, const double *g1, int nsplit, int ncol,
                   double2 *F, int ncolF, int colF0, int rs, cudaStream_t s,
                   const double *const *gcol = nullptr, const double *mul = nullptr, int nmul = 0,
                   const double *add0 = nullptr, const double *add1 = nullptr);
// F -> grid (two destinations split at nsplit, or column c at ocol[c]),
// scaled per row by `rs`.
int launch_fft_inv(const sht_plan *p, const double2 *F, int ncolF, int colF0, int ncol,
                   double *g0, double *g1, int nsplit, int rs, cudaStream_t s,
                   double *const *ocol = nullptr);

// --- Legendre contraction, FP64 (sht_legendre.cu)
int pick_fp64_kernel(const sht_plan *p);  // 1 per-band, 2 paired, 3 latitude-chunked
int launch_leg_fwd_fp64(const sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s);
int launch_leg_inv_fp64(const sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s);

// --- persistent paired-band FP64 contraction (sht_legendre_v2.cu)
bool split_supported(const sht_plan *p);
// Whether a contraction runs in split precision: always under SHT_PREC_SPLIT;
// under SHT_PREC_AUTO when it is at least 128 terms long (jm/2 latitudes in
// the analysis, (nm+3)/2 degrees of one parity in the synthesis), where the
// int8 digit kernel measured faster than the FP64 tensor path on B200 (T170
// analysis 0.41 against 0.44 ms; T341 3.09 / 2.77 against 3.78 / 3.52 ms; T170
// synthesis, 86 terms, 0.48 against 0.40 ms).
// --- whole plain transforms of small grids in one kernel (sht_small.cu)
bool small_supported(const sht_plan *p);
int launch_small_fwd(const sht_plan *p, const double *g, const double *const *gcol, int ncol, double *w,
                     double *const *wcol, cudaStream_t s);
int launch_small_inv(const sht_plan *p, const double *w, const double *const *wcol, int ncol, double *g,
                     double *const *gcol, cudaStream_t s);

inline bool use_split(const sht_plan *p, bool analysis)
{
  if (p->precision == SHT_PREC_SPLIT) return true;
  if (p->precision != SHT_PREC_AUTO || !split_supported(p)) return false;
  return (analysis ? p->JH : (p->N + 3) / 2) >= 128;
}

// plain analysis / synthesis by the single-kernel small-grid transform:
// chosen with SHT_OPT_LEGENDRE_KERNEL = 4, and by the automatic choice for
// im = 32 (16 complex points per row), the only size where it measured
// faster than the batched kernels (T10, 480 field-levels: round trip 31
// against 59 us); in FP64 only (split precision keeps the batched path)
inline bool use_small(const sht_plan *p, bool analysis)
{
  const bool want = p->leg_kernel == 4 || (p->leg_kernel == 0 && p->NC == 16);
  return want && !use_split(p, analysis) && small_supported(p);
}

// SMs a plan's persistent kernels size their grids for
inline int grid_sms(const sht_plan *p)
{
  const int n = p->num_sms > 0 ? p->num_sms : 1;
  return (p->sm_cap > 0 && p->sm_cap < n) ? p->sm_cap : n;
}
bool leg_pair_supported(const sht_plan *p);
int launch_leg_fwd_pair(const sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s);
int launch_leg_inv_pair(const sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s);

// --- persistent latitude-chunked FP64 contraction for large grids (sht_legendre_v3.cu)
bool leg_chunk_supported(const sht_plan *p);
int launch_leg_fwd_chunk(const sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s);
int launch_leg_inv_chunk(const sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s);

// --- Legendre contraction, split precision on tcgen05 (sht_legendre_tc.cu)
int launch_leg_fwd_split(sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s);
int launch_leg_inv_split(sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s);
void free_split_tables(sht_plan *p);
int split_error_status(sht_plan *p);  // reads and clears the device error word (synchronous)
// one block whose bounded wait runs out on purpose and sets the error word (synchronous)
int wait_selftest(sht_plan *p, unsigned long long limit_ns);
// Reads and clears every device error word of the plan (synchronous).
int device_error_status(sht_plan *p);

// --- column-table pipelines (sht_capi.cu), used by the multi-instance batches
// F holds (N+1) J ncol complex values, S holds R ncol; the plan mutex is held
// by the caller.
int run_analysis_cols(sht_plan *p, const double *const *gcol, int ncol, double *const *wcol, double2 *F,
                      double2 *S, cudaStream_t s);
int run_synthesis_cols(sht_plan *p, const double *const *wcol, int ncol, double *const *gcol, double2 *F,
                       double2 *S, cudaStream_t s);

// --- spectral-side kernels (sht_spectral.cu)
// internal S (ncolS columns; set A at col 0, set B at col nb) -> SPML wa outputs
// (field-level b at w0 + b L, or at wcol[b] when a column table is given;
// tables serve the single-output operators)
int launch_pack(const sht_plan *p, int op, const double2 *S, int ncolS, int nb, double *w0,
                double *w1, cudaStream_t s, double *const *wcol = nullptr);
// SPML inputs -> internal S (ncolS columns); wcol as for launch_pack
int launch_unpack(const sht_plan *p, int op, const double *w0, const double *w1, int nb,
                  double2 *S, int ncolS, cudaStream_t s, const double *const *wcol = nullptr);
int launch_lapla(const sht_plan *p, const double *w, int nb, double *out, bool inverse,
                 cudaStream_t s);
int launch_diffuse(const sht_plan *p, double *w, int nb, const double *coef, double dt,
                   const double *filter, cudaStream_t s);
int launch_lonlat_reduce(const sht_plan *p, const double *g, int nb, double *out, int kind,
                         cudaStream_t s);

}  // namespace sht
