// sht_legendre_v2.cu -- persistent FP64 Legendre contraction with paired bands.
//
// The triangular band of order m has N+2-m degrees.  Pairing m with N-m makes
// every pair hold N+4 degrees.  A work item is (pair, 8 (analysis at JH = 64)
// or 16 complex field-level columns), so all items cost the same.  Each
// thread block is resident and takes a contiguous slice of the pair-major
// item list.  So it reloads the pair's Legendre rows (P) at most a few times,
// and the blocks finish together.  The products run on the FP64 tensor path
// (mma.sync.m8n8k4.f64).  The analysis runs two blocks per SM, each with one
// data panel, so one block's panel load overlaps the other's products; the
// synthesis runs one block per SM and fetches the next item's panel with
// cp.async while the current one is contracted.
// Shared-memory row strides are chosen so that every 16-lane phase of a
// fragment load touches 16 distinct double-word bank pairs:
//   P rows (stride-2 rows of one parity):  PS = 2 (mod 8) doubles (synthesis,
//     8-byte fragment loads), 4 (mod 8) (analysis, 16-byte fragment loads)
//   data rows (columns of one panel):      CS = 2 (mod 4) doubles: a lane's
//     16-byte B load sits at chunk (row CS/2 + 2q) mod 8 of its row pair, and an
//     odd CS/2 puts the two rows of a quarter-warp on the odd and even chunks
//     (CS = 8 (mod 16) put both on the even ones: a 2-way conflict per load)
//   coefficient rows (stride-2 rows):      AS = 2 (mod 8) doubles
// Used when a pair's P rows and the data panels fit in shared memory (T85 and
// smaller); larger grids use the chunked kernels of sht_legendre_v3.cu.
//
// Analysis follows space_discretization.tex:197-200 and synthesis :212-216.
// Symmetric and antisymmetric latitude halves use Pbar(-mu) = (-1)^{n-m} Pbar(mu);
// the longitude transforms deliver Gs/Ga and take the even/odd-degree sums at
// F[m][col][jh] and F[m][col][JH + jh].
#include "sht_internal.h"
#include "sht_dmma.cuh"
#include "sht_l2.cuh"

namespace sht {

namespace {

constexpr int kW = 8;            // warps per block
constexpr int kT = kW * 32;      // threads per block
constexpr int kCT = 16;          // complex columns per item (synthesis)
// complex columns per analysis item: 8 at JH = 64 (one panel per block, two
// blocks per SM), 16 below, where an item's contraction is short; the plan's
// SHT_OPT_LEGENDRE_TILE (8 or 16) overrides it where the panel fits
__host__ __device__ constexpr int ct_fwd(int JH) { return JH >= 64 ? 8 : 16; }

struct Geo {
  int PS, CS, AS;      // strides (doubles)
  int prow_cap;        // P rows reserved per pair (N+4 plus padding)
  int arow_cap;        // coefficient rows reserved per m (rounded, zero tail)
};

__host__ __device__ inline int round_mod(int x, int r, int mod)
{
  while (x % mod != r) ++x;
  return x;
}

__host__ __device__ inline Geo make_geo(int N, int J, bool analysis)
{
  Geo g;
  const int JH = J / 2;
  g.PS = round_mod(JH, analysis ? 4 : 2, 8);
  g.CS = round_mod(2 * J, 2, 4);
  g.AS = round_mod(2 * kCT, 2, 8);
  g.prow_cap = N + 4;
  g.arow_cap = (N + 2 + 8 + 7) & ~7;  // rows of the larger band plus a zeroed tail (a k-step reads up to 7 rows past it)
  return g;
}

struct V2Args {
  const double2 *F;   // analysis input
  double2 *S;         // analysis output
  const double2 *Sc;  // synthesis input
  double2 *Fo;        // synthesis output
  const double *P;
  const long long *poff;
  const int *rowoff;
  const int2 *pairs;  // (ma, mb), mb = -1 for a lone band
  int ntiles, nitems, per_cta;
  int N, J, JH, ncol;
};

using dmma::cp16;
using dmma::cp_commit;
using dmma::cp_wait0;
using dmma::cp_wait1;
using dmma::mma884;

// Stage the Legendre rows of the pair: m_a rows at 0.., m_b rows right after.
template <int JH>
__device__ void load_pair_P(const V2Args &a, const Geo &g, double *Pbuf, int ma, int mb)
{
  constexpr int cpr = JH / 2;  // 16-byte chunks per row
  const int Ra = a.N + 2 - ma, Rb = (mb >= 0) ? a.N + 2 - mb : 0;
  const int total = (Ra + Rb) * cpr;
  const double *Pa = a.P + a.poff[ma];
  const double *Pb = (mb >= 0) ? a.P + a.poff[mb] : Pa;
  for (int q = threadIdx.x; q < total; q += kT) {
    const int row = q / cpr, ch = q % cpr;
    const double *src = (row < Ra) ? Pa + (long long)row * JH : Pb + (long long)(row - Ra) * JH;
    cp16(Pbuf + row * g.PS + 2 * ch, src + 2 * ch, true);
  }
}

// ------------------------------------------------------------------ analysis
// Thread q copies latitude (q mod J) of column rows q/J, q/J + kT/J, ...
template <int JH, int CT>
__device__ void load_F_panels(const V2Args &a, const Geo &g, double *buf, int ma, int mb, int col0)
{
  constexpr int J = 2 * JH, RSTEP = kT / J;  // column rows covered per pass
  const int nrow = (mb >= 0) ? 2 * CT : CT;
  const int j = threadIdx.x % J;
#pragma unroll 4
  for (int row = threadIdx.x / J; row < nrow; row += RSTEP) {
    const int mi = row / CT, b = row % CT;
    const int m = mi ? mb : ma;
    const bool ok = col0 + b < a.ncol;
    const double2 *src = ok ? a.F + ((long long)m * a.ncol + col0 + b) * J + j : a.F;
    cp16(buf + row * g.CS + 2 * j, src, ok);
  }
}

template <int JH, int CT>
__global__ void __launch_bounds__(kT, 2) k_leg_fwd_pair(V2Args a)
{
  // One data panel per block and two blocks per SM: each block's panel load
  // overlaps the other block's products.
  extern __shared__ __align__(16) double sm[];
  const Geo g = make_geo(a.N, 2 * JH, true);
  double *Pbuf = sm;
  double *const G0 = sm + g.prow_cap * g.PS;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int it0 = blockIdx.x * a.per_cta;
  const int it1 = min(a.nitems, it0 + a.per_cta);
  if (it0 >= it1) return;

  int cur = -1;
  for (int it = it0; it < it1; ++it) {
    const int pidx = it / a.ntiles, col0 = (it - pidx * a.ntiles) * CT;
    const int2 pr = a.pairs[pidx];
    if (pidx != cur) {
      load_pair_P<JH>(a, g, Pbuf, pr.x, pr.y);
      cur = pidx;
    }
    load_F_panels<JH, CT>(a, g, G0, pr.x, pr.y, col0);
    cp_commit();
    cp_wait0();
    __syncthreads();
    double *const Gcur = G0;  // column rows: Gs at [0, JH), Ga at [JH, J)
    {
      // The panel's Fourier lines are in shared memory now and no later kernel
      // reads them: drop them from L2 without a write-back.  A column row is
      // J complex values, a whole number of 128-byte lines.
      constexpr int LPR = 2 * JH * 16 / 128;
      const int nrow = (pr.y >= 0) ? 2 * CT : CT;
      for (int q = threadIdx.x; q < nrow * LPR; q += kT) {
        const int row = q / LPR, b = row % CT, m = (row / CT) ? pr.y : pr.x;
        if (col0 + b < a.ncol)
          l2::discard_line(reinterpret_cast<const char *>(a.F + ((long long)m * a.ncol + col0 + b) * (2 * JH)) +
                           128 * (q % LPR));
      }
    }

    // jobs: (band, parity, 16-row group)
    const int Ra = a.N + 2 - pr.x, Rb = (pr.y >= 0) ? a.N + 2 - pr.y : 0;
    const int gEa = ((Ra + 1) / 2 + 15) / 16, gOa = (Ra / 2 + 15) / 16;
    const int gEb = ((Rb + 1) / 2 + 15) / 16, gOb = (Rb / 2 + 15) / 16;
    const int njobs = gEa + gOa + gEb + gOb;
    for (int job = warp; job < njobs; job += kW) {
      int mi, par, gi;
      if (job < gEa) { mi = 0; par = 0; gi = job; }
      else if (job < gEa + gOa) { mi = 0; par = 1; gi = job - gEa; }
      else if (job < gEa + gOa + gEb) { mi = 1; par = 0; gi = job - gEa - gOa; }
      else { mi = 1; par = 1; gi = job - gEa - gOa - gEb; }
      const int m = mi ? pr.y : pr.x, R = mi ? Rb : Ra;
      const double *Pm = Pbuf + (mi ? Ra : 0) * g.PS;
      const double *G = Gcur + mi * CT * g.CS + (par ? 2 * JH : 0);
      const int r0 = par + 2 * (16 * gi + (lane >> 2));
      const int r1 = r0 + 16;
      // the job's second 8-row tile holds rows of this parity only when the
      // parity has more than 16 gi + 8 of them; otherwise its products are
      // skipped (an eighth to a quarter of the tiles at T42-T85)
      const int cnt = par ? R / 2 : (R + 1) / 2;
      const bool two = 16 * gi + 8 < cnt;
      // K order within each pair of k-steps: lane q = lane & 3 takes latitude
      // 8j + 2q in the first and 8j + 2q + 1 in the second, so one 16-byte
      // load gives a lane both A values.  The columns form four 8-column
      // tiles (colrow half h, real / imaginary part): one 16-byte load gives a
      // lane the B values (re, im) of its colrow for two tiles.
      const int q = lane & 3;
      const double *pa0 = Pm + min(r0, R - 1) * g.PS + 2 * q;
      const double *pa1 = Pm + min(r1, R - 1) * g.PS + 2 * q;
      const double *gb = G + (lane >> 2) * g.CS + 4 * q;
      constexpr int NH = CT / 8;
      double acc[2][NH][2][2];  // [row tile][colrow half][re/im][2 columns]
#pragma unroll
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int h = 0; h < NH; ++h)
#pragma unroll
          for (int pt = 0; pt < 2; ++pt) acc[t][h][pt][0] = acc[t][h][pt][1] = 0.0;
      if (two) {
#pragma unroll
        for (int kb = 0; kb < JH; kb += 8) {
          const double2 a0 = *reinterpret_cast<const double2 *>(pa0 + kb);
          const double2 a1 = *reinterpret_cast<const double2 *>(pa1 + kb);
#pragma unroll
          for (int h = 0; h < NH; ++h) {
            const double2 be = *reinterpret_cast<const double2 *>(gb + 8 * h * g.CS + 2 * kb);      // latitude 8j + 2q
            const double2 bo = *reinterpret_cast<const double2 *>(gb + 8 * h * g.CS + 2 * kb + 2);  // latitude 8j + 2q + 1
            mma884(acc[0][h][0], a0.x, be.x);
            mma884(acc[0][h][1], a0.x, be.y);
            mma884(acc[1][h][0], a1.x, be.x);
            mma884(acc[1][h][1], a1.x, be.y);
            mma884(acc[0][h][0], a0.y, bo.x);
            mma884(acc[0][h][1], a0.y, bo.y);
            mma884(acc[1][h][0], a1.y, bo.x);
            mma884(acc[1][h][1], a1.y, bo.y);
          }
        }
      } else {
#pragma unroll
        for (int kb = 0; kb < JH; kb += 8) {
          const double2 a0 = *reinterpret_cast<const double2 *>(pa0 + kb);
#pragma unroll
          for (int h = 0; h < NH; ++h) {
            const double2 be = *reinterpret_cast<const double2 *>(gb + 8 * h * g.CS + 2 * kb);
            const double2 bo = *reinterpret_cast<const double2 *>(gb + 8 * h * g.CS + 2 * kb + 2);
            mma884(acc[0][h][0], a0.x, be.x);
            mma884(acc[0][h][1], a0.x, be.y);
            mma884(acc[0][h][0], a0.y, bo.x);
            mma884(acc[0][h][1], a0.y, bo.y);
          }
        }
      }
      const long long rowbase = a.rowoff[m];
#pragma unroll
      for (int t = 0; t < 2; ++t) {
        const int r = par + 2 * (16 * gi + 8 * t + (lane >> 2));
        if (r >= R) continue;
#pragma unroll
        for (int h = 0; h < NH; ++h)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int c = col0 + 8 * h + 2 * q + e;
            if (c < a.ncol) a.S[(rowbase + r) * a.ncol + c] = make_double2(acc[t][h][0][e], acc[t][h][1][e]);
          }
      }
    }
    __syncthreads();
  }
  cp_wait0();
}

// ----------------------------------------------------------------- synthesis
// Thread q copies column (q mod kCT) of coefficient rows q/kCT, q/kCT + kT/kCT, ...
__device__ void load_S_panels(const V2Args &a, const Geo &g, double *buf, int ma, int mb, int col0)
{
  constexpr int RSTEP = kT / kCT;
  const int nm = (mb >= 0) ? 2 : 1;
  const int c = threadIdx.x % kCT;
  const bool cok = col0 + c < a.ncol;
  const int Ra = a.N + 2 - ma, Rb = (mb >= 0) ? a.N + 2 - mb : 0;
  const double2 *Sa = a.Sc + (long long)a.rowoff[ma] * a.ncol + col0 + c;
  const double2 *Sb = (mb >= 0) ? a.Sc + (long long)a.rowoff[mb] * a.ncol + col0 + c : Sa;
#pragma unroll 4
  for (int row = threadIdx.x / kCT; row < nm * g.arow_cap; row += RSTEP) {
    const bool second = row >= g.arow_cap;
    const int r = second ? row - g.arow_cap : row;
    const bool ok = cok && r < (second ? Rb : Ra);
    const double2 *src = ok ? (second ? Sb : Sa) + (long long)r * a.ncol : a.Sc;
    cp16(buf + row * g.AS + 2 * c, src, ok);
  }
}

template <int JH>
__global__ void __launch_bounds__(kT, 1) k_leg_inv_pair(V2Args a)
{
  extern __shared__ __align__(16) double sm[];
  const Geo g = make_geo(a.N, 2 * JH, false);
  double *Pbuf = sm;
  const int abuf = 2 * g.arow_cap * g.AS;
  double *const A0 = sm + g.prow_cap * g.PS, *const A1 = A0 + abuf;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int it0 = blockIdx.x * a.per_cta;
  const int it1 = min(a.nitems, it0 + a.per_cta);
  if (it0 >= it1) return;
  // units: (latitude tile of 8, group of column tiles) over the 8 warps
  constexpr int ntj = JH / 8;             // 2, 4 or 8
  constexpr int ngrp = kW / ntj;          // 4, 2 or 1
  constexpr int nnt = 4 / ngrp;           // column tiles (of 8 reals) per unit
  const int jt = warp % ntj, grp = warp / ntj;
  const uint64_t keep = l2::keep_policy();  // the Fourier runs stay in L2 for the longitude transform

  {
    const int2 pr = a.pairs[it0 / a.ntiles];
    load_S_panels(a, g, A0, pr.x, pr.y, (it0 % a.ntiles) * kCT);
    cp_commit();
  }
  int cur = -1;
  for (int it = it0; it < it1; ++it) {
    const int bsel = (it - it0) & 1;
    const int pidx = it / a.ntiles, col0 = (it - pidx * a.ntiles) * kCT;
    const int2 pr = a.pairs[pidx];
    if (pidx != cur) {
      load_pair_P<JH>(a, g, Pbuf, pr.x, pr.y);
      cur = pidx;
    }
    cp_commit();
    if (it + 1 < it1) {
      const int2 pn = a.pairs[(it + 1) / a.ntiles];
      load_S_panels(a, g, bsel ? A0 : A1, pn.x, pn.y, ((it + 1) % a.ntiles) * kCT);
    }
    cp_commit();
    cp_wait1();
    __syncthreads();

    const int Ra = a.N + 2 - pr.x;
    const int nm = (pr.y >= 0) ? 2 : 1;
    for (int mi = 0; mi < nm; ++mi) {
      const int m = mi ? pr.y : pr.x, R = a.N + 2 - m;
      const double *Pm = Pbuf + (mi ? Ra : 0) * g.PS;
      const double *A = (bsel ? A1 : A0) + mi * g.arow_cap * g.AS;
      double acc[2][4][2];  // [parity][column tile][2]
#pragma unroll
      for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) acc[p][nt][0] = acc[p][nt][1] = 0.0;
      const int jcol = 8 * jt + (lane >> 2);
      // both parities in one loop (8 independent product chains per warp):
      // the odd rows run to the even count, their coefficient rows past R are
      // the zeroed tail of the panel
      const int kp = (R + 1) / 2;
      if constexpr (nnt % 2 == 0) {
        // columns as (real part, imaginary part) tile pairs of 8 complex
        // columns: one 16-byte load gives a lane its B values for both tiles
        const int cb = 4 * grp * nnt;  // first complex column of this warp
        for (int t0 = 0; t0 < kp; t0 += 4) {
          const int r = 2 * (t0 + (lane & 3));
          const double av0 = Pm[min(r, R - 1) * g.PS + jcol], av1 = Pm[min(r + 1, R - 1) * g.PS + jcol];
          const double *brow = A + r * g.AS + 2 * (cb + (lane >> 2));
#pragma unroll
          for (int u2 = 0; u2 < nnt / 2; ++u2) {
            const double2 b0 = *reinterpret_cast<const double2 *>(brow + 16 * u2);
            const double2 b1 = *reinterpret_cast<const double2 *>(brow + g.AS + 16 * u2);
            mma884(acc[0][2 * u2], av0, b0.x);
            mma884(acc[0][2 * u2 + 1], av0, b0.y);
            mma884(acc[1][2 * u2], av1, b1.x);
            mma884(acc[1][2 * u2 + 1], av1, b1.y);
          }
        }
        const int jh = 8 * jt + (lane >> 2);
#pragma unroll
        for (int u2 = 0; u2 < nnt / 2; ++u2)
#pragma unroll
          for (int e = 0; e < 2; ++e) {
            const int c = col0 + cb + 8 * u2 + 2 * (lane & 3) + e;
            if (c >= a.ncol) continue;
            double2 *Fc = a.Fo + ((long long)m * a.ncol + c) * (2 * JH);
            l2::st_keep(Fc + jh, make_double2(acc[0][2 * u2][e], acc[0][2 * u2 + 1][e]), keep);       // even degrees
            l2::st_keep(Fc + JH + jh, make_double2(acc[1][2 * u2][e], acc[1][2 * u2 + 1][e]), keep);  // odd degrees
          }
      } else {
        for (int t0 = 0; t0 < kp; t0 += 4) {
          const int r = 2 * (t0 + (lane & 3));
          const double av0 = Pm[min(r, R - 1) * g.PS + jcol], av1 = Pm[min(r + 1, R - 1) * g.PS + jcol];
          const double *brow = A + r * g.AS + (lane >> 2);
#pragma unroll
          for (int q = 0; q < 4; ++q)
            if (q < nnt) {
              mma884(acc[0][q], av0, brow[8 * (grp * nnt + q)]);
              mma884(acc[1][q], av1, brow[g.AS + 8 * (grp * nnt + q)]);
            }
        }
        const int jh = 8 * jt + (lane >> 2);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          if (q >= nnt) continue;
          const int c = col0 + 4 * (grp * nnt + q) + (lane & 3);
          if (c >= a.ncol) continue;
          double2 *Fc = a.Fo + ((long long)m * a.ncol + c) * (2 * JH);
          l2::st_keep(Fc + jh, make_double2(acc[0][q][0], acc[0][q][1]), keep);       // even degrees
          l2::st_keep(Fc + JH + jh, make_double2(acc[1][q][0], acc[1][q][1]), keep);  // odd degrees
        }
      }
    }
    __syncthreads();
  }
  cp_wait0();
}

size_t fwd_smem(int N, int J, int ct)
{
  const Geo g = make_geo(N, J, true);
  return sizeof(double) * ((size_t)g.prow_cap * g.PS + 2 * ct * (size_t)g.CS);
}

// analysis columns per item: the plan's tile choice when its panel fits
int fwd_ct(const sht_plan *p)
{
  const int t = p->leg_tile;
  if ((t == 8 || t == 16) && fwd_smem(p->N, p->J, t) <= 227 * 1024) return t;
  return ct_fwd(p->JH);
}
size_t inv_smem(int N, int J)
{
  const Geo g = make_geo(N, J, false);
  return sizeof(double) * ((size_t)g.prow_cap * g.PS + 2 * 2 * (size_t)g.arow_cap * g.AS);
}

int get_pairs(const sht_plan *p, const int2 **out, int *n)
{
  // The pair list is a pure function of N; it is kept per plan in d_pairs.
  *out = p->d_pairs;
  *n = p->n_pairs;
  return (p->d_pairs && p->n_pairs > 0) ? SHT_OK : SHT_ERR_NOT_INITIALIZED;
}

int launch_pair(const sht_plan *p, bool inverse, const double2 *in, int ncol, double2 *out, cudaStream_t s)
{
  V2Args a{};
  if (inverse) { a.Sc = in; a.Fo = out; } else { a.F = in; a.S = out; }
  a.P = p->d_P; a.poff = p->d_poff; a.rowoff = p->d_rowoff;
  a.N = p->N; a.J = p->J; a.JH = p->JH; a.ncol = ncol;
  int npairs = 0;
  int rc = get_pairs(p, &a.pairs, &npairs);
  if (rc) { set_error("legendre: pair table missing"); return rc; }
  const int ct = inverse ? kCT : fwd_ct(p);
  a.ntiles = (ncol + ct - 1) / ct;
  a.nitems = npairs * a.ntiles;
  const size_t smem = inverse ? inv_smem(p->N, p->J) : fwd_smem(p->N, p->J, ct);
  void (*kern)(V2Args) = nullptr;
  switch (p->JH * 100 + (inverse ? 0 : ct)) {
  case 1600: case 3200: case 6400:
    kern = p->JH == 16 ? k_leg_inv_pair<16> : p->JH == 32 ? k_leg_inv_pair<32> : k_leg_inv_pair<64>;
    break;
  case 1608: kern = k_leg_fwd_pair<16, 8>; break;
  case 1616: kern = k_leg_fwd_pair<16, 16>; break;
  case 3208: kern = k_leg_fwd_pair<32, 8>; break;
  case 3216: kern = k_leg_fwd_pair<32, 16>; break;
  case 6408: kern = k_leg_fwd_pair<64, 8>; break;
  case 6416: kern = k_leg_fwd_pair<64, 16>; break;
  default: set_error("legendre: latitude count outside the paired kernels"); return SHT_ERR_UNSUPPORTED_SIZE;
  }
  int per_sm = 0;
  cudaError_t e = kernel_setup((const void *)kern, smem, kT, &per_sm);
  if (e != cudaSuccess || per_sm < 1) return cuda_fail(e == cudaSuccess ? cudaErrorInvalidConfiguration : e, "legendre pair occupancy");
  const int slots = grid_sms(p) * per_sm;
  a.per_cta = (a.nitems + slots - 1) / slots;
  const int grid = (a.nitems + a.per_cta - 1) / a.per_cta;
  kern<<<grid, kT, smem, s>>>(a);
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, inverse ? "k_leg_inv_pair" : "k_leg_fwd_pair");
}

}  // namespace

bool leg_pair_supported(const sht_plan *p)
{
  if (p->J % 16 != 0 || (p->JH != 16 && p->JH != 32 && p->JH != 64)) return false;
  const size_t lim = 227 * 1024;
  return fwd_smem(p->N, p->J, ct_fwd(p->JH)) <= lim && inv_smem(p->N, p->J) <= lim;
}

int launch_leg_fwd_pair(const sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  return launch_pair(p, false, F, ncol, S, s);
}

int launch_leg_inv_pair(const sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  return launch_pair(p, true, S, ncol, F, s);
}

}  // namespace sht
