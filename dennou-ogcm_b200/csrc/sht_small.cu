// sht_small.cu -- whole plain transforms of small grids, one kernel per
// direction (SHT_OPT_LEGENDRE_KERNEL = 4).
//
// For im <= 128 the longitude transform, the Legendre contraction and the
// SPML layout conversion of a group of G = 2 field-levels run in one thread
// block, and the Fourier coefficients and the spectra never leave shared
// memory:
//
//   analysis  (w_xy):  grid rows --FFT--> Gs/Ga[m][jh] (shared) --P-->
//             S(n, m) --> wa row in SPML order (staged, written contiguously)
//   synthesis (xy_w):  wa row --> a(n, m) (shared) --P--> E/O[m][jh] (shared)
//             --inverse FFT--> grid rows
//
// HBM traffic is the grid and the spectra once each, against the Fourier
// array and the internal spectral array written and read between the four
// kernels of the batched path.  The FFT tiles are the batched kernels' own
// (sht_fft_tile.cuh).  The contractions run on the FP64 tensor path
// (mma.sync.m8n8k4.f64): M = 8 output rows (degrees of one parity in the
// analysis, latitudes in the synthesis), K = latitudes or degrees in steps of
// 4, N = the 2G real columns (re and im of each level; half of the 8 columns
// stay empty).  Warps take (order, parity, 8-row group) units in turn.  The
// sums follow space_discretization.tex:197-200 (analysis) and :212-216
// (synthesis) with the same row factors, parities and SPML scaling (sqrt 2
// for m > 0, SpmlUtil's wa layout) as the batched path.
//
// It is faster than the batched path only for the smallest grids (T10: 480
// field-levels round trip 31 against 59 us): each block re-reads the Legendre
// table for its two levels, where the batched kernels use every table row on
// 8 to 16 columns, and its phases (loads, transform, contraction, stores) run
// one after the other in blocks that the shared-memory arrays keep few per SM.
// The multi-instance tuner times it beside the batched kernels per plan.
#include "sht_fft_tile.cuh"
#include "sht_dmma.cuh"

namespace sht {

namespace {

constexpr double kSqrt2s = 1.41421356237309504880;
constexpr double kRSqrt2s = 0.70710678118654752440;

struct SmallArgs {
  FftArgs f;                   // rowscale, twiddles, I, J, JH, N (grid pointers unused)
  const double *g;             // analysis: input grids, level c at g + c I J (or gcol[c])
  const double *const *gcol;
  double *go;                  // synthesis: output grids (or gocol[c])
  double *const *gocol;
  const double *w;             // synthesis: input spectra, level c at w + c L (or wcol[c])
  const double *const *wcol;
  double *wo;                  // analysis: output spectra (or wocol[c])
  double *const *wocol;
  const double *P;             // Legendre rows: band m, row r = n - m at P + table_off(m) + r JH
  int ncol, L, bufe;
};

// offset of band m in a level's coefficient array (rows n = m..N)
__device__ __forceinline__ int band_off(int N, int m) { return m * (N + 1) - m * (m - 1) / 2; }
// offset of band m in the Legendre table (N + 2 - m rows of JH latitudes each;
// the plan's offset list in closed form, so no load precedes the table reads)
__device__ __forceinline__ int table_off(int N, int JH, int m) { return JH * (m * (N + 2) - m * (m - 1) / 2); }

template <int A, int B, int NT, int G>
struct SmallShape {
  using S = FftShape<A, B, NT>;
  static size_t smem_fwd(int N, int J, int bufe)
  {
    const size_t L = (size_t)(N + 1) * (N + 1);
    return sizeof(double2) * (2 * (size_t)S::NC + bufe + (size_t)G * (N + 1) * J) + sizeof(double) * G * L;
  }
  static size_t smem_inv(int N, int J, int bufe)
  {
    const size_t R = (size_t)(N + 1) * (N + 2) / 2;
    return sizeof(double2) * (2 * (size_t)S::NC + bufe + (size_t)G * (N + 1) * J + (size_t)G * R);
  }
};

// ------------------------------------------------------------------ analysis
template <int A, int B, int NT, int G>
__global__ void __launch_bounds__(NT, 1) k_small_fwd(SmallArgs a)
{
  using S = FftShape<A, B, NT>;
  constexpr int R1 = S::R1, R2 = S::R2, NC = S::NC, T = S::T, JTh = S::JT / 2, NW = NT / 32;
  extern __shared__ __align__(16) double2 smem_all[];
  const FftArgs &f = a.f;
  const int N = f.N, J = f.J, JH = f.JH, L = a.L, M1 = N + 1;
  double2 *stw = smem_all, *stwI = stw + NC, *cur = stwI + NC;
  double2 *Fs = cur + a.bufe;                                       // [G][M1][J]: Gs at jh, Ga at JH + jh
  double *Sout = reinterpret_cast<double *>(Fs + (size_t)G * M1 * J);  // [G][L]
  load_twiddles<T, NC, NT>(f, stw, stwI);
  __syncthreads();

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r = tid / T, u = tid % T;
  const int ntile = (JH + JTh - 1) / JTh;
  const long long IJ = (long long)f.I * J;
  const int ngroups = (a.ncol + G - 1) / G;
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const int c0 = grp * G, ng = min(G, a.ncol - c0);
    // 1. the longitude transforms of the group's levels, into Fs
    for (int t = 0; t < ng * ntile; ++t) {
      const int g = t / ntile, h0 = (t - g * ntile) * JTh, col = c0 + g;
      const int jh = h0 + (r % JTh), j = r < JTh ? JH + jh : JH - 1 - jh;
      const bool valid = jh < JH;
      const double *gb = a.gcol ? a.gcol[col] : a.g + (long long)col * IJ;
      const double2 *src = reinterpret_cast<const double2 *>(gb) + (long long)(valid ? j : 0) * NC;
      double2 v[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) v[n1] = valid ? __ldcs(src + R2 * n1 + u) : make_double2(0.0, 0.0);
      fwd_tile<A, B, NT, true>(f, v, cur, stw, stwI, col, h0, j, valid, Fs + (size_t)g * M1 * J);
      __syncthreads();  // the tile buffer is reused; Fs is complete after the last tile
    }
    // 2. the contraction, S(n, m) = sum_jh P[m][n - m][jh] (Gs or Ga)[m][jh],
    //    staged in SPML order (sqrt 2 on m > 0)
    {
      const int bcol = lane >> 2, lev_b = bcol >> 1, part_b = bcol & 1, kq = lane & 3;
      int uc = 0;
      for (int m = 0; m <= N; ++m) {
        const int Rp = N + 1 - m;
        const double *Pm = a.P + table_off(N, JH, m);
        for (int par = 0; par < 2; ++par) {
          const int rows = par ? Rp / 2 : (Rp + 1) / 2;
          for (int g8 = 0; g8 < rows; g8 += 8, ++uc) {
            if (uc % NW != warp) continue;
            const int ra = g8 + (lane >> 2);  // this lane's A row (index within the parity)
            const bool oka = ra < rows;
            const double *pa = Pm + (long long)(par + 2 * ra) * JH + kq;
            const double *pb = reinterpret_cast<const double *>(Fs + (size_t)lev_b * M1 * J + m * J + par * JH) +
                               2 * kq + part_b;
            const bool okb = lev_b < ng;
            // eight k-steps' fragments are loaded before their products (the
            // table reads overlap one another), and the products alternate
            // between two accumulators (two dependence chains)
            double acc[2] = {0.0, 0.0}, acc2[2] = {0.0, 0.0};
            const int KK = JH;
            for (int k0 = 0; k0 < JH; k0 += 32) {
              double av[8], bv[8];
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const int kb = k0 + 4 * q;
                av[q] = (oka && kb < JH) ? __ldg(pa + kb) : 0.0;
                bv[q] = (okb && kb < JH) ? pb[2 * kb] : 0.0;
              }
#pragma unroll
              for (int q = 0; q < 8; q += 2) {  // no products past the contraction's end (uniform)
                if (k0 + 4 * q < KK) dmma::mma884(acc, av[q], bv[q]);
                if (k0 + 4 * q + 4 < KK) dmma::mma884(acc2, av[q + 1], bv[q + 1]);
              }
            }
            acc[0] += acc2[0];
            acc[1] += acc2[1];
            // this lane: row g8 + lane/4, columns 2 (lane % 4) + {0, 1} = re, im of level lane % 4
            const int lev = lane & 3, rc = g8 + (lane >> 2);
            if (lev < ng && rc < rows) {
              const int n = m + par + 2 * rc;
              const double s = m == 0 ? 1.0 : kSqrt2s;
              double *so = Sout + (size_t)lev * L;
              so[n * (n + 1) + m] = acc[0] * s;
              if (m > 0) so[n * (n + 1) - m] = acc[1] * s;
            }
          }
        }
      }
    }
    __syncthreads();
    // 3. each level's spectrum as one contiguous row
    for (int g = 0; g < ng; ++g) {
      double *wo = a.wocol ? a.wocol[c0 + g] : a.wo + (long long)(c0 + g) * L;
      for (int l = tid; l < L; l += NT) wo[l] = Sout[(size_t)g * L + l];
    }
    __syncthreads();  // Fs, Sout and the tile buffer are refilled by the next group
  }
}

// ----------------------------------------------------------------- synthesis
template <int A, int B, int NT, int G>
__global__ void __launch_bounds__(NT, 1) k_small_inv(SmallArgs a)
{
  using S = FftShape<A, B, NT>;
  constexpr int R1 = S::R1, R2 = S::R2, NC = S::NC, T = S::T, JTh = S::JT / 2, NW = NT / 32;
  constexpr int NS = R1 / T;
  extern __shared__ __align__(16) double2 smem_all[];
  const FftArgs &f = a.f;
  const int N = f.N, J = f.J, JH = f.JH, L = a.L, M1 = N + 1;
  const int R = (N + 1) * (N + 2) / 2;
  double2 *stw = smem_all, *stwI = stw + NC, *cur = stwI + NC;
  double2 *Fs = cur + a.bufe;              // [G][M1][J]: E at jh, O at JH + jh
  double2 *Ain = Fs + (size_t)G * M1 * J;  // [G][R]: a(n, m) at band_off(m) + n - m
  load_twiddles<T, NC, NT>(f, stw, stwI);
  __syncthreads();

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int r = tid / T, u = tid % T;
  const int ntile = (JH + JTh - 1) / JTh;
  const long long IJ = (long long)f.I * J;
  const int ngroups = (a.ncol + G - 1) / G;
  for (int grp = blockIdx.x; grp < ngroups; grp += gridDim.x) {
    const int c0 = grp * G, ng = min(G, a.ncol - c0);
    // 1. the group's spectra, read as contiguous rows: entry l = n (n + 1) +- m
    //    is the cos (+) or sin (-) part of a(n, m), scaled by 1/sqrt 2 for m > 0
    for (int g = 0; g < ng; ++g) {
      const double *w = a.wcol ? a.wcol[c0 + g] : a.w + (long long)(c0 + g) * L;
      double2 *ag = Ain + (size_t)g * R;
      // warps over degrees n, lanes over orders m: the cos parts of a degree
      // are one contiguous run of w, the sin parts another
      for (int n = warp; n <= N; n += NW) {
        const int base = n * (n + 1);
        for (int m = lane; m <= n; m += 32) {
          const double c = __ldg(w + base + m);
          const double sn = m > 0 ? __ldg(w + base - m) : 0.0;
          const double sc = m == 0 ? 1.0 : kRSqrt2s;
          ag[band_off(N, m) + (n - m)] = make_double2(c * sc, sn * sc);
        }
      }
    }
    __syncthreads();
    // 2. the contraction, E/O[m][jh] = sum over degrees n of the parity of
    //    P[m][n - m][jh] a(n, m)
    {
      const int bcol = lane >> 2, lev_b = bcol >> 1, part_b = bcol & 1, kq = lane & 3;
      const int njg = (JH + 7) / 8;
      int uc = 0;
      for (int m = 0; m <= N; ++m) {
        const int Rp = N + 1 - m;
        const double *Pm = a.P + table_off(N, JH, m);
        for (int par = 0; par < 2; ++par) {
          const int rows = par ? Rp / 2 : (Rp + 1) / 2;
          for (int jg = 0; jg < njg; ++jg, ++uc) {
            if (uc % NW != warp) continue;
            const int jh_a = 8 * jg + (lane >> 2);  // this lane's A row (latitude)
            const bool oka = jh_a < JH;
            const double *pa = Pm + (long long)(par + 2 * kq) * JH + jh_a;
            const double *pb = reinterpret_cast<const double *>(Ain + (size_t)lev_b * R + band_off(N, m) + par + 2 * kq) +
                               part_b;
            const bool okb = lev_b < ng;
            double acc[2] = {0.0, 0.0}, acc2[2] = {0.0, 0.0};
            const int KK = rows;
            for (int k0 = 0; k0 < rows; k0 += 32) {
              double av[8], bv[8];
#pragma unroll
              for (int q = 0; q < 8; ++q) {
                const int kb = k0 + 4 * q;
                const bool okk = kb + kq < rows;
                av[q] = (oka && okk) ? __ldg(pa + (long long)(2 * kb) * JH) : 0.0;
                bv[q] = (okb && okk) ? pb[4 * kb] : 0.0;
              }
#pragma unroll
              for (int q = 0; q < 8; q += 2) {  // no products past the contraction's end (uniform)
                if (k0 + 4 * q < KK) dmma::mma884(acc, av[q], bv[q]);
                if (k0 + 4 * q + 4 < KK) dmma::mma884(acc2, av[q + 1], bv[q + 1]);
              }
            }
            acc[0] += acc2[0];
            acc[1] += acc2[1];
            // this lane: latitude 8 jg + lane/4, re and im of level lane % 4
            const int lev = lane & 3, jc = 8 * jg + (lane >> 2);
            if (lev < ng && jc < JH) Fs[(size_t)lev * M1 * J + m * J + par * JH + jc] = make_double2(acc[0], acc[1]);
          }
        }
      }
    }
    __syncthreads();
    // 3. the inverse longitude transforms of the group's levels
    for (int t = 0; t < ng * ntile; ++t) {
      const int g = t / ntile, h0 = (t - g * ntile) * JTh, col = c0 + g;
      const int jh = h0 + (r % JTh), j = r < JTh ? JH + jh : JH - 1 - jh;
      const bool valid = jh < JH;
      // this row's G^k: north = E + O (rows < JTh), south = E - O
      const double2 *Fg = Fs + (size_t)g * M1 * J + h0 + (r % JTh);
      const double sgn = r < JTh ? 1.0 : -1.0;
      auto gm = [&](int k) {
        const double2 e = valid ? Fg[k * J] : make_double2(0.0, 0.0);
        const double2 o = valid ? Fg[k * J + JH] : make_double2(0.0, 0.0);
        return make_double2(e.x + sgn * o.x, e.y + sgn * o.y);
      };
      double2 v[R1];
      inv_pack<A, B, NT>(N, gm, stwI, v);
      inv_transform<A, B, NT>(v, cur, stw, [&](const double2 (&z)[NS][R2]) {
        if (!valid) return;
        double *dst = a.gocol ? a.gocol[col] : a.go + (long long)col * IJ;
        double2 *rowp = reinterpret_cast<double2 *>(dst + (long long)j * f.I);
        const double sc = __ldg(f.rowscale + j);
#pragma unroll
        for (int s = 0; s < NS; ++s)
#pragma unroll
          for (int k2 = 0; k2 < R2; ++k2) {
            const double2 w = z[s][brev<B>(k2)];
            rowp[u + T * s + R1 * k2] = make_double2(w.x * sc, w.y * sc);
          }
      });
      __syncthreads();  // the tile buffer is reused by the next tile
    }
  }
}

// Shapes: T42 (NC 64) in 256-thread blocks, smaller grids in 128-thread
// blocks; two levels per group (four measured no faster at T21 and slower at
// T10: fewer blocks per SM).
template <int A, int B>
struct SmallCfg {
  static constexpr int NC = 1 << (A + B);
  static constexpr int NT = NC >= 64 ? 256 : 128;
  static constexpr int G = 2;
};

template <int A, int B>
int run_small(bool inverse, const sht_plan *p, SmallArgs a, cudaStream_t s)
{
  using C = SmallCfg<A, B>;
  using Sh = SmallShape<A, B, C::NT, C::G>;
  a.bufe = FftShape<A, B, C::NT>::buf_elems(p->N);
  const size_t smem = inverse ? Sh::smem_inv(p->N, p->J, a.bufe) : Sh::smem_fwd(p->N, p->J, a.bufe);
  if (smem > 227 * 1024) { set_error("small-grid transform: shared memory too large"); return SHT_ERR_UNSUPPORTED_SIZE; }
  const int ngroups = (a.ncol + C::G - 1) / C::G;
  void (*kern)(SmallArgs) = inverse ? k_small_inv<A, B, C::NT, C::G> : k_small_fwd<A, B, C::NT, C::G>;
  int occ = 0;
  cudaError_t e = kernel_setup((const void *)kern, smem, C::NT, &occ);
  if (e != cudaSuccess) return cuda_fail(e, "small-grid transform smem attribute");
  const int g = (occ < 1 ? 1 : occ) * grid_sms(p);
  kern<<<ngroups < g ? ngroups : g, C::NT, smem, s>>>(a);
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, inverse ? "k_small_inv" : "k_small_fwd");
}

// shared memory of the larger of the two directions' blocks on this plan
template <int A, int B>
size_t small_smem(const sht_plan *p)
{
  using C = SmallCfg<A, B>;
  using Sh = SmallShape<A, B, C::NT, C::G>;
  const int bufe = FftShape<A, B, C::NT>::buf_elems(p->N);
  const size_t f = Sh::smem_fwd(p->N, p->J, bufe), i = Sh::smem_inv(p->N, p->J, bufe);
  return f > i ? f : i;
}

int dispatch_small(bool inverse, const sht_plan *p, const SmallArgs &a, cudaStream_t s)
{
  switch (p->NC) {
  case 16: return run_small<2, 2>(inverse, p, a, s);
  case 32: return run_small<3, 2>(inverse, p, a, s);
  case 64: return run_small<3, 3>(inverse, p, a, s);
  default: set_error("small-grid transform: unsupported longitude count"); return SHT_ERR_UNSUPPORTED_SIZE;
  }
}

SmallArgs small_args(const sht_plan *p, int ncol, int rs)
{
  SmallArgs a{};
  a.f.rowscale = p->d_rowscale + (size_t)rs * p->J;
  a.f.tw = p->d_tw; a.f.twI = p->d_twI;
  a.f.I = p->I; a.f.J = p->J; a.f.JH = p->JH; a.f.N = p->N;
  a.P = p->d_P;
  a.ncol = ncol; a.L = p->L;
  return a;
}

}  // namespace

bool small_supported(const sht_plan *p)
{
  if (p->zonal || p->direct_dft || p->JH % 4 != 0 || p->JH > 64 || p->N + 1 > p->NC) return false;
  // the group's Fourier arrays must fit in one block's shared memory (not so
  // for, e.g., im = 128 with jm = 128 and nm = 63)
  const size_t lim = 227 * 1024;
  switch (p->NC) {
  case 16: return small_smem<2, 2>(p) <= lim;
  case 32: return small_smem<3, 2>(p) <= lim;
  case 64: return small_smem<3, 3>(p) <= lim;
  default: return false;
  }
}

int launch_small_fwd(const sht_plan *p, const double *g, const double *const *gcol, int ncol, double *w,
                     double *const *wcol, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  SmallArgs a = small_args(p, ncol, RS_FWD_PLAIN);
  a.g = g; a.gcol = gcol; a.wo = w; a.wocol = wcol;
  return dispatch_small(false, p, a, s);
}

int launch_small_inv(const sht_plan *p, const double *w, const double *const *wcol, int ncol, double *g,
                     double *const *gcol, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  SmallArgs a = small_args(p, ncol, RS_INV_PLAIN);
  a.w = w; a.wcol = wcol; a.go = g; a.gocol = gcol;
  return dispatch_small(true, p, a, s);
}

}  // namespace sht
