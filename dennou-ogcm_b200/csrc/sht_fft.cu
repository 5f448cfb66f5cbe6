// sht_fft.cu -- batched real FFT in longitude, FP64.
//
// Forward:  G^m(mu_j) = s_j * (1/I) sum_i q_ij e^{-i m lambda_i}, m = 0..N
//           (space_discretization.tex:190-193; s_j folds the Gauss weight and
//           the operator's row factor, e.g. 1/(1-mu^2) for w_DivMu_xy).
// Inverse:  q_ij = s_j sum_{m=-N..N} G^m e^{i m lambda_i}, G^{-m} = conj G^m
//           (space_discretization.tex:217-222).
//
// A real row of I = 2 NC points is packed as NC complex points, transformed by
// a four-step FFT with NC = R1 R2 (R1-point DFTs in registers, a twiddle, a
// transpose through shared memory, R2-point DFTs in registers), and unpacked
// with the usual half-length real-FFT identity.  Each tile of a thread block
// holds JT/2 mirrored pairs of Gauss rows of one field-level (north row
// JH + jh and south row JH - 1 - jh for jh0 <= jh < jh0 + JT/2), T = R2
// threads per row.  The Fourier array carries the equatorial symmetry that
// the Legendre contraction uses: F[m][col][jh] = G(north) + G(south) and
// F[m][col][JH + jh] = G(north) - G(south) in the analysis (Gs, Ga); in the
// synthesis the contraction writes the even- and odd-degree sums E and O
// there, and the inverse transform forms G(north) = E + O, G(south) = E - O.
// The output is staged in shared memory and written as runs of JT/2 rows.
// Shared-memory strides are padded so that each 8-lane phase of a 16-byte
// access touches eight distinct bank groups.
#include "sht_fft_tile.cuh"

#include <type_traits>

namespace sht {

// Forward transform, persistent over tiles (field-level, JT latitude rows).
// Each thread loads its R1 elements of row r (stride R2) from global memory
// straight into registers; the block's one shared buffer takes the transpose
// and the output staging.  Staging the tile with cp.async as well, in a
// second pair of buffers, cost blocks per SM and measured the same at T85 and
// 7-18 % slower at T170/T341.  Up to 16-point first passes the plain
// transform also holds the block's next tile in registers while it works on
// this one (3 instead of 4 blocks per SM at T85; forward 53 -> 52 us at T85,
// 0.314 -> 0.283 ms at T170, the same at T42).
// MUL: 0 plain, 1 product with the factor grid (FftArgs::mul), read the same way.
template <int A, int B, int NT, int MUL>
__global__ void __launch_bounds__(NT) k_fft_fwd(FftArgs a)
{
  using S = FftShape<A, B, NT>;
  constexpr int R1 = S::R1, R2 = S::R2, NC = S::NC, T = S::T, JT = S::JT;
  extern __shared__ __align__(16) double2 smem_all[];
  double2 *stw = smem_all, *stwI = smem_all + NC, *cur = smem_all + 2 * NC;
  load_twiddles<T, NC, NT>(a, stw, stwI);
  __syncthreads();

  constexpr int JTh = JT / 2;
  const int tid = threadIdx.x, r = tid / T, u = tid % T;
  const int ntile = (a.JH + JTh - 1) / JTh;
  // tile indices fit in 32 bits (the launcher checks), so the per-tile
  // division is a 32-bit one
  const unsigned ntot = (unsigned)a.ncol * (unsigned)ntile;
  const long long IJ = (long long)a.I * a.J;
  // tile t -> (column, first row pair); this thread's row j and whether it exists
  auto where = [&](unsigned t, int &col, int &h0, int &j, bool &valid) {
    // last column first: when a synthesis has just written the grid, its
    // last columns are the likeliest to be still in L2
    t = ntot - 1 - t;
    const int c2 = (int)(t / (unsigned)ntile);
    h0 = (int)(t - (unsigned)c2 * (unsigned)ntile) * JTh;
    col = a.mul_pair ? (c2 >> 1) + (c2 & 1) * a.nsplit : c2;
    const int jh = h0 + (r % JTh);
    j = r < JTh ? a.JH + jh : a.JH - 1 - jh;
    valid = jh < a.JH;
  };
  auto row_src = [&](int col, int j, bool valid) {
    const double *gb = a.gcol ? a.gcol[col]
                     : (col < a.nsplit) ? a.g0 + (long long)col * IJ : a.g1 + (long long)(col - a.nsplit) * IJ;
    return reinterpret_cast<const double2 *>(gb) + (long long)(valid ? j : 0) * NC;
  };
  if (MUL == 0 && A <= 4) {
    // The rows of the block's next tile are loaded into registers before
    // this tile is transformed, so their DRAM latency overlaps the DFTs
    // (not at 32-point first passes, where the second set would spill).
    unsigned t = blockIdx.x;
    double2 v[R1];
    if (t < ntot) {
      int col, h0, j; bool valid;
      where(t, col, h0, j, valid);
      const double2 *src = row_src(col, j, valid);
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) v[n1] = valid ? __ldcs(src + R2 * n1 + u) : make_double2(0.0, 0.0);
    }
    for (; t < ntot; t += gridDim.x) {
      double2 vn[R1];
      const unsigned tn = t + gridDim.x;
      if (tn < ntot) {
        int coln, h0n, jn; bool validn;
        where(tn, coln, h0n, jn, validn);
        const double2 *src = row_src(coln, jn, validn);
#pragma unroll
        for (int n1 = 0; n1 < R1; ++n1) vn[n1] = validn ? __ldcs(src + R2 * n1 + u) : make_double2(0.0, 0.0);
      }
      int col, h0, j; bool valid;
      where(t, col, h0, j, valid);
      fwd_tile<A, B, NT>(a, v, cur, stw, stwI, col, h0, j, valid);
      __syncthreads();  // the output runs are read; the next tile reuses the buffer
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) v[n1] = vn[n1];
    }
    return;
  }
  for (unsigned t = blockIdx.x; t < ntot; t += gridDim.x) {
    int col, h0, j; bool valid;
    where(t, col, h0, j, valid);
    const double2 *src = row_src(col, j, valid);
    double2 v[R1];
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) v[n1] = valid ? __ldcs(src + R2 * n1 + u) : make_double2(0.0, 0.0);
    if (MUL == 0) {
      fwd_tile<A, B, NT>(a, v, cur, stw, stwI, col, h0, j, valid);
      __syncthreads();
      continue;
    }
    const double2 *frow = reinterpret_cast<const double2 *>(a.mul + (long long)(col % a.nmul) * IJ) + (long long)(valid ? j : 0) * NC;
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) {
      const double2 q = valid ? __ldg(frow + R2 * n1 + u) : make_double2(0.0, 0.0);
      v[n1] = make_double2(v[n1].x * q.x, v[n1].y * q.y);
    }
    if (a.add0) {
      const double *zb = col < a.nsplit ? a.add0 + (long long)col * IJ : a.add1 + (long long)(col - a.nsplit) * IJ;
      const double2 *zrow = reinterpret_cast<const double2 *>(zb) + (long long)(valid ? j : 0) * NC;
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) {
        const double2 z = valid ? __ldg(zrow + R2 * n1 + u) : make_double2(0.0, 0.0);
        v[n1] = make_double2(v[n1].x + z.x, v[n1].y + z.y);
      }
    }
    fwd_tile<A, B, NT>(a, v, cur, stw, stwI, col, h0, j, valid);
    __syncthreads();  // the output runs are read; the next tile reuses the buffer
  }
}

// Inverse transform, persistent over tiles; the Fourier runs of tile
// t+gridDim.x stream into one buffer while tile t is transformed in place.
template <int A, int B, int NT>
__global__ void __launch_bounds__(NT, (A == 4 && B == 3) ? 4 : 1) k_fft_inv(FftArgs a, int bufe)
{
  using S = FftShape<A, B, NT>;
  constexpr int R1 = S::R1, R2 = S::R2, NC = S::NC, T = S::T, JT = S::JT, JTp = S::JTp;
  constexpr int NS = R1 / T;
  extern __shared__ __align__(16) double2 smem_all[];
  double2 *stw = smem_all, *stwI = smem_all + NC, *sm = smem_all + 2 * NC;
  load_twiddles<T, NC, NT>(a, stw, stwI);

  constexpr int JTh = JT / 2;  // mirrored row pairs per tile
  const int tid = threadIdx.x, r = tid / T, u = tid % T;
  const int ntile = (a.JH + JTh - 1) / JTh;
  // Tile indices fit in 32 bits (the launcher checks).  Up to 16-point first
  // passes the per-tile division is a 32-bit one (T85 / T170 inverse 1-4 %
  // faster); at 32 points, where the kernel sits at the 255-register cap, the
  // 64-bit form measured faster (T341 inverse 1.58 against 1.84 ms).
  using Idx = typename std::conditional<(A <= 4), unsigned, long long>::type;
  const Idx ntot = (Idx)a.ncol * (Idx)ntile;
  const long long mstride = (long long)a.ncolF * a.J;

  // rows [0, JTh) of a staged tile take E (then north), rows [JTh, JT) take O (then south)
  auto issue = [&](Idx t, double2 *buf) {
    const int col = (int)(t / (Idx)ntile), h0 = (int)(t - (Idx)col * (Idx)ntile) * JTh;
    const double2 *Fb = a.Fc + (long long)(a.colF0 + col) * a.J + h0;
    const int nh = min(JTh, a.JH - h0);
    // NT is a multiple of JT: this thread keeps staged row rr and steps the orders
    constexpr int MS = NT / JT;
    const int rr = tid % JT, i = rr % JTh;
    const bool in = i < nh;
    const double2 *src = Fb + (rr < JTh ? 0 : a.JH) + i + (long long)(tid / JT) * mstride;
    for (int m = tid / JT; m <= a.N; m += MS, src += MS * mstride)
      cp_async16(buf + m * JTp + rr, in ? src : Fb, in);
  };

  // Up to 16-point first passes the next tile's runs stream into the second
  // buffer while this one is transformed.  At 32 points a buffer is 67 KB and
  // the kernel needs 254 registers: one buffer per block, so that two blocks
  // share an SM and one block's loads overlap the other's transform.  At 128
  // complex points (I = 256) one buffer and a 128-register cap give 4 blocks
  // per SM instead of 3 (inverse 55.0 -> 53.9 us at T85, 480 field-levels).
  constexpr bool kDB = A <= 4 && !(A == 4 && B == 3);
  Idx t = blockIdx.x;
  if (t < ntot) issue(t, sm);
  cp_async_commit();
  for (int it = 0; t < ntot; t += gridDim.x, ++it) {
    double2 *cur = kDB ? sm + (it & 1) * bufe : sm;
    if constexpr (kDB) {
      if (t + gridDim.x < ntot) issue(t + gridDim.x, sm + ((it + 1) & 1) * bufe);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();

    const int col = (int)(t / (Idx)ntile), h0 = (int)(t - (Idx)col * (Idx)ntile) * JTh;
    const int jh = h0 + (r % JTh), j = r < JTh ? a.JH + jh : a.JH - 1 - jh;
    const bool valid = jh < a.JH;

    // this row's G^m: north = E + O (rows < JTh), south = E - O
    const int ri = r % JTh;
    const double sgn = r < JTh ? 1.0 : -1.0;
    auto gm = [&](int k) {
      const double2 e = cur[k * JTp + ri], o = cur[k * JTp + JTh + ri];
      return make_double2(e.x + sgn * o.x, e.y + sgn * o.y);
    };

    double2 v[R1];
    inv_pack<A, B, NT>(a.N, gm, stwI, v);
    __syncthreads();  // the staged runs are consumed; the buffer is reused below
    if constexpr (JTh * 16 % 128 == 0) {
      // Each E and O run of this tile is a whole number of 128-byte lines
      // (when JH is a multiple of the run) that no later kernel reads: drop
      // them from L2 without a write-back.
      if (a.JH % JTh == 0) {
        constexpr int LPR = JTh * 16 / 128;
        const double2 *Fb = a.Fc + (long long)(a.colF0 + col) * a.J + h0;
        for (int q = tid; q < (a.N + 1) * 2 * LPR; q += NT) {
          const int m = q / (2 * LPR), rest = q - m * 2 * LPR;
          l2::discard_line(reinterpret_cast<const char *>(Fb + m * mstride + (rest < LPR ? 0 : a.JH)) +
                           128 * (rest % LPR));
        }
      }
    }

    inv_transform<A, B, NT>(v, cur, stw, [&](const double2 (&z)[NS][R2]) {
      if (!valid) return;
      const long long IJ = (long long)a.I * a.J;
      double *dst = a.ocol ? a.ocol[col]
                  : (col < a.nsplit) ? a.o0 + (long long)col * IJ : a.o1 + (long long)(col - a.nsplit) * IJ;
      double2 *rowp = reinterpret_cast<double2 *>(dst + (long long)j * a.I);
      const double sc = __ldg(a.rowscale + j);
#pragma unroll
      for (int s = 0; s < NS; ++s)
#pragma unroll
        for (int k2 = 0; k2 < R2; ++k2) {
          const double2 w = z[s][brev<B>(k2)];
          rowp[u + T * s + R1 * k2] = make_double2(w.x * sc, w.y * sc);  // default policy: may stay in L2 for an analysis
        }
    });
    __syncthreads();  // the buffer is refilled by the prefetch of the next iteration
    if constexpr (!kDB) {
      if (t + gridDim.x < ntot) issue(t + gridDim.x, sm);
      cp_async_commit();
    }
  }
  cp_async_wait<0>();
}

// Zonal plans (im = 1, the wa_zonal_module transform): the longitude
// transform of a single point is the identity, so only the row scale remains,
// G^0_j = s_j q_j (forward) and q_j = s_j Re G^0_j (inverse).
__global__ void __launch_bounds__(256) k_zonal_fwd(FftArgs a)
{
  const long long total = (long long)a.ncol * a.JH;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int col = (int)(k / a.JH), jh = (int)(k - (long long)col * a.JH);
    const int jn = a.JH + jh, js = a.JH - 1 - jh;
    const double *src = a.gcol ? a.gcol[col] : (col < a.nsplit) ? a.g0 + (long long)col * a.J : a.g1 + (long long)(col - a.nsplit) * a.J;
    double gn = src[jn] * __ldg(a.rowscale + jn), gs = src[js] * __ldg(a.rowscale + js);
    if (a.mul) {
      const double *f = a.mul + (long long)(col % a.nmul) * a.J;
      gn *= f[jn];
      gs *= f[js];
      if (a.add0) {
        const double *z = col < a.nsplit ? a.add0 + (long long)col * a.J : a.add1 + (long long)(col - a.nsplit) * a.J;
        gn += z[jn] * __ldg(a.rowscale + jn);
        gs += z[js] * __ldg(a.rowscale + js);
      }
    }
    double2 *F = a.F + (long long)(a.colF0 + col) * a.J;
    F[jh] = make_double2(gn + gs, 0.0);
    F[a.JH + jh] = make_double2(gn - gs, 0.0);
  }
}

__global__ void __launch_bounds__(256) k_zonal_inv(FftArgs a)
{
  const long long total = (long long)a.ncol * a.JH;
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int col = (int)(k / a.JH), jh = (int)(k - (long long)col * a.JH);
    const int jn = a.JH + jh, js = a.JH - 1 - jh;
    double *dst = a.ocol ? a.ocol[col] : (col < a.nsplit) ? a.o0 + (long long)col * a.J : a.o1 + (long long)(col - a.nsplit) * a.J;
    const double2 *F = a.Fc + (long long)(a.colF0 + col) * a.J;
    const double e = F[jh].x, o = F[a.JH + jh].x;
    dst[jn] = (e + o) * __ldg(a.rowscale + jn);
    dst[js] = (e - o) * __ldg(a.rowscale + js);
  }
}

// Longitude counts that are not powers of two (factors 3 and 5, as in
// 96, 192, 320 or 640 points, which ISPACK's FFT covers): the transform by
// direct summation, G^m = s_j sum_i q_i e^{-2 pi i m i / I} for m <= N and its
// inverse, with e^{-2 pi i t / I} = twI[t] for t < I/2 and -twI[t - I/2]
// otherwise.  A block handles four mirrored row pairs of one field-level
// (eight rows staged in shared memory); the outputs take the same Gs/Ga and
// E/O layouts as the four-step kernels.
constexpr int kDftPairs = 4;
constexpr int kDftThreads = 256;

__device__ __forceinline__ double2 dft_twiddle(const double2 *__restrict__ twI, int t, int NC)
{
  const double2 w = __ldg(twI + (t < NC ? t : t - NC));
  return t < NC ? w : make_double2(-w.x, -w.y);
}

__global__ void __launch_bounds__(kDftThreads) k_dft_fwd(FftArgs a)
{
  extern __shared__ __align__(16) double dsm[];
  const int I = a.I, NC = I / 2, JH = a.JH, N = a.N;
  double2 *tw = reinterpret_cast<double2 *>(dsm);  // e^{-2 pi i t / I}, t < I
  double *rows = dsm + 2 * I;                      // 2 kDftPairs rows of I points
  for (int t = threadIdx.x; t < I; t += blockDim.x) tw[t] = dft_twiddle(a.twI, t, NC);
  const int ntile = (JH + kDftPairs - 1) / kDftPairs;
  const long long ntot = (long long)a.ncol * ntile;
  const long long IJ = (long long)I * a.J;
  const long long mstride = (long long)a.ncolF * a.J;
  for (long long tile = blockIdx.x; tile < ntot; tile += gridDim.x) {
    const int col = (int)(tile / ntile), h0 = (int)(tile - (long long)col * ntile) * kDftPairs;
    const double *gb = a.gcol ? a.gcol[col]
                     : (col < a.nsplit) ? a.g0 + (long long)col * IJ : a.g1 + (long long)(col - a.nsplit) * IJ;
    const double *fb = a.mul ? a.mul + (long long)(col % a.nmul) * IJ : nullptr;
    const double *zb = (a.mul && a.add0)
                           ? (col < a.nsplit ? a.add0 + (long long)col * IJ : a.add1 + (long long)(col - a.nsplit) * IJ)
                           : nullptr;
    __syncthreads();  // the previous tile's rows are consumed
    for (int idx = threadIdx.x; idx < 2 * kDftPairs * I; idx += blockDim.x) {
      const int r = idx / I, i = idx - r * I, jh = h0 + r % kDftPairs;
      const int j = r < kDftPairs ? JH + jh : JH - 1 - jh;
      double v = 0.0;
      if (jh < JH) {
        v = gb[(long long)j * I + i];
        if (fb) v *= fb[(long long)j * I + i];
        if (zb) v += zb[(long long)j * I + i];
      }
      rows[idx] = v;
    }
    __syncthreads();
    for (int o = threadIdx.x; o < kDftPairs * (N + 1); o += blockDim.x) {
      const int pr = o / (N + 1), m = o - pr * (N + 1), jh = h0 + pr;
      if (jh >= JH) continue;
      const double *rn = rows + pr * I, *rs = rows + (kDftPairs + pr) * I;
      double nr = 0.0, ni = 0.0, sr = 0.0, si = 0.0;
      int t = 0;
      for (int i = 0; i < I; ++i) {
        const double2 w = tw[t];
        nr = fma(rn[i], w.x, nr);
        ni = fma(rn[i], w.y, ni);
        sr = fma(rs[i], w.x, sr);
        si = fma(rs[i], w.y, si);
        t += m;
        if (t >= I) t -= I;
      }
      const double scn = __ldg(a.rowscale + JH + jh), scs = __ldg(a.rowscale + JH - 1 - jh);
      nr *= scn; ni *= scn; sr *= scs; si *= scs;
      if (m == 0) ni = si = 0.0;
      double2 *Fb = a.F + (long long)m * mstride + (long long)(a.colF0 + col) * a.J;
      Fb[jh] = make_double2(nr + sr, ni + si);
      Fb[JH + jh] = make_double2(nr - sr, ni - si);
    }
  }
}

__global__ void __launch_bounds__(kDftThreads) k_dft_inv(FftArgs a)
{
  extern __shared__ __align__(16) double dsm[];
  const int I = a.I, NC = I / 2, JH = a.JH, N = a.N;
  double2 *tw = reinterpret_cast<double2 *>(dsm);     // e^{+2 pi i t / I}, t < I
  double2 *g = tw + I;                                // 2 kDftPairs rows of N + 1 coefficients
  for (int t = threadIdx.x; t < I; t += blockDim.x) {
    const double2 w = dft_twiddle(a.twI, t, NC);
    tw[t] = make_double2(w.x, -w.y);
  }
  const int ntile = (JH + kDftPairs - 1) / kDftPairs;
  const long long ntot = (long long)a.ncol * ntile;
  const long long IJ = (long long)I * a.J;
  const long long mstride = (long long)a.ncolF * a.J;
  for (long long tile = blockIdx.x; tile < ntot; tile += gridDim.x) {
    const int col = (int)(tile / ntile), h0 = (int)(tile - (long long)col * ntile) * kDftPairs;
    __syncthreads();  // the previous tile's coefficients are consumed
    // row r < kDftPairs: north = E + O; row kDftPairs + r: south = E - O
    for (int idx = threadIdx.x; idx < kDftPairs * (N + 1); idx += blockDim.x) {
      const int pr = idx / (N + 1), m = idx - pr * (N + 1), jh = h0 + pr;
      double2 e = make_double2(0.0, 0.0), od = e;
      if (jh < JH) {
        const double2 *Fb = a.Fc + (long long)m * mstride + (long long)(a.colF0 + col) * a.J;
        e = Fb[jh];
        od = Fb[JH + jh];
      }
      double2 gn = make_double2(e.x + od.x, e.y + od.y), gs = make_double2(e.x - od.x, e.y - od.y);
      if (m == 0) gn.y = gs.y = 0.0;
      g[pr * (N + 1) + m] = gn;
      g[(kDftPairs + pr) * (N + 1) + m] = gs;
    }
    __syncthreads();
    double *ob = a.ocol ? a.ocol[col]
               : (col < a.nsplit) ? a.o0 + (long long)col * IJ : a.o1 + (long long)(col - a.nsplit) * IJ;
    for (int o = threadIdx.x; o < 2 * kDftPairs * I; o += blockDim.x) {
      const int r = o / I, i = o - r * I, jh = h0 + r % kDftPairs;
      if (jh >= JH) continue;
      const int j = r < kDftPairs ? JH + jh : JH - 1 - jh;
      const double2 *gr = g + r * (N + 1);
      // q_i = G^0 + 2 Re sum_{m >= 1} G^m e^{i m lambda_i}
      double acc = 0.0;
      int t = i;
      for (int m = 1; m <= N; ++m) {
        const double2 w = tw[t], c = gr[m];
        acc = fma(c.x, w.x, fma(-c.y, w.y, acc));
        t += i;
        if (t >= I) t -= I;
      }
      ob[(long long)j * I + i] = (gr[0].x + 2.0 * acc) * __ldg(a.rowscale + j);
    }
  }
}

namespace {
constexpr int kFftThreads = 128;

int run_dft(bool inverse, const sht_plan *p, const FftArgs &a, cudaStream_t s)
{
  const long long ntiles = (long long)a.ncol * ((p->JH + kDftPairs - 1) / kDftPairs);
  if (ntiles <= 0) return SHT_OK;
  const size_t smem = inverse ? sizeof(double2) * ((size_t)p->I + 2 * kDftPairs * (size_t)(p->N + 1))
                              : sizeof(double) * (2 * (size_t)p->I + 2 * kDftPairs * (size_t)p->I);
  if (smem > 227 * 1024) { set_error("fft: longitude count too large for the direct transform"); return SHT_ERR_UNSUPPORTED_SIZE; }
  void (*kern)(FftArgs) = inverse ? k_dft_inv : k_dft_fwd;
  int occ = 0;
  cudaError_t e = kernel_setup((const void *)kern, smem, kDftThreads, &occ);
  if (e != cudaSuccess) return cuda_fail(e, "dft smem attribute");
  const long long g = (long long)(occ < 1 ? 1 : occ) * grid_sms(p);
  kern<<<(int)(ntiles < g ? ntiles : g), kDftThreads, smem, s>>>(a);
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, inverse ? "k_dft_inv" : "k_dft_fwd");
}

// Persistent grids: as many blocks as fit on the device at once, never more
// than there are tiles.
template <int A, int B>
int run_fft(bool inverse, const sht_plan *p, const FftArgs &a, cudaStream_t s)
{
  using S = FftShape<A, B, kFftThreads>;
  // inverse up to 16-point first passes: two buffers (staged Fourier runs of
  // the next tile beside the current one); otherwise one buffer
  const int bufe = S::buf_elems(p->N);
  const size_t smem = sizeof(double2) * (2 * (size_t)S::NC + (inverse && A <= 4 && !(A == 4 && B == 3) ? 2 : 1) * (size_t)bufe);
  const long long ntiles = (long long)a.ncol * ((p->JH + S::JT / 2 - 1) / (S::JT / 2));
  if (ntiles <= 0) return SHT_OK;
  if (ntiles > 0x7fffffffLL) { set_error("fft: too many field-levels for one call"); return SHT_ERR_TOO_LARGE; }
  if (smem > 227 * 1024) { set_error("fft: shared-memory tile too large for this truncation"); return SHT_ERR_UNSUPPORTED_SIZE; }
  cudaError_t e = cudaSuccess;
  auto go = [&](auto kern, auto... extra) {
    int occ = 0;
    if ((e = kernel_setup((const void *)kern, smem, kFftThreads, &occ)) != cudaSuccess) return;
    const long long g = (long long)(occ < 1 ? 1 : occ) * grid_sms(p);
    kern<<<(int)(ntiles < g ? ntiles : g), kFftThreads, smem, s>>>(a, extra...);
  };
  if (inverse) go(k_fft_inv<A, B, kFftThreads>, bufe);
  else if (a.mul) go(k_fft_fwd<A, B, kFftThreads, 1>);
  else go(k_fft_fwd<A, B, kFftThreads, 0>);
  if (e != cudaSuccess) return cuda_fail(e, "fft smem attribute");
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, inverse ? "k_fft_inv" : "k_fft_fwd");
}

int dispatch(bool inverse, const sht_plan *p, const FftArgs &args, cudaStream_t s)
{
  if (p->zonal) {
    const long long total = (long long)args.ncol * p->JH;
    if (total <= 0) return SHT_OK;
    long long g = (total + 255) / 256;
    if (g > 148 * 8) g = 148 * 8;
    if (inverse) k_zonal_inv<<<(unsigned)g, 256, 0, s>>>(args);
    else k_zonal_fwd<<<(unsigned)g, 256, 0, s>>>(args);
    count_launch();
    cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SHT_OK : cuda_fail(e, inverse ? "k_zonal_inv" : "k_zonal_fwd");
  }
  if (p->direct_dft) return run_dft(inverse, p, args, s);
  switch (p->NC) {
  case 8: return run_fft<2, 1>(inverse, p, args, s);
  case 16: return run_fft<2, 2>(inverse, p, args, s);
  case 32: return run_fft<3, 2>(inverse, p, args, s);
  case 64: return run_fft<3, 3>(inverse, p, args, s);
  case 128: return run_fft<4, 3>(inverse, p, args, s);
  case 256: return run_fft<4, 4>(inverse, p, args, s);
  case 512: return run_fft<5, 4>(inverse, p, args, s);
  case 1024: return run_fft<5, 5>(inverse, p, args, s);
  default: set_error("fft: unsupported longitude count"); return SHT_ERR_UNSUPPORTED_SIZE;
  }
}
}  // namespace

int launch_fft_fwd(const sht_plan *p, const double *g0, const double *g1, int nsplit, int ncol,
                   double2 *F, int ncolF, int colF0, int rs, cudaStream_t s, const double *const *gcol,
                   const double *mul, int nmul, const double *add0, const double *add1)
{
  FftArgs a{};
  a.gcol = gcol;
  a.mul = mul;
  a.add0 = mul ? add0 : nullptr;
  a.add1 = mul ? (add1 ? add1 : add0) : nullptr;
  a.nmul = nmul > 0 ? nmul : 1;
  // the two inputs' tiles of one level run back to back, so the level's
  // factor grid comes from L2 the second time
  a.mul_pair = (mul && !gcol && g1 && ncol == 2 * nsplit) ? 1 : 0;
  a.g0 = g0; a.g1 = g1 ? g1 : g0; a.nsplit = nsplit; a.ncol = ncol;
  a.F = F; a.ncolF = ncolF; a.colF0 = colF0;
  a.rowscale = p->d_rowscale + (size_t)rs * p->J;
  a.tw = p->d_tw; a.twI = p->d_twI;
  a.I = p->I; a.J = p->J; a.JH = p->JH; a.N = p->N;
  return dispatch(false, p, a, s);
}

int launch_fft_inv(const sht_plan *p, const double2 *F, int ncolF, int colF0, int ncol,
                   double *g0, double *g1, int nsplit, int rs, cudaStream_t s, double *const *ocol)
{
  FftArgs a{};
  a.ocol = ocol;
  a.o0 = g0; a.o1 = g1 ? g1 : g0; a.nsplit = nsplit; a.ncol = ncol;
  a.Fc = F; a.ncolF = ncolF; a.colF0 = colF0;
  a.rowscale = p->d_rowscale + (size_t)rs * p->J;
  a.tw = p->d_tw; a.twI = p->d_twI;
  a.I = p->I; a.J = p->J; a.JH = p->JH; a.N = p->N;
  return dispatch(true, p, a, s);
}

}  // namespace sht
