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
// with the usual half-length real-FFT identity.  Each thread block owns JT
// consecutive latitude rows of one field-level and T = R2 threads per row;
// its Fourier output is staged in shared memory and written as JT-long
// contiguous runs of F[m][col][j] (coalesced), which is the layout the
// Legendre contraction reads.  Shared-memory strides are padded so that each
// 8-lane phase of a 16-byte access touches eight distinct bank groups.
#include "sht_internal.h"

namespace sht {

// cos(pi q / 16), q = 0..8 (standard constants to 32 significant digits)
__host__ __device__ constexpr double cos_pi16(int q)
{
  return q == 0 ? 1.0
       : q == 1 ? 0.98078528040323044912618223613424
       : q == 2 ? 0.92387953251128675612818318939679
       : q == 3 ? 0.83146961230254523707878837761791
       : q == 4 ? 0.70710678118654752440084436210485
       : q == 5 ? 0.55557023301960222474283081394853
       : q == 6 ? 0.38268343236508977172845998403040
       : q == 7 ? 0.19509032201612826784828486847702
       : 0.0;
}
// cos(2 pi t / 32) and sin(2 pi t / 32), t in [0, 32)
__host__ __device__ constexpr double cos32(int t)
{
  return t <= 8 ? cos_pi16(t) : t <= 16 ? -cos_pi16(16 - t) : t <= 24 ? -cos_pi16(t - 16) : cos_pi16(32 - t);
}
__host__ __device__ constexpr double sin32(int t) { return cos32((t + 24) & 31); }

template <int LOG>
__host__ __device__ constexpr int brev(int i)
{
  int r = 0;
  for (int b = 0; b < LOG; ++b) r |= ((i >> b) & 1) << (LOG - 1 - b);
  return r;
}

__device__ __forceinline__ double2 cmul(double2 a, double2 b)
{
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cmulc(double2 a, double2 b)  // a * conj(b)
{
  return make_double2(a.x * b.x + a.y * b.y, a.y * b.x - a.x * b.y);
}

// In-register radix-2 decimation-in-frequency DFT of size 2^LOG (<= 32),
// sign -1 (forward) or +1 (INV).  Output is left in bit-reversed order:
// X[k] = v[brev<LOG>(k)].
template <int LOG, bool INV>
__device__ __forceinline__ void dft_reg(double2 (&v)[1 << LOG])
{
  constexpr int R = 1 << LOG;
#pragma unroll
  for (int st = 0; st < LOG; ++st) {
    const int h = R >> (st + 1);
#pragma unroll
    for (int b = 0; b < R; b += 2 * h) {
#pragma unroll
      for (int k = 0; k < h; ++k) {
        const double2 a = v[b + k], c = v[b + k + h];
        v[b + k] = make_double2(a.x + c.x, a.y + c.y);
        const double dx = a.x - c.x, dy = a.y - c.y;
        const int t = k * (32 / (2 * h));  // W_{2h}^k = exp(-+ 2 pi i t / 32)
        if (t == 0) {
          v[b + k + h] = make_double2(dx, dy);
        } else {
          const double wr = cos32(t);
          const double wi = INV ? sin32(t) : -sin32(t);
          v[b + k + h] = make_double2(dx * wr - dy * wi, dx * wi + dy * wr);
        }
      }
    }
  }
}

template <int R1, int R2, int T>
__host__ __device__ constexpr int fft_row_stride()
{
  int s = R2 * (R1 + 1);
  if (T < 8)
    while (s % 8 != T) ++s;
  return s;
}
__host__ __device__ constexpr int fft_out_stride(int JT, int T)
{
  int s = JT;
  if (T >= 8) {
    if (s % 2 == 0) s += 1;
  } else {
    while (s % 8 != 8 / T) ++s;
  }
  return s;
}

struct FftArgs {
  const double *g0, *g1;  // forward sources
  double *o0, *o1;        // inverse destinations
  int nsplit, ncol;
  double2 *F;             // forward output
  const double2 *Fc;      // inverse input
  int ncolF, colF0;
  const double *rowscale;
  const double2 *tw, *twI;
  int I, J, N;
};

template <int A, int B, int NT>
__global__ void __launch_bounds__(NT) k_fft_fwd(FftArgs a)
{
  constexpr int R1 = 1 << A, R2 = 1 << B, NC = R1 * R2, T = R2, JT = NT / T;
  constexpr int RS = fft_row_stride<R1, R2, T>();
  constexpr int JTp = fft_out_stride(JT, T);
  constexpr int NS = R1 / T;
  extern __shared__ double2 sm[];

  const int tid = threadIdx.x, r = tid / T, u = tid % T;
  const int ntile = (a.J + JT - 1) / JT;
  const int col = blockIdx.x / ntile, jt = blockIdx.x - col * ntile;
  const int j0 = jt * JT, j = j0 + r;
  const bool valid = j < a.J;
  const long long IJ = (long long)a.I * a.J;
  const double *src = (col < a.nsplit) ? a.g0 + (long long)col * IJ : a.g1 + (long long)(col - a.nsplit) * IJ;

  // pass A: R1-point DFTs over elements strided by R2
  double2 v[R1];
  if (valid) {
    const double2 *rowp = reinterpret_cast<const double2 *>(src + (long long)j * a.I);
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) v[n1] = __ldcs(rowp + R2 * n1 + u);
  } else {
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) v[n1] = make_double2(0.0, 0.0);
  }
  dft_reg<A, false>(v);
  double2 *srow = sm + r * RS;
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    double2 y = v[brev<A>(k1)];
    if (k1 != 0) y = cmul(y, __ldg(a.tw + u * k1));
    srow[u * (R1 + 1) + k1] = y;
  }
  __syncthreads();

  // pass B: R2-point DFTs
  double2 z[NS][R2];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k1 = u + T * s;
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) z[s][n2] = srow[n2 * (R1 + 1) + k1];
    dft_reg<B, false>(z[s]);
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < NS; ++s)
#pragma unroll
    for (int k2 = 0; k2 < R2; ++k2) srow[(u + T * s) + R1 * k2] = z[s][brev<B>(k2)];
  __syncthreads();

  // real unpack: X_m = E - i W^m D, E/D = (Z_m +- conj Z_{NC-m})/2, W = e^{-2 pi i/I}
  const double sc = valid ? __ldg(a.rowscale + j) : 0.0;
  double2 xo[R1];
#pragma unroll
  for (int q = 0; q < R1; ++q) {
    const int m = u + T * q;
    xo[q] = make_double2(0.0, 0.0);
    if (m <= a.N) {
      const int mm = (NC - m) & (NC - 1);
      const double2 zm = srow[m], zc = srow[mm];
      const double er = 0.5 * (zm.x + zc.x), ei = 0.5 * (zm.y - zc.y);
      const double dr = 0.5 * (zm.x - zc.x), di = 0.5 * (zm.y + zc.y);
      const double2 w = __ldg(a.twI + m);
      const double tr = w.x * dr - w.y * di, ti = w.x * di + w.y * dr;
      xo[q] = make_double2((er + ti) * sc, (m == 0) ? 0.0 : (ei - tr) * sc);
    }
  }
  __syncthreads();
#pragma unroll
  for (int q = 0; q < R1; ++q) {
    const int m = u + T * q;
    if (m <= a.N) sm[m * JTp + r] = xo[q];
  }
  __syncthreads();

  const int nrows = min(JT, a.J - j0);
  const int total = (a.N + 1) * JT;
  double2 *Fb = a.F + (long long)(a.colF0 + col) * a.J + j0;
  const long long mstride = (long long)a.ncolF * a.J;
  for (int idx = tid; idx < total; idx += NT) {
    const int m = idx / JT, rr = idx - m * JT;
    if (rr < nrows) Fb[m * mstride + rr] = sm[m * JTp + rr];
  }
  (void)NC;
}

template <int A, int B, int NT>
__global__ void __launch_bounds__(NT) k_fft_inv(FftArgs a)
{
  constexpr int R1 = 1 << A, R2 = 1 << B, NC = R1 * R2, T = R2, JT = NT / T;
  constexpr int RS = fft_row_stride<R1, R2, T>();
  constexpr int JTp = fft_out_stride(JT, T);
  constexpr int NS = R1 / T;
  extern __shared__ double2 sm[];

  const int tid = threadIdx.x, r = tid / T, u = tid % T;
  const int ntile = (a.J + JT - 1) / JT;
  const int col = blockIdx.x / ntile, jt = blockIdx.x - col * ntile;
  const int j0 = jt * JT, j = j0 + r;
  const bool valid = j < a.J;
  const int nrows = min(JT, a.J - j0);

  // stage G^m for the tile's rows
  const double2 *Fb = a.Fc + (long long)(a.colF0 + col) * a.J + j0;
  const long long mstride = (long long)a.ncolF * a.J;
  for (int idx = tid; idx < (a.N + 1) * JT; idx += NT) {
    const int m = idx / JT, rr = idx - m * JT;
    sm[m * JTp + rr] = (rr < nrows) ? Fb[m * mstride + rr] : make_double2(0.0, 0.0);
  }
  __syncthreads();

  // real pack: Z_k = (X_k + Y_k) + i w^k (X_k - Y_k), Y_k = conj X_{NC-k}, w = e^{+2 pi i/I}
  double2 v[R1];
#pragma unroll
  for (int n1 = 0; n1 < R1; ++n1) {
    const int k = R2 * n1 + u;
    double2 X = make_double2(0.0, 0.0), Y = make_double2(0.0, 0.0);
    if (k <= a.N) {
      X = sm[k * JTp + r];
      if (k == 0) X.y = 0.0;
    }
    const int kk = NC - k;
    if (k > 0 && kk <= a.N) {
      const double2 t = sm[kk * JTp + r];
      Y = make_double2(t.x, -t.y);
    }
    const double2 wI = __ldg(a.twI + k);
    const double wr = wI.x, wi = -wI.y;
    const double dr = X.x - Y.x, di = X.y - Y.y;
    const double tr = wr * dr - wi * di, ti = wr * di + wi * dr;
    v[n1] = make_double2((X.x + Y.x) - ti, (X.y + Y.y) + tr);
  }
  __syncthreads();

  dft_reg<A, true>(v);
  double2 *srow = sm + r * RS;
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    double2 y = v[brev<A>(k1)];
    if (k1 != 0) y = cmulc(y, __ldg(a.tw + u * k1));
    srow[u * (R1 + 1) + k1] = y;
  }
  __syncthreads();

  double2 z[NS][R2];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k1 = u + T * s;
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) z[s][n2] = srow[n2 * (R1 + 1) + k1];
    dft_reg<B, true>(z[s]);
  }
  if (valid) {
    const long long IJ = (long long)a.I * a.J;
    double *dst = (col < a.nsplit) ? a.o0 + (long long)col * IJ : a.o1 + (long long)(col - a.nsplit) * IJ;
    double2 *rowp = reinterpret_cast<double2 *>(dst + (long long)j * a.I);
    const double sc = __ldg(a.rowscale + j);
#pragma unroll
    for (int s = 0; s < NS; ++s)
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) {
        const double2 w = z[s][brev<B>(k2)];
        __stcs(rowp + (u + T * s + R1 * k2), make_double2(w.x * sc, w.y * sc));
      }
  }
  (void)NC;
}

namespace {
constexpr int kFftThreads = 128;

template <int A, int B>
size_t fft_smem_bytes(int N)
{
  constexpr int R1 = 1 << A, R2 = 1 << B, T = R2, JT = kFftThreads / T;
  constexpr int RS = fft_row_stride<R1, R2, T>();
  const size_t s1 = (size_t)JT * RS;
  const size_t s2 = (size_t)(N + 1) * fft_out_stride(JT, T);
  return sizeof(double2) * (s1 > s2 ? s1 : s2);
}

template <int A, int B>
int run_fft(bool inverse, const sht_plan *p, const FftArgs &args, cudaStream_t s)
{
  constexpr int T = 1 << B, JT = kFftThreads / T;
  const size_t smem = fft_smem_bytes<A, B>(p->N);
  const long long nblk = (long long)args.ncol * ((p->J + JT - 1) / JT);
  if (nblk <= 0) return SHT_OK;
  if (nblk > 0x7fffffffLL) { set_error("fft: too many columns"); return SHT_ERR_TOO_LARGE; }
  cudaError_t e;
  if (inverse) {
    auto kern = k_fft_inv<A, B, kFftThreads>;
    if (smem > 48 * 1024 && (e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
      return cuda_fail(e, "fft_inv smem attribute");
    kern<<<(unsigned)nblk, kFftThreads, smem, s>>>(args);
  } else {
    auto kern = k_fft_fwd<A, B, kFftThreads>;
    if (smem > 48 * 1024 && (e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)) != cudaSuccess)
      return cuda_fail(e, "fft_fwd smem attribute");
    kern<<<(unsigned)nblk, kFftThreads, smem, s>>>(args);
  }
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, inverse ? "k_fft_inv" : "k_fft_fwd");
}

int dispatch(bool inverse, const sht_plan *p, const FftArgs &args, cudaStream_t s)
{
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
                   double2 *F, int ncolF, int colF0, int rs, cudaStream_t s)
{
  FftArgs a{};
  a.g0 = g0; a.g1 = g1 ? g1 : g0; a.nsplit = nsplit; a.ncol = ncol;
  a.F = F; a.ncolF = ncolF; a.colF0 = colF0;
  a.rowscale = p->d_rowscale + (size_t)rs * p->J;
  a.tw = p->d_tw; a.twI = p->d_twI;
  a.I = p->I; a.J = p->J; a.N = p->N;
  return dispatch(false, p, a, s);
}

int launch_fft_inv(const sht_plan *p, const double2 *F, int ncolF, int colF0, int ncol,
                   double *g0, double *g1, int nsplit, int rs, cudaStream_t s)
{
  FftArgs a{};
  a.o0 = g0; a.o1 = g1 ? g1 : g0; a.nsplit = nsplit; a.ncol = ncol;
  a.Fc = F; a.ncolF = ncolF; a.colF0 = colF0;
  a.rowscale = p->d_rowscale + (size_t)rs * p->J;
  a.tw = p->d_tw; a.twI = p->d_twI;
  a.I = p->I; a.J = p->J; a.N = p->N;
  return dispatch(true, p, a, s);
}

}  // namespace sht
