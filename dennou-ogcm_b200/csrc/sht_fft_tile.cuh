// sht_fft_tile.cuh -- the tile machinery of the FP64 longitude transforms:
// register DFTs, four-step twiddles, the real (un)pack and the forward and
// inverse tile steps, shared by the batched kernels of sht_fft.cu and the
// single-kernel small-grid transforms of sht_small.cu.  Conventions and
// layouts are described at the top of sht_fft.cu.
#pragma once

#include "sht_internal.h"
#include "sht_l2.cuh"

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

// a e^{-2 pi i t / 32} for a t known at compile time (after unrolling)
__device__ __forceinline__ double2 rot32(double2 a, int t)
{
  if (t == 0) return a;
  if (t == 8) return make_double2(a.y, -a.x);
  const double c = cos32(t), s = sin32(t);
  return make_double2(a.x * c + a.y * s, a.y * c - a.x * s);
}

// The twiddles of thread column u.  Pass A: W^{u k1} (W = e^{-2 pi i / NC})
// from the table entries k1 = 1, 2, 3 and k1 = 4, 8, ...: W^{u k1} =
// W^{u (k1 mod 4)} W^{u 4 (k1 div 4)}, at most one product, 3 + R1/4 - 1
// shared-memory reads instead of R1 - 1.  Real (un)pack: e^{-2 pi i m / I} for
// m = u + T q is e^{-2 pi i u / I} e^{-2 pi i q / (2 R1)}, the second factor a
// constant of the unrolled loop (R1 <= 16), so one read per tile instead of R1.
// Each value is a product of two correctly rounded factors.
template <int R1, int T>
struct PassTwiddles {
  static constexpr int NB = R1 / 4 > 1 ? R1 / 4 : 1;
  double2 ta[4], tb[NB];
  __device__ __forceinline__ void load(const double2 *stw, int u)
  {
#pragma unroll
    for (int t = 1; t < 4 && t < R1; ++t) ta[t] = stw[t * T + u];
#pragma unroll
    for (int s = 1; s < NB; ++s) tb[s] = stw[4 * s * T + u];
  }
  __device__ __forceinline__ double2 operator()(int k1) const  // k1 >= 1, known at compile time
  {
    const int t = k1 & 3, s = k1 >> 2;
    if (s == 0) return ta[t];
    if (t == 0) return tb[s];
    return cmul(ta[t], tb[s]);
  }
};

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
        } else if (t == 8) {  // W = -+i
          v[b + k + h] = INV ? make_double2(-dy, dx) : make_double2(dy, -dx);
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
  int I, J, JH, N;
  const double *const *gcol;  // optional per-column grid sources (forward)
  double *const *ocol;        // optional per-column grid destinations (inverse)
  // forward product mode: column col is multiplied point by point by the
  // grid field mul + (col mod nmul) I J before the transform
  const double *mul;
  int nmul;
  int mul_pair;    // columns c and nsplit + c share a factor: visit them one after the other
  // multiply-add mode (with mul): column col becomes col * factor + z, z from
  // add0 + col I J (col < nsplit) or add1 + (col - nsplit) I J
  const double *add0, *add1;
};

// Shared-memory plan of one thread block: the twiddle tables (2 NC entries),
// then the tile buffers (two in the inverse, whose next tile's Fourier runs
// stream into one while the other is transformed; one in the forward, whose
// rows go from global memory straight to registers), each large enough for
// the in-place DFT rows and the m-major staging.
template <int A, int B, int NT>
struct FftShape {
  static constexpr int R1 = 1 << A, R2 = 1 << B, NC = R1 * R2, T = R2, JT = NT / T;
  static constexpr int RS = fft_row_stride<R1, R2, T>();
  static constexpr int JTp = fft_out_stride(JT, T);
  static int buf_elems(int N)  // double2 per buffer: the in-place DFT rows and the m-major staging
  {
    int b = JT * RS;
    b = b > (N + 1) * JTp ? b : (N + 1) * JTp;
    return (b + 7) & ~7;
  }
};

__device__ __forceinline__ void cp_async16(void *dst_smem, const void *src, bool fill)
{
  // src-size 0 writes 16 zero bytes and reads nothing
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"((uint32_t)__cvta_generic_to_shared(dst_smem)),
               "l"(src), "r"(fill ? 16 : 0));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int NPEND>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(NPEND)); }

// Both twiddle tables go to shared memory once per block (L1 keeps little
// room next to the staging buffers): stw[k1 T + u] = e^{-2 pi i u k1 / NC}
// for the four-step twiddle of thread column u, stwI[m] = e^{-2 pi i m / I}.
// The first barrier of the tile loop publishes them.
template <int T, int NC, int NT>
__device__ __forceinline__ void load_twiddles(const FftArgs &a, double2 *stw, double2 *stwI)
{
  for (int q = threadIdx.x; q < NC; q += NT) {
    stw[q] = __ldg(a.tw + (q % T) * (q / T));
    stwI[q] = __ldg(a.twI + q);
  }
}

// One forward tile after its rows are in registers (v: this thread's R1
// elements of row r, stride R2, already multiplied by any factor): the
// four-step DFT, the real unpack and the Gs/Ga output runs.  cur is the
// block's tile buffer, free for reuse on entry.
template <int A, int B, int NT, bool SMEM = false>
__device__ __forceinline__ void fwd_tile(const FftArgs &a, double2 (&v)[1 << A], double2 *cur, const double2 *stw,
                                         const double2 *stwI, int col, int h0, int j, bool valid,
                                         double2 *smF = nullptr)
{
  using S = FftShape<A, B, NT>;
  constexpr int R1 = S::R1, R2 = S::R2, T = S::T, JT = S::JT, RS = S::RS, JTp = S::JTp;
  constexpr int NS = R1 / T;
  constexpr int JTh = JT / 2;
  const int tid = threadIdx.x, r = tid / T, u = tid % T;
  const long long mstride = (long long)a.ncolF * a.J;
  dft_reg<A, false>(v);
  double2 *srow = cur + r * RS;
  PassTwiddles<R1, T> tw;
  tw.load(stw, u);
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    double2 y = v[brev<A>(k1)];
    if (k1 != 0) y = cmul(y, tw(k1));
    srow[u * (R1 + 1) + k1] = y;
  }
  __syncthreads();

  // pass B: R2-point DFTs; this thread then holds Z_m for
  // m = k1 + R1 k2, k1 = u + T s, i.e. m = u + T q with q = s + NS k2
  double2 z[NS][R2];
#pragma unroll
  for (int s = 0; s < NS; ++s) {
    const int k1 = u + T * s;
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) z[s][n2] = srow[n2 * (R1 + 1) + k1];
    dft_reg<B, false>(z[s]);
  }
  // Z_{NC-m}: for u != 0 it sits in lane T - u of the same row at
  // (s, k2) -> (NS-1-s, R2-1-k2); for u = 0 in this thread, at (0, -k2 mod R2)
  // when s = 0 and at (NS-s, R2-1-k2) otherwise
  const int lane = tid & 31, partner = (lane & ~(T - 1)) | ((T - u) & (T - 1));
  __syncthreads();  // every row's pass-B reads are done; the staging below overwrites them

  // real unpack: X_m = E - i W^m D, E/D = (Z_m +- conj Z_{NC-m})/2, W = e^{-2 pi i/I},
  // written transposed (m-major) for the output runs
  const double sc = valid ? __ldg(a.rowscale + j) : 0.0;
  const double2 cu = stwI[u];
#pragma unroll
  for (int q = 0; q < R1; ++q) {
    const int s = q % NS, k2 = q / NS, m = u + T * q;
    const double2 src = z[NS - 1 - s][brev<B>(R2 - 1 - k2)];
    double2 zc;
    zc.x = __shfl_sync(0xffffffffu, src.x, partner);
    zc.y = __shfl_sync(0xffffffffu, src.y, partner);
    if (u == 0) zc = (s == 0) ? z[0][brev<B>((R2 - k2) & (R2 - 1))] : z[s == 0 ? 0 : NS - s][brev<B>(R2 - 1 - k2)];
    if (m <= a.N) {
      const double2 zm = z[s][brev<B>(k2)];
      const double er = 0.5 * (zm.x + zc.x), ei = 0.5 * (zm.y - zc.y);
      const double dr = 0.5 * (zm.x - zc.x), di = 0.5 * (zm.y + zc.y);
      const double2 w = R1 <= 16 ? rot32(cu, q * (16 / R1)) : stwI[m];  // e^{-2 pi i m / I}
      const double tr = w.x * dr - w.y * di, ti = w.x * di + w.y * dr;
      cur[m * JTp + r] = make_double2((er + ti) * sc, (m == 0) ? 0.0 : (ei - tr) * sc);
    }
  }
  __syncthreads();

  // runs Gs = north + south at F[m][col][jh], Ga = north - south at F[m][col][JH + jh],
  // kept in L2 for the Legendre contraction that reads them next (SMEM: at
  // smF[m J + jh] and smF[m J + JH + jh], a whole level's array in shared memory)
  const int nh = min(JTh, a.JH - h0);
  if constexpr (SMEM) {
    for (int idx = tid; idx < (a.N + 1) * JTh; idx += NT) {
      const int m = idx / JTh, i = idx - m * JTh;
      if (i < nh) {
        const double2 gn = cur[m * JTp + i], gs = cur[m * JTp + JTh + i];
        smF[m * a.J + h0 + i] = make_double2(gn.x + gs.x, gn.y + gs.y);
        smF[m * a.J + a.JH + h0 + i] = make_double2(gn.x - gs.x, gn.y - gs.y);
      }
    }
    return;
  }
  double2 *Fb = a.F + (long long)(a.colF0 + col) * a.J + h0;
  const uint64_t keep = l2::keep_policy();
  for (int idx = tid; idx < (a.N + 1) * JTh; idx += NT) {
    const int m = idx / JTh, i = idx - m * JTh;
    if (i < nh) {
      const double2 gn = cur[m * JTp + i], gs = cur[m * JTp + JTh + i];
      l2::st_keep(Fb + m * mstride + i, make_double2(gn.x + gs.x, gn.y + gs.y), keep);
      l2::st_keep(Fb + m * mstride + a.JH + i, make_double2(gn.x - gs.x, gn.y - gs.y), keep);
    }
  }
}

// Inverse tile, first half: the real pack of this thread's R1 inputs,
// v[n1] = Z_k for k = R2 n1 + u, Z_k = (X_k + Y_k) + i w^k (X_k - Y_k),
// Y_k = conj X_{NC-k}, w = e^{+2 pi i/I}, from the orders X_k = G^k of the
// thread's row (gm(k), k <= N; the imaginary part of G^0 is dropped).  Up to
// R1 = 16 the thread reads X_k for its own k only and takes X_{NC-k} from
// lane T - u of the same row at n1' = R1-1-n1 (u != 0) or from itself at
// n1' = -n1 mod R1 (u = 0); at R1 = 32 the extra registers would spill, so
// both come from gm.
template <int A, int B, int NT, class GM>
__device__ __forceinline__ void inv_pack(int N, const GM &gm, const double2 *stwI, double2 (&v)[1 << A])
{
  using S = FftShape<A, B, NT>;
  constexpr int R1 = S::R1, R2 = S::R2, NC = S::NC, T = S::T;
  const int tid = threadIdx.x, u = tid % T;
  constexpr bool kShfl = R1 <= 16;
  double2 xk[kShfl ? R1 : 1];
  if constexpr (kShfl) {
#pragma unroll
    for (int n1 = 0; n1 < R1; ++n1) {
      const int k = R2 * n1 + u;
      xk[n1] = make_double2(0.0, 0.0);
      if (k <= N) {
        xk[n1] = gm(k);
        if (k == 0) xk[n1].y = 0.0;
      }
    }
  }
  const int lane = tid & 31, partner = (lane & ~(T - 1)) | ((T - u) & (T - 1));
  const double2 cu = stwI[u];
#pragma unroll
  for (int n1 = 0; n1 < R1; ++n1) {
    const int k = R2 * n1 + u;
    double2 X = make_double2(0.0, 0.0), Y = make_double2(0.0, 0.0);
    if constexpr (kShfl) {
      X = xk[n1];
      double2 q;
      q.x = __shfl_sync(0xffffffffu, xk[R1 - 1 - n1].x, partner);
      q.y = __shfl_sync(0xffffffffu, xk[R1 - 1 - n1].y, partner);
      if (u == 0) q = (n1 == 0) ? make_double2(0.0, 0.0) : xk[(R1 - n1) & (R1 - 1)];
      Y = make_double2(q.x, -q.y);
    } else {
      if (k <= N) {
        X = gm(k);
        if (k == 0) X.y = 0.0;
      }
      const int kk = NC - k;
      if (k > 0 && kk <= N) {
        const double2 q = gm(kk);
        Y = make_double2(q.x, -q.y);
      }
    }
    const double2 wI = kShfl ? rot32(cu, n1 * (16 / R1)) : stwI[k];  // e^{-2 pi i k / I}
    const double wr = wI.x, wi = -wI.y;
    const double dr = X.x - Y.x, di = X.y - Y.y;
    const double tr = wr * dr - wi * di, ti = wr * di + wi * dr;
    v[n1] = make_double2((X.x + Y.x) - ti, (X.y + Y.y) + tr);
  }
}

// Inverse tile, second half: the four-step inverse DFT of v through the
// scratch rows cur (free on entry; one barrier inside), then store(z) with
// z[s][brev(k2)] the row's complex points u + T s + R1 k2.
template <int A, int B, int NT, class Store>
__device__ __forceinline__ void inv_transform(double2 (&v)[1 << A], double2 *cur, const double2 *stw,
                                              const Store &store)
{
  using S = FftShape<A, B, NT>;
  constexpr int R1 = S::R1, R2 = S::R2, T = S::T, RS = S::RS;
  constexpr int NS = R1 / T;
  const int tid = threadIdx.x, r = tid / T, u = tid % T;
  dft_reg<A, true>(v);
  double2 *srow = cur + r * RS;
  PassTwiddles<R1, T> tw;
  tw.load(stw, u);
#pragma unroll
  for (int k1 = 0; k1 < R1; ++k1) {
    double2 y = v[brev<A>(k1)];
    if (k1 != 0) y = cmulc(y, tw(k1));
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
  store(z);
}

}  // namespace sht
