// sht_spectral.cu -- spectral-side kernels: conversion between the SPML
// real layout wa[b][l] and the internal complex layout S[row][col], fused
// with the derivative recurrences of the operators, plus the diagonal
// spectral operators and the Gauss-weighted grid integrals.
//
//   analysis side ("pack", internal c -> wa):
//     plain      w_xy                              c_n
//     divlambda  w_DivLambda_xy                    i m c_n
//     divmu      w_DivMu_xy                        D(c)_n = -((n+1) eps_n c_{n-1} - n eps_{n+1} c_{n+1})
//     alpha      w_AlphaOptr_xy(A,B)               (i m cA_n + D(cB)_n) / a
//     vordiv     calc_UVCosLat2VorDiv(Ucos,Vcos)   vor = (i m cV - D(cU))/a, div = (i m cU + D(cV))/a
//   synthesis side ("unpack", wa -> internal a, n = m..N+1):
//     plain      xy_w                              a_n
//     gradlambda xy_GradLambda_w / GradLon         i m a_n
//     hgrad      GradLon and GradLat together      i m a_n and R(a)_n (two column sets)
//     gradmu     xy_GradMu_w / GradLat             R(a)_n = (n+2) eps_{n+1} a_{n+1} - (n-1) eps_n a_{n-1}
//     alpha      xy_AlphaOptr_w(A,B)               i m aA_n + R(aB)_n
//     vordiv2uv  calc_VorDiv2UV(vor,div)           psi,chi = -a^2 x/(n(n+1));
//                                                  U = i m chi - R(psi), V = i m psi + R(chi)
// The eps recurrence is space_discretization.tex:250-257; the U, V form is
// :369-379; D is the by-parts form of :262-267; the 1/a factors are
// SpmlUtil_mod.f90:410,426 and the a^2 LaplaInv at SpmlUtil_mod.f90:335-336.
//
// Both conversions tile by (total degree n, a chunk of 32 orders m, 32
// field-levels) so that global reads and writes are 256-512 byte runs.
#include "sht_internal.h"

namespace sht {

namespace {
constexpr int kMC = 32;  // orders per tile
constexpr int kBC = 32;  // field-levels per tile
constexpr double kSqrt2 = 1.41421356237309504880;
constexpr double kRSqrt2 = 0.70710678118654752440;

struct SpecArgs {
  const double2 *S;   // pack input
  double2 *So;        // unpack output
  int ncolS;
  const double *w0, *w1;  // unpack inputs
  double *o0, *o1;        // pack outputs
  int nb, N, L;
  double radius;
  const double *eps;      // [m][n], n = 0..N+2
  const int2 *tiles;      // (n, m0) per tile
  double *const *ocol;        // optional per-field-level pack destinations
  const double *const *icol;  // optional per-field-level unpack sources
  int M;                      // orders present: N + 1, or 1 for a zonal plan
  int zonal;                  // SPML index l = n (wa_zonal_module) instead of n(n+1) +- m
};

// 0-based SPML index of (n, m), cos (sn = 0) or sin (sn = 1) part
__device__ __forceinline__ long long spml_l(const SpecArgs &a, int n, int m, int sn)
{
  return a.zonal ? (long long)n : (long long)n * (n + 1) + (sn ? -m : m);
}

__device__ __forceinline__ double eps_at(const SpecArgs &a, int m, int n)
{
  return (n < 0 || n > a.N + 2) ? 0.0 : __ldg(a.eps + (long long)m * (a.N + 3) + n);
}

// Internal row of (m, n): rowoff(m) + n - m, with rowoff(m) = sum over m' < m
// of the N + 2 - m' rows of band m' (the plan's row table in closed form, so
// that no dependent load precedes the coefficient loads)
__device__ __forceinline__ int spec_row(int N, int m, int n) { return m * (N + 2) - m * (m - 1) / 2 + (n - m); }
__device__ __forceinline__ double2 cadd(double2 x, double2 y) { return make_double2(x.x + y.x, x.y + y.y); }
__device__ __forceinline__ double2 csub(double2 x, double2 y) { return make_double2(x.x - y.x, x.y - y.y); }
__device__ __forceinline__ double2 cscale(double2 x, double s) { return make_double2(x.x * s, x.y * s); }
__device__ __forceinline__ double2 times_im(double2 x, int m) { return make_double2(-m * x.y, m * x.x); }

// Which internal rows a pack operator reads: degree offset dn in -1..1 of
// column set `set` (0: the first input's columns, 1: the second's).
template <int OP>
__host__ __device__ constexpr bool pack_needs(int dn, int set)
{
  return OP == PACK_PLAIN || OP == PACK_DIVLAMBDA ? (dn == 0 && set == 0)
       : OP == PACK_DIVMU                         ? (dn != 0 && set == 0)
       : OP == PACK_ALPHA                         ? (set == 0 ? dn == 0 : dn != 0)
                                                  : true;  // VORDIV
}

template <int OP>
__global__ void __launch_bounds__(256) k_pack(SpecArgs a)
{
  __shared__ double out[2][2][kMC][kBC + 1];  // [array][cos/sin][m][b]
  const int2 t = a.tiles[blockIdx.x];
  const int n = t.x, m0 = t.y;
  const int b0 = blockIdx.y * kBC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int b = b0 + lane;
  constexpr int NOUT = (OP == PACK_VORDIV) ? 2 : 1;
  constexpr int NI = kMC / 8;  // orders per warp
  // every load of the thread is issued before any is used: out-of-range
  // entries read element 0 and are replaced by zero
  double2 c[NI][3][2];
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    const int m = m0 + warp + 8 * i;
    const bool ok = m <= n && m < a.M && b < a.nb;
    const long long base = ok ? (long long)spec_row(a.N, m, n) * a.ncolS + b : 0;
#pragma unroll
    for (int dn = -1; dn <= 1; ++dn)
#pragma unroll
      for (int set = 0; set < 2; ++set) {
        c[i][dn + 1][set] = make_double2(0.0, 0.0);
        if (!pack_needs<OP>(dn, set)) continue;
        const bool okk = ok && n + dn >= m && n + dn <= a.N + 1;
        const double2 x = a.S[okk ? base + (long long)dn * a.ncolS + set * a.nb : 0];
        if (okk) c[i][dn + 1][set] = x;
      }
  }
#pragma unroll
  for (int i = 0; i < NI; ++i) {
    const int mi = warp + 8 * i, m = m0 + mi;
    double2 v0 = make_double2(0.0, 0.0), v1 = make_double2(0.0, 0.0);
    if (m <= n && m < a.M && b < a.nb) {
      auto D = [&](int set) -> double2 {  // -( (n+1) eps_n c_{n-1} - n eps_{n+1} c_{n+1} )
        const double e0 = (n + 1) * eps_at(a, m, n), e1 = n * eps_at(a, m, n + 1);
        const double2 cm = c[i][0][set], cp = c[i][2][set];
        return make_double2(e1 * cp.x - e0 * cm.x, e1 * cp.y - e0 * cm.y);
      };
      if (OP == PACK_PLAIN) {
        v0 = c[i][1][0];
      } else if (OP == PACK_DIVLAMBDA) {
        v0 = times_im(c[i][1][0], m);
      } else if (OP == PACK_DIVMU) {
        v0 = D(0);
      } else if (OP == PACK_ALPHA) {
        v0 = cscale(cadd(times_im(c[i][1][0], m), D(1)), 1.0 / a.radius);
      } else {  // PACK_VORDIV: set 0 = U cos, set 1 = V cos
        v0 = cscale(csub(times_im(c[i][1][1], m), D(0)), 1.0 / a.radius);
        v1 = cscale(cadd(times_im(c[i][1][0], m), D(1)), 1.0 / a.radius);
      }
    }
    const double s = (m == 0) ? 1.0 : kSqrt2;
    out[0][0][mi][lane] = v0.x * s;
    out[0][1][mi][lane] = v0.y * s;
    if (NOUT == 2) {
      out[1][0][mi][lane] = v1.x * s;
      out[1][1][mi][lane] = v1.y * s;
    }
  }
  __syncthreads();
  // write runs w[b][n(n+1) + m] and w[b][n(n+1) - m]
  const int mi = lane, m = m0 + mi;
  if (m > n || m >= a.M) return;
  const long long lc = spml_l(a, n, m, 0), ls = spml_l(a, n, m, 1);
#pragma unroll
  for (int q = 0; q < kBC / 8; ++q) {
    const int bi = warp + 8 * q, bb = b0 + bi;
    if (bb >= a.nb) break;
#pragma unroll
    for (int o = 0; o < NOUT; ++o) {
      double *w = (o == 0 && a.ocol) ? a.ocol[bb] : ((o == 0) ? a.o0 : a.o1) + (long long)bb * a.L;
      w[lc] = out[o][0][mi][bi];
      if (m > 0) w[ls] = out[o][1][mi][bi];
    }
  }
}

// Which staged runs an unpack operator reads.  A run is (input, degree offset
// dn = -1/0/+1, cos/sin part); runs are numbered in*6 + (dn+1)*2 + part.
template <int OP>
__host__ __device__ constexpr bool unpack_needs(int in, int dn)
{
  return OP == UNPACK_PLAIN || OP == UNPACK_GRADLAMBDA ? (in == 0 && dn == 0)
       : OP == UNPACK_GRADMU                          ? (in == 0 && dn != 0)
       : OP == UNPACK_HGRAD                           ? (in == 0)
       : OP == UNPACK_ALPHA                           ? (in == 0 ? dn == 0 : dn != 0)
                                                      : true;  // VORDIV2UV
}
template <int OP>
__host__ __device__ constexpr int unpack_slot(int run)  // compact shared-memory slot of a needed run
{
  int s = 0;
  for (int r = 0; r < run; ++r) s += unpack_needs<OP>(r / 6, (r % 6) / 2 - 1) ? 1 : 0;
  return s;
}
template <int OP>
__host__ __device__ constexpr int unpack_nslots() { return unpack_slot<OP>(12); }

template <int OP>
__global__ void __launch_bounds__(256) k_unpack(SpecArgs a)
{
  constexpr int NIN = (OP == UNPACK_ALPHA || OP == UNPACK_VORDIV2UV) ? 2 : 1;
  extern __shared__ double ws_dyn[];  // [slot][m][b]
  auto ws = reinterpret_cast<double(*)[kMC][kBC + 1]>(ws_dyn);
  const int2 t = a.tiles[blockIdx.x];
  const int n = t.x, m0 = t.y;
  const int b0 = blockIdx.y * kBC;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  // Stage the SPML entries the operator reads (degrees n-1..n+1 as needed,
  // orders m0..m0+31, both parts).  Warp w takes field-levels b0 + 8i' + w of
  // every run, so the run of each unrolled load is a compile-time constant;
  // all loads of a warp are issued before any of them is stored.
  constexpr int NQ = kBC / 8;
  constexpr int PER = NIN * 6 * NQ;
  double val[PER];
  const int m = m0 + lane;
  // the row of each of this warp's field-levels, and the SPML offset of each
  // run (-1 where the entry does not exist), formed once for all loads
  const double *wr[NIN][NQ];
#pragma unroll
  for (int in = 0; in < NIN; ++in)
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      const int bb = b0 + 8 * q + warp;
      wr[in][q] = bb >= a.nb ? nullptr
                : (in == 0 && a.icol) ? a.icol[bb] : ((in == 0) ? a.w0 : a.w1) + (long long)bb * a.L;
    }
  int off[6];
#pragma unroll
  for (int r = 0; r < 6; ++r) {
    const int nn = n + r / 2 - 1, sn = r & 1;
    const bool ok = nn >= 0 && nn <= a.N && m <= nn && m < a.M && !(sn && m == 0);
    off[r] = ok ? (int)spml_l(a, nn, m, sn) : -1;
  }
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int run = i / NQ;
    val[i] = 0.0;
    if (!unpack_needs<OP>(run / 6, (run % 6) / 2 - 1)) continue;
    const double *w = wr[run / 6][i % NQ];
    const int o = off[run % 6];
    if (w && o >= 0) val[i] = __ldg(w + o);
  }
#pragma unroll
  for (int i = 0; i < PER; ++i) {
    const int run = i / (kBC / 8);
    if (unpack_needs<OP>(run / 6, (run % 6) / 2 - 1))
      ws[unpack_slot<OP>(run)][lane][8 * (i % (kBC / 8)) + warp] = val[i];
  }
  __syncthreads();
  const int b = b0 + lane;
  if (b >= a.nb) return;
  int rows[kMC / 8];  // internal rows of this warp's orders
#pragma unroll
  for (int i = 0; i < kMC / 8; ++i) {
    const int m = m0 + warp + 8 * i;
    rows[i] = (m <= n && m <= a.N && m < a.M) ? spec_row(a.N, m, n) : -1;
  }
#pragma unroll
  for (int i = 0; i < kMC / 8; ++i) {
    const int mi = warp + 8 * i, m = m0 + mi;
    if (rows[i] < 0) continue;
    const double s = (m == 0) ? 1.0 : kRSqrt2;
    auto coef = [&](int in, int dn) -> double2 {
      const int run = in * 6 + (dn + 1) * 2;
      return make_double2(ws[unpack_slot<OP>(run)][mi][lane] * s, ws[unpack_slot<OP>(run + 1)][mi][lane] * s);
    };
    auto R = [&](int in, double mult0) -> double2 {  // (n+2) eps_{n+1} x_{n+1} - (n-1) eps_n x_{n-1}, x scaled per degree
      const double ep = (n + 2) * eps_at(a, m, n + 1), em = (n - 1) * eps_at(a, m, n);
      double2 xp = coef(in, 1), xm = coef(in, -1);
      if (mult0 != 0.0) {  // inverse Laplacian scaling -a^2/(k(k+1)) per degree
        const double kp = n + 1.0, km = n - 1.0;
        const double sp = -mult0 / (kp * (kp + 1.0));
        const double sm_ = (km >= 1.0) ? -mult0 / (km * (km + 1.0)) : 0.0;
        xp = cscale(xp, sp);
        xm = cscale(xm, sm_);
      }
      return make_double2(ep * xp.x - em * xm.x, ep * xp.y - em * xm.y);
    };
    double2 v0, v1 = make_double2(0.0, 0.0);
    if (OP == UNPACK_PLAIN) {
      v0 = coef(0, 0);
    } else if (OP == UNPACK_GRADLAMBDA) {
      v0 = times_im(coef(0, 0), m);
    } else if (OP == UNPACK_GRADMU) {
      v0 = R(0, 0.0);
    } else if (OP == UNPACK_HGRAD) {
      v0 = times_im(coef(0, 0), m);
      v1 = R(0, 0.0);
    } else if (OP == UNPACK_ALPHA) {
      v0 = cadd(times_im(coef(0, 0), m), R(1, 0.0));
    } else {  // UNPACK_VORDIV2UV: input 0 = vor, 1 = div
      const double a2 = a.radius * a.radius;
      const double sn = (n >= 1) ? -a2 / ((double)n * (n + 1.0)) : 0.0;
      const double2 psi = cscale(coef(0, 0), sn), chi = cscale(coef(1, 0), sn);
      v0 = csub(times_im(chi, m), R(0, a2));
      v1 = cadd(times_im(psi, m), R(1, a2));
    }
    const long long row = rows[i];
    a.So[row * a.ncolS + b] = v0;
    if (OP == UNPACK_VORDIV2UV || OP == UNPACK_HGRAD) a.So[row * a.ncolS + a.nb + b] = v1;
  }
}

// --------------------------------------------------------- diagonal ops
__global__ void k_lapla(const double *__restrict__ w, const double *__restrict__ rn, long long total, int L,
                        double *__restrict__ out, int inverse)
{
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const double e = __ldg(rn + (k % L));
    out[k] = inverse ? ((e == 0.0) ? 0.0 : w[k] / e) : w[k] * e;
  }
}

__global__ void k_diffuse(double *__restrict__ w, long long total, int L, const double *__restrict__ coef,
                          double dt, const double *__restrict__ filter)
{
  for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < total; k += (long long)gridDim.x * blockDim.x) {
    const int l = (int)(k % L);
    const double f = filter ? __ldg(filter + l) : 1.0;
    w[k] = f * w[k] / (1.0 - dt * __ldg(coef + l));
  }
}

// kind 0: IntLonLat, 1: AvrLonLat, 2: ya_IntLon, 3: ya_AvrLon
__global__ void __launch_bounds__(256) k_lonlat(const double *__restrict__ g, int I, int J,
                                                const double *__restrict__ wgt, double *__restrict__ out, int kind)
{
  __shared__ double part[8];
  const int b = blockIdx.x;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const double *gb = g + (long long)b * I * J;
  const double dl = 2.0 * M_PI / I;
  double acc = 0.0;
  for (int j = warp; j < J; j += 8) {
    double s = 0.0;
    for (int i = lane; i < I; i += 32) s += __ldg(gb + (long long)j * I + i);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (kind >= 2) {
      if (lane == 0) out[(long long)b * J + j] = (kind == 3) ? s / I : s * dl;
    } else {
      acc += s * dl * 2.0 * __ldg(wgt + j);
    }
  }
  if (kind < 2) {
    if (lane == 0) part[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < 8; ++w) t += part[w];
      out[b] = (kind == 1) ? t / (4.0 * M_PI) : t;
    }
  }
}

}  // namespace

int launch_pack(const sht_plan *p, int op, const double2 *S, int ncolS, int nb, double *w0,
                double *w1, cudaStream_t s, double *const *wcol)
{
  if (nb <= 0) return SHT_OK;
  SpecArgs a{};
  a.ocol = wcol;
  a.S = S; a.ncolS = ncolS; a.o0 = w0; a.o1 = w1 ? w1 : w0;
  a.nb = nb; a.N = p->N; a.L = p->L; a.radius = p->radius;
  a.eps = p->d_eps; a.tiles = p->d_spec_tiles;
  a.M = p->M; a.zonal = p->zonal ? 1 : 0;
  dim3 grid(p->n_pack_tiles, (nb + kBC - 1) / kBC);
  switch (op) {
  case PACK_PLAIN: k_pack<PACK_PLAIN><<<grid, 256, 0, s>>>(a); break;
  case PACK_DIVLAMBDA: k_pack<PACK_DIVLAMBDA><<<grid, 256, 0, s>>>(a); break;
  case PACK_DIVMU: k_pack<PACK_DIVMU><<<grid, 256, 0, s>>>(a); break;
  case PACK_ALPHA: k_pack<PACK_ALPHA><<<grid, 256, 0, s>>>(a); break;
  case PACK_VORDIV: k_pack<PACK_VORDIV><<<grid, 256, 0, s>>>(a); break;
  default: set_error("pack: unknown operator"); return SHT_ERR_INVALID_ARG;
  }
  count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, "k_pack");
}

int launch_unpack(const sht_plan *p, int op, const double *w0, const double *w1, int nb,
                  double2 *S, int ncolS, cudaStream_t s, const double *const *wcol)
{
  if (nb <= 0) return SHT_OK;
  SpecArgs a{};
  a.icol = wcol;
  a.So = S; a.ncolS = ncolS; a.w0 = w0; a.w1 = w1 ? w1 : w0;
  a.nb = nb; a.N = p->N; a.L = p->L; a.radius = p->radius;
  a.eps = p->d_eps; a.tiles = p->d_spec_tiles;
  a.M = p->M; a.zonal = p->zonal ? 1 : 0;
  dim3 grid(p->n_spec_tiles, (nb + kBC - 1) / kBC);
  const size_t one = sizeof(double) * kMC * (kBC + 1);  // one staged run
  cudaError_t e = cudaSuccess;
  auto run = [&](auto kern, int nslots) {
    const size_t smem = one * nslots;
    e = kernel_setup((const void *)kern, smem, 256);
    if (e == cudaSuccess) kern<<<grid, 256, smem, s>>>(a);
  };
  switch (op) {
  case UNPACK_PLAIN: run(k_unpack<UNPACK_PLAIN>, unpack_nslots<UNPACK_PLAIN>()); break;
  case UNPACK_GRADLAMBDA: run(k_unpack<UNPACK_GRADLAMBDA>, unpack_nslots<UNPACK_GRADLAMBDA>()); break;
  case UNPACK_GRADMU: run(k_unpack<UNPACK_GRADMU>, unpack_nslots<UNPACK_GRADMU>()); break;
  case UNPACK_ALPHA: run(k_unpack<UNPACK_ALPHA>, unpack_nslots<UNPACK_ALPHA>()); break;
  case UNPACK_VORDIV2UV: run(k_unpack<UNPACK_VORDIV2UV>, unpack_nslots<UNPACK_VORDIV2UV>()); break;
  case UNPACK_HGRAD: run(k_unpack<UNPACK_HGRAD>, unpack_nslots<UNPACK_HGRAD>()); break;
  default: set_error("unpack: unknown operator"); return SHT_ERR_INVALID_ARG;
  }
  if (e != cudaSuccess) return cuda_fail(e, "k_unpack smem attribute");
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, "k_unpack");
}

static unsigned grid_for(long long total)
{
  long long g = (total + 255) / 256;
  if (g > 148 * 16) g = 148 * 16;
  return (unsigned)(g > 0 ? g : 1);
}

int launch_lapla(const sht_plan *p, const double *w, int nb, double *out, bool inverse, cudaStream_t s)
{
  const long long total = (long long)nb * p->L;
  if (total <= 0) return SHT_OK;
  k_lapla<<<grid_for(total), 256, 0, s>>>(w, p->d_rn, total, p->L, out, inverse ? 1 : 0);
  count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, "k_lapla");
}

int launch_diffuse(const sht_plan *p, double *w, int nb, const double *coef, double dt,
                   const double *filter, cudaStream_t s)
{
  const long long total = (long long)nb * p->L;
  if (total <= 0) return SHT_OK;
  k_diffuse<<<grid_for(total), 256, 0, s>>>(w, total, p->L, coef, dt, filter);
  count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, "k_diffuse");
}

int launch_lonlat_reduce(const sht_plan *p, const double *g, int nb, double *out, int kind, cudaStream_t s)
{
  if (nb <= 0) return SHT_OK;
  k_lonlat<<<nb, 256, 0, s>>>(g, p->I, p->J, p->d_wgt, out, kind);
  count_launch();
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, "k_lonlat");
}

}  // namespace sht
