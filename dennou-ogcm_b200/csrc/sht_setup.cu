// sht_setup.cu -- plan tables: Gauss-Legendre nodes/weights and the
// associated-Legendre table, both generated on the device in FP64, plus the
// small host-built tables (twiddles, recurrence coefficients, row scales).
//
// Follows doc/description/ogcm/space_discretization.tex:33-38 (Gauss grid,
// mu ascending), :205-209 (weights normalised to sum 1), :169 (Pbar
// normalised to 2) and :250-257 (normalised three-term recurrence), which is
// what wa_Initial sets up inside SPMODEL (SpmlUtil_mod.f90:218-223).
#include "sht_internal.h"

#include <cmath>
#include <cstring>

namespace sht {

// One thread per positive root of P_J: Newton iteration on the three-term
// recurrence, started from the Tricomi-type estimate cos(pi (k+3/4)/(J+1/2)).
__global__ void k_gauss_nodes(int J, double *mu, double *wgt)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= (J + 1) / 2) return;
  double x = cos(M_PI * (k + 0.75) / (J + 0.5));
  double dp = 1.0;
  for (int it = 0; it < 100; ++it) {
    double p0 = 1.0, p1 = x;
    for (int n = 2; n <= J; ++n) {
      const double p2 = ((2.0 * n - 1.0) * x * p1 - (n - 1.0) * p0) / n;
      p0 = p1;
      p1 = p2;
    }
    dp = J * (x * p1 - p0) / (x * x - 1.0);
    const double dx = p1 / dp;
    x -= dx;
    if (fabs(dx) < 1e-16 * (1.0 + fabs(x)) && it > 2) break;
  }
  // derivative at the converged root
  {
    double p0 = 1.0, p1 = x;
    for (int n = 2; n <= J; ++n) {
      const double p2 = ((2.0 * n - 1.0) * x * p1 - (n - 1.0) * p0) / n;
      p0 = p1;
      p1 = p2;
    }
    dp = J * (x * p1 - p0) / (x * x - 1.0);
  }
  const double w = 1.0 / ((1.0 - x * x) * dp * dp);  // sums to 1 over all J roots
  mu[J - 1 - k] = x;
  mu[k] = -x;
  wgt[J - 1 - k] = w;
  wgt[k] = w;
  if ((J & 1) && k == J / 2) mu[k] = 0.0;
}

// Pbar_n^m(mu_j) for the northern rows, one thread per (m, jh):
//   Pbar_m^m = prod_{k<=m} sqrt((2k+1)/(2k)) (1-mu^2)^{m/2}
//   Pbar_{n+1}^m = (mu Pbar_n^m - eps_n^m Pbar_{n-1}^m) / eps_{n+1}^m.
__global__ void k_legendre_table(int N, int J, int JH, const double *__restrict__ mu,
                                 const double *__restrict__ eps, const long long *__restrict__ poff,
                                 double *__restrict__ P)
{
  const int jh = blockIdx.x * blockDim.x + threadIdx.x;
  const int m = blockIdx.y;
  if (jh >= JH || m > N) return;
  const double x = mu[J - JH + jh];
  const double s = sqrt((1.0 - x) * (1.0 + x));
  double pmm = 1.0;
  for (int k = 1; k <= m; ++k) pmm *= sqrt((2.0 * k + 1.0) / (2.0 * k)) * s;
  double *col = P + poff[m] + jh;
  const double *e = eps + (long long)m * (N + 3);
  double pm2 = 0.0, pm1 = pmm;
  col[0] = pmm;
  for (int n = m + 1; n <= N + 1; ++n) {
    const double pn = (x * pm1 - e[n - 1] * pm2) / e[n];
    col[(long long)(n - m) * JH] = pn;
    pm2 = pm1;
    pm1 = pn;
  }
}

static int ilog2_exact(int n)
{
  int l = 0;
  if (n <= 0) return -1;
  while ((1 << l) < n) ++l;
  return ((1 << l) == n) ? l : -1;
}

template <typename T>
static int dalloc(T **ptr, size_t count)
{
  cudaError_t e = cudaMalloc((void **)ptr, sizeof(T) * (count ? count : 1));
  if (e != cudaSuccess) return cuda_fail(e, "cudaMalloc(plan table)");
  return SHT_OK;
}

int build_tables(sht_plan *p)
{
  const int I = p->I, J = p->J, N = p->N, JH = p->JH, NC = p->NC;
  int lg = p->zonal ? 0 : ilog2_exact(NC);
  p->fb = lg / 2;
  p->fa = lg - p->fb;
  p->R = (long long)(N + 1) * (N + 4) / 2;
  p->M = p->zonal ? 1 : N + 1;
  p->L = p->zonal ? N + 1 : (N + 1) * (N + 1);
  int rc;
  // --- Gauss nodes and weights on the device
  if ((rc = dalloc(&p->d_mu, J)) || (rc = dalloc(&p->d_wgt, J))) return rc;
  k_gauss_nodes<<<(J / 2 + 127) / 128, 128, 0, p->stream>>>(J, p->d_mu, p->d_wgt);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return cuda_fail(e, "k_gauss_nodes");
  p->h_mu.resize(J);
  p->h_wgt.resize(J);
  if ((e = cudaMemcpyAsync(p->h_mu.data(), p->d_mu, sizeof(double) * J, cudaMemcpyDeviceToHost, p->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(p->h_wgt.data(), p->d_wgt, sizeof(double) * J, cudaMemcpyDeviceToHost, p->stream)) != cudaSuccess ||
      (e = cudaStreamSynchronize(p->stream)) != cudaSuccess)
    return cuda_fail(e, "gauss nodes readback");

  // --- recurrence coefficients eps_n^m, n = 0..N+2 (host: closed form)
  std::vector<double> eps((size_t)(N + 1) * (N + 3));
  for (int m = 0; m <= N; ++m)
    for (int n = 0; n <= N + 2; ++n)
      eps[(size_t)m * (N + 3) + n] = (n < m || n == 0) ? 0.0 : std::sqrt(((double)n * n - (double)m * m) / (4.0 * n * n - 1.0));
  if ((rc = dalloc(&p->d_eps, eps.size()))) return rc;
  if ((e = cudaMemcpyAsync(p->d_eps, eps.data(), sizeof(double) * eps.size(), cudaMemcpyHostToDevice, p->stream)) != cudaSuccess)
    return cuda_fail(e, "eps upload");

  // --- Legendre table on the device
  std::vector<long long> poff(N + 2);
  long long off = 0;
  for (int m = 0; m <= N; ++m) { poff[m] = off; off += (long long)(N + 2 - m) * JH; }
  poff[N + 1] = off;
  if ((rc = dalloc(&p->d_poff, N + 2)) || (rc = dalloc(&p->d_P, (size_t)off))) return rc;
  if ((e = cudaMemcpyAsync(p->d_poff, poff.data(), sizeof(long long) * (N + 2), cudaMemcpyHostToDevice, p->stream)) != cudaSuccess)
    return cuda_fail(e, "poff upload");
  dim3 grid((JH + 127) / 128, N + 1);
  k_legendre_table<<<grid, 128, 0, p->stream>>>(N, J, JH, p->d_mu, p->d_eps, p->d_poff, p->d_P);
  count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "k_legendre_table");

  // --- internal row offsets
  p->h_rowoff.resize(N + 2);
  int ro = 0;
  for (int m = 0; m <= N; ++m) { p->h_rowoff[m] = ro; ro += N + 2 - m; }
  p->h_rowoff[N + 1] = ro;
  if ((rc = dalloc(&p->d_rowoff, N + 2))) return rc;
  if ((e = cudaMemcpyAsync(p->d_rowoff, p->h_rowoff.data(), sizeof(int) * (N + 2), cudaMemcpyHostToDevice, p->stream)) != cudaSuccess)
    return cuda_fail(e, "rowoff upload");

  // --- twiddles (long double on the host, rounded once)
  std::vector<double2> tw(NC), twI(NC);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int k = 0; k < NC; ++k) {
    long double t = -2.0L * pi * k / NC;
    tw[k] = make_double2((double)cosl(t), (double)sinl(t));
    long double u = -2.0L * pi * k / I;
    twI[k] = make_double2((double)cosl(u), (double)sinl(u));
  }
  if ((rc = dalloc(&p->d_tw, NC)) || (rc = dalloc(&p->d_twI, NC))) return rc;
  if ((e = cudaMemcpyAsync(p->d_tw, tw.data(), sizeof(double2) * NC, cudaMemcpyHostToDevice, p->stream)) != cudaSuccess ||
      (e = cudaMemcpyAsync(p->d_twI, twI.data(), sizeof(double2) * NC, cudaMemcpyHostToDevice, p->stream)) != cudaSuccess)
    return cuda_fail(e, "twiddle upload");

  // --- row scales
  std::vector<double> rs((size_t)RS_COUNT * J);
  for (int j = 0; j < J; ++j) {
    const double mu = p->h_mu[j], w = p->h_wgt[j];
    const double c2 = (1.0 - mu) * (1.0 + mu), c = std::sqrt(c2);
    rs[RS_FWD_PLAIN * J + j] = w / I;
    rs[RS_FWD_INV1MMU2 * J + j] = w / (I * c2);
    rs[RS_INV_PLAIN * J + j] = 1.0;
    rs[RS_INV_INVCOS * J + j] = 1.0 / c;
    rs[RS_INV_INVA1MMU2 * J + j] = 1.0 / (p->radius * c2);
    rs[RS_INV_INVACOS * J + j] = 1.0 / (p->radius * c);
    rs[RS_FWD_INVCOS * J + j] = w / (I * c);
  }
  if ((rc = dalloc(&p->d_rowscale, rs.size()))) return rc;
  if ((e = cudaMemcpyAsync(p->d_rowscale, rs.data(), sizeof(double) * rs.size(), cudaMemcpyHostToDevice, p->stream)) != cudaSuccess)
    return cuda_fail(e, "rowscale upload");

  // --- Laplacian eigenvalues rn(l,1) = -n(n+1) (zonal layout: l = n)
  std::vector<double> rn(p->L);
  for (int n = 0; n <= N; ++n)
    for (int m = -n; m <= n; ++m)
      if (!p->zonal) rn[n * (n + 1) + m] = -(double)n * (n + 1);
      else if (m == 0) rn[n] = -(double)n * (n + 1);
  if ((rc = dalloc(&p->d_rn, p->L))) return rc;
  if ((e = cudaMemcpyAsync(p->d_rn, rn.data(), sizeof(double) * p->L, cudaMemcpyHostToDevice, p->stream)) != cudaSuccess)
    return cuda_fail(e, "rn upload");
  // --- tiles (n, m0) of the spectral layout conversions, n ascending
  std::vector<int2> tiles;
  for (int n = 0; n <= N + 1; ++n) {
    if (n == N + 1) p->n_pack_tiles = (int)tiles.size();
    const int mmax = p->zonal ? 0 : (n < N ? n : N);
    for (int m0 = 0; m0 <= mmax; m0 += 32) tiles.push_back(make_int2(n, m0));
  }
  p->n_spec_tiles = (int)tiles.size();
  // --- band pairs (m, N-m) with N+4 degrees each, plus the middle band of even N
  std::vector<int2> pairs;
  if (p->zonal) {
    pairs.push_back(make_int2(0, -1));  // the m = 0 band alone
  } else {
    for (int m = 0; m < N - m; ++m) pairs.push_back(make_int2(m, N - m));
    if (N % 2 == 0) pairs.push_back(make_int2(N / 2, -1));
  }
  p->n_pairs = (int)pairs.size();
  if ((rc = dalloc(&p->d_pairs, pairs.size()))) return rc;
  if ((e = cudaMemcpyAsync(p->d_pairs, pairs.data(), sizeof(int2) * pairs.size(), cudaMemcpyHostToDevice, p->stream)) != cudaSuccess)
    return cuda_fail(e, "pair table upload");
  if ((e = cudaDeviceGetAttribute(&p->num_sms, cudaDevAttrMultiProcessorCount, p->device)) != cudaSuccess)
    return cuda_fail(e, "SM count");
  if ((rc = dalloc(&p->d_spec_tiles, tiles.size()))) return rc;
  if ((e = cudaMemcpyAsync(p->d_spec_tiles, tiles.data(), sizeof(int2) * tiles.size(), cudaMemcpyHostToDevice, p->stream)) != cudaSuccess)
    return cuda_fail(e, "spectral tiles upload");
  if ((e = cudaStreamSynchronize(p->stream)) != cudaSuccess) return cuda_fail(e, "plan tables");
  return SHT_OK;
}

}  // namespace sht
