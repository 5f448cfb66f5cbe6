// sht_legendre_v3.cu -- persistent FP64 Legendre contraction for large grids,
// latitude-chunked (half-latitude counts that are multiples of 32: T170 and
// T341; the smaller grids use the paired kernels).
//
// Work items are (band pair (m, N-m), 16 complex field-level columns) as in
// the paired kernels: every pair holds N+4 degrees, so all items cost the
// same and each resident block takes a contiguous slice of the pair-major list.
// A pair's Legendre rows and data do not fit in shared memory at these sizes,
// so each item streams through two stages in latitude chunks, filled with
// 16-byte cp.async copies (zero-filling what lies outside the data).  The
// stage rows are 128-512 bytes long: per-row bulk copies would cost one copy
// request each, and at this length the request rate, not the bytes, would
// bound the fill.
//
//   analysis:  chunk = KC half-latitudes jh: the P rows of both bands for those
//              jh, and per column the runs of Gs and Ga (delivered by the
//              longitude transform at jh and JH + jh).  Each warp keeps up to JPW
//              (16 degrees x 32 real columns) accumulator blocks in registers
//              over the chunks of an item.
//   synthesis: chunk = KL half-latitudes of the output (32, or 16 at T341);
//              the coefficient panel of the item (both bands, all degrees) is
//              resident.  Each warp owns one 8-latitude tile for one parity and
//              4 (KL = 32) or 2 (KL = 16) of the four 8-column tiles, so each P
//              fragment feeds that many products, and writes its parity's sums
//              (the inverse longitude transform forms the north and south rows).
//              Rows past a band's last degree are zero coefficients (and finite
//              P rows), so the degree loop needs no bounds checks.
//
// The symmetric/antisymmetric split is Pbar(-mu) = (-1)^{n-m} Pbar(mu); the
// analysis follows space_discretization.tex:197-200, the synthesis :212-216.
// Shared-memory strides keep the FP64 fragment loads conflict-free: P rows
// PS = 2 (mod 8) doubles, data rows CS = 8 (mod 16), coefficient rows
// AS = 2 (mod 8).
#include "sht_internal.h"
#include "sht_dmma.cuh"

namespace sht {

namespace {

using dmma::cp16;
using dmma::cp_commit;
using dmma::cp_wait0;
using dmma::mma884;

constexpr int kW = 8;        // warps per block
constexpr int kT = kW * 32;  // threads per block
constexpr int kCT = 16;      // complex columns per item

struct V3Args {
  const double2 *F;   // analysis input F[m][col][j]
  double2 *S;         // analysis output S[row][col]
  const double2 *Sc;  // synthesis input
  double2 *Fo;        // synthesis output
  const double *P;
  const long long *poff;
  const int *rowoff;
  const int2 *pairs;
  int ntiles, nitems, per_cta;
  int N, J, JH, ncol;
};

__host__ __device__ __forceinline__ int band_rows(int N, int m) { return m >= 0 ? N + 2 - m : 0; }

// ------------------------------------------------------------------ analysis
template <int KC>
struct FwdGeo {
  static constexpr int PS = KC + 2;      // P row stride
  static constexpr int CS = 4 * KC + 8;  // data row: north run, south run (complex)
  static_assert(PS % 8 == 2 && CS % 16 == 8, "conflict-free strides");
};

template <int KC>
__device__ void issue_fwd_chunk(const V3Args &a, double *Pst, double *Gst, int2 pr, int col0, int k0)
{
  using G = FwdGeo<KC>;
  constexpr int CPR = KC / 2;  // 16-byte copies per P row
  const int Ra = band_rows(a.N, pr.x), Rb = band_rows(a.N, pr.y);
  const double *Pa = a.P + a.poff[pr.x] + k0;
  const double *Pb = (pr.y >= 0 ? a.P + a.poff[pr.y] : a.P) + k0;
  for (int q = threadIdx.x; q < (Ra + Rb) * CPR; q += kT) {
    const int row = q / CPR, ch = q % CPR;
    const double *src = (row < Ra ? Pa + (long long)row * a.JH : Pb + (long long)(row - Ra) * a.JH) + 2 * ch;
    cp16(Pst + row * G::PS + 2 * ch, src, true);
  }
  // per column row: the Gs run at jh = k0.. and the Ga run at JH + k0..
  const int nrow = (pr.y >= 0 ? 2 : 1) * kCT;
  for (int q = threadIdx.x; q < nrow * 2 * KC; q += kT) {
    const int row = q / (2 * KC), e = q % (2 * KC);
    const int run = e / KC, i = e % KC;
    const int b = row % kCT, m = (row < kCT) ? pr.x : pr.y;
    const bool ok = col0 + b < a.ncol;
    const int j = run * a.JH + k0 + i;
    const double2 *src = ok ? a.F + ((long long)m * a.ncol + col0 + b) * a.J + j : a.F;
    cp16(Gst + row * G::CS + 2 * (run * KC + i), src, ok);
  }
}

// jobs of a pair: (band, parity, 16-degree group), band a then band b
struct Jobs {
  int Ra, Rb, gEa, gOa, gEb, gOb, n;
  __device__ Jobs(int N, int2 pr)
  {
    Ra = band_rows(N, pr.x);
    Rb = band_rows(N, pr.y);
    gEa = ((Ra + 1) / 2 + 15) / 16; gOa = (Ra / 2 + 15) / 16;
    gEb = ((Rb + 1) / 2 + 15) / 16; gOb = (Rb / 2 + 15) / 16;
    n = gEa + gOa + gEb + gOb;
  }
  __device__ void decode(int job, int &mi, int &par, int &gi) const
  {
    if (job < gEa) { mi = 0; par = 0; gi = job; }
    else if (job < gEa + gOa) { mi = 0; par = 1; gi = job - gEa; }
    else if (job < gEa + gOa + gEb) { mi = 1; par = 0; gi = job - gEa - gOa; }
    else { mi = 1; par = 1; gi = job - gEa - gOa - gEb; }
  }
};

template <int KC, int JPW>
__global__ void __launch_bounds__(kT, 1) k_leg_fwd_chunk(V3Args a)
{
  using G = FwdGeo<KC>;
  extern __shared__ __align__(16) double sm[];
  const int Pst = (a.N + 4) * G::PS, Gst = 2 * kCT * G::CS;
  double *const P0 = sm, *const G0 = sm + Pst, *const P1 = sm + Pst + Gst, *const G1 = P1 + Pst;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int it0 = blockIdx.x * a.per_cta;
  const int it1 = min(a.nitems, it0 + a.per_cta);
  if (it0 >= it1) return;
  const int nch = a.JH / KC;
  const int total = (it1 - it0) * nch;
  issue_fwd_chunk<KC>(a, P0, G0, a.pairs[it0 / a.ntiles], (it0 % a.ntiles) * kCT, 0);
  cp_commit();

  double acc[JPW][2][4][2];
  for (int c = 0; c < total; ++c) {
    const int it = it0 + c / nch, kc = c % nch, st = c & 1;
    const int2 pr = a.pairs[it / a.ntiles];
    const int col0 = (it % a.ntiles) * kCT;
    double *const Pc = st ? P1 : P0, *const Gc = st ? G1 : G0;
    cp_wait0();
    __syncthreads();  // chunk c is in; every warp is done with chunk c-1's stage
    if (c + 1 < total) {
      const int itn = it0 + (c + 1) / nch, kn = (c + 1) % nch;
      issue_fwd_chunk<KC>(a, st ? P0 : P1, st ? G0 : G1, a.pairs[itn / a.ntiles], (itn % a.ntiles) * kCT, kn * KC);
    }
    cp_commit();

    const Jobs jb(a.N, pr);
    if (kc == 0) {
#pragma unroll
      for (int t = 0; t < JPW; ++t)
#pragma unroll
        for (int h = 0; h < 2; ++h)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) acc[t][h][nt][0] = acc[t][h][nt][1] = 0.0;
    }
#pragma unroll
    for (int t = 0; t < JPW; ++t) {
      const int job = warp + kW * t;
      if (job >= jb.n) break;
      int mi, par, gi;
      jb.decode(job, mi, par, gi);
      const int R = mi ? jb.Rb : jb.Ra;
      const double *Pm = Pc + (mi ? jb.Ra : 0) * G::PS;
      const double *Gp = Gc + mi * kCT * G::CS + (par ? 2 * KC : 0);
      const int r0 = par + 2 * (16 * gi + (lane >> 2));
      const double *pa0 = Pm + min(r0, R - 1) * G::PS + (lane & 3);
      const double *pa1 = Pm + min(r0 + 16, R - 1) * G::PS + (lane & 3);
      const double *gb = Gp + (lane >> 3) * G::CS + ((lane >> 2) & 1) + 2 * (lane & 3);
#pragma unroll
      for (int kb = 0; kb < KC; kb += 4) {
        const double a0 = pa0[kb], a1 = pa1[kb];
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          const double b = gb[4 * nt * G::CS + 2 * kb];
          mma884(acc[t][0][nt], a0, b);
          mma884(acc[t][1][nt], a1, b);
        }
      }
    }
    if (kc == nch - 1) {
#pragma unroll
      for (int t = 0; t < JPW; ++t) {
        const int job = warp + kW * t;
        if (job >= jb.n) break;
        int mi, par, gi;
        jb.decode(job, mi, par, gi);
        const int m = mi ? pr.y : pr.x, R = mi ? jb.Rb : jb.Ra;
        const long long rowbase = a.rowoff[m];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int r = par + 2 * (16 * gi + 8 * h + (lane >> 2));
          if (r >= R) continue;
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) {
            const int col = col0 + 4 * nt + (lane & 3);
            if (col < a.ncol) a.S[(rowbase + r) * a.ncol + col] = make_double2(acc[t][h][nt][0], acc[t][h][nt][1]);
          }
        }
      }
    }
  }
  cp_wait0();
}

// ----------------------------------------------------------------- synthesis
constexpr int kAS = 2 * kCT + 2;  // coefficient row stride
static_assert(kAS % 8 == 2, "conflict-free strides");

template <int KL>
struct InvGeo {
  static constexpr int PS = KL + 2;            // P chunk row stride
  static constexpr int NLT = KL / 8;           // 8-latitude tiles per chunk
  static constexpr int CG = kW / (2 * NLT);    // column groups (warps per tile and parity)
  static constexpr int CPW = 4 / CG;           // 8-column tiles per warp
  static_assert(PS % 8 == 2 && CG * CPW == 4, "layout");
};

// coefficient rows of a pair: band a at 0, band b at acap(Ra); at least 8
// zero rows after each band (a degree step reads up to 5 past the last
// degree).  Both bands hold N+4 degrees, so acap(Ra) + acap(Rb) <= N + 34 <=
// coef_rows(N).
__host__ __device__ __forceinline__ int acap(int R) { return (R + 8 + 7) & ~7; }
__host__ __device__ __forceinline__ int coef_rows(int N) { return (N + 4 + 30 + 7) & ~7; }
// P rows of a stage: both bands and 8 rows of slack that stay finite
__host__ __device__ __forceinline__ int pinv_rows(int N) { return N + 4 + 8; }

// Coefficient panel of an item: the valid columns of every degree row of both
// bands, zeros for the columns past ncol and for the 8+ rows after each band.
__device__ void issue_coef(const V3Args &a, double *Ast, int2 pr, int col0)
{
  const int Ra = band_rows(a.N, pr.x), Rb = band_rows(a.N, pr.y);
  const int ca = acap(Ra), rows = ca + (pr.y >= 0 ? acap(Rb) : 0);
  const int c = threadIdx.x % kCT;
  const bool cok = col0 + c < a.ncol;
  const double2 *Sa = a.Sc + (long long)a.rowoff[pr.x] * a.ncol + col0 + c;
  const double2 *Sb = pr.y >= 0 ? a.Sc + (long long)a.rowoff[pr.y] * a.ncol + col0 + c : Sa;
  for (int row = threadIdx.x / kCT; row < rows; row += kT / kCT) {
    const bool second = row >= ca;
    const int r = second ? row - ca : row;
    const bool ok = cok && r < (second ? Rb : Ra);
    cp16(Ast + row * kAS + 2 * c, ok ? (second ? Sb : Sa) + (long long)r * a.ncol : a.Sc, ok);
  }
}

template <int KL>
__device__ void issue_pinv_chunk(const V3Args &a, double *Pst, int2 pr, int l0)
{
  constexpr int CPR = KL / 2;
  const int Ra = band_rows(a.N, pr.x), Rb = band_rows(a.N, pr.y);
  const double *Pa = a.P + a.poff[pr.x] + l0;
  const double *Pb = (pr.y >= 0 ? a.P + a.poff[pr.y] : a.P) + l0;
  for (int q = threadIdx.x; q < (Ra + Rb) * CPR; q += kT) {
    const int row = q / CPR, ch = q % CPR;
    const double *src = (row < Ra ? Pa + (long long)row * a.JH : Pb + (long long)(row - Ra) * a.JH) + 2 * ch;
    cp16(Pst + row * InvGeo<KL>::PS + 2 * ch, src, true);
  }
}

// DB: two coefficient panels (the next item's streams in with the last chunk
// of the current one); otherwise one, loaded at the start of each item.
template <int KL, bool DB>
__global__ void __launch_bounds__(kT, 1) k_leg_inv_chunk(V3Args a)
{
  using G = InvGeo<KL>;
  constexpr int NLT = G::NLT, CPW = G::CPW;
  extern __shared__ __align__(16) double sm[];
  const int Pst = pinv_rows(a.N) * G::PS;
  const int Ast = coef_rows(a.N) * kAS;
  double *const P0 = sm, *const P1 = sm + Pst, *const A0 = sm + 2 * Pst, *const A1 = DB ? A0 + Ast : A0;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int it0 = blockIdx.x * a.per_cta;
  const int it1 = min(a.nitems, it0 + a.per_cta);
  if (it0 >= it1) return;
  const int nch = a.JH / KL;
  const int total = (it1 - it0) * nch;
  // this warp: latitude tile lt, parity par, column tiles cg*CPW .. +CPW
  const int lt = warp % NLT, par = (warp / NLT) & 1, cg = warp / (2 * NLT);

  // P stages start at zero so that slack rows read past the last band stay finite
  for (int q = threadIdx.x; q < 2 * Pst; q += kT) sm[q] = 0.0;
  __syncthreads();
  issue_coef(a, A0, a.pairs[it0 / a.ntiles], (it0 % a.ntiles) * kCT);
  issue_pinv_chunk<KL>(a, P0, a.pairs[it0 / a.ntiles], 0);
  cp_commit();

  for (int c = 0; c < total; ++c) {
    const int it = it0 + c / nch, kc = c % nch, st = c & 1;
    const int ii = (it - it0) & 1;
    const int2 pr = a.pairs[it / a.ntiles];
    const int col0 = (it % a.ntiles) * kCT;
    double *const Pc = st ? P1 : P0;
    double *const Ac = (DB && ii) ? A1 : A0;
    cp_wait0();
    __syncthreads();  // chunk c is in; chunk c-1's stages are free
    if (!DB && kc == 0 && c > 0) {
      // the single coefficient panel is free only now
      issue_coef(a, A0, pr, col0);
      cp_commit();
      cp_wait0();
      __syncthreads();
    }
    if (c + 1 < total) {
      const int itn = it0 + (c + 1) / nch, kn = (c + 1) % nch;
      const int2 pn = a.pairs[itn / a.ntiles];
      issue_pinv_chunk<KL>(a, st ? P0 : P1, pn, kn * KL);
      if (DB && kn == 0) issue_coef(a, ii ? A0 : A1, pn, (itn % a.ntiles) * kCT);
    }
    cp_commit();

    const int Ra = band_rows(a.N, pr.x);
    const int nm = (pr.y >= 0) ? 2 : 1;
    double acc[2][CPW][2];  // [band][column tile][2]
#pragma unroll
    for (int mi = 0; mi < 2; ++mi) {
#pragma unroll
      for (int ct = 0; ct < CPW; ++ct) acc[mi][ct][0] = acc[mi][ct][1] = 0.0;
      if (mi >= nm) continue;
      const int R = mi ? band_rows(a.N, pr.y) : Ra;
      const int steps = ((R - par + 1) / 2 + 3) / 4;  // 4 degrees of this parity per step
      const int r = par + 2 * (lane & 3);
      const double *pa = Pc + ((mi ? Ra : 0) + r) * G::PS + 8 * lt + (lane >> 2);
      const double *pb = Ac + ((mi ? acap(Ra) : 0) + r) * kAS + 8 * CPW * cg + (lane >> 2);
#pragma unroll 2
      for (int s = 0; s < steps; ++s) {
        const double av = pa[0];
#pragma unroll
        for (int ct = 0; ct < CPW; ++ct) mma884(acc[mi][ct], av, pb[8 * ct]);
        pa += 8 * G::PS;
        pb += 8 * kAS;
      }
    }
    // each warp writes its parity: even-degree sums at F[m][col][jh], odd at JH + jh
    const int jh = kc * KL + 8 * lt + (lane >> 2);
#pragma unroll
    for (int mi = 0; mi < 2; ++mi) {
      if (mi >= nm) continue;
      const int m = mi ? pr.y : pr.x;
#pragma unroll
      for (int ct = 0; ct < CPW; ++ct) {
        const int col = col0 + 4 * (CPW * cg + ct) + (lane & 3);
        if (col >= a.ncol) continue;
        a.Fo[((long long)m * a.ncol + col) * a.J + par * a.JH + jh] = make_double2(acc[mi][ct][0], acc[mi][ct][1]);
      }
    }
  }
  cp_wait0();
}

// ------------------------------------------------------------------ launch
struct Choice {
  int KC, JPW, KL;
  bool DB;
  size_t fwd_smem, inv_smem;
};

int max_jobs(int N)
{
  int best = 0;
  for (int m = 0; m <= N - m; ++m) {
    const int mb = (m == N - m) ? -1 : N - m;
    const int Ra = N + 2 - m, Rb = mb >= 0 ? N + 2 - mb : 0;
    const int n = ((Ra + 1) / 2 + 15) / 16 + (Ra / 2 + 15) / 16 + ((Rb + 1) / 2 + 15) / 16 + (Rb / 2 + 15) / 16;
    best = n > best ? n : best;
  }
  return best;
}

bool choose_tile(const sht_plan *p, int want, Choice *c)
{
  const size_t lim = 227 * 1024;
  if (p->JH % 32 != 0) return false;
  // latitudes per chunk: 32 up to JH = 128, 16 above; the plan's
  // SHT_OPT_LEGENDRE_TILE (16 or 32) overrides it where the stages fit
  c->KC = (want == 16 || want == 32) ? want : (p->JH <= 128) ? 32 : 16;
  c->KL = c->KC;
  const int jobs = max_jobs(p->N);
  c->JPW = (jobs + kW - 1) / kW;
  if (c->JPW < 2) c->JPW = 2;
  if (c->JPW > 4) return false;
  const int prow = p->N + 4;
  c->fwd_smem = sizeof(double) * 2 * ((size_t)prow * (c->KC + 2) + 2 * kCT * (4 * (size_t)c->KC + 8));
  const size_t pst = (size_t)pinv_rows(p->N) * (c->KL + 2);
  const size_t ast = (size_t)coef_rows(p->N) * kAS;
  c->DB = sizeof(double) * (2 * pst + 2 * ast) <= lim;
  c->inv_smem = sizeof(double) * (2 * pst + (c->DB ? 2 : 1) * ast);
  return c->fwd_smem <= lim && c->inv_smem <= lim;
}

// the plan's tile choice, or the automatic one where that does not fit
bool choose(const sht_plan *p, Choice *c)
{
  if (choose_tile(p, p->leg_tile, c)) return true;
  return p->leg_tile != 0 && choose_tile(p, 0, c);
}

template <typename K>
int run(K kern, size_t smem, const sht_plan *p, V3Args &a, cudaStream_t s, const char *name)
{
  int per_sm = 0;
  cudaError_t e = kernel_setup((const void *)kern, smem, kT, &per_sm);
  if (e != cudaSuccess || per_sm < 1) return cuda_fail(e == cudaSuccess ? cudaErrorInvalidConfiguration : e, name);
  const int slots = grid_sms(p) * per_sm;
  a.per_cta = (a.nitems + slots - 1) / slots;
  const int grid = (a.nitems + a.per_cta - 1) / a.per_cta;
  kern<<<grid, kT, smem, s>>>(a);
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, name);
}

int launch_chunk(const sht_plan *p, bool inverse, const double2 *in, int ncol, double2 *out, cudaStream_t s)
{
  Choice c;
  if (!choose(p, &c)) { set_error("legendre: grid outside the chunked kernels"); return SHT_ERR_UNSUPPORTED_SIZE; }
  V3Args a{};
  if (inverse) { a.Sc = in; a.Fo = out; } else { a.F = in; a.S = out; }
  a.P = p->d_P; a.poff = p->d_poff; a.rowoff = p->d_rowoff; a.pairs = p->d_pairs;
  a.N = p->N; a.J = p->J; a.JH = p->JH; a.ncol = ncol;
  a.ntiles = (ncol + kCT - 1) / kCT;
  a.nitems = p->n_pairs * a.ntiles;
  if (inverse) {
    if (c.KL == 32)
      return c.DB ? run(k_leg_inv_chunk<32, true>, c.inv_smem, p, a, s, "k_leg_inv_chunk")
                  : run(k_leg_inv_chunk<32, false>, c.inv_smem, p, a, s, "k_leg_inv_chunk");
    return c.DB ? run(k_leg_inv_chunk<16, true>, c.inv_smem, p, a, s, "k_leg_inv_chunk")
                : run(k_leg_inv_chunk<16, false>, c.inv_smem, p, a, s, "k_leg_inv_chunk");
  }
  switch (c.KC * 10 + c.JPW) {
  case 322: return run(k_leg_fwd_chunk<32, 2>, c.fwd_smem, p, a, s, "k_leg_fwd_chunk");
  case 323: return run(k_leg_fwd_chunk<32, 3>, c.fwd_smem, p, a, s, "k_leg_fwd_chunk");
  case 324: return run(k_leg_fwd_chunk<32, 4>, c.fwd_smem, p, a, s, "k_leg_fwd_chunk");
  case 162: return run(k_leg_fwd_chunk<16, 2>, c.fwd_smem, p, a, s, "k_leg_fwd_chunk");
  case 163: return run(k_leg_fwd_chunk<16, 3>, c.fwd_smem, p, a, s, "k_leg_fwd_chunk");
  case 164: return run(k_leg_fwd_chunk<16, 4>, c.fwd_smem, p, a, s, "k_leg_fwd_chunk");
  default: set_error("legendre: chunked kernel configuration"); return SHT_ERR_UNSUPPORTED_SIZE;
  }
}

}  // namespace

bool leg_chunk_supported(const sht_plan *p)
{
  Choice c;
  return p->n_pairs > 0 && choose(p, &c);
}

int launch_leg_fwd_chunk(const sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  return launch_chunk(p, false, F, ncol, S, s);
}

int launch_leg_inv_chunk(const sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  return launch_chunk(p, true, S, ncol, F, s);
}

}  // namespace sht
