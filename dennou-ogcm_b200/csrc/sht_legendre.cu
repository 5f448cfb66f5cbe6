// sht_legendre.cu -- per-zonal-wavenumber Legendre contraction in FP64.
//
// Analysis (space_discretization.tex:197-200), per m and 16 complex
// field-level columns:
//     c_n = sum_{jh} Pbar_n^m(mu_jh) * (n-m even ? Gs : Ga)[jh],
//     Gs/Ga = G(mu_N) +- G(mu_S) over the mirrored Gauss rows, which the
//     longitude transform delivers at F[m][col][jh] and F[m][col][JH + jh]
//     (the Gauss weight already folded in).
// Synthesis (:212-216):
//     Ge/Go[jh] = sum_{n-m even/odd} Pbar_n^m(mu_jh) a_n, written to
//     F[m][col][jh] and F[m][col][JH + jh]; the inverse longitude transform
//     forms G(mu_N) = Ge + Go and G(mu_S) = Ge - Go.
// Both are dense contractions run on the FP64 tensor pipe with
// mma.sync.m8n8k4.f64 (16 rows x 32 real columns per warp).  A thread block
// owns one m and one 16-column tile.  Its 8 warps split the rows (analysis) or
// latitudes (synthesis) into 16-wide groups.  When a band has fewer groups
// than warps (large m), the contraction dimension is split across warps as
// well, and the partial sums are reduced through shared memory.  Every warp
// therefore carries about the same share of the triangular band.
#include "sht_internal.h"

namespace sht {

namespace {
constexpr int kWarps = 8;
constexpr int kThreads = kWarps * 32;
constexpr int kCT = 16;              // complex columns per tile (32 real)
constexpr int kKC = 32;              // contraction chunk (latitudes or degrees)
constexpr int kGS = 2 * kCT + 4;     // 36 doubles: row stride, = 4 (mod 16) for conflict-free fragments
constexpr int kPS = kKC + 4;         // analysis P staging row stride (36)
constexpr int kPT = 16 + 4;          // synthesis P^T staging row stride (20)

struct LegArgs {
  const double2 *F;   // analysis input  F[m][col][j]
  double2 *S;         // analysis output S[row][col]
  const double2 *Sc;  // synthesis input
  double2 *Fo;        // synthesis output
  const double *P;
  const long long *poff;
  const int *rowoff;
  int N, J, JH, ncol;
};

__device__ __forceinline__ void dmma(double (&d)[2], double a, double b)
{
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

__device__ __forceinline__ int ksplit_for(int groups)
{
  int ks = 1;
  while (ks < kWarps && groups * ks * 2 <= kWarps) ks <<= 1;
  return ks;
}

// ------------------------------------------------------------------ analysis
template <int MAXU>
__global__ void __launch_bounds__(kThreads) k_leg_fwd_dmma(LegArgs a)
{
  extern __shared__ double smem[];
  double(*Gs)[kGS] = reinterpret_cast<double(*)[kGS]>(smem);
  double(*Ga)[kGS] = reinterpret_cast<double(*)[kGS]>(smem + kKC * kGS);
  double(*Pst)[16][kPS] = reinterpret_cast<double(*)[16][kPS]>(smem + 2 * kKC * kGS);
  double *red = smem + 2 * kKC * kGS;  // aliases Pst after the contraction

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int col0 = blockIdx.x * kCT, m = blockIdx.y;
  const int N = a.N, JH = a.JH;
  const int R = N + 2 - m, Re = (R + 1) >> 1, Ro = R >> 1;
  const int ngE = (Re + 15) >> 4, ngO = (Ro + 15) >> 4, ng = ngE + ngO;
  const int ks = ksplit_for(ng);
  const int nunits = ng * ks;
  const double *Pm = a.P + __ldg(a.poff + m);

  double acc[MAXU][2][4][2];
#pragma unroll
  for (int q = 0; q < MAXU; ++q)
#pragma unroll
    for (int t = 0; t < 2; ++t)
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) acc[q][t][nt][0] = acc[q][t][nt][1] = 0.0;

  for (int k0 = 0; k0 < JH; k0 += kKC) {
    const int kc = min(kKC, JH - k0);
    // stage Gs/Ga for this chunk: 16 columns x 32 half-latitudes
    for (int idx = tid; idx < kCT * kKC; idx += kThreads) {
      const int jh = idx % kKC, c = idx / kKC;
      double2 gs = make_double2(0.0, 0.0), ga = gs;
      if (jh < kc && col0 + c < a.ncol) {
        const double2 *Fc = a.F + ((long long)m * a.ncol + col0 + c) * a.J;
        gs = Fc[k0 + jh];
        ga = Fc[JH + k0 + jh];
      }
      Gs[jh][2 * c] = gs.x;
      Gs[jh][2 * c + 1] = gs.y;
      Ga[jh][2 * c] = ga.x;
      Ga[jh][2 * c + 1] = ga.y;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXU; ++q) {
      const int u = warp + kWarps * q;
      if (u < nunits) {
        const int g = u / ks, s = u - g * ks;
        const int par = (g < ngE) ? 0 : 1, gi = par ? g - ngE : g;
        // stage P rows r_i = par + 2 (16 gi + i), i < 16, for the chunk
        for (int e = lane; e < 16 * kKC; e += 32) {
          const int i = e / kKC, kk = e - i * kKC;
          const int r = par + 2 * (16 * gi + i);
          Pst[warp][i][kk] = (r < R && kk < kc) ? __ldg(Pm + (long long)r * JH + k0 + kk) : 0.0;
        }
        __syncwarp();
        const double(*G)[kGS] = par ? Ga : Gs;
        for (int st = s; st < kKC / 4; st += ks) {
          const int kb = 4 * st;
          const double a0 = Pst[warp][lane >> 2][kb + (lane & 3)];
          const double a1 = Pst[warp][8 + (lane >> 2)][kb + (lane & 3)];
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) {
            const double b = G[kb + (lane & 3)][8 * nt + (lane >> 2)];
            dmma(acc[q][0][nt], a0, b);
            dmma(acc[q][1][nt], a1, b);
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
  }

  // reduce the contraction splits
  if (ks > 1) {
    if (warp < nunits) {
      double *dst = red + ((long long)warp * 32 + lane) * 16;
#pragma unroll
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) {
          dst[(t * 4 + nt) * 2] = acc[0][t][nt][0];
          dst[(t * 4 + nt) * 2 + 1] = acc[0][t][nt][1];
        }
    }
    __syncthreads();
    if (warp < nunits && (warp % ks) == 0) {
      for (int s2 = 1; s2 < ks; ++s2) {
        const double *src = red + ((long long)(warp + s2) * 32 + lane) * 16;
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) {
            acc[0][t][nt][0] += src[(t * 4 + nt) * 2];
            acc[0][t][nt][1] += src[(t * 4 + nt) * 2 + 1];
          }
      }
    }
  }
  // write c_n for rows r = par + 2 (16 gi + 8 t + lane/4), complex column 4 nt + lane%4
  const long long rowbase = __ldg(a.rowoff + m);
#pragma unroll
  for (int q = 0; q < MAXU; ++q) {
    const int u = warp + kWarps * q;
    if (u >= nunits || (u % ks) != 0) continue;
    const int g = u / ks, par = (g < ngE) ? 0 : 1, gi = par ? g - ngE : g;
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int r = par + 2 * (16 * gi + 8 * t + (lane >> 2));
      if (r >= R) continue;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int c = col0 + 4 * nt + (lane & 3);
        if (c < a.ncol) a.S[(rowbase + r) * a.ncol + c] = make_double2(acc[q][t][nt][0], acc[q][t][nt][1]);
      }
    }
  }
}

// ----------------------------------------------------------------- synthesis
template <int MAXU>
__global__ void __launch_bounds__(kThreads) k_leg_inv_dmma(LegArgs a)
{
  extern __shared__ double smem[];
  double(*Ae)[kGS] = reinterpret_cast<double(*)[kGS]>(smem);             // [16][kGS]
  double(*Ao)[kGS] = reinterpret_cast<double(*)[kGS]>(smem + 16 * kGS);  // [16][kGS]
  double(*Pst)[2][16][kPT] = reinterpret_cast<double(*)[2][16][kPT]>(smem + 32 * kGS);
  double *red = smem + 32 * kGS;  // aliases Pst after the contraction

  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int col0 = blockIdx.x * kCT, m = blockIdx.y;
  const int N = a.N, JH = a.JH;
  const int R = N + 2 - m;
  const int ngj = (JH + 15) >> 4;
  const int ks = ksplit_for(ngj);
  const int nunits = ngj * ks;
  const double *Pm = a.P + __ldg(a.poff + m);
  const long long rowbase = __ldg(a.rowoff + m);

  double acc[MAXU][2][2][4][2];  // [unit][parity][jh tile][col tile][2]
#pragma unroll
  for (int q = 0; q < MAXU; ++q)
#pragma unroll
    for (int p = 0; p < 2; ++p)
#pragma unroll
      for (int t = 0; t < 2; ++t)
#pragma unroll
        for (int nt = 0; nt < 4; ++nt) acc[q][p][t][nt][0] = acc[q][p][t][nt][1] = 0.0;

  for (int r0 = 0; r0 < R; r0 += kKC) {
    // stage coefficient rows r0..r0+31 split by parity (16 each)
    for (int idx = tid; idx < kCT * kKC; idx += kThreads) {
      const int c = idx % kCT, rr = idx / kCT;
      const int r = r0 + rr;
      double2 v = make_double2(0.0, 0.0);
      if (r < R && col0 + c < a.ncol) v = a.Sc[(rowbase + r) * a.ncol + col0 + c];
      double(*A)[kGS] = (rr & 1) ? Ao : Ae;
      A[rr >> 1][2 * c] = v.x;
      A[rr >> 1][2 * c + 1] = v.y;
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < MAXU; ++q) {
      const int u = warp + kWarps * (q + MAXU * (int)blockIdx.z);
      if (u < nunits) {
        const int g = u / ks, s = u - g * ks;
        const int jh0 = 16 * g;
        // stage P^T: Pst[p][t][jh] = Pbar_{m + r0 + 2t + p}(mu_{jh0 + jh})
        for (int e = lane; e < 2 * 16 * 16; e += 32) {
          const int rr = e >> 4, jh = e & 15;
          const int r = r0 + rr;
          Pst[warp][rr & 1][rr >> 1][jh] = (r < R && jh0 + jh < JH) ? __ldg(Pm + (long long)r * JH + jh0 + jh) : 0.0;
        }
        __syncwarp();
        for (int st = s; st < 8; st += ks) {  // 8 steps: 4 per parity
          const int p = st >> 2, tb = 4 * (st & 3);
          const double(*A)[kGS] = p ? Ao : Ae;
          const double a0 = Pst[warp][p][tb + (lane & 3)][lane >> 2];
          const double a1 = Pst[warp][p][tb + (lane & 3)][8 + (lane >> 2)];
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) {
            const double b = A[tb + (lane & 3)][8 * nt + (lane >> 2)];
            if (p == 0) {
              dmma(acc[q][0][0][nt], a0, b);
              dmma(acc[q][0][1][nt], a1, b);
            } else {
              dmma(acc[q][1][0][nt], a0, b);
              dmma(acc[q][1][1][nt], a1, b);
            }
          }
        }
        __syncwarp();
      }
    }
    __syncthreads();
  }

  if (ks > 1) {
    if (warp < nunits) {
      double *dst = red + ((long long)warp * 32 + lane) * 32;
#pragma unroll
      for (int p = 0; p < 2; ++p)
#pragma unroll
        for (int t = 0; t < 2; ++t)
#pragma unroll
          for (int nt = 0; nt < 4; ++nt) {
            const int o = ((p * 2 + t) * 4 + nt) * 2;
            dst[o] = acc[0][p][t][nt][0];
            dst[o + 1] = acc[0][p][t][nt][1];
          }
    }
    __syncthreads();
    if (warp < nunits && (warp % ks) == 0) {
      for (int s2 = 1; s2 < ks; ++s2) {
        const double *src = red + ((long long)(warp + s2) * 32 + lane) * 32;
#pragma unroll
        for (int p = 0; p < 2; ++p)
#pragma unroll
          for (int t = 0; t < 2; ++t)
#pragma unroll
            for (int nt = 0; nt < 4; ++nt) {
              const int o = ((p * 2 + t) * 4 + nt) * 2;
              acc[0][p][t][nt][0] += src[o];
              acc[0][p][t][nt][1] += src[o + 1];
            }
      }
    }
  }
  // Ge at F[m][col][jh], Go at F[m][col][JH + jh]
#pragma unroll
  for (int q = 0; q < MAXU; ++q) {
    const int u = warp + kWarps * (q + MAXU * (int)blockIdx.z);
    if (u >= nunits || (u % ks) != 0) continue;
    const int jh0 = 16 * (u / ks);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int jh = jh0 + 8 * t + (lane >> 2);
      if (jh >= JH) continue;
#pragma unroll
      for (int nt = 0; nt < 4; ++nt) {
        const int c = col0 + 4 * nt + (lane & 3);
        if (c >= a.ncol) continue;
        const double er = acc[q][0][t][nt][0], ei = acc[q][0][t][nt][1];
        const double orr = acc[q][1][t][nt][0], oi = acc[q][1][t][nt][1];
        double2 *Fc = a.Fo + ((long long)m * a.ncol + c) * a.J;
        Fc[jh] = make_double2(er, ei);
        Fc[JH + jh] = make_double2(orr, oi);
      }
    }
  }
}

size_t fwd_smem() { return sizeof(double) * (2 * kKC * kGS + kWarps * 16 * kPS); }
size_t inv_smem()
{
  const size_t pst = (size_t)kWarps * 2 * 16 * kPT, red = (size_t)kWarps * 32 * 32;
  return sizeof(double) * (32 * kGS + (pst > red ? pst : red));
}

template <typename K>
int launch(K kern, dim3 grid, size_t smem, cudaStream_t s, const LegArgs &args, const char *name)
{
  cudaError_t e;
  if ((e = kernel_setup((const void *)kern, smem, kThreads)) != cudaSuccess) return cuda_fail(e, name);
  kern<<<grid, kThreads, smem, s>>>(args);
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, name);
}
}  // namespace

// Kernel for the plan's SHT_OPT_LEGENDRE_KERNEL setting: 1 per-band (this
// file), 2 paired persistent, 3 latitude-chunked persistent; 0 picks the
// paired kernel where the pair fits in shared memory, else the chunked one,
// else the per-band one.  A forced choice that does not cover the grid falls
// back the same way.
int pick_fp64_kernel(const sht_plan *p)
{
  const int want = p->leg_kernel;
  if (want == 1) return 1;
  if (want == 2 && leg_pair_supported(p)) return 2;
  if (want == 3 && leg_chunk_supported(p)) return 3;
  if (leg_pair_supported(p)) return 2;
  if (leg_chunk_supported(p)) return 3;
  return 1;
}

int launch_leg_fwd_fp64(const sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  switch (pick_fp64_kernel(p)) {
  case 2: return launch_leg_fwd_pair(p, F, ncol, S, s);
  case 3: return launch_leg_fwd_chunk(p, F, ncol, S, s);
  default: break;
  }
  LegArgs a{};
  a.F = F; a.S = S; a.P = p->d_P; a.poff = p->d_poff; a.rowoff = p->d_rowoff;
  a.N = p->N; a.J = p->J; a.JH = p->JH; a.ncol = ncol;
  const int R0 = p->N + 2, ng0 = ((R0 + 1) / 2 + 15) / 16 + (R0 / 2 + 15) / 16;
  const int maxu = (ng0 + kWarps - 1) / kWarps;
  dim3 grid((ncol + kCT - 1) / kCT, p->M);
  // the red buffer (8 x 32 x 16 doubles) fits inside the P staging area
  static_assert(kWarps * 16 * kPS >= kWarps * 32 * 16, "reduction buffer must fit in the P staging area");
  const size_t smem = fwd_smem();
  switch (maxu) {
  case 1: return launch(k_leg_fwd_dmma<1>, grid, smem, s, a, "k_leg_fwd_dmma");
  case 2: return launch(k_leg_fwd_dmma<2>, grid, smem, s, a, "k_leg_fwd_dmma");
  case 3: return launch(k_leg_fwd_dmma<3>, grid, smem, s, a, "k_leg_fwd_dmma");
  case 4: return launch(k_leg_fwd_dmma<4>, grid, smem, s, a, "k_leg_fwd_dmma");
  case 5: case 6: return launch(k_leg_fwd_dmma<6>, grid, smem, s, a, "k_leg_fwd_dmma");
  default: set_error("legendre: truncation too large"); return SHT_ERR_UNSUPPORTED_SIZE;
  }
}

int launch_leg_inv_fp64(const sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  switch (pick_fp64_kernel(p)) {
  case 2: return launch_leg_inv_pair(p, S, ncol, F, s);
  case 3: return launch_leg_inv_chunk(p, S, ncol, F, s);
  default: break;
  }
  LegArgs a{};
  a.Sc = S; a.Fo = F; a.P = p->d_P; a.poff = p->d_poff; a.rowoff = p->d_rowoff;
  a.N = p->N; a.J = p->J; a.JH = p->JH; a.ncol = ncol;
  const int ngj = (p->JH + 15) / 16;
  const int maxu = (ngj + kWarps - 1) / kWarps;
  dim3 grid((ncol + kCT - 1) / kCT, p->M);
  const size_t smem = inv_smem();
  // up to two 16-latitude units per warp; beyond that (JH > 256) the units
  // are split over two blocks (grid z), each staging the coefficient rows
  // itself, rather than four accumulator sets per warp that spill
  switch (maxu) {
  case 1: return launch(k_leg_inv_dmma<1>, grid, smem, s, a, "k_leg_inv_dmma");
  case 2: return launch(k_leg_inv_dmma<2>, grid, smem, s, a, "k_leg_inv_dmma");
  case 3: case 4: grid.z = 2; return launch(k_leg_inv_dmma<2>, grid, smem, s, a, "k_leg_inv_dmma");
  default: set_error("legendre: too many latitudes"); return SHT_ERR_UNSUPPORTED_SIZE;
  }
}

}  // namespace sht
