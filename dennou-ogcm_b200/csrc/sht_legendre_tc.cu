// sht_legendre_tc.cu -- split-precision Legendre contraction on tcgen05.
//
// Both FP64 operands of c_n = sum_jh P_n(mu_jh) G(mu_jh) are written as
// power-of-two scaled fixed-point numbers in balanced base-256 digits:
//     x = 2^e * sum_{s=0..6} d_s 2^{-7-8s},   d_s integers, |d_s| <= 128,
// with one exponent e per row of the Legendre table and one per field-level
// column of the data.  Every digit is exact in BF16.  Every digit product is
// an integer of at most 2^14, so the sum over up to 128 latitudes (or degrees)
// and up to 7 digit pairs of one significance level stays below 2^24.  It is
// therefore exact in the FP32 accumulator of tcgen05.mma kind::f16.
// The pairs with s + t <= 6 are kept (28 MMAs per K step).  Each level lands
// in its own TMEM accumulator.  The levels are recombined in FP64 with the
// two exponents (the Ozaki error-free splitting, Ozaki-Ogita-Oishi-Rump,
// Numer. Algorithms 59 (2012)).  Each operand keeps 56 bits (the digit
// residual is below 2^-56 of its row or column maximum), and the dropped
// products are below 2^-62.
//
// Layout of one CTA (128 threads, one per real data column):
//   M = 128 data columns (64 complex field-levels), N = rows of one parity
//   (analysis) or Gauss rows (synthesis), K = 64 per chunk.  A (data digits)
//   and B (table digits) are K-major, in the interleaved canonical layout
//   (8-row x 16-byte core matrices, LBO = 128 B along K, SBO = 1024 B across
//   row groups).  D is FP32 in TMEM, lane = data column.  One thread issues
//   the MMAs and commits them to an mbarrier.  Waits are bounded: a timeout
//   sets the plan's device error word and the kernel unwinds (frees TMEM).
//
// The table digits are built once per plan on the device (k_slice_table_*).
// Follows space_discretization.tex:197-200 (analysis) and :212-216 (synthesis).
#include "sht_internal.h"
#include "sht_tc.cuh"

#include <cuda_bf16.h>
#include <vector>

namespace sht {

namespace {

constexpr int kS = 7;             // digits per operand
constexpr int kKC = 64;           // K per chunk (4 MMA K-steps of 16)
constexpr int kM = 128;           // data columns per CTA (64 complex)
constexpr int kTileBytesPerRow = kKC * 2;  // 128 B per row of one digit tile
constexpr uint64_t kWaitLimit = 2000000000ull;  // 2 s per bounded wait

// byte offset of element (row, k) inside a canonical K-major tile of 64 k
__host__ __device__ inline uint32_t canon(int row, int k)
{
  return (uint32_t)((row >> 3) * 1024 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void digits6(double x, float (&d)[kS])
{
  // x in (-1, 1): balanced digits, d0 in [-128,128], |r| <= 1/2 after each step,
  // so |x - sum_s d_s 2^{-7-8s}| <= 2^{-7-8 kS}
  double v = x * 128.0;
#pragma unroll
  for (int s = 0; s < kS; ++s) {
    const double q = rint(v);
    d[s] = (float)q;
    v = (v - q) * 256.0;
  }
}

struct SplitTables {
  // analysis operand B: per (m, p): rows = degrees of parity p, K = latitudes
  __nv_bfloat16 *fwd = nullptr;
  long long *fwd_off = nullptr;  // element offset per (m,p)
  int *fwd_exp = nullptr;        // exponent per row
  int *fwd_eoff = nullptr;       // row offset per (m,p) into fwd_exp
  int *fwd_npad = nullptr;       // padded rows per (m,p)
  // synthesis operand B: per (m, p): rows = latitudes, K = degrees of parity p
  __nv_bfloat16 *inv = nullptr;
  long long *inv_off = nullptr;
  int *inv_exp = nullptr;        // exponent per latitude, per (m,p): [m*2+p][JH]
  int *inv_kch = nullptr;        // K chunks per (m,p)
  int npad_max = 0;
  int *d_err = nullptr;          // device error word
  int fwd_kch = 0;               // K chunks of the analysis (latitudes)
};

__host__ __device__ inline int rows_of_parity(int N, int m, int p)
{
  const int R = N + 2 - m;
  return p ? R / 2 : (R + 1) / 2;
}
__host__ __device__ inline int round_up(int x, int r) { return (x + r - 1) / r * r; }

// one thread per (m, p, row i): digits of Pbar_{m+p+2i}^m over the latitudes
__global__ void k_slice_table_fwd(int N, int JH, const double *__restrict__ P, const long long *__restrict__ poff,
                                  __nv_bfloat16 *tab, const long long *__restrict__ off, int *exps,
                                  const int *__restrict__ eoff, const int *__restrict__ npad, int kch)
{
  const int mp = blockIdx.y, m = mp >> 1, p = mp & 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > N || i >= rows_of_parity(N, m, p)) return;
  const double *row = P + poff[m] + (long long)(p + 2 * i) * JH;
  double mx = 0.0;
  for (int k = 0; k < JH; ++k) mx = fmax(mx, fabs(row[k]));
  int e = 0;
  frexp(mx, &e);
  exps[eoff[mp] + i] = e;
  const int np = npad[mp];
  for (int k = 0; k < JH; ++k) {
    float d[kS];
    digits6(ldexp(row[k], -e), d);
    const int kc = k / kKC, kk = k % kKC;
#pragma unroll
    for (int s = 0; s < kS; ++s) {
      char *tile = reinterpret_cast<char *>(tab + off[mp]) + ((size_t)(kc * kS + s) * np) * kTileBytesPerRow;
      *reinterpret_cast<__nv_bfloat16 *>(tile + canon(i, kk)) = __float2bfloat16_rn(d[s]);
    }
  }
  (void)kch;
}

// one thread per (m, p, latitude jh): digits of Pbar_{m+p+2i}^m over the degrees i
__global__ void k_slice_table_inv(int N, int JH, const double *__restrict__ P, const long long *__restrict__ poff,
                                  __nv_bfloat16 *tab, const long long *__restrict__ off, int *exps, int npad_rows)
{
  const int mp = blockIdx.y, m = mp >> 1, p = mp & 1;
  const int jh = blockIdx.x * blockDim.x + threadIdx.x;
  if (m > N || jh >= JH) return;
  const int Rp = rows_of_parity(N, m, p);
  const double *base = P + poff[m] + jh;
  double mx = 0.0;
  for (int i = 0; i < Rp; ++i) mx = fmax(mx, fabs(base[(long long)(p + 2 * i) * JH]));
  int e = 0;
  frexp(mx, &e);
  exps[mp * JH + jh] = e;
  for (int i = 0; i < Rp; ++i) {
    float d[kS];
    digits6(ldexp(base[(long long)(p + 2 * i) * JH], -e), d);
    const int kc = i / kKC, kk = i % kKC;
#pragma unroll
    for (int s = 0; s < kS; ++s) {
      char *tile = reinterpret_cast<char *>(tab + off[mp]) + ((size_t)(kc * kS + s) * npad_rows) * kTileBytesPerRow;
      *reinterpret_cast<__nv_bfloat16 *>(tile + canon(jh, kk)) = __float2bfloat16_rn(d[s]);
    }
  }
}

struct TcArgs {
  const double2 *F;   // analysis input F[m][col][j]
  double2 *S;         // analysis output
  const double2 *Sc;  // synthesis input
  double2 *Fo;        // synthesis output
  const int *rowoff;
  const __nv_bfloat16 *tab;
  const long long *toff;
  const int *texp;
  const int *teoff;   // analysis: row-exponent offsets
  const int *tnpad;   // analysis: padded rows
  int N, J, JH, ncol, fwd_kch;
  int *err;
};

// Issue the 21 digit-pair MMAs of one K chunk into D_L = tbase + L*ncols_per_level.
__device__ __forceinline__ void issue_chunk(uint32_t tbase, int dstride, uint32_t a_base, uint32_t b_base,
                                            int npad, bool first_chunk)
{
  const uint32_t idesc = tc::idesc_bf16_f32(kM, npad);
  const uint32_t a_tile = kM * kTileBytesPerRow;   // bytes per digit tile of A
  const uint32_t b_tile = npad * kTileBytesPerRow; // bytes per digit tile of B
#pragma unroll
  for (int L = 0; L < kS; ++L) {
#pragma unroll
    for (int s = 0; s <= L; ++s) {
      const int t = L - s;
#pragma unroll
      for (int ks = 0; ks < kKC / 16; ++ks) {
        const uint64_t ad = tc::smem_desc(a_base + s * a_tile + ks * 256, 128, 1024);
        const uint64_t bd = tc::smem_desc(b_base + t * b_tile + ks * 256, 128, 1024);
        const uint32_t acc = (first_chunk && s == 0 && ks == 0) ? 0u : 1u;
        tc::mma_bf16(tbase + (uint32_t)(L * dstride), ad, bd, idesc, acc);
      }
    }
  }
}

// ------------------------------------------------------------------ analysis
template <int NPAD>
__global__ void __launch_bounds__(128, 1) k_leg_fwd_split(TcArgs a)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  unsigned char *Asm = smem;                              // kS x 128 x 64 bf16 = 96 KB
  unsigned char *Bsm = smem + kS * kM * kTileBytesPerRow; // kS x NPAD x 64 bf16
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m = blockIdx.y, col0 = blockIdx.x * (kM / 2);
  const int b = col0 + (tid >> 1), part = tid & 1;
  const bool valid = b < a.ncol;
  const int JH = a.JH;

  if (warp == 0) {
    tc::tmem_alloc(&tslot, 512);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(&mbar, 1);
    tc::mbar_fence_init();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tbase = tslot;
  uint32_t phase = 0;
  bool ok = true;

  // column exponents of the symmetric and antisymmetric halves
  const double *col = reinterpret_cast<const double *>(a.F + ((long long)m * a.ncol + (valid ? b : 0)) * a.J) + part;
  double mxs = 0.0, mxa = 0.0;
  if (valid)
    for (int jh = 0; jh < JH; ++jh) {
      const double gn = col[2 * (JH + jh)], gs = col[2 * (JH - 1 - jh)];
      mxs = fmax(mxs, fabs(gn + gs));
      mxa = fmax(mxa, fabs(gn - gs));
    }
  int es = 0, ea = 0;
  frexp(mxs, &es);
  frexp(mxa, &ea);

  for (int p = 0; p < 2 && ok; ++p) {
    const int mp = m * 2 + p;
    const int Rp = rows_of_parity(a.N, m, p);
    const int np = a.tnpad[mp];
    const int e = p ? ea : es;
    const char *tab = reinterpret_cast<const char *>(a.tab + a.toff[mp]);
    for (int kc = 0; kc < a.fwd_kch && ok; ++kc) {
      // data digits of this thread's column into A (row = tid)
      for (int kk = 0; kk < kKC; kk += 8) {
        uint4 pk[kS];
        unsigned short *pkh = reinterpret_cast<unsigned short *>(pk);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int jh = kc * kKC + kk + q;
          float d[kS];
          double x = 0.0;
          if (valid && jh < JH) {
            const double gn = col[2 * (JH + jh)], gs = col[2 * (JH - 1 - jh)];
            x = ldexp(p ? gn - gs : gn + gs, -e);
          }
          digits6(x, d);
#pragma unroll
          for (int s = 0; s < kS; ++s) pkh[s * 8 + q] = __bfloat16_as_ushort(__float2bfloat16_rn(d[s]));
        }
#pragma unroll
        for (int s = 0; s < kS; ++s)
          *reinterpret_cast<uint4 *>(Asm + s * kM * kTileBytesPerRow + canon(tid, kk)) = pk[s];
      }
      // table digits for (m, p, chunk): kS tiles of np rows, contiguous
      {
        const uint4 *src = reinterpret_cast<const uint4 *>(tab + (size_t)kc * kS * np * kTileBytesPerRow);
        uint4 *dst = reinterpret_cast<uint4 *>(Bsm);
        const int n16 = kS * np * kTileBytesPerRow / 16;
        for (int q = tid; q < n16; q += 128) dst[q] = src[q];
      }
      tc::fence_proxy_async();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after();
        issue_chunk(tbase, NPAD, tc::smem_addr(Asm), tc::smem_addr(Bsm), np, kc == 0);
        tc::mma_commit(&mbar);
      }
      __syncwarp();
      bool done = tc::mbar_wait(&mbar, phase, kWaitLimit);
      if (!done && (tid & 31) == 0) atomicExch(a.err, SHT_ERR_DEVICE_TIMEOUT);
      ok = __syncthreads_and(done) != 0;  // every thread takes the same path
      if (ok) phase ^= 1;
      tc::fence_after();
    }
    if (!ok) break;
    // read the levels back: lane = this thread's column, columns = degrees of parity p
    double acc[NPAD];
#pragma unroll
    for (int n = 0; n < NPAD; ++n) acc[n] = 0.0;
    const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int L = kS - 1; L >= 0; --L) {
#pragma unroll
      for (int q = 0; q < NPAD / 16; ++q) {
        uint32_t r[16];
        tc::tmem_ld16(lane_base + (uint32_t)(L * NPAD + 16 * q), r);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[16 * q + i] = acc[16 * q + i] * (1.0 / 256.0) + (double)__uint_as_float(r[i]);
      }
    }
    // acc = sum_L 2^{-8L} D_L; value = acc * 2^(e + f_n - 14)
    if (valid) {
      const int *fe = a.texp + a.teoff[mp];
      const long long rowbase = a.rowoff[m];
#pragma unroll
      for (int n = 0; n < NPAD; ++n) {
        if (n < Rp) {
          const double v = ldexp(acc[n], e + fe[n] - 14);
          reinterpret_cast<double *>(a.S + (rowbase + p + 2 * n) * a.ncol + b)[part] = v;
        }
      }
    }
    tc::fence_before();  // TMEM reads above precede the next parity's MMAs
    __syncthreads();
  }
  if (!ok) tc::mbar_wait(&mbar, phase, kWaitLimit);  // give in-flight MMAs a bounded chance to drain
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 512);
}

// ----------------------------------------------------------------- synthesis
template <int JHT>
__global__ void __launch_bounds__(128, 1) k_leg_inv_split(TcArgs a)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint64_t mbar;
  __shared__ uint32_t tslot;
  unsigned char *Asm = smem;                               // kS x 128 x 64 bf16
  unsigned char *Bsm = smem + kS * kM * kTileBytesPerRow;  // kS x JHT x 64 bf16
  const int tid = threadIdx.x, warp = tid >> 5;
  const int m = blockIdx.y, col0 = blockIdx.x * (kM / 2);
  const int b = col0 + (tid >> 1), part = tid & 1;
  const bool valid = b < a.ncol;
  const int JH = a.JH;

  if (warp == 0) {
    tc::tmem_alloc(&tslot, 512);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(&mbar, 1);
    tc::mbar_fence_init();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tbase = tslot;
  uint32_t phase = 0;
  bool ok = true;
  const long long rowbase = a.rowoff[m];

  for (int p = 0; p < 2 && ok; ++p) {
    const int mp = m * 2 + p;
    const int Rp = rows_of_parity(a.N, m, p);
    const int kch = (Rp + kKC - 1) / kKC;
    // coefficient exponent of this column over the degrees of parity p
    const double *cf = reinterpret_cast<const double *>(a.Sc + rowbase * a.ncol + (valid ? b : 0)) + part;
    double mx = 0.0;
    if (valid)
      for (int i = 0; i < Rp; ++i) mx = fmax(mx, fabs(cf[2 * (long long)(p + 2 * i) * a.ncol]));
    int e = 0;
    frexp(mx, &e);
    const char *tab = reinterpret_cast<const char *>(a.tab + a.toff[mp]);
    for (int kc = 0; kc < kch && ok; ++kc) {
      for (int kk = 0; kk < kKC; kk += 8) {
        uint4 pk[kS];
        unsigned short *pkh = reinterpret_cast<unsigned short *>(pk);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int i = kc * kKC + kk + q;
          float d[kS];
          double x = 0.0;
          if (valid && i < Rp) x = ldexp(cf[2 * (long long)(p + 2 * i) * a.ncol], -e);
          digits6(x, d);
#pragma unroll
          for (int s = 0; s < kS; ++s) pkh[s * 8 + q] = __bfloat16_as_ushort(__float2bfloat16_rn(d[s]));
        }
#pragma unroll
        for (int s = 0; s < kS; ++s)
          *reinterpret_cast<uint4 *>(Asm + s * kM * kTileBytesPerRow + canon(tid, kk)) = pk[s];
      }
      {
        const uint4 *src = reinterpret_cast<const uint4 *>(tab + (size_t)kc * kS * JHT * kTileBytesPerRow);
        uint4 *dst = reinterpret_cast<uint4 *>(Bsm);
        const int n16 = kS * JHT * kTileBytesPerRow / 16;
        for (int q = tid; q < n16; q += 128) dst[q] = src[q];
      }
      tc::fence_proxy_async();
      __syncthreads();
      if (tid == 0) {
        tc::fence_after();
        issue_chunk(tbase, JHT, tc::smem_addr(Asm), tc::smem_addr(Bsm), JHT, kc == 0);
        tc::mma_commit(&mbar);
      }
      __syncwarp();
      bool done = tc::mbar_wait(&mbar, phase, kWaitLimit);
      if (!done && (tid & 31) == 0) atomicExch(a.err, SHT_ERR_DEVICE_TIMEOUT);
      ok = __syncthreads_and(done) != 0;  // every thread takes the same path
      if (ok) phase ^= 1;
      tc::fence_after();
    }
    if (!ok) break;
    double acc[JHT];
#pragma unroll
    for (int n = 0; n < JHT; ++n) acc[n] = 0.0;
    const uint32_t lane_base = tbase + ((uint32_t)(warp * 32) << 16);
#pragma unroll
    for (int L = kS - 1; L >= 0; --L) {
#pragma unroll
      for (int q = 0; q < JHT / 16; ++q) {
        uint32_t r[16];
        tc::tmem_ld16(lane_base + (uint32_t)(L * JHT + 16 * q), r);
        tc::tmem_wait_ld();
#pragma unroll
        for (int i = 0; i < 16; ++i) acc[16 * q + i] = acc[16 * q + i] * (1.0 / 256.0) + (double)__uint_as_float(r[i]);
      }
    }
    // The even half Ge is parked in this thread's northern output slots and
    // combined with the odd half Go on the second pass (same thread, same addresses).
    const int *ge = a.texp + mp * JH;
    if (valid) {
      double *Fc = reinterpret_cast<double *>(a.Fo + ((long long)m * a.ncol + b) * a.J) + part;
      if (p == 0) {
#pragma unroll
        for (int jh = 0; jh < JHT; ++jh)
          if (jh < JH) Fc[2 * (JH + jh)] = ldexp(acc[jh], e + ge[jh] - 14);
      } else {
#pragma unroll
        for (int jh = 0; jh < JHT; ++jh) {
          if (jh < JH) {
            const double go = ldexp(acc[jh], e + ge[jh] - 14), gev = Fc[2 * (JH + jh)];
            Fc[2 * (JH + jh)] = gev + go;
            Fc[2 * (JH - 1 - jh)] = gev - go;
          }
        }
      }
    }
    tc::fence_before();  // TMEM reads above precede the next parity's MMAs
    __syncthreads();
  }
  if (!ok) tc::mbar_wait(&mbar, phase, kWaitLimit);  // give in-flight MMAs a bounded chance to drain
  tc::fence_before();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(tbase, 512);
}

SplitTables *tables(sht_plan *p) { return static_cast<SplitTables *>(p->tc_tables); }

int build_split_tables(sht_plan *p)
{
  if (p->tc_tables) return SHT_OK;
  const int N = p->N, JH = p->JH;
  auto *t = new SplitTables();
  // analysis table sizes
  std::vector<long long> foff(2 * (N + 1)), ioff(2 * (N + 1));
  std::vector<int> feoff(2 * (N + 1)), fnpad(2 * (N + 1));
  const int fkch = (JH + kKC - 1) / kKC;
  long long fsz = 0, isz = 0;
  int erows = 0, npmax = 0;
  const int inpad = round_up(JH, 16);
  for (int m = 0; m <= N; ++m)
    for (int pp = 0; pp < 2; ++pp) {
      const int mp = 2 * m + pp, Rp = rows_of_parity(N, m, pp);
      const int np = round_up(Rp > 0 ? Rp : 1, 16);
      fnpad[mp] = np;
      npmax = np > npmax ? np : npmax;
      foff[mp] = fsz;
      fsz += (long long)fkch * kS * np * kKC;
      feoff[mp] = erows;
      erows += Rp;
      ioff[mp] = isz;
      isz += (long long)((Rp + kKC - 1) / kKC) * kS * inpad * kKC;
    }
  t->npad_max = npmax;
  t->fwd_kch = fkch;
  cudaError_t e;
  auto fail = [&](cudaError_t err, const char *what) {
    cudaFree(t->fwd); cudaFree(t->fwd_off); cudaFree(t->fwd_exp); cudaFree(t->fwd_eoff); cudaFree(t->fwd_npad);
    cudaFree(t->inv); cudaFree(t->inv_off); cudaFree(t->inv_exp); cudaFree(t->d_err);
    delete t;
    return cuda_fail(err, what);
  };
  if ((e = cudaMalloc(&t->fwd, sizeof(__nv_bfloat16) * (size_t)fsz)) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->inv, sizeof(__nv_bfloat16) * (size_t)isz)) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->fwd_off, sizeof(long long) * foff.size())) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->inv_off, sizeof(long long) * ioff.size())) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->fwd_eoff, sizeof(int) * feoff.size())) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->fwd_npad, sizeof(int) * fnpad.size())) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->fwd_exp, sizeof(int) * (erows > 0 ? erows : 1))) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->inv_exp, sizeof(int) * 2 * (N + 1) * JH)) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->d_err, sizeof(int))) != cudaSuccess) return fail(e, "split table");
  cudaStream_t s = p->stream;
  if ((e = cudaMemsetAsync(t->fwd, 0, sizeof(__nv_bfloat16) * (size_t)fsz, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(t->inv, 0, sizeof(__nv_bfloat16) * (size_t)isz, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(t->d_err, 0, sizeof(int), s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(t->fwd_off, foff.data(), sizeof(long long) * foff.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(t->inv_off, ioff.data(), sizeof(long long) * ioff.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(t->fwd_eoff, feoff.data(), sizeof(int) * feoff.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(t->fwd_npad, fnpad.data(), sizeof(int) * fnpad.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return fail(e, "split table upload");
  const int maxrows = (N + 3) / 2;
  dim3 gf((maxrows + 127) / 128, 2 * (N + 1));
  k_slice_table_fwd<<<gf, 128, 0, s>>>(N, JH, p->d_P, p->d_poff, t->fwd, t->fwd_off, t->fwd_exp, t->fwd_eoff, t->fwd_npad, fkch);
  count_launch();
  dim3 gi((JH + 127) / 128, 2 * (N + 1));
  k_slice_table_inv<<<gi, 128, 0, s>>>(N, JH, p->d_P, p->d_poff, t->inv, t->inv_off, t->inv_exp, inpad);
  count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "split table build");
  p->tc_tables = t;
  return SHT_OK;
}

size_t fwd_smem(int npad) { return (size_t)kS * kM * kTileBytesPerRow + (size_t)kS * npad * kTileBytesPerRow; }
size_t inv_smem(int jht) { return (size_t)kS * kM * kTileBytesPerRow + (size_t)kS * jht * kTileBytesPerRow; }

template <typename K>
int launch_tc(K kern, dim3 grid, size_t smem, cudaStream_t s, const TcArgs &a, const char *name)
{
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return cuda_fail(e, name);
  kern<<<grid, 128, smem, s>>>(a);
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, name);
}

}  // namespace

bool split_supported(const sht_plan *p)
{
  // TMEM holds the kS levels of one parity: kS * NPAD <= 512 columns.
  const int npmax = round_up((p->N + 3) / 2, 16);
  return p->JH <= kKC && (p->JH % 16) == 0 && npmax * kS <= 512 && p->JH * kS <= 512;
}

int launch_leg_fwd_split(sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  if (!split_supported(p)) {
    set_error("split precision: this grid is not covered by the tensor-core kernel (needs jm <= 128 with jm/2 a multiple of 16, nm <= 125)");
    return SHT_ERR_UNSUPPORTED_SIZE;
  }
  int rc = build_split_tables(p);
  if (rc) return rc;
  SplitTables *t = tables(p);
  TcArgs a{};
  a.F = F; a.S = S; a.rowoff = p->d_rowoff; a.tab = t->fwd; a.toff = t->fwd_off; a.texp = t->fwd_exp;
  a.teoff = t->fwd_eoff; a.tnpad = t->fwd_npad; a.N = p->N; a.J = p->J; a.JH = p->JH; a.ncol = ncol;
  a.fwd_kch = t->fwd_kch; a.err = t->d_err;
  dim3 grid((ncol + kM / 2 - 1) / (kM / 2), p->N + 1);
  const int np = t->npad_max;
  switch (np) {
  case 16: return launch_tc(k_leg_fwd_split<16>, grid, fwd_smem(16), s, a, "k_leg_fwd_split");
  case 32: return launch_tc(k_leg_fwd_split<32>, grid, fwd_smem(32), s, a, "k_leg_fwd_split");
  case 48: return launch_tc(k_leg_fwd_split<48>, grid, fwd_smem(48), s, a, "k_leg_fwd_split");
  case 64: return launch_tc(k_leg_fwd_split<64>, grid, fwd_smem(64), s, a, "k_leg_fwd_split");
  default: set_error("split precision: unsupported row count"); return SHT_ERR_UNSUPPORTED_SIZE;
  }
}

int launch_leg_inv_split(sht_plan *p, const double2 *Sp, int ncol, double2 *F, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  if (!split_supported(p)) {
    set_error("split precision: this grid is not covered by the tensor-core kernel (needs jm <= 128 with jm/2 a multiple of 16, nm <= 125)");
    return SHT_ERR_UNSUPPORTED_SIZE;
  }
  int rc = build_split_tables(p);
  if (rc) return rc;
  SplitTables *t = tables(p);
  TcArgs a{};
  a.Sc = Sp; a.Fo = F; a.rowoff = p->d_rowoff; a.tab = t->inv; a.toff = t->inv_off; a.texp = t->inv_exp;
  a.N = p->N; a.J = p->J; a.JH = p->JH; a.ncol = ncol; a.err = t->d_err;
  dim3 grid((ncol + kM / 2 - 1) / (kM / 2), p->N + 1);
  switch (p->JH) {
  case 16: return launch_tc(k_leg_inv_split<16>, grid, inv_smem(16), s, a, "k_leg_inv_split");
  case 32: return launch_tc(k_leg_inv_split<32>, grid, inv_smem(32), s, a, "k_leg_inv_split");
  case 48: return launch_tc(k_leg_inv_split<48>, grid, inv_smem(48), s, a, "k_leg_inv_split");
  case 64: return launch_tc(k_leg_inv_split<64>, grid, inv_smem(64), s, a, "k_leg_inv_split");
  default: set_error("split precision: unsupported latitude count"); return SHT_ERR_UNSUPPORTED_SIZE;
  }
}

int split_error_status(sht_plan *p)
{
  SplitTables *t = tables(p);
  if (!t) return SHT_OK;
  int h = 0;
  cudaError_t e = cudaMemcpy(&h, t->d_err, sizeof(int), cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return cuda_fail(e, "split error word");
  if (h) {
    cudaMemset(t->d_err, 0, sizeof(int));
    set_error("split precision: a bounded tensor-core wait timed out");
    return h;
  }
  return SHT_OK;
}

void free_split_tables(sht_plan *p)
{
  SplitTables *t = tables(p);
  if (!t) return;
  cudaFree(t->fwd); cudaFree(t->fwd_off); cudaFree(t->fwd_exp); cudaFree(t->fwd_eoff); cudaFree(t->fwd_npad);
  cudaFree(t->inv); cudaFree(t->inv_off); cudaFree(t->inv_exp); cudaFree(t->d_err);
  delete t;
  p->tc_tables = nullptr;
}

}  // namespace sht
