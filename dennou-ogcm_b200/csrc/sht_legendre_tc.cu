// sht_legendre_tc.cu -- split-precision Legendre contraction on tcgen05.
//
// Both FP64 operands of c_n = sum_jh P_n(mu_jh) G(mu_jh) are written as
// power-of-two scaled fixed-point numbers in balanced base-256 digits:
//     x = 2^{e-7} * sum_{s=0..6} d_s 2^{-8s},   d_s integers, |d_s| <= 128,
// with one exponent e per row of the Legendre table and one per field-level
// column of the data.  Digit s is stored as the BF16 value d_s 2^{-8s}
// (exact: 8 significant bits and a power-of-two scale), so the product of
// digits s and t carries its weight 2^{-8(s+t)} by itself.  The pairs with
// s + t <= 6 are kept (28 MMAs per K step).  Pairs of level L = s + t < 5 go
// to accumulator L: every such product is an integer multiple of 2^{-8L} of
// magnitude at most 2^{14-8L}, so the FP32 sum over K <= 256 of the L + 1
// pairs of levels 0..3 stays an exact multiple of at most 2^{24-8L} -- exact;
// level 4 is exact for K <= 204 and beyond that rounds only where its partial
// sums pass 4/5 of their bound.  Levels 5 and 6 share a sixth accumulator.
// Each MMA's sum is rounded into the FP32 accumulator, and nothing is assumed
// about the direction, so the error of a shared accumulator is bounded by the
// number of MMAs into it times the ulp of its largest level: levels 4..6 in one
// accumulator reached 1.3e-11 of a field's maximum at T341 (K = 172..256,
// 288 roundings at 2^{-45} of the result's scale), levels 3..6 reached 3e-11
// at T42; from level 5 on it is 2^{-52} per rounding.  The six accumulators
// are summed in FP64 (smallest first) and scaled by the two exponents (the Ozaki error-free
// splitting, Ozaki-Ogita-Oishi-Rump, Numer. Algorithms 59 (2012)).  Each
// operand keeps 56 bits (the digit residual is below 2^-56 of its row or column
// maximum), and the dropped products are below 2^-62.
//
// Kernel organisation (one resident CTA of 256 threads per SM):
//   * Work item = (band pair (m, N-m), 64 complex field-level columns).  The
//     pair keeps every item about the same cost.  An item has up to four
//     sub-items (m, parity); the output dimension of a sub-item (degrees in
//     the analysis, Gauss rows in the synthesis) is cut into segments of at
//     most kSeg columns, and each segment runs its K chunks of 32.
//   * The data digits of chunk u+1 (and its table digits) are written into
//     the other of two shared-memory stages while the tensor core runs the
//     asynchronous MMAs of chunk u, issued by one thread.
//   * When a segment's last chunk completes, all threads read its six TMEM
//     accumulators, 16 columns at a time (the two warp halves take alternate
//     groups), and recombine them in FP64.
//   * M = 128 data columns (re/im of 64 field-levels; TMEM lane = column).
//     A and B are K-major in the interleaved canonical layout (8-row x
//     16-byte core matrices, LBO = 128 B along K, SBO = 512 B across row
//     groups).
//   * Every wait is bounded in time.  A timeout sets the plan's device error
//     word, and the kernel unwinds and frees its TMEM.
// The table digits are built once per plan on the device (k_slice_table_*).
// Follows space_discretization.tex:197-200 (analysis) and :212-216 (synthesis).
#include "sht_internal.h"
#include "sht_tc.cuh"

#include <cuda_bf16.h>
#include <vector>

namespace sht {

namespace {

constexpr int kS = 7;                      // digits per operand
constexpr int kAcc = 6;                    // TMEM accumulators: levels 0, 1, 2, 3, 4 and 5..6
constexpr int kSeg = 80;                   // analysis: output columns per segment (kAcc x kSeg <= 512 TMEM columns)
constexpr int kSegInv = 64;                // synthesis with output staging: Gauss rows per segment
constexpr int kStg = 2 * 16 + 2;           // doubles per field-level row of the synthesis output staging
constexpr int kKC = 32;                    // K per chunk (2 MMA K-steps of 16)
constexpr int kM = 128;                    // data columns per CTA (64 complex)
constexpr int kRowB = kKC * 2;             // 64 bytes per row of one digit tile
constexpr int kThreads = 256;
constexpr uint64_t kWaitLimit = 2000000000ull;  // 2 s per bounded wait

// byte offset of element (row, k) inside a canonical K-major tile of 32 k
__host__ __device__ inline uint32_t canon(int row, int k)
{
  return (uint32_t)((row >> 3) * 512 + (k >> 3) * 128 + (row & 7) * 16 + (k & 7) * 2);
}

__device__ __forceinline__ void digits(double x, float (&d)[kS])
{
  // x in (-1, 1): balanced digits, d0 in [-128,128], |r| <= 1/2 after each step,
  // so |x - 2^-7 sum_s d_s 2^{-8s}| <= 2^{-7-8 kS}; digit s is returned as d_s 2^{-8s}
  double v = x * 128.0;
#pragma unroll
  for (int s = 0; s < kS; ++s) {
    const double q = rint(v);
    d[s] = ldexpf((float)q, -8 * s);
    v = (v - q) * 256.0;
  }
}

// The same scaled digits as BF16 bit patterns without conversion
// instructions: adding 1.5*2^52 rounds |v| < 2^51 to the nearest integer,
// which lands in the low word; an integer d with |d| <= 128 becomes an exact
// FP32 value through 1.5*2^23 + d, the scale 2^{-8s} is an exact multiply, and
// the top 16 bits of the FP32 value are its BF16 encoding.
__device__ __forceinline__ void digits_bf16(double x, unsigned short (&h)[kS])
{
  const double M52 = 6755399441055744.0;  // 1.5 * 2^52
  double v = x * 128.0;
  float scale = 1.0f;
#pragma unroll
  for (int s = 0; s < kS; ++s) {
    const double t = v + M52;
    const int di = __double2loint(t);
    const double q = t - M52;
    v = (v - q) * 256.0;
    const float f = (__int_as_float(0x4B400000 + di) - 12582912.0f) * scale;
    h[s] = (unsigned short)(__float_as_uint(f) >> 16);
    scale *= (1.0f / 256.0f);
  }
}

__host__ __device__ inline int rows_of_parity(int N, int m, int p)
{
  const int R = N + 2 - m;
  return p ? R / 2 : (R + 1) / 2;
}
__host__ __device__ inline int round_up(int x, int r) { return (x + r - 1) / r * r; }

struct SplitTables {
  // analysis operand B per (m, p): rows = degrees of parity p, K = latitudes
  __nv_bfloat16 *fwd = nullptr;
  long long *fwd_off = nullptr;  // element offset per (m,p)
  int *fwd_exp = nullptr;        // exponent per row
  int *fwd_eoff = nullptr;       // row offset per (m,p) into fwd_exp
  int fwd_npad_max = 0;
  // synthesis operand B per (m, p): rows = latitudes, K = degrees of parity p
  __nv_bfloat16 *inv = nullptr;
  long long *inv_off = nullptr;
  int *inv_exp = nullptr;        // exponent per latitude: [m*2+p][JH]
  int inv_npad = 0;
  int *d_err = nullptr;          // device error word
};

// one thread per (m, p, row i): digits of Pbar_{m+p+2i}^m over the latitudes
__global__ void k_slice_table_fwd(int N, int JH, const double *__restrict__ P, const long long *__restrict__ poff,
                                  __nv_bfloat16 *tab, const long long *__restrict__ off, int *exps,
                                  const int *__restrict__ eoff)
{
  const int mp = blockIdx.y, m = mp >> 1, p = mp & 1;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int Rp = rows_of_parity(N, m, p);
  if (m > N || i >= Rp) return;
  const int np = round_up(Rp, 16);
  const double *row = P + poff[m] + (long long)(p + 2 * i) * JH;
  double mx = 0.0;
  for (int k = 0; k < JH; ++k) mx = fmax(mx, fabs(row[k]));
  int e = 0;
  frexp(mx, &e);
  exps[eoff[mp] + i] = e;
  for (int k = 0; k < JH; ++k) {
    float d[kS];
    digits(ldexp(row[k], -e), d);
    const int h = k / kKC, kk = k % kKC;
#pragma unroll
    for (int s = 0; s < kS; ++s) {
      char *tile = reinterpret_cast<char *>(tab + off[mp]) + ((size_t)(h * kS + s) * np) * kRowB;
      *reinterpret_cast<__nv_bfloat16 *>(tile + canon(i, kk)) = __float2bfloat16_rn(d[s]);
    }
  }
}

// one thread per (m, p, latitude jh): digits of Pbar_{m+p+2i}^m over the degrees i
__global__ void k_slice_table_inv(int N, int JH, const double *__restrict__ P, const long long *__restrict__ poff,
                                  __nv_bfloat16 *tab, const long long *__restrict__ off, int *exps, int np)
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
    digits(ldexp(base[(long long)(p + 2 * i) * JH], -e), d);
    const int h = i / kKC, kk = i % kKC;
#pragma unroll
    for (int s = 0; s < kS; ++s) {
      char *tile = reinterpret_cast<char *>(tab + off[mp]) + ((size_t)(h * kS + s) * np) * kRowB;
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
  const int2 *pairs;
  const __nv_bfloat16 *tab;
  const long long *toff;
  const int *texp;
  const int *teoff;   // analysis: row-exponent offsets
  int N, J, JH, ncol;
  int ntiles, nitems, per_cta;
  int npad_max;       // TMEM columns per accumulator (largest segment)
  int npad_max_table; // rows of one synthesis digit tile (latitudes, padded)
  int seg_inv;        // synthesis segment (kSegInv with staged output, else kSeg)
  int *err;
};

// Segment bookkeeping shared by both directions: sub-item (m, parity p) and
// the segment [row0, row0 + npad) of its output dimension.
struct Sub {
  int m, p, Rp, nrow, seg, nseg, row0, npad, nch, slot;
};

template <bool INV>
__device__ __forceinline__ Sub make_sub(const TcArgs &a, int m, int p, int seg, int q)
{
  Sub s;
  s.m = m;
  s.p = p;
  s.Rp = rows_of_parity(a.N, m, p);
  s.nrow = INV ? a.JH : s.Rp;  // output rows of the sub-item
  const int cap = INV ? a.seg_inv : kSeg;
  s.nseg = (s.nrow + cap - 1) / cap;
  s.seg = seg;
  s.row0 = seg * cap;
  s.npad = round_up(min(cap, s.nrow - s.row0), 16);
  s.nch = INV ? (s.Rp + kKC - 1) / kKC : (a.JH + kKC - 1) / kKC;
  s.slot = q & 3;
  return s;
}

// Unit iterator: (item, sub-item, segment, chunk) in order, uniform across the CTA.
struct Cursor {
  int it, sub, seg, h, q;  // item, sub-item within the item, segment, chunk, running sub-item count
};

template <bool INV>
__device__ __forceinline__ void cursor_sub(const TcArgs &a, const Cursor &c, Sub &out)
{
  const int2 pr = a.pairs[c.it / a.ntiles];
  const int m = (c.sub < 2) ? pr.x : pr.y;
  out = make_sub<INV>(a, m, c.sub & 1, c.seg, c.q);
}

template <bool INV>
__device__ __forceinline__ void cursor_next(const TcArgs &a, Cursor &c)
{
  Sub s;
  cursor_sub<INV>(a, c, s);
  if (++c.h < s.nch) return;
  c.h = 0;
  if (++c.seg < s.nseg) return;
  c.seg = 0;
  ++c.q;
  const int2 pr = a.pairs[c.it / a.ntiles];
  const int nsub = (pr.y >= 0) ? 4 : 2;
  if (++c.sub < nsub) return;
  c.sub = 0;
  ++c.it;
}

// Issue the 28 digit-pair MMAs of one K chunk; level L = s + t goes to
// accumulator min(L, kAcc - 1) at tbase + acc*dstride.  The first product into each
// accumulator in the segment's first chunk overwrites it.
__device__ __forceinline__ void issue_chunk(uint32_t tbase, int dstride, uint32_t a_base, uint32_t b_base, int npad,
                                            bool first_chunk)
{
  const uint32_t idesc = tc::idesc_bf16_f32(kM, npad);
  const uint32_t a_tile = kM * kRowB;    // bytes per digit tile of A
  const uint32_t b_tile = npad * kRowB;  // bytes per digit tile of B
#pragma unroll
  for (int L = 0; L < kS; ++L) {
    const int d = L < kAcc - 1 ? L : kAcc - 1;
#pragma unroll
    for (int s = 0; s <= L; ++s) {
      const int t = L - s;
#pragma unroll
      for (int ks = 0; ks < kKC / 16; ++ks) {
        const uint64_t ad = tc::smem_desc(a_base + s * a_tile + ks * 256, 128, 512);
        const uint64_t bd = tc::smem_desc(b_base + t * b_tile + ks * 256, 128, 512);
        const uint32_t acc = (first_chunk && s == 0 && ks == 0 && L == d) ? 0u : 1u;
        tc::mma_bf16(tbase + (uint32_t)(d * dstride), ad, bd, idesc, acc);
      }
    }
  }
}

struct Smem {
  unsigned char *A[2];
  unsigned char *B[2];
  int *exps;      // [4 slots][128 columns]
  double *part;   // [2][2][128] partial maxima
  double *stage;  // synthesis: [2 halves][64 field-levels][kStg] output staging
};

// Column exponents of the sub-items that start at this chunk.
template <bool INV>
__device__ void column_exponents(const TcArgs &a, const Sub &s, int col0, const Smem &sm)
{
  const int tid = threadIdx.x, c = tid & 127, half = tid >> 7;
  const int b = col0 + (c >> 1), part = c & 1;
  const bool valid = b < a.ncol;
  double m0 = 0.0, m1 = 0.0;
  // loads are issued 8 at a time so that they are in flight together
  if (!INV) {
    // Gs (parity 0) at jh and Ga (parity 1) at JH + jh, over all half-latitudes
    // (done at the first chunk of (m, 0))
    const double *col = reinterpret_cast<const double *>(a.F + ((long long)s.m * a.ncol + (valid ? b : 0)) * a.J) + part;
    const int JH = a.JH, hh = (JH + 1) / 2;
    const int j0 = half * hh, j1 = min(JH, (half + 1) * hh);
    if (valid)
      for (int jb = j0; jb < j1; jb += 8) {
        double gs[8], ga[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const int jh = min(jb + q, j1 - 1);
          gs[q] = col[2 * jh];
          ga[q] = col[2 * (JH + jh)];
        }
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          m0 = fmax(m0, fabs(gs[q]));
          m1 = fmax(m1, fabs(ga[q]));
        }
      }
  } else {
    const double *cf = reinterpret_cast<const double *>(a.Sc + (long long)a.rowoff[s.m] * a.ncol + (valid ? b : 0)) + part;
    const int hh = (s.Rp + 1) / 2;
    const int i0 = half * hh, i1 = min(s.Rp, (half + 1) * hh);
    if (valid)
      for (int ib = i0; ib < i1; ib += 8) {
        double v[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) v[q] = cf[2 * (long long)(s.p + 2 * min(ib + q, i1 - 1)) * a.ncol];
#pragma unroll
        for (int q = 0; q < 8; ++q) m0 = fmax(m0, fabs(v[q]));
      }
  }
  sm.part[(0 * 2 + half) * 128 + c] = m0;
  sm.part[(1 * 2 + half) * 128 + c] = m1;
  __syncthreads();
  if (half == 0) {
    int e0 = 0, e1 = 0;
    frexp(fmax(sm.part[0 * 128 + c], sm.part[1 * 128 + c]), &e0);
    frexp(fmax(sm.part[2 * 128 + c], sm.part[3 * 128 + c]), &e1);
    sm.exps[s.slot * 128 + c] = e0;
    if (!INV) sm.exps[((s.slot + 1) & 3) * 128 + c] = e1;  // the (m, 1) sub-item follows in the next slot
  }
  __syncthreads();
}

// Digits of chunk h of sub-item s into stage st (A), and the table chunk (B).
template <bool INV>
__device__ void prepare(const TcArgs &a, const Sub &s, int h, int col0, const Smem &sm, int st)
{
  const int tid = threadIdx.x;
  const int JH = a.JH;
  // A: 128 rows x 4 k-groups of 8; two tasks per thread
  for (int task = tid; task < kM * (kKC / 8); task += kThreads) {
    const int c = task & 127, kg = task >> 7;
    const int b = col0 + (c >> 1), part = c & 1;
    const bool valid = b < a.ncol;
    const int e = sm.exps[s.slot * 128 + c];
    uint4 pk[kS];
    unsigned short *pkh = reinterpret_cast<unsigned short *>(pk);
    if (!INV) {
      // Gs (p = 0) at jh, Ga (p = 1) at JH + jh
      const double *col = reinterpret_cast<const double *>(a.F + ((long long)s.m * a.ncol + (valid ? b : 0)) * a.J) +
                          part + 2 * s.p * JH;
      const double sc = ldexp(1.0, -e);
      double gv[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int jh = min(h * kKC + kg * 8 + q, JH - 1);
        gv[q] = valid ? col[2 * jh] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int jh = h * kKC + kg * 8 + q;
        double x = 0.0;
        if (jh < JH) x = gv[q] * sc;
        unsigned short d[kS];
        digits_bf16(x, d);
#pragma unroll
        for (int k = 0; k < kS; ++k) pkh[k * 8 + q] = d[k];
      }
    } else {
      const double *cf = reinterpret_cast<const double *>(a.Sc + (long long)a.rowoff[s.m] * a.ncol + (valid ? b : 0)) + part;
      const double sc = ldexp(1.0, -e);
      double cv[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int i = min(h * kKC + kg * 8 + q, s.Rp - 1);
        cv[q] = valid ? cf[2 * (long long)(s.p + 2 * i) * a.ncol] : 0.0;
      }
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int i = h * kKC + kg * 8 + q;
        double x = 0.0;
        if (i < s.Rp) x = cv[q] * sc;
        unsigned short d[kS];
        digits_bf16(x, d);
#pragma unroll
        for (int k = 0; k < kS; ++k) pkh[k * 8 + q] = d[k];
      }
    }
#pragma unroll
    for (int k = 0; k < kS; ++k) *reinterpret_cast<uint4 *>(sm.A[st] + k * kM * kRowB + canon(c, kg * 8)) = pk[k];
  }
  // B: the table chunk (kS tiles of npad rows x 32 k), contiguous; copied
  // asynchronously (all 16-byte pieces in flight at once), completed below
  // the segment's rows [row0, row0 + npad) of each digit tile are one run of
  // npad * 64 bytes (row0 is a multiple of 8, whole core-matrix groups)
  const int mp = s.m * 2 + s.p;
  const int tile_rows = INV ? a.npad_max_table : round_up(s.Rp, 16);
  const char *src = reinterpret_cast<const char *>(a.tab + a.toff[mp]) + ((size_t)h * kS * tile_rows + s.row0) * kRowB;
  const int per_tile = s.npad * kRowB / 16;  // 16-byte pieces per digit tile
  for (int q = tid; q < kS * per_tile; q += kThreads) {
    const int t = q / per_tile, r = q - t * per_tile;
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(tc::smem_addr(sm.B[st] + (size_t)t * s.npad * kRowB + 16 * r)),
                 "l"(src + (size_t)t * tile_rows * kRowB + 16 * r));
  }
  asm volatile("cp.async.commit_group;\n" ::);
}

__device__ __forceinline__ void prepare_done() { asm volatile("cp.async.wait_group 0;\n" ::); }

// Read the seven TMEM levels of sub-item s and write the results.
template <bool INV>
__device__ void readout(const TcArgs &a, const Sub &s, int col0, const Smem &sm, uint32_t tbase)
{
  const int tid = threadIdx.x, warp = tid >> 5, c = tid & 127, half = tid >> 7;
  const int b = col0 + (c >> 1), part = c & 1;
  const bool valid = b < a.ncol;
  const int e = sm.exps[s.slot * 128 + c];
  const uint32_t lane_base = tbase + ((uint32_t)((warp & 3) * 32) << 16);
  const int ngroups = s.npad / 16;
  for (int g = half; g < ngroups; g += 2) {
    // all accumulators of the group in flight at once, one wait
    uint32_t r[kAcc][16];
#pragma unroll
    for (int d = 0; d < kAcc; ++d) tc::tmem_ld16(lane_base + (uint32_t)(d * a.npad_max + 16 * g), r[d]);
    tc::tmem_wait_ld();
    double acc[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) {
      double t = 0.0;
#pragma unroll
      for (int d = kAcc - 1; d >= 0; --d) t += (double)__uint_as_float(r[d][i]);  // smallest first
      acc[i] = t;
    }
    if (!INV) {
      if (!valid) continue;
      const int *fe = a.texp + a.teoff[s.m * 2 + s.p];
      const long long rowbase = a.rowoff[s.m];
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int n = s.row0 + 16 * g + i;
        if (n < s.Rp)
          reinterpret_cast<double *>(a.S + (rowbase + s.p + 2 * n) * a.ncol + b)[part] = ldexp(acc[i], e + fe[n] - 14);
      }
    } else if (a.seg_inv != kSegInv) {
      // even-degree sums at F[m][col][jh], odd at F[m][col][JH + jh], straight
      // from the registers (no room for the staging next to kSeg-row segments)
      if (!valid) continue;
      const int *ge = a.texp + (s.m * 2 + s.p) * a.JH;
      double *Fc = reinterpret_cast<double *>(a.Fo + ((long long)s.m * a.ncol + b) * a.J) + part + 2 * s.p * a.JH;
      const int j0 = s.row0 + 16 * g;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int jh = j0 + i;
        if (jh < a.JH) Fc[2 * jh] = ldexp(acc[i], e + ge[jh] - 14);
      }
    } else {
      // staged per half of the CTA so that each warp writes 256-byte runs of
      // one field-level
      const int *ge = a.texp + (s.m * 2 + s.p) * a.JH;
      const int j0 = s.row0 + 16 * g;
      double *stg = sm.stage + half * 64 * kStg;
#pragma unroll
      for (int i = 0; i < 16; ++i) {
        const int jh = j0 + i;
        stg[(c >> 1) * kStg + 2 * i + part] = (jh < a.JH) ? ldexp(acc[i], e + ge[jh] - 14) : 0.0;
      }
      asm volatile("bar.sync %0, 128;\n" ::"r"(1 + half));
      const int wl = warp & 3, lane = tid & 31;
      const int i = lane >> 1, prt = lane & 1;
      if (j0 + i < a.JH) {
#pragma unroll 4
        for (int q = 0; q < 16; ++q) {
          const int bl = 16 * wl + q, col = col0 + bl;
          if (col < a.ncol)
            reinterpret_cast<double *>(a.Fo + ((long long)s.m * a.ncol + col) * a.J + s.p * a.JH + j0 + i)[prt] =
                stg[bl * kStg + lane];
        }
      }
      asm volatile("bar.sync %0, 128;\n" ::"r"(1 + half));
    }
  }
}

template <bool INV>
__global__ void __launch_bounds__(kThreads, 1) k_leg_split(TcArgs a)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint64_t mbar_stage[2], mbar_tmem;
  __shared__ uint32_t tslot;
  const int bstage = kS * a.npad_max * kRowB;
  Smem sm;
  sm.A[0] = smem;
  sm.A[1] = smem + kS * kM * kRowB;
  sm.B[0] = smem + 2 * kS * kM * kRowB;
  sm.B[1] = sm.B[0] + bstage;
  sm.exps = reinterpret_cast<int *>(sm.B[1] + bstage);
  sm.part = reinterpret_cast<double *>(sm.exps + 4 * 128);
  sm.stage = sm.part + 4 * 128;
  const int tid = threadIdx.x, warp = tid >> 5;

  const int it0 = blockIdx.x * a.per_cta;
  const int it1 = min(a.nitems, it0 + a.per_cta);
  if (it0 >= it1) return;

  if (warp == 0) {
    tc::tmem_alloc(&tslot, 512);
    tc::tmem_relinquish();
  }
  if (tid == 0) {
    tc::mbar_init(&mbar_stage[0], 1);
    tc::mbar_init(&mbar_stage[1], 1);
    tc::mbar_init(&mbar_tmem, 1);
    tc::mbar_fence_init();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tbase = tslot;
  uint32_t ph_stage[2] = {0, 0}, ph_tmem = 0;
  bool ok = true;

  Cursor cur{it0, 0, 0, 0, 0};
  Sub s;
  cursor_sub<INV>(a, cur, s);
  {
    const int col0 = (cur.it % a.ntiles) * (kM / 2);
    column_exponents<INV>(a, s, col0, sm);
    prepare<INV>(a, s, 0, col0, sm, 0);
    prepare_done();
    tc::fence_proxy_async();
    __syncthreads();
  }
  for (int u = 0;; ++u) {
    const int st = u & 1;
    const int col0 = (cur.it % a.ntiles) * (kM / 2);
    cursor_sub<INV>(a, cur, s);
    const bool last_chunk = (cur.h + 1 == s.nch);
    if (tid == 0) {
      tc::fence_after();
      issue_chunk(tbase, a.npad_max, tc::smem_addr(sm.A[st]), tc::smem_addr(sm.B[st]), s.npad, cur.h == 0);
      tc::mma_commit(&mbar_stage[st]);
      if (last_chunk) tc::mma_commit(&mbar_tmem);
    }
    __syncwarp();
    // prepare the next unit in the other stage while these MMAs run
    Cursor nxt = cur;
    cursor_next<INV>(a, nxt);
    const bool more = nxt.it < it1;
    if (more) {
      Sub sn;
      cursor_sub<INV>(a, nxt, sn);
      const int ncol0 = (nxt.it % a.ntiles) * (kM / 2);
      if (u >= 1) {  // the other stage is free once the MMAs of unit u-1 are done
        const bool d = tc::mbar_wait(&mbar_stage[st ^ 1], ph_stage[st ^ 1], kWaitLimit);
        if (!d && (tid & 31) == 0) atomicExch(a.err, SHT_ERR_DEVICE_TIMEOUT);
        ok = __syncthreads_and(d) != 0;
        ph_stage[st ^ 1] ^= 1;
      }
      if (ok) {
        if (nxt.h == 0 && nxt.seg == 0 && (INV || sn.p == 0)) column_exponents<INV>(a, sn, ncol0, sm);
        prepare<INV>(a, sn, nxt.h, ncol0, sm, st ^ 1);
        prepare_done();
        tc::fence_proxy_async();
      }
    }
    if (last_chunk && ok) {
      const bool d = tc::mbar_wait(&mbar_tmem, ph_tmem, kWaitLimit);
      if (!d && (tid & 31) == 0) atomicExch(a.err, SHT_ERR_DEVICE_TIMEOUT);
      ok = __syncthreads_and(d) != 0;
      ph_tmem ^= 1;
      tc::fence_after();
      if (ok) readout<INV>(a, s, col0, sm, tbase);
      tc::fence_before();
    }
    ok = __syncthreads_and(ok) != 0;
    if (!more || !ok) break;
    cur = nxt;
  }
  if (!ok) tc::mbar_wait(&mbar_tmem, ph_tmem, kWaitLimit);  // give in-flight MMAs a bounded chance to drain
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
  std::vector<long long> foff(2 * (N + 1)), ioff(2 * (N + 1));
  std::vector<int> feoff(2 * (N + 1));
  const int fch = (JH + kKC - 1) / kKC;
  const int inpad = round_up(JH, 16);
  long long fsz = 0, isz = 0;
  int erows = 0, npmax = 16;
  for (int m = 0; m <= N; ++m)
    for (int pp = 0; pp < 2; ++pp) {
      const int mp = 2 * m + pp, Rp = rows_of_parity(N, m, pp);
      const int np = round_up(Rp > 0 ? Rp : 1, 16);
      npmax = np > npmax ? np : npmax;
      foff[mp] = fsz;
      fsz += (long long)fch * kS * np * kKC;
      feoff[mp] = erows;
      erows += Rp;
      ioff[mp] = isz;
      isz += (long long)((Rp + kKC - 1) / kKC) * kS * inpad * kKC;
    }
  t->fwd_npad_max = npmax;
  t->inv_npad = inpad;
  cudaError_t e;
  auto fail = [&](cudaError_t err, const char *what) {
    cudaFree(t->fwd); cudaFree(t->fwd_off); cudaFree(t->fwd_exp); cudaFree(t->fwd_eoff);
    cudaFree(t->inv); cudaFree(t->inv_off); cudaFree(t->inv_exp); cudaFree(t->d_err);
    delete t;
    return cuda_fail(err, what);
  };
  if ((e = cudaMalloc(&t->fwd, sizeof(__nv_bfloat16) * (size_t)fsz)) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->inv, sizeof(__nv_bfloat16) * (size_t)isz)) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->fwd_off, sizeof(long long) * foff.size())) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->inv_off, sizeof(long long) * ioff.size())) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->fwd_eoff, sizeof(int) * feoff.size())) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->fwd_exp, sizeof(int) * (erows > 0 ? erows : 1))) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->inv_exp, sizeof(int) * 2 * (N + 1) * JH)) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMalloc(&t->d_err, sizeof(int))) != cudaSuccess) return fail(e, "split table");
  cudaStream_t s = p->stream;
  if ((e = cudaMemsetAsync(t->fwd, 0, sizeof(__nv_bfloat16) * (size_t)fsz, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(t->inv, 0, sizeof(__nv_bfloat16) * (size_t)isz, s)) != cudaSuccess ||
      (e = cudaMemsetAsync(t->d_err, 0, sizeof(int), s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(t->fwd_off, foff.data(), sizeof(long long) * foff.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(t->inv_off, ioff.data(), sizeof(long long) * ioff.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess ||
      (e = cudaMemcpyAsync(t->fwd_eoff, feoff.data(), sizeof(int) * feoff.size(), cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return fail(e, "split table upload");
  const int maxrows = (N + 3) / 2;
  dim3 gf((maxrows + 127) / 128, 2 * (N + 1));
  k_slice_table_fwd<<<gf, 128, 0, s>>>(N, JH, p->d_P, p->d_poff, t->fwd, t->fwd_off, t->fwd_exp, t->fwd_eoff);
  count_launch();
  dim3 gi((JH + 127) / 128, 2 * (N + 1));
  k_slice_table_inv<<<gi, 128, 0, s>>>(N, JH, p->d_P, p->d_poff, t->inv, t->inv_off, t->inv_exp, inpad);
  count_launch();
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "split table build");
  p->tc_tables = t;
  return SHT_OK;
}

size_t split_smem(int npad_max, bool staged)
{
  return 2 * (size_t)kS * kM * kRowB + 2 * (size_t)kS * npad_max * kRowB + 4 * 128 * sizeof(int) + 4 * 128 * sizeof(double) +
         (staged ? 2 * 64 * (size_t)kStg * sizeof(double) : 0);
}

int launch_split(sht_plan *p, bool inverse, const double2 *in, int ncol, double2 *out, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  if (!split_supported(p)) {
    set_error("split precision: this grid is not covered by the tensor-core kernel "
              "(needs jm <= 512 and nm <= 509, so that no exact level sums over more than 256 terms)");
    return SHT_ERR_UNSUPPORTED_SIZE;
  }
  int rc = build_split_tables(p);
  if (rc) return rc;
  SplitTables *t = tables(p);
  TcArgs a{};
  if (inverse) {
    a.Sc = in; a.Fo = out; a.tab = t->inv; a.toff = t->inv_off; a.texp = t->inv_exp;
    // staged output (64-row segments) where its buffer fits beside the stages
    a.seg_inv = split_smem(kSegInv, true) <= 227 * 1024 && p->JH <= 128 ? kSegInv : kSeg;
    a.npad_max = t->inv_npad < a.seg_inv ? t->inv_npad : a.seg_inv;
    a.npad_max_table = t->inv_npad;
  } else {
    a.F = in; a.S = out; a.tab = t->fwd; a.toff = t->fwd_off; a.texp = t->fwd_exp; a.teoff = t->fwd_eoff;
    a.npad_max = t->fwd_npad_max < kSeg ? t->fwd_npad_max : kSeg;
  }
  a.rowoff = p->d_rowoff; a.pairs = p->d_pairs;
  a.N = p->N; a.J = p->J; a.JH = p->JH; a.ncol = ncol; a.err = t->d_err;
  a.ntiles = (ncol + kM / 2 - 1) / (kM / 2);
  a.nitems = p->n_pairs * a.ntiles;
  const int slots = p->num_sms;
  a.per_cta = (a.nitems + slots - 1) / slots;
  const int grid = (a.nitems + a.per_cta - 1) / a.per_cta;
  const size_t smem = split_smem(a.npad_max, inverse && a.seg_inv == kSegInv);
  auto kern = inverse ? k_leg_split<true> : k_leg_split<false>;
  cudaError_t e = kernel_setup((const void *)kern, smem, kThreads);
  if (e != cudaSuccess) return cuda_fail(e, "split smem attribute");
  kern<<<grid, kThreads, smem, s>>>(a);
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, inverse ? "k_leg_split<inv>" : "k_leg_split<fwd>");
}

}  // namespace

bool split_supported(const sht_plan *p)
{
  // TMEM holds the kAcc accumulators of one segment (kAcc * kSeg <= 512
  // columns); the exact levels sum over at most 256 latitudes (analysis) or
  // degrees of one parity (synthesis).
  static_assert(kAcc * kSeg <= 512, "TMEM columns");
  const int Rmax = (p->N + 3) / 2;
  return p->JH <= 256 && Rmax <= 256 && split_smem(kSeg, false) <= 227 * 1024;
}

int launch_leg_fwd_split(sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s)
{
  return launch_split(p, false, F, ncol, S, s);
}

int launch_leg_inv_split(sht_plan *p, const double2 *Sp, int ncol, double2 *F, cudaStream_t s)
{
  return launch_split(p, true, Sp, ncol, F, s);
}

// The failure path of the bounded waits, run on purpose: one block waits on a
// shared-memory barrier that nothing arrives at, through the same
// tc::mbar_wait the split kernel uses, gives up after limit_ns and records the
// timeout in the plan's error word as the split kernel does.  It holds no
// TMEM and waits on nothing outside its own block.
__global__ void __launch_bounds__(128) k_wait_selftest(int *err, unsigned long long limit_ns)
{
  __shared__ __align__(8) uint64_t mbar;
  if (threadIdx.x == 0) {
    tc::mbar_init(&mbar, 1);
    tc::mbar_fence_init();
  }
  __syncthreads();
  const bool done = tc::mbar_wait(&mbar, 0, limit_ns);
  if (!done && (threadIdx.x & 31) == 0) atomicExch(err, SHT_ERR_DEVICE_TIMEOUT);
  __syncthreads();
}

int wait_selftest(sht_plan *p, unsigned long long limit_ns)
{
  if (!split_supported(p)) {
    set_error("device timeout self-test: this grid has no split-precision error word");
    return SHT_ERR_UNSUPPORTED_SIZE;
  }
  int rc = build_split_tables(p);
  if (rc) return rc;
  k_wait_selftest<<<1, 128, 0, p->stream>>>(tables(p)->d_err, limit_ns);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, "k_wait_selftest");
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
  cudaFree(t->fwd); cudaFree(t->fwd_off); cudaFree(t->fwd_exp); cudaFree(t->fwd_eoff);
  cudaFree(t->inv); cudaFree(t->inv_off); cudaFree(t->inv_exp); cudaFree(t->d_err);
  delete t;
  p->tc_tables = nullptr;
}

}  // namespace sht
