// sht_legendre_i8.cu -- split-precision Legendre contraction on the sm_100a
// tensor cores: FP64 operands as signed 8-bit digits (eight per data value,
// seven per table value; sht_i8digits.cuh),
// digit products by tcgen05.mma.kind::i8 into exact 32-bit TMEM accumulators,
// one accumulator per digit level, recombined in FP64.
//
// Analysis (space_discretization.tex:197-200):  S[n][col] = sum_jh P[n][jh] G[jh][col]
// Synthesis (space_discretization.tex:212-216): F[jh][col] = sum_n  P[n][jh] S[n][col]
// per order m and degree parity p (Pbar(-mu) = (-1)^(n-m) Pbar(mu)); the
// longitude transforms deliver Gs/Ga and take the even/odd-degree sums at
// F[m][col][jh] and F[m][col][JH + jh].
//
// MMA shape: M = 128 data columns (re and im of 64 field-levels; TMEM lane =
// column), K = latitudes (analysis) or degrees of one parity (synthesis) in
// chunks of 64, N = output rows (degrees / latitudes) in segments of 32.
// Level stacking: the table digits of a segment are stored digit after digit
// ([P_0; P_1; ...; P_6], Npad rows each), so the single MMA of data digit s
// against the table digits t < min(7, 8 - s) writes the level sums
// L = s + t of all its pairs into the accumulator columns starting at
// s Npad: 8 MMAs per K step (9 in a segment's first, which initialises each
// level once) carry the 35 digit pairs of levels 0..7, and each
// accumulator set holds 8 x Npad <= 256 TMEM columns (two sets: a segment's
// readout overlaps the next one's MMAs).
//
// Warp roles (one CTA of 448 threads per SM, persistent over a contiguous
// slice of (band pair, 64-column tile, band, parity) sub-items):
//   warp 0      table producer: bulk copies of the segment's table digits
//   warp 1      TMEM allocation; one thread issues the MMAs and commits
//   converters  FP64 data -> column exponent -> digits in shared memory (one
//               FMA and a few byte permutes per value): 8 warps in the
//               analysis, 4 in the synthesis
//   epilogue    TMEM level sums -> FP64 -> scaled outputs: 4 warps in the
//               analysis, 8 in the synthesis (two per TMEM lane quadrant,
//               alternate 4-row groups)
// Stages: two data-digit stages, two table stages, two accumulator sets and
// four column-exponent slots, each with full/empty mbarriers.  Every wait is
// bounded by 2 s of %globaltimer; a timeout sets the plan's device error word
// and an abort flag that every role polls, and the CTA unwinds (waiting,
// again bounded, for its own MMAs and copies) and frees its TMEM.
//
// A sub-item's data are converted once per group of two output segments
// (once in all at T85 and below), K chunk by K chunk; when K spans several
// chunks, the column exponents come from a first pass over all of them.
#include "sht_internal.h"
#include "sht_tc.cuh"
#include "sht_i8digits.cuh"
#include "sht_l2.cuh"

#include <vector>

namespace sht {

namespace {

using i8::kDigitsData;
using i8::kDigitsTable;
using i8::kLevels;

constexpr int kKC = 64;                              // K per chunk = bytes per row of a digit tile
constexpr int kSeg = 32;                             // output rows per segment
constexpr int kM = 128;                              // data columns per tile (64 complex)
constexpr int kTileA = kM * kKC;                     // one data digit tile
constexpr int kStageA = kDigitsData * kTileA;        // one data stage (64 KB)
constexpr int kStageP = 2 * kDigitsTable * kSeg * kKC;  // one table stage: up to two segments (28 KB)
constexpr int kSetCols = 256;                        // TMEM columns per accumulator set
// Warps per role by direction: the side with three times the values gets 8
// (the analysis converts J (N+1) values per column into (N+1)(N+4)/2 outputs,
// the synthesis the reverse).  14 warps put at most 4 on a scheduler, so each
// thread may hold 128 registers.
template <bool INV>
struct Roles {
  static constexpr int kConvW = INV ? 4 : 8, kEpiW = INV ? 8 : 4;
  static constexpr int kConv0 = 2, kEpi0 = kConv0 + kConvW;
  // values per thread in flight in the column-exponent pass over a sub-item's
  // other K chunks: 16 in the synthesis (strided coefficient rows), 4 in the
  // analysis (contiguous Fourier runs; 16 measured slower at T341)
  static constexpr int kPreBatch = INV ? 16 : 4;
  static constexpr int kThreads = 32 * (kEpi0 + kEpiW);
};
constexpr int kThreads = 448;
static_assert(Roles<false>::kThreads == kThreads && Roles<true>::kThreads == kThreads, "block size");
constexpr int kSlots = 4;                            // column-exponent slots
constexpr uint64_t kWaitLimit = 2000000000ull;       // 2 s per bounded wait
static_assert(kLevels * kSeg <= kSetCols && 2 * kSetCols <= 512, "TMEM columns");

// barrier indices
enum : int {
  B_PFULL = 0, B_PEMPTY = 2, B_DFULL = 4, B_DEMPTY = 6, B_AFULL = 8, B_AEMPTY = 10,
  B_EFULL = 12, B_EEMPTY = 16, B_DONE = 20, B_CFULL = 21, B_SREADY = 23, B_COUNT = 25
};

__host__ __device__ inline int rows_of_parity(int N, int m, int p)
{
  const int R = N + 2 - m;
  return p ? R / 2 : (R + 1) / 2;
}
__host__ __device__ inline int seg_npad(int nrow, int seg)
{
  int r = nrow - seg * kSeg;
  r = r < kSeg ? r : kSeg;
  return (r + 15) & ~15;
}
__host__ __device__ inline int nseg_of(int nrow) { return (nrow + kSeg - 1) / kSeg; }
__host__ __device__ inline int npad_total(int nrow) { return kSeg * (nseg_of(nrow) - 1) + seg_npad(nrow, nseg_of(nrow) - 1); }
// byte offset of (row, K-core kc) in a canonical K-major tile with 64-byte rows
// (8-row x 16-byte core matrices; K-cores 128 B apart, row groups 512 B apart)
__host__ __device__ inline uint32_t canon(int row, int kc) { return (uint32_t)((row >> 3) * 512 + kc * 128 + (row & 7) * 16); }

struct I8Tables {
  uint8_t *tab[2] = {nullptr, nullptr};      // [0] analysis, [1] synthesis
  long long *toff[2] = {nullptr, nullptr};   // byte offset per (m, p)
  double *tfac[2] = {nullptr, nullptr};      // row scale factors 2^(e_row - kShift)
  int *teoff[2] = {nullptr, nullptr};        // first row exponent per (m, p)
  uint8_t *scr[2] = {nullptr, nullptr};      // digit cache: per CTA, two slots of the chunks of one sub-item
  long long scr_cta[2] = {0, 0};             // its bytes per CTA
  int *d_err = nullptr;                      // device error word
};

I8Tables *tables(sht_plan *p) { return static_cast<I8Tables *>(p->tc_tables); }

// Table digits, one thread per (m p, row, 16 K values).  Analysis rows are
// degrees n = m + p + 2 r over the latitudes; synthesis rows are latitudes
// over the degrees of parity p.  Layout per (m, p): K chunk, segment, digit,
// then a canonical tile of npad rows x 64 bytes.
template <bool INV>
__global__ void k_i8_table(int N, int JH, const double *__restrict__ P, const long long *__restrict__ poff,
                           uint8_t *tab, const long long *__restrict__ toff, double *tfac, const int *__restrict__ teoff)
{
  const int mp = blockIdx.y, m = mp >> 1, p = mp & 1;
  if (m > N) return;
  const int Rp = rows_of_parity(N, m, p);
  const int rows = INV ? JH : Rp, K = INV ? Rp : JH;
  const int nk16 = (K + 15) / 16;
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= rows * nk16) return;
  const int r = idx / nk16, k16 = idx - r * nk16;
  const double *base = P + poff[m];
  auto val = [&](int k) -> double {
    return INV ? base[(long long)(p + 2 * k) * JH + r] : base[(long long)(p + 2 * r) * JH + k];
  };
  double mx = 0.0;
  for (int k = 0; k < K; ++k) mx = fmax(mx, fabs(val(k)));
  const int e = i8::exp_of(mx);
  if (k16 == 0) tfac[teoff[mp] + r] = i8::pow2(e - i8::kShift);
  const double sc = i8::pow2(i8::kBitsTable - e);
  uint32_t w[kDigitsTable][4] = {};
  for (int i = 0; i < 16; ++i) {
    const int k = 16 * k16 + i;
    int8_t d[kDigitsTable];
    i8::digits_table(k < K ? val(k) : 0.0, sc, d);
    for (int s = 0; s < kDigitsTable; ++s) w[s][i >> 2] |= (uint32_t)(uint8_t)d[s] << (8 * (i & 3));
  }
  const int npt = npad_total(rows);
  const int k0 = 16 * k16, ch = k0 / kKC, kc = (k0 % kKC) / 16;
  const int seg = r / kSeg, rr = r % kSeg, npad = seg_npad(rows, seg);
  uint8_t *dst = tab + toff[mp] + (long long)ch * kDigitsTable * kKC * npt + (long long)seg * kDigitsTable * kKC * kSeg;
  for (int s = 0; s < kDigitsTable; ++s)
    *reinterpret_cast<uint4 *>(dst + (size_t)s * npad * kKC + canon(rr, kc)) = make_uint4(w[s][0], w[s][1], w[s][2], w[s][3]);
}

struct I8Args {
  const double2 *F;   // analysis input  F[m][col][j]
  double2 *S;         // analysis output S[row][col]
  const double2 *Sc;  // synthesis input
  double2 *Fo;        // synthesis output
  const int *rowoff;
  const int2 *pairs;
  const uint8_t *tab;
  const long long *toff;
  const double *tfac;
  const int *teoff;
  int N, J, JH, ncol, npairs;
  int ntiles, nsub, per_cta;
  int *err;
  uint8_t *scr;        // digit cache (null when no sub-item has more than two segments)
  long long scr_cta;   // bytes of it per CTA: two slots of nchmax data stages
};

// Shared-memory copies of the small lookup tables (band pairs, internal row
// offsets per order, table offsets per order and parity), filled at kernel
// start so that no unit waits on a dependent global load to find its data.
struct Lut {
  const int2 *pairs;
  const int *rowoff;
  const long long *toff;
  const int *teoff;
};
__host__ __device__ inline size_t lut_bytes(int N, int npairs)
{
  return (size_t)2 * (N + 1) * sizeof(long long) + (size_t)npairs * sizeof(int2) + (size_t)(N + 1) * sizeof(int) +
         (size_t)2 * (N + 1) * sizeof(int);
}

// One unit of work: a K chunk of a sub-item (band m, parity p, column tile),
// for a group of at most two of its segments (the two accumulator sets).
struct Unit {
  int g;                  // sub-item: item g / 4, band/parity g % 4
  int m, p, Rp, K, nrow, nseg, nch;
  int seg, ch;            // first segment of this unit's group, K chunk
  int col0;
  int sub_count;          // sub-items this CTA began before this one
  int seg_base;           // segments this CTA began before this sub-item
  int csub;               // sub-items with more than two segments this CTA began before this one
  int rowoff, teoff;      // internal row of degree m, first row factor of (m, p)
  long long toff;         // table bytes of (m, p)
};

// Sub-item g = 4 item + sub, item = tile npairs + i: column tile by column
// tile, and within a tile the band pairs taken alternately from both ends of
// the list (m = 0, the last pair, m = 1, ...).  A pair (m, N - m) holds N + 4
// rows, but its cost goes with the number of 64-deep K chunks and 32-row
// segments of its four sub-items, which is largest for small m; pair-major
// order had given the CTAs on the first pairs half as much work again as
// those on the last.
template <bool INV>
__device__ __forceinline__ bool setup_sub(const I8Args &a, const Lut &t, int g, Unit &u)
{
  const int item = g >> 2, sub = g & 3;
  const int tile = item / a.npairs, i = item - tile * a.npairs;
  const int2 pr = t.pairs[(i & 1) ? a.npairs - 1 - (i >> 1) : (i >> 1)];
  if (sub >= 2 && pr.y < 0) return false;
  u.g = g;
  u.m = sub < 2 ? pr.x : pr.y;
  u.p = sub & 1;
  u.Rp = rows_of_parity(a.N, u.m, u.p);
  u.K = INV ? u.Rp : a.JH;
  u.nrow = INV ? a.JH : u.Rp;
  u.nseg = nseg_of(u.nrow);
  u.nch = (u.K + kKC - 1) / kKC;
  u.seg = 0;
  u.ch = 0;
  u.col0 = tile * (kM / 2);
  u.rowoff = t.rowoff[u.m];
  u.toff = t.toff[2 * u.m + u.p];
  u.teoff = t.teoff[2 * u.m + u.p];
  return u.nrow > 0 && u.K > 0;
}

template <bool INV>
__device__ __forceinline__ bool first_unit(const I8Args &a, const Lut &t, int g0, int g1, Unit &u)
{
  for (int g = g0; g < g1; ++g)
    if (setup_sub<INV>(a, t, g, u)) {
      u.sub_count = 0;
      u.seg_base = 0;
      u.csub = 0;
      return true;
    }
  return false;
}

template <bool INV>
__device__ __forceinline__ bool next_unit(const I8Args &a, const Lut &t, int g1, Unit &u)
{
  if (++u.ch < u.nch) return true;
  u.ch = 0;
  if ((u.seg += 2) < u.nseg) return true;
  const int sc = u.sub_count + 1, sb = u.seg_base + u.nseg, cs = u.csub + (u.nseg > 2 ? 1 : 0);
  for (int g = u.g + 1; g < g1; ++g)
    if (setup_sub<INV>(a, t, g, u)) {
      u.sub_count = sc;
      u.seg_base = sb;
      u.csub = cs;
      return true;
    }
  return false;
}

// Digit cache: a sub-item with more than two output segments is converted by
// the converters once, in its first segment group, which also writes the
// digit stages to the CTA's cache slot; its later groups take the stages from
// there by bulk copy.
__device__ __forceinline__ bool unit_cached(const Unit &u) { return u.nseg > 2 && u.seg >= 2; }
__device__ __forceinline__ uint8_t *cache_stage(const I8Args &a, const Unit &u)
{
  return a.scr + blockIdx.x * a.scr_cta + (u.csub & 1) * (a.scr_cta / 2) + (long long)u.ch * kStageA;
}

struct Ctl {
  uint64_t *bar;
  volatile int *abort_flag;
  int *err;
};

// Bounded wait on a phase; false on timeout (which also raises the abort
// flag and the error word) or when another role has aborted.
__device__ bool wait_ph(const Ctl &c, int b, uint32_t parity)
{
  const uint32_t addr = tc::smem_addr(c.bar + b);
  if (tc::mbar_try(addr, parity)) return true;
  const uint64_t t0 = tc::globaltimer_ns();
  while (true) {
    // the thread is suspended inside the call until the phase completes (or
    // 1 ms passes), so a waiting warp takes no issue slots from working ones
    if (tc::mbar_try_sleep(addr, parity, 1000000u)) return true;
    if (*c.abort_flag) return false;
    if (tc::globaltimer_ns() - t0 > kWaitLimit) {
      *c.abort_flag = 1;
      atomicExch(c.err, SHT_ERR_DEVICE_TIMEOUT);
      return false;
    }
  }
}
// the same for a whole warp: lane 0 waits (acquiring the phase), and the
// shuffle both gives every lane the outcome and orders the lanes' later
// accesses after lane 0's acquire
__device__ __forceinline__ bool warp_wait(const Ctl &c, int b, uint32_t parity)
{
  int ok = 0;
  if ((threadIdx.x & 31) == 0) ok = wait_ph(c, b, parity) ? 1 : 0;
  return __shfl_sync(0xffffffffu, ok, 0) != 0;
}

// No memory clobber: nothing in the kernel reads these outputs, and the
// compiler stays free to overlap the stores with the next rows' arithmetic.
__device__ __forceinline__ void st_keep_f64(double *ptr, double v, uint64_t policy)
{
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;\n" ::"l"(ptr), "d"(v), "l"(policy));
}

// Four rows of one segment: level sums -> FP64 results, computed branch-free
// (independent chains the scheduler can interleave), then stored.
template <bool INV, bool FAST>
__device__ __forceinline__ void epilogue_rows(const I8Args &a, const Unit &u, int row0, int col, bool cv, int part,
                                              const uint32_t (&r)[kLevels][4], const double (&fr)[4], double fcol,
                                              uint64_t keep)
{
  double v[4];
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    int32_t lv[kLevels];
#pragma unroll
    for (int L = 0; L < kLevels; ++L) lv[L] = (int32_t)r[L][i];
    v[i] = i8::combine_levels(lv, FAST) * fcol * fr[i];
  }
  if (!cv) return;
  if (!INV) {
    double *dst = reinterpret_cast<double *>(a.S + ((long long)u.rowoff + u.p + 2 * row0) * a.ncol + col) + part;
    const long long step = 4 * (long long)a.ncol;  // two internal rows (one parity) per output row, in doubles
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (row0 + i < u.nrow) dst[i * step] = v[i];
  } else {
    double *dst = reinterpret_cast<double *>(a.Fo + ((long long)u.m * a.ncol + col) * a.J + u.p * a.JH + row0) + part;
#pragma unroll
    for (int i = 0; i < 4; ++i)
      if (row0 + i < u.nrow) st_keep_f64(dst + 2 * i, v[i], keep);
  }
}

// ---------------------------------------------------------------- roles

template <bool INV, bool CACHE>
__device__ void role_producer(const I8Args &a, const Ctl &c, unsigned char *Ps, unsigned char *As, const Lut &t, Unit u,
                              bool have, int g1)
{
  int k = 0, nc[2] = {0, 0};
  int cpend[2] = {-1, -1};  // phase parity of the last cache copy into each data stage
  for (; have; have = next_unit<INV>(a, t, g1, u), ++k) {
    const int st = k & 1;
    if (k >= 2 && !wait_ph(c, B_PEMPTY + st, ((k >> 1) - 1) & 1)) break;
    const int s0 = u.seg, s1 = min(u.seg + 2, u.nseg);
    const int npt = npad_total(u.nrow);
    const uint8_t *src = a.tab + u.toff + (long long)u.ch * kDigitsTable * kKC * npt +
                         (long long)s0 * kDigitsTable * kKC * kSeg;
    uint32_t bytes = 0;
    for (int s = s0; s < s1; ++s) bytes += kDigitsTable * kKC * seg_npad(u.nrow, s);
    tc::mbar_arrive_expect_tx(c.bar + B_PFULL + st, bytes);
    uint32_t off = 0;
    for (int s = s0; s < s1; ++s) {
      const uint32_t b = kDigitsTable * kKC * seg_npad(u.nrow, s);
      tc::bulk_g2s(Ps + st * kStageP + off, src + off, b, c.bar + B_PFULL + st);
      off += b;
    }
    if (CACHE && unit_cached(u)) {
      // the data digits of a later segment group: the converters wrote them to
      // the cache slot in the sub-item's first group; the stage is free once
      // the MMAs of unit k - 2 are done
      if (u.seg == 2 && u.ch == 0 && !wait_ph(c, B_SREADY + (u.csub & 1), (u.csub >> 1) & 1)) break;
      if (k >= 2 && !wait_ph(c, B_DEMPTY + st, ((k >> 1) - 1) & 1)) break;
      tc::mbar_arrive_expect_tx(c.bar + B_CFULL + st, kStageA);
      tc::bulk_g2s(As + st * kStageA, cache_stage(a, u), kStageA, c.bar + B_CFULL + st);
      cpend[st] = nc[st] & 1;
      ++nc[st];
    }
  }
  // copies issued but never consumed (after an abort) must land before the CTA exits
  for (int j = (k >= 2 ? k - 2 : 0); j < k; ++j) wait_ph(Ctl{c.bar, c.abort_flag, c.err}, B_PFULL + (j & 1), (j >> 1) & 1);
  for (int st = 0; st < 2; ++st)
    if (cpend[st] >= 0) wait_ph(c, B_CFULL + st, (uint32_t)cpend[st]);
}

template <bool INV, bool CACHE>
__device__ void role_mma(const I8Args &a, const Ctl &c, uint32_t As, uint32_t Ps, uint32_t tbase, const Lut &t, Unit u, bool have, int g1)
{
  int k = 0, nd[2] = {0, 0}, nc[2] = {0, 0};
  for (; have; have = next_unit<INV>(a, t, g1, u), ++k) {
    const int st = k & 1;
    if (!wait_ph(c, B_PFULL + st, (k >> 1) & 1)) break;
    // the data stage comes from the converters or, for a cached unit, from
    // the producer's copy of the digit cache
    if ((CACHE && unit_cached(u)) ? !wait_ph(c, B_CFULL + st, nc[st]++ & 1) : !wait_ph(c, B_DFULL + st, nd[st]++ & 1))
      break;
    tc::fence_after();
    const int s0 = u.seg, s1 = min(u.seg + 2, u.nseg);
    const int kvalid = min(kKC, u.K - u.ch * kKC);
    const int nks = (kvalid + 31) / 32;
    uint32_t pb = Ps + st * kStageP;
    bool ok = true;
    for (int s = s0; s < s1 && ok; ++s) {
      const int npad = seg_npad(u.nrow, s);
      const int ord = u.seg_base + s, set = ord & 1, use = ord >> 1;
      if (u.ch == 0 && use >= 1) {
        ok = wait_ph(c, B_AEMPTY + set, (use - 1) & 1);
        if (!ok) break;
        tc::fence_after();
      }
      const uint32_t d0 = tbase + (uint32_t)(set * kSetCols);
      // descriptors built once; the start address (bits 0..13, in 16-byte
      // units, below 256 KB of shared memory) then steps by plain adds
      const uint64_t ad0 = tc::smem_desc(As + st * kStageA, 128, 512);
      const uint64_t bd0 = tc::smem_desc(pb, 128, 512);
      const uint32_t id0 = tc::idesc_s8_s32(kM, 0);
      // MMA of data digit sd against table digits [t0, t0 + nt): level sums
      // L = sd + t go to accumulator columns from (sd + t0) npad on
      auto mma = [&](int ks, int sd, int t0, int nt, uint32_t acc) {
        const uint64_t ad = ad0 + (uint64_t)((sd * kTileA + ks * 256) >> 4);
        const uint64_t bd = bd0 + (uint64_t)((t0 * npad * kKC + ks * 256) >> 4);
        tc::mma_s8(d0 + (uint32_t)((sd + t0) * npad), ad, bd, id0 | ((uint32_t)(nt * npad) >> 3) << 17, acc);
      };
      static_assert(kLevels == kDigitsTable + 1, "data digits 0 and 1 pair with every table digit");
      for (int ks = 0; ks < nks; ++ks) {
        if (u.ch == 0 && ks == 0) {
          // the segment's first K step initialises every level exactly once:
          // digit 1 against t = 0..6 sets levels 1..7, digit 0 against t = 0
          // sets level 0, and digit 0 against t = 1..6 adds to levels 1..6
          mma(ks, 1, 0, kDigitsTable, 0u);
          mma(ks, 0, 0, 1, 0u);
          mma(ks, 0, 1, kDigitsTable - 1, 1u);
        } else {
          mma(ks, 0, 0, kDigitsTable, 1u);
          mma(ks, 1, 0, kDigitsTable, 1u);
        }
#pragma unroll
        for (int sd = 2; sd < kDigitsData; ++sd) mma(ks, sd, 0, kLevels - sd, 1u);  // t < 8 - sd
      }
      if (u.ch == u.nch - 1) tc::mma_commit(c.bar + B_AFULL + set);
      pb += kDigitsTable * kKC * npad;
    }
    if (!ok) break;
    tc::mma_commit(c.bar + B_DEMPTY + st);
    tc::mma_commit(c.bar + B_PEMPTY + st);
  }
  tc::mma_commit(c.bar + B_DONE);
}

// Load NV consecutive K values (k0 + i) of this thread's complex column.
template <bool INV, int NV>
__device__ __forceinline__ void loadn(const I8Args &a, const Unit &u, int col, bool cv, int k0, double2 (&x)[NV])
{
  if (!INV) {
    const double2 *src = a.F + ((long long)u.m * a.ncol + (cv ? col : 0)) * a.J + u.p * a.JH;
#pragma unroll
    for (int i = 0; i < NV; ++i) x[i] = (cv && k0 + i < u.K) ? src[k0 + i] : make_double2(0.0, 0.0);
  } else {
    // one row pointer advanced by two internal rows (one parity) per value:
    // no per-value 64-bit index products held for the whole batch of loads
    const size_t step = (size_t)2 * a.ncol;
    const double2 *src = a.Sc + ((long long)u.rowoff + u.p + 2 * k0) * a.ncol + (cv ? col : 0);
    const int nv = cv ? u.K - k0 : 0;
#pragma unroll
    for (int i = 0; i < NV; ++i) {
      x[i] = i < nv ? *src : make_double2(0.0, 0.0);
      src += step;
    }
  }
}
template <bool INV>
__device__ __forceinline__ void load16(const I8Args &a, const Unit &u, int col, bool cv, int k0, double2 (&x)[16])
{
  loadn<INV, 16>(a, u, col, cv, k0, x);
}

// r, im <- the largest high word (sign cleared) of the real and imaginary
// parts of NV values and r, im
template <int NV>
__device__ __forceinline__ void hmaxn(const double2 (&y)[NV], int &r, int &im)
{
#pragma unroll
  for (int i = 0; i < NV; ++i) {
    r = max(r, __double2hiint(y[i].x) & 0x7FFFFFFF);
    im = max(im, __double2hiint(y[i].y) & 0x7FFFFFFF);
  }
}

template <bool INV, bool CACHE>
__device__ void role_convert(const I8Args &a, const Ctl &c, unsigned char *As, int *exps, const Lut &t, Unit u, bool have, int g1)
{
  using R = Roles<INV>;
  constexpr int kPass = 8 / R::kConvW;  // column passes: 64 columns, 8 per warp and pass
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int c8 = lane & 7, q = lane >> 3;
  // half of the lanes write the imaginary row first, so that each 8-lane
  // phase of a 16-byte store covers the eight rows of a core matrix
  const int first_part = (c8 >> 2) & 1;
  static_assert(kPass <= 2, "two exponent pairs per thread");
  int er0 = 0, ei0 = 0, er1 = 0, ei1 = 0;  // column exponents of passes 0 and 1
  int k = 0;
  for (; have; have = next_unit<INV>(a, t, g1, u), ++k) {
    const int st = k & 1;
    if (CACHE && unit_cached(u)) {
      // the producer copies these digits from the cache; the converters still
      // step through the stage's phases one at a time (a parity wait only
      // tells the last two phases apart), so they wait for unit k - 2 here
      if (k >= 2 && !warp_wait(c, B_DEMPTY + st, ((k >> 1) - 1) & 1)) break;
      continue;
    }
    const int k0 = u.ch * kKC + 16 * q;
    // a sub-item with more than two segments keeps its digits for its later groups
    uint8_t *const cache = (CACHE && u.nseg > 2) ? cache_stage(a, u) : nullptr;
    const bool first = u.seg == 0 && u.ch == 0;
    const int slot = u.sub_count & (kSlots - 1);
    if (first && u.sub_count >= kSlots && !warp_wait(c, B_EEMPTY + slot, (u.sub_count / kSlots - 1) & 1)) break;
    bool ok = true, stage_free = k < 2;
    unsigned char *stage = As + st * kStageA;
#pragma unroll 1
    for (int ps = 0; ps < kPass; ++ps) {
      const int cl = 8 * (warp - R::kConv0) + c8 + 8 * R::kConvW * ps;  // complex column within the tile
      const int col = u.col0 + cl;
      const bool cv = col < a.ncol;
      // the exponent of a column's largest magnitude is that of the largest
      // high word (sign cleared): integer maxima, no FP64 chain
      int mr = 0, mi = 0;
      // the largest high word (sign cleared) of 16 values
      auto hmax = [](const double2 (&y)[16], int &r, int &im) {
        int hr[8], hi[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          hr[i] = max(__double2hiint(y[i].x) & 0x7FFFFFFF, __double2hiint(y[i + 8].x) & 0x7FFFFFFF);
          hi[i] = max(__double2hiint(y[i].y) & 0x7FFFFFFF, __double2hiint(y[i + 8].y) & 0x7FFFFFFF);
        }
#pragma unroll
        for (int w = 4; w >= 1; w >>= 1)
#pragma unroll
          for (int i = 0; i < w; ++i) {
            hr[i] = max(hr[i], hr[i + w]);
            hi[i] = max(hi[i], hi[i + w]);
          }
        r = max(r, hr[0]);
        im = max(im, hi[0]);
      };
      if (first) {
        // column exponents over the sub-item's other K chunks (the first
        // unit converts chunk 0), kPreBatch values of this thread in flight
        // at a time, before this chunk's values take their registers
        constexpr int PB = Roles<INV>::kPreBatch;
        for (int kc = 1; kc < u.nch; ++kc)
#pragma unroll 1
          for (int i0 = 0; i0 < 16; i0 += PB) {
            double2 y[PB];
            loadn<INV, PB>(a, u, col, cv, kc * kKC + 16 * q + i0, y);
            hmaxn<PB>(y, mr, mi);
          }
      }
      double2 x[16];
      load16<INV>(a, u, col, cv, k0, x);
      if (first) {
        hmax(x, mr, mi);
        mr = max(mr, __shfl_xor_sync(0xffffffffu, mr, 8));
        mr = max(mr, __shfl_xor_sync(0xffffffffu, mr, 16));
        mi = max(mi, __shfl_xor_sync(0xffffffffu, mi, 8));
        mi = max(mi, __shfl_xor_sync(0xffffffffu, mi, 16));
        const int e_r = i8::exp_of_hi(mr), e_i = i8::exp_of_hi(mi);
        if (ps) { er1 = e_r; ei1 = e_i; } else { er0 = e_r; ei0 = e_i; }
        if (q == 0) {
          exps[slot * kM + 2 * cl] = e_r;
          exps[slot * kM + 2 * cl + 1] = e_i;
        }
      }
      if (!INV && u.nseg <= 2 && u.nch == 1 && cv && (a.JH & 7) == 0) {
        // each 128-byte line of this column's run is read once, by this thread:
        // drop it from L2 without a write-back (the values are in registers)
        const double2 *src = a.F + ((long long)u.m * a.ncol + col) * a.J + u.p * a.JH + k0;
#pragma unroll
        for (int h = 0; h < 2; ++h)
          if (k0 + 8 * h + 8 <= u.K) l2::discard_line(src + 8 * h);
      }
      if (!stage_free) {
        if (!warp_wait(c, B_DEMPTY + st, ((k >> 1) - 1) & 1)) { ok = false; break; }
        stage_free = true;
      }
      // K positions at or past K meet zero table digits, so whatever the stage
      // holds there adds nothing: those 16-value groups are not converted
      if (k0 < u.K)
#pragma unroll
      for (int pp = 0; pp < 2; ++pp) {
        const int part = pp ^ first_part;
        const double sc = i8::pow2(i8::kBitsData - (part ? (ps ? ei1 : ei0) : (ps ? er1 : er0)));
        // four values at a time: conversions, then their byte permutes (the
        // groups are independent, and fewer words are live at once)
        uint32_t w[4][kDigitsData];
#pragma unroll
        for (int g = 0; g < 4; ++g) {
          uint32_t lo[4], hi[4];
#pragma unroll
          for (int i = 0; i < 4; ++i) {
            const unsigned long long y = i8::data_word(part ? x[4 * g + i].y : x[4 * g + i].x, sc);
            lo[i] = (uint32_t)y;
            hi[i] = (uint32_t)(y >> 32);
          }
          i8::digit_words_data(lo, hi, w[g]);
        }
        const uint32_t off = canon(2 * cl + part, q);
#pragma unroll
        for (int s = 0; s < kDigitsData; ++s) {
          const uint4 d4 = make_uint4(w[0][s], w[1][s], w[2][s], w[3][s]);
          *reinterpret_cast<uint4 *>(stage + s * kTileA + off) = d4;
          if (cache) *reinterpret_cast<uint4 *>(cache + s * kTileA + off) = d4;
        }
      }
    }
    if (!ok) break;
    if (first) {
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(c.bar + B_EFULL + slot);
    }
    tc::fence_proxy_async();
    if (cache) tc::fence_proxy_async_global();
    __syncwarp();
    if (lane == 0) {
      tc::mbar_arrive(c.bar + B_DFULL + st);
      // the sub-item's first group is written to the cache: its later groups may be copied
      if (cache && u.ch == u.nch - 1) tc::mbar_arrive(c.bar + B_SREADY + (u.csub & 1));
    }
  }
}

template <bool INV>
__device__ void role_epilogue(const I8Args &a, const Ctl &c, const int *exps, uint32_t tbase, const Lut &t, Unit u, bool have, int g1)
{
  using R = Roles<INV>;
  constexpr int kGs = R::kEpiW / 4;  // warps per TMEM lane quadrant
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int quad = warp & 3, gi = (warp - R::kEpi0) >> 2;
  const int rl = 32 * quad + lane;  // TMEM lane = data column of the tile
  const int cl = rl >> 1, part = rl & 1;
  const uint32_t tl = tbase + ((uint32_t)(32 * quad) << 16);
  const uint64_t keep = l2::keep_policy();
  int ecol = 0;
  for (; have; have = next_unit<INV>(a, t, g1, u)) {
    const int col = u.col0 + cl;
    const bool cv = col < a.ncol;
    if (u.seg == 0 && u.ch == 0) {
      const int slot = u.sub_count & (kSlots - 1), use = u.sub_count / kSlots;
      if (!warp_wait(c, B_EFULL + slot, use & 1)) break;
      ecol = exps[slot * kM + rl];
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(c.bar + B_EEMPTY + slot);
    }
    if (u.ch != u.nch - 1) continue;  // no segment completes in this unit
    const int s0 = u.seg, s1 = min(u.seg + 2, u.nseg);
    const double *frow = a.tfac + u.teoff;
    const double fcol = i8::pow2(ecol < 1023 ? ecol : 1023);
    const bool fast = u.K <= 64;
    bool ok = true;
    for (int s = s0; s < s1; ++s) {
      const int npad = seg_npad(u.nrow, s);
      const int ord = u.seg_base + s, set = ord & 1, use = ord >> 1;
      if (!warp_wait(c, B_AFULL + set, use & 1)) { ok = false; break; }
      tc::fence_after();
      for (int g4 = gi; g4 < npad / 4; g4 += kGs) {
        // the group's row factors first, so that their loads overlap the TMEM reads
        double fr[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) {
          const int row = s * kSeg + 4 * g4 + i;
          fr[i] = row < u.nrow ? __ldg(frow + row) : 0.0;
        }
        uint32_t r[kLevels][4];
#pragma unroll
        for (int L = 0; L < kLevels; ++L) tc::tmem_ld4(tl + (uint32_t)(set * kSetCols + L * npad + 4 * g4), r[L]);
        tc::tmem_wait_ld();
        if (fast)
          epilogue_rows<INV, true>(a, u, s * kSeg + 4 * g4, col, cv, part, r, fr, fcol, keep);
        else
          epilogue_rows<INV, false>(a, u, s * kSeg + 4 * g4, col, cv, part, r, fr, fcol, keep);
      }
      tc::fence_before();
      __syncwarp();
      if (lane == 0) tc::mbar_arrive(c.bar + B_AEMPTY + set);
    }
    if (!ok) break;
  }
}

template <bool INV, bool CACHE>
__global__ void __launch_bounds__(kThreads, 1) k_leg_i8(I8Args a)
{
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ __align__(8) uint64_t bar[B_COUNT];
  __shared__ uint32_t tslot;
  __shared__ int abort_flag;
  unsigned char *As = smem;
  unsigned char *Ps = smem + 2 * kStageA;
  int *exps = reinterpret_cast<int *>(Ps + 2 * kStageP);
  long long *s_toff = reinterpret_cast<long long *>(exps + kSlots * kM);
  int2 *s_pairs = reinterpret_cast<int2 *>(s_toff + 2 * (a.N + 1));
  int *s_rowoff = reinterpret_cast<int *>(s_pairs + a.npairs);
  int *s_teoff = s_rowoff + (a.N + 1);

  const int g0 = blockIdx.x * a.per_cta;
  const int g1 = min(a.nsub, g0 + a.per_cta);
  if (g0 >= g1) return;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

  if (warp == 1) {
    tc::tmem_alloc(&tslot, 512);
    tc::tmem_relinquish();
  }
  for (int i = threadIdx.x; i < 2 * (a.N + 1); i += blockDim.x) {
    s_toff[i] = a.toff[i];
    s_teoff[i] = a.teoff[i];
  }
  for (int i = threadIdx.x; i < a.npairs; i += blockDim.x) s_pairs[i] = a.pairs[i];
  for (int i = threadIdx.x; i < a.N + 1; i += blockDim.x) s_rowoff[i] = a.rowoff[i];
  const Lut t{s_pairs, s_rowoff, s_toff, s_teoff};
  if (threadIdx.x == 0) {
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(bar + B_PFULL + i, 1);
      tc::mbar_init(bar + B_PEMPTY + i, 1);
      tc::mbar_init(bar + B_DFULL + i, Roles<INV>::kConvW);
      tc::mbar_init(bar + B_DEMPTY + i, 1);
      tc::mbar_init(bar + B_AFULL + i, 1);
      tc::mbar_init(bar + B_AEMPTY + i, Roles<INV>::kEpiW);
    }
    for (int i = 0; i < kSlots; ++i) {
      tc::mbar_init(bar + B_EFULL + i, Roles<INV>::kConvW);
      tc::mbar_init(bar + B_EEMPTY + i, Roles<INV>::kEpiW);
    }
    for (int i = 0; i < 2; ++i) {
      tc::mbar_init(bar + B_CFULL + i, 1);
      tc::mbar_init(bar + B_SREADY + i, Roles<INV>::kConvW);
    }
    tc::mbar_init(bar + B_DONE, 1);
    abort_flag = 0;
    tc::mbar_fence_init();
  }
  tc::fence_before();
  __syncthreads();
  tc::fence_after();
  const uint32_t tbase = tslot;
  const Ctl c{bar, &abort_flag, a.err};

  Unit u;
  const bool have = first_unit<INV>(a, t, g0, g1, u);
  if (warp == 0) {
    if (lane == 0) role_producer<INV, CACHE>(a, c, Ps, As, t, u, have, g1);
  } else if (warp == 1) {
    if (lane == 0) role_mma<INV, CACHE>(a, c, tc::smem_addr(As), tc::smem_addr(Ps), tbase, t, u, have, g1);
  } else if (warp < Roles<INV>::kEpi0) {
    role_convert<INV, CACHE>(a, c, As, exps, t, u, have, g1);
  } else {
    role_epilogue<INV>(a, c, exps, tbase, t, u, have, g1);
  }

  tc::fence_before();
  __syncthreads();
  if (warp == 1) {
    // the MMA thread's last commit: every MMA it issued has completed
    if (lane == 0) {
      const uint32_t addr = tc::smem_addr(bar + B_DONE);
      const uint64_t t0 = tc::globaltimer_ns();
      while (!tc::mbar_try(addr, 0) && tc::globaltimer_ns() - t0 < kWaitLimit) {
      }
    }
    __syncwarp();
    tc::fence_after();
    tc::tmem_dealloc(tbase, 512);
  }
}

int build_i8_tables(sht_plan *p)
{
  if (p->tc_tables) return SHT_OK;
  const int N = p->N, JH = p->JH, nmp = 2 * (N + 1);
  auto *t = new I8Tables();
  std::vector<long long> toff[2];
  std::vector<int> teoff[2];
  long long tsz[2] = {0, 0};
  int esz[2] = {0, 0};
  for (int d = 0; d < 2; ++d) {
    toff[d].resize(nmp);
    teoff[d].resize(nmp);
    for (int m = 0; m <= N; ++m)
      for (int pp = 0; pp < 2; ++pp) {
        const int mp = 2 * m + pp, Rp = rows_of_parity(N, m, pp);
        const int rows = d ? JH : Rp, K = d ? Rp : JH;
        toff[d][mp] = tsz[d];
        teoff[d][mp] = esz[d];
        if (rows > 0 && K > 0) tsz[d] += (long long)((K + kKC - 1) / kKC) * kDigitsTable * kKC * npad_total(rows);
        esz[d] += rows;
      }
  }
  cudaError_t e = cudaSuccess;
  auto fail = [&](cudaError_t err, const char *what) {
    for (int d = 0; d < 2; ++d) {
      cudaFree(t->tab[d]); cudaFree(t->toff[d]); cudaFree(t->tfac[d]); cudaFree(t->teoff[d]); cudaFree(t->scr[d]);
    }
    cudaFree(t->d_err);
    delete t;
    return cuda_fail(err, what);
  };
  cudaStream_t s = p->stream;
  for (int d = 0; d < 2; ++d) {
    if ((e = cudaMalloc(&t->tab[d], (size_t)(tsz[d] > 0 ? tsz[d] : 16))) != cudaSuccess) return fail(e, "split table");
    if ((e = cudaMalloc(&t->toff[d], sizeof(long long) * nmp)) != cudaSuccess) return fail(e, "split table");
    if ((e = cudaMalloc(&t->tfac[d], sizeof(double) * (esz[d] > 0 ? esz[d] : 1))) != cudaSuccess) return fail(e, "split table");
    if ((e = cudaMalloc(&t->teoff[d], sizeof(int) * nmp)) != cudaSuccess) return fail(e, "split table");
    if ((e = cudaMemsetAsync(t->tab[d], 0, (size_t)(tsz[d] > 0 ? tsz[d] : 16), s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(t->toff[d], toff[d].data(), sizeof(long long) * nmp, cudaMemcpyHostToDevice, s)) != cudaSuccess ||
        (e = cudaMemcpyAsync(t->teoff[d], teoff[d].data(), sizeof(int) * nmp, cudaMemcpyHostToDevice, s)) != cudaSuccess)
      return fail(e, "split table upload");
  }
  // digit cache for sub-items with more than two 32-row output segments:
  // analysis rows are the degrees of one parity, synthesis rows the latitudes
  for (int d = 0; d < 2; ++d) {
    const int nrow = d ? JH : (N + 3) / 2, K = d ? (N + 3) / 2 : JH;
    if (nrow <= 2 * kSeg) continue;
    t->scr_cta[d] = 2LL * ((K + kKC - 1) / kKC) * kStageA;
    const size_t bytes = (size_t)t->scr_cta[d] * (p->num_sms > 0 ? p->num_sms : 1);
    if ((e = cudaMalloc(&t->scr[d], bytes)) != cudaSuccess) return fail(e, "split digit cache");
  }
  if ((e = cudaMalloc(&t->d_err, sizeof(int))) != cudaSuccess) return fail(e, "split table");
  if ((e = cudaMemsetAsync(t->d_err, 0, sizeof(int), s)) != cudaSuccess) return fail(e, "split table upload");
  {
    const int maxrows = (N + 3) / 2, nk16 = (JH + 15) / 16;
    dim3 g((maxrows * nk16 + 127) / 128, nmp);
    k_i8_table<false><<<g, 128, 0, s>>>(N, JH, p->d_P, p->d_poff, t->tab[0], t->toff[0], t->tfac[0], t->teoff[0]);
    count_launch();
  }
  {
    const int nk16 = ((N + 3) / 2 + 15) / 16;
    dim3 g((JH * nk16 + 127) / 128, nmp);
    k_i8_table<true><<<g, 128, 0, s>>>(N, JH, p->d_P, p->d_poff, t->tab[1], t->toff[1], t->tfac[1], t->teoff[1]);
    count_launch();
  }
  if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(s)) != cudaSuccess) return fail(e, "split table build");
  p->tc_tables = t;
  return SHT_OK;
}

constexpr size_t kSmemFixed = 2 * (size_t)kStageA + 2 * (size_t)kStageP + kSlots * kM * sizeof(int);

int launch_i8(sht_plan *p, bool inverse, const double2 *in, int ncol, double2 *out, cudaStream_t s)
{
  if (ncol <= 0) return SHT_OK;
  int rc = build_i8_tables(p);
  if (rc) return rc;
  I8Tables *t = tables(p);
  const int d = inverse ? 1 : 0;
  I8Args a{};
  if (inverse) { a.Sc = in; a.Fo = out; } else { a.F = in; a.S = out; }
  a.rowoff = p->d_rowoff; a.pairs = p->d_pairs;
  a.tab = t->tab[d]; a.toff = t->toff[d]; a.tfac = t->tfac[d]; a.teoff = t->teoff[d];
  a.scr = t->scr[d]; a.scr_cta = t->scr_cta[d];
  a.N = p->N; a.J = p->J; a.JH = p->JH; a.ncol = ncol; a.err = t->d_err; a.npairs = p->n_pairs;
  a.ntiles = (ncol + kM / 2 - 1) / (kM / 2);
  a.nsub = 4 * p->n_pairs * a.ntiles;
  const int slots = grid_sms(p);  // never above the SM count the digit cache is sized for
  a.per_cta = (a.nsub + slots - 1) / slots;
  const int grid = (a.nsub + a.per_cta - 1) / a.per_cta;
  // the digit-cache instance where some sub-item has more than two output
  // segments (T170 and up), the plain one elsewhere
  auto kern = inverse ? (a.scr ? k_leg_i8<true, true> : k_leg_i8<true, false>)
                      : (a.scr ? k_leg_i8<false, true> : k_leg_i8<false, false>);
  const size_t smem = kSmemFixed + lut_bytes(p->N, p->n_pairs);
  if (smem > 227 * 1024) {
    set_error("split precision: the truncation's lookup tables do not fit beside the stages");
    return SHT_ERR_UNSUPPORTED_SIZE;
  }
  cudaError_t e = kernel_setup((const void *)kern, smem, kThreads);
  if (e != cudaSuccess) return cuda_fail(e, "split smem attribute");
  kern<<<grid, kThreads, smem, s>>>(a);
  count_launch();
  e = cudaGetLastError();
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, inverse ? "k_leg_i8<inv>" : "k_leg_i8<fwd>");
}

}  // namespace

bool split_supported(const sht_plan *p)
{
  // exact 32-bit level sums need fewer than 2^14 terms per contraction
  return p->JH < 16384 && p->N < 16384;
}

int launch_leg_fwd_split(sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s)
{
  return launch_i8(p, false, F, ncol, S, s);
}

int launch_leg_inv_split(sht_plan *p, const double2 *Sp, int ncol, double2 *F, cudaStream_t s)
{
  return launch_i8(p, true, Sp, ncol, F, s);
}

// The failure path of the bounded waits, run on purpose: one block waits on a
// shared-memory barrier that nothing arrives at, through the same bounded
// poll the split kernel uses, gives up after limit_ns and records the
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
  int rc = build_i8_tables(p);
  if (rc) return rc;
  k_wait_selftest<<<1, 128, 0, p->stream>>>(tables(p)->d_err, limit_ns);
  count_launch();
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaStreamSynchronize(p->stream);
  return e == cudaSuccess ? SHT_OK : cuda_fail(e, "k_wait_selftest");
}

int split_error_status(sht_plan *p)
{
  I8Tables *t = tables(p);
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
  I8Tables *t = tables(p);
  if (!t) return;
  for (int d = 0; d < 2; ++d) {
    cudaFree(t->tab[d]); cudaFree(t->toff[d]); cudaFree(t->tfac[d]); cudaFree(t->teoff[d]); cudaFree(t->scr[d]);
  }
  cudaFree(t->d_err);
  delete t;
  p->tc_tables = nullptr;
}

}  // namespace sht
