// sht_i8digits.cuh -- the fixed-point digit representation of the
// split-precision Legendre contraction (host and device).
//
// A value x of a row (or column) whose magnitudes are below 2^e becomes the
// integer X = round(x 2^(B-e)), |X| <= 2^B, written in balanced base-256
// digits c_s in [-128, 127] (most significant first), stored as signed 8-bit
// integers (the kind::i8 operand format of the tensor cores):
//   data  (converted on the fly): B = 58, eight digits, |c_0| <= 4;
//   table (converted once per plan): B = 54, seven digits, |c_0| <= 64.
// Representation error: 2^-59 (data) and 2^-55 (table) of the row or column
// bound.  The data keeps more bits because a column can span a large range
// (Gauss-weighted rows divided by 1 - mu^2 grow towards the poles, and every
// value is fixed-point against the column's largest).
// Both come from the exact 64-bit integer X plus the offset 0x80808080808080:
// byte b < 7 of the sum is c_{D-1-b} + 128, and for the data its top byte is
// c_0 in two's complement.
//
// Products are sums of digit products c_s c'_t of weight 256^(13-s-t); level
// L = s + t collects the pairs of equal weight.  The contraction keeps the
// levels L < 8 (35 pairs) as exact 32-bit integer sums (|c_s c'_t| <= 2^14,
// at most 7 pairs, K < 18000 terms).  The result is
//     sum_k x_k p_k ~= 2^(e_x + e_p - 64) sum_{L<8} A_L 256^(7-L);
// the dropped levels (L >= 8, six pairs) are below 6 K 2^-58 of the product
// bound.
#pragma once

#include <cmath>
#include <cstdint>
#include <cuda_runtime.h>

namespace sht {
namespace i8 {

constexpr int kDigitsData = 8;   // digits of a data value
constexpr int kDigitsTable = 7;  // digits of a table value
constexpr int kLevels = 8;       // levels kept: digit pairs with s + t < kLevels
constexpr int kBitsData = 58;    // |X| <= 2^58 for the data operand
constexpr int kBitsTable = 54;   // |X| <= 2^54 for the Legendre table
constexpr int kShift = kBitsData + kBitsTable - 8 * ((kDigitsData - 1) + (kDigitsTable - 1) - (kLevels - 1));  // 64
constexpr int kExpMin = -950;    // exponents are kept >= this, so that every scale is a normal double
constexpr long long kOffset7 = 0x80808080808080LL;  // 128 in each of the low seven bytes

__host__ __device__ inline int64_t dbits(double x)
{
#ifdef __CUDA_ARCH__
  return __double_as_longlong(x);
#else
  int64_t b;
  __builtin_memcpy(&b, &x, 8);
  return b;
#endif
}
__host__ __device__ inline double bits2d(int64_t b)
{
#ifdef __CUDA_ARCH__
  return __longlong_as_double(b);
#else
  double x;
  __builtin_memcpy(&x, &b, 8);
  return x;
#endif
}

// e with 0 <= mx < 2^e (mx >= 0), kept >= kExpMin
__host__ __device__ inline int exp_of(double mx)
{
  const int E = (int)((dbits(mx) >> 52) & 0x7FF);
  const int e = E - 1022;
  return e < kExpMin ? kExpMin : e;
}

// the same from the high word of the largest magnitude (sign bit clear)
__host__ __device__ inline int exp_of_hi(int hi)
{
  const int e = (hi >> 20) - 1022;
  return e < kExpMin ? kExpMin : e;
}

// 2^e for -1022 <= e <= 1023
__host__ __device__ inline double pow2(int e) { return bits2d((int64_t)(e + 1023) << 52); }

__host__ __device__ inline uint32_t bperm(uint32_t x, uint32_t y, uint32_t s)
{
#ifdef __CUDA_ARCH__
  return __byte_perm(x, y, s);
#else
  uint8_t in[8];
  for (int i = 0; i < 4; ++i) { in[i] = (uint8_t)(x >> (8 * i)); in[4 + i] = (uint8_t)(y >> (8 * i)); }
  uint32_t r = 0;
  for (int i = 0; i < 4; ++i) r |= (uint32_t)in[(s >> (4 * i)) & 7] << (8 * i);
  return r;
#endif
}

// byte b of four words -> one word (word i gives byte i), for b = 0..3
__host__ __device__ inline void transpose4(const uint32_t (&v)[4], uint32_t (&o)[4])
{
  const uint32_t t0 = bperm(v[0], v[1], 0x5140), t1 = bperm(v[2], v[3], 0x5140);
  const uint32_t t2 = bperm(v[0], v[1], 0x7362), t3 = bperm(v[2], v[3], 0x7362);
  o[0] = bperm(t0, t1, 0x5410);
  o[1] = bperm(t0, t1, 0x7632);
  o[2] = bperm(t2, t3, 0x5410);
  o[3] = bperm(t2, t3, 0x7632);
}

__host__ __device__ inline long long d2ll(double y)
{
#ifdef __CUDA_ARCH__
  return __double2ll_rn(y);
#else
  return llrint(y);
#endif
}

// The exact 64-bit integer of a data value (scale 2^(58-e)) plus the offset:
// its low seven bytes are c_{7-b} + 128 and its top byte is c_0.  The product
// with the power-of-two scale is exact; the conversion rounds once.
__host__ __device__ inline unsigned long long data_word(double x, double sc)
{
  return (unsigned long long)(d2ll(x * sc) + kOffset7);
}

// The words of four consecutive data values (low and high halves) -> w[s] =
// the four signed digits c_s, one byte each (K order, lowest address first).
__host__ __device__ inline void digit_words_data(const uint32_t (&lo)[4], const uint32_t (&hi)[4], uint32_t (&w)[kDigitsData])
{
  uint32_t l[4], h[4];
  transpose4(lo, l);
  transpose4(hi, h);
  w[0] = h[3];  // top byte: c_0 in two's complement
  w[1] = h[2] ^ 0x80808080u;
  w[2] = h[1] ^ 0x80808080u;
  w[3] = h[0] ^ 0x80808080u;
  w[4] = l[3] ^ 0x80808080u;
  w[5] = l[2] ^ 0x80808080u;
  w[6] = l[1] ^ 0x80808080u;
  w[7] = l[0] ^ 0x80808080u;
}

// Four data values and their scale -> their digit words.
__host__ __device__ inline void slice4_data(double x0, double x1, double x2, double x3, double sc,
                                            uint32_t (&w)[kDigitsData])
{
  const unsigned long long y[4] = {data_word(x0, sc), data_word(x1, sc), data_word(x2, sc), data_word(x3, sc)};
  digit_words_data({(uint32_t)y[0], (uint32_t)y[1], (uint32_t)y[2], (uint32_t)y[3]},
                   {(uint32_t)(y[0] >> 32), (uint32_t)(y[1] >> 32), (uint32_t)(y[2] >> 32), (uint32_t)(y[3] >> 32)}, w);
}

// Table digits of one value (scale 2^(54-e)): c_s in d[s].
__host__ __device__ inline void digits_table(double x, double sc, int8_t (&d)[kDigitsTable])
{
  const unsigned long long Y = (unsigned long long)(d2ll(x * sc) + kOffset7);
#pragma unroll
  for (int s = 0; s < kDigitsTable; ++s) d[s] = (int8_t)(uint8_t)(((Y >> (8 * (kDigitsTable - 1 - s))) & 0xFF) ^ 0x80);
}

// exact int32 -> double with one integer and one FP64 operation
__host__ __device__ inline double i2d(int32_t v)
{
  const uint32_t u = (uint32_t)v ^ 0x80000000u;
  return bits2d((int64_t)(((uint64_t)0x43300000u << 32) | u)) - 4503601774854144.0;  // 2^52 + 2^31
}

// sum_{L<8} A_L 256^(7-L) from the eight level sums.  For K <= 64 terms the
// pairs (A_0, A_1), ..., (A_6, A_7) combine exactly in 32 bits (with |c_0| <= 4
// in the data and <= 64 in the table: |A_0| <= 2^8 K, |A_1| <= 8704 K,
// |A_L| <= (8704 + (L - 1) 2^14) K for L = 2..6, |A_7| <= (8192 + 6 2^14) K;
// the largest pair, A_6 256 + A_7, stays below 1.5e9 at K = 64), so four
// conversions suffice.
__host__ __device__ inline double combine_levels(const int32_t (&a)[kLevels], bool k_le_64)
{
  static_assert(kLevels == 8, "level pairing below assumes eight levels");
  if (k_le_64) {
    const int32_t h1 = a[0] * 256 + a[1], h2 = a[2] * 256 + a[3], h3 = a[4] * 256 + a[5], h4 = a[6] * 256 + a[7];
    return fma(fma(fma(i2d(h1), 65536.0, i2d(h2)), 65536.0, i2d(h3)), 65536.0, i2d(h4));
  }
  double d = i2d(a[0]);
#pragma unroll
  for (int L = 1; L < kLevels; ++L) d = fma(d, 256.0, i2d(a[L]));
  return d;
}

}  // namespace i8
}  // namespace sht
