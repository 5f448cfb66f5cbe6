// sht_dmma.cuh -- helpers shared by the FP64 tensor-path Legendre kernels:
// 16-byte cp.async copies (zero-filling when the source is out of range) and
// the FP64 mma.sync.m8n8k4 fragment product.
#pragma once

namespace sht {
namespace dmma {

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void cp16(void *dst, const void *src, bool valid)
{
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem_u32(dst)), "l"(src),
               "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
__device__ __forceinline__ void cp_wait1() { asm volatile("cp.async.wait_group 1;\n" ::); }
__device__ __forceinline__ void cp_wait0() { asm volatile("cp.async.wait_group 0;\n" ::); }

// d (8x8 FP64 tile, two values per lane) += a (8x4, one per lane) * b (4x8, one per lane)
__device__ __forceinline__ void mma884(double (&d)[2], double a, double b)
{
  // no side effects beyond d: left non-volatile so that the compiler may
  // schedule fragment loads across the products
  asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
      : "+d"(d[0]), "+d"(d[1])
      : "d"(a), "d"(b));
}

}  // namespace dmma
}  // namespace sht
