// sht_l2.cuh -- L2 residency of the Fourier array between the longitude
// transform and the Legendre contraction.
//
// Each direction writes the Fourier array (84 MB at T85 with 480 field-levels)
// in one kernel and reads every 128-byte line of it exactly once in the next.
// The writer marks its stores evict_last, so that the grid rows streamed
// through L2 with evict-first loads do not push them out first, and the
// reader drops each line with discard.global.L2 once its copy in shared
// memory is complete, so that a line read from L2 is never written back to
// DRAM.  Both are hints about cache state only: the values read are the values
// written either way.
#pragma once

#include <cstdint>

namespace sht {
namespace l2 {

__device__ __forceinline__ uint64_t keep_policy()
{
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;\n" : "=l"(p));
  return p;
}

__device__ __forceinline__ void st_keep(double2 *ptr, double2 v, uint64_t policy)
{
  asm volatile("st.global.L2::cache_hint.v2.f64 [%0], {%1, %2}, %3;\n" ::"l"(ptr), "d"(v.x), "d"(v.y), "l"(policy)
               : "memory");
}

// ptr: a 128-byte aligned line that no later kernel reads
__device__ __forceinline__ void discard_line(const void *ptr)
{
  asm volatile("discard.global.L2 [%0], 128;\n" ::"l"(ptr) : "memory");
}

}  // namespace l2
}  // namespace sht
