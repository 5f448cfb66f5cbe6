// sht_legendre_tc.cu -- split-precision Legendre contraction on tcgen05 (placeholder).
#include "sht_internal.h"

namespace sht {

int launch_leg_fwd_split(sht_plan *p, const double2 *F, int ncol, double2 *S, cudaStream_t s)
{
  (void)p; (void)F; (void)ncol; (void)S; (void)s;
  set_error("split precision: not available in this build");
  return SHT_ERR_UNSUPPORTED_SIZE;
}

int launch_leg_inv_split(sht_plan *p, const double2 *S, int ncol, double2 *F, cudaStream_t s)
{
  (void)p; (void)S; (void)ncol; (void)F; (void)s;
  set_error("split precision: not available in this build");
  return SHT_ERR_UNSUPPORTED_SIZE;
}

void free_split_tables(sht_plan *p) { (void)p; }

}  // namespace sht
