// sht_noalloc.cu -- grid -> spectral analysis that allocates no device memory.
//
// Who needs this: hosts that must not allocate device memory while they run
// their time loop.  One example is a model whose device memory is reserved up
// front by another allocator, such as a caching pool that owns the GPU, where
// a cudaMalloc would fail or fragment that pool.  Another is a caller that
// cannot afford the implicit device-wide synchronisation cudaMalloc/cudaFree
// can perform in the middle of a timestep.  Another is a host whose policy
// forbids allocation after start-up.  For them, sht_wa_xya_dev_noalloc runs
// the batched kernels of sht_wa_xya_dev (longitude transform, contraction,
// spectral conversion; at im = 32, where sht_wa_xya_dev takes its single
// fused kernel instead, the two agree to rounding).  Its intermediate Fourier
// and spectral arrays live in one fixed, file-scope device array instead of
// the plan's growable workspace.  The plan itself (Gauss and Legendre tables) is still
// built by sht_init beforehand.
//
// Rules a user must know:
//   * The scratch array is SHT_NOALLOC_SCRATCH_BYTES (32 MiB) and is held by
//     every GPU that loads this library until the process exits.  A batch
//     that needs more is rejected with SHT_ERR_TOO_LARGE before any work.
//   * All calls share the one array, and it keeps whatever the last call left
//     in it.  Nothing in it needs to start at zero: each call writes every
//     scratch element before reading it.
//   * Calls that overlap on the GPU (for example two streams, or two plans,
//     running this entry point at the same time) race on the array.  Order
//     them on one stream or finish one before starting the next.
//   * The first call on a device looks up the array's device address with
//     cudaGetSymbolAddress (once per device, with that device current).  Make
//     that first call before any stream capture begins.
//   * In split precision the plan's digit tables must exist already: the first
//     split-precision call of an ordinary entry point allocates them.  Until
//     then this entry point refuses (SHT_ERR_INVALID_ARG) instead of allocating.
#include "sht_internal.h"

#include <cstdio>

#define SHT_NOALLOC_SCRATCH_BYTES (32ull << 20)

namespace {

static __device__ __align__(256) unsigned char g_noalloc_scratch[SHT_NOALLOC_SCRATCH_BYTES];

// Device address of the scratch array on the plan's device (which must be
// current).  The address is kept in the plan, so a plan created after a
// device reset looks it up again.
int scratch_address(sht_plan *p, void **out)
{
  if (!p->noalloc_scratch) {
    void *ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
    if (e != cudaSuccess) return sht::cuda_fail(e, "noalloc: cudaGetSymbolAddress(scratch)");
    p->noalloc_scratch = ptr;
  }
  *out = p->noalloc_scratch;
  return SHT_OK;
}

size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace

extern "C" SHT_API unsigned long long sht_noalloc_scratch_bytes(void) { return SHT_NOALLOC_SCRATCH_BYTES; }

extern "C" SHT_API int sht_wa_xya_dev_noalloc(sht_plan *p, const double *xya, int nb, double *wa)
{
  using namespace sht;
  if (!p || p->magic != kPlanMagic) {
    set_error("noalloc: plan is not initialised");
    return SHT_ERR_NOT_INITIALIZED;
  }
  if (nb < 0 || (nb > 0 && (!xya || !wa))) {
    set_error("noalloc: bad argument");
    return SHT_ERR_INVALID_ARG;
  }
  if (nb > 0 && (reinterpret_cast<uintptr_t>(xya) & 15u) != 0) {
    set_error("noalloc: device grid arrays must be 16-byte aligned");
    return SHT_ERR_INVALID_ARG;
  }
  const size_t fbytes = align256(sizeof(double2) * (size_t)(p->N + 1) * nb * p->J);
  const size_t sbytes = align256(sizeof(double2) * (size_t)p->R * nb);
  if (fbytes + sbytes > SHT_NOALLOC_SCRATCH_BYTES) {
    const size_t per = align256(sizeof(double2) * (size_t)(p->N + 1) * p->J) + sizeof(double2) * (size_t)p->R;
    char buf[256];
    snprintf(buf, sizeof(buf),
             "noalloc: %d field-levels need %zu bytes of scratch; the fixed limit is %llu bytes "
             "(at most about %zu field-levels per call on this grid)",
             nb, fbytes + sbytes, SHT_NOALLOC_SCRATCH_BYTES, (size_t)(SHT_NOALLOC_SCRATCH_BYTES / per));
    set_error(buf);
    return SHT_ERR_TOO_LARGE;
  }
  std::lock_guard<std::mutex> lk(p->mtx);
  if (use_split(p, true) && !p->tc_tables) {
    // the split kernel's digit tables are allocated by the first split-precision
    // transform of a plan; this entry point must not be the one to do it
    set_error("noalloc: split precision needs the plan's digit tables, which the first split-precision "
              "call of an ordinary entry point allocates; make one such call first, or use FP64");
    return SHT_ERR_INVALID_ARG;
  }
  int prev = -1;
  cudaGetDevice(&prev);
  if (prev != p->device && cudaSetDevice(p->device) != cudaSuccess) {
    set_error("noalloc: cudaSetDevice failed");
    return SHT_ERR_CUDA;
  }
  void *base = nullptr;
  int rc = scratch_address(p, &base);
  if (!rc && nb > 0) {
    double2 *F = static_cast<double2 *>(base);
    double2 *S = reinterpret_cast<double2 *>(static_cast<char *>(base) + fbytes);
    cudaStream_t s = p->stream;
    rc = launch_fft_fwd(p, xya, nullptr, nb, nb, F, nb, 0, RS_FWD_PLAIN, s);
    if (!rc) rc = use_split(p, true) ? launch_leg_fwd_split(p, F, nb, S, s)
                                                   : launch_leg_fwd_fp64(p, F, nb, S, s);
    if (!rc) rc = launch_pack(p, PACK_PLAIN, S, nb, nb, wa, nullptr, s);
  }
  if (prev >= 0 && prev != p->device) cudaSetDevice(prev);
  return rc;
}
