// fp64_peak.cu -- FP64 throughput probe of the current device, the roofline
// denominator of the FP64 Legendre contraction in the benchmark (the measured
// peaks of the GPU pool cover HBM copy bandwidth and BF16 GEMM only).  It is a
// measurement aid loaded by bench.py, not part of the transform library.
// Two dependency-free loops: DFMA on the CUDA cores and mma.sync.m8n8k4.f64
// on the FP64 tensor path, timed with CUDA events on a private stream.
#include <cuda_runtime.h>

namespace {

__global__ void k_probe_dfma(double *out, int iters, double a, double b)
{
  double x[8];
#pragma unroll
  for (int k = 0; k < 8; ++k) x[k] = threadIdx.x + k;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int r = 0; r < 16; ++r)
#pragma unroll
      for (int k = 0; k < 8; ++k) x[k] = fma(x[k], a, b);
  }
  double s = 0.0;
#pragma unroll
  for (int k = 0; k < 8; ++k) s += x[k];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

__global__ void k_probe_dmma(double *out, int iters)
{
  const double a = threadIdx.x * 1e-3, b = threadIdx.x * 2e-3;
  double c[8][2];
#pragma unroll
  for (int t = 0; t < 8; ++t) c[t][0] = c[t][1] = 0.0;
  for (int i = 0; i < iters; ++i) {
#pragma unroll
    for (int t = 0; t < 8; ++t)
      asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
                   : "+d"(c[t][0]), "+d"(c[t][1])
                   : "d"(a), "d"(b));
  }
  double s = 0.0;
#pragma unroll
  for (int t = 0; t < 8; ++t) s += c[t][0] + c[t][1];
  out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Best of three timed runs of each loop, in TFLOP/s; 0 or a cudaError_t code.
extern "C" __attribute__((visibility("default"))) int fp64_peak_tflops(double *tflops_dfma, double *tflops_dmma)
{
  int dev = 0, sms = 0;
  cudaError_t e;
  if ((e = cudaGetDevice(&dev)) != cudaSuccess) return (int)e;
  if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return (int)e;
  const int blocks = sms * 4, threads = 256, iters = 4096;
  double *out = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  int rc = 0;
  if ((e = cudaMalloc(&out, sizeof(double) * blocks * threads)) != cudaSuccess) return (int)e;
  if ((e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) != cudaSuccess ||
      (e = cudaEventCreate(&e0)) != cudaSuccess || (e = cudaEventCreate(&e1)) != cudaSuccess) {
    rc = (int)e;
  }
  double best_f = 0.0, best_m = 0.0;
  for (int rep = 0; rep < 3 && !rc; ++rep) {
    float ms = 0.f;
    k_probe_dfma<<<blocks, threads, 0, s>>>(out, iters / 4, 0.999, 1e-3);
    cudaEventRecord(e0, s);
    k_probe_dfma<<<blocks, threads, 0, s>>>(out, iters, 0.999, 1e-3);
    cudaEventRecord(e1, s);
    if ((e = cudaEventSynchronize(e1)) != cudaSuccess) { rc = (int)e; break; }
    cudaEventElapsedTime(&ms, e0, e1);
    const double f1 = 2.0 * 8 * 16 * (double)iters * blocks * threads / (ms * 1e-3) / 1e12;
    k_probe_dmma<<<blocks, threads, 0, s>>>(out, iters / 4);
    cudaEventRecord(e0, s);
    k_probe_dmma<<<blocks, threads, 0, s>>>(out, iters);
    cudaEventRecord(e1, s);
    if ((e = cudaEventSynchronize(e1)) != cudaSuccess) { rc = (int)e; break; }
    cudaEventElapsedTime(&ms, e0, e1);
    const double f2 = 2.0 * 256 * 8 * (double)iters * blocks * (threads / 32) / (ms * 1e-3) / 1e12;
    if (f1 > best_f) best_f = f1;
    if (f2 > best_m) best_m = f2;
  }
  if (tflops_dfma) *tflops_dfma = best_f;
  if (tflops_dmma) *tflops_dmma = best_m;
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  if (s) cudaStreamDestroy(s);
  cudaFree(out);
  return rc;
}
