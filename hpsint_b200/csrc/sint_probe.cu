// Measured FMA throughput of the device (FP64 and FP32), the denominator of
// the ALU roofline of the cell kernels: every thread runs 8 independent FMA
// chains; the rate is timed with CUDA events.
#include <string>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  template <typename R>
  __global__ void __launch_bounds__(256) fma_probe_kernel(int iters, R a, R b, R *out)
  {
    R x[8];
#pragma unroll
    for (int k = 0; k < 8; ++k)
      x[k] = R(threadIdx.x + k) * R(1e-3);
    for (int it = 0; it < iters; ++it)
      {
#pragma unroll
        for (int k = 0; k < 8; ++k)
          x[k] = x[k] * a + b;
      }
    R s = R(0);
#pragma unroll
    for (int k = 0; k < 8; ++k)
      s += x[k];
    if (s == R(12345.678)) // never true; keeps the chains alive
      out[0] = s;
  }

  template <typename R>
  static int probe(double *tflops, cudaStream_t s)
  {
    int dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
      return cuda_fail(e, "fma probe: device query");
    R *out = nullptr;
    if ((e = cudaMalloc(&out, sizeof(R))) != cudaSuccess)
      return cuda_fail(e, "fma probe: alloc");
    const int    blocks = sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t  e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_probe_kernel<R><<<blocks, threads, 0, s>>>(iters / 8, R(0.999999), R(1e-7), out); // warm-up
    cudaEventRecord(e0, s);
    fma_probe_kernel<R><<<blocks, threads, 0, s>>>(iters, R(0.999999), R(1e-7), out);
    cudaEventRecord(e1, s);
    count_launches(2);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess)
      e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess)
      return cuda_fail(e, "fma probe: timing");
    const double flops = 2.0 * 8.0 * double(iters) * double(blocks) * threads;
    *tflops            = flops / (double(ms) * 1e-3) / 1e12;
    return SINT_OK;
  }
} // namespace sint

extern "C" int sint_device_fma_peak(int precision, double *tflops, sint_stream_t stream)
{
  if (!tflops || (precision != 32 && precision != 64))
    {
      sint::set_error("sint_device_fma_peak: precision must be 32 or 64 and tflops non-null");
      return SINT_ERR_ARG;
    }
  return precision == 64 ? sint::probe<double>(tflops, stream) : sint::probe<float>(tflops, stream);
}
