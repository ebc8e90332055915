// Measured FMA throughput of the device (FP64 and FP32): the denominator of
// the ALU roofline that bench.py reports for the cell kernels.  Every thread
// runs 8 independent FMA chains; the rate is timed with CUDA events.
//
// This is a measurement aid of the benchmark, built as its own library
// (libfma_probe.so); it is not part of the operator's C ABI.
#include <cuda_runtime.h>

namespace
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
  cudaError_t probe(double *tflops, cudaStream_t s)
  {
    int         dev = 0, sms = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e == cudaSuccess)
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess)
      return e;
    R *out = nullptr;
    if ((e = cudaMalloc(&out, sizeof(R))) != cudaSuccess)
      return e;
    const int   blocks = sms * 8, threads = 256, iters = 1 << 14;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    fma_probe_kernel<R><<<blocks, threads, 0, s>>>(iters / 8, R(0.999999), R(1e-7), out); // warm-up
    cudaEventRecord(e0, s);
    fma_probe_kernel<R><<<blocks, threads, 0, s>>>(iters, R(0.999999), R(1e-7), out);
    cudaEventRecord(e1, s);
    e = cudaEventSynchronize(e1);
    float ms = 0.f;
    if (e == cudaSuccess)
      e = cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(out);
    if (e != cudaSuccess)
      return e;
    const double flops = 2.0 * 8.0 * double(iters) * double(blocks) * threads;
    *tflops            = flops / (double(ms) * 1e-3) / 1e12;
    return cudaSuccess;
  }
} // namespace

// FMA throughput of the current device in TFLOP/s (precision 64 or 32).
// Synchronous.  Returns a cudaError_t code (0 = success).
extern "C" int fma_probe_tflops(int precision, double *tflops, void *stream)
{
  if (!tflops || (precision != 32 && precision != 64))
    return int(cudaErrorInvalidValue);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  return int(precision == 64 ? probe<double>(tflops, s) : probe<float>(tflops, s));
}
