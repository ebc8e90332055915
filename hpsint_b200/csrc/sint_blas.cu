// BLAS-1 on block vectors (DynamicBlockVector, lac/dynamic_block_vector.h:346-516)
// and the fused multi-vector kernels used by GMRES's Gram-Schmidt step.
// Reductions are deterministic: a fixed grid of NB_RED blocks writes block
// partials in FP64, one block sums them in a fixed tree order.
#include <string>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  constexpr int RED_THREADS = 256;

  __device__ __forceinline__ double warp_sum(double v)
  {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
  }

  // Block-wide sum of one value per thread (RED_THREADS threads); result valid in thread 0.
  __device__ __forceinline__ double block_sum(double v, double *s_w)
  {
    v              = warp_sum(v);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (lane == 0)
      s_w[wid] = v;
    __syncthreads();
    double r = 0.0;
    if (wid == 0)
      {
        r = lane < RED_THREADS / 32 ? s_w[lane] : 0.0;
        r = warp_sum(r);
      }
    __syncthreads();
    return r;
  }

  // partial[j * NB_RED + blockIdx.x] = sum over this block's slice of w . V_j
  template <typename R, int M>
  __global__ void __launch_bounds__(RED_THREADS)
    multidot_kernel(long long n, const R *__restrict__ w, const R *__restrict__ V, long long stride, int m,
                    double *__restrict__ partial)
  {
    __shared__ double s_w[RED_THREADS / 32];
    double            acc[M];
#pragma unroll
    for (int j = 0; j < M; ++j)
      acc[j] = 0.0;
    for (long long i = (long long)blockIdx.x * RED_THREADS + threadIdx.x; i < n; i += (long long)NB_RED * RED_THREADS)
      {
        const double wi = double(w[i]);
#pragma unroll
        for (int j = 0; j < M; ++j)
          if (j < m)
            acc[j] += wi * double(V[j * stride + i]);
      }
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (j < m)
        {
          const double s = block_sum(acc[j], s_w);
          if (threadIdx.x == 0)
            partial[j * NB_RED + blockIdx.x] = s;
        }
  }

  // out[j] = sum_b partial[j * NB_RED + b] (one block per j, fixed order)
  __global__ void __launch_bounds__(RED_THREADS) finish_kernel(const double *__restrict__ partial, double *__restrict__ out)
  {
    __shared__ double s_w[RED_THREADS / 32];
    double            v = 0.0;
    for (int b = threadIdx.x; b < NB_RED; b += RED_THREADS)
      v += partial[blockIdx.x * NB_RED + b];
    v = block_sum(v, s_w);
    if (threadIdx.x == 0)
      out[blockIdx.x] = v;
  }

  template <typename R>
  static int launch_multidot(Ctx *c, long long n, const R *w, const R *V, long long stride, int m, double *out,
                             cudaStream_t s)
  {
    if (m < 1 || m > MAX_MULTIDOT)
      {
        set_error("multidot: m out of range");
        return SINT_ERR_ARG;
      }
    for (int j0 = 0; j0 < m; j0 += 8)
      {
        const int mm = m - j0 < 8 ? m - j0 : 8;
        // one pass per 8 vectors keeps the accumulators in registers
        multidot_kernel<R, 8><<<NB_RED, RED_THREADS, 0, s>>>(n, w, V + j0 * stride, stride, mm,
                                                             c->red + (size_t)j0 * NB_RED);
        count_launches(1);
      }
    finish_kernel<<<m, RED_THREADS, 0, s>>>(c->red, out);
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "multidot");
  }

  template <typename R>
  int multidot(Ctx *c, long long n, const R *w, const R *V, long long stride, int m, double *out, cudaStream_t s)
  {
    return launch_multidot<R>(c, n, w, V, stride, m, out, s);
  }
  template int multidot<double>(Ctx *, long long, const double *, const double *, long long, int, double *,
                                cudaStream_t);
  template int multidot<float>(Ctx *, long long, const float *, const float *, long long, int, double *,
                               cudaStream_t);

  int dot_f64(Ctx *c, long long n, const double *x, const double *y, double *out, cudaStream_t s)
  {
    return launch_multidot<double>(c, n, x, y, 0, 1, out, s);
  }
  int dot_f32(Ctx *c, long long n, const float *x, const float *y, double *out, cudaStream_t s)
  {
    return launch_multidot<float>(c, n, x, y, 0, 1, out, s);
  }

  // w -= sum_j coef[j] V_j
  template <typename R, int M>
  __global__ void __launch_bounds__(256) multiaxpy_kernel(long long n, R *__restrict__ w, const R *__restrict__ V,
                                                          long long stride, int m, const double *__restrict__ coef)
  {
    __shared__ R s_c[M];
    if (threadIdx.x < M)
      s_c[threadIdx.x] = threadIdx.x < m ? R(coef[threadIdx.x]) : R(0);
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        R acc = w[i];
#pragma unroll
        for (int j = 0; j < M; ++j)
          if (j < m)
            acc -= s_c[j] * V[j * stride + i];
        w[i] = acc;
      }
  }

  template <typename R>
  int multiaxpy(long long n, R *w, const R *V, long long stride, int m, const double *coef, cudaStream_t s)
  {
    for (int j0 = 0; j0 < m; j0 += 8)
      {
        const int mm = m - j0 < 8 ? m - j0 : 8;
        multiaxpy_kernel<R, 8><<<1184, 256, 0, s>>>(n, w, V + j0 * stride, stride, mm, coef + j0);
        count_launches(1);
      }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "multiaxpy");
  }
  template int multiaxpy<double>(long long, double *, const double *, long long, int, const double *, cudaStream_t);
  template int multiaxpy<float>(long long, float *, const float *, long long, int, const double *, cudaStream_t);

  // y += sum_j coef[j] V_j
  template <typename R, int M>
  __global__ void __launch_bounds__(256) lincomb_kernel(long long n, R *__restrict__ y, const R *__restrict__ V,
                                                        long long stride, int m, const double *__restrict__ coef)
  {
    __shared__ R s_c[M];
    if (threadIdx.x < M)
      s_c[threadIdx.x] = threadIdx.x < m ? R(coef[threadIdx.x]) : R(0);
    __syncthreads();
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        R acc = y[i];
#pragma unroll
        for (int j = 0; j < M; ++j)
          if (j < m)
            acc += s_c[j] * V[j * stride + i];
        y[i] = acc;
      }
  }

  template <typename R>
  int lincomb(long long n, R *y, const R *V, long long stride, int m, const double *coef, cudaStream_t s)
  {
    for (int j0 = 0; j0 < m; j0 += 8)
      {
        const int mm = m - j0 < 8 ? m - j0 : 8;
        lincomb_kernel<R, 8><<<1184, 256, 0, s>>>(n, y, V + j0 * stride, stride, mm, coef + j0);
        count_launches(1);
      }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "lincomb");
  }
  template int lincomb<double>(long long, double *, const double *, long long, int, const double *, cudaStream_t);
  template int lincomb<float>(long long, float *, const float *, long long, int, const double *, cudaStream_t);

  template <typename R>
  __global__ void axpby_kernel(long long n, R a, const R *__restrict__ x, R b, R *__restrict__ y)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      y[i] = (b == R(0) ? R(0) : b * y[i]) + (a == R(0) ? R(0) : a * x[i]);
  }

  template <typename R>
  int axpby(long long n, double a, const R *x, double b, R *y, cudaStream_t s)
  {
    axpby_kernel<R><<<1184, 256, 0, s>>>(n, R(a), x, R(b), y);
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "axpby");
  }
  template int axpby<double>(long long, double, const double *, double, double *, cudaStream_t);
  template int axpby<float>(long long, double, const float *, double, float *, cudaStream_t);

  template <typename S, typename D>
  __global__ void convert_kernel(long long n, const S *__restrict__ x, D *__restrict__ y)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      y[i] = D(x[i]);
  }

  template <typename S, typename D>
  int convert(long long n, const S *x, D *y, cudaStream_t s)
  {
    convert_kernel<S, D><<<1184, 256, 0, s>>>(n, x, y);
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "convert");
  }
  template int convert<double, float>(long long, const double *, float *, cudaStream_t);
  template int convert<float, double>(long long, const float *, double *, cudaStream_t);

  __global__ void sqrt_kernel(double *x) { x[0] = sqrt(x[0]); }
} // namespace sint

using namespace sint;

static int check_ptrs(const void *a, const void *b, int64_t n)
{
  if (n < 0 || (n > 0 && (!a || !b)))
    {
      set_error("BLAS-1: null pointer or negative size");
      return SINT_ERR_ARG;
    }
  return SINT_OK;
}

extern "C" {

int sint_vec_axpy_f64(int64_t n, double a, const double *x, double *y, sint_stream_t s)
{
  if (int e = check_ptrs(x, y, n))
    return e;
  return n ? axpby<double>(n, a, x, 1.0, y, s) : SINT_OK;
}

int sint_vec_sadd_f64(int64_t n, double sc, double a, const double *x, double *y, sint_stream_t s)
{
  if (int e = check_ptrs(x, y, n))
    return e;
  return n ? axpby<double>(n, a, x, sc, y, s) : SINT_OK;
}

int sint_vec_scale_f64(int64_t n, double a, double *x, sint_stream_t s)
{
  if (int e = check_ptrs(x, x, n))
    return e;
  return n ? axpby<double>(n, 0.0, x, a, x, s) : SINT_OK;
}

int sint_vec_axpy_f32(int64_t n, float a, const float *x, float *y, sint_stream_t s)
{
  if (int e = check_ptrs(x, y, n))
    return e;
  return n ? axpby<float>(n, a, x, 1.0, y, s) : SINT_OK;
}

int sint_vec_dot_f64(sint_ctx *c, int64_t n, const double *x, const double *y, double *result, sint_stream_t s)
{
  if (!c || !result)
    {
      set_error("sint_vec_dot_f64: null context or result");
      return SINT_ERR_ARG;
    }
  if (int e = check_ptrs(x, y, n))
    return e;
  return dot_f64(c, n, x, y, result, s);
}

int sint_vec_norm2_f64(sint_ctx *c, int64_t n, const double *x, double *result, sint_stream_t s)
{
  if (!c || !result)
    {
      set_error("sint_vec_norm2_f64: null context or result");
      return SINT_ERR_ARG;
    }
  if (int e = check_ptrs(x, x, n))
    return e;
  if (int e = dot_f64(c, n, x, x, result, s))
    return e;
  sqrt_kernel<<<1, 1, 0, s>>>(result);
  count_launches(1);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_vec_norm2_f64");
}

int sint_vec_dot_f32(sint_ctx *c, int64_t n, const float *x, const float *y, double *result, sint_stream_t s)
{
  if (!c || !result)
    {
      set_error("sint_vec_dot_f32: null context or result");
      return SINT_ERR_ARG;
    }
  if (int e = check_ptrs(x, y, n))
    return e;
  return dot_f32(c, n, x, y, result, s);
}

int sint_vec_norm2_f32(sint_ctx *c, int64_t n, const float *x, double *result, sint_stream_t s)
{
  if (!c || !result)
    {
      set_error("sint_vec_norm2_f32: null context or result");
      return SINT_ERR_ARG;
    }
  if (int e = check_ptrs(x, x, n))
    return e;
  if (int e = dot_f32(c, n, x, x, result, s))
    return e;
  sqrt_kernel<<<1, 1, 0, s>>>(result);
  count_launches(1);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_vec_norm2_f32");
}

int sint_vec_f64_to_f32(int64_t n, const double *x, float *y, sint_stream_t s)
{
  if (int e = check_ptrs(x, y, n))
    return e;
  return n ? convert<double, float>(n, x, y, s) : SINT_OK;
}

int sint_vec_f32_to_f64(int64_t n, const float *x, double *y, sint_stream_t s)
{
  if (int e = check_ptrs(x, y, n))
    return e;
  return n ? convert<float, double>(n, x, y, s) : SINT_OK;
}

} // extern "C"
