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

  // --- 16-byte packs ---------------------------------------------------------
  // The Krylov kernels move 16 bytes per load (2 doubles or 4 floats) when
  // every pointer is 16-byte aligned and n, stride are multiples of the pack;
  // otherwise one element per load (E = 1).  Block vectors of a context
  // always qualify: ld is a multiple of 32.
  template <typename R, int E>
  struct Pack
  {
    R v[E];
  };

  template <typename R, int E>
  __device__ __forceinline__ Pack<R, E> ld_pack(const R *__restrict__ p, long long c)
  {
    Pack<R, E> x;
    if constexpr (E * sizeof(R) == 16 && sizeof(R) == 8)
      {
        const double2 t = reinterpret_cast<const double2 *>(p)[c];
        x.v[0] = t.x, x.v[1] = t.y;
      }
    else if constexpr (E * sizeof(R) == 16 && sizeof(R) == 4)
      {
        const float4 t = reinterpret_cast<const float4 *>(p)[c];
        x.v[0] = t.x, x.v[1] = t.y, x.v[2] = t.z, x.v[3] = t.w;
      }
    else
      {
#pragma unroll
        for (int e = 0; e < E; ++e)
          x.v[e] = p[c * E + e];
      }
    return x;
  }

  template <typename R, int E>
  __device__ __forceinline__ void st_pack(R *__restrict__ p, long long c, const Pack<R, E> &x)
  {
    if constexpr (E * sizeof(R) == 16 && sizeof(R) == 8)
      reinterpret_cast<double2 *>(p)[c] = make_double2(x.v[0], x.v[1]);
    else if constexpr (E * sizeof(R) == 16 && sizeof(R) == 4)
      reinterpret_cast<float4 *>(p)[c] = make_float4(x.v[0], x.v[1], x.v[2], x.v[3]);
    else
      {
#pragma unroll
        for (int e = 0; e < E; ++e)
          p[c * E + e] = x.v[e];
      }
  }

  template <typename R>
  constexpr int pack_of()
  {
    return 16 / int(sizeof(R));
  }

  inline bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15u) == 0; }

  // Live chunks (grain cut-off): bit k of live is clear when elements
  // [k * LIVE_CHUNK, (k + 1) * LIVE_CHUNK) of every Krylov vector are known
  // to be zero; nullptr = all live.  A warp's packs never straddle a chunk.
  __device__ __forceinline__ bool chunk_live(const uint32_t *__restrict__ live, long long elem)
  {
    if (!live)
      return true;
    const long long k = elem / LIVE_CHUNK;
    return (live[k >> 5] >> (k & 31)) & 1u;
  }

  template <typename R>
  inline bool can_pack(long long n, long long stride, const void *a, const void *b)
  {
    constexpr int E = pack_of<R>();
    return n % E == 0 && stride % E == 0 && aligned16(a) && aligned16(b);
  }

  // Fused finish of a reduction: every block has written its partials
  // (rows 0..m-1, NB_RED blocks each); the block that takes the last ticket
  // sums each row in a fixed order (lane l adds blocks l, l + 32, ..., then a
  // fixed butterfly), writes out[0..m) and resets the ticket.  The result does
  // not depend on which block finishes last.
  __device__ __forceinline__ void finish_if_last(const double *__restrict__ rows, int m, double *__restrict__ out,
                                                 unsigned *ticket)
  {
    __shared__ bool last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
      last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    __syncthreads();
    if (!last)
      return;
    __threadfence();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    for (int j = warp; j < m; j += RED_THREADS / 32)
      {
        double v = 0.0;
        for (int b = lane; b < NB_RED; b += 32)
          v += __ldcg(rows + (size_t)j * NB_RED + b);
        v = warp_sum(v);
        if (lane == 0)
          out[j] = v;
      }
    if (threadIdx.x == 0)
      *ticket = 0u;
  }

  // partial[j * NB_RED + blockIdx.x] = sum over this block's chunks of w . V_j
  // (FP64 products and sums; m <= M).
  template <typename R, int M, int E>
  __global__ void __launch_bounds__(RED_THREADS)
    multidot_kernel(long long nc, const R *__restrict__ w, const R *__restrict__ V, long long stride, int m,
                    double *__restrict__ partial, const int *__restrict__ cond, const double *__restrict__ rows,
                    int m_total, double *__restrict__ out, unsigned *ticket, const uint32_t *__restrict__ live)
  {
    if (cond && *cond == 0)
      return;
    __shared__ double s_w[RED_THREADS / 32];
    double            acc[M];
#pragma unroll
    for (int j = 0; j < M; ++j)
      acc[j] = 0.0;
    for (long long c = (long long)blockIdx.x * RED_THREADS + threadIdx.x; c < nc; c += (long long)NB_RED * RED_THREADS)
      {
        if (!chunk_live(live, c * E))
          continue;
        const Pack<R, E> wi = ld_pack<R, E>(w, c);
#pragma unroll
        for (int j = 0; j < M; ++j)
          if (j < m)
            {
              const Pack<R, E> vj = ld_pack<R, E>(V + j * stride, c);
#pragma unroll
              for (int e = 0; e < E; ++e)
                acc[j] += double(wi.v[e]) * double(vj.v[e]);
            }
      }
#pragma unroll
    for (int j = 0; j < M; ++j)
      if (j < m)
        {
          const double s = block_sum(acc[j], s_w);
          if (threadIdx.x == 0)
            partial[j * NB_RED + blockIdx.x] = s;
        }
    if (out)
      finish_if_last(rows, m_total, out, ticket);
  }

  constexpr int MD = 16; // vectors per multidot / multiaxpy pass (accumulators in registers)

  template <typename R>
  static int launch_multidot(Ctx *c, long long n, const R *w, const R *V, long long stride, int m, double *out,
                             cudaStream_t s, const int *cond = nullptr, const uint32_t *live = nullptr)
  {
    if (m < 1 || m > MAX_MULTIDOT)
      {
        set_error("multidot: m out of range");
        return SINT_ERR_ARG;
      }
    constexpr int E    = pack_of<R>();
    const bool    pack = can_pack<R>(n, stride, w, V);
    for (int j0 = 0; j0 < m; j0 += MD)
      {
        const int mm   = m - j0 < MD ? m - j0 : MD;
        double   *pp   = c->red + (size_t)j0 * NB_RED;
        double   *outl = j0 + MD >= m ? out : nullptr; // the last pass sums all rows
        if (pack)
          multidot_kernel<R, MD, E><<<NB_RED, RED_THREADS, 0, s>>>(n / E, w, V + j0 * stride, stride, mm, pp, cond,
                                                                   c->red, m, outl, c->red_ticket, live);
        else
          multidot_kernel<R, MD, 1><<<NB_RED, RED_THREADS, 0, s>>>(n, w, V + j0 * stride, stride, mm, pp, cond,
                                                                   c->red, m, outl, c->red_ticket, live);
        count_launches(1);
      }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "multidot");
  }

  template <typename R>
  int multidot(Ctx *c, long long n, const R *w, const R *V, long long stride, int m, double *out, cudaStream_t s,
               const uint32_t *live)
  {
    return launch_multidot<R>(c, n, w, V, stride, m, out, s, nullptr, live);
  }
  template int multidot<double>(Ctx *, long long, const double *, const double *, long long, int, double *,
                                cudaStream_t, const uint32_t *);
  template int multidot<float>(Ctx *, long long, const float *, const float *, long long, int, double *,
                               cudaStream_t, const uint32_t *);

  template <typename R>
  int multidot_if(Ctx *c, long long n, const R *w, const R *V, long long stride, int m, double *out, const int *cond,
                  cudaStream_t s, const uint32_t *live)
  {
    return launch_multidot<R>(c, n, w, V, stride, m, out, s, cond, live);
  }
  template int multidot_if<double>(Ctx *, long long, const double *, const double *, long long, int, double *,
                                   const int *, cudaStream_t, const uint32_t *);
  template int multidot_if<float>(Ctx *, long long, const float *, const float *, long long, int, double *,
                                  const int *, cudaStream_t, const uint32_t *);

  int dot_f64(Ctx *c, long long n, const double *x, const double *y, double *out, cudaStream_t s)
  {
    return launch_multidot<double>(c, n, x, y, 0, 1, out, s);
  }
  int dot_f32(Ctx *c, long long n, const float *x, const float *y, double *out, cudaStream_t s)
  {
    return launch_multidot<float>(c, n, x, y, 0, 1, out, s);
  }

  // w -= sum_j coef[j] V_j (j < m <= M); with `partial`, also the block
  // partials of |w|^2 after the update (FP64), for the norm that follows.
  template <typename R, int M, int E>
  __global__ void __launch_bounds__(RED_THREADS)
    multiaxpy_kernel(long long nc, R *__restrict__ w, const R *__restrict__ V, long long stride, int m,
                     const double *__restrict__ coef, double *__restrict__ partial, const int *__restrict__ cond,
                     double *__restrict__ norm2_out, unsigned *ticket, const uint32_t *__restrict__ live)
  {
    if (cond && *cond == 0)
      return;
    __shared__ R      s_c[M];
    __shared__ double s_w[RED_THREADS / 32];
    if (threadIdx.x < M)
      s_c[threadIdx.x] = threadIdx.x < m ? R(coef[threadIdx.x]) : R(0);
    __syncthreads();
    double nrm = 0.0;
    for (long long c = (long long)blockIdx.x * RED_THREADS + threadIdx.x; c < nc; c += (long long)gridDim.x * RED_THREADS)
      {
        if (!chunk_live(live, c * E)) // w and every V_j are zero there: w stays zero
          continue;
        Pack<R, E> acc = ld_pack<R, E>(w, c);
#pragma unroll
        for (int j = 0; j < M; ++j)
          if (j < m)
            {
              const Pack<R, E> vj = ld_pack<R, E>(V + j * stride, c);
#pragma unroll
              for (int e = 0; e < E; ++e)
                acc.v[e] -= s_c[j] * vj.v[e];
            }
        st_pack<R, E>(w, c, acc);
        if (partial)
          {
#pragma unroll
            for (int e = 0; e < E; ++e)
              nrm += double(acc.v[e]) * double(acc.v[e]);
          }
      }
    if (partial)
      {
        const double t = block_sum(nrm, s_w);
        if (threadIdx.x == 0)
          partial[blockIdx.x] = t;
        finish_if_last(partial, 1, norm2_out, ticket);
      }
  }

  template <typename R>
  static int launch_multiaxpy(Ctx *c, long long n, R *w, const R *V, long long stride, int m, const double *coef,
                              double *norm2_out, cudaStream_t s, const int *cond = nullptr,
                              const uint32_t *live = nullptr)
  {
    constexpr int E    = pack_of<R>();
    const bool    pack = can_pack<R>(n, stride, w, V);
    for (int j0 = 0; j0 < m; j0 += MD)
      {
        const int mm   = m - j0 < MD ? m - j0 : MD;
        double   *part = (norm2_out && j0 + MD >= m) ? c->red : nullptr; // norm in the last pass
        unsigned *tk   = c ? c->red_ticket : nullptr;
        if (pack)
          multiaxpy_kernel<R, MD, E><<<NB_RED, RED_THREADS, 0, s>>>(n / E, w, V + j0 * stride, stride, mm, coef + j0,
                                                                    part, cond, norm2_out, tk, live);
        else
          multiaxpy_kernel<R, MD, 1><<<NB_RED, RED_THREADS, 0, s>>>(n, w, V + j0 * stride, stride, mm, coef + j0,
                                                                    part, cond, norm2_out, tk, live);
        count_launches(1);
      }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "multiaxpy");
  }

  template <typename R>
  int multiaxpy(long long n, R *w, const R *V, long long stride, int m, const double *coef, cudaStream_t s)
  {
    return launch_multiaxpy<R>(nullptr, n, w, V, stride, m, coef, nullptr, s);
  }
  template int multiaxpy<double>(long long, double *, const double *, long long, int, const double *, cudaStream_t);
  template int multiaxpy<float>(long long, float *, const float *, long long, int, const double *, cudaStream_t);

  template <typename R>
  int multiaxpy_norm2(Ctx *c, long long n, R *w, const R *V, long long stride, int m, const double *coef,
                      double *norm2_out, cudaStream_t s, const uint32_t *live)
  {
    return launch_multiaxpy<R>(c, n, w, V, stride, m, coef, norm2_out, s, nullptr, live);
  }
  template int multiaxpy_norm2<double>(Ctx *, long long, double *, const double *, long long, int, const double *,
                                       double *, cudaStream_t, const uint32_t *);
  template int multiaxpy_norm2<float>(Ctx *, long long, float *, const float *, long long, int, const double *,
                                      double *, cudaStream_t, const uint32_t *);

  template <typename R>
  int multiaxpy_norm2_if(Ctx *c, long long n, R *w, const R *V, long long stride, int m, const double *coef,
                         double *norm2_out, const int *cond, cudaStream_t s, const uint32_t *live)
  {
    return launch_multiaxpy<R>(c, n, w, V, stride, m, coef, norm2_out, s, cond, live);
  }
  template int multiaxpy_norm2_if<double>(Ctx *, long long, double *, const double *, long long, int, const double *,
                                          double *, const int *, cudaStream_t, const uint32_t *);
  template int multiaxpy_norm2_if<float>(Ctx *, long long, float *, const float *, long long, int, const double *,
                                         double *, const int *, cudaStream_t, const uint32_t *);

  // y += sum_j coef[j] V_j
  template <typename R, int M, int E>
  __global__ void __launch_bounds__(256) lincomb_kernel(long long nc, R *__restrict__ y, const R *__restrict__ V,
                                                        long long stride, int m, const double *__restrict__ coef,
                                                        const uint32_t *__restrict__ live)
  {
    __shared__ R s_c[M];
    if (threadIdx.x < M)
      s_c[threadIdx.x] = threadIdx.x < m ? R(coef[threadIdx.x]) : R(0);
    __syncthreads();
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x)
      {
        if (!chunk_live(live, c * E)) // y and every V_j are zero there
          continue;
        Pack<R, E> acc = ld_pack<R, E>(y, c);
#pragma unroll
        for (int j = 0; j < M; ++j)
          if (j < m)
            {
              const Pack<R, E> vj = ld_pack<R, E>(V + j * stride, c);
#pragma unroll
              for (int e = 0; e < E; ++e)
                acc.v[e] += s_c[j] * vj.v[e];
            }
        st_pack<R, E>(y, c, acc);
      }
  }

  template <typename R>
  int lincomb(long long n, R *y, const R *V, long long stride, int m, const double *coef, cudaStream_t s,
              const uint32_t *live)
  {
    constexpr int E    = pack_of<R>();
    const bool    pack = can_pack<R>(n, stride, y, V);
    for (int j0 = 0; j0 < m; j0 += MD)
      {
        const int mm = m - j0 < MD ? m - j0 : MD;
        if (pack)
          lincomb_kernel<R, MD, E><<<1184, 256, 0, s>>>(n / E, y, V + j0 * stride, stride, mm, coef + j0, live);
        else
          lincomb_kernel<R, MD, 1><<<1184, 256, 0, s>>>(n, y, V + j0 * stride, stride, mm, coef + j0, live);
        count_launches(1);
      }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "lincomb");
  }
  template int lincomb<double>(long long, double *, const double *, long long, int, const double *, cudaStream_t,
                               const uint32_t *);
  template int lincomb<float>(long long, float *, const float *, long long, int, const double *, cudaStream_t,
                              const uint32_t *);

  // y = b y + a x; a term whose factor is 0 is dropped, so NaN in an unused
  // operand does not spread.  With d_div: a = 1 / d_div[0] read on the device.
  // Chunks that are not live are written as zero without reading.
  template <typename R, int E>
  __global__ void axpby_kernel(long long nc, R a, const R *__restrict__ x, R b, R *__restrict__ y,
                               const double *__restrict__ d_div, const uint32_t *__restrict__ live)
  {
    if (d_div)
      a = R(1.0 / d_div[0]);
    for (long long c = (long long)blockIdx.x * blockDim.x + threadIdx.x; c < nc; c += (long long)gridDim.x * blockDim.x)
      {
        if (!chunk_live(live, c * E))
          {
            st_pack<R, E>(y, c, Pack<R, E>{});
            continue;
          }
        Pack<R, E> xv{}, yv{}, out;
        if (a != R(0))
          xv = ld_pack<R, E>(x, c);
        if (b != R(0))
          yv = ld_pack<R, E>(y, c);
#pragma unroll
        for (int e = 0; e < E; ++e)
          out.v[e] = (b == R(0) ? R(0) : b * yv.v[e]) + (a == R(0) ? R(0) : a * xv.v[e]);
        st_pack<R, E>(y, c, out);
      }
  }

  template <typename R>
  static int launch_axpby(long long n, double a, const R *x, double b, R *y, const double *d_div, cudaStream_t s,
                          const uint32_t *live = nullptr)
  {
    constexpr int E = pack_of<R>();
    if (can_pack<R>(n, 0, x, y))
      axpby_kernel<R, E><<<1184, 256, 0, s>>>(n / E, R(a), x, R(b), y, d_div, live);
    else
      axpby_kernel<R, 1><<<1184, 256, 0, s>>>(n, R(a), x, R(b), y, d_div, live);
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "axpby");
  }

  template <typename R>
  int axpby(long long n, double a, const R *x, double b, R *y, cudaStream_t s, const uint32_t *live)
  {
    return launch_axpby<R>(n, a, x, b, y, nullptr, s, live);
  }
  template int axpby<double>(long long, double, const double *, double, double *, cudaStream_t, const uint32_t *);
  template int axpby<float>(long long, double, const float *, double, float *, cudaStream_t, const uint32_t *);

  template <typename R>
  int scale_by_device(long long n, const R *x, const double *d_div, R *y, cudaStream_t s, const uint32_t *live)
  {
    return launch_axpby<R>(n, 1.0, x, 0.0, y, d_div, s, live);
  }
  template int scale_by_device<double>(long long, const double *, const double *, double *, cudaStream_t,
                                       const uint32_t *);
  template int scale_by_device<float>(long long, const float *, const double *, float *, cudaStream_t,
                                      const uint32_t *);

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

  __global__ void select_kernel(long long n, const double *__restrict__ a, const double *__restrict__ b,
                                const double *__restrict__ na, const double *__restrict__ nb, double *out)
  {
    const double *src = *na <= *nb ? a : b;
    if (src == out)
      return;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      out[i] = src[i];
  }
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

int sint_vec_select_f64(int64_t n, const double *a, const double *b, const double *norm_a, const double *norm_b,
                        double *out, sint_stream_t s)
{
  if (int e = check_ptrs(a, b, n))
    return e;
  if (!norm_a || !norm_b || !out)
    {
      set_error("sint_vec_select_f64: null pointer");
      return SINT_ERR_ARG;
    }
  if (n == 0)
    return SINT_OK;
  select_kernel<<<1184, 256, 0, s>>>(n, a, b, norm_a, norm_b, out);
  count_launches(1);
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_vec_select_f64");
}

int sint_vec_f32_to_f64(int64_t n, const float *x, double *y, sint_stream_t s)
{
  if (int e = check_ptrs(x, y, n))
    return e;
  return n ? convert<float, double>(n, x, y, s) : SINT_OK;
}

} // extern "C"
