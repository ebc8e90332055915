// FP32 building blocks of the learned Newton initial guess: 3x3 convolution
// (forward, data gradient via the flipped/transposed kernel, weight and bias
// gradients with deterministic two-level reduction), leaky-ReLU, sum pooling
// and broadcast over the grain streams, mean-squared error, Adam, and the
// extraction of network inputs/targets from solver states.
//
// Tensors are NCHW float32: [batch][channel][height][width]; the grain
// streams of sample b are batch entries b * G + i.
#include <cstdint>
#include <string>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  // --- 3x3 convolution, zero padding, stride 1 -----------------------------
  // Block: 16 x 16 output pixels of one batch entry, COB output channels;
  // each thread one pixel and COB accumulators.  Input tile (18 x 18) and the
  // COB x 9 weights of one input channel are staged in shared memory.
  constexpr int CT  = 16;
  constexpr int COB = 16;

  __global__ void __launch_bounds__(CT *CT)
    conv3x3_kernel(const float *__restrict__ in, int Cin, int H, int W, const float *__restrict__ w,
                   const float *__restrict__ bias, float *__restrict__ out, int Cout, int accumulate)
  {
    __shared__ float s_in[CT + 2][CT + 3];
    __shared__ float s_w[COB][9];
    const int b   = blockIdx.z;
    const int co0 = blockIdx.y * COB;
    const int tx = threadIdx.x % CT, ty = threadIdx.x / CT;
    const int tiles_x = (W + CT - 1) / CT;
    const int x0 = (blockIdx.x % tiles_x) * CT, y0 = (blockIdx.x / tiles_x) * CT;
    const int x = x0 + tx, y = y0 + ty;
    float     acc[COB];
#pragma unroll
    for (int j = 0; j < COB; ++j)
      acc[j] = 0.f;
    for (int ci = 0; ci < Cin; ++ci)
      {
        const float *src = in + ((long long)b * Cin + ci) * H * W;
        for (int i = threadIdx.x; i < (CT + 2) * (CT + 2); i += CT * CT)
          {
            const int yy = y0 - 1 + i / (CT + 2), xx = x0 - 1 + i % (CT + 2);
            s_in[i / (CT + 2)][i % (CT + 2)] = (yy >= 0 && yy < H && xx >= 0 && xx < W) ? src[yy * W + xx] : 0.f;
          }
        for (int i = threadIdx.x; i < COB * 9; i += CT * CT)
          {
            const int j = i / 9, k = i % 9;
            s_w[j][k]  = (co0 + j < Cout) ? w[((long long)(co0 + j) * Cin + ci) * 9 + k] : 0.f;
          }
        __syncthreads();
        float v[9];
#pragma unroll
        for (int k = 0; k < 9; ++k)
          v[k] = s_in[ty + k / 3][tx + k % 3];
#pragma unroll
        for (int j = 0; j < COB; ++j)
#pragma unroll
          for (int k = 0; k < 9; ++k)
            acc[j] += s_w[j][k] * v[k];
        __syncthreads();
      }
    if (x < W && y < H)
      for (int j = 0; j < COB && co0 + j < Cout; ++j)
        {
          float *o = out + (((long long)b * Cout + co0 + j) * H + y) * W + x;
          float  r = acc[j] + (bias ? bias[co0 + j] : 0.f);
          *o       = accumulate ? *o + r : r;
        }
  }

  // wT[ci][co][8 - k] = w[co][ci][k]: the data gradient of a convolution is the
  // convolution of the output gradient with this kernel.
  __global__ void conv3x3_flip_kernel(const float *__restrict__ w, int Cout, int Cin, float *__restrict__ wT)
  {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= Cout * Cin * 9)
      return;
    const int co = i / (Cin * 9), ci = (i / 9) % Cin, k = i % 9;
    wT[((long long)ci * Cout + co) * 9 + (8 - k)] = w[i];
  }

  // Weight/bias gradient, level 1: one block per (16 x 16 pixel tile, batch
  // entry) stages the output gradient [Cout][256] and the input tile with
  // halo [Cin][18 x 18] in shared memory; each thread owns up to 4 output
  // channels x 9 taps of one input channel and sums their products over the
  // tile's pixels.  partial[block][co][ci * 9 + k], partial_b[block][co].
  constexpr int WG_THREADS = 256;
  __global__ void __launch_bounds__(WG_THREADS)
    conv3x3_wgrad_kernel(const float *__restrict__ in, const float *__restrict__ dout, int Cin, int Cout, int H, int W,
                         float *__restrict__ partial, float *__restrict__ partial_b)
  {
    extern __shared__ float smem_nn[];
    float    *s_d  = smem_nn;                 // [Cout][CT * CT]
    float    *s_in = smem_nn + Cout * CT * CT; // [Cin][(CT + 2) * (CT + 2)]
    const int b       = blockIdx.y;
    const int tiles_x = (W + CT - 1) / CT;
    const int x0 = (blockIdx.x % tiles_x) * CT, y0 = (blockIdx.x / tiles_x) * CT;
    const long long blk = (long long)blockIdx.y * gridDim.x + blockIdx.x;
    for (int i = threadIdx.x; i < Cout * CT * CT; i += WG_THREADS)
      {
        const int co = i / (CT * CT), p = i % (CT * CT), y = y0 + p / CT, x = x0 + p % CT;
        s_d[i] = (y < H && x < W) ? dout[(((long long)b * Cout + co) * H + y) * W + x] : 0.f;
      }
    constexpr int HT = (CT + 2) * (CT + 2);
    for (int i = threadIdx.x; i < Cin * HT; i += WG_THREADS)
      {
        const int ci = i / HT, p = i % HT, y = y0 - 1 + p / (CT + 2), x = x0 - 1 + p % (CT + 2);
        s_in[i] = (y >= 0 && y < H && x >= 0 && x < W) ? in[(((long long)b * Cin + ci) * H + y) * W + x] : 0.f;
      }
    __syncthreads();
    const int ngrp = (Cout + 3) / 4;
    for (int item = threadIdx.x; item < ngrp * Cin; item += WG_THREADS)
      {
        const int cg = item / Cin, ci = item % Cin;
        float     acc[4][9];
#pragma unroll
        for (int j = 0; j < 4; ++j)
#pragma unroll
          for (int k = 0; k < 9; ++k)
            acc[j][k] = 0.f;
        const float *si = s_in + ci * HT;
        for (int p = 0; p < CT * CT; ++p)
          {
            const int py = p / CT, px = p % CT;
            float     v[9];
#pragma unroll
            for (int k = 0; k < 9; ++k)
              v[k] = si[(py + k / 3) * (CT + 2) + px + k % 3];
#pragma unroll
            for (int j = 0; j < 4; ++j)
              {
                const float d = (4 * cg + j < Cout) ? s_d[(4 * cg + j) * CT * CT + p] : 0.f;
#pragma unroll
                for (int k = 0; k < 9; ++k)
                  acc[j][k] += d * v[k];
              }
          }
#pragma unroll
        for (int j = 0; j < 4; ++j)
          if (4 * cg + j < Cout)
#pragma unroll
            for (int k = 0; k < 9; ++k)
              partial[(blk * Cout + 4 * cg + j) * Cin * 9 + ci * 9 + k] = acc[j][k];
      }
    if (partial_b)
      for (int co = threadIdx.x; co < Cout; co += WG_THREADS)
        {
          float s = 0.f;
          for (int p = 0; p < CT * CT; ++p)
            s += s_d[co * CT * CT + p];
          partial_b[blk * Cout + co] = s;
        }
  }

  // level 2: out[i] (+)= sum_c partial[c][i] in a fixed order
  __global__ void reduce_chunks_kernel(const float *__restrict__ partial, int chunks, long long n, float *__restrict__ out,
                                       int accumulate)
  {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n)
      return;
    float s = 0.f;
    for (int c = 0; c < chunks; ++c)
      s += partial[c * n + i];
    out[i] = accumulate ? out[i] + s : s;
  }

  __global__ void leaky_fwd_kernel(long long n, float slope, const float *__restrict__ x, float *__restrict__ y)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        const float v = x[i];
        y[i]          = v > 0.f ? v : slope * v;
      }
  }

  // dx = dy * f'(pre) (may alias dy)
  __global__ void leaky_bwd_kernel(long long n, float slope, const float *__restrict__ pre, const float *dy, float *dx)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      dx[i] = pre[i] > 0.f ? dy[i] : slope * dy[i];
  }

  // P[b] = sum_i h[b G + i] (fixed order)
  __global__ void grain_sum_kernel(const float *__restrict__ h, int B, int G, long long chw, float *__restrict__ P)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < B * chw;
         i += (long long)gridDim.x * blockDim.x)
      {
        const long long b = i / chw, r = i % chw;
        float           s = 0.f;
        for (int g = 0; g < G; ++g)
          s += h[(b * G + g) * chw + r];
        P[i] = s;
      }
  }

  // Z[b G + i] += Q[b]
  __global__ void grain_bcast_add_kernel(const float *__restrict__ Q, int B, int G, long long chw, float *__restrict__ Z)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < (long long)B * G * chw;
         i += (long long)gridDim.x * blockDim.x)
      {
        const long long bg = i / chw, r = i % chw;
        Z[i] += Q[(bg / G) * chw + r];
      }
  }

  // Adam (Kingma & Ba) with bias correction: m, v moments, step t >= 1.
  __global__ void adam_kernel(long long n, float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                              float *__restrict__ v, float lr, float b1, float b2, float eps, float c1, float c2)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        const float gi = g[i];
        const float mi = b1 * m[i] + (1.f - b1) * gi;
        const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
        m[i]           = mi;
        v[i]           = vi;
        p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
      }
  }

  // Mean squared error over n elements, weights w (nullable): loss = sum w d^2 / n,
  // grad = 2 w d / n; block partial sums in double, summed by the host-side
  // second launch.
  // out = w (p - t)   (w may be NULL = 1)
  __global__ void weighted_diff_kernel(long long n, const float *__restrict__ p, const float *__restrict__ t,
                                       const float *__restrict__ w, float *__restrict__ out)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      out[i] = (w ? w[i] : 1.f) * (p[i] - t[i]);
  }

  // y += alpha a x   (a may be NULL = 1)
  __global__ void mul_add_kernel(long long n, float alpha, const float *__restrict__ a, const float *__restrict__ x,
                                 float *__restrict__ y)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      y[i] += alpha * (a ? a[i] : 1.f) * x[i];
  }

  __global__ void mse_kernel(long long n, const float *__restrict__ pred, const float *__restrict__ target,
                             const float *__restrict__ wt, float *__restrict__ grad, double *__restrict__ partial)
  {
    __shared__ double s_red[8];
    double            acc = 0.0;
    const float       inv = 1.f / float(n);
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        const float d  = pred[i] - target[i];
        const float wi = wt ? wt[i] : 1.f;
        acc += double(wi * d * d);
        if (grad)
          grad[i] = 2.f * wi * d * inv;
      }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1)
      acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0)
      s_red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0)
      {
        double s = 0.0;
        for (int i = 0; i < (int)(blockDim.x >> 5); ++i)
          s += s_red[i];
        partial[blockIdx.x] = s / double(n);
      }
  }

  __global__ void sum_partials_kernel(const double *__restrict__ partial, int nb, double *__restrict__ out)
  {
    if (threadIdx.x == 0 && blockIdx.x == 0)
      {
        double s = 0.0;
        for (int i = 0; i < nb; ++i)
          s += partial[i];
        out[0] = s;
      }
  }

  // Network features of a 2D window of solver states (FP64 block vectors,
  // x-fastest nodes of an nx-wide mesh) -- see sint_nn_features in the header.
  __global__ void features_kernel(const double *__restrict__ u_n, const double *__restrict__ u_nm1, long long ld,
                                  int nx, int ny, int G, int x0, int y0, int Hc, int Wc, float ratio,
                                  const float *__restrict__ scale, float *__restrict__ grain_in,
                                  float *__restrict__ shared_in, int b)
  {
    const long long npix = (long long)Hc * Wc;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x)
      {
        const int yy = y0 + int(i / Wc), xx = x0 + int(i % Wc);
        const bool ok = yy >= 0 && yy < ny && xx >= 0 && xx < nx;
        const long long node = ok ? (long long)yy * nx + xx : 0;
        // shared: c, c-increment, mu, mu-increment (extrapolated increments)
        for (int k = 0; k < 2; ++k)
          {
            const double a  = ok ? u_n[k * ld + node] : 0.0;
            const double d  = ok ? (u_n[k * ld + node] - u_nm1[k * ld + node]) * ratio : 0.0;
            shared_in[((long long)b * 4 + 2 * k) * npix + i]     = float(a) * scale[2 * k];
            shared_in[((long long)b * 4 + 2 * k + 1) * npix + i] = float(d) * scale[2 * k + 1];
          }
        for (int g = 0; g < G; ++g)
          {
            const double a = ok ? u_n[(2 + g) * ld + node] : 0.0;
            const double d = ok ? (u_n[(2 + g) * ld + node] - u_nm1[(2 + g) * ld + node]) * ratio : 0.0;
            grain_in[(((long long)b * G + g) * 2 + 0) * npix + i] = float(a) * scale[4];
            grain_in[(((long long)b * G + g) * 2 + 1) * npix + i] = float(d) * scale[5];
          }
      }
  }

  // Training targets of a window: the increment's deviation from linear
  // extrapolation, t = (u_{n+1} - u_n - ratio (u_n - u_{n-1})) * oscale,
  // oscale = {c, mu, eta}; shared_t [b][2][Hc][Wc], grain_t [b G + g][1][Hc][Wc].
  __global__ void targets_kernel(const double *__restrict__ u_np1, const double *__restrict__ u_n,
                                 const double *__restrict__ u_nm1, long long ld, int nx, int ny, int G, int x0, int y0,
                                 int Hc, int Wc, float ratio, const float *__restrict__ oscale,
                                 float *__restrict__ grain_t, float *__restrict__ shared_t, int b)
  {
    const long long npix = (long long)Hc * Wc;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < npix; i += (long long)gridDim.x * blockDim.x)
      {
        const int       yy = y0 + int(i / Wc), xx = x0 + int(i % Wc);
        const bool      ok = yy >= 0 && yy < ny && xx >= 0 && xx < nx;
        const long long node = ok ? (long long)yy * nx + xx : 0;
        for (int k = 0; k < 2 + G; ++k)
          {
            double t = 0.0;
            if (ok)
              {
                const long long o = k * ld + node;
                t = (u_np1[o] - u_n[o]) - double(ratio) * (u_n[o] - u_nm1[o]);
              }
            const float v = float(t) * oscale[k < 2 ? k : 2];
            if (k < 2)
              shared_t[((long long)b * 2 + k) * npix + i] = v;
            else
              grain_t[((long long)b * G + (k - 2)) * npix + i] = v;
          }
      }
  }

  // Newton initial guess over the whole mesh from the network outputs:
  // u = u_n + ratio (u_n - u_{n-1}) + out / oscale.
  __global__ void apply_guess_kernel(const double *__restrict__ u_n, const double *__restrict__ u_nm1, long long ld,
                                     long long N, int G, float ratio, const float *__restrict__ oscale,
                                     const float *__restrict__ grain_out, const float *__restrict__ shared_out,
                                     double *__restrict__ guess)
  {
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
      for (int k = 0; k < 2 + G; ++k)
        {
          const long long o   = k * ld + i;
          const float     out = k < 2 ? shared_out[(long long)k * N + i] : grain_out[(long long)(k - 2) * N + i];
          guess[o] = u_n[o] + double(ratio) * (u_n[o] - u_nm1[o]) + double(out / oscale[k < 2 ? k : 2]);
        }
  }

  // Largest extrapolated increment |ratio (u_n - u_{n-1})| of c, mu and the
  // order parameters over all nodes.  Non-negative floats order like their
  // bit patterns, so an unsigned atomicMax gives the same result in any order.
  __global__ void increment_max_kernel(const double *__restrict__ u_n, const double *__restrict__ u_nm1, long long ld,
                                       long long N, int G, float ratio, unsigned *__restrict__ work)
  {
    float m[3] = {0.f, 0.f, 0.f};
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < N; i += (long long)gridDim.x * blockDim.x)
      for (int k = 0; k < 2 + G; ++k)
        {
          const long long o = k * ld + i;
          const float     d = fabsf(float((u_n[o] - u_nm1[o]) * double(ratio)));
          const int       g = k < 2 ? k : 2;
          m[g]              = fmaxf(m[g], d);
        }
#pragma unroll
    for (int g = 0; g < 3; ++g)
      {
        float v = m[g];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1)
          v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, o));
        if ((threadIdx.x & 31) == 0)
          atomicMax(work + g, __float_as_uint(v));
      }
  }

  // scale = (base_c, 1/m_c, base_mu, 1/m_mu, base_eta, 1/m_eta),
  // oscale = (k_c/(m_c dt), k_mu/(m_mu dt), k_eta/(m_eta dt)); base = (base_c,
  // base_mu, base_eta, k_c, k_mu, k_eta).  A zero increment keeps 1/m = 1.
  __global__ void increment_scales_kernel(const unsigned *__restrict__ work, const float *__restrict__ base,
                                          float dt, float *__restrict__ scale, float *__restrict__ oscale)
  {
    if (threadIdx.x != 0)
      return;
    for (int g = 0; g < 3; ++g)
      {
        const float m   = __uint_as_float(work[g]);
        const float inv = m > 1e-30f ? 1.f / m : 1.f;
        scale[2 * g]     = base[g];
        scale[2 * g + 1] = inv;
        oscale[g]        = base[3 + g] * inv / dt;
      }
  }

  // --- 3D windows ------------------------------------------------------------
  // A 3D window of D x H x W nodes is held depth-major with one zero slice
  // before and after: [sample][D + 2][channels][H][W].  Every depth slice of
  // every sample is then one contiguous [channels][H][W] image, so a 3x3x3
  // convolution is three 3x3 convolutions of the slice batch shifted by one
  // slice (the zero slices are the padding in depth).
  __device__ __forceinline__ bool window_node3(int nx, int ny, int nz, int x0, int y0, int z0, int H, int W,
                                               long long i, int &z, long long &node, long long &pix)
  {
    const long long hw = (long long)H * W;
    z                  = int(i / hw);
    pix                = i % hw;
    const int yy = y0 + int(pix / W), xx = x0 + int(pix % W), zz = z0 + z;
    const bool ok = xx >= 0 && xx < nx && yy >= 0 && yy < ny && zz >= 0 && zz < nz;
    node          = ok ? ((long long)zz * ny + yy) * nx + xx : 0;
    return ok;
  }

  __global__ void features3d_kernel(const double *__restrict__ u_n, const double *__restrict__ u_nm1, long long ld,
                                    int nx, int ny, int nz, int G, int x0, int y0, int z0, int D, int H, int W,
                                    float ratio, const float *__restrict__ scale, float *__restrict__ grain_in,
                                    float *__restrict__ shared_in, int b)
  {
    const long long hw = (long long)H * W, n = hw * D;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        int       z;
        long long node, pix;
        const bool ok = window_node3(nx, ny, nz, x0, y0, z0, H, W, i, z, node, pix);
        for (int k = 0; k < 2; ++k)
          {
            const double a = ok ? u_n[k * ld + node] : 0.0;
            const double d = ok ? (u_n[k * ld + node] - u_nm1[k * ld + node]) * ratio : 0.0;
            float *o       = shared_in + (((long long)b * (D + 2) + z + 1) * 4 + 2 * k) * hw + pix;
            o[0]           = float(a) * scale[2 * k];
            o[hw]          = float(d) * scale[2 * k + 1];
          }
        for (int g = 0; g < G; ++g)
          {
            const double a = ok ? u_n[(2 + g) * ld + node] : 0.0;
            const double d = ok ? (u_n[(2 + g) * ld + node] - u_nm1[(2 + g) * ld + node]) * ratio : 0.0;
            float *o       = grain_in + ((((long long)b * G + g) * (D + 2) + z + 1) * 2) * hw + pix;
            o[0]           = float(a) * scale[4];
            o[hw]          = float(d) * scale[5];
          }
      }
  }

  __global__ void targets3d_kernel(const double *__restrict__ u_np1, const double *__restrict__ u_n,
                                   const double *__restrict__ u_nm1, long long ld, int nx, int ny, int nz, int G,
                                   int x0, int y0, int z0, int D, int H, int W, float ratio,
                                   const float *__restrict__ oscale, float *__restrict__ grain_t,
                                   float *__restrict__ shared_t, int b)
  {
    const long long hw = (long long)H * W, n = hw * D;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        int       z;
        long long node, pix;
        const bool ok = window_node3(nx, ny, nz, x0, y0, z0, H, W, i, z, node, pix);
        for (int k = 0; k < 2 + G; ++k)
          {
            double t = 0.0;
            if (ok)
              {
                const long long o = k * ld + node;
                t = (u_np1[o] - u_n[o]) - double(ratio) * (u_n[o] - u_nm1[o]);
              }
            const float v = float(t) * oscale[k < 2 ? k : 2];
            if (k < 2)
              shared_t[(((long long)b * (D + 2) + z + 1) * 2 + k) * hw + pix] = v;
            else
              grain_t[(((long long)b * G + (k - 2)) * (D + 2) + z + 1) * hw + pix] = v;
          }
      }
  }

  // Guess at the nodes of depth slices z0 .. z0 + D - 1 of the mesh from the
  // outputs of a whole-plane window (H = ny, W = nx) whose slice 1 + off + j
  // holds mesh slice z0 + j (off: the window's halo in depth).
  __global__ void apply_guess3d_kernel(const double *__restrict__ u_n, const double *__restrict__ u_nm1, long long ld,
                                       int nx, int ny, int G, int z0, int D, int off, int Dw, float ratio,
                                       const float *__restrict__ oscale, const float *__restrict__ grain_out,
                                       const float *__restrict__ shared_out, double *__restrict__ guess)
  {
    const long long hw = (long long)nx * ny, n = hw * D;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        const int       z    = int(i / hw);
        const long long pix  = i % hw;
        const long long node = (long long)(z0 + z) * hw + pix;
        const long long ws   = 1 + off + z; // window slice
        for (int k = 0; k < 2 + G; ++k)
          {
            const long long o = k * ld + node;
            const float out = k < 2 ? shared_out[(ws * 2 + k) * hw + pix]
                                    : grain_out[((long long)(k - 2) * (Dw + 2) + ws) * hw + pix];
            guess[o] = u_n[o] + double(ratio) * (u_n[o] - u_nm1[o]) + double(out / oscale[k < 2 ? k : 2]);
          }
      }
  }

  // zero slices 0 and D2 - 1 of each of S samples of slice_elems floats
  __global__ void zero_pad_slices_kernel(float *__restrict__ x, int S, int D2, long long slice_elems)
  {
    const long long n = 2ll * S * slice_elems;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
      {
        const long long s = i / (2 * slice_elems), r = i % (2 * slice_elems);
        const long long sl = r < slice_elems ? 0 : D2 - 1;
        x[(s * D2 + sl) * slice_elems + r % slice_elems] = 0.f;
      }
  }

  static int launch_err(const char *what)
  {
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, what);
  }
} // namespace sint

using namespace sint;

extern "C" {

int sint_nn_conv3x3_f32(const float *in, int B, int Cin, int H, int W, const float *w, const float *bias,
                        float *out, int Cout, int accumulate, sint_stream_t s)
{
  if (!in || !w || !out || B < 1 || Cin < 1 || Cout < 1 || H < 1 || W < 1)
    {
      set_error("sint_nn_conv3x3_f32: bad argument");
      return SINT_ERR_ARG;
    }
  const int tiles = ((W + CT - 1) / CT) * ((H + CT - 1) / CT);
  dim3      grid(tiles, (Cout + COB - 1) / COB, B);
  conv3x3_kernel<<<grid, CT * CT, 0, s>>>(in, Cin, H, W, w, bias, out, Cout, accumulate);
  return launch_err("sint_nn_conv3x3_f32");
}

int sint_nn_conv3x3_flip_f32(const float *w, int Cout, int Cin, float *wT, sint_stream_t s)
{
  if (!w || !wT || Cout < 1 || Cin < 1)
    {
      set_error("sint_nn_conv3x3_flip_f32: bad argument");
      return SINT_ERR_ARG;
    }
  conv3x3_flip_kernel<<<(Cout * Cin * 9 + 255) / 256, 256, 0, s>>>(w, Cout, Cin, wT);
  return launch_err("sint_nn_conv3x3_flip_f32");
}

int64_t sint_nn_conv3x3_wgrad_workspace(int B, int Cin, int Cout, int H, int W)
{
  const int64_t blocks = (int64_t)B * ((W + CT - 1) / CT) * ((H + CT - 1) / CT);
  return blocks * Cout * (Cin * 9 + 1);
}

int sint_nn_conv3x3_wgrad_f32(const float *in, const float *dout, int B, int Cin, int Cout, int H, int W, float *dw,
                              float *db, int accumulate, float *work, sint_stream_t s)
{
  if (!in || !dout || !dw || !work || B < 1 || Cin < 1 || Cout < 1 || H < 1 || W < 1)
    {
      set_error("sint_nn_conv3x3_wgrad_f32: bad argument");
      return SINT_ERR_ARG;
    }
  const int    tiles  = ((W + CT - 1) / CT) * ((H + CT - 1) / CT);
  const int    blocks = tiles * B;
  float       *pw = work, *pb = work + (long long)blocks * Cout * Cin * 9;
  const size_t smem = sizeof(float) * (size_t(Cout) * CT * CT + size_t(Cin) * (CT + 2) * (CT + 2));
  if (smem > 48 * 1024)
    {
      const cudaError_t e =
        cudaFuncSetAttribute(conv3x3_wgrad_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem));
      if (e != cudaSuccess)
        return cuda_fail(e, "sint_nn_conv3x3_wgrad_f32: smem");
    }
  conv3x3_wgrad_kernel<<<dim3(tiles, B), WG_THREADS, smem, s>>>(in, dout, Cin, Cout, H, W, pw, db ? pb : nullptr);
  if (int rc = launch_err("sint_nn_conv3x3_wgrad_f32"))
    return rc;
  const long long nw = (long long)Cout * Cin * 9;
  reduce_chunks_kernel<<<(unsigned)((nw + 255) / 256), 256, 0, s>>>(pw, blocks, nw, dw, accumulate);
  if (int rc = launch_err("sint_nn_conv3x3_wgrad_f32: reduce"))
    return rc;
  if (db)
    {
      reduce_chunks_kernel<<<(Cout + 255) / 256, 256, 0, s>>>(pb, blocks, Cout, db, accumulate);
      return launch_err("sint_nn_conv3x3_wgrad_f32: bias");
    }
  return SINT_OK;
}

int sint_nn_leaky_relu_f32(int64_t n, float slope, const float *x, float *y, sint_stream_t s)
{
  leaky_fwd_kernel<<<1184, 256, 0, s>>>(n, slope, x, y);
  return launch_err("sint_nn_leaky_relu_f32");
}

int sint_nn_leaky_relu_bwd_f32(int64_t n, float slope, const float *pre, const float *dy, float *dx, sint_stream_t s)
{
  leaky_bwd_kernel<<<1184, 256, 0, s>>>(n, slope, pre, dy, dx);
  return launch_err("sint_nn_leaky_relu_bwd_f32");
}

int sint_nn_grain_sum_f32(const float *h, int B, int G, int64_t chw, float *P, sint_stream_t s)
{
  grain_sum_kernel<<<1184, 256, 0, s>>>(h, B, G, chw, P);
  return launch_err("sint_nn_grain_sum_f32");
}

int sint_nn_grain_bcast_add_f32(const float *Q, int B, int G, int64_t chw, float *Z, sint_stream_t s)
{
  grain_bcast_add_kernel<<<1184, 256, 0, s>>>(Q, B, G, chw, Z);
  return launch_err("sint_nn_grain_bcast_add_f32");
}

int sint_nn_adam_f32(int64_t n, float *p, const float *g, float *m, float *v, float lr, float beta1, float beta2,
                     float eps, int step, sint_stream_t s)
{
  if (step < 1)
    {
      set_error("sint_nn_adam_f32: step must be >= 1");
      return SINT_ERR_ARG;
    }
  const float c1 = 1.f - powf(beta1, float(step)), c2 = 1.f - powf(beta2, float(step));
  adam_kernel<<<1184, 256, 0, s>>>(n, p, g, m, v, lr, beta1, beta2, eps, c1, c2);
  return launch_err("sint_nn_adam_f32");
}

int sint_nn_weighted_diff_f32(int64_t n, const float *pred, const float *target, const float *weight, float *out,
                              sint_stream_t s)
{
  if (!pred || !target || !out || n < 0)
    {
      set_error("sint_nn_weighted_diff_f32: bad argument");
      return SINT_ERR_ARG;
    }
  if (n == 0)
    return SINT_OK;
  weighted_diff_kernel<<<1184, 256, 0, s>>>(n, pred, target, weight, out);
  return launch_err("sint_nn_weighted_diff_f32");
}

int sint_nn_mul_add_f32(int64_t n, float alpha, const float *a, const float *x, float *y, sint_stream_t s)
{
  if (!x || !y || n < 0)
    {
      set_error("sint_nn_mul_add_f32: bad argument");
      return SINT_ERR_ARG;
    }
  if (n == 0)
    return SINT_OK;
  mul_add_kernel<<<1184, 256, 0, s>>>(n, alpha, a, x, y);
  return launch_err("sint_nn_mul_add_f32");
}

int64_t sint_nn_mse_workspace(void) { return 1184 + 1; }

int sint_nn_mse_f32(int64_t n, const float *pred, const float *target, const float *weight, float *grad,
                    double *loss, double *work, sint_stream_t s)
{
  if (!pred || !target || !loss || !work || n < 1)
    {
      set_error("sint_nn_mse_f32: bad argument");
      return SINT_ERR_ARG;
    }
  mse_kernel<<<1184, 256, 0, s>>>(n, pred, target, weight, grad, work);
  if (int rc = launch_err("sint_nn_mse_f32"))
    return rc;
  sum_partials_kernel<<<1, 32, 0, s>>>(work, 1184, loss);
  return launch_err("sint_nn_mse_f32: sum");
}

int sint_nn_features_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int nx, int ny, int G, int x0,
                         int y0, int Hc, int Wc, float ratio, const float *scale, float *grain_in, float *shared_in,
                         int b, sint_stream_t s)
{
  if (!u_n || !u_nm1 || !scale || !grain_in || !shared_in || G < 1 || Hc < 1 || Wc < 1)
    {
      set_error("sint_nn_features_f64: bad argument");
      return SINT_ERR_ARG;
    }
  features_kernel<<<592, 256, 0, s>>>(u_n, u_nm1, block_stride, nx, ny, G, x0, y0, Hc, Wc, ratio, scale, grain_in,
                                      shared_in, b);
  return launch_err("sint_nn_features_f64");
}

int sint_nn_targets_f64(const double *u_np1, const double *u_n, const double *u_nm1, int64_t block_stride, int nx,
                        int ny, int G, int x0, int y0, int Hc, int Wc, float ratio, const float *oscale,
                        float *grain_t, float *shared_t, int b, sint_stream_t s)
{
  if (!u_np1 || !u_n || !u_nm1 || !oscale || !grain_t || !shared_t || G < 1 || Hc < 1 || Wc < 1)
    {
      set_error("sint_nn_targets_f64: bad argument");
      return SINT_ERR_ARG;
    }
  targets_kernel<<<592, 256, 0, s>>>(u_np1, u_n, u_nm1, block_stride, nx, ny, G, x0, y0, Hc, Wc, ratio, oscale,
                                     grain_t, shared_t, b);
  return launch_err("sint_nn_targets_f64");
}

int sint_nn_apply_guess_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int64_t n_nodes, int G,
                            float ratio, const float *oscale, const float *grain_out, const float *shared_out,
                            double *guess, sint_stream_t s)
{
  if (!u_n || !u_nm1 || !oscale || !grain_out || !shared_out || !guess || G < 1 || n_nodes < 1)
    {
      set_error("sint_nn_apply_guess_f64: bad argument");
      return SINT_ERR_ARG;
    }
  apply_guess_kernel<<<1184, 256, 0, s>>>(u_n, u_nm1, block_stride, n_nodes, G, ratio, oscale, grain_out, shared_out,
                                          guess);
  return launch_err("sint_nn_apply_guess_f64");
}

int sint_nn_increment_scales_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int64_t n_nodes, int G,
                                 float ratio, float dt, const float *base, unsigned *work, float *scale,
                                 float *oscale, sint_stream_t s)
{
  if (!u_n || !u_nm1 || !base || !work || !scale || !oscale || G < 1 || n_nodes < 1 || !(dt > 0.f))
    {
      set_error("sint_nn_increment_scales_f64: bad argument");
      return SINT_ERR_ARG;
    }
  const cudaError_t e = cudaMemsetAsync(work, 0, 3 * sizeof(unsigned), s);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_nn_increment_scales_f64: memset");
  increment_max_kernel<<<592, 256, 0, s>>>(u_n, u_nm1, block_stride, n_nodes, G, ratio, work);
  if (int rc = launch_err("sint_nn_increment_scales_f64"))
    return rc;
  increment_scales_kernel<<<1, 32, 0, s>>>(work, base, dt, scale, oscale);
  return launch_err("sint_nn_increment_scales_f64: scales");
}

int sint_nn_features3d_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int nx, int ny, int nz,
                           int G, int x0, int y0, int z0, int D, int H, int W, float ratio, const float *scale,
                           float *grain_in, float *shared_in, int b, sint_stream_t s)
{
  if (!u_n || !u_nm1 || !scale || !grain_in || !shared_in || G < 1 || D < 1 || H < 1 || W < 1 || b < 0)
    {
      set_error("sint_nn_features3d_f64: bad argument");
      return SINT_ERR_ARG;
    }
  features3d_kernel<<<1184, 256, 0, s>>>(u_n, u_nm1, block_stride, nx, ny, nz, G, x0, y0, z0, D, H, W, ratio, scale,
                                         grain_in, shared_in, b);
  return launch_err("sint_nn_features3d_f64");
}

int sint_nn_targets3d_f64(const double *u_np1, const double *u_n, const double *u_nm1, int64_t block_stride, int nx,
                          int ny, int nz, int G, int x0, int y0, int z0, int D, int H, int W, float ratio,
                          const float *oscale, float *grain_t, float *shared_t, int b, sint_stream_t s)
{
  if (!u_np1 || !u_n || !u_nm1 || !oscale || !grain_t || !shared_t || G < 1 || D < 1 || H < 1 || W < 1 || b < 0)
    {
      set_error("sint_nn_targets3d_f64: bad argument");
      return SINT_ERR_ARG;
    }
  targets3d_kernel<<<1184, 256, 0, s>>>(u_np1, u_n, u_nm1, block_stride, nx, ny, nz, G, x0, y0, z0, D, H, W, ratio,
                                        oscale, grain_t, shared_t, b);
  return launch_err("sint_nn_targets3d_f64");
}

int sint_nn_apply_guess3d_f64(const double *u_n, const double *u_nm1, int64_t block_stride, int nx, int ny, int G,
                              int z0, int D, int halo, int Dw, float ratio, const float *oscale, const float *grain_out,
                              const float *shared_out, double *guess, sint_stream_t s)
{
  if (!u_n || !u_nm1 || !oscale || !grain_out || !shared_out || !guess || G < 1 || D < 1 || halo < 0 ||
      halo + D > Dw || nx < 1 || ny < 1 || z0 < 0)
    {
      set_error("sint_nn_apply_guess3d_f64: bad argument");
      return SINT_ERR_ARG;
    }
  apply_guess3d_kernel<<<1184, 256, 0, s>>>(u_n, u_nm1, block_stride, nx, ny, G, z0, D, halo, Dw, ratio, oscale,
                                            grain_out, shared_out, guess);
  return launch_err("sint_nn_apply_guess3d_f64");
}

int sint_nn_zero_pad_slices_f32(float *x, int S, int D2, int64_t slice_elems, sint_stream_t s)
{
  if (!x || S < 1 || D2 < 2 || slice_elems < 1)
    {
      set_error("sint_nn_zero_pad_slices_f32: bad argument");
      return SINT_ERR_ARG;
    }
  zero_pad_slices_kernel<<<592, 256, 0, s>>>(x, S, D2, slice_elems);
  return launch_err("sint_nn_zero_pad_slices_f32");
}

} // extern "C"
