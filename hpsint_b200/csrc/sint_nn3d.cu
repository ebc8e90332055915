// 3D convolution of the learned Newton guess for inference, in one pass.
//
// The 3D network works on depth-padded windows [S][D + 2][C][H][W]: slices 1
// .. D hold the data, slices 0 and D + 1 are zero (the depth padding).  The
// training path evaluates a 3x3x3 convolution as three slice-shifted 3x3
// convolutions (sint_nn.cu), which reads and writes every activation three
// times and needs a separate pass to clear the padding.  This kernel does the
// 27 taps, a second input, the bias, a broadcast addend and the leaky ReLU in
// one pass: every output is written once, the input tile once staged.
//
// Block: 32 (x) x 8 (y) threads; each thread owns a column of ZB consecutive
// output slices at its (x, y) for all COUT output channels (ZB x COUT FP32
// accumulators).  Per input channel the block stages the (ZB + 2) x 10 x 34
// input box (zero outside the window) and that channel's 27 x COUT weights
// in shared memory with cp.async, double-buffered: the next channel's copies
// are in flight while this one is computed.  A thread reads, per (dy, dx)
// tap column, ZB + 2 input values and per dz the COUT weights (one broadcast
// read serves the warp), and issues 3 ZB COUT fused multiply-adds, as packed
// FP32 pairs of output channels (FFMA2) when COUT is a multiple of 4.
#include <cstdint>
#include <cuda_runtime.h>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  namespace
  {
    constexpr int C3_TX = 32, C3_TY = 8, C3_THREADS = C3_TX * C3_TY;
    constexpr int C3_PX = C3_TX + 3; // row pitch of the staged box (34 used)

    struct Conv3dArgs
    {
      int          S, D, H, W;
      const float *x[2];   // inputs, [S][D + 2][c][H][W]
      const float *w[2];   // weights [3 (dz)][cout][c][3 (dy)][3 (dx)]
      int          c[2];   // input channels (c[1] = 0: no second input)
      const float *bias;   // [cout] or nullptr
      const float *addend; // [S / addend_group][D + 2][cout][H][W] or nullptr
      int          addend_group;
      int          leaky;
      float        slope;
      float       *out; // [S][D + 2][cout][H][W]
      int          cout;
      int          accumulate;
    };

    // output slices per thread: ZB x COUT accumulators stay within 64 registers,
    // the two staged boxes within the 48 KB of static shared memory
    template <int COUT>
    __host__ __device__ constexpr int conv3d_zb()
    {
      return COUT >= 32 ? 1 : COUT >= 16 ? 4 : COUT >= 8 ? 8 : 12;
    }

    // 4-byte asynchronous global->shared copy; !valid writes zero (source size 0)
    __device__ __forceinline__ void cp_async4(float *dst, const float *src, bool valid)
    {
      const unsigned sa = (unsigned)__cvta_generic_to_shared(dst);
      asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;\n" ::"r"(sa), "l"(src), "r"(valid ? 4 : 0));
    }
    __device__ __forceinline__ void cp_async_commit_group() { asm volatile("cp.async.commit_group;\n" ::); }
    template <int N>
    __device__ __forceinline__ void cp_async_wait_group()
    {
      asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
    }

    template <int COUT>
    __global__ void __launch_bounds__(C3_THREADS, 2) conv3d_kernel(const Conv3dArgs a)
    {
      constexpr int ZB = conv3d_zb<COUT>();
      constexpr int BZ = ZB + 2, BY = C3_TY + 2, BX = C3_TX + 2;
      // double-buffered input box and weights of one input channel
      __shared__ float s_in[2][BZ][BY][C3_PX];
      __shared__ __align__(16) float s_w[2][27][COUT];

      const int tiles_x = (a.W + C3_TX - 1) / C3_TX;
      const int x0 = (blockIdx.x % tiles_x) * C3_TX, y0 = (blockIdx.x / tiles_x) * C3_TY;
      const int z0 = 1 + blockIdx.y * ZB; // first output slice (window slice index)
      const int s  = blockIdx.z;
      const int tx = threadIdx.x % C3_TX, ty = threadIdx.x / C3_TX;
      const long long hw = (long long)a.H * a.W;
      const int       D2 = a.D + 2;
      const int       nch = a.c[0] + a.c[1];

      // stage input channel g (of x1 then x2) into buffer b: each warp copies
      // whole box rows, lane l the row entries l and l + 32 (< BX); entries
      // outside the window are zero-filled
      auto stage = [&](int g, int b) {
        // selects, not a dynamic index into the parameter arrays (which would
        // copy them to local memory)
        const bool   k   = g >= a.c[0];
        const int    ci  = k ? g - a.c[0] : g;
        const int    ck  = k ? a.c[1] : a.c[0];
        const float *xk  = k ? a.x[1] : a.x[0];
        const float *wk  = k ? a.w[1] : a.w[0];
        const float *src = xk + (long long)s * D2 * ck * hw + (long long)ci * hw;
        for (int row = ty; row < BZ * BY; row += C3_TY)
          {
            const int  bz = row / BY, by = row % BY;
            const int  zz = z0 - 1 + bz, yy = y0 - 1 + by;
            const bool rv = zz >= 1 && zz <= a.D && yy >= 0 && yy < a.H;
            const float *rp = src + (long long)zz * ck * hw + (long long)yy * a.W;
#pragma unroll
            for (int h = 0; h < 2; ++h)
              {
                const int bx = tx + 32 * h;
                if (bx < BX)
                  {
                    const int  xx = x0 - 1 + bx;
                    const bool v  = rv && xx >= 0 && xx < a.W;
                    cp_async4(&s_in[b][bz][by][bx], v ? rp + xx : a.x[0], v);
                  }
              }
          }
        for (int i = threadIdx.x; i < 27 * COUT; i += C3_THREADS)
          {
            const int  tap = i / COUT, co = i % COUT, dz = tap / 9, t9 = tap % 9;
            const bool v   = co < a.cout;
            cp_async4(&s_w[b][tap][co], v ? wk + (((long long)dz * a.cout + co) * ck + ci) * 9 + t9 : a.w[0], v);
          }
      };

      // accumulators: scalar, or channel pairs when COUT is a multiple of 4
      constexpr bool PAIRS = COUT % 4 == 0;
      float          acc[PAIRS ? 1 : ZB][PAIRS ? 1 : COUT];
      float2         acc2[PAIRS ? ZB : 1][PAIRS ? COUT / 2 : 1];
#pragma unroll
      for (int z = 0; z < ZB; ++z)
#pragma unroll
        for (int co = 0; co < COUT; ++co)
          {
            if constexpr (PAIRS)
              (co & 1 ? acc2[z][co / 2].y : acc2[z][co / 2].x) = 0.f;
            else
              acc[z][co] = 0.f;
          }

      stage(0, 0);
      cp_async_commit_group();
      for (int g = 0; g < nch; ++g)
        {
          const int b = g & 1;
          if (g + 1 < nch)
            stage(g + 1, b ^ 1);
          cp_async_commit_group();
          cp_async_wait_group<1>(); // channel g has landed (only g + 1 may be pending)
          __syncthreads();
#pragma unroll
          for (int dy = 0; dy < 3; ++dy)
#pragma unroll
            for (int dx = 0; dx < 3; ++dx)
              {
                float col[BZ];
#pragma unroll
                for (int z = 0; z < BZ; ++z)
                  col[z] = s_in[b][z][ty + dy][tx + dx];
                if constexpr (COUT % 4 == 0)
                  {
                    // packed FP32 pairs: two output channels per FFMA2 (each
                    // lane rounds as fmaf does), the input value in both lanes
                    float2 cc[BZ];
#pragma unroll
                    for (int z = 0; z < BZ; ++z)
                      cc[z] = make_float2(col[z], col[z]);
#pragma unroll
                    for (int dz = 0; dz < 3; ++dz)
                      {
                        const float *wr = s_w[b][(dz * 3 + dy) * 3 + dx];
#pragma unroll
                        for (int co = 0; co < COUT; co += 4)
                          {
                            const float4 q  = *reinterpret_cast<const float4 *>(wr + co);
                            const float2 w0 = make_float2(q.x, q.y), w1 = make_float2(q.z, q.w);
#pragma unroll
                            for (int z = 0; z < ZB; ++z)
                              {
                                acc2[z][co / 2]     = __ffma2_rn(w0, cc[z + dz], acc2[z][co / 2]);
                                acc2[z][co / 2 + 1] = __ffma2_rn(w1, cc[z + dz], acc2[z][co / 2 + 1]);
                              }
                          }
                      }
                  }
                else
                  {
#pragma unroll
                    for (int dz = 0; dz < 3; ++dz)
                      {
                        const float *wr = s_w[b][(dz * 3 + dy) * 3 + dx];
                        float        wv[COUT];
#pragma unroll
                        for (int co = 0; co < COUT; ++co)
                          wv[co] = wr[co];
#pragma unroll
                        for (int z = 0; z < ZB; ++z)
#pragma unroll
                          for (int co = 0; co < COUT; ++co)
                            acc[z][co] = fmaf(wv[co], col[z + dz], acc[z][co]);
                      }
                  }
              }
          // the next iteration's copies overwrite the buffer read here
          __syncthreads();
        }
      cp_async_wait_group<0>();

      const int x = x0 + tx, y = y0 + ty;
      if (x >= a.W || y >= a.H)
        return;
      const long long pix = (long long)y * a.W + x;
      // slice z0, channel 0 of this thread's output and addend columns
      const long long zs = (long long)a.cout * hw;
      float          *op = a.out + ((long long)s * D2 + z0) * zs + pix;
      const float    *ap = a.addend ? a.addend + ((long long)(s / a.addend_group) * D2 + z0) * zs + pix : nullptr;
#pragma unroll
      for (int z = 0; z < ZB; ++z)
        {
          if (z0 + z > a.D)
            break;
#pragma unroll
          for (int co = 0; co < COUT; ++co)
            {
              if (co >= a.cout)
                break;
              const long long o = z * zs + co * hw;
              float           v;
              if constexpr (PAIRS)
                v = co & 1 ? acc2[z][co / 2].y : acc2[z][co / 2].x;
              else
                v = acc[z][co];
              if (a.bias)
                v += a.bias[co];
              if (ap)
                v += ap[o];
              if (a.accumulate)
                v += op[o];
              if (a.leaky && v < 0.f)
                v *= a.slope;
              op[o] = v;
            }
        }
      // the depth padding of the output: slice 0 by the first z tile, D + 1 by the last
      if (blockIdx.y == 0 || blockIdx.y == gridDim.y - 1)
        for (int co = 0; co < a.cout; ++co)
          {
            if (blockIdx.y == 0)
              a.out[(((long long)s * D2 + 0) * a.cout + co) * hw + pix] = 0.f;
            if (blockIdx.y == gridDim.y - 1)
              a.out[(((long long)s * D2 + a.D + 1) * a.cout + co) * hw + pix] = 0.f;
          }
    }

    template <int COUT>
    cudaError_t launch_conv3d(const Conv3dArgs &a, cudaStream_t st)
    {
      constexpr int ZB      = conv3d_zb<COUT>();
      const int     tiles_x = (a.W + C3_TX - 1) / C3_TX, tiles_y = (a.H + C3_TY - 1) / C3_TY;
      const dim3    grid(unsigned(tiles_x * tiles_y), unsigned((a.D + ZB - 1) / ZB), unsigned(a.S));
      conv3d_kernel<COUT><<<grid, C3_THREADS, 0, st>>>(a);
      count_launches(1);
      return cudaGetLastError();
    }
  } // namespace
} // namespace sint

using namespace sint;

extern "C" {

int sint_nn_conv3d_f32(int S, int D, int H, int W, const float *x1, int c1, const float *w1, const float *x2, int c2,
                       const float *w2, const float *bias, const float *addend, int addend_group, int leaky,
                       float slope, float *out, int cout, int accumulate, sint_stream_t stream)
{
  if (S < 1 || D < 1 || H < 1 || W < 1 || !x1 || !w1 || c1 < 1 || c2 < 0 || (c2 > 0 && (!x2 || !w2)) || !out ||
      cout < 1 || cout > 32 || (addend && (addend_group < 1 || S % addend_group != 0)) ||
      (long long)((W + C3_TX - 1) / C3_TX) * ((H + C3_TY - 1) / C3_TY) >= (1ll << 31) || S > 65535)
    {
      set_error("sint_nn_conv3d_f32: bad argument");
      return SINT_ERR_ARG;
    }
  Conv3dArgs a{};
  a.S = S, a.D = D, a.H = H, a.W = W;
  a.x[0] = x1, a.x[1] = c2 > 0 ? x2 : nullptr;
  a.w[0] = w1, a.w[1] = c2 > 0 ? w2 : nullptr;
  a.c[0] = c1, a.c[1] = c2;
  a.bias = bias, a.addend = addend, a.addend_group = addend ? addend_group : 1;
  a.leaky = leaky, a.slope = slope, a.out = out, a.cout = cout, a.accumulate = accumulate;
  cudaError_t e;
  if (cout <= 1)
    e = launch_conv3d<1>(a, stream);
  else if (cout <= 2)
    e = launch_conv3d<2>(a, stream);
  else if (cout <= 4)
    e = launch_conv3d<4>(a, stream);
  else if (cout <= 8)
    e = launch_conv3d<8>(a, stream);
  else if (cout <= 16)
    e = launch_conv3d<16>(a, stream);
  else
    e = launch_conv3d<32>(a, stream);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_nn_conv3d_f32");
}

} // extern "C"
