// Tensor-core 3x3 convolution for the learned guess's inference (sm_100a).
//
// Implicit GEMM on the 5th-generation tensor cores without an im2col copy:
// a CTA tile is 16 x 8 output pixels (M = 128 GEMM rows) times all 32 output
// channels (N = 32).  The CTA stages the 18 x 10 input patch of the tile (all
// input channels, zero outside the image) in shared memory, channel-minor in
// 16-byte chunks of 4 channels: chunk (kc, patch row, patch column) at
// ((kc * 18 + row) * 10 + column) * 16 bytes.  In that layout the A operand of
// tap (dy, dx) -- row r = 8 g + j of the GEMM is pixel (g, j) of the tile,
// shifted by (dy, dx) -- is the K-major, no-swizzle canonical layout with
// core matrices of 8 consecutive pixels of one patch row (stride byte offset
// = one patch row, 160 bytes; leading byte offset = one channel chunk plane,
// 2880 bytes), starting (dy + 1) * 160 + (dx + 1) * 16 bytes into the patch.
// So the 3x3 convolution is 9 taps x Cin/8 tcgen05.mma.kind::tf32 (K = 8)
// accumulating into one 32-column TMEM tile, issued by one thread and
// signalled by tcgen05.commit on an mbarrier.  The weights sit in shared
// memory as B[tap][kc][co] chunks for the whole kernel.  The epilogue reads
// the accumulator with tcgen05.ld (lane = pixel, column = output channel).
// The patch of the next tile is loaded by cp.async into a second buffer
// while this tile's MMAs and epilogue run; two CTAs share an SM.
// TF32 reads the FP32 bit patterns directly.
//
// Every wait is bounded: a CTA whose MMA does not complete within about a
// second records a status, frees its TMEM and returns.
#include <cstdint>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  namespace tc
  {
    constexpr int TY = 16, TX = 8;          // output tile (rows x columns)
    constexpr int PY = TY + 2, PX = TX + 2; // input patch
    constexpr int M       = TY * TX;        // 128 GEMM rows (TMEM lanes)
    constexpr int NMAX    = 32;             // output channels (TMEM columns)
    constexpr int TMEM_COLS = 32;           // smallest TMEM allocation
    constexpr int THREADS = 256;            // warps w and w + 4 read the same TMEM lanes, different columns
    constexpr int CTAS_PER_SM = 2;
    constexpr int CIN_MAX = 32;

    __host__ __device__ constexpr int chunks_of(int cin) { return (cin + 7) / 8 * 2; } // 4-channel chunks, K padded to 8
    __host__ __device__ constexpr size_t patch_bytes(int kc) { return size_t(kc) * PY * PX * 16; }
    __host__ __device__ constexpr size_t weight_bytes(int kc, int n) { return size_t(9) * kc * n * 16; }
    // two patch buffers (the next tile's loads overlap this tile's MMAs), the weights, mbarrier + TMEM address
    __host__ __device__ constexpr size_t smem_bytes(int kc, int n) { return 2 * patch_bytes(kc) + weight_bytes(kc, n) + 16; }

    __device__ __forceinline__ uint32_t smem_u32(const void *p)
    {
      return static_cast<uint32_t>(__cvta_generic_to_shared(p));
    }

    // Shared-memory matrix descriptor: start, leading and stride byte offsets
    // (>> 4), descriptor version 1 (bit 46), no swizzle (bits 61-63 = 0).
    __device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t lbo, uint32_t sbo)
    {
      return uint64_t((addr >> 4) & 0x3FFFu) | (uint64_t((lbo >> 4) & 0x3FFFu) << 16) |
             (uint64_t((sbo >> 4) & 0x3FFFu) << 32) | (uint64_t(1) << 46);
    }

    // Instruction descriptor of kind::tf32: F32 accumulator (bits 4-5 = 1),
    // A and B TF32 (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bit 17,
    // M >> 4 at bit 24.
    template <int N>
    __host__ __device__ constexpr uint32_t instr_desc()
    {
      return (1u << 4) | (2u << 7) | (2u << 10) | (uint32_t(N >> 3) << 17) | (uint32_t(M >> 4) << 24);
    }

    __device__ __forceinline__ bool mbar_try_wait(uint32_t addr, uint32_t phase)
    {
      uint32_t ok;
      asm volatile("{\n\t.reg .pred P1;\n\t"
                   "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
                   "selp.b32 %0, 1, 0, P1;\n\t}"
                   : "=r"(ok)
                   : "r"(addr), "r"(phase)
                   : "memory");
      return ok != 0;
    }

    // false if the phase did not complete within ~2e9 cycles
    __device__ __forceinline__ bool mbar_wait_bounded(uint32_t addr, uint32_t phase)
    {
      const long long t0 = clock64();
      while (!mbar_try_wait(addr, phase))
        if (clock64() - t0 > 2000000000ll)
          return false;
      return true;
    }

    // N = GEMM width (16 or 32), Cout <= N output channels are stored (weights of the rest are zero).
    // Queue the patch of output tile (b, y0, x0) into sP with 4-byte cp.async
    // copies (zero-filled outside the image and for padded channels) and
    // commit them as one group.  Consecutive threads take consecutive patch
    // positions of one channel, so a warp's loads are row segments.
    __device__ __forceinline__ void load_patch(const float *__restrict__ in, int Cin, int H, int W, int KC, int b,
                                               int y0, int x0, uint32_t sP)
    {
      const int    HW  = H * W;
      const float *inb = in + size_t(b) * Cin * HW;
      const int    n   = KC * 4 * PY * PX;
      for (int i = threadIdx.x; i < n; i += THREADS)
        {
          const int  pos = i % (PY * PX), ce = i / (PY * PX); // ce = 4 kc + e = channel
          const int  y = y0 + pos / PX - 1, x = x0 + pos % PX - 1;
          const bool ok = ce < Cin && y >= 0 && y < H && x >= 0 && x < W;
          const float   *src = ok ? inb + size_t(ce) * HW + y * W + x : inb;
          const uint32_t dst = sP + uint32_t(((ce >> 2) * PY * PX + pos) * 16 + (ce & 3) * 4);
          asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(ok ? 4 : 0)
                       : "memory");
        }
      asm volatile("cp.async.commit_group;" ::: "memory");
    }

    template <int N>
    __global__ void __launch_bounds__(THREADS, CTAS_PER_SM)
      conv3x3_tc_kernel(const float *__restrict__ in, int B, int Cin, int H, int W, const float *__restrict__ w,
                        const float *__restrict__ bias, float *__restrict__ out, int Cout, int accumulate,
                        const float *__restrict__ addend, int add_group, int act, float slope, int *status)
    {
      extern __shared__ __align__(1024) unsigned char smem_raw[];
      const int KC = chunks_of(Cin);                           // 4-channel chunks per tap
      // [2][KC][PY][PX] patches, [9][KC][N] weights
      float4   *sB = reinterpret_cast<float4 *>(smem_raw + 2 * patch_bytes(KC));
      uint64_t *mbar    = reinterpret_cast<uint64_t *>(smem_raw + 2 * patch_bytes(KC) + weight_bytes(KC, N));
      uint32_t *s_taddr = reinterpret_cast<uint32_t *>(mbar + 1);
      const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int K9 = Cin * 9;

      // weights once per CTA: sB[t][kc][n] = w[n][4 kc .. 4 kc + 3][t] (0 for padded channels and n >= Cout)
      for (int i = threadIdx.x; i < 9 * KC * N; i += THREADS)
        {
          const int  n = i % N, kc = (i / N) % KC, t = i / (N * KC), c0 = 4 * kc;
          const bool on = n < Cout;
          float4     v;
          v.x = on && c0 + 0 < Cin ? w[n * K9 + (c0 + 0) * 9 + t] : 0.f;
          v.y = on && c0 + 1 < Cin ? w[n * K9 + (c0 + 1) * 9 + t] : 0.f;
          v.z = on && c0 + 2 < Cin ? w[n * K9 + (c0 + 2) * 9 + t] : 0.f;
          v.w = on && c0 + 3 < Cin ? w[n * K9 + (c0 + 3) * 9 + t] : 0.f;
          sB[i] = v;
        }
      if (warp == 0)
        {
          asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(s_taddr)),
                       "r"(TMEM_COLS));
          asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
        }
      if (threadIdx.x == 0)
        {
          asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(mbar)), "r"(1) : "memory");
          asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t taddr = *s_taddr;
      const uint32_t pbase = smem_u32(smem_raw), b0 = smem_u32(sB), mb = smem_u32(mbar);
      const uint32_t pbytes = uint32_t(patch_bytes(KC));

      const int       HW = H * W, tiles_x = (W + TX - 1) / TX, tiles_img = tiles_x * ((H + TY - 1) / TY);
      const long long n_tiles = (long long)B * tiles_img;
      auto            origin  = [&](long long tile, int &b, int &y0, int &x0) {
        b              = int(tile / tiles_img);
        const int tt   = int(tile - (long long)b * tiles_img);
        y0             = (tt / tiles_x) * TY;
        x0             = (tt % tiles_x) * TX;
      };
      uint32_t phase = 0;
      bool     failed = false;
      int      buf = 0;
      // this thread's epilogue columns never change: keep their biases in registers
      constexpr int NH = N / 2;
      const int     c0 = (warp >> 2) * NH;
      float         bias_r[NH];
#pragma unroll
      for (int j = 0; j < NH; ++j)
        bias_r[j] = (bias && c0 + j < Cout) ? bias[c0 + j] : 0.f;
      if (blockIdx.x < n_tiles)
        {
          int b, y0, x0;
          origin(blockIdx.x, b, y0, x0);
          load_patch(in, Cin, H, W, KC, b, y0, x0, pbase);
        }
      for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, buf ^= 1)
        {
          int b, y0, x0;
          origin(tile, b, y0, x0);
          const uint32_t p0 = pbase + uint32_t(buf) * pbytes;
          // queue the next tile's patch into the other buffer (its last MMAs completed a tile ago)
          if (tile + gridDim.x < n_tiles)
            {
              int nb, ny0, nx0;
              origin(tile + gridDim.x, nb, ny0, nx0);
              load_patch(in, Cin, H, W, KC, nb, ny0, nx0, pbase + uint32_t(buf ^ 1) * pbytes);
              asm volatile("cp.async.wait_group 1;" ::: "memory");
            }
          else
            asm volatile("cp.async.wait_group 0;" ::: "memory");
          // generic-proxy smem writes -> visible to the tensor core's async proxy
          asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
          asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
          __syncthreads();
          if (threadIdx.x == 0)
            {
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
              constexpr uint32_t idesc = instr_desc<N>();
              constexpr uint32_t lbo_a = PY * PX * 16, sbo_a = PX * 16;
              for (int t = 0; t < 9; ++t)
                {
                  const uint32_t shift = uint32_t((t / 3) * PX + (t % 3)) * 16;
                  for (int s = 0; s < KC / 2; ++s)
                    {
                      const uint64_t ad = smem_desc(p0 + uint32_t(2 * s) * lbo_a + shift, lbo_a, sbo_a);
                      const uint64_t bd = smem_desc(b0 + uint32_t(t * KC + 2 * s) * N * 16, N * 16, 128);
                      const uint32_t acc = (t | s) != 0;
                      asm volatile("{\n\t.reg .pred p;\n\t"
                                   "setp.ne.b32 p, %4, 0;\n\t"
                                   "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(taddr),
                                   "l"(ad), "l"(bd), "r"(idesc), "r"(acc));
                    }
                }
              asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mb)
                           : "memory");
            }
          // the decision to stop is taken by the whole block (a barrier with a vote), never by a thread alone
          if (__syncthreads_or(!mbar_wait_bounded(mb, phase)))
            {
              failed = true;
              break;
            }
          phase ^= 1u;
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          // epilogue: warp w reads TMEM lanes 32 (w % 4) .. + 31 (pixels), columns (w / 4) N/2 .. + N/2 - 1
          {
            const int      row  = 32 * (warp & 3) + lane;
            const uint32_t addr = taddr + (uint32_t(32 * (warp & 3)) << 16) + uint32_t(c0);
            uint32_t       d[NH];
            if constexpr (NH == 16)
              asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                           "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                           : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                             "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]), "=r"(d[13]),
                             "=r"(d[14]), "=r"(d[15])
                           : "r"(addr));
            else
              asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
                           : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                             "=r"(d[7])
                           : "r"(addr));
            asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
            const int y = y0 + row / TX, x = x0 + row % TX;
            if (y < H && x < W)
              {
                float *ob = out + size_t(b) * Cout * HW + y * W + x;
#pragma unroll
                for (int j = 0; j < NH; ++j)
                  {
                    const int co = c0 + j;
                    if (co >= Cout)
                      break;
                    float v = __uint_as_float(d[j]) + bias_r[j];
                    if (accumulate)
                      v += ob[size_t(co) * HW];
                    if (addend) // one addend image per group of add_group batch entries
                      v += addend[(size_t(b / add_group) * Cout + co) * HW + y * W + x];
                    if (act)
                      v = v > 0.f ? v : slope * v;
                    ob[size_t(co) * HW] = v;
                  }
              }
          }
        }
      asm volatile("cp.async.wait_all;" ::: "memory"); // no copy may still target this CTA's shared memory
      if (failed && threadIdx.x == 0)
        atomicExch(status, 1);
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      if (warp == 0)
        {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(TMEM_COLS));
        }
    }
  } // namespace tc
} // namespace sint

using namespace sint;

namespace
{
  template <int N>
  int launch_tc(const float *in, int B, int Cin, int H, int W, const float *w, const float *bias, float *out, int Cout,
                int accumulate, const float *addend, int add_group, int act, float slope, int *status,
                cudaStream_t s)
  {
    static int grid_cap = 0;
    auto       k        = tc::conv3x3_tc_kernel<N>;
    if (grid_cap == 0)
      {
        int         dev = 0, sms = 0;
        const int   smax = int(tc::smem_bytes(tc::chunks_of(tc::CIN_MAX), N));
        cudaError_t e    = cudaGetDevice(&dev);
        if (e == cudaSuccess)
          e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (e == cudaSuccess)
          e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
        if (e == cudaSuccess) // all of the unified L1 / shared storage as shared memory
          e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
        if (e != cudaSuccess)
          return cuda_fail(e, "sint_nn_conv3x3_tc_f32: setup");
        // two CTAs per SM: the launch bound caps registers at 128 and the largest
        // configuration takes 83 KB of shared memory, so both fit on every SM
        grid_cap = sms * tc::CTAS_PER_SM;
      }
    const int       KC    = tc::chunks_of(Cin);
    const long long tiles = (long long)B * ((H + tc::TY - 1) / tc::TY) * ((W + tc::TX - 1) / tc::TX);
    const int       grid  = int(tiles < grid_cap ? tiles : grid_cap);
    k<<<grid, tc::THREADS, tc::smem_bytes(KC, N), s>>>(in, B, Cin, H, W, w, bias, out, Cout, accumulate, addend,
                                                       add_group, act, slope, status);
    count_launches(1);
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_nn_conv3x3_tc_f32");
  }
} // namespace

extern "C" {

int sint_nn_conv3x3_tc_ex_f32(const float *in, int B, int Cin, int H, int W, const float *w, const float *bias,
                              float *out, int Cout, int accumulate, const float *addend, int addend_group,
                              int leaky, float slope, int *status, sint_stream_t s)
{
  if (!in || !w || !out || !status || B < 1 || Cin < 1 || Cin > tc::CIN_MAX || Cout < 1 || Cout > tc::NMAX || H < 1 ||
      W < 1 || (addend && (addend_group < 1 || B % addend_group != 0)))
    {
      set_error("sint_nn_conv3x3_tc_f32: bad argument (needs 1 <= Cin <= 32, 1 <= Cout <= 32, "
                "addend_group dividing B)");
      return SINT_ERR_ARG;
    }
  return Cout <= 16 ? launch_tc<16>(in, B, Cin, H, W, w, bias, out, Cout, accumulate, addend, addend_group, leaky,
                                    slope, status, s)
                    : launch_tc<32>(in, B, Cin, H, W, w, bias, out, Cout, accumulate, addend, addend_group, leaky,
                                    slope, status, s);
}

int sint_nn_conv3x3_tc_f32(const float *in, int B, int Cin, int H, int W, const float *w, const float *bias,
                           float *out, int Cout, int accumulate, int *status, sint_stream_t s)
{
  return sint_nn_conv3x3_tc_ex_f32(in, B, Cin, H, W, w, bias, out, Cout, accumulate, nullptr, 1, 0, 0.f, status, s);
}

} // extern "C"
