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
// accumulating into a 32-column TMEM tile.  The weights sit in shared memory
// as B[tap][kc][co] chunks for the whole kernel.  Loader warps, one MMA
// thread and epilogue warps form a pipeline through mbarriers (a ring of
// patch buffers, two TMEM accumulators; see the kernel).  TF32 reads the FP32
// bit patterns directly.
//
// Every wait is bounded: a CTA whose pipeline stalls for about a second
// records a status, frees its TMEM and returns.
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
    // Warp-specialised pipeline (256 threads):
    //   warp 0, lane 0   MMA issuer: waits for a loaded patch and a free
    //                    accumulator, issues the tile's 9 * KC/2 MMAs, commits
    //                    them to the accumulator's "done" and the stage's
    //                    "empty" barriers;
    //   warps 1-3        loaders: 4-byte cp.async copies of the patch into a
    //                    ring of STAGES buffers; a stage is announced "full"
    //                    once the copies of the tile after it are queued
    //                    (so two tiles' copies are in flight);
    //   warps 4-7        epilogue: read accumulator (tile & 1) with
    //                    tcgen05.ld (warp w: TMEM lanes 32 (w - 4) ..), free
    //                    it, then add bias / output / addend, apply the
    //                    activation and store NCHW.
    // Two 32-column accumulators, so tile k + 1's MMAs run during tile k's
    // epilogue.  Every wait gives up after ~1 s or when another role has
    // failed; the CTA then records a status, frees its TMEM and returns.
    constexpr int STAGES = 3, LOADERS = 96, EPI0 = 128;

    __host__ __device__ constexpr size_t ws_smem_bytes(int kc, int n)
    {
      return STAGES * patch_bytes(kc) + weight_bytes(kc, n) + 8 * (2 * STAGES + 4) + 16;
    }

    __device__ __forceinline__ void mbar_init(uint32_t addr, int count)
    {
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(addr), "r"(count) : "memory");
    }

    __device__ __forceinline__ void mbar_arrive(uint32_t addr)
    {
      asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(addr) : "memory");
    }

    // try_wait with a suspend-time hint: the thread sleeps in hardware until
    // the phase completes or ~1 ms passes, instead of spinning on issue slots
    __device__ __forceinline__ bool mbar_try_wait_sleep(uint32_t addr, uint32_t phase)
    {
      uint32_t ok;
      asm volatile("{\n\t.reg .pred P1;\n\t"
                   "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2, %3;\n\t"
                   "selp.b32 %0, 1, 0, P1;\n\t}"
                   : "=r"(ok)
                   : "r"(addr), "r"(phase), "r"(1000000u)
                   : "memory");
      return ok != 0;
    }

    // wait for the phase of parity `phase`; false on timeout or when *fail is set
    __device__ __forceinline__ bool mbar_wait_ws(uint32_t addr, uint32_t phase, volatile int *fail)
    {
      const long long t0 = clock64();
      while (!mbar_try_wait_sleep(addr, phase))
        {
          if (*fail)
            return false;
          if (clock64() - t0 > 2000000000ll)
            {
              *fail = 1;
              return false;
            }
        }
      return true;
    }

    template <int N>
    __global__ void __launch_bounds__(THREADS, CTAS_PER_SM)
      conv3x3_tc_kernel(const float *__restrict__ in, int B, int Cin, int H, int W, const float *__restrict__ w,
                        const float *__restrict__ bias, float *__restrict__ out, int Cout, int accumulate,
                        const float *__restrict__ addend, int add_group, int act, float slope, int *status)
    {
      extern __shared__ __align__(1024) unsigned char smem_raw[];
      const int KC = chunks_of(Cin); // 4-channel chunks per tap
      // [STAGES][KC][PY][PX] patches, [9][KC][N] weights, barriers, TMEM address
      const size_t pb   = patch_bytes(KC);
      float4      *sB   = reinterpret_cast<float4 *>(smem_raw + STAGES * pb);
      uint64_t    *bars = reinterpret_cast<uint64_t *>(smem_raw + STAGES * pb + weight_bytes(KC, N));
      // bars: full[STAGES], empty[STAGES], done[2], free[2]
      uint32_t     *s_taddr = reinterpret_cast<uint32_t *>(bars + 2 * STAGES + 4);
      __shared__ int s_fail;
      const int      warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
      const int      K9   = Cin * 9;

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
                       "r"(2 * TMEM_COLS));
          asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
        }
      const uint32_t bar0 = smem_u32(bars);
      auto full  = [&](int s) { return bar0 + 8u * uint32_t(s); };
      auto empty = [&](int s) { return bar0 + 8u * uint32_t(STAGES + s); };
      auto done  = [&](int a) { return bar0 + 8u * uint32_t(2 * STAGES + a); };
      auto freed = [&](int a) { return bar0 + 8u * uint32_t(2 * STAGES + 2 + a); };
      if (threadIdx.x == 0)
        {
          for (int s = 0; s < STAGES; ++s)
            {
              mbar_init(full(s), LOADERS);
              mbar_init(empty(s), 1);
            }
          for (int a = 0; a < 2; ++a)
            {
              mbar_init(done(a), 1);
              mbar_init(freed(a), THREADS - EPI0);
            }
          s_fail = 0;
          asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
      // generic-proxy weight stores -> visible to the tensor core
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      __syncthreads();
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      const uint32_t taddr = *s_taddr;
      const uint32_t pbase = smem_u32(smem_raw), b0 = smem_u32(sB);
      volatile int  *fail  = &s_fail;

      const int       HW = H * W, tiles_x = (W + TX - 1) / TX, tiles_img = tiles_x * ((H + TY - 1) / TY);
      const long long n_tiles = (long long)B * tiles_img;
      auto            origin  = [&](long long tile, int &b, int &y0, int &x0) {
        b            = int(tile / tiles_img);
        const int tt = int(tile - (long long)b * tiles_img);
        y0           = (tt / tiles_x) * TY;
        x0           = (tt % tiles_x) * TX;
      };

      if (warp == 0)
        {
          if (lane == 0)
            {
              // --- MMA issuer ---
              constexpr uint32_t idesc = instr_desc<N>();
              constexpr uint32_t lbo_a = PY * PX * 16, sbo_a = PX * 16;
              int                k     = 0;
              for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++k)
                {
                  const int st = k % STAGES, acc = k & 1;
                  if (!mbar_wait_ws(full(st), uint32_t((k / STAGES) & 1), fail) ||
                      !mbar_wait_ws(freed(acc), uint32_t(((k >> 1) & 1) ^ 1), fail))
                    break;
                  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
                  const uint32_t p0 = pbase + uint32_t(st) * uint32_t(pb);
                  const uint32_t d  = taddr + uint32_t(acc * TMEM_COLS);
                  for (int t = 0; t < 9; ++t)
                    {
                      const uint32_t shift = uint32_t((t / 3) * PX + (t % 3)) * 16;
                      for (int s = 0; s < KC / 2; ++s)
                        {
                          const uint64_t ad = smem_desc(p0 + uint32_t(2 * s) * lbo_a + shift, lbo_a, sbo_a);
                          const uint64_t bd = smem_desc(b0 + uint32_t(t * KC + 2 * s) * N * 16, N * 16, 128);
                          const uint32_t en = (t | s) != 0;
                          asm volatile("{\n\t.reg .pred p;\n\t"
                                       "setp.ne.b32 p, %4, 0;\n\t"
                                       "tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
                                       "l"(ad), "l"(bd), "r"(idesc), "r"(en));
                        }
                    }
                  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 done(acc))
                               : "memory");
                  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                                 empty(st))
                               : "memory");
                }
              // the last "empty" arrival lands before this CTA's shared memory goes away
              if (k > 0)
                mbar_wait_ws(empty((k - 1) % STAGES), uint32_t(((k - 1) / STAGES) & 1), fail);
            }
        }
      else if (warp < 4)
        {
          // --- loaders ---
          const int t   = threadIdx.x - 32;
          const int n   = KC * 4 * PY * PX;
          int       k   = 0;
          bool      ok_ = true;
          for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++k)
            {
              const int st = k % STAGES;
              if (!mbar_wait_ws(empty(st), uint32_t(((k / STAGES) & 1) ^ 1), fail))
                {
                  ok_ = false;
                  break;
                }
              int b, y0, x0;
              origin(tile, b, y0, x0);
              const float   *inb = in + size_t(b) * Cin * HW;
              const uint32_t sP  = pbase + uint32_t(st) * uint32_t(pb);
              for (int i = t; i < n; i += LOADERS)
                {
                  const int  pos = i % (PY * PX), ce = i / (PY * PX);
                  const int  y = y0 + pos / PX - 1, x = x0 + pos % PX - 1;
                  const bool ok = ce < Cin && y >= 0 && y < H && x >= 0 && x < W;
                  const float   *src = ok ? inb + size_t(ce) * HW + y * W + x : inb;
                  const uint32_t dst = sP + uint32_t(((ce >> 2) * PY * PX + pos) * 16 + (ce & 3) * 4);
                  asm volatile("cp.async.ca.shared.global [%0], [%1], 4, %2;" ::"r"(dst), "l"(src), "r"(ok ? 4 : 0)
                               : "memory");
                }
              asm volatile("cp.async.commit_group;" ::: "memory");
              if (k >= 1)
                {
                  // the previous tile's copies are complete: announce its stage
                  asm volatile("cp.async.wait_group 1;" ::: "memory");
                  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                  mbar_arrive(full((k - 1) % STAGES));
                }
            }
          asm volatile("cp.async.wait_group 0;" ::: "memory");
          if (ok_ && k >= 1)
            {
              asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
              mbar_arrive(full((k - 1) % STAGES));
            }
        }
      else
        {
          // --- epilogue ---
          const int q = warp - 4, row = 32 * q + lane;
          float     bias_r[N];
#pragma unroll
          for (int j = 0; j < N; ++j)
            bias_r[j] = (bias && j < Cout) ? bias[j] : 0.f;
          int k = 0;
          for (long long tile = blockIdx.x; tile < n_tiles; tile += gridDim.x, ++k)
            {
              const int acc = k & 1;
              if (!mbar_wait_ws(done(acc), uint32_t((k >> 1) & 1), fail))
                break;
              asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
              const uint32_t addr = taddr + (uint32_t(32 * q) << 16) + uint32_t(acc * TMEM_COLS);
              uint32_t       d[N];
              if constexpr (N == 32)
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 "
                             "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                             "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                             : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                               "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]),
                               "=r"(d[13]), "=r"(d[14]), "=r"(d[15]), "=r"(d[16]), "=r"(d[17]), "=r"(d[18]),
                               "=r"(d[19]), "=r"(d[20]), "=r"(d[21]), "=r"(d[22]), "=r"(d[23]), "=r"(d[24]),
                               "=r"(d[25]), "=r"(d[26]), "=r"(d[27]), "=r"(d[28]), "=r"(d[29]), "=r"(d[30]),
                               "=r"(d[31])
                             : "r"(addr));
              else
                asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                             "{%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15}, [%16];"
                             : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]),
                               "=r"(d[7]), "=r"(d[8]), "=r"(d[9]), "=r"(d[10]), "=r"(d[11]), "=r"(d[12]),
                               "=r"(d[13]), "=r"(d[14]), "=r"(d[15])
                             : "r"(addr));
              asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
              asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
              mbar_arrive(freed(acc)); // the accumulator may be overwritten now
              int b, y0, x0;
              origin(tile, b, y0, x0);
              const int y = y0 + row / TX, x = x0 + row % TX;
              if (y < H && x < W)
                {
                  float *ob = out + size_t(b) * Cout * HW + y * W + x;
#pragma unroll
                  for (int co = 0; co < N; ++co)
                    {
                      if (co >= Cout)
                        break;
                      float v = __uint_as_float(d[co]) + bias_r[co];
                      if (accumulate)
                        v += ob[size_t(co) * HW];
                      if (addend)
                        v += addend[(size_t(b / add_group) * Cout + co) * HW + y * W + x];
                      if (act)
                        v = v > 0.f ? v : slope * v;
                      ob[size_t(co) * HW] = v;
                    }
                }
            }
        }
      __syncthreads();
      if (threadIdx.x == 0 && s_fail)
        atomicExch(status, 1);
      if (warp == 0)
        {
          asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
          asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(2 * TMEM_COLS));
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
    static DeviceCache cache; // per device: attributes set, grid size
    auto               k        = tc::conv3x3_tc_kernel<N>;
    int                grid_cap = 0;
    const cudaError_t  es       = per_device(cache, grid_cap, [&](int dev, int &cap) {
      int         sms  = 0;
      const int   smax = int(tc::ws_smem_bytes(tc::chunks_of(tc::CIN_MAX), N));
      cudaError_t e    = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, smax);
      if (e == cudaSuccess) // all of the unified L1 / shared storage as shared memory
        e = cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, 100);
      // two CTAs per SM: the launch bound caps registers at 128 and the largest
      // configuration takes 83 KB of shared memory, so both fit on every SM
      cap = sms * tc::CTAS_PER_SM;
      return e;
    });
    if (es != cudaSuccess)
      return cuda_fail(es, "sint_nn_conv3x3_tc_f32: setup");
    const int       KC    = tc::chunks_of(Cin);
    const long long tiles = (long long)B * ((H + tc::TY - 1) / tc::TY) * ((W + tc::TX - 1) / tc::TX);
    const int       grid  = int(tiles < grid_cap ? tiles : grid_cap);
    k<<<grid, tc::THREADS, tc::ws_smem_bytes(KC, N), s>>>(in, B, Cin, H, W, w, bias, out, Cout, accumulate, addend,
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
