// Definitions of the launchers declared in sint_launch.h; included by the
// sint_inst_*.cu translation units, each of which instantiates one
// (dimension, mobility) combination for all grain counts.
#pragma once
#include <type_traits>

#include "sint_kernels.cuh"
#include "sint_launch.h"

namespace sint
{
  // Dynamic shared memory above the 48 KB default, and a shared-memory
  // carveout just large enough for `blocks` resident blocks (the rest of the
  // unified storage stays L1).
  template <typename Kernel>
  inline cudaError_t prepare_smem(Kernel k, size_t bytes, int blocks = 2)
  {
    cudaError_t e = cudaSuccess;
    if (bytes > 48 * 1024 && (e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, int(bytes))) !=
                               cudaSuccess)
      return e;
    int                dev = 0, per_sm = 0;
    cudaFuncAttributes fa{};
    if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
        (e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess ||
        (e = cudaFuncGetAttributes(&fa, k)) != cudaSuccess)
      return e;
    // dynamic + static shared memory + the per-block reservation
    const size_t need = size_t(blocks) * (bytes + fa.sharedSizeBytes + 1024);
    const int    pct  = need >= size_t(per_sm) ? 100 : int((need * 100 + per_sm - 1) / per_sm);
    return cudaFuncSetAttribute(k, cudaFuncAttributePreferredSharedMemoryCarveout, pct);
  }

  // Persistent grid of kernel k on the current device: its shared-memory
  // attributes set, as many blocks as are resident at once (once per device).
  template <typename Kernel>
  inline cudaError_t persistent_grid(DeviceCache &cache, Kernel k, size_t smem, int blocks_per_sm, int threads,
                                     int &grid_cap)
  {
    return per_device(cache, grid_cap, [&](int dev, int &cap) {
      cudaError_t e = prepare_smem(k, smem, blocks_per_sm);
      int         sms = 0, per_sm = 0;
      if (e != cudaSuccess || (e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess ||
          (e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem)) != cudaSuccess)
        return e;
      cap = sms * (per_sm > 0 ? per_sm : 1);
      return cudaSuccess;
    });
  }

  template <int DIM, int G, bool TENS, typename R, bool CUT, bool ADV>
  cudaError_t launch_jvp_g(const Grid &g, const Phys &p, const R *lin, const R *src, R *dst, R *partial,
                           const CutTiles &ct, const AdvData &adv, cudaStream_t s)
  {
    const size_t smem = ThreePhaseSmem<DIM, G, TENS, true, false, ADV>::TOTAL * sizeof(R);
    auto         k    = jvp_kernel<DIM, G, TENS, R, CUT, ADV>;
    static DeviceCache cache;
    int                grid_cap = 0;
    if (const cudaError_t e =
          persistent_grid(cache, k, smem, jvp_blocks_per_sm<DIM, G, R>(), Tile<DIM>::THREADS, grid_cap))
      return e;
    const long long blocks = g.n_tiles < grid_cap ? g.n_tiles : grid_cap;
    k<<<dim3((unsigned)blocks), Tile<DIM>::THREADS, smem, s>>>(g, p, lin, src, dst, partial, ct, adv);
    count_launches(1);
    return cudaGetLastError();
  }

  template <int DIM, int G, bool TENS, bool CUT = false>
  cudaError_t launch_jvp_pair_g(const Grid &g, const Phys &p, const float *lin, const float *src, float *dst,
                                float *partial, cudaStream_t s, const CutTiles &ct = CutTiles())
  {
    const size_t smem = ThreePhaseSmem<DIM, G, TENS, true, false, false>::TOTAL * sizeof(F2);
    auto         k    = jvp_pair_kernel<DIM, G, TENS, CUT>;
    static DeviceCache cache;
    int                grid_cap = 0;
    if (const cudaError_t e =
          persistent_grid(cache, k, smem, jvp_pair_blocks_per_sm<DIM, G>(), Tile<DIM>::THREADS, grid_cap))
      return e;
    // the class size of the cut-off lives on the device: a full persistent grid
    const long long pairs  = CUT ? (long long)grid_cap : (g.n_tiles + 1) / 2;
    const long long blocks = pairs < grid_cap ? pairs : grid_cap;
    k<<<dim3((unsigned)blocks), Tile<DIM>::THREADS, smem, s>>>(g, p, lin, src, dst, partial, ct);
    count_launches(1);
    return cudaGetLastError();
  }

  template <int DIM, int G, bool TENS, int WTD, bool CUT, bool ADV>
  cudaError_t launch_residual_g(const Grid &g, const Phys &p, const double *src, const double *const *hist,
                                double *dst, double *partial, const CutTiles &ct, const AdvData &adv,
                                cudaStream_t s)
  {
    const size_t  smem     = ThreePhaseSmem<DIM, G, TENS, false, WTD == 2, ADV>::TOTAL * sizeof(double);
    auto          k        = residual_kernel<DIM, G, TENS, WTD, CUT, ADV>;
    static DeviceCache cache;
    int                grid_cap = 0;
    if (const cudaError_t e =
          persistent_grid(cache, k, smem, residual_blocks_per_sm<DIM, G>(), Tile<DIM>::THREADS, grid_cap))
      return e;
    const double *h0     = WTD == 2 ? hist[0] : nullptr;
    const double *h1     = (WTD == 2 && p.order > 1) ? hist[1] : nullptr;
    const double *h2     = (WTD == 2 && p.order > 2) ? hist[2] : nullptr;
    const long long blocks = g.n_tiles < grid_cap ? g.n_tiles : grid_cap;
    k<<<dim3((unsigned)blocks), Tile<DIM>::THREADS, smem, s>>>(g, p, src, h0, h1, h2, dst, partial, ct, adv);
    count_launches(1);
    return cudaGetLastError();
  }

  template <int DIM, int G, bool TENS, bool CUT, bool ADV>
  cudaError_t launch_diag_g(const Grid &g, const Phys &p, const double *lin, double *dst, double *partial,
                            const uint16_t *mask, const AdvData &adv, cudaStream_t s)
  {
    const size_t smem = smem_diag(DIM, G, ADV);
    auto         k    = diag_kernel<DIM, G, TENS, CUT, ADV>;
    cudaError_t  e    = prepare_smem(k, smem);
    if (e != cudaSuccess)
      return e;
    k<<<dim3((unsigned)g.n_tiles), Tile<DIM>::THREADS, smem, s>>>(g, p, lin, dst, partial, mask, adv);
    count_launches(1);
    return cudaGetLastError();
  }

#define SINT_G_SWITCH(CALL)                                                                                       \
  switch (G)                                                                                                      \
    {                                                                                                             \
      case 1: return CALL(1);                                                                                     \
      case 2: return CALL(2);                                                                                     \
      case 3: return CALL(3);                                                                                     \
      case 4: return CALL(4);                                                                                     \
      case 5: return CALL(5);                                                                                     \
      case 6: return CALL(6);                                                                                     \
      case 7: return CALL(7);                                                                                     \
      case 8: return CALL(8);                                                                                     \
      case 9: return CALL(9);                                                                                     \
      case 10: return CALL(10);                                                                                   \
      case 11: return CALL(11);                                                                                   \
      case 12: return CALL(12);                                                                                   \
      default: return cudaErrorInvalidValue;                                                                      \
    }

  // The same over the grain-count classes 0..12 of the grain cut-off.
#define SINT_CLASS_SWITCH(K, CALL)                                                                                \
  switch (K)                                                                                                      \
    {                                                                                                             \
      case 0: return CALL(0);                                                                                     \
      case 1: return CALL(1);                                                                                     \
      case 2: return CALL(2);                                                                                     \
      case 3: return CALL(3);                                                                                     \
      case 4: return CALL(4);                                                                                     \
      case 5: return CALL(5);                                                                                     \
      case 6: return CALL(6);                                                                                     \
      case 7: return CALL(7);                                                                                     \
      case 8: return CALL(8);                                                                                     \
      case 9: return CALL(9);                                                                                     \
      case 10: return CALL(10);                                                                                   \
      case 11: return CALL(11);                                                                                   \
      case 12: return CALL(12);                                                                                   \
      default: return cudaErrorInvalidValue;                                                                      \
    }

  template <int DIM, bool TENS, typename R, bool ADV>
  cudaError_t launch_jvp_class(int K, const Grid &g, const Phys &p, const R *lin, const R *src, R *dst, R *partial,
                               const CutTiles &ct, const AdvData &adv, cudaStream_t s)
  {
    // FP32: the class without grains (c and mu only, the bulk of a packing's
    // vapour) runs on tile pairs
    if constexpr (std::is_same_v<R, float> && !ADV)
      if (K == 0)
        return launch_jvp_pair_g<DIM, 0, TENS, true>(g, p, lin, src, dst, partial, s, ct);
#define SINT_CALL(GG) launch_jvp_g<DIM, GG, TENS, R, true, ADV>(g, p, lin, src, dst, partial, ct, adv, s)
    SINT_CLASS_SWITCH(K, SINT_CALL)
#undef SINT_CALL
  }

  // cut == nullptr: the full operator; otherwise the grain cut-off, one
  // launch per grain-count class 0..G (classes without tiles return at once).
  // ADV: the kernels with the advection terms.
  template <int DIM, bool TENS, typename R, bool ADV>
  cudaError_t launch_jvp_impl(int G, const Grid &g, const Phys &p, const R *lin, const R *src, R *dst, R *partial,
                              const CutTiles *cut, const AdvData &adv, cudaStream_t s)
  {
    if (cut)
      {
        for (int K = 0; K <= G; ++K)
          if (const cudaError_t e =
                launch_jvp_class<DIM, TENS, R, ADV>(K, g, p, lin, src, dst, partial, *cut, adv, s))
            return e;
        return cudaSuccess;
      }
    if constexpr (std::is_same_v<R, float> && !ADV)
      {
        // the full FP32 operator runs on tile pairs (packed FP32)
#define SINT_CALL(GG) launch_jvp_pair_g<DIM, GG, TENS>(g, p, lin, src, dst, partial, s)
        SINT_G_SWITCH(SINT_CALL)
#undef SINT_CALL
      }
    else
      {
        const CutTiles none;
#define SINT_CALL(GG) launch_jvp_g<DIM, GG, TENS, R, false, ADV>(g, p, lin, src, dst, partial, none, adv, s)
        SINT_G_SWITCH(SINT_CALL)
#undef SINT_CALL
      }
  }

  // The advection kernels are instantiated in their own translation units
  // (launch_jvp_adv, launch_residual_adv).
  template <int DIM, bool TENS, typename R>
  cudaError_t launch_jvp(int G, const Grid &g, const Phys &p, const R *lin, const R *src, R *dst, R *partial,
                         const CutTiles *cut, const AdvData *adv, cudaStream_t s)
  {
    if (adv)
      return launch_jvp_adv<DIM, TENS, R>(G, g, p, lin, src, dst, partial, cut, *adv, s);
    return launch_jvp_impl<DIM, TENS, R, false>(G, g, p, lin, src, dst, partial, cut, AdvData(), s);
  }

  // G = the grain count (full operator, 1..12) or the class (grain cut-off, 0..12)
  template <int DIM, bool TENS, bool CUT, int WTD, bool ADV>
  cudaError_t launch_residual_w(int G, const Grid &g, const Phys &p, const double *src, const double *const *hist,
                                double *dst, double *partial, const CutTiles &ct, const AdvData &adv,
                                cudaStream_t s)
  {
#define SINT_CALL(GG) launch_residual_g<DIM, GG, TENS, WTD, CUT, ADV>(g, p, src, hist, dst, partial, ct, adv, s)
    if constexpr (CUT)
      {
        SINT_CLASS_SWITCH(G, SINT_CALL)
      }
    else
      {
        SINT_G_SWITCH(SINT_CALL)
      }
#undef SINT_CALL
  }

  template <int DIM, bool TENS, bool CUT, bool ADV>
  cudaError_t launch_residual_c(int G, int wtd, const Grid &g, const Phys &p, const double *src,
                                const double *const *hist, double *dst, double *partial, const CutTiles &ct,
                                const AdvData &adv, cudaStream_t s)
  {
    if (wtd == 0)
      return launch_residual_w<DIM, TENS, CUT, 0, ADV>(G, g, p, src, hist, dst, partial, ct, adv, s);
    if (wtd == 1)
      return launch_residual_w<DIM, TENS, CUT, 1, ADV>(G, g, p, src, hist, dst, partial, ct, adv, s);
    return launch_residual_w<DIM, TENS, CUT, 2, ADV>(G, g, p, src, hist, dst, partial, ct, adv, s);
  }

  template <int DIM, bool TENS, bool ADV>
  cudaError_t launch_residual_impl(int G, int wtd, const Grid &g, const Phys &p, const double *src,
                                   const double *const *hist, double *dst, double *partial, const CutTiles *cut,
                                   const AdvData &adv, cudaStream_t s)
  {
    if (cut)
      {
        for (int K = 0; K <= G; ++K)
          if (const cudaError_t e =
                launch_residual_c<DIM, TENS, true, ADV>(K, wtd, g, p, src, hist, dst, partial, *cut, adv, s))
            return e;
        return cudaSuccess;
      }
    return launch_residual_c<DIM, TENS, false, ADV>(G, wtd, g, p, src, hist, dst, partial, CutTiles(), adv, s);
  }

  template <int DIM, bool TENS>
  cudaError_t launch_residual(int G, int wtd, const Grid &g, const Phys &p, const double *src,
                              const double *const *hist, double *dst, double *partial, const CutTiles *cut,
                              const AdvData *adv, cudaStream_t s)
  {
    if (adv)
      return launch_residual_adv<DIM, TENS>(G, wtd, g, p, src, hist, dst, partial, cut, *adv, s);
    return launch_residual_impl<DIM, TENS, false>(G, wtd, g, p, src, hist, dst, partial, cut, AdvData(), s);
  }

  template <int DIM, bool TENS, bool ADV>
  cudaError_t launch_diag_impl(int G, const Grid &g, const Phys &p, const double *lin, double *dst, double *partial,
                               const uint16_t *mask, const AdvData &adv, cudaStream_t s)
  {
    if (mask)
      {
#define SINT_CALL(GG) launch_diag_g<DIM, GG, TENS, true, ADV>(g, p, lin, dst, partial, mask, adv, s)
        SINT_G_SWITCH(SINT_CALL)
#undef SINT_CALL
      }
#define SINT_CALL(GG) launch_diag_g<DIM, GG, TENS, false, ADV>(g, p, lin, dst, partial, nullptr, adv, s)
    SINT_G_SWITCH(SINT_CALL)
#undef SINT_CALL
  }

  template <int DIM, bool TENS>
  cudaError_t launch_diag(int G, const Grid &g, const Phys &p, const double *lin, double *dst, double *partial,
                          const uint16_t *mask, const AdvData *adv, cudaStream_t s)
  {
    if (adv)
      return launch_diag_adv<DIM, TENS>(G, g, p, lin, dst, partial, mask, *adv, s);
    return launch_diag_impl<DIM, TENS, false>(G, g, p, lin, dst, partial, mask, AdvData(), s);
  }
} // namespace sint
