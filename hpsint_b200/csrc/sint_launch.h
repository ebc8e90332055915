// Host-side launchers of the cell kernels.  The runtime number of grains is
// mapped onto a compile-time template argument here, the way hpsint's
// EXPAND_OPERATIONS maps n_grains onto n_comp
// (applications/sintering/include/pf-applications/sintering/instantiation.h:97-141).
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdint>

#include "sint_common.cuh"

namespace sint
{
  // Launch set-up that belongs to one device: function attributes live in the
  // device's context, persistent grids follow its SM count.  A kernel keeps
  // one value per device ordinal (0 = not set up yet); `setup(dev, value)`
  // runs once per ordinal, with that device current.  Concurrent first calls
  // may both run the (idempotent) set-up.  A process that resets a device
  // (cudaDeviceReset) must not call this library on it again.
  constexpr int MAX_DEVICES = 64;
  using DeviceCache         = std::atomic<int>[MAX_DEVICES];

  template <typename Setup>
  inline cudaError_t per_device(DeviceCache &cache, int &value, Setup setup)
  {
    int         dev = 0;
    cudaError_t e   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return e;
    if (dev < 0 || dev >= MAX_DEVICES)
      return cudaErrorInvalidDevice;
    int v = cache[dev].load(std::memory_order_acquire);
    if (v == 0)
      {
        if ((e = setup(dev, v)) != cudaSuccess)
          return e;
        cache[dev].store(v, std::memory_order_release);
      }
    value = v;
    return cudaSuccess;
  }

  // Dynamic shared memory of the diagonal kernel (bytes); adv: with the
  // grains' velocities per point.
  size_t smem_diag(int dim, int G, bool adv = false);

  // cut: the grain cut-off's tile classes, nullptr for the full operator;
  // adv: the grains' rigid-body velocities, nullptr for no advection
  template <int DIM, bool TENS, typename R>
  cudaError_t launch_jvp(int G, const Grid &g, const Phys &p, const R *lin, const R *src, R *dst, R *partial,
                         const CutTiles *cut, const AdvData *adv, cudaStream_t s);

  template <int DIM, bool TENS>
  cudaError_t launch_residual(int G, int wtd, const Grid &g, const Phys &p, const double *src,
                              const double *const *hist, double *dst, double *partial, const CutTiles *cut,
                              const AdvData *adv, cudaStream_t s);

  // The same with the advection terms (instantiated in sint_inst_adv_*.cu).
  template <int DIM, bool TENS, typename R>
  cudaError_t launch_jvp_adv(int G, const Grid &g, const Phys &p, const R *lin, const R *src, R *dst, R *partial,
                             const CutTiles *cut, const AdvData &adv, cudaStream_t s);

  template <int DIM, bool TENS>
  cudaError_t launch_residual_adv(int G, int wtd, const Grid &g, const Phys &p, const double *src,
                                  const double *const *hist, double *dst, double *partial, const CutTiles *cut,
                                  const AdvData &adv, cudaStream_t s);

  // mask: the cut-off's per-cell grain masks, nullptr for the full operator;
  // adv: the advection velocities, nullptr for none
  template <int DIM, bool TENS>
  cudaError_t launch_diag(int G, const Grid &g, const Phys &p, const double *lin, double *dst, double *partial,
                          const uint16_t *mask, const AdvData *adv, cudaStream_t s);

  // The same with the advection terms (instantiated in sint_inst_adv_diag_*.cu).
  template <int DIM, bool TENS>
  cudaError_t launch_diag_adv(int G, const Grid &g, const Phys &p, const double *lin, double *dst, double *partial,
                              const uint16_t *mask, const AdvData &adv, cudaStream_t s);

  // tile_mask: per tile id, the grains whose partials the tile wrote (grain
  // cut-off); nullptr = every component of every tile
  // epi: the residual's epilogue hook ((sum - sub) * scale), nullptr for none
  template <int DIM, typename R>
  cudaError_t launch_combine(int ncomp, const Grid &g, const R *partial, R *dst, const uint16_t *tile_mask,
                             cudaStream_t s, const ResidualHooks *epi = nullptr);

  // Periodic constraints after the combine step: slave rows added to their
  // masters, then set to src (mode 0, J v), zero (mode 1, residual) or the
  // identity of the preconditioner's outputs (mode 2).  No-op without
  // periodic directions.
  template <typename R>
  cudaError_t launch_periodic_condense(const Grid &g, int ncomp, R *dst, const R *src, int mode, cudaStream_t s);
  // slaves <- masters (AffineConstraints::distribute)
  cudaError_t launch_periodic_distribute(const Grid &g, int ncomp, double *u, cudaStream_t s);

  // Counts kernel launches issued by this library.
  void count_launches(int n);
} // namespace sint
