// Allocation-free FP64 Jacobian-vector product.
//
// Some callers cannot call cudaMalloc: code that runs while a foreign
// framework owns the device memory pool (and forbids raw allocations), code
// inside callbacks or host functions of a stream, or embedded solvers whose
// memory budget is fixed up front.  sint_jvp_f64_noalloc serves them: it
// takes the mesh, the parameters, the time weights and the linearisation
// point directly (no context), and the only scratch the product needs -- the
// tile-face partial sums between the cell kernel and the combine kernel --
// lives in a fixed device array of this file instead of an allocation.
#include <mutex>
#include <string>

#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  // Scratch of the allocation-free product: tile-face partial sums, at most
  // SINT_NOALLOC_SCRATCH_BYTES.  Every GPU that loads this library holds it
  // until the process exits.  All calls share it.
  static __device__ __align__(256) double noalloc_scratch[SINT_NOALLOC_SCRATCH_BYTES / sizeof(double)];

  constexpr int NOALLOC_MAX_DEVICES = 64;

  // Device address of noalloc_scratch per device ordinal.  The host-side
  // symbol is only a stand-in; its device address is looked up once per
  // device, with that device current.
  static double    *noalloc_addr[NOALLOC_MAX_DEVICES] = {};
  static std::mutex noalloc_mutex;

  static int noalloc_scratch_address(double **out)
  {
    int         dev = 0;
    cudaError_t e   = cudaGetDevice(&dev);
    if (e != cudaSuccess)
      return cuda_fail(e, "sint_jvp_f64_noalloc: cudaGetDevice");
    if (dev < 0 || dev >= NOALLOC_MAX_DEVICES)
      {
        set_error("sint_jvp_f64_noalloc: device ordinal " + std::to_string(dev) + " beyond the supported " +
                  std::to_string(NOALLOC_MAX_DEVICES));
        return SINT_ERR_ARG;
      }
    std::lock_guard<std::mutex> lock(noalloc_mutex);
    if (!noalloc_addr[dev])
      {
        double *ptr = nullptr;
        e           = cudaGetSymbolAddress((void **)&ptr, noalloc_scratch);
        if (e != cudaSuccess)
          return cuda_fail(e, "sint_jvp_f64_noalloc: cudaGetSymbolAddress");
        noalloc_addr[dev] = ptr;
      }
    *out = noalloc_addr[dev];
    return SINT_OK;
  }
} // namespace sint

using namespace sint;

extern "C" int sint_jvp_f64_noalloc(const sint_mesh *mesh, const sint_params *params, double w0, double w_alg,
                                    const double *lin, const double *src, double *dst, sint_stream_t stream)
{
  if (!mesh || !params || !lin || !src || !dst)
    {
      set_error("sint_jvp_f64_noalloc: null argument");
      return SINT_ERR_ARG;
    }
  if (((reinterpret_cast<uintptr_t>(lin) | reinterpret_cast<uintptr_t>(src) | reinterpret_cast<uintptr_t>(dst)) &
       15) != 0)
    {
      set_error("sint_jvp_f64_noalloc: pointers must be 16-byte aligned");
      return SINT_ERR_ARG;
    }
  // the operator description lives on the stack; nothing is allocated
  Ctx c;
  if (int rc = describe_operator(mesh, params, &c))
    return rc;
  const int       box   = mesh->dim == 3 ? Tile<3>::BOX : Tile<2>::BOX;
  const long long need  = c.grid.n_tiles * (long long)c.C * box * (long long)sizeof(double);
  if (need > (long long)SINT_NOALLOC_SCRATCH_BYTES)
    {
      set_error("sint_jvp_f64_noalloc: this mesh needs " + std::to_string(need) +
                " bytes of scratch, more than the fixed " + std::to_string((long long)SINT_NOALLOC_SCRATCH_BYTES) +
                "; use sint_create + sint_jvp_f64");
      return SINT_ERR_ARG;
    }
  c.phys.w0    = w0;
  c.phys.w_alg = w_alg;
  if (int rc = noalloc_scratch_address(&c.partial))
    return rc;
  // every scratch slot the combine kernel reads is written earlier in the same
  // call, so nothing needs clearing between calls
  const cudaError_t e = dispatch_jvp<double>(&c, lin, src, dst, stream);
  if (e != cudaSuccess)
    return cuda_fail(e, "sint_jvp_f64_noalloc");
  return SINT_OK;
}
