// Periodic constraints (DoFTools::make_periodicity_constraints, set up in
// sintering/driver.h:629-643): in a periodic direction d the nodes at
// coordinate n[d] are slaves of the nodes at 0 (chains resolved: a node with
// several such coordinates has the node with all of them at 0 as master).
// The constrained operators of deal.II (OperatorBase::vmult,
// operator_base.h:294-353, and the cell loops' read_dof_values /
// distribute_local_to_global) then
//   * read the master's value wherever a cell touches a slave (the cell
//     kernels' box loads do this, BoxNode::lidx),
//   * add the slave rows' contributions to the master rows, and
//   * give the slave rows the identity in J v (dst = src) and zero in the
//     residual (periodic_condense_kernel, after the combine step).
#include "sint_internal.h"
#include "sint_launch.h"

namespace sint
{
  __device__ __forceinline__ void node_coords(const Grid &g, long long n, int (&co)[3])
  {
    co[0] = int(n % g.nn[0]);
    co[1] = int((n / g.nn[0]) % g.nn[1]);
    co[2] = int(n / ((long long)g.nn[0] * g.nn[1]));
  }

  // Slave value of output component comp (mode 2: the preconditioner's
  // outputs, CH 2x2 blocks (J_cc, J_cmu, J_muc, J_mumu) then the AC diagonal).
  template <typename R>
  __device__ __forceinline__ R slave_value(int mode, int comp, const R *src, long long idx)
  {
    if (mode == 0)
      return src[idx];
    if (mode == 1)
      return R(0);
    return (comp == 1 || comp == 2) ? R(0) : R(1);
  }

  // One thread per master node (a node at coordinate 0 in some periodic
  // direction and at n[d] in none): its slaves' rows are added to its row in
  // a fixed order (subsets of those directions by increasing bit pattern),
  // then the slave rows get their constraint value.  Every slave belongs to
  // exactly one master, so no two threads touch the same entry.
  template <typename R>
  __global__ void periodic_condense_kernel(Grid g, int ncomp, R *__restrict__ dst, const R *__restrict__ src, int mode)
  {
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.N)
      return;
    int co[3];
    node_coords(g, n, co);
    unsigned p0 = 0;
    for (int d = 0; d < 3; ++d)
      if ((g.periodic >> d) & 1)
        {
          if (co[d] == g.n[d])
            return; // a slave
          if (co[d] == 0)
            p0 |= 1u << d;
        }
    if (!p0)
      return;
    long long slave[7];
    int       ns = 0;
    for (unsigned S = 1; S < 8; ++S)
      if ((S & ~p0) == 0u)
        slave[ns++] = node_index(g, (S & 1) ? g.n[0] : co[0], (S & 2) ? g.n[1] : co[1], (S & 4) ? g.n[2] : co[2]);
    for (int comp = 0; comp < ncomp; ++comp)
      {
        const long long off = comp * g.ld;
        R               acc = dst[off + n];
        for (int t = 0; t < ns; ++t)
          acc += dst[off + slave[t]];
        dst[off + n] = acc;
        for (int t = 0; t < ns; ++t)
          dst[off + slave[t]] = slave_value(mode, comp, src, off + slave[t]);
      }
  }

  // AffineConstraints::distribute: every slave takes its master's value.
  __global__ void periodic_distribute_kernel(Grid g, int ncomp, double *__restrict__ u)
  {
    const long long n = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (n >= g.N)
      return;
    int co[3];
    node_coords(g, n, co);
    bool slave = false;
    for (int d = 0; d < 3; ++d)
      if (((g.periodic >> d) & 1) && co[d] == g.n[d])
        {
          co[d] = 0;
          slave = true;
        }
    if (!slave)
      return;
    const long long m = node_index(g, co[0], co[1], co[2]);
    for (int comp = 0; comp < ncomp; ++comp)
      u[comp * g.ld + n] = u[comp * g.ld + m];
  }

  template <typename R>
  cudaError_t launch_periodic_condense(const Grid &g, int ncomp, R *dst, const R *src, int mode, cudaStream_t s)
  {
    if (!g.periodic)
      return cudaSuccess;
    periodic_condense_kernel<R><<<dim3((unsigned)((g.N + 255) / 256)), 256, 0, s>>>(g, ncomp, dst, src, mode);
    count_launches(1);
    return cudaGetLastError();
  }
  template cudaError_t launch_periodic_condense<double>(const Grid &, int, double *, const double *, int,
                                                        cudaStream_t);
  template cudaError_t launch_periodic_condense<float>(const Grid &, int, float *, const float *, int, cudaStream_t);

  cudaError_t launch_periodic_distribute(const Grid &g, int ncomp, double *u, cudaStream_t s)
  {
    if (!g.periodic)
      return cudaSuccess;
    periodic_distribute_kernel<<<dim3((unsigned)((g.N + 255) / 256)), 256, 0, s>>>(g, ncomp, u);
    count_launches(1);
    return cudaGetLastError();
  }
} // namespace sint

using namespace sint;

int sint_set_periodicity(sint_ctx *c, unsigned directions)
{
  if (!c)
    {
      set_error("null context");
      return SINT_ERR_ARG;
    }
  if (directions >> c->grid.dim)
    {
      set_error("sint_set_periodicity: direction bits beyond the mesh dimension");
      return SINT_ERR_ARG;
    }
  for (int d = 0; d < c->grid.dim; ++d)
    if (((directions >> d) & 1) && c->grid.n[d] < 2)
      {
        set_error("sint_set_periodicity: a periodic direction needs at least 2 cells");
        return SINT_ERR_ARG;
      }
  if (c->grid.periodic != int(directions))
    c->has_pc = false; // the preconditioner's diagonals change with the constraints
  c->grid.periodic = int(directions);
  return SINT_OK;
}

int sint_distribute_constraints(sint_ctx *c, double *u, sint_stream_t stream)
{
  if (!c || !u)
    {
      set_error("sint_distribute_constraints: null argument");
      return SINT_ERR_ARG;
    }
  const cudaError_t e = launch_periodic_distribute(c->grid, c->C, u, stream);
  return e == cudaSuccess ? SINT_OK : cuda_fail(e, "sint_distribute_constraints");
}
