// Adjoint kernels (lbm_adjoint.cuh), instantiated for FP64 and FP32.
#include "lbm_adjoint.cuh"
#include "lbm_internal.h"

namespace lbm {

template <typename V> static cudaError_t step(const AdjArgs<V> &a, cudaStream_t st)
{
  dim3 grid, block;
  cell_launch_shape(a.g, grid, block);
  adjoint_step_kernel<V><<<grid, block, 0, st>>>(a);
  return cudaGetLastError();
}

template <typename V>
static cudaError_t seed(const Grid &g, int xo, double inv_count, void *lam,
    const uint32_t *mask, cudaStream_t st)
{
  dim3 grid, block;
  cell_launch_shape(g, grid, block);
  adjoint_seed_kernel<V><<<grid, block, 0, st>>>(g, xo, inv_count, (V *)lam, mask);
  return cudaGetLastError();
}

cudaError_t launch_adjoint_step_f64(const AdjArgs<double> &a, cudaStream_t st)
{
  return step(a, st);
}
cudaError_t launch_adjoint_step_f32(const AdjArgs<float> &a, cudaStream_t st)
{
  return step(a, st);
}
cudaError_t launch_adjoint_seed(int precision, const Grid &g, int xo, double inv_count,
    void *lam, const uint32_t *mask, cudaStream_t st)
{
  return precision == kF64 ? seed<double>(g, xo, inv_count, lam, mask, st)
                           : seed<float>(g, xo, inv_count, lam, mask, st);
}

} // namespace lbm
