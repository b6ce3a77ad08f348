// Internal interfaces between the translation units of liblbmb200.so.
// Not installed; the public C ABI is include/lbm_b200.h.
#pragma once

#include <cuda_runtime.h>

#include "lbm_b200.h"

#include "lbm_adjoint.cuh"
#include "lbm_step.cuh"
#include "lbm_step_cp.cuh"
#include "lbm_step_tma.cuh"
#include "lbm_step_x2.cuh"

namespace lbm {

enum Precision { kF64 = 0, kF32 = 1, kF16 = 2 };

// Step launchers: FP64 one cell per thread (lbm_step_f64.cu, compiled with
// --fmad=false for bit-exact reference arithmetic), FP32/FP16 storage two
// cells per thread (lbm_step_lp.cu).
cudaError_t launch_step_f64(int kind, bool force, bool brink, const StepArgs<StoreF64> &a,
    dim3 grid, dim3 block, cudaStream_t st);
// Bulk-copy pipelined FP64 step (lbm_step_tma.cuh): `groups` consumer
// groups of 8 warps (1..3), `blocks` persistent CTAs.
cudaError_t launch_step_tma_f64(int kind, bool force, const TmaArgs<StoreF64> &a, int groups,
    int blocks, cudaStream_t st);
cudaError_t launch_step_x2_f32(int kind, bool force, bool brink, const StepArgs2<StoreF32> &a,
    cudaStream_t st);
cudaError_t launch_step_x2_f16(int kind, bool force, bool brink, const StepArgs2<StoreF16> &a,
    cudaStream_t st);

// Compact (fluid-only) layout steps: FP64 one cell per thread
// (lbm_step_cp.cuh, in lbm_step_f64.cu without contraction), FP32/FP16
// storage with the pair arithmetic (lbm_step_cp2.cuh, in lbm_step_lp.cu).
cudaError_t launch_step_cp_f64(int kind, bool force, const StepArgs<StoreF64> &a, dim3 grid,
    dim3 block, cudaStream_t st);
cudaError_t launch_step_cp2_f32(int kind, bool force, const StepArgs2<StoreF32> &a,
    cudaStream_t st);
cudaError_t launch_step_cp2_f16(int kind, bool force, const StepArgs2<StoreF16> &a,
    cudaStream_t st);

// Zou-He pressure boundary on the state after a step (lbm_step_f64.cu):
// marks is [2][ny][nz] (caller's box; 0 = inlet plane x = 0, 1 = outlet
// plane x = nx - 1), nonzero where the boundary applies.
cudaError_t launch_pressure_bc(int precision, const Grid &g, const UserBox &u, int orient,
    void *state, const uint32_t *mask, const uint8_t *marks, double rho_in, double rho_out,
    float scale, cudaStream_t st);

// Adjoint launchers (lbm_adjoint.cu): one reverse step; seed of lambda at
// the final state for the outlet objective on device plane x = xo.
cudaError_t launch_adjoint_step_f64(const AdjArgs<double> &a, cudaStream_t st);
cudaError_t launch_adjoint_step_f32(const AdjArgs<float> &a, cudaStream_t st);
cudaError_t launch_adjoint_seed(int precision, const Grid &g, int xo, double inv_count,
    void *lam, const uint32_t *mask, cudaStream_t st);

// Records the message returned by lbm_last_error() and returns `code`.
int record_error(int code, const char *fmt, ...);

// The solver's own x planes (a slab's, without ghosts) and its CUDA device,
// for host drivers in other translation units; -1 for NULL.
int solver_planes(const lbm_solver *s);
int solver_device(const lbm_solver *s);

// Block/grid shape of the per-cell kernels: z across lanes, then y, one
// x-plane per grid.z.
inline void cell_launch_shape(const Grid &g, dim3 &grid, dim3 &block)
{
  int tz = 32;
  while (tz < g.nz && tz < kStepThreads)
    tz *= 2;
  int ty = kStepThreads / tz;
  block = dim3(tz, ty, 1);
  grid = dim3((g.nz + tz - 1) / tz, (g.ny + ty - 1) / ty, g.nx);
}

// SM count of the current device, looked up once per device (concurrent
// first calls store the same value); 0 if it cannot be read.
inline int sm_count()
{
  static int cache[64];
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64)
    return 0;
  if (cache[dev] == 0) {
    int n = 0;
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
      return 0;
    cache[dev] = n;
  }
  return cache[dev];
}

// Prefetch distance in x-planes of the compact AA odd step: `tenths` / 10
// waves of blocks (a wave: SMs x resident blocks per SM), rounded up to
// whole planes of `blocks_per_plane`; 0 (no prefetch) when tenths is 0 or
// when the rounding lands more than 1.5 waves ahead. Measured on the porous
// channel: FP64 AA odd gained 3% at 1.3 waves (256^3) and lost 5% at 1.7
// (512^3) and 10% at 2.2 (256^3); FP32 gained 8% at 1.1 waves and 2% at 1.7.
inline uint32_t prefetch_planes(int tenths, int blocks_per_sm, unsigned blocks_per_plane)
{
  if (tenths <= 0 || blocks_per_plane == 0)
    return 0;
  const long long wave = (long long)sm_count() * blocks_per_sm;
  const long long want = wave * tenths;
  const long long planes = (want + 10LL * blocks_per_plane - 1) / (10LL * blocks_per_plane);
  if (2 * planes * (long long)blocks_per_plane > 3 * wave)
    return 0;
  return (uint32_t)planes;
}

} // namespace lbm
