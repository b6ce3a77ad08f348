// Fused stream-collide-bounce-back(-force) step kernels.
//
// One thread per lattice cell, z (the unit-stride axis) across the lanes of
// a warp, so every population plane is read and written in 32-wide
// contiguous runs. Obstacle cells return after reading their mask word.
//
// The reference runs a dense sweep and then a serial bounce-back list pass
// (src/kernel_pull_soa.c:94-204, src/kernel_push_soa.c:94-204,
// src/kernel_aa_soa.c:42-278). Here the list pass disappears: a population
// that would enter a wall is written straight back into a slot of its own
// cell that no fluid neighbour uses, and the reader of that slot is
// redirected there by the same mask bit. Per fluid cell and direction d
// (bb(d) = neighbour x + c_d is a wall, F_d the body-force term):
//
//   pull     read  bb(inv d) ? src[inv d][x] : src[d][x - c_d]
//            write dst[d][x] = out_d + (bb(d) ? F_inv d : F_d)
//   push     read  src[d][x]
//            write bb(d) ? dst[inv d][x] = out_d + F_inv d
//                        : dst[d][x + c_d] = out_d + F_d
//   AA even  read  A[d][x];  write A[inv d][x] = out_d + (bb(d) ? F_inv d : F_d)
//   AA odd   read  bb(inv d) ? A[d][x] : A[inv d][x - c_d]
//            write bb(d) ? A[inv d][x] = out_d + F_inv d
//                        : A[d][x + c_d] = out_d + F_d
//
// Every value stored is fl(out_d + F), the same single rounding the
// reference performs when kernelAddBodyForce (src/lbm.c:902-922) adds the
// force to the populations a fluid cell receives, so the FP64 kernels are
// bit-identical to the reference's. In the AA odd step each cell's read
// set equals its write set ({(d, x + c_d) : fluid} plus {(d, x) : bounced})
// and the sets of different cells are disjoint, so the in-place update is
// race-free.
#pragma once

#include "lbm_device.cuh"

namespace lbm {

constexpr int kStepThreads = 128;

template <class ST> struct StepArgs {
  using S = typename ST::S;
  using V = typename ST::V;
  Grid g;
  const S *src;          // pull/push source; AA: the single lattice
  S *dst;                // pull/push destination; AA: the single lattice
  const uint32_t *mask;
  const float *porosity; // Brinkman only
  V *u_save;             // Brinkman only, optional: momentum per cell (3 planes)
  Consts<V> c;
};

template <class ST, int KIND, bool FORCE, bool BRINK>
__global__ void __launch_bounds__(kStepThreads) step_kernel(StepArgs<ST> a)
{
  using S = typename ST::S;
  using V = typename ST::V;
  const Grid &g = a.g;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.nz || y >= g.ny)
    return;
  const long long cell = cell_index(g, x, y, z);
  const uint32_t mask = a.mask[cell];
  if (mask & kSolidBit)
    return;

  Nbhd nb;
  if (KIND != kAAEvenStep)
    nb = make_nbhd(g, x, y, z);

  const S *src = a.src;
  S *dst = a.dst;
  const long long P = g.plane;

  V f[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const bool back = (mask >> inv(d)) & 1u; // x - c_d is a wall
    const S *p;
    if (KIND == kPullStep)
      p = back ? src + inv(d) * P + cell : src + d * P + behind(nb, d);
    else if (KIND == kPushStep || KIND == kAAEvenStep)
      p = src + d * P + cell;
    else
      p = back ? src + d * P + cell : src + inv(d) * P + behind(nb, d);
    f[d] = ST::load(p, d, a.c.inv_scale);
  }

  V kappa = V(0);
  if (BRINK)
    kappa = a.c.alpha * (V(1.0) - V(a.porosity[cell]));
  V o[Q];
  V u3[3];
  collide<V, BRINK>(f, o, a.c, kappa, BRINK ? u3 : nullptr);
  if (BRINK && a.u_save) {
    a.u_save[cell] = u3[0];
    a.u_save[P + cell] = u3[1];
    a.u_save[2 * P + cell] = u3[2];
  }

#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const bool bb = (mask >> d) & 1u; // x + c_d is a wall
    V v = o[d];
    if (FORCE)
      v = v + (bb ? a.c.force[inv(d)] : a.c.force[d]);
    S *p;
    if (KIND == kPullStep)
      p = dst + d * P + cell;
    else if (KIND == kAAEvenStep)
      p = dst + inv(d) * P + cell;
    else
      p = bb ? dst + inv(d) * P + cell : dst + d * P + nb.at(d);
    ST::store(p, v, a.c.scale);
  }
}

} // namespace lbm
