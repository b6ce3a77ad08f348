// Fused stream-collide-bounce-back(-force) step kernels.
//
// One thread per lattice cell, z (the unit-stride axis) across the lanes of
// a warp, so every population plane is read and written in 32-wide
// contiguous runs. Wall cells return after reading their mask word (in pull
// and push, those that share a 32-byte sector with fluid cells first fill
// their own destination slots, see step_kernel).
//
// The reference runs a dense sweep and then a serial bounce-back list pass
// (src/kernel_pull_soa.c:94-204, src/kernel_push_soa.c:94-204,
// src/kernel_aa_soa.c:42-278). Here the list pass disappears: a population
// that bounces off a wall is kept in a slot of its own cell that no
// neighbour uses, and its reader is redirected there by the same mask bit.
// Per fluid cell x and direction d, with bb(d) = "x + c_d is a wall" and
// back(d) = bb(inv d) = "x - c_d is a wall":
//
//            read f_d(x)                         write out_d
//   pull     back(d) ? src[inv d][x]             dst[d][x], + F_inv d if bb(d) else + F_d
//                    : src[d][x - c_d]
//   push     src[d][x]                           bb(d) ? dst[inv d][x] = out_d + F_inv d
//                                                      : dst[d][x + c_d] = out_d + F_d
//   AA even  A[d][x]                             A[inv d][x], + F_inv d if bb(d) else + F_d
//   AA odd   back(d) ? A[d][x]                   bb(d) ? A[inv d][x] = out_d + F_inv d
//                    : A[inv d][x - c_d]               : A[d][x + c_d] = out_d + F_d
//
// (With LBM_STORE_MIRROR, measured slower, push and AA odd store every
// population to [d][x + c_d], a bounced one into the wall cell's unread
// slot, and the bounced value again into [inv d][x].) Every stored value is
// fl(out_d + F), the single
// rounding the reference performs when kernelAddBodyForce
// (src/lbm.c:902-922) adds the force to the populations a fluid cell
// receives, so the FP64 kernels are bit-identical to the reference's.
// Race freedom of the in-place AA odd step: a cell reads
// {(e, x + c_e) : x + c_e fluid} and {(d, x) : back(d)}, and writes the same
// sets; the sets of different cells are disjoint and wall cells do not
// update.
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
  int x0 = 0;            // first storage x plane of the launch (grid.z planes from there)
  uint32_t c0 = 0, cn = 0; // compact layout, local steps: storage indices [c0, c0 + cn)
  uint32_t pf_planes = 0;  // compact AA odd step: L2 prefetch distance in x-planes (0 = none)
};

// Minimum resident blocks per SM requested from the compiler (caps the
// registers per thread: 65536 / (128 * n)).
#ifndef LBM_MINB_F64
#define LBM_MINB_F64 6
#endif
#ifndef LBM_MINB_LP
#define LBM_MINB_LP 4
#endif
// Per kind for FP64, from sweeps on the 256^3 porous channel (B200): the
// AA odd step is fastest at 7 CTAs per SM (72 registers), AA even at 6
// (80); with the partial-sector fill, pull at 6 (80) and push at 5 (96).
// 8 spills.
#ifndef LBM_MINB_F64_ODD
#define LBM_MINB_F64_ODD 7
#endif
#ifndef LBM_MINB_F64_PULL
#define LBM_MINB_F64_PULL 6
#endif
#ifndef LBM_MINB_F64_PUSH
#define LBM_MINB_F64_PUSH 5
#endif
template <class ST, int KIND> struct StepOccupancy {
  static constexpr int value = sizeof(typename ST::S) != 8 ? LBM_MINB_LP
      : KIND == kAAOddStep ? LBM_MINB_F64_ODD
      : KIND == kPullStep ? LBM_MINB_F64_PULL
      : KIND == kPushStep ? LBM_MINB_F64_PUSH : LBM_MINB_F64;
};

// Read-only loads of the two-lattice patterns may take the non-coherent
// path; the in-place AA lattice is read and written by the same kernel.
template <bool NC, typename S> __device__ __forceinline__ S ldg(const S *p)
{
  if constexpr (NC)
    return __ldg(p);
  else
    return *p;
}

template <class ST, int KIND, bool FORCE, bool BRINK>
__global__ void __launch_bounds__(kStepThreads, (StepOccupancy<ST, KIND>::value))
    step_kernel(StepArgs<ST> a)
{
  using S = typename ST::S;
  using V = typename ST::V;
  constexpr bool kNC = (KIND == kPullStep || KIND == kPushStep);
  const Grid &g = a.g;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = a.x0 + (int)blockIdx.z;
  if (z >= g.nz || y >= g.ny)
    return;
  const uint32_t cell = cell_index(g, x, y, z);
  const uint32_t mask = a.mask[cell];
  if constexpr (kNC) {
    // Pull and push write a lattice the kernel has not read. A 32-byte
    // sector of it that holds both fluid and solid cells would be written in
    // part, and the L2 fetches such a sector from DRAM to merge the write
    // (14% of the sectors in a 20%-solid porous channel). The solid cells of
    // those sectors therefore fill their own destination slots, which no
    // step or transfer reads (a wall's slots hold no population in either
    // pattern), so the sector is written whole. Lane l holds z = l mod 4 of
    // its sector: rows start on 32-byte boundaries, blockDim.x % 32 == 0.
    const unsigned fluid = __ballot_sync(__activemask(), !(mask & kSolidBit));
    if (mask & kSolidBit) {
      const int lane = threadIdx.x & 31;
      if ((fluid >> (lane & ~3)) & 0xFu) {
#pragma unroll
        for (int d = 0; d < Q; ++d)
          a.dst[d * g.plane + cell] = ST::encode(typename ST::V(0), a.c.scale);
      }
      return;
    }
  } else if (mask & kSolidBit) {
    return;
  }
  const Offs of = make_offs(g, x, y, z);
  const S *src = a.src;
  S *dst = a.dst;
  const long long P = g.plane;

  V f[Q];
  // warp-uniform: warps none of whose cells has a wall link take branch-free
  // addressing (the decision is the same for every lane)
  const bool links = __any_sync(__activemask(), (mask & 0x7FFFFu) != 0u);
  if (!links) {
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const S *p;
      if (KIND == kPullStep)
        p = src + d * P + (uint32_t)(cell + of.at(inv(d)));
      else if (KIND == kPushStep || KIND == kAAEvenStep)
        p = src + d * P + cell;
      else
        p = src + inv(d) * P + (uint32_t)(cell + of.at(inv(d)));
      f[d] = ST::decode(ldg<kNC>(p), a.c.inv_scale);
    }
  } else {
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const bool back = (mask >> inv(d)) & 1u;
      const S *p;
      if (KIND == kPullStep)
        p = back ? src + inv(d) * P + cell : src + d * P + (uint32_t)(cell + of.at(inv(d)));
      else if (KIND == kPushStep || KIND == kAAEvenStep)
        p = src + d * P + cell;
      else
        p = back ? src + d * P + cell : src + inv(d) * P + (uint32_t)(cell + of.at(inv(d)));
      f[d] = ST::decode(ldg<kNC>(p), a.c.inv_scale);
    }
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
    const bool bb = (mask >> d) & 1u;
    if (KIND == kPullStep || KIND == kAAEvenStep) {
      const V v = FORCE ? o[d] + (bb ? a.c.force[inv(d)] : a.c.force[d]) : o[d];
      S *p = (KIND == kPullStep) ? dst + d * P + cell : dst + inv(d) * P + cell;
      *p = ST::encode(v, a.c.scale);
    } else {
#ifndef LBM_STORE_MIRROR
      // one store per population: a bounced one goes straight to (inv d, x)
      const V v = FORCE ? o[d] + (bb ? a.c.force[inv(d)] : a.c.force[d]) : o[d];
      S *p = bb ? dst + inv(d) * P + cell : dst + d * P + (uint32_t)(cell + of.at(d));
      *p = ST::encode(v, a.c.scale);
#else
      const V v = FORCE ? o[d] + a.c.force[d] : o[d];
      dst[d * P + (uint32_t)(cell + of.at(d))] = ST::encode(v, a.c.scale);
      if (d != dC && links && bb) {
        const V w = FORCE ? o[d] + a.c.force[inv(d)] : o[d];
        dst[inv(d) * P + cell] = ST::encode(w, a.c.scale);
      }
#endif
    }
  }
}

} // namespace lbm
