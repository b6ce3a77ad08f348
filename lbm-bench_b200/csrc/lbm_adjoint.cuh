// Discrete adjoint of the Brinkman TRT step (no counterpart in the
// reference; the forward step is the reference's, src/kernel_pull_soa.c:
// 118-198, plus the Brinkman resistance of collide() in lbm_device.cuh).
//
// Forward step in the receiver view: out(x) = C(f(x); u(x), phi(x)) is the
// collision of cell x, and population d of it goes to r(x, d) =
// (d, x + c_d), or to (inv d, x) if x + c_d is a wall; the body force is a
// constant. For an objective J of the final state, with
// lambda_d(x) = dJ / df_d(x) kept in the natural layout (plane d, cell x):
//   mu_d(x)       = lambda^{t+1}[r(x, d)]
//   lambda^t_k(x) = sum_d mu_d(x) d out_d / d f_k (x)
//   dJ/dphi(x)   += sum_d mu_d(x) d out_d / d phi (x)
// The collision Jacobian depends only on the momentum u(x, t) of the
// populations the cell collided at step t, which the forward kernels save
// during the segment recomputation. With oE = omega, oO = omegaOdd,
// kappa = alpha (1 - phi), D = rho - 1.5 |u|^2, pairs (a, b = inv a) with
// weight w and ui = c_a . u:
//   out_a = f_a - oE (f_a+f_b)/2 - oO (f_a-f_b)/2 + oE w (4.5 ui^2 + D)
//           + 3 w (oO - kappa) ui            (out_b: signs of the odd terms flip)
//   out_C = f_C - oE (f_C - w0 D)
// so that
//   lambda_a = (1 - (oE+oO)/2) mu_a + ((oO-oE)/2) mu_b + sD + g . c_a
//   lambda_C = (1 - oE) mu_C + sD
//   sD = oE (w0 mu_C + sum_pairs w (mu_a + mu_b))
//   g  = sum_pairs [oE 9 w ui (mu_a + mu_b) + 3 w (oO - kappa)(mu_a - mu_b)] c_a - 3 u sD
//   dJ/dphi += sum_pairs 3 w alpha ui (mu_a - mu_b).
#pragma once

#include "lbm_device.cuh"

namespace lbm {

template <typename V> struct AdjArgs {
  Grid g;
  const V *lam_next; // lambda^{t+1}, natural layout
  V *lam;            // lambda^t
  const V *u;        // momentum at step t, 3 planes (x, y, z)
  const uint32_t *mask;
  const float *porosity;
  double *grad;      // dJ/dphi accumulator per cell
  V oE, oO, w0, w1, w2, alpha;
};

// 6 CTAs of 128 per SM (80 registers): fastest in a sweep at 128^3 (B200)
#ifndef LBM_MINB_ADJ
#define LBM_MINB_ADJ 6
#endif
template <typename V>
__global__ void __launch_bounds__(128, LBM_MINB_ADJ) adjoint_step_kernel(AdjArgs<V> a)
{
  const Grid &g = a.g;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.nz || y >= g.ny)
    return;
  const uint32_t cell = cell_index(g, x, y, z);
  const uint32_t mask = a.mask[cell];
  // The step writes lambda into a lattice it has not read. The solid cells
  // of 32-byte sectors that also hold fluid cells store their own lambda
  // (0, as the seed sets it; no step reads a wall's slots), so that such
  // sectors are written whole and the L2 does not fetch them from DRAM to
  // merge a partial write. Lane l holds z = l mod (32 / sizeof(V)) of its
  // sector: rows start on 32-byte boundaries and blockDim.x % 32 == 0.
  const unsigned fluid = __ballot_sync(__activemask(), !(mask & kSolidBit));
  if (mask & kSolidBit) {
    constexpr int kSectorLanes = 32 / (int)sizeof(V);
    const int lane = threadIdx.x & 31;
    if ((fluid >> (lane & ~(kSectorLanes - 1))) & ((1u << kSectorLanes) - 1u)) {
#pragma unroll
      for (int k = 0; k < Q; ++k)
        a.lam[k * g.plane + cell] = V(0);
    }
    return;
  }
  const Offs of = make_offs(g, x, y, z);
  const long long P = g.plane;

  V mu[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const bool bb = (mask >> d) & 1u;
    mu[d] = bb ? a.lam_next[inv(d) * P + cell] : a.lam_next[d * P + (uint32_t)(cell + of.at(d))];
  }
  const V ux = a.u[cell], uy = a.u[P + cell], uz = a.u[2 * P + cell];
  const V kappa = a.alpha * (V(1) - V(a.porosity[cell]));
  const V oE = a.oE, oO = a.oO;
  const V cdir = V(1) - V(0.5) * oE - V(0.5) * oO, ccross = V(0.5) * oO - V(0.5) * oE;

  // first the sums every output needs (sD, g, the porosity gradient), then
  // each output from mu directly, stored at once: no array of partial
  // results stays live next to mu
  V sD = oE * a.w0 * mu[dC];
  V gx = 0, gy = 0, gz = 0, gphi = 0;
  auto pair = [&](int pa, int pb, V w) {
    const V ui = V(cx(pa)) * ux + V(cy(pa)) * uy + V(cz(pa)) * uz;
    const V ms = mu[pa] + mu[pb], md = mu[pa] - mu[pb];
    sD += oE * w * ms;
    const V sp = oE * V(9) * w * ui * ms + V(3) * w * (oO - kappa) * md;
    gx += sp * V(cx(pa));
    gy += sp * V(cy(pa));
    gz += sp * V(cz(pa));
    gphi += V(3) * w * a.alpha * ui * md;
  };
  pair(dN, dS, a.w1);
  pair(dE, dW, a.w1);
  pair(dT, dB, a.w1);
  pair(dNW, dSE, a.w2);
  pair(dNE, dSW, a.w2);
  pair(dTW, dBE, a.w2);
  pair(dTE, dBW, a.w2);
  pair(dTS, dBN, a.w2);
  pair(dTN, dBS, a.w2);
  gx -= V(3) * ux * sD;
  gy -= V(3) * uy * sD;
  gz -= V(3) * uz * sD;
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    const V part = (k == dC) ? (V(1) - oE) * mu[dC] : cdir * mu[k] + ccross * mu[inv(k)];
    a.lam[k * P + cell] = part + sD + gx * V(cx(k)) + gy * V(cy(k)) + gz * V(cz(k));
  }
  a.grad[cell] += (double)gphi;
}

// lambda^N = dJ/df^N for J = mean over the fluid cells of device plane
// x = xo of sum_k c_kx f_k: c_kx / count there, 0 elsewhere.
template <typename V>
__global__ void adjoint_seed_kernel(Grid g, int xo, double inv_count, V *lam,
    const uint32_t *__restrict__ mask)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.nz || y >= g.ny)
    return;
  const uint32_t cell = cell_index(g, x, y, z);
  const bool on = x == xo && !(mask[cell] & kSolidBit);
#pragma unroll
  for (int k = 0; k < Q; ++k)
    lam[k * g.plane + cell] = on ? V(cx(k) * inv_count) : V(0);
}

} // namespace lbm
