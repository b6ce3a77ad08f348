// Step kernels for the reduced-precision storage modes (shifted populations
// g_d = f_d - w_d stored as FP32, or as FP16 scaled by S = 2^k), processing
// two z-adjacent cells per thread.
//
// Why two cells: at 76 or 152 bytes per update the one-cell kernel runs out
// of instruction issue before it runs out of bandwidth. With a cell pair
//   * every access whose z offset is 0 (9 of 19 directions in the shifted
//     patterns, all 19 in the local ones) is one aligned half2/float2
//     load or store for both cells;
//   * the collision runs on float2 with Blackwell's packed FP32 operations
//     (__fadd2_rn/__fmul2_rn/__ffma2_rn), one instruction for both cells;
//   * FP16 values are kept in scaled units G = S g: only the two quadratic
//     terms of the equilibrium carry a 1/S factor, folded into constants,
//     so no population is rescaled on load or store.
// Bounce-back, body force and the Brinkman term follow the same rules as
// step_kernel (lbm_step.cuh). A wall cell paired with a fluid cell computes
// a throwaway value that is never stored.
#pragma once

#include "lbm_device.cuh"
#include "lbm_step.cuh"

namespace lbm {

// Collision constants in the storage units of the pair kernels.
struct Consts2 {
  float oE, oO, w0, w1, w2, w1X3, w2X3;
  float w1NHq, w2NHq; // 4.5 w / S
  float c15q;         // 1.5 / S
  float force[Q];     // S ((3 w_d) c_dx) F
  float alpha;
};

// v + the body force a population of direction d carries into each cell of
// a pair: force[d], or force[inv d] for a population that bounces back at
// the pair's cell (bit d of m0 / m1). For c_x = 0 both are the same signed
// zero; otherwise force[inv d] is -force[d] bit for bit (Consts2 rounds one
// product with the sign of c_x), so the select is a sign flip, with no
// branch and the same result as selecting the constant.
__device__ __forceinline__ float2 add_force2(float2 v, int d, uint32_t m0, uint32_t m1,
    const float (&force)[Q])
{
  if (cx(d) == 0)
    return __fadd2_rn(v, make_float2(force[d], force[d]));
  const uint32_t fb = __float_as_uint(force[d]);
  return __fadd2_rn(v, make_float2(__uint_as_float(fb ^ (((m0 >> d) & 1u) << 31)),
                                   __uint_as_float(fb ^ (((m1 >> d) & 1u) << 31))));
}

template <class ST> struct PairOf;
template <> struct PairOf<StoreF32> {
  using S = float;
  using P = float2;
  __device__ static float2 dec(P p) { return p; }
  __device__ static P enc(float2 v) { return v; }
  __device__ static float dec1(S s) { return s; }
  __device__ static S enc1(float v) { return v; }
};
template <> struct PairOf<StoreF16> {
  using S = __half;
  using P = __half2;
  __device__ static float2 dec(P p) { return __half22float2(p); }
  __device__ static P enc(float2 v) { return __float22half2_rn(v); }
  __device__ static float dec1(S s) { return __half2float(s); }
  __device__ static S enc1(float v) { return __float2half_rn(v); }
};

__device__ __forceinline__ float2 f2(float s) { return make_float2(s, s); }
__device__ __forceinline__ float2 add2(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 sub2(float2 a, float2 b)
{
  return __fadd2_rn(a, make_float2(-b.x, -b.y));
}
__device__ __forceinline__ float2 mul2(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 fma2(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

// TRT collision of two cells at once (same formulas as collide() in
// lbm_device.cuh, in storage units).
template <bool BRINK>
__device__ __forceinline__ void collide2(const float2 (&f)[Q], float2 (&o)[Q], const Consts2 &c,
    float2 kappa, float2 *u_out)
{
  const float2 ux = sub2(add2(add2(add2(add2(f[dE], f[dNE]), f[dSE]), f[dTE]), f[dBE]),
      add2(add2(add2(add2(f[dW], f[dNW]), f[dSW]), f[dTW]), f[dBW]));
  const float2 uy = sub2(add2(add2(add2(add2(f[dN], f[dNE]), f[dNW]), f[dTN]), f[dBN]),
      add2(add2(add2(add2(f[dS], f[dSE]), f[dSW]), f[dTS]), f[dBS]));
  const float2 uz = sub2(add2(add2(add2(add2(f[dT], f[dTE]), f[dTW]), f[dTN]), f[dTS]),
      add2(add2(add2(add2(f[dB], f[dBE]), f[dBW]), f[dBN]), f[dBS]));
  float2 dens = f[dC];
#pragma unroll
  for (int d = 0; d < Q - 1; ++d)
    dens = add2(dens, f[d]);
  if (u_out) {
    u_out[0] = ux;
    u_out[1] = uy;
    u_out[2] = uz;
  }
  const float2 usq = fma2(uz, uz, fma2(uy, uy, mul2(ux, ux)));
  const float2 D = fma2(f2(-c.c15q), usq, dens);
  const float2 oE = f2(c.oE), oO = f2(c.oO), h = f2(0.5f);
  // centre: g_C - oE (g_C - w0 D)
  o[dC] = fma2(oE, fma2(f2(c.w0), D, make_float2(-f[dC].x, -f[dC].y)), f[dC]);
  const float2 w1D = mul2(f2(c.w1), D), w2D = mul2(f2(c.w2), D);

  auto pair = [&](int a, int b, float2 ui, float wnhq, float wx3, float2 wD) {
    const float2 sum = add2(f[a], f[b]), dif = sub2(f[a], f[b]);
    const float2 q = fma2(f2(wnhq), mul2(ui, ui), wD);             // 4.5 w ui^2 / S + w D
    const float2 evenPart = mul2(oE, fma2(h, sum, make_float2(-q.x, -q.y)));
    const float2 uw = mul2(ui, f2(wx3));
    const float2 oddPart = mul2(oO, fma2(h, dif, make_float2(-uw.x, -uw.y)));
    float2 ra = sub2(sub2(f[a], evenPart), oddPart);
    float2 rb = add2(sub2(f[b], evenPart), oddPart);
    if (BRINK) {
      const float2 bterm = mul2(kappa, uw);
      ra = sub2(ra, bterm);
      rb = add2(rb, bterm);
    }
    o[a] = ra;
    o[b] = rb;
  };
  pair(dN, dS, uy, c.w1NHq, c.w1X3, w1D);
  pair(dE, dW, ux, c.w1NHq, c.w1X3, w1D);
  pair(dT, dB, uz, c.w1NHq, c.w1X3, w1D);
  pair(dNW, dSE, sub2(uy, ux), c.w2NHq, c.w2X3, w2D);
  pair(dNE, dSW, add2(ux, uy), c.w2NHq, c.w2X3, w2D);
  pair(dTW, dBE, sub2(uz, ux), c.w2NHq, c.w2X3, w2D);
  pair(dTE, dBW, add2(ux, uz), c.w2NHq, c.w2X3, w2D);
  pair(dTS, dBN, sub2(uz, uy), c.w2NHq, c.w2X3, w2D);
  pair(dTN, dBS, add2(uy, uz), c.w2NHq, c.w2X3, w2D);
}

// collide2 for one cell: the same IEEE operations in the same order on
// scalars, so a cell collided alone gets exactly the value it gets as one
// half of a pair.
__device__ __forceinline__ void collide1(const float (&f)[Q], float (&o)[Q], const Consts2 &c)
{
  auto add = [](float a, float b) { return __fadd_rn(a, b); };
  auto sub = [](float a, float b) { return __fadd_rn(a, -b); };
  auto mul = [](float a, float b) { return __fmul_rn(a, b); };
  auto fma = [](float a, float b, float d) { return __fmaf_rn(a, b, d); };
  const float ux = sub(add(add(add(add(f[dE], f[dNE]), f[dSE]), f[dTE]), f[dBE]),
      add(add(add(add(f[dW], f[dNW]), f[dSW]), f[dTW]), f[dBW]));
  const float uy = sub(add(add(add(add(f[dN], f[dNE]), f[dNW]), f[dTN]), f[dBN]),
      add(add(add(add(f[dS], f[dSE]), f[dSW]), f[dTS]), f[dBS]));
  const float uz = sub(add(add(add(add(f[dT], f[dTE]), f[dTW]), f[dTN]), f[dTS]),
      add(add(add(add(f[dB], f[dBE]), f[dBW]), f[dBN]), f[dBS]));
  float dens = f[dC];
#pragma unroll
  for (int d = 0; d < Q - 1; ++d)
    dens = add(dens, f[d]);
  const float usq = fma(uz, uz, fma(uy, uy, mul(ux, ux)));
  const float D = fma(-c.c15q, usq, dens);
  const float oE = c.oE, oO = c.oO, h = 0.5f;
  o[dC] = fma(oE, fma(c.w0, D, -f[dC]), f[dC]);
  const float w1D = mul(c.w1, D), w2D = mul(c.w2, D);
  auto pair = [&](int a, int b, float ui, float wnhq, float wx3, float wD) {
    const float sum = add(f[a], f[b]), dif = sub(f[a], f[b]);
    const float q = fma(wnhq, mul(ui, ui), wD);
    const float evenPart = mul(oE, fma(h, sum, -q));
    const float uw = mul(ui, wx3);
    const float oddPart = mul(oO, fma(h, dif, -uw));
    o[a] = sub(sub(f[a], evenPart), oddPart);
    o[b] = add(sub(f[b], evenPart), oddPart);
  };
  pair(dN, dS, uy, c.w1NHq, c.w1X3, w1D);
  pair(dE, dW, ux, c.w1NHq, c.w1X3, w1D);
  pair(dT, dB, uz, c.w1NHq, c.w1X3, w1D);
  pair(dNW, dSE, sub(uy, ux), c.w2NHq, c.w2X3, w2D);
  pair(dNE, dSW, add(ux, uy), c.w2NHq, c.w2X3, w2D);
  pair(dTW, dBE, sub(uz, ux), c.w2NHq, c.w2X3, w2D);
  pair(dTE, dBW, add(ux, uz), c.w2NHq, c.w2X3, w2D);
  pair(dTS, dBN, sub(uz, uy), c.w2NHq, c.w2X3, w2D);
  pair(dTN, dBS, add(uy, uz), c.w2NHq, c.w2X3, w2D);
}

template <class ST> struct StepArgs2 {
  using S = typename ST::S;
  Grid g;
  const S *src;
  S *dst;
  const uint32_t *mask;
  const float *porosity;
  float *u_save;
  Consts2 c;
  int no_shuffle; // host-side switch: use the generic two-cell kernel only
  int no_quad;    // host-side switch: AA in FP16 storage on the two-cell kernels
  int x0 = 0;     // first storage x plane of the launch (grid.z planes from there)
  int planes = 0; // x planes of the launch
  uint32_t c0 = 0, cn = 0; // compact layout, local steps: storage indices [c0, c0 + cn)
  uint32_t pf_planes = 0; // compact AA odd step: L2 prefetch distance in x-planes (0 = none)
};

// Minimum resident CTAs per SM of the pair kernels, per storage type and
// kind, from a sweep of the shuffle-aligned kernels on the 256^3 porous
// channel (B200): pull 8, AA odd 7 (FP16) or 4 (FP32), everything else 6.
// The generic kernel keeps 6 for AA odd (at 7 it spills).
#ifndef LBM_MINB_X2
#define LBM_MINB_X2 6
#endif
template <class ST, int KIND, bool SHUFFLE> struct PairOccupancy {
  static constexpr bool kHalf = sizeof(typename ST::S) == 2;
  static constexpr int value = KIND == kPullStep ? 8
      : (KIND == kAAOddStep && SHUFFLE) ? (kHalf ? 7 : 4) : LBM_MINB_X2;
};

template <class ST, int KIND, bool FORCE, bool BRINK>
__global__ void __launch_bounds__(kStepThreads, (PairOccupancy<ST, KIND, false>::value))
    step_kernel_x2(StepArgs2<ST> a)
{
  using PT = PairOf<ST>;
  using S = typename PT::S;
  using P = typename PT::P;
  const Grid &g = a.g;
  const int z = 2 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = a.x0 + (int)blockIdx.z;
  if (z >= g.nz || y >= g.ny)
    return;
  // the pair starts on an even element (pz is even), so pair
  // accesses to a z-aligned slot are 4-byte (FP16) / 8-byte (FP32) aligned
  const uint32_t cell = cell_index(g, x, y, z);
  // mask words of the pair (8-byte aligned); a cell z + 1 = nz is padding
  // and carries the wall bit
  const uint2 mm = *reinterpret_cast<const uint2 *>(a.mask + cell);
  const uint32_t m0 = mm.x, m1 = mm.y;
  const bool solid0 = m0 & kSolidBit, solid1 = m1 & kSolidBit;
  if (solid0 && solid1)
    return;
  const bool both = !(solid0 || solid1);
  // neighbour offsets: x/y parts shared, z parts per cell
  const Offs o0 = make_offs(g, x, y, z);
  const Offs o1 = make_offs(g, x, y, z + 1);
  const long long PL = g.plane;
  const S *src = a.src;
  S *dst = a.dst;

  // warp-uniform switches: any wall link (redirects and bounce-back
  // stores), any pair with exactly one wall cell (per-cell stores, so a wall
  // cell never writes into a neighbour's slot)
  const unsigned act = __activemask();
  const bool links = __any_sync(act, ((m0 | m1) & 0x7FFFFu) != 0u);
  const bool mixed = __any_sync(act, !both);

  // main loads first (no control flow), then the bounce-back redirects of
  // warps that have wall links, so all main loads are in flight together
  float2 f[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    if (KIND == kAAEvenStep || KIND == kPushStep) {
      f[d] = PT::dec(*reinterpret_cast<const P *>(src + d * PL + cell));
      continue;
    }
    // pull reads (d, x - c_d), AA odd reads (inv d, x - c_d)
    const int pl = (KIND == kPullStep) ? d : inv(d);
    const int e = inv(d); // x - c_d = x + c_e
    if (cz(e) == 0) {
      // both cells share x and y, and the fluid one is never on a
      // non-periodic face, so the neighbouring row exists
      f[d] = PT::dec(*reinterpret_cast<const P *>(src + pl * PL + (uint32_t)(cell + o0.at(e))));
    } else {
      // a wall cell of the pair may sit at a row end: it reads its own slot
      f[d].x = PT::dec1(src[pl * PL + (solid0 ? cell : (uint32_t)(cell + o0.at(e)))]);
      f[d].y = PT::dec1(src[pl * PL + (solid1 ? cell + 1u : (uint32_t)(cell + 1u + o1.at(e)))]);
    }
  }
  if ((KIND == kPullStep || KIND == kAAOddStep) && links) {
    // a population that bounced off the wall x - c_d is in the own slot:
    // pull (inv d, x), AA odd (d, x)
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const int e = inv(d);
      const int own = (KIND == kPullStep) ? inv(d) : d;
      const S *ob = src + own * PL + cell;
      if ((m0 >> e) & 1u)
        f[d].x = PT::dec1(ob[0]);
      if ((m1 >> e) & 1u)
        f[d].y = PT::dec1(ob[1]);
    }
  }

  float2 kappa = f2(0.f);
  if (BRINK) {
    const float2 por = *reinterpret_cast<const float2 *>(a.porosity + cell);
    kappa = make_float2(a.c.alpha * (1.f - por.x), a.c.alpha * (1.f - por.y));
  }
  float2 out[Q];
  float2 u3[3];
  collide2<BRINK>(f, out, a.c, kappa, BRINK ? u3 : nullptr);
  if (BRINK && a.u_save) {
    *reinterpret_cast<float2 *>(a.u_save + cell) = u3[0];
    *reinterpret_cast<float2 *>(a.u_save + PL + cell) = u3[1];
    *reinterpret_cast<float2 *>(a.u_save + 2 * PL + cell) = u3[2];
  }

#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const bool bb0 = (m0 >> d) & 1u, bb1 = (m1 >> d) & 1u; // x + c_d is a wall
    if (KIND == kPullStep || KIND == kAAEvenStep) {
      // local: pull (d, x), AA even (inv d, x); a bounced population carries
      // the force of the direction it is read as. A wall cell's own slot is
      // never read, so both cells are written.
      float2 v = out[d];
      if (FORCE) {
        v = add_force2(v, d, m0, m1, a.c.force);
      }
      const int pl = (KIND == kPullStep) ? d : inv(d);
      *reinterpret_cast<P *>(dst + pl * PL + cell) = PT::enc(v);
      continue;
    }
    // push / AA odd: (d, x + c_d) for every population (a bounced one lands
    // in the wall's slot, never read), then the bounced value into (inv d, x)
    const float2 v = FORCE ? add2(out[d], f2(a.c.force[d])) : out[d];
    if (cz(d) == 0 && (!mixed || both)) {
      *reinterpret_cast<P *>(dst + d * PL + (uint32_t)(cell + o0.at(d))) = PT::enc(v);
    } else {
      if (!solid0)
        dst[d * PL + (uint32_t)(cell + o0.at(d))] = PT::enc1(v.x);
      if (!solid1)
        dst[d * PL + (uint32_t)(cell + 1u + o1.at(d))] = PT::enc1(v.y);
    }
    if (d != dC && links && (bb0 || bb1)) {
      const float2 w = FORCE ? add2(out[d], f2(a.c.force[inv(d)])) : out[d];
      if (bb0 && bb1) {
        *reinterpret_cast<P *>(dst + inv(d) * PL + cell) = PT::enc(w);
      } else if (bb0) {
        dst[inv(d) * PL + cell] = PT::enc1(w.x);
      } else {
        dst[inv(d) * PL + cell + 1u] = PT::enc1(w.y);
      }
    }
  }
}

// AA even step, FP16 storage, four z-consecutive cells per thread: every
// plane is read with one 8-byte access per thread, so a warp moves 256
// contiguous bytes per plane (as the FP64 kernel does) instead of 128, which
// the DRAM serves more efficiently; the two cell pairs are then collided
// and stored one after the other exactly as step_kernel_x2 does, so the
// results are bit-identical to it. Needs pz % 4 == 0 (FP16 rows are padded
// to 16 elements) and no Brinkman term.
#ifndef LBM_MINB_QUAD
#define LBM_MINB_QUAD 5
#endif
template <bool FORCE>
__global__ void __launch_bounds__(kStepThreads, LBM_MINB_QUAD)
    step_kernel_even_quad(StepArgs2<StoreF16> a)
{
  using PT = PairOf<StoreF16>;
  using P = PT::P;
  const Grid &g = a.g;
  const int z = 4 * (blockIdx.x * blockDim.x + threadIdx.x);
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = a.x0 + (int)blockIdx.z;
  if (z >= g.nz || y >= g.ny)
    return;
  const long long PL = g.plane;
  const uint32_t cell = cell_index(g, x, y, z);
  // masks of the four cells; cells z + k >= nz are row padding (wall bit)
  const uint4 mq = *reinterpret_cast<const uint4 *>(a.mask + cell);
  uint2 raw[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d)
    raw[d] = *reinterpret_cast<const uint2 *>(a.src + d * PL + cell);
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t m0 = h ? mq.z : mq.x, m1 = h ? mq.w : mq.y;
    if ((m0 & kSolidBit) && (m1 & kSolidBit))
      continue;
    float2 f[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const P *pp = reinterpret_cast<const P *>(&raw[d]);
      f[d] = PT::dec(pp[h]);
    }
    float2 out[Q];
    collide2<false>(f, out, a.c, f2(0.f), nullptr);
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      float2 v = out[d];
      if (FORCE) {
        v = add_force2(v, d, m0, m1, a.c.force);
      }
      *reinterpret_cast<P *>(a.dst + inv(d) * PL + cell + 2 * h) = PT::enc(v);
    }
  }
}

inline void quad_launch_shape(const Grid &g, dim3 &grid, dim3 &block)
{
  const int nq = (g.nz + 3) / 4;
  int tz = 32;
  while (tz < nq && tz < kStepThreads)
    tz *= 2;
  block = dim3(tz, kStepThreads / tz, 1);
  grid = dim3((nq + tz - 1) / tz, (g.ny + block.y - 1) / block.y, g.nx);
}

// Launch shape of the pair kernels: pairs of z across lanes.
inline void pair_launch_shape(const Grid &g, dim3 &grid, dim3 &block)
{
  const int npairs = (g.nz + 1) / 2;
  int tz = 32;
  while (tz < npairs && tz < kStepThreads)
    tz *= 2;
  const int ty = kStepThreads / tz;
  block = dim3(tz, ty, 1);
  grid = dim3((npairs + tz - 1) / tz, (g.ny + ty - 1) / ty, g.nx);
}

} // namespace lbm
