// Four-cell shuffle-aligned step kernel for the shifted patterns (pull
// gather, push scatter, AA odd gather + scatter) in FP16 storage. The
// solver runs it for AA odd steps (256^3 porous channel on a B200: 0.47 ms
// against 0.54 ms for the two-cell kernel); for pull and push it was slower
// (0.44 / 0.47 ms against 0.33 / 0.44 ms): each cell pair's local store
// covers every other 4 bytes of the warp's 256-byte span, twice the store
// sectors of the two-cell kernel's contiguous 128 bytes.
//
// A warp owns 128 z-consecutive cells of one (x, y) row, lane l the four
// cells z0 + 4l .. z0 + 4l + 3. Every plane is read with one aligned 8-byte
// access per lane at the lane's own z position in the source row, so a warp
// moves 256 contiguous bytes per plane. A source shifted by s = -1 / +1 in z
// is realigned in the packed 16-bit domain: one warp shuffle brings the
// neighbouring lane's edge word and two byte permutes rebuild the lane's two
// pairs; only lane 0 (s = -1) or lane 31 (s = +1) loads a single element
// from the next 128-cell segment of the row (wrapping around a periodic z).
// Bounce-back redirects replace single 16-bit halves before decoding. The
// two cell pairs (z, z+1) and (z+2, z+3) are then decoded, collided and
// stored one after the other with exactly the operations of
// step_kernel_x2s (lbm_step_x2s.cuh), so the results are bit-identical to
// it. Requires nz % 128 == 0, blockDim.x == 32 and no Brinkman term.
#pragma once

#include "lbm_step_x2s.cuh"

namespace lbm {

// 4 CTAs/SM (128 registers): at 5 the AA odd kernel spills and runs 10% slower
#ifndef LBM_MINB_X4S
#define LBM_MINB_X4S 4
#endif

// half k (0..3) of a packed four-element word pair replaced by the 16-bit
// value v
__device__ __forceinline__ void put_half(uint2 &w, int k, uint32_t v)
{
  uint32_t &word = (k < 2) ? w.x : w.y;
  word = __byte_perm(word, v, (k & 1) ? 0x5410 : 0x3254);
}

template <int KIND, bool FORCE>
__global__ void __launch_bounds__(kStepThreads, LBM_MINB_X4S)
    step_kernel_x4s(StepArgs2<StoreF16> a)
{
  using PT = PairOf<StoreF16>;
  using S = __half;
  using P = __half2;
  using U = unsigned short;
  const Grid &g = a.g;
  const int lane = threadIdx.x; // blockDim.x == 32
  const int z = 128 * blockIdx.x + 4 * lane;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = a.x0 + (int)blockIdx.z;
  if (y >= g.ny) // uniform across the warp
    return;
  const uint32_t cell = cell_index(g, x, y, z);
  const uint4 mq = *reinterpret_cast<const uint4 *>(a.mask + cell);
  const uint32_t m[4] = { mq.x, mq.y, mq.z, mq.w };
  bool fl[4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    fl[k] = !(m[k] & kSolidBit);
  if (!__any_sync(kFull, fl[0] || fl[1] || fl[2] || fl[3])) // uniform
    return;
  // directions in which any cell of the warp has a wall link (uniform)
  const uint32_t wlinks = __reduce_or_sync(kFull, (m[0] | m[1] | m[2] | m[3]) & 0x7FFFFu);
  const bool links = wlinks != 0u;

  const Offs of = make_offs(g, x, y, z);
  auto row = [&](int d) -> uint32_t {
    uint32_t o = 0u;
    if (cx(d) < 0)
      o += of.xm;
    else if (cx(d) > 0)
      o += of.xp;
    if (cy(d) < 0)
      o += of.ym;
    else if (cy(d) > 0)
      o += of.yp;
    return o;
  };
  // element offsets of the edge lanes' single accesses, relative to the
  // lane's own position: one before the segment (lane 0) and four after
  // (lane 31), wrapped around a periodic z
  const bool pz = (g.per >> 2) & 1;
  const int lo = (z == 0) ? (pz ? g.nz - 1 : 0) : -1;
  const int hi = (z + 4 == g.nz) ? (pz ? -(g.nz - 4) : 0) : 4;
  const long long PL = g.plane;
  const S *src = a.src;
  S *dst = a.dst;

  // gather: (1) the aligned four elements of every direction and the edge
  // lanes' single elements, no control flow; (2) realignment of z-shifted
  // sources; (3) bounce-back redirects of warps with wall links
  uint2 raw[Q];
  if (KIND == kPushStep) {
#pragma unroll
    for (int d = 0; d < Q; ++d)
      raw[d] = *reinterpret_cast<const uint2 *>(src + d * PL + cell);
  } else {
    uint32_t edge[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      // pull reads (d, x - c_d), AA odd (inv d, x - c_d)
      const int pl = (KIND == kPullStep) ? d : inv(d);
      const int e = inv(d); // x - c_d = x + c_e
      const S *base = src + pl * PL + (uint32_t)(cell + row(e));
      const U *bu = reinterpret_cast<const U *>(base);
      raw[d] = *reinterpret_cast<const uint2 *>(base);
      edge[d] = 0u;
      if (cz(e) < 0)
        edge[d] = (lane == 0 && fl[0]) ? (uint32_t)bu[lo] : 0u;
      else if (cz(e) > 0)
        edge[d] = (lane == 31 && fl[3]) ? (uint32_t)bu[hi] : 0u;
    }
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const int e = inv(d);
      if (cz(e) < 0) { // sources z - 1 .. z + 2
        uint32_t prev = __shfl_up_sync(kFull, raw[d].y, 1);
        if (lane == 0)
          prev = edge[d] << 16;
        raw[d] = make_uint2(__byte_perm(prev, raw[d].x, 0x5432),
            __byte_perm(raw[d].x, raw[d].y, 0x5432));
      } else if (cz(e) > 0) { // sources z + 1 .. z + 4
        uint32_t next = __shfl_down_sync(kFull, raw[d].x, 1);
        if (lane == 31)
          next = edge[d];
        raw[d] = make_uint2(__byte_perm(raw[d].x, raw[d].y, 0x5432),
            __byte_perm(raw[d].y, next, 0x5432));
      }
    }
    if (links) {
      // a population that bounced off the wall x - c_d is in the own slot:
      // pull (inv d, x), AA odd (d, x)
#pragma unroll
      for (int d = 0; d < Q; ++d) {
        const int e = inv(d);
        const int own = (KIND == kPullStep) ? inv(d) : d;
        const U *ob = reinterpret_cast<const U *>(src + own * PL + cell);
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if ((m[k] >> e) & 1u)
            put_half(raw[d], k, ob[k]);
      }
    }
  }

#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const uint32_t m0 = m[2 * h], m1 = m[2 * h + 1];
    const bool fluid0 = fl[2 * h], fluid1 = fl[2 * h + 1];
    if (!fluid0 && !fluid1)
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
      const bool bb0 = (m0 >> d) & 1u, bb1 = (m1 >> d) & 1u; // x + c_d is a wall
      if (KIND == kPullStep) {
        // local store (d, x); a bounced population carries F_inv d
        float2 v = out[d];
        if (FORCE) {
          v = add_force2(v, d, m0, m1, a.c.force);
        }
        *reinterpret_cast<P *>(dst + d * PL + cell + 2 * h) = PT::enc(v);
        continue;
      }
      // push / AA odd: every population to (d, x + c_d)
      const float2 v = FORCE ? add2(out[d], f2(a.c.force[d])) : out[d];
      S *base = dst + d * PL + (uint32_t)(cell + row(d));
      if (cz(d) == 0) {
        if (fluid0 && fluid1)
          *reinterpret_cast<P *>(base + 2 * h) = PT::enc(v);
        else if (fluid0)
          base[2 * h] = PT::enc1(v.x);
        else
          base[2 * h + 1] = PT::enc1(v.y);
      } else {
        // shifted in z: each fluid cell stores its own element at k + cz(d),
        // which wraps at the row ends (lo for k = 0 going down, hi for
        // k = 3 going up)
        const int t0 = 2 * h + cz(d), t1 = 2 * h + 1 + cz(d);
        if (fluid0)
          base[t0 < 0 ? lo : t0] = PT::enc1(v.x);
        if (fluid1)
          base[t1 > 3 ? hi : t1] = PT::enc1(v.y);
      }
      if (d != dC && ((wlinks >> d) & 1u)) {
        // bounce-back: the bounced value into (inv d, x)
        const float2 w = FORCE ? add2(out[d], f2(a.c.force[inv(d)])) : out[d];
        S *ob = dst + inv(d) * PL + cell + 2 * h;
        if (bb0)
          ob[0] = PT::enc1(w.x);
        if (bb1)
          ob[1] = PT::enc1(w.y);
      }
    }
  }
}

// Launch shape of the four-cell kernel: one warp per 128-cell row segment,
// four rows (y) per block.
inline void quad_shuffle_launch_shape(const Grid &g, dim3 &grid, dim3 &block)
{
  block = dim3(32, kStepThreads / 32, 1);
  grid = dim3(g.nz / 128, (g.ny + block.y - 1) / block.y, g.nx);
}

} // namespace lbm
