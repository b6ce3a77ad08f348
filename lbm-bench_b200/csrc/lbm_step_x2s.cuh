// Shuffle-aligned two-cell step kernels for the shifted patterns (pull
// gather, push scatter, AA odd gather + scatter) in the reduced-precision
// storage modes.
//
// A warp owns 64 z-consecutive cells of one (x, y) row, lane l the pair
// (z0 + 2l, z0 + 2l + 1). Every global access is an aligned pair
// (half2 / float2) at the lane's own z position in the neighbour row:
//   * a gather whose source is shifted by s = -1 / +1 in z takes the
//     missing half from the neighbouring lane with one warp shuffle; only
//     lane 0 (s = -1) or lane 31 (s = +1) loads a single element from the
//     next 64-cell segment of the row (wrapping around a periodic z);
//   * a scatter shifted by s stores each fluid cell's own element (two
//     16-bit stores per lane; realigning them into pairs with shuffles,
//     which needs per-lane ownership of the target pairs, measured slower).
// The bounce-back redirects are predicated single-element accesses. Requires
// nz % 64 == 0 and blockDim.x == 32; other extents use step_kernel_x2.
// Bounce-back, force and the Brinkman term follow step_kernel
// (lbm_step.cuh): a population that bounced off the wall x - c_d is read
// from the cell's own slot, and in push / AA odd every population is
// written to (d, x + c_d) - a bounced one into the wall's slot, which
// nothing reads - and the bounced value additionally into (inv d, x).
#pragma once

#include "lbm_step_x2.cuh"

namespace lbm {

constexpr unsigned kFull = 0xFFFFFFFFu;

template <class ST, int KIND, bool FORCE, bool BRINK>
__global__ void __launch_bounds__(kStepThreads, (PairOccupancy<ST, KIND, true>::value))
    step_kernel_x2s(StepArgs2<ST> a)
{
  using PT = PairOf<ST>;
  using S = typename PT::S;
  using P = typename PT::P;
  const Grid &g = a.g;
  const int lane = threadIdx.x; // blockDim.x == 32
  const int z = 64 * blockIdx.x + 2 * lane;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = a.x0 + (int)blockIdx.z;
  if (y >= g.ny) // uniform across the warp
    return;
  const uint32_t cell = cell_index(g, x, y, z);
  const uint2 mm = *reinterpret_cast<const uint2 *>(a.mask + cell);
  const uint32_t m0 = mm.x, m1 = mm.y;
  const bool fluid0 = !(m0 & kSolidBit), fluid1 = !(m1 & kSolidBit);
  if (!__any_sync(kFull, fluid0 || fluid1)) // uniform
    return;
  // directions in which any cell of the warp has a wall link (uniform)
  const uint32_t wlinks = __reduce_or_sync(kFull, (m0 | m1) & 0x7FFFFu);
  const bool links = wlinks != 0u;
  if (KIND == kPushStep) {
    // Push writes a lattice this kernel has not read, and only the fluid
    // cells' targets: a 32-byte sector holding solid cells too would be
    // written in part and fetched from DRAM by the L2 to merge the write.
    // The solid cells of sectors that hold fluid fill their own slots
    // (d, x), which nothing reads (a bounced population may land there too,
    // an equally unread value), so the sector is written whole.
    constexpr int kSectorLanes = 16 / (int)sizeof(S); // two cells per lane
    const unsigned lanes = __ballot_sync(kFull, fluid0 || fluid1);
    const unsigned group = (lanes >> (lane & ~(kSectorLanes - 1))) & ((1u << kSectorLanes) - 1u);
    if (group && !(fluid0 && fluid1)) {
#pragma unroll
      for (int d = 0; d < Q; ++d) {
        S *own = a.dst + d * g.plane + cell;
        if (!fluid0 && !fluid1)
          *reinterpret_cast<P *>(own) = PT::enc(f2(0.f));
        else if (!fluid0)
          own[0] = PT::enc1(0.f);
        else
          own[1] = PT::enc1(0.f);
      }
    }
  }

  // x/y parts of the neighbour offsets (uniform across the warp); the z
  // shift is handled by shuffles and the two edge lanes
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
  // lane's own position: one before the segment (lane 0) and two after
  // (lane 31), wrapped around a periodic z
  // (signed: they are added to pointers)
  const bool pz = (g.per >> 2) & 1;
  const int lo = (z == 0) ? (pz ? g.nz - 1 : 0) : -1;
  const int hi = (z + 2 == g.nz) ? (pz ? -(g.nz - 2) : 0) : 2;
  const long long PL = g.plane;
  const S *src = a.src;
  S *dst = a.dst;

  // gather in three phases so that all main loads are in flight together:
  // (1) the aligned pair of every direction and the edge lanes' single
  //     elements, no control flow; (2) shuffles that realign z-shifted
  //     sources; (3) warps with wall links replace bounced populations with
  //     the cell's own slot.
  float2 f[Q];
  if (KIND == kPushStep) {
#pragma unroll
    for (int d = 0; d < Q; ++d)
      f[d] = PT::dec(*reinterpret_cast<const P *>(src + d * PL + cell));
  } else {
    P raw[Q];
    S edge[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      // pull reads (d, x - c_d), AA odd (inv d, x - c_d)
      const int pl = (KIND == kPullStep) ? d : inv(d);
      const int e = inv(d); // x - c_d = x + c_e
      const S *base = src + pl * PL + (uint32_t)(cell + row(e));
      raw[d] = *reinterpret_cast<const P *>(base);
      if (cz(e) < 0)
        edge[d] = (lane == 0 && fluid0) ? base[lo] : PT::enc1(0.f);
      else if (cz(e) > 0)
        edge[d] = (lane == 31 && fluid1) ? base[hi] : PT::enc1(0.f);
    }
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const int e = inv(d);
      const float2 pv = PT::dec(raw[d]);
      if (cz(e) == 0) {
        f[d] = pv;
      } else if (cz(e) < 0) { // sources z - 1, z
        const float up = __shfl_up_sync(kFull, pv.y, 1);
        f[d] = make_float2(lane == 0 ? PT::dec1(edge[d]) : up, pv.x);
      } else { // sources z + 1, z + 2
        const float dn = __shfl_down_sync(kFull, pv.x, 1);
        f[d] = make_float2(pv.y, lane == 31 ? PT::dec1(edge[d]) : dn);
      }
    }
    if (links) {
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
    if (KIND == kPullStep) {
      // local store (d, x); a bounced population carries F_inv d
      float2 v = out[d];
      if (FORCE) {
        v = add_force2(v, d, m0, m1, a.c.force);
      }
      *reinterpret_cast<P *>(dst + d * PL + cell) = PT::enc(v);
      continue;
    }
    // push / AA odd: every population to (d, x + c_d); unshifted in z the
    // aligned pair (z, z+1) of the target row is written whole when both
    // cells are fluid, otherwise half by half
    const float2 v = FORCE ? add2(out[d], f2(a.c.force[d])) : out[d];
    S *base = dst + d * PL + (uint32_t)(cell + row(d));
    float2 t;
    bool tx, ty;
    if (cz(d) == 0) {
      t = v;
      tx = fluid0;
      ty = fluid1;
    } else {
      // shifted in z: each fluid cell stores its own element, at offset lo
      // (z -> z - 1) or hi (z + 1 -> z + 2), which wrap at the row ends
      if (fluid0)
        base[cz(d) < 0 ? lo : 1] = PT::enc1(v.x);
      if (fluid1)
        base[cz(d) < 0 ? 0 : hi] = PT::enc1(v.y);
      t = v;
      tx = ty = false;
    }
    if (tx && ty)
      *reinterpret_cast<P *>(base) = PT::enc(t);
    if (tx && !ty)
      base[0] = PT::enc1(t.x);
    if (ty && !tx)
      base[1] = PT::enc1(t.y);
    if (d != dC && ((wlinks >> d) & 1u)) {
      // bounce-back: the bounced value into (inv d, x)
      const float2 w = FORCE ? add2(out[d], f2(a.c.force[inv(d)])) : out[d];
      S *ob = dst + inv(d) * PL + cell;
      if (bb0)
        ob[0] = PT::enc1(w.x);
      if (bb1)
        ob[1] = PT::enc1(w.y);
    }
  }
}

// Launch shape of the shuffle-aligned kernels: one warp per 64-cell row
// segment, four rows (y) per block.
inline void shuffle_launch_shape(const Grid &g, dim3 &grid, dim3 &block)
{
  block = dim3(32, kStepThreads / 32, 1);
  grid = dim3(g.nz / 64, (g.ny + block.y - 1) / block.y, g.nx);
}

} // namespace lbm
