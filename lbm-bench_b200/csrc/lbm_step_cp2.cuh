// Reduced-precision steps (FP32 arithmetic on shifted populations stored as
// FP32 or FP16) in the compact (fluid-only) layout, with the pair
// arithmetic of lbm_step_x2.cuh: two cells share every float2 operation of
// collide2 (Blackwell's packed FP32 add/multiply/FMA), and populations stay
// in storage units. Each cell's values go through exactly the operations the
// dense layout's pair kernels apply to it, so the two layouts give
// bit-identical states in FP32 and FP16 storage too.
//
//   step_kernel_cp2_local   AA even (local): N consecutive stored cells per
//                           thread (N = 2; 4 is supported for FP16), so every
//                           plane is one aligned 4- or 8-byte access per
//                           thread and a warp moves 128 or 256 contiguous
//                           bytes per plane, with no index lookup at all.
//   pull, AA odd            step_kernel_cp2_pair below: two cells per thread
//                           (z and z + 32 of one row) sharing the row's
//                           index words and every float2 operation. At
//                           256^3: FP16 AA odd 0.366 against 0.381 ms for one
//                           cell per thread, FP16 pull 0.329 against 0.359,
//                           FP32 AA odd 0.429 against 0.455 (64 registers;
//                           at 6, 7, 9 or 10 CTAs/SM it is slower).
//   push                    step_kernel_cp (lbm_step_cp.cuh), one cell per
//                           thread, with CpMathUnits below: the pair
//                           arithmetic on one cell (collide1). The two-cell
//                           kernel spills there (FP16 push 0.539 against
//                           0.361 ms). An earlier two-cell form that paired
//                           consecutive stored cells took 0.61 ms for FP16 AA
//                           odd: its cells came from different rows.
#pragma once

#include <type_traits>

#include "lbm_step_cp.cuh"
#include "lbm_step_x2.cuh"

namespace lbm {

// Register caps (minimum CTAs per SM) of the compact pair kernels.
#ifndef LBM_MINB_CP2_EVEN
#define LBM_MINB_CP2_EVEN 6
#endif
// FP16 local step: two cells per thread at 8 CTAs/SM took 0.193 ms at 256^3
// against 0.210 ms for four cells per thread at 5 CTAs/SM (96 registers
// with spills) and 0.211 ms for two cells at 6 CTAs/SM.
#ifndef LBM_MINB_CP2_EVEN16
#define LBM_MINB_CP2_EVEN16 8
#endif

// Cells per thread of the local kernel in FP16 storage (2 or 4; FP32 takes
// 2, one 8-byte access per plane).
#ifndef LBM_CP2_LOCAL16
#define LBM_CP2_LOCAL16 2
#endif
template <class ST> struct LocalCells {
  static constexpr int value = sizeof(typename ST::S) == 2 ? LBM_CP2_LOCAL16 : 2;
};

// Collides the cell pair (f0, f1) of the local (AA even) step and stores it
// into slot inv d of cells c and c + 1 (st0 / st1: whether each is stored).
template <class ST, bool FORCE>
__device__ __forceinline__ void cp2_local_pair(const StepArgs2<ST> &a, const float2 (&f)[Q],
    uint32_t m0, uint32_t m1, uint32_t c, bool st0, bool st1, bool vec)
{
  using PT = PairOf<ST>;
  using P = typename PT::P;
  const long long PL = a.g.plane;
  float2 out[Q];
  collide2<false>(f, out, a.c, f2(0.f), nullptr);
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    float2 v = out[d];
    if (FORCE)
      v = add_force2(v, d, m0, m1, a.c.force);
    typename PT::S *p = a.dst + inv(d) * PL + c;
    if (vec) {
      *reinterpret_cast<P *>(p) = PT::enc(v);
    } else {
      if (st0)
        p[0] = PT::enc1(v.x);
      if (st1)
        p[1] = PT::enc1(v.y);
    }
  }
}

// One group of N consecutive stored cells from `first` (N-aligned) of the
// local step, of which those in [lo, hi) are updated. `whole`: all N are,
// and every access is one aligned 8-byte load or store per plane (plane
// strides are multiples of 128 elements; the mask array is padded with wall
// words to the plane stride, so a group's mask load stays inside it).
template <class ST, bool FORCE, bool WHOLE>
__device__ __forceinline__ void cp2_local_group(const StepArgs2<ST> &a, uint32_t first,
    uint32_t lo, uint32_t hi)
{
  using PT = PairOf<ST>;
  using S = typename PT::S;
  using P = typename PT::P;
  constexpr int N = LocalCells<ST>::value;
  const long long PL = a.g.plane;
  uint32_t m[N];
  if constexpr (N == 4) {
    const uint4 mq = *reinterpret_cast<const uint4 *>(a.mask + first);
    m[0] = mq.x;
    m[1] = mq.y;
    m[2] = mq.z;
    m[3] = mq.w;
  } else {
    const uint2 mp = *reinterpret_cast<const uint2 *>(a.mask + first);
    m[0] = mp.x;
    m[1] = mp.y;
  }
  using Word = typename std::conditional<N * sizeof(S) == 8, uint2, uint32_t>::type;
  Word raw[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const S *p = a.src + d * PL + first;
    if (WHOLE) {
      raw[d] = *reinterpret_cast<const Word *>(p);
    } else {
      Word r {};
      S *v = reinterpret_cast<S *>(&r);
#pragma unroll
      for (int k = 0; k < N; ++k)
        if (first + k >= lo && first + k < hi)
          v[k] = p[k];
      raw[d] = r;
    }
  }
#pragma unroll
  for (int h = 0; h < N / 2; ++h) {
    const uint32_t c = first + 2 * h;
    const bool in0 = WHOLE || (c >= lo && c < hi), in1 = WHOLE || (c + 1 >= lo && c + 1 < hi);
    if (!in0 && !in1)
      continue;
    float2 f[Q];
#pragma unroll
    for (int d = 0; d < Q; ++d)
      f[d] = PT::dec(reinterpret_cast<const P *>(&raw[d])[h]);
    cp2_local_pair<ST, FORCE>(a, f, m[2 * h], m[2 * h + 1], c, in0, in1, WHOLE);
  }
}

// AA even step, compact layout, whole groups: thread t takes the N stored
// cells from ceil(c0 / N) N + N t, up to the last whole group in
// [c0, c0 + cn). Partial groups at either end: step_kernel_cp2_local_ends.
template <class ST> struct CP2LocalOcc {
  static constexpr int value = sizeof(typename ST::S) == 2 ? LBM_MINB_CP2_EVEN16 : LBM_MINB_CP2_EVEN;
};

template <class ST, bool FORCE>
__global__ void __launch_bounds__(kStepThreads, (CP2LocalOcc<ST>::value))
    step_kernel_cp2_local(StepArgs2<ST> a)
{
  constexpr uint32_t N = LocalCells<ST>::value;
  const uint32_t lo = (a.c0 + N - 1) / N * N, hi = (a.c0 + a.cn) / N * N;
  const uint32_t first = lo + N * (blockIdx.x * blockDim.x + threadIdx.x);
  if (first >= hi)
    return;
  cp2_local_group<ST, FORCE, true>(a, first, a.c0, a.c0 + a.cn);
}

// The (at most two) partial groups at the ends of [c0, c0 + cn): thread 0
// the group holding c0, thread 1 the group holding the last cell, when it
// is another, partial group.
template <class ST, bool FORCE>
__global__ void step_kernel_cp2_local_ends(StepArgs2<ST> a)
{
  constexpr uint32_t N = LocalCells<ST>::value;
  const uint32_t end = a.c0 + a.cn;
  const uint32_t g_first = a.c0 / N * N, g_last = (end - 1) / N * N;
  const bool first_partial = a.c0 % N != 0 || g_first == g_last && end % N != 0;
  const bool last_partial = end % N != 0 && g_last != g_first;
  if (threadIdx.x == 0 && first_partial)
    cp2_local_group<ST, FORCE, false>(a, g_first, a.c0, end);
  if (threadIdx.x == 1 && last_partial)
    cp2_local_group<ST, FORCE, false>(a, g_last, a.c0, end);
}

// Arithmetic policy of step_kernel_cp (lbm_step_cp.cuh) for FP32/FP16
// storage: values stay in storage units and collide1 repeats collide2's
// operations on one cell, so the compact layout's shifted steps give the
// dense pair kernels' values bit for bit.
template <class ST> struct CpMathUnits {
  using Args = StepArgs2<ST>;
  using PT = PairOf<ST>;
  using S = typename PT::S;
  using V = float;
  __device__ static V ld(const Args &, S s) { return PT::dec1(s); }
  __device__ static S st(const Args &, V v) { return PT::enc1(v); }
  __device__ static void coll(const Args &a, const V (&f)[Q], V (&o)[Q]) { collide1(f, o, a.c); }
  __device__ static V plus(V x, V y) { return __fadd_rn(x, y); }
};

// Two cells per thread for the non-local kinds (pull, push, AA odd): z and
// z + 32 of one row, so a warp covers 64 consecutive z and each half of it
// gathers and scatters exactly as a warp of step_kernel_cp does (32 lanes,
// coalesced per plane). The two cells share the row's index words, the
// prologue, the kernel parameters and every float2 operation of collide2 and
// add_force2 - the dense pair kernels' arithmetic, bit for bit. A solid (or
// past-the-row) partner is carried with zeros and never loaded or stored.
// Block (32, 4): four rows of one word pair; grid (ceil(W / 2), ceil(ny / 4),
// planes).
#ifndef LBM_MINB_CP2_PAIR
#define LBM_MINB_CP2_PAIR 8
#endif
// Kinds (bit 1 << Kind) that take the two-cell kernel; the others take
// step_kernel_cp with CpMathUnits. LBM_CP2_PAIR_REGS: its gather takes the
// row tables from registers (1) or from their shared copies (0).
#ifndef LBM_CP2_PAIR_KINDS
#define LBM_CP2_PAIR_KINDS ((1 << kPullStep) | (1 << kAAOddStep))
#endif
#ifndef LBM_CP2_PAIR_REGS
#define LBM_CP2_PAIR_REGS LBM_CP_GATHER_REGS
#endif

template <class ST, int KIND, bool FORCE, bool ZPER, typename OFF>
__global__ void __launch_bounds__(kStepThreads, LBM_MINB_CP2_PAIR)
    step_kernel_cp2_pair(StepArgs2<ST> a)
{
  using PT = PairOf<ST>;
  using S = typename PT::S;
  constexpr bool kNC = (KIND == kPullStep || KIND == kPushStep);
  constexpr bool kScatter = (KIND == kPushStep || KIND == kAAOddStep);
  constexpr bool kInner = LBM_CP_INNER_ROWS &&
      (KIND == kAAOddStep || (KIND == kPullStep && sizeof(S) == 2));
  constexpr bool kRegs = LBM_CP2_PAIR_REGS != 0;
  const Grid &g = a.g;
  const int lane = threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = a.x0 + (int)blockIdx.z;
  if (cp_prefetches<KIND, sizeof(S)>() && a.pf_planes)
    cp_plane_prefetch(g, a.src, a.mask, x, a.pf_planes);
  if (y >= g.ny)
    return;
  const uint32_t wi0 = 2u * blockIdx.x; // words wi0 and wi0 + 1 of the row
  const bool has1 = wi0 + 1u < (uint32_t)g.W;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t k0 = ((uint32_t)x * (uint32_t)g.ny + (uint32_t)y) * (uint32_t)g.W + wi0;
  const uint2 wb0 = __ldg(g.wb + k0);
  const uint2 wb1 = has1 ? __ldg(g.wb + k0 + 1u) : make_uint2(0u, 0u);
  const bool fl0 = (wb0.x >> lane) & 1u, fl1 = (wb1.x >> lane) & 1u;
  if (!LBM_CP_EARLY_ROWS && !fl0 && !fl1)
    return;
  const uint32_t cell0 = wb0.y + (uint32_t)__popc(wb0.x & lt);
  const uint32_t cell1 = wb1.y + (uint32_t)__popc(wb1.x & lt);
  // a cell that is not there has no links: nothing redirects, nothing moves
  const uint32_t m0 = fl0 ? __ldg(a.mask + cell0) : 0u;
  const uint32_t m1 = fl1 ? __ldg(a.mask + cell1) : 0u;
  const S *src = a.src;
  S *dst = a.dst;
  const OFF P = (OFF)g.plane;
  auto el = [&](int plane, uint32_t i) { return (OFF)plane * P + (OFF)i; };
  // base + (plane offset + index); (base + index) + plane offset measured
  // 47% slower (FP16 AA odd 0.537 against 0.364 ms at 256^3)
  auto gaddr = [&](int plane, uint32_t i) { return src + el(plane, i); };
  auto saddr = [&](int plane, uint32_t i) { return dst + el(plane, i); };
  auto ld = [&](bool fl, const S *p) { return fl ? PT::dec1(ldg<kNC>(p)) : 0.0f; };

  RowTab<ZPER> t0, t1;
  if (kScatter && LBM_CP_SMEM_TAB) {
    __shared__ uint32_t tab[2 * kTabRows * kStepThreads];
    const int tid = threadIdx.y * blockDim.x + threadIdx.x;
    t0.sB = tab + tid;
    t1.sB = tab + kTabRows * kStepThreads + tid;
  }
  const int z0 = 32 * (int)wi0 + lane;
  t0.template build<kInner>(g, x, y, z0, cell0, wi0, lt, lane, k0);
  if (has1)
    t1.template build<kInner>(g, x, y, z0 + 32, cell1, wi0 + 1u, lt, lane, k0 + 1u);
  if (LBM_CP_EARLY_ROWS && !fl0 && !fl1) // rows and masks were loaded together
    return;

  float2 f[Q];
  if (KIND == kPushStep) {
#pragma unroll
    for (int d = 0; d < Q; ++d)
      f[d] = make_float2(ld(fl0, gaddr(d, cell0)), ld(fl1, gaddr(d, cell1)));
  } else if (!__any_sync(__activemask(), ((m0 | m1) & 0x7FFFFu) != 0u)) {
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const int pl = (KIND == kPullStep) ? d : inv(d);
      f[d] = make_float2(ld(fl0, gaddr(pl, t0.at(g, inv(d), kRegs))),
                         ld(fl1, gaddr(pl, t1.at(g, inv(d), kRegs))));
    }
  } else {
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const bool b0 = (m0 >> inv(d)) & 1u, b1 = (m1 >> inv(d)) & 1u;
      const S *p0, *p1;
      if (KIND == kPullStep) {
        p0 = b0 ? gaddr(inv(d), cell0) : gaddr(d, t0.at(g, inv(d), kRegs));
        p1 = b1 ? gaddr(inv(d), cell1) : gaddr(d, t1.at(g, inv(d), kRegs));
      } else {
        p0 = b0 ? gaddr(d, cell0) : gaddr(inv(d), t0.at(g, inv(d), kRegs));
        p1 = b1 ? gaddr(d, cell1) : gaddr(inv(d), t1.at(g, inv(d), kRegs));
      }
      f[d] = make_float2(ld(fl0, p0), ld(fl1, p1));
    }
  }

  float2 o[Q];
  collide2<false>(f, o, a.c, make_float2(0.0f, 0.0f), nullptr);

#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const float2 v = FORCE ? add_force2(o[d], d, m0, m1, a.c.force) : o[d];
    S *q0, *q1;
    if (KIND == kPullStep) {
      q0 = saddr(d, cell0);
      q1 = saddr(d, cell1);
    } else {
      q0 = ((m0 >> d) & 1u) ? saddr(inv(d), cell0) : saddr(d, t0.at(g, d));
      q1 = ((m1 >> d) & 1u) ? saddr(inv(d), cell1) : saddr(d, t1.at(g, d));
    }
    if (fl0)
      *q0 = PT::enc1(v.x);
    if (fl1)
      *q1 = PT::enc1(v.y);
  }
}

} // namespace lbm
