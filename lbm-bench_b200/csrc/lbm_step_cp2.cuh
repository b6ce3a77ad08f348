// Reduced-precision steps (FP32 arithmetic on shifted populations stored as
// FP32 or FP16) in the compact (fluid-only) layout, with the pair
// arithmetic of lbm_step_x2.cuh: two cells share every float2 operation of
// collide2 (Blackwell's packed FP32 add/multiply/FMA), and populations stay
// in storage units. Each cell's values go through exactly the operations the
// dense layout's pair kernels apply to it, so the two layouts give
// bit-identical states in FP32 and FP16 storage too.
//
//   step_kernel_cp2_local   AA even (local): N consecutive stored cells per
//                           thread (N = 4 for FP16, 2 for FP32), so every
//                           plane is one aligned 8-byte access per thread and
//                           a warp moves 256 contiguous bytes per plane, with
//                           no index lookup at all.
//   pull, push, AA odd      step_kernel_cp (lbm_step_cp.cuh), one cell per
//                           thread, with CpMathUnits below: the pair
//                           arithmetic on one cell (collide1). Two cells per
//                           thread measured slower there (FP16 AA odd 0.61
//                           against 0.47 ms at 256^3): their accesses are
//                           per-cell gathers anyway, and the pair halved the
//                           threads in flight.
#pragma once

#include <type_traits>

#include "lbm_step_cp.cuh"
#include "lbm_step_x2.cuh"

namespace lbm {

// Register caps (minimum CTAs per SM) of the compact pair kernels.
#ifndef LBM_MINB_CP2_EVEN
#define LBM_MINB_CP2_EVEN 6
#endif
#ifndef LBM_MINB_CP2_EVEN16
#define LBM_MINB_CP2_EVEN16 5
#endif

// Cells per thread of the local kernel: 8-byte accesses in both storages.
#ifndef LBM_CP2_LOCAL16
#define LBM_CP2_LOCAL16 4
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

} // namespace lbm
