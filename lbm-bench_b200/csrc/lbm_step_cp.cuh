// Step kernels of the compact (fluid-only) layout: the same fused
// stream-collide-bounce-back(-force) step as step_kernel (lbm_step.cuh,
// whose header gives the per-pattern read and write rules and the
// bit-exactness argument), with every population plane and the link masks
// holding fluid cells only, in row order (Grid, lbm_device.cuh).
//
// The dense layout stores every cell, and a 128-byte line that holds both
// fluid and solid cells is fetched whole from HBM: in a 20%-solid porous
// channel that is 14% (FP64) to 26% (FP16) more DRAM traffic than the
// algorithmic 2 x 19 x S bytes per fluid update. The reference sweeps the
// dense box too (src/kernel_pull_soa.c:94-96). Here no solid cell occupies
// storage, so every fetched sector belongs to fluid cells.
//
// Threads still map to device cells - z across the lanes, one warp per 32
// consecutive z of one (x, y) row, starting at a multiple of 32 - and a
// solid lane leaves after one fluid-bit test. Because a warp's lanes share
// the row and the fluid-bit word, the storage index of a fluid cell and of
// its neighbours comes from nine warp-uniform word pairs (own row and the
// eight rows (x +- 1, y +- 1), one 8-byte load each): with B_q = base +
// popc(word_q & bits below z) and f_q the fluid bit of (row q, z),
//     index of (row q, z)     = B_q
//     index of (row q, z + 1) = B_q + f_q      (when that cell is fluid)
//     index of (row q, z - 1) = B_q - 1        (when that cell is fluid)
// which also holds across word boundaries (base of word w + 1 is base of
// word w plus its popcount). Only a periodic z axis breaks it at z = 0 and
// z = nz - 1; those lanes look the wrapped neighbour up directly. Whether a
// neighbour is fluid comes from the cell's link mask, as in the dense
// kernel, so a wall neighbour never needs an index.
#pragma once

#include "lbm_step.cuh"

namespace lbm {

// Register caps of the compact kernels (minimum CTAs per SM), per kind and
// storage width from sweeps on the 256^3 porous channel (B200). FP64: AA odd
// and pull are fastest at 8 CTAs/SM (64 registers; odd 0.963 ms at 6 with
// the row table in registers, 0.803 at 6 and 0.764 at 8 with it in shared
// memory), push at 7 (0.699 ms; 0.717 at 6, 0.757 at 8, with the row words
// and mask loaded together). FP32 and FP16 move
// a half and a quarter of the bytes and are bound by instruction issue, so
// more warps in flight pay: AA odd FP32 0.479 / 0.469 / 0.457 / 0.498 ms at
// 8 / 10 / 12 / 14, FP16 0.437 / 0.430 / 0.410 / 0.404; pull FP32 0.440 /
// 0.421 / 0.410 / 0.400, FP16 0.382 / 0.363 / 0.367 / 0.368; push stays at
// 8 (FP32 0.435 ms, FP16 0.362; 10 and 12 are slower). The local AA even
// step (at the HBM limit) does not care.
#ifndef LBM_MINB_CP_ODD
#define LBM_MINB_CP_ODD 8
#endif
#ifndef LBM_MINB_CP_ODD_F32
#define LBM_MINB_CP_ODD_F32 12
#endif
#ifndef LBM_MINB_CP_ODD_F16
#define LBM_MINB_CP_ODD_F16 14
#endif
#ifndef LBM_MINB_CP_PULL
#define LBM_MINB_CP_PULL 8
#endif
#ifndef LBM_MINB_CP_PULL_F32
#define LBM_MINB_CP_PULL_F32 14
#endif
#ifndef LBM_MINB_CP_PULL_F16
#define LBM_MINB_CP_PULL_F16 10
#endif
#ifndef LBM_MINB_CP_PUSH_F64
#define LBM_MINB_CP_PUSH_F64 7
#endif
#ifndef LBM_MINB_CP_PUSH_F32
#define LBM_MINB_CP_PUSH_F32 8
#endif
#ifndef LBM_MINB_CP_PUSH_F16
#define LBM_MINB_CP_PUSH_F16 8
#endif
#ifndef LBM_MINB_CP_EVEN
#define LBM_MINB_CP_EVEN 6
#endif
// SB: bytes of one stored population (8, 4 or 2).
template <int KIND, int SB> struct CpOccupancy {
  static constexpr int push = SB == 8 ? LBM_MINB_CP_PUSH_F64
      : SB == 4 ? LBM_MINB_CP_PUSH_F32 : LBM_MINB_CP_PUSH_F16;
  static constexpr int odd = SB == 8 ? LBM_MINB_CP_ODD
      : SB == 4 ? LBM_MINB_CP_ODD_F32 : LBM_MINB_CP_ODD_F16;
  static constexpr int pull = SB == 8 ? LBM_MINB_CP_PULL
      : SB == 4 ? LBM_MINB_CP_PULL_F32 : LBM_MINB_CP_PULL_F16;
  static constexpr int value = KIND == kAAEvenStep ? LBM_MINB_CP_EVEN
      : KIND == kAAOddStep ? odd : KIND == kPullStep ? pull : push;
};

// Storage indices of the 18 neighbours of one fluid cell (compact layout).
// Kernels that scatter (push, AA odd) need them again after the collision;
// they keep them in shared memory (one column per thread) rather than in
// registers across it. Entry q = (dx + 1) * 3 + (dy + 1) (q != 4) holds B_q,
// the index of (x + dx, y + dy, z) or of the next fluid z; entries 9..12
// hold B_q + f_q for the four axis rows q = 1, 3, 5, 7, the index of
// (row q, z + 1). ZPER: the z axis is periodic, and lanes on z = 0 or
// z = nz - 1 look their wrapped z neighbours up directly.
#ifndef LBM_CP_SMEM_TAB
#define LBM_CP_SMEM_TAB 1
#endif
// LBM_CP_INNER_ROWS: rows whose 3 x 3 neighbourhood does not wrap (almost
// all) find their neighbours' index words at fixed strides from their own.
// Used where it measured faster (256^3 porous channel): AA odd in every
// precision (FP16 0.404 -> 0.388 ms) and FP16 pull (0.364 -> 0.360); push
// (FP64 0.751 -> 0.806 ms) and FP32 pull (0.402 -> 0.418) were slower.
// LBM_CP_GATHER_REGS: the gather takes the table from registers; only the
// scatter after the collision reads the shared copy.
#ifndef LBM_CP_INNER_ROWS
#define LBM_CP_INNER_ROWS 1
#endif
#ifndef LBM_CP_GATHER_REGS
#define LBM_CP_GATHER_REGS 1
#endif
// LBM_CP_EARLY_ROWS: the neighbour rows' index words and the link mask are
// loaded together, before the solid lanes leave, instead of the mask first
// and the rows after the fluid test.
#ifndef LBM_CP_EARLY_ROWS
#define LBM_CP_EARLY_ROWS 1
#endif
constexpr int kTabRows = 13;

template <bool ZPER> struct RowTab {
  uint32_t B[kTabRows];
  uint32_t *sB = nullptr; // shared copy: sB[k * kStepThreads]
  bool zwrap = false;
  int x, y, z;

  __device__ __forceinline__ static int axis_slot(int q)
  {
    return q == 1 ? 9 : q == 3 ? 10 : q == 5 ? 11 : 12;
  }

  __device__ __forceinline__ void row(const Grid &g, int q, uint32_t k, uint32_t lt, int lane)
  {
    const uint2 wb = __ldg(g.wb + k);
    const uint32_t w = wb.x;
    B[q] = wb.y + (uint32_t)__popc(w & lt);
    if (q == 1 || q == 3 || q == 5 || q == 7)
      B[axis_slot(q)] = B[q] + ((w >> lane) & 1u);
  }

  // k0: index word of the thread's own row, ((x * ny) + y) * W + wi.
  // INNER: take the stride path for rows away from the box faces.
  template <bool INNER>
  __device__ __forceinline__ void build(const Grid &g, int x_, int y_, int z_, uint32_t cell,
      uint32_t wi, uint32_t lt, int lane, uint32_t k0)
  {
    x = x_;
    y = y_;
    z = z_;
    B[4] = cell;
    if (INNER && x > 0 && x < g.nx - 1 && y > 0 && y < g.ny - 1) {
      // warp-uniform branch: x is the block's plane, y the warp's row
      const uint32_t sy = (uint32_t)g.W, sx = (uint32_t)g.ny * sy;
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        if (q == 4)
          continue;
        const int dx = q / 3 - 1, dy = q % 3 - 1;
        uint32_t k = k0;
        k = dx < 0 ? k - sx : dx > 0 ? k + sx : k;
        k = dy < 0 ? k - sy : dy > 0 ? k + sy : k;
        row(g, q, k, lt, lane);
      }
    } else {
#pragma unroll
      for (int q = 0; q < 9; ++q) {
        if (q == 4)
          continue;
        int xr = x + q / 3 - 1, yr = y + q % 3 - 1;
        // out-of-range rows only occur on non-periodic faces, whose cells
        // are walls (the mask says so and the index is never used): wrap
        xr = xr < 0 ? g.nx - 1 : xr >= g.nx ? 0 : xr;
        yr = yr < 0 ? g.ny - 1 : yr >= g.ny ? 0 : yr;
        row(g, q, ((uint32_t)xr * (uint32_t)g.ny + (uint32_t)yr) * (uint32_t)g.W + wi, lt,
            lane);
      }
    }
    if (sB) {
#pragma unroll
      for (int k = 0; k < kTabRows; ++k)
        if (k != 4)
          sB[k * kStepThreads] = B[k];
    }
    if (ZPER)
      zwrap = z == 0 || z == g.nz - 1;
  }

  __device__ __forceinline__ uint32_t entry(int k, bool regs) const
  {
    return (!regs && sB && k != 4) ? sB[k * kStepThreads] : B[k];
  }

  // storage index of x + c_d; meaningful only when that cell is fluid.
  // regs: take the table from registers (while they still hold it)
  __device__ __forceinline__ uint32_t at(const Grid &g, int d, bool regs = false) const
  {
    const int q = (cx(d) + 1) * 3 + (cy(d) + 1);
    if (ZPER && cz(d) != 0 && zwrap) {
      int a = x + cx(d), b = y + cy(d), c = z + cz(d);
      a = a < 0 ? g.nx - 1 : a >= g.nx ? 0 : a;
      b = b < 0 ? g.ny - 1 : b >= g.ny ? 0 : b;
      c = c < 0 ? g.nz - 1 : c >= g.nz ? 0 : c;
      return packed_index(g, a, b, c);
    }
    if (cz(d) > 0)
      return q == 4 ? B[4] + 1u : entry(axis_slot(q), regs);
    if (cz(d) < 0)
      return entry(q, regs) - 1u;
    return entry(q, regs);
  }
};

// L2 prefetch of the compact AA odd step in FP64 and FP32 storage
// (cp_plane_prefetch below), its distance in tenths of a wave of blocks
// (prefetch_planes(); 0 turns it off). At 256^3 one wave ahead took FP64 AA
// odd from 0.743 to 0.722 ms and FP32 from 0.434 to 0.401 ms; two and four
// waves were slower than none. FP16 AA odd (0.365 -> 0.383 ms) and pull
// (FP64 0.665 -> 0.785 ms, FP16 0.317 -> 0.335 ms) got slower, so those
// kernels are compiled without it (push was not measured and has none).
#ifndef LBM_CP_PF_TENTHS
#define LBM_CP_PF_TENTHS 10
#endif
template <int KIND, int SB> constexpr bool cp_prefetches()
{
  return LBM_CP_PF_TENTHS > 0 && KIND == kAAOddStep && SB >= 4;
}

// Asks the L2 for the bytes [lo_b, hi_b) from `base`, widened to 16-byte
// bounds (cp.async.bulk.prefetch: a hint that returns no data). The caller
// keeps the widened range inside one allocation.
__device__ __forceinline__ void l2_prefetch_bytes(const void *base, unsigned long long lo_b,
    unsigned long long hi_b)
{
  lo_b &= ~15ull;
  hi_b = (hi_b + 15ull) & ~15ull;
  if (hi_b > lo_b)
    asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;"
                 :: "l"(static_cast<const char *>(base) + lo_b), "r"((uint32_t)(hi_b - lo_b)));
}

// L2 prefetch of the AA odd step. The stored cells of one x-plane are one
// contiguous range of every population plane and of the mask array - from
// the base of the plane's first index word to the end of its last - so the
// blocks of plane x share out the range of plane x + pf: thread t < 19 of a
// block asks for the block's slice of population plane t, thread 19 for
// its slice of the masks. By the time the blocks of plane x + pf run, their
// own and their neighbours' rows are in the L2. Slices stay inside the
// range, and the 16-byte widening inside the plane stride (a multiple of
// 256 bytes) or the mask array (padded to the plane stride).
template <typename S>
__device__ __forceinline__ void cp_plane_prefetch(const Grid &g, const S *src,
    const uint32_t *mask, int x, uint32_t pf)
{
  const unsigned t = threadIdx.y * blockDim.x + threadIdx.x;
  const long long xp = (long long)x + pf;
  if (t > (unsigned)Q || xp >= g.nx)
    return;
  const uint32_t rw = (uint32_t)g.ny * (uint32_t)g.W; // index words per plane
  const uint32_t kb = (uint32_t)xp * rw;
  const uint32_t s = __ldg(g.wb + kb).y;
  const uint2 we = __ldg(g.wb + kb + rw - 1u);
  const uint32_t e = we.y + (uint32_t)__popc(we.x);
  const unsigned long long nblk = (unsigned long long)gridDim.x * gridDim.y;
  const unsigned long long chunk = ((unsigned long long)(e - s) + nblk - 1) / nblk;
  const unsigned long long cb =
      s + chunk * ((unsigned long long)blockIdx.y * gridDim.x + blockIdx.x);
  if (cb >= e)
    return;
  const unsigned long long ce = cb + chunk < e ? cb + chunk : e;
  if (t < (unsigned)Q)
    l2_prefetch_bytes(src + (long long)t * g.plane, cb * sizeof(S), ce * sizeof(S));
  else
    l2_prefetch_bytes(mask, cb * 4ull, ce * 4ull);
}

// Arithmetic of the compact kernels. CpMathDirect: values as stored and
// collide() - the FP64 reference arithmetic (bit-identical to LBM-Bench).
// CpMathUnits (lbm_step_cp2.cuh): FP32/FP16 storage units and the pair
// kernels' arithmetic, one cell at a time.
template <class ST> struct CpMathDirect {
  using Args = StepArgs<ST>;
  using S = typename ST::S;
  using V = typename ST::V;
  __device__ static V ld(const Args &a, S s) { return ST::decode(s, a.c.inv_scale); }
  __device__ static S st(const Args &a, V v) { return ST::encode(v, a.c.scale); }
  __device__ static void coll(const Args &a, const V (&f)[Q], V (&o)[Q])
  {
    collide<V, false>(f, o, a.c, V(0));
  }
  __device__ static V plus(V x, V y) { return x + y; }
};

// The body-force term of direction d for a cell whose link d is (bb) or is
// not a wall: force[inv d] or force[d]. Both constants are rounded once from
// ((3 w_d) c_dx) F, so for c_dx = 0 they are the same value and otherwise
// force[inv d] is -force[d] bit for bit: the select is a sign flip of one
// constant, with the same result as loading and selecting two.
__device__ __forceinline__ float force_term(const float (&force)[Q], int d, bool bb)
{
  if (cx(d) == 0)
    return force[d];
  return __uint_as_float(__float_as_uint(force[d]) ^ ((uint32_t)bb << 31));
}
__device__ __forceinline__ double force_term(const double (&force)[Q], int d, bool bb)
{
  if (cx(d) == 0)
    return force[d];
  return __longlong_as_double(
      (long long)((unsigned long long)__double_as_longlong(force[d]) ^ ((unsigned long long)bb << 63)));
}

// OFF: type of element offsets within the state (uint32_t when all 19
// planes fit below 2^32 elements, which keeps address arithmetic 32-bit).
template <class M, int KIND, bool FORCE, bool ZPER, typename OFF>
__global__ void __launch_bounds__(kStepThreads, (CpOccupancy<KIND, sizeof(typename M::S)>::value))
    step_kernel_cp(typename M::Args a)
{
  using S = typename M::S;
  using V = typename M::V;
  constexpr bool kNC = (KIND == kPullStep || KIND == kPushStep);
  const Grid &g = a.g;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = a.x0 + (int)blockIdx.z;
  if (cp_prefetches<KIND, sizeof(S)>() && a.pf_planes)
    cp_plane_prefetch(g, a.src, a.mask, x, a.pf_planes);
  if (z >= g.nz || y >= g.ny)
    return;
  const int lane = z & 31;
  const uint32_t lt = (1u << lane) - 1u;
  const uint32_t wi = (uint32_t)(z >> 5);
  const uint32_t k0 = ((uint32_t)x * (uint32_t)g.ny + (uint32_t)y) * (uint32_t)g.W + wi;
  const uint2 wb0 = __ldg(g.wb + k0);
  const uint32_t w0 = wb0.x;
  const bool fluid = (w0 >> lane) & 1u;
  const uint32_t cell = wb0.y + (uint32_t)__popc(w0 & lt);
  const S *src = a.src;
  S *dst = a.dst;
  const OFF P = (OFF)g.plane;
  auto el = [&](int plane, uint32_t i) { return (OFF)plane * P + (OFF)i; };

  RowTab<ZPER> t;
  constexpr bool kScatter = (KIND == kPushStep || KIND == kAAOddStep);
  if (kScatter && LBM_CP_SMEM_TAB) {
    __shared__ uint32_t tab[kTabRows * kStepThreads];
    t.sB = tab + (threadIdx.y * blockDim.x + threadIdx.x);
  }
  constexpr bool kInner = LBM_CP_INNER_ROWS &&
      (KIND == kAAOddStep || (KIND == kPullStep && sizeof(S) == 2));
  uint32_t mask;
  if (LBM_CP_EARLY_ROWS && KIND != kAAEvenStep) {
    // the mask and the neighbour rows' words in one round trip, before the
    // solid lanes leave (a solid lane's number may be one past the last
    // stored cell: it reads word 0 instead)
    mask = __ldg(a.mask + (fluid ? cell : 0u));
    t.template build<kInner>(g, x, y, z, cell, wi, lt, lane, k0);
    if (!fluid)
      return;
  } else {
    if (!fluid)
      return;
    mask = __ldg(a.mask + cell);
    if (KIND != kAAEvenStep)
      t.template build<kInner>(g, x, y, z, cell, wi, lt, lane, k0);
  }
  constexpr bool kRegs = LBM_CP_GATHER_REGS != 0;

  V f[Q];
  if (KIND == kPushStep || KIND == kAAEvenStep) {
    // local loads: issued without waiting for the mask
#pragma unroll
    for (int d = 0; d < Q; ++d)
      f[d] = M::ld(a, ldg<kNC>(src + el(d, cell)));
  } else if (!__any_sync(__activemask(), (mask & 0x7FFFFu) != 0u)) {
    // no lane of the warp has a wall link: no redirects
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const OFF o = (KIND == kPullStep) ? el(d, t.at(g, inv(d), kRegs))
                                        : el(inv(d), t.at(g, inv(d), kRegs));
      f[d] = M::ld(a, ldg<kNC>(src + o));
    }
  } else {
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const bool back = (mask >> inv(d)) & 1u;
      OFF o;
      if (KIND == kPullStep)
        o = back ? el(inv(d), cell) : el(d, t.at(g, inv(d), kRegs));
      else
        o = back ? el(d, cell) : el(inv(d), t.at(g, inv(d), kRegs));
      f[d] = M::ld(a, ldg<kNC>(src + o));
    }
  }

  V o[Q];
  M::coll(a, f, o);

#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const bool bb = (mask >> d) & 1u;
    const V v = FORCE ? M::plus(o[d], force_term(a.c.force, d, bb)) : o[d];
    OFF off;
    if (KIND == kPullStep)
      off = el(d, cell);
    else if (KIND == kAAEvenStep)
      off = el(inv(d), cell);
    else
      off = bb ? el(inv(d), cell) : el(d, t.at(g, d));
    dst[off] = M::st(a, v);
  }
}

// The AA even step in the compact layout is local - a cell reads and writes
// only its own 19 slots - so threads map straight to storage indices: thread
// i updates cell c0 + i, a warp touches 32 consecutive elements of every
// plane, and the mask and population loads are issued together with no
// index lookup in front of them. Only the link mask (bounce-back force
// direction) is read besides the populations.
template <class ST, bool FORCE>
__global__ void __launch_bounds__(kStepThreads, (CpOccupancy<kAAEvenStep, sizeof(typename ST::S)>::value))
    step_kernel_cp_local(StepArgs<ST> a)
{
  using S = typename ST::S;
  using V = typename ST::V;
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= a.cn)
    return;
  const uint32_t cell = a.c0 + i;
  const uint32_t mask = __ldg(a.mask + cell);
  const long long P = a.g.plane;
  V f[Q];
#pragma unroll
  for (int d = 0; d < Q; ++d)
    f[d] = ST::decode(a.src[d * P + cell], a.c.inv_scale);
  V o[Q];
  collide<V, false>(f, o, a.c, V(0));
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const bool bb = (mask >> d) & 1u;
    const V v = FORCE ? o[d] + force_term(a.c.force, d, bb) : o[d];
    a.dst[inv(d) * P + cell] = ST::encode(v, a.c.scale);
  }
}

} // namespace lbm
