// Bulk-copy pipelined step kernels (cp.async.bulk + mbarrier, sm_90 and up).
//
// The one-cell-per-thread kernels of lbm_step.cuh keep 19 loads per thread
// in flight, and with the registers the collision needs only 6 CTAs of 128
// threads fit on an SM: those kernels are latency-bound (long-scoreboard
// stalls) below the HBM bandwidth. Here a producer warp copies whole rows
// into shared memory with cp.async.bulk, several tiles ahead, so the bytes
// in flight no longer depend on registers or occupancy:
//
//   tile    = T consecutive y rows (all of z) of one x plane
//   stage   = the 19 rows each direction reads for the tile, [d][T][pz], plus
//             the tile's link-mask rows; a ring of `stages` stages
//   CTA     = persistent over tiles blockIdx.x, + gridDim.x, ...; warp 0
//             produces (lane d issues direction d's rows, lane 19 the mask
//             rows); GROUPS groups of 8 consumer warps take the tiles in turn
//             and compute one cell per thread
//   barriers  full[s]: the stage's copies have landed (20 arrivals with
//             expect_tx); empty[s]: the 8 warps of the group that used it
//             are done with it
//
// The row of direction d is the source of f_d for every cell of the tile:
//   pull     plane d     of row (x - c_dx, y - c_dy)  (shifted rows)
//   AA odd   plane inv d of row (x - c_dx, y - c_dy)
//   push     plane d     of row (x, y)                 (local rows)
//   AA even  plane d     of row (x, y)
// so the z shift of a gather is an index shift in shared memory (wrapping
// within the row for a periodic z). Everything else - the bounce-back
// redirect to the cell's own slot, the collision, the stores, the force -
// is step_kernel's, operation for operation: results are bit-identical.
//
// Race freedom follows from the slot ownership of step_kernel: every slot
// of a copied row belongs to exactly one cell of the tile (or is row
// padding), so tiles never read what another tile writes in the same step.
// A row outside a non-periodic axis is not copied: the cells next to it are
// walls or see it through a wall link.
//
// `stages` must be a multiple of GROUPS: then stage s is always used by
// group s % GROUPS, one tile after another, so the barrier a consumer waits
// on is at most one phase behind it - a parity wait can only tell the
// current phase from the one before. (With stages % GROUPS != 0 a group
// could reach a stage whose previous tile, another group's, has not landed
// yet, and its parity wait would pass on the phase before that.)
//
// Waits are bounded (kWaitTries polls): a consumer whose stage never lands
// sets *err and leaves; the producer, whose empty barrier then never
// completes, sets *err, waits (bounded) for its copies in flight and leaves.
#pragma once

#include "lbm_step.cuh"

namespace lbm {

template <class ST> struct TmaArgs {
  StepArgs<ST> s;
  int T;                 // rows per tile
  int stages;            // pipeline depth
  int ytiles;            // tiles per x plane
  int ntiles;            // nx * ytiles
  uint32_t stage_bytes;  // one stage, 128-byte multiple
  unsigned int *err;     // set when a copy wait runs out
};

constexpr uint32_t kWaitTries = 1u << 24;

__device__ __forceinline__ uint32_t smem_addr(const void *p)
{
  return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint32_t bar, uint32_t count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(bar), "r"(count) : "memory");
}

__device__ __forceinline__ void fence_mbar_init()
{
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint32_t bar, uint32_t bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint32_t bar)
{
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(bar) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint32_t bar, uint32_t parity)
{
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\t"
               "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
               "selp.u32 %0, 1, 0, p;\n\t}"
               : "=r"(ok)
               : "r"(bar), "r"(parity)
               : "memory");
  return ok != 0u;
}

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity)
{
  for (uint32_t i = 0; i < kWaitTries; ++i)
    if (mbar_try_wait(bar, parity))
      return true;
  return false;
}

// global -> shared bulk copy completing on `bar` (addresses and size are
// 16-byte multiples: rows start on 32-byte sectors, planes on 256 bytes)
__device__ __forceinline__ void bulk_copy(uint32_t dst, const void *src, uint32_t bytes,
    uint32_t bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes "
               "[%0], [%1], %2, [%3];" ::"r"(dst),
               "l"(src), "r"(bytes), "r"(bar)
               : "memory");
}

// The copies of lane `lane` (0..18: direction, 19: the mask rows) of tile t
// into the stage at shared address `base`: expect_tx of their byte count on
// `bar` (arrival count 20, one per lane), then the copies.
template <class ST, int KIND>
__device__ void issue_lane(const TmaArgs<ST> &a, int t, int lane, uint32_t base, uint32_t bar)
{
  using S = typename ST::S;
  constexpr bool kGather = (KIND == kPullStep || KIND == kAAOddStep);
  const Grid &g = a.s.g;
  const int x = t / a.ytiles;
  const int y0 = (t - x * a.ytiles) * a.T;
  const int R = min(a.T, g.ny - y0);
  const uint32_t row_bytes = (uint32_t)g.pz * (uint32_t)sizeof(S);
  if (lane == Q) {
    const uint32_t mbytes = (uint32_t)R * (uint32_t)g.pz * 4u;
    mbar_expect_tx(bar, mbytes);
    const uint32_t *m = a.s.mask + ((size_t)x * (size_t)g.ny + (size_t)y0) * (size_t)g.pz;
    bulk_copy(base + (uint32_t)(Q * a.T) * row_bytes, m, mbytes, bar);
    return;
  }
  const int d = lane;
  const bool px = g.per & 1, py = (g.per >> 1) & 1;
  const int plane = (KIND == kAAOddStep) ? inv(d) : d;
  int xs = x, ys0 = y0;
  bool skip = false;
  if (kGather) {
    xs = x - cx(d);
    ys0 = y0 - cy(d);
    if (xs < 0 || xs >= g.nx) {
      if (px)
        xs = xs < 0 ? g.nx - 1 : 0;
      else
        skip = true;
    }
  }
  // at most two runs (a periodic wrap), each inside [0, ny)
  int js[3], ysv[3], runs[3], n = 0;
  uint32_t total = 0;
  for (int j = 0; j < R && !skip && n < 3;) {
    int ys = ys0 + j;
    if (ys < 0 || ys >= g.ny) {
      if (!py) {
        ++j;
        continue;
      }
      ys = ys < 0 ? ys + g.ny : ys - g.ny;
    }
    const int run = min(R - j, g.ny - ys);
    js[n] = j;
    ysv[n] = ys;
    runs[n] = run;
    ++n;
    total += (uint32_t)run * row_bytes;
    j += run;
  }
  mbar_expect_tx(bar, total);
  const S *src0 = a.s.src + (size_t)plane * (size_t)g.plane + (size_t)xs * (size_t)g.ny * g.pz;
  for (int i = 0; i < n; ++i)
    bulk_copy(base + ((uint32_t)(d * a.T + js[i])) * row_bytes,
        src0 + (size_t)ysv[i] * (size_t)g.pz, (uint32_t)runs[i] * row_bytes, bar);
}

// Warp 0 produces; GROUPS groups of kGroupWarps consumer warps take the
// tiles in turn (group i the tiles k = i, i + GROUPS, ...), so several tiles
// are computed at once.
constexpr int kGroupWarps = 8;
__host__ __device__ constexpr int tma_threads(int groups)
{
  return 32 * (kGroupWarps * groups + 1);
}

template <class ST, int KIND, bool FORCE, int GROUPS>
__global__ void __launch_bounds__(tma_threads(GROUPS), 1) step_kernel_tma(TmaArgs<ST> a)
{
  using S = typename ST::S;
  using V = typename ST::V;
  constexpr bool kGather = (KIND == kPullStep || KIND == kAAOddStep);
  constexpr bool kNC = (KIND == kPullStep || KIND == kPushStep);
  extern __shared__ __align__(128) unsigned char smem[];
  __shared__ __align__(8) uint64_t full[8], empty[8];
  const Grid &g = a.s.g;
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const S *src = a.s.src;
  S *dst = a.s.dst;
  const long long P = g.plane;
  const uint32_t row_elems = (uint32_t)g.pz;

  if (tid == 0) {
    for (int s = 0; s < a.stages; ++s) {
      mbar_init(smem_addr(&full[s]), Q + 1);
      mbar_init(smem_addr(&empty[s]), kGroupWarps);
    }
    fence_mbar_init();
  }
  __syncthreads();

  if (warp == 0) {
    // producer: tile k into stage k % stages once its previous use is done
    int k = 0;
    for (int t = blockIdx.x; t < a.ntiles; t += gridDim.x, ++k) {
      const int s = k % a.stages;
      if (k >= a.stages &&
          !mbar_wait(smem_addr(&empty[s]), (uint32_t)(((k / a.stages) - 1) & 1))) {
        if (lane == 0)
          atomicOr(a.err, 1u);
        break;
      }
      if (lane <= Q)
        issue_lane<ST, KIND>(a, t, lane, smem_addr(smem + (size_t)s * a.stage_bytes),
            smem_addr(&full[s]));
    }
    // drain: every issued stage has landed before the producer leaves
    if (lane == 0)
      for (int kk = (k > a.stages ? k - a.stages : 0); kk < k; ++kk)
        mbar_wait(smem_addr(&full[kk % a.stages]), (uint32_t)((kk / a.stages) & 1));
    return;
  }

  const int grp = (warp - 1) / kGroupWarps;
  const int ct = tid - 32 - grp * 32 * kGroupWarps, nct = 32 * kGroupWarps;
  for (int k = grp, t = blockIdx.x + grp * gridDim.x; t < a.ntiles;
       k += GROUPS, t += GROUPS * gridDim.x) {
    const int s = k % a.stages;
    if (!mbar_wait(smem_addr(&full[s]), (uint32_t)((k / a.stages) & 1))) {
      if (lane == 0)
        atomicOr(a.err, 1u);
      return;
    }
    const S *pops = reinterpret_cast<const S *>(smem + (size_t)s * a.stage_bytes);
    const uint32_t *msk = reinterpret_cast<const uint32_t *>(pops + (size_t)Q * a.T * row_elems);
    const int x = t / a.ytiles;
    const int y0 = (t - x * a.ytiles) * a.T;
    const int R = min(a.T, g.ny - y0);
    const int cells = R * g.nz;
    for (int c = ct; c < cells; c += nct) {
      const int j = c / g.nz;
      const int z = c - j * g.nz;
      const int y = y0 + j;
      const uint32_t mask = msk[j * row_elems + z];
      if (mask & kSolidBit)
        continue;
      const uint32_t cell = cell_index(g, x, y, z);
      const bool links = __any_sync(__activemask(), (mask & 0x7FFFFu) != 0u);
      V f[Q];
#pragma unroll
      for (int d = 0; d < Q; ++d) {
        const S *row = pops + (size_t)(d * a.T + j) * row_elems;
        S v;
        if (kGather) {
          int zs = z - cz(d);
          if (zs < 0)
            zs += g.nz;
          else if (zs >= g.nz)
            zs -= g.nz;
          v = row[zs];
          if (links && ((mask >> inv(d)) & 1u)) {
            // bounced off the wall x - c_d: the cell's own slot
            const S *p = (KIND == kPullStep) ? src + inv(d) * P + cell : src + d * P + cell;
            v = ldg<kNC>(p);
          }
        } else {
          v = row[z];
        }
        f[d] = ST::decode(v, a.s.c.inv_scale);
      }

      V o[Q];
      collide<V, false>(f, o, a.s.c, V(0), nullptr);

      const Offs of = make_offs(g, x, y, z);
#pragma unroll
      for (int d = 0; d < Q; ++d) {
        const bool bb = (mask >> d) & 1u;
        const V v = FORCE ? o[d] + (bb ? a.s.c.force[inv(d)] : a.s.c.force[d]) : o[d];
        S *p;
        if (KIND == kPullStep)
          p = dst + d * P + cell;
        else if (KIND == kAAEvenStep)
          p = dst + inv(d) * P + cell;
        else
          p = bb ? dst + inv(d) * P + cell : dst + d * P + (uint32_t)(cell + of.at(d));
        *p = ST::encode(v, a.s.c.scale);
      }
    }
    __syncwarp();
    if (lane == 0)
      mbar_arrive(smem_addr(&empty[s]));
  }
}

// Shape of the pipelined kernels for a grid, or false when two stages of
// one row do not fit (then the step_kernel path runs).
struct TmaShape {
  int T, stages, ytiles, ntiles, blocks;
  uint32_t stage_bytes;
};

inline bool tma_shape(const Grid &g, size_t elem, int want_T, int want_stages,
    size_t smem_limit, TmaShape &sh)
{
  const size_t row = (size_t)g.pz * elem;
  const size_t per_row = (size_t)Q * row + (size_t)g.pz * 4u;
  int T = want_T > 0 ? want_T : (int)(40960 / per_row);
  if (T < 1)
    T = 1;
  if (T > g.ny)
    T = g.ny;
  const size_t stage = ((size_t)T * per_row + 127) / 128 * 128;
  int stages = want_stages > 0 ? want_stages : (int)(smem_limit / stage);
  if (stages > 8)
    stages = 8;
  if (stages < 2 || (size_t)stages * stage > smem_limit)
    return false;
  sh.T = T;
  sh.stages = stages;
  sh.ytiles = (g.ny + T - 1) / T;
  sh.ntiles = g.nx * sh.ytiles;
  sh.stage_bytes = (uint32_t)stage;
  sh.blocks = 1;
  return true;
}

} // namespace lbm
