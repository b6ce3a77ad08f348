// Device-side building blocks of the D3Q19 TRT stream-collide-bounce-back
// step: lattice tables, the per-cell collision, population storage codecs
// and the orientation rules that let every propagation pattern fuse the
// bounce-back copies of the reference into its own loads and stores.
//
// Reference semantics (LBM-Bench):
//   collision      src/kernel_pull_soa.c:118-198 (identical in push and AA)
//   bounce-back    src/lbm.c:465-568 (index lists) applied by
//                  src/kernel_pull_soa.c:203-204, src/kernel_aa_soa.c:154-155,277-278
//   body force     src/lbm.c:902-922, applied after every step under -DVERIFICATION
//
// Device layout ("plane layout"): population d of cell index c lives at
//   f[d * plane + c]
// with the cell index of struct Grid below: z is the unit-stride axis, as
// in the reference's indexSoA (src/lbm.h:113-116); periodic neighbours are
// addressed by wrapping instead of through ghost copies.
//
// Link mask: one 32-bit word per cell. Bit d (0..18) is set when the
// neighbour x + c_d is an obstacle, so the population leaving along d
// bounces back. Bit 31 marks a wall cell (obstacle, frame or row padding),
// which is never computed.
#pragma once

#include <cuda_fp16.h>
#include <stdint.h>

namespace lbm {

constexpr int Q = 19;
constexpr uint32_t kSolidBit = 0x80000000u;

// Reference direction order N,S,E,W,NE,SE,NW,SW,T,TN,TE,TW,TS,B,BS,BN,BW,BE,C
// (src/lbm.h:20-38, src/lbm.c:20-29); it fixes the plane order.
enum Dir {
  dN = 0, dS, dE, dW, dNE, dSE, dNW, dSW, dT, dTN, dTE, dTW, dTS, dB, dBS, dBN, dBW, dBE, dC
};

__host__ __device__ constexpr int cx(int d)
{
  return (d == dE || d == dNE || d == dSE || d == dTE || d == dBE) ? 1
       : (d == dW || d == dNW || d == dSW || d == dTW || d == dBW) ? -1 : 0;
}
__host__ __device__ constexpr int cy(int d)
{
  return (d == dN || d == dNE || d == dNW || d == dTN || d == dBN) ? 1
       : (d == dS || d == dSE || d == dSW || d == dTS || d == dBS) ? -1 : 0;
}
__host__ __device__ constexpr int cz(int d)
{
  return (d == dT || d == dTN || d == dTE || d == dTW || d == dTS) ? 1
       : (d == dB || d == dBS || d == dBN || d == dBW || d == dBE) ? -1 : 0;
}
__host__ __device__ constexpr int inv(int d)
{
  return d == dN ? dS : d == dS ? dN : d == dE ? dW : d == dW ? dE
       : d == dNE ? dSW : d == dSW ? dNE : d == dSE ? dNW : d == dNW ? dSE
       : d == dT ? dB : d == dB ? dT : d == dTN ? dBS : d == dBS ? dTN
       : d == dTE ? dBW : d == dBW ? dTE : d == dTW ? dBE : d == dBE ? dTW
       : d == dTS ? dBN : d == dBN ? dTS : dC;
}
// lattice weight class: 0 -> 1/3 (centre), 1 -> 1/18 (axis), 2 -> 1/36 (diagonal)
__host__ __device__ constexpr int wclass(int d)
{
  return d == dC ? 0 : (cx(d) * cx(d) + cy(d) * cy(d) + cz(d) * cz(d) == 1 ? 1 : 2);
}

// Propagation patterns and the state orientations they leave behind.
enum Pattern { kPull = 0, kPush = 1, kAA = 2 };
enum Orientation {
  kNatural = 0,   // f_d(x) at (d, x): push state, AA after an odd step, initial AA state
  kPullState = 1, // f_d(x) at (d, x - c_d); at (inv d, x) if x - c_d is a wall
  kAAEven = 2     // f_d(x) at (inv d, x - c_d); at (d, x) if x - c_d is a wall
};
enum Kind { kPullStep = 0, kPushStep = 1, kAAEvenStep = 2, kAAOddStep = 3 };

// Storage codecs. Value type V is what the collision computes on:
// the population itself in FP64 mode (bit-exact reference arithmetic), the
// shifted deviation g_d = f_d - w_d in the reduced-precision modes.
struct StoreF64 {
  using S = double;
  using V = double;
  static constexpr bool kShifted = false;
  __device__ static V decode(S s, V) { return s; }
  __device__ static S encode(V v, V) { return v; }
  __device__ static V load(const S *p, int, V) { return *p; }
  __device__ static void store(S *p, V v, V) { *p = v; }
};
struct StoreF32 {
  using S = float;
  using V = float;
  static constexpr bool kShifted = true;
  __device__ static V decode(S s, V) { return s; }
  __device__ static S encode(V v, V) { return v; }
  __device__ static V load(const S *p, int, V) { return *p; }
  __device__ static void store(S *p, V v, V) { *p = v; }
};
// FP16 holds g_d * scale (scale a power of two), round-to-nearest-even.
struct StoreF16 {
  using S = __half;
  using V = float;
  static constexpr bool kShifted = true;
  __device__ static V decode(S s, V inv_scale) { return __half2float(s) * inv_scale; }
  __device__ static S encode(V v, V scale) { return __float2half_rn(v * scale); }
  __device__ static V load(const S *p, int, V inv_scale) { return __half2float(*p) * inv_scale; }
  __device__ static void store(S *p, V v, V scale) { *p = __float2half_rn(v * scale); }
};

template <typename V> struct Consts {
  V omegaEven, omegaOdd;
  V w0, w1, w2, w1X3, w1NineHalf, w2X3, w2NineHalf;
  V force[Q];  // ((3 w_d) c_dx) F, added to every population a fluid cell receives
  V scale;     // FP16 storage scale (1 otherwise)
  V inv_scale;
  V alpha;     // Brinkman coefficient scale
};

// One cell's TRT collision (src/kernel_pull_soa.c:118-198), operation for
// operation in the reference's order; FP64 translation units are compiled
// with --fmad=false so no multiply-add is contracted. In the shifted modes
// the same formulas hold with f -> g and rho -> rho - 1 because the shift is
// the rest equilibrium w_d. kappa != 0 adds the Brinkman resistance
// F_b = -kappa u as 3 w_d c_d . F_b = -/+ kappa (c_d . u) 3 w_d on each pair.
template <typename V, bool BRINK>
__device__ __forceinline__ void collide(const V (&f)[Q], V (&o)[Q], const Consts<V> &c, V kappa,
    V *u_out = nullptr)
{
  const V ux = f[dE] + f[dNE] + f[dSE] + f[dTE] + f[dBE] - f[dW] - f[dNW] - f[dSW] - f[dTW] - f[dBW];
  const V uy = f[dN] + f[dNE] + f[dNW] + f[dTN] + f[dBN] - f[dS] - f[dSE] - f[dSW] - f[dTS] - f[dBS];
  const V uz = f[dT] + f[dTE] + f[dTW] + f[dTN] + f[dTS] - f[dB] - f[dBE] - f[dBW] - f[dBN] - f[dBS];
  const V dens = f[dC] + f[dN] + f[dE] + f[dS] + f[dW] + f[dNE] + f[dSE] + f[dSW] + f[dNW] + f[dT] +
                 f[dTN] + f[dTE] + f[dTS] + f[dTW] + f[dB] + f[dBN] + f[dBE] + f[dBS] + f[dBW];
  const V dirIndepTrm = dens - (ux * ux + uy * uy + uz * uz) * V(3.0) / V(2.0);
  if (u_out) {
    u_out[0] = ux;
    u_out[1] = uy;
    u_out[2] = uz;
  }
  const V oE = c.omegaEven, oO = c.omegaOdd;
  o[dC] = f[dC] - oE * (f[dC] - c.w0 * dirIndepTrm);
  const V w1Indep = c.w1 * dirIndepTrm;
  const V w2Indep = c.w2 * dirIndepTrm;

  auto pair = [&](int a, int b, V ui, V wnh, V wx3, V windep) {
    const V evenPart = oE * (V(0.5) * (f[a] + f[b]) - ui * ui * wnh - windep);
    const V oddPart = oO * (V(0.5) * (f[a] - f[b]) - ui * wx3);
    if (BRINK) {
      const V bterm = kappa * ui * wx3;
      o[a] = f[a] - evenPart - oddPart - bterm;
      o[b] = f[b] - evenPart + oddPart + bterm;
    } else {
      o[a] = f[a] - evenPart - oddPart;
      o[b] = f[b] - evenPart + oddPart;
    }
  };
  pair(dN, dS, uy, c.w1NineHalf, c.w1X3, w1Indep);
  pair(dE, dW, ux, c.w1NineHalf, c.w1X3, w1Indep);
  pair(dT, dB, uz, c.w1NineHalf, c.w1X3, w1Indep);
  pair(dNW, dSE, -ux + uy, c.w2NineHalf, c.w2X3, w2Indep);
  pair(dNE, dSW, ux + uy, c.w2NineHalf, c.w2X3, w2Indep);
  pair(dTW, dBE, -ux + uz, c.w2NineHalf, c.w2X3, w2Indep);
  pair(dTE, dBW, ux + uz, c.w2NineHalf, c.w2X3, w2Indep);
  pair(dTS, dBN, -uy + uz, c.w2NineHalf, c.w2X3, w2Indep);
  pair(dTN, dBS, uy + uz, c.w2NineHalf, c.w2X3, w2Indep);
}

// Geometry of the device lattice, passed by value to every kernel.
// Cell (x, y, z), 0 <= x < nx etc., lives at cell = (x * ny + y) * pz + z;
// rows start on 32-byte sectors (pz rounds nz up) and the plane is rounded
// to 256 bytes. Periodic axes wrap. On a non-periodic axis every face cell
// is a wall: the reference's geometries put obstacle cells there
// (src/lbm.c:104-129), and where a caller's flags leave fluid on such a
// face the host embeds the box in a one-cell solid frame, so a fluid cell's
// neighbour always exists and a bounced population always has a wall slot
// to sit in (as in the reference's obstacle and ghost slots,
// src/lbm.c:532-566).
//
// Compact ("fluid-only") layout, when `wb` is set: only fluid cells hold
// storage. The fluid cells of one (x, y) row sit consecutively in z order,
// rows follow in (x, y) order, and a cell's storage index is its rank among
// all fluid cells. Per row, W pairs (word, base): `word` holds one fluid bit
// per z (bit z % 32 of pair z / 32), `base` the index of the first fluid
// cell at or after z = 32 w, so a fluid cell's index is
// base + popc(word & bits below z); one 8-byte load fetches both. Plane
// stride and mask array then count fluid cells only; no solid cell shares a
// 32-byte sector with a fluid one.
struct Grid {
  int nx, ny, nz;  // device extent (the caller's box plus frames)
  int pz;          // z pitch of a row, elements
  int per;         // periodic axes: bit 0 x, bit 1 y, bit 2 z
  long long plane; // elements per direction plane
  const uint2 *wb = nullptr; // compact layout: (fluid bits, first index) [nx*ny rows][W]
  int W = 0;                 // compact layout: words per row
};

// Caller's box inside the device box: offsets and extent.
struct UserBox {
  int ox, oy, oz;
  int nx, ny, nz;
};

// Cell index of device coordinates (below 2^32, checked at creation).
__device__ __forceinline__ uint32_t cell_index(const Grid &g, int x, int y, int z)
{
  return ((uint32_t)x * (uint32_t)g.ny + (uint32_t)y) * (uint32_t)g.pz + (uint32_t)z;
}

// Neighbour offsets of one cell, in cells, as 32-bit unsigned values:
// cell + at(d) (mod 2^32) is the neighbour x + c_d, wrapped across periodic
// axes. Only meaningful for fluid cells (which never sit on a non-periodic
// face). The x and y parts are uniform across a warp (a warp never spans
// two (x, y) rows); the z parts differ only at the ends of a row.
struct Offs {
  uint32_t xm, xp, ym, yp, zm, zp;
  __device__ __forceinline__ uint32_t at(int d) const
  {
    uint32_t o = 0u;
    if (cx(d) < 0)
      o += xm;
    else if (cx(d) > 0)
      o += xp;
    if (cy(d) < 0)
      o += ym;
    else if (cy(d) > 0)
      o += yp;
    if (cz(d) < 0)
      o += zm;
    else if (cz(d) > 0)
      o += zp;
    return o;
  }
};

__device__ __forceinline__ Offs make_offs(const Grid &g, int x, int y, int z)
{
  const uint32_t sy = (uint32_t)g.pz, sx = (uint32_t)g.ny * (uint32_t)g.pz;
  const bool px = g.per & 1, py = (g.per >> 1) & 1, pzz = (g.per >> 2) & 1;
  Offs o;
  o.xm = (px && x == 0) ? (uint32_t)(g.nx - 1) * sx : 0u - sx;
  o.xp = (px && x == g.nx - 1) ? 0u - (uint32_t)(g.nx - 1) * sx : sx;
  o.ym = (py && y == 0) ? (uint32_t)(g.ny - 1) * sy : 0u - sy;
  o.yp = (py && y == g.ny - 1) ? 0u - (uint32_t)(g.ny - 1) * sy : sy;
  o.zm = (pzz && z == 0) ? (uint32_t)(g.nz - 1) : 0u - 1u;
  o.zp = (pzz && z == g.nz - 1) ? 0u - (uint32_t)(g.nz - 1) : 1u;
  return o;
}

// Compact layout: storage index of the fluid cell (x, y, z) (device
// coordinates; the cell must be fluid).
__device__ __forceinline__ uint32_t packed_index(const Grid &g, int x, int y, int z)
{
  const uint32_t k =
      ((uint32_t)x * (uint32_t)g.ny + (uint32_t)y) * (uint32_t)g.W + (uint32_t)(z >> 5);
  const uint2 wb = __ldg(g.wb + k);
  return wb.y + (uint32_t)__popc(wb.x & ((1u << (z & 31)) - 1u));
}

// Storage index and link mask of the device cell (x, y, z) in either
// layout; false for a cell that is not updated (obstacle, frame, padding,
// ghost plane).
__device__ __forceinline__ bool locate(const Grid &g, const uint32_t *mask, int x, int y, int z,
    uint32_t &cell, uint32_t &m)
{
  if (g.wb) {
    const uint32_t k =
        ((uint32_t)x * (uint32_t)g.ny + (uint32_t)y) * (uint32_t)g.W + (uint32_t)(z >> 5);
    const uint2 wb = __ldg(g.wb + k);
    if (!((wb.x >> (z & 31)) & 1u))
      return false;
    cell = wb.y + (uint32_t)__popc(wb.x & ((1u << (z & 31)) - 1u));
  } else {
    cell = cell_index(g, x, y, z);
  }
  m = mask[cell];
  return !(m & kSolidBit);
}

// Neighbours of one fluid cell in either layout: at(d) is the storage
// index of x + c_d (wrapped across periodic axes), meaningful only when
// that neighbour is fluid (mask bit d clear).
struct Nbr {
  Offs o;
  uint32_t cell;
  int x, y, z;
  const Grid *g;
  __device__ __forceinline__ uint32_t at(int d) const
  {
    if (!g->wb)
      return cell + o.at(d);
    int a = x + cx(d), b = y + cy(d), c = z + cz(d);
    a = a < 0 ? g->nx - 1 : a >= g->nx ? 0 : a;
    b = b < 0 ? g->ny - 1 : b >= g->ny ? 0 : b;
    c = c < 0 ? g->nz - 1 : c >= g->nz ? 0 : c;
    return packed_index(*g, a, b, c);
  }
};

__device__ __forceinline__ Nbr make_nbr(const Grid &g, int x, int y, int z, uint32_t cell)
{
  Nbr n;
  n.o = make_offs(g, x, y, z);
  n.cell = cell;
  n.x = x;
  n.y = y;
  n.z = z;
  n.g = &g;
  return n;
}

// Where f_d(x) of a fluid cell lives in a state of orientation `o` (plane
// index, cell index). A population that bounced off the wall x - c_d is kept
// in a slot of the cell itself that no neighbour uses.
__device__ __forceinline__ void state_slot(int o, int d, uint32_t mask, uint32_t cell,
    const Nbr &n, int &plane_out, uint32_t &cell_out)
{
  const bool back = (mask >> inv(d)) & 1u; // x - c_d is a wall
  if (o == kNatural) {
    plane_out = d;
    cell_out = cell;
  } else if (o == kPullState) {
    plane_out = back ? inv(d) : d;
    cell_out = back ? cell : n.at(inv(d));
  } else {
    plane_out = back ? d : inv(d);
    cell_out = back ? cell : n.at(inv(d));
  }
}

// The same with the dense layout's neighbour offsets.
__device__ __forceinline__ void state_slot(int o, int d, uint32_t mask, uint32_t cell,
    const Offs &n, int &plane_out, uint32_t &cell_out)
{
  const bool back = (mask >> inv(d)) & 1u; // x - c_d is a wall
  if (o == kNatural) {
    plane_out = d;
    cell_out = cell;
  } else if (o == kPullState) {
    plane_out = back ? inv(d) : d;
    cell_out = back ? cell : cell + n.at(inv(d));
  } else {
    plane_out = back ? d : inv(d);
    cell_out = back ? cell : cell + n.at(inv(d));
  }
}

} // namespace lbm
