// liblbmb200: solver object and flat C ABI (include/lbm_b200.h).
//
// Replaces, for the SoA pull/push/AA kernels of LBM-Bench:
//   kernelInitInternal (src/lbm.c:400-599)  -> lbm_create: device buffers
//     and a per-cell link mask instead of bounce-back index lists;
//   kd->Kernel time loops (src/kernel_{pull,push,aa}_soa.c)  -> lbm_run;
//   Get/SetNode (src/lbm.c:193-294)  -> lbm_get_state / lbm_set_state,
//     converting between the caller's f[d][x][y][z] and the device
//     orientation of the pattern;
//   kernelDensity (src/lbm.c:928-947)  -> lbm_mass_momentum (FP64, on device);
//   kernelDeinit (src/lbm.c:660-670)  -> lbm_destroy.
// There is no CPU path: without a CUDA device every call that needs one
// fails with LBM_ERR_NODEV.
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <vector>

#include "lbm_b200.h"
#include "lbm_internal.h"

using namespace lbm;

static thread_local char g_err[512] = "";

static int fail(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

#define CUDA_TRY(call)                                                                      \
  do {                                                                                      \
    cudaError_t e_ = (call);                                                                \
    if (e_ != cudaSuccess)                                                                  \
      return fail(e_ == cudaErrorMemoryAllocation ? LBM_ERR_ALLOC : LBM_ERR_CUDA,          \
          "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__);     \
  } while (0)

struct lbm_solver {
  int nx, ny, nz; // caller's box
  int periodic[3];
  int pattern, precision;
  Grid g;     // device box (caller's box plus solid frames where needed)
  UserBox ub; // caller's box inside the device box
  int device;
  cudaStream_t stream;
  cudaEvent_t ev[2];
  void *buf[2];
  size_t state_bytes;
  int cur; // pull/push: buffer holding the state
  long long steps_done;
  uint32_t *mask;
  float *porosity;
  double alpha;
  double *staging; // one dense plane, nx*ny*nz doubles
  void *pstaging;  // one plane of the reference's padded layout (allocated on first use)
  size_t pstaging_bytes;
  double *red;     // reduction partials
  long long n_fluid;
  double omega, lambda, xforce;
  int force_on;
  double fp16_scale;
  long long launches;
  size_t dev_bytes;
  int no_shuffle; // reduced precision: never use the shuffle-aligned kernels
  int no_quad;    // FP16 AA: never use the four-cell kernels
  void *u_save_next; // adjoint recomputation: momentum output of the next step
  int slab;          // x-slab of a decomposed domain: device planes 0 and nx+1 are ghosts
  int tma;           // FP64 steps use the bulk-copy pipelined kernels (shape in tma_shape)
  int tma_groups;    // consumer groups of 8 warps per CTA
  TmaShape tma_shape;
  unsigned int *dev_err; // set by kernels whose bounded waits ran out
  uint8_t *bc_marks;     // [2][ny][nz]: inlet / outlet cells of the pressure boundary, or NULL
  int bc_on;
  double rho_in, rho_out;
  // split steps (lbm_step_begin / _planes / _end)
  cudaStream_t side;     // second stream, created on first use
  cudaEvent_t fork_ev, join_ev;
  int split;             // a split step is open
  uint8_t *split_done;   // host: x planes of the open step already launched (nx bytes)
  int split_left;        // planes still to launch
  // compact (fluid-only) layout: fluid bits and word bases per row (Grid)
  int compact;
  uint2 *cwb; // compact layout: (fluid bits, first index) per row word
  std::vector<uint32_t> *cplane0; // storage index of the first fluid cell of each x plane (nx+1)
};

extern "C" const char *lbm_last_error(void) { return g_err; }

int lbm::record_error(int code, const char *fmt, ...)
{
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}

extern "C" int lbm_compact_index(const unsigned char *fluid, long long rows, int nz, int pitch,
    unsigned int *bits, unsigned int *base, unsigned long long *total)
{
  if (!fluid || !bits || !base || rows < 0 || nz <= 0 || pitch < nz)
    return fail(LBM_ERR_ARG, "lbm_compact_index: bad arguments");
  const int W = (nz + 31) / 32;
  unsigned long long run = 0;
  for (long long r = 0; r < rows; ++r)
    for (int w = 0; w < W; ++w) {
      uint32_t word = 0;
      for (int b = 0; b < 32 && 32 * w + b < nz; ++b)
        word |= (uint32_t)(fluid[r * pitch + 32 * w + b] != 0) << b;
      bits[r * W + w] = word;
      base[r * W + w] = (uint32_t)run;
      run += (unsigned long long)__builtin_popcount(word);
    }
  if (run >= (1ull << 32))
    return fail(LBM_ERR_ARG, "lbm_compact_index: %llu fluid cells exceed the 32-bit numbering",
        run);
  if (total)
    *total = run;
  return LBM_OK;
}

extern "C" int lbm_device_count(void)
{
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n;
}

static size_t storage_size(int precision)
{
  return precision == LBM_F64 ? 8 : precision == LBM_F32 ? 4 : 2;
}

static int orientation(const lbm_solver *s)
{
  if (s->pattern == LBM_PULL)
    return kPullState;
  if (s->pattern == LBM_PUSH)
    return kNatural;
  return (s->steps_done & 1) ? kAAEven : kNatural;
}

// Lattice weights by direction.
static double weight(int d)
{
  int c = wclass(d);
  return c == 0 ? 1.0 / 3.0 : c == 1 ? 1.0 / 18.0 : 1.0 / 36.0;
}

// Kernel constants, computed in double exactly as the reference does
// (src/kernel_pull_soa.c:18-28, src/lbm.c:904-919) and rounded to V.
template <typename V> static Consts<V> make_consts(const lbm_solver *s)
{
  Consts<V> c;
  const double w0 = 1.0 / 3.0, w1 = 1.0 / 18.0, w2 = 1.0 / 36.0;
  c.omegaEven  = (V)s->omega;
  c.omegaOdd   = (V)(1.0 / (0.5 + s->lambda / (1.0 / s->omega - 0.5)));
  c.w0         = (V)w0;
  c.w1         = (V)w1;
  c.w2         = (V)w2;
  c.w1X3       = (V)(w1 * 3.0);
  c.w1NineHalf = (V)(w1 * 9.0 / 2.0);
  c.w2X3       = (V)(w2 * 3.0);
  c.w2NineHalf = (V)(w2 * 9.0 / 2.0);
  for (int d = 0; d < Q; ++d)
    c.force[d] = (V)(3.0 * weight(d) * (double)cx(d) * s->xforce);
  c.scale     = (V)(s->precision == LBM_F16 ? s->fp16_scale : 1.0);
  c.inv_scale = (V)(s->precision == LBM_F16 ? 1.0 / s->fp16_scale : 1.0);
  c.alpha     = (V)s->alpha;
  return c;
}

// Constants of the two-cell reduced-precision kernels, in storage units
// G = S g (S = 1 for FP32): the linear terms are unchanged, the quadratic
// ones (4.5 w ui^2 and 1.5 |u|^2) carry 1/S, forces carry S.
static Consts2 make_consts2(const lbm_solver *s)
{
  const double S = s->precision == LBM_F16 ? s->fp16_scale : 1.0;
  const double w1 = 1.0 / 18.0, w2 = 1.0 / 36.0;
  Consts2 c;
  c.oE    = (float)s->omega;
  c.oO    = (float)(1.0 / (0.5 + s->lambda / (1.0 / s->omega - 0.5)));
  c.w0    = (float)(1.0 / 3.0);
  c.w1    = (float)w1;
  c.w2    = (float)w2;
  c.w1X3  = (float)(w1 * 3.0);
  c.w2X3  = (float)(w2 * 3.0);
  c.w1NHq = (float)(w1 * 4.5 / S);
  c.w2NHq = (float)(w2 * 4.5 / S);
  c.c15q  = (float)(1.5 / S);
  // ((S 3 w_d) c_dx) F rounded once: force[inv d] is -force[d] bit for bit,
  // and force[d] = force[inv d] for c_dx = 0 (the compact local kernel
  // relies on both)
  for (int d = 0; d < Q; ++d)
    c.force[d] = (float)(S * 3.0 * weight(d) * (double)cx(d) * s->xforce);
  c.alpha = (float)s->alpha;
  return c;
}

// ---------------------------------------------------------------------------
// Auxiliary kernels
// ---------------------------------------------------------------------------

// One thread per device cell (z < pz): fluid cells get their link mask,
// every other cell (obstacle, frame, row padding) the wall bit.
// With ghost_x the planes x = 0 and x = nx-1 hold the neighbouring slabs'
// boundary cells: they are never updated here (wall bit), but the links of
// this slab's cells toward them follow their real flags.
__global__ void mask_kernel(Grid g, const uint8_t *fluid, uint32_t *mask, int ghost_x)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.pz || y >= g.ny)
    return;
  const uint32_t cell = cell_index(g, x, y, z);
  if (z >= g.nz || !fluid[cell] || (ghost_x && (x == 0 || x == g.nx - 1))) {
    mask[cell] = kSolidBit;
    return;
  }
  const bool px = g.per & 1, py = (g.per >> 1) & 1, pz = (g.per >> 2) & 1;
  uint32_t m = 0;
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    int a = x + cx(d), b = y + cy(d), c = z + cz(d);
    bool wall = false;
    if (a < 0 || a >= g.nx) {
      if (px)
        a = a < 0 ? g.nx - 1 : 0;
      else
        wall = true;
    }
    if (b < 0 || b >= g.ny) {
      if (py)
        b = b < 0 ? g.ny - 1 : 0;
      else
        wall = true;
    }
    if (c < 0 || c >= g.nz) {
      if (pz)
        c = c < 0 ? g.nz - 1 : 0;
      else
        wall = true;
    }
    if (!wall && !fluid[cell_index(g, a, b, c)])
      wall = true;
    if (wall)
      m |= 1u << d;
  }
  mask[cell] = m;
}

// Compact layout: the dense link masks of the fluid cells, moved to their
// storage indices.
__global__ void compact_mask_kernel(Grid g, const uint32_t *__restrict__ dense_mask,
    uint32_t *mask)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= g.nz || y >= g.ny)
    return;
  const uint32_t m = dense_mask[cell_index(g, x, y, z)];
  if (!(m & kSolidBit))
    mask[packed_index(g, x, y, z)] = m;
}

// Index of caller cell (x, y, z) in the caller's dense arrays.
__device__ __forceinline__ long long dense_index(const UserBox &u, int x, int y, int z)
{
  return ((long long)x * u.ny + y) * u.nz + z;
}

// Dense plane d (caller layout) -> device state in orientation `orient`.
template <class ST>
__global__ void pack_plane_kernel(Grid g, UserBox u, int d, int orient,
    const double *__restrict__ dense, typename ST::S *state, const uint32_t *__restrict__ mask,
    float scale, double wd)
{
  using V = typename ST::V;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= u.nz || y >= u.ny)
    return;
  uint32_t cell, m;
  if (!locate(g, mask, x + u.ox, y + u.oy, z + u.oz, cell, m))
    return;
  const Nbr nb = make_nbr(g, x + u.ox, y + u.oy, z + u.oz, cell);
  int p;
  uint32_t c;
  state_slot(orient, d, m, cell, nb, p, c);
  double v = dense[dense_index(u, x, y, z)];
  if (ST::kShifted)
    v -= wd;
  ST::store(state + (long long)p * g.plane + c, (V)v, (V)scale);
}

// Device state -> dense plane d (caller layout); obstacles get 0.
template <class ST>
__global__ void unpack_plane_kernel(Grid g, UserBox u, int d, int orient,
    double *__restrict__ dense, const typename ST::S *state, const uint32_t *__restrict__ mask,
    float inv_scale, double wd)
{
  using V = typename ST::V;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= u.nz || y >= u.ny)
    return;
  uint32_t cell, m;
  if (!locate(g, mask, x + u.ox, y + u.oy, z + u.oz, cell, m)) {
    dense[dense_index(u, x, y, z)] = 0.0;
    return;
  }
  const Nbr nb = make_nbr(g, x + u.ox, y + u.oy, z + u.oz, cell);
  int p;
  uint32_t c;
  state_slot(orient, d, m, cell, nb, p, c);
  double v = (double)ST::load(state + (long long)p * g.plane + c, d, (V)inv_scale);
  if (ST::kShifted)
    v += wd;
  dense[dense_index(u, x, y, z)] = v;
}

// Density and momentum of one fluid cell in FP64. For shifted storage the
// density is 1 + sum g (the shift sums to 1, its first moment to 0).
template <class ST>
__device__ __forceinline__ void cell_moments(const Grid &g, const typename ST::S *state,
    int orient, uint32_t m, uint32_t cell, const Nbr &nb, float inv_scale, double &rho,
    double &jx, double &jy, double &jz, bool &finite)
{
  using V = typename ST::V;
  rho = ST::kShifted ? 1.0 : 0.0;
  jx = jy = jz = 0.0;
  finite = true;
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    int p;
    uint32_t c;
    state_slot(orient, d, m, cell, nb, p, c);
    const double v = (double)ST::load(state + (long long)p * g.plane + c, d, (V)inv_scale);
    finite = finite && isfinite(v);
    rho += v;
    jx += cx(d) * v;
    jy += cy(d) * v;
    jz += cz(d) * v;
  }
}

// quantity: 0 rho, 1 ux, 2 uy, 3 uz (momentum) -> dense cell array
template <class ST>
__global__ void moments_kernel(Grid g, UserBox u, int orient, int quantity,
    const typename ST::S *state, const uint32_t *__restrict__ mask, float inv_scale, double *out)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= u.nz || y >= u.ny)
    return;
  uint32_t cell, m;
  double r = 0.0;
  if (locate(g, mask, x + u.ox, y + u.oy, z + u.oz, cell, m)) {
    const Nbr nb = make_nbr(g, x + u.ox, y + u.oy, z + u.oz, cell);
    double rho, jx, jy, jz;
    bool fin;
    cell_moments<ST>(g, state, orient, m, cell, nb, inv_scale, rho, jx, jy, jz, fin);
    r = quantity == 0 ? rho : quantity == 1 ? jx : quantity == 2 ? jy : jz;
  }
  out[dense_index(u, x, y, z)] = r;
}

constexpr int kRedThreads = 256;
constexpr int kRedBlocks = 592; // 4 per SM on a 148-SM B200; fixed for determinism
constexpr int kRedVals = 6;

// Fixed-shape tree reduction of kRedVals doubles inside one block.
// ops: bit k set -> value k is reduced with max instead of +.
__device__ void block_reduce(double (&v)[kRedVals], double *out, unsigned ops)
{
  __shared__ double sh[kRedVals][kRedThreads];
  for (int k = 0; k < kRedVals; ++k)
    sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int s = kRedThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int k = 0; k < kRedVals; ++k) {
        double a = sh[k][threadIdx.x], b = sh[k][threadIdx.x + s];
        sh[k][threadIdx.x] = ((ops >> k) & 1u) ? fmax(a, b) : a + b;
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < kRedVals; ++k)
      out[k] = sh[k][0];
}

// Per-block partial sums over cells i = blockIdx.x*T + threadIdx.x + k*grid*T
// of the dense box: mass, jx, jy, jz, non-finite cells.
template <class ST>
__global__ void __launch_bounds__(kRedThreads) mass_kernel(Grid g, int orient,
    const typename ST::S *state, const uint32_t *__restrict__ mask, float inv_scale,
    double *partial)
{
  double v[kRedVals] = { 0, 0, 0, 0, 0, 0 };
  const long long n = (long long)g.nx * g.ny * g.nz;
  for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kRedThreads) {
    const int z = (int)(i % g.nz);
    const long long r = i / g.nz;
    const int y = (int)(r % g.ny);
    const int x = (int)(r / g.ny);
    uint32_t cell, m;
    if (!locate(g, mask, x, y, z, cell, m))
      continue;
    const Nbr nb = make_nbr(g, x, y, z, cell);
    double rho, jx, jy, jz;
    bool fin;
    cell_moments<ST>(g, state, orient, m, cell, nb, inv_scale, rho, jx, jy, jz, fin);
    v[0] += rho;
    v[1] += jx;
    v[2] += jy;
    v[3] += jz;
    v[4] += fin ? 0.0 : 1.0;
  }
  block_reduce(v, partial + (size_t)blockIdx.x * kRedVals, 0u);
}

// Sum (or max, per ops) of nblocks partial rows in a fixed order.
__global__ void __launch_bounds__(kRedThreads) final_reduce_kernel(const double *partial,
    int nblocks, unsigned ops, double *out)
{
  double v[kRedVals];
  for (int k = 0; k < kRedVals; ++k)
    v[k] = 0.0;
  for (int b = threadIdx.x; b < nblocks; b += kRedThreads)
    for (int k = 0; k < kRedVals; ++k) {
      double x = partial[(size_t)b * kRedVals + k];
      v[k] = ((ops >> k) & 1u) ? fmax(v[k], x) : v[k] + x;
    }
  block_reduce(v, out, ops);
}

// Velocity/density differences of two states over the same geometry.
template <class SA, class SB>
__global__ void __launch_bounds__(kRedThreads) compare_kernel(Grid ga, Grid gb, int oa, int ob,
    const typename SA::S *sa, const typename SB::S *sb, const uint32_t *__restrict__ mask_a,
    const uint32_t *__restrict__ mask_b, float inv_a, float inv_b, double *partial)
{
  double v[kRedVals] = { 0, 0, 0, 0, 0, 0 };
  const long long n = (long long)ga.nx * ga.ny * ga.nz;
  for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kRedThreads) {
    const int z = (int)(i % ga.nz);
    const long long r = i / ga.nz;
    const int y = (int)(r % ga.ny);
    const int x = (int)(r / ga.ny);
    uint32_t ca, cb, ma, mb;
    if (!locate(ga, mask_a, x, y, z, ca, ma) || !locate(gb, mask_b, x, y, z, cb, mb))
      continue;
    const Nbr na = make_nbr(ga, x, y, z, ca), nbb = make_nbr(gb, x, y, z, cb);
    double ra, xa, ya, za, rb, xb, yb, zb;
    bool fa, fb;
    cell_moments<SA>(ga, sa, oa, ma, ca, na, inv_a, ra, xa, ya, za, fa);
    cell_moments<SB>(gb, sb, ob, mb, cb, nbb, inv_b, rb, xb, yb, zb, fb);
    const double dx = xa - xb, dy = ya - yb, dz = za - zb, dr = ra - rb;
    const double du2 = dx * dx + dy * dy + dz * dz, ub2 = xb * xb + yb * yb + zb * zb;
    v[0] += du2;
    v[1] += ub2;
    v[2] += dr * dr;
    v[3] += rb * rb;
    v[4] = fmax(v[4], sqrt(du2));
    v[5] = fmax(v[5], sqrt(ub2));
  }
  block_reduce(v, partial + (size_t)blockIdx.x * kRedVals, 0x30u);
}

// Sum of the x momentum and fluid count over the plane x = nx-1.
template <class ST>
__global__ void __launch_bounds__(kRedThreads) outlet_kernel(Grid g, int x, int orient,
    const typename ST::S *state, const uint32_t *__restrict__ mask, float inv_scale,
    double *partial)
{
  double v[kRedVals] = { 0, 0, 0, 0, 0, 0 };
  const long long n = (long long)g.ny * g.nz;
  for (long long i = (long long)blockIdx.x * kRedThreads + threadIdx.x; i < n;
       i += (long long)gridDim.x * kRedThreads) {
    const int z = (int)(i % g.nz);
    const int y = (int)(i / g.nz);
    uint32_t cell, m;
    if (!locate(g, mask, x, y, z, cell, m))
      continue;
    const Nbr nb = make_nbr(g, x, y, z, cell);
    double rho, jx, jy, jz;
    bool fin;
    cell_moments<ST>(g, state, orient, m, cell, nb, inv_scale, rho, jx, jy, jz, fin);
    v[0] += jx;
    v[1] += 1.0;
  }
  block_reduce(v, partial + (size_t)blockIdx.x * kRedVals, 0u);
}

// ---------------------------------------------------------------------------
// Helpers
// ---------------------------------------------------------------------------

static const void *state_ptr(const lbm_solver *s)
{
  return s->pattern == LBM_AA ? s->buf[0] : s->buf[s->cur];
}

static int need_device(void)
{
  if (lbm_device_count() <= 0)
    return fail(LBM_ERR_NODEV, "no CUDA device visible; liblbmb200 has no CPU path");
  return LBM_OK;
}

static void free_all(lbm_solver *s)
{
  if (!s)
    return;
  cudaFree(s->buf[0]);
  cudaFree(s->buf[1]);
  cudaFree(s->mask);
  cudaFree(s->porosity);
  cudaFree(s->staging);
  cudaFree(s->pstaging);
  cudaFree(s->red);
  cudaFree(s->dev_err);
  cudaFree(s->bc_marks);
  cudaFree(s->cwb);
  delete s->cplane0;
  free(s->split_done);
  if (s->fork_ev)
    cudaEventDestroy(s->fork_ev);
  if (s->join_ev)
    cudaEventDestroy(s->join_ev);
  if (s->side)
    cudaStreamDestroy(s->side);
  if (s->ev[0])
    cudaEventDestroy(s->ev[0]);
  if (s->ev[1])
    cudaEventDestroy(s->ev[1]);
  if (s->stream)
    cudaStreamDestroy(s->stream);
  free(s);
}

static int dev_alloc(lbm_solver *s, void **p, size_t bytes, const char *what)
{
  cudaError_t e = cudaMalloc(p, bytes);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *p = NULL;
    return fail(e == cudaErrorMemoryAllocation ? LBM_ERR_ALLOC : LBM_ERR_CUDA,
        "cudaMalloc of %.3f GB for %s failed: %s", bytes / 1e9, what, cudaGetErrorString(e));
  }
  s->dev_bytes += bytes;
  return LBM_OK;
}

// ---------------------------------------------------------------------------
// C ABI
// ---------------------------------------------------------------------------

// slab = 1: flags has nx + 2 planes in x (x fastest); planes 0 and nx + 1
// are the neighbouring slabs' boundary planes and become ghost planes.
static int create_impl(lbm_solver **out, int nx, int ny, int nz, const int *flags,
    int periodic_x, int periodic_y, int periodic_z, int pattern, int precision, int slab,
    int compact = 0)
{
  if (!out)
    return fail(LBM_ERR_ARG, "lbm_create: out is NULL");
  *out = NULL;
  if (nx <= 0 || ny <= 0 || nz <= 0 || !flags)
    return fail(LBM_ERR_ARG, "lbm_create: bad dimensions %dx%dx%d or NULL flags", nx, ny, nz);
  if (pattern != LBM_PULL && pattern != LBM_PUSH && pattern != LBM_AA)
    return fail(LBM_ERR_ARG, "lbm_create: unknown pattern %d", pattern);
  if (precision != LBM_F64 && precision != LBM_F32 && precision != LBM_F16)
    return fail(LBM_ERR_ARG, "lbm_create: unknown precision %d", precision);
  int rc = need_device();
  if (rc)
    return rc;

  lbm_solver *s = (lbm_solver *)calloc(1, sizeof(lbm_solver));
  if (!s)
    return fail(LBM_ERR_ALLOC, "lbm_create: host allocation failed");
  s->nx = nx;
  s->ny = ny;
  s->nz = nz;
  s->slab = slab;
  s->periodic[0] = periodic_x && !slab ? 1 : 0;
  s->periodic[1] = periodic_y ? 1 : 0;
  s->periodic[2] = periodic_z ? 1 : 0;
  s->pattern = pattern;
  s->precision = precision;
  s->omega = 1.0;
  s->lambda = 1.0 / 12.0;
  s->xforce = 1e-5;
  s->force_on = 0;
  s->fp16_scale = 16384.0;
  {
    const char *ns = getenv("LBM_B200_NO_SHUFFLE");
    s->no_shuffle = (ns && ns[0] == '1') ? 1 : 0;
    const char *nq = getenv("LBM_B200_NO_QUAD");
    s->no_quad = (nq && nq[0] == '1') ? 1 : 0;
  }
  cudaGetDevice(&s->device);

  const size_t S = storage_size(precision);
  const int zq = (int)(32 / S); // z pitch quantum: rows start on a 32-byte sector
  // a non-periodic axis whose faces hold fluid gets a one-cell solid frame
  int frame[3] = { 0, 0, 0 };
  const int dims[3] = { nx, ny, nz };
  const int fx = nx + 2 * slab; // x extent of the flags array
  for (int a = slab ? 1 : 0; a < 3; ++a) {
    if (s->periodic[a])
      continue;
    for (int x = 0; x < nx && !frame[a]; ++x)
      for (int y = 0; y < ny && !frame[a]; ++y)
        for (int z = 0; z < nz; ++z) {
          const int c[3] = { x, y, z };
          if ((c[a] == 0 || c[a] == dims[a] - 1) && flags[((long long)z * ny + y) * fx + x + slab]) {
            frame[a] = 1;
            break;
          }
        }
  }
  if (slab)
    frame[0] = 1; // the ghost planes take the place of an x frame
  s->ub.ox = frame[0];
  s->ub.oy = frame[1];
  s->ub.oz = frame[2];
  s->ub.nx = nx;
  s->ub.ny = ny;
  s->ub.nz = nz;
  s->g.nx = nx + 2 * frame[0];
  s->g.ny = ny + 2 * frame[1];
  s->g.nz = nz + 2 * frame[2];
  s->g.pz = (s->g.nz + zq - 1) / zq * zq;
  s->g.per = s->periodic[0] | (s->periodic[1] << 1) | (s->periodic[2] << 2);
  long long cells = (long long)s->g.nx * s->g.ny * s->g.pz;
  if (s->g.nx > 65535) {
    free(s);
    return fail(LBM_ERR_ARG, "lbm_create: x extent %d exceeds 65535", s->g.nx);
  }
  if (cells >= (1LL << 32)) {
    free(s);
    return fail(LBM_ERR_ARG, "lbm_create: %lld cells (with z padding) exceed the 2^32 limit "
        "of the 32-bit cell index", cells);
  }
  const long long pq = 256 / (long long)S;
  s->g.plane = (cells + pq - 1) / pq * pq;

  // fluid bytes in device cell order (frames and padding = wall)
  std::vector<uint8_t> fluid((size_t)cells, 0);
  long long nf = 0;
  for (int x = -slab; x < nx + slab; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        uint8_t f = flags[((long long)z * ny + y) * fx + x + slab] != 0;
        fluid[((size_t)(x + frame[0]) * s->g.ny + (y + frame[1])) * s->g.pz + z + frame[2]] = f;
        if (x >= 0 && x < nx)
          nf += f;
      }
  s->n_fluid = nf;

  // compact layout: one fluid bit per cell and the storage index of the
  // first fluid cell of every 32-cell word, rows in (x, y) order
  std::vector<uint32_t> hbits, hbase;
  s->compact = compact;
  if (s->compact) {
    const int W = (s->g.nz + 31) / 32;
    const size_t rows = (size_t)s->g.nx * s->g.ny;
    hbits.assign(rows * W, 0u);
    hbase.assign(rows * W, 0u);
    unsigned long long total = 0;
    lbm_compact_index(fluid.data(), (long long)rows, s->g.nz, s->g.pz, hbits.data(), hbase.data(),
        &total);
    const uint32_t run = (uint32_t)total;
    s->g.W = W;
    s->cplane0 = new std::vector<uint32_t>((size_t)s->g.nx + 1);
    for (int x = 0; x < s->g.nx; ++x)
      (*s->cplane0)[x] = hbase[(size_t)x * s->g.ny * W];
    (*s->cplane0)[s->g.nx] = run;
    s->g.plane = ((long long)run + pq - 1) / pq * pq;
    if (s->g.plane == 0)
      s->g.plane = pq;
  }
  s->state_bytes = (size_t)Q * (size_t)s->g.plane * S;

#define TRY(x)                                                                              \
  do {                                                                                      \
    int r_ = (x);                                                                           \
    if (r_) {                                                                               \
      free_all(s);                                                                          \
      return r_;                                                                            \
    }                                                                                       \
  } while (0)
#define TRYC(x)                                                                             \
  do {                                                                                      \
    cudaError_t e_ = (x);                                                                   \
    if (e_ != cudaSuccess) {                                                                \
      free_all(s);                                                                          \
      return fail(LBM_ERR_CUDA, "%s failed: %s", #x, cudaGetErrorString(e_));               \
    }                                                                                       \
  } while (0)

  if (slab) {
    // a slab's stream carries the halo exchange and the boundary planes of
    // split steps: it outranks the second stream with the interior planes
    int least = 0, greatest = 0;
    TRYC(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    TRYC(cudaStreamCreateWithPriority(&s->stream, cudaStreamNonBlocking, greatest));
  } else {
    TRYC(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking));
  }
  TRYC(cudaEventCreate(&s->ev[0]));
  TRYC(cudaEventCreate(&s->ev[1]));
  TRY(dev_alloc(s, &s->buf[0], s->state_bytes, "the population lattice"));
  if (pattern != LBM_AA)
    TRY(dev_alloc(s, &s->buf[1], s->state_bytes, "the second population lattice"));
  TRY(dev_alloc(s, (void **)&s->mask, (size_t)s->g.plane * 4, "the link masks"));
  TRY(dev_alloc(s, (void **)&s->staging, sizeof(double) * (size_t)nx * ny * nz,
      "the transfer plane"));
  TRY(dev_alloc(s, (void **)&s->red, sizeof(double) * kRedVals * (kRedBlocks + 1),
      "reduction partials"));
  TRYC(cudaMemsetAsync(s->buf[0], 0, s->state_bytes, s->stream));
  if (s->buf[1])
    TRYC(cudaMemsetAsync(s->buf[1], 0, s->state_bytes, s->stream));

  TRY(dev_alloc(s, (void **)&s->dev_err, sizeof(unsigned int), "the kernel error word"));
  TRYC(cudaMemsetAsync(s->dev_err, 0, sizeof(unsigned int), s->stream));
  {
    // pipelined FP64 kernels (lbm_step_tma.cuh): with LBM_B200_TMA=1;
    // LBM_B200_TMA_T / _STAGES / _GROUPS set the tile rows, pipeline depth
    // and consumer groups
    const char *e = getenv("LBM_B200_TMA");
    const auto env_int = [](const char *n) {
      const char *v = getenv(n);
      return v ? atoi(v) : 0;
    };
    int optin = 0, sms = 0;
    cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, s->device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    s->tma = precision == LBM_F64 && !s->compact && e && e[0] == '1' && optin > 1024 &&
        tma_shape(s->g, storage_size(precision), env_int("LBM_B200_TMA_T"),
            env_int("LBM_B200_TMA_STAGES"), (size_t)optin - 1024, s->tma_shape);
    s->tma_groups = env_int("LBM_B200_TMA_GROUPS");
    if (s->tma_groups < 1 || s->tma_groups > 3)
      s->tma_groups = 2;
    if (s->tma) {
      // each stage belongs to one consumer group: a multiple of the groups
      s->tma_shape.stages -= s->tma_shape.stages % s->tma_groups;
      s->tma = s->tma_shape.stages >= s->tma_groups;
      s->tma_shape.blocks = s->tma_shape.ntiles < sms ? s->tma_shape.ntiles : sms;
    }
  }

  {
    // cells of the Zou-He pressure boundary (src/lbm.c:693-700): flag 2 on
    // x = 0 and flag 4 on x = nx - 1, on the interior rows 1..ny-2, 1..nz-2
    std::vector<uint8_t> marks((size_t)2 * ny * nz, 0);
    bool any = false;
    for (int side = 0; side < 2 && !slab; ++side)
      for (int y = 1; y < ny - 1; ++y)
        for (int z = 1; z < nz - 1; ++z) {
          const int x = side ? nx - 1 : 0;
          if (flags[((long long)z * ny + y) * nx + x] == (side ? 4 : 2)) {
            marks[((size_t)side * ny + y) * nz + z] = 1;
            any = true;
          }
        }
    if (any) {
      TRY(dev_alloc(s, (void **)&s->bc_marks, marks.size(), "the pressure-boundary marks"));
      TRYC(cudaMemcpy(s->bc_marks, marks.data(), marks.size(), cudaMemcpyHostToDevice));
    }
  }

  // the link masks: built on the dense cells, then (compact layout) moved to
  // the fluid cells' storage indices
  if (s->compact) {
    const size_t nw = hbits.size() * sizeof(uint32_t);
    std::vector<uint2> hwb(hbits.size());
    for (size_t k = 0; k < hwb.size(); ++k)
      hwb[k] = make_uint2(hbits[k], hbase[k]);
    TRY(dev_alloc(s, (void **)&s->cwb, 2 * nw, "the compact layout's index"));
    TRYC(cudaMemcpy(s->cwb, hwb.data(), 2 * nw, cudaMemcpyHostToDevice));
    s->g.wb = s->cwb;
  }
  Grid gd = s->g; // dense view of the box for the mask build
  gd.wb = nullptr;
  const long long dense_plane = (cells + pq - 1) / pq * pq;
  uint32_t *dmask = s->mask;
  if (s->compact)
    TRYC(cudaMalloc((void **)&dmask, (size_t)dense_plane * 4));
  uint8_t *dfluid = NULL;
  cudaError_t e = cudaMalloc((void **)&dfluid, (size_t)cells);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(dfluid, fluid.data(), (size_t)cells, cudaMemcpyHostToDevice, s->stream);
  if (e == cudaSuccess) {
    Grid gp = gd;
    gp.nz = s->g.pz; // cover the row padding too
    dim3 grid, block;
    cell_launch_shape(gp, grid, block);
    mask_kernel<<<grid, block, 0, s->stream>>>(gd, dfluid, dmask, s->slab);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess && s->compact) {
    e = cudaMemsetAsync(s->mask, 0xFF, (size_t)s->g.plane * 4, s->stream); // unused: walls
    dim3 grid, block;
    cell_launch_shape(s->g, grid, block);
    if (e == cudaSuccess)
      compact_mask_kernel<<<grid, block, 0, s->stream>>>(s->g, dmask, s->mask);
    if (e == cudaSuccess)
      e = cudaGetLastError();
  }
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(s->stream);
  cudaFree(dfluid);
  if (s->compact)
    cudaFree(dmask);
  if (e != cudaSuccess) {
    free_all(s);
    return fail(LBM_ERR_CUDA, "lbm_create: mask build failed: %s", cudaGetErrorString(e));
  }
  // cells beyond the box inside the rounded plane stay unused; mark them as
  // walls so no kernel that walks the whole plane treats them as fluid
  if (!s->compact && s->g.plane > cells) {
    std::vector<uint32_t> pad((size_t)(s->g.plane - cells), kSolidBit);
    TRYC(cudaMemcpy(s->mask + cells, pad.data(), pad.size() * 4, cudaMemcpyHostToDevice));
  }
#undef TRY
#undef TRYC
  *out = s;
  return LBM_OK;
}

extern "C" int lbm_create(lbm_solver **out, int nx, int ny, int nz, const int *flags,
    int periodic_x, int periodic_y, int periodic_z, int pattern, int precision)
{
  return create_impl(out, nx, ny, nz, flags, periodic_x, periodic_y, periodic_z, pattern,
      precision, 0);
}

extern "C" int lbm_create_compact(lbm_solver **out, int nx, int ny, int nz, const int *flags,
    int periodic_x, int periodic_y, int periodic_z, int pattern, int precision)
{
  return create_impl(out, nx, ny, nz, flags, periodic_x, periodic_y, periodic_z, pattern,
      precision, 0, 1);
}

extern "C" int lbm_is_compact(const lbm_solver *s) { return s ? s->compact : -1; }

extern "C" int lbm_create_slab_compact(lbm_solver **out, int nx, int ny, int nz,
    const int *flags, int periodic_y, int periodic_z, int pattern, int precision)
{
  return create_impl(out, nx, ny, nz, flags, 0, periodic_y, periodic_z, pattern, precision, 1,
      1);
}

extern "C" int lbm_create_slab(lbm_solver **out, int nx, int ny, int nz, const int *flags,
    int periodic_y, int periodic_z, int pattern, int precision)
{
  return create_impl(out, nx, ny, nz, flags, 0, periodic_y, periodic_z, pattern, precision, 1);
}

extern "C" int lbm_destroy(lbm_solver *s)
{
  if (!s)
    return LBM_OK;
  cudaStreamSynchronize(s->stream);
  free_all(s);
  return LBM_OK;
}

extern "C" int lbm_set_params(lbm_solver *s, double omega, double lambda, double xforce,
    int force_on)
{
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_set_params: NULL solver");
  if (!(omega > 0.0 && omega < 2.0))
    return fail(LBM_ERR_ARG, "lbm_set_params: omega = %g outside (0, 2)", omega);
  if (!(lambda > 0.0) || !isfinite(xforce))
    return fail(LBM_ERR_ARG, "lbm_set_params: bad Lambda %g or force %g", lambda, xforce);
  s->omega = omega;
  s->lambda = lambda;
  s->xforce = xforce;
  s->force_on = force_on ? 1 : 0;
  return LBM_OK;
}

extern "C" int lbm_set_fp16_scale(lbm_solver *s, double scale)
{
  if (!s || s->precision != LBM_F16)
    return fail(LBM_ERR_ARG, "lbm_set_fp16_scale: not an FP16 solver");
  int ex;
  if (!(scale > 0.0) || frexp(scale, &ex) != 0.5)
    return fail(LBM_ERR_ARG, "lbm_set_fp16_scale: %g is not a power of two", scale);
  s->fp16_scale = scale;
  return LBM_OK;
}

extern "C" int lbm_set_porosity(lbm_solver *s, const float *porosity, double alpha)
{
  if (s && s->compact)
    return fail(LBM_ERR_ARG, "lbm_set_porosity: the compact layout has no Brinkman term "
        "(use lbm_create)");
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_set_porosity: NULL solver");
  if (alpha == 0.0) {
    s->alpha = 0.0;
    return LBM_OK;
  }
  if (!porosity || !(alpha > 0.0))
    return fail(LBM_ERR_ARG, "lbm_set_porosity: NULL porosity or alpha %g <= 0", alpha);
  if (!s->porosity) {
    int rc = dev_alloc(s, (void **)&s->porosity, sizeof(float) * (size_t)s->g.plane,
        "the porosity field");
    if (rc)
      return rc;
    CUDA_TRY(cudaMemsetAsync(s->porosity, 0, sizeof(float) * (size_t)s->g.plane, s->stream));
  }
  for (int x = 0; x < s->nx; ++x)
    for (int y = 0; y < s->ny; ++y)
      CUDA_TRY(cudaMemcpyAsync(s->porosity + ((size_t)(x + s->ub.ox) * s->g.ny + (y + s->ub.oy)) *
                                                  s->g.pz + s->ub.oz,
          porosity + ((size_t)x * s->ny + y) * s->nz, sizeof(float) * s->nz,
          cudaMemcpyHostToDevice, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  s->alpha = alpha;
  return LBM_OK;
}

// Launch shape covering the caller's box.
static void user_launch_shape(const lbm_solver *s, dim3 &grid, dim3 &block)
{
  Grid gu = s->g;
  gu.nx = s->ub.nx;
  gu.ny = s->ub.ny;
  gu.nz = s->ub.nz;
  cell_launch_shape(gu, grid, block);
}

template <class ST> static int pack_all(lbm_solver *s, const double *f)
{
  dim3 grid, block;
  user_launch_shape(s, grid, block);
  const int o = orientation(s);
  const size_t plane_host = (size_t)s->nx * s->ny * s->nz;
  using Sx = typename ST::S;
  Sx *state = (Sx *)state_ptr(s);
  for (int d = 0; d < Q; ++d) {
    CUDA_TRY(cudaMemcpyAsync(s->staging, f + d * plane_host, sizeof(double) * plane_host,
        cudaMemcpyHostToDevice, s->stream));
    pack_plane_kernel<ST><<<grid, block, 0, s->stream>>>(s->g, s->ub, d, o, s->staging, state,
        s->mask,
        (float)(s->precision == LBM_F16 ? s->fp16_scale : 1.0), weight(d));
    CUDA_TRY(cudaGetLastError());
  }
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

template <class ST> static int unpack_all(lbm_solver *s, double *f)
{
  dim3 grid, block;
  user_launch_shape(s, grid, block);
  const int o = orientation(s);
  const size_t plane_host = (size_t)s->nx * s->ny * s->nz;
  using Sx = typename ST::S;
  const Sx *state = (const Sx *)state_ptr(s);
  for (int d = 0; d < Q; ++d) {
    unpack_plane_kernel<ST><<<grid, block, 0, s->stream>>>(s->g, s->ub, d, o, s->staging, state,
        s->mask, (float)(s->precision == LBM_F16 ? 1.0 / s->fp16_scale : 1.0), weight(d));
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(f + d * plane_host, s->staging, sizeof(double) * plane_host,
        cudaMemcpyDeviceToHost, s->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

extern "C" int lbm_set_state(lbm_solver *s, const double *f)
{
  if (!s || !f)
    return fail(LBM_ERR_ARG, "lbm_set_state: NULL argument");
  if (s->split)
    return fail(LBM_ERR_STATE, "lbm_set_state: a split step is open");
  CUDA_TRY(cudaSetDevice(s->device));
  switch (s->precision) {
  case LBM_F64: return pack_all<StoreF64>(s, f);
  case LBM_F32: return pack_all<StoreF32>(s, f);
  default: return pack_all<StoreF16>(s, f);
  }
}

extern "C" int lbm_get_state(lbm_solver *s, double *f)
{
  if (!s || !f)
    return fail(LBM_ERR_ARG, "lbm_get_state: NULL argument");
  if (s->split)
    return fail(LBM_ERR_STATE, "lbm_get_state: a split step is open");
  CUDA_TRY(cudaSetDevice(s->device));
  switch (s->precision) {
  case LBM_F64: return unpack_all<StoreF64>(s, f);
  case LBM_F32: return unpack_all<StoreF32>(s, f);
  default: return unpack_all<StoreF16>(s, f);
  }
}

// ---------------------------------------------------------------------------
// Checkpoint / resume of a solver's state on the host
// ---------------------------------------------------------------------------

// File: this header, then the state as lbm_get_state returns it (FP64,
// f[d][x][y][z], little-endian). Decoding FP32/FP16 storage to FP64 and
// encoding it again are exact, so a solver of the same precision (and FP16
// scale) that loads the file continues bit for bit.
struct StateFileHeader {
  char magic[8];        // "LBMB200S"
  uint32_t version;     // 1
  int32_t nx, ny, nz;
  int32_t pattern, precision;
  int64_t steps_done;   // sets the orientation the state continues from
  int64_t fluid_cells;  // must match the loading solver's geometry
  double fp16_scale;
};
static const char kStateMagic[8] = { 'L', 'B', 'M', 'B', '2', '0', '0', 'S' };

extern "C" int lbm_save_state(lbm_solver *s, const char *path)
{
  if (!s || !path)
    return fail(LBM_ERR_ARG, "lbm_save_state: NULL argument");
  std::vector<double> f;
  try {
    f.resize((size_t)Q * s->nx * s->ny * s->nz);
  } catch (...) {
    return fail(LBM_ERR_ALLOC, "lbm_save_state: host allocation failed");
  }
  int rc = lbm_get_state(s, f.data());
  if (rc)
    return rc;
  StateFileHeader h;
  memset(&h, 0, sizeof(h));
  memcpy(h.magic, kStateMagic, 8);
  h.version = 1;
  h.nx = s->nx;
  h.ny = s->ny;
  h.nz = s->nz;
  h.pattern = s->pattern;
  h.precision = s->precision;
  h.steps_done = s->steps_done;
  h.fluid_cells = s->n_fluid;
  h.fp16_scale = s->fp16_scale;
  FILE *fp = fopen(path, "wb");
  if (!fp)
    return fail(LBM_ERR_ARG, "lbm_save_state: cannot open %s for writing", path);
  const bool ok = fwrite(&h, sizeof(h), 1, fp) == 1 && fwrite(f.data(), sizeof(double), f.size(),
      fp) == f.size();
  if (fclose(fp) != 0 || !ok)
    return fail(LBM_ERR_ARG, "lbm_save_state: writing %s failed", path);
  return LBM_OK;
}

extern "C" int lbm_load_state(lbm_solver *s, const char *path)
{
  if (!s || !path)
    return fail(LBM_ERR_ARG, "lbm_load_state: NULL argument");
  if (s->split)
    return fail(LBM_ERR_STATE, "lbm_load_state: a split step is open");
  FILE *fp = fopen(path, "rb");
  if (!fp)
    return fail(LBM_ERR_ARG, "lbm_load_state: cannot open %s", path);
  StateFileHeader h;
  if (fread(&h, sizeof(h), 1, fp) != 1 || memcmp(h.magic, kStateMagic, 8) != 0 ||
      h.version != 1) {
    fclose(fp);
    return fail(LBM_ERR_ARG, "lbm_load_state: %s is not a liblbmb200 state file", path);
  }
  if (h.nx != s->nx || h.ny != s->ny || h.nz != s->nz || h.fluid_cells != s->n_fluid ||
      h.pattern != s->pattern || h.steps_done < 0) {
    fclose(fp);
    return fail(LBM_ERR_ARG, "lbm_load_state: %s holds a %dx%dx%d state with %lld fluid cells "
        "of pattern %d; the solver is %dx%dx%d with %lld fluid cells, pattern %d", path, h.nx,
        h.ny, h.nz, (long long)h.fluid_cells, h.pattern, s->nx, s->ny, s->nz, s->n_fluid,
        s->pattern);
  }
  std::vector<double> f;
  try {
    f.resize((size_t)Q * s->nx * s->ny * s->nz);
  } catch (...) {
    fclose(fp);
    return fail(LBM_ERR_ALLOC, "lbm_load_state: host allocation failed");
  }
  const bool ok = fread(f.data(), sizeof(double), f.size(), fp) == f.size();
  fclose(fp);
  if (!ok)
    return fail(LBM_ERR_ARG, "lbm_load_state: %s is truncated", path);
  // the step count fixes the AA orientation the state is written in
  const long long saved = s->steps_done;
  s->steps_done = h.steps_done;
  int rc = lbm_set_state(s, f.data());
  if (rc)
    s->steps_done = saved;
  return rc;
}

// ---------------------------------------------------------------------------
// Transfers in the reference's own padded layout (for the drop-in kernels)
// ---------------------------------------------------------------------------

// Slot of f_d(x) in the reference's padded SoA array, relative to one
// direction plane (indexSoA, src/lbm.h:113-116, ghost offset 1): push and
// AA odd/initial states keep f_d(x) at (x, d), pull at (x - c_d, d), AA
// after an even iteration at (x - c_d, inv d) (src/lbm.c:193-294). For a
// padded plane p the kernel handles direction d = p, or inv p in the AA
// even orientation.
__device__ __forceinline__ long long ref_index(int rx, int ry, int rz, int ref_orient, int d,
    int x, int y, int z)
{
  int a = x + 1, b = y + 1, c = z + 1;
  if (ref_orient != LBM_REF_NATURAL) {
    a -= cx(d);
    b -= cy(d);
    c -= cz(d);
  }
  return ((long long)a * ry + b) * rz + c;
}

template <class ST, typename H>
__global__ void pack_ref_kernel(Grid g, UserBox u, int p, int ref_orient, int orient,
    const H *__restrict__ plane, typename ST::S *state, const uint32_t *__restrict__ mask,
    float scale)
{
  using V = typename ST::V;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= u.nz || y >= u.ny)
    return;
  uint32_t cell, m;
  if (!locate(g, mask, x + u.ox, y + u.oy, z + u.oz, cell, m))
    return;
  const int d = (ref_orient == LBM_REF_AA_EVEN) ? inv(p) : p;
  const Nbr nb = make_nbr(g, x + u.ox, y + u.oy, z + u.oz, cell);
  int sp;
  uint32_t sc;
  state_slot(orient, d, m, cell, nb, sp, sc);
  double v = (double)plane[ref_index(u.nx + 2, u.ny + 2, u.nz + 2, ref_orient, d, x, y, z)];
  if (ST::kShifted) {
    const int wc = wclass(d);
    v -= wc == 0 ? 1.0 / 3.0 : wc == 1 ? 1.0 / 18.0 : 1.0 / 36.0;
  }
  ST::store(state + (long long)sp * g.plane + sc, (V)v, (V)scale);
}

template <class ST, typename H>
__global__ void unpack_ref_kernel(Grid g, UserBox u, int p, int ref_orient, int orient,
    H *__restrict__ plane, const typename ST::S *state, const uint32_t *__restrict__ mask,
    float inv_scale)
{
  using V = typename ST::V;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= u.nz || y >= u.ny)
    return;
  uint32_t cell, m;
  if (!locate(g, mask, x + u.ox, y + u.oy, z + u.oz, cell, m))
    return;
  const int d = (ref_orient == LBM_REF_AA_EVEN) ? inv(p) : p;
  const Nbr nb = make_nbr(g, x + u.ox, y + u.oy, z + u.oz, cell);
  int sp;
  uint32_t sc;
  state_slot(orient, d, m, cell, nb, sp, sc);
  double v = (double)ST::load(state + (long long)sp * g.plane + sc, d, (V)inv_scale);
  if (ST::kShifted) {
    const int wc = wclass(d);
    v += wc == 0 ? 1.0 / 3.0 : wc == 1 ? 1.0 / 18.0 : 1.0 / 36.0;
  }
  plane[ref_index(u.nx + 2, u.ny + 2, u.nz + 2, ref_orient, d, x, y, z)] = (H)v;
}

// The same transfer for the reference's AoS array (indexAoS,
// src/lbm.h:118-121): padded x-planes [a0, a0 + gridDim.z) of it sit in
// `chunk`, and each thread takes the 19 contiguous slots of one padded cell.
// A slot maps back to the fluid cell whose population it holds (the inverse
// of ref_index); on download slots that hold none are written as 0.
template <class ST, typename H, bool UP>
__global__ void aos_ref_kernel(Grid g, UserBox u, int a0, int ref_orient, int orient,
    H *__restrict__ chunk, typename ST::S *state, const uint32_t *__restrict__ mask, float scale)
{
  using V = typename ST::V;
  const int rz = u.nz + 2, ry = u.ny + 2;
  const int c = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y * blockDim.y + threadIdx.y;
  const int a = a0 + (int)blockIdx.z;
  if (c >= rz || b >= ry)
    return;
  H *slots = chunk + (((long long)blockIdx.z * ry + b) * rz + c) * Q;
#pragma unroll 1
  for (int p = 0; p < Q; ++p) {
    const int d = (ref_orient == LBM_REF_AA_EVEN) ? inv(p) : p;
    int x = a - 1, y = b - 1, z = c - 1;
    if (ref_orient != LBM_REF_NATURAL) {
      x += cx(d);
      y += cy(d);
      z += cz(d);
    }
    bool own = x >= 0 && x < u.nx && y >= 0 && y < u.ny && z >= 0 && z < u.nz;
    uint32_t cell = 0, m = kSolidBit;
    if (own)
      own = locate(g, mask, x + u.ox, y + u.oy, z + u.oz, cell, m);
    if (!own) {
      if (!UP)
        slots[p] = (H)0;
      continue;
    }
    const Nbr nb = make_nbr(g, x + u.ox, y + u.oy, z + u.oz, cell);
    int sp;
    uint32_t sc;
    state_slot(orient, d, m, cell, nb, sp, sc);
    const int wc = wclass(d);
    const double w = wc == 0 ? 1.0 / 3.0 : wc == 1 ? 1.0 / 18.0 : 1.0 / 36.0;
    if (UP) {
      double v = (double)slots[p];
      if (ST::kShifted)
        v -= w;
      ST::store(state + (long long)sp * g.plane + sc, (V)v, (V)scale);
    } else {
      double v = (double)ST::load(state + (long long)sp * g.plane + sc, d, (V)scale);
      if (ST::kShifted)
        v += w;
      slots[p] = (H)v;
    }
  }
}

template <class ST, typename H>
static int ref_transfer_aos(lbm_solver *s, void *host, int ref_orient, bool upload)
{
  const int ra = s->nx + 2, ry = s->ny + 2, rz = s->nz + 2;
  const size_t xplane = (size_t)ry * rz * Q; // values of one padded x-plane
  // as many x-planes per chunk as fit the staging of one SoA direction plane
  const size_t gpl = (size_t)ra * ry * rz;
  const int per = (int)(gpl / xplane) > 0 ? (int)(gpl / xplane) : 1;
  const size_t bytes = (size_t)per * xplane * sizeof(H);
  if (s->pstaging_bytes < bytes) {
    cudaFree(s->pstaging);
    s->pstaging = NULL;
    s->pstaging_bytes = 0;
    int rc = dev_alloc(s, &s->pstaging, bytes, "the padded transfer plane");
    if (rc)
      return rc;
    s->pstaging_bytes = bytes;
  }
  const int o = orientation(s);
  const float sc = (float)(s->precision == LBM_F16 ? s->fp16_scale : 1.0);
  using Sx = typename ST::S;
  H *hp = (H *)host;
  H *dp = (H *)s->pstaging;
  const dim3 block(32, 8, 1);
  for (int a0 = 0; a0 < ra; a0 += per) {
    const int n = ra - a0 < per ? ra - a0 : per;
    const dim3 grid((rz + 31) / 32, (ry + 7) / 8, n);
    const size_t nbytes = (size_t)n * xplane * sizeof(H);
    H *hc = hp + (size_t)a0 * xplane;
    if (upload) {
      CUDA_TRY(cudaMemcpyAsync(dp, hc, nbytes, cudaMemcpyHostToDevice, s->stream));
      aos_ref_kernel<ST, H, true><<<grid, block, 0, s->stream>>>(s->g, s->ub, a0, ref_orient, o,
          dp, (Sx *)state_ptr(s), s->mask, sc);
      CUDA_TRY(cudaGetLastError());
    } else {
      aos_ref_kernel<ST, H, false><<<grid, block, 0, s->stream>>>(s->g, s->ub, a0, ref_orient,
          o, dp, (Sx *)state_ptr(s), s->mask, 1.0f / sc);
      CUDA_TRY(cudaGetLastError());
      CUDA_TRY(cudaMemcpyAsync(hc, dp, nbytes, cudaMemcpyDeviceToHost, s->stream));
    }
  }
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

template <class ST, typename H>
static int ref_transfer(lbm_solver *s, void *host, int ref_orient, bool upload)
{
  if (ref_orient & LBM_REF_AOS)
    return ref_transfer_aos<ST, H>(s, host, ref_orient & ~LBM_REF_AOS, upload);
  const size_t gpl = (size_t)(s->nx + 2) * (s->ny + 2) * (s->nz + 2);
  const size_t bytes = gpl * sizeof(H);
  if (s->pstaging_bytes < bytes) {
    cudaFree(s->pstaging);
    s->pstaging = NULL;
    s->pstaging_bytes = 0;
    int rc = dev_alloc(s, &s->pstaging, bytes, "the padded transfer plane");
    if (rc)
      return rc;
    s->pstaging_bytes = bytes;
  }
  dim3 grid, block;
  user_launch_shape(s, grid, block);
  const int o = orientation(s);
  const float sc = (float)(s->precision == LBM_F16 ? s->fp16_scale : 1.0);
  using Sx = typename ST::S;
  H *hp = (H *)host;
  H *dp = (H *)s->pstaging;
  for (int p = 0; p < Q; ++p) {
    if (upload) {
      CUDA_TRY(cudaMemcpyAsync(dp, hp + p * gpl, bytes, cudaMemcpyHostToDevice, s->stream));
      pack_ref_kernel<ST, H><<<grid, block, 0, s->stream>>>(s->g, s->ub, p, ref_orient, o, dp,
          (Sx *)state_ptr(s), s->mask, sc);
      CUDA_TRY(cudaGetLastError());
    } else {
      // slots that hold no fluid population come back as 0
      CUDA_TRY(cudaMemsetAsync(dp, 0, bytes, s->stream));
      unpack_ref_kernel<ST, H><<<grid, block, 0, s->stream>>>(s->g, s->ub, p, ref_orient, o, dp,
          (const Sx *)state_ptr(s), s->mask, 1.0f / sc);
      CUDA_TRY(cudaGetLastError());
      CUDA_TRY(cudaMemcpyAsync(hp + p * gpl, dp, bytes, cudaMemcpyDeviceToHost, s->stream));
    }
  }
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

static int ref_dispatch(lbm_solver *s, void *host, int elem_size, int ref_orient, bool upload)
{
  const int o = ref_orient & ~LBM_REF_AOS;
  if (!s || !host || (elem_size != 8 && elem_size != 4) || o < LBM_REF_NATURAL ||
      o > LBM_REF_AA_EVEN)
    return fail(LBM_ERR_ARG, "padded transfer: bad arguments");
  if (s->split)
    return fail(LBM_ERR_STATE, "padded transfer: a split step is open");
  CUDA_TRY(cudaSetDevice(s->device));
  if (elem_size == 8) {
    if (s->precision == LBM_F64)
      return ref_transfer<StoreF64, double>(s, host, ref_orient, upload);
    if (s->precision == LBM_F32)
      return ref_transfer<StoreF32, double>(s, host, ref_orient, upload);
    return ref_transfer<StoreF16, double>(s, host, ref_orient, upload);
  }
  if (s->precision == LBM_F64)
    return ref_transfer<StoreF64, float>(s, host, ref_orient, upload);
  if (s->precision == LBM_F32)
    return ref_transfer<StoreF32, float>(s, host, ref_orient, upload);
  return ref_transfer<StoreF16, float>(s, host, ref_orient, upload);
}

extern "C" int lbm_set_state_padded(lbm_solver *s, const void *pdfs, int elem_size,
    int ref_orientation)
{
  return ref_dispatch(s, const_cast<void *>(pdfs), elem_size, ref_orientation, true);
}

extern "C" int lbm_get_state_padded(lbm_solver *s, void *pdfs, int elem_size,
    int ref_orientation)
{
  return ref_dispatch(s, pdfs, elem_size, ref_orientation, false);
}

// Launches the step kernel of the next step over device x planes
// [x0, x0 + planes) on stream st, without advancing the bookkeeping. The
// pipelined FP64 kernels only serve whole steps.
static int launch_kernel(lbm_solver *s, int x0, int planes, cudaStream_t st, int *kind_out)
{
  dim3 grid, block;
  cell_launch_shape(s->g, grid, block);
  grid.z = planes;
  const bool whole = x0 == 0 && planes == s->g.nx;
  int kind;
  const void *src;
  void *dst;
  if (s->pattern == LBM_AA) {
    kind = (s->steps_done & 1) ? kAAOddStep : kAAEvenStep;
    src = dst = s->buf[0];
  } else {
    kind = s->pattern == LBM_PULL ? kPullStep : kPushStep;
    src = s->buf[s->cur];
    dst = s->buf[s->cur ^ 1];
  }
  const bool brink = s->alpha != 0.0 && s->porosity;
  const bool force = s->force_on || brink;
  cudaError_t e;
  if (s->compact) {
    // compact layout: one cell per thread in every precision (no Brinkman term)
    if (s->precision == LBM_F64) {
      StepArgs<StoreF64> a;
      a.g = s->g;
      a.src = (const double *)src;
      a.dst = (double *)dst;
      a.mask = s->mask;
      a.porosity = nullptr;
      a.u_save = nullptr;
      a.c = make_consts<double>(s);
      a.x0 = x0;
      a.c0 = (*s->cplane0)[x0];
      a.cn = (*s->cplane0)[x0 + planes] - a.c0;
      e = launch_step_cp_f64(kind, force, a, grid, block, st);
    } else {
      // FP32 / FP16 storage: pair arithmetic, bit-identical to the dense layout
      StepArgs2<StoreF32> a32;
      StepArgs2<StoreF16> a16;
      auto fill = [&](auto &a) {
        a.g = s->g;
        a.mask = s->mask;
        a.porosity = nullptr;
        a.u_save = nullptr;
        a.c = make_consts2(s);
        a.no_shuffle = s->no_shuffle;
        a.no_quad = s->no_quad;
        a.x0 = x0;
        a.planes = planes;
        a.c0 = (*s->cplane0)[x0];
        a.cn = (*s->cplane0)[x0 + planes] - a.c0;
      };
      if (s->precision == LBM_F32) {
        fill(a32);
        a32.src = (const float *)src;
        a32.dst = (float *)dst;
        e = launch_step_cp2_f32(kind, force, a32, st);
      } else {
        fill(a16);
        a16.src = (const __half *)src;
        a16.dst = (__half *)dst;
        e = launch_step_cp2_f16(kind, force, a16, st);
      }
    }
  } else if (s->precision == LBM_F64) {
    StepArgs<StoreF64> a;
    a.g = s->g;
    a.src = (const double *)src;
    a.dst = (double *)dst;
    a.mask = s->mask;
    a.porosity = s->porosity;
    a.u_save = brink ? (double *)s->u_save_next : nullptr;
    a.c = make_consts<double>(s);
    a.x0 = x0;
    if (s->tma && !brink && whole) {
      TmaArgs<StoreF64> t;
      t.s = a;
      t.T = s->tma_shape.T;
      t.stages = s->tma_shape.stages;
      t.ytiles = s->tma_shape.ytiles;
      t.ntiles = s->tma_shape.ntiles;
      t.stage_bytes = s->tma_shape.stage_bytes;
      t.err = s->dev_err;
      e = launch_step_tma_f64(kind, force, t, s->tma_groups, s->tma_shape.blocks, st);
    } else {
      e = launch_step_f64(kind, force, brink, a, grid, block, st);
    }
  } else if (s->precision == LBM_F32) {
    StepArgs2<StoreF32> a;
    a.g = s->g;
    a.src = (const float *)src;
    a.dst = (float *)dst;
    a.mask = s->mask;
    a.porosity = s->porosity;
    a.u_save = brink ? (float *)s->u_save_next : nullptr;
    a.c = make_consts2(s);
    a.no_shuffle = s->no_shuffle;
    a.no_quad = s->no_quad;
    a.x0 = x0;
    a.planes = planes;
    e = launch_step_x2_f32(kind, force, brink, a, st);
  } else {
    StepArgs2<StoreF16> a;
    a.g = s->g;
    a.src = (const __half *)src;
    a.dst = (__half *)dst;
    a.mask = s->mask;
    a.porosity = s->porosity;
    a.u_save = nullptr;
    a.c = make_consts2(s);
    a.no_shuffle = s->no_shuffle;
    a.no_quad = s->no_quad;
    a.x0 = x0;
    a.planes = planes;
    e = launch_step_x2_f16(kind, force, brink, a, st);
  }
  if (e != cudaSuccess)
    return fail(LBM_ERR_CUDA, "step launch failed: %s", cudaGetErrorString(e));
  s->launches++;
  if (kind_out)
    *kind_out = kind;
  return LBM_OK;
}

// After all planes of a step: the lattice swap and step count, then the
// pressure boundary of the new state.
static int finish_step(lbm_solver *s)
{
  if (s->pattern != LBM_AA)
    s->cur ^= 1;
  s->steps_done++;
  if (s->bc_on) {
    cudaError_t e;
    e = launch_pressure_bc(s->precision, s->g, s->ub, orientation(s), (void *)state_ptr(s),
        s->mask, s->bc_marks, s->rho_in, s->rho_out,
        (float)(s->precision == LBM_F16 ? s->fp16_scale : 1.0), s->stream);
    if (e != cudaSuccess)
      return fail(LBM_ERR_CUDA, "pressure boundary launch failed: %s", cudaGetErrorString(e));
  }
  return LBM_OK;
}

// Launches one whole step and advances the bookkeeping.
static int launch_one(lbm_solver *s, int *kind_out)
{
  if (s->split)
    return fail(LBM_ERR_STATE, "a split step is open (lbm_step_begin without lbm_step_end)");
  // the compact layout stores the fluid cells of a slab's ghost planes too
  // (they are read and written by the boundary planes' steps), and its
  // kernels select cells by their fluid bit: launch the own planes only
  const int gx = (s->compact && s->slab) ? 1 : 0;
  int rc = launch_kernel(s, gx, s->g.nx - 2 * gx, s->stream, kind_out);
  return rc ? rc : finish_step(s);
}

extern "C" int lbm_step_begin(lbm_solver *s)
{
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_step_begin: NULL solver");
  if (s->split)
    return fail(LBM_ERR_STATE, "lbm_step_begin: a split step is already open");
  CUDA_TRY(cudaSetDevice(s->device));
  if (!s->side) {
    int least = 0, greatest = 0;
    CUDA_TRY(cudaDeviceGetStreamPriorityRange(&least, &greatest));
    CUDA_TRY(cudaStreamCreateWithPriority(&s->side, cudaStreamNonBlocking, least));
    CUDA_TRY(cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming));
    CUDA_TRY(cudaEventCreateWithFlags(&s->join_ev, cudaEventDisableTiming));
  }
  if (!s->split_done) {
    s->split_done = (uint8_t *)malloc((size_t)s->nx);
    if (!s->split_done)
      return fail(LBM_ERR_ALLOC, "lbm_step_begin: host allocation failed");
  }
  memset(s->split_done, 0, (size_t)s->nx);
  s->split_left = s->nx;
  // the side stream starts after everything queued on the solver's stream
  CUDA_TRY(cudaEventRecord(s->fork_ev, s->stream));
  CUDA_TRY(cudaStreamWaitEvent(s->side, s->fork_ev, 0));
  s->split = 1;
  return LBM_OK;
}

extern "C" int lbm_step_planes(lbm_solver *s, int x_begin, int x_end, int on_side)
{
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_step_planes: NULL solver");
  if (!s->split)
    return fail(LBM_ERR_STATE, "lbm_step_planes: no split step open (lbm_step_begin)");
  if (x_begin < 0 || x_end > s->nx || x_begin >= x_end)
    return fail(LBM_ERR_ARG, "lbm_step_planes: planes [%d, %d) outside [0, %d)", x_begin, x_end,
        s->nx);
  for (int x = x_begin; x < x_end; ++x)
    if (s->split_done[x])
      return fail(LBM_ERR_ARG, "lbm_step_planes: plane %d already updated in this step", x);
  CUDA_TRY(cudaSetDevice(s->device));
  int rc = launch_kernel(s, x_begin + s->ub.ox, x_end - x_begin, on_side ? s->side : s->stream,
      NULL);
  if (rc)
    return rc;
  memset(s->split_done + x_begin, 1, (size_t)(x_end - x_begin));
  s->split_left -= x_end - x_begin;
  return LBM_OK;
}

extern "C" int lbm_step_end(lbm_solver *s)
{
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_step_end: NULL solver");
  if (!s->split)
    return fail(LBM_ERR_STATE, "lbm_step_end: no split step open (lbm_step_begin)");
  if (s->split_left) {
    int x = 0;
    while (x < s->nx && s->split_done[x])
      ++x;
    return fail(LBM_ERR_STATE, "lbm_step_end: %d plane(s) not updated, the first is %d",
        s->split_left, x);
  }
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaEventRecord(s->join_ev, s->side));
  CUDA_TRY(cudaStreamWaitEvent(s->stream, s->join_ev, 0));
  s->split = 0;
  return finish_step(s);
}

extern "C" int lbm_set_pressure_bc(lbm_solver *s, double rho_in, double rho_out, int on)
{
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_set_pressure_bc: NULL solver");
  if (!on) {
    s->bc_on = 0;
    return LBM_OK;
  }
  if (!(rho_in > 0.0) || !(rho_out > 0.0) || !isfinite(rho_in) || !isfinite(rho_out))
    return fail(LBM_ERR_ARG, "lbm_set_pressure_bc: densities %g, %g must be positive", rho_in,
        rho_out);
  if (!s->bc_marks)
    return fail(LBM_ERR_STATE, "lbm_set_pressure_bc: the flags have no inlet (2) cells on x = 0 "
        "or outlet (4) cells on x = nx-1 inside the y/z walls");
  s->rho_in = rho_in;
  s->rho_out = rho_out;
  s->bc_on = 1;
  return LBM_OK;
}

extern "C" int lbm_run(lbm_solver *s, int steps)
{
  if (!s || steps < 0)
    return fail(LBM_ERR_ARG, "lbm_run: bad arguments");
  CUDA_TRY(cudaSetDevice(s->device));
  for (int i = 0; i < steps; ++i) {
    int rc = launch_one(s, NULL);
    if (rc)
      return rc;
  }
  return LBM_OK;
}

// Reads the kernels' error word after the stream has drained.
static int check_kernel_error(lbm_solver *s)
{
  unsigned int err = 0;
  CUDA_TRY(cudaMemcpy(&err, s->dev_err, sizeof(err), cudaMemcpyDeviceToHost));
  if (err) {
    CUDA_TRY(cudaMemset(s->dev_err, 0, sizeof(err)));
    return fail(LBM_ERR_CUDA, "a pipelined step kernel gave up waiting for its bulk copies; "
        "the state is undefined");
  }
  return LBM_OK;
}

extern "C" int lbm_synchronize(lbm_solver *s)
{
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_synchronize: NULL solver");
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  if (s->side)
    CUDA_TRY(cudaStreamSynchronize(s->side));
  return check_kernel_error(s);
}

extern "C" int lbm_run_timed(lbm_solver *s, int steps, double *ms)
{
  if (!s || steps < 0 || !ms)
    return fail(LBM_ERR_ARG, "lbm_run_timed: bad arguments");
  CUDA_TRY(cudaSetDevice(s->device));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  CUDA_TRY(cudaEventRecord(s->ev[0], s->stream));
  int rc = lbm_run(s, steps);
  if (rc)
    return rc;
  CUDA_TRY(cudaEventRecord(s->ev[1], s->stream));
  CUDA_TRY(cudaEventSynchronize(s->ev[1]));
  float t = 0.f;
  CUDA_TRY(cudaEventElapsedTime(&t, s->ev[0], s->ev[1]));
  *ms = t;
  return check_kernel_error(s);
}

extern "C" int lbm_time_launches(lbm_solver *s, int steps, double *ms_sum, int *count,
    double *region_ms)
{
  if (!s || steps < 0 || !ms_sum || !count)
    return fail(LBM_ERR_ARG, "lbm_time_launches: bad arguments");
  CUDA_TRY(cudaSetDevice(s->device));
  for (int k = 0; k < 4; ++k) {
    ms_sum[k] = 0.0;
    count[k] = 0;
  }
  std::vector<cudaEvent_t> ev(2 * (size_t)steps);
  std::vector<int> kinds((size_t)steps);
  for (auto &e : ev)
    CUDA_TRY(cudaEventCreate(&e));
  int rc = LBM_OK;
  for (int i = 0; i < steps && !rc; ++i) {
    cudaEventRecord(ev[2 * i], s->stream);
    rc = launch_one(s, &kinds[i]);
    cudaEventRecord(ev[2 * i + 1], s->stream);
  }
  cudaError_t e = cudaStreamSynchronize(s->stream);
  for (int i = 0; i < steps && !rc && e == cudaSuccess; ++i) {
    float t = 0.f;
    e = cudaEventElapsedTime(&t, ev[2 * i], ev[2 * i + 1]);
    ms_sum[kinds[i]] += t;
    count[kinds[i]] += 1;
  }
  if (region_ms) {
    float t = 0.f;
    if (steps > 0 && !rc && e == cudaSuccess)
      e = cudaEventElapsedTime(&t, ev[0], ev[2 * (size_t)steps - 1]);
    *region_ms = t;
  }
  for (auto &x : ev)
    cudaEventDestroy(x);
  if (rc)
    return rc;
  if (e != cudaSuccess)
    return fail(LBM_ERR_CUDA, "lbm_time_launches: %s", cudaGetErrorString(e));
  return check_kernel_error(s);
}

template <class ST> static int moments_t(lbm_solver *s, double *q[4])
{
  dim3 grid, block;
  user_launch_shape(s, grid, block);
  const size_t n = (size_t)s->nx * s->ny * s->nz;
  const float inv = (float)(s->precision == LBM_F16 ? 1.0 / s->fp16_scale : 1.0);
  for (int k = 0; k < 4; ++k) {
    if (!q[k])
      continue;
    moments_kernel<ST><<<grid, block, 0, s->stream>>>(s->g, s->ub, orientation(s), k,
        (const typename ST::S *)state_ptr(s), s->mask, inv, s->staging);
    CUDA_TRY(cudaGetLastError());
    CUDA_TRY(cudaMemcpyAsync(q[k], s->staging, sizeof(double) * n, cudaMemcpyDeviceToHost,
        s->stream));
  }
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

extern "C" int lbm_moments(lbm_solver *s, double *rho, double *ux, double *uy, double *uz)
{
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_moments: NULL solver");
  CUDA_TRY(cudaSetDevice(s->device));
  double *q[4] = { rho, ux, uy, uz };
  switch (s->precision) {
  case LBM_F64: return moments_t<StoreF64>(s, q);
  case LBM_F32: return moments_t<StoreF32>(s, q);
  default: return moments_t<StoreF16>(s, q);
  }
}

template <class ST> static void mass_launch(lbm_solver *s, double *partial)
{
  const float inv = (float)(s->precision == LBM_F16 ? 1.0 / s->fp16_scale : 1.0);
  mass_kernel<ST><<<kRedBlocks, kRedThreads, 0, s->stream>>>(s->g, orientation(s),
      (const typename ST::S *)state_ptr(s), s->mask, inv, partial);
}

extern "C" int lbm_mass_momentum(lbm_solver *s, double out[4], long long *nonfinite)
{
  if (!s || !out)
    return fail(LBM_ERR_ARG, "lbm_mass_momentum: NULL argument");
  CUDA_TRY(cudaSetDevice(s->device));
  if (s->precision == LBM_F64)
    mass_launch<StoreF64>(s, s->red);
  else if (s->precision == LBM_F32)
    mass_launch<StoreF32>(s, s->red);
  else
    mass_launch<StoreF16>(s, s->red);
  CUDA_TRY(cudaGetLastError());
  double *fin = s->red + (size_t)kRedBlocks * kRedVals;
  final_reduce_kernel<<<1, kRedThreads, 0, s->stream>>>(s->red, kRedBlocks, 0u, fin);
  CUDA_TRY(cudaGetLastError());
  double h[kRedVals];
  CUDA_TRY(cudaMemcpyAsync(h, fin, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  for (int k = 0; k < 4; ++k)
    out[k] = h[k];
  long long bad = (long long)h[4];
  if (nonfinite)
    *nonfinite = bad;
  if (bad)
    return fail(LBM_ERR_NONFINITE, "state holds NaN/Inf in %lld fluid cells", bad);
  return LBM_OK;
}

template <class SA, class SB> static void compare_launch(lbm_solver *a, lbm_solver *b)
{
  const float ia = (float)(a->precision == LBM_F16 ? 1.0 / a->fp16_scale : 1.0);
  const float ib = (float)(b->precision == LBM_F16 ? 1.0 / b->fp16_scale : 1.0);
  compare_kernel<SA, SB><<<kRedBlocks, kRedThreads, 0, a->stream>>>(a->g, b->g,
      orientation(a), orientation(b), (const typename SA::S *)state_ptr(a),
      (const typename SB::S *)state_ptr(b), a->mask, b->mask, ia, ib, a->red);
}

template <class SA> static void compare_b(lbm_solver *a, lbm_solver *b)
{
  if (b->precision == LBM_F64)
    compare_launch<SA, StoreF64>(a, b);
  else if (b->precision == LBM_F32)
    compare_launch<SA, StoreF32>(a, b);
  else
    compare_launch<SA, StoreF16>(a, b);
}

extern "C" int lbm_compare(lbm_solver *a, lbm_solver *b, double out[6])
{
  if (!a || !b || !out)
    return fail(LBM_ERR_ARG, "lbm_compare: NULL argument");
  if (a->nx != b->nx || a->ny != b->ny || a->nz != b->nz || a->device != b->device ||
      a->g.nx != b->g.nx || a->g.ny != b->g.ny || a->g.nz != b->g.nz || a->ub.ox != b->ub.ox ||
      a->ub.oy != b->ub.oy || a->ub.oz != b->ub.oz)
    return fail(LBM_ERR_ARG, "lbm_compare: solvers differ in geometry or device");
  CUDA_TRY(cudaSetDevice(a->device));
  CUDA_TRY(cudaStreamSynchronize(b->stream));
  if (a->precision == LBM_F64)
    compare_b<StoreF64>(a, b);
  else if (a->precision == LBM_F32)
    compare_b<StoreF32>(a, b);
  else
    compare_b<StoreF16>(a, b);
  CUDA_TRY(cudaGetLastError());
  double *fin = a->red + (size_t)kRedBlocks * kRedVals;
  final_reduce_kernel<<<1, kRedThreads, 0, a->stream>>>(a->red, kRedBlocks, 0x30u, fin);
  CUDA_TRY(cudaGetLastError());
  double h[kRedVals];
  CUDA_TRY(cudaMemcpyAsync(h, fin, sizeof(h), cudaMemcpyDeviceToHost, a->stream));
  CUDA_TRY(cudaStreamSynchronize(a->stream));
  for (int k = 0; k < 6; ++k)
    out[k] = h[k];
  return LBM_OK;
}

template <class ST> static void outlet_launch(lbm_solver *s)
{
  const float inv = (float)(s->precision == LBM_F16 ? 1.0 / s->fp16_scale : 1.0);
  outlet_kernel<ST><<<kRedBlocks, kRedThreads, 0, s->stream>>>(s->g,
      s->ub.ox + s->ub.nx - 1, orientation(s),
      (const typename ST::S *)state_ptr(s), s->mask, inv, s->red);
}

extern "C" int lbm_objective(lbm_solver *s, double *j)
{
  if (!s || !j)
    return fail(LBM_ERR_ARG, "lbm_objective: NULL argument");
  CUDA_TRY(cudaSetDevice(s->device));
  if (s->precision == LBM_F64)
    outlet_launch<StoreF64>(s);
  else if (s->precision == LBM_F32)
    outlet_launch<StoreF32>(s);
  else
    outlet_launch<StoreF16>(s);
  CUDA_TRY(cudaGetLastError());
  double *fin = s->red + (size_t)kRedBlocks * kRedVals;
  final_reduce_kernel<<<1, kRedThreads, 0, s->stream>>>(s->red, kRedBlocks, 0u, fin);
  CUDA_TRY(cudaGetLastError());
  double h[kRedVals];
  CUDA_TRY(cudaMemcpyAsync(h, fin, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  *j = h[1] > 0 ? h[0] / h[1] : 0.0;
  return LBM_OK;
}

// ---------------------------------------------------------------------------
// Halo exchange of x-slabs
// ---------------------------------------------------------------------------
//
// A slab's step reads or writes, across each x face, only the five
// populations with c_x = +1 (set P) or c_x = -1 (set M). Which slots of
// which plane move, per propagation pattern:
//   before a pull step   own last plane P -> right ghost, own first plane M -> left ghost
//   before an AA odd step own last plane M -> right ghost, own first plane P -> left ghost
//   after a push or AA odd step  right ghost P -> own first plane of the
//                                right slab, left ghost M -> own last plane of the left slab,
//                                only into slots that arrived over a fluid link
// (pull gathers slot d of x - c_d; the AA odd step reads slot inv d of
// x - c_d and writes slot d of x + c_d; push writes slot d of x + c_d.)
// AA even steps and push's reads are local. A message is 5 slots x ny x nz
// storage elements in the caller's y-z order.
//
// The pull state and the AA state after an odd number of steps keep some
// populations of a boundary cell in the neighbouring cell (slot d of
// x - c_d, or slot inv d of x - c_d), i.e. in a ghost plane: exactly the
// before-step slot sets. So a before-step exchange also makes such a state
// readable (lbm_get_state, moments), and LBM_HALO_SCATTER sends what
// lbm_set_state wrote into the ghost planes to the neighbours' own planes.

// k-th direction (0..4) with c_x == sgn
__device__ __forceinline__ int halo_dir(int sgn, int k)
{
  int n = 0;
#pragma unroll
  for (int d = 0; d < Q; ++d)
    if (cx(d) == sgn) {
      if (n == k)
        return d;
      ++n;
    }
  return 0;
}

// to_buf: state -> message; else message -> state. guard (unpacks into own
// planes): slot d of a cell is written only if the cell is fluid and the
// link the slot's population uses is fluid - mask bit inv d (kGuardInv:
// the population arrived from x - c_d, after a push or AA odd step) or bit
// d (kGuardOwn: the pull state keeps x + c_d's population d there). Across a
// wall the cell itself keeps a bounced population in that slot, and the
// neighbour's ghost slot holds nothing.
enum HaloGuard { kGuardNone = 0, kGuardInv = 1, kGuardOwn = 2 };

template <typename T>
__global__ void halo_copy_kernel(Grid g, UserBox u, int xplane, int sgn, T *state, T *buf,
    int to_buf, const uint32_t *__restrict__ mask, int guarded)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z;
  if (z >= u.nz || y >= u.ny)
    return;
  const int d = halo_dir(sgn, k);
  const size_t bi = ((size_t)k * u.ny + y) * u.nz + z;
  uint32_t cell;
  if (g.wb) {
    // compact layout: only stored (fluid) cells take part; a solid cell
    // sends 0 and receives nothing
    const uint32_t wk = ((uint32_t)xplane * (uint32_t)g.ny + (uint32_t)(y + u.oy)) *
        (uint32_t)g.W + (uint32_t)((z + u.oz) >> 5);
    if (!((g.wb[wk].x >> ((z + u.oz) & 31)) & 1u)) {
      if (to_buf)
        buf[bi] = T(0);
      return;
    }
    cell = packed_index(g, xplane, y + u.oy, z + u.oz);
  } else {
    cell = cell_index(g, xplane, y + u.oy, z + u.oz);
  }
  const size_t si = (size_t)d * g.plane + cell;
  if (to_buf) {
    buf[bi] = state[si];
    return;
  }
  if (guarded && (mask[cell] & (kSolidBit | (1u << (guarded == kGuardInv ? inv(d) : d)))))
    return;
  state[si] = buf[bi];
}

// The lattice an exchange reads and writes: the state, except for an
// after-step exchange inside a split step of pull / push, whose messages are
// in the lattice the open step writes (the lattices swap at lbm_step_end).
static void *halo_lattice(const lbm_solver *s, int when)
{
  if (s->pattern == LBM_AA)
    return s->buf[0];
  return s->buf[s->cur ^ ((s->split && when == LBM_HALO_AFTER) ? 1 : 0)];
}

static int halo_copy(lbm_solver *s, void *st, int xplane, int sgn, void *buf, int to_buf,
    int guarded = 0)
{
  dim3 block(32, 8, 1);
  dim3 grid((s->ub.nz + 31) / 32, (s->ub.ny + 7) / 8, 5);
  switch (storage_size(s->precision)) {
  case 8:
    halo_copy_kernel<uint64_t><<<grid, block, 0, s->stream>>>(s->g, s->ub, xplane, sgn,
        (uint64_t *)st, (uint64_t *)buf, to_buf, s->mask, guarded);
    break;
  case 4:
    halo_copy_kernel<uint32_t><<<grid, block, 0, s->stream>>>(s->g, s->ub, xplane, sgn,
        (uint32_t *)st, (uint32_t *)buf, to_buf, s->mask, guarded);
    break;
  default:
    halo_copy_kernel<uint16_t><<<grid, block, 0, s->stream>>>(s->g, s->ub, xplane, sgn,
        (uint16_t *)st, (uint16_t *)buf, to_buf, s->mask, guarded);
  }
  CUDA_TRY(cudaGetLastError());
  return LBM_OK;
}

extern "C" size_t lbm_halo_bytes(const lbm_solver *s)
{
  if (!s || !s->slab)
    return 0;
  return (size_t)5 * s->ub.ny * s->ub.nz * storage_size(s->precision);
}

extern "C" int lbm_halo_shifted(const lbm_solver *s)
{
  return s && s->slab && orientation(s) != kNatural;
}

extern "C" int lbm_halo_needs(const lbm_solver *s)
{
  if (!s || !s->slab)
    return 0;
  if (s->pattern == LBM_PULL)
    return LBM_HALO_BEFORE;
  if (s->pattern == LBM_PUSH)
    return LBM_HALO_AFTER;
  return (s->steps_done & 1) ? (LBM_HALO_BEFORE | LBM_HALO_AFTER) : 0;
}

static int halo_check(const lbm_solver *s, int when, const void *a, const void *b,
    const char *fn)
{
  if (!s || !s->slab || !a || !b)
    return fail(LBM_ERR_ARG, "%s: needs a slab solver and two device buffers", fn);
  if (when != LBM_HALO_BEFORE && when != LBM_HALO_AFTER && when != LBM_HALO_SCATTER)
    return fail(LBM_ERR_ARG, "%s: when = %d is not LBM_HALO_BEFORE, _AFTER or _SCATTER", fn,
        when);
  // before: the next step's needs (and a shifted state's ghost data, which
  // are the same slots); after: the last step's, or the open split step's;
  // scatter: shifted states, outside split steps
  const long long done = s->steps_done + ((s->split && when == LBM_HALO_AFTER) ? 1 : 0);
  bool ok;
  if (when == LBM_HALO_SCATTER)
    ok = lbm_halo_shifted(s) && !s->split;
  else if (s->pattern == LBM_PULL)
    ok = when == LBM_HALO_BEFORE;
  else if (s->pattern == LBM_PUSH)
    ok = when == LBM_HALO_AFTER;
  else
    ok = when == LBM_HALO_BEFORE ? (s->steps_done & 1) : (done > 0 && !(done & 1));
  if (!ok)
    return fail(LBM_ERR_STATE, "%s: no %s exchange at step %lld of this pattern", fn,
        when == LBM_HALO_BEFORE ? "before-step" : when == LBM_HALO_AFTER ? "after-step" :
        "scatter", s->steps_done);
  CUDA_TRY(cudaSetDevice(s->device));
  return LBM_OK;
}

extern "C" int lbm_halo_pack(lbm_solver *s, int when, void *to_left, void *to_right)
{
  int rc = halo_check(s, when, to_left, to_right, "lbm_halo_pack");
  if (rc)
    return rc;
  void *lat = halo_lattice(s, when);
  const int first = 1, last = s->g.nx - 2;
  // slots of a shifted state in the left ghost: pull P, AA M (right: opposite)
  const int left_ghost_set = s->pattern == LBM_PULL ? +1 : -1;
  if (when == LBM_HALO_BEFORE) {
    if ((rc = halo_copy(s, lat, last, left_ghost_set, to_right, 1)))
      return rc;
    return halo_copy(s, lat, first, -left_ghost_set, to_left, 1);
  }
  if (when == LBM_HALO_SCATTER) {
    if ((rc = halo_copy(s, lat, 0, left_ghost_set, to_left, 1)))
      return rc;
    return halo_copy(s, lat, s->g.nx - 1, -left_ghost_set, to_right, 1);
  }
  if ((rc = halo_copy(s, lat, s->g.nx - 1, +1, to_right, 1)))
    return rc;
  return halo_copy(s, lat, 0, -1, to_left, 1);
}

extern "C" int lbm_halo_unpack(lbm_solver *s, int when, const void *from_left,
    const void *from_right)
{
  int rc = halo_check(s, when, from_left, from_right, "lbm_halo_unpack");
  if (rc)
    return rc;
  void *lat = halo_lattice(s, when);
  const int first = 1, last = s->g.nx - 2;
  const int left_ghost_set = s->pattern == LBM_PULL ? +1 : -1;
  if (when == LBM_HALO_BEFORE) {
    // the left slab sent its last plane's slots of our left ghost's set
    if ((rc = halo_copy(s, lat, 0, left_ghost_set, (void *)from_left, 0)))
      return rc;
    return halo_copy(s, lat, s->g.nx - 1, -left_ghost_set, (void *)from_right, 0);
  }
  if (when == LBM_HALO_SCATTER) {
    // the left slab sent its right ghost (our first plane's share of its
    // boundary cells' populations); the pull state keeps population d of
    // x + c_d in slot d of x, the AA state population inv d of x - c_d
    const int gm = s->pattern == LBM_PULL ? kGuardOwn : kGuardInv;
    if ((rc = halo_copy(s, lat, first, -left_ghost_set, (void *)from_left, 0, gm)))
      return rc;
    return halo_copy(s, lat, last, left_ghost_set, (void *)from_right, 0, gm);
  }
  if ((rc = halo_copy(s, lat, first, +1, (void *)from_left, 0, kGuardInv)))
    return rc;
  return halo_copy(s, lat, last, -1, (void *)from_right, 0, kGuardInv);
}

extern "C" void *lbm_stream(const lbm_solver *s) { return s ? (void *)s->stream : NULL; }

int lbm::solver_planes(const lbm_solver *s) { return s ? s->nx : -1; }
int lbm::solver_device(const lbm_solver *s) { return s ? s->device : -1; }

// ---------------------------------------------------------------------------
// Seeded initial state on the device
// ---------------------------------------------------------------------------

// splitmix64 (Steele, Lea, Flood 2014), the same counter-based stream as
// lbm_perturbed_equilibrium in host/lbm_host.c: cell c (caller's dense
// index) draws from state seed ^ mix(c * golden + 1), advanced by the
// golden-ratio increment, so host and device produce identical values.
__device__ __forceinline__ uint64_t mix64_d(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

template <class ST>
__global__ void init_equilibrium_kernel(Grid g, UserBox u, int orient, typename ST::S *state,
    const uint32_t *__restrict__ mask, unsigned long long seed, double amp, double rho, float scale)
{
  using V = typename ST::V;
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= u.nz || y >= u.ny)
    return;
  uint32_t cell, m;
  if (!locate(g, mask, x + u.ox, y + u.oy, z + u.oz, cell, m))
    return;
  const long long c = dense_index(u, x, y, z);
  uint64_t st = (uint64_t)seed ^ mix64_d((uint64_t)c * 0x9E3779B97F4A7C15ull + 1ull);
  // explicit round-to-nearest operations: no multiply-add contraction, so
  // the values equal the host generator's (compiled without contraction)
  double uu[3];
  for (int k = 0; k < 3; ++k) {
    st += 0x9E3779B97F4A7C15ull;
    const double r = __dmul_rn((double)(mix64_d(st) >> 11), 1.0 / 9007199254740992.0);
    uu[k] = __dmul_rn(amp, __dadd_rn(__dmul_rn(2.0, r), -1.0));
  }
  const double usq = __dadd_rn(__dadd_rn(__dmul_rn(uu[0], uu[0]), __dmul_rn(uu[1], uu[1])),
      __dmul_rn(uu[2], uu[2]));
  const Nbr nb = make_nbr(g, x + u.ox, y + u.oy, z + u.oz, cell);
#pragma unroll
  for (int d = 0; d < Q; ++d) {
    const int wc = wclass(d);
    const double w = wc == 0 ? 1.0 / 3.0 : wc == 1 ? 1.0 / 18.0 : 1.0 / 36.0;
    const double cu = __dadd_rn(__dadd_rn(__dmul_rn(cx(d), uu[0]), __dmul_rn(cy(d), uu[1])),
        __dmul_rn(cz(d), uu[2]));
    const double t = __dadd_rn(__dadd_rn(__dadd_rn(rho, -__dmul_rn(1.5, usq)),
        __dmul_rn(3.0, cu)), __dmul_rn(__dmul_rn(4.5, cu), cu));
    double v = __dmul_rn(w, t);
    if (ST::kShifted)
      v = __dadd_rn(v, -w);
    int p;
    uint32_t sc;
    state_slot(orient, d, m, cell, nb, p, sc);
    ST::store(state + (long long)p * g.plane + sc, (V)v, (V)scale);
  }
}

template <class ST> static int init_eq_t(lbm_solver *s, unsigned long long seed, double amp,
    double rho)
{
  dim3 grid, block;
  user_launch_shape(s, grid, block);
  init_equilibrium_kernel<ST><<<grid, block, 0, s->stream>>>(s->g, s->ub, orientation(s),
      (typename ST::S *)state_ptr(s), s->mask, seed, amp, rho,
      (float)(s->precision == LBM_F16 ? s->fp16_scale : 1.0));
  CUDA_TRY(cudaGetLastError());
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  return LBM_OK;
}

extern "C" int lbm_init_equilibrium(lbm_solver *s, unsigned long long seed, double amplitude,
    double rho)
{
  if (!s)
    return fail(LBM_ERR_ARG, "lbm_init_equilibrium: NULL solver");
  CUDA_TRY(cudaSetDevice(s->device));
  switch (s->precision) {
  case LBM_F64: return init_eq_t<StoreF64>(s, seed, amplitude, rho);
  case LBM_F32: return init_eq_t<StoreF32>(s, seed, amplitude, rho);
  default: return init_eq_t<StoreF16>(s, seed, amplitude, rho);
  }
}

extern "C" int lbm_device_memory(size_t *free_bytes, size_t *total_bytes)
{
  size_t f = 0, t = 0;
  CUDA_TRY(cudaMemGetInfo(&f, &t));
  if (free_bytes)
    *free_bytes = f;
  if (total_bytes)
    *total_bytes = t;
  return LBM_OK;
}

// ---------------------------------------------------------------------------
// Adjoint of the Brinkman step with checkpointing
// ---------------------------------------------------------------------------

// Sum of the x momentum and number of fluid cells on the caller's plane
// x = nx-1.
static int outlet_sums(lbm_solver *s, double *sum, double *count)
{
  if (s->precision == LBM_F64)
    outlet_launch<StoreF64>(s);
  else if (s->precision == LBM_F32)
    outlet_launch<StoreF32>(s);
  else
    outlet_launch<StoreF16>(s);
  CUDA_TRY(cudaGetLastError());
  double *fin = s->red + (size_t)kRedBlocks * kRedVals;
  final_reduce_kernel<<<1, kRedThreads, 0, s->stream>>>(s->red, kRedBlocks, 0u, fin);
  CUDA_TRY(cudaGetLastError());
  double h[kRedVals];
  CUDA_TRY(cudaMemcpyAsync(h, fin, sizeof(h), cudaMemcpyDeviceToHost, s->stream));
  CUDA_TRY(cudaStreamSynchronize(s->stream));
  *sum = h[0];
  *count = h[1];
  return LBM_OK;
}

// per-cell gradient (device cell order) -> caller's dense order
__global__ void grad_to_dense_kernel(Grid g, UserBox u, const double *__restrict__ grad,
    const uint32_t *__restrict__ mask, double *dense)
{
  const int z = blockIdx.x * blockDim.x + threadIdx.x;
  const int y = blockIdx.y * blockDim.y + threadIdx.y;
  const int x = blockIdx.z;
  if (z >= u.nz || y >= u.ny)
    return;
  const uint32_t cell = cell_index(g, x + u.ox, y + u.oy, z + u.oz);
  dense[dense_index(u, x, y, z)] = (mask[cell] & kSolidBit) ? 0.0 : grad[cell];
}

extern "C" int lbm_adjoint_gradient(lbm_solver *s, int steps, int checkpoint_every,
    double *grad, double *j_out, double *info)
{
  if (!s || steps < 1 || !grad)
    return fail(LBM_ERR_ARG, "lbm_adjoint_gradient: bad arguments");
  if (s->split)
    return fail(LBM_ERR_STATE, "lbm_adjoint_gradient: a split step is open");
  if (s->pattern != LBM_AA)
    return fail(LBM_ERR_ARG, "lbm_adjoint_gradient: needs an AA solver");
  if (s->slab)
    return fail(LBM_ERR_ARG, "lbm_adjoint_gradient: not available on slab solvers");
  if (s->bc_on)
    return fail(LBM_ERR_ARG, "lbm_adjoint_gradient: not available with the pressure boundary");
  if (s->precision == LBM_F16)
    return fail(LBM_ERR_ARG, "lbm_adjoint_gradient: FP16 storage is not supported (FP64/FP32)");
  if (!s->porosity || s->alpha == 0.0)
    return fail(LBM_ERR_STATE, "lbm_adjoint_gradient: set a porosity field first");
  CUDA_TRY(cudaSetDevice(s->device));
  const bool f64 = s->precision == LBM_F64;
  const size_t vs = f64 ? sizeof(double) : sizeof(float);
  const size_t P = (size_t)s->g.plane;
  const size_t ubytes = 3 * P * vs;  // momentum of one step
  const size_t lbytes = Q * P * vs;  // one adjoint lattice
  // checkpoint interval: given; 0 = the one that minimises checkpoints
  // (steps/k states) plus the segment's saved momenta (k momentum sets);
  // LBM_CKPT_AUTO = the longest interval (least recomputation: steps - k
  // steps are recomputed) whose memory fits in 90% of the free device memory
  const auto mem_for = [&](long long kk) {
    return (double)((steps + kk - 1) / kk) * (double)s->state_bytes + (double)kk * ubytes +
        2.0 * lbytes + (double)P * 8;
  };
  int k = checkpoint_every;
  const int k_sqrt = std::max(1, (int)ceil(sqrt((double)steps * (double)s->state_bytes /
      (double)ubytes)));
  if (k == LBM_CKPT_AUTO) {
    size_t free_b = 0, total_b = 0;
    CUDA_TRY(cudaMemGetInfo(&free_b, &total_b));
    const double budget = 0.9 * (double)free_b;
    k = std::min(k_sqrt, steps);
    // memory grows with k beyond k_sqrt; the largest fitting k by bisection
    long long lo = k, hi = steps;
    if (mem_for(hi) <= budget)
      lo = hi;
    while (hi - lo > 1) {
      const long long mid = (lo + hi) / 2;
      if (mem_for(mid) <= budget)
        lo = mid;
      else
        hi = mid;
    }
    k = (int)lo;
  } else if (k <= 0) {
    k = k_sqrt;
  }
  if (k > steps)
    k = steps;
  const int nck = (steps + k - 1) / k;
  const size_t extra = (size_t)nck * s->state_bytes + (size_t)k * ubytes + 2 * lbytes + P * 8;

  char *ck = NULL, *ub = NULL, *lam = NULL;
  double *dg = NULL;
  cudaEvent_t e0 = NULL, e1 = NULL;
  int rc = LBM_OK;
#define ATRY(x)                                                                               do {                                                                                          cudaError_t err_ = (x);                                                                     if (err_ != cudaSuccess) {                                                                    rc = fail(err_ == cudaErrorMemoryAllocation ? LBM_ERR_ALLOC : LBM_ERR_CUDA,                    "lbm_adjoint_gradient: %s: %s", #x, cudaGetErrorString(err_));                         goto done;                                                                                }                                                                                         } while (0)
#define RTRY(x)                                                                               do {                                                                                          rc = (x);                                                                                   if (rc)                                                                                       goto done;                                                                              } while (0)
  {
    ATRY(cudaMalloc((void **)&ck, (size_t)nck * s->state_bytes));
    ATRY(cudaMalloc((void **)&ub, (size_t)k * ubytes));
    ATRY(cudaMalloc((void **)&lam, 2 * lbytes));
    ATRY(cudaMalloc((void **)&dg, P * 8));
    ATRY(cudaEventCreate(&e0));
    ATRY(cudaEventCreate(&e1));
    const long long t0 = s->steps_done;
    void *state = s->buf[0];

    // forward sweep: checkpoint every k steps; the last segment saves its
    // momenta directly, so the reverse sweep does not recompute it
    ATRY(cudaEventRecord(e0, s->stream));
    for (int c = 0; c < nck; ++c) {
      ATRY(cudaMemcpyAsync(ck + (size_t)c * s->state_bytes, state, s->state_bytes,
          cudaMemcpyDeviceToDevice, s->stream));
      const int len = std::min(k, steps - c * k);
      if (c < nck - 1) {
        RTRY(lbm_run(s, len));
        continue;
      }
      for (int i = 0; i < len; ++i) {
        s->u_save_next = ub + (size_t)i * ubytes;
        rc = launch_one(s, NULL);
        s->u_save_next = NULL;
        if (rc)
          goto done;
      }
    }
    ATRY(cudaEventRecord(e1, s->stream));
    ATRY(cudaEventSynchronize(e1));
    float fwd_ms = 0.f;
    ATRY(cudaEventElapsedTime(&fwd_ms, e0, e1));

    double jsum = 0.0, jcount = 0.0;
    RTRY(outlet_sums(s, &jsum, &jcount));
    if (j_out)
      *j_out = jcount > 0 ? jsum / jcount : 0.0;

    // reverse sweep
    ATRY(cudaEventRecord(e0, s->stream));
    ATRY(launch_adjoint_seed(f64 ? kF64 : kF32, s->g, s->ub.ox + s->ub.nx - 1,
        jcount > 0 ? 1.0 / jcount : 0.0, lam, s->mask, s->stream));
    ATRY(cudaMemsetAsync(dg, 0, P * 8, s->stream));
    int cur = 0; // lambda^{t+1} lives in lam + cur * lbytes
    float adj_ms = 0.f;
    for (int c = nck - 1; c >= 0; --c) {
      const int tc = c * k, len = std::min(k, steps - tc);
      if (c < nck - 1) {
        ATRY(cudaMemcpyAsync(state, ck + (size_t)c * s->state_bytes, s->state_bytes,
            cudaMemcpyDeviceToDevice, s->stream));
        s->steps_done = t0 + tc;
      }
      for (int i = 0; i < len && c < nck - 1; ++i) {
        s->u_save_next = ub + (size_t)i * ubytes;
        rc = launch_one(s, NULL);
        s->u_save_next = NULL;
        if (rc)
          goto done;
      }
      for (int i = len - 1; i >= 0; --i) {
        if (f64) {
          AdjArgs<double> a;
          a.g = s->g;
          a.lam_next = (const double *)(lam + cur * lbytes);
          a.lam = (double *)(lam + (cur ^ 1) * lbytes);
          a.u = (const double *)(ub + (size_t)i * ubytes);
          a.mask = s->mask;
          a.porosity = s->porosity;
          a.grad = dg;
          a.oE = s->omega;
          a.oO = 1.0 / (0.5 + s->lambda / (1.0 / s->omega - 0.5));
          a.w0 = 1.0 / 3.0;
          a.w1 = 1.0 / 18.0;
          a.w2 = 1.0 / 36.0;
          a.alpha = s->alpha;
          ATRY(launch_adjoint_step_f64(a, s->stream));
        } else {
          AdjArgs<float> a;
          a.g = s->g;
          a.lam_next = (const float *)(lam + cur * lbytes);
          a.lam = (float *)(lam + (cur ^ 1) * lbytes);
          a.u = (const float *)(ub + (size_t)i * ubytes);
          a.mask = s->mask;
          a.porosity = s->porosity;
          a.grad = dg;
          a.oE = (float)s->omega;
          a.oO = (float)(1.0 / (0.5 + s->lambda / (1.0 / s->omega - 0.5)));
          a.w0 = (float)(1.0 / 3.0);
          a.w1 = (float)(1.0 / 18.0);
          a.w2 = (float)(1.0 / 36.0);
          a.alpha = (float)s->alpha;
          ATRY(launch_adjoint_step_f32(a, s->stream));
        }
        cur ^= 1;
      }
    }
    ATRY(cudaEventRecord(e1, s->stream));
    ATRY(cudaEventSynchronize(e1));
    ATRY(cudaEventElapsedTime(&adj_ms, e0, e1));

    // leave the solver at the initial state
    ATRY(cudaMemcpyAsync(state, ck, s->state_bytes, cudaMemcpyDeviceToDevice, s->stream));
    s->steps_done = t0;
    {
      dim3 grid, block;
      user_launch_shape(s, grid, block);
      grad_to_dense_kernel<<<grid, block, 0, s->stream>>>(s->g, s->ub, dg, s->mask, s->staging);
      ATRY(cudaGetLastError());
      ATRY(cudaMemcpyAsync(grad, s->staging, sizeof(double) * (size_t)s->nx * s->ny * s->nz,
          cudaMemcpyDeviceToHost, s->stream));
      ATRY(cudaStreamSynchronize(s->stream));
    }
    if (info) {
      info[0] = fwd_ms;
      info[1] = adj_ms;
      info[2] = k;
      info[3] = nck;
      info[4] = (double)extra;
      info[5] = (double)(s->dev_bytes + extra);
    }
  }
done:
  s->u_save_next = NULL;
  cudaFree(ck);
  cudaFree(ub);
  cudaFree(lam);
  cudaFree(dg);
  if (e0)
    cudaEventDestroy(e0);
  if (e1)
    cudaEventDestroy(e1);
#undef ATRY
#undef RTRY
  return rc;
}

extern "C" int lbm_pin_host(void *ptr, size_t bytes)
{
  if (!ptr || !bytes)
    return fail(LBM_ERR_ARG, "lbm_pin_host: NULL or empty buffer");
  CUDA_TRY(cudaHostRegister(ptr, bytes, cudaHostRegisterDefault));
  return LBM_OK;
}

extern "C" int lbm_unpin_host(void *ptr)
{
  if (!ptr)
    return fail(LBM_ERR_ARG, "lbm_unpin_host: NULL buffer");
  CUDA_TRY(cudaHostUnregister(ptr));
  return LBM_OK;
}

extern "C" long long lbm_fluid_cells(const lbm_solver *s) { return s ? s->n_fluid : -1; }
extern "C" long long lbm_steps_done(const lbm_solver *s) { return s ? s->steps_done : -1; }
extern "C" size_t lbm_device_bytes(const lbm_solver *s) { return s ? s->dev_bytes : 0; }
extern "C" long long lbm_launch_count(const lbm_solver *s) { return s ? s->launches : -1; }
extern "C" double lbm_bytes_per_update(const lbm_solver *s)
{
  return s ? 2.0 * Q * (double)storage_size(s->precision) : 0.0;
}
