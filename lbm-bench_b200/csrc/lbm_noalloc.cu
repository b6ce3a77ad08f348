// lbm_mass_momentum_noalloc: the FP64 mass/momentum/NaN reduction of
// lbm_mass_momentum, for callers that must not allocate device memory.
//
// Who cannot allocate: a plug-in inside a host application whose caching
// allocator already holds the device's memory (a cudaMalloc behind its back
// can fail or fragment that pool), and control loops where the device-wide
// synchronisation that cudaMalloc/cudaFree may imply is not acceptable. Such
// a caller owns the population and flag buffers and only wants the
// diagnostic.
//
// The reduction needs scratch for its per-block partial sums. Here that
// scratch is a file-scope device array of fixed size: one row per x-plane,
// at most kMaxPlanes planes, plus one row for the final result. Every GPU
// that loads this library holds the array (kMaxPlanes+1 rows of 6 doubles,
// about 384 KiB) until the process exits. All calls share it; a call writes
// every row it later reads, so no clearing is needed, but two calls whose
// kernels overlap on the GPU race on the rows - serialise them (one stream,
// or synchronise in between). The call itself is synchronous: it copies the
// totals to the host and synchronises the caller's stream.
//
// Host code cannot use the array's name as a device address (in host code
// it names a host-side stand-in). The device address is looked up once per
// device, with that device current, through cudaGetSymbolAddress on the
// first call made on that device; make that first call before any stream
// capture is started on the device.
#include <mutex>

#include "lbm_b200.h"
#include "lbm_internal.h"

using namespace lbm;

namespace {

constexpr int kMaxPlanes = LBM_NOALLOC_MAX_PLANES;
constexpr int kThreads = 256;
constexpr int kVals = 6; // mass, jx, jy, jz, non-finite cells, (unused)
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_noalloc_rows[(kMaxPlanes + 1) * kVals];

std::mutex g_mu;
double *g_rows_addr[kMaxDevices] = {};

// Fixed-shape tree sum of kVals doubles over one block.
__device__ void tree_sum(double (&v)[kVals], double *out)
{
  __shared__ double sh[kVals][kThreads];
  for (int k = 0; k < kVals; ++k)
    sh[k][threadIdx.x] = v[k];
  __syncthreads();
  for (int s = kThreads / 2; s > 0; s >>= 1) {
    if ((int)threadIdx.x < s)
      for (int k = 0; k < kVals; ++k)
        sh[k][threadIdx.x] += sh[k][threadIdx.x + s];
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int k = 0; k < kVals; ++k)
      out[k] = sh[k][0];
}

// Block x sums the fluid cells of plane x into rows[x].
// f: [19][nx][ny][nz] doubles (z fastest); flags: [nz][ny][nx] ints.
__global__ void __launch_bounds__(kThreads) plane_sums(const double *__restrict__ f,
    const int *__restrict__ flags, int nx, int ny, int nz, double *rows)
{
  const int x = blockIdx.x;
  const long long n = (long long)nx * ny * nz;
  const long long nyz = (long long)ny * nz;
  double v[kVals] = { 0, 0, 0, 0, 0, 0 };
  for (long long i = threadIdx.x; i < nyz; i += kThreads) {
    const int y = (int)(i / nz), z = (int)(i % nz);
    if (!flags[((long long)z * ny + y) * nx + x])
      continue;
    const long long c = (long long)x * nyz + i;
    double rho = 0.0, jx = 0.0, jy = 0.0, jz = 0.0;
    bool finite = true;
#pragma unroll
    for (int d = 0; d < Q; ++d) {
      const double p = f[d * n + c];
      finite = finite && isfinite(p);
      rho += p;
      jx += cx(d) * p;
      jy += cy(d) * p;
      jz += cz(d) * p;
    }
    v[0] += rho;
    v[1] += jx;
    v[2] += jy;
    v[3] += jz;
    v[4] += finite ? 0.0 : 1.0;
  }
  tree_sum(v, rows + (size_t)x * kVals);
}

// One block sums rows[0..nx) in a fixed order into rows[kMaxPlanes].
__global__ void __launch_bounds__(kThreads) rows_total(double *rows, int nx)
{
  double v[kVals] = { 0, 0, 0, 0, 0, 0 };
  for (int r = threadIdx.x; r < nx; r += kThreads)
    for (int k = 0; k < kVals; ++k)
      v[k] += rows[(size_t)r * kVals + k];
  tree_sum(v, rows + (size_t)kMaxPlanes * kVals);
}

// Device address of the scratch rows on the current device (looked up once).
int rows_on_current_device(double **out)
{
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess)
    return record_error(LBM_ERR_CUDA, "lbm_mass_momentum_noalloc: cudaGetDevice failed: %s",
        cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return record_error(LBM_ERR_ARG, "lbm_mass_momentum_noalloc: device %d out of range", dev);
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_rows_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_rows);
    if (e != cudaSuccess || !p)
      return record_error(LBM_ERR_CUDA,
          "lbm_mass_momentum_noalloc: cudaGetSymbolAddress of the scratch failed: %s",
          cudaGetErrorString(e));
    g_rows_addr[dev] = (double *)p;
  }
  *out = g_rows_addr[dev];
  return LBM_OK;
}

// LBM_OK if p is device memory of the current device (or managed memory).
int on_current_device(const void *p, const char *name)
{
  int dev = -1;
  cudaError_t e = cudaGetDevice(&dev);
  cudaPointerAttributes a {};
  if (e == cudaSuccess)
    e = cudaPointerGetAttributes(&a, p);
  if (e != cudaSuccess) {
    cudaGetLastError();
    return record_error(LBM_ERR_ARG, "lbm_mass_momentum_noalloc: %s is not a device pointer (%s)",
        name, cudaGetErrorString(e));
  }
  if (a.type == cudaMemoryTypeManaged)
    return LBM_OK;
  if (a.type != cudaMemoryTypeDevice || a.device != dev)
    return record_error(LBM_ERR_ARG,
        "lbm_mass_momentum_noalloc: %s must be device memory of the current device %d "
        "(memory type %d, device %d)",
        name, dev, (int)a.type, a.device);
  return LBM_OK;
}

} // namespace

extern "C" int lbm_mass_momentum_noalloc(const double *f, const int *flags, int nx, int ny,
    int nz, double out[4], long long *nonfinite, void *stream)
{
  if (!f || !flags || !out || nx <= 0 || ny <= 0 || nz <= 0)
    return record_error(LBM_ERR_ARG, "lbm_mass_momentum_noalloc: NULL pointer or empty box");
  if (nx > kMaxPlanes)
    return record_error(LBM_ERR_ARG,
        "lbm_mass_momentum_noalloc: nx = %d exceeds the maximum of %d x-planes that its "
        "fixed scratch array holds",
        nx, kMaxPlanes);
  double *rows = nullptr;
  int rc = rows_on_current_device(&rows);
  if (rc)
    return rc;
  rc = on_current_device(f, "f");
  if (!rc)
    rc = on_current_device(flags, "flags");
  if (rc)
    return rc;
  cudaStream_t st = (cudaStream_t)stream;
  plane_sums<<<nx, kThreads, 0, st>>>(f, flags, nx, ny, nz, rows);
  rows_total<<<1, kThreads, 0, st>>>(rows, nx);
  cudaError_t e = cudaGetLastError();
  double h[kVals];
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(h, rows + (size_t)kMaxPlanes * kVals, sizeof(h), cudaMemcpyDeviceToHost,
        st);
  if (e == cudaSuccess)
    e = cudaStreamSynchronize(st);
  if (e != cudaSuccess)
    return record_error(LBM_ERR_CUDA, "lbm_mass_momentum_noalloc: %s", cudaGetErrorString(e));
  for (int k = 0; k < 4; ++k)
    out[k] = h[k];
  const long long bad = (long long)h[4];
  if (nonfinite)
    *nonfinite = bad;
  if (bad)
    return record_error(LBM_ERR_NONFINITE, "state holds NaN/Inf in %lld fluid cells", bad);
  return LBM_OK;
}
