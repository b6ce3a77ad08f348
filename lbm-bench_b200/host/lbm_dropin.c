/* LBM-Bench-compatible Init / Kernel / Deinit and node accessors on top of
 * the flat liblbmb200 API (include/lbm_b200_dropin.h). */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "lbm_b200.h"
#include "lbm_b200_dropin.h"

#define Q 19

/* D3Q19 velocity set in the reference's direction order (src/lbm.c:20-29). */
static const int CX[Q] = { 0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0 };
static const int CY[Q] = { 1, -1, 0, 0, 1, -1, 1, -1, 0, 1, 0, 0, -1, 0, -1, 1, 0, 0, 0 };
static const int CZ[Q] = { 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, 0 };
static const int INV[Q] = { 1, 0, 3, 2, 7, 6, 5, 4, 13, 14, 16, 17, 15, 8, 9, 12, 10, 11, 18 };

/* Device-side state kept behind the public KernelDataType (first member, so
 * the caller's KernelDataType* points at it). */
typedef struct {
  KernelDataType kd;
  lbm_solver *solver;
  int pattern;
  int aos; /* host lattices in indexAoS order (pull-aos / push-aos) */
  size_t pdf_bytes;
  int pinned[2];
} CudaKernelData;

static double g_lambda = 1.0 / 12.0;
static int g_force     = -1;

void lbmB200SetMagicParameter(double lambda) { g_lambda = lambda; }
void lbmB200SetBodyForce(int on) { g_force = on; }

static int body_force_on(void)
{
  if (g_force >= 0)
    return g_force;
  const char *e = getenv("LBM_B200_BODY_FORCE");
  return e && e[0] == '1';
}

/* Storage layout of the drop-in solvers: the compact (fluid-only) layout
 * for FP64, where it is faster for every pattern, and the dense layout for
 * the reduced-precision names, whose multi-cell kernels are written for it.
 * The environment variable LBM_B200_LAYOUT=dense or =compact overrides the
 * choice; results are the same either way (FP64 bit for bit). */
static int use_compact(int precision)
{
  const char *e = getenv("LBM_B200_LAYOUT");
  if (e && strcmp(e, "dense") == 0)
    return 0;
  if (e && strcmp(e, "compact") == 0)
    return 1;
  return precision == LBM_F64;
}

static void die(const char *what)
{
  printf("ERROR: %s: %s\n", what, lbm_last_error());
  exit(EXIT_FAILURE);
}

/* indexSoA of the reference (src/lbm.h:113-116) in 64-bit */
static long long soa(const int *g, int x, int y, int z, int d)
{
  return (((long long)d * g[0] + x) * g[1] + y) * g[2] + z;
}

/* indexAoS of the reference (src/lbm.h:118-121) in 64-bit */
static long long aos(const int *g, int x, int y, int z, int d)
{
  return (((long long)x * g[1] + y) * g[2] + z) * Q + d;
}

/* Node accessors with the reference's slot rules (src/lbm.c:193-294):
 * push (x, d); pull (x - c_d, d); AA (x - c_d, inv d) after an even
 * iteration, (x, d) otherwise. Coordinates include the ghost offset. */
static long long slot_push(KernelDataType *kd, int x, int y, int z, int d)
{
  return soa(kd->GlobalDims, x + kd->Offsets[0], y + kd->Offsets[1], z + kd->Offsets[2], d);
}
static long long slot_pull(KernelDataType *kd, int x, int y, int z, int d)
{
  return soa(kd->GlobalDims, x + kd->Offsets[0] - CX[d], y + kd->Offsets[1] - CY[d],
      z + kd->Offsets[2] - CZ[d], d);
}
static long long slot_aa(KernelDataType *kd, int x, int y, int z, int d)
{
  if (kd->Iteration % 2 == 0)
    return soa(kd->GlobalDims, x + kd->Offsets[0] - CX[d], y + kd->Offsets[1] - CY[d],
        z + kd->Offsets[2] - CZ[d], INV[d]);
  return slot_push(kd, x, y, z, d);
}

#define ACCESSORS(NAME, SLOT)                                                                \
  static void getNode##NAME(KernelDataType *kd, int x, int y, int z, PdfType *pdfs)          \
  {                                                                                         \
    for (int d = 0; d < Q; ++d)                                                              \
      pdfs[d] = kd->PdfsActive[SLOT(kd, x, y, z, d)];                                        \
  }                                                                                         \
  static void setNode##NAME(KernelDataType *kd, int x, int y, int z, PdfType *pdfs)          \
  {                                                                                         \
    for (int d = 0; d < Q; ++d)                                                              \
      kd->PdfsActive[SLOT(kd, x, y, z, d)] = pdfs[d];                                        \
  }                                                                                         \
  static void bcGet##NAME(KernelDataType *kd, int x, int y, int z, int d, PdfType *pdf)     \
  {                                                                                         \
    *pdf = kd->PdfsActive[SLOT(kd, x, y, z, d)];                                             \
  }                                                                                         \
  static void bcSet##NAME(KernelDataType *kd, int x, int y, int z, int d, PdfType pdf)      \
  {                                                                                         \
    kd->PdfsActive[SLOT(kd, x, y, z, d)] = pdf;                                              \
  }

/* the AoS kernels' accessors: the same slots in indexAoS order
 * (src/lbm.c:227-258) */
static long long slot_push_aos(KernelDataType *kd, int x, int y, int z, int d)
{
  return aos(kd->GlobalDims, x + kd->Offsets[0], y + kd->Offsets[1], z + kd->Offsets[2], d);
}
static long long slot_pull_aos(KernelDataType *kd, int x, int y, int z, int d)
{
  return aos(kd->GlobalDims, x + kd->Offsets[0] - CX[d], y + kd->Offsets[1] - CY[d],
      z + kd->Offsets[2] - CZ[d], d);
}

ACCESSORS(Push, slot_push)
ACCESSORS(Pull, slot_pull)
ACCESSORS(Aa, slot_aa)
ACCESSORS(PushAos, slot_push_aos)
ACCESSORS(PullAos, slot_pull_aos)

/* Number of entries the reference's bounce-back list would hold for this
 * lattice (src/lbm.c:465-494): for every fluid cell and direction, the
 * neighbour (x - c_d for pull, x + c_d otherwise) either leaves the box
 * across a periodic axis or is an in-box obstacle. */
static int count_bounce_back(const LatticeDescType *ld, int pattern)
{
  const int nx = ld->Dims[0], ny = ld->Dims[1], nz = ld->Dims[2];
  int n = 0;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        if (ld->Lattice[((long long)z * ny + y) * nx + x] == 0)
          continue;
        for (int d = 0; d < Q; ++d) {
          const int s = (pattern == LBM_PULL) ? -1 : 1;
          const int a = x + s * CX[d], b = y + s * CY[d], c = z + s * CZ[d];
          const int outx = a < 0 || a >= nx, outy = b < 0 || b >= ny, outz = c < 0 || c >= nz;
          if ((outx && ld->PeriodicX) || (outy && ld->PeriodicY) || (outz && ld->PeriodicZ))
            ++n;
          else if (outx || outy || outz)
            continue;
          else if (ld->Lattice[((long long)c * ny + b) * nx + a] == 0)
            ++n;
        }
      }
  return n;
}

static void cudaKernel(LatticeDescType *ld, KernelDataType *kd, CaseDataType *cd)
{
  CudaKernelData *ck = (CudaKernelData *)kd;
  (void)ld;
  if (lbm_set_params(ck->solver, (double)cd->Omega, g_lambda, (double)cd->XForce,
          body_force_on()) != LBM_OK)
    die("cuda kernel parameters");
  int steps = cd->MaxIterations;
  if (ck->pattern == LBM_AA && (steps & 1))
    ++steps; /* the reference's AA loop runs whole even/odd pairs */

  /* like the reference, every run starts from Pdfs[0] in the pattern's
   * natural orientation (src/kernel_pull_soa.c:35, src/kernel_aa_soa.c:29) */
  const int ref_o = ((ck->pattern == LBM_PULL) ? LBM_REF_PULL : LBM_REF_NATURAL) |
      (ck->aos ? LBM_REF_AOS : 0);
  if (lbm_set_state_padded(ck->solver, kd->Pdfs[0], (int)sizeof(PdfType), ref_o) != LBM_OK)
    die("cuda kernel upload");
  double ms = 0.0;
  if (lbm_run_timed(ck->solver, steps, &ms) != LBM_OK)
    die("cuda kernel run");
  kd->Duration = ms * 1e-3;

  /* pull/push end in Pdfs[steps % 2] after their pointer swaps
   * (src/kernel_pull_soa.c:211-217); AA ends in Pdfs[0] after an odd
   * iteration (src/kernel_aa_soa.c:280-289) */
  PdfType *outbuf = (ck->pattern == LBM_AA) ? kd->Pdfs[0] : kd->Pdfs[steps % 2];
  if (lbm_get_state_padded(ck->solver, outbuf, (int)sizeof(PdfType), ref_o) != LBM_OK)
    die("cuda kernel download");
  kd->PdfsActive = outbuf;
  if (ck->pattern == LBM_AA)
    kd->Iteration = steps - 1;
}

/* Host layouts of the registered kernels: SoA, the AoS order of the
 * reference's pull-aos / push-aos, or SoA with the 8^3 blocking the
 * reference's blk-*-soa kernels record in kd->Blk (src/lbm.c:629-651). The
 * device state is SoA in every case. */
enum { HOST_SOA, HOST_AOS, HOST_BLK };

static void initCuda(LatticeDescType *ld, KernelDataType **kdp, int pattern, int precision,
    const char *name, int host_layout)
{
  CudaKernelData *ck = (CudaKernelData *)calloc(1, sizeof(CudaKernelData));
  if (!ck) {
    printf("ERROR: %s: host allocation failed\n", name);
    exit(EXIT_FAILURE);
  }
  KernelDataType *kd = &ck->kd;
  ck->pattern        = pattern;
  ck->aos            = host_layout == HOST_AOS;
  for (int a = 0; a < 3; ++a) {
    kd->Dims[a]       = ld->Dims[a];
    kd->GlobalDims[a] = ld->Dims[a] + 2;
    kd->Offsets[a]    = 1;
    kd->Blk[a]        = host_layout == HOST_BLK ? 8 : kd->GlobalDims[a];
  }
  kd->Iteration = -1;
  const long long cells =
      (long long)kd->GlobalDims[0] * kd->GlobalDims[1] * (long long)kd->GlobalDims[2];
  ck->pdf_bytes          = sizeof(PdfType) * (size_t)Q * (size_t)cells;
  const size_t align     = 2u * 1024u * 1024u;
  const size_t allocated = (ck->pdf_bytes + align - 1) / align * align;
  const int nbuf         = (pattern == LBM_AA) ? 1 : 2;
  for (int b = 0; b < nbuf; ++b) {
    kd->Pdfs[b] = (PdfType *)aligned_alloc(align, allocated);
    if (!kd->Pdfs[b]) {
      printf("ERROR: %s: host allocation of %.1f MiB failed\n", name, allocated / 1048576.0);
      exit(EXIT_FAILURE);
    }
    memset(kd->Pdfs[b], 0, allocated);
    ck->pinned[b] = lbm_pin_host(kd->Pdfs[b], allocated) == LBM_OK;
  }
  kd->PdfsActive        = kd->Pdfs[0];
  kd->BounceBackPdfsSrc = NULL;
  kd->BounceBackPdfsDst = NULL;
  kd->nBounceBackPdfs   = count_bounce_back(ld, pattern);
  kd->LoopBalance       = 2.0 * Q * sizeof(PdfType);
  if (pattern == LBM_PUSH && ck->aos) {
    kd->GetNode                  = getNodePushAos;
    kd->SetNode                  = setNodePushAos;
    kd->BoundaryConditionsGetPdf = bcGetPushAos;
    kd->BoundaryConditionsSetPdf = bcSetPushAos;
  } else if (pattern == LBM_PULL && ck->aos) {
    kd->GetNode                  = getNodePullAos;
    kd->SetNode                  = setNodePullAos;
    kd->BoundaryConditionsGetPdf = bcGetPullAos;
    kd->BoundaryConditionsSetPdf = bcSetPullAos;
  } else if (pattern == LBM_PUSH) {
    kd->GetNode                  = getNodePush;
    kd->SetNode                  = setNodePush;
    kd->BoundaryConditionsGetPdf = bcGetPush;
    kd->BoundaryConditionsSetPdf = bcSetPush;
  } else if (pattern == LBM_PULL) {
    kd->GetNode                  = getNodePull;
    kd->SetNode                  = setNodePull;
    kd->BoundaryConditionsGetPdf = bcGetPull;
    kd->BoundaryConditionsSetPdf = bcSetPull;
  } else {
    kd->GetNode                  = getNodeAa;
    kd->SetNode                  = setNodeAa;
    kd->BoundaryConditionsGetPdf = bcGetAa;
    kd->BoundaryConditionsSetPdf = bcSetAa;
  }
  kd->Kernel = cudaKernel;
  const int compact = use_compact(precision);
  if ((compact ? lbm_create_compact : lbm_create)(&ck->solver, ld->Dims[0], ld->Dims[1],
          ld->Dims[2], ld->Lattice, ld->PeriodicX, ld->PeriodicY, ld->PeriodicZ, pattern,
          precision) != LBM_OK)
    die(name);
  printf("# %s: %lld LB nodes with padding, host %.1f MiB (%s), device %.1f MiB (%s layout)\n",
      name, cells, nbuf * ck->pdf_bytes / 1048576.0,
      nbuf == 1 ? "single lattice" : "both lattices", lbm_device_bytes(ck->solver) / 1048576.0,
      compact ? "compact" : "dense");
  printf("# bounce-back PDFs: %d\n", kd->nBounceBackPdfs);
  if (host_layout == HOST_BLK)
    printf("# blocking x: %3d y: %3d z: %3d\n", kd->Blk[0], kd->Blk[1], kd->Blk[2]);
  *kdp = kd;
}

#ifdef PRECISION_SP
#define NATIVE_PRECISION LBM_F32
#else
#define NATIVE_PRECISION LBM_F64
#endif

void kernelInitCudaPullSoA(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PULL, NATIVE_PRECISION, "cuda-pull-soa", HOST_SOA);
}
void kernelInitCudaPushSoA(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PUSH, NATIVE_PRECISION, "cuda-push-soa", HOST_SOA);
}
void kernelInitCudaAaSoA(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_AA, NATIVE_PRECISION, "cuda-aa-soa", HOST_SOA);
}
void kernelInitCudaPullAoS(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PULL, NATIVE_PRECISION, "cuda-pull-aos", HOST_AOS);
}
void kernelInitCudaPushAoS(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PUSH, NATIVE_PRECISION, "cuda-push-aos", HOST_AOS);
}
void kernelInitCudaBlkPushSoA(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PUSH, NATIVE_PRECISION, "cuda-blk-push-soa", HOST_BLK);
}
void kernelInitCudaBlkPullSoA(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PULL, NATIVE_PRECISION, "cuda-blk-pull-soa", HOST_BLK);
}
void kernelInitCudaPullSoAFp32(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PULL, LBM_F32, "cuda-pull-soa-fp32", HOST_SOA);
}
void kernelInitCudaPushSoAFp32(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PUSH, LBM_F32, "cuda-push-soa-fp32", HOST_SOA);
}
void kernelInitCudaAaSoAFp32(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_AA, LBM_F32, "cuda-aa-soa-fp32", HOST_SOA);
}
void kernelInitCudaPullSoAFp16(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PULL, LBM_F16, "cuda-pull-soa-fp16", HOST_SOA);
}
void kernelInitCudaPushSoAFp16(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_PUSH, LBM_F16, "cuda-push-soa-fp16", HOST_SOA);
}
void kernelInitCudaAaSoAFp16(LatticeDescType *ld, KernelDataType **kd, CaseDataType *cd)
{
  (void)cd;
  initCuda(ld, kd, LBM_AA, LBM_F16, "cuda-aa-soa-fp16", HOST_SOA);
}

void kernelDeinitCuda(LatticeDescType *ld, KernelDataType **kdp)
{
  (void)ld;
  if (!kdp || !*kdp)
    return;
  CudaKernelData *ck = (CudaKernelData *)*kdp;
  lbm_destroy(ck->solver);
  for (int b = 0; b < 2; ++b) {
    if (!ck->kd.Pdfs[b])
      continue;
    if (ck->pinned[b])
      lbm_unpin_host(ck->kd.Pdfs[b]);
    free(ck->kd.Pdfs[b]);
  }
  free(ck);
  *kdp = NULL;
}

/* the reference's seven names in its order (src/lbm.c:33-41), then the
 * reduced-precision storage variants */
const KernelFunctionsType LbmB200Kernels[] = {
  { "cuda-pull-soa", kernelInitCudaPullSoA, kernelDeinitCuda },
  { "cuda-pull-aos", kernelInitCudaPullAoS, kernelDeinitCuda },
  { "cuda-push-soa", kernelInitCudaPushSoA, kernelDeinitCuda },
  { "cuda-push-aos", kernelInitCudaPushAoS, kernelDeinitCuda },
  { "cuda-blk-push-soa", kernelInitCudaBlkPushSoA, kernelDeinitCuda },
  { "cuda-blk-pull-soa", kernelInitCudaBlkPullSoA, kernelDeinitCuda },
  { "cuda-aa-soa", kernelInitCudaAaSoA, kernelDeinitCuda },
  { "cuda-pull-soa-fp32", kernelInitCudaPullSoAFp32, kernelDeinitCuda },
  { "cuda-push-soa-fp32", kernelInitCudaPushSoAFp32, kernelDeinitCuda },
  { "cuda-aa-soa-fp32", kernelInitCudaAaSoAFp32, kernelDeinitCuda },
  { "cuda-pull-soa-fp16", kernelInitCudaPullSoAFp16, kernelDeinitCuda },
  { "cuda-push-soa-fp16", kernelInitCudaPushSoAFp16, kernelDeinitCuda },
  { "cuda-aa-soa-fp16", kernelInitCudaAaSoAFp16, kernelDeinitCuda },
};
const int LBM_B200_N_KERNELS = (int)(sizeof(LbmB200Kernels) / sizeof(LbmB200Kernels[0]));
