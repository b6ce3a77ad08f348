/* Test infrastructure only: a thin driver around LBM-Bench's own, unmodified
 * C sources (src/lbm.c, src/kernel_*.c, src/timing.c, src/allocate.c), which
 * oracle/Makefile compiles straight from the reference tree into
 * oracle/_ref/. Nothing in the product links this file; tests, the golden
 * fixture generator and bench.py's CPU-baseline leg load the resulting
 * shared libraries through ctypes.
 *
 * The driver does what src/main.c:34-189 does for one run, but with the
 * lattice flags, the initial state and the parameters supplied by the
 * caller instead of the CLI:
 *   - builds a LatticeDescType from a flag array in latticeIndex order
 *     (x fastest, src/lbm.h:108-111) and counts fluid/obstacle cells the way
 *     geometryCreate does (src/lbm.c:162-186);
 *   - looks the kernel up by name in GKernels[] (src/main.c:93-99) and calls
 *     its Init (src/lbm.c:601-658);
 *   - injects the caller's populations f_d(x) for every fluid cell through
 *     kd->SetNode (src/lbm.c:193-294), i.e. in the kernel's own orientation;
 *   - runs kd->Kernel (src/main.c:133), which times itself into kd->Duration;
 *   - reads every fluid cell back through kd->GetNode and calls Deinit.
 *
 * Host state layout on both sides of this driver: f[d][x][y][z], z fastest,
 * no padding, (nx*ny*nz) doubles per direction; obstacle entries are ignored
 * on input and left untouched on output.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "lbm.h"

#ifdef _OPENMP
#include <omp.h>
#endif

static long long dense_index(int nx, int ny, int nz, int x, int y, int z)
{
  return ((long long)x * ny + y) * nz + z;
}

/* Number of kernels in the reference's registry and their names, so the
 * Python side can iterate the same list the reference's -l prints
 * (src/cli.c:79-83). */
int ref_n_kernels(void) { return G_N_KERNELS; }

const char *ref_kernel_name(int i)
{
  if (i < 0 || i >= G_N_KERNELS)
    return NULL;
  return GKernels[i].Name;
}

int ref_pdf_size(void) { return (int)sizeof(PdfType); }

int ref_max_threads(void)
{
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Calls the reference's geometryCreate (src/lbm.c:52-187) and copies its flag
 * array out. counts = {nFluid, nObst}; periodic_out gets the periodicity that
 * geometryCreate forces for channel/pipe/blocks/fluid (src/lbm.c:96-102). */
int ref_geometry(const char *type, int nx, int ny, int nz, const int periodic_in[3],
    int *flags_out, int periodic_out[3], int counts[2])
{
  int dims[3]     = { nx, ny, nz };
  int periodic[3] = { periodic_in[0], periodic_in[1], periodic_in[2] };
  LatticeDescType ld;
  geometryCreate(type, dims, periodic, &ld);
  memcpy(flags_out, ld.Lattice, sizeof(int) * (size_t)nx * ny * nz);
  periodic_out[0] = ld.PeriodicX;
  periodic_out[1] = ld.PeriodicY;
  periodic_out[2] = ld.PeriodicZ;
  counts[0]       = ld.nFluid;
  counts[1]       = ld.nObst;
  free(ld.Lattice);
  return 0;
}

/* One run of reference kernel `name`.
 * flags: nx*ny*nz ints in latticeIndex order (LAT_CELL_* values).
 * pdfs_in / pdfs_out: 19*nx*ny*nz doubles in f[d][x][y][z] order.
 * inject == 0 leaves the lattice as Init left it (all zeros, as the
 * reference's benchmark build does, src/main.c:112-117).
 * Returns 0 on success, -1 if the kernel name is unknown. */
int ref_run(const char *name, int nx, int ny, int nz, const int *flags, int px, int py,
    int pz, double omega, double xforce, int iterations, int inject, const double *pdfs_in,
    double *pdfs_out, double *duration, int *iteration_out, int *n_bounce_back)
{
  KernelFunctionsType *kf = NULL;
  for (int j = 0; j < G_N_KERNELS; ++j)
    if (!strcasecmp(name, GKernels[j].Name)) {
      kf = &GKernels[j];
      break;
    }
  if (kf == NULL)
    return -1;

  LatticeDescType ld;
  memset(&ld, 0, sizeof(ld));
  ld.Dims[0]   = nx;
  ld.Dims[1]   = ny;
  ld.Dims[2]   = nz;
  ld.nCells    = nx * ny * nz;
  ld.PeriodicX = px;
  ld.PeriodicY = py;
  ld.PeriodicZ = pz;
  ld.Name      = "harness";
  ld.Lattice   = (LatticeType *)malloc(sizeof(LatticeType) * (size_t)ld.nCells);
  memcpy(ld.Lattice, flags, sizeof(LatticeType) * (size_t)ld.nCells);
  for (int i = 0; i < ld.nCells; ++i) {
    if (flags[i] == LAT_CELL_OBSTACLE)
      ld.nObst++;
    else
      ld.nFluid++;
  }

  CaseDataType cd;
  cd.Omega             = (PdfType)omega;
  cd.RhoIn             = (PdfType)1.0;
  cd.RhoOut            = (PdfType)1.0;
  cd.XForce            = (PdfType)xforce;
  cd.MaxIterations     = iterations;
  cd.StatisticsModulus = 100;

  KernelDataType *kd = NULL;
  kf->Init(&ld, &kd, &cd);
  if (n_bounce_back)
    *n_bounce_back = kd->nBounceBackPdfs;

  PdfType pdfs[N_D3Q19];
  if (inject) {
    for (int x = 0; x < nx; ++x)
      for (int y = 0; y < ny; ++y)
        for (int z = 0; z < nz; ++z) {
          if (flags[latticeIndex(ld.Dims, x, y, z)] == LAT_CELL_OBSTACLE)
            continue;
          for (int d = 0; d < N_D3Q19; ++d)
            pdfs[d] = (PdfType)pdfs_in[(long long)d * ld.nCells +
                                       dense_index(nx, ny, nz, x, y, z)];
          kd->SetNode(kd, x, y, z, pdfs);
        }
  }

  kd->Kernel(&ld, kd, &cd);

  if (duration)
    *duration = kd->Duration;
  if (iteration_out)
    *iteration_out = kd->Iteration;

  if (pdfs_out) {
    for (int x = 0; x < nx; ++x)
      for (int y = 0; y < ny; ++y)
        for (int z = 0; z < nz; ++z) {
          if (flags[latticeIndex(ld.Dims, x, y, z)] == LAT_CELL_OBSTACLE)
            continue;
          kd->GetNode(kd, x, y, z, pdfs);
          for (int d = 0; d < N_D3Q19; ++d)
            pdfs_out[(long long)d * ld.nCells + dense_index(nx, ny, nz, x, y, z)] =
                (double)pdfs[d];
        }
  }

  kf->Deinit(&ld, &kd);
  free(ld.Lattice);
  return 0;
}

/* ref_run with the reference's Zou-He pressure boundary
 * (kernelComputeBoundaryConditions, src/lbm.c:676-785) applied after every
 * kd->Kernel call of one iteration: one step for pull and push, two for AA
 * (src/kernel_aa_soa.c:36 runs iterations in pairs). `calls` kernel calls
 * are made. flags carry 2 (inlet, x = 0) and 4 (outlet, x = nx-1). */
int ref_run_pressure(const char *name, int nx, int ny, int nz, const int *flags, int px, int py,
    int pz, double omega, double xforce, double rho_in, double rho_out, int calls,
    const double *pdfs_in, double *pdfs_out)
{
  KernelFunctionsType *kf = NULL;
  for (int j = 0; j < G_N_KERNELS; ++j)
    if (!strcasecmp(name, GKernels[j].Name)) {
      kf = &GKernels[j];
      break;
    }
  if (kf == NULL)
    return -1;
  LatticeDescType ld;
  memset(&ld, 0, sizeof(ld));
  ld.Dims[0]   = nx;
  ld.Dims[1]   = ny;
  ld.Dims[2]   = nz;
  ld.nCells    = nx * ny * nz;
  ld.PeriodicX = px;
  ld.PeriodicY = py;
  ld.PeriodicZ = pz;
  ld.Name      = "harness";
  ld.Lattice   = (LatticeType *)malloc(sizeof(LatticeType) * (size_t)ld.nCells);
  memcpy(ld.Lattice, flags, sizeof(LatticeType) * (size_t)ld.nCells);
  for (int i = 0; i < ld.nCells; ++i) {
    if (flags[i] == LAT_CELL_OBSTACLE)
      ld.nObst++;
    else
      ld.nFluid++;
    ld.nInlet += flags[i] == LAT_CELL_INLET;
    ld.nOutlet += flags[i] == LAT_CELL_OUTLET;
  }
  CaseDataType cd;
  cd.Omega             = (PdfType)omega;
  cd.RhoIn             = (PdfType)rho_in;
  cd.RhoOut            = (PdfType)rho_out;
  cd.XForce            = (PdfType)xforce;
  cd.MaxIterations     = 1;
  cd.StatisticsModulus = 100;
  KernelDataType *kd = NULL;
  kf->Init(&ld, &kd, &cd);
  PdfType pdfs[N_D3Q19];
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        if (flags[latticeIndex(ld.Dims, x, y, z)] == LAT_CELL_OBSTACLE)
          continue;
        for (int d = 0; d < N_D3Q19; ++d)
          pdfs[d] = (PdfType)pdfs_in[(long long)d * ld.nCells + dense_index(nx, ny, nz, x, y, z)];
        kd->SetNode(kd, x, y, z, pdfs);
      }
  for (int c = 0; c < calls; ++c) {
    kd->Kernel(&ld, kd, &cd);
    // pull and push start every call from Pdfs[0] (src/kernel_pull_soa.c:35-36):
    // make the lattice the call ended in the next call's source
    if (kd->PdfsActive != kd->Pdfs[0]) {
      PdfType *t = kd->Pdfs[0];
      kd->Pdfs[0] = kd->Pdfs[1];
      kd->Pdfs[1] = t;
    }
    kernelComputeBoundaryConditions(kd, &ld, &cd);
  }
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        if (flags[latticeIndex(ld.Dims, x, y, z)] == LAT_CELL_OBSTACLE)
          continue;
        kd->GetNode(kd, x, y, z, pdfs);
        for (int d = 0; d < N_D3Q19; ++d)
          pdfs_out[(long long)d * ld.nCells + dense_index(nx, ny, nz, x, y, z)] = (double)pdfs[d];
      }
  kf->Deinit(&ld, &kd);
  free(ld.Lattice);
  return 0;
}

/* The reference's Poiseuille check (src/lbm.c:964-1023) on a state supplied
 * by the caller: the state is injected into an AA kernel's lattice (natural
 * orientation, Iteration = -1) and kernelVerify is called on it. */
int ref_verify(int nx, int ny, int nz, const int *flags, int px, int py, int pz, double omega,
    double xforce, const double *pdfs, double *error_norm)
{
  LatticeDescType ld;
  memset(&ld, 0, sizeof(ld));
  ld.Dims[0]   = nx;
  ld.Dims[1]   = ny;
  ld.Dims[2]   = nz;
  ld.nCells    = nx * ny * nz;
  ld.PeriodicX = px;
  ld.PeriodicY = py;
  ld.PeriodicZ = pz;
  ld.Lattice   = (LatticeType *)malloc(sizeof(LatticeType) * (size_t)ld.nCells);
  memcpy(ld.Lattice, flags, sizeof(LatticeType) * (size_t)ld.nCells);
  for (int i = 0; i < ld.nCells; ++i) {
    if (flags[i] == LAT_CELL_OBSTACLE)
      ld.nObst++;
    else
      ld.nFluid++;
  }
  CaseDataType cd;
  memset(&cd, 0, sizeof(cd));
  cd.Omega          = (PdfType)omega;
  cd.XForce         = (PdfType)xforce;
  cd.RhoIn          = (PdfType)1.0;
  cd.RhoOut         = (PdfType)1.0;
  cd.MaxIterations  = 1;
  KernelDataType *kd = NULL;
  kernelInitAaSoA(&ld, &kd, &cd);
  PdfType p[N_D3Q19];
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        if (flags[latticeIndex(ld.Dims, x, y, z)] == LAT_CELL_OBSTACLE)
          continue;
        for (int d = 0; d < N_D3Q19; ++d)
          p[d] = (PdfType)pdfs[(long long)d * ld.nCells + dense_index(nx, ny, nz, x, y, z)];
        kd->SetNode(kd, x, y, z, p);
      }
  PdfType err = 0;
  kernelVerify(&ld, kd, &cd, &err);
  *error_norm = (double)err;
  kernelDeinit(&ld, &kd);
  free(ld.Lattice);
  return 0;
}

/* The reference's equilibrium initialisation (src/lbm.c:791-896), exactly as
 * main.c calls it under -V (src/main.c:113-116), read back per fluid cell. */
int ref_initial_state(const char *name, int nx, int ny, int nz, const int *flags, int px,
    int py, int pz, double omega, double *pdfs_out)
{
  KernelFunctionsType *kf = NULL;
  for (int j = 0; j < G_N_KERNELS; ++j)
    if (!strcasecmp(name, GKernels[j].Name)) {
      kf = &GKernels[j];
      break;
    }
  if (kf == NULL)
    return -1;
  LatticeDescType ld;
  memset(&ld, 0, sizeof(ld));
  ld.Dims[0]   = nx;
  ld.Dims[1]   = ny;
  ld.Dims[2]   = nz;
  ld.nCells    = nx * ny * nz;
  ld.PeriodicX = px;
  ld.PeriodicY = py;
  ld.PeriodicZ = pz;
  ld.Lattice   = (LatticeType *)malloc(sizeof(LatticeType) * (size_t)ld.nCells);
  memcpy(ld.Lattice, flags, sizeof(LatticeType) * (size_t)ld.nCells);
  for (int i = 0; i < ld.nCells; ++i) {
    if (flags[i] == LAT_CELL_OBSTACLE)
      ld.nObst++;
    else
      ld.nFluid++;
  }
  CaseDataType cd;
  memset(&cd, 0, sizeof(cd));
  cd.Omega  = (PdfType)omega;
  cd.RhoIn  = (PdfType)1.0;
  cd.RhoOut = (PdfType)1.0;
  KernelDataType *kd = NULL;
  kf->Init(&ld, &kd, &cd);
  kernelSetInitialDensity(&ld, kd, &cd);
  kernelSetInitialVelocity(&ld, kd, &cd);
  PdfType p[N_D3Q19];
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        if (flags[latticeIndex(ld.Dims, x, y, z)] == LAT_CELL_OBSTACLE)
          continue;
        kd->GetNode(kd, x, y, z, p);
        for (int d = 0; d < N_D3Q19; ++d)
          pdfs_out[(long long)d * ld.nCells + dense_index(nx, ny, nz, x, y, z)] = (double)p[d];
      }
  kf->Deinit(&ld, &kd);
  free(ld.Lattice);
  return 0;
}
