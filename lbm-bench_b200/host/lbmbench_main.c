/* lbmbench-b200: command-line driver with LBM-Bench's flags and output
 * (src/main.c:34-189, src/cli.c:44-123), running the liblbmb200 CUDA
 * kernels through the drop-in registry (include/lbm_b200_dropin.h).
 *
 * Same flags as the reference: -d XxYxZ -g TYPE -i N -o OMEGA -f F -k NAME
 * -l -V -x -y -z -h. Additions:
 *   -g porous        porous channel: channel walls plus seeded spheres
 *   -S FRACTION      solid fraction of -g porous (default 0.2)
 *   -R RMIN:RMAX     sphere radii of -g porous (default 4:8)
 *   -s SEED          seed of -g porous (default 42)
 *   -L LAMBDA        TRT magic parameter (default 1/12, the reference's)
 *   -F 0|1           add the body force -f after every step (the reference
 *                    does so only in -DVERIFICATION builds; -V implies -F 1)
 * The reference's equilibrium initialisation for -V scales the
 * equilibrium by omega (src/lbm.c:799-801); -V forces omega = 1, where that
 * equals the plain equilibrium w_d rho used here.
 */
#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>
#include <unistd.h>

#include "lbm_b200.h"
#include "lbm_b200_dropin.h"

#define Q 19

static const int CX[Q] = { 0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0 };

#define HELPTEXT                                                                           \
  "Usage: lbmbench-b200 [options]\n"                                                       \
  "  -d XxYxZ             Geometry dimensions\n"                                           \
  "  -g TYPE              box|channel|pipe|blocks-N|fluid|porous\n"                        \
  "  -i N                 Number of iterations\n"                                          \
  "  -o V                 Relaxation parameter (omega)\n"                                  \
  "  -f V                 X-direction body force\n"                                        \
  "  -k NAME              Kernel to use\n"                                                 \
  "  -l                   List available kernels\n"                                        \
  "  -V                   Run verification\n"                                              \
  "  -x/-y/-z             Enable periodic BC in x/y/z\n"                                   \
  "  -S F -R A:B -s N     porous: solid fraction, sphere radii, seed\n"                    \
  "  -L V                 TRT magic parameter Lambda\n"                                    \
  "  -F 0|1               Apply the body force after every step\n"                         \
  "  -h                   Print this help\n"

static int parse_dims(const char *p, int dims[3])
{
  char *end;
  for (int a = 0; a < 3; ++a) {
    long v = strtol(p, &end, 10);
    if (v <= 0) {
      printf("ERROR: %c dimension must be > 0.\n", "XYZ"[a]);
      return 0;
    }
    dims[a] = (int)v;
    if (a < 2) {
      if (*end != 'x') {
        printf("ERROR: %c dimension is missing.\n", "XYZ"[a + 1]);
        return 0;
      }
      p = end + 1;
    }
  }
  return 1;
}

static double weight(int d)
{
  if (d == Q - 1)
    return 1.0 / 3.0;
  return (d < 4 || d == 8 || d == 13) ? 1.0 / 18.0 : 1.0 / 36.0;
}

/* average density over fluid cells through GetNode (src/lbm.c:928-947) */
static double average_density(LatticeDescType *ld, KernelDataType *kd)
{
  PdfType p[Q];
  double sum = 0.0;
  for (int z = 0; z < ld->Dims[2]; ++z)
    for (int y = 0; y < ld->Dims[1]; ++y)
      for (int x = 0; x < ld->Dims[0]; ++x) {
        if (!ld->Lattice[((long long)z * ld->Dims[1] + y) * ld->Dims[0] + x])
          continue;
        kd->GetNode(kd, x, y, z, p);
        double local = 0.0;
        for (int d = 0; d < Q; ++d)
          local += p[d];
        sum += local;
      }
  return sum / ld->nFluid;
}

/* Plane-Poiseuille check of the reference (src/lbm.c:964-1023): u_x on the
 * plane x = nx/2 (plus half the force) against F (R^2 - r^2) / (2 nu) across
 * z, averaged over the middle y rows; L2 norm of the relative error. */
static double verify(LatticeDescType *ld, KernelDataType *kd, double omega, double force)
{
  const int nx = ld->Dims[0], ny = ld->Dims[1], nz = ld->Dims[2];
  const double nu = (1.0 / omega - 0.5) / 3.0;
  double *ux = (double *)calloc((size_t)ny * nz, sizeof(double));
  PdfType p[Q];
  const int xp = nx / 2;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y) {
      if (!ld->Lattice[((long long)z * ny + y) * nx + xp])
        continue;
      kd->GetNode(kd, xp, y, z, p);
      double u = 0.0;
      for (int d = 0; d < Q; ++d)
        u += CX[d] * (double)p[d];
      ux[y * nz + z] = u + 0.5 * force;
    }
  const double center = ny / 2.0, rmax2 = (ny / 2.0 - 1.0) * (ny / 2.0 - 1.0);
  const int even = (ny % 2 == 0), y0 = (ny - even - 1) / 2;
  double dev = 0.0;
  for (int z = 0; z < nz; ++z) {
    const double r2 = (z - center + 0.5) * (z - center + 0.5);
    const double exact = r2 >= rmax2 ? 0.0 : force * (rmax2 - r2) / (2.0 * nu);
    const double got = even ? 0.5 * (ux[y0 * nz + z] + ux[(y0 + 1) * nz + z]) : ux[y0 * nz + z];
    if (exact != 0.0)
      dev += pow(fabs(exact - got) / exact, 2);
  }
  free(ux);
  const double err = sqrt(dev);
  printf("# Kernel validation: L2 error norm of relative error: %e\n", err);
  return err;
}

int main(int argc, char **argv)
{
  int dims[3] = { 20, 20, 20 }, periodic[3] = { 0, 0, 0 }, verifyRun = 0, iterations = 10;
  const char *geometry = "channel", *kernel = "cuda-aa-soa";
  double omega = 1.0, force = 1e-5, lambda = 1.0 / 12.0, solid = 0.2, rmin = 4.0, rmax = 8.0;
  unsigned long long seed = 42;
  int forceFlag = -1, opt;

  printf("LBM Benchmark Kernels (B200 CUDA), type: benchmark\n");
  while ((opt = getopt(argc, argv, "d:g:i:o:f:k:lVxyzhS:R:s:L:F:")) != -1) {
    switch (opt) {
    case 'd':
      if (!parse_dims(optarg, dims))
        exit(EXIT_FAILURE);
      break;
    case 'g': geometry = optarg; break;
    case 'i':
      iterations = (int)strtol(optarg, NULL, 0);
      if (iterations <= 0) {
        printf("ERROR: iterations must be > 0.\n");
        exit(EXIT_FAILURE);
      }
      break;
    case 'o': omega = strtod(optarg, NULL); break;
    case 'f': force = strtod(optarg, NULL); break;
    case 'k': kernel = optarg; break;
    case 'l':
      printf("Available kernels:\n");
      for (int j = 0; j < LBM_B200_N_KERNELS; ++j)
        printf("   %s\n", LbmB200Kernels[j].Name);
      exit(EXIT_SUCCESS);
    case 'V':
      verifyRun   = 1;
      omega       = 1.0;
      geometry    = "box";
      dims[0]     = dims[1] = dims[2] = 16;
      force       = 1e-5;
      iterations  = 1000;
      periodic[0] = periodic[1] = 1;
      periodic[2] = 0;
      printf("#\n# VERIFICATION: verifying flow profile of channel flow.\n#\n");
      break;
    case 'x': periodic[0] = 1; break;
    case 'y': periodic[1] = 1; break;
    case 'z': periodic[2] = 1; break;
    case 'S': solid = strtod(optarg, NULL); break;
    case 'R':
      if (sscanf(optarg, "%lf:%lf", &rmin, &rmax) != 2) {
        printf("ERROR: -R expects RMIN:RMAX.\n");
        exit(EXIT_FAILURE);
      }
      break;
    case 's': seed = strtoull(optarg, NULL, 0); break;
    case 'L': lambda = strtod(optarg, NULL); break;
    case 'F': forceFlag = atoi(optarg) ? 1 : 0; break;
    case 'h': printf(HELPTEXT); exit(EXIT_SUCCESS);
    default:
      printf("ERROR: unknown option.\n");
      printf(HELPTEXT);
      exit(EXIT_FAILURE);
    }
  }

  LatticeDescType ld;
  memset(&ld, 0, sizeof(ld));
  for (int a = 0; a < 3; ++a)
    ld.Dims[a] = dims[a];
  ld.nCells  = dims[0] * dims[1] * dims[2];
  ld.Lattice = (LatticeType *)malloc(sizeof(LatticeType) * (size_t)ld.nCells);
  if (!ld.Lattice) {
    printf("ERROR: host allocation failed\n");
    exit(EXIT_FAILURE);
  }
  long long counts[2];
  if (strncasecmp(geometry, "porous", 6) == 0) {
    double frac;
    int spheres;
    if (lbm_porous_channel(dims[0], dims[1], dims[2], solid, rmin, rmax, seed, ld.Lattice, &frac,
            &spheres) != LBM_OK) {
      printf("ERROR: bad porous geometry parameters.\n");
      exit(EXIT_FAILURE);
    }
    periodic[0] = 1;
    periodic[1] = periodic[2] = 0;
    ld.Name = "porous";
    counts[0] = 0;
    for (int i = 0; i < ld.nCells; ++i)
      counts[0] += ld.Lattice[i] != 0;
    counts[1] = ld.nCells - counts[0];
    printf("# porous channel: %d spheres, radii %g-%g, solid fraction %.4f, seed %llu\n",
        spheres, rmin, rmax, frac, seed);
  } else {
    if (lbm_geometry_create(geometry, dims[0], dims[1], dims[2], periodic, ld.Lattice, counts) !=
        LBM_OK) {
      printf("ERROR: unknown geometry type '%s'.\n", geometry);
      exit(EXIT_FAILURE);
    }
    ld.Name = geometry;
  }
  ld.nFluid    = (int)counts[0];
  ld.nObst     = (int)counts[1];
  ld.PeriodicX = periodic[0];
  ld.PeriodicY = periodic[1];
  ld.PeriodicZ = periodic[2];

  CaseDataType cd;
  cd.MaxIterations     = iterations;
  cd.RhoIn             = 1.0;
  cd.RhoOut            = 1.0;
  cd.Omega             = (PdfType)omega;
  cd.XForce            = (PdfType)force;
  cd.StatisticsModulus = 100;

  printf("#\n");
  printf("# - iterations:        %d\n", cd.MaxIterations);
  printf("# - geometry:\n");
  printf("#   type:              %s\n", ld.Name);
  printf("#   dimensions:        %d x %d x %d\n", ld.Dims[0], ld.Dims[1], ld.Dims[2]);
  printf("#   nodes total:       %10d\n", ld.nObst + ld.nFluid);
  printf("#   nodes fluid:       %10d\n", ld.nFluid);
  printf("#   nodes obstacles:   %10d\n", ld.nObst);
  printf("#   periodicity:       x: %d y: %d z: %d\n", ld.PeriodicX, ld.PeriodicY, ld.PeriodicZ);
  printf("# - flow:\n");
  printf("#   omega:             %f\n", omega);
  printf("#   Lambda:            %f\n", lambda);
  printf("#   rho in:            %e\n", 1.0);
  printf("#   rho out:           %e\n", 1.0);
  printf("#   body force:        %e (%s)\n", force,
      (verifyRun || forceFlag == 1) ? "applied" : "not applied");

  const KernelFunctionsType *kf = NULL;
  for (int j = 0; j < LBM_B200_N_KERNELS; ++j)
    if (!strcasecmp(kernel, LbmB200Kernels[j].Name)) {
      kf = &LbmB200Kernels[j];
      break;
    }
  if (!kf) {
    printf("ERROR: kernel \"%s\" not found.\n", kernel);
    return 1;
  }
  printf("#\n# - kernel:            %s\n#\n", kf->Name);

  lbmB200SetMagicParameter(lambda);
  lbmB200SetBodyForce((verifyRun || forceFlag == 1) ? 1 : 0);
  KernelDataType *kd = NULL;
  kf->Init(&ld, &kd, &cd);

  if (verifyRun) {
    /* equilibrium at rest with rho = 1 on every fluid cell */
    PdfType p[Q];
    for (int d = 0; d < Q; ++d)
      p[d] = (PdfType)weight(d);
    for (int z = 0; z < dims[2]; ++z)
      for (int y = 0; y < dims[1]; ++y)
        for (int x = 0; x < dims[0]; ++x)
          if (ld.Lattice[((long long)z * dims[1] + y) * dims[0] + x])
            kd->SetNode(kd, x, y, z, p);
  }

  printf("# starting kernel...\n");
  kd->Kernel(&ld, kd, &cd);

  printf("# iter: %4d   avg density: %e\n", cd.MaxIterations, average_density(&ld, kd));
  double err = -1.0;
  if (verifyRun)
    err = verify(&ld, kd, omega, force);

  const double duration = kd->Duration;
  const double gbytes   = kd->LoopBalance * ld.nFluid * (double)cd.MaxIterations / 1e9;
  const double perf     = (double)ld.nFluid * (double)cd.MaxIterations / duration / 1.0e6;
  kf->Deinit(&ld, &kd);

  printf("#\n");
  printf("# Evaluation Stats\n");
  printf("#   runtime:           \t%.3f s\n", duration);
  printf("#   iterations:        \t%d\n", cd.MaxIterations);
  printf("#   fluid cells:       \t%d\n", ld.nFluid);
  printf("# Derived metrics\n");
  printf("#   MEM data vol.:     \t%.2f GByte\n", gbytes);
  printf("#   MEM bandwidth:     \t%.2f GByte/s\n", gbytes / duration);
  printf("#   performance:       \t%.3f MFLUP/s\n", perf);
  printf("P:   %f MFLUP/s  d: %f s  iter: %d  fnodes: %f x1e6  geo: %s  kernel: %s\n", perf,
      duration, cd.MaxIterations, ld.nFluid / 1e6, geometry, kernel);

  int exitCode = 0;
  if (verifyRun) {
    printf("# VERIFICATION: deviation from analytical solution: %e\n", err);
    if (!(err <= 0.1)) {
      printf("# VERIFICATION FAILED.\n");
      exitCode = 1;
    } else {
      printf("# VERIFICATION SUCCEEDED.\n");
    }
  }
  free(ld.Lattice);
  return exitCode;
}
