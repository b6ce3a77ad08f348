/* Host services of liblbmb200 (no GPU needed): geometry generators and the
 * seeded initial state. Declared in include/lbm_b200.h. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <strings.h>

#include "lbm_b200.h"

#define Q 19

static const int CX[Q] = { 0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0 };
static const int CY[Q] = { 1, -1, 0, 0, 1, -1, 1, -1, 0, 1, 0, 0, -1, 0, -1, 1, 0, 0, 0 };
static const int CZ[Q] = { 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, 0 };

static double weight(int d)
{
  if (d == Q - 1)
    return 1.0 / 3.0;
  return (CX[d] * CX[d] + CY[d] * CY[d] + CZ[d] * CZ[d]) == 1 ? 1.0 / 18.0 : 1.0 / 36.0;
}

static long long lat(int nx, int ny, int x, int y, int z)
{
  return ((long long)z * ny + y) * nx + x;
}

/* Same geometries and the same rules as the reference's geometryCreate
 * (src/lbm.c:52-187): every cell starts as fluid; channel/pipe/blocks force
 * x-periodicity and fluid forces all three axes (src/lbm.c:96-102); each
 * non-periodic axis gets obstacle cells at index 0 and n-1
 * (src/lbm.c:104-129); pipe removes everything outside a circle of radius
 * min(ny,nz)/2 - 1 around the y-z centre (src/lbm.c:131-142); blocks-N
 * places N-cubes on a 2N checkerboard in y and z at x % 2N >= N
 * (src/lbm.c:143-156). */
int lbm_geometry_create(const char *type, int nx, int ny, int nz, int periodic[3], int *flags,
    long long counts[2])
{
  enum { BOX, CHANNEL, PIPE, BLOCKS, FLUID } kind;
  int nb = 8;
  if (!type || !periodic || !flags || nx <= 0 || ny <= 0 || nz <= 0)
    return LBM_ERR_ARG;
  if (strncasecmp(type, "channel", 7) == 0)
    kind = CHANNEL;
  else if (strncasecmp(type, "box", 3) == 0)
    kind = BOX;
  else if (strncasecmp(type, "pipe", 4) == 0)
    kind = PIPE;
  else if (strncasecmp(type, "blocks", 6) == 0) {
    kind = BLOCKS;
    if (strlen(type) > 7) {
      nb = atoi(type + 7);
      if (nb <= 0)
        nb = 8;
    }
  } else if (strncasecmp(type, "fluid", 5) == 0)
    kind = FLUID;
  else
    return LBM_ERR_ARG;

  if (kind == CHANNEL || kind == PIPE || kind == BLOCKS)
    periodic[0] = 1;
  else if (kind == FLUID)
    periodic[0] = periodic[1] = periodic[2] = 1;

  const long long n = (long long)nx * ny * nz;
  for (long long i = 0; i < n; ++i)
    flags[i] = 1;
  for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
      for (int x = 0; x < nx; ++x) {
        int wall = (!periodic[0] && (x == 0 || x == nx - 1)) ||
                   (!periodic[1] && (y == 0 || y == ny - 1)) ||
                   (!periodic[2] && (z == 0 || z == nz - 1));
        if (wall)
          flags[lat(nx, ny, x, y, z)] = 0;
      }
  if (kind == PIPE) {
    const double cy = ny / 2.0 - 0.5, cz = nz / 2.0 - 0.5;
    const double dmin = ny < nz ? ny : nz;
    const double r = dmin / 2 - 1;
    for (int z = 0; z < nz; ++z)
      for (int y = 0; y < ny; ++y)
        if ((z - cz) * (z - cz) + (y - cy) * (y - cy) >= r * r)
          for (int x = 0; x < nx; ++x)
            flags[lat(nx, ny, x, y, z)] = 0;
  } else if (kind == BLOCKS) {
    for (int z = 0; z < nz; ++z) {
      if ((z % (2 * nb)) < nb)
        continue;
      for (int y = 0; y < ny; ++y) {
        if ((y % (2 * nb)) < nb)
          continue;
        for (int x = 0; x < nx; ++x)
          if ((x % (2 * nb)) >= nb)
            flags[lat(nx, ny, x, y, z)] = 0;
      }
    }
  }
  if (counts) {
    long long fl = 0;
    for (long long i = 0; i < n; ++i)
      fl += flags[i] != 0;
    counts[0] = fl;
    counts[1] = n - fl;
  }
  return LBM_OK;
}

/* splitmix64 (Steele, Lea, Flood 2014): a 64-bit state advanced by the
 * golden-ratio increment and finalised by two xor-shift-multiply rounds. */
static uint64_t mix64(uint64_t z)
{
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

static uint64_t next64(uint64_t *state)
{
  *state += 0x9E3779B97F4A7C15ull;
  return mix64(*state);
}

/* uniform double in [0, 1) from the top 53 bits */
static double u01(uint64_t v) { return (double)(v >> 11) * (1.0 / 9007199254740992.0); }

int lbm_porous_channel(int nx, int ny, int nz, double solid_fraction, double rmin, double rmax,
    unsigned long long seed, int *flags, double *fraction_out, int *spheres_out)
{
  if (!flags || nx <= 0 || ny <= 0 || nz <= 0 || !(rmin > 0.0) || rmax < rmin ||
      !(solid_fraction >= 0.0 && solid_fraction < 0.95))
    return LBM_ERR_ARG;
  int periodic[3] = { 1, 0, 0 };
  long long counts[2];
  int rc = lbm_geometry_create("channel", nx, ny, nz, periodic, flags, counts);
  if (rc)
    return rc;
  const long long total = (long long)nx * ny * nz;
  long long solid = counts[1];
  uint64_t st = (uint64_t)seed;
  int spheres = 0;
  const long long max_spheres = 100000000LL;
  while ((double)solid < solid_fraction * (double)total && spheres < max_spheres) {
    const double cxs = u01(next64(&st)) * nx;
    const double cys = u01(next64(&st)) * ny;
    const double czs = u01(next64(&st)) * nz;
    const double r = rmin + (rmax - rmin) * u01(next64(&st));
    const int ir = (int)ceil(r);
    const double r2 = r * r;
    for (int dz = -ir - 1; dz <= ir + 1; ++dz) {
      const int z = (int)floor(czs) + dz;
      if (z < 0 || z >= nz)
        continue;
      const double ez = z - czs;
      for (int dy = -ir - 1; dy <= ir + 1; ++dy) {
        const int y = (int)floor(cys) + dy;
        if (y < 0 || y >= ny)
          continue;
        const double ey = y - cys;
        if (ez * ez + ey * ey > r2)
          continue;
        for (int dx = -ir - 1; dx <= ir + 1; ++dx) {
          int x = (int)floor(cxs) + dx;
          const double ex = x - cxs;
          if (ex * ex + ey * ey + ez * ez > r2)
            continue;
          x = ((x % nx) + nx) % nx; /* x is periodic */
          long long i = lat(nx, ny, x, y, z);
          if (flags[i]) {
            flags[i] = 0;
            ++solid;
          }
        }
      }
    }
    ++spheres;
  }
  if (fraction_out)
    *fraction_out = (double)solid / (double)total;
  if (spheres_out)
    *spheres_out = spheres;
  return LBM_OK;
}

int lbm_perturbed_equilibrium(int nx, int ny, int nz, const int *flags, unsigned long long seed,
    double amplitude, double rho, double *f)
{
  if (!flags || !f || nx <= 0 || ny <= 0 || nz <= 0)
    return LBM_ERR_ARG;
  const long long n = (long long)nx * ny * nz;
  double w[Q];
  for (int d = 0; d < Q; ++d)
    w[d] = weight(d);
#pragma omp parallel for schedule(static)
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z) {
        const long long c = ((long long)x * ny + y) * nz + z;
        if (!flags[lat(nx, ny, x, y, z)]) {
          for (int d = 0; d < Q; ++d)
            f[d * n + c] = 0.0;
          continue;
        }
        /* counter-based: each cell's draws depend only on (seed, cell) */
        uint64_t base = (uint64_t)seed ^ mix64((uint64_t)c * 0x9E3779B97F4A7C15ull + 1ull);
        double u[3];
        for (int k = 0; k < 3; ++k)
          u[k] = amplitude * (2.0 * u01(next64(&base)) - 1.0);
        const double usq = u[0] * u[0] + u[1] * u[1] + u[2] * u[2];
        for (int d = 0; d < Q; ++d) {
          const double cu = CX[d] * u[0] + CY[d] * u[1] + CZ[d] * u[2];
          f[d * n + c] = w[d] * (rho - 1.5 * usq + 3.0 * cu + 4.5 * cu * cu);
        }
      }
  return LBM_OK;
}
