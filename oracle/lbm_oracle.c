/* Test infrastructure only (never linked into the product): plain C
 * restatement of the LBM-Bench D3Q19 TRT step, written in the receiver view.
 *
 * One step, for every fluid cell x (src/kernel_pull_soa.c:94-199 computes
 * the same update in pull form, src/kernel_push_soa.c:94-199 in push form,
 * src/kernel_aa_soa.c:42-274 as two in-place half steps):
 *   1. moments of the cell's populations f_d(x): u = sum c_d f_d,
 *      rho = sum f_d, in the reference's summation order
 *      (src/kernel_pull_soa.c:118-128);
 *   2. TRT relaxation of the centre and of the nine (d, inv d) pairs
 *      (src/kernel_pull_soa.c:131-198) with
 *      omegaOdd = 1 / (1/2 + Lambda / (1/omega - 1/2)) (src/kernel_pull_soa.c:21);
 *      the reference hard-codes Lambda = 1/12 (src/kernel_pull_soa.c:20), here
 *      it is a parameter;
 *   3. streaming of out_d(x) to the neighbour x + c_d, wrapped on periodic
 *      axes; if that neighbour is an obstacle (or lies outside a
 *      non-periodic axis), link-wise half-way bounce-back returns it to
 *      x as direction inv d, which is what the bounce-back index lists of
 *      src/lbm.c:465-568 and the copy loops at src/kernel_pull_soa.c:203-204
 *      achieve;
 *   4. the Luo body force (src/lbm.c:902-922), f_d += ((3 w_d) c_dx) F, on
 *      every population a fluid cell receives, when force_on is set
 *      (the reference applies it only in -DVERIFICATION builds,
 *      src/kernel_pull_soa.c:206-209).
 * Every floating-point operation is the reference's, in the reference's
 * order, so with -ffp-contract=off the result is bit-identical to the
 * reference's pull, push and AA kernels compiled the same way.
 *
 * A fluid cell on a non-periodic face of the box (never produced by the
 * reference's geometries, whose non-periodic faces are obstacle cells,
 * src/lbm.c:104-129) sees the outside as a wall here. The reference instead
 * reads an unmaintained ghost cell there; that case is outside the parity
 * contract.
 */
#include "lbm_oracle.h"

#include <stdlib.h>
#include <string.h>

#define Q 19

/* D3Q19 velocity set and inverse map in the reference's direction order
 * N,S,E,W,NE,SE,NW,SW,T,TN,TE,TW,TS,B,BS,BN,BW,BE,C (src/lbm.h:20-38,
 * src/lbm.c:20-29); the order fixes the SoA plane order. */
static const int CX[Q]  = { 0, 0, 1, -1, 1, 1, -1, -1, 0, 0, 1, -1, 0, 0, 0, 0, -1, 1, 0 };
static const int CY[Q]  = { 1, -1, 0, 0, 1, -1, 1, -1, 0, 1, 0, 0, -1, 0, -1, 1, 0, 0, 0 };
static const int CZ[Q]  = { 0, 0, 0, 0, 0, 0, 0, 0, 1, 1, 1, 1, 1, -1, -1, -1, -1, -1, 0 };
static const int INV[Q] = { 1, 0, 3, 2, 7, 6, 5, 4, 13, 14, 16, 17, 15, 8, 9, 12, 10, 11, 18 };

enum { N_ = 0, S_, E_, W_, NE_, SE_, NW_, SW_, T_, TN_, TE_, TW_, TS_, B_, BS_, BN_, BW_, BE_, C_ };

typedef struct {
  double omegaEven, omegaOdd;
  double w0, w1, w2, w1X3, w1NineHalf, w2X3, w2NineHalf;
  double force[Q];
  int force_on;
  double alpha; /* Brinkman scale; 0 disables the term */
} Params;

static void make_params(Params *p, double omega, double lambda, double xforce, int force_on,
    double alpha)
{
  /* src/kernel_pull_soa.c:18-28 */
  p->omegaEven  = omega;
  p->omegaOdd   = 1.0 / (0.5 + lambda / (1.0 / omega - 0.5));
  p->w0         = 1.0 / 3.0;
  p->w1         = 1.0 / 18.0;
  p->w2         = 1.0 / 36.0;
  p->w1X3       = p->w1 * 3.0;
  p->w1NineHalf = p->w1 * 9.0 / 2.0;
  p->w2X3       = p->w2 * 3.0;
  p->w2NineHalf = p->w2 * 9.0 / 2.0;
  /* src/lbm.c:904-919: ((3 * w[d]) * c_dx) * F */
  const double w[Q] = { p->w1, p->w1, p->w1, p->w1, p->w2, p->w2, p->w2, p->w2, p->w1, p->w2,
    p->w2, p->w2, p->w2, p->w1, p->w2, p->w2, p->w2, p->w2, p->w0 };
  for (int d = 0; d < Q; ++d)
    p->force[d] = 3.0 * w[d] * (double)CX[d] * xforce;
  p->force_on = force_on;
  p->alpha    = alpha;
}

/* One cell's collision. f: populations before collision, out: after.
 * kappa is the Brinkman coefficient of this cell (0 when unused). The
 * Brinkman force F_b = -kappa u adds 3 w_d c_d . F_b = -kappa (c_d . u) 3 w_d
 * to direction d, i.e. -bterm to the first member of each pair and +bterm
 * to the second. Outputs u (momentum) for the adjoint. */
static void collide(const Params *p, const double *f, double *out, double kappa, double *u3)
{
  double pdfN = f[N_], pdfS = f[S_], pdfE = f[E_], pdfW = f[W_];
  double pdfNE = f[NE_], pdfSE = f[SE_], pdfNW = f[NW_], pdfSW = f[SW_];
  double pdfT = f[T_], pdfTN = f[TN_], pdfTE = f[TE_], pdfTW = f[TW_], pdfTS = f[TS_];
  double pdfB = f[B_], pdfBS = f[BS_], pdfBN = f[BN_], pdfBW = f[BW_], pdfBE = f[BE_];
  double pdfC = f[C_];

  double ux = pdfE + pdfNE + pdfSE + pdfTE + pdfBE - pdfW - pdfNW - pdfSW - pdfTW - pdfBW;
  double uy = pdfN + pdfNE + pdfNW + pdfTN + pdfBN - pdfS - pdfSE - pdfSW - pdfTS - pdfBS;
  double uz = pdfT + pdfTE + pdfTW + pdfTN + pdfTS - pdfB - pdfBE - pdfBW - pdfBN - pdfBS;
  double dens = pdfC + pdfN + pdfE + pdfS + pdfW + pdfNE + pdfSE + pdfSW + pdfNW + pdfT +
                pdfTN + pdfTE + pdfTS + pdfTW + pdfB + pdfBN + pdfBE + pdfBS + pdfBW;
  double dirIndepTrm = dens - (ux * ux + uy * uy + uz * uz) * 3.0 / 2.0;
  if (u3) {
    u3[0] = ux;
    u3[1] = uy;
    u3[2] = uz;
  }

  const double oE = p->omegaEven, oO = p->omegaOdd;
  out[C_] = pdfC - oE * (pdfC - p->w0 * dirIndepTrm);

  double w1Indep = p->w1 * dirIndepTrm;
  double w2Indep = p->w2 * dirIndepTrm;
  double ui, evenPart, oddPart, bterm;

#define PAIR(A, B, UI, WNH, WX3, WIND)                                                      \
  ui       = (UI);                                                                          \
  evenPart = oE * (0.5 * (f[A] + f[B]) - ui * ui * (WNH) - (WIND));                         \
  oddPart  = oO * (0.5 * (f[A] - f[B]) - ui * (WX3));                                       \
  if (kappa != 0.0) {                                                                       \
    bterm  = kappa * ui * (WX3);                                                            \
    out[A] = f[A] - evenPart - oddPart - bterm;                                             \
    out[B] = f[B] - evenPart + oddPart + bterm;                                             \
  } else {                                                                                  \
    out[A] = f[A] - evenPart - oddPart;                                                     \
    out[B] = f[B] - evenPart + oddPart;                                                     \
  }

  PAIR(N_, S_, uy, p->w1NineHalf, p->w1X3, w1Indep);
  PAIR(E_, W_, ux, p->w1NineHalf, p->w1X3, w1Indep);
  PAIR(T_, B_, uz, p->w1NineHalf, p->w1X3, w1Indep);
  PAIR(NW_, SE_, -ux + uy, p->w2NineHalf, p->w2X3, w2Indep);
  PAIR(NE_, SW_, ux + uy, p->w2NineHalf, p->w2X3, w2Indep);
  PAIR(TW_, BE_, -ux + uz, p->w2NineHalf, p->w2X3, w2Indep);
  PAIR(TE_, BW_, ux + uz, p->w2NineHalf, p->w2X3, w2Indep);
  PAIR(TS_, BN_, -uy + uz, p->w2NineHalf, p->w2X3, w2Indep);
  PAIR(TN_, BS_, uy + uz, p->w2NineHalf, p->w2X3, w2Indep);
#undef PAIR
}

typedef struct {
  int nx, ny, nz, px, py, pz;
  long long ncells;
  unsigned char *fluid; /* dense, f's cell order */
} Grid;

static long long cidx(const Grid *g, int x, int y, int z)
{
  return ((long long)x * g->ny + y) * g->nz + z;
}

static int grid_init(Grid *g, int nx, int ny, int nz, const int *flags, int px, int py, int pz)
{
  if (nx <= 0 || ny <= 0 || nz <= 0 || !flags)
    return -1;
  g->nx     = nx;
  g->ny     = ny;
  g->nz     = nz;
  g->px     = px;
  g->py     = py;
  g->pz     = pz;
  g->ncells = (long long)nx * ny * nz;
  g->fluid  = (unsigned char *)malloc((size_t)g->ncells);
  if (!g->fluid)
    return -1;
  for (int x = 0; x < nx; ++x)
    for (int y = 0; y < ny; ++y)
      for (int z = 0; z < nz; ++z)
        g->fluid[cidx(g, x, y, z)] = flags[((long long)z * ny + y) * nx + x] != 0;
  return 0;
}

/* Receiver of direction d leaving (x,y,z): returns the dense index of the
 * neighbour, or -1 if the link bounces back. */
static long long receiver(const Grid *g, int x, int y, int z, int d)
{
  int a = x + CX[d], b = y + CY[d], c = z + CZ[d];
  if (a < 0 || a >= g->nx) {
    if (!g->px)
      return -1;
    a = (a + g->nx) % g->nx;
  }
  if (b < 0 || b >= g->ny) {
    if (!g->py)
      return -1;
    b = (b + g->ny) % g->ny;
  }
  if (c < 0 || c >= g->nz) {
    if (!g->pz)
      return -1;
    c = (c + g->nz) % g->nz;
  }
  long long n = cidx(g, a, b, c);
  return g->fluid[n] ? n : -1;
}

static void step(const Grid *g, const Params *p, const float *porosity, const double *src,
    double *dst, double *u_save)
{
  const long long nc = g->ncells;
#pragma omp parallel for schedule(static)
  for (int x = 0; x < g->nx; ++x) {
    double f[Q], out[Q], u3[3];
    for (int y = 0; y < g->ny; ++y)
      for (int z = 0; z < g->nz; ++z) {
        long long i = cidx(g, x, y, z);
        if (!g->fluid[i])
          continue;
        for (int d = 0; d < Q; ++d)
          f[d] = src[d * nc + i];
        double kappa = 0.0;
        if (porosity && p->alpha != 0.0)
          kappa = p->alpha * (1.0 - (double)porosity[i]);
        collide(p, f, out, kappa, u3);
        if (u_save) {
          u_save[i]          = u3[0];
          u_save[nc + i]     = u3[1];
          u_save[2 * nc + i] = u3[2];
        }
        for (int d = 0; d < Q; ++d) {
          long long r = receiver(g, x, y, z, d);
          if (r >= 0)
            dst[d * nc + r] = p->force_on ? out[d] + p->force[d] : out[d];
          else
            dst[INV[d] * nc + i] = p->force_on ? out[d] + p->force[INV[d]] : out[d];
        }
      }
  }
}

/* Zou-He pressure boundary after a step (src/lbm.c:676-785,
 * kernelComputeBoundaryConditions), in the receiver view: on the interior
 * rows (1 <= y <= ny-2, 1 <= z <= nz-2) of plane x = 0 every cell flagged 2
 * (LAT_CELL_INLET) gets the five populations that enter from x - 1 (E, NE,
 * SE, TE, BE) chosen so that its density is rho_in; on plane x = nx-1 every
 * cell flagged 4 (LAT_CELL_OUTLET) gets W, NW, SW, TW, BW for rho_out. The
 * operations are the reference's, in its order. */
enum { dN = 0, dS, dE, dW, dNE, dSE, dNW, dSW, dT, dTN, dTE, dTW, dTS, dB, dBS, dBN, dBW, dBE, dC };

static void pressure_bc(const Grid *g, const int *flags, double rho_in, double rho_out,
    double *f)
{
  const long long nc = g->ncells;
  const double third = 1.0 / 3.0, quarter = 1.0 / 4.0, sixth = 1.0 / 6.0;
  const double in_inv = 1.0 / rho_in, out_inv = 1.0 / rho_out;
  for (int z = 1; z < g->nz - 1; ++z)
    for (int y = 1; y < g->ny - 1; ++y) {
      for (int side = 0; side < 2; ++side) {
        const int x = side ? g->nx - 1 : 0;
        if (flags[((long long)z * g->ny + y) * g->nx + x] != (side ? 4 : 2))
          continue;
        double *p = f + cidx(g, x, y, z);
#define F_(d) p[(long long)(d) * nc]
        const double rest = F_(dC) + (F_(dT) + F_(dB) + F_(dS) + F_(dN)) +
            (F_(dTS) + F_(dBS) + F_(dTN) + F_(dBN));
        if (!side) {
          const double dens = rho_in;
          const double ux = 1.0 -
              (rest + 2.0 * (F_(dSW) + F_(dTW) + F_(dW) + F_(dBW) + F_(dNW))) * in_inv;
          const double ind = sixth * dens * ux;
          F_(dE)  = F_(dW) + third * dens * ux;
          F_(dNE) = F_(dSW) - quarter * (F_(dN) - F_(dS)) + ind;
          F_(dSE) = F_(dNW) + quarter * (F_(dN) - F_(dS)) + ind;
          F_(dTE) = F_(dBW) - quarter * (F_(dT) - F_(dB)) + ind;
          F_(dBE) = F_(dTW) + quarter * (F_(dT) - F_(dB)) + ind;
        } else {
          const double dens = rho_out;
          const double ux = -1.0 +
              (rest + 2.0 * (F_(dNE) + F_(dBE) + F_(dE) + F_(dTE) + F_(dSE))) * out_inv;
          const double ind = sixth * dens * ux;
          F_(dW)  = F_(dE) - third * dens * ux;
          F_(dSW) = F_(dNE) + quarter * (F_(dN) - F_(dS)) - ind;
          F_(dNW) = F_(dSE) - quarter * (F_(dN) - F_(dS)) - ind;
          F_(dBW) = F_(dTE) + quarter * (F_(dT) - F_(dB)) - ind;
          F_(dTW) = F_(dBE) - quarter * (F_(dT) - F_(dB)) - ind;
        }
#undef F_
      }
    }
}

static int run_common_bc(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, int force_on, double alpha,
    const float *porosity, int steps, const double *f_in, double *f_out, int bc_every,
    double rho_in, double rho_out);

static int run_common(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, int force_on, double alpha,
    const float *porosity, int steps, const double *f_in, double *f_out)
{
  return run_common_bc(nx, ny, nz, flags, px, py, pz, omega, lambda, xforce, force_on, alpha,
      porosity, steps, f_in, f_out, 0, 1.0, 1.0);
}

static int run_common_bc(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, int force_on, double alpha,
    const float *porosity, int steps, const double *f_in, double *f_out, int bc_every,
    double rho_in, double rho_out)
{
  Grid g;
  if (grid_init(&g, nx, ny, nz, flags, px, py, pz) != 0 || steps < 0 || !f_in || !f_out)
    return -1;
  Params p;
  make_params(&p, omega, lambda, xforce, force_on, alpha);
  size_t bytes = sizeof(double) * Q * (size_t)g.ncells;
  double *a = (double *)malloc(bytes), *b = (double *)malloc(bytes);
  if (!a || !b) {
    free(a);
    free(b);
    free(g.fluid);
    return -1;
  }
  memcpy(a, f_in, bytes);
  memcpy(b, f_in, bytes);
  for (int s = 0; s < steps; ++s) {
    step(&g, &p, porosity, a, b, NULL);
    double *t = a;
    a         = b;
    b         = t;
    if (bc_every > 0 && (s + 1) % bc_every == 0)
      pressure_bc(&g, flags, rho_in, rho_out, a);
  }
  memcpy(f_out, a, bytes);
  free(a);
  free(b);
  free(g.fluid);
  return 0;
}

int orc_run(int nx, int ny, int nz, const int *flags, int px, int py, int pz, double omega,
    double lambda, double xforce, int force_on, int steps, const double *f_in, double *f_out)
{
  return run_common(nx, ny, nz, flags, px, py, pz, omega, lambda, xforce, force_on, 0.0, NULL,
      steps, f_in, f_out);
}

int orc_run_brinkman(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, double alpha, const float *porosity, int steps,
    const double *f_in, double *f_out)
{
  return run_common(nx, ny, nz, flags, px, py, pz, omega, lambda, xforce, 1, alpha, porosity,
      steps, f_in, f_out);
}

double orc_objective(int nx, int ny, int nz, const int *flags, const double *f)
{
  Grid g;
  if (grid_init(&g, nx, ny, nz, flags, 0, 0, 0) != 0)
    return 0.0;
  const long long nc = g.ncells;
  double sum = 0.0;
  long long count = 0;
  int x = nx - 1;
  for (int y = 0; y < ny; ++y)
    for (int z = 0; z < nz; ++z) {
      long long i = cidx(&g, x, y, z);
      if (!g.fluid[i])
        continue;
      double ux = 0.0;
      for (int d = 0; d < Q; ++d)
        ux += (double)CX[d] * f[d * nc + i];
      sum += ux;
      ++count;
    }
  free(g.fluid);
  return count ? sum / (double)count : 0.0;
}

/* Transpose of one cell's collision Jacobian applied to mu (sensitivities
 * of the post-collision populations), written for the TRT + Brinkman map
 * of collide():
 *   out_a = f_a - w+ (f_a+f_b)/2 - w- (f_a-f_b)/2 + w+ w (4.5 ui^2 + D)
 *           + 3 w (w- - kappa) ui
 *   out_b = f_b - w+ (f_a+f_b)/2 + w- (f_a-f_b)/2 + w+ w (4.5 ui^2 + D)
 *           - 3 w (w- - kappa) ui
 *   out_C = f_C - w+ (f_C - w0 D),  D = rho - 1.5 |u|^2, ui = c_a . u.
 * Returns lambda_k = sum_d mu_d d out_d / d f_k and the porosity
 * sensitivity sum_d mu_d d out_d / d phi (d kappa / d phi = -alpha). */
static void collide_adjoint(const Params *p, const double *u, const double *mu, double kappa,
    double *lam, double *dphi)
{
  static const int PA[9] = { N_, E_, T_, NW_, NE_, TW_, TE_, TS_, TN_ };
  static const int PB[9] = { S_, W_, B_, SE_, SW_, BE_, BW_, BN_, BS_ };
  const double oE = p->omegaEven, oO = p->omegaOdd;
  double sD = oE * p->w0 * mu[C_];
  double gu[3] = { 0.0, 0.0, 0.0 };
  double g_phi = 0.0;
  for (int k = 0; k < Q; ++k)
    lam[k] = 0.0;
  lam[C_] = (1.0 - oE) * mu[C_];
  for (int q = 0; q < 9; ++q) {
    int a = PA[q], b = PB[q];
    double w  = (q < 3) ? p->w1 : p->w2;
    double ui = CX[a] * u[0] + CY[a] * u[1] + CZ[a] * u[2];
    double ms = mu[a] + mu[b], md = mu[a] - mu[b];
    lam[a] += (1.0 - 0.5 * oE - 0.5 * oO) * mu[a] + (0.5 * oO - 0.5 * oE) * mu[b];
    lam[b] += (1.0 - 0.5 * oE - 0.5 * oO) * mu[b] + (0.5 * oO - 0.5 * oE) * mu[a];
    sD += oE * w * ms;
    double sp = oE * 9.0 * w * ui * ms + 3.0 * w * (oO - kappa) * md;
    gu[0] += sp * CX[a];
    gu[1] += sp * CY[a];
    gu[2] += sp * CZ[a];
    g_phi += 3.0 * w * p->alpha * ui * md;
  }
  for (int i = 0; i < 3; ++i)
    gu[i] -= 3.0 * u[i] * sD;
  for (int k = 0; k < Q; ++k)
    lam[k] += sD + gu[0] * CX[k] + gu[1] * CY[k] + gu[2] * CZ[k];
  *dphi = g_phi;
}

int orc_adjoint_brinkman(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, double alpha, const float *porosity, int steps,
    const double *f_in, double *grad, double *j_out)
{
  Grid g;
  if (grid_init(&g, nx, ny, nz, flags, px, py, pz) != 0 || steps < 0 || !porosity || !grad)
    return -1;
  Params p;
  make_params(&p, omega, lambda, xforce, 1, alpha);
  const long long nc = g.ncells;
  size_t sbytes = sizeof(double) * Q * (size_t)nc;
  /* forward trajectory: states 0..steps and the momenta of steps 0..steps-1 */
  double *traj = (double *)malloc(sbytes * (size_t)(steps + 1));
  double *uall = (double *)malloc(sizeof(double) * 3 * (size_t)nc * (size_t)(steps ? steps : 1));
  double *lam  = (double *)calloc((size_t)Q * nc, sizeof(double));
  double *lam2 = (double *)calloc((size_t)Q * nc, sizeof(double));
  if (!traj || !uall || !lam || !lam2) {
    free(traj);
    free(uall);
    free(lam);
    free(lam2);
    free(g.fluid);
    return -1;
  }
  memcpy(traj, f_in, sbytes);
  for (int s = 0; s < steps; ++s) {
    memcpy(traj + (size_t)(s + 1) * Q * nc, traj + (size_t)s * Q * nc, sbytes);
    step(&g, &p, porosity, traj + (size_t)s * Q * nc, traj + (size_t)(s + 1) * Q * nc,
        uall + (size_t)s * 3 * nc);
  }
  if (j_out)
    *j_out = orc_objective(nx, ny, nz, flags, traj + (size_t)steps * Q * nc);

  /* seed: dJ/df_k at the final state */
  long long count = 0;
  for (int y = 0; y < ny; ++y)
    for (int z = 0; z < nz; ++z)
      count += g.fluid[cidx(&g, nx - 1, y, z)];
  for (int y = 0; y < ny && count; ++y)
    for (int z = 0; z < nz; ++z) {
      long long i = cidx(&g, nx - 1, y, z);
      if (!g.fluid[i])
        continue;
      for (int d = 0; d < Q; ++d)
        lam[d * nc + i] = (double)CX[d] / (double)count;
    }
  for (long long i = 0; i < nc; ++i)
    grad[i] = 0.0;

  for (int s = steps - 1; s >= 0; --s) {
    const double *u = uall + (size_t)s * 3 * nc;
    for (int x = 0; x < nx; ++x)
      for (int y = 0; y < ny; ++y)
        for (int z = 0; z < nz; ++z) {
          long long i = cidx(&g, x, y, z);
          if (!g.fluid[i])
            continue;
          double mu[Q], l[Q], uc[3] = { u[i], u[nc + i], u[2 * nc + i] }, dphi;
          for (int d = 0; d < Q; ++d) {
            long long r = receiver(&g, x, y, z, d);
            mu[d] = (r >= 0) ? lam[d * nc + r] : lam[INV[d] * nc + i];
          }
          double kappa = alpha * (1.0 - (double)porosity[i]);
          collide_adjoint(&p, uc, mu, kappa, l, &dphi);
          for (int d = 0; d < Q; ++d)
            lam2[d * nc + i] = l[d];
          grad[i] += dphi;
        }
    double *t = lam;
    lam       = lam2;
    lam2      = t;
  }
  free(traj);
  free(uall);
  free(lam);
  free(lam2);
  free(g.fluid);
  return 0;
}

int orc_run_pressure(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, int force_on, double rho_in, double rho_out,
    int bc_every, int steps, const double *f_in, double *f_out)
{
  if (bc_every < 1 || !(rho_in > 0.0) || !(rho_out > 0.0))
    return -1;
  return run_common_bc(nx, ny, nz, flags, px, py, pz, omega, lambda, xforce, force_on, 0.0, NULL,
      steps, f_in, f_out, bc_every, rho_in, rho_out);
}
