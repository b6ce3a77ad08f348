/* Test infrastructure only (never linked into the product): a plain C
 * restatement of LBM-Bench's D3Q19 TRT stream-collide-bounce-back step, used
 * by tests/ as the checker for the CUDA kernels. Pinned against the
 * reference's own sources (oracle/_ref) and the committed golden fixtures in
 * tests/golden/.
 *
 * State layout: f[d][x][y][z] doubles, z fastest, no padding; entry (d, x)
 * holds f_d(x), the population of direction d that cell x collides next
 * (what the reference's kd->GetNode returns, src/lbm.c:193-294).
 * Flags: nx*ny*nz ints in the reference's latticeIndex order (x fastest,
 * src/lbm.h:108-111); 0 = obstacle, anything else = fluid.
 */
#ifndef LBM_ORACLE_H
#define LBM_ORACLE_H

#ifdef __cplusplus
extern "C" {
#endif

/* Runs `steps` TRT steps. force_on = 1 adds the Luo body force after every
 * step like the reference's -DVERIFICATION build (src/lbm.c:902-922); 0 runs
 * the benchmark build's step (no force). Returns 0, or -1 on bad input. */
int orc_run(int nx, int ny, int nz, const int *flags, int px, int py, int pz, double omega,
    double lambda, double xforce, int force_on, int steps, const double *f_in, double *f_out);

/* Same step with a Brinkman resistance term: after collision every
 * population gets f_d += 3 w_d c_d . F_b with F_b = -alpha (1 - phi(x)) j(x),
 * j the momentum of the pre-collision populations. porosity is nx*ny*nz
 * floats in f's cell order (z fastest). With alpha = 0 this is orc_run. */
int orc_run_brinkman(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, double alpha, const float *porosity, int steps,
    const double *f_in, double *f_out);

/* orc_run with the Zou-He pressure boundary of src/lbm.c:676-785 applied
 * after every bc_every-th step: cells flagged 2 on plane x = 0 (inlet,
 * density rho_in) and 4 on plane x = nx-1 (outlet, rho_out), interior y/z
 * rows only. Returns 0, or -1 on bad input. */
int orc_run_pressure(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, int force_on, double rho_in, double rho_out,
    int bc_every, int steps, const double *f_in, double *f_out);

/* Objective J = mean over the fluid cells of plane x = nx-1 of the x
 * momentum sum_d c_dx f_d. */
double orc_objective(int nx, int ny, int nz, const int *flags, const double *f);

/* Discrete adjoint of orc_run_brinkman followed by orc_objective: writes
 * dJ/dphi for every cell (0 on obstacles) into grad (f's cell order), and
 * returns J through *j_out. Stores the whole forward trajectory; small
 * cases only. */
int orc_adjoint_brinkman(int nx, int ny, int nz, const int *flags, int px, int py, int pz,
    double omega, double lambda, double xforce, double alpha, const float *porosity, int steps,
    const double *f_in, double *grad, double *j_out);

#ifdef __cplusplus
}
#endif

#endif
