/* liblbmb200 - B200-native D3Q19 TRT lattice-Boltzmann solver, flat C ABI.
 *
 * Plain pointers and sizes only; every function returns an int status
 * (LBM_OK = 0, negative on error; lbm_last_error() gives the message) unless
 * stated otherwise. All solver state lives in device memory; the host arrays
 * below are read or written only by the calls that take them.
 *
 * Array conventions
 *   flags  int[nx*ny*nz] in LBM-Bench's latticeIndex order, x fastest
 *          (src/lbm.h:108-111): 0 = obstacle (LAT_CELL_OBSTACLE), any other
 *          value = fluid (LAT_CELL_FLUID/INLET/OUTLET, src/lbm.h:47-52).
 *   f      double[19*nx*ny*nz], f[((d*nx + x)*ny + y)*nz + z]: the
 *          population of direction d that cell (x,y,z) collides next, i.e.
 *          what the reference's kd->GetNode returns (src/lbm.c:193-294);
 *          z is the unit-stride axis as in the reference's indexSoA
 *          (src/lbm.h:113-116), without the ghost layer. Direction order
 *          N,S,E,W,NE,SE,NW,SW,T,TN,TE,TW,TS,B,BS,BN,BW,BE,C (src/lbm.h:20-38).
 *   cell arrays (porosity, moments, gradients): [nx*ny*nz], same cell order
 *          as one plane of f.
 *
 * Threading: a solver is driven by one host thread at a time; its GPU work
 * runs in order on the solver's own CUDA stream.
 */
#ifndef LBM_B200_H
#define LBM_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define LBM_OK 0
#define LBM_ERR_ARG (-1)       /* invalid argument or unsupported size */
#define LBM_ERR_CUDA (-2)      /* a CUDA runtime call failed */
#define LBM_ERR_ALLOC (-3)     /* device or pinned-host allocation failed */
#define LBM_ERR_NONFINITE (-4) /* the state holds NaN or Inf */
#define LBM_ERR_STATE (-5)     /* call not valid in the solver's current state */
#define LBM_ERR_NODEV (-6)     /* no CUDA device (the product has no CPU path) */
#define LBM_ERR_COMM (-7)      /* NCCL missing, or a communicator call failed */
#define LBM_ERR_TIMEOUT (-8)   /* a bounded wait on a peer ran out; the communicator was aborted */

/* Propagation patterns, numbered as the reference's PROP_* (src/lbm.h:148). */
#define LBM_PUSH 0
#define LBM_PULL 1
#define LBM_AA 2

/* Storage/arithmetic precision. F64: FP64 populations and arithmetic,
 * bit-identical to the reference. F32: FP32 arithmetic on shifted
 * populations f_d - w_d stored as FP32. F16: FP32 arithmetic, shifted
 * populations stored as FP16 scaled by a power of two. */
#define LBM_F64 0
#define LBM_F32 1
#define LBM_F16 2

typedef struct lbm_solver lbm_solver;

/* Creates a solver on the current CUDA device for an nx*ny*nz box with the
 * given flags and periodicity. The state starts at zero (as the reference's
 * Init leaves it, src/lbm.c:452-463). Replaces the reference's
 * kernelInitInternal (src/lbm.c:400-599) for the pull/push/AA SoA kernels:
 * instead of bounce-back index lists it builds one 32-bit link mask per
 * cell on the device. */
int lbm_create(lbm_solver **out, int nx, int ny, int nz, const int *flags, int periodic_x,
    int periodic_y, int periodic_z, int pattern, int precision);

/* One x-slab of a domain decomposed along x (x is the slowest axis of the
 * reference's indexSoA, src/lbm.h:113-116). `flags` holds nx + 2 planes in
 * x (x fastest): planes 0 and nx + 1 are the boundary planes of the left and
 * right neighbouring slabs (periodic wrap at the ends of the ring). They
 * become ghost planes: never updated here, filled and drained through the
 * halo functions below. y and z are as in lbm_create. No counterpart in the
 * reference (single-node OpenMP only). */
int lbm_create_slab(lbm_solver **out, int nx, int ny, int nz, const int *flags, int periodic_y,
    int periodic_z, int pattern, int precision);

/* The same slab in the compact layout (lbm_create_compact): the fluid cells
 * of its own planes and of both ghost planes are stored; the halo calls
 * exchange the same messages as for a dense slab (a solid cell sends 0). */
int lbm_create_slab_compact(lbm_solver **out, int nx, int ny, int nz, const int *flags,
    int periodic_y, int periodic_z, int pattern, int precision);

/* The same solver in the compact (fluid-only) layout: populations and link
 * masks are stored for fluid cells only, packed row by row in z order, so no
 * obstacle cell shares a memory sector with a fluid one and every byte moved
 * belongs to a fluid cell. The reference sweeps its dense box
 * (src/kernel_pull_soa.c:94-96) and has no such layout. Results are
 * identical to lbm_create's (FP64: bit for bit, like the reference); every
 * call below works on it except lbm_set_porosity / lbm_adjoint_gradient
 * (no Brinkman term). Slabs: lbm_create_slab_compact. */
int lbm_create_compact(lbm_solver **out, int nx, int ny, int nz, const int *flags,
    int periodic_x, int periodic_y, int periodic_z, int pattern, int precision);

/* 1 if the solver uses the compact layout, 0 if not, -1 for NULL. */
int lbm_is_compact(const lbm_solver *s);

/* The compact layout's index, built on the host (no GPU needed): fluid is
 * rows x pitch bytes (nonzero = fluid, z fastest, the first nz of each row
 * used). For each row and each 32-cell word w (W = (nz + 31) / 32 words per
 * row) bits[r*W + w] gets one bit per fluid z and base[r*W + w] the number
 * of fluid cells before it in row order, so the fluid cell (r, z) is stored
 * at base + popcount(bits & bits below z). *total gets the fluid count.
 * No counterpart in the reference. */
int lbm_compact_index(const unsigned char *fluid, long long rows, int nz, int pitch,
    unsigned int *bits, unsigned int *base, unsigned long long *total);

/* Frees everything the solver owns (src/lbm.c:660-670). NULL is a no-op. */
int lbm_destroy(lbm_solver *s);

/* Relaxation rate omega (src/main.c:46, -o), TRT magic parameter Lambda
 * (hard-coded 1/12 at src/kernel_pull_soa.c:20), body force F in x
 * (src/main.c:47, -f) and whether it is applied after every step (the
 * reference applies it only in -DVERIFICATION builds,
 * src/kernel_pull_soa.c:206-209). Defaults: 1.0, 1/12, 1e-5, 0. */
int lbm_set_params(lbm_solver *s, double omega, double lambda, double xforce, int force_on);

/* FP16 storage scale (power of two, default 16384). F16 solvers only;
 * only valid before the first lbm_set_state. */
int lbm_set_fp16_scale(lbm_solver *s, double scale);

/* Per-cell porosity phi in [0,1] (float[nx*ny*nz]) and Brinkman scale alpha:
 * every fluid cell's collision adds the resistance force
 * F_b = -alpha (1 - phi) j (j = momentum). alpha = 0 switches it off.
 * No counterpart in the reference. */
int lbm_set_porosity(lbm_solver *s, const float *porosity, double alpha);

/* Uploads / downloads the state (array f above). Obstacle entries are
 * ignored on upload and written as 0 on download. The solver keeps the
 * state in its pattern's own orientation (like the reference's
 * Get/SetNode, src/lbm.c:193-294) and converts on the way. */
int lbm_set_state(lbm_solver *s, const double *f);
int lbm_get_state(lbm_solver *s, double *f);

/* Checkpoint / resume on the host. lbm_save_state writes the state (as
 * lbm_get_state returns it, FP64) and the step count to a file;
 * lbm_load_state reads it into a solver of the same box, geometry (fluid
 * cell count) and pattern and continues from that step, so an AA solver
 * resumes in the right orientation. A solver of the same precision (and
 * FP16 scale) continues bit for bit; another precision converts. No
 * counterpart in the reference (it keeps no state between runs). */
int lbm_save_state(lbm_solver *s, const char *path);
int lbm_load_state(lbm_solver *s, const char *path);

/* Orientation of a state held in LBM-Bench's own padded SoA array
 * (indexSoA with a one-cell ghost layer, (nx+2)*(ny+2)*(nz+2) values per
 * direction, src/lbm.h:113-116): where kd->GetNode finds f_d(x)
 * (src/lbm.c:193-294). NATURAL: push kernels, AA before its first and
 * after every odd iteration; PULL: pull kernels; AA_EVEN: AA after an even
 * iteration. */
#define LBM_REF_NATURAL 0
#define LBM_REF_PULL 1
#define LBM_REF_AA_EVEN 2
/* OR into ref_orientation: the array is in the reference's AoS order
 * (indexAoS, src/lbm.h:118-121: the 19 values of a padded cell are
 * contiguous), as its pull-aos / push-aos kernels keep it. */
#define LBM_REF_AOS 16

/* Uploads / downloads the state from / to an array in the reference's
 * padded layout and the given orientation; elem_size 8 (PdfType double) or
 * 4 (float, the reference's PRECISION_SP build). Only the slots GetNode
 * reads for fluid cells are used; on download every other slot is set to 0.
 * Replaces the host-side SetNode/GetNode loops around a kd->Kernel call. */
int lbm_set_state_padded(lbm_solver *s, const void *pdfs, int elem_size, int ref_orientation);
int lbm_get_state_padded(lbm_solver *s, void *pdfs, int elem_size, int ref_orientation);

/* Zou-He pressure boundary (src/lbm.c:676-785, kernelComputeBoundaryConditions,
 * which LBM-Bench defines but never calls). With on = 1, after every step
 * the cells flagged 2 (LAT_CELL_INLET) on the plane x = 0 get the five
 * populations entering from x - 1 (E, NE, SE, TE, BE) that give them density
 * rho_in, and the cells flagged 4 (LAT_CELL_OUTLET) on x = nx-1 the five
 * entering from x + 1 (W, NW, SW, TW, BW) for rho_out; as in the reference
 * only the interior rows 1 <= y <= ny-2, 1 <= z <= nz-2 take part. The
 * FP64 state equals the reference's pull and push kernels each followed by
 * that function (the reference's AA kernel can only apply it after a pair
 * of steps; here it follows every step of every pattern). x should not be
 * periodic. LBM_ERR_STATE if the flags of lbm_create had no such cells; not
 * available on slab solvers or with lbm_adjoint_gradient. on = 0 turns it
 * off. */
int lbm_set_pressure_bc(lbm_solver *s, double rho_in, double rho_out, int on);

/* Halo exchange of slab solvers. lbm_halo_needs tells which exchanges the
 * next step takes (LBM_HALO_BEFORE: pull, AA odd; LBM_HALO_AFTER: push, AA
 * odd; none for an AA even step). lbm_halo_pack writes the two messages
 * (lbm_halo_bytes each) into device buffers, to_left for the left
 * neighbour and to_right for the right one; after the transport,
 * lbm_halo_unpack reads what the left and right neighbours sent. Both are
 * ordered on the solver's stream (lbm_stream). `when` is LBM_HALO_BEFORE
 * (before lbm_run(s, 1)) or LBM_HALO_AFTER (after it). */
#define LBM_HALO_BEFORE 1
#define LBM_HALO_AFTER 2
/* The pull state, and the AA state after an odd number of steps, keep
 * populations of a slab's boundary cells in the ghost planes
 * (lbm_halo_shifted returns 1). Then a LBM_HALO_BEFORE exchange must come
 * before reading the state (lbm_get_state, lbm_moments, lbm_mass_momentum,
 * lbm_compare), and a LBM_HALO_SCATTER exchange after lbm_set_state, which
 * sends those ghost slots to the neighbours' own planes. */
#define LBM_HALO_SCATTER 4
size_t lbm_halo_bytes(const lbm_solver *s);
int lbm_halo_needs(const lbm_solver *s);
int lbm_halo_shifted(const lbm_solver *s);
int lbm_halo_pack(lbm_solver *s, int when, void *to_left, void *to_right);
int lbm_halo_unpack(lbm_solver *s, int when, const void *from_left, const void *from_right);
/* The solver's CUDA stream (cudaStream_t), for ordering a transport on it. */
void *lbm_stream(const lbm_solver *s);

/* One step split into ranges of x planes, so that a slab's interior update
 * overlaps its halo exchange (no reference counterpart: LBM-Bench has no
 * decomposition). lbm_step_begin opens the step and forks a second stream
 * after the work queued on the solver's stream; lbm_step_planes launches
 * the step on the solver's own planes [x_begin, x_end) (0 <= x_begin <
 * x_end <= nx, each plane once per step) on the solver's stream (on_side =
 * 0) or on the second stream (on_side = 1); lbm_step_end checks that every
 * plane was launched, joins the second stream into the solver's stream and
 * advances the step. Halo packs and unpacks between begin and end run on
 * the solver's stream. For a slab the exchanged slots and the interior
 * planes 1 .. nx-2 touch disjoint memory: the interior can run on the side
 * stream while the solver's stream packs, exchanges and unpacks the BEFORE
 * messages, updates planes 0 and nx-1, and exchanges the AFTER messages.
 * Results are bit-identical to lbm_run(s, 1). While a step is open,
 * lbm_run, the state transfers and the adjoint return LBM_ERR_STATE. */
int lbm_step_begin(lbm_solver *s);
int lbm_step_planes(lbm_solver *s, int x_begin, int x_end, int on_side);
int lbm_step_end(lbm_solver *s);

/* Native ring of x-slabs: the halo exchange of lbm_create_slab solvers
 * between ring neighbours over NCCL point-to-point (send/recv of the
 * lbm_halo_pack messages, ordered on the solver's stream), with the step
 * loop - split steps, packs, transports, unpacks - issued from C, one ring
 * per rank and GPU. No counterpart in the reference (LBM-Bench has no
 * decomposition, src/main.c). NCCL is loaded when first needed (dlopen of
 * libnccl.so.2, or of the file named by the environment variable
 * LBM_B200_NCCL; a copy already loaded in the process is reused), so the
 * library does not depend on it.
 *
 * lbm_ring_unique_id fills the 128-byte id that rank 0 creates and every
 * rank passes to lbm_ring_create (broadcast it over any host channel); it
 * needs no GPU. lbm_ring_create: rank in [0, nranks), the ring's left
 * neighbour is rank - 1 and the right one rank + 1 (wrapped). With id NULL
 * and nranks 1 the slab is its own neighbour on both sides (an x-periodic
 * domain in one slab) and the messages move by device copies, without NCCL.
 * Every wait on the communicator or on the stream - its creation, each
 * exchange's group, lbm_ring_synchronize, and the run loop, which keeps at
 * most 32 steps queued - gives up after timeout_ms (0: 60000), aborts the
 * communicator (which ends NCCL kernels waiting for a peer) and returns
 * LBM_ERR_TIMEOUT; after that, or after LBM_ERR_COMM, every call but
 * lbm_ring_destroy returns LBM_ERR_STATE.
 *
 * lbm_ring_run enqueues `steps` steps with the exchanges that lbm_halo_needs
 * asks for. overlap = 1 splits each step (lbm_step_begin/_planes/_end): the
 * interior planes run on the solver's second stream while its own stream
 * exchanges and updates the boundary planes. lbm_ring_gather and
 * lbm_ring_scatter are the LBM_HALO_BEFORE / LBM_HALO_SCATTER exchanges that
 * lbm_halo_shifted states need before reading and after setting the state.
 * All ranks make the same calls in the same order. */
typedef struct lbm_ring lbm_ring;
#define LBM_RING_ID_BYTES 128
int lbm_ring_unique_id(unsigned char *id);
int lbm_ring_create(lbm_ring **out, lbm_solver *s, int rank, int nranks,
    const unsigned char *id, int timeout_ms);
int lbm_ring_run(lbm_ring *r, int steps, int overlap);
int lbm_ring_gather(lbm_ring *r);
int lbm_ring_scatter(lbm_ring *r);
int lbm_ring_synchronize(lbm_ring *r);
/* Exchanges issued so far (each one: a pack, one send and one receive per
 * neighbour, an unpack); -1 for NULL. */
long long lbm_ring_exchanges(const lbm_ring *r);
/* 1 if the messages travel over NCCL, 0 for the device-copy ring of one. */
int lbm_ring_uses_nccl(const lbm_ring *r);
int lbm_ring_destroy(lbm_ring *r);

/* Sets the state on the device to the seeded initial condition of
 * lbm_perturbed_equilibrium (identical values, no host array): for domains
 * whose FP64 host state would not fit in host memory. */
int lbm_init_equilibrium(lbm_solver *s, unsigned long long seed, double amplitude, double rho);

/* Free and total memory of the current CUDA device (cudaMemGetInfo). */
int lbm_device_memory(size_t *free_bytes, size_t *total_bytes);

/* Enqueues `steps` time steps on the solver's stream (asynchronous).
 * Replaces the time loop of kd->Kernel (src/kernel_pull_soa.c:44-214,
 * src/kernel_push_soa.c:44-214, src/kernel_aa_soa.c:36-286); an AA solver
 * runs single steps, so odd counts are allowed. */
int lbm_run(lbm_solver *s, int steps);
int lbm_synchronize(lbm_solver *s);

/* Runs `steps` steps between two CUDA events on the solver's stream, waits,
 * and returns the elapsed device time in milliseconds. */
int lbm_run_timed(lbm_solver *s, int steps, double *ms);

/* Runs `steps` steps with an event pair around every launch and returns, per
 * kernel kind (0 pull, 1 push, 2 AA even, 3 AA odd), the summed device time
 * (ms_sum[4]) and the launch count (count[4]); *region_ms (may be NULL) gets
 * the device time from the first launch's start to the last one's end. */
int lbm_time_launches(lbm_solver *s, int steps, double *ms_sum, int *count, double *region_ms);

/* Page-locks (pins) / releases a caller-owned host buffer so that the state
 * transfers of lbm_set_state / lbm_get_state run as DMA at full PCIe speed. */
int lbm_pin_host(void *ptr, size_t bytes);
int lbm_unpin_host(void *ptr);

/* Per-cell density and momentum (the reference's ux is the momentum,
 * src/kernel_pull_soa.c:118-126) into host arrays of nx*ny*nz doubles;
 * obstacle cells get 0. Any pointer may be NULL. */
int lbm_moments(lbm_solver *s, double *rho, double *ux, double *uy, double *uz);

/* FP64 totals over fluid cells: out[0] = mass, out[1..3] = momentum, with
 * a fixed-order (deterministic) reduction. *nonfinite (may be NULL) gets
 * the number of fluid cells holding a NaN/Inf population; if it is
 * non-zero the call returns LBM_ERR_NONFINITE after filling out.
 * kernelDensity (src/lbm.c:928-947) is out[0] / lbm_fluid_cells(). */
int lbm_mass_momentum(lbm_solver *s, double out[4], long long *nonfinite);

/* No counterpart in the reference. Same totals as lbm_mass_momentum, for a
 * caller that holds the populations itself and must not allocate device
 * memory: a plug-in inside a host application whose own caching allocator
 * already owns the GPU's memory (a cudaMalloc from the plug-in can fail or
 * fragment the pool behind the application's back), and control loops that
 * cannot afford the device-wide synchronisation cudaMalloc and cudaFree may
 * imply. This call allocates nothing: its scratch is a fixed array inside
 * the library that every GPU loading the library holds until exit
 * ((LBM_NOALLOC_MAX_PLANES + 1) rows of 6 doubles, 384 KiB).
 *   f      device pointer, double[19*nx*ny*nz] in the f[d][x][y][z] layout
 *   flags  device pointer, int[nx*ny*nz] in latticeIndex order, 0 = obstacle
 *   out    host double[4]: mass, momentum x, y, z over fluid cells (FP64)
 *   nonfinite  host, may be NULL: fluid cells holding NaN/Inf (if non-zero
 *          the call returns LBM_ERR_NONFINITE after filling out)
 *   stream cudaStream_t as void* (NULL = default stream). The call is
 *          synchronous: it copies the totals to the host and waits on that
 *          stream (cudaStreamSynchronize) before it returns.
 * f and flags must live on the device that is current at the call (the
 * scratch address is looked up for that device); a pointer on another
 * device is rejected with LBM_ERR_ARG.
 * Limit: nx <= LBM_NOALLOC_MAX_PLANES (one scratch row per x-plane); larger
 * boxes are rejected with LBM_ERR_ARG. One block sums each x-plane, so a
 * box with few x-planes (e.g. 8 x 1024 x 1024) runs on few SMs and takes
 * longer than lbm_mass_momentum; flags are read with a stride of nx ints
 * between neighbouring threads.
 * The first call on each device looks up the scratch's device address
 * (cudaGetSymbolAddress) with that device current; make that first call
 * before any stream capture is started on the device.
 * Calls share the scratch: every row a call reads it has written first, but
 * calls whose work overlaps on the GPU (two streams, two host threads) race
 * on the rows, so serialise them. */
#define LBM_NOALLOC_MAX_PLANES 8192
int lbm_mass_momentum_noalloc(const double *f, const int *flags, int nx, int ny, int nz,
    double out[4], long long *nonfinite, void *stream);

/* Difference of two solvers over the same geometry (the first is compared
 * against the second, e.g. an FP16 run against an FP64 run):
 * out[0] = sum |u_a - u_b|^2, out[1] = sum |u_b|^2,
 * out[2] = sum (rho_a - rho_b)^2, out[3] = sum rho_b^2,
 * out[4] = max |u_a - u_b|,     out[5] = max |u_b|  (u = momentum vector),
 * all over fluid cells, in FP64 on the device. */
int lbm_compare(lbm_solver *a, lbm_solver *b, double out[6]);

/* Objective J = mean over the fluid cells of the plane x = nx-1 of the x
 * momentum. No counterpart in the reference. */
int lbm_objective(lbm_solver *s, double *j);

/* Gradient of J (lbm_objective) after `steps` Brinkman steps from the
 * current state, with respect to the porosity field: the discrete adjoint
 * of the step, reverse in time. AA solvers with FP64 or FP32 storage and a
 * porosity field set (lbm_set_porosity). The forward sweep keeps a
 * checkpoint every `checkpoint_every` steps (0: the interval that minimises
 * checkpoint plus segment memory, about sqrt(steps * state / momentum);
 * LBM_CKPT_AUTO: the longest interval that fits in 90% of the free device
 * memory, up to `steps`, i.e. the least recomputation); the reverse sweep
 * recomputes each segment but the last once, saving the momentum of every
 * step (the forward sweep saves the last segment's), and runs the adjoint
 * steps over it. grad: double[nx*ny*nz] (0 on
 * obstacles); *j_out (may be NULL): J of the final state; info (may be NULL,
 * 6 doubles): forward ms, reverse ms (recomputation + adjoint), interval,
 * checkpoints, extra device bytes, peak device bytes. The solver's state is
 * left at the initial state. No counterpart in the reference. */
#define LBM_CKPT_AUTO (-1)
int lbm_adjoint_gradient(lbm_solver *s, int steps, int checkpoint_every, double *grad,
    double *j_out, double *info);

long long lbm_fluid_cells(const lbm_solver *s);
long long lbm_steps_done(const lbm_solver *s);
/* Device bytes the solver holds (state, masks, porosity, scratch). */
size_t lbm_device_bytes(const lbm_solver *s);
/* Algorithmic bytes moved per fluid lattice update: 2 * 19 * storage size. */
double lbm_bytes_per_update(const lbm_solver *s);
/* Number of step-kernel launches issued since creation. */
long long lbm_launch_count(const lbm_solver *s);

const char *lbm_last_error(void);
/* Number of visible CUDA devices (0 if none or no driver). */
int lbm_device_count(void);

/* ---- host services (no GPU needed) ---- */

/* LBM-Bench's geometries (src/lbm.c:52-187): "box", "channel", "pipe",
 * "blocks[-N]", "fluid". periodic[3] is read and updated (channel, pipe and
 * blocks force x-periodic, fluid forces all three). counts = {fluid,
 * obstacle}. flags as above. Returns LBM_ERR_ARG for an unknown type. */
int lbm_geometry_create(const char *type, int nx, int ny, int nz, int periodic[3], int *flags,
    long long counts[2]);

/* Porous channel: a "channel" (x-periodic, obstacle walls at y,z = 0 and
 * n-1) plus solid spheres with seeded uniform centres (x distance taken
 * periodically) and radii uniform in [rmin, rmax], added until the solid
 * fraction (obstacles / all cells, walls included) reaches solid_fraction.
 * No counterpart in the reference. */
int lbm_porous_channel(int nx, int ny, int nz, double solid_fraction, double rmin, double rmax,
    unsigned long long seed, int *flags, double *fraction_out, int *spheres_out);

/* Seeded initial state: equilibrium of the incompressible model
 * w_d (rho - 1.5 u.u + 3 c_d.u + 4.5 (c_d.u)^2) with density rho and
 * u ~ U(-amplitude, amplitude)^3 per fluid cell (splitmix64); obstacle
 * entries 0. */
int lbm_perturbed_equilibrium(int nx, int ny, int nz, const int *flags, unsigned long long seed,
    double amplitude, double rho, double *f);

#ifdef __cplusplus
}
#endif

#endif
