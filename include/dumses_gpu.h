/*
 * dumses_gpu.h -- C-ABI of libdumses_gpu, the sm_100a implementation of the
 * DUMSES-Hybrid (v2.2.0) second-order Godunov MHD step.
 *
 * The reference exposes this path as argument-less Fortran subroutines that
 * work on module globals (uin, dt, time, input_params).  Each entry point below
 * replaces one of them; the Fortran driver keeps its loop and calls these
 * through ISO_C_BINDING shims:
 *
 *   dg_init          <- init_param/allocate_workspace   src/subroutines/init.f90:18-71, 348-419
 *   dg_upload        <- !$acc data copy(uin)            src/dumses.f90:59
 *   dg_download      <- !$acc update host(uin)          src/dumses.f90:62,122,133,138,144
 *   dg_compute_dt    <- compute_dt(dt)                  src/subroutines/physics.f90:18-132
 *   dg_godunov       <- godunov                         src/subroutines/scheme.f90:104-189
 *   dg_fargo_update  <- fargo_update                    src/subroutines/fargo.f90:17-124
 *   dg_boundary      <- boundary                        src/subroutines/boundary.f90:18-92
 *   dg_dissipation   <- dissipation                     src/subroutines/physics.f90:272-664
 *   dg_history       <- history (MRI problem variant)   src/problem/mri/history.f90:19-174
 *   dg_history_variant <- history of the other problems  src/subroutines/history.f90:19-171 (NDIM 3)
 *   dg_step          <- one pass of the loop body       src/dumses.f90:82-120
 *   dg_finalize      <- deallocate_workspace            src/subroutines/finalize.f90
 *
 * Conventions
 *  - All host arrays use the reference's own layout: Fortran column-major
 *    uin(iu1:iu2, ju1:ju2, ku1:ku2, 1:11) with nghost = 3 ghost cells on each
 *    side of every active dimension (ju1=ju2=1 when ndim<2, ku1=ku2=1 when
 *    ndim<3).  Variables: 1 rho, 2-4 rho*v, 5 total energy, 6-8 B on the left
 *    x/y/z faces, 9-11 B on the right faces.
 *  - Every function returns DG_OK (0) or a negative DG_ERR_* code; the text of
 *    the last error of the calling thread is available from dg_last_error().
 *  - Calls are ordered on the context's CUDA stream.  dg_compute_dt,
 *    dg_download, dg_history and dg_sync wait for the stream with a bounded
 *    poll and return DG_ERR_TIMEOUT rather than block forever.
 *  - One host thread per context (the reference runs MPI_THREAD_FUNNELED).
 */
#ifndef DUMSES_GPU_H
#define DUMSES_GPU_H

#ifdef __cplusplus
extern "C" {
#endif

/* status codes */
#define DG_OK              0
#define DG_ERR_ARG        -1   /* invalid argument or parameter combination   */
#define DG_ERR_CUDA       -2   /* a CUDA runtime call failed                   */
#define DG_ERR_NOMEM      -3   /* device allocation failed                    */
#define DG_ERR_TIMEOUT    -4   /* a bounded wait on the device ran out        */
#define DG_ERR_STATE      -5   /* non-finite or non-physical state detected   */
#define DG_ERR_DT         -6   /* the CFL reduction gave dt <= 0 or non-finite */
#define DG_ERR_NODEVICE   -7   /* no CUDA device is visible                   */
#define DG_ERR_UNSUPPORTED -8  /* option the library does not implement       */

/* Riemann solver ids: the reference's own numbering (src/modules/commons.f90:98-105) */
#define DG_RIEMANN_LLF     2
#define DG_RIEMANN_HLL     3
#define DG_RIEMANN_HLLD    4
#define DG_RIEMANN_UPWIND  5
#define DG_RIEMANN_HLLA    8   /* 2D (EMF) solver only */

/* boundary types, one per direction (input_params bdtypex/y/z, commons.f90:123-126) */
#define DG_BC_PERIODIC      0
#define DG_BC_ZERO_GRADIENT 1
#define DG_BC_SHEARINGBOX   2  /* x only, ndim == 3 (boundary.f90:40-52) */

/* arithmetic of the step */
#define DG_PREC_FP64   0   /* plain path: bit-identical to the FP64 reference arithmetic */
#define DG_PREC_FP32   1   /* FP32 trace/Riemann/CT, compensated FP32 hi/lo state        */

/* POD mirror of the reference's &scheme_params / &model_params namelists
 * (src/subroutines/init.f90:153-173) plus the compile-time switches NDIM/ISO. */
typedef struct dg_params {
    int    ndim;             /* 1, 2 or 3 (reference NDIM; 1: FP64, slope_type <= 2,   */
                             /* no dissipation)                                        */
    int    iso;              /* 1: isothermal EOS (reference ISO=1), 0: adiabatic      */
    int    nx, ny, nz;       /* active cells (nz = 1 when ndim = 2, ny = nz = 1 when 1) */
    double xmin, xmax, ymin, ymax, zmin, zmax;
    double gamma;            /* ratio of specific heats                                */
    double ciso;             /* isothermal sound speed                                 */
    double omega0;           /* rotation rate; > 0 enables Coriolis + shear terms      */
    double courant;          /* CFL number                                             */
    int    slope_type;       /* 0 none, 1 minmod, 2 MC, 3 multi-D (scheme.f90:253-656) */
    int    iriemann;         /* 1D solver: LLF, HLL, HLLD, UPWIND                      */
    int    iriemann2d;       /* 2D solver: LLF, HLLD, UPWIND, HLLA                     */
    int    bc[3];            /* DG_BC_* per direction                                  */
    int    fargo;            /* 1: FARGO orbital advection after the Godunov step      */
    int    precision;        /* DG_PREC_*                                              */
    int    surrogate;        /* 1: learned flux surrogate with HLLD fallback (FP32)    */
    int    device;           /* CUDA device ordinal                                    */
    double nu;               /* kinematic viscosity (physics.f90:459-664); 0 = off     */
    double eta;              /* Ohmic resistivity (physics.f90:295-455); 0 = off       */
    /* z-slab decomposition (the reference's &mpi_params nzslice and the rank's
     * zposition, init.f90:159,190-197, parallel.f90:197-257), z only: nz is this
     * slab's share (nzglob = nz * nzslice), zmin/zmax bound the whole box, and the
     * slab's z ghost planes come from its neighbours (dg_halo_pack/unpack).
     * nzslice = 0 or 1: one domain. */
    int    nzslice;
    int    zposition;        /* 0 .. nzslice-1, from the bottom of the box             */
    int    reserved[4];
} dg_params;

typedef struct dg_ctx dg_ctx;

/* fill *p with the reference's default_parameters (init.f90:244-302) */
void dg_default_params(dg_params *p);

/* number of doubles in one host uin array: (nx+6)(ny+6)(nz+6) * 11 for ndim=3 */
long long dg_uin_size(const dg_params *p);

int  dg_init(const dg_params *p, dg_ctx **ctx);
int  dg_finalize(dg_ctx *ctx);
int  dg_upload(dg_ctx *ctx, const double *uin);
int  dg_download(dg_ctx *ctx, double *uin);

/* CFL step (physics.f90:18-132); returns dt to the host */
int  dg_compute_dt(dg_ctx *ctx, double *dt);
/* one Godunov update of the active cells with the given dt, at the given time (scheme.f90:104-189) */
int  dg_godunov(dg_ctx *ctx, double dt, double time);
/* FARGO shift of the state after the Godunov update (fargo.f90:17-124) */
int  dg_fargo_update(dg_ctx *ctx, double dt);
/* ghost fill, shear-periodic remap at time+dt (boundary.f90:18-92) */
int  dg_boundary(dg_ctx *ctx, double time, double dt);

/* dissipation (src/subroutines/physics.f90:272-664), called by the reference after
 * boundary when nu > 0 or eta > 0 (dumses.f90:104): Ohmic resistivity (edge EMFs
 * -eta J dt and constrained transport), Navier-Stokes viscosity (face fluxes of
 * momentum and, adiabatic, energy; conservative update), then boundary at
 * time + dt.  A no-op when nu = eta = 0. */
int  dg_dissipation(dg_ctx *ctx, double time, double dt);

/* Loop body of dumses.f90:82-120: compute_dt, godunov, fargo (if on), boundary,
 * dissipation (if nu > 0 or eta > 0), time += dt.  dt and time stay on the device; nsteps steps are enqueued without
 * any host synchronisation.  On return *time and *dt hold the values after the
 * last step (this waits for the stream). */
int  dg_run(dg_ctx *ctx, int nsteps, double *time, double *dt);
/* one step, as dg_run(ctx, 1, ...) */
int  dg_step(dg_ctx *ctx, double *time, double *dt);

/* Fortran 'binary' dumps: output (src/subroutines/output.f90:224-235, io_type =
 * 'binary') and restart (src/subroutines/restart.f90:212-221).  The file is an
 * unformatted sequential file as gfortran writes it (4-byte record markers; a
 * record over 2147483639 bytes split into subrecords with signed markers):
 *   record 1  int32  nx, ny, nz, nxslice, nyslice, nzslice   (slices = 1 here)
 *   record 2  double time, dt, dx, dy, dz
 *   record 3  double xmin, xmax, ymin, ymax, zmin, zmax
 *   record 4  double gamma, ciso
 *   record 5  double uin(iu1:iu2, ju1:ju2, ku1:ku2, 1:11) in the host layout above
 * The reference names the file output_NNNNNN/data.RRRRRR.bin (get_filename,
 * src/modules/file.f90); dumpy reads it (utils/dumpy/data/rd_dumses.py). */
typedef struct dg_dump_info {
    int       nx, ny, nz, nxslice, nyslice, nzslice;
    double    time, dt, dx, dy, dz;
    double    xmin, xmax, ymin, ymax, zmin, zmax;
    double    gamma, ciso;
    long long uin_bytes;     /* length of the uin record                               */
} dg_dump_info;

/* header of a dump, and the length of its uin record (no device needed) */
int  dg_dump_header(const char *path, dg_dump_info *info);
/* dump of the context's state, streamed from the device plane by plane through two
 * pinned buffers (the copy of one plane overlaps the file write of the previous
 * one); FP32 contexts write hi + lo.  time and dt go to record 2. */
int  dg_dump_write(dg_ctx *ctx, const char *path, double time, double dt);
/* restart: the dump must hold the context's grid, domain, gamma and ciso (else
 * DG_ERR_ARG) and one rank (else DG_ERR_UNSUPPORTED).  Loads the state (the
 * right-face B of vars 9-10 is derived, as dg_upload does) and returns time and
 * dt of record 2.  The ghost cells come from the file, as in the reference's
 * restart (init.f90:114-120 calls no boundary after restart_run). */
int  dg_dump_read(dg_ctx *ctx, const char *path, double *time, double *dt);
/* the same two operations on a host uin array of grid p (no device needed) */
int  dg_dump_write_host(const char *path, const dg_params *p, double time, double dt, const double *uin);
int  dg_dump_read_host(const char *path, const dg_params *p, double *time, double *dt, double *uin);

/* MRI history sums (src/problem/mri/history.f90:60-125) of the current state:
 * out[0] mass, out[1] maxwell, out[2] reynolds, out[3] maxwell+reynolds,
 * out[4] magp, out[5..7] <B>, out[8] divB.  FP64 sums in a fixed tree order. */
int  dg_history(dg_ctx *ctx, double out[9]);

/* The history sums of either history routine of the reference (the history.f90 of a
 * problem directory replaces the default one at link time): DG_HISTORY_MRI is dg_history;
 * DG_HISTORY_DEFAULT is src/subroutines/history.f90:57-125 (NDIM 3), used by the problems
 * without their own history, which takes the Maxwell stress of B_x and B_z and the Reynolds
 * stress of v_x and v_z about their y-z means.  Same output order and file format. */
#define DG_HISTORY_MRI     0
#define DG_HISTORY_DEFAULT 1
int  dg_history_variant(dg_ctx *ctx, int variant, double out[9]);

/* MRI history sums of a state that the caller keeps on the device, with no
 * device allocation.  No counterpart in the reference: it is for callers that
 * cannot let the library allocate, e.g. a Fortran driver whose uin lives in
 * its OpenACC runtime (device pointers from `host_data use_device`) or a job
 * under a fixed device-memory budget.
 *   uin_dev  device array in the reference layout uin(iu1:iu2,ju1:ju2,ku1:ku2,1:11)
 *            (only variables 1-8 are read), on the calling thread's current device
 *   out_dev  9 device doubles, the same quantities as dg_history
 *   stream   cudaStream_t to enqueue on (NULL: the legacy default stream)
 * Needs ndim = 3, a non-empty domain and nx <= DG_HISTORY_NOALLOC_MAX_NX
 * (DG_ERR_ARG otherwise).  uin_dev and out_dev must be device or managed memory
 * of the current device: a host array (e.g. uin without `host_data use_device`)
 * or another device's memory is refused with DG_ERR_ARG before any launch.  A
 * CUDA error already pending in the calling thread is reported (DG_ERR_CUDA) and
 * left pending for the caller.
 * The reduction scratch is one file-scope device array per GPU (about 280 KB),
 * held until the process exits; its address is looked up the first time the
 * call runs on a device, so make that first call before any stream capture.
 * With lazy module loading (the CUDA default) the driver places that array in
 * device memory when the library's kernels are first used on a device, so make
 * the first call at start-up, or run with CUDA_MODULE_LOADING=EAGER, if device
 * memory must not grow later.  All calls share the array: calls that overlap on
 * the GPU (different streams, no ordering) race.  The call is asynchronous;
 * out_dev is valid once the stream reaches it (in the bounds-checked debug
 * library the call waits for its kernels). */
#define DG_HISTORY_NOALLOC_MAX_NX 16384
int  dg_history_noalloc(const dg_params *p, const double *uin_dev, double *out_dev, void *stream);

/* ---- z-slab decomposition ----------------------------------------------------
 * The reference decomposes the box over MPI ranks (parallel.f90:197-697) and
 * exchanges 3-deep ghost slabs of uin after each boundary call, with
 * MPI_Sendrecv or ncclSend/ncclRecv (boundary_z, parallel.f90:480-590).  Here
 * the box is split in z only (x keeps the shear-periodic boundary local and
 * FARGO needs whole y lines); each slab is one context (one per GPU, or several
 * on one GPU), and the caller moves the halos between them with any transport
 * (NCCL, MPI, a device copy): after dg_boundary (and after dg_dissipation) of
 * every slab, pack both sides of every slab, send side 0 to the lower
 * neighbour and side 1 to the upper one (periodic in zposition), and unpack
 * what arrives: from the lower neighbour into side 0, from the upper into side 1.
 * The CFL step is the minimum of every slab's dg_compute_dt (the reference's
 * MPI_Allreduce(MIN), physics.f90:123-129).  A zero-gradient z boundary is
 * applied by the bottom and top slabs themselves; their outer sides need no
 * halo.  dg_run refuses slab contexts (the exchange is the caller's).
 * Halo layout: 3 planes (the x and y ghosts included) of every stored state
 * plane, plane by plane: dg_halo_count doubles. */
long long dg_halo_count(const dg_ctx *ctx);
/* side 0: the slab's 3 lowest active planes; side 1: its 3 highest, into the
 * device buffer dev_buf (dg_halo_count doubles, any device that can read the
 * context's memory); enqueued on the context's stream */
int  dg_halo_pack(dg_ctx *ctx, int side, double *dev_buf);
/* side 0: dev_buf into the 3 ghost planes below the slab; side 1: above it */
int  dg_halo_unpack(dg_ctx *ctx, int side, const double *dev_buf);
/* MRI history of a decomposed box in two phases, as compute_yz_mean and
 * vol_average do it with MPI (src/problem/mri/history.f90:176-245):
 *   phase 1: col[2(i-1)], col[2(i-1)+1] = this slab's sums of v_x and v_y over
 *            the cells of x column i (2 nx doubles, host);
 *   the caller sums col over the slabs and divides by ny * nz * nzslice;
 *   phase 2: this slab's share of the 9 history values (dg_history's order,
 *            volume-normalised by the whole box) with those column means;
 *            the box's values are the sums of the shares. */
int  dg_history_columns(dg_ctx *ctx, double *col);
int  dg_history_share(dg_ctx *ctx, const double *colmean, double out[9]);

/* wait for all work of the context (bounded) */
int  dg_sync(dg_ctx *ctx);

/* Per-kernel CUDA-event timing on the context's stream (no counterpart in the
 * reference, whose timers are host system_clock calls inserted by its
 * preprocessor, utils/pyutils/preproc/preprocess.py:330-355).
 * dg_profile(ctx, 1) starts recording an event pair around every kernel;
 * dg_profile_read fills ms[slot] and count[slot] for the launches since the
 * last read (slots named by dg_profile_slot_name) and resets them. */
#define DG_PROFILE_SLOTS 15
int  dg_profile(dg_ctx *ctx, int on);
int  dg_profile_read(dg_ctx *ctx, double *ms, long long *count, int nslots);
const char *dg_profile_slot_name(int slot);

/* Self-test of the bounded device-side waits: one block waits on an mbarrier with the
 * wait every tensor-core kernel of the library uses (1 s bound on %globaltimer).  With
 * arrive = 1 a thread arrives and the call returns DG_OK; with arrive = 0 nothing
 * arrives, the wait runs out and the call returns DG_ERR_TIMEOUT after about a second,
 * the device staying usable.  *seconds (may be NULL) receives the elapsed wall time. */
int  dg_wait_selftest(int device, int arrive, double *seconds);

/* Accesses of the step kernels that fell outside every registered device buffer, since
 * the library was loaded, in the bounds-checked build (libdumses_gpu_chk.so, compiled with
 * -DDG_CHECK_BOUNDS, where such an access is counted and not made); -1 in the normal build. */
long long dg_debug_oob_count(void);

/* number of kernels the library launched on this context since dg_init */
long long dg_kernel_launches(const dg_ctx *ctx);

/* the context's CUDA stream (a cudaStream_t), so a caller can order its own work */
void *dg_stream(dg_ctx *ctx);

/* Test hook: copy one device work array of the last step to the host.
 *   which 0..2  face fluxes of direction x/y/z over faces [1,nx+1]x[1,ny+1]x[1,nz+1],
 *               face-major: rho, E, rho u, rho v, rho w (scaled by area*dt as compflux
 *               does), p*_T (6 values per face in 3D), then in 2D the B_z flux and 0
 *               (8 values per face)
 *   which 3..5  edge EMFs x/y/z (already multiplied by dt) over the same index space
 *   which 6     primitive variables (8) on the ghosted grid
 * count is the number of doubles the host buffer holds; returns the number of
 * doubles copied in *copied.  No counterpart in the reference (its arrays are
 * module globals). */
int  dg_debug_copy(dg_ctx *ctx, int which, double *host, long long count, long long *copied);

/* message of the last failing call on this thread ("" if none) */
const char *dg_last_error(void);

/* ---- learned face-flux surrogate --------------------------------------------
 * No counterpart in the reference, whose face solver is always an exact one
 * (src/modules/solvers/solver.f90:163-187).  A 17 -> 64 -> 64 -> 8 MLP (by default)
 * with SmeLU hidden activations (the smooth ReLU: 0, (z+1)^2/4 or z), BF16
 * weights and FP32 accumulation on the tensor cores, trained on the device by
 * the library's own forward, backward and Adam kernels.  Per interface
 * it predicts HLLD minus LLF of the same states.  States are scaled by the
 * interface's density rho0 = (rhoL+rhoR)/2, a speed a0 >= both fast speeds and the
 * field unit sqrt(rho0) a0 (rho / rho0, velocities / a0, P / (rho0 a0^2), fields
 * / (sqrt(rho0) a0)); J is the norm of the scaled right-minus-left jump of rho,
 * u_n, v_t1, v_t2, P, B_t1, B_t2.
 *   inputs (17): mean u_n, v_t1, v_t2, P, B_n, B_t1, B_t2; the jump of rho, u_n,
 *                v_t1, v_t2, P, B_t1, B_t2 divided by J; J; ln(J)/10; gamma - 1
 *   outputs (8): mass, energy, normal momentum (HLLD flux + p*_T), t1 momentum,
 *                B_t1, t2 momentum and B_t2 fluxes, and p*_T - (ptotL+ptotR)/2,
 *                each divided by J and by its unit (rho0 a0, rho0 a0^3, rho0 a0^2,
 *                sqrt(rho0) a0^2, rho0 a0^2)
 * Shape: 17 inputs, dg_nn_shape's depth hidden layers of its width, 8 outputs
 * (the library's build fixes them; 64 x 2 by default, width 32, 64 or 128, depth
 * 1 to 3).  Parameters, in dg_nn_get_params order, for width H and depth L:
 * W1[17][H], b1[H], then L - 1 times W[H][H], b[H], then W[H][8], b[8]
 * (W[k][n]: input k, output n); 5832 of them at the default shape.
 * Batches are multiples of 128 rows.  On a context with precision FP32 and
 * surrogate = 1, an attached network replaces HLLD on faces that pass its gates
 * (positive states, relative pressure and density jumps and compression below
 * the thresholds, inputs inside the training envelope, outputs inside the
 * training range); the other faces get exact HLLD. */
typedef struct dg_nn dg_nn;
#define DG_NN_INPUTS  17
#define DG_NN_OUTPUTS 8
long long dg_nn_param_count(void);
/* hidden width and number of hidden layers of this build's network */
int  dg_nn_shape(int *width, int *depth);
int  dg_nn_create(int device, unsigned long long seed, dg_nn **out);
int  dg_nn_destroy(dg_nn *nn);
/* training samples: x[count][17], t[count][8] (scaled as above) */
int  dg_nn_set_samples(dg_nn *nn, const float *x, const float *t, long long count);
int  dg_nn_reserve_samples(dg_nn *nn, long long count);
long long dg_nn_sample_count(const dg_nn *nn);
int  dg_nn_samples_copy(dg_nn *nn, long long first, long long count, float *x, float *t);
/* append the interfaces of the context's current state (every stride-th face of
 * each direction, in a fixed order) with FP64 HLLD labels; FP32 contexts only */
int  dg_nn_harvest(dg_ctx *ctx, dg_nn *nn, int stride, long long *added);
/* `steps` Adam steps on random batches; *loss = mean squared error of the last */
int  dg_nn_train(dg_nn *nn, int steps, int batch, float lr, float *loss);
/* loss and parameter gradients of one batch, without an update */
int  dg_nn_gradients(dg_nn *nn, const float *x, const float *t, int batch, float *loss, float *grad);
int  dg_nn_forward(dg_nn *nn, const float *x, long long count, float *y);
int  dg_nn_get_params(dg_nn *nn, float *params, long long count);
int  dg_nn_set_params(dg_nn *nn, const float *params, long long count);
/* the envelope of the current samples (widened by margin x its width) becomes
 * the confidence gate */
int  dg_nn_fit_envelope(dg_nn *nn, float margin);
/* standardise inputs (mean, standard deviation) and outputs (root mean square) by
 * the current samples; call before training (identity until then) */
int  dg_nn_fit_scaling(dg_nn *nn);
int  dg_nn_set_gates(dg_nn *nn, float jump, float compress);
/* use `nn` (NULL: none) for the faces of an FP32 context made with surrogate = 1 */
int  dg_attach_surrogate(dg_ctx *ctx, dg_nn *nn);
/* faces seen by the surrogate and faces that fell back to HLLD since the last call */
int  dg_surrogate_stats(dg_ctx *ctx, long long *faces, long long *fallback);

/* Host-side initial conditions written straight into a reference-layout uin
 * (11 variables, ghosts included), followed by the reference's first boundary
 * call being the caller's job (dg_upload + dg_boundary(ctx, 0, 0)).
 *   DG_IC_FIELD_LOOP  2D field-loop advection (magnetic_loop/condinit.f90 form)
 *   DG_IC_ORSZAG_TANG 3D Orszag-Tang-type vortex
 *   DG_IC_MRI         shearing-box MRI, net vertical field, seeded velocity kicks
 *   DG_IC_MRI_TEST    the reference's deterministic MRI "Test" setup
 *                     (mri/condinit.f90:73-105 with type='Test', amp=0) */
#define DG_IC_FIELD_LOOP  1
#define DG_IC_ORSZAG_TANG 2
#define DG_IC_MRI         3
#define DG_IC_MRI_TEST    4
int  dg_condinit(const dg_params *p, int ic, double beta, double amp,
                 unsigned long long seed, double *uin);

#ifdef __cplusplus
}
#endif
#endif /* DUMSES_GPU_H */
