/*
 * dcm.h -- C-ABI of the B200 dynamical core (MPDATA advection + BiCGSTAB
 * pressure solve) of UoM-maul1609/dynamical-cloud-model.
 *
 * Plain C types only: pointers, sizes, doubles.  Every 3-D field argument is
 * a HOST array in the reference's own Fortran layout and kind:
 *     real(c_double) :: a(0:kp+1, 0:jp+1, 0:ip+1)      (halo 1, k fastest)
 * passed as its base address, exactly what a Fortran caller passes for a
 * dimension(*) dummy through ISO_C_BINDING.  1-D profiles are
 * real(c_double) :: p(0:n+1).  The library copies in and out and never keeps
 * a host pointer.  Calls on one handle are synchronous and must not overlap.
 *
 * The MPI arguments of the reference routines (comm3d, id, rank, dims,
 * coords) are not part of the ABI: the whole domain lives on one GPU, so the
 * caller checks dims = [1,1,1] with dcm_check_decomposition() once.
 *
 * Every function returns a dcm_status.  Where the reference calls STOP, the
 * library returns an error code instead; a Fortran interface module over
 * this header prints the reference's message and stops.
 */
#ifndef DCM_H
#define DCM_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum {
    DCM_OK = 0,
    DCM_E_NOCONV = 1,      /* bicgstab: no convergence in itmax iterations
                              (dynamics.f90:431-434)                        */
    DCM_E_BREAKDOWN = 2,   /* bicgstab: |omega| < tiny (dynamics.f90:414-417) */
    DCM_E_NONFINITE = 3,   /* a residual norm became NaN / Inf              */
    DCM_E_CUDA = 4,        /* a CUDA call failed; see dcm_last_error()      */
    DCM_E_TIMEOUT = 5,     /* a bounded device wait expired                 */
    DCM_E_DECOMP = 6,      /* process grid is not 1 x 1 x 1                 */
    DCM_E_ARG = 7,         /* invalid argument                              */
    DCM_E_UNSUPPORTED = 8, /* configuration outside the implemented path    */
    DCM_E_IO = 9           /* writing an output file failed                 */
} dcm_status;

/* Grid description.  All arrays are host pointers, length n+2 (index 0..n+1),
 * as built by allocate_and_set (initialisation.f90:428-446, :505-578). */
typedef struct {
    int ip, jp, kp;
    const double *dx, *dxn;        /* ip+2 */
    const double *dy, *dyn;        /* jp+2 */
    const double *dz, *dzn;        /* kp+2 */
    const double *rhoa, *rhoan;    /* kp+2 */
    const double *theta, *thetan;  /* kp+2 */
    const double *xg, *yg, *zg;    /* ip+2, jp+2, kp+2 (bicgstab test_solver) */
} dcm_grid;

/* Optional terms of sources (dynamics.f90:800-873); NULL = all off. */
typedef struct {
    int damping_layer, forcing, divergence;
    const double *dampfacn, *dampfac;  /* kp+2 */
    const double *u_force, *v_force;   /* kp+2 */
    const double *w_subs;              /* kp+2 */
    double forcing_tau;
} dcm_forcing;

typedef struct dcm_handle dcm_handle;

/* ---- lifetime ----------------------------------------------------------- */
/* Replaces the first-call set-up of bicgstab (allocation of a_e..a_c and
 * set_mat_a, dynamics.f90:330-352): the stencil coefficients are computed
 * here once from the 1-D metrics.  device = CUDA ordinal. */
int dcm_create(const dcm_grid *grid, int device, dcm_handle **out);
int dcm_destroy(dcm_handle *h);
const char *dcm_status_string(int status);
const char *dcm_last_error(const dcm_handle *h);
/* mpi_cart_initialise (mpi_module.f90:109-297): only dims = [1,1,1] runs
 * here; anything else returns DCM_E_DECOMP. */
int dcm_check_decomposition(const int dims[3]);

/* ---- per-call drop-ins (host arrays in, host arrays out) -------------------- */

/* bicgstab, dynamics.f90:293-444.  x: inout (warm start / solution),
 * b: inout (replaced by the Gaussian test field when test_solver != 0 on the
 * first call, :354-364), sw: in (bottom fix-up x(0)=x(1)-sw(0)dzn(0),
 * :437-442).  tol = ptol; itmax = 9999 in the reference.  iters / err may be
 * NULL.  Interior and the top/bottom rows of x follow the reference; the x/y
 * halo columns are those of the input (the reference leaves solver residue
 * there and the driver overwrites them with exchange_along_dim_wo). */
int dcm_bicgstab(dcm_handle *h, double *x, double *b, const double *sw,
                 double tol, int test_solver, int itmax, int *iters,
                 double *err);

/* sources, dynamics.f90:639-1000 with viscous = .false.: su, sv, sw (out,
 * halos by exchange_full + surface/lid rows), sth (inout: += damping, then
 * exchange_full), rhs (inout: k = 0..kp+1 over the interior columns).
 * ubar..thbar are 1-D (kp+2).  zu, zv, zw are read only when damping or
 * forcing is on. */
int dcm_sources(dcm_handle *h, const dcm_forcing *forcing,
                const double *ubar, const double *vbar, const double *wbar,
                const double *thbar, const double *zu, const double *zv,
                const double *zw, const double *u, const double *v,
                const double *w, const double *th, double *su, double *sv,
                double *sw, double *sth, double *rhs);

/* advance_momentum, dynamics.f90:1019-1099: u,v,w (inout) for k = 0..kp,
 * interior columns; the driver passes 2*dt (driver_code.f90:592-594). */
int dcm_advance_momentum(dcm_handle *h, double dt, double *u, double *v,
                         double *w, const double *zu, const double *zv,
                         const double *zw, const double *su,
                         const double *sv, const double *sw,
                         const double *p);

/* first_order_upstream_3d, pamm/sfvt/advection_3d.F90:39-116 (interior
 * update only; neumann 0/1/2). */
int dcm_first_order_upstream_3d(dcm_handle *h, double dt, const double *u,
                                const double *v, const double *w,
                                double *psi, int neumann);

/* mpdata_3d, pamm/sfvt/advection_3d.F90:219-714.  lbc / ubc inout (shifted
 * and unshifted as the reference does).  limiter: 0 = the linked
 * pamm/sfvt form (:542-675), 1 = the sfvt/advection_3d.F90 form (:544-704). */
int dcm_mpdata_3d(dcm_handle *h, double dt, const double *u, const double *v,
                  const double *w, double *psi, double *lbc, double *ubc,
                  int kord, int monotone, int neumann, int limiter);

/* mpdata_vec_3d, pamm/sfvt/advection_3d.F90:1250-1753: psi holds nq
 * consecutive fields (Fortran psi(:,:,:,1:nq)); lbc/ubc have length nq. */
int dcm_mpdata_vec_3d(dcm_handle *h, double dt, const double *u,
                      const double *v, const double *w, double *psi, int nq,
                      double *lbc, double *ubc, int kord, int monotone,
                      int neumann, int limiter);

/* adv_ref_state, pamm/sfvt/advection_3d.F90:1148-1218 (psi_ref = thetan in
 * the driver, driver_code.f90:518-519). */
int dcm_adv_ref_state(dcm_handle *h, double dt, const double *w, double *psi,
                      const double *psi_ref);

/* mpdata_3d_add, pamm/sfvt/advection_3d.F90:139-190. */
int dcm_mpdata_3d_add(dcm_handle *h, double dt, const double *u,
                      const double *v, const double *w, double *psi,
                      const double *psi_1d, double *lbc, double *ubc,
                      int kord, int monotone, int neumann, int limiter);

/* horizontal_means, diagnostics.f90:31-107: bars are (kp+2) each, qbar is
 * nq*(kp+2) (Fortran qbar(0:kp+1, nq)); q may be NULL when moisture = 0. */
int dcm_horizontal_means(dcm_handle *h, int moisture, int nq,
                         const double *u, const double *v, const double *w,
                         const double *th, const double *q, double *ubar,
                         double *vbar, double *wbar, double *thbar,
                         double *qbar);

/* divergence_calc, diagnostics.f90:120-153 (interior of div written). */
int dcm_divergence_calc(dcm_handle *h, const double *u, const double *v,
                        const double *w, double *div);

/* advance_scalar_fields_3d, sgm/subgrid_3d.f90:582-624 (whole arrays). */
int dcm_advance_scalar_fields_3d(dcm_handle *h, double dt, double *q,
                                 const double *sq, double *th,
                                 const double *sth, int nq, int moisture);

/* The PAMM microphysics' sedimentation transport, mpdata_vec_1d
 * (pamm/sfvt/advection_1d.F90:463-778, with first_order_upstream_1d :35-74)
 * for ncol independent columns at once, each with the caller's sub-stepping
 * loop (pamm/microphysics.f90:3139-3145, 3158-3164, 3177-3183): column c takes
 * nsub[c] passes of dt[c]/nsub[c] (nsub NULL: one pass).  Host arrays, column
 * after column: w, ncol x (kp+l_h+r_h), each row w(-l_h+1:kp+r_h); psi, ncol x
 * nq x (kp+2 r_h), each column psi_in(-r_h+1:kp+r_h, 1:nq) in Fortran order,
 * advanced in place; dz, dzn, rhoa, rhoan shared by all columns
 * (metric_stride 0, kp+l_h+r_h values each) or one row per column
 * (metric_stride = kp+l_h+r_h).  kord, monotone, neumann as the reference's.
 * Runs on the calling thread's current device and returns when psi is back
 * on the host.  DCM_E_ARG for l_h or r_h < 1, nsub[c] < 1, or a column too
 * tall for one warp's shared memory (above 200 KiB: (nq+4)(kp+2 r_h) +
 * 3(kp+l_h+r_h) + nq doubles with kord > 1, (nq+1)(kp+2 r_h) + kp+l_h+r_h +
 * nq with kord <= 1). */
int dcm_mpdata_vec_1d(int ncol, int kp, int nq, int l_h, int r_h, const double *dt,
                      const int *nsub, const double *dz, const double *dzn,
                      const double *rhoa, const double *rhoan, int metric_stride,
                      const double *w, double *psi, int kord, int monotone, int neumann);
/* The same with every array in device memory, queued on `stream` (NULL: the
 * default stream): for a host that keeps the columns on the GPU.  Allocates
 * nothing, returns when the work is queued; nsub[c] < 1 counts as one pass.
 * A CUDA error already pending on the calling thread returns DCM_E_CUDA at
 * once, queueing nothing. */
int dcm_mpdata_vec_1d_device(int ncol, int kp, int nq, int l_h, int r_h, const double *dt,
                             const int *nsub, const double *dz, const double *dzn,
                             const double *rhoa, const double *rhoan, int metric_stride,
                             const double *w, double *psi, int kord, int monotone,
                             int neumann, void *stream);

/* Halo exchanges of mpi_module.f90 for one rank: exchange_full (:926-1271),
 * exchange_along_dim (:700-910), exchange_along_dim_wo (:1285-1494),
 * exchange_full_wo (:1511-1855). */
int dcm_exchange_full(dcm_handle *h, double *a, double lbc, double ubc);
int dcm_exchange_along_dim(dcm_handle *h, double *a, double lbc, double ubc);
int dcm_exchange_along_dim_wo(dcm_handle *h, double *a);
int dcm_exchange_full_wo(dcm_handle *h, double *a);

/* calculate_subgrid_3d, sgm/subgrid_3d.f90:38-357 (the Smagorinsky model,
 * with richardson :448-493 and monin_obukhov :373-433), one rank.  z(1) is
 * the grid's zg[1] (dcm_create needs zg); lamsq has kp+2 values.  In:
 * u, v, w, zu, zv, zw, th (and q: nq consecutive fields, read only when
 * moisture != 0).  Inout as in the reference: vism, vist (interior, the
 * surface row and their exchange_full_wo images), strain (interior), the six
 * stresses (interior and their exchange_along_dim(0, 0) images), su, sv, sw,
 * sth (+= the stress / diffusion terms, then exchange_full(0, 0)); with
 * moisture, viss (nq fields, each set to vist) and sq (nq fields, += the
 * diffusion of each q, then exchange_full(0, 0)).  The arguments dt, z, zn
 * and the metric arrays of the Fortran interface come from the handle. */
int dcm_calculate_subgrid_3d(dcm_handle *h, const double *lamsq, double z0,
                             double z0th, const double *u, const double *v,
                             const double *w, const double *zu,
                             const double *zv, const double *zw,
                             const double *th, int nq, const double *q,
                             double *vism, double *vist, double *viss,
                             double *strain, double *tau11, double *tau22,
                             double *tau33, double *tau12, double *tau13,
                             double *tau23, double *su, double *sv,
                             double *sw, double *sth, double *sq,
                             int moisture);

/* ---- device-resident time loop ------------------------------------------- */
/* Configuration of model_driver's dry step (driver_code.f90:304-676) with
 * output, microphysics, radiation and land surface off; the subgrid model
 * (sources with viscous = .true.) on when viscous != 0. */
typedef struct {
    double dt, ptol;
    int advection_scheme;   /* 0 upwind, 1 mpdata, 2 mpdata_3d_add        */
    int kord, monotone, limiter;
    int itmax;              /* 9999 in the reference                       */
    int moisture, nq, ncat; /* q categories advected by mpdata_vec_3d      */
    const int *c_s, *c_e;   /* 1-based category bounds (ncat each)         */
    double thbase, thtop;   /* lbc / ubc of scheme 2                       */
    int precision;          /* 0 = FP64 (the reference's VAR_TYPE=1);
                               1 = FP32 fields; FP32 BiCGSTAB iterations on
                               an FP64 pressure with FP64 reliable updates,
                               converged to ptol on the FP64 residual      */
    double inner_tol;       /* precision 1: reliable-update factor: the FP32
                               recursion stops for an FP64 update of p and
                               of the true residual when its residual has
                               fallen by this factor (0 -> 0.1)            */
    dcm_forcing forcing;
    int viscous;            /* 1: sources calls calculate_subgrid_3d
                               (dynamics.f90:878-893); needs the grid's zg */
    const double *lamsq;    /* kp+2: mixing length squared on the w-levels
                               (initialisation.f90:449-450)                */
    double z0, z0th;        /* roughness lengths for momentum and scalars  */
    int precond;            /* precision 1: preconditioner of the FP32
                               iterations.  0: the reference's three Jacobi
                               sweeps (dynamics.f90:241-270); 1: the same
                               three sweeps with Chebyshev weights on
                               [precond_lo, 2] of the spectrum of D^-1 A
                               (fewer iterations, same cost per iteration).
                               FP64 always uses the reference's sweeps.     */
    double precond_lo;      /* lower end of that interval (0 -> 0.05)      */
} dcm_config;

/* Host fields of the driver (all Fortran layout, double).  The three
 * velocity time levels are passed in their current roles: u,v,w (current),
 * zu,zv,zw (previous), tu,tv,tw (next / scratch). */
typedef struct {
    double *u, *v, *w, *zu, *zv, *zw, *tu, *tv, *tw;
    double *th, *p, *su, *sv, *sw, *psrc, *div, *sth;
    double *q, *sq;                            /* nq fields each, or NULL */
    double *ubar, *vbar, *wbar, *thbar, *qbar; /* kp+2 (qbar nq*(kp+2))   */
} dcm_fields;

typedef struct {
    int steps;              /* steps taken in this call                   */
    int iters_last;         /* BiCGSTAB iterations of the last step       */
    long long iters_total;  /* summed over the call                       */
    double err_last;        /* final relative residual of the last solve  */
    double ms_total;        /* device time of the call (CUDA events)      */
    int updates_last;       /* precision 1: FP64 reliable updates of the
                               last solve (0 for FP64)                     */
    int restarts_last;      /* precision 1: of those, restarts after a
                               breakdown of the FP32 recursion             */
} dcm_step_stats;

/* Upload the driver state; roles as in dcm_fields. */
int dcm_state_upload(dcm_handle *h, const dcm_config *cfg,
                     const dcm_fields *f);
/* model_driver's pre-loop rows (driver_code.f90:287-295) on the resident
 * previous-level velocities. */
int dcm_driver_start(dcm_handle *h);
/* nsteps passes of the time loop on the device. */
int dcm_step(dcm_handle *h, int nsteps, dcm_step_stats *stats);
/* Download the state; velocities come back in their current roles. */
int dcm_state_download(dcm_handle *h, dcm_fields *f);

/* ---- output (driver_code.f90:725-1145) ---------------------------------- */
/* The reference's output routine for the resident state: a netCDF classic
 * file (CDF-1, CDF-2 when an offset needs 64 bits) with the reference's
 * dimensions (times, ip, jp, kp [, nq, nprec, l_q_names]), variables
 * (time, x, y, z, rhoa, thetan, trefn, th, u, v, w, p, div [, q_names, q,
 * precip]), "units" attributes and FP32 values; q and precip have the q
 * index fastest as the reference's reshape writes them.  precip (the
 * microphysics' output) is written as zeros.
 * dcm_output_open writes the header and the fixed variables: x (ip+2), y
 * (jp+2), z (kp+2), trefn (kp+2, NULL: zeros) as the driver holds them,
 * rhoa and thetan from the handle; nq must be the resident number of q
 * fields (0 without moisture), q_names nq blank-padded names of 20 chars.
 * dcm_output_write appends one record of the current state with the given
 * time, as output() does at each output time: it queues a packing kernel on
 * the handle's stream and returns; a copy stream and a writer thread put the
 * record in the file while later dcm_step calls run (two records in flight;
 * a third write waits for the first).  dcm_output_flush waits until every
 * queued record is in the file; dcm_output_close flushes and closes.  Close
 * the output before dcm_destroy or a new dcm_state_upload. */
typedef struct dcm_output dcm_output;
int dcm_output_open(dcm_handle *h, const char *path, const double *x,
                    const double *y, const double *z, const double *trefn,
                    int nq, const char *q_names, int nprec, dcm_output **out);
int dcm_output_write(dcm_output *o, double time);
int dcm_output_flush(dcm_output *o);
int dcm_output_close(dcm_output *o);
const char *dcm_output_last_error(const dcm_output *o);

/* ---- horizontal means without device allocation ------------------------- */
/* No counterpart in the reference.  Same per-level means as
 * dcm_horizontal_means (u, v, w, th over the interior columns for
 * k = 0..kp+1, written to means[0:4*(kp+2)] as ubar, vbar, wbar, thbar), for
 * hosts that keep the fields on the device and do not allow library code to
 * allocate or free device memory (their memory belongs to their own pool or
 * budget, and cudaFree would synchronise the whole device).  All pointers
 * are device pointers; stream is a cudaStream_t (NULL = default stream) and
 * the work is queued on it without waiting.  The reduction's scratch is a
 * fixed 4 MiB device array inside the library, shared by every call on a
 * device: calls whose work overlaps on the GPU race and must be serialised
 * by the caller.  The first call on each device resolves that array's
 * device address (with the device current); make that first call before any
 * stream capture.  The address is kept for the life of the process: after a
 * cudaDeviceReset the array may move, so do not call this entry point again
 * in that process.  kp > DCM_NOALLOC_MAX_KP returns DCM_E_ARG.  A CUDA error
 * already pending on the calling thread makes it return DCM_E_CUDA at once,
 * queueing nothing and leaving that error pending for the caller's own
 * check. */
#define DCM_NOALLOC_MAX_KP 1024
int dcm_horizontal_means_noalloc(int ip, int jp, int kp, const double *u,
                                 const double *v, const double *w,
                                 const double *th, double *means,
                                 void *stream);

/* ---- diagnostics (no counterpart in the reference) ----------------------- */
/* Per-kernel-class launch counts (always kept during dcm_step) and device
 * time (CUDA events recorded on the launching stream around every launch of
 * dcm_step while timing is enabled).  dcm_profile_enable resets both.
 * Classes:
 * 0 solver setup, 1 Jacobi sweeps, 2 matvecs, 3 x/r update, 4 solver post,
 * 5 means+divergence, 6 sources, 7 Poisson rhs, 8 adv_ref_state,
 * 9 MPDATA shift, 10 donor cell, 11 antidiffusive velocities, 12 beta,
 * 13 limiter, 14 MPDATA restore, 15 momentum, 16 other. */
#define DCM_PROF_NCAT 17
int dcm_profile_enable(dcm_handle *h, int on);
int dcm_profile_read(dcm_handle *h, double *ms, long long *launches, int ncat);
/* Pressure-solve driver (default 1).  1: each solve is one CUDA graph whose
 * iteration loop is a conditional WHILE node, set by the last kernel of
 * every iteration from the device scalars (in the mixed form: a WHILE node of
 * FP64 update cycles, each holding a WHILE node of FP32 iterations and an IF
 * node for the FP64 reliable update), captured once and relaunched while its
 * arguments stay the same; the kernels of an iteration are launched with
 * programmatic dependent launch where the runtime takes it.  2: the same
 * graphs without programmatic dependent launch.  0: the host launches
 * iterations in chunks of 4 and polls the device scalars between chunks.
 * All launch the same kernels in the same order and give bit-identical
 * results; while event timing is enabled the host-driven loop is used. */
int dcm_solver_graphs(dcm_handle *h, int on);

/* Small domains (no counterpart in the reference): FP64 pressure solves of
 * domains with at most max_points interior points (default 8192, the
 * 128 x 1 x 64 shear layer; 0 = never) run as one kernel on one cluster of
 * eight blocks (one per SM): the whole of bicgstab (dynamics.f90:367-435) in
 * the reference's algebra, passes separated by cluster barriers, dot products
 * summed in a fixed order through distributed shared memory, instead of nine
 * kernels per iteration whose launch latency bounds such a domain.  The
 * statuses and the iteration counts reported are those of the multi-kernel
 * solve. */
int dcm_set_small_solver(dcm_handle *h, int max_points);

/* MPDATA launch shape (no counterpart in the reference).  fuse = 0 (the
 * default): one kernel per stage of an antidiffusive iteration
 * (antidiffusive velocities, betas, limited velocities, donor cell).
 * fuse = 1: each antidiffusive iteration of mpdata_3d / mpdata_vec_3d with
 * the linked limiter (or without the limiter) runs as one kernel that
 * forms those four stages plane by plane in shared memory, so that only the
 * limited velocities and the new field reach memory (9 field passes per
 * iteration instead of 27).  On a B200 the fused form is 2-3.4x slower: the
 * antidiffusive velocities read about 40 neighbour values per point and
 * depend on L1, which the fused kernel's shared-memory planes take.
 * max_rows (3..32) caps the rows of a block of the fused kernel (32: as many
 * as its shared memory holds).  Both give the same arithmetic per point. */
int dcm_set_mpdata_shape(dcm_handle *h, int fuse, int max_rows);

/* Limits of the pressure solve's failure paths (no counterpart in the
 * reference; the tests use them to reach DCM_E_TIMEOUT and DCM_E_BREAKDOWN
 * without a singular system).  max_rounds > 0 bounds a graph-driven solve
 * (dcm_solver_graphs 1 or 2) to that many loop rounds, after which it stops
 * with DCM_E_TIMEOUT; 0 restores the default budget, itmax + 1 rounds
 * (itmax + reliable updates + 1 in the mixed form), which a solve that
 * behaves never reaches.  tiny >= 0 replaces the breakdown threshold of an
 * FP64 solve, |omega| < tiny -> DCM_E_BREAKDOWN (dynamics.f90:414-417); a
 * negative tiny restores the reference's 1.e-16 (a default-real literal,
 * :321).  The FP32 iterations of the mixed form keep their own restart test.
 * Applies to every later solve of this handle (drop-in and resident). */
int dcm_solver_limits(dcm_handle *h, int max_rounds, double tiny);

/* *programmatic = 1 when this handle's graph-driven solves launch their
 * iteration kernels with programmatic dependent launch (mode 1 of
 * dcm_solver_graphs, and the runtime accepted such launches inside a WHILE
 * node when the first handle was created), else 0. */
int dcm_solver_graph_info(dcm_handle *h, int *programmatic);

/* ---- solver launch-shape autotuner (no counterpart in the reference) ---- */
/* Chooses, for this handle's grid shape and the given precision (0 FP64,
 * 1 the FP32 iterations of the mixed form), the launch shape of the solver
 * kernels: warps per block of the Jacobi sweeps (by: 2, 4, 8), warp tasks per
 * warp of the reducing kernels (tasks: 0 = as many blocks as are resident,
 * each warp striding over many tasks; 1, 2 = that many tasks per warp), the
 * depth, the number of i-planes the first Jacobi sweep and the reducing
 * kernels (the solve's set-up and the two matvecs) march over (1, 2, 4, 8),
 * and in FP32 whether the three sweeps of each preconditioner
 * application run fused in one kernel (fuse 1: columns of at most 128
 * levels), and whether that kernel of phase C also forms t = A cs with its
 * dots (t,t), (t,s) as a fourth stage (fuse 2; otherwise the matvec is a
 * kernel of its own), and in FP32 the vector width of the separate stencil
 * and update kernels (vec: 4 levels per lane, 16-byte vectors, so that a
 * warp task covers 128 levels; or 2 levels per lane, 8-byte vectors and 64
 * levels per warp task, which keeps more lanes busy on short columns; the
 * fused kernel always uses 4; FP64 uses 2, 16-byte vectors).
 * It times 12 BiCGSTAB iterations of each candidate on a synthetic
 * right-hand side and applies the fastest to the handle for that precision
 * (each precision keeps its own launch shape).  With use_cache the result is
 * looked up first in, and otherwise appended to, a text file:
 * $DCM_TUNE_CACHE, or $HOME/.cache/dcm_b200_solver_tune.txt (one line per SM
 * count, grid shape and precision).  Uses the handle's scratch fields; call
 * it before dcm_state_upload or between steps, not concurrently with other
 * calls on the handle. */
int dcm_tune(dcm_handle *h, int precision, int use_cache, int *by, int *tasks,
             int *depth, int *fuse, int *vec);
/* Sets the launch shape of one precision explicitly (same meaning and ranges
 * as dcm_tune's results; by <= 8, depth <= 63, fuse 0..2 and vec 2 or 4 only
 * for precision 1, a fused preconditioner only with vec 4; vec 2 for
 * precision 0).  Default: by 8, tasks 0, depth 1, fuse 1, vec 4 (FP32) /
 * depth 4, fuse 0, vec 2 (FP64). */
int dcm_set_launch_shape(dcm_handle *h, int precision, int by, int tasks,
                         int depth, int fuse, int vec);

/* ---- batched ensemble (no counterpart in the reference) ------------------ */
/* Independent domains of possibly different sizes on one device.  Each
 * member is a full handle (dcm_ensemble_member): upload its state with
 * dcm_state_upload + dcm_driver_start, optionally dcm_tune it, read it back
 * with dcm_state_download.  dcm_ensemble_step advances every member by one
 * time step per launch of ONE CUDA graph: a fork into one branch per member
 * holding that member's whole step; each member's pressure solve is its own
 * conditional WHILE loop, so a converged member stops iterating while the
 * others continue (per-member convergence masks).  Three graphs (the
 * velocity-role phases of the leapfrog rotation) are captured on first use
 * and recaptured after a member's state upload or tuning.  Members must be
 * at the same step count and use advection_scheme 0 or 1 without moisture
 * and with t1 = t2 = 0 (the dry configurations). */
typedef struct dcm_ensemble dcm_ensemble;
typedef struct {
    int steps;              /* ensemble steps taken in this call           */
    long long iters_total;  /* solver iterations, all members and steps    */
    int iters_max_last;     /* most iterations of any member, last step    */
    double ms_total;        /* device time of the graph launches           */
} dcm_ensemble_stats;
int dcm_ensemble_create(int nmembers, const dcm_grid *grids, int device,
                        dcm_ensemble **e);
int dcm_ensemble_destroy(dcm_ensemble *e);
int dcm_ensemble_member(dcm_ensemble *e, int member, dcm_handle **h);
int dcm_ensemble_step(dcm_ensemble *e, int nsteps, dcm_ensemble_stats *stats);
const char *dcm_ensemble_last_error(const dcm_ensemble *e);

#ifdef __cplusplus
}
#endif
#endif /* DCM_H */
