/*
 * dcm_oracle.h -- CPU restatement (FP64) of the reference dynamical-core
 * timestep of UoM-maul1609/dynamical-cloud-model.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the product links this library; only
 * tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference arm
 * load it, as the parity reference or as the timed CPU baseline.
 *
 * PARITY UNPINNED: the reference is Fortran 90 and no Fortran compiler exists
 * in this image, and the reference ships no tests, fixtures or golden vectors.
 * This restatement is cross-checked against an independent numpy restatement
 * (tests/golden/np_reference.py) and against analytic invariants instead.
 *
 * Layout: every 3-D field is the reference's own Fortran column-major array
 * a(0:kp+1, 0:jp+1, 0:ip+1) (halo width 1, main.f90:80-81), i.e. element
 * (k,j,i) lives at  k + (kp+2)*(j + (jp+2)*i).  1-D metric arrays carry the
 * same halo: dx(0:ip+1), dy(0:jp+1), dz(0:kp+1) ...
 */
#ifndef DCM_ORACLE_H
#define DCM_ORACLE_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    int ip, jp, kp;
    /* 1-D grid metrics, halo-inclusive (length n+2, index 0..n+1) */
    const double *dx, *dxn;          /* ip+2 */
    const double *dy, *dyn;          /* jp+2 */
    const double *dz, *dzn;          /* kp+2 */
    const double *rhoa, *rhoan;      /* kp+2: density on w-levels / scalar levels */
    const double *theta, *thetan;    /* kp+2: base-state potential temperature */
    const double *xg, *yg, *zg;      /* coordinates, used by bicgstab(test_solver) */
} orc_grid;

/* optional forcing terms of sources (dynamics.f90:800-873) */
typedef struct {
    int damping_layer, forcing, divergence;
    const double *dampfacn, *dampfac;       /* kp+2 */
    const double *u_force, *v_force;        /* kp+2 */
    const double *w_subs;                   /* kp+2 */
    double forcing_tau;
} orc_forcing;

/* status codes (mirror the C-ABI's) */
enum { ORC_OK = 0, ORC_E_NOCONV = 1, ORC_E_BREAKDOWN = 2 };

/* threading of the stencil loops (OpenMP); reductions stay serial unless
 * parallel_reductions is set, which changes the summation order.           */
void orc_set_threads(int nthreads, int parallel_reductions);

/* ---- halo exchange, single-rank semantics (mpi_module.f90:584-1494) ---- */
void orc_exchange_full(const orc_grid *g, double *a, double lbc, double ubc);
void orc_exchange_along_dim(const orc_grid *g, double *a, double lbc, double ubc);
void orc_exchange_along_dim_wo(const orc_grid *g, double *a);
void orc_exchange_full_wo(const orc_grid *g, double *a);

/* ---- pressure solver (dynamics.f90:34-482) ---- */
double orc_inn_prod(const orc_grid *g, const double *x, const double *y);
void orc_mat_ax(const orc_grid *g, double *x, double *ax);
void orc_precondition(const orc_grid *g, const double *r, double *s, int prit);
/* bicgstab: x (inout) warm start / solution, b (inout) RHS.  *first_call is
 * the module flag bicgstab_first; test_solver replaces b on the first call.
 * itmax = 9999 in the reference.  Returns ORC_* status.                     */
int orc_bicgstab(const orc_grid *g, double *x, double *b, const double *sw,
                 double tol, int test_solver, int *first_call, int itmax,
                 int *iters, double *err);
/* Breakdown threshold of |omega| for later orc_bicgstab calls (process-wide;
 * negative: the reference's tiny).  For tests of the breakdown stop.        */
void orc_set_breakdown_tiny(double tiny);

/* ---- sources / momentum (dynamics.f90:639-1099) ---- */
int orc_sources(const orc_grid *g, const orc_forcing *f,
                const double *ubar, const double *vbar, const double *wbar,
                const double *thbar,
                const double *zu, const double *zv, const double *zw,
                const double *u, const double *v, const double *w,
                const double *th,
                double *su, double *sv, double *sw, double *sth, double *rhs);
/* sources with viscous = .true. (dynamics.f90:878-893): the subgrid model
 * replaces the full exchange of su, sv, sw, sth.  lamsq: kp+2; vism, vist,
 * strain: inout 3-D; q / sq (nq fields) used when moisture is set.          */
typedef struct {
    int viscous;
    const double *lamsq;
    double z0, z0th;
} orc_viscous;
int orc_sources_viscous(const orc_grid *g, const orc_forcing *f, const orc_viscous *vis,
                        const double *ubar, const double *vbar, const double *wbar,
                        const double *thbar,
                        const double *zu, const double *zv, const double *zw,
                        const double *u, const double *v, const double *w,
                        const double *th, int nq, const double *q, int moisture,
                        double *vism, double *vist, double *strain,
                        double *su, double *sv, double *sw, double *sth, double *sq,
                        double *rhs);
void orc_advance_momentum(const orc_grid *g, double dt,
                          double *u, double *v, double *w,
                          const double *zu, const double *zv, const double *zw,
                          const double *su, const double *sv, const double *sw,
                          const double *p);

/* ---- advection (pamm/sfvt/advection_3d.F90) ---- */
void orc_first_order_upstream_3d(const orc_grid *g, double dt,
                                 const double *u, const double *v,
                                 const double *w, double *psi, int neumann);
/* limiter_variant: 0 = linked pamm/sfvt form, 1 = sfvt/ interface-copy form */
void orc_mpdata_3d(const orc_grid *g, double dt, const double *u,
                   const double *v, const double *w, double *psi,
                   double *lbc, double *ubc, int kord, int monotone,
                   int neumann, int limiter_variant);
void orc_mpdata_vec_3d(const orc_grid *g, double dt, const double *u,
                       const double *v, const double *w, double *psi, int nq,
                       double *lbc, double *ubc, int kord, int monotone,
                       int neumann, int limiter_variant);
void orc_adv_ref_state(const orc_grid *g, double dt, const double *w,
                       double *psi, const double *psi_ref);
void orc_mpdata_3d_add(const orc_grid *g, double dt, const double *u,
                       const double *v, const double *w, double *psi,
                       const double *psi_1d, double *lbc, double *ubc,
                       int kord, int monotone, int neumann,
                       int limiter_variant);

/* ---- Smagorinsky subgrid model (sgm/subgrid_3d.f90:38-493) ----
 * z = g->zg (z(1) only).  viss / q / sq (nq fields each) are used only when
 * moisture is set.                                                          */
void orc_calculate_subgrid_3d(const orc_grid *g, const double *lamsq, double z0,
                              double z0th, const double *u, const double *v,
                              const double *w, const double *zu, const double *zv,
                              const double *zw, const double *th, int nq, const double *q,
                              double *vism, double *vist, double *viss, double *strain,
                              double *tau11, double *tau22, double *tau33, double *tau12,
                              double *tau13, double *tau23, double *su, double *sv,
                              double *sw, double *sth, double *sq, int moisture);

/* ---- diagnostics (diagnostics.f90) and scalar update (sgm/subgrid_3d.f90) */
void orc_horizontal_means(const orc_grid *g, int moisture, int nq,
                          const double *u, const double *v, const double *w,
                          const double *th, const double *q, double *ubar,
                          double *vbar, double *wbar, double *thbar,
                          double *qbar);
void orc_divergence_calc(const orc_grid *g, const double *u, const double *v,
                         const double *w, double *div);
void orc_advance_scalar_fields_3d(const orc_grid *g, double dt, double *q,
                                  const double *sq, double *th,
                                  const double *sth, int nq, int moisture);

/* ---- one time step of model_driver (driver_code.f90:304-676), dry
 *      physics switched off, optional passive q categories advected with
 *      mpdata_vec_3d and null microphysics.                                 */
typedef struct {
    double dt, ptol;
    int advection_scheme;   /* 0 upwind, 1 mpdata, 2 mpdata_add */
    int kord, monotone, limiter_variant;
    int moisture, nq, ncat;
    const int *c_s, *c_e;   /* 1-based category bounds, length ncat */
    double thbase, thtop;   /* lbc/ubc for scheme 2 */
    orc_forcing forcing;
    orc_viscous viscous;    /* subgrid model in sources (viscous = 0: off) */
} orc_config;

typedef struct {
    /* three leap-frog velocity buffers; cur[] selects roles */
    double *ut, *vt, *wt, *zut, *zvt, *zwt, *tut, *tvt, *twt;
    double *th, *p, *su, *sv, *sw, *psrc, *div, *sth;
    double *q, *sq;                       /* nq fields (may be NULL) */
    double *ubar, *vbar, *wbar, *thbar, *qbar;   /* kp+2 (qbar: nq*(kp+2)) */
    double t1, t2;                        /* saved lbc/ubc of theta */
    double *q1, *q2;                      /* lbc/ubc per q (length nq) */
    int n;                                /* steps taken (drives rotation) */
    int bicgstab_first;
    int last_iters;
    double last_err;
    double *vism, *vist, *strain;         /* subgrid fields (viscous only) */
} orc_state;

/* ---- PAMM sedimentation transport (dcm_oracle_col.c): mpdata_vec_1d of
 *      one column (pamm/sfvt/advection_1d.F90:463-778; w, dz, dzn, rhoa,
 *      rhoan as w(-l_h+1:kp+r_h), psi_in(-r_h+1:kp+r_h, 1:nq)), and ncol
 *      columns with the caller's nsub passes of dt/nsub each
 *      (pamm/microphysics.f90:3139-3183).                                     */
void orc_mpdata_vec_1d(double dt, const double *dz, const double *dzn, const double *rhoa,
                       const double *rhoan, int kp, int nq, int l_h, int r_h, const double *w,
                       double *psi_in, int kord, int monotone, int neumann);
void orc_mpdata_vec_1d_columns(int ncol, int kp, int nq, int l_h, int r_h, const double *dt,
                               const int *nsub, const double *dz, const double *dzn,
                               const double *rhoa, const double *rhoan, int metric_stride,
                               const double *w, double *psi, int kord, int monotone,
                               int neumann);

/* pre-loop velocity boundary fix-up (driver_code.f90:287-295) */
void orc_driver_start(const orc_grid *g, orc_state *s);
/* one pass of the time loop; returns ORC_* status of the pressure solve */
int orc_model_step(const orc_grid *g, const orc_config *c, orc_state *s);
/* current role pointers after rotation */
void orc_state_roles(const orc_state *s, double **u, double **v, double **w,
                     double **zu, double **zv, double **zw, double **tu,
                     double **tv, double **tw);

#ifdef __cplusplus
}
#endif
#endif
