/*
 * dcm_oracle.c -- CPU restatement (FP64) of the reference dynamical-core
 * timestep of UoM-maul1609/dynamical-cloud-model.
 *
 * TEST INFRASTRUCTURE ONLY (the tests' parity reference and the timed CPU
 * baseline).  The product never links it.  PARITY UNPINNED: the Fortran reference cannot be
 * compiled in this image and ships no golden vectors; see dcm_oracle.h.
 * Instead, independent numpy restatements of the same Fortran, array
 * statement by array statement (the tests/..._np.py files), agree with this file bit
 * for bit: the pressure solve, sources, advance_momentum, divergence_calc,
 * adv_ref_state, the donor cell, the three MPDATA entry points with both
 * limiters, the subgrid model (dcm_oracle_sgm.c) and the whole dry time step
 * of model_driver (tests/test_oracle.py).
 *
 * Every routine restates one reference routine statement by statement, in
 * the reference's evaluation order (Fortran evaluates a+b+c and a*b/c left to
 * right; parentheses are kept), on the reference's own Fortran layout.  Each
 * function cites the file:line it follows.  Halo exchanges follow the
 * single-rank (dims = [1,1,1]) branches of mpi_module.f90 under MPICH, where
 * MPI_PROC_NULL = -1.
 */
#include "dcm_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define SMALL 1e-60 /* pamm/sfvt/advection_3d.F90:19 */
#define GRAV 9.81   /* dynamics.f90:18 */

static int g_par_reduce = 0;

void orc_set_threads(int nthreads, int parallel_reductions) {
#ifdef _OPENMP
    if (nthreads > 0) omp_set_num_threads(nthreads);
#else
    (void)nthreads;
#endif
    g_par_reduce = parallel_reductions;
}

/* Fortran a(0:kp+1, 0:jp+1, 0:ip+1), k fastest */
#define KK (g->kp + 2)
#define JJ (g->jp + 2)
#define II (g->ip + 2)
#define A3(a, k, j, i) \
    (a)[(size_t)(k) + (size_t)KK * ((size_t)(j) + (size_t)JJ * (size_t)(i))]
#define NTOT ((size_t)KK * (size_t)JJ * (size_t)II)

static double *falloc(const orc_grid *g) {
    return (double *)calloc(NTOT, sizeof(double));
}

static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

/* ------------------------------------------------------------------------ */
/* halo exchange                                                            */
/* ------------------------------------------------------------------------ */

/* exchange_along_dim_wo, mpi_module.f90:1285-1494: x faces then y faces for
 * k = 1..kp only; top and bottom untouched.                               */
void orc_exchange_along_dim_wo(const orc_grid *g, double *a) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    for (int j = 1; j <= jp; j++)
        for (int k = 1; k <= kp; k++) {
            A3(a, k, j, 0) = A3(a, k, j, ip);
            A3(a, k, j, ip + 1) = A3(a, k, j, 1);
        }
    for (int i = 1; i <= ip; i++)
        for (int k = 1; k <= kp; k++) {
            A3(a, k, 0, i) = A3(a, k, jp, i);
            A3(a, k, jp + 1, i) = A3(a, k, 1, i);
        }
}

/* exchange_along_dim, mpi_module.f90:700-910: faces (self-copy branch
 * :857-873), then with no rank above/below (s_top == s_bottom == -1) the
 * whole top / bottom planes are set to ubc / lbc (:874-883).              */
void orc_exchange_along_dim(const orc_grid *g, double *a, double lbc,
                            double ubc) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    orc_exchange_along_dim_wo(g, a);
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++) A3(a, kp + 1, j, i) = ubc;
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++) A3(a, 0, j, i) = lbc;
}

/* The 12 edges and 8 corners written after the face exchange by both
 * exchange_full (mpi_module.f90:965-1136) and exchange_full_wo (:1549-1720).
 * Their send buffers are pre-filled with this rank's own data (:1180,
 * :1244-1246, :1764, :1828-1830); with dims(3) = 1 every up/down neighbour is
 * MPI_PROC_NULL, the receive is a no-op, and the buffers are written
 * unconditionally (edges :1113-1126, :1697-1710) or because recv /= id
 * (corners :1129-1136, :1713-1720).  Net effect: each edge and corner holds
 * the fully periodic image of an interior cell.                             */
static void edges_and_corners(const orc_grid *g, double *a) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    /* edges along k (ws_bt, wn_bt, es_bt, en_bt) */
    for (int k = 1; k <= kp; k++) {
        A3(a, k, jp + 1, ip + 1) = A3(a, k, 1, 1);
        A3(a, k, 0, ip + 1) = A3(a, k, jp, 1);
        A3(a, k, jp + 1, 0) = A3(a, k, 1, ip);
        A3(a, k, 0, 0) = A3(a, k, jp, ip);
    }
    /* edges along i (bs_we, bn_we, ts_we, tn_we) */
    for (int i = 1; i <= ip; i++) {
        A3(a, kp + 1, jp + 1, i) = A3(a, 1, 1, i);
        A3(a, kp + 1, 0, i) = A3(a, 1, jp, i);
        A3(a, 0, jp + 1, i) = A3(a, kp, 1, i);
        A3(a, 0, 0, i) = A3(a, kp, jp, i);
    }
    /* edges along j (bw_sn, be_sn, tw_sn, te_sn) */
    for (int j = 1; j <= jp; j++) {
        A3(a, kp + 1, j, ip + 1) = A3(a, 1, j, 1);
        A3(a, kp + 1, j, 0) = A3(a, 1, j, ip);
        A3(a, 0, j, ip + 1) = A3(a, kp, j, 1);
        A3(a, 0, j, 0) = A3(a, kp, j, ip);
    }
    /* corners (wsb, wnb, wst, wnt, esb, enb, est, ent) */
    A3(a, kp + 1, jp + 1, ip + 1) = A3(a, 1, 1, 1);
    A3(a, kp + 1, 0, ip + 1) = A3(a, 1, jp, 1);
    A3(a, 0, jp + 1, ip + 1) = A3(a, kp, 1, 1);
    A3(a, 0, 0, ip + 1) = A3(a, kp, jp, 1);
    A3(a, kp + 1, jp + 1, 0) = A3(a, 1, 1, ip);
    A3(a, kp + 1, 0, 0) = A3(a, 1, jp, ip);
    A3(a, 0, jp + 1, 0) = A3(a, kp, 1, ip);
    A3(a, 0, 0, 0) = A3(a, kp, jp, ip);
}

/* exchange_full, mpi_module.f90:926-1271: exchange_along_dim (faces, then
 * the top / bottom planes set to ubc / lbc), then the edges and corners.
 * Net effect: every halo cell holds the fully periodic image of an interior
 * cell, except the interior of the top and bottom planes (ubc / lbc).      */
void orc_exchange_full(const orc_grid *g, double *a, double lbc, double ubc) {
    orc_exchange_along_dim(g, a, lbc, ubc);
    edges_and_corners(g, a);
}

/* exchange_full_wo, mpi_module.f90:1511-1855: exchange_along_dim_wo (faces
 * for k = 1..kp only), then the same edges and corners.  The interior of the
 * top and bottom planes (k = 0 and kp+1, j = 1..jp, i = 1..ip) is left as it
 * was; every other halo cell holds the periodic image of an interior cell
 * (so k = 0 halo columns take level kp's values and k = kp+1 level 1's).   */
void orc_exchange_full_wo(const orc_grid *g, double *a) {
    orc_exchange_along_dim_wo(g, a);
    edges_and_corners(g, a);
}

/* ------------------------------------------------------------------------ */
/* pressure solver                                                          */
/* ------------------------------------------------------------------------ */

/* set_mat_a, dynamics.f90:84-96 (a_c = 0, :62; halo a_p = 1, :55) */
static inline double ae_(const orc_grid *g, int i) {
    return 1.0 / (g->dx[i - 1] * g->dxn[i]);
}
static inline double aw_(const orc_grid *g, int i) {
    return 1.0 / (g->dx[i - 1] * g->dxn[i - 1]);
}
static inline double an_(const orc_grid *g, int j) {
    return 1.0 / (g->dy[j - 1] * g->dyn[j]);
}
static inline double as_(const orc_grid *g, int j) {
    return 1.0 / (g->dy[j - 1] * g->dyn[j - 1]);
}
static inline double au_(const orc_grid *g, int k) {
    return 1.0 / (g->dz[k - 1] * g->dzn[k]);
}
static inline double ad_(const orc_grid *g, int k) {
    return 1.0 / (g->dz[k - 1] * g->dzn[k - 1]);
}
static inline double ap_(const orc_grid *g, int k, int j, int i) {
    return -1.0 / (g->dx[i - 1] * g->dxn[i]) -
           1.0 / (g->dx[i - 1] * g->dxn[i - 1]) -
           1.0 / (g->dy[j - 1] * g->dyn[j]) -
           1.0 / (g->dy[j - 1] * g->dyn[j - 1]) -
           1.0 / (g->dz[k - 1] * g->dzn[k]) -
           1.0 / (g->dz[k - 1] * g->dzn[k - 1]);
}
static inline int interior(const orc_grid *g, int k, int j, int i) {
    return k >= 1 && k <= g->kp && j >= 1 && j <= g->jp && i >= 1 &&
           i <= g->ip;
}
static inline double ap_all(const orc_grid *g, int k, int j, int i) {
    return interior(g, k, j, i) ? ap_(g, k, j, i) : 1.0;
}

/* inn_prod, dynamics.f90:458-482 (serial i, j, k order; Allreduce of one
 * rank is the identity) */
double orc_inn_prod(const orc_grid *g, const double *x, const double *y) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    double s = 0.0;
    if (g_par_reduce) {
#pragma omp parallel for reduction(+ : s) schedule(static)
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++) s += A3(x, k, j, i) * A3(y, k, j, i);
        return s;
    }
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) s += A3(x, k, j, i) * A3(y, k, j, i);
    return s;
}

/* mat_ax, dynamics.f90:187-229 */
void orc_mat_ax(const orc_grid *g, double *x, double *ax) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    orc_exchange_along_dim(g, x, 0.0, 0.0);
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++) {
            A3(x, 0, j, i) = A3(x, 1, j, i);
            A3(x, kp + 1, j, i) = A3(x, kp, j, i);
        }
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < NTOT; q++) ax[q] = 0.0;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                A3(ax, k, j, i) = aw_(g, i) * A3(x, k, j, i - 1) +
                                  ae_(g, i) * A3(x, k, j, i + 1) +
                                  as_(g, j) * A3(x, k, j - 1, i) +
                                  an_(g, j) * A3(x, k, j + 1, i) +
                                  ad_(g, k) * A3(x, k - 1, j, i) +
                                  au_(g, k) * A3(x, k + 1, j, i) +
                                  ap_(g, k, j, i) * A3(x, k, j, i) + 0.0;
            }
}

/* precondition, dynamics.f90:241-270 (whole-array statements include the
 * halo, where a_p = 1) */
void orc_precondition(const orc_grid *g, const double *r, double *s,
                      int prit) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    double *t = falloc(g);
#pragma omp parallel for schedule(static)
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++)
            for (int k = 0; k <= kp + 1; k++)
                A3(s, k, j, i) = A3(r, k, j, i) / ap_all(g, k, j, i);
    for (int it = 1; it <= prit; it++) {
        orc_mat_ax(g, s, t);
#pragma omp parallel for schedule(static)
        for (int i = 0; i <= ip + 1; i++)
            for (int j = 0; j <= jp + 1; j++)
                for (int k = 0; k <= kp + 1; k++)
                    A3(s, k, j, i) = A3(s, k, j, i) +
                                     (A3(r, k, j, i) - A3(t, k, j, i)) /
                                         ap_all(g, k, j, i);
    }
    free(t);
}

/* Breakdown threshold of bicgstab.  The reference's tiny = 1.e-16 is a
 * default-real (single precision) literal, :321; a test may raise it with
 * orc_set_breakdown_tiny to reach the breakdown stop (:414-417) on a
 * well-posed system.  A negative value restores the reference's. */
static double g_tiny = -1.0;
void orc_set_breakdown_tiny(double tiny) { g_tiny = tiny < 0.0 ? -1.0 : tiny; }

/* bicgstab, dynamics.f90:293-444 */
int orc_bicgstab(const orc_grid *g, double *x, double *b, const double *sw,
                 double tol, int test_solver, int *first_call, int itmax,
                 int *iters, double *err_out) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const size_t n = NTOT;
    const double tiny = g_tiny >= 0.0 ? g_tiny : (double)1.e-16f; /* :321 */
    const int prit = 3; /* :322 */
    double sc_err, err, rho, alf, omg, bet, nrm, tt, ts;
    int status = ORC_OK;
    if (*first_call) {
        if (test_solver) {
            for (int i = 1; i <= ip; i++)
                for (int j = 1; j <= jp; j++)
                    for (int k = 1; k <= kp; k++)
                        A3(b, k, j, i) =
                            exp(-1.0 / 5.e6 *
                                (g->xg[i] * g->xg[i] + g->yg[j] * g->yg[j] +
                                 pow(g->zg[k] - 4000.0, 2.0)));
        }
        *first_call = 0;
    }
    double *ax = falloc(g), *r = falloc(g), *cr = falloc(g), *cs = falloc(g),
           *p = falloc(g), *v1 = falloc(g), *t = falloc(g), *s = falloc(g);

    sc_err = sqrt(orc_inn_prod(g, b, b));
    sc_err = dmax(sc_err, 0.01);

    orc_mat_ax(g, x, ax);
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < n; q++) {
        r[q] = b[q] - ax[q];
        cr[q] = r[q];
        p[q] = 0.0;
        v1[q] = 0.0;
    }
    err = sqrt(orc_inn_prod(g, r, r)) / sc_err;
    *iters = 0;
    if (err < tol) {
        *err_out = err;
        goto done; /* early return skips the halo fix-up (:383) */
    }
    alf = 1.0;
    omg = 1.0;
    nrm = 1.0;
    {
        int it;
        for (it = 1; it <= itmax; it++) {
            rho = orc_inn_prod(g, r, cr);
            bet = (rho / nrm) * (alf / omg);
#pragma omp parallel for schedule(static)
            for (size_t q = 0; q < n; q++) t[q] = r[q] - bet * (omg * v1[q]);
            orc_precondition(g, t, s, prit);
#pragma omp parallel for schedule(static)
            for (size_t q = 0; q < n; q++) p[q] = s[q] + bet * p[q];
            orc_mat_ax(g, p, v1);
            nrm = orc_inn_prod(g, cr, v1);
            alf = rho / nrm;
#pragma omp parallel for schedule(static)
            for (size_t q = 0; q < n; q++) s[q] = r[q] - alf * v1[q];
            orc_precondition(g, s, cs, prit);
            orc_mat_ax(g, cs, t);
            tt = orc_inn_prod(g, t, t);
            ts = orc_inn_prod(g, t, s);
            omg = ts / tt;
            if (fabs(omg) < tiny) {
                status = ORC_E_BREAKDOWN; /* :414-417 stop */
                *iters = it;
                *err_out = err;
                goto done;
            }
#pragma omp parallel for schedule(static)
            for (size_t q = 0; q < n; q++) {
                x[q] = x[q] + alf * p[q] + omg * cs[q];
                r[q] = s[q] - omg * t[q];
            }
            err = sqrt(orc_inn_prod(g, r, r)) / sc_err;
            nrm = rho;
            if (err < tol) break;
        }
        *iters = it > itmax ? itmax : it;
    }
    *err_out = err;
    if (err > tol) {
        status = ORC_E_NOCONV; /* :431-434 stop */
        goto done;
    }
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++) A3(x, kp + 1, j, i) = A3(x, kp, j, i);
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++)
            A3(x, 0, j, i) = A3(x, 1, j, i) - A3(sw, 0, j, i) * g->dzn[0];
done:
    free(ax); free(r); free(cr); free(cs); free(p); free(v1); free(t); free(s);
    return status;
}

/* ------------------------------------------------------------------------ */
/* sources and momentum                                                     */
/* ------------------------------------------------------------------------ */

/* sources, dynamics.f90:639-1000; vis == NULL or vis->viscous == 0 is the
 * viscous = .false. branch */
static int sources_impl(const orc_grid *g, const orc_forcing *f, const orc_viscous *vis,
                        const double *ubar, const double *vbar, const double *wbar,
                        const double *thbar, const double *zu, const double *zv,
                        const double *zw, const double *u, const double *v, const double *w,
                        const double *th, int nq, const double *q, int moisture,
                        double *vism, double *vist, double *strain, double *su, double *sv,
                        double *sw, double *sth, double *sq, double *rhs) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const double *dx = g->dx, *dy = g->dy, *dz = g->dz, *dxn = g->dxn,
                 *dyn = g->dyn, *dzn = g->dzn, *rhoa = g->rhoa,
                 *rhoan = g->rhoan, *theta = g->theta;
    (void)vbar;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++) /* :743 i = 2-l_h, ip */
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++)
                A3(su, k, j, i) =
                    rhoan[k] *
                    (((A3(u, k, j, i - 1) * (A3(u, k, j, i) + A3(u, k, j, i - 1)) -
                       A3(u, k, j, i + 1) * (A3(u, k, j, i) + A3(u, k, j, i + 1))) /
                          (2.0 * (dx[i] + dx[i - 1])) +
                      (A3(u, k, j - 1, i) * (A3(v, k, j - 1, i) + A3(v, k, j - 1, i + 1)) -
                       A3(u, k, j + 1, i) * (A3(v, k, j, i) + A3(v, k, j, i + 1))) /
                          (2.0 * (dyn[j] + dyn[j - 1])) +
                      (A3(u, k - 1, j, i) * (A3(w, k - 1, j, i) + A3(w, k - 1, j, i + 1)) -
                       A3(u, k + 1, j, i) * (A3(w, k, j, i) + A3(w, k, j, i + 1))) /
                          (2.0 * (dzn[k] + dzn[k - 1]))));
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++) /* :762 */
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++)
                A3(sv, k, j, i) =
                    rhoan[k] *
                    (((A3(v, k, j, i - 1) * (A3(u, k, j, i - 1) + A3(u, k, j + 1, i - 1)) -
                       A3(v, k, j, i + 1) * (A3(u, k, j, i) + A3(u, k, j + 1, i))) /
                          (2.0 * (dxn[i] + dxn[i - 1])) +
                      (A3(v, k, j - 1, i) * (A3(v, k, j, i) + A3(v, k, j - 1, i)) -
                       A3(v, k, j + 1, i) * (A3(v, k, j, i) + A3(v, k, j + 1, i))) /
                          (2.0 * (dy[j] + dy[j - 1])) +
                      (A3(v, k - 1, j, i) * (A3(w, k - 1, j, i) + A3(w, k - 1, j + 1, i)) -
                       A3(v, k + 1, j, i) * (A3(w, k, j, i) + A3(w, k, j + 1, i))) /
                          (2.0 * (dzn[k] + dzn[k - 1]))));
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++) /* :781 */
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++)
                A3(sw, k, j, i) =
                    rhoa[k] *
                    (((A3(w, k, j, i - 1) * (A3(u, k, j, i - 1) + A3(u, k + 1, j, i - 1)) -
                       A3(w, k, j, i + 1) * (A3(u, k, j, i) + A3(u, k + 1, j, i))) /
                          (2.0 * (dxn[i] + dxn[i - 1])) +
                      (A3(w, k, j - 1, i) * (A3(v, k, j - 1, i) + A3(v, k + 1, j - 1, i)) -
                       A3(w, k, j + 1, i) * (A3(v, k, j, i) + A3(v, k + 1, j, i))) /
                          (2.0 * (dyn[j] + dyn[j - 1])) +
                      (A3(w, k - 1, j, i) * (A3(w, k, j, i) + A3(w, k - 1, j, i)) -
                       A3(w, k + 1, j, i) * (A3(w, k, j, i) + A3(w, k + 1, j, i))) /
                          (2.0 * (dz[k] + dz[k - 1]))) +
                     GRAV * (A3(th, k, j, i) + A3(th, k + 1, j, i)) /
                         (2.0 * theta[k] + thbar[k] + thbar[k + 1]));

    if (f && f->damping_layer) { /* :802-839 */
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++) {
                    A3(su, k, j, i) = A3(su, k, j, i) +
                                      rhoan[k] * f->dampfacn[k] * (A3(zu, k, j, i) - ubar[k]);
                }
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++)
                    A3(sv, k, j, i) = A3(sv, k, j, i) +
                                      rhoan[k] * f->dampfacn[k] * (A3(zv, k, j, i) - vbar[k]);
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++)
                    A3(sw, k, j, i) = A3(sw, k, j, i) +
                                      rhoa[k] * f->dampfac[k] * (A3(zw, k, j, i) - 0.0);
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++)
                    A3(sth, k, j, i) = A3(sth, k, j, i) + f->dampfacn[k] * (A3(th, k, j, i) - 0.0);
    }
    if (f && f->forcing) { /* :841-860 */
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++)
                    A3(su, k, j, i) = A3(su, k, j, i) -
                                      rhoan[k] * (A3(zu, k, j, i) - f->u_force[k]) / f->forcing_tau;
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++)
                    A3(sv, k, j, i) = A3(sv, k, j, i) -
                                      rhoan[k] * (A3(zv, k, j, i) - f->v_force[k]) / f->forcing_tau;
    }
    if (f && f->divergence) { /* :863-873 */
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++)
                    A3(sw, k, j, i) = A3(sw, k, j, i) - rhoan[k] * (wbar[k] - f->w_subs[k]);
    }
    if (vis && vis->viscous) {
        /* subgrid model, :878-893; its stresses are locals of sources (:736-737) */
        const size_t n = NTOT;
        double *tau = (double *)calloc(6 * n, sizeof(double));
        double *viss = (moisture && nq > 0) ? (double *)calloc((size_t)nq * n, sizeof(double))
                                            : NULL;
        orc_calculate_subgrid_3d(g, vis->lamsq, vis->z0, vis->z0th, u, v, w, zu, zv, zw, th, nq,
                                 q, vism, vist, viss, strain, tau, tau + n, tau + 2 * n,
                                 tau + 3 * n, tau + 4 * n, tau + 5 * n, su, sv, sw, sth, sq,
                                 moisture);
        free(tau);
        free(viss);
    } else {
        /* non-viscous branch: full exchange, :909-916 */
        orc_exchange_full(g, su, 0.0, 0.0);
        orc_exchange_full(g, sv, 0.0, 0.0);
        orc_exchange_full(g, sw, 0.0, 0.0);
        orc_exchange_full(g, sth, 0.0, 0.0);
    }
    /* surface / lid conditions, :922-973 */
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++) {
            A3(su, 0, j, i) = -A3(su, 1, j, i);
            A3(sv, 0, j, i) = -A3(sv, 1, j, i);
            A3(sw, 0, j, i) = 0.0;
        }
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++)
            for (int k = kp; k <= kp + 1; k++) {
                A3(sw, k, j, i) = 0.0;
                A3(su, k, j, i) = 0.0;
                A3(sv, k, j, i) = 0.0;
            }
    /* rhs of Poisson, :977-998 */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp + 1; k++)
                A3(rhs, k, j, i) =
                    ((A3(su, k, j, i) - A3(su, k, j, i - 1)) / dx[i - 1] +
                     (A3(sv, k, j, i) - A3(sv, k, j - 1, i)) / dy[j - 1] +
                     (A3(sw, k, j, i) - A3(sw, k - 1, j, i)) / dz[k - 1]);
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            A3(rhs, 0, j, i) = ((A3(su, 0, j, i) - A3(su, 0, j, i - 1)) / dx[i - 1] +
                                (A3(sv, 0, j, i) - A3(sv, 0, j - 1, i)) / dy[j - 1] +
                                (A3(sw, 0, j, i) + A3(sw, 1, j, i)) / dz[1]);
    return ORC_OK;
}

int orc_sources(const orc_grid *g, const orc_forcing *f, const double *ubar,
                const double *vbar, const double *wbar, const double *thbar,
                const double *zu, const double *zv, const double *zw,
                const double *u, const double *v, const double *w,
                const double *th, double *su, double *sv, double *sw,
                double *sth, double *rhs) {
    return sources_impl(g, f, NULL, ubar, vbar, wbar, thbar, zu, zv, zw, u, v, w, th, 0, NULL,
                        0, NULL, NULL, NULL, su, sv, sw, sth, NULL, rhs);
}

int orc_sources_viscous(const orc_grid *g, const orc_forcing *f, const orc_viscous *vis,
                        const double *ubar, const double *vbar, const double *wbar,
                        const double *thbar, const double *zu, const double *zv,
                        const double *zw, const double *u, const double *v, const double *w,
                        const double *th, int nq, const double *q, int moisture,
                        double *vism, double *vist, double *strain, double *su, double *sv,
                        double *sw, double *sth, double *sq, double *rhs) {
    return sources_impl(g, f, vis, ubar, vbar, wbar, thbar, zu, zv, zw, u, v, w, th, nq, q,
                        moisture, vism, vist, strain, su, sv, sw, sth, sq, rhs);
}

/* advance_momentum, dynamics.f90:1019-1099 */
void orc_advance_momentum(const orc_grid *g, double dt, double *u, double *v,
                          double *w, const double *zu, const double *zv,
                          const double *zw, const double *su, const double *sv,
                          const double *sw, const double *p) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 0; k <= kp; k++) {
                A3(u, k, j, i) = A3(zu, k, j, i) +
                                 ((A3(su, k, j, i) - (A3(p, k, j, i + 1) - A3(p, k, j, i)) / (g->dxn[i])) * dt) /
                                     g->rhoan[k];
                A3(v, k, j, i) = A3(zv, k, j, i) +
                                 ((A3(sv, k, j, i) - (A3(p, k, j + 1, i) - A3(p, k, j, i)) / (g->dyn[j])) * dt) /
                                     g->rhoan[k];
                A3(w, k, j, i) = A3(zw, k, j, i) +
                                 ((A3(sw, k, j, i) - (A3(p, k + 1, j, i) - A3(p, k, j, i)) / (g->dzn[k])) * dt) /
                                     g->rhoa[k];
            }
}

/* ------------------------------------------------------------------------ */
/* advection                                                                */
/* ------------------------------------------------------------------------ */

/* first_order_upstream_3d, pamm/sfvt/advection_3d.F90:39-116 */
void orc_first_order_upstream_3d(const orc_grid *g, double dt, const double *u,
                                 const double *v, const double *w, double *psi,
                                 int neumann) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const double *dxn = g->dxn, *dyn = g->dyn, *dzn = g->dzn, *rhoa = g->rhoa,
                 *rhoan = g->rhoan;
    const size_t m = (size_t)ip * jp * kp;
    double *fxr = malloc(m * sizeof(double)), *fxl = malloc(m * sizeof(double));
    double *fyr = malloc(m * sizeof(double)), *fyl = malloc(m * sizeof(double));
    double *fzr = malloc(m * sizeof(double)), *fzl = malloc(m * sizeof(double));
#define F3(a, k, j, i) \
    (a)[(size_t)((k)-1) + (size_t)kp * ((size_t)((j)-1) + (size_t)jp * (size_t)((i)-1))]
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                double uc = A3(u, k, j, i), um = A3(u, k, j, i - 1);
                double vc = A3(v, k, j, i), vm = A3(v, k, j - 1, i);
                double wc = A3(w, k, j, i), wm = A3(w, k - 1, j, i);
                F3(fxr, k, j, i) = ((uc + fabs(uc)) * A3(psi, k, j, i) +
                                    (uc - fabs(uc)) * A3(psi, k, j, i + 1)) *
                                   dt / (2.0 * dxn[i]);
                F3(fxl, k, j, i) = ((um + fabs(um)) * A3(psi, k, j, i - 1) +
                                    (um - fabs(um)) * A3(psi, k, j, i)) *
                                   dt / (2.0 * dxn[i]);
                F3(fyr, k, j, i) = ((vc + fabs(vc)) * A3(psi, k, j, i) +
                                    (vc - fabs(vc)) * A3(psi, k, j + 1, i)) *
                                   dt / (2.0 * dyn[j]);
                F3(fyl, k, j, i) = ((vm + fabs(vm)) * A3(psi, k, j - 1, i) +
                                    (vm - fabs(vm)) * A3(psi, k, j, i)) *
                                   dt / (2.0 * dyn[j]);
                F3(fzr, k, j, i) = ((wc + fabs(wc)) * rhoa[k] * A3(psi, k, j, i) +
                                    (wc - fabs(wc)) * rhoa[k] * A3(psi, k + 1, j, i)) *
                                   dt / (2.0 * dzn[k] * rhoan[k]);
                F3(fzl, k, j, i) = ((wm + fabs(wm)) * rhoa[k - 1] * A3(psi, k - 1, j, i) +
                                    (wm - fabs(wm)) * rhoa[k - 1] * A3(psi, k, j, i)) *
                                   dt / (2.0 * dzn[k] * rhoan[k]);
            }
    if (neumann == 1) { /* :98-104 */
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++) {
                F3(fzl, 1, j, i) = F3(fzr, 1, j, i);
                F3(fzr, kp, j, i) = F3(fzl, kp, j, i);
            }
    } else if (neumann == 2) { /* :105-111 */
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++) {
                F3(fzl, 1, j, i) = -F3(fzr, 1, j, i);
                F3(fzr, kp, j, i) = -F3(fzl, kp, j, i);
            }
    }
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++)
                A3(psi, k, j, i) = A3(psi, k, j, i) -
                                   (F3(fxr, k, j, i) - F3(fxl, k, j, i)) -
                                   (F3(fyr, k, j, i) - F3(fyl, k, j, i)) -
                                   (F3(fzr, k, j, i) - F3(fzl, k, j, i));
#undef F3
    free(fxr); free(fxl); free(fyr); free(fyl); free(fzr); free(fzl);
}

/* antidiffusive velocities, pamm/sfvt/advection_3d.F90:320-505 (identical
 * in mpdata_vec_3d, :1354-1539): Smolarkiewicz (1984) eqs 13/14/38, G = rho */
static void antidiffusive(const orc_grid *g, double dt, const double *ut,
                          const double *vt, const double *wt,
                          const double *pso, double *uts, double *vts,
                          double *wts) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const double *dx = g->dx, *dy = g->dy, *dz = g->dz, *dxn = g->dxn,
                 *dyn = g->dyn, *dzn = g->dzn, *rhoa = g->rhoa,
                 *rhoan = g->rhoan;
#define U(k, j, i) A3(ut, k, j, i)
#define V(k, j, i) A3(vt, k, j, i)
#define W(k, j, i) A3(wt, k, j, i)
#define P(k, j, i) A3(pso, k, j, i)
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                const double g_bar1 = rhoan[k];
                const double g_bar2 = rhoan[k];
                const double g_bar3 = 0.5 * (rhoan[k] + rhoan[k + 1]);
                const double u_div1 =
                    (rhoa[k] * (W(k, j, i) + W(k, j, i + 1)) -
                     rhoa[k - 1] * (W(k - 1, j, i) + W(k - 1, j, i + 1))) /
                        (dz[k - 1] * g_bar1) +
                    (rhoan[k] * (V(k, j, i) + V(k, j, i + 1) - V(k, j - 1, i) -
                                 V(k, j - 1, i + 1))) /
                        (dy[j - 1] * g_bar1);
                const double u_div2 =
                    (rhoa[k] * (W(k, j, i) + W(k, j + 1, i)) -
                     rhoa[k - 1] * (W(k - 1, j, i) + W(k - 1, j + 1, i))) /
                        (dz[k - 1] * g_bar2) +
                    (rhoan[k] * (U(k, j, i) + U(k, j + 1, i) - U(k, j, i - 1) -
                                 U(k, j + 1, i - 1))) /
                        (dx[i - 1] * g_bar2);
                const double u_div3 =
                    (rhoan[k] * (U(k, j, i) - U(k, j, i - 1)) +
                     rhoan[k + 1] * (U(k + 1, j, i) - U(k + 1, j, i - 1))) /
                        (dx[i - 1] * g_bar3) +
                    (rhoan[k] * (V(k, j, i) - V(k, j - 1, i)) +
                     rhoan[k + 1] * (V(k + 1, j, i) - V(k + 1, j - 1, i))) /
                        (dy[j - 1] * g_bar3);
                const double u_j_bar1 =
                    0.5 * dt * U(k, j, i) *
                    (0.25 *
                         (rhoa[k] * W(k, j, i + 1) + rhoa[k] * W(k, j, i) +
                          rhoa[k - 1] * W(k - 1, j, i + 1) +
                          rhoa[k - 1] * W(k - 1, j, i)) /
                         g_bar1 *
                         (P(k + 1, j, i + 1) + P(k + 1, j, i) - P(k - 1, j, i + 1) -
                          P(k - 1, j, i)) /
                         (P(k + 1, j, i + 1) + P(k + 1, j, i) + P(k - 1, j, i + 1) +
                          P(k - 1, j, i) + SMALL) /
                         (0.5 * (dzn[k - 1] + dzn[k])) +
                     0.25 *
                         (rhoan[k] * V(k, j, i + 1) + rhoan[k] * V(k, j, i) +
                          rhoan[k] * V(k, j - 1, i + 1) + rhoan[k] * V(k, j - 1, i)) /
                         g_bar1 *
                         (P(k, j + 1, i + 1) + P(k, j + 1, i) - P(k, j - 1, i + 1) -
                          P(k, j - 1, i)) /
                         (P(k, j + 1, i + 1) + P(k, j + 1, i) + P(k, j - 1, i + 1) +
                          P(k, j - 1, i) + SMALL) /
                         (0.5 * (dyn[j - 1] + dyn[j])));
                const double u_j_bar2 =
                    0.5 * dt * V(k, j, i) *
                    (0.25 *
                         (rhoa[k] * W(k, j + 1, i) + rhoa[k] * W(k, j, i) +
                          rhoa[k - 1] * W(k - 1, j + 1, i) +
                          rhoa[k - 1] * W(k - 1, j, i)) /
                         g_bar2 *
                         (P(k + 1, j + 1, i) + P(k + 1, j, i) - P(k - 1, j + 1, i) -
                          P(k - 1, j, i)) /
                         (P(k + 1, j + 1, i) + P(k + 1, j, i) + P(k - 1, j + 1, i) +
                          P(k - 1, j, i) + SMALL) /
                         (0.5 * (dzn[k - 1] + dzn[k])) +
                     0.25 *
                         (rhoan[k] * U(k, j + 1, i) + rhoan[k] * U(k, j, i) +
                          rhoan[k] * U(k, j + 1, i - 1) + rhoan[k] * U(k, j, i - 1)) /
                         g_bar2 *
                         (P(k, j + 1, i + 1) + P(k, j, i + 1) - P(k, j + 1, i - 1) -
                          P(k, j, i - 1)) /
                         (P(k, j + 1, i + 1) + P(k, j, i + 1) + P(k, j + 1, i - 1) +
                          P(k, j, i - 1) + SMALL) /
                         (0.5 * (dxn[i - 1] + dxn[i])));
                const double u_j_bar3 =
                    0.5 * dt * W(k, j, i) *
                    (0.25 *
                         (rhoan[k + 1] * V(k + 1, j, i) + rhoan[k] * V(k, j, i) +
                          rhoan[k + 1] * V(k + 1, j - 1, i) +
                          rhoan[k] * V(k, j - 1, i)) /
                         g_bar3 *
                         (P(k + 1, j + 1, i) + P(k, j + 1, i) - P(k + 1, j - 1, i) -
                          P(k, j - 1, i)) /
                         (P(k + 1, j + 1, i) + P(k, j + 1, i) + P(k + 1, j - 1, i) +
                          P(k, j - 1, i) + SMALL) /
                         (0.5 * (dyn[j - 1] + dyn[j])) +
                     0.25 *
                         (rhoan[k + 1] * U(k + 1, j, i) + rhoan[k] * U(k, j, i) +
                          rhoan[k + 1] * U(k + 1, j, i - 1) +
                          rhoan[k] * U(k, j, i - 1)) /
                         g_bar3 *
                         (P(k + 1, j, i + 1) + P(k, j, i + 1) - P(k + 1, j, i - 1) -
                          P(k, j, i - 1)) /
                         (P(k + 1, j, i + 1) + P(k, j, i + 1) + P(k + 1, j, i - 1) +
                          P(k, j, i - 1) + SMALL) /
                         (0.5 * (dxn[i - 1] + dxn[i])));
                double us = (fabs(U(k, j, i)) * dx[i] - dt * U(k, j, i) * U(k, j, i)) *
                                (P(k, j, i + 1) - P(k, j, i)) /
                                (P(k, j, i + 1) + P(k, j, i) + SMALL) / dxn[i] -
                            u_j_bar1;
                double vs = (fabs(V(k, j, i)) * dy[j] - dt * V(k, j, i) * V(k, j, i)) *
                                (P(k, j + 1, i) - P(k, j, i)) /
                                (P(k, j + 1, i) + P(k, j, i) + SMALL) / dyn[j] -
                            u_j_bar2;
                double ws = (fabs(W(k, j, i)) * dz[k] -
                             dt * (rhoa[k] / g_bar3) * W(k, j, i) * W(k, j, i)) *
                                (P(k + 1, j, i) - P(k, j, i)) /
                                (P(k + 1, j, i) + P(k, j, i) + SMALL) / dzn[k] -
                            u_j_bar3;
                us = us - 0.25 * dt * U(k, j, i) *
                              ((U(k, j, i + 1) - U(k, j, i - 1)) / dx[i - 1] + u_div1);
                vs = vs - 0.25 * dt * V(k, j, i) *
                              ((V(k, j + 1, i) - V(k, j - 1, i)) / dy[j - 1] + u_div2);
                ws = ws - 0.25 * dt * W(k, j, i) *
                              ((rhoa[k + 1] * W(k + 1, j, i) - rhoa[k - 1] * W(k - 1, j, i)) /
                                   (dz[k - 1] * g_bar3) +
                               u_div3);
                A3(uts, k, j, i) = us;
                A3(vts, k, j, i) = vs;
                A3(wts, k, j, i) = ws;
            }
#undef U
#undef V
#undef W
#undef P
}

static double max14(const double *x) {
    double m = x[0];
    for (int q = 1; q < 14; q++) m = dmax(m, x[q]);
    return m;
}
static double min14(const double *x) {
    double m = x[0];
    for (int q = 1; q < 14; q++) m = dmin(m, x[q]);
    return m;
}

/* FCT limiter of the linked copy, pamm/sfvt/advection_3d.F90:542-675 (also
 * mpdata_vec_3d :1576-1709): psi_max/psi_min over 14 points, rho-weighted
 * denominators, two beta arrays; writes limited velocities into *_sav.     */
static void limiter_linked(const orc_grid *g, double dt, const double *psi,
                           const double *pso, const double *ut,
                           const double *vt, const double *wt, double *uts,
                           double *vts, double *wts) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const double *dxn = g->dxn, *dyn = g->dyn, *dzn = g->dzn, *rhoa = g->rhoa,
                 *rhoan = g->rhoan;
    double *bup = falloc(g), *bdn = falloc(g);
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                double s[14] = {A3(psi, k, j, i),     A3(psi, k, j, i - 1),
                                A3(psi, k, j, i + 1), A3(psi, k, j - 1, i),
                                A3(psi, k, j + 1, i), A3(psi, k - 1, j, i),
                                A3(psi, k + 1, j, i), A3(pso, k, j, i),
                                A3(pso, k, j, i - 1), A3(pso, k, j, i + 1),
                                A3(pso, k, j - 1, i), A3(pso, k, j + 1, i),
                                A3(pso, k - 1, j, i), A3(pso, k + 1, j, i)};
                const double pmax = max14(s), pmin = min14(s);
                const double pc = A3(pso, k, j, i);
                const double denom1 =
                    dt * ((dmax(A3(ut, k, j, i - 1), 0.0) * rhoan[k] * A3(pso, k, j, i - 1) -
                           dmin(A3(ut, k, j, i), 0.0) * rhoan[k] * A3(pso, k, j, i + 1)) /
                              dxn[i] +
                          (dmax(A3(vt, k, j - 1, i), 0.0) * rhoan[k] * A3(pso, k, j - 1, i) -
                           dmin(A3(vt, k, j, i), 0.0) * rhoan[k] * A3(pso, k, j + 1, i)) /
                              dyn[j] +
                          (dmax(A3(wt, k - 1, j, i), 0.0) * rhoa[k - 1] * A3(pso, k - 1, j, i) -
                           dmin(A3(wt, k, j, i), 0.0) * rhoa[k] * A3(pso, k + 1, j, i)) /
                              dzn[k]) +
                    SMALL;
                const double denom2 =
                    dt * ((dmax(A3(ut, k, j, i), 0.0) * rhoan[k] * pc -
                           dmin(A3(ut, k, j, i - 1), 0.0) * rhoan[k] * pc) /
                              dxn[i] +
                          (dmax(A3(vt, k, j, i), 0.0) * rhoan[k] * pc -
                           dmin(A3(vt, k, j - 1, i), 0.0) * rhoan[k] * pc) /
                              dyn[j] +
                          (dmax(A3(wt, k, j, i), 0.0) * rhoa[k] * pc -
                           dmin(A3(wt, k - 1, j, i), 0.0) * rhoa[k - 1] * pc) /
                              dzn[k] +
                          SMALL);
                A3(bup, k, j, i) = rhoan[k] * (pmax - pc) / denom1;
                A3(bdn, k, j, i) = rhoan[k] * (pc - pmin) / denom2;
            }
    orc_exchange_along_dim(g, bup, 0.0, 0.0);
    orc_exchange_along_dim(g, bdn, 0.0, 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                const double uc = A3(ut, k, j, i), vc = A3(vt, k, j, i),
                             wc = A3(wt, k, j, i);
                A3(uts, k, j, i) =
                    dmin(dmin(1.0, A3(bdn, k, j, i)), A3(bup, k, j, i + 1)) * dmax(uc, 0.0) +
                    dmin(dmin(1.0, A3(bup, k, j, i)), A3(bdn, k, j, i + 1)) * dmin(uc, 0.0);
                A3(vts, k, j, i) =
                    dmin(dmin(1.0, A3(bdn, k, j, i)), A3(bup, k, j + 1, i)) * dmax(vc, 0.0) +
                    dmin(dmin(1.0, A3(bup, k, j, i)), A3(bdn, k, j + 1, i)) * dmin(vc, 0.0);
                A3(wts, k, j, i) =
                    dmin(dmin(1.0, A3(bdn, k, j, i)), A3(bup, k + 1, j, i)) * dmax(wc, 0.0) +
                    dmin(dmin(1.0, A3(bup, k, j, i)), A3(bdn, k + 1, j, i)) * dmin(wc, 0.0);
            }
    free(bup);
    free(bdn);
}

/* FCT limiter of the interface copy, sfvt/advection_3d.F90:544-704:
 * per-direction max/min over 6 points, unweighted denominators divided by
 * dx(i-1)/dy(j-1)/dz(k-1), six beta arrays.                               */
static void limiter_sfvt(const orc_grid *g, double dt, const double *psi,
                         const double *pso, const double *ut, const double *vt,
                         const double *wt, double *uts, double *vts,
                         double *wts) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const double *dx = g->dx, *dy = g->dy, *dz = g->dz;
    double *b[6];
    for (int q = 0; q < 6; q++) b[q] = falloc(g);
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                const double pc = A3(pso, k, j, i);
                double imax = dmax(dmax(dmax(dmax(dmax(A3(psi, k, j, i - 1), A3(psi, k, j, i)),
                                                   A3(psi, k, j, i + 1)),
                                              A3(pso, k, j, i - 1)),
                                         pc),
                                    A3(pso, k, j, i + 1));
                double imin = dmin(dmin(dmin(dmin(dmin(A3(psi, k, j, i - 1), A3(psi, k, j, i)),
                                                   A3(psi, k, j, i + 1)),
                                              A3(pso, k, j, i - 1)),
                                         pc),
                                    A3(pso, k, j, i + 1));
                double jmax = dmax(dmax(dmax(dmax(dmax(A3(psi, k, j - 1, i), A3(psi, k, j, i)),
                                                   A3(psi, k, j + 1, i)),
                                              A3(pso, k, j - 1, i)),
                                         pc),
                                    A3(pso, k, j + 1, i));
                double jmin = dmin(dmin(dmin(dmin(dmin(A3(psi, k, j - 1, i), A3(psi, k, j, i)),
                                                   A3(psi, k, j + 1, i)),
                                              A3(pso, k, j - 1, i)),
                                         pc),
                                    A3(pso, k, j + 1, i));
                double kmax = dmax(dmax(dmax(dmax(dmax(A3(psi, k - 1, j, i), A3(psi, k, j, i)),
                                                   A3(psi, k + 1, j, i)),
                                              A3(pso, k - 1, j, i)),
                                         pc),
                                    A3(pso, k + 1, j, i));
                double kmin = dmin(dmin(dmin(dmin(dmin(A3(psi, k - 1, j, i), A3(psi, k, j, i)),
                                                   A3(psi, k + 1, j, i)),
                                              A3(pso, k - 1, j, i)),
                                         pc),
                                    A3(pso, k + 1, j, i));
                const double denom1 =
                    (dt * ((dmax(A3(ut, k, j, i - 1), 0.0) * A3(pso, k, j, i - 1) -
                            dmin(A3(ut, k, j, i), 0.0) * A3(pso, k, j, i + 1)) /
                               dx[i - 1] +
                           (dmax(A3(vt, k, j - 1, i), 0.0) * A3(pso, k, j - 1, i) -
                            dmin(A3(vt, k, j, i), 0.0) * A3(pso, k, j + 1, i)) /
                               dy[j - 1] +
                           (dmax(A3(wt, k - 1, j, i), 0.0) * A3(pso, k - 1, j, i) -
                            dmin(A3(wt, k, j, i), 0.0) * A3(pso, k + 1, j, i)) /
                               dz[k - 1] +
                           SMALL));
                const double denom2 =
                    (dt * ((dmax(A3(ut, k, j, i), 0.0) * pc - dmin(A3(ut, k, j, i - 1), 0.0) * pc) /
                               dx[i - 1] +
                           (dmax(A3(vt, k, j, i), 0.0) * pc - dmin(A3(vt, k, j - 1, i), 0.0) * pc) /
                               dy[j - 1] +
                           (dmax(A3(wt, k, j, i), 0.0) * pc - dmin(A3(wt, k - 1, j, i), 0.0) * pc) /
                               dz[k - 1] +
                           SMALL));
                A3(b[0], k, j, i) = (imax - pc) / denom1;
                A3(b[1], k, j, i) = (pc - imin) / denom2;
                A3(b[2], k, j, i) = (jmax - pc) / denom1;
                A3(b[3], k, j, i) = (pc - jmin) / denom2;
                A3(b[4], k, j, i) = (kmax - pc) / denom1;
                A3(b[5], k, j, i) = (pc - kmin) / denom2;
            }
    for (int q = 0; q < 6; q++) orc_exchange_along_dim(g, b[q], 0.0, 0.0);
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                const double uc = A3(ut, k, j, i), vc = A3(vt, k, j, i),
                             wc = A3(wt, k, j, i);
                A3(uts, k, j, i) =
                    dmin(dmin(1.0, A3(b[1], k, j, i)), A3(b[0], k, j, i + 1)) * dmax(uc, 0.0) +
                    dmin(dmin(1.0, A3(b[0], k, j, i)), A3(b[1], k, j, i + 1)) * dmin(uc, 0.0);
                A3(vts, k, j, i) =
                    dmin(dmin(1.0, A3(b[3], k, j, i)), A3(b[2], k, j + 1, i)) * dmax(vc, 0.0) +
                    dmin(dmin(1.0, A3(b[2], k, j, i)), A3(b[3], k, j + 1, i)) * dmin(vc, 0.0);
                A3(wts, k, j, i) =
                    dmin(dmin(1.0, A3(b[5], k, j, i)), A3(b[4], k + 1, j, i)) * dmax(wc, 0.0) +
                    dmin(dmin(1.0, A3(b[4], k, j, i)), A3(b[5], k + 1, j, i)) * dmin(wc, 0.0);
            }
    for (int q = 0; q < 6; q++) free(b[q]);
}

/* shared MPDATA iteration (pamm/sfvt/advection_3d.F90:290-698 and
 * :1324-1735): antidiffusive velocities computed from field 0 of psis,
 * all nq fields upwinded with the same velocities.  psi_store is the
 * shifted input of field 0.                                               */
static void mpdata_core(const orc_grid *g, double dt, const double *u,
                        const double *v, const double *w, double *psis,
                        int nq, const double *lbc, const double *ubc,
                        int kord, int monotone, int neumann,
                        int limiter_variant) {
    const size_t n = NTOT;
    double *us1 = falloc(g), *us2 = falloc(g), *vs1 = falloc(g),
           *vs2 = falloc(g), *ws1 = falloc(g), *ws2 = falloc(g);
    double *psi_store = NULL;
    const double *ut = u, *vt = v, *wt = w;
    double *uts = us1, *vts = vs1, *wts = ws1;
    const double *psi = NULL;
    double *psi_old = psis; /* field 0 */
    if (kord > 1) {
        psi_store = malloc(n * sizeof(double));
        memcpy(psi_store, psis, n * sizeof(double));
        psi = psi_store;
    }
    int it2 = 0;
    for (int it = 1; it <= kord; it++) {
        if (it > 1) {
            it2++;
            antidiffusive(g, dt, ut, vt, wt, psi_old, uts, vts, wts);
            if (it2 % 2 == 1) {
                ut = us1; vt = vs1; wt = ws1;
                uts = us2; vts = vs2; wts = ws2;
            } else {
                ut = us2; vt = vs2; wt = ws2;
                uts = us1; vts = vs1; wts = ws1;
            }
            orc_exchange_full(g, (double *)ut, 0.0, 0.0);
            orc_exchange_full(g, (double *)vt, 0.0, 0.0);
            orc_exchange_full(g, (double *)wt, 0.0, 0.0);
        }
        if (it > 1 && monotone) {
            it2++;
            if (limiter_variant == 1)
                limiter_sfvt(g, dt, psi, psi_old, ut, vt, wt, uts, vts, wts);
            else
                limiter_linked(g, dt, psi, psi_old, ut, vt, wt, uts, vts, wts);
            ut = us2; vt = vs2; wt = ws2;
            uts = us1; vts = vs1; wts = ws1;
            orc_exchange_full(g, (double *)ut, 0.0, 0.0);
            orc_exchange_full(g, (double *)vt, 0.0, 0.0);
            orc_exchange_full(g, (double *)wt, 0.0, 0.0);
        }
        for (int q = 0; q < nq; q++) {
            orc_first_order_upstream_3d(g, dt, ut, vt, wt, psis + (size_t)q * n,
                                        neumann);
            if (it <= kord && kord >= 1)
                orc_exchange_full(g, psis + (size_t)q * n, lbc[q], ubc[q]);
        }
    }
    free(us1); free(us2); free(vs1); free(vs2); free(ws1); free(ws2);
    free(psi_store);
}

/* mpdata_3d, pamm/sfvt/advection_3d.F90:219-714 */
void orc_mpdata_3d(const orc_grid *g, double dt, const double *u,
                   const double *v, const double *w, double *psi, double *lbc,
                   double *ubc, int kord, int monotone, int neumann,
                   int limiter_variant) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const size_t n = NTOT;
    /* min over the whole array including halos, :275 */
    double mn = psi[0];
    for (size_t q = 1; q < n; q++) mn = dmin(mn, psi[q]);
    mn = dmin(dmin(mn, *lbc), *ubc);
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < n; q++) psi[q] = psi[q] - mn;
    *lbc = *lbc - mn;
    *ubc = *ubc - mn;
    double sum = 0.0; /* :282, interior, array-element order */
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) sum += A3(psi, k, j, i);
    if (sum < SMALL) { /* psi_sum .lt. small, :284-289 */
        for (size_t q = 0; q < n; q++) psi[q] = psi[q] + mn;
        *lbc = *lbc + mn;
        *ubc = *ubc + mn;
        return;
    }
    mpdata_core(g, dt, u, v, w, psi, 1, lbc, ubc, kord, monotone, neumann,
                limiter_variant);
#pragma omp parallel for schedule(static)
    for (size_t q = 0; q < n; q++) psi[q] = psi[q] + mn;
    *lbc = *lbc + mn;
    *ubc = *ubc + mn;
}

/* mpdata_vec_3d, pamm/sfvt/advection_3d.F90:1250-1753 */
void orc_mpdata_vec_3d(const orc_grid *g, double dt, const double *u,
                       const double *v, const double *w, double *psi, int nq,
                       double *lbc, double *ubc, int kord, int monotone,
                       int neumann, int limiter_variant) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const size_t n = NTOT;
    double *mn = malloc((size_t)nq * sizeof(double));
    for (int q = 0; q < nq; q++) { /* :1306-1312, interior minimum */
        double *a = psi + (size_t)q * n;
        double m = A3(a, 1, 1, 1);
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++) m = dmin(m, A3(a, k, j, i));
        m = dmin(dmin(m, lbc[q]), ubc[q]);
        mn[q] = m;
        for (size_t e = 0; e < n; e++) a[e] = a[e] - m;
        lbc[q] = lbc[q] - m;
        ubc[q] = ubc[q] - m;
    }
    double sum = 0.0; /* :1314, field 1 only */
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) sum += A3(psi, k, j, i);
    if (sum < SMALL) {
        for (int q = 0; q < nq; q++) {
            double *a = psi + (size_t)q * n;
            for (size_t e = 0; e < n; e++) a[e] = a[e] + mn[q];
            lbc[q] = lbc[q] + mn[q];
            ubc[q] = ubc[q] + mn[q];
        }
        free(mn);
        return;
    }
    mpdata_core(g, dt, u, v, w, psi, nq, lbc, ubc, kord, monotone, neumann,
                limiter_variant);
    for (int q = 0; q < nq; q++) {
        double *a = psi + (size_t)q * n;
        for (size_t e = 0; e < n; e++) a[e] = a[e] + mn[q];
        lbc[q] = lbc[q] + mn[q];
        ubc[q] = ubc[q] + mn[q];
    }
    free(mn);
}

/* adv_ref_state, pamm/sfvt/advection_3d.F90:1148-1218 (i, j include the
 * halo; k = 1..kp) */
void orc_adv_ref_state(const orc_grid *g, double dt, const double *w,
                       double *psi, const double *psi_ref) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const double *dz = g->dz, *rhoa = g->rhoa, *rhoan = g->rhoan;
#pragma omp parallel for schedule(static)
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++)
            for (int k = 1; k <= kp; k++)
                A3(psi, k, j, i) =
                    A3(psi, k, j, i) -
                    dt * (0.5 / dz[k - 1] * A3(w, k - 1, j, i) * rhoa[k - 1] *
                              (psi_ref[k] - psi_ref[k - 1]) +
                          0.5 / dz[k] * A3(w, k, j, i) * rhoa[k] *
                              (psi_ref[k + 1] - psi_ref[k])) /
                        rhoan[k];
}

/* mpdata_3d_add, pamm/sfvt/advection_3d.F90:139-190 */
void orc_mpdata_3d_add(const orc_grid *g, double dt, const double *u,
                       const double *v, const double *w, double *psi,
                       const double *psi_1d, double *lbc, double *ubc,
                       int kord, int monotone, int neumann,
                       int limiter_variant) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++)
            for (int k = 0; k <= kp + 1; k++)
                A3(psi, k, j, i) = A3(psi, k, j, i) + psi_1d[k];
    orc_mpdata_3d(g, dt, u, v, w, psi, lbc, ubc, kord, monotone, neumann,
                  limiter_variant);
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++)
            for (int k = 0; k <= kp + 1; k++)
                A3(psi, k, j, i) = A3(psi, k, j, i) - psi_1d[k];
}

/* ------------------------------------------------------------------------ */
/* diagnostics and scalar update                                           */
/* ------------------------------------------------------------------------ */

/* horizontal_means, diagnostics.f90:31-107.  Sums over (j,i) in array
 * order for k = 0..kp+1; divided by ip*jp.  (The reference's Allreduce
 * count (4+nq)*(kp+2) leaves the top levels of the last q mean unreduced;
 * qbar does not enter the dry step.)                                      */
void orc_horizontal_means(const orc_grid *g, int moisture, int nq,
                          const double *u, const double *v, const double *w,
                          const double *th, const double *q, double *ubar,
                          double *vbar, double *wbar, double *thbar,
                          double *qbar) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const double area = (double)(ip * jp);
    for (int k = 0; k <= kp + 1; k++) {
        double su = 0, sv = 0, sw = 0, st = 0;
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++) {
                su += A3(u, k, j, i);
                sv += A3(v, k, j, i);
                sw += A3(w, k, j, i);
                st += A3(th, k, j, i);
            }
        ubar[k] = su / area;
        vbar[k] = sv / area;
        wbar[k] = sw / area;
        thbar[k] = st / area;
    }
    if (moisture && q && qbar) {
        for (int n = 0; n < nq; n++) {
            const double *a = q + (size_t)n * NTOT;
            for (int k = 0; k <= kp + 1; k++) {
                double s = 0;
                for (int i = 1; i <= ip; i++)
                    for (int j = 1; j <= jp; j++) s += A3(a, k, j, i);
                qbar[(size_t)n * (kp + 2) + k] = s / area;
            }
        }
    }
}

/* divergence_calc, diagnostics.f90:120-153 */
void orc_divergence_calc(const orc_grid *g, const double *u, const double *v,
                         const double *w, double *div) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++)
                A3(div, k, j, i) =
                    g->rhoan[k] * (A3(u, k, j, i) - A3(u, k, j, i - 1)) / g->dx[i - 1] +
                    g->rhoan[k] * (A3(v, k, j, i) - A3(v, k, j - 1, i)) / g->dy[j - 1] +
                    (g->rhoa[k] * A3(w, k, j, i) - g->rhoa[k - 1] * A3(w, k - 1, j, i)) /
                        g->dz[k - 1];
}

/* advance_scalar_fields_3d, sgm/subgrid_3d.f90:582-624 (whole array) */
void orc_advance_scalar_fields_3d(const orc_grid *g, double dt, double *q,
                                  const double *sq, double *th,
                                  const double *sth, int nq, int moisture) {
    const size_t n = NTOT;
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < n; e++) th[e] = th[e] + sth[e] * dt;
    if (moisture)
        for (size_t e = 0; e < (size_t)nq * n; e++) q[e] = q[e] + sq[e] * dt;
}

/* ------------------------------------------------------------------------ */
/* the time step                                                            */
/* ------------------------------------------------------------------------ */

void orc_state_roles(const orc_state *s, double **u, double **v, double **w,
                     double **zu, double **zv, double **zw, double **tu,
                     double **tv, double **tw) {
    /* driver_code.f90:281-283 and the rotation :634-646: after n steps the
     * roles (u, zu, tu) point at buffers (0,1,2), (2,0,1), (1,2,0) for
     * n mod 3 = 0, 1, 2                                                    */
    double *U[3] = {s->ut, s->zut, s->tut};
    double *V[3] = {s->vt, s->zvt, s->tvt};
    double *W[3] = {s->wt, s->zwt, s->twt};
    static const int cu[3] = {0, 2, 1}, cz[3] = {1, 0, 2}, ct[3] = {2, 1, 0};
    const int m = s->n % 3;
    if (u) *u = U[cu[m]];
    if (v) *v = V[cu[m]];
    if (w) *w = W[cu[m]];
    if (zu) *zu = U[cz[m]];
    if (zv) *zv = V[cz[m]];
    if (zw) *zw = W[cz[m]];
    if (tu) *tu = U[ct[m]];
    if (tv) *tv = V[ct[m]];
    if (tw) *tw = W[ct[m]];
}

/* driver_code.f90:287-295 */
void orc_driver_start(const orc_grid *g, orc_state *s) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    double *zu, *zv, *zw;
    orc_state_roles(s, NULL, NULL, NULL, &zu, &zv, &zw, NULL, NULL, NULL);
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++) {
            A3(zw, 0, j, i) = -A3(zw, 1, j, i);
            A3(zu, 1, j, i) = 0.0;
            A3(zv, 1, j, i) = 0.0;
        }
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++) {
            A3(zw, kp, j, i) = -A3(zw, kp - 1, j, i);
            A3(zw, kp + 1, j, i) = 0.0;
            A3(zu, kp, j, i) = 0.0;
            A3(zv, kp, j, i) = 0.0;
        }
}

/* one pass of the time loop, driver_code.f90:304-676 (output, microphysics,
 * radiation and land surface off; the subgrid model when c->viscous is set) */
int orc_model_step(const orc_grid *g, const orc_config *c, orc_state *s) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const size_t n = NTOT;
    double *u, *v, *w, *zu, *zv, *zw, *tu, *tv, *tw;
    orc_state_roles(s, &u, &v, &w, &zu, &zv, &zw, &tu, &tv, &tw);
    const double dt = c->dt;

    memset(s->sth, 0, n * sizeof(double)); /* :340 */
    if (c->moisture && s->sq) memset(s->sq, 0, (size_t)c->nq * n * sizeof(double));

    orc_horizontal_means(g, c->moisture, c->nq, u, v, w, s->th, s->q, s->ubar,
                         s->vbar, s->wbar, s->thbar, s->qbar); /* :433 */
    orc_divergence_calc(g, u, v, w, s->div);                      /* :443 */
    if (c->viscous.viscous) { /* :455-479 with viscous = .true. */
        const size_t nn = NTOT;
        double *tmp[3] = {NULL, NULL, NULL};
        double **own[3] = {&s->vism, &s->vist, &s->strain};
        double *fld[3];
        for (int a = 0; a < 3; a++) {
            fld[a] = *own[a];
            if (!fld[a]) fld[a] = tmp[a] = (double *)calloc(nn, sizeof(double));
        }
        orc_sources_viscous(g, &c->forcing, &c->viscous, s->ubar, s->vbar, s->wbar, s->thbar,
                            zu, zv, zw, u, v, w, s->th, c->nq, s->q, c->moisture && s->q,
                            fld[0], fld[1], fld[2], s->su, s->sv, s->sw, s->sth, s->sq,
                            s->psrc);
        for (int a = 0; a < 3; a++) free(tmp[a]);
    } else {
        orc_sources(g, &c->forcing, s->ubar, s->vbar, s->wbar, s->thbar, zu, zv,
                    zw, u, v, w, s->th, s->su, s->sv, s->sw, s->sth, s->psrc);
    }
    orc_exchange_along_dim_wo(g, s->psrc); /* :485 */
    int it = 0;
    double err = 0.0;
    int st = orc_bicgstab(g, s->p, s->psrc, s->sw, c->ptol, 0,
                          &s->bicgstab_first, 9999, &it, &err); /* :496 */
    s->last_iters = it;
    s->last_err = err;
    if (st != ORC_OK) return st;
    orc_exchange_along_dim_wo(g, s->p); /* :506 */

    if (c->advection_scheme == 0 || c->advection_scheme == 1) { /* :514-529 */
        orc_adv_ref_state(g, dt, w, s->th, g->thetan);
        orc_exchange_full(g, s->th, 0.0, 0.0);
    }
    switch (c->advection_scheme) { /* :537-560 */
    case 0:
        orc_first_order_upstream_3d(g, dt, u, v, w, s->th, 0);
        orc_exchange_full(g, s->th, s->t1, s->t2);
        break;
    case 1:
        orc_mpdata_3d(g, dt, u, v, w, s->th, &s->t1, &s->t2, c->kord,
                      c->monotone, 0, c->limiter_variant);
        break;
    case 2: {
        double lb = c->thbase, ub = c->thtop;
        orc_mpdata_3d_add(g, dt, u, v, w, s->th, g->thetan, &lb, &ub, c->kord,
                          c->monotone, 0, c->limiter_variant);
        break;
    }
    default:
        return -1;
    }
    if (c->moisture && s->q) { /* :568-585 */
        for (int cat = 0; cat < c->ncat; cat++) {
            const int a = c->c_s[cat] - 1, b = c->c_e[cat] - 1;
            orc_mpdata_vec_3d(g, dt, u, v, w, s->q + (size_t)a * n, b - a + 1,
                              s->q1 + a, s->q2 + a, c->kord, c->monotone, 0,
                              c->limiter_variant);
        }
    }
    orc_advance_momentum(g, 2.0 * dt, tu, tv, tw, zu, zv, zw, s->su, s->sv,
                         s->sw, s->p); /* :592-594 */
    orc_advance_scalar_fields_3d(g, dt, s->q, s->sq, s->th, s->sth, c->nq,
                                 c->moisture); /* :601 */
#pragma omp parallel for schedule(static)
    for (size_t e = 0; e < n; e++) { /* time filter :618-626 */
        const double ut_ = 0.99 * u[e] + 0.01 * zu[e];
        const double vt_ = 0.99 * v[e] + 0.01 * zv[e];
        const double wt_ = 0.99 * w[e] + 0.01 * zw[e];
        zu[e] = 0.01 * u[e] + 0.99 * zu[e];
        zv[e] = 0.01 * v[e] + 0.99 * zv[e];
        zw[e] = 0.01 * w[e] + 0.99 * zw[e];
        u[e] = ut_;
        v[e] = vt_;
        w[e] = wt_;
    }
    s->n += 1; /* pointer rotation :634-646 */
    orc_state_roles(s, &u, &v, &w, NULL, NULL, NULL, NULL, NULL, NULL);
    orc_exchange_full(g, u, 0.0, 0.0); /* :656-661 */
    orc_exchange_full(g, v, 0.0, 0.0);
    orc_exchange_full(g, w, 0.0, 0.0);
    for (int i = 0; i <= ip + 1; i++) /* :663-674 */
        for (int j = 0; j <= jp + 1; j++) {
            A3(w, 0, j, i) = 0.0;
            A3(u, 0, j, i) = -A3(u, 1, j, i);
            A3(v, 0, j, i) = -A3(v, 1, j, i);
        }
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++) {
            A3(w, kp + 1, j, i) = 0.0;
            A3(u, kp + 1, j, i) = A3(u, kp, j, i);
            A3(v, kp + 1, j, i) = A3(v, kp, j, i);
        }
    return ORC_OK;
}
