/*
 * dcm_oracle_sgm.c -- CPU restatement (FP64) of the Smagorinsky subgrid
 * model of UoM-maul1609/dynamical-cloud-model (sgm/subgrid_3d.f90:38-493):
 * calculate_subgrid_3d with its richardson and monin_obukhov helpers.
 *
 * TEST INFRASTRUCTURE ONLY (the tests' parity reference).  The product never
 * links it.
 * PARITY UNPINNED: the Fortran reference cannot be compiled in this image and
 * ships no golden vectors; the restatement is cross-checked against an
 * independent numpy restatement in the tests instead.
 *
 * Statement order and the left-to-right evaluation of each Fortran
 * expression are kept (a+b+c = (a+b)+c, a*b/c = (a*b)/c; x**2 = x*x; real
 * exponents through pow / sqrt).  Layout as in dcm_oracle.c: a(0:kp+1,
 * 0:jp+1, 0:ip+1), k fastest.  Single rank: coords(3) = 0 = dims(3)-1, so
 * both the lid zeroing (:162-166) and the surface layer (:167-173) apply.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dcm_oracle.h"

#define KK (g->kp + 2)
#define JJ (g->jp + 2)
#define II (g->ip + 2)
#define A3(a, k, j, i) \
    (a)[(size_t)(k) + (size_t)KK * ((size_t)(j) + (size_t)JJ * (size_t)(i))]
#define NTOT ((size_t)KK * (size_t)JJ * (size_t)II)

/* module parameters, sgm/subgrid_3d.f90:13-16 */
static const double PRN = 0.95, SUBB = 40.0, SUBC = 16.0, SUBG = 1.2, SUBH = 0.0,
                    SUBR = 4.0, RIC = 0.25, GRAV_ = 9.81, SMALL_ = 1.e-10, KVON = 0.4;
#define SUBA (1.0 / PRN)
#define SUBF SUBA
/* richardson's guard `1.e-15` (:470) is a default-kind (single precision)
 * literal: the reference builds without -fdefault-real-8 (Makefile:37). */
#define RI_EPS ((double)1.e-15f)

static inline double sq_(double x) { return x * x; }

/* richardson, sgm/subgrid_3d.f90:448-493, for one point */
static void richardson_pt(double strain, double th_k, double th_k1, double thetan_k,
                          double thetan_k1, double dzn_k, double *fm, double *fh) {
    const double rip = GRAV_ * ((th_k1) / thetan_k1 - (th_k) / thetan_k) / dzn_k /
                       (strain + RI_EPS); /* :469-470 */
    if (rip < 0.0) {                      /* :478-481 */
        *fm = pow(1.0 - SUBC * rip, 0.5);
        *fh = SUBA * pow(1.0 - SUBB * rip, 0.5);
    } else if ((rip >= 0.0) && (rip < RIC)) { /* :482-484 */
        *fm = pow(1.0 - rip / RIC, SUBR) * (1.0 - SUBH * rip);
        *fh = SUBF * pow(1.0 - rip / RIC, SUBR) * (1.0 - SUBG * rip);
    } else {
        *fm = 0.0;
        *fh = 0.0;
    }
}

/* calculate_subgrid_3d, sgm/subgrid_3d.f90:38-357.  z is the grid's zg (only
 * z(1) is used, by monin_obukhov); dt, zn and dzn's role as in the
 * reference.  viss (nq fields) is written only when moisture is set, and sq
 * is updated only then; q / viss / sq may be NULL otherwise.               */
void orc_calculate_subgrid_3d(const orc_grid *g, const double *lamsq, double z0,
                              double z0th, const double *u, const double *v,
                              const double *w, const double *zu, const double *zv,
                              const double *zw, const double *th, int nq, const double *q,
                              double *vism, double *vist, double *viss, double *strain,
                              double *tau11, double *tau22, double *tau33, double *tau12,
                              double *tau13, double *tau23, double *su, double *sv,
                              double *sw, double *sth, double *sq, int moisture) {
    const int ip = g->ip, jp = g->jp, kp = g->kp;
    const double *dx = g->dx, *dy = g->dy, *dz = g->dz, *dxn = g->dxn, *dyn = g->dyn,
                 *dzn = g->dzn, *rhoa = g->rhoa, *rhoan = g->rhoan, *theta = g->theta,
                 *thetan = g->thetan, *z = g->zg;
    const size_t n = NTOT;
    double *fm = (double *)calloc(n, sizeof(double));
    double *fh = (double *)calloc(n, sizeof(double));

    /* strain rate on w-points, :91-133 */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                double s;
                s = sq_((A3(u, k + 1, j, i) - A3(u, k + 1, j, i - 1)) / dx[i - 1]) +
                    sq_((A3(u, k, j, i) - A3(u, k, j, i - 1)) / dx[i - 1]);
                s = s + sq_((A3(v, k + 1, j, i) - A3(v, k + 1, j - 1, i)) / dy[j - 1]) +
                    sq_((A3(v, k, j, i) - A3(v, k, j - 1, i)) / dy[j - 1]);
                s = s + sq_((A3(w, k, j, i) - A3(w, k - 1, j, i)) / dz[k - 1]) +
                    sq_((A3(w, k + 1, j, i) - A3(w, k, j, i)) / dz[k]);
                s = s + 0.5 * (sq_((A3(u, k + 1, j, i) - A3(u, k, j, i)) / dzn[k] +
                                   (A3(w, k, j, i + 1) - A3(w, k, j, i)) / dxn[i]) +
                               sq_((A3(u, k + 1, j, i - 1) - A3(u, k, j, i - 1)) / dz[k] +
                                   (A3(w, k, j, i) - A3(w, k, j, i - 1)) / dxn[i - 1]));
                s = s + 0.5 * (sq_((A3(w, k, j, i) - A3(w, k, j - 1, i)) / dyn[j - 1] +
                                   (A3(v, k + 1, j - 1, i) - A3(v, k, j - 1, i)) / dzn[k]) +
                               sq_((A3(w, k, j + 1, i) - A3(w, k, j, i)) / dyn[j] +
                                   (A3(v, k + 1, j, i) - A3(v, k, j, i)) / dzn[k]));
                /* the sixth of the eight s12 terms repeats the second (:128) */
                s = s + 0.125 *
                            (sq_((A3(u, k, j, i - 1) - A3(u, k, j - 1, i - 1)) / dyn[j - 1] +
                                 (A3(v, k, j - 1, i) - A3(v, k, j - 1, i - 1)) / dxn[i - 1]) +
                             sq_((A3(u, k, j + 1, i - 1) - A3(u, k, j, i - 1)) / dyn[j] +
                                 (A3(v, k, j, i) - A3(v, k, j, i - 1)) / dxn[i - 1]) +
                             sq_((A3(u, k, j, i) - A3(u, k, j - 1, i)) / dyn[j - 1] +
                                 (A3(v, k, j - 1, i + 1) - A3(v, k, j - 1, i)) / dxn[i]) +
                             sq_((A3(u, k, j + 1, i) - A3(u, k, j, i)) / dyn[j] +
                                 (A3(v, k, j, i + 1) - A3(v, k, j, i)) / dxn[i]) +
                             sq_((A3(u, k + 1, j, i - 1) - A3(u, k + 1, j - 1, i - 1)) /
                                     dyn[j - 1] +
                                 (A3(v, k + 1, j - 1, i) - A3(v, k + 1, j - 1, i - 1)) /
                                     dxn[i - 1]) +
                             sq_((A3(u, k, j + 1, i - 1) - A3(u, k, j, i - 1)) / dyn[j] +
                                 (A3(v, k, j, i) - A3(v, k, j, i - 1)) / dxn[i - 1]) +
                             sq_((A3(u, k + 1, j, i) - A3(u, k + 1, j - 1, i)) / dyn[j - 1] +
                                 (A3(v, k + 1, j - 1, i + 1) - A3(v, k + 1, j - 1, i)) /
                                     dxn[i]) +
                             sq_((A3(u, k + 1, j + 1, i) - A3(u, k + 1, j, i)) / dyn[j] +
                                 (A3(v, k + 1, j, i + 1) - A3(v, k + 1, j, i)) / dxn[i]));
                A3(strain, k, j, i) = s;
            }

    /* Richardson number functions, :137 -> :464-491 */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++)
                richardson_pt(A3(strain, k, j, i), A3(th, k, j, i), A3(th, k + 1, j, i),
                              thetan[k], thetan[k + 1], dzn[k], &A3(fm, k, j, i),
                              &A3(fh, k, j, i));

    /* viscosities on w-points, :142-160 */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                A3(vism, k, j, i) = lamsq[k] * sqrt(A3(strain, k, j, i)) * A3(fm, k, j, i);
                A3(vist, k, j, i) =
                    lamsq[k] * sqrt(A3(strain, k, j, i)) * A3(fh, k, j, i) * rhoa[k];
            }
    /* lid, :162-166 (all columns, halos included) */
    for (int i = 0; i <= ip + 1; i++)
        for (int j = 0; j <= jp + 1; j++)
            for (int k = kp - 1; k <= kp; k++) {
                A3(vism, k, j, i) = 0.0;
                A3(vist, k, j, i) = 0.0;
            }
    /* surface layer, monin_obukhov (:171 -> :393-429) */
    {
        const double z1 = z[1];
        const double kv2 = KVON * KVON;
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++) {
                const double vmag =
                    0.5 * sqrt(sq_(A3(u, 1, j, i) + A3(u, 1, j, i - 1)) +
                               sq_(A3(v, 1, j, i) + A3(v, 1, j - 1, i))) +
                    SMALL_;
                const double dth = A3(th, 1, j, i) + thetan[1] - theta[0];
                const double rib = GRAV_ * dth * sq_(z1 - z0) /
                                   (theta[0] * sq_(vmag) * (z1 - z0th));
                double gm, gh;
                if (rib <= 0.0) {
                    gm = 1.0 - 9.4 * rib /
                                   (1.0 + 70.0 * kv2 * sqrt(fabs(rib * z1 / z0)) /
                                              sq_(log(z1 / z0)));
                    gh = 1.0 - 9.4 * rib /
                                   (1.0 + 50.0 * kv2 * sqrt(fabs(rib * z1 / z0)) /
                                              sq_(log(z1 / z0)));
                } else {
                    gm = 1.0 / sq_(1.0 + 4.7 * rib);
                    gh = 1.0 / sq_(1.0 + 4.7 * rib);
                }
                const double ustar = KVON * vmag / log(z1 / z0) * sqrt(gm);
                const double thstar =
                    kv2 * vmag * dth / (ustar * PRN * sq_(log(z1 / z0))) * gh;
                A3(vism, 0, j, i) = sq_(ustar) * (z1 - z0) / vmag;
                A3(vist, 0, j, i) = ustar * thstar / (dth / (z1 - z0th) + SMALL_);
            }
    }
    /* :177-180 */
    orc_exchange_full_wo(g, vism);
    orc_exchange_full_wo(g, vist);
    if (moisture) /* :182-187 */
        for (int m = 0; m < nq; m++) memcpy(viss + (size_t)m * n, vist, n * sizeof(double));

    /* tau on p-points in the vertical, :191-207 */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                const double vm = A3(vism, k, j, i) + A3(vism, k - 1, j, i);
                A3(tau11, k, j, i) = rhoan[k] * 1.0 * vm *
                                     (A3(zu, k, j, i) - A3(zu, k, j, i - 1)) / dx[i - 1];
                A3(tau22, k, j, i) = rhoan[k] * 1.0 * vm *
                                     (A3(zv, k, j, i) - A3(zv, k, j - 1, i)) / dy[j - 1];
                A3(tau33, k, j, i) = rhoan[k] * 1.0 * vm *
                                     (A3(zw, k, j, i) - A3(zw, k - 1, j, i)) / dz[k - 1];
                A3(tau12, k, j, i) =
                    rhoan[k] * 0.125 *
                    (A3(vism, k, j, i) + A3(vism, k, j + 1, i) + A3(vism, k - 1, j, i) +
                     A3(vism, k - 1, j + 1, i) + A3(vism, k, j, i + 1) +
                     A3(vism, k, j + 1, i + 1) + A3(vism, k - 1, j, i + 1) +
                     A3(vism, k - 1, j + 1, i + 1)) *
                    ((A3(zu, k, j + 1, i) - A3(zu, k, j, i)) / dyn[j] +
                     (A3(zv, k, j, i + 1) - A3(zv, k, j, i)) / dxn[i]);
            }
    /* tau on w-points in the vertical, :211-222 */
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++)
            for (int k = 1; k <= kp; k++) {
                A3(tau13, k, j, i) =
                    rhoa[k] * 0.5 * (A3(vism, k, j, i) + A3(vism, k, j, i + 1)) *
                    ((A3(zu, k + 1, j, i) - A3(zu, k, j, i)) / dzn[k] +
                     (A3(zw, k, j, i + 1) - A3(zw, k, j, i)) / dxn[i]);
                A3(tau23, k, j, i) =
                    rhoa[k] * 0.5 * (A3(vism, k, j, i) + A3(vism, k, j + 1, i)) *
                    ((A3(zw, k, j + 1, i) - A3(zw, k, j, i)) / dyn[j] +
                     (A3(zv, k + 1, j, i) - A3(zv, k, j, i)) / dzn[k]);
            }
    /* :226-237 */
    orc_exchange_along_dim(g, tau11, 0.0, 0.0);
    orc_exchange_along_dim(g, tau22, 0.0, 0.0);
    orc_exchange_along_dim(g, tau33, 0.0, 0.0);
    orc_exchange_along_dim(g, tau12, 0.0, 0.0);
    orc_exchange_along_dim(g, tau13, 0.0, 0.0);
    orc_exchange_along_dim(g, tau23, 0.0, 0.0);

    /* momentum sources of the stresses, :240-276 (ktmp = kp-1, ktmp1 = 2) */
    const int ktmp = kp - 1, ktmp1 = 2;
#pragma omp parallel for schedule(static)
    for (int i = 1; i <= ip; i++)
        for (int j = 1; j <= jp; j++) {
            for (int k = 1; k <= ktmp; k++)
                A3(sw, k, j, i) =
                    A3(sw, k, j, i) +
                    ((A3(tau33, k + 1, j, i) - A3(tau33, k, j, i)) / dzn[k] +
                     (A3(tau13, k, j, i) - A3(tau13, k, j, i - 1)) / dx[i - 1] +
                     (A3(tau23, k, j, i) - A3(tau23, k, j - 1, i)) / dy[j - 1]);
            for (int k = ktmp1; k <= ktmp; k++) {
                A3(su, k, j, i) =
                    A3(su, k, j, i) +
                    ((A3(tau11, k, j, i + 1) - A3(tau11, k, j, i)) / dxn[i] +
                     (A3(tau12, k, j, i) - A3(tau12, k, j - 1, i)) / dy[j - 1] +
                     (A3(tau13, k, j, i) - A3(tau13, k - 1, j, i)) / dz[k - 1]);
                A3(sv, k, j, i) =
                    A3(sv, k, j, i) +
                    ((A3(tau22, k, j + 1, i) - A3(tau22, k, j, i)) / dyn[j] +
                     (A3(tau12, k, j, i) - A3(tau12, k, j, i - 1)) / dx[i - 1] +
                     (A3(tau23, k, j, i) - A3(tau23, k - 1, j, i)) / dz[k - 1]);
            }
        }
    /* :279-284 */
    orc_exchange_full(g, su, 0.0, 0.0);
    orc_exchange_full(g, sv, 0.0, 0.0);
    orc_exchange_full(g, sw, 0.0, 0.0);

    /* diffusion of a scalar, :289-311 (th) and :319-341 (each q); vist
     * already carries rhoa */
    for (int m = -1; m < (moisture ? nq : 0); m++) {
        const double *s = m < 0 ? th : q + (size_t)m * n;
        double *ds = m < 0 ? sth : sq + (size_t)m * n;
#pragma omp parallel for schedule(static)
        for (int i = 1; i <= ip; i++)
            for (int j = 1; j <= jp; j++)
                for (int k = 1; k <= kp; k++)
                    A3(ds, k, j, i) =
                        A3(ds, k, j, i) +
                        (0.25 *
                             ((A3(vist, k, j, i) + A3(vist, k, j, i - 1) + A3(vist, k - 1, j, i) +
                               A3(vist, k - 1, j, i - 1)) *
                                  (A3(s, k, j, i - 1) - A3(s, k, j, i)) / dxn[i - 1] -
                              (A3(vist, k, j, i + 1) + A3(vist, k, j, i) +
                               A3(vist, k - 1, j, i + 1) + A3(vist, k - 1, j, i)) *
                                  (A3(s, k, j, i) - A3(s, k, j, i + 1)) / dxn[i]) /
                             dx[i - 1] +
                         0.25 *
                             ((A3(vist, k, j, i) + A3(vist, k, j - 1, i) + A3(vist, k - 1, j, i) +
                               A3(vist, k - 1, j - 1, i)) *
                                  (A3(s, k, j - 1, i) - A3(s, k, j, i)) / dyn[j - 1] -
                              (A3(vist, k, j + 1, i) + A3(vist, k, j, i) +
                               A3(vist, k - 1, j + 1, i) + A3(vist, k - 1, j, i)) *
                                  (A3(s, k, j, i) - A3(s, k, j + 1, i)) / dyn[j]) /
                             dy[j - 1] +
                         (A3(vist, k - 1, j, i) * (A3(s, k - 1, j, i) - A3(s, k, j, i)) /
                              dz[k - 1] -
                          A3(vist, k, j, i) * (A3(s, k, j, i) - A3(s, k + 1, j, i)) / dz[k]) /
                             dz[k - 1]) /
                            rhoan[k];
        orc_exchange_full(g, ds, 0.0, 0.0); /* :315-316, :344-345 */
    }
    free(fm);
    free(fh);
}
