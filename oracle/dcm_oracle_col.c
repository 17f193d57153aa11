/*
 * dcm_oracle_col.c -- CPU restatement (FP64) of the column transport that
 * the PAMM microphysics uses for sedimentation in UoM-maul1609/dynamical-
 * cloud-model: mpdata_vec_1d with first_order_upstream_1d
 * (pamm/sfvt/advection_1d.F90:35-74, 463-778), and the caller's sub-stepping
 * loop around it (pamm/microphysics.f90:3139-3145, 3158-3164, 3177-3183:
 * n_step passes of dt/n_step).
 *
 * TEST INFRASTRUCTURE ONLY (the tests' parity reference).  The product never
 * links it.
 * PARITY UNPINNED: the Fortran reference cannot be compiled in this image and
 * ships no golden vectors; the restatement is cross-checked against an
 * independent numpy restatement in the tests instead.
 *
 * Statement order and the left-to-right evaluation of each Fortran
 * expression are kept (a*b*c = (a*b)*c, a*b/c = (a*b)/c).  The Fortran
 * intrinsic sum over k is taken in index order.  Layout of one column, as the
 * caller's arrays: w, dz, dzn, rhoa, rhoan are w(-l_h+1:kp+r_h) (index k at
 * k + l_h - 1); psi is psi_in(-r_h+1:kp+r_h, 1:nq), Fortran order (index (k,
 * n) at k + r_h - 1 + (kp + 2 r_h) (n - 1)).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "dcm_oracle.h"

#define SMALL 1e-60 /* pamm/sfvt/advection_1d.F90:18 */

static double dmax(double a, double b) { return a > b ? a : b; }
static double dmin(double a, double b) { return a < b ? a : b; }

/* first_order_upstream_1d, advection_1d.F90:35-74.  w, dzn, rhoa, rhoan at
 * level k: X[k] with the caller's offset applied (pointers to level 0);
 * psi: pointer to level 0 of the field. */
static void upstream_1d(double dt, const double *dzn, const double *rhoa, const double *rhoan,
                        int kp, const double *w, double *psi, int neumann, double *fz_r,
                        double *fz_l) {
    for (int k = 1; k <= kp; k++) {
        fz_r[k] = ((w[k] + fabs(w[k])) * rhoa[k] * psi[k] +
                   (w[k] - fabs(w[k])) * rhoa[k] * psi[k + 1]) * dt /
                  (2.0 * dzn[k] * rhoan[k]);
        fz_l[k] = ((w[k - 1] + fabs(w[k - 1])) * rhoa[k - 1] * psi[k - 1] +
                   (w[k - 1] - fabs(w[k - 1])) * rhoa[k - 1] * psi[k]) * dt /
                  (2.0 * dzn[k] * rhoan[k]);
    }
    if (neumann == 1) { /* :65-67 */
        fz_l[1] = fz_r[1];
        fz_r[kp] = fz_l[kp];
    } else if (neumann == 2) { /* :68-70 */
        fz_l[1] = -fz_r[1];
        fz_r[kp] = -fz_l[kp];
    }
    for (int k = 1; k <= kp; k++) psi[k] = psi[k] - (fz_r[k] - fz_l[k]); /* :73 */
}

/* mpdata_vec_1d, advection_1d.F90:463-778, one column */
void orc_mpdata_vec_1d(double dt, const double *dz_, const double *dzn_, const double *rhoa_,
                       const double *rhoan_, int kp, int nq, int l_h, int r_h, const double *w_,
                       double *psi_in, int kord, int monotone, int neumann) {
    const int nw = kp + l_h + r_h, npsi = kp + 2 * r_h;
    /* level-0 views */
    const double *dz = dz_ + (l_h - 1), *dzn = dzn_ + (l_h - 1);
    const double *rhoa = rhoa_ + (l_h - 1), *rhoan = rhoan_ + (l_h - 1);
    const double *w = w_ + (l_h - 1);
    double *ws1b = calloc((size_t)nw, sizeof(double)), *ws2b = calloc((size_t)nw, sizeof(double));
    double *storeb = malloc((size_t)npsi * sizeof(double));
    double *pmaxb = calloc((size_t)npsi, sizeof(double)), *pminb = calloc((size_t)npsi, sizeof(double));
    double *bupb = calloc((size_t)npsi, sizeof(double)), *bdnb = calloc((size_t)npsi, sizeof(double));
    double *fz_r = malloc((size_t)(kp + 1) * sizeof(double)), *fz_l = malloc((size_t)(kp + 1) * sizeof(double));
    double *minglobal = malloc((size_t)(nq > 0 ? nq : 1) * sizeof(double));
    double *w_store1 = ws1b + (l_h - 1), *w_store2 = ws2b + (l_h - 1);
    double *psi_store = storeb + (r_h - 1);
    double *psi_max = pmaxb + (r_h - 1), *psi_min = pminb + (r_h - 1);
    double *beta_up = bupb + (r_h - 1), *beta_down = bdnb + (r_h - 1);
#define PSI(n) (psi_in + (size_t)npsi * (size_t)(n) + (r_h - 1))

    /* positive definite (:507-516) */
    for (int n = 0; n < nq; n++) {
        double *p = PSI(n);
        double m = p[1];
        for (int k = 2; k <= kp; k++) m = p[k] < m ? p[k] : m; /* minval */
        minglobal[n] = m;
        for (int k = -r_h + 1; k <= kp + r_h; k++) p[k] = p[k] - m;
    }
    double psi_sum = 0.0;
    {
        const double *p = PSI(0);
        for (int k = 1; k <= kp; k++) psi_sum += p[k]; /* :518 */
    }
    if (psi_sum < SMALL) { /* :524-529 */
        for (int n = 0; n < nq; n++) {
            double *p = PSI(n);
            for (int k = -r_h + 1; k <= kp + r_h; k++) p[k] = p[k] + minglobal[n];
        }
        goto out;
    }
    for (int k = -l_h + 1; k <= kp + r_h; k++) w_store2[k] = 0.0; /* :530 */
    const double *wt = w; /* :534-535 */
    double *wt_sav = w_store1;
    const double *psi = NULL;
    double *psi_old = PSI(0); /* :547 */
    if (kord > 1) {           /* :542-545 */
        memcpy(storeb, psi_in, (size_t)npsi * sizeof(double));
        psi = psi_store;
    }
    int it2 = 0;
    for (int it = 1; it <= kord; it++) {
        if (it > 1) { /* antidiffusive velocities, :553-635 */
            it2 = it2 + 1;
            for (int k = 1; k <= kp; k++) {
                const double g_bar3 = 0.5 * (rhoan[k] + rhoan[k + 1]);
                const double u_div3 = 0.0, u_j_bar3 = 0.0;
                double v = (fabs(wt[k]) * dz[k] - dt * (rhoa[k] / g_bar3) * wt[k] * wt[k]) *
                               (psi_old[k + 1] - psi_old[k]) /
                               (psi_old[k + 1] + psi_old[k] + SMALL) / dzn[k] -
                           u_j_bar3;
                v = v - 0.25 * dt * wt[k] *
                            ((rhoa[k + 1] * wt[k + 1] - rhoa[k - 1] * wt[k - 1]) / dz[k - 1] +
                             u_div3) /
                            g_bar3;
                wt_sav[k] = v;
            }
            double *nw_, *ns_;
            if (it2 % 2 == 1) { /* :641-648 */
                nw_ = w_store1;
                ns_ = w_store2;
            } else {
                nw_ = w_store2;
                ns_ = w_store1;
            }
            nw_[0] = nw_[1]; /* :656-657 */
            nw_[kp] = nw_[kp - 1];
            nw_[kp + 1] = nw_[kp - 1];
            wt = nw_;
            wt_sav = ns_;
        }
        if (it > 1 && monotone) { /* NFT limiter, :666-745 */
            it2 = it2 + 1;
            for (int k = 1; k <= kp; k++) {
                double mx = psi[k - 1], mn = psi[k - 1];
                const double c[5] = {psi[k], psi[k + 1], psi_old[k - 1], psi_old[k], psi_old[k + 1]};
                for (int q = 0; q < 5; q++) {
                    mx = dmax(mx, c[q]);
                    mn = dmin(mn, c[q]);
                }
                psi_max[k] = mx;
                psi_min[k] = mn;
            }
            for (int k = 1; k <= kp; k++) {
                const double denom1 = dt *
                                          (dmax(wt[k - 1], 0.0) * rhoa[k - 1] * psi_old[k - 1] -
                                           dmin(wt[k], 0.0) * rhoa[k] * psi_old[k + 1]) /
                                          dzn[k] +
                                      SMALL;
                const double denom2 = dt *
                                          (dmax(wt[k], 0.0) * rhoa[k] * psi_old[k] -
                                           dmin(wt[k - 1], 0.0) * rhoa[k - 1] * psi_old[k]) /
                                          dzn[k] +
                                      SMALL;
                beta_up[k] = rhoan[k] * (psi_max[k] - psi_old[k]) / denom1;
                beta_down[k] = rhoan[k] * (psi_old[k] - psi_min[k]) / denom2;
            }
            for (int k = 1 - r_h; k <= 0; k++) beta_up[k] = beta_down[k] = 0.0; /* :698-701 */
            for (int k = kp + 1; k <= kp + r_h; k++) beta_up[k] = beta_down[k] = 0.0;
            for (int k = 1; k <= kp; k++) /* :709-715 */
                wt_sav[k] = dmin(dmin(1.0, beta_down[k]), beta_up[k + 1]) * dmax(wt[k], 0.0) +
                            dmin(dmin(1.0, beta_up[k]), beta_down[k + 1]) * dmin(wt[k], 0.0);
            w_store2[0] = w_store2[1]; /* :722-733 */
            w_store2[kp] = w_store2[kp - 1];
            w_store2[kp + 1] = w_store2[kp - 1];
            wt = w_store2;
            wt_sav = w_store1;
        }
        for (int n = 0; n < nq; n++) { /* :748-764 */
            double *p = PSI(n);
            upstream_1d(dt, dzn, rhoa, rhoan, kp, wt, p, neumann, fz_r, fz_l);
            if (it <= kord && kord >= 1) {
                p[0] = 0.0;
                p[kp + 1] = 0.0;
            }
        }
    }
    for (int n = 0; n < nq; n++) { /* :775-777 */
        double *p = PSI(n);
        for (int k = -r_h + 1; k <= kp + r_h; k++) p[k] = p[k] + minglobal[n];
    }
out:
#undef PSI
    free(ws1b);
    free(ws2b);
    free(storeb);
    free(pmaxb);
    free(pminb);
    free(bupb);
    free(bdnb);
    free(fz_r);
    free(fz_l);
    free(minglobal);
}

/* ncol independent columns, each nsub[c] passes of dt[c]/nsub[c] (the
 * sedimentation loops of pamm/microphysics.f90:3139-3183; nsub NULL: one
 * pass).  metric_stride 0: dz, dzn, rhoa, rhoan shared by all columns;
 * otherwise each column's at + c*metric_stride. */
void orc_mpdata_vec_1d_columns(int ncol, int kp, int nq, int l_h, int r_h, const double *dt,
                               const int *nsub, const double *dz, const double *dzn,
                               const double *rhoa, const double *rhoan, int metric_stride,
                               const double *w, double *psi, int kord, int monotone,
                               int neumann) {
    const size_t nw = (size_t)(kp + l_h + r_h), npsi = (size_t)(kp + 2 * r_h);
#pragma omp parallel for schedule(dynamic, 16)
    for (int c = 0; c < ncol; c++) {
        const size_t mo = (size_t)c * (size_t)metric_stride;
        const int ns = nsub ? nsub[c] : 1;
        for (int s = 0; s < ns; s++)
            orc_mpdata_vec_1d(dt[c] / (double)ns, dz + mo, dzn + mo, rhoa + mo, rhoan + mo, kp,
                              nq, l_h, r_h, w + (size_t)c * nw,
                              psi + (size_t)c * npsi * (size_t)nq, kord, monotone, neumann);
    }
}
