// k_mpdata.cu -- MPDATA advection of the linked copy
// pamm/sfvt/advection_3d.F90: first_order_upstream_3d (:39-116),
// mpdata_3d (:219-714), mpdata_vec_3d (:1250-1753), with the FCT limiter of
// Smolarkiewicz & Grabowski (1990) in the linked form (:542-675) or the
// sfvt/advection_3d.F90 interface-copy form (:544-704).
//
// One kernel per stage of the reference's iteration, each writing its own
// exchange images (see dcm_common.cuh), so no halo pass runs between
// stages:
//   k_upwind    donor cell (+ the positive-definite shift on the first pass,
//               the unshift and the scalar source update on the last)
//   k_antidiff  antidiffusive pseudo-velocities (eqs 13/14/38, G = rho)
//   k_beta      beta_up / beta_down (eqs 19/20)
//   k_limit     limited velocities (eq 18)
#include <algorithm>

#include "dcm_internal.h"
#include "dcm_prof.h"

namespace dcm {

#define SMALLV 1e-60

template <typename T>
struct Vel {
    const T *u, *v, *w;
};
template <typename T>
struct VelOut {
    T *u, *v, *w;
};

template <typename T>
__device__ __forceinline__ T small_of() { return T(SMALLV); }

// periodic index into 1..n
__device__ __forceinline__ int wrapj(int q, int n) { return ((q - 1) % n + n) % n + 1; }
template <>
__device__ __forceinline__ float small_of<float>() { return 1e-30f; }

// ---- positive-definite shift: min over the whole array or the interior ---
// mpdata_3d takes minval over the whole array including halos (:275);
// mpdata_vec_3d over the interior only (:1307).
// Each block strides over the i-planes (blockIdx.z, step gridDim.z), so the
// grid has a few thousand blocks rather than one per plane.
template <typename T, bool INTERIOR>
__global__ void __launch_bounds__(256) k_min(Dims d, const T* __restrict__ a,
                                             double lbc, double ubc,
                                             double* partials,
                                             unsigned int* ticket,
                                             MpScalars* M) {
    __shared__ double smem[32];
    double v[1] = {1e300};
    const int k = (INTERIOR ? 1 : 0) + blockIdx.x * BX + threadIdx.x;
    const int j = (INTERIOR ? 1 : 0) + blockIdx.y * BY + threadIdx.y;
    const int kmax = INTERIOR ? d.kp : d.kp + 1, jmax = INTERIOR ? d.jp : d.jp + 1;
    const int imax = INTERIOR ? d.ip : d.ip + 1;
    if (k <= kmax && j <= jmax) {
        T m = a[d.at(k, j, (INTERIOR ? 1 : 0) + blockIdx.z)];
        for (int i = (INTERIOR ? 1 : 0) + blockIdx.z + gridDim.z; i <= imax; i += gridDim.z)
            m = fmin(m, a[d.at(k, j, i)]);
        v[0] = (double)m;
    }
    block_reduce<R_MIN, 1>(v, smem);
    const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    if (publish_partials<1>(v, partials, ticket, nb)) {
        double s[1];
        final_reduce<R_MIN, 1>(s, partials, ticket, nb, smem);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            T m = (T)s[0];
            m = fmin(fmin((double)m, lbc), ubc);
            M->m = (double)m;
            M->lbc = (double)((T)lbc - m);
            M->ubc = (double)((T)ubc - m);
            M->early = 0;
        }
    }
}

// ---- donor cell ---------------------------------------------------------------
// FIRST: source = psi_in - m (the shifted copy of :278) and sum the shifted
//        interior for the early return of :284-289.
// EXCH:  0 = interior only (the bare first_order_upstream_3d)
//        1 = exchange_full(lbc', ubc') images (the call at :694-695)
// LAST:  unshift (:711-713): write v + m, bcs lbc' + m / ubc' + m; if sadd
//        is given also add sadd*dt_add per written cell
//        (advance_scalar_fields_3d, sgm/subgrid_3d.f90:603-609).
// Donor-cell update of one interior point (:60-115) from the face
// velocities around it (uc, um = u at i, i-1; vc, vm; wc, wm) and psi read
// through P(kk, jj, ii).
template <typename T, typename PF>
__device__ __forceinline__ T donor_point(const Dims& d, const Metrics<T>& mt, T dt, int neumann,
                                         int k, int j, int i, T uc, T um, T vc, T vm, T wc,
                                         T wm, PF P) {
    const T two = T(2);
    const T pc = P(k, j, i);
    const T dxn = ld(mt.dxn + i), dyn = ld(mt.dyn + j), dzn = ld(mt.dzn + k);
    const T ra = ld(mt.rhoa + k), ram = ld(mt.rhoa + k - 1), rn = ld(mt.rhoan + k);
    const T fxr = ((uc + fabs(uc)) * pc + (uc - fabs(uc)) * P(k, j, i + 1)) * dt / (two * dxn);
    const T fxl = ((um + fabs(um)) * P(k, j, i - 1) + (um - fabs(um)) * pc) * dt / (two * dxn);
    const T fyr = ((vc + fabs(vc)) * pc + (vc - fabs(vc)) * P(k, j + 1, i)) * dt / (two * dyn);
    const T fyl = ((vm + fabs(vm)) * P(k, j - 1, i) + (vm - fabs(vm)) * pc) * dt / (two * dyn);
    T fzr = ((wc + fabs(wc)) * ra * pc + (wc - fabs(wc)) * ra * P(k + 1, j, i)) * dt /
            (two * dzn * rn);
    T fzl = ((wm + fabs(wm)) * ram * P(k - 1, j, i) + (wm - fabs(wm)) * ram * pc) * dt /
            (two * dzn * rn);
    if (neumann == 1) {  // :98-104
        if (k == 1) fzl = fzr;
        if (k == d.kp) fzr = fzl;
    } else if (neumann == 2) {  // :105-111
        if (k == 1) fzl = -fzr;
        if (k == d.kp) fzr = -fzl;
    }
    return pc - (fxr - fxl) - (fyr - fyl) - (fzr - fzl);  // :115
}

// Where a donor-cell result nv at an interior point goes.
// exch 0: the point only (the bare first_order_upstream_3d); exch 1: with its
// exchange_full(lbc', ubc') images (:694-695).  LAST: unshifted (:711-713),
// boundary values lbc' + m / ubc' + m, and with sadd every written cell also
// gets sadd * dt_add (advance_scalar_fields_3d, sgm/subgrid_3d.f90:603-609).
template <typename T, bool LAST>
__device__ __forceinline__ void donor_store(T* __restrict__ dst, const Dims& d, int k, int j,
                                            int i, T nv, int exch, const T* __restrict__ sadd,
                                            T dt_add, const MpScalars* M, T m) {
    if (LAST) {
        const T lb = (T)M->lbc + m, ub = (T)M->ubc + m;
        if (exch == 0) {
            dst[d.at(k, j, i)] = nv + m;
        } else if (sadd) {
            // write every image with its own source term
            T* a = dst;
            const T vv = nv + m;
            a[d.at(k, j, i)] = vv + sadd[d.at(k, j, i)] * dt_add;
            const bool edge = (i == 1) | (i == d.ip) | (j == 1) | (j == d.jp) | (k == 1) |
                              (k == d.kp);
            if (edge) {
                int ks[3], js[3], is[3];
                const int nk = images(k, d.kp, ks), nj = images(j, d.jp, js),
                          ni = images(i, d.ip, is);
                for (int a3 = 0; a3 < nk; a3++)
                    for (int b3 = 0; b3 < nj; b3++)
                        for (int c3 = 0; c3 < ni; c3++) {
                            if ((a3 | b3 | c3) == 0) continue;
                            const int kk = ks[a3], jj = js[b3], ii = is[c3];
                            T val = vv;
                            if ((kk == 0 || kk == d.kp + 1) && b3 == 0 && c3 == 0)
                                val = (kk == 0) ? lb : ub;
                            const int o = d.at(kk, jj, ii);
                            a[o] = val + sadd[o] * dt_add;
                        }
            }
        } else {
            put_full(dst, d, k, j, i, nv + m, lb, ub);
        }
    } else {
        if (exch == 0)
            dst[d.at(k, j, i)] = nv;
        else
            put_full(dst, d, k, j, i, nv, (T)M->lbc, (T)M->ubc);
    }
}

// ---- donor cell ---------------------------------------------------------------
// FIRST: source = psi_in - m (the shifted copy of :278) and sum the shifted
//        interior for the early return of :284-289.
// EXCH:  0 = interior only (the bare first_order_upstream_3d)
//        1 = exchange_full(lbc', ubc') images (the call at :694-695)
// LAST:  unshift (:711-713): write v + m, bcs lbc' + m / ubc' + m; if sadd
//        is given also add sadd*dt_add per written cell
//        (advance_scalar_fields_3d, sgm/subgrid_3d.f90:603-609).
template <typename T, bool FIRST, bool LAST>
__global__ void __launch_bounds__(256) k_upwind(Dims d, Metrics<T> mt, T dt,
                                                Vel<T> V,
                                                const T* __restrict__ src,
                                                T* __restrict__ dst, int neumann,
                                                int exch, const T* __restrict__ sadd,
                                                T dt_add, double* partials,
                                                unsigned int* ticket, MpScalars* M,
                                                const MpScalars* Mgate) {
    __shared__ double smem[32];
    if (!FIRST && Mgate && Mgate->early) return;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const T m = FIRST || LAST ? (T)M->m : T(0);
    double acc[1] = {0.0};
    const bool in = k <= d.kp && j <= d.jp;
    // the first pass also sums the shifted field (the early-return test):
    // its blocks stride over the i-planes, so that a few thousand blocks,
    // not one per plane, publish reduction partials
    const int istep = FIRST ? (int)gridDim.z : d.ip;
    for (int i = 1 + blockIdx.z; i <= d.ip; i += istep)
    if (in) {
        auto P = [&](int kk, int jj, int ii) -> T {
            const T x = src[d.at(kk, jj, ii)];
            return FIRST ? x - m : x;
        };
        const T nv = donor_point(d, mt, dt, neumann, k, j, i, V.u[d.at(k, j, i)],
                                 V.u[d.at(k, j, i - 1)], V.v[d.at(k, j, i)],
                                 V.v[d.at(k, j - 1, i)], V.w[d.at(k, j, i)],
                                 V.w[d.at(k - 1, j, i)], P);
        if (FIRST) acc[0] += (double)P(k, j, i);
        donor_store<T, LAST>(dst, d, k, j, i, nv, exch, sadd, dt_add, M, m);
    }
    if (FIRST) {
        block_reduce<R_SUM, 1>(acc, smem);
        const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
        if (publish_partials<1>(acc, partials, ticket, nb)) {
            double s[1];
            final_reduce<R_SUM, 1>(s, partials, ticket, nb, smem);
            if (threadIdx.x == 0 && threadIdx.y == 0) M->early = (s[0] < SMALLV) ? 1 : 0;
        }
    }
}

// ---- antidiffusive velocities (:320-505) ------------------------------------
// Quotients of the antidiffusive velocities: FP64 (the parity path) the
// correctly rounded divide; FP32 (the mixed form, whose fields carry 1e-7)
// the two-instruction approximate divide, within 2 ulp for divisors of
// magnitude 2^-126..2^126 (the denominators here are grid spacings, densities
// and sums of shifted, non-negative psi plus 1e-30)
__device__ __forceinline__ double adiv(double a, double b) { return a / b; }
__device__ __forceinline__ float adiv(float a, float b) { return __fdividef(a, b); }

// Antidiffusive pseudo-velocities (eqs 13/14/38 of Smolarkiewicz 1984,
// divergent flow, G = rho) at the interior point (k, j, i) from the velocity
// set Vt and psi (:320-505), every term in the reference's order.
template <typename T>
__device__ __forceinline__ void antidiff_point(const Dims& d, const Metrics<T>& mt, T dt,
                                               const Vel<T>& Vt, const T* __restrict__ pso,
                                               int k, int j, int i, T& us, T& vs, T& ws) {
    const T small = small_of<T>();
    auto U = [&](int kk, int jj, int ii) { return Vt.u[d.at(kk, jj, ii)]; };
    auto V = [&](int kk, int jj, int ii) { return Vt.v[d.at(kk, jj, ii)]; };
    auto W = [&](int kk, int jj, int ii) { return Vt.w[d.at(kk, jj, ii)]; };
    auto P = [&](int kk, int jj, int ii) { return pso[d.at(kk, jj, ii)]; };
    const T dx = ld(mt.dx + i), dxm = ld(mt.dx + i - 1), dxn = ld(mt.dxn + i),
            dxnm = ld(mt.dxn + i - 1);
    const T dy = ld(mt.dy + j), dym = ld(mt.dy + j - 1), dyn = ld(mt.dyn + j),
            dynm = ld(mt.dyn + j - 1);
    const T dz = ld(mt.dz + k), dzm = ld(mt.dz + k - 1), dzn = ld(mt.dzn + k),
            dznm = ld(mt.dzn + k - 1);
    const T ra = ld(mt.rhoa + k), ram = ld(mt.rhoa + k - 1), rap = ld(mt.rhoa + k + 1);
    const T rn = ld(mt.rhoan + k), rnp = ld(mt.rhoan + k + 1);
    const T h = T(0.5), q4 = T(0.25);
    const T g_bar1 = rn, g_bar2 = rn;
    const T g_bar3 = h * (rn + rnp);

    // every quotient through adiv: FP64 divides exactly as written (the
    // reference's arithmetic), FP32 with the approximate divide
    const T u_div1 = adiv(ra * (W(k, j, i) + W(k, j, i + 1)) - ram * (W(k - 1, j, i) + W(k - 1, j, i + 1)),
                          dzm * g_bar1) +
                     adiv(rn * (V(k, j, i) + V(k, j, i + 1) - V(k, j - 1, i) - V(k, j - 1, i + 1)),
                          dym * g_bar1);
    const T u_div2 = adiv(ra * (W(k, j, i) + W(k, j + 1, i)) - ram * (W(k - 1, j, i) + W(k - 1, j + 1, i)),
                          dzm * g_bar2) +
                     adiv(rn * (U(k, j, i) + U(k, j + 1, i) - U(k, j, i - 1) - U(k, j + 1, i - 1)),
                          dxm * g_bar2);
    const T u_div3 = adiv(rn * (U(k, j, i) - U(k, j, i - 1)) + rnp * (U(k + 1, j, i) - U(k + 1, j, i - 1)),
                          dxm * g_bar3) +
                     adiv(rn * (V(k, j, i) - V(k, j - 1, i)) + rnp * (V(k + 1, j, i) - V(k + 1, j - 1, i)),
                          dym * g_bar3);

    const T uc = U(k, j, i), vc = V(k, j, i), wc = W(k, j, i);
    // q4 * A / g * B / C / E, evaluated left to right as the reference does
    auto term = [&](T A, T g, T B, T Cd, T E) { return adiv(adiv(adiv(q4 * A, g) * B, Cd), E); };
    const T u_j_bar1 =
        h * dt * uc *
        (term(ra * W(k, j, i + 1) + ra * W(k, j, i) + ram * W(k - 1, j, i + 1) + ram * W(k - 1, j, i),
              g_bar1,
              P(k + 1, j, i + 1) + P(k + 1, j, i) - P(k - 1, j, i + 1) - P(k - 1, j, i),
              P(k + 1, j, i + 1) + P(k + 1, j, i) + P(k - 1, j, i + 1) + P(k - 1, j, i) + small,
              h * (dznm + dzn)) +
         term(rn * V(k, j, i + 1) + rn * V(k, j, i) + rn * V(k, j - 1, i + 1) + rn * V(k, j - 1, i),
              g_bar1,
              P(k, j + 1, i + 1) + P(k, j + 1, i) - P(k, j - 1, i + 1) - P(k, j - 1, i),
              P(k, j + 1, i + 1) + P(k, j + 1, i) + P(k, j - 1, i + 1) + P(k, j - 1, i) + small,
              h * (dynm + dyn)));
    const T u_j_bar2 =
        h * dt * vc *
        (term(ra * W(k, j + 1, i) + ra * W(k, j, i) + ram * W(k - 1, j + 1, i) + ram * W(k - 1, j, i),
              g_bar2,
              P(k + 1, j + 1, i) + P(k + 1, j, i) - P(k - 1, j + 1, i) - P(k - 1, j, i),
              P(k + 1, j + 1, i) + P(k + 1, j, i) + P(k - 1, j + 1, i) + P(k - 1, j, i) + small,
              h * (dznm + dzn)) +
         term(rn * U(k, j + 1, i) + rn * U(k, j, i) + rn * U(k, j + 1, i - 1) + rn * U(k, j, i - 1),
              g_bar2,
              P(k, j + 1, i + 1) + P(k, j, i + 1) - P(k, j + 1, i - 1) - P(k, j, i - 1),
              P(k, j + 1, i + 1) + P(k, j, i + 1) + P(k, j + 1, i - 1) + P(k, j, i - 1) + small,
              h * (dxnm + dxn)));
    const T u_j_bar3 =
        h * dt * wc *
        (term(rnp * V(k + 1, j, i) + rn * V(k, j, i) + rnp * V(k + 1, j - 1, i) + rn * V(k, j - 1, i),
              g_bar3,
              P(k + 1, j + 1, i) + P(k, j + 1, i) - P(k + 1, j - 1, i) - P(k, j - 1, i),
              P(k + 1, j + 1, i) + P(k, j + 1, i) + P(k + 1, j - 1, i) + P(k, j - 1, i) + small,
              h * (dynm + dyn)) +
         term(rnp * U(k + 1, j, i) + rn * U(k, j, i) + rnp * U(k + 1, j, i - 1) + rn * U(k, j, i - 1),
              g_bar3,
              P(k + 1, j, i + 1) + P(k, j, i + 1) - P(k + 1, j, i - 1) - P(k, j, i - 1),
              P(k + 1, j, i + 1) + P(k, j, i + 1) + P(k + 1, j, i - 1) + P(k, j, i - 1) + small,
              h * (dxnm + dxn)));

    const T pc = P(k, j, i);
    us = adiv(adiv((fabs(uc) * dx - dt * uc * uc) * (P(k, j, i + 1) - pc),
                     P(k, j, i + 1) + pc + small),
                dxn) -
           u_j_bar1;
    vs = adiv(adiv((fabs(vc) * dy - dt * vc * vc) * (P(k, j + 1, i) - pc),
                     P(k, j + 1, i) + pc + small),
                dyn) -
           u_j_bar2;
    ws = adiv(adiv((fabs(wc) * dz - dt * adiv(ra, g_bar3) * wc * wc) * (P(k + 1, j, i) - pc),
                     P(k + 1, j, i) + pc + small),
                dzn) -
           u_j_bar3;
    us = us - q4 * dt * uc * (adiv(U(k, j, i + 1) - U(k, j, i - 1), dxm) + u_div1);  // :489-499
    vs = vs - q4 * dt * vc * (adiv(V(k, j + 1, i) - V(k, j - 1, i), dym) + u_div2);
    ws = ws - q4 * dt * wc * (adiv(rap * W(k + 1, j, i) - ram * W(k - 1, j, i), dzm * g_bar3) + u_div3);
}

template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) k_antidiff(Dims d, Metrics<T> mt, T dt,
                                                  Vel<T> Vt,
                                                  const T* __restrict__ pso,
                                                  VelOut<T> out,
                                                  const MpScalars* Mgate) {
    if (Mgate->early) return;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    T us, vs, ws;
    antidiff_point(d, mt, dt, Vt, pso, k, j, i, us, vs, ws);
    // exchange_full(..., 0, 0) of the new velocities, :528-533
    put_full(out.u, d, k, j, i, us, T(0), T(0));
    put_full(out.v, d, k, j, i, vs, T(0), T(0));
    put_full(out.w, d, k, j, i, ws, T(0), T(0));
}

// beta_up / beta_down of the linked FCT limiter (eqs 19/20, :549-623) at the
// interior point (k, j, i): psi_store = psi_in - m and psi_old (pso) from
// memory, and the six face velocities of the point (U at i-1 and i, V at
// j-1 and j, W at k-1 and k) as arguments.
template <typename T>
__device__ __forceinline__ void beta0_point(const Dims& d, const Metrics<T>& mt, T dt, T m,
                                            const T* __restrict__ psi_in,
                                            const T* __restrict__ pso, int k, int j, int i,
                                            T Uim, T Uc, T Vjm, T Vc, T Wkm, T Wc, T& bup,
                                            T& bdn) {
    const T z = T(0);
    const T small = small_of<T>();
    auto PS = [&](int kk, int jj, int ii) { return psi_in[d.at(kk, jj, ii)] - m; };  // psi_store
    auto PO = [&](int kk, int jj, int ii) { return pso[d.at(kk, jj, ii)]; };
    const T pc = PO(k, j, i);
    const T rn = ld(mt.rhoan + k), ra = ld(mt.rhoa + k), ram = ld(mt.rhoa + k - 1);
    const T dxn = ld(mt.dxn + i), dyn = ld(mt.dyn + j), dzn = ld(mt.dzn + k);
    const T s[14] = {PS(k, j, i),     PS(k, j, i - 1), PS(k, j, i + 1), PS(k, j - 1, i),
                     PS(k, j + 1, i), PS(k - 1, j, i), PS(k + 1, j, i), pc,
                     PO(k, j, i - 1), PO(k, j, i + 1), PO(k, j - 1, i), PO(k, j + 1, i),
                     PO(k - 1, j, i), PO(k + 1, j, i)};
    T pmax = s[0], pmin = s[0];
#pragma unroll
    for (int q = 1; q < 14; q++) {
        pmax = fmax(pmax, s[q]);
        pmin = fmin(pmin, s[q]);
    }
    const T denom1 =
        dt * ((fmax(Uim, z) * rn * PO(k, j, i - 1) - fmin(Uc, z) * rn * PO(k, j, i + 1)) /
                  dxn +
              (fmax(Vjm, z) * rn * PO(k, j - 1, i) - fmin(Vc, z) * rn * PO(k, j + 1, i)) /
                  dyn +
              (fmax(Wkm, z) * ram * PO(k - 1, j, i) - fmin(Wc, z) * ra * PO(k + 1, j, i)) /
                  dzn) +
        small;
    const T denom2 =
        dt * ((fmax(Uc, z) * rn * pc - fmin(Uim, z) * rn * pc) / dxn +
              (fmax(Vc, z) * rn * pc - fmin(Vjm, z) * rn * pc) / dyn +
              (fmax(Wc, z) * ra * pc - fmin(Wkm, z) * ram * pc) / dzn + small);
    bup = rn * (pmax - pc) / denom1;
    bdn = rn * (pc - pmin) / denom2;
}

// one limited velocity component (eq 18, :634-656): c the antidiffusive
// velocity, (up_o, dn_o) the betas at the point, (up_n, dn_n) at the next
// point along the component's direction
template <typename T>
__device__ __forceinline__ T limit_comp(T c, T up_o, T dn_o, T up_n, T dn_n) {
    const T z = T(0), one = T(1);
    return fmin(fmin(one, dn_o), up_n) * fmax(c, z) + fmin(fmin(one, up_o), dn_n) * fmin(c, z);
}

// ---- beta (eqs 19/20) -----------------------------------------------------
// VARIANT 0 (linked :549-627): 14-point max/min, rho-weighted, 2 betas.
// VARIANT 1 (sfvt :551-659):  per-direction 6-point max/min, unweighted,
//                             6 betas.
template <typename T, int VARIANT>
__global__ void __launch_bounds__(256) k_beta(Dims d, Metrics<T> mt, T dt,
                                              const T* __restrict__ psi_in,
                                              const T* __restrict__ pso, Vel<T> Vt,
                                              T* __restrict__ b0, T* __restrict__ b1,
                                              T* __restrict__ b2, T* __restrict__ b3,
                                              T* __restrict__ b4, T* __restrict__ b5,
                                              const MpScalars* M) {
    if (M->early) return;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const T m = (T)M->m;
    const T small = small_of<T>();
    auto PS = [&](int kk, int jj, int ii) { return psi_in[d.at(kk, jj, ii)] - m; };  // psi_store
    auto PO = [&](int kk, int jj, int ii) { return pso[d.at(kk, jj, ii)]; };
    auto U = [&](int kk, int jj, int ii) { return Vt.u[d.at(kk, jj, ii)]; };
    auto V = [&](int kk, int jj, int ii) { return Vt.v[d.at(kk, jj, ii)]; };
    auto W = [&](int kk, int jj, int ii) { return Vt.w[d.at(kk, jj, ii)]; };
    const T z = T(0);
    const T pc = PO(k, j, i);
    if (VARIANT == 0) {
        T bup, bdn;
        beta0_point(d, mt, dt, m, psi_in, pso, k, j, i, U(k, j, i - 1), U(k, j, i),
                    V(k, j - 1, i), V(k, j, i), W(k - 1, j, i), W(k, j, i), bup, bdn);
        // exchange_along_dim(..., 0, 0), :624-627
        put_dim(b0, d, k, j, i, bup, z, z);
        put_dim(b1, d, k, j, i, bdn, z, z);
    } else {
        const T dxm = ld(mt.dx + i - 1), dym = ld(mt.dy + j - 1), dzm = ld(mt.dz + k - 1);
        auto mx6 = [](T a, T b, T c, T e, T f, T g) {
            return fmax(fmax(fmax(fmax(fmax(a, b), c), e), f), g);
        };
        auto mn6 = [](T a, T b, T c, T e, T f, T g) {
            return fmin(fmin(fmin(fmin(fmin(a, b), c), e), f), g);
        };
        const T imax = mx6(PS(k, j, i - 1), PS(k, j, i), PS(k, j, i + 1), PO(k, j, i - 1), pc, PO(k, j, i + 1));
        const T imin = mn6(PS(k, j, i - 1), PS(k, j, i), PS(k, j, i + 1), PO(k, j, i - 1), pc, PO(k, j, i + 1));
        const T jmax = mx6(PS(k, j - 1, i), PS(k, j, i), PS(k, j + 1, i), PO(k, j - 1, i), pc, PO(k, j + 1, i));
        const T jmin = mn6(PS(k, j - 1, i), PS(k, j, i), PS(k, j + 1, i), PO(k, j - 1, i), pc, PO(k, j + 1, i));
        const T kmax = mx6(PS(k - 1, j, i), PS(k, j, i), PS(k + 1, j, i), PO(k - 1, j, i), pc, PO(k + 1, j, i));
        const T kmin = mn6(PS(k - 1, j, i), PS(k, j, i), PS(k + 1, j, i), PO(k - 1, j, i), pc, PO(k + 1, j, i));
        const T denom1 =
            (dt * ((fmax(U(k, j, i - 1), z) * PO(k, j, i - 1) - fmin(U(k, j, i), z) * PO(k, j, i + 1)) / dxm +
                   (fmax(V(k, j - 1, i), z) * PO(k, j - 1, i) - fmin(V(k, j, i), z) * PO(k, j + 1, i)) / dym +
                   (fmax(W(k - 1, j, i), z) * PO(k - 1, j, i) - fmin(W(k, j, i), z) * PO(k + 1, j, i)) / dzm +
                   small));
        const T denom2 =
            (dt * ((fmax(U(k, j, i), z) * pc - fmin(U(k, j, i - 1), z) * pc) / dxm +
                   (fmax(V(k, j, i), z) * pc - fmin(V(k, j - 1, i), z) * pc) / dym +
                   (fmax(W(k, j, i), z) * pc - fmin(W(k - 1, j, i), z) * pc) / dzm + small));
        put_dim(b0, d, k, j, i, (imax - pc) / denom1, z, z);
        put_dim(b1, d, k, j, i, (pc - imin) / denom2, z, z);
        put_dim(b2, d, k, j, i, (jmax - pc) / denom1, z, z);
        put_dim(b3, d, k, j, i, (pc - jmin) / denom2, z, z);
        put_dim(b4, d, k, j, i, (kmax - pc) / denom1, z, z);
        put_dim(b5, d, k, j, i, (pc - kmin) / denom2, z, z);
    }
}

// ---- limited velocities (eq 18, :634-656) ---------------------------------
template <typename T, int VARIANT>
__global__ void __launch_bounds__(256) k_limit(Dims d, Vel<T> Vt, const T* __restrict__ b0,
                                               const T* __restrict__ b1, const T* __restrict__ b2,
                                               const T* __restrict__ b3, const T* __restrict__ b4,
                                               const T* __restrict__ b5, VelOut<T> out,
                                               const MpScalars* M) {
    if (M->early) return;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const T z = T(0);
    const int o = d.at(k, j, i);
    const T uc = Vt.u[o], vc = Vt.v[o], wc = Vt.w[o];
    // beta arrays per direction: (up, down)
    const T *iup = b0, *idn = b1, *jup = VARIANT ? b2 : b0, *jdn = VARIANT ? b3 : b1,
            *kup = VARIANT ? b4 : b0, *kdn = VARIANT ? b5 : b1;
    const T lu = limit_comp(uc, iup[o], idn[o], iup[d.at(k, j, i + 1)], idn[d.at(k, j, i + 1)]);
    const T lv = limit_comp(vc, jup[o], jdn[o], jup[d.at(k, j + 1, i)], jdn[d.at(k, j + 1, i)]);
    const T lw = limit_comp(wc, kup[o], kdn[o], kup[d.at(k + 1, j, i)], kdn[d.at(k + 1, j, i)]);
    // exchange_full(..., 0, 0), :669-674
    put_full(out.u, d, k, j, i, lu, z, z);
    put_full(out.v, d, k, j, i, lv, z, z);
    put_full(out.w, d, k, j, i, lw, z, z);
}

// ---- one antidiffusive iteration in one kernel --------------------------------
// Antidiffusive velocities, the linked FCT limiter (beta, eq 18) and the
// donor-cell pass of field 0 (:319-695), fused along i-planes.  A block owns
// the output rows j0..j0+JT-1 of an i-chunk [i0, i1] and keeps R = JT + H + 1
// warps, one per row j0-H .. j0+JT (H = 2 with the limiter, 1 without; halo
// rows take the periodic image of their j).  A warp covers whole columns
// (k = 1 + lane + 32c, c < NC), so every k neighbour is in the block and the
// boundary planes k = 0, kp+1 hold the exchanges' value 0.  The stages march
// over the planes skewed by one plane:
//   step f:  A (antidiffusive velocities) at plane f     (rows 0..R-1)
//            beta at plane f                              (rows 1..R-1)
//            L (limited velocities) at plane f-1          (rows 1..R-2)
//            donor cell of field 0 at plane f-1           (owned rows)
// with a barrier between stages.  j and k neighbours of a stage's inputs
// come from shared planes (the v and w components of A, the two betas of
// planes f-1 and f, the v and w components of L); i neighbours and a
// point's own values stay in registers.  Only the limited velocities
// (exchange_full images, the next iteration's input) and the new field 0
// reach memory; A and beta never do.  Without the limiter the donor cell
// runs on A at plane f and A is the output set.  Each quantity is the same
// point function as the separate kernels evaluate.
template <typename T>
struct MpIterArgs {
    Dims d;
    Metrics<T> mt;
    T dt;
    Vel<T> Vt;              // this iteration's velocities (with their images)
    const T* psi_in;        // field 0 as given (psi_store = psi_in - m)
    const T* pso;           // field 0 before this iteration (shifted, with images)
    VelOut<T> vout;         // output velocities (limited, or antidiffusive)
    T* dst;                 // field 0 after this iteration's donor cell
    int neumann;
    const T* sadd;          // LAST: scalar source (or null)
    T dt_add;
    const MpScalars* M;     // field 0's shift and boundary values
    const MpScalars* gate;  // early return of the whole call
    int JT, ni, P;          // owned rows, planes per chunk, k pitch of a shared plane
};

// threads per block of the fused iteration: 24 warps (FP32, <= 85 registers)
// or 12 (FP64, <= 170 registers)
template <typename T>
constexpr int mp_iter_max_rows() { return sizeof(T) == 4 ? 24 : 12; }

template <typename T, bool MONO, bool LAST>
__global__ void __launch_bounds__(32 * mp_iter_max_rows<T>()) k_mpdata_iter(MpIterArgs<T> a) {
    extern __shared__ __align__(16) unsigned char mp_smem[];
    T* sm = reinterpret_cast<T*>(mp_smem);
    if (a.gate->early) return;
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5, R = blockDim.x >> 5;
    const int P = a.P, PL = R * P, kp = d.kp;
    constexpr int H = MONO ? 2 : 1;
    const int j0 = 1 + blockIdx.x * a.JT;
    const int jr = wrapj(j0 - H + r, d.jp);
    const int i0 = 1 + blockIdx.y * a.ni, i1 = min(i0 + a.ni - 1, d.ip);
    const bool owned = r >= H && r <= R - 2 && j0 - H + r <= d.jp;
    const T m = (T)a.M->m;
    // shared planes [row][k], k = 0..kp+1, by plane parity f & 1:
    //   A[2][u, v, w] (0..5); MONO also B[2][up, dn] (6..9), Lu[2] (10, 11),
    //   Lv (12), Lw (13)
    constexpr int NPL = MONO ? 14 : 6;
    auto A_ = [&](int par, int comp) { return sm + (par * 3 + comp) * PL; };
    auto B_ = [&](int par, int comp) { return sm + (6 + par * 2 + comp) * PL; };
    auto Lu_ = [&](int par) { return sm + (10 + par) * PL; };
    T* const sLv = sm + 12 * PL;
    T* const sLw = sm + 13 * PL;
    for (int q = threadIdx.x; q < NPL * R; q += blockDim.x) {
        sm[q * P] = T(0);
        sm[q * P + kp + 1] = T(0);
    }
    auto Pf = [&](int kk, int jj, int ii) -> T { return a.pso[d.at(kk, jj, ii)]; };
    const int fstart = i0 - (MONO ? 2 : 1), fend = MONO ? i1 + 1 : i1;
    for (int f = fstart; f <= fend; f++) {
        const int fi = wrapj(f, d.ip);
        const int par = f & 1, pp = par ^ 1;
        // ---- A at plane f (every row)
        {
            T* const Au = A_(par, 0);
            T* const Av = A_(par, 1);
            T* const Aw = A_(par, 2);
            for (int k = 1 + lane; k <= kp; k += 32) {
                T us, vs, ws;
                antidiff_point(d, a.mt, a.dt, a.Vt, a.pso, k, jr, fi, us, vs, ws);
                Au[r * P + k] = us;
                Av[r * P + k] = vs;
                Aw[r * P + k] = ws;
            }
        }
        __syncthreads();
        if (MONO) {
            // ---- beta at plane f
            if (f >= i0 - 1 && r >= 1) {
                const T *Au = A_(par, 0), *Av = A_(par, 1), *Aw = A_(par, 2), *Aup = A_(pp, 0);
                T* const Bu = B_(par, 0);
                T* const Bd = B_(par, 1);
                for (int k = 1 + lane; k <= kp; k += 32) {
                    const int o = r * P + k;
                    T bu, bd;
                    beta0_point(d, a.mt, a.dt, m, a.psi_in, a.pso, k, jr, fi, Aup[o], Au[o],
                                Av[o - P], Av[o], Aw[o - 1], Aw[o], bu, bd);
                    Bu[o] = bu;
                    Bd[o] = bd;
                }
            }
            __syncthreads();
            // ---- L at plane f-1
            const int fm = wrapj(f - 1, d.ip);
            if (f >= i0 && r >= 1 && r <= R - 2) {
                const T *Au = A_(pp, 0), *Av = A_(pp, 1), *Aw = A_(pp, 2);
                const T *Bpu = B_(pp, 0), *Bpd = B_(pp, 1), *Bu = B_(par, 0), *Bd = B_(par, 1);
                T* const Lu = Lu_(pp);
                for (int k = 1 + lane; k <= kp; k += 32) {
                    const int o = r * P + k;
                    const T up = Bpu[o], dn = Bpd[o];
                    const T lu = limit_comp(Au[o], up, dn, Bu[o], Bd[o]);
                    const T lv = limit_comp(Av[o], up, dn, Bpu[o + P], Bpd[o + P]);
                    const T lw = limit_comp(Aw[o], up, dn, Bpu[o + 1], Bpd[o + 1]);
                    Lu[o] = lu;
                    sLv[o] = lv;
                    sLw[o] = lw;
                    if (owned && f - 1 >= i0) {  // exchange_full(..., 0, 0), :669-674
                        put_full(a.vout.u, d, k, jr, fm, lu, T(0), T(0));
                        put_full(a.vout.v, d, k, jr, fm, lv, T(0), T(0));
                        put_full(a.vout.w, d, k, jr, fm, lw, T(0), T(0));
                    }
                }
            }
            __syncthreads();
            // ---- donor cell of field 0 at plane f-1
            if (f >= i0 + 1 && owned) {
                const T *Lu = Lu_(pp), *Lum = Lu_(par);  // L_u at planes f-1, f-2
                for (int k = 1 + lane; k <= kp; k += 32) {
                    const int o = r * P + k;
                    const T nv = donor_point(d, a.mt, a.dt, a.neumann, k, jr, fm, Lu[o], Lum[o],
                                             sLv[o], sLv[o - P], sLw[o], sLw[o - 1], Pf);
                    donor_store<T, LAST>(a.dst, d, k, jr, fm, nv, 1, a.sadd, a.dt_add, a.M, m);
                }
            }
        } else {
            // ---- donor cell of field 0 at plane f on A
            if (f >= i0 && owned) {
                const T *Au = A_(par, 0), *Av = A_(par, 1), *Aw = A_(par, 2), *Aup = A_(pp, 0);
                for (int k = 1 + lane; k <= kp; k += 32) {
                    const int o = r * P + k;
                    const T nv = donor_point(d, a.mt, a.dt, a.neumann, k, jr, fi, Au[o], Aup[o],
                                             Av[o], Av[o - P], Aw[o], Aw[o - 1], Pf);
                    put_full(a.vout.u, d, k, jr, fi, Au[o], T(0), T(0));  // :528-533
                    put_full(a.vout.v, d, k, jr, fi, Av[o], T(0), T(0));
                    put_full(a.vout.w, d, k, jr, fi, Aw[o], T(0), T(0));
                    donor_store<T, LAST>(a.dst, d, k, jr, fi, nv, 1, a.sadd, a.dt_add, a.M, m);
                }
            }
        }
    }
}

// Launch shape of the fused iteration: rows per block from the shared-memory
// budget and the row cap; i-chunks so that the grid fills every SM with as
// many blocks as fit on it at once, with chunks of at least 4 planes.
struct MpIterShape {
    int R = 0, JT = 0, ni = 0, P = 0, nstrips = 0, nchunks = 0;
    size_t smem = 0;
};

template <typename T, bool MONO, bool LAST>
__global__ void k_mpdata_iter(MpIterArgs<T> a);

template <typename T>
static MpIterShape mp_iter_shape(const Dims& d, bool mono, int max_rows) {
    MpIterShape s;
    const int H = mono ? 2 : 1, npl = mono ? 14 : 6;
    s.P = d.kp + 2;
    const size_t row_bytes = (size_t)npl * s.P * sizeof(T);
    const size_t budget = 200 * 1024;
    int R = (int)std::min<size_t>(mp_iter_max_rows<T>(), budget / row_bytes);
    R = std::min(R, max_rows);
    R = std::min(R, d.jp + H + 1);  // no more rows than the domain has
    if (R < H + 2) return s;        // not even one owned row
    s.R = R;
    s.JT = R - H - 1;
    s.smem = row_bytes * R;
    s.nstrips = (d.jp + s.JT - 1) / s.JT;
    int sms = 148;
    {
        int dev = 0;
        if (cudaGetDevice(&dev) == cudaSuccess)
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    int per_sm = 1;
    if (mono)
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mpdata_iter<T, true, false>,
                                                      32 * R, s.smem);
    else
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_mpdata_iter<T, false, false>,
                                                      32 * R, s.smem);
    per_sm = std::max(per_sm, 1);
    const int want = (sms * per_sm + s.nstrips - 1) / s.nstrips;
    const int nch = std::max(1, std::min((d.ip + 3) / 4, want));
    s.ni = (d.ip + nch - 1) / nch;
    s.nchunks = (d.ip + s.ni - 1) / s.ni;
    return s;
}

template <typename T, bool MONO, bool LAST>
static bool launch_mp_iter(const MpIterArgs<T>& args, const MpIterShape& s, cudaStream_t st) {
    const dim3 grid(s.nstrips, s.nchunks), block(32 * s.R);
    k_mpdata_iter<T, MONO, LAST><<<grid, block, s.smem, st>>>(args);
    return true;
}

// the opt-in shared-memory limit of every fused-iteration kernel (called
// once at handle creation, outside any stream capture)
template <typename T, bool MONO, bool LAST>
static void mp_iter_attrs() {
    cudaFuncSetAttribute(k_mpdata_iter<T, MONO, LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         210 * 1024);
}

void mpdata_init() {
    mp_iter_attrs<float, true, true>();
    mp_iter_attrs<float, true, false>();
    mp_iter_attrs<float, false, true>();
    mp_iter_attrs<float, false, false>();
    mp_iter_attrs<double, true, true>();
    mp_iter_attrs<double, true, false>();
    mp_iter_attrs<double, false, true>();
    mp_iter_attrs<double, false, false>();
}

// ---- early return of :284-289: psi = (psi - m) + m everywhere --------------
template <typename T>
__global__ void __launch_bounds__(256) k_restore(Dims d, const T* __restrict__ src,
                                                 T* __restrict__ dst,
                                                 const T* __restrict__ sadd, T dt_add,
                                                 const MpScalars* Mgate,
                                                 const MpScalars* Mshift) {
    if (!Mgate->early) return;
    const int k = blockIdx.x * BX + threadIdx.x;
    const int j = blockIdx.y * BY + threadIdx.y;
    const int i = blockIdx.z;
    if (k > d.kp + 1 || j > d.jp + 1) return;
    const int o = d.at(k, j, i);
    const T m = (T)Mshift->m;
    T v = (src[o] - m) + m;
    if (sadd) v = v + sadd[o] * dt_add;
    dst[o] = v;
}

// ---- host orchestration --------------------------------------------------------
// psi_in[q] is read-only; psi_out[q] receives the unshifted result and may
// alias psi_in[q] when kord >= 2 (the last donor-cell pass reads only the
// scratch copies).  w.M[q] holds the shift of field q; the early return is
// decided by field 0 alone (:284, :1316).
template <typename T>
int mpdata_run(MpdataWork<T>& w, const Dims& d, const Metrics<T>& mt, T dt,
               const T* u, const T* v, const T* wv, T* const* psi_in, T* const* psi_out,
               int nq, const double* lbc, const double* ubc, int kord, int monotone,
               int neumann, int variant, bool vec, const T* const* sadd, T dt_add,
               cudaStream_t st) {
    const dim3 g = interior_grid(d, d.kp), b(BX, BY);
    const dim3 gf = full_grid(d);
    for (int q = 0; q < nq; q++) {
        if (vec)
            { ProfScope ps_(P_MPMIN, st);
            k_min<T, true><<<dim3(g.x, g.y, min(g.z, 16u)), b, 0, st>>>(
                d, psi_in[q], lbc[q], ubc[q], w.partials, w.ticket, w.M + q);
            }
        else
            { ProfScope ps_(P_MPMIN, st);
            k_min<T, false><<<dim3(gf.x, gf.y, min(gf.z, 16u)), b, 0, st>>>(
                d, psi_in[q], lbc[q], ubc[q], w.partials, w.ticket, w.M + q);
            }
    }
    const MpScalars* gate = w.M;
    if (kord < 1) {
        // empty iteration loop: psi = (psi - m) + m
        for (int q = 0; q < nq; q++)
            { ProfScope ps_(P_RESTORE, st);
            k_restore<T><<<gf, b, 0, st>>>(d, psi_in[q], psi_out[q], sadd ? sadd[q] : nullptr,
                                           dt_add, w.Mone, w.M + q);
            }
        return cudaGetLastError() == cudaSuccess ? 0 : DCM_E_CUDA;
    }
    const Vel<T> V0{u, v, wv};
    const dim3 gfirst(g.x, g.y, std::min(g.z, 16u));  // blocks stride over i
    // it = 1: donor cell of the shifted input (:684)
    for (int q = 0; q < nq; q++) {
        const T* sa = sadd ? sadd[q] : nullptr;
        if (kord == 1)
            { ProfScope ps_(P_UPWIND, st);
            k_upwind<T, true, true><<<gfirst, b, 0, st>>>(d, mt, dt, V0, psi_in[q], psi_out[q],
                                                          neumann, 1, sa, dt_add, w.partials,
                                                          w.ticket, w.M + q, nullptr);
            }
        else
            { ProfScope ps_(P_UPWIND, st);
            k_upwind<T, true, false><<<gfirst, b, 0, st>>>(d, mt, dt, V0, psi_in[q], w.pa[q],
                                                           neumann, 1, nullptr, T(0), w.partials,
                                                           w.ticket, w.M + q, nullptr);
            }
    }
    // velocity sets: A receives antidiffusive velocities, L limited ones
    VelOut<T> A{w.va[0], w.va[1], w.va[2]}, L{w.vl[0], w.vl[1], w.vl[2]};
    Vel<T> Vcur = V0;
    T* const* cur = w.pa;
    T* const* nxt = w.pb;
    for (int it = 2; it <= kord; it++) {
        const bool last = it == kord;
        // the fused iteration: antidiffusive velocities, the linked limiter
        // and field 0's donor cell in one kernel (the sfvt limiter variant,
        // and columns whose planes do not fit in shared memory, take the
        // separate kernels)
        const MpIterShape fs = (w.fuse && (variant == 0 || !monotone))
                                   ? mp_iter_shape<T>(d, monotone != 0, w.fuse_rows)
                                   : MpIterShape{};
        if (fs.R) {
            // the output set must not be the set this iteration reads
            VelOut<T> O = monotone ? (Vcur.u == L.u ? A : L) : A;
            MpIterArgs<T> ia;
            ia.d = d; ia.mt = mt; ia.dt = dt; ia.Vt = Vcur; ia.psi_in = psi_in[0];
            ia.pso = cur[0]; ia.vout = O; ia.dst = last ? psi_out[0] : nxt[0];
            ia.neumann = neumann; ia.sadd = (last && sadd) ? sadd[0] : nullptr;
            ia.dt_add = dt_add; ia.M = w.M; ia.gate = gate;
            ia.JT = fs.JT; ia.ni = fs.ni; ia.P = fs.P;
            bool okl;
            {
                ProfScope ps_(P_ANTIDIFF, st);
                if (monotone)
                    okl = last ? launch_mp_iter<T, true, true>(ia, fs, st)
                               : launch_mp_iter<T, true, false>(ia, fs, st);
                else
                    okl = last ? launch_mp_iter<T, false, true>(ia, fs, st)
                               : launch_mp_iter<T, false, false>(ia, fs, st);
            }
            if (!okl) return DCM_E_UNSUPPORTED;
            Vel<T> Vuse{O.u, O.v, O.w};
            if (!monotone) std::swap(A, L);
            Vcur = Vuse;
            // the other fields of a category: donor cell on the same velocities
            for (int q = 1; q < nq; q++) {
                const T* sa = sadd ? sadd[q] : nullptr;
                if (last)
                    { ProfScope ps_(P_UPWIND, st);
                    k_upwind<T, false, true><<<g, b, 0, st>>>(d, mt, dt, Vuse, cur[q], psi_out[q],
                                                              neumann, 1, sa, dt_add, nullptr,
                                                              nullptr, w.M + q, gate);
                    }
                else
                    { ProfScope ps_(P_UPWIND, st);
                    k_upwind<T, false, false><<<g, b, 0, st>>>(d, mt, dt, Vuse, cur[q], nxt[q],
                                                               neumann, 1, nullptr, T(0), nullptr,
                                                               nullptr, w.M + q, gate);
                    }
            }
            std::swap(cur, nxt);
            continue;
        }
        { ProfScope ps_(P_ANTIDIFF, st);
        k_antidiff<T><<<g, b, 0, st>>>(d, mt, dt, Vcur, cur[0], A, gate);
        }
        Vel<T> Vuse{A.u, A.v, A.w};
        if (monotone) {
            if (variant == 1) {
                { ProfScope ps_(P_BETA, st);
                k_beta<T, 1><<<g, b, 0, st>>>(d, mt, dt, psi_in[0], cur[0], Vuse, w.beta[0],
                                              w.beta[1], w.beta[2], w.beta[3], w.beta[4],
                                              w.beta[5], gate);
                }
                { ProfScope ps_(P_LIMIT, st);
                k_limit<T, 1><<<g, b, 0, st>>>(d, Vuse, w.beta[0], w.beta[1], w.beta[2],
                                               w.beta[3], w.beta[4], w.beta[5], L, gate);
                }
            } else {
                { ProfScope ps_(P_BETA, st);
                k_beta<T, 0><<<g, b, 0, st>>>(d, mt, dt, psi_in[0], cur[0], Vuse, w.beta[0],
                                              w.beta[1], nullptr, nullptr, nullptr, nullptr, gate);
                }
                { ProfScope ps_(P_LIMIT, st);
                k_limit<T, 0><<<g, b, 0, st>>>(d, Vuse, w.beta[0], w.beta[1], nullptr, nullptr,
                                               nullptr, nullptr, L, gate);
                }
            }
            // antidiff always writes A from the limited set L (:513-525, :662-667)
            Vuse = Vel<T>{L.u, L.v, L.w};
        } else {
            // the antidiffusive set is the next input: alternate the sets
            std::swap(A, L);
        }
        Vcur = Vuse;
        for (int q = 0; q < nq; q++) {
            const T* sa = sadd ? sadd[q] : nullptr;
            if (last)
                { ProfScope ps_(P_UPWIND, st);
                k_upwind<T, false, true><<<g, b, 0, st>>>(d, mt, dt, Vuse, cur[q], psi_out[q],
                                                          neumann, 1, sa, dt_add, nullptr, nullptr,
                                                          w.M + q, gate);
                }
            else
                { ProfScope ps_(P_UPWIND, st);
                k_upwind<T, false, false><<<g, b, 0, st>>>(d, mt, dt, Vuse, cur[q], nxt[q],
                                                           neumann, 1, nullptr, T(0), nullptr,
                                                           nullptr, w.M + q, gate);
                }
        }
        std::swap(cur, nxt);
    }
    for (int q = 0; q < nq; q++)
        { ProfScope ps_(P_RESTORE, st);
        k_restore<T><<<gf, b, 0, st>>>(d, psi_in[q], psi_out[q], sadd ? sadd[q] : nullptr, dt_add,
                                       gate, w.M + q);
        }
    return cudaGetLastError() == cudaSuccess ? 0 : DCM_E_CUDA;
}

// bare donor cell: first_order_upstream_3d (interior update only)
template <typename T>
int upwind_run(MpdataWork<T>& w, const Dims& d, const Metrics<T>& mt, T dt, const T* u,
               const T* v, const T* wv, const T* psi_in, T* psi_out, int neumann,
               cudaStream_t st) {
    const dim3 g = interior_grid(d, d.kp), b(BX, BY);
    Vel<T> V0{u, v, wv};
    { ProfScope ps_(P_UPWIND, st);
    k_upwind<T, false, false><<<g, b, 0, st>>>(d, mt, dt, V0, psi_in, psi_out, neumann, 0, nullptr,
                                               T(0), nullptr, nullptr, w.Mzero, nullptr);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : DCM_E_CUDA;
}

template int mpdata_run<double>(MpdataWork<double>&, const Dims&, const Metrics<double>&, double,
                                const double*, const double*, const double*, double* const*,
                                double* const*, int, const double*, const double*, int, int, int,
                                int, bool, const double* const*, double, cudaStream_t);
template int mpdata_run<float>(MpdataWork<float>&, const Dims&, const Metrics<float>&, float,
                               const float*, const float*, const float*, float* const*,
                               float* const*, int, const double*, const double*, int, int, int,
                               int, bool, const float* const*, float, cudaStream_t);
template int upwind_run<float>(MpdataWork<float>&, const Dims&, const Metrics<float>&, float,
                               const float*, const float*, const float*, const float*, float*,
                               int, cudaStream_t);
template int upwind_run<double>(MpdataWork<double>&, const Dims&, const Metrics<double>&, double,
                                const double*, const double*, const double*, const double*,
                                double*, int, cudaStream_t);

}  // namespace dcm
