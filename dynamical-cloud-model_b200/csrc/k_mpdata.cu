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
// donor-cell pass of field 0 (:319-695), fused along i-planes over tiles of
// rows and k-levels.  A block owns the output rows j0..j0+JT-1 of an i-chunk
// [i0, i1] and of a k-tile of MPK_OUT levels kb..kb+MPK_OUT-1; it keeps
// R = JT + H + 1 warps, one per row j0-H .. j0+JT (H = 2 with the limiter,
// 1 without; halo rows take the periodic image of their j), and lane l of a
// warp holds level kb - 2 + l, so a warp covers its tile with a halo of two
// levels below and two above.  Levels outside 1..kp hold the exchanges'
// boundary value 0 of every stage.  The stages march over the planes skewed
// by one plane each:
//   step f:  A (antidiffusive velocities) at plane f     (rows 0..R-1)
//            beta at plane f-1                            (rows 1..R-1)
//            L (limited velocities) at plane f-2          (rows 1..R-2)
//            donor cell of field 0 at plane f-3           (owned rows)
// with one barrier per step: every value a stage takes from another warp
// was written in the previous step, so the four stages of a step are
// independent chains a warp can overlap.  k neighbours of a stage's inputs
// are the neighbour lanes (shuffles), j neighbours the neighbour warps'
// values in small shared planes (the v component of A, the betas, the v
// component of L; two plane parities each), i neighbours and a point's own
// values registers.
// Only the limited velocities (exchange_full images, the next iteration's
// input) and the new field 0 reach memory; A and beta never do.  Without the
// limiter the donor cell runs on A at plane f and A is the output set.  Each
// quantity is the same point function as the separate kernels evaluate.
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
    int JT, ni;             // owned rows, planes per chunk
};

constexpr int MPK_OUT = 28;  // output levels of a k-tile (32 lanes, a halo of 2 each side)

// rows (warps) per block of the fused iteration: 24 (FP32, <= 85 registers a
// thread, the occupancy of the separate antidiffusive-velocity kernel) or 8
// (FP64)
template <typename T>
constexpr int mp_iter_max_rows() { return sizeof(T) == 4 ? 24 : 8; }

template <typename T, bool MONO, bool LAST>
__global__ void __launch_bounds__(32 * mp_iter_max_rows<T>()) k_mpdata_iter(MpIterArgs<T> a) {
    extern __shared__ __align__(16) unsigned char mp_smem[];
    T* sm = reinterpret_cast<T*>(mp_smem);
    if (a.gate->early) return;
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31, r = threadIdx.x >> 5, R = blockDim.x >> 5;
    const int kp = d.kp;
    constexpr int H = MONO ? 2 : 1;
    const int j0 = 1 + blockIdx.x * a.JT;
    const int jr = wrapj(j0 - H + r, d.jp);
    const int i0 = 1 + blockIdx.y * a.ni, i1 = min(i0 + a.ni - 1, d.ip);
    const int k = 1 + MPK_OUT * (int)blockIdx.z - 2 + lane;
    const bool inK = k >= 1 && k <= kp;
    const bool rowown = r >= H && r <= R - 2 && j0 - H + r <= d.jp;
    const bool own = rowown && inK && lane >= 2 && lane < 2 + MPK_OUT;
    const T m = (T)a.M->m;
    const T z = T(0);
    constexpr unsigned FULL = 0xffffffffu;
    // shared planes [parity][row][lane]: A_v (0, 1), beta_up (2, 3), beta_dn
    // (4, 5), L_v (6, 7); a plane's values are read one step after they are
    // written, so one barrier per step orders them
    auto sp = [&](int plane, int par, int row) -> T& {
        return sm[((plane * 2 + par) * R + row) * 32 + lane];
    };
    auto Pf = [&](int kk, int jj, int ii) -> T { return a.pso[d.at(kk, jj, ii)]; };
    // own-point windows along i
    T A1u = z, A1v = z, A1w = z;  // A at plane f-1
    T A2u = z, A2v = z, A2w = z;  // A at plane f-2
    T B2u = z, B2d = z;           // beta at plane f-2
    T L3u = z, L3v = z, L3w = z;  // L at plane f-3
    T L4u = z;                    // L_u at plane f-4
    if (MONO) {
        // step f: A at f, beta at f-1, L at f-2, donor cell at f-3
        for (int f = i0 - 2; f <= i1 + 3; f++) {
            const int p0 = f & 1, p1 = p0 ^ 1;  // parities of planes f (and f-2), f-1 (and f-3)
            // ---- A at plane f (every row; lane 31 is never read)
            T Au = z, Av = z, Aw = z;
            if (f <= i1 + 1 && inK && lane < 31)
                antidiff_point(d, a.mt, a.dt, a.Vt, a.pso, k, jr, wrapj(f, d.ip), Au, Av, Aw);
            sp(0, p0, r) = Av;
            // ---- beta at plane f-1 (lanes 1..30)
            T Bu = z, Bd = z;
            const T A1wm = __shfl_up_sync(FULL, A1w, 1);  // A_w at k-1, plane f-1
            if (f >= i0 && f <= i1 + 2 && r >= 1 && inK && lane >= 1 && lane <= 30)
                beta0_point(d, a.mt, a.dt, m, a.psi_in, a.pso, k, jr, wrapj(f - 1, d.ip), A2u,
                            A1u, sp(0, p1, r - 1), A1v, A1wm, A1w, Bu, Bd);
            sp(1, p1, r) = Bu;
            sp(2, p1, r) = Bd;
            // ---- L at plane f-2 (lanes 1..29)
            const T b2un = __shfl_down_sync(FULL, B2u, 1), b2dn = __shfl_down_sync(FULL, B2d, 1);
            T Lu = z, Lv = z, Lw = z;
            if (f >= i0 + 1 && f <= i1 + 2 && r >= 1 && r <= R - 2 && inK && lane >= 1 &&
                lane <= 29) {
                Lu = limit_comp(A2u, B2u, B2d, Bu, Bd);
                Lv = limit_comp(A2v, B2u, B2d, sp(1, p0, r + 1), sp(2, p0, r + 1));
                Lw = limit_comp(A2w, B2u, B2d, b2un, b2dn);
                if (own && f - 2 >= i0) {  // exchange_full(..., 0, 0), :669-674
                    const int fm = wrapj(f - 2, d.ip);
                    put_full(a.vout.u, d, k, jr, fm, Lu, z, z);
                    put_full(a.vout.v, d, k, jr, fm, Lv, z, z);
                    put_full(a.vout.w, d, k, jr, fm, Lw, z, z);
                }
            }
            sp(3, p0, r) = Lv;
            // ---- donor cell of field 0 at plane f-3 (lanes 2..29, owned rows)
            const T L3wm = __shfl_up_sync(FULL, L3w, 1);
            if (f >= i0 + 3 && own) {
                const int f3 = wrapj(f - 3, d.ip);
                const T nv = donor_point(d, a.mt, a.dt, a.neumann, k, jr, f3, L3u, L4u, L3v,
                                         sp(3, p1, r - 1), L3w, L3wm, Pf);
                donor_store<T, LAST>(a.dst, d, k, jr, f3, nv, 1, a.sadd, a.dt_add, a.M, m);
            }
            __syncthreads();
            A2u = A1u; A2v = A1v; A2w = A1w;
            A1u = Au; A1v = Av; A1w = Aw;
            B2u = Bu; B2d = Bd;
            L4u = L3u;
            L3u = Lu; L3v = Lv; L3w = Lw;
        }
    } else {
        // step f: A at f, donor cell on A at f-1
        for (int f = i0 - 1; f <= i1 + 1; f++) {
            const int p0 = f & 1, p1 = p0 ^ 1;
            T Au = z, Av = z, Aw = z;
            if (f <= i1 && inK && lane < 31)
                antidiff_point(d, a.mt, a.dt, a.Vt, a.pso, k, jr, wrapj(f, d.ip), Au, Av, Aw);
            sp(0, p0, r) = Av;
            const T A1wm = __shfl_up_sync(FULL, A1w, 1);
            if (f >= i0 + 1 && own) {
                const int f1 = wrapj(f - 1, d.ip);
                const T nv = donor_point(d, a.mt, a.dt, a.neumann, k, jr, f1, A1u, A2u, A1v,
                                         sp(0, p1, r - 1), A1w, A1wm, Pf);
                put_full(a.vout.u, d, k, jr, f1, A1u, z, z);  // :528-533
                put_full(a.vout.v, d, k, jr, f1, A1v, z, z);
                put_full(a.vout.w, d, k, jr, f1, A1w, z, z);
                donor_store<T, LAST>(a.dst, d, k, jr, f1, nv, 1, a.sadd, a.dt_add, a.M, m);
            }
            __syncthreads();
            A2u = A1u;
            A1u = Au; A1v = Av; A1w = Aw;
        }
    }
}

// Launch shape of the fused iteration: R rows per block (the row cap), k-tiles
// of MPK_OUT levels, and i-chunks so that the grid fills every SM with as
// many blocks as fit on it at once, with chunks of at least 4 planes.
struct MpIterShape {
    int R = 0, JT = 0, ni = 0, nstrips = 0, nchunks = 0, ntiles = 0;
    size_t smem = 0;
};

template <typename T, bool MONO, bool LAST>
__global__ void k_mpdata_iter(MpIterArgs<T> a);

template <typename T>
static MpIterShape mp_iter_shape(const Dims& d, bool mono, int max_rows) {
    MpIterShape s;
    const int H = mono ? 2 : 1;
    int R = std::min(mp_iter_max_rows<T>(), max_rows);
    R = std::min(R, d.jp + H + 1);  // no more rows than the domain has
    if (R < H + 2) return s;        // not even one owned row
    s.R = R;
    s.JT = R - H - 1;
    s.smem = (size_t)8 * R * 32 * sizeof(T);
    s.nstrips = (d.jp + s.JT - 1) / s.JT;
    s.ntiles = (d.kp + MPK_OUT - 1) / MPK_OUT;
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
    const long long plane_blocks = (long long)s.nstrips * s.ntiles;
    const long long want = ((long long)sms * per_sm + plane_blocks - 1) / plane_blocks;
    const int nch = (int)std::max(1LL, std::min((long long)(d.ip + 3) / 4, want));
    s.ni = (d.ip + nch - 1) / nch;
    s.nchunks = (d.ip + s.ni - 1) / s.ni;
    return s;
}

template <typename T, bool MONO, bool LAST>
static bool launch_mp_iter(const MpIterArgs<T>& args, const MpIterShape& s, cudaStream_t st) {
    const dim3 grid(s.nstrips, s.nchunks, s.ntiles), block(32 * s.R);
    k_mpdata_iter<T, MONO, LAST><<<grid, block, s.smem, st>>>(args);
    return true;
}

// the opt-in shared-memory limit of every fused-iteration kernel (called
// once at handle creation, outside any stream capture)
template <typename T, bool MONO, bool LAST>
static void mp_iter_attrs() {
    // the shared planes are small (6 x rows x 32 values); prefer L1 for the
    // stencil reads of the antidiffusive velocities
    cudaFuncSetAttribute(k_mpdata_iter<T, MONO, LAST>,
                         cudaFuncAttributePreferredSharedMemoryCarveout, 10);
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
            ia.JT = fs.JT; ia.ni = fs.ni;
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
