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
        const T two = T(2);
        const T uc = V.u[d.at(k, j, i)], um = V.u[d.at(k, j, i - 1)];
        const T vc = V.v[d.at(k, j, i)], vm = V.v[d.at(k, j - 1, i)];
        const T wc = V.w[d.at(k, j, i)], wm = V.w[d.at(k - 1, j, i)];
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
        const T nv = pc - (fxr - fxl) - (fyr - fyl) - (fzr - fzl);  // :115
        if (FIRST) acc[0] += (double)pc;
        if (LAST) {
            const T lb = (T)M->lbc + m, ub = (T)M->ubc + m;
            if (exch == 0) {
                dst[d.at(k, j, i)] = nv + m;
            } else if (sadd) {
                // write every image with its own source term
                T* a = dst;
                const T vv = nv + m;
                a[d.at(k, j, i)] = vv + sadd[d.at(k, j, i)] * dt_add;
                const bool edge = (i == 1) | (i == d.ip) | (j == 1) | (j == d.jp) |
                                  (k == 1) | (k == d.kp);
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
    T us = adiv(adiv((fabs(uc) * dx - dt * uc * uc) * (P(k, j, i + 1) - pc),
                     P(k, j, i + 1) + pc + small),
                dxn) -
           u_j_bar1;
    T vs = adiv(adiv((fabs(vc) * dy - dt * vc * vc) * (P(k, j + 1, i) - pc),
                     P(k, j + 1, i) + pc + small),
                dyn) -
           u_j_bar2;
    T ws = adiv(adiv((fabs(wc) * dz - dt * adiv(ra, g_bar3) * wc * wc) * (P(k + 1, j, i) - pc),
                     P(k + 1, j, i) + pc + small),
                dzn) -
           u_j_bar3;
    us = us - q4 * dt * uc * (adiv(U(k, j, i + 1) - U(k, j, i - 1), dxm) + u_div1);  // :489-499
    vs = vs - q4 * dt * vc * (adiv(V(k, j + 1, i) - V(k, j - 1, i), dym) + u_div2);
    ws = ws - q4 * dt * wc * (adiv(rap * W(k + 1, j, i) - ram * W(k - 1, j, i), dzm * g_bar3) + u_div3);
    // exchange_full(..., 0, 0) of the new velocities, :528-533
    put_full(out.u, d, k, j, i, us, T(0), T(0));
    put_full(out.v, d, k, j, i, vs, T(0), T(0));
    put_full(out.w, d, k, j, i, ws, T(0), T(0));
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
            dt * ((fmax(U(k, j, i - 1), z) * rn * PO(k, j, i - 1) - fmin(U(k, j, i), z) * rn * PO(k, j, i + 1)) /
                      dxn +
                  (fmax(V(k, j - 1, i), z) * rn * PO(k, j - 1, i) - fmin(V(k, j, i), z) * rn * PO(k, j + 1, i)) /
                      dyn +
                  (fmax(W(k - 1, j, i), z) * ram * PO(k - 1, j, i) - fmin(W(k, j, i), z) * ra * PO(k + 1, j, i)) /
                      dzn) +
            small;
        const T denom2 =
            dt * ((fmax(U(k, j, i), z) * rn * pc - fmin(U(k, j, i - 1), z) * rn * pc) / dxn +
                  (fmax(V(k, j, i), z) * rn * pc - fmin(V(k, j - 1, i), z) * rn * pc) / dyn +
                  (fmax(W(k, j, i), z) * ra * pc - fmin(W(k - 1, j, i), z) * ram * pc) / dzn + small);
        const T bup = rn * (pmax - pc) / denom1;
        const T bdn = rn * (pc - pmin) / denom2;
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
    const T z = T(0), one = T(1);
    const int o = d.at(k, j, i);
    const T uc = Vt.u[o], vc = Vt.v[o], wc = Vt.w[o];
    // beta arrays per direction: (up, down)
    const T *iup = b0, *idn = b1, *jup = VARIANT ? b2 : b0, *jdn = VARIANT ? b3 : b1,
            *kup = VARIANT ? b4 : b0, *kdn = VARIANT ? b5 : b1;
    const T lu = fmin(fmin(one, idn[o]), iup[d.at(k, j, i + 1)]) * fmax(uc, z) +
                 fmin(fmin(one, iup[o]), idn[d.at(k, j, i + 1)]) * fmin(uc, z);
    const T lv = fmin(fmin(one, jdn[o]), jup[d.at(k, j + 1, i)]) * fmax(vc, z) +
                 fmin(fmin(one, jup[o]), jdn[d.at(k, j + 1, i)]) * fmin(vc, z);
    const T lw = fmin(fmin(one, kdn[o]), kup[d.at(k + 1, j, i)]) * fmax(wc, z) +
                 fmin(fmin(one, kup[o]), kdn[d.at(k + 1, j, i)]) * fmin(wc, z);
    // exchange_full(..., 0, 0), :669-674
    put_full(out.u, d, k, j, i, lu, z, z);
    put_full(out.v, d, k, j, i, lv, z, z);
    put_full(out.w, d, k, j, i, lw, z, z);
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
        const bool last = it == kord;
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
