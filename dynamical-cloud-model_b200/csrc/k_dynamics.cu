// k_dynamics.cu -- the non-solver, non-advection parts of the time step:
// horizontal means and divergence (diagnostics.f90), momentum sources and
// the Poisson right-hand side (dynamics.f90:639-1000), the leap-frog
// momentum update with the time filter and velocity boundary rows
// (dynamics.f90:1019-1099, driver_code.f90:592-674), adv_ref_state
// (pamm/sfvt/advection_3d.F90:1148-1218), advance_scalar_fields_3d
// (sgm/subgrid_3d.f90:582-624) and the stand-alone halo exchanges.
#include <algorithm>

#include "dcm_internal.h"
#include "dcm_prof.h"

namespace dcm {

// ---- stand-alone exchanges ------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_exchange(Dims d, T* __restrict__ a, int mode,
                                                  T lbc, T ubc) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const T v = a[d.at(k, j, i)];
    if (mode == HALO_FULL)
        put_full(a, d, k, j, i, v, lbc, ubc);
    else if (mode == HALO_FULL_WO)
        put_full<T, true>(a, d, k, j, i, v, lbc, ubc);
    else if (mode == HALO_DIM)
        put_dim(a, d, k, j, i, v, lbc, ubc);
    else
        put_wo(a, d, k, j, i, v);
}

template <typename T>
void launch_exchange(const Dims& d, T* a, int mode, T lbc, T ubc, cudaStream_t st) {
    { ProfScope ps_(P_OTHER, st);
    k_exchange<T><<<interior_grid(d, d.kp), dim3(BX, BY), 0, st>>>(d, a, mode, lbc, ubc);
    }
}

// ---- horizontal means (+ divergence) --------------------------------------
// threadIdx.x -> k (0..kp+1), threadIdx.y + blockIdx.y -> a fixed strided
// set of (j,i) columns; per-(field, k) partials reduced in a fixed order by
// the last block.  means layout: [field][k], k = 0..kp+1.

template <typename T, int NF, typename D>
__global__ void __launch_bounds__(256) k_means(Dims d, Metrics<D> mt, const T* f0, const T* f1,
                                               const T* f2, const T* f3, T* __restrict__ means,
                                               D* __restrict__ div, double* partials,
                                               unsigned int* ticket) {
    __shared__ double red[NF][BY][BX];
    const int k = blockIdx.x * BX + threadIdx.x;
    const int ncol = d.ip * d.jp;
    const T* f[4] = {f0, f1, f2, f3};
    double acc[NF];
#pragma unroll
    for (int q = 0; q < NF; q++) acc[q] = 0.0;
    if (k <= d.kp + 1) {
        for (int c = blockIdx.y * BY + threadIdx.y; c < ncol; c += gridDim.y * BY) {
            const int j = 1 + c % d.jp, i = 1 + c / d.jp;
            const int o = d.at(k, j, i);
#pragma unroll
            for (int q = 0; q < NF; q++) acc[q] += (double)f[q][o];
            if (div && k >= 1 && k <= d.kp) {
                // divergence_calc, diagnostics.f90:144-146
                // in D (FP64 for the mixed-precision form: the divergence check)
                const T* u = f0;
                const T* v = f1;
                const T* w = f2;
                const D rn = ld(mt.rhoan + k);
                div[o] = rn * ((D)u[o] - (D)u[d.at(k, j, i - 1)]) / ld(mt.dx + i - 1) +
                         rn * ((D)v[o] - (D)v[d.at(k, j - 1, i)]) / ld(mt.dy + j - 1) +
                         (ld(mt.rhoa + k) * (D)w[o] - ld(mt.rhoa + k - 1) * (D)w[d.at(k - 1, j, i)]) /
                             ld(mt.dz + k - 1);
            }
        }
    }
#pragma unroll
    for (int q = 0; q < NF; q++) red[q][threadIdx.y][threadIdx.x] = acc[q];
    __syncthreads();
    const unsigned int nbk = gridDim.x, nby = gridDim.y;
    const int K2 = d.kp + 2;
    if (threadIdx.y == 0 && k <= d.kp + 1) {
#pragma unroll
        for (int q = 0; q < NF; q++) {
            double s = 0.0;
            for (int y = 0; y < BY; y++) s += red[q][y][threadIdx.x];
            partials[((size_t)q * K2 + k) * nby + blockIdx.y] = s;
        }
    }
    __shared__ bool s_last;
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0 && threadIdx.y == 0) {
        const unsigned int t = atomicAdd(ticket, 1u);
        s_last = (t == nbk * nby - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const double area = (double)(d.ip * d.jp);
    const int tid = threadIdx.x + BX * threadIdx.y;
    for (int e = tid; e < NF * K2; e += BX * BY) {
        const volatile double* p = partials + (size_t)e * nby;
        double s = 0.0;
        for (unsigned int b = 0; b < nby; b++) s += p[b];
        means[e] = (T)(s / area);  // diagnostics.f90:90-95
    }
    if (tid == 0) *ticket = 0u;
}

template <typename T, typename D>
void launch_means_div(const Dims& d, const Metrics<D>& mt, const T* u, const T* v, const T* w,
                      const T* th, T* const* q, int nq, T* means, D* div, double* partials,
                      unsigned int* ticket, cudaStream_t st) {
    const int K2 = d.kp + 2;
    const dim3 g((K2 + BX - 1) / BX, MEAN_GY), b(BX, BY);
    { ProfScope ps_(P_MEANS, st);
    k_means<T, 4, D><<<g, b, 0, st>>>(d, mt, u, v, w, th, means, div, partials, ticket);
    }
    for (int q0 = 0; q0 < nq; q0 += 4) {
        const int n = nq - q0 < 4 ? nq - q0 : 4;
        T* out = means + (size_t)(4 + q0) * K2;
        if (n == 4)
            { ProfScope ps_(P_MEANS, st);
            k_means<T, 4, D><<<g, b, 0, st>>>(d, mt, q[q0], q[q0 + 1], q[q0 + 2], q[q0 + 3], out,
                                           nullptr, partials, ticket);
            }
        else if (n == 3)
            { ProfScope ps_(P_MEANS, st);
            k_means<T, 3, D><<<g, b, 0, st>>>(d, mt, q[q0], q[q0 + 1], q[q0 + 2], nullptr, out,
                                           nullptr, partials, ticket);
            }
        else if (n == 2)
            { ProfScope ps_(P_MEANS, st);
            k_means<T, 2, D><<<g, b, 0, st>>>(d, mt, q[q0], q[q0 + 1], nullptr, nullptr, out,
                                           nullptr, partials, ticket);
            }
        else
            { ProfScope ps_(P_MEANS, st);
            k_means<T, 1, D><<<g, b, 0, st>>>(d, mt, q[q0], nullptr, nullptr, nullptr, out,
                                           nullptr, partials, ticket);
            }
    }
}

// ---- sources ----------------------------------------------------------------
// One thread per interior cell computes su, sv, sw (dynamics.f90:743-797),
// the optional damping / forcing / subsidence terms (:802-873), then writes
// the exchange_full(0,0) images (:909-916) combined with the surface / lid
// rows (:922-973):
//   su, sv: level 0 = -(level 1 images), levels kp and kp+1 = 0
//   sw:     level 0 = 0, levels kp and kp+1 = 0
//   sth:    exchange_full(0,0) images
template <typename T>
__global__ void __launch_bounds__(256) k_sources(Dims d, Metrics<T> mt, Forcing<T> F,
                                                 const T* __restrict__ ubar,
                                                 const T* __restrict__ vbar,
                                                 const T* __restrict__ wbar,
                                                 const T* __restrict__ thbar,
                                                 const T* __restrict__ zu,
                                                 const T* __restrict__ zv,
                                                 const T* __restrict__ zw,
                                                 const T* __restrict__ u,
                                                 const T* __restrict__ v,
                                                 const T* __restrict__ w,
                                                 const T* __restrict__ th, T* __restrict__ su,
                                                 T* __restrict__ sv, T* __restrict__ sw,
                                                 T* __restrict__ sth, int sth_reset,
                                                 int interior_only) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    auto U = [&](int kk, int jj, int ii) { return u[d.at(kk, jj, ii)]; };
    auto V = [&](int kk, int jj, int ii) { return v[d.at(kk, jj, ii)]; };
    auto W = [&](int kk, int jj, int ii) { return w[d.at(kk, jj, ii)]; };
    const T two = T(2);
    const T dx = ld(mt.dx + i), dxm = ld(mt.dx + i - 1), dxn = ld(mt.dxn + i),
            dxnm = ld(mt.dxn + i - 1);
    const T dy = ld(mt.dy + j), dym = ld(mt.dy + j - 1), dyn = ld(mt.dyn + j),
            dynm = ld(mt.dyn + j - 1);
    const T dz = ld(mt.dz + k), dzm = ld(mt.dz + k - 1), dzn = ld(mt.dzn + k),
            dznm = ld(mt.dzn + k - 1);
    const T rn = ld(mt.rhoan + k), ra = ld(mt.rhoa + k);
    const int o = d.at(k, j, i);
    // :746-754
    T vsu = rn * (((U(k, j, i - 1) * (U(k, j, i) + U(k, j, i - 1)) -
                    U(k, j, i + 1) * (U(k, j, i) + U(k, j, i + 1))) /
                       (two * (dx + dxm)) +
                   (U(k, j - 1, i) * (V(k, j - 1, i) + V(k, j - 1, i + 1)) -
                    U(k, j + 1, i) * (V(k, j, i) + V(k, j, i + 1))) /
                       (two * (dyn + dynm)) +
                   (U(k - 1, j, i) * (W(k - 1, j, i) + W(k - 1, j, i + 1)) -
                    U(k + 1, j, i) * (W(k, j, i) + W(k, j, i + 1))) /
                       (two * (dzn + dznm))));
    // :765-773
    T vsv = rn * (((V(k, j, i - 1) * (U(k, j, i - 1) + U(k, j + 1, i - 1)) -
                    V(k, j, i + 1) * (U(k, j, i) + U(k, j + 1, i))) /
                       (two * (dxn + dxnm)) +
                   (V(k, j - 1, i) * (V(k, j, i) + V(k, j - 1, i)) -
                    V(k, j + 1, i) * (V(k, j, i) + V(k, j + 1, i))) /
                       (two * (dy + dym)) +
                   (V(k - 1, j, i) * (W(k - 1, j, i) + W(k - 1, j + 1, i)) -
                    V(k + 1, j, i) * (W(k, j, i) + W(k, j + 1, i))) /
                       (two * (dzn + dznm))));
    // :784-794
    T vsw = ra * (((W(k, j, i - 1) * (U(k, j, i - 1) + U(k + 1, j, i - 1)) -
                    W(k, j, i + 1) * (U(k, j, i) + U(k + 1, j, i))) /
                       (two * (dxn + dxnm)) +
                   (W(k, j - 1, i) * (V(k, j - 1, i) + V(k + 1, j - 1, i)) -
                    W(k, j + 1, i) * (V(k, j, i) + V(k + 1, j, i))) /
                       (two * (dyn + dynm)) +
                   (W(k - 1, j, i) * (W(k, j, i) + W(k - 1, j, i)) -
                    W(k + 1, j, i) * (W(k, j, i) + W(k + 1, j, i))) /
                       (two * (dz + dzm))) +
                  T(9.81) * (th[o] + th[d.at(k + 1, j, i)]) /
                      (two * ld(mt.theta + k) + ld(thbar + k) + ld(thbar + k + 1)));
    T vsth = sth_reset ? T(0) : sth[o];
    if (F.damping_layer) {
        vsu = vsu + rn * ld(F.dampfacn + k) * (zu[o] - ld(ubar + k));
        vsv = vsv + rn * ld(F.dampfacn + k) * (zv[o] - ld(vbar + k));
        vsw = vsw + ra * ld(F.dampfac + k) * (zw[o] - T(0));
        vsth = vsth + ld(F.dampfacn + k) * (th[o] - T(0));
    }
    if (F.forcing) {
        vsu = vsu - rn * (zu[o] - ld(F.u_force + k)) / F.forcing_tau;
        vsv = vsv - rn * (zv[o] - ld(F.v_force + k)) / F.forcing_tau;
    }
    if (F.divergence) vsw = vsw - rn * (ld(wbar + k) - ld(F.w_subs + k));
    if (interior_only) {
        // viscous = .true.: the subgrid model adds to these values and writes
        // the images and rows (dynamics.f90:878-893)
        su[o] = vsu;
        sv[o] = vsv;
        sw[o] = vsw;
        sth[o] = vsth;
        return;
    }
    const T z = T(0);
    put_full(sth, d, k, j, i, vsth, z, z);
    if (k == d.kp) {
        put_plane_images(su, d, d.kp, j, i, z);
        put_plane_images(su, d, d.kp + 1, j, i, z);
        put_plane_images(sv, d, d.kp, j, i, z);
        put_plane_images(sv, d, d.kp + 1, j, i, z);
        put_plane_images(sw, d, d.kp, j, i, z);
        put_plane_images(sw, d, d.kp + 1, j, i, z);
    } else {
        put_plane_images(su, d, k, j, i, vsu);
        put_plane_images(sv, d, k, j, i, vsv);
        put_plane_images(sw, d, k, j, i, vsw);
        if (k == 1) {
            put_plane_images(su, d, 0, j, i, -vsu);
            put_plane_images(sv, d, 0, j, i, -vsv);
            put_plane_images(sw, d, 0, j, i, z);
        }
    }
}

// rhs of the Poisson equation, dynamics.f90:977-998 (k = 0..kp+1); with wo
// also the driver's exchange_along_dim_wo(psrc), driver_code.f90:485-487
template <typename T, typename R>
__global__ void __launch_bounds__(256) k_rhs(Dims d, Metrics<R> mt, const T* __restrict__ su,
                                             const T* __restrict__ sv,
                                             const T* __restrict__ sw, R* __restrict__ rhs,
                                             int wo) {
    const int k = blockIdx.x * BX + threadIdx.x;  // 0..kp+1
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp + 1 || j > d.jp) return;
    const int o = d.at(k, j, i);
    // in R: FP64 in the mixed-precision form, so that the right-hand side of
    // the singular (periodic / Neumann) Poisson problem sums to zero to FP64
    // round-off and the FP64-refined solve stays consistent
    R r;
    if (k >= 1) {
        r = (((R)su[o] - (R)su[d.at(k, j, i - 1)]) / ld(mt.dx + i - 1) +
             ((R)sv[o] - (R)sv[d.at(k, j - 1, i)]) / ld(mt.dy + j - 1) +
             ((R)sw[o] - (R)sw[d.at(k - 1, j, i)]) / ld(mt.dz + k - 1));
    } else {
        r = (((R)su[o] - (R)su[d.at(0, j, i - 1)]) / ld(mt.dx + i - 1) +
             ((R)sv[o] - (R)sv[d.at(0, j - 1, i)]) / ld(mt.dy + j - 1) +
             ((R)sw[o] + (R)sw[d.at(1, j, i)]) / ld(mt.dz + 1));
    }
    if (wo && k >= 1 && k <= d.kp)
        put_wo(rhs, d, k, j, i, r);
    else
        rhs[o] = r;
}

template <typename T, typename R>
void launch_sources(const Dims& d, const Metrics<T>& mt, const Metrics<R>& mtr,
                    const Forcing<T>& f, const T* ubar, const T* vbar, const T* wbar,
                    const T* thbar, const T* zu, const T* zv, const T* zw, const T* u, const T* v,
                    const T* w, const T* th, T* su, T* sv, T* sw, T* sth, R* rhs, int sth_reset,
                    int rhs_wo, cudaStream_t st, const SgsStep<T>* sg) {
    const dim3 b(BX, BY);
    { ProfScope ps_(P_SOURCES, st);
    k_sources<T><<<interior_grid(d, d.kp), b, 0, st>>>(d, mt, f, ubar, vbar, wbar, thbar, zu, zv,
                                                       zw, u, v, w, th, su, sv, sw, sth,
                                                       sth_reset, sg ? 1 : 0);
    }
    if (sg) {
        // the subgrid model, then the rows of sources on su, sv, sw; sq is
        // zeroed each step by the driver (driver_code.f90:342), so each q's
        // diffusion term replaces it
        ScalarSet<T> sets[SGS_MAX_SETS];
        const int ns = make_scalar_sets<T>(th, sth, 0, sg->q, sg->sq, sg->nq, 1, sets,
                                           SGS_MAX_SETS);
        launch_subgrid<T>(d, mt, sg->P, u, v, w, zu, zv, zw, th, sg->vism, sg->vist, sg->strain,
                          sg->tau, su, sv, sw, sets, ns < 0 ? 0 : ns, true, st);
    }
    { ProfScope ps_(P_RHS, st);
    k_rhs<T, R><<<interior_grid(d, d.kp + 2), b, 0, st>>>(d, mtr, su, sv, sw, rhs, rhs_wo);
    }
}

// ---- advance_momentum (drop-in, k = 0..kp, dynamics.f90:1053-1094) --------
template <typename T>
__global__ void __launch_bounds__(256) k_advance_momentum(Dims d, Metrics<T> mt, T dt,
                                                          T* __restrict__ u, T* __restrict__ v,
                                                          T* __restrict__ w,
                                                          const T* __restrict__ zu,
                                                          const T* __restrict__ zv,
                                                          const T* __restrict__ zw,
                                                          const T* __restrict__ su,
                                                          const T* __restrict__ sv,
                                                          const T* __restrict__ sw,
                                                          const T* __restrict__ p) {
    const int k = blockIdx.x * BX + threadIdx.x;  // 0..kp
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const int o = d.at(k, j, i);
    const T pc = p[o];
    u[o] = zu[o] + ((su[o] - (p[d.at(k, j, i + 1)] - pc) / (ld(mt.dxn + i))) * dt) /
                       ld(mt.rhoan + k);
    v[o] = zv[o] + ((sv[o] - (p[d.at(k, j + 1, i)] - pc) / (ld(mt.dyn + j))) * dt) /
                       ld(mt.rhoan + k);
    w[o] = zw[o] + ((sw[o] - (p[d.at(k + 1, j, i)] - pc) / (ld(mt.dzn + k))) * dt) /
                       ld(mt.rhoa + k);
}

template <typename T>
void launch_advance_momentum(const Dims& d, const Metrics<T>& mt, T dt, T* u, T* v, T* w,
                             const T* zu, const T* zv, const T* zw, const T* su, const T* sv,
                             const T* sw, const T* p, cudaStream_t st) {
    { ProfScope ps_(P_MOMENTUM, st);
    k_advance_momentum<T><<<interior_grid(d, d.kp + 1), dim3(BX, BY), 0, st>>>(
        d, mt, dt, u, v, w, zu, zv, zw, su, sv, sw, p);
    }
}

// ---- resident momentum step ---------------------------------------------------
// Every cell (halo included): time filter u <- 0.99 u + 0.01 zu in place
// (driver_code.f90:618-626; the smoothed zu is never read again after the
// rotation :634-646, so it is not formed).  Interior cells k = 1..kp: the
// leap-frog update into tu (dynamics.f90:1056-1091 with 2dt), written with
// the exchange_full(0,0) images of the rotated u (:656-661) and the rows of
// :663-674: u(0) = -u(1), v(0) = -v(1), w(0) = 0, u(kp+1) = u(kp),
// v(kp+1) = v(kp), w(kp+1) = 0.
template <typename T, typename P>
__global__ void __launch_bounds__(256) k_momentum_step(Dims d, Metrics<T> mt, Metrics<P> mtp, T dt2,
                                                       T* __restrict__ u, T* __restrict__ v,
                                                       T* __restrict__ w,
                                                       const T* __restrict__ zu,
                                                       const T* __restrict__ zv,
                                                       const T* __restrict__ zw,
                                                       T* __restrict__ tu, T* __restrict__ tv,
                                                       T* __restrict__ tw,
                                                       const T* __restrict__ su,
                                                       const T* __restrict__ sv,
                                                       const T* __restrict__ sw,
                                                       const P* __restrict__ p) {
    const int k = blockIdx.x * BX + threadIdx.x;  // 0..kp+1
    const int j = blockIdx.y * BY + threadIdx.y;  // 0..jp+1
    const int i = blockIdx.z;                     // 0..ip+1
    if (k > d.kp + 1 || j > d.jp + 1) return;
    const int o = d.at(k, j, i);
    const T c99 = T(0.99), c01 = T(0.01);
    const T zuo = zu[o], zvo = zv[o], zwo = zw[o];
    u[o] = c99 * u[o] + c01 * zuo;
    v[o] = c99 * v[o] + c01 * zvo;
    w[o] = c99 * w[o] + c01 * zwo;
    if (k < 1 || k > d.kp || j < 1 || j > d.jp || i < 1 || i > d.ip) return;
    // pressure gradient in P (FP64 in the mixed-precision form, where p is
    // the refined FP64 solution), the rest in T
    const P pc = p[o];
    const T gx = (T)((p[d.at(k, j, i + 1)] - pc) / (ld(mtp.dxn + i)));
    const T gy = (T)((p[d.at(k, j + 1, i)] - pc) / (ld(mtp.dyn + j)));
    const T gz = (T)((p[d.at(k + 1, j, i)] - pc) / (ld(mtp.dzn + k)));
    const T nu = zuo + ((su[o] - gx) * dt2) / ld(mt.rhoan + k);
    const T nv = zvo + ((sv[o] - gy) * dt2) / ld(mt.rhoan + k);
    const T nw = zwo + ((sw[o] - gz) * dt2) / ld(mt.rhoa + k);
    put_plane_images(tu, d, k, j, i, nu);
    put_plane_images(tv, d, k, j, i, nv);
    put_plane_images(tw, d, k, j, i, nw);
    if (k == 1) {
        put_plane_images(tu, d, 0, j, i, -nu);
        put_plane_images(tv, d, 0, j, i, -nv);
        put_plane_images(tw, d, 0, j, i, T(0));
    }
    if (k == d.kp) {
        put_plane_images(tu, d, d.kp + 1, j, i, nu);
        put_plane_images(tv, d, d.kp + 1, j, i, nv);
        put_plane_images(tw, d, d.kp + 1, j, i, T(0));
    }
}

template <typename T, typename P>
void launch_momentum_step(const Dims& d, const Metrics<T>& mt, const Metrics<P>& mtp, T dt2,
                          T* u, T* v, T* w, const T* zu, const T* zv, const T* zw, T* tu, T* tv,
                          T* tw, const T* su, const T* sv, const T* sw, const P* p,
                          cudaStream_t st) {
    { ProfScope ps_(P_MOMENTUM, st);
    k_momentum_step<T, P><<<full_grid(d), dim3(BX, BY), 0, st>>>(d, mt, mtp, dt2, u, v, w, zu,
                                                                 zv, zw, tu, tv, tw, su, sv, sw,
                                                                 p);
    }
}

// ---- adv_ref_state -----------------------------------------------------------
// exch = 0: the subroutine alone (i, j over the halo too, k = 1..kp);
// exch = 1: followed by the driver's exchange_full(th, 0, 0), which
//           overwrites every halo cell, so only the interior is computed.
template <typename T>
__global__ void __launch_bounds__(256) k_adv_ref(Dims d, Metrics<T> mt, T dt,
                                                 const T* __restrict__ w,
                                                 const T* __restrict__ psi, T* __restrict__ out,
                                                 const T* __restrict__ ref, int exch) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = (exch ? 1 : 0) + blockIdx.y * BY + threadIdx.y;
    const int i = (exch ? 1 : 0) + blockIdx.z;
    if (k > d.kp || j > (exch ? d.jp : d.jp + 1)) return;
    const int o = d.at(k, j, i);
    const T h = T(0.5);
    const T v = psi[o] - dt *
                             (h / ld(mt.dz + k - 1) * w[d.at(k - 1, j, i)] * ld(mt.rhoa + k - 1) *
                                  (ld(ref + k) - ld(ref + k - 1)) +
                              h / ld(mt.dz + k) * w[o] * ld(mt.rhoa + k) *
                                  (ld(ref + k + 1) - ld(ref + k))) /
                             ld(mt.rhoan + k);
    if (exch)
        put_full(out, d, k, j, i, v, T(0), T(0));
    else
        out[o] = v;
}

template <typename T>
void launch_adv_ref_state(const Dims& d, const Metrics<T>& mt, T dt, const T* w, const T* psi,
                          T* out, const T* psi_ref, int exch, cudaStream_t st) {
    const dim3 g = exch ? interior_grid(d, d.kp)
                        : dim3((d.kp + BX - 1) / BX, (d.J + BY - 1) / BY, d.I);
    { ProfScope ps_(P_ADVREF, st);
    k_adv_ref<T><<<g, dim3(BX, BY), 0, st>>>(d, mt, dt, w, psi, out, psi_ref, exch);
    }
}

// ---- whole-array updates -------------------------------------------------------
template <typename T>
__global__ void k_axpy_all(size_t n, T dt, T* __restrict__ a, const T* __restrict__ s) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) a[e] = a[e] + s[e] * dt;
}

template <typename T>
void launch_advance_scalar(const Dims& d, T dt, T* a, const T* s, cudaStream_t st) {
    const size_t n = d.n();
    { ProfScope ps_(P_OTHER, st);
    k_axpy_all<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, dt, a, s);
    }
}

template <typename T>
__global__ void k_add_profile(Dims d, T* __restrict__ a, const T* __restrict__ prof, T sign) {
    const size_t n = d.n();
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n) return;
    const int k = (int)(e % d.K);
    if (k > d.kp + 1) return;  // column padding of the pitched layout
    a[e] = sign > T(0) ? a[e] + prof[k] : a[e] - prof[k];
}

template <typename T>
void launch_add_profile(const Dims& d, T* a, const T* prof, T sign, cudaStream_t st) {
    const size_t n = d.n();
    { ProfScope ps_(P_OTHER, st);
    k_add_profile<T><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(d, a, prof, sign);
    }
}

#define INST(T, D)                                                                              \
    template void launch_exchange<T>(const Dims&, T*, int, T, T, cudaStream_t);                 \
    template void launch_means_div<T, D>(const Dims&, const Metrics<D>&, const T*, const T*,    \
                                         const T*, const T*, T* const*, int, T*, D*, double*,   \
                                         unsigned int*, cudaStream_t);                          \
    template void launch_sources<T, D>(const Dims&, const Metrics<T>&, const Metrics<D>&,       \
                                       const Forcing<T>&, const T*, const T*, const T*,         \
                                       const T*, const T*, const T*, const T*, const T*,        \
                                       const T*, const T*, const T*, T*, T*, T*, T*, D*, int,   \
                                       int, cudaStream_t, const SgsStep<T>*);                   \
    template void launch_advance_momentum<T>(const Dims&, const Metrics<T>&, T, T*, T*, T*,     \
                                             const T*, const T*, const T*, const T*,            \
                                             const T*, const T*, const T*, cudaStream_t);       \
    template void launch_momentum_step<T, D>(const Dims&, const Metrics<T>&, const Metrics<D>&, \
                                             T, T*, T*, T*, const T*, const T*, const T*, T*,   \
                                             T*, T*, const T*, const T*, const T*, const D*,    \
                                             cudaStream_t);                                     \
    template void launch_adv_ref_state<T>(const Dims&, const Metrics<T>&, T, const T*,          \
                                          const T*, T*, const T*, int, cudaStream_t);           \
    template void launch_advance_scalar<T>(const Dims&, T, T*, const T*, cudaStream_t);         \
    template void launch_add_profile<T>(const Dims&, T*, const T*, T, cudaStream_t);

INST(double, double)
INST(float, double)

// ---- precision conversion of whole arrays ------------------------------------
template <typename TO, typename FROM>
__global__ void k_convert(size_t n, TO* __restrict__ to, const FROM* __restrict__ from) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e < n) to[e] = (TO)from[e];
}

template <typename TO, typename FROM>
void launch_convert(size_t n, TO* to, const FROM* from, cudaStream_t st) {
    if (!n) return;
    k_convert<TO, FROM><<<(unsigned)((n + 255) / 256), 256, 0, st>>>(n, to, from);
}
template void launch_convert<float, double>(size_t, float*, const double*, cudaStream_t);
template void launch_convert<double, float>(size_t, double*, const float*, cudaStream_t);

// dense host-layout columns (hd.K = kp+2 levels) -> pitched device columns
// (d.K levels), converting to TO: one warp per column, lanes along k
template <typename TO>
__global__ void __launch_bounds__(256) k_repitch(Dims hd, Dims d, TO* __restrict__ dst,
                                                 const double* __restrict__ src) {
    const int lane = threadIdx.x & 31;
    const size_t ncol = (size_t)hd.J * hd.I;
    const size_t w0 = (blockIdx.x * (size_t)blockDim.x + threadIdx.x) >> 5;
    const size_t nw = (gridDim.x * (size_t)blockDim.x) >> 5;
    for (size_t col = w0; col < ncol; col += nw) {
        const double* __restrict__ s = src + col * hd.K;
        TO* __restrict__ t = dst + col * d.K;
        for (int k = lane; k < hd.K; k += 32) t[k] = (TO)s[k];
    }
}
template <typename TO>
void launch_repitch(const Dims& hd, const Dims& d, TO* dst, const double* src, cudaStream_t st) {
    const size_t ncol = (size_t)hd.J * hd.I;
    const unsigned nb = (unsigned)std::min<size_t>((ncol + 7) / 8, 148 * 32);
    k_repitch<TO><<<nb, 256, 0, st>>>(hd, d, dst, src);
}
template void launch_repitch<double>(const Dims&, const Dims&, double*, const double*,
                                     cudaStream_t);
template void launch_repitch<float>(const Dims&, const Dims&, float*, const double*,
                                    cudaStream_t);

}  // namespace dcm
