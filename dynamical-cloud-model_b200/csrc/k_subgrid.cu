// k_subgrid.cu -- the Smagorinsky subgrid model of sources with
// viscous = .true. (dynamics.f90:878-893 -> sgm/subgrid_3d.f90:38-493):
// strain rate, Richardson-number functions, eddy viscosities with the
// Monin-Obukhov surface layer, the six stresses, and the stress / diffusion
// source terms of u, v, w, theta and the q fields.
//
// Four kernels, one thread per interior cell (threadIdx.x -> 32 consecutive
// k-levels of one column, so every field access of a warp is one coalesced
// column segment; the +-1 neighbours in j and i come from L1 / L2):
//   k_sgs_visc    strain, vism, vist (+ the surface row k = 0) and the
//                 exchange_full_wo images of vism / vist      (:91-180)
//   k_sgs_tau     the six stresses with their exchange_along_dim images
//                 (:191-237)
//   k_sgs_mom     su, sv, sw += stress divergence (:240-284)
//   k_sgs_scalar  sth and every sq += diffusion (:289-345), th and the q
//                 fields in one pass so that vist's stencil is loaded once
// In FP64 these kernels are bound by the latency of the IEEE divisions that
// parity with the reference keeps (about 30 per cell in k_sgs_visc), not by
// HBM.  The stresses therefore go through six arrays, as in the reference:
// evaluating each once and re-reading it costs 12 field passes of HBM,
// re-evaluating the 15 that a cell's momentum sources name costs about twice
// the divisions.
// The image writers are those of dcm_common.cuh; in the time step the
// momentum kernel also applies the surface / lid rows of sources
// (dynamics.f90:922-973), as k_sources does in the inviscid step.
#include "dcm_internal.h"
#include "dcm_prof.h"

namespace dcm {

namespace {

// module parameters, sgm/subgrid_3d.f90:13-16
struct SgsConst {
    static constexpr double prn = 0.95, subb = 40.0, subc = 16.0, subg = 1.2, subh = 0.0,
                            subr = 4.0, ric = 0.25, grav = 9.81, small = 1.e-10, kvon = 0.4;
};

__device__ __forceinline__ double sg_sqrt(double x) { return sqrt(x); }
__device__ __forceinline__ float sg_sqrt(float x) { return sqrtf(x); }
__device__ __forceinline__ double sg_pow(double x, double y) { return pow(x, y); }
__device__ __forceinline__ float sg_pow(float x, float y) { return powf(x, y); }

template <typename T>
__device__ __forceinline__ T sq2(T x) { return x * x; }

// The stresses at interior cell (k, j, i), sgm/subgrid_3d.f90:194-220.
template <typename T>
struct Stress {
    Dims d;
    Metrics<T> mt;
    const T* __restrict__ vm;
    const T* __restrict__ zu;
    const T* __restrict__ zv;
    const T* __restrict__ zw;
    __device__ __forceinline__ T V(int k, int j, int i) const { return vm[d.at(k, j, i)]; }
    __device__ __forceinline__ T t11(int k, int j, int i) const {
        return ld(mt.rhoan + k) * T(1) * (V(k, j, i) + V(k - 1, j, i)) *
               (zu[d.at(k, j, i)] - zu[d.at(k, j, i - 1)]) / ld(mt.dx + i - 1);
    }
    __device__ __forceinline__ T t22(int k, int j, int i) const {
        return ld(mt.rhoan + k) * T(1) * (V(k, j, i) + V(k - 1, j, i)) *
               (zv[d.at(k, j, i)] - zv[d.at(k, j - 1, i)]) / ld(mt.dy + j - 1);
    }
    __device__ __forceinline__ T t33(int k, int j, int i) const {
        return ld(mt.rhoan + k) * T(1) * (V(k, j, i) + V(k - 1, j, i)) *
               (zw[d.at(k, j, i)] - zw[d.at(k - 1, j, i)]) / ld(mt.dz + k - 1);
    }
    __device__ __forceinline__ T t12(int k, int j, int i) const {
        return ld(mt.rhoan + k) * T(0.125) *
               (V(k, j, i) + V(k, j + 1, i) + V(k - 1, j, i) + V(k - 1, j + 1, i) +
                V(k, j, i + 1) + V(k, j + 1, i + 1) + V(k - 1, j, i + 1) +
                V(k - 1, j + 1, i + 1)) *
               ((zu[d.at(k, j + 1, i)] - zu[d.at(k, j, i)]) / ld(mt.dyn + j) +
                (zv[d.at(k, j, i + 1)] - zv[d.at(k, j, i)]) / ld(mt.dxn + i));
    }
    __device__ __forceinline__ T t13(int k, int j, int i) const {
        return ld(mt.rhoa + k) * T(0.5) * (V(k, j, i) + V(k, j, i + 1)) *
               ((zu[d.at(k + 1, j, i)] - zu[d.at(k, j, i)]) / ld(mt.dzn + k) +
                (zw[d.at(k, j, i + 1)] - zw[d.at(k, j, i)]) / ld(mt.dxn + i));
    }
    __device__ __forceinline__ T t23(int k, int j, int i) const {
        return ld(mt.rhoa + k) * T(0.5) * (V(k, j, i) + V(k, j + 1, i)) *
               ((zw[d.at(k, j + 1, i)] - zw[d.at(k, j, i)]) / ld(mt.dyn + j) +
                (zv[d.at(k + 1, j, i)] - zv[d.at(k, j, i)]) / ld(mt.dzn + k));
    }
};

}  // namespace

// ---- strain, Richardson functions, viscosities, surface layer -------------
template <typename T>
__global__ void __launch_bounds__(256, 4) k_sgs_visc(Dims d, Metrics<T> mt, SgsParams<T> P,
                                                  const T* __restrict__ u,
                                                  const T* __restrict__ v,
                                                  const T* __restrict__ w,
                                                  const T* __restrict__ th, T* __restrict__ vism,
                                                  T* __restrict__ vist,
                                                  T* __restrict__ strain) {
    using C = SgsConst;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    auto U = [&](int kk, int jj, int ii) { return u[d.at(kk, jj, ii)]; };
    auto Vv = [&](int kk, int jj, int ii) { return v[d.at(kk, jj, ii)]; };
    auto W = [&](int kk, int jj, int ii) { return w[d.at(kk, jj, ii)]; };
    const T dxm = ld(mt.dx + i - 1), dym = ld(mt.dy + j - 1), dz = ld(mt.dz + k),
            dzm = ld(mt.dz + k - 1), dzn = ld(mt.dzn + k), dxn = ld(mt.dxn + i),
            dxnm = ld(mt.dxn + i - 1), dyn = ld(mt.dyn + j), dynm = ld(mt.dyn + j - 1);
    // :96-131, statement by statement
    T s = sq2((U(k + 1, j, i) - U(k + 1, j, i - 1)) / dxm) + sq2((U(k, j, i) - U(k, j, i - 1)) / dxm);
    s = s + sq2((Vv(k + 1, j, i) - Vv(k + 1, j - 1, i)) / dym) +
        sq2((Vv(k, j, i) - Vv(k, j - 1, i)) / dym);
    s = s + sq2((W(k, j, i) - W(k - 1, j, i)) / dzm) + sq2((W(k + 1, j, i) - W(k, j, i)) / dz);
    s = s + T(0.5) * (sq2((U(k + 1, j, i) - U(k, j, i)) / dzn + (W(k, j, i + 1) - W(k, j, i)) / dxn) +
                      sq2((U(k + 1, j, i - 1) - U(k, j, i - 1)) / dz +
                          (W(k, j, i) - W(k, j, i - 1)) / dxnm));
    s = s + T(0.5) * (sq2((W(k, j, i) - W(k, j - 1, i)) / dynm +
                          (Vv(k + 1, j - 1, i) - Vv(k, j - 1, i)) / dzn) +
                      sq2((W(k, j + 1, i) - W(k, j, i)) / dyn + (Vv(k + 1, j, i) - Vv(k, j, i)) / dzn));
    {
        // the eight s12 terms; the sixth repeats the second, as the reference does (:128)
        const T f2 = sq2((U(k, j + 1, i - 1) - U(k, j, i - 1)) / dyn +
                         (Vv(k, j, i) - Vv(k, j, i - 1)) / dxnm);
        T a = sq2((U(k, j, i - 1) - U(k, j - 1, i - 1)) / dynm +
                  (Vv(k, j - 1, i) - Vv(k, j - 1, i - 1)) / dxnm);
        a = a + f2;
        a = a + sq2((U(k, j, i) - U(k, j - 1, i)) / dynm + (Vv(k, j - 1, i + 1) - Vv(k, j - 1, i)) / dxn);
        a = a + sq2((U(k, j + 1, i) - U(k, j, i)) / dyn + (Vv(k, j, i + 1) - Vv(k, j, i)) / dxn);
        a = a + sq2((U(k + 1, j, i - 1) - U(k + 1, j - 1, i - 1)) / dynm +
                    (Vv(k + 1, j - 1, i) - Vv(k + 1, j - 1, i - 1)) / dxnm);
        a = a + f2;
        a = a + sq2((U(k + 1, j, i) - U(k + 1, j - 1, i)) / dynm +
                    (Vv(k + 1, j - 1, i + 1) - Vv(k + 1, j - 1, i)) / dxn);
        a = a + sq2((U(k + 1, j + 1, i) - U(k + 1, j, i)) / dyn +
                    (Vv(k + 1, j, i + 1) - Vv(k + 1, j, i)) / dxn);
        s = s + T(0.125) * a;
    }
    const int o = d.at(k, j, i);
    strain[o] = s;
    // richardson, :469-489 (1.e-15 is a single-precision literal there)
    const T rip = T(C::grav) * ((th[d.at(k + 1, j, i)]) / ld(mt.thetan + k + 1) -
                                (th[o]) / ld(mt.thetan + k)) /
                  dzn / (s + T((double)1.e-15f));
    T fm, fh;
    const T suba = T(1.0 / C::prn);
    if (rip < T(0)) {
        fm = sg_sqrt(T(1) - T(C::subc) * rip);
        fh = suba * sg_sqrt(T(1) - T(C::subb) * rip);
    } else if ((rip >= T(0)) && (rip < T(C::ric))) {
        const T pr = sg_pow(T(1) - rip / T(C::ric), T(C::subr));
        fm = pr * (T(1) - T(C::subh) * rip);
        fh = suba * pr * (T(1) - T(C::subg) * rip);
    } else {
        fm = T(0);
        fh = T(0);
    }
    // :146, :157; the lid rows kp-1, kp are zero (:164-165)
    T vm = ld(P.lamsq + k) * sg_sqrt(s) * fm;
    T vt = ld(P.lamsq + k) * sg_sqrt(s) * fh * ld(mt.rhoa + k);
    if (k >= d.kp - 1) {
        vm = T(0);
        vt = T(0);
    }
    put_full<T, true>(vism, d, k, j, i, vm, T(0), T(0));
    put_full<T, true>(vist, d, k, j, i, vt, T(0), T(0));
    if (k == 1) {
        // monin_obukhov, :397-426: the surface row k = 0 of this column, in
        // FP64 for both field precisions: over a calm first level (vmag = the
        // 1e-10 guard) the bulk Richardson number reaches 1e19 and
        // (1 + 4.7 rib)**2 would overflow FP32 (then ustar = 0 and
        // thstar = x / 0 turn the row into NaN); one thread per column
        using C64 = SgsConst;
        const double kv = C64::kvon, kv2 = kv * kv;
        const double z1 = P.z1, z0 = P.z0, z0th = P.z0th;
        const double u1 = (double)U(1, j, i) + (double)U(1, j, i - 1);
        const double v1 = (double)Vv(1, j, i) + (double)Vv(1, j - 1, i);
        const double vmag = 0.5 * sqrt(u1 * u1 + v1 * v1) + C64::small;
        const double theta0 = (double)ld(mt.theta + 0);
        const double dth = (double)th[d.at(1, j, i)] + (double)ld(mt.thetan + 1) - theta0;
        const double rib = C64::grav * dth * sq2(z1 - z0) / (theta0 * sq2(vmag) * (z1 - z0th));
        const double lg = log(z1 / z0);
        double gm, gh;
        if (rib <= 0.0) {
            gm = 1.0 - 9.4 * rib / (1.0 + 70.0 * kv2 * sqrt(fabs(rib * z1 / z0)) / sq2(lg));
            gh = 1.0 - 9.4 * rib / (1.0 + 50.0 * kv2 * sqrt(fabs(rib * z1 / z0)) / sq2(lg));
        } else {
            gm = 1.0 / sq2(1.0 + 4.7 * rib);
            gh = 1.0 / sq2(1.0 + 4.7 * rib);
        }
        const double ustar = kv * vmag / lg * sqrt(gm);
        const double thstar = kv2 * vmag * dth / (ustar * C64::prn * sq2(lg)) * gh;
        vism[d.at(0, j, i)] = (T)(sq2(ustar) * (z1 - z0) / vmag);
        vist[d.at(0, j, i)] = (T)(ustar * thstar / (dth / (z1 - z0th) + C64::small));
    }
}

// ---- the six stresses with their exchange_along_dim(0, 0) images ----------
template <typename T>
__global__ void __launch_bounds__(256) k_sgs_tau(Dims d, Metrics<T> mt, const T* __restrict__ vism,
                                                 const T* __restrict__ zu,
                                                 const T* __restrict__ zv,
                                                 const T* __restrict__ zw, T* __restrict__ t11,
                                                 T* __restrict__ t22, T* __restrict__ t33,
                                                 T* __restrict__ t12, T* __restrict__ t13,
                                                 T* __restrict__ t23) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const Stress<T> S{d, mt, vism, zu, zv, zw};
    const T z = T(0);
    put_dim(t11, d, k, j, i, S.t11(k, j, i), z, z);
    put_dim(t22, d, k, j, i, S.t22(k, j, i), z, z);
    put_dim(t33, d, k, j, i, S.t33(k, j, i), z, z);
    put_dim(t12, d, k, j, i, S.t12(k, j, i), z, z);
    put_dim(t13, d, k, j, i, S.t13(k, j, i), z, z);
    put_dim(t23, d, k, j, i, S.t23(k, j, i), z, z);
}

// ---- su, sv, sw += divergence of the stresses -----------------------------
// The stresses come from k_sgs_tau's arrays, halo faces included (the images
// of exchange_along_dim).  ROWS = false: the exchange_full(0, 0) images of
// su, sv, sw (:279-284).  ROWS = true: those images followed by the surface /
// lid rows of sources (dynamics.f90:922-973): levels 0 = -(level 1) for su,
// sv and 0 for sw, levels kp, kp+1 = 0.
template <typename T, bool ROWS>
__global__ void __launch_bounds__(256) k_sgs_mom(Dims d, Metrics<T> mt, const T* __restrict__ t11,
                                                 const T* __restrict__ t22,
                                                 const T* __restrict__ t33,
                                                 const T* __restrict__ t12,
                                                 const T* __restrict__ t13,
                                                 const T* __restrict__ t23, T* __restrict__ su,
                                                 T* __restrict__ sv, T* __restrict__ sw) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const int o = d.at(k, j, i);
    const T z = T(0);
    if (ROWS && k == d.kp) {
        put_plane_images(su, d, d.kp, j, i, z);
        put_plane_images(su, d, d.kp + 1, j, i, z);
        put_plane_images(sv, d, d.kp, j, i, z);
        put_plane_images(sv, d, d.kp + 1, j, i, z);
        put_plane_images(sw, d, d.kp, j, i, z);
        put_plane_images(sw, d, d.kp + 1, j, i, z);
        return;
    }
    T vsu = su[o], vsv = sv[o], vsw = sw[o];
    const T dxm = ld(mt.dx + i - 1), dym = ld(mt.dy + j - 1);
    if (k <= d.kp - 1) {  // :256-261
        const T c13 = t13[o], c23 = t23[o];
        vsw = vsw + ((t33[d.at(k + 1, j, i)] - t33[o]) / ld(mt.dzn + k) +
                     (c13 - t13[d.at(k, j, i - 1)]) / dxm + (c23 - t23[d.at(k, j - 1, i)]) / dym);
        if (k >= 2) {  // :262-274
            const T c12 = t12[o];
            const T dzm = ld(mt.dz + k - 1);
            vsu = vsu + ((t11[d.at(k, j, i + 1)] - t11[o]) / ld(mt.dxn + i) +
                         (c12 - t12[d.at(k, j - 1, i)]) / dym + (c13 - t13[d.at(k - 1, j, i)]) / dzm);
            vsv = vsv + ((t22[d.at(k, j + 1, i)] - t22[o]) / ld(mt.dyn + j) +
                         (c12 - t12[d.at(k, j, i - 1)]) / dxm + (c23 - t23[d.at(k - 1, j, i)]) / dzm);
        }
    }
    if (ROWS) {
        put_plane_images(su, d, k, j, i, vsu);
        put_plane_images(sv, d, k, j, i, vsv);
        put_plane_images(sw, d, k, j, i, vsw);
        if (k == 1) {
            put_plane_images(su, d, 0, j, i, -vsu);
            put_plane_images(sv, d, 0, j, i, -vsv);
            put_plane_images(sw, d, 0, j, i, z);
        }
    } else {
        put_full(su, d, k, j, i, vsu, z, z);
        put_full(sv, d, k, j, i, vsv, z, z);
        put_full(sw, d, k, j, i, vsw, z, z);
    }
}

// ---- sth, sq += diffusion (vist carries rhoa), exchange_full(0, 0) --------
template <typename T>
__global__ void __launch_bounds__(256, 4) k_sgs_scalar(Dims d, Metrics<T> mt,
                                                    const T* __restrict__ vist, ScalarSet<T> set) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    auto Vt = [&](int kk, int jj, int ii) { return vist[d.at(kk, jj, ii)]; };
    const T c0 = Vt(k, j, i), cm = Vt(k - 1, j, i);
    // the four-point sums of :293-306, in the reference's order
    const T axm = c0 + Vt(k, j, i - 1) + cm + Vt(k - 1, j, i - 1);
    const T axp = Vt(k, j, i + 1) + c0 + Vt(k - 1, j, i + 1) + cm;
    const T aym = c0 + Vt(k, j - 1, i) + cm + Vt(k - 1, j - 1, i);
    const T ayp = Vt(k, j + 1, i) + c0 + Vt(k - 1, j + 1, i) + cm;
    const T dxm = ld(mt.dx + i - 1), dxnm = ld(mt.dxn + i - 1), dxn = ld(mt.dxn + i);
    const T dym = ld(mt.dy + j - 1), dynm = ld(mt.dyn + j - 1), dyn = ld(mt.dyn + j);
    const T dzm = ld(mt.dz + k - 1), dz = ld(mt.dz + k), rn = ld(mt.rhoan + k);
    const int o = d.at(k, j, i);
    for (int m = 0; m < set.n; m++) {
        const T* __restrict__ s = set.s[m];
        T* __restrict__ ds = set.ds[m];
        const T sc = s[o];
        const T term =
            (T(0.25) * (axm * (s[d.at(k, j, i - 1)] - sc) / dxnm - axp * (sc - s[d.at(k, j, i + 1)]) / dxn) /
                 dxm +
             T(0.25) * (aym * (s[d.at(k, j - 1, i)] - sc) / dynm - ayp * (sc - s[d.at(k, j + 1, i)]) / dyn) /
                 dym +
             (cm * (s[d.at(k - 1, j, i)] - sc) / dzm - c0 * (sc - s[d.at(k + 1, j, i)]) / dz) / dzm) /
            rn;
        const T base = ((set.reset >> m) & 1u) ? T(0) : ds[o];
        put_full(ds, d, k, j, i, base + term, T(0), T(0));
    }
}

// ---- launchers ---------------------------------------------------------------
template <typename T>
void launch_subgrid(const Dims& d, const Metrics<T>& mt, const SgsParams<T>& P, const T* u,
                    const T* v, const T* w, const T* zu, const T* zv, const T* zw, const T* th,
                    T* vism, T* vist, T* strain, T* const* tau, T* su, T* sv, T* sw,
                    const ScalarSet<T>* sets, int nsets, bool rows, cudaStream_t st) {
    const dim3 b(BX, BY), g = interior_grid(d, d.kp);
    ProfScope ps_(P_SOURCES, st);
    k_sgs_visc<T><<<g, b, 0, st>>>(d, mt, P, u, v, w, th, vism, vist, strain);
    k_sgs_tau<T><<<g, b, 0, st>>>(d, mt, vism, zu, zv, zw, tau[0], tau[1], tau[2], tau[3],
                                  tau[4], tau[5]);
    if (rows)
        k_sgs_mom<T, true><<<g, b, 0, st>>>(d, mt, tau[0], tau[1], tau[2], tau[3], tau[4],
                                            tau[5], su, sv, sw);
    else
        k_sgs_mom<T, false><<<g, b, 0, st>>>(d, mt, tau[0], tau[1], tau[2], tau[3], tau[4],
                                             tau[5], su, sv, sw);
    for (int c = 0; c < nsets; c++) k_sgs_scalar<T><<<g, b, 0, st>>>(d, mt, vist, sets[c]);
}

template <typename T>
void launch_subgrid_scalars(const Dims& d, const Metrics<T>& mt, const T* vist,
                            const ScalarSet<T>* sets, int nsets, cudaStream_t st) {
    const dim3 b(BX, BY), g = interior_grid(d, d.kp);
    ProfScope ps_(P_SOURCES, st);
    for (int c = 0; c < nsets; c++) k_sgs_scalar<T><<<g, b, 0, st>>>(d, mt, vist, sets[c]);
}

template <typename T>
int make_scalar_sets(const T* th, T* sth, int sth_reset, T* const* q, T* const* sq, int nq,
                     int sq_reset, ScalarSet<T>* sets, int max_sets) {
    int ns = 0, m = 0;
    auto add = [&](const T* s, T* ds, int reset) {
        if (ns == 0 || sets[ns - 1].n == SGS_MAXS) {
            if (ns == max_sets) return false;
            sets[ns] = ScalarSet<T>{};
            ns++;
        }
        ScalarSet<T>& c = sets[ns - 1];
        c.s[c.n] = s;
        c.ds[c.n] = ds;
        if (reset) c.reset |= 1u << c.n;
        c.n++;
        return true;
    };
    if (th && !add(th, sth, sth_reset)) return -1;
    for (m = 0; m < nq; m++)
        if (!add(q[m], sq[m], sq_reset)) return -1;
    return ns;
}

#define DCM_SGS_INST(T)                                                                           \
    template void launch_subgrid<T>(const Dims&, const Metrics<T>&, const SgsParams<T>&,         \
                                    const T*, const T*, const T*, const T*, const T*, const T*,  \
                                    const T*, T*, T*, T*, T* const*, T*, T*, T*,                  \
                                    const ScalarSet<T>*, int, bool, cudaStream_t);                \
    template void launch_subgrid_scalars<T>(const Dims&, const Metrics<T>&, const T*,           \
                                            const ScalarSet<T>*, int, cudaStream_t);              \
    template int make_scalar_sets<T>(const T*, T*, int, T* const*, T* const*, int, int,          \
                                     ScalarSet<T>*, int);
DCM_SGS_INST(double)
DCM_SGS_INST(float)
#undef DCM_SGS_INST

}  // namespace dcm
