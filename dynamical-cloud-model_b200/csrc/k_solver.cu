// k_solver.cu -- Jacobi-preconditioned BiCGSTAB for the anelastic pressure
// equation, dynamics.f90:293-444 (set_mat_a :34-175, mat_ax :187-229,
// precondition :241-270, inn_prod :458-482).
//
// The operator is the reference's 7-point metric stencil with constant
// coefficients taken from the 1-D grid spacings (a_e = 1/(dx(i-1)dxn(i)) ...,
// a_c = 0), periodic in x and y and mirrored (x(0)=x(1), x(kp+1)=x(kp)) in
// z.  Instead of materialising 8 coefficient arrays and exchanging halos
// before every matvec, each kernel reads the six per-axis coefficients from
// small 1-D tables and maps neighbour indices (wrap / mirror) directly.
//
// One BiCGSTAB iteration = 9 kernels in three dependent phases separated by
// the global dot products (39 field passes):
//   B1-B3  three Jacobi sweeps of precondition(s <- t), t = r - bet*(omg*v1)
//          formed on the fly; B3 also writes p = s + bet*p
//   B4     v1 = A p and (cr, v1)                 -> alf = rho / (cr,v1)
//   C1-C3  three Jacobi sweeps of precondition(cs <- s), s = r - alf*v1
//   C4     t = A cs, (t,t), (t,s)                -> omg = ts / tt
//   D      x += alf p + omg cs, r = s - omg t, (r,r), (r,cr) -> err, rho, bet
// Dot products are reduced deterministically (fixed block order) and the
// scalar recurrences run in the last block of each reducing kernel, so the
// host never waits inside an iteration.  Every kernel first checks the
// device-side `done` flag, which lets the host launch iterations in chunks.
#include "dcm_internal.h"
#include "dcm_prof.h"

namespace dcm {

// --- operator --------------------------------------------------------------
template <typename T>
struct Coef {
    const T *ae, *aw;  // per i
    const T *an, *as;  // per j
    const T *au, *ad;  // per k
};

template <typename T, typename F>
__device__ __forceinline__ T apply_A(const Dims& d, const Coef<T>& c, int k,
                                     int j, int i, T& ap, F&& X) {
    const int iw = i == 1 ? d.ip : i - 1, ie = i == d.ip ? 1 : i + 1;
    const int js = j == 1 ? d.jp : j - 1, jn = j == d.jp ? 1 : j + 1;
    const int kd = k == 1 ? 1 : k - 1, ku = k == d.kp ? d.kp : k + 1;
    const T ae = ld(c.ae + i), aw = ld(c.aw + i), an = ld(c.an + j),
            as = ld(c.as + j), au = ld(c.au + k), ad = ld(c.ad + k);
    // a_p exactly as set_mat_a forms it (dynamics.f90:93-95)
    ap = -ae - aw - an - as - au - ad;
    return aw * X(k, j, iw) + ae * X(k, j, ie) + as * X(k, js, i) +
           an * X(k, jn, i) + ad * X(kd, j, i) + au * X(ku, j, i) +
           ap * X(k, j, i) + T(0);
}

template <typename T>
__device__ __forceinline__ T diag_ap(const Coef<T>& c, int k, int j, int i) {
    return -ld(c.ae + i) - ld(c.aw + i) - ld(c.an + j) - ld(c.as + j) -
           ld(c.au + k) - ld(c.ad + k);
}

struct SolverArgs {
    Dims d;
    int itmax;
    double tol;
};

// --- setup: r = b - A x, cr = r, (b,b), (r,r) -------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_bicg_setup(SolverArgs a, Coef<T> c,
                                                    const T* __restrict__ x,
                                                    const T* __restrict__ b,
                                                    T* __restrict__ r,
                                                    T* __restrict__ cr,
                                                    double* partials,
                                                    unsigned int* ticket,
                                                    SolverScalars* S) {
    __shared__ double smem[64];
    const Dims& d = a.d;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    double v[2] = {0.0, 0.0};
    if (k <= d.kp && j <= d.jp) {
        T ap;
        const T ax = apply_A(d, c, k, j, i, ap,
                             [&](int kk, int jj, int ii) { return x[d.at(kk, jj, ii)]; });
        const int o = d.at(k, j, i);
        const T bv = b[o];
        const T rv = bv - ax;
        r[o] = rv;
        cr[o] = rv;
        v[0] = (double)bv * (double)bv;
        v[1] = (double)rv * (double)rv;
    }
    block_reduce<R_SUM, 2>(v, smem);
    const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    if (publish_partials<2>(v, partials, ticket, nb)) {
        double s[2];
        final_reduce<R_SUM, 2>(s, partials, ticket, nb, smem);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            double sc = sqrt(s[0]);
            sc = sc > 0.01 ? sc : 0.01;  // dynamics.f90:370-371
            const double err = sqrt(s[1]) / sc;
            S->sc_err = sc;
            S->err = err;
            S->it = 0;
            S->status = 0;
            S->early = 0;
            S->done = 0;
            if (err < a.tol) {  // :382-383 early return
                S->early = 1;
                S->done = 1;
            } else if (!(err == err)) {
                S->status = DCM_E_NONFINITE;
                S->done = 1;
            } else {
                S->alf = 1.0;  // :385-387
                S->omg = 1.0;
                S->nrm = 1.0;
                S->rho = s[1];  // (r,cr) with cr = r
                S->bet = (S->rho / S->nrm) * (S->alf / S->omg);
            }
        }
    }
}

// --- Jacobi sweeps -----------------------------------------------------------
// MODE 0: phase B (q = t = r - bet*(omg*v1), v1 = 0 on the first iteration)
// MODE 1: phase C (q = s = r - alf*v1)
template <typename T, int MODE>
__device__ __forceinline__ T qval(const T* __restrict__ r,
                                  const T* __restrict__ v1, int o, T bet,
                                  T omg, T alf, bool first) {
    if (MODE == 0) return first ? r[o] - bet * (omg * T(0)) : r[o] - bet * (omg * v1[o]);
    return r[o] - alf * v1[o];
}

// SWEEP 1: s_prev = q / a_p formed on the fly at the neighbours
// SWEEP 2,3: s_prev read from `sin`
// LASTP (phase B, sweep 3): out = p = s_new + bet * p_old (in place)
template <typename T, int MODE, int SWEEP, bool LASTP>
__global__ void __launch_bounds__(256) k_jacobi(SolverArgs a, Coef<T> c,
                                                const T* __restrict__ r,
                                                const T* __restrict__ v1,
                                                const T* __restrict__ sin,
                                                T* __restrict__ out,
                                                const SolverScalars* S) {
    if (S->done) return;
    const Dims& d = a.d;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const T bet = (T)S->bet, omg = (T)S->omg, alf = (T)S->alf;
    const bool first = S->it == 0;
    T ap;
    T As;
    if (SWEEP == 1) {
        As = apply_A(d, c, k, j, i, ap, [&](int kk, int jj, int ii) {
            const int o = d.at(kk, jj, ii);
            return qval<T, MODE>(r, v1, o, bet, omg, alf, first) / diag_ap(c, kk, jj, ii);
        });
    } else {
        As = apply_A(d, c, k, j, i, ap,
                     [&](int kk, int jj, int ii) { return sin[d.at(kk, jj, ii)]; });
    }
    const int o = d.at(k, j, i);
    const T q = qval<T, MODE>(r, v1, o, bet, omg, alf, first);
    const T sp = SWEEP == 1 ? q / ap : sin[o];
    const T sn = sp + (q - As) / ap;  // dynamics.f90:264
    if (LASTP) {
        out[o] = first ? sn + bet * T(0) : sn + bet * out[o];  // :397
    } else {
        out[o] = sn;
    }
}

// --- B4: v1 = A p, (cr, v1) -> alf -------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_bicg_matvec_p(SolverArgs a, Coef<T> c,
                                                       const T* __restrict__ p,
                                                       const T* __restrict__ cr,
                                                       T* __restrict__ v1,
                                                       double* partials,
                                                       unsigned int* ticket,
                                                       SolverScalars* S) {
    __shared__ double smem[32];
    if (S->done) return;
    const Dims& d = a.d;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    double v[1] = {0.0};
    if (k <= d.kp && j <= d.jp) {
        T ap;
        const T av = apply_A(d, c, k, j, i, ap,
                             [&](int kk, int jj, int ii) { return p[d.at(kk, jj, ii)]; });
        const int o = d.at(k, j, i);
        v1[o] = av;
        v[0] = (double)cr[o] * (double)av;
    }
    block_reduce<R_SUM, 1>(v, smem);
    const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    if (publish_partials<1>(v, partials, ticket, nb)) {
        double s[1];
        final_reduce<R_SUM, 1>(s, partials, ticket, nb, smem);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            S->nrm = s[0];               // :401
            S->alf = S->rho / S->nrm;    // :403
        }
    }
}

// --- C4: t = A cs, (t,t), (t,s) -> omg ----------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) k_bicg_matvec_cs(SolverArgs a, Coef<T> c,
                                                        const T* __restrict__ cs,
                                                        const T* __restrict__ r,
                                                        const T* __restrict__ v1,
                                                        T* __restrict__ t,
                                                        double* partials,
                                                        unsigned int* ticket,
                                                        SolverScalars* S) {
    __shared__ double smem[64];
    if (S->done) return;
    const Dims& d = a.d;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    const T alf = (T)S->alf;
    double v[2] = {0.0, 0.0};
    if (k <= d.kp && j <= d.jp) {
        T ap;
        const T tv = apply_A(d, c, k, j, i, ap,
                             [&](int kk, int jj, int ii) { return cs[d.at(kk, jj, ii)]; });
        const int o = d.at(k, j, i);
        t[o] = tv;
        const T sv = r[o] - alf * v1[o];  // s of :404
        v[0] = (double)tv * (double)tv;
        v[1] = (double)tv * (double)sv;
    }
    block_reduce<R_SUM, 2>(v, smem);
    const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    if (publish_partials<2>(v, partials, ticket, nb)) {
        double s[2];
        final_reduce<R_SUM, 2>(s, partials, ticket, nb, smem);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            S->tt = s[0];
            S->ts = s[1];
            S->omg = S->ts / S->tt;  // :412
            const double tiny = (double)1.e-16f;  // default-real literal, :321
            if (fabs(S->omg) < tiny) {  // :414-417
                S->status = DCM_E_BREAKDOWN;
                S->it = S->it + 1;
                S->done = 1;
            }
        }
    }
}

// --- D: x, r updates, (r,r), (r,cr) -> err, next rho and bet -----------------
template <typename T>
__global__ void __launch_bounds__(256) k_bicg_update(SolverArgs a,
                                                     T* __restrict__ x,
                                                     const T* __restrict__ p,
                                                     const T* __restrict__ cs,
                                                     T* __restrict__ r,
                                                     const T* __restrict__ v1,
                                                     const T* __restrict__ t,
                                                     const T* __restrict__ cr,
                                                     double* partials,
                                                     unsigned int* ticket,
                                                     SolverScalars* S) {
    __shared__ double smem[64];
    if (S->done) return;
    const Dims& d = a.d;
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    const T alf = (T)S->alf, omg = (T)S->omg;
    double v[2] = {0.0, 0.0};
    if (k <= d.kp && j <= d.jp) {
        const int o = d.at(k, j, i);
        const T sv = r[o] - alf * v1[o];
        x[o] = x[o] + alf * p[o] + omg * cs[o];  // :419
        const T rn = sv - omg * t[o];             // :420
        r[o] = rn;
        v[0] = (double)rn * (double)rn;
        v[1] = (double)rn * (double)cr[o];
    }
    block_reduce<R_SUM, 2>(v, smem);
    const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    if (publish_partials<2>(v, partials, ticket, nb)) {
        double s[2];
        final_reduce<R_SUM, 2>(s, partials, ticket, nb, smem);
        if (threadIdx.x == 0 && threadIdx.y == 0) {
            const int it = S->it + 1;
            S->it = it;
            const double err = sqrt(s[0]) / S->sc_err;  // :423
            S->err = err;
            S->nrm = S->rho;  // :425
            if (err < a.tol) {  // :428
                S->done = 1;
            } else if (!(err == err)) {
                S->status = DCM_E_NONFINITE;
                S->done = 1;
            } else if (it >= a.itmax) {
                S->status = DCM_E_NOCONV;  // :431-434
                S->done = 1;
            } else {
                S->rho = s[1];  // (r,cr) of the next iteration, :391
                S->bet = (S->rho / S->nrm) * (S->alf / S->omg);  // :392
            }
        }
    }
}

// --- after the solve: halo fix-up of x (dynamics.f90:437-442) and, when
//     `wo` is set, the driver's exchange_along_dim_wo(p) (driver_code.f90:506)
template <typename T>
__global__ void __launch_bounds__(256) k_bicg_post(Dims d, T* __restrict__ x,
                                                   const T* __restrict__ sw,
                                                   const T* __restrict__ dzn,
                                                   const SolverScalars* S,
                                                   int wo) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const int o = d.at(k, j, i);
    const T v = x[o];
    if (wo) put_wo(x, d, k, j, i, v);
    if (S->status != 0) return;
    if (S->early) {
        // the early return (:383) leaves the rows set by mat_ax's
        // exchange_along_dim + Neumann copy (:203-211)
        if (k == 1) put_plane_images(x, d, 0, j, i, v);
        if (k == d.kp) put_plane_images(x, d, d.kp + 1, j, i, v);
        return;
    }
    if (k == d.kp) {
        int js[3], is[3];
        const int nj = images(j, d.jp, js), ni = images(i, d.ip, is);
        for (int b3 = 0; b3 < nj; b3++)
            for (int c3 = 0; c3 < ni; c3++) x[d.at(d.kp + 1, js[b3], is[c3])] = v;
    }
    if (k == 1) {
        int js[3], is[3];
        const int nj = images(j, d.jp, js), ni = images(i, d.ip, is);
        const T dz0 = ld(dzn);
        for (int b3 = 0; b3 < nj; b3++)
            for (int c3 = 0; c3 < ni; c3++) {
                const int jj = js[b3], ii = is[c3];
                x[d.at(0, jj, ii)] = v - sw[d.at(0, jj, ii)] * dz0;
            }
    }
}

// --- host orchestration --------------------------------------------------------
template <typename T>
static Coef<T> coef_of(const SolverWork<T>& w) {
    Coef<T> c;
    c.ae = w.ae; c.aw = w.aw; c.an = w.an; c.as = w.as; c.au = w.au; c.ad = w.ad;
    return c;
}

template <typename T>
static void launch_iteration(const SolverArgs& a, const Coef<T>& c,
                             SolverWork<T>& w, T* x, cudaStream_t st) {
    const dim3 g = interior_grid(a.d, a.d.kp), b(BX, BY);
    // phase B
    { ProfScope ps(P_JACOBI, st);
      k_jacobi<T, 0, 1, false><<<g, b, 0, st>>>(a, c, w.r, w.v1, nullptr, w.sA, w.S); }
    { ProfScope ps(P_JACOBI, st);
      k_jacobi<T, 0, 2, false><<<g, b, 0, st>>>(a, c, w.r, w.v1, w.sA, w.sB, w.S); }
    { ProfScope ps(P_JACOBI, st);
      k_jacobi<T, 0, 3, true><<<g, b, 0, st>>>(a, c, w.r, w.v1, w.sB, w.p, w.S); }
    { ProfScope ps(P_MATVEC, st);
      k_bicg_matvec_p<T><<<g, b, 0, st>>>(a, c, w.p, w.cr, w.v1, w.partials, w.ticket, w.S); }
    // phase C
    { ProfScope ps(P_JACOBI, st);
      k_jacobi<T, 1, 1, false><<<g, b, 0, st>>>(a, c, w.r, w.v1, nullptr, w.sA, w.S); }
    { ProfScope ps(P_JACOBI, st);
      k_jacobi<T, 1, 2, false><<<g, b, 0, st>>>(a, c, w.r, w.v1, w.sA, w.sB, w.S); }
    { ProfScope ps(P_JACOBI, st);
      k_jacobi<T, 1, 3, false><<<g, b, 0, st>>>(a, c, w.r, w.v1, w.sB, w.sA, w.S); }
    { ProfScope ps(P_MATVEC, st);
      k_bicg_matvec_cs<T><<<g, b, 0, st>>>(a, c, w.sA, w.r, w.v1, w.t, w.partials, w.ticket,
                                           w.S); }
    // phase D
    { ProfScope ps(P_UPDATE, st);
      k_bicg_update<T><<<g, b, 0, st>>>(a, x, w.p, w.sA, w.r, w.v1, w.t, w.cr, w.partials,
                                        w.ticket, w.S); }
}

template <typename T>
int solver_run(SolverWork<T>& w, const Dims& d, T* x, const T* b, const T* sw,
               const T* dzn, double tol, int itmax, int wo, int chunk,
               cudaStream_t st, SolverScalars* host_S, int* launched_iters) {
    SolverArgs a;
    a.d = d;
    a.itmax = itmax;
    a.tol = tol;
    const Coef<T> c = coef_of(w);
    const dim3 g = interior_grid(d, d.kp), bl(BX, BY);
    { ProfScope ps(P_SETUP, st);
      k_bicg_setup<T><<<g, bl, 0, st>>>(a, c, x, b, w.r, w.cr, w.partials, w.ticket, w.S); }
    if (cudaGetLastError() != cudaSuccess) return DCM_E_CUDA;
    int launched = 0;
    for (;;) {
        cudaMemcpyAsync(host_S, w.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return DCM_E_CUDA;
        if (host_S->done) break;
        if (launched >= itmax) break;
        for (int q = 0; q < chunk && launched < itmax; q++, launched++)
            launch_iteration<T>(a, c, w, x, st);
        if (cudaGetLastError() != cudaSuccess) return DCM_E_CUDA;
    }
    { ProfScope ps(P_POST, st);
      k_bicg_post<T><<<g, bl, 0, st>>>(d, x, sw, dzn, w.S, wo); }
    cudaMemcpyAsync(host_S, w.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return DCM_E_CUDA;
    if (launched_iters) *launched_iters = launched;
    return host_S->status;
}

template int solver_run<double>(SolverWork<double>&, const Dims&, double*, const double*,
                                const double*, const double*, double, int, int, int,
                                cudaStream_t, SolverScalars*, int*);

}  // namespace dcm
