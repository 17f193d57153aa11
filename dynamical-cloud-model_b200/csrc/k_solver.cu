// k_solver.cu -- Jacobi-preconditioned BiCGSTAB for the anelastic pressure
// equation, dynamics.f90:293-444 (set_mat_a :34-175, mat_ax :187-229,
// precondition :241-270, inn_prod :458-482).
//
// The operator is the reference's 7-point metric stencil with constant
// coefficients taken from the 1-D grid spacings (a_e = 1/(dx(i-1)dxn(i)) ...,
// a_c = 0), periodic in x and y and mirrored (x(0)=x(1), x(kp+1)=x(kp)) in
// z.  Instead of materialising 8 coefficient arrays and exchanging halos
// before every matvec, the kernels read six per-axis coefficient tables and
// map neighbour indices (wrap / mirror) directly.
//
// Kernels take one interior point per thread (a warp = 32 consecutive
// k-levels of one column) at full occupancy; k neighbours come from adjacent
// lanes by warp shuffle.  Dot products are reduced per block, then per group
// of 64 blocks and finally across groups, each level in a fixed order (two
// tickets, see reduce2), so the sums are deterministic and the atomics are
// spread over many addresses.
//
// One BiCGSTAB iteration = 9 kernels in three dependent phases separated by
// the global dot products:
//   B1-B3  three Jacobi sweeps of precondition(s <- t), t = r - bet*(omg*v1)
//          formed on the fly; B3 also writes p = s + bet*p
//   B4     v1 = A p and (cr, v1)                 -> alf = rho / (cr,v1)
//   C1-C3  three Jacobi sweeps of precondition(cs <- s), s = r - alf*v1
//   C4     t = A cs, (t,t), (t,s)                -> omg = ts / tt
//   D      x += alf p + omg cs, r = s - omg t, (r,r), (r,cr) -> err, rho, bet
// The scalar recurrences run in the last block of each reducing kernel, so
// the host never waits inside an iteration; every kernel first checks the
// device-side `done` flag, which lets the host launch iterations in chunks.
//
// Preconditioner arithmetic: the reference forms s0 = q/a_p and sweeps
// s <- s + (q - A s)/a_p (dynamics.f90:260-264).  Here the kernels that
// produce r and v1 also store r/a_p and v1/a_p, so q/a_p is an axpy of those
// and no sweep divides neighbour values; each sweep divides its own A s by
// a_p once.  The result agrees with the reference's order of operations to a
// few ulp per sweep, far below the 1e-10 parity bar.  The iteration then
// moves 41 field passes instead of 39.
#include "dcm_internal.h"
#include "dcm_prof.h"

namespace dcm {

template <typename T>
struct Coef {
    const T *ae, *aw;  // per i
    const T *an, *as;  // per j
    const T *au, *ad;  // per k
};

struct SolverArgs {
    Dims d;
    int itmax;
    double tol;
    int ich;       // i-planes per tile
    int nkt, njt;  // tiles in k, j
    int ntiles;
};

// a_p exactly as set_mat_a forms it (dynamics.f90:93-95)
template <typename T>
__device__ __forceinline__ T diag_ap(const Coef<T>& c, int k, int j, int i) {
    return -ld(c.ae + i) - ld(c.aw + i) - ld(c.an + j) - ld(c.as + j) - ld(c.au + k) -
           ld(c.ad + k);
}

// operator kinds of the stencil marcher
enum SOp {
    OP_SETUP = 0,  // X = x:   r = b - A x, cr = r, rh = r/a_p, dots (b,b), (r,r)
    OP_SW1,        // X = s0 = q/a_p from rh, vh: out = s1
    OP_SW,         // X = s_prev: out = s_next
    OP_SW3P,       // X = s_prev: p = s3 + bet p (in place)
    OP_MATP,       // X = p:   v1 = A p, vh = v1/a_p, dot (cr, v1)
    OP_MATC        // X = cs:  t = A cs, dots (t,t), (t,s)
};

struct SolverBufs {
    const void *x, *b, *r, *v1, *rh, *vh, *sin, *cr;
    void *out, *out2, *out3;
};

// q / a_p of the preconditioner input, formed from rh = r/a_p and vh = v1/a_p:
// MODE 0: t = r - bet*(omg*v1) (dynamics.f90:393); MODE 1: s = r - alf*v1 (:404)
template <typename T, int MODE>
__device__ __forceinline__ T s0val(const T* __restrict__ rh, const T* __restrict__ vh, int o,
                                   T bet, T omg, T alf, bool first) {
    if (MODE == 0) return first ? rh[o] - bet * (omg * T(0)) : rh[o] - bet * (omg * vh[o]);
    return rh[o] - alf * vh[o];
}

// 7-point stencil kernel, one interior point per thread: threadIdx.x -> k
// (one warp = 32 consecutive levels of a column), threadIdx.y -> j,
// blockIdx.z -> i.  k neighbours come from the adjacent lanes by shuffle
// (Neumann mirror at k = 1 and kp, dynamics.f90:206-211), j and i
// neighbours (periodic) through L1/L2.
template <typename T, int OP, int MODE>
struct StenCtx {
    Dims d;
    Coef<T> c;
    const T* gx;
    const T* rh;
    const T* vh;
    SolverBufs B;
    T bet, omg, alf;
    bool first;
};

// one warp task: 32 consecutive k-levels (k0 = 1 + 32 kt) of column (j, i)
template <typename T, int OP, int MODE, int NV>
__device__ __forceinline__ void sten_task(const StenCtx<T, OP, MODE>& C, int kt, int j, int i,
                                          double (&acc)[NV]) {
    const Dims& d = C.d;
    const int lane = threadIdx.x & 31;
    const int ip = d.ip, jp = d.jp, kp = d.kp;
    const int k = 1 + kt * BX + lane;
    const bool valid = k <= kp;
    auto X = [&](int kk, int jj, int ii) -> T {
        const int o = d.at(kk, jj, ii);
        if (OP == OP_SW1) return s0val<T, MODE>(C.rh, C.vh, o, C.bet, C.omg, C.alf, C.first);
        return C.gx[o];
    };
    const int km = min(k, kp);
    const T xc = X(km, j, i);
    T xd = __shfl_up_sync(0xffffffffu, xc, 1);
    T xu = __shfl_down_sync(0xffffffffu, xc, 1);
    if (lane == 0) xd = X(max(km - 1, 1), j, i);
    if (lane == BX - 1) xu = X(min(km + 1, kp), j, i);
    if (!valid) return;
    const Coef<T>& c = C.c;
    const T xm = X(k, j, i == 1 ? ip : i - 1), xp = X(k, j, i == ip ? 1 : i + 1);
    const T xs = X(k, j == 1 ? jp : j - 1, i), xn = X(k, j == jp ? 1 : j + 1, i);
    const T ae = ld(c.ae + i), aw = ld(c.aw + i), an = ld(c.an + j), as = ld(c.as + j),
            au = ld(c.au + k), ad = ld(c.ad + k);
    const T ap = -ae - aw - an - as - au - ad;
    // mat_ax, dynamics.f90:219-222 (a_c = 0)
    const T Ax = aw * xm + ae * xp + as * xs + an * xn + ad * xd + au * xu + ap * xc + T(0);
    const int o = d.at(k, j, i);
    const SolverBufs& B = C.B;
    T* __restrict__ out = (T*)B.out;
    if (OP == OP_SETUP) {
        const T bv = ((const T*)B.b)[o];
        const T rv = bv - Ax;  // :377
        out[o] = rv;
        ((T*)B.out2)[o] = rv;
        ((T*)B.out3)[o] = rv / ap;
        acc[0] += (double)bv * (double)bv;
        acc[NV - 1] += (double)rv * (double)rv;
    } else if (OP == OP_MATP) {
        out[o] = Ax;
        ((T*)B.out3)[o] = Ax / ap;
        acc[0] += (double)((const T*)B.cr)[o] * (double)Ax;
    } else if (OP == OP_MATC) {
        out[o] = Ax;
        const T sv = ((const T*)B.r)[o] - C.alf * ((const T*)B.v1)[o];  // s of :404
        acc[0] += (double)Ax * (double)Ax;
        acc[NV - 1] += (double)Ax * (double)sv;
    } else {
        // precondition, dynamics.f90:260-264:
        //   s_new = s + (q - A s)/a_p = s + q/a_p - (A s)/a_p
        const T s0c =
            OP == OP_SW1 ? xc : s0val<T, MODE>(C.rh, C.vh, o, C.bet, C.omg, C.alf, C.first);
        const T sn = xc + s0c - Ax / ap;
        if (OP == OP_SW3P)
            out[o] = C.first ? sn + C.bet * T(0) : sn + C.bet * out[o];  // :397
        else
            out[o] = sn;
    }
}

// Sweeps (no reduction): one warp task per warp, grid (k-chunks, j/8, i).
// Reducing kernels: persistent blocks, each warp strides over the warp tasks
// and the block publishes one partial.
template <typename T, int OP, int MODE>
__global__ void __launch_bounds__(256) k_sten(SolverArgs a, Coef<T> c, SolverBufs B, Red2 R,
                                              SolverScalars* S) {
    constexpr int NV = (OP == OP_SETUP || OP == OP_MATC) ? 2 : 1;
    constexpr bool RED = OP == OP_SETUP || OP == OP_MATC || OP == OP_MATP;
    __shared__ double smem[64];
    if (OP != OP_SETUP && S->done) return;
    StenCtx<T, OP, MODE> C;
    C.d = a.d;
    C.c = c;
    C.gx = (const T*)(OP == OP_SETUP ? B.x : B.sin);
    C.rh = (const T*)B.rh;
    C.vh = (const T*)B.vh;
    C.B = B;
    C.bet = (T)S->bet;
    C.omg = (T)S->omg;
    C.alf = (T)S->alf;
    C.first = S->it == 0;
    const Dims& d = a.d;
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) acc[q] = 0.0;
    if (!RED) {
        const int j = 1 + blockIdx.y * BY + threadIdx.y;
        if (j <= d.jp) sten_task<T, OP, MODE, NV>(C, blockIdx.x, j, 1 + blockIdx.z, acc);
        return;
    }
    const int nkt = a.nkt;
    const long long ntask = (long long)nkt * d.jp * d.ip;
    const int warps = blockDim.y;
    for (long long t = (long long)blockIdx.x * warps + threadIdx.y; t < ntask;
         t += (long long)gridDim.x * warps) {
        const int kt = (int)(t % nkt);
        const long long r2 = t / nkt;
        const int j = 1 + (int)(r2 % d.jp);
        const int i = 1 + (int)(r2 / d.jp);
        sten_task<T, OP, MODE, NV>(C, kt, j, i, acc);
    }
    block_reduce<R_SUM, NV>(acc, smem);
    double s[NV];
    if (reduce2<NV>(acc, R, smem, s) && threadIdx.x == 0 && threadIdx.y == 0) {
        if (OP == OP_SETUP) {
            double sc = sqrt(s[0]);
            sc = sc > 0.01 ? sc : 0.01;  // dynamics.f90:370-371
            const double err = sqrt(s[NV - 1]) / sc;
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
                S->rho = s[NV - 1];  // (r,cr) with cr = r
                S->bet = (S->rho / S->nrm) * (S->alf / S->omg);
            }
        } else if (OP == OP_MATP) {
            S->nrm = s[0];             // :401
            S->alf = S->rho / S->nrm;  // :403
        } else if (OP == OP_MATC) {
            S->tt = s[0];
            S->ts = s[NV - 1];
            S->omg = S->ts / S->tt;               // :412
            const double tiny = (double)1.e-16f;  // default-real literal, :321
            if (fabs(S->omg) < tiny) {            // :414-417
                S->status = DCM_E_BREAKDOWN;
                S->it = S->it + 1;
                S->done = 1;
            }
        }
    }
}

// --- D: x, r updates, (r,r), (r,cr) -> err, next rho and bet -----------------
template <typename T>
__global__ void __launch_bounds__(256) k_bicg_update(SolverArgs a, Coef<T> c,
                                                     T* __restrict__ x,
                                                     const T* __restrict__ p,
                                                     const T* __restrict__ cs,
                                                     T* __restrict__ r,
                                                     const T* __restrict__ v1,
                                                     const T* __restrict__ t,
                                                     const T* __restrict__ cr,
                                                     T* __restrict__ rh, Red2 R,
                                                     SolverScalars* S) {
    __shared__ double smem[64];
    if (S->done) return;
    const Dims& d = a.d;
    const T alf = (T)S->alf, omg = (T)S->omg;
    double acc[2] = {0.0, 0.0};
    const int nkt = a.nkt;
    const long long ntask = (long long)nkt * d.jp * d.ip;
    const int warps = blockDim.y;
    for (long long tk = (long long)blockIdx.x * warps + threadIdx.y; tk < ntask;
         tk += (long long)gridDim.x * warps) {
        const int kt = (int)(tk % nkt);
        const long long r2 = tk / nkt;
        const int j = 1 + (int)(r2 % d.jp);
        const int i = 1 + (int)(r2 / d.jp);
        const int k = 1 + kt * BX + threadIdx.x;
        if (k > d.kp) continue;
        const int o = d.at(k, j, i);
        const T sv = r[o] - alf * v1[o];
        x[o] = x[o] + alf * p[o] + omg * cs[o];  // :419
        const T rn = sv - omg * t[o];             // :420
        r[o] = rn;
        rh[o] = rn / diag_ap(c, k, j, i);
        acc[0] += (double)rn * (double)rn;
        acc[1] += (double)rn * (double)cr[o];
    }
    block_reduce<R_SUM, 2>(acc, smem);
    double s[2];
    if (reduce2<2>(acc, R, smem, s) && threadIdx.x == 0 && threadIdx.y == 0) {
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

// --- after the solve: halo rows of x (dynamics.f90:437-442 or, after the
//     early return, mat_ax's rows :203-211) and the driver's
//     exchange_along_dim_wo(p) (driver_code.f90:506)
template <typename T>
__global__ void __launch_bounds__(256) k_bicg_post(Dims d, T* __restrict__ x,
                                                   const T* __restrict__ sw,
                                                   const T* __restrict__ dzn,
                                                   const SolverScalars* S, int wo) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const int o = d.at(k, j, i);
    const T v = x[o];
    if (wo) put_wo(x, d, k, j, i, v);
    if (S->status != 0) return;
    if (S->early) {
        if (k == 1) put_plane_images(x, d, 0, j, i, v);
        if (k == d.kp) put_plane_images(x, d, d.kp + 1, j, i, v);
        return;
    }
    if (k == d.kp) put_plane_images(x, d, d.kp + 1, j, i, v);
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

static int sm_count() {
    static int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    }
    return sms;
}

// resident blocks of a persistent reducing kernel
template <typename K>
static int persistent_grid(K kernel) {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, BX * BY, 0);
    return sm_count() * (per > 0 ? per : 1);
}

template <typename T, int OP, int MODE>
static void sten(const SolverArgs& a, const Coef<T>& c, const SolverBufs& B, SolverWork<T>& w,
                 cudaStream_t st, int cat) {
    ProfScope ps(cat, st);
    constexpr bool RED = OP == OP_SETUP || OP == OP_MATC || OP == OP_MATP;
    if (RED) {
        static int g = 0;
        if (!g) g = persistent_grid(k_sten<T, OP, MODE>);
        k_sten<T, OP, MODE><<<g, dim3(BX, BY), 0, st>>>(a, c, B, w.red, w.S);
    } else {
        k_sten<T, OP, MODE><<<interior_grid(a.d, a.d.kp), dim3(BX, BY), 0, st>>>(a, c, B, w.red,
                                                                                   w.S);
    }
}

template <typename T>
static void launch_iteration(const SolverArgs& a, const Coef<T>& c, SolverWork<T>& w, T* x,
                             cudaStream_t st) {
    SolverBufs B{};
    B.r = w.r;
    B.v1 = w.v1;
    B.rh = w.rh;
    B.vh = w.vh;
    // phase B: precondition(s <- t), p = s + bet p, v1 = A p
    B.out = w.sA;
    sten<T, OP_SW1, 0>(a, c, B, w, st, P_JACOBI);
    B.sin = w.sA;
    B.out = w.sB;
    sten<T, OP_SW, 0>(a, c, B, w, st, P_JACOBI);
    B.sin = w.sB;
    B.out = w.p;
    sten<T, OP_SW3P, 0>(a, c, B, w, st, P_JACOBI);
    B.sin = w.p;
    B.cr = w.cr;
    B.out = w.v1;
    B.out3 = w.vh;
    sten<T, OP_MATP, 0>(a, c, B, w, st, P_MATVEC);
    // phase C: precondition(cs <- s), t = A cs
    B.sin = nullptr;
    B.out = w.sA;
    sten<T, OP_SW1, 1>(a, c, B, w, st, P_JACOBI);
    B.sin = w.sA;
    B.out = w.sB;
    sten<T, OP_SW, 1>(a, c, B, w, st, P_JACOBI);
    B.sin = w.sB;
    B.out = w.sA;
    sten<T, OP_SW, 1>(a, c, B, w, st, P_JACOBI);
    B.sin = w.sA;
    B.out = w.t;
    sten<T, OP_MATC, 1>(a, c, B, w, st, P_MATVEC);
    // phase D
    {
        ProfScope ps(P_UPDATE, st);
        static int g = 0;
        if (!g) g = persistent_grid(k_bicg_update<T>);
        k_bicg_update<T><<<g, dim3(BX, BY), 0, st>>>(a, c, x, w.p, w.sA, w.r, w.v1, w.t, w.cr,
                                                     w.rh, w.red, w.S);
    }
}

int solver_ich = 16;  // i-planes per tile

template <typename T>
int solver_run(SolverWork<T>& w, const Dims& d, T* x, const T* b, const T* sw, const T* dzn,
               double tol, int itmax, int wo, int chunk, cudaStream_t st, SolverScalars* host_S,
               int* launched_iters) {
    SolverArgs a;
    a.d = d;
    a.itmax = itmax;
    a.tol = tol;
    a.ich = solver_ich;
    a.nkt = (d.kp + BX - 1) / BX;
    a.njt = (d.jp + BY - 1) / BY;
    a.ntiles = a.nkt * a.njt * ((d.ip + a.ich - 1) / a.ich);
    const Coef<T> c = coef_of(w);
    SolverBufs B{};
    B.x = x;
    B.b = b;
    B.out = w.r;
    B.out2 = w.cr;
    B.out3 = w.rh;
    sten<T, OP_SETUP, 0>(a, c, B, w, st, P_SETUP);
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
    {
        ProfScope ps(P_POST, st);
        k_bicg_post<T><<<interior_grid(d, d.kp), dim3(BX, BY), 0, st>>>(d, x, sw, dzn, w.S, wo);
    }
    cudaMemcpyAsync(host_S, w.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return DCM_E_CUDA;
    if (launched_iters) *launched_iters = launched;
    return host_S->status;
}

template int solver_run<double>(SolverWork<double>&, const Dims&, double*, const double*,
                                const double*, const double*, double, int, int, int,
                                cudaStream_t, SolverScalars*, int*);

}  // namespace dcm
