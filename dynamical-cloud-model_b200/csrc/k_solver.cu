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
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <mutex>
#include <type_traits>

#include <cooperative_groups.h>

#include "dcm_internal.h"
#include "dcm_prof.h"

namespace dcm {

// Programmatic dependent launch.  Inside a graph-driven iteration every
// kernel but the first is launched with programmatic stream serialisation,
// so it is launched while its predecessor finishes instead of after it.
// pdl_wait holds the kernel until the predecessor has completed and its
// writes are visible (for a kernel launched without the attribute nothing
// is in flight and it returns at once); pdl_launch then lets the next kernel
// be launched.  No kernel reads anything before pdl_wait.
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;" ::: "memory"); }
__device__ __forceinline__ void pdl_launch() {
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

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
    double sc_floor;  // max(||b||, sc_floor) scales the residual (0.01, :371)
    int nkt;          // k-chunks of a warp task
    int max_updates;  // mixed form: reliable updates before DCM_E_NOCONV
    int max_cycle;    // mixed form: FP32 iterations between updates before a restart
    int by;           // warps per block of the non-reducing sweeps
    int tasks;        // warp tasks per warp of the reducing kernels (0: fill the GPU)
    int max_blocks;   // blocks a reducing kernel may use (partials capacity)
    int ni;           // i-planes a stencil warp task marches over
    int fuse;         // FP32: the three sweeps of a phase as one kernel (k_precond3)
    int fuse_mv = 0;  // with fuse: phase C's matvec as the fused kernel's fourth stage
    int vw = 0;       // FP32 levels per lane of the separate kernels (2 or 4; 0 = 4)
    // Chebyshev-weighted sweeps (mixed form only): x1 = cw[0] s0, then
    // x_m+1 = x_m + cw[m] (s0 - (A x_m)/a_p), m = 1..3, in place of the
    // reference's x1 = s0, x_m+1 = x_m + s0 - (A x_m)/a_p
    int cheb;
    double cw[4];
    // graph-driven loops: the update kernel sets the condition of the WHILE
    // node around the iteration (cond) itself, bounded by cond_max
    // iterations; cond_max = 0 outside a graph loop
    cudaGraphConditionalHandle cond = 0;
    int cond_max = 0;
    // launch with programmatic stream serialisation (pdl_wait)
    int pdl = 0;
    // |omega| below this ends an FP64 solve with DCM_E_BREAKDOWN; the
    // reference's tiny is the default-real literal 1.e-16 (dynamics.f90:321)
    double tiny = (double)1.e-16f;
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
    int sweep;  // 1..3: which Jacobi sweep of the preconditioner a launch is
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
// (A x)/a_p of a Jacobi sweep.  FP32 (the mixed form's preconditioner):
// the two-instruction approximate divide (within 2 ulp, as the full-range
// sequence that -prec-div=false gives, for |a_p| in [2^-126, 2^126], which
// any grid spacing between 1e-19 m and 1e19 m keeps); FP64: the correctly
// rounded divide of the reference's arithmetic.
__device__ __forceinline__ float sweep_div(float a, float b) { return __fdividef(a, b); }
__device__ __forceinline__ double sweep_div(double a, double b) { return a / b; }

// One Chebyshev-weighted sweep at a point, every rounding of the update
// explicit (the fused and the separate sweeps differ only in how the
// compiler contracts the operator's products):
//     res = sc x + w (s0 - sc (A x)/a_p),   q = (A x)/a_p
// sc = w1 on the first sweep (its operand is w1 s0, applied here by
// linearity instead of to the seven operand values), 1 on the others.
__device__ __forceinline__ float cheb_update(float xc, float s0, float q, float sc, float w) {
    return __fmaf_rn(w, __fsub_rn(s0, __fmul_rn(q, sc)), __fmul_rn(xc, sc));
}
// the same with sc = 1 (every sweep but the first): the two products by 1
// are exact, so this is bit for bit cheb_update(xc, s0, q, 1, w)
__device__ __forceinline__ float cheb_update1(float xc, float s0, float q, float w) {
    return __fmaf_rn(w, __fsub_rn(s0, q), xc);
}
__device__ __forceinline__ double cheb_update(double xc, double s0, double q, double sc,
                                              double w) {
    return __fma_rn(w, __dsub_rn(s0, __dmul_rn(q, sc)), __dmul_rn(xc, sc));
}

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
    bool cheb;  // weighted sweeps (cheb_update)
    T wx;       // first sweep: the scale w1 of its operand s0 (1 otherwise)
    T ws;       // this sweep's weight
};

// Ask L2 for the line holding p ahead of its use (no register is written).
__device__ __forceinline__ void prefetch_l2(const void* p) {
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// Warp-task iterator of the persistent kernels: task t = kt + nkt*(jr +
// njr*(i-1)), visited at start, start+stride, ...; the stride is split into
// its (kt, jr, i) parts once so that each step is a carry chain, not a divide.
struct TaskIter {
    int kt, jr, i;
    int dkt, djr, di, nkt, njr;
    __device__ __forceinline__ TaskIter(unsigned start, unsigned stride, int nkt_, int njr_)
        : nkt(nkt_), njr(njr_) {
        kt = (int)(start % (unsigned)nkt);
        const unsigned q = start / (unsigned)nkt;
        jr = (int)(q % (unsigned)njr);
        i = 1 + (int)(q / (unsigned)njr);
        dkt = (int)(stride % (unsigned)nkt);
        const unsigned sq = stride / (unsigned)nkt;
        djr = (int)(sq % (unsigned)njr);
        di = (int)(sq / (unsigned)njr);
    }
    __device__ __forceinline__ void next() {
        kt += dkt;
        const int c1 = kt >= nkt;
        kt -= c1 ? nkt : 0;
        jr += djr + c1;
        const int c2 = jr >= njr;
        jr -= c2 ? njr : 0;
        i += di + c2;
    }
};

// 16-byte vectors of consecutive k-levels: the pitched layout puts k = 1 of
// every column on a 32-byte boundary, so the vector starting at
// k0 = 1 + V m is aligned.
template <typename T>
struct KVec;
template <>
struct KVec<float> {
    static constexpr int V = 4;
    using type = float4;
};
template <>
struct KVec<double> {
    static constexpr int V = 2;
    using type = double2;
};

// the vector type of N consecutive k-levels (16 or 8 bytes)
template <typename T, int N>
struct VecT;
template <>
struct VecT<float, 4> {
    using type = float4;
};
template <>
struct VecT<float, 2> {
    using type = float2;
};
template <>
struct VecT<double, 2> {
    using type = double2;
};

template <typename VT, typename T, int N>
__device__ __forceinline__ void vunpack(const VT& a, T (&v)[N]) {
    if constexpr (N == 4) {
        v[0] = a.x; v[1] = a.y; v[2] = a.z; v[3] = a.w;
    } else {
        v[0] = a.x; v[1] = a.y;
    }
}

template <typename T, int N>
__device__ __forceinline__ void vld(const T* p, T (&v)[N]) {
    using VT = typename VecT<T, N>::type;
    vunpack(__ldg(reinterpret_cast<const VT*>(p)), v);
}
// coherent load, for an array the kernel also writes
template <typename T, int N>
__device__ __forceinline__ void vld_rw(const T* p, T (&v)[N]) {
    using VT = typename VecT<T, N>::type;
    vunpack(*reinterpret_cast<const VT*>(p), v);
}
// store the levels k0 + c <= kp (a whole vector when all are)
template <typename T, int N>
__device__ __forceinline__ void vst(T* p, const T (&v)[N], int nvalid) {
    using VT = typename VecT<T, N>::type;
    if (nvalid >= N) {
        VT a;
        if constexpr (N == 4) {
            a.x = v[0]; a.y = v[1]; a.z = v[2]; a.w = v[3];
        } else {
            a.x = v[0]; a.y = v[1];
        }
        *reinterpret_cast<VT*>(p) = a;
    } else {
#pragma unroll
        for (int c = 0; c < N; c++)
            if (c < nvalid) p[c] = v[c];
    }
}

// X values of a vector: the operand field, or for the first sweep s0 = q/a_p
// formed from rh and vh
template <typename T, int OP, int MODE, int V>
__device__ __forceinline__ void xload(const StenCtx<T, OP, MODE>& C, int o, T (&x)[V]) {
    if (OP == OP_SW1) {
        T a[V], b[V];
        vld(C.rh + o, a);
        if (MODE == 0 && C.first) {
#pragma unroll
            for (int c = 0; c < V; c++) x[c] = a[c] - C.bet * (C.omg * T(0));
            return;
        }
        vld(C.vh + o, b);
#pragma unroll
        for (int c = 0; c < V; c++)
            x[c] = MODE == 0 ? a[c] - C.bet * (C.omg * b[c]) : a[c] - C.alf * b[c];
    } else {
        vld(C.gx + o, x);
    }
}
template <typename T, int OP, int MODE>
__device__ __forceinline__ T xload1(const StenCtx<T, OP, MODE>& C, int o) {
    if (OP == OP_SW1) return s0val<T, MODE>(C.rh, C.vh, o, C.bet, C.omg, C.alf, C.first);
    return C.gx[o];
}

// One warp task: V x 32 consecutive k-levels (lane l holds k0 = 1 +
// V (32 kc + l) .. k0 + V - 1) of row j, marching over the planes
// i0 .. i0 + ni - 1.  k neighbours are the adjacent vector elements, the
// neighbour lanes' end elements by shuffle, and at the warp's two ends one
// scalar load each; Neumann mirror at k = 1, kp (dynamics.f90:206-211).  j
// neighbours (periodic) are vector loads of the adjacent columns; the i
// neighbours are the previous and the next plane of the march, kept in
// registers, so each plane loads its i + 1 column and its two j neighbours.
template <typename T, int OP, int MODE, int NV, bool MARCH, int V>
__device__ __forceinline__ void sten_task(const StenCtx<T, OP, MODE>& C, int kc, int j, int i0,
                                          int ni, double (&acc)[NV]) {
    if (!MARCH) ni = 1;
    // V: levels per lane (16-byte vectors by default; 8-byte in FP32 for short columns)
    const Dims& d = C.d;
    const int lane = threadIdx.x & 31;
    const int ip = d.ip, jp = d.jp, kp = d.kp;
    const int k0 = 1 + V * (kc * BX + lane);
    const bool live = k0 <= kp;
    const int nvalid = live ? min(V, kp - k0 + 1) : 0;
    const int K = d.K, KJ = d.K * d.J;
    const int col = (live ? k0 : 1) + K * j;  // idle lanes read the column start
    const int dsj = (j == 1 ? jp - 1 : -1) * K, dnj = (j == jp ? 1 - jp : 1) * K;
    const Coef<T>& c = C.c;
    T au[V], ad[V];
    vld(c.au + (live ? k0 : 1), au);
    vld(c.ad + (live ? k0 : 1), ad);
    const T an = ld(c.an + j), as = ld(c.as + j);
    const int iend = MARCH ? min(i0 + ni - 1, ip) : i0;
    T xw[V], xc[V], xe[V];
    xload(C, col + KJ * (i0 == 1 ? ip : i0 - 1), xw);
    xload(C, col + KJ * i0, xc);
    for (int i = i0; i <= iend; i++) {
    const int o = col + KJ * i;
    T xs[V], xn[V];
    xload(C, col + KJ * (i == ip ? 1 : i + 1), xe);
    xload(C, o + dsj, xs);
    xload(C, o + dnj, xn);
    T prev = __shfl_up_sync(0xffffffffu, xc[V - 1], 1);
    T next = __shfl_down_sync(0xffffffffu, xc[0], 1);
    if (lane == 0 && live && k0 > 1) prev = xload1(C, o - 1);
    if (lane == BX - 1 && live && k0 + V <= kp) next = xload1(C, o + V);
    const T ae = ld(c.ae + i), aw = ld(c.aw + i);
    const T sij = -ae - aw - an - as;
    T ap[V], Ax[V];
#pragma unroll
    for (int q = 0; q < V; q++) {
        const int kk = k0 + q;
        T xd = q == 0 ? prev : xc[q - 1];
        T xu = q == V - 1 ? next : xc[q + 1];
        xd = kk == 1 ? xc[q] : xd;
        xu = kk == kp ? xc[q] : xu;
        ap[q] = sij - au[q] - ad[q];  // a_p, dynamics.f90:93-95 (same order)
        if constexpr (std::is_same<T, double>::value) {
            // mat_ax, dynamics.f90:219-222 (a_c = 0), in the reference's form
            Ax[q] = aw * xw[q] + ae * xe[q] + as * xs[q] + an * xn[q] + ad[q] * xd +
                    au[q] * xu + ap[q] * xc[q] + T(0);
        } else {
            // FP32 (mixed form): the same operator as differences to the
            // centre.  a_p rounded in FP32 no longer cancels its neighbours
            // exactly, which would give the singular (Neumann / periodic)
            // operator a spurious eigenvalue ~1e-7 a_p along the constants;
            // the Krylov recursion then stalls and drifts in p's constant.
            // In difference form constants are an exact null vector.
            const T c0 = xc[q];
            Ax[q] = aw * (xw[q] - c0) + ae * (xe[q] - c0) + as * (xs[q] - c0) +
                    an * (xn[q] - c0) + ad[q] * (xd - c0) + au[q] * (xu - c0);
        }
    }
    const SolverBufs& B = C.B;
    T* __restrict__ out = (T*)B.out;
    T res[V];
    if (OP == OP_SETUP) {
        T bv[V], res3[V];
        vld((const T*)B.b + o, bv);
#pragma unroll
        for (int q = 0; q < V; q++) {
            res[q] = bv[q] - Ax[q];  // :377
            res3[q] = res[q] / ap[q];
            if (q < nvalid) {
                acc[0] += (double)bv[q] * (double)bv[q];
                acc[NV - 1] += (double)res[q] * (double)res[q];
            }
        }
        vst(out + o, res, nvalid);
        vst((T*)B.out2 + o, res, nvalid);
        vst((T*)B.out3 + o, res3, nvalid);
    } else if (OP == OP_MATP) {
        T cr[V], res3[V];
        vld((const T*)B.cr + o, cr);
#pragma unroll
        for (int q = 0; q < V; q++) {
            res3[q] = Ax[q] / ap[q];
            if (q < nvalid) acc[0] += (double)cr[q] * (double)Ax[q];
        }
        vst(out + o, Ax, nvalid);
        vst((T*)B.out3 + o, res3, nvalid);
    } else if (OP == OP_MATC) {
        T r[V], v1[V];
        vld((const T*)B.r + o, r);
        vld((const T*)B.v1 + o, v1);
#pragma unroll
        for (int q = 0; q < V; q++) {
            const T sv = r[q] - C.alf * v1[q];  // s of :404
            if (q < nvalid) {
                acc[0] += (double)Ax[q] * (double)Ax[q];
                acc[NV - 1] += (double)Ax[q] * (double)sv;
            }
        }
        vst(out + o, Ax, nvalid);
    } else {
        // precondition, dynamics.f90:260-264:
        //   s_new = s + (q - A s)/a_p = s + q/a_p - (A s)/a_p
        T s0[V];
        if (OP == OP_SW1) {
#pragma unroll
            for (int q = 0; q < V; q++) s0[q] = xc[q];
        } else {
            StenCtx<T, OP_SW1, MODE> C1;
            C1.rh = C.rh; C1.vh = C.vh; C1.bet = C.bet; C1.omg = C.omg; C1.alf = C.alf;
            C1.first = C.first;
            xload(C1, o, s0);
        }
        if (C.cheb) {
#pragma unroll
            for (int q = 0; q < V; q++)
                res[q] = cheb_update(xc[q], s0[q], sweep_div(Ax[q], ap[q]), C.wx, C.ws);
        } else {
#pragma unroll
            for (int q = 0; q < V; q++) res[q] = xc[q] + s0[q] - sweep_div(Ax[q], ap[q]);
        }
        if (OP == OP_SW3P) {
            T pold[V];
            if (C.first) {
#pragma unroll
                for (int q = 0; q < V; q++) res[q] = res[q] + C.bet * T(0);  // :397
            } else {
                vld_rw(out + o, pold);
#pragma unroll
                for (int q = 0; q < V; q++) res[q] = res[q] + C.bet * pold[q];
            }
        }
        if (live) vst(out + o, res, nvalid);
    }
#pragma unroll
    for (int q = 0; q < V; q++) {
        xw[q] = xc[q];
        xc[q] = xe[q];
    }
    }
}

// block and grid reduction of a reducing stencil kernel, then the scalar
// recurrences in the last block
template <int OP, int NV>
__device__ __forceinline__ void reduce_tail(const SolverArgs& a, double (&acc)[NV], const Red2& R,
                                            double* smem, SolverScalars* S) {
    block_reduce<R_SUM, NV>(acc, smem);
    double s[NV];
    if (reduce2<NV>(acc, R, smem, s) && threadIdx.x == 0 && threadIdx.y == 0) {
        if (OP == OP_SETUP) {
            double sc = sqrt(s[0]);
            sc = sc > a.sc_floor ? sc : a.sc_floor;  // dynamics.f90:370-371
            const double err = sc > 0.0 ? sqrt(s[NV - 1]) / sc : 0.0;
            S->sc_err = sc;
            S->err = err;
            S->it = 0;
            S->status = 0;
            S->early = 0;
            S->done = 0;
            S->rounds = 0;
            S->cycles = 0;
            S->ru_runs = 0;
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
            if (S->ru && !(isfinite(S->alf) && S->nrm != 0.0)) {
                S->restart = isfinite(s[0]) ? 1 : 2;  // FP32 breakdown: restart
                S->pause = 1;
            }
        } else if (OP == OP_MATC) {
            S->tt = s[0];
            S->ts = s[NV - 1];
            S->omg = S->ts / S->tt;               // :412
            const double tiny = a.tiny;  // default-real literal 1.e-16, :321
            if (S->ru && !(fabs(S->omg) >= tiny)) {
                S->restart = (isfinite(s[0]) && isfinite(s[NV - 1])) ? 1 : 2;
                S->pause = 1;
            } else if (fabs(S->omg) < tiny) {     // :414-417
                S->status = DCM_E_BREAKDOWN;
                S->it = S->it + 1;
                S->done = 1;
            }
        }
    }
}

// Sweeps (no reduction): one warp task per warp, grid (k-chunks, j/8, i).
// Reducing kernels: persistent blocks, each warp strides over the warp tasks
// and the block publishes one partial.
template <typename T, int OP, int MODE, int V = KVec<T>::V, bool RM = false>
__global__ void __launch_bounds__(256) k_sten(SolverArgs a, Coef<T> c, SolverBufs B, Red2 R,
                                              SolverScalars* S) {
    constexpr int NV = (OP == OP_SETUP || OP == OP_MATC) ? 2 : 1;
    constexpr bool RED = OP == OP_SETUP || OP == OP_MATC || OP == OP_MATP;
    __shared__ double smem[64];
    pdl_wait();
    pdl_launch();
    if (OP != OP_SETUP && (S->done || S->pause)) return;
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
    C.first = S->it == 0 || S->fresh;
    C.cheb = a.cheb != 0;
    C.wx = (OP == OP_SW1 && a.cheb) ? (T)a.cw[0] : T(1);
    // (selected, not indexed: a run-time index would copy a.cw to the stack)
    C.ws = !a.cheb ? T(1) : (T)(B.sweep == 3 ? a.cw[3] : B.sweep == 2 ? a.cw[2] : a.cw[1]);
    const Dims& d = a.d;
    double acc[NV];
#pragma unroll
    for (int q = 0; q < NV; q++) acc[q] = 0.0;
    // only the first sweep marches: it rebuilds s0 from r/a_p and v1/a_p at
    // every neighbour, and the march reuses the i-1 and i+1 values; for the
    // other kernels the extra registers cost more occupancy than they save
    constexpr bool MARCH = OP == OP_SW1;
    const int ni = MARCH ? a.ni : 1;
    if constexpr (!RED) {
        const int j = 1 + blockIdx.y * blockDim.y + threadIdx.y;
        if (j <= d.jp)
            sten_task<T, OP, MODE, NV, MARCH, V>(C, blockIdx.x, j, 1 + blockIdx.z * ni, ni, acc);
    } else {
        const int lane = threadIdx.x & 31;
        // RM: a warp task is a column chunk over `rn` consecutive i-planes
        // (the march depth of the launch shape): the march keeps the i-1 and
        // i columns in registers, so each plane loads its i+1 column and its
        // two j neighbours (a variant of its own: the march's registers would
        // cost the unmarched kernel occupancy)
        const int rn = RM && a.ni > 1 ? a.ni : 1;
        const int nch = (d.ip + rn - 1) / rn;
        for (TaskIter t(blockIdx.x * blockDim.y + threadIdx.y, gridDim.x * blockDim.y, a.nkt,
                        d.jp);
             t.i <= nch; t.next()) {
            // the next task's streamed columns into L2 while this one runs:
            // a warp's tasks are otherwise serialised by their stores
            TaskIter u = t;
            u.next();
            if (u.i <= nch) {
                const int k0 = min(1 + V * (u.kt * BX + lane), d.kp);
                const int o = d.at(k0, 1 + u.jr, 1 + (u.i - 1) * rn);
                prefetch_l2(C.gx + o);
                if (OP == OP_SETUP) prefetch_l2((const T*)B.b + o);
                if (OP == OP_MATP) prefetch_l2((const T*)B.cr + o);
                if (OP == OP_MATC) {
                    prefetch_l2((const T*)B.r + o);
                    prefetch_l2((const T*)B.v1 + o);
                }
            }
            if constexpr (RM)
                sten_task<T, OP, MODE, NV, true, V>(C, t.kt, 1 + t.jr, 1 + (t.i - 1) * rn, rn,
                                                    acc);
            else
                sten_task<T, OP, MODE, NV, false, V>(C, t.kt, 1 + t.jr, t.i, 1, acc);
        }
        reduce_tail<OP, NV>(a, acc, R, smem, S);
    }
}

// --- fused preconditioner: the three Jacobi sweeps of one phase in one kernel
// (FP32, columns of at most 128 levels: one warp holds a whole column).
//
// precondition() (dynamics.f90:241-270) with s0 = q/a_p:
//     s1 = s0 + s0 - (A s0)/a_p,  s2 = s1 + s0 - (A s1)/a_p,  s3 = s2 + s0 - (A s2)/a_p
// A block owns PJ output rows j0 .. j0+PJ-1 of an i-chunk and keeps PJ + 6
// warps, one per row j0-3 .. j0+PJ+2.  The warps march over the planes with
// the stages skewed by one plane: at step b, stage 0 forms s0 at plane b+3
// (from r/a_p and v1/a_p in HBM), stage 1 sweeps plane b+2, stage 2 plane b+1
// and stage 3 plane b, which it writes out.  A warp's own i-1, i, i+1 values
// of each stage stay in registers (rings shifted every step); its j-1, j+1
// values come from the neighbouring warps' previous-step results in shared
// memory (double-buffered, one barrier per step); k neighbours are vector
// elements and shuffles.  Edge warps compute only the stages their neighbours
// need (a shrinking halo of 3, 2, 1 rows).  Each output point sees exactly the
// arithmetic of the three unfused sweeps.
constexpr int PJ = 16;        // output rows per block
constexpr int PW = PJ + 6;    // warps per block
constexpr int PD = 2;         // planes of r/a_p, v1/a_p (and old p) copied ahead
constexpr int PR = 3;         // planes of 1/a_p kept (formed by stage 1, used by 2 and 3)

// 16-byte asynchronous global -> shared copy (cp.async, L2 only) and its
// group bookkeeping: a lane reads back only the slots it filled itself, so
// waiting on its own groups is enough (no barrier).  The memory clobbers keep
// the compiler from moving a read of a ring slot below the copy that refills
// it, or above the wait for the copy that fills it.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;" ::: "memory");
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

__device__ __forceinline__ int wrapn(int q, int n) { return ((q - 1) % n + n) % n + 1; }

// MV (phase C only): a fourth stage forms t = A cs at plane b-1 of the
// output rows with the dots (t,t) and (t,s), s = r - alf v1 (the matvec of
// :409-413 that otherwise runs as its own kernel), so the block keeps one
// more halo row each side (stage 3 runs on the rows j0-1 .. j0+PJ, whose cs
// it keeps in shared memory only) and marches one plane further.
template <int MODE, bool MV>
constexpr int precond3_warps() { return MV ? PJ + 8 : PW; }
template <int MODE, bool MV>
constexpr size_t precond3_smem() {
    // [stage slots][2][warp][lane] + copy-ahead [PD][arrays][warp][lane]
    // + 1/a_p ring [PR][warp][lane], float4 each
    return sizeof(float4) * ((MV ? 4 : 3) * 2 + PD * (MODE == 0 ? 3 : 2) + PR) *
           precond3_warps<MODE, MV>() * 32;
}

template <int MODE, bool CHEB, bool MV = false>
__global__ void __launch_bounds__(precond3_warps<MODE, MV>() * 32, 1)
    k_precond3(SolverArgs a, Coef<float> c, SolverBufs B, SolverScalars* S, int ni, Red2 R) {
    static_assert(!MV || MODE == 1, "the fused matvec stage is phase C's");
    constexpr int PWK = precond3_warps<MODE, MV>();
    constexpr int HW = MV ? 4 : 3;              // rows before the first output row
    constexpr int NSL = MV ? 4 : 3;             // stages with shared slots
    constexpr int NARR = MODE == 0 ? 3 : 2;     // streamed arrays: r/a_p, v1/a_p (, old p)
    constexpr int E = MV ? 1 : 0;               // extra planes of lead
    // [stage 0..NSL-1][buffer 0..1][warp][lane], then the copy-ahead ring
    // [PD][rh, vh (, p)][warp][lane], then the 1/a_p ring
    extern __shared__ float4 sbuf[];
    float4* ring = sbuf + NSL * 2 * PWK * 32;
    float4* rring = ring + PD * NARR * PWK * 32;  // [PR][warp][lane]: 1/a_p of a plane
    __shared__ double red_smem[64];
    double acc[2] = {0.0, 0.0};  // MV: (t,t), (t,s)
    pdl_wait();
    pdl_launch();
    if (S->done || S->pause) return;
    const Dims& d = a.d;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int kp = d.kp, jp = d.jp, ip = d.ip;
    const int k0 = 1 + 4 * lane;
    const bool live = k0 <= kp;
    const int nvalid = live ? min(4, kp - k0 + 1) : 0;
    const int j0 = 1 + blockIdx.x * PJ;
    const int jrow = j0 - HW + w;
    const int jw = wrapn(jrow, jp);
    const bool outrow = w >= HW && w < HW + PJ && jrow <= jp;
    const bool st1 = w >= 1 && w <= PWK - 2, st2 = w >= 2 && w <= PWK - 3;
    const bool st3 = MV ? (w >= 3 && w <= PWK - 4) : outrow;
    const int i0 = 1 + blockIdx.y * ni, i1 = min(i0 + ni - 1, ip);
    const int K = d.K, KJ = d.K * d.J;
    const int col = (live ? k0 : 1) + K * jw;
    // the k part of a_p per lane, the same in every warp: kept in shared
    // memory (stage 1 reads it once per step), written by warp 0 before the
    // first step's barrier (stage 1 starts at the third step)
    __shared__ float4 s_apk[32];
    float au[4], ad[4];
    vld(c.au + (live ? k0 : 1), au);
    vld(c.ad + (live ? k0 : 1), ad);
    if (w == 0)
        s_apk[lane] = make_float4(-au[0] - ad[0], -au[1] - ad[1], -au[2] - ad[2], -au[3] - ad[3]);
    // Neumann rows (dynamics.f90:206-211): the mirrored neighbour equals the
    // centre, so its difference term vanishes; zeroing its coefficient here
    // replaces a select per element and sweep
    if (k0 == 1) ad[0] = 0.0f;
#pragma unroll
    for (int e = 0; e < 4; e++)
        if (k0 + e == kp) au[e] = 0.0f;
    const float an = ld(c.an + jw), as = ld(c.as + jw);
    const float bet = (float)S->bet, omg = (float)S->omg, alf = (float)S->alf;
    const bool first = S->it == 0 || S->fresh;
    // CHEB: weighted sweeps (cheb_update); stage 1's operand is w1 s0, and
    // stages 1..3 weigh their corrections by w2..w4
    const float w1 = CHEB ? (float)a.cw[0] : 1.0f, w2 = CHEB ? (float)a.cw[1] : 1.0f,
                w3 = CHEB ? (float)a.cw[2] : 1.0f, w4 = CHEB ? (float)a.cw[3] : 1.0f;
    const float* __restrict__ rh = (const float*)B.rh;
    const float* __restrict__ vh = (const float*)B.vh;
    float* __restrict__ out = (float*)B.out;
    auto slot = [&](int stage, int buf, int warp) -> float4& {
        return sbuf[((stage * 2 + buf) * PWK + warp) * 32 + lane];
    };
    auto f4 = [](const float (&v)[4]) { return make_float4(v[0], v[1], v[2], v[3]); };
    auto rslot = [&](int step, int arr) -> float4& {
        return ring[(((step % PD) * NARR + arr) * PWK + w) * 32 + lane];
    };
    // copy-ahead of step t: r/a_p and v1/a_p at plane b+3, old p at plane b
    const int bstart = i0 - 6 - E, bend = i1 + E, nsteps = bend - bstart + 1;
    int qf = wrapn(bstart + 3, ip);  // plane of the next fetch, wrapped into 1..ip
    auto fetch = [&](int t) {
        if (t < nsteps) {
            const int b = bstart + t;
            const int o = col + KJ * qf;
            qf = qf == ip ? 1 : qf + 1;
            cp_async16(&rslot(t, 0), rh + o);
            if (!(MODE == 0 && first)) cp_async16(&rslot(t, 1), vh + o);
            if (MODE == 0 && !first && outrow && b >= i0) cp_async16(&rslot(t, 2), out + col + KJ * b);
        }
        cp_async_commit();  // an empty group keeps the group count per step
    };
    // s0 = q / a_p from r/a_p and v1/a_p (s0val, :393 / :404)
    auto s0_at = [&](int t, float (&s)[4]) {
        const float4 x4 = rslot(t, 0);
        const float x[4] = {x4.x, x4.y, x4.z, x4.w};
        if (MODE == 0 && first) {
#pragma unroll
            for (int e = 0; e < 4; e++) s[e] = x[e] - bet * (omg * 0.0f);
            return;
        }
        const float4 y4 = rslot(t, 1);
        const float y[4] = {y4.x, y4.y, y4.z, y4.w};
#pragma unroll
        for (int e = 0; e < 4; e++) s[e] = MODE == 0 ? x[e] - bet * (omg * y[e]) : x[e] - alf * y[e];
    };
    // one Jacobi sweep at plane q: res = xc + s0c - (A x)/a_p (the
    // reference's sweep), or with CHEB cheb_update(xc, s0c, (A x)/a_p, sc, wv);
    // A in the FP32 difference form of sten_task.  (A x)/a_p is formed as
    // (A x) * (1/a_p): stage 1 (FIRST) forms 1/a_p of its plane and keeps it
    // in this lane's slot of the 1/a_p ring, where stages 2 and 3 find it
    // one and two steps later (a lane reads back only its own slot).
    auto sweep = [&](auto first_c, int iq, const float (&xm)[4], const float (&xc)[4],
                     const float (&xp)[4], const float4 xs4, const float4 xn4,
                     const float (&s0c)[4], float (&res)[4], float sc, float wv, float4& rslot4) {
        constexpr bool FIRST = decltype(first_c)::value;
        const float ae = ld(c.ae + iq), aw = ld(c.aw + iq);
        const float xs[4] = {xs4.x, xs4.y, xs4.z, xs4.w}, xn[4] = {xn4.x, xn4.y, xn4.z, xn4.w};
        float ri[4];
        if (FIRST) {
            const float sij = -ae - aw - an - as;
            const float4 k4 = s_apk[lane];
            const float apk[4] = {k4.x, k4.y, k4.z, k4.w};
#pragma unroll
            for (int e = 0; e < 4; e++) ri[e] = __fdividef(1.0f, sij + apk[e]);
            rslot4 = make_float4(ri[0], ri[1], ri[2], ri[3]);
        } else {
            const float4 r4 = rslot4;
            ri[0] = r4.x;
            ri[1] = r4.y;
            ri[2] = r4.z;
            ri[3] = r4.w;
        }
        const float prev = __shfl_up_sync(0xffffffffu, xc[3], 1);
        const float next = __shfl_down_sync(0xffffffffu, xc[0], 1);
#pragma unroll
        for (int e = 0; e < 4; e++) {
            const float xd = e == 0 ? prev : xc[e - 1];
            const float xu = e == 3 ? next : xc[e + 1];
            const float c0 = xc[e];
            const float Ax = aw * (xm[e] - c0) + ae * (xp[e] - c0) + as * (xs[e] - c0) +
                             an * (xn[e] - c0) + ad[e] * (xd - c0) + au[e] * (xu - c0);
            const float q = Ax * ri[e];
            if (CHEB)
                res[e] = FIRST ? cheb_update(xc[e], s0c[e], q, sc, wv)
                               : cheb_update1(xc[e], s0c[e], q, wv);
            else
                res[e] = xc[e] + s0c[e] - q;
        }
    };
    auto rinv_slot = [&](int r) -> float4& { return rring[(r * PWK + w) * 32 + lane]; };
    float R0[4][4], R1[3][4], R2[3][4];  // s0 at b..b+3, s1 at b..b+2, s2 at b-1..b+1
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int e = 0; e < 4; e++) R0[r][e] = 0.0f;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int e = 0; e < 4; e++) R1[r][e] = R2[r][e] = 0.0f;
#pragma unroll
    for (int t = 0; t < PD; t++) fetch(t);
    int q1 = wrapn(bstart + 1, ip), q2 = wrapn(bstart + 2, ip);  // planes b+1, b+2 wrapped
    // 1/a_p ring slots: plane b (stage 3), b+1 (stage 2), b+2 (stage 1)
    int r3 = 0, r2 = 1, r1 = 2;
    using yes = std::integral_constant<bool, true>;
    using no = std::integral_constant<bool, false>;
    float xm4[4] = {0.0f, 0.0f, 0.0f, 0.0f};  // MV: own cs at plane b-2
    const float* __restrict__ rr = (const float*)B.r;
    const float* __restrict__ rv1 = (const float*)B.v1;
    float* __restrict__ tout = (float*)B.out2;
    for (int b = bstart; b <= bend; b++) {
        const int t = b - bstart;
        const int cur = t & 1, prv = cur ^ 1;
        cp_async_wait<PD - 1>();  // this lane's copies of step t have landed
        // stage 0: s0 at plane b+3
        s0_at(t, R0[3]);
        // stage 1: s1 at plane b+2 (j neighbours: s0 at b+2 from the last step)
        if (st1 && b >= i0 - 4 - E) {
            sweep(yes{}, q2, R0[1], R0[2], R0[3], slot(0, prv, w - 1), slot(0, prv, w + 1), R0[2],
                  R1[2], w1, w2, rinv_slot(r1));
        }
        // stage 2: s2 at plane b+1
        if (st2 && b >= i0 - 2 - E) {
            sweep(no{}, q1, R1[0], R1[1], R1[2], slot(1, prv, w - 1), slot(1, prv, w + 1), R0[1],
                  R2[2], 1.0f, w3, rinv_slot(r2));
        }
        // stage 3: s3 at plane b, the output
        float s3[4];
        if (st3 && b >= i0 - E) {
            const int qb = MV ? wrapn(b, ip) : b;
            sweep(no{}, qb, R2[0], R2[1], R2[2], slot(2, prv, w - 1), slot(2, prv, w + 1), R0[0],
                  s3, 1.0f, w4, rinv_slot(r3));
            const int o = col + KJ * b;
            if (MODE == 0) {
                if (first) {
#pragma unroll
                    for (int e = 0; e < 4; e++) s3[e] = s3[e] + bet * 0.0f;  // :397
                } else {
                    const float4 p4 = rslot(t, 2);  // old p, copied ahead
                    const float po[4] = {p4.x, p4.y, p4.z, p4.w};
#pragma unroll
                    for (int e = 0; e < 4; e++) s3[e] = s3[e] + bet * po[e];
                }
            }
            if (MV) slot(3, cur, w) = f4(s3);
            if (live && outrow && b >= i0 && b <= i1) vst(out + o, s3, nvalid);
        }
        // stage 4 (MV): t = A cs at plane b-1 of the output rows, (t,t), (t,s)
        if (MV && outrow && b >= i0) {
            // r and v1 of the next step's plane into L2 ahead of their use
            if (live && b + 1 <= bend) {
                const int on = col + KJ * wrapn(b, ip);
                prefetch_l2(rr + on);
                prefetch_l2(rv1 + on);
            }
            const float4 c4 = slot(3, prv, w);  // own cs at plane b-1
            const float xc[4] = {c4.x, c4.y, c4.z, c4.w};
            if (b >= i0 + 1) {
                const int qm = wrapn(b - 1, ip);
                const float ae = ld(c.ae + qm), aw = ld(c.aw + qm);
                const float4 xs4 = slot(3, prv, w - 1), xn4 = slot(3, prv, w + 1);
                const float xs[4] = {xs4.x, xs4.y, xs4.z, xs4.w};
                const float xn[4] = {xn4.x, xn4.y, xn4.z, xn4.w};
                const float prev = __shfl_up_sync(0xffffffffu, xc[3], 1);
                const float next = __shfl_down_sync(0xffffffffu, xc[0], 1);
                const int o = col + KJ * qm;
                float rv[4], v1v[4], t[4];
                vld(rr + o, rv);
                vld(rv1 + o, v1v);
#pragma unroll
                for (int e = 0; e < 4; e++) {
                    const float xd = e == 0 ? prev : xc[e - 1];
                    const float xu = e == 3 ? next : xc[e + 1];
                    const float c0 = xc[e];
                    // the FP32 difference form of sten_task (mat_ax, :219-222)
                    t[e] = aw * (xm4[e] - c0) + ae * (s3[e] - c0) + as * (xs[e] - c0) +
                           an * (xn[e] - c0) + ad[e] * (xd - c0) + au[e] * (xu - c0);
                    const float sv = rv[e] - alf * v1v[e];  // s of :404
                    if (e < nvalid) {
                        acc[0] += (double)t[e] * (double)t[e];
                        acc[1] += (double)t[e] * (double)sv;
                    }
                }
                if (live) vst(tout + o, t, nvalid);
            }
#pragma unroll
            for (int e = 0; e < 4; e++) xm4[e] = xc[e];
        }
        // this step's values for the neighbours' next step
        slot(0, cur, w) = f4(R0[3]);
        slot(1, cur, w) = f4(R1[2]);
        slot(2, cur, w) = f4(R2[2]);
        fetch(t + PD);  // into the ring slot step t has finished with
        q1 = q2;
        q2 = q2 == ip ? 1 : q2 + 1;
        {  // plane b+3 (stage 1's next plane) takes the slot plane b used
            const int rr = r3;
            r3 = r2;
            r2 = r1;
            r1 = rr;
        }
        __syncthreads();
#pragma unroll
        for (int e = 0; e < 4; e++) {
            R0[0][e] = R0[1][e];
            R0[1][e] = R0[2][e];
            R0[2][e] = R0[3][e];
            R1[0][e] = R1[1][e];
            R1[1][e] = R1[2][e];
            R2[0][e] = R2[1][e];
            R2[1][e] = R2[2][e];
        }
    }
    cp_async_wait<0>();
    if (MV) reduce_tail<OP_MATC, 2>(a, acc, R, red_smem, S);  // omega, :411-417
}

// Condition of a graph-driven loop: one more iteration while the solve has
// neither finished nor paused for a reliable update.  The round budget bounds
// the loop whatever the scalars do: past it the solve stops with
// DCM_E_TIMEOUT.
__device__ __forceinline__ unsigned loop_cond(cudaGraphConditionalHandle h, SolverScalars* S,
                                              int max_rounds) {
    unsigned go = (S->done || S->pause) ? 0u : 1u;
    if (go) {
        if (S->rounds >= max_rounds) {
            S->status = DCM_E_TIMEOUT;
            S->done = 1;
            go = 0u;
        } else {
            S->rounds = S->rounds + 1;
        }
    }
    cudaGraphSetConditional(h, go);
    return go;
}

// --- D: x, r updates, (r,r), (r,cr) -> err, next rho and bet -----------------
template <typename T, int V = KVec<T>::V>
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
    pdl_wait();
    pdl_launch();
    if (S->done || S->pause) {
        // stopped earlier in this iteration: end the graph loop
        if (a.cond_max && blockIdx.x == 0 && threadIdx.x == 0 && threadIdx.y == 0)
            cudaGraphSetConditional(a.cond, 0u);
        return;
    }
    const Dims& d = a.d;
    const T alf = (T)S->alf, omg = (T)S->omg;
    double acc[2] = {0.0, 0.0};
    const int lane = threadIdx.x;
    for (TaskIter tk(blockIdx.x * blockDim.y + threadIdx.y, gridDim.x * blockDim.y, a.nkt, d.jp);
         tk.i <= d.ip; tk.next()) {
        {
            TaskIter u = tk;  // the next task's seven streamed columns into L2
            u.next();
            if (u.i <= d.ip) {
                const int on = d.at(min(1 + V * (u.kt * BX + lane), d.kp), 1 + u.jr, u.i);
                prefetch_l2(x + on);
                prefetch_l2(p + on);
                prefetch_l2(cs + on);
                prefetch_l2(r + on);
                prefetch_l2(v1 + on);
                prefetch_l2(t + on);
                prefetch_l2(cr + on);
            }
        }
        const int k0 = 1 + V * (tk.kt * BX + lane);
        if (k0 > d.kp) continue;
        const int nvalid = min(V, d.kp - k0 + 1);
        const int j = 1 + tk.jr, i = tk.i;
        const int o = d.at(k0, j, i);
        T xv[V], pv[V], csv[V], rv[V], v1v[V], tv[V], crv[V], au[V], ad[V], rhv[V];
        vld_rw(x + o, xv);
        vld(p + o, pv);
        vld(cs + o, csv);
        vld_rw(r + o, rv);
        vld(v1 + o, v1v);
        vld(t + o, tv);
        vld(cr + o, crv);
        vld(c.au + k0, au);
        vld(c.ad + k0, ad);
        const T sij = -ld(c.ae + i) - ld(c.aw + i) - ld(c.an + j) - ld(c.as + j);
#pragma unroll
        for (int q = 0; q < V; q++) {
            const T sv = rv[q] - alf * v1v[q];
            xv[q] = xv[q] + alf * pv[q] + omg * csv[q];  // :419
            rv[q] = sv - omg * tv[q];                    // :420
            rhv[q] = rv[q] / (sij - au[q] - ad[q]);
            if (q < nvalid) {
                acc[0] += (double)rv[q] * (double)rv[q];
                acc[1] += (double)rv[q] * (double)crv[q];
            }
        }
        vst(x + o, xv, nvalid);
        vst(r + o, rv, nvalid);
        vst(rh + o, rhv, nvalid);
    }
    block_reduce<R_SUM, 2>(acc, smem);
    double s[2];
    if (reduce2<2>(acc, R, smem, s) && threadIdx.x == 0 && threadIdx.y == 0) {
        const int it = S->it + 1;
        S->it = it;
        const double err = sqrt(s[0]) / S->sc_err;  // :423
        S->err = err;
        S->nrm = S->rho;  // :425
        S->fresh = 0;
        if (S->ru && !(isfinite(s[0]) && isfinite(s[1]))) {
            S->restart = 2;  // the FP32 vectors went non-finite
            S->pause = 1;
        } else if (S->ru && !(err < a.tol) &&
                   (!(fabs(s[1]) > 1e-10 * sqrt(s[0] * S->crnorm)) ||
                    ++S->cycle_it > a.max_cycle)) {
            // (r, cr) collapsed, or the FP32 recursion stagnated: restart
            // from the FP64 residual with cr = r
            S->restart = 1;
            S->pause = 1;
        } else if (S->ru && (err < a.tol || sqrt(s[0]) < S->delta * S->ru_norm)) {
            // reliable update (mixed-precision form): the host replaces r by
            // the FP64 residual before the iteration continues
            S->pause = 1;
            S->rho = s[1];
        } else if (err < a.tol) {  // :428
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
        if (a.cond_max) loop_cond(a.cond, S, a.cond_max);
    }
}

// --- after the solve: halo rows of x (dynamics.f90:437-442 or, after the
//     early return, mat_ax's rows :203-211) and the driver's
//     exchange_along_dim_wo(p) (driver_code.f90:506)
template <typename T, typename TS>
__global__ void __launch_bounds__(256) k_bicg_post(Dims d, T* __restrict__ x,
                                                   const TS* __restrict__ sw,
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
                x[d.at(0, jj, ii)] = v - (T)sw[d.at(0, jj, ii)] * dz0;
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
    // function-local statics are initialised once, thread-safely
    static const int sms = [] {
        int dev = 0, n = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        return n;
    }();
    return sms;
}

// resident blocks of a persistent reducing kernel
template <typename K>
static int persistent_grid(K kernel) {
    int per = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, BX * BY, 0);
    return sm_count() * (per > 0 ? per : 1);
}

// Warp tasks: (k-chunk of 32 V levels, j, i).
template <typename T>
static int kchunks(const Dims& d, int vw = 0) {
    const int V = vw > 0 ? vw : KVec<T>::V;
    return (d.kp + V * BX - 1) / (V * BX);
}

// levels per lane of the FP32 iteration kernels: a.vw (2 or 4), 4 by default
static inline bool narrow(const SolverArgs& a) { return a.vw == 2; }

// a kernel launch, with programmatic stream serialisation when `pdl`
template <typename... P, typename... A>
static void launch(bool pdl, void (*kern)(P...), dim3 grid, dim3 block, size_t smem,
                   cudaStream_t st, A... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = at;
    cfg.numAttrs = pdl ? 1 : 0;
    cudaLaunchKernelEx(&cfg, kern, args...);
}

// blocks of a reducing kernel: all resident blocks (tasks = 0: persistent,
// each warp strides over many tasks), or enough blocks for `tasks` warp
// tasks per warp (tasks = 1: one task per warp, as many blocks as tasks / 8),
// never more than the reduction buffers hold
static int red_grid(const SolverArgs& a, int full, int nkt, int ni = 1) {
    long long want = full;
    if (a.tasks > 0) {
        const long long ntask = (long long)nkt * a.d.jp * ((a.d.ip + ni - 1) / ni);
        want = (ntask + (long long)BY * a.tasks - 1) / ((long long)BY * a.tasks);
    }
    if (a.max_blocks > 0) want = std::min(want, (long long)a.max_blocks);
    return (int)std::max(1LL, want);
}

template <typename T, int OP, int MODE, int V>
static void sten_v(const SolverArgs& a, const Coef<T>& c, const SolverBufs& B, SolverWork<T>& w,
                   cudaStream_t st) {
    constexpr bool RED = OP == OP_SETUP || OP == OP_MATC || OP == OP_MATP;
    if (RED) {
        if (a.ni > 1) {
            static const int full = persistent_grid(k_sten<T, OP, MODE, V, true>);
            launch(a.pdl, k_sten<T, OP, MODE, V, true>, dim3(red_grid(a, full, a.nkt, a.ni)),
                   dim3(BX, BY), 0, st, a, c, B, w.red, w.S);
        } else {
            static const int full = persistent_grid(k_sten<T, OP, MODE, V>);
            launch(a.pdl, k_sten<T, OP, MODE, V>, dim3(red_grid(a, full, a.nkt, 1)),
                   dim3(BX, BY), 0, st, a, c, B, w.red, w.S);
        }
    } else {
        // at most 256 threads: the kernels are compiled with __launch_bounds__(256)
        const int by = a.by >= 1 && a.by <= 256 / BX ? a.by : BY;
        const int ni = OP == OP_SW1 ? a.ni : 1;
        const dim3 grid(a.nkt, (a.d.jp + by - 1) / by, (a.d.ip + ni - 1) / ni);
        launch(a.pdl, k_sten<T, OP, MODE, V>, grid, dim3(BX, by), 0, st, a, c, B, w.red, w.S);
    }
}

template <typename T, int OP, int MODE>
static void sten(const SolverArgs& a, const Coef<T>& c, const SolverBufs& B, SolverWork<T>& w,
                 cudaStream_t st, int cat) {
    ProfScope ps(cat, st);
    if constexpr (std::is_same<T, float>::value) {
        if (narrow(a)) {
            sten_v<T, OP, MODE, 2>(a, c, B, w, st);
            return;
        }
    }
    sten_v<T, OP, MODE, KVec<T>::V>(a, c, B, w, st);
}


// the fused preconditioner applies (FP32, one k-chunk per column)
template <typename T>
static bool fused_ok(const SolverArgs& a) {
    return std::is_same<T, float>::value && a.fuse && !narrow(a) && a.nkt == 1;
}

// one fused preconditioner launch: PJ-row strips x i-chunks, at most one
// block per SM so that the chunks (and their 6-plane warm-up) are as long as
// the SM count allows, and no chunk shorter than 8 planes
// mv: phase C with the matvec t = A cs and its dots as a fourth stage
static void precond3(const SolverArgs& a, const Coef<float>& c, const SolverBufs& B,
                     SolverScalars* S, int mode, bool mv, const Red2& R, cudaStream_t st) {
    ProfScope ps(P_JACOBI, st);
    const int nstrips = (a.d.jp + PJ - 1) / PJ;
    // chunks of at least 8 planes (each carries a 6-plane warm-up)
    const int nch = std::max(1, std::min((a.d.ip + 7) / 8, sm_count() / nstrips));
    const int ni = (a.d.ip + nch - 1) / nch;
    const dim3 grid(nstrips, (a.d.ip + ni - 1) / ni);
    auto go = [&](auto kern, int warps, size_t smem) {
        launch(a.pdl, kern, grid, dim3(warps * 32), smem, st, a, c, B, S, ni, R);
    };
    if (mode == 0) {
        constexpr int wp = precond3_warps<0, false>();
        constexpr size_t sm = precond3_smem<0, false>();
        a.cheb ? go(k_precond3<0, true>, wp, sm) : go(k_precond3<0, false>, wp, sm);
    } else if (!mv) {
        constexpr int wp = precond3_warps<1, false>();
        constexpr size_t sm = precond3_smem<1, false>();
        a.cheb ? go(k_precond3<1, true>, wp, sm) : go(k_precond3<1, false>, wp, sm);
    } else {
        constexpr int wp = precond3_warps<1, true>();
        constexpr size_t sm = precond3_smem<1, true>();
        a.cheb ? go(k_precond3<1, true, true>, wp, sm) : go(k_precond3<1, false, true>, wp, sm);
    }
}

// programmatic edges inside the graph-driven iterations (probed once)
static int g_pdl_graphs = 0;
static bool probe_pdl_graphs();

void solver_init() {
    const int sm0 = (int)precond3_smem<0, false>(), sm1 = (int)precond3_smem<1, false>(),
              sm1m = (int)precond3_smem<1, true>();
    cudaFuncSetAttribute(k_precond3<0, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm0);
    cudaFuncSetAttribute(k_precond3<1, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm1);
    cudaFuncSetAttribute(k_precond3<0, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm0);
    cudaFuncSetAttribute(k_precond3<1, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, sm1);
    cudaFuncSetAttribute(k_precond3<1, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         sm1m);
    cudaFuncSetAttribute(k_precond3<1, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         sm1m);
    static std::once_flag probed;  // handles may be created from several threads
    std::call_once(probed, [] { g_pdl_graphs = probe_pdl_graphs() ? 1 : 0; });
}

bool solver_pdl_available() { return g_pdl_graphs != 0; }

template <typename T>
static void launch_iteration(const SolverArgs& a, const Coef<T>& c, SolverWork<T>& w, T* x,
                             cudaStream_t st) {
    SolverBufs B{};
    B.r = w.r;
    B.v1 = w.v1;
    B.rh = w.rh;
    B.vh = w.vh;
    const bool fused = fused_ok<T>(a);
    SolverArgs a0 = a;  // the first kernel follows no kernel of this iteration
    a0.pdl = 0;
    // phase B: precondition(s <- t), p = s + bet p, v1 = A p
    if (fused) {
        if constexpr (std::is_same<T, float>::value) {
            B.out = w.p;
            precond3(a0, c, B, w.S, 0, false, w.red, st);
        }
    } else {
        B.out = w.sA;
        B.sweep = 1;
        sten<T, OP_SW1, 0>(a0, c, B, w, st, P_JACOBI);
        B.sin = w.sA;
        B.out = w.sB;
        B.sweep = 2;
        sten<T, OP_SW, 0>(a, c, B, w, st, P_JACOBI);
        B.sin = w.sB;
        B.out = w.p;
        B.sweep = 3;
        sten<T, OP_SW3P, 0>(a, c, B, w, st, P_JACOBI);
    }
    B.sin = w.p;
    B.cr = w.cr;
    B.out = w.v1;
    B.out3 = w.vh;
    sten<T, OP_MATP, 0>(a, c, B, w, st, P_MATVEC);
    // phase C: precondition(cs <- s), t = A cs
    B.sin = nullptr;
    const bool mv = fused && a.fuse_mv;
    if (fused) {
        if constexpr (std::is_same<T, float>::value) {
            B.out = w.sA;
            B.out2 = w.t;
            precond3(a, c, B, w.S, 1, mv, w.red, st);
        }
    } else {
        B.out = w.sA;
        B.sweep = 1;
        sten<T, OP_SW1, 1>(a, c, B, w, st, P_JACOBI);
        B.sin = w.sA;
        B.out = w.sB;
        B.sweep = 2;
        sten<T, OP_SW, 1>(a, c, B, w, st, P_JACOBI);
        B.sin = w.sB;
        B.out = w.sA;
        B.sweep = 3;
        sten<T, OP_SW, 1>(a, c, B, w, st, P_JACOBI);
    }
    if (!mv) {
        B.sin = w.sA;
        B.out = w.t;
        sten<T, OP_MATC, 1>(a, c, B, w, st, P_MATVEC);
    }
    // phase D
    {
        ProfScope ps(P_UPDATE, st);
        auto go = [&](auto kern) {
            static const int full = persistent_grid(kern);
            launch(a.pdl, kern, dim3(red_grid(a, full, a.nkt)), dim3(BX, BY), 0, st, a, c, x,
                   (const T*)w.p, (const T*)w.sA, w.r, (const T*)w.v1, (const T*)w.t,
                   (const T*)w.cr, w.rh, w.red, w.S);
        };
        if constexpr (std::is_same<T, float>::value) {
            if (narrow(a))
                go(k_bicg_update<T, 2>);
            else
                go(k_bicg_update<T>);
        } else {
            go(k_bicg_update<T>);
        }
    }
}

// ---- graph-driven loops ------------------------------------------------------
// Iterations per body of a WHILE node.  Each iteration's update kernel
// counts and tests the loop (loop_cond) and the last one's result decides
// the next body; an iteration that follows the end of the solve (or a pause
// for a reliable update) in the same body launches kernels that return at
// once.  Two per body halve the per-body cost of the conditional node.
constexpr int ITERS_PER_BODY = 2;

// The first condition of an iteration loop, before its WHILE node; the update
// kernel sets it after every iteration (loop_cond).
__global__ void k_loop_cond(cudaGraphConditionalHandle h, SolverScalars* S, int max_rounds) {
    loop_cond(h, S, max_rounds);
}

// Mixed form: the start of an FP64 update cycle, the first condition of its
// loop of FP32 iterations.
__global__ void k_cycle_start(cudaGraphConditionalHandle h, SolverScalars* S, int max_rounds) {
    S->cycles = S->cycles + 1;
    loop_cond(h, S, max_rounds);
}

// Mixed form: condition of the outer WHILE node, another cycle while the
// solve has not finished.
__global__ void k_outer_cond(cudaGraphConditionalHandle h, const SolverScalars* S) {
    cudaGraphSetConditional(h, S->done ? 0u : 1u);
}

// Condition of the IF node of the mixed solve: the FP32 iterations paused
// for a reliable update (otherwise they finished).
__global__ void k_branch_pause(cudaGraphConditionalHandle h, SolverScalars* S) {
    const unsigned go = S->pause ? 1u : 0u;
    if (go) S->ru_runs = S->ru_runs + 1;
    cudaGraphSetConditional(h, go);
}

namespace {

bool ok(cudaError_t e) { return e == cudaSuccess; }

// Add a conditional node after the work captured so far on `st` (which must
// be capturing); the handle is created on the capturing graph first so that
// kernels captured before the node can set it.
bool capture_cond_handle(cudaStream_t st, cudaGraphConditionalHandle* h, unsigned dflt) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    if (!ok(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, nullptr, nullptr)) ||
        cs != cudaStreamCaptureStatusActive)
        return false;
    return ok(cudaGraphConditionalHandleCreate(h, cg, dflt, 0));
}
bool capture_cond_node(cudaStream_t st, cudaGraphConditionalHandle h,
                       cudaGraphConditionalNodeType type, unsigned size, cudaGraph_t* bodies) {
    cudaStreamCaptureStatus cs;
    cudaGraph_t cg = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    if (!ok(cudaStreamGetCaptureInfo(st, &cs, nullptr, &cg, &deps, &nd)) ||
        cs != cudaStreamCaptureStatusActive)
        return false;
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = type;
    p.conditional.size = size;
    cudaGraphNode_t node;
    if (!ok(cudaGraphAddNode(&node, cg, deps, nd, &p))) return false;
    for (unsigned q = 0; q < size; q++) bodies[q] = p.conditional.phGraph_out[q];
    return ok(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies));
}

// capture launches into an existing (body) graph on a side stream
template <typename F>
bool capture_into(cudaStream_t side, cudaGraph_t body, F&& launches) {
    if (!ok(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0,
                                          cudaStreamCaptureModeRelaxed)))
        return false;
    launches(side);
    const bool launched = cudaPeekAtLastError() == cudaSuccess;
    cudaGraph_t out = body;
    return ok(cudaStreamEndCapture(side, &out)) && launched;
}

struct CaptureGuard {  // launches inside a capture are counted per run instead
    CaptureGuard() {
        if (g_prof) g_prof->capturing = true;
    }
    ~CaptureGuard() {
        if (g_prof) g_prof->capturing = false;
    }
};

bool side_streams(SolveGraph& G) {
    for (cudaStream_t& s : G.side)
        if (!s && !ok(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking))) return false;
    return true;
}

}  // namespace

__global__ void k_pdl_probe() {
    pdl_wait();
    pdl_launch();
}

// Whether this runtime takes a programmatic edge between two kernels captured
// into the body of a WHILE node, as the graph-driven solves place them.  A
// graph of that shape is instantiated, never launched; without the edges the
// solves launch each kernel after its predecessor.
static bool probe_pdl_graphs() {
    cudaStream_t s = nullptr;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t ge = nullptr;
    cudaGraphConditionalHandle h{};
    bool good = ok(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)) &&
                ok(cudaGraphCreate(&g, 0)) && ok(cudaGraphConditionalHandleCreate(&h, g, 0, 0));
    cudaGraphNodeParams p = {};
    p.type = cudaGraphNodeTypeConditional;
    p.conditional.handle = h;
    p.conditional.type = cudaGraphCondTypeWhile;
    p.conditional.size = 1;
    cudaGraphNode_t node;
    good = good && ok(cudaGraphAddNode(&node, g, nullptr, 0, &p));
    good = good && capture_into(s, p.conditional.phGraph_out[0], [&](cudaStream_t s2) {
               launch(false, k_pdl_probe, dim3(1), dim3(32), 0, s2);
               launch(true, k_pdl_probe, dim3(1), dim3(32), 0, s2);
           });
    good = good && ok(cudaGraphInstantiate(&ge, g, 0));
    if (ge) cudaGraphExecDestroy(ge);
    if (g) cudaGraphDestroy(g);
    if (s) cudaStreamDestroy(s);
    cudaGetLastError();
    return good;
}

// Weights of the Chebyshev-weighted sweeps: the preconditioned operator is
// 1 - R(D^-1 A) with R(mu) = prod_m (1 - mu / theta_m), theta_m the four
// roots of the degree-4 Chebyshev polynomial on [lo, 2]
// (theta_m = (2 + lo)/2 + (2 - lo)/2 cos((2m - 1) pi / 8)); the reference's
// sweeps are theta_m = 1, R(mu) = (1 - mu)^4, which vanishes at mu = 0 and at
// the checkerboard modes' mu = 2 alike.  Same three operator applications.
// The largest weight comes first (it scales s0 itself), the smallest last:
// the later sweeps' corrections are near-cancelling FP32 differences, and
// weighing them by up to 8 (lo = 0.05) made the FP32 recursion erratic at
// 512x512x256 (one step took 741 iterations against about 200 in this order).
static void cheb_weights(double lo, double (&w)[4]) {
    const double pi = 3.14159265358979323846;
    for (int m = 1; m <= 4; m++)
        w[4 - m] = 1.0 / ((2.0 + lo) / 2.0 + (2.0 - lo) / 2.0 * std::cos((2 * m - 1) * pi / 8.0));
}

static void no_cheb(SolverArgs& a) {
    a.cheb = 0;
    for (double& x : a.cw) x = 1.0;
}

// --- small domains: the whole FP64 solve in one cluster ----------------------
// A domain of a few thousand points (the 128 x 1 x 64 shear layer: 8,192)
// leaves the multi-kernel iteration bound by launch latency: nine kernels of
// a few microseconds each.  Here one thread-block cluster of SMALL_CL blocks
// of SMALL_THREADS threads (one block per SM) runs the whole of bicgstab
// (dynamics.f90:367-435) in the reference's own algebra: setup, and per
// iteration t = r - bet (omg v1), the three Jacobi sweeps of precondition
// (:241-270; s = q/a_p, then s + (q - A s)/a_p), p = s + bet p, v1 = A p,
// s = r - alf v1, cs = M s, t = A cs, the x and r updates.  The points are
// dealt to the cluster's threads in turn; passes are separated by cluster
// barriers (release / acquire at cluster scope, so the next pass reads the
// neighbours other blocks wrote).  Pointwise statements share a pass with
// the statement before or after them (t and s with s/a_p, p with the last
// sweep, (r,cr) with the r update), sums taken together share one barrier,
// and a pass that a sum follows leaves its barrier to the sum's: 11 cluster
// barriers per iteration, each value computed as the separate statements
// compute it.  Every dot product is a fixed-order sum:
// within a block by a shuffle tree, across the cluster by reading the blocks'
// partials through distributed shared memory in rank order, so every thread
// gets the same value.  Vectors stay in global memory (L2-resident at these
// sizes).  The scalars and statuses are those of the multi-kernel path.
constexpr int SMALL_THREADS = 1024;
constexpr int SMALL_CL = 8;  // blocks of the cluster (the portable maximum)

// sum over the block, the same value in every thread (a fixed reduction tree)
__device__ __forceinline__ double small_sum(double v, double* sh) {
    constexpr unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();  // the partials of the previous sum have been read
    if (lane == 0) sh[w] = v;
    __syncthreads();
    double t = lane < (int)(blockDim.x >> 5) ? sh[lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(FULL, t, o);
    return t;
}

// two sums over the block in one tree (each as small_sum forms it)
__device__ __forceinline__ void small_sum2(double& a, double& b, double* sh) {
    constexpr unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(FULL, a, o);
        b += __shfl_xor_sync(FULL, b, o);
    }
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    __syncthreads();  // the partials of the previous sum have been read
    if (lane == 0) {
        sh[w] = a;
        sh[32 + w] = b;
    }
    __syncthreads();
    const bool in = lane < (int)(blockDim.x >> 5);
    a = in ? sh[lane] : 0.0;
    b = in ? sh[32 + lane] : 0.0;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        a += __shfl_xor_sync(FULL, a, o);
        b += __shfl_xor_sync(FULL, b, o);
    }
}

struct SmallOp {
    Dims d;
    Coef<double> c;
    // the interior point of flat index q (k fastest)
    __device__ __forceinline__ void at(int q, int& k, int& j, int& i) const {
        k = 1 + q % d.kp;
        const int r = q / d.kp;
        j = 1 + r % d.jp;
        i = 1 + r / d.jp;
    }
    __device__ __forceinline__ double ap(int k, int j, int i) const {
        return -ld(c.ae + i) - ld(c.aw + i) - ld(c.an + j) - ld(c.as + j) - ld(c.au + k) -
               ld(c.ad + k);  // set_mat_a, dynamics.f90:93-95
    }
    // mat_ax (:219-222, a_c = 0) with the exchange's periodic x, y images and
    // the Neumann rows x(0) = x(1), x(kp+1) = x(kp) (:206-211)
    __device__ __forceinline__ double ax(const double* __restrict__ x, int k, int j, int i,
                                         double ap_) const {
        const int o = d.at(k, j, i);
        const double xc = x[o];
        const double xw = x[d.at(k, j, i == 1 ? d.ip : i - 1)];
        const double xe = x[d.at(k, j, i == d.ip ? 1 : i + 1)];
        const double xs = x[d.at(k, j == 1 ? d.jp : j - 1, i)];
        const double xn = x[d.at(k, j == d.jp ? 1 : j + 1, i)];
        const double xd = k == 1 ? xc : x[o - 1];
        const double xu = k == d.kp ? xc : x[o + 1];
        return ld(c.aw + i) * xw + ld(c.ae + i) * xe + ld(c.as + j) * xs + ld(c.an + j) * xn +
               ld(c.ad + k) * xd + ld(c.au + k) * xu + ap_ * xc + 0.0;
    }
};

__global__ void __launch_bounds__(SMALL_THREADS, 1)
    k_bicgstab_small(SolverArgs a, SmallOp op, double* __restrict__ x,
                     const double* __restrict__ b, double* __restrict__ r,
                     double* __restrict__ cr, double* __restrict__ p, double* __restrict__ v1,
                     double* __restrict__ tq, double* __restrict__ sa, double* __restrict__ sb,
                     double* __restrict__ sv, SolverScalars* S, int max_rounds) {
    __shared__ double sh[64];
    __shared__ double part[2][2];  // this block's partials of the current sums (two buffers)
    namespace cg = cooperative_groups;
    cg::cluster_group cl = cg::this_cluster();
    const Dims& d = a.d;
    const int n = d.ip * d.jp * d.kp;
    const int rank = (int)cl.block_rank(), nb = (int)cl.num_blocks();
    const int tid = threadIdx.x, nt = blockDim.x;
    const int first = rank * nt + tid, stride = nb * nt;
    // a pass over this thread's points; `pass` ends with the cluster barrier,
    // `each` leaves it to the cluster sum that follows (its barrier orders
    // the pass's writes and reads before every later pass)
    auto each = [&](auto body) {
        for (int q = first; q < n; q += stride) {
            int k, j, i;
            op.at(q, k, j, i);
            body(d.at(k, j, i), k, j, i);
        }
    };
    auto pass = [&](auto body) {
        each(body);
        cl.sync();
    };
    int pb = 0;  // partial buffer of the next sums
    // two sums over the cluster, the same values in every thread: the
    // block's shuffle-tree sums, then the blocks' partials in rank order
    auto csum2 = [&](double& u, double& v) {
        small_sum2(u, v, sh);
        if (tid == 0) {
            part[pb][0] = u;
            part[pb][1] = v;
        }
        cl.sync();
        double tu = 0.0, tv = 0.0;
        for (int r2 = 0; r2 < nb; r2++) {
            const double* pr = cl.map_shared_rank(&part[pb][0], r2);
            tu += pr[0];
            tv += pr[1];
        }
        pb ^= 1;  // the next sums write the other buffer while this one may still be read
        u = tu;
        v = tv;
    };
    auto csum1 = [&](double v) {
        const double bs = small_sum(v, sh);
        if (tid == 0) part[pb][0] = bs;
        cl.sync();
        double t = 0.0;
        for (int r2 = 0; r2 < nb; r2++) t += *cl.map_shared_rank(&part[pb][0], r2);
        pb ^= 1;
        return t;
    };
    // precondition (:241-270) of the q that set_q forms and stores at a
    // point: s = q/a_p in the same pass, then three Jacobi sweeps (sa/sb
    // ping-pong, the result in sb); with bp the last sweep also forms
    // p = s + bet p (:397) at its point
    // (qv is not restrict-qualified: set_q writes the same array)
    auto precondition = [&](const double* qv, auto set_q, bool bp, double bet) {
        pass([&](int o, int k, int j, int i) { sa[o] = set_q(o) / op.ap(k, j, i); });
        for (int sweep = 0; sweep < 3; sweep++) {
            const double* __restrict__ src = sweep == 1 ? sb : sa;
            double* __restrict__ dst = sweep == 1 ? sa : sb;
            pass([&](int o, int k, int j, int i) {
                const double apv = op.ap(k, j, i);
                const double sn = src[o] + (qv[o] - op.ax(src, k, j, i, apv)) / apv;
                dst[o] = sn;
                if (bp && sweep == 2) p[o] = sn + bet * p[o];
            });
        }
    };
    // ---- set-up (:367-383); cr = r, so (r,cr) of the first iteration is (r,r)
    double bb = 0.0, rr = 0.0;
    each([&](int o, int k, int j, int i) {
        const double rv = b[o] - op.ax(x, k, j, i, op.ap(k, j, i));
        r[o] = rv;
        cr[o] = rv;
        p[o] = 0.0;
        v1[o] = 0.0;
        bb += b[o] * b[o];
        rr += rv * rv;
    });
    csum2(bb, rr);
    double sc = sqrt(bb);
    sc = sc > a.sc_floor ? sc : a.sc_floor;  // :370-371
    double err = sc > 0.0 ? sqrt(rr) / sc : 0.0;
    int status = 0, it = 0, early = 0;
    double rho = 0.0, alf = 1.0, omg = 1.0, nrm = 1.0, bet = 0.0, tt = 0.0, ts = 0.0;
    double rc = rr;  // (r,cr) for the next iteration
    if (err < a.tol) {
        early = 1;  // :382-383
    } else if (!(err == err)) {
        status = DCM_E_NONFINITE;
    } else {
        for (it = 1;; it++) {
            if (it > max_rounds) {  // the round budget, as the graph-driven loop bounds it
                status = DCM_E_TIMEOUT;
                it = it - 1;
                break;
            }
            rho = rc;                                // :391
            bet = (rho / nrm) * (alf / omg);         // :392
            // t = r - bet (omg v1) (:393) and s = M t, p = s + bet p (:394-397)
            precondition(tq, [&](int o) { return tq[o] = r[o] - bet * (omg * v1[o]); }, true,
                         bet);
            double cv = 0.0;
            each([&](int o, int k, int j, int i) {
                const double v = op.ax(p, k, j, i, op.ap(k, j, i));  // :399-400
                v1[o] = v;
                cv += cr[o] * v;
            });
            nrm = csum1(cv);                         // :401
            alf = rho / nrm;                         // :403
            // s = r - alf v1 (:404) and cs = M s (:405-407), cs in sb
            precondition(sv, [&](int o) { return sv[o] = r[o] - alf * v1[o]; }, false, 0.0);
            double t2 = 0.0, t3 = 0.0;
            each([&](int o, int k, int j, int i) {
                const double tv = op.ax(sb, k, j, i, op.ap(k, j, i));  // :408-409
                tq[o] = tv;
                t2 += tv * tv;
                t3 += tv * sv[o];
            });
            csum2(t2, t3);
            tt = t2;                                 // :410
            ts = t3;                                 // :411
            omg = ts / tt;                           // :412
            if (fabs(omg) < a.tiny) {                // :414-417
                status = DCM_E_BREAKDOWN;
                break;
            }
            // x and r (:419-420), with (r,r) for the test and (r,cr) for the
            // next iteration's rho
            double r2s = 0.0, rcs = 0.0;
            each([&](int o, int, int, int) {
                x[o] = x[o] + alf * p[o] + omg * sb[o];  // :419
                const double rv = sv[o] - omg * tq[o];   // :420
                r[o] = rv;
                r2s += rv * rv;
                rcs += rv * cr[o];
            });
            csum2(r2s, rcs);
            rc = rcs;
            err = sqrt(r2s) / sc;                    // :423
            nrm = rho;                               // :425
            if (err < a.tol) break;                  // :428
            if (!(err == err)) {
                status = DCM_E_NONFINITE;
                break;
            }
            if (it >= a.itmax) {
                status = DCM_E_NOCONV;               // :431-434
                break;
            }
        }
    }
    if (tid == 0 && rank == 0) {
        S->sc_err = sc;
        S->err = err;
        S->rho = rho;
        S->alf = alf;
        S->omg = omg;
        S->bet = bet;
        S->nrm = nrm;
        S->tt = tt;
        S->ts = ts;
        S->it = it;
        S->rounds = it;
        S->status = status;
        S->early = early;
        S->done = 1;
        S->pause = 0;
        S->ru = 0;
    }
    cl.sync();  // no block leaves while another may still read its partials
}

// the one-cluster solve applies (FP64, interior points <= w.small_max)
template <typename T>
static bool small_ok(const SolverWork<T>& w, const Dims& d) {
    return std::is_same<T, double>::value && w.small_max > 0 &&
           (long long)d.ip * d.jp * d.kp <= w.small_max;
}

template <typename T>
int solver_run(SolverWork<T>& w, const Dims& d, T* x, const T* b, const T* sw, const T* dzn,
               double tol, int itmax, int wo, int chunk, cudaStream_t st, SolverScalars* host_S,
               int* launched_iters, double sc_floor, bool post) {
    SolverArgs a;
    a.d = d;
    a.itmax = itmax;
    a.tol = tol;
    a.sc_floor = sc_floor;
    a.vw = std::is_same<T, float>::value ? w.vw : 0;
    a.nkt = kchunks<T>(d, a.vw);
    a.max_updates = 0;
    a.max_cycle = 0;
    a.by = w.by;
    a.tasks = w.tasks;
    a.max_blocks = w.max_blocks;
    a.ni = w.ni >= 1 ? w.ni : 1;
    a.fuse = w.fuse;
    a.fuse_mv = w.fuse == 2 ? 1 : 0;
    no_cheb(a);  // the FP64 path keeps the reference's sweeps
    if (w.tiny >= 0.0) a.tiny = w.tiny;
    const Coef<T> c = coef_of(w);
    SolverBufs B{};
    B.x = x;
    B.b = b;
    B.out = w.r;
    B.out2 = w.cr;
    B.out3 = w.rh;
    const int max_rounds = w.round_budget > 0 ? w.round_budget : itmax + 1;
    auto post_launch = [&](cudaStream_t s) {
        if (post) {
            ProfScope ps(P_POST, s);
            k_bicg_post<T, T><<<interior_grid(d, d.kp), dim3(BX, BY), 0, s>>>(d, x, sw, dzn, w.S,
                                                                              wo);
        }
    };
    if constexpr (std::is_same<T, double>::value) {
        if (small_ok(w, d)) {
            // the whole solve as one block, then the halo fix-up: the same two
            // launches whether captured into a graph or not
            SmallOp op{d, c};
            {
                ProfScope ps(P_SETUP, st);
                cudaLaunchAttribute at[1];
                at[0].id = cudaLaunchAttributeClusterDimension;
                at[0].val.clusterDim.x = SMALL_CL;
                at[0].val.clusterDim.y = 1;
                at[0].val.clusterDim.z = 1;
                cudaLaunchConfig_t cfg = {};
                cfg.gridDim = dim3(SMALL_CL);
                cfg.blockDim = dim3(SMALL_THREADS);
                cfg.stream = st;
                cfg.attrs = at;
                cfg.numAttrs = 1;
                cudaLaunchKernelEx(&cfg, k_bicgstab_small, a, op, x, b, w.r, w.cr, w.p, w.v1, w.t,
                                   w.sA, w.sB, w.rh, w.S, max_rounds);
            }
            post_launch(st);
            if (w.graph && w.emit) return cudaPeekAtLastError() == cudaSuccess ? DCM_OK : DCM_E_CUDA;
            cudaMemcpyAsync(host_S, w.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return DCM_E_CUDA;
            if (launched_iters) *launched_iters = host_S->rounds;
            return host_S->status;
        }
    }
    // the whole solve into the graph being captured on `s`: setup, the
    // WHILE loop of iterations, the halo fix-up
    auto emit = [&](cudaStream_t s, SolveGraph& G) {
        if (!side_streams(G)) return false;
        CaptureGuard cg;
        cudaGraphConditionalHandle hw{};
        cudaGraph_t body[1] = {nullptr};
        sten<T, OP_SETUP, 0>(a, c, B, w, s, P_SETUP);
        bool good = capture_cond_handle(s, &hw, 0);
        if (good) k_loop_cond<<<1, 1, 0, s>>>(hw, w.S, max_rounds);
        good = good && capture_cond_node(s, hw, cudaGraphCondTypeWhile, 1, body);
        SolverArgs ai = a;  // the update kernel sets the loop's condition
        ai.cond = hw;
        ai.cond_max = max_rounds;
        ai.pdl = g_pdl_graphs && w.pdl;
        good = good && capture_into(G.side[0], body[0], [&](cudaStream_t s2) {
                   for (int n = 0; n < ITERS_PER_BODY; n++) launch_iteration<T>(ai, c, w, x, s2);
               });
        post_launch(s);
        return good && cudaPeekAtLastError() == cudaSuccess;
    };
    if (w.graph && w.emit) return emit(st, *w.graph) ? DCM_OK : DCM_E_CUDA;
    const bool use_graph = w.graph && !(g_prof && g_prof->on);
    if (use_graph) {
        SolveGraph& G = *w.graph;
        const void* kp[6] = {x, b, sw, dzn, w.r, w.S};
        const double kd[3] = {tol, sc_floor, a.tiny};
        // launch shape: by < 16, tasks < 16, ni < 64, fuse < 4, pdl < 2, vw < 8
        const int shape = a.by + 16 * a.tasks + 256 * a.ni + 16384 * a.fuse +
                          65536 * (w.pdl ? 1 : 0) + 131072 * a.vw;
        const int ki[6] = {itmax, wo, (post ? 1 : 0) + 2 * max_rounds, (int)sizeof(T) + 16 * shape,
                           d.ip * 4096 + d.jp, d.kp};
        if (!G.matches(kp, kd, ki)) {
            G.release();
            bool good = ok(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            if (good) good = emit(st, G);
            cudaGraph_t gr = nullptr;
            const bool ended = ok(cudaStreamEndCapture(st, &gr));
            G.graph = gr;
            if (!good || !ended || !ok(cudaGraphInstantiate(&G.exec, gr, 0))) {
                G.release();
                cudaGetLastError();
                return DCM_E_CUDA;
            }
            for (int q = 0; q < 6; q++) {
                G.key_ptr[q] = kp[q];
                G.key_i[q] = ki[q];
            }
            for (int q = 0; q < 3; q++) G.key_d[q] = kd[q];
        }
        if (!ok(cudaGraphLaunch(G.exec, st))) return DCM_E_CUDA;
        cudaMemcpyAsync(host_S, w.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
        if (cudaStreamSynchronize(st) != cudaSuccess) return DCM_E_CUDA;
        const long long r = host_S->rounds;  // iterations run
        if (g_prof) {
            g_prof->add(P_SETUP, 1);
            g_prof->add(P_JACOBI, (fused_ok<T>(a) ? 2 : 6) * r);
            g_prof->add(P_MATVEC, (fused_ok<T>(a) && a.fuse_mv ? 1 : 2) * r);
            g_prof->add(P_UPDATE, r);
            g_prof->add(P_OTHER, 1);
            if (post) g_prof->add(P_POST, 1);
        }
        if (launched_iters) *launched_iters = (int)r;
        return host_S->status;
    }
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
    post_launch(st);
    cudaMemcpyAsync(host_S, w.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return DCM_E_CUDA;
    if (launched_iters) *launched_iters = launched;
    return host_S->status;
}

template int solver_run<double>(SolverWork<double>&, const Dims&, double*, const double*,
                                const double*, const double*, double, int, int, int,
                                cudaStream_t, SolverScalars*, int*, double, bool);
template int solver_run<float>(SolverWork<float>&, const Dims&, float*, const float*,
                               const float*, const float*, double, int, int, int, cudaStream_t,
                               SolverScalars*, int*, double, bool);

// =============================================================================
// Mixed precision: FP32 BiCGSTAB with FP64 reliable updates
// =============================================================================
// The pressure x and the residual that decides convergence are FP64; every
// vector of the BiCGSTAB recursion and every stencil sweep is FP32, and all
// dot products are summed in FP64.  One Krylov iteration runs from start to
// convergence; whenever its recursive FP32 residual has fallen by `delta`
// since the last FP64 residual (or below the tolerance), the iteration pauses
// and the host performs an FP64 refinement step:
//     x64 += dx32, dx32 = 0;   r = b - A x64 (FP64);   r32 = r, r32/a_p
// and the recursion resumes from the replaced residual with
// rho = (r, cr) -- iterative refinement that keeps the Krylov space
// (reliable updates, Sleijpen & van der Vorst 1996).  Convergence is the
// reference's ||r|| / max(||b||, 0.01) < ptol on the FP64 residual
// (dynamics.f90:370-428).

// r = b - A x (FP64) -> r32, r32/a_p; FIRST also cr = r32 and (b,b).
// Warp tasks as in sten_task: 2 x 32 consecutive k-levels (one 16-byte
// vector per lane) of row j, marching over a.ni planes with the i
// neighbours in registers; k neighbours by shuffle and, at the warp's ends,
// one scalar load each; Neumann mirror at k = 1, kp.
template <bool FIRST>
__global__ void __launch_bounds__(256) k_ru_residual(SolverArgs a, Coef<double> c,
                                                     Coef<float> cf,
                                                     const double* __restrict__ x,
                                                     const double* __restrict__ b,
                                                     float* __restrict__ r32,
                                                     float* __restrict__ rh32,
                                                     float* __restrict__ cr32, Red2 R,
                                                     SolverScalars* S) {
    __shared__ double smem[96];
    constexpr int V = KVec<double>::V;
    const Dims& d = a.d;
    const int ip = d.ip, jp = d.jp, kp = d.kp;
    const int K = d.K, KJ = d.K * d.J;
    const int ni = a.ni, nib = (ip + ni - 1) / ni;
    double acc[3] = {0.0, 0.0, 0.0};
    const int lane = threadIdx.x;
    // a first residual, or a restart after a breakdown: cr = r
    const bool reset = FIRST || S->restart != 0;
    for (TaskIter t(blockIdx.x * blockDim.y + threadIdx.y, gridDim.x * blockDim.y, a.nkt, jp);
         t.i <= nib; t.next()) {
        const int j = 1 + t.jr, i0 = 1 + (t.i - 1) * ni, iend = min(i0 + ni - 1, ip);
        const int k0 = 1 + V * (t.kt * BX + lane);
        const bool live = k0 <= kp;
        const int nvalid = live ? min(V, kp - k0 + 1) : 0;
        const int kl = live ? k0 : 1;  // idle lanes read the column start
        const int col = kl + K * j;
        const int dsj = (j == 1 ? jp - 1 : -1) * K, dnj = (j == jp ? 1 - jp : 1) * K;
        double au[V], ad[V];
        vld(c.au + kl, au);
        vld(c.ad + kl, ad);
        const double an = ld(c.an + j), as = ld(c.as + j);
        const float anf = ld(cf.an + j), asf = ld(cf.as + j);
        float auf[V], adf[V];
#pragma unroll
        for (int q = 0; q < V; q++) {
            auf[q] = ld(cf.au + min(kl + q, kp));
            adf[q] = ld(cf.ad + min(kl + q, kp));
        }
        double xw[V], xc[V], xe[V];
        vld(x + col + KJ * (i0 == 1 ? ip : i0 - 1), xw);
        vld(x + col + KJ * i0, xc);
        for (int i = i0; i <= iend; i++) {
            const int o = col + KJ * i;
            double xs[V], xn[V], bv[V];
            vld(x + col + KJ * (i == ip ? 1 : i + 1), xe);
            vld(x + o + dsj, xs);
            vld(x + o + dnj, xn);
            vld(b + o, bv);
            if (i < iend) {  // the next plane's streamed columns into L2
                const int on = o + KJ;
                prefetch_l2(x + col + KJ * (i + 1 == ip ? 1 : i + 2));
                prefetch_l2(x + on + dsj);
                prefetch_l2(x + on + dnj);
                prefetch_l2(b + on);
            }
            double prev = __shfl_up_sync(0xffffffffu, xc[V - 1], 1);
            double next = __shfl_down_sync(0xffffffffu, xc[0], 1);
            if (lane == 0 && live && k0 > 1) prev = x[o - 1];
            if (lane == BX - 1 && live && k0 + V <= kp) next = x[o + V];
            const double ae = ld(c.ae + i), aw = ld(c.aw + i);
            // diag_ap(cf, k, j, i), left to right
            const float s4f = -ld(cf.ae + i) - ld(cf.aw + i) - anf - asf;
            float crv[V] = {0.0f, 0.0f};
            if (!reset && live) {
                if (nvalid == V) {
                    const float2 c2 = *reinterpret_cast<const float2*>(cr32 + o);
                    crv[0] = c2.x;
                    crv[1] = c2.y;
                } else {
                    crv[0] = cr32[o];
                }
            }
            float rf[V], rhf[V];
#pragma unroll
            for (int q = 0; q < V; q++) {
                const int kk = k0 + q;
                double xd = q == 0 ? prev : xc[q - 1];
                double xu = q == V - 1 ? next : xc[q + 1];
                xd = kk == 1 ? xc[q] : xd;
                xu = kk == kp ? xc[q] : xu;
                const double ap = -ae - aw - an - as - au[q] - ad[q];
                const double Ax = aw * xw[q] + ae * xe[q] + as * xs[q] + an * xn[q] +
                                  ad[q] * xd + au[q] * xu + ap * xc[q];
                const double rv = bv[q] - Ax;
                rf[q] = (float)rv;
                rhf[q] = rf[q] / (s4f - auf[q] - adf[q]);
                if (reset) crv[q] = rf[q];
                if (q < nvalid) {
                    acc[0] += bv[q] * bv[q];
                    acc[1] += rv * rv;
                    acc[2] += (double)rf[q] * (double)crv[q];
                }
            }
            if (live) {
                if (nvalid == V) {
                    *reinterpret_cast<float2*>(r32 + o) = make_float2(rf[0], rf[1]);
                    *reinterpret_cast<float2*>(rh32 + o) = make_float2(rhf[0], rhf[1]);
                    if (reset) *reinterpret_cast<float2*>(cr32 + o) = make_float2(rf[0], rf[1]);
                } else {
                    r32[o] = rf[0];
                    rh32[o] = rhf[0];
                    if (reset) cr32[o] = rf[0];
                }
            }
#pragma unroll
            for (int q = 0; q < V; q++) {
                xw[q] = xc[q];
                xc[q] = xe[q];
            }
        }
    }
    block_reduce<R_SUM, 3>(acc, smem);
    double s[3];
    if (reduce2<3>(acc, R, smem, s) && threadIdx.x == 0 && threadIdx.y == 0) {
        if (FIRST) {
            double sc = sqrt(s[0]);
            sc = sc > 0.01 ? sc : 0.01;  // dynamics.f90:370-371
            S->sc_err = sc;
            S->it = 0;
            S->status = 0;
            S->updates = 0;
            S->rounds = 0;
            S->cycles = 0;
            S->ru_runs = 0;
            S->restarts = 0;
            S->fresh = 0;
        }
        const double err = sqrt(s[1]) / S->sc_err;
        S->err = err;
        S->ru_norm = sqrt(s[1]);
        S->pause = 0;
        S->done = 0;
        S->early = 0;
        S->cycle_it = 0;
        if (err < a.tol) {
            S->done = 1;
            S->early = FIRST ? 1 : 0;
        } else if (!(err == err)) {
            S->status = DCM_E_NONFINITE;
            S->done = 1;
        } else if (!FIRST && S->updates >= a.max_updates) {
            S->status = DCM_E_NOCONV;
            S->done = 1;
        } else {
            if (reset) {
                // BiCGSTAB from r with cr = r: alf = omg = nrm = 1 (:385-387);
                // after a breakdown the next iteration also starts with p = v1 = 0
                S->alf = 1.0;
                S->omg = 1.0;
                S->nrm = 1.0;
                S->crnorm = s[2];
                if (!FIRST) {
                    S->restarts = S->restarts + 1;
                    S->fresh = 1;
                }
            }
            S->rho = s[2];  // (r, cr) of the replaced residual
            S->bet = (S->rho / S->nrm) * (S->alf / S->omg);
            if (!FIRST) S->updates = S->updates + 1;
        }
        S->restart = 0;
    }
}

// x (FP64) += dx (FP32); dx = 0 (interior)
__global__ void __launch_bounds__(256) k_ru_add(Dims d, double* __restrict__ x,
                                                float* __restrict__ dx,
                                                const SolverScalars* S) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const int o = d.at(k, j, i);
    // after a non-finite breakdown the correction since the last update is
    // dropped (x64 keeps its last FP64-checked value)
    if (S->restart != 2) x[o] = x[o] + (double)dx[o];
    dx[o] = 0.0f;
}

// reliable-update controls of the FP32 scalars (start of a mixed solve)
__global__ void k_ru_begin(SolverScalars* S, double delta) {
    S->ru = 1;
    S->delta = delta;
    S->pause = 0;
}

// end of a mixed solve: the FP32 scalars back to plain mode, the outcome into
// the FP64 scalars that the halo fix-up (k_bicg_post) reads
__global__ void k_ru_end(SolverScalars* Sin, SolverScalars* Sout) {
    Sin->ru = 0;
    Sout->early = Sin->early;
    Sout->status = Sin->status;
    Sout->it = Sin->it;
    Sout->err = Sin->err;
}

int refine_run(SolverWork<float>& wf, SolverWork<double>& wd, const Dims& d, double* x,
               const double* b, const float* sw, const double* dzn, float* dx, double tol,
               double delta, int itmax, int max_updates, cudaStream_t st,
               SolverScalars* hS_out, SolverScalars* hS_in, RefineStats* rs) {
    SolverArgs a;
    a.d = d;
    a.itmax = itmax;
    a.tol = tol;
    a.sc_floor = 0.01;
    a.nkt = kchunks<double>(d);  // vector warp tasks of the FP64 residual
    a.max_updates = max_updates;
    a.max_cycle = 250;
    a.by = wf.by;
    a.tasks = wf.tasks;
    a.max_blocks = wf.max_blocks;
    a.ni = 4;                      // planes a warp task of the FP64 residual marches over
    a.fuse = 0;
    no_cheb(a);
    SolverArgs af = a;             // vector warp tasks of the FP32 iterations
    af.vw = wf.vw;
    af.nkt = kchunks<float>(d, af.vw);
    af.ni = wf.ni >= 1 ? wf.ni : 1;
    af.fuse = wf.fuse;
    af.fuse_mv = wf.fuse == 2 ? 1 : 0;
    if (wf.cheb) {
        af.cheb = 1;
        cheb_weights(wf.cheb_lo, af.cw);
    }
    Coef<double> cd;
    cd.ae = wd.ae; cd.aw = wd.aw; cd.an = wd.an; cd.as = wd.as; cd.au = wd.au; cd.ad = wd.ad;
    const Coef<float> cf = coef_of(wf);
    static const int gfull = persistent_grid(k_ru_residual<false>);
    const int g = red_grid(a, gfull, a.nkt, a.ni);
    const dim3 gi = interior_grid(d, d.kp), bl(BX, BY);
    auto begin = [&](cudaStream_t s) {
        cudaMemsetAsync(dx, 0, d.n() * sizeof(float), s);
        k_ru_begin<<<1, 1, 0, s>>>(wf.S, delta);
        ProfScope ps(P_SETUP, s);
        k_ru_residual<true><<<g, bl, 0, s>>>(a, cd, cf, x, b, wf.r, wf.rh, wf.cr, wd.red, wf.S);
    };
    auto update = [&](cudaStream_t s) {  // x64 += dx32; FP64 residual
        {
            ProfScope ps(P_UPDATE, s);
            k_ru_add<<<gi, bl, 0, s>>>(d, x, dx, wf.S);
        }
        ProfScope ps(P_SETUP, s);
        k_ru_residual<false><<<g, bl, 0, s>>>(a, cd, cf, x, b, wf.r, wf.rh, wf.cr, wd.red, wf.S);
    };
    auto finish = [&](cudaStream_t s) {
        {
            // the correction accumulated since the last update (zero after one)
            ProfScope ps(P_UPDATE, s);
            k_ru_add<<<gi, bl, 0, s>>>(d, x, dx, wf.S);
        }
        k_ru_end<<<1, 1, 0, s>>>(wf.S, wd.S);
        ProfScope ps(P_POST, s);
        k_bicg_post<double, float><<<gi, bl, 0, s>>>(d, x, sw, dzn, wd.S, 1);
    };
    const int max_rounds = wf.round_budget > 0 ? wf.round_budget : itmax + max_updates + 1;
    // the whole mixed solve into the graph being captured on `s0`:
    //   WHILE (not done) {                           one FP64 update cycle
    //       WHILE (not done, not paused) { FP32 iteration }
    //       IF (paused) { reliable update }
    //   }
    // The update kernel of each FP32 iteration sets the inner condition, so
    // an iteration is its five (or nine) kernels and nothing else.  Both
    // loops are bounded: a cycle starts with pause = 0, so every cycle that
    // does not end the solve counts an iteration against max_rounds.
    auto emit = [&](cudaStream_t s0, SolveGraph& G) {
        if (!side_streams(G)) return false;
        CaptureGuard cgd;
        cudaGraphConditionalHandle ho{};
        cudaGraph_t body[1] = {nullptr};
        begin(s0);
        bool good = capture_cond_handle(s0, &ho, 0);
        if (good) k_outer_cond<<<1, 1, 0, s0>>>(ho, wf.S);
        good = good && capture_cond_node(s0, ho, cudaGraphCondTypeWhile, 1, body);
        good = good && capture_into(G.side[0], body[0], [&](cudaStream_t s) {
                   cudaGraphConditionalHandle hi{}, hb{};
                   cudaGraph_t in[1] = {nullptr}, br[1] = {nullptr};
                   SolverArgs ai = af;
                   bool g2 = capture_cond_handle(s, &hi, 0);
                   if (g2) k_cycle_start<<<1, 1, 0, s>>>(hi, wf.S, max_rounds);
                   g2 = g2 && capture_cond_node(s, hi, cudaGraphCondTypeWhile, 1, in);
                   ai.cond = hi;
                   ai.cond_max = max_rounds;
                   ai.pdl = g_pdl_graphs && wf.pdl;
                   g2 = g2 && capture_into(G.side[1], in[0], [&](cudaStream_t s2) {
                            for (int n = 0; n < ITERS_PER_BODY; n++)
                                launch_iteration<float>(ai, cf, wf, dx, s2);
                        });
                   g2 = g2 && capture_cond_handle(s, &hb, 0);
                   if (g2) k_branch_pause<<<1, 1, 0, s>>>(hb, wf.S);
                   g2 = g2 && capture_cond_node(s, hb, cudaGraphCondTypeIf, 1, br);
                   g2 = g2 && capture_into(G.side[1], br[0], update);
                   k_outer_cond<<<1, 1, 0, s>>>(ho, wf.S);
                   if (!g2) good = false;
               });
        finish(s0);
        return good && cudaPeekAtLastError() == cudaSuccess;
    };
    if (wf.graph && wf.emit) return emit(st, *wf.graph) ? DCM_OK : DCM_E_CUDA;
    const bool use_graph = wf.graph && !(g_prof && g_prof->on);
    if (use_graph) {
        SolveGraph& G = *wf.graph;
        const void* kp[6] = {x, b, sw, dzn, dx, wf.S};
        const double kd[3] = {tol, delta, af.cheb ? wf.cheb_lo : 0.0};
        const int shape = af.by + 16 * af.tasks + 256 * af.ni + 16384 * af.fuse +
                          65536 * af.cheb + 131072 * (wf.pdl ? 1 : 0) + 262144 * af.vw;
        const int ki[6] = {itmax, max_updates, 1 + 2 * max_rounds, 16 * shape,
                           d.ip * 4096 + d.jp, d.kp};
        if (!G.matches(kp, kd, ki)) {
            G.release();
            bool good = ok(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed));
            if (good) good = emit(st, G);
            cudaGraph_t gr = nullptr;
            const bool ended = ok(cudaStreamEndCapture(st, &gr));
            G.graph = gr;
            if (!good || !ended || !ok(cudaGraphInstantiate(&G.exec, gr, 0))) {
                G.release();
                cudaGetLastError();
                return DCM_E_CUDA;
            }
            for (int q = 0; q < 6; q++) {
                G.key_ptr[q] = kp[q];
                G.key_i[q] = ki[q];
            }
            for (int q = 0; q < 3; q++) G.key_d[q] = kd[q];
        }
        if (!ok(cudaGraphLaunch(G.exec, st))) return DCM_E_CUDA;
    } else {
        begin(st);
        int launched = 0;
        for (int round = 0;; round++) {
            cudaMemcpyAsync(hS_in, wf.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
            if (cudaStreamSynchronize(st) != cudaSuccess) return DCM_E_CUDA;
            if (hS_in->done || round > max_rounds) break;
            if (hS_in->pause) {
                update(st);
                continue;
            }
            if (launched >= itmax) break;
            for (int q = 0; q < 4 && launched < itmax; q++, launched++)
                launch_iteration<float>(af, cf, wf, dx, st);
            if (cudaGetLastError() != cudaSuccess) return DCM_E_CUDA;
        }
        finish(st);
    }
    cudaMemcpyAsync(hS_in, wf.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(hS_out, wd.S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, st);
    if (cudaStreamSynchronize(st) != cudaSuccess) return DCM_E_CUDA;
    int status = hS_out->status;
    if (status == DCM_OK && !hS_in->done) status = DCM_E_NOCONV;  // host loop ran out
    if (use_graph && g_prof) {
        // iterations, reliable updates and cycles the graph ran
        const long long itr = hS_in->rounds, u = hS_in->ru_runs, cyc = hS_in->cycles;
        g_prof->add(P_SETUP, u + 1);
        g_prof->add(P_JACOBI, (fused_ok<float>(af) ? 2 : 6) * itr);
        g_prof->add(P_MATVEC, (fused_ok<float>(af) && af.fuse_mv ? 1 : 2) * itr);
        g_prof->add(P_UPDATE, itr + u + 1);
        g_prof->add(P_POST, 1);
        g_prof->add(P_OTHER, 3 * cyc + 3);
    }
    if (rs) {
        rs->outer = hS_in->updates;
        rs->inner = hS_in->it;
        rs->restarts = hS_in->restarts;
        rs->err = hS_in->err;
    }
    return status;
}

}  // namespace dcm
