// dcm_column.cu -- the PAMM microphysics' sedimentation transport on the GPU:
// mpdata_vec_1d with first_order_upstream_1d (pamm/sfvt/advection_1d.F90:35-74,
// 463-778) for many independent columns at once, each with the caller's
// sub-stepping loop (pamm/microphysics.f90:3139-3145, 3158-3164, 3177-3183:
// n_step passes of dt/n_step, n_step from the column's largest fall speed).
//
// One warp per column.  The column's fields, a copy of the first field (the
// limiter's psi), the input and two working velocity columns, a flux buffer
// and the limiter's beta_up / beta_down sit in shared memory; every statement
// of the Fortran is a pass of the 32 lanes over the levels, separated by
// __syncwarp.  Reductions over k (minval, the positivity test's sum) are warp
// shuffles.  All arithmetic is FP64 in the reference's order of terms.
#include <algorithm>

#include "dcm_internal.h"

namespace {

constexpr double COL_SMALL = 1e-60;  // pamm/sfvt/advection_1d.F90:18
constexpr int COL_WARPS = 4;         // columns per block at most

struct ColArgs {
    int ncol, kp, nq, l_h, r_h, nw, npsi, per_warp;  // per_warp: doubles of shared memory
    int mstride, kord, monotone, neumann;
    const double *dt, *dz, *dzn, *rhoa, *rhoan, *w;
    const int* nsub;
    double* psi;
};

__device__ __forceinline__ double wmin(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_xor_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double wsum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// first_order_upstream_1d (:35-74) on one field p (level-0 pointer), the new
// values through tmp so that every lane reads the old neighbours
__device__ void col_upstream(double dt, const double* dzn, const double* rhoa,
                             const double* rhoan, int kp, const double* w, double* p,
                             int neumann, double* tmp, int lane) {
    for (int k = 1 + lane; k <= kp; k += 32) {
        const double den = 2.0 * dzn[k] * rhoan[k];
        const double wk = w[k], wm = w[k - 1];
        double fr = ((wk + fabs(wk)) * rhoa[k] * p[k] + (wk - fabs(wk)) * rhoa[k] * p[k + 1]) *
                    dt / den;
        double fl = ((wm + fabs(wm)) * rhoa[k - 1] * p[k - 1] +
                     (wm - fabs(wm)) * rhoa[k - 1] * p[k]) *
                    dt / den;
        if (neumann == 1) {  // :65-67, in the reference's order
            if (k == 1) fl = fr;
            if (k == kp) fr = fl;
        } else if (neumann == 2) {  // :68-70
            if (k == 1) fl = -fr;
            if (k == kp) fr = -fl;
        }
        tmp[k] = p[k] - (fr - fl);  // :73
    }
    __syncwarp();
    for (int k = 1 + lane; k <= kp; k += 32) p[k] = tmp[k];
    __syncwarp();
    if (lane == 0) {  // halos after each pass (:755-761)
        p[0] = 0.0;
        p[kp + 1] = 0.0;
    }
    __syncwarp();
}

// halos of a working velocity column (:656-657, :732-733)
__device__ __forceinline__ void col_w_halos(double* w, int kp, int lane) {
    if (lane == 0) {
        w[0] = w[1];
        w[kp] = w[kp - 1];
        w[kp + 1] = w[kp - 1];
    }
    __syncwarp();
}

// one call of mpdata_vec_1d (:463-778) on the column in shared memory
__device__ void col_mpdata(const ColArgs& a, double dt, const double* dz, const double* dzn,
                           const double* rhoa, const double* rhoan, const double* win,
                           double* psi, double* store, double* ws1, double* ws2, double* tmp,
                           double* bup, double* bdn, double* ming, int lane) {
    const int kp = a.kp, nq = a.nq, npsi = a.npsi, nw = a.nw;
    const int op = a.r_h - 1;
    auto P = [&](int n) { return psi + (size_t)n * npsi + op; };
    // positive definite (:507-516): minval over the interior, shift every
    // element (halos included)
    for (int n = 0; n < nq; n++) {
        double* p = P(n);
        double m = INFINITY;
        for (int k = 1 + lane; k <= kp; k += 32) m = fmin(m, p[k]);
        m = wmin(m);
        if (lane == 0) ming[n] = m;
        for (int k = -a.r_h + 1 + lane; k <= kp + a.r_h; k += 32) p[k] = p[k] - m;
    }
    __syncwarp();
    // :518-529; the interior sum is a shuffle tree here (index order in the
    // reference): it only meets the 1e-60 threshold, and the terms are >= 0
    double s = 0.0;
    for (int k = 1 + lane; k <= kp; k += 32) s += P(0)[k];
    s = wsum(s);
    if (s < COL_SMALL) {
        for (int n = 0; n < nq; n++)
            for (int k = -a.r_h + 1 + lane; k <= kp + a.r_h; k += 32) P(n)[k] += ming[n];
        __syncwarp();
        return;
    }
    const int ow = a.l_h - 1;
    const bool anti = a.kord > 1;
    double* w1 = anti ? ws1 + ow : nullptr;  // level-0 views of the working velocities
    double* w2 = anti ? ws2 + ow : nullptr;
    if (anti)
        for (int i = lane; i < nw; i += 32) ws2[i] = 0.0;  // :530 (read only when kord > 1)
    const double* wt = win + ow;                        // :534-535
    double* wt_sav = w1;
    const double* ps = anti ? store + op : nullptr;  // the limiter's psi (:542-545)
    double* po = P(0);              // psi_old (:547)
    if (a.kord > 1)
        for (int i = lane; i < npsi; i += 32) store[i] = psi[i];
    __syncwarp();
    int it2 = 0;
    for (int it = 1; it <= a.kord; it++) {
        if (it > 1) {  // antidiffusive velocities (:553-635)
            it2 = it2 + 1;
            for (int k = 1 + lane; k <= kp; k += 32) {
                const double g_bar3 = 0.5 * (rhoan[k] + rhoan[k + 1]);
                const double wk = wt[k];
                double v = (fabs(wk) * dz[k] - dt * (rhoa[k] / g_bar3) * wk * wk) *
                               (po[k + 1] - po[k]) / (po[k + 1] + po[k] + COL_SMALL) / dzn[k] -
                           0.0;
                v = v - 0.25 * dt * wk *
                            ((rhoa[k + 1] * wt[k + 1] - rhoa[k - 1] * wt[k - 1]) / dz[k - 1] +
                             0.0) /
                            g_bar3;
                wt_sav[k] = v;
            }
            __syncwarp();
            double* nwt = (it2 % 2 == 1) ? w1 : w2;  // :641-648
            wt_sav = (it2 % 2 == 1) ? w2 : w1;
            col_w_halos(nwt, kp, lane);
            wt = nwt;
        }
        if (it > 1 && a.monotone) {  // the NFT limiter (:666-745)
            it2 = it2 + 1;
            double* bu = bup + op;
            double* bd = bdn + op;
            for (int k = 1 + lane; k <= kp; k += 32) {
                const double mx = fmax(fmax(fmax(ps[k - 1], ps[k]), fmax(ps[k + 1], po[k - 1])),
                                       fmax(po[k], po[k + 1]));
                const double mn = fmin(fmin(fmin(ps[k - 1], ps[k]), fmin(ps[k + 1], po[k - 1])),
                                       fmin(po[k], po[k + 1]));
                const double denom1 = dt *
                                          (fmax(wt[k - 1], 0.0) * rhoa[k - 1] * po[k - 1] -
                                           fmin(wt[k], 0.0) * rhoa[k] * po[k + 1]) /
                                          dzn[k] +
                                      COL_SMALL;
                const double denom2 = dt *
                                          (fmax(wt[k], 0.0) * rhoa[k] * po[k] -
                                           fmin(wt[k - 1], 0.0) * rhoa[k - 1] * po[k]) /
                                          dzn[k] +
                                      COL_SMALL;
                bu[k] = rhoan[k] * (mx - po[k]) / denom1;
                bd[k] = rhoan[k] * (po[k] - mn) / denom2;
            }
            for (int k = 1 - a.r_h + lane; k <= 0; k += 32) bu[k] = bd[k] = 0.0;  // :698-701
            for (int k = kp + 1 + lane; k <= kp + a.r_h; k += 32) bu[k] = bd[k] = 0.0;
            __syncwarp();
            for (int k = 1 + lane; k <= kp; k += 32)  // :709-715
                wt_sav[k] = fmin(fmin(1.0, bd[k]), bu[k + 1]) * fmax(wt[k], 0.0) +
                            fmin(fmin(1.0, bu[k]), bd[k + 1]) * fmin(wt[k], 0.0);
            __syncwarp();
            wt_sav = w1;  // :720-721: the limited velocities are in w_store2
            col_w_halos(w2, kp, lane);
            wt = w2;
        }
        for (int n = 0; n < nq; n++)  // :748-764
            col_upstream(dt, dzn, rhoa, rhoan, kp, wt, P(n), a.neumann, tmp + op, lane);
    }
    for (int n = 0; n < nq; n++)  // :775-777
        for (int k = -a.r_h + 1 + lane; k <= kp + a.r_h; k += 32) P(n)[k] += ming[n];
    __syncwarp();
}

// 8 blocks of 4 warps per SM (64 registers): the donor-cell form (the
// sedimentation calls) took 0.237 ms for 65,536 columns of 128 levels and two
// fields at this bound, 0.267 ms at 6 blocks and 0.361 ms unbounded (126
// registers, 4 blocks)
__global__ void __launch_bounds__(32 * COL_WARPS, 8) k_column_mpdata(ColArgs a) {
    extern __shared__ double col_sm[];
    const int wib = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int c = blockIdx.x * (blockDim.x >> 5) + wib;
    if (c >= a.ncol) return;  // the whole warp: no block-wide barrier follows
    // [nq][npsi] fields, then with kord > 1 the limiter's psi, the input and
    // the two working velocities, the flux buffer, beta_up, beta_down, the
    // minima; with kord <= 1 (the donor cell alone) the flux buffer, the
    // input velocity and the minima only, so that more columns fit an SM
    double* psi = col_sm + (size_t)wib * a.per_warp;
    double* rest = psi + (size_t)a.nq * a.npsi;
    double *store = nullptr, *ws1 = nullptr, *ws2 = nullptr, *bup = nullptr, *bdn = nullptr;
    double *tmp, *win, *ming;
    if (a.kord > 1) {
        store = rest;
        win = store + a.npsi;
        ws1 = win + a.nw;
        ws2 = ws1 + a.nw;
        tmp = ws2 + a.nw;
        bup = tmp + a.npsi;
        bdn = bup + a.npsi;
        ming = bdn + a.npsi;
    } else {
        tmp = rest;
        win = tmp + a.npsi;
        ming = win + a.nw;
    }
    double* gpsi = a.psi + (size_t)c * a.nq * a.npsi;
#pragma unroll 4
    for (int i = lane; i < a.nq * a.npsi; i += 32) psi[i] = gpsi[i];
#pragma unroll 4
    for (int i = lane; i < a.nw; i += 32) win[i] = a.w[(size_t)c * a.nw + i];
    if (ws1)
        for (int i = lane; i < a.nw; i += 32) ws1[i] = 0.0;
    __syncwarp();
    const size_t mo = (size_t)c * a.mstride + (a.l_h - 1);
    const double *dz = a.dz + mo, *dzn = a.dzn + mo, *rhoa = a.rhoa + mo, *rhoan = a.rhoan + mo;
    const int ns = a.nsub ? max(a.nsub[c], 1) : 1;
    const double dt = a.dt[c] / (double)ns;
    for (int s = 0; s < ns; s++)
        col_mpdata(a, dt, dz, dzn, rhoa, rhoan, win, psi, store, ws1, ws2, tmp, bup, bdn, ming,
                   lane);
#pragma unroll 4
    for (int i = lane; i < a.nq * a.npsi; i += 32) gpsi[i] = psi[i];
}

}  // namespace

// shape checks shared by both entry points; fills the launch shape
static int column_shape(int ncol, int kp, int nq, int l_h, int r_h, int metric_stride,
                        int kord, int neumann, ColArgs& a, int& warps, size_t& smem) {
    if (ncol < 0 || kp < 1 || nq < 1 || l_h < 1 || r_h < 1 || kord < 0 || neumann < 0 ||
        neumann > 2)
        return DCM_E_ARG;
    const int nw = kp + l_h + r_h, npsi = kp + 2 * r_h;
    if (metric_stride != 0 && metric_stride != nw) return DCM_E_ARG;
    const int per_warp = kord > 1 ? (nq + 4) * npsi + 3 * nw + nq : (nq + 1) * npsi + nw + nq;
    const size_t warp_bytes = (size_t)per_warp * sizeof(double);
    constexpr size_t max_bytes = 200 * 1024;
    if (warp_bytes > max_bytes) return DCM_E_ARG;  // a column too tall for shared memory
    warps = std::max(1, std::min<int>(COL_WARPS, (int)(max_bytes / warp_bytes)));
    smem = (size_t)warps * warp_bytes;
    a = ColArgs{};
    a.ncol = ncol;
    a.kp = kp;
    a.nq = nq;
    a.l_h = l_h;
    a.r_h = r_h;
    a.nw = nw;
    a.npsi = npsi;
    a.per_warp = per_warp;
    a.mstride = metric_stride;
    a.kord = kord;
    a.neumann = neumann;
    return DCM_OK;
}

static bool column_launch(const ColArgs& a, int warps, size_t smem, cudaStream_t st) {
    if (smem > 48 * 1024 &&
        cudaFuncSetAttribute(k_column_mpdata, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem) != cudaSuccess)
        return false;
    k_column_mpdata<<<(a.ncol + warps - 1) / warps, 32 * warps, smem, st>>>(a);
    return cudaPeekAtLastError() == cudaSuccess;
}

extern "C" int dcm_mpdata_vec_1d_device(int ncol, int kp, int nq, int l_h, int r_h,
                                        const double* dt, const int* nsub, const double* dz,
                                        const double* dzn, const double* rhoa,
                                        const double* rhoan, int metric_stride,
                                        const double* w, double* psi, int kord, int monotone,
                                        int neumann, void* stream) {
    ColArgs a;
    int warps = 1;
    size_t smem = 0;
    const int st = column_shape(ncol, kp, nq, l_h, r_h, metric_stride, kord, neumann, a,
                                warps, smem);
    if (st != DCM_OK || ncol == 0) return st;
    if (!dt || !dz || !dzn || !rhoa || !rhoan || !w || !psi) return DCM_E_ARG;
    if (cudaPeekAtLastError() != cudaSuccess) return DCM_E_CUDA;  // not ours to clear
    a.monotone = monotone ? 1 : 0;
    a.dt = dt;
    a.nsub = nsub;
    a.dz = dz;
    a.dzn = dzn;
    a.rhoa = rhoa;
    a.rhoan = rhoan;
    a.w = w;
    a.psi = psi;
    return column_launch(a, warps, smem, (cudaStream_t)stream) ? DCM_OK : DCM_E_CUDA;
}

extern "C" int dcm_mpdata_vec_1d(int ncol, int kp, int nq, int l_h, int r_h, const double* dt,
                                 const int* nsub, const double* dz, const double* dzn,
                                 const double* rhoa, const double* rhoan, int metric_stride,
                                 const double* w, double* psi, int kord, int monotone,
                                 int neumann) {
    ColArgs a;
    int warps = 1;
    size_t smem = 0;
    const int st = column_shape(ncol, kp, nq, l_h, r_h, metric_stride, kord, neumann, a,
                                warps, smem);
    if (st != DCM_OK || ncol == 0) return st;
    if (!dt || !dz || !dzn || !rhoa || !rhoan || !w || !psi) return DCM_E_ARG;
    if (nsub)
        for (int c = 0; c < ncol; c++)
            if (nsub[c] < 1) return DCM_E_ARG;
    const int nw = a.nw, npsi = a.npsi;
    const size_t nmet = (size_t)(metric_stride ? ncol : 1) * nw;
    const size_t bytes_dt = (size_t)ncol * sizeof(double), bytes_ns = (size_t)ncol * sizeof(int);
    const size_t bytes_met = nmet * sizeof(double), bytes_w = (size_t)ncol * nw * sizeof(double);
    const size_t bytes_psi = (size_t)ncol * nq * npsi * sizeof(double);
    const size_t al = 256;
    auto up = [&](size_t b) { return (b + al - 1) / al * al; };
    const size_t total = up(bytes_dt) + up(bytes_ns) + 4 * up(bytes_met) + up(bytes_w) +
                         up(bytes_psi);
    char* buf = nullptr;
    if (cudaMalloc(&buf, total) != cudaSuccess) return DCM_E_CUDA;
    size_t off = 0;
    auto take = [&](size_t b) {
        char* p = buf + off;
        off += up(b);
        return p;
    };
    double* d_dt = (double*)take(bytes_dt);
    int* d_ns = (int*)take(bytes_ns);
    double* d_met[4];
    for (double*& m : d_met) m = (double*)take(bytes_met);
    double* d_w = (double*)take(bytes_w);
    double* d_psi = (double*)take(bytes_psi);
    const double* h_met[4] = {dz, dzn, rhoa, rhoan};
    bool good = cudaMemcpy(d_dt, dt, bytes_dt, cudaMemcpyHostToDevice) == cudaSuccess;
    if (good && nsub) good = cudaMemcpy(d_ns, nsub, bytes_ns, cudaMemcpyHostToDevice) == cudaSuccess;
    for (int q = 0; q < 4 && good; q++)
        good = cudaMemcpy(d_met[q], h_met[q], bytes_met, cudaMemcpyHostToDevice) == cudaSuccess;
    if (good) good = cudaMemcpy(d_w, w, bytes_w, cudaMemcpyHostToDevice) == cudaSuccess;
    if (good) good = cudaMemcpy(d_psi, psi, bytes_psi, cudaMemcpyHostToDevice) == cudaSuccess;
    a.monotone = monotone ? 1 : 0;
    a.dt = d_dt;
    a.nsub = nsub ? d_ns : nullptr;
    a.dz = d_met[0];
    a.dzn = d_met[1];
    a.rhoa = d_met[2];
    a.rhoan = d_met[3];
    a.w = d_w;
    a.psi = d_psi;
    if (good) good = column_launch(a, warps, smem, 0);
    if (good) good = cudaMemcpy(psi, d_psi, bytes_psi, cudaMemcpyDeviceToHost) == cudaSuccess;
    const bool freed = cudaFree(buf) == cudaSuccess;
    return good && freed ? DCM_OK : DCM_E_CUDA;
}
