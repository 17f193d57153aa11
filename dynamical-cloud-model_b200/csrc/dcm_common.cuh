// dcm_common.cuh -- layout, halo semantics and reductions shared by every
// kernel of the B200 dynamical core.
//
// Layout in HBM: the reference's own Fortran column-major array
// a(0:kp+1, 0:jp+1, 0:ip+1) (halo 1, main.f90:80-81), k fastest.  Keeping
// the caller's layout on the device makes every host<->device copy one
// contiguous cudaMemcpy and lets a warp read 32 consecutive k-levels of one
// column (256 B for FP64, 128 B for FP32) in one coalesced access.
//
// Halo semantics.  The single-rank exchanges of mpi_module.f90 reduce to
// three rules, which the kernels apply by having the thread that produces an
// interior value also write every halo cell that is a copy of it
// ("images").  This replaces a separate halo pass after each stage.
//   exchange_full(lbc,ubc)    (mpi_module.f90:926-1271): every halo cell is
//       the fully periodic image of an interior cell, except the interior of
//       the top / bottom planes, which hold ubc / lbc.
//   exchange_along_dim(lbc,ubc) (:700-910): x and y faces for k = 1..kp are
//       periodic images; the whole top / bottom planes are ubc / lbc;
//       vertical edges are left alone.
//   exchange_along_dim_wo     (:1285-1494): x and y faces for k = 1..kp.
//   exchange_full_wo          (:1511-1855): as exchange_full, but the
//       interior of the top / bottom planes is left as it was.
#pragma once
#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

namespace dcm {

struct Dims {
    int ip, jp, kp;  // interior extents
    int K, J, I;     // kp+2, jp+2, ip+2
    __host__ __device__ __forceinline__ int at(int k, int j, int i) const {
        return k + K * (j + J * i);
    }
    __host__ __device__ __forceinline__ size_t n() const {
        return (size_t)K * J * I;
    }
};

// Dense Fortran layout a(0:kp+1, 0:jp+1, 0:ip+1): the layout of host arrays
// and of device arrays a caller owns.
inline Dims make_dims(int ip, int jp, int kp) {
    Dims d;
    d.ip = ip; d.jp = jp; d.kp = kp;
    d.K = kp + 2; d.J = jp + 2; d.I = ip + 2;
    return d;
}

// Pitched device layout of the fields a handle owns.  The leading (k)
// dimension is padded to K = round_up(kp + 4, 8) and every field pointer
// sits FIELD_SHIFT elements past a 256-byte aligned allocation, so element
// (1, j, i) of every column starts on a 32-byte boundary (64 bytes for
// double).  Stencil kernels then move 16-byte vectors of consecutive
// k-levels; a vector that starts at k <= kp ends at k <= kp + 3 < K, inside
// its own column.  A field takes n() + FIELD_PAD elements.
constexpr int FIELD_ALIGN = 8;
constexpr int FIELD_SHIFT = FIELD_ALIGN - 1;
constexpr int FIELD_PAD = FIELD_ALIGN;
inline Dims make_dims_pitched(int ip, int jp, int kp) {
    Dims d = make_dims(ip, jp, kp);
    d.K = (kp + 4 + FIELD_ALIGN - 1) / FIELD_ALIGN * FIELD_ALIGN;
    return d;
}

// 1-D metrics on the device, halo-inclusive, in the field precision T.
template <typename T>
struct Metrics {
    const T *dx, *dxn, *dy, *dyn, *dz, *dzn, *rhoa, *rhoan, *theta, *thetan;
};

template <typename T>
__device__ __forceinline__ T ld(const T* p) { return __ldg(p); }

// periodic wrap of a halo index onto the interior 1..n
__device__ __forceinline__ int wrapc(int c, int n) {
    return c < 1 ? c + n : (c > n ? c - n : c);
}

// list the images of interior coordinate c (1..n) along one axis:
// itself, n+1 if c == 1, 0 if c == n
__device__ __forceinline__ int images(int c, int n, int* out) {
    int m = 0;
    out[m++] = c;
    if (c == 1) out[m++] = n + 1;
    if (c == n) out[m++] = 0;
    return m;
}

// ---- exchange_full images of v (interior cell k,j,i) -------------------
// WO = true gives exchange_full_wo (mpi_module.f90:1511-1855): the same
// images, except that the interior of the top / bottom planes is left as it
// was (lbc / ubc unused).
template <typename T, bool WO = false>
__device__ __forceinline__ void put_full(T* __restrict__ a, const Dims& d,
                                         int k, int j, int i, T v, T lbc,
                                         T ubc) {
    a[d.at(k, j, i)] = v;
    const bool edge = (i == 1) | (i == d.ip) | (j == 1) | (j == d.jp) |
                      (k == 1) | (k == d.kp);
    if (!edge) return;
    int ks[3], js[3], is[3];
    const int nk = images(k, d.kp, ks), nj = images(j, d.jp, js),
              ni = images(i, d.ip, is);
    for (int a3 = 0; a3 < nk; a3++)
        for (int b3 = 0; b3 < nj; b3++)
            for (int c3 = 0; c3 < ni; c3++) {
                if ((a3 | b3 | c3) == 0) continue;
                const int kk = ks[a3], jj = js[b3], ii = is[c3];
                T val = v;
                if ((kk == 0 || kk == d.kp + 1) && b3 == 0 && c3 == 0) {
                    if (WO) continue;
                    val = (kk == 0) ? lbc : ubc;
                }
                a[d.at(kk, jj, ii)] = val;
            }
}

// images in j and i only, at a given level kk (used for plane fills)
template <typename T>
__device__ __forceinline__ void put_plane_images(T* __restrict__ a,
                                                 const Dims& d, int kk, int j,
                                                 int i, T v) {
    int js[3], is[3];
    const int nj = images(j, d.jp, js), ni = images(i, d.ip, is);
    for (int b3 = 0; b3 < nj; b3++)
        for (int c3 = 0; c3 < ni; c3++) a[d.at(kk, js[b3], is[c3])] = v;
}

// ---- exchange_along_dim_wo images (faces, k = 1..kp) --------------------
template <typename T>
__device__ __forceinline__ void put_wo(T* __restrict__ a, const Dims& d,
                                       int k, int j, int i, T v) {
    a[d.at(k, j, i)] = v;
    if (i == 1) a[d.at(k, j, d.ip + 1)] = v;
    if (i == d.ip) a[d.at(k, j, 0)] = v;
    if (j == 1) a[d.at(k, d.jp + 1, i)] = v;
    if (j == d.jp) a[d.at(k, 0, i)] = v;
}

// ---- exchange_along_dim images: faces + constant top / bottom planes ----
template <typename T>
__device__ __forceinline__ void put_dim(T* __restrict__ a, const Dims& d,
                                        int k, int j, int i, T v, T lbc,
                                        T ubc) {
    put_wo(a, d, k, j, i, v);
    if (k == 1) put_plane_images(a, d, d.kp + 1, j, i, ubc);
    if (k == d.kp) put_plane_images(a, d, 0, j, i, lbc);
}

// ---- launch geometry -----------------------------------------------------
// Interior kernels: threadIdx.x -> k (32 consecutive levels, one warp),
// threadIdx.y -> j, blockIdx.z -> i.
constexpr int BX = 32, BY = 8;

inline dim3 interior_grid(const Dims& d, int k_extent) {
    return dim3((k_extent + BX - 1) / BX, (d.jp + BY - 1) / BY, d.ip);
}
inline dim3 full_grid(const Dims& d) {
    return dim3((d.kp + 2 + BX - 1) / BX, (d.J + BY - 1) / BY, d.I);
}

// ---- deterministic reductions -------------------------------------------
// Block partials in fixed order, then the last block to finish reduces the
// partials in fixed order (threadfence + ticket).  Same grid -> same bits.
__device__ __forceinline__ double warp_sum(double v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_min(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmin(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}
__device__ __forceinline__ double warp_max(double v) {
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_down_sync(0xffffffffu, v, o));
    return v;
}

enum ROp { R_SUM = 0, R_MIN = 1, R_MAX = 2 };

template <int OP>
__device__ __forceinline__ double rcomb(double a, double b) {
    return OP == R_SUM ? a + b : (OP == R_MIN ? fmin(a, b) : fmax(a, b));
}
template <int OP>
__device__ __forceinline__ double rwarp(double v) {
    return OP == R_SUM ? warp_sum(v) : (OP == R_MIN ? warp_min(v) : warp_max(v));
}

// Reduce NV values per thread across the block; result valid in thread 0.
// smem must hold NV * 32 doubles.
template <int OP, int NV>
__device__ __forceinline__ void block_reduce(double (&v)[NV], double* smem) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const int lane = tid & 31, wid = tid >> 5, nw = (nthreads + 31) >> 5;
#pragma unroll
    for (int q = 0; q < NV; q++) {
        v[q] = rwarp<OP>(v[q]);
        if (lane == 0) smem[q * 32 + wid] = v[q];
    }
    __syncthreads();
    if (wid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) {
            double x = lane < nw ? smem[q * 32 + lane]
                                 : (OP == R_SUM ? 0.0 : (OP == R_MIN ? 1e300 : -1e300));
            x = rwarp<OP>(x);
            v[q] = x;
        }
    }
    __syncthreads();
}

// Publish this block's NV partials; returns true in every thread of the
// block that finished last.  partials layout: [q][block].
template <int NV>
__device__ __forceinline__ bool publish_partials(const double (&v)[NV],
                                                 double* partials,
                                                 unsigned int* ticket,
                                                 unsigned int nblocks) {
    __shared__ bool s_last;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) partials[(size_t)q * nblocks + bid] = v[q];
        __threadfence();
        const unsigned int t = atomicAdd(ticket, 1u);
        s_last = (t == nblocks - 1);
    }
    __syncthreads();
    if (s_last) __threadfence();
    return s_last;
}

// In the last block: reduce the partials in a fixed order.  Result valid in
// thread 0.  Resets the ticket.
template <int OP, int NV>
__device__ __forceinline__ void final_reduce(double (&out)[NV],
                                             const double* partials,
                                             unsigned int* ticket,
                                             unsigned int nblocks,
                                             double* smem) {
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const double ident = OP == R_SUM ? 0.0 : (OP == R_MIN ? 1e300 : -1e300);
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double acc = ident;
        const volatile double* pq = partials + (size_t)q * nblocks;
        for (unsigned int b = tid; b < nblocks; b += nthreads) acc = rcomb<OP>(acc, pq[b]);
        out[q] = acc;
    }
    block_reduce<OP, NV>(out, smem);
    if (tid == 0) *ticket = 0u;
}

inline unsigned int nblocks_of(dim3 g) { return g.x * g.y * g.z; }

// Two-level deterministic reduction for grids of many blocks: blocks are
// grouped by consecutive index (RGROUP per group); the last block of a group
// (group ticket) sums the group's partials in a fixed order, and the last
// group (global ticket) sums the group partials in a fixed order.  The
// atomics spread over many addresses instead of one.  Call with the block
// result valid in thread 0 of v; returns true in the single block that holds
// the final result (valid in thread 0 of out).  Tickets are reset for reuse.
constexpr int RGROUP = 64;

struct Red2 {
    double* partials;     // NV * nblocks
    double* gpartials;    // NV * ngroups
    unsigned int* gtick;  // ngroups
    unsigned int* ticket; // 1
};

template <int NV>
__device__ __forceinline__ bool reduce2(const double (&v)[NV], const Red2& R, double* smem,
                                        double (&out)[NV]) {
    __shared__ int s_flag;
    const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
    const int nthreads = blockDim.x * blockDim.y * blockDim.z;
    const unsigned int nb = gridDim.x * gridDim.y * gridDim.z;
    const unsigned int bid = blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z);
    const unsigned int ng = (nb + RGROUP - 1) / RGROUP;
    const unsigned int g = bid / RGROUP;
    const unsigned int gsize = min((unsigned int)RGROUP, nb - g * RGROUP);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) R.partials[(size_t)q * nb + bid] = v[q];
        __threadfence();
        s_flag = (atomicAdd(R.gtick + g, 1u) == gsize - 1);
    }
    __syncthreads();
    if (!s_flag) return false;
    __threadfence();
    double x[NV];
#pragma unroll
    for (int q = 0; q < NV; q++)
        x[q] = tid < (int)gsize ? __ldcg(R.partials + (size_t)q * nb + g * RGROUP + tid) : 0.0;
    block_reduce<R_SUM, NV>(x, smem);
    if (tid == 0) {
#pragma unroll
        for (int q = 0; q < NV; q++) R.gpartials[(size_t)q * ng + g] = x[q];
        R.gtick[g] = 0u;
        __threadfence();
        s_flag = (atomicAdd(R.ticket, 1u) == ng - 1);
    }
    __syncthreads();
    if (!s_flag) return false;
    __threadfence();
#pragma unroll
    for (int q = 0; q < NV; q++) {
        double acc = 0.0;
        for (unsigned int b = tid; b < ng; b += nthreads) acc += __ldcg(R.gpartials + (size_t)q * ng + b);
        out[q] = acc;
    }
    block_reduce<R_SUM, NV>(out, smem);
    if (tid == 0) *R.ticket = 0u;
    return true;
}


}  // namespace dcm
