// dcm_capi.cu -- the extern "C" boundary (include/dcm.h): handle lifetime,
// per-call drop-ins for the reference subroutines, and the device-resident
// time loop of model_driver (driver_code.f90:304-676).
#include <cmath>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <cstdio>
#include <cstring>
#include <type_traits>
#include <string>
#include <vector>

#include "dcm_internal.h"
#include "dcm_prof.h"

using namespace dcm;

namespace dcm {
// per host thread: a handle is driven by one thread at a time, and a launch
// made by another thread (another handle, the allocation-free entry point)
// must never touch this handle's profiler
thread_local Profiler* g_prof = nullptr;
}

namespace {

constexpr int NQMAX = 64;

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
};

// resident fields of one precision (velocity time levels in buffers 0..2)
template <typename T>
struct State {
    T *U[3]{}, *V[3]{}, *W[3]{};
    T *th = nullptr, *th2 = nullptr, *su = nullptr, *sv = nullptr, *sw = nullptr,
      *sth = nullptr, *means = nullptr;
    std::vector<T*> q, sq, qtmp;
    // subgrid model (viscous): viscosities, strain rate, lamsq (kp+2) and
    // the six stresses (scratch of each step)
    T *vism = nullptr, *vist = nullptr, *strain = nullptr, *lamsq = nullptr;
    T* tau[6]{};
    double* lamsq64 = nullptr;
};

}  // namespace

struct dcm_handle {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    Dims d{};      // pitched device layout of the fields
    Dims hd{};     // dense layout of the caller's host arrays
    size_t n = 0;  // elements of a device field (pitched, without FIELD_PAD)
    size_t nh = 0; // elements of a host field
    std::string err;

    // 1-D metrics (device) and the per-axis stencil coefficients
    double* metric_block = nullptr;
    Metrics<double> mt{};
    double *ae = nullptr, *aw = nullptr, *an = nullptr, *as = nullptr, *au = nullptr,
           *ad = nullptr;
    std::vector<double> h_xg, h_yg, h_zg;

    // reductions
    double* partials = nullptr;
    size_t npartials = 0;
    unsigned int* ticket = nullptr;
    double* gpartials = nullptr;  // two-level reductions
    unsigned int* gtick = nullptr;
    unsigned int* ticket2 = nullptr;
    SolverScalars* S = nullptr;
    SolverScalars* hS = nullptr;  // pinned
    MpScalars* M = nullptr;       // NQMAX + 2 (Mone, Mzero)
    MpScalars* hM = nullptr;      // pinned mirror

    // named full-size scratch buffers
    std::vector<double*> slots;
    double* sg_lamsq = nullptr;  // lamsq of dcm_calculate_subgrid_3d (kp+2)
    double* dense_stage = nullptr;  // one field in the host layout (uploads)
    int first_call = 1;  // bicgstab_first, dynamics.f90:17

    // FP32 copies for the mixed-precision form
    float* metric_block_f = nullptr;
    Metrics<float> mtf{};
    float *aef = nullptr, *awf = nullptr, *anf = nullptr, *asf = nullptr, *auf = nullptr,
          *adf = nullptr;
    std::vector<float*> fslots;
    SolverScalars* S2 = nullptr;   // scalars of the inner (FP32) solve
    SolverScalars* hS2 = nullptr;  // pinned
    // captured pressure solves (FP64 and mixed), rebuilt when their
    // arguments change
    SolveGraph g64, g32;
    // solver loops: 1 graph-driven, 2 graph-driven without programmatic
    // dependent launch, 0 host-polled
    int graphs = 1;
    // launch shape of the solver kernels per precision (dcm_tune; [0] FP64,
    // [1] the FP32 iterations of the mixed form): warps per sweep block, warp
    // tasks per warp of the reducing kernels (0 = fill the GPU), marching depth
    int tune_by[2] = {8, 8}, tune_tasks[2] = {0, 0}, tune_ni[2] = {4, 1}, tune_fuse[2] = {0, 1};
    int tune_vec[2] = {2, 4};  // levels per lane (FP64 fixed at 2)
    // dcm_solver_limits: round budget of graph-driven solves (0: default) and
    // the FP64 breakdown threshold (< 0: the reference's tiny)
    int round_budget = 0;
    double tiny = -1.0;
    // dcm_set_small_solver: FP64 solves of at most this many interior points
    // run as one thread-block cluster
    long long small_max = 8192;
    // dcm_set_mpdata_shape: fused antidiffusive iterations (off by default:
    // slower on B200, see dcm.h), their row cap
    int mp_fuse = 0, mp_rows = 32;
    // bumped whenever captured pointers or launch shapes change (state
    // upload, tuning); an ensemble rebuilds its step graphs when it moves
    unsigned generation = 0;

    // ---- resident state -------------------------------------------------------
    bool resident = false;
    dcm_config cfg{};
    std::vector<int> cs, ce;
    double* forcing_dev = nullptr;
    float* forcing_f = nullptr;
    int nstep = 0;
    int prec = 0;  // 0 FP64, 1 FP32 fields + FP64 refinement
    State<double> s64;
    State<float> s32;
    double *p = nullptr, *div = nullptr, *psrc = nullptr;  // FP64 in both forms
    double t1 = 0.0, t2 = 0.0;
    std::vector<double> q1, q2;
    std::vector<void*> owned;
    int last_iters = 0;
    double last_err = 0.0;
    RefineStats last_refine{};
    long long refine_outer_total = 0;
    Profiler prof;
};

namespace {

int fail(dcm_handle* h, int code, const char* what) {
    if (h) h->err = what;
    return code;
}

int cuda_fail(dcm_handle* h, cudaError_t e, const char* where) {
    if (h) {
        h->err = std::string(where) + ": " + cudaGetErrorString(e);
    }
    return DCM_E_CUDA;
}

#define CK(call)                                                  \
    do {                                                          \
        cudaError_t e_ = (call);                                  \
        if (e_ != cudaSuccess) return cuda_fail(h, e_, #call);    \
    } while (0)

// A device field in the pitched layout: the returned pointer is FIELD_SHIFT
// elements into a zeroed allocation of n + FIELD_PAD elements (free with
// free_field).
template <typename T>
T* alloc_field(dcm_handle* h) {
    T* raw = nullptr;
    const size_t cnt = h->n + FIELD_PAD;
    if (cudaMalloc(&raw, cnt * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemsetAsync(raw, 0, cnt * sizeof(T), h->st);
    return raw + FIELD_SHIFT;
}
template <typename T>
void free_field(T* p) {
    if (p) cudaFree(p - FIELD_SHIFT);
}

double* slot(dcm_handle* h, int idx) {
    if ((int)h->slots.size() <= idx) h->slots.resize(idx + 1, nullptr);
    if (!h->slots[idx]) h->slots[idx] = alloc_field<double>(h);
    return h->slots[idx];
}

float* fslot(dcm_handle* h, int idx) {
    if ((int)h->fslots.size() <= idx) h->fslots.resize(idx + 1, nullptr);
    if (!h->fslots[idx]) h->fslots[idx] = alloc_field<float>(h);
    return h->fslots[idx];
}

// slot numbering of the per-call drop-ins
enum {
    S_U = 0, S_V, S_W, S_ZU, S_ZV, S_ZW, S_SU, S_SV, S_SW, S_P, S_TH, S_STH, S_RHS, S_X, S_B,
    // solver work
    S_R, S_CR, S_PP, S_V1, S_T, S_SA, S_SB, S_RH, S_VH,
    // mpdata work
    S_VA0, S_VA1, S_VA2, S_VL0, S_VL1, S_VL2, S_B0, S_B1, S_B2, S_B3, S_B4, S_B5,
    S_PSI_OUT, S_STAGE,
    // subgrid drop-in: vism, vist, strain, tau11, tau22, tau33, tau12, tau13, tau23, q, sq
    S_SG = 40,
    S_DYN = 64  // psi fields / scratch for vec: S_DYN + 4*q + {in, out, pa, pb}
};

// n = 0: a whole field, dense host columns of kp+2 into pitched device
// columns of K (one 2-D copy); n > 0: n contiguous elements (1-D profiles).
// A whole field goes as one contiguous copy into a dense staging buffer and is
// re-pitched (and converted to TO) on the device: a pitched 2-D host-to-device
// copy of 1 KB rows ran at a sixth of the rate of the contiguous one.  The
// stream orders the next field's copy into the stage after this kernel.
template <typename TO>
int upload_field(dcm_handle* h, TO* dst, const double* src) {
    if (!src) return DCM_OK;
    if (!h->dense_stage) CK(cudaMalloc(&h->dense_stage, h->nh * sizeof(double)));
    CK(cudaMemcpyAsync(h->dense_stage, src, h->nh * sizeof(double), cudaMemcpyHostToDevice,
                       h->st));
    launch_repitch<TO>(h->hd, h->d, dst, h->dense_stage, h->st);
    return DCM_OK;
}

int upload(dcm_handle* h, double* dst, const double* src, size_t n = 0) {
    if (!src) return DCM_OK;
    if (n) {
        CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyHostToDevice, h->st));
        return DCM_OK;
    }
    return upload_field<double>(h, dst, src);
}
int download(dcm_handle* h, double* dst, const double* src, size_t n = 0) {
    if (!dst) return DCM_OK;
    if (n) {
        CK(cudaMemcpyAsync(dst, src, n * sizeof(double), cudaMemcpyDeviceToHost, h->st));
        return DCM_OK;
    }
    const size_t w = (size_t)h->hd.K * sizeof(double);
    CK(cudaMemcpy2DAsync(dst, w, src, (size_t)h->d.K * sizeof(double), w,
                         (size_t)h->d.J * h->d.I, cudaMemcpyDeviceToHost, h->st));
    return DCM_OK;
}
int sync(dcm_handle* h) {
    CK(cudaStreamSynchronize(h->st));
    CK(cudaGetLastError());
    return DCM_OK;
}

SolverWork<double> solver_work(dcm_handle* h) {
    SolverWork<double> w;
    w.r = slot(h, S_R); w.cr = slot(h, S_CR); w.p = slot(h, S_PP); w.v1 = slot(h, S_V1);
    w.t = slot(h, S_T); w.sA = slot(h, S_SA); w.sB = slot(h, S_SB);
    w.rh = slot(h, S_RH); w.vh = slot(h, S_VH);
    w.ae = h->ae; w.aw = h->aw; w.an = h->an; w.as = h->as; w.au = h->au; w.ad = h->ad;
    w.partials = h->partials; w.ticket = h->ticket; w.S = h->S;
    w.red.partials = h->partials; w.red.gpartials = h->gpartials; w.red.gtick = h->gtick;
    w.red.ticket = h->ticket2;
    w.graph = h->graphs ? &h->g64 : nullptr;
    w.pdl = h->graphs == 1;
    w.by = h->tune_by[0];
    w.tasks = h->tune_tasks[0];
    w.ni = h->tune_ni[0];
    w.fuse = 0;
    w.max_blocks = (int)std::min<size_t>(h->npartials / 3, (size_t)1 << 30);
    w.round_budget = h->round_budget;
    w.tiny = h->tiny;
    w.small_max = h->small_max;
    return w;
}

// The FP64 side of a mixed solve: scalars, reductions and coefficients only
// (the FP64 residual is formed from x and b directly, no FP64 work vectors).
SolverWork<double> solver_scalars(dcm_handle* h) {
    SolverWork<double> w{};
    w.max_blocks = (int)std::min<size_t>(h->npartials / 3, (size_t)1 << 30);
    w.ae = h->ae; w.aw = h->aw; w.an = h->an; w.as = h->as; w.au = h->au; w.ad = h->ad;
    w.partials = h->partials; w.ticket = h->ticket; w.S = h->S;
    w.red.partials = h->partials; w.red.gpartials = h->gpartials; w.red.gtick = h->gtick;
    w.red.ticket = h->ticket2;
    return w;
}

struct MpBufs {
    MpdataWork<double> w;
    std::vector<double*> pa, pb;
};

bool mpdata_work(dcm_handle* h, int nq, MpBufs& b) {
    b.pa.resize(nq);
    b.pb.resize(nq);
    for (int q = 0; q < nq; q++) {
        b.pa[q] = slot(h, S_DYN + 4 * q + 2);
        b.pb[q] = slot(h, S_DYN + 4 * q + 3);
        if (!b.pa[q] || !b.pb[q]) return false;
    }
    b.w.pa = b.pa.data();
    b.w.pb = b.pb.data();
    const int va[3] = {S_VA0, S_VA1, S_VA2}, vl[3] = {S_VL0, S_VL1, S_VL2};
    for (int c = 0; c < 3; c++) {
        b.w.va[c] = slot(h, va[c]);
        b.w.vl[c] = slot(h, vl[c]);
        if (!b.w.va[c] || !b.w.vl[c]) return false;
    }
    const int bt[6] = {S_B0, S_B1, S_B2, S_B3, S_B4, S_B5};
    for (int c = 0; c < 6; c++) {
        b.w.beta[c] = slot(h, bt[c]);
        if (!b.w.beta[c]) return false;
    }
    b.w.partials = h->partials;
    b.w.ticket = h->ticket;
    b.w.M = h->M;
    b.w.Mone = h->M + NQMAX;
    b.w.Mzero = h->M + NQMAX + 1;
    b.w.fuse = h->mp_fuse;
    b.w.fuse_rows = h->mp_rows;
    return true;
}

Forcing<double> forcing_of(dcm_handle* h, const dcm_forcing* f, double* dev, int* rc) {
    Forcing<double> F{};
    *rc = DCM_OK;
    if (!f) return F;
    F.damping_layer = f->damping_layer;
    F.forcing = f->forcing;
    F.divergence = f->divergence;
    F.forcing_tau = f->forcing_tau;
    const size_t K2 = h->d.kp + 2;
    const double* src[5] = {f->dampfacn, f->dampfac, f->u_force, f->v_force, f->w_subs};
    for (int c = 0; c < 5; c++) {
        if (src[c]) {
            if (cudaMemcpyAsync(dev + c * K2, src[c], K2 * sizeof(double), cudaMemcpyHostToDevice,
                                h->st) != cudaSuccess)
                *rc = DCM_E_CUDA;
        }
    }
    F.dampfacn = dev;
    F.dampfac = dev + K2;
    F.u_force = dev + 2 * K2;
    F.v_force = dev + 3 * K2;
    F.w_subs = dev + 4 * K2;
    if ((f->damping_layer && (!f->dampfacn || !f->dampfac)) ||
        (f->forcing && (!f->u_force || !f->v_force)) || (f->divergence && !f->w_subs))
        *rc = DCM_E_ARG;
    return F;
}

}  // namespace

// =============================================================================
// lifetime
// =============================================================================
extern "C" const char* dcm_status_string(int s) {
    switch (s) {
        case DCM_OK: return "ok";
        case DCM_E_NOCONV: return "convergence failure";
        case DCM_E_BREAKDOWN: return "convergence problem (omega breakdown)";
        case DCM_E_NONFINITE: return "non-finite residual";
        case DCM_E_CUDA: return "CUDA error";
        case DCM_E_TIMEOUT: return "device wait timed out";
        case DCM_E_DECOMP: return "only a 1x1x1 process grid is supported";
        case DCM_E_ARG: return "invalid argument";
        case DCM_E_UNSUPPORTED: return "unsupported configuration";
        case DCM_E_IO: return "output file error";
        default: return "unknown status";
    }
}

extern "C" const char* dcm_last_error(const dcm_handle* h) { return h ? h->err.c_str() : ""; }

extern "C" int dcm_check_decomposition(const int dims[3]) {
    if (!dims) return DCM_E_ARG;
    return (dims[0] == 1 && dims[1] == 1 && dims[2] == 1) ? DCM_OK : DCM_E_DECOMP;
}

extern "C" int dcm_create(const dcm_grid* g, int device, dcm_handle** out) {
    if (!g || !out) return DCM_E_ARG;
    *out = nullptr;
    if (g->ip < 1 || g->jp < 1 || g->kp < 3) return DCM_E_ARG;
    const double* req[10] = {g->dx, g->dxn, g->dy, g->dyn, g->dz,
                             g->dzn, g->rhoa, g->rhoan, g->theta, g->thetan};
    for (auto p : req)
        if (!p) return DCM_E_ARG;
    const Dims d = make_dims_pitched(g->ip, g->jp, g->kp);
    if (d.n() + FIELD_PAD >= (size_t)1 << 31) return DCM_E_UNSUPPORTED;  // int32 indexing
    dcm_handle* h = new dcm_handle();
    h->device = device;
    h->d = d;
    h->hd = make_dims(g->ip, g->jp, g->kp);
    h->n = d.n();
    h->nh = h->hd.n();
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    solver_init();
    mpdata_init();
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    const size_t I2 = g->ip + 2, J2 = g->jp + 2, K2 = g->kp + 2;
    // metrics block: dx dxn (I2) dy dyn (J2) dz dzn rhoa rhoan theta thetan (K2)
    //                ae aw (I2) an as (J2) au ad (K2)
    // Each table starts FIELD_SHIFT elements past a multiple of FIELD_ALIGN,
    // so its element 1 is aligned like the fields' k = 1 (16-byte vector
    // loads of per-level coefficients); FIELD_PAD spare elements follow each.
    auto slot_len = [](size_t len) {
        return (len + FIELD_PAD + FIELD_ALIGN - 1) / FIELD_ALIGN * FIELD_ALIGN;
    };
    const size_t nm = 4 * slot_len(I2) + 4 * slot_len(J2) + 8 * slot_len(K2) + FIELD_ALIGN;
    std::vector<double> hm(nm, 0.0);
    size_t o = FIELD_SHIFT;
    auto put = [&](const double* src, size_t len) {
        const size_t at = o;
        std::memcpy(hm.data() + o, src, len * sizeof(double));
        o += slot_len(len);
        return at;
    };
    const size_t o_dx = put(g->dx, I2), o_dxn = put(g->dxn, I2), o_dy = put(g->dy, J2),
                 o_dyn = put(g->dyn, J2), o_dz = put(g->dz, K2), o_dzn = put(g->dzn, K2),
                 o_ra = put(g->rhoa, K2), o_rn = put(g->rhoan, K2), o_th = put(g->theta, K2),
                 o_thn = put(g->thetan, K2);
    // set_mat_a, dynamics.f90:87-92 (index 0 unused)
    std::vector<double> ae(I2, 0), aw(I2, 0), an(J2, 0), as(J2, 0), au(K2, 0), ad(K2, 0);
    for (int i = 1; i <= g->ip; i++) {
        ae[i] = 1.0 / (g->dx[i - 1] * g->dxn[i]);
        aw[i] = 1.0 / (g->dx[i - 1] * g->dxn[i - 1]);
    }
    for (int j = 1; j <= g->jp; j++) {
        an[j] = 1.0 / (g->dy[j - 1] * g->dyn[j]);
        as[j] = 1.0 / (g->dy[j - 1] * g->dyn[j - 1]);
    }
    for (int k = 1; k <= g->kp; k++) {
        au[k] = 1.0 / (g->dz[k - 1] * g->dzn[k]);
        ad[k] = 1.0 / (g->dz[k - 1] * g->dzn[k - 1]);
    }
    const size_t o_ae = put(ae.data(), I2), o_aw = put(aw.data(), I2), o_an = put(an.data(), J2),
                 o_as = put(as.data(), J2), o_au = put(au.data(), K2), o_ad = put(ad.data(), K2);
    CK(cudaMalloc(&h->metric_block, nm * sizeof(double)));
    CK(cudaMemcpy(h->metric_block, hm.data(), nm * sizeof(double), cudaMemcpyHostToDevice));
    double* mb = h->metric_block;
    h->mt.dx = mb + o_dx; h->mt.dxn = mb + o_dxn; h->mt.dy = mb + o_dy; h->mt.dyn = mb + o_dyn;
    h->mt.dz = mb + o_dz; h->mt.dzn = mb + o_dzn; h->mt.rhoa = mb + o_ra; h->mt.rhoan = mb + o_rn;
    h->mt.theta = mb + o_th; h->mt.thetan = mb + o_thn;
    h->ae = mb + o_ae; h->aw = mb + o_aw; h->an = mb + o_an; h->as = mb + o_as;
    h->au = mb + o_au; h->ad = mb + o_ad;
    if (g->xg) h->h_xg.assign(g->xg, g->xg + I2);
    if (g->yg) h->h_yg.assign(g->yg, g->yg + J2);
    if (g->zg) h->h_zg.assign(g->zg, g->zg + K2);
    // reduction partials: the largest grid of any reducing kernel, x2 values
    const dim3 gi = interior_grid(d, d.kp), gf = full_grid(d);
    size_t np = std::max<size_t>(nblocks_of(gi), nblocks_of(gf));
    np = std::max<size_t>(np, (size_t)4 * K2 * 128);
    h->npartials = 2 * np;
    CK(cudaMalloc(&h->partials, h->npartials * sizeof(double)));
    CK(cudaMalloc(&h->ticket, sizeof(unsigned int)));
    CK(cudaMemset(h->ticket, 0, sizeof(unsigned int)));
    {
        const size_t ng = np / RGROUP + 2;
        CK(cudaMalloc(&h->gpartials, 2 * ng * sizeof(double)));
        CK(cudaMalloc(&h->gtick, ng * sizeof(unsigned int)));
        CK(cudaMemset(h->gtick, 0, ng * sizeof(unsigned int)));
        CK(cudaMalloc(&h->ticket2, sizeof(unsigned int)));
        CK(cudaMemset(h->ticket2, 0, sizeof(unsigned int)));
    }
    CK(cudaMalloc(&h->S, sizeof(SolverScalars)));
    CK(cudaMemset(h->S, 0, sizeof(SolverScalars)));
    CK(cudaMallocHost(&h->hS, sizeof(SolverScalars)));
    CK(cudaMalloc(&h->M, (NQMAX + 2) * sizeof(MpScalars)));
    CK(cudaMallocHost(&h->hM, (NQMAX + 2) * sizeof(MpScalars)));
    std::memset(h->hM, 0, (NQMAX + 2) * sizeof(MpScalars));
    h->hM[NQMAX].early = 1;  // Mone
    CK(cudaMemcpy(h->M, h->hM, (NQMAX + 2) * sizeof(MpScalars), cudaMemcpyHostToDevice));
    CK(cudaMalloc(&h->forcing_dev, 5 * K2 * sizeof(double)));
    CK(cudaMemset(h->forcing_dev, 0, 5 * K2 * sizeof(double)));
    CK(cudaMalloc(&h->forcing_f, 5 * K2 * sizeof(float)));
    CK(cudaMemset(h->forcing_f, 0, 5 * K2 * sizeof(float)));
    // FP32 copies of the metric block for the mixed-precision form
    CK(cudaMalloc(&h->metric_block_f, nm * sizeof(float)));
    launch_convert<float, double>(nm, h->metric_block_f, h->metric_block, h->st);
    float* mf = h->metric_block_f;
    h->mtf.dx = mf + o_dx; h->mtf.dxn = mf + o_dxn; h->mtf.dy = mf + o_dy; h->mtf.dyn = mf + o_dyn;
    h->mtf.dz = mf + o_dz; h->mtf.dzn = mf + o_dzn; h->mtf.rhoa = mf + o_ra;
    h->mtf.rhoan = mf + o_rn; h->mtf.theta = mf + o_th; h->mtf.thetan = mf + o_thn;
    h->aef = mf + o_ae; h->awf = mf + o_aw; h->anf = mf + o_an; h->asf = mf + o_as;
    h->auf = mf + o_au; h->adf = mf + o_ad;
    CK(cudaMalloc(&h->S2, sizeof(SolverScalars)));
    CK(cudaMemset(h->S2, 0, sizeof(SolverScalars)));
    CK(cudaMallocHost(&h->hS2, sizeof(SolverScalars)));
    CK(cudaStreamSynchronize(h->st));
    *out = h;
    return DCM_OK;
}

static void free_state(dcm_handle* h) {
    h->g64.release();  // captured solves hold the old field pointers
    h->g32.release();
    for (void* p : h->owned) cudaFree(p);
    h->owned.clear();
    h->s64 = State<double>();
    h->s32 = State<float>();
    h->p = h->div = h->psrc = nullptr;
    h->resident = false;
}

extern "C" int dcm_destroy(dcm_handle* h) {
    if (!h) return DCM_OK;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    free_state(h);
    for (double* p : h->slots) free_field(p);
    for (float* p : h->fslots) free_field(p);
    cudaFree(h->metric_block_f);
    cudaFree(h->sg_lamsq);
    cudaFree(h->dense_stage);
    cudaFree(h->S2);
    cudaFreeHost(h->hS2);
    cudaFree(h->forcing_f);
    cudaFree(h->metric_block);
    cudaFree(h->partials);
    cudaFree(h->ticket);
    cudaFree(h->gpartials);
    cudaFree(h->gtick);
    cudaFree(h->ticket2);
    cudaFree(h->S);
    cudaFreeHost(h->hS);
    cudaFree(h->M);
    cudaFreeHost(h->hM);
    cudaFree(h->forcing_dev);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->st) cudaStreamDestroy(h->st);
    delete h;
    return DCM_OK;
}

// =============================================================================
// per-call drop-ins
// =============================================================================
#define CHECK_H()                                   \
    do {                                            \
        if (!h) return DCM_E_ARG;                   \
        CK(cudaSetDevice(h->device));               \
    } while (0)
#define RC(x)                      \
    do {                           \
        int rc_ = (x);             \
        if (rc_ != DCM_OK) return rc_; \
    } while (0)
#define NEED(p)                               \
    do {                                      \
        if (!(p)) return fail(h, DCM_E_CUDA, "device allocation failed"); \
    } while (0)

extern "C" int dcm_bicgstab(dcm_handle* h, double* x, double* b, const double* sw, double tol,
                            int test_solver, int itmax, int* iters, double* err) {
    CHECK_H();
    if (!x || !b || !sw || itmax < 1) return fail(h, DCM_E_ARG, "bicgstab: bad argument");
    const Dims& d = h->d;
    if (h->first_call) {
        if (test_solver) {  // dynamics.f90:354-364
            if (h->h_xg.empty() || h->h_yg.empty() || h->h_zg.empty())
                return fail(h, DCM_E_ARG, "bicgstab: test_solver needs xg, yg, zg");
            for (int i = 1; i <= d.ip; i++)
                for (int j = 1; j <= d.jp; j++)
                    for (int k = 1; k <= d.kp; k++)
                        b[h->hd.at(k, j, i)] =
                            std::exp(-1.0 / 5.e6 *
                                     (h->h_xg[i] * h->h_xg[i] + h->h_yg[j] * h->h_yg[j] +
                                      std::pow(h->h_zg[k] - 4000.0, 2.0)));
        }
        h->first_call = 0;
    }
    double *X = slot(h, S_X), *B = slot(h, S_B), *SW = slot(h, S_SW);
    NEED(X); NEED(B); NEED(SW);
    SolverWork<double> w = solver_work(h);
    NEED(w.r); NEED(w.sB); NEED(w.rh); NEED(w.vh);
    RC(upload(h, X, x));
    RC(upload(h, B, b));
    RC(upload(h, SW, sw));
    const int st = solver_run<double>(w, d, X, B, SW, h->mt.dzn, tol, itmax, 1, 4, h->st, h->hS,
                                      nullptr);
    if (st == DCM_E_CUDA) return cuda_fail(h, cudaGetLastError(), "bicgstab");
    RC(download(h, x, X));
    RC(sync(h));
    if (iters) *iters = h->hS->it;
    if (err) *err = h->hS->err;
    if (st != DCM_OK) h->err = dcm_status_string(st);
    return st;
}

extern "C" int dcm_sources(dcm_handle* h, const dcm_forcing* forcing, const double* ubar,
                           const double* vbar, const double* wbar, const double* thbar,
                           const double* zu, const double* zv, const double* zw, const double* u,
                           const double* v, const double* w, const double* th, double* su,
                           double* sv, double* sw, double* sth, double* rhs) {
    CHECK_H();
    if (!thbar || !u || !v || !w || !th || !su || !sv || !sw || !sth || !rhs)
        return fail(h, DCM_E_ARG, "sources: bad argument");
    const Dims& d = h->d;
    const size_t K2 = d.kp + 2;
    int rc = DCM_OK;
    Forcing<double> F = forcing_of(h, forcing, h->forcing_dev, &rc);
    if (rc != DCM_OK) return fail(h, rc, "sources: forcing arrays");
    if (forcing && (forcing->damping_layer || forcing->forcing) && (!zu || !zv || !zw))
        return fail(h, DCM_E_ARG, "sources: damping/forcing need zu, zv, zw");
    if (forcing && forcing->damping_layer && (!ubar || !vbar))
        return fail(h, DCM_E_ARG, "sources: damping needs ubar, vbar");
    if (forcing && forcing->divergence && !wbar)
        return fail(h, DCM_E_ARG, "sources: subsidence needs wbar");
    double *U = slot(h, S_U), *V = slot(h, S_V), *W = slot(h, S_W), *TH = slot(h, S_TH),
           *ZU = slot(h, S_ZU), *ZV = slot(h, S_ZV), *ZW = slot(h, S_ZW), *SU = slot(h, S_SU),
           *SV = slot(h, S_SV), *SWd = slot(h, S_SW), *STH = slot(h, S_STH),
           *RHS = slot(h, S_RHS), *BARS = slot(h, S_B);
    NEED(U); NEED(V); NEED(W); NEED(TH); NEED(ZU); NEED(ZV); NEED(ZW); NEED(SU); NEED(SV);
    NEED(SWd); NEED(STH); NEED(RHS); NEED(BARS);
    RC(upload(h, U, u)); RC(upload(h, V, v)); RC(upload(h, W, w)); RC(upload(h, TH, th));
    RC(upload(h, ZU, zu)); RC(upload(h, ZV, zv)); RC(upload(h, ZW, zw));
    RC(upload(h, STH, sth)); RC(upload(h, RHS, rhs));
    RC(upload(h, BARS, ubar, K2)); RC(upload(h, BARS + K2, vbar, K2));
    RC(upload(h, BARS + 2 * K2, wbar, K2)); RC(upload(h, BARS + 3 * K2, thbar, K2));
    launch_sources<double, double>(d, h->mt, h->mt, F, BARS, BARS + K2, BARS + 2 * K2,
                                   BARS + 3 * K2, ZU, ZV, ZW, U, V, W, TH, SU, SV, SWd, STH, RHS,
                                   0, 0, h->st);
    CK(cudaGetLastError());
    RC(download(h, su, SU)); RC(download(h, sv, SV)); RC(download(h, sw, SWd));
    RC(download(h, sth, STH)); RC(download(h, rhs, RHS));
    return sync(h);
}

extern "C" int dcm_advance_momentum(dcm_handle* h, double dt, double* u, double* v, double* w,
                                    const double* zu, const double* zv, const double* zw,
                                    const double* su, const double* sv, const double* sw,
                                    const double* p) {
    CHECK_H();
    if (!u || !v || !w || !zu || !zv || !zw || !su || !sv || !sw || !p)
        return fail(h, DCM_E_ARG, "advance_momentum: bad argument");
    double *U = slot(h, S_U), *V = slot(h, S_V), *W = slot(h, S_W), *ZU = slot(h, S_ZU),
           *ZV = slot(h, S_ZV), *ZW = slot(h, S_ZW), *SU = slot(h, S_SU), *SV = slot(h, S_SV),
           *SWd = slot(h, S_SW), *P = slot(h, S_P);
    NEED(U); NEED(V); NEED(W); NEED(ZU); NEED(ZV); NEED(ZW); NEED(SU); NEED(SV); NEED(SWd);
    NEED(P);
    RC(upload(h, U, u)); RC(upload(h, V, v)); RC(upload(h, W, w));
    RC(upload(h, ZU, zu)); RC(upload(h, ZV, zv)); RC(upload(h, ZW, zw));
    RC(upload(h, SU, su)); RC(upload(h, SV, sv)); RC(upload(h, SWd, sw)); RC(upload(h, P, p));
    launch_advance_momentum<double>(h->d, h->mt, dt, U, V, W, ZU, ZV, ZW, SU, SV, SWd, P, h->st);
    CK(cudaGetLastError());
    RC(download(h, u, U)); RC(download(h, v, V)); RC(download(h, w, W));
    return sync(h);
}

extern "C" int dcm_first_order_upstream_3d(dcm_handle* h, double dt, const double* u,
                                           const double* v, const double* w, double* psi,
                                           int neumann) {
    CHECK_H();
    if (!u || !v || !w || !psi || neumann < 0 || neumann > 2)
        return fail(h, DCM_E_ARG, "first_order_upstream_3d: bad argument");
    double *U = slot(h, S_U), *V = slot(h, S_V), *W = slot(h, S_W), *PI = slot(h, S_TH),
           *PO = slot(h, S_PSI_OUT);
    NEED(U); NEED(V); NEED(W); NEED(PI); NEED(PO);
    MpBufs mb;
    if (!mpdata_work(h, 1, mb)) return fail(h, DCM_E_CUDA, "device allocation failed");
    RC(upload(h, U, u)); RC(upload(h, V, v)); RC(upload(h, W, w)); RC(upload(h, PI, psi));
    CK(cudaMemcpyAsync(PO, PI, h->n * sizeof(double), cudaMemcpyDeviceToDevice, h->st));
    RC(upwind_run<double>(mb.w, h->d, h->mt, dt, U, V, W, PI, PO, neumann, h->st));
    RC(download(h, psi, PO));
    return sync(h);
}

static int mpdata_dropin(dcm_handle* h, double dt, const double* u, const double* v,
                         const double* w, double* psi, int nq, double* lbc, double* ubc, int kord,
                         int monotone, int neumann, int limiter, bool vec) {
    if (!u || !v || !w || !psi || !lbc || !ubc || nq < 1 || nq > NQMAX || neumann < 0 ||
        neumann > 2 || limiter < 0 || limiter > 1)
        return fail(h, DCM_E_ARG, "mpdata: bad argument");
    double *U = slot(h, S_U), *V = slot(h, S_V), *W = slot(h, S_W);
    NEED(U); NEED(V); NEED(W);
    std::vector<double*> pin(nq), pout(nq);
    for (int q = 0; q < nq; q++) {
        pin[q] = slot(h, S_DYN + 4 * q);
        pout[q] = slot(h, S_DYN + 4 * q + 1);
        NEED(pin[q]); NEED(pout[q]);
    }
    MpBufs mb;
    if (!mpdata_work(h, nq, mb)) return fail(h, DCM_E_CUDA, "device allocation failed");
    RC(upload(h, U, u)); RC(upload(h, V, v)); RC(upload(h, W, w));
    for (int q = 0; q < nq; q++) RC(upload(h, pin[q], psi + (size_t)q * h->nh));
    RC(mpdata_run<double>(mb.w, h->d, h->mt, dt, U, V, W, pin.data(), pout.data(), nq, lbc, ubc,
                          kord, monotone, neumann, limiter, vec, nullptr, 0.0, h->st));
    for (int q = 0; q < nq; q++) RC(download(h, psi + (size_t)q * h->nh, pout[q]));
    CK(cudaMemcpyAsync(h->hM, h->M, nq * sizeof(MpScalars), cudaMemcpyDeviceToHost, h->st));
    RC(sync(h));
    for (int q = 0; q < nq; q++) {  // :711-713 / :1748-1752
        lbc[q] = h->hM[q].lbc + h->hM[q].m;
        ubc[q] = h->hM[q].ubc + h->hM[q].m;
    }
    return DCM_OK;
}

extern "C" int dcm_mpdata_3d(dcm_handle* h, double dt, const double* u, const double* v,
                             const double* w, double* psi, double* lbc, double* ubc, int kord,
                             int monotone, int neumann, int limiter) {
    CHECK_H();
    return mpdata_dropin(h, dt, u, v, w, psi, 1, lbc, ubc, kord, monotone, neumann, limiter,
                         false);
}

extern "C" int dcm_mpdata_vec_3d(dcm_handle* h, double dt, const double* u, const double* v,
                                 const double* w, double* psi, int nq, double* lbc, double* ubc,
                                 int kord, int monotone, int neumann, int limiter) {
    CHECK_H();
    return mpdata_dropin(h, dt, u, v, w, psi, nq, lbc, ubc, kord, monotone, neumann, limiter,
                         true);
}

extern "C" int dcm_adv_ref_state(dcm_handle* h, double dt, const double* w, double* psi,
                                 const double* psi_ref) {
    CHECK_H();
    if (!w || !psi || !psi_ref) return fail(h, DCM_E_ARG, "adv_ref_state: bad argument");
    double *W = slot(h, S_W), *PI = slot(h, S_TH), *REF = slot(h, S_B);
    NEED(W); NEED(PI); NEED(REF);
    RC(upload(h, W, w)); RC(upload(h, PI, psi)); RC(upload(h, REF, psi_ref, h->d.kp + 2));
    launch_adv_ref_state<double>(h->d, h->mt, dt, W, PI, PI, REF, 0, h->st);
    CK(cudaGetLastError());
    RC(download(h, psi, PI));
    return sync(h);
}

extern "C" int dcm_mpdata_3d_add(dcm_handle* h, double dt, const double* u, const double* v,
                                 const double* w, double* psi, const double* psi_1d, double* lbc,
                                 double* ubc, int kord, int monotone, int neumann, int limiter) {
    CHECK_H();
    if (!psi_1d) return fail(h, DCM_E_ARG, "mpdata_3d_add: bad argument");
    if (!u || !v || !w || !psi || !lbc || !ubc)
        return fail(h, DCM_E_ARG, "mpdata_3d_add: bad argument");
    double *U = slot(h, S_U), *V = slot(h, S_V), *W = slot(h, S_W), *REF = slot(h, S_B);
    double *PI = slot(h, S_DYN), *PO = slot(h, S_DYN + 1);
    NEED(U); NEED(V); NEED(W); NEED(REF); NEED(PI); NEED(PO);
    MpBufs mb;
    if (!mpdata_work(h, 1, mb)) return fail(h, DCM_E_CUDA, "device allocation failed");
    RC(upload(h, U, u)); RC(upload(h, V, v)); RC(upload(h, W, w)); RC(upload(h, PI, psi));
    RC(upload(h, REF, psi_1d, h->d.kp + 2));
    launch_add_profile<double>(h->d, PI, REF, 1.0, h->st);  // :175-177
    RC(mpdata_run<double>(mb.w, h->d, h->mt, dt, U, V, W, &PI, &PO, 1, lbc, ubc, kord, monotone,
                          neumann, limiter, false, nullptr, 0.0, h->st));
    launch_add_profile<double>(h->d, PO, REF, -1.0, h->st);  // :186-188
    CK(cudaGetLastError());
    RC(download(h, psi, PO));
    CK(cudaMemcpyAsync(h->hM, h->M, sizeof(MpScalars), cudaMemcpyDeviceToHost, h->st));
    RC(sync(h));
    *lbc = h->hM[0].lbc + h->hM[0].m;
    *ubc = h->hM[0].ubc + h->hM[0].m;
    return DCM_OK;
}

extern "C" int dcm_horizontal_means(dcm_handle* h, int moisture, int nq, const double* u,
                                    const double* v, const double* w, const double* th,
                                    const double* q, double* ubar, double* vbar, double* wbar,
                                    double* thbar, double* qbar) {
    CHECK_H();
    if (!u || !v || !w || !th || !ubar || !vbar || !wbar || !thbar)
        return fail(h, DCM_E_ARG, "horizontal_means: bad argument");
    if (moisture && (!q || !qbar || nq < 1 || nq > NQMAX))
        return fail(h, DCM_E_ARG, "horizontal_means: bad q arguments");
    const size_t K2 = h->d.kp + 2;
    const int nqq = moisture ? nq : 0;
    double *U = slot(h, S_U), *V = slot(h, S_V), *W = slot(h, S_W), *TH = slot(h, S_TH);
    NEED(U); NEED(V); NEED(W); NEED(TH);
    std::vector<double*> Q(nqq);
    for (int c = 0; c < nqq; c++) {
        Q[c] = slot(h, S_DYN + 4 * c);
        NEED(Q[c]);
    }
    double* OUT = slot(h, S_PSI_OUT);  // (4+nq)*(kp+2) <= n for the sizes used
    NEED(OUT);
    if ((4 + (size_t)nqq) * K2 > h->n) return fail(h, DCM_E_ARG, "horizontal_means: too many q");
    RC(upload(h, U, u)); RC(upload(h, V, v)); RC(upload(h, W, w)); RC(upload(h, TH, th));
    for (int c = 0; c < nqq; c++) RC(upload(h, Q[c], q + (size_t)c * h->nh));
    launch_means_div<double, double>(h->d, h->mt, U, V, W, TH, Q.data(), nqq, OUT, nullptr, h->partials,
                             h->ticket, h->st);
    CK(cudaGetLastError());
    RC(download(h, ubar, OUT, K2)); RC(download(h, vbar, OUT + K2, K2));
    RC(download(h, wbar, OUT + 2 * K2, K2)); RC(download(h, thbar, OUT + 3 * K2, K2));
    if (nqq) RC(download(h, qbar, OUT + 4 * K2, nqq * K2));
    return sync(h);
}

extern "C" int dcm_divergence_calc(dcm_handle* h, const double* u, const double* v,
                                   const double* w, double* div) {
    CHECK_H();
    if (!u || !v || !w || !div) return fail(h, DCM_E_ARG, "divergence_calc: bad argument");
    double *U = slot(h, S_U), *V = slot(h, S_V), *W = slot(h, S_W), *DV = slot(h, S_TH),
           *OUT = slot(h, S_PSI_OUT);
    NEED(U); NEED(V); NEED(W); NEED(DV); NEED(OUT);
    RC(upload(h, U, u)); RC(upload(h, V, v)); RC(upload(h, W, w)); RC(upload(h, DV, div));
    launch_means_div<double, double>(h->d, h->mt, U, V, W, W, nullptr, 0, OUT, DV, h->partials,
                             h->ticket, h->st);
    CK(cudaGetLastError());
    RC(download(h, div, DV));
    return sync(h);
}

extern "C" int dcm_advance_scalar_fields_3d(dcm_handle* h, double dt, double* q,
                                            const double* sq, double* th, const double* sth,
                                            int nq, int moisture) {
    CHECK_H();
    if (!th || !sth || (moisture && (!q || !sq || nq < 1)))
        return fail(h, DCM_E_ARG, "advance_scalar_fields_3d: bad argument");
    double *A = slot(h, S_TH), *S = slot(h, S_STH);
    NEED(A); NEED(S);
    RC(upload(h, A, th)); RC(upload(h, S, sth));
    launch_advance_scalar<double>(h->d, dt, A, S, h->st);
    RC(download(h, th, A));
    if (moisture) {
        for (int c = 0; c < nq; c++) {
            RC(upload(h, A, q + (size_t)c * h->nh)); RC(upload(h, S, sq + (size_t)c * h->nh));
            launch_advance_scalar<double>(h->d, dt, A, S, h->st);
            RC(download(h, q + (size_t)c * h->nh, A));
        }
    }
    CK(cudaGetLastError());
    return sync(h);
}

static int exchange_dropin(dcm_handle* h, double* a, int mode, double lbc, double ubc) {
    CHECK_H();
    if (!a) return fail(h, DCM_E_ARG, "exchange: bad argument");
    double* A = slot(h, S_TH);
    NEED(A);
    RC(upload(h, A, a));
    launch_exchange<double>(h->d, A, mode, lbc, ubc, h->st);
    CK(cudaGetLastError());
    RC(download(h, a, A));
    return sync(h);
}
extern "C" int dcm_exchange_full(dcm_handle* h, double* a, double lbc, double ubc) {
    return exchange_dropin(h, a, HALO_FULL, lbc, ubc);
}
extern "C" int dcm_exchange_along_dim(dcm_handle* h, double* a, double lbc, double ubc) {
    return exchange_dropin(h, a, HALO_DIM, lbc, ubc);
}
extern "C" int dcm_exchange_along_dim_wo(dcm_handle* h, double* a) {
    return exchange_dropin(h, a, HALO_WO, 0.0, 0.0);
}
extern "C" int dcm_exchange_full_wo(dcm_handle* h, double* a) {
    return exchange_dropin(h, a, HALO_FULL_WO, 0.0, 0.0);
}

// calculate_subgrid_3d (sgm/subgrid_3d.f90:38-357) on the caller's host arrays
extern "C" int dcm_calculate_subgrid_3d(dcm_handle* h, const double* lamsq, double z0,
                                        double z0th, const double* u, const double* v,
                                        const double* w, const double* zu, const double* zv,
                                        const double* zw, const double* th, int nq,
                                        const double* q, double* vism, double* vist,
                                        double* viss, double* strain, double* tau11,
                                        double* tau22, double* tau33, double* tau12,
                                        double* tau13, double* tau23, double* su, double* sv,
                                        double* sw, double* sth, double* sq, int moisture) {
    CHECK_H();
    double* out[13] = {vism, vist, strain, tau11, tau22, tau33, tau12, tau13, tau23,
                       su, sv, sw, sth};
    const double* in[7] = {u, v, w, zu, zv, zw, th};
    for (const double* a : in)
        if (!a) return fail(h, DCM_E_ARG, "calculate_subgrid_3d: missing input field");
    for (double* a : out)
        if (!a) return fail(h, DCM_E_ARG, "calculate_subgrid_3d: missing inout field");
    if (!lamsq || !(z0 > 0.0) || !(z0th > 0.0))
        return fail(h, DCM_E_ARG, "calculate_subgrid_3d: lamsq, z0 > 0 and z0th > 0 needed");
    if (moisture && (nq < 1 || !q || !viss || !sq))
        return fail(h, DCM_E_ARG, "calculate_subgrid_3d: moisture needs nq, q, viss, sq");
    if (h->h_zg.size() < 2)
        return fail(h, DCM_E_ARG, "calculate_subgrid_3d: the grid's zg is needed (z(1))");
    const size_t K2 = h->d.kp + 2;
    if (!h->sg_lamsq) CK(cudaMalloc(&h->sg_lamsq, K2 * sizeof(double)));
    CK(cudaMemcpyAsync(h->sg_lamsq, lamsq, K2 * sizeof(double), cudaMemcpyHostToDevice, h->st));
    const int in_slot[7] = {S_U, S_V, S_W, S_ZU, S_ZV, S_ZW, S_TH};
    double* I[7];
    for (int c = 0; c < 7; c++) {
        I[c] = slot(h, in_slot[c]);
        NEED(I[c]);
        RC(upload(h, I[c], in[c]));
    }
    double* O[13];
    for (int c = 0; c < 13; c++) {
        O[c] = c < 9 ? slot(h, S_SG + c) : slot(h, c == 9 ? S_SU : c == 10 ? S_SV
                                                      : c == 11 ? S_SW : S_STH);
        NEED(O[c]);
        RC(upload(h, O[c], out[c]));
    }
    const SgsParams<double> P{h->sg_lamsq, h->h_zg[1], z0, z0th};
    ScalarSet<double> set;
    make_scalar_sets<double>(I[6], O[12], 0, nullptr, nullptr, 0, 0, &set, 1);
    launch_subgrid<double>(h->d, h->mt, P, I[0], I[1], I[2], I[3], I[4], I[5], I[6], O[0], O[1],
                           O[2], O + 3, O[9], O[10], O[11], &set, 1, false, h->st);
    CK(cudaGetLastError());
    for (int c = 0; c < 13; c++) RC(download(h, out[c], O[c]));
    if (moisture) {
        // viss(:,:,:,n) = vist (:182-187); then each q's diffusion (:319-346)
        double *Q = slot(h, S_SG + 9), *SQ = slot(h, S_SG + 10);
        NEED(Q); NEED(SQ);
        for (int c = 0; c < nq; c++) {
            RC(download(h, viss + (size_t)c * h->nh, O[1]));
            RC(upload(h, Q, q + (size_t)c * h->nh));
            RC(upload(h, SQ, sq + (size_t)c * h->nh));
            make_scalar_sets<double>(Q, SQ, 0, nullptr, nullptr, 0, 0, &set, 1);
            launch_subgrid_scalars<double>(h->d, h->mt, O[1], &set, 1, h->st);
            CK(cudaGetLastError());
            RC(download(h, sq + (size_t)c * h->nh, SQ));
        }
    }
    return sync(h);
}

// =============================================================================
// device-resident time loop
// =============================================================================
namespace {

// n = 0: a pitched field; n > 0: n contiguous elements
template <typename T>
T* alloc_owned(dcm_handle* h, size_t n = 0) {
    T* raw = nullptr;
    const size_t cnt = n ? n : h->n + FIELD_PAD;
    if (cudaMalloc(&raw, cnt * sizeof(T)) != cudaSuccess) return nullptr;
    cudaMemsetAsync(raw, 0, cnt * sizeof(T), h->st);
    h->owned.push_back(raw);
    return n ? raw : raw + FIELD_SHIFT;
}

// velocity roles after n steps: (u, zu, tu) -> buffers (0,1,2), (2,0,1),
// (1,2,0) for n mod 3 = 0, 1, 2 (driver_code.f90:281-283, :634-646)
void roles_of(int phase, int& cu, int& cz, int& ct) {
    static const int RU[3] = {0, 2, 1}, RZ[3] = {1, 0, 2}, RT[3] = {2, 1, 0};
    const int m = phase % 3;
    cu = RU[m];
    cz = RZ[m];
    ct = RT[m];
}
void roles(const dcm_handle* h, int& cu, int& cz, int& ct) { roles_of(h->nstep, cu, cz, ct); }

template <typename T>
__global__ void k_driver_start(Dims d, T* zu, T* zv, T* zw) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j > d.jp + 1) return;
    zw[d.at(0, j, i)] = -zw[d.at(1, j, i)];  // driver_code.f90:288
    zu[d.at(1, j, i)] = T(0);
    zv[d.at(1, j, i)] = T(0);
    zw[d.at(d.kp, j, i)] = -zw[d.at(d.kp - 1, j, i)];  // :292-294
    zw[d.at(d.kp + 1, j, i)] = T(0);
    zu[d.at(d.kp, j, i)] = T(0);
    zv[d.at(d.kp, j, i)] = T(0);
}

template <typename T>
State<T>& state_of(dcm_handle* h);
template <>
State<double>& state_of<double>(dcm_handle* h) { return h->s64; }
template <>
State<float>& state_of<float>(dcm_handle* h) { return h->s32; }

template <typename T>
const Metrics<T>& metrics_of(dcm_handle* h);
template <>
const Metrics<double>& metrics_of<double>(dcm_handle* h) { return h->mt; }
template <>
const Metrics<float>& metrics_of<float>(dcm_handle* h) { return h->mtf; }

// MPDATA scratch in the field precision (slots for FP64, fslots for FP32)
template <typename T>
struct MpBufsT {
    MpdataWork<T> w;
    std::vector<T*> pa, pb;
};

template <typename T>
T* tslot(dcm_handle* h, int idx);
template <>
double* tslot<double>(dcm_handle* h, int idx) { return slot(h, idx); }
template <>
float* tslot<float>(dcm_handle* h, int idx) { return fslot(h, idx); }

template <typename T>
bool mpdata_work_t(dcm_handle* h, int nq, MpBufsT<T>& b) {
    b.pa.resize(nq);
    b.pb.resize(nq);
    for (int q = 0; q < nq; q++) {
        b.pa[q] = tslot<T>(h, S_DYN + 4 * q + 2);
        b.pb[q] = tslot<T>(h, S_DYN + 4 * q + 3);
        if (!b.pa[q] || !b.pb[q]) return false;
    }
    b.w.pa = b.pa.data();
    b.w.pb = b.pb.data();
    const int va[3] = {S_VA0, S_VA1, S_VA2}, vl[3] = {S_VL0, S_VL1, S_VL2};
    for (int c = 0; c < 3; c++) {
        b.w.va[c] = tslot<T>(h, va[c]);
        b.w.vl[c] = tslot<T>(h, vl[c]);
        if (!b.w.va[c] || !b.w.vl[c]) return false;
    }
    const int bt[6] = {S_B0, S_B1, S_B2, S_B3, S_B4, S_B5};
    for (int c = 0; c < 6; c++) {
        b.w.beta[c] = tslot<T>(h, bt[c]);
        if (!b.w.beta[c]) return false;
    }
    b.w.partials = h->partials;
    b.w.ticket = h->ticket;
    b.w.M = h->M;
    b.w.Mone = h->M + NQMAX;
    b.w.Mzero = h->M + NQMAX + 1;
    b.w.fuse = h->mp_fuse;
    b.w.fuse_rows = h->mp_rows;
    return true;
}

SolverWork<float> solver_work_f(dcm_handle* h) {
    SolverWork<float> w;
    w.r = fslot(h, S_R); w.cr = fslot(h, S_CR); w.p = fslot(h, S_PP); w.v1 = fslot(h, S_V1);
    w.t = fslot(h, S_T); w.sA = fslot(h, S_SA); w.sB = fslot(h, S_SB);
    w.rh = fslot(h, S_RH); w.vh = fslot(h, S_VH);
    w.ae = h->aef; w.aw = h->awf; w.an = h->anf; w.as = h->asf; w.au = h->auf; w.ad = h->adf;
    w.partials = h->partials; w.ticket = h->ticket; w.S = h->S2;
    w.red.partials = h->partials; w.red.gpartials = h->gpartials; w.red.gtick = h->gtick;
    w.red.ticket = h->ticket2;
    w.graph = h->graphs ? &h->g32 : nullptr;
    w.pdl = h->graphs == 1;
    w.by = h->tune_by[1];
    w.tasks = h->tune_tasks[1];
    w.ni = h->tune_ni[1];
    w.fuse = h->tune_fuse[1];
    w.vw = h->tune_vec[1];
    w.max_blocks = (int)std::min<size_t>(h->npartials / 3, (size_t)1 << 30);
    w.cheb = h->cfg.precond == 1 ? 1 : 0;
    w.cheb_lo = h->cfg.precond_lo > 0.0 ? h->cfg.precond_lo : 0.05;
    w.round_budget = h->round_budget;
    return w;
}

template <typename T>
Forcing<T> forcing_t(dcm_handle* h);
template <>
Forcing<double> forcing_t<double>(dcm_handle* h) {
    const size_t K2 = h->d.kp + 2;
    Forcing<double> F{};
    const dcm_config& c = h->cfg;
    F.damping_layer = c.forcing.damping_layer;
    F.forcing = c.forcing.forcing;
    F.divergence = c.forcing.divergence;
    F.forcing_tau = c.forcing.forcing_tau;
    double* f = h->forcing_dev;
    F.dampfacn = f; F.dampfac = f + K2; F.u_force = f + 2 * K2; F.v_force = f + 3 * K2;
    F.w_subs = f + 4 * K2;
    return F;
}
template <>
Forcing<float> forcing_t<float>(dcm_handle* h) {
    const size_t K2 = h->d.kp + 2;
    Forcing<float> F{};
    const dcm_config& c = h->cfg;
    F.damping_layer = c.forcing.damping_layer;
    F.forcing = c.forcing.forcing;
    F.divergence = c.forcing.divergence;
    F.forcing_tau = (float)c.forcing.forcing_tau;
    float* f = h->forcing_f;
    F.dampfacn = f; F.dampfac = f + K2; F.u_force = f + 2 * K2; F.v_force = f + 3 * K2;
    F.w_subs = f + 4 * K2;
    return F;
}

// One pass of the time loop (driver_code.f90:304-676) with fields in T and
// the pressure in FP64, on stream `st` with the velocity roles of `phase`
// (= steps taken mod 3).  emit = false: run it (the pressure solve as its own
// graph, host reads of the solver scalars).  emit = true: `st` is capturing
// a larger graph (an ensemble time step) and the step, its solve included,
// is only recorded into it: no host synchronisation, no host state changes.
template <typename T>
int step_body(dcm_handle* h, cudaStream_t st, int phase, bool emit) {
    const Dims& d = h->d;
    const dcm_config& c = h->cfg;
    State<T>& S = state_of<T>(h);
    const Metrics<T>& mt = metrics_of<T>(h);
    const size_t K2 = d.kp + 2;
    int cu, cz, ct;
    roles_of(phase, cu, cz, ct);
    T *u = S.U[cu], *v = S.V[cu], *w = S.W[cu];
    T *zu = S.U[cz], *zv = S.V[cz], *zw = S.W[cz];
    T *tu = S.U[ct], *tv = S.V[ct], *tw = S.W[ct];
    const int nqq = c.moisture ? c.nq : 0;
    const T dt = (T)c.dt;
    // horizontal_means + divergence_calc (FP64 divergence), driver_code.f90:433-444
    launch_means_div<T, double>(d, h->mt, u, v, w, S.th, S.q.data(), nqq, S.means, h->div,
                                h->partials, h->ticket, st);
    // sources (sth = 0 first, :340) + exchange_along_dim_wo(psrc), :455-487
    const Forcing<T> F = forcing_t<T>(h);
    const T* ubar = S.means;
    // viscous: the subgrid model inside sources (dynamics.f90:878-893)
    SgsStep<T> sg{};
    if (c.viscous) {
        sg.P = SgsParams<T>{S.lamsq, h->h_zg[1], c.z0, c.z0th};
        sg.vism = S.vism;
        sg.vist = S.vist;
        sg.strain = S.strain;
        sg.tau = S.tau;
        sg.q = S.q.data();
        sg.sq = S.sq.data();
        sg.nq = nqq;
    }
    launch_sources<T, double>(d, mt, h->mt, F, ubar, ubar + K2, ubar + 2 * K2, ubar + 3 * K2, zu,
                              zv, zw, u, v, w, S.th, S.su, S.sv, S.sw, S.sth, h->psrc, 1, 1,
                              st, c.viscous ? &sg : nullptr);
    CK(cudaGetLastError());
    // pressure: bicgstab + exchange_along_dim_wo(p), :496-507
    if (!emit) h->first_call = 0;
    int rc;
    if constexpr (std::is_same<T, double>::value) {
        SolverWork<double> swd = solver_work(h);
        NEED(swd.r); NEED(swd.sB); NEED(swd.rh); NEED(swd.vh);
        if (emit) {
            swd.graph = &h->g64;
            swd.emit = true;
        }
        rc = solver_run<double>(swd, d, h->p, h->psrc, S.sw, h->mt.dzn, c.ptol, c.itmax, 1, 4,
                                st, h->hS, nullptr);
        if (!emit) {
            h->last_iters = h->hS->it;
            h->last_err = h->hS->err;
        }
    } else {
        SolverWork<double> swd = solver_scalars(h);
        SolverWork<float> swf = solver_work_f(h);
        NEED(swf.r); NEED(swf.sB); NEED(swf.rh); NEED(swf.vh);
        if (emit) {
            swf.graph = &h->g32;
            swf.emit = true;
        }
        float* dx = fslot(h, S_B);
        NEED(dx);
        rc = refine_run(swf, swd, d, h->p, h->psrc, S.sw, h->mt.dzn, dx, c.ptol,
                        c.inner_tol > 0 ? c.inner_tol : 0.1, c.itmax, 1000, st, h->hS,
                        h->hS2, &h->last_refine);
        if (!emit) {
            h->last_iters = h->last_refine.inner;
            h->last_err = h->last_refine.err;
            h->refine_outer_total += h->last_refine.outer;
        }
    }
    if (rc != DCM_OK) {
        h->err = dcm_status_string(rc);
        return rc;
    }
    // scalar advection, :514-560, with advance_scalar_fields_3d (:601) fused
    MpBufsT<T> mb;
    if (!mpdata_work_t<T>(h, std::max(1, nqq), mb))
        return fail(h, DCM_E_CUDA, "device allocation");
    if (c.advection_scheme == 0 || c.advection_scheme == 1)
        launch_adv_ref_state<T>(d, mt, dt, w, S.th, S.th2, mt.thetan, 1, st);
    if (c.advection_scheme == 1) {
        double lb = h->t1, ub = h->t2;
        T* pin = S.th2;
        T* pout = S.th;
        const T* sadd = S.sth;
        RC(mpdata_run<T>(mb.w, d, mt, dt, u, v, w, &pin, &pout, 1, &lb, &ub, c.kord, c.monotone,
                         0, c.limiter, false, &sadd, dt, st));
        // t1, t2 return as (t - m) + m, which is exactly t when t = 0
        if (h->t1 != 0.0 || h->t2 != 0.0) {
            if (emit) return fail(h, DCM_E_UNSUPPORTED, "captured step: t1, t2 must be 0");
            CK(cudaMemcpyAsync(h->hM, h->M, sizeof(MpScalars), cudaMemcpyDeviceToHost, st));
            RC(sync(h));
            h->t1 = h->hM[0].lbc + h->hM[0].m;
            h->t2 = h->hM[0].ubc + h->hM[0].m;
        }
    } else if (c.advection_scheme == 0) {
        // donor cell + exchange_full(th, t1, t2), :539-545, then th += sth*dt
        CK(cudaMemcpyAsync(S.th, S.th2, h->n * sizeof(T), cudaMemcpyDeviceToDevice, st));
        RC(upwind_run<T>(mb.w, d, mt, dt, u, v, w, S.th2, S.th, 0, st));
        launch_exchange<T>(d, S.th, HALO_FULL, (T)h->t1, (T)h->t2, st);
        launch_advance_scalar<T>(d, dt, S.th, S.sth, st);
    } else if (c.advection_scheme == 2) {
        if (emit) return fail(h, DCM_E_UNSUPPORTED, "captured step: advection_scheme 2");
        // mpdata_3d_add with thetan, thbase, thtop, :552-556
        double lb = c.thbase, ub = c.thtop;
        launch_add_profile<T>(d, S.th, mt.thetan, T(1), st);
        T* pin = S.th;
        T* pout = S.th2;
        RC(mpdata_run<T>(mb.w, d, mt, dt, u, v, w, &pin, &pout, 1, &lb, &ub, c.kord, c.monotone,
                         0, c.limiter, false, nullptr, T(0), st));
        launch_add_profile<T>(d, S.th2, mt.thetan, T(-1), st);
        launch_advance_scalar<T>(d, dt, S.th2, S.sth, st);
        std::swap(S.th, S.th2);
    } else {
        return fail(h, DCM_E_UNSUPPORTED, "advection_scheme");
    }
    // q categories, :568-585, then q += sq*dt
    if (nqq && emit) return fail(h, DCM_E_UNSUPPORTED, "captured step: moisture");
    if (nqq) {
        for (int cat = 0; cat < c.ncat; cat++) {
            const int a = h->cs[cat] - 1, b = h->ce[cat] - 1;
            const int nc = b - a + 1;
            std::vector<T*> qin(nc), qout(nc);
            std::vector<const T*> sadd(nc);
            for (int e = 0; e < nc; e++) {
                // the current q becomes the read-only input; the result goes
                // to the other buffer of the pair (no copy)
                std::swap(S.q[a + e], S.qtmp[a + e]);
                qin[e] = S.qtmp[a + e];
                qout[e] = S.q[a + e];
                sadd[e] = S.sq[a + e];
            }
            RC(mpdata_run<T>(mb.w, d, mt, dt, u, v, w, qin.data(), qout.data(), nc,
                             h->q1.data() + a, h->q2.data() + a, c.kord, c.monotone, 0, c.limiter,
                             true, sadd.data(), dt, st));
        }
    }
    // advance_momentum(2dt) + time filter + rotation + exchange + rows, :592-674
    launch_momentum_step<T, double>(d, mt, h->mt, (T)(2.0 * c.dt), u, v, w, zu, zv, zw, tu, tv,
                                    tw, S.su, S.sv, S.sw, h->p, st);
    CK(cudaGetLastError());
    return DCM_OK;
}

template <typename T>
int one_step(dcm_handle* h) {
    RC(step_body<T>(h, h->st, h->nstep % 3, false));
    h->nstep += 1;
    return DCM_OK;
}

// host double field -> device field of precision T (through the dense
// staging buffer; the caller synchronises once at the end)
template <typename T>
int put_field(dcm_handle* h, T* dst, const double* src) {
    return upload_field<T>(h, dst, src);
}
template <typename T>
int get_field(dcm_handle* h, double* dst, const T* src, size_t n = 0) {
    if (!dst) return DCM_OK;
    if constexpr (std::is_same<T, double>::value) return download(h, dst, src, n);
    double* stage = slot(h, S_STAGE);
    NEED(stage);
    // the staging slot is reused by the next field; the stream orders that
    // field's conversion after this copy, so no host synchronisation here
    launch_convert<double, T>(n ? n : h->n, stage, src, h->st);
    RC(download(h, dst, stage, n));
    return DCM_OK;
}

// A resident buffer of an earlier upload with the same layout is zeroed and
// kept (the state it then holds is the one a fresh allocation would give);
// otherwise a new zeroed buffer.  Keeping the buffers keeps the pointers that
// the captured pressure solves were built on.
template <typename U>
bool reuse_or_alloc(dcm_handle* h, U*& ptr, size_t n = 0) {
    if (ptr) {
        U* raw = n ? ptr : ptr - FIELD_SHIFT;
        return cudaMemsetAsync(raw, 0, (n ? n : h->n + FIELD_PAD) * sizeof(U), h->st) ==
               cudaSuccess;
    }
    ptr = alloc_owned<U>(h, n);
    return ptr != nullptr;
}

template <typename T>
int upload_state_t(dcm_handle* h, const dcm_fields* f, const double* lamsq_host) {
    State<T>& S = state_of<T>(h);
    const dcm_config& cfg = h->cfg;
    const int nqq = cfg.moisture ? cfg.nq : 0;
    const double* in3[9] = {f->u, f->zu, f->tu, f->v, f->zv, f->tv, f->w, f->zw, f->tw};
    T** dst3[9] = {&S.U[0], &S.U[1], &S.U[2], &S.V[0], &S.V[1],
                   &S.V[2], &S.W[0], &S.W[1], &S.W[2]};
    for (int c = 0; c < 9; c++) {
        if (!in3[c]) return fail(h, DCM_E_ARG, "state_upload: missing velocity");
        if (!reuse_or_alloc(h, *dst3[c])) return fail(h, DCM_E_CUDA, "device allocation failed");
        RC(put_field<T>(h, *dst3[c], in3[c]));
    }
    T** fl[6] = {&S.th, &S.th2, &S.su, &S.sv, &S.sw, &S.sth};
    for (auto pp : fl)
        if (!reuse_or_alloc(h, *pp)) return fail(h, DCM_E_CUDA, "device allocation failed");
    if (!f->th || !f->p) return fail(h, DCM_E_ARG, "state_upload: missing th or p");
    const double* src[5] = {f->th, f->su, f->sv, f->sw, f->sth};
    T* dst[5] = {S.th, S.su, S.sv, S.sw, S.sth};
    for (int c = 0; c < 5; c++) {
        RC(put_field<T>(h, dst[c], src[c]));
    }
    const size_t K2 = h->d.kp + 2;
    if (!reuse_or_alloc(h, S.means, (4 + nqq) * K2))
        return fail(h, DCM_E_CUDA, "device allocation failed");
    S.q.resize(nqq, nullptr);
    S.sq.resize(nqq, nullptr);
    S.qtmp.resize(nqq, nullptr);
    for (int c = 0; c < nqq; c++) {
        if (!reuse_or_alloc(h, S.q[c]) || !reuse_or_alloc(h, S.sq[c]) ||
            !reuse_or_alloc(h, S.qtmp[c]))
            return fail(h, DCM_E_CUDA, "device allocation failed");
        // sq is zeroed by the driver each step (:342); without the subgrid
        // model nothing in the dry step writes it, so it stays zero
        RC(put_field<T>(h, S.q[c], f->q + (size_t)c * h->nh));
    }
    if constexpr (std::is_same<T, float>::value) {
        launch_convert<float, double>(5 * K2, h->forcing_f, h->forcing_dev, h->st);
    }
    if (cfg.viscous) {
        // vism, vist, strain and the stresses are recomputed every step
        // (their previous values are never read); lamsq in the field precision
        T** sg[9] = {&S.vism, &S.vist, &S.strain, &S.tau[0], &S.tau[1],
                     &S.tau[2], &S.tau[3], &S.tau[4], &S.tau[5]};
        for (auto pp : sg)
            if (!reuse_or_alloc(h, *pp)) return fail(h, DCM_E_CUDA, "device allocation failed");
        if (!reuse_or_alloc(h, S.lamsq, K2) || !reuse_or_alloc(h, S.lamsq64, K2))
            return fail(h, DCM_E_CUDA, "device allocation failed");
        double* l64 = S.lamsq64;
        RC(upload(h, l64, lamsq_host, K2));
        if constexpr (std::is_same<T, float>::value)
            launch_convert<float, double>(K2, S.lamsq, l64, h->st);
        else
            CK(cudaMemcpyAsync(S.lamsq, l64, K2 * sizeof(double), cudaMemcpyDeviceToDevice,
                               h->st));
    }
    return DCM_OK;
}

template <typename T>
int download_state_t(dcm_handle* h, dcm_fields* f) {
    State<T>& S = state_of<T>(h);
    int cu, cz, ct;
    roles(h, cu, cz, ct);
    RC(get_field<T>(h, f->u, S.U[cu])); RC(get_field<T>(h, f->v, S.V[cu]));
    RC(get_field<T>(h, f->w, S.W[cu]));
    RC(get_field<T>(h, f->zu, S.U[cz])); RC(get_field<T>(h, f->zv, S.V[cz]));
    RC(get_field<T>(h, f->zw, S.W[cz]));
    RC(get_field<T>(h, f->tu, S.U[ct])); RC(get_field<T>(h, f->tv, S.V[ct]));
    RC(get_field<T>(h, f->tw, S.W[ct]));
    RC(get_field<T>(h, f->th, S.th));
    RC(download(h, f->p, h->p));
    RC(get_field<T>(h, f->su, S.su)); RC(get_field<T>(h, f->sv, S.sv));
    RC(get_field<T>(h, f->sw, S.sw));
    RC(download(h, f->psrc, h->psrc));
    RC(download(h, f->div, h->div));
    RC(get_field<T>(h, f->sth, S.sth));
    const size_t K2 = h->d.kp + 2;
    RC(get_field<T>(h, f->ubar, S.means, K2));
    RC(get_field<T>(h, f->vbar, S.means + K2, K2));
    RC(get_field<T>(h, f->wbar, S.means + 2 * K2, K2));
    RC(get_field<T>(h, f->thbar, S.means + 3 * K2, K2));
    const int nqq = h->cfg.moisture ? h->cfg.nq : 0;
    if (nqq && f->qbar) {
        if constexpr (std::is_same<T, double>::value) {
            RC(download(h, f->qbar, S.means + 4 * K2, nqq * K2));
        } else {
            RC(get_field<T>(h, f->qbar, S.means + 4 * K2, nqq * K2));
        }
    }
    for (int c = 0; c < nqq; c++) {
        if (f->q) RC(get_field<T>(h, f->q + (size_t)c * h->nh, S.q[c]));
        if (f->sq) RC(get_field<T>(h, f->sq + (size_t)c * h->nh, S.sq[c]));
    }
    return sync(h);
}

}  // namespace

extern "C" int dcm_state_upload(dcm_handle* h, const dcm_config* cfg, const dcm_fields* f) {
    CHECK_H();
    if (!cfg || !f) return fail(h, DCM_E_ARG, "state_upload: bad argument");
    if (cfg->precision != 0 && cfg->precision != 1)
        return fail(h, DCM_E_UNSUPPORTED, "precision must be 0 (FP64) or 1 (mixed)");
    if (cfg->advection_scheme < 0 || cfg->advection_scheme > 2 || cfg->itmax < 1 || cfg->dt <= 0)
        return fail(h, DCM_E_ARG, "state_upload: bad config");
    if (cfg->moisture && (cfg->nq < 1 || cfg->nq > NQMAX || cfg->ncat < 1 || !cfg->c_s ||
                          !cfg->c_e || !f->q))
        return fail(h, DCM_E_ARG, "state_upload: bad moisture config");
    if (cfg->precond != 0 && cfg->precond != 1)
        return fail(h, DCM_E_ARG, "state_upload: precond must be 0 or 1");
    if (cfg->precond == 1 && !(cfg->precond_lo >= 0.0 && cfg->precond_lo < 2.0))
        return fail(h, DCM_E_ARG, "state_upload: precond_lo must lie in [0, 2)");
    if (cfg->viscous && (!cfg->lamsq || !(cfg->z0 > 0.0) || !(cfg->z0th > 0.0)))
        return fail(h, DCM_E_ARG, "state_upload: viscous needs lamsq, z0 > 0 and z0th > 0");
    if (cfg->viscous && h->h_zg.size() < 2)
        return fail(h, DCM_E_ARG, "state_upload: viscous needs the grid's zg (z(1))");
    // buffers of the resident state are kept when the layout is the same
    // (no cudaFree, which synchronises the device; the captured solves stay
    // valid); a changed layout frees them
    const bool same_layout = h->resident && h->prec == cfg->precision &&
                             (h->cfg.moisture ? h->cfg.nq : 0) ==
                                 (cfg->moisture ? cfg->nq : 0) &&
                             (h->cfg.viscous != 0) == (cfg->viscous != 0);
    if (!same_layout) free_state(h);
    h->cfg = *cfg;
    h->cfg.lamsq = nullptr;  // copied to the device below; no host pointer is kept
    h->prec = cfg->precision;
    const int nqq = cfg->moisture ? cfg->nq : 0;
    if (nqq) {
        h->cs.assign(cfg->c_s, cfg->c_s + cfg->ncat);
        h->ce.assign(cfg->c_e, cfg->c_e + cfg->ncat);
        for (int c = 0; c < cfg->ncat; c++)
            if (h->cs[c] < 1 || h->ce[c] > nqq || h->ce[c] < h->cs[c])
                return fail(h, DCM_E_ARG, "state_upload: bad category bounds");
        h->cfg.c_s = h->cs.data();
        h->cfg.c_e = h->ce.data();
    }
    int rc = DCM_OK;
    forcing_of(h, &cfg->forcing, h->forcing_dev, &rc);
    if (rc != DCM_OK) return fail(h, rc, "state_upload: forcing arrays");
    h->nstep = 0;
    if (!reuse_or_alloc(h, h->p) || !reuse_or_alloc(h, h->div) || !reuse_or_alloc(h, h->psrc))
        return fail(h, DCM_E_CUDA, "device allocation failed");
    RC(upload(h, h->p, f->p));
    RC(upload(h, h->div, f->div));
    RC(upload(h, h->psrc, f->psrc));
    RC(h->prec == 0 ? upload_state_t<double>(h, f, cfg->lamsq)
                    : upload_state_t<float>(h, f, cfg->lamsq));
    h->q1.assign(nqq, 0.0);  // driver_code.f90:275-276
    h->q2.assign(nqq, 0.0);
    h->t1 = h->t2 = 0.0;  // saved locals, :260
    h->refine_outer_total = 0;
    h->resident = true;
    h->generation += 1;
    return sync(h);
}

extern "C" int dcm_driver_start(dcm_handle* h) {
    CHECK_H();
    if (!h->resident) return fail(h, DCM_E_ARG, "driver_start: no state");
    int cu, cz, ct;
    roles(h, cu, cz, ct);
    const dim3 g((h->d.J + 127) / 128, h->d.I);
    if (h->prec == 0)
        k_driver_start<double><<<g, 128, 0, h->st>>>(h->d, h->s64.U[cz], h->s64.V[cz],
                                                     h->s64.W[cz]);
    else
        k_driver_start<float><<<g, 128, 0, h->st>>>(h->d, h->s32.U[cz], h->s32.V[cz],
                                                    h->s32.W[cz]);
    CK(cudaGetLastError());
    return sync(h);
}

extern "C" int dcm_step(dcm_handle* h, int nsteps, dcm_step_stats* stats) {
    CHECK_H();
    if (!h->resident || nsteps < 0) return fail(h, DCM_E_ARG, "step: no state");
    long long tot = 0;
    g_prof = &h->prof;
    CK(cudaEventRecord(h->ev0, h->st));
    int done = 0;
    int rc = DCM_OK;
    for (; done < nsteps; done++) {
        rc = h->prec == 0 ? one_step<double>(h) : one_step<float>(h);
        tot += h->last_iters;
        if (rc != DCM_OK) break;
    }
    CK(cudaEventRecord(h->ev1, h->st));
    CK(cudaEventSynchronize(h->ev1));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, h->ev0, h->ev1);
    if (h->prof.on) h->prof.harvest();
    g_prof = nullptr;
    if (stats) {
        stats->steps = done;
        stats->iters_last = h->last_iters;
        stats->iters_total = tot;
        stats->err_last = h->last_err;
        stats->ms_total = ms;
        stats->updates_last = h->prec ? h->last_refine.outer : 0;
        stats->restarts_last = h->prec ? h->last_refine.restarts : 0;
    }
    return rc;
}

extern "C" int dcm_state_download(dcm_handle* h, dcm_fields* f) {
    CHECK_H();
    if (!h->resident || !f) return fail(h, DCM_E_ARG, "state_download: no state");
    return h->prec == 0 ? download_state_t<double>(h, f) : download_state_t<float>(h, f);
}

// =============================================================================
// diagnostics
// =============================================================================
extern "C" int dcm_solver_graphs(dcm_handle* h, int on) {
    CHECK_H();
    const int mode = on == 0 ? 0 : on == 2 ? 2 : 1;
    if (mode != h->graphs) h->generation += 1;  // an ensemble recaptures its steps
    h->graphs = mode;
    return DCM_OK;
}

extern "C" int dcm_set_small_solver(dcm_handle* h, int max_points) {
    CHECK_H();
    if (max_points < 0) return fail(h, DCM_E_ARG, "set_small_solver: max_points");
    if (max_points != h->small_max) h->generation += 1;
    h->small_max = max_points;
    return DCM_OK;
}

extern "C" int dcm_set_mpdata_shape(dcm_handle* h, int fuse, int max_rows) {
    CHECK_H();
    if (max_rows < 3 || max_rows > 32) return fail(h, DCM_E_ARG, "set_mpdata_shape: max_rows");
    const int f = fuse ? 1 : 0;
    if (f != h->mp_fuse || max_rows != h->mp_rows) h->generation += 1;
    h->mp_fuse = f;
    h->mp_rows = max_rows;
    return DCM_OK;
}

extern "C" int dcm_solver_limits(dcm_handle* h, int max_rounds, double tiny) {
    CHECK_H();
    if (max_rounds < 0 || !(tiny == tiny)) return fail(h, DCM_E_ARG, "solver_limits");
    if (max_rounds != h->round_budget || tiny != h->tiny) h->generation += 1;
    h->round_budget = max_rounds;
    h->tiny = tiny < 0.0 ? -1.0 : tiny;
    return DCM_OK;
}

extern "C" int dcm_solver_graph_info(dcm_handle* h, int* programmatic) {
    CHECK_H();
    if (!programmatic) return DCM_E_ARG;
    *programmatic = h->graphs == 1 && solver_pdl_available() ? 1 : 0;
    return DCM_OK;
}

extern "C" int dcm_profile_enable(dcm_handle* h, int on) {
    CHECK_H();
    h->prof.reset();
    h->prof.on = on != 0;
    return DCM_OK;
}

extern "C" int dcm_profile_read(dcm_handle* h, double* ms, long long* launches, int ncat) {
    CHECK_H();
    if (!ms || !launches || ncat < P_NCAT) return fail(h, DCM_E_ARG, "profile_read: ncat");
    for (int c = 0; c < P_NCAT; c++) {
        ms[c] = h->prof.ms[c];
        launches[c] = h->prof.count[c];
    }
    return DCM_OK;
}

// =============================================================================
// solver launch-shape autotuner (no counterpart in the reference)
// =============================================================================
namespace {

std::string tune_cache_path() {
    if (const char* p = std::getenv("DCM_TUNE_CACHE")) return p;
    const char* home = std::getenv("HOME");
    return std::string(home ? home : ".") + "/.cache/dcm_b200_solver_tune.txt";
}

// cache lines: "<sms> <ip> <jp> <kp> <precision> <by> <tasks> <depth> <fuse> <vec>
// <ms per iteration> v2" (lines without the v2 tag, from before the vector
// width was tuned, are ignored)
bool tune_lookup(int sms, const Dims& d, int prec, int* by, int* tasks, int* depth, int* fuse,
                 int* vec) {
    std::ifstream f(tune_cache_path());
    std::string line;
    bool found = false;
    while (std::getline(f, line)) {
        std::istringstream is(line);
        int a[10];
        double ms;
        std::string tag;
        if (!(is >> a[0] >> a[1] >> a[2] >> a[3] >> a[4] >> a[5] >> a[6] >> a[7] >> a[8] >> a[9] >>
              ms >> tag) ||
            tag != "v2")
            continue;
        if (a[0] == sms && a[1] == d.ip && a[2] == d.jp && a[3] == d.kp && a[4] == prec) {
            *by = a[5];
            *tasks = a[6];
            *depth = a[7];
            *fuse = a[8];
            *vec = a[9];
            found = true;  // the last entry wins
        }
    }
    return found;
}

void tune_store(int sms, const Dims& d, int prec, int by, int tasks, int depth, int fuse, int vec,
                double ms) {
    std::ofstream f(tune_cache_path(), std::ios::app);
    if (f) f << sms << ' ' << d.ip << ' ' << d.jp << ' ' << d.kp << ' ' << prec << ' ' << by << ' '
             << tasks << ' ' << depth << ' ' << fuse << ' ' << vec << ' ' << ms << " v2\n";
}

template <typename T>
__global__ void k_tune_rhs(Dims d, T* b, T* x) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    // hashed noise in [-1, 1): every mode of the operator is present, so the
    // solve cannot finish early (a single eigenmode would converge in one
    // iteration and then break down); x starts at zero
    unsigned int hsh = (unsigned)k * 73856093u ^ (unsigned)j * 19349663u ^ (unsigned)i * 83492791u;
    hsh ^= hsh >> 13;
    hsh *= 0x5bd1e995u;
    hsh ^= hsh >> 15;
    b[d.at(k, j, i)] = (T)((double)(hsh & 0xffffffu) / 8388608.0 - 1.0);
    x[d.at(k, j, i)] = T(0);
}

// device time of `iters` iterations of the solver in precision T with the
// given launch shape (graph-driven, tolerance unreachable, itmax = iters)
template <typename T>
double tune_time(dcm_handle* h, int by, int tasks, int depth, int fuse, int vec, int iters) {
    SolverWork<T> w;
    T *x, *b;
    if constexpr (std::is_same<T, double>::value) {
        w = solver_work(h);
        x = slot(h, S_X);
        b = slot(h, S_RHS);
    } else {
        w = solver_work_f(h);
        x = fslot(h, S_X);
        b = fslot(h, S_RHS);
    }
    if (!x || !b || !w.r || !w.sB || !w.rh || !w.vh) return -1.0;
    SolveGraph G;
    w.graph = &G;
    w.by = by;
    w.tasks = tasks;
    w.ni = depth;
    w.fuse = fuse;
    w.vw = std::is_same<T, float>::value ? vec : 0;
    const Metrics<T>& mt = metrics_of<T>(h);
    double best = 1e30;
    for (int rep = 0; rep < 3; rep++) {
        k_tune_rhs<T><<<interior_grid(h->d, h->d.kp), dim3(BX, BY), 0, h->st>>>(h->d, b, x);
        cudaEventRecord(h->ev0, h->st);
        // tolerance out of reach: exactly `iters` iterations, ending NOCONV
        const int rc = solver_run<T>(w, h->d, x, b, x, mt.dzn, 1e-300, iters, 0, 4, h->st, h->hS,
                                     nullptr, 0.01, false);
        if (rc != DCM_E_NOCONV || h->hS->it != iters) return -1.0;
        cudaEventRecord(h->ev1, h->st);
        cudaEventSynchronize(h->ev1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, h->ev0, h->ev1);
        if (rep > 0) best = std::min(best, (double)ms / iters);  // rep 0 builds the graph
    }
    return cudaGetLastError() == cudaSuccess ? best : -1.0;
}

}  // namespace

extern "C" int dcm_tune(dcm_handle* h, int precision, int use_cache, int* by, int* tasks,
                        int* depth, int* fuse, int* vec) {
    CHECK_H();
    if (precision != 0 && precision != 1) return fail(h, DCM_E_ARG, "tune: precision");
    int sms = 0;
    CK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, h->device));
    int b0 = 8, t0 = 0, n0 = 4, f0 = 0, v0 = precision == 1 ? 4 : 2;
    if (!(use_cache && tune_lookup(sms, h->d, precision, &b0, &t0, &n0, &f0, &v0))) {
        static const int BYS[3] = {2, 4, 8}, TASKS[3] = {0, 1, 2}, DEPTHS[4] = {1, 2, 4, 8};
        double best = 1e30;
        auto consider = [&](int bv, int tv, int nv, int fv, int vv) -> bool {
            const double ms = precision == 0 ? tune_time<double>(h, bv, tv, nv, 0, 0, 12)
                                             : tune_time<float>(h, bv, tv, nv, fv, vv, 12);
            if (ms < 0) return false;
            if (ms < best) {
                best = ms;
                b0 = bv;
                t0 = tv;
                n0 = nv;
                f0 = fv;
                v0 = vv;
            }
            return true;
        };
        // FP32: 16-byte (4 levels per lane) and 8-byte (2 levels) vectors of
        // the separate kernels; FP64 keeps 16-byte vectors (2 levels)
        const int nvec = precision == 1 ? 2 : 1;
        for (int vi = 0; vi < nvec; vi++) {
            const int vv = precision == 1 ? (vi == 0 ? 4 : 2) : 2;
            for (int bi = 0; bi < 3; bi++)
                for (int ti = 0; ti < 3; ti++)
                    for (int ni = 0; ni < 4; ni++)
                        if (!consider(BYS[bi], TASKS[ti], DEPTHS[ni], 0, vv))
                            return fail(h, DCM_E_CUDA, "tune: a candidate launch shape failed");
        }
        // the fused preconditioner (FP32, 16-byte vectors), without (1) and
        // with (2) phase C's matvec as its fourth stage: the sweep shape does
        // not apply; the depth is the march of the reducing kernels
        if (precision == 1)
            for (int fv = 1; fv <= 2; fv++)
                for (int ti = 0; ti < 3; ti++)
                    for (int ni = 0; ni < 4; ni++)
                        if (!consider(8, TASKS[ti], DEPTHS[ni], fv, 4))
                            return fail(h, DCM_E_CUDA, "tune: a candidate launch shape failed");
        tune_store(sms, h->d, precision, b0, t0, n0, f0, v0, best);
    }
    h->tune_by[precision] = b0;
    h->tune_tasks[precision] = t0;
    h->tune_ni[precision] = n0;
    h->tune_fuse[precision] = precision == 1 ? f0 : 0;
    h->tune_vec[precision] = precision == 1 ? v0 : 2;
    h->generation += 1;
    if (by) *by = b0;
    if (tasks) *tasks = t0;
    if (depth) *depth = n0;
    if (fuse) *fuse = h->tune_fuse[precision];
    if (vec) *vec = h->tune_vec[precision];
    return DCM_OK;
}

extern "C" int dcm_set_launch_shape(dcm_handle* h, int precision, int by, int tasks, int depth,
                                    int fuse, int vec) {
    CHECK_H();
    if ((precision != 0 && precision != 1) || by < 1 || by > 8 || tasks < 0 || tasks > 15 ||
        depth < 1 || depth > 63 || fuse < 0 || fuse > 2 ||
        (precision == 1 ? (vec != 2 && vec != 4) : vec != 2) || (fuse && vec != 4))
        return fail(h, DCM_E_ARG, "set_launch_shape: bad argument");
    h->tune_by[precision] = by;
    h->tune_tasks[precision] = tasks;
    h->tune_ni[precision] = depth;
    h->tune_fuse[precision] = precision == 1 ? fuse : 0;
    h->tune_vec[precision] = vec;
    h->generation += 1;
    return DCM_OK;
}

// =============================================================================
// batched ensemble (no counterpart in the reference)
// =============================================================================
struct dcm_ensemble {
    int device = 0;
    std::vector<dcm_handle*> m;
    cudaStream_t st = nullptr;
    std::vector<cudaStream_t> mst;
    cudaEvent_t fork = nullptr, ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> join;
    cudaGraph_t graph[3] = {nullptr, nullptr, nullptr};
    cudaGraphExec_t exec[3] = {nullptr, nullptr, nullptr};
    std::vector<unsigned> gen[3];  // member generations each graph was built for
    std::string err;
};

namespace {

void ens_release(dcm_ensemble* e, int p) {
    if (e->exec[p]) cudaGraphExecDestroy(e->exec[p]);
    if (e->graph[p]) cudaGraphDestroy(e->graph[p]);
    e->exec[p] = nullptr;
    e->graph[p] = nullptr;
    e->gen[p].clear();
}

int ens_fail(dcm_ensemble* e, int code, const std::string& what) {
    e->err = what;
    return code;
}

// one CUDA graph for a time step of every member at velocity phase p: a
// fork into one capture stream per member, each member's whole step (its
// pressure solve as its own WHILE loop: converged members stop iterating
// while the others continue), the solver scalars copied to pinned host
// memory, and a join
int ens_build(dcm_ensemble* e, int p) {
    ens_release(e, p);
    if (cudaStreamBeginCapture(e->st, cudaStreamCaptureModeRelaxed) != cudaSuccess)
        return ens_fail(e, DCM_E_CUDA, "ensemble: begin capture");
    int rc = DCM_OK;
    cudaEventRecord(e->fork, e->st);
    Profiler* saved = g_prof;
    g_prof = nullptr;
    for (size_t q = 0; q < e->m.size() && rc == DCM_OK; q++) {
        dcm_handle* h = e->m[q];
        cudaStream_t s = e->mst[q];
        cudaStreamWaitEvent(s, e->fork, 0);
        rc = h->prec == 0 ? step_body<double>(h, s, p, true) : step_body<float>(h, s, p, true);
        if (rc != DCM_OK) {
            e->err = "member " + std::to_string(q) + ": " + h->err;
            break;
        }
        cudaMemcpyAsync(h->hS, h->S, sizeof(SolverScalars), cudaMemcpyDeviceToHost, s);
        if (h->prec) cudaMemcpyAsync(h->hS2, h->S2, sizeof(SolverScalars), cudaMemcpyDeviceToHost, s);
        cudaEventRecord(e->join[q], s);
        cudaStreamWaitEvent(e->st, e->join[q], 0);
    }
    g_prof = saved;
    cudaGraph_t g = nullptr;
    const cudaError_t ce = cudaStreamEndCapture(e->st, &g);
    e->graph[p] = g;
    if (rc != DCM_OK || ce != cudaSuccess || !g ||
        cudaGraphInstantiate(&e->exec[p], g, 0) != cudaSuccess) {
        ens_release(e, p);
        cudaGetLastError();
        return rc != DCM_OK ? rc : ens_fail(e, DCM_E_CUDA, "ensemble: capture / instantiate");
    }
    for (dcm_handle* h : e->m) e->gen[p].push_back(h->generation);
    return DCM_OK;
}

}  // namespace

extern "C" int dcm_ensemble_create(int nmembers, const dcm_grid* grids, int device,
                                   dcm_ensemble** out) {
    if (!out || !grids || nmembers < 1) return DCM_E_ARG;
    *out = nullptr;
    dcm_ensemble* e = new dcm_ensemble();
    e->device = device;
    for (int q = 0; q < nmembers; q++) {
        dcm_handle* h = nullptr;
        const int rc = dcm_create(&grids[q], device, &h);
        if (rc != DCM_OK) {
            for (dcm_handle* x : e->m) dcm_destroy(x);
            delete e;
            return rc;
        }
        e->m.push_back(h);
    }
    bool good = cudaSetDevice(device) == cudaSuccess &&
                cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking) == cudaSuccess &&
                cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming) == cudaSuccess &&
                cudaEventCreate(&e->ev0) == cudaSuccess && cudaEventCreate(&e->ev1) == cudaSuccess;
    e->mst.assign(nmembers, nullptr);
    e->join.assign(nmembers, nullptr);
    for (int q = 0; q < nmembers && good; q++)
        good = cudaStreamCreateWithFlags(&e->mst[q], cudaStreamNonBlocking) == cudaSuccess &&
               cudaEventCreateWithFlags(&e->join[q], cudaEventDisableTiming) == cudaSuccess;
    *out = e;
    return good ? DCM_OK : DCM_E_CUDA;
}

extern "C" int dcm_ensemble_destroy(dcm_ensemble* e) {
    if (!e) return DCM_OK;
    cudaSetDevice(e->device);
    if (e->st) cudaStreamSynchronize(e->st);
    for (int p = 0; p < 3; p++) ens_release(e, p);
    for (cudaStream_t s : e->mst)
        if (s) cudaStreamDestroy(s);
    for (cudaEvent_t v : e->join)
        if (v) cudaEventDestroy(v);
    if (e->fork) cudaEventDestroy(e->fork);
    if (e->ev0) cudaEventDestroy(e->ev0);
    if (e->ev1) cudaEventDestroy(e->ev1);
    if (e->st) cudaStreamDestroy(e->st);
    for (dcm_handle* h : e->m) dcm_destroy(h);
    delete e;
    return DCM_OK;
}

extern "C" int dcm_ensemble_member(dcm_ensemble* e, int member, dcm_handle** h) {
    if (!e || !h || member < 0 || member >= (int)e->m.size()) return DCM_E_ARG;
    *h = e->m[member];
    return DCM_OK;
}

extern "C" const char* dcm_ensemble_last_error(const dcm_ensemble* e) {
    return e ? e->err.c_str() : "";
}

extern "C" int dcm_ensemble_step(dcm_ensemble* e, int nsteps, dcm_ensemble_stats* stats) {
    if (!e || nsteps < 0) return DCM_E_ARG;
    if (cudaSetDevice(e->device) != cudaSuccess) return ens_fail(e, DCM_E_CUDA, "set device");
    const int n0 = e->m[0]->nstep;
    for (dcm_handle* h : e->m) {
        if (!h->resident) return ens_fail(e, DCM_E_ARG, "ensemble: a member has no state");
        if (h->nstep != n0) return ens_fail(e, DCM_E_ARG, "ensemble: members at different steps");
    }
    long long iters = 0;
    int imax = 0, done = 0, rc = DCM_OK;
    float ms_total = 0.f;
    for (; done < nsteps; done++) {
        const int p = (n0 + done) % 3;
        bool fresh = e->exec[p] != nullptr && e->gen[p].size() == e->m.size();
        for (size_t q = 0; fresh && q < e->m.size(); q++) fresh = e->gen[p][q] == e->m[q]->generation;
        if (!fresh && (rc = ens_build(e, p)) != DCM_OK) break;
        cudaEventRecord(e->ev0, e->st);
        if (cudaGraphLaunch(e->exec[p], e->st) != cudaSuccess) {
            rc = ens_fail(e, DCM_E_CUDA, "ensemble: graph launch");
            break;
        }
        cudaEventRecord(e->ev1, e->st);
        if (cudaEventSynchronize(e->ev1) != cudaSuccess) {
            rc = ens_fail(e, DCM_E_CUDA, std::string("ensemble: ") +
                                             cudaGetErrorString(cudaGetLastError()));
            break;
        }
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e->ev0, e->ev1);
        ms_total += ms;
        imax = 0;
        for (size_t q = 0; q < e->m.size(); q++) {
            dcm_handle* h = e->m[q];
            const SolverScalars* S = h->prec ? h->hS2 : h->hS;
            const int st = h->hS->status;  // the mixed solve copies its outcome there
            h->last_iters = S->it;
            h->last_err = S->err;
            if (h->prec) {
                h->last_refine.outer = S->updates;
                h->last_refine.inner = S->it;
                h->last_refine.restarts = S->restarts;
                h->last_refine.err = S->err;
            }
            h->nstep += 1;
            iters += S->it;
            imax = std::max(imax, S->it);
            if (st != DCM_OK && rc == DCM_OK)
                rc = ens_fail(e, st, "member " + std::to_string(q) + ": " + dcm_status_string(st));
        }
        if (rc != DCM_OK) {
            done++;
            break;
        }
    }
    if (stats) {
        stats->steps = done;
        stats->iters_total = iters;
        stats->iters_max_last = imax;
        stats->ms_total = ms_total;
    }
    return rc;
}

// =============================================================================
// read-only view of the resident state for the output writer (dcm_output.cu)
// =============================================================================
namespace dcm {

int resident_view(dcm_handle* h, ResidentView* out) {
    if (!h || !out || !h->resident) return DCM_E_ARG;
    int cu, cz, ct;
    roles_of(h->nstep % 3, cu, cz, ct);
    ResidentView& v = *out;
    v.d = h->d;
    v.prec = h->prec;
    v.p = h->p;
    v.div = h->div;
    v.st = h->st;
    v.device = h->device;
    v.q.clear();
    auto fill = [&](auto& S) {
        v.u = S.U[cu];
        v.v = S.V[cu];
        v.w = S.W[cu];
        v.th = S.th;
        for (auto* q : S.q) v.q.push_back(q);
    };
    if (h->prec == 0)
        fill(h->s64);
    else
        fill(h->s32);
    return DCM_OK;
}

int host_profiles(dcm_handle* h, std::vector<double>* rhoa, std::vector<double>* thetan) {
    if (!h || !rhoa || !thetan) return DCM_E_ARG;
    const size_t K2 = h->d.kp + 2;
    rhoa->assign(K2, 0.0);
    thetan->assign(K2, 0.0);
    if (cudaSetDevice(h->device) != cudaSuccess) return DCM_E_CUDA;
    if (cudaMemcpy(rhoa->data(), h->mt.rhoa, K2 * sizeof(double), cudaMemcpyDeviceToHost) !=
            cudaSuccess ||
        cudaMemcpy(thetan->data(), h->mt.thetan, K2 * sizeof(double), cudaMemcpyDeviceToHost) !=
            cudaSuccess)
        return DCM_E_CUDA;
    return DCM_OK;
}

}  // namespace dcm
