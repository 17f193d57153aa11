// dcm_capi.cu -- the extern "C" boundary (include/dcm.h): handle lifetime,
// per-call drop-ins for the reference subroutines, and the device-resident
// time loop of model_driver (driver_code.f90:304-676).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dcm_internal.h"
#include "dcm_prof.h"

using namespace dcm;

namespace dcm {
Profiler* g_prof = nullptr;
}

namespace {

constexpr int NQMAX = 64;

template <typename T>
struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
};

}  // namespace

struct dcm_handle {
    int device = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    Dims d{};
    size_t n = 0;
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
    int first_call = 1;  // bicgstab_first, dynamics.f90:17

    // ---- resident state -------------------------------------------------------
    bool resident = false;
    dcm_config cfg{};
    std::vector<int> cs, ce;
    std::vector<double> forcing_host;  // 5*(kp+2)
    double* forcing_dev = nullptr;
    double *U[3]{}, *V[3]{}, *W[3]{};
    int nstep = 0;
    double *th = nullptr, *th2 = nullptr, *p = nullptr, *su = nullptr, *sv = nullptr,
           *sw = nullptr, *psrc = nullptr, *div = nullptr, *sth = nullptr;
    std::vector<double*> q, sq, qtmp;
    double* means = nullptr;
    double t1 = 0.0, t2 = 0.0;
    std::vector<double> q1, q2;
    std::vector<double*> owned;
    int last_iters = 0;
    double last_err = 0.0;
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

double* slot(dcm_handle* h, int idx) {
    if ((int)h->slots.size() <= idx) h->slots.resize(idx + 1, nullptr);
    if (!h->slots[idx]) {
        double* p = nullptr;
        if (cudaMalloc(&p, h->n * sizeof(double)) != cudaSuccess) return nullptr;
        cudaMemsetAsync(p, 0, h->n * sizeof(double), h->st);
        h->slots[idx] = p;
    }
    return h->slots[idx];
}

// slot numbering of the per-call drop-ins
enum {
    S_U = 0, S_V, S_W, S_ZU, S_ZV, S_ZW, S_SU, S_SV, S_SW, S_P, S_TH, S_STH, S_RHS, S_X, S_B,
    // solver work
    S_R, S_CR, S_PP, S_V1, S_T, S_SA, S_SB, S_RH, S_VH,
    // mpdata work
    S_VA0, S_VA1, S_VA2, S_VL0, S_VL1, S_VL2, S_B0, S_B1, S_B2, S_B3, S_B4, S_B5,
    S_PSI_OUT,
    S_DYN = 64  // psi fields / scratch for vec: S_DYN + 4*q + {in, out, pa, pb}
};

int upload(dcm_handle* h, double* dst, const double* src, size_t n = 0) {
    if (!src) return DCM_OK;
    const size_t cnt = n ? n : h->n;
    CK(cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyHostToDevice, h->st));
    return DCM_OK;
}
int download(dcm_handle* h, double* dst, const double* src, size_t n = 0) {
    if (!dst) return DCM_OK;
    const size_t cnt = n ? n : h->n;
    CK(cudaMemcpyAsync(dst, src, cnt * sizeof(double), cudaMemcpyDeviceToHost, h->st));
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
    const Dims d = make_dims(g->ip, g->jp, g->kp);
    if (d.n() >= (size_t)1 << 31) return DCM_E_UNSUPPORTED;  // int32 indexing
    dcm_handle* h = new dcm_handle();
    h->device = device;
    h->d = d;
    h->n = d.n();
    CK(cudaSetDevice(device));
    CK(cudaStreamCreateWithFlags(&h->st, cudaStreamNonBlocking));
    CK(cudaEventCreate(&h->ev0));
    CK(cudaEventCreate(&h->ev1));
    const size_t I2 = g->ip + 2, J2 = g->jp + 2, K2 = g->kp + 2;
    // metrics block: dx dxn (I2) dy dyn (J2) dz dzn rhoa rhoan theta thetan (K2)
    //                ae aw (I2) an as (J2) au ad (K2)
    const size_t nm = 2 * I2 + 2 * J2 + 6 * K2 + 2 * I2 + 2 * J2 + 2 * K2;
    std::vector<double> hm(nm, 0.0);
    size_t o = 0;
    auto put = [&](const double* src, size_t len) {
        const size_t at = o;
        std::memcpy(hm.data() + o, src, len * sizeof(double));
        o += len;
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
    *out = h;
    return DCM_OK;
}

static void free_state(dcm_handle* h) {
    for (double* p : h->owned) cudaFree(p);
    h->owned.clear();
    h->q.clear(); h->sq.clear(); h->qtmp.clear();
    h->resident = false;
}

extern "C" int dcm_destroy(dcm_handle* h) {
    if (!h) return DCM_OK;
    cudaSetDevice(h->device);
    if (h->st) cudaStreamSynchronize(h->st);
    free_state(h);
    for (double* p : h->slots)
        if (p) cudaFree(p);
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
                        b[d.at(k, j, i)] =
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
    launch_sources<double>(d, h->mt, F, BARS, BARS + K2, BARS + 2 * K2, BARS + 3 * K2, ZU, ZV, ZW,
                           U, V, W, TH, SU, SV, SWd, STH, RHS, 0, 0, h->st);
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
    for (int q = 0; q < nq; q++) RC(upload(h, pin[q], psi + (size_t)q * h->n));
    RC(mpdata_run<double>(mb.w, h->d, h->mt, dt, U, V, W, pin.data(), pout.data(), nq, lbc, ubc,
                          kord, monotone, neumann, limiter, vec, nullptr, 0.0, h->st));
    for (int q = 0; q < nq; q++) RC(download(h, psi + (size_t)q * h->n, pout[q]));
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
    for (int c = 0; c < nqq; c++) RC(upload(h, Q[c], q + (size_t)c * h->n));
    launch_means_div<double>(h->d, h->mt, U, V, W, TH, Q.data(), nqq, OUT, nullptr, h->partials,
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
    launch_means_div<double>(h->d, h->mt, U, V, W, W, nullptr, 0, OUT, DV, h->partials,
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
            RC(upload(h, A, q + (size_t)c * h->n)); RC(upload(h, S, sq + (size_t)c * h->n));
            launch_advance_scalar<double>(h->d, dt, A, S, h->st);
            RC(download(h, q + (size_t)c * h->n, A));
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

// =============================================================================
// device-resident time loop
// =============================================================================
namespace {

double* alloc_owned(dcm_handle* h) {
    double* p = nullptr;
    if (cudaMalloc(&p, h->n * sizeof(double)) != cudaSuccess) return nullptr;
    cudaMemsetAsync(p, 0, h->n * sizeof(double), h->st);
    h->owned.push_back(p);
    return p;
}

// velocity roles after n steps: (u, zu, tu) -> buffers (0,1,2), (2,0,1),
// (1,2,0) for n mod 3 = 0, 1, 2 (driver_code.f90:281-283, :634-646)
void roles(const dcm_handle* h, int& cu, int& cz, int& ct) {
    static const int RU[3] = {0, 2, 1}, RZ[3] = {1, 0, 2}, RT[3] = {2, 1, 0};
    const int m = h->nstep % 3;
    cu = RU[m];
    cz = RZ[m];
    ct = RT[m];
}

__global__ void k_driver_start(Dims d, double* zu, double* zv, double* zw) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const int i = blockIdx.y;
    if (j > d.jp + 1) return;
    zw[d.at(0, j, i)] = -zw[d.at(1, j, i)];  // driver_code.f90:288
    zu[d.at(1, j, i)] = 0.0;
    zv[d.at(1, j, i)] = 0.0;
    zw[d.at(d.kp, j, i)] = -zw[d.at(d.kp - 1, j, i)];  // :292-294
    zw[d.at(d.kp + 1, j, i)] = 0.0;
    zu[d.at(d.kp, j, i)] = 0.0;
    zv[d.at(d.kp, j, i)] = 0.0;
}

int one_step(dcm_handle* h) {
    const Dims& d = h->d;
    const dcm_config& c = h->cfg;
    const size_t K2 = d.kp + 2;
    int cu, cz, ct;
    roles(h, cu, cz, ct);
    double *u = h->U[cu], *v = h->V[cu], *w = h->W[cu];
    double *zu = h->U[cz], *zv = h->V[cz], *zw = h->W[cz];
    double *tu = h->U[ct], *tv = h->V[ct], *tw = h->W[ct];
    const int nqq = c.moisture ? c.nq : 0;
    // horizontal_means + divergence_calc, driver_code.f90:433-444
    launch_means_div<double>(d, h->mt, u, v, w, h->th, h->q.data(), nqq, h->means, h->div,
                             h->partials, h->ticket, h->st);
    // sources (sth = 0 first, :340) + exchange_along_dim_wo(psrc), :455-487
    int rc = DCM_OK;
    Forcing<double> F = forcing_of(h, nullptr, h->forcing_dev, &rc);
    F.damping_layer = c.forcing.damping_layer;
    F.forcing = c.forcing.forcing;
    F.divergence = c.forcing.divergence;
    F.forcing_tau = c.forcing.forcing_tau;
    F.dampfacn = h->forcing_dev; F.dampfac = h->forcing_dev + K2;
    F.u_force = h->forcing_dev + 2 * K2; F.v_force = h->forcing_dev + 3 * K2;
    F.w_subs = h->forcing_dev + 4 * K2;
    const double* ubar = h->means;
    launch_sources<double>(d, h->mt, F, ubar, ubar + K2, ubar + 2 * K2, ubar + 3 * K2, zu, zv, zw,
                           u, v, w, h->th, h->su, h->sv, h->sw, h->sth, h->psrc, 1, 1, h->st);
    CK(cudaGetLastError());
    // bicgstab + exchange_along_dim_wo(p), :496-507
    SolverWork<double> sw = solver_work(h);
    NEED(sw.r); NEED(sw.sB); NEED(sw.rh); NEED(sw.vh);
    h->first_call = 0;
    const int st = solver_run<double>(sw, d, h->p, h->psrc, h->sw, h->mt.dzn, c.ptol, c.itmax, 1,
                                      4, h->st, h->hS, nullptr);
    h->last_iters = h->hS->it;
    h->last_err = h->hS->err;
    if (st != DCM_OK) {
        h->err = dcm_status_string(st);
        return st;
    }
    // scalar advection, :514-560, with advance_scalar_fields_3d (:601) fused
    MpBufs mb;
    if (!mpdata_work(h, std::max(1, nqq), mb)) return fail(h, DCM_E_CUDA, "device allocation");
    if (c.advection_scheme == 0 || c.advection_scheme == 1) {
        launch_adv_ref_state<double>(d, h->mt, c.dt, w, h->th, h->th2, h->mt.thetan, 1, h->st);
    }
    if (c.advection_scheme == 1) {
        double lb = h->t1, ub = h->t2;
        double* pin = h->th2;
        double* pout = h->th;
        const double* sadd = h->sth;
        RC(mpdata_run<double>(mb.w, d, h->mt, c.dt, u, v, w, &pin, &pout, 1, &lb, &ub, c.kord,
                              c.monotone, 0, c.limiter, false, &sadd, c.dt, h->st));
        // t1, t2 return unshifted: (t - m) + m; kept on the host.  (0 - m) + m == 0
        // exactly, so the values only change when they start non-zero.
        if (h->t1 != 0.0 || h->t2 != 0.0) {
            CK(cudaMemcpyAsync(h->hM, h->M, sizeof(MpScalars), cudaMemcpyDeviceToHost, h->st));
            RC(sync(h));
            h->t1 = h->hM[0].lbc + h->hM[0].m;
            h->t2 = h->hM[0].ubc + h->hM[0].m;
        }
    } else if (c.advection_scheme == 0) {
        // donor cell + exchange_full(th, t1, t2), :539-545, then th += sth*dt
        CK(cudaMemcpyAsync(h->th, h->th2, h->n * sizeof(double), cudaMemcpyDeviceToDevice,
                           h->st));
        RC(upwind_run<double>(mb.w, d, h->mt, c.dt, u, v, w, h->th2, h->th, 0, h->st));
        launch_exchange<double>(d, h->th, HALO_FULL, h->t1, h->t2, h->st);
        launch_advance_scalar<double>(d, c.dt, h->th, h->sth, h->st);
    } else if (c.advection_scheme == 2) {
        // mpdata_3d_add with thetan, thbase, thtop, :552-556
        double lb = c.thbase, ub = c.thtop;
        launch_add_profile<double>(d, h->th, h->mt.thetan, 1.0, h->st);
        double* pin = h->th;
        double* pout = h->th2;
        RC(mpdata_run<double>(mb.w, d, h->mt, c.dt, u, v, w, &pin, &pout, 1, &lb, &ub, c.kord,
                              c.monotone, 0, c.limiter, false, nullptr, 0.0, h->st));
        launch_add_profile<double>(d, h->th2, h->mt.thetan, -1.0, h->st);
        launch_advance_scalar<double>(d, c.dt, h->th2, h->sth, h->st);
        std::swap(h->th, h->th2);
    } else {
        return fail(h, DCM_E_UNSUPPORTED, "advection_scheme");
    }
    // q categories, :568-585, then q += sq*dt
    if (nqq) {
        for (int cat = 0; cat < c.ncat; cat++) {
            const int a = h->cs[cat] - 1, b = h->ce[cat] - 1;
            const int nc = b - a + 1;
            std::vector<double*> qin(nc), qout(nc);
            std::vector<const double*> sadd(nc);
            for (int e = 0; e < nc; e++) {
                CK(cudaMemcpyAsync(h->qtmp[a + e], h->q[a + e], h->n * sizeof(double),
                                   cudaMemcpyDeviceToDevice, h->st));
                qin[e] = h->qtmp[a + e];
                qout[e] = h->q[a + e];
                sadd[e] = h->sq[a + e];
            }
            RC(mpdata_run<double>(mb.w, d, h->mt, c.dt, u, v, w, qin.data(), qout.data(), nc,
                                  h->q1.data() + a, h->q2.data() + a, c.kord, c.monotone, 0,
                                  c.limiter, true, sadd.data(), c.dt, h->st));
        }
    }
    // advance_momentum(2dt) + time filter + rotation + exchange + rows, :592-674
    launch_momentum_step<double>(d, h->mt, 2.0 * c.dt, u, v, w, zu, zv, zw, tu, tv, tw, h->su,
                                 h->sv, h->sw, h->p, h->st);
    CK(cudaGetLastError());
    h->nstep += 1;
    return DCM_OK;
}

}  // namespace

extern "C" int dcm_state_upload(dcm_handle* h, const dcm_config* cfg, const dcm_fields* f) {
    CHECK_H();
    if (!cfg || !f) return fail(h, DCM_E_ARG, "state_upload: bad argument");
    if (cfg->precision != 0) return fail(h, DCM_E_UNSUPPORTED, "precision");
    if (cfg->advection_scheme < 0 || cfg->advection_scheme > 2 || cfg->itmax < 1 || cfg->dt <= 0)
        return fail(h, DCM_E_ARG, "state_upload: bad config");
    if (cfg->moisture && (cfg->nq < 1 || cfg->nq > NQMAX || cfg->ncat < 1 || !cfg->c_s ||
                          !cfg->c_e || !f->q || !f->sq))
        return fail(h, DCM_E_ARG, "state_upload: bad moisture config");
    free_state(h);
    h->cfg = *cfg;
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
    double* in3[9] = {f->u, f->zu, f->tu, f->v, f->zv, f->tv, f->w, f->zw, f->tw};
    double** dst3[9] = {&h->U[0], &h->U[1], &h->U[2], &h->V[0], &h->V[1],
                        &h->V[2], &h->W[0], &h->W[1], &h->W[2]};
    for (int c = 0; c < 9; c++) {
        *dst3[c] = alloc_owned(h);
        NEED(*dst3[c]);
        if (!in3[c]) return fail(h, DCM_E_ARG, "state_upload: missing velocity");
        RC(upload(h, *dst3[c], in3[c]));
    }
    h->nstep = 0;
    double** fl[9] = {&h->th, &h->th2, &h->p, &h->su, &h->sv, &h->sw, &h->psrc, &h->div, &h->sth};
    for (auto pp : fl) {
        *pp = alloc_owned(h);
        NEED(*pp);
    }
    if (!f->th || !f->p) return fail(h, DCM_E_ARG, "state_upload: missing th or p");
    RC(upload(h, h->th, f->th)); RC(upload(h, h->p, f->p));
    RC(upload(h, h->su, f->su)); RC(upload(h, h->sv, f->sv)); RC(upload(h, h->sw, f->sw));
    RC(upload(h, h->psrc, f->psrc)); RC(upload(h, h->div, f->div)); RC(upload(h, h->sth, f->sth));
    const size_t K2 = h->d.kp + 2;
    CK(cudaMalloc(&h->means, (4 + nqq) * K2 * sizeof(double)));
    h->owned.push_back(h->means);
    CK(cudaMemsetAsync(h->means, 0, (4 + nqq) * K2 * sizeof(double), h->st));
    for (int c = 0; c < nqq; c++) {
        double* a = alloc_owned(h);
        double* s = alloc_owned(h);
        double* t = alloc_owned(h);
        NEED(a); NEED(s); NEED(t);
        RC(upload(h, a, f->q + (size_t)c * h->n));
        RC(upload(h, s, f->sq + (size_t)c * h->n));
        h->q.push_back(a);
        h->sq.push_back(s);
        h->qtmp.push_back(t);
    }
    h->q1.assign(nqq, 0.0);  // driver_code.f90:275-276
    h->q2.assign(nqq, 0.0);
    h->t1 = h->t2 = 0.0;  // saved locals, :260
    // forcing profiles
    int rc = DCM_OK;
    forcing_of(h, &cfg->forcing, h->forcing_dev, &rc);
    if (rc != DCM_OK) return fail(h, rc, "state_upload: forcing arrays");
    h->resident = true;
    return sync(h);
}

extern "C" int dcm_driver_start(dcm_handle* h) {
    CHECK_H();
    if (!h->resident) return fail(h, DCM_E_ARG, "driver_start: no state");
    int cu, cz, ct;
    roles(h, cu, cz, ct);
    const dim3 g((h->d.J + 127) / 128, h->d.I);
    k_driver_start<<<g, 128, 0, h->st>>>(h->d, h->U[cz], h->V[cz], h->W[cz]);
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
        rc = one_step(h);
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
    }
    return rc;
}

extern "C" int dcm_state_download(dcm_handle* h, dcm_fields* f) {
    CHECK_H();
    if (!h->resident || !f) return fail(h, DCM_E_ARG, "state_download: no state");
    int cu, cz, ct;
    roles(h, cu, cz, ct);
    RC(download(h, f->u, h->U[cu])); RC(download(h, f->v, h->V[cu]));
    RC(download(h, f->w, h->W[cu]));
    RC(download(h, f->zu, h->U[cz])); RC(download(h, f->zv, h->V[cz]));
    RC(download(h, f->zw, h->W[cz]));
    RC(download(h, f->tu, h->U[ct])); RC(download(h, f->tv, h->V[ct]));
    RC(download(h, f->tw, h->W[ct]));
    RC(download(h, f->th, h->th)); RC(download(h, f->p, h->p));
    RC(download(h, f->su, h->su)); RC(download(h, f->sv, h->sv)); RC(download(h, f->sw, h->sw));
    RC(download(h, f->psrc, h->psrc)); RC(download(h, f->div, h->div));
    RC(download(h, f->sth, h->sth));
    const size_t K2 = h->d.kp + 2;
    RC(download(h, f->ubar, h->means, K2)); RC(download(h, f->vbar, h->means + K2, K2));
    RC(download(h, f->wbar, h->means + 2 * K2, K2));
    RC(download(h, f->thbar, h->means + 3 * K2, K2));
    const int nqq = h->cfg.moisture ? h->cfg.nq : 0;
    if (nqq && f->qbar) RC(download(h, f->qbar, h->means + 4 * K2, nqq * K2));
    for (int c = 0; c < nqq; c++) {
        if (f->q) RC(download(h, f->q + (size_t)c * h->n, h->q[c]));
        if (f->sq) RC(download(h, f->sq + (size_t)c * h->n, h->sq[c]));
    }
    return sync(h);
}

// =============================================================================
// diagnostics
// =============================================================================
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
