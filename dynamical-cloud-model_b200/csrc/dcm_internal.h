// dcm_internal.h -- device work areas and host-side entry points shared by
// the kernel files and the C-ABI layer.
#pragma once
#include <vector>
#include <cuda_runtime.h>

#include <utility>

#include "../../include/dcm.h"
#include "dcm_common.cuh"

namespace dcm {

// scalars of one pressure solve, resident in device memory
struct SolverScalars {
    double sc_err, err, rho, alf, omg, bet, nrm, tt, ts;
    int it, done, status, early;
    // reliable updates of the mixed-precision solve: pause the FP32
    // iteration when its residual has fallen by `delta` since the last FP64
    // residual (ru_norm) or below the tolerance
    double ru_norm, delta;
    int ru, pause, updates;
    // breakdown of the FP32 recursion in the mixed form: 1 = restart from the
    // FP64 residual keeping the FP32 correction, 2 = its vectors went
    // non-finite, drop the correction since the last update
    int restart;
    int rounds;    // iterations of a graph-driven solve (bounded, see k_loop_cond)
    int cycles;    // mixed form, graph-driven: FP64 update cycles (outer loop rounds)
    int ru_runs;   // mixed form, graph-driven: reliable-update branches taken
    int fresh;     // the next iteration starts a recursion (p = v1 = 0)
    int restarts;  // restarts of this solve
    int cycle_it;  // FP32 iterations since the last FP64 update
    double crnorm;  // (cr, cr) of the shadow residual
};

// One pressure solve captured as a CUDA graph: the iteration loop is a
// conditional WHILE node whose condition a device kernel sets, so the host
// neither polls nor launches per iteration.  Rebuilt when any captured
// argument changes (key).
struct SolveGraph {
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t side[2] = {nullptr, nullptr};  // capture streams of the loop bodies
    // key: everything the captured launches depend on
    const void* key_ptr[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
    double key_d[3] = {0, 0, 0};
    int key_i[6] = {0, 0, 0, 0, 0, 0};
    bool matches(const void* const* p, const double* dv, const int* iv) const {
        for (int q = 0; q < 6; q++)
            if (key_ptr[q] != p[q] || key_i[q] != iv[q]) return false;
        for (int q = 0; q < 3; q++)
            if (key_d[q] != dv[q]) return false;
        return exec != nullptr;
    }
    void release() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
    }
    ~SolveGraph() {
        release();
        for (cudaStream_t& s : side)
            if (s) cudaStreamDestroy(s);
    }
};

template <typename T>
struct SolverWork {
    T *r, *cr, *p, *v1, *t, *sA, *sB;   // full-size vectors (halo layout)
    T *rh, *vh;                          // r / a_p and v1 / a_p
    const T *ae, *aw, *an, *as, *au, *ad;  // per-axis stencil coefficients
    double* partials;
    unsigned int* ticket;
    Red2 red;
    SolverScalars* S;
    SolveGraph* graph = nullptr;  // null: host-driven loop
    // emit the solve into the graph being captured on the caller's stream
    // (a whole time step captured with other work) instead of running it
    bool emit = false;
    // launch shape (tuning): warps per block of the non-reducing sweeps, and
    // warp tasks per warp of the persistent reducing kernels (0 = as many
    // resident blocks as the occupancy allows)
    int by = 8;
    int tasks = 0;
    // most blocks a reducing kernel may use: the partials buffer holds
    // 3 values per block (the largest NV of any reducing kernel)
    int max_blocks = 0;
    // i-planes each stencil warp task marches over (tuning)
    int ni = 4;
    // FP32: fuse the three Jacobi sweeps of a phase (columns of <= 128 levels)
    int fuse = 1;
    // FP32: levels per lane of the separate stencil and update kernels (4:
    // 16-byte vectors; 2: 8-byte vectors, for short columns that would leave
    // lanes of a 128-level warp task idle); 0 = 4
    int vw = 0;
    // FP32 iterations of the mixed form: Chebyshev-weighted Jacobi sweeps on
    // the interval [cheb_lo, 2] of the spectrum of D^-1 A (0: the reference's
    // unweighted sweeps)
    int cheb = 0;
    double cheb_lo = 0.05;
    // graph-driven iterations launch their kernels with programmatic
    // dependent launch (where the runtime takes it; solver_pdl_available)
    int pdl = 1;
    // failure-path limits: rounds a graph-driven solve may run before it
    // stops with DCM_E_TIMEOUT (0: itmax + 1, or itmax + max_updates + 1 in
    // the mixed form), and the breakdown threshold of omega in an FP64 solve
    // (< 0: the reference's tiny)
    int round_budget = 0;
    double tiny = -1.0;
    // FP64: domains of at most this many interior points solve in one
    // thread-block cluster (k_bicgstab_small); 0 = never
    long long small_max = 0;
};

// one-time setup of the solver kernels (shared-memory limits, the probe of
// programmatic launches in graphs); called at handle creation, outside any
// stream capture
void solver_init();
// whether graph-driven iterations can use programmatic dependent launch
bool solver_pdl_available();

// per-field scalars of one MPDATA call
struct MpScalars {
    double m, lbc, ubc;  // shift and shifted boundary values
    int early;
    int pad;
};

template <typename T>
struct MpdataWork {
    T** pa;            // [nq] scratch copies (ping)
    T** pb;            // [nq] scratch copies (pong)
    T* va[3];          // antidiffusive velocities
    T* vl[3];          // limited velocities
    T* beta[6];        // beta_up / beta_down (6 for the sfvt limiter)
    double* partials;
    unsigned int* ticket;
    MpScalars* M;      // [nq]
    MpScalars* Mone;   // early = 1 (used when kord < 1)
    MpScalars* Mzero;  // all zero
    // antidiffusive iterations fused into one kernel each (k_mpdata_iter);
    // fuse_rows caps its rows per block (32 = no cap)
    int fuse = 0;
    int fuse_rows = 32;
};

// one-time setup of the MPDATA kernels (shared-memory limits of the fused
// iteration); called at handle creation, outside any stream capture
void mpdata_init();

// Jacobi-preconditioned BiCGSTAB (dynamics.f90:293-444) on x, b in the
// pitched layout.  With w.graph set (and event profiling off) the whole solve
// runs as one CUDA graph; otherwise the host launches iterations in chunks
// and polls the device scalars between chunks.
template <typename T>
int solver_run(SolverWork<T>& w, const Dims& d, T* x, const T* b, const T* sw,
               const T* dzn, double tol, int itmax, int wo, int chunk,
               cudaStream_t st, SolverScalars* host_S, int* launched_iters,
               double sc_floor = 0.01, bool post = true);

struct RefineStats {
    int outer, inner, restarts;
    double err;
};

// mixed-precision pressure solve: FP32 BiCGSTAB with FP64 reliable updates
// of the residual; x is the FP64 pressure, dx FP32 scratch
int refine_run(SolverWork<float>& wf, SolverWork<double>& wd, const Dims& d,
               double* x, const double* b, const float* sw, const double* dzn,
               float* dx, double tol, double delta, int itmax, int max_updates,
               cudaStream_t st, SolverScalars* hS_out, SolverScalars* hS_in,
               RefineStats* rs);

template <typename T>
int mpdata_run(MpdataWork<T>& w, const Dims& d, const Metrics<T>& mt, T dt,
               const T* u, const T* v, const T* wv, T* const* psi_in,
               T* const* psi_out, int nq, const double* lbc, const double* ubc,
               int kord, int monotone, int neumann, int variant, bool vec,
               const T* const* sadd, T dt_add, cudaStream_t st);

template <typename T>
int upwind_run(MpdataWork<T>& w, const Dims& d, const Metrics<T>& mt, T dt,
               const T* u, const T* v, const T* wv, const T* psi_in,
               T* psi_out, int neumann, cudaStream_t st);

// --- dcm_capi.cu: a read-only view of the resident state (output writer) ----
struct ResidentView {
    Dims d;              // pitched device layout
    int prec = 0;        // 0: FP64 fields; 1: FP32 fields (p and div are FP64 in both)
    const void *u = nullptr, *v = nullptr, *w = nullptr, *th = nullptr;  // current roles
    const double *p = nullptr, *div = nullptr;
    std::vector<const void*> q;  // nq fields when moisture is on
    cudaStream_t st = nullptr;   // the handle's stream (orders the view after the step)
    int device = 0;
};
// DCM_E_ARG when no state is resident
int resident_view(dcm_handle* h, ResidentView* out);
// host copies of the handle's rhoa and thetan (kp+2 each)
int host_profiles(dcm_handle* h, std::vector<double>* rhoa, std::vector<double>* thetan);

// --- k_dynamics.cu ---------------------------------------------------------
enum HaloMode { HALO_FULL = 0, HALO_DIM = 1, HALO_WO = 2, HALO_FULL_WO = 3 };

template <typename T>
void launch_exchange(const Dims& d, T* a, int mode, T lbc, T ubc,
                     cudaStream_t st);

template <typename T>
struct Forcing {
    int damping_layer, forcing, divergence;
    const T *dampfacn, *dampfac, *u_force, *v_force, *w_subs;
    T forcing_tau;
};

// blocks per level of the means reduction (its partials are 4 x (kp+2) x MEAN_GY)
constexpr int MEAN_GY = 128;

// means of u,v,w,th (+ nq q fields) per level k = 0..kp+1 and, when div is
// non-null, the divergence of rho*u (diagnostics.f90:31-153)
template <typename T, typename D>
void launch_means_div(const Dims& d, const Metrics<D>& mt, const T* u,
                      const T* v, const T* w, const T* th, T* const* q, int nq,
                      T* means /* (4+nq)*(kp+2) */, D* div, double* partials,
                      unsigned int* ticket, cudaStream_t st);

// --- k_subgrid.cu ----------------------------------------------------------
// Smagorinsky subgrid model, sgm/subgrid_3d.f90:38-493.
template <typename T>
struct SgsParams {
    const T* lamsq;             // mixing length squared on the w-levels, kp+2
    double z1, z0, z0th;        // z(1) and the roughness lengths of monin_obukhov
};
// scalars diffused in one pass: ds[m] += div(vist grad s[m]) / rhoan, or
// ds[m] = that term alone where bit m of reset is set
constexpr int SGS_MAXS = 9;
constexpr int SGS_MAX_SETS = 8;  // th and up to 71 q fields in one step
template <typename T>
struct ScalarSet {
    const T* s[SGS_MAXS];
    T* ds[SGS_MAXS];
    int n;
    unsigned reset;
};
// tau: six fields (tau11, tau22, tau33, tau12, tau13, tau23); rows = true applies the surface / lid rows of sources to su, sv, sw
// instead of their exchange_full images alone
template <typename T>
void launch_subgrid(const Dims& d, const Metrics<T>& mt, const SgsParams<T>& P, const T* u,
                    const T* v, const T* w, const T* zu, const T* zv, const T* zw, const T* th,
                    T* vism, T* vist, T* strain, T* const* tau, T* su, T* sv, T* sw,
                    const ScalarSet<T>* sets, int nsets, bool rows, cudaStream_t st);
// the scalar diffusion pass alone (vist already computed)
template <typename T>
void launch_subgrid_scalars(const Dims& d, const Metrics<T>& mt, const T* vist,
                            const ScalarSet<T>* sets, int nsets, cudaStream_t st);
// groups th (if non-null) and the nq q fields into sets; returns the number
// of sets, or -1 when more than max_sets are needed
template <typename T>
int make_scalar_sets(const T* th, T* sth, int sth_reset, T* const* q, T* const* sq, int nq,
                     int sq_reset, ScalarSet<T>* sets, int max_sets);
// the subgrid model inside the resident time step (sources with
// viscous = .true.)
template <typename T>
struct SgsStep {
    SgsParams<T> P;
    T *vism, *vist, *strain;
    T* const* tau; // six stress fields (scratch)
    T* const* q;   // nq current q fields
    T* const* sq;  // their sources
    int nq;
};

// sources (dynamics.f90:639-998); sth_reset applies the driver's sth = 0
// first; rhs_wo applies the driver's exchange_along_dim_wo(psrc); sg
// non-null is the viscous = .true. branch (the subgrid model)
template <typename T, typename R>
void launch_sources(const Dims& d, const Metrics<T>& mt, const Metrics<R>& mtr,
                    const Forcing<T>& f, const T* ubar, const T* vbar,
                    const T* wbar, const T* thbar, const T* zu, const T* zv,
                    const T* zw, const T* u, const T* v, const T* w,
                    const T* th, T* su, T* sv, T* sw, T* sth, R* rhs,
                    int sth_reset, int rhs_wo, cudaStream_t st,
                    const SgsStep<T>* sg = nullptr);

template <typename T>
void launch_advance_momentum(const Dims& d, const Metrics<T>& mt, T dt, T* u,
                             T* v, T* w, const T* zu, const T* zv, const T* zw,
                             const T* su, const T* sv, const T* sw, const T* p,
                             cudaStream_t st);

// resident step: advance_momentum(2dt) into tu, time filter of u in place,
// then the exchange + boundary rows of the rotated velocities
// (driver_code.f90:592-674)
template <typename T, typename P>
void launch_momentum_step(const Dims& d, const Metrics<T>& mt,
                          const Metrics<P>& mtp, T dt2, T* u, T* v, T* w,
                          const T* zu, const T* zv, const T* zw, T* tu, T* tv,
                          T* tw, const T* su, const T* sv, const T* sw,
                          const P* p, cudaStream_t st);

// adv_ref_state (+ optional exchange_full(0,0)) from psi into out
template <typename T>
void launch_adv_ref_state(const Dims& d, const Metrics<T>& mt, T dt,
                          const T* w, const T* psi, T* out, const T* psi_ref,
                          int exch, cudaStream_t st);

template <typename T>
void launch_advance_scalar(const Dims& d, T dt, T* a, const T* s,
                           cudaStream_t st);

// element-wise precision conversion of n values
template <typename TO, typename FROM>
void launch_convert(size_t n, TO* to, const FROM* from, cudaStream_t st);
// dense host-layout field (hd) -> pitched device field (d), converted to TO
template <typename TO>
void launch_repitch(const Dims& hd, const Dims& d, TO* dst, const double* src, cudaStream_t st);

// psi (+/-) psi_1d(k) over the whole array (mpdata_3d_add :175-188)
template <typename T>
void launch_add_profile(const Dims& d, T* a, const T* prof, T sign,
                        cudaStream_t st);

}  // namespace dcm
