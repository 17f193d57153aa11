// dcm_prof.h -- optional per-kernel-class timing with CUDA events recorded on
// the launching stream around every launch.  Off unless a handle enables it;
// used by the benchmark to time the dominant kernel inside the timed region.
#pragma once
#include <cuda_runtime.h>

#include <vector>

namespace dcm {

enum ProfCat {
    P_SETUP = 0, P_JACOBI, P_MATVEC, P_UPDATE, P_POST, P_MEANS, P_SOURCES, P_RHS, P_ADVREF,
    P_MPMIN, P_UPWIND, P_ANTIDIFF, P_BETA, P_LIMIT, P_RESTORE, P_MOMENTUM, P_OTHER, P_NCAT
};

struct Profiler {
    bool on = false;
    bool capturing = false;  // launches are being captured into a graph
    std::vector<cudaEvent_t> pool;
    size_t used = 0;
    struct Rec { int cat; size_t e0, e1; };
    std::vector<Rec> recs;
    double ms[P_NCAT] = {0};
    long long launches[P_NCAT] = {0};  // timed launches
    long long count[P_NCAT] = {0};     // all launches

    cudaEvent_t get() {
        if (used == pool.size()) {
            cudaEvent_t e;
            cudaEventCreate(&e);
            pool.push_back(e);
        }
        return pool[used++];
    }
    // accumulate the recorded pairs (call after the stream is synchronised)
    void harvest() {
        for (const Rec& r : recs) {
            float t = 0.f;
            if (cudaEventElapsedTime(&t, pool[r.e0], pool[r.e1]) == cudaSuccess) {
                ms[r.cat] += t;
                launches[r.cat] += 1;
            }
        }
        recs.clear();
        used = 0;
    }
    // launches that ran inside a graph, counted from the device scalars
    void add(int cat, long long n) { count[cat] += n; }
    void reset() {
        for (int c = 0; c < P_NCAT; c++) { ms[c] = 0; launches[c] = 0; count[c] = 0; }
        recs.clear();
        used = 0;
    }
    ~Profiler() {
        for (cudaEvent_t e : pool) cudaEventDestroy(e);
    }
};

// the profiler of the handle this host thread is running (set by the C-ABI
// layer around dcm_step, null elsewhere); one per thread, so launches that
// other threads make are never counted or timed into it
extern thread_local Profiler* g_prof;

struct ProfScope {
    int cat;
    size_t e0 = 0;
    cudaStream_t st;
    bool timed;
    ProfScope(int c, cudaStream_t s)
        : cat(c), st(s), timed(g_prof && g_prof->on && !g_prof->capturing) {
        if (g_prof && !g_prof->capturing) g_prof->count[c] += 1;  // launches are always counted
        if (timed) {
            e0 = g_prof->used;
            cudaEventRecord(g_prof->get(), st);
        }
    }
    ~ProfScope() {
        if (timed) {
            const size_t e1 = g_prof->used;
            cudaEventRecord(g_prof->get(), st);
            g_prof->recs.push_back({cat, e0, e1});
        }
    }
};

}  // namespace dcm
