// dcm_noalloc.cu -- horizontal means through an entry point that allocates
// no device memory.
//
// Who needs it: a host that owns every byte of device memory through its own
// pool or budget (a framework allocator, a job-level memory cap) and does
// not let library code call cudaMalloc / cudaFree -- cudaFree also
// synchronises the whole device, which stalls the host's other streams.
// Such a caller already holds the fields on the device and passes device
// pointers and a stream; the per-level partial sums and the ticket of the
// deterministic reduction live in the fixed array below instead of buffers
// a handle would allocate.
#include <mutex>

#include "dcm_internal.h"

namespace {

// Scratch of the reduction: the first 256 bytes hold the ticket, the rest the
// 4 x (kp+2) x 128 block partials.  Sized for kp <= DCM_NOALLOC_MAX_KP
// (4 MiB); every GPU that loads the library keeps it until the process ends.
constexpr size_t kScratchDoubles = 32 + (size_t)4 * (DCM_NOALLOC_MAX_KP + 2) * dcm::MEAN_GY;
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_mu;
void* g_addr[128] = {nullptr};  // device address of the scratch, per device

// Device address of the scratch on the current device, resolved once per
// device with that device current (the array's name is only a host-side
// stand-in).
void* scratch_address(int dev, cudaError_t* err) {
    std::lock_guard<std::mutex> lk(g_mu);
    *err = cudaSuccess;
    if (dev < 0 || dev >= 128) {
        *err = cudaErrorInvalidDevice;
        return nullptr;
    }
    if (!g_addr[dev]) {
        void* p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (*err != cudaSuccess) return nullptr;
        g_addr[dev] = p;
    }
    return g_addr[dev];
}

}  // namespace

extern "C" int dcm_horizontal_means_noalloc(int ip, int jp, int kp, const double* u,
                                            const double* v, const double* w, const double* th,
                                            double* means, void* stream) {
    if (ip < 1 || jp < 1 || kp < 1 || kp > DCM_NOALLOC_MAX_KP) return DCM_E_ARG;
    if (!u || !v || !w || !th || !means) return DCM_E_ARG;
    const dcm::Dims d = dcm::make_dims(ip, jp, kp);
    if (d.n() >= (size_t)1 << 31) return DCM_E_ARG;
    // an error still pending from the caller's own work is left for the
    // caller's own check (not consumed here), and nothing is queued on top
    if (cudaPeekAtLastError() != cudaSuccess) return DCM_E_CUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return DCM_E_CUDA;
    cudaError_t e = cudaSuccess;
    char* base = (char*)scratch_address(dev, &e);
    if (!base) return DCM_E_CUDA;
    cudaStream_t st = (cudaStream_t)stream;
    unsigned int* ticket = (unsigned int*)base;
    double* partials = (double*)(base + 256);
    // the ticket must start at zero; a call that faulted earlier may have left
    // it set, so clear it on the caller's stream before the kernel
    if (cudaMemsetAsync(ticket, 0, sizeof(unsigned int), st) != cudaSuccess) return DCM_E_CUDA;
    dcm::Metrics<double> none{};  // the divergence is not formed here
    dcm::launch_means_div<double, double>(d, none, u, v, w, th, nullptr, 0, means, nullptr, partials,
                                  ticket, st);
    // no error was pending before the launches, so this reads (and clears)
    // only their own launch status
    return cudaGetLastError() == cudaSuccess ? DCM_OK : DCM_E_CUDA;
}
