// dcm_output.cu -- the reference's output routine (driver_code.f90:725-1145)
// for the device-resident state: a netCDF classic file with the reference's
// dimensions, variables, units and FP32 on-disk values, written without
// stalling the time loop.
//
// Per record (one dcm_output_write):
//   1. a packing kernel on the handle's stream turns the resident fields of
//      the current roles into the record's bytes: FP32, big-endian (XDR), in
//      the variables' on-disk order (th, u, v, w, p, div with k fastest; q
//      and precip with the q index fastest, as the reference's reshape
//      writes them), into one of two device staging buffers;
//   2. a copy stream waits for the packing kernel and moves the record to a
//      pinned host buffer, while the handle's stream goes on with the next
//      steps;
//   3. a writer thread waits for that copy, writes the record at its offset
//      and then the new record count in the header.
// A third write waits only for the first of the two buffers to come free.
//
// File layout (the netCDF classic format, CDF-1; CDF-2 when an offset needs
// 64 bits): dims times (unlimited), ip, jp, kp [, nq, nprec, l_q_names = 20];
// variables in the reference's order of definition (:816-957): time(times),
// x(ip), y(jp), z(kp), rhoa(kp), thetan(kp), trefn(kp), th, u, v, w, p, div
// (times, ip, jp, kp) [, q_names(nq, l_q_names), q and precip
// (times, ip, jp, kp, nq / nprec)], each with its "units" attribute; fixed
// variables first, then the records.  precip comes from the microphysics,
// which is not on this path: its values are zero.
#include <condition_variable>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <deque>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "dcm_internal.h"

using namespace dcm;

namespace {

constexpr int LQ = 20;  // character(len=20) :: q_name

// ---- the netCDF classic header ----------------------------------------------
struct Xdr {
    std::vector<uint8_t> b;
    void u32(uint32_t v) {
        for (int s = 24; s >= 0; s -= 8) b.push_back((uint8_t)(v >> s));
    }
    void u64(uint64_t v) {
        for (int s = 56; s >= 0; s -= 8) b.push_back((uint8_t)(v >> s));
    }
    void pad() {
        while (b.size() % 4) b.push_back(0);
    }
    void name(const std::string& s) {
        u32((uint32_t)s.size());
        b.insert(b.end(), s.begin(), s.end());
        pad();
    }
};

enum { NC_CHAR = 2, NC_FLOAT = 5, NC_DIMENSION = 10, NC_VARIABLE = 11, NC_ATTRIBUTE = 12 };

struct Var {
    std::string name, units;
    std::vector<int> dims;  // dimension ids, slowest first (times first for records)
    int type;
    bool record;
    uint64_t vsize = 0;     // bytes (per record for record variables), multiple of 4
    uint64_t begin = 0;
};

struct Layout {
    std::vector<std::pair<std::string, uint64_t>> dims;  // length 0: the record dimension
    std::vector<Var> vars;
    int version = 1;
    uint64_t header = 0, rec_begin = 0, recsize = 0;
};

std::vector<uint8_t> encode(const Layout& L, uint32_t numrecs) {
    Xdr x;
    const uint8_t magic[4] = {'C', 'D', 'F', (uint8_t)L.version};
    x.b.insert(x.b.end(), magic, magic + 4);
    x.u32(numrecs);
    x.u32(NC_DIMENSION);
    x.u32((uint32_t)L.dims.size());
    for (auto& d : L.dims) {
        x.name(d.first);
        x.u32((uint32_t)d.second);
    }
    x.u32(0);  // no global attributes (ABSENT)
    x.u32(0);
    x.u32(NC_VARIABLE);
    x.u32((uint32_t)L.vars.size());
    for (const Var& v : L.vars) {
        x.name(v.name);
        x.u32((uint32_t)v.dims.size());
        for (int d : v.dims) x.u32((uint32_t)d);
        if (v.units.empty()) {
            x.u32(0);
            x.u32(0);
        } else {
            x.u32(NC_ATTRIBUTE);
            x.u32(1);
            x.name("units");
            x.u32(NC_CHAR);
            x.u32((uint32_t)v.units.size());
            x.b.insert(x.b.end(), v.units.begin(), v.units.end());
            x.pad();
        }
        x.u32((uint32_t)v.type);
        x.u32((uint32_t)v.vsize);
        if (L.version == 1)
            x.u32((uint32_t)v.begin);
        else
            x.u64(v.begin);
    }
    return x.b;
}

// begins of every variable: the header, the fixed variables in order, then
// the record variables of record 0 in order
bool place(Layout& L) {
    for (int version = 1; version <= 2; version++) {
        L.version = version;
        L.header = encode(L, 0).size();  // the begins' widths fix the size
        uint64_t off = L.header;
        for (Var& v : L.vars)
            if (!v.record) {
                v.begin = off;
                off += v.vsize;
            }
        L.rec_begin = off;
        L.recsize = 0;
        for (Var& v : L.vars)
            if (v.record) {
                v.begin = off;
                off += v.vsize;
                L.recsize += v.vsize;
            }
        uint64_t last = 0;
        for (const Var& v : L.vars) last = v.begin > last ? v.begin : last;
        if (version == 2 || last <= 0x7fffffffull) return true;
    }
    return false;
}

__device__ __forceinline__ unsigned be32(float f) {
    return __byte_perm(__float_as_uint(f), 0, 0x0123);
}

template <typename T>
__device__ __forceinline__ float to_f32(T v) {
    return (float)v;  // round to nearest, as netCDF's double -> float conversion
}

// one record's field bytes (the time value is filled on the host)
template <typename T>
__global__ void __launch_bounds__(256)
    k_pack_record(Dims d, const T* __restrict__ u, const T* __restrict__ v,
                  const T* __restrict__ w, const T* __restrict__ th,
                  const double* __restrict__ p, const double* __restrict__ div,
                  const T* const* __restrict__ q, int nq, unsigned* __restrict__ rec,
                  size_t off_th, size_t off_q) {
    const int k = 1 + blockIdx.x * BX + threadIdx.x;
    const int j = 1 + blockIdx.y * BY + threadIdx.y;
    const int i = 1 + blockIdx.z;
    if (k > d.kp || j > d.jp) return;
    const int o = d.at(k, j, i);
    const size_t n = (size_t)d.kp * d.jp * d.ip;
    const size_t e = (size_t)(k - 1) + (size_t)d.kp * ((size_t)(j - 1) + (size_t)d.jp * (i - 1));
    unsigned* f = rec + off_th / 4;
    // th, u, v, w, p, div: the reference's order of definition (:880-931)
    f[e] = be32(to_f32(th[o]));
    f[n + e] = be32(to_f32(u[o]));
    f[2 * n + e] = be32(to_f32(v[o]));
    f[3 * n + e] = be32(to_f32(w[o]));
    f[4 * n + e] = be32(to_f32(p[o]));
    f[5 * n + e] = be32(to_f32(div[o]));
    // q(nq, kp, jp, ip): the q index fastest (:1112-1117)
    unsigned* fq = rec + off_q / 4;
    for (int m = 0; m < nq; m++) fq[(size_t)m + (size_t)nq * e] = be32(to_f32(q[m][o]));
}

struct Job {
    int slot;
    long long rec;
    double time;
};

}  // namespace

struct dcm_output {
    dcm_handle* h = nullptr;
    int device = 0;
    Layout L;
    FILE* f = nullptr;
    int nq = 0;
    size_t off_th = 0, off_q = 0;  // within a record
    long long nrec = 0;            // records queued
    float* dev[2] = {nullptr, nullptr};
    float* host[2] = {nullptr, nullptr};
    const void** dq = nullptr;     // device array of the q field pointers
    cudaEvent_t packed[2] = {nullptr, nullptr}, copied[2] = {nullptr, nullptr};
    cudaStream_t st = nullptr;     // the copy stream
    std::thread writer;
    std::mutex mu;
    std::condition_variable cv;
    std::deque<Job> jobs;
    bool busy[2] = {false, false};
    bool stop = false;
    int err = DCM_OK;
    std::string what;
};

namespace {

void fail_io(dcm_output* o, const std::string& what) {
    std::lock_guard<std::mutex> lk(o->mu);
    if (o->err == DCM_OK) {
        o->err = DCM_E_IO;
        o->what = what;
    }
}

void writer_loop(dcm_output* o) {
    cudaSetDevice(o->device);
    for (;;) {
        Job job;
        {
            std::unique_lock<std::mutex> lk(o->mu);
            o->cv.wait(lk, [&] { return o->stop || !o->jobs.empty(); });
            if (o->jobs.empty()) return;
            job = o->jobs.front();
        }
        bool good = cudaEventSynchronize(o->copied[job.slot]) == cudaSuccess;
        if (!good) fail_io(o, "output: device copy failed");
        if (good) {
            // time is the first record variable (:816-818, :1071-1073)
            const float t = (float)job.time;
            uint32_t tb;
            std::memcpy(&tb, &t, 4);
            uint8_t* r = (uint8_t*)o->host[job.slot];
            for (int s = 0; s < 4; s++) r[s] = (uint8_t)(tb >> (24 - 8 * s));
            const uint64_t at = o->L.rec_begin + (uint64_t)job.rec * o->L.recsize;
            good = fseeko(o->f, (off_t)at, SEEK_SET) == 0 &&
                   fwrite(r, 1, o->L.recsize, o->f) == o->L.recsize;
            // the record count (numrecs, header offset 4)
            const uint32_t nr = (uint32_t)(job.rec + 1);
            const uint8_t nb[4] = {(uint8_t)(nr >> 24), (uint8_t)(nr >> 16), (uint8_t)(nr >> 8),
                                   (uint8_t)nr};
            good = good && fseeko(o->f, 4, SEEK_SET) == 0 && fwrite(nb, 1, 4, o->f) == 4 &&
                   fflush(o->f) == 0;
            if (!good) fail_io(o, "output: writing the file failed");
        }
        {
            std::lock_guard<std::mutex> lk(o->mu);
            o->jobs.pop_front();
            o->busy[job.slot] = false;
        }
        o->cv.notify_all();
    }
}

void release(dcm_output* o) {
    if (!o) return;
    if (o->writer.joinable()) {
        {
            std::lock_guard<std::mutex> lk(o->mu);
            o->stop = true;
        }
        o->cv.notify_all();
        o->writer.join();
    }
    if (o->st) cudaStreamSynchronize(o->st);
    for (int s = 0; s < 2; s++) {
        if (o->dev[s]) cudaFree(o->dev[s]);
        if (o->host[s]) cudaFreeHost(o->host[s]);
        if (o->packed[s]) cudaEventDestroy(o->packed[s]);
        if (o->copied[s]) cudaEventDestroy(o->copied[s]);
    }
    if (o->dq) cudaFree(o->dq);
    if (o->st) cudaStreamDestroy(o->st);
    if (o->f) fclose(o->f);
    delete o;
}

}  // namespace

extern "C" int dcm_output_open(dcm_handle* h, const char* path, const double* x,
                               const double* y, const double* z, const double* trefn, int nq,
                               const char* q_names, int nprec, dcm_output** out) {
    if (!h || !path || !x || !y || !z || !out) return DCM_E_ARG;
    *out = nullptr;
    ResidentView V;
    if (resident_view(h, &V) != DCM_OK) return DCM_E_ARG;  // no state uploaded
    const int nqs = (int)V.q.size();
    if (nq != nqs) return DCM_E_ARG;  // the q fields are the resident ones
    if (nq > 0 && (!q_names || nprec < 1)) return DCM_E_ARG;
    const Dims& d = V.d;
    const uint64_t n = (uint64_t)d.ip * d.jp * d.kp;
    if (4 * n * (uint64_t)(nq > nprec ? nq : nprec) > 0xfffffffcull || 4 * n > 0xfffffffcull)
        return DCM_E_UNSUPPORTED;  // a variable's record would not fit the 32-bit vsize
    std::vector<double> rhoa, thetan;
    if (host_profiles(h, &rhoa, &thetan) != DCM_OK) return DCM_E_CUDA;

    dcm_output* o = new dcm_output();
    o->h = h;
    o->device = V.device;
    o->nq = nq;
    Layout& L = o->L;
    // dimensions (:794-802): ids 0 times, 1 ip, 2 jp, 3 kp, 4 nq, 5 nprec, 6 l_q_names
    L.dims = {{"times", 0}, {"ip", (uint64_t)d.ip}, {"jp", (uint64_t)d.jp}, {"kp", (uint64_t)d.kp}};
    if (nq > 0) {
        L.dims.push_back({"nq", (uint64_t)nq});
        L.dims.push_back({"nprec", (uint64_t)nprec});
        L.dims.push_back({"l_q_names", (uint64_t)LQ});
    }
    auto r4 = [](uint64_t b) { return (b + 3) / 4 * 4; };
    auto var = [&](const char* nm, const char* units, std::vector<int> dims, int type,
                   uint64_t vsize) {
        Var v;
        v.name = nm;
        v.units = units;
        v.dims = dims;
        v.type = type;
        v.record = !dims.empty() && dims[0] == 0;
        v.vsize = r4(vsize);
        L.vars.push_back(v);
    };
    // variables in the reference's order of definition (:816-957); a
    // Fortran dimension list (kp, jp, ip, times) is (times, ip, jp, kp) here
    var("time", "seconds", {0}, NC_FLOAT, 4);
    var("x", "m", {1}, NC_FLOAT, 4 * (uint64_t)d.ip);
    var("y", "m", {2}, NC_FLOAT, 4 * (uint64_t)d.jp);
    var("z", "m", {3}, NC_FLOAT, 4 * (uint64_t)d.kp);
    var("rhoa", "kg/m3", {3}, NC_FLOAT, 4 * (uint64_t)d.kp);
    var("thetan", "K", {3}, NC_FLOAT, 4 * (uint64_t)d.kp);
    var("trefn", "K", {3}, NC_FLOAT, 4 * (uint64_t)d.kp);
    const char* names[6] = {"th", "u", "v", "w", "p", "div"};
    const char* units[6] = {"K", "m/s", "m/s", "m/s", "pa", "m/s**2"};
    for (int c = 0; c < 6; c++) var(names[c], units[c], {0, 1, 2, 3}, NC_FLOAT, 4 * n);
    if (nq > 0) {
        var("q_names", "", {4, 6}, NC_CHAR, (uint64_t)nq * LQ);
        var("q", "kg or number per kg", {0, 1, 2, 3, 4}, NC_FLOAT, 4 * n * (uint64_t)nq);
        var("precip", "mm hr-1 or number per m-2 s-1", {0, 1, 2, 3, 5}, NC_FLOAT,
            4 * n * (uint64_t)nprec);
    }
    if (!place(L)) {
        release(o);
        return DCM_E_UNSUPPORTED;
    }
    for (const Var& v : L.vars) {
        if (v.name == "th") o->off_th = v.begin - L.rec_begin;
        if (v.name == "q") o->off_q = v.begin - L.rec_begin;
    }
    // the header, the fixed variables (:1024-1050, the q names :962-966)
    o->f = fopen(path, "wb+");
    if (!o->f) {
        release(o);
        return DCM_E_IO;
    }
    std::vector<uint8_t> file = encode(L, 0);
    file.resize(L.rec_begin, 0);
    auto put_f32 = [&](uint64_t at, double val) {
        const float fv = (float)val;
        uint32_t b;
        std::memcpy(&b, &fv, 4);
        for (int s = 0; s < 4; s++) file[at + s] = (uint8_t)(b >> (24 - 8 * s));
    };
    for (const Var& v : L.vars) {
        if (v.record) continue;
        const double* src = v.name == "x" ? x : v.name == "y" ? y : v.name == "z" ? z
                          : v.name == "rhoa" ? rhoa.data() : v.name == "thetan" ? thetan.data()
                          : v.name == "trefn" ? trefn : nullptr;
        if (v.name == "q_names") {
            // Fortran character(len=20) names, blank padded
            std::memcpy(&file[v.begin], q_names, (size_t)nq * LQ);
            continue;
        }
        const uint64_t cnt = v.vsize / 4;
        for (uint64_t e = 0; e < cnt; e++) put_f32(v.begin + 4 * e, src ? src[1 + e] : 0.0);
    }
    if (fwrite(file.data(), 1, file.size(), o->f) != file.size() || fflush(o->f) != 0) {
        release(o);
        return DCM_E_IO;
    }
    // staging: two records on the device and in pinned host memory
    bool good = cudaSetDevice(o->device) == cudaSuccess &&
                cudaStreamCreateWithFlags(&o->st, cudaStreamNonBlocking) == cudaSuccess;
    for (int s = 0; s < 2 && good; s++) {
        good = cudaMalloc(&o->dev[s], L.recsize) == cudaSuccess &&
               cudaMemset(o->dev[s], 0, L.recsize) == cudaSuccess &&  // precip stays 0
               cudaMallocHost(&o->host[s], L.recsize) == cudaSuccess &&
               cudaEventCreateWithFlags(&o->packed[s], cudaEventDisableTiming) == cudaSuccess &&
               cudaEventCreateWithFlags(&o->copied[s], cudaEventDisableTiming) == cudaSuccess;
    }
    if (good && nq > 0)
        good = cudaMalloc(&o->dq, nq * sizeof(void*)) == cudaSuccess &&
               cudaMemcpy(o->dq, V.q.data(), nq * sizeof(void*), cudaMemcpyHostToDevice) ==
                   cudaSuccess;
    if (!good) {
        release(o);
        return DCM_E_CUDA;
    }
    o->writer = std::thread(writer_loop, o);
    *out = o;
    return DCM_OK;
}

extern "C" int dcm_output_write(dcm_output* o, double time) {
    if (!o) return DCM_E_ARG;
    ResidentView V;
    if (resident_view(o->h, &V) != DCM_OK || (int)V.q.size() != o->nq) return DCM_E_ARG;
    const int s = (int)(o->nrec % 2);
    {
        std::unique_lock<std::mutex> lk(o->mu);
        o->cv.wait(lk, [&] { return !o->busy[s] || o->err != DCM_OK; });
        if (o->err != DCM_OK) return o->err;
        o->busy[s] = true;
    }
    if (o->nq > 0)
        cudaMemcpyAsync(o->dq, V.q.data(), o->nq * sizeof(void*), cudaMemcpyHostToDevice, V.st);
    const Dims& d = V.d;
    const dim3 b(BX, BY), g = interior_grid(d, d.kp);
    unsigned* rec = (unsigned*)o->dev[s];
    if (V.prec == 0)
        k_pack_record<double><<<g, b, 0, V.st>>>(
            d, (const double*)V.u, (const double*)V.v, (const double*)V.w, (const double*)V.th,
            V.p, V.div, (const double* const*)o->dq, o->nq, rec, o->off_th, o->off_q);
    else
        k_pack_record<float><<<g, b, 0, V.st>>>(
            d, (const float*)V.u, (const float*)V.v, (const float*)V.w, (const float*)V.th,
            V.p, V.div, (const float* const*)o->dq, o->nq, rec, o->off_th, o->off_q);
    bool good = cudaGetLastError() == cudaSuccess &&
                cudaEventRecord(o->packed[s], V.st) == cudaSuccess &&
                cudaStreamWaitEvent(o->st, o->packed[s], 0) == cudaSuccess &&
                cudaMemcpyAsync(o->host[s], o->dev[s], o->L.recsize, cudaMemcpyDeviceToHost,
                                o->st) == cudaSuccess &&
                cudaEventRecord(o->copied[s], o->st) == cudaSuccess;
    if (!good) {
        std::lock_guard<std::mutex> lk(o->mu);
        o->busy[s] = false;
        return DCM_E_CUDA;
    }
    {
        std::lock_guard<std::mutex> lk(o->mu);
        o->jobs.push_back(Job{s, o->nrec, time});
    }
    o->nrec += 1;
    o->cv.notify_all();
    return DCM_OK;
}

extern "C" int dcm_output_flush(dcm_output* o) {
    if (!o) return DCM_E_ARG;
    std::unique_lock<std::mutex> lk(o->mu);
    o->cv.wait(lk, [&] { return o->jobs.empty(); });
    return o->err;
}

extern "C" int dcm_output_close(dcm_output* o) {
    if (!o) return DCM_OK;
    const int rc = dcm_output_flush(o);
    release(o);
    return rc;
}

extern "C" const char* dcm_output_last_error(const dcm_output* o) {
    return o ? o->what.c_str() : "";
}
