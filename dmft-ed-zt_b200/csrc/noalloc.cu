// noalloc.cu — edzt_lanczos_iteration_noalloc: the persistent Lanczos kernel
// run from a fixed, statically allocated scratch area.
//
// For callers that cannot call cudaMalloc/cudaFree: a host program whose
// device memory is all owned by another allocator (a framework's caching
// allocator, a fixed memory budget) or a latency-critical loop that must not
// take the device-wide synchronisation an allocation or free can cause.  The
// call uses no device memory but the scratch array below and the context's
// model tables, which an earlier allocating call on the same sector built.
//
// Scratch: one file-scope __device__ array of kNoAllocScratchBytes (13.1 MiB)
// that every GPU which loads the library holds until the process exits.  It
// limits the sector to EDZT_NOALLOC_MAX_DIM states and the run to
// EDZT_NOALLOC_MAX_STEPS steps.  The first call on each device looks the
// array's address up (cudaGetSymbolAddress) with that device current; that
// first call should come before any stream capture.  The address is kept for
// the life of the process, so cudaDeviceReset (which tears down the device's
// context and with it the array) is not supported while the library is
// loaded.  Calls share the one array per device, so calls whose GPU work
// overlaps (two contexts or two host threads on the same device) race and
// must be serialised by the caller.
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <vector>
#include <string>
#include <cuda_runtime.h>
#include "../../include/edzt.h"
#include "edzt_internal.h"

namespace {

constexpr int kMaxDevices = 64;
constexpr int kMaxGrid = 2048;                         // CTAs of the persistent launch
constexpr size_t kAlign = 256;
constexpr size_t al(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

// scratch layout (byte offsets)
constexpr size_t kOffJob = 0;
constexpr size_t kOffState = kOffJob + al(2048);        // LzJob
constexpr size_t kOffPrefix = kOffState + al(2 * sizeof(LzState));
// the jobs' first tiles, the CTA ranges and the column phase's slab order
// (at most one slab per two up strings)
constexpr size_t kOffStatus = kOffPrefix + al((4 + 2 * (kMaxGrid + 1) + EDZT_NOALLOC_MAX_DIM / 2) * sizeof(long long));
constexpr size_t kOffSync = kOffStatus + al(sizeof(int));
constexpr size_t kSyncBytes = al(sizeof(unsigned) * (128 + 32 * ((kMaxGrid + 15) / 16)));
constexpr size_t kOffSlots = kOffSync + kSyncBytes;     // [2 phases * kMaxGrid][2] doubles
constexpr size_t kOffAB = kOffSlots + al(sizeof(double) * 4 * kMaxGrid);
constexpr size_t kOffYW = kOffAB + al(sizeof(double) * 2 * EDZT_NOALLOC_MAX_STEPS);
constexpr size_t kYWBytes = sizeof(double2) * (size_t)EDZT_NOALLOC_MAX_DIM;
constexpr size_t kOffD = kOffYW + 2 * kYWBytes;
// D is slab-major with slabs of up to 8 columns: up to 7 padding columns of
// every row past the sector's own states
constexpr size_t kDDoubles = 2 * (size_t)EDZT_NOALLOC_MAX_DIM;
constexpr size_t kNoAllocScratchBytes = kOffD + sizeof(double) * kDDoubles;

static_assert(sizeof(LzJob) <= 2048, "job descriptor outgrew its scratch slot");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_setup_mu;
unsigned char* g_scratch_ptr[kMaxDevices] = {};

// Set-up, once per device, with that device current: the scratch address.
int scratch_for(int device, unsigned char** out, std::string& why)
{
    if (device < 0 || device >= kMaxDevices) {
        why = "device ordinal beyond the no-allocation table";
        return EDZT_ERR_ARG;
    }
    std::lock_guard<std::mutex> lk(g_setup_mu);
    if (!g_scratch_ptr[device]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) {
            cudaGetLastError();
            why = std::string("cudaGetSymbolAddress(no-allocation scratch): ") + cudaGetErrorString(e);
            return EDZT_ERR_CUDA;
        }
        g_scratch_ptr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_scratch_ptr[device];
    return EDZT_OK;
}

struct Fail {
    int code;
    std::string msg;
};

// True when the kernel can read p directly: device memory of `device` or
// managed memory.  Device memory of another GPU is rejected.
bool is_device_ptr(const void* p, int device)
{
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    if (at.type == cudaMemoryTypeDevice && at.device != device)
        throw Fail{EDZT_ERR_ARG, "v_init is device memory of GPU " + std::to_string(at.device) +
                                     ", not of the context's GPU " + std::to_string(device)};
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

#define NA_CK(call)                                                                                \
    do {                                                                                           \
        const cudaError_t _e = (call);                                                             \
        if (_e != cudaSuccess) throw Fail{EDZT_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)}; \
    } while (0)

void run(edzt_ctx* c, int ne_up, int ne_dn, const double* v_init, int maxnstep, int* nstep, double* a, double* b)
{
    if (!v_init || !nstep || !a || !b) throw Fail{EDZT_ERR_ARG, "null argument"};
    if (maxnstep < 1 || maxnstep > EDZT_NOALLOC_MAX_STEPS)
        throw Fail{EDZT_ERR_ARG, "maxnstep " + std::to_string(maxnstep) + " outside [1, " +
                                     std::to_string(EDZT_NOALLOC_MAX_STEPS) + "] (no-allocation limit)"};
    const int device = edzt_ctx_device(c);
    NA_CK(cudaSetDevice(device));
    const long long dim = edzt_sector_dim(c, ne_up, ne_dn);
    if (dim > EDZT_NOALLOC_MAX_DIM)
        throw Fail{EDZT_ERR_ARG, "sector dimension " + std::to_string(dim) + " exceeds the no-allocation limit of " +
                                     std::to_string(EDZT_NOALLOC_MAX_DIM) + " states"};
    DevSector S;
    const char* why = nullptr;
    int rc = edzt_ctx_ready_sector(c, ne_up, ne_dn, &S, &why);
    if (rc != EDZT_OK) throw Fail{rc, why};
    if (S.dim < 1) throw Fail{EDZT_ERR_ARG, "empty sector"};
    unsigned char* base = nullptr;
    std::string swhy;
    rc = scratch_for(device, &base, swhy);
    if (rc != EDZT_OK) throw Fail{rc, swhy};
    const cudaStream_t st = edzt_ctx_stream(c);

    LzJob* d_job = reinterpret_cast<LzJob*>(base + kOffJob);
    LzState* d_state = reinterpret_cast<LzState*>(base + kOffState);
    long long* d_prefix = reinterpret_cast<long long*>(base + kOffPrefix);
    int* d_status = reinterpret_cast<int*>(base + kOffStatus);
    unsigned* d_sync = reinterpret_cast<unsigned*>(base + kOffSync);
    double* d_slots = reinterpret_cast<double*>(base + kOffSlots);
    double* d_a = reinterpret_cast<double*>(base + kOffAB);
    double* d_b = d_a + EDZT_NOALLOC_MAX_STEPS;
    double2* d_yw0 = reinterpret_cast<double2*>(base + kOffYW);
    double2* d_yw1 = reinterpret_cast<double2*>(base + kOffYW + kYWBytes);
    double* d_d = reinterpret_cast<double*>(base + kOffD);

    LzJob J;
    std::memset(&J, 0, sizeof(J));
    J.S = S;
    J.YW[0] = d_yw0;
    J.YW[1] = d_yw1;
    J.D = d_d;
    J.a = d_a;
    J.b = d_b;
    J.maxnstep = maxnstep;
    J.mode = LZ_COEFF;
    J.init = LZ_INIT_COPY;
    J.st = d_state;
    // the same tile shapes, grid and shared memory as the allocating path
    std::vector<long long> prefix;
    const LzPlan P = lz_plan(device, &J, 1, prefix);
    if (P.grid <= 0) throw Fail{EDZT_ERR_CUDA, "persistent kernel cannot be resident (shared memory too large)"};
    if (P.grid > kMaxGrid) throw Fail{EDZT_ERR_CUDA, "persistent grid larger than the no-allocation sync area"};
    if ((size_t)((S.up.count + J.ph[0].width - 1) / J.ph[0].width) * J.ph[0].width * S.dn.count > kDDoubles)
        throw Fail{EDZT_ERR_ARG, "sector's column slabs exceed the no-allocation scratch"};
    // The start vector is read in the first step only (both phases), which
    // writes YW[1]; a host vector is staged in YW[0], first written by step 2.
    if (is_device_ptr(v_init, device)) {
        J.src = v_init;
    } else {
        NA_CK(cudaMemcpyAsync(d_yw0, v_init, sizeof(double) * S.dim, cudaMemcpyHostToDevice, st));
        J.src = reinterpret_cast<const double*>(d_yw0);
    }
    LzState hs[2];
    std::memset(hs, 0, sizeof(hs));
    hs[1].active = 1;                                    // the state before phase 0 (parity 1)
    // what must start at zero: the barrier's sync words (but the count of
    // runs still going, one), status, a, b
    const unsigned runs_going = 1u;
    NA_CK(cudaMemsetAsync(d_sync, 0, lz_sync_bytes(P.grid), st));
    NA_CK(cudaMemcpyAsync(d_sync + 64, &runs_going, sizeof(unsigned), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    NA_CK(cudaMemsetAsync(d_a, 0, sizeof(double) * 2 * EDZT_NOALLOC_MAX_STEPS, st));
    NA_CK(cudaMemcpyAsync(d_job, &J, sizeof(J), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(d_state, hs, sizeof(hs), cudaMemcpyHostToDevice, st));
    NA_CK(cudaMemcpyAsync(d_prefix, prefix.data(), sizeof(long long) * prefix.size(), cudaMemcpyHostToDevice, st));
    LzBatch B;
    std::memset(&B, 0, sizeof(B));
    B.njobs = 1;
    B.grid = P.grid;
    B.block = P.block;
    B.smem = P.smem;
    B.total[0] = P.total[0];
    B.total[1] = P.total[1];
    B.max_phases = 2 * maxnstep + 4;
    B.stall_cta = -1;
    NA_CK(launch_lanczos_persistent(B, d_job, d_prefix, d_slots, d_sync, d_status, st));
    edzt_count_launches(c, 1);
    int status = 0;
    NA_CK(cudaMemcpyAsync(hs, d_state, sizeof(hs), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(&status, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    NA_CK(cudaMemcpyAsync(a, d_a, sizeof(double) * maxnstep, cudaMemcpyDefault, st));
    NA_CK(cudaMemcpyAsync(b, d_b, sizeof(double) * maxnstep, cudaMemcpyDefault, st));
    NA_CK(cudaStreamSynchronize(st));
    if (status == EDZT_DEV_BARRIER_TIMEOUT)
        throw Fail{EDZT_ERR_TIMEOUT, "persistent Lanczos kernel: grid barrier wait timed out"};
    if (status != 0) throw Fail{EDZT_ERR_CUDA, "persistent Lanczos kernel reported status " + std::to_string(status)};
    const LzState* fin = !hs[0].active ? &hs[0] : (!hs[1].active ? &hs[1] : nullptr);
    if (!fin) throw Fail{EDZT_ERR_NUMERIC, "Lanczos run did not finish within the pass limit"};
    *nstep = fin->nstep;
}

}  // namespace

extern "C" int edzt_lanczos_iteration_noalloc(edzt_ctx* c, int ne_up, int ne_dn, const double* v_init, int maxnstep,
                                              int* nstep, double* a, double* b)
{
    if (!c) return EDZT_ERR_ARG;
    try {
        run(c, ne_up, ne_dn, v_init, maxnstep, nstep, a, b);
        edzt_ctx_set_error(c, "");
        return EDZT_OK;
    } catch (const Fail& f) {
        edzt_ctx_set_error(c, f.msg.c_str());
        return f.code;
    } catch (const std::exception& e) {
        edzt_ctx_set_error(c, e.what());
        return EDZT_ERR_CUDA;
    }
}
