// shtc_synthesis_noalloc: the synthesis (MakeGridDH / MakeGridGLQ) of
// shtc_synthesis with its workspace taken from a fixed array compiled into
// the library instead of from the caller.
//
// Who needs it: callers that must not allocate device memory inside their
// own calls -- programs whose GPU memory is owned by a pool or budget manager
// that forbids outside cudaMalloc, and latency-sensitive loops that cannot
// afford cudaMalloc's implicit device synchronisation -- but that still want
// a transform without managing a workspace buffer themselves.
//
// The array, g_scratch, is a file-scope __device__ array of
// SHTC_NOALLOC_SCRATCH_BYTES (16 MiB).  A call fits when
// shtc_workspace_bytes(plan, nfield) does: that size includes the plan's
// analysis partial-sum tiles (which follow its tile shape, set by the
// autotuner or shtc_plan_set_tuning) and, for a plan of tensor-core
// precision, the coefficient image of that path.  Every GPU that loads this library
// holds it until the process exits.  Host code cannot use the name
// g_scratch as a device address (it is a host-side stand-in), so the first
// call on each device looks up the real address with cudaGetSymbolAddress,
// with that device current, and caches it; make that first call before any
// stream capture.  The call itself allocates nothing: no cudaMalloc,
// cudaFree or allocating library routine.
//
// All calls share the one array and it keeps the last call's contents.
// Every byte the synthesis kernels read from it is written earlier in the
// same call (the packed coefficients and the per-ring Fourier sums), so
// nothing needs clearing between calls.  Calls whose kernels overlap on the
// GPU (different streams without ordering) race on the array: serialise
// them.
#include <cuda_runtime.h>

#include <mutex>

#include "shtc_internal.cuh"

namespace {

constexpr size_t kScratchBytes = SHTC_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_scratch_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};

// Device address of g_scratch on the current device (set-up on first use).
int scratch_address(void** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return SHTC_ECUDA;
    if (dev < 0 || dev >= kMaxDevices) return SHTC_EUNSUP;
    std::lock_guard<std::mutex> g(g_scratch_mu);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess || !p) return SHTC_ECUDA;
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return SHTC_OK;
}

}  // namespace

extern "C" SHTC_API int shtc_synthesis_noalloc(
    const shtc_plan* plan, const double* cilm, long long csf, long long csk,
    long long csl, long long csm, int cilm_dim, double* grid, long long gsf,
    long long gsr, long long gsc, int nfield, void* stream) {
    if (!plan || !cilm || !grid) return SHTC_EHANDLE;
    if (nfield < 1) return SHTC_EBOUND;
    // the plan's device must be current before the first call sets up the
    // array's address there (otherwise a device the caller never uses would
    // be initialised, and the synthesis would refuse the call anyway)
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return SHTC_ECUDA;
    if (dev != plan->device) return SHTC_EHANDLE;
    const size_t need = shtc_workspace_bytes(plan, nfield);
    if (need == 0) return SHTC_EHANDLE;
    if (need > kScratchBytes) return SHTC_EWORK;   // beyond the fixed array
    void* ws = nullptr;
    int rc = scratch_address(&ws);
    if (rc) return rc;
    return shtc_synthesis(plan, cilm, csf, csk, csl, csm, cilm_dim, grid, gsf,
                          gsr, gsc, nfield, ws, kScratchBytes, stream);
}
