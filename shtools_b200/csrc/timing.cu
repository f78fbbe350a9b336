// Per-kernel device timing of libshtcuda: when enabled, every kernel stage of
// a transform is bracketed by CUDA events recorded on the launching stream.
// The benchmark reads the summed stage times to compute the roofline of the
// dominant kernel without a profiler; disabled (the default) it costs one
// branch per launch.
#include <cuda_runtime.h>

#include <mutex>
#include <vector>

#include "shtc_internal.cuh"

namespace shtc {

namespace {
struct Rec {
    int stage;
    cudaEvent_t a, b;
};
std::mutex g_mu;
std::vector<Rec> g_recs;
std::vector<cudaEvent_t> g_pool;
volatile int g_on = 0;
thread_local Rec t_open = {-1, nullptr, nullptr};

cudaEvent_t take_event() {
    if (!g_pool.empty()) {
        cudaEvent_t e = g_pool.back();
        g_pool.pop_back();
        return e;
    }
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    return e;
}
}  // namespace

void stage_begin(int stage, cudaStream_t st) {
    if (!g_on) return;
    std::lock_guard<std::mutex> g(g_mu);
    t_open.stage = stage;
    t_open.a = take_event();
    t_open.b = take_event();
    cudaEventRecord(t_open.a, st);
}

void stage_end(int stage, cudaStream_t st) {
    if (!g_on || t_open.stage != stage) return;
    std::lock_guard<std::mutex> g(g_mu);
    cudaEventRecord(t_open.b, st);
    g_recs.push_back(t_open);
    t_open.stage = -1;
}

}  // namespace shtc

using namespace shtc;

extern "C" SHTC_API int shtc_timing_enable(int on) {
    g_on = on ? 1 : 0;
    return SHTC_OK;
}

// Waits for the recorded events, writes per-stage total milliseconds and
// launch counts for stages 0..n-1 and forgets the records.
extern "C" SHTC_API int shtc_timing_collect(double* ms, int* counts, int n) {
    std::lock_guard<std::mutex> g(g_mu);
    for (int i = 0; i < n; ++i) {
        ms[i] = 0.0;
        counts[i] = 0;
    }
    int rc = SHTC_OK;
    for (const Rec& r : g_recs) {
        float t = 0.0f;
        if (cudaEventSynchronize(r.b) != cudaSuccess ||
            cudaEventElapsedTime(&t, r.a, r.b) != cudaSuccess)
            rc = SHTC_ECUDA;
        if (r.stage >= 0 && r.stage < n) {
            ms[r.stage] += t;
            counts[r.stage] += 1;
        }
        g_pool.push_back(r.a);
        g_pool.push_back(r.b);
    }
    g_recs.clear();
    return rc;
}
