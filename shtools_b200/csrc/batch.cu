// Batched transforms of many fields on several grids (e.g. GLQ grids of
// uneven lmax): one persistent Legendre launch over (grid group, order m,
// ring tile, field chunk) work items, plus one launch each for packing and
// for all longitude FFTs, so a whole batch is a handful of launches that a
// CUDA graph can capture and replay.
//
// A batch references plans (one per distinct grid and option set); fields
// of one plan form a group and share the Legendre recursion.  Work items are
// sorted by cost, longest first, and handed out through a global counter:
// the persistent CTAs then finish together (longest-processing-time-first
// scheduling).  Layout of the caller's arrays: the groups one after another,
// a group holding nf fields as (nf, 2, lc+1, lc+1) coefficients and
// (nf, nlat, nlon) grids, C order (offsets from shtc_batch_layout).
#include <cuda_runtime.h>

#include <algorithm>
#include <new>
#include <vector>

#include "fft.cuh"
#include "legendre.cuh"
#include "shtc_internal.cuh"

namespace shtc {

struct BatchGroup {
    const double2* rec;
    const double* pmm;
    const double* rtab;
    const double* z;
    const int* rowN;
    const int* rowS;
    const int* arowN;
    const int* arowS;
    const double* wN;
    const double* wS;
    const double* nrm3;
    int lc, npair, nf, norm, nlat, nlon, fft_jobs, tiles;
    double inv_nlon;
    long long nlm;
    long long cilm_off;   // caller coefficients (doubles)
    long long grid_off;   // caller grids (doubles)
    long long pack_off;   // workspace: packed coefficients / analysis partials (double2)
    long long spec_off;   // workspace: ring spectra (double2)
};

// synthesis: four fields per recursion (eight measured 12% slower on B200
// for 4096 fields of lmax 31..511)
constexpr int kBatchSynthNF = 4;
constexpr int kBatchThreads = 128;        // synthesis: ring pairs per tile (T = 1)
// analysis: 2 warps x 4 ring pairs per lane = 256 pairs per tile, one tile
// per order for lmax <= 511; two fields share each recursion (7% faster
// than one on the same batch), and per degree a lane does 24 FP64
// operations against 4 shared-memory stores and loads, which keeps the
// transpose reduction off the critical path
constexpr int kBatchAnalWarps = 2;
constexpr int kBatchAnalT = 4;
constexpr int kBatchAnalNF = 2;
constexpr int kBatchAnalPairs = 32 * kBatchAnalWarps * kBatchAnalT;

// ---------------------------------------------------------------------------
// kernels
// ---------------------------------------------------------------------------
// pack: item (g, m); coefficients (nf, 2, D, D) -> packed [(l,m)][nf] {C, S},
// premultiplied by D(l - m) of the rescaled recursion
__global__ void k_batch_pack(const BatchGroup* __restrict__ G,
                             const int2* __restrict__ items,
                             const double* __restrict__ cilm,
                             double2* __restrict__ work) {
    const int2 it = items[blockIdx.x];
    const BatchGroup& g = G[it.x];
    const int m = it.y, lc = g.lc, D = lc + 1, nf = g.nf;
    const long long o = packed_off(m, lc);
    const double* c = cilm + g.cilm_off;
    double2* pk = work + g.pack_off;
    for (int l = m + threadIdx.x; l <= lc; l += blockDim.x) {
        // D(l - m) of the rescaled recursion (legendre.cuh)
        const double d = g.rec[o + (l - m)].y;
        for (int f = 0; f < nf; ++f) {
            const double* b = c + (long long)f * 2 * D * D + (long long)l * D + m;
            const double cs = b[0];
            const double sn = m == 0 ? 0.0 : b[(long long)D * D];
            pk[(o + (l - m)) * nf + f] = make_double2(cs * d, sn * d);
        }
    }
}

// unpack: item (g, m); tile sums, normalisation (SHExpandDH.f95:674-702)
__global__ void k_batch_unpack(const BatchGroup* __restrict__ G,
                               const int2* __restrict__ items,
                               const double2* __restrict__ work,
                               double* __restrict__ cilm) {
    const double pi = 3.141592653589793238462643383279502884;
    const int2 it = items[blockIdx.x];
    const BatchGroup& g = G[it.x];
    const int m = it.y, lc = g.lc, D = lc + 1, nf = g.nf;
    const long long o = packed_off(m, lc);
    const double2* part = work + g.pack_off;
    double* c = cilm + g.cilm_off;
    for (int l = m + threadIdx.x; l <= lc; l += blockDim.x) {
        const long long idx = o + (l - m);
        for (int f = 0; f < nf; ++f) {
            double cs = 0.0, sn = 0.0;
            for (int t = 0; t < g.tiles; ++t) {
                const double2 v = part[((long long)t * nf + f) * g.nlm + idx];
                cs += v.x;
                sn += v.y;
            }
            switch (g.norm) {
                case 1: cs = cs / (4 * pi); sn = sn / (4 * pi); break;
                case 2:
                    cs = cs * (2 * l + 1) / (4 * pi);
                    sn = sn * (2 * l + 1) / (4 * pi);
                    break;
                case 3: cs = cs / g.nrm3[idx]; sn = sn / g.nrm3[idx]; break;
                default: break;
            }
            double* b = c + (long long)f * 2 * D * D + (long long)l * D + m;
            b[0] = cs;
            b[(long long)D * D] = m == 0 ? 0.0 : sn;
        }
    }
}

__device__ __forceinline__ int next_item(int* counter, int* s_item) {
    if (threadIdx.x == 0) *s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = *s_item;
    __syncthreads();
    return it;
}

// persistent synthesis: item (g, m, tile, f0)
__global__ void __launch_bounds__(kBatchThreads)
k_batch_synth(const BatchGroup* __restrict__ G, const int4* __restrict__ items,
              int nitems, int* __restrict__ counter, double2* __restrict__ work) {
    __shared__ __align__(16) SynthStage<kBatchSynthNF> sm;
    __shared__ int s_item;
    for (;;) {
        const int i = next_item(counter, &s_item);
        if (i >= nitems) return;
        const int4 w = items[i];
        const BatchGroup& g = G[w.x];
        synth_order<1, kBatchSynthNF>(sm, g.rec, g.pmm, g.rtab, g.z, work + g.pack_off,
                                      work + g.spec_off, g.lc, g.npair, g.nf, w.y, w.z,
                                      w.w, min(kBatchSynthNF, g.nf - w.w));
    }
}

// persistent analysis: item (g, m, tile, f0), fields f0 .. f0+kBatchAnalNF-1
__global__ void __launch_bounds__(32 * kBatchAnalWarps)
k_batch_anal(const BatchGroup* __restrict__ G, const int4* __restrict__ items,
             int nitems, int* __restrict__ counter, double2* __restrict__ work) {
    extern __shared__ __align__(16) double smem_anal[];
    __shared__ __align__(16) double2 rstage[2][kAnalStage];
    __shared__ int s_item;
    for (;;) {
        const int i = next_item(counter, &s_item);
        if (i >= nitems) return;
        const int4 w = items[i];
        const BatchGroup& g = G[w.x];
        const int f0 = w.w;
        const long long sstride = (long long)g.npair * (g.lc + 1) * 2;
        anal_order<kBatchAnalT, kBatchAnalNF>(smem_anal, rstage, g.rec, g.pmm, g.rtab, g.z,
                                    work + g.spec_off + f0 * sstride, sstride,
                                    work + g.pack_off + ((long long)w.z * g.nf + f0) * g.nlm,
                                    g.nlm, g.lc, g.npair, w.y, w.z,
                                    min(kBatchAnalNF, g.nf - f0));
    }
}

// Persistent FFT kernels: items (g, f, job) are handed out through a global
// counter, so CTAs stay busy across groups of different FFT lengths; the
// group's FftArgs are read in place from global memory, and the input lines
// of the CTA's next item are prefetched into L2 while the current FFT runs.
// The jobs are split into classes, one persistent launch each: groups whose
// radices are all <= 8 (every Bluestein length among them) run in a
// register-capped build (MAXR = 8, more CTAs per SM), the others (factors 11
// or 13) in the full build; within each, rings of up to 512 points run in
// 128-thread CTAs with their own (small) shared memory, longer ones in
// 256- or 512-thread CTAs.
template <int MAXR>
__global__ void __launch_bounds__(512, MAXR <= 8 ? 2 : 1)
k_batch_c2r(const BatchGroup* __restrict__ G, const FftArgs* __restrict__ FA,
            const int4* __restrict__ jobs, int njobs, int* __restrict__ counter,
            const double2* __restrict__ work, double* __restrict__ grid) {
    extern __shared__ double2 smem_fft[];
    __shared__ int s_item;
    int i = next_item(counter, &s_item);
    while (i < njobs) {
        const int nx = next_item(counter, &s_item);
        if (nx < njobs) {
            const int4 jn = jobs[nx];
            const BatchGroup& gn = G[jn.x];
            fft_c2r_prefetch(FA[jn.x].mode, jn.z, jn.y, work + gn.spec_off, gn.lc, gn.npair);
        }
        const int4 j = jobs[i];
        const BatchGroup& g = G[j.x];
        const FftArgs& F = FA[j.x];
        fft_c2r_body<double, MAXR>(F, F.tw, smem_fft, j.z, j.y, work + g.spec_off,
                             grid + g.grid_off, (long long)g.nlat * g.nlon, g.nlon, 1,
                             g.rowN, g.rowS, nullptr, nullptr, 1.0, g.lc, g.npair, 0);
        __syncthreads();
        i = nx;
    }
}

template <int MAXR>
__global__ void __launch_bounds__(512, MAXR <= 8 ? 2 : 1)
k_batch_r2c(const BatchGroup* __restrict__ G, const FftArgs* __restrict__ FA,
            const int4* __restrict__ jobs, int njobs, int* __restrict__ counter,
            const double* __restrict__ grid, double2* __restrict__ work) {
    extern __shared__ double2 smem_fft[];
    __shared__ int s_item;
    int i = next_item(counter, &s_item);
    while (i < njobs) {
        const int nx = next_item(counter, &s_item);
        if (nx < njobs) {
            const int4 jn = jobs[nx];
            const BatchGroup& gn = G[jn.x];
            const FftArgs& Fn = FA[jn.x];
            fft_r2c_prefetch<double>(Fn.mode, Fn.n, jn.z, jn.y, grid + gn.grid_off,
                                     (long long)gn.nlat * gn.nlon, gn.nlon, 1, gn.arowN,
                                     gn.arowS, 0);
        }
        const int4 j = jobs[i];
        const BatchGroup& g = G[j.x];
        const FftArgs& F = FA[j.x];
        fft_r2c_body<double, MAXR>(F, F.tw, smem_fft, j.z, j.y, grid + g.grid_off,
                             (long long)g.nlat * g.nlon, g.nlon, 1, work + g.spec_off,
                             g.arowN, g.arowS, g.wN, g.wS, g.inv_nlon, g.lc, g.npair, 0);
        __syncthreads();
        i = nx;
    }
}

}  // namespace shtc

using namespace shtc;

struct shtc_batch {
    int ngroup = 0;
    int device = 0;
    std::vector<BatchGroup> h_groups;
    BatchGroup* d_groups = nullptr;
    FftArgs* d_fft = nullptr;
    int2* d_pitems = nullptr;
    int npitems = 0;
    int4* d_sitems = nullptr;
    int nsitems = 0;
    int4* d_aitems = nullptr;
    int naitems = 0;
    // FFT job classes (fft_class): 2 * (a radix above 8) + (more than 128
    // threads); classes 0, 1 run the register-capped kernels
    static constexpr int kClasses = 4;
    int4* d_jobs[kClasses] = {};
    int njobs[kClasses] = {};
    int* d_counter = nullptr;   // [0] Legendre items, [1 + c] FFT jobs of class c
    size_t work_bytes = 0;
    size_t fft_smem[kClasses] = {};
    int fft_threads[kClasses] = {128, 128, 128, 128};
    int synth_ctas = 0;
    int anal_ctas = 0;
    int fft_ctas[kClasses] = {};
    long long cilm_total = 0;
    long long grid_total = 0;
};

static void batch_free(shtc_batch* B) {
    cudaFree(B->d_groups);
    cudaFree(B->d_fft);
    cudaFree(B->d_pitems);
    cudaFree(B->d_sitems);
    cudaFree(B->d_aitems);
    for (int c = 0; c < shtc_batch::kClasses; ++c) cudaFree(B->d_jobs[c]);
    cudaFree(B->d_counter);
}

// persistent CTAs of one FFT class: shared-memory size and carveout set on
// both kernels, as many CTAs as fit on every SM, at most one per job
template <typename KC, typename KR>
static int fft_class_ctas(KC kc, KR kr, int sm, int njobs, int threads, size_t smem) {
    if (njobs == 0) return 0;
    for (const void* fn : {(const void*)kc, (const void*)kr}) {
        cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    }
    int pc = 0, pr = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pc, kc, threads, smem);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&pr, kr, threads, smem);
    return std::min(njobs, sm * std::max(1, std::min(pc, pr)));
}

template <typename Tp>
static int upload(Tp** d, const std::vector<Tp>& h, cudaStream_t st) {
    if (cudaMalloc((void**)d, sizeof(Tp) * (h.empty() ? 1 : h.size())) != cudaSuccess)
        return SHTC_EALLOC;
    if (h.empty()) return SHTC_OK;
    return map_cuda(cudaMemcpyAsync(*d, h.data(), sizeof(Tp) * h.size(),
                                    cudaMemcpyHostToDevice, st));
}

extern "C" SHTC_API int shtc_batch_create(shtc_batch** out, int ngroup,
                                          shtc_plan* const* plans,
                                          const int* nfields, void* stream) {
    if (!out || !plans || !nfields || ngroup < 1) return SHTC_EHANDLE;
    *out = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    shtc_batch* B = new (std::nothrow) shtc_batch();
    if (!B) return SHTC_EALLOC;
    cudaGetDevice(&B->device);
    B->ngroup = ngroup;
    std::vector<FftArgs> fa(ngroup);
    long long pack = 0, spec = 0, coff = 0, goff = 0;
    constexpr int NC = shtc_batch::kClasses;
    size_t smem[NC] = {};
    int threads[NC] = {128, 128, 128, 128};
    struct Cost { double c; int4 it; };
    std::vector<Cost> sc, ac;
    std::vector<int2> pitems;
    std::vector<int4> jobs[NC];
    for (int gi = 0; gi < ngroup; ++gi) {
        const shtc_plan* P = plans[gi];
        const int nf = nfields[gi];
        if (!P || nf < 1 || P->device != B->device || P->extend != 0 || P->cplx) {
            delete B;
            return P && (P->extend != 0 || P->cplx) ? SHTC_EBOUND : SHTC_EHANDLE;
        }
        if (P->fft.gmem) {   // batched FFTs keep every ring in shared memory
            delete B;
            return SHTC_EUNSUP;
        }
        BatchGroup g;
        g.rec = P->d_rec; g.pmm = P->d_pmm; g.rtab = P->d_rtab; g.z = P->d_z;
        g.rowN = P->d_rowN; g.rowS = P->d_rowS; g.arowN = P->d_arowN;
        g.arowS = P->d_arowS; g.wN = P->d_wN; g.wS = P->d_wS; g.nrm3 = P->d_nrm;
        g.lc = P->lc; g.npair = P->npair; g.nf = nf; g.norm = P->norm;
        g.nlat = P->nlat; g.nlon = P->nlon;
        g.fft_jobs = P->fft.mode == 0 ? P->npair : 2 * P->npair;
        g.tiles = (P->npair + kBatchAnalPairs - 1) / kBatchAnalPairs;   // analysis tiles
        g.inv_nlon = 1.0 / (double)P->nlon;
        g.nlm = P->nlm;
        g.cilm_off = coff;
        g.grid_off = goff;
        g.pack_off = pack;
        g.spec_off = spec;
        coff += (long long)nf * 2 * (P->lc + 1) * (P->lc + 1);
        goff += (long long)nf * P->nlat * P->nlon;
        pack += (long long)P->nlm * nf * std::max(1, g.tiles);
        spec += (long long)nf * P->npair * (P->lc + 1) * 2;
        B->h_groups.push_back(g);
        fa[gi] = fft_args(P->fft);
        int cls = P->fft.threads > 128 ? 1 : 0;
        for (int i = 0; i < P->fft.nfac; ++i)
            if (P->fft.fac[i] > 8) cls = 2 + (cls & 1);
        smem[cls] = std::max(smem[cls], P->fft.smem_data);   // twiddles stay in global memory
        threads[cls] = std::max(threads[cls], P->fft.threads);
        // work items, with costs for longest-first ordering
        const int lc = P->lc;
        for (int m = 0; m <= lc; ++m) {
            pitems.push_back(make_int2(gi, m));
            const int stiles = (P->npair + kBatchThreads - 1) / kBatchThreads;
            for (int t = 0; t < stiles; ++t) {
                const int pairs = std::min(kBatchThreads, P->npair - t * kBatchThreads);
                for (int f0 = 0; f0 < nf; f0 += kBatchSynthNF) {
                    const int nv = std::min(kBatchSynthNF, nf - f0);
                    sc.push_back({(double)(lc - m + 1) * pairs * (4.0 + 2.0 * nv),
                                  make_int4(gi, m, t, f0)});
                }
            }
            for (int t = 0; t < g.tiles; ++t) {
                const int pairs = std::min(kBatchAnalPairs, P->npair - t * kBatchAnalPairs);
                for (int f0 = 0; f0 < nf; f0 += kBatchAnalNF) {
                    const int nv = std::min(kBatchAnalNF, nf - f0);
                    ac.push_back({(double)(lc - m + 1) * pairs * (2.0 + 2.5 * nv),
                                  make_int4(gi, m, t, f0)});
                }
            }
        }
        for (int f = 0; f < nf; ++f)
            for (int j = 0; j < g.fft_jobs; ++j) jobs[cls].push_back(make_int4(gi, f, j, 0));
    }
    // the spectra follow all packed-coefficient regions in the workspace
    for (BatchGroup& g : B->h_groups) g.spec_off += pack;
    auto by_cost = [](const Cost& a, const Cost& b) { return a.c > b.c; };
    std::stable_sort(sc.begin(), sc.end(), by_cost);
    std::stable_sort(ac.begin(), ac.end(), by_cost);
    std::vector<int4> si(sc.size()), ai(ac.size());
    for (size_t i = 0; i < sc.size(); ++i) si[i] = sc[i].it;
    for (size_t i = 0; i < ac.size(); ++i) ai[i] = ac[i].it;
    B->npitems = (int)pitems.size();
    B->nsitems = (int)si.size();
    B->naitems = (int)ai.size();
    for (int c = 0; c < NC; ++c) {
        B->njobs[c] = (int)jobs[c].size();
        B->fft_smem[c] = smem[c];
        B->fft_threads[c] = threads[c];
    }
    B->cilm_total = coff;
    B->grid_total = goff;
    B->work_bytes = (size_t)(pack + spec) * sizeof(double2);
    int rc = SHTC_OK;
    if (!rc) rc = upload(&B->d_groups, B->h_groups, st);
    if (!rc) rc = upload(&B->d_fft, fa, st);
    if (!rc) rc = upload(&B->d_pitems, pitems, st);
    if (!rc) rc = upload(&B->d_sitems, si, st);
    if (!rc) rc = upload(&B->d_aitems, ai, st);
    for (int c = 0; c < NC && !rc; ++c) rc = upload(&B->d_jobs[c], jobs[c], st);
    if (!rc && cudaMalloc((void**)&B->d_counter, (1 + NC) * sizeof(int)) != cudaSuccess)
        rc = SHTC_EALLOC;
    if (!rc) {
        int sm = 0, per = 0;
        cudaDeviceGetAttribute(&sm, cudaDevAttrMultiProcessorCount, B->device);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_synth, kBatchThreads, 0);
        B->synth_ctas = sm * std::max(1, per);
        const size_t asmem = anal_smem_bytes(kBatchAnalWarps, kBatchAnalNF);
        cudaFuncSetAttribute(k_batch_anal, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)asmem);
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, k_batch_anal,
                                                      32 * kBatchAnalWarps, asmem);
        B->anal_ctas = sm * std::max(1, per);
        for (int c = 0; c < NC; ++c)
            B->fft_ctas[c] = c < 2 ? fft_class_ctas(k_batch_c2r<8>, k_batch_r2c<8>, sm,
                                                    B->njobs[c], B->fft_threads[c],
                                                    B->fft_smem[c])
                                   : fft_class_ctas(k_batch_c2r<13>, k_batch_r2c<13>, sm,
                                                    B->njobs[c], B->fft_threads[c],
                                                    B->fft_smem[c]);
        rc = map_cuda(cudaStreamSynchronize(st));
    }
    if (rc) {
        batch_free(B);
        delete B;
        return rc;
    }
    *out = B;
    return SHTC_OK;
}

extern "C" SHTC_API int shtc_batch_destroy(shtc_batch* B) {
    if (!B) return SHTC_EHANDLE;
    batch_free(B);
    delete B;
    return SHTC_OK;
}

extern "C" SHTC_API size_t shtc_batch_workspace_bytes(const shtc_batch* B) {
    return B ? B->work_bytes : 0;
}

extern "C" SHTC_API int shtc_batch_layout(const shtc_batch* B, long long* cilm_off,
                                          long long* grid_off) {
    if (!B || !cilm_off || !grid_off) return SHTC_EHANDLE;
    for (int g = 0; g < B->ngroup; ++g) {
        cilm_off[g] = B->h_groups[g].cilm_off;
        grid_off[g] = B->h_groups[g].grid_off;
    }
    cilm_off[B->ngroup] = B->cilm_total;
    grid_off[B->ngroup] = B->grid_total;
    return SHTC_OK;
}

static int batch_check(const shtc_batch* B, const void* a, const void* b,
                       void* work, size_t wb) {
    if (!B || !a || !b) return SHTC_EHANDLE;
    if (!work || wb < B->work_bytes) return SHTC_EWORK;
    int dev = -1;
    cudaGetDevice(&dev);
    return dev == B->device ? SHTC_OK : SHTC_EHANDLE;
}

extern "C" SHTC_API int shtc_batch_synthesis(const shtc_batch* B, const double* cilm,
                                             double* grid, void* work, size_t wb,
                                             void* stream) {
    int rc = batch_check(B, cilm, grid, work, wb);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    double2* w = (double2*)work;
    stage_begin(SHTC_STAGE_PACK, st);
    k_batch_pack<<<B->npitems, 128, 0, st>>>(B->d_groups, B->d_pitems, cilm, w);
    stage_end(SHTC_STAGE_PACK, st);
    if ((rc = map_cuda(cudaGetLastError()))) return rc;
    if ((rc = map_cuda(cudaMemsetAsync(B->d_counter, 0, sizeof(int), st)))) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_SYNTH, st);
    k_batch_synth<<<B->synth_ctas, kBatchThreads, 0, st>>>(B->d_groups, B->d_sitems,
                                                           B->nsitems, B->d_counter, w);
    stage_end(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if ((rc = map_cuda(cudaGetLastError()))) return rc;
    stage_begin(SHTC_STAGE_FFT_C2R, st);
    if ((rc = map_cuda(cudaMemsetAsync(B->d_counter + 1, 0,
                                       shtc_batch::kClasses * sizeof(int), st))))
        return rc;
    for (int c = 0; c < shtc_batch::kClasses; ++c) {
        if (!B->njobs[c]) continue;
        if (c < 2)
            k_batch_c2r<8><<<B->fft_ctas[c], B->fft_threads[c], B->fft_smem[c], st>>>(
                B->d_groups, B->d_fft, B->d_jobs[c], B->njobs[c], B->d_counter + 1 + c, w,
                grid);
        else
            k_batch_c2r<13><<<B->fft_ctas[c], B->fft_threads[c], B->fft_smem[c], st>>>(
                B->d_groups, B->d_fft, B->d_jobs[c], B->njobs[c], B->d_counter + 1 + c, w,
                grid);
    }
    stage_end(SHTC_STAGE_FFT_C2R, st);
    return map_cuda(cudaGetLastError());
}

extern "C" SHTC_API int shtc_batch_analysis(const shtc_batch* B, const double* grid,
                                            double* cilm, void* work, size_t wb,
                                            void* stream) {
    int rc = batch_check(B, grid, cilm, work, wb);
    if (rc) return rc;
    cudaStream_t st = (cudaStream_t)stream;
    double2* w = (double2*)work;
    stage_begin(SHTC_STAGE_FFT_R2C, st);
    if ((rc = map_cuda(cudaMemsetAsync(B->d_counter + 1, 0,
                                       shtc_batch::kClasses * sizeof(int), st))))
        return rc;
    for (int c = 0; c < shtc_batch::kClasses; ++c) {
        if (!B->njobs[c]) continue;
        if (c < 2)
            k_batch_r2c<8><<<B->fft_ctas[c], B->fft_threads[c], B->fft_smem[c], st>>>(
                B->d_groups, B->d_fft, B->d_jobs[c], B->njobs[c], B->d_counter + 1 + c, grid,
                w);
        else
            k_batch_r2c<13><<<B->fft_ctas[c], B->fft_threads[c], B->fft_smem[c], st>>>(
                B->d_groups, B->d_fft, B->d_jobs[c], B->njobs[c], B->d_counter + 1 + c, grid,
                w);
    }
    stage_end(SHTC_STAGE_FFT_R2C, st);
    if ((rc = map_cuda(cudaGetLastError()))) return rc;
    if ((rc = map_cuda(cudaMemsetAsync(B->d_counter, 0, sizeof(int), st)))) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_ANAL, st);
    k_batch_anal<<<B->anal_ctas, 32 * kBatchAnalWarps, anal_smem_bytes(kBatchAnalWarps, kBatchAnalNF),
                   st>>>(B->d_groups, B->d_aitems, B->naitems, B->d_counter, w);
    stage_end(SHTC_STAGE_LEGENDRE_ANAL, st);
    if ((rc = map_cuda(cudaGetLastError()))) return rc;
    if ((rc = map_cuda(cudaMemsetAsync(cilm, 0, sizeof(double) * B->cilm_total, st))))
        return rc;
    stage_begin(SHTC_STAGE_UNPACK, st);
    k_batch_unpack<<<B->npitems, 128, 0, st>>>(B->d_groups, B->d_pitems, w, cilm);
    stage_end(SHTC_STAGE_UNPACK, st);
    return map_cuda(cudaGetLastError());
}
