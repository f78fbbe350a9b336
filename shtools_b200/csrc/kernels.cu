// FP64 transform kernels of libshtcuda (sm_100a).
//
// Synthesis (MakeGridDH / MakeGridGLQ):
//   k_pack_coef       cilm (any strides)          -> packed {C, S} per (l, m)
//   k_legendre_synth  packed coefficients          -> spec[pair][m][ring]
//   k_fft_c2r         spec                         -> grid rows (+extend column)
// Analysis (SHExpandDH / SHExpandGLQ):
//   k_fft_r2c         grid rows                    -> weighted spec
//   k_legendre_anal   spec                         -> packed {C, S} partial sums
//   k_unpack_coef     packed partial sums          -> cilm, normalised
// The adjoints used by autograd run the same kernels in transposed order
// with different ring weights and coefficient scalings (see api.cu).
//
// The Legendre stages themselves live in legendre.cuh (shared with the
// persistent batched kernels of batch.cu).  Where the reference loops over
// latitude and then m, one CTA here owns one order m for a tile of ring
// pairs and each thread owns T ring pairs; the (l, m) tables and
// coefficients are read once per CTA and broadcast to all rings.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <map>
#include <mutex>
#include <tuple>
#include <utility>

#include "fft.cuh"
#include "legendre.cuh"
#include "shtc_internal.cuh"

namespace shtc {

int map_cuda(cudaError_t e) { return e == cudaSuccess ? SHTC_OK : SHTC_ECUDA; }

// ---------------------------------------------------------------------------
// coefficient packing
// ---------------------------------------------------------------------------
// scale_mode 0: copy; 1: multiply by the analysis normalisation factor
// (the adjoint of the final divide of SHExpandDH.f95:674-702); 0 and 1 also
// multiply by the recursion's D(l - m); 2 and 3 are 0 and 1 without it (the
// INT8 tensor-core synthesis).
__device__ __forceinline__ double anal_norm_factor(int norm, int l,
                                                   const double* nrm3,
                                                   long long idx) {
    const double pi = 3.141592653589793238462643383279502884;
    switch (norm) {
        case 1: return 1.0 / (4 * pi);
        case 2: return (double)(2 * l + 1) / (4 * pi);
        case 3: return 1.0 / nrm3[idx];
        default: return 1.0;
    }
}

// (l, m) tiles of kCoefTile x kCoefTile staged in shared memory: the
// coefficient arrays (C order, contiguous along m) and the packed arrays
// (contiguous along l for one m) are then both accessed along their fast
// dimension.
constexpr int kCoefTile = 32;
constexpr int kCoefRows = 8;   // blockDim = (kCoefTile, kCoefRows)

template <typename CT>
__global__ void __launch_bounds__(kCoefTile * kCoefRows)
k_pack_coef(const CT* __restrict__ cilm, long long sf, long long sk, long long sl,
            long long sm, int cdim, double2* __restrict__ packed, int lc, int nfield,
            int norm, const double* __restrict__ nrm3, int scale_mode,
            const double2* __restrict__ rec, int f_off) {
    __shared__ double2 tile[kCoefTile][kCoefTile + 1];   // [m - m0][l - l0]
    // the fields of one tile are adjacent blocks: their 16-byte entries of
    // the field-interleaved packed array share sectors, which L2 then
    // writes to DRAM whole
    const int f = blockIdx.x;
    const int l0 = blockIdx.y * kCoefTile, m0 = blockIdx.z * kCoefTile;
    if (m0 > l0 + kCoefTile - 1) return;   // tile above the diagonal (uniform)
    const int tx = threadIdx.x;
    for (int j = threadIdx.y; j < kCoefTile; j += kCoefRows) {
        const int l = l0 + j, m = m0 + tx;
        double c = 0.0, s = 0.0;
        if (m <= l && l <= lc && l < cdim) {
            const CT* b = cilm + f * sf + l * sl + m * sm;
            c = (double)b[0];
            s = (m == 0) ? 0.0 : (double)b[sk];
        }
        tile[tx][j] = make_double2(c, s);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kCoefTile; j += kCoefRows) {
        const int m = m0 + j, l = l0 + tx;
        if (m > l || l > lc) continue;
        const long long idx = packed_off(m, lc) + (l - m);
        double2 v = tile[j][tx];
        if (scale_mode == 1 || scale_mode == 3) {
            const double a = anal_norm_factor(norm, l, nrm3, idx);
            v.x *= a;
            v.y *= a;
        }
        // D(l - m) of the rescaled recursion (legendre.cuh); scale_modes 2
        // and 3 keep the plain coefficients (the INT8 tensor-core synthesis)
        const double d = scale_mode >= 2 ? 1.0 : rec[idx].y;
        packed[idx * nfield + f_off + f] = make_double2(v.x * d, v.y * d);
    }
}

// ---------------------------------------------------------------------------
// Legendre synthesis
// ---------------------------------------------------------------------------
// spec[((f*npair + p)*(lc+1) + m)*2 + h], h = 0 north ring, 1 south ring,
// holds the c2r input of the ring: (a_m - i b_m) * (m ? 1/2 : 1) with
// a_m = sum_l C_lm P_lm, b_m = sum_l S_lm P_lm (MakeGridDH.f95:566-612).
// ---------------------------------------------------------------------------
// per-plan Legendre kernels: one CTA per (ring-pair tile, order m, field
// group); the grid runs m = 0, 1, ... so the longest recursions start first
// and the hardware scheduler balances the triangular work
// ---------------------------------------------------------------------------
template <int T, int NF>
__global__ void __launch_bounds__(128)
k_legendre_synth(const double2* __restrict__ rec, const double* __restrict__ pmm,
                 const double* __restrict__ rtab, const double* __restrict__ zp,
                 const double2* __restrict__ coef, double2* __restrict__ spec,
                 int lc, int npair, int nfield) {
    __shared__ __align__(16) SynthStage<NF> sm;
    synth_order<T, NF>(sm, rec, pmm, rtab, zp, coef, spec, lc, npair, nfield,
                       blockIdx.y, blockIdx.x, blockIdx.z * NF, NF);
}

// The same kernels with the registers capped for more resident warps: the
// T = 8 single-field synthesis at 3 CTAs per SM (<= 168 registers) and the
// T = 8 analysis at 2 x 256 threads (<= 128), measured on B200 at lmax 2047
// 2% and 5% faster than the uncapped builds (other shapes are not capped:
// they were slower or unchanged).
template <int T, int NF>
__global__ void __launch_bounds__(128, 3)
k_legendre_synth_capped(const double2* __restrict__ rec, const double* __restrict__ pmm,
                 const double* __restrict__ rtab, const double* __restrict__ zp,
                 const double2* __restrict__ coef, double2* __restrict__ spec,
                 int lc, int npair, int nfield) {
    __shared__ __align__(16) SynthStage<NF> sm;
    synth_order<T, NF>(sm, rec, pmm, rtab, zp, coef, spec, lc, npair, nfield,
                       blockIdx.y, blockIdx.x, blockIdx.z * NF, NF);
}

template <int T, int NF>
__global__ void __launch_bounds__(256)
k_legendre_anal(const double2* __restrict__ rec, const double* __restrict__ pmm,
                const double* __restrict__ rtab, const double* __restrict__ zp,
                const double2* __restrict__ spec, double2* __restrict__ partial,
                int lc, int npair, long long nlm, int nfield) {
    extern __shared__ __align__(16) double smem_anal[];
    __shared__ __align__(16) double2 rstage[2][kAnalStage];
    const int f0 = blockIdx.z * NF;
    const long long sstride = (long long)npair * (lc + 1) * 2;
    anal_order<T, NF>(smem_anal, rstage, rec, pmm, rtab, zp, spec + f0 * sstride, sstride,
                      partial + ((long long)blockIdx.x * nfield + f0) * nlm, nlm, lc, npair,
                      blockIdx.y, blockIdx.x, min(NF, nfield - f0));
}

template <int T, int NF>
__global__ void __launch_bounds__(256, 2)
k_legendre_anal_capped(const double2* __restrict__ rec, const double* __restrict__ pmm,
                const double* __restrict__ rtab, const double* __restrict__ zp,
                const double2* __restrict__ spec, double2* __restrict__ partial,
                int lc, int npair, long long nlm, int nfield) {
    extern __shared__ __align__(16) double smem_anal[];
    __shared__ __align__(16) double2 rstage[2][kAnalStage];
    const int f0 = blockIdx.z * NF;
    const long long sstride = (long long)npair * (lc + 1) * 2;
    anal_order<T, NF>(smem_anal, rstage, rec, pmm, rtab, zp, spec + f0 * sstride, sstride,
                      partial + ((long long)blockIdx.x * nfield + f0) * nlm, nlm, lc, npair,
                      blockIdx.y, blockIdx.x, min(NF, nfield - f0));
}

// ---------------------------------------------------------------------------
// coefficient unpacking + analysis normalisation
// ---------------------------------------------------------------------------
// normalise 1: divide by the integral of Ylm^2 exactly as the reference
// (SHExpandDH.f95:674-702); 0: no normalisation (synthesis adjoint).
template <typename CT>
__global__ void __launch_bounds__(kCoefTile * kCoefRows)
k_unpack_coef(const double2* __restrict__ partial, int ntiles, CT* __restrict__ cilm,
              long long sf, long long sk, long long sl, long long sm, int cdim, int lc,
              long long nlm, int nfield, int norm, const double* __restrict__ nrm3,
              int normalise) {
    const double pi = 3.141592653589793238462643383279502884;
    __shared__ double2 tile[kCoefTile][kCoefTile + 1];   // [m - m0][l - l0]
    const int l0 = blockIdx.x * kCoefTile, m0 = blockIdx.y * kCoefTile;
    const int f = blockIdx.z;
    const int tx = threadIdx.x;
    for (int j = threadIdx.y; j < kCoefTile; j += kCoefRows) {
        const int m = m0 + j, l = l0 + tx;
        double c = 0.0, s = 0.0;
        if (m <= l && l <= lc && l < cdim) {
            const long long idx = packed_off(m, lc) + (l - m);
            for (int t = 0; t < ntiles; ++t) {
                const double2 v = partial[((long long)t * nfield + f) * nlm + idx];
                c += v.x;
                s += v.y;
            }
            if (normalise) {
                switch (norm) {
                    case 1:
                        c = c / (4 * pi);
                        s = s / (4 * pi);
                        break;
                    case 2:
                        c = c * (2 * l + 1) / (4 * pi);
                        s = s * (2 * l + 1) / (4 * pi);
                        break;
                    case 3:
                        c = c / nrm3[idx];
                        s = s / nrm3[idx];
                        break;
                    default:
                        break;
                }
            }
            if (m == 0) s = 0.0;
        }
        tile[j][tx] = make_double2(c, s);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kCoefTile; j += kCoefRows) {
        const int l = l0 + j, m = m0 + tx;
        if (l >= cdim || m >= cdim) continue;
        const double2 v = tile[tx][j];
        CT* b = cilm + f * sf + l * sl + m * sm;
        b[0] = (CT)v.x;
        b[sk] = (CT)v.y;
    }
}

// ---------------------------------------------------------------------------
// per-plan FFT kernels: CTA = (job, field); job = ring pair (odd n) or
// 2*pair + ring (even n)
// ---------------------------------------------------------------------------
// Persistent FFT kernels: CTA b handles the items b, b + gridDim.x, ... of
// the nitems = jobs * nfield (job, field) pairs; while one item's FFT runs,
// the next item's input lines are prefetched into L2.  With tw_smem the
// plan's twiddles are copied once per CTA behind the two data buffers.
__device__ __forceinline__ const double2* fft_stage_twiddles(const FftArgs& F,
                                                             double2* smem_fft,
                                                             int tw_smem) {
    if (!tw_smem) return F.tw;
    const int len = F.bluestein ? F.mb : F.m;
    // behind the two data buffers, or at the start when those are global
    double2* tws = F.gmem ? smem_fft : smem_fft + 2 * len;
    for (int i = threadIdx.x; i < F.ntw; i += blockDim.x) tws[i] = F.tw[i];
    return tws;   // made visible by the barrier that opens fft_exec
}

// the CTA's two data buffers: shared memory, or its slice of the global
// scratch (F.gmem); __syncthreads orders the passes in either
__device__ __forceinline__ double2* fft_buffers(const FftArgs& F, double2* smem_fft,
                                                double2* gbuf) {
    if (!F.gmem) return smem_fft;
    const int len = F.bluestein ? F.mb : F.m;
    return gbuf + (size_t)blockIdx.x * 2 * len;
}

// MAXR = 8: plans whose radices are all <= 8, built for <= 64 registers
// (four 256-thread CTAs per SM); MAXR = 10 the same with the radix-10 pass,
// in one 1024-thread CTA for rings too long for two CTAs' shared memory
// (MAXT = 1024); MAXR = 13 carries the radix-11/13 passes
template <int MAXR, int MAXT>
constexpr int fft_min_ctas() { return MAXR <= 10 ? 65536 / (64 * MAXT) : 1; }

template <typename GT, int MAXR, int MAXT = 512>
__global__ void __launch_bounds__(MAXT, fft_min_ctas<MAXR, MAXT>())
k_fft_c2r(FftArgs F, int tw_smem, int jobs, int nitems, const double2* __restrict__ spec,
          GT* __restrict__ grid, long long gf, long long grs, long long gcs,
          const int* __restrict__ rowN, const int* __restrict__ rowS,
          const double* __restrict__ wN, const double* __restrict__ wS, double wscale,
          int lc, int npair, int extend_col, double2* __restrict__ gbuf) {
    extern __shared__ double2 smem_fft[];
    const double2* tw = fft_stage_twiddles(F, smem_fft, tw_smem);
    double2* bufs = fft_buffers(F, smem_fft, gbuf);
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int nx = it + gridDim.x;
        if (nx < nitems) fft_c2r_prefetch(F.mode, nx % jobs, nx / jobs, spec, lc, npair);
        fft_c2r_body<GT, MAXR>(F, tw, bufs, it % jobs, it / jobs, spec, grid, gf, grs, gcs,
                         rowN, rowS, wN, wS, wscale, lc, npair, extend_col);
        __syncthreads();
    }
}

template <typename GT, int MAXR, int MAXT = 512>
__global__ void __launch_bounds__(MAXT, fft_min_ctas<MAXR, MAXT>())
k_fft_r2c(FftArgs F, int tw_smem, int jobs, int nitems, const GT* __restrict__ grid,
          long long gf, long long grs, long long gcs, double2* __restrict__ spec,
          const int* __restrict__ rowN, const int* __restrict__ rowS,
          const double* __restrict__ wN, const double* __restrict__ wS, double wscale,
          int lc, int npair, int fold_extend, const GT* __restrict__ grid2, double2* __restrict__ gbuf) {
    extern __shared__ double2 smem_fft[];
    const double2* tw = fft_stage_twiddles(F, smem_fft, tw_smem);
    double2* bufs = fft_buffers(F, smem_fft, gbuf);
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        const int nx = it + gridDim.x;
        if (nx < nitems)
            fft_r2c_prefetch<GT>(F.mode, F.n, nx % jobs, nx / jobs, grid, gf, grs, gcs, rowN,
                                 rowS, fold_extend);
        fft_r2c_body<GT, MAXR>(F, tw, bufs, it % jobs, it / jobs, grid, gf, grs, gcs, spec,
                         rowN, rowS, wN, wS, wscale, lc, npair, fold_extend, grid2);
        __syncthreads();
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
// Host-side launch configuration, cached: a kernel's shared-memory
// attributes are set once per device (again only for a larger size), and
// its resident CTAs per device once per (device, kernel, CTA shape), so a
// transform issues no attribute or occupancy calls after its first run.
namespace {
std::mutex g_launch_mu;
std::map<std::pair<int, const void*>, size_t> g_smem_set;
std::map<std::tuple<int, const void*, int, size_t>, int> g_resident;
}  // namespace

// the dynamic shared memory limit of kernel fn raised to smem; with
// max_shared the largest carveout is preferred (kernels that live on shared
// memory, so that registers, not the L1 split, limit the resident CTAs)
int kernel_smem_attr(const void* fn, size_t smem, bool max_shared) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return map_cuda(e);
    std::lock_guard<std::mutex> g(g_launch_mu);
    const auto key = std::make_pair(dev, fn);
    auto it = g_smem_set.find(key);
    if (it != g_smem_set.end() && it->second >= smem) return SHTC_OK;
    e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess && max_shared)
        e = cudaFuncSetAttribute(fn, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return map_cuda(e);
    g_smem_set[key] = smem;
    return SHTC_OK;
}

FftArgs fft_args(const FftPlan& f) {
    FftArgs a;
    a.n = f.n; a.mode = f.mode; a.m = f.m; a.nfac = f.nfac;
    a.bluestein = f.bluestein; a.mb = f.mb; a.ntw = f.ntw; a.gmem = f.gmem;
    for (int i = 0; i < kMaxFactors; ++i) {
        a.fac[i] = i < f.nfac ? f.fac[i] : 0;
        a.tw_off[i] = i < f.nfac ? f.tw_off[i] : 0;
    }
    a.tw = f.d_tw; a.twn = f.d_twn; a.chirp = f.d_chirp; a.kern = f.d_kern;
    return a;
}

int launch_pack_coef(const shtc_plan* P, const void* cilm, int dtype, long long sf,
                     long long sk, long long sl, long long sm, int cdim,
                     double2* packed, int nfield, int scale_mode,
                     cudaStream_t st, int nfield_total, int f_off) {
    // fields f_off .. f_off+nfield-1 of a packed array of nfield_total fields
    // (nfield_total = 0: nfield, f_off = 0)
    const int ntot = nfield_total > 0 ? nfield_total : nfield;
    const int lc = P->lc;
    const int nt = (lc + kCoefTile) / kCoefTile;
    const dim3 grid(nfield, nt, nt), block(kCoefTile, kCoefRows);
    if (dtype == SHTC_F32)
        k_pack_coef<float><<<grid, block, 0, st>>>((const float*)cilm, sf, sk, sl, sm, cdim,
                                                 packed, lc, ntot, P->norm, P->d_nrm,
                                                 scale_mode, P->d_rec, f_off);
    else
        k_pack_coef<double><<<grid, block, 0, st>>>((const double*)cilm, sf, sk, sl, sm, cdim,
                                                  packed, lc, ntot, P->norm, P->d_nrm,
                                                  scale_mode, P->d_rec, f_off);
    return map_cuda(cudaGetLastError());
}

template <int T, int NF>
static void launch_synth_t(const shtc_plan* P, const double2* packed,
                           double2* spec, int nfield, cudaStream_t st) {
    const int threads = 128;
    const int tiles = (P->npair + threads * T - 1) / (threads * T);
    dim3 grid(tiles, P->lc + 1, nfield / NF);
    if constexpr (T == 8 && NF == 1)
        k_legendre_synth_capped<T, NF><<<grid, threads, 0, st>>>(
            P->d_rec, P->d_pmm, P->d_rtab, P->d_z, packed, spec, P->lc, P->npair, nfield);
    else
        k_legendre_synth<T, NF><<<grid, threads, 0, st>>>(
            P->d_rec, P->d_pmm, P->d_rtab, P->d_z, packed, spec, P->lc, P->npair, nfield);
}

int launch_legendre_synth(const shtc_plan* P, const double2* packed,
                          double2* spec, int nfield, cudaStream_t st) {
    const int np = P->npair;
    if (nfield % 8 == 0) {
        // one recursion per 8 fields; T = 1 keeps the 8 x 4 accumulators in
        // registers
        if (np > 512) launch_synth_t<2, 8>(P, packed, spec, nfield, st);
        else launch_synth_t<1, 8>(P, packed, spec, nfield, st);
    } else if (nfield % 4 == 0) {
        launch_synth_t<2, 4>(P, packed, spec, nfield, st);
    } else if (nfield % 2 == 0 && nfield >= 2) {
        if (np > 512) launch_synth_t<4, 2>(P, packed, spec, nfield, st);
        else launch_synth_t<2, 2>(P, packed, spec, nfield, st);
    } else if (nfield % 3 == 0) {
        // the three sums of a MakeGradientDH field share one recursion
        if (np > 512) launch_synth_t<2, 3>(P, packed, spec, nfield, st);
        else launch_synth_t<1, 3>(P, packed, spec, nfield, st);
    } else {
        // heuristic from the autotuner's sweeps on B200 (lmax 63..2799)
        int T = P->tune_synth_T;
        if (T == 0) T = np > 768 ? 8 : (np > 256 ? 2 : 1);
        switch (T) {
            case 8: launch_synth_t<8, 1>(P, packed, spec, nfield, st); break;
            case 4: launch_synth_t<4, 1>(P, packed, spec, nfield, st); break;
            case 2: launch_synth_t<2, 1>(P, packed, spec, nfield, st); break;
            default: launch_synth_t<1, 1>(P, packed, spec, nfield, st); break;
        }
    }
    return map_cuda(cudaGetLastError());
}

// The tensor-path analysis (legendre_mma.cu) takes 8 or more fields on grids
// with at least one full tile of ring pairs
static bool anal_use_mma(const shtc_plan* P, int nfield) {
    return nfield >= 8 && P->npair >= anal_mma_pairs();
}

// analysis CTA shape for nfield (internal) fields: T pairs per thread, W warps
static void anal_shape(const shtc_plan* P, int nfield, int* T, int* W, int* tiles) {
    const int np = P->npair;
    if (anal_use_mma(P, nfield)) {
        *T = 1;
        *W = anal_mma_pairs() / 32;
        *tiles = (np + anal_mma_pairs() - 1) / anal_mma_pairs();
        return;
    }
    int w = P->tune_anal_W ? P->tune_anal_W : 2;
    int t = P->tune_anal_T;
    if (t == 0) {
        // largest T (at most 4) that leaves at least two CTA tiles of ring
        // pairs: what the autotuner's sweeps on B200 select for lmax 63..2799
        t = 1;
        while (t < 4 && 32 * w * (2 * t) <= np / 2) t *= 2;
    }
    if (nfield > 1 && t == 8) {
        // T = 8 runs each field alone (T*NF <= 8); with several fields T = 4
        // and 2 warps, two fields per recursion, is faster on B200 (16 DH
        // fields at lmax 2799: 57.0 ms against 67.4 ms; 2 and 4 GLQ fields
        // at lmax 2047 within 2% of the best shape)
        t = 4;
        w = 2;
    }
    *T = t;
    *W = w;
    *tiles = (np + 32 * t * w - 1) / (32 * t * w);
}

int anal_tiles(const shtc_plan* P, int nfield) {
    int T, W, tiles;
    anal_shape(P, nfield, &T, &W, &tiles);
    return tiles;
}

template <int T, int NF>
static int launch_anal_t(const shtc_plan* P, const double2* spec,
                         double2* partial, int nfield, int W, int tiles,
                         cudaStream_t st) {
    const int threads = 32 * W;
    const size_t smem = anal_smem_bytes(W, NF);
    void (*kern)(const double2*, const double*, const double*, const double*,
                 const double2*, double2*, int, int, long long, int);
    if constexpr (T == 8) kern = k_legendre_anal_capped<T, NF>;
    else kern = k_legendre_anal<T, NF>;
    const int rc = kernel_smem_attr((const void*)kern, smem, false);
    if (rc) return rc;
    dim3 grid(tiles, P->lc + 1, (nfield + NF - 1) / NF);
    kern<<<grid, threads, smem, st>>>(
        P->d_rec, P->d_pmm, P->d_rtab, P->d_z, spec, partial, P->lc, P->npair,
        P->nlm, nfield);
    return map_cuda(cudaGetLastError());
}

// Fields share the recursion in groups of NF.  The group's G values take
// 4*T*NF registers, so NF is chosen to keep T*NF <= 8 (about 128 registers):
// NF = 4 for T <= 2, 2 for T = 4, 1 for T = 8.
template <int T>
static int launch_anal_nf(const shtc_plan* P, const double2* spec, double2* partial,
                          int nfield, int W, int tiles, cudaStream_t st) {
    if constexpr (T <= 2) {
        if (nfield % 4 == 0) return launch_anal_t<T, 4>(P, spec, partial, nfield, W, tiles, st);
    }
    if constexpr (T <= 4) {
        if (nfield % 2 == 0) return launch_anal_t<T, 2>(P, spec, partial, nfield, W, tiles, st);
    }
    return launch_anal_t<T, 1>(P, spec, partial, nfield, W, tiles, st);
}

int launch_legendre_anal(const shtc_plan* P, const double2* spec,
                         double2* partial, int ntiles_out, int nfield,
                         cudaStream_t st) {
    int T, W, tiles;
    anal_shape(P, nfield, &T, &W, &tiles);
    if (tiles != ntiles_out) return SHTC_EBOUND;
    if (anal_use_mma(P, nfield))
        return launch_legendre_anal_mma(P, spec, partial, tiles, nfield, st);
    switch (T) {
        case 8: return launch_anal_nf<8>(P, spec, partial, nfield, W, tiles, st);
        case 4: return launch_anal_nf<4>(P, spec, partial, nfield, W, tiles, st);
        case 2: return launch_anal_nf<2>(P, spec, partial, nfield, W, tiles, st);
        default: return launch_anal_nf<1>(P, spec, partial, nfield, W, tiles, st);
    }
}

int launch_unpack_coef(const shtc_plan* P, const double2* partial, int ntiles,
                       void* cilm, int dtype, long long sf, long long sk, long long sl,
                       long long sm, int cdim, int nfield, int normalise,
                       cudaStream_t st) {
    const int lc = P->lc;
    const int nt = (cdim + kCoefTile - 1) / kCoefTile;
    const dim3 grid(nt, nt, nfield), block(kCoefTile, kCoefRows);
    if (dtype == SHTC_F32)
        k_unpack_coef<float><<<grid, block, 0, st>>>(partial, ntiles, (float*)cilm, sf, sk,
                                                   sl, sm, cdim, lc, P->nlm, nfield,
                                                   P->norm, P->d_nrm, normalise);
    else
        k_unpack_coef<double><<<grid, block, 0, st>>>(partial, ntiles, (double*)cilm, sf, sk,
                                                    sl, sm, cdim, lc, P->nlm, nfield,
                                                    P->norm, P->d_nrm, normalise);
    return map_cuda(cudaGetLastError());
}

// Which FFT build runs a plan: 0 the full one (the plan's CTA size); 1 the
// register-capped one (radices <= 8, every Bluestein length among them)
// when shared memory leaves room for more than one CTA per SM; 2 the
// register-capped one in 1024-thread CTAs, with the radix-10 pass, for
// rings of more than 4096 points held in shared memory (one CTA per SM
// either way, but twice the warps; with 512 threads the cap alone cost 2-3%
// at lmax 2799)
static int fft_variant(const FftPlan& f) {
    int maxr = 0;
    for (int i = 0; i < f.nfac; ++i) maxr = std::max(maxr, f.fac[i]);
    const int len = f.bluestein ? f.mb : f.m;
    const bool long_ring = !f.gmem && len > 4096;
    if (maxr > 10) return 0;
    if (maxr == 10) return long_ring ? 2 : 0;
    if (f.smem <= 100 * 1024) return 1;
    return long_ring ? 2 : 0;
}

// the plan's FFT arguments with the CTA size of the build that runs them
template <int MAXT>
static FftPlan fft_shape(const FftPlan& f) {
    FftPlan g = f;
    if (MAXT > 512) g.threads = MAXT;
    return g;
}

// persistent grid of an FFT kernel: as many CTAs as fit on the device at
// once, at most one per item (and one per global-scratch slice)
static int fft_launch_setup(const void* fn, const FftPlan& f, int nitems, int* blocks) {
    int rc = kernel_smem_attr(fn, f.smem, true);
    if (rc) return rc;
    int dev = 0;
    cudaGetDevice(&dev);
    long long cap;
    {
        std::lock_guard<std::mutex> g(g_launch_mu);
        const auto key = std::make_tuple(dev, fn, f.threads, f.smem);
        auto it = g_resident.find(key);
        if (it != g_resident.end()) {
            cap = it->second;
        } else {
            int sms = 0, occ = 0;
            cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
            cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, fn, f.threads,
                                                                          f.smem);
            if (e != cudaSuccess) return map_cuda(e);
            cap = (long long)(sms > 0 ? sms : 1) * (occ > 0 ? occ : 1);
            g_resident[key] = (int)cap;
        }
    }
    if (f.gmem && cap > f.gmem_ctas) cap = f.gmem_ctas;   // one scratch slice per CTA
    *blocks = (int)(nitems < cap ? nitems : cap);
    return SHTC_OK;
}

size_t fft_scratch_bytes(const shtc_plan* P) {
    const FftPlan& f = P->fft;
    if (!f.gmem) return 0;
    const size_t len = (size_t)(f.bluestein ? f.mb : f.m);
    return (size_t)f.gmem_ctas * 2 * len * sizeof(double2);
}

template <typename GT, int MAXR, int MAXT = 512>
static int launch_c2r_t(const shtc_plan* P, const double2* spec, GT* grid, long long gf,
                        long long grs, long long gcs, int nfield, int weighted,
                        cudaStream_t st, double2* gbuf) {
    const FftPlan f = fft_shape<MAXT>(P->fft);
    if (f.gmem && !gbuf) return SHTC_EWORK;
    int rc;
    const int jobs = f.mode == 0 ? P->npair : 2 * P->npair;
    const int nitems = jobs * nfield;
    int blocks = 0;
    if ((rc = fft_launch_setup((const void*)k_fft_c2r<GT, MAXR, MAXT>, f, nitems, &blocks))) return rc;
    if (blocks == 0) return SHTC_OK;
    // synthesis uses the synthesis ring map (with the extend row and column);
    // the analysis adjoint uses the analysis ring map and ring weights
    if (weighted) {
        k_fft_c2r<GT, MAXR, MAXT><<<blocks, f.threads, f.smem, st>>>(
            fft_args(f), f.tw_smem, jobs, nitems, spec, grid, gf, grs, gcs, P->d_arowN,
            P->d_arowS, P->d_wN, P->d_wS, 1.0 / (double)P->nlon, P->lc, P->npair, 0, gbuf);
    } else {
        k_fft_c2r<GT, MAXR, MAXT><<<blocks, f.threads, f.smem, st>>>(
            fft_args(f), f.tw_smem, jobs, nitems, spec, grid, gf, grs, gcs, P->d_rowN,
            P->d_rowS, nullptr, nullptr, 1.0, P->lc, P->npair, P->extend, gbuf);
    }
    return map_cuda(cudaGetLastError());
}

int launch_fft_c2r(const shtc_plan* P, const double2* spec, void* grid, int dtype,
                   long long gf, long long grs, long long gcs, int nfield,
                   int weighted, cudaStream_t st, double2* gbuf) {
    const int v = fft_variant(P->fft);
    if (v == 1)
        return dtype == SHTC_F32
                   ? launch_c2r_t<float, 8>(P, spec, (float*)grid, gf, grs, gcs, nfield,
                                            weighted, st, gbuf)
                   : launch_c2r_t<double, 8>(P, spec, (double*)grid, gf, grs, gcs, nfield,
                                             weighted, st, gbuf);
    if (v == 2)
        return dtype == SHTC_F32
                   ? launch_c2r_t<float, 10, 1024>(P, spec, (float*)grid, gf, grs, gcs, nfield,
                                                  weighted, st, gbuf)
                   : launch_c2r_t<double, 10, 1024>(P, spec, (double*)grid, gf, grs, gcs,
                                                   nfield, weighted, st, gbuf);
    return dtype == SHTC_F32
               ? launch_c2r_t<float, 13>(P, spec, (float*)grid, gf, grs, gcs, nfield, weighted,
                                         st, gbuf)
               : launch_c2r_t<double, 13>(P, spec, (double*)grid, gf, grs, gcs, nfield,
                                          weighted, st, gbuf);
}

template <typename GT, int MAXR, int MAXT = 512>
static int launch_r2c_t(const shtc_plan* P, const GT* grid, long long gf, long long grs,
                        long long gcs, double2* spec, int nfield, int weighted,
                        int fold_extend, cudaStream_t st, const GT* grid2, double2* gbuf) {
    const FftPlan f = fft_shape<MAXT>(P->fft);
    if (f.gmem && !gbuf) return SHTC_EWORK;
    int rc;
    const int jobs = f.mode == 0 ? P->npair : 2 * P->npair;
    const int nitems = jobs * nfield;
    int blocks = 0;
    if ((rc = fft_launch_setup((const void*)k_fft_r2c<GT, MAXR, MAXT>, f, nitems, &blocks))) return rc;
    if (blocks == 0) return SHTC_OK;
    if (weighted) {
        // analysis: fcoef = (w * Re) / nlong, the reference's order of operations
        // is reproduced up to one rounding by folding 1/nlong into the weight
        k_fft_r2c<GT, MAXR, MAXT><<<blocks, f.threads, f.smem, st>>>(
            fft_args(f), f.tw_smem, jobs, nitems, grid, gf, grs, gcs, spec, P->d_arowN,
            P->d_arowS, P->d_wN, P->d_wS, 1.0 / (double)P->nlon, P->lc, P->npair, 0,
            grid2, gbuf);
    } else {
        // synthesis adjoint: plain (Re, -Im) of the rows of the cotangent
        k_fft_r2c<GT, MAXR, MAXT><<<blocks, f.threads, f.smem, st>>>(
            fft_args(f), f.tw_smem, jobs, nitems, grid, gf, grs, gcs, spec, P->d_rowN,
            P->d_rowS, nullptr, nullptr, 1.0, P->lc, P->npair, fold_extend, grid2, gbuf);
    }
    return map_cuda(cudaGetLastError());
}

// analysis r2c of the pointwise products grid * grid2 (float64 grids)
int launch_fft_r2c_product(const shtc_plan* P, const double* grid, const double* grid2,
                           long long gf, long long grs, long long gcs, double2* spec,
                           int nfield, cudaStream_t st, double2* gbuf) {
    switch (fft_variant(P->fft)) {
        case 1:
            return launch_r2c_t<double, 8>(P, grid, gf, grs, gcs, spec, nfield, 1, 0, st,
                                           grid2, gbuf);
        case 2:
            return launch_r2c_t<double, 10, 1024>(P, grid, gf, grs, gcs, spec, nfield, 1, 0, st,
                                                 grid2, gbuf);
        default:
            return launch_r2c_t<double, 13>(P, grid, gf, grs, gcs, spec, nfield, 1, 0, st,
                                            grid2, gbuf);
    }
}

int launch_fft_r2c(const shtc_plan* P, const void* grid, int dtype, long long gf,
                   long long grs, long long gcs, double2* spec, int nfield,
                   int weighted, int fold_extend, cudaStream_t st, double2* gbuf) {
    const int v = fft_variant(P->fft);
    if (v == 1)
        return dtype == SHTC_F32
                   ? launch_r2c_t<float, 8>(P, (const float*)grid, gf, grs, gcs, spec, nfield,
                                            weighted, fold_extend, st, nullptr, gbuf)
                   : launch_r2c_t<double, 8>(P, (const double*)grid, gf, grs, gcs, spec,
                                             nfield, weighted, fold_extend, st, nullptr, gbuf);
    if (v == 2)
        return dtype == SHTC_F32
                   ? launch_r2c_t<float, 10, 1024>(P, (const float*)grid, gf, grs, gcs, spec,
                                                  nfield, weighted, fold_extend, st, nullptr,
                                                  gbuf)
                   : launch_r2c_t<double, 10, 1024>(P, (const double*)grid, gf, grs, gcs, spec,
                                                   nfield, weighted, fold_extend, st, nullptr,
                                                   gbuf);
    return dtype == SHTC_F32
               ? launch_r2c_t<float, 13>(P, (const float*)grid, gf, grs, gcs, spec, nfield,
                                         weighted, fold_extend, st, nullptr, gbuf)
               : launch_r2c_t<double, 13>(P, (const double*)grid, gf, grs, gcs, spec, nfield,
                                          weighted, fold_extend, st, nullptr, gbuf);
}

// ---------------------------------------------------------------------------
// complex transforms (MakeGridDHC / SHExpandDHC, MakeGridGLQC / SHExpandGLQC)
// ---------------------------------------------------------------------------
// pack: complex cilm[u][k][l][m] (k = 0 the order +m, 1 the order -m) ->
// packed [(l, m)][2u + k] = (Re, Im) * D(l - m); the -0 entry is ignored as in
// the reference.  Same 32x32 shared-memory tiles as k_pack_coef; grid.z =
// 2 * fields.
__global__ void __launch_bounds__(kCoefTile * kCoefRows)
k_pack_coef_c(const double2* __restrict__ cilm, long long sf, long long sk, long long sl,
              long long sm, int cdim, double2* __restrict__ packed, int lc, int nfield2,
              const double2* __restrict__ rec) {
    __shared__ double2 tile[kCoefTile][kCoefTile + 1];   // [m - m0][l - l0]
    const int l0 = blockIdx.x * kCoefTile, m0 = blockIdx.y * kCoefTile;
    const int fk = blockIdx.z, u = fk >> 1, k = fk & 1;
    if (m0 > l0 + kCoefTile - 1) return;
    const int tx = threadIdx.x;
    for (int j = threadIdx.y; j < kCoefTile; j += kCoefRows) {
        const int l = l0 + j, m = m0 + tx;
        double2 v = make_double2(0.0, 0.0);
        if (m <= l && l <= lc && l < cdim && !(k == 1 && m == 0))
            v = cilm[u * sf + k * sk + l * sl + m * sm];
        tile[tx][j] = v;
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kCoefTile; j += kCoefRows) {
        const int m = m0 + j, l = l0 + tx;
        if (m > l || l > lc) continue;
        const long long idx = packed_off(m, lc) + (l - m);
        const double2 v = tile[j][tx];
        const double d = rec[idx].y;
        packed[idx * nfield2 + fk] = make_double2(v.x * d, v.y * d);
    }
}

// unpack: tile sums of the internal fields 2u + k -> complex cilm[u][k][l][m],
// divided by the integral of Y_lm Y*_lm (SHExpandDHC.f95:689-723); the -0
// entry is zero.
__global__ void __launch_bounds__(kCoefTile * kCoefRows)
k_unpack_coef_c(const double2* __restrict__ partial, int ntiles, double2* __restrict__ cilm,
                long long sf, long long sk, long long sl, long long sm, int cdim, int lc,
                long long nlm, int nfield2, int norm, const double* __restrict__ nrm3) {
    const double pi = 3.141592653589793238462643383279502884;
    __shared__ double2 tile[kCoefTile][kCoefTile + 1];   // [m - m0][l - l0]
    const int l0 = blockIdx.x * kCoefTile, m0 = blockIdx.y * kCoefTile;
    const int fk = blockIdx.z, u = fk >> 1, k = fk & 1;
    const int tx = threadIdx.x;
    for (int j = threadIdx.y; j < kCoefTile; j += kCoefRows) {
        const int m = m0 + j, l = l0 + tx;
        double c = 0.0, s = 0.0;
        if (m <= l && l <= lc && l < cdim && !(k == 1 && m == 0)) {
            const long long idx = packed_off(m, lc) + (l - m);
            for (int t = 0; t < ntiles; ++t) {
                const double2 v = partial[((long long)t * nfield2 + fk) * nlm + idx];
                c += v.x;
                s += v.y;
            }
            switch (norm) {
                case 1:
                    c = c / (4 * pi);
                    s = s / (4 * pi);
                    break;
                case 2:
                    c = c * (2 * l + 1) / (4 * pi);
                    s = s * (2 * l + 1) / (4 * pi);
                    break;
                case 3:
                    c = c / nrm3[idx];
                    s = s / nrm3[idx];
                    break;
                default:
                    break;
            }
        }
        tile[j][tx] = make_double2(c, s);
    }
    __syncthreads();
    for (int j = threadIdx.y; j < kCoefTile; j += kCoefRows) {
        const int l = l0 + j, m = m0 + tx;
        if (l >= cdim || m >= cdim) continue;
        cilm[u * sf + k * sk + l * sl + m * sm] = tile[tx][j];
    }
}

// persistent complex-grid FFT kernels over (job, field) items, as k_fft_c2r
template <int MAXR, int MAXT = 512>
__global__ void __launch_bounds__(MAXT, fft_min_ctas<MAXR, MAXT>())
k_fft_c2c_synth(FftArgs F, int tw_smem, int jobs, int nitems,
                const double2* __restrict__ spec, double2* __restrict__ grid, long long gf,
                long long grs, long long gcs, const int* __restrict__ rowN,
                const int* __restrict__ rowS, int lc, int npair, int extend_col, double2* __restrict__ gbuf) {
    extern __shared__ double2 smem_fft[];
    const double2* tw = fft_stage_twiddles(F, smem_fft, tw_smem);
    double2* bufs = fft_buffers(F, smem_fft, gbuf);
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        fft_c2c_synth_body<MAXR>(F, tw, bufs, it % jobs, it / jobs, spec, grid, gf, grs, gcs,
                           rowN, rowS, lc, npair, extend_col);
        __syncthreads();
    }
}

template <int MAXR, int MAXT = 512>
__global__ void __launch_bounds__(MAXT, fft_min_ctas<MAXR, MAXT>())
k_fft_c2c_anal(FftArgs F, int tw_smem, int jobs, int nitems,
               const double2* __restrict__ grid, long long gf, long long grs, long long gcs,
               double2* __restrict__ spec, const int* __restrict__ rowN,
               const int* __restrict__ rowS, const double* __restrict__ wN,
               const double* __restrict__ wS, double wscale, int lc, int npair, double2* __restrict__ gbuf) {
    extern __shared__ double2 smem_fft[];
    const double2* tw = fft_stage_twiddles(F, smem_fft, tw_smem);
    double2* bufs = fft_buffers(F, smem_fft, gbuf);
    for (int it = blockIdx.x; it < nitems; it += gridDim.x) {
        fft_c2c_anal_body<MAXR>(F, tw, bufs, it % jobs, it / jobs, grid, gf, grs, gcs, spec,
                          rowN, rowS, wN, wS, wscale, lc, npair);
        __syncthreads();
    }
}

int launch_pack_coef_c(const shtc_plan* P, const double2* cilm, long long sf, long long sk,
                       long long sl, long long sm, int cdim, double2* packed, int nfield,
                       cudaStream_t st) {
    const int nt = (P->lc + kCoefTile) / kCoefTile;
    const dim3 grid(nt, nt, 2 * nfield), block(kCoefTile, kCoefRows);
    k_pack_coef_c<<<grid, block, 0, st>>>(cilm, sf, sk, sl, sm, cdim, packed, P->lc,
                                          2 * nfield, P->d_rec);
    return map_cuda(cudaGetLastError());
}

int launch_unpack_coef_c(const shtc_plan* P, const double2* partial, int ntiles,
                         double2* cilm, long long sf, long long sk, long long sl,
                         long long sm, int cdim, int nfield, cudaStream_t st) {
    const int nt = (cdim + kCoefTile - 1) / kCoefTile;
    const dim3 grid(nt, nt, 2 * nfield), block(kCoefTile, kCoefRows);
    k_unpack_coef_c<<<grid, block, 0, st>>>(partial, ntiles, cilm, sf, sk, sl, sm, cdim,
                                            P->lc, P->nlm, 2 * nfield, P->norm, P->d_nrm);
    return map_cuda(cudaGetLastError());
}

template <int MAXR, int MAXT = 512>
static int launch_c2c_synth_t(const shtc_plan* P, const double2* spec, double2* grid,
                              long long gf, long long grs, long long gcs, int nfield,
                              cudaStream_t st, double2* gbuf) {
    const FftPlan f = fft_shape<MAXT>(P->fft);
    if (f.gmem && !gbuf) return SHTC_EWORK;
    int rc;
    const int jobs = 2 * P->npair;
    const int nitems = jobs * nfield;
    int blocks = 0;
    if ((rc = fft_launch_setup((const void*)k_fft_c2c_synth<MAXR, MAXT>, f, nitems, &blocks))) return rc;
    if (blocks == 0) return SHTC_OK;
    k_fft_c2c_synth<MAXR, MAXT><<<blocks, f.threads, f.smem, st>>>(
        fft_args(f), f.tw_smem, jobs, nitems, spec, grid, gf, grs, gcs, P->d_rowN,
        P->d_rowS, P->lc, P->npair, P->extend, gbuf);
    return map_cuda(cudaGetLastError());
}

template <int MAXR, int MAXT = 512>
static int launch_c2c_anal_t(const shtc_plan* P, const double2* grid, long long gf,
                             long long grs, long long gcs, double2* spec, int nfield,
                             cudaStream_t st, double2* gbuf) {
    const FftPlan f = fft_shape<MAXT>(P->fft);
    if (f.gmem && !gbuf) return SHTC_EWORK;
    int rc;
    const int jobs = 2 * P->npair;
    const int nitems = jobs * nfield;
    int blocks = 0;
    if ((rc = fft_launch_setup((const void*)k_fft_c2c_anal<MAXR, MAXT>, f, nitems, &blocks))) return rc;
    if (blocks == 0) return SHTC_OK;
    k_fft_c2c_anal<MAXR, MAXT><<<blocks, f.threads, f.smem, st>>>(
        fft_args(f), f.tw_smem, jobs, nitems, grid, gf, grs, gcs, spec, P->d_arowN,
        P->d_arowS, P->d_wN, P->d_wS, 1.0 / (double)P->nlon, P->lc, P->npair, gbuf);
    return map_cuda(cudaGetLastError());
}

int launch_fft_c2c_synth(const shtc_plan* P, const double2* spec, double2* grid,
                         long long gf, long long grs, long long gcs, int nfield,
                         cudaStream_t st, double2* gbuf) {
    switch (fft_variant(P->fft)) {
        case 1: return launch_c2c_synth_t<8>(P, spec, grid, gf, grs, gcs, nfield, st, gbuf);
        case 2:
            return launch_c2c_synth_t<10, 1024>(P, spec, grid, gf, grs, gcs, nfield, st, gbuf);
        default: return launch_c2c_synth_t<13>(P, spec, grid, gf, grs, gcs, nfield, st, gbuf);
    }
}

int launch_fft_c2c_anal(const shtc_plan* P, const double2* grid, long long gf,
                        long long grs, long long gcs, double2* spec, int nfield,
                        cudaStream_t st, double2* gbuf) {
    switch (fft_variant(P->fft)) {
        case 1: return launch_c2c_anal_t<8>(P, grid, gf, grs, gcs, spec, nfield, st, gbuf);
        case 2:
            return launch_c2c_anal_t<10, 1024>(P, grid, gf, grs, gcs, spec, nfield, st, gbuf);
        default: return launch_c2c_anal_t<13>(P, grid, gf, grs, gcs, spec, nfield, st, gbuf);
    }
}

// ---------------------------------------------------------------------------
// MakeGradientDH (src/MakeGradientDH.f95): horizontal gradient on a DH grid.
// With (1 - z^2) dP_l/dz = a_l P_(l-1) - l z P_l, a_l = sqrt((2l+1)(l-m)(l+m)/(2l-1)),
// the theta sums are (S1 - z S2)/u^2 with S1 = sum_l c_(l+1) a_(l+1) P_l and
// S2 = sum_l l c_l P_l, and the phi sums are i m S0 with S0 = sum_l c_l P_l:
// three ordinary Legendre sums per field (internal fields 3u, 3u+1, 3u+2),
// evaluated by the synthesis kernels in one recursion pass.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double grad_a(int l, int m) {
    // sqr(2l+1) * sqr(l-m) * sqr(l+m) / sqr(2l-1), MakeGradientDH.f95:487
    return sqrt((double)(2 * l + 1)) * sqrt((double)(l - m)) * sqrt((double)(l + m)) /
           sqrt((double)(2 * l - 1));
}

__global__ void k_pack_grad(const double* __restrict__ cilm, long long sf, long long sk,
                            long long sl, long long sm, int cdim,
                            double2* __restrict__ packed, int lc, int nfield,
                            const double2* __restrict__ rec) {
    const int m = blockIdx.y;
    const int l = m + blockIdx.x * blockDim.x + threadIdx.x;
    const int u = blockIdx.z;
    if (l > lc) return;
    const long long idx = packed_off(m, lc) + (l - m);
    const double* b = cilm + u * sf;
    double c = 0.0, s = 0.0, c1 = 0.0, s1 = 0.0;
    if (l < cdim) {
        c = b[l * sl + m * sm];
        s = m == 0 ? 0.0 : b[sk + l * sl + m * sm];
    }
    if (l + 1 <= lc && l + 1 < cdim) {
        const double a = grad_a(l + 1, m);
        c1 = b[(l + 1) * sl + m * sm] * a;
        s1 = m == 0 ? 0.0 : b[sk + (l + 1) * sl + m * sm] * a;
    }
    const double d = rec[idx].y;
    double2* o = packed + idx * (3LL * nfield) + 3 * u;
    o[0] = make_double2(c * d, s * d);
    o[1] = make_double2(c1 * d, s1 * d);
    o[2] = make_double2((double)l * c * d, (double)l * s * d);
}

// spec fields 3u..3u+2 -> c2r inputs of the theta (field u) and phi (field
// nfield + u) grids, with the per-ring factors -sin(theta)/(r u^2) and
// 1/(r sin(theta)) (MakeGradientDH.f95:539, 548); zero on the pole rows.
__global__ void k_grad_combine(const double2* __restrict__ spec, double2* __restrict__ out,
                               const double* __restrict__ zp, int npair, int lc, int nlat,
                               int nfield, double inv_r) {
    const long long per = (long long)npair * (lc + 1) * 2;   // one field
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int u = blockIdx.y;
    if (i >= per) return;
    const int h = (int)(i & 1);
    const int m = (int)((i >> 1) % (lc + 1));
    const int p = (int)((i >> 1) / (lc + 1));
    const double2 x0 = spec[(3LL * u + 0) * per + i];
    const double2 x1 = spec[(3LL * u + 1) * per + i];
    const double2 x2 = spec[(3LL * u + 2) * per + i];
    double2 t = make_double2(0.0, 0.0), f = make_double2(0.0, 0.0);
    if (p > 0) {
        const double z = h ? -zp[p] : zp[p];
        const double uu = sqrt((1.0 - z) * (1.0 + z));
        const double st = 2 * p == nlat ? 1.0 : sinpi((double)p / (double)nlat);
        const double ct = -st * inv_r / (uu * uu);
        t = make_double2(ct * (x1.x - z * x2.x), ct * (x1.y - z * x2.y));
        const double cp = (double)m * inv_r / st;
        f = make_double2(-cp * x0.y, cp * x0.x);
    }
    out[(long long)u * per + i] = t;
    out[((long long)nfield + u) * per + i] = f;
}

int launch_pack_grad(const shtc_plan* P, const double* cilm, long long sf, long long sk,
                     long long sl, long long sm, int cdim, double2* packed, int nfield,
                     cudaStream_t st) {
    const int lc = P->lc;
    dim3 grid((lc + 1 + 127) / 128, lc + 1, nfield);
    k_pack_grad<<<grid, 128, 0, st>>>(cilm, sf, sk, sl, sm, cdim, packed, lc, nfield,
                                      P->d_rec);
    return map_cuda(cudaGetLastError());
}

int launch_gradient_dh(const shtc_plan* P, const double* cilm, long long sf, long long sk,
                       long long sl, long long sm, int cdim, double* theta, double* phi,
                       long long gf, long long grs, long long gcs, double radius,
                       int nfield, double2* packed, double2* spec, double2* spec2,
                       cudaStream_t st, double2* gbuf) {
    const int lc = P->lc;
    stage_begin(SHTC_STAGE_PACK, st);
    int rc = launch_pack_grad(P, cilm, sf, sk, sl, sm, cdim, packed, nfield, st);
    stage_end(SHTC_STAGE_PACK, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_SYNTH, st);
    rc = launch_legendre_synth(P, packed, spec, 3 * nfield, st);
    stage_end(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_FFT_C2R, st);
    {
        const long long per = (long long)P->npair * (lc + 1) * 2;
        dim3 grid((unsigned)((per + 255) / 256), nfield);
        k_grad_combine<<<grid, 256, 0, st>>>(spec, spec2, P->d_z, P->npair, lc, P->nlat,
                                             nfield, 1.0 / radius);
        rc = map_cuda(cudaGetLastError());
        if (!rc) rc = launch_fft_c2r(P, spec2, theta, SHTC_F64, gf, grs, gcs, nfield, 0, st,
                                     gbuf);
        if (!rc) rc = launch_fft_c2r(P, spec2 + (long long)nfield * per, phi, SHTC_F64, gf,
                                     grs, gcs, nfield, 0, st, gbuf);
    }
    stage_end(SHTC_STAGE_FFT_C2R, st);
    return rc;
}

}  // namespace shtc
