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
// The Legendre kernels follow the reference's on-the-fly recursion
// (src/MakeGridDH.f95:504-591, src/SHExpandDH.f95:463-580): the sectoral
// start value is scaled by 1e-280, the three-term recursion
//     P(l) = z*ff1(l,m)*P(l-1) - ff2(l,m)*P(l-2)
// runs on the scaled values, and the sum is multiplied by u^m * 1e280.
// Where the reference loops over latitude and then m, one CTA here owns a
// pair of orders (m, lc-m), which balances the triangular work, and each
// thread owns T ring pairs; the (l, m) tables and coefficients are read once
// per CTA and broadcast to all rings.
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include "shtc_internal.cuh"

namespace shtc {

// ---------------------------------------------------------------------------
// recursion step
// ---------------------------------------------------------------------------
// P(l) = (z*ff1)*P(l-1) - ff2*P(l-2), rounded as the reference's
// non-fused expression when SHTC_EXACT_RECURSION is set (4 ops), otherwise
// with one fused multiply-add (3 ops).
__device__ __forceinline__ double rec_step(double z, double2 f, double q1,
                                           double q2) {
#if SHTC_EXACT_RECURSION
    return __dsub_rn(__dmul_rn(__dmul_rn(z, f.x), q1), __dmul_rn(f.y, q2));
#else
    return fma(z * f.x, q1, -(f.y * q2));
#endif
}

int map_cuda(cudaError_t e) { return e == cudaSuccess ? SHTC_OK : SHTC_ECUDA; }

// 16-byte asynchronous global -> shared copies (sm_80+ cp.async), used to
// prefetch the next chunk of per-degree data while the current one is used.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::);
}
template <int N>
__device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ---------------------------------------------------------------------------
// coefficient packing
// ---------------------------------------------------------------------------
// scale_mode 0: copy; 1: multiply by the analysis normalisation factor
// (the adjoint of the final divide of SHExpandDH.f95:674-702).
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

__global__ void k_pack_coef(const double* __restrict__ cilm, long long sf,
                            long long sk, long long sl, long long sm, int cdim,
                            double2* __restrict__ packed, int lc, int nfield,
                            int norm, const double* __restrict__ nrm3,
                            int scale_mode) {
    const int m = blockIdx.y;
    const int l = m + blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.z;
    if (l > lc) return;
    const long long idx = packed_off(m, lc) + (l - m);
    double c = 0.0, s = 0.0;
    if (l < cdim) {
        const double* b = cilm + f * sf + l * sl + m * sm;
        c = b[0];
        s = (m == 0) ? 0.0 : b[sk];
    }
    if (scale_mode == 1) {
        const double a = anal_norm_factor(norm, l, nrm3, idx);
        c *= a;
        s *= a;
    }
    packed[idx * nfield + f] = make_double2(c, s);
}

// ---------------------------------------------------------------------------
// Legendre synthesis
// ---------------------------------------------------------------------------
// spec[((f*npair + p)*(lc+1) + m)*2 + h], h = 0 north ring, 1 south ring,
// holds the c2r input of the ring: (a_m - i b_m) * (m ? 1/2 : 1) with
// a_m = sum_l C_lm P_lm, b_m = sum_l S_lm P_lm (MakeGridDH.f95:566-612).
template <int T, int NF>
__device__ __forceinline__ void synth_step(bool odd, double2 f, const double2* c,
                                           const double* z, double* q1, double* q2,
                                           double (*eR)[NF], double (*eI)[NF],
                                           double (*oR)[NF], double (*oI)[NF]) {
#pragma unroll
    for (int t = 0; t < T; ++t) {
        const double p = rec_step(z[t], f, q1[t], q2[t]);
        q2[t] = q1[t];
        q1[t] = p;
#pragma unroll
        for (int j = 0; j < NF; ++j) {
            if (odd) {
                oR[t][j] = fma(c[j].x, p, oR[t][j]);
                oI[t][j] = fma(c[j].y, p, oI[t][j]);
            } else {
                eR[t][j] = fma(c[j].x, p, eR[t][j]);
                eI[t][j] = fma(c[j].y, p, eI[t][j]);
            }
        }
    }
}

// CTA = (ring-pair tile, order m); the grid runs m = 0, 1, ... so the
// longest recursions start first and the hardware scheduler balances the
// triangular work.  Per degree the CTA needs {ff1, ff2} and NF x {C, S}
// (16 bytes each); chunks of kSynthChunk degrees are copied into shared
// memory with cp.async one chunk ahead of their use.
constexpr int kSynthChunk = 32;

template <int T, int NF>
__global__ void __launch_bounds__(128)
k_legendre_synth(const double2* __restrict__ rec, const double* __restrict__ pmm,
                 const double* __restrict__ rtab, const double* __restrict__ zp,
                 const double2* __restrict__ coef, double2* __restrict__ spec,
                 int lc, int npair, int nfield) {
    constexpr int R = 1 + NF;                       // 16-byte items per degree
    __shared__ __align__(16) double2 stage[2][kSynthChunk * R];
    const int m = blockIdx.y;
    const int f0 = blockIdx.z * NF;
    const int p0 = blockIdx.x * (blockDim.x * T) + threadIdx.x;
    double z[T];
    int pv[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        pv[t] = p0 + t * blockDim.x;
        z[t] = pv[t] < npair ? zp[pv[t]] : 0.0;
    }
    const long long o = packed_off(m, lc);
    const double2* __restrict__ rm = rec + o;
    const double2* __restrict__ cm = coef + o * nfield + f0;
    const int nsteps = lc - m;                      // degrees l = m+1 .. lc
    const int nchunks = (nsteps + kSynthChunk - 1) / kSynthChunk;

    auto load_chunk = [&](int c) {
        double2* dst = stage[c & 1];
        const int s0 = 1 + c * kSynthChunk;
        for (int it = threadIdx.x; it < kSynthChunk * R; it += blockDim.x) {
            const int k = it / R, j = it - k * R;
            const int sidx = s0 + k;
            if (sidx <= nsteps)
                cp_async16(&dst[it], j == 0 ? (const void*)&rm[sidx]
                                            : (const void*)&cm[(long long)sidx * nfield + (j - 1)]);
        }
        cp_async_commit();
    };
    if (nchunks > 0) load_chunk(0);

    const double start = pmm[m];
    double q1[T], q2[T];
    double eR[T][NF], eI[T][NF], oR[T][NF], oI[T][NF];
#pragma unroll
    for (int j = 0; j < NF; ++j) {
        const double2 c = cm[j];
#pragma unroll
        for (int t = 0; t < T; ++t) {
            eR[t][j] = c.x * start;
            eI[t][j] = c.y * start;
            oR[t][j] = 0.0;
            oI[t][j] = 0.0;
        }
    }
#pragma unroll
    for (int t = 0; t < T; ++t) { q1[t] = start; q2[t] = 0.0; }

    for (int c = 0; c < nchunks; ++c) {
        if (c + 1 < nchunks) {
            load_chunk(c + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double2* st = stage[c & 1];
        const int cn = min(kSynthChunk, nsteps - c * kSynthChunk);
        // s = 1 + c*kSynthChunk + k: odd for even k (the chunk length is even)
        if (cn == kSynthChunk) {
#pragma unroll
            for (int k = 0; k < kSynthChunk; ++k)
                synth_step<T, NF>((k & 1) == 0, st[k * R], &st[k * R + 1], z, q1, q2,
                                  eR, eI, oR, oI);
        } else {
            for (int k = 0; k < cn; ++k)
                synth_step<T, NF>((k & 1) == 0, st[k * R], &st[k * R + 1], z, q1, q2,
                                  eR, eI, oR, oI);
        }
        __syncthreads();
    }

    const double h = m ? 0.5 : 1.0;
#pragma unroll
    for (int t = 0; t < T; ++t) {
        if (pv[t] >= npair) continue;
        const double r = rtab[(long long)m * npair + pv[t]];
#pragma unroll
        for (int j = 0; j < NF; ++j) {
            double nR = 0.0, nI = 0.0, sR = 0.0, sI = 0.0;
            if (r != 0.0) {
                nR = (eR[t][j] + oR[t][j]) * r;
                nI = (eI[t][j] + oI[t][j]) * r;
                sR = (eR[t][j] - oR[t][j]) * r;
                sI = (eI[t][j] - oI[t][j]) * r;
            }
            double2* o2 = spec + (((long long)(f0 + j) * npair + pv[t]) * (lc + 1) + m) * 2;
            o2[0] = make_double2(nR * h, -nI * h);
            o2[1] = make_double2(sR * h, -sI * h);
        }
    }
}

// ---------------------------------------------------------------------------
// Legendre analysis
// ---------------------------------------------------------------------------
// Input spec[((f*npair + p)*(lc+1) + m)*2 + h] = weighted (Re, -Im) Fourier
// coefficients of the rings (SHExpandDH.f95:470-479).  For each (l, m) the
// sum over ring pairs of P_lm(z_p) * (F_north +- F_south) * u^m/scalef is
// reduced across the CTA: each lane sums its T pairs, a shared-memory
// transpose sums the 32 lanes of a warp for 16 consecutive degrees at a time,
// and warp 0 adds the warps in a fixed order (deterministic).  With more than
// one CTA tile per order the per-tile sums go to partial[tile][...] and the
// unpack kernel adds them, again in a fixed order.
constexpr int kAnalChunk = 16;
constexpr int kAnalPad = 33;

// one degree step of the analysis for T ring pairs: returns the lane's sums
// over its pairs of P * G, G the symmetric (even l-m) or antisymmetric (odd)
// combination of the two rings
template <int T>
__device__ __forceinline__ void anal_step(bool odd, double2 fr, const double* z,
                                          double* q1, double* q2,
                                          const double* gsR, const double* gsI,
                                          const double* gaR, const double* gaI,
                                          double& accR, double& accI) {
    accR = 0.0;
    accI = 0.0;
#pragma unroll
    for (int t = 0; t < T; ++t) {
        const double p = rec_step(z[t], fr, q1[t], q2[t]);
        q2[t] = q1[t];
        q1[t] = p;
        accR = fma(p, odd ? gaR[t] : gsR[t], accR);
        accI = fma(p, odd ? gaI[t] : gsI[t], accI);
    }
}

// CTA = (ring-pair tile, order m), m = 0, 1, ... in launch order (longest
// first).  The {ff1, ff2} of each chunk of kAnalChunk degrees are prefetched
// into shared memory with cp.async one chunk ahead.
template <int T>
__global__ void __launch_bounds__(256)
k_legendre_anal(const double2* __restrict__ rec, const double* __restrict__ pmm,
                const double* __restrict__ rtab, const double* __restrict__ zp,
                const double2* __restrict__ spec, double2* __restrict__ partial,
                int lc, int npair, long long nlm, int nfield) {
    extern __shared__ double smem_anal[];
    __shared__ __align__(16) double2 rstage[2][kAnalChunk];
    const int nwarps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    double* bufRe = smem_anal + warp * (2 * kAnalChunk * kAnalPad);
    double* bufIm = bufRe + kAnalChunk * kAnalPad;
    // two buffers of per-warp chunk sums, alternating between chunks
    double* wsum = smem_anal + nwarps * (2 * kAnalChunk * kAnalPad);   // [2][nwarps][32]

    const int tile = blockIdx.x;
    const int m = blockIdx.y;
    const int f = blockIdx.z;
    const int p0 = tile * (blockDim.x * T) + threadIdx.x;
    double z[T];
    int pv[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        pv[t] = p0 + t * blockDim.x;
        z[t] = pv[t] < npair ? zp[pv[t]] : 0.0;
    }
    const double2* __restrict__ sp = spec + (long long)f * npair * (lc + 1) * 2;
    double2* __restrict__ outp = partial + ((long long)tile * nfield + f) * nlm;
    const long long o = packed_off(m, lc);
    const double2* __restrict__ rm = rec + o;
    const int nsteps = lc - m + 1;   // degrees l = m .. lc, s = l - m
    const int nchunks = (nsteps + kAnalChunk - 1) / kAnalChunk;
    auto load_chunk = [&](int c) {
        const int sidx = c * kAnalChunk + threadIdx.x;
        if (threadIdx.x < kAnalChunk && sidx < nsteps)
            cp_async16(&rstage[c & 1][threadIdx.x], &rm[sidx]);
        cp_async_commit();
    };
    load_chunk(0);

    const double start = pmm[m];
    // symmetric (l-m even) and antisymmetric (l-m odd) combinations
    double gsR[T], gsI[T], gaR[T], gaI[T], q1[T], q2[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        gsR[t] = gsI[t] = gaR[t] = gaI[t] = 0.0;
        if (pv[t] < npair) {
            const double r = rtab[(long long)m * npair + pv[t]];
            if (r != 0.0) {
                const double2 a = sp[((long long)pv[t] * (lc + 1) + m) * 2 + 0];
                const double2 b = sp[((long long)pv[t] * (lc + 1) + m) * 2 + 1];
                const double aR = a.x * r, aI = a.y * r;
                const double bR = b.x * r, bI = b.y * r;
                gsR[t] = aR + bR; gsI[t] = aI + bI;
                gaR[t] = aR - bR; gaI[t] = aI - bI;
            }
        }
        q1[t] = start;
        q2[t] = 0.0;
    }
    int buf = 0;
    for (int c = 0; c < nchunks; ++c) {
        const int c0 = c * kAnalChunk;
        const int cn = min(kAnalChunk, nsteps - c0);
        if (c + 1 < nchunks) {
            load_chunk(c + 1);
            cp_async_wait<1>();
        } else {
            cp_async_wait<0>();
        }
        __syncthreads();
        const double2* wcoef = rstage[c & 1];
        double accR, accI;
        if (cn == kAnalChunk) {
            // c0 is a multiple of the (even) chunk length: the parity of
            // s = c0 + k is that of k, fixed by the unrolling
#pragma unroll
            for (int k = 0; k < kAnalChunk; ++k) {
                if (k == 0 && c0 == 0) {
                    accR = 0.0;
                    accI = 0.0;
#pragma unroll
                    for (int t = 0; t < T; ++t) {
                        accR = fma(q1[t], gsR[t], accR);
                        accI = fma(q1[t], gsI[t], accI);
                    }
                } else {
                    anal_step<T>((k & 1) != 0, wcoef[k], z, q1, q2, gsR, gsI, gaR, gaI,
                                 accR, accI);
                }
                bufRe[k * kAnalPad + lane] = accR;
                bufIm[k * kAnalPad + lane] = accI;
            }
        } else {
            for (int k = 0; k < cn; ++k) {
                if (k == 0 && c0 == 0) {
                    accR = 0.0;
                    accI = 0.0;
#pragma unroll
                    for (int t = 0; t < T; ++t) {
                        accR = fma(q1[t], gsR[t], accR);
                        accI = fma(q1[t], gsI[t], accI);
                    }
                } else {
                    anal_step<T>((k & 1) != 0, wcoef[k], z, q1, q2, gsR, gsI, gaR, gaI,
                                 accR, accI);
                }
                bufRe[k * kAnalPad + lane] = accR;
                bufIm[k * kAnalPad + lane] = accI;
            }
        }
        __syncwarp();
        // lane j < 16 sums the real parts of degree c0+j, lane j >= 16 the
        // imaginary parts of degree c0+j-16, over the 32 lanes of the warp
        {
            const int row = lane & (kAnalChunk - 1);
            const double* b = (lane < kAnalChunk ? bufRe : bufIm) + row * kAnalPad;
            double sum = 0.0;
            if (row < cn) {
#pragma unroll 8
                for (int i = 0; i < 32; ++i) sum += b[i];
            }
            wsum[(buf * nwarps + warp) * 32 + lane] = sum;
        }
        __syncthreads();
        if (warp == 0) {
            double sum = 0.0;
            for (int w = 0; w < nwarps; ++w) sum += wsum[(buf * nwarps + w) * 32 + lane];
            const int row = lane & (kAnalChunk - 1);
            if (row < cn) {
                double* dst = reinterpret_cast<double*>(outp + o + c0 + row);
                dst[lane < kAnalChunk ? 0 : 1] = sum;
            }
        }
        buf ^= 1;
    }
}

// ---------------------------------------------------------------------------
// coefficient unpacking + analysis normalisation
// ---------------------------------------------------------------------------
// normalise 1: divide by the integral of Ylm^2 exactly as the reference
// (SHExpandDH.f95:674-702); 0: no normalisation (synthesis adjoint).
__global__ void k_unpack_coef(const double2* __restrict__ partial, int ntiles,
                              double* __restrict__ cilm, long long sf,
                              long long sk, long long sl, long long sm, int cdim,
                              int lc, long long nlm, int nfield, int norm,
                              const double* __restrict__ nrm3, int normalise) {
    const double pi = 3.141592653589793238462643383279502884;
    const int m = blockIdx.y;
    const int l = blockIdx.x * blockDim.x + threadIdx.x;
    const int f = blockIdx.z;
    if (l >= cdim) return;
    double c = 0.0, s = 0.0;
    if (m <= l && l <= lc) {
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
    double* b = cilm + f * sf + l * sl + m * sm;
    b[0] = c;
    b[sk] = s;
}

// ---------------------------------------------------------------------------
// FFT: Stockham autosort passes in shared memory
// ---------------------------------------------------------------------------
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// table entries are exp(-2 pi i t / len); SIGN > 0 takes the conjugate
template <int SIGN>
__device__ __forceinline__ double2 twv(const double2* tw, int t) {
    double2 w = tw[t];
    if (SIGN > 0) w.y = -w.y;
    return w;
}

// cos and sin of 2*pi*u/R for the odd radices, 1 <= u <= (R-1)/2 (values
// of the circular functions rounded to double, evaluated in extended
// precision).  With the butterfly loops unrolled, u is a compile-time
// constant and these fold to immediates.
__host__ __device__ constexpr double root_cos(int R, int u) {
    return R == 3 ? -0.5
         : R == 5 ? (u == 1 ? 0.30901699437494745 : -0.8090169943749475)
         : R == 7 ? (u == 1 ? 0.6234898018587335 : u == 2 ? -0.2225209339563144
                             : -0.9009688679024191)
         : R == 11 ? (u == 1 ? 0.8412535328311812 : u == 2 ? 0.41541501300188644
                     : u == 3 ? -0.14231483827328514 : u == 4 ? -0.6548607339452851
                     : -0.9594929736144974)
         : (u == 1 ? 0.8854560256532099 : u == 2 ? 0.5680647467311558
            : u == 3 ? 0.12053668025532305 : u == 4 ? -0.3546048870425356
            : u == 5 ? -0.7485107481711011 : -0.970941817426052);
}
__host__ __device__ constexpr double root_sin(int R, int u) {
    return R == 3 ? 0.8660254037844386
         : R == 5 ? (u == 1 ? 0.9510565162951535 : 0.5877852522924731)
         : R == 7 ? (u == 1 ? 0.7818314824680298 : u == 2 ? 0.9749279121818236
                             : 0.4338837391175581)
         : R == 11 ? (u == 1 ? 0.5406408174555976 : u == 2 ? 0.9096319953545183
                     : u == 3 ? 0.9898214418809327 : u == 4 ? 0.7557495743542583
                     : 0.28173255684142967)
         : (u == 1 ? 0.46472317204376856 : u == 2 ? 0.8229838658936564
            : u == 3 ? 0.992708874098054 : u == 4 ? 0.9350162426854148
            : u == 5 ? 0.6631226582407952 : 0.23931566428755777);
}

// radix-R DFT of v[] in place (R = 2, 4, or an odd prime <= 13)
template <int R, int SIGN>
__device__ __forceinline__ void dft_small(double2* v) {
    if (R == 2) {
        const double2 a = v[0], b = v[1];
        v[0] = make_double2(a.x + b.x, a.y + b.y);
        v[1] = make_double2(a.x - b.x, a.y - b.y);
    } else if (R == 4) {
        const double2 s0 = make_double2(v[0].x + v[2].x, v[0].y + v[2].y);
        const double2 d0 = make_double2(v[0].x - v[2].x, v[0].y - v[2].y);
        const double2 s1 = make_double2(v[1].x + v[3].x, v[1].y + v[3].y);
        const double2 d1 = make_double2(v[1].x - v[3].x, v[1].y - v[3].y);
        // forward: multiply d1 by -i; backward: by +i
        const double2 e = SIGN < 0 ? make_double2(d1.y, -d1.x) : make_double2(-d1.y, d1.x);
        v[0] = make_double2(s0.x + s1.x, s0.y + s1.y);
        v[2] = make_double2(s0.x - s1.x, s0.y - s1.y);
        v[1] = make_double2(d0.x + e.x, d0.y + e.y);
        v[3] = make_double2(d0.x - e.x, d0.y - e.y);
    } else {
        // odd R: pair q with R-q; y_s = x0 + sum_q cos(2pi sq/R) a_q -+ i sum_q sin b_q
        constexpr int H = (R - 1) / 2;
        double2 a[H + 1], b[H + 1];
        double2 y0 = v[0];
#pragma unroll
        for (int q = 1; q <= H; ++q) {
            a[q] = make_double2(v[q].x + v[R - q].x, v[q].y + v[R - q].y);
            b[q] = make_double2(v[q].x - v[R - q].x, v[q].y - v[R - q].y);
            y0.x += a[q].x;
            y0.y += a[q].y;
        }
        const double2 x0 = v[0];
        v[0] = y0;
#pragma unroll
        for (int s = 1; s <= H; ++s) {
            double2 re = x0, im = make_double2(0.0, 0.0);
#pragma unroll
            for (int q = 1; q <= H; ++q) {
                const int t = (s * q) % R;
                const int u = t <= H ? t : R - t;
                const double c = root_cos(R, u);
                const double sn = t <= H ? root_sin(R, u) : -root_sin(R, u);
                re.x = fma(c, a[q].x, re.x);
                re.y = fma(c, a[q].y, re.y);
                im.x = fma(sn, b[q].x, im.x);
                im.y = fma(sn, b[q].y, im.y);
            }
            // forward: y_s = re - i im, y_{R-s} = re + i im
            if (SIGN < 0) {
                v[s] = make_double2(re.x + im.y, re.y - im.x);
                v[R - s] = make_double2(re.x - im.y, re.y + im.x);
            } else {
                v[s] = make_double2(re.x - im.y, re.y + im.x);
                v[R - s] = make_double2(re.x + im.y, re.y - im.x);
            }
        }
    }
}

// One Stockham pass of radix R from x to y (ping-pong shared buffers).
template <int R, int SIGN>
__device__ __forceinline__ void fft_pass(const double2* __restrict__ x,
                                         double2* __restrict__ y, int M, int ns,
                                         const double2* __restrict__ tw) {
    const int nr = M / R;
    const int step = M / (ns * R);
    for (int j = threadIdx.x; j < nr; j += blockDim.x) {
        const int k = j % ns;
        double2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = x[j + q * nr];
        if (k != 0) {
#pragma unroll
            for (int q = 1; q < R; ++q) v[q] = cmul(v[q], twv<SIGN>(tw, k * q * step));
        }
        dft_small<R, SIGN>(v);
        const int d = (j - k) * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) y[d + q * ns] = v[q];
    }
}

// Runs the passes; the data starts in a, the result pointer is returned.
template <int SIGN>
__device__ double2* fft_run(double2* a, double2* b, int M, const int* fac,
                            int nfac, const double2* __restrict__ tw) {
    int ns = 1;
    for (int i = 0; i < nfac; ++i) {
        __syncthreads();
        const int r = fac[i];
        switch (r) {
            case 2: fft_pass<2, SIGN>(a, b, M, ns, tw); break;
            case 3: fft_pass<3, SIGN>(a, b, M, ns, tw); break;
            case 4: fft_pass<4, SIGN>(a, b, M, ns, tw); break;
            case 5: fft_pass<5, SIGN>(a, b, M, ns, tw); break;
            case 7: fft_pass<7, SIGN>(a, b, M, ns, tw); break;
            case 11: fft_pass<11, SIGN>(a, b, M, ns, tw); break;
            case 13: fft_pass<13, SIGN>(a, b, M, ns, tw); break;
            default: break;
        }
        ns *= r;
        double2* t = a;
        a = b;
        b = t;
    }
    __syncthreads();
    return a;
}

struct FftArgs {
    int n, mode, m, nfac, bluestein, mb;
    int fac[kMaxFactors];
    const double2* tw;
    const double2* twn;
    const double2* chirp;
    const double2* kern;
};

// Complex DFT of length F.m of buf with sign SIGN; buf and tmp each hold
// F.mb (Bluestein) or F.m elements.  Returns the pointer holding the result.
template <int SIGN>
__device__ double2* fft_exec(const FftArgs& F, double2* buf, double2* tmp) {
    __syncthreads();
    if (!F.bluestein) return fft_run<SIGN>(buf, tmp, F.m, F.fac, F.nfac, F.tw);
    // Bluestein: X_k = c_k sum_j (x_j c_j) conj(c_{k-j}), c_t = exp(-+ i pi t^2/m)
    const int m = F.m, mb = F.mb;
    for (int t = threadIdx.x; t < mb; t += blockDim.x) {
        if (t < m) {
            double2 c = F.chirp[t];
            if (SIGN > 0) c.y = -c.y;
            buf[t] = cmul(buf[t], c);
        } else {
            buf[t] = make_double2(0.0, 0.0);
        }
    }
    double2* r = fft_run<-1>(buf, tmp, mb, F.fac, F.nfac, F.tw);
    double2* o = (r == buf) ? tmp : buf;
    for (int t = threadIdx.x; t < mb; t += blockDim.x) {
        double2 kf;
        if (SIGN < 0) {
            kf = F.kern[t];
        } else {
            kf = F.kern[(mb - t) & (mb - 1)];
            kf.y = -kf.y;
        }
        r[t] = cmul(r[t], kf);
    }
    double2* r2 = fft_run<+1>(r, o, mb, F.fac, F.nfac, F.tw);
    const double inv = 1.0 / (double)mb;
    for (int t = threadIdx.x; t < m; t += blockDim.x) {
        double2 c = F.chirp[t];
        if (SIGN > 0) c.y = -c.y;
        const double2 v = make_double2(r2[t].x * inv, r2[t].y * inv);
        r2[t] = cmul(v, c);
    }
    __syncthreads();
    return r2;
}

// c2r: spec -> grid.  mode 0 (odd n): CTA = (pair, field), the two rings are
// the real and imaginary parts of one complex length-n inverse DFT.  mode 1
// (even n): CTA = (pair*2 + ring, field), the ring is computed by a complex
// length-n/2 inverse DFT and the even/odd split.  Output rows are scaled by
// the ring weight when wN/wS are given (analysis adjoint).
__global__ void __launch_bounds__(512) k_fft_c2r(FftArgs F, const double2* __restrict__ spec,
                          double* __restrict__ grid, long long gf, long long grs,
                          long long gcs, const int* __restrict__ rowN,
                          const int* __restrict__ rowS,
                          const double* __restrict__ wN,
                          const double* __restrict__ wS, double wscale, int lc,
                          int npair, int extend_col) {
    extern __shared__ double2 smem_fft[];
    const int f = blockIdx.y;
    const int job = blockIdx.x;
    const int len = F.bluestein ? F.mb : F.m;
    double2* a = smem_fft;
    double2* b = smem_fft + len;
    const int n = F.n;
    if (F.mode == 0) {
        const int p = job;
        const int rN = rowN[p], rS = rowS[p];
        const double2* X = spec + ((long long)f * npair + p) * (lc + 1) * 2;
        for (int k = threadIdx.x; k < n; k += blockDim.x) a[k] = make_double2(0.0, 0.0);
        __syncthreads();
        for (int k = threadIdx.x; k <= lc; k += blockDim.x) {
            double2 xn = X[2 * k + 0];
            double2 xs = rS >= 0 ? X[2 * k + 1] : make_double2(0.0, 0.0);
            if (k == 0) {
                xn.y = 0.0;
                xs.y = 0.0;
            }
            // Z_k = X^N_k + i X^S_k ; Z_{n-k} = conj(X^N_k) + i conj(X^S_k)
            a[k] = make_double2(xn.x - xs.y, xn.y + xs.x);
            if (k > 0) a[n - k] = make_double2(xn.x + xs.y, -xn.y + xs.x);
        }
        const double2* r = fft_exec<+1>(F, a, b);
        const double sN = wN ? wN[p] * wscale : 1.0;
        const double sS = wS ? wS[p] * wscale : 1.0;
        double* gN = rN >= 0 ? grid + f * gf + rN * grs : nullptr;
        double* gS = rS >= 0 ? grid + f * gf + rS * grs : nullptr;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double2 v = r[j];
            if (gN) gN[j * gcs] = v.x * sN;
            if (gS) gS[j * gcs] = v.y * sS;
        }
        if (extend_col && threadIdx.x == 0) {
            if (gN) gN[(long long)n * gcs] = r[0].x * sN;
            if (gS) gS[(long long)n * gcs] = r[0].y * sS;
        }
    } else {
        const int p = job >> 1;
        const int h = job & 1;
        const int row = h ? rowS[p] : rowN[p];
        if (row < 0) return;
        const int M = F.m;   // n/2
        const double2* X = spec + ((long long)f * npair + p) * (lc + 1) * 2 + h;
        // Z'_k = (X_k + conj X_{M-k}) + i w^{-k} (X_k - conj X_{M-k}), w = exp(-2 pi i/n)
        for (int k = threadIdx.x; k < M; k += blockDim.x) {
            double2 xk = k <= lc ? X[2 * k] : make_double2(0.0, 0.0);
            if (k == 0) xk.y = 0.0;
            const int km = M - k;
            double2 xm = (km <= lc && km < M) ? X[2 * km] : make_double2(0.0, 0.0);
            if (km == 0) xm.y = 0.0;
            const double2 A = make_double2(xk.x + xm.x, xk.y - xm.y);
            const double2 B = make_double2(xk.x - xm.x, xk.y + xm.y);
            double2 w = F.twn[k];
            w.y = -w.y;                         // exp(+2 pi i k/n)
            const double2 wb = cmul(w, B);
            a[k] = make_double2(A.x - wb.y, A.y + wb.x);
        }
        const double2* r = fft_exec<+1>(F, a, b);
        const double sc = (h ? (wS ? wS[p] * wscale : 1.0) : (wN ? wN[p] * wscale : 1.0));
        double* g = grid + f * gf + row * grs;
        for (int j = threadIdx.x; j < M; j += blockDim.x) {
            const double2 v = r[j];
            g[(2LL * j) * gcs] = v.x * sc;
            g[(2LL * j + 1) * gcs] = v.y * sc;
        }
        if (extend_col && threadIdx.x == 0) g[(long long)n * gcs] = r[0].x * sc;
    }
}

// r2c: grid rows -> spec (m = 0..lc), each multiplied by the ring weight
// (times wscale) as (Re, -Im), the reference's fcoef (SHExpandGLQ.f95:535-547).
// fold_extend adds column n into column 0 (adjoint of the extend copy).
__global__ void __launch_bounds__(512) k_fft_r2c(FftArgs F, const double* __restrict__ grid,
                          long long gf, long long grs, long long gcs,
                          double2* __restrict__ spec, const int* __restrict__ rowN,
                          const int* __restrict__ rowS,
                          const double* __restrict__ wN,
                          const double* __restrict__ wS, double wscale, int lc,
                          int npair, int fold_extend) {
    extern __shared__ double2 smem_fft[];
    const int f = blockIdx.y;
    const int job = blockIdx.x;
    const int len = F.bluestein ? F.mb : F.m;
    double2* a = smem_fft;
    double2* b = smem_fft + len;
    const int n = F.n;
    if (F.mode == 0) {
        const int p = job;
        const int rN = rowN[p], rS = rowS[p];
        const double* gN = rN >= 0 ? grid + f * gf + rN * grs : nullptr;
        const double* gS = rS >= 0 ? grid + f * gf + rS * grs : nullptr;
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            double xn = gN ? gN[j * gcs] : 0.0;
            double xs = gS ? gS[j * gcs] : 0.0;
            if (fold_extend && j == 0) {
                if (gN) xn += gN[(long long)n * gcs];
                if (gS) xs += gS[(long long)n * gcs];
            }
            a[j] = make_double2(xn, xs);
        }
        const double2* r = fft_exec<-1>(F, a, b);
        const double sN = wN ? wN[p] * wscale : wscale;
        const double sS = wS ? wS[p] * wscale : wscale;
        double2* X = spec + ((long long)f * npair + p) * (lc + 1) * 2;
        for (int k = threadIdx.x; k <= lc; k += blockDim.x) {
            const double2 zk = r[k];
            const double2 zm = r[k == 0 ? 0 : n - k];
            // X^N = (Z_k + conj Z_{n-k})/2 ; X^S = (Z_k - conj Z_{n-k})/(2i)
            const double nr = 0.5 * (zk.x + zm.x), ni = 0.5 * (zk.y - zm.y);
            const double sr = 0.5 * (zk.y + zm.y), si = -0.5 * (zk.x - zm.x);
            X[2 * k + 0] = make_double2(sN * nr, -(sN * ni));
            X[2 * k + 1] = make_double2(sS * sr, -(sS * si));
        }
    } else {
        const int p = job >> 1;
        const int h = job & 1;
        const int row = h ? rowS[p] : rowN[p];
        double2* X = spec + ((long long)f * npair + p) * (lc + 1) * 2 + h;
        if (row < 0) {
            for (int k = threadIdx.x; k <= lc; k += blockDim.x) X[2 * k] = make_double2(0.0, 0.0);
            return;
        }
        const int M = F.m;
        const double* g = grid + f * gf + row * grs;
        for (int j = threadIdx.x; j < M; j += blockDim.x) {
            double x0 = g[(2LL * j) * gcs];
            const double x1 = g[(2LL * j + 1) * gcs];
            if (fold_extend && j == 0) x0 += g[(long long)n * gcs];
            a[j] = make_double2(x0, x1);
        }
        const double2* r = fft_exec<-1>(F, a, b);
        const double sc = h ? (wS ? wS[p] * wscale : wscale) : (wN ? wN[p] * wscale : wscale);
        for (int k = threadIdx.x; k <= lc; k += blockDim.x) {
            const double2 zk = r[k == M ? 0 : k];
            const double2 zm = r[k == 0 ? 0 : M - k];
            // E = (Z_k + conj Z_{M-k})/2, O = (Z_k - conj Z_{M-k})/(2i), X = E + w^k O
            const double2 E = make_double2(0.5 * (zk.x + zm.x), 0.5 * (zk.y - zm.y));
            const double2 O = make_double2(0.5 * (zk.y + zm.y), -0.5 * (zk.x - zm.x));
            const double2 wo = cmul(F.twn[k], O);
            const double xr = E.x + wo.x, xi = E.y + wo.y;
            X[2 * k] = make_double2(sc * xr, -(sc * xi));
        }
    }
}

// ---------------------------------------------------------------------------
// launchers
// ---------------------------------------------------------------------------
static FftArgs fft_args(const FftPlan& f) {
    FftArgs a;
    a.n = f.n; a.mode = f.mode; a.m = f.m; a.nfac = f.nfac;
    a.bluestein = f.bluestein; a.mb = f.mb;
    for (int i = 0; i < kMaxFactors; ++i) a.fac[i] = i < f.nfac ? f.fac[i] : 0;
    a.tw = f.d_tw; a.twn = f.d_twn; a.chirp = f.d_chirp; a.kern = f.d_kern;
    return a;
}

int launch_pack_coef(const shtc_plan* P, const double* cilm, long long sf,
                     long long sk, long long sl, long long sm, int cdim,
                     double2* packed, int nfield, int scale_mode,
                     cudaStream_t st) {
    const int lc = P->lc;
    dim3 grid((lc + 1 + 127) / 128, lc + 1, nfield);
    k_pack_coef<<<grid, 128, 0, st>>>(cilm, sf, sk, sl, sm, cdim, packed, lc,
                                      nfield, P->norm, P->d_nrm, scale_mode);
    return map_cuda(cudaGetLastError());
}

template <int T, int NF>
static void launch_synth_t(const shtc_plan* P, const double2* packed,
                           double2* spec, int nfield, cudaStream_t st) {
    const int threads = 128;
    const int tiles = (P->npair + threads * T - 1) / (threads * T);
    dim3 grid(tiles, P->lc + 1, nfield / NF);
    k_legendre_synth<T, NF><<<grid, threads, 0, st>>>(
        P->d_rec, P->d_pmm, P->d_rtab, P->d_z, packed, spec, P->lc, P->npair,
        nfield);
}

int launch_legendre_synth(const shtc_plan* P, const double2* packed,
                          double2* spec, int nfield, cudaStream_t st) {
    const int np = P->npair;
    if (nfield % 4 == 0 && nfield >= 8) {
        launch_synth_t<2, 4>(P, packed, spec, nfield, st);
    } else if (nfield % 2 == 0 && nfield >= 2) {
        if (np > 512) launch_synth_t<4, 2>(P, packed, spec, nfield, st);
        else launch_synth_t<2, 2>(P, packed, spec, nfield, st);
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

// analysis CTA shape: T pairs per thread, W warps
static void anal_shape(const shtc_plan* P, int* T, int* W, int* tiles) {
    const int np = P->npair;
    int w = P->tune_anal_W ? P->tune_anal_W : 2;
    int t = P->tune_anal_T;
    if (t == 0) {
        // largest T (at most 4) that leaves at least two CTA tiles of ring
        // pairs: what the autotuner's sweeps on B200 select for lmax 63..2799
        t = 1;
        while (t < 4 && 32 * w * (2 * t) <= np / 2) t *= 2;
    }
    *T = t;
    *W = w;
    *tiles = (np + 32 * t * w - 1) / (32 * t * w);
}

int anal_tiles(const shtc_plan* P) {
    int T, W, tiles;
    anal_shape(P, &T, &W, &tiles);
    return tiles;
}

template <int T>
static int launch_anal_t(const shtc_plan* P, const double2* spec,
                         double2* partial, int nfield, int W, int tiles,
                         cudaStream_t st) {
    const int threads = 32 * W;
    const size_t smem = (size_t)W * (2 * kAnalChunk * kAnalPad) * sizeof(double)
                        + (size_t)2 * W * 32 * sizeof(double);
    cudaError_t e = cudaFuncSetAttribute(k_legendre_anal<T>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem);
    if (e != cudaSuccess) return map_cuda(e);
    dim3 grid(tiles, P->lc + 1, nfield);
    k_legendre_anal<T><<<grid, threads, smem, st>>>(
        P->d_rec, P->d_pmm, P->d_rtab, P->d_z, spec, partial, P->lc, P->npair,
        P->nlm, nfield);
    return map_cuda(cudaGetLastError());
}

int launch_legendre_anal(const shtc_plan* P, const double2* spec,
                         double2* partial, int ntiles_out, int nfield,
                         cudaStream_t st) {
    int T, W, tiles;
    anal_shape(P, &T, &W, &tiles);
    if (tiles != ntiles_out) return SHTC_EBOUND;
    switch (T) {
        case 8: return launch_anal_t<8>(P, spec, partial, nfield, W, tiles, st);
        case 4: return launch_anal_t<4>(P, spec, partial, nfield, W, tiles, st);
        case 2: return launch_anal_t<2>(P, spec, partial, nfield, W, tiles, st);
        default: return launch_anal_t<1>(P, spec, partial, nfield, W, tiles, st);
    }
}

int launch_unpack_coef(const shtc_plan* P, const double2* partial, int ntiles,
                       double* cilm, long long sf, long long sk, long long sl,
                       long long sm, int cdim, int nfield, int normalise,
                       cudaStream_t st) {
    const int lc = P->lc;
    dim3 grid((cdim + 127) / 128, cdim, nfield);
    k_unpack_coef<<<grid, 128, 0, st>>>(partial, ntiles, cilm, sf, sk, sl, sm,
                                        cdim, lc, P->nlm, nfield, P->norm,
                                        P->d_nrm, normalise);
    return map_cuda(cudaGetLastError());
}

static int fft_smem_setup(const void* fn, const FftPlan& f) {
    return map_cuda(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)f.smem));
}

int launch_fft_c2r(const shtc_plan* P, const double2* spec, double* grid,
                   long long gf, long long grs, long long gcs, int nfield,
                   int weighted, cudaStream_t st) {
    const FftPlan& f = P->fft;
    int rc = fft_smem_setup((const void*)k_fft_c2r, f);
    if (rc) return rc;
    const int jobs = f.mode == 0 ? P->npair : 2 * P->npair;
    dim3 g(jobs, nfield);
    // synthesis uses the synthesis ring map (with the extend row and column);
    // the analysis adjoint uses the analysis ring map and ring weights
    if (weighted) {
        k_fft_c2r<<<g, f.threads, f.smem, st>>>(fft_args(f), spec, grid, gf, grs,
                                                gcs, P->d_arowN, P->d_arowS,
                                                P->d_wN, P->d_wS,
                                                1.0 / (double)P->nlon, P->lc,
                                                P->npair, 0);
    } else {
        k_fft_c2r<<<g, f.threads, f.smem, st>>>(fft_args(f), spec, grid, gf, grs,
                                                gcs, P->d_rowN, P->d_rowS,
                                                nullptr, nullptr, 1.0, P->lc,
                                                P->npair, P->extend);
    }
    return map_cuda(cudaGetLastError());
}

int launch_fft_r2c(const shtc_plan* P, const double* grid, long long gf,
                   long long grs, long long gcs, double2* spec, int nfield,
                   int weighted, int fold_extend, cudaStream_t st) {
    const FftPlan& f = P->fft;
    int rc = fft_smem_setup((const void*)k_fft_r2c, f);
    if (rc) return rc;
    const int jobs = f.mode == 0 ? P->npair : 2 * P->npair;
    dim3 g(jobs, nfield);
    if (weighted) {
        // analysis: fcoef = (w * Re) / nlong, the reference's order of operations
        // is reproduced up to one rounding by folding 1/nlong into the weight
        k_fft_r2c<<<g, f.threads, f.smem, st>>>(fft_args(f), grid, gf, grs, gcs,
                                                spec, P->d_arowN, P->d_arowS,
                                                P->d_wN, P->d_wS,
                                                1.0 / (double)P->nlon, P->lc,
                                                P->npair, 0);
    } else {
        // synthesis adjoint: plain (Re, -Im) of the rows of the cotangent
        k_fft_r2c<<<g, f.threads, f.smem, st>>>(fft_args(f), grid, gf, grs, gcs,
                                                spec, P->d_rowN, P->d_rowS,
                                                nullptr, nullptr, 1.0, P->lc,
                                                P->npair, fold_extend);
    }
    return map_cuda(cudaGetLastError());
}

}  // namespace shtc
