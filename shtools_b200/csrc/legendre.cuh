// Device code of the FP64 Legendre stages, shared by the per-plan kernels
// (kernels.cu) and the persistent batched kernels (batch.cu).
//
// They follow the reference's on-the-fly recursion (src/MakeGridDH.f95:504-591,
// src/SHExpandDH.f95:463-580): the sectoral start value is scaled by 1e-280,
// the three-term recursion
//     P(l) = z*ff1(l,m)*P(l-1) - ff2(l,m)*P(l-2)
// runs on the scaled values, and the sums are multiplied by u^m * 1e280.
// One work item is one order m for one tile of ring pairs (and one group of
// fields); each thread owns T ring pairs, and the per-degree data of the
// order is read once per item into shared memory and broadcast to all rings.
#pragma once

#include <cuda_runtime.h>

#include "shtc_internal.cuh"

namespace shtc {

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
// synthesis
// ---------------------------------------------------------------------------
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

// Per degree the item needs {ff1, ff2} and NF x {C, S} (16 bytes each);
// chunks of kSynthChunk degrees are copied into shared memory with cp.async
// one chunk ahead of their use.
constexpr int kSynthChunk = 32;

template <int NF>
struct SynthStage {
    double2 buf[2][kSynthChunk * (1 + NF)];
};

// Synthesis of order m for the ring pairs of tile `tile` and the fields
// f0 .. f0+nvalid-1 (nvalid <= NF) of a plan:
//   coef: packed {C, S}, layout [packed (l, m)][nfield] + field
//   spec: [field][pair][m][ring] c2r inputs (a_m - i b_m) * (m ? 1/2 : 1),
//         a_m = sum_l C_lm P_lm, b_m = sum_l S_lm P_lm (MakeGridDH.f95:566-612)
// Ends with a barrier: the shared stage can be reused by the next item.
template <int T, int NF>
__device__ __forceinline__ void synth_order(
    SynthStage<NF>& sm, const double2* __restrict__ rec,
    const double* __restrict__ pmm, const double* __restrict__ rtab,
    const double* __restrict__ zp, const double2* __restrict__ coef,
    double2* __restrict__ spec, int lc, int npair, int nfield, int m, int tile,
    int f0, int nvalid) {
    constexpr int R = 1 + NF;                       // 16-byte items per degree
    const int p0 = tile * (blockDim.x * T) + threadIdx.x;
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
        double2* dst = sm.buf[c & 1];
        const int s0 = 1 + c * kSynthChunk;
        for (int it = threadIdx.x; it < kSynthChunk * R; it += blockDim.x) {
            const int k = it / R, j = it - k * R;
            const int sidx = s0 + k;
            if (sidx <= nsteps && j <= nvalid)
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
        const double2 c = j < nvalid ? cm[j] : make_double2(0.0, 0.0);
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
        const double2* st = sm.buf[c & 1];
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
            if (j >= nvalid) continue;
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
// analysis
// ---------------------------------------------------------------------------
// Input spec[((f*npair + p)*(lc+1) + m)*2 + h] = weighted (Re, -Im) Fourier
// coefficients of the rings (SHExpandDH.f95:470-479).  For each (l, m) the
// sum over ring pairs of P_lm(z_p) * (F_north +- F_south) * u^m/scalef is
// reduced across the CTA: each lane sums its T pairs, a shared-memory
// transpose sums the 32 lanes of a warp for 16 consecutive degrees at a time,
// and warp 0 adds the warps in a fixed order (deterministic).  With more than
// one tile per order the per-tile sums go to partial[tile][...] and the
// unpack kernel adds them, again in a fixed order.
constexpr int kAnalChunk = 16;
constexpr int kAnalPad = 33;

// dynamic shared memory of an analysis CTA of W warps
__host__ __device__ inline size_t anal_smem_bytes(int W) {
    return (size_t)W * (2 * kAnalChunk * kAnalPad) * sizeof(double) +
           (size_t)2 * W * 32 * sizeof(double);
}

// one degree step of the analysis for T ring pairs: the lane's sums over its
// pairs of P * G, G the symmetric (even l-m) or antisymmetric (odd)
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

// Analysis of order m for the ring pairs of tile `tile` of one field:
//   sp:   the field's spec, [pair][m][ring]
//   outp: the tile's packed {C, S} sums of the field, [packed (l, m)]
// smem: anal_smem_bytes(W) bytes; rstage: 2 x kAnalChunk staged {ff1, ff2}.
// Ends with the tile's sums written by warp 0 after a barrier; the caller
// must pass another barrier before reusing the shared memory.
template <int T>
__device__ __forceinline__ void anal_order(
    double* smem, double2 (*rstage)[kAnalChunk], const double2* __restrict__ rec,
    const double* __restrict__ pmm, const double* __restrict__ rtab,
    const double* __restrict__ zp, const double2* __restrict__ sp,
    double2* __restrict__ outp, int lc, int npair, int m, int tile) {
    const int nwarps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    double* bufRe = smem + warp * (2 * kAnalChunk * kAnalPad);
    double* bufIm = bufRe + kAnalChunk * kAnalPad;
    // two buffers of per-warp chunk sums, alternating between chunks
    double* wsum = smem + nwarps * (2 * kAnalChunk * kAnalPad);   // [2][nwarps][32]

    const int p0 = tile * (blockDim.x * T) + threadIdx.x;
    double z[T];
    int pv[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        pv[t] = p0 + t * blockDim.x;
        z[t] = pv[t] < npair ? zp[pv[t]] : 0.0;
    }
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

}  // namespace shtc
