// Device code of the FP64 Legendre stages, shared by the per-plan kernels
// (kernels.cu) and the persistent batched kernels (batch.cu).
//
// They follow the reference's on-the-fly recursion (src/MakeGridDH.f95:504-591,
// src/SHExpandDH.f95:463-580): the sectoral start value is scaled by 1e-280,
// the three-term recursion
//     P(l) = z*ff1(l,m)*P(l-1) - ff2(l,m)*P(l-2)
// runs on the scaled values, and the sums are multiplied by u^m * 1e280.
//
// The recursion is run in a rescaled form with two FP64 operations per
// degree instead of four.  With s = l - m, a(s) = ff1, b(s) = ff2 and
// segments of kRecSegment degrees (s0, s0 + kRecSegment], s0 a multiple of
// kRecSegment,
//     P(s) = D(s) * Q(s),   D(s) = a(s0+1) * ... * a(s),
//     Q(s) = z * Q(s-1) - beta(s) * Q(s-2),   beta(s) = b(s) / (a(s) a(s-1)),
// which is the same recursion (D(s-2)/D(s) = 1/(a(s) a(s-1)) across a
// segment start too, once both recursion values are multiplied by the
// segment's last D when it ends).  The table rec[] holds {beta(s), D(s)};
// synthesis coefficients are premultiplied by D(s) when packed and analysis
// sums are multiplied by D(s) when reduced.  Every a(s) >= 1, so Q <= P in
// magnitude; D stays below ~1e24 for lmax <= 2800 and the Q values stay in
// the normal double range.
//
// One work item is one order m for one tile of ring pairs (and one group of
// fields); each thread owns T ring pairs, and the per-degree data of the
// order is read once per item into shared memory and broadcast to all rings.
#pragma once

#include <cuda_runtime.h>

#include "shtc_internal.cuh"

namespace shtc {

// one step of the rescaled recursion: Q(s) = z*Q(s-1) - beta(s)*Q(s-2),
// f = {beta(s), D(s)}
__device__ __forceinline__ double rec_step(double z, double2 f, double q1,
                                           double q2) {
    return fma(z, q1, -(f.x * q2));
}

// end of a recursion segment: both recursion values back to P units
template <int T>
__device__ __forceinline__ void rec_rescale(double d, double* q1, double* q2) {
#pragma unroll
    for (int t = 0; t < T; ++t) {
        q1[t] *= d;
        q2[t] *= d;
    }
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
// RAD: the contraction uses q^s Q(s) for a per-ring factor q (the radial
// factor (r0/r)^l of a potential): qs[] holds q^s and advances by qstep[]
template <int T, int NF, bool RAD = false>
__device__ __forceinline__ void synth_step(bool odd, double2 f, const double2* c,
                                           const double* z, double* qs, const double* qstep,
                                           double* q1, double* q2, double (*eR)[NF],
                                           double (*eI)[NF], double (*oR)[NF],
                                           double (*oI)[NF]) {
#pragma unroll
    for (int t = 0; t < T; ++t) {
        double p = rec_step(z[t], f, q1[t], q2[t]);
        q2[t] = q1[t];
        q1[t] = p;
        if constexpr (RAD) {
            p *= qs[t];
            qs[t] *= qstep[t];
        }
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
// chunks of kSynthChunk degrees are copied into shared memory with cp.async.
// Up to 4 fields: three buffers, each chunk copied two chunks ahead of its
// use and the copy issued after the barrier that ends the buffer's last
// use, so one CTA barrier per chunk suffices (on B200 2.5% faster for one
// field at lmax 2047, 1% for the 4-field groups of the batched launch, the
// same for 2 fields).  8 fields: two buffers, one chunk ahead, two barriers
// per chunk (three buffers measured 2.5-4.5% slower at lmax 719 and 2799).
constexpr int kSynthChunk = 32;
static_assert(kSynthChunk % kRecSegment == 0, "chunks hold whole segments");

__host__ __device__ constexpr int synth_buffers(int NF) { return NF <= 4 ? 3 : 2; }

template <int NF>
struct SynthStage {
    double2 buf[synth_buffers(NF)][kSynthChunk * (1 + NF)];
};

// Synthesis of order m for the ring pairs of tile `tile` and the fields
// f0 .. f0+nvalid-1 (nvalid <= NF) of a plan:
//   coef: packed {C, S}, layout [packed (l, m)][nfield] + field
//   spec: [field][pair][m][ring] c2r inputs (a_m - i b_m) * (m ? 1/2 : 1),
//         a_m = sum_l C_lm P_lm, b_m = sum_l S_lm P_lm (MakeGridDH.f95:566-612)
// Ends with a barrier: the shared stage can be reused by the next item.
// RAD: sums of c_l q^l P_lm for a per-pair factor q, radq[p] = {q, log q}:
// the recursion is the plain one (z exact); each term is multiplied by q^s,
// s = l - m, taken at the first degree of every recursion segment from
// qtab[p * nseg + k] = q^(16k + 1) (accurate powers) and advanced by q
// within the segment; the epilogue multiplies by q^m = exp(m log q).  A
// q^s built by repeated multiplication alone would carry s times the
// rounding of q, and folding q into z and beta would perturb z itself.
template <int T, int NF, bool RAD = false>
__device__ __forceinline__ void synth_order(
    SynthStage<NF>& sm, const double2* __restrict__ rec,
    const double* __restrict__ pmm, const double* __restrict__ rtab,
    const double* __restrict__ zp, const double2* __restrict__ coef,
    double2* __restrict__ spec, int lc, int npair, int nfield, int m, int tile,
    int f0, int nvalid, const double2* __restrict__ radq = nullptr,
    const double* __restrict__ qtab = nullptr, int nseg = 0) {
    constexpr int R = 1 + NF;                       // 16-byte items per degree
    constexpr int NB = synth_buffers(NF);
    const int p0 = tile * (blockDim.x * T) + threadIdx.x;
    double z[T], qs[T], qstep[T], lq[T];
    int pv[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        pv[t] = p0 + t * blockDim.x;
        z[t] = pv[t] < npair ? zp[pv[t]] : 0.0;
        qs[t] = 1.0;
        if constexpr (RAD) {
            const double2 rq = pv[t] < npair ? radq[pv[t]] : make_double2(1.0, 0.0);
            qstep[t] = rq.x;
            lq[t] = rq.y;
        } else {
            qstep[t] = 1.0;
            lq[t] = 0.0;
        }
    }
    // q^s at the first step of segment seg (RAD)
    auto seg_power = [&](int seg) {
#pragma unroll
        for (int t = 0; t < T; ++t)
            qs[t] = pv[t] < npair ? qtab[(long long)pv[t] * nseg + seg] : 1.0;
    };
    const long long o = packed_off(m, lc);
    const double2* __restrict__ rm = rec + o;
    const double2* __restrict__ cm = coef + o * nfield + f0;
    const int nsteps = lc - m;                      // degrees l = m+1 .. lc
    const int nchunks = (nsteps + kSynthChunk - 1) / kSynthChunk;

    auto load_chunk = [&](int c) {
        double2* dst = sm.buf[c % NB];
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
    if (NB == 3 && nchunks > 1) load_chunk(1);

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
        if constexpr (NB == 3) {
            if (c + 1 < nchunks) cp_async_wait<1>(); else cp_async_wait<0>();
            __syncthreads();
            if (c + 2 < nchunks) load_chunk(c + 2);
        } else {
            if (c + 1 < nchunks) {
                load_chunk(c + 1);
                cp_async_wait<1>();
            } else {
                cp_async_wait<0>();
            }
            __syncthreads();
        }
        const double2* st = sm.buf[c % NB];
        const int cn = min(kSynthChunk, nsteps - c * kSynthChunk);
        // s = 1 + c*kSynthChunk + k: odd for even k (the chunk length is even)
        // segments end at s = 32c + 16 and 32c + 32, i.e. k = 15 and 31
        if (cn == kSynthChunk) {
#pragma unroll
            for (int k = 0; k < kSynthChunk; ++k) {
                if constexpr (RAD) {
                    if ((k & (kRecSegment - 1)) == 0)
                        seg_power((c * kSynthChunk + k) / kRecSegment);
                }
                synth_step<T, NF, RAD>((k & 1) == 0, st[k * R], &st[k * R + 1], z, qs,
                                       qstep, q1, q2, eR, eI, oR, oI);
                if ((k & (kRecSegment - 1)) == kRecSegment - 1)
                    rec_rescale<T>(st[k * R].y, q1, q2);
            }
        } else {
            for (int k = 0; k < cn; ++k) {
                if constexpr (RAD) {
                    if ((k & (kRecSegment - 1)) == 0)
                        seg_power((c * kSynthChunk + k) / kRecSegment);
                }
                synth_step<T, NF, RAD>((k & 1) == 0, st[k * R], &st[k * R + 1], z, qs,
                                       qstep, q1, q2, eR, eI, oR, oI);
                if ((k & (kRecSegment - 1)) == kRecSegment - 1)
                    rec_rescale<T>(st[k * R].y, q1, q2);
            }
        }
        if constexpr (NB == 2) __syncthreads();
    }
    if constexpr (NB == 3) __syncthreads();

    const double h = m ? 0.5 : 1.0;
#pragma unroll
    for (int t = 0; t < T; ++t) {
        if (pv[t] >= npair) continue;
        double r = rtab[(long long)m * npair + pv[t]];
        if constexpr (RAD) r *= exp((double)m * lq[t]);
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
// coefficients of the rings (SHExpandDH.f95:470-479).  For each (l, m) and
// field the sum over ring pairs of P_lm(z_p) * (F_north +- F_south) *
// u^m/scalef is reduced across the CTA: each lane sums its T pairs, a
// shared-memory transpose sums the 32 lanes of a warp for a chunk of
// degrees at a time, and warp 0 adds the warps in a fixed order
// (deterministic).  With more than one tile per order the per-tile sums go
// to partial[tile][field][...] and the unpack kernel adds them, again in a
// fixed order.  NF fields share one recursion: per degree a lane does 2T
// recursion operations and 2*T*NF multiply-adds.
constexpr int kAnalChunk = 16;   // degrees per transpose of one field (NF = 1)
// row pitch of the per-warp transpose, in doubles: even, so every row starts
// on 16 bytes and is summed with 16-byte loads; with 34 the 8 lanes of each
// load phase hit disjoint banks
constexpr int kAnalPad = 34;
static_assert(kAnalChunk == kRecSegment, "segment ends fall on chunk starts");
// degrees per stage of staged {beta, D} and per CTA barrier: 32 measured 2%
// faster than 16 at lmax 2047 (no gain at 64)
constexpr int kAnalStage = 32;
static_assert(kAnalStage % kRecSegment == 0, "stages hold whole segments");

// degrees per transpose chunk for NF fields: 2*NF*CH = 32 rows, one per lane
__host__ __device__ constexpr int anal_chunk(int NF) { return kAnalChunk / NF; }

// dynamic shared memory of an analysis CTA of W warps for NF fields
__host__ __device__ inline size_t anal_smem_bytes(int W, int NF) {
    return (size_t)W * 32 * kAnalPad * sizeof(double) +             // per-warp transpose
           (size_t)2 * W * (2 * NF * kAnalStage) * sizeof(double);  // per-warp stage sums x2
}

// one degree step for T ring pairs and NF fields: the lane's sums over its
// pairs of P * G, G the symmetric (even l-m) or antisymmetric (odd)
// combination of the two rings of each pair
template <int T, int NF>
__device__ __forceinline__ void anal_step(bool odd, double2 fr, const double* z,
                                          double* q1, double* q2,
                                          const double (*gsR)[NF], const double (*gsI)[NF],
                                          const double (*gaR)[NF], const double (*gaI)[NF],
                                          double* accR, double* accI) {
    double p[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        p[t] = rec_step(z[t], fr, q1[t], q2[t]);
        q2[t] = q1[t];
        q1[t] = p[t];
    }
#pragma unroll
    for (int j = 0; j < NF; ++j) {
        double r = 0.0, i = 0.0;
#pragma unroll
        for (int t = 0; t < T; ++t) {
            r = fma(p[t], odd ? gaR[t][j] : gsR[t][j], r);
            i = fma(p[t], odd ? gaI[t][j] : gsI[t][j], i);
        }
        accR[j] = r;
        accI[j] = i;
    }
}

// Analysis of order m for the ring pairs of tile `tile` and the fields
// f0 .. f0+nvalid-1 (nvalid <= NF):
//   sp:   spec of field f0, [pair][m][ring]; field j at sp + j*sstride
//   outp: the tile's packed {C, S} sums of field f0, [packed (l, m)];
//         field j at outp + j*ostride
// smem: anal_smem_bytes(W, NF) bytes, 16-byte aligned; rstage: 2 x kAnalStage staged
// {beta, D}.  Degrees go in stages of kAnalStage (one CTA barrier each),
// each stage in transpose chunks of kAnalChunk/NF degrees (warp-local); the
// recursion is rescaled at the first step of every chunk that starts a
// segment.
// Ends with the tile's sums written by warp 0 after a barrier; the caller
// must pass another barrier before reusing the shared memory.
template <int T, int NF>
__device__ __forceinline__ void anal_order(
    double* smem, double2 (*rstage)[kAnalStage], const double2* __restrict__ rec,
    const double* __restrict__ pmm, const double* __restrict__ rtab,
    const double* __restrict__ zp, const double2* __restrict__ sp, long long sstride,
    double2* __restrict__ outp, long long ostride, int lc, int npair, int m, int tile,
    int nvalid) {
    constexpr int CH = anal_chunk(NF);
    constexpr int SROWS = 2 * NF * kAnalStage;   // (field, Re/Im, degree) rows per stage
    static_assert(2 * NF * CH == 32, "one transpose row per lane");
    const int nwarps = blockDim.x >> 5;
    const int warp = threadIdx.x >> 5;
    const int lane = threadIdx.x & 31;
    double* tb = smem + warp * (32 * kAnalPad);
    // two buffers of per-warp stage sums, alternating between stages
    double* wsum = smem + nwarps * (32 * kAnalPad);   // [2][nwarps][SROWS]

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
    const int nstages = (nsteps + kAnalStage - 1) / kAnalStage;
    // the first warp copies a stage: kAnalStage = 32 entries, one per lane
    static_assert(kAnalStage == 32, "one stage entry per lane of a warp");
    auto load_stage = [&](int c) {
        const int sidx = c * kAnalStage + threadIdx.x;
        if (threadIdx.x < kAnalStage && sidx < nsteps)
            cp_async16(&rstage[c & 1][threadIdx.x], &rm[sidx]);
        cp_async_commit();
    };
    load_stage(0);
    if (nstages > 1) load_stage(1);

    const double start = pmm[m];
    // symmetric (l-m even) and antisymmetric (l-m odd) combinations
    double gsR[T][NF], gsI[T][NF], gaR[T][NF], gaI[T][NF], q1[T], q2[T];
#pragma unroll
    for (int t = 0; t < T; ++t) {
        const double r = pv[t] < npair ? rtab[(long long)m * npair + pv[t]] : 0.0;
#pragma unroll
        for (int j = 0; j < NF; ++j) {
            gsR[t][j] = gsI[t][j] = gaR[t][j] = gaI[t][j] = 0.0;
            if (j < nvalid && r != 0.0) {
                const double2* x = sp + j * sstride + ((long long)pv[t] * (lc + 1) + m) * 2;
                const double2 a = x[0];
                const double2 b = x[1];
                const double aR = a.x * r, aI = a.y * r;
                const double bR = b.x * r, bI = b.y * r;
                gsR[t][j] = aR + bR; gsI[t][j] = aI + bI;
                gaR[t][j] = aR - bR; gaI[t][j] = aI - bI;
            }
        }
        // the step s = 0 of the table (beta = -1) turns this into Q(0) = start
        q1[t] = 0.0;
        q2[t] = start;
    }
    if (nstages > 1) cp_async_wait<1>(); else cp_async_wait<0>();
    __syncthreads();
    int buf = 0;
    for (int sg = 0; sg < nstages; ++sg) {
        const int s0 = sg * kAnalStage;
        const double2* stg = rstage[sg & 1];
        double* ws = wsum + (buf * nwarps + warp) * SROWS;
        // a chunk whose first degree is a multiple of kRecSegment starts by
        // ending a recursion segment (D(0) = 1 for the first one)
#pragma unroll 1
        for (int ci = 0; ci < kAnalStage / CH; ++ci) {
            const int c0 = s0 + ci * CH;
            const int cn = min(CH, nsteps - c0);
            if (cn <= 0) break;
            const double2* wcoef = stg + ci * CH;
            double accR[NF], accI[NF];
            // parity of s = c0 + k is that of k (c0 even)
            if (cn == CH) {
#pragma unroll
                for (int k = 0; k < CH; ++k) {
                    anal_step<T, NF>((k & 1) != 0, wcoef[k], z, q1, q2, gsR, gsI, gaR, gaI,
                                     accR, accI);
                    if (k == 0 && ci % NF == 0) rec_rescale<T>(wcoef[0].y, q1, q2);
#pragma unroll
                    for (int j = 0; j < NF; ++j) {
                        tb[((2 * j + 0) * CH + k) * kAnalPad + lane] = accR[j];
                        tb[((2 * j + 1) * CH + k) * kAnalPad + lane] = accI[j];
                    }
                }
            } else {
                for (int k = 0; k < cn; ++k) {
                    anal_step<T, NF>((k & 1) != 0, wcoef[k], z, q1, q2, gsR, gsI, gaR, gaI,
                                     accR, accI);
                    if (k == 0 && ci % NF == 0) rec_rescale<T>(wcoef[0].y, q1, q2);
#pragma unroll
                    for (int j = 0; j < NF; ++j) {
                        tb[((2 * j + 0) * CH + k) * kAnalPad + lane] = accR[j];
                        tb[((2 * j + 1) * CH + k) * kAnalPad + lane] = accI[j];
                    }
                }
            }
            __syncwarp();
            // row = lane = (2*field + Re/Im)*CH + degree: sum over the 32
            // lanes of the warp, four interleaved partial sums
            {
                const int k = lane % CH;
                const double* b = tb + lane * kAnalPad;
                double sum = 0.0;
                if (k < cn) {
                    // element q of the row goes to partial sum q % 4
                    double s4[4] = {0.0, 0.0, 0.0, 0.0};
                    const double2* b2 = reinterpret_cast<const double2*>(b);
#pragma unroll
                    for (int q = 0; q < 16; ++q) {
                        const double2 v = b2[q];
                        s4[(2 * q) & 3] += v.x;
                        s4[(2 * q + 1) & 3] += v.y;
                    }
                    sum = ((s4[0] + s4[1]) + (s4[2] + s4[3])) * wcoef[k].y;   // Q -> P sums
                }
                // stage row layout: (2*field + Re/Im)*kAnalStage + degree in stage
                ws[(lane / CH) * kAnalStage + ci * CH + k] = sum;
            }
            __syncwarp();
        }
        // stage sums of all warps are in wsum[buf]; the next stage's {beta, D}
        // were issued a stage ahead
        if (sg + 1 < nstages) cp_async_wait<0>();
        __syncthreads();
        if (sg + 2 < nstages) load_stage(sg + 2);
        if (warp == 0) {
            const int sn = min(kAnalStage, nsteps - s0);
#pragma unroll
            for (int i = 0; i < SROWS / 32; ++i) {
                const int r = lane + 32 * i;
                const int k = r % kAnalStage;
                const int fc = r / kAnalStage;   // 2*field + Re/Im
                double sum = 0.0;
                for (int w = 0; w < nwarps; ++w) sum += wsum[(buf * nwarps + w) * SROWS + r];
                if (k < sn && (fc >> 1) < nvalid) {
                    double* dst = reinterpret_cast<double*>(outp + (fc >> 1) * ostride + o +
                                                            s0 + k);
                    dst[fc & 1] = sum;
                }
            }
        }
        buf ^= 1;
    }
}

}  // namespace shtc
