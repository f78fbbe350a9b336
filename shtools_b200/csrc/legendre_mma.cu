// Multi-field Legendre analysis on the FP64 tensor path (mma.sync m8n8k4
// f64; tcgen05 has no FP64 kind).
//
// For one order m and a tile of ring pairs the analysis of F fields is a
// matrix product: C[l][n] = sum_p P(l, p) G_par(l)[p][n], n = (field,
// Re/Im), G the symmetric (l - m even) or antisymmetric (odd) combination of
// the pair's two rings times the ring weight (SHExpandDH.f95:463-580,
// SHExpandGLQ.f95:445-649).  The scalar kernel (legendre.cuh, anal_order)
// runs the recursion once per group of at most four fields and reduces every
// degree across the lanes; here each lane runs the recursion for one pair,
// once for all the fields of the CTA, writes its 16 values of a recursion
// segment to shared memory, and the warp multiplies them by the pair
// combinations held in registers as B fragments:
//   A (8 x 4): 8 degrees of one parity x 4 pairs, read from shared memory;
//   B (4 x 8): 4 pairs x 8 columns, G_sym or G_anti;
//   C (8 x 8): degrees x columns, accumulated over the warp's 32 pairs.
// Each warp keeps two A tiles: while the products of one 16-degree stage
// issue, the lane's recursion writes the next stage's values into the other
// tile (8% faster on B200 than recursion, then products).  The warps'
// partial sums (scaled by the segment's D(s)) meet in shared memory, stored
// as 16-byte pairs in rows padded to avoid bank conflicts, and are added in
// warp order (deterministic), giving the tile's partial sums in the layout
// of the scalar kernel: partial[tile][field][packed (l, m)] as (Re, Im).
//
// The synthesis has no such kernel: written the same way (the coefficient
// rows as shared B fragments, 32 pairs x 16 columns accumulated per warp)
// it ran 4% slower on B200 than the scalar synthesis with 8 fields per
// recursion (16 fields at lmax 2799: 37.6 against 36.2 ms).  The FP64
// tensor path issues multiply-adds at the FP64 pipe's rate, and the scalar
// synthesis has no cross-lane reduction to remove.
#include <cuda_runtime.h>

#include "legendre.cuh"
#include "shtc_internal.cuh"

namespace shtc {

constexpr int kMmaWarps = 8;                    // warps per CTA, 32 ring pairs each
constexpr int kMmaPitch = 34;                   // doubles per degree row of a warp's
                                                // recursion values: conflict-free A loads

// d (8 x 8, 2 per lane) += a (8 x 4, 1 per lane) * b (4 x 8, 1 per lane); not
// volatile, so the compiler may interleave it with the recursion
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
    asm("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0, %1}, {%2}, {%3}, {%0, %1};\n"
        : "+d"(d[0]), "+d"(d[1])
        : "d"(a), "d"(b));
}

// row pitch (doubles) of a warp's partial sums for NT column tiles: 8 NT + 4,
// so the 16-byte stores of a quarter warp (rows 2g, g = 0, 1) hit 8
// distinct 16-byte bank groups
__host__ __device__ constexpr int mma_sum_pitch(int NT) { return 8 * NT + 4; }

// shared memory of a CTA for NT column tiles (8 columns each)
__host__ __device__ constexpr size_t anal_mma_smem(int NT) {
    return sizeof(double) * ((size_t)2 * kMmaWarps * kAnalChunk * kMmaPitch +  // A tiles x2
                             (size_t)2 * kMmaWarps * kAnalChunk * mma_sum_pitch(NT));  // sums x2
}

// CTA = (tile of 32 * kMmaWarps ring pairs, order m, group of 4 NT fields)
template <int NT>
__global__ void __launch_bounds__(32 * kMmaWarps, NT <= 2 ? 2 : 1)
k_legendre_anal_mma(const double2* __restrict__ rec, const double* __restrict__ pmm,
                    const double* __restrict__ rtab, const double* __restrict__ zp,
                    const double2* __restrict__ spec, double2* __restrict__ partial, int lc,
                    int npair, long long nlm, int nfield) {
    constexpr int NC = 8 * NT;                  // columns: (field, Re/Im)
    constexpr int FG = NC / 2;                  // fields per CTA
    constexpr int WP = mma_sum_pitch(NT);
    constexpr int TILE = kAnalChunk * kMmaPitch;   // one A tile (16 degrees x 32 pairs)
    extern __shared__ __align__(16) double smem_mma[];
    __shared__ __align__(16) double2 rstage[3][kAnalChunk];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane >> 2, t = lane & 3;      // fragment row group, thread in group
    const int m = blockIdx.y, tile = blockIdx.x, f0 = blockIdx.z * FG;
    const int nvalid = min(FG, nfield - f0);
    const int pbase = tile * 32 * kMmaWarps + warp * 32;
    double* pwb = smem_mma + warp * (2 * TILE);                  // two A tiles per warp
    double* wsum = smem_mma + kMmaWarps * 2 * TILE;              // [2][warps][16][WP]

    const long long o = packed_off(m, lc);
    const double2* __restrict__ rm = rec + o;
    const int nsteps = lc - m + 1;
    const int nstages = (nsteps + kAnalChunk - 1) / kAnalChunk;
    // {beta, D} of stage c into rstage[c % 3], issued three stages ahead
    auto load_stage = [&](int c) {
        const int sidx = c * kAnalChunk + threadIdx.x;
        if (threadIdx.x < kAnalChunk && sidx < nsteps)
            cp_async16(&rstage[c % 3][threadIdx.x], &rm[sidx]);
        cp_async_commit();
    };
    load_stage(0);
    load_stage(1);
    load_stage(2);

    // B fragments: K-step s covers pairs pbase + 4s .. +3; this lane holds
    // pair pbase + 4s + t, column 8j + g = (field (8j + g) / 2, Re/Im)
    double bs[8][NT], ba[8][NT];
#pragma unroll
    for (int s = 0; s < 8; ++s) {
        const int kp = pbase + 4 * s + t;
        const double r = kp < npair ? rtab[(long long)m * npair + kp] : 0.0;
#pragma unroll
        for (int j = 0; j < NT; ++j) {
            const int n = 8 * j + g, f = n >> 1;
            double vs = 0.0, va = 0.0;
            if (f < nvalid && r != 0.0) {
                const double2* x =
                    spec + ((((long long)(f0 + f) * npair + kp) * (lc + 1)) + m) * 2;
                const double2 a = x[0], b = x[1];
                const double aR = ((n & 1) ? a.y : a.x) * r;
                const double bR = ((n & 1) ? b.y : b.x) * r;
                vs = aR + bR;
                va = aR - bR;
            }
            bs[s][j] = vs;
            ba[s][j] = va;
        }
    }
    // this lane's recursion: pair pbase + lane; step s = 0 of the table
    // (beta = -1) turns q1 = 0, q2 = start into Q(0) = start
    const int p = pbase + lane;
    const double z = p < npair ? zp[p] : 0.0;
    double q1 = 0.0, q2 = pmm[m];
    // degree k of a stage (k = 0 starts a recursion segment: back to P units)
    auto rec_k = [&](const double2* stg, int k, double* pwt) {
        const double pv = rec_step(z, stg[k], q1, q2);
        q2 = q1;
        q1 = pv;
        if (k == 0) {
            q1 *= stg[0].y;
            q2 *= stg[0].y;
        }
        pwt[k * kMmaPitch + lane] = pv;
    };
    // a stage of cn < 16 degrees: zero beyond the last
    auto rec_partial = [&](const double2* stg, int cn, double* pwt) {
#pragma unroll
        for (int k = 0; k < kAnalChunk; ++k) {
            if (k < cn) rec_k(stg, k, pwt);
            else pwt[k * kMmaPitch + lane] = 0.0;
        }
    };

    cp_async_wait<1>();                         // stages 0 and 1
    __syncthreads();
    {
        const int cn0 = min(kAnalChunk, nsteps);
        if (cn0 == kAnalChunk) {
#pragma unroll
            for (int k = 0; k < kAnalChunk; ++k) rec_k(rstage[0], k, pwb);
        } else {
            rec_partial(rstage[0], cn0, pwb);
        }
    }
    __syncwarp();
    int buf = 0;
    for (int sg = 0; sg < nstages; ++sg) {
        const int s0 = sg * kAnalChunk;
        const int cn = min(kAnalChunk, nsteps - s0);
        const int cnn = sg + 1 < nstages ? min(kAnalChunk, nsteps - s0 - kAnalChunk) : 0;
        const double* cur = pwb + (sg & 1) * TILE;
        double* nxt = pwb + ((sg + 1) & 1) * TILE;
        const double2* stn = rstage[(sg + 1) % 3];
        // degrees s0 + 2i (l - m even: G_sym) and s0 + 2i + 1 (odd: G_anti);
        // the next stage's recursion runs between the products
        double ce[NT][2], co[NT][2];
#pragma unroll
        for (int j = 0; j < NT; ++j) ce[j][0] = ce[j][1] = co[j][0] = co[j][1] = 0.0;
        auto mma_s = [&](int s) {
            const double ae = cur[(2 * g) * kMmaPitch + 4 * s + t];
            const double ao = cur[(2 * g + 1) * kMmaPitch + 4 * s + t];
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                dmma(ce[j], ae, bs[s][j]);
                dmma(co[j], ao, ba[s][j]);
            }
        };
        if (cnn == kAnalChunk) {
#pragma unroll
            for (int s = 0; s < 8; ++s) {
                mma_s(s);
                rec_k(stn, 2 * s, nxt);
                rec_k(stn, 2 * s + 1, nxt);
            }
        } else {
#pragma unroll
            for (int s = 0; s < 8; ++s) mma_s(s);
            if (cnn > 0) rec_partial(stn, cnn, nxt);
        }
        // warp partials in P units (times D(s)), rows 2g and 2g + 1 of the stage
        {
            const double2* stg = rstage[sg % 3];
            const double de = stg[2 * g].y, dd = stg[2 * g + 1].y;
            double* ws = wsum + (buf * kMmaWarps + warp) * (kAnalChunk * WP);
#pragma unroll
            for (int j = 0; j < NT; ++j) {
                *reinterpret_cast<double2*>(&ws[(2 * g) * WP + 8 * j + 2 * t]) =
                    make_double2(ce[j][0] * de, ce[j][1] * de);
                *reinterpret_cast<double2*>(&ws[(2 * g + 1) * WP + 8 * j + 2 * t]) =
                    make_double2(co[j][0] * dd, co[j][1] * dd);
            }
        }
        // all warps' partials are in wsum[buf] and every lane's next A tile
        // is written; stage sg + 2 has landed; stage sg's buffer is free for
        // stage sg + 3
        cp_async_wait<0>();
        __syncthreads();
        if (sg + 3 < nstages) load_stage(sg + 3);
        for (int idx = threadIdx.x; idx < kAnalChunk * NC; idx += blockDim.x) {
            const int k = idx / NC, n = idx - k * NC, f = n >> 1;
            if (k >= cn || f >= nvalid) continue;
            double sum = 0.0;
            for (int w = 0; w < kMmaWarps; ++w)
                sum += wsum[(buf * kMmaWarps + w) * (kAnalChunk * WP) + k * WP + n];
            double* dst = reinterpret_cast<double*>(
                partial + ((long long)tile * nfield + f0 + f) * nlm + o + s0 + k);
            dst[n & 1] = sum;
        }
        buf ^= 1;
    }
}

template <int NT>
static int launch_mma_t(const shtc_plan* P, const double2* spec, double2* partial,
                        int ntiles, int nfield, cudaStream_t st) {
    constexpr size_t smem = anal_mma_smem(NT);
    static_assert(smem <= 200 * 1024, "shared memory of the tensor analysis");
    // two CTAs of 110 KB per SM: the whole carveout
    const int rc = kernel_smem_attr((const void*)k_legendre_anal_mma<NT>, smem, true);
    if (rc) return rc;
    dim3 grid(ntiles, P->lc + 1, (nfield + 4 * NT - 1) / (4 * NT));
    k_legendre_anal_mma<NT><<<grid, 32 * kMmaWarps, smem, st>>>(
        P->d_rec, P->d_pmm, P->d_rtab, P->d_z, spec, partial, P->lc, P->npair, P->nlm,
        nfield);
    return map_cuda(cudaGetLastError());
}

int anal_mma_pairs() { return 32 * kMmaWarps; }

// 8 fields per CTA (NT = 2: 126 registers, two CTAs per SM); 16 per CTA
// (NT = 4: 208 registers, one CTA) measured slower on B200 for 16 fields,
// before the recursion overlapped the products (lmax 2799: 43.2 against
// 40.4 ms; 8 complex fields at lmax 719: 1.08 against 0.90 ms), the
// recursion run twice notwithstanding
int launch_legendre_anal_mma(const shtc_plan* P, const double2* spec, double2* partial,
                             int ntiles, int nfield, cudaStream_t st) {
    return launch_mma_t<2>(P, spec, partial, ntiles, nfield, st);
}

}  // namespace shtc
