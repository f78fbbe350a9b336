// Legendre synthesis on the 5th-generation tensor cores (tcgen05, kind::i8)
// with an error-free split of the FP64 operands (Ozaki scheme).
//
// For one order m and a tile of 128 ring pairs the synthesis of F fields is
// a matrix product over the degrees (MakeGridDH.f95:566-612,
// MakeGridGLQ.f95:604-650):
//     E[p][n] = sum_{l - m even} P_lm(z_p) C[l][n],
//     O[p][n] = sum_{l - m odd}  P_lm(z_p) C[l][n],
// n = (field, cos/sin); the north ring takes E + O, the south ring E - O.
//
// Both operands become fixed-point integers written with DA (P_lm) and DB
// (coefficients) balanced base-256 digits d_i in [-128, 127] (the bytes of
// X + 0x80...80 with their top bit flipped):
//   A[p][l] = round(P_lm(z_p) 2^a),   one exponent a per plan, from the bound
//             |P_lm| <= sqrt(2l+1) of the 4pi functions (Schmidt: 1,
//             orthonormal: sqrt((2l+1)/4pi)); |A| < 2^(8 DA - 10);
//   B[l][n] = round(C[l][n] 2^b(m,n)), one exponent per (order, column) from
//             max_l |C[l][n]|;                  |B| < 2^(8 DB - 10).
// The products of digits i (of A) and j (of B) are summed exactly in INT32
// per weight w = i + j - (DA + DB - 1 - KW), for the KW highest weights; the
// dropped lower products are below 2^-8 of the last kept weight each and,
// the digits being balanced, have no systematic sign.  The epilogue combines
// the weights in 64-bit integers and FP64 and scales by 2^-(a+b).
// Precisions (shtc_plan_set_precision): INT8X6 = 6 x 6 digits, 7 weights;
// INT8X7 = 7 x 7 digits, 8 weights.  Per-degree errors against the FP64
// path are stated by the tests.
//
// One MMA per (A digit i, parity): B is the window of KW coefficient digits
// j = top - KW + 1 - i .. top - i of a shared-memory stack in which each
// parity's DB digit tiles sit between zero tiles, so the N' = KW x N
// columns of the MMA land on the KW weight blocks of that parity's
// accumulator.
//
// The P_lm recursion stays in FP64 (the rescaled recursion of legendre.cuh).
// Eight producer warps: warps w and w + 4 own the same 32 TMEM lanes (ring
// pairs); both run the pair's recursion (two FP64 operations per degree),
// warp w turns the even degrees (l - m) into fixed point and digits, warp
// w + 4 the odd ones, and each stores its parity's digit words of a 64-degree
// K-tile to tensor memory (A operand, K-major: lane = pair, K = degree).  A
// ninth warp issues the MMAs with B from shared memory, filled by bulk copies
// from a global image of the coefficient digits prepared per call
// (k_i8_coef_image), and the A operand is double-buffered so that the
// producers fill one buffer while the MMAs read the other.
//
// Tensor memory per CTA (N = 16 columns = 2 x 8 fields of a group):
//   D: [parity][weight] x N columns of INT32 accumulators (2 KW N)
//   A: 2 buffers x [parity][digit] x 8 columns (32 degrees of 8 bits)
//
// Every wait on an mbarrier is bounded; on a timeout the CTA records
// SHTC_ETIMEOUT in the error word, stops issuing work, waits (bounded) for
// its own copies and MMAs in flight and frees its tensor memory.
#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "legendre.cuh"
#include "shtc_internal.cuh"

namespace shtc {
namespace i8 {

constexpr int kPairs = 128;          // ring pairs per CTA (TMEM lanes, MMA M)
constexpr int kTileDeg = 64;         // degrees per K-tile (32 of each parity)
constexpr int kStages = 8;           // B / recursion-table stages in shared memory
constexpr int kProducers = 256;      // eight producer warps
constexpr int kThreads = kProducers + 64;   // + MMA warp + stage-loader warp
constexpr unsigned kSpinLimit = 1u << 22;   // bounded mbarrier waits (seconds)
constexpr int kTmemAlloc = 512;

// digits, kept weights and fixed-point bits of a precision
template <int D> struct Digits;
// kBitsA / kBitsB: |A| < 2^kBitsA (P_lm: the rounding trick of tile_digits
// keeps it below 2^51), |B| < 2^kBitsB (coefficients)
template <> struct Digits<6> {
    static constexpr int KW = 7;                        // weights kept
    static constexpr int kBitsA = 46, kBitsB = 46;
    static constexpr long long kBalance = 0x808080808080LL;
};
template <> struct Digits<7> {
    static constexpr int KW = 8;
    static constexpr int kBitsA = 50, kBitsB = 54;
    static constexpr long long kBalance = 0x80808080808080LL;
};

// bytes of one B tile (N columns x 32 degrees of one parity) and of the
// 2 DB tiles of a K-tile in the global image ([parity][digit])
__host__ __device__ constexpr int btile_bytes(int N) { return N * 32; }
__host__ __device__ constexpr int bimage_bytes(int N, int DB) { return 2 * DB * btile_bytes(N); }
// shared-memory stack of one parity: KW - DB zero tiles, the DB digit
// tiles, DA - 1 zero tiles
__host__ __device__ constexpr int bstack_tiles(int DA, int DB, int KW) { return DA + KW - 1; }
constexpr int kRecBytes = kTileDeg * 32;   // 64 x {gamma, delta, D, 0}
__host__ __device__ constexpr int stage_bytes(int N, int DA, int DB, int KW) {
    return 2 * bstack_tiles(DA, DB, KW) * btile_bytes(N) + kRecBytes;
}
__host__ __device__ constexpr int tmem_cols_d(int N, int KW) { return 2 * KW * N; }
__host__ __device__ constexpr int tmem_cols_a(int DA) { return 2 * DA * 8; }

// 2^e as a compile-time constant
__host__ __device__ constexpr double pow2i(int e) {
    return e == 0 ? 1.0 : (e > 0 ? 2.0 * pow2i(e - 1) : 0.5 * pow2i(e + 1));
}

__host__ __device__ inline int ntiles_of(int lc, int m) {
    return (lc - m + 1 + kTileDeg - 1) / kTileDeg;
}

// ------------------------------------------------------------------ PTX
__device__ __forceinline__ uint32_t smem_u32(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}

// tcgen05 shared-memory matrix descriptor, no swizzle: start address, LBO
// (byte distance of the two 16-byte K chunks), SBO (of 8-row groups),
// version 1
__device__ __forceinline__ uint64_t smem_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((saddr >> 4) & 0x3FFF) | ((uint64_t)((lbo >> 4) & 0x3FFF) << 16) |
           ((uint64_t)((sbo >> 4) & 0x3FFF) << 32) | ((uint64_t)1 << 46);
}

// instruction descriptor of kind::i8: D = S32, A/B u8 or s8, both K-major
__host__ __device__ constexpr uint32_t idesc_i8(int M, int N, int a_signed, int b_signed) {
    return (2u << 4) | ((uint32_t)a_signed << 7) | ((uint32_t)b_signed << 10) |
           ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* b) {
    asm volatile("{\n\t.reg .b64 st;\n\tmbarrier.arrive.shared::cta.b64 st, [%0];\n\t}" ::"r"(
                     smem_u32(b))
                 : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* b, uint32_t bytes) {
    asm volatile(
        "{\n\t.reg .b64 st;\n\tmbarrier.arrive.expect_tx.shared::cta.b64 st, [%0], %1;\n\t}" ::"r"(
            smem_u32(b)),
        "r"(bytes)
        : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
// error word of the tensor-core kernels on this device: 0, or SHTC_ETIMEOUT
// after a bounded wait ran out (read and cleared by shtc_mixed_status)
__device__ int g_i8_status;

__device__ __forceinline__ void raise_timeout(volatile int* abort_flag) {
    *abort_flag = 1;
    atomicExch(&g_i8_status, SHTC_ETIMEOUT);
}

__device__ __forceinline__ bool mbar_test(uint64_t* b, uint32_t parity) {
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred P1;\n\tmbarrier.test_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
constexpr unsigned long long kWaitNs = 2000000000ull;   // a wait gives up after 2 s

// bounded wait: false on a timeout or when another thread raised the abort
// flag.  Polls with test_wait first (no suspension when the phase is about
// to complete), then suspends in try_wait; every 256 tries it checks the
// abort flag and the 2-second deadline, so the bound does not depend on how
// long one try_wait may suspend.
__device__ __forceinline__ bool mbar_wait(uint64_t* b, uint32_t parity, volatile int* abort_flag) {
    for (int it = 0; it < 64; ++it)
        if (mbar_test(b, parity)) return true;
    const unsigned long long t0 = global_ns();
    for (unsigned it = 0; it < kSpinLimit; ++it) {
        if (mbar_try(b, parity)) return true;
        if ((it & 255) == 255) {
            if (*abort_flag) return false;
            if (global_ns() - t0 > kWaitNs) break;
        }
    }
    raise_timeout(abort_flag);
    return false;
}

// 1-D bulk copy global -> shared, completion on an mbarrier (no multicast)
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(b))
        : "memory");
}

// true in one lane of the (converged) warp
__device__ __forceinline__ bool elect_one() {
    uint32_t pred;
    asm volatile(
        "{\n\t.reg .pred p;\n\telect.sync _|p, 0xffffffff;\n\tselp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(pred));
    return pred != 0;
}

__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_commit(uint64_t* b) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(b))
                 : "memory");
}
// D (tmem) += A (tmem) x B (smem descriptor); acc = 0 overwrites D
__device__ __forceinline__ void mma_ts(uint32_t d, uint32_t a, uint64_t bdesc, uint32_t idesc,
                                       uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], [%1], %2, %3, p;\n\t}" ::"r"(d),
        "r"(a), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// --------------------------------------------------------------------------
// coefficient image: per (order m, field group g) the K-tiles of the B
// operand, tile (t, parity q, digit j) = N columns x 32 degrees of one
// parity (s = 64 t + 2 k + q) in the K-major core-matrix layout of the MMA
// (column n, degree k at (n % 8) * 16 + (n / 8) * 256 + (k / 16) * 128 +
// k % 16), byte = balanced digit j of round(C 2^b(m, n)).
// colinv[(m * ngroups + g) * N + n] = 2^-b(m, n).  coef: packed {C, S}
// without the recursion's D factor, [packed (l, m)][nfield].
// --------------------------------------------------------------------------
template <int N, int DB>
__global__ void __launch_bounds__(256)
k_i8_coef_image(const double2* __restrict__ coef, uint32_t* __restrict__ image,
                const long long* __restrict__ toff, double* __restrict__ colinv, int lc,
                int nfield, int ngroups) {
    constexpr int NFG = N / 2;
    constexpr int kBits = Digits<DB>::kBitsB;
    const int m = blockIdx.x, g = blockIdx.y;
    const int nsteps = lc - m + 1;
    const int nt = ntiles_of(lc, m);
    const long long o = packed_off(m, lc);
    __shared__ unsigned long long cmax[N];
    __shared__ double cscale[N];
    for (int n = threadIdx.x; n < N; n += blockDim.x) cmax[n] = 0ull;
    __syncthreads();
    // column maxima over the degrees (non-negative doubles order as integers)
    for (int idx = threadIdx.x; idx < nsteps * NFG; idx += blockDim.x) {
        const int s = idx / NFG, f = idx - s * NFG;
        const int fg = g * NFG + f;
        if (fg >= nfield) continue;
        const double2 c = coef[(o + s) * nfield + fg];
        atomicMax(&cmax[2 * f], (unsigned long long)__double_as_longlong(fabs(c.x)));
        atomicMax(&cmax[2 * f + 1], (unsigned long long)__double_as_longlong(fabs(c.y)));
    }
    __syncthreads();
    for (int n = threadIdx.x; n < N; n += blockDim.x) {
        const double mx = __longlong_as_double((long long)cmax[n]);
        double sc = 0.0, inv = 0.0;
        if (mx > 0.0) {
            int e;
            frexp(mx, &e);                   // mx < 2^e
            sc = ldexp(1.0, kBits - e);      // |C| sc < 2^kBits
            inv = ldexp(1.0, e - kBits);
        }
        cscale[n] = sc;
        colinv[((long long)m * ngroups + g) * N + n] = inv;
    }
    __syncthreads();
    // one thread per (tile, parity, word): 4 degrees of one column, DB words
    constexpr int WPT = btile_bytes(N) / 4;      // words per tile
    uint32_t* base = image + (toff[m] * ngroups + (long long)g * nt) * (bimage_bytes(N, DB) / 4);
    for (int idx = threadIdx.x; idx < nt * 2 * WPT; idx += blockDim.x) {
        const int wi = idx % WPT, tq = idx / WPT, t = tq >> 1, q = tq & 1;
        const int k4lo = wi & 3, n8 = (wi >> 2) & 7, k4hi = (wi >> 5) & 1, ng = wi >> 6;
        const int n = ng * 8 + n8, k4 = k4hi * 4 + k4lo;
        const int f = n >> 1, fg = g * NFG + f;
        uint32_t w[DB];
#pragma unroll
        for (int j = 0; j < DB; ++j) w[j] = 0u;
#pragma unroll
        for (int u = 0; u < 4; ++u) {
            const int s = kTileDeg * t + 2 * (4 * k4 + u) + q;
            long long x = 0;
            if (s < nsteps && fg < nfield) {
                const double2 c = coef[(o + s) * nfield + fg];
                x = __double2ll_rn(((n & 1) ? c.y : c.x) * cscale[n]);
            }
            x += Digits<DB>::kBalance;   // balanced digits: bytes of X + 0x80..80, top bit flipped
#pragma unroll
            for (int j = 0; j < DB; ++j)
                w[j] |= (uint32_t)(((x >> (8 * j)) & 0xFF) ^ 0x80) << (8 * u);
        }
        uint32_t* tb = base + (long long)(t * 2 + q) * DB * WPT;
#pragma unroll
        for (int j = 0; j < DB; ++j) tb[j * WPT + wi] = w[j];
    }
}

// --------------------------------------------------------------------------
// tensor memory stores and loads of one warp (32 lanes x 32-bit columns)
// --------------------------------------------------------------------------
__device__ __forceinline__ void tmem_st8(uint32_t taddr, const uint32_t* w) {
    asm volatile(
        "tcgen05.st.sync.aligned.32x32b.x8.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8};" ::"r"(taddr),
        "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3]), "r"(w[4]), "r"(w[5]), "r"(w[6]), "r"(w[7])
        : "memory");
}
__device__ __forceinline__ void tmem_st4(uint32_t taddr, const uint32_t* w) {
    asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(taddr),
                 "r"(w[0]), "r"(w[1]), "r"(w[2]), "r"(w[3])
                 : "memory");
}
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t* v) {
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
        : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
          "=r"(v[7])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_ld2(uint32_t taddr, uint32_t* v) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0, %1}, [%2];"
                 : "=r"(v[0]), "=r"(v[1])
                 : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_st() {
    asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_wait_ld() {
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// digit words of four values: byte u of word i = digit i of value u
// (top bit of every byte flipped: balanced digits); lo/hi: the two 32-bit
// halves of X + kBalance of the four values
template <int DA>
__device__ __forceinline__ void pack4(const uint32_t* lo, const uint32_t* hi, uint32_t* w) {
    const uint32_t t0 = __byte_perm(lo[0], lo[1], 0x5140), t1 = __byte_perm(lo[2], lo[3], 0x5140);
    const uint32_t t2 = __byte_perm(lo[0], lo[1], 0x7362), t3 = __byte_perm(lo[2], lo[3], 0x7362);
    w[0] = __byte_perm(t0, t1, 0x5410) ^ 0x80808080u;
    w[1] = __byte_perm(t0, t1, 0x7632) ^ 0x80808080u;
    w[2] = __byte_perm(t2, t3, 0x5410) ^ 0x80808080u;
    w[3] = __byte_perm(t2, t3, 0x7632) ^ 0x80808080u;
    const uint32_t u0 = __byte_perm(hi[0], hi[1], 0x5140), u1 = __byte_perm(hi[2], hi[3], 0x5140);
    w[4] = __byte_perm(u0, u1, 0x5410) ^ 0x80808080u;
    w[5] = __byte_perm(u0, u1, 0x7632) ^ 0x80808080u;
    if constexpr (DA == 7) {
        const uint32_t u2 = __byte_perm(hi[0], hi[1], 0x7362), u3 = __byte_perm(hi[2], hi[3], 0x7362);
        w[6] = __byte_perm(u2, u3, 0x5410) ^ 0x80808080u;
    }
}

struct SynthArgs {
    const double4* rec2;     // plan {gamma, delta, D, 0} per packed (l, m)
    const double* pmm;       // sectoral start values
    const double* rtab;      // u^m / 1e-280 per (m, pair)
    const double* zp;        // z of the northern ring of each pair
    const uint8_t* image;    // coefficient image (k_i8_coef_image)
    const long long* toff;   // K-tiles before order m
    const double* colinv;    // 2^-b per (m, group, column)
    double2* spec;           // c2r inputs [field][pair][m][ring]
    int lc, npair, nfield, ngroups, ptiles;
    double ascale;           // 2^a: the A operand's fixed-point scale
};

// work item -> (m, field group, pair tile); m slowest, so the longest items
// go first
__device__ __forceinline__ void item_decode(long long i, int ptiles, int ngroups, int* m,
                                            int* g, int* tile) {
    const long long per_m = (long long)ptiles * ngroups;
    *m = (int)(i / per_m);
    const int r = (int)(i - (long long)(*m) * per_m);
    *g = r / ptiles;
    *tile = r - (*g) * ptiles;
}

// One 64-degree K-tile of a producer thread: advances the chain of the
// pair's recursion values of parity QR (degrees s = 64 t + j, j % 2 = QR)
// by 32 steps of the same-parity two-step form of the rescaled recursion
//     Q(r) = (z^2 - gamma(r)) Q(r-2) - delta(r) Q(r-4),
//     gamma(r) = beta(r-1) + beta(r),  delta(r) = beta(r-1) beta(r-2)
// (recs[j] = {gamma, delta, D, 0}), and writes the digit words of those
// degrees: W[i * 8 + g] holds digit i of the K indices 4 g .. 4 g + 3 of the
// parity; groups G0 .. G1 - 1 of 8 degrees.  c1, c2 = Q(r-2), Q(r-4).  Segment ends (s % 16 == 0) rescale the
// chains as the one-step form rescales at s: the even chain after Q(s), the
// odd chain before Q(s+1), both by D(s).  The first tile starts the chains
// from Q(0) = start, Q(-2) = start (beta(0) = -1) and Q(1) = z start,
// Q(-1) = 0, set by the caller.  Degrees past lc in the last tile read stale
// table entries: their digits are garbage but finite integers, and the
// coefficient image is zero there.
template <int DA, int QR, int G0, int G1>
__device__ __forceinline__ void tile_digits(const double4* recs, double z2, double rp,
                                            bool first, double& c1, double& c2, uint32_t* W) {
    // 1.5 * 2^52 + 0x808080808080: for |X| < 2^46 the low 48 bits of the
    // rounded sum are X + 0x808080808080 (DA = 6)
    constexpr double kMagic6 = 6896688841130112.0;
    constexpr double kMagic = 6755399441055744.0;                 // 1.5 * 2^52
    constexpr unsigned long long kOffset7 = 0xBD48808080808080ull;   // 0x80..80 - bits(kMagic)
#pragma unroll
    for (int g8 = G0; g8 < G1; ++g8) {
        uint32_t lo[4], hi[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const int j = g8 * 8 + 2 * k + QR;
            const double4 f = recs[j];
            if (QR == 1 && (j & (kRecSegment - 1)) == 1) {
                const double d = recs[j - 1].z;
                c1 *= d;
                c2 *= d;
            }
            double q;
            if (j < 2 && first) {
                q = c1;                          // Q(0) or Q(1), set by the caller
            } else {
                q = fma(z2 - f.x, c1, -(f.y * c2));
                c2 = c1;
                c1 = q;
            }
            unsigned long long y;
            if constexpr (DA == 6) {
                y = (unsigned long long)__double_as_longlong(fma(q * f.z, rp, kMagic6));
            } else {
                // bits(1.5 * 2^52 + X) = 0x4338000000000000 + X for |X| < 2^51;
                // adding kOffset7 leaves X + 0x80..80 (7 bytes)
                y = (unsigned long long)__double_as_longlong(fma(q * f.z, rp, kMagic)) + kOffset7;
            }
            lo[k] = (uint32_t)y;
            hi[k] = (uint32_t)(y >> 32);
            if (QR == 0 && (j & (kRecSegment - 1)) == 0) {
                c1 *= f.z;
                c2 *= f.z;
            }
        }
        uint32_t w[DA];
        pack4<DA>(lo, hi, w);
#pragma unroll
        for (int i = 0; i < DA; ++i) W[i * 8 + g8] = w[i];
    }
}

// --------------------------------------------------------------------------
// the synthesis kernel: persistent CTAs of eight producer warps and one MMA
// warp over the work items (m, field group, tile of 128 pairs)
// --------------------------------------------------------------------------
template <int N, int DA>
__global__ void __launch_bounds__(kThreads, 1) k_legendre_synth_i8(SynthArgs a) {
    constexpr int DB = DA;
    constexpr int KW = Digits<DA>::KW;
    constexpr int TOP = DA + DB - 2;                 // weight of the two top digits
    constexpr int WB = TOP - KW + 1;                 // weight of accumulator block 0
    constexpr int NBLK = bstack_tiles(DA, DB, KW);
    constexpr int BT = btile_bytes(N);
    constexpr int SB = stage_bytes(N, DA, DB, KW);
    constexpr int NFG = N / 2;
    constexpr uint32_t kColA = tmem_cols_d(N, KW);
    static_assert(tmem_cols_d(N, KW) + 2 * tmem_cols_a(DA) <= kTmemAlloc, "tensor memory budget");
    static_assert(KW * N <= 256 && (KW * N) % 16 == 0, "MMA N");
    static_assert(KW >= DB, "leading zero tiles");
    extern __shared__ __align__(1024) uint8_t smem_i8[];   // kStages x SB
    __shared__ __align__(8) uint64_t full[kStages], empty[kStages];
    __shared__ __align__(8) uint64_t afull[2], mdone[2], dfree;
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long nitems = (long long)(a.lc + 1) * a.ptiles * a.ngroups;

    if (warp == 8) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(kTmemAlloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < kStages; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&afull[b], kProducers);
            mbar_init(&mdone[b], 1);
        }
        mbar_init(&dfree, kProducers);
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    // the zero tiles of every stage's two stacks (never written by the copies)
    for (int st = 0; st < kStages; ++st)
        for (int q = 0; q < 2; ++q) {
            uint8_t* stk = smem_i8 + st * SB + q * NBLK * BT;
            uint4* z0 = reinterpret_cast<uint4*>(stk);
            for (int k = tid; k < (KW - DB) * BT / 16; k += kThreads) z0[k] = make_uint4(0, 0, 0, 0);
            uint4* z1 = reinterpret_cast<uint4*>(stk + (KW - DB + DB) * BT);
            for (int k = tid; k < (DA - 1) * BT / 16; k += kThreads) z1[k] = make_uint4(0, 0, 0, 0);
        }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 9) {
        // ------------------------------------------------ stage loader
        // fills stage T % kStages with the coefficient digits and the
        // recursion table of K-tile T, item by item; the image and table
        // addresses are set up once per item
        if (lane == 0) {
            long long L = 0;                  // stages issued
            for (long long it = blockIdx.x; it < nitems && !abort_flag; it += gridDim.x) {
                int m, g, tile;
                item_decode(it, a.ptiles, a.ngroups, &m, &g, &tile);
                const int nt = ntiles_of(a.lc, m);
                const int nsteps = a.lc - m + 1;
                const uint8_t* src0 =
                    a.image + ((a.toff[m] * a.ngroups + (long long)g * nt) *
                               (long long)bimage_bytes(N, DB));
                const double4* rsrc0 = a.rec2 + packed_off(m, a.lc);
                for (int t = 0; t < nt && !abort_flag; ++t, ++L) {
                    const int st = (int)(L % kStages);
                    // the MMAs of the stage's previous tile have completed
                    if (L >= kStages &&
                        !mbar_wait(&empty[st], (uint32_t)((L / kStages - 1) & 1), &abort_flag))
                        break;
                    const int rdeg = min(kTileDeg, nsteps - kTileDeg * t);
                    uint8_t* sb = smem_i8 + st * SB;
                    const uint8_t* src = src0 + (long long)t * bimage_bytes(N, DB);
                    constexpr uint32_t half = DB * BT;
                    mbar_expect_tx(&full[st], (uint32_t)(2 * half + rdeg * 32));
                    bulk_g2s(sb + (KW - DB) * BT, src, half, &full[st]);
                    bulk_g2s(sb + NBLK * BT + (KW - DB) * BT, src + half, half, &full[st]);
                    bulk_g2s(sb + 2 * NBLK * BT, rsrc0 + kTileDeg * t, (uint32_t)(rdeg * 32),
                             &full[st]);
                }
            }
            // drain (bounded): every copy issued has landed before exit
            for (long long T = L - kStages < 0 ? 0 : L - kStages; T < L; ++T)
                for (unsigned k = 0; k < kSpinLimit; ++k)
                    if (mbar_try(&full[T % kStages], (uint32_t)((T / kStages) & 1))) break;
        }
        __syncwarp();
    } else if (warp == 8) {
        // ------------------------------------------------ MMA issue
        // The whole warp runs the loop on warp-uniform values (the TMEM base
        // broadcast from lane 0, descriptors from the shared-memory base and
        // loop counters), so they stay in uniform registers; one elected lane
        // issues each MMA and commit.  A single thread computing per-lane
        // values spends about 100 cycles per MMA on moving them into uniform
        // registers (measured on B200), more than the MMA itself.
        const uint32_t tm = __shfl_sync(0xffffffffu, tmem, 0);
        const bool leader = elect_one();
        const uint64_t desc0 = smem_desc(smem_u32(smem_i8), 128, 256);
        constexpr uint32_t idesc = idesc_i8(128, KW * N, 1, 1);
        long long T = 0;                      // tiles multiplied
        int kitem = 0;
        for (long long it = blockIdx.x; it < nitems && !abort_flag; it += gridDim.x, ++kitem) {
            int m, g, tile;
            item_decode(it, a.ptiles, a.ngroups, &m, &g, &tile);
            const int nt = ntiles_of(a.lc, m);
            for (int t = 0; t < nt && !abort_flag; ++t) {
                const int st = (int)(T % kStages);
                const int buf = (int)(T & 1);
                bool ok = mbar_wait(&full[st], (uint32_t)((T / kStages) & 1), &abort_flag) &&
                          mbar_wait(&afull[buf], (uint32_t)((T >> 1) & 1), &abort_flag) &&
                          (t > 0 || kitem == 0 ||
                           mbar_wait(&dfree, (uint32_t)((kitem - 1) & 1), &abort_flag));
                if (!__all_sync(0xffffffffu, ok)) break;
                tc_fence_after();
                // descriptor start addresses advance in 16-byte units
                const uint64_t dst = desc0 + (uint64_t)((st * SB) >> 4);
                // A digit i times the window of coefficient digits
                // TOP - KW + 1 - i .. TOP - i into the KW weight blocks of
                // the parity's accumulator; the parities alternate.  The
                // first MMA of an item overwrites every block.
#pragma unroll
                for (int i = 0; i < DA; ++i) {
#pragma unroll
                    for (int q = 0; q < 2; ++q) {
                        const uint32_t acc = (t > 0 || i > 0) ? 1u : 0u;
                        const uint32_t d = tm + (uint32_t)(q * KW * N);
                        const uint32_t at =
                            tm + kColA + (uint32_t)(buf * tmem_cols_a(DA) + (q * DA + i) * 8);
                        const uint64_t bd =
                            dst + (uint64_t)((q * NBLK * BT + (DA - 1 - i) * BT) >> 4);
                        if (leader) mma_ts(d, at, bd, idesc, acc);
                    }
                }
                if (leader) {
                    tc_commit(&mdone[buf]);
                    tc_commit(&empty[st]);
                }
                __syncwarp();
                ++T;
            }
        }
        // drain (bounded): the MMAs of the last tile
        if (T > 0) {
            const long long Tl = T - 1;
            for (unsigned k = 0; k < kSpinLimit; ++k)
                if (mbar_try(&mdone[Tl & 1], (uint32_t)((Tl >> 1) & 1))) break;
        }
        __syncwarp();
    } else {
        // ------------------------------------------------ producers
        const int lq = warp & 3;          // TMEM lane quarter (32 ring pairs)
        const int qrole = warp >> 2;      // parity of the degrees this warp converts
        long long T = 0;
        int kitem = 0;
        const uint32_t lane_base = tmem + ((uint32_t)(lq * 32) << 16);
        for (long long it = blockIdx.x; it < nitems && !abort_flag; it += gridDim.x, ++kitem) {
            int m, g, tile;
            item_decode(it, a.ptiles, a.ngroups, &m, &g, &tile);
            const int nt = ntiles_of(a.lc, m);
            const int p = tile * kPairs + lq * 32 + lane;
            const bool valid = p < a.npair;
            const double z = valid ? a.zp[p] : 0.0;
            const double rp = valid ? a.rtab[(long long)m * a.npair + p] * a.ascale : 0.0;
            // the chain of this warp's parity: Q(0) = start, Q(-2) = start
            // (with beta(0) = -1 the two-step form gives Q(2)), or Q(1) =
            // z start, Q(-1) = 0
            const double start = a.pmm[m];
            double c1 = qrole == 0 ? start : z * start;
            double c2 = qrole == 0 ? start : 0.0;
            const double z2 = z * z;
            // output scales of this warp's epilogue columns, loaded early:
            // 2^(8 WB) 2^-a 2^-b(m, n)
            double sc[8];
            {
                const int c0 = (qrole * 8) % N;
                const double* ci = a.colinv + ((long long)m * a.ngroups + g) * N + c0;
                const double k = pow2i(8 * WB) / a.ascale;
#pragma unroll
                for (int c = 0; c < 8; ++c) sc[c] = ci[c] * k;
            }
            // the A stores of a tile are waited for (and announced) at the
            // start of the next tile, so their latency overlaps its wait
            bool pending = false;
            int pbuf = 0;
            for (int t = 0; t < nt; ++t, ++T) {
                const int st = (int)(T % kStages);
                const int buf = (int)(T & 1);
                // warp-uniform outcome: the tcgen05 loads and stores below
                // are .sync.aligned
                if (!__all_sync(0xffffffffu,
                                mbar_wait(&full[st], (uint32_t)((T / kStages) & 1), &abort_flag)))
                    break;
                if (pending) {
                    tmem_wait_st();
                    tc_fence_before();
                    mbar_arrive(&afull[pbuf]);
                    pending = false;
                }
                const double4* recs =
                    reinterpret_cast<const double4*>(smem_i8 + st * SB + 2 * NBLK * BT);
                uint32_t W[DA * 8];     // [digit][word]: word g8 = K indices 4 g8 .. 4 g8 + 3
                const uint32_t acol = kColA + (uint32_t)(buf * tmem_cols_a(DA) + qrole * DA * 8);
                // first half of the tile (32 degrees), then its stores, which
                // overlap the second half; the MMAs of tile T - 2 have read
                // this A buffer before the first store
                if (qrole == 0) tile_digits<DA, 0, 0, 4>(recs, z2, rp, t == 0, c1, c2, W);
                else tile_digits<DA, 1, 0, 4>(recs, z2, rp, t == 0, c1, c2, W);
                if (!__all_sync(0xffffffffu,
                                T < 2 || mbar_wait(&mdone[buf], (uint32_t)(((T >> 1) - 1) & 1),
                                                   &abort_flag)))
                    break;
                tc_fence_after();
#pragma unroll
                for (int i = 0; i < DA; ++i) tmem_st4(lane_base + acol + i * 8, W + i * 8);
                if (qrole == 0) tile_digits<DA, 0, 4, 8>(recs, z2, rp, t == 0, c1, c2, W);
                else tile_digits<DA, 1, 4, 8>(recs, z2, rp, t == 0, c1, c2, W);
#pragma unroll
                for (int i = 0; i < DA; ++i) tmem_st4(lane_base + acol + i * 8 + 4, W + i * 8 + 4);
                pending = true;
                pbuf = buf;
            }
            if (pending) {
                tmem_wait_st();
                tc_fence_before();
                mbar_arrive(&afull[pbuf]);
            }
            if (abort_flag) break;
            // epilogue: D of this item, columns [qrole * 8, qrole * 8 + 8)
            const long long Tl = T - 1;
            if (!__all_sync(0xffffffffu, mbar_wait(&mdone[Tl & 1], (uint32_t)((Tl >> 1) & 1),
                                                   &abort_flag)))
                break;
            tc_fence_after();
            const int c0 = qrole * 8;
            double v[2][8];
            if (c0 < N) {
#pragma unroll
                for (int q = 0; q < 2; ++q) {
                    uint32_t acc[KW][8];
#pragma unroll
                    for (int w = 0; w < KW; ++w)
                        tmem_ld8(lane_base + (uint32_t)((q * KW + w) * N + c0), acc[w]);
                    tmem_wait_ld();
#pragma unroll
                    for (int c = 0; c < 8; ++c) {
                        long long gsum[3] = {0, 0, 0};
#pragma unroll
                        for (int w = 0; w < KW; ++w)
                            gsum[w / 3] += (long long)(int)acc[w][c] << (8 * (w % 3));
                        // weights 2^(8 w) relative to block 0
                        v[q][c] = fma((double)gsum[2], 281474976710656.0,
                                      fma((double)gsum[1], 16777216.0, (double)gsum[0])) * sc[c];
                    }
                }
            }
            // the accumulators are in registers: the next item's MMAs may
            // overwrite them while the results are stored
            tc_fence_before();
            mbar_arrive(&dfree);
            if (c0 < N && valid) {
                const double h = m ? 0.5 : 1.0;
#pragma unroll
                for (int c = 0; c < 8; c += 2) {
                    const int f = (c0 + c) >> 1, fg = g * NFG + f;
                    if (fg >= a.nfield) continue;
                    const double eR = v[0][c], oR = v[1][c];
                    const double eI = v[0][c + 1], oI = v[1][c + 1];
                    double2* o2 = a.spec + (((long long)fg * a.npair + p) * (a.lc + 1) + m) * 2;
                    o2[0] = make_double2((eR + oR) * h, -(eI + oI) * h);
                    o2[1] = make_double2((eR - oR) * h, -(eI - oI) * h);
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 8) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kTmemAlloc));
    }
}

// --------------------------------------------------------------------------
// {gamma(r), delta(r), D(r), 0} of the same-parity two-step recursion from
// the plan's {beta(r), D(r)}: gamma = beta(r-1) + beta(r), delta =
// beta(r-1) beta(r-2) (r >= 2; entries r < 2 are not used by the chains)
// --------------------------------------------------------------------------
__global__ void k_i8_rec2(const double2* __restrict__ rec, double4* __restrict__ rec2, int lc) {
    const int m = blockIdx.y;
    const int r = blockIdx.x * blockDim.x + threadIdx.x;
    if (m + r > lc) return;
    const long long o = packed_off(m, lc);
    const double2 f = rec[o + r];
    double g = 0.0, d = 0.0;
    if (r >= 2) {
        const double b1 = rec[o + r - 1].x, b2 = rec[o + r - 2].x;
        g = b1 + f.x;
        d = b1 * b2;
    }
    rec2[o + r] = make_double4(g, d, f.y, 0.0);
}

#include "legendre_i8_table.cuh"
#include "legendre_i8_anal.cuh"

// --------------------------------------------------------------------------
// host side
// --------------------------------------------------------------------------
static bool has_table(const shtc_plan* P) {
    return P->d_i8_tab != nullptr && P->i8_tab_prec == P->precision;
}

// columns of a field group: 2 x 8 fields (on-the-fly kernel: MMA N of the
// weight window = KW x 16 = 112 or 128); the table-driven kernel takes
// 2 x 16 fields when there are more than 8.  Groups of fewer fields leave
// columns empty.
static int group_cols(const shtc_plan* P, int nfield) {
    return has_table(P) && nfield > 8 ? 32 : 16;
}

static int prec_digits(int precision) { return precision == SHTC_PREC_INT8X7 ? 7 : 6; }

static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

}  // namespace i8

using namespace i8;

// scratch of the tensor-core synthesis (the coefficient image and the column
// scales) and of the tensor-core analysis (the ring-sum image and its
// scales): one region serves both directions, so its size does not depend on
// whether the plan holds its table
static size_t synth_image_bytes(const shtc_plan* P, int nfield, int N) {
    const int ngroups = (nfield + N / 2 - 1) / (N / 2);
    const int DB = prec_digits(P->precision);
    return align256((size_t)P->i8_ntot * ngroups * bimage_bytes(N, DB)) +
           align256((size_t)(P->lc + 1) * ngroups * N * sizeof(double));
}

static int anal_cols(int nfield) { return nfield > 8 ? 32 : 16; }

static size_t anal_image_bytes(const shtc_plan* P, int nfield) {
    const int N = anal_cols(nfield), ngroups = (nfield + N / 2 - 1) / (N / 2);
    const int DB = prec_digits(P->precision);
    const int ptiles = (P->npair + kPairs - 1) / kPairs;
    return align256((size_t)(P->lc + 1) * ptiles * 2 * ngroups * gimage_bytes(N, DB)) +
           align256((size_t)(P->lc + 1) * 2 * ngroups * N * sizeof(double)) +
           align256((size_t)(P->lc + 1) * nfield * 4 * sizeof(unsigned long long));
}

size_t synth_i8_bytes(const shtc_plan* P, int nfield) {
    // either column count of the synthesis (16 on the fly, 32 from the table
    // for more than 8 fields), or the analysis
    const size_t s16 = synth_image_bytes(P, nfield, 16), s32 = synth_image_bytes(P, nfield, 32);
    const size_t s = s16 > s32 ? s16 : s32;
    const size_t a = anal_image_bytes(P, nfield);
    return s > a ? s : a;
}

int set_precision_tables(shtc_plan* P, int precision) {
    if (precision == SHTC_PREC_F64) {
        P->precision = precision;
        return SHTC_OK;
    }
    if (precision != SHTC_PREC_INT8X6 && precision != SHTC_PREC_INT8X7) return SHTC_EBOUND;
    if (P->cplx || P->norm == 3) return SHTC_EUNSUP;
    // a table of the other precision's digits is of no use
    if (P->d_i8_tab && P->i8_tab_prec != precision) free_i8_table(P);
    if (!P->d_i8_toff) {
        std::vector<long long> toff(P->lc + 2);
        long long acc = 0;
        for (int m = 0; m <= P->lc; ++m) {
            toff[m] = acc;
            acc += ntiles_of(P->lc, m);
        }
        toff[P->lc + 1] = acc;
        long long* d = nullptr;
        if (cudaMalloc((void**)&d, sizeof(long long) * toff.size()) != cudaSuccess)
            return SHTC_EALLOC;
        if (cudaMemcpy(d, toff.data(), sizeof(long long) * toff.size(),
                       cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(d);
            return SHTC_ECUDA;
        }
        P->d_i8_toff = d;
        P->i8_ntot = acc;
    }
    if (!P->d_i8_uoff) {
        std::vector<long long> uoff(P->lc + 2);
        long long acc = 0;
        for (int m = 0; m <= P->lc; ++m) {
            uoff[m] = acc;
            acc += nsuper_of(P->lc, m);
        }
        uoff[P->lc + 1] = acc;
        long long* d = nullptr;
        if (cudaMalloc((void**)&d, sizeof(long long) * uoff.size()) != cudaSuccess)
            return SHTC_EALLOC;
        if (cudaMemcpy(d, uoff.data(), sizeof(long long) * uoff.size(),
                       cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaFree(d);
            return SHTC_ECUDA;
        }
        P->d_i8_uoff = d;
        P->i8_utot = acc;
    }
    if (!P->d_i8_rec2) {
        double4* d = nullptr;
        if (cudaMalloc((void**)&d, sizeof(double4) * (size_t)P->nlm) != cudaSuccess)
            return SHTC_EALLOC;
        k_i8_rec2<<<dim3((P->lc + 1 + 127) / 128, P->lc + 1), 128>>>(P->d_rec, d, P->lc);
        if (cudaGetLastError() != cudaSuccess || cudaDeviceSynchronize() != cudaSuccess) {
            cudaFree(d);
            return SHTC_ECUDA;
        }
        P->d_i8_rec2 = d;
    }
    // |P_lm| bound over l <= lc: sqrt(2l+1) (4pi), 1 (Schmidt), sqrt((2l+1)/4pi)
    const double pi = 3.141592653589793238462643383279502884;
    double bound = 1.0;
    if (P->norm == 1) bound = sqrt(2.0 * P->lc + 1.0);
    else if (P->norm == 4) bound = sqrt((2.0 * P->lc + 1.0) / (4.0 * pi));
    int e;
    frexp(bound * (1.0 + 1e-9), &e);   // bound < 2^e
    const int bits = prec_digits(precision) == 7 ? Digits<7>::kBitsA : Digits<6>::kBitsA;
    P->i8_ascale = ldexp(1.0, bits - e);
    P->precision = precision;
    return SHTC_OK;
}

static int sm_count(int dev) {
    static int nsm[64] = {0};
    if (dev >= 0 && dev < 64 && nsm[dev] == 0)
        cudaDeviceGetAttribute(&nsm[dev], cudaDevAttrMultiProcessorCount, dev);
    return dev >= 0 && dev < 64 && nsm[dev] > 0 ? nsm[dev] : 148;
}

template <int N, int DA>
static int launch_synth_i8_n(const shtc_plan* P, const double2* coef, double2* spec, int nfield,
                             void* scratch, cudaStream_t st) {
    constexpr int KW = Digits<DA>::KW;
    const int ngroups = (nfield + N / 2 - 1) / (N / 2);
    uint8_t* image = (uint8_t*)scratch;
    double* colinv =
        (double*)((char*)scratch + align256((size_t)P->i8_ntot * ngroups * bimage_bytes(N, DA)));
    k_i8_coef_image<N, DA><<<dim3(P->lc + 1, ngroups), 256, 0, st>>>(
        coef, (uint32_t*)image, P->d_i8_toff, colinv, P->lc, nfield, ngroups);
    int rc = map_cuda(cudaGetLastError());
    if (rc) return rc;
    // at least 120 KB of shared memory keeps one CTA (and one 512-column
    // TMEM allocation) per SM
    constexpr size_t stages = (size_t)kStages * stage_bytes(N, DA, DA, KW);
    const size_t smem = stages > 120 * 1024 ? stages : 120 * 1024;
    static_assert(stages <= 200 * 1024, "stages fit in shared memory");
    if ((rc = kernel_smem_attr((const void*)k_legendre_synth_i8<N, DA>, smem, true))) return rc;
    const int sms = sm_count(P->device);
    SynthArgs a;
    a.rec2 = P->d_i8_rec2;
    a.pmm = P->d_pmm;
    a.rtab = P->d_rtab;
    a.zp = P->d_z;
    a.image = image;
    a.toff = P->d_i8_toff;
    a.colinv = colinv;
    a.spec = spec;
    a.lc = P->lc;
    a.npair = P->npair;
    a.nfield = nfield;
    a.ngroups = ngroups;
    a.ptiles = (P->npair + kPairs - 1) / kPairs;
    a.ascale = P->i8_ascale;
    const long long nitems = (long long)(P->lc + 1) * a.ptiles * ngroups;
    const int grid = (int)(nitems < sms ? nitems : sms);
    k_legendre_synth_i8<N, DA><<<grid, kThreads, smem, st>>>(a);
    return map_cuda(cudaGetLastError());
}

// the table-driven synthesis: coefficient image, then the streaming kernel
template <int N, int DA>
static int launch_synth_tab_n(const shtc_plan* P, const double2* coef, double2* spec, int nfield,
                              void* scratch, cudaStream_t st) {
    const int ngroups = (nfield + N / 2 - 1) / (N / 2);
    uint8_t* image = (uint8_t*)scratch;
    double* colinv =
        (double*)((char*)scratch + align256((size_t)P->i8_ntot * ngroups * bimage_bytes(N, DA)));
    k_i8_coef_image<N, DA><<<dim3(P->lc + 1, ngroups), 256, 0, st>>>(
        coef, (uint32_t*)image, P->d_i8_toff, colinv, P->lc, nfield, ngroups);
    int rc = map_cuda(cudaGetLastError());
    if (rc) return rc;
    constexpr size_t smem = (size_t)tab_stages(N, DA) * tab_stage_bytes(N, DA);
    static_assert(smem >= 120 * 1024 && smem <= 220 * 1024, "one CTA per SM, stages fit");
    if ((rc = kernel_smem_attr((const void*)k_legendre_synth_tab<N, DA>, smem, true))) return rc;
    TabSynthArgs a;
    a.tab = P->d_i8_tab;
    a.off = P->d_i8_tab_off;
    a.u0 = P->d_i8_tab_u0;
    a.image = image;
    a.toff = P->d_i8_toff;
    a.colinv = colinv;
    a.spec = spec;
    a.lc = P->lc;
    a.npair = P->npair;
    a.nfield = nfield;
    a.ngroups = ngroups;
    a.ptiles = (P->npair + kPairs - 1) / kPairs;
    a.ascale = P->i8_ascale;
    const long long nitems = (long long)(P->lc + 1) * a.ptiles * ngroups;
    const int sms = sm_count(P->device);
    const int grid = (int)(nitems < sms ? nitems : sms);
    k_legendre_synth_tab<N, DA><<<grid, kTabThreads, smem, st>>>(a);
    return map_cuda(cudaGetLastError());
}

int launch_legendre_synth_i8(const shtc_plan* P, const double2* coef, double2* spec,
                             int nfield, void* scratch, cudaStream_t st) {
    if (!P->d_i8_toff) return SHTC_EBOUND;
    const bool seven = P->precision == SHTC_PREC_INT8X7;
    if (P->precision != SHTC_PREC_INT8X6 && !seven) return SHTC_EBOUND;
    if (has_table(P)) {
        if (group_cols(P, nfield) == 32)
            return seven ? launch_synth_tab_n<32, 7>(P, coef, spec, nfield, scratch, st)
                         : launch_synth_tab_n<32, 6>(P, coef, spec, nfield, scratch, st);
        return seven ? launch_synth_tab_n<16, 7>(P, coef, spec, nfield, scratch, st)
                     : launch_synth_tab_n<16, 6>(P, coef, spec, nfield, scratch, st);
    }
    return seven ? launch_synth_i8_n<16, 7>(P, coef, spec, nfield, scratch, st)
                 : launch_synth_i8_n<16, 6>(P, coef, spec, nfield, scratch, st);
}

// the table-driven analysis: ring-sum image, then the streaming kernel
template <int N, int DA>
static int launch_anal_tab_n(const shtc_plan* P, const double2* spec, double2* partial,
                             int nfield, void* scratch, cudaStream_t st) {
    const int ngroups = (nfield + N / 2 - 1) / (N / 2);
    const int ptiles = (P->npair + kPairs - 1) / kPairs;
    uint8_t* image = (uint8_t*)scratch;
    const size_t ib = align256((size_t)(P->lc + 1) * ptiles * 2 * ngroups * gimage_bytes(N, DA));
    double* colinv = (double*)((char*)scratch + ib);
    unsigned long long* gmax = (unsigned long long*)(
        (char*)scratch + ib + align256((size_t)(P->lc + 1) * 2 * ngroups * N * sizeof(double)));
    const size_t gmb = (size_t)(P->lc + 1) * nfield * 4 * sizeof(unsigned long long);
    int rc = map_cuda(cudaMemsetAsync(gmax, 0, gmb, st));
    if (rc) return rc;
    k_i8_anal_max<<<dim3((P->lc + 1 + 127) / 128, nfield, (P->npair + kMaxPairs - 1) / kMaxPairs),
                    128, 0, st>>>(spec, gmax, P->lc, P->npair);
    k_i8_anal_digits<N, DA><<<dim3(P->lc + 1, ptiles, ngroups), 16 * N, 0, st>>>(
        spec, gmax, (uint32_t*)image, colinv, P->lc, P->npair, nfield, ngroups, ptiles);
    if ((rc = map_cuda(cudaGetLastError()))) return rc;
    constexpr int NBUF = 1;                   // two CTAs per SM, one accumulator buffer each
    constexpr size_t smem = anal_smem(N, DA, NBUF);
    if ((rc = kernel_smem_attr((const void*)k_legendre_anal_tab<N, DA, NBUF>, smem, true)))
        return rc;
    TabAnalArgs a;
    a.tab = P->d_i8_tab;
    a.off = P->d_i8_tab_off;
    a.u0 = P->d_i8_tab_u0;
    a.uoff = P->d_i8_uoff;
    a.image = image;
    a.colinv = colinv;
    a.partial = partial;
    a.nlm = P->nlm;
    a.lc = P->lc;
    a.npair = P->npair;
    a.nfield = nfield;
    a.ngroups = ngroups;
    a.ptiles = ptiles;
    a.ascale = P->i8_ascale;
    const long long nitems = 2LL * ngroups * P->i8_utot;
    const int ctas = sm_count(P->device) * (NBUF == 1 ? 2 : 1);
    const int grid = (int)(nitems < ctas ? nitems : ctas);
    k_legendre_anal_tab<N, DA, NBUF><<<grid, kTabThreads, smem, st>>>(a);
    return map_cuda(cudaGetLastError());
}

bool anal_i8_ready(const shtc_plan* P) {
    return (P->precision == SHTC_PREC_INT8X6 || P->precision == SHTC_PREC_INT8X7) &&
           !P->cplx && has_table(P) && P->d_i8_uoff != nullptr;
}

int launch_legendre_anal_i8(const shtc_plan* P, const double2* spec, double2* partial,
                            int nfield, void* scratch, cudaStream_t st) {
    if (!anal_i8_ready(P)) return SHTC_EBOUND;
    const bool seven = P->precision == SHTC_PREC_INT8X7;
    if (anal_cols(nfield) == 32)
        return seven ? launch_anal_tab_n<32, 7>(P, spec, partial, nfield, scratch, st)
                     : launch_anal_tab_n<32, 6>(P, spec, partial, nfield, scratch, st);
    return seven ? launch_anal_tab_n<16, 7>(P, spec, partial, nfield, scratch, st)
                 : launch_anal_tab_n<16, 6>(P, spec, partial, nfield, scratch, st);
}

void free_i8_table(shtc_plan* P) {
    if (P->d_i8_tab) P->device_bytes -= P->i8_tab_bytes;
    cudaFree(P->d_i8_tab);
    cudaFree(P->d_i8_tab_off);
    cudaFree(P->d_i8_tab_u0);
    P->d_i8_tab = nullptr;
    P->d_i8_tab_off = nullptr;
    P->d_i8_tab_u0 = nullptr;
    P->i8_tab_bytes = 0;
    P->i8_tab_prec = 0;
}

// Two passes of the recursion over every (m, pair tile): the first finds the
// leading all-zero super-tiles, the second writes the stored ones into the
// zeroed table.
template <int DA>
static int build_i8_table_n(shtc_plan* P) {
    const int ptiles = (P->npair + kPairs - 1) / kPairs;
    const long long nitem = (long long)(P->lc + 1) * ptiles;
    TabBuildArgs a;
    a.rec = P->d_rec;
    a.pmm = P->d_pmm;
    a.rtab = P->d_rtab;
    a.zp = P->d_z;
    a.lc = P->lc;
    a.npair = P->npair;
    a.ptiles = ptiles;
    a.ascale = P->i8_ascale;
    a.off = nullptr;
    a.tab = nullptr;
    int* u0 = nullptr;
    long long* off = nullptr;
    uint8_t* tab = nullptr;
    std::vector<int> hu0((size_t)nitem);
    std::vector<long long> hoff((size_t)nitem);
    int rc = SHTC_OK;
    auto fail = [&](int code) {
        cudaFree(u0);
        cudaFree(off);
        cudaFree(tab);
        return code;
    };
    if (cudaMalloc((void**)&u0, sizeof(int) * (size_t)nitem) != cudaSuccess) return fail(SHTC_EALLOC);
    a.u0 = u0;
    const dim3 grid(ptiles, P->lc + 1);
    k_i8_table<DA, false><<<grid, kPairs>>>(a);
    if ((rc = map_cuda(cudaGetLastError()))) return fail(rc);
    if ((rc = map_cuda(cudaMemcpy(hu0.data(), u0, sizeof(int) * (size_t)nitem,
                                  cudaMemcpyDeviceToHost))))
        return fail(rc);
    long long acc = 0;
    for (int m = 0; m <= P->lc; ++m)
        for (int pt = 0; pt < ptiles; ++pt) {
            const long long i = (long long)m * ptiles + pt;
            hoff[i] = acc;
            acc += nsuper_of(P->lc, m) - hu0[i];
        }
    const unsigned long long bytes = (unsigned long long)acc * tab_super_bytes(DA);
    if (cudaMalloc((void**)&off, sizeof(long long) * (size_t)nitem) != cudaSuccess)
        return fail(SHTC_EALLOC);
    if (cudaMalloc((void**)&tab, (size_t)(bytes ? bytes : 256)) != cudaSuccess) {
        cudaGetLastError();
        return fail(SHTC_EALLOC);
    }
    if ((rc = map_cuda(cudaMemcpy(off, hoff.data(), sizeof(long long) * (size_t)nitem,
                                  cudaMemcpyHostToDevice))))
        return fail(rc);
    if ((rc = map_cuda(cudaMemset(tab, 0, (size_t)(bytes ? bytes : 256))))) return fail(rc);
    a.off = off;
    a.tab = tab;
    if (bytes) {
        k_i8_table<DA, true><<<grid, kPairs>>>(a);
        if ((rc = map_cuda(cudaGetLastError()))) return fail(rc);
    }
    if ((rc = map_cuda(cudaDeviceSynchronize()))) return fail(rc);
    P->d_i8_tab = tab;
    P->d_i8_tab_off = off;
    P->d_i8_tab_u0 = u0;
    P->i8_tab_bytes = bytes;
    P->i8_tab_prec = P->precision;
    P->device_bytes += bytes;
    return SHTC_OK;
}

}  // namespace shtc

using namespace shtc;

extern "C" int shtc_plan_set_precision(shtc_plan* P, int precision) {
    if (!P) return SHTC_EHANDLE;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != P->device) return SHTC_EHANDLE;
    return set_precision_tables(P, precision);
}

extern "C" int shtc_plan_legendre_table(shtc_plan* P, int enable, unsigned long long* bytes) {
    if (!P) return SHTC_EHANDLE;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != P->device) return SHTC_EHANDLE;
    int rc = SHTC_OK;
    if (!enable) {
        free_i8_table(P);
    } else if (!has_table(P)) {
        if (P->precision != SHTC_PREC_INT8X6 && P->precision != SHTC_PREC_INT8X7)
            return SHTC_EBOUND;
        free_i8_table(P);
        rc = P->precision == SHTC_PREC_INT8X7 ? build_i8_table_n<7>(P) : build_i8_table_n<6>(P);
    }
    if (bytes) *bytes = P->i8_tab_bytes;
    return rc;
}

namespace shtc {
namespace i8 {
// One thread waits, through the tensor kernels' bounded wait, on an mbarrier
// that nothing arrives on: the wait runs out, records SHTC_ETIMEOUT in the
// error word and returns (no trap, no unbounded loop)
__global__ void k_i8_wait_selftest() {
    __shared__ __align__(8) uint64_t bar;
    __shared__ volatile int abort_flag;
    mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    mbar_wait(&bar, 0, &abort_flag);
}
}  // namespace i8
}  // namespace shtc

extern "C" int shtc_mixed_wait_selftest(void* stream) {
    i8::k_i8_wait_selftest<<<1, 1, 0, (cudaStream_t)stream>>>();
    int rc = map_cuda(cudaGetLastError());
    if (!rc) rc = map_cuda(cudaStreamSynchronize((cudaStream_t)stream));
    return rc;
}

extern "C" int shtc_mixed_status(int* status, void* stream) {
    if (!status) return SHTC_EHANDLE;
    cudaStream_t st = (cudaStream_t)stream;
    int* d = nullptr;
    int rc = map_cuda(cudaGetSymbolAddress((void**)&d, i8::g_i8_status));
    if (rc) return rc;
    int h = 0;
    rc = map_cuda(cudaMemcpyAsync(&h, d, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaMemsetAsync(d, 0, sizeof(int), st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    if (rc) return rc;
    *status = h;
    return SHTC_OK;
}
