// Table-driven Legendre analysis on the tensor cores (tcgen05 kind::i8) with
// the error-free split of legendre_i8.cu (SHExpandDH.f95:463-580,
// SHExpandGLQ.f95:445-649).  For one order m, one parity q and one
// super-tile u of the plan's P_lm digit table (128 degrees of that parity,
// s = l - m = 256 u + 2 d + q) the analysis of F fields is a matrix product
// over the ring pairs:
//     C[d][n] = sum_p P_lm(z_p) G_q[p][n],
// G_0 = north + south ring spectra, G_1 = north - south (the r2c has applied
// the ring weights), n = (field, Re/Im).
//
//   A = the table's digit block of (m, pair tile, u, q), read MN-major
//       (M = 128 degrees, K = 32 pairs per MMA; legendre_i8_table.cuh);
//   B = digits of round(G_q[p][n] 2^b(m, q, n)), one exponent per order,
//       parity and column from max_p |G_q[p][n]| (k_i8_anal_digits), K-major.
// Digit i of A meets the window of B digits j = max(0, WB - i) .. DB - 1 in
// one MMA whose (DB - j0) N columns land on the accumulator's weight blocks
// w = i + j - WB, as in the synthesis.  The K loop runs over the pair tiles
// whose stored super-tiles include u (the skipped ones are exactly zero).
// The INT32 sums are exact: at most DB products of 2^14 per weight and pair,
// |sum| < DB 2^14 npair < 2^31 for npair < 18000.
//
// Two CTAs per SM (NBUF = 1; 20% faster at lmax 2799 x16 than one CTA per SM
// with two accumulator buffers, NBUF = 2): in each, warp 9 streams the
// table's digit blocks (16 KB each, a ring of NA) and the B tiles (a ring of
// NB) with bulk copies, warp 8 issues the MMAs from one elected lane, warps
// 0-7 read the accumulators (256 tensor-memory columns per CTA), combine the
// weights in 64-bit integers and FP64, and write the coefficients of the
// item's degrees; while one CTA's epilogue holds its accumulators, the other
// CTA's MMAs and copies keep the SM busy.  Every wait is bounded
// (legendre_i8.cu).

// one B digit tile: N columns x 128 pairs; byte (n, k) at
// (n / 8) * 1024 + (k / 16) * 128 + (n % 8) * 16 + k % 16
__host__ __device__ constexpr int gtile_bytes(int N) { return N * kPairs; }
__host__ __device__ constexpr int gimage_bytes(int N, int DB) { return DB * gtile_bytes(N); }
// shared-memory slots: one CTA per SM with two accumulator buffers, or
// (NBUF = 1) two CTAs per SM with one each
__host__ __device__ constexpr int anal_astages(int N, int NBUF) {
    return NBUF == 2 ? (N == 32 ? 9 : 10) : (N == 32 ? 3 : 5);
}
__host__ __device__ constexpr int anal_bstages(int N, int NBUF) {
    return NBUF == 2 ? (N == 32 ? 2 : 3) : 2;
}
__host__ __device__ constexpr int anal_smem(int N, int DB, int NBUF) {
    return anal_astages(N, NBUF) * kTabDigit + anal_bstages(N, NBUF) * gimage_bytes(N, DB);
}
// tensor-memory columns allocated by an analysis CTA (a power of two >= 32)
__host__ __device__ constexpr int anal_tmem_cols(int DC, int NBUF) {
    return NBUF == 2 ? 512 : (DC <= 128 ? 128 : 256);
}

// --------------------------------------------------------------------------
// ring-sum image: per (m, pair tile pt, parity q, field group g) the DB digit
// tiles of B, tile index ((m * ptiles + pt) * 2 + q) * ngroups + g; byte =
// balanced digit j of round(G_q[p][n] 2^b).  colinv[((m * 2 + q) * ngroups +
// g) * N + n] = 2^-b.  spec: r2c output [field][pair][m][ring] (Re, Im).
// Two passes over spec: the column maxima (k_i8_anal_max), then the digits
// (k_i8_anal_digits), each reading every 32-byte ring pair once.
// --------------------------------------------------------------------------
constexpr int kMaxPairs = 64;     // ring pairs per block of the maxima pass

// gmax[(f * (lc + 1) + m) * 4 + k] = max_p |G|, k = (q, Re/Im): the bits of
// non-negative doubles, which order as integers (zeroed by the caller)
__global__ void __launch_bounds__(128)
k_i8_anal_max(const double2* __restrict__ spec, unsigned long long* __restrict__ gmax, int lc,
              int npair) {
    const int m = blockIdx.x * 128 + threadIdx.x;
    const int f = blockIdx.y;
    const int p0 = blockIdx.z * kMaxPairs;
    if (m > lc) return;
    const int p1 = min(npair, p0 + kMaxPairs);
    const double4* x = reinterpret_cast<const double4*>(spec) +
                       ((long long)f * npair + p0) * (lc + 1) + m;
    double mx[4] = {0.0, 0.0, 0.0, 0.0};
    for (int p = p0; p < p1; ++p, x += lc + 1) {
        const double4 v = *x;                     // north (Re, Im), south (Re, Im)
        mx[0] = fmax(mx[0], fabs(v.x + v.z));
        mx[1] = fmax(mx[1], fabs(v.y + v.w));
        mx[2] = fmax(mx[2], fabs(v.x - v.z));
        mx[3] = fmax(mx[3], fabs(v.y - v.w));
    }
    unsigned long long* o = gmax + ((long long)f * (lc + 1) + m) * 4;
#pragma unroll
    for (int k = 0; k < 4; ++k)
        if (mx[k] > 0.0) atomicMax(&o[k], (unsigned long long)__double_as_longlong(mx[k]));
}

// Block (m, pt, g) of 32 NFG threads: thread (k4, fl, kc, ng) converts the
// four pairs kc * 16 + k4 * 4 + 0..3 of field ng * 4 + fl, both parities and
// both Re and Im, reading each pair's 32 bytes once.
template <int N, int DB>
__global__ void __launch_bounds__(16 * N)
k_i8_anal_digits(const double2* __restrict__ spec, const unsigned long long* __restrict__ gmax,
                 uint32_t* __restrict__ image, double* __restrict__ colinv, int lc, int npair,
                 int nfield, int ngroups, int ptiles) {
    constexpr int NFG = N / 2;
    constexpr int kBits = Digits<DB>::kBitsB;
    constexpr int WPT = gtile_bytes(N) / 4;
    const int m = blockIdx.x, pt = blockIdx.y, g = blockIdx.z;
    const int tid = threadIdx.x;
    const int k4 = tid & 3, fl = (tid >> 2) & 3, kc = (tid >> 4) & 7, ng = tid >> 7;
    const int fi = ng * 4 + fl, fg = g * NFG + fi;
    const bool fok = fg < nfield;
    double sc[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const double mx =
            fok ? __longlong_as_double((long long)gmax[((long long)fg * (lc + 1) + m) * 4 + k])
                : 0.0;
        double inv = 0.0;
        sc[k] = 0.0;
        if (mx > 0.0) {
            int e;
            frexp(mx, &e);                   // mx < 2^e
            sc[k] = ldexp(1.0, kBits - e);   // |G| sc < 2^kBits
            inv = ldexp(1.0, e - kBits);
        }
        if (pt == 0 && kc == 0 && k4 == 0)
            colinv[(((long long)m * 2 + (k >> 1)) * ngroups + g) * N + 2 * fi + (k & 1)] = inv;
    }
    uint32_t w[4][DB];
#pragma unroll
    for (int k = 0; k < 4; ++k)
#pragma unroll
        for (int j = 0; j < DB; ++j) w[k][j] = 0u;
#pragma unroll
    for (int u = 0; u < 4; ++u) {
        const int p = pt * kPairs + kc * 16 + k4 * 4 + u;
        double4 v = make_double4(0.0, 0.0, 0.0, 0.0);
        if (fok && p < npair)
            v = reinterpret_cast<const double4*>(spec)[((long long)fg * npair + p) * (lc + 1) + m];
        const double gv[4] = {v.x + v.z, v.y + v.w, v.x - v.z, v.y - v.w};
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            const long long x = __double2ll_rn(gv[k] * sc[k]) + Digits<DB>::kBalance;
#pragma unroll
            for (int j = 0; j < DB; ++j)
                w[k][j] |= (uint32_t)(((x >> (8 * j)) & 0xFF) ^ 0x80) << (8 * u);
        }
    }
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        const int q = k >> 1, n8 = 2 * fl + (k & 1);
        uint32_t* tb = image + ((((long long)m * ptiles + pt) * 2 + q) * ngroups + g) *
                                   (long long)(gimage_bytes(N, DB) / 4) +
                       ng * 256 + kc * 32 + n8 * 4 + k4;
#pragma unroll
        for (int j = 0; j < DB; ++j) tb[j * WPT] = w[k][j];
    }
}

struct TabAnalArgs {
    const uint8_t* tab;      // the table (k_i8_table)
    const long long* off;    // per (m * ptiles + pt): super-tiles stored before it
    const int* u0;           // per (m * ptiles + pt): first stored super-tile
    const long long* uoff;   // super-tiles of all orders before m (lc + 2 entries)
    const uint8_t* image;    // ring-sum image (k_i8_anal_digits<N, DB>)
    const double* colinv;    // 2^-b per (m, parity, group, column)
    double2* partial;        // [field][packed (l, m)] (Re, Im) sums
    long long nlm;
    int lc, npair, nfield, ngroups, ptiles;
    double ascale;           // 2^a: the A operand's fixed-point scale
};

// work item -> (m, super-tile u, parity q, field group g); m slowest (the
// longest items first), the groups of one (m, u, q) adjacent so that their
// reads of the same table blocks meet in L2
__device__ __forceinline__ void anal_item_decode(long long it, const long long* uoff, int lc,
                                                 int ngroups, int* m, int* u, int* q, int* g) {
    const long long per = 2LL * ngroups;
    const long long su = it / per;               // global super-tile index
    int lo = 0, hi = lc;                         // largest m with uoff[m] <= su
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (uoff[mid] <= su) lo = mid;
        else hi = mid - 1;
    }
    *m = lo;
    *u = (int)(su - uoff[lo]);
    const int r = (int)(it - su * per);
    *q = r / ngroups;
    *g = r - (*q) * ngroups;
}

// true when some pair tile of order m stores super-tile u
__device__ __forceinline__ bool anal_has_work(const int* u0, int m, int ptiles, int u) {
    for (int pt = 0; pt < ptiles; ++pt)
        if (u0[(long long)m * ptiles + pt] <= u) return true;
    return false;
}

template <int N, int DA, int NBUF>
__global__ void __launch_bounds__(kTabThreads, NBUF == 1 ? 2 : 1) k_legendre_anal_tab(TabAnalArgs a) {
    constexpr int DB = DA;
    constexpr int KW = Digits<DA>::KW;
    constexpr int TOP = DA + DB - 2;
    constexpr int WB = TOP - KW + 1;                 // weight of accumulator block 0
    constexpr int NA = anal_astages(N, NBUF), NB = anal_bstages(N, NBUF);
    constexpr int kAlloc = anal_tmem_cols(KW * N, NBUF);
    constexpr int BT = gtile_bytes(N);
    constexpr int BB = gimage_bytes(N, DB);
    constexpr int DC = KW * N;                       // tensor-memory columns of one D buffer
    constexpr int NFG = N / 2;
    constexpr int CW = N / 2;                        // columns of one epilogue warp
    static_assert(NBUF * DC <= kAlloc && (NBUF == 1 || NBUF == 2), "tensor memory budget");
    static_assert(DB * N <= 256 && N % 16 == 0, "MMA N");
    static_assert(KW == DB + 1 && WB == DA - 2, "weight windows");
    static_assert(anal_smem(N, DB, NBUF) <= (NBUF == 1 ? 110 * 1024 : kTabSmemBudget),
                  "stages fit");
    extern __shared__ __align__(1024) uint8_t smem_an[];   // NA A blocks | NB B tiles
    __shared__ __align__(8) uint64_t afull[NA], aempty[NA], bfull[NB], bempty[NB];
    __shared__ __align__(8) uint64_t dfull[2], dfree[2];
    __shared__ uint32_t tmem_base;
    __shared__ volatile int abort_flag;
    uint8_t* smem_a = smem_an;
    uint8_t* smem_b = smem_an + NA * kTabDigit;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const long long nitems = 2LL * a.ngroups * a.uoff[a.lc + 1];

    if (warp == 8) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(
                         smem_u32(&tmem_base)),
                     "r"(kAlloc));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    if (tid == 0) {
        for (int s = 0; s < NA; ++s) {
            mbar_init(&afull[s], 1);
            mbar_init(&aempty[s], 1);
        }
        for (int s = 0; s < NB; ++s) {
            mbar_init(&bfull[s], 1);
            mbar_init(&bempty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&dfull[b], 1);
            mbar_init(&dfree[b], kTabEpilogue);
        }
        abort_flag = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base;

    if (warp == 9) {
        // ------------------------------------------------ loader
        if (lane == 0) {
            long long LA = 0, LB = 0;         // A blocks and B tiles issued
            bool ok = true;
            for (long long it = blockIdx.x; it < nitems && ok && !abort_flag; it += gridDim.x) {
                int m, u, q, g;
                anal_item_decode(it, a.uoff, a.lc, a.ngroups, &m, &u, &q, &g);
                for (int pt = 0; pt < a.ptiles && ok; ++pt) {
                    const long long item = (long long)m * a.ptiles + pt;
                    const int u0 = a.u0[item];
                    if (u < u0) continue;
                    const int bs = (int)(LB % NB);
                    if (LB >= NB &&
                        !(ok = mbar_wait(&bempty[bs], (uint32_t)((LB / NB - 1) & 1), &abort_flag)))
                        break;
                    mbar_expect_tx(&bfull[bs], (uint32_t)BB);
                    bulk_g2s(smem_b + bs * BB,
                             a.image + ((item * 2 + q) * a.ngroups + g) * (long long)BB, BB,
                             &bfull[bs]);
                    ++LB;
                    const uint8_t* ab = a.tab +
                                        (a.off[item] + u - u0) * (long long)tab_super_bytes(DA) +
                                        (long long)q * DA * kTabDigit;
                    // digits from the top: the first MMAs of an item overwrite D
                    for (int i = DA - 1; i >= 0; --i, ++LA) {
                        const int as = (int)(LA % NA);
                        if (LA >= NA &&
                            !(ok = mbar_wait(&aempty[as], (uint32_t)((LA / NA - 1) & 1),
                                             &abort_flag)))
                            break;
                        mbar_expect_tx(&afull[as], (uint32_t)kTabDigit);
                        bulk_g2s(smem_a + as * kTabDigit, ab + (long long)i * kTabDigit, kTabDigit,
                                 &afull[as]);
                    }
                }
            }
            // drain (bounded): every copy issued has landed before exit
            for (long long T = LA - NA < 0 ? 0 : LA - NA; T < LA; ++T)
                for (unsigned k = 0; k < kSpinLimit; ++k)
                    if (mbar_try(&afull[T % NA], (uint32_t)((T / NA) & 1))) break;
            for (long long T = LB - NB < 0 ? 0 : LB - NB; T < LB; ++T)
                for (unsigned k = 0; k < kSpinLimit; ++k)
                    if (mbar_try(&bfull[T % NB], (uint32_t)((T / NB) & 1))) break;
        }
        __syncwarp();
    } else if (warp == 8) {
        // ------------------------------------------------ MMA issue
        const uint32_t tm = __shfl_sync(0xffffffffu, tmem, 0);
        const bool leader = elect_one();
        // A (MN-major): 16-degree chunks 2048 bytes apart (SBO), 8-pair
        // groups 128 apart (LBO); a K-step of 32 pairs advances 512 bytes.
        // B (K-major): 16-pair chunks 128 apart (LBO), 8-column groups 1024
        // apart (SBO), digit tiles BT apart; a K-step advances 256 bytes.
        const uint64_t adesc0 = smem_desc(smem_u32(smem_a), 128, 2048);
        const uint64_t bdesc0 = smem_desc(smem_u32(smem_b), 128, 1024);
        constexpr uint32_t kTransA = 1u << 15;    // A is MN-major
        long long TA = 0, TB = 0;
        int kwork = 0;
        bool ok = true;
        for (long long it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
            int m, u, q, g;
            anal_item_decode(it, a.uoff, a.lc, a.ngroups, &m, &u, &q, &g);
            if (!anal_has_work(a.u0, m, a.ptiles, u)) continue;
            const int buf = kwork % NBUF, use = kwork / NBUF;
            // the epilogue has read this buffer's previous item
            ok = kwork < NBUF ||
                 mbar_wait(&dfree[buf], (uint32_t)((use - 1) & 1), &abort_flag);
            if (!__all_sync(0xffffffffu, ok)) { ok = false; break; }
            tc_fence_after();
            const uint32_t d0 = tm + (uint32_t)(buf * DC);
            bool first = true;
            for (int pt = 0; pt < a.ptiles && ok; ++pt) {
                if (u < a.u0[(long long)m * a.ptiles + pt]) continue;
                const int bs = (int)(TB % NB);
                ok = mbar_wait(&bfull[bs], (uint32_t)((TB / NB) & 1), &abort_flag);
                if (!__all_sync(0xffffffffu, ok)) { ok = false; break; }
                const uint64_t bd = bdesc0 + (uint64_t)((bs * BB) >> 4);
                for (int i = DA - 1; i >= 0; --i, ++TA) {
                    const int as = (int)(TA % NA);
                    ok = mbar_wait(&afull[as], (uint32_t)((TA / NA) & 1), &abort_flag);
                    if (!__all_sync(0xffffffffu, ok)) { ok = false; break; }
                    tc_fence_after();
                    const uint64_t ad = adesc0 + (uint64_t)((as * kTabDigit) >> 4);
#pragma unroll
                    for (int ks = 0; ks < kPairs / 32; ++ks) {
                        const uint64_t a_k = ad + (uint64_t)((ks * 512) >> 4);
                        const uint64_t b_k = bd + (uint64_t)((ks * 256) >> 4);
                        const bool init = first && ks == 0;
                        if (i == DA - 1) {
                            // coefficient digits 0 .. DB-1 -> blocks 1 .. KW-1
                            if (leader)
                                mma_ss(d0 + N, a_k, b_k, idesc_i8(128, DB * N, 1, 1) | kTransA,
                                       init ? 0u : 1u);
                        } else if (i == DA - 2) {
                            if (init) {
                                // block 0 written alone, then blocks 1 .. KW-2
                                if (leader) {
                                    mma_ss(d0, a_k, b_k, idesc_i8(128, N, 1, 1) | kTransA, 0u);
                                    mma_ss(d0 + N, a_k, b_k + (uint64_t)(BT >> 4),
                                           idesc_i8(128, (DB - 1) * N, 1, 1) | kTransA, 1u);
                                }
                            } else if (leader) {
                                mma_ss(d0, a_k, b_k, idesc_i8(128, DB * N, 1, 1) | kTransA, 1u);
                            }
                        } else {
                            const int j0 = WB - i;
                            if (leader)
                                mma_ss(d0, a_k, b_k + (uint64_t)((j0 * BT) >> 4),
                                       idesc_i8(128, (DB - j0) * N, 1, 1) | kTransA, 1u);
                        }
                    }
                    if (leader) tc_commit(&aempty[as]);
                    __syncwarp();
                }
                if (!ok) break;
                if (leader) tc_commit(&bempty[bs]);
                __syncwarp();
                ++TB;
                first = false;
            }
            if (!ok) break;
            if (leader) tc_commit(&dfull[buf]);
            __syncwarp();
            ++kwork;
        }
        // drain (bounded): the MMAs of the last item
        if (kwork > 0) {
            const int kl = kwork - 1;
            for (unsigned k = 0; k < kSpinLimit; ++k)
                if (mbar_try(&dfull[kl % NBUF], (uint32_t)((kl / NBUF) & 1))) break;
        }
        __syncwarp();
    } else {
        // ------------------------------------------------ epilogue
        const int lq = warp & 3;              // TMEM lane quarter (32 degrees)
        const int c0 = (warp >> 2) * CW;      // this warp's columns
        const uint32_t lane_base = tmem + ((uint32_t)(lq * 32) << 16);
        const int d = lq * 32 + lane;         // degree row of the item
        int kwork = 0;
        for (long long it = blockIdx.x; it < nitems && !abort_flag; it += gridDim.x) {
            int m, u, q, g;
            anal_item_decode(it, a.uoff, a.lc, a.ngroups, &m, &u, &q, &g);
            const int s = 256 * u + 2 * d + q;
            const bool valid = s <= a.lc - m;
            const bool work = anal_has_work(a.u0, m, a.ptiles, u);
            const double kscale = pow2i(8 * WB) / a.ascale;
            const double* ci = a.colinv + (((long long)m * 2 + q) * a.ngroups + g) * N + c0;
            const long long o = packed_off(m, a.lc) + s;
            if constexpr (NBUF == 2) {
                double v[CW];
                if (work) {
                    double sc[CW];
#pragma unroll
                    for (int c = 0; c < CW; ++c) sc[c] = ci[c] * kscale;
                    const int buf = kwork & 1;
                    if (!__all_sync(0xffffffffu,
                                    mbar_wait(&dfull[buf], (uint32_t)((kwork >> 1) & 1),
                                              &abort_flag)))
                        break;
                    tc_fence_after();
                    const uint32_t dcol = (uint32_t)(buf * DC + c0);
#pragma unroll
                    for (int c8 = 0; c8 < CW; c8 += 8) {
                        uint32_t acc[KW][8];
#pragma unroll
                        for (int w = 0; w < KW; ++w)
                            tmem_ld8(lane_base + dcol + (uint32_t)(w * N + c8), acc[w]);
                        tmem_wait_ld();
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            long long gsum[3] = {0, 0, 0};
#pragma unroll
                            for (int w = 0; w < KW; ++w)
                                gsum[w / 3] += (long long)(int)acc[w][c] << (8 * (w % 3));
                            v[c8 + c] = fma((double)gsum[2], 281474976710656.0,
                                            fma((double)gsum[1], 16777216.0, (double)gsum[0])) *
                                        sc[c8 + c];
                        }
                    }
                    // D is in registers: the MMAs two items on may overwrite it
                    tc_fence_before();
                    mbar_arrive(&dfree[buf]);
                    ++kwork;
                } else {
#pragma unroll
                    for (int c = 0; c < CW; ++c) v[c] = 0.0;
                }
                if (valid) {
#pragma unroll
                    for (int c = 0; c < CW; c += 2) {
                        const int fg = g * NFG + ((c0 + c) >> 1);
                        if (fg < a.nfield)
                            a.partial[(long long)fg * a.nlm + o] = make_double2(v[c], v[c + 1]);
                    }
                }
            } else {
                // one buffer: each column pair is read, combined and stored
                // at once (few registers, two CTAs per SM); D is released
                // after its last pair
                if (work) {
                    if (!__all_sync(0xffffffffu,
                                    mbar_wait(&dfull[0], (uint32_t)(kwork & 1), &abort_flag)))
                        break;
                    tc_fence_after();
                    const uint32_t dcol = (uint32_t)c0;
#pragma unroll 1
                    for (int c = 0; c < CW; c += 2) {
                        uint32_t acc[KW][2];
#pragma unroll
                        for (int w = 0; w < KW; ++w)
                            tmem_ld2(lane_base + dcol + (uint32_t)(w * N + c), acc[w]);
                        tmem_wait_ld();
                        double v2[2];
#pragma unroll
                        for (int e = 0; e < 2; ++e) {
                            long long gsum[3] = {0, 0, 0};
#pragma unroll
                            for (int w = 0; w < KW; ++w)
                                gsum[w / 3] += (long long)(int)acc[w][e] << (8 * (w % 3));
                            v2[e] = fma((double)gsum[2], 281474976710656.0,
                                        fma((double)gsum[1], 16777216.0, (double)gsum[0])) *
                                    (ci[c + e] * kscale);
                        }
                        const int fg = g * NFG + ((c0 + c) >> 1);
                        if (valid && fg < a.nfield)
                            a.partial[(long long)fg * a.nlm + o] = make_double2(v2[0], v2[1]);
                    }
                    tc_fence_before();
                    mbar_arrive(&dfree[0]);
                    ++kwork;
                } else if (valid) {
#pragma unroll 1
                    for (int c = 0; c < CW; c += 2) {
                        const int fg = g * NFG + ((c0 + c) >> 1);
                        if (fg < a.nfield)
                            a.partial[(long long)fg * a.nlm + o] = make_double2(0.0, 0.0);
                    }
                }
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 8) {
        tc_fence_after();
        asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem),
                     "r"(kAlloc));
    }
}
