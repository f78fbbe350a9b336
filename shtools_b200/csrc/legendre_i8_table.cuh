// Table-driven tensor-core Legendre sums: the P_lm digits of a plan are
// computed once and kept in HBM in a layout that is, at once, the K-major A
// operand of the synthesis MMA (M = ring pairs, K = degrees) and the
// MN-major A operand of the analysis MMA (M = degrees, K = ring pairs).
// Each call streams the digits with bulk copies and multiplies them with the
// coefficient (synthesis) or ring-sum (analysis) digits on the tensor cores.
// The table holds the P_lm of the FP64 kernels' one-step recursion rounded to
// the fixed point (same scale and balanced digits as the on-the-fly kernel,
// whose same-parity two-step recursion rounds differently): the analysis of
// the high degrees weighs every P_lm error by the whole field, and the
// two-step values put the lmax-2799 analysis 1e-8 per degree away from FP64.
//
// Table layout.  Work item (m, ring-pair tile pt of 128 pairs) owns the
// super-tiles u0(m, pt) .. nu(m) - 1 of 256 degrees (four K-tiles of 64); a
// super-tile is [parity q][digit i] x 16384 bytes, one digit block holding
// the 128 degrees d of that parity (s = l - m = 256 u + 2 d + q) of the 128
// pairs r, byte (d, r) at
//     (d / 16) * 2048 + (r / 8) * 128 + (r % 8) * 16 + d % 16.
// Every 16-byte row is one pair's 16 consecutive same-parity degrees.  The
// 4096 bytes of degrees d = 32 k .. 32 k + 31 (K-tile 4 u + k) are
// contiguous: the synthesis A tile, K-major with the K core matrices 2048
// bytes apart and the 8-pair groups 128 apart.  Read as M = 128 degrees x
// K = 32 pairs the block is MN-major: degree chunks of 16 at 2048 bytes,
// 8-pair groups at 128.  The leading super-tiles whose digits are all zero
// (P_lm below half a unit of the fixed point: high orders near the poles,
// where P_lm decays like sin^m of the colatitude) are not stored; u0 is the
// first super-tile with a non-zero digit over the item's 128 pairs and both
// parities, so the skipped ones contribute exactly nothing.  Degrees past
// lc in the last super-tile hold finite garbage digits (synthesis: the
// coefficient image is zero there; analysis: those rows are not written).
//
// Synthesis kernel: one CTA per SM, warps 0-7 the epilogue, warp 8 the MMA
// issue, warp 9 the bulk-copy loader.  A stage holds one parity of one
// K-tile: the DA digit tiles of A (from the table) and the DB digit tiles of
// B (coefficient image).  Digit i of A meets the coefficient digits
// j = max(0, WB - i) .. DB - 1 in one MMA whose N' = (DB - j0) N columns land
// on the accumulator's weight blocks w = i + j - WB (no zero padding: the
// window starts at the first kept product).  D = [parity][weight] x N
// INT32 columns (2 KW N <= 512), single-buffered: the MMAs of an item wait
// until the epilogue of the previous item has read D, while the loader keeps
// streaming the next stages.

constexpr int kTabAT = kPairs * 32;              // bytes of one A digit tile (32 degrees)
constexpr int kTabSub = 4;                       // K-tiles per super-tile
constexpr int kTabDigit = kTabSub * kTabAT;      // one digit block: 128 degrees x 128 pairs
__host__ __device__ constexpr int tab_super_bytes(int DA) { return 2 * DA * kTabDigit; }
__host__ __device__ inline int nsuper_of(int lc, int m) {
    return (ntiles_of(lc, m) + kTabSub - 1) / kTabSub;
}
constexpr int kTabSmemBudget = 220 * 1024;
__host__ __device__ constexpr int tab_stage_bytes(int N, int DA) {
    return DA * kTabAT + DA * btile_bytes(N);
}
__host__ __device__ constexpr int tab_stages(int N, int DA) {
    return kTabSmemBudget / tab_stage_bytes(N, DA) > 8 ? 8
                                                       : kTabSmemBudget / tab_stage_bytes(N, DA);
}

struct TabBuildArgs {
    const double2* rec;      // the plan's {beta, D} per packed (l, m) (FP64 path)
    const double* pmm;       // sectoral start values
    const double* rtab;      // u^m / 1e-280 per (m, pair)
    const double* zp;        // z of the northern ring of each pair
    int* u0;                 // per item (m * ptiles + pt): first stored super-tile
    const long long* off;    // per item: super-tiles stored before it (fill pass)
    uint8_t* tab;            // the table (fill pass; zeroed beforehand)
    int lc, npair, ptiles;
    double ascale;
};

// Digit words of one 64-degree K-tile of one pair from the one-step rescaled
// recursion of the FP64 kernels (legendre.cuh: Q(s) = z Q(s-1) - beta(s)
// Q(s-2), P(s) = Q(s) D(s), both values multiplied by D(s) at the end of
// every 16-degree segment), so that the table holds the FP64 path's P_lm
// rounded to the fixed point.  W0 / W1: the even / odd degrees, word i * 8 +
// g of digit i holding the K indices 4 g .. 4 g + 3 of the parity.  q1, q2:
// Q(s-1), Q(s-2) (at s = 0: 0 and the sectoral start, beta(0) = -1).
template <int DA>
__device__ __forceinline__ void tile_digits_1step(const double2* recs, double z, double rp,
                                                  double& q1, double& q2, uint32_t* W0,
                                                  uint32_t* W1) {
    constexpr double kMagic6 = 6896688841130112.0;                // 1.5 * 2^52 + 0x80..80
    constexpr double kMagic = 6755399441055744.0;                 // 1.5 * 2^52
    constexpr unsigned long long kOffset7 = 0xBD48808080808080ull;
#pragma unroll
    for (int g8 = 0; g8 < 8; ++g8) {
        uint32_t lo[2][4], hi[2][4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
            for (int par = 0; par < 2; ++par) {
                const int j = g8 * 8 + 2 * u + par;
                const double2 f = recs[j];
                const double pv = fma(z, q1, -(f.x * q2));
                q2 = q1;
                q1 = pv;
                unsigned long long y;
                if constexpr (DA == 6) {
                    y = (unsigned long long)__double_as_longlong(fma(pv * f.y, rp, kMagic6));
                } else {
                    y = (unsigned long long)__double_as_longlong(fma(pv * f.y, rp, kMagic)) +
                        kOffset7;
                }
                lo[par][u] = (uint32_t)y;
                hi[par][u] = (uint32_t)(y >> 32);
                if ((j & (kRecSegment - 1)) == 0) {
                    q1 *= f.y;
                    q2 *= f.y;
                }
            }
        }
        uint32_t w[DA];
        pack4<DA>(lo[0], hi[0], w);
#pragma unroll
        for (int i = 0; i < DA; ++i) W0[i * 8 + g8] = w[i];
        pack4<DA>(lo[1], hi[1], w);
#pragma unroll
        for (int i = 0; i < DA; ++i) W1[i * 8 + g8] = w[i];
    }
}

// Runs the recursion of item (pt = blockIdx.x, m = blockIdx.y), one thread
// per pair, over all its K-tiles.  FILL = false: records the first
// super-tile with a non-zero digit (nu when there is none).  FILL = true:
// writes the digit tiles of the K-tiles of super-tiles u >= u0 (K-tiles past
// the last degree stay zero).
template <int DA, bool FILL>
__global__ void __launch_bounds__(kPairs) k_i8_table(TabBuildArgs a) {
    const int pt = blockIdx.x, m = blockIdx.y;
    const int r = threadIdx.x;                    // row of the pair in the tile
    const int p = pt * kPairs + r;
    const bool valid = p < a.npair;
    const int nsteps = a.lc - m + 1;
    const int nt = ntiles_of(a.lc, m);
    const int nu = nsuper_of(a.lc, m);
    const long long item = (long long)m * a.ptiles + pt;
    __shared__ double2 recs[kTileDeg];
    __shared__ int tmin;
    const double z = valid ? a.zp[p] : 0.0;
    const double rp = valid ? a.rtab[(long long)m * a.npair + p] * a.ascale : 0.0;
    double q1 = 0.0, q2 = a.pmm[m];
    const double2* rsrc = a.rec + packed_off(m, a.lc);
    int u0 = nu;
    long long base = 0;                           // super-tile u sits at base + u - u0
    if (FILL) {
        u0 = a.u0[item];
        base = a.off[item];
    } else if (threadIdx.x == 0) {
        tmin = nu;
    }
    const long long rowoff = (long long)(r / 8) * 128 + (r % 8) * 16;
    int first = nu;
    for (int t = 0; t < nt; ++t) {
        __syncthreads();                          // the previous tile's entries are consumed
        for (int j = threadIdx.x; j < kTileDeg; j += blockDim.x) {
            const int s = kTileDeg * t + j;
            recs[j] = s < nsteps ? rsrc[s] : make_double2(0.0, 0.0);
        }
        __syncthreads();
        // the recursion advances through every tile, stored or not
        uint32_t W[2][DA * 8];
        tile_digits_1step<DA>(recs, z, rp, q1, q2, W[0], W[1]);
        const int u = t / kTabSub;
        if (!FILL) {
            if (first == nu) {
                uint32_t any = 0u;
#pragma unroll
                for (int k = 0; k < DA * 8; ++k) any |= W[0][k] | W[1][k];
                if (any) first = u;
            }
        } else if (u >= u0) {
            // K-tile t = 4 u + k: degrees d = 32 k .. 32 k + 31 of each parity
            uint8_t* tb = a.tab + (base + u - u0) * (long long)tab_super_bytes(DA) +
                          (t % kTabSub) * kTabAT + rowoff;
#pragma unroll
            for (int q = 0; q < 2; ++q)
#pragma unroll
                for (int i = 0; i < DA; ++i) {
                    uint4* d = reinterpret_cast<uint4*>(tb + (q * DA + i) * kTabDigit);
                    d[0] = make_uint4(W[q][i * 8 + 0], W[q][i * 8 + 1], W[q][i * 8 + 2],
                                      W[q][i * 8 + 3]);
                    d[128] = make_uint4(W[q][i * 8 + 4], W[q][i * 8 + 5], W[q][i * 8 + 6],
                                        W[q][i * 8 + 7]);
                }
        }
    }
    if (!FILL) {
        if (first < nu) atomicMin(&tmin, first);
        __syncthreads();
        if (threadIdx.x == 0) a.u0[item] = tmin;
    }
}

struct TabSynthArgs {
    const uint8_t* tab;      // the table (k_i8_table)
    const long long* off;    // per item (m * ptiles + pt): super-tiles stored before it
    const int* u0;           // per item: first stored super-tile
    const uint8_t* image;    // coefficient image (k_i8_coef_image<N, DB>)
    const long long* toff;   // K-tiles of the image before order m
    const double* colinv;    // 2^-b per (m, group, column)
    double2* spec;           // c2r inputs [field][pair][m][ring]
    int lc, npair, nfield, ngroups, ptiles;
    double ascale;           // 2^a: the A operand's fixed-point scale
};

// D (tmem) += A (smem descriptor) x B (smem descriptor); acc = 0 overwrites D
__device__ __forceinline__ void mma_ss(uint32_t d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                       uint32_t acc) {
    asm volatile(
        "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n\t}" ::"r"(d),
        "l"(adesc), "l"(bdesc), "r"(idesc), "r"(acc)
        : "memory");
}

// work item -> (m, pair tile, field group); m slowest (longest items first),
// the field groups of one (m, pair tile) adjacent so that their reads of the
// same table tiles meet in L2
__device__ __forceinline__ void tab_item_decode(long long i, int ptiles, int ngroups, int* m,
                                                int* pt, int* g) {
    const long long per_m = (long long)ptiles * ngroups;
    *m = (int)(i / per_m);
    const int r = (int)(i - (long long)(*m) * per_m);
    *pt = r / ngroups;
    *g = r - (*pt) * ngroups;
}

constexpr int kTabEpilogue = 256;                // eight epilogue warps
constexpr int kTabThreads = kTabEpilogue + 64;   // + MMA warp + loader warp

template <int N, int DA>
__global__ void __launch_bounds__(kTabThreads, 1) k_legendre_synth_tab(TabSynthArgs a) {
    constexpr int DB = DA;
    constexpr int KW = Digits<DA>::KW;
    constexpr int TOP = DA + DB - 2;
    constexpr int WB = TOP - KW + 1;                 // weight of accumulator block 0
    constexpr int ABYTES = DA * kTabAT;              // A: one parity of a K-tile
    constexpr int BT = btile_bytes(N);
    constexpr int BBYTES = DB * BT;                  // B: one parity of a K-tile
    constexpr int SB = tab_stage_bytes(N, DA);
    constexpr int NS = tab_stages(N, DA);
    constexpr int NFG = N / 2;
    constexpr int CW = N / 2;                        // columns of one epilogue warp
    static_assert(2 * KW * N <= kTmemAlloc, "tensor memory budget");
    static_assert(DB * N <= 256 && N % 16 == 0, "MMA N");
    static_assert(KW == DB + 1 && WB == DA - 2, "weight windows");
    static_assert(SB % 128 == 0 && NS >= 2, "stages");
    extern __shared__ __align__(1024) uint8_t smem_tab[];   // NS x SB
    __shared__ __align__(8) uint64_t full[NS], empty[NS];
    __shared__ __align__(8) uint64_t mdone, dfree;
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
        for (int s = 0; s < NS; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        mbar_init(&mdone, 1);
        mbar_init(&dfree, kTabEpilogue);
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
            long long L = 0;                  // stages issued
            for (long long it = blockIdx.x; it < nitems && !abort_flag; it += gridDim.x) {
                int m, pt, g;
                tab_item_decode(it, a.ptiles, a.ngroups, &m, &pt, &g);
                const long long item = (long long)m * a.ptiles + pt;
                const int nt = ntiles_of(a.lc, m);
                const int t0 = kTabSub * a.u0[item];      // first K-tile stored
                const uint8_t* asrc = a.tab + a.off[item] * (long long)tab_super_bytes(DA);
                const uint8_t* bsrc = a.image + (a.toff[m] * a.ngroups + (long long)g * nt) *
                                                    (long long)bimage_bytes(N, DB);
                const int ns = nt > t0 ? 2 * (nt - t0) : 0;
                for (int s = 0; s < ns && !abort_flag; ++s, ++L) {
                    const int st = (int)(L % NS);
                    if (L >= NS && !mbar_wait(&empty[st], (uint32_t)((L / NS - 1) & 1), &abort_flag))
                        break;
                    const int t = t0 + (s >> 1), q = s & 1;
                    uint8_t* sb = smem_tab + st * SB;
                    mbar_expect_tx(&full[st], (uint32_t)(ABYTES + BBYTES));
                    // the DA digit tiles of (t, q), 16 KB apart in the table
                    const uint8_t* at = asrc + (long long)((t - t0) / kTabSub) * tab_super_bytes(DA) +
                                        (long long)q * DA * kTabDigit + (t % kTabSub) * kTabAT;
#pragma unroll
                    for (int i = 0; i < DA; ++i)
                        bulk_g2s(sb + i * kTabAT, at + (long long)i * kTabDigit, kTabAT, &full[st]);
                    bulk_g2s(sb + ABYTES, bsrc + (long long)t * bimage_bytes(N, DB) + q * BBYTES,
                             BBYTES, &full[st]);
                }
            }
            // drain (bounded): every copy issued has landed before exit
            for (long long T = L - NS < 0 ? 0 : L - NS; T < L; ++T)
                for (unsigned k = 0; k < kSpinLimit; ++k)
                    if (mbar_try(&full[T % NS], (uint32_t)((T / NS) & 1))) break;
        }
        __syncwarp();
    } else if (warp == 8) {
        // ------------------------------------------------ MMA issue
        const uint32_t tm = __shfl_sync(0xffffffffu, tmem, 0);
        const bool leader = elect_one();
        // A tiles: K core matrices 2048 bytes apart, 8-pair groups 128;
        // B (coefficient image): K core matrices 128 apart, column groups 256
        const uint64_t adesc0 = smem_desc(smem_u32(smem_tab), 2048, 128);
        const uint64_t bdesc0 = smem_desc(smem_u32(smem_tab) + ABYTES, 128, 256);
        long long T = 0;                      // stages consumed
        int kwork = 0;                        // items with MMAs
        bool ok = true;
        for (long long it = blockIdx.x; it < nitems && ok; it += gridDim.x) {
            int m, pt, g;
            tab_item_decode(it, a.ptiles, a.ngroups, &m, &pt, &g);
            const long long item = (long long)m * a.ptiles + pt;
            const int nt = ntiles_of(a.lc, m), t0 = kTabSub * a.u0[item];
            const int ns = nt > t0 ? 2 * (nt - t0) : 0;
            if (ns == 0) continue;
            // the epilogue of the previous item has read D
            ok = kwork == 0 || mbar_wait(&dfree, (uint32_t)((kwork - 1) & 1), &abort_flag);
            if (!__all_sync(0xffffffffu, ok)) { ok = false; break; }
            for (int s = 0; s < ns; ++s, ++T) {
                const int st = (int)(T % NS);
                ok = mbar_wait(&full[st], (uint32_t)((T / NS) & 1), &abort_flag);
                if (!__all_sync(0xffffffffu, ok)) { ok = false; break; }
                tc_fence_after();
                const int q = s & 1;
                const bool first = s < 2;
                const uint64_t ad = adesc0 + (uint64_t)((st * SB) >> 4);
                const uint64_t bd = bdesc0 + (uint64_t)((st * SB) >> 4);
                const uint32_t dq = tm + (uint32_t)(q * KW * N);
                // top A digit: coefficient digits 0 .. DB-1 -> blocks 1 .. KW-1
                if (leader)
                    mma_ss(dq + N, ad + (uint64_t)(((DA - 1) * kTabAT) >> 4), bd,
                           idesc_i8(128, DB * N, 1, 1), first ? 0u : 1u);
                // A digit DA-2: block 0 (first product written alone on the
                // item's first stage, which overwrites it) and blocks 1 .. KW-2
                if (first) {
                    if (leader) {
                        mma_ss(dq, ad + (uint64_t)(((DA - 2) * kTabAT) >> 4), bd,
                               idesc_i8(128, N, 1, 1), 0u);
                        mma_ss(dq + N, ad + (uint64_t)(((DA - 2) * kTabAT) >> 4),
                               bd + (uint64_t)(BT >> 4), idesc_i8(128, (DB - 1) * N, 1, 1), 1u);
                    }
                } else if (leader) {
                    mma_ss(dq, ad + (uint64_t)(((DA - 2) * kTabAT) >> 4), bd,
                           idesc_i8(128, DB * N, 1, 1), 1u);
                }
                // lower A digits i: coefficient digits WB - i .. DB-1 -> blocks 0 ..
#pragma unroll
                for (int i = DA - 3; i >= 0; --i) {
                    const int j0 = WB - i;
                    if (leader)
                        mma_ss(dq, ad + (uint64_t)((i * kTabAT) >> 4),
                               bd + (uint64_t)((j0 * BT) >> 4), idesc_i8(128, (DB - j0) * N, 1, 1),
                               1u);
                }
                if (leader) tc_commit(&empty[st]);
                __syncwarp();
            }
            if (!ok) break;
            if (leader) tc_commit(&mdone);
            __syncwarp();
            ++kwork;
        }
        // drain (bounded): the MMAs of the last item
        if (kwork > 0)
            for (unsigned k = 0; k < kSpinLimit; ++k)
                if (mbar_try(&mdone, (uint32_t)((kwork - 1) & 1))) break;
        __syncwarp();
    } else {
        // ------------------------------------------------ epilogue
        const int lq = warp & 3;              // TMEM lane quarter (32 ring pairs)
        const int c0 = (warp >> 2) * CW;      // this warp's columns
        const uint32_t lane_base = tmem + ((uint32_t)(lq * 32) << 16);
        int kwork = 0;
        for (long long it = blockIdx.x; it < nitems && !abort_flag; it += gridDim.x) {
            int m, pt, g;
            tab_item_decode(it, a.ptiles, a.ngroups, &m, &pt, &g);
            const long long item = (long long)m * a.ptiles + pt;
            const bool work = ntiles_of(a.lc, m) > kTabSub * a.u0[item];
            const int p = pt * kPairs + lq * 32 + lane;
            const bool valid = p < a.npair;
            double v[2][CW];
            if (work) {
                double sc[CW];
                {
                    const double* ci = a.colinv + ((long long)m * a.ngroups + g) * N + c0;
                    const double k = pow2i(8 * WB) / a.ascale;
#pragma unroll
                    for (int c = 0; c < CW; ++c) sc[c] = ci[c] * k;
                }
                if (!__all_sync(0xffffffffu,
                                mbar_wait(&mdone, (uint32_t)(kwork & 1), &abort_flag)))
                    break;
                tc_fence_after();
#pragma unroll
                for (int q = 0; q < 2; ++q) {
#pragma unroll
                    for (int c8 = 0; c8 < CW; c8 += 8) {
                        uint32_t acc[KW][8];
#pragma unroll
                        for (int w = 0; w < KW; ++w)
                            tmem_ld8(lane_base + (uint32_t)((q * KW + w) * N + c0 + c8), acc[w]);
                        tmem_wait_ld();
#pragma unroll
                        for (int c = 0; c < 8; ++c) {
                            long long gsum[3] = {0, 0, 0};
#pragma unroll
                            for (int w = 0; w < KW; ++w)
                                gsum[w / 3] += (long long)(int)acc[w][c] << (8 * (w % 3));
                            v[q][c8 + c] = fma((double)gsum[2], 281474976710656.0,
                                               fma((double)gsum[1], 16777216.0, (double)gsum[0])) *
                                           sc[c8 + c];
                        }
                    }
                }
                // D is in registers: the next item's MMAs may overwrite it
                tc_fence_before();
                mbar_arrive(&dfree);
                ++kwork;
            } else {
#pragma unroll
                for (int c = 0; c < CW; ++c) v[0][c] = v[1][c] = 0.0;
            }
            if (valid) {
                const double h = m ? 0.5 : 1.0;
#pragma unroll
                for (int c = 0; c < CW; c += 2) {
                    const int fg = g * NFG + ((c0 + c) >> 1);
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
