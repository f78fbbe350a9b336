// Device code of the longitude FFTs (c2r for synthesis, r2c for analysis),
// shared by the per-plan kernels (kernels.cu) and the batched kernels
// (batch.cu).  Stockham autosort passes ping-pong between two shared
// buffers (per-plan kernels whose buffers exceed shared memory keep them in
// a per-CTA global scratch instead, L2-resident, with the same barriers);
// radix 2, 3, 4, 5, 7, 8, 11, 13 butterflies; Bluestein's algorithm for
// lengths with other prime factors.  Conventions are those of FFTW's
// unnormalised r2c / c2r (src/FFTW3.f95:212-271).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <type_traits>

#include "shtc_internal.cuh"

namespace shtc {

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

// radix-4 DFT of a, b, c, d in place (forward for SIGN < 0)
template <int SIGN>
__device__ __forceinline__ void dft4(double2& a, double2& b, double2& c, double2& d) {
    const double2 s0 = make_double2(a.x + c.x, a.y + c.y);
    const double2 d0 = make_double2(a.x - c.x, a.y - c.y);
    const double2 s1 = make_double2(b.x + d.x, b.y + d.y);
    const double2 d1 = make_double2(b.x - d.x, b.y - d.y);
    // forward: multiply d1 by -i; backward: by +i
    const double2 e = SIGN < 0 ? make_double2(d1.y, -d1.x) : make_double2(-d1.y, d1.x);
    a = make_double2(s0.x + s1.x, s0.y + s1.y);
    c = make_double2(s0.x - s1.x, s0.y - s1.y);
    b = make_double2(d0.x + e.x, d0.y + e.y);
    d = make_double2(d0.x - e.x, d0.y - e.y);
}

// radix-R DFT of v[] in place (R = 2, 4, 8, 10, or an odd prime <= 13)
template <int R, int SIGN>
__device__ __forceinline__ void dft_small(double2* v) {
    if constexpr (R == 10) {
        // two radix-5 DFTs of the even and odd samples, then
        // X_k = E_k + w^k O_k, X_{k+5} = E_k - w^k O_k, w = exp(-+ 2 pi i / 10);
        // cos and sin of 36 and 72 degrees are those of 144 and 72
        double2 e[5], o[5];
#pragma unroll
        for (int q = 0; q < 5; ++q) {
            e[q] = v[2 * q];
            o[q] = v[2 * q + 1];
        }
        dft_small<5, SIGN>(e);
        dft_small<5, SIGN>(o);
        constexpr double c36 = -root_cos(5, 2), s36 = root_sin(5, 2);
        constexpr double c72 = root_cos(5, 1), s72 = root_sin(5, 1);
        constexpr double ck[5] = {1.0, c36, c72, -c72, -c36};
        constexpr double sk[5] = {0.0, s36, s72, s72, s36};
        v[0] = make_double2(e[0].x + o[0].x, e[0].y + o[0].y);
        v[5] = make_double2(e[0].x - o[0].x, e[0].y - o[0].y);
#pragma unroll
        for (int k = 1; k < 5; ++k) {
            const double2 w = make_double2(ck[k], SIGN < 0 ? -sk[k] : sk[k]);
            const double2 t = cmul(o[k], w);
            v[k] = make_double2(e[k].x + t.x, e[k].y + t.y);
            v[k + 5] = make_double2(e[k].x - t.x, e[k].y - t.y);
        }
    } else if (R == 8) {
        // two radix-4 DFTs of the even and odd samples, then
        // X_k = E_k + w^k O_k, X_{k+4} = E_k - w^k O_k, w = exp(-+ 2 pi i / 8)
        double2 e0 = v[0], e1 = v[2], e2 = v[4], e3 = v[6];
        double2 o0 = v[1], o1 = v[3], o2 = v[5], o3 = v[7];
        dft4<SIGN>(e0, e1, e2, e3);
        dft4<SIGN>(o0, o1, o2, o3);
        const double h = 0.70710678118654752440;   // 1/sqrt(2)
        // w^1 o1, w^2 o2, w^3 o3 with w = (1 -+ i)/sqrt(2)
        double2 t1, t2, t3;
        if (SIGN < 0) {
            t1 = make_double2(h * (o1.x + o1.y), h * (o1.y - o1.x));
            t2 = make_double2(o2.y, -o2.x);
            t3 = make_double2(h * (o3.y - o3.x), -h * (o3.x + o3.y));
        } else {
            t1 = make_double2(h * (o1.x - o1.y), h * (o1.y + o1.x));
            t2 = make_double2(-o2.y, o2.x);
            t3 = make_double2(-h * (o3.x + o3.y), h * (o3.x - o3.y));
        }
        v[0] = make_double2(e0.x + o0.x, e0.y + o0.y);
        v[4] = make_double2(e0.x - o0.x, e0.y - o0.y);
        v[1] = make_double2(e1.x + t1.x, e1.y + t1.y);
        v[5] = make_double2(e1.x - t1.x, e1.y - t1.y);
        v[2] = make_double2(e2.x + t2.x, e2.y + t2.y);
        v[6] = make_double2(e2.x - t2.x, e2.y - t2.y);
        v[3] = make_double2(e3.x + t3.x, e3.y + t3.y);
        v[7] = make_double2(e3.x - t3.x, e3.y - t3.y);
    } else if (R == 2) {
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

// v[q] *= w^q, q = 1 .. R-1.  Up to radix 8, w^q = w^(q/2) * w^(q - q/2): a
// product tree of depth log2(R) instead of a chain of R-2 dependent
// multiplications; radix 10 runs the chain, which keeps two powers live
// instead of nine (the 64-register builds)
template <int R, int SIGN>
__device__ __forceinline__ void apply_twiddles(double2* v, double2 w) {
    if constexpr (R >= 10) {
        double2 wq = w;
#pragma unroll
        for (int q = 1; q < R; ++q) {
            v[q] = cmul(v[q], wq);
            if (q + 1 < R) wq = cmul(wq, w);
        }
    } else {
        double2 wp[R];
        wp[1] = w;
#pragma unroll
        for (int q = 2; q < R; ++q) wp[q] = cmul(wp[q / 2], wp[q - q / 2]);
#pragma unroll
        for (int q = 1; q < R; ++q) v[q] = cmul(v[q], wp[q]);
    }
}

// One Stockham pass of radix R from x to y (ping-pong shared buffers).
// tw: this pass's base twiddles, entry k < ns = exp(-2 pi i k/(ns R)); the
// powers w^q, q >= 2, are formed by multiplication.
template <int R, int SIGN>
__device__ __forceinline__ void fft_pass(const double2* __restrict__ x,
                                         double2* __restrict__ y, int M, int ns,
                                         const double2* __restrict__ tw) {
    const int nr = M / R;
    // k = j mod ns, updated incrementally as j advances by blockDim.x
    const int kstep = (int)(blockDim.x % (unsigned)ns);
    int k = (int)(threadIdx.x % (unsigned)ns);
    for (int j = threadIdx.x; j < nr; j += blockDim.x) {
        double2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = x[j + q * nr];
        if (k != 0) apply_twiddles<R, SIGN>(v, twv<SIGN>(tw, k));
        dft_small<R, SIGN>(v);
        const int d = (j - k) * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) y[d + q * ns] = v[q];
        k += kstep;
        if (k >= ns) k -= ns;
    }
}

// The same pass with its inputs read through ld(i) and its outputs written
// through st(i, v): the first pass of a transform reading a grid row or the
// last one writing it, without a staging copy through shared memory.  Reads
// x[j + q nr] and writes y[j' + q ns] are coalesced across the threads for
// each q: the first pass (ns = 1) reads and the last pass (ns = M/R, where
// d = j) writes contiguous runs.
template <int R, int SIGN, typename Ld, typename St>
__device__ __forceinline__ void fft_pass_io(Ld ld, St st, int M, int ns,
                                            const double2* __restrict__ tw) {
    const int nr = M / R;
    const int kstep = (int)(blockDim.x % (unsigned)ns);
    int k = (int)(threadIdx.x % (unsigned)ns);
    for (int j = threadIdx.x; j < nr; j += blockDim.x) {
        double2 v[R];
#pragma unroll
        for (int q = 0; q < R; ++q) v[q] = ld(j + q * nr);
        if (k != 0) apply_twiddles<R, SIGN>(v, twv<SIGN>(tw, k));
        dft_small<R, SIGN>(v);
        const int d = (j - k) * R + k;
#pragma unroll
        for (int q = 0; q < R; ++q) st(d + q * ns, v[q]);
        k += kstep;
        if (k >= ns) k -= ns;
    }
}

template <int SIGN, int MAXR, typename Ld, typename St>
__device__ __forceinline__ void fft_pass_io_r(int r, Ld ld, St st, int M, int ns,
                                              const double2* __restrict__ t) {
    switch (r) {
        case 2: fft_pass_io<2, SIGN>(ld, st, M, ns, t); break;
        case 3: fft_pass_io<3, SIGN>(ld, st, M, ns, t); break;
        case 4: fft_pass_io<4, SIGN>(ld, st, M, ns, t); break;
        case 8: fft_pass_io<8, SIGN>(ld, st, M, ns, t); break;
        case 10:
            if constexpr (MAXR >= 10) fft_pass_io<10, SIGN>(ld, st, M, ns, t);
            break;
        case 5: fft_pass_io<5, SIGN>(ld, st, M, ns, t); break;
        case 7: fft_pass_io<7, SIGN>(ld, st, M, ns, t); break;
        case 11:
            if constexpr (MAXR >= 11) fft_pass_io<11, SIGN>(ld, st, M, ns, t);
            break;
        case 13:
            if constexpr (MAXR >= 13) fft_pass_io<13, SIGN>(ld, st, M, ns, t);
            break;
        default: break;
    }
}

// L2 prefetch of the 128-byte lines of [p, p + bytes), spread over the CTA;
// every address issued lies inside the range's lines
__device__ __forceinline__ void prefetch_l2_range(const void* p, size_t bytes) {
    if (bytes == 0) return;
    const uintptr_t b = (uintptr_t)p;
    const uintptr_t e = b + bytes;
    for (uintptr_t a = (b & ~(uintptr_t)127) + (uintptr_t)threadIdx.x * 128; a < e;
         a += (uintptr_t)blockDim.x * 128) {
        const size_t g = __cvta_generic_to_global((const void*)(a < b ? b : a));
        asm volatile("prefetch.global.L2 [%0];" ::"l"(g));
    }
}

// Runs the passes; the data starts in a, the result pointer is returned.
// MAXR: the largest radix compiled in (8: plans whose factors are all <= 8,
// which need far fewer registers than the radix-11/13 butterflies; 10: the
// same with the radix-10 pass of the long rings).
template <int SIGN, int MAXR = 13>
__device__ __forceinline__ double2* fft_run(double2* a, double2* b, int M, const int* fac,
                            int nfac, const double2* __restrict__ tw,
                            const int* tw_off) {
    int ns = 1;
    for (int i = 0; i < nfac; ++i) {
        __syncthreads();
        const int r = fac[i];
        const double2* t = tw + tw_off[i];
        switch (r) {
            case 2: fft_pass<2, SIGN>(a, b, M, ns, t); break;
            case 3: fft_pass<3, SIGN>(a, b, M, ns, t); break;
            case 4: fft_pass<4, SIGN>(a, b, M, ns, t); break;
            case 8: fft_pass<8, SIGN>(a, b, M, ns, t); break;
            case 10:
                if constexpr (MAXR >= 10) fft_pass<10, SIGN>(a, b, M, ns, t);
                break;
            case 5: fft_pass<5, SIGN>(a, b, M, ns, t); break;
            case 7: fft_pass<7, SIGN>(a, b, M, ns, t); break;
            case 11:
                if constexpr (MAXR >= 11) fft_pass<11, SIGN>(a, b, M, ns, t);
                break;
            case 13:
                if constexpr (MAXR >= 13) fft_pass<13, SIGN>(a, b, M, ns, t);
                break;
            default: break;
        }
        ns *= r;
        double2* sw = a;
        a = b;
        b = sw;
    }
    __syncthreads();
    return a;
}

// Transforms of at least this length read or write their grid rows in the
// first / last pass (fft_run_io); shorter ones stage them through shared
// memory.  On B200 the direct passes made lengths 1440..5600 3-11% faster
// and lengths up to 512 up to 9% (r2c) and 48% (c2r) slower.
constexpr int kFftIoMin = 1024;

// fft_run with the first pass reading through ld(i) (LD) and/or the last
// pass writing through st(i, v) (ST); the middle passes ping-pong between a
// and b as in fft_run.  Needs nfac >= 1.  Returns the buffer that holds the
// result when the last pass does not write through st.
template <int SIGN, int MAXR, bool LD, bool ST, typename Ld, typename St>
__device__ __forceinline__ double2* fft_run_io(double2* a, double2* b, int M, const int* fac,
                                               int nfac, const double2* __restrict__ tw,
                                               const int* tw_off, Ld ld, St st) {
    int ns = 1;
    for (int i = 0; i < nfac; ++i) {
        __syncthreads();
        const int r = fac[i];
        const double2* t = tw + tw_off[i];
        const bool first = LD && i == 0, last = ST && i == nfac - 1;
        if (first || last) {
            const double2* x = a;
            double2* y = b;
            auto lds = [x](int q) { return x[q]; };
            auto sts = [y](int q, double2 v) { y[q] = v; };
            if (first && last) fft_pass_io_r<SIGN, MAXR>(r, ld, st, M, ns, t);
            else if (first) fft_pass_io_r<SIGN, MAXR>(r, ld, sts, M, ns, t);
            else fft_pass_io_r<SIGN, MAXR>(r, lds, st, M, ns, t);
        } else {
            switch (r) {
                case 2: fft_pass<2, SIGN>(a, b, M, ns, t); break;
                case 3: fft_pass<3, SIGN>(a, b, M, ns, t); break;
                case 4: fft_pass<4, SIGN>(a, b, M, ns, t); break;
                case 8: fft_pass<8, SIGN>(a, b, M, ns, t); break;
                case 10:
                    if constexpr (MAXR >= 10) fft_pass<10, SIGN>(a, b, M, ns, t);
                    break;
                case 5: fft_pass<5, SIGN>(a, b, M, ns, t); break;
                case 7: fft_pass<7, SIGN>(a, b, M, ns, t); break;
                case 11:
                    if constexpr (MAXR >= 11) fft_pass<11, SIGN>(a, b, M, ns, t);
                    break;
                case 13:
                    if constexpr (MAXR >= 13) fft_pass<13, SIGN>(a, b, M, ns, t);
                    break;
                default: break;
            }
        }
        ns *= r;
        double2* sw = a;
        a = b;
        b = sw;
    }
    __syncthreads();
    return a;
}

struct FftArgs {
    int n, mode, m, nfac, bluestein, mb, ntw, gmem;
    int fac[kMaxFactors];
    int tw_off[kMaxFactors];
    const double2* tw;
    const double2* twn;
    const double2* chirp;
    const double2* kern;
};

// Complex DFT of length F.m of buf with sign SIGN; buf and tmp each hold
// F.mb (Bluestein) or F.m elements; tw: the plan's twiddles (F.tw, or a
// copy in shared memory).  Returns the pointer holding the result.
template <int SIGN, int MAXR = 13>
__device__ __forceinline__ double2* fft_exec(const FftArgs& F, const double2* tw, double2* buf,
                             double2* tmp) {
    __syncthreads();
    if (!F.bluestein) return fft_run<SIGN, MAXR>(buf, tmp, F.m, F.fac, F.nfac, tw, F.tw_off);
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
    double2* r = fft_run<-1, MAXR>(buf, tmp, mb, F.fac, F.nfac, tw, F.tw_off);
    double2* o = (r == buf) ? tmp : buf;
    for (int t = threadIdx.x; t < mb; t += blockDim.x) {
        double2 kf;
        if (SIGN < 0) {
            kf = F.kern[t];
        } else {
            kf = F.kern[t == 0 ? 0 : mb - t];
            kf.y = -kf.y;
        }
        r[t] = cmul(r[t], kf);
    }
    double2* r2 = fft_run<+1, MAXR>(r, o, mb, F.fac, F.nfac, tw, F.tw_off);
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
template <typename GT, int MAXR = 13>
__device__ __forceinline__ void fft_c2r_body(
    const FftArgs& F, const double2* tw, double2* smem_fft, int job, int f,
    const double2* __restrict__ spec, GT* __restrict__ grid, long long gf,
    long long grs, long long gcs, const int* __restrict__ rowN,
    const int* __restrict__ rowS, const double* __restrict__ wN,
    const double* __restrict__ wS, double wscale, int lc, int npair,
    int extend_col) {
    const int len = F.bluestein ? F.mb : F.m;
    double2* a = smem_fft;
    double2* b = smem_fft + len;
    const int n = F.n;
    if (F.mode == 0) {
        const int p = job;
        const int rN = rowN[p], rS = rowS[p];
        const double2* X = spec + ((long long)f * npair + p) * (lc + 1) * 2;
        const double sN = wN ? wN[p] * wscale : 1.0;
        const double sS = wS ? wS[p] * wscale : 1.0;
        GT* gN = rN >= 0 ? grid + f * gf + rN * grs : nullptr;
        GT* gS = rS >= 0 ? grid + f * gf + rS * grs : nullptr;
        // the spectra are staged in shared memory: each X_k feeds two entries
        // (reading them in the first pass instead, twice, measured 12-14%
        // slower at lmax 1023 and 2047)
        for (int k = threadIdx.x; k < n; k += blockDim.x) a[k] = make_double2(0.0, 0.0);
        __syncthreads();
#pragma unroll 4
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
        if (!F.bluestein && F.nfac > 0 && F.m >= kFftIoMin) {
            // the last pass writes the two rings
            auto st = [&](int j, double2 v) {
                if (gN) gN[j * gcs] = (GT)(v.x * sN);
                if (gS) gS[j * gcs] = (GT)(v.y * sS);
                if (extend_col && j == 0) {
                    if (gN) gN[(long long)n * gcs] = (GT)(v.x * sN);
                    if (gS) gS[(long long)n * gcs] = (GT)(v.y * sS);
                }
            };
            // the last pass writes the two rings
            fft_run_io<+1, MAXR, false, true>(a, b, F.m, F.fac, F.nfac, tw, F.tw_off,
                                               [](int) { return make_double2(0.0, 0.0); }, st);
            return;
        }
        const double2* r = fft_exec<+1, MAXR>(F, tw, a, b);
#pragma unroll 4
        for (int j = threadIdx.x; j < n; j += blockDim.x) {
            const double2 v = r[j];
            if (gN) gN[j * gcs] = (GT)(v.x * sN);
            if (gS) gS[j * gcs] = (GT)(v.y * sS);
        }
        if (extend_col && threadIdx.x == 0) {
            if (gN) gN[(long long)n * gcs] = (GT)(r[0].x * sN);
            if (gS) gS[(long long)n * gcs] = (GT)(r[0].y * sS);
        }
    } else {
        const int p = job >> 1;
        const int h = job & 1;
        const int row = h ? rowS[p] : rowN[p];
        if (row < 0) return;
        const int M = F.m;   // n/2
        const double2* X = spec + ((long long)f * npair + p) * (lc + 1) * 2 + h;
        // Z'_k = (X_k + conj X_{M-k}) + i w^{-k} (X_k - conj X_{M-k}), w = exp(-2 pi i/n)
        auto ld = [&](int k) {
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
            return make_double2(A.x - wb.y, A.y + wb.x);
        };
        const double sc = (h ? (wS ? wS[p] * wscale : 1.0) : (wN ? wN[p] * wscale : 1.0));
        GT* g = grid + f * gf + row * grs;
        using GT2 = typename std::conditional<sizeof(GT) == 8, double2, float2>::type;
        const bool vec = gcs == 1 && ((uintptr_t)g & (2 * sizeof(GT) - 1)) == 0;
        if (!F.bluestein && F.nfac > 0 && F.m >= kFftIoMin) {
            // the last pass writes the ring: sample pair j from element j
            auto st = [&](int j, double2 v) {
                if (vec) {
                    GT2 o;
                    o.x = (GT)(v.x * sc);
                    o.y = (GT)(v.y * sc);
                    reinterpret_cast<GT2*>(g)[j] = o;
                } else {
                    g[(2LL * j) * gcs] = (GT)(v.x * sc);
                    g[(2LL * j + 1) * gcs] = (GT)(v.y * sc);
                }
                if (extend_col && j == 0) g[(long long)n * gcs] = (GT)(v.x * sc);
            };
            // the first pass reads the spectra, the last writes the ring
            fft_run_io<+1, MAXR, true, true>(a, b, M, F.fac, F.nfac, tw, F.tw_off, ld, st);
            return;
        }
#pragma unroll 4
        for (int k = threadIdx.x; k < M; k += blockDim.x) a[k] = ld(k);
        const double2* r = fft_exec<+1, MAXR>(F, tw, a, b);
        if (vec) {
            // contiguous, aligned row: one vector store per sample pair
            GT2* g2 = reinterpret_cast<GT2*>(g);
#pragma unroll 4
            for (int j = threadIdx.x; j < M; j += blockDim.x) {
                const double2 v = r[j];
                GT2 o;
                o.x = (GT)(v.x * sc);
                o.y = (GT)(v.y * sc);
                g2[j] = o;
            }
        } else {
#pragma unroll 4
            for (int j = threadIdx.x; j < M; j += blockDim.x) {
                const double2 v = r[j];
                g[(2LL * j) * gcs] = (GT)(v.x * sc);
                g[(2LL * j + 1) * gcs] = (GT)(v.y * sc);
            }
        }
        if (extend_col && threadIdx.x == 0) g[(long long)n * gcs] = (GT)(r[0].x * sc);
    }
}

// r2c: grid rows -> spec (m = 0..lc), each multiplied by the ring weight
// (times wscale) as (Re, -Im), the reference's fcoef (SHExpandGLQ.f95:535-547).
// fold_extend adds column n into column 0 (adjoint of the extend copy).
// grid2 (nullable): the transform of the pointwise product grid * grid2
// (SHMultiply); the product is formed as each sample is loaded.
template <typename GT, int MAXR = 13>
__device__ __forceinline__ void fft_r2c_body(
    const FftArgs& F, const double2* tw, double2* smem_fft, int job, int f,
    const GT* __restrict__ grid, long long gf, long long grs, long long gcs,
    double2* __restrict__ spec, const int* __restrict__ rowN,
    const int* __restrict__ rowS, const double* __restrict__ wN,
    const double* __restrict__ wS, double wscale, int lc, int npair,
    int fold_extend, const GT* __restrict__ grid2 = nullptr) {
    const int len = F.bluestein ? F.mb : F.m;
    double2* a = smem_fft;
    double2* b = smem_fft + len;
    const int n = F.n;
    if (F.mode == 0) {
        const int p = job;
        const int rN = rowN[p], rS = rowS[p];
        const GT* gN = rN >= 0 ? grid + f * gf + rN * grs : nullptr;
        const GT* gS = rS >= 0 ? grid + f * gf + rS * grs : nullptr;
        // sample j of the two rings as one complex value
        auto ld = [&](int j) {
            double xn = gN ? (double)gN[j * gcs] : 0.0;
            double xs = gS ? (double)gS[j * gcs] : 0.0;
            if (fold_extend && j == 0) {
                if (gN) xn += (double)gN[(long long)n * gcs];
                if (gS) xs += (double)gS[(long long)n * gcs];
            }
            if (grid2) {
                if (gN) xn = xn * (double)(grid2 + f * gf + rN * grs)[j * gcs];
                if (gS) xs = xs * (double)(grid2 + f * gf + rS * grs)[j * gcs];
            }
            return make_double2(xn, xs);
        };
        const double2* r;
        if (!F.bluestein && F.nfac > 0 && F.m >= kFftIoMin) {
            // the first pass reads the rings
            r = fft_run_io<-1, MAXR, true, false>(a, b, F.m, F.fac, F.nfac, tw, F.tw_off, ld,
                                                  [](int, double2) {});
        } else {
#pragma unroll 4
            for (int j = threadIdx.x; j < n; j += blockDim.x) a[j] = ld(j);
            r = fft_exec<-1, MAXR>(F, tw, a, b);
        }
        const double sN = wN ? wN[p] * wscale : wscale;
        const double sS = wS ? wS[p] * wscale : wscale;
        double2* X = spec + ((long long)f * npair + p) * (lc + 1) * 2;
#pragma unroll 4
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
        const GT* g = grid + f * gf + row * grs;
        using GT2 = typename std::conditional<sizeof(GT) == 8, double2, float2>::type;
        const bool vec = gcs == 1 && ((uintptr_t)g & (2 * sizeof(GT) - 1)) == 0;
        // samples 2j and 2j + 1 of the ring as one complex value
        auto ld = [&](int j) {
            double x0, x1;
            if (vec) {
                const GT2 v = reinterpret_cast<const GT2*>(g)[j];
                x0 = (double)v.x;
                x1 = (double)v.y;
            } else {
                x0 = (double)g[(2LL * j) * gcs];
                x1 = (double)g[(2LL * j + 1) * gcs];
            }
            if (fold_extend && j == 0) x0 += (double)g[(long long)n * gcs];
            if (grid2) {
                const GT* g2 = grid2 + f * gf + row * grs;
                x0 = x0 * (double)g2[(2LL * j) * gcs];
                x1 = x1 * (double)g2[(2LL * j + 1) * gcs];
            }
            return make_double2(x0, x1);
        };
        const double2* r;
        if (!F.bluestein && F.nfac > 0 && F.m >= kFftIoMin) {
            // the first pass reads the ring
            r = fft_run_io<-1, MAXR, true, false>(a, b, M, F.fac, F.nfac, tw, F.tw_off, ld,
                                                  [](int, double2) {});
        } else {
#pragma unroll 4
            for (int j = threadIdx.x; j < M; j += blockDim.x) a[j] = ld(j);
            r = fft_exec<-1, MAXR>(F, tw, a, b);
        }
        const double sc = h ? (wS ? wS[p] * wscale : wscale) : (wN ? wN[p] * wscale : wscale);
#pragma unroll 4
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
// complex grids (MakeGridDHC / SHExpandDHC, MakeGridGLQC / SHExpandGLQC)
// ---------------------------------------------------------------------------
// Item (job, u): job = pair*2 + ring (0 north, 1 south), u the user field,
// whose orders +m and -m are the internal fields 2u and 2u+1 of spec.
//
// Synthesis: the Legendre stage wrote spec = (a_m*h, -b_m*h), h = m ? 1/2 : 1,
// the real c2r convention; undone exactly here.  Bin m takes the +m sums, bin
// n-m the -m sums times (-1)^m (MakeGridDHC.f95:612-616); the ring is the
// unnormalised backward DFT of length n.
template <int MAXR = 13>
__device__ __forceinline__ void fft_c2c_synth_body(
    const FftArgs& F, const double2* tw, double2* smem_fft, int job, int u,
    const double2* __restrict__ spec, double2* __restrict__ grid, long long gf,
    long long grs, long long gcs, const int* __restrict__ rowN,
    const int* __restrict__ rowS, int lc, int npair, int extend_col) {
    const int p = job >> 1;
    const int h = job & 1;
    const int row = h ? rowS[p] : rowN[p];
    if (row < 0) return;
    const int len = F.bluestein ? F.mb : F.m;
    double2* a = smem_fft;
    double2* b = smem_fft + len;
    const int n = F.m;
    const long long fstride = (long long)npair * (lc + 1) * 2;
    const double2* Xp = spec + (2LL * u) * fstride + (long long)p * (lc + 1) * 2 + h;
    const double2* Xn = Xp + fstride;
    // bin j: +m sums for j = m <= lc, -m sums for j = n - m (m <= lc; n > 2 lc,
    // so the two ranges do not meet), zero elsewhere
    auto ld = [&](int j) {
        if (j <= lc) {
            const double2 v = Xp[2 * j];
            return j == 0 ? make_double2(v.x, -v.y) : make_double2(2.0 * v.x, -2.0 * v.y);
        }
        const int m = n - j;
        if (m > lc) return make_double2(0.0, 0.0);
        const double2 w = Xn[2 * m];
        const double sg = (m & 1) ? -2.0 : 2.0;
        return make_double2(sg * w.x, -sg * w.y);
    };
    double2* g = grid + u * gf + row * grs;
    if (!F.bluestein && F.nfac > 0 && F.m >= kFftIoMin) {
        // the first pass reads the bins, the last writes the ring
        auto st = [&](int j, double2 v) {
            g[j * gcs] = v;
            if (extend_col && j == 0) g[(long long)n * gcs] = v;
        };
        fft_run_io<+1, MAXR, true, true>(a, b, n, F.fac, F.nfac, tw, F.tw_off, ld, st);
        return;
    }
    for (int j = threadIdx.x; j < n; j += blockDim.x) a[j] = ld(j);
    const double2* r = fft_exec<+1, MAXR>(F, tw, a, b);
#pragma unroll 4
    for (int j = threadIdx.x; j < n; j += blockDim.x) g[j * gcs] = r[j];
    if (extend_col && threadIdx.x == 0) g[(long long)n * gcs] = r[0];
}

// Analysis: the forward DFT of the ring times its weight w/n gives
// fcoef (SHExpandDHC.f95:478); spec of field 2u takes fcoef(m), field 2u+1
// fcoef(n-m) * (-1)^m (SHExpandDHC.f95:596-600), both as (Re, Im).
template <int MAXR = 13>
__device__ __forceinline__ void fft_c2c_anal_body(
    const FftArgs& F, const double2* tw, double2* smem_fft, int job, int u,
    const double2* __restrict__ grid, long long gf, long long grs, long long gcs,
    double2* __restrict__ spec, const int* __restrict__ rowN,
    const int* __restrict__ rowS, const double* __restrict__ wN,
    const double* __restrict__ wS, double wscale, int lc, int npair) {
    const int p = job >> 1;
    const int h = job & 1;
    const int row = h ? rowS[p] : rowN[p];
    const long long fstride = (long long)npair * (lc + 1) * 2;
    double2* Xp = spec + (2LL * u) * fstride + (long long)p * (lc + 1) * 2 + h;
    double2* Xn = Xp + fstride;
    if (row < 0) {
        for (int m = threadIdx.x; m <= lc; m += blockDim.x) {
            Xp[2 * m] = make_double2(0.0, 0.0);
            Xn[2 * m] = make_double2(0.0, 0.0);
        }
        return;
    }
    const int len = F.bluestein ? F.mb : F.m;
    double2* a = smem_fft;
    double2* b = smem_fft + len;
    const int n = F.m;
    const double2* g = grid + u * gf + row * grs;
    const double sc = (h ? wS[p] : wN[p]) * wscale;
    if (!F.bluestein && F.nfac > 0 && F.m >= kFftIoMin) {
        // the first pass reads the ring; the last writes bin i to the +m
        // sums (i = m <= lc) or the -m sums (i = n - m, m <= lc)
        auto ld = [&](int j) { return g[j * gcs]; };
        auto st = [&](int i, double2 z) {
            if (i <= lc) Xp[2 * i] = make_double2(sc * z.x, sc * z.y);
            if (i == 0) {
                Xn[0] = make_double2(0.0, 0.0);
            } else if (n - i <= lc) {
                const int m = n - i;
                const double sg = (m & 1) ? -sc : sc;
                Xn[2 * m] = make_double2(sg * z.x, sg * z.y);
            }
        };
        fft_run_io<-1, MAXR, true, true>(a, b, n, F.fac, F.nfac, tw, F.tw_off, ld, st);
        return;
    }
#pragma unroll 4
    for (int j = threadIdx.x; j < n; j += blockDim.x) a[j] = g[j * gcs];
    const double2* r = fft_exec<-1, MAXR>(F, tw, a, b);
    for (int m = threadIdx.x; m <= lc; m += blockDim.x) {
        const double2 zp = r[m];
        Xp[2 * m] = make_double2(sc * zp.x, sc * zp.y);
        if (m == 0) {
            Xn[0] = make_double2(0.0, 0.0);
        } else {
            const double2 zn = r[n - m];
            const double sg = (m & 1) ? -sc : sc;
            Xn[2 * m] = make_double2(sg * zn.x, sg * zn.y);
        }
    }
}

// L2 prefetch of the input of the c2r item (job, f): the pair's spectrum row
__device__ __forceinline__ void fft_c2r_prefetch(int mode, int job, int f,
                                                 const double2* spec, int lc, int npair) {
    const int p = mode == 0 ? job : (job >> 1);
    prefetch_l2_range(spec + ((long long)f * npair + p) * (lc + 1) * 2,
                      (size_t)(lc + 1) * 2 * sizeof(double2));
}

// L2 prefetch of the input of the r2c item (job, f): its grid rows
// (contiguous rows only)
template <typename GT>
__device__ __forceinline__ void fft_r2c_prefetch(int mode, int n, int job, int f,
                                                 const GT* grid, long long gf, long long grs,
                                                 long long gcs, const int* rowN,
                                                 const int* rowS, int extra) {
    if (gcs != 1) return;
    const size_t bytes = (size_t)(n + extra) * sizeof(GT);
    if (mode == 0) {
        const int rN = rowN[job], rS = rowS[job];
        if (rN >= 0) prefetch_l2_range(grid + f * gf + rN * grs, bytes);
        if (rS >= 0) prefetch_l2_range(grid + f * gf + rS * grs, bytes);
    } else {
        const int p = job >> 1;
        const int row = (job & 1) ? rowS[p] : rowN[p];
        if (row >= 0) prefetch_l2_range(grid + f * gf + row * grs, bytes);
    }
}

// FftArgs of a plan's FFT (kernels.cu)
FftArgs fft_args(const FftPlan& f);

}  // namespace shtc
