// Plan construction for libshtcuda: recursion tables, sectoral start values,
// rescale tables, ring geometry and quadrature weights, FFT plans, and the
// GPU quadrature kernels (PreGLQ, DHaj).
//
// Everything here is computed once per (grid, lmax, lmax_calc, norm,
// csphase) and reused by every transform on that plan; the reference
// recomputes the same tables per call and caches them in threadprivate
// storage keyed on (lmax_comp, norm) (MakeGridDH.f95:258-386).
#include <cuda_runtime.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include <new>
#include <vector>

#include "shtc_internal.cuh"

namespace shtc {

// ---------------------------------------------------------------------------
// recursion tables ff1/ff2 (MakeGridDH.f95:321-381), one thread per (l, m),
// stored in the packed (l, m) order.  sqrt and division are correctly
// rounded in device code, so the entries equal those of a host build.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double sq(int k) { return sqrt((double)k); }

__global__ void k_rec_tables(double2* __restrict__ rec, int lc, int norm) {
    const int m = blockIdx.y;
    const int l = m + blockIdx.x * blockDim.x + threadIdx.x;
    if (l > lc) return;
    double f1 = 0.0, f2 = 0.0;
    if (l > m) {
        if (norm == 1 || norm == 4) {
            if (m == 0) {
                if (l == 1) {
                    f1 = sq(3);
                    f2 = 0.0;
                } else {
                    f1 = __ddiv_rn(__dmul_rn(sq(2 * l - 1), sq(2 * l + 1)), (double)l);
                    f2 = __ddiv_rn(__ddiv_rn(__dmul_rn((double)(l - 1), sq(2 * l + 1)),
                                             sq(2 * l - 3)), (double)l);
                }
            } else {
                // l = m+1 uses the Fortran DO variable left at l-1 (MakeGridDH.f95:341),
                // which is the general expression with m = l-1
                f1 = __ddiv_rn(__ddiv_rn(__dmul_rn(sq(2 * l + 1), sq(2 * l - 1)), sq(l + m)),
                               sq(l - m));
                if (l == m + 1) {
                    f2 = 0.0;
                } else {
                    double t = __dmul_rn(__dmul_rn(sq(2 * l + 1), sq(l - m - 1)), sq(l + m - 1));
                    t = __ddiv_rn(t, sq(2 * l - 3));
                    t = __ddiv_rn(t, sq(l + m));
                    f2 = __ddiv_rn(t, sq(l - m));
                }
            }
        } else if (norm == 2) {
            if (m == 0) {
                if (l == 1) {
                    f1 = 1.0;
                    f2 = 0.0;
                } else {
                    f1 = __ddiv_rn((double)(2 * l - 1), (double)l);
                    f2 = __ddiv_rn((double)(l - 1), (double)l);
                }
            } else {
                f1 = __ddiv_rn(__ddiv_rn((double)(2 * l - 1), sq(l + m)), sq(l - m));
                if (l == m + 1) {
                    f2 = 0.0;
                } else {
                    double t = __dmul_rn(sq(l - m - 1), sq(l + m - 1));
                    t = __ddiv_rn(t, sq(l + m));
                    f2 = __ddiv_rn(t, sq(l - m));
                }
            }
        } else {
            if (m == 0) {
                f1 = __ddiv_rn((double)(2 * l - 1), (double)l);
                f2 = __ddiv_rn((double)(l - 1), (double)l);
            } else {
                f1 = __ddiv_rn((double)(2 * l - 1), (double)(l - m));
                f2 = __ddiv_rn((double)(l + m - 1), (double)(l - m));
            }
        }
    }
    rec[packed_off(m, lc) + (l - m)] = make_double2(f1, f2);
}

// rescaled recursion table (legendre.cuh): from {ff1, ff2} per packed
// (l, m), s = l - m, a = ff1, b = ff2:
//   beta(s) = b(s) / (a(s) a(s-1))  (s >= 2; 0 for s <= 1),
//   D(s)    = a(s0+1) * ... * a(s), s0 = kRecSegment * floor((s-1)/kRecSegment),
//   D(0)    = 1, beta(0) = -1: from the state Q(-1) = 0, Q(-2) = start the
//   step s = 0 yields Q(0) = start exactly, so the analysis runs one
//   uniform step per degree from s = 0.
__global__ void k_rec_scaled(const double2* __restrict__ ff, double2* __restrict__ out,
                             int lc) {
    const int m = blockIdx.y;
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (m + s > lc) return;
    const double2* f = ff + packed_off(m, lc);
    double beta = s == 0 ? -1.0 : 0.0, d = 1.0;
    if (s >= 1) {
        const int s0 = ((s - 1) / kRecSegment) * kRecSegment;
        for (int i = s0 + 1; i <= s; ++i) d *= f[i].x;
        if (s >= 2) beta = f[s].y / (f[s].x * f[s - 1].x);
    }
    out[packed_off(m, lc) + s] = make_double2(beta, d);
}

// rescale table: rtab[m*npair + p] = (1/scalef) * u_p^m by repeated
// multiplication, as rescalem in MakeGridDH.f95:548-552; m = 0 is unscaled.
__global__ void k_rtab(double* __restrict__ rtab, const double* __restrict__ u,
                       int lc, int npair) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npair) return;
    const double up = u[p];
    rtab[p] = 1.0;
    double r = 1.0 / kScalef;
    for (int m = 1; m <= lc; ++m) {
        r = __dmul_rn(r, up);
        rtab[(long long)m * npair + p] = r;
    }
}

// PreGLQ (PreGLQ.f95:93-149): one thread per root, Newton iteration on P_n
// with the same non-fused arithmetic.  The starting guesses
// cos(pi (i - 1/4) / (n + 1/2)) (PreGLQ.f95:101) come from the host's libm,
// as in the reference: the weight is taken at the last-but-one iterate, so a
// start one ulp away can move it by far more than an ulp.  status[0] is set
// to 5 when a root does not converge within itermax iterations.
__global__ void k_preglq(double x1, double x2, int n, const double* __restrict__ guess,
                         double* __restrict__ zero, double* __restrict__ w, int itermax,
                         int* __restrict__ status) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int mroots = (n + 1) / 2;
    if (i > mroots) return;
    const double eps = 1.0e-15;
    const double xm = __ddiv_rn(__dadd_rn(x2, x1), 2.0);
    const double xu = __ddiv_rn(__dsub_rn(x2, x1), 2.0);
    double z = guess[i - 1];
    double p1, p2, p3, pp, z1;
    int iter = 0;
    for (;;) {
        iter = iter + 1;
        p1 = 1.0;
        p2 = 0.0;
        for (int j = 1; j <= n; ++j) {
            p3 = p2;
            p2 = p1;
            p1 = __ddiv_rn(__dsub_rn(__dmul_rn(__dmul_rn((double)(2 * j - 1), z), p2),
                                     __dmul_rn((double)(j - 1), p3)),
                           (double)j);
        }
        pp = __ddiv_rn(__dmul_rn((double)n, __dsub_rn(__dmul_rn(z, p1), p2)),
                       __dsub_rn(__dmul_rn(z, z), 1.0));
        z1 = z;
        z = __dsub_rn(z1, __ddiv_rn(p1, pp));
        if (fabs(__dsub_rn(z, z1)) <= eps) break;
        if (iter > itermax) {
            atomicExch(status, SHTC_ENOZERO);
            return;
        }
    }
    zero[i - 1] = __dadd_rn(xm, __dmul_rn(xu, z));
    zero[n - i] = __dsub_rn(xm, __dmul_rn(xu, z));
    const double wi = __ddiv_rn(__dmul_rn(2.0, xu),
                                __dmul_rn(__dmul_rn(__dsub_rn(1.0, __dmul_rn(z, z)), pp), pp));
    w[i - 1] = wi;
    w[n - i] = wi;
}

// DHaj (DHaj.f95:91-105): one thread per latitude j.
__global__ void k_dhaj(int n, double* __restrict__ aj, int extend) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    const double pi = 3.141592653589793238462643383279502884;
    if (j < n) {
        double sum1 = 0.0;
        for (int l = 0; l <= n / 2 - 1; ++l) {
            const double a = __ddiv_rn(__dmul_rn(__dmul_rn((double)(2 * l + 1), pi), (double)j),
                                       (double)n);
            sum1 = __dadd_rn(sum1, __ddiv_rn(sin(a), (double)(2 * l + 1)));
        }
        const double s = sin(__ddiv_rn(__dmul_rn(pi, (double)j), (double)n));
        aj[j] = __ddiv_rn(__dmul_rn(__dmul_rn(sum1, s), sqrt(8.0)), (double)n);
    }
    if (extend && j == n) aj[n] = 0.0;
}

// ring weights of the analysis from DH a_j or GLQ w_i
//   DH : sqrt(2 pi) * (a_j * sqrt(4 pi))   (SHExpandDH.f95:294, 470)
//   GLQ: (2 * w_i) * pi                     (SHExpandGLQ.f95:535)
__global__ void k_ring_weights(const double* __restrict__ q,
                               const int* __restrict__ arowN,
                               const int* __restrict__ arowS,
                               double* __restrict__ wN, double* __restrict__ wS,
                               int npair, int kind) {
    const int p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= npair) return;
    const double pi = 3.141592653589793238462643383279502884;
    const int rN = arowN[p], rS = arowS[p];
    double a = 0.0, b = 0.0;
    if (kind == SHTC_GRID_DH) {
        const double s4 = sqrt(4.0 * pi), s2 = sqrt(2.0 * pi);
        if (rN >= 0) a = __dmul_rn(s2, __dmul_rn(q[rN], s4));
        if (rS >= 0) b = __dmul_rn(s2, __dmul_rn(q[rS], s4));
    } else {
        if (rN >= 0) a = __dmul_rn(__dmul_rn(2.0, q[rN]), pi);
        if (rS >= 0) b = __dmul_rn(__dmul_rn(2.0, q[rS]), pi);
    }
    wN[p] = a;
    wS[p] = b;
}

// ---------------------------------------------------------------------------
// FFT plan
// ---------------------------------------------------------------------------
// Pass order: the odd radices first, then 8, 4, 2.  A Stockham pass writes
// y[(j - k) R + k + q ns], k = j mod ns: with ns = 1 consecutive threads
// write R elements apart, an R-way shared-memory bank conflict for R = 8
// (16-byte elements, 8 threads per 128-byte wavefront) but none for odd R;
// with ns >= 3 the writes of consecutive threads are contiguous runs.
// with pair10, factors 5 and 2 are merged into radix-10 passes where that
// lowers the number of passes (5600 = 7 * 10 * 10 * 8: four passes instead
// of five, and no pass of more than 1024 butterflies).  Passes run odd
// radices first, then 10, 8, 4, 2: with the radix-7 pass first the lmax
// 2799 FFTs were 3-7% faster than with the radix-10 passes first.
static int factor_len(int n, int* fac, bool pair10 = false) {
    int k = 0;
    int m = n;
    int p2 = 0;
    while (m % 2 == 0) { m /= 2; ++p2; }
    auto groups2 = [](int e) { return e / 3 + (e % 3 ? 1 : 0); };
    int n5 = 0;
    {
        int r = m;
        while (r % 5 == 0) { r /= 5; ++n5; }
    }
    int tens = 0;
    if (pair10) {
        for (int t = 1; t <= std::min(n5, p2); ++t)
            if (groups2(p2 - t) < groups2(p2 - tens)) tens = t;
    }
    p2 -= tens;
    int t10 = 0;
    for (int p = 3; p <= m; p += 2) {
        while (m % p == 0) {
            if (p > kMaxRadix || (p != 3 && p != 5 && p != 7 && p != 11 && p != 13))
                return -1;
            if (p == 5 && tens > 0) {
                --tens;
                ++t10;
            } else {
                fac[k++] = p;
            }
            m /= p;
        }
    }
    while (t10-- > 0) fac[k++] = 10;
    while (p2 >= 3) { fac[k++] = 8; p2 -= 3; }
    if (p2 == 2) fac[k++] = 4;
    if (p2 == 1) fac[k++] = 2;
    return k;
}

// Base twiddles of every Stockham pass, pass after pass: for the pass of
// radix R applied after sub-transforms of length ns, entry k < ns holds
// w_k = exp(-2 pi i k / (ns R)); the butterfly forms w_k^q, q = 2..R-1, by
// repeated complex multiplication (a few ulp for R <= 13).  Threads of
// consecutive k read consecutive entries.
static int pass_twiddles(const int* fac, int nfac, std::vector<double2>& out, int* off) {
    out.clear();
    const long double tp = 2.0L * 3.141592653589793238462643383279502884L;
    int ns = 1;
    for (int i = 0; i < nfac; ++i) {
        const int R = fac[i];
        off[i] = (int)out.size();
        for (int k = 0; k < ns; ++k) {
            const long double a = tp * (long double)k / (long double)((long long)ns * R);
            out.push_back(make_double2((double)cosl(a), (double)(-sinl(a))));
        }
        ns *= R;
    }
    return (int)out.size();
}

int build_fft_plan(FftPlan* f, int n, int cplx, cudaStream_t st) {
    memset(f, 0, sizeof(*f));
    f->n = n;
    f->mode = cplx ? 2 : ((n % 2 == 0) ? 1 : 0);
    f->m = f->mode == 1 ? n / 2 : n;
    int fac[kMaxFactors];
    int nf = factor_len(f->m, fac);
    std::vector<double2> tw, twn, chirp, kern;
    if (nf < 0) {
        f->bluestein = 1;
        // convolution length: the smallest 7-smooth mb >= 2m - 1 (Stockham
        // radices 2, 3, 4, 5, 7), on average ~30% below the next power of two
        int mb = 2 * f->m - 1;
        for (;; ++mb) {
            int r = mb;
            for (int p : {2, 3, 5, 7})
                while (r % p == 0) r /= p;
            if (r == 1) break;
        }
        f->mb = mb;
        nf = factor_len(mb, fac);
        chirp.resize(f->m);
        const long double pi = 3.141592653589793238462643383279502884L;
        for (long long t = 0; t < f->m; ++t) {
            const long long r = (t * t) % (2LL * f->m);
            const long double a = pi * (long double)r / (long double)f->m;
            chirp[t] = make_double2((double)cosl(a), (double)(-sinl(a)));
        }
        // FFT_mb of the kernel conj(c_t), t in (-m, m), computed on the host
        // by a direct O(mb * m) sum in long double (plan time only)
        std::vector<long double> kr(mb, 0.0L), ki(mb, 0.0L);
        for (int t = 0; t < f->m; ++t) {
            kr[t] = chirp[t].x; ki[t] = -chirp[t].y;
            if (t) { kr[mb - t] = chirp[t].x; ki[mb - t] = -chirp[t].y; }
        }
        kern.resize(mb);
        const long double tp = 2.0L * pi;
        std::vector<long double> cr(mb), ci(mb);
        for (int t = 0; t < mb; ++t) {
            cr[t] = cosl(tp * t / mb);
            ci[t] = -sinl(tp * t / mb);
        }
        for (int k = 0; k < mb; ++k) {
            long double sr = 0.0L, si = 0.0L;
            for (int t = 0; t < mb; ++t) {
                if (kr[t] == 0.0L && ki[t] == 0.0L) continue;
                const int idx = (int)(((long long)k * t) % mb);
                sr += kr[t] * cr[idx] - ki[t] * ci[idx];
                si += kr[t] * ci[idx] + ki[t] * cr[idx];
            }
            kern[k] = make_double2((double)sr, (double)si);
        }
    }
    if (nf > kMaxFactors) return SHTC_EUNSUP;
    int maxsmem = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&maxsmem, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    // rings of more than 4096 points held in shared memory run in
    // 1024-thread CTAs, whose passes are short of butterflies with radices
    // below 8: they take the radix-10 passes
    if (!f->bluestein && f->m > 4096 && 2 * (size_t)f->m * sizeof(double2) <= (size_t)maxsmem)
        nf = factor_len(f->m, fac, true);
    f->ntw = pass_twiddles(fac, nf, tw, f->tw_off);
    f->nfac = nf;
    for (int i = 0; i < nf; ++i) f->fac[i] = fac[i];
    if (f->mode == 1) {
        twn.resize(n / 2);
        const long double tp = 2.0L * 3.141592653589793238462643383279502884L;
        for (int k = 0; k < n / 2; ++k) {
            const long double a = tp * (long double)k / (long double)n;
            twn[k] = make_double2((double)cosl(a), (double)(-sinl(a)));
        }
    }
    const int len = f->bluestein ? f->mb : f->m;
    // two shared buffers: Stockham passes ping-pong between them; the
    // per-plan kernels also keep the twiddles in shared memory when they fit
    f->smem_data = 2 * (size_t)len * sizeof(double2);
    f->threads = len > 2048 ? 512 : (len > 512 ? 256 : 128);
    if (maxsmem > 0 && f->smem_data > (size_t)maxsmem) {
        // too long for shared memory: the data buffers go to a global scratch
        // (one pair per persistent CTA, L2-resident), the twiddles stay in
        // shared memory when they fit
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        f->gmem = 1;
        f->gmem_ctas = sms > 0 ? sms : 1;
        const size_t tb = (size_t)f->ntw * sizeof(double2);
        f->tw_smem = tb <= (size_t)maxsmem ? 1 : 0;
        f->smem = f->tw_smem ? tb : 0;
    } else {
        const size_t with_tw = f->smem_data + (size_t)f->ntw * sizeof(double2);
        f->tw_smem = (maxsmem > 0 && with_tw <= (size_t)maxsmem) ? 1 : 0;
        f->smem = f->tw_smem ? with_tw : f->smem_data;
    }
    auto up = [&](double2** d, const std::vector<double2>& h) -> int {
        if (h.empty()) { *d = nullptr; return SHTC_OK; }
        if (cudaMalloc((void**)d, h.size() * sizeof(double2)) != cudaSuccess) return SHTC_EALLOC;
        return map_cuda(cudaMemcpyAsync(*d, h.data(), h.size() * sizeof(double2),
                                        cudaMemcpyHostToDevice, st));
    };
    int rc;
    if ((rc = up(&f->d_tw, tw))) return rc;
    if ((rc = up(&f->d_twn, twn))) return rc;
    if ((rc = up(&f->d_chirp, chirp))) return rc;
    if ((rc = up(&f->d_kern, kern))) return rc;
    // the host vectors are released on return: make the copies complete first
    return map_cuda(cudaStreamSynchronize(st));
}

void free_fft_plan(FftPlan* f) {
    cudaFree(f->d_tw);
    cudaFree(f->d_twn);
    cudaFree(f->d_chirp);
    cudaFree(f->d_kern);
    f->d_tw = f->d_twn = f->d_chirp = f->d_kern = nullptr;
}

}  // namespace shtc

using namespace shtc;

// ---------------------------------------------------------------------------
// plan creation (C ABI)
// ---------------------------------------------------------------------------
static void plan_free_tables(shtc_plan* P) {
    free_i8_table(P);
    cudaFree(P->d_i8_toff);
    cudaFree(P->d_i8_uoff);
    cudaFree(P->d_i8_rec2);
    cudaFree(P->d_rec);
    cudaFree(P->d_pmm);
    cudaFree(P->d_rtab);
    cudaFree(P->d_z);
    cudaFree(P->d_rowN);
    cudaFree(P->d_rowS);
    cudaFree(P->d_arowN);
    cudaFree(P->d_arowS);
    cudaFree(P->d_wN);
    cudaFree(P->d_wS);
    cudaFree(P->d_nrm);
    free_fft_plan(&P->fft);
}

// sectoral start values, replicating the running product of the reference
// (MakeGridDH.f95:542-603): pm2 for m < lc, the final pmm (without the
// rescale factor) for m = lc, and P00 for m = 0.
// Complex transforms start the sectoral recursion without the real
// harmonics' sqrt(2) (MakeGridDHC.f95:442-446).
static void host_pmm(int lc, int norm, int csphase, int cplx, double* out) {
    const double pi = acos(-1.0);
    out[0] = norm == 4 ? 1.0 / sqrt(4.0 * pi) : 1.0;
    if (lc == 0) return;
    double pmm;
    const double s2 = cplx ? 1.0 : sqrt(2.0);
    switch (norm) {
        case 1: case 2: pmm = cplx ? kScalef : s2 * kScalef; break;
        case 3: pmm = kScalef; break;
        default: pmm = cplx ? kScalef / sqrt(4.0 * pi) : s2 * kScalef / sqrt(4.0 * pi); break;
    }
    for (int m = 1; m <= lc - 1; ++m) {
        switch (norm) {
            case 1: case 4:
                pmm = csphase * pmm * sqrt((double)(2 * m + 1)) / sqrt((double)(2 * m));
                out[m] = pmm;
                break;
            case 2:
                pmm = csphase * pmm * sqrt((double)(2 * m + 1)) / sqrt((double)(2 * m));
                out[m] = pmm / sqrt((double)(2 * m + 1));
                break;
            default:
                pmm = csphase * pmm * (double)(2 * m - 1);
                out[m] = pmm;
                break;
        }
    }
    switch (norm) {
        case 1: case 4:
            out[lc] = csphase * pmm * sqrt((double)(2 * lc + 1)) / sqrt((double)(2 * lc));
            break;
        case 2:
            out[lc] = csphase * pmm / sqrt((double)(2 * lc));
            break;
        default:
            out[lc] = csphase * pmm * (double)(2 * lc - 1);
            break;
    }
}

// norm-3 divisors of SHExpandDH.f95:685-700 per packed (l, m); the complex
// transforms omit the halving for m >= 1 (SHExpandDHC.f95:708-720)
static void host_nrm3(int lc, int cplx, std::vector<double>& out) {
    const double pi = acos(-1.0);
    out.assign((size_t)(lc + 1) * (lc + 2) / 2, 1.0);
    for (int l = 0; l <= lc; ++l) {
        double prod = 4 * pi / (double)(2 * l + 1);
        out[packed_off(0, lc) + l] = prod;
        if (!cplx) prod = prod / 2.0;
        for (int m = 1; m <= l - 1; ++m) {
            prod = prod * (l + m) * (l - m + 1);
            out[packed_off(m, lc) + (l - m)] = prod;
        }
        if (l != 0) out[packed_off(l, lc)] = prod * 2 * l;
    }
}

template <typename Tp>
static int dev_upload(Tp** d, const Tp* h, size_t count, cudaStream_t st,
                      size_t* acc) {
    if (cudaMalloc((void**)d, count * sizeof(Tp)) != cudaSuccess) {
        *d = nullptr;
        return SHTC_EALLOC;
    }
    *acc += count * sizeof(Tp);
    if (h) return map_cuda(cudaMemcpyAsync(*d, h, count * sizeof(Tp),
                                           cudaMemcpyHostToDevice, st));
    return SHTC_OK;
}

// Common part: kind, lmax, lc, norm, csphase, sampling, extend set; z/u given
// on the host (with exact equator values); weights source q on the device.
static int plan_finish(shtc_plan* P, const std::vector<double>& z,
                       const std::vector<double>& u,
                       const std::vector<int>& rowN,
                       const std::vector<int>& rowS,
                       const std::vector<int>& arowN,
                       const std::vector<int>& arowS, const double* d_q,
                       cudaStream_t st) {
    int rc;
    const int lc = P->lc, np = P->npair;
    P->nlm = (long long)(lc + 1) * (lc + 2) / 2;
    size_t acc = 0;
    std::vector<double> pmm(lc + 1);
    host_pmm(lc, P->norm, P->csphase, P->cplx, pmm.data());
    double* d_u = nullptr;
    double2* d_ff = nullptr;   // {ff1, ff2}, only needed to build d_rec
    if ((rc = dev_upload(&P->d_rec, (const double2*)nullptr, (size_t)P->nlm, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_pmm, pmm.data(), (size_t)lc + 1, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_rtab, (const double*)nullptr, (size_t)(lc + 1) * np, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_z, z.data(), (size_t)np, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_rowN, rowN.data(), (size_t)np, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_rowS, rowS.data(), (size_t)np, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_arowN, arowN.data(), (size_t)np, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_arowS, arowS.data(), (size_t)np, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_wN, (const double*)nullptr, (size_t)np, st, &acc))) return rc;
    if ((rc = dev_upload(&P->d_wS, (const double*)nullptr, (size_t)np, st, &acc))) return rc;
    if (P->norm == 3) {
        std::vector<double> n3;
        host_nrm3(lc, P->cplx, n3);
        if ((rc = dev_upload(&P->d_nrm, n3.data(), n3.size(), st, &acc))) return rc;
        if ((rc = map_cuda(cudaStreamSynchronize(st)))) return rc;
    }
    if ((rc = dev_upload(&d_u, u.data(), (size_t)np, st, &acc))) return rc;
    if ((rc = dev_upload(&d_ff, (const double2*)nullptr, (size_t)P->nlm, st, &acc))) {
        cudaFree(d_u);
        return rc;
    }
    {
        dim3 g((lc + 1 + 127) / 128, lc + 1);
        k_rec_tables<<<g, 128, 0, st>>>(d_ff, lc, P->norm);
        k_rec_scaled<<<g, 128, 0, st>>>(d_ff, P->d_rec, lc);
        k_rtab<<<(np + 127) / 128, 128, 0, st>>>(P->d_rtab, d_u, lc, np);
        k_ring_weights<<<(np + 127) / 128, 128, 0, st>>>(d_q, P->d_arowN, P->d_arowS,
                                                         P->d_wN, P->d_wS, np, P->kind);
    }
    rc = map_cuda(cudaGetLastError());
    // host vectors (z, u, rows, pmm) die on return: finish the copies
    cudaError_t e = cudaStreamSynchronize(st);
    cudaFree(d_u);
    cudaFree(d_ff);
    acc -= (size_t)np * sizeof(double) + (size_t)P->nlm * sizeof(double2);
    if (rc) return rc;
    if (e != cudaSuccess) return SHTC_ECUDA;
    if ((rc = build_fft_plan(&P->fft, P->nlon, P->cplx, st))) return rc;
    size_t fb = 0;
    const int len = P->fft.bluestein ? P->fft.mb : P->fft.m;
    fb += (size_t)len * sizeof(double2);
    if (P->fft.mode == 1) fb += (size_t)(P->nlon / 2) * sizeof(double2);
    if (P->fft.bluestein) fb += (size_t)(P->fft.m + P->fft.mb) * sizeof(double2);
    P->device_bytes = acc + fb;
    cudaGetDevice(&P->device);
    return SHTC_OK;
}

static int create_dh(shtc_plan** out, int lmax, int sampling, int lmax_calc, int norm,
                     int csphase, int extend, int cplx, void* stream) {
    if (!out) return SHTC_EHANDLE;
    *out = nullptr;
    if (lmax < 0) return SHTC_EBOUND;
    if (sampling != 1 && sampling != 2) return SHTC_EBOUND;
    if (extend != 0 && extend != 1) return SHTC_EBOUND;
    if (norm < 1 || norm > 4) return SHTC_EBOUND;
    if (csphase != 1 && csphase != -1) return SHTC_EBOUND;
    if (lmax_calc > lmax) return SHTC_EBOUND;
    cudaStream_t st = (cudaStream_t)stream;
    shtc_plan* P = new (std::nothrow) shtc_plan();
    if (!P) return SHTC_EALLOC;
    memset(P, 0, sizeof(*P));
    P->kind = SHTC_GRID_DH;
    P->cplx = cplx;
    P->lmax = lmax;
    P->lc = lmax_calc < 0 ? lmax : lmax_calc;
    P->norm = norm;
    P->csphase = csphase;
    P->sampling = sampling;
    P->extend = extend;
    const int n = 2 * lmax + 2;
    P->nlat = n;
    P->nlon = sampling * n;
    P->nlat_out = n + extend;
    P->nlon_out = sampling * n + extend;
    P->npair = n / 2 + 1;
    const int np = P->npair;
    std::vector<double> z(np), u(np);
    std::vector<int> rowN(np), rowS(np), arowN(np), arowS(np);
    const double pi = acos(-1.0);
    for (int p = 0; p < np; ++p) {
        if (p == n / 2) {
            z[p] = 0.0;
            u[p] = 1.0;
        } else {
            const double theta = pi * (double)p / (double)n;   // MakeGridDH.f95:508
            z[p] = cos(theta);
            u[p] = sqrt((1.0 - z[p]) * (1.0 + z[p]));
        }
        rowN[p] = p;
        arowN[p] = p;
        if (p == n / 2) {
            rowS[p] = -1;
            arowS[p] = -1;
        } else if (p == 0) {
            rowS[p] = extend ? n : -1;
            arowS[p] = -1;
        } else {
            rowS[p] = n - p;
            arowS[p] = n - p;
        }
    }
    double* d_aj = nullptr;
    int rc = SHTC_OK;
    if (cudaMalloc((void**)&d_aj, sizeof(double) * (size_t)(n + 1)) != cudaSuccess) rc = SHTC_EALLOC;
    if (!rc) {
        k_dhaj<<<(n + 1 + 127) / 128, 128, 0, st>>>(n, d_aj, 0);
        rc = map_cuda(cudaGetLastError());
    }
    if (!rc) rc = plan_finish(P, z, u, rowN, rowS, arowN, arowS, d_aj, st);
    cudaFree(d_aj);
    if (rc) {
        plan_free_tables(P);
        delete P;
        return rc;
    }
    *out = P;
    return SHTC_OK;
}

extern "C" int shtc_plan_create_dh(shtc_plan** out, int lmax, int sampling,
                                   int lmax_calc, int norm, int csphase,
                                   int extend, void* stream) {
    return create_dh(out, lmax, sampling, lmax_calc, norm, csphase, extend, 0, stream);
}

extern "C" int shtc_plan_create_dhc(shtc_plan** out, int lmax, int sampling,
                                    int lmax_calc, int norm, int csphase,
                                    int extend, void* stream) {
    return create_dh(out, lmax, sampling, lmax_calc, norm, csphase, extend, 1, stream);
}

extern "C" int shtc_preglq(double x1, double x2, int n, double* zero, double* w,
                           void* stream);

static int create_glq(shtc_plan** out, int lmax, const double* zero_host,
                      const double* w_host, int lmax_calc, int norm, int csphase,
                      int extend, int cplx, void* stream) {
    if (!out) return SHTC_EHANDLE;
    *out = nullptr;
    if (lmax < 0) return SHTC_EBOUND;
    if (extend != 0 && extend != 1) return SHTC_EBOUND;
    if (norm < 1 || norm > 4) return SHTC_EBOUND;
    if (csphase != 1 && csphase != -1) return SHTC_EBOUND;
    if (lmax_calc > lmax) return SHTC_EBOUND;
    cudaStream_t st = (cudaStream_t)stream;
    shtc_plan* P = new (std::nothrow) shtc_plan();
    if (!P) return SHTC_EALLOC;
    memset(P, 0, sizeof(*P));
    P->kind = SHTC_GRID_GLQ;
    P->cplx = cplx;
    P->lmax = lmax;
    P->lc = lmax_calc < 0 ? lmax : lmax_calc;
    P->norm = norm;
    P->csphase = csphase;
    P->sampling = 1;
    P->extend = extend;
    const int nlat = lmax + 1;
    P->nlat = nlat;
    P->nlon = 2 * lmax + 1;
    P->nlat_out = nlat;
    P->nlon_out = 2 * lmax + 1 + extend;
    P->npair = (nlat + 1) / 2;
    const int np = P->npair;
    int rc = SHTC_OK;
    // nodes and weights: from the caller, or from the GPU PreGLQ
    double *d_zero = nullptr, *d_w = nullptr;
    std::vector<double> zh(nlat), wh(nlat);
    if (cudaMalloc((void**)&d_zero, sizeof(double) * nlat) != cudaSuccess ||
        cudaMalloc((void**)&d_w, sizeof(double) * nlat) != cudaSuccess)
        rc = SHTC_EALLOC;
    if (!rc) {
        if (zero_host && w_host) {
            memcpy(zh.data(), zero_host, sizeof(double) * nlat);
            memcpy(wh.data(), w_host, sizeof(double) * nlat);
        } else {
            rc = shtc_preglq(-1.0, 1.0, nlat, d_zero, d_w, stream);
            if (!rc) rc = map_cuda(cudaMemcpyAsync(zh.data(), d_zero, sizeof(double) * nlat,
                                                   cudaMemcpyDeviceToHost, st));
            if (!rc) rc = map_cuda(cudaMemcpyAsync(wh.data(), d_w, sizeof(double) * nlat,
                                                   cudaMemcpyDeviceToHost, st));
            if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
            if (zero_host && !rc) memcpy(zh.data(), zero_host, sizeof(double) * nlat);
            if (w_host && !rc) memcpy(wh.data(), w_host, sizeof(double) * nlat);
        }
    }
    if (!rc) rc = map_cuda(cudaMemcpyAsync(d_w, wh.data(), sizeof(double) * nlat,
                                           cudaMemcpyHostToDevice, st));
    std::vector<double> z(np), u(np);
    std::vector<int> rowN(np), rowS(np);
    for (int p = 0; p < np; ++p) {
        const int ps = nlat - 1 - p;
        rowN[p] = p;
        if (ps == p) {
            rowS[p] = -1;
            z[p] = 0.0;            // equator branch, MakeGridGLQ.f95:472-474
            u[p] = 1.0;
        } else {
            rowS[p] = ps;
            z[p] = zh[p];
            u[p] = sqrt((1.0 - z[p]) * (1.0 + z[p]));
        }
    }
    if (!rc) rc = plan_finish(P, z, u, rowN, rowS, rowN, rowS, d_w, st);
    cudaFree(d_zero);
    cudaFree(d_w);
    if (rc) {
        plan_free_tables(P);
        delete P;
        return rc;
    }
    *out = P;
    return SHTC_OK;
}

extern "C" int shtc_plan_create_glq(shtc_plan** out, int lmax,
                                    const double* zero_host,
                                    const double* w_host, int lmax_calc,
                                    int norm, int csphase, int extend,
                                    void* stream) {
    return create_glq(out, lmax, zero_host, w_host, lmax_calc, norm, csphase, extend, 0,
                      stream);
}

extern "C" int shtc_plan_create_glqc(shtc_plan** out, int lmax,
                                     const double* zero_host,
                                     const double* w_host, int lmax_calc,
                                     int norm, int csphase, int extend,
                                     void* stream) {
    return create_glq(out, lmax, zero_host, w_host, lmax_calc, norm, csphase, extend, 1,
                      stream);
}

extern "C" int shtc_plan_destroy(shtc_plan* P) {
    if (!P) return SHTC_EHANDLE;
    plan_free_tables(P);
    delete P;
    return SHTC_OK;
}

extern "C" int shtc_preglq(double x1, double x2, int n, double* zero, double* w,
                           void* stream) {
    if (n < 1 || !zero || !w) return SHTC_EBOUND;
    cudaStream_t st = (cudaStream_t)stream;
    const int mroots = (n + 1) / 2;
    // starting guesses with the host libm, in the reference's operation order
    std::vector<double> guess(mroots);
    const double pi = acos(-1.0);
    for (int i = 1; i <= mroots; ++i) guess[i - 1] = cos(pi * (i - 0.25) / (n + 0.5));
    // one allocation: the status word, then the guesses (8-byte aligned)
    void* d_buf = nullptr;
    if (cudaMalloc(&d_buf, sizeof(double) * (1 + mroots)) != cudaSuccess) return SHTC_EALLOC;
    int* d_status = (int*)d_buf;
    double* d_guess = (double*)d_buf + 1;
    int rc = map_cuda(cudaMemsetAsync(d_status, 0, sizeof(int), st));
    if (!rc) rc = map_cuda(cudaMemcpyAsync(d_guess, guess.data(), sizeof(double) * mroots,
                                           cudaMemcpyHostToDevice, st));
    if (!rc) rc = map_cuda(cudaMemsetAsync(zero, 0, sizeof(double) * n, st));
    if (!rc) rc = map_cuda(cudaMemsetAsync(w, 0, sizeof(double) * n, st));
    if (!rc) {
        k_preglq<<<(mroots + 63) / 64, 64, 0, st>>>(x1, x2, n, d_guess, zero, w, 1000,
                                                    d_status);
        rc = map_cuda(cudaGetLastError());
    }
    int hs = 0;
    if (!rc) rc = map_cuda(cudaMemcpyAsync(&hs, d_status, sizeof(int), cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    else cudaStreamSynchronize(st);
    cudaFree(d_buf);
    if (rc) return rc;
    return hs;
}

extern "C" int shtc_dhaj(int n, double* aj, int extend, void* stream) {
    if (n % 2 != 0 || n < 2) return SHTC_EBOUND;
    if (extend != 0 && extend != 1) return SHTC_EBOUND;
    if (!aj) return SHTC_EBOUND;
    cudaStream_t st = (cudaStream_t)stream;
    k_dhaj<<<(n + extend + 127) / 128, 128, 0, st>>>(n, aj, extend);
    return map_cuda(cudaGetLastError());
}

extern "C" int shtc_plan_set_tuning(shtc_plan* P, int synth_T, int anal_T,
                                    int anal_W) {
    if (!P) return SHTC_EHANDLE;
    auto ok = [](int v) { return v == 0 || v == 1 || v == 2 || v == 4 || v == 8; };
    if (!ok(synth_T) || !ok(anal_T) || !ok(anal_W)) return SHTC_EBOUND;
    P->tune_synth_T = synth_T;
    P->tune_anal_T = anal_T;
    P->tune_anal_W = anal_W;
    return SHTC_OK;
}

extern "C" int shtc_plan_info(const shtc_plan* P, long long* info, int ninfo) {
    if (!P || !info) return SHTC_EHANDLE;
    long long v[16] = {P->kind, P->lmax, P->lc, P->norm, P->csphase, P->sampling,
                       P->extend, P->nlat, P->nlon, P->nlat_out, P->nlon_out,
                       P->npair, P->nlm, (long long)P->device_bytes,
                       P->fft.bluestein, P->fft.mode};
    for (int i = 0; i < ninfo && i < 16; ++i) info[i] = v[i];
    return SHTC_OK;
}
