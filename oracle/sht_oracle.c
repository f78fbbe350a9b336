/*
 * sht_oracle.c -- CPU restatement of the SHTOOLS real spherical-harmonic
 * transforms on Driscoll-Healy and Gauss-Legendre grids.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the parity oracle for the CUDA
 * engine in shtools_b200/.  Only tests/, the smoke check and the CPU
 * baseline leg of bench.py may load it; the product path never does.
 *
 * The arithmetic follows the reference Fortran statement by statement
 * (same recursion tables, same 1e-280 Holmes-Featherstone scaling points,
 * same per-latitude summation order, same north/south folding, same
 * equator and pole special cases, same final normalisation).  It is built
 * with -ffp-contract=off so that, like a default x86-64 gfortran build of
 * the reference, no multiply-add is fused.
 *
 *   recursion tables ........ src/MakeGridDH.f95:258-386
 *   MakeGridDH .............. src/MakeGridDH.f95:107-648
 *   SHExpandDH .............. src/SHExpandDH.f95:116-704
 *   MakeGridGLQ ............. src/MakeGridGLQ.f95:106-678 (on-the-fly branch)
 *   SHExpandGLQ ............. src/SHExpandGLQ.f95:98-691  (on-the-fly branch)
 *   PreGLQ .................. src/PreGLQ.f95:54-151
 *   DHaj .................... src/DHaj.f95:41-107
 *   complex transforms ...... src/MakeGridDHC.f95, SHExpandDHC.f95,
 *                             MakeGridGLQC.f95, SHExpandGLQC.f95
 *
 * FFTW (third-party, not vendored; environment.yml pins fftw>=3.3.8) is
 * replaced by the project-written FFT below: unnormalised DFTs with the
 * same sign conventions as fftw_plan_dft_r2c_1d / fftw_plan_dft_c2r_1d
 * (src/FFTW3.f95:212-271).  Lengths factor into radices 2,3,4,5,7 and
 * small odd primes; lengths with a prime factor above 61 use Bluestein's
 * chirp-z algorithm over a power-of-two convolution.
 *
 * Array layouts are the numpy C-order layouts of the Python API:
 *   cilm[k][l][m]  (2, cilm_dim, cilm_dim)
 *   grid[i][j]     (rows, cols), row-major
 *
 * Parity status: the reference binary cannot be built in this container
 * (no Fortran compiler, no FFTW).  The restatement is pinned against
 * independent known answers instead (scipy associated Legendre functions,
 * numpy FFTs, numpy Gauss-Legendre nodes, exact DH quadrature and
 * band-limited round trips): see tests/test_oracle.py.
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_OK 0
#define ORC_EDIM 1
#define ORC_EBOUND 2
#define ORC_EALLOC 3
#define ORC_ECONV 5

static const double SCALEF = 1.0e-280;

/* ------------------------------------------------------------------------ */
/*  FFT                                                                      */
/* ------------------------------------------------------------------------ */

typedef struct {
    int n;
    int nfac;
    int fac[40];
    double *wr, *wi;        /* exp(-2 pi i t / n), t = 0..n-1 */
    int bluestein;
    int nb;                 /* power-of-two convolution length */
    double *chr, *chi;      /* chirp exp(-i pi t^2 / n), t = 0..n-1 */
    double *kfr, *kfi;      /* FFT of the conjugate chirp kernel, length nb */
    struct orc_fft *sub;    /* power-of-two plan of length nb */
} orc_fft;

static int fft_factor(int n, int *fac) {
    int k = 0;
    while (n % 4 == 0) { fac[k++] = 4; n /= 4; }
    while (n % 2 == 0) { fac[k++] = 2; n /= 2; }
    for (int p = 3; p <= n; p += 2) {
        while (n % p == 0) {
            if (p > 61) return -1;
            fac[k++] = p;
            n /= p;
        }
    }
    return k;
}

static orc_fft *fft_plan(int n);
void orc_fft_exec(const orc_fft *p, double *re, double *im, int sign);

static void fft_roots(int n, double **wr, double **wi) {
    *wr = (double *)malloc(sizeof(double) * (size_t)n);
    *wi = (double *)malloc(sizeof(double) * (size_t)n);
    const double tp = 2.0 * acos(-1.0);
    for (int t = 0; t < n; ++t) {
        double a = tp * (double)t / (double)n;
        (*wr)[t] = cos(a);
        (*wi)[t] = -sin(a);
    }
}

static orc_fft *fft_plan(int n) {
    orc_fft *p = (orc_fft *)calloc(1, sizeof(orc_fft));
    p->n = n;
    fft_roots(n, &p->wr, &p->wi);
    p->nfac = fft_factor(n, p->fac);
    if (p->nfac < 0) {
        /* Bluestein: X_k = c_k * sum_j (x_j c_j) conj(c_{k-j}) */
        p->bluestein = 1;
        int nb = 1;
        while (nb < 2 * n - 1) nb <<= 1;
        p->nb = nb;
        p->chr = (double *)malloc(sizeof(double) * (size_t)n);
        p->chi = (double *)malloc(sizeof(double) * (size_t)n);
        const double pi = acos(-1.0);
        for (long long t = 0; t < n; ++t) {
            long long r = (t * t) % (2LL * n);
            double a = pi * (double)r / (double)n;
            p->chr[t] = cos(a);
            p->chi[t] = -sin(a);
        }
        p->sub = (struct orc_fft *)fft_plan(nb);
        p->kfr = (double *)calloc((size_t)nb, sizeof(double));
        p->kfi = (double *)calloc((size_t)nb, sizeof(double));
        p->kfr[0] = p->chr[0];
        p->kfi[0] = -p->chi[0];
        for (int t = 1; t < n; ++t) {
            p->kfr[t] = p->chr[t];
            p->kfi[t] = -p->chi[t];
            p->kfr[nb - t] = p->chr[t];
            p->kfi[nb - t] = -p->chi[t];
        }
        orc_fft_exec((orc_fft *)p->sub, p->kfr, p->kfi, -1);
    }
    return p;
}

static void fft_free(orc_fft *p) {
    if (!p) return;
    free(p->wr); free(p->wi);
    if (p->bluestein) {
        free(p->chr); free(p->chi); free(p->kfr); free(p->kfi);
        fft_free((orc_fft *)p->sub);
    }
    free(p);
}

/* One Stockham pass of radix r over n points; ns = size of the sub-DFTs
 * combined so far.  sign = -1 forward, +1 backward. */
static void fft_pass(const orc_fft *p, int r, int ns, const double *xr,
                     const double *xi, double *yr, double *yi, int sign) {
    const int n = p->n;
    const int nr = n / r;
    const int step = n / (ns * r);     /* twiddle index stride in the n-root table */
    const int rstep = n / r;           /* index stride of the r-th roots */
    double vr[64], vi[64], tr[64], ti[64];
    for (int j = 0; j < nr; ++j) {
        const int k = j % ns;
        for (int q = 0; q < r; ++q) {
            double ar = xr[j + q * nr], ai = xi[j + q * nr];
            if (k != 0 && q != 0) {
                int t = (int)(((long long)k * q * step) % n);
                double wr = p->wr[t], wi = sign < 0 ? p->wi[t] : -p->wi[t];
                double br = ar * wr - ai * wi;
                double bi = ar * wi + ai * wr;
                ar = br; ai = bi;
            }
            vr[q] = ar; vi[q] = ai;
        }
        if (r == 2) {
            tr[0] = vr[0] + vr[1]; ti[0] = vi[0] + vi[1];
            tr[1] = vr[0] - vr[1]; ti[1] = vi[0] - vi[1];
        } else if (r == 4) {
            double s0r = vr[0] + vr[2], s0i = vi[0] + vi[2];
            double d0r = vr[0] - vr[2], d0i = vi[0] - vi[2];
            double s1r = vr[1] + vr[3], s1i = vi[1] + vi[3];
            double d1r = vr[1] - vr[3], d1i = vi[1] - vi[3];
            /* multiply d1 by -i (forward) or +i (backward) */
            double er = sign < 0 ? d1i : -d1i;
            double ei = sign < 0 ? -d1r : d1r;
            tr[0] = s0r + s1r; ti[0] = s0i + s1i;
            tr[2] = s0r - s1r; ti[2] = s0i - s1i;
            tr[1] = d0r + er;  ti[1] = d0i + ei;
            tr[3] = d0r - er;  ti[3] = d0i - ei;
        } else {
            for (int s = 0; s < r; ++s) {
                double accr = 0.0, acci = 0.0;
                for (int q = 0; q < r; ++q) {
                    int t = (int)(((long long)s * q) % r) * rstep;
                    double wr = p->wr[t], wi = sign < 0 ? p->wi[t] : -p->wi[t];
                    accr += vr[q] * wr - vi[q] * wi;
                    acci += vr[q] * wi + vi[q] * wr;
                }
                tr[s] = accr; ti[s] = acci;
            }
        }
        const int d = (j / ns) * ns * r + k;
        for (int s = 0; s < r; ++s) {
            yr[d + s * ns] = tr[s];
            yi[d + s * ns] = ti[s];
        }
    }
}

/* In-place unnormalised complex DFT, sign -1: exp(-2 pi i jk/n). */
void orc_fft_exec(const orc_fft *p, double *re, double *im, int sign) {
    const int n = p->n;
    if (n == 1) return;
    if (p->bluestein) {
        const orc_fft *s = (const orc_fft *)p->sub;
        const int nb = p->nb;
        double *ar = (double *)calloc((size_t)nb, sizeof(double));
        double *ai = (double *)calloc((size_t)nb, sizeof(double));
        for (int t = 0; t < n; ++t) {
            double cr = p->chr[t], ci = sign < 0 ? p->chi[t] : -p->chi[t];
            ar[t] = re[t] * cr - im[t] * ci;
            ai[t] = re[t] * ci + im[t] * cr;
        }
        orc_fft_exec(s, ar, ai, -1);
        for (int t = 0; t < nb; ++t) {
            double kr = p->kfr[t], ki = p->kfi[t];
            if (sign > 0) {
                /* kernel of the conjugate chirp: FFT(conj(k))[t] = conj(FFT(k)[-t]) */
                int u = (nb - t) % nb;
                kr = p->kfr[u]; ki = -p->kfi[u];
            }
            double br = ar[t] * kr - ai[t] * ki;
            double bi = ar[t] * ki + ai[t] * kr;
            ar[t] = br; ai[t] = bi;
        }
        orc_fft_exec(s, ar, ai, +1);
        const double inv = 1.0 / (double)nb;
        for (int t = 0; t < n; ++t) {
            double cr = p->chr[t], ci = sign < 0 ? p->chi[t] : -p->chi[t];
            double xr = ar[t] * inv, xi = ai[t] * inv;
            re[t] = xr * cr - xi * ci;
            im[t] = xr * ci + xi * cr;
        }
        free(ar); free(ai);
        return;
    }
    double *br = (double *)malloc(sizeof(double) * (size_t)n);
    double *bi = (double *)malloc(sizeof(double) * (size_t)n);
    double *xr = re, *xi = im, *yr = br, *yi = bi;
    int ns = 1;
    for (int f = 0; f < p->nfac; ++f) {
        fft_pass(p, p->fac[f], ns, xr, xi, yr, yi, sign);
        ns *= p->fac[f];
        double *t;
        t = xr; xr = yr; yr = t;
        t = xi; xi = yi; yi = t;
    }
    if (xr != re) {
        memcpy(re, xr, sizeof(double) * (size_t)n);
        memcpy(im, xi, sizeof(double) * (size_t)n);
    }
    free(br); free(bi);
}

/* r2c as fftw_plan_dft_r2c_1d: out[k] = sum_j x_j exp(-2 pi i jk/n), k=0..n/2 */
static void fft_r2c(const orc_fft *p, const double *x, double *outr,
                    double *outi, double *wr, double *wi) {
    const int n = p->n;
    for (int j = 0; j < n; ++j) { wr[j] = x[j]; wi[j] = 0.0; }
    orc_fft_exec(p, wr, wi, -1);
    for (int k = 0; k <= n / 2; ++k) { outr[k] = wr[k]; outi[k] = wi[k]; }
}

/* c2r as fftw_plan_dft_c2r_1d: x_j = sum over the Hermitian extension of
 * in[0..n/2] of in_k exp(+2 pi i jk/n).  As in FFTW, the imaginary parts of
 * the DC term and (n even) of the Nyquist term do not contribute. */
static void fft_c2r(const orc_fft *p, const double *inr, const double *ini,
                    double *x, double *wr, double *wi) {
    const int n = p->n;
    wr[0] = inr[0]; wi[0] = 0.0;
    for (int k = 1; k < (n + 1) / 2; ++k) {
        wr[k] = inr[k]; wi[k] = ini[k];
        wr[n - k] = inr[k]; wi[n - k] = -ini[k];
    }
    if (n % 2 == 0) { wr[n / 2] = inr[n / 2]; wi[n / 2] = 0.0; }
    orc_fft_exec(p, wr, wi, +1);
    for (int j = 0; j < n; ++j) x[j] = wr[j];
}

/* exported for the FFT unit tests: forward (sign=-1) or backward complex DFT */
int orc_fft_c2c(int n, double *re, double *im, int sign) {
    if (n < 1) return ORC_EBOUND;
    orc_fft *p = fft_plan(n);
    orc_fft_exec(p, re, im, sign < 0 ? -1 : 1);
    fft_free(p);
    return ORC_OK;
}

int orc_fft_r2c(int n, const double *x, double *outr, double *outi) {
    if (n < 1) return ORC_EBOUND;
    orc_fft *p = fft_plan(n);
    double *wr = (double *)malloc(sizeof(double) * (size_t)n);
    double *wi = (double *)malloc(sizeof(double) * (size_t)n);
    fft_r2c(p, x, outr, outi, wr, wi);
    free(wr); free(wi);
    fft_free(p);
    return ORC_OK;
}

int orc_fft_c2r(int n, const double *inr, const double *ini, double *x) {
    if (n < 1) return ORC_EBOUND;
    orc_fft *p = fft_plan(n);
    double *wr = (double *)malloc(sizeof(double) * (size_t)n);
    double *wi = (double *)malloc(sizeof(double) * (size_t)n);
    fft_c2r(p, inr, ini, x, wr, wi);
    free(wr); free(wi);
    fft_free(p);
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/*  Recursion tables  (MakeGridDH.f95:258-386; identical in the other three) */
/* ------------------------------------------------------------------------ */

typedef struct {
    int lc;          /* lmax_comp */
    int norm;
    double *sqr;     /* sqr[k] = sqrt(k), k = 0..2lc+1  (Fortran sqr(k)) */
    double *ff1;     /* ff1[l*(lc+1)+m]  (Fortran ff1(l+1,m+1)) */
    double *ff2;
} rec_tab;

static int rec_build(rec_tab *t, int lc, int norm) {
    const int d = lc + 1;
    t->lc = lc; t->norm = norm;
    t->sqr = (double *)calloc((size_t)(2 * lc + 2), sizeof(double));
    t->ff1 = (double *)calloc((size_t)d * d, sizeof(double));
    t->ff2 = (double *)calloc((size_t)d * d, sizeof(double));
    if (!t->sqr || !t->ff1 || !t->ff2) return ORC_EALLOC;
    double *sqr = t->sqr, *ff1 = t->ff1, *ff2 = t->ff2;
#define F1(l, m) ff1[(size_t)(l) * d + (m)]
#define F2(l, m) ff2[(size_t)(l) * d + (m)]
    for (int k = 1; k <= 2 * lc + 1; ++k) sqr[k] = sqrt((double)k);
    if (norm == 1 || norm == 4) {
        if (lc != 0) { F1(1, 0) = sqr[3]; F2(1, 0) = 0.0; }
        for (int l = 2; l <= lc; ++l) {
            F1(l, 0) = sqr[2 * l - 1] * sqr[2 * l + 1] / (double)l;
            F2(l, 0) = (double)(l - 1) * sqr[2 * l + 1] / sqr[2 * l - 3] / (double)l;
            int m;
            for (m = 1; m <= l - 2; ++m) {
                F1(l, m) = sqr[2 * l + 1] * sqr[2 * l - 1] / sqr[l + m] / sqr[l - m];
                F2(l, m) = sqr[2 * l + 1] * sqr[l - m - 1] * sqr[l + m - 1]
                           / sqr[2 * l - 3] / sqr[l + m] / sqr[l - m];
            }
            /* Fortran leaves the DO variable at l-1 here (MakeGridDH.f95:341) */
            m = l - 1;
            F1(l, l - 1) = sqr[2 * l + 1] * sqr[2 * l - 1] / sqr[l + m] / sqr[l - m];
            F2(l, l - 1) = 0.0;
        }
    } else if (norm == 2) {
        if (lc != 0) { F1(1, 0) = 1.0; F2(1, 0) = 0.0; }
        for (int l = 2; l <= lc; ++l) {
            F1(l, 0) = (double)(2 * l - 1) / (double)l;
            F2(l, 0) = (double)(l - 1) / (double)l;
            int m;
            for (m = 1; m <= l - 2; ++m) {
                F1(l, m) = (double)(2 * l - 1) / sqr[l + m] / sqr[l - m];
                F2(l, m) = sqr[l - m - 1] * sqr[l + m - 1] / sqr[l + m] / sqr[l - m];
            }
            m = l - 1;
            F1(l, l - 1) = (double)(2 * l - 1) / sqr[l + m] / sqr[l - m];
            F2(l, l - 1) = 0.0;
        }
    } else {
        for (int l = 1; l <= lc; ++l) {
            F1(l, 0) = (double)(2 * l - 1) / (double)l;
            F2(l, 0) = (double)(l - 1) / (double)l;
            for (int m = 1; m <= l - 1; ++m) {
                F1(l, m) = (double)(2 * l - 1) / (double)(l - m);
                F2(l, m) = (double)(l + m - 1) / (double)(l - m);
            }
        }
    }
#undef F1
#undef F2
    return ORC_OK;
}

static void rec_free(rec_tab *t) {
    free(t->sqr); free(t->ff1); free(t->ff2);
}

/* exported so tests can inspect the tables (ff1/ff2 laid out [l][m]) */
int orc_rec_tables(int lc, int norm, double *ff1, double *ff2) {
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    memcpy(ff1, t.ff1, sizeof(double) * (size_t)(lc + 1) * (lc + 1));
    memcpy(ff2, t.ff2, sizeof(double) * (size_t)(lc + 1) * (lc + 1));
    rec_free(&t);
    return ORC_OK;
}

/* start value P00 for the given normalisation */
static double p00(int norm) {
    const double pi = acos(-1.0);
    return norm == 4 ? 1.0 / sqrt(4.0 * pi) : 1.0;
}

static double pmm_start(int norm) {
    const double pi = acos(-1.0);
    switch (norm) {
        case 1: case 2: return sqrt(2.0) * SCALEF;     /* sqr(2) * scalef */
        case 3: return SCALEF;
        default: return sqrt(2.0) * SCALEF / sqrt(4.0 * pi);
    }
}

/* ------------------------------------------------------------------------ */
/*  Synthesis kernel for one latitude ring pair                             */
/*  (MakeGridDH.f95:504-621, MakeGridGLQ.f95:547-663)                       */
/*  Writes coef (north) and coefs (south) for m = 0..lc; the caller halves   */
/*  and zero-pads them.                                                      */
/* ------------------------------------------------------------------------ */

#define CIL(k, l, m) cilm[((size_t)(k) * cdim + (size_t)(l)) * cdim + (size_t)(m)]

static void synth_ring(const rec_tab *t, const double *cilm, int cdim, int phase,
                       double z, double u, double *cr, double *ci, double *csr,
                       double *csi) {
    const int lc = t->lc, d = lc + 1, norm = t->norm;
    const double *sqr = t->sqr, *ff1 = t->ff1, *ff2 = t->ff2;
    double pm2, pm1, p, pmm, rescalem, tempr;
    double coef0 = 0.0, coef0s = 0.0;

    pm2 = p00(norm);
    tempr = CIL(0, 0, 0) * pm2;
    coef0 = coef0 + tempr;
    coef0s = coef0s + tempr;

    pm1 = ff1[(size_t)1 * d + 0] * z * pm2;
    tempr = CIL(0, 1, 0) * pm1;
    coef0 = coef0 + tempr;
    coef0s = coef0s - tempr;

    for (int l = 2; l <= lc; ++l) {
        p = ff1[(size_t)l * d + 0] * z * pm1 - ff2[(size_t)l * d + 0] * pm2;
        tempr = CIL(0, l, 0) * p;
        coef0 = coef0 + tempr;
        coef0s = coef0s + tempr * (double)(((l) % 2 == 0) ? 1 : -1);
        pm2 = pm1;
        pm1 = p;
    }
    cr[0] = coef0; ci[0] = 0.0;
    csr[0] = coef0s; csi[0] = 0.0;

    pmm = pmm_start(norm);
    rescalem = 1.0 / SCALEF;

    for (int m = 1; m <= lc - 1; ++m) {
        rescalem = rescalem * u;
        switch (norm) {
            case 1: case 4:
                pmm = phase * pmm * sqr[2 * m + 1] / sqr[2 * m];
                pm2 = pmm;
                break;
            case 2:
                pmm = phase * pmm * sqr[2 * m + 1] / sqr[2 * m];
                pm2 = pmm / sqr[2 * m + 1];
                break;
            default:
                pmm = phase * pmm * (double)(2 * m - 1);
                pm2 = pmm;
                break;
        }
        /* tempc = cmplx(C, -S) * pm2 */
        double tr_ = CIL(0, m, m) * pm2, ti_ = -CIL(1, m, m) * pm2;
        double ar = tr_, ai = ti_, sr = tr_, si = ti_;

        pm1 = z * ff1[(size_t)(m + 1) * d + m] * pm2;
        tr_ = CIL(0, m + 1, m) * pm1; ti_ = -CIL(1, m + 1, m) * pm1;
        ar = ar + tr_; ai = ai + ti_;
        sr = sr - tr_; si = si - ti_;

        for (int l = m + 2; l <= lc; ++l) {
            p = z * ff1[(size_t)l * d + m] * pm1 - ff2[(size_t)l * d + m] * pm2;
            pm2 = pm1;
            pm1 = p;
            tr_ = CIL(0, l, m) * p; ti_ = -CIL(1, l, m) * p;
            ar = ar + tr_; ai = ai + ti_;
            if ((l - m) % 2 == 0) { sr = sr + tr_; si = si + ti_; }
            else { sr = sr + tr_ * -1.0; si = si + ti_ * -1.0; }
        }
        cr[m] = ar * rescalem; ci[m] = ai * rescalem;
        csr[m] = sr * rescalem; csi[m] = si * rescalem;
    }

    rescalem = rescalem * u;
    switch (norm) {
        case 1: case 4:
            pmm = phase * pmm * sqr[2 * lc + 1] / sqr[2 * lc] * rescalem; break;
        case 2:
            pmm = phase * pmm / sqr[2 * lc] * rescalem; break;
        default:
            pmm = phase * pmm * (double)(2 * lc - 1) * rescalem; break;
    }
    {
        double tr_ = CIL(0, lc, lc) * pmm, ti_ = -CIL(1, lc, lc) * pmm;
        cr[lc] = tr_; ci[lc] = ti_;
        csr[lc] = tr_; csi[lc] = ti_;
    }
}

/* Equator ring: z = 0, u = 1, even l-m only
 * (MakeGridDH.f95:424-502, MakeGridGLQ.f95:472-545).  Returns coef already
 * multiplied by rescalem; the caller halves m >= 1. */
static void synth_equator(const rec_tab *t, const double *cilm, int cdim,
                          int phase, double *cr, double *ci) {
    const int lc = t->lc, d = lc + 1, norm = t->norm;
    const double *sqr = t->sqr, *ff2 = t->ff2;
    double pm2, p, pmm, rescalem;
    double coef0 = 0.0;

    pm2 = p00(norm);
    coef0 = coef0 + CIL(0, 0, 0) * pm2;
    for (int l = 2; l <= lc; l += 2) {
        p = -ff2[(size_t)l * d + 0] * pm2;
        pm2 = p;
        coef0 = coef0 + CIL(0, l, 0) * p;
    }
    pmm = pmm_start(norm);
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        switch (norm) {
            case 1: case 4:
                pmm = phase * pmm * sqr[2 * m + 1] / sqr[2 * m];
                pm2 = pmm; break;
            case 2:
                pmm = phase * pmm * sqr[2 * m + 1] / sqr[2 * m];
                pm2 = pmm / sqr[2 * m + 1]; break;
            default:
                pmm = phase * pmm * (double)(2 * m - 1);
                pm2 = pmm; break;
        }
        double ar = CIL(0, m, m) * pm2, ai = -CIL(1, m, m) * pm2;
        for (int l = m + 2; l <= lc; l += 2) {
            p = -ff2[(size_t)l * d + m] * pm2;
            ar = ar + CIL(0, l, m) * p;
            ai = ai + -CIL(1, l, m) * p;
            pm2 = p;
        }
        cr[m] = ar * rescalem; ci[m] = ai * rescalem;
    }
    switch (norm) {
        case 1: case 4:
            pmm = phase * pmm * sqr[2 * lc + 1] / sqr[2 * lc]; break;
        case 2:
            pmm = phase * pmm / sqr[2 * lc]; break;
        default:
            pmm = phase * pmm * (double)(2 * lc - 1); break;
    }
    cr[lc] = CIL(0, lc, lc) * pmm * rescalem;
    ci[lc] = -CIL(1, lc, lc) * pmm * rescalem;
    cr[0] = coef0; ci[0] = 0.0;
}

/* ------------------------------------------------------------------------ */
/*  Analysis kernel for one latitude ring pair                              */
/*  (SHExpandDH.f95:481-580, SHExpandGLQ.f95:549-643)                        */
/*  f1/f2: weighted Fourier coefficients (re, -im) of the north / south      */
/*  rings for m = 0..lc, modified in place by the rescaling as in Fortran.   */
/* ------------------------------------------------------------------------ */

static void anal_ring(const rec_tab *t, double *cilm, int cdim, int phase,
                      double z, double u, double *f1r, double *f1i,
                      double *f2r, double *f2i) {
    const int lc = t->lc, d = lc + 1, norm = t->norm;
    const double *sqr = t->sqr, *ff1 = t->ff1, *ff2 = t->ff2;
    double pm2, pm1, p, pmm, rescalem;
    double ffcr[2], ffci[2];   /* [0]: fsymsign -1, [1]: fsymsign +1 */

    pm2 = p00(norm);
    CIL(0, 0, 0) = CIL(0, 0, 0) + pm2 * (f1r[0] + f2r[0]);
    if (lc == 0) return;
    pm1 = ff1[(size_t)1 * d + 0] * z * pm2;
    CIL(0, 1, 0) = CIL(0, 1, 0) + pm1 * (f1r[0] - f2r[0]);
    ffcr[0] = f1r[0] - f2r[0];
    ffcr[1] = f1r[0] + f2r[0];
    for (int l = 2; l <= lc; ++l) {
        p = ff1[(size_t)l * d + 0] * z * pm1 - ff2[(size_t)l * d + 0] * pm2;
        pm2 = pm1;
        pm1 = p;
        CIL(0, l, 0) = CIL(0, l, 0) + p * ffcr[(l % 2 == 0) ? 1 : 0];
    }
    pmm = pmm_start(norm);
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        rescalem = rescalem * u;
        switch (norm) {
            case 1: case 4:
                pmm = phase * pmm * sqr[2 * m + 1] / sqr[2 * m];
                pm2 = pmm; break;
            case 2:
                pmm = phase * pmm * sqr[2 * m + 1] / sqr[2 * m];
                pm2 = pmm / sqr[2 * m + 1]; break;
            default:
                pmm = phase * pmm * (double)(2 * m - 1);
                pm2 = pmm; break;
        }
        f1r[m] = f1r[m] * rescalem; f1i[m] = f1i[m] * rescalem;
        f2r[m] = f2r[m] * rescalem; f2i[m] = f2i[m] * rescalem;
        CIL(0, m, m) = CIL(0, m, m) + pm2 * (f1r[m] + f2r[m]);
        CIL(1, m, m) = CIL(1, m, m) + pm2 * (f1i[m] + f2i[m]);
        pm1 = z * ff1[(size_t)(m + 1) * d + m] * pm2;
        CIL(0, m + 1, m) = CIL(0, m + 1, m) + pm1 * (f1r[m] - f2r[m]);
        CIL(1, m + 1, m) = CIL(1, m + 1, m) + pm1 * (f1i[m] - f2i[m]);
        ffcr[0] = f1r[m] - f2r[m]; ffci[0] = f1i[m] - f2i[m];
        ffcr[1] = f1r[m] + f2r[m]; ffci[1] = f1i[m] + f2i[m];
        for (int l = m + 2; l <= lc; ++l) {
            p = z * ff1[(size_t)l * d + m] * pm1 - ff2[(size_t)l * d + m] * pm2;
            pm2 = pm1;
            pm1 = p;
            const int s = ((l - m) % 2 == 0) ? 1 : 0;
            CIL(0, l, m) = CIL(0, l, m) + p * ffcr[s];
            CIL(1, l, m) = CIL(1, l, m) + p * ffci[s];
        }
    }
    rescalem = rescalem * u;
    switch (norm) {
        case 1: case 4:
            pmm = phase * pmm * sqr[2 * lc + 1] / sqr[2 * lc] * rescalem; break;
        case 2:
            pmm = phase * pmm / sqr[2 * lc] * rescalem; break;
        default:
            pmm = phase * pmm * (double)(2 * lc - 1) * rescalem; break;
    }
    CIL(0, lc, lc) = CIL(0, lc, lc) + pmm * (f1r[lc] + f2r[lc]);
    CIL(1, lc, lc) = CIL(1, lc, lc) + pmm * (f1i[lc] + f2i[lc]);
}

/* Equator ring of the analysis (SHExpandDH.f95:583-664, SHExpandGLQ.f95:447-528) */
static void anal_equator(const rec_tab *t, double *cilm, int cdim, int phase,
                         double *f1r, double *f1i) {
    const int lc = t->lc, d = lc + 1, norm = t->norm;
    const double *sqr = t->sqr, *ff2 = t->ff2;
    double pm2, p, pmm, rescalem;
    pm2 = p00(norm);
    CIL(0, 0, 0) = CIL(0, 0, 0) + pm2 * f1r[0];
    if (lc == 0) return;
    for (int l = 2; l <= lc; l += 2) {
        p = -ff2[(size_t)l * d + 0] * pm2;
        pm2 = p;
        CIL(0, l, 0) = CIL(0, l, 0) + p * f1r[0];
    }
    pmm = pmm_start(norm);
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        switch (norm) {
            case 1: case 4:
                pmm = phase * pmm * sqr[2 * m + 1] / sqr[2 * m];
                pm2 = pmm; break;
            case 2:
                pmm = phase * pmm * sqr[2 * m + 1] / sqr[2 * m];
                pm2 = pmm / sqr[2 * m + 1]; break;
            default:
                pmm = phase * pmm * (double)(2 * m - 1);
                pm2 = pmm; break;
        }
        f1r[m] = f1r[m] * rescalem; f1i[m] = f1i[m] * rescalem;
        CIL(0, m, m) = CIL(0, m, m) + pm2 * f1r[m];
        CIL(1, m, m) = CIL(1, m, m) + pm2 * f1i[m];
        for (int l = m + 2; l <= lc; l += 2) {
            p = -ff2[(size_t)l * d + m] * pm2;
            pm2 = p;
            CIL(0, l, m) = CIL(0, l, m) + p * f1r[m];
            CIL(1, l, m) = CIL(1, l, m) + p * f1i[m];
        }
    }
    switch (norm) {
        case 1: case 4:
            pmm = phase * pmm * sqr[2 * lc + 1] / sqr[2 * lc] * rescalem; break;
        case 2:
            pmm = phase * pmm / sqr[2 * lc] * rescalem; break;
        default:
            pmm = phase * pmm * (double)(2 * lc - 1) * rescalem; break;
    }
    CIL(0, lc, lc) = CIL(0, lc, lc) + pmm * f1r[lc];
    CIL(1, lc, lc) = CIL(1, lc, lc) + pmm * f1i[lc];
}

/* Divide by the integral of Ylm^2 (SHExpandDH.f95:674-702, SHExpandGLQ.f95:659-689) */
static void anal_normalise(double *cilm, int cdim, int lc, int norm) {
    const double pi = acos(-1.0);
    if (norm == 1) {
        for (int l = 0; l <= lc; ++l)
            for (int m = 0; m <= l; ++m) {
                CIL(0, l, m) = CIL(0, l, m) / (4 * pi);
                CIL(1, l, m) = CIL(1, l, m) / (4 * pi);
            }
    } else if (norm == 2) {
        for (int l = 0; l <= lc; ++l)
            for (int m = 0; m <= l; ++m) {
                CIL(0, l, m) = CIL(0, l, m) * (2 * l + 1) / (4 * pi);
                CIL(1, l, m) = CIL(1, l, m) * (2 * l + 1) / (4 * pi);
            }
    } else if (norm == 3) {
        for (int l = 0; l <= lc; ++l) {
            double prod = 4 * pi / (double)(2 * l + 1);
            CIL(0, l, 0) = CIL(0, l, 0) / prod;
            prod = prod / 2.0;
            for (int m = 1; m <= l - 1; ++m) {
                prod = prod * (l + m) * (l - m + 1);
                CIL(0, l, m) = CIL(0, l, m) / prod;
                CIL(1, l, m) = CIL(1, l, m) / prod;
            }
            if (l != 0) {
                CIL(0, l, l) = CIL(0, l, l) / (prod * 2 * l);
                CIL(1, l, l) = CIL(1, l, l) / (prod * 2 * l);
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/*  DHaj  (DHaj.f95:41-107)                                                  */
/* ------------------------------------------------------------------------ */

int orc_dhaj(int n, double *aj, int extend) {
    const double pi = acos(-1.0);
    if (n % 2 != 0) return ORC_EBOUND;
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    for (int j = 0; j <= n - 1; ++j) {
        double sum1 = 0.0;
        for (int l = 0; l <= n / 2 - 1; ++l)
            sum1 = sum1 + sin((double)(2 * l + 1) * pi * (double)j / (double)n)
                              / (double)(2 * l + 1);
        aj[j] = sum1 * sin(pi * (double)j / (double)n) * sqrt(8.0) / (double)n;
    }
    if (extend == 1) aj[n] = 0.0;
    return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/*  PreGLQ  (PreGLQ.f95:54-151)                                              */
/* ------------------------------------------------------------------------ */

int orc_preglq_iter(double x1, double x2, int n, double *zero, double *w,
                    int itermax) {
    const double eps = 1.0e-15;
    const double pi = acos(-1.0);
    for (int i = 0; i < n; ++i) { zero[i] = 0.0; w[i] = 0.0; }
    const int m = (n + 1) / 2;
    const double xm = (x2 + x1) / 2.0;
    const double xu = (x2 - x1) / 2.0;
    for (int i = 1; i <= m; ++i) {
        int iter = 0;
        double z = cos(pi * (i - 0.25) / (n + 0.5));
        double p1, p2, p3, pp, z1;
        for (;;) {
            iter = iter + 1;
            p1 = 1.0;
            p2 = 0.0;
            for (int j = 1; j <= n; ++j) {
                p3 = p2;
                p2 = p1;
                p1 = ((double)(2 * j - 1) * z * p2 - (double)(j - 1) * p3) / (double)j;
            }
            pp = (double)n * (z * p1 - p2) / (z * z - 1.0);
            z1 = z;
            z = z1 - p1 / pp;
            if (fabs(z - z1) <= eps) break;
            if (iter > itermax) return ORC_ECONV;
        }
        zero[i - 1] = xm + xu * z;
        zero[n - i] = xm - xu * z;
        w[i - 1] = 2.0 * xu / ((1.0 - z * z) * pp * pp);
        w[n - i] = w[i - 1];
    }
    return ORC_OK;
}

int orc_preglq(double x1, double x2, int n, double *zero, double *w) {
    return orc_preglq_iter(x1, x2, n, zero, w, 1000);
}

/* ------------------------------------------------------------------------ */
/*  MakeGridDH  (MakeGridDH.f95:107-648)                                     */
/*  grid: (n+extend) x (nlong+extend) row-major.  Rows of ring pairs with   */
/*  index i in [pair_lo, pair_hi) are computed (1-based Fortran i-1); the   */
/*  public entry point computes them all, the windowed one exists for the   */
/*  bounded CPU-baseline sample.                                            */
/* ------------------------------------------------------------------------ */

static int makegrid_dh_impl(double *grid, const double *cilm, int cdim, int lmax,
                            int norm, int sampling, int csphase, int lmax_calc,
                            int extend, int pair_lo, int pair_hi) {
    if (sampling != 1 && sampling != 2) return ORC_EBOUND;
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    if (lmax_calc > lmax) return ORC_EBOUND;
    const int n = 2 * lmax + 2;
    const int nlong = sampling == 1 ? n : 2 * n;
    const int nlat_out = n + extend, nlong_out = nlong + extend;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax) lc = lmax;
    if (lc > cdim - 1) lc = cdim - 1;
    const double pi = acos(-1.0);

    if (lc == 0) {
        const double pm2 = p00(norm);
        for (int i = 0; i < nlat_out; ++i)
            for (int j = 0; j < nlong_out; ++j)
                grid[(size_t)i * nlong_out + j] = CIL(0, 0, 0) * pm2;
        return ORC_OK;
    }
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    const int nh = nlong / 2 + 1;
    double *cr = calloc((size_t)nh + lmax + 2, sizeof(double));
    double *ci = calloc((size_t)nh + lmax + 2, sizeof(double));
    double *csr = calloc((size_t)nh + lmax + 2, sizeof(double));
    double *csi = calloc((size_t)nh + lmax + 2, sizeof(double));
    double *wr = malloc(sizeof(double) * (size_t)nlong);
    double *wi = malloc(sizeof(double) * (size_t)nlong);
    double *row = malloc(sizeof(double) * (size_t)nlong);
    const int i_eq = n / 2 + 1;  /* 1-based */
    if (pair_lo < 0) pair_lo = 0;
    if (pair_hi > i_eq) pair_hi = i_eq;

    /* equator (pair index i_eq-1) */
    if (pair_lo <= i_eq - 1 && i_eq - 1 < pair_hi) {
        for (int k = 0; k < nh; ++k) { cr[k] = 0.0; ci[k] = 0.0; }
        synth_equator(&t, cilm, cdim, csphase, cr, ci);
        for (int m = 1; m <= lmax; ++m) { cr[m] = cr[m] / 2.0; ci[m] = ci[m] / 2.0; }
        fft_c2r(plan, cr, ci, row, wr, wi);
        memcpy(&grid[(size_t)(i_eq - 1) * nlong_out], row, sizeof(double) * (size_t)nlong);
    }
    for (int i = 1; i <= i_eq - 1; ++i) {
        if (i - 1 < pair_lo || i - 1 >= pair_hi) continue;
        const int i_s = 2 * i_eq - i;
        const double theta = pi * (double)(i - 1) / (double)n;
        const double z = cos(theta);
        const double u = sqrt((1.0 - z) * (1.0 + z));
        for (int k = 0; k < nh; ++k) { cr[k] = ci[k] = csr[k] = csi[k] = 0.0; }
        synth_ring(&t, cilm, cdim, csphase, z, u, cr, ci, csr, csi);
        for (int m = 1; m <= lmax; ++m) { cr[m] = cr[m] / 2.0; ci[m] = ci[m] / 2.0; }
        fft_c2r(plan, cr, ci, row, wr, wi);
        memcpy(&grid[(size_t)(i - 1) * nlong_out], row, sizeof(double) * (size_t)nlong);
        if (!(i == 1 && extend == 0)) {
            for (int m = 1; m <= lmax; ++m) { csr[m] = csr[m] / 2.0; csi[m] = csi[m] / 2.0; }
            fft_c2r(plan, csr, csi, row, wr, wi);
            memcpy(&grid[(size_t)(i_s - 1) * nlong_out], row, sizeof(double) * (size_t)nlong);
        }
    }
    if (extend == 1)
        for (int i = 0; i < nlat_out; ++i)
            grid[(size_t)i * nlong_out + nlong] = grid[(size_t)i * nlong_out];
    free(cr); free(ci); free(csr); free(csi); free(wr); free(wi); free(row);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

int orc_makegrid_dh(double *grid, const double *cilm, int cdim, int lmax,
                    int norm, int sampling, int csphase, int lmax_calc,
                    int extend) {
    return makegrid_dh_impl(grid, cilm, cdim, lmax, norm, sampling, csphase,
                            lmax_calc, extend, 0, 1 << 30);
}

int orc_makegrid_dh_window(double *grid, const double *cilm, int cdim, int lmax,
                           int norm, int sampling, int csphase, int lmax_calc,
                           int extend, int pair_lo, int pair_hi) {
    return makegrid_dh_impl(grid, cilm, cdim, lmax, norm, sampling, csphase,
                            lmax_calc, extend, pair_lo, pair_hi);
}

/* ------------------------------------------------------------------------ */
/*  SHExpandDH  (SHExpandDH.f95:116-704)                                     */
/*  grid: n x ncols row-major (ncols >= nlong; extra columns ignored).       */
/*  cilm: (2, cdim, cdim) zeroed and filled for l,m <= lmax_comp.           */
/* ------------------------------------------------------------------------ */

static int shexpand_dh_impl(double *cilm, int cdim, const double *grid, int n,
                            int ncols, int norm, int sampling, int csphase,
                            int lmax_calc, int pair_lo, int pair_hi) {
    const int lmax = n / 2 - 1;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax) return ORC_EBOUND;
    if (sampling != 1 && sampling != 2) return ORC_EBOUND;
    if (n % 2 != 0) return ORC_EBOUND;
    if (cdim < lc + 1) return ORC_EDIM;
    const int nlong = sampling == 1 ? n : 2 * n;
    if (ncols < nlong) return ORC_EDIM;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    const double pi = acos(-1.0);
    memset(cilm, 0, sizeof(double) * 2 * (size_t)cdim * cdim);
    double *aj = malloc(sizeof(double) * (size_t)n);
    orc_dhaj(n, aj, 0);
    for (int i = 0; i < n; ++i) aj[i] = aj[i] * sqrt(4.0 * pi);
    rec_tab t;
    if (rec_build(&t, lc, norm)) { free(aj); return ORC_EALLOC; }
    orc_fft *plan = fft_plan(nlong);
    const int nh = nlong / 2 + 1;
    double *ccr = malloc(sizeof(double) * (size_t)nh), *cci = malloc(sizeof(double) * (size_t)nh);
    double *f1r = malloc(sizeof(double) * (size_t)(n / 2 + 1)), *f1i = malloc(sizeof(double) * (size_t)(n / 2 + 1));
    double *f2r = malloc(sizeof(double) * (size_t)(n / 2 + 1)), *f2i = malloc(sizeof(double) * (size_t)(n / 2 + 1));
    double *wr = malloc(sizeof(double) * (size_t)nlong), *wi = malloc(sizeof(double) * (size_t)nlong);
    const int i_eq = n / 2 + 1;
    if (pair_lo < 0) pair_lo = 0;
    if (pair_hi > i_eq) pair_hi = i_eq;
    const double s2p = sqrt(2 * pi);
    for (int i = 2; i <= i_eq - 1; ++i) {
        if (i - 1 < pair_lo || i - 1 >= pair_hi) continue;
        const double theta = (i - 1) * pi / (double)n;
        const double z = cos(theta);
        const double u = sqrt((1.0 - z) * (1.0 + z));
        fft_r2c(plan, &grid[(size_t)(i - 1) * ncols], ccr, cci, wr, wi);
        for (int k = 0; k < n / 2; ++k) {
            f1r[k] = s2p * aj[i - 1] * ccr[k] / (double)nlong;
            f1i[k] = -s2p * aj[i - 1] * cci[k] / (double)nlong;
        }
        const int i_s = 2 * i_eq - i;
        fft_r2c(plan, &grid[(size_t)(i_s - 1) * ncols], ccr, cci, wr, wi);
        for (int k = 0; k < n / 2; ++k) {
            f2r[k] = s2p * aj[i_s - 1] * ccr[k] / (double)nlong;
            f2i[k] = -s2p * aj[i_s - 1] * cci[k] / (double)nlong;
        }
        anal_ring(&t, cilm, cdim, csphase, z, u, f1r, f1i, f2r, f2i);
    }
    if (pair_lo <= i_eq - 1 && i_eq - 1 < pair_hi) {
        const int i = i_eq;
        fft_r2c(plan, &grid[(size_t)(i - 1) * ncols], ccr, cci, wr, wi);
        for (int k = 0; k < n / 2; ++k) {
            f1r[k] = s2p * aj[i - 1] * ccr[k] / (double)nlong;
            f1i[k] = -s2p * aj[i - 1] * cci[k] / (double)nlong;
        }
        anal_equator(&t, cilm, cdim, csphase, f1r, f1i);
    }
    anal_normalise(cilm, cdim, lc, norm);
    free(aj); free(ccr); free(cci); free(f1r); free(f1i); free(f2r); free(f2i);
    free(wr); free(wi);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

int orc_shexpand_dh(double *cilm, int cdim, const double *grid, int n, int ncols,
                    int norm, int sampling, int csphase, int lmax_calc) {
    return shexpand_dh_impl(cilm, cdim, grid, n, ncols, norm, sampling, csphase,
                            lmax_calc, 0, 1 << 30);
}

int orc_shexpand_dh_window(double *cilm, int cdim, const double *grid, int n,
                           int ncols, int norm, int sampling, int csphase,
                           int lmax_calc, int pair_lo, int pair_hi) {
    return shexpand_dh_impl(cilm, cdim, grid, n, ncols, norm, sampling, csphase,
                            lmax_calc, pair_lo, pair_hi);
}

/* ------------------------------------------------------------------------ */
/*  MakeGridGLQ  (MakeGridGLQ.f95:106-678, on-the-fly branch :467-669)        */
/*  grid: (lmax+1) x (2lmax+1+extend) row-major.                             */
/* ------------------------------------------------------------------------ */

static int makegrid_glq_impl(double *grid, const double *cilm, int cdim,
                             int lmax, const double *zero, int norm,
                             int csphase, int lmax_calc, int extend,
                             int pair_lo, int pair_hi) {
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    if (!zero) return ORC_ECONV;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    if (lmax_calc > lmax) return ORC_EBOUND;
    const int nlong = 2 * lmax + 1, nlat = lmax + 1;
    const int nlong_out = nlong + extend;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > cdim - 1) lc = cdim - 1;
    if (lc == 0) {
        const double pm2 = p00(norm);
        for (int i = 0; i < nlat; ++i)
            for (int j = 0; j < nlong_out; ++j)
                grid[(size_t)i * nlong_out + j] = CIL(0, 0, 0) * pm2;
        return ORC_OK;
    }
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    const int nh = lmax + 1;
    double *cr = calloc((size_t)nh, sizeof(double)), *ci = calloc((size_t)nh, sizeof(double));
    double *csr = calloc((size_t)nh, sizeof(double)), *csi = calloc((size_t)nh, sizeof(double));
    double *wr = malloc(sizeof(double) * (size_t)nlong), *wi = malloc(sizeof(double) * (size_t)nlong);
    double *row = malloc(sizeof(double) * (size_t)nlong);
    if (pair_lo < 0) pair_lo = 0;
    for (int i = 1; i <= (nlat + 1) / 2; ++i) {
        if (i - 1 < pair_lo || i - 1 >= pair_hi) continue;
        for (int k = 0; k < nh; ++k) { cr[k] = ci[k] = csr[k] = csi[k] = 0.0; }
        if (i == (nlat + 1) / 2 && nlat % 2 != 0) {
            synth_equator(&t, cilm, cdim, csphase, cr, ci);
            for (int m = 1; m <= lc; ++m) { cr[m] = cr[m] / 2.0; ci[m] = ci[m] / 2.0; }
            fft_c2r(plan, cr, ci, row, wr, wi);
            memcpy(&grid[(size_t)(i - 1) * nlong_out], row, sizeof(double) * (size_t)nlong);
        } else {
            const double z = zero[i - 1];
            const double u = sqrt((1.0 - z) * (1.0 + z));
            const int i_s = nlat + 1 - i;
            synth_ring(&t, cilm, cdim, csphase, z, u, cr, ci, csr, csi);
            for (int m = 1; m <= lc; ++m) { cr[m] = cr[m] / 2.0; ci[m] = ci[m] / 2.0; }
            fft_c2r(plan, cr, ci, row, wr, wi);
            memcpy(&grid[(size_t)(i - 1) * nlong_out], row, sizeof(double) * (size_t)nlong);
            for (int m = 1; m <= lc; ++m) { csr[m] = csr[m] / 2.0; csi[m] = csi[m] / 2.0; }
            fft_c2r(plan, csr, csi, row, wr, wi);
            memcpy(&grid[(size_t)(i_s - 1) * nlong_out], row, sizeof(double) * (size_t)nlong);
        }
    }
    if (extend == 1)
        for (int i = 0; i < nlat; ++i)
            grid[(size_t)i * nlong_out + nlong] = grid[(size_t)i * nlong_out];
    free(cr); free(ci); free(csr); free(csi); free(wr); free(wi); free(row);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

int orc_makegrid_glq(double *grid, const double *cilm, int cdim, int lmax,
                     const double *zero, int norm, int csphase, int lmax_calc,
                     int extend) {
    return makegrid_glq_impl(grid, cilm, cdim, lmax, zero, norm, csphase,
                             lmax_calc, extend, 0, 1 << 30);
}

int orc_makegrid_glq_window(double *grid, const double *cilm, int cdim,
                            int lmax, const double *zero, int norm, int csphase,
                            int lmax_calc, int extend, int pair_lo, int pair_hi) {
    return makegrid_glq_impl(grid, cilm, cdim, lmax, zero, norm, csphase,
                             lmax_calc, extend, pair_lo, pair_hi);
}

/* ------------------------------------------------------------------------ */
/*  SHExpandGLQ  (SHExpandGLQ.f95:98-691, on-the-fly branch :445-649)        */
/*  grid: (lmax+1) x ncols row-major, ncols >= 2lmax+1.                      */
/* ------------------------------------------------------------------------ */

static int shexpand_glq_impl(double *cilm, int cdim, int lmax, const double *grid,
                             int ncols, const double *w, const double *zero,
                             int norm, int csphase, int lmax_calc, int pair_lo,
                             int pair_hi) {
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax) return ORC_EBOUND;
    if (cdim < lc + 1) return ORC_EDIM;
    if (ncols < 2 * lmax + 1) return ORC_EDIM;
    if (!zero) return ORC_ECONV;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    const int nlong = 2 * (lmax + 1) - 1, nlat = lmax + 1;
    const double pi = acos(-1.0);
    memset(cilm, 0, sizeof(double) * 2 * (size_t)cdim * cdim);
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    const int nh = nlong / 2 + 1;
    double *ccr = malloc(sizeof(double) * (size_t)nh), *cci = malloc(sizeof(double) * (size_t)nh);
    double *f1r = malloc(sizeof(double) * (size_t)(lmax + 1)), *f1i = malloc(sizeof(double) * (size_t)(lmax + 1));
    double *f2r = malloc(sizeof(double) * (size_t)(lmax + 1)), *f2i = malloc(sizeof(double) * (size_t)(lmax + 1));
    double *wr = malloc(sizeof(double) * (size_t)nlong), *wi = malloc(sizeof(double) * (size_t)nlong);
    if (pair_lo < 0) pair_lo = 0;
    for (int i = 1; i <= (nlat + 1) / 2; ++i) {
        if (i - 1 < pair_lo || i - 1 >= pair_hi) continue;
        fft_r2c(plan, &grid[(size_t)(i - 1) * ncols], ccr, cci, wr, wi);
        for (int k = 0; k <= lmax; ++k) {
            f1r[k] = 2 * w[i - 1] * pi * ccr[k] / (double)nlong;
            f1i[k] = -2 * w[i - 1] * pi * cci[k] / (double)nlong;
        }
        if (i == (nlat + 1) / 2 && nlat % 2 != 0) {
            anal_equator(&t, cilm, cdim, csphase, f1r, f1i);
        } else {
            const double z = zero[i - 1];
            const double u = sqrt((1.0 - z) * (1.0 + z));
            const int i_s = nlat + 1 - i;
            fft_r2c(plan, &grid[(size_t)(i_s - 1) * ncols], ccr, cci, wr, wi);
            for (int k = 0; k <= lmax; ++k) {
                f2r[k] = 2 * w[i_s - 1] * pi * ccr[k] / (double)nlong;
                f2i[k] = -2 * w[i_s - 1] * pi * cci[k] / (double)nlong;
            }
            anal_ring(&t, cilm, cdim, csphase, z, u, f1r, f1i, f2r, f2i);
        }
    }
    anal_normalise(cilm, cdim, lc, norm);
    free(ccr); free(cci); free(f1r); free(f1i); free(f2r); free(f2i); free(wr); free(wi);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

int orc_shexpand_glq(double *cilm, int cdim, int lmax, const double *grid,
                     int ncols, const double *w, const double *zero, int norm,
                     int csphase, int lmax_calc) {
    return shexpand_glq_impl(cilm, cdim, lmax, grid, ncols, w, zero, norm,
                             csphase, lmax_calc, 0, 1 << 30);
}

int orc_shexpand_glq_window(double *cilm, int cdim, int lmax, const double *grid,
                            int ncols, const double *w, const double *zero,
                            int norm, int csphase, int lmax_calc, int pair_lo,
                            int pair_hi) {
    return shexpand_glq_impl(cilm, cdim, lmax, grid, ncols, w, zero, norm,
                             csphase, lmax_calc, pair_lo, pair_hi);
}

/* ======================================================================== */
/*  Complex transforms                                                      */
/*    MakeGridDHC  ........ src/MakeGridDHC.f95:100-643                      */
/*    SHExpandDHC  ........ src/SHExpandDHC.f95:100-725                      */
/*    MakeGridGLQC ........ src/MakeGridGLQC.f95 (on-the-fly branch)         */
/*    SHExpandGLQC ........ src/SHExpandGLQC.f95 (on-the-fly branch)         */
/*  cilm[k][l][m][re/im] (2, cdim, cdim) complex: k = 0 the order +m, k = 1  */
/*  the order -m (Y*_lm = (-1)^m Y_l,-m); grids [i][j][re/im].  The tables  */
/*  ff1/ff2 are those of the real transforms; the sectoral start omits the  */
/*  real transforms' sqrt(2), and the norm-3 divisors omit their 1/2.       */
/*  Longitude transforms are complex DFTs of length nlong (FFTW backward    */
/*  for synthesis, forward for analysis, both unnormalised).                */
/* ======================================================================== */

#define CCR(k, l, m) cilm[((((size_t)(k) * cdim + (size_t)(l)) * cdim + (size_t)(m)) * 2)]
#define CCI(k, l, m) cilm[((((size_t)(k) * cdim + (size_t)(l)) * cdim + (size_t)(m)) * 2) + 1]

static double pmm_start_c(int norm) {
    const double pi = acos(-1.0);
    return norm == 4 ? SCALEF / sqrt(4.0 * pi) : SCALEF;   /* no sqr(2) */
}

/* pmm update of the sectoral recursion; returns pm2 (the m-th start value) */
static double pmm_step(const rec_tab *t, int phase, int m, double *pmm) {
    const double *sqr = t->sqr;
    switch (t->norm) {
        case 1: case 4:
            *pmm = phase * *pmm * sqr[2 * m + 1] / sqr[2 * m];
            return *pmm;
        case 2:
            *pmm = phase * *pmm * sqr[2 * m + 1] / sqr[2 * m];
            return *pmm / sqr[2 * m + 1];
        default:
            *pmm = phase * *pmm * (double)(2 * m - 1);
            return *pmm;
    }
}

/* pmm of m = lc, times rescalem (the closing term of every latitude) */
static double pmm_last(const rec_tab *t, int phase, double pmm, double rescalem) {
    const double *sqr = t->sqr;
    const int lc = t->lc;
    switch (t->norm) {
        case 1: case 4: return phase * pmm * sqr[2 * lc + 1] / sqr[2 * lc] * rescalem;
        case 2: return phase * pmm / sqr[2 * lc] * rescalem;
        default: return phase * pmm * (double)(2 * lc - 1) * rescalem;
    }
}

static double msign(int m) { return (m % 2 == 0) ? 1.0 : -1.0; }

/* Synthesis of one ring pair (MakeGridDHC.f95:530-620): coef (north) and
 * coefs (south), complex arrays of length nlong, zero on entry. */
static void synthc_ring(const rec_tab *t, const double *cilm, int cdim, int phase,
                        double z, double u, int nlong, double *cr, double *ci,
                        double *sr, double *si) {
    const int lc = t->lc, d = lc + 1, norm = t->norm;
    const double *ff1 = t->ff1, *ff2 = t->ff2;
    double pm2, pm1, p, pmm, rescalem, tr, ti;

    pm2 = p00(norm);
    tr = CCR(0, 0, 0) * pm2; ti = CCI(0, 0, 0) * pm2;
    cr[0] += tr; ci[0] += ti;
    sr[0] += tr; si[0] += ti;

    pm1 = ff1[(size_t)1 * d + 0] * z * pm2;
    tr = CCR(0, 1, 0) * pm1; ti = CCI(0, 1, 0) * pm1;
    cr[0] += tr; ci[0] += ti;
    sr[0] -= tr; si[0] -= ti;

    for (int l = 2; l <= lc; ++l) {
        p = ff1[(size_t)l * d + 0] * z * pm1 - ff2[(size_t)l * d + 0] * pm2;
        tr = CCR(0, l, 0) * p; ti = CCI(0, l, 0) * p;
        cr[0] += tr; ci[0] += ti;
        const double fs = (l % 2 == 0) ? 1.0 : -1.0;
        sr[0] += tr * fs; si[0] += ti * fs;
        pm2 = pm1;
        pm1 = p;
    }

    pmm = pmm_start_c(norm);
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        const int mn = nlong - m;            /* Fortran nlong-(m-1), 0-based */
        rescalem = rescalem * u;
        pm2 = pmm_step(t, phase, m, &pmm);

        tr = CCR(0, m, m) * pm2; ti = CCI(0, m, m) * pm2;
        cr[m] += tr; ci[m] += ti; sr[m] += tr; si[m] += ti;
        tr = CCR(1, m, m) * pm2; ti = CCI(1, m, m) * pm2;
        cr[mn] += tr; ci[mn] += ti; sr[mn] += tr; si[mn] += ti;

        pm1 = z * ff1[(size_t)(m + 1) * d + m] * pm2;
        tr = CCR(0, m + 1, m) * pm1; ti = CCI(0, m + 1, m) * pm1;
        cr[m] += tr; ci[m] += ti; sr[m] -= tr; si[m] -= ti;
        tr = CCR(1, m + 1, m) * pm1; ti = CCI(1, m + 1, m) * pm1;
        cr[mn] += tr; ci[mn] += ti; sr[mn] -= tr; si[mn] -= ti;

        for (int l = m + 2; l <= lc; ++l) {
            p = z * ff1[(size_t)l * d + m] * pm1 - ff2[(size_t)l * d + m] * pm2;
            pm2 = pm1;
            pm1 = p;
            const double fs = ((l - m) % 2 == 0) ? 1.0 : -1.0;
            tr = CCR(0, l, m) * p; ti = CCI(0, l, m) * p;
            cr[m] += tr; ci[m] += ti; sr[m] += tr * fs; si[m] += ti * fs;
            tr = CCR(1, l, m) * p; ti = CCI(1, l, m) * p;
            cr[mn] += tr; ci[mn] += ti; sr[mn] += tr * fs; si[mn] += ti * fs;
        }
        cr[m] = cr[m] * rescalem; ci[m] = ci[m] * rescalem;
        sr[m] = sr[m] * rescalem; si[m] = si[m] * rescalem;
        cr[mn] = cr[mn] * rescalem * msign(m); ci[mn] = ci[mn] * rescalem * msign(m);
        sr[mn] = sr[mn] * rescalem * msign(m); si[mn] = si[mn] * rescalem * msign(m);
    }

    rescalem = rescalem * u;
    pmm = pmm_last(t, phase, pmm, rescalem);
    tr = CCR(0, lc, lc) * pmm; ti = CCI(0, lc, lc) * pmm;
    cr[lc] += tr; ci[lc] += ti; sr[lc] += tr; si[lc] += ti;
    tr = CCR(1, lc, lc) * pmm * msign(lc); ti = CCI(1, lc, lc) * pmm * msign(lc);
    cr[nlong - lc] += tr; ci[nlong - lc] += ti;
    sr[nlong - lc] += tr; si[nlong - lc] += ti;
}

/* Equator ring (MakeGridDHC.f95:424-497): z = 0, even l-m only */
static void synthc_equator(const rec_tab *t, const double *cilm, int cdim, int phase,
                           int nlong, double *cr, double *ci) {
    const int lc = t->lc, d = lc + 1, norm = t->norm;
    const double *ff2 = t->ff2;
    double pm2, p, pmm, rescalem;

    pm2 = p00(norm);
    cr[0] += CCR(0, 0, 0) * pm2; ci[0] += CCI(0, 0, 0) * pm2;
    for (int l = 2; l <= lc; l += 2) {
        p = -ff2[(size_t)l * d + 0] * pm2;
        pm2 = p;
        cr[0] += CCR(0, l, 0) * p; ci[0] += CCI(0, l, 0) * p;
    }
    pmm = pmm_start_c(norm);
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        const int mn = nlong - m;
        pm2 = pmm_step(t, phase, m, &pmm);
        cr[m] += CCR(0, m, m) * pm2; ci[m] += CCI(0, m, m) * pm2;
        cr[mn] += CCR(1, m, m) * pm2; ci[mn] += CCI(1, m, m) * pm2;
        for (int l = m + 2; l <= lc; l += 2) {
            p = -ff2[(size_t)l * d + m] * pm2;
            cr[m] += CCR(0, l, m) * p; ci[m] += CCI(0, l, m) * p;
            cr[mn] += CCR(1, l, m) * p; ci[mn] += CCI(1, l, m) * p;
            pm2 = p;
        }
        cr[m] = cr[m] * rescalem; ci[m] = ci[m] * rescalem;
        cr[mn] = cr[mn] * rescalem * msign(m); ci[mn] = ci[mn] * rescalem * msign(m);
    }
    pmm = pmm_last(t, phase, pmm, rescalem);
    cr[lc] += CCR(0, lc, lc) * pmm; ci[lc] += CCI(0, lc, lc) * pmm;
    cr[nlong - lc] += CCR(1, lc, lc) * pmm * msign(lc);
    ci[nlong - lc] += CCI(1, lc, lc) * pmm * msign(lc);
}

/* Analysis of one ring pair (SHExpandDHC.f95:552-658); f1/f2 are the
 * weighted complex spectra of the north / south rings (length nlong),
 * rescaled in place as in Fortran. */
static void analc_ring(const rec_tab *t, double *cilm, int cdim, int phase, double z,
                       double u, int nlong, double *f1r, double *f1i, double *f2r,
                       double *f2i) {
    const int lc = t->lc, d = lc + 1, norm = t->norm;
    const double *ff1 = t->ff1, *ff2 = t->ff2;
    double pm2, pm1, p, pmm, rescalem;
    double a1r[2], a1i[2], a2r[2], a2i[2];   /* [0]: fsymsign -1, [1]: +1 */

    pm2 = p00(norm);
    CCR(0, 0, 0) += pm2 * (f1r[0] + f2r[0]);
    CCI(0, 0, 0) += pm2 * (f1i[0] + f2i[0]);
    if (lc == 0) return;
    pm1 = ff1[(size_t)1 * d + 0] * z * pm2;
    CCR(0, 1, 0) += pm1 * (f1r[0] - f2r[0]);
    CCI(0, 1, 0) += pm1 * (f1i[0] - f2i[0]);
    a1r[0] = f1r[0] - f2r[0]; a1i[0] = f1i[0] - f2i[0];
    a1r[1] = f1r[0] + f2r[0]; a1i[1] = f1i[0] + f2i[0];
    for (int l = 2; l <= lc; ++l) {
        p = ff1[(size_t)l * d + 0] * z * pm1 - ff2[(size_t)l * d + 0] * pm2;
        pm2 = pm1;
        pm1 = p;
        const int s = (l % 2 == 0) ? 1 : 0;
        CCR(0, l, 0) += p * a1r[s];
        CCI(0, l, 0) += p * a1i[s];
    }
    pmm = pmm_start_c(norm);
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        const int mn = nlong - m;
        rescalem = rescalem * u;
        pm2 = pmm_step(t, phase, m, &pmm);
        f1r[m] = f1r[m] * rescalem; f1i[m] = f1i[m] * rescalem;
        f1r[mn] = f1r[mn] * rescalem * msign(m); f1i[mn] = f1i[mn] * rescalem * msign(m);
        f2r[m] = f2r[m] * rescalem; f2i[m] = f2i[m] * rescalem;
        f2r[mn] = f2r[mn] * rescalem * msign(m); f2i[mn] = f2i[mn] * rescalem * msign(m);

        CCR(0, m, m) += pm2 * (f1r[m] + f2r[m]);
        CCI(0, m, m) += pm2 * (f1i[m] + f2i[m]);
        CCR(1, m, m) += pm2 * (f1r[mn] + f2r[mn]);
        CCI(1, m, m) += pm2 * (f1i[mn] + f2i[mn]);

        pm1 = z * ff1[(size_t)(m + 1) * d + m] * pm2;
        CCR(0, m + 1, m) += pm1 * (f1r[m] - f2r[m]);
        CCI(0, m + 1, m) += pm1 * (f1i[m] - f2i[m]);
        CCR(1, m + 1, m) += pm1 * (f1r[mn] - f2r[mn]);
        CCI(1, m + 1, m) += pm1 * (f1i[mn] - f2i[mn]);

        a1r[0] = f1r[m] - f2r[m]; a1i[0] = f1i[m] - f2i[m];
        a1r[1] = f1r[m] + f2r[m]; a1i[1] = f1i[m] + f2i[m];
        a2r[0] = f1r[mn] - f2r[mn]; a2i[0] = f1i[mn] - f2i[mn];
        a2r[1] = f1r[mn] + f2r[mn]; a2i[1] = f1i[mn] + f2i[mn];
        for (int l = m + 2; l <= lc; ++l) {
            p = z * ff1[(size_t)l * d + m] * pm1 - ff2[(size_t)l * d + m] * pm2;
            pm2 = pm1;
            pm1 = p;
            const int s = ((l - m) % 2 == 0) ? 1 : 0;
            CCR(0, l, m) += p * a1r[s]; CCI(0, l, m) += p * a1i[s];
            CCR(1, l, m) += p * a2r[s]; CCI(1, l, m) += p * a2i[s];
        }
    }
    rescalem = rescalem * u;
    pmm = pmm_last(t, phase, pmm, rescalem);
    CCR(0, lc, lc) += pmm * (f1r[lc] + f2r[lc]);
    CCI(0, lc, lc) += pmm * (f1i[lc] + f2i[lc]);
    CCR(1, lc, lc) += msign(lc) * pmm * (f1r[nlong - lc] + f2r[nlong - lc]);
    CCI(1, lc, lc) += msign(lc) * pmm * (f1i[nlong - lc] + f2i[nlong - lc]);
}

/* Equator ring of the analysis (SHExpandDHC.f95:465-548) */
static void analc_equator(const rec_tab *t, double *cilm, int cdim, int phase,
                          int nlong, double *f1r, double *f1i) {
    const int lc = t->lc, d = lc + 1, norm = t->norm;
    const double *ff2 = t->ff2;
    double pm2, p, pmm, rescalem;
    pm2 = p00(norm);
    CCR(0, 0, 0) += pm2 * f1r[0];
    CCI(0, 0, 0) += pm2 * f1i[0];
    if (lc == 0) return;
    for (int l = 2; l <= lc; l += 2) {
        p = -ff2[(size_t)l * d + 0] * pm2;
        pm2 = p;
        CCR(0, l, 0) += p * f1r[0];
        CCI(0, l, 0) += p * f1i[0];
    }
    pmm = pmm_start_c(norm);
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        const int mn = nlong - m;
        pm2 = pmm_step(t, phase, m, &pmm);
        f1r[m] = f1r[m] * rescalem; f1i[m] = f1i[m] * rescalem;
        f1r[mn] = f1r[mn] * rescalem * msign(m); f1i[mn] = f1i[mn] * rescalem * msign(m);
        CCR(0, m, m) += pm2 * f1r[m]; CCI(0, m, m) += pm2 * f1i[m];
        CCR(1, m, m) += pm2 * f1r[mn]; CCI(1, m, m) += pm2 * f1i[mn];
        for (int l = m + 2; l <= lc; l += 2) {
            p = -ff2[(size_t)l * d + m] * pm2;
            pm2 = p;
            CCR(0, l, m) += p * f1r[m]; CCI(0, l, m) += p * f1i[m];
            CCR(1, l, m) += p * f1r[mn]; CCI(1, l, m) += p * f1i[mn];
        }
    }
    pmm = pmm_last(t, phase, pmm, rescalem);
    CCR(0, lc, lc) += pmm * f1r[lc];
    CCI(0, lc, lc) += pmm * f1i[lc];
    CCR(1, lc, lc) += msign(lc) * pmm * f1r[nlong - lc];
    CCI(1, lc, lc) += msign(lc) * pmm * f1i[nlong - lc];
}

/* Divide by the integral of Ylm Ylm* (SHExpandDHC.f95:689-723) */
static void analc_normalise(double *cilm, int cdim, int lc, int norm) {
    const double pi = acos(-1.0);
    for (int l = 0; l <= lc; ++l) {
        if (norm == 1 || norm == 2) {
            for (int k = 0; k < 2; ++k)
                for (int m = 0; m <= l; ++m) {
                    if (norm == 1) {
                        CCR(k, l, m) = CCR(k, l, m) / (4 * pi);
                        CCI(k, l, m) = CCI(k, l, m) / (4 * pi);
                    } else {
                        CCR(k, l, m) = CCR(k, l, m) * (2 * l + 1) / (4 * pi);
                        CCI(k, l, m) = CCI(k, l, m) * (2 * l + 1) / (4 * pi);
                    }
                }
        } else if (norm == 3) {
            double prod = 4 * pi / (double)(2 * l + 1);
            CCR(0, l, 0) = CCR(0, l, 0) / prod;
            CCI(0, l, 0) = CCI(0, l, 0) / prod;
            for (int m = 1; m <= l - 1; ++m) {
                prod = prod * (l + m) * (l - m + 1);
                for (int k = 0; k < 2; ++k) {
                    CCR(k, l, m) = CCR(k, l, m) / prod;
                    CCI(k, l, m) = CCI(k, l, m) / prod;
                }
            }
            if (l != 0)
                for (int k = 0; k < 2; ++k) {
                    CCR(k, l, l) = CCR(k, l, l) / (prod * 2 * l);
                    CCI(k, l, l) = CCI(k, l, l) / (prod * 2 * l);
                }
        }
    }
}

/* writes the backward DFT of (cr, ci) into grid row `row` (complex, ncols) */
static void c2c_row(orc_fft *plan, int nlong, double *cr, double *ci, double *grid,
                    int row, int ncols) {
    orc_fft_exec(plan, cr, ci, +1);
    for (int j = 0; j < nlong; ++j) {
        grid[((size_t)row * ncols + j) * 2] = cr[j];
        grid[((size_t)row * ncols + j) * 2 + 1] = ci[j];
    }
}

int orc_makegrid_dhc(double *grid, const double *cilm, int cdim, int lmax, int norm,
                     int sampling, int csphase, int lmax_calc, int extend) {
    if (sampling != 1 && sampling != 2) return ORC_EBOUND;
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    if (lmax_calc > lmax) return ORC_EBOUND;
    const int n = 2 * lmax + 2;
    const int nlong = sampling == 1 ? n : 2 * n;
    const int nlat_out = n + extend, nlong_out = nlong + extend;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > cdim - 1) lc = cdim - 1;
    const double pi = acos(-1.0);
    if (lc == 0) {
        const double pm2 = p00(norm);
        for (int i = 0; i < nlat_out; ++i)
            for (int j = 0; j < nlong_out; ++j) {
                grid[((size_t)i * nlong_out + j) * 2] = CCR(0, 0, 0) * pm2;
                grid[((size_t)i * nlong_out + j) * 2 + 1] = CCI(0, 0, 0) * pm2;
            }
        return ORC_OK;
    }
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    double *cr = malloc(sizeof(double) * (size_t)nlong), *ci = malloc(sizeof(double) * (size_t)nlong);
    double *sr = malloc(sizeof(double) * (size_t)nlong), *si = malloc(sizeof(double) * (size_t)nlong);
    const int i_eq = n / 2 + 1;   /* 1-based */
    memset(cr, 0, sizeof(double) * (size_t)nlong); memset(ci, 0, sizeof(double) * (size_t)nlong);
    synthc_equator(&t, cilm, cdim, csphase, nlong, cr, ci);
    c2c_row(plan, nlong, cr, ci, grid, i_eq - 1, nlong_out);
    for (int i = 1; i <= i_eq - 1; ++i) {
        const int i_s = 2 * i_eq - i;
        const double theta = pi * (double)(i - 1) / (double)n;
        const double z = cos(theta);
        const double u = sqrt((1.0 - z) * (1.0 + z));
        memset(cr, 0, sizeof(double) * (size_t)nlong); memset(ci, 0, sizeof(double) * (size_t)nlong);
        memset(sr, 0, sizeof(double) * (size_t)nlong); memset(si, 0, sizeof(double) * (size_t)nlong);
        synthc_ring(&t, cilm, cdim, csphase, z, u, nlong, cr, ci, sr, si);
        c2c_row(plan, nlong, cr, ci, grid, i - 1, nlong_out);
        if (!(i == 1 && extend == 0)) c2c_row(plan, nlong, sr, si, grid, i_s - 1, nlong_out);
    }
    if (extend == 1)
        for (int i = 0; i < nlat_out; ++i) {
            grid[((size_t)i * nlong_out + nlong) * 2] = grid[((size_t)i * nlong_out) * 2];
            grid[((size_t)i * nlong_out + nlong) * 2 + 1] = grid[((size_t)i * nlong_out) * 2 + 1];
        }
    free(cr); free(ci); free(sr); free(si);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

/* forward DFT of complex grid row `row` times scale: out = cc * s */
static void row_spectrum(orc_fft *plan, const double *grid, int row, int ncols, int nlong,
                         double *fr, double *fi) {
    for (int j = 0; j < nlong; ++j) {
        fr[j] = grid[((size_t)row * ncols + j) * 2];
        fi[j] = grid[((size_t)row * ncols + j) * 2 + 1];
    }
    orc_fft_exec(plan, fr, fi, -1);
}

int orc_shexpand_dhc(double *cilm, int cdim, const double *grid, int n, int ncols,
                     int norm, int sampling, int csphase, int lmax_calc) {
    const int lmax = n / 2 - 1;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax) return ORC_EBOUND;
    if (sampling != 1 && sampling != 2) return ORC_EBOUND;
    if (n % 2 != 0) return ORC_EBOUND;
    if (cdim < lc + 1) return ORC_EDIM;
    const int nlong = sampling == 1 ? n : 2 * n;
    if (ncols < nlong) return ORC_EDIM;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    const double pi = acos(-1.0);
    memset(cilm, 0, sizeof(double) * 4 * (size_t)cdim * cdim);
    double *aj = malloc(sizeof(double) * (size_t)n);
    orc_dhaj(n, aj, 0);
    for (int i = 0; i < n; ++i) aj[i] = aj[i] * sqrt(4.0 * pi);
    rec_tab t;
    if (rec_build(&t, lc, norm)) { free(aj); return ORC_EALLOC; }
    orc_fft *plan = fft_plan(nlong);
    double *f1r = malloc(sizeof(double) * (size_t)nlong), *f1i = malloc(sizeof(double) * (size_t)nlong);
    double *f2r = malloc(sizeof(double) * (size_t)nlong), *f2i = malloc(sizeof(double) * (size_t)nlong);
    const int i_eq = n / 2 + 1;
    const double s2p = sqrt(2 * pi);
    /* equator first (SHExpandDHC.f95:465) */
    row_spectrum(plan, grid, i_eq - 1, ncols, nlong, f1r, f1i);
    for (int k = 0; k < nlong; ++k) {
        f1r[k] = f1r[k] * s2p * aj[i_eq - 1] / (double)nlong;
        f1i[k] = f1i[k] * s2p * aj[i_eq - 1] / (double)nlong;
    }
    analc_equator(&t, cilm, cdim, csphase, nlong, f1r, f1i);
    for (int i = 2; i <= i_eq - 1; ++i) {
        const double theta = (i - 1) * pi / (double)n;
        const double z = cos(theta);
        const double u = sqrt((1.0 - z) * (1.0 + z));
        const int i_s = 2 * i_eq - i;
        row_spectrum(plan, grid, i - 1, ncols, nlong, f1r, f1i);
        row_spectrum(plan, grid, i_s - 1, ncols, nlong, f2r, f2i);
        for (int k = 0; k < nlong; ++k) {
            f1r[k] = f1r[k] * s2p * aj[i - 1] / (double)nlong;
            f1i[k] = f1i[k] * s2p * aj[i - 1] / (double)nlong;
            f2r[k] = f2r[k] * s2p * aj[i_s - 1] / (double)nlong;
            f2i[k] = f2i[k] * s2p * aj[i_s - 1] / (double)nlong;
        }
        analc_ring(&t, cilm, cdim, csphase, z, u, nlong, f1r, f1i, f2r, f2i);
    }
    analc_normalise(cilm, cdim, lc, norm);
    free(aj); free(f1r); free(f1i); free(f2r); free(f2i);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

int orc_makegrid_glqc(double *grid, const double *cilm, int cdim, int lmax,
                      const double *zero, int norm, int csphase, int lmax_calc,
                      int extend) {
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    if (!zero) return ORC_ECONV;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    if (lmax_calc > lmax) return ORC_EBOUND;
    const int nlong = 2 * lmax + 1, nlat = lmax + 1;
    const int nlong_out = nlong + extend;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > cdim - 1) lc = cdim - 1;
    if (lc == 0) {
        const double pm2 = p00(norm);
        for (int i = 0; i < nlat; ++i)
            for (int j = 0; j < nlong_out; ++j) {
                grid[((size_t)i * nlong_out + j) * 2] = CCR(0, 0, 0) * pm2;
                grid[((size_t)i * nlong_out + j) * 2 + 1] = CCI(0, 0, 0) * pm2;
            }
        return ORC_OK;
    }
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    double *cr = malloc(sizeof(double) * (size_t)nlong), *ci = malloc(sizeof(double) * (size_t)nlong);
    double *sr = malloc(sizeof(double) * (size_t)nlong), *si = malloc(sizeof(double) * (size_t)nlong);
    for (int i = 1; i <= (nlat + 1) / 2; ++i) {
        memset(cr, 0, sizeof(double) * (size_t)nlong); memset(ci, 0, sizeof(double) * (size_t)nlong);
        memset(sr, 0, sizeof(double) * (size_t)nlong); memset(si, 0, sizeof(double) * (size_t)nlong);
        if (i == (nlat + 1) / 2 && nlat % 2 != 0) {
            synthc_equator(&t, cilm, cdim, csphase, nlong, cr, ci);
            c2c_row(plan, nlong, cr, ci, grid, i - 1, nlong_out);
        } else {
            const double z = zero[i - 1];
            const double u = sqrt((1.0 - z) * (1.0 + z));
            const int i_s = nlat + 1 - i;
            synthc_ring(&t, cilm, cdim, csphase, z, u, nlong, cr, ci, sr, si);
            c2c_row(plan, nlong, cr, ci, grid, i - 1, nlong_out);
            c2c_row(plan, nlong, sr, si, grid, i_s - 1, nlong_out);
        }
    }
    if (extend == 1)
        for (int i = 0; i < nlat; ++i) {
            grid[((size_t)i * nlong_out + nlong) * 2] = grid[((size_t)i * nlong_out) * 2];
            grid[((size_t)i * nlong_out + nlong) * 2 + 1] = grid[((size_t)i * nlong_out) * 2 + 1];
        }
    free(cr); free(ci); free(sr); free(si);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

int orc_shexpand_glqc(double *cilm, int cdim, int lmax, const double *grid, int ncols,
                      const double *w, const double *zero, int norm, int csphase,
                      int lmax_calc) {
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax) return ORC_EBOUND;
    if (cdim < lc + 1) return ORC_EDIM;
    if (ncols < 2 * lmax + 1) return ORC_EDIM;
    if (!zero) return ORC_ECONV;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    const int nlong = 2 * (lmax + 1) - 1, nlat = lmax + 1;
    const double pi = acos(-1.0);
    memset(cilm, 0, sizeof(double) * 4 * (size_t)cdim * cdim);
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    double *f1r = malloc(sizeof(double) * (size_t)nlong), *f1i = malloc(sizeof(double) * (size_t)nlong);
    double *f2r = malloc(sizeof(double) * (size_t)nlong), *f2i = malloc(sizeof(double) * (size_t)nlong);
    for (int i = 1; i <= (nlat + 1) / 2; ++i) {
        row_spectrum(plan, grid, i - 1, ncols, nlong, f1r, f1i);
        for (int k = 0; k < nlong; ++k) {
            const double s = 2 * w[i - 1] * pi;
            f1r[k] = s * f1r[k] / (double)nlong;
            f1i[k] = s * f1i[k] / (double)nlong;
        }
        if (i == (nlat + 1) / 2 && nlat % 2 != 0) {
            analc_equator(&t, cilm, cdim, csphase, nlong, f1r, f1i);
        } else {
            const double z = zero[i - 1];
            const double u = sqrt((1.0 - z) * (1.0 + z));
            const int i_s = nlat + 1 - i;
            row_spectrum(plan, grid, i_s - 1, ncols, nlong, f2r, f2i);
            for (int k = 0; k < nlong; ++k) {
                const double s = 2 * w[i_s - 1] * pi;
                f2r[k] = s * f2r[k] / (double)nlong;
                f2i[k] = s * f2i[k] / (double)nlong;
            }
            analc_ring(&t, cilm, cdim, csphase, z, u, nlong, f1r, f1i, f2r, f2i);
        }
    }
    analc_normalise(cilm, cdim, lc, norm);
    free(f1r); free(f1i); free(f2r); free(f2i);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

/* ======================================================================== */
/*  MakeGradientDH (src/MakeGradientDH.f95:1-658): horizontal gradient of a  */
/*  4-pi normalised real field (csphase 1) on a DH grid,                     */
/*      theta = (1/r) dF/dtheta,  phi = 1/(r sin theta) dF/dphi,             */
/*  dP/dz from (1-z^2) dP_l/dz = a_l P_(l-1) - l z P_l; zero at the poles.   */
/*  theta, phi: (n+extend) x (nlong+extend) row-major.                       */
/* ======================================================================== */

/* one ring's m = 0..lc sums for the c2r (halved for m >= 1 by the caller):
 * north (t, p) and south (ts, ps); rounding order of MakeGradientDH.f95:427-549 */
static void grad_ring(const rec_tab *t, const double *cilm, int cdim, double z, double u,
                      double *tr, double *ti, double *pr, double *pi_, double *tsr,
                      double *tsi, double *psr, double *psi) {
    const int lc = t->lc, d = lc + 1;
    const double *sqr = t->sqr, *ff1 = t->ff1, *ff2 = t->ff2;
    double pm2, pm1, p, pmm, rescalem, dpl, tempr, c_r, c_i;
    double coeft0 = 0.0, coefts0 = 0.0;

    pm2 = 1.0;
    pm1 = 0.0;
    if (lc != 0) {
        pm1 = ff1[(size_t)1 * d + 0] * z;
        dpl = ff1[(size_t)1 * d + 0];
        tempr = CIL(0, 1, 0) * dpl;
        coeft0 = coeft0 + tempr;
        coefts0 = coefts0 + tempr;
    }
    for (int l = 2; l <= lc; ++l) {
        p = ff1[(size_t)l * d + 0] * z * pm1 - ff2[(size_t)l * d + 0] * pm2;
        dpl = l * (sqr[2 * l + 1] / sqr[2 * l - 1] * pm1 - z * p) / (u * u);
        tempr = CIL(0, l, 0) * dpl;
        coeft0 = coeft0 + tempr;
        coefts0 = coefts0 - tempr * ((l % 2 == 0) ? 1.0 : -1.0);
        pm2 = pm1;
        pm1 = p;
    }
    tr[0] = coeft0; ti[0] = 0.0; tsr[0] = coefts0; tsi[0] = 0.0;
    pr[0] = 0.0; pi_[0] = 0.0; psr[0] = 0.0; psi[0] = 0.0;

    pmm = sqr[2] * SCALEF;   /* sqr(2) * scalef */
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        double atr = 0, ati = 0, atsr = 0, atsi = 0, apr = 0, api = 0, apsr = 0, apsi = 0;
        rescalem = rescalem * u;
        pmm = pmm * sqr[2 * m + 1] / sqr[2 * m];
        pm2 = pmm;
        /* (m, m): tempc = cmplx(S, C) * pm2 * m */
        c_r = CIL(1, m, m) * pm2 * m; c_i = CIL(0, m, m) * pm2 * m;
        apr += c_r; api += c_i; apsr += c_r; apsi += c_i;
        dpl = -m * z * pm2 / (u * u);
        c_r = CIL(0, m, m) * dpl; c_i = -CIL(1, m, m) * dpl;
        atr += c_r; ati += c_i; atsr -= c_r; atsi -= c_i;

        pm1 = z * ff1[(size_t)(m + 1) * d + m] * pm2;
        c_r = CIL(1, m + 1, m) * pm1 * m; c_i = CIL(0, m + 1, m) * pm1 * m;
        apr += c_r; api += c_i; apsr -= c_r; apsi -= c_i;
        dpl = (sqr[2 * m + 3] * pmm - z * (m + 1) * pm1) / (u * u);
        c_r = CIL(0, m + 1, m) * dpl; c_i = -CIL(1, m + 1, m) * dpl;
        atr += c_r; ati += c_i; atsr += c_r; atsi += c_i;

        for (int l = m + 2; l <= lc; ++l) {
            p = z * ff1[(size_t)l * d + m] * pm1 - ff2[(size_t)l * d + m] * pm2;
            const double fs = ((l - m) % 2 == 0) ? 1.0 : -1.0;
            c_r = CIL(1, l, m) * p * m; c_i = CIL(0, l, m) * p * m;
            apr += c_r; api += c_i; apsr += c_r * fs; apsi += c_i * fs;
            dpl = (sqr[2 * l + 1] * sqr[l - m] * sqr[l + m] / sqr[2 * l - 1] * pm1
                   - z * l * p) / (u * u);
            c_r = CIL(0, l, m) * dpl; c_i = -CIL(1, l, m) * dpl;
            atr += c_r; ati += c_i; atsr -= c_r * fs; atsi -= c_i * fs;
            pm2 = pm1;
            pm1 = p;
        }
        tr[m] = atr * rescalem; ti[m] = ati * rescalem;
        tsr[m] = atsr * rescalem; tsi[m] = atsi * rescalem;
        pr[m] = apr * rescalem; pi_[m] = api * rescalem;
        psr[m] = apsr * rescalem; psi[m] = apsi * rescalem;
    }
    if (lc != 0) {
        rescalem = rescalem * u;
        pmm = pmm * sqr[2 * lc + 1] / sqr[2 * lc] * rescalem;
        c_r = CIL(1, lc, lc) * pmm * lc; c_i = CIL(0, lc, lc) * pmm * lc;
        pr[lc] = c_r; pi_[lc] = c_i; psr[lc] = c_r; psi[lc] = c_i;
        dpl = -lc * z * pmm / (u * u);
        c_r = CIL(0, lc, lc) * dpl; c_i = -CIL(1, lc, lc) * dpl;
        tr[lc] = c_r; ti[lc] = c_i; tsr[lc] = -c_r; tsi[lc] = -c_i;
    }
}

/* c2r of m = 0..lc sums (m >= 1 halved, the rest zero) into row `row` times s */
static void grad_row(orc_fft *plan, int nlong, int lc, const double *cr, const double *ci,
                     double *wr, double *wi, double *row, double s, double sfac_div,
                     double *out) {
    const int nh = nlong / 2 + 1;
    double *ar = malloc(sizeof(double) * (size_t)nh), *ai = malloc(sizeof(double) * (size_t)nh);
    for (int k = 0; k < nh; ++k) { ar[k] = 0.0; ai[k] = 0.0; }
    ar[0] = cr[0]; ai[0] = 0.0;
    for (int m = 1; m <= lc && m < nh; ++m) { ar[m] = cr[m] / 2.0; ai[m] = ci[m] / 2.0; }
    fft_c2r(plan, ar, ai, row, wr, wi);
    for (int j = 0; j < nlong; ++j) out[j] = sfac_div != 0.0 ? row[j] / s / sfac_div : s * row[j];
    free(ar); free(ai);
}

int orc_makegradient_dh(double *theta_g, double *phi_g, const double *cilm, int cdim,
                        int lmax, int sampling, int lmax_calc, int extend, double radius) {
    if (sampling != 1 && sampling != 2) return ORC_EBOUND;
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    if (lmax_calc > lmax) return ORC_EBOUND;
    const int n = 2 * lmax + 2;
    const int nlong = sampling == 1 ? n : 2 * n;
    const int nlong_out = nlong + extend, nlat_out = n + extend;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > cdim - 1) lc = cdim - 1;
    const double pi = acos(-1.0);
    const double r = radius;
    rec_tab t;
    if (rec_build(&t, lc, 1)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    const int L2 = lc + 2;
    double *b[8];
    for (int k = 0; k < 8; ++k) b[k] = calloc((size_t)L2, sizeof(double));
    double *wr = malloc(sizeof(double) * (size_t)nlong), *wi = malloc(sizeof(double) * (size_t)nlong);
    double *row = malloc(sizeof(double) * (size_t)nlong);
    const int i_eq = n / 2 + 1;
    memset(theta_g, 0, sizeof(double) * (size_t)nlat_out * nlong_out);
    memset(phi_g, 0, sizeof(double) * (size_t)nlat_out * nlong_out);
    for (int i = 1; i <= i_eq; ++i) {
        const double theta = i == i_eq ? pi / 2.0 : pi * (double)(i - 1) / (double)n;
        const double z = i == i_eq ? 0.0 : cos(theta);
        const double u = i == i_eq ? 1.0 : sqrt((1.0 - z) * (1.0 + z));
        const int i_s = 2 * i_eq - i;
        if (i == 1) continue;   /* undefined at the poles: zero rows */
        for (int k = 0; k < 8; ++k) memset(b[k], 0, sizeof(double) * (size_t)L2);
        grad_ring(&t, cilm, cdim, z, u, b[0], b[1], b[2], b[3], b[4], b[5], b[6], b[7]);
        const double st = sin(theta);
        /* theta = -sin(theta) * grid / r ; phi = grid / r / sin(theta) */
        grad_row(plan, nlong, lc, b[0], b[1], wr, wi, row, -st, 0.0,
                 &theta_g[(size_t)(i - 1) * nlong_out]);
        for (int j = 0; j < nlong; ++j) theta_g[(size_t)(i - 1) * nlong_out + j] /= r;
        grad_row(plan, nlong, lc, b[2], b[3], wr, wi, row, r, st,
                 &phi_g[(size_t)(i - 1) * nlong_out]);
        if (i != i_eq) {
            grad_row(plan, nlong, lc, b[4], b[5], wr, wi, row, -st, 0.0,
                     &theta_g[(size_t)(i_s - 1) * nlong_out]);
            for (int j = 0; j < nlong; ++j) theta_g[(size_t)(i_s - 1) * nlong_out + j] /= r;
            grad_row(plan, nlong, lc, b[6], b[7], wr, wi, row, r, st,
                     &phi_g[(size_t)(i_s - 1) * nlong_out]);
        }
    }
    if (extend == 1)
        for (int i = 0; i < nlat_out; ++i) {
            theta_g[(size_t)i * nlong_out + nlong] = theta_g[(size_t)i * nlong_out];
            phi_g[(size_t)i * nlong_out + nlong] = phi_g[(size_t)i * nlong_out];
        }
    for (int k = 0; k < 8; ++k) free(b[k]);
    free(wr); free(wi); free(row);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

/* ======================================================================== */
/*  SHMultiply (src/SHMultiply.f95:1-375): the product of two fields of      */
/*  degrees lmax1 and lmax2 expanded to lmax1 + lmax2 through a GLQ grid of */
/*  that degree: MakeGridGLQ of both, pointwise product, SHExpandGLQ.       */
/*  cilm arrays are (2, dim, dim); cilmout must have dim >= lmax1+lmax2+1.  */
/* ======================================================================== */
int orc_shmultiply(double *cout, int cdout, const double *c1, int cd1, int lmax1,
                   const double *c2, int cd2, int lmax2, int norm, int csphase) {
    if (cd1 < lmax1 + 1 || cd2 < lmax2 + 1 || cdout < lmax1 + lmax2 + 1) return ORC_EDIM;
    const int lo = lmax1 + lmax2;
    const int nlat = lo + 1, nlong = 2 * lo + 1;
    double *zero = malloc(sizeof(double) * (size_t)nlat), *w = malloc(sizeof(double) * (size_t)nlat);
    int rc = orc_preglq(-1.0, 1.0, nlat, zero, w);
    /* the fields restricted to their degrees (cilm1(1:2,1:lmax1+1,1:lmax1+1)) */
    double *a1 = calloc((size_t)2 * (lmax1 + 1) * (lmax1 + 1), sizeof(double));
    double *a2 = calloc((size_t)2 * (lmax2 + 1) * (lmax2 + 1), sizeof(double));
    for (int k = 0; k < 2; ++k)
        for (int l = 0; l <= lmax1; ++l)
            for (int m = 0; m <= lmax1; ++m)
                a1[((size_t)k * (lmax1 + 1) + l) * (lmax1 + 1) + m] =
                    c1[((size_t)k * cd1 + l) * cd1 + m];
    for (int k = 0; k < 2; ++k)
        for (int l = 0; l <= lmax2; ++l)
            for (int m = 0; m <= lmax2; ++m)
                a2[((size_t)k * (lmax2 + 1) + l) * (lmax2 + 1) + m] =
                    c2[((size_t)k * cd2 + l) * cd2 + m];
    double *g1 = malloc(sizeof(double) * (size_t)nlat * nlong);
    double *g2 = malloc(sizeof(double) * (size_t)nlat * nlong);
    if (!rc) rc = orc_makegrid_glq(g1, a1, lmax1 + 1, lo, zero, norm, csphase, -1, 0);
    if (!rc) rc = orc_makegrid_glq(g2, a2, lmax2 + 1, lo, zero, norm, csphase, -1, 0);
    if (!rc) {
        for (size_t i = 0; i < (size_t)nlat * nlong; ++i) g1[i] = g1[i] * g2[i];
        rc = orc_shexpand_glq(cout, cdout, lo, g1, nlong, w, zero, norm, csphase, lo);
    }
    free(zero); free(w); free(a1); free(a2); free(g1); free(g2);
    return rc;
}

/* ======================================================================== */
/*  NormalGravity (src/NormalGravity.f95): normal gravity on a rotating     */
/*  flattened ellipsoid (Somigliana), at geocentric latitude in degrees.     */
/* ======================================================================== */
double orc_normal_gravity(double geocentric_lat, double gm, double omega, double a,
                          double b) {
    const double pi = acos(-1.0);
    if (a == b && omega == 0.0) return gm / (a * a);
    if (a == b) {
        const double c = cos(geocentric_lat * pi / 180.0);
        const double g = gm * gm / ((a * a) * (a * a))
                         + a * (omega * omega) * (c * c) * (a * (omega * omega)
                                                            - 2.0 * gm / (a * a));
        return sqrt(g);
    }
    const double m = (omega * omega) * (a * a) * b / gm;
    const double bigE = sqrt(a * a - b * b);       /* linear eccentricity */
    const double ep = bigE / b;                    /* second eccentricity */
    const double be = b / bigE;
    const double q0 = 0.50 * ((1.0 + 3.0 * (be * be)) * atan(bigE / b) - 3.0 * b / bigE);
    const double q0p = 3.0 * (1.0 + (be * be)) * (1.0 - b / bigE * atan(bigE / b)) - 1.0;
    const double ga = gm / (a * b) * (1.0 - m - m * ep * q0p / 6.0 / q0);
    const double gb = gm / (a * a) * (1.0 + m * ep * q0p / 3.0 / q0);
    const double ab = a / b;
    const double gl = atan((ab * ab) * tan(geocentric_lat * pi / 180.0));
    const double cg = cos(gl), sg = sin(gl);
    double ng = a * ga * (cg * cg) + b * gb * (sg * sg);
    return ng / sqrt((a * a) * (cg * cg) + (b * b) * (sg * sg));
}

/* ======================================================================== */
/*  MakeGravGridDH (src/MakeGravGridDH.f95:1-1069): gravity vector          */
/*  (radial positive up, theta, phi), its magnitude and the potential on a  */
/*  DH grid over a flattened ellipsoid of semi-major axis a and flattening  */
/*  f.  V = GM/r sum_l (r0/r)^l sum_m C_lm Y_lm (4pi, no Condon-Shortley);  */
/*  r on ring i is the ellipsoid radius r_ex at the ring's geocentric        */
/*  latitude, applied through prefactor(l) = (r0/r_ex)^l.                   */
/* ======================================================================== */

/* accumulators of one ring: 8 complex sums over m = 0..lc (north and south
 * of rad, pot, theta, phi) */
enum { GR = 0, GRS, GU, GUS, GT, GTS, GP, GPS, GNSUM };

/* one ring's sums, rounding order of MakeGravGridDH.f95:657-877 (the
 * equator block, 383-585, is this with z = 0, u = 1) */
static void grav_ring(const rec_tab *t, const double *cilm, int cdim, double z, double u,
                      const double *pref, int calcu, double **sr, double **si) {
    const int lc = t->lc, d = lc + 1;
    const double *sqr = t->sqr, *ff1 = t->ff1, *ff2 = t->ff2;
    const double uu = u * u;
    const int deriv = u != 0.0;   /* theta/phi sums are not used on the poles */
    double pm2, pm1, p, pmm, rescalem, dpl, tempr;
    double r0 = 0.0, rs0 = 0.0, u0 = 0.0, us0 = 0.0, t0 = 0.0, ts0 = 0.0;

    pm2 = 1.0;
    pm1 = 0.0;
    tempr = -CIL(0, 0, 0) * pm2;
    r0 = r0 + tempr; rs0 = rs0 + tempr;
    if (calcu) { tempr = CIL(0, 0, 0) * pm2; u0 = u0 + tempr; us0 = us0 + tempr; }
    if (lc != 0) {
        pm1 = ff1[(size_t)1 * d + 0] * z;
        tempr = CIL(0, 1, 0) * pm1 * (-2.0) * pref[1];
        r0 = r0 + tempr; rs0 = rs0 - tempr;
        if (calcu) { tempr = CIL(0, 1, 0) * pm1 * pref[1]; u0 = u0 + tempr; us0 = us0 - tempr; }
        dpl = ff1[(size_t)1 * d + 0];
        tempr = CIL(0, 1, 0) * dpl * pref[1];
        t0 = t0 + tempr; ts0 = ts0 + tempr;
    }
    for (int l = 2; l <= lc; ++l) {
        const double fs = (l % 2 == 0) ? 1.0 : -1.0;
        p = ff1[(size_t)l * d + 0] * z * pm1 - ff2[(size_t)l * d + 0] * pm2;
        tempr = CIL(0, l, 0) * p * (double)(-(l + 1)) * pref[l];
        r0 = r0 + tempr; rs0 = rs0 + tempr * fs;
        if (calcu) {
            tempr = CIL(0, l, 0) * p * pref[l];
            u0 = u0 + tempr; us0 = us0 + tempr * fs;
        }
        if (deriv) {
            dpl = l * (sqr[2 * l + 1] / sqr[2 * l - 1] * pm1 - z * p) / uu;
            tempr = CIL(0, l, 0) * dpl * pref[l];
            t0 = t0 + tempr; ts0 = ts0 - tempr * fs;
        }
        pm2 = pm1;
        pm1 = p;
    }
    sr[GR][0] = r0; sr[GRS][0] = rs0; sr[GU][0] = u0; sr[GUS][0] = us0;
    sr[GT][0] = t0; sr[GTS][0] = ts0; sr[GP][0] = 0.0; sr[GPS][0] = 0.0;
    for (int k = 0; k < GNSUM; ++k) si[k][0] = 0.0;

    pmm = sqr[2] * SCALEF;
    rescalem = 1.0 / SCALEF;
    for (int m = 1; m <= lc - 1; ++m) {
        double ar[GNSUM] = {0}, ai[GNSUM] = {0};
        double cr, ci;
        rescalem = rescalem * u;
        pmm = pmm * sqr[2 * m + 1] / sqr[2 * m];
        pm2 = pmm;
        /* (m, m), fsymsign = 1 */
        cr = CIL(0, m, m) * pm2 * (double)(-m - 1) * pref[m];
        ci = -CIL(1, m, m) * pm2 * (double)(-m - 1) * pref[m];
        ar[GR] += cr; ai[GR] += ci; ar[GRS] += cr; ai[GRS] += ci;
        if (calcu) {
            cr = CIL(0, m, m) * pm2 * pref[m]; ci = -CIL(1, m, m) * pm2 * pref[m];
            ar[GU] += cr; ai[GU] += ci; ar[GUS] += cr; ai[GUS] += ci;
        }
        cr = CIL(1, m, m) * pm2 * pref[m] * m; ci = CIL(0, m, m) * pm2 * pref[m] * m;
        ar[GP] += cr; ai[GP] += ci; ar[GPS] += cr; ai[GPS] += ci;
        if (deriv) {
            dpl = -m * z * pm2 / uu;
            cr = CIL(0, m, m) * dpl * pref[m]; ci = -CIL(1, m, m) * dpl * pref[m];
            ar[GT] += cr; ai[GT] += ci; ar[GTS] -= cr; ai[GTS] -= ci;
        }
        /* (m+1, m), fsymsign = -1 */
        pm1 = z * ff1[(size_t)(m + 1) * d + m] * pm2;
        cr = CIL(0, m + 1, m) * pm1 * (double)(-m - 2) * pref[m + 1];
        ci = -CIL(1, m + 1, m) * pm1 * (double)(-m - 2) * pref[m + 1];
        ar[GR] += cr; ai[GR] += ci; ar[GRS] -= cr; ai[GRS] -= ci;
        if (calcu) {
            cr = CIL(0, m + 1, m) * pm1 * pref[m + 1];
            ci = -CIL(1, m + 1, m) * pm1 * pref[m + 1];
            ar[GU] += cr; ai[GU] += ci; ar[GUS] -= cr; ai[GUS] -= ci;
        }
        cr = CIL(1, m + 1, m) * pm1 * pref[m + 1] * m;
        ci = CIL(0, m + 1, m) * pm1 * pref[m + 1] * m;
        ar[GP] += cr; ai[GP] += ci; ar[GPS] -= cr; ai[GPS] -= ci;
        if (deriv) {
            dpl = (sqr[2 * m + 3] * pmm - z * (m + 1) * pm1) / uu;
            cr = CIL(0, m + 1, m) * dpl * pref[m + 1];
            ci = -CIL(1, m + 1, m) * dpl * pref[m + 1];
            ar[GT] += cr; ai[GT] += ci; ar[GTS] += cr; ai[GTS] += ci;
        }
        for (int l = m + 2; l <= lc; ++l) {
            const double fs = ((l - m) % 2 == 0) ? 1.0 : -1.0;
            p = z * ff1[(size_t)l * d + m] * pm1 - ff2[(size_t)l * d + m] * pm2;
            cr = CIL(0, l, m) * p * (double)(-(l + 1)) * pref[l];
            ci = -CIL(1, l, m) * p * (double)(-(l + 1)) * pref[l];
            ar[GR] += cr; ai[GR] += ci; ar[GRS] += cr * fs; ai[GRS] += ci * fs;
            if (calcu) {
                cr = CIL(0, l, m) * p * pref[l]; ci = -CIL(1, l, m) * p * pref[l];
                ar[GU] += cr; ai[GU] += ci; ar[GUS] += cr * fs; ai[GUS] += ci * fs;
            }
            cr = CIL(1, l, m) * p * pref[l] * m; ci = CIL(0, l, m) * p * pref[l] * m;
            ar[GP] += cr; ai[GP] += ci; ar[GPS] += cr * fs; ai[GPS] += ci * fs;
            if (deriv) {
                dpl = (sqr[2 * l + 1] * sqr[l - m] * sqr[l + m] / sqr[2 * l - 1] * pm1
                       - z * l * p) / uu;
                cr = CIL(0, l, m) * dpl * pref[l]; ci = -CIL(1, l, m) * dpl * pref[l];
                ar[GT] += cr; ai[GT] += ci; ar[GTS] -= cr * fs; ai[GTS] -= ci * fs;
            }
            pm2 = pm1;
            pm1 = p;
        }
        for (int k = 0; k < GNSUM; ++k) {
            sr[k][m] = ar[k] * rescalem;
            si[k][m] = ai[k] * rescalem;
        }
    }
    if (lc != 0) {
        double cr, ci;
        for (int k = 0; k < GNSUM; ++k) { sr[k][lc] = 0.0; si[k][lc] = 0.0; }
        rescalem = rescalem * u;
        pmm = pmm * sqr[2 * lc + 1] / sqr[2 * lc] * rescalem;
        cr = CIL(0, lc, lc) * pmm * (double)(-lc - 1) * pref[lc];
        ci = -CIL(1, lc, lc) * pmm * (double)(-lc - 1) * pref[lc];
        sr[GR][lc] = cr; si[GR][lc] = ci; sr[GRS][lc] = cr; si[GRS][lc] = ci;
        if (calcu) {
            cr = CIL(0, lc, lc) * pmm * pref[lc]; ci = -CIL(1, lc, lc) * pmm * pref[lc];
            sr[GU][lc] = cr; si[GU][lc] = ci; sr[GUS][lc] = cr; si[GUS][lc] = ci;
        }
        cr = CIL(1, lc, lc) * pmm * pref[lc] * lc; ci = CIL(0, lc, lc) * pmm * pref[lc] * lc;
        sr[GP][lc] = cr; si[GP][lc] = ci; sr[GPS][lc] = cr; si[GPS][lc] = ci;
        if (deriv) {
            dpl = -lc * z * pmm / uu;
            cr = CIL(0, lc, lc) * dpl * pref[lc]; ci = -CIL(1, lc, lc) * dpl * pref[lc];
            sr[GT][lc] = cr; si[GT][lc] = ci; sr[GTS][lc] = -cr; si[GTS][lc] = -ci;
        }
    }
}

/* c2r of the m = 0..lc sums (m >= 1 halved, the rest, Nyquist included,
 * zero) into row[0..nlong-1] */
static void grav_c2r(orc_fft *plan, int nlong, int lc, const double *cr, const double *ci,
                     double *wr, double *wi, double *row) {
    const int nh = nlong / 2 + 1;
    double *ar = calloc((size_t)nh, sizeof(double)), *ai = calloc((size_t)nh, sizeof(double));
    ar[0] = cr[0];
    for (int m = 1; m <= lc && m < nh; ++m) { ar[m] = cr[m] / 2.0; ai[m] = ci[m] / 2.0; }
    fft_c2r(plan, ar, ai, row, wr, wi);
    free(ar); free(ai);
}

/* rad, theta, phi, total: (n+extend) x (nlong+extend) row-major; pot may be
 * NULL.  has_omega = 0 is the reference's absent OMEGA (no rotation terms).
 * Returns the reference's exit status (5: normal gravity without omega). */
int orc_makegravgrid_dh(double *rad, double *theta_g, double *phi_g, double *total,
                        double *pot, const double *cilm, int cdim, int lmax, double gm,
                        double r0, double a, double f, int sampling, int lmax_calc,
                        int has_omega, double omega, int normal_gravity,
                        double normal_gravity_gm, int extend) {
    if (cdim < 1) return ORC_EDIM;
    if (sampling != 1 && sampling != 2) return ORC_EBOUND;
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    if (normal_gravity != 0 && normal_gravity != 1) return ORC_EBOUND;
    if (normal_gravity == 1 && !has_omega) return 5;
    if (lmax_calc > lmax) return ORC_EBOUND;
    const int n = 2 * lmax + 2;
    const int nlong = sampling == 1 ? n : 2 * n;
    const int nlong_out = nlong + extend, nlat_out = n + extend;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > cdim - 1) lc = cdim - 1;
    if (lc > lmax) lc = lmax;
    const int calcu = pot != NULL;
    const double pi = acos(-1.0);
    rec_tab t;
    if (rec_build(&t, lc, 1)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    const int L2 = lc + 2;
    double *sr[GNSUM], *si[GNSUM];
    for (int k = 0; k < GNSUM; ++k) {
        sr[k] = calloc((size_t)L2, sizeof(double));
        si[k] = calloc((size_t)L2, sizeof(double));
    }
    double *pref = calloc((size_t)L2, sizeof(double));
    double *wr = malloc(sizeof(double) * (size_t)nlong), *wi = malloc(sizeof(double) * (size_t)nlong);
    double *row = malloc(sizeof(double) * (size_t)nlong);
    const size_t gsz = (size_t)nlat_out * nlong_out;
    memset(rad, 0, sizeof(double) * gsz);
    memset(theta_g, 0, sizeof(double) * gsz);
    memset(phi_g, 0, sizeof(double) * gsz);
    memset(total, 0, sizeof(double) * gsz);
    if (calcu) memset(pot, 0, sizeof(double) * gsz);
    const int i_eq = n / 2 + 1;
    for (int i = 1; i <= i_eq; ++i) {
        const int eq = i == i_eq;
        const double theta = eq ? pi / 2.0 : pi * (double)(i - 1) / (double)n;
        const double z = eq ? 0.0 : cos(theta);
        const double u = eq ? 1.0 : sqrt((1.0 - z) * (1.0 + z));
        const int i_s = 2 * i_eq - i;
        double r_ex;
        if (eq) {
            r_ex = a;
        } else if (i == 1) {
            r_ex = a * (1.0 - f);
        } else {
            const double lat = pi / 2.0 - theta;
            const double cl = cos(lat), sl = sin(lat);
            r_ex = cl * cl + sl * sl / ((1.0 - f) * (1.0 - f));
            r_ex = a * sqrt(1.0 / r_ex);
        }
        if (lc != 0) {
            pref[1] = r0 / r_ex;
            for (int l = 2; l <= lc; ++l) pref[l] = pref[l - 1] * r0 / r_ex;
        }
        grav_ring(&t, cilm, cdim, z, u, pref, calcu, sr, si);
        const double st = sin(theta);
        const double r2 = r_ex * r_ex;
        /* north ring (or the equator) */
        double *o;
        o = &rad[(size_t)(i - 1) * nlong_out];
        grav_c2r(plan, nlong, lc, sr[GR], si[GR], wr, wi, row);
        for (int j = 0; j < nlong; ++j) o[j] = row[j] * gm / r2;
        if (calcu) {
            o = &pot[(size_t)(i - 1) * nlong_out];
            grav_c2r(plan, nlong, lc, sr[GU], si[GU], wr, wi, row);
            for (int j = 0; j < nlong; ++j) o[j] = row[j] * gm / r_ex;
        }
        if (i != 1) {
            o = &theta_g[(size_t)(i - 1) * nlong_out];
            grav_c2r(plan, nlong, lc, sr[GT], si[GT], wr, wi, row);
            for (int j = 0; j < nlong; ++j) o[j] = -st * row[j] * gm / r2;
            o = &phi_g[(size_t)(i - 1) * nlong_out];
            grav_c2r(plan, nlong, lc, sr[GP], si[GP], wr, wi, row);
            for (int j = 0; j < nlong; ++j) o[j] = row[j] * (gm / r2) / st;
        }
        /* south ring; the south pole only with extend */
        if (!eq && !(i == 1 && extend == 0)) {
            o = &rad[(size_t)(i_s - 1) * nlong_out];
            grav_c2r(plan, nlong, lc, sr[GRS], si[GRS], wr, wi, row);
            for (int j = 0; j < nlong; ++j) o[j] = row[j] * gm / r2;
            if (calcu) {
                o = &pot[(size_t)(i_s - 1) * nlong_out];
                grav_c2r(plan, nlong, lc, sr[GUS], si[GUS], wr, wi, row);
                for (int j = 0; j < nlong; ++j) o[j] = row[j] * gm / r_ex;
            }
            if (i != 1) {
                o = &theta_g[(size_t)(i_s - 1) * nlong_out];
                grav_c2r(plan, nlong, lc, sr[GTS], si[GTS], wr, wi, row);
                for (int j = 0; j < nlong; ++j) o[j] = -st * row[j] * gm / r2;
                o = &phi_g[(size_t)(i_s - 1) * nlong_out];
                grav_c2r(plan, nlong, lc, sr[GPS], si[GPS], wr, wi, row);
                for (int j = 0; j < nlong; ++j) o[j] = row[j] * (gm / r2) / st;
            }
        }
    }
    /* rotation (MakeGravGridDH.f95:987-1013) */
    if (has_omega) {
        for (int i = 1; i <= nlat_out; ++i) {
            const double theta = pi * (double)(i - 1) / (double)n;
            const double lat = pi / 2.0 - theta;
            const double tl = tan(lat);
            double r_ex = (1.0 + tl * tl) / (1.0 + tl * tl / ((1.0 - f) * (1.0 - f)));
            r_ex = a * sqrt(r_ex);
            const double st = sin(theta), ct = cos(theta);
            const double so = st * omega;
            const double rr = r_ex * (so * so);
            const double tt = st * ct * r_ex * (omega * omega);
            const double ro = r_ex * st * omega;
            const double pp = 0.50 * (ro * ro);
            for (int j = 0; j < nlong; ++j) {
                rad[(size_t)(i - 1) * nlong_out + j] += rr;
                theta_g[(size_t)(i - 1) * nlong_out + j] += tt;
                if (calcu) pot[(size_t)(i - 1) * nlong_out + j] += pp;
            }
        }
    }
    for (int i = 0; i < nlat_out; ++i)
        for (int j = 0; j < nlong; ++j) {
            const size_t k = (size_t)i * nlong_out + j;
            total[k] = sqrt(rad[k] * rad[k] + phi_g[k] * phi_g[k] + theta_g[k] * theta_g[k]);
        }
    if (normal_gravity == 1) {
        const double b = a * (1.0 - f);
        for (int i = 1; i <= nlat_out; ++i) {
            const double theta = pi * (double)(i - 1) / (double)n;
            const double lat = (pi / 2.0 - theta) * 180.0 / pi;
            const double ng = orc_normal_gravity(lat, normal_gravity_gm, omega, a, b);
            for (int j = 0; j < nlong; ++j) total[(size_t)(i - 1) * nlong_out + j] -= ng;
        }
    }
    if (extend == 1)
        for (int i = 0; i < nlat_out; ++i) {
            const size_t k = (size_t)i * nlong_out;
            rad[k + nlong] = rad[k];
            theta_g[k + nlong] = theta_g[k];
            phi_g[k + nlong] = phi_g[k];
            total[k + nlong] = total[k];
            if (calcu) pot[k + nlong] = pot[k];
        }
    for (int k = 0; k < GNSUM; ++k) { free(sr[k]); free(si[k]); }
    free(pref); free(wr); free(wi); free(row);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

/* Number of host threads OpenMP would use (1 when built without OpenMP). */
int orc_max_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/*  Transposes (adjoints) of the four real transforms, built from the same   */
/*  ring loops: they pin the GPU's autograd backward passes.                 */
/*  The synthesis writes per ring x_j = sum_m (a_m cos m phi_j + b_m sin m   */
/*  phi_j) with a_m = sum_l C_lm P_lm, b_m = sum_l S_lm P_lm                 */
/*  (MakeGridDH.f95:504-639, c2r of (a_m - i b_m)/2 for m >= 1), so its      */
/*  transpose takes Y = r2c(row) of the grid cotangent, unweighted, and      */
/*  accumulates C_lm += P_lm Re Y_m, S_lm += P_lm (-Im Y_m) over every ring   */
/*  the synthesis writes (poles included, the extend column folded into      */
/*  column 0), without the analysis normalisation.  The analysis             */
/*  (SHExpandDH.f95:463-702) is C = N^-1 sum_i w_i P_lm (Re, -Im) Y_m(row i)   */
/*  with w_i = sqrt(2 pi) a_i sqrt(4 pi) / nlong (DH) or 2 pi w_i / nlong     */
/*  (GLQ); its transpose is the synthesis of N^-1 cbar with row i scaled by   */
/*  w_i.                                                                     */
/* ------------------------------------------------------------------------ */

/* grid: (n + extend) x (nlong + extend) row-major (the synthesis output shape) */
int orc_makegrid_dh_adjoint(double *cilm, int cdim, const double *grid, int lmax,
                            int norm, int sampling, int csphase, int lmax_calc,
                            int extend) {
    if (sampling != 1 && sampling != 2) return ORC_EBOUND;
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    const int n = 2 * lmax + 2;
    const int nlong = sampling == 1 ? n : 2 * n;
    const int ncols = nlong + extend;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax) lc = lmax;
    if (lc > cdim - 1) lc = cdim - 1;
    const double pi = acos(-1.0);
    memset(cilm, 0, sizeof(double) * 2 * (size_t)cdim * cdim);
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    const int nh = nlong / 2 + 1;
    double *row = malloc(sizeof(double) * (size_t)nlong);
    double *ccr = malloc(sizeof(double) * (size_t)nh), *cci = malloc(sizeof(double) * (size_t)nh);
    double *f1r = calloc((size_t)lmax + 2, sizeof(double)), *f1i = calloc((size_t)lmax + 2, sizeof(double));
    double *f2r = calloc((size_t)lmax + 2, sizeof(double)), *f2i = calloc((size_t)lmax + 2, sizeof(double));
    double *wr = malloc(sizeof(double) * (size_t)nlong), *wi = malloc(sizeof(double) * (size_t)nlong);
    const int i_eq = n / 2 + 1;
    /* spectrum (Re Y, -Im Y) of a row with the extend column folded in */
    #define ROWSPEC(r, fr, fi) do {                                              \
        for (int j = 0; j < nlong; ++j) row[j] = grid[(size_t)(r) * ncols + j];  \
        if (extend) row[0] += grid[(size_t)(r) * ncols + nlong];                \
        fft_r2c(plan, row, ccr, cci, wr, wi);                                    \
        for (int k = 0; k <= lc; ++k) { fr[k] = ccr[k]; fi[k] = -cci[k]; }        \
    } while (0)
    for (int i = 1; i <= i_eq - 1; ++i) {
        const double theta = pi * (double)(i - 1) / (double)n;
        const double z = cos(theta);
        const double u = sqrt((1.0 - z) * (1.0 + z));
        const int i_s = 2 * i_eq - i;
        ROWSPEC(i - 1, f1r, f1i);
        if (i == 1 && extend == 0) {
            for (int k = 0; k <= lc; ++k) { f2r[k] = 0.0; f2i[k] = 0.0; }
        } else {
            ROWSPEC(i_s - 1, f2r, f2i);
        }
        if (lc == 0) {
            CIL(0, 0, 0) += p00(norm) * (f1r[0] + f2r[0]);
        } else {
            anal_ring(&t, cilm, cdim, csphase, z, u, f1r, f1i, f2r, f2i);
        }
    }
    ROWSPEC(i_eq - 1, f1r, f1i);
    if (lc == 0) CIL(0, 0, 0) += p00(norm) * f1r[0];
    else anal_equator(&t, cilm, cdim, csphase, f1r, f1i);
    #undef ROWSPEC
    free(row); free(ccr); free(cci); free(f1r); free(f1i); free(f2r); free(f2i);
    free(wr); free(wi);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

/* grid: (lmax + 1) x (2 lmax + 1 + extend) row-major */
int orc_makegrid_glq_adjoint(double *cilm, int cdim, const double *grid, int lmax,
                             const double *zero, int norm, int csphase, int lmax_calc,
                             int extend) {
    if (extend != 0 && extend != 1) return ORC_EBOUND;
    if (!zero) return ORC_ECONV;
    if (norm < 1 || norm > 4) return ORC_EBOUND;
    if (csphase != 1 && csphase != -1) return ORC_EBOUND;
    const int nlong = 2 * lmax + 1, nlat = lmax + 1, ncols = nlong + extend;
    int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax) lc = lmax;
    if (lc > cdim - 1) lc = cdim - 1;
    memset(cilm, 0, sizeof(double) * 2 * (size_t)cdim * cdim);
    rec_tab t;
    if (rec_build(&t, lc, norm)) return ORC_EALLOC;
    orc_fft *plan = fft_plan(nlong);
    const int nh = nlong / 2 + 1;
    double *row = malloc(sizeof(double) * (size_t)nlong);
    double *ccr = malloc(sizeof(double) * (size_t)nh), *cci = malloc(sizeof(double) * (size_t)nh);
    double *f1r = calloc((size_t)lmax + 2, sizeof(double)), *f1i = calloc((size_t)lmax + 2, sizeof(double));
    double *f2r = calloc((size_t)lmax + 2, sizeof(double)), *f2i = calloc((size_t)lmax + 2, sizeof(double));
    double *wr = malloc(sizeof(double) * (size_t)nlong), *wi = malloc(sizeof(double) * (size_t)nlong);
    #define ROWSPEC(r, fr, fi) do {                                              \
        for (int j = 0; j < nlong; ++j) row[j] = grid[(size_t)(r) * ncols + j];  \
        if (extend) row[0] += grid[(size_t)(r) * ncols + nlong];                \
        fft_r2c(plan, row, ccr, cci, wr, wi);                                    \
        for (int k = 0; k <= lc; ++k) { fr[k] = ccr[k]; fi[k] = -cci[k]; }        \
    } while (0)
    for (int i = 1; i <= (nlat + 1) / 2; ++i) {
        ROWSPEC(i - 1, f1r, f1i);
        if (i == (nlat + 1) / 2 && nlat % 2 != 0) {
            if (lc == 0) CIL(0, 0, 0) += p00(norm) * f1r[0];
            else anal_equator(&t, cilm, cdim, csphase, f1r, f1i);
        } else {
            const double z = zero[i - 1];
            const double u = sqrt((1.0 - z) * (1.0 + z));
            ROWSPEC(nlat - i, f2r, f2i);
            if (lc == 0) CIL(0, 0, 0) += p00(norm) * (f1r[0] + f2r[0]);
            else anal_ring(&t, cilm, cdim, csphase, z, u, f1r, f1i, f2r, f2i);
        }
    }
    #undef ROWSPEC
    free(row); free(ccr); free(cci); free(f1r); free(f1i); free(f2r); free(f2i);
    free(wr); free(wi);
    fft_free(plan);
    rec_free(&t);
    return ORC_OK;
}

/* grid (output): n x nlong row-major; cilm: (2, cdim, cdim), l, m <= lmax_calc used */
int orc_shexpand_dh_adjoint(double *grid, const double *cilm, int cdim, int n, int norm,
                            int sampling, int csphase, int lmax_calc) {
    if (n % 2 != 0) return ORC_EBOUND;
    if (sampling != 1 && sampling != 2) return ORC_EBOUND;
    const int lmax = n / 2 - 1;
    const int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax || cdim < lc + 1) return ORC_EBOUND;
    const int nlong = sampling == 1 ? n : 2 * n;
    const double pi = acos(-1.0);
    double *cn = calloc(2 * (size_t)cdim * cdim, sizeof(double));
    memcpy(cn, cilm, sizeof(double) * 2 * (size_t)cdim * cdim);
    anal_normalise(cn, cdim, lc, norm);
    int rc = orc_makegrid_dh(grid, cn, cdim, lmax, norm, sampling, csphase, lc, 0);
    free(cn);
    if (rc) return rc;
    double *aj = malloc(sizeof(double) * (size_t)n);
    orc_dhaj(n, aj, 0);
    for (int i = 0; i < n; ++i) {
        const double wi = sqrt(2 * pi) * (aj[i] * sqrt(4.0 * pi)) / (double)nlong;
        for (int j = 0; j < nlong; ++j) grid[(size_t)i * nlong + j] *= wi;
    }
    free(aj);
    return ORC_OK;
}

/* grid (output): (lmax + 1) x (2 lmax + 1) row-major */
int orc_shexpand_glq_adjoint(double *grid, const double *cilm, int cdim, int lmax,
                             const double *w, const double *zero, int norm, int csphase,
                             int lmax_calc) {
    const int lc = lmax_calc < 0 ? lmax : lmax_calc;
    if (lc > lmax || cdim < lc + 1) return ORC_EBOUND;
    if (!w || !zero) return ORC_ECONV;
    const int nlong = 2 * lmax + 1, nlat = lmax + 1;
    const double pi = acos(-1.0);
    double *cn = calloc(2 * (size_t)cdim * cdim, sizeof(double));
    memcpy(cn, cilm, sizeof(double) * 2 * (size_t)cdim * cdim);
    anal_normalise(cn, cdim, lc, norm);
    int rc = orc_makegrid_glq(grid, cn, cdim, lmax, zero, norm, csphase, lc, 0);
    free(cn);
    if (rc) return rc;
    for (int i = 0; i < nlat; ++i) {
        const double wi = 2 * w[i] * pi / (double)nlong;
        for (int j = 0; j < nlong; ++j) grid[(size_t)i * nlong + j] *= wi;
    }
    return ORC_OK;
}
