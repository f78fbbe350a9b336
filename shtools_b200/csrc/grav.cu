// MakeGravGridDH (src/MakeGravGridDH.f95) and NormalGravity
// (src/NormalGravity.f95) on the GPU.
//
// The potential V = GM/r sum_l (r0/r)^l sum_m C_lm Y_lm is evaluated on a DH
// grid whose ring i lies on the ellipsoid of semi-major axis a and flattening
// f, at radius r_i.  Per ring and order the reference accumulates four sums
// of c_l (r0/r_i)^l times P_lm, dP_lm/dz and their radial factors
// (MakeGravGridDH.f95:657-877).  Here, with q = r0 / r_i per ring pair and
// (1 - z^2) dP_l/dz = a_l P_(l-1) - l z P_l, a_l = sqrt((2l+1)(l-m)(l+m)/(2l-1)),
// everything follows from three ordinary Legendre sums per field
//     S0 = sum_l c_l q^l P_l,  S1 = sum_l c_(l+1) a_(l+1) q^l P_l,
//     S2 = sum_l l c_l q^l P_l,
// which the synthesis kernels evaluate in one recursion pass (internal
// fields 3u, 3u+1, 3u+2).  The factor q^l = q^m q^s multiplies each term
// (legendre.cuh, RAD): q^s from a table of accurate powers at every
// recursion segment, q^m = exp(m log q) in the epilogue, log q computed
// from q to twice double precision, so that the powers carry no s-fold
// rounding of q.  Per ring (g2 = GM/r^2, g1 = GM/r):
//     rad   = -(S2 + S0) g2                    (sum of -(l+1) c_l q^l P_l)
//     pot   =  S0 g1
//     theta = -sin(theta) (q S1 - z S2) / u^2 g2   (zero on the poles)
//     phi   =  i m S0 g2 / sin(theta)              (zero on the poles)
// The centrifugal terms of a row (MakeGravGridDH.f95:987-1013) are constants
// added to the m = 0 Fourier bin, which adds them to every sample of the
// c2r output; four c2r FFTs then write rad, theta, phi and pot, and one
// pointwise pass forms |g| and removes the normal gravity (:1015-1044).
#include <cuda_runtime.h>
#include <math.h>

#include "legendre.cuh"
#include "shtc_internal.cuh"

namespace shtc {

constexpr double kPi = 3.141592653589793238462643383279502884;

// NormalGravity.f95:73-110, Somigliana's formula for a rotating ellipsoid
// (geocentric latitude in degrees); a == b gives the spherical branches
__host__ __device__ double normal_gravity(double geocentric_lat, double gm, double omega,
                                          double a, double b) {
    if (a == b && omega == 0.0) return gm / (a * a);
    if (a == b) {
        const double c = cos(geocentric_lat * kPi / 180.0);
        return sqrt(gm * gm / ((a * a) * (a * a)) +
                    a * (omega * omega) * (c * c) * (a * (omega * omega) - 2.0 * gm / (a * a)));
    }
    const double m = (omega * omega) * (a * a) * b / gm;
    const double bigE = sqrt(a * a - b * b);   // linear eccentricity
    const double ep = bigE / b;                // second eccentricity
    const double be = b / bigE;
    const double at = atan(bigE / b);
    const double q0 = 0.5 * ((1.0 + 3.0 * (be * be)) * at - 3.0 * b / bigE);
    const double q0p = 3.0 * (1.0 + be * be) * (1.0 - b / bigE * at) - 1.0;
    const double ga = gm / (a * b) * (1.0 - m - m * ep * q0p / 6.0 / q0);
    const double gb = gm / (a * a) * (1.0 + m * ep * q0p / 3.0 / q0);
    const double ab = a / b;
    const double gl = atan((ab * ab) * tan(geocentric_lat * kPi / 180.0));
    const double cg = cos(gl), sg = sin(gl);
    return (a * ga * (cg * cg) + b * gb * (sg * sg)) /
           sqrt((a * a) * (cg * cg) + (b * b) * (sg * sg));
}

// Per ring pair p (theta = pi p / n): the ellipsoid radius r (a(1-f) on the
// poles, a on the equator, MakeGravGridDH.f95:383, 644-652), q = r0 / r,
// radq = {q, log q}, ringg = {GM/r^2, GM/r}.  log q = log(qh) + ql / qh with
// q = qh + ql to twice double precision (ql from the exact remainder
// r0 - qh r).  Per output row i: the centrifugal terms {r sin^2 w^2,
// sin cos r w^2, (r sin w)^2 / 2} with the row's radius in the reference's
// tan form (:991-995) and the normal gravity.
__global__ void k_grav_setup(int npair, int n, int nlat_out, GravParams g,
                             double2* __restrict__ radq, double2* __restrict__ ringg,
                             double* __restrict__ rows) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < npair) {
        double rex;
        if (2 * i == n) {
            rex = g.a;
        } else if (i == 0) {
            rex = g.a * (1.0 - g.f);
        } else {
            const double lat = kPi / 2.0 - kPi * (double)i / (double)n;
            const double cl = cos(lat), sl = sin(lat);
            rex = g.a * sqrt(1.0 / (cl * cl + sl * sl / ((1.0 - g.f) * (1.0 - g.f))));
        }
        const double qh = g.r0 / rex;
        const double ql = fma(-qh, rex, g.r0) / rex;
        radq[i] = make_double2(qh, log(qh) + ql / qh);
        ringg[i] = make_double2(g.gm / (rex * rex), g.gm / rex);
    } else if (i < npair + nlat_out) {
        const int r = i - npair;
        const double theta = kPi * (double)r / (double)n;
        double rr = 0.0, tt = 0.0, pp = 0.0, ng = 0.0;
        if (g.has_omega) {
            const double tl = tan(kPi / 2.0 - theta);
            const double rex =
                g.a * sqrt((1.0 + tl * tl) / (1.0 + tl * tl / ((1.0 - g.f) * (1.0 - g.f))));
            const double st = sin(theta), ct = cos(theta);
            const double so = st * g.omega, ro = rex * st * g.omega;
            rr = rex * (so * so);
            tt = st * ct * rex * (g.omega * g.omega);
            pp = 0.5 * (ro * ro);
        }
        if (g.normal_gravity)
            ng = normal_gravity((kPi / 2.0 - theta) * 180.0 / kPi, g.ng_gm, g.omega, g.a,
                                g.a * (1.0 - g.f));
        rows[4 * r + 0] = rr;
        rows[4 * r + 1] = tt;
        rows[4 * r + 2] = pp;
        rows[4 * r + 3] = ng;
    }
}

// qtab[p * nseg + k] = q_p^(16k + 1) = exp((16k + 1) log q_p)
__global__ void k_grav_qpow(const double2* __restrict__ radq, int npair, int nseg,
                            double* __restrict__ qtab) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= (long long)npair * nseg) return;
    const int p = (int)(i / nseg), k = (int)(i % nseg);
    qtab[i] = exp((double)(kRecSegment * k + 1) * radq[p].y);
}

static int grav_nseg(const shtc_plan* P) { return P->lc / kRecSegment + 1; }

// synthesis of the three sums with the radial factor (legendre.cuh, RAD)
template <int T, int NF>
__global__ void __launch_bounds__(128)
k_legendre_synth_rad(const double2* __restrict__ rec, const double* __restrict__ pmm,
                     const double* __restrict__ rtab, const double* __restrict__ zp,
                     const double2* __restrict__ radq, const double* __restrict__ qtab,
                     int nseg, const double2* __restrict__ coef, double2* __restrict__ spec,
                     int lc, int npair, int nfield) {
    __shared__ __align__(16) SynthStage<NF> sm;
    synth_order<T, NF, true>(sm, rec, pmm, rtab, zp, coef, spec, lc, npair, nfield,
                             blockIdx.y, blockIdx.x, blockIdx.z * NF, NF, radq, qtab, nseg);
}

template <int T, int NF>
static int launch_synth_rad_t(const shtc_plan* P, const double2* packed, double2* spec,
                              int nfield, const double2* radq, const double* qtab,
                              cudaStream_t st) {
    const int threads = 128;
    const int tiles = (P->npair + threads * T - 1) / (threads * T);
    dim3 grid(tiles, P->lc + 1, nfield / NF);
    k_legendre_synth_rad<T, NF><<<grid, threads, 0, st>>>(
        P->d_rec, P->d_pmm, P->d_rtab, P->d_z, radq, qtab, grav_nseg(P), packed, spec, P->lc,
        P->npair, nfield);
    return map_cuda(cudaGetLastError());
}

// nfield internal fields (three sums per user field) share the recursion and
// the radial powers in groups of NF, with the plain synthesis' shapes
static int launch_synth_rad(const shtc_plan* P, const double2* packed, double2* spec,
                            int nfield, const double2* radq, const double* qtab,
                            cudaStream_t st) {
    const bool wide = P->npair > 512;
    if (nfield % 8 == 0)
        return wide ? launch_synth_rad_t<2, 8>(P, packed, spec, nfield, radq, qtab, st)
                    : launch_synth_rad_t<1, 8>(P, packed, spec, nfield, radq, qtab, st);
    if (nfield % 4 == 0)
        return launch_synth_rad_t<2, 4>(P, packed, spec, nfield, radq, qtab, st);
    if (nfield % 2 == 0)
        return wide ? launch_synth_rad_t<4, 2>(P, packed, spec, nfield, radq, qtab, st)
                    : launch_synth_rad_t<2, 2>(P, packed, spec, nfield, radq, qtab, st);
    return wide ? launch_synth_rad_t<2, 3>(P, packed, spec, nfield, radq, qtab, st)
                : launch_synth_rad_t<1, 3>(P, packed, spec, nfield, radq, qtab, st);
}

// spec fields 3u..3u+2 -> c2r inputs of rad (field u), theta (nfield + u),
// phi (2 nfield + u) and pot (3 nfield + u); with rotation, the m = 0 bins
// of rad, theta and pot also take the row's centrifugal terms
__global__ void k_grav_combine(const double2* __restrict__ spec, double2* __restrict__ out,
                               const double* __restrict__ zp, const double2* __restrict__ radq,
                               const double2* __restrict__ ringg, const int* __restrict__ rowN,
                               const int* __restrict__ rowS, const double* __restrict__ rows,
                               int has_omega, int npair, int lc, int n, int nfield) {
    const long long per = (long long)npair * (lc + 1) * 2;   // one field
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    const int u = blockIdx.y;
    if (i >= per) return;
    const int h = (int)(i & 1);
    const int m = (int)((i >> 1) % (lc + 1));
    const int p = (int)((i >> 1) / (lc + 1));
    const double2 x0 = spec[(3LL * u + 0) * per + i];
    const double2 x1 = spec[(3LL * u + 1) * per + i];
    const double2 x2 = spec[(3LL * u + 2) * per + i];
    const double2 gg = ringg[p];
    const double q = radq[p].x;
    double2 rad = make_double2(-(x2.x + x0.x) * gg.x, -(x2.y + x0.y) * gg.x);
    double2 pot = make_double2(x0.x * gg.y, x0.y * gg.y);
    double2 t = make_double2(0.0, 0.0), f = make_double2(0.0, 0.0);
    if (p > 0) {
        const double z = h ? -zp[p] : zp[p];
        const double uu = (1.0 - z) * (1.0 + z);
        const double st = 2 * p == n ? 1.0 : sinpi((double)p / (double)n);
        const double ct = -st * gg.x / uu;
        t = make_double2(ct * (q * x1.x - z * x2.x), ct * (q * x1.y - z * x2.y));
        const double cp = (double)m * gg.x / st;
        f = make_double2(-cp * x0.y, cp * x0.x);
    }
    if (has_omega && m == 0) {
        const int row = h ? rowS[p] : rowN[p];
        if (row >= 0) {
            rad.x += rows[4 * row + 0];
            t.x += rows[4 * row + 1];
            pot.x += rows[4 * row + 2];
        }
    }
    out[(long long)u * per + i] = rad;
    out[((long long)nfield + u) * per + i] = t;
    out[(2LL * nfield + u) * per + i] = f;
    out[(3LL * nfield + u) * per + i] = pot;
}

// |g| and the normal gravity, per grid point of every output row (the
// extend column included: it repeats column 0)
__global__ void k_grav_post(const double* __restrict__ rad, const double* __restrict__ theta,
                            const double* __restrict__ phi, double* __restrict__ total,
                            long long gf, long long grs, long long gcs, int ncol,
                            const double* __restrict__ rows) {
    const int col = blockIdx.x * blockDim.x + threadIdx.x;
    if (col >= ncol) return;
    const int row = blockIdx.y;
    const long long o = (long long)blockIdx.z * gf + (long long)row * grs + (long long)col * gcs;
    const double r = rad[o], t = theta[o], ph = phi[o];
    total[o] = sqrt(r * r + ph * ph + t * t) - rows[4 * row + 3];
}

// radq, ringg (double2 per pair) | qtab (nseg per pair) | rows (4 per row)
size_t grav_table_bytes(const shtc_plan* P) {
    return sizeof(double) * ((4 + (size_t)grav_nseg(P)) * P->npair + 4 * (size_t)P->nlat_out);
}

int launch_gravity_dh(const shtc_plan* P, const double* cilm, long long sf, long long sk,
                      long long sl, long long sm, int cdim, const GravParams& g,
                      double* rad, double* theta, double* phi, double* total, double* pot,
                      long long gf, long long grs, long long gcs, int nfield,
                      double2* packed, double2* spec, double2* spec2, double* tab,
                      cudaStream_t st, double2* gbuf) {
    const int lc = P->lc, np = P->npair;
    // double2 tables first: tab is 256-byte aligned, np may be odd
    const int nseg = grav_nseg(P);
    double2* radq = (double2*)tab;
    double2* ringg = (double2*)(tab + 2 * (size_t)np);
    double* qtab = tab + 4 * (size_t)np;
    double* rows = qtab + (size_t)nseg * np;
    stage_begin(SHTC_STAGE_PACK, st);
    {
        const int nt = np + P->nlat_out;
        k_grav_setup<<<(nt + 127) / 128, 128, 0, st>>>(np, P->nlat, P->nlat_out, g, radq,
                                                       ringg, rows);
        const long long nq = (long long)np * nseg;
        k_grav_qpow<<<(unsigned)((nq + 255) / 256), 256, 0, st>>>(radq, np, nseg, qtab);
    }
    int rc = map_cuda(cudaGetLastError());
    if (!rc) rc = launch_pack_grad(P, cilm, sf, sk, sl, sm, cdim, packed, nfield, st);
    stage_end(SHTC_STAGE_PACK, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_SYNTH, st);
    rc = launch_synth_rad(P, packed, spec, 3 * nfield, radq, qtab, st);
    stage_end(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_FFT_C2R, st);
    {
        const long long per = (long long)np * (lc + 1) * 2;
        dim3 grid((unsigned)((per + 255) / 256), nfield);
        k_grav_combine<<<grid, 256, 0, st>>>(spec, spec2, P->d_z, radq, ringg, P->d_rowN,
                                             P->d_rowS, rows, g.has_omega, np, lc, P->nlat,
                                             nfield);
        rc = map_cuda(cudaGetLastError());
        double* outs[4] = {rad, theta, phi, pot};
        for (int k = 0; k < 4 && !rc; ++k) {
            if (!outs[k]) continue;
            rc = launch_fft_c2r(P, spec2 + (long long)k * nfield * per, outs[k], SHTC_F64, gf,
                                grs, gcs, nfield, 0, st, gbuf);
        }
        if (!rc) {
            dim3 pg((unsigned)((P->nlon_out + 255) / 256), P->nlat_out, nfield);
            k_grav_post<<<pg, 256, 0, st>>>(rad, theta, phi, total, gf, grs, gcs,
                                            P->nlon_out, rows);
            rc = map_cuda(cudaGetLastError());
        }
    }
    stage_end(SHTC_STAGE_FFT_C2R, st);
    return rc;
}

}  // namespace shtc

// NormalGravity.f95:1 through include/shtools.h:952-956
extern "C" SHTC_API double NormalGravity(const double geocentric_lat, const double gm,
                                         const double omega, const double a, const double b) {
    return shtc::normal_gravity(geocentric_lat, gm, omega, a, b);
}
