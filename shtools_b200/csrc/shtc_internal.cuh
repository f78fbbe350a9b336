// Internal declarations shared by the libshtcuda translation units.
//
// Terminology (follows the reference Fortran, src/MakeGridDH.f95 and
// src/MakeGridGLQ.f95):
//   L      bandwidth (lmax) that fixes the grid
//   lc     lmax_comp = min(L, lmax_calc, cilm_dim-1): highest degree computed
//   ring   one latitude row of the grid
//   pair   a northern ring and its mirror ring (z -> -z) that share one
//          Legendre recursion through P_lm(-z) = (-1)^(l+m) P_lm(z)
//   spec   per (pair, m) Fourier coefficients of the two rings; the hand-off
//          buffer between the Legendre kernels and the longitude FFTs
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stddef.h>

#include "../../include/shtcuda.h"

namespace shtc {

// The Holmes-Featherstone scale factor of the reference (MakeGridDH.f95:228).
constexpr double kScalef = 1.0e-280;
// degrees per segment of the rescaled Legendre recursion (legendre.cuh)
constexpr int kRecSegment = 16;

// Maximum FFT radix handled by the in-shared-memory Stockham passes; other
// prime factors go through Bluestein's algorithm.
constexpr int kMaxRadix = 13;
constexpr int kMaxFactors = 40;

struct FftPlan {
    int n;             // real transform length (grid columns, nlong)
    int mode;          // 0: two rings in one complex length-n FFT (odd n)
                       // 1: one ring via a complex FFT of length n/2 (even n)
                       // 2: complex grids, one ring per complex length-n FFT
    int m;             // complex FFT length executed in shared memory
    int nfac;          // radices of the length-m (or Bluestein) FFT
    int fac[kMaxFactors];
    int bluestein;     // 1 if m has a prime factor > kMaxRadix
    int mb;            // Bluestein convolution length (7-smooth, >= 2m - 1)
    double2* d_tw;     // per-pass base twiddles: pass i (radix R after sub-transforms
                       // of length ns) at tw_off[i], entry k < ns = exp(-2 pi i k/(ns R)),
                       // of the length-(mb or m) FFT
    int tw_off[kMaxFactors];
    int ntw;           // entries of d_tw (sum of ns over the passes)
    double2* d_twn;    // mode 1: exp(-2 pi i k / n), k < n/2
    double2* d_chirp;  // Bluestein: exp(-i pi t^2 / m), t < m
    double2* d_kern;   // Bluestein: FFT_mb of the conjugate chirp kernel
    size_t smem_data;  // shared bytes of the two data buffers
    size_t smem;       // dynamic shared memory bytes per CTA of the per-plan kernels:
                       // smem_data, plus the twiddles when tw_smem
    int tw_smem;       // per-plan kernels copy d_tw into shared memory
    int gmem;          // 1: the two data buffers exceed shared memory and live in
                       // a global scratch of gmem_ctas x 2 x len points (caller's
                       // workspace); the passes then run through L2
    int gmem_ctas;     // persistent CTAs of the global-buffer kernels
    int threads;       // CTA size
};

}  // namespace shtc

// The opaque plan handle of the C ABI.
struct shtc_plan {
    int kind;          // SHTC_GRID_DH or SHTC_GRID_GLQ
    int lmax;          // L
    int lc;            // lmax_comp
    int norm;          // 1..4
    int csphase;       // +1 / -1
    int sampling;      // DH: 1 or 2; GLQ: 1
    int extend;        // synthesis output has the extra column (and DH row)
    int cplx;          // complex transforms (MakeGridDHC & co.): 2 internal fields
                       // (orders +m and -m) per user field, c2c FFTs
    int nlat;          // rings of the grid without the extend row
    int nlon;          // longitudes without the extend column (FFT length)
    int nlat_out;      // synthesis output rows (with extend)
    int nlon_out;      // synthesis output columns (with extend)
    int npair;         // ring pairs
    long long nlm;     // packed (l, m) count, (lc+1)(lc+2)/2
    // device tables (owned)
    double2* d_rec;    // {beta, D} of the rescaled recursion per packed (l, m)
    double* d_pmm;     // sectoral start value per m
    double* d_rtab;    // rescale factor u^m / scalef per (m, pair)
    double* d_z;       // cos(colatitude) of the northern ring of each pair
    int* d_rowN;       // synthesis rows of a pair (-1: none)
    int* d_rowS;
    int* d_arowN;      // analysis rows of a pair (-1: not used)
    int* d_arowS;
    double* d_wN;      // analysis ring weights (quadrature x 2pi or sqrt(2pi)...)
    double* d_wS;
    double* d_nrm;     // per packed (l, m): analysis normalisation divisor
    shtc::FftPlan fft;
    int tune_synth_T;  // ring pairs per thread of the synthesis (0: heuristic)
    int tune_anal_T;   // ring pairs per thread of the analysis (0: heuristic)
    int tune_anal_W;   // warps per CTA of the analysis (0: heuristic)
    size_t device_bytes;
    int device;        // CUDA device the tables live on
    // Legendre arithmetic (shtc_plan_set_precision): SHTC_PREC_F64, or
    // SHTC_PREC_INT8X6 for the tensor-core synthesis (legendre_i8.cu)
    int precision;
    long long* d_i8_toff;   // INT8X6: K-tiles of 64 degrees before each order (lc + 2)
    double4* d_i8_rec2;     // INT8X6: {gamma, delta, D, 0} per packed (l, m): the
                            // same-parity two-step form of the rescaled recursion
    long long i8_ntot;      // INT8X6: K-tiles of all orders
    long long* d_i8_uoff;   // INT8X6: super-tiles of 256 degrees before each order (lc + 2)
    long long i8_utot;      // INT8X6: super-tiles of all orders
    double i8_ascale;       // INT8X6: 2^a, fixed-point scale of the P_lm operand
    // table-driven tensor-core synthesis (shtc_plan_legendre_table)
    uint8_t* d_i8_tab;          // P_lm digit table (legendre_i8_table.cuh)
    long long* d_i8_tab_off;    // per (m, pair tile): super-tiles stored before it
    int* d_i8_tab_u0;           // per (m, pair tile): first stored super-tile
    unsigned long long i8_tab_bytes;
    int i8_tab_prec;            // precision the table holds digits of (0: none)
};

namespace shtc {

// Packed (l, m) layout: for m = 0..lc, l = m..lc; offset of (m, m).
__host__ __device__ inline long long packed_off(int m, int lc) {
    return (long long)m * (2LL * lc + 3 - m) / 2;
}

// plan.cu
int build_fft_plan(FftPlan* f, int n, int cplx, cudaStream_t stream);
void free_fft_plan(FftPlan* f);

// kernels.cu launchers (return cudaGetLastError() mapped to SHTC codes)
int launch_pack_coef(const shtc_plan* P, const void* cilm, int dtype, long long sf,
                     long long sk, long long sl, long long sm, int cdim,
                     double2* packed, int nfield, int scale_mode,
                     cudaStream_t st, int nfield_total = 0, int f_off = 0);
int launch_fft_r2c_product(const shtc_plan* P, const double* grid, const double* grid2,
                           long long gf, long long grs, long long gcs, double2* spec,
                           int nfield, cudaStream_t st, double2* gbuf = nullptr);
int launch_legendre_synth(const shtc_plan* P, const double2* packed,
                          double2* spec, int nfield, cudaStream_t st);
// gbuf: the FFT scratch of the workspace (fft_scratch_bytes), needed when
// P->fft.gmem
int launch_fft_c2r(const shtc_plan* P, const double2* spec, void* grid, int dtype,
                   long long gf, long long grs, long long gcs, int nfield,
                   int weighted, cudaStream_t st, double2* gbuf = nullptr);
int launch_fft_r2c(const shtc_plan* P, const void* grid, int dtype, long long gf,
                   long long grs, long long gcs, double2* spec, int nfield,
                   int weighted, int fold_extend, cudaStream_t st,
                   double2* gbuf = nullptr);
size_t fft_scratch_bytes(const shtc_plan* P);
int launch_legendre_anal(const shtc_plan* P, const double2* spec,
                         double2* partial, int ntiles_out, int nfield,
                         cudaStream_t st);
int launch_unpack_coef(const shtc_plan* P, const double2* partial, int ntiles,
                       void* cilm, int dtype, long long sf, long long sk, long long sl,
                       long long sm, int cdim, int nfield, int normalise,
                       cudaStream_t st);
int anal_tiles(const shtc_plan* P, int nfield);
// kernels.cu: raise the dynamic shared memory limit of kernel fn to smem
// (with max_shared, prefer the largest carveout); set once per device and
// kernel, later calls return at once
int kernel_smem_attr(const void* fn, size_t smem, bool max_shared);
// legendre_mma.cu: the analysis of 8 or more fields on the FP64 tensor path,
// tiles of anal_mma_pairs() ring pairs, output as launch_legendre_anal
int anal_mma_pairs();
int launch_legendre_anal_mma(const shtc_plan* P, const double2* spec, double2* partial,
                             int ntiles, int nfield, cudaStream_t st);
// complex plans: cilm (nfield, 2, cdim, cdim) and grids of interleaved complex
// doubles, strides in complex elements; internal fields 2u (+m), 2u+1 (-m)
int launch_pack_coef_c(const shtc_plan* P, const double2* cilm, long long sf, long long sk,
                       long long sl, long long sm, int cdim, double2* packed, int nfield,
                       cudaStream_t st);
int launch_unpack_coef_c(const shtc_plan* P, const double2* partial, int ntiles,
                         double2* cilm, long long sf, long long sk, long long sl,
                         long long sm, int cdim, int nfield, cudaStream_t st);
int launch_fft_c2c_synth(const shtc_plan* P, const double2* spec, double2* grid,
                         long long gf, long long grs, long long gcs, int nfield,
                         cudaStream_t st, double2* gbuf = nullptr);
// MakeGradientDH: workspace = packed (3 nfield) | spec (3 nfield) | spec2 (2 nfield)
int launch_gradient_dh(const shtc_plan* P, const double* cilm, long long sf, long long sk,
                       long long sl, long long sm, int cdim, double* theta, double* phi,
                       long long gf, long long grs, long long gcs, double radius,
                       int nfield, double2* packed, double2* spec, double2* spec2,
                       cudaStream_t st, double2* gbuf = nullptr);
// MakeGravGridDH (grav.cu): the three sums of a field packed as for the
// gradient (c, c_(l+1) a_(l+1), l c); workspace = packed (3 nfield) | spec
// (3 nfield) | spec2 (4 nfield) | tables (grav_table_bytes)
int launch_pack_grad(const shtc_plan* P, const double* cilm, long long sf, long long sk,
                     long long sl, long long sm, int cdim, double2* packed, int nfield,
                     cudaStream_t st);
struct GravParams {
    double gm, r0, a, f, omega, ng_gm;
    int has_omega;        // the reference's OMEGA present (rotation terms)
    int normal_gravity;   // 1: total minus the normal gravity
};
size_t grav_table_bytes(const shtc_plan* P);
int launch_gravity_dh(const shtc_plan* P, const double* cilm, long long sf, long long sk,
                      long long sl, long long sm, int cdim, const GravParams& g,
                      double* rad, double* theta, double* phi, double* total, double* pot,
                      long long gf, long long grs, long long gcs, int nfield,
                      double2* packed, double2* spec, double2* spec2, double* tab,
                      cudaStream_t st, double2* gbuf);
__host__ __device__ double normal_gravity(double geocentric_lat, double gm, double omega,
                                          double a, double b);
int launch_fft_c2c_anal(const shtc_plan* P, const double2* grid, long long gf,
                        long long grs, long long gcs, double2* spec, int nfield,
                        cudaStream_t st, double2* gbuf = nullptr);
int map_cuda(cudaError_t e);
// legendre_i8.cu: INT8 error-free split synthesis (SHTC_PREC_INT8X6 plans)
size_t synth_i8_bytes(const shtc_plan* P, int nfield);
int launch_legendre_synth_i8(const shtc_plan* P, const double2* coef, double2* spec,
                             int nfield, void* scratch, cudaStream_t st);
int set_precision_tables(shtc_plan* P, int precision);
// the analysis of a mixed plan runs on the tensor cores once the plan holds
// its P_lm digit table (real plans)
bool anal_i8_ready(const shtc_plan* P);
int launch_legendre_anal_i8(const shtc_plan* P, const double2* spec, double2* partial,
                            int nfield, void* scratch, cudaStream_t st);
void free_i8_table(shtc_plan* P);

// timing.cu: event brackets around kernel stages (SHTC_STAGE_* ids)
void stage_begin(int stage, cudaStream_t st);
void stage_end(int stage, cudaStream_t st);

}  // namespace shtc
