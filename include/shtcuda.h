/*
 * shtcuda.h -- C ABI of libshtcuda, the B200 (sm_100a) engine for the real
 * spherical harmonic transforms of SHTOOLS on Driscoll-Healy (DH) and
 * Gauss-Legendre (GLQ) grids.
 *
 * Two layers are exported:
 *
 *  1. The device API (shtc_*): plans, caller-owned device buffers, a CUDA
 *     stream argument, batches of fields, arbitrary element strides, int
 *     status return.  Nothing in a transform call allocates or synchronises;
 *     the caller passes a workspace of shtc_workspace_bytes() bytes.
 *
 *  2. Host-array drop-ins with exactly the names, arguments and Fortran
 *     column-major layouts of the reference C interface include/shtools.h
 *     (lines cited per function).  They copy to the GPU, run the device API
 *     and copy back, so a program linked against libSHTOOLS for these
 *     routines can link against libshtcuda instead.
 *
 * Status codes keep the meanings of the reference's exitstatus
 * (src/MakeGridDH.f95:62-70, src/MakeGridGLQ.f95:196, src/PreGLQ.f95:129-139)
 * and add codes for GPU-side failures.
 */
#ifndef SHTCUDA_H
#define SHTCUDA_H

#include <stddef.h>

#if defined(__GNUC__)
#define SHTC_API __attribute__((visibility("default")))
#else
#define SHTC_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

#define SHTC_OK 0
#define SHTC_EDIM 1      /* improper dimensions of an input array            */
#define SHTC_EBOUND 2    /* improper bounds for an input variable            */
#define SHTC_EALLOC 3    /* error allocating memory                          */
#define SHTC_EIO 4       /* file IO error (unused; kept for the code table)  */
#define SHTC_ENOZERO 5   /* GLQ nodes missing or PreGLQ did not converge     */
#define SHTC_ECUDA 6     /* CUDA runtime or kernel launch error              */
#define SHTC_EHANDLE 7   /* null plan handle or null required pointer        */
#define SHTC_EUNSUP 8    /* FFT length or size beyond the supported range    */
#define SHTC_EWORK 9     /* workspace smaller than shtc_workspace_bytes()    */
#define SHTC_ETIMEOUT 10 /* a bounded wait inside a tensor-core kernel ran out */

/* Legendre arithmetic of a plan (shtc_plan_set_precision) */
#define SHTC_PREC_F64 0     /* FP64 recursion and sums (default; the parity path) */
#define SHTC_PREC_INT8X6 1  /* FP64 recursion, synthesis sums on INT8 tensor cores:
                               6-byte fixed-point operands, 7 byte-product weights */
#define SHTC_PREC_INT8X7 2  /* as INT8X6 with 7-byte operands and 8 weights */

#define SHTC_GRID_DH 1
#define SHTC_GRID_GLQ 2

typedef struct shtc_plan shtc_plan;

/* Precision of the Legendre sums of a plan (no counterpart in the reference,
 * whose transforms are FP64 only).  SHTC_PREC_INT8X6 / INT8X7 run the
 * synthesis of real plans with norm 1, 2 or 4 on the tcgen05 tensor cores:
 * P_lm and the coefficients as 46-bit (54-bit) fixed-point integers split
 * into 6 (7) balanced byte digits, the significant byte products summed
 * exactly in INT32; the recursion stays FP64.  Other transforms of the plan
 * keep FP64.  Returns SHTC_EUNSUP for norm 3 or complex plans.  Allocates a
 * small table and synchronises. */
SHTC_API int shtc_plan_set_precision(shtc_plan* plan, int precision);

/* Table-driven mixed transforms (no counterpart in the reference; the
 * reference's plx table of MakeGridGLQ.f95:441-465 holds FP64 P_lm for the
 * GLQ syntheses).  enable != 0 computes, once, the fixed-point digits of
 * every P_lm of the plan at its current mixed precision (INT8X6 or INT8X7)
 * and keeps them in device memory in a layout that is the tensor cores' A
 * operand of both directions.  The digits are those of the FP64 kernels'
 * recursion rounded to the fixed point.  Later syntheses of that precision
 * stream the table instead of running the recursion, and the analyses and
 * synthesis adjoints run their
 * Legendre sums on the tensor cores from it (ring sums split into the same
 * balanced digits; per-degree errors against FP64 are stated by the tests).
 * Leading 256-degree tiles whose digits are all zero are not stored.  Size:
 * about npair * (lmax+1)^2 / 2 * 7 bytes before that saving (lmax 2799,
 * sampling 2: 77 GB; lmax 2047 GLQ: 15 GB).  enable == 0
 * frees the table; so does switching the plan to the other mixed precision.
 * bytes (may be NULL) receives the table size.  SHTC_EBOUND when the plan's
 * precision is FP64, SHTC_EALLOC when the table does not fit.  Synchronises. */
SHTC_API int shtc_plan_legendre_table(shtc_plan* plan, int enable, unsigned long long* bytes);

/* Error word of the tensor-core kernels on the current device: 0 or
 * SHTC_ETIMEOUT (a bounded in-kernel wait ran out; the outputs of that call
 * are invalid).  Reads and clears it; synchronises the stream. */
SHTC_API int shtc_mixed_status(int* status, void* stream);

/* Self-test of that error path (no counterpart in the reference): one GPU
 * thread waits, through the bounded wait of the tensor-core kernels, on an
 * mbarrier that nothing completes; within about two seconds the wait gives up
 * and records SHTC_ETIMEOUT, which the next shtc_mixed_status returns.  No fault
 * and no trap: the context stays usable.  Synchronises the stream. */
SHTC_API int shtc_mixed_wait_selftest(void* stream);

/* Library version as 10000*major + 100*minor + patch. */
SHTC_API int shtc_version(void);

/* Human-readable text of a status code (static storage). */
SHTC_API const char* shtc_status_string(int status);

/* ------------------------------------------------------------------------ */
/* Plans.  A plan holds the device tables of one grid and option set:       */
/* recursion factors ff1/ff2 (MakeGridDH.f95:321-381), sectoral start       */
/* values, the u^m/1e-280 rescale table, ring geometry, quadrature weights  */
/* and the longitude FFT plan.  Creation allocates device memory and        */
/* synchronises the stream; transforms on a plan do neither.                */
/* lmax_calc < 0 means lmax_calc = lmax.                                    */
/* ------------------------------------------------------------------------ */

/* DH grid of n = 2*lmax+2 rings, sampling*n longitudes (MakeGridDH.f95:109-156). */
SHTC_API int shtc_plan_create_dh(shtc_plan** plan, int lmax, int sampling, int lmax_calc,
                        int norm, int csphase, int extend, void* stream);

/* GLQ grid of lmax+1 rings, 2*lmax+1 longitudes (MakeGridGLQ.f95:108-109).
 * zero/w: host arrays of lmax+1 nodes (descending) and weights, e.g. from
 * SHGLQ; NULL computes them with the GPU PreGLQ. */
SHTC_API int shtc_plan_create_glq(shtc_plan** plan, int lmax, const double* zero,
                         const double* w, int lmax_calc, int norm, int csphase,
                         int extend, void* stream);

/* Plans of the complex transforms (MakeGridDHC.f95:100-160,
 * MakeGridGLQC.f95): same grids and arguments as above; the transforms on
 * them are shtc_synthesis_c / shtc_analysis_c. */
SHTC_API int shtc_plan_create_dhc(shtc_plan** plan, int lmax, int sampling, int lmax_calc,
                                  int norm, int csphase, int extend, void* stream);
SHTC_API int shtc_plan_create_glqc(shtc_plan** plan, int lmax, const double* zero,
                                   const double* w, int lmax_calc, int norm, int csphase,
                                   int extend, void* stream);

SHTC_API int shtc_plan_destroy(shtc_plan* plan);

/* info[0..15] = kind, lmax, lmax_comp, norm, csphase, sampling, extend,
 * nlat, nlon, nlat_out, nlon_out, npair, nlm, device_bytes, bluestein,
 * fft_mode (2 for the plans of the complex transforms) */
SHTC_API int shtc_plan_info(const shtc_plan* plan, long long* info, int ninfo);

/* Tile shapes of the Legendre kernels (no counterpart in the reference):
 * ring pairs per thread of the single-field synthesis, and ring pairs per
 * thread and warps per CTA of the analysis; each 1, 2, 4 or 8, or 0 for the
 * built-in heuristic.  Used by the autotuner; query shtc_workspace_bytes
 * after changing them. */
SHTC_API int shtc_plan_set_tuning(shtc_plan* plan, int synth_T, int anal_T,
                                  int anal_W);

/* Device workspace bytes needed by any transform of nfield fields. */
SHTC_API size_t shtc_workspace_bytes(const shtc_plan* plan, int nfield);

/* ------------------------------------------------------------------------ */
/* Transforms on device buffers.  Strides are in elements.                 */
/*   cilm: element (f, k, l, m) at cilm[f*csf + k*csk + l*csl + m*csm],     */
/*         k = 0 cosine (Clm), k = 1 sine (Slm), 0 <= l, m < cilm_dim.       */
/*   grid: element (f, i, j) at grid[f*gsf + i*gsr + j*gsc].                */
/* ------------------------------------------------------------------------ */

/* MakeGridDH / MakeGridGLQ: cilm -> grid of nlat_out x nlon_out. */
SHTC_API int shtc_synthesis(const shtc_plan* plan, const double* cilm, long long csf,
                   long long csk, long long csl, long long csm, int cilm_dim,
                   double* grid, long long gsf, long long gsr, long long gsc,
                   int nfield, void* work, size_t work_bytes, void* stream);

/* SHExpandDH / SHExpandGLQ: grid of nlat x nlon -> cilm (cilm_dim >=
 * lmax_comp+1; entries beyond lmax_comp and with m > l are set to zero). */
SHTC_API int shtc_analysis(const shtc_plan* plan, const double* grid, long long gsf,
                  long long gsr, long long gsc, double* cilm, long long csf,
                  long long csk, long long csl, long long csm, int cilm_dim,
                  int nfield, void* work, size_t work_bytes, void* stream);

/* Adjoint of shtc_synthesis: grid cotangent (nlat_out x nlon_out) ->
 * coefficient cotangent.  The Legendre functions are recomputed, not
 * stored. */
SHTC_API int shtc_synthesis_adjoint(const shtc_plan* plan, const double* grid,
                           long long gsf, long long gsr, long long gsc,
                           double* cilm, long long csf, long long csk,
                           long long csl, long long csm, int cilm_dim,
                           int nfield, void* work, size_t work_bytes,
                           void* stream);

/* Adjoint of shtc_analysis: coefficient cotangent -> grid cotangent
 * (nlat x nlon): the quadrature-weighted transpose of the analysis. */
SHTC_API int shtc_analysis_adjoint(const shtc_plan* plan, const double* cilm,
                          long long csf, long long csk, long long csl,
                          long long csm, int cilm_dim, double* grid,
                          long long gsf, long long gsr, long long gsc,
                          int nfield, void* work, size_t work_bytes,
                          void* stream);

/* ------------------------------------------------------------------------ */
/* Batches of fields on several grids (no single counterpart in the         */
/* reference, which transforms one field per call): e.g. thousands of GLQ   */
/* fields of uneven lmax.  A batch references existing plans (one per grid  */
/* and option set, extend = 0), which must outlive it; the nf fields of a   */
/* plan share its Legendre recursion.  A batched transform is one pack      */
/* launch, one persistent Legendre launch over cost-sorted work items and   */
/* one launch for all longitude FFTs (plus an unpack for the analysis), so  */
/* it can be captured in a CUDA graph.  Caller arrays hold the groups one   */
/* after another: per group (nf, 2, lc+1, lc+1) coefficients and            */
/* (nf, nlat, nlon) grids, C order, at the offsets of shtc_batch_layout.    */
/* ------------------------------------------------------------------------ */
typedef struct shtc_batch shtc_batch;
SHTC_API int shtc_batch_create(shtc_batch** batch, int nplans,
                               shtc_plan* const* plans, const int* nfields,
                               void* stream);
SHTC_API int shtc_batch_destroy(shtc_batch* batch);
/* cilm_off / grid_off: nplans+1 element offsets (the last is the total). */
SHTC_API int shtc_batch_layout(const shtc_batch* batch, long long* cilm_off,
                               long long* grid_off);
SHTC_API size_t shtc_batch_workspace_bytes(const shtc_batch* batch);
SHTC_API int shtc_batch_synthesis(const shtc_batch* batch, const double* cilm,
                                  double* grid, void* work, size_t work_bytes,
                                  void* stream);
SHTC_API int shtc_batch_analysis(const shtc_batch* batch, const double* grid,
                                 double* cilm, void* work, size_t work_bytes,
                                 void* stream);

/* The same four transforms with the element type of each array given by a
 * dtype code, SHTC_F64 or SHTC_F32 (no counterpart in the reference, which is
 * float64 only).  Arithmetic stays in FP64 inside the kernels; float32
 * arrays are converted on load and store (e.g. float32 grids with float64
 * coefficients, or both float32). */
#define SHTC_F64 0
#define SHTC_F32 1
SHTC_API int shtc_synthesis_ex(const shtc_plan* plan, const void* cilm, int cilm_dtype,
                               long long csf, long long csk, long long csl,
                               long long csm, int cilm_dim, void* grid, int grid_dtype,
                               long long gsf, long long gsr, long long gsc, int nfield,
                               void* work, size_t work_bytes, void* stream);
SHTC_API int shtc_analysis_ex(const shtc_plan* plan, const void* grid, int grid_dtype,
                              long long gsf, long long gsr, long long gsc, void* cilm,
                              int cilm_dtype, long long csf, long long csk,
                              long long csl, long long csm, int cilm_dim, int nfield,
                              void* work, size_t work_bytes, void* stream);
SHTC_API int shtc_synthesis_adjoint_ex(const shtc_plan* plan, const void* grid,
                                       int grid_dtype, long long gsf, long long gsr,
                                       long long gsc, void* cilm, int cilm_dtype,
                                       long long csf, long long csk, long long csl,
                                       long long csm, int cilm_dim, int nfield,
                                       void* work, size_t work_bytes, void* stream);
SHTC_API int shtc_analysis_adjoint_ex(const shtc_plan* plan, const void* cilm,
                                      int cilm_dtype, long long csf, long long csk,
                                      long long csl, long long csm, int cilm_dim,
                                      void* grid, int grid_dtype, long long gsf,
                                      long long gsr, long long gsc, int nfield,
                                      void* work, size_t work_bytes, void* stream);

/* Quadrature on the GPU (device output arrays).
 * PreGLQ.f95:1-151: n nodes (descending) and weights on [x1, x2];
 * returns SHTC_ENOZERO if Newton's iteration does not converge.  Synchronises
 * the stream. */
SHTC_API int shtc_preglq(double x1, double x2, int n, double* zero, double* w,
                void* stream);
/* DHaj.f95:1-107: the n (+extend) Driscoll-Healy weights. */
SHTC_API int shtc_dhaj(int n, double* aj, int extend, void* stream);

/* Synthesis without allocation.  No counterpart in the reference: it is
 * shtc_synthesis with the workspace taken from a fixed array inside the
 * library, for callers that must not allocate device memory inside their own
 * calls (memory owned by a pool or budget manager, or loops that cannot
 * afford cudaMalloc's implicit synchronisation).  The array holds
 * SHTC_NOALLOC_SCRATCH_BYTES on every GPU that loads the library, until
 * exit.  Transforms needing more (shtc_workspace_bytes(plan, nfield) above
 * that size, e.g. one DH field beyond lmax ~600; that size includes the
 * plan's analysis tiles, set by its tile shape, and its precision's
 * scratch) return SHTC_EWORK without launching; a plan of another device
 * than the current one returns SHTC_EHANDLE.  The first call on a device looks up the array's device
 * address (cudaGetSymbolAddress) and caches it: make it before any stream
 * capture.  All calls share the array; calls that overlap on the GPU race. */
#define SHTC_NOALLOC_SCRATCH_BYTES (16u << 20)
SHTC_API int shtc_synthesis_noalloc(const shtc_plan* plan, const double* cilm,
                                    long long csf, long long csk, long long csl,
                                    long long csm, int cilm_dim, double* grid,
                                    long long gsf, long long gsr, long long gsc,
                                    int nfield, void* stream);

/* ------------------------------------------------------------------------ */
/* Stage timing (no counterpart in the reference, which times whole calls  */
/* with cpu_time, examples/fortran/TimingAccuracy/TimingAccuracyDH.f95:96). */
/* When enabled, each kernel stage of a transform is bracketed by CUDA      */
/* events on its stream; collect() waits for them and returns the summed    */
/* milliseconds and launch counts per stage id.                             */
/* ------------------------------------------------------------------------ */
#define SHTC_STAGE_PACK 0
#define SHTC_STAGE_LEGENDRE_SYNTH 1
#define SHTC_STAGE_FFT_C2R 2
#define SHTC_STAGE_FFT_R2C 3
#define SHTC_STAGE_LEGENDRE_ANAL 4
#define SHTC_STAGE_UNPACK 5
#define SHTC_NUM_STAGES 6

SHTC_API int shtc_timing_enable(int on);
SHTC_API int shtc_timing_collect(double* ms, int* counts, int nstages);

/* ------------------------------------------------------------------------ */
/* Complex transforms on device buffers (plans from shtc_plan_create_dhc /  */
/* _glqc).  cilm and grid hold interleaved complex doubles (the layout of   */
/* double _Complex); strides are in complex elements.                       */
/*   cilm: (f, k, l, m), k = 0 the order +m, k = 1 the order -m             */
/*         (Y*_lm = (-1)^m Y_l,-m; cilm[k=1][l][0] is ignored / returned 0).*/
/* The workspace is shtc_workspace_bytes(plan, nfield) of the complex plan. */
/* ------------------------------------------------------------------------ */

/* MakeGridDHC / MakeGridGLQC (src/MakeGridDHC.f95:1, src/MakeGridGLQC.f95:1) */
SHTC_API int shtc_synthesis_c(const shtc_plan* plan, const void* cilm, long long csf,
                              long long csk, long long csl, long long csm, int cilm_dim,
                              void* grid, long long gsf, long long gsr, long long gsc,
                              int nfield, void* work, size_t work_bytes, void* stream);

/* SHExpandDHC / SHExpandGLQC (src/SHExpandDHC.f95:1, src/SHExpandGLQC.f95:1) */
SHTC_API int shtc_analysis_c(const shtc_plan* plan, const void* grid, long long gsf,
                             long long gsr, long long gsc, void* cilm, long long csf,
                             long long csk, long long csl, long long csm, int cilm_dim,
                             int nfield, void* work, size_t work_bytes, void* stream);

/* MakeGradientDH (src/MakeGradientDH.f95:1) on device buffers: the theta and
 * phi components of the horizontal gradient, (1/r) dF/dtheta and
 * 1/(r sin theta) dF/dphi, on the grids of a real DH plan created with
 * norm 1 and csphase 1 (the reference's only normalisation); zero on the
 * pole rows.  Strides as above; theta and phi share the grid strides.  The
 * workspace is shtc_gradient_workspace_bytes(plan, nfield). */
SHTC_API size_t shtc_gradient_workspace_bytes(const shtc_plan* plan, int nfield);
SHTC_API int shtc_gradient_dh(const shtc_plan* plan, const double* cilm, long long csf,
                              long long csk, long long csl, long long csm, int cilm_dim,
                              double* theta, double* phi, long long gsf, long long gsr,
                              long long gsc, double radius, int nfield, void* work,
                              size_t work_bytes, void* stream);

/* MakeGravGridDH (src/MakeGravGridDH.f95:1) on device buffers: the gravity
 * vector of the potential V = GM/r sum_l (r0/r)^l C_lm Y_lm on a flattened
 * ellipsoid (semi-major axis a, flattening f): rad (positive up), theta,
 * phi, the magnitude total and, when pot is not NULL, the potential.
 * has_omega = 0 is the reference's absent OMEGA (no centrifugal terms);
 * normal_gravity = 1 removes the normal gravity of GM normal_gravity_gm
 * from total (needs has_omega).  A real DH plan with norm 1 and csphase 1;
 * the five grids share the strides; workspace
 * shtc_gravity_workspace_bytes(plan, nfield). */
SHTC_API size_t shtc_gravity_workspace_bytes(const shtc_plan* plan, int nfield);
SHTC_API int shtc_gravity_dh(const shtc_plan* plan, const double* cilm, long long csf,
                             long long csk, long long csl, long long csm, int cilm_dim,
                             double gm, double r0, double a, double f, int has_omega,
                             double omega, int normal_gravity, double normal_gravity_gm,
                             double* rad, double* theta, double* phi, double* total,
                             double* pot, long long gsf, long long gsr, long long gsc,
                             int nfield, void* work, size_t work_bytes, void* stream);

/* SHMultiply (src/SHMultiply.f95:1) on device buffers: the product of fields
 * of degrees lmax1 and lmax2, expanded to lmax1 + lmax2, through the GLQ grid
 * of a plan created with shtc_plan_create_glq for lmax = lmax1 + lmax2
 * (extend 0, lmax_calc = lmax).  cilm1/cilm2 are read up to their own
 * degree; cilmout has cilm_dim_out >= lmax1 + lmax2 + 1.  Workspace:
 * shtc_multiply_workspace_bytes(plan, nfield). */
SHTC_API size_t shtc_multiply_workspace_bytes(const shtc_plan* plan, int nfield);
SHTC_API int shtc_multiply(const shtc_plan* plan, const double* cilm1, long long c1sf,
                           long long c1sk, long long c1sl, long long c1sm, int lmax1,
                           const double* cilm2, long long c2sf, long long c2sk,
                           long long c2sl, long long c2sm, int lmax2, double* cilmout,
                           long long csf, long long csk, long long csl, long long csm,
                           int cilm_dim_out, int nfield, void* work, size_t work_bytes,
                           void* stream);

/* ------------------------------------------------------------------------ */
/* Drop-ins of the reference C interface, include/shtools.h.  Host arrays,  */
/* Fortran column-major: cilm(2, cilm_dim, cilm_dim), grid(d0, d1).  NULL  */
/* optional arguments take the reference defaults.  The plx arguments of   */
/* the GLQ routines (precomputed Legendre tables) are accepted only as     */
/* NULL; a non-NULL plx returns exitstatus 2.                              */
/* ------------------------------------------------------------------------ */

/* include/shtools.h:104-116 (src/MakeGridDH.f95:1) */
SHTC_API void MakeGridDH(double* griddh, const int griddh_d0, const int griddh_d1,
                int* n, const double* cilm, const int cilm_dim, const int lmax,
                const int* norm, const int* sampling, const int* csphase,
                const int* lmax_calc, const int* extend, int* exitstatus);

/* include/shtools.h:92-103 (src/SHExpandDH.f95:1) */
SHTC_API void SHExpandDH(const double* grid, const int grid_d0, const int grid_d1,
                const int n, double* cilm, const int cilm_dim, int* lmax,
                const int* norm, const int* sampling, const int* csphase,
                const int* lmax_calc, int* exitstatus);

/* Complex drop-ins: complex arrays are passed as shtc_complex, which has
 * the layout of C's double _Complex (interleaved re, im). */
#ifdef __cplusplus
typedef struct shtc_complex_s { double re, im; } shtc_complex;
#else
typedef double _Complex shtc_complex;
#endif

/* include/shtools.h:117-128 (src/SHExpandDHC.f95:1) */
SHTC_API void SHExpandDHC(const shtc_complex* grid, const int grid_d0, const int grid_d1,
                          const int n, shtc_complex* cilm, const int cilm_dim, int* lmax,
                          const int* norm, const int* sampling, const int* csphase,
                          const int* lmax_calc, int* exitstatus);

/* include/shtools.h:129-141 (src/MakeGridDHC.f95:1) */
SHTC_API void MakeGridDHC(shtc_complex* griddh, const int griddh_d0, const int griddh_d1,
                          int* n, const shtc_complex* cilm, const int cilm_dim,
                          const int lmax, const int* norm, const int* sampling,
                          const int* csphase, const int* lmax_calc, const int* extend,
                          int* exitstatus);

/* include/shtools.h:174-184 (src/SHExpandGLQC.f95:1) */
SHTC_API void SHExpandGLQC(shtc_complex* cilm, const int cilm_dim, const int lmax,
                           const shtc_complex* gridglq, const double* w, const double* plx,
                           const double* zero, const int* norm, const int* csphase,
                           const int* lmax_calc, int* exitstatus);

/* include/shtools.h:185-197 (src/MakeGridGLQC.f95:1) */
SHTC_API void MakeGridGLQC(shtc_complex* gridglq, const int gridglq_d0,
                           const int gridglq_d1, const shtc_complex* cilm,
                           const int cilm_dim, const int lmax, const double* plx,
                           const double* zero, const int* norm, const int* csphase,
                           const int* lmax_calc, const int* extend, int* exitstatus);

/* src/cWrapper.f95:295-317, bind(c, name="MakeGradientDH") (src/MakeGradientDH.f95:1);
 * theta and phi are (d0, d1) column-major */
SHTC_API void MakeGradientDH(const double* cilm, const int cilm_dim, const int lmax,
                             double* theta, double* phi, const int theta_d0,
                             const int theta_d1, int* n, const int* sampling,
                             const int* lmax_calc, const int* extend, const double* radius,
                             int* exitstatus);

/* include/shtools.h:726-746, src/cWrapper.f95:1484-1514 (src/MakeGravGridDH.f95:1);
 * rad, theta, phi, total and pot (NULL: not computed) are (nlat, nlon)
 * column-major; the normal gravity uses gm.  exitstatus 5: normal_gravity
 * 1 without omega, as the reference. */
SHTC_API void MakeGravGridDH(const double* cilm, const int cilm_dim, const int lmax,
                             const double gm, const double r0, const double a,
                             const double f, double* rad, const int nlon, const int nlat,
                             double* theta, double* phi, double* total, int* n,
                             const int* sampling, const int* lmax_calc, const double* omega,
                             const int* normal_gravity, double* pot, const int* extend,
                             int* exitstatus);

/* include/shtools.h:952-956 (src/NormalGravity.f95:1); host arithmetic */
SHTC_API double NormalGravity(const double geocentric_lat, const double gm,
                              const double omega, const double a, const double b);

/* include/shtools.h:254-265 (src/SHMultiply.f95:1); precomp is ignored */
SHTC_API void SHMultiply(double* cilmout, const int cilmout_dim, const double* cilm1,
                         const int cilm1_dim, const int lmax1, const double* cilm2,
                         const int cilm2_dim, const int lmax2, const int* precomp,
                         const int* norm, const int* csphase, int* exitstatus);

/* include/shtools.h:153-165 (src/MakeGridGLQ.f95:1) */
SHTC_API void MakeGridGLQ(double* gridglq, const int gridglq_d0, const int gridglq_d1,
                 const double* cilm, const int cilm_dim, const int lmax,
                 const double* plx, const double* zero, const int* norm,
                 const int* csphase, const int* lmax_calc, const int* extend,
                 int* exitstatus);

/* include/shtools.h:142-152 (src/SHExpandGLQ.f95:1); gridglq is
 * (lmax+1, 2*lmax+1) column-major as in src/cWrapper.f95:340 */
SHTC_API void SHExpandGLQ(double* cilm, const int cilm_dim, const int lmax,
                 const double* gridglq, const double* w, const double* plx,
                 const double* zero, const int* norm, const int* csphase,
                 const int* lmax_calc, int* exitstatus);

/* include/shtools.h:134-141 (src/SHGLQ.f95:1); plx must be NULL */
SHTC_API void SHGLQ(const int lmax, double* zero, double* w, double* plx,
           const int* norm, const int* csphase, const int* cnorm,
           int* exitstatus);

/* include/shtools.h:1025-1030 (src/PreGLQ.f95:1) */
SHTC_API void PreGLQ(const double x1, const double x2, const int n, double* zero,
            double* w, int* exitstatus);

/* include/shtools.h:198-206 (src/GLQGridCoord.f95:1, src/cWrapper.f95:419-434):
 * latitudes (degrees, north first) of the lmax+1 Gauss-Legendre nodes and
 * the 2 lmax + 1 (+extend) longitudes of a GLQ grid */
SHTC_API void GLQGridCoord(double* latglq, const int latglq_d0, double* longlq,
                           const int longlq_d0, const int lmax, int* nlat, int* nlong,
                           const int* extend, int* exitstatus);
/* include/shtools.h:1034-1038 (src/DHaj.f95:1) */
SHTC_API void DHaj(const int n, double* aj, const int aj_d0, const int* extend,
          int* exitstatus);

#ifdef __cplusplus
}
#endif

#endif /* SHTCUDA_H */
