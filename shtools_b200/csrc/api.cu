// C ABI of libshtcuda: device transforms, their adjoints, and the host-array
// drop-ins of the reference C interface (include/shtools.h).
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "shtc_internal.cuh"

using namespace shtc;

extern "C" int shtc_version(void) { return 100; }

extern "C" const char* shtc_status_string(int s) {
    switch (s) {
        case SHTC_OK: return "No errors.";
        case SHTC_EDIM: return "Improper dimensions of input array.";
        case SHTC_EBOUND: return "Improper bounds for input variable.";
        case SHTC_EALLOC: return "Error allocating memory.";
        case SHTC_EIO: return "File IO error.";
        case SHTC_ENOZERO: return "Gauss-Legendre nodes missing or not converged.";
        case SHTC_ECUDA: return "CUDA runtime or kernel launch error.";
        case SHTC_EHANDLE: return "Null plan handle or required pointer.";
        case SHTC_EUNSUP: return "Transform size not supported.";
        case SHTC_EWORK: return "Workspace too small.";
        case SHTC_ETIMEOUT: return "A bounded wait inside a tensor-core kernel ran out.";
        default: return "Unknown status.";
    }
}

// workspace layout: [coef region | spec region], each 256-byte aligned
static size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

static size_t coef_region(const shtc_plan* P, int nfield) {
    const int tiles = anal_tiles(P, nfield);
    return align256((size_t)P->nlm * nfield * sizeof(double2) * (tiles > 1 ? tiles : 1));
}

static size_t spec_region(const shtc_plan* P, int nfield) {
    return align256((size_t)nfield * P->npair * (P->lc + 1) * 2 * sizeof(double2));
}

// longitude FFTs too long for shared memory use a scratch behind the other
// regions (fft_scratch_bytes, zero otherwise)
static size_t fft_region(const shtc_plan* P) { return align256(fft_scratch_bytes(P)); }

static double2* fft_scratch(const shtc_plan* P, void* work, size_t offset) {
    return P->fft.gmem ? (double2*)((char*)work + offset) : nullptr;
}

// complex plans carry two internal fields (orders +m and -m) per field
// INT8X6 plans: the tensor-core synthesis scratch behind the FFT region
static size_t i8_region(const shtc_plan* P, int nfield) {
    return P->precision != SHTC_PREC_F64 && !P->cplx ? align256(synth_i8_bytes(P, nfield)) : 0;
}

// Legendre analysis stage of a real plan: the tensor-core analysis when the
// plan is mixed-precision and holds its P_lm digit table (its sums arrive as
// one partial tile), else the FP64 kernels (anal_tiles partial tiles)
static int legendre_anal_stage(const shtc_plan* P, const double2* spec, double2* partial,
                               int nfield, void* work, int* tiles, cudaStream_t st) {
    if (anal_i8_ready(P)) {
        *tiles = 1;
        return launch_legendre_anal_i8(
            P, spec, partial, nfield,
            (char*)work + coef_region(P, nfield) + spec_region(P, nfield) + fft_region(P), st);
    }
    *tiles = anal_tiles(P, nfield);
    return launch_legendre_anal(P, spec, partial, *tiles, nfield, st);
}

extern "C" size_t shtc_workspace_bytes(const shtc_plan* P, int nfield) {
    if (!P || nfield < 1) return 0;
    const int nf = P->cplx ? 2 * nfield : nfield;
    return coef_region(P, nf) + spec_region(P, nf) + fft_region(P) + i8_region(P, nf);
}

static int check_call(const shtc_plan* P, const void* a, const void* b,
                      int nfield, void* work, size_t wb) {
    if (!P || !a || !b) return SHTC_EHANDLE;
    if (nfield < 1) return SHTC_EBOUND;
    if (!work || wb < shtc_workspace_bytes(P, nfield)) return SHTC_EWORK;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != P->device) return SHTC_EHANDLE;
    return SHTC_OK;
}

static int check_dtypes(int a, int b) {
    auto ok = [](int d) { return d == SHTC_F64 || d == SHTC_F32; };
    return ok(a) && ok(b) ? SHTC_OK : SHTC_EBOUND;
}

// real entry points need a real plan, the complex ones a complex plan
static int check_kind(const shtc_plan* P, int cplx) {
    return P && P->cplx != cplx ? SHTC_EBOUND : SHTC_OK;
}

extern "C" int shtc_synthesis_ex(const shtc_plan* P, const void* cilm, int cdt,
                                 long long csf, long long csk, long long csl,
                                 long long csm, int cdim, void* grid, int gdt,
                                 long long gsf, long long gsr, long long gsc,
                                 int nfield, void* work, size_t wb, void* stream) {
    int rc = check_call(P, cilm, grid, nfield, work, wb);
    if (rc) return rc;
    if ((rc = check_kind(P, 0))) return rc;
    if ((rc = check_dtypes(cdt, gdt))) return rc;
    if (cdim < 1) return SHTC_EDIM;
    cudaStream_t st = (cudaStream_t)stream;
    double2* packed = (double2*)work;
    double2* spec = (double2*)((char*)work + coef_region(P, nfield));
    double2* fbuf = fft_scratch(P, work, coef_region(P, nfield) + spec_region(P, nfield));
    const bool i8 = P->precision != SHTC_PREC_F64;
    stage_begin(SHTC_STAGE_PACK, st);
    rc = launch_pack_coef(P, cilm, cdt, csf, csk, csl, csm, cdim, packed, nfield, i8 ? 2 : 0,
                          st);
    stage_end(SHTC_STAGE_PACK, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if (i8)
        rc = launch_legendre_synth_i8(
            P, packed, spec, nfield,
            (char*)work + coef_region(P, nfield) + spec_region(P, nfield) + fft_region(P), st);
    else
        rc = launch_legendre_synth(P, packed, spec, nfield, st);
    stage_end(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_FFT_C2R, st);
    rc = launch_fft_c2r(P, spec, grid, gdt, gsf, gsr, gsc, nfield, 0, st, fbuf);
    stage_end(SHTC_STAGE_FFT_C2R, st);
    return rc;
}

extern "C" int shtc_analysis_ex(const shtc_plan* P, const void* grid, int gdt,
                                long long gsf, long long gsr, long long gsc,
                                void* cilm, int cdt, long long csf, long long csk,
                                long long csl, long long csm, int cdim, int nfield,
                                void* work, size_t wb, void* stream) {
    int rc = check_call(P, grid, cilm, nfield, work, wb);
    if (rc) return rc;
    if ((rc = check_kind(P, 0))) return rc;
    if ((rc = check_dtypes(cdt, gdt))) return rc;
    if (cdim < P->lc + 1) return SHTC_EDIM;
    cudaStream_t st = (cudaStream_t)stream;
    double2* partial = (double2*)work;
    double2* spec = (double2*)((char*)work + coef_region(P, nfield));
    double2* fbuf = fft_scratch(P, work, coef_region(P, nfield) + spec_region(P, nfield));
    int tiles = 0;
    stage_begin(SHTC_STAGE_FFT_R2C, st);
    rc = launch_fft_r2c(P, grid, gdt, gsf, gsr, gsc, spec, nfield, 1, 0, st, fbuf);
    stage_end(SHTC_STAGE_FFT_R2C, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_ANAL, st);
    rc = legendre_anal_stage(P, spec, partial, nfield, work, &tiles, st);
    stage_end(SHTC_STAGE_LEGENDRE_ANAL, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_UNPACK, st);
    rc = launch_unpack_coef(P, partial, tiles, cilm, cdt, csf, csk, csl, csm, cdim, nfield,
                            1, st);
    stage_end(SHTC_STAGE_UNPACK, st);
    return rc;
}

extern "C" int shtc_synthesis_adjoint_ex(const shtc_plan* P, const void* grid, int gdt,
                                         long long gsf, long long gsr, long long gsc,
                                         void* cilm, int cdt, long long csf,
                                         long long csk, long long csl, long long csm,
                                         int cdim, int nfield, void* work, size_t wb,
                                         void* stream) {
    int rc = check_call(P, grid, cilm, nfield, work, wb);
    if (rc) return rc;
    if ((rc = check_kind(P, 0))) return rc;
    if ((rc = check_dtypes(cdt, gdt))) return rc;
    if (cdim < 1) return SHTC_EDIM;
    cudaStream_t st = (cudaStream_t)stream;
    double2* partial = (double2*)work;
    double2* spec = (double2*)((char*)work + coef_region(P, nfield));
    double2* fbuf = fft_scratch(P, work, coef_region(P, nfield) + spec_region(P, nfield));
    int tiles = 0;
    stage_begin(SHTC_STAGE_FFT_R2C, st);
    rc = launch_fft_r2c(P, grid, gdt, gsf, gsr, gsc, spec, nfield, 0, P->extend, st, fbuf);
    stage_end(SHTC_STAGE_FFT_R2C, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_ANAL, st);
    rc = legendre_anal_stage(P, spec, partial, nfield, work, &tiles, st);
    stage_end(SHTC_STAGE_LEGENDRE_ANAL, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_UNPACK, st);
    rc = launch_unpack_coef(P, partial, tiles, cilm, cdt, csf, csk, csl, csm, cdim, nfield,
                            0, st);
    stage_end(SHTC_STAGE_UNPACK, st);
    return rc;
}

extern "C" int shtc_analysis_adjoint_ex(const shtc_plan* P, const void* cilm, int cdt,
                                        long long csf, long long csk, long long csl,
                                        long long csm, int cdim, void* grid, int gdt,
                                        long long gsf, long long gsr, long long gsc,
                                        int nfield, void* work, size_t wb, void* stream) {
    int rc = check_call(P, cilm, grid, nfield, work, wb);
    if (rc) return rc;
    if ((rc = check_kind(P, 0))) return rc;
    if ((rc = check_dtypes(cdt, gdt))) return rc;
    if (cdim < 1) return SHTC_EDIM;
    cudaStream_t st = (cudaStream_t)stream;
    double2* packed = (double2*)work;
    double2* spec = (double2*)((char*)work + coef_region(P, nfield));
    double2* fbuf = fft_scratch(P, work, coef_region(P, nfield) + spec_region(P, nfield));
    const bool i8 = P->precision != SHTC_PREC_F64;
    stage_begin(SHTC_STAGE_PACK, st);
    rc = launch_pack_coef(P, cilm, cdt, csf, csk, csl, csm, cdim, packed, nfield, i8 ? 3 : 1,
                          st);
    stage_end(SHTC_STAGE_PACK, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if (i8)
        rc = launch_legendre_synth_i8(
            P, packed, spec, nfield,
            (char*)work + coef_region(P, nfield) + spec_region(P, nfield) + fft_region(P), st);
    else
        rc = launch_legendre_synth(P, packed, spec, nfield, st);
    stage_end(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_FFT_C2R, st);
    rc = launch_fft_c2r(P, spec, grid, gdt, gsf, gsr, gsc, nfield, 1, st, fbuf);
    stage_end(SHTC_STAGE_FFT_C2R, st);
    return rc;
}

extern "C" int shtc_synthesis(const shtc_plan* P, const double* cilm, long long csf,
                              long long csk, long long csl, long long csm, int cdim,
                              double* grid, long long gsf, long long gsr, long long gsc,
                              int nfield, void* work, size_t wb, void* stream) {
    return shtc_synthesis_ex(P, cilm, SHTC_F64, csf, csk, csl, csm, cdim, grid, SHTC_F64,
                             gsf, gsr, gsc, nfield, work, wb, stream);
}

extern "C" int shtc_analysis(const shtc_plan* P, const double* grid, long long gsf,
                             long long gsr, long long gsc, double* cilm, long long csf,
                             long long csk, long long csl, long long csm, int cdim,
                             int nfield, void* work, size_t wb, void* stream) {
    return shtc_analysis_ex(P, grid, SHTC_F64, gsf, gsr, gsc, cilm, SHTC_F64, csf, csk, csl,
                            csm, cdim, nfield, work, wb, stream);
}

extern "C" int shtc_synthesis_adjoint(const shtc_plan* P, const double* grid,
                                      long long gsf, long long gsr, long long gsc,
                                      double* cilm, long long csf, long long csk,
                                      long long csl, long long csm, int cdim,
                                      int nfield, void* work, size_t wb, void* stream) {
    return shtc_synthesis_adjoint_ex(P, grid, SHTC_F64, gsf, gsr, gsc, cilm, SHTC_F64, csf,
                                     csk, csl, csm, cdim, nfield, work, wb, stream);
}

extern "C" int shtc_analysis_adjoint(const shtc_plan* P, const double* cilm,
                                     long long csf, long long csk, long long csl,
                                     long long csm, int cdim, double* grid, long long gsf,
                                     long long gsr, long long gsc, int nfield, void* work,
                                     size_t wb, void* stream) {
    return shtc_analysis_adjoint_ex(P, cilm, SHTC_F64, csf, csk, csl, csm, cdim, grid,
                                    SHTC_F64, gsf, gsr, gsc, nfield, work, wb, stream);
}

// ---------------------------------------------------------------------------
// complex transforms: the Legendre stages run on 2 internal fields per field
// (orders +m and -m, sharing one recursion), the longitude transforms are
// complex DFTs
// ---------------------------------------------------------------------------
extern "C" int shtc_synthesis_c(const shtc_plan* P, const void* cilm, long long csf,
                                long long csk, long long csl, long long csm, int cdim,
                                void* grid, long long gsf, long long gsr, long long gsc,
                                int nfield, void* work, size_t wb, void* stream) {
    int rc = check_call(P, cilm, grid, nfield, work, wb);
    if (rc) return rc;
    if ((rc = check_kind(P, 1))) return rc;
    if (cdim < 1) return SHTC_EDIM;
    cudaStream_t st = (cudaStream_t)stream;
    const int nf2 = 2 * nfield;
    double2* packed = (double2*)work;
    double2* spec = (double2*)((char*)work + coef_region(P, nf2));
    double2* fbuf = fft_scratch(P, work, coef_region(P, nf2) + spec_region(P, nf2));
    stage_begin(SHTC_STAGE_PACK, st);
    rc = launch_pack_coef_c(P, (const double2*)cilm, csf, csk, csl, csm, cdim, packed, nfield,
                            st);
    stage_end(SHTC_STAGE_PACK, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_SYNTH, st);
    rc = launch_legendre_synth(P, packed, spec, nf2, st);
    stage_end(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_FFT_C2R, st);
    rc = launch_fft_c2c_synth(P, spec, (double2*)grid, gsf, gsr, gsc, nfield, st, fbuf);
    stage_end(SHTC_STAGE_FFT_C2R, st);
    return rc;
}

extern "C" int shtc_analysis_c(const shtc_plan* P, const void* grid, long long gsf,
                               long long gsr, long long gsc, void* cilm, long long csf,
                               long long csk, long long csl, long long csm, int cdim,
                               int nfield, void* work, size_t wb, void* stream) {
    int rc = check_call(P, grid, cilm, nfield, work, wb);
    if (rc) return rc;
    if ((rc = check_kind(P, 1))) return rc;
    if (cdim < P->lc + 1) return SHTC_EDIM;
    cudaStream_t st = (cudaStream_t)stream;
    const int nf2 = 2 * nfield;
    double2* partial = (double2*)work;
    double2* spec = (double2*)((char*)work + coef_region(P, nf2));
    double2* fbuf = fft_scratch(P, work, coef_region(P, nf2) + spec_region(P, nf2));
    const int tiles = anal_tiles(P, nf2);
    stage_begin(SHTC_STAGE_FFT_R2C, st);
    rc = launch_fft_c2c_anal(P, (const double2*)grid, gsf, gsr, gsc, spec, nfield, st, fbuf);
    stage_end(SHTC_STAGE_FFT_R2C, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_ANAL, st);
    rc = launch_legendre_anal(P, spec, partial, tiles, nf2, st);
    stage_end(SHTC_STAGE_LEGENDRE_ANAL, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_UNPACK, st);
    rc = launch_unpack_coef_c(P, partial, tiles, (double2*)cilm, csf, csk, csl, csm, cdim,
                              nfield, st);
    stage_end(SHTC_STAGE_UNPACK, st);
    return rc;
}

// ---------------------------------------------------------------------------
// MakeGradientDH: a real DH plan with norm 1 and csphase 1 (the reference's
// only case); workspace = packed (3 nfield) | spectra (3 nfield) | (2 nfield)
// ---------------------------------------------------------------------------
extern "C" size_t shtc_gradient_workspace_bytes(const shtc_plan* P, int nfield) {
    if (!P || nfield < 1) return 0;
    return coef_region(P, 3 * nfield) + spec_region(P, 3 * nfield) +
           spec_region(P, 2 * nfield) + fft_region(P);
}

extern "C" int shtc_gradient_dh(const shtc_plan* P, const double* cilm, long long csf,
                                long long csk, long long csl, long long csm, int cdim,
                                double* theta, double* phi, long long gsf, long long gsr,
                                long long gsc, double radius, int nfield, void* work,
                                size_t wb, void* stream) {
    if (!P || !cilm || !theta || !phi) return SHTC_EHANDLE;
    if (nfield < 1) return SHTC_EBOUND;
    if (P->kind != SHTC_GRID_DH || P->cplx || P->norm != 1 || P->csphase != 1)
        return SHTC_EBOUND;
    if (!(radius > 0.0) && !(radius < 0.0)) return SHTC_EBOUND;
    if (cdim < 1) return SHTC_EDIM;
    if (!work || wb < shtc_gradient_workspace_bytes(P, nfield)) return SHTC_EWORK;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != P->device) return SHTC_EHANDLE;
    char* w = (char*)work;
    double2* packed = (double2*)w;
    double2* spec = (double2*)(w + coef_region(P, 3 * nfield));
    const size_t o2 = coef_region(P, 3 * nfield) + spec_region(P, 3 * nfield);
    double2* spec2 = (double2*)(w + o2);
    double2* fbuf = fft_scratch(P, work, o2 + spec_region(P, 2 * nfield));
    return launch_gradient_dh(P, cilm, csf, csk, csl, csm, cdim, theta, phi, gsf, gsr, gsc,
                              radius, nfield, packed, spec, spec2, (cudaStream_t)stream, fbuf);
}

// ---------------------------------------------------------------------------
// MakeGravGridDH: a real DH plan with norm 1 and csphase 1; workspace =
// packed (3 nfield) | spectra (3 nfield) | (4 nfield) | ring and row tables
// ---------------------------------------------------------------------------
extern "C" size_t shtc_gravity_workspace_bytes(const shtc_plan* P, int nfield) {
    if (!P || nfield < 1) return 0;
    return coef_region(P, 3 * nfield) + spec_region(P, 3 * nfield) +
           spec_region(P, 4 * nfield) + align256(grav_table_bytes(P)) + fft_region(P);
}

extern "C" int shtc_gravity_dh(const shtc_plan* P, const double* cilm, long long csf,
                               long long csk, long long csl, long long csm, int cdim,
                               double gm, double r0, double a, double f, int has_omega,
                               double omega, int normal_gravity, double normal_gravity_gm,
                               double* rad, double* theta, double* phi, double* total,
                               double* pot, long long gsf, long long gsr, long long gsc,
                               int nfield, void* work, size_t wb, void* stream) {
    if (!P || !cilm || !rad || !theta || !phi || !total) return SHTC_EHANDLE;
    if (nfield < 1) return SHTC_EBOUND;
    if (P->kind != SHTC_GRID_DH || P->cplx || P->norm != 1 || P->csphase != 1)
        return SHTC_EBOUND;
    if (normal_gravity != 0 && normal_gravity != 1) return SHTC_EBOUND;
    if (normal_gravity == 1 && !has_omega) return SHTC_EBOUND;
    if (cdim < 1) return SHTC_EDIM;
    if (!work || wb < shtc_gravity_workspace_bytes(P, nfield)) return SHTC_EWORK;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != P->device) return SHTC_EHANDLE;
    GravParams g;
    g.gm = gm; g.r0 = r0; g.a = a; g.f = f; g.omega = has_omega ? omega : 0.0;
    g.ng_gm = normal_gravity_gm; g.has_omega = has_omega ? 1 : 0;
    g.normal_gravity = normal_gravity;
    char* w = (char*)work;
    size_t o = 0;
    double2* packed = (double2*)(w + o);
    o += coef_region(P, 3 * nfield);
    double2* spec = (double2*)(w + o);
    o += spec_region(P, 3 * nfield);
    double2* spec2 = (double2*)(w + o);
    o += spec_region(P, 4 * nfield);
    double* tab = (double*)(w + o);
    o += align256(grav_table_bytes(P));
    double2* fbuf = fft_scratch(P, work, o);
    return launch_gravity_dh(P, cilm, csf, csk, csl, csm, cdim, g, rad, theta, phi, total,
                             pot, gsf, gsr, gsc, nfield, packed, spec, spec2, tab,
                             (cudaStream_t)stream, fbuf);
}

// ---------------------------------------------------------------------------
// SHMultiply: both fields synthesised on the GLQ grid of the plan (degree
// lmax1 + lmax2), the analysis FFT reads the two grids and transforms their
// pointwise product.  Workspace: packed / partial sums (2 nfield) | spectra
// (2 nfield) | grids (2 nfield x nlat x nlon doubles).
// ---------------------------------------------------------------------------
static size_t grid_region(const shtc_plan* P, int nfield) {
    return align256((size_t)nfield * P->nlat * P->nlon * sizeof(double));
}

extern "C" size_t shtc_multiply_workspace_bytes(const shtc_plan* P, int nfield) {
    if (!P || nfield < 1) return 0;
    return coef_region(P, 2 * nfield) + spec_region(P, 2 * nfield) +
           grid_region(P, 2 * nfield) + fft_region(P);
}

extern "C" int shtc_multiply(const shtc_plan* P, const double* cilm1, long long c1sf,
                             long long c1sk, long long c1sl, long long c1sm, int lmax1,
                             const double* cilm2, long long c2sf, long long c2sk,
                             long long c2sl, long long c2sm, int lmax2, double* cilmout,
                             long long csf, long long csk, long long csl, long long csm,
                             int cdim_out, int nfield, void* work, size_t wb, void* stream) {
    if (!P || !cilm1 || !cilm2 || !cilmout) return SHTC_EHANDLE;
    if (nfield < 1 || lmax1 < 0 || lmax2 < 0) return SHTC_EBOUND;
    if (P->kind != SHTC_GRID_GLQ || P->cplx || P->extend || P->lmax != lmax1 + lmax2 ||
        P->lc != P->lmax)
        return SHTC_EBOUND;
    if (cdim_out < P->lmax + 1) return SHTC_EDIM;
    if (!work || wb < shtc_multiply_workspace_bytes(P, nfield)) return SHTC_EWORK;
    int dev = -1;
    cudaGetDevice(&dev);
    if (dev != P->device) return SHTC_EHANDLE;
    cudaStream_t st = (cudaStream_t)stream;
    char* w = (char*)work;
    double2* packed = (double2*)w;
    double2* spec = (double2*)(w + coef_region(P, 2 * nfield));
    double* grids = (double*)(w + coef_region(P, 2 * nfield) + spec_region(P, 2 * nfield));
    double2* fbuf = fft_scratch(P, work, coef_region(P, 2 * nfield) +
                                             spec_region(P, 2 * nfield) +
                                             grid_region(P, 2 * nfield));
    const long long gf = (long long)P->nlat * P->nlon;
    const int tiles = anal_tiles(P, nfield);
    stage_begin(SHTC_STAGE_PACK, st);
    int rc = launch_pack_coef(P, cilm1, SHTC_F64, c1sf, c1sk, c1sl, c1sm, lmax1 + 1, packed,
                              nfield, 0, st, 2 * nfield, 0);
    if (!rc) rc = launch_pack_coef(P, cilm2, SHTC_F64, c2sf, c2sk, c2sl, c2sm, lmax2 + 1,
                                   packed, nfield, 0, st, 2 * nfield, nfield);
    stage_end(SHTC_STAGE_PACK, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_SYNTH, st);
    rc = launch_legendre_synth(P, packed, spec, 2 * nfield, st);
    stage_end(SHTC_STAGE_LEGENDRE_SYNTH, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_FFT_C2R, st);
    rc = launch_fft_c2r(P, spec, grids, SHTC_F64, gf, P->nlon, 1, 2 * nfield, 0, st, fbuf);
    stage_end(SHTC_STAGE_FFT_C2R, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_FFT_R2C, st);
    rc = launch_fft_r2c_product(P, grids, grids + (long long)nfield * gf, gf, P->nlon, 1, spec,
                                nfield, st, fbuf);
    stage_end(SHTC_STAGE_FFT_R2C, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_LEGENDRE_ANAL, st);
    rc = launch_legendre_anal(P, spec, packed, tiles, nfield, st);
    stage_end(SHTC_STAGE_LEGENDRE_ANAL, st);
    if (rc) return rc;
    stage_begin(SHTC_STAGE_UNPACK, st);
    rc = launch_unpack_coef(P, packed, tiles, cilmout, SHTC_F64, csf, csk, csl, csm, cdim_out,
                            nfield, 1, st);
    stage_end(SHTC_STAGE_UNPACK, st);
    return rc;
}

// ---------------------------------------------------------------------------
// host drop-ins of include/shtools.h
// ---------------------------------------------------------------------------
namespace {

struct PlanKey {
    int kind, lmax, lc, norm, csphase, sampling, extend, device, cplx;
    std::vector<double> zero;
    bool operator<(const PlanKey& o) const {
        return std::tie(kind, lmax, lc, norm, csphase, sampling, extend, device, cplx, zero) <
               std::tie(o.kind, o.lmax, o.lc, o.norm, o.csphase, o.sampling, o.extend,
                        o.device, o.cplx, o.zero);
    }
};

std::mutex g_mu;
std::map<PlanKey, shtc_plan*> g_plans;

// Plans of the host drop-ins are cached per option set and device for the
// life of the process, like the reference's saved tables.
int cached_plan(int kind, int lmax, int lc, int norm, int csphase, int sampling,
                int extend, const double* zero, const double* w, shtc_plan** out,
                cudaStream_t st, int cplx = 0) {
    PlanKey k;
    k.kind = kind; k.lmax = lmax; k.lc = lc; k.norm = norm; k.csphase = csphase;
    k.sampling = sampling; k.extend = extend; k.cplx = cplx;
    cudaGetDevice(&k.device);
    if (zero) k.zero.assign(zero, zero + lmax + 1);
    if (w) k.zero.insert(k.zero.end(), w, w + lmax + 1);
    std::lock_guard<std::mutex> g(g_mu);
    auto it = g_plans.find(k);
    if (it != g_plans.end()) { *out = it->second; return SHTC_OK; }
    shtc_plan* p = nullptr;
    int rc;
    if (kind == SHTC_GRID_DH)
        rc = cplx ? shtc_plan_create_dhc(&p, lmax, sampling, lc, norm, csphase, extend, st)
                  : shtc_plan_create_dh(&p, lmax, sampling, lc, norm, csphase, extend, st);
    else
        rc = cplx ? shtc_plan_create_glqc(&p, lmax, zero, w, lc, norm, csphase, extend, st)
                  : shtc_plan_create_glq(&p, lmax, zero, w, lc, norm, csphase, extend, st);
    if (rc) return rc;
    g_plans[k] = p;
    *out = p;
    return SHTC_OK;
}

struct DevBuf {
    void* p = nullptr;
    ~DevBuf() { if (p) cudaFree(p); }
    int alloc(size_t b) { return cudaMalloc(&p, b ? b : 8) == cudaSuccess ? SHTC_OK : SHTC_EALLOC; }
};

void set_status(int* exitstatus, int rc) {
    if (exitstatus) *exitstatus = rc;
}

int opt(const int* p, int def) { return p ? *p : def; }

}  // namespace

extern "C" void MakeGridDH(double* griddh, const int d0, const int d1, int* n,
                           const double* cilm, const int cdim, const int lmax,
                           const int* norm, const int* sampling,
                           const int* csphase, const int* lmax_calc,
                           const int* extend, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int nn = 2 * lmax + 2;
    if (n) *n = nn;
    const int samp = opt(sampling, 1), ext = opt(extend, 0), nrm = opt(norm, 1),
              cs = opt(csphase, 1);
    if (samp != 1 && samp != 2) return set_status(exitstatus, SHTC_EBOUND);
    if (ext != 0 && ext != 1) return set_status(exitstatus, SHTC_EBOUND);
    const int nlat_out = nn + ext, nlon_out = samp * nn + ext;
    if (d0 < nlat_out || d1 < nlon_out) return set_status(exitstatus, SHTC_EDIM);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    int lc = lmax < cdim - 1 ? lmax : cdim - 1;
    if (lmax_calc) {
        if (*lmax_calc > lmax) return set_status(exitstatus, SHTC_EBOUND);
        if (*lmax_calc < lc) lc = *lmax_calc;
    }
    if (lc < 0) return set_status(exitstatus, SHTC_EDIM);
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_DH, lmax, lc, nrm, cs, samp, ext, nullptr, nullptr, &P, st);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t wb = shtc_workspace_bytes(P, 1);
    if ((rc = dc.alloc(sizeof(double) * 2 * (size_t)cdim * cdim)) ||
        (rc = dg.alloc(sizeof(double) * (size_t)d0 * d1)) || (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dc.p, cilm, sizeof(double) * 2 * (size_t)cdim * cdim,
                                  cudaMemcpyHostToDevice, st));
    if (!rc) rc = shtc_synthesis(P, (const double*)dc.p, 0, 1, 2, 2LL * cdim, cdim,
                                 (double*)dg.p, 0, 1, d0, 1, dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpy2DAsync(griddh, sizeof(double) * d0, dg.p,
                                             sizeof(double) * d0,
                                             sizeof(double) * nlat_out, nlon_out,
                                             cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

extern "C" void SHExpandDH(const double* grid, const int d0, const int d1,
                           const int n, double* cilm, const int cdim, int* lmax,
                           const int* norm, const int* sampling,
                           const int* csphase, const int* lmax_calc,
                           int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int L = n / 2 - 1;
    if (lmax) *lmax = L;
    int lc = L;
    if (lmax_calc) {
        if (*lmax_calc > L) return set_status(exitstatus, SHTC_EBOUND);
        lc = *lmax_calc < L ? *lmax_calc : L;
    }
    const int samp = opt(sampling, 1), nrm = opt(norm, 1), cs = opt(csphase, 1);
    if (samp != 1 && samp != 2) return set_status(exitstatus, SHTC_EBOUND);
    if (n % 2 != 0) return set_status(exitstatus, SHTC_EBOUND);
    if (cdim < lc + 1) return set_status(exitstatus, SHTC_EDIM);
    if (d0 < n || d1 < samp * n) return set_status(exitstatus, SHTC_EDIM);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_DH, L, lc, nrm, cs, samp, 0, nullptr, nullptr, &P, st);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t wb = shtc_workspace_bytes(P, 1);
    if ((rc = dc.alloc(sizeof(double) * 2 * (size_t)cdim * cdim)) ||
        (rc = dg.alloc(sizeof(double) * (size_t)d0 * d1)) || (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dg.p, grid, sizeof(double) * (size_t)d0 * d1,
                                  cudaMemcpyHostToDevice, st));
    if (!rc) rc = shtc_analysis(P, (const double*)dg.p, 0, 1, d0, (double*)dc.p, 0, 1, 2,
                                2LL * cdim, cdim, 1, dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpyAsync(cilm, dc.p, sizeof(double) * 2 * (size_t)cdim * cdim,
                                           cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

extern "C" void MakeGridGLQ(double* gridglq, const int d0, const int d1,
                            const double* cilm, const int cdim, const int lmax,
                            const double* plx, const double* zero,
                            const int* norm, const int* csphase,
                            const int* lmax_calc, const int* extend,
                            int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int ext = opt(extend, 0), nrm = opt(norm, 1), cs = opt(csphase, 1);
    if (ext != 0 && ext != 1) return set_status(exitstatus, SHTC_EBOUND);
    const int nlat = lmax + 1, nlon_out = 2 * lmax + 1 + ext;
    if (d1 < nlon_out || d0 < nlat) return set_status(exitstatus, SHTC_EDIM);
    if (plx) return set_status(exitstatus, SHTC_EBOUND);
    if (!zero) return set_status(exitstatus, SHTC_ENOZERO);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    int lc = lmax < cdim - 1 ? lmax : cdim - 1;
    if (lmax_calc) {
        if (*lmax_calc > lmax) return set_status(exitstatus, SHTC_EBOUND);
        if (*lmax_calc < lc) lc = *lmax_calc;
    }
    if (lc < 0) return set_status(exitstatus, SHTC_EDIM);
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    // the analysis weights are not needed for a synthesis: nodes only
    int rc = cached_plan(SHTC_GRID_GLQ, lmax, lc, nrm, cs, 1, ext, zero, nullptr, &P, st);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t wb = shtc_workspace_bytes(P, 1);
    if ((rc = dc.alloc(sizeof(double) * 2 * (size_t)cdim * cdim)) ||
        (rc = dg.alloc(sizeof(double) * (size_t)d0 * d1)) || (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dc.p, cilm, sizeof(double) * 2 * (size_t)cdim * cdim,
                                  cudaMemcpyHostToDevice, st));
    if (!rc) rc = shtc_synthesis(P, (const double*)dc.p, 0, 1, 2, 2LL * cdim, cdim,
                                 (double*)dg.p, 0, 1, d0, 1, dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpy2DAsync(gridglq, sizeof(double) * d0, dg.p,
                                             sizeof(double) * d0, sizeof(double) * nlat,
                                             nlon_out, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

extern "C" void SHExpandGLQ(double* cilm, const int cdim, const int lmax,
                            const double* gridglq, const double* w,
                            const double* plx, const double* zero,
                            const int* norm, const int* csphase,
                            const int* lmax_calc, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    int lc = lmax;
    if (lmax_calc) {
        if (*lmax_calc > lmax) return set_status(exitstatus, SHTC_EBOUND);
        lc = *lmax_calc < lmax ? *lmax_calc : lmax;
    }
    if (cdim < lc + 1) return set_status(exitstatus, SHTC_EDIM);
    if (!w) return set_status(exitstatus, SHTC_EDIM);
    if (plx) return set_status(exitstatus, SHTC_EBOUND);
    if (!zero) return set_status(exitstatus, SHTC_ENOZERO);
    const int nrm = opt(norm, 1), cs = opt(csphase, 1);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    const int nlat = lmax + 1, nlon = 2 * lmax + 1;
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_GLQ, lmax, lc, nrm, cs, 1, 0, zero, w, &P, st);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t wb = shtc_workspace_bytes(P, 1);
    if ((rc = dc.alloc(sizeof(double) * 2 * (size_t)cdim * cdim)) ||
        (rc = dg.alloc(sizeof(double) * (size_t)nlat * nlon)) || (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dg.p, gridglq, sizeof(double) * (size_t)nlat * nlon,
                                  cudaMemcpyHostToDevice, st));
    if (!rc) rc = shtc_analysis(P, (const double*)dg.p, 0, 1, nlat, (double*)dc.p, 0, 1, 2,
                                2LL * cdim, cdim, 1, dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpyAsync(cilm, dc.p, sizeof(double) * 2 * (size_t)cdim * cdim,
                                           cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

extern "C" void PreGLQ(const double x1, const double x2, const int n,
                       double* zero, double* w, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    if (n < 1 || !zero || !w) return set_status(exitstatus, SHTC_EDIM);
    cudaStream_t st = cudaStreamPerThread;
    DevBuf dz, dw;
    int rc;
    if ((rc = dz.alloc(sizeof(double) * n)) || (rc = dw.alloc(sizeof(double) * n)))
        return set_status(exitstatus, rc);
    rc = shtc_preglq(x1, x2, n, (double*)dz.p, (double*)dw.p, st);
    if (!rc) rc = map_cuda(cudaMemcpyAsync(zero, dz.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaMemcpyAsync(w, dw.p, sizeof(double) * n, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

// Complex drop-ins (include/shtools.h:117-141, 174-197): the same argument
// handling as the real ones; arrays of interleaved complex doubles.
extern "C" void MakeGridDHC(shtc_complex* griddh, const int d0, const int d1, int* n,
                            const shtc_complex* cilm, const int cdim, const int lmax,
                            const int* norm, const int* sampling, const int* csphase,
                            const int* lmax_calc, const int* extend, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int nn = 2 * lmax + 2;
    if (n) *n = nn;
    const int samp = opt(sampling, 1), ext = opt(extend, 0), nrm = opt(norm, 1),
              cs = opt(csphase, 1);
    if (samp != 1 && samp != 2) return set_status(exitstatus, SHTC_EBOUND);
    if (ext != 0 && ext != 1) return set_status(exitstatus, SHTC_EBOUND);
    const int nlat_out = nn + ext, nlon_out = samp * nn + ext;
    if (d0 < nlat_out || d1 < nlon_out) return set_status(exitstatus, SHTC_EDIM);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    int lc = lmax < cdim - 1 ? lmax : cdim - 1;
    if (lmax_calc) {
        if (*lmax_calc > lmax) return set_status(exitstatus, SHTC_EBOUND);
        if (*lmax_calc < lc) lc = *lmax_calc;
    }
    if (lc < 0) return set_status(exitstatus, SHTC_EDIM);
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_DH, lmax, lc, nrm, cs, samp, ext, nullptr, nullptr, &P, st,
                         1);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t cb = sizeof(double2) * 2 * (size_t)cdim * cdim;
    const size_t wb = shtc_workspace_bytes(P, 1);
    if ((rc = dc.alloc(cb)) || (rc = dg.alloc(sizeof(double2) * (size_t)d0 * d1)) ||
        (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dc.p, cilm, cb, cudaMemcpyHostToDevice, st));
    if (!rc) rc = shtc_synthesis_c(P, dc.p, 0, 1, 2, 2LL * cdim, cdim, dg.p, 0, 1, d0, 1,
                                   dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpy2DAsync(griddh, sizeof(double2) * d0, dg.p,
                                             sizeof(double2) * d0, sizeof(double2) * nlat_out,
                                             nlon_out, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

extern "C" void SHExpandDHC(const shtc_complex* grid, const int d0, const int d1,
                            const int n, shtc_complex* cilm, const int cdim, int* lmax,
                            const int* norm, const int* sampling, const int* csphase,
                            const int* lmax_calc, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int L = n / 2 - 1;
    if (lmax) *lmax = L;
    int lc = L;
    if (lmax_calc) {
        if (*lmax_calc > L) return set_status(exitstatus, SHTC_EBOUND);
        lc = *lmax_calc < L ? *lmax_calc : L;
    }
    const int samp = opt(sampling, 1), nrm = opt(norm, 1), cs = opt(csphase, 1);
    if (samp != 1 && samp != 2) return set_status(exitstatus, SHTC_EBOUND);
    if (n % 2 != 0) return set_status(exitstatus, SHTC_EBOUND);
    if (cdim < lc + 1) return set_status(exitstatus, SHTC_EDIM);
    if (d0 < n || d1 < samp * n) return set_status(exitstatus, SHTC_EDIM);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_DH, L, lc, nrm, cs, samp, 0, nullptr, nullptr, &P, st, 1);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t cb = sizeof(double2) * 2 * (size_t)cdim * cdim;
    const size_t wb = shtc_workspace_bytes(P, 1);
    if ((rc = dc.alloc(cb)) || (rc = dg.alloc(sizeof(double2) * (size_t)d0 * d1)) ||
        (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dg.p, grid, sizeof(double2) * (size_t)d0 * d1,
                                  cudaMemcpyHostToDevice, st));
    if (!rc) rc = map_cuda(cudaMemsetAsync(dc.p, 0, cb, st));
    if (!rc) rc = shtc_analysis_c(P, dg.p, 0, 1, d0, dc.p, 0, 1, 2, 2LL * cdim, cdim, 1,
                                  dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpyAsync(cilm, dc.p, cb, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

extern "C" void MakeGridGLQC(shtc_complex* gridglq, const int d0, const int d1,
                             const shtc_complex* cilm, const int cdim, const int lmax,
                             const double* plx, const double* zero, const int* norm,
                             const int* csphase, const int* lmax_calc, const int* extend,
                             int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int ext = opt(extend, 0), nrm = opt(norm, 1), cs = opt(csphase, 1);
    if (ext != 0 && ext != 1) return set_status(exitstatus, SHTC_EBOUND);
    const int nlat = lmax + 1, nlon_out = 2 * lmax + 1 + ext;
    if (d1 < nlon_out || d0 < nlat) return set_status(exitstatus, SHTC_EDIM);
    if (plx) return set_status(exitstatus, SHTC_EBOUND);
    if (!zero) return set_status(exitstatus, SHTC_ENOZERO);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    int lc = lmax < cdim - 1 ? lmax : cdim - 1;
    if (lmax_calc) {
        if (*lmax_calc > lmax) return set_status(exitstatus, SHTC_EBOUND);
        if (*lmax_calc < lc) lc = *lmax_calc;
    }
    if (lc < 0) return set_status(exitstatus, SHTC_EDIM);
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_GLQ, lmax, lc, nrm, cs, 1, ext, zero, nullptr, &P, st, 1);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t cb = sizeof(double2) * 2 * (size_t)cdim * cdim;
    const size_t wb = shtc_workspace_bytes(P, 1);
    if ((rc = dc.alloc(cb)) || (rc = dg.alloc(sizeof(double2) * (size_t)d0 * d1)) ||
        (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dc.p, cilm, cb, cudaMemcpyHostToDevice, st));
    if (!rc) rc = shtc_synthesis_c(P, dc.p, 0, 1, 2, 2LL * cdim, cdim, dg.p, 0, 1, d0, 1,
                                   dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpy2DAsync(gridglq, sizeof(double2) * d0, dg.p,
                                             sizeof(double2) * d0, sizeof(double2) * nlat,
                                             nlon_out, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

extern "C" void SHExpandGLQC(shtc_complex* cilm, const int cdim, const int lmax,
                             const shtc_complex* gridglq, const double* w,
                             const double* plx, const double* zero, const int* norm,
                             const int* csphase, const int* lmax_calc, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    int lc = lmax;
    if (lmax_calc) {
        if (*lmax_calc > lmax) return set_status(exitstatus, SHTC_EBOUND);
        lc = *lmax_calc < lmax ? *lmax_calc : lmax;
    }
    if (cdim < lc + 1) return set_status(exitstatus, SHTC_EDIM);
    if (!w) return set_status(exitstatus, SHTC_EDIM);
    if (plx) return set_status(exitstatus, SHTC_EBOUND);
    if (!zero) return set_status(exitstatus, SHTC_ENOZERO);
    const int nrm = opt(norm, 1), cs = opt(csphase, 1);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    const int nlat = lmax + 1, nlon = 2 * lmax + 1;
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_GLQ, lmax, lc, nrm, cs, 1, 0, zero, w, &P, st, 1);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t cb = sizeof(double2) * 2 * (size_t)cdim * cdim;
    const size_t wb = shtc_workspace_bytes(P, 1);
    if ((rc = dc.alloc(cb)) || (rc = dg.alloc(sizeof(double2) * (size_t)nlat * nlon)) ||
        (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dg.p, gridglq, sizeof(double2) * (size_t)nlat * nlon,
                                  cudaMemcpyHostToDevice, st));
    if (!rc) rc = map_cuda(cudaMemsetAsync(dc.p, 0, cb, st));
    if (!rc) rc = shtc_analysis_c(P, dg.p, 0, 1, nlat, dc.p, 0, 1, 2, 2LL * cdim, cdim, 1,
                                  dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpyAsync(cilm, dc.p, cb, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

// src/cWrapper.f95:295-317 (src/MakeGradientDH.f95:1)
extern "C" void MakeGradientDH(const double* cilm, const int cdim, const int lmax,
                               double* theta, double* phi, const int d0, const int d1,
                               int* n, const int* sampling, const int* lmax_calc,
                               const int* extend, const double* radius, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int nn = 2 * lmax + 2;
    if (n) *n = nn;
    const int samp = opt(sampling, 1), ext = opt(extend, 0);
    const double r = radius ? *radius : 1.0;
    if (samp != 1 && samp != 2) return set_status(exitstatus, SHTC_EBOUND);
    if (ext != 0 && ext != 1) return set_status(exitstatus, SHTC_EBOUND);
    const int nlat_out = nn + ext, nlon_out = samp * nn + ext;
    if (d0 < nlat_out || d1 < nlon_out) return set_status(exitstatus, SHTC_EDIM);
    int lc = lmax < cdim - 1 ? lmax : cdim - 1;
    if (lmax_calc) {
        if (*lmax_calc > lmax) return set_status(exitstatus, SHTC_EBOUND);
        if (*lmax_calc < lc) lc = *lmax_calc;
    }
    if (lc < 0) return set_status(exitstatus, SHTC_EDIM);
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_DH, lmax, lc, 1, 1, samp, ext, nullptr, nullptr, &P, st);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dt, dp, dw;
    const size_t wb = shtc_gradient_workspace_bytes(P, 1);
    const size_t gb = sizeof(double) * (size_t)d0 * d1;
    if ((rc = dc.alloc(sizeof(double) * 2 * (size_t)cdim * cdim)) || (rc = dt.alloc(gb)) ||
        (rc = dp.alloc(gb)) || (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(dc.p, cilm, sizeof(double) * 2 * (size_t)cdim * cdim,
                                  cudaMemcpyHostToDevice, st));
    if (!rc) rc = shtc_gradient_dh(P, (const double*)dc.p, 0, 1, 2, 2LL * cdim, cdim,
                                   (double*)dt.p, (double*)dp.p, 0, 1, d0, r, 1, dw.p, wb, st);
    if (!rc) rc = map_cuda(cudaMemcpy2DAsync(theta, sizeof(double) * d0, dt.p,
                                             sizeof(double) * d0, sizeof(double) * nlat_out,
                                             nlon_out, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaMemcpy2DAsync(phi, sizeof(double) * d0, dp.p,
                                             sizeof(double) * d0, sizeof(double) * nlat_out,
                                             nlon_out, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

// include/shtools.h:726-746 via src/cWrapper.f95:1484-1514 (src/MakeGravGridDH.f95:1)
extern "C" void MakeGravGridDH(const double* cilm, const int cdim, const int lmax,
                               const double gm, const double r0, const double a,
                               const double f, double* rad, const int nlon, const int nlat,
                               double* theta, double* phi, double* total, int* n,
                               const int* sampling, const int* lmax_calc, const double* omega,
                               const int* normal_gravity, double* pot, const int* extend,
                               int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int nn = 2 * lmax + 2;
    if (n) *n = nn;
    const int samp = opt(sampling, 1), ext = opt(extend, 0), ng = opt(normal_gravity, 0);
    if (samp != 1 && samp != 2) return set_status(exitstatus, SHTC_EBOUND);
    if (ext != 0 && ext != 1) return set_status(exitstatus, SHTC_EBOUND);
    if (cdim < 1) return set_status(exitstatus, SHTC_EDIM);
    const int nlat_out = nn + ext, nlon_out = samp * nn + ext;
    if (nlat < nlat_out || nlon < nlon_out) return set_status(exitstatus, SHTC_EDIM);
    if (ng != 0 && ng != 1) return set_status(exitstatus, SHTC_EBOUND);
    if (ng == 1 && !omega) return set_status(exitstatus, 5);   // MakeGravGridDH.f95:244-252
    int lc = lmax < cdim - 1 ? lmax : cdim - 1;
    if (lmax_calc) {
        if (*lmax_calc > lmax) return set_status(exitstatus, SHTC_EBOUND);
        if (*lmax_calc < lc) lc = *lmax_calc;
    }
    if (lc < 0) return set_status(exitstatus, SHTC_EDIM);
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_DH, lmax, lc, 1, 1, samp, ext, nullptr, nullptr, &P, st);
    if (rc) return set_status(exitstatus, rc);
    DevBuf dc, dg, dw;
    const size_t wb = shtc_gravity_workspace_bytes(P, 1);
    const size_t gb = sizeof(double) * (size_t)nlat * nlon;
    const int ngrid = pot ? 5 : 4;
    if ((rc = dc.alloc(sizeof(double) * 2 * (size_t)cdim * cdim)) ||
        (rc = dg.alloc(gb * ngrid)) || (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    double* d[5];
    for (int k = 0; k < 5; ++k) d[k] = k < ngrid ? (double*)((char*)dg.p + gb * k) : nullptr;
    rc = map_cuda(cudaMemcpyAsync(dc.p, cilm, sizeof(double) * 2 * (size_t)cdim * cdim,
                                  cudaMemcpyHostToDevice, st));
    // grids (nlat, nlon) column-major: row stride 1, column stride nlat
    if (!rc) rc = shtc_gravity_dh(P, (const double*)dc.p, 0, 1, 2, 2LL * cdim, cdim, gm, r0, a,
                                  f, omega ? 1 : 0, omega ? *omega : 0.0, ng, gm, d[0], d[1],
                                  d[2], d[3], d[4], 0, 1, nlat, 1, dw.p, wb, st);
    double* host[5] = {rad, theta, phi, total, pot};
    for (int k = 0; k < ngrid && !rc; ++k)
        rc = map_cuda(cudaMemcpy2DAsync(host[k], sizeof(double) * nlat, d[k],
                                        sizeof(double) * nlat, sizeof(double) * nlat_out,
                                        nlon_out, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

// include/shtools.h:254-265 (src/SHMultiply.f95:1); precomp is accepted and
// ignored (it selects the reference's precomputed Legendre tables)
extern "C" void SHMultiply(double* cilmout, const int cdout, const double* cilm1,
                           const int cd1, const int lmax1, const double* cilm2,
                           const int cd2, const int lmax2, const int* precomp,
                           const int* norm, const int* csphase, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    (void)precomp;
    if (lmax1 < 0 || lmax2 < 0) return set_status(exitstatus, SHTC_EBOUND);
    if (cd1 < lmax1 + 1 || cd2 < lmax2 + 1 || cdout < lmax1 + lmax2 + 1)
        return set_status(exitstatus, SHTC_EDIM);
    const int nrm = opt(norm, 1), cs = opt(csphase, 1);
    if (nrm < 1 || nrm > 4) return set_status(exitstatus, SHTC_EBOUND);
    if (cs != 1 && cs != -1) return set_status(exitstatus, SHTC_EBOUND);
    const int lo = lmax1 + lmax2;
    cudaStream_t st = cudaStreamPerThread;
    shtc_plan* P = nullptr;
    int rc = cached_plan(SHTC_GRID_GLQ, lo, lo, nrm, cs, 1, 0, nullptr, nullptr, &P, st);
    if (rc) return set_status(exitstatus, rc);
    DevBuf d1, d2, dout, dw;
    const size_t wb = shtc_multiply_workspace_bytes(P, 1);
    const size_t b1 = sizeof(double) * 2 * (size_t)cd1 * cd1;
    const size_t b2 = sizeof(double) * 2 * (size_t)cd2 * cd2;
    const size_t bo = sizeof(double) * 2 * (size_t)cdout * cdout;
    if ((rc = d1.alloc(b1)) || (rc = d2.alloc(b2)) || (rc = dout.alloc(bo)) ||
        (rc = dw.alloc(wb)))
        return set_status(exitstatus, rc);
    rc = map_cuda(cudaMemcpyAsync(d1.p, cilm1, b1, cudaMemcpyHostToDevice, st));
    if (!rc) rc = map_cuda(cudaMemcpyAsync(d2.p, cilm2, b2, cudaMemcpyHostToDevice, st));
    if (!rc) rc = map_cuda(cudaMemsetAsync(dout.p, 0, bo, st));
    // Fortran column-major (2, dim, dim): k stride 1, l stride 2, m stride 2 dim
    if (!rc) rc = shtc_multiply(P, (const double*)d1.p, 0, 1, 2, 2LL * cd1, lmax1,
                                (const double*)d2.p, 0, 1, 2, 2LL * cd2, lmax2,
                                (double*)dout.p, 0, 1, 2, 2LL * cdout, cdout, 1, dw.p, wb,
                                st);
    if (!rc) rc = map_cuda(cudaMemcpyAsync(cilmout, dout.p, bo, cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}

extern "C" void SHGLQ(const int lmax, double* zero, double* w, double* plx,
                      const int* norm, const int* csphase, const int* cnorm,
                      int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    if (plx) return set_status(exitstatus, SHTC_EBOUND);
    if (lmax < 0) return set_status(exitstatus, SHTC_EBOUND);
    PreGLQ(-1.0, 1.0, lmax + 1, zero, w, exitstatus);
}

// GLQGridCoord (GLQGridCoord.f95:1-121): latitudes asin(z_i) in degrees of
// the GPU PreGLQ nodes (:116-118), longitudes 360 (i-1) / nlong (:112-114).
extern "C" void GLQGridCoord(double* latglq, const int latglq_d0, double* longlq,
                             const int longlq_d0, const int lmax, int* nlat, int* nlong,
                             const int* extend, int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    if (lmax < 0) return set_status(exitstatus, SHTC_EBOUND);
    const int nl = lmax + 1, nlo = 2 * lmax + 1, ext = opt(extend, 0);
    if (nlat) *nlat = nl;
    if (nlong) *nlong = nlo;
    if (ext != 0 && ext != 1) return set_status(exitstatus, SHTC_EBOUND);
    if (!latglq || !longlq || latglq_d0 < nl || longlq_d0 < nlo + ext)
        return set_status(exitstatus, SHTC_EDIM);
    std::vector<double> zero(nl), w(nl);
    int rc = SHTC_OK;
    PreGLQ(-1.0, 1.0, nl, zero.data(), w.data(), &rc);
    if (rc) return set_status(exitstatus, rc);
    const double pi = acos(-1.0);
    for (int i = 0; i < nlo + ext; ++i) longlq[i] = 360.0 * (double)i / (double)nlo;
    for (int i = 0; i < nl; ++i) latglq[i] = asin(zero[i]) * 180.0 / pi;
}

extern "C" void DHaj(const int n, double* aj, const int aj_d0, const int* extend,
                     int* exitstatus) {
    set_status(exitstatus, SHTC_OK);
    const int ext = opt(extend, 0);
    if (n % 2 != 0) return set_status(exitstatus, SHTC_EBOUND);
    if (ext != 0 && ext != 1) return set_status(exitstatus, SHTC_EBOUND);
    if (aj_d0 < n + ext) return set_status(exitstatus, SHTC_EDIM);
    cudaStream_t st = cudaStreamPerThread;
    DevBuf da;
    int rc;
    if ((rc = da.alloc(sizeof(double) * (n + ext)))) return set_status(exitstatus, rc);
    rc = shtc_dhaj(n, (double*)da.p, ext, st);
    if (!rc) rc = map_cuda(cudaMemcpyAsync(aj, da.p, sizeof(double) * (n + ext),
                                           cudaMemcpyDeviceToHost, st));
    if (!rc) rc = map_cuda(cudaStreamSynchronize(st));
    set_status(exitstatus, rc);
}
