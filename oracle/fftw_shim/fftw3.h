/*
 * FFTW-API shim for the CPU oracle.  TEST INFRASTRUCTURE ONLY: nothing in the
 * GPU product path includes or links this.
 *
 * The reference (annehutter/polyspectrum) calls FFTW >= 3.3.3 (README.rst:17,23),
 * which is not installed on this machine.  This header declares the subset of
 * the FFTW 3 API that the reference's serial build uses, with FFTW's published
 * semantics:
 *   - fftw_complex is `double _Complex` (FFTW's documented behaviour when
 *     <complex.h> is included before <fftw3.h>, which every reference file does);
 *   - fftw_plan_dft_3d(n0,n1,n2,in,out,sign,flags): row-major 3D c2c DFT,
 *     X[k] = sum_j x[j] exp(sign * 2*pi*i * j.k / n), unnormalised in both
 *     directions (fft.c:30-36, fft.c:50-56 call it with FFTW_FORWARD / FFTW_BACKWARD);
 *   - fftw_malloc / fftw_free / fftw_alloc_complex / fftw_cleanup.
 * The transform itself is this repository's own FP64 code (fftw_shim.c), checked
 * against numpy.fft (pocketfft) in tests/test_oracle_cpu.py.
 */
#ifndef PS_FFTW_SHIM_FFTW3_H
#define PS_FFTW_SHIM_FFTW3_H

#include <stddef.h>
#include <complex.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double _Complex fftw_complex;
typedef struct ps_shim_plan *fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_MEASURE (0U)
#define FFTW_ESTIMATE (1U << 6)

fftw_plan fftw_plan_dft_3d(int n0, int n1, int n2, fftw_complex *in, fftw_complex *out,
                           int sign, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
void *fftw_malloc(size_t n);
void fftw_free(void *p);
fftw_complex *fftw_alloc_complex(size_t n);
void fftw_cleanup(void);

/* Shim-only extras (not FFTW API): thread count used by fftw_execute
 * (default: PS_SHIM_THREADS env var, else all online cores). */
void ps_shim_set_threads(int nthreads);
int ps_shim_get_threads(void);

#ifdef __cplusplus
}
#endif

#endif
