/*
 * Test infrastructure (oracle), not product code.
 *
 * Declarations of the six FFTW3 entry points that empi's workspace calls
 * (inc/fftw.hpp:33,43,112,125,137,152 in the reference), written for this
 * project so that the reference's unmodified sources compile and link without
 * FFTW, which is not installed here.  The implementation is fftw_shim.c, a
 * textbook FP64 Cooley-Tukey FFT.  Only the subset of FFTW's published API that
 * the reference uses is declared; flag values follow FFTW's documented
 * constants and are ignored by the shim.
 */
#ifndef EMPI_ORACLE_FFTW3_SHIM_H
#define EMPI_ORACLE_FFTW3_SHIM_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef double fftw_complex[2];
typedef struct empi_shim_plan* fftw_plan;

#define FFTW_FORWARD (-1)
#define FFTW_BACKWARD (+1)
#define FFTW_DESTROY_INPUT (1U << 0)
#define FFTW_ESTIMATE (1U << 6)

void* fftw_malloc(size_t n);
void fftw_free(void* p);
fftw_plan fftw_plan_dft_1d(int n, fftw_complex* in, fftw_complex* out, int sign, unsigned flags);
fftw_plan fftw_plan_dft_r2c_1d(int n, double* in, fftw_complex* out, unsigned flags);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);

#ifdef __cplusplus
}
#endif

#endif
