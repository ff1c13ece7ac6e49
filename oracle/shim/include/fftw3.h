/* FFTW3 shim (TEST INFRASTRUCTURE): the subset the reference's CPU path uses,
 * computed with the oracle's own DFT (selm_oracle.c). */
#ifndef SHIM_FFTW3_H
#define SHIM_FFTW3_H
#include <stddef.h>
typedef double fftw_complex[2];
typedef struct shim_fftw_plan_s* fftw_plan;
#define FFTW_ESTIMATE (1U << 6)
#ifdef __cplusplus
extern "C" {
#endif
double* fftw_alloc_real(size_t n);
void fftw_free(void* p);
void fftw_execute(const fftw_plan p);
void fftw_destroy_plan(fftw_plan p);
#ifdef __cplusplus
}
#endif
#endif
