// Test-harness stand-in for the GSL quasi-random generator used only by the
// reference's averaging method 1, which the harness compiles but never runs;
// the functions abort if called.
#pragma once
#ifdef __cplusplus
extern "C" {
#endif
typedef struct gsl_qrng_type_s gsl_qrng_type;
typedef struct gsl_qrng_s gsl_qrng;
extern const gsl_qrng_type* gsl_qrng_sobol;
extern const gsl_qrng_type* gsl_qrng_niederreiter_2;
gsl_qrng* gsl_qrng_alloc(const gsl_qrng_type* T, unsigned int d);
int gsl_qrng_get(const gsl_qrng* q, double x[]);
void gsl_qrng_free(gsl_qrng* q);
#ifdef __cplusplus
}
#endif
