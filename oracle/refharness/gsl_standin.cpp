// GSL stand-in of the reference-code harness — TEST INFRASTRUCTURE ONLY.
// gsl_qrng_sobol as the Bratley-Fox construction of dtfe_b200/csrc/sobol.h,
// the only quasi-random generator the reference's averaging method 1 uses
// (averaged_interpolation_1.cc:35).  Linked into every harness library that
// compiles the reference's triangulation.cpp.

#include <cstdio>
#include <cstdlib>

#include <gsl/gsl_qrng.h>

#include "../../dtfe_b200/csrc/sobol.h"

extern "C" {

struct gsl_qrng_type_s {
  int id;
};
struct gsl_qrng_s {
  mutable dtfe::Sobol3 seq;
};
static const gsl_qrng_type kSobolType{1};
static const gsl_qrng_type kNiederreiterType{2};
const gsl_qrng_type* gsl_qrng_sobol = &kSobolType;
const gsl_qrng_type* gsl_qrng_niederreiter_2 = &kNiederreiterType;
gsl_qrng* gsl_qrng_alloc(const gsl_qrng_type* T, unsigned int d) {
  if (T != gsl_qrng_sobol || d != 3) {
    std::fprintf(stderr, "reference harness: only the 3-dimensional Sobol generator is available\n");
    std::abort();
  }
  return new gsl_qrng;
}
int gsl_qrng_get(const gsl_qrng* q, double* x) { return q->seq.next(x) ? 0 : 1; }
void gsl_qrng_free(gsl_qrng* q) { delete q; }

}  // extern "C"
