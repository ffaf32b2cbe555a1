// Extra entry of the reference-main harness library (oracle/_ref/
// libdtfe_refmain.so) — TEST INFRASTRUCTURE ONLY.  It times the reference's
// own computeDivergenceShearVorticity (src/DTFE.cpp:436-475, compiled in the
// same library from the reference's DTFE.cpp), which DTFE() runs once on the
// main grid after DTFE_parallel (src/DTFE.cpp:248-249), so the timed
// reference step produces the same fields as the GPU step.

#include <chrono>
#include <cstdint>
#include <cstring>
#include <vector>

#include "define.h"
#include "quantities.h"
#include "user_options.h"

void computeDivergenceShearVorticity(Field& fields, int const verboseLevel, Quantities* q);

extern "C" {

// grad: G cells x 9 floats (the velocity gradient of the main grid); div (G),
// shear (5G), vort (3G) receive the reference's results (may be NULL);
// *seconds the wall time of computeDivergenceShearVorticity alone.
int ref_derived_timed(int64_t G, const float* grad, float* div, float* shear, float* vort, double* seconds) {
  Quantities q;
  q.velocity_gradient.resize((size_t)G);
  std::memcpy(q.velocity_gradient.data(), grad, sizeof(float) * 9 * (size_t)G);
  Field f;
  f.velocity_gradient = true;  // keep the gradient, as a caller that asked for it
  f.velocity_divergence = f.velocity_shear = f.velocity_vorticity = true;
  const auto t0 = std::chrono::steady_clock::now();
  computeDivergenceShearVorticity(f, 0, &q);
  const auto t1 = std::chrono::steady_clock::now();
  if (seconds) *seconds = std::chrono::duration<double>(t1 - t0).count();
  if ((int64_t)q.velocity_divergence.size() != G || (int64_t)q.velocity_shear.size() != G ||
      (int64_t)q.velocity_vorticity.size() != G)
    return 1;
  if (div) std::memcpy(div, q.velocity_divergence.data(), sizeof(float) * (size_t)G);
  if (shear) std::memcpy(shear, q.velocity_shear.data(), sizeof(float) * 5 * (size_t)G);
  if (vort) std::memcpy(vort, q.velocity_vorticity.data(), sizeof(float) * 3 * (size_t)G);
  return 0;
}

}  // extern "C"
