// Unpolarised LDA pieces shared by the f_xc kernel block, V_xc and their
// tests: the Perdew-Zunger correlation potential (libxc's "PZ Original"
// parameters, LIB/libxc/src/lda_c_pz.c) and the Slater exchange potential
// (LIB/libxc/src/lda_x.c), both in Hartree.
#pragma once
#include <cmath>

namespace ngw {

__host__ __device__ __forceinline__ double pz_vc(double rho) {
  const double gamma = -0.1423, beta1 = 1.0529, beta2 = 0.3334;
  const double a = 0.0311, b = -0.048, c = 0.0020, d = -0.0116;
  const double rs = cbrt(3.0 / (4.0 * M_PI * rho));
  if (rs >= 1.0) {
    const double srs = sqrt(rs);
    const double den = 1.0 + beta1 * srs + beta2 * rs;
    const double ec = gamma / den;
    return ec * (1.0 + 7.0 / 6.0 * beta1 * srs + 4.0 / 3.0 * beta2 * rs) / den;
  }
  const double lrs = log(rs);
  return a * lrs + (b - a / 3.0) + 2.0 / 3.0 * c * rs * lrs + (2.0 * d - c) * rs / 3.0;
}

// v_x = (4/3) eps_x,  eps_x = -(3/4) (3/pi)^(1/3) rho^(1/3)
__host__ __device__ __forceinline__ double slater_vx(double rho) {
  return -cbrt(3.0 / M_PI) * cbrt(rho);
}

}  // namespace ngw
