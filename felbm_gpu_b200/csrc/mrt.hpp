// D3Q19 multiple-relaxation-time moment basis.
//
// The reference uploads felbm_local's EquilibriumDistributionMRT::m_mass_matrix
// and its inverse (include/felbm_gpu/multiphase_gpu.cuh:349-350,
// device_engine.cuh:65-81); those values live in the absent felbm_local tree.
// The rate vector the reference builds (device_engine.cuh:623-625,641-643),
//   s = {0,s0,s0,0,s1,0,s1,0,s1, s0 x7, s1 x3},
// fixes the moment order to d'Humieres et al. (2002), Phil. Trans. R. Soc. A
// 360:437: (rho, e, eps, jx, qx, jy, qy, jz, qz, 3pxx, 3pixx, pww, piww,
// pxy, pyz, pxz, mx, my, mz). The rows below are that published basis, as
// polynomials of the velocity, evaluated on the D3Q19 order of d3q19.hpp.
// The rows are mutually orthogonal, so M^-1 = M^T diag(1/|row_j|^2).
#pragma once
#include "d3q19.hpp"

namespace fe {

// Entry M[j][k] of the moment matrix (small integers).
FE_HD constexpr int mrt_M(int j, int k) {
  const int x = lat_cx(k), y = lat_cy(k), z = lat_cz(k);
  const int c2 = x * x + y * y + z * z;
  switch (j) {
    case 0: return 1;
    case 1: return 19 * c2 - 30;
    case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2;
    case 3: return x;
    case 4: return (5 * c2 - 9) * x;
    case 5: return y;
    case 6: return (5 * c2 - 9) * y;
    case 7: return z;
    case 8: return (5 * c2 - 9) * z;
    case 9: return 3 * x * x - c2;
    case 10: return (3 * c2 - 5) * (3 * x * x - c2);
    case 11: return y * y - z * z;
    case 12: return (3 * c2 - 5) * (y * y - z * z);
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return (y * y - z * z) * x;
    case 17: return (z * z - x * x) * y;
    case 18: return (x * x - y * y) * z;
  }
  return 0;
}

// |row_j|^2 = sum_k M[j][k]^2.
FE_HD constexpr int mrt_norm2(int j) {
  int s = 0;
  for (int k = 0; k < Q; ++k) s += mrt_M(j, k) * mrt_M(j, k);
  return s;
}

// Which relaxation rate each moment uses. Conserved moments (rho, j) are
// never relaxed (rate 0 in the reference's vector).
enum MrtKind : int { MK_CONS = 0, MK_E = 1, MK_EPS = 2, MK_Q = 3, MK_NU = 4, MK_PI = 5, MK_M = 6 };
FE_HD constexpr int mrt_kind(int j) {
  return j == 0 || j == 3 || j == 5 || j == 7 ? MK_CONS
       : j == 1 ? MK_E
       : j == 2 ? MK_EPS
       : (j == 4 || j == 6 || j == 8) ? MK_Q
       : (j == 10 || j == 12) ? MK_PI
       : (j >= 16) ? MK_M
       : MK_NU;
}

// How a rate kind is set. RATE_S0: the site's BGK rate 1/(tau+1/2);
// RATE_MAGIC: 2 tau / (2 Lambda + tau) with the same tau (reference
// device_engine.cuh:623-624); RATE_FIXED: a constant.
enum MrtRateMode : int { RATE_S0 = 0, RATE_MAGIC = 1, RATE_FIXED = 2 };

// The reference's assignment: e, eps, nu, pi follow s0; q and m use the
// magic-parameter rate.
FE_HD constexpr int mrt_reference_mode(int kind) {
  return (kind == MK_Q || kind == MK_M) ? RATE_MAGIC : RATE_S0;
}

}  // namespace fe
