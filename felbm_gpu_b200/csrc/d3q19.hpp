// D3Q19 velocity set and the equilibrium constants of the Lee–Liu step.
//
// Direction order, weights and opposite pairing follow the reference's
// include/felbm_gpu/d3q19.cuh:9-50 (which in turn mirrors felbm_local's
// lbm_velocity_set.h). The order has to be identical because the state
// layout k*n+i exchanged through the C-ABI, checkpoints and HDF5 files is
// indexed by it, and because the MRT moment matrix rows are written against it.
//
//   0:( 0, 0, 0)
//   1:( 1, 0, 0)  2:(-1, 0, 0)  3:( 0, 1, 0)  4:( 0,-1, 0)  5:( 0, 0, 1)  6:( 0, 0,-1)
//   7:( 1, 1, 0)  8:(-1,-1, 0)  9:( 1,-1, 0) 10:(-1, 1, 0)
//  11:( 0, 1, 1) 12:( 0,-1,-1) 13:( 0, 1,-1) 14:( 0,-1, 1)
//  15:( 1, 0, 1) 16:(-1, 0,-1) 17:( 1, 0,-1) 18:(-1, 0, 1)
//
// weights 1/3, 1/18 (axis), 1/36 (diagonal); cs^2 = 1/3.
#pragma once

#ifndef FE_HD
#if defined(__CUDACC__)
#define FE_HD __host__ __device__ __forceinline__
#else
#define FE_HD inline
#endif
#endif

namespace fe {

constexpr int Q = 19;

// Lattice vectors and opposites as constexpr functions, usable in host and
// device code; in the fully unrolled direction loops they fold to constants.
FE_HD constexpr int lat_cx(int k) {
  constexpr int t[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
  return t[k];
}
FE_HD constexpr int lat_cy(int k) {
  constexpr int t[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0};
  return t[k];
}
FE_HD constexpr int lat_cz(int k) {
  constexpr int t[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
  return t[k];
}
FE_HD constexpr int lat_opp(int k) { return k == 0 ? 0 : ((k & 1) ? k + 1 : k - 1); }

// Weight of direction k, as an exact rational evaluated in the working type.
template <typename T>
FE_HD constexpr T weight(int k) {
  return k == 0 ? T(1) / T(3) : (k < 7 ? T(1) / T(18) : T(1) / T(36));
}

// Equilibrium constants (reference d3q19.cuh:45-50): ALPHA = 1/cs^2,
// GAMMA = 1/(2 cs^2), BETA = 1/(2 cs^4).
constexpr double CS2 = 1.0 / 3.0;
constexpr double ALPHA = 3.0;
constexpr double GAMMA = 1.5;
constexpr double BETA = 4.5;

// Plain equilibrium of direction k (reference k_open_bnd,
// device_engine.cuh:790-797): h_k = w c (1 + u_term), g_k = w (p + rho cs^2
// u_term), u_term = e.u (ALPHA + BETA e.u) - GAMMA u.u. The host's initial
// state (fe_init_equilibrium) and the device's (fe_upload_equilibrium, at
// rest) both evaluate it here.
FE_HD void equilibrium_k(int k, double c, double p, double rho, double vx, double vy, double vz, double& h,
                         double& g) {
  const double w = weight<double>(k);
  const double u_sq = vx * vx + vy * vy + vz * vz;
  const double uk = vx * lat_cx(k) + vy * lat_cy(k) + vz * lat_cz(k);
  const double u_term = uk * (ALPHA + BETA * uk) - GAMMA * u_sq;
  h = c * w * (1.0 + u_term);
  g = w * (p + rho * CS2 * u_term);
}

}  // namespace fe
