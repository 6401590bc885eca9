// Passive tracers on the GPU (the reference's host ParticleManager, driven at
// felbm_gpu_main.cu:421-581,752-777; its felbm_local source is not available,
// so the integrator below is this library's definition):
//  * velocity: trilinear interpolation, with periodic wrap, of a node-indexed
//    snapshot of the corrected velocity (solid nodes hold 0). As in the
//    reference driver, which writes the same snapshot into its current and
//    next arrays (felbm_gpu_main.cu:466-481), the velocity is constant over a
//    step; the snapshot is refreshed every velocity_skip steps;
//  * advection: `substeps` substeps of dt = 1/substeps per lattice step,
//    explicit Euler (order 1) or Heun's trapezoid (order 2);
//  * diffusion: per tracer molecular diffusivity Dm, a kick sqrt(2 Dm dt) N(0,1)
//    per axis and substep; no kick along z in a 2-D lattice (nz == 1,
//    reference README "2D runs"), where tracers do not move along z at all;
//    Dm == 0 draws no random numbers;
//  * random numbers: Philox4x32-10 (Salmon et al., SC'11, "Parallel random
//    numbers: as easy as 1, 2, 3"), counter (tracer id, step, substep, draw),
//    key = the 64-bit seed, so a trajectory does not depend on the thread
//    that computes it; normals by the Box-Muller transform of 53-bit
//    uniforms;
//  * walls: a substep whose end position's nearest node is solid is
//    rejected (the tracer stays where it was for that substep);
//  * stretching (optional; reference README "Lagrangian stretching" and
//    docs/HANDOFF_stretching.md section 2): each tracer carries a material
//    line element as a unit orientation rho_hat and a log-length log_rho
//    (Benettin renormalisation). Per accepted substep, with J the velocity
//    gradient (the gradient of the trilinear interpolant) at the substep's
//    start position: lambda_s = rho_hat . J rho_hat (Eq. 12), then
//    rho* = rho_hat + dt J rho_hat, log_rho += log|rho*|, rho_hat = rho*/|rho*|.
//    A tracer is active for the step when no substep was rejected; the step's
//    row averages lambda_s over the active tracers and their substeps, and
//    splits it by the phase of the node nearest to the substep's start
//    (c < 1/2: wetting) when an order-parameter snapshot is attached.
#pragma once
#include <cstdint>

namespace fe {

struct TracerDesc {
  int64_t n;                  // tracers
  int nx, ny, nz;
  int substeps, order;
  uint64_t seed;
  double* pos;                // [3][n]
  double* vel;                // [3][n] interpolated velocity at the end of the step
  const double* dm;           // [n]
  const int64_t* id;          // [n]
  const double* u[3];         // node-indexed velocity snapshot
  const uint8_t* solid;       // [nodes]
  int stretch;                // 1: material line elements carried
  double* rho_hat;            // [3][n] unit orientation
  double* log_rho;            // [n]
  const double* cgrid;        // node-indexed order parameter, or null (no phase split)
  double* part;               // [blocks][NSTR] partial sums of the step
};

// Partial sums of a stretching step: active tracers, sum of lambda_s, wetting
// sum and samples, non-wetting sum and samples, sum of log_rho, of log_rho^2.
constexpr int NSTR = 8;
// Row of the stretching time series: step, lambda, mean_log_rho,
// var_log_rho, n_active, lambda_w, lambda_nw, n_w, n_nw.
constexpr int NROW = 9;
constexpr int TRC = 128;  // tracer-kernel block

// One Philox4x32-10 block: 10 rounds of two 32x32->64 multiplies, the key
// bumped by the Weyl constants between rounds.
__host__ __device__ __forceinline__ void philox4x32_10(uint32_t c[4], uint32_t k0, uint32_t k1) {
  for (int r = 0; r < 10; ++r) {
    const uint64_t p0 = (uint64_t)c[0] * 0xD2511F53u, p1 = (uint64_t)c[2] * 0xCD9E8D57u;
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k0, n2 = hi0 ^ c[3] ^ k1;
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
    k0 += 0x9E3779B9u;
    k1 += 0xBB67AE85u;
  }
}

// Two standard normals from one Philox block (Box-Muller on two uniforms of
// 53 bits each; the first uniform is shifted into (0, 1]).
__device__ __forceinline__ void normal_pair(uint64_t seed, int64_t id, int64_t step, int sub, int draw, double& z0,
                                            double& z1) {
  uint32_t c[4] = {(uint32_t)id, (uint32_t)((uint64_t)id >> 32), (uint32_t)step,
                   (uint32_t)(sub * 2 + draw)};
  philox4x32_10(c, (uint32_t)seed, (uint32_t)(seed >> 32));
  const double inv53 = 1.0 / 9007199254740992.0;  // 2^-53
  const double u1 = ((double)(((uint64_t)(c[0] >> 5) << 26) | (c[1] >> 6)) + 1.0) * inv53;
  const double u2 = (double)(((uint64_t)(c[2] >> 5) << 26) | (c[3] >> 6)) * inv53;
  const double r = sqrt(-2.0 * log(u1));
  double sv, cv;
  sincospi(2.0 * u2, &sv, &cv);
  z0 = r * cv;
  z1 = r * sv;
}

// Periodic wrap into [0, L) (a tiny negative x would round to L itself).
__device__ __forceinline__ double wrap(double x, int L) {
  x = fmod(x, (double)L);
  if (x < 0.0) x += L;
  return x >= L ? x - L : x;
}

// Trilinear interpolation of the velocity snapshot at a wrapped position.
__device__ __forceinline__ void interp(const TracerDesc& T, double x, double y, double z, double v[3]) {
  const double fx = floor(x), fy = floor(y), fz = floor(z);
  const double ax = x - fx, ay = y - fy, az = z - fz;
  const int x0 = (int)fx % T.nx, y0 = (int)fy % T.ny, z0 = (int)fz % T.nz;
  const int x1 = (x0 + 1) % T.nx, y1 = (y0 + 1) % T.ny, z1 = (z0 + 1) % T.nz;
  const int64_t sy = T.nx, sz = (int64_t)T.nx * T.ny;
  const int64_t idx[8] = {x0 + y0 * sy + z0 * sz, x1 + y0 * sy + z0 * sz, x0 + y1 * sy + z0 * sz,
                          x1 + y1 * sy + z0 * sz, x0 + y0 * sy + z1 * sz, x1 + y0 * sy + z1 * sz,
                          x0 + y1 * sy + z1 * sz, x1 + y1 * sy + z1 * sz};
  const double w[8] = {(1 - ax) * (1 - ay) * (1 - az), ax * (1 - ay) * (1 - az), (1 - ax) * ay * (1 - az),
                       ax * ay * (1 - az),             (1 - ax) * (1 - ay) * az, ax * (1 - ay) * az,
                       (1 - ax) * ay * az,             ax * ay * az};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double s = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) s += w[q] * T.u[a][idx[q]];
    v[a] = s;
  }
}

// The same interpolation (identical velocity values) and its gradient
// J[a][b] = d u_a / d x_b, piecewise constant derivative weights of the
// trilinear interpolant.
__device__ __forceinline__ void interp_grad(const TracerDesc& T, double x, double y, double z, double v[3],
                                            double J[3][3]) {
  const double fx = floor(x), fy = floor(y), fz = floor(z);
  const double ax = x - fx, ay = y - fy, az = z - fz;
  const int x0 = (int)fx % T.nx, y0 = (int)fy % T.ny, z0 = (int)fz % T.nz;
  const int x1 = (x0 + 1) % T.nx, y1 = (y0 + 1) % T.ny, z1 = (z0 + 1) % T.nz;
  const int64_t sy = T.nx, sz = (int64_t)T.nx * T.ny;
  const int64_t idx[8] = {x0 + y0 * sy + z0 * sz, x1 + y0 * sy + z0 * sz, x0 + y1 * sy + z0 * sz,
                          x1 + y1 * sy + z0 * sz, x0 + y0 * sy + z1 * sz, x1 + y0 * sy + z1 * sz,
                          x0 + y1 * sy + z1 * sz, x1 + y1 * sy + z1 * sz};
  const double w[8] = {(1 - ax) * (1 - ay) * (1 - az), ax * (1 - ay) * (1 - az), (1 - ax) * ay * (1 - az),
                       ax * ay * (1 - az),             (1 - ax) * (1 - ay) * az, ax * (1 - ay) * az,
                       (1 - ax) * ay * az,             ax * ay * az};
  // corner q = bx + 2 by + 4 bz: d/dx of its weight is (2 bx - 1) wy wz, ...
  const double wy[2] = {1 - ay, ay}, wz[2] = {1 - az, az}, wx[2] = {1 - ax, ax};
#pragma unroll
  for (int a = 0; a < 3; ++a) {
    double s = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      const int bx = q & 1, by = (q >> 1) & 1, bz = q >> 2;
      const double uq = T.u[a][idx[q]];
      s += w[q] * uq;
      gx += (bx ? 1.0 : -1.0) * wy[by] * wz[bz] * uq;
      gy += (by ? 1.0 : -1.0) * wx[bx] * wz[bz] * uq;
      gz += (bz ? 1.0 : -1.0) * wx[bx] * wy[by] * uq;
    }
    v[a] = s;
    J[a][0] = gx;
    J[a][1] = gy;
    J[a][2] = gz;
  }
}

__device__ __forceinline__ int64_t nearest_node(const TracerDesc& T, double x, double y, double z) {
  const int ix = (int)floor(x + 0.5) % T.nx, iy = (int)floor(y + 0.5) % T.ny, iz = (int)floor(z + 0.5) % T.nz;
  return ix + (int64_t)T.nx * (iy + (int64_t)T.ny * iz);
}

__device__ __forceinline__ bool blocked(const TracerDesc& T, double x, double y, double z) {
  const int ix = (int)floor(x + 0.5) % T.nx, iy = (int)floor(y + 0.5) % T.ny, iz = (int)floor(z + 0.5) % T.nz;
  return T.solid[ix + (int64_t)T.nx * (iy + (int64_t)T.ny * iz)] != 0;
}

// One lattice step of every tracer (step = the tracer step counter). With
// stretching, each block leaves its NSTR partial sums in T.part (fixed-order
// tree: deterministic).
__global__ void __launch_bounds__(TRC) k_tracers(TracerDesc T, int64_t step) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  double acc[NSTR] = {0, 0, 0, 0, 0, 0, 0, 0};
  if (p < T.n) {
    double x = T.pos[p], y = T.pos[T.n + p], z = T.pos[2 * T.n + p];
    const double dm = T.dm[p];
    const int64_t id = T.id[p];
    const double dt = 1.0 / T.substeps;
    const double kick = dm > 0.0 ? sqrt(2.0 * dm * dt) : 0.0;
    double rh[3] = {0, 0, 0}, lr = 0.0;
    if (T.stretch) {
      rh[0] = T.rho_hat[p];
      rh[1] = T.rho_hat[T.n + p];
      rh[2] = T.rho_hat[2 * T.n + p];
      lr = T.log_rho[p];
    }
    bool active = true;
    double lam = 0.0, lam_w = 0.0, lam_nw = 0.0, cnt_w = 0.0, cnt_nw = 0.0;
    for (int s = 0; s < T.substeps; ++s) {
      double k1[3], J[3][3], nx, ny, nz;
      if (T.stretch) interp_grad(T, x, y, z, k1, J);
      else interp(T, x, y, z, k1);
      if (T.order == 1) {
        nx = x + dt * k1[0];
        ny = y + dt * k1[1];
        nz = z + dt * k1[2];
      } else {
        double k2[3];
        interp(T, wrap(x + dt * k1[0], T.nx), wrap(y + dt * k1[1], T.ny), wrap(z + dt * k1[2], T.nz), k2);
        nx = x + 0.5 * dt * (k1[0] + k2[0]);
        ny = y + 0.5 * dt * (k1[1] + k2[1]);
        nz = z + 0.5 * dt * (k1[2] + k2[2]);
      }
      if (kick > 0.0) {
        double g0, g1, g2, g3;
        normal_pair(T.seed, id, step, s, 0, g0, g1);
        nx += kick * g0;
        ny += kick * g1;
        if (T.nz > 1) {
          normal_pair(T.seed, id, step, s, 1, g2, g3);
          nz += kick * g2;
        }
      }
      nx = wrap(nx, T.nx);
      ny = wrap(ny, T.ny);
      nz = T.nz > 1 ? wrap(nz, T.nz) : z;  // a 2-D lattice: no motion along z
      if (blocked(T, nx, ny, nz)) {
        active = false;
        continue;
      }
      if (T.stretch) {
        double jr[3];
#pragma unroll
        for (int i = 0; i < 3; ++i) jr[i] = J[i][0] * rh[0] + J[i][1] * rh[1] + J[i][2] * rh[2];
        const double ls = rh[0] * jr[0] + rh[1] * jr[1] + rh[2] * jr[2];
        lam += ls;
        if (T.cgrid) {
          const double cv = T.cgrid[nearest_node(T, x, y, z)];
          if (cv < 0.5) {
            lam_w += ls;
            cnt_w += 1.0;
          } else if (cv >= 0.5) {  // a NaN (no order parameter given) is neither
            lam_nw += ls;
            cnt_nw += 1.0;
          }
        }
        const double r0 = rh[0] + dt * jr[0], r1 = rh[1] + dt * jr[1], r2 = rh[2] + dt * jr[2];
        const double g = sqrt(r0 * r0 + r1 * r1 + r2 * r2);
        lr += log(g);
        rh[0] = r0 / g;
        rh[1] = r1 / g;
        rh[2] = r2 / g;
      }
      x = nx;
      y = ny;
      z = nz;
    }
    T.pos[p] = x;
    T.pos[T.n + p] = y;
    T.pos[2 * T.n + p] = z;
    double v[3];
    interp(T, x, y, z, v);
    T.vel[p] = v[0];
    T.vel[T.n + p] = v[1];
    T.vel[2 * T.n + p] = v[2];
    if (T.stretch) {
      T.rho_hat[p] = rh[0];
      T.rho_hat[T.n + p] = rh[1];
      T.rho_hat[2 * T.n + p] = rh[2];
      T.log_rho[p] = lr;
      if (active) {
        acc[0] = 1.0;
        acc[1] = lam;
        acc[2] = lam_w;
        acc[3] = cnt_w;
        acc[4] = lam_nw;
        acc[5] = cnt_nw;
      }
      acc[6] = lr;
      acc[7] = lr * lr;
    }
  }
  if (!T.stretch) return;  // uniform over the launch
  __shared__ double red[NSTR][TRC];
#pragma unroll
  for (int q = 0; q < NSTR; ++q) red[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int h = TRC / 2; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int q = 0; q < NSTR; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x < NSTR) T.part[(int64_t)blockIdx.x * NSTR + threadIdx.x] = red[threadIdx.x][0];
}

// The step's row of the stretching time series from the blocks' partials
// (each thread a fixed strided subset, then a fixed tree), into slot
// row % cap of the row ring.
__global__ void __launch_bounds__(256) k_stretch_row(const double* __restrict__ part, int nblocks, int substeps,
                                                     int64_t n, int64_t row, double* __restrict__ ring, int cap) {
  __shared__ double red[NSTR][256];
  double acc[NSTR] = {0, 0, 0, 0, 0, 0, 0, 0};
  for (int b = threadIdx.x; b < nblocks; b += 256)
#pragma unroll
    for (int q = 0; q < NSTR; ++q) acc[q] += part[(int64_t)b * NSTR + q];
#pragma unroll
  for (int q = 0; q < NSTR; ++q) red[q][threadIdx.x] = acc[q];
  __syncthreads();
  for (int h = 128; h > 0; h >>= 1) {
    if ((int)threadIdx.x < h)
#pragma unroll
      for (int q = 0; q < NSTR; ++q) red[q][threadIdx.x] += red[q][threadIdx.x + h];
    __syncthreads();
  }
  if (threadIdx.x == 0) {
    const double nact = red[0][0], S = (double)substeps, nan = __longlong_as_double(0x7ff8000000000000ll);
    const double mean = red[6][0] / (double)n;
    double* r = ring + (row % cap) * NROW;
    r[0] = (double)row;
    r[1] = nact > 0.0 ? red[1][0] / (nact * S) : nan;
    r[2] = mean;
    r[3] = red[7][0] / (double)n - mean * mean;
    r[4] = nact;
    r[5] = red[3][0] > 0.0 ? red[2][0] / red[3][0] : nan;
    r[6] = red[5][0] > 0.0 ? red[4][0] / red[5][0] : nan;
    r[7] = red[3][0] / S;
    r[8] = red[5][0] / S;
  }
}

// Isotropic initial orientations: three standard normals per tracer from
// the Philox stream of `seed` (counter: tracer id, step 2^32 - 1, draws 0, 1,
// a step number the advance never reaches), normalised; log_rho = 0.
__global__ void k_stretch_init(TracerDesc T, uint64_t seed) {
  const int64_t p = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= T.n) return;
  double a, b, c, d;
  normal_pair(seed, T.id[p], (int64_t)0xFFFFFFFFll, 0, 0, a, b);
  normal_pair(seed, T.id[p], (int64_t)0xFFFFFFFFll, 0, 1, c, d);
  const double g = sqrt(a * a + b * b + c * c);
  T.rho_hat[p] = a / g;
  T.rho_hat[T.n + p] = b / g;
  T.rho_hat[2 * T.n + p] = c / g;
  T.log_rho[p] = 0.0;
}

}  // namespace fe
