// B200 (sm_100a) kernels of the Lee–Liu D3Q19 step.
//
// One step is four brick-parallel passes, separated by the grid-wide
// dependencies of the scheme (reference MultiPhaseGPU::step,
// multiphase_gpu.cuh:522-631):
//   P1 k_moments  pull-stream h,g (19+19 loads), write c, p, j; M,W partials
//                 of the order-parameter mass (and, last block, lambda)
//   P2 k_cfield   c stencil (grad_cd, Laplacian + wetting BC) -> mu, p
//                 (velocity/pressure correction)
//   P3 k_lapmu    mu stencil -> Laplacian of mu
//   P4 k_collide  c, p stencils to distance 2, lap(mu) to distance 1, pull g:
//                 equilibria + Guo force + BGK/MRT relaxation, write h, g
// Every CTA owns one brick: it stages the site indices of the brick plus a
// halo into shared memory (from the per-brick occupancy words), stages the
// stencil fields into shared memory tiles, and then runs one thread per fluid
// site of the brick. All stencil case logic (central / one-sided / biased,
// halfway bounce-back) is derived from tile occupancy, so no per-site tables
// are read from HBM.
//
// Streaming is pull, fused into P1 and P4: the post-collision value f*_k at
// x - e_k moves to site x, or f*_opp(k)(x) when x - e_k is solid (halfway
// bounce-back). The state between steps is therefore post-collision; uploads
// and downloads apply the (bijective) pull permutation.
#pragma once
#include <cuda_fp16.h>
#include <cuda_bf16.h>
#include <cstdint>

#include "d3q19.hpp"
#include "layout.hpp"
#include "mrt.hpp"

namespace fe {

// ---------------------------------------------------------------------------
// storage traits
// ---------------------------------------------------------------------------
struct StF64 {
  using pop = double;
  using fld = double;
  using real = double;
  static constexpr bool shifted = false;
};
struct StF32 {
  using pop = float;
  using fld = float;
  using real = float;
  static constexpr bool shifted = false;
};
// FP16 / BF16: population k stored as (f_k - w_k * ref) * scale, ref = c_ref
// for h and p_ref for g; arithmetic in FP32.
struct StF16S {
  using pop = __half;
  using fld = float;
  using real = float;
  static constexpr bool shifted = true;
};
struct StBF16S {
  using pop = __nv_bfloat16;
  using fld = float;
  using real = float;
  static constexpr bool shifted = true;
};

template <class T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <class T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

// AoSoA population index of (site i, direction k)
__device__ __forceinline__ int64_t pidx(int64_t i, int k) {
  return (i >> 5) * (int64_t)(Q * AOSOA) + k * AOSOA + (i & (AOSOA - 1));
}

// Shift parameters for the 16-bit formats (unused otherwise).
struct Shift {
  float ref, inv_scale, scale;
};

template <class S>
__device__ __forceinline__ typename S::real ld_pop(const typename S::pop* __restrict__ a, int64_t idx, int k,
                                                   const Shift& sh) {
  if constexpr (S::shifted) {
    return to_f(a[idx]) * sh.inv_scale + weight<float>(k) * sh.ref;
  } else {
    return a[idx];
  }
}
template <class S>
__device__ __forceinline__ void st_pop(typename S::pop* __restrict__ a, int64_t idx, int k,
                                       typename S::real v, const Shift& sh) {
  if constexpr (S::shifted) {
    a[idx] = from_f<typename S::pop>((v - weight<float>(k) * sh.ref) * sh.scale);
  } else {
    a[idx] = v;
  }
}

// ---------------------------------------------------------------------------
// brick tile staging
// ---------------------------------------------------------------------------
constexpr int MAX_SEG = 4;      // distinct bricks a tile can touch per axis
constexpr int MAX_T = 24;       // tile extent per axis
constexpr int MAX_SLOTS = 512;  // nodes per brick
constexpr int CTA = 256;

struct TileShared {
  uint8_t seg[3][MAX_T];        // tile coordinate -> neighbour-brick segment
  uint8_t loc[3][MAX_T];        // tile coordinate -> local coordinate in that brick
  int32_t ucoord[3][MAX_SEG];   // segment -> brick coordinate
  int32_t nseg[3];
  int32_t T[3];                 // tile extents
  int32_t org[3];               // tile position of the brick's local (0,0,0)
  int32_t nbr[MAX_SEG * MAX_SEG * MAX_SEG];
  int32_t off1[Q], off2[Q];     // tile offsets of +e_k and +2 e_k
  int32_t first, cnt, ntile;
  uint16_t slot_of[MAX_SLOTS];
  double red[CTA / 32][6];      // block reductions
  float ff;                     // forcing factor of this step
  double lambda;                // mass-correction lambda of this step
  int last;
};

__device__ __forceinline__ int mod_pos(int a, int n) {
  int r = a % n;
  return r < 0 ? r + n : r;
}

// Build the axis tables, neighbour-brick ids and the brick's slot list.
// H = halo depth (1 or 2). Axes of extent 1 get no halo and no offsets.
template <int H>
__device__ void tile_setup(const LatDesc& D, int brick, TileShared& ts) {
  const int tid = threadIdx.x;
  if (tid < 3) {
    const int a = tid;
    const int N = a == 0 ? D.nx : (a == 1 ? D.ny : D.nz);
    const int lb = a == 0 ? D.lbx : (a == 1 ? D.lby : D.lbz);
    const int B = 1 << lb;
    const int h = N > 1 ? H : 0;
    const int T = B + 2 * h;
    const int origin = D.brick_xyz[brick * 3 + a] * B - h;
    // A tile spans B + 2h <= 20 consecutive positions (mod N), which touch at
    // most 4 distinct bricks per axis (two partial bricks across the wrap);
    // the bound check below only guards against a layout the host never builds.
    int nu = 0;
    for (int t = 0; t < T && t < MAX_T; ++t) {
      const int X = mod_pos(origin + t, N);
      const int bc = X >> lb;
      int s = 0;
      while (s < nu && ts.ucoord[a][s] != bc) ++s;
      if (s == nu) {
        if (nu == MAX_SEG) { atomicOr(&D.ctl->status, 2); s = 0; }
        else { ts.ucoord[a][nu] = bc; ++nu; }
      }
      ts.seg[a][t] = (uint8_t)s;
      ts.loc[a][t] = (uint8_t)(X & (B - 1));
    }
    ts.nseg[a] = nu;
    ts.T[a] = T;
    ts.org[a] = h;
  }
  __syncthreads();
  const int nsx = ts.nseg[0], nsy = ts.nseg[1], nsz = ts.nseg[2];
  for (int q = tid; q < nsx * nsy * nsz; q += blockDim.x) {
    const int sx = q % nsx, sy = (q / nsx) % nsy, sz = q / (nsx * nsy);
    const int ux = ts.ucoord[0][sx], uy = ts.ucoord[1][sy], uz = ts.ucoord[2][sz];
    ts.nbr[sx + MAX_SEG * (sy + MAX_SEG * sz)] = D.brick_grid[((int64_t)uz * D.nby + uy) * D.nbx + ux];
  }
  if (tid < Q) {
    const int k = tid;
    const int TX = ts.T[0], TY = ts.T[1];
    const int ex = D.nx > 1 ? lat_cx(k) : 0, ey = D.ny > 1 ? lat_cy(k) : 0, ez = D.nz > 1 ? lat_cz(k) : 0;
    ts.off1[k] = ex + TX * (ey + TY * ez);
    ts.off2[k] = 2 * ts.off1[k];
  }
  // own slot list
  const int W = D.words, C = W * 64;
  const int first = D.base[(int64_t)brick * W];
  for (int s = tid; s < C; s += blockDim.x) {
    const int w = s >> 6, b = s & 63;
    const uint64_t m = D.mask[(int64_t)brick * W + w];
    if ((m >> b) & 1ull) {
      const int r = D.base[(int64_t)brick * W + w] - first + __popcll(m & ((1ull << b) - 1ull));
      ts.slot_of[r] = (uint16_t)s;
    }
  }
  if (tid == 0) {
    const uint64_t ml = D.mask[(int64_t)brick * W + W - 1];
    ts.first = first;
    ts.cnt = D.base[(int64_t)brick * W + W - 1] - first + __popcll(ml);
    ts.ntile = ts.T[0] * ts.T[1] * ts.T[2];
  }
  __syncthreads();
}

// Site index of every tile position (-1 = solid or outside any stored brick).
__device__ __forceinline__ int tile_site(const LatDesc& D, const TileShared& ts, int t) {
  const int TX = ts.T[0], TY = ts.T[1];
  const int tx = t % TX, r = t / TX, ty = r % TY, tz = r / TY;
  const int id = ts.nbr[ts.seg[0][tx] + MAX_SEG * (ts.seg[1][ty] + MAX_SEG * ts.seg[2][tz])];
  if (id < 0) return -1;
  const int slot = ts.loc[0][tx] | (ts.loc[1][ty] << D.lbx) | (ts.loc[2][tz] << (D.lbx + D.lby));
  const int w = slot >> 6, b = slot & 63;
  const uint64_t m = __ldg(&D.mask[(int64_t)id * D.words + w]);
  if (!((m >> b) & 1ull)) return -1;
  return __ldg(&D.base[(int64_t)id * D.words + w]) + __popcll(m & ((1ull << b) - 1ull));
}

// tile position of the brick slot s
__device__ __forceinline__ int slot_pos(const LatDesc& D, const TileShared& ts, int s) {
  const int lx = s & ((1 << D.lbx) - 1);
  const int ly = (s >> D.lbx) & ((1 << D.lby) - 1);
  const int lz = s >> (D.lbx + D.lby);
  return (lx + ts.org[0]) + ts.T[0] * ((ly + ts.org[1]) + ts.T[1] * (lz + ts.org[2]));
}

// forcing_factor_at (reference felbm_gpu_main.cu:587-594)
__device__ __forceinline__ double forcing_factor_dev(const DevPrm& P, const Ctl& C) {
  if (!C.ff_auto) return C.ff_manual;
  const double PI = 3.14159265358979323846;
  if (P.forcing_timedep == 1) return sin(2.0 * PI * double(C.t) / P.forcing_period);
  if (P.forcing_timedep == 2) {
    const double x = sin(2.0 * PI * double(C.t) / P.forcing_period);
    return (x < 0) ? -1.0 : ((x > 0) ? 1.0 : 0.0);
  }
  return 1.0;
}

// Block sum of NV doubles into ts.red[0][*] (thread 0 holds the result).
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], TileShared& ts, bool is_max_last = false) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
    const bool mx = is_max_last && q == NV - 1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = mx ? fmax(x, y) : x + y;
    }
    if (lane == 0) ts.red[wid][q] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = blockDim.x >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double x = ts.red[0][q];
      const bool mx = is_max_last && q == NV - 1;
      for (int w = 1; w < nw; ++w) x = mx ? fmax(x, ts.red[w][q]) : x + ts.red[w][q];
      v[q] = x;
    }
  }
}

// Deterministic sum over `count` partial records of stride `stride` (one
// CTA): each thread sums a fixed strided subset, then a fixed tree.
template <int NV>
__device__ void sum_partials(const double* __restrict__ part, int count, int stride, double (&out)[NV],
                             TileShared& ts, bool is_max_last = false) {
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int r = threadIdx.x; r < count; r += blockDim.x) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const double x = __ldcg(&part[(int64_t)r * stride + q]);
      acc[q] = (is_max_last && q == NV - 1) ? fmax(acc[q], x) : acc[q] + x;
    }
  }
  block_sum<NV>(acc, ts, is_max_last);
#pragma unroll
  for (int q = 0; q < NV; ++q) out[q] = acc[q];
}

// Returns true in every thread of the block that finished last (per lattice).
__device__ __forceinline__ bool last_block(unsigned int* counter, unsigned int total, TileShared& ts) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int prev = atomicAdd(counter, 1u);
    ts.last = (prev == total - 1) ? 1 : 0;
  }
  __syncthreads();
  return ts.last != 0;
}

// ---------------------------------------------------------------------------
// P1: pull streaming + moments (reference k_moments, device_engine.cuh:116-135,
// with the streaming of the previous step's k_stream_gather, :882-889, fused
// in as a pull, and k_mass_weight, :1109-1126, fused as block partials).
// ---------------------------------------------------------------------------
template <class S>
__global__ void __launch_bounds__(CTA) k_moments(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                  int parity) {
  using R = typename S::real;
  using P = typename S::pop;
  using F = typename S::fld;
  __shared__ TileShared ts;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int brick = wk.y;
  tile_setup<1>(D, brick, ts);
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);
  for (int t = threadIdx.x; t < ts.ntile; t += blockDim.x) s_idx[t] = tile_site(D, ts, t);
  __syncthreads();
  const P* __restrict__ hin = static_cast<const P*>(D.pop[parity][0]);
  const P* __restrict__ gin = static_cast<const P*>(D.pop[parity][1]);
  F* __restrict__ fc = static_cast<F*>(D.c);
  F* __restrict__ fp = static_cast<F*>(D.p);
  F* __restrict__ fjx = static_cast<F*>(D.jx);
  F* __restrict__ fjy = static_cast<F*>(D.jy);
  F* __restrict__ fjz = static_cast<F*>(D.jz);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  const Shift shg{(float)D.prm.p_ref, (float)(1.0 / D.prm.g_scale), (float)D.prm.g_scale};
  double acc[2] = {0.0, 0.0};
  for (int r = threadIdx.x; r < ts.cnt; r += blockDim.x) {
    const int s = ts.slot_of[r];
    const int64_t i = ts.first + r;
    const int pos = slot_pos(D, ts, s);
    R c = 0, p = 0, jx = 0, jy = 0, jz = 0;
    double cd = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      const int up = s_idx[pos - ts.off1[k]];
      const int64_t a = up >= 0 ? pidx(up, k) : pidx(i, lat_opp(k));
      const int kk = up >= 0 ? k : lat_opp(k);
      const R hv = ld_pop<S>(hin, a, kk, shh);
      const R gv = ld_pop<S>(gin, a, kk, shg);
      c += hv;
      cd += (double)hv;
      p += gv;
      if (lat_cx(k)) jx += R(lat_cx(k)) * gv;
      if (lat_cy(k)) jy += R(lat_cy(k)) * gv;
      if (lat_cz(k)) jz += R(lat_cz(k)) * gv;
    }
    fc[i] = (F)c;
    fp[i] = (F)p;
    fjx[i] = (F)jx;
    fjy[i] = (F)jy;
    fjz[i] = (F)jz;
    double phi = cd * (1.0 - cd);
    if (phi < 0.0) phi = 0.0;
    acc[0] += cd;
    acc[1] += phi;
  }
  if (!D.prm.correct_mass) return;
  block_sum<2>(acc, ts);
  if (threadIdx.x == 0) {
    D.part1[(int64_t)brick * 2 + 0] = acc[0];
    D.part1[(int64_t)brick * 2 + 1] = acc[1];
  }
  if (!last_block(&D.ctl->count1, (unsigned)D.nbricks, ts)) return;
  double tot[2];
  sum_partials<2>(D.part1, D.nbricks, 2, tot, ts);
  if (threadIdx.x == 0) {
    Ctl* C = D.ctl;
    C->M = tot[0];
    C->W = tot[1];
    double lam = 0.0;
    if (C->pending) {
      const double drift = tot[0] - C->target_mass;
      C->drift = drift;
      if (tot[1] > 0.0 && drift != 0.0) lam = drift / tot[1];
    }
    C->lambda = lam;
    C->count1 = 0;
  }
}

// corrected order parameter c' = c - lambda * max(c(1-c), 0) (the reference's
// k_inject_mass, device_engine.cuh:1128-1139, applied to c instead of h; h is
// never read by the collision, so this is the same state)
template <class R>
__device__ __forceinline__ R corr_c(R c, double lambda) {
  if (lambda == 0.0) return c;
  const double cd = (double)c;
  const double phi = cd * (1.0 - cd);
  return phi > 0.0 ? (R)(cd - lambda * phi) : c;
}

template <class S>
__device__ __forceinline__ void load_step_scalars(const LatDesc& D, TileShared& ts) {
  if (threadIdx.x == 0) {
    const Ctl& C = *D.ctl;
    ts.ff = (float)forcing_factor_dev(D.prm, C);
    ts.lambda = C.lambda;
  }
}

// Stage c' (and the site indices) of the tile; returns nothing.
template <class S>
__device__ __forceinline__ void stage_field(const LatDesc& D, const TileShared& ts, const int32_t* s_idx,
                                            typename S::real* s_v, const typename S::fld* __restrict__ f,
                                            bool correct, double lambda) {
  using R = typename S::real;
  for (int t = threadIdx.x; t < ts.ntile; t += blockDim.x) {
    const int j = s_idx[t];
    R v = R(0);
    if (j >= 0) {
      v = (R)f[j];
      if (correct) v = corr_c<R>(v, lambda);
    }
    s_v[t] = v;
  }
}

// ---------------------------------------------------------------------------
// P2: grad_cd(c), Laplacian(c) with the wetting term, mu, velocity/pressure
// correction (reference k_grad_cd_mf :897-913, k_pack_lap_c :159-165,
// k_lap_mf :996-1010, k_mu_axpy :149-153, k_vel_press_corr :177-196; the
// near-wall cases of the table builders multiphase_gpu.cuh:93-193).
// OUT != 0: also write c, rho, u, p, mu in the reference site order (download).
// ---------------------------------------------------------------------------
struct FieldOut {
  double *rho, *c, *ux, *uy, *uz, *p, *mu;
};

template <class S, int OUT>
__global__ void __launch_bounds__(CTA) k_cfield(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                 FieldOut out) {
  using R = typename S::real;
  using F = typename S::fld;
  __shared__ TileShared ts;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  tile_setup<1>(D, wk.y, ts);
  load_step_scalars<S>(D, ts);
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);
  for (int t = threadIdx.x; t < ts.ntile; t += blockDim.x) s_idx[t] = tile_site(D, ts, t);
  __syncthreads();
  R* s_c = reinterpret_cast<R*>(dsm + ((ts.ntile * 4 + 15) & ~15));
  stage_field<S>(D, ts, s_idx, s_c, static_cast<const F*>(D.c), true, ts.lambda);
  __syncthreads();
  const DevPrm& Pm = D.prm;
  const R alpha = R(ALPHA), cs2 = R(CS2);
  const R rho1 = (R)Pm.rho1, drho = (R)Pm.drho, kappa = (R)Pm.kappa, four_beta = (R)Pm.four_beta;
  const R bnd_coeff = (R)Pm.bnd_coeff, ff = (R)ts.ff;
  const bool hbb = Pm.hbb != 0;
  const F* __restrict__ fjx = static_cast<const F*>(D.jx);
  const F* __restrict__ fjy = static_cast<const F*>(D.jy);
  const F* __restrict__ fjz = static_cast<const F*>(D.jz);
  F* __restrict__ fp = static_cast<F*>(D.p);
  F* __restrict__ fmu = static_cast<F*>(D.mu);
  for (int r = threadIdx.x; r < ts.cnt; r += blockDim.x) {
    const int s = ts.slot_of[r];
    const int64_t i = ts.first + r;
    const int pos = slot_pos(D, ts, s);
    const R c0 = s_c[pos];
    const R bnd = bnd_coeff * c0 * (R(1) - c0);
    R gx = 0, gy = 0, gz = 0, lap = 0;
#pragma unroll
    for (int k = 1; k < Q; ++k) {
      const int o = ts.off1[k];
      const bool b1 = s_idx[pos - o] >= 0, f1 = s_idx[pos + o] >= 0;
      const R cm = s_c[pos - o], cp = s_c[pos + o];
      R cdv = 0;
      if (b1 && f1) cdv = R(0.5) * (cp - cm);
      else if (hbb && b1) cdv = R(0.5) * (c0 - cm);
      else if (hbb && f1) cdv = R(0.5) * (cp - c0);
      const R aw = alpha * weight<R>(k);
      if (lat_cx(k)) gx += aw * R(lat_cx(k)) * cdv;
      if (lat_cy(k)) gy += aw * R(lat_cy(k)) * cdv;
      if (lat_cz(k)) gz += aw * R(lat_cz(k)) * cdv;
      R lv = 0;
      if (b1 && f1) lv = cm - R(2) * c0 + cp;
      else if (b1 || f1) {
        const R f1v = b1 ? cm : cp;
        lv = hbb ? (f1v - c0 - bnd) : (R(2) * f1v - R(2) * c0 - R(2) * bnd);
      }
      lap += aw * lv;
    }
    uint8_t flag = 0;
    if (Pm.open_bnd) flag = D.bcflag[i];
    const R cm_ = (flag & BC_SITE) ? (R) static_cast<const F*>(D.c_raw_bc)[i] : c0;
    const R rho = rho1 + drho * c0;
    const R mu = four_beta * (cm_ * (R(1) - cm_)) * (R(0.5) - cm_) + (-kappa * lap);
    R ux, uy, uz;
    F* ubc = static_cast<F*>(D.u_bc);
    if (flag & BC_SITE) {
      ux = (R)ubc[i]; uy = (R)ubc[D.n + i]; uz = (R)ubc[2 * D.n + i];
    } else {
      const R inv = R(1) / (cs2 * rho);
      ux = (R)fjx[i] * inv; uy = (R)fjy[i] * inv; uz = (R)fjz[i] * inv;
    }
    R p = (R)fp[i];
    if (!(flag & BC_PROC)) {
      const R mor = mu / rho;
      ux = ux + R(0.5) * ((R)Pm.gx + (R)Pm.fx * ff / rho + mor * gx);
      uy = uy + R(0.5) * ((R)Pm.gy + (R)Pm.fy * ff / rho + mor * gy);
      uz = uz + R(0.5) * ((R)Pm.gz + (R)Pm.fz * ff / rho + mor * gz);
      const R u_dot_drho = drho * (ux * gx + uy * gy + uz * gz);
      p += R(0.5) * u_dot_drho * cs2;
      fp[i] = (F)p;
    }
    fmu[i] = (F)mu;
    if (flag & BC_SITE) { ubc[i] = (F)ux; ubc[D.n + i] = (F)uy; ubc[2 * D.n + i] = (F)uz; }
    if (OUT) {
      const int64_t q = D.ref_of[i];
      out.c[q] = (double)c0;
      out.rho[q] = (double)rho;
      out.ux[q] = (double)ux;
      out.uy[q] = (double)uy;
      out.uz[q] = (double)uz;
      out.p[q] = (double)p;
      out.mu[q] = (double)mu;
    }
  }
}

// ---------------------------------------------------------------------------
// P3: Laplacian of mu, boundary half zero (reference k_pack_lap_zero :168-173
// + k_lap_mf).
// ---------------------------------------------------------------------------
template <class S>
__global__ void __launch_bounds__(CTA) k_lapmu(const LatDesc* __restrict__ descs, const int2* __restrict__ work) {
  using R = typename S::real;
  using F = typename S::fld;
  __shared__ TileShared ts;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  tile_setup<1>(D, wk.y, ts);
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);
  for (int t = threadIdx.x; t < ts.ntile; t += blockDim.x) s_idx[t] = tile_site(D, ts, t);
  __syncthreads();
  R* s_m = reinterpret_cast<R*>(dsm + ((ts.ntile * 4 + 15) & ~15));
  stage_field<S>(D, ts, s_idx, s_m, static_cast<const F*>(D.mu), false, 0.0);
  __syncthreads();
  const bool hbb = D.prm.hbb != 0;
  const R alpha = R(ALPHA);
  F* __restrict__ flm = static_cast<F*>(D.lapmu);
  for (int r = threadIdx.x; r < ts.cnt; r += blockDim.x) {
    const int s = ts.slot_of[r];
    const int64_t i = ts.first + r;
    const int pos = slot_pos(D, ts, s);
    const R m0 = s_m[pos];
    R lap = 0;
#pragma unroll
    for (int k = 1; k < Q; ++k) {
      const int o = ts.off1[k];
      const bool b1 = s_idx[pos - o] >= 0, f1 = s_idx[pos + o] >= 0;
      R lv = 0;
      if (b1 && f1) lv = s_m[pos - o] - R(2) * m0 + s_m[pos + o];
      else if (b1 || f1) {
        const R f1v = b1 ? s_m[pos - o] : s_m[pos + o];
        lv = hbb ? (f1v - m0) : (R(2) * f1v - R(2) * m0);
      }
      lap += alpha * weight<R>(k) * lv;
    }
    flm[i] = (F)lap;
  }
}

// ---------------------------------------------------------------------------
// P4: fused equilibria + Guo force + BGK/MRT collision (reference
// k_collide_fused_mrt :547-651 and k_collide_fused_bgk :459-545, with the
// directional helpers cd_dir_val/bd_dir_val/avg_dir_val :89-113 evaluated
// from the staged tiles, and the open-boundary overwrite of g,
// k_open_bnd/k_open_bnd_buf :761-798,826-846, folded in). The corrected
// velocity is rebuilt from the pulled g (same g as P1) instead of being
// stored. Writes post-collision h, g to the other buffer.
// ---------------------------------------------------------------------------
template <class R>
struct DirVals {
  R cdc, cdp, bdc, bdp;
};

template <class R>
__device__ __forceinline__ DirVals<R> dir_vals(const int32_t* s_idx, const R* s_c, const R* s_p, int pos, int o1,
                                               int o2, R c0, R p0, bool hbb) {
  const bool b1 = s_idx[pos - o1] >= 0, f1 = s_idx[pos + o1] >= 0;
  DirVals<R> v;
  // central-difference pair (multiphase_gpu.cuh:118-120)
  if (b1 && f1) { v.cdc = R(0.5) * (s_c[pos + o1] - s_c[pos - o1]); v.cdp = R(0.5) * (s_p[pos + o1] - s_p[pos - o1]); }
  else if (hbb && b1) { v.cdc = R(0.5) * (c0 - s_c[pos - o1]); v.cdp = R(0.5) * (p0 - s_p[pos - o1]); }
  else if (hbb && f1) { v.cdc = R(0.5) * (s_c[pos + o1] - c0); v.cdp = R(0.5) * (s_p[pos + o1] - p0); }
  else { v.cdc = 0; v.cdp = 0; }
  // biased cases (multiphase_gpu.cuh:142-152, device_engine.cuh:96-107)
  if (f1) {
    const bool f2 = s_idx[pos + o2] >= 0;
    const R c1 = s_c[pos + o1], p1 = s_p[pos + o1];
    if (f2) {
      v.bdc = R(-1.5) * c0 + R(2.0) * c1 + R(-0.5) * s_c[pos + o2];
      v.bdp = R(-1.5) * p0 + R(2.0) * p1 + R(-0.5) * s_p[pos + o2];
    } else if (!hbb) {
      v.bdc = R(-2.0) * c0 + R(2.0) * c1;
      v.bdp = R(-2.0) * p0 + R(2.0) * p1;
    } else {
      v.bdc = R(-1.5) * c0 + R(1.5) * c1;
      v.bdp = R(-1.5) * p0 + R(1.5) * p1;
    }
  } else if (!hbb) {
    v.bdc = 0; v.bdp = 0;
    if (b1 && s_idx[pos - o2] >= 0) {
      v.bdc = R(-1.5) * c0 + R(2.0) * s_c[pos - o1] + R(-0.5) * s_c[pos - o2];
      v.bdp = R(-1.5) * p0 + R(2.0) * s_p[pos - o1] + R(-0.5) * s_p[pos - o2];
    }
  } else if (b1) {
    v.bdc = R(0.5) * c0 + R(-0.5) * s_c[pos - o1];
    v.bdp = R(0.5) * p0 + R(-0.5) * s_p[pos - o1];
  } else {
    v.bdc = 0; v.bdp = 0;
  }
  return v;
}

// M^-1 S M applied to x (S diagonal, conserved rows zero), with the moment
// matrix folded at compile time. srate[kind] = rate of that moment kind.
template <class R>
__device__ __forceinline__ void mrt_apply(R (&x)[Q], const R (&srate)[7]) {
  R m[Q];
#pragma unroll
  for (int j = 0; j < Q; ++j) {
    if (mrt_kind(j) == MK_CONS) { m[j] = R(0); continue; }
    R acc = R(0);
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      const int mk = mrt_M(j, k);
      if (mk == 1) acc += x[k];
      else if (mk == -1) acc -= x[k];
      else if (mk != 0) acc += R(mk) * x[k];
    }
    m[j] = acc * (srate[mrt_kind(j)] * (R(1) / R(mrt_norm2(j))));
  }
#pragma unroll
  for (int k = 0; k < Q; ++k) {
    R acc = R(0);
#pragma unroll
    for (int j = 0; j < Q; ++j) {
      if (mrt_kind(j) == MK_CONS) continue;
      const int mk = mrt_M(j, k);
      if (mk == 1) acc += m[j];
      else if (mk == -1) acc -= m[j];
      else if (mk != 0) acc += R(mk) * m[j];
    }
    x[k] = acc;
  }
}

template <class S, int MRT>
__global__ void __launch_bounds__(CTA) k_collide(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                  int parity) {
  using R = typename S::real;
  using P = typename S::pop;
  using F = typename S::fld;
  __shared__ TileShared ts;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int brick = wk.y;
  tile_setup<2>(D, brick, ts);
  load_step_scalars<S>(D, ts);
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);
  for (int t = threadIdx.x; t < ts.ntile; t += blockDim.x) s_idx[t] = tile_site(D, ts, t);
  __syncthreads();
  const int nt16 = (ts.ntile * 4 + 15) & ~15;
  const int ntr = (ts.ntile * (int)sizeof(R) + 15) & ~15;
  R* s_c = reinterpret_cast<R*>(dsm + nt16);
  R* s_p = reinterpret_cast<R*>(dsm + nt16 + ntr);
  R* s_l = reinterpret_cast<R*>(dsm + nt16 + 2 * ntr);
  stage_field<S>(D, ts, s_idx, s_c, static_cast<const F*>(D.c), true, ts.lambda);
  stage_field<S>(D, ts, s_idx, s_p, static_cast<const F*>(D.p), false, 0.0);
  stage_field<S>(D, ts, s_idx, s_l, static_cast<const F*>(D.lapmu), false, 0.0);
  __syncthreads();

  const DevPrm& Pm = D.prm;
  const bool hbb = Pm.hbb != 0;
  const R cs2 = R(CS2), alpha = R(ALPHA), beta_c = R(BETA), gamma_c = R(GAMMA);
  const R rho1 = (R)Pm.rho1, drho = (R)Pm.drho, mobility = (R)Pm.mobility;
  const R tau0 = (R)Pm.tau0, tau1 = (R)Pm.tau1, ffac = (R)ts.ff;
  const R gxa = (R)Pm.gx, gya = (R)Pm.gy, gza = (R)Pm.gz;
  const R fxa = (R)Pm.fx * ffac, fya = (R)Pm.fy * ffac, fza = (R)Pm.fz * ffac;
  const P* __restrict__ gin = static_cast<const P*>(D.pop[parity][1]);
  P* __restrict__ hout = static_cast<P*>(D.pop[parity ^ 1][0]);
  P* __restrict__ gout = static_cast<P*>(D.pop[parity ^ 1][1]);
  const F* __restrict__ fmu = static_cast<const F*>(D.mu);
  const Shift shh{(float)Pm.c_ref, (float)(1.0 / Pm.h_scale), (float)Pm.h_scale};
  const Shift shg{(float)Pm.p_ref, (float)(1.0 / Pm.g_scale), (float)Pm.g_scale};
  double st[6] = {0, 0, 0, 0, 0, 0};
  int bad = 0;

  for (int r = threadIdx.x; r < ts.cnt; r += blockDim.x) {
    const int s = ts.slot_of[r];
    const int64_t i = ts.first + r;
    const int pos = slot_pos(D, ts, s);
    const R c = s_c[pos], p = s_p[pos], lmu = s_l[pos];
    const R mu = (R)fmu[i];
    // pulled g (identical to what P1 read)
    R g[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      const int up = s_idx[pos - ts.off1[k]];
      const int64_t a = up >= 0 ? pidx(up, k) : pidx(i, lat_opp(k));
      g[k] = ld_pop<S>(gin, a, up >= 0 ? k : lat_opp(k), shg);
    }
    // gradients of c and p: central (eq) and biased (force) from the tiles
    R e_dcx = 0, e_dcy = 0, e_dcz = 0, e_dpx = 0, e_dpy = 0, e_dpz = 0;
    R b_dcx = 0, b_dcy = 0, b_dcz = 0, b_dpx = 0, b_dpy = 0, b_dpz = 0;
#pragma unroll
    for (int k = 1; k < Q; ++k) {
      const DirVals<R> v = dir_vals<R>(s_idx, s_c, s_p, pos, ts.off1[k], ts.off2[k], c, p, hbb);
      const R aw = alpha * weight<R>(k);
      if (lat_cx(k)) {
        const R e = aw * R(lat_cx(k));
        e_dcx += e * v.cdc; e_dpx += e * v.cdp; b_dcx += e * v.bdc; b_dpx += e * v.bdp;
      }
      if (lat_cy(k)) {
        const R e = aw * R(lat_cy(k));
        e_dcy += e * v.cdc; e_dpy += e * v.cdp; b_dcy += e * v.bdc; b_dpy += e * v.bdp;
      }
      if (lat_cz(k)) {
        const R e = aw * R(lat_cz(k));
        e_dcz += e * v.cdc; e_dpz += e * v.cdp; b_dcz += e * v.bdc; b_dpz += e * v.bdp;
      }
    }
    const R f_dcx = R(0.5) * (e_dcx + b_dcx), f_dcy = R(0.5) * (e_dcy + b_dcy), f_dcz = R(0.5) * (e_dcz + b_dcz);
    const R f_dpx = R(0.5) * (e_dpx + b_dpx), f_dpy = R(0.5) * (e_dpy + b_dpy), f_dpz = R(0.5) * (e_dpz + b_dpz);

    const uint8_t flag = Pm.open_bnd ? D.bcflag[i] : 0;
    const R rho = rho1 + drho * c;
    const R cm_ = (flag & BC_SITE) ? (R) static_cast<const F*>(D.c_raw_bc)[i] : c;
    // relaxation rate (reference k_moments :130-132)
    const R cpc = cm_ < R(0) ? R(0) : (cm_ > R(1) ? R(1) : cm_);
    const R tau = R(1) / (cpc / tau0 + (R(1) - cpc) / tau1);
    const R s0 = R(1) / (tau + R(0.5));
    // corrected velocity (k_moments + k_vel_press_corr)
    R ux, uy, uz;
    if (flag & BC_SITE) {
      const F* ubc = static_cast<const F*>(D.u_bc);
      ux = (R)ubc[i]; uy = (R)ubc[D.n + i]; uz = (R)ubc[2 * D.n + i];
    } else {
      R jx = 0, jy = 0, jz = 0;
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        if (lat_cx(k)) jx += R(lat_cx(k)) * g[k];
        if (lat_cy(k)) jy += R(lat_cy(k)) * g[k];
        if (lat_cz(k)) jz += R(lat_cz(k)) * g[k];
      }
      const R inv = R(1) / (cs2 * rho);
      const R mor = mu / rho;
      ux = jx * inv + R(0.5) * (gxa + fxa / rho + mor * e_dcx);
      uy = jy * inv + R(0.5) * (gya + fya / rho + mor * e_dcy);
      uz = jz * inv + R(0.5) * (gza + fza / rho + mor * e_dcz);
    }
    // open-boundary overwrite of g by the plain equilibrium (apply_open_bnd)
    if (flag & BC_G_OVER) {
      const int64_t sb = D.bcsrc[i];
      const F* ubc = static_cast<const F*>(D.u_bc);
      const R bux = (R)ubc[sb], buy = (R)ubc[D.n + sb], buz = (R)ubc[2 * D.n + sb];
      const R bp = (R) static_cast<const F*>(D.p)[sb];
      const R bc = (R) static_cast<const F*>(D.c)[sb];
      const R brho = rho1 + drho * bc;
      const R bu_sq = bux * bux + buy * buy + buz * buz;
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        const R uk = bux * R(lat_cx(k)) + buy * R(lat_cy(k)) + buz * R(lat_cz(k));
        const R u_term = uk * (alpha + beta_c * uk) - gamma_c * bu_sq;
        g[k] = weight<R>(k) * (bp + brho * cs2 * u_term);
      }
    }
    const R bfx = rho * gxa + fxa, bfy = rho * gya + fya, bfz = rho * gza + fza;
    const R u2 = ux * ux + uy * uy + uz * uz;
    st[0] += (double)ux; st[1] += (double)uy; st[2] += (double)uz; st[3] += (double)u2; st[4] += (double)c;
    st[5] = fmax(st[5], (double)u2);
    bad |= !(u2 < R(1e30));

    R x[Q];   // MRT: raw collision term eq_g - g;  BGK: unused
    R gpf[Q]; // g + force_g (MRT) or the new g (BGK)
    if (MRT) {
      const R drho_cs2 = drho * cs2, rho_cs2 = rho * cs2, c_over = c / rho_cs2;
      const R drcx = drho_cs2 * e_dcx, drcy = drho_cs2 * e_dcy, drcz = drho_cs2 * e_dcz;
      const R e_fgx = mu * e_dcx + bfx, e_fgy = mu * e_dcy + bfy, e_fgz = mu * e_dcz + bfz;
      const R e_fhx = e_dcx - c_over * (e_dpx - e_fgx), e_fhy = e_dcy - c_over * (e_dpy - e_fgy),
              e_fhz = e_dcz - c_over * (e_dpz - e_fgz);
      const R gamma_u_sq = gamma_c * u2;
      const R u_term_h = ux * e_fhx + uy * e_fhy + uz * e_fhz;
      const R u_force_g = ux * e_fgx + uy * e_fgy + uz * e_fgz;
      const R u_drho = ux * drcx + uy * drcy + uz * drcz;
      const R drmx = drho_cs2 * f_dcx, drmy = drho_cs2 * f_dcy, drmz = drho_cs2 * f_dcz;
      const R f_fgx = mu * f_dcx + bfx, f_fgy = mu * f_dcy + bfy, f_fgz = mu * f_dcz + bfz;
      const R f_fhx = f_dcx - c_over * (f_dpx - f_fgx), f_fhy = f_dcy - c_over * (f_dpy - f_fgy),
              f_fhz = f_dcz - c_over * (f_dpz - f_fgz);
      const R u_fh_f = ux * f_fhx + uy * f_fhy + uz * f_fhz;
      const R u_drm = ux * drmx + uy * drmy + uz * drmz;
      const R u_fg_f = ux * f_fgx + uy * f_fgy + uz * f_fgz;
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        const R w = weight<R>(k);
        const R uk = ux * R(lat_cx(k)) + uy * R(lat_cy(k)) + uz * R(lat_cz(k));
        const R u_term = uk * (alpha + beta_c * uk) - gamma_u_sq;
        const R G = w * (R(1) + u_term);
        const R w_u_term = G - w;
        const R f_proj = bfx * R(lat_cx(k)) + bfy * R(lat_cy(k)) + bfz * R(lat_cz(k));
        DirVals<R> v{0, 0, 0, 0};
        R avgk = lmu;
        if (k > 0) {
          v = dir_vals<R>(s_idx, s_c, s_p, pos, ts.off1[k], ts.off2[k], c, p, hbb);
          if (s_idx[pos + ts.off1[k]] >= 0) avgk = R(0.5) * (lmu + s_l[pos + ts.off1[k]]);
        }
        const R drho_dk = drho_cs2 * v.cdc;
        const R eh = c * G + R(0.5) * G * (u_term_h - v.cdc + c_over * (v.cdp - mu * v.cdc - f_proj));
        const R eg = w * p + rho_cs2 * w_u_term +
                     R(0.5) * ((u_drho - drho_dk) * w_u_term + (u_force_g + mu * v.cdc + f_proj) * G);
        const R dc_dk = R(0.5) * (v.cdc + v.bdc), dp_dk = R(0.5) * (v.cdp + v.bdp);
        const R drho_dk2 = drho_cs2 * dc_dk;
        const R ffk = mu * dc_dk + f_proj;
        const R fh = G * (dc_dk - c_over * (dp_dk - ffk) - u_fh_f + mobility * avgk);
        const R fg = (drho_dk2 - u_drm) * w_u_term + (ffk - u_fg_f) * G;
        st_pop<S>(hout, pidx(i, k), k, eh + fh, shh);
        x[k] = eg - g[k];
        gpf[k] = g[k] + fg;
      }
      // rates (reference device_engine.cuh:623-625 with per-kind modes)
      const R taus = R(1) / s0 - R(0.5);
      const R s1 = R(2) * taus / (R(2) * (R)Pm.mrt_lambda + taus);
      R srate[7];
#pragma unroll
      for (int q = 0; q < 7; ++q)
        srate[q] = Pm.rate_mode[q] == RATE_S0 ? s0 : (Pm.rate_mode[q] == RATE_MAGIC ? s1 : (R)Pm.rate_value[q]);
      mrt_apply<R>(x, srate);
#pragma unroll
      for (int k = 0; k < Q; ++k) st_pop<S>(gout, pidx(i, k), k, gpf[k] + x[k], shg);
    } else {
      const R relax = s0;
      const R drcx = drho * e_dcx * cs2, drcy = drho * e_dcy * cs2, drcz = drho * e_dcz * cs2;
      const R e_fgx = mu * e_dcx + bfx, e_fgy = mu * e_dcy + bfy, e_fgz = mu * e_dcz + bfz;
      const R a_over_rho = alpha / rho;
      const R e_fhx = e_dcx - c * a_over_rho * (e_dpx - e_fgx), e_fhy = e_dcy - c * a_over_rho * (e_dpy - e_fgy),
              e_fhz = e_dcz - c * a_over_rho * (e_dpz - e_fgz);
      const R u_fh_e = ux * e_fhx + uy * e_fhy + uz * e_fhz;
      const R u_drhocd = ux * drcx + uy * drcy + uz * drcz;
      const R u_fg_e = ux * e_fgx + uy * e_fgy + uz * e_fgz;
      const R drho_cs2 = drho * cs2;
      const R drmx = drho_cs2 * f_dcx, drmy = drho_cs2 * f_dcy, drmz = drho_cs2 * f_dcz;
      const R c_over = c / cs2 / rho;
      const R f_fgx = mu * f_dcx + bfx, f_fgy = mu * f_dcy + bfy, f_fgz = mu * f_dcz + bfz;
      const R f_fhx = f_dcx - c_over * (f_dpx - f_fgx), f_fhy = f_dcy - c_over * (f_dpy - f_fgy),
              f_fhz = f_dcz - c_over * (f_dpz - f_fgz);
      const R u_fh_f = ux * f_fhx + uy * f_fhy + uz * f_fhz;
      const R u_drm = ux * drmx + uy * drmy + uz * drmz;
      const R u_fg_f = ux * f_fgx + uy * f_fgy + uz * f_fgz;
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        const R w = weight<R>(k);
        const R uk = ux * R(lat_cx(k)) + uy * R(lat_cy(k)) + uz * R(lat_cz(k));
        const R u_term = uk * (alpha + beta_c * uk) - gamma_c * u2;
        const R G = w * (R(1) + u_term);
        const R f_proj = bfx * R(lat_cx(k)) + bfy * R(lat_cy(k)) + bfz * R(lat_cz(k));
        DirVals<R> v{0, 0, 0, 0};
        R avgk = lmu;
        if (k > 0) {
          v = dir_vals<R>(s_idx, s_c, s_p, pos, ts.off1[k], ts.off2[k], c, p, hbb);
          if (s_idx[pos + ts.off1[k]] >= 0) avgk = R(0.5) * (lmu + s_l[pos + ts.off1[k]]);
        }
        const R drho_dk = drho * v.cdc * cs2;
        R eh = c * G;
        eh -= R(0.5) * G * (v.cdc - c * a_over_rho * (v.cdp - mu * v.cdc - f_proj));
        eh += R(0.5) * G * u_fh_e;
        R eg = w * (p + rho * cs2 * u_term);
        eg -= R(0.5) * (drho_dk * (G - w) + (mu * v.cdc + f_proj) * G);
        eg += R(0.5) * ((G - w) * u_drhocd + G * u_fg_e);
        const R dGk = G - w;
        const R dc_dk = R(0.5) * (v.cdc + v.bdc), dp_dk = R(0.5) * (v.cdp + v.bdp);
        const R drho_dk2 = drho_cs2 * dc_dk;
        const R ffk = mu * dc_dk + f_proj;
        const R fh = G * (dc_dk - c_over * (dp_dk - ffk) - u_fh_f + mobility * avgk);
        const R fg = (drho_dk2 - u_drm) * dGk + (ffk - u_fg_f) * G;
        st_pop<S>(hout, pidx(i, k), k, eh + fh, shh);
        st_pop<S>(gout, pidx(i, k), k, g[k] + relax * (eg - g[k]) + fg, shg);
      }
      (void)x; (void)gpf;
    }
  }
  // flow-statistics partials (reference k_flow_stats :660-683, summed on demand)
  block_sum<6>(st, ts, true);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int q = 0; q < 6; ++q) D.part4[(int64_t)brick * 6 + q] = st[q];
    if (bad) atomicOr(&D.ctl->status, 1);
  }
  if (!last_block(&D.ctl->count4, (unsigned)D.nbricks, ts)) return;
  if (threadIdx.x == 0) {
    Ctl* C = D.ctl;
    C->t += 1;
    if (Pm.open_bnd) C->open_step += 1;
    C->pending = (C->auto_correct && Pm.correct_mass) ? 1 : 0;
    C->lambda = 0.0;
    C->count4 = 0;
  }
}

// ---------------------------------------------------------------------------
// open-boundary field enforcement (reference enforce_open_bnd_fields,
// multiphase_gpu.cuh:404-418: k_open_bnd_fields :738-759 and the injection
// gate d_inlet_gate :699-728), run between P1 and P2. Saves each boundary
// site's moment value of c (for mu and tau, which the reference keeps from
// the moments) and its velocity, then imposes the prescribed fields.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double inlet_gate(const DevPrm& P, unsigned step, double coord) {
  const double w = P.inlet_ramp;
  if (P.inlet_mode == 1) {
    const double Per = P.inlet_period;
    if (Per <= 0.0) return 1.0;
    const double tau = (double)step - Per * floor((double)step / Per);
    const double lo = 0.5 * Per - 0.5 * P.inlet_duty * Per, hi = 0.5 * Per + 0.5 * P.inlet_duty * Per;
    if (w <= 0.0) return (tau >= lo && tau < hi) ? 1.0 : 0.0;
    return 0.5 * (tanh(2.0 * (tau - lo) / w) - tanh(2.0 * (tau - hi) / w));
  }
  if (P.inlet_mode == 2) {
    const double x = coord - P.split_pos;
    if (w <= 0.0) return (x < 0.0) ? 1.0 : 0.0;
    return 0.5 * (1.0 - tanh(2.0 * x / w));
  }
  if (P.inlet_mode == 3) {
    const double Per = P.inlet_period;
    if (Per <= 0.0) return 1.0;
    double t = coord - P.split_pos;
    t = t - Per * floor(t / Per);
    const double lo = 0.5 * Per - 0.5 * P.inlet_duty * Per, hi = 0.5 * Per + 0.5 * P.inlet_duty * Per;
    if (w <= 0.0) return (t >= lo && t < hi) ? 1.0 : 0.0;
    return 0.5 * (tanh(2.0 * (t - lo) / w) - tanh(2.0 * (t - hi) / w));
  }
  return 1.0;
}

template <class S>
__global__ void k_bc_fields(const LatDesc* __restrict__ descs, int lat) {
  using R = typename S::real;
  using F = typename S::fld;
  const LatDesc& D = descs[lat];
  const DevPrm& Pm = D.prm;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D.n_inlet + D.n_outlet) return;
  const bool inlet = j < D.n_inlet;
  const int64_t i = D.bc_list[j];
  F* fc = static_cast<F*>(D.c);
  F* fp = static_cast<F*>(D.p);
  F* ubc = static_cast<F*>(D.u_bc);
  const R c_raw = (R)fc[i];
  static_cast<F*>(D.c_raw_bc)[i] = (F)c_raw;
  const R rho_raw = (R)Pm.rho1 + (R)Pm.drho * c_raw;
  const R inv = R(1) / (R(CS2) * rho_raw);
  R ux = (R) static_cast<const F*>(D.jx)[i] * inv;
  R uy = (R) static_cast<const F*>(D.jy)[i] * inv;
  R uz = (R) static_cast<const F*>(D.jz)[i] * inv;
  if (inlet) {
    if (Pm.use_in_vel) { ux = (R)Pm.u_in[0]; uy = (R)Pm.u_in[1]; uz = (R)Pm.u_in[2]; }
    if (Pm.use_in_prs) fp[i] = (F)Pm.p_in;
    if (Pm.use_in_fluid) {
      const double gate = inlet_gate(Pm, (unsigned)D.ctl->open_step, D.bc_coord ? D.bc_coord[j] : 0.0);
      const R cc = (R(1) - (R)Pm.inlet_c_a) + (R(2) * (R)Pm.inlet_c_a - R(1)) * (R)gate;
      fc[i] = (F)cc;
    }
  } else {
    if (Pm.use_out_prs) fp[i] = (F)Pm.p_out;
    if (Pm.use_out_fluid) fc[i] = (F)Pm.c_out_fixed;
  }
  ubc[i] = (F)ux; ubc[D.n + i] = (F)uy; ubc[2 * D.n + i] = (F)uz;
}

// copy_to_buffers field copy (k_open_bnd_buf_fields :807-815)
template <class S>
__global__ void k_bc_buffers(const LatDesc* __restrict__ descs, int lat) {
  using F = typename S::fld;
  const LatDesc& D = descs[lat];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D.n_buf) return;
  const int64_t b = D.buf_verts[j], r = D.buf_refs[j];
  F* fc = static_cast<F*>(D.c);
  F* fp = static_cast<F*>(D.p);
  F* ubc = static_cast<F*>(D.u_bc);
  static_cast<F*>(D.c_raw_bc)[b] = fc[b];
  fc[b] = fc[r];
  fp[b] = fp[r];
  ubc[b] = ubc[r]; ubc[D.n + b] = ubc[D.n + r]; ubc[2 * D.n + b] = ubc[2 * D.n + r];
}

// ---------------------------------------------------------------------------
// state transfer and reductions
// ---------------------------------------------------------------------------
// Post-stream state in the reference layout f[k*n + ref(i)] (double), with a
// queued mass correction injected as the reference's k_inject_mass does.
template <class S>
__global__ void __launch_bounds__(CTA) k_download_state(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                         int parity, double* __restrict__ h_out,
                                                         double* __restrict__ g_out, int apply_lambda) {
  using R = typename S::real;
  using P = typename S::pop;
  __shared__ TileShared ts;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  tile_setup<1>(D, wk.y, ts);
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);
  for (int t = threadIdx.x; t < ts.ntile; t += blockDim.x) s_idx[t] = tile_site(D, ts, t);
  __syncthreads();
  const P* hin = static_cast<const P*>(D.pop[parity][0]);
  const P* gin = static_cast<const P*>(D.pop[parity][1]);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  const Shift shg{(float)D.prm.p_ref, (float)(1.0 / D.prm.g_scale), (float)D.prm.g_scale};
  const double lambda = apply_lambda ? D.ctl->lambda : 0.0;
  const int64_t n = D.n;
  for (int r = threadIdx.x; r < ts.cnt; r += blockDim.x) {
    const int s = ts.slot_of[r];
    const int64_t i = ts.first + r;
    const int pos = slot_pos(D, ts, s);
    const int64_t q = D.ref_of[i];
    R hv[Q];
    double cd = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      const int up = s_idx[pos - ts.off1[k]];
      const int64_t a = up >= 0 ? pidx(up, k) : pidx(i, lat_opp(k));
      const int kk = up >= 0 ? k : lat_opp(k);
      hv[k] = ld_pop<S>(hin, a, kk, shh);
      cd += (double)hv[k];
      g_out[k * n + q] = (double)ld_pop<S>(gin, a, kk, shg);
    }
    const double phi = cd * (1.0 - cd);
    const bool inj = lambda != 0.0 && phi > 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      R v = hv[k];
      if (inj) v += (R)(weight<double>(k) * (-lambda * phi));
      h_out[k * n + q] = (double)v;
    }
  }
}

// Inverse of the pull: place post-stream values so that the next P1 pulls
// them back (reference upload_state, multiphase_gpu.cuh:354-359).
template <class S>
__global__ void __launch_bounds__(CTA) k_upload_state(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                       int parity, const double* __restrict__ h_in,
                                                       const double* __restrict__ g_in) {
  using P = typename S::pop;
  __shared__ TileShared ts;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  tile_setup<1>(D, wk.y, ts);
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);
  for (int t = threadIdx.x; t < ts.ntile; t += blockDim.x) s_idx[t] = tile_site(D, ts, t);
  __syncthreads();
  P* hb = static_cast<P*>(D.pop[parity][0]);
  P* gb = static_cast<P*>(D.pop[parity][1]);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  const Shift shg{(float)D.prm.p_ref, (float)(1.0 / D.prm.g_scale), (float)D.prm.g_scale};
  const int64_t n = D.n;
  for (int r = threadIdx.x; r < ts.cnt; r += blockDim.x) {
    const int s = ts.slot_of[r];
    const int64_t i = ts.first + r;
    const int pos = slot_pos(D, ts, s);
    const int64_t q = D.ref_of[i];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      const int up = s_idx[pos - ts.off1[k]];
      const int64_t a = up >= 0 ? pidx(up, k) : pidx(i, lat_opp(k));
      const int kk = up >= 0 ? k : lat_opp(k);
      st_pop<S>(hb, a, kk, (typename S::real)h_in[k * n + q], shh);
      st_pop<S>(gb, a, kk, (typename S::real)g_in[k * n + q], shg);
    }
  }
}

// M = sum c, W = sum c(1-c)^+ of the post-stream state (reference
// k_mass_weight :1109-1126) into ctl->M, ctl->W; with `queue` the lambda of a
// queued correction is formed as in P1.
template <class S>
__global__ void __launch_bounds__(CTA) k_mass(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                               int parity, double* __restrict__ part) {
  using R = typename S::real;
  using P = typename S::pop;
  __shared__ TileShared ts;
  extern __shared__ __align__(16) unsigned char dsm[];
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int brick = wk.y;
  tile_setup<1>(D, brick, ts);
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);
  for (int t = threadIdx.x; t < ts.ntile; t += blockDim.x) s_idx[t] = tile_site(D, ts, t);
  __syncthreads();
  const P* hin = static_cast<const P*>(D.pop[parity][0]);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  double acc[2] = {0.0, 0.0};
  for (int r = threadIdx.x; r < ts.cnt; r += blockDim.x) {
    const int s = ts.slot_of[r];
    const int64_t i = ts.first + r;
    const int pos = slot_pos(D, ts, s);
    double cd = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      const int up = s_idx[pos - ts.off1[k]];
      const int64_t a = up >= 0 ? pidx(up, k) : pidx(i, lat_opp(k));
      cd += (double)ld_pop<S>(hin, a, up >= 0 ? k : lat_opp(k), shh);
    }
    double phi = cd * (1.0 - cd);
    if (phi < 0.0) phi = 0.0;
    acc[0] += cd;
    acc[1] += phi;
  }
  block_sum<2>(acc, ts);
  if (threadIdx.x == 0) {
    part[(int64_t)brick * 2 + 0] = acc[0];
    part[(int64_t)brick * 2 + 1] = acc[1];
  }
  if (!last_block(&D.ctl->countm, (unsigned)D.nbricks, ts)) return;
  double tot[2];
  sum_partials<2>(part, D.nbricks, 2, tot, ts);
  if (threadIdx.x == 0) {
    Ctl* C = D.ctl;
    C->M = tot[0];
    C->W = tot[1];
    double lam = 0.0;
    if (C->pending) {
      const double drift = tot[0] - C->target_mass;
      C->drift = drift;
      if (tot[1] > 0.0 && drift != 0.0) lam = drift / tot[1];
    }
    C->lambda = lam;
    C->countm = 0;
  }
}

// Sum the flow-statistics partials of the last collision pass into ctl->stats.
__global__ void __launch_bounds__(CTA) k_stats_finalize(const LatDesc* __restrict__ descs, int lat) {
  __shared__ TileShared ts;
  const LatDesc& D = descs[lat];
  double tot[6];
  sum_partials<6>(D.part4, D.nbricks, 6, tot, ts, true);
  if (threadIdx.x == 0)
    for (int q = 0; q < 6; ++q) D.ctl->stats[q] = tot[q];
}

}  // namespace fe
