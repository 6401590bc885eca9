// B200 (sm_100a) kernels of the Lee–Liu D3Q19 step.
//
// One step is four brick-parallel passes, separated by the grid-wide
// dependencies of the scheme (reference MultiPhaseGPU::step,
// multiphase_gpu.cuh:522-631):
//   P1 k_moments  own-site h,g (19+19 loads), write c, p, j; M,W partials
//                 of the order-parameter mass (and, last block, lambda)
//   P2 k_cfield   c stencil (grad_cd, Laplacian + wetting BC) -> mu, p
//                 (velocity/pressure correction)
//   P3 k_lapmu    mu stencil -> Laplacian of mu
//   P4 k_collide  c, p stencils to distance 2, lap(mu) to distance 1, own g:
//                 equilibria + Guo force + BGK/MRT relaxation, push h, g
// The stencil passes (P2, P3, P4) run one CTA per brick. The stencil fields
// live on a dense node grid (solid nodes NaN), so
// a brick's field tile (brick + halo) is one box of the grid: one thread
// issues the box copies (TMA, cp.async.bulk.tensor) and a bulk copy of the
// brick's slot list, all completing on one mbarrier, and the CTA waits for
// them once; solid positions arrive as NaN, so one load gives value and
// occupancy. Then one thread per fluid site of the brick. All stencil case
// logic (central / one-sided / biased, halfway bounce-back, wetting) is
// derived from tile occupancy with selects, so no per-site tables are read
// from HBM. P1 and the state transfers touch only a site's own populations
// and run over flat chunks of CHUNK sites. Grid positions outside the
// lattice hold the periodic images of fluid nodes, refreshed by k_images
// after each pass that writes the field.
//
// Streaming is push, fused into P4: the post-collision value f*_k of site x
// is written to slot k of x + e_k, or to slot opp(k) of x itself when x + e_k
// is solid (halfway bounce-back). The state between steps is therefore the
// post-stream state of the reference, and P1 reads it coalesced.
#pragma once
#include <cuda_bf16.h>
#include <cuda_fp16.h>

#include <cstdint>

#include "bulk.cuh"
#include "d3q19.hpp"
#include "layout.hpp"
#include "mrt.hpp"
#include "pair2.cuh"

namespace fe {

// ---------------------------------------------------------------------------
// storage traits
// ---------------------------------------------------------------------------
struct StF64 {
  using pop = double;
  using fld = double;
  using real = double;
  static constexpr bool shifted = false;
  using hpop = pop;
  using gpop = pop;
  static constexpr bool hshift = shifted, gshift = shifted;
};
struct StF32 {
  using pop = float;
  using fld = float;
  using real = float;
  static constexpr bool shifted = false;
  using hpop = pop;
  using gpop = pop;
  static constexpr bool hshift = shifted, gshift = shifted;
};
// FP16 / BF16: population k stored as (f_k - w_k * ref) * scale, ref = c_ref
// for h and p_ref for g; arithmetic in FP32.
struct StF16S {
  using pop = __half;
  using fld = float;
  using real = float;
  static constexpr bool shifted = true;
  using hpop = pop;
  using gpop = pop;
  static constexpr bool hshift = shifted, gshift = shifted;
};
struct StBF16S {
  using pop = __nv_bfloat16;
  using fld = float;
  using real = float;
  static constexpr bool shifted = true;
  using hpop = pop;
  using gpop = pop;
  static constexpr bool hshift = shifted, gshift = shifted;
};

// Mixed storage: h in FP32 (the order parameter spans 0..1, so a shift
// gains it no precision), g as scaled FP16 / BF16 deviations from w_k p_ref.
struct StF16G {
  using pop = float;
  using fld = float;
  using real = float;
  static constexpr bool shifted = false;
  using hpop = float;
  using gpop = __half;
  static constexpr bool hshift = false, gshift = true;
};
struct StBF16G {
  using pop = float;
  using fld = float;
  using real = float;
  static constexpr bool shifted = false;
  using hpop = float;
  using gpop = __nv_bfloat16;
  static constexpr bool hshift = false, gshift = true;
};

// The h and the g view of a storage, for ld_pop / st_pop.
template <class S>
struct HV {
  using pop = typename S::hpop;
  using real = typename S::real;
  static constexpr bool shifted = S::hshift;
};
template <class S>
struct GV {
  using pop = typename S::gpop;
  using real = typename S::real;
  static constexpr bool shifted = S::gshift;
};

template <class T> __device__ __forceinline__ float to_f(T v);
template <> __device__ __forceinline__ float to_f<__half>(__half v) { return __half2float(v); }
template <> __device__ __forceinline__ float to_f<__nv_bfloat16>(__nv_bfloat16 v) { return __bfloat162float(v); }
template <class T> __device__ __forceinline__ T from_f(float v);
template <> __device__ __forceinline__ __half from_f<__half>(float v) { return __float2half_rn(v); }
template <> __device__ __forceinline__ __nv_bfloat16 from_f<__nv_bfloat16>(float v) { return __float2bfloat16_rn(v); }

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
__device__ __forceinline__ void st_pop(typename S::pop* __restrict__ a, int64_t idx, int k, typename S::real v,
                                       const Shift& sh) {
  if constexpr (S::shifted) {
    a[idx] = from_f<typename S::pop>((v - weight<float>(k) * sh.ref) * sh.scale);
  } else {
    a[idx] = v;
  }
}

template <class R>
__device__ __forceinline__ R nan_v() {
  return __int_as_float(0x7fc00000);
}
template <>
__device__ __forceinline__ double nan_v<double>() {
  return __longlong_as_double(0x7ff8000000000000ll);
}
template <class R>
__device__ __forceinline__ bool is_site(R v) {
  return v == v;  // solid tile positions hold NaN
}

// ---------------------------------------------------------------------------
// brick shapes and tiles
// ---------------------------------------------------------------------------
constexpr int CTA = 256;
// Threads per collide CTA; each collide warp leaves one flow-statistics
// record. (128-thread CTAs measured slower: shared memory then limits an SM
// to three of them, 12 warps instead of 16.)
constexpr int P4T = 256;
constexpr int P4W = P4T / 32;

template <int BX_, int BY_, int BZ_>
struct BrickShape {
  static constexpr int BX = BX_, BY = BY_, BZ = BZ_;
  static constexpr int LBX = BX == 16 ? 4 : (BX == 8 ? 3 : (BX == 4 ? 2 : (BX == 2 ? 1 : 0)));
  static constexpr int LBY = BY == 16 ? 4 : (BY == 8 ? 3 : (BY == 4 ? 2 : (BY == 2 ? 1 : 0)));
  static constexpr int C = BX * BY * BZ;
  static constexpr int W = (C + 63) / 64;
  static constexpr int HZ = BZ > 1 ? 1 : 0;  // the z axis has a halo (3-D bricks)
  static_assert((1 << LBX) == BX && (1 << LBY) == BY, "power-of-two brick");
};
using Shape3D = BrickShape<8, 8, 8>;
using Shape2D = BrickShape<16, 16, 1>;
// Alternative 3-D bricks the autotuner chooses from (FP64 and FP32 storage):
// half height (256 slots, one collide-pass iteration for any fill) and
// double width (1024 slots, a shorter per-site prologue for sparse media).
using Shape3D_H = BrickShape<8, 8, 4>;
using Shape3D_W = BrickShape<16, 8, 8>;

template <class Sh, int H>
struct Tile {
  static constexpr int TX = Sh::BX + 2 * H, TY = Sh::BY + 2 * H, TZ = Sh::BZ + 2 * H * Sh::HZ;
  static constexpr int N = TX * TY * TZ;
  static constexpr int SY = TX, SZ = TX * TY;
  // tile offset of +e_k and of the brick slot s
  __device__ static constexpr int off(int k) { return lat_cx(k) + SY * lat_cy(k) + SZ * lat_cz(k) * Sh::HZ; }
  __device__ static __forceinline__ int pos(int s) {
    const int lx = s & (Sh::BX - 1), ly = (s >> Sh::LBX) & (Sh::BY - 1), lz = s >> (Sh::LBX + Sh::LBY);
    return (lx + H) + SY * (ly + H) + SZ * (lz + H * Sh::HZ);
  }
};

// A field tile staged from the dense grid: halo H along y and z (z only for
// 3-D bricks) and always 2 along x, so every box starts on a 16-byte
// boundary of the grid. Same indexing as Tile (Tile<Sh, 2> is TileX<Sh, 2>).
template <class Sh, int H>
struct TileX {
  static constexpr int TX = Sh::BX + 4, TY = Sh::BY + 2 * H, TZ = Sh::BZ + 2 * H * Sh::HZ;
  static constexpr int N = TX * TY * TZ;
  static constexpr int SY = TX, SZ = TX * TY;
  __device__ static constexpr int off(int k) { return lat_cx(k) + SY * lat_cy(k) + SZ * lat_cz(k) * Sh::HZ; }
  __device__ static __forceinline__ int pos(int s) {
    const int lx = s & (Sh::BX - 1), ly = (s >> Sh::LBX) & (Sh::BY - 1), lz = s >> (Sh::LBX + Sh::LBY);
    return (lx + 2) + SY * (ly + H) + SZ * (lz + H * Sh::HZ);
  }
};

// Prologue state in shared memory (static part).
template <class Sh>
struct Pro {
  BrickRec rec;
  uint64_t nmask[64][Sh::W];
  int32_t nbase[64][Sh::W];
  uint16_t slot_of[Sh::C];
  double lambda;
  double ff;
};

// forcing_factor_at (reference felbm_gpu_main.cu:587-594); a field refresh
// without a step (ff_auto == 2) takes the factor of the last step, as the
// reference's download_raw reads the DevParams value the driver set last.
__device__ __forceinline__ double forcing_factor_dev(const DevPrm& P, const Ctl& C) {
  if (C.ff_auto == 2) return C.ff_last;
  if (!C.ff_auto) return C.ff_manual;
  const double PI = 3.14159265358979323846;
  if (P.forcing_timedep == 1) return sin(2.0 * PI * double(C.t) / P.forcing_period);
  if (P.forcing_timedep == 2) {
    const double x = sin(2.0 * PI * double(C.t) / P.forcing_period);
    return (x < 0) ? -1.0 : ((x > 0) ? 1.0 : 0.0);
  }
  return 1.0;
}

// The step scalars of the lattice's control block into the prologue state
// (called by one thread).
template <class SMem>
__device__ __forceinline__ void load_step_scalars(const LatDesc& D, SMem& s) {
  {
    const Ctl& C = *D.ctl;
    s.ff = forcing_factor_dev(D.prm, C);
    s.lambda = C.lambda;
  }
}

// Shared state of the reductions of the flat (chunk) kernels; Pro<Sh> has the
// same two members.
struct Red {
  double red[CTA / 32][6];
  int last;
};

// Load the brick record and the neighbour bricks' occupancy into shared
// memory, and list the brick's fluid slots in site order.
template <class Sh, int NT = CTA, bool SCALARS = true>
__device__ __forceinline__ void prologue(const LatDesc& D, int brick, Pro<Sh>& s) {
  const int tid = threadIdx.x;
  {
    const int4* src = reinterpret_cast<const int4*>(D.rec + brick);
    int4* dst = reinterpret_cast<int4*>(&s.rec);
    constexpr int N4 = sizeof(BrickRec) / 16;
    static_assert(N4 <= NT - 32, "the record is copied by the leading warps");
    if (tid < N4) dst[tid] = __ldg(src + tid);
    // the step scalars load in parallel, from the last warp
    if (SCALARS && tid == NT - 1) load_step_scalars(D, s);
  }
  __syncthreads();
  for (int q = tid; q < 64 * Sh::W; q += NT) {
    const int slot = q / Sh::W, w = q - slot * Sh::W;
    const int id = s.rec.nbr[slot];
    if (id >= 0) {
      s.nmask[slot][w] = __ldg(&D.mask[(int64_t)id * Sh::W + w]);
      s.nbase[slot][w] = __ldg(&D.base[(int64_t)id * Sh::W + w]);
    }
  }
  __syncthreads();
  const int own = s.rec.seg[0][HMAX] + 4 * (s.rec.seg[1][HMAX] + 4 * s.rec.seg[2][Sh::HZ ? HMAX : 0]);
  for (int q = tid; q < Sh::C; q += NT) {
    const int w = q >> 6, b = q & 63;
    const uint64_t m = s.nmask[own][w];
    if ((m >> b) & 1ull) s.slot_of[s.nbase[own][w] - s.rec.first + __popcll(m & ((1ull << b) - 1ull))] = (uint16_t)q;
  }
}

// Site indices of a whole halo-H tile, built row by row: for each (y, z) row
// and each neighbour brick it crosses, the row's occupancy bits and first site
// index, then per position one popcount. Ends with a barrier.
template <class Sh, int H, int NT = CTA>
__device__ __forceinline__ void build_idx_tile(const Pro<Sh>& s, int32_t* __restrict__ s_idx,
                                               uint32_t* __restrict__ s_rbits, int32_t* __restrict__ s_rbase) {
  using T = Tile<Sh, H>;
  constexpr int ROWS = T::TY * T::TZ;
  for (int q = threadIdx.x; q < ROWS * 4; q += NT) {
    const int row = q >> 2, sx = q & 3;
    const int ty = row % T::TY, tz = row / T::TY;
    const int ay = ty + (HMAX - H), az = Sh::HZ ? tz + (HMAX - H) : 0;
    const int seg = sx + 4 * (s.rec.seg[1][ay] + 4 * s.rec.seg[2][az]);
    uint32_t bits = 0;
    int32_t base = 0;
    if (s.rec.nbr[seg] >= 0) {
      const int slot0 = (s.rec.loc[1][ay] << Sh::LBX) | (s.rec.loc[2][az] << (Sh::LBX + Sh::LBY));
      const int w = slot0 >> 6, b0 = slot0 & 63;
      const uint64_t m = s.nmask[seg][w];
      bits = (uint32_t)((m >> b0) & ((1ull << Sh::BX) - 1ull));
      base = s.nbase[seg][w] + __popcll(m & ((1ull << b0) - 1ull));
    }
    s_rbits[q] = bits;
    s_rbase[q] = base;
  }
  __syncthreads();
  for (int t = threadIdx.x; t < T::N; t += NT) {
    const int row = t / T::TX, tx = t - row * T::TX;
    const int ax = tx + (HMAX - H);
    const int q = row * 4 + s.rec.seg[0][ax];
    const uint32_t bits = s_rbits[q];
    const int lx = s.rec.loc[0][ax];
    s_idx[t] = ((bits >> lx) & 1u) ? s_rbase[q] + __popc(bits & ((1u << lx) - 1u)) : -1;
  }
  __syncthreads();
}

// Shared-memory arrays of a halo-H site-index tile.
template <class Sh, int H>
struct IdxTile {
  using T = Tile<Sh, H>;
  int32_t idx[T::N];
  uint32_t rbits[T::TY * T::TZ * 4];
  int32_t rbase[T::TY * T::TZ * 4];
};

// Per-CTA head of the stencil passes: the brick's fluid slots in site order,
// its site range, brick coordinates and the step scalars.
template <class Sh>
struct alignas(16) Head {
  uint16_t slot_of[Sh::C];
  double lambda;
  double ff;  // forcing factor in double: narrowed to the arithmetic type where used
  int first, cnt;
  int bx, by, bz;
};

// Grid entry of slot `slot` of the brick at brick coordinates (bx, by, bz).
template <class Sh>
__device__ __forceinline__ int64_t grid_entry(const LatDesc& D, int bx, int by, int bz, int slot) {
  const int x = bx * Sh::BX + (slot & (Sh::BX - 1)) + 2;
  const int y = by * Sh::BY + ((slot >> Sh::LBX) & (Sh::BY - 1)) + 2;
  const int z = bz * Sh::BZ + (slot >> (Sh::LBX + Sh::LBY)) + 2 * D.hz;
  return x + D.gsy * y + D.gsz * z;
}

// The tensor map `id` of the lattice (a CUtensorMap in device memory).
__device__ __forceinline__ const void* tmap_of(const LatDesc& D, int id) {
  return static_cast<const char*>(D.tmap) + 128 * id;
}

// Box copy of the halo-H tile of brick (bx, by, bz) from a stencil-field
// grid into shared memory. XM is the number of tensor-map elements a node
// holds (the pair grid of FP64 fields counts 8-byte elements, two a node);
// x0 = bx * BX * XM elements, 16-byte aligned for the 4- and 8-byte element
// types.
template <class Sh, int H, int XM = 1>
__device__ __forceinline__ void tile_copy(void* dst, const LatDesc& D, int id, int bx, int by, int bz,
                                          uint64_t* bar) {
  tma_box3(dst, tmap_of(D, id), bx * Sh::BX * XM, by * Sh::BY + 2 - H, D.hz ? bz * Sh::BZ + 2 - H : 0, bar);
}

// A stencil pass's prologue: thread 0 sets up the transaction barrier and
// the whole CTA passes a block barrier (no thread polls it before), then
// thread 0 reads the brick's head and issues the slot-list copy and the
// caller's tile copies (their bytes in `tile_bytes`) on that barrier.
__device__ __forceinline__ void head_init(uint64_t* bar) {
  if (threadIdx.x == 0) mbar_init(bar);
  __syncthreads();
}
template <class Sh>
__device__ __forceinline__ void head_begin(const LatDesc& D, int brick, Head<Sh>& s, uint64_t* bar, uint32_t tile_bytes) {
  s.first = __ldg(&D.rec[brick].first);
  s.cnt = __ldg(&D.rec[brick].cnt);
  s.bx = __ldg(&D.brick_xyz[3 * brick + 0]);
  s.by = __ldg(&D.brick_xyz[3 * brick + 1]);
  s.bz = __ldg(&D.brick_xyz[3 * brick + 2]);
  // the slot list up to the brick's site count, in whole 16-byte pieces
  const uint32_t sb = ((uint32_t)s.cnt * (uint32_t)sizeof(uint16_t) + 15u) & ~15u;
  mbar_arrive_expect_tx(bar, tile_bytes + sb);
  bulk_g2s(s.slot_of, D.slots + (int64_t)brick * Sh::C, sb, bar);
}

// Every thread waits for the prologue's copies (bounded). False in every
// thread of the CTA when any thread's wait ran out: the CTA then computes
// nothing and the control block's status records it.
__device__ __forceinline__ bool head_wait(const LatDesc& D, uint64_t* bar) {
  const bool ok = mbar_wait(bar, 0, 1 << 22);
  if (!__syncthreads_and(ok)) {
    if (threadIdx.x == 0) atomicOr(&D.ctl->status, 4);
    return false;
  }
  return true;
}

// Setup: the halo-1 tile of push targets of the collide pass and the slot
// list of every brick, from the occupancy words; one CTA per brick, run once
// per lattice. With 32-bit population offsets (wide == 0) a tile entry is
// the site's AoSoA population base (below 2^32 - 1; 0xffffffff: no site), so
// a push target is one add; with 64-bit offsets it is the site index (-1).
template <class Sh>
__global__ void __launch_bounds__(CTA) k_build_tiles(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                      int wide) {
  using T1 = Tile<Sh, 1>;
  __shared__ Pro<Sh> s;
  __shared__ IdxTile<Sh, 1> t1;
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int brick = wk.y;
  prologue<Sh, CTA, false>(D, brick, s);
  build_idx_tile<Sh, 1>(s, t1.idx, t1.rbits, t1.rbase);
  int32_t* g1 = const_cast<int32_t*>(D.tile1) + (int64_t)brick * T1::N;
  uint16_t* gs = const_cast<uint16_t*>(D.slots) + (int64_t)brick * Sh::C;
  for (int t = threadIdx.x; t < T1::N; t += CTA) {
    const int32_t v = t1.idx[t];
    g1[t] = (wide || v < 0) ? v : (int32_t)((uint32_t)(v >> 5) * (uint32_t)(Q * AOSOA) + (uint32_t)(v & (AOSOA - 1)));
  }
  for (int r = threadIdx.x; r < Sh::C; r += CTA) gs[r] = r < s.rec.cnt ? s.slot_of[r] : (uint16_t)0;
}

// Block reduction of NV doubles into thread 0 (the last one as a max when mx).
// SMem is Pro<Sh> or Red.
template <int NV, class SMem>
__device__ __forceinline__ void block_sum(double (&v)[NV], SMem& s, bool mx_last = false) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double x = v[q];
    const bool mx = mx_last && q == NV - 1;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = mx ? fmax(x, y) : x + y;
    }
    if (lane == 0) s.red[wid][q] = x;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    const int nw = CTA / 32;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double x = s.red[0][q];
      const bool mx = mx_last && q == NV - 1;
      for (int w = 1; w < nw; ++w) x = mx ? fmax(x, s.red[w][q]) : x + s.red[w][q];
      v[q] = x;
    }
  }
  __syncthreads();
}

// Deterministic sum over `count` partial records (fixed strided subsets, then
// a fixed tree), result in thread 0.
template <int NV, class SMem>
__device__ void sum_partials(const double* __restrict__ part, int count, int stride, double (&out)[NV], SMem& s,
                             bool mx_last = false) {
  double acc[NV];
#pragma unroll
  for (int q = 0; q < NV; ++q) acc[q] = 0.0;
  for (int r = threadIdx.x; r < count; r += CTA) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      const double x = __ldcg(&part[(int64_t)r * stride + q]);
      acc[q] = (mx_last && q == NV - 1) ? fmax(acc[q], x) : acc[q] + x;
    }
  }
  block_sum<NV>(acc, s, mx_last);
#pragma unroll
  for (int q = 0; q < NV; ++q) out[q] = acc[q];
}

// True in every thread of the block that finished last (per lattice).
template <class SMem>
__device__ __forceinline__ bool last_block(unsigned int* counter, unsigned int total, SMem& s) {
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) s.last = (atomicAdd(counter, 1u) == total - 1) ? 1 : 0;
  __syncthreads();
  return s.last != 0;
}

// lambda of the queued mass correction from the M, W sums (multiphase_gpu.cuh:689-700)
__device__ __forceinline__ void finish_mass(Ctl* C, double M, double Wt) {
  C->M = M;
  C->W = Wt;
  double lam = 0.0;
  if (C->pending) {
    const double drift = M - C->target_mass;
    C->drift = drift;
    if (Wt > 0.0 && drift != 0.0) lam = drift / Wt;
  }
  C->lambda = lam;
}

// ---------------------------------------------------------------------------
// P1: moments of the post-stream state (reference k_moments,
// device_engine.cuh:116-135, with k_mass_weight, :1109-1126, fused as chunk
// partials + last-block lambda). One CTA per chunk of CHUNK sites; a site's 38
// populations sit at one AoSoA base with constant offsets, so each warp reads
// 38 full 128-byte lines (FP32) and issues them back to back.
// ---------------------------------------------------------------------------
constexpr int CHUNK = 2 * CTA;

// AoSoA index of (site i, direction 0); direction k adds k * AOSOA.
__device__ __forceinline__ int64_t pbase(int64_t i) { return (i >> 5) * (int64_t)(Q * AOSOA) + (i & (AOSOA - 1)); }

template <class S>
__global__ void __launch_bounds__(CTA) k_moments(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                  int parity, int write_j) {
  using R = typename S::real;
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  using F = typename S::fld;
  __shared__ Red s;
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int chunk = wk.y;
  const PH* __restrict__ hin = static_cast<const PH*>(D.pop[parity][0]);
  const PG* __restrict__ gin = static_cast<const PG*>(D.pop[parity][1]);
  F* __restrict__ fc = static_cast<F*>(D.c);
  F* fp = static_cast<F*>(D.p);
  F* __restrict__ fjx = static_cast<F*>(D.jx);
  F* __restrict__ fjy = static_cast<F*>(D.jy);
  F* __restrict__ fjz = static_cast<F*>(D.jz);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  const Shift shg{(float)D.prm.p_ref, (float)(1.0 / D.prm.g_scale), (float)D.prm.g_scale};
  double acc[2] = {0.0, 0.0};
  write_j |= D.prm.need_j;
  const int64_t i0 = (int64_t)chunk * CHUNK;
  const int64_t iend = i0 + CHUNK < D.n ? i0 + CHUNK : D.n;
  for (int64_t i = i0 + threadIdx.x; i < iend; i += CTA) {
    const int64_t a = pbase(i);
    R hv[Q], gv[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      hv[k] = ld_pop<HV<S>>(hin, a + k * AOSOA, k, shh);
      gv[k] = ld_pop<GV<S>>(gin, a + k * AOSOA, k, shg);
    }
    R c = 0, p = 0, jx = 0, jy = 0, jz = 0;
    double cd = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      c += hv[k];
      cd += (double)hv[k];
      p += gv[k];
      if (lat_cx(k)) jx += R(lat_cx(k)) * gv[k];
      if (lat_cy(k)) jy += R(lat_cy(k)) * gv[k];
      if (lat_cz(k)) jz += R(lat_cz(k)) * gv[k];
    }
    const int64_t de = __ldg(&D.dense_of[i]);
    fc[de] = (F)c;
    fp[de] = (F)p;
    if (write_j) {  // read only by P2's pressure correction (drho != 0), the
      fjx[i] = (F)jx;  // open-boundary kernels and field downloads (need_j | forced)
      fjy[i] = (F)jy;
      fjz[i] = (F)jz;
    }
    double phi = cd * (1.0 - cd);
    if (phi < 0.0) phi = 0.0;
    acc[0] += cd;
    acc[1] += phi;
  }
  if (!D.prm.correct_mass) return;
  block_sum<2>(acc, s);
  if (threadIdx.x == 0) {
    D.part1[(int64_t)chunk * 2 + 0] = acc[0];
    D.part1[(int64_t)chunk * 2 + 1] = acc[1];
  }
  if (!last_block(&D.ctl->count1, (unsigned)D.nchunks, s)) return;
  double tot[2];
  sum_partials<2>(D.part1, D.nchunks, 2, tot, s);
  if (threadIdx.x == 0) {
    finish_mass(D.ctl, tot[0], tot[1]);
    D.ctl->count1 = 0;
  }
}

// ---------------------------------------------------------------------------
// Persistent, double-buffered brick pipeline (P2, P3, in-place P1):
// a CTA takes the work items blockIdx.x, blockIdx.x + gridDim.x, ... and
// while it computes one brick from one stage, the copy engine fills the
// other stage with the next brick's head, slot list and halo-H tile (one
// mbarrier per stage, phases counted per use). The block barrier after each
// wait orders the next issue into a stage after every thread has left it.
// ---------------------------------------------------------------------------
template <class Sh, class F, int N>
struct StencilStages {
  // each stage's tile starts on a 128-byte boundary (a TMA destination)
  static constexpr int NA = ((N * (int)sizeof(F) + 127) / 128 * 128) / (int)sizeof(F);
  F tile[2][NA];
  Head<Sh> head[2];
  uint64_t bar[2];
};

// copies(D, brick, head, tile, bar), run by thread 0, starts a brick's
// copies on bar (head_begin and the tile's copy); body(D, brick, head, tile)
// computes it, every thread.
template <class Sh, class F, int N, bool SCALARS, class Copies, class Body>
__device__ __forceinline__ void brick_pipeline(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                               int nwork, StencilStages<Sh, F, N>& sm, Copies&& copies,
                                               Body&& body) {
  if (threadIdx.x == 0) {
    mbar_init(&sm.bar[0]);
    mbar_init(&sm.bar[1]);
  }
  __syncthreads();
  auto issue = [&](int item, int st) {
    if (threadIdx.x == 0) {
      const int2 wk = work[item];
      copies(descs[wk.x], wk.y, sm.head[st], sm.tile[st], &sm.bar[st]);
    }
    if (SCALARS && threadIdx.x == CTA - 1) load_step_scalars(descs[work[item].x], sm.head[st]);
  };
  int w = blockIdx.x;
  if (w < nwork) issue(w, 0);
  for (int j = 0; w < nwork; w += (int)gridDim.x, ++j) {
    const int st = j & 1, wn = w + (int)gridDim.x;
    if (wn < nwork) issue(wn, st ^ 1);
    const int2 wk = work[w];
    const LatDesc& D = descs[wk.x];
    if (!__syncthreads_and(mbar_wait(&sm.bar[st], (uint32_t)((j >> 1) & 1), 1 << 22))) {
      if (threadIdx.x == 0) atomicOr(&D.ctl->status, 4);
      // the next brick's copies land before the CTA leaves (bounded)
      if (wn < nwork) mbar_wait(&sm.bar[st ^ 1], (uint32_t)(((j + 1) >> 1) & 1), 1 << 22);
      return;
    }
    body(D, wk.y, sm.head[st], sm.tile[st]);
    __syncthreads();
  }
}

// The stencil passes' pipeline: the halo-H box of the field grid `tmap_id`.
template <class Sh, class F, int H, bool SCALARS, class Body>
__device__ __forceinline__ void stencil_pipeline(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                 int nwork, int tmap_id, StencilStages<Sh, F, TileX<Sh, H>::N>& sm,
                                                 Body&& body) {
  using T = TileX<Sh, H>;
  brick_pipeline<Sh, F, T::N, SCALARS>(
      descs, work, nwork, sm,
      [&](const LatDesc& D, int brick, Head<Sh>& h, F* tile, uint64_t* bar) {
        head_begin<Sh>(D, brick, h, bar, (uint32_t)(T::N * sizeof(F)));
        tile_copy<Sh, H>(tile, D, tmap_id, h.bx, h.by, h.bz, bar);
      },
      body);
}

// ---------------------------------------------------------------------------
// The in-place (AA) population layout keeps one buffer. A step taken from the
// standard layout (phase 0) writes each site's post-collision f*_k into its
// own slot opp(k); the state between the two steps is then: post-stream
// f_k(x) = f*_k(x - e_k), found in slot opp(k) of the upstream site x - e_k,
// or, when x - e_k is solid (halfway bounce-back), in x's own slot k (phase
// 1). A step taken from phase 1 reads there and pushes f*_k into slot k of
// x + e_k (or slot opp(k) of x), which is the standard layout again. Both
// steps read and write the same 19 slots per site, so no other site's data
// is overwritten before it is read.
// ---------------------------------------------------------------------------
// AoSoA index of the post-stream population k of the site at base a0 (slot
// position pos1 in the brick's halo-1 tile of population bases) in phase 1.
template <class T1>
__device__ __forceinline__ uint32_t aa_src(const int32_t* __restrict__ s_idx, int pos1, uint32_t a0, int k) {
  const uint32_t b = (uint32_t)s_idx[pos1 - T1::off(k)];
  return b != 0xffffffffu ? b + (uint32_t)(lat_opp(k) * AOSOA) : a0 + (uint32_t)(k * AOSOA);
}

// P1 from phase 1 of the in-place layout: the same moments and writes as
// k_moments, on the persistent brick pipeline (the halo-1 tile of population
// bases by bulk copy); mass partials per brick, summed by the CTA whose brick
// is the lattice's last to finish (work items of several lattices may share
// a launch).
template <class S, class Sh>
__global__ void __launch_bounds__(CTA, 4) k_moments_aa(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                     int nwork, int write_j) {
  using R = typename S::real;
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  using F = typename S::fld;
  using T1 = Tile<Sh, 1>;
  __shared__ __align__(128) StencilStages<Sh, int32_t, T1::N> sm;
  __shared__ Red red;
  brick_pipeline<Sh, int32_t, T1::N, false>(
      descs, work, nwork, sm,
      [&](const LatDesc& D, int brick, Head<Sh>& h, int32_t* tile, uint64_t* bar) {
        head_begin<Sh>(D, brick, h, bar, (uint32_t)(T1::N * 4));
        bulk_g2s(tile, D.tile1 + (int64_t)brick * T1::N, (uint32_t)(T1::N * 4), bar);
      },
      [&](const LatDesc& D, int brick, const Head<Sh>& s, const int32_t* s_idx) {
        const PH* __restrict__ hin = static_cast<const PH*>(D.pop[0][0]);
        const PG* __restrict__ gin = static_cast<const PG*>(D.pop[0][1]);
        F* __restrict__ fc = static_cast<F*>(D.c);
        F* __restrict__ fp = static_cast<F*>(D.p);
        F* __restrict__ fjx = static_cast<F*>(D.jx);
        F* __restrict__ fjy = static_cast<F*>(D.jy);
        F* __restrict__ fjz = static_cast<F*>(D.jz);
        const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
        const Shift shg{(float)D.prm.p_ref, (float)(1.0 / D.prm.g_scale), (float)D.prm.g_scale};
        const int wj = write_j | D.prm.need_j;
        double acc[2] = {0.0, 0.0};
        for (int r = threadIdx.x; r < s.cnt; r += CTA) {
          const int64_t i = s.first + r;
          const int slot = s.slot_of[r];
          const int pos1 = T1::pos(slot);
          const uint32_t a0 = (uint32_t)pbase(i);
          R hv[Q], gv[Q];
#pragma unroll
          for (int k = 0; k < Q; ++k) {
            const uint32_t a = k == 0 ? a0 : aa_src<T1>(s_idx, pos1, a0, k);
            hv[k] = ld_pop<HV<S>>(hin, a, k, shh);
            gv[k] = ld_pop<GV<S>>(gin, a, k, shg);
          }
          R c = 0, p = 0, jx = 0, jy = 0, jz = 0;
          double cd = 0.0;
#pragma unroll
          for (int k = 0; k < Q; ++k) {
            c += hv[k];
            cd += (double)hv[k];
            p += gv[k];
            if (lat_cx(k)) jx += R(lat_cx(k)) * gv[k];
            if (lat_cy(k)) jy += R(lat_cy(k)) * gv[k];
            if (lat_cz(k)) jz += R(lat_cz(k)) * gv[k];
          }
          const int64_t de = grid_entry<Sh>(D, s.bx, s.by, s.bz, slot);
          fc[de] = (F)c;
          fp[de] = (F)p;
          if (wj) {
            fjx[i] = (F)jx;
            fjy[i] = (F)jy;
            fjz[i] = (F)jz;
          }
          double phi = cd * (1.0 - cd);
          if (phi < 0.0) phi = 0.0;
          acc[0] += cd;
          acc[1] += phi;
        }
        if (!D.prm.correct_mass) return;
        block_sum<2>(acc, red);
        if (threadIdx.x == 0) {
          D.part1[(int64_t)brick * 2 + 0] = acc[0];
          D.part1[(int64_t)brick * 2 + 1] = acc[1];
        }
        if (!last_block(&D.ctl->count1, (unsigned)D.nbricks, red)) return;
        double tot[2];
        sum_partials<2>(D.part1, D.nbricks, 2, tot, red);
        if (threadIdx.x == 0) {
          finish_mass(D.ctl, tot[0], tot[1]);
          D.ctl->count1 = 0;
        }
      });
}

// Phase 1 of the in-place layout to the standard layout, in place: for the
// leading direction k of each opposite pair, slot k of x (holding f*_opp(k)
// of x, bound for x - e_k) and slot opp(k) of x - e_k (holding f*_k of
// x - e_k, bound for x) trade places; with x - e_k solid both are where the
// standard layout keeps them. Every slot takes part in at most one trade.
template <class S, class Sh>
__global__ void __launch_bounds__(CTA) k_aa_swap(const LatDesc* __restrict__ descs, const int2* __restrict__ work) {
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  using T1 = Tile<Sh, 1>;
  __shared__ Head<Sh> s;
  __shared__ uint64_t s_bar;
  __shared__ __align__(128) int32_t s_idx[T1::N];
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int brick = wk.y;
  head_init(&s_bar);
  if (threadIdx.x == 0) {
    head_begin<Sh>(D, brick, s, &s_bar, (uint32_t)(T1::N * 4));
    bulk_g2s(s_idx, D.tile1 + (int64_t)brick * T1::N, (uint32_t)(T1::N * 4), &s_bar);
  }
  if (!head_wait(D, &s_bar)) return;
  PH* __restrict__ h = static_cast<PH*>(D.pop[0][0]);
  PG* __restrict__ g = static_cast<PG*>(D.pop[0][1]);
  for (int r = threadIdx.x; r < s.cnt; r += CTA) {
    const int slot = s.slot_of[r];
    const int pos1 = T1::pos(slot);
    const uint32_t a0 = (uint32_t)pbase(s.first + r);
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      const uint32_t b = (uint32_t)s_idx[pos1 - T1::off(k)];
      if (b == 0xffffffffu) continue;
      const uint32_t x = a0 + (uint32_t)(k * AOSOA), y = b + (uint32_t)((k + 1) * AOSOA);
      const PH hx = h[x], hy = h[y];
      h[x] = hy;
      h[y] = hx;
      const PG gx = g[x], gy = g[y];
      g[x] = gy;
      g[y] = gx;
    }
  }
}

// corrected order parameter c' = c - lambda * max(c(1-c), 0): the reference's
// k_inject_mass (device_engine.cuh:1128-1139) applied to c instead of h; h is
// never read by the collision (the h update is eq_h + force_h), so the next
// step sees the same state.
template <class R>
__device__ __forceinline__ R corr_c(R c, double lambda) {
  if (lambda == 0.0) return c;
  const double cd = (double)c;
  const double phi = cd * (1.0 - cd);
  return phi > 0.0 ? (R)(cd - lambda * phi) : c;
}

// Apply a queued mass correction to a staged order-parameter tile (solid
// positions stay NaN); every thread its strided positions.
template <int N, int NT, class R>
__device__ __forceinline__ void correct_tile(R* __restrict__ t, double lambda) {
  if (lambda == 0.0) return;
  for (int q = threadIdx.x; q < N; q += NT) {
    const R x = t[q];
    if (is_site(x)) t[q] = corr_c<R>(x, lambda);
  }
}

// ---------------------------------------------------------------------------
// near-wall stencil cases (table builders multiphase_gpu.cuh:93-193, helpers
// device_engine.cuh:89-113,897-1010), from NaN-marked tile values
// ---------------------------------------------------------------------------
// central-difference value of direction k (cd_dir_val)
template <class R>
__device__ __forceinline__ R cd_val(R f0, R fm, R fp, bool hbb) {
  const bool b1 = is_site(fm), f1 = is_site(fp);
  if (hbb) return R(0.5) * ((f1 ? fp : f0) - (b1 ? fm : f0));
  return (b1 && f1) ? R(0.5) * (fp - fm) : R(0);
}
// The central stencil value of direction k (cd_dir_val), branch free with
// the near-wall case fixed at compile time by HBB (one-sided next to a solid
// neighbour under halfway bounce-back, else zero).
template <bool HBB, class R>
__device__ __forceinline__ R cd_sel(R f0, R fm, R fp, bool sm, bool sp) {
  if (HBB) return R(0.5) * ((sp ? fp : f0) - (sm ? fm : f0));
  return (sm && sp) ? R(0.5) * (fp - fm) : R(0);
}
// The central and the biased (bd_dir_val: fp2 = f(x + 2e), fm2 = f(x - 2e))
// stencil values on two-lane (c, p) pairs (c and p share their solid
// positions): both fields per instruction. Biased: the 3-point difference
// when x + e and x + 2e are fluid, 2-point when only x + e is, one-sided
// backwards (or zero) when x + e is solid.
template <bool HBB, class R>
__device__ __forceinline__ V2<R> cd_sel2(V2<R> f0, V2<R> fm, V2<R> fp, bool sm, bool sp) {
  using V = V2<R>;
  if (HBB) return V(R(0.5)) * (sel(sp, fp, f0) - sel(sm, fm, f0));
  return sel(sm && sp, V(R(0.5)) * (fp - fm), V(R(0)));
}
template <bool HBB, class R>
__device__ __forceinline__ V2<R> bd_sel2(V2<R> f0, V2<R> fm, V2<R> fp, V2<R> fm2, V2<R> fp2, bool sm, bool sp,
                                         bool sm2, bool sp2) {
  using V = V2<R>;
  const V two = fma2(V(R(-0.5)), fp2, fma2(V(R(2)), fp, V(R(-1.5)) * f0));
  const V one = HBB ? fma2(V(R(1.5)), fp, V(R(-1.5)) * f0) : fma2(V(R(2)), fp, V(R(-2)) * f0);
  const V back = HBB ? sel(sm, fma2(V(R(-0.5)), fm, V(R(0.5)) * f0), V(R(0)))
                     : sel(sm && sm2, fma2(V(R(-0.5)), fm2, fma2(V(R(2)), fm, V(R(-1.5)) * f0)), V(R(0)));
  return sel(sp, sel(sp2, two, one), back);
}
// One opposite pair of (c, p): central value for +e, biased values for +e
// (ba) and -e (bb); the solid positions are read from the c lane.
template <bool HBB, class R>
__device__ __forceinline__ void pair_derivs2(V2<R> f0, V2<R> fm, V2<R> fp, V2<R> fm2, V2<R> fp2, V2<R>& cd,
                                             V2<R>& ba, V2<R>& bb) {
  const bool sm = is_site(fm.x()), sp = is_site(fp.x()), sm2 = is_site(fm2.x()), sp2 = is_site(fp2.x());
  cd = cd_sel2<HBB>(f0, fm, fp, sm, sp);
  ba = bd_sel2<HBB>(f0, fm, fp, fm2, fp2, sm, sp, sm2, sp2);
  bb = bd_sel2<HBB>(f0, fp, fm, fp2, fm2, sp, sm, sp2, sm2);
}

// Laplacian term of direction k (k_lap_mf), boundary half `bnd`
template <class R>
__device__ __forceinline__ R lap_val(R f0, R fm, R fp, R bnd, bool hbb) {
  const bool b1 = is_site(fm), f1 = is_site(fp);
  if (b1 && f1) return fm - R(2) * f0 + fp;
  if (!(b1 || f1)) return R(0);
  const R f1v = b1 ? fm : fp;
  return hbb ? (f1v - f0 - bnd) : (R(2) * f1v - R(2) * f0 - R(2) * bnd);
}

// lap_val, branch free with the near-wall rule fixed at compile time and the
// two neighbour flags given.
template <bool HBB, class R>
__device__ __forceinline__ R lap_sel(R f0, R fm, R fp, R bnd, bool sm, bool sp) {
  const R both = fm - R(2) * f0 + fp;
  const R f1v = sm ? fm : fp;
  const R one = HBB ? (f1v - f0 - bnd) : (R(2) * f1v - R(2) * f0 - R(2) * bnd);
  return (sm && sp) ? both : ((sm || sp) ? one : R(0));
}

// ---------------------------------------------------------------------------
// P2: grad_cd(c), Laplacian(c) with the wetting term, mu, velocity/pressure
// correction (reference k_grad_cd_mf :897-913, k_pack_lap_c :159-165,
// k_lap_mf :996-1010, k_mu_axpy :149-153, k_vel_press_corr :177-196).
// Open-boundary nodes were resolved by k_bc_final: their mu, p are final.
// OUT == 1: also write c, rho, u, p, mu in the reference site order (download);
// OUT == 2: the same, indexed by node x + nx*(y + ny*z) (dense grids for tracers).
// ---------------------------------------------------------------------------
struct FieldOut {
  double *rho, *c, *ux, *uy, *uz, *p, *mu;  // any may be null
  __device__ __forceinline__ void put(int64_t q, double vc, double vrho, double vx, double vy, double vz, double vp,
                                      double vmu) const {
    if (c) c[q] = vc;
    if (rho) rho[q] = vrho;
    if (ux) ux[q] = vx;
    if (uy) uy[q] = vy;
    if (uz) uz[q] = vz;
    if (p) p[q] = vp;
    if (mu) mu[q] = vmu;
  }
};

// Node index x + nx*(y + ny*z) of slot `slot` of brick `brick`.
template <class Sh>
__device__ __forceinline__ int64_t node_of(const LatDesc& D, int brick, int slot) {
  const int x = D.brick_xyz[3 * brick + 0] * Sh::BX + (slot & (Sh::BX - 1));
  const int y = D.brick_xyz[3 * brick + 1] * Sh::BY + ((slot >> Sh::LBX) & (Sh::BY - 1));
  const int z = D.brick_xyz[3 * brick + 2] * Sh::BZ + (slot >> (Sh::LBX + Sh::LBY));
  return x + (int64_t)D.nx * (y + (int64_t)D.ny * z);
}

// One brick of P2 from its staged halo-1 tile of c (s_c) and head (s).
template <class S, class Sh, int OUT, bool HBB>
__device__ __forceinline__ void cfield_brick(const LatDesc& D, int brick, const Head<Sh>& s,
                                             typename S::fld* __restrict__ s_c, const FieldOut& out) {
  using R = typename S::real;
  using F = typename S::fld;
  using T = TileX<Sh, 1>;
  correct_tile<T::N, CTA>(s_c, s.lambda);
  __syncthreads();
  const DevPrm& Pm = D.prm;
  const R alpha = R(ALPHA), cs2 = R(CS2);
  const R rho1 = (R)Pm.rho1, drho = (R)Pm.drho, kappa = (R)Pm.kappa, four_beta = (R)Pm.four_beta;
  const R bnd_coeff = (R)Pm.bnd_coeff, ff = (R)s.ff;
  const F* __restrict__ fjx = static_cast<const F*>(D.jx);
  const F* __restrict__ fjy = static_cast<const F*>(D.jy);
  const F* __restrict__ fjz = static_cast<const F*>(D.jz);
  F* __restrict__ fp = static_cast<F*>(D.p);
  F* __restrict__ fmu = static_cast<F*>(D.mu);
  V2<F>* __restrict__ fcp = static_cast<V2<F>*>(D.cp);
  const int first = s.first, cnt = s.cnt;
  for (int r = threadIdx.x; r < cnt; r += CTA) {
    const int64_t i = first + r;
    const int slot = s.slot_of[r];
    const int pos = T::pos(slot);
    const int64_t di = grid_entry<Sh>(D, s.bx, s.by, s.bz, slot);
    const R c0 = (R)s_c[pos];
    const uint8_t flag = Pm.open_bnd ? D.bcflag[i] : 0;
    if (flag & BC_SITE) {
      fcp[di] = V2<F>((F)c0, fp[di]);
      if (OUT) {
        const int64_t q = OUT == 2 ? node_of<Sh>(D, brick, slot) : (int64_t)D.ref_of[i];
        const F* ub = static_cast<const F*>(D.u_bc);
        out.put(q, (double)c0, (double)(rho1 + drho * c0), (double)ub[i], (double)ub[D.n + i],
                (double)ub[2 * D.n + i], (double)fp[di], (double)fmu[di]);
      } else if (D.snap_u[0]) {
        const int64_t q = node_of<Sh>(D, brick, slot);
        const F* ub = static_cast<const F*>(D.u_bc);
        D.snap_u[0][q] = (double)ub[i];
        D.snap_u[1][q] = (double)ub[D.n + i];
        D.snap_u[2][q] = (double)ub[2 * D.n + i];
        if (D.snap_c) D.snap_c[q] = (double)c0;
      }
      continue;  // fields resolved by the open-boundary kernels
    }
    const R bnd = bnd_coeff * c0 * (R(1) - c0);
    // opposite pairs: the Laplacian term is symmetric and the central
    // difference antisymmetric, so each pair counts its leading direction twice
    R lap = 0;
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      const R cm = (R)s_c[pos - T::off(k)], cp = (R)s_c[pos + T::off(k)];
      const R aw2 = R(2) * alpha * weight<R>(k);
      lap += aw2 * lap_sel<HBB>(c0, cm, cp, bnd, is_site(cm), is_site(cp));
    }
    const R rho = rho1 + drho * c0;
    const R mu = four_beta * (c0 * (R(1) - c0)) * (R(0.5) - c0) + (-kappa * lap);
    fmu[di] = (F)mu;
    const F p_in = fp[di];
    // the correction changes p only through drho (k_vel_press_corr :194-195);
    // u (and the gradient of c) is needed here only for that, for output, or
    // for the tracers' snapshot
    if (Pm.drho == 0.0) fcp[di] = V2<F>((F)c0, p_in);
    if (Pm.drho != 0.0 || OUT || D.snap_u[0]) {
      R gx = 0, gy = 0, gz = 0;
#pragma unroll
      for (int k = 1; k < Q; k += 2) {
        const R cm = (R)s_c[pos - T::off(k)], cp = (R)s_c[pos + T::off(k)];
        const R aw2 = R(2) * alpha * weight<R>(k);
        const R cdv = cd_sel<HBB>(c0, cm, cp, is_site(cm), is_site(cp));
        if (lat_cx(k)) gx += aw2 * R(lat_cx(k)) * cdv;
        if (lat_cy(k)) gy += aw2 * R(lat_cy(k)) * cdv;
        if (lat_cz(k)) gz += aw2 * R(lat_cz(k)) * cdv;
      }
      const R irho = R(1) / rho;
      const R inv = irho * R(1.0 / CS2);
      const R mor = mu * irho;
      const R ux = (R)fjx[i] * inv + R(0.5) * ((R)Pm.gx + (R)Pm.fx * ff * irho + mor * gx);
      const R uy = (R)fjy[i] * inv + R(0.5) * ((R)Pm.gy + (R)Pm.fy * ff * irho + mor * gy);
      const R uz = (R)fjz[i] * inv + R(0.5) * ((R)Pm.gz + (R)Pm.fz * ff * irho + mor * gz);
      const R p = (R)p_in + R(0.5) * (drho * (ux * gx + uy * gy + uz * gz)) * cs2;
      if (Pm.drho != 0.0) {
        fp[di] = (F)p;
        fcp[di] = V2<F>((F)c0, (F)p);
      }
      if (OUT) {
        const int64_t q = OUT == 2 ? node_of<Sh>(D, brick, slot) : (int64_t)D.ref_of[i];
        out.put(q, (double)c0, (double)rho, (double)ux, (double)uy, (double)uz, (double)p, (double)mu);
      } else if (D.snap_u[0]) {
        const int64_t q = node_of<Sh>(D, brick, slot);
        D.snap_u[0][q] = (double)ux;
        D.snap_u[1][q] = (double)uy;
        D.snap_u[2][q] = (double)uz;
        if (D.snap_c) D.snap_c[q] = (double)c0;
      }
    }
  }
}

// P2 over `nwork` bricks on a persistent grid (at most the CTAs that fit
// the GPU at once): four CTAs an SM with FP32 arithmetic (64 registers),
// three with FP64.
template <class S>
struct CfieldMinBlocks {
  static constexpr int value = sizeof(typename S::real) == 8 ? 3 : 4;
};
template <class S, class Sh, int OUT, bool HBB>
__global__ void __launch_bounds__(CTA, CfieldMinBlocks<S>::value)
    k_cfield(const LatDesc* __restrict__ descs, const int2* __restrict__ work, int nwork, FieldOut out) {
  using F = typename S::fld;
  __shared__ __align__(128) StencilStages<Sh, F, TileX<Sh, 1>::N> sm;
  stencil_pipeline<Sh, F, 1, true>(descs, work, nwork, TM_C1, sm,
                                   [&](const LatDesc& D, int brick, const Head<Sh>& s, F* s_c) {
                                     cfield_brick<S, Sh, OUT, HBB>(D, brick, s, s_c, out);
                                   });
}

// ---------------------------------------------------------------------------
// P3: Laplacian of mu, boundary half zero (reference k_pack_lap_zero :168-173
// + k_lap_mf); symmetric within an opposite pair. Persistent like P2.
// ---------------------------------------------------------------------------
template <class S, class Sh, bool HBB>
__device__ __forceinline__ void lapmu_brick(const LatDesc& D, const Head<Sh>& s,
                                            const typename S::fld* __restrict__ s_m) {
  using R = typename S::real;
  using F = typename S::fld;
  using T = TileX<Sh, 1>;
  const R alpha = R(ALPHA);
  F* __restrict__ flm = static_cast<F*>(D.lapmu);
  const int cnt = s.cnt;
  for (int r = threadIdx.x; r < cnt; r += CTA) {
    const int slot = s.slot_of[r];
    const int pos = T::pos(slot);
    const R m0 = (R)s_m[pos];
    R lap = 0;
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      const R mm = (R)s_m[pos - T::off(k)], mp = (R)s_m[pos + T::off(k)];
      lap += R(2) * alpha * weight<R>(k) * lap_sel<HBB>(m0, mm, mp, R(0), is_site(mm), is_site(mp));
    }
    flm[grid_entry<Sh>(D, s.bx, s.by, s.bz, slot)] = (F)lap;
  }
}

template <class S, class Sh, bool HBB>
__global__ void __launch_bounds__(CTA) k_lapmu(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                int nwork) {
  using F = typename S::fld;
  __shared__ __align__(128) StencilStages<Sh, F, TileX<Sh, 1>::N> sm;
  stencil_pipeline<Sh, F, 1, false>(descs, work, nwork, TM_MU1, sm,
                                    [&](const LatDesc& D, int, const Head<Sh>& s, F* s_m) {
                                      lapmu_brick<S, Sh, HBB>(D, s, s_m);
                                    });
}

// P4 (k_collide) lives in collide.cuh.

// ---------------------------------------------------------------------------
// open boundaries, run between P1 and P2 (reference enforce_open_bnd_fields,
// multiphase_gpu.cuh:404-418, and the velocity/pressure correction of the
// boundary nodes). Three small kernels over the boundary node lists:
//  k_bc_fields  (inlet, outlet) save the moment value of c (mu and tau keep
//               it, as in the reference), form u from j, impose u/p/c
//               (k_open_bnd_fields :738-759, gate d_inlet_gate :699-728);
//  k_bc_buffers (buffers) copy the reference vertex's fields
//               (k_open_bnd_buf_fields :807-815);
//  k_bc_final   (all) mu, and the correction of u and p where the node is
//               not imposed, so that P2 and P4 only read final values.
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
  const int64_t di = D.dense_of[i];
  F* fc = static_cast<F*>(D.c);
  F* fp = static_cast<F*>(D.p);
  F* ubc = static_cast<F*>(D.u_bc);
  const R c_raw = (R)fc[di];
  static_cast<F*>(D.c_raw_bc)[i] = (F)c_raw;
  const R rho_raw = (R)Pm.rho1 + (R)Pm.drho * c_raw;
  const R inv = R(1) / (R(CS2) * rho_raw);
  R ux = (R) static_cast<const F*>(D.jx)[i] * inv;
  R uy = (R) static_cast<const F*>(D.jy)[i] * inv;
  R uz = (R) static_cast<const F*>(D.jz)[i] * inv;
  if (inlet) {
    if (Pm.use_in_vel) { ux = (R)Pm.u_in[0]; uy = (R)Pm.u_in[1]; uz = (R)Pm.u_in[2]; }
    if (Pm.use_in_prs) fp[di] = (F)Pm.p_in;
    if (Pm.use_in_fluid) {
      const double gate = inlet_gate(Pm, (unsigned)D.ctl->open_step, D.bc_coord ? D.bc_coord[j] : 0.0);
      const R cc = (R(1) - (R)Pm.inlet_c_a) + (R(2) * (R)Pm.inlet_c_a - R(1)) * (R)gate;
      fc[di] = (F)cc;
    }
  } else {
    if (Pm.use_out_prs) fp[di] = (F)Pm.p_out;
    if (Pm.use_out_fluid) fc[di] = (F)Pm.c_out_fixed;
  }
  ubc[i] = (F)ux; ubc[D.n + i] = (F)uy; ubc[2 * D.n + i] = (F)uz;
}

template <class S>
__global__ void k_bc_buffers(const LatDesc* __restrict__ descs, int lat) {
  using F = typename S::fld;
  const LatDesc& D = descs[lat];
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D.n_buf) return;
  const int64_t b = D.buf_verts[j], r = D.buf_refs[j];
  const int64_t db = D.dense_of[b], dr = D.dense_of[r];
  F* fc = static_cast<F*>(D.c);
  F* fp = static_cast<F*>(D.p);
  F* ubc = static_cast<F*>(D.u_bc);
  static_cast<F*>(D.c_raw_bc)[b] = fc[db];
  fc[db] = fc[dr];
  fp[db] = fp[dr];
  ubc[b] = ubc[r]; ubc[D.n + b] = ubc[D.n + r]; ubc[2 * D.n + b] = ubc[2 * D.n + r];
}

// Grid entry of node (x, y, z), periodic in each axis (solid nodes hold NaN).
__device__ __forceinline__ int64_t grid_entry_node(const LatDesc& D, int x, int y, int z) {
  x = (x % D.nx + D.nx) % D.nx;
  y = (y % D.ny + D.ny) % D.ny;
  z = (z % D.nz + D.nz) % D.nz;
  return (x + 2) + D.gsy * (y + 2) + D.gsz * (z + 2 * D.hz);
}

// mu and the velocity/pressure correction of every boundary node, exactly as
// P2 computes them for interior sites (the node's own c enters the wetting
// term and the chemical potential keeps the moment value of c).
template <class S>
__global__ void k_bc_final(const LatDesc* __restrict__ descs, int lat) {
  using R = typename S::real;
  using F = typename S::fld;
  const LatDesc& D = descs[lat];
  const DevPrm& Pm = D.prm;
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= D.n_inlet + D.n_outlet + D.n_buf) return;
  const int64_t i = j < D.n_inlet + D.n_outlet ? D.bc_list[j] : D.buf_verts[j - D.n_inlet - D.n_outlet];
  const int64_t di = D.dense_of[i];
  F* fc = static_cast<F*>(D.c);
  F* fp = static_cast<F*>(D.p);
  F* ubc = static_cast<F*>(D.u_bc);
  const int x = D.bc_xyz[3 * j], y = D.bc_xyz[3 * j + 1], z = D.bc_xyz[3 * j + 2];
  const R c0 = (R)fc[di];
  const R bnd = (R)Pm.bnd_coeff * c0 * (R(1) - c0);
  const bool hbb = Pm.hbb != 0;
  R gx = 0, gy = 0, gz = 0, lap = 0;
  for (int k = 1; k < Q; ++k) {
    const int ex = D.nx > 1 ? lat_cx(k) : 0, ey = D.ny > 1 ? lat_cy(k) : 0, ez = D.nz > 1 ? lat_cz(k) : 0;
    const R cm = (R)fc[grid_entry_node(D, x - ex, y - ey, z - ez)];
    const R cp = (R)fc[grid_entry_node(D, x + ex, y + ey, z + ez)];
    const R aw = R(ALPHA) * weight<R>(k);
    const R cdv = cd_val(c0, cm, cp, hbb);
    gx += aw * R(lat_cx(k)) * cdv;
    gy += aw * R(lat_cy(k)) * cdv;
    gz += aw * R(lat_cz(k)) * cdv;
    lap += aw * lap_val(c0, cm, cp, bnd, hbb);
  }
  const R craw = (R) static_cast<const F*>(D.c_raw_bc)[i];
  const R mu = (R)Pm.four_beta * (craw * (R(1) - craw)) * (R(0.5) - craw) + (-(R)Pm.kappa * lap);
  static_cast<F*>(D.mu)[di] = (F)mu;
  if (D.bcflag[i] & BC_PROC) return;
  const R rho = (R)Pm.rho1 + (R)Pm.drho * c0;
  const R ff = (R)forcing_factor_dev(Pm, *D.ctl);
  const R mor = mu / rho;
  const R ux = (R)ubc[i] + R(0.5) * ((R)Pm.gx + (R)Pm.fx * ff / rho + mor * gx);
  const R uy = (R)ubc[D.n + i] + R(0.5) * ((R)Pm.gy + (R)Pm.fy * ff / rho + mor * gy);
  const R uz = (R)ubc[2 * D.n + i] + R(0.5) * ((R)Pm.gz + (R)Pm.fz * ff / rho + mor * gz);
  ubc[i] = (F)ux; ubc[D.n + i] = (F)uy; ubc[2 * D.n + i] = (F)uz;
  fp[di] = (F)((R)fp[di] + R(0.5) * ((R)Pm.drho * (ux * gx + uy * gy + uz * gz)) * R(CS2));
}

// ---------------------------------------------------------------------------
// periodic images in the stencil-field grids
// ---------------------------------------------------------------------------
// Grid positions outside the lattice (node coordinates outside [0, n) on an
// axis) whose wrapped node is fluid: image[j] = {grid entry, entry of the
// node it wraps to}, built on the host. Each work item (lattice, block) copies
// IMG_BLOCK of them for the fields in `fields` (bit 0 c, 1 mu, 2 lap mu,
// 3 the (c', p') pairs). Sources are lattice nodes, never images.
constexpr int IMG_BLOCK = CTA;
enum : int { GF_C = 1, GF_MU = 2, GF_LAPMU = 4, GF_CP = 8 };
template <class F>
__global__ void __launch_bounds__(CTA) k_images(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                 int fields) {
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int64_t j = (int64_t)wk.y * IMG_BLOCK + threadIdx.x;
  if (j >= D.n_images) return;
  const int2 e = __ldg(&D.images[j]);
  F* const f[3] = {static_cast<F*>(D.c), static_cast<F*>(D.mu), static_cast<F*>(D.lapmu)};
#pragma unroll
  for (int b = 0; b < 3; ++b)
    if (fields & (1 << b)) f[b][e.x] = f[b][e.y];
  if (fields & GF_CP) {
    V2<F>* cp = static_cast<V2<F>*>(D.cp);
    cp[e.x] = cp[e.y];
  }
}

// ---------------------------------------------------------------------------
// state transfer and reductions
// ---------------------------------------------------------------------------
// Post-stream state in the reference layout f[k*n + ref(i)] (double), with a
// queued mass correction injected as the reference's k_inject_mass does.
// Out = float for the storages with FP32 arithmetic: the values are the same
// (each is an FP32 number), widened to double on the host.
template <class S, class Out = double>
__global__ void __launch_bounds__(CTA) k_download_state(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                         int parity, Out* __restrict__ h_out,
                                                         Out* __restrict__ g_out, int apply_lambda) {
  using R = typename S::real;
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const PH* hin = static_cast<const PH*>(D.pop[parity][0]);
  const PG* gin = static_cast<const PG*>(D.pop[parity][1]);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  const Shift shg{(float)D.prm.p_ref, (float)(1.0 / D.prm.g_scale), (float)D.prm.g_scale};
  const double lambda = apply_lambda ? D.ctl->lambda : 0.0;
  const int64_t n = D.n, i0 = (int64_t)wk.y * CHUNK;
  const int64_t iend = i0 + CHUNK < n ? i0 + CHUNK : n;
  for (int64_t i = i0 + threadIdx.x; i < iend; i += CTA) {
    const int64_t a = pbase(i), q = D.ref_of[i];
    R hv[Q];
    double cd = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      hv[k] = ld_pop<HV<S>>(hin, a + k * AOSOA, k, shh);
      cd += (double)hv[k];
      g_out[k * n + q] = (Out)ld_pop<GV<S>>(gin, a + k * AOSOA, k, shg);
    }
    const double phi = cd * (1.0 - cd);
    const bool inj = lambda != 0.0 && phi > 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      R v = hv[k];
      if (inj) v += (R)(weight<double>(k) * (-lambda * phi));
      h_out[k * n + q] = (Out)v;
    }
  }
}

// A queued mass correction written into the stored h (the reference's
// k_inject_mass, device_engine.cuh:1128-1139), with the arithmetic of
// k_download_state's injection, so the stored state becomes what a download
// returns; lambda from ctl (formed by k_mass).
template <class S>
__global__ void __launch_bounds__(CTA) k_inject(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                 int parity) {
  using R = typename S::real;
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  PH* h = static_cast<PH*>(D.pop[parity][0]);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  const double lambda = D.ctl->lambda;
  if (lambda == 0.0) return;
  const int64_t n = D.n, i0 = (int64_t)wk.y * CHUNK;
  const int64_t iend = i0 + CHUNK < n ? i0 + CHUNK : n;
  for (int64_t i = i0 + threadIdx.x; i < iend; i += CTA) {
    const int64_t a = pbase(i);
    R hv[Q];
    double cd = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      hv[k] = ld_pop<HV<S>>(h, a + k * AOSOA, k, shh);
      cd += (double)hv[k];
    }
    const double phi = cd * (1.0 - cd);
    if (!(phi > 0.0)) continue;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      R v = hv[k];
      v += (R)(weight<double>(k) * (-lambda * phi));
      st_pop<HV<S>>(h, a + k * AOSOA, k, v, shh);
    }
  }
}

// Post-stream state from the reference layout (reference upload_state,
// multiphase_gpu.cuh:354-359).
// In = float for the storages with FP32 arithmetic: the host narrowed each
// value as the conversion below would.
template <class S, class In = double>
__global__ void __launch_bounds__(CTA) k_upload_state(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                                       int parity, const In* __restrict__ h_in,
                                                       const In* __restrict__ g_in) {
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  PH* hb = static_cast<PH*>(D.pop[parity][0]);
  PG* gb = static_cast<PG*>(D.pop[parity][1]);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  const Shift shg{(float)D.prm.p_ref, (float)(1.0 / D.prm.g_scale), (float)D.prm.g_scale};
  const int64_t n = D.n, i0 = (int64_t)wk.y * CHUNK;
  const int64_t iend = i0 + CHUNK < n ? i0 + CHUNK : n;
  for (int64_t i = i0 + threadIdx.x; i < iend; i += CTA) {
    const int64_t a = pbase(i), q = D.ref_of[i];
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      st_pop<HV<S>>(hb, a + k * AOSOA, k, (typename S::real)h_in[k * n + q], shh);
      st_pop<GV<S>>(gb, a + k * AOSOA, k, (typename S::real)g_in[k * n + q], shg);
    }
  }
}

// The equilibrium state at rest of per-site c and p (reference site order;
// p_in null: p_uniform everywhere), built on the device: the values
// fe_init_equilibrium gives at zero velocity, stored as k_upload_state
// stores them, so the state equals that of fe_upload_state on the host's
// arrays.
template <class S>
__global__ void __launch_bounds__(CTA) k_upload_equilibrium(const LatDesc* __restrict__ descs,
                                                             const int2* __restrict__ work, int parity,
                                                             const double* __restrict__ c_in,
                                                             const double* __restrict__ p_in, double p_uniform) {
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  PH* hb = static_cast<PH*>(D.pop[parity][0]);
  PG* gb = static_cast<PG*>(D.pop[parity][1]);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  const Shift shg{(float)D.prm.p_ref, (float)(1.0 / D.prm.g_scale), (float)D.prm.g_scale};
  const double rho0 = D.prm.rho0, rho1 = D.prm.rho1;
  const int64_t n = D.n, i0 = (int64_t)wk.y * CHUNK;
  const int64_t iend = i0 + CHUNK < n ? i0 + CHUNK : n;
  for (int64_t i = i0 + threadIdx.x; i < iend; i += CTA) {
    const int64_t a = pbase(i), q = D.ref_of[i];
    const double c = c_in[q], p = p_in ? p_in[q] : p_uniform;
    const double rho = rho1 + (rho0 - rho1) * c;
#pragma unroll
    for (int k = 0; k < Q; ++k) {
      double hv, gv;
      equilibrium_k(k, c, p, rho, 0.0, 0.0, 0.0, hv, gv);
      st_pop<HV<S>>(hb, a + k * AOSOA, k, (typename S::real)hv, shh);
      st_pop<GV<S>>(gb, a + k * AOSOA, k, (typename S::real)gv, shg);
    }
  }
}

// M = sum c, W = sum c(1-c)^+ of the post-stream state (reference
// k_mass_weight :1109-1126) into ctl->M, ctl->W, and the lambda of a queued
// correction as P1 forms it.
template <class S>
__global__ void __launch_bounds__(CTA) k_mass(const LatDesc* __restrict__ descs, const int2* __restrict__ work,
                                               int parity, double* __restrict__ part) {
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  __shared__ Red s;
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int chunk = wk.y;
  const PH* hin = static_cast<const PH*>(D.pop[parity][0]);
  const Shift shh{(float)D.prm.c_ref, (float)(1.0 / D.prm.h_scale), (float)D.prm.h_scale};
  double acc[2] = {0.0, 0.0};
  const int64_t i0 = (int64_t)chunk * CHUNK;
  const int64_t iend = i0 + CHUNK < D.n ? i0 + CHUNK : D.n;
  for (int64_t i = i0 + threadIdx.x; i < iend; i += CTA) {
    const int64_t a = pbase(i);
    double cd = 0.0;
#pragma unroll
    for (int k = 0; k < Q; ++k) cd += (double)ld_pop<HV<S>>(hin, a + k * AOSOA, k, shh);
    double phi = cd * (1.0 - cd);
    if (phi < 0.0) phi = 0.0;
    acc[0] += cd;
    acc[1] += phi;
  }
  block_sum<2>(acc, s);
  if (threadIdx.x == 0) {
    part[(int64_t)chunk * 2 + 0] = acc[0];
    part[(int64_t)chunk * 2 + 1] = acc[1];
  }
  if (!last_block(&D.ctl->countm, (unsigned)D.nchunks, s)) return;
  double tot[2];
  sum_partials<2>(part, D.nchunks, 2, tot, s);
  if (threadIdx.x == 0) {
    finish_mass(D.ctl, tot[0], tot[1]);
    D.ctl->countm = 0;
  }
}

// Sum the flow-statistics partials of the last collision pass (one record
// per collide warp) into ctl->stats. Each of the STATS_BLOCKS blocks sums a
// fixed contiguous range of records into blk[block]; the last block to finish
// sums those in block order, so every call adds in the same order.
constexpr int STATS_BLOCKS = 148;
template <class Sh>
__global__ void __launch_bounds__(CTA) k_stats_finalize(const LatDesc* __restrict__ descs, int lat,
                                                         double* __restrict__ blk) {
  __shared__ Red s;
  const LatDesc& D = descs[lat];
  const int count = D.nbricks * P4W;
  const int per = (count + (int)gridDim.x - 1) / (int)gridDim.x;
  const int r0 = min(count, (int)blockIdx.x * per), r1 = min(count, r0 + per);
  double tot[6];
  sum_partials<6>(D.part4 + (int64_t)r0 * 6, r1 - r0, 6, tot, s, true);
  if (threadIdx.x == 0)
    for (int q = 0; q < 6; ++q) blk[blockIdx.x * 6 + q] = tot[q];
  if (last_block(&D.ctl->counts, gridDim.x, s)) {
    sum_partials<6>(blk, gridDim.x, 6, tot, s, true);
    if (threadIdx.x == 0) {
      for (int q = 0; q < 6; ++q) D.ctl->stats[q] = tot[q];
      D.ctl->counts = 0;
    }
  }
}

}  // namespace fe
