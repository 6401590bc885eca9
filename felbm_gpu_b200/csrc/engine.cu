// Host side of the B200 engine: brick/site layout builder, device state,
// step sequencing (plain launches and CUDA graphs), state transfer and the
// C-ABI of include/felbm_b200.h.
//
// It plays the role of the reference's struct MultiPhaseGPU
// (include/felbm_gpu/multiphase_gpu.cuh:23-783); the reference's per-site
// neighbour/case tables (:93-193), streaming source table (:196-208) and
// in-place op program (:213-283) are replaced by the brick occupancy layout
// of layout.hpp, from which the kernels derive the same cases.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <string>
#include <type_traits>
#include <vector>

#include <cuda.h>
#include <mutex>
#include <cudaTypedefs.h>
#include "../../include/felbm_b200.h"
#include "collide.cuh"
#include "fe_internal.hpp"
#include "kernels.cuh"
#include "staging.hpp"
#include "tracers.cuh"

namespace fe {

static thread_local std::string g_last_error;
int fe_fail(int status, const std::string& msg) {
  g_last_error = msg;
  return status;
}
void fe_clear_error() { g_last_error.clear(); }

#define FE_CUDA(call)                                                                              \
  do {                                                                                             \
    cudaError_t err_ = (call);                                                                     \
    if (err_ != cudaSuccess)                                                                       \
      return fe_fail(FE_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(err_) + " (" +   \
                                      __FILE__ + ":" + std::to_string(__LINE__) + ")");            \
  } while (0)

// Run CALL with S (storage traits) and Sh (brick shape) bound to the engine's.
// Inside CALL, write template argument commas as FE_COMMA. Shapes: 0 8x8x8,
// 1 16x16x1, 2 8x8x4 (FP64 and FP32 only), 3 16x8x8.
#define FE_COMMA ,
#define FE_SHAPES_ALL(E, ...)                                                  \
  switch ((E).shape) {                                                         \
    case 1: { using Sh = Shape2D; __VA_ARGS__; } break;                       \
    case 2: { using Sh = Shape3D_H; __VA_ARGS__; } break;                     \
    case 3: { using Sh = Shape3D_W; __VA_ARGS__; } break;                     \
    default: { using Sh = Shape3D; __VA_ARGS__; } break;                      \
  }
#define FE_SHAPES_BASE(E, ...)                                                 \
  switch ((E).shape) {                                                         \
    case 1: { using Sh = Shape2D; __VA_ARGS__; } break;                       \
    case 3: { using Sh = Shape3D_W; __VA_ARGS__; } break;                     \
    default: { using Sh = Shape3D; __VA_ARGS__; } break;                      \
  }
#define FE_DISPATCH(E, ...)                                                    \
  switch ((E).storage) {                                                       \
    case FE_F64: { using S = StF64; FE_SHAPES_ALL(E, __VA_ARGS__) } break;     \
    case FE_F32: { using S = StF32; FE_SHAPES_ALL(E, __VA_ARGS__) } break;     \
    case FE_F16S: { using S = StF16S; FE_SHAPES_BASE(E, __VA_ARGS__) } break;  \
    case FE_BF16S: { using S = StBF16S; FE_SHAPES_BASE(E, __VA_ARGS__) } break; \
    case FE_F16G: { using S = StF16G; FE_SHAPES_BASE(E, __VA_ARGS__) } break;  \
    default: { using S = StBF16G; FE_SHAPES_BASE(E, __VA_ARGS__) } break;      \
  }

template <class Sh>
struct ShTag {
  using type = Sh;
};
template <class S, class Fn>
static void with_shape(int shape, Fn&& fn);

// Storages with the 8x8x4 brick compiled.
template <class S>
constexpr bool kAllShapes = std::is_same<S, StF64>::value || std::is_same<S, StF32>::value;
constexpr int NSHAPE = 4;
// log2 of the brick extents per shape
constexpr int kShapeLb[NSHAPE][3] = {{3, 3, 3}, {4, 4, 0}, {3, 3, 2}, {4, 3, 3}};
// Call fn(ShTag<Sh>) with the brick shape of index `shape`.
template <class S, class Fn>
static void with_shape(int shape, Fn&& fn) {
  if (shape == 1) {
    fn(ShTag<Shape2D>{});
  } else if (shape == 2) {
    if constexpr (kAllShapes<S>) fn(ShTag<Shape3D_H>{});
  } else if (shape == 3) {
    fn(ShTag<Shape3D_W>{});
  } else {
    fn(ShTag<Shape3D>{});
  }
}

static uint64_t morton3(uint32_t x, uint32_t y, uint32_t z) {
  auto spread = [](uint64_t v) {
    v &= 0x1fffff;
    v = (v | v << 32) & 0x1f00000000ffffull;
    v = (v | v << 16) & 0x1f0000ff0000ffull;
    v = (v | v << 8) & 0x100f00f00f00f00full;
    v = (v | v << 4) & 0x10c30c30c30c30c3ull;
    v = (v | v << 2) & 0x1249249249249249ull;
    return v;
  };
  return spread(x) | (spread(y) << 1) | (spread(z) << 2);
}

// Host copy of one lattice's brick layout.
struct HostLayout {
  int nx, ny, nz, lb[3], nb[3], words;
  int shape;
  bool shape2d;  // no halo along z (16x16x1 bricks of a one-layer lattice)
  int64_t n;
  std::vector<int32_t> brick_grid, base, brick_xyz, ref_of, site_of_ref, node_of;
  std::vector<uint64_t> mask;
  std::vector<BrickRec> rec;
  int nbricks() const { return (int)brick_xyz.size() / 3; }
};

// Brick shape (kShapeLb): 16x16x1 for quasi-2-D lattices (nz == 1), one of
// the 3-D bricks otherwise. Axes shorter than the brick simply leave slots
// empty; tile positions wrap periodically, so any extent works.
static int build_layout(const uint8_t* solid, int nx, int ny, int nz, int shape, HostLayout& L) {
  L.nx = nx; L.ny = ny; L.nz = nz;
  L.shape = shape;
  L.shape2d = shape == 1;
  for (int a = 0; a < 3; ++a) L.lb[a] = kShapeLb[shape][a];
  const int B[3] = {1 << L.lb[0], 1 << L.lb[1], 1 << L.lb[2]};
  const int N[3] = {nx, ny, nz};
  for (int a = 0; a < 3; ++a) L.nb[a] = (N[a] + B[a] - 1) / B[a];
  const int C = B[0] * B[1] * B[2];
  L.words = (C + 63) / 64;
  const int64_t total = (int64_t)nx * ny * nz;
  // reference order: fluid nodes by increasing node index
  std::vector<int32_t> ref_of_node(total, -1);
  int64_t nref = 0;
  for (int64_t node = 0; node < total; ++node)
    if (!solid[node]) ref_of_node[node] = (int32_t)nref++;
  L.n = nref;
  struct Bk { uint64_t key; int bx, by, bz; };
  std::vector<Bk> bricks;
  const int64_t nbt = (int64_t)L.nb[0] * L.nb[1] * L.nb[2];
  std::vector<int32_t> cnt(nbt, 0);
  for (int64_t node = 0; node < total; ++node) {
    if (solid[node]) continue;
    const int x = (int)(node % nx), y = (int)((node / nx) % ny), z = (int)(node / ((int64_t)nx * ny));
    ++cnt[(x >> L.lb[0]) + (int64_t)L.nb[0] * ((y >> L.lb[1]) + (int64_t)L.nb[1] * (z >> L.lb[2]))];
  }
  for (int bz = 0; bz < L.nb[2]; ++bz)
    for (int by = 0; by < L.nb[1]; ++by)
      for (int bx = 0; bx < L.nb[0]; ++bx)
        if (cnt[bx + (int64_t)L.nb[0] * (by + (int64_t)L.nb[1] * bz)] > 0)
          bricks.push_back({morton3(bx, by, bz), bx, by, bz});
  std::sort(bricks.begin(), bricks.end(), [](const Bk& a, const Bk& b) { return a.key < b.key; });
  const int nbk = (int)bricks.size();
  L.brick_grid.assign(nbt, -1);
  L.brick_xyz.resize((size_t)nbk * 3);
  L.mask.assign((size_t)nbk * L.words, 0ull);
  L.base.assign((size_t)nbk * L.words, 0);
  L.ref_of.assign(L.n, 0);
  L.site_of_ref.assign(L.n, 0);
  L.node_of.assign(L.n, 0);
  int64_t site = 0;
  for (int b = 0; b < nbk; ++b) {
    const Bk& k = bricks[b];
    L.brick_grid[k.bx + (int64_t)L.nb[0] * (k.by + (int64_t)L.nb[1] * k.bz)] = b;
    L.brick_xyz[b * 3 + 0] = k.bx; L.brick_xyz[b * 3 + 1] = k.by; L.brick_xyz[b * 3 + 2] = k.bz;
    for (int s = 0; s < C; ++s) {
      const int w = s >> 6;
      if ((s & 63) == 0) L.base[(size_t)b * L.words + w] = (int32_t)site;
      const int lx = s & (B[0] - 1), ly = (s >> L.lb[0]) & (B[1] - 1), lz = s >> (L.lb[0] + L.lb[1]);
      const int x = k.bx * B[0] + lx, y = k.by * B[1] + ly, z = k.bz * B[2] + lz;
      if (x >= nx || y >= ny || z >= nz) continue;
      const int64_t node = x + (int64_t)nx * (y + (int64_t)ny * z);
      if (solid[node]) continue;
      L.mask[(size_t)b * L.words + w] |= 1ull << (s & 63);
      L.ref_of[site] = ref_of_node[node];
      L.site_of_ref[ref_of_node[node]] = (int32_t)site;
      L.node_of[site] = (int32_t)node;
      ++site;
    }
  }
  // per-brick records: per-axis tile tables over coordinates [-HMAX, B+HMAX)
  // (wrapped periodically) and the ids of the neighbour bricks they touch
  L.rec.assign(nbk, BrickRec{});
  for (int b = 0; b < nbk; ++b) {
    BrickRec& R = L.rec[b];
    std::memset(&R, 0, sizeof(R));
    int ucoord[3][4], nseg[3];
    for (int a = 0; a < 3; ++a) {
      const bool halo = !(L.shape2d && a == 2);
      const int T = halo ? B[a] + 2 * HMAX : 1;
      const int origin = L.brick_xyz[b * 3 + a] * B[a] - (halo ? HMAX : 0);
      nseg[a] = 0;
      for (int t = 0; t < T; ++t) {
        const int X = ((origin + t) % N[a] + N[a]) % N[a];
        const int bc = X >> L.lb[a];
        int s = 0;
        while (s < nseg[a] && ucoord[a][s] != bc) ++s;
        if (s == nseg[a]) {
          if (nseg[a] == 4) return fe_fail(FE_ERR_ARG, "brick tile touches more than 4 bricks along an axis");
          ucoord[a][nseg[a]++] = bc;
        }
        R.seg[a][t] = (uint8_t)s;
        R.loc[a][t] = (uint8_t)(X & (B[a] - 1));
      }
    }
    for (int q = 0; q < 64; ++q) R.nbr[q] = -1;
    for (int sz = 0; sz < nseg[2]; ++sz)
      for (int sy = 0; sy < nseg[1]; ++sy)
        for (int sx = 0; sx < nseg[0]; ++sx)
          R.nbr[sx + 4 * (sy + 4 * sz)] =
              L.brick_grid[ucoord[0][sx] + (int64_t)L.nb[0] * (ucoord[1][sy] + (int64_t)L.nb[1] * ucoord[2][sz])];
    R.first = L.base[(size_t)b * L.words];
    int c = 0;
    for (int w = 0; w < L.words; ++w) c += __builtin_popcountll(L.mask[(size_t)b * L.words + w]);
    R.cnt = c;
  }
  return FE_OK;
}

// Sets the control block's correction flag (fe_apply_mass_correction).
__global__ void k_queue_correction(Ctl* c) { c->pending = 1; }

enum KernelId { K_P1 = 0, K_BC = 1, K_P2 = 2, K_P3 = 3, K_P4 = 4, K_N = 5 };

// The collide-pass variants: collision model (0 BGK, 1 MRT, 2 MRT in the
// two-rate form, built for halfway bounce-back with 32-bit offsets only; the
// general MRT serves every other case), near-wall rule, and 64-bit
// population offsets for lattices whose arrays reach 2^32 entries.
template <class S, class Sh, int MRT, bool HBB>
static void launch_collide_w(bool wide, int nwork, size_t smem, cudaStream_t st, const LatDesc* desc,
                             const int2* work, int par) {
  if (wide) k_collide<S, Sh, MRT, HBB, true><<<nwork, P4T, smem, st>>>(desc, work, par);
  else k_collide<S, Sh, MRT, HBB, false><<<nwork, P4T, smem, st>>>(desc, work, par);
}
// The in-place layout's two phases (aap 1: from the standard layout, 2: from
// the swapped one), FP64 and FP32 storage with 32-bit offsets.
template <class S>
struct InPlaceStorage {
  static constexpr bool value = std::is_same<S, StF32>::value || std::is_same<S, StF64>::value;
};
template <class S, class Sh, int AAP>
static void launch_collide_aa(int mrt, bool hbb, int nwork, size_t smem, cudaStream_t st, const LatDesc* desc,
                              const int2* work, int par) {
  if constexpr (InPlaceStorage<S>::value) {
    if (mrt == 2 && hbb) k_collide<S, Sh, 2, true, false, AAP><<<nwork, P4T, smem, st>>>(desc, work, par);
    else if (mrt && hbb) k_collide<S, Sh, 1, true, false, AAP><<<nwork, P4T, smem, st>>>(desc, work, par);
    else if (mrt) k_collide<S, Sh, 1, false, false, AAP><<<nwork, P4T, smem, st>>>(desc, work, par);
    else if (hbb) k_collide<S, Sh, 0, true, false, AAP><<<nwork, P4T, smem, st>>>(desc, work, par);
    else k_collide<S, Sh, 0, false, false, AAP><<<nwork, P4T, smem, st>>>(desc, work, par);
  }
}
template <class S, class Sh>
static void launch_collide(int mrt, bool hbb, bool wide, int nwork, size_t smem, cudaStream_t st,
                           const LatDesc* desc, const int2* work, int par, int aap = 0) {
  if (aap == 1) return launch_collide_aa<S, Sh, 1>(mrt == 3 ? 2 : mrt, hbb, nwork, smem, st, desc, work, par);
  if (aap == 2) return launch_collide_aa<S, Sh, 2>(mrt == 3 ? 2 : mrt, hbb, nwork, smem, st, desc, work, par);
  if (mrt == 3 && hbb && !wide) k_collide<S, Sh, 3, true, false><<<nwork, P4T, smem, st>>>(desc, work, par);
  else if (mrt >= 2 && hbb && !wide) k_collide<S, Sh, 2, true, false><<<nwork, P4T, smem, st>>>(desc, work, par);
  else if (mrt && hbb) launch_collide_w<S, Sh, 1, true>(wide, nwork, smem, st, desc, work, par);
  else if (mrt) launch_collide_w<S, Sh, 1, false>(wide, nwork, smem, st, desc, work, par);
  else if (hbb) launch_collide_w<S, Sh, 0, true>(wide, nwork, smem, st, desc, work, par);
  else launch_collide_w<S, Sh, 0, false>(wide, nwork, smem, st, desc, work, par);
}
// CTAs of a persistent stencil pass: as many as the GPU holds at once
// (occupancy of the kernel, once per kernel and device), at most one per
// work item.
static int resident_grid(const void* kernel, int nwork) {
  static std::mutex mu;
  static std::vector<std::pair<std::pair<const void*, int>, int>> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  int full = 0;
  {
    std::lock_guard<std::mutex> lk(mu);
    for (const auto& e : cache)
      if (e.first.first == kernel && e.first.second == dev) full = e.second;
  }
  if (!full) {
    int per = 0, sms = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, CTA, 0) != cudaSuccess || per < 1) per = 1;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms < 1) sms = 1;
    full = per * sms;
    std::lock_guard<std::mutex> lk(mu);
    cache.push_back({{kernel, dev}, full});
  }
  return nwork < full ? nwork : full;
}
template <class S, class Sh, int OUT>
static void launch_cfield(bool hbb, int nwork, cudaStream_t st, const LatDesc* desc, const int2* work,
                          const FieldOut& o) {
  if (nwork <= 0) return;
  if (hbb) {
    auto k = k_cfield<S, Sh, OUT, true>;
    k<<<resident_grid((const void*)k, nwork), CTA, 0, st>>>(desc, work, nwork, o);
  } else {
    auto k = k_cfield<S, Sh, OUT, false>;
    k<<<resident_grid((const void*)k, nwork), CTA, 0, st>>>(desc, work, nwork, o);
  }
}
template <class S, class Sh>
static void launch_moments_aa(int nwork, int write_j, cudaStream_t st, const LatDesc* desc, const int2* work) {
  auto k = k_moments_aa<S, Sh>;
  k<<<resident_grid((const void*)k, nwork), CTA, 0, st>>>(desc, work, nwork, write_j);
}
template <class S, class Sh>
static void launch_lapmu(bool hbb, int nwork, cudaStream_t st, const LatDesc* desc, const int2* work) {
  if (nwork <= 0) return;
  if (hbb) {
    auto k = k_lapmu<S, Sh, true>;
    k<<<resident_grid((const void*)k, nwork), CTA, 0, st>>>(desc, work, nwork);
  } else {
    auto k = k_lapmu<S, Sh, false>;
    k<<<resident_grid((const void*)k, nwork), CTA, 0, st>>>(desc, work, nwork);
  }
}
template <class S, class Sh>
static cudaError_t collide_smem_attr(int bytes) {
  const auto a = cudaFuncAttributeMaxDynamicSharedMemorySize;
  cudaError_t e = cudaSuccess;
  auto set = [&](const void* f) {
    if (e == cudaSuccess) e = cudaFuncSetAttribute(f, a, bytes);
  };
  set((const void*)k_collide<S, Sh, 0, false, false>);
  set((const void*)k_collide<S, Sh, 0, false, true>);
  set((const void*)k_collide<S, Sh, 0, true, false>);
  set((const void*)k_collide<S, Sh, 0, true, true>);
  set((const void*)k_collide<S, Sh, 1, false, false>);
  set((const void*)k_collide<S, Sh, 1, false, true>);
  set((const void*)k_collide<S, Sh, 1, true, false>);
  set((const void*)k_collide<S, Sh, 1, true, true>);
  set((const void*)k_collide<S, Sh, 2, true, false>);
  set((const void*)k_collide<S, Sh, 3, true, false>);
  if constexpr (InPlaceStorage<S>::value) {
    set((const void*)k_collide<S, Sh, 0, false, false, 1>);
    set((const void*)k_collide<S, Sh, 0, true, false, 1>);
    set((const void*)k_collide<S, Sh, 1, false, false, 1>);
    set((const void*)k_collide<S, Sh, 1, true, false, 1>);
    set((const void*)k_collide<S, Sh, 2, true, false, 1>);
    set((const void*)k_collide<S, Sh, 0, false, false, 2>);
    set((const void*)k_collide<S, Sh, 0, true, false, 2>);
    set((const void*)k_collide<S, Sh, 1, false, false, 2>);
    set((const void*)k_collide<S, Sh, 1, true, false, 2>);
    set((const void*)k_collide<S, Sh, 2, true, false, 2>);
  }
  return e;
}
// cuTensorMapEncodeTiled from the driver (no link against libcuda), looked
// up once.
static PFN_cuTensorMapEncodeTiled_v12000 tmap_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    else
      cudaGetLastError();
  });
  return fn;
}

// True when the lattice's population arrays reach 2^32 entries.
static bool pops_wide(int64_t n) { return (uint64_t)((n + AOSOA - 1) / AOSOA) * AOSOA * Q >= (1ull << 32); }

struct Engine {
  fe_params P{};
  int storage = FE_F64;
  int shape2d = 0;
  int shape = 0;              // kShapeLb index
  int graph_steps = 2;        // steps per graph launch of fe_run
  int wide = 0;               // 64-bit population offsets in the collide pass
  int aa = 0;                 // in-place population layout (one buffer; parity = its phase)
  int device = 0;
  HostLayout L;
  LatDesc hd{};               // host copy of the descriptor
  LatDesc* d_desc = nullptr;
  int2* d_work = nullptr;   // (lattice, brick) of the stencil passes
  int2* d_cwork = nullptr;  // (lattice, chunk) of the flat passes
  int2* d_iwork = nullptr;  // (lattice, block) of the image refresh
  Ctl* d_ctl = nullptr;
  cudaStream_t stream = nullptr;
  std::vector<void*> allocs;
  double* d_tmp = nullptr;    // state/field transfer buffer
  int64_t tmp_len = 0;
  double* d_partm = nullptr;
  double* d_stats_blk = nullptr;  // [STATS_BLOCKS][6] block sums of k_stats_finalize
  int parity = 0;             // buffer holding the current state
  int64_t t_host = 0;
  int64_t launches = 0;
  size_t smem_p4 = 0;
  bool open_bnd = false;
  double ff_manual = 1.0;
  int step_mode = 0;          // control mode of the last stepping call (0 fe_step, 1 fe_run)
  int ctl_mode = 0;           // run mode and forcing factor last written to
  double ctl_ff = 1.0;        // the control block (its initial values)
  cudaGraphExec_t graph1[2] = {nullptr, nullptr};
  cudaGraphExec_t graph2[2] = {nullptr, nullptr};
  cudaEvent_t ev_stats = nullptr;
  bool stats_pending = false;
  double* h_stats = nullptr;  // pinned [6]
  double target_mass_host = 0.0;
  struct Batch* owner = nullptr;  // batch the engine is a member of
  std::vector<struct Tracers*> tracer_sets;  // tracers advected on this engine (detached at destroy)
  // The tracer set whose velocity snapshot P2 writes on every step: its
  // advance after step t is deferred to the next single step, whose P2 forms
  // the velocity of that state anyway (tracers.cuh, Tracers::advance).
  struct Tracers* fused = nullptr;
  int64_t state_id = 0;       // bumps whenever the populations change
  int base_need_j = 0;        // need_j without the snapshot
  int tracer_hook(int nsteps, int64_t before, bool after);  // defined after Tracers

  ~Engine() { release(); }
  void release() {
    drop_graphs();
    for (void* a : allocs) cudaFree(a);
    allocs.clear();
    if (d_tmp) cudaFree(d_tmp);
    d_tmp = nullptr;
    if (h_stats) cudaFreeHost(h_stats);
    h_stats = nullptr;
    if (ev_stats) cudaEventDestroy(ev_stats);
    ev_stats = nullptr;
    if (stream) cudaStreamDestroy(stream);
    stream = nullptr;
  }

  template <class T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    const size_t bytes = std::max<size_t>(count, 1) * sizeof(T);
    cudaError_t err = cudaMalloc(&q, bytes);
    if (err != cudaSuccess) {
      cudaGetLastError();
      return fe_fail(FE_ERR_MEMORY, "cudaMalloc of " + std::to_string(bytes) + " bytes: " + cudaGetErrorString(err));
    }
    allocs.push_back(q);
    *p = static_cast<T*>(q);
    return FE_OK;
  }
  template <class T>
  int upload_vec(T** p, const std::vector<T>& v) {
    int rc = alloc(p, v.size());
    if (rc) return rc;
    if (!v.empty()) FE_CUDA(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return FE_OK;
  }

  // bytes of one h (f = 0) or g (f = 1) population
  size_t pop_size(int f) const {
    if (storage == FE_F64) return 8;
    if (storage == FE_F32) return 4;
    if (storage == FE_F16G || storage == FE_BF16G) return f == 0 ? 4 : 2;
    return 2;
  }
  size_t fld_size() const { return storage == FE_F64 ? 8 : 4; }

  // The collide kernel this lattice runs: 0 BGK, 1 MRT, 2 MRT in the
  // two-rate form (halfway bounce-back, 32-bit offsets).
  int collide_variant() const {
    if (!hd.prm.use_mrt) return 0;
    if (!(hd.prm.two_rate && hd.prm.hbb && !wide)) return 1;
    return hd.prm.drho == 0.0 ? 3 : 2;  // 3: no density contrast
  }

  void fill_prm() {
    DevPrm& d = hd.prm;
    d.rho0 = P.rho0; d.rho1 = P.rho1; d.drho = P.rho0 - P.rho1;
    d.kappa = P.kappa; d.four_beta = 4.0 * P.beta; d.bnd_coeff = P.bnd_coeff;
    d.tau0 = P.tau0; d.tau1 = P.tau1; d.mobility = P.mobility;
    d.gx = P.gx; d.gy = P.gy; d.gz = P.gz; d.fx = P.fx; d.fy = P.fy; d.fz = P.fz;
    d.mrt_lambda = P.mrt_lambda;
    for (int q = 0; q < 7; ++q) {
      d.rate_mode[q] = P.mrt_rate_mode[q];
      d.rate_value[q] = P.mrt_rate_value[q];
    }
    d.use_mrt = P.use_mrt; d.hbb = P.use_halfway_bb; d.correct_mass = P.correct_op_mass;
    {
      // one rate per moment parity (FELBM_GENERAL_MRT=1 keeps the general
      // transform, for tests)
      auto same = [&](int a, int b) {
        return P.mrt_rate_mode[a] == P.mrt_rate_mode[b] &&
               (P.mrt_rate_mode[a] != FE_RATE_FIXED || P.mrt_rate_value[a] == P.mrt_rate_value[b]);
      };
      const char* gm = std::getenv("FELBM_GENERAL_MRT");
      d.two_rate = same(FE_MRT_E, FE_MRT_EPS) && same(FE_MRT_E, FE_MRT_NU) && same(FE_MRT_E, FE_MRT_PI) &&
                   same(FE_MRT_Q, FE_MRT_M) && !(gm && gm[0] == '1');
    }
    d.need_j = (P.rho0 != P.rho1 || open_bnd) ? 1 : 0;
    d.forcing_timedep = P.forcing_timedep; d.forcing_period = P.forcing_period;
    d.c_ref = P.c_ref; d.p_ref = P.p_ref;
    // 16-bit deviations: h_k - w_k c_ref spans about w_k, g_k - w_k p_ref about
    // w_k |p|; a power-of-two scale keeps the stored values near 1.
    d.h_scale = (storage == FE_F16S || storage == FE_BF16S) ? 64.0 : 1.0;
    d.g_scale = storage >= FE_F16S ? 64.0 : 1.0;
  }
  int upload_desc() {
    FE_CUDA(cudaMemcpyAsync(d_desc, &hd, sizeof(LatDesc), cudaMemcpyHostToDevice, stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    return FE_OK;
  }

  // Brick shape and graph length: as requested in the parameters, else the
  // autotuner's choice for this size class, else the default brick (16x8x8,
  // 16x16x1 when nz == 1) and two steps per graph.
  int choose_layout(int nx, int ny, int nz, const uint8_t* solid) {
    const int64_t nodes = (int64_t)nx * ny * nz;
    int64_t fluid = 0;
    for (int64_t q = 0; q < nodes; ++q) fluid += solid[q] == 0;
    int brick = P.brick, gs = P.graph_steps;
    int tb = 0, tg = 0;
    if ((brick == FE_BRICK_AUTO || gs <= 0) &&
        tune_lookup(nz == 1, storage, P.use_mrt != 0, P.use_halfway_bb != 0, (double)fluid / (double)nodes, fluid,
                    &tb, &tg)) {
      if (brick == FE_BRICK_AUTO) brick = tb;
      if (gs <= 0) gs = tg;
    }
    // 16x8x8 measured fastest for FP64 and FP32 at every porosity from 0.2 to
    // fully fluid (128^3 and 300^3), and for the 16-bit storages by 16-19 %
    // over 8x8x8 at 300^3
    if (brick == FE_BRICK_AUTO) brick = nz == 1 ? FE_BRICK_16x16x1 : FE_BRICK_16x8x8;
    if (brick < FE_BRICK_8x8x8 || brick > FE_BRICK_16x8x8) return fe_fail(FE_ERR_ARG, "unknown brick shape");
    if ((nz == 1) != (brick == FE_BRICK_16x16x1))
      return fe_fail(FE_ERR_ARG, "16x16x1 bricks are for lattices with nz == 1, and only they");
    if (brick == FE_BRICK_8x8x4 && storage != FE_F64 && storage != FE_F32)
      return fe_fail(FE_ERR_ARG, "8x8x4 bricks exist for FP64 and FP32 storage");
    shape = brick - 1;
    graph_steps = gs > 0 ? gs : 2;
    if (graph_steps > 1024) return fe_fail(FE_ERR_ARG, "graph_steps above 1024");
    return FE_OK;
  }

  int create(const fe_params* p, int nx, int ny, int nz, const uint8_t* solid, int dev) {
    P = *p;
    storage = P.storage;
    if (storage < FE_F64 || storage > FE_BF16G) return fe_fail(FE_ERR_ARG, "unknown storage");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      return fe_fail(FE_ERR_NO_DEVICE, "no CUDA device");
    }
    if (dev >= 0) FE_CUDA(cudaSetDevice(dev));
    FE_CUDA(cudaGetDevice(&device));
    FE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    int rc;
    if ((rc = choose_layout(nx, ny, nz, solid))) return rc;
    if ((rc = build_layout(solid, nx, ny, nz, shape, L))) return rc;
    if (L.n == 0) return fe_fail(FE_ERR_ARG, "geometry has no fluid site");
    if (L.n >= (int64_t)1 << 31) return fe_fail(FE_ERR_ARG, "more than 2^31 sites");
    shape2d = L.shape2d ? 1 : 0;
    // FELBM_WIDE_OFFSETS=1 takes the 64-bit variant at any size (tests)
    {
      const char* w = std::getenv("FELBM_WIDE_OFFSETS");
      wide = (pops_wide(L.n) || (w && w[0] == '1')) ? 1 : 0;
    }
    aa = P.pop_layout == FE_POP_IN_PLACE ? 1 : 0;
    if (P.pop_layout != FE_POP_TWO_BUFFERS && P.pop_layout != FE_POP_IN_PLACE)
      return fe_fail(FE_ERR_ARG, "unknown pop_layout");
    if (aa && storage != FE_F64 && storage != FE_F32)
      return fe_fail(FE_ERR_ARG, "the in-place population layout takes FE_F64 or FE_F32 storage");
    if (aa && wide) return fe_fail(FE_ERR_ARG, "the in-place population layout takes lattices below 2^32 population entries");
    const int nbk = L.nbricks();
    LatDesc& D = hd;
    D.nx = nx; D.ny = ny; D.nz = nz;
    D.lbx = L.lb[0]; D.lby = L.lb[1]; D.lbz = L.lb[2];
    D.nbx = L.nb[0]; D.nby = L.nb[1]; D.nbz = L.nb[2];
    D.words = L.words;
    D.nbricks = nbk;
    D.n = L.n;
    D.nchunks = (int)((L.n + CHUNK - 1) / CHUNK);
    D.n_pad = (L.n + AOSOA - 1) / AOSOA * AOSOA;
    int32_t *bg, *bs, *bx, *rf;
    uint64_t* mk;
    BrickRec* rec;
    if ((rc = upload_vec(&bg, L.brick_grid))) return rc;
    if ((rc = upload_vec(&mk, L.mask))) return rc;
    if ((rc = upload_vec(&bs, L.base))) return rc;
    if ((rc = upload_vec(&bx, L.brick_xyz))) return rc;
    if ((rc = upload_vec(&rf, L.ref_of))) return rc;
    if ((rc = upload_vec(&rec, L.rec))) return rc;
    D.brick_grid = bg; D.mask = mk; D.base = bs; D.brick_xyz = bx; D.ref_of = rf; D.rec = rec;
    const size_t popn = (size_t)Q * D.n_pad;
    for (int b = 0; b < 2; ++b)
      for (int f = 0; f < 2; ++f) {
        if (aa && b == 1) {  // one buffer: both phases address it
          D.pop[1][f] = D.pop[0][f];
          continue;
        }
        unsigned char* q;
        if ((rc = alloc(&q, popn * pop_size(f)))) return rc;
        FE_CUDA(cudaMemset(q, 0, popn * pop_size(f)));
        D.pop[b][f] = q;
      }
    // momentum per site; the stencil fields on the dense node grid, NaN
    // everywhere until the passes write the fluid nodes
    for (void** f : {&D.jx, &D.jy, &D.jz}) {
      unsigned char* q;
      if ((rc = alloc(&q, (size_t)D.n * fld_size()))) return rc;
      FE_CUDA(cudaMemset(q, 0, (size_t)D.n * fld_size()));
      *f = q;
    }
    if ((rc = setup_grid(solid))) return rc;
    if ((rc = alloc(&D.part1, (size_t)std::max(D.nchunks, nbk) * 2))) return rc;  // per chunk, or per brick
    if ((rc = alloc(&D.part4, (size_t)nbk * P4W * 6))) return rc;
    FE_CUDA(cudaMemset(D.part4, 0, (size_t)nbk * P4W * 6 * 8));
    if ((rc = alloc(&d_partm, (size_t)D.nchunks * 2))) return rc;
    if ((rc = alloc(&d_stats_blk, (size_t)STATS_BLOCKS * 6))) return rc;
    if ((rc = alloc(&d_ctl, 1))) return rc;
    Ctl c0{};
    c0.ff_manual = 1.0;
    c0.ff_last = 1.0;
    FE_CUDA(cudaMemcpy(d_ctl, &c0, sizeof(Ctl), cudaMemcpyHostToDevice));
    D.ctl = d_ctl;
    fill_prm();
    if ((rc = alloc(&d_desc, 1))) return rc;
    std::vector<int2> work(nbk);
    for (int b = 0; b < nbk; ++b) work[b] = make_int2(0, b);
    if ((rc = upload_vec(&d_work, work))) return rc;
    std::vector<int2> cwork(D.nchunks);
    for (int b = 0; b < D.nchunks; ++b) cwork[b] = make_int2(0, b);
    if ((rc = upload_vec(&d_cwork, cwork))) return rc;
    FE_DISPATCH(*this, rc = set_attrs<S FE_COMMA Sh>());
    if (rc) return rc;
    FE_CUDA(cudaMallocHost(&h_stats, 6 * sizeof(double)));
    FE_CUDA(cudaEventCreateWithFlags(&ev_stats, cudaEventDisableTiming));
    FE_DISPATCH(*this, rc = alloc_tiles<Sh>());
    if (rc) return rc;
    if ((rc = upload_desc())) return rc;
    FE_DISPATCH(*this, (k_build_tiles<Sh><<<nbk, CTA, 0, stream>>>(d_desc, d_work, wide)));
    FE_CUDA(cudaGetLastError());
    FE_CUDA(cudaStreamSynchronize(stream));
    return FE_OK;
  }

  // Halo-1 site-index tiles (push targets) and slot lists of every brick,
  // built once on the device by k_build_tiles and read by the stencil passes.
  template <class Sh>
  int alloc_tiles() {
    int32_t* t1;
    uint16_t* sl;
    const size_t nbk = (size_t)hd.nbricks;
    int rc;
    if ((rc = alloc(&t1, nbk * Tile<Sh, 1>::N)) || (rc = alloc(&sl, nbk * Sh::C))) return rc;
    hd.tile1 = t1;
    hd.slots = sl;
    return FE_OK;
  }

  // The dense node grids of c, p, mu, lap(mu) (node coordinates [-2, nb B + 2)
  // per axis; z only for 3-D bricks), the site -> grid entry table, the
  // tensor maps of their halo boxes, and the image positions of fluid nodes.
  int setup_grid(const uint8_t* solid_mask) {
    LatDesc& D = hd;
    const int B[3] = {1 << L.lb[0], 1 << L.lb[1], 1 << L.lb[2]};
    D.hz = L.shape2d ? 0 : 1;
    D.gdx = L.nb[0] * B[0] + 4;
    D.gdy = L.nb[1] * B[1] + 4;
    D.gdz = D.hz ? L.nb[2] * B[2] + 4 : 1;
    D.gsy = D.gdx;
    D.gsz = (int64_t)D.gdx * D.gdy;
    const int64_t cells = D.gsz * D.gdz;
    if (cells >= ((int64_t)1 << 31)) return fe_fail(FE_ERR_ARG, "lattice too large for the 32-bit field grid");
    const size_t es = fld_size();
    for (void** f : {&D.c, &D.p, &D.mu, &D.lapmu, &D.cp}) {
      const size_t bytes = (size_t)cells * es * (f == &D.cp ? 2 : 1);
      unsigned char* q;
      int rc;
      if ((rc = alloc(&q, bytes))) return rc;
      FE_CUDA(cudaMemset(q, 0xff, bytes));  // all-ones: a NaN in FP32 and FP64
      *f = q;
    }
    std::vector<int32_t> dense((size_t)D.n);
    for (int64_t i = 0; i < D.n; ++i) {
      const int64_t node = L.node_of[i];
      const int64_t x = node % D.nx, y = (node / D.nx) % D.ny, z = node / ((int64_t)D.nx * D.ny);
      dense[i] = (int32_t)((x + 2) + D.gsy * (y + 2) + D.gsz * (z + 2 * D.hz));
    }
    int32_t* dd;
    int rc;
    if ((rc = upload_vec(&dd, dense))) return rc;
    D.dense_of = dd;
    // image positions of fluid nodes: every grid position outside the
    // lattice whose wrapped node is fluid
    std::vector<int2> img;
    const int zlo = D.hz ? -2 : 0, zhi = D.hz ? D.gdz - 2 : 1;
    auto wrapc = [](int c, int n) { c %= n; return c < 0 ? c + n : c; };
    for (int z = zlo; z < zhi; ++z)
      for (int y = -2; y < D.gdy - 2; ++y)
        for (int x = -2; x < D.gdx - 2; ++x) {
          if (x >= 0 && x < D.nx && y >= 0 && y < D.ny && z >= 0 && z < D.nz) continue;
          const int wx = wrapc(x, D.nx), wy = wrapc(y, D.ny), wz = wrapc(z, D.nz);
          if (solid_mask[wx + (int64_t)D.nx * (wy + (int64_t)D.ny * wz)]) continue;
          img.push_back(make_int2((int)((x + 2) + D.gsy * (y + 2) + D.gsz * (z + 2 * D.hz)),
                                  (int)((wx + 2) + D.gsy * (wy + 2) + D.gsz * (wz + 2 * D.hz))));
        }
    int2* di;
    if ((rc = upload_vec(&di, img))) return rc;
    D.images = di;
    D.n_images = (int64_t)img.size();
    D.image_blocks = (int)((img.size() + IMG_BLOCK - 1) / IMG_BLOCK);
    std::vector<int2> iw(std::max(D.image_blocks, 1));
    for (int b = 0; b < D.image_blocks; ++b) iw[b] = make_int2(0, b);
    if ((rc = upload_vec(&d_iwork, iw))) return rc;
    FE_DISPATCH(*this, rc = build_tmaps<S FE_COMMA Sh>());
    return rc;
  }

  // Tensor maps of the halo boxes: c with halo 1 (P2), mu with halo 1 (P3),
  // the (c', p') pairs and lap(mu) with halo 2 (P4); x halo 2 in every box.
  // A node of the pair grid is one 8-byte element (FP32 pairs) or two (FP64
  // pairs); the copy moves bits, so the element type only sets the size.
  template <class S, class Sh>
  int build_tmaps() {
    using F = typename S::fld;
    auto enc = tmap_encoder();
    if (!enc) return fe_fail(FE_ERR_CUDA, "cuTensorMapEncodeTiled not available from the driver");
    const LatDesc& D = hd;
    alignas(64) CUtensorMap maps[TM_N];
    auto make = [&](int id, void* base, int H, size_t node_bytes) -> int {
      const size_t es = node_bytes >= 8 ? 8 : 4, xm = node_bytes / es;
      const cuuint64_t dims[3] = {(cuuint64_t)D.gdx * xm, (cuuint64_t)D.gdy, (cuuint64_t)D.gdz};
      const cuuint64_t strides[2] = {(cuuint64_t)D.gdx * node_bytes, (cuuint64_t)D.gsz * node_bytes};
      const cuuint32_t box[3] = {(cuuint32_t)((Sh::BX + 4) * xm), (cuuint32_t)(Sh::BY + 2 * H),
                                 (cuuint32_t)(D.hz ? Sh::BZ + 2 * H : 1)};
      const cuuint32_t estr[3] = {1, 1, 1};
      const CUresult r = enc(&maps[id], es == 8 ? CU_TENSOR_MAP_DATA_TYPE_UINT64 : CU_TENSOR_MAP_DATA_TYPE_UINT32,
                             3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                             CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                             CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
      if (r != CUDA_SUCCESS) return fe_fail(FE_ERR_CUDA, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
      return FE_OK;
    };
    int rc;
    if ((rc = make(TM_C1, D.c, 1, sizeof(F))) || (rc = make(TM_CP2, D.cp, 2, 2 * sizeof(F))) ||
        (rc = make(TM_MU1, D.mu, 1, sizeof(F))) || (rc = make(TM_L2, D.lapmu, 2, sizeof(F))))
      return rc;
    unsigned char* q;
    if ((rc = alloc(&q, sizeof(maps)))) return rc;
    FE_CUDA(cudaMemcpy(q, maps, sizeof(maps), cudaMemcpyHostToDevice));
    hd.tmap = q;
    return FE_OK;
  }

  // Dynamic shared memory of the collide pass (CollideSmem).
  template <class S, class Sh>
  int set_attrs() {
    smem_p4 = CollideSmem<S, Sh>::BYTES;
    FE_CUDA((collide_smem_attr<S, Sh>((int)smem_p4)));
    return FE_OK;
  }

  // ---- one step (plain launches) -----------------------------------------
  template <class S>
  void launch_bc(cudaStream_t st) {
    const int nio = hd.n_inlet + hd.n_outlet, nb = hd.n_buf, nall = nio + nb;
    if (nio) { k_bc_fields<S><<<(nio + 127) / 128, 128, 0, st>>>(d_desc, 0); ++launches; }
    if (nb) { k_bc_buffers<S><<<(nb + 127) / 128, 128, 0, st>>>(d_desc, 0); ++launches; }
    if (nall) { k_bc_final<S><<<(nall + 127) / 128, 128, 0, st>>>(d_desc, 0); ++launches; }
  }
  template <class S, class Sh>
  void launch_step_t(int par, cudaStream_t st, cudaEvent_t* ev) {
    const int nb = hd.nbricks;
    auto rec = [&](int q) { if (ev) cudaEventRecord(ev[q], st); };
    using F = typename S::fld;
    rec(0);
    if (aa && par) launch_moments_aa<S, Sh>(nb, 0, st, d_desc, d_work);
    else k_moments<S><<<hd.nchunks, CTA, 0, st>>>(d_desc, d_cwork, par, 0);
    rec(1);
    if (open_bnd) launch_bc<S>(st);
    if (hd.image_blocks) k_images<F><<<hd.image_blocks, CTA, 0, st>>>(d_desc, d_iwork, GF_C);
    rec(2);
    launch_cfield<S, Sh, 0>(hd.prm.hbb != 0, nb, st, d_desc, d_work, FieldOut{});
    if (hd.image_blocks) k_images<F><<<hd.image_blocks, CTA, 0, st>>>(d_desc, d_iwork, GF_MU | GF_CP);
    rec(3);
    launch_lapmu<S, Sh>(hd.prm.hbb != 0, nb, st, d_desc, d_work);
    if (hd.image_blocks) k_images<F><<<hd.image_blocks, CTA, 0, st>>>(d_desc, d_iwork, GF_LAPMU);
    rec(4);
    launch_collide<S, Sh>(collide_variant(), hd.prm.hbb != 0, wide != 0, nb, smem_p4, st, d_desc, d_work, par,
                          aa ? 1 + par : 0);
    rec(5);
    launches += hd.image_blocks ? 7 : 4;
  }
  void launch_step(int par, cudaStream_t st, cudaEvent_t* ev = nullptr) {
    FE_DISPATCH(*this, launch_step_t<S FE_COMMA Sh>(par, st, ev));
  }
  int kernels_per_step() const {
    int k = hd.image_blocks ? 7 : 4;  // four passes (and three image refreshes)
    if (open_bnd) {
      const int nio = hd.n_inlet + hd.n_outlet;
      k += (nio ? 1 : 0) + (hd.n_buf ? 1 : 0) + (nio + hd.n_buf ? 1 : 0);
    }
    return k;
  }

  // run_mode 1: fe_run (corrections queued after each step, forcing factor
  // from the step counter); 0: fe_step (factor ff); 2: a field refresh
  // without a step (no correction queued, the last step's factor)
  int set_ctl_mode(int run_mode, double ff) {
    if (run_mode != 2) step_mode = run_mode;
    if (run_mode == ctl_mode && ff == ctl_ff) return FE_OK;  // already on the device
    // auto_correct, ff_auto, ff_manual are contiguous in Ctl
    struct { int32_t auto_correct, ff_auto; double ff_manual; } m{run_mode == 1 ? 1 : 0, run_mode, ff};
    static_assert(offsetof(Ctl, ff_auto) == offsetof(Ctl, auto_correct) + 4, "Ctl layout");
    static_assert(offsetof(Ctl, ff_manual) == offsetof(Ctl, auto_correct) + 8, "Ctl layout");
    FE_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(d_ctl) + offsetof(Ctl, auto_correct), &m, sizeof(m),
                            cudaMemcpyHostToDevice, stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    ctl_mode = run_mode;
    ctl_ff = ff;
    return FE_OK;
  }

  int step(int nsteps) {
    int rc;
    const int64_t before = state_id;
    if ((rc = tracer_hook(nsteps, before, false))) return rc;
    if ((rc = set_ctl_mode(0, ff_manual))) return rc;
    for (int s = 0; s < nsteps; ++s) {
      launch_step(parity, stream);
      parity ^= 1;
    }
    FE_CUDA(cudaGetLastError());
    t_host += nsteps;
    state_id += nsteps;
    return tracer_hook(nsteps, before, true);
  }

  int build_graphs() {
    for (int p = 0; p < 2; ++p) {
      for (int len = 1; len <= 2; ++len) {
        cudaGraph_t g;
        FE_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        const int64_t saved = launches;
        const int steps = len == 1 ? 1 : graph_steps;
        for (int s = 0; s < steps; ++s) launch_step(p ^ (s & 1), stream);
        launches = saved;
        cudaError_t e1 = cudaStreamEndCapture(stream, &g);
        if (e1 != cudaSuccess) return fe_fail(FE_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e1));
        cudaGraphExec_t ex;
        cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) return fe_fail(FE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
        (len == 1 ? graph1 : graph2)[p] = ex;
      }
    }
    return FE_OK;
  }
  void drop_graphs() {
    for (int p = 0; p < 2; ++p) {
      if (graph1[p]) cudaGraphExecDestroy(graph1[p]);
      if (graph2[p]) cudaGraphExecDestroy(graph2[p]);
      graph1[p] = graph2[p] = nullptr;
    }
  }

  int run(int nsteps) {
    int rc;
    const int64_t before = state_id;
    if ((rc = tracer_hook(nsteps, before, false))) return rc;
    if ((rc = set_ctl_mode(1, ff_manual))) return rc;
    if (!graph1[0] && (rc = build_graphs())) return rc;
    const int kps = kernels_per_step();
    int s = 0;
    while (s < nsteps) {
      if (graph_steps > 1 && nsteps - s >= graph_steps) {
        FE_CUDA(cudaGraphLaunch(graph2[parity], stream));
        s += graph_steps;
        parity ^= graph_steps & 1;
        launches += (int64_t)graph_steps * kps;
      } else {
        FE_CUDA(cudaGraphLaunch(graph1[parity], stream));
        parity ^= 1;
        s += 1;
        launches += kps;
      }
    }
    t_host += nsteps;
    state_id += nsteps;
    FE_CUDA(cudaGetLastError());
    return tracer_hook(nsteps, before, true);
  }

  int ensure_tmp(int64_t len) {
    if (tmp_len >= len) return FE_OK;
    if (d_tmp) cudaFree(d_tmp);
    d_tmp = nullptr;
    tmp_len = 0;
    cudaError_t err = cudaMalloc(&d_tmp, (size_t)len * sizeof(double));
    if (err != cudaSuccess) {
      cudaGetLastError();
      return fe_fail(FE_ERR_MEMORY, "transfer buffer");
    }
    tmp_len = len;
    return FE_OK;
  }

  // The in-place layout's phase 1 turned into the standard layout (phase 0)
  // in place, before a pass that reads each site's own slots.
  template <class S, class Sh>
  void to_standard_t() {
    k_aa_swap<S, Sh><<<hd.nbricks, CTA, 0, stream>>>(d_desc, d_work);
    ++launches;
  }
  int to_standard() {
    if (!aa || parity == 0) return FE_OK;
    FE_DISPATCH(*this, to_standard_t<S FE_COMMA Sh>());
    FE_CUDA(cudaGetLastError());
    parity = 0;
    return FE_OK;
  }

  int mass_pass() {
    int rc;
    if ((rc = to_standard())) return rc;
    FE_DISPATCH(*this, (k_mass<S><<<hd.nchunks, CTA, 0, stream>>>(d_desc, d_cwork, parity, d_partm)));
    ++launches;
    FE_CUDA(cudaGetLastError());
    return FE_OK;
  }

  // Queue the order-parameter mass correction for the next step: the flag is
  // set by a one-thread kernel in stream order, so the host does not wait.
  int queue_correction() {
    k_queue_correction<<<1, 1, 0, stream>>>(d_ctl);
    ++launches;
    FE_CUDA(cudaGetLastError());
    return FE_OK;
  }

  // The control block, and the problems the kernels recorded in it: tile
  // copies of a stencil pass that did not land (bits 4, 8) or a non-finite
  // velocity in the collision pass (bit 1).
  int read_ctl(Ctl* c) {
    FE_CUDA(cudaMemcpyAsync(c, d_ctl, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    if (c->status & 12)
      return fe_fail(FE_ERR_CUDA, "a stencil pass's tile copies did not complete (status " + std::to_string(c->status) + ")");
    if (c->status & 1) return fe_fail(FE_ERR_DIVERGED, "non-finite velocity in the collision pass");
    return FE_OK;
  }
  int write_ctl_field(size_t off, const void* v, size_t sz) {
    FE_CUDA(cudaMemcpyAsync(reinterpret_cast<char*>(d_ctl) + off, v, sz, cudaMemcpyHostToDevice, stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    return FE_OK;
  }

  int download(double* h, double* g) {
    const int64_t Vn = (int64_t)Q * hd.n;
    int rc;
    if ((rc = ensure_tmp(2 * Vn))) return rc;
    if ((rc = to_standard())) return rc;
    Ctl c;
    if ((rc = read_ctl(&c))) return rc;
    int apply = 0;
    if (c.pending && hd.prm.correct_mass) {
      if ((rc = mass_pass())) return rc;
      apply = 1;
    }
    Staging* sg = narrow_transfers(Vn);
    if (sg) {  // FP32 values on the link, widened on the host (exact)
      float* t = reinterpret_cast<float*>(d_tmp);
      FE_DISPATCH(*this, (k_download_state<S, float><<<hd.nchunks, CTA, 0, stream>>>(d_desc, d_cwork, parity, t,
                                                                                         t + Vn, apply)));
      ++launches;
      FE_CUDA(cudaGetLastError());
      FE_CUDA(sg->to_host_widen(h, t, (size_t)Vn, stream));
      FE_CUDA(sg->to_host_widen(g, t + Vn, (size_t)Vn, stream));
    } else {
      FE_DISPATCH(*this, (k_download_state<S><<<hd.nchunks, CTA, 0, stream>>>(d_desc, d_cwork, parity, d_tmp,
                                                                                    d_tmp + Vn, apply)));
      ++launches;
      FE_CUDA(cudaGetLastError());
      FE_CUDA(copy_to_host(h, d_tmp, Vn * sizeof(double)));
      FE_CUDA(copy_to_host(g, d_tmp + Vn, Vn * sizeof(double)));
    }
    FE_CUDA(cudaStreamSynchronize(stream));
    return FE_OK;
  }
  // The staging area for state transfers of Vn values per lattice in FP32
  // (storages whose arithmetic is FP32: their values are FP32 numbers, so
  // narrowing on the host is what the device's conversion does and widening
  // is exact), or nullptr for the FP64 path (also taken under
  // FELBM_FP64_TRANSFERS=1, for tests).
  Staging* narrow_transfers(int64_t Vn) const {
    if (storage == FE_F64 || (size_t)Vn * sizeof(float) < (size_t(4) << 20)) return nullptr;
    const char* w = std::getenv("FELBM_FP64_TRANSFERS");
    if (w && w[0] == '1') return nullptr;
    return Staging::get();
  }
  // Large transfers through the pinned staging buffers (plain copies if
  // those cannot be allocated).
  cudaError_t copy_to_host(void* dst, const void* src, size_t bytes) {
    Staging* s = bytes >= (size_t(4) << 20) ? Staging::get() : nullptr;
    return s ? s->to_host(dst, src, bytes, stream) : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, stream);
  }
  cudaError_t copy_to_device(void* dst, const void* src, size_t bytes) {
    Staging* s = bytes >= (size_t(4) << 20) ? Staging::get() : nullptr;
    return s ? s->to_device(dst, src, bytes, stream) : cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, stream);
  }

  // A queued mass correction written into the stored h now (instead of at
  // the next pass); the queue is then empty.
  int settle_correction() {
    Ctl c;
    int rc;
    if ((rc = tracer_hook(-1, state_id, false))) return rc;
    if ((rc = read_ctl(&c))) return rc;
    if (!c.pending || !hd.prm.correct_mass) return FE_OK;
    if ((rc = mass_pass())) return rc;  // (in the standard layout from here)
    FE_DISPATCH(*this, (k_inject<S><<<hd.nchunks, CTA, 0, stream>>>(d_desc, d_cwork, parity)));
    ++launches;
    FE_CUDA(cudaGetLastError());
    struct { int32_t pending; } z{0};
    if ((rc = write_ctl_field(offsetof(Ctl, pending), &z, 4))) return rc;
    double zero = 0.0;
    return write_ctl_field(offsetof(Ctl, lambda), &zero, 8);
  }

  int upload(const double* h, const double* g) {
    const int64_t Vn = (int64_t)Q * hd.n;
    int rc;
    if ((rc = tracer_hook(-1, state_id, false))) return rc;  // deferred tracer advances see the old state
    ++state_id;
    if ((rc = ensure_tmp(2 * Vn))) return rc;
    if (aa) parity = 0;  // the upload writes the standard layout
    Staging* sg = narrow_transfers(Vn);
    if (sg) {  // narrowed on the host, as the device's conversion would
      float* t = reinterpret_cast<float*>(d_tmp);
      FE_CUDA(sg->to_device_narrow(t, h, (size_t)Vn, stream));
      FE_CUDA(sg->to_device_narrow(t + Vn, g, (size_t)Vn, stream));
      FE_DISPATCH(*this, (k_upload_state<S, float><<<hd.nchunks, CTA, 0, stream>>>(d_desc, d_cwork, parity, t,
                                                                                       t + Vn)));
    } else {
      FE_CUDA(copy_to_device(d_tmp, h, Vn * sizeof(double)));
      FE_CUDA(copy_to_device(d_tmp + Vn, g, Vn * sizeof(double)));
      FE_DISPATCH(*this, (k_upload_state<S><<<hd.nchunks, CTA, 0, stream>>>(d_desc, d_cwork, parity, d_tmp,
                                                                                  d_tmp + Vn)));
    }
    ++launches;
    FE_CUDA(cudaGetLastError());
    int32_t zero = 0;
    if ((rc = write_ctl_field(offsetof(Ctl, pending), &zero, 4))) return rc;
    FE_CUDA(cudaStreamSynchronize(stream));
    return FE_OK;
  }

  // The equilibrium state at rest of per-site c and p (reference site order;
  // p null: p_uniform), built on the device from n (or 2n) uploaded values
  // instead of the 38n of a host-built state; the same state as upload() of
  // fe_init_equilibrium's arrays.
  int upload_equilibrium(const double* c, const double* p, double p_uniform) {
    const int64_t n = hd.n;
    int rc;
    if ((rc = tracer_hook(-1, state_id, false))) return rc;
    ++state_id;
    if ((rc = ensure_tmp(2 * n))) return rc;
    if (aa) parity = 0;
    FE_CUDA(copy_to_device(d_tmp, c, n * sizeof(double)));
    if (p) FE_CUDA(copy_to_device(d_tmp + n, p, n * sizeof(double)));
    FE_DISPATCH(*this, (k_upload_equilibrium<S><<<hd.nchunks, CTA, 0, stream>>>(d_desc, d_cwork, parity, d_tmp,
                                                                                   p ? d_tmp + n : nullptr,
                                                                                   p_uniform)));
    ++launches;
    FE_CUDA(cudaGetLastError());
    int32_t zero = 0;
    if ((rc = write_ctl_field(offsetof(Ctl, pending), &zero, 4))) return rc;
    FE_CUDA(cudaStreamSynchronize(stream));
    return FE_OK;
  }

  // download()/download_raw(): P1 (+BC) and P2 in output mode, no step.
  // OUT 1: reference site order; OUT 2: node-indexed grids.
  template <class S, class Sh, int OUT>
  void fields_launch(FieldOut o) {
    if (aa && parity) {
      launch_moments_aa<S, Sh>(hd.nbricks, 1, stream, d_desc, d_work);
    } else {
      k_moments<S><<<hd.nchunks, CTA, 0, stream>>>(d_desc, d_cwork, parity, 1);
    }
    if (open_bnd) launch_bc<S>(stream);
    if (hd.image_blocks)
      k_images<typename S::fld><<<hd.image_blocks, CTA, 0, stream>>>(d_desc, d_iwork, GF_C);
    launch_cfield<S, Sh, OUT>(hd.prm.hbb != 0, hd.nbricks, stream, d_desc, d_work, o);
    launches += hd.image_blocks ? 3 : 2;
  }
  // Corrected velocity of the current state into node-indexed device grids
  // (solid nodes are left as they are), on the engine stream.
  // The forcing factor is the one the next step takes (the mode of the last
  // stepping call), as in the velocity the next step's field pass forms.
  int velocity_grid(double* ux, double* uy, double* uz, double* c = nullptr) {
    int rc;
    if ((rc = set_ctl_mode(step_mode, ff_manual))) return rc;
    FieldOut o{nullptr, c, ux, uy, uz, nullptr, nullptr};
    FE_DISPATCH(*this, (fields_launch<S FE_COMMA Sh FE_COMMA 2>(o)));
    FE_CUDA(cudaGetLastError());
    double zero = 0.0;  // as fields(): the step recomputes lambda
    return write_ctl_field(offsetof(Ctl, lambda), &zero, 8);
  }
  int fields(const fe_fields* f) {
    const int64_t n = hd.n;
    int rc;
    if ((rc = ensure_tmp(7 * n))) return rc;
    // the moment pass forms the lambda of a queued correction (the pending flag
    // stays set: no collision runs, so the correction is still owed); the
    // forcing factor is the last step's
    if ((rc = set_ctl_mode(2, ff_manual))) return rc;
    FieldOut o{d_tmp + 0 * n, d_tmp + 1 * n, d_tmp + 2 * n, d_tmp + 3 * n, d_tmp + 4 * n, d_tmp + 5 * n,
               d_tmp + 6 * n};
    FE_DISPATCH(*this, (fields_launch<S FE_COMMA Sh FE_COMMA 1>(o)));
    FE_CUDA(cudaGetLastError());
    double* dst[7] = {f->rho, f->c, f->ux, f->uy, f->uz, f->p, f->mu};
    for (int q = 0; q < 7; ++q)
      if (dst[q]) FE_CUDA(copy_to_host(dst[q], d_tmp + q * n, n * sizeof(double)));
    FE_CUDA(cudaStreamSynchronize(stream));
    double zero = 0.0;
    return write_ctl_field(offsetof(Ctl, lambda), &zero, 8);
  }

  int stats_launch() {
    FE_DISPATCH(*this, (k_stats_finalize<Sh><<<STATS_BLOCKS, CTA, 0, stream>>>(d_desc, 0, d_stats_blk)));
    ++launches;
    FE_CUDA(cudaGetLastError());
    FE_CUDA(cudaMemcpyAsync(h_stats, reinterpret_cast<char*>(d_ctl) + offsetof(Ctl, stats), 6 * sizeof(double),
                            cudaMemcpyDeviceToHost, stream));
    FE_CUDA(cudaEventRecord(ev_stats, stream));
    stats_pending = true;
    return FE_OK;
  }
  int stats_collect(double out[6]) {
    if (!stats_pending) return fe_fail(FE_ERR_STATE, "no flow statistics pending");
    FE_CUDA(cudaEventSynchronize(ev_stats));
    for (int q = 0; q < 6; ++q) out[q] = h_stats[q];
    stats_pending = false;
    return FE_OK;
  }
};

// ---------------------------------------------------------------------------
// Batch: many lattices advanced together, one launch per pass over the
// concatenated work lists of all members (P1 over their site chunks, P2-P4
// over their bricks, grouped by brick shape and collision kind), captured as
// CUDA graphs. Members keep their own buffers, control blocks and
// reductions; every kernel finds its lattice through the work item, so the
// result of a member is the one it gets alone. A rebuild (membership change,
// or a member stepped on its own) maps each member's current buffer to slot
// 0 of its batch descriptor, so the batch parity is uniform.
// ---------------------------------------------------------------------------
struct Batch {
  struct Group {
    int shape = 0, mrt = 0, hbb = 0, wide = 0, aa = 0;
    int2* d_work = nullptr;
    int nwork = 0;
  };
  int device = 0;
  int storage = -1;
  cudaStream_t stream = nullptr;
  std::vector<Engine*> mem;
  std::vector<int> join_parity;     // member parity at the last rebuild
  std::vector<Group> groups;
  LatDesc* d_desc = nullptr;
  int2* d_cwork = nullptr;
  int2* d_gwork = nullptr;          // the groups' work lists, one after another
  int2* d_iwork = nullptr;          // the members' image-refresh blocks
  int2* d_cwork_std = nullptr;      // chunks of the two-buffer members
  int2* d_bwork_aa = nullptr;       // bricks of the in-place members (their phase-1 P1)
  size_t cap_desc = 0, cap_cwork = 0, cap_gwork = 0, cap_iwork = 0;  // bytes (grow-only)
  size_t cap_cwork_std = 0, cap_bwork_aa = 0;
  int ncwork = 0, niwork = 0, ncwork_std = 0, nbwork_aa = 0;
  int aa_off[NSHAPE] = {}, aa_cnt[NSHAPE] = {};  // the in-place bricks of each shape in d_bwork_aa
  int64_t since_build = 0;          // steps since the last rebuild
  bool dirty = true;
  int64_t same_members = 0;  // launches since the last membership change
  int inflight = 0;                 // steps launched by fe_batch_launch, not yet waited for
  cudaGraphExec_t graph1[2] = {nullptr, nullptr};
  cudaGraphExec_t graph2[2] = {nullptr, nullptr};  // graph_steps steps
  int64_t launches = 0;

  ~Batch() {
    if (stream) cudaStreamSynchronize(stream);
    if (inflight) finish(inflight);
    inflight = 0;
    settle();
    for (Engine* e : mem) e->owner = nullptr;
    drop_graphs();
    free_arrays();
    if (stream) cudaStreamDestroy(stream);
  }
  void free_arrays() {
    for (void* a : {(void*)d_desc, (void*)d_cwork, (void*)d_gwork, (void*)d_iwork, (void*)d_cwork_std,
                    (void*)d_bwork_aa})
      if (a) cudaFree(a);
    groups.clear();
    d_desc = nullptr;
    d_cwork = d_gwork = d_iwork = d_cwork_std = d_bwork_aa = nullptr;
    cap_desc = cap_cwork = cap_gwork = cap_iwork = cap_cwork_std = cap_bwork_aa = 0;
    ncwork = niwork = ncwork_std = nbwork_aa = 0;
  }
  void drop_graphs() {
    for (int p = 0; p < 2; ++p) {
      if (graph1[p]) cudaGraphExecDestroy(graph1[p]);
      if (graph2[p]) cudaGraphExecDestroy(graph2[p]);
      graph1[p] = graph2[p] = nullptr;
    }
  }
  int create(int dev) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) {
      cudaGetLastError();
      return fe_fail(FE_ERR_NO_DEVICE, "no CUDA device");
    }
    if (dev >= 0) FE_CUDA(cudaSetDevice(dev));
    FE_CUDA(cudaGetDevice(&device));
    FE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    return FE_OK;
  }
  int find(const Engine* e) const {
    for (size_t q = 0; q < mem.size(); ++q)
      if (mem[q] == e) return (int)q;
    return -1;
  }
  int add(Engine* e) {
    if (inflight) return fe_fail(FE_ERR_STATE, "batch steps in flight (fe_batch_wait first)");
    if (find(e) >= 0) return fe_fail(FE_ERR_STATE, "engine already in the batch");
    if (e->owner) return fe_fail(FE_ERR_STATE, "engine is a member of another batch");
    if (e->device != device) return fe_fail(FE_ERR_ARG, "engine and batch on different devices");
    if (storage >= 0 && e->storage != storage) return fe_fail(FE_ERR_ARG, "a batch holds one storage type");
    int rc;
    if ((rc = e->tracer_hook(-1, e->state_id, false))) return rc;  // batch steps do not run tracer advances
    storage = e->storage;
    cudaStreamSynchronize(e->stream);
    e->owner = this;
    mem.push_back(e);
    dirty = true;
    return FE_OK;
  }
  int remove(Engine* e) {
    const int q = find(e);
    if (q < 0) return fe_fail(FE_ERR_STATE, "engine not in the batch");
    if (inflight) {  // a member that goes away: finish the steps in flight first
      int rc;
      if ((rc = wait())) return rc;
    }
    FE_CUDA(cudaStreamSynchronize(stream));
    settle();
    e->owner = nullptr;
    mem.erase(mem.begin() + q);
    if (q < (int)join_parity.size()) join_parity.erase(join_parity.begin() + q);
    if (mem.empty()) storage = -1;
    dirty = true;
    return FE_OK;
  }
  // members' own parity after the batch steps since the rebuild
  void settle() {
    if (dirty) return;  // no batch step since the members' parity was read
    for (size_t q = 0; q < mem.size() && q < join_parity.size(); ++q)
      mem[q]->parity = join_parity[q] ^ (int)(since_build & 1);
  }
  // Copies v to *p, growing the buffer (capacity *cap bytes) only when it is
  // too small, so membership changes allocate and free nothing.
  template <class T>
  int upload_vec(T** p, size_t* cap, const std::vector<T>& v) {
    const size_t bytes = std::max<size_t>(v.size(), 1) * sizeof(T);
    if (bytes > *cap) {
      if (*p) cudaFree(*p);
      *p = nullptr;
      *cap = 0;
      void* q = nullptr;
      const size_t want = bytes + bytes / 2;
      if (cudaMalloc(&q, want) != cudaSuccess) {
        cudaGetLastError();
        return fe_fail(FE_ERR_MEMORY, "batch arrays");
      }
      *p = static_cast<T*>(q);
      *cap = want;
    }
    if (!v.empty()) FE_CUDA(cudaMemcpy(*p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return FE_OK;
  }
  int rebuild() {
    drop_graphs();
    groups.clear();
    since_build = 0;
    join_parity.assign(mem.size(), 0);
    std::vector<LatDesc> descs(mem.size());
    std::vector<int2> cw, cws, bwa, iw;
    int rc;
    for (size_t q = 0; q < mem.size(); ++q) {
      Engine* e = mem[q];
      // an in-place member joins in the standard layout, so the batch's step
      // parity is its phase
      if ((rc = e->to_standard())) return rc;
      FE_CUDA(cudaStreamSynchronize(e->stream));
      join_parity[q] = e->parity;
      LatDesc d = e->hd;
      for (int f = 0; f < 2; ++f) {
        d.pop[0][f] = e->hd.pop[e->parity][f];
        d.pop[1][f] = e->hd.pop[e->parity ^ 1][f];
      }
      descs[q] = d;
      for (int c = 0; c < d.nchunks; ++c) cw.push_back(make_int2((int)q, c));
      if (!e->aa)
        for (int c = 0; c < d.nchunks; ++c) cws.push_back(make_int2((int)q, c));
      for (int b = 0; b < d.image_blocks; ++b) iw.push_back(make_int2((int)q, b));
      if ((rc = e->set_ctl_mode(1, e->ff_manual))) return rc;  // queued correction, forcing from t
    }
    std::vector<int2> gw;
    std::vector<size_t> offs;
    // one group per collide variant, so each member runs the kernel it runs
    // alone (the offset width included: it decides what a member's push-target
    // tiles hold)
    for (int sh = 0; sh < NSHAPE; ++sh)
      for (int mrt = 0; mrt < 4; ++mrt)
        for (int hbb = 0; hbb < 2; ++hbb)
          for (int wd = 0; wd < 2; ++wd)
            for (int aa = 0; aa < 2; ++aa) {
              const size_t off = gw.size();
              for (size_t q = 0; q < mem.size(); ++q)
                if (mem[q]->shape == sh && mem[q]->collide_variant() == mrt &&
                    (mem[q]->hd.prm.hbb != 0) == (hbb != 0) && (mem[q]->wide != 0) == (wd != 0) &&
                    (mem[q]->aa != 0) == (aa != 0))
                  for (int b = 0; b < mem[q]->hd.nbricks; ++b) gw.push_back(make_int2((int)q, b));
              if (gw.size() == off) continue;
              Group g;
              g.wide = wd;
              g.aa = aa;
              g.shape = sh;
              g.mrt = mrt;
              g.hbb = hbb;
              g.nwork = (int)(gw.size() - off);
              groups.push_back(g);
              offs.push_back(off);
            }
    if ((rc = upload_vec(&d_gwork, &cap_gwork, gw))) return rc;
    for (size_t k = 0; k < groups.size(); ++k) groups[k].d_work = d_gwork + offs[k];
    if ((rc = upload_vec(&d_desc, &cap_desc, descs))) return rc;
    if ((rc = upload_vec(&d_cwork, &cap_cwork, cw))) return rc;
    if ((rc = upload_vec(&d_cwork_std, &cap_cwork_std, cws))) return rc;
    // the in-place members' bricks, one run per brick shape
    for (int sh = 0; sh < NSHAPE; ++sh) {
      aa_off[sh] = (int)bwa.size();
      for (size_t q = 0; q < mem.size(); ++q)
        if (mem[q]->aa && mem[q]->shape == sh)
          for (int b = 0; b < mem[q]->hd.nbricks; ++b) bwa.push_back(make_int2((int)q, b));
      aa_cnt[sh] = (int)bwa.size() - aa_off[sh];
    }
    if ((rc = upload_vec(&d_bwork_aa, &cap_bwork_aa, bwa))) return rc;
    if ((rc = upload_vec(&d_iwork, &cap_iwork, iw))) return rc;
    ncwork = (int)cw.size();
    ncwork_std = (int)cws.size();
    nbwork_aa = (int)bwa.size();
    niwork = (int)iw.size();
    dirty = false;
    return FE_OK;
  }

  template <class S, class Sh>
  void launch_group_p2(const Group& g, cudaStream_t st) {
    launch_cfield<S, Sh, 0>(g.hbb != 0, g.nwork, st, d_desc, g.d_work, FieldOut{});
  }
  template <class S, class Sh>
  void launch_group_p3(const Group& g, cudaStream_t st) {
    launch_lapmu<S, Sh>(g.hbb != 0, g.nwork, st, d_desc, g.d_work);
  }
  template <class S, class Sh>
  void launch_group_p4(const Group& g, int par, cudaStream_t st) {
    const size_t sm = CollideSmem<S, Sh>::BYTES;
    launch_collide<S, Sh>(g.mrt, g.hbb != 0, g.wide != 0, g.nwork, sm, st, d_desc, g.d_work, par,
                          g.aa ? 1 + par : 0);
  }
  template <class S>
  void launch_step_t(int par, cudaStream_t st) {
    if (par == 0 || !nbwork_aa) {
      k_moments<S><<<ncwork, CTA, 0, st>>>(d_desc, d_cwork, par, 0);
    } else {  // the in-place members' phase 1: their P1 gathers, per brick shape
      if (ncwork_std) k_moments<S><<<ncwork_std, CTA, 0, st>>>(d_desc, d_cwork_std, par, 0);
      for (int sh = 0; sh < NSHAPE; ++sh)
        if (aa_cnt[sh])
          with_shape<S>(sh, [&](auto t) {
            launch_moments_aa<S, typename decltype(t)::type>(aa_cnt[sh], 0, st, d_desc, d_bwork_aa + aa_off[sh]);
          });
    }
    for (size_t q = 0; q < mem.size(); ++q) {
      const Engine* e = mem[q];
      if (!e->open_bnd) continue;
      const int nio = e->hd.n_inlet + e->hd.n_outlet, nb = e->hd.n_buf, nall = nio + nb;
      if (nio) k_bc_fields<S><<<(nio + 127) / 128, 128, 0, st>>>(d_desc, (int)q);
      if (nb) k_bc_buffers<S><<<(nb + 127) / 128, 128, 0, st>>>(d_desc, (int)q);
      if (nall) k_bc_final<S><<<(nall + 127) / 128, 128, 0, st>>>(d_desc, (int)q);
    }
    using F = typename S::fld;
    if (niwork) k_images<F><<<niwork, CTA, 0, st>>>(d_desc, d_iwork, GF_C);
    for (const Group& g : groups)
      with_shape<S>(g.shape, [&](auto t) { launch_group_p2<S, typename decltype(t)::type>(g, st); });
    if (niwork) k_images<F><<<niwork, CTA, 0, st>>>(d_desc, d_iwork, GF_MU | GF_CP);
    for (const Group& g : groups)
      with_shape<S>(g.shape, [&](auto t) { launch_group_p3<S, typename decltype(t)::type>(g, st); });
    if (niwork) k_images<F><<<niwork, CTA, 0, st>>>(d_desc, d_iwork, GF_LAPMU);
    for (const Group& g : groups)
      with_shape<S>(g.shape, [&](auto t) { launch_group_p4<S, typename decltype(t)::type>(g, par, st); });
  }
  void launch_step(int par, cudaStream_t st) {
    switch (storage) {
      case FE_F64: launch_step_t<StF64>(par, st); break;
      case FE_F32: launch_step_t<StF32>(par, st); break;
      case FE_F16S: launch_step_t<StF16S>(par, st); break;
      case FE_BF16S: launch_step_t<StBF16S>(par, st); break;
      case FE_F16G: launch_step_t<StF16G>(par, st); break;
      default: launch_step_t<StBF16G>(par, st); break;
    }
  }
  // kernels of one step of parity par, the count launch_step_t makes
  int64_t launches_per_step(int par) const {
    int64_t k = 1 + 3 * (int64_t)groups.size() + (niwork ? 3 : 0);
    if (par && nbwork_aa) {
      k -= ncwork_std ? 0 : 1;
      for (int sh = 0; sh < NSHAPE; ++sh) k += aa_cnt[sh] ? 1 : 0;
    }
    for (const Engine* e : mem)
      if (e->open_bnd) {
        const int nio = e->hd.n_inlet + e->hd.n_outlet, nb = e->hd.n_buf;
        k += (nio ? 1 : 0) + (nb ? 1 : 0) + (nio + nb ? 1 : 0);
      }
    return k;
  }
  int build_graphs() {
    for (int p = 0; p < 2; ++p)
      for (int len = 1; len <= 2; ++len) {
        cudaGraph_t g;
        FE_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        for (int s = 0; s < len; ++s) launch_step(p ^ (s & 1), stream);
        cudaError_t e1 = cudaStreamEndCapture(stream, &g);
        if (e1 != cudaSuccess) return fe_fail(FE_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e1));
        cudaGraphExec_t ex;
        cudaError_t e2 = cudaGraphInstantiate(&ex, g, 0);
        cudaGraphDestroy(g);
        if (e2 != cudaSuccess) return fe_fail(FE_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e2));
        (len == 1 ? graph1 : graph2)[p] = ex;
      }
    return FE_OK;
  }
  // descriptors, control blocks and graphs ready for a run
  int prepare() {
    int rc;
    // a member stepped on its own since the rebuild: remap its buffers
    for (size_t q = 0; q < mem.size() && !dirty; ++q)
      if (mem[q]->parity != (join_parity[q] ^ (int)(since_build & 1))) dirty = true;
    if (dirty) {
      if ((rc = rebuild())) return rc;
      same_members = 0;
    } else {
      for (Engine* e : mem) {
        FE_CUDA(cudaStreamSynchronize(e->stream));
        if ((rc = e->set_ctl_mode(1, e->ff_manual))) return rc;
      }
      ++same_members;
    }
    // graphs pay off once a membership is launched again (a request loop
    // changes members often; capturing and instantiating four graphs costs
    // more than the plain launches of one chunk)
    if (!graph1[0] && same_members >= 1 && (rc = build_graphs())) return rc;
    return FE_OK;
  }
  // nsteps on the batch stream (after prepare): graph launches, or plain
  // launches while the membership is new
  int run_async(int nsteps) {
    int par = (int)(since_build & 1);
    int s = 0;
    if (!graph1[0]) {
      for (; s < nsteps; ++s, par ^= 1) {
        launch_step(par, stream);
        launches += launches_per_step(par);
      }
    }
    while (s < nsteps) {
      if (nsteps - s >= 2) {
        FE_CUDA(cudaGraphLaunch(graph2[par], stream));
        s += 2;
        launches += launches_per_step(0) + launches_per_step(1);
      } else {
        FE_CUDA(cudaGraphLaunch(graph1[par], stream));
        launches += launches_per_step(par);
        par ^= 1;
        s += 1;
      }
    }
    FE_CUDA(cudaGetLastError());
    return FE_OK;
  }
  int finish(int nsteps) {
    since_build += nsteps;
    for (Engine* e : mem) {
      e->t_host += nsteps;
      e->state_id += nsteps;
    }
    settle();
    return FE_OK;
  }
  int run(int nsteps) {
    int rc;
    if ((rc = launch(nsteps))) return rc;
    return wait();
  }
  // queue nsteps and return; members must not be used until wait()
  int launch(int nsteps) {
    if (inflight) return fe_fail(FE_ERR_STATE, "batch steps already in flight");
    if (mem.empty() || nsteps == 0) return FE_OK;
    int rc;
    // deferred tracer advances of members use the state before these steps
    for (Engine* e : mem)
      if ((rc = e->tracer_hook(-1, e->state_id, false))) return rc;
    if ((rc = prepare())) return rc;
    if ((rc = run_async(nsteps))) return rc;
    inflight = nsteps;
    return FE_OK;
  }
  int wait() {
    if (!inflight) return FE_OK;
    const int n = inflight;
    inflight = 0;
    FE_CUDA(cudaStreamSynchronize(stream));
    return finish(n);
  }
};

// ---------------------------------------------------------------------------
// Tracers of one engine (tracers.cuh): positions, diffusivities and ids on
// the device, advected on a node-indexed snapshot of the engine's velocity.
// ---------------------------------------------------------------------------
struct Tracers {
  Engine* E = nullptr;
  TracerDesc T{};
  std::vector<void*> allocs;
  int velocity_skip = 1;
  int64_t step = 0;             // tracer steps taken
  bool have_u = false;
  bool frozen = false;          // a caller-given velocity snapshot (fe_tracers_set_velocity)
  bool pending = false;         // an advance waits for the engine's next single step
  int64_t grid_for = -1;        // engine state whose velocity the snapshot holds
  cudaStream_t stream = nullptr;
  // stretching time series: rows 1..step, ring of ROWCAP rows on the device
  static constexpr int ROWCAP = 65536;
  double* ring = nullptr;
  int64_t drained = 0;          // rows handed out by rows()
  int blocks = 0;

  ~Tracers() {
    if (E) {
      auto& v = E->tracer_sets;
      v.erase(std::remove(v.begin(), v.end(), this), v.end());
      unfuse();
    }
    if (stream) cudaStreamSynchronize(stream);
    for (void* a : allocs) cudaFree(a);
  }
  // The engine is going away: finish the queued work on its stream and drop
  // both; later calls fail with FE_ERR_STATE.
  void detach() {
    if (stream) cudaStreamSynchronize(stream);
    stream = nullptr;
    E = nullptr;
  }
  // Let the engine's field pass write this set's velocity snapshot on every
  // step (velocity_skip 1, one set per engine, not while in a batch).
  int fuse() {
    if (E->fused || E->owner || velocity_skip != 1 || T.n == 0) return FE_OK;
    E->fused = this;
    for (int a = 0; a < 3; ++a) E->hd.snap_u[a] = const_cast<double*>(T.u[a]);
    E->hd.snap_c = const_cast<double*>(T.cgrid);
    E->hd.prm.need_j = 1;
    return E->upload_desc();
  }
  void unfuse() {
    if (!E || E->fused != this) return;
    E->fused = nullptr;
    for (int a = 0; a < 3; ++a) E->hd.snap_u[a] = nullptr;
    E->hd.snap_c = nullptr;
    E->hd.prm.need_j = (E->P.rho0 != E->P.rho1 || E->open_bnd) ? 1 : 0;
    E->upload_desc();
  }
  template <class T_>
  int alloc(T_** p, size_t count) {
    void* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(count, 1) * sizeof(T_)) != cudaSuccess) {
      cudaGetLastError();
      return fe_fail(FE_ERR_MEMORY, "tracer arrays");
    }
    allocs.push_back(q);
    *p = static_cast<T_*>(q);
    return FE_OK;
  }
  int create(Engine* e, const fe_tracer_config* cfg, int64_t n, const double* pos, const double* dm,
             const int64_t* id) {
    E = e;
    stream = e->stream;
    e->tracer_sets.push_back(this);
    T.n = n;
    T.nx = e->hd.nx;
    T.ny = e->hd.ny;
    T.nz = e->hd.nz;
    T.substeps = cfg->substeps;
    T.order = cfg->order;
    T.seed = cfg->seed;
    T.stretch = cfg->stretching ? 1 : 0;
    blocks = (int)((n + TRC - 1) / TRC);
    velocity_skip = cfg->velocity_skip > 0 ? cfg->velocity_skip : 1;
    const int64_t nodes = (int64_t)T.nx * T.ny * T.nz;
    double *p, *v, *d, *u;
    int64_t* ids;
    uint8_t* sol;
    int rc;
    if ((rc = alloc(&p, 3 * n)) || (rc = alloc(&v, 3 * n)) || (rc = alloc(&d, n)) || (rc = alloc(&ids, n)) ||
        (rc = alloc(&u, 3 * nodes)) || (rc = alloc(&sol, nodes)))
      return rc;
    std::vector<uint8_t> solid(nodes, 1);
    for (int64_t i = 0; i < e->hd.n; ++i) solid[e->L.node_of[i]] = 0;
    for (int64_t q = 0; q < n; ++q) {
      const int64_t x = (int64_t)std::floor(pos[q] + 0.5), y = (int64_t)std::floor(pos[n + q] + 0.5),
                    z = (int64_t)std::floor(pos[2 * n + q] + 0.5);
      if (pos[q] < 0 || pos[q] >= T.nx || pos[n + q] < 0 || pos[n + q] >= T.ny || pos[2 * n + q] < 0 ||
          pos[2 * n + q] >= T.nz)
        return fe_fail(FE_ERR_ARG, "tracer outside the lattice");
      if (solid[(x % T.nx) + T.nx * ((y % T.ny) + (int64_t)T.ny * (z % T.nz))])
        return fe_fail(FE_ERR_ARG, "tracer seeded on a solid node");
      if (!(dm[q] >= 0.0)) return fe_fail(FE_ERR_ARG, "negative diffusivity");
    }
    std::vector<int64_t> idv(n);
    for (int64_t q = 0; q < n; ++q) idv[q] = id ? id[q] : q;
    FE_CUDA(cudaMemcpy(p, pos, 3 * n * sizeof(double), cudaMemcpyHostToDevice));
    FE_CUDA(cudaMemset(v, 0, 3 * n * sizeof(double)));
    FE_CUDA(cudaMemcpy(d, dm, n * sizeof(double), cudaMemcpyHostToDevice));
    FE_CUDA(cudaMemcpy(ids, idv.data(), n * sizeof(int64_t), cudaMemcpyHostToDevice));
    FE_CUDA(cudaMemset(u, 0, 3 * nodes * sizeof(double)));  // solid nodes stay 0
    FE_CUDA(cudaMemcpy(sol, solid.data(), nodes, cudaMemcpyHostToDevice));
    T.pos = p;
    T.vel = v;
    T.dm = d;
    T.id = ids;
    T.solid = sol;
    for (int a = 0; a < 3; ++a) T.u[a] = u + a * nodes;
    if (T.stretch) {
      double *rh, *lr, *part, *cg = nullptr;
      if ((rc = alloc(&rh, 3 * n)) || (rc = alloc(&lr, n)) || (rc = alloc(&part, (size_t)blocks * NSTR)) ||
          (rc = alloc(&ring, (size_t)ROWCAP * NROW)) || (cfg->phase_split && (rc = alloc(&cg, nodes))))
        return rc;
      if (cg) FE_CUDA(cudaMemset(cg, 0xFF, nodes * sizeof(double)));  // NaN on solid nodes
      T.rho_hat = rh;
      T.log_rho = lr;
      T.part = part;
      T.cgrid = cg;
      if (n > 0) k_stretch_init<<<(unsigned)((n + TRC - 1) / TRC), TRC, 0, stream>>>(T, cfg->stretching_seed);
      FE_CUDA(cudaGetLastError());
      FE_CUDA(cudaStreamSynchronize(stream));
    }
    return fuse();
  }
  int refresh() {
    double* u = const_cast<double*>(T.u[0]);
    const int64_t nodes = (int64_t)T.nx * T.ny * T.nz;
    int rc = E->velocity_grid(u, u + nodes, u + 2 * nodes, const_cast<double*>(T.cgrid));
    if (!rc) {
      have_u = true;
      grid_for = E->state_id;
    }
    return rc;
  }
  // A deferred advance now, on a snapshot of the current state.
  int flush() {
    if (!pending) return FE_OK;
    pending = false;
    int rc = refresh();
    return rc ? rc : launch_advance();
  }
  // A caller-given node-indexed velocity [3][nodes] (and order parameter
  // [nodes], optional) used from now on instead of the engine's; u == NULL
  // returns to the engine's velocity.
  int set_velocity(const double* u, const double* c) {
    const int64_t nodes = (int64_t)T.nx * T.ny * T.nz;
    int rc;
    if ((rc = flush())) return rc;
    if (!u) {
      frozen = false;
      have_u = false;
      return FE_OK;
    }
    unfuse();  // the engine must not overwrite the caller's field
    FE_CUDA(cudaMemcpyAsync(const_cast<double*>(T.u[0]), u, 3 * nodes * sizeof(double), cudaMemcpyHostToDevice,
                            stream));
    if (c && T.cgrid)
      FE_CUDA(cudaMemcpyAsync(const_cast<double*>(T.cgrid), c, nodes * sizeof(double), cudaMemcpyHostToDevice,
                              stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    frozen = true;
    have_u = true;
    return FE_OK;
  }
  // One lattice step of the tracers on the engine's current velocity.
  // One lattice step of the tracers on the engine's current velocity. A
  // fused set defers it: the engine's next single step forms that velocity
  // in its field pass, and the advance runs right after it on the engine's
  // stream (same values as a refresh now; anything that needs the tracers
  // earlier flushes the deferred advance through a refresh).
  int advance() {
    int rc;
    if (!frozen && E->fused == this) {
      if (grid_for != E->state_id) {
        if ((rc = flush())) return rc;
        if (grid_for != E->state_id) {
          pending = true;
          return FE_OK;
        }
      }
      return launch_advance();
    }
    if (!frozen && (!have_u || step % velocity_skip == 0))
      if ((rc = refresh())) return rc;
    return launch_advance();
  }
  int launch_advance() {
    if (T.n > 0) {
      k_tracers<<<(unsigned)blocks, TRC, 0, stream>>>(T, step);
      if (T.stretch) k_stretch_row<<<1, 256, 0, stream>>>(T.part, blocks, T.substeps, T.n, step + 1, ring, ROWCAP);
    }
    FE_CUDA(cudaGetLastError());
    ++step;
    return FE_OK;
  }
  // Rows produced since the last call (oldest first), at most max_rows.
  int rows(double* out, int64_t max_rows, int64_t* count) {
    *count = 0;
    int rc;
    if ((rc = flush())) return rc;
    if (!T.stretch) return fe_fail(FE_ERR_STATE, "tracers created without stretching");
    const int64_t made = T.n > 0 ? step : 0;
    if (made - drained > ROWCAP) {
      const int64_t lost = made - drained - ROWCAP;
      drained = made - ROWCAP;
      return fe_fail(FE_ERR_STATE, "stretching rows overwritten before they were read (" + std::to_string(lost) +
                                       " lost; read them at least every " + std::to_string(ROWCAP) + " steps)");
    }
    const int64_t k = std::min<int64_t>(made - drained, std::max<int64_t>(max_rows, 0));
    for (int64_t r = 0; r < k; ++r) {
      const int64_t row = drained + 1 + r;  // rows are numbered from 1
      FE_CUDA(cudaMemcpyAsync(out + r * NROW, ring + (row % ROWCAP) * NROW, NROW * sizeof(double),
                              cudaMemcpyDeviceToHost, stream));
    }
    FE_CUDA(cudaStreamSynchronize(stream));
    drained += k;
    *count = k;
    return FE_OK;
  }
  int stretch_state(double* rho_hat, double* log_rho, bool upload) {
    if (!T.stretch) return fe_fail(FE_ERR_STATE, "tracers created without stretching");
    int rc;
    if ((rc = flush())) return rc;
    const auto dir = upload ? cudaMemcpyHostToDevice : cudaMemcpyDeviceToHost;
    if (rho_hat)
      FE_CUDA(upload ? cudaMemcpyAsync(T.rho_hat, rho_hat, 3 * T.n * sizeof(double), dir, stream)
                     : cudaMemcpyAsync(rho_hat, T.rho_hat, 3 * T.n * sizeof(double), dir, stream));
    if (log_rho)
      FE_CUDA(upload ? cudaMemcpyAsync(T.log_rho, log_rho, T.n * sizeof(double), dir, stream)
                     : cudaMemcpyAsync(log_rho, T.log_rho, T.n * sizeof(double), dir, stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    return FE_OK;
  }
  int download(double* pos, double* vel) {
    int rc;
    if ((rc = flush())) return rc;
    if (pos) FE_CUDA(cudaMemcpyAsync(pos, T.pos, 3 * T.n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    if (vel) FE_CUDA(cudaMemcpyAsync(vel, T.vel, 3 * T.n * sizeof(double), cudaMemcpyDeviceToHost, stream));
    FE_CUDA(cudaStreamSynchronize(stream));
    return FE_OK;
  }
};

// Deferred tracer advances around an engine step (Engine::fused).
int Engine::tracer_hook(int nsteps, int64_t before, bool after) {
  Tracers* t = fused;
  if (!t || !t->pending) return FE_OK;
  if (!after) return nsteps == 1 ? FE_OK : t->flush();
  if (nsteps != 1) return FE_OK;
  // this step's field pass wrote the velocity of the state it started from
  t->pending = false;
  t->grid_for = before;
  t->have_u = true;
  return t->launch_advance();
}

}  // namespace fe

using fe::Engine;

struct fe_engine {
  Engine e;
};

static const char* FE_VERSION = "felbm_b200 0.2 (sm_100a)";

#define FE_GUARD(e) \
  if (!(e)) return fe_fail(FE_ERR_ARG, "null engine")

extern "C" {

const char* fe_last_error(void) { return fe::g_last_error.c_str(); }
const char* fe_version(void) { return FE_VERSION; }

int fe_params_default(fe_params* p) {
  if (!p) return fe_fail(FE_ERR_ARG, "null params");
  std::memset(p, 0, sizeof(*p));
  p->rho0 = 1.0; p->rho1 = 1.0; p->tau0 = 1.0; p->tau1 = 1.0;
  p->interface_width = 4.0; p->surface_tension = 1e-3; p->mobility_coeff = 0.02; p->phi = 0.0;
  p->forcing_timedep = FE_FORCING_CONSTANT; p->forcing_period = 10000.0;
  p->use_mrt = 0; p->mrt_lambda = 0.1875;
  for (int q = 1; q < 7; ++q) p->mrt_rate_mode[q] = fe::mrt_reference_mode(q);
  p->use_halfway_bb = 1;
  p->storage = FE_F64;
  p->c_ref = 0.5; p->p_ref = 1.0;  // p_ref: the initial pressure level p0 = 1
  return fe_params_derive(p);
}

int fe_params_derive(fe_params* p) {
  if (!p) return fe_fail(FE_ERR_ARG, "null params");
  if (p->interface_width <= 0) return fe_fail(FE_ERR_ARG, "interface_width must be > 0");
  p->kappa = 1.5 * p->interface_width * p->surface_tension;
  p->beta = 12.0 * p->surface_tension / p->interface_width;
  p->mobility = p->beta != 0.0 ? p->mobility_coeff / p->beta : 0.0;
  p->bnd_coeff = (std::fabs(p->kappa) < 1e-16) ? 0.0 : p->phi / p->kappa;
  return FE_OK;
}

int fe_engine_create(const fe_params* p, int nx, int ny, int nz, const uint8_t* solid, int device,
                     fe_engine** out) {
  if (!p || !solid || !out || nx < 1 || ny < 1 || nz < 1) return fe_fail(FE_ERR_ARG, "fe_engine_create: bad arguments");
  *out = nullptr;
  fe_engine* e = new (std::nothrow) fe_engine();
  if (!e) return fe_fail(FE_ERR_MEMORY, "host allocation");
  const int rc = e->e.create(p, nx, ny, nz, solid, device);
  if (rc) {
    delete e;
    return rc;
  }
  *out = e;
  return FE_OK;
}

int fe_engine_destroy(fe_engine* e) {
  if (!e) return FE_OK;
  if (e->e.owner) e->e.owner->remove(&e->e);
  for (fe::Tracers* t : std::vector<fe::Tracers*>(e->e.tracer_sets)) t->detach();
  e->e.tracer_sets.clear();
  cudaStreamSynchronize(e->e.stream);
  delete e;
  return FE_OK;
}

int fe_engine_layout(const fe_engine* e, int* brick, int* graph_steps) {
  FE_GUARD(e);
  if (brick) *brick = e->e.shape + 1;
  if (graph_steps) *graph_steps = e->e.graph_steps;
  return FE_OK;
}

int fe_engine_size(const fe_engine* e, int64_t* n, int64_t* vn) {
  FE_GUARD(e);
  if (n) *n = e->e.hd.n;
  if (vn) *vn = (int64_t)fe::Q * e->e.hd.n;
  return FE_OK;
}

void* fe_engine_stream(fe_engine* e) { return e ? (void*)e->e.stream : nullptr; }

int fe_set_params(fe_engine* e, const fe_params* p) {
  FE_GUARD(e);
  if (!p) return fe_fail(FE_ERR_ARG, "null params");
  if (p->storage != e->e.storage) return fe_fail(FE_ERR_ARG, "storage cannot change after create");
  if ((p->pop_layout == FE_POP_IN_PLACE) != (e->e.aa != 0))
    return fe_fail(FE_ERR_ARG, "pop_layout cannot change after create");
  if (p->correct_op_mass && e->e.open_bnd)
    return fe_fail(FE_ERR_ARG, "correct_op_mass must be false with open boundaries");
  // fill_prm leaves the open-boundary block of fe_set_open_bnd untouched
  e->e.P = *p;
  e->e.fill_prm();
  e->e.drop_graphs();
  return e->e.upload_desc();
}

int fe_upload_state(fe_engine* e, const double* h, const double* g, int64_t vn) {
  FE_GUARD(e);
  if (!h || !g || vn != (int64_t)fe::Q * e->e.hd.n) return fe_fail(FE_ERR_ARG, "fe_upload_state: size mismatch");
  return e->e.upload(h, g);
}

int fe_upload_equilibrium(fe_engine* e, const double* c, const double* p, double p_uniform, int64_t n) {
  FE_GUARD(e);
  if (!c || n != e->e.hd.n) return fe_fail(FE_ERR_ARG, "fe_upload_equilibrium: size mismatch");
  return e->e.upload_equilibrium(c, p, p_uniform);
}

int fe_download_state(fe_engine* e, double* h, double* g, int64_t vn) {
  FE_GUARD(e);
  if (!h || !g || vn != (int64_t)fe::Q * e->e.hd.n) return fe_fail(FE_ERR_ARG, "fe_download_state: size mismatch");
  return e->e.download(h, g);
}

int fe_set_open_bnd(fe_engine* e, const fe_open_bnd* b) {
  FE_GUARD(e);
  if (!b) return fe_fail(FE_ERR_ARG, "null open boundary");
  Engine& E = e->e;
  if (E.P.correct_op_mass)
    return fe_fail(FE_ERR_ARG, "correct_op_mass must be false with open boundaries (felbm_gpu_main.cu:245-252)");
  if (E.open_bnd) return fe_fail(FE_ERR_STATE, "open boundaries already set");
  const int64_t n = E.hd.n;
  auto check = [&](const int32_t* a, int cnt) {
    if (cnt < 0 || (cnt > 0 && !a)) return false;
    for (int j = 0; j < cnt; ++j)
      if (a[j] < 0 || a[j] >= n) return false;
    return true;
  };
  if (!check(b->inlet, b->n_inlet) || !check(b->outlet, b->n_outlet) ||
      !check(b->buf_verts, b->n_buf) || !check(b->buf_refs, b->n_buf))
    return fe_fail(FE_ERR_ARG, "fe_set_open_bnd: site index out of range");
  // convert reference-order site indices to engine order
  auto conv = [&](const int32_t* a, int cnt) {
    std::vector<int32_t> v(cnt);
    for (int j = 0; j < cnt; ++j) v[j] = E.L.site_of_ref[a[j]];
    return v;
  };
  const int nbuf = b->copy_to_buffers ? b->n_buf : 0;
  std::vector<int32_t> io = conv(b->inlet, b->n_inlet), out = conv(b->outlet, b->n_outlet);
  io.insert(io.end(), out.begin(), out.end());
  std::vector<int32_t> bv = conv(b->buf_verts, nbuf), br = conv(b->buf_refs, nbuf);
  // node coordinates of inlet, outlet and buffer sites (for k_bc_final)
  std::vector<int32_t> xyz;
  for (const std::vector<int32_t>* lst : {&io, &bv})
    for (int32_t i : *lst) {
      const int64_t node = E.L.node_of[i];
      xyz.push_back((int32_t)(node % E.hd.nx));
      xyz.push_back((int32_t)((node / E.hd.nx) % E.hd.ny));
      xyz.push_back((int32_t)(node / ((int64_t)E.hd.nx * E.hd.ny)));
    }
  // flags (BC_PROC as the is_processed mask, multiphase_gpu.cuh:378-389)
  std::vector<uint8_t> flag(n, 0);
  std::vector<int32_t> src(n, 0);
  const bool in_proc = b->use_in_vel || b->use_in_prs || b->use_in_fluid;
  const bool out_proc = b->use_out_prs || b->use_out_fluid;
  for (int j = 0; j < b->n_inlet; ++j) {
    const int32_t i = io[j];
    flag[i] |= fe::BC_SITE | (in_proc ? fe::BC_PROC : 0) | (b->copy_to_buffers ? 0 : fe::BC_G_OVER);
    src[i] = i;
  }
  for (int j = 0; j < b->n_outlet; ++j) {
    const int32_t i = io[b->n_inlet + j];
    flag[i] |= fe::BC_SITE | (out_proc ? fe::BC_PROC : 0) | (b->copy_to_buffers ? 0 : fe::BC_G_OVER);
    src[i] = i;
  }
  for (int j = 0; j < nbuf; ++j) {
    flag[bv[j]] |= fe::BC_SITE | fe::BC_PROC | fe::BC_G_OVER;
    src[bv[j]] = br[j];
  }
  int rc;
  uint8_t* dflag;
  int32_t *dsrc, *dlist, *dxyz, *dbv = nullptr, *dbr = nullptr;
  double* dcoord = nullptr;
  unsigned char *craw, *ubc;
  if ((rc = E.upload_vec(&dflag, flag))) return rc;
  if ((rc = E.upload_vec(&dsrc, src))) return rc;
  if ((rc = E.upload_vec(&dlist, io))) return rc;
  if ((rc = E.upload_vec(&dxyz, xyz))) return rc;
  if ((rc = E.alloc(&craw, n * E.fld_size()))) return rc;
  if ((rc = E.alloc(&ubc, 3 * n * E.fld_size()))) return rc;
  FE_CUDA(cudaMemset(craw, 0, n * E.fld_size()));
  FE_CUDA(cudaMemset(ubc, 0, 3 * n * E.fld_size()));
  if (b->inlet_coord && b->n_inlet) {
    if ((rc = E.upload_vec(&dcoord, std::vector<double>(b->inlet_coord, b->inlet_coord + b->n_inlet)))) return rc;
  }
  if (nbuf) {
    if ((rc = E.upload_vec(&dbv, bv))) return rc;
    if ((rc = E.upload_vec(&dbr, br))) return rc;
  }
  fe::LatDesc& D = E.hd;
  D.bcflag = dflag; D.bcsrc = dsrc; D.bc_list = dlist; D.bc_coord = dcoord; D.bc_xyz = dxyz;
  D.c_raw_bc = craw; D.u_bc = ubc;
  D.n_inlet = b->n_inlet; D.n_outlet = b->n_outlet; D.n_buf = nbuf;
  D.buf_verts = dbv; D.buf_refs = dbr;
  fe::DevPrm& d = D.prm;
  d.open_bnd = 1; d.copy_to_buf = b->copy_to_buffers;
  d.use_in_vel = b->use_in_vel; d.use_in_prs = b->use_in_prs; d.use_in_fluid = b->use_in_fluid;
  d.use_out_prs = b->use_out_prs; d.use_out_fluid = b->use_out_fluid;
  d.u_in[0] = b->u_in_x; d.u_in[1] = b->u_in_y; d.u_in[2] = b->u_in_z;
  d.p_in = b->p_in; d.p_out = b->p_out; d.c_out_fixed = b->c_out_fixed; d.rho_out_fixed = b->rho_out_fixed;
  d.inlet_c_a = b->inlet_c_a; d.inlet_mode = b->inlet_mode;
  d.inlet_period = b->inlet_period; d.inlet_duty = b->inlet_duty; d.inlet_ramp = b->inlet_ramp;
  d.split_pos = b->split_pos;
  d.need_j = 1;
  E.open_bnd = true;
  E.drop_graphs();
  return E.upload_desc();
}

int fe_step(fe_engine* e, int nsteps) {
  FE_GUARD(e);
  if (nsteps < 0) return fe_fail(FE_ERR_ARG, "nsteps < 0");
  return e->e.step(nsteps);
}

int fe_run(fe_engine* e, int nsteps) {
  FE_GUARD(e);
  if (nsteps < 0) return fe_fail(FE_ERR_ARG, "nsteps < 0");
  return e->e.run(nsteps);
}

int fe_set_time(fe_engine* e, int64_t t) {
  FE_GUARD(e);
  e->e.t_host = t;
  return e->e.write_ctl_field(offsetof(fe::Ctl, t), &t, 8);
}

int fe_get_time(const fe_engine* e, int64_t* t) {
  FE_GUARD(e);
  fe::Ctl c;
  int rc = const_cast<Engine&>(e->e).read_ctl(&c);
  if (rc) return rc;
  if (t) *t = c.t;
  return FE_OK;
}

int fe_set_forcing_factor(fe_engine* e, double ff) {
  FE_GUARD(e);
  e->e.ff_manual = ff;
  return FE_OK;
}

int fe_apply_mass_correction(fe_engine* e, double* drift) {
  FE_GUARD(e);
  Engine& E = e->e;
  if (!E.P.correct_op_mass) {
    if (drift) *drift = 0.0;
    return FE_OK;
  }
  int rc;
  if ((rc = E.queue_correction())) return rc;
  if (!drift) return FE_OK;
  // form M and lambda now so that the drift can be returned
  if ((rc = E.mass_pass())) return rc;
  fe::Ctl c;
  if ((rc = E.read_ctl(&c))) return rc;
  *drift = c.drift;
  return FE_OK;
}

int fe_settle_mass_correction(fe_engine* e) {
  FE_GUARD(e);
  return e->e.settle_correction();
}

int fe_record_target_mass(fe_engine* e) {
  FE_GUARD(e);
  Engine& E = e->e;
  int rc;
  if ((rc = E.mass_pass())) return rc;
  fe::Ctl c;
  if ((rc = E.read_ctl(&c))) return rc;
  // a queued correction moves the total to the old target; record that value
  double m = c.M;
  if (c.pending && E.hd.prm.correct_mass && c.W > 0.0 && c.lambda != 0.0) m = c.M - c.lambda * c.W;
  E.target_mass_host = m;
  return E.write_ctl_field(offsetof(fe::Ctl, target_mass), &m, 8);
}

int fe_set_target_mass(fe_engine* e, double m0) {
  FE_GUARD(e);
  e->e.target_mass_host = m0;
  return e->e.write_ctl_field(offsetof(fe::Ctl, target_mass), &m0, 8);
}

int fe_get_target_mass(const fe_engine* e, double* m0) {
  FE_GUARD(e);
  if (m0) *m0 = e->e.target_mass_host;
  return FE_OK;
}

int fe_current_mass(fe_engine* e, double* m) {
  FE_GUARD(e);
  Engine& E = e->e;
  int rc;
  if ((rc = E.mass_pass())) return rc;
  fe::Ctl c;
  if ((rc = E.read_ctl(&c))) return rc;
  double v = c.M;
  if (c.pending && E.hd.prm.correct_mass && c.W > 0.0 && c.lambda != 0.0) v = c.M - c.lambda * c.W;
  if (m) *m = v;
  return FE_OK;
}

int fe_download_fields(fe_engine* e, const fe_fields* f) {
  FE_GUARD(e);
  if (!f) return fe_fail(FE_ERR_ARG, "null fields");
  return e->e.fields(f);
}

int fe_flow_stats(fe_engine* e, double out[6]) {
  FE_GUARD(e);
  int rc;
  if ((rc = e->e.stats_launch())) return rc;
  return e->e.stats_collect(out);
}
int fe_flow_stats_launch(fe_engine* e) {
  FE_GUARD(e);
  return e->e.stats_launch();
}
int fe_flow_stats_ready(fe_engine* e, int* ready) {
  FE_GUARD(e);
  if (!ready) return fe_fail(FE_ERR_ARG, "null");
  if (!e->e.stats_pending) { *ready = 0; return FE_OK; }
  cudaError_t q = cudaEventQuery(e->e.ev_stats);
  if (q != cudaSuccess && q != cudaErrorNotReady) return fe_fail(FE_ERR_CUDA, cudaGetErrorString(q));
  *ready = (q == cudaSuccess) ? 1 : 0;
  return FE_OK;
}
int fe_flow_stats_collect(fe_engine* e, double out[6]) {
  FE_GUARD(e);
  return e->e.stats_collect(out);
}

int fe_time_run(fe_engine* e, int nsteps, float* ms_total) {
  FE_GUARD(e);
  Engine& E = e->e;
  int rc = E.set_ctl_mode(1, E.ff_manual);
  if (!rc && !E.graph1[0]) rc = E.build_graphs();
  if (rc) return rc;
  cudaEvent_t a, b;
  FE_CUDA(cudaEventCreate(&a));
  FE_CUDA(cudaEventCreate(&b));
  FE_CUDA(cudaStreamSynchronize(E.stream));
  FE_CUDA(cudaEventRecord(a, E.stream));
  rc = E.run(nsteps);
  FE_CUDA(cudaEventRecord(b, E.stream));
  FE_CUDA(cudaEventSynchronize(b));
  float ms = 0.f;
  FE_CUDA(cudaEventElapsedTime(&ms, a, b));
  cudaEventDestroy(a);
  cudaEventDestroy(b);
  if (ms_total) *ms_total = ms;
  return rc;
}

// Per-kernel device time over nsteps plain-launched steps: out[0] P1, [1] the
// open-boundary kernels, [2] P2, [3] P3, [4] P4 (summed ms).
int fe_time_kernels(fe_engine* e, int nsteps, float* ms, int nk) {
  FE_GUARD(e);
  if (!ms || nk < fe::K_N) return fe_fail(FE_ERR_ARG, "need 5 outputs");
  Engine& E = e->e;
  cudaEvent_t ev[6];
  for (auto& x : ev) FE_CUDA(cudaEventCreate(&x));
  for (int q = 0; q < fe::K_N; ++q) ms[q] = 0.f;
  int rc = E.tracer_hook(-1, E.state_id, false);
  if (!rc) rc = E.set_ctl_mode(1, E.ff_manual);
  if (rc) return rc;
  E.state_id += nsteps;
  for (int s = 0; s < nsteps; ++s) {
    E.launch_step(E.parity, E.stream, ev);
    E.parity ^= 1;
    FE_CUDA(cudaEventSynchronize(ev[5]));
    for (int q = 0; q < fe::K_N; ++q) {
      float t = 0.f;
      FE_CUDA(cudaEventElapsedTime(&t, ev[q], ev[q + 1]));
      ms[q] += t;
    }
  }
  E.t_host += nsteps;
  for (auto& x : ev) cudaEventDestroy(x);
  FE_CUDA(cudaGetLastError());
  return FE_OK;
}

int fe_launch_count(const fe_engine* e, int64_t* count) {
  FE_GUARD(e);
  if (count) *count = e->e.launches;
  return FE_OK;
}

// ---- batches ---------------------------------------------------------------
struct fe_batch {
  fe::Batch b;
};

#define FE_BGUARD(b) \
  if (!(b)) return fe_fail(FE_ERR_ARG, "null batch")

int fe_batch_create(int device, fe_batch** out) {
  if (!out) return fe_fail(FE_ERR_ARG, "null output");
  *out = nullptr;
  fe_batch* b = new (std::nothrow) fe_batch();
  if (!b) return fe_fail(FE_ERR_MEMORY, "host allocation");
  const int rc = b->b.create(device);
  if (rc) {
    delete b;
    return rc;
  }
  *out = b;
  return FE_OK;
}

int fe_batch_destroy(fe_batch* b) {
  delete b;
  return FE_OK;
}

int fe_batch_add(fe_batch* b, fe_engine* e) {
  FE_BGUARD(b);
  FE_GUARD(e);
  return b->b.add(&e->e);
}

int fe_batch_remove(fe_batch* b, fe_engine* e) {
  FE_BGUARD(b);
  FE_GUARD(e);
  return b->b.remove(&e->e);
}

int fe_batch_size(const fe_batch* b, int* members, int64_t* sites) {
  FE_BGUARD(b);
  if (members) *members = (int)b->b.mem.size();
  if (sites) {
    int64_t n = 0;
    for (const Engine* e : b->b.mem) n += e->hd.n;
    *sites = n;
  }
  return FE_OK;
}

int fe_batch_run(fe_batch* b, int nsteps) {
  FE_BGUARD(b);
  if (nsteps < 0) return fe_fail(FE_ERR_ARG, "nsteps < 0");
  return b->b.run(nsteps);
}

int fe_batch_launch(fe_batch* b, int nsteps) {
  FE_BGUARD(b);
  if (nsteps < 0) return fe_fail(FE_ERR_ARG, "nsteps < 0");
  return b->b.launch(nsteps);
}

int fe_batch_wait(fe_batch* b) {
  FE_BGUARD(b);
  return b->b.wait();
}

int fe_batch_time_run(fe_batch* b, int nsteps, float* ms) {
  FE_BGUARD(b);
  if (nsteps < 1 || !ms) return fe_fail(FE_ERR_ARG, "fe_batch_time_run: bad arguments");
  fe::Batch& B = b->b;
  if (B.mem.empty()) return fe_fail(FE_ERR_STATE, "empty batch");
  if (B.inflight) return fe_fail(FE_ERR_STATE, "batch steps in flight");
  int rc;
  // graphs and descriptors ready before the timed region
  if ((rc = B.prepare())) return rc;
  if (!B.graph1[0] && (rc = B.build_graphs())) return rc;
  cudaEvent_t e0, e1;
  FE_CUDA(cudaEventCreate(&e0));
  FE_CUDA(cudaEventCreate(&e1));
  FE_CUDA(cudaEventRecord(e0, B.stream));
  if ((rc = B.run_async(nsteps))) return rc;
  FE_CUDA(cudaEventRecord(e1, B.stream));
  FE_CUDA(cudaEventSynchronize(e1));
  FE_CUDA(cudaEventElapsedTime(ms, e0, e1));
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return B.finish(nsteps);
}

// ---- tracers ---------------------------------------------------------------
struct fe_tracers {
  fe::Tracers t;
};

int fe_tracers_create(fe_engine* e, const fe_tracer_config* cfg, int64_t n, const double* pos, const double* dm,
                      const int64_t* id, fe_tracers** out) {
  FE_GUARD(e);
  if (!cfg || !out || n < 0 || (n > 0 && (!pos || !dm))) return fe_fail(FE_ERR_ARG, "fe_tracers_create: bad arguments");
  if (cfg->substeps < 1 || (cfg->order != 1 && cfg->order != 2))
    return fe_fail(FE_ERR_ARG, "fe_tracers_create: substeps >= 1, order 1 or 2");
  *out = nullptr;
  fe_tracers* t = new (std::nothrow) fe_tracers();
  if (!t) return fe_fail(FE_ERR_MEMORY, "host allocation");
  const int rc = t->t.create(&e->e, cfg, n, pos, dm, id);
  if (rc) {
    delete t;
    return rc;
  }
  *out = t;
  return FE_OK;
}

int fe_tracers_destroy(fe_tracers* t) {
  delete t;
  return FE_OK;
}

int fe_tracers_step(fe_tracers* t) {
  if (!t) return fe_fail(FE_ERR_ARG, "null tracers");
  if (!t->t.E) return fe_fail(FE_ERR_STATE, "the tracers' engine was destroyed");
  if (t->t.E->owner && t->t.E->owner->inflight) return fe_fail(FE_ERR_STATE, "engine's batch steps in flight");
  return t->t.advance();
}

int fe_tracers_download(fe_tracers* t, double* pos, double* vel) {
  if (!t) return fe_fail(FE_ERR_ARG, "null tracers");
  if (!t->t.E) return fe_fail(FE_ERR_STATE, "the tracers' engine was destroyed");
  return t->t.download(pos, vel);
}

int fe_tracers_stretch_rows(fe_tracers* t, double* rows, int64_t max_rows, int64_t* count) {
  if (!t || !count || (max_rows > 0 && !rows)) return fe_fail(FE_ERR_ARG, "fe_tracers_stretch_rows: bad arguments");
  if (!t->t.E) return fe_fail(FE_ERR_STATE, "the tracers' engine was destroyed");
  return t->t.rows(rows, max_rows, count);
}

int fe_tracers_stretch_state(fe_tracers* t, double* rho_hat, double* log_rho) {
  if (!t) return fe_fail(FE_ERR_ARG, "null tracers");
  if (!t->t.E) return fe_fail(FE_ERR_STATE, "the tracers' engine was destroyed");
  return t->t.stretch_state(rho_hat, log_rho, false);
}

int fe_tracers_set_stretch_state(fe_tracers* t, const double* rho_hat, const double* log_rho) {
  if (!t) return fe_fail(FE_ERR_ARG, "null tracers");
  if (!t->t.E) return fe_fail(FE_ERR_STATE, "the tracers' engine was destroyed");
  if (rho_hat)
    for (int64_t p = 0; p < t->t.T.n; ++p) {
      const int64_t n = t->t.T.n;
      const double g = std::sqrt(rho_hat[p] * rho_hat[p] + rho_hat[n + p] * rho_hat[n + p] +
                                 rho_hat[2 * n + p] * rho_hat[2 * n + p]);
      if (!(std::fabs(g - 1.0) <= 1e-6)) return fe_fail(FE_ERR_ARG, "rho_hat is not a unit vector");
    }
  return t->t.stretch_state(const_cast<double*>(rho_hat), const_cast<double*>(log_rho), true);
}

int fe_tracers_set_velocity(fe_tracers* t, const double* u, const double* c) {
  if (!t) return fe_fail(FE_ERR_ARG, "null tracers");
  if (!t->t.E) return fe_fail(FE_ERR_STATE, "the tracers' engine was destroyed");
  if (t->t.E->owner && t->t.E->owner->inflight) return fe_fail(FE_ERR_STATE, "engine's batch steps in flight");
  return t->t.set_velocity(u, c);
}

int fe_batch_launch_count(const fe_batch* b, int64_t* count) {
  FE_BGUARD(b);
  if (count) *count = b->b.launches;
  return FE_OK;
}

}  // extern "C"
