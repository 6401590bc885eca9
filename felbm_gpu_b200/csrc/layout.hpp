// Device-side description of one lattice (one solve) and its control block.
//
// Site layout in HBM:
//  - the lattice is cut into bricks of BX x BY x BZ nodes (powers of two);
//    only bricks holding at least one fluid node are stored;
//  - bricks are ordered along a Morton curve of their brick coordinates and
//    sites (fluid nodes) are numbered brick by brick, slot by slot inside a
//    brick (slot = lx + BX*(ly + BY*lz)); so the sites of one brick are one
//    contiguous index range;
//  - per brick, one 64-bit occupancy word per 64 slots plus the site index of
//    that word's first site ("base"): the site index of any fluid node is
//    base[word] + popc(mask[word] & below(slot)). This is the whole
//    neighbour table: ~12 B per 64 nodes instead of the reference's
//    ~163 ints per site of case/column tables (multiphase_gpu.cuh:52-58);
//  - populations are AoSoA with width 32: f(i, k) lives at
//    (i >> 5) * 19*32 + k*32 + (i & 31), so a warp's 32 sites read each
//    direction as one contiguous 128-byte (FP32) line;
//  - h and g each have two such arrays (ping-pong), state streamed by pull.
#pragma once
#include <cstdint>

namespace fe {

constexpr int AOSOA = 32;
constexpr int HMAX = 3;  // deepest halo the per-brick tile tables cover

// Per-brick record, built on the host. A kernel's tile with halo H <= HMAX
// covers brick coordinates [-H, B + H) per axis; tile coordinate t maps to
// table index t + HMAX - H. seg[a][.] names which distinct neighbour brick the
// (periodically wrapped) coordinate falls in along axis a (at most 4, see
// the host builder) and loc[a][.] the local coordinate inside it; nbr holds
// the brick id of each segment combination sx + 4*(sy + 4*sz) (-1: no fluid).
struct alignas(16) BrickRec {
  int32_t nbr[64];
  uint8_t seg[3][24];
  uint8_t loc[3][24];
  int32_t first, cnt;  // the brick's site range
  int32_t pad[2];
};
static_assert(sizeof(BrickRec) % 16 == 0, "BrickRec is copied as int4");

// Per-lattice control block in device memory. Written by the kernels' last
// block and by small host copies; read by every CTA at start.
struct Ctl {
  int64_t t;             // driver step counter (forcing_factor_at argument)
  int32_t open_step;     // number of open-boundary applications so far
  int32_t pending;       // 1: a mass correction is queued for the next pass
  int32_t auto_correct;  // 1: queue a correction after each step (fe_run)
  int32_t ff_auto;       // 1: forcing factor from t; 0: ff_manual; 2: ff_last
  double ff_manual;
  double target_mass;    // M0
  double M, W;           // sums of the last moment pass
  double lambda;         // correction lambda used by the current pass
  double drift;          // M - M0 at the last queued correction
  unsigned int count1;   // last-block counters (reset by the last block)
  unsigned int count4;
  unsigned int countm;
  unsigned int counts;   // owned by k_stats_finalize, launched on the engine's stream only
  double stats[6];       // flow statistics of the last finalize
  int32_t status;        // nonzero: a kernel detected a problem
  int32_t pad_;
  double ff_last;        // forcing factor of the last collision pass (field refreshes use it)
};

// Physics parameters of one lattice, in double (each kernel converts to its
// arithmetic type on entry).
struct DevPrm {
  double rho0, rho1, drho, kappa, four_beta, bnd_coeff, tau0, tau1, mobility;
  double gx, gy, gz, fx, fy, fz;
  double mrt_lambda;
  double rate_value[7];
  int rate_mode[7];
  int use_mrt, hbb, correct_mass;
  // MRT rates that depend on the moment's parity only (every even kind one
  // rate, every odd kind another): the collide pass may take the two-rate form
  int two_rate;
  int need_j;  // P1 writes the momentum (drho != 0 or open boundaries)
  int forcing_timedep;
  double forcing_period;
  // open boundary
  int open_bnd, copy_to_buf;
  int use_in_vel, use_in_prs, use_in_fluid, use_out_prs, use_out_fluid;
  int inlet_mode;
  double u_in[3], p_in, p_out, c_out_fixed, rho_out_fixed, inlet_c_a;
  double inlet_period, inlet_duty, inlet_ramp, split_pos;
  // FP16/BF16 shifted storage: stored = (f - w_k * ref) * scale
  double c_ref, p_ref, h_scale, g_scale;
};

// The tensor maps of a lattice's stencil-field grids: the field and the
// halo of the box (the x halo of every box is 2, so the box starts on a
// 16-byte boundary). TM_CP2 covers the (c', p') pair grid.
enum TensorMapId { TM_C1 = 0, TM_CP2 = 1, TM_MU1 = 2, TM_L2 = 3, TM_N = 4 };

// Per-site open-boundary flags (bcflag[i]).
enum : uint8_t {
  BC_SITE = 1,      // fields imposed/copied: c_raw_bc, u_bc hold this site's values
  BC_PROC = 2,      // excluded from the velocity/pressure correction
  BC_G_OVER = 4,    // g replaced by the plain equilibrium before the collision
};

struct LatDesc {
  // geometry
  int nx, ny, nz;
  int lbx, lby, lbz;     // log2 of the brick dims
  int nbx, nby, nbz;     // brick grid
  int words;             // 64-bit occupancy words per brick
  int nbricks;
  int nchunks;           // flat chunks of CHUNK sites (P1, transfers)
  int64_t n;             // sites
  int64_t n_pad;         // rounded up to AOSOA
  const int32_t* brick_grid;   // [nbz][nby][nbx] -> brick or -1
  const uint64_t* mask;        // [nbricks][words]
  const int32_t* base;         // [nbricks][words]
  const int32_t* brick_xyz;    // [nbricks][3]
  const BrickRec* rec;         // [nbricks]
  const int32_t* ref_of;       // site -> reference-order index
  const int32_t* tile1;        // [nbricks][halo-1 tile] (k_build_tiles): with 32-bit population
                               // offsets the site's AoSoA population base (0xffffffff: no site),
                               // with 64-bit ones the site index (-1: no site)
  const uint16_t* slots;       // [nbricks][brick slots] fluid slots in site order
  // state: pop[buffer][0 = h, 1 = g]
  void* pop[2][2];
  // fields (FP64 for FP64 storage, FP32 otherwise). The stencil fields c,
  // p, mu, lap(mu) and the (c', p') pairs live on a dense node grid covering
  // node coordinates
  // [-2, nb * B + 2) per axis (z: [0, 1) without a z halo), x fastest;
  // solid nodes hold NaN, and positions outside the lattice hold the
  // periodic image of the node they wrap to (k_images copies those of fluid
  // nodes after each pass that writes the field). A brick's halo tile is
  // then one box of the grid, loaded by one TMA copy. The momentum jx, jy, jz
  // is per site. cp is the grid of (c', p') pairs that P2 writes for the
  // collision: the order parameter with the queued mass correction applied
  // and the corrected pressure, interleaved. P2 writes each pair whole (with
  // P1 storing p into the second lane and P2 the order parameter into the
  // first, P2 ran six times slower; the cause was not found).
  void *c, *p, *jx, *jy, *jz, *mu, *lapmu, *cp;
  int gdx, gdy, gdz;           // grid extents (gdx a multiple of 16 bytes of entries)
  int hz;                      // 1: the z axis has a halo (3-D bricks)
  int64_t gsy, gsz;            // entry strides of y and z (x: 1)
  const int32_t* dense_of;     // site -> grid entry of its node
  const int2* images;          // {grid entry, entry of its fluid node} of each image position
  int64_t n_images;
  int image_blocks;            // work items of one k_images pass
  const void* tmap;            // CUtensorMap[TM_N] of the stencil fields (64-byte aligned)
  // open boundary (null when off)
  const uint8_t* bcflag;
  const int32_t* bcsrc;
  void* c_raw_bc;
  void* u_bc;                  // [3][n]
  // node-indexed velocity (and order parameter) snapshot that P2 writes on
  // every step while tracers are attached (null: none)
  double* snap_u[3];
  double* snap_c;
  const int32_t* bc_list;      // inlet sites, then outlet sites
  const int32_t* bc_xyz;       // node coordinates of inlet, outlet, buffer sites [3 each]
  const double* bc_coord;      // inlet coordinate along the split axis
  int n_inlet, n_outlet, n_buf;
  const int32_t* buf_verts;
  const int32_t* buf_refs;
  // reductions
  double* part1;               // [nchunks][2] M, W partials of the moment pass
  double* part4;               // [nbricks][6] flow-statistics partials
  Ctl* ctl;
  DevPrm prm;
};

}  // namespace fe
