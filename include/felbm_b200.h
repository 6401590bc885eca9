/*
 * felbm_b200 — C-ABI of the B200-native Lee–Liu free-energy multiphase D3Q19
 * step over the sparse fluid-site set of a porous geometry.
 *
 * Every entry point replaces one member of the reference's header-only engine
 * `struct felbm_gpu::MultiPhaseGPU` (include/felbm_gpu/multiphase_gpu.cuh) or a
 * piece of its driver (src/felbm_gpu_main.cu). The citation above each
 * declaration names the reference interface it stands for.
 *
 * Conventions (differences from the reference are deliberate):
 *  - every call returns an int status (FE_OK = 0); nothing calls exit()
 *    (the reference exits the process on any CUDA error, gpu_common.cuh:14-22);
 *    fe_last_error() returns a message for the last failure on this thread;
 *  - distributions cross the boundary as double, in the reference's layout
 *    f[k*n + i], with sites i numbered in the reference order: fluid nodes in
 *    increasing node index x + nx*(y + ny*z);
 *  - the engine owns all device memory; host arrays belong to the caller;
 *  - one engine is driven by one host thread at a time; all its work is
 *    queued on the engine's own CUDA stream.
 */
#ifndef FELBM_B200_H
#define FELBM_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define FE_OK 0
#define FE_ERR_ARG 1        /* invalid argument / size mismatch            */
#define FE_ERR_CUDA 2       /* CUDA runtime error                           */
#define FE_ERR_NO_DEVICE 3  /* no usable CUDA device                        */
#define FE_ERR_MEMORY 4     /* device or host allocation refused            */
#define FE_ERR_STATE 5      /* call not valid in the engine's current state */
#define FE_ERR_IO 6         /* file could not be read or written            */
#define FE_ERR_DIVERGED 7   /* non-finite or runaway state detected         */

/* Population storage of the state arrays. Arithmetic is FP64 for FE_F64 and
 * FP32 in registers for the others; FE_F16S / FE_BF16S store each population as
 * a scaled deviation from its rest-state value w_k*(c_ref | p_ref). */
#define FE_F64 0
#define FE_F32 1
#define FE_F16S 2
#define FE_BF16S 3
/* Mixed: h in FP32 (the order parameter spans 0..1, so a shift gains it no
 * precision), g as the FP16 / BF16 deviation from w_k*p_ref. */
#define FE_F16G 4
#define FE_BF16G 5

/* forcing_timedep (reference felbm_gpu_main.cu:587-594) */
#define FE_FORCING_CONSTANT 0
#define FE_FORCING_SINUSOIDAL 1
#define FE_FORCING_SQUARE 2

/* MRT rate kinds (index into mrt_rate_mode / mrt_rate_value) and modes. */
#define FE_MRT_E 1
#define FE_MRT_EPS 2
#define FE_MRT_Q 3
#define FE_MRT_NU 4
#define FE_MRT_PI 5
#define FE_MRT_M 6
#define FE_RATE_S0 0    /* the site's BGK rate 1/(tau+1/2)               */
#define FE_RATE_MAGIC 1 /* 2 tau/(2 Lambda + tau), reference default     */
#define FE_RATE_FIXED 2 /* mrt_rate_value[kind]                          */

/* Physics and solver switches. Field names follow the reference's cfg keys
 * (params.cfg / settings.cfg) and DevParams (device_engine.cuh:31-59). Fill
 * the raw keys, then call fe_params_derive() for kappa, beta, mobility and
 * bnd_coeff (reference compare_cpu_gpu.cu:115-118). */
typedef struct fe_params {
  /* params.cfg */
  double rho0, rho1;             /* phase densities (phase 0 has c = 1)      */
  double tau0, tau1;             /* relaxation times                         */
  double interface_width;        /* W                                        */
  double surface_tension;        /* sigma                                    */
  double mobility_coeff;         /* mobility = mobility_coeff / beta         */
  double phi;                    /* wetting potential, 6 sigma cos(theta)    */
  /* derived by fe_params_derive */
  double kappa, beta, mobility, bnd_coeff;
  /* settings.cfg */
  double gx, gy, gz;             /* acceleration_[xyz]                       */
  double fx, fy, fz;             /* forcing_[xyz], scaled by forcing_factor  */
  int forcing_timedep;           /* FE_FORCING_*                             */
  double forcing_period;
  int use_mrt;
  double mrt_lambda;             /* magic parameter, default 0.1875          */
  int mrt_rate_mode[7];          /* per FE_MRT_* kind; [0] unused            */
  double mrt_rate_value[7];
  int use_halfway_bb;
  int correct_op_mass;
  /* fast-path switches of the reference (cfg keys). All of them select the
   * one fused path here; they are kept so configs and logs round-trip. */
  int stream_matrix_free, grad_matrix_free, fused, fuse_collision;
  int mrt_fast_transform, stream_inplace;
  /* storage of the populations, FE_F64 .. FE_BF16G */
  int storage;
  /* reference scale of the FE_F16S/FE_BF16S deviations (ignored otherwise) */
  double c_ref, p_ref;
  /* layout of this library (no reference counterpart): the brick shape,
   * FE_BRICK_AUTO = the autotuner's choice for the size class (fe_autotune)
   * or the default, and the steps per CUDA-graph launch of fe_run (0 = the
   * tuned or default 2) */
  int brick;
  int graph_steps;
  /* population layout (no reference counterpart; the reference's own
   * in-place streaming is the op program of stream_inplace): FE_POP_TWO_BUFFERS
   * (default) streams from one buffer into the other; FE_POP_IN_PLACE keeps
   * one buffer and alternates the two phases of the AA pattern (a step from
   * the standard layout writes each site's post-collision populations into
   * its own opposite slots; the next step reads them from the upstream sites
   * and pushes its results to the downstream ones, which restores the
   * standard layout). Half the population memory; FE_F64 and FE_F32 storage,
   * lattices whose population arrays stay below 2^32 entries. */
  int pop_layout;
} fe_params;

#define FE_POP_TWO_BUFFERS 0
#define FE_POP_IN_PLACE 1

/* Brick shapes. 16x16x1 is the one for lattices with nz == 1; 8x8x4 exists
 * for FE_F64 and FE_F32 storage. Without a tuned choice, 3-D lattices get
 * 16x8x8. */
#define FE_BRICK_AUTO 0
#define FE_BRICK_8x8x8 1
#define FE_BRICK_16x16x1 2
#define FE_BRICK_8x8x4 3
#define FE_BRICK_16x8x8 4

/* Open inlet/outlet (reference MultiPhaseGPU::set_open_bnd,
 * multiphase_gpu.cuh:369-400, plus the DevParams open-boundary block
 * device_engine.cuh:45-58 that the driver fills, felbm_gpu_main.cu:334-380).
 * Node lists are site indices in the reference order. */
typedef struct fe_open_bnd {
  int n_inlet;  const int32_t* inlet;
  const double* inlet_coord;     /* per inlet node, coordinate along split axis
                                    (modes split/stripes), or NULL */
  int n_outlet; const int32_t* outlet;
  int n_buf;    const int32_t* buf_verts; const int32_t* buf_refs;
  int copy_to_buffers;
  int use_in_vel, use_in_prs, use_in_fluid, use_out_prs, use_out_fluid;
  double u_in_x, u_in_y, u_in_z;
  double p_in, p_out;
  double c_out_fixed, rho_out_fixed;
  double inlet_c_a;              /* 1 - inlet_fluid                          */
  int inlet_mode;                /* 0 single, 1 alternate, 2 split, 3 stripes */
  int split_axis;
  double inlet_period, inlet_duty, inlet_ramp, split_pos;
} fe_open_bnd;

/* ---- configuration files ------------------------------------------------
 * The reference driver's settings.cfg (and the params.cfg its `param_file`
 * names, relative to the settings file), read as felbm_gpu reads them
 * (src/felbm_gpu_main.cu:190-235 and the Settings keys it uses through
 * felbm_local's util::ConfigFile): `key = value`, `#` comments, quoted
 * strings, booleans true/false. The driver-level keys land here; the
 * physics and solver keys in fe_params (its fields carry the key names:
 * acceleration_* -> gx..gz, forcing_* -> fx..fz, the six fast-path switches,
 * use_mrt, mrt_lambda, use_halfway_bb, correct_op_mass; rho0 .. phi from
 * params.cfg); the open-boundary flags and values in fe_open_bnd (its node
 * lists come from the geometry, fe_geom_open_lists). */
typedef struct fe_driver_cfg {
  char model[32];
  char output_dir[256], output_name[128], timeseries_file[128], log_file[128];
  char param_file[256], velocity_set[16];
  char domain_geometry[64], domain_cfg_file[256];
  char fluid_initializer[64], fluid_init_filename[256];
  char restart_file[256];        /* [gpu] resume from this checkpoint ("" none) */
  int size_x, size_y, size_z;
  int64_t max_iterations;
  int log_skip, file_skip;
  uint32_t checkpoint_skip;      /* [gpu] checkpoint every N steps (0 never)   */
  int output_deflate;            /* [gpu] gzip level 0-9 of field files        */
  int output_float32;            /* [gpu] float32 instead of float64 fields    */
  int gpu_device;                /* [gpu] -1: leave the device as it is        */
  int logging, console;
  int use_open_bnd, in_out_dir, buffer_layers, empty_layers, extrude_buffers;
  int image_periodic, transverse_periodic;
  int particles_enable;
  int64_t particles_number;
  char particles_init_mode[32], particles_plane_offsets[256], particles_dm_groups[512];
  int particles_int_order, particles_substeps, particles_file_skip;
  double particles_dt;
  int unknown_keys;              /* keys of either file this reader ignored    */
} fe_driver_cfg;

/* Defaults of the driver-level keys. */
int fe_driver_cfg_default(fe_driver_cfg* d);
/* Read settings.cfg (+ params.cfg) over the given parameter block (keys
 * absent from the files keep p's values), then derive kappa, beta, mobility,
 * bnd_coeff. ob may be NULL. Refuses what the reference driver refuses
 * (model single_phase; correct_op_mass with open boundaries,
 * felbm_gpu_main.cu:242-254). */
int fe_cfg_read(const char* settings_path, fe_params* p, fe_open_bnd* ob, fe_driver_cfg* d);
/* How each of the six fast-path switches of p maps onto this engine, one
 * line per key, into buf (NUL-terminated; FE_ERR_ARG if len is too small). */
int fe_cfg_switch_log(const fe_params* p, char* buf, int len);

/* Macroscopic fields, each n doubles in the reference site order
 * (reference RawFields, multiphase_gpu.cuh:730). Any pointer may be NULL. */
typedef struct fe_fields {
  double *rho, *c, *ux, *uy, *uz, *p, *mu;
} fe_fields;

typedef struct fe_engine fe_engine;

/* ---- parameters -------------------------------------------------------- */
/* Defaults of the reference: switches off, BGK, lambda 0.1875, reference MRT
 * rate assignment, FP64 storage. */
int fe_params_default(fe_params* p);
/* kappa = 1.5 W sigma, beta = 12 sigma / W, mobility = coeff / beta,
 * bnd_coeff = phi / kappa (reference compare_cpu_gpu.cu:115-118). */
int fe_params_derive(fe_params* p);

/* ---- lifecycle --------------------------------------------------------- */
/* Replaces MultiPhaseGPU::init (multiphase_gpu.cuh:75-351). The geometry is a
 * solid mask over nx*ny*nz nodes (1 = solid), node index x + nx*(y + ny*z);
 * streaming wraps periodically on every axis (reference README "What is and
 * isn't periodic"). device < 0 keeps the current device. */
int fe_engine_create(const fe_params* p, int nx, int ny, int nz,
                     const uint8_t* solid, int device, fe_engine** out);
/* Replaces MultiPhaseGPU::free (multiphase_gpu.cuh:759-782). */
int fe_engine_destroy(fe_engine* e);
/* Number of sites n and state size Vn = 19 n (reference state_size(),
 * multiphase_gpu.cuh:457). */
int fe_engine_size(const fe_engine* e, int64_t* n, int64_t* vn);
/* Replaces writes to MultiPhaseGPU::params() (multiphase_gpu.cuh:362) for the
 * physics block; takes effect at the next step. */
int fe_set_params(fe_engine* e, const fe_params* p);
/* The CUDA stream the engine queues its work on (cudaStream_t). */
void* fe_engine_stream(fe_engine* e);

/* ---- state ------------------------------------------------------------- */
/* Replaces upload_state (multiphase_gpu.cuh:354-359): h, g are Vn doubles.
 * Large states of the storages other than FE_F64 cross the link as FP32
 * (narrowed on the host, the conversion the device would apply); the
 * stored state is the same either way. */
int fe_upload_state(fe_engine* e, const double* h, const double* g, int64_t vn);
/* No counterpart in the reference: the equilibrium state at rest of per-site
 * order parameter c and pressure p (n doubles each, reference site order;
 * p NULL: p_uniform at every site), built on the device. The stored state is
 * the one fe_upload_state gives for the arrays of fe_init_equilibrium(n, c,
 * p, NULL, NULL, NULL, ...), from n (or 2n) values across the link instead
 * of 38n. */
int fe_upload_equilibrium(fe_engine* e, const double* c, const double* p, double p_uniform, int64_t n);
/* Replaces download_state (multiphase_gpu.cuh:449-455); includes a pending
 * order-parameter mass correction, as the reference's state would. Storages
 * other than FE_F64 hold FP32 values, which large downloads move as FP32 and
 * widen on the host (exact). */
int fe_download_state(fe_engine* e, double* h, double* g, int64_t vn);

/* ---- open boundaries --------------------------------------------------- */
/* Replaces set_open_bnd + the driver's DevParams fill. Call before stepping. */
int fe_set_open_bnd(fe_engine* e, const fe_open_bnd* b);

/* ---- stepping ---------------------------------------------------------- */
/* Replaces MultiPhaseGPU::step() (multiphase_gpu.cuh:522-631), nsteps times,
 * without mass correction (the driver calls that separately). */
int fe_step(fe_engine* e, int nsteps);
/* Replaces apply_mass_correction() (multiphase_gpu.cuh:689-700). When drift
 * is non-NULL the drift M - M0 is computed now and returned (a blocking
 * reduction, as in the reference); when NULL the correction is queued and
 * fused into the next step's moment pass. No-op unless correct_op_mass.
 * Unlike the reference, the stored populations take the correction later:
 * fe_current_mass (and a reduction of a state taken by other means) sees the
 * corrected total only after fe_settle_mass_correction, the next step, or a
 * download (fe_download_state, fe_download_fields, checkpoints), which all
 * apply the queued correction first. */
int fe_apply_mass_correction(fe_engine* e, double* drift);
/* The driver's hot loop (felbm_gpu_main.cu:741-745): nsteps x (step + mass
 * correction), with forcing_factor_at(t) evaluated per step from the
 * engine's step counter; replayed through a CUDA graph. */
int fe_run(fe_engine* e, int nsteps);
/* Step counter t used by forcing_factor_at and by fe_run (the driver's loop
 * index, felbm_gpu_main.cu:701); set it after a restart. */
int fe_set_time(fe_engine* e, int64_t t);
int fe_get_time(const fe_engine* e, int64_t* t);
/* Replaces the driver's `gpu.P.forcing_factor = ...` (felbm_gpu_main.cu:743)
 * for fe_step; fe_run computes it from the step counter instead. */
int fe_set_forcing_factor(fe_engine* e, double ff);

/* ---- order-parameter mass target -------------------------------------- */
/* record_target_mass / set_target_mass / get_target_mass / current_mass
 * (multiphase_gpu.cuh:458-459,685-687). */
int fe_record_target_mass(fe_engine* e);
int fe_set_target_mass(fe_engine* e, double m0);
int fe_get_target_mass(const fe_engine* e, double* m0);
int fe_current_mass(fe_engine* e, double* m);

/* ---- readout ----------------------------------------------------------- */
/* Replaces download()/download_raw() (multiphase_gpu.cuh:704-757): refresh the
 * macroscopic fields from the current state (moments, open-boundary field
 * enforcement, mu, velocity/pressure correction) and copy them out. The
 * velocity correction takes the forcing factor of the last step (1 before
 * any step), as the reference's refresh reads the DevParams forcing_factor
 * the driver set for the last step. */
int fe_download_fields(fe_engine* e, const fe_fields* f);
/* Replaces flow_stats (multiphase_gpu.cuh:645-651): out = {sum ux, sum uy,
 * sum uz, sum u^2, sum c, max u^2} of the fields of the last step. */
int fe_flow_stats(fe_engine* e, double out[6]);
/* Asynchronous form (flow_stats_launch / _ready / _collect, :658-683). */
int fe_flow_stats_launch(fe_engine* e);
int fe_flow_stats_ready(fe_engine* e, int* ready);
int fe_flow_stats_collect(fe_engine* e, double out[6]);

/* ---- geometry and initial-condition front end -------------------------
 * Replace the felbm_local DomainInitializer_* / InitializerMultiPhase_* the
 * reference driver calls (felbm_gpu_main.cu:256-311); seeded and
 * platform-independent. Masks: nx*ny*nz uint8, 1 = solid. */
/* Gaussian random field, correlation exp(-r^2/(2 corr_len^2)), fluid below the
 * porosity quantile, largest cluster percolating along flow_axis kept
 * (flow_axis < 0: largest cluster; open_flow: no wrap along flow_axis). */
int fe_geom_grf(int nx, int ny, int nz, double corr_len, double porosity, uint64_t seed,
                int flow_axis, int open_flow, uint8_t* solid, double* porosity_out);
/* Random sequential disc pack (radii U[rmin,rmax], periodic gap) extruded in z. */
int fe_geom_cylinders(int nx, int ny, int nz, double rmin, double rmax, double porosity, double gap,
                      uint64_t seed, int keep_largest, uint8_t* solid, double* porosity_out);
/* Up to max_number spheres of one radius, centre distance >= 2r + distance
 * (compare_cpu_gpu.cu:165-175 "spheres_repulsive"). */
int fe_geom_spheres(int nx, int ny, int nz, double radius, int max_number, double distance,
                    uint64_t seed, uint8_t* solid);
/* Open inlet/outlet padding (empty_layers, buffer_layers, extrude_buffers). */
int fe_geom_pad_open(const uint8_t* medium, int mx, int my, int mz, int flow_axis, int empty_layers,
                     int buffer_layers, int* dims_out, uint8_t* out_solid);
/* SubDomain::inlet_verts/outlet_verts/buffer_verts/buffer_refs of a padded domain. */
int fe_geom_open_lists(const uint8_t* solid, int nx, int ny, int nz, int flow_axis, int buffer_layers,
                       int split_axis, int32_t* n_counts, int32_t* inlet, int32_t* outlet,
                       int32_t* buf_verts, int32_t* buf_refs, double* inlet_coord);
/* Segmented TIFF stack (reference domain_geometry = 3d_image; keys of
 * cfg/3d_image/domain.cfg). paths: the files in z order (each page one z
 * slice; baseline TIFF, either byte order, grey 1/8/16 bits, uncompressed or
 * PackBits). Solid where the voxel is nonzero (solid_nonzero, the
 * interface_solid key) or zero, inverted when invert (invert_image).
 * subvolume (x0, y0, z0, sx, sy, sz in full-resolution voxels, or NULL:
 * use_subvolume) is cut first; then coarsening_levels halvings of every axis
 * longer than 1 (trailing odd layer dropped; solid when at least half the
 * fine voxels are). dims out: nx, ny, nz; solid NULL asks for dims only. */
int fe_geom_tiff_stack(const char* const* paths, int npaths, int solid_nonzero, int invert, int coarsening_levels,
                       const int* subvolume, int* dims, uint8_t* solid, int64_t capacity);
/* Site count and node index of each site (SubDomain::idx_to_coords). */
int fe_geom_sites(const uint8_t* solid, int nx, int ny, int nz, int64_t* n, int64_t* nodes);
/* Order parameter per site: kind 0 uniform, 1 slab_interface, 2 spherical_droplet. */
int fe_init_order_parameter(const uint8_t* solid, int nx, int ny, int nz, int kind, const double* a,
                            double width, double* c_out);
/* Plain equilibrium h, g of per-site fields (u may be NULL). */
int fe_init_equilibrium(int64_t n, const double* c, const double* p, const double* ux, const double* uy,
                        const double* uz, double rho0, double rho1, double* h, double* g);

/* ---- allocation-free reduction -----------------------------------------
 * No counterpart in the reference. For callers that cannot allocate device
 * memory (their pool allocator owns the GPU's memory, or their loop must not
 * enter cudaMalloc/cudaFree, which can synchronize the device): the
 * order-parameter mass M = sum_i c_i and interface weight
 * W = sum_i max(c_i (1 - c_i), 0), c_i = sum_k h[k*n + i], of FP64
 * populations h in the caller's device memory, written to d_out[0], d_out[1]
 * (caller's device memory) on `stream` (cudaStream_t, NULL = legacy default).
 * It allocates nothing: its partial sums live in one fixed array of 262,400
 * bytes inside the library, present on every GPU that loads the library
 * until the process exits. n above FE_NOALLOC_MAX_SITES is rejected with
 * FE_ERR_ARG. All calls on a device share that array: calls whose work
 * overlaps on the GPU race and give wrong results. The first call on each
 * device sets up the array's address (with that device current); make it
 * before starting any stream capture. The address is kept for the life of
 * the process: after a cudaDeviceReset the library must not be called on
 * that device again. */
#define FE_NOALLOC_MAX_SITES 33554432LL
int fe_mass_weight_noalloc(const double* d_h, int64_t n, double* d_out, void* stream);

/* ---- batches -------------------------------------------------------------
 * No counterpart in the reference (one MultiPhaseGPU per process there).
 * A batch advances many engines (independent lattices of any size, same
 * device and storage type) together: each pass of the step is one launch
 * over the concatenated brick/chunk lists of all members, captured as CUDA
 * graphs, so small lattices share the GPU instead of each leaving it idle.
 * Every member keeps its own state, parameters, mass target and statistics,
 * and gets bit-for-bit the result it gets from fe_run alone. fe_batch_run
 * behaves as fe_run on every member (queued mass correction after each step,
 * forcing factor from the step counter) and returns when the steps are done.
 * Engines stay usable on their own between batch runs; fe_engine_destroy of
 * a member removes it first. A member with the in-place population layout
 * joins in the standard layout (a pending phase is swapped back in place),
 * so the batch's step parity is its phase. */
typedef struct fe_batch fe_batch;
int fe_batch_create(int device, fe_batch** out);
int fe_batch_destroy(fe_batch* b);
int fe_batch_add(fe_batch* b, fe_engine* e);
int fe_batch_remove(fe_batch* b, fe_engine* e);
int fe_batch_size(const fe_batch* b, int* members, int64_t* sites);
int fe_batch_run(fe_batch* b, int nsteps);
/* fe_batch_run in two halves: fe_batch_launch queues the steps on the batch
 * stream and returns at once, so the caller's host work (creating and
 * uploading the next engines, reading back retired ones) overlaps them;
 * fe_batch_wait waits for them. In between, members must not be used and
 * fe_batch_add fails (fe_batch_remove waits first). */
int fe_batch_launch(fe_batch* b, int nsteps);
int fe_batch_wait(fe_batch* b);
/* fe_batch_run of nsteps timed with CUDA events on the batch stream. */
int fe_batch_time_run(fe_batch* b, int nsteps, float* ms);
int fe_batch_launch_count(const fe_batch* b, int64_t* count);

/* ---- serving -------------------------------------------------------------
 * No counterpart in the reference. A request loop on its own host thread.
 * Solves submitted at any time wait in a queue and are admitted (engine
 * created, state uploaded, kept resident on the device) while a slot is free
 * and their estimated footprint fits the memory budget: the device memory
 * free at fe_server_create minus hbm_reserve_frac of the device's total.
 * Resident solves advance in chunks of at most chunk_steps steps; each chunk
 * runs the resident solves with the least remaining work (sites x remaining
 * steps) together in one batch, adding solves until their sites reach
 * fill_sites (<= 0: all of them), so a small solve is not held to the step
 * rate of a large batch. Admission and retirement happen between chunks and
 * their host work (engine creation, upload, read-back) overlaps the chunk on
 * the GPU: continuous batching. A solve retires after its step count or,
 * when conv_tol > 0, once the mean velocity changes by less than conv_tol
 * (relative) between two of its chunks. Results carry the time-to-result
 * (submit -> results read back) and, on request, the fields. Every solve
 * gets bit-for-bit the result it gets alone (fe_batch). Requests with open
 * boundaries are not served. */
typedef struct fe_server fe_server;
typedef struct fe_server_config {
  int device;
  int max_active;             /* resident solves at most (<= 0: no limit)  */
  double hbm_reserve_frac;    /* device memory kept free (fraction of total) */
  int chunk_steps;            /* steps between admission points (> 0)     */
  int storage;                /* FE_F64 .. FE_BF16S, all requests          */
  int64_t fill_sites;         /* sites per chunk (<= 0: every resident solve) */
  int pop_layout;             /* FE_POP_TWO_BUFFERS or FE_POP_IN_PLACE (FE_F64 /
                                 FE_F32 storage): the population layout of
                                 every solve, and of its charged footprint  */
  int latency_first;          /* nonzero (with fill_sites > 0): a chunk also
                                 holds no more sites than 2 s1 + 131072, s1
                                 the sites of its solve with the least
                                 remaining work, so small requests step at
                                 about their own rate (lower time-to-result
                                 under light load, fewer sites a chunk)     */
} fe_server_config;
typedef struct fe_request {
  int64_t id;
  fe_params params;           /* params.storage is overridden by the server's */
  int nx, ny, nz;
  const uint8_t* solid;       /* nz*ny*nx, copied at submit                */
  const double* h0;           /* initial state (reference layout, copied)  */
  const double* g0;           /* or NULL: built from the init fields below */
  int init_kind;              /* fe_init_order_parameter kind              */
  double init_a[5];
  double init_width;
  double init_p;              /* initial pressure level                    */
  int64_t steps;              /* retire after this many steps              */
  double conv_tol;            /* > 0: convergence test (see above)         */
  int want_fields;            /* 1: the result carries rho, c, u, p        */
} fe_request;
typedef struct fe_result {
  int64_t id;
  int status;                 /* FE_OK, or the failing call's status       */
  char message[160];
  int64_t sites, steps_done;
  double t_submit, t_admit, t_done;   /* seconds since fe_server_create   */
  double mass0, mass_final;   /* order-parameter mass at admission / end   */
  double stats[6];            /* flow statistics at retirement             */
  double *rho, *c, *ux, *uy, *uz, *p; /* n each (reference order) or NULL */
} fe_result;
typedef struct fe_server_stats {
  int64_t submitted, admitted, completed, queued, active, peak_active; /* active = resident */
  int64_t site_steps;         /* fluid-site updates done                   */
  double busy_seconds;        /* time inside batch runs                    */
  double elapsed_seconds;     /* since fe_server_create                    */
  double mlups_busy, mlups_wall;
  double ttr_p50, ttr_p99, ttr_max;   /* time-to-result of completed solves */
} fe_server_stats;
int fe_server_create(const fe_server_config* cfg, fe_server** out);
/* Thread-safe; copies the request's arrays. */
int fe_server_submit(fe_server* s, const fe_request* r);
/* Moves up to max finished results into out; *n = how many. */
int fe_server_poll(fe_server* s, fe_result* out, int max, int* n);
int fe_server_free_result(fe_result* r);
/* Blocks until nothing is queued or active (or timeout_s passes: FE_ERR_STATE). */
int fe_server_wait_idle(fe_server* s, double timeout_s);
int fe_server_get_stats(fe_server* s, fe_server_stats* st);
/* Stops the loop (active solves are dropped) and frees everything. */
int fe_server_destroy(fe_server* s);

/* ---- tracers ---------------------------------------------------------------
 * Replace the reference's host ParticleManager path (felbm_gpu_main.cu:
 * 421-581, 752-777: velocity copied to the host and scattered every step).
 * Here tracers live on the GPU beside their engine. fe_tracers_step advances
 * them one lattice step on the engine's current corrected velocity
 * (trilinear interpolation of a node-indexed snapshot refreshed every
 * velocity_skip steps, the reference's particles_velocity_skip), with
 * `substeps` Euler (order 1) or Heun (order 2) substeps, a Brownian kick
 * sqrt(2 Dm dt) N(0,1) per axis from a counter-based Philox4x32-10 stream
 * keyed by seed and tracer id (none along z in a 2-D lattice; Dm = 0 draws
 * nothing), and moves onto solid nodes rejected. Call it after each engine
 * step, as the reference driver calls pm.update(). Positions are node
 * coordinates, periodic, [3][n] (all x, then y, then z). Tracers use their
 * engine's stream and must be destroyed before it. */
typedef struct fe_tracers fe_tracers;
typedef struct fe_tracer_config {
  int substeps;               /* >= 1 */
  int order;                  /* 1 or 2 */
  int velocity_skip;          /* refresh the velocity every this many steps */
  uint64_t seed;
  int stretching;             /* 1: material line elements (particles_stretching) */
  int phase_split;            /* 1: split lambda by phase (particles_phase_split) */
  uint64_t stretching_seed;   /* initial orientations (particles_stretching_seed) */
} fe_tracer_config;
/* n tracers at pos [3][n] with diffusivities dm [n] and ids [n] (NULL: 0..n-1;
 * the random stream of a tracer depends on its id). */
int fe_tracers_create(fe_engine* e, const fe_tracer_config* cfg, int64_t n, const double* pos,
                      const double* dm, const int64_t* id, fe_tracers** out);
int fe_tracers_destroy(fe_tracers* t);
int fe_tracers_step(fe_tracers* t);
/* pos, vel: [3][n] host arrays (either may be NULL); vel is the velocity
 * interpolated at each tracer's position at the end of the last step. */
int fe_tracers_download(fe_tracers* t, double* pos, double* vel);
/* Lagrangian stretching (reference README "Lagrangian stretching"; its
 * ParticleManager half is in the absent felbm_local tree, the method is the
 * one docs/HANDOFF_stretching.md section 2 states). Each tracer carries a unit
 * orientation rho_hat (isotropic at creation, from stretching_seed) and
 * log_rho (0 at creation); per accepted substep, with J the gradient of the
 * interpolated velocity at the substep's start: lambda_s = rho_hat.J rho_hat
 * (Eq. 12), r = rho_hat + dt J rho_hat, log_rho += log|r|,
 * rho_hat = r / |r|. Every step leaves one row of the stretching.txt
 * time series (felbm_gpu_main.cu:643-655): step (1, 2, ... since creation),
 * lambda (mean over the active tracers and their substeps), mean_log_rho,
 * var_log_rho (over all tracers), n_active (tracers with no rejected
 * substep), lambda_w, lambda_nw (split by the phase of the nearest node,
 * c < 1/2 wetting; NaN when that phase has no sample or phase_split is off),
 * n_w, n_nw (samples / substeps; n_w + n_nw = n_active with phase_split).
 * fe_tracers_stretch_rows hands out the rows made since its last call, oldest
 * first, at most max_rows of 9 doubles; the device keeps the last 65536. */
int fe_tracers_stretch_rows(fe_tracers* t, double* rows, int64_t max_rows, int64_t* count);
/* rho_hat [3][n] and log_rho [n] (either may be NULL), for particle files
 * and restarts; the setter checks that rho_hat holds unit vectors. */
int fe_tracers_stretch_state(fe_tracers* t, double* rho_hat, double* log_rho);
int fe_tracers_set_stretch_state(fe_tracers* t, const double* rho_hat, const double* log_rho);
/* Advect on a caller-given node-indexed velocity u [3][nodes] (solid nodes 0)
 * and, with phase_split, order parameter c [nodes] (may be NULL), held until
 * the next call, instead of the engine's; u == NULL returns to the engine's
 * velocity. (A frozen field, or an analytic one for tests.) */
int fe_tracers_set_velocity(fe_tracers* t, const double* u, const double* c);
/* Seeding (reference particles_init_mode): mode 0 uniform in the fluid
 * volume (count tracers); mode 1 planes normal to `axis` at the coordinates
 * offsets[0..nplanes-1], count tracers per plane, each plane resampled until
 * its quota of non-solid points is reached. pos_out [3][total],
 * plane_out [total] (plane index, or 0 for mode 0). */
int fe_tracers_seed(const uint8_t* solid, int nx, int ny, int nz, int mode, int axis, const double* offsets,
                    int nplanes, int64_t count, uint64_t seed, double* pos_out, int32_t* plane_out);

/* ---- files ----------------------------------------------------------------
 * The reference driver's on-disk formats (felbm_gpu_main.cu:86-189), HDF5
 * with the same dataset names, shapes and types, written without libhdf5
 * (contiguous datasets). Fields of the current state (refreshed as
 * fe_download_fields): density, concentration, u_x, u_y, u_z, pressure, n
 * values each in the reference order, float32 or float64 (output_float32);
 * deflate 1-9 (output_deflate) stores each as one chunk through the gzip
 * filter at that level, as write_fields_h5 does (felbm_gpu_main.cu:94-98). */
int fe_write_fields_h5(fe_engine* e, const char* path, int float32, int deflate);
/* geometry.h5: coords [n][3] int (x, y, z of each site) and size [3] int. */
int fe_write_geometry_h5(const char* path, const uint8_t* solid, int nx, int ny, int nz);
/* Checkpoint (write_checkpoint / read_checkpoint, :151-189): h, g (Vn
 * doubles), step (uint), target_mass, Vn (int). Reading refuses a Vn that
 * differs from the engine's, uploads the state and keeps the file's M0. */
int fe_checkpoint_write(fe_engine* e, const char* path, uint32_t step);
/* Writes a queued mass correction into the stored populations now, where
 * it would otherwise be applied at the next step (the state is then what
 * fe_download_state returns). fe_checkpoint_write calls it first, so the run
 * that continues and a restart from the file hold the same state. */
int fe_settle_mass_correction(fe_engine* e);
int fe_checkpoint_read(fe_engine* e, const char* path, uint32_t* step);
/* particles_<step>.h5: position [n][3], velocity [n][3] (if vel), id, Dm (if
 * dm), plane_id (if plane_id), rho_hat [n][3] and log_rho [n] (if given);
 * pos, vel and rho_hat as [3][n] (fe_tracers_download). */
int fe_write_particles_h5(const char* path, int64_t n, const double* pos, const double* vel, const int64_t* id,
                          const double* dm, const int32_t* plane_id, const double* rho_hat, const double* log_rho);
/* The driver's text time series (felbm_gpu_main.cu:600-698), one line per
 * call; header != 0 truncates the file and writes the column line first.
 * series.txt (timeseries_file): iter max_speed mean_ux mean_uy mean_uz mean_v2
 * total_order_parameter, from the six fe_flow_stats sums of n sites.
 * stretching.txt (particles_stretching_file): nrows rows of
 * fe_tracers_stretch_rows (step lambda mean_log_rho var_log_rho n_active
 * lambda_w lambda_nw n_w n_nw). */
int fe_write_series(const char* path, int header, uint32_t iter, const double stats[6], int64_t n);
int fe_write_stretching(const char* path, int header, const double* rows, int64_t nrows);
/* A new file holding one dataset (type as below, rank 1 or 2), contiguous,
 * or with deflate 1-9 one chunk through the gzip filter at that level. */
int fe_h5_write_dataset(const char* path, const char* name, int type, int rank, const int64_t* dims,
                        const void* data, int deflate);
/* One dataset of a file written here: type 0 double, 1 float, 2 int32,
 * 3 uint32; dims[rank]; raw bytes into data (NULL: shape only). */
int fe_h5_read_dataset(const char* path, const char* name, int* type, int64_t* dims, int* rank, void* data,
                       int64_t capacity_bytes);

/* ---- diagnostics ------------------------------------------------------- */
/* Time nsteps of fe_run with CUDA events on the engine's stream; ms_total is
 * the device time. */
int fe_time_run(fe_engine* e, int nsteps, float* ms_total);

/* ---- autotuner (no reference counterpart) -------------------------------
 * Times the brick shapes this lattice can use (3-D: 8x8x8, 16x8x8, and for
 * FP64/FP32 storage 8x8x4; nz == 1: 16x16x1), then 2, 8 and 32 steps per
 * graph launch with the fastest brick, each on its own engine over the given
 * geometry (steps timed after 3 warm-up steps, CUDA events), and records the
 * fastest pair for the size class: dimensionality, storage, collision,
 * near-wall rule, porosity in 0.05 bins, site count in powers of two.
 * Engines created afterwards with brick = FE_BRICK_AUTO (graph_steps = 0) in
 * that class take it. The table lives in the process; fe_tune_save/load keep
 * it in a text file. */
typedef struct fe_tune_report {
  int brick;                  /* chosen FE_BRICK_* */
  int graph_steps;            /* chosen steps per graph launch */
  int ncand;                  /* candidates timed */
  int cand_brick[8];
  int cand_graph_steps[8];
  double cand_mlups[8];
} fe_tune_report;
/* The brick (FE_BRICK_*) and graph length an engine was created with. */
int fe_engine_layout(const fe_engine* e, int* brick, int* graph_steps);
int fe_autotune(const fe_params* p, int nx, int ny, int nz, const uint8_t* solid, int device, int steps,
                fe_tune_report* out);
int fe_tune_save(const char* path);
int fe_tune_load(const char* path);
int fe_tune_clear(void);
/* Device time of each pass summed over nsteps plain steps: [0] moments,
 * [1] open-boundary kernels, [2] c field, [3] Laplacian of mu, [4] collide. */
int fe_time_kernels(fe_engine* e, int nsteps, float* ms_per_kernel, int nkernels);
/* Number of kernels the engine launched since creation. */
int fe_launch_count(const fe_engine* e, int64_t* count);
const char* fe_last_error(void);
const char* fe_version(void);

#ifdef __cplusplus
}
#endif
#endif /* FELBM_B200_H */
