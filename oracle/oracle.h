/*
 * CPU oracle for the Lee–Liu D3Q19 step — TEST INFRASTRUCTURE ONLY.
 *
 * A plain FP64 restatement of the reference GPU engine (matNBI/felbm_gpu,
 * include/felbm_gpu/device_engine.cuh + multiphase_gpu.cuh) in the reference's
 * own data layout (f[k*n+i]) and with the reference's own neighbour/case
 * tables. Only tests/, __graft_entry__.smoke() and bench.py's CPU baseline
 * leg use it, to compare against; the product never links or calls it.
 *
 * Parity pin: the reference's CPU engine (felbm_local EngineMultiPhase) is not
 * part of the reference snapshot, so this oracle restates the reference's GPU
 * kernels, which the reference documents as equal to EngineMultiPhase to
 * ~1e-15 (README.md:10-14). The restatement itself is pinned against the
 * reference's own kernels (device_engine.cuh compiled unmodified for sm_100a
 * by oracle/ref/build_ref.sh) through golden vectors in tests/golden/.
 * Semantics that live only in felbm_local (site set, is_known, streaming rows,
 * MRT matrix values, initial conditions) are this project's definitions,
 * written once in the kernels and once here, and are unpinned.
 */
#ifndef FE_ORACLE_H
#define FE_ORACLE_H
#include <stdint.h>
#include "../include/felbm_b200.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct or_engine or_engine;

/* inplace = 1 streams through the reference's disjoint in-place op program
 * (multiphase_gpu.cuh:213-283) instead of the gather table. */
or_engine* or_create(const fe_params* p, int nx, int ny, int nz, const uint8_t* solid, int inplace);
void or_destroy(or_engine* e);
int64_t or_n(const or_engine* e);
/* site index (reference order) -> node index x + nx*(y + ny*z) */
void or_site_nodes(const or_engine* e, int64_t* node);
int or_set_open_bnd(or_engine* e, const fe_open_bnd* b);
void or_set_params(or_engine* e, const fe_params* p);
void or_upload(or_engine* e, const double* h, const double* g);
void or_download(const or_engine* e, double* h, double* g);
void or_set_forcing_factor(or_engine* e, double ff);
void or_step(or_engine* e);
double or_apply_mass_correction(or_engine* e);
void or_record_target_mass(or_engine* e);
double or_target_mass(const or_engine* e);
void or_set_target_mass(or_engine* e, double m0);
double or_current_mass(or_engine* e);
/* fields as left by the last step (start-of-step values, as compare_cpu_gpu reads) */
void or_fields(const or_engine* e, const fe_fields* f);
/* download()/download_raw(): refresh fields from the current state */
void or_download_fields(or_engine* e, const fe_fields* f);
void or_flow_stats(const or_engine* e, double out[6]);
/* the in-place op program counts (swaps, avgs, zeros); -1 if not reducible */
void or_inplace_counts(const or_engine* e, int64_t out[3]);
/* reference tables, for table-level tests: which = 0 cdm,1 cdp,2 bcase,3 bc1,
 * 4 bc2,5 lcase,6 lc1,7 lc2 ((Q-1)*n each), 8 avgnext (Q*n), 9 src (Q*n) */
void or_table(const or_engine* e, int which, int32_t* out);
/* the in-place op program (a, b, type); returns its length, -1 if unused */
int64_t or_inplace_program(const or_engine* e, int32_t* a, int32_t* b, uint8_t* t);
/* fe_run equivalent: nsteps x (forcing factor of step t, step, mass correction) */
void or_run(or_engine* e, int nsteps, int64_t t0);
void or_mrt_matrices(double* M, double* Minv);
/* OpenMP threads the oracle's loops use (omp_get_max_threads / omp_set_num_threads) */
int or_threads(void);
void or_set_threads(int n);

#ifdef __cplusplus
}
#endif
#endif
