// Harness around the reference's own GPU kernels — TEST INFRASTRUCTURE ONLY.
//
// Compiles matNBI/felbm_gpu's include/felbm_gpu/device_engine.cuh unmodified
// (FP64, or FP32 with -DFELBM_SINGLE) for sm_100a and drives its kernels in the
// order of MultiPhaseGPU::step (include/felbm_gpu/multiphase_gpu.cuh:522-631,
// production path: matrix-free tables, fuse_collision, optional
// mrt_fast_transform and stream_inplace) and apply_mass_correction (:689-700).
// multiphase_gpu.cuh itself needs felbm_local and is not compiled; the
// neighbour/case tables, streaming table, in-place program and MRT matrices
// are passed in from the CPU oracle, which restates the reference's builders.
// This code is built by oracle/ref/build_ref.sh into oracle/_ref/ and used by
// the tests to pin the oracle to the reference's kernels, and by the bench as
// the same-GPU reference-kernel baseline.
#include <felbm_gpu/device_engine.cuh>

#include <cstdint>
#include <cstring>
#include <vector>

#include "../../include/felbm_b200.h"

using namespace felbm_gpu;

namespace {
struct Ref {
  int n = 0, Vn = 0;
  bool mrt = false, correct_mass = false, inplace = false;
  DevParams P{};
  real_t *h = 0, *g = 0, *h2 = 0, *g2 = 0;
  real_t *c = 0, *p = 0, *rho = 0, *mu = 0, *ux = 0, *uy = 0, *uz = 0, *lapc = 0, *lapmu = 0, *relax = 0;
  real_t *gcc[3] = {}, *gcb[3] = {}, *gcm[3] = {}, *gpc[3] = {}, *gpb[3] = {}, *gpm[3] = {};
  real_t* xtnd = 0;
  int *cdm = 0, *cdp = 0, *bcase = 0, *bc1 = 0, *bc2 = 0, *avgnext = 0, *lcase = 0, *lc1 = 0, *lc2 = 0, *src = 0;
  int n_sops = 0;
  int *sop_a = 0, *sop_b = 0;
  unsigned char* sop_t = 0;
  unsigned char *solid = 0, *stream = 0, *bcproc = 0;
  int *inlet = 0, *outlet = 0, *bufv = 0, *bufr = 0;
  real_t* inlet_coord = 0;
  double* reduce = 0;
  double target_mass = 0.0;
  unsigned open_step = 0;
  std::vector<void*> allocs;
  template <class T>
  T* A(size_t cnt) {
    T* q = nullptr;
    if (cudaMalloc(&q, std::max<size_t>(cnt, 1) * sizeof(T)) != cudaSuccess) return nullptr;
    allocs.push_back(q);
    return q;
  }
  template <class T>
  T* up(const T* src_, size_t cnt) {
    T* d = A<T>(cnt);
    if (d && cnt) cudaMemcpy(d, src_, cnt * sizeof(T), cudaMemcpyHostToDevice);
    return d;
  }
};

// enforce_open_bnd_fields (multiphase_gpu.cuh:404-418)
void enforce(Ref* R) {
  if (!R->P.open_bnd) return;
  if (R->P.n_inlet)
    k_open_bnd_fields<<<grid_1d(R->P.n_inlet, BLOCK), BLOCK>>>(R->P, R->open_step, 1, R->inlet, R->inlet_coord,
                                                              R->c, R->rho, R->p, R->ux, R->uy, R->uz);
  if (R->P.n_outlet)
    k_open_bnd_fields<<<grid_1d(R->P.n_outlet, BLOCK), BLOCK>>>(R->P, R->open_step, 0, R->outlet,
                                                               (real_t const*)0, R->c, R->rho, R->p, R->ux,
                                                               R->uy, R->uz);
  if (R->P.copy_to_buf && R->P.n_buf)
    k_open_bnd_buf_fields<<<grid_1d(R->P.n_buf, BLOCK), BLOCK>>>(R->P.n_buf, R->bufv, R->bufr, R->c, R->rho, R->p,
                                                                R->ux, R->uy, R->uz);
}

// apply_open_bnd (multiphase_gpu.cuh:427-446)
void apply_bc(Ref* R) {
  if (!R->P.open_bnd) return;
  if (R->P.copy_to_buf) {
    if (R->P.n_buf)
      k_open_bnd_buf<<<grid_1d(R->P.n_buf, BLOCK), BLOCK>>>(R->P, R->P.n_buf, R->bufv, R->bufr, R->c, R->rho, R->p,
                                                           R->ux, R->uy, R->uz, R->h, R->g);
  } else {
    if (R->P.n_inlet)
      k_open_bnd<<<grid_1d(R->P.n_inlet, BLOCK), BLOCK>>>(R->P, R->open_step, 1, R->inlet, R->inlet_coord, R->c,
                                                         R->rho, R->p, R->ux, R->uy, R->uz, R->h, R->g);
    if (R->P.n_outlet)
      k_open_bnd<<<grid_1d(R->P.n_outlet, BLOCK), BLOCK>>>(R->P, R->open_step, 0, R->outlet, (real_t const*)0,
                                                          R->c, R->rho, R->p, R->ux, R->uy, R->uz, R->h, R->g);
  }
  ++R->open_step;
}

void fields(Ref* R, bool full) {
  const int n = R->n;
  dim3 gN = grid_1d(n, BLOCK);
  k_moments<<<gN, BLOCK>>>(R->P, R->h, R->g, R->c, R->p, R->rho, R->mu, R->ux, R->uy, R->uz, R->relax);
  enforce(R);
  k_grad_cd_mf<<<gN, BLOCK>>>(n, R->P.alpha, R->cdm, R->cdp, R->c, R->gcc[0], R->gcc[1], R->gcc[2]);
  if (full) {
    k_grad_bd_mf<<<gN, BLOCK>>>(n, R->P.alpha, R->bcase, R->bc1, R->bc2, R->c, R->gcb[0], R->gcb[1], R->gcb[2]);
    k_grad_md<<<gN, BLOCK>>>(n, R->gcc[0], R->gcc[1], R->gcc[2], R->gcb[0], R->gcb[1], R->gcb[2], R->gcm[0],
                             R->gcm[1], R->gcm[2]);
  }
  k_pack_lap_c<<<gN, BLOCK>>>(R->P, R->c, R->xtnd);
  k_lap_mf<<<gN, BLOCK>>>(n, R->P.alpha, R->xtnd, R->lcase, R->lc1, R->lc2, R->lapc);
  k_mu_axpy<<<gN, BLOCK>>>(n, R->P.kappa, R->lapc, R->mu);
  if (full) {
    k_pack_lap_zero<<<gN, BLOCK>>>(n, R->mu, R->xtnd);
    k_lap_mf<<<gN, BLOCK>>>(n, R->P.alpha, R->xtnd, R->lcase, R->lc1, R->lc2, R->lapmu);
  }
  k_vel_press_corr<<<gN, BLOCK>>>(R->P, R->mu, R->rho, R->gcc[0], R->gcc[1], R->gcc[2], R->ux, R->uy, R->uz, R->p,
                                  R->bcproc);
  if (full) {
    k_grad_cd_mf<<<gN, BLOCK>>>(n, R->P.alpha, R->cdm, R->cdp, R->p, R->gpc[0], R->gpc[1], R->gpc[2]);
    k_grad_bd_mf<<<gN, BLOCK>>>(n, R->P.alpha, R->bcase, R->bc1, R->bc2, R->p, R->gpb[0], R->gpb[1], R->gpb[2]);
    k_grad_md<<<gN, BLOCK>>>(n, R->gpc[0], R->gpc[1], R->gpc[2], R->gpb[0], R->gpb[1], R->gpb[2], R->gpm[0],
                             R->gpm[1], R->gpm[2]);
  }
}

void reduce_mass_weight(Ref* R, double& M, double& W) {
  double zero[2] = {0.0, 0.0};
  cudaMemcpy(R->reduce, zero, sizeof(zero), cudaMemcpyHostToDevice);
  k_mass_weight<<<grid_1d(R->n, BLOCK), BLOCK>>>(R->P, R->stream, R->h, R->reduce);
  double h2[2];
  cudaMemcpy(h2, R->reduce, sizeof(h2), cudaMemcpyDeviceToHost);
  M = h2[0];
  W = h2[1];
}
}  // namespace

extern "C" {

int ref_real_size(void) { return (int)sizeof(real_t); }

// tables: cdm,cdp,bcase,bc1,bc2,lcase,lc1,lc2 ((Q-1)n each), avgnext, src (Qn);
// op program (n_sops >= 0 selects stream_inplace); M, Minv row-major 19x19.
void* ref_create(const fe_params* p, int n, const int32_t* const* tables, int n_sops, const int32_t* sop_a,
                 const int32_t* sop_b, const uint8_t* sop_t, const double* M, const double* Minv) {
  Ref* R = new Ref();
  R->n = n;
  R->Vn = Q * n;
  const size_t Q1n = (size_t)(Q - 1) * n, Vn = (size_t)Q * n;
  upload_d3q19_constants();
  upload_mrt_matrices(M, Minv);
  R->cdm = R->up(tables[0], Q1n); R->cdp = R->up(tables[1], Q1n);
  R->bcase = R->up(tables[2], Q1n); R->bc1 = R->up(tables[3], Q1n); R->bc2 = R->up(tables[4], Q1n);
  R->lcase = R->up(tables[5], Q1n); R->lc1 = R->up(tables[6], Q1n); R->lc2 = R->up(tables[7], Q1n);
  R->avgnext = R->up(tables[8], Vn); R->src = R->up(tables[9], Vn);
  R->inplace = n_sops >= 0;
  if (R->inplace) {
    R->n_sops = n_sops;
    R->sop_a = R->up(sop_a, n_sops); R->sop_b = R->up(sop_b, n_sops); R->sop_t = R->up(sop_t, n_sops);
  }
  R->h = R->A<real_t>(Vn); R->g = R->A<real_t>(Vn);
  if (!R->inplace) { R->h2 = R->A<real_t>(Vn); R->g2 = R->A<real_t>(Vn); }
  real_t** f[] = {&R->c, &R->p, &R->rho, &R->mu, &R->ux, &R->uy, &R->uz, &R->lapc, &R->lapmu, &R->relax};
  for (real_t** q : f) *q = R->A<real_t>(n);
  for (int d = 0; d < 3; ++d) {
    R->gcc[d] = R->A<real_t>(n); R->gcb[d] = R->A<real_t>(n); R->gcm[d] = R->A<real_t>(n);
    R->gpc[d] = R->A<real_t>(n); R->gpb[d] = R->A<real_t>(n); R->gpm[d] = R->A<real_t>(n);
  }
  R->xtnd = R->A<real_t>(2 * (size_t)n);
  R->reduce = R->A<double>(2);
  std::vector<unsigned char> ones(n, 1), zeros(n, 0);
  R->solid = R->up(zeros.data(), n);
  R->stream = R->up(ones.data(), n);
  // DevParams fill (multiphase_gpu.cuh:331-343)
  DevParams& P = R->P;
  P.n = n;
  P.rho0 = (real_t)p->rho0; P.rho1 = (real_t)p->rho1; P.drho = P.rho0 - P.rho1;
  P.kappa = (real_t)p->kappa; P.beta = (real_t)p->beta; P.four_beta = (real_t)(4.0 * p->beta);
  P.bnd_coeff = (real_t)p->bnd_coeff;
  P.tau0 = (real_t)p->tau0; P.tau1 = (real_t)p->tau1;
  P.cs2 = (real_t)CS2; P.alpha = (real_t)ALPHA; P.gamma_c = (real_t)GAMMA; P.beta_c = (real_t)BETA;
  P.mobility = (real_t)p->mobility; P.forcing_factor = (real_t)1.0;
  P.gx = (real_t)p->gx; P.gy = (real_t)p->gy; P.gz = (real_t)p->gz;
  P.fx = (real_t)p->fx; P.fy = (real_t)p->fy; P.fz = (real_t)p->fz;
  P.mrt_lambda = (real_t)p->mrt_lambda;
  P.mrt_fast = p->mrt_fast_transform ? 1 : 0;
  P.stream_inplace = R->inplace ? 1 : 0;
  R->mrt = p->use_mrt != 0;
  R->correct_mass = p->correct_op_mass != 0;
  return R;
}

int ref_set_open_bnd(void* h, const fe_open_bnd* b) {
  Ref* R = static_cast<Ref*>(h);
  DevParams& P = R->P;
  P.open_bnd = 1;
  P.use_in_vel = b->use_in_vel; P.use_in_prs = b->use_in_prs; P.use_in_fluid = b->use_in_fluid;
  P.use_out_prs = b->use_out_prs; P.use_out_fluid = b->use_out_fluid;
  P.u_in_x = (real_t)b->u_in_x; P.u_in_y = (real_t)b->u_in_y; P.u_in_z = (real_t)b->u_in_z;
  P.p_in = (real_t)b->p_in; P.p_out = (real_t)b->p_out;
  P.c_out_fixed = (real_t)b->c_out_fixed; P.rho_out_fixed = (real_t)b->rho_out_fixed;
  P.inlet_c_a = (real_t)b->inlet_c_a; P.inlet_mode = b->inlet_mode; P.split_axis = b->split_axis;
  P.inlet_period = (real_t)b->inlet_period; P.inlet_duty = (real_t)b->inlet_duty;
  P.inlet_ramp = (real_t)b->inlet_ramp; P.split_pos = (real_t)b->split_pos;
  // set_open_bnd (multiphase_gpu.cuh:369-400)
  P.n_inlet = b->n_inlet; P.n_outlet = b->n_outlet;
  std::vector<unsigned char> bp(R->n, 0);
  if (P.use_in_vel || P.use_in_prs || P.use_in_fluid)
    for (int q = 0; q < b->n_inlet; ++q) bp[b->inlet[q]] = 1;
  if (P.use_out_prs || P.use_out_fluid)
    for (int q = 0; q < b->n_outlet; ++q) bp[b->outlet[q]] = 1;
  if (b->copy_to_buffers)
    for (int q = 0; q < b->n_buf; ++q) bp[b->buf_verts[q]] = 1;
  R->bcproc = R->up(bp.data(), R->n);
  if (P.n_inlet) R->inlet = R->up(b->inlet, P.n_inlet);
  if (P.n_outlet) R->outlet = R->up(b->outlet, P.n_outlet);
  if (b->inlet_coord && P.n_inlet) {
    std::vector<real_t> ic(b->inlet_coord, b->inlet_coord + P.n_inlet);
    R->inlet_coord = R->up(ic.data(), ic.size());
  }
  P.n_buf = b->n_buf;
  P.copy_to_buf = b->copy_to_buffers ? 1 : 0;
  if (P.n_buf) { R->bufv = R->up(b->buf_verts, P.n_buf); R->bufr = R->up(b->buf_refs, P.n_buf); }
  return 0;
}

void ref_set_forcing_factor(void* h, double ff) { static_cast<Ref*>(h)->P.forcing_factor = (real_t)ff; }

int ref_upload(void* h, const double* hh, const double* gg) {
  Ref* R = static_cast<Ref*>(h);
  std::vector<real_t> t(R->Vn);
  for (int j = 0; j < R->Vn; ++j) t[j] = (real_t)hh[j];
  cudaMemcpy(R->h, t.data(), R->Vn * sizeof(real_t), cudaMemcpyHostToDevice);
  for (int j = 0; j < R->Vn; ++j) t[j] = (real_t)gg[j];
  cudaMemcpy(R->g, t.data(), R->Vn * sizeof(real_t), cudaMemcpyHostToDevice);
  return (int)cudaGetLastError();
}

int ref_download(void* h, double* hh, double* gg) {
  Ref* R = static_cast<Ref*>(h);
  std::vector<real_t> t(R->Vn);
  cudaMemcpy(t.data(), R->h, R->Vn * sizeof(real_t), cudaMemcpyDeviceToHost);
  for (int j = 0; j < R->Vn; ++j) hh[j] = (double)t[j];
  cudaMemcpy(t.data(), R->g, R->Vn * sizeof(real_t), cudaMemcpyDeviceToHost);
  for (int j = 0; j < R->Vn; ++j) gg[j] = (double)t[j];
  return (int)cudaGetLastError();
}

// MultiPhaseGPU::step, fuse_collision + matrix-free path (:522-631)
int ref_step(void* h) {
  Ref* R = static_cast<Ref*>(h);
  const int n = R->n;
  dim3 gN = grid_1d(n, BLOCK), gVn = grid_1d(R->Vn, BLOCK);
  fields(R, true);
  apply_bc(R);
  if (R->mrt)
    k_collide_fused_mrt<<<gN, BLOCK>>>(R->P, R->stream, R->c, R->rho, R->p, R->mu, R->ux, R->uy, R->uz, R->gpc[0],
                                       R->gpc[1], R->gpc[2], R->gcc[0], R->gcc[1], R->gcc[2], R->gpm[0], R->gpm[1],
                                       R->gpm[2], R->gcm[0], R->gcm[1], R->gcm[2], R->lapmu, R->relax, R->cdm,
                                       R->cdp, R->bcase, R->bc1, R->bc2, R->avgnext, R->h, R->g);
  else
    k_collide_fused_bgk<<<gN, BLOCK>>>(R->P, R->solid, R->stream, R->c, R->rho, R->p, R->mu, R->ux, R->uy, R->uz,
                                       R->gpc[0], R->gpc[1], R->gpc[2], R->gcc[0], R->gcc[1], R->gcc[2], R->gpm[0],
                                       R->gpm[1], R->gpm[2], R->gcm[0], R->gcm[1], R->gcm[2], R->lapmu, R->relax,
                                       R->cdm, R->cdp, R->bcase, R->bc1, R->bc2, R->avgnext, R->h, R->g);
  if (R->inplace) {
    k_stream_inplace<<<(R->n_sops + BLOCK - 1) / BLOCK, BLOCK>>>(R->n_sops, R->sop_a, R->sop_b, R->sop_t, R->h,
                                                                  R->g);
  } else {
    k_stream_gather<<<gVn, BLOCK>>>(R->Vn, n, R->src, R->h, R->h2);
    k_stream_gather<<<gVn, BLOCK>>>(R->Vn, n, R->src, R->g, R->g2);
    std::swap(R->h, R->h2);
    std::swap(R->g, R->g2);
  }
  return (int)cudaGetLastError();
}

void ref_record_target_mass(void* h) {
  Ref* R = static_cast<Ref*>(h);
  double M, W;
  reduce_mass_weight(R, M, W);
  R->target_mass = M;
}
void ref_set_target_mass(void* h, double m) { static_cast<Ref*>(h)->target_mass = m; }

// apply_mass_correction (:689-700)
double ref_apply_mass_correction(void* h) {
  Ref* R = static_cast<Ref*>(h);
  if (!R->correct_mass) return 0.0;
  double M, W;
  reduce_mass_weight(R, M, W);
  const double drift = M - R->target_mass;
  if (W > 0.0 && drift != 0.0)
    k_inject_mass<<<grid_1d(R->n, BLOCK), BLOCK>>>(R->P, R->stream, drift / W, R->h);
  return drift;
}

// fields of the last step (as compare_cpu_gpu reads them) or refreshed
// (download_raw, :731-757); order rho, c, ux, uy, uz, p, mu
int ref_fields(void* h, int refresh, double* const* out) {
  Ref* R = static_cast<Ref*>(h);
  if (refresh) fields(R, false);
  real_t* src[7] = {R->rho, R->c, R->ux, R->uy, R->uz, R->p, R->mu};
  std::vector<real_t> t(R->n);
  for (int q = 0; q < 7; ++q) {
    if (!out[q]) continue;
    cudaMemcpy(t.data(), src[q], R->n * sizeof(real_t), cudaMemcpyDeviceToHost);
    for (int i = 0; i < R->n; ++i) out[q][i] = (double)t[i];
  }
  return (int)cudaGetLastError();
}

int ref_sync(void) { return (int)cudaDeviceSynchronize(); }

void ref_destroy(void* h) {
  Ref* R = static_cast<Ref*>(h);
  for (void* a : R->allocs) cudaFree(a);
  delete R;
}

}  // extern "C"
