// felbm_b200.hpp — header-only C++ drop-in over the C-ABI of felbm_b200.h.
//
// Mirrors the member functions of the reference's struct
// felbm_gpu::MultiPhaseGPU (include/felbm_gpu/multiphase_gpu.cuh:23-783) that
// its drivers call (src/felbm_gpu_main.cu, src/compare_cpu_gpu.cu):
//   step(), apply_mass_correction(), record_target_mass(), set/get_target_mass(),
//   current_mass(), upload_state(), download_state(), download(),
//   flow_stats(), flow_stats_launch/pending/ready/collect(), state_size(), free(),
// plus set_open_bnd() with the reference's argument meaning. Construction takes
// the solid mask and parameter block instead of felbm_local's SubDomain /
// Settings / ParametersMultiPhase objects (read_cfg() fills the parameter
// block from the reference's settings.cfg / params.cfg); errors throw
// fe::Error instead of exiting the process. The reference driver copies the
// device velocity (d_ux, d_uy, d_uz, d_c) to the host for its tracer worker
// (felbm_gpu_main.cu:760-763); here the tracers run on the device beside the
// engine (fe_tracers_*), and download() returns the fields.
#pragma once
#include <stdexcept>
#include <string>
#include <vector>

#include "felbm_b200.h"

namespace fe {

struct Error : std::runtime_error {
  int status;
  Error(int s, const std::string& m) : std::runtime_error(m), status(s) {}
};

inline void check(int status) {
  if (status != FE_OK) throw Error(status, fe_last_error());
}

// settings.cfg (+ the params.cfg it names) over p; the six fast-path switches
// are logged by switch_log()
inline void read_cfg(const std::string& settings, fe_params& p, fe_open_bnd& ob, fe_driver_cfg& d) {
  check(fe_cfg_read(settings.c_str(), &p, &ob, &d));
}
inline std::string switch_log(const fe_params& p) {
  std::string buf(4096, '\0');
  check(fe_cfg_switch_log(&p, &buf[0], (int)buf.size()));
  buf.resize(std::char_traits<char>::length(buf.c_str()));
  return buf;
}

class MultiPhaseGPU {
 public:
  MultiPhaseGPU() = default;
  MultiPhaseGPU(const fe_params& p, int nx, int ny, int nz, const uint8_t* solid, int device = -1) {
    init(p, nx, ny, nz, solid, device);
  }
  ~MultiPhaseGPU() { free(); }
  MultiPhaseGPU(const MultiPhaseGPU&) = delete;
  MultiPhaseGPU& operator=(const MultiPhaseGPU&) = delete;

  // multiphase_gpu.cuh:75-351
  void init(const fe_params& p, int nx, int ny, int nz, const uint8_t* solid, int device = -1) {
    free();
    check(fe_engine_create(&p, nx, ny, nz, solid, device, &e_));
    int64_t n = 0, vn = 0;
    check(fe_engine_size(e_, &n, &vn));
    n_ = n;
    Vn_ = vn;
  }
  // :759-782
  void free() {
    if (e_) fe_engine_destroy(e_);
    e_ = nullptr;
  }
  // :354-359 (host FP64, layout k*n+i)
  void upload_state(const double* h, const double* g) { check(fe_upload_state(e_, h, g, Vn_)); }
  // the equilibrium state at rest of per-site c and p (p null: p_uniform)
  void upload_equilibrium(const double* c, const double* p, double p_uniform = 1.0) {
    check(fe_upload_equilibrium(e_, c, p, p_uniform, Vn_ / 19));
  }
  // :449-455
  void download_state(std::vector<double>& h, std::vector<double>& g) {
    h.resize(Vn_);
    g.resize(Vn_);
    check(fe_download_state(e_, h.data(), g.data(), Vn_));
  }
  // :369-400 (site indices in the reference order)
  void set_open_bnd(fe_open_bnd b) { check(fe_set_open_bnd(e_, &b)); }
  // :522-631; the forcing factor is the driver's `P.forcing_factor`
  void step() { check(fe_step(e_, 1)); }
  void set_forcing_factor(double ff) { check(fe_set_forcing_factor(e_, ff)); }
  // fused driver loop: nsteps x (step + apply_mass_correction), CUDA graph
  void run(int nsteps) { check(fe_run(e_, nsteps)); }
  // :689-700
  double apply_mass_correction() {
    double d = 0.0;
    check(fe_apply_mass_correction(e_, &d));
    return d;
  }
  // queue the correction without the blocking drift readback
  void apply_mass_correction_async() { check(fe_apply_mass_correction(e_, nullptr)); }
  // :685-687, :458-459
  void record_target_mass() { check(fe_record_target_mass(e_)); }
  double get_target_mass() const {
    double m = 0.0;
    check(fe_get_target_mass(e_, &m));
    return m;
  }
  void set_target_mass(double m) { check(fe_set_target_mass(e_, m)); }
  double current_mass() {
    double m = 0.0;
    check(fe_current_mass(e_, &m));
    return m;
  }
  // :704-722 download(c, rho, ux, uy, uz, p)
  void download(std::vector<double>& c, std::vector<double>& rho, std::vector<double>& ux,
                std::vector<double>& uy, std::vector<double>& uz, std::vector<double>& p) {
    for (auto* v : {&c, &rho, &ux, &uy, &uz, &p}) v->resize(n_);
    fe_fields f{rho.data(), c.data(), ux.data(), uy.data(), uz.data(), p.data(), nullptr};
    check(fe_download_fields(e_, &f));
  }
  // the same with the chemical potential mu (download_raw's field set + mu)
  void download(std::vector<double>& c, std::vector<double>& rho, std::vector<double>& ux,
                std::vector<double>& uy, std::vector<double>& uz, std::vector<double>& p, std::vector<double>& mu) {
    for (auto* v : {&c, &rho, &ux, &uy, &uz, &p, &mu}) v->resize(n_);
    fe_fields f{rho.data(), c.data(), ux.data(), uy.data(), uz.data(), p.data(), mu.data()};
    check(fe_download_fields(e_, &f));
  }
  // :645-683
  void flow_stats(double out[6]) { check(fe_flow_stats(e_, out)); }
  void flow_stats_launch() {
    check(fe_flow_stats_launch(e_));
    pending_ = true;
  }
  bool flow_stats_pending() const { return pending_; }
  bool flow_stats_ready() {
    int r = 0;
    check(fe_flow_stats_ready(e_, &r));
    return r != 0;
  }
  void flow_stats_collect(double out[6]) {
    check(fe_flow_stats_collect(e_, out));
    pending_ = false;
  }
  // :457
  int state_size() const { return (int)Vn_; }
  int64_t size_sites() const { return n_; }
  fe_engine* handle() const { return e_; }

 private:
  fe_engine* e_ = nullptr;
  int64_t n_ = 0, Vn_ = 0;
  bool pending_ = false;
};

}  // namespace fe
