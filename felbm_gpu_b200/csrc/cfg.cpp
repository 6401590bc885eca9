// Reader of the reference driver's configuration files (host C++).
//
// The reference's felbm_gpu reads settings.cfg through felbm_local's
// util::ConfigFile and Settings (absent from the reference snapshot), the
// physics block from the params.cfg named by `param_file`, and a handful of
// felbm_gpu-only keys directly (src/felbm_gpu_main.cu:198-235). This reader
// takes the same files: `key = value` lines, `#` starts a comment, values may
// be double-quoted, booleans are true/false (or 1/0). It fills the engine's
// parameter block (the fe_params fields carry the cfg key names), the
// open-boundary flags and values the driver copies into DevParams
// (felbm_gpu_main.cu:334-360), and the driver-level keys. Keys it does not
// know are counted and left alone, as felbm_local leaves keys it does not ask
// for.
#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>

#include "../../include/felbm_b200.h"
#include "fe_internal.hpp"

namespace fe {
namespace {

using KV = std::map<std::string, std::string>;

std::string trim(const std::string& s) {
  size_t a = 0, b = s.size();
  while (a < b && std::isspace((unsigned char)s[a])) ++a;
  while (b > a && std::isspace((unsigned char)s[b - 1])) --b;
  return s.substr(a, b - a);
}

// key = value lines; a '#' outside double quotes starts a comment.
int parse_file(const std::string& path, KV& kv, std::string& err) {
  std::ifstream in(path);
  if (!in) {
    err = "cannot open " + path;
    return FE_ERR_IO;
  }
  std::string line;
  int lineno = 0;
  while (std::getline(in, line)) {
    ++lineno;
    bool q = false;
    size_t cut = line.size();
    for (size_t i = 0; i < line.size(); ++i) {
      if (line[i] == '"') q = !q;
      if (line[i] == '#' && !q) {
        cut = i;
        break;
      }
    }
    line = trim(line.substr(0, cut));
    if (line.empty()) continue;
    const size_t eq = line.find('=');
    if (eq == std::string::npos) {
      err = path + ":" + std::to_string(lineno) + ": expected key = value";
      return FE_ERR_ARG;
    }
    std::string key = trim(line.substr(0, eq)), val = trim(line.substr(eq + 1));
    if (val.size() >= 2 && val.front() == '"' && val.back() == '"') val = val.substr(1, val.size() - 2);
    if (key.empty()) {
      err = path + ":" + std::to_string(lineno) + ": empty key";
      return FE_ERR_ARG;
    }
    kv[key] = val;
  }
  return FE_OK;
}

struct Reader {
  const KV& kv;
  std::string err;
  std::map<std::string, bool> used;
  bool has(const char* k) {
    auto it = kv.find(k);
    if (it == kv.end()) return false;
    used[k] = true;
    return true;
  }
  bool get_double(const char* k, double& out) {
    if (!has(k)) return true;
    const std::string& v = kv.at(k);
    char* end = nullptr;
    const double x = std::strtod(v.c_str(), &end);
    if (end == v.c_str() || *end != '\0') {
      err = std::string("key ") + k + ": not a number: " + v;
      return false;
    }
    out = x;
    return true;
  }
  bool get_int(const char* k, int& out) {
    double x = out;
    if (!get_double(k, x)) return false;
    if (x != std::floor(x)) {
      err = std::string("key ") + k + ": not an integer";
      return false;
    }
    out = (int)x;
    return true;
  }
  bool get_i64(const char* k, int64_t& out) {
    double x = (double)out;
    if (!get_double(k, x)) return false;
    out = (int64_t)x;
    return true;
  }
  bool get_bool(const char* k, int& out) {
    if (!has(k)) return true;
    std::string v = kv.at(k);
    for (auto& ch : v) ch = (char)std::tolower((unsigned char)ch);
    if (v == "true" || v == "1" || v == "yes" || v == "on") out = 1;
    else if (v == "false" || v == "0" || v == "no" || v == "off") out = 0;
    else {
      err = std::string("key ") + k + ": not a boolean: " + kv.at(k);
      return false;
    }
    return true;
  }
  bool get_str(const char* k, char* dst, size_t cap) {
    if (!has(k)) return true;
    const std::string& v = kv.at(k);
    if (v.size() + 1 > cap) {
      err = std::string("key ") + k + ": value longer than " + std::to_string(cap - 1) + " characters";
      return false;
    }
    std::memcpy(dst, v.c_str(), v.size() + 1);
    return true;
  }
};

void set_str(char* dst, size_t cap, const char* v) {
  std::snprintf(dst, cap, "%s", v);
}

std::string dir_of(const std::string& path) {
  const size_t s = path.find_last_of('/');
  return s == std::string::npos ? std::string() : path.substr(0, s + 1);
}

}  // namespace
}  // namespace fe

extern "C" {

int fe_driver_cfg_default(fe_driver_cfg* d) {
  if (!d) return fe::fe_fail(FE_ERR_ARG, "fe_driver_cfg_default: null");
  std::memset(d, 0, sizeof(*d));
  fe::set_str(d->model, sizeof(d->model), "multi_phase");
  fe::set_str(d->output_dir, sizeof(d->output_dir), "./");
  fe::set_str(d->output_name, sizeof(d->output_name), "output");
  fe::set_str(d->timeseries_file, sizeof(d->timeseries_file), "series.txt");
  fe::set_str(d->log_file, sizeof(d->log_file), "log.txt");
  fe::set_str(d->param_file, sizeof(d->param_file), "params.cfg");
  fe::set_str(d->velocity_set, sizeof(d->velocity_set), "d3q19");
  d->size_x = d->size_y = d->size_z = 1;
  d->max_iterations = 0;
  d->log_skip = 1;
  d->file_skip = 0;
  d->gpu_device = -1;
  d->in_out_dir = 0;
  d->particles_int_order = 2;
  d->particles_substeps = 1;
  d->particles_dt = 1.0;
  return FE_OK;
}

int fe_cfg_read(const char* settings_path, fe_params* p, fe_open_bnd* ob, fe_driver_cfg* d) {
  using namespace fe;
  if (!settings_path || !p || !d) return fe_fail(FE_ERR_ARG, "fe_cfg_read: null argument");
  KV kv;
  std::string err;
  int rc = parse_file(settings_path, kv, err);
  if (rc) return fe_fail(rc, "fe_cfg_read: " + err);
  Reader R{kv, {}, {}};
  fe_driver_cfg dc;
  fe_driver_cfg_default(&dc);
  fe_params P = *p;
  bool ok = true;
  // ---- driver-level keys (felbm_gpu_main.cu:198-235 and the Settings the
  // driver reads: output, logging, run length, domain, initializer, tracers)
  ok = ok && R.get_str("model", dc.model, sizeof(dc.model));
  ok = ok && R.get_str("output_dir", dc.output_dir, sizeof(dc.output_dir));
  ok = ok && R.get_str("output_name", dc.output_name, sizeof(dc.output_name));
  ok = ok && R.get_str("timeseries_file", dc.timeseries_file, sizeof(dc.timeseries_file));
  ok = ok && R.get_str("log_file", dc.log_file, sizeof(dc.log_file));
  ok = ok && R.get_str("param_file", dc.param_file, sizeof(dc.param_file));
  ok = ok && R.get_str("velocity_set", dc.velocity_set, sizeof(dc.velocity_set));
  ok = ok && R.get_str("domain_geometry", dc.domain_geometry, sizeof(dc.domain_geometry));
  ok = ok && R.get_str("domain_cfg_file", dc.domain_cfg_file, sizeof(dc.domain_cfg_file));
  ok = ok && R.get_str("fluid_initializer", dc.fluid_initializer, sizeof(dc.fluid_initializer));
  ok = ok && R.get_str("fluid_init_filename", dc.fluid_init_filename, sizeof(dc.fluid_init_filename));
  ok = ok && R.get_str("restart_file", dc.restart_file, sizeof(dc.restart_file));
  ok = ok && R.get_int("size_x", dc.size_x) && R.get_int("size_y", dc.size_y) && R.get_int("size_z", dc.size_z);
  ok = ok && R.get_i64("max_iterations", dc.max_iterations);
  ok = ok && R.get_int("log_skip", dc.log_skip) && R.get_int("file_skip", dc.file_skip);
  {
    int cs = 0;
    ok = ok && R.get_int("checkpoint_skip", cs);
    if (cs < 0) {
      R.err = "key checkpoint_skip: negative";
      ok = false;
    }
    dc.checkpoint_skip = (uint32_t)cs;
  }
  ok = ok && R.get_int("output_deflate", dc.output_deflate);
  if (ok && (dc.output_deflate < 0 || dc.output_deflate > 9)) {
    R.err = "key output_deflate: gzip level 0-9";
    ok = false;
  }
  ok = ok && R.get_bool("output_float32", dc.output_float32);
  ok = ok && R.get_int("gpu_device", dc.gpu_device);
  ok = ok && R.get_bool("logging", dc.logging) && R.get_bool("console", dc.console);
  ok = ok && R.get_bool("use_open_bnd", dc.use_open_bnd) && R.get_int("in_out_dir", dc.in_out_dir);
  ok = ok && R.get_int("buffer_layers", dc.buffer_layers) && R.get_int("empty_layers", dc.empty_layers);
  ok = ok && R.get_bool("extrude_buffers", dc.extrude_buffers) && R.get_bool("image_periodic", dc.image_periodic);
  ok = ok && R.get_bool("transverse_periodic", dc.transverse_periodic);
  ok = ok && R.get_bool("particles_enable", dc.particles_enable);
  ok = ok && R.get_i64("particles_number", dc.particles_number);
  ok = ok && R.get_str("particles_init_mode", dc.particles_init_mode, sizeof(dc.particles_init_mode));
  ok = ok && R.get_str("particles_plane_offsets", dc.particles_plane_offsets, sizeof(dc.particles_plane_offsets));
  ok = ok && R.get_str("particles_dm_groups", dc.particles_dm_groups, sizeof(dc.particles_dm_groups));
  ok = ok && R.get_int("particles_int_order", dc.particles_int_order);
  ok = ok && R.get_int("particles_substeps", dc.particles_substeps);
  ok = ok && R.get_double("particles_dt", dc.particles_dt);
  ok = ok && R.get_int("particles_file_skip", dc.particles_file_skip);
  // ---- solver keys of settings.cfg into the parameter block
  ok = ok && R.get_double("acceleration_x", P.gx) && R.get_double("acceleration_y", P.gy) &&
       R.get_double("acceleration_z", P.gz);
  ok = ok && R.get_double("forcing_x", P.fx) && R.get_double("forcing_y", P.fy) && R.get_double("forcing_z", P.fz);
  if (ok && R.has("forcing_timedep")) {
    // the driver matches by substring (felbm_gpu_main.cu:590-591)
    const std::string& v = kv.at("forcing_timedep");
    P.forcing_timedep = v.find("sinusoidal") != std::string::npos ? FE_FORCING_SINUSOIDAL
                        : v.find("square") != std::string::npos   ? FE_FORCING_SQUARE
                                                                  : FE_FORCING_CONSTANT;
  }
  ok = ok && R.get_double("forcing_period", P.forcing_period);
  ok = ok && R.get_bool("use_mrt", P.use_mrt) && R.get_double("mrt_lambda", P.mrt_lambda);
  ok = ok && R.get_bool("use_halfway_bb", P.use_halfway_bb) && R.get_bool("correct_op_mass", P.correct_op_mass);
  ok = ok && R.get_bool("stream_matrix_free", P.stream_matrix_free) &&
       R.get_bool("grad_matrix_free", P.grad_matrix_free) && R.get_bool("fused", P.fused) &&
       R.get_bool("fuse_collision", P.fuse_collision) && R.get_bool("mrt_fast_transform", P.mrt_fast_transform) &&
       R.get_bool("stream_inplace", P.stream_inplace);
  // ---- open-boundary flags and values (felbm_gpu_main.cu:340-365)
  fe_open_bnd B{};
  if (ob) B = *ob;
  int in_vel = B.use_in_vel, in_prs = B.use_in_prs, in_fluid = B.use_in_fluid;
  int out_prs = B.use_out_prs, out_fluid = B.use_out_fluid, copybuf = B.copy_to_buffers;
  ok = ok && R.get_bool("use_inlet_velocity", in_vel) && R.get_bool("use_inlet_pressure", in_prs) &&
       R.get_bool("use_inlet_fluid", in_fluid) && R.get_bool("use_outlet_pressure", out_prs) &&
       R.get_bool("use_outlet_fluid", out_fluid) && R.get_bool("copy_to_buffers", copybuf);
  ok = ok && R.get_double("u_inlet_x", B.u_in_x) && R.get_double("u_inlet_y", B.u_in_y) &&
       R.get_double("u_inlet_z", B.u_in_z);
  ok = ok && R.get_double("pressure_inlet", B.p_in) && R.get_double("pressure_outlet", B.p_out);
  int inlet_fluid = 0, outlet_fluid = 0;
  ok = ok && R.get_int("inlet_fluid", inlet_fluid) && R.get_int("outlet_fluid", outlet_fluid);
  ok = ok && R.get_double("inlet_period", B.inlet_period) && R.get_double("inlet_duty", B.inlet_duty) &&
       R.get_double("inlet_ramp", B.inlet_ramp) && R.get_double("inlet_split_pos", B.split_pos);
  if (ok && R.has("inlet_mode")) {
    const std::string& im = kv.at("inlet_mode");
    B.inlet_mode = im == "alternate" ? 1 : (im == "split" ? 2 : (im == "stripes" ? 3 : 0));
  }
  if (ok && R.has("inlet_split_dir")) {
    const std::string& sd = kv.at("inlet_split_dir");
    B.split_axis = sd == "y" ? 1 : (sd == "z" ? 2 : 0);
  }
  if (!ok) return fe_fail(FE_ERR_ARG, std::string("fe_cfg_read: ") + settings_path + ": " + R.err);
  // the driver's refusals (felbm_gpu_main.cu:242-254)
  if (std::strstr(dc.model, "single_phase"))
    return fe_fail(FE_ERR_ARG, "fe_cfg_read: model = single_phase: this engine is the multi-phase solver");
  if (dc.use_open_bnd && P.correct_op_mass)
    return fe_fail(FE_ERR_ARG, "fe_cfg_read: correct_op_mass must be false with open boundaries "
                               "(order-parameter mass enters and leaves)");
  // ---- params.cfg (relative to the settings file)
  {
    std::string pf = dc.param_file;
    if (!pf.empty() && pf[0] != '/') pf = dir_of(settings_path) + pf;
    KV pk;
    rc = parse_file(pf, pk, err);
    if (rc) return fe_fail(rc, "fe_cfg_read: param_file: " + err);
    Reader Q{pk, {}, {}};
    bool okp = Q.get_double("rho0", P.rho0) && Q.get_double("rho1", P.rho1) && Q.get_double("tau0", P.tau0) &&
               Q.get_double("tau1", P.tau1) && Q.get_double("interface_width", P.interface_width) &&
               Q.get_double("surface_tension", P.surface_tension) &&
               Q.get_double("mobility_coeff", P.mobility_coeff) && Q.get_double("phi", P.phi);
    if (!okp) return fe_fail(FE_ERR_ARG, "fe_cfg_read: " + pf + ": " + Q.err);
    double dens_solid = 0.0;
    Q.get_double("density_solid", dens_solid);  // felbm_local key, no role on this path
    dc.unknown_keys += (int)(pk.size() - Q.used.size());
  }
  // phase densities of the open-boundary block (felbm_gpu_main.cu:352-355)
  B.c_out_fixed = 1.0 - (double)outlet_fluid;
  B.rho_out_fixed = outlet_fluid == 0 ? P.rho0 : P.rho1;
  B.inlet_c_a = 1.0 - (double)inlet_fluid;
  B.use_in_vel = in_vel;
  B.use_in_prs = in_prs;
  B.use_in_fluid = in_fluid;
  B.use_out_prs = out_prs;
  B.use_out_fluid = out_fluid;
  B.copy_to_buffers = copybuf;
  dc.unknown_keys += (int)(kv.size() - R.used.size());
  if ((rc = fe_params_derive(&P))) return rc;
  *p = P;
  if (ob) *ob = B;
  *d = dc;
  return FE_OK;
}

int fe_cfg_switch_log(const fe_params* p, char* buf, int len) {
  using namespace fe;
  if (!p || !buf || len <= 0) return fe_fail(FE_ERR_ARG, "fe_cfg_switch_log: bad arguments");
  std::ostringstream o;
  auto on = [](int v) { return v ? "true" : "false"; };
  o << "stream_matrix_free = " << on(p->stream_matrix_free)
    << " -> push streaming fused into the collision pass over per-brick occupancy words (always)\n";
  o << "grad_matrix_free   = " << on(p->grad_matrix_free)
    << " -> gradients and Laplacians from shared-memory tiles with near-wall cases from tile occupancy (always)\n";
  o << "fused              = " << on(p->fused)
    << " -> four passes a step: moments, c stencil, mu stencil, collision (always)\n";
  o << "fuse_collision     = " << on(p->fuse_collision)
    << " -> equilibria, Guo force, collision and streaming in one pass (always)\n";
  o << "mrt_fast_transform = " << on(p->mrt_fast_transform) << " -> MRT in the storage's arithmetic type ("
    << (p->storage == FE_F64 ? "FP64" : "FP32 registers") << "), two-rate closed form when the rates depend on "
    << "the moment's parity only (always)\n";
  o << "stream_inplace     = " << on(p->stream_inplace)
    << " -> populations in two buffers, written by push streaming (always)\n";
  const std::string s = o.str();
  const int n = (int)std::min<size_t>(s.size(), (size_t)len - 1);
  std::memcpy(buf, s.data(), (size_t)n);
  buf[n] = '\0';
  return (int)s.size() + 1 > len ? fe_fail(FE_ERR_ARG, "fe_cfg_switch_log: buffer too small") : FE_OK;
}

}  // extern "C"
