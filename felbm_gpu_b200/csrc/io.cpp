// On-disk formats of the reference driver (felbm_gpu_main.cu:86-189), over
// the public C-ABI: field dumps <output_name>_<iter>.h5, geometry.h5, the
// checkpoint, and particles_<step>.h5. Same dataset names, shapes and types;
// field files optionally gzip-compressed as the reference's output_deflate
// (one chunk per dataset); the rest contiguous.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/felbm_b200.h"
#include "fe_internal.hpp"
#include "h5.hpp"

using fe::h5::Dataset;

extern "C" {

int fe_write_fields_h5(fe_engine* e, const char* path, int float32, int deflate) {
  if (!e || !path || deflate < 0 || deflate > 9) return fe_fail(FE_ERR_ARG, "fe_write_fields_h5: bad arguments");
  int64_t n = 0;
  int rc = fe_engine_size(e, &n, nullptr);
  if (rc) return rc;
  std::vector<double> v(6 * (size_t)n);
  fe_fields f{v.data(), v.data() + n, v.data() + 2 * n, v.data() + 3 * n, v.data() + 4 * n, v.data() + 5 * n,
              nullptr};
  if ((rc = fe_download_fields(e, &f))) return rc;
  const char* names[6] = {"density", "concentration", "u_x", "u_y", "u_z", "pressure"};
  std::vector<float> vf;
  if (float32) vf.assign(v.begin(), v.end());
  std::vector<Dataset> sets;
  for (int q = 0; q < 6; ++q) {
    Dataset d;
    d.name = names[q];
    d.dims = {(uint64_t)n};
    d.type = float32 ? fe::h5::F32 : fe::h5::F64;
    d.data = float32 ? (const void*)(vf.data() + q * n) : (const void*)(v.data() + q * n);
    d.deflate = deflate;
    sets.push_back(d);
  }
  return fe::h5::write(path, sets);
}

int fe_write_geometry_h5(const char* path, const uint8_t* solid, int nx, int ny, int nz) {
  if (!path || !solid || nx < 1 || ny < 1 || nz < 1) return fe_fail(FE_ERR_ARG, "fe_write_geometry_h5: bad arguments");
  std::vector<int32_t> coords;
  int32_t mx = 0, my = 0, mz = 0;
  for (int64_t node = 0; node < (int64_t)nx * ny * nz; ++node) {
    if (solid[node]) continue;
    const int32_t x = (int32_t)(node % nx), y = (int32_t)((node / nx) % ny), z = (int32_t)(node / ((int64_t)nx * ny));
    coords.insert(coords.end(), {x, y, z});
    mx = std::max(mx, x);
    my = std::max(my, y);
    mz = std::max(mz, z);
  }
  const int32_t size[3] = {mx + 1, my + 1, mz + 1};
  Dataset c{"coords", fe::h5::I32, {(uint64_t)coords.size() / 3, 3}, coords.data()};
  Dataset s{"size", fe::h5::I32, {3}, size};
  return fe::h5::write(path, {c, s});
}

int fe_checkpoint_write(fe_engine* e, const char* path, uint32_t step) {
  if (!e || !path) return fe_fail(FE_ERR_ARG, "fe_checkpoint_write: bad arguments");
  int64_t n = 0, vn = 0;
  int rc = fe_engine_size(e, &n, &vn);
  if (rc) return rc;
  if (vn > INT32_MAX) return fe_fail(FE_ERR_ARG, "state too large for the checkpoint's int Vn");
  std::vector<double> h(vn), g(vn);
  double m0 = 0.0;
  // a queued correction goes into the engine's own state first, so the run
  // that continues holds exactly the state a restart reads back
  if ((rc = fe_settle_mass_correction(e))) return rc;
  if ((rc = fe_download_state(e, h.data(), g.data(), vn)) || (rc = fe_get_target_mass(e, &m0))) return rc;
  const int32_t vni = (int32_t)vn;
  const uint32_t st = step;
  return fe::h5::write(path, {{"h", fe::h5::F64, {(uint64_t)vn}, h.data()},
                              {"g", fe::h5::F64, {(uint64_t)vn}, g.data()},
                              {"step", fe::h5::U32, {1}, &st},
                              {"target_mass", fe::h5::F64, {1}, &m0},
                              {"Vn", fe::h5::I32, {1}, &vni}});
}

int fe_checkpoint_read(fe_engine* e, const char* path, uint32_t* step) {
  if (!e || !path || !step) return fe_fail(FE_ERR_ARG, "fe_checkpoint_read: bad arguments");
  int64_t n = 0, vn = 0;
  int rc = fe_engine_size(e, &n, &vn);
  if (rc) return rc;
  std::vector<fe::h5::Read> sets;
  if ((rc = fe::h5::read(path, sets))) return rc;
  auto find = [&](const char* nm) -> const fe::h5::Read* {
    for (const fe::h5::Read& r : sets)
      if (r.name == nm) return &r;
    return nullptr;
  };
  const fe::h5::Read *rh = find("h"), *rg = find("g"), *rs = find("step"), *rm = find("target_mass"),
                     *rv = find("Vn");
  if (!rh || !rg || !rs || !rm || !rv) return fe_fail(FE_ERR_IO, std::string(path) + ": not a checkpoint");
  int32_t vfile = 0;
  std::memcpy(&vfile, rv->bytes.data(), 4);
  // reference read_checkpoint (felbm_gpu_main.cu:171-189): refuse a state of
  // another geometry
  if (vfile != vn || rh->bytes.size() != (size_t)vn * 8 || rg->bytes.size() != (size_t)vn * 8)
    return fe_fail(FE_ERR_ARG, "checkpoint Vn does not match the engine (geometry mismatch)");
  if ((rc = fe_upload_state(e, reinterpret_cast<const double*>(rh->bytes.data()),
                            reinterpret_cast<const double*>(rg->bytes.data()), vn)))
    return rc;
  double m0 = 0.0;
  std::memcpy(&m0, rm->bytes.data(), 8);
  std::memcpy(step, rs->bytes.data(), 4);
  // the original M0 is kept (README "checkpoint": recomputing it would lock
  // the drift to the wrong target)
  return fe_set_target_mass(e, m0);
}

int fe_write_particles_h5(const char* path, int64_t n, const double* pos, const double* vel, const int64_t* id,
                          const double* dm, const int32_t* plane_id, const double* rho_hat, const double* log_rho) {
  if (!path || n < 1 || !pos) return fe_fail(FE_ERR_ARG, "fe_write_particles_h5: bad arguments");
  std::vector<double> p(3 * n), v;
  for (int64_t q = 0; q < n; ++q)
    for (int a = 0; a < 3; ++a) p[3 * q + a] = pos[a * n + q];
  std::vector<Dataset> sets = {{"position", fe::h5::F64, {(uint64_t)n, 3}, p.data()}};
  if (vel) {
    v.resize(3 * n);
    for (int64_t q = 0; q < n; ++q)
      for (int a = 0; a < 3; ++a) v[3 * q + a] = vel[a * n + q];
    sets.push_back({"velocity", fe::h5::F64, {(uint64_t)n, 3}, v.data()});
  }
  std::vector<int32_t> ids(n);
  for (int64_t q = 0; q < n; ++q) ids[q] = (int32_t)(id ? id[q] : q);
  sets.push_back({"id", fe::h5::I32, {(uint64_t)n}, ids.data()});
  if (dm) sets.push_back({"Dm", fe::h5::F64, {(uint64_t)n}, dm});
  if (plane_id) sets.push_back({"plane_id", fe::h5::I32, {(uint64_t)n}, plane_id});
  std::vector<double> rh;
  if (rho_hat) {
    rh.resize(3 * n);
    for (int64_t q = 0; q < n; ++q)
      for (int a = 0; a < 3; ++a) rh[3 * q + a] = rho_hat[a * n + q];
    sets.push_back({"rho_hat", fe::h5::F64, {(uint64_t)n, 3}, rh.data()});
  }
  if (log_rho) sets.push_back({"log_rho", fe::h5::F64, {(uint64_t)n}, log_rho});
  return fe::h5::write(path, sets);
}

// Text time series of the reference driver (felbm_gpu_main.cu:600-698): one
// line per call, the header first when `header` (the file is then truncated).
int fe_write_series(const char* path, int header, uint32_t iter, const double stats[6], int64_t n) {
  if (!path || !stats || n < 1) return fe_fail(FE_ERR_ARG, "fe_write_series: bad arguments");
  FILE* f = std::fopen(path, header ? "w" : "a");
  if (!f) return fe_fail(FE_ERR_IO, std::string("cannot open ") + path);
  if (header) std::fprintf(f, "# iter   max_speed   mean_ux   mean_uy   mean_uz   mean_v2   total_order_parameter\n");
  const double inv = 1.0 / (double)n;
  std::fprintf(f, "%u  %.10g  %.10g  %.10g  %.10g  %.10g  %.10g\n", iter, std::sqrt(stats[5]), stats[0] * inv,
               stats[1] * inv, stats[2] * inv, stats[3] * inv, stats[4]);
  const int bad = std::ferror(f);
  std::fclose(f);
  return bad ? fe_fail(FE_ERR_IO, std::string("write failed: ") + path) : FE_OK;
}

int fe_write_stretching(const char* path, int header, const double* rows, int64_t nrows) {
  if (!path || nrows < 0 || (nrows > 0 && !rows)) return fe_fail(FE_ERR_ARG, "fe_write_stretching: bad arguments");
  FILE* f = std::fopen(path, header ? "w" : "a");
  if (!f) return fe_fail(FE_ERR_IO, std::string("cannot open ") + path);
  if (header)
    std::fprintf(f,
                 "# Stretching of the tracers' material line elements, one row per tracer step.\n"
                 "# lambda: mean of rho_hat . (grad u) rho_hat over the active tracers and substeps;\n"
                 "# mean_log_rho, var_log_rho: over all tracers; n_active: tracers with no rejected\n"
                 "# substep; lambda_w / lambda_nw: the same mean split by phase (c < 0.5 wetting),\n"
                 "# nan when the phase has no sample; n_w, n_nw: phase samples / substeps.\n"
                 "# step   lambda   mean_log_rho   var_log_rho   n_active   lambda_w   lambda_nw   n_w   n_nw\n");
  for (int64_t r = 0; r < nrows; ++r) {
    const double* v = rows + 9 * r;
    std::fprintf(f, "%lld  %.10g  %.10g  %.10g  %lld  %.10g  %.10g  %.10g  %.10g\n", (long long)v[0], v[1], v[2],
                 v[3], (long long)v[4], v[5], v[6], v[7], v[8]);
  }
  const int bad = std::ferror(f);
  std::fclose(f);
  return bad ? fe_fail(FE_ERR_IO, std::string("write failed: ") + path) : FE_OK;
}

// Generic read of one dataset of a file written here (tests, tools): the
// element type (FE_H5_*), the dimensions and the raw little-endian bytes.
int fe_h5_write_dataset(const char* path, const char* name, int type, int rank, const int64_t* dims,
                        const void* data, int deflate) {
  if (!path || !name || !dims || !data || type < 0 || type > 3 || rank < 1 || rank > 2)
    return fe_fail(FE_ERR_ARG, "fe_h5_write_dataset: bad arguments");
  Dataset d;
  d.name = name;
  d.type = (fe::h5::Type)type;
  for (int a = 0; a < rank; ++a) {
    if (dims[a] < 0) return fe_fail(FE_ERR_ARG, "fe_h5_write_dataset: negative extent");
    d.dims.push_back((uint64_t)dims[a]);
  }
  d.data = data;
  d.deflate = deflate;
  return fe::h5::write(path, {d});
}

int fe_h5_read_dataset(const char* path, const char* name, int* type, int64_t* dims, int* rank, void* data,
                       int64_t capacity_bytes) {
  if (!path || !name || !type || !dims || !rank) return fe_fail(FE_ERR_ARG, "fe_h5_read_dataset: bad arguments");
  std::vector<fe::h5::Read> sets;
  int rc = fe::h5::read(path, sets);
  if (rc) return rc;
  for (const fe::h5::Read& r : sets) {
    if (r.name != name) continue;
    *type = (int)r.type;
    *rank = (int)r.dims.size();
    for (size_t a = 0; a < r.dims.size(); ++a) dims[a] = (int64_t)r.dims[a];
    if (data) {
      if ((int64_t)r.bytes.size() > capacity_bytes) return fe_fail(FE_ERR_ARG, "fe_h5_read_dataset: buffer too small");
      std::memcpy(data, r.bytes.data(), r.bytes.size());
    }
    return FE_OK;
  }
  return fe_fail(FE_ERR_IO, std::string(path) + ": no dataset " + name);
}

}  // extern "C"
