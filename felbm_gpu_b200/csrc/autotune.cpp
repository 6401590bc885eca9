// Autotuner: brick shape and steps per CUDA-graph launch per size class,
// measured on the caller's geometry through the public entry points, kept in
// a process-wide table that fe_engine_create consults for FE_BRICK_AUTO.
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <tuple>
#include <vector>

#include "../../include/felbm_b200.h"
#include "fe_internal.hpp"

namespace fe {

namespace {

using Key = std::tuple<int, int, int, int, int, int>;

struct Choice {
  int brick, graph_steps;
};

std::mutex g_tune_mu;
std::map<Key, Choice> g_tune;

Key make_key(int dim2, int storage, int mrt, int hbb, double porosity, int64_t sites) {
  const int pb = (int)std::floor(porosity * 20.0);
  const int sb = sites > 0 ? (int)std::floor(std::log2((double)sites)) : 0;
  return Key(dim2 ? 1 : 0, storage, mrt ? 1 : 0, hbb ? 1 : 0, pb, sb);
}

}  // namespace

bool tune_lookup(int dim2, int storage, int mrt, int hbb, double porosity, int64_t sites, int* brick,
                 int* graph_steps) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  auto it = g_tune.find(make_key(dim2, storage, mrt, hbb, porosity, sites));
  if (it == g_tune.end()) return false;
  *brick = it->second.brick;
  *graph_steps = it->second.graph_steps;
  return true;
}

void tune_store(int dim2, int storage, int mrt, int hbb, double porosity, int64_t sites, int brick, int graph_steps) {
  std::lock_guard<std::mutex> lk(g_tune_mu);
  g_tune[make_key(dim2, storage, mrt, hbb, porosity, sites)] = Choice{brick, graph_steps};
}

}  // namespace fe

namespace {

// MLUPS of `steps` timed steps (after 3 warm-up steps) of one engine over the
// geometry with a uniform order parameter 1/2 at rest; -1 when the layout is
// refused.
int time_one(const fe_params& p, int nx, int ny, int nz, const uint8_t* solid, int device, int steps,
             double* mlups) {
  *mlups = -1.0;
  fe_engine* e = nullptr;
  int rc = fe_engine_create(&p, nx, ny, nz, solid, device, &e);
  if (rc) return rc;
  int64_t n = 0, vn = 0;
  if (!(rc = fe_engine_size(e, &n, &vn))) {
    std::vector<double> c(n), pr(n, 1.0), h(vn), g(vn);
    const double half = 0.5;
    if (!(rc = fe_init_order_parameter(solid, nx, ny, nz, 0, &half, 4.0, c.data())) &&
        !(rc = fe_init_equilibrium(n, c.data(), pr.data(), nullptr, nullptr, nullptr, p.rho0, p.rho1, h.data(),
                                   g.data())) &&
        !(rc = fe_upload_state(e, h.data(), g.data(), vn)) && !(rc = fe_run(e, 3))) {
      float ms = 0.0f;
      if (!(rc = fe_time_run(e, steps, &ms)) && ms > 0.0f) *mlups = (double)n * steps / (ms * 1e3);
    }
  }
  fe_engine_destroy(e);
  return rc;
}

}  // namespace

extern "C" {

int fe_autotune(const fe_params* p, int nx, int ny, int nz, const uint8_t* solid, int device, int steps,
                fe_tune_report* out) {
  if (!p || !solid || !out || nx < 1 || ny < 1 || nz < 1 || steps < 1)
    return fe_fail(FE_ERR_ARG, "fe_autotune: bad arguments");
  *out = fe_tune_report{};
  std::vector<int> bricks;
  if (nz == 1) bricks = {FE_BRICK_16x16x1};
  else if (p->storage == FE_F64 || p->storage == FE_F32) bricks = {FE_BRICK_8x8x8, FE_BRICK_8x8x4, FE_BRICK_16x8x8};
  else bricks = {FE_BRICK_8x8x8, FE_BRICK_16x8x8};
  int best_brick = 0, best_graph = 2, rc;
  double best = -1.0;
  auto add = [&](int brick, int gs, double v) {
    if (out->ncand < 8) {
      out->cand_brick[out->ncand] = brick;
      out->cand_graph_steps[out->ncand] = gs;
      out->cand_mlups[out->ncand] = v;
      ++out->ncand;
    }
  };
  for (int b : bricks) {
    fe_params q = *p;
    q.brick = b;
    q.graph_steps = 2;
    double v = 0.0;
    if ((rc = time_one(q, nx, ny, nz, solid, device, steps, &v))) return rc;
    add(b, 2, v);
    if (v > best) {
      best = v;
      best_brick = b;
    }
  }
  for (int gs : {8, 32}) {
    fe_params q = *p;
    q.brick = best_brick;
    q.graph_steps = gs;
    double v = 0.0;
    if ((rc = time_one(q, nx, ny, nz, solid, device, steps, &v))) return rc;
    add(best_brick, gs, v);
    if (v > best) {
      best = v;
      best_graph = gs;
    }
  }
  int64_t fluid = 0;
  const int64_t nodes = (int64_t)nx * ny * nz;
  for (int64_t q = 0; q < nodes; ++q) fluid += solid[q] == 0;
  fe::tune_store(nz == 1, p->storage, p->use_mrt != 0, p->use_halfway_bb != 0, (double)fluid / (double)nodes, fluid,
                 best_brick, best_graph);
  out->brick = best_brick;
  out->graph_steps = best_graph;
  return FE_OK;
}

int fe_tune_save(const char* path) {
  if (!path) return fe_fail(FE_ERR_ARG, "fe_tune_save: null path");
  FILE* f = std::fopen(path, "w");
  if (!f) return fe_fail(FE_ERR_IO, std::string("cannot open ") + path);
  std::fprintf(f, "# felbm_b200 autotune table: dim2 storage mrt hbb porosity_bin20 log2_sites brick graph_steps\n");
  {
    std::lock_guard<std::mutex> lk(fe::g_tune_mu);
    for (const auto& kv : fe::g_tune) {
      const auto& k = kv.first;
      std::fprintf(f, "%d %d %d %d %d %d %d %d\n", std::get<0>(k), std::get<1>(k), std::get<2>(k), std::get<3>(k),
                   std::get<4>(k), std::get<5>(k), kv.second.brick, kv.second.graph_steps);
    }
  }
  const int bad = std::ferror(f);
  std::fclose(f);
  return bad ? fe_fail(FE_ERR_IO, std::string("write failed: ") + path) : FE_OK;
}

int fe_tune_load(const char* path) {
  if (!path) return fe_fail(FE_ERR_ARG, "fe_tune_load: null path");
  FILE* f = std::fopen(path, "r");
  if (!f) return fe_fail(FE_ERR_IO, std::string("cannot open ") + path);
  char line[256];
  int bad = 0;
  std::vector<std::pair<fe::Key, fe::Choice>> rows;
  while (std::fgets(line, sizeof line, f)) {
    if (line[0] == '#' || line[0] == '\n') continue;
    int v[8];
    if (std::sscanf(line, "%d %d %d %d %d %d %d %d", &v[0], &v[1], &v[2], &v[3], &v[4], &v[5], &v[6], &v[7]) != 8 ||
        v[6] < FE_BRICK_8x8x8 || v[6] > FE_BRICK_16x8x8 || v[7] < 1) {
      bad = 1;
      break;
    }
    rows.push_back({fe::Key(v[0], v[1], v[2], v[3], v[4], v[5]), fe::Choice{v[6], v[7]}});
  }
  std::fclose(f);
  if (bad) return fe_fail(FE_ERR_IO, std::string(path) + ": not an autotune table");
  std::lock_guard<std::mutex> lk(fe::g_tune_mu);
  for (const auto& r : rows) fe::g_tune[r.first] = r.second;
  return FE_OK;
}

int fe_tune_clear(void) {
  std::lock_guard<std::mutex> lk(fe::g_tune_mu);
  fe::g_tune.clear();
  return FE_OK;
}

}  // extern "C"
