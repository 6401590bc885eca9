// Geometry and initial-condition front end (host C++).
//
// The reference builds its geometry and initial state with felbm_local
// (DomainInitializer_*, InitializerMultiPhase_*; src/felbm_gpu_main.cu:256-311),
// which is not part of the reference snapshot. These are this project's own
// seeded generators for the workloads the engine is measured on:
//   - a Gaussian random field thresholded at a porosity quantile, largest
//     percolating cluster kept (3-D porous media);
//   - random sequential addition of non-overlapping discs (2-D packs,
//     the idea of the reference's scripts/geometry/periodic_disk_mesh.py:48)
//     and spheres (the compare_cpu_gpu "spheres_repulsive" case);
//   - open inlet/outlet padding with empty and buffer layers.
// Masks are uint8 over nx*ny*nz nodes, node index x + nx*(y + ny*z), 1 = solid.
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "../../include/felbm_b200.h"
#include "d3q19.hpp"
#include "fe_internal.hpp"

namespace fe {
namespace {

// splitmix64: seeded, platform-independent random stream.
struct Rng {
  uint64_t s;
  explicit Rng(uint64_t seed) : s(seed) {}
  uint64_t next() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  }
  double uniform() { return (double)(next() >> 11) * (1.0 / 9007199254740992.0); }
};

// Standard normal from a counter-based hash of (seed, index), so the field is
// identical however the loop is split across threads.
inline double normal_at(uint64_t seed, uint64_t idx) {
  Rng r(seed ^ (idx * 0xD1B54A32D192ED03ull));
  double u1 = r.uniform(), u2 = r.uniform();
  if (u1 < 1e-300) u1 = 1e-300;
  return std::sqrt(-2.0 * std::log(u1)) * std::cos(6.283185307179586 * u2);
}

inline int64_t wrapi(int64_t a, int64_t n) { return ((a % n) + n) % n; }

// One periodic 1-D Gaussian convolution pass along `axis`.
void convolve_axis(std::vector<double>& f, int nx, int ny, int nz, int axis, const std::vector<double>& ker) {
  const int R = (int)ker.size() / 2;
  const int64_t N[3] = {nx, ny, nz};
  const int64_t stride[3] = {1, nx, (int64_t)nx * ny};
  const int64_t len = N[axis];
  if (len == 1) return;
  const int64_t total = (int64_t)nx * ny * nz;
  const int64_t nlines = total / len;
  std::vector<double> out(total);
#pragma omp parallel
  {
    std::vector<double> line(len);
#pragma omp for schedule(static)
    for (int64_t l = 0; l < nlines; ++l) {
      // base node of line l: enumerate nodes with coordinate[axis] == 0
      int64_t base;
      if (axis == 0) base = l * nx;
      else if (axis == 1) base = (l / nx) * (int64_t)nx * ny + (l % nx);
      else base = l;
      for (int64_t a = 0; a < len; ++a) line[a] = f[base + a * stride[axis]];
      for (int64_t a = 0; a < len; ++a) {
        double s = 0.0;
        for (int r = -R; r <= R; ++r) s += ker[r + R] * line[wrapi(a + r, len)];
        out[base + a * stride[axis]] = s;
      }
    }
  }
  f.swap(out);
}

// Union-find over fluid nodes with the 18 D3Q19 links (periodic along the
// axes flagged in `wrap`). Returns per-node root (-1 for solid).
struct DSU {
  std::vector<int64_t> p;
  explicit DSU(int64_t n) : p(n) { std::iota(p.begin(), p.end(), 0); }
  int64_t find(int64_t a) {
    while (p[a] != a) { p[a] = p[p[a]]; a = p[a]; }
    return a;
  }
  void unite(int64_t a, int64_t b) {
    a = find(a); b = find(b);
    if (a != b) { if (a < b) std::swap(a, b); p[a] = b; }
  }
};

}  // namespace

// Keep one connected fluid cluster; everything else becomes solid. With
// flow_axis >= 0 the kept cluster must touch both faces normal to that axis
// (links across that axis do not wrap when open_flow is set); the largest such
// cluster is kept. With flow_axis < 0 the largest cluster is kept.
// Returns the number of fluid nodes left (0 if no cluster qualifies).
int64_t keep_largest_cluster(uint8_t* solid, int nx, int ny, int nz, int flow_axis, bool open_flow) {
  const int64_t total = (int64_t)nx * ny * nz;
  DSU d(total);
  const int N[3] = {nx, ny, nz};
  for (int64_t node = 0; node < total; ++node) {
    if (solid[node]) continue;
    const int x = (int)(node % nx), y = (int)((node / nx) % ny), z = (int)(node / ((int64_t)nx * ny));
    const int c[3] = {x, y, z};
    for (int k = 1; k < Q; k += 2) {  // one of each opposite pair
      const int e[3] = {lat_cx(k), lat_cy(k), lat_cz(k)};
      int q[3];
      bool ok = true;
      for (int a = 0; a < 3; ++a) {
        q[a] = c[a] + e[a];
        if (q[a] < 0 || q[a] >= N[a]) {
          if (open_flow && a == flow_axis) { ok = false; break; }
          q[a] = (q[a] + N[a]) % N[a];
        }
      }
      if (!ok) continue;
      const int64_t nb = q[0] + (int64_t)nx * (q[1] + (int64_t)ny * q[2]);
      if (!solid[nb]) d.unite(node, nb);
    }
  }
  std::vector<int64_t> size(total, 0);
  std::vector<uint8_t> lo(flow_axis >= 0 ? total : 0, 0), hi(flow_axis >= 0 ? total : 0, 0);
  for (int64_t node = 0; node < total; ++node) {
    if (solid[node]) continue;
    const int64_t r = d.find(node);
    ++size[r];
    if (flow_axis >= 0) {
      const int x = (int)(node % nx), y = (int)((node / nx) % ny), z = (int)(node / ((int64_t)nx * ny));
      const int c = flow_axis == 0 ? x : (flow_axis == 1 ? y : z);
      if (c == 0) lo[r] = 1;
      if (c == N[flow_axis] - 1) hi[r] = 1;
    }
  }
  int64_t best = -1, best_size = 0;
  for (int64_t r = 0; r < total; ++r)
    if (size[r] > best_size && (flow_axis < 0 || (lo[r] && hi[r]))) { best = r; best_size = size[r]; }
  if (best < 0) {
    std::fill(solid, solid + total, 1);
    return 0;
  }
  for (int64_t node = 0; node < total; ++node)
    if (!solid[node] && d.find(node) != best) solid[node] = 1;
  return best_size;
}

}  // namespace fe

using namespace fe;

extern "C" {

// Gaussian random field: white noise convolved with a Gaussian kernel whose
// width sigma = corr_len / sqrt(2) gives a field correlation exp(-r^2 /
// (2 corr_len^2)); fluid where the field is below its `porosity` quantile;
// then the largest cluster percolating along flow_axis is kept (flow_axis < 0:
// largest cluster). open_flow: the flow axis does not wrap for connectivity.
int fe_geom_grf(int nx, int ny, int nz, double corr_len, double porosity, uint64_t seed,
                int flow_axis, int open_flow, uint8_t* solid, double* porosity_out) {
  if (nx < 1 || ny < 1 || nz < 1 || !solid || porosity <= 0.0 || porosity > 1.0 || corr_len <= 0.0)
    return fe_fail(FE_ERR_ARG, "fe_geom_grf: bad arguments");
  const int64_t total = (int64_t)nx * ny * nz;
  std::vector<double> f(total);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < total; ++i) f[i] = normal_at(seed, (uint64_t)i);
  const double sigma = corr_len / std::sqrt(2.0);
  const int R = std::max(1, (int)std::ceil(3.0 * sigma));
  std::vector<double> ker(2 * R + 1);
  double ks = 0.0;
  for (int r = -R; r <= R; ++r) ks += (ker[r + R] = std::exp(-0.5 * r * r / (sigma * sigma)));
  for (double& v : ker) v /= ks;
  for (int a = 0; a < 3; ++a) convolve_axis(f, nx, ny, nz, a, ker);
  std::vector<double> sorted(f);
  const int64_t kq = std::min<int64_t>(total - 1, (int64_t)std::floor(porosity * (double)total));
  std::nth_element(sorted.begin(), sorted.begin() + kq, sorted.end());
  const double thr = sorted[kq];
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < total; ++i) solid[i] = (porosity >= 1.0 || f[i] < thr) ? 0 : 1;
  const int64_t nf = keep_largest_cluster(solid, nx, ny, nz, flow_axis, open_flow != 0);
  if (porosity_out) *porosity_out = (double)nf / (double)total;
  return nf > 0 ? FE_OK : fe_fail(FE_ERR_ARG, "fe_geom_grf: no percolating cluster");
}

// Random sequential addition of non-overlapping discs (axis z, extruded) with
// radii U[rmin, rmax] and periodic distance >= r1 + r2 + gap, until the solid
// fraction reaches 1 - porosity or max_tries placements fail in a row. The
// largest fluid cluster is kept when keep_largest.
int fe_geom_cylinders(int nx, int ny, int nz, double rmin, double rmax, double porosity, double gap,
                      uint64_t seed, int keep_largest, uint8_t* solid, double* porosity_out) {
  if (nx < 1 || ny < 1 || nz < 1 || !solid || rmin <= 0 || rmax < rmin)
    return fe_fail(FE_ERR_ARG, "fe_geom_cylinders: bad arguments");
  Rng rng(seed);
  struct Disc { double x, y, r; };
  std::vector<Disc> discs;
  const int64_t plane = (int64_t)nx * ny;
  std::vector<uint8_t> m(plane, 0);
  int64_t nsolid = 0;
  const int64_t target = (int64_t)std::ceil((1.0 - porosity) * (double)plane);
  int fails = 0;
  auto pdist2 = [&](double ax, double ay, double bx, double by) {
    double dx = std::fabs(ax - bx), dy = std::fabs(ay - by);
    dx = std::min(dx, nx - dx); dy = std::min(dy, ny - dy);
    return dx * dx + dy * dy;
  };
  while (nsolid < target && fails < 20000) {
    const double x = rng.uniform() * nx, y = rng.uniform() * ny;
    const double r = rmin + (rmax - rmin) * rng.uniform();
    bool ok = true;
    for (const Disc& d : discs) {
      const double lim = d.r + r + gap;
      if (pdist2(x, y, d.x, d.y) < lim * lim) { ok = false; break; }
    }
    if (!ok) { ++fails; continue; }
    fails = 0;
    discs.push_back({x, y, r});
    const int R = (int)std::ceil(r) + 1;
    for (int dy = -R; dy <= R; ++dy)
      for (int dx = -R; dx <= R; ++dx) {
        const int64_t px = wrapi((int64_t)std::floor(x) + dx, nx), py = wrapi((int64_t)std::floor(y) + dy, ny);
        if (pdist2((double)px + 0.5, (double)py + 0.5, x, y) <= r * r && !m[px + nx * py]) {
          m[px + nx * py] = 1;
          ++nsolid;
        }
      }
  }
  for (int z = 0; z < nz; ++z) std::memcpy(solid + z * plane, m.data(), plane);
  int64_t nf = (int64_t)nx * ny * nz - nsolid * nz;
  if (keep_largest) nf = keep_largest_cluster(solid, nx, ny, nz, -1, false);
  if (porosity_out) *porosity_out = (double)nf / ((double)nx * ny * nz);
  return nf > 0 ? FE_OK : fe_fail(FE_ERR_ARG, "fe_geom_cylinders: no fluid left");
}

// Random sequential addition of up to max_number spheres of a fixed radius
// with centre distance >= 2 radius + distance (periodic).
int fe_geom_spheres(int nx, int ny, int nz, double radius, int max_number, double distance,
                    uint64_t seed, uint8_t* solid) {
  if (nx < 1 || ny < 1 || nz < 1 || !solid || radius <= 0 || max_number < 0)
    return fe_fail(FE_ERR_ARG, "fe_geom_spheres: bad arguments");
  Rng rng(seed);
  struct S { double x, y, z; };
  std::vector<S> sp;
  auto pd = [](double a, double b, int n) { double d = std::fabs(a - b); return std::min(d, n - d); };
  int tries = 0;
  while ((int)sp.size() < max_number && tries < 100000) {
    ++tries;
    const S s{rng.uniform() * nx, rng.uniform() * ny, rng.uniform() * nz};
    bool ok = true;
    for (const S& o : sp) {
      const double dx = pd(s.x, o.x, nx), dy = pd(s.y, o.y, ny), dz = pd(s.z, o.z, nz);
      const double lim = 2 * radius + distance;
      if (dx * dx + dy * dy + dz * dz < lim * lim) { ok = false; break; }
    }
    if (ok) sp.push_back(s);
  }
  std::memset(solid, 0, (size_t)nx * ny * nz);
  for (const S& s : sp)
    for (int64_t z = 0; z < nz; ++z)
      for (int64_t y = 0; y < ny; ++y)
        for (int64_t x = 0; x < nx; ++x) {
          const double dx = pd(x + 0.5, s.x, nx), dy = pd(y + 0.5, s.y, ny), dz = pd(z + 0.5, s.z, nz);
          if (dx * dx + dy * dy + dz * dz <= radius * radius) solid[x + nx * (y + ny * z)] = 1;
        }
  return FE_OK;
}

// Open inlet/outlet padding along flow_axis. The medium (mx,my,mz) is placed
// after buffer_layers + empty_layers layers and followed by empty_layers +
// buffer_layers layers. Empty layers are fluid. Buffer layers repeat the
// solid pattern of the adjacent face layer (extrusion). The padded size is
// written to dims_out; out_solid must hold the padded node count (query with
// out_solid = NULL first).
int fe_geom_pad_open(const uint8_t* medium, int mx, int my, int mz, int flow_axis, int empty_layers,
                     int buffer_layers, int* dims_out, uint8_t* out_solid) {
  if (!medium || flow_axis < 0 || flow_axis > 2 || empty_layers < 0 || buffer_layers < 0 || !dims_out)
    return fe_fail(FE_ERR_ARG, "fe_geom_pad_open: bad arguments");
  int d[3] = {mx, my, mz};
  const int pad = empty_layers + buffer_layers;
  d[flow_axis] += 2 * pad;
  dims_out[0] = d[0]; dims_out[1] = d[1]; dims_out[2] = d[2];
  if (!out_solid) return FE_OK;
  const int M[3] = {mx, my, mz};
  for (int64_t z = 0; z < d[2]; ++z)
    for (int64_t y = 0; y < d[1]; ++y)
      for (int64_t x = 0; x < d[0]; ++x) {
        int64_t c[3] = {x, y, z};
        const int64_t a = c[flow_axis];
        uint8_t s;
        if (a >= pad && a < pad + M[flow_axis]) {
          c[flow_axis] = a - pad;
          s = medium[c[0] + (int64_t)mx * (c[1] + (int64_t)my * c[2])];
        } else if (a >= buffer_layers && a < d[flow_axis] - buffer_layers) {
          s = 0;  // empty layer
        } else {
          s = 2;  // buffer, filled below
        }
        out_solid[x + (int64_t)d[0] * (y + (int64_t)d[1] * z)] = s;
      }
  // extrusion: buffer nodes copy the nearest non-buffer layer
  for (int64_t z = 0; z < d[2]; ++z)
    for (int64_t y = 0; y < d[1]; ++y)
      for (int64_t x = 0; x < d[0]; ++x) {
        const int64_t node = x + (int64_t)d[0] * (y + (int64_t)d[1] * z);
        if (out_solid[node] != 2) continue;
        int64_t c[3] = {x, y, z};
        c[flow_axis] = c[flow_axis] < buffer_layers ? buffer_layers : d[flow_axis] - buffer_layers - 1;
        out_solid[node] = out_solid[c[0] + (int64_t)d[0] * (c[1] + (int64_t)d[1] * c[2])];
      }
  return FE_OK;
}

// Inlet/outlet/buffer site lists of a padded open domain (site indices in the
// reference order). Inlet = fluid sites of the first non-buffer layer along
// flow_axis, outlet = of the last; buffer sites reference the inlet/outlet
// site with the same transverse coordinates. Arrays may be NULL to query the
// counts; inlet_coord (may be NULL) receives the coordinate along split_axis.
int fe_geom_open_lists(const uint8_t* solid, int nx, int ny, int nz, int flow_axis, int buffer_layers,
                       int split_axis, int32_t* n_counts, int32_t* inlet, int32_t* outlet,
                       int32_t* buf_verts, int32_t* buf_refs, double* inlet_coord) {
  if (!solid || flow_axis < 0 || flow_axis > 2 || !n_counts)
    return fe_fail(FE_ERR_ARG, "fe_geom_open_lists: bad arguments");
  const int64_t total = (int64_t)nx * ny * nz;
  std::vector<int32_t> site(total, -1);
  int32_t n = 0;
  for (int64_t node = 0; node < total; ++node)
    if (!solid[node]) site[node] = n++;
  const int N[3] = {nx, ny, nz};
  const int lo = buffer_layers, hi = N[flow_axis] - buffer_layers - 1;
  int32_t ni = 0, no = 0, nb = 0;
  for (int64_t node = 0; node < total; ++node) {
    if (solid[node]) continue;
    int c[3] = {(int)(node % nx), (int)((node / nx) % ny), (int)(node / ((int64_t)nx * ny))};
    const int a = c[flow_axis];
    if (a == lo) {
      if (inlet) inlet[ni] = site[node];
      if (inlet_coord) inlet_coord[ni] = (double)c[split_axis];
      ++ni;
    } else if (a == hi) {
      if (outlet) outlet[no] = site[node];
      ++no;
    } else if (a < lo || a > hi) {
      int r[3] = {c[0], c[1], c[2]};
      r[flow_axis] = a < lo ? lo : hi;
      const int64_t rn = r[0] + (int64_t)nx * (r[1] + (int64_t)ny * r[2]);
      if (site[rn] < 0) return fe_fail(FE_ERR_ARG, "fe_geom_open_lists: buffer vertex reference does not exist");
      if (buf_verts) { buf_verts[nb] = site[node]; buf_refs[nb] = site[rn]; }
      ++nb;
    }
  }
  n_counts[0] = ni; n_counts[1] = no; n_counts[2] = nb;
  return FE_OK;
}

// Number of sites (fluid nodes) and, optionally, their node indices in the
// reference order.
int fe_geom_sites(const uint8_t* solid, int nx, int ny, int nz, int64_t* n, int64_t* nodes) {
  if (!solid || !n) return fe_fail(FE_ERR_ARG, "fe_geom_sites: bad arguments");
  const int64_t total = (int64_t)nx * ny * nz;
  int64_t c = 0;
  for (int64_t node = 0; node < total; ++node)
    if (!solid[node]) { if (nodes) nodes[c] = node; ++c; }
  *n = c;
  return FE_OK;
}

// Order-parameter field of the initial condition per site (reference order).
// kind 0 uniform (c = a0); 1 slab: phase c = 1 inside the periodic slab of
// `thickness` that starts at (a0,a1,a2) along axis (int)a3, tanh profile of
// width W; 2 droplet: c = 1 inside the periodic sphere centre (a0,a1,a2)
// radius a3. Profiles are c = (1 + tanh(2 d / W)) / 2 with d the signed
// distance to the nearest interface (positive inside).
int fe_init_order_parameter(const uint8_t* solid, int nx, int ny, int nz, int kind, const double* a,
                            double width, double* c_out) {
  if (!solid || !c_out || !a) return fe_fail(FE_ERR_ARG, "fe_init_order_parameter: bad arguments");
  const int N[3] = {nx, ny, nz};
  auto value = [&](double x, double y, double z) -> double {
    if (kind == 0) return a[0];
    const double pos[3] = {x, y, z};
    if (kind == 1) {
      const int axis = (int)a[3];
      const double L = N[axis], T = a[4];
      double sd = std::fmod(pos[axis] - a[axis], L);
      if (sd < 0) sd += L;
      // sd in [0, L): inside when sd + 0.5 in (0, T)
      const double u = sd + 0.5;
      const double d = (u < T) ? std::min(u, T - u) : -std::min(u - T, L - u);
      return 0.5 * (1.0 + std::tanh(2.0 * d / width));
    }
    double r2 = 0.0;
    for (int q = 0; q < 3; ++q) {
      double dd = std::fabs(pos[q] - a[q]);
      dd = std::min(dd, N[q] - dd);
      r2 += dd * dd;
    }
    const double d = a[3] - std::sqrt(r2);
    return 0.5 * (1.0 + std::tanh(2.0 * d / width));
  };
  // sites in node order: the fluid nodes of each (z, y) row are counted,
  // the rows' first sites follow by prefix sum, then rows fill in parallel
  const int64_t rows = (int64_t)ny * nz;
  std::vector<int64_t> first(rows + 1, 0);
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < rows; ++r) {
    const uint8_t* row = solid + r * nx;
    int64_t k = 0;
    for (int x = 0; x < nx; ++x) k += row[x] == 0;
    first[r + 1] = k;
  }
  for (int64_t r = 0; r < rows; ++r) first[r + 1] += first[r];
#pragma omp parallel for schedule(static)
  for (int64_t r = 0; r < rows; ++r) {
    const uint8_t* row = solid + r * nx;
    const double y = (double)(r % ny), z = (double)(r / ny);
    int64_t s = first[r];
    for (int x = 0; x < nx; ++x)
      if (!row[x]) c_out[s++] = value((double)x, y, z);
  }
  return FE_OK;
}

// Equilibrium distributions h_k = w_k c (1 + u_term), g_k = w_k (p + rho cs2
// u_term) of given per-site fields (u may be NULL for rest), in the
// reference layout f[k*n + i] (the plain equilibrium of the reference's
// open-boundary kernel, device_engine.cuh:790-797).
int fe_init_equilibrium(int64_t n, const double* c, const double* p, const double* ux, const double* uy,
                        const double* uz, double rho0, double rho1, double* h, double* g) {
  if (!c || !p || !h || !g || n < 0) return fe_fail(FE_ERR_ARG, "fe_init_equilibrium: bad arguments");
#pragma omp parallel for schedule(static) if (n > 65536)
  for (int64_t i = 0; i < n; ++i) {
    const double vx = ux ? ux[i] : 0.0, vy = uy ? uy[i] : 0.0, vz = uz ? uz[i] : 0.0;
    const double rho = rho1 + (rho0 - rho1) * c[i];
    for (int k = 0; k < Q; ++k) equilibrium_k(k, c[i], p[i], rho, vx, vy, vz, h[k * n + i], g[k * n + i]);
  }
  return FE_OK;
}

// Tracer seeding (reference particles_init_mode volume / plane_xz with
// particles_plane_offsets): uniform points whose nearest node is fluid, drawn
// from one seeded stream; each plane resampled until its quota is reached.
int fe_tracers_seed(const uint8_t* solid, int nx, int ny, int nz, int mode, int axis, const double* offsets,
                    int nplanes, int64_t count, uint64_t seed, double* pos_out, int32_t* plane_out) {
  if (!solid || !pos_out || !plane_out || nx < 1 || ny < 1 || nz < 1 || count < 0 || (mode != 0 && mode != 1) ||
      (mode == 1 && (!offsets || nplanes < 1 || axis < 0 || axis > 2)))
    return fe_fail(FE_ERR_ARG, "fe_tracers_seed: bad arguments");
  const int N[3] = {nx, ny, nz};
  int64_t fluid = 0;
  for (int64_t q = 0; q < (int64_t)nx * ny * nz; ++q) fluid += solid[q] ? 0 : 1;
  if (fluid == 0 && count > 0) return fe_fail(FE_ERR_ARG, "fe_tracers_seed: no fluid node");
  const int planes = mode == 1 ? nplanes : 1;
  const int64_t total = count * planes;
  Rng rng(seed);
  auto fluid_at = [&](const double* x) {
    int64_t i[3];
    for (int a = 0; a < 3; ++a) {
      i[a] = (int64_t)std::floor(x[a] + 0.5) % N[a];
      if (i[a] < 0) i[a] += N[a];
    }
    return solid[i[0] + (int64_t)nx * (i[1] + (int64_t)ny * i[2])] == 0;
  };
  int64_t k = 0;
  for (int pl = 0; pl < planes; ++pl) {
    int64_t got = 0, tries = 0;
    while (got < count) {
      if (++tries > 1000 * (count + 1000)) return fe_fail(FE_ERR_ARG, "fe_tracers_seed: plane has no fluid");
      double x[3];
      for (int a = 0; a < 3; ++a) x[a] = N[a] > 1 ? rng.uniform() * N[a] : 0.0;
      if (mode == 1) {
        double c = std::fmod(offsets[pl], (double)N[axis]);
        x[axis] = c < 0 ? c + N[axis] : c;
      }
      if (!fluid_at(x)) continue;
      for (int a = 0; a < 3; ++a) pos_out[a * total + k] = x[a];
      plane_out[k] = mode == 1 ? pl : 0;
      ++k;
      ++got;
    }
  }
  return FE_OK;
}

}  // extern "C"
