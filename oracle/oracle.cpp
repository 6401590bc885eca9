// CPU oracle for the Lee–Liu D3Q19 step — TEST INFRASTRUCTURE ONLY (see oracle.h).
//
// Each function restates one reference kernel or builder of matNBI/felbm_gpu,
// cited by file:line (paths relative to that project). Layout, tables and
// operation order follow the reference so that the restatement can be pinned
// against the reference's own kernels at the 1e-15 level.
#include "oracle.h"

#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>
#include <algorithm>
#include <omp.h>

namespace {

constexpr int Q = 19;
// reference include/felbm_gpu/d3q19.cuh:33-36
const int CX[Q] = {0, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1, 0, 0, 0, 0, 1, -1, 1, -1};
const int CY[Q] = {0, 0, 0, 1, -1, 0, 0, 1, -1, -1, 1, 1, -1, 1, -1, 0, 0, 0, 0};
const int CZ[Q] = {0, 0, 0, 0, 0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1};
const int OPP[Q] = {0, 2, 1, 4, 3, 6, 5, 8, 7, 10, 9, 12, 11, 14, 13, 16, 15, 18, 17};
// reference d3q19.cuh:39-44
double W(int k) { return k == 0 ? 1.0 / 3.0 : (k < 7 ? 1.0 / 18.0 : 1.0 / 36.0); }
// reference d3q19.cuh:45-50
const double CS2 = 1.0 / 3.0, ALPHA = 3.0, GAMMA = 1.5, BETA = 4.5;

// D3Q19 moment basis of d'Humieres et al. (2002) on the order above. The
// reference reads these values from felbm_local (multiphase_gpu.cuh:349-350),
// which is absent; the inverse is formed by Gauss-Jordan elimination.
double mrt_entry(int j, int k) {
  const int x = CX[k], y = CY[k], z = CZ[k], c2 = x * x + y * y + z * z;
  switch (j) {
    case 0: return 1;
    case 1: return 19 * c2 - 30;
    case 2: return (21 * c2 * c2 - 53 * c2 + 24) / 2;
    case 3: return x;
    case 4: return (5 * c2 - 9) * x;
    case 5: return y;
    case 6: return (5 * c2 - 9) * y;
    case 7: return z;
    case 8: return (5 * c2 - 9) * z;
    case 9: return 3 * x * x - c2;
    case 10: return (3 * c2 - 5) * (3 * x * x - c2);
    case 11: return y * y - z * z;
    case 12: return (3 * c2 - 5) * (y * y - z * z);
    case 13: return x * y;
    case 14: return y * z;
    case 15: return x * z;
    case 16: return (y * y - z * z) * x;
    case 17: return (z * z - x * x) * y;
    case 18: return (x * x - y * y) * z;
  }
  return 0;
}

void build_mrt(double M[Q][Q], double Minv[Q][Q]) {
  double A[Q][2 * Q];
  for (int j = 0; j < Q; ++j)
    for (int k = 0; k < Q; ++k) {
      M[j][k] = mrt_entry(j, k);
      A[j][k] = M[j][k];
      A[j][Q + k] = (j == k) ? 1.0 : 0.0;
    }
  for (int c = 0; c < Q; ++c) {
    int piv = c;
    for (int r = c + 1; r < Q; ++r)
      if (std::fabs(A[r][c]) > std::fabs(A[piv][c])) piv = r;
    if (piv != c)
      for (int k = 0; k < 2 * Q; ++k) std::swap(A[c][k], A[piv][k]);
    const double d = A[c][c];
    for (int k = 0; k < 2 * Q; ++k) A[c][k] /= d;
    for (int r = 0; r < Q; ++r)
      if (r != c) {
        const double f = A[r][c];
        if (f != 0.0)
          for (int k = 0; k < 2 * Q; ++k) A[r][k] -= f * A[c][k];
      }
  }
  for (int j = 0; j < Q; ++j)
    for (int k = 0; k < Q; ++k) Minv[j][k] = A[j][Q + k];
}

int mrt_kind(int j) {  // reference rate vector layout, device_engine.cuh:625
  if (j == 0 || j == 3 || j == 5 || j == 7) return 0;
  if (j == 1) return FE_MRT_E;
  if (j == 2) return FE_MRT_EPS;
  if (j == 4 || j == 6 || j == 8) return FE_MRT_Q;
  if (j == 10 || j == 12) return FE_MRT_PI;
  if (j >= 16) return FE_MRT_M;
  return FE_MRT_NU;
}

}  // namespace

struct or_engine {
  int nx, ny, nz;
  int64_t n;
  fe_params P;
  double forcing_factor = 1.0;
  std::vector<int64_t> node_of;  // site -> node
  std::vector<int64_t> site_of;  // node -> site or -1 (solid)
  // reference tables (multiphase_gpu.cuh:52-58), (Q-1)*n or Q*n
  std::vector<int32_t> cdm, cdp, bcase, bc1, bc2, avgnext, lcase, lc1, lc2, src;
  // in-place program (multiphase_gpu.cuh:45-46)
  bool inplace = false;
  std::vector<int64_t> op_a, op_b;
  std::vector<uint8_t> op_t;
  int64_t n_swap = 0, n_avg = 0, n_zero = 0;
  // state + fields (multiphase_gpu.cuh:64-71)
  std::vector<double> h, g, h2, g2;
  std::vector<double> c, p, rho, mu, ux, uy, uz, lapc, lapmu, relax;
  std::vector<double> gcc[3], gcb[3], gcm[3], gpc[3], gpb[3], gpm[3];
  std::vector<double> xtnd;
  double M[Q][Q], Minv[Q][Q];
  double target_mass = 0.0;
  // open boundary (multiphase_gpu.cuh:47-51, device_engine.cuh:45-58)
  bool open_bnd = false;
  fe_open_bnd B{};
  std::vector<int32_t> inlet, outlet, buf_verts, buf_refs;
  std::vector<double> inlet_coord;
  std::vector<uint8_t> bcproc;
  unsigned open_step = 0;
};

namespace {

inline int64_t wrap(int64_t a, int64_t n) { return ((a % n) + n) % n; }

// coords_to_idx with periodic wrap (multiphase_gpu.cuh:107-112,135-138); -1
// stands for a solid node (sd.is_solid(idx) is true exactly for it).
inline int64_t CI(const or_engine* e, int64_t x, int64_t y, int64_t z) {
  const int64_t node = wrap(x, e->nx) + e->nx * (wrap(y, e->ny) + e->ny * wrap(z, e->nz));
  return e->site_of[node];
}

void coords(const or_engine* e, int64_t i, int64_t& x, int64_t& y, int64_t& z) {
  const int64_t node = e->node_of[i];
  x = node % e->nx;
  y = (node / e->nx) % e->ny;
  z = node / ((int64_t)e->nx * e->ny);
}

// is_known(i, m): population m at site i arrives from a fluid node, i.e. the
// upstream node x - e_m is not solid. (felbm_local SubDomain::is_known is
// absent from the reference snapshot; this is the project's definition.)
inline bool is_known(const or_engine* e, int64_t x, int64_t y, int64_t z, int m) {
  return CI(e, x - CX[m], y - CY[m], z - CZ[m]) >= 0;
}

// Tables of multiphase_gpu.cuh:93-193 (grad_cd pairs, grad_bd cases, avg_dir,
// laplacian cases).
void build_tables(or_engine* e) {
  const int64_t n = e->n, Q1n = (Q - 1) * n, Vn = Q * n;
  const bool hbb = e->P.use_halfway_bb != 0;
  e->cdm.assign(Q1n, -1); e->cdp.assign(Q1n, -1);
  e->bcase.assign(Q1n, 0); e->bc1.assign(Q1n, -1); e->bc2.assign(Q1n, -1);
  e->avgnext.assign(Vn, -1);
  e->lcase.assign(Q1n, 0); e->lc1.assign(Q1n, -1); e->lc2.assign(Q1n, -1);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t x, y, z;
    coords(e, i, x, y, z);
    for (int m = 1; m < Q; ++m) {  // :105-122
      const int ex = CX[m], ey = CY[m], ez = CZ[m], mo = OPP[m];
      const int64_t inx = CI(e, x + ex, y + ey, z + ez), ipx = CI(e, x - ex, y - ey, z - ez);
      const bool Km = is_known(e, x, y, z, m), Ko = is_known(e, x, y, z, mo);
      const bool Nok = inx >= 0, Pok = ipx >= 0;
      int64_t a = -1, b = -1;
      if (Km && Ko && Pok && Nok) { a = ipx; b = inx; }
      else if (hbb && Km && Pok) { a = ipx; b = i; }
      else if (hbb && Ko && Nok) { a = i; b = inx; }
      e->cdm[(m - 1) * n + i] = (int32_t)a;
      e->cdp[(m - 1) * n + i] = (int32_t)b;
    }
    for (int m = 1; m < Q; ++m) {  // :133-154
      const int ex = CX[m], ey = CY[m], ez = CZ[m], mo = OPP[m];
      const int64_t inx = CI(e, x + ex, y + ey, z + ez), in2 = CI(e, x + 2 * ex, y + 2 * ey, z + 2 * ez);
      const int64_t ipx = CI(e, x - ex, y - ey, z - ez), ip2 = CI(e, x - 2 * ex, y - 2 * ey, z - 2 * ez);
      const bool Km = is_known(e, x, y, z, m), Ko = is_known(e, x, y, z, mo);
      int cs = 0;
      int64_t c1 = -1, c2 = -1;
      if (Ko && inx >= 0) {
        int64_t xn, yn, zn;
        coords(e, inx, xn, yn, zn);
        if (is_known(e, xn, yn, zn, mo) && in2 >= 0) { cs = 1; c1 = inx; c2 = in2; }
        else if (!hbb) { cs = 2; c1 = inx; }
        else { cs = 3; c1 = inx; }
      } else {
        if (!hbb) {
          if (Km && ipx >= 0) {
            int64_t xp, yp, zp;
            coords(e, ipx, xp, yp, zp);
            if (is_known(e, xp, yp, zp, m) && ip2 >= 0) { cs = 1; c1 = ipx; c2 = ip2; }
          }
        } else {
          if (Km && ipx >= 0) { cs = 4; c1 = ipx; }
        }
      }
      e->bcase[(m - 1) * n + i] = cs;
      e->bc1[(m - 1) * n + i] = (int32_t)c1;
      e->bc2[(m - 1) * n + i] = (int32_t)c2;
    }
    for (int m = 0; m < Q; ++m) {  // :173-177
      const int64_t nxi = CI(e, x + CX[m], y + CY[m], z + CZ[m]);
      e->avgnext[m * n + i] = (is_known(e, x, y, z, OPP[m]) && nxi >= 0) ? (int32_t)nxi : -1;
    }
    for (int m = 1; m < Q; ++m) {  // :178-188
      const int ex = CX[m], ey = CY[m], ez = CZ[m], mo = OPP[m];
      const int64_t inx = CI(e, x + ex, y + ey, z + ez), ipx = CI(e, x - ex, y - ey, z - ez);
      const bool Km = is_known(e, x, y, z, m), Ko = is_known(e, x, y, z, mo);
      const bool Pok = ipx >= 0, Nok = inx >= 0;
      int cs = 0;
      int64_t c1 = -1, c2 = -1;
      if (Km && Ko && Pok && Nok) { cs = 1; c1 = ipx; c2 = inx; }
      else if (Km && Pok) { cs = hbb ? 3 : 2; c1 = ipx; }
      else if (Ko && Nok) { cs = hbb ? 3 : 2; c1 = inx; }
      e->lcase[(m - 1) * n + i] = cs;
      e->lc1[(m - 1) * n + i] = (int32_t)c1;
      e->lc2[(m - 1) * n + i] = (int32_t)c2;
    }
  }
  // Streaming source table (multiphase_gpu.cuh:196-208). The rows of felbm_local's
  // StreamingOperator are absent; the project's rule: pull from x - e_k with
  // periodic wrap, halfway bounce-back (own opposite slot) when that node is solid.
  e->src.assign(Vn, -2);
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    int64_t x, y, z;
    coords(e, i, x, y, z);
    for (int k = 0; k < Q; ++k) {
      const int64_t up = CI(e, x - CX[k], y - CY[k], z - CZ[k]);
      e->src[k * n + i] = (int32_t)(up >= 0 ? k * n + up : OPP[k] * n + i);
    }
  }
}

// In-place op program + host verification (multiphase_gpu.cuh:213-283).
bool build_inplace(or_engine* e) {
  const int64_t n = e->n, Vn = Q * n;
  std::vector<char> dn(Vn, 0);
  e->op_a.clear(); e->op_b.clear(); e->op_t.clear();
  for (int64_t j = 0; j < Vn; ++j) {
    if (dn[j]) continue;
    const int64_t k = j / n, i = j - k * n, kb = OPP[k], jb = kb * n + i, sc = e->src[j];
    if (sc == jb) { dn[j] = 1; }
    else if (sc >= 0) {
      const int64_t sk = sc / n, x = sc - sk * n, q = kb * n + x;
      if (sk != k || e->src[q] != kb * n + i || dn[q]) return false;
      e->op_a.push_back(j); e->op_b.push_back(q); e->op_t.push_back(0);
      dn[j] = dn[q] = 1;
    } else if (sc == -1) {
      if (e->src[jb] != -1 || dn[jb]) return false;
      e->op_a.push_back(j); e->op_b.push_back(jb); e->op_t.push_back(1);
      dn[j] = dn[jb] = 1;
    } else {
      e->op_a.push_back(j); e->op_b.push_back(j); e->op_t.push_back(2);
      dn[j] = 1;
    }
  }
  std::vector<double> f(Vn), ref(Vn), r(Vn);
  unsigned long long seed = 0x243F6A8885A308D3ull;
  for (int64_t j = 0; j < Vn; ++j) {
    seed = seed * 6364136223846793005ull + 1442695040888963407ull;
    f[j] = (double)(seed >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
  for (int64_t j = 0; j < Vn; ++j) {
    const int64_t k = j / n, i = j - k * n, jb = OPP[k] * n + i, sc = e->src[j];
    ref[j] = sc >= 0 ? f[sc] : (sc == -1 ? 0.5 * (f[j] + f[jb]) : 0.0);
    r[j] = f[jb];
  }
  for (size_t q = 0; q < e->op_a.size(); ++q) {
    const int64_t a = e->op_a[q], b = e->op_b[q];
    if (e->op_t[q] == 0) std::swap(r[a], r[b]);
    else if (e->op_t[q] == 1) { const double m = 0.5 * (r[a] + r[b]); r[a] = m; r[b] = m; }
    else r[a] = 0.0;
  }
  for (int64_t j = 0; j < Vn; ++j)
    if (r[j] != ref[j]) return false;
  e->n_swap = e->n_avg = e->n_zero = 0;
  for (uint8_t t : e->op_t) (t == 0 ? e->n_swap : (t == 1 ? e->n_avg : e->n_zero))++;
  return true;
}

// cd_dir_val / bd_dir_val / avg_dir_val (device_engine.cuh:89-113)
inline double cd_dir_val(const or_engine* e, const double* f, int64_t i, int m) {
  if (m == 0) return 0.0;
  const int64_t idx = (m - 1) * e->n + i;
  const int32_t cm = e->cdm[idx];
  return (cm < 0) ? 0.0 : 0.5 * (f[e->cdp[idx]] - f[cm]);
}
inline double bd_dir_val(const or_engine* e, const double* f, double f0, int64_t i, int m) {
  if (m == 0) return 0.0;
  const int64_t idx = (m - 1) * e->n + i;
  const int cs = e->bcase[idx];
  if (cs == 0) return 0.0;
  const double f1 = f[e->bc1[idx]];
  if (cs == 1) { const double f2 = f[e->bc2[idx]]; return -1.5 * f0 + 2.0 * f1 + -0.5 * f2; }
  else if (cs == 2) return -2.0 * f0 + 2.0 * f1;
  else if (cs == 3) return -1.5 * f0 + 1.5 * f1;
  else return 0.5 * f0 + -0.5 * f1;
}
inline double avg_dir_val(const or_engine* e, const double* x, double xi, int64_t i, int m) {
  const int32_t nx = e->avgnext[m * e->n + i];
  return (nx < 0) ? xi : 0.5 * (xi + x[nx]);
}

// k_moments (device_engine.cuh:116-135)
void moments(or_engine* e) {
  const fe_params& P = e->P;
  const int64_t n = e->n;
  const double drho = P.rho0 - P.rho1, four_beta = 4.0 * P.beta;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double c = 0, p = 0, ux = 0, uy = 0, uz = 0;
    for (int k = 0; k < Q; ++k) {
      const double hv = e->h[k * n + i], gv = e->g[k * n + i];
      c += hv; p += gv; ux += (double)CX[k] * gv; uy += (double)CY[k] * gv; uz += (double)CZ[k] * gv;
    }
    const double c_log = c * (1.0 - c);
    const double rho = P.rho1 + drho * c;
    const double inv = 1.0 / (CS2 * rho);
    ux *= inv; uy *= inv; uz *= inv;
    const double mu = four_beta * c_log * (0.5 - c);
    const double cp = c < 0.0 ? 0.0 : (c > 1.0 ? 1.0 : c);
    const double tau = 1.0 / (cp / P.tau0 + (1.0 - cp) / P.tau1);
    const double rp = 1.0 / (tau + 0.5);
    e->c[i] = c; e->p[i] = p; e->rho[i] = rho; e->mu[i] = mu;
    e->ux[i] = ux; e->uy[i] = uy; e->uz[i] = uz; e->relax[i] = rp;
  }
}

// d_inlet_gate (device_engine.cuh:699-728)
double inlet_gate(const or_engine* e, unsigned step, double coord) {
  const fe_open_bnd& B = e->B;
  const double w = B.inlet_ramp;
  if (B.inlet_mode == 1) {
    const double Per = B.inlet_period;
    if (Per <= 0.0) return 1.0;
    const double tau = (double)step - Per * std::floor((double)step / Per);
    const double lo = 0.5 * Per - 0.5 * B.inlet_duty * Per, hi = 0.5 * Per + 0.5 * B.inlet_duty * Per;
    if (w <= 0.0) return (tau >= lo && tau < hi) ? 1.0 : 0.0;
    return 0.5 * (std::tanh(2.0 * (tau - lo) / w) - std::tanh(2.0 * (tau - hi) / w));
  }
  if (B.inlet_mode == 2) {
    const double x = coord - B.split_pos;
    if (w <= 0.0) return (x < 0.0) ? 1.0 : 0.0;
    return 0.5 * (1.0 - std::tanh(2.0 * x / w));
  }
  if (B.inlet_mode == 3) {
    const double Per = B.inlet_period;
    if (Per <= 0.0) return 1.0;
    double t = coord - B.split_pos;
    t = t - Per * std::floor(t / Per);
    const double lo = 0.5 * Per - 0.5 * B.inlet_duty * Per, hi = 0.5 * Per + 0.5 * B.inlet_duty * Per;
    if (w <= 0.0) return (t >= lo && t < hi) ? 1.0 : 0.0;
    return 0.5 * (std::tanh(2.0 * (t - lo) / w) - std::tanh(2.0 * (t - hi) / w));
  }
  return 1.0;
}

// enforce_open_bnd_fields: k_open_bnd_fields + k_open_bnd_buf_fields
// (multiphase_gpu.cuh:404-418; device_engine.cuh:738-759,807-815)
void enforce_open_bnd_fields(or_engine* e) {
  if (!e->open_bnd) return;
  const fe_open_bnd& B = e->B;
  const fe_params& P = e->P;
  for (size_t j = 0; j < e->inlet.size(); ++j) {
    const int64_t i = e->inlet[j];
    if (B.use_in_vel) { e->ux[i] = B.u_in_x; e->uy[i] = B.u_in_y; e->uz[i] = B.u_in_z; }
    if (B.use_in_prs) e->p[i] = B.p_in;
    if (B.use_in_fluid) {
      const double gate = inlet_gate(e, e->open_step, e->inlet_coord.empty() ? 0.0 : e->inlet_coord[j]);
      const double c = (1.0 - B.inlet_c_a) + (2.0 * B.inlet_c_a - 1.0) * gate;
      e->c[i] = c; e->rho[i] = c * P.rho0 + (1.0 - c) * P.rho1;
    }
  }
  for (size_t j = 0; j < e->outlet.size(); ++j) {
    const int64_t i = e->outlet[j];
    if (B.use_out_prs) e->p[i] = B.p_out;
    if (B.use_out_fluid) { e->c[i] = B.c_out_fixed; e->rho[i] = B.rho_out_fixed; }
  }
  if (B.copy_to_buffers)
    for (size_t j = 0; j < e->buf_verts.size(); ++j) {
      const int64_t bid = e->buf_verts[j], rid = e->buf_refs[j];
      e->c[bid] = e->c[rid]; e->rho[bid] = e->rho[rid]; e->p[bid] = e->p[rid];
      e->ux[bid] = e->ux[rid]; e->uy[bid] = e->uy[rid]; e->uz[bid] = e->uz[rid];
    }
}

// k_grad_cd_mf (device_engine.cuh:897-913)
void grad_cd(const or_engine* e, const double* f, double* gx, double* gy, double* gz) {
  const int64_t n = e->n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double sx = 0, sy = 0, sz = 0;
    for (int m = 1; m < Q; ++m) {
      const int64_t idx = (m - 1) * n + i;
      const int32_t cm = e->cdm[idx];
      if (cm < 0) continue;
      const double d = f[e->cdp[idx]] - f[cm];
      const double coef = ALPHA * 0.5 * W(m);
      sx += coef * (double)CX[m] * d; sy += coef * (double)CY[m] * d; sz += coef * (double)CZ[m] * d;
    }
    gx[i] = sx; gy[i] = sy; gz[i] = sz;
  }
}

// k_grad_bd_mf (device_engine.cuh:924-945)
void grad_bd(const or_engine* e, const double* f, double* gx, double* gy, double* gz) {
  const int64_t n = e->n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    double sx = 0, sy = 0, sz = 0;
    const double f0 = f[i];
    for (int m = 1; m < Q; ++m) {
      const int64_t idx = (m - 1) * n + i;
      const int cs = e->bcase[idx];
      if (cs == 0) continue;
      const double f1 = f[e->bc1[idx]];
      double val;
      if (cs == 1) { const double f2 = f[e->bc2[idx]]; val = -1.5 * f0 + 2.0 * f1 + -0.5 * f2; }
      else if (cs == 2) val = -2.0 * f0 + 2.0 * f1;
      else if (cs == 3) val = -1.5 * f0 + 1.5 * f1;
      else val = 0.5 * f0 + -0.5 * f1;
      const double base = ALPHA * W(m);
      sx += base * (double)CX[m] * val; sy += base * (double)CY[m] * val; sz += base * (double)CZ[m] * val;
    }
    gx[i] = sx; gy[i] = sy; gz[i] = sz;
  }
}

// k_grad_md (device_engine.cuh:138-146)
void grad_md(const or_engine* e, std::vector<double>* cd, std::vector<double>* bd, std::vector<double>* md) {
  for (int d = 0; d < 3; ++d)
    for (int64_t i = 0; i < e->n; ++i) md[d][i] = 0.5 * (cd[d][i] + bd[d][i]);
}

// k_lap_mf over the 2n input [field, bnd] (device_engine.cuh:996-1010)
void laplacian(const or_engine* e, const double* xtnd, double* out) {
  const int64_t n = e->n;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double f0 = xtnd[i], bnd = xtnd[n + i];
    double s = 0;
    for (int m = 1; m < Q; ++m) {
      const int64_t idx = (m - 1) * n + i;
      const int cs = e->lcase[idx];
      if (cs == 0) continue;
      const double w = ALPHA * W(m);
      if (cs == 1) { const double f1 = xtnd[e->lc1[idx]], f2 = xtnd[e->lc2[idx]]; s += w * (f1 - 2.0 * f0 + f2); }
      else if (cs == 2) { const double f1 = xtnd[e->lc1[idx]]; s += w * (2.0 * f1 - 2.0 * f0 - 2.0 * bnd); }
      else { const double f1 = xtnd[e->lc1[idx]]; s += w * (f1 - f0 - bnd); }
    }
    out[i] = s;
  }
}

// k_vel_press_corr (device_engine.cuh:177-196)
void vel_press_corr(or_engine* e) {
  const fe_params& P = e->P;
  const double drho = P.rho0 - P.rho1, ff = e->forcing_factor;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < e->n; ++i) {
    if (!e->bcproc.empty() && e->bcproc[i]) continue;
    const double mu = e->mu[i], rho = e->rho[i];
    const double gx = e->gcc[0][i], gy = e->gcc[1][i], gz = e->gcc[2][i];
    const double mor = mu / rho;
    const double ux = e->ux[i] + 0.5 * (P.gx + P.fx * ff / rho + mor * gx);
    const double uy = e->uy[i] + 0.5 * (P.gy + P.fy * ff / rho + mor * gy);
    const double uz = e->uz[i] + 0.5 * (P.gz + P.fz * ff / rho + mor * gz);
    e->ux[i] = ux; e->uy[i] = uy; e->uz[i] = uz;
    const double u_dot_drho = drho * (ux * gx + uy * gy + uz * gz);
    e->p[i] += 0.5 * u_dot_drho * CS2;
  }
}

// compute_fields half of step() (multiphase_gpu.cuh:526-541); `full` also
// forms the p gradients and grad(mu) inputs needed by the collision.
void compute_fields(or_engine* e, bool full) {
  const int64_t n = e->n;
  moments(e);
  enforce_open_bnd_fields(e);
  grad_cd(e, e->c.data(), e->gcc[0].data(), e->gcc[1].data(), e->gcc[2].data());
  if (full) {
    grad_bd(e, e->c.data(), e->gcb[0].data(), e->gcb[1].data(), e->gcb[2].data());
    grad_md(e, e->gcc, e->gcb, e->gcm);
  }
  // k_pack_lap_c (device_engine.cuh:159-165), laplacian, k_mu_axpy (:149-153)
  for (int64_t i = 0; i < n; ++i) {
    const double cv = e->c[i];
    e->xtnd[i] = cv;
    e->xtnd[n + i] = e->P.bnd_coeff * cv * (1.0 - cv);
  }
  laplacian(e, e->xtnd.data(), e->lapc.data());
  for (int64_t i = 0; i < n; ++i) e->mu[i] += -e->P.kappa * e->lapc[i];
  if (full) {
    // k_pack_lap_zero (:168-173), laplacian -> lapmu
    for (int64_t i = 0; i < n; ++i) { e->xtnd[i] = e->mu[i]; e->xtnd[n + i] = 0.0; }
    laplacian(e, e->xtnd.data(), e->lapmu.data());
  }
  vel_press_corr(e);
  if (full) {
    grad_cd(e, e->p.data(), e->gpc[0].data(), e->gpc[1].data(), e->gpc[2].data());
    grad_bd(e, e->p.data(), e->gpb[0].data(), e->gpb[1].data(), e->gpb[2].data());
    grad_md(e, e->gpc, e->gpb, e->gpm);
  }
}

// apply_open_bnd: k_open_bnd / k_open_bnd_buf (multiphase_gpu.cuh:427-446;
// device_engine.cuh:761-798,826-846)
void plain_eq(or_engine* e, int64_t i, double ux, double uy, double uz, double pp, double rho, double c) {
  const int64_t n = e->n;
  const double u_sq = ux * ux + uy * uy + uz * uz;
  for (int k = 0; k < Q; ++k) {
    const double w = W(k);
    const double uk = ux * CX[k] + uy * CY[k] + uz * CZ[k];
    const double u_term = uk * (ALPHA + BETA * uk) - GAMMA * u_sq;
    e->h[k * n + i] = c * w * (1.0 + u_term);
    e->g[k * n + i] = w * (pp + rho * CS2 * u_term);
  }
}

void apply_open_bnd(or_engine* e) {
  if (!e->open_bnd) return;
  const fe_open_bnd& B = e->B;
  const fe_params& P = e->P;
  if (B.copy_to_buffers) {
    for (size_t j = 0; j < e->buf_verts.size(); ++j) {
      const int64_t bid = e->buf_verts[j], rid = e->buf_refs[j];
      plain_eq(e, bid, e->ux[rid], e->uy[rid], e->uz[rid], e->p[rid], e->rho[rid], e->c[rid]);
    }
  } else {
    for (size_t j = 0; j < e->inlet.size(); ++j) {
      const int64_t i = e->inlet[j];
      double ux, uy, uz, pp, rho, c;
      if (B.use_in_vel) { ux = B.u_in_x; uy = B.u_in_y; uz = B.u_in_z; }
      else { ux = e->ux[i]; uy = e->uy[i]; uz = e->uz[i]; }
      pp = B.use_in_prs ? B.p_in : e->p[i];
      if (B.use_in_fluid) {
        const double gate = inlet_gate(e, e->open_step, e->inlet_coord.empty() ? 0.0 : e->inlet_coord[j]);
        c = (1.0 - B.inlet_c_a) + (2.0 * B.inlet_c_a - 1.0) * gate;
        rho = c * P.rho0 + (1.0 - c) * P.rho1;
      } else { rho = e->rho[i]; c = e->c[i]; }
      plain_eq(e, i, ux, uy, uz, pp, rho, c);
    }
    for (size_t j = 0; j < e->outlet.size(); ++j) {
      const int64_t i = e->outlet[j];
      const double ux = e->ux[i], uy = e->uy[i], uz = e->uz[i];
      const double pp = B.use_out_prs ? B.p_out : e->p[i];
      double rho, c;
      if (B.use_out_fluid) { rho = B.rho_out_fixed; c = B.c_out_fixed; }
      else { rho = e->rho[i]; c = e->c[i]; }
      plain_eq(e, i, ux, uy, uz, pp, rho, c);
    }
  }
  ++e->open_step;
}

// MRT rates of one site (device_engine.cuh:641-643) with the per-kind modes.
void mrt_rates(const or_engine* e, double s0, double s[Q]) {
  const double tau = 1.0 / s0 - 0.5;
  const double s1 = 2.0 * tau / (2.0 * e->P.mrt_lambda + tau);
  for (int j = 0; j < Q; ++j) {
    const int kind = mrt_kind(j);
    if (kind == 0) { s[j] = 0.0; continue; }
    const int mode = e->P.mrt_rate_mode[kind];
    s[j] = mode == FE_RATE_S0 ? s0 : (mode == FE_RATE_MAGIC ? s1 : e->P.mrt_rate_value[kind]);
  }
}

// k_collide_fused_mrt (device_engine.cuh:547-651) and k_collide_fused_bgk
// (:459-545), writing into h/g in place (standard slots); the in-place
// streaming's reversed-slot write is a permutation applied by stream().
void collide(or_engine* e) {
  const fe_params& P = e->P;
  const int64_t n = e->n;
  const double drho = P.rho0 - P.rho1, ffac = e->forcing_factor;
  const bool mrt = P.use_mrt != 0;
#pragma omp parallel for schedule(static)
  for (int64_t i = 0; i < n; ++i) {
    const double c = e->c[i], rho = e->rho[i], p = e->p[i], mu = e->mu[i];
    const double ux = e->ux[i], uy = e->uy[i], uz = e->uz[i], lmu = e->lapmu[i];
    const double bfx = rho * P.gx + P.fx * ffac, bfy = rho * P.gy + P.fy * ffac, bfz = rho * P.gz + P.fz * ffac;
    const double f_dpx = e->gpm[0][i], f_dpy = e->gpm[1][i], f_dpz = e->gpm[2][i];
    const double f_dcx = e->gcm[0][i], f_dcy = e->gcm[1][i], f_dcz = e->gcm[2][i];
    const double e_dpx = e->gpc[0][i], e_dpy = e->gpc[1][i], e_dpz = e->gpc[2][i];
    const double e_dcx = e->gcc[0][i], e_dcy = e->gcc[1][i], e_dcz = e->gcc[2][i];
    if (mrt) {
      const double drho_cs2 = drho * CS2, rho_cs2 = rho * CS2, c_over = c / rho_cs2;
      const double drcx = drho_cs2 * e_dcx, drcy = drho_cs2 * e_dcy, drcz = drho_cs2 * e_dcz;
      const double e_fgx = mu * e_dcx + bfx, e_fgy = mu * e_dcy + bfy, e_fgz = mu * e_dcz + bfz;
      const double e_fhx = e_dcx - c_over * (e_dpx - e_fgx), e_fhy = e_dcy - c_over * (e_dpy - e_fgy),
                   e_fhz = e_dcz - c_over * (e_dpz - e_fgz);
      const double gamma_u_sq = GAMMA * (ux * ux + uy * uy + uz * uz);
      const double u_term_h = ux * e_fhx + uy * e_fhy + uz * e_fhz;
      const double u_force_g = ux * e_fgx + uy * e_fgy + uz * e_fgz;
      const double u_drho = ux * drcx + uy * drcy + uz * drcz;
      const double drmx = drho_cs2 * f_dcx, drmy = drho_cs2 * f_dcy, drmz = drho_cs2 * f_dcz;
      const double f_fgx = mu * f_dcx + bfx, f_fgy = mu * f_dcy + bfy, f_fgz = mu * f_dcz + bfz;
      const double f_fhx = f_dcx - c_over * (f_dpx - f_fgx), f_fhy = f_dcy - c_over * (f_dpy - f_fgy),
                   f_fhz = f_dcz - c_over * (f_dpz - f_fgz);
      const double u_fh_f = ux * f_fhx + uy * f_fhy + uz * f_fhz;
      const double u_drm = ux * drmx + uy * drmy + uz * drmz;
      const double u_fg_f = ux * f_fgx + uy * f_fgy + uz * f_fgz;
      double cg[Q], fgs[Q], go[Q];
      for (int k = 0; k < Q; ++k) {
        const double w = W(k);
        const double uk = ux * CX[k] + uy * CY[k] + uz * CZ[k];
        const double u_term = uk * (ALPHA + BETA * uk) - gamma_u_sq;
        const double G = w * (1.0 + u_term);
        const double w_u_term = G - w;
        const double f_proj = bfx * CX[k] + bfy * CY[k] + bfz * CZ[k];
        const double cd_c = cd_dir_val(e, e->c.data(), i, k), cd_p = cd_dir_val(e, e->p.data(), i, k);
        const double drho_dk = drho_cs2 * cd_c;
        const double eh = c * G + 0.5 * G * (u_term_h - cd_c + c_over * (cd_p - mu * cd_c - f_proj));
        const double eg = w * p + rho_cs2 * w_u_term +
                          0.5 * ((u_drho - drho_dk) * w_u_term + (u_force_g + mu * cd_c + f_proj) * G);
        const double dGk = G - w;
        const double bd_c = bd_dir_val(e, e->c.data(), c, i, k), bd_p = bd_dir_val(e, e->p.data(), p, i, k);
        const double dc_dk = 0.5 * (cd_c + bd_c), dp_dk = 0.5 * (cd_p + bd_p);
        const double drho_dk2 = drho_cs2 * dc_dk;
        const double ff = mu * dc_dk + f_proj;
        const double avgk = avg_dir_val(e, e->lapmu.data(), lmu, i, k);
        const double fh = G * (dc_dk - c_over * (dp_dk - ff) - u_fh_f + P.mobility * avgk);
        const double fg = (drho_dk2 - u_drm) * dGk + (ff - u_fg_f) * G;
        const double gk = e->g[k * n + i];
        e->h[k * n + i] = eh + fh;
        cg[k] = eg - gk; fgs[k] = fg; go[k] = gk;
      }
      double s[Q], xx[Q];
      mrt_rates(e, e->relax[i], s);
      for (int k = 0; k < Q; ++k) xx[k] = 0.0;
      for (int nn = 0; nn < Q; ++nn) {
        const double y = cg[nn];
        for (int m = 1; m < Q; ++m) xx[m] += s[m] * e->M[m][nn] * y;
      }
      for (int m = 0; m < Q; ++m) {
        double acc = 0.0;
        for (int nn = 0; nn < Q; ++nn) acc += e->Minv[m][nn] * xx[nn];
        cg[m] = acc;
      }
      for (int k = 0; k < Q; ++k) e->g[k * n + i] = go[k] + cg[k] + fgs[k];
    } else {
      const double relax = e->relax[i];
      const double drcx = drho * e_dcx * CS2, drcy = drho * e_dcy * CS2, drcz = drho * e_dcz * CS2;
      const double e_fgx = mu * e_dcx + bfx, e_fgy = mu * e_dcy + bfy, e_fgz = mu * e_dcz + bfz;
      const double a_over_rho = ALPHA / rho;
      const double e_fhx = e_dcx - c * a_over_rho * (e_dpx - e_fgx), e_fhy = e_dcy - c * a_over_rho * (e_dpy - e_fgy),
                   e_fhz = e_dcz - c * a_over_rho * (e_dpz - e_fgz);
      const double u_sq = ux * ux + uy * uy + uz * uz;
      const double u_fh_e = ux * e_fhx + uy * e_fhy + uz * e_fhz;
      const double u_drhocd = ux * drcx + uy * drcy + uz * drcz;
      const double u_fg_e = ux * e_fgx + uy * e_fgy + uz * e_fgz;
      const double drho_cs2 = drho * CS2;
      const double drmx = drho_cs2 * f_dcx, drmy = drho_cs2 * f_dcy, drmz = drho_cs2 * f_dcz;
      const double c_over = c / CS2 / rho;
      const double f_fgx = mu * f_dcx + bfx, f_fgy = mu * f_dcy + bfy, f_fgz = mu * f_dcz + bfz;
      const double f_fhx = f_dcx - c_over * (f_dpx - f_fgx), f_fhy = f_dcy - c_over * (f_dpy - f_fgy),
                   f_fhz = f_dcz - c_over * (f_dpz - f_fgz);
      const double u_fh_f = ux * f_fhx + uy * f_fhy + uz * f_fhz;
      const double u_drm = ux * drmx + uy * drmy + uz * drmz;
      const double u_fg_f = ux * f_fgx + uy * f_fgy + uz * f_fgz;
      for (int k = 0; k < Q; ++k) {
        const double w = W(k);
        const double uk = ux * CX[k] + uy * CY[k] + uz * CZ[k];
        const double u_term = uk * (ALPHA + BETA * uk) - GAMMA * u_sq;
        const double G = w * (1.0 + u_term);
        const double f_proj = bfx * CX[k] + bfy * CY[k] + bfz * CZ[k];
        const double cd_c = cd_dir_val(e, e->c.data(), i, k), cd_p = cd_dir_val(e, e->p.data(), i, k);
        const double drho_dk = drho * cd_c * CS2;
        double eh = c * G;
        eh -= 0.5 * G * (cd_c - c * a_over_rho * (cd_p - mu * cd_c - f_proj));
        eh += 0.5 * G * u_fh_e;
        double eg = w * (p + rho * CS2 * u_term);
        eg -= 0.5 * (drho_dk * (G - w) + (mu * cd_c + f_proj) * G);
        eg += 0.5 * ((G - w) * u_drhocd + G * u_fg_e);
        const double dGk = G - w;
        const double bd_c = bd_dir_val(e, e->c.data(), c, i, k), bd_p = bd_dir_val(e, e->p.data(), p, i, k);
        const double dc_dk = 0.5 * (cd_c + bd_c), dp_dk = 0.5 * (cd_p + bd_p);
        const double drho_dk2 = drho_cs2 * dc_dk;
        const double ff = mu * dc_dk + f_proj;
        const double avgk = avg_dir_val(e, e->lapmu.data(), lmu, i, k);
        const double fh = G * (dc_dk - c_over * (dp_dk - ff) - u_fh_f + P.mobility * avgk);
        const double fg = (drho_dk2 - u_drm) * dGk + (ff - u_fg_f) * G;
        const double gk = e->g[k * n + i];
        e->h[k * n + i] = eh + fh;
        e->g[k * n + i] = gk + relax * (eg - gk) + fg;
      }
    }
  }
}

// streaming: k_stream_gather (device_engine.cuh:882-889) + pointer swap, or the
// reversed-slot layout followed by k_stream_inplace (:859-873).
void stream(or_engine* e) {
  const int64_t n = e->n, Vn = Q * n;
  if (e->inplace) {
    // the fused collision writes direction k into slot opp(k) (:612,649)
    std::vector<double> rh(Vn), rg(Vn);
    for (int k = 0; k < Q; ++k)
      for (int64_t i = 0; i < n; ++i) {
        rh[OPP[k] * n + i] = e->h[k * n + i];
        rg[OPP[k] * n + i] = e->g[k * n + i];
      }
    for (size_t q = 0; q < e->op_a.size(); ++q) {
      const int64_t a = e->op_a[q], b = e->op_b[q];
      const uint8_t t = e->op_t[q];
      if (t == 0) { std::swap(rh[a], rh[b]); std::swap(rg[a], rg[b]); }
      else if (t == 1) {
        const double mh = 0.5 * (rh[a] + rh[b]); rh[a] = mh; rh[b] = mh;
        const double mg = 0.5 * (rg[a] + rg[b]); rg[a] = mg; rg[b] = mg;
      } else { rh[a] = 0; rg[a] = 0; }
    }
    e->h.swap(rh); e->g.swap(rg);
    return;
  }
#pragma omp parallel for schedule(static)
  for (int64_t j = 0; j < Vn; ++j) {
    const int32_t s = e->src[j];
    if (s >= 0) { e->h2[j] = e->h[s]; e->g2[j] = e->g[s]; }
    else if (s == -1) {
      const int64_t k = j / n, i = j - k * n, o = OPP[k] * n + i;
      e->h2[j] = 0.5 * (e->h[j] + e->h[o]); e->g2[j] = 0.5 * (e->g[j] + e->g[o]);
    } else { e->h2[j] = 0.0; e->g2[j] = 0.0; }
  }
  e->h.swap(e->h2); e->g.swap(e->g2);
}

// k_mass_weight (device_engine.cuh:1109-1126): M = sum c, W = sum c(1-c)^+
// Summed in fixed blocks of 4096 sites, then block partials in order, so the
// result does not depend on the thread count.
void mass_weight(const or_engine* e, double& M, double& Wt) {
  const int64_t n = e->n, BS = 4096, nb = (n + BS - 1) / BS;
  std::vector<double> pm(nb, 0.0), pw(nb, 0.0);
#pragma omp parallel for schedule(static)
  for (int64_t b = 0; b < nb; ++b) {
    double m = 0.0, w = 0.0;
    for (int64_t i = b * BS; i < std::min(n, (b + 1) * BS); ++i) {
      double c = 0.0;
      for (int k = 0; k < Q; ++k) c += e->h[k * n + i];
      double phi = c * (1.0 - c);
      if (phi < 0.0) phi = 0.0;
      m += c; w += phi;
    }
    pm[b] = m; pw[b] = w;
  }
  M = 0.0; Wt = 0.0;
  for (int64_t b = 0; b < nb; ++b) { M += pm[b]; Wt += pw[b]; }
}

}  // namespace

extern "C" {

or_engine* or_create(const fe_params* p, int nx, int ny, int nz, const uint8_t* solid, int inplace) {
  or_engine* e = new or_engine();
  e->nx = nx; e->ny = ny; e->nz = nz;
  e->P = *p;
  const int64_t nn = (int64_t)nx * ny * nz;
  e->site_of.assign(nn, -1);
  for (int64_t node = 0; node < nn; ++node)
    if (!solid[node]) { e->site_of[node] = (int64_t)e->node_of.size(); e->node_of.push_back(node); }
  e->n = (int64_t)e->node_of.size();
  const int64_t n = e->n, Vn = Q * n;
  build_tables(e);
  e->inplace = inplace && build_inplace(e);
  e->h.assign(Vn, 0.0); e->g.assign(Vn, 0.0);
  if (!e->inplace) { e->h2.assign(Vn, 0.0); e->g2.assign(Vn, 0.0); }
  for (auto* v : {&e->c, &e->p, &e->rho, &e->mu, &e->ux, &e->uy, &e->uz, &e->lapc, &e->lapmu, &e->relax})
    v->assign(n, 0.0);
  for (int d = 0; d < 3; ++d)
    for (auto* v : {&e->gcc[d], &e->gcb[d], &e->gcm[d], &e->gpc[d], &e->gpb[d], &e->gpm[d]}) v->assign(n, 0.0);
  e->xtnd.assign(2 * n, 0.0);
  build_mrt(e->M, e->Minv);
  return e;
}

void or_destroy(or_engine* e) { delete e; }
int64_t or_n(const or_engine* e) { return e->n; }
void or_site_nodes(const or_engine* e, int64_t* node) { std::copy(e->node_of.begin(), e->node_of.end(), node); }
void or_set_params(or_engine* e, const fe_params* p) { e->P = *p; }

int or_set_open_bnd(or_engine* e, const fe_open_bnd* b) {
  e->B = *b;
  e->open_bnd = true;
  e->inlet.assign(b->inlet, b->inlet + b->n_inlet);
  e->outlet.assign(b->outlet, b->outlet + b->n_outlet);
  if (b->inlet_coord) e->inlet_coord.assign(b->inlet_coord, b->inlet_coord + b->n_inlet);
  else e->inlet_coord.clear();
  if (b->n_buf) {
    e->buf_verts.assign(b->buf_verts, b->buf_verts + b->n_buf);
    e->buf_refs.assign(b->buf_refs, b->buf_refs + b->n_buf);
  }
  // is_processed mask (multiphase_gpu.cuh:378-389)
  e->bcproc.assign(e->n, 0);
  if (b->use_in_vel || b->use_in_prs || b->use_in_fluid)
    for (int32_t i : e->inlet) e->bcproc[i] = 1;
  if (b->use_out_prs || b->use_out_fluid)
    for (int32_t i : e->outlet) e->bcproc[i] = 1;
  if (b->copy_to_buffers)
    for (int32_t i : e->buf_verts) e->bcproc[i] = 1;
  return 0;
}

void or_upload(or_engine* e, const double* h, const double* g) {
  std::copy(h, h + Q * e->n, e->h.begin());
  std::copy(g, g + Q * e->n, e->g.begin());
}
void or_download(const or_engine* e, double* h, double* g) {
  std::copy(e->h.begin(), e->h.end(), h);
  std::copy(e->g.begin(), e->g.end(), g);
}
void or_set_forcing_factor(or_engine* e, double ff) { e->forcing_factor = ff; }

// MultiPhaseGPU::step (multiphase_gpu.cuh:522-631), fuse_collision path
void or_step(or_engine* e) {
  compute_fields(e, true);
  apply_open_bnd(e);
  collide(e);
  stream(e);
}

// apply_mass_correction (multiphase_gpu.cuh:689-700) with k_inject_mass
// (device_engine.cuh:1128-1139)
double or_apply_mass_correction(or_engine* e) {
  if (!e->P.correct_op_mass) return 0.0;
  double M, Wt;
  mass_weight(e, M, Wt);
  const double drift = M - e->target_mass;
  if (Wt > 0.0 && drift != 0.0) {
    const double lambda = drift / Wt;
    const int64_t n = e->n;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < n; ++i) {
      double c = 0.0;
      for (int k = 0; k < Q; ++k) c += e->h[k * n + i];
      const double phi = c * (1.0 - c);
      if (phi <= 0.0) continue;
      const double delta_c = -lambda * phi;
      for (int k = 0; k < Q; ++k) e->h[k * n + i] += W(k) * delta_c;
    }
  }
  return drift;
}

void or_record_target_mass(or_engine* e) { double M, Wt; mass_weight(e, M, Wt); e->target_mass = M; }
double or_target_mass(const or_engine* e) { return e->target_mass; }
void or_set_target_mass(or_engine* e, double m0) { e->target_mass = m0; }
double or_current_mass(or_engine* e) { double M, Wt; mass_weight(e, M, Wt); return M; }

void or_fields(const or_engine* e, const fe_fields* f) {
  const int64_t n = e->n;
  auto put = [&](double* dst, const std::vector<double>& v) { if (dst) std::copy(v.begin(), v.begin() + n, dst); };
  put(f->rho, e->rho); put(f->c, e->c); put(f->ux, e->ux); put(f->uy, e->uy);
  put(f->uz, e->uz); put(f->p, e->p); put(f->mu, e->mu);
}

// download_raw (multiphase_gpu.cuh:731-757): moments, BC fields, grad_cd(c),
// laplacian(c), mu axpy, velocity/pressure correction.
void or_download_fields(or_engine* e, const fe_fields* f) {
  compute_fields(e, false);
  or_fields(e, f);
}

// k_flow_stats (device_engine.cuh:660-683) over the current fields
void or_flow_stats(const or_engine* e, double out[6]) {
  double sx = 0, sy = 0, sz = 0, s2 = 0, sc = 0, mx = 0;
  for (int64_t i = 0; i < e->n; ++i) {
    const double vx = e->ux[i], vy = e->uy[i], vz = e->uz[i], v2 = vx * vx + vy * vy + vz * vz;
    sx += vx; sy += vy; sz += vz; s2 += v2; sc += e->c[i];
    if (v2 > mx) mx = v2;
  }
  out[0] = sx; out[1] = sy; out[2] = sz; out[3] = s2; out[4] = sc; out[5] = mx;
}

void or_inplace_counts(const or_engine* e, int64_t out[3]) {
  if (!e->inplace) { out[0] = out[1] = out[2] = -1; return; }
  out[0] = e->n_swap; out[1] = e->n_avg; out[2] = e->n_zero;
}

int64_t or_inplace_program(const or_engine* e, int32_t* a, int32_t* b, uint8_t* t) {
  if (!e->inplace) return -1;
  for (size_t q = 0; q < e->op_a.size(); ++q) {
    if (a) a[q] = (int32_t)e->op_a[q];
    if (b) b[q] = (int32_t)e->op_b[q];
    if (t) t[q] = e->op_t[q];
  }
  return (int64_t)e->op_a.size();
}

void or_table(const or_engine* e, int which, int32_t* out) {
  const std::vector<int32_t>* t[] = {&e->cdm, &e->cdp, &e->bcase, &e->bc1, &e->bc2,
                                     &e->lcase, &e->lc1, &e->lc2, &e->avgnext, &e->src};
  if (which < 0 || which > 9) return;
  std::copy(t[which]->begin(), t[which]->end(), out);
}

// forcing_factor_at (felbm_gpu_main.cu:587-594)
static double forcing_factor_at(const fe_params& P, int64_t t) {
  const double PI = 3.14159265358979323846;
  if (P.forcing_timedep == FE_FORCING_SINUSOIDAL) return std::sin(2.0 * PI * double(t) / P.forcing_period);
  if (P.forcing_timedep == FE_FORCING_SQUARE) {
    const double x = std::sin(2.0 * PI * double(t) / P.forcing_period);
    return (x < 0) ? -1.0 : ((x > 0) ? 1.0 : 0.0);
  }
  return 1.0;
}

// the driver's hot loop body (felbm_gpu_main.cu:741-745)
void or_run(or_engine* e, int nsteps, int64_t t0) {
  for (int s = 0; s < nsteps; ++s) {
    e->forcing_factor = forcing_factor_at(e->P, t0 + s);
    or_step(e);
    or_apply_mass_correction(e);
  }
}

int or_threads(void) { return omp_get_max_threads(); }
void or_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
}

void or_mrt_matrices(double* M, double* Minv) {
  double A[Q][Q], B[Q][Q];
  build_mrt(A, B);
  for (int j = 0; j < Q; ++j)
    for (int k = 0; k < Q; ++k) { M[j * Q + k] = A[j][k]; Minv[j * Q + k] = B[j][k]; }
}

}  // extern "C"
