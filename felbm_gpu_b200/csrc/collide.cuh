// P4: fused equilibria + Guo force + BGK/MRT collision of the Lee–Liu step,
// push-streamed (reference k_collide_fused_mrt, device_engine.cuh:547-651, and
// k_collide_fused_bgk, :459-545, with cd_dir_val / bd_dir_val / avg_dir_val,
// :89-113, evaluated from shared-memory tiles, and the open-boundary overwrite
// of g, k_open_bnd / k_open_bnd_buf, :761-798,826-846, folded in).
//
// Arithmetic layout (same algebra as the reference, reordered):
//  * directions are processed in opposite pairs (k, k+1), e_{k+1} = -e_k: the
//    neighbour values are loaded once per pair, the central-difference value is
//    exactly antisymmetric (cd_{k+1} = -cd_k), and G_k, G_{k+1} share all
//    terms but +-alpha w u.e_k;
//  * a pre-pass over the pairs evaluates the near-wall cases once, sums the
//    four gradients (central / biased, of c and p) and keeps the six
//    per-pair derivative values in a per-thread shared-memory stash; then all
//    site scalars are known and the main pass stores h_k at once;
//  * the MRT transform uses the row parity of the moment basis: even rows see
//    x_k + x_{k+1}, odd rows x_k - x_{k+1}, and the back transform gives the
//    pair as E +- O; only g + force_g (19 values) and the 15 relaxed moments
//    stay live until the g stores.
#pragma once
#include <type_traits>

#include "kernels.cuh"

namespace fe {

// Resident CTAs per SM: FP32 arithmetic fits 128 registers a thread, FP64
// needs the full budget of 255.
template <class S>
struct CollideMinBlocks {
  static constexpr int value = 65536 / ((sizeof(typename S::real) == 8 ? 256 : 128) * P4T);
};

constexpr int NPAIR = (Q - 1) / 2;   // 9 opposite pairs
constexpr int NSTASH = 6 * NPAIR;    // stashed values per thread

// Dynamic shared memory of the collide pass: site indices, c / p / lap(mu)
// tiles (halo 2) and the per-thread derivative stash.
template <class Sh, class R>
struct CollideSmem {
  using T = Tile<Sh, 2>;
  static constexpr int NT16 = (T::N * 4 + 15) & ~15;
  static constexpr int NTR = (T::N * (int)sizeof(R) + 15) & ~15;
  static constexpr int STASH = NSTASH * P4T * (int)sizeof(R);
  static constexpr int BYTES = NT16 + 3 * NTR + STASH;
};

// Per-site scalars shared by every direction of the collision.
template <class R>
struct SiteScal {
  R c, p, mu, rho_cs2, c_over, drho_cs2, mob;
  R gu2;                  // gamma |u|^2
  R u_force_g, u_drho;    // u.e_fg, drho cs2 u.grad_cd c
  R S_h, u_fg_f, u_drm;   // gradient-dependent terms of h and force_g
};

// One direction: h_k, and x_k = eq_g,k - g_k, Z_k = g_k + force_g,k. The MRT
// equilibrium of g carries +(mu dc_k + f_proj) G / 2 where the BGK one carries
// -(...) (device_engine.cuh:517 vs :598).
template <class R, int MRT>
__device__ __forceinline__ void dir_terms(const SiteScal<R>& q, R w, R uk, R fproj, R cdc, R cdp, R bdc, R bdp,
                                          R avg, R gk, R& h, R& x, R& Z) {
  const R u_term = uk * (R(ALPHA) + R(BETA) * uk) - q.gu2;
  const R G = w * (R(1) + u_term);
  const R wut = G - w;
  const R dc = R(0.5) * (cdc + bdc), dp = R(0.5) * (cdp + bdp);
  const R ffk = q.mu * dc + fproj;
  // eq_h + force_h (device_engine.cuh:596,608)
  h = G * (q.c + R(0.5) * (-cdc + q.c_over * (cdp - q.mu * cdc - fproj)) + (dc - q.c_over * (dp - ffk)) +
           q.mob * avg + q.S_h);
  // eq_g (:597-598) and g + force_g (:609)
  const R mcf = MRT ? q.mu * cdc + fproj : -(q.mu * cdc + fproj);
  const R eg = w * q.p + q.rho_cs2 * wut + R(0.5) * ((q.u_drho - q.drho_cs2 * cdc) * wut + (q.u_force_g + mcf) * G);
  x = eg - gk;
  Z = gk + (q.drho_cs2 * dc - q.u_drm) * wut + (ffk - q.u_fg_f) * G;
}

template <class S, class Sh, int MRT, bool HBB, bool WIDE>
__global__ void __launch_bounds__(P4T, CollideMinBlocks<S>::value)
    k_collide(const LatDesc* __restrict__ descs, const int2* __restrict__ work, int parity) {
  using R = typename S::real;
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  using F = typename S::fld;
  using T = Tile<Sh, 2>;
  using SM = CollideSmem<Sh, R>;
  // population offsets: 32-bit while the lattice's arrays stay below 2^32
  // entries (the host picks WIDE otherwise)
  using IX = typename std::conditional<WIDE, int64_t, uint32_t>::type;
  __shared__ Head<Sh> s;
  extern __shared__ __align__(16) unsigned char dsm[];
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);
  R* s_c = reinterpret_cast<R*>(dsm + SM::NT16);
  R* s_p = reinterpret_cast<R*>(dsm + SM::NT16 + SM::NTR);
  R* s_l = reinterpret_cast<R*>(dsm + SM::NT16 + 2 * SM::NTR);
  R* s_st = reinterpret_cast<R*>(dsm + SM::NT16 + 3 * SM::NTR) + threadIdx.x;  // [v * P4T]
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int brick = wk.y;
  load_brick<Sh, 2, P4T>(D, brick, s, s_idx);
  {
    const F* const src[3] = {static_cast<const F*>(D.c), static_cast<const F*>(D.p),
                             static_cast<const F*>(D.lapmu)};
    R* const dst[3] = {s_c, s_p, s_l};
    stage<Sh, 2, 3, P4T>(src, dst, true, s.lambda, s_idx);
  }
  __syncthreads();

  const DevPrm& Pm = D.prm;
  const R cs2 = R(CS2), alpha = R(ALPHA);
  const R rho1 = (R)Pm.rho1, drho = (R)Pm.drho;
  // per-lattice reciprocals once per brick: the site formulas multiply
  const R itau0 = (R)(1.0 / Pm.tau0), itau1 = (R)(1.0 / Pm.tau1), ffac = (R)s.ff;
  const R gxa = (R)Pm.gx, gya = (R)Pm.gy, gza = (R)Pm.gz;
  const R fxa = (R)Pm.fx * ffac, fya = (R)Pm.fy * ffac, fza = (R)Pm.fz * ffac;
  const PG* __restrict__ gin = static_cast<const PG*>(D.pop[parity][1]);
  PH* __restrict__ hout = static_cast<PH*>(D.pop[parity ^ 1][0]);
  PG* __restrict__ gout = static_cast<PG*>(D.pop[parity ^ 1][1]);
  const F* __restrict__ fmu = static_cast<const F*>(D.mu);
  const Shift shh{(float)Pm.c_ref, (float)(1.0 / Pm.h_scale), (float)Pm.h_scale};
  const Shift shg{(float)Pm.p_ref, (float)(1.0 / Pm.g_scale), (float)Pm.g_scale};
  double st[6] = {0, 0, 0, 0, 0, 0};
  int bad = 0;
  const int first = s.first, cnt = s.cnt;

  for (int r = threadIdx.x; r < cnt; r += P4T) {
    const int64_t i = first + r;
    const int pos = T::pos(s.slot_of[r]);
    SiteScal<R> q;
    q.c = s_c[pos];
    q.p = s_p[pos];
    const R lmu = s_l[pos];
    q.mu = (R)fmu[i];
    const uint8_t flag = Pm.open_bnd ? D.bcflag[i] : 0;
    // post-stream g of the site (what P1 read)
    const IX a0 = (IX)pbase(i);
    R g[Q];
#pragma unroll
    for (int k = 0; k < Q; ++k) g[k] = ld_pop<GV<S>>(gin, a0 + k * AOSOA, k, shg);
    // push target of direction k: slot k of x + e_k, or slot opp(k) of x
    // (halfway bounce-back) when x + e_k is solid
    auto dst = [&](int k) -> IX {
      const int dn = s_idx[pos + T::off(k)];
      return dn >= 0 ? (IX)(dn >> 5) * (IX)(Q * AOSOA) + (IX)(k * AOSOA + (dn & (AOSOA - 1)))
                     : a0 + (IX)(lat_opp(k) * AOSOA);
    };
    // ---- pre-pass: near-wall cases once, the four gradients, stash -----------
    R ecx = 0, ecy = 0, ecz = 0, epx = 0, epy = 0, epz = 0;
    R bcx = 0, bcy = 0, bcz = 0, bpx = 0, bpy = 0, bpz = 0;
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      const int o = T::off(k), v = 6 * (k >> 1);
      const R cm = s_c[pos - o], cp = s_c[pos + o], cm2 = s_c[pos - 2 * o], cp2 = s_c[pos + 2 * o];
      const R pm = s_p[pos - o], pp = s_p[pos + o], pm2 = s_p[pos - 2 * o], pp2 = s_p[pos + 2 * o];
      R cdc, cdp, bca, bcb, bpa, bpb;
      pair_derivs<HBB>(q.c, cm, cp, cm2, cp2, q.p, pm, pp, pm2, pp2, cdc, cdp, bca, bcb, bpa, bpb);
      s_st[(v + 0) * P4T] = cdc;
      s_st[(v + 1) * P4T] = cdp;
      s_st[(v + 2) * P4T] = bca;
      s_st[(v + 3) * P4T] = bcb;
      s_st[(v + 4) * P4T] = bpa;
      s_st[(v + 5) * P4T] = bpb;
      // pairs: central terms count twice, biased ones as a difference
      const R aw = alpha * weight<R>(k);
      const R dbc = bca - bcb, dbp = bpa - bpb;
      if (lat_cx(k)) {
        const R e = aw * R(lat_cx(k));
        ecx += R(2) * e * cdc; epx += R(2) * e * cdp; bcx += e * dbc; bpx += e * dbp;
      }
      if (lat_cy(k)) {
        const R e = aw * R(lat_cy(k));
        ecy += R(2) * e * cdc; epy += R(2) * e * cdp; bcy += e * dbc; bpy += e * dbp;
      }
      if (lat_cz(k)) {
        const R e = aw * R(lat_cz(k));
        ecz += R(2) * e * cdc; epz += R(2) * e * cdp; bcz += e * dbc; bpz += e * dbp;
      }
    }
    const R rho = rho1 + drho * q.c;
    const R irho = R(1) / rho;
    const R cm_ = (flag & BC_SITE) ? (R) static_cast<const F*>(D.c_raw_bc)[i] : q.c;
    // relaxation rate (reference k_moments :130-132)
    const R cpc = cm_ < R(0) ? R(0) : (cm_ > R(1) ? R(1) : cm_);
    // 1/tau = cpc/tau0 + (1-cpc)/tau1; s0 = 1/(tau + 1/2) = itau / (1 + itau/2)
    const R itau = cpc * itau0 + (R(1) - cpc) * itau1;
    const R s0 = itau / (R(1) + R(0.5) * itau);
    // corrected velocity (k_moments + k_vel_press_corr)
    R ux, uy, uz;
    if (flag & BC_SITE) {
      const F* ubc = static_cast<const F*>(D.u_bc);
      ux = (R)ubc[i]; uy = (R)ubc[D.n + i]; uz = (R)ubc[2 * D.n + i];
    } else {
      R jx = 0, jy = 0, jz = 0;
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        if (lat_cx(k)) jx += R(lat_cx(k)) * g[k];
        if (lat_cy(k)) jy += R(lat_cy(k)) * g[k];
        if (lat_cz(k)) jz += R(lat_cz(k)) * g[k];
      }
      const R inv = irho * R(1.0 / CS2);
      const R mor = q.mu * irho;
      ux = jx * inv + R(0.5) * (gxa + fxa * irho + mor * ecx);
      uy = jy * inv + R(0.5) * (gya + fya * irho + mor * ecy);
      uz = jz * inv + R(0.5) * (gza + fza * irho + mor * ecz);
    }
    // open-boundary overwrite of g by the plain equilibrium (apply_open_bnd)
    if (flag & BC_G_OVER) {
      const int64_t sb = D.bcsrc[i];
      const F* ubc = static_cast<const F*>(D.u_bc);
      const R bux = (R)ubc[sb], buy = (R)ubc[D.n + sb], buz = (R)ubc[2 * D.n + sb];
      const R bp = (R) static_cast<const F*>(D.p)[sb];
      const R brho = rho1 + drho * (R) static_cast<const F*>(D.c)[sb];
      const R bu_sq = bux * bux + buy * buy + buz * buz;
#pragma unroll
      for (int k = 0; k < Q; ++k) {
        const R uk = bux * R(lat_cx(k)) + buy * R(lat_cy(k)) + buz * R(lat_cz(k));
        const R u_term = uk * (alpha + R(BETA) * uk) - R(GAMMA) * bu_sq;
        g[k] = weight<R>(k) * (bp + brho * cs2 * u_term);
      }
    }
    // site scalars (device_engine.cuh:563-583)
    q.rho_cs2 = rho * cs2;
    q.c_over = q.c * irho * R(1.0 / CS2);
    q.drho_cs2 = drho * cs2;
    q.mob = (R)Pm.mobility;
    const R bfx = rho * gxa + fxa, bfy = rho * gya + fya, bfz = rho * gza + fza;
    const R u2 = ux * ux + uy * uy + uz * uz;
    q.gu2 = R(GAMMA) * u2;
    const R efgx = q.mu * ecx + bfx, efgy = q.mu * ecy + bfy, efgz = q.mu * ecz + bfz;
    const R efhx = ecx - q.c_over * (epx - efgx), efhy = ecy - q.c_over * (epy - efgy),
            efhz = ecz - q.c_over * (epz - efgz);
    const R fdcx = R(0.5) * (ecx + bcx), fdcy = R(0.5) * (ecy + bcy), fdcz = R(0.5) * (ecz + bcz);
    const R fdpx = R(0.5) * (epx + bpx), fdpy = R(0.5) * (epy + bpy), fdpz = R(0.5) * (epz + bpz);
    const R ffgx = q.mu * fdcx + bfx, ffgy = q.mu * fdcy + bfy, ffgz = q.mu * fdcz + bfz;
    const R ffhx = fdcx - q.c_over * (fdpx - ffgx), ffhy = fdcy - q.c_over * (fdpy - ffgy),
            ffhz = fdcz - q.c_over * (fdpz - ffgz);
    q.u_force_g = ux * efgx + uy * efgy + uz * efgz;
    q.u_drho = q.drho_cs2 * (ux * ecx + uy * ecy + uz * ecz);
    q.S_h = R(0.5) * (ux * efhx + uy * efhy + uz * efhz) - (ux * ffhx + uy * ffhy + uz * ffhz);
    q.u_fg_f = ux * ffgx + uy * ffgy + uz * ffgz;
    q.u_drm = q.drho_cs2 * (ux * fdcx + uy * fdcy + uz * fdcz);
    st[0] += (double)ux; st[1] += (double)uy; st[2] += (double)uz; st[3] += (double)u2; st[4] += (double)q.c;
    st[5] = fmax(st[5], (double)u2);
    bad |= !(u2 < R(1e30));

    // ---- main pass over the pairs ------------------------------------------
    R Z[Q], mom[Q];
#pragma unroll
    for (int j = 0; j < Q; ++j) mom[j] = R(0);
    {  // rest direction: no derivatives, avg = lap(mu) of the site
      R h0, x0;
      dir_terms<R, MRT>(q, weight<R>(0), R(0), R(0), R(0), R(0), R(0), R(0), lmu, g[0], h0, x0, Z[0]);
      st_pop<HV<S>>(hout, a0, 0, h0, shh);
      if (MRT) {
#pragma unroll
        for (int j = 0; j < Q; ++j)
          if (mrt_kind(j) != MK_CONS && mrt_M(j, 0) != 0) mom[j] += R(mrt_M(j, 0)) * x0;
      } else {
        st_pop<GV<S>>(gout, a0, 0, Z[0] + s0 * x0, shg);
      }
    }
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      const int o = T::off(k), v = 6 * (k >> 1);
      const R cdc = s_st[(v + 0) * P4T], cdp = s_st[(v + 1) * P4T];
      const R bca = s_st[(v + 2) * P4T], bcb = s_st[(v + 3) * P4T];
      const R bpa = s_st[(v + 4) * P4T], bpb = s_st[(v + 5) * P4T];
      const R lm = s_l[pos - o], lp = s_l[pos + o];
      const R avg_a = is_site(lp) ? R(0.5) * (lmu + lp) : lmu;
      const R avg_b = is_site(lm) ? R(0.5) * (lmu + lm) : lmu;
      const R w = weight<R>(k);
      const R uk = ux * R(lat_cx(k)) + uy * R(lat_cy(k)) + uz * R(lat_cz(k));
      const R fproj = bfx * R(lat_cx(k)) + bfy * R(lat_cy(k)) + bfz * R(lat_cz(k));
      R ha, hb, xa, xb;
      dir_terms<R, MRT>(q, w, uk, fproj, cdc, cdp, bca, bpa, avg_a, g[k], ha, xa, Z[k]);
      dir_terms<R, MRT>(q, w, -uk, -fproj, -cdc, -cdp, bcb, bpb, avg_b, g[k + 1], hb, xb, Z[k + 1]);
      st_pop<HV<S>>(hout, dst(k), k, ha, shh);
      st_pop<HV<S>>(hout, dst(k + 1), k + 1, hb, shh);
      if (MRT) {
        const R sx = xa + xb, dx = xa - xb;
#pragma unroll
        for (int j = 0; j < Q; ++j) {
          if (mrt_kind(j) == MK_CONS) continue;
          const int mjk = mrt_M(j, k);
          const bool odd = (j == 4 || j == 6 || j == 8 || j >= 16);
          const R vv = odd ? dx : sx;
          if (mjk == 1) mom[j] += vv;
          else if (mjk == -1) mom[j] -= vv;
          else if (mjk != 0) mom[j] += R(mjk) * vv;
        }
      } else {
        st_pop<GV<S>>(gout, dst(k), k, Z[k] + s0 * xa, shg);
        st_pop<GV<S>>(gout, dst(k + 1), k + 1, Z[k + 1] + s0 * xb, shg);
      }
    }
    if (MRT) {
      // rates (reference device_engine.cuh:623-625, with per-kind modes)
      // s1 = 2 tau / (2 Lambda + tau) with tau = 1 / s0 - 1/2 = 1 / itau
      const R s1 = R(2) / (R(2) * (R)Pm.mrt_lambda * itau + R(1));
      R srate[7];
#pragma unroll
      for (int k = 0; k < 7; ++k)
        srate[k] = Pm.rate_mode[k] == RATE_S0 ? s0 : (Pm.rate_mode[k] == RATE_MAGIC ? s1 : (R)Pm.rate_value[k]);
#pragma unroll
      for (int j = 0; j < Q; ++j)
        if (mrt_kind(j) != MK_CONS) mom[j] *= srate[mrt_kind(j)] * (R(1) / R(mrt_norm2(j)));
      R back0 = 0;
#pragma unroll
      for (int j = 0; j < Q; ++j)
        if (mrt_kind(j) != MK_CONS && mrt_M(j, 0) != 0) back0 += R(mrt_M(j, 0)) * mom[j];
      st_pop<GV<S>>(gout, a0, 0, Z[0] + back0, shg);
#pragma unroll
      for (int k = 1; k < Q; k += 2) {
        R E = 0, O = 0;
#pragma unroll
        for (int j = 0; j < Q; ++j) {
          if (mrt_kind(j) == MK_CONS) continue;
          const int mjk = mrt_M(j, k);
          const bool odd = (j == 4 || j == 6 || j == 8 || j >= 16);
          R& acc = odd ? O : E;
          if (mjk == 1) acc += mom[j];
          else if (mjk == -1) acc -= mom[j];
          else if (mjk != 0) acc += R(mjk) * mom[j];
        }
        st_pop<GV<S>>(gout, dst(k), k, Z[k] + (E + O), shg);
        st_pop<GV<S>>(gout, dst(k + 1), k + 1, Z[k + 1] + (E - O), shg);
      }
    }
  }
  // flow-statistics partials per warp (reference k_flow_stats :660-683, summed
  // on demand), no block barrier
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int qv = 0; qv < 6; ++qv) {
    double x = st[qv];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      const double y = __shfl_down_sync(0xffffffffu, x, o);
      x = (qv == 5) ? fmax(x, y) : x + y;
    }
    st[qv] = x;
  }
  bad = __any_sync(0xffffffffu, bad);
  if (lane == 0) {
    double* part = D.part4 + ((int64_t)brick * P4W + wid) * 6;
#pragma unroll
    for (int qv = 0; qv < 6; ++qv) part[qv] = st[qv];
    if (bad) atomicOr(&D.ctl->status, 1);
    // the last warp of the launch (per lattice) advances the step counter and
    // queues the next mass correction; it reads nothing the other warps wrote
    // (the partials are summed by a later launch), so no fence precedes the
    // count
    if (atomicAdd(&D.ctl->count4, 1u) == (unsigned)(D.nbricks * P4W) - 1u) {
      Ctl* C = D.ctl;
      C->t += 1;
      if (Pm.open_bnd) C->open_step += 1;
      C->pending = (C->auto_correct && Pm.correct_mass) ? 1 : 0;
      C->lambda = 0.0;
      C->count4 = 0;
    }
  }
}

}  // namespace fe
