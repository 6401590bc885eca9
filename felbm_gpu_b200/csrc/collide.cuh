// P4: fused equilibria + Guo force + BGK/MRT collision of the Lee–Liu step,
// push-streamed (reference k_collide_fused_mrt, device_engine.cuh:547-651, and
// k_collide_fused_bgk, :459-545, with cd_dir_val / bd_dir_val / avg_dir_val,
// :89-113, evaluated from shared-memory tiles, and the open-boundary overwrite
// of g, k_open_bnd / k_open_bnd_buf, :761-798,826-846, folded in).
//
// Arithmetic layout (same algebra as the reference, regrouped):
//  * the work comes in twins, done two lanes at a time (V2: one f32x2
//    instruction for both lanes in FP32): the pre-pass evaluates the stencils
//    of c and p together, the main pass the two directions of an opposite
//    pair (k, k+1), e_{k+1} = -e_k;
//  * within a pair every quantity is even or odd in e: odd ones (u.e, F.e,
//    the central difference, exactly antisymmetric) enter as (v, -v), so the
//    pair needs each of them once;
//  * the central differences cancel from eq_h + force_h: with
//    dc = (cd + bd) / 2 and ffk = mu dc + F.e, the bracket of h_k reduces to
//    c + S_h + mob avg + (1 + c_o mu) bd_c / 2 - c_o bd_p / 2 + c_o F.e / 2
//    (c_o = c / (rho cs^2)); eq_g splits the same way (see the main pass);
//  * a pre-pass over the pairs evaluates the near-wall cases once, sums the
//    four gradients (central / biased, of c and p) and keeps the five
//    per-pair values the main pass needs (cd_c, bd_c and bd_p of both
//    directions) in a per-thread shared-memory stash;
//  * the MRT transform (MRT == 1) uses the row parity of the moment basis:
//    even rows see x_k + x_{k+1}, odd rows x_k - x_{k+1}, and the back
//    transform gives the pair as E +- O; only g + force_g (19 values) and the
//    15 relaxed moments stay live until the g stores;
//  * with one rate s_e for every even non-conserved moment and one rate s_o
//    for every odd one (the reference's own assignment, device_engine.cuh:625),
//    M^-1 S M is exact in closed form (MRT == 2): the even rows with rho span
//    the even subspace and the odd rows with j the odd one, so the collision
//    adds s_e (x+ - sum(x) / 19) + s_o (x- - e.J / 10), x+- = (x_k +- x_{k+1})
//    / 2 and J = sum_k e_k x_k; the 19x15 transforms become two sums.
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

constexpr int NPAIR = (Q - 1) / 2;  // 9 opposite pairs

// Dynamic shared memory of the collide pass (each region 128-byte aligned,
// the alignment of a TMA destination): the halo-1 tile of push targets, the
// (c', p') pair tile and the lap(mu) tile (halo 2), and the per-thread stash
// (two pairs and one scalar per opposite pair).
template <class S, class Sh>
struct CollideSmem {
  using R = typename S::real;
  using F = typename S::fld;
  using T = Tile<Sh, 2>;
  using T1 = Tile<Sh, 1>;
  static_assert(sizeof(R) == sizeof(F), "the pair tile is copied as stored");
  static constexpr int al(int b) { return (b + 127) & ~127; }
  static constexpr int IDX = al(T1::N * 4);
  static constexpr int CP = al(T::N * (int)sizeof(V2<R>));
  static constexpr int LT = al(T::N * (int)sizeof(F));
  static constexpr int STV = 2 * NPAIR * P4T * (int)sizeof(V2<R>);
  static constexpr int STS = NPAIR * P4T * (int)sizeof(R);
  static constexpr int OFF_CP = IDX, OFF_L = OFF_CP + CP, OFF_ST = OFF_L + LT;
  static constexpr int BYTES = OFF_ST + al(STV + STS);
};

// Per-site scalars shared by every direction of the collision.
template <class R>
struct SiteScal {
  R mu, gu2, mob;
  R C0;            // c + S_h
  R hk1, hco;      // (1 + c_o mu) / 2, c_o / 2
  R A1, A2;        // eq_g: w A1 + A2 w u_term (even part)
  R hdr, u_drm, u_fg_f, drho_cs2;
};

// AAP: 0 two population buffers; 1, 2 the in-place layout from phase 0
// (reads the own slots, writes f*_k into the own slot opp(k)) and from phase
// 1 (reads f_k where the last step left it, pushes like the two-buffer pass).
// MRT_: 0 BGK, 1 general MRT, 2 two-rate MRT, 3 two-rate MRT of a lattice
// without density contrast (rho0 = rho1: the drho terms are zero and dropped;
// the same results bit for bit).
template <class S, class Sh, int MRT_, bool HBB, bool WIDE, int AAP = 0>
__global__ void __launch_bounds__(P4T, CollideMinBlocks<S>::value)
    k_collide(const LatDesc* __restrict__ descs, const int2* __restrict__ work, int parity) {
  constexpr int MRT = MRT_ == 3 ? 2 : MRT_;
  constexpr bool NODRHO = MRT_ == 3;
  static_assert(AAP == 0 || !WIDE, "the in-place layout takes 32-bit population offsets");
  using R = typename S::real;
  using V = V2<R>;
  using PH = typename S::hpop;
  using PG = typename S::gpop;
  using F = typename S::fld;
  using T = Tile<Sh, 2>;
  using T1 = Tile<Sh, 1>;
  using SM = CollideSmem<S, Sh>;
  // population offsets: 32-bit while the lattice's arrays stay below 2^32
  // entries (the host picks WIDE otherwise)
  using IX = typename std::conditional<WIDE, int64_t, uint32_t>::type;
  // keep the 32-bit push targets of the h stores for the g stores of the
  // moment forms (the in-place layout's own-slot targets are one add)
  constexpr bool KEEP_DST = MRT != 0 && !WIDE && AAP != 1;
  __shared__ Head<Sh> s;
  __shared__ uint64_t s_bar;
  extern __shared__ __align__(128) unsigned char dsm[];
  int32_t* s_idx = reinterpret_cast<int32_t*>(dsm);  // halo-1 tile
  V* s_cp = reinterpret_cast<V*>(dsm + SM::OFF_CP);
  F* s_l = reinterpret_cast<F*>(dsm + SM::OFF_L);
  V* s_sv = reinterpret_cast<V*>(dsm + SM::OFF_ST) + threadIdx.x;                  // [(2 pr + j) P4T]
  R* s_sc = reinterpret_cast<R*>(dsm + SM::OFF_ST + SM::STV) + threadIdx.x;         // [pr P4T]
  const int2 wk = work[blockIdx.x];
  const LatDesc& D = descs[wk.x];
  const int brick = wk.y;
  // the copy engine writes 128-byte aligned boxes
  if (smem_u32(dsm) & 127u) {
    if (threadIdx.x == 0) atomicOr(&D.ctl->status, 8);
    return;
  }
  // prologue: the brick's slot list, its halo-1 tile of push targets and the
  // (c', p') and lap(mu) tiles (halo 2) by copy engine, on one barrier; P2
  // wrote the pairs with the queued mass correction applied, so the tiles
  // are used as they land
  head_init(&s_bar);
  if (threadIdx.x == 0) {
    head_begin<Sh>(D, brick, s, &s_bar, (uint32_t)(T::N * (sizeof(V) + sizeof(F)) + T1::N * 4));
    tile_copy<Sh, 2, (int)sizeof(V) / 8>(s_cp, D, TM_CP2, s.bx, s.by, s.bz, &s_bar);
    tile_copy<Sh, 2>(s_l, D, TM_L2, s.bx, s.by, s.bz, &s_bar);
    bulk_g2s(s_idx, D.tile1 + (int64_t)brick * T1::N, (uint32_t)(T1::N * 4), &s_bar);
  }
  if (threadIdx.x == P4T - 1) load_step_scalars(D, s);
  // the brick's own g blocks (its sites are one contiguous AoSoA range) into
  // L2 while the tiles land, so the per-site g loads below hit L2
  if constexpr (AAP != 2) {
    if (threadIdx.x >= 32 && threadIdx.x < 64) {
      const int first = __ldg(&D.rec[brick].first), cnt = __ldg(&D.rec[brick].cnt);
      const PG* gsrc = static_cast<const PG*>(D.pop[parity][1]);
      for (int64_t b = (first >> 5) + (threadIdx.x - 32); b <= (int64_t)((first + cnt - 1) >> 5); b += 32)
        bulk_prefetch_l2(gsrc + b * (Q * AOSOA), (uint32_t)(Q * AOSOA * sizeof(PG)));
    }
  }
  if (!head_wait(D, &s_bar)) return;

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
    const int slot = s.slot_of[r];
    const int pos = T::pos(slot), pos1 = T1::pos(slot);
    const V cp0 = s_cp[pos];
    const R c = cp0.x(), p = cp0.y();
    const R lmu = (R)s_l[pos];
    SiteScal<R> q;
    q.mu = (R)fmu[grid_entry<Sh>(D, s.bx, s.by, s.bz, slot)];
    const uint8_t flag = Pm.open_bnd ? D.bcflag[i] : 0;
    // post-stream g of the site (what P1 read), the pairs (k, k+1) together
    const IX a0 = (IX)pbase(i);
    R g0 = ld_pop<GV<S>>(gin, a0, 0, shg);
    V gp[NPAIR];
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      if constexpr (AAP == 2)
        gp[k >> 1] = V(ld_pop<GV<S>>(gin, aa_src<T1>(s_idx, pos1, (uint32_t)a0, k), k, shg),
                       ld_pop<GV<S>>(gin, aa_src<T1>(s_idx, pos1, (uint32_t)a0, k + 1), k + 1, shg));
      else
        gp[k >> 1] = V(ld_pop<GV<S>>(gin, a0 + k * AOSOA, k, shg), ld_pop<GV<S>>(gin, a0 + (k + 1) * AOSOA, k + 1, shg));
    }
    // push target of direction k: slot k of x + e_k, or slot opp(k) of x
    // (halfway bounce-back) when x + e_k is solid
    auto dst = [&](int k) -> IX {
      if constexpr (AAP == 1) {
        return a0 + (IX)(lat_opp(k) * AOSOA);
      } else if constexpr (WIDE) {
        const int dn = s_idx[pos1 + T1::off(k)];
        return dn >= 0 ? (IX)(dn >> 5) * (IX)(Q * AOSOA) + (IX)(k * AOSOA + (dn & (AOSOA - 1)))
                       : a0 + (IX)(lat_opp(k) * AOSOA);
      } else {
        const uint32_t b = (uint32_t)s_idx[pos1 + T1::off(k)];
        return b != 0xffffffffu ? b + (uint32_t)(k * AOSOA) : a0 + (uint32_t)(lat_opp(k) * AOSOA);
      }
    };
    // ---- pre-pass: near-wall cases once, the four gradients, stash -----------
    // lanes (c, p): ec central sums, eb biased sums, per axis
    V ec[3] = {V(R(0)), V(R(0)), V(R(0))}, eb[3] = {V(R(0)), V(R(0)), V(R(0))};
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      const int o = T::off(k), pr = k >> 1;
      const V fm = s_cp[pos - o], fp = s_cp[pos + o], fm2 = s_cp[pos - 2 * o], fp2 = s_cp[pos + 2 * o];
      V cd, ba, bb;
      pair_derivs2<HBB>(cp0, fm, fp, fm2, fp2, cd, ba, bb);
      s_sc[pr * P4T] = cd.x();
      s_sv[(2 * pr) * P4T] = V(ba.x(), bb.x());
      s_sv[(2 * pr + 1) * P4T] = V(ba.y(), bb.y());
      // pairs: central terms count twice, biased ones as a difference
      const R aw = alpha * weight<R>(k);
      const V db = ba - bb;
      if (lat_cx(k)) {
        const R e = aw * R(lat_cx(k));
        ec[0] = fma2(V(R(2) * e), cd, ec[0]);
        eb[0] = fma2(V(e), db, eb[0]);
      }
      if (lat_cy(k)) {
        const R e = aw * R(lat_cy(k));
        ec[1] = fma2(V(R(2) * e), cd, ec[1]);
        eb[1] = fma2(V(e), db, eb[1]);
      }
      if (lat_cz(k)) {
        const R e = aw * R(lat_cz(k));
        ec[2] = fma2(V(R(2) * e), cd, ec[2]);
        eb[2] = fma2(V(e), db, eb[2]);
      }
    }
    const R ecx = ec[0].x(), ecy = ec[1].x(), ecz = ec[2].x();
    const R epx = ec[0].y(), epy = ec[1].y(), epz = ec[2].y();
    const R bcx = eb[0].x(), bcy = eb[1].x(), bcz = eb[2].x();
    const R bpx = eb[0].y(), bpy = eb[1].y(), bpz = eb[2].y();
    const R rho = NODRHO ? rho1 : rho1 + drho * c;
    const R irho = R(1) / rho;
    const R cm_ = (flag & BC_SITE) ? (R) static_cast<const F*>(D.c_raw_bc)[i] : c;
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
      // g_k - g_{k+1} per pair carries the pair's momentum
      R jx = 0, jy = 0, jz = 0;
#pragma unroll
      for (int k = 1; k < Q; k += 2) {
        const R dg = gp[k >> 1].x() - gp[k >> 1].y();
        if (lat_cx(k)) jx += R(lat_cx(k)) * dg;
        if (lat_cy(k)) jy += R(lat_cy(k)) * dg;
        if (lat_cz(k)) jz += R(lat_cz(k)) * dg;
      }
      const R inv = irho * R(1.0 / CS2);
      const R mor = q.mu * irho;
      ux = jx * inv + R(0.5) * (gxa + fxa * irho + mor * ecx);
      uy = jy * inv + R(0.5) * (gya + fya * irho + mor * ecy);
      uz = jz * inv + R(0.5) * (gza + fza * irho + mor * ecz);
    }
    // open-boundary overwrite of g by the plain equilibrium (apply_open_bnd)
    if (flag & BC_G_OVER) {
      const int64_t sb = D.bcsrc[i], dsb = D.dense_of[sb];
      const F* ubc = static_cast<const F*>(D.u_bc);
      const R bux = (R)ubc[sb], buy = (R)ubc[D.n + sb], buz = (R)ubc[2 * D.n + sb];
      const R bp = (R) static_cast<const F*>(D.p)[dsb];
      const R brho = rho1 + drho * (R) static_cast<const F*>(D.c)[dsb];
      const R bu_sq = bux * bux + buy * buy + buz * buz;
      g0 = weight<R>(0) * (bp - brho * cs2 * R(GAMMA) * bu_sq);
#pragma unroll
      for (int k = 1; k < Q; k += 2) {
        const R uk = bux * R(lat_cx(k)) + buy * R(lat_cy(k)) + buz * R(lat_cz(k));
        const R ua = uk * (alpha + R(BETA) * uk) - R(GAMMA) * bu_sq;
        const R ub = -uk * (alpha - R(BETA) * uk) - R(GAMMA) * bu_sq;
        gp[k >> 1] = V(weight<R>(k) * (bp + brho * cs2 * ua), weight<R>(k) * (bp + brho * cs2 * ub));
      }
    }
    // site scalars (device_engine.cuh:563-583)
    const R rho_cs2 = rho * cs2;
    const R c_over = c * irho * R(1.0 / CS2);
    q.drho_cs2 = NODRHO ? R(0) : drho * cs2;
    q.hdr = R(0.5) * q.drho_cs2;
    q.mob = (R)Pm.mobility;
    const R bfx = rho * gxa + fxa, bfy = rho * gya + fya, bfz = rho * gza + fza;
    const R u2 = ux * ux + uy * uy + uz * uz;
    q.gu2 = R(GAMMA) * u2;
    const R efgx = q.mu * ecx + bfx, efgy = q.mu * ecy + bfy, efgz = q.mu * ecz + bfz;
    const R efhx = ecx - c_over * (epx - efgx), efhy = ecy - c_over * (epy - efgy), efhz = ecz - c_over * (epz - efgz);
    const R fdcx = R(0.5) * (ecx + bcx), fdcy = R(0.5) * (ecy + bcy), fdcz = R(0.5) * (ecz + bcz);
    const R fdpx = R(0.5) * (epx + bpx), fdpy = R(0.5) * (epy + bpy), fdpz = R(0.5) * (epz + bpz);
    const R ffgx = q.mu * fdcx + bfx, ffgy = q.mu * fdcy + bfy, ffgz = q.mu * fdcz + bfz;
    const R ffhx = fdcx - c_over * (fdpx - ffgx), ffhy = fdcy - c_over * (fdpy - ffgy),
            ffhz = fdcz - c_over * (fdpz - ffgz);
    const R u_force_g = ux * efgx + uy * efgy + uz * efgz;
    const R u_drho = NODRHO ? R(0) : q.drho_cs2 * (ux * ecx + uy * ecy + uz * ecz);
    const R S_h = R(0.5) * (ux * efhx + uy * efhy + uz * efhz) - (ux * ffhx + uy * ffhy + uz * ffhz);
    q.u_fg_f = ux * ffgx + uy * ffgy + uz * ffgz;
    q.u_drm = NODRHO ? R(0) : q.drho_cs2 * (ux * fdcx + uy * fdcy + uz * fdcz);
    q.C0 = c + S_h;
    q.hk1 = R(0.5) * (R(1) + c_over * q.mu);
    q.hco = R(0.5) * c_over;
    q.A1 = p + R(0.5) * u_force_g;
    q.A2 = NODRHO ? rho_cs2 + R(0.5) * u_force_g : rho_cs2 + R(0.5) * (u_drho + u_force_g);
    st[0] += (double)ux; st[1] += (double)uy; st[2] += (double)uz; st[3] += (double)u2; st[4] += (double)c;
    st[5] = fmax(st[5], (double)u2);
    bad |= !(u2 < R(1e30));

    // ---- main pass over the pairs ------------------------------------------
    const R hl = R(0.5) * lmu;
    R z0, mom[Q];
    V zp[NPAIR];
#pragma unroll
    for (int j = 0; j < Q; ++j) mom[j] = R(0);
    // two-rate form: the parity rates, sum(x) and J
    R hse = R(0), hso = R(0), sumx = R(0), jsx = R(0), jsy = R(0), jsz = R(0);
    if (MRT == 2) {
      const R s1 = R(2) / (R(2) * (R)Pm.mrt_lambda * itau + R(1));
      const int me = Pm.rate_mode[MK_E], mo = Pm.rate_mode[MK_Q];
      hse = R(0.5) * (me == RATE_S0 ? s0 : (me == RATE_MAGIC ? s1 : (R)Pm.rate_value[MK_E]));
      hso = R(0.5) * (mo == RATE_S0 ? s0 : (mo == RATE_MAGIC ? s1 : (R)Pm.rate_value[MK_Q]));
    }
    {  // rest direction: no derivatives, avg = lap(mu) of the site
      const R w = weight<R>(0);
      const R wut = -w * q.gu2, G = w + wut;
      const R h0 = G * (q.C0 + q.mob * lmu);
      const R x0 = (w * q.A1 + q.A2 * wut) - g0;
      z0 = NODRHO ? g0 - q.u_fg_f * G : g0 - q.u_drm * wut - q.u_fg_f * G;
      st_pop<HV<S>>(hout, a0, 0, h0, shh);
      if (MRT == 1) {
#pragma unroll
        for (int j = 0; j < Q; ++j)
          if (mrt_kind(j) != MK_CONS && mrt_M(j, 0) != 0) mom[j] += R(mrt_M(j, 0)) * x0;
      } else if (MRT == 2) {
        sumx = x0;
        z0 += R(2) * hse * x0;
      } else {
        st_pop<GV<S>>(gout, a0, 0, z0 + s0 * x0, shg);
      }
    }
#pragma unroll
    for (int k = 1; k < Q; k += 2) {
      const int o = T::off(k), pr = k >> 1;
      const R cdc = s_sc[pr * P4T];
      const V BC = s_sv[(2 * pr) * P4T], BP = s_sv[(2 * pr + 1) * P4T];
      const R lm = (R)s_l[pos - o], lp = (R)s_l[pos + o];
      // avg of +e takes the +e neighbour, of -e the -e one
      const V la = fma2(V(R(0.5)), V(lp, lm), V(hl));
      const V AVG(is_site(lp) ? la.x() : lmu, is_site(lm) ? la.y() : lmu);
      const R w = weight<R>(k);
      const R uk = ux * R(lat_cx(k)) + uy * R(lat_cy(k)) + uz * R(lat_cz(k));
      const R fproj = bfx * R(lat_cx(k)) + bfy * R(lat_cy(k)) + bfz * R(lat_cz(k));
      // w u_term of +e and -e: w (beta (u.e)^2 - gamma u^2) +- w alpha u.e
      const R we = w * (R(BETA) * uk * uk - q.gu2), wa = (w * alpha) * uk;
      const V WUT(we + wa, we - wa);
      const V G = WUT + V(w);
      // eq_h + force_h = G (c + S_h + mob avg + hk1 bd_c - c_o bd_p / 2 +- c_o F.e / 2)
      const R oh = q.hco * fproj;
      V hb = fma2(V(q.hk1), BC, V(q.C0 + oh, q.C0 - oh));
      hb = fma2(V(-q.hco), BP, hb);
      hb = fma2(V(q.mob), AVG, hb);
      const V H = G * hb;
      // eq_g = w A1 + A2 wut +- (w m1 / 2 + (m1 / 2 - drho cs2 cd_c / 2) wut),
      // m1 = mu cd_c + F.e in the MRT equilibrium, -(mu cd_c + F.e) in the BGK
      // one (device_engine.cuh:517 vs :598)
      const R m1 = MRT ? q.mu * cdc + fproj : -(q.mu * cdc + fproj);
      const R o1 = (R(0.5) * w) * m1, o2 = NODRHO ? R(0.5) * m1 : R(0.5) * m1 - q.hdr * cdc;
      const R wa1 = w * q.A1;
      const V EG = fma2(V(q.A2), WUT, fma2(V(o2, -o2), WUT, V(wa1 + o1, wa1 - o1)));
      const V X = EG - gp[pr];
      // g + force_g = g + (drho cs2 dc - u.drm) wut + (mu dc +- F.e - u.fg_f) G,
      // dc = (+-cd_c + bd_c) / 2 (device_engine.cuh:609)
      const R hc = R(0.5) * cdc;
      const V DC = fma2(V(R(0.5)), BC, V(hc, -hc));
      const V T2 = fma2(V(q.mu), DC, V(fproj - q.u_fg_f, -fproj - q.u_fg_f));
      V Zk;
      if constexpr (NODRHO) {
        Zk = fma2(T2, G, gp[pr]);
      } else {
        const V T1 = fma2(V(q.drho_cs2), DC, V(-q.u_drm));
        Zk = fma2(T2, G, fma2(T1, WUT, gp[pr]));
      }
      const IX tk = dst(k), tk1 = dst(k + 1);
      st_pop<HV<S>>(hout, tk, k, H.x(), shh);
      st_pop<HV<S>>(hout, tk1, k + 1, H.y(), shh);
      // the pair's push targets wait in its (now read) stash slot for the g
      // stores after the moment sums
      if constexpr (KEEP_DST) *reinterpret_cast<uint2*>(&s_sv[(2 * pr) * P4T]) = make_uint2(tk, tk1);
      if (MRT == 2) {
        const R sx = X.x() + X.y(), dx = X.x() - X.y();
        sumx += sx;
        if (lat_cx(k)) jsx += R(lat_cx(k)) * dx;
        if (lat_cy(k)) jsy += R(lat_cy(k)) * dx;
        if (lat_cz(k)) jsz += R(lat_cz(k)) * dx;
        const R te = hse * sx, to = hso * dx;
        zp[pr] = Zk + V(te + to, te - to);
      } else if (MRT == 1) {
        zp[pr] = Zk;
        const R sx = X.x() + X.y(), dx = X.x() - X.y();
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
        const V out = fma2(V(s0), X, Zk);
        st_pop<GV<S>>(gout, dst(k), k, out.x(), shg);
        st_pop<GV<S>>(gout, dst(k + 1), k + 1, out.y(), shg);
      }
    }
    if (MRT == 2) {
      // remove the mass and momentum parts of the relaxation
      const R mx = R(2) * hse * sumx * R(1.0 / 19.0);
      const R qx = R(0.2) * hso * jsx, qy = R(0.2) * hso * jsy, qz = R(0.2) * hso * jsz;
      st_pop<GV<S>>(gout, a0, 0, z0 - mx, shg);
#pragma unroll
      for (int k = 1; k < Q; k += 2) {
        const R ej = qx * R(lat_cx(k)) + qy * R(lat_cy(k)) + qz * R(lat_cz(k));
        const V out = zp[k >> 1] - V(mx + ej, mx - ej);
        if constexpr (KEEP_DST) {
          const uint2 t = *reinterpret_cast<const uint2*>(&s_sv[(2 * (k >> 1)) * P4T]);
          st_pop<GV<S>>(gout, (IX)t.x, k, out.x(), shg);
          st_pop<GV<S>>(gout, (IX)t.y, k + 1, out.y(), shg);
        } else {
          st_pop<GV<S>>(gout, dst(k), k, out.x(), shg);
          st_pop<GV<S>>(gout, dst(k + 1), k + 1, out.y(), shg);
        }
      }
    }
    if (MRT == 1) {
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
      st_pop<GV<S>>(gout, a0, 0, z0 + back0, shg);
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
        const V out = zp[k >> 1] + V(E + O, E - O);
        if constexpr (KEEP_DST) {
          const uint2 t = *reinterpret_cast<const uint2*>(&s_sv[(2 * (k >> 1)) * P4T]);
          st_pop<GV<S>>(gout, (IX)t.x, k, out.x(), shg);
          st_pop<GV<S>>(gout, (IX)t.y, k + 1, out.y(), shg);
        } else {
          st_pop<GV<S>>(gout, dst(k), k, out.x(), shg);
          st_pop<GV<S>>(gout, dst(k + 1), k + 1, out.y(), shg);
        }
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
      C->ff_last = s.ff;
      C->t += 1;
      if (Pm.open_bnd) C->open_step += 1;
      C->pending = (C->auto_correct && Pm.correct_mass) ? 1 : 0;
      C->lambda = 0.0;
      C->count4 = 0;
    }
  }
}

}  // namespace fe
