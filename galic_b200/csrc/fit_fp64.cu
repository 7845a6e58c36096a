// Merit function and optimisation repetition (built with --fmad=false).
//
//  k_fit_smooth / k_fit_diff / k_fit_final   calc_global_fit (main.c:251-362)
//  k_propose      the proposal part of optimize (main.c:365-441)
//  k_eval_terms   the nine stack terms of eval_fit_mod (main.c:1021-1217), one
//                 CTA per term of each evaluation; k_accept combines them
//  k_accept       the accept branch of optimize (main.c:468-507)
//  k_delta_cols   the _delta accumulation (main.c:477-486) and commit_updates
//                 (main.c:818-827): per bin, the accepted particles'
//                 new - old values are summed in particle order, as the
//                 reference's sequential loop does, then added to the
//                 committed grid.
//  k_compact      the accepted positions of a repetition, in order
//  k_inst_delta   add_to_energy_grid of the accepted particles
//                 (main.c:488-498) and its commit (main.c:830-835).
#include <cuda_runtime.h>

#include <mutex>

#include "galic_gpu.h"
#include "grng.h"
#include "kernels.cuh"
#include "rep.cuh"
#include "stack.cuh"

namespace {

__global__ void __launch_bounds__(1024) k_fit_smooth(FitArgs f)
{
  extern __shared__ double sm[];
  const int type = blockIdx.x / NG_COMMITTED, g = blockIdx.x % NG_COMMITTED;
  if(type < 1 || !f.present[type]) return;
  const int off = ((1 << (2 * f.L)) - 1) / 3;
  const double *src = f.committed + ((size_t) type * NG_COMMITTED + g) * f.Ngrid;
  for(int i = threadIdx.x; i < f.Ngrid; i += blockDim.x) sm[off + i] = src[i];
  __syncthreads();
  stack_smooth_cta(sm, f.L);
  double *dst = f.stacks + ((size_t) type * NG_COMMITTED + g) * f.Nstack;
  for(int i = threadIdx.x; i < f.Nstack; i += blockDim.x) dst[i] = sm[i];
}

// raw[type][w]: w = 0 S, 1 Sdisp_r, 2 Sdisp_t, 3 Sdisp_p, 4 Sdisp_q
__global__ void __launch_bounds__(1024) k_fit_diff(FitArgs f, double *raw)
{
  extern __shared__ double sm[];
  const int type = blockIdx.x / 5, w = blockIdx.x % 5;
  if(type < 1 || !f.present[type]) return;
  const double *stk = f.stacks + (size_t) type * NG_COMMITTED * f.Nstack;
  const double *tg = f.targets + (size_t) type * NT_TARGET * f.Nstack;
  const double *d1, *d2, *r1, *r2, *dist;
  double thr;
  int flag;
  if(w == 0) {
    d1 = stk + (size_t) GALIC_GRID_MASS_S * f.Nstack;
    d2 = tg + (size_t) T_DGM * f.Nstack;
    r1 = d2;
    r2 = nullptr;
    dist = f.dgs_distance;
    thr = f.thr_d[type];
    flag = 0;
  } else {
    const int gi[5] = {0, GALIC_GRID_R_I, GALIC_GRID_T_I, GALIC_GRID_P_I, GALIC_GRID_Q_I};
    const int ti[5] = {0, T_R, T_T, T_P, T_Q};
    d1 = stk + (size_t) gi[w] * f.Nstack;
    d2 = tg + (size_t) ti[w] * f.Nstack;
    r1 = stk + (size_t) GALIC_GRID_MASS_I * f.Nstack;
    r2 = tg + (size_t) T_EGM * f.Nstack;
    dist = nullptr;
    thr = f.thr_e[type];
    flag = 1;
  }
  for(int i = threadIdx.x; i < f.Nstack; i += blockDim.x) sm[i] = d1[i];
  __syncthreads();
  double v = stack_diff_cta(sm, d2, r1, r2, dist, thr, flag, 0, f.L, f.R200_20, f.LowerDispLimit);
  if(threadIdx.x == 0) raw[type * 5 + w] = v;
}

__global__ void k_fit_final(FitArgs f, const double *raw)
{
  const int type = threadIdx.x;
  if(type < 1 || type > 3 || !f.present[type]) return;
  const double *tg = f.targets + (size_t) type * NT_TARGET * f.Nstack;
  double S = raw[type * 5 + 0];
  S *= 1.0 / tg[T_DGM * f.Nstack + 0];
  double sr = raw[type * 5 + 1], st = raw[type * 5 + 2], sp = raw[type * 5 + 3], sq = raw[type * 5 + 4];
  double count;
  if(f.tovs[type] == 0 || f.tovs[type] == 1) {
    count = 3.0;
    sq = 0;
  } else
    count = 4.0;
  double *o = f.fit + type * 7;
  double srel = o[5];
  if(f.firstrun[type] == 0) {
    srel = S / ((sr + st + sp + sq) / count);
    f.firstrun[type] = 1;
  }
  o[0] = S;
  o[1] = sr * srel;
  o[2] = st * srel;
  o[3] = sp * srel;
  o[4] = sq * srel;
  o[5] = srel;
  o[6] = count;
}

// ---------------------------------------------------------------- optimize

__global__ void k_propose(DevModel M, RepArgs R)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= R.count) return;
  LogConsts L = make_log_consts(M);
  const int n = R.idx[k];
  const int type = R.p_type[n];
  const int tovs = M.tovs[type];
  const double *pos = &R.p_pos[3 * n];
  grng_t g;
  // repetition k / per_rep of a window of repetitions draws from its own serial
  grng_init(&g, R.seed, (uint32_t) n, R.rep_serial + (uint32_t) (R.per_rep > 0 ? k / R.per_rep : 0));
  (void) grng_uniform(&g);  // dir_rnd (main.c:370)
  double phi = gm_atan2(pos[1], pos[0]);
  double Rv[3], Tv[3], Qv[3];
  if(tovs == 2) {
    double c = gm_cos(phi), s = gm_sin(phi);
    Rv[0] = c; Rv[1] = s; Rv[2] = 0;
    Tv[0] = -s; Tv[1] = c; Tv[2] = 0;
    Qv[0] = 0; Qv[1] = 0; Qv[2] = 1;
  } else {
    double theta = gm_acos(pos[2] / sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]));
    double st = gm_sin(theta), ct = gm_cos(theta), sp = gm_sin(phi), cp = gm_cos(phi);
    Rv[0] = st * cp; Rv[1] = st * sp; Rv[2] = ct;
    Tv[0] = -ct * cp; Tv[1] = -ct * sp; Tv[2] = st;
    Qv[0] = -sp; Qv[1] = cp; Qv[2] = 0;
  }
  const double *tg = &R.p_targets[4 * n];
  double sigma_r = sqrt(tg[0]), sigma_t = sqrt(tg[1]), sigma_p = sqrt(tg[2]);
  double vstr = vstream_at(M, fg_coord(M, L, pos), type);
  double v_new[3], v2_new;
  int iter = 0, st_code = 0;
  do {
    double vr_new = grng_gaussian(&g, sigma_r);
    double vt_new = grng_gaussian(&g, sigma_t);
    double vq_new = vstr + grng_gaussian(&g, sigma_p);
    for(int j = 0; j < 3; j++) v_new[j] = vr_new * Rv[j] + vt_new * Tv[j] + vq_new * Qv[j];
    v2_new = v_new[0] * v_new[0] + v_new[1] * v_new[1] + v_new[2] * v_new[2];
    iter++;
    if(iter > 100000) {  // main.c:432-433
      st_code = GALIC_ERR_REJECTION_CAP;
      break;
    }
  } while(sqrt(v2_new) >= M.MaxVelInUnitsVesc * R.p_vesc[n]);
  if(st_code) atomicMax(R.status, st_code);
  for(int j = 0; j < 3; j++) {
    R.vel_try[3 * k + j] = v_new[j];
    R.b_pos[3 * (2 * k) + j] = pos[j];
    R.b_pos[3 * (2 * k + 1) + j] = pos[j];
    R.b_vel[3 * (2 * k) + j] = R.p_vel[3 * n + j];
    R.b_vel[3 * (2 * k + 1) + j] = v_new[j];
  }
  R.b_mass[2 * k] = R.b_mass[2 * k + 1] = R.p_mass[n];
  R.b_time[2 * k] = R.b_time[2 * k + 1] = R.p_tint[n];
  R.b_type[2 * k] = R.b_type[2 * k + 1] = type;
}

// The nine stack terms of eval_fit_mod (main.c:1021-1217), one CTA per
// (particle k, which, term): which 0 = F_base, 1 = F_try; term 0 the
// density term (main.c:1033-1047), 1-4 the time-averaged dispersion terms
// r, t, q, p (main.c:1052-1120), 5-8 the instantaneous terms r, t, p, q
// (main.c:1125-1176).  Each writes its stack difference to
// R.F[(2k + which) * NTERM + term]; k_accept combines them into F in the
// reference's order.
// The base evaluation's instantaneous terms (which 0, terms 5-8) are not
// launched per particle: its velocity is the particle's own, whose
// projections are the committed ones (p_vdisp was computed from p_vel by
// the same disp_components), so the change it adds to the energy grid is
// exactly zero and the term is its type's committed misfit, computed once
// per repetition by k_base_inst.  Each particle launches 5 + 9 CTAs.
enum { NTERM = 9, NLAUNCH = 14 };

__global__ void __launch_bounds__(512) k_eval_terms(DevModel M, RepArgs R, FitArgs f)
{
  // levels 0 .. L-1 of the evaluated stack; its finest level is formed on
  // the fly from the committed stack and the orbit grids (stack.cuh:*_from)
  extern __shared__ double sm[];
  __shared__ double sh_d[4];
  __shared__ Cell sh_c;
  const int j = blockIdx.x % NLAUNCH, k = blockIdx.x / NLAUNCH;
  const int which = j < 5 ? 0 : 1, term = j < 5 ? j : j - 5;
  const int n = R.idx[k];
  const int type = R.p_type[n];
  const int L = f.L, G = f.Ngrid, Ns = f.Nstack;
  const int off = ((1 << (2 * L)) - 1) / 3;
  const double *gold = R.grids + (size_t) (2 * k) * NF_ORBIT * G;
  const double *gnew = R.grids + (size_t) (2 * k + which) * NF_ORBIT * G;
  // the orbit grids are stored unscaled: x mass/tall on the fly, the
  // operation k_scale_dense would have applied
  const double fo = R.b_mass[2 * k] / R.b_tall[2 * k];
  const double fn = R.b_mass[2 * k + which] / R.b_tall[2 * k + which];
  const double *stk = f.stacks + (size_t) type * NG_COMMITTED * Ns;
  const double *tg = f.targets + (size_t) type * NT_TARGET * Ns;
  double v;
  if(term == 0) {
    // density term: committed + new - old
    const double *c = stk + (size_t) GALIC_GRID_MASS_S * Ns + off;
    const double *gn = gnew + F_M * G, *go = gold + F_M * G;
    auto fin = [&](int i) { return c[i] + gn[i] * fn - go[i] * fo; };
    stack_smooth_cta_from(sm, L, fin);
    v = stack_diff_cta_from(sm, fin, tg + T_DGM * Ns, tg + T_DGM * Ns, nullptr, f.dgs_distance, f.thr_d[type], 0, 0,
                            L, f.R200_20, f.LowerDispLimit);
  } else if(term <= 4) {
    // time-averaged dispersion terms r, t, q, p
    const int a = term - 1;
    const int fs[4] = {F_R, F_T, F_Q, F_P};
    const int gs[4] = {GALIC_GRID_R_S, GALIC_GRID_T_S, GALIC_GRID_Q_S, GALIC_GRID_P_S};
    const int ts[4] = {T_R, T_T, T_Q, T_P};
    const double *c = stk + (size_t) gs[a] * Ns + off;
    const double *gn = gnew + fs[a] * G, *go = gold + fs[a] * G;
    auto fin = [&](int i) { return c[i] + gn[i] * fn - go[i] * fo; };
    stack_smooth_cta_from(sm, L, fin);
    v = stack_diff_cta_from(sm, fin, tg + ts[a] * Ns, tg + T_DGM * Ns, tg + ts[a] * Ns, f.dgs_distance,
                            f.thr_d[type], 2, 1, L, f.R200_20, f.LowerDispLimit);
  } else {
    // instantaneous terms r, t, p, q of the trial velocity: its change of the
    // particle's projections at its energy-grid cell
    const int a = term - 5;
    if(threadIdx.x == 0) {
      LogConsts Lc = make_log_consts(M);
      const double *vel = which ? &R.vel_try[3 * k] : &R.p_vel[3 * n];
      disp_components(M, Lc, type, &R.p_pos[3 * n], vel, sh_d);
      sh_c = energy_cell(M, Lc, &R.p_pos[3 * n]);
    }
    __syncthreads();
    const double mass = R.p_mass[n];
    const double *vd = &R.p_vdisp[4 * n];
    // add_to_energy_grid: vr2 *= mass etc. (main.c:885-888); order r, t, p, q
    const double dv = (sh_d[a] - vd[a]) * mass;
    const int gi[4] = {GALIC_GRID_R_I, GALIC_GRID_T_I, GALIC_GRID_P_I, GALIC_GRID_Q_I};
    const int ti[4] = {T_R, T_T, T_P, T_Q};
    const Cell cc = sh_c;
    const int Nb = 1 << L;
    const int c00 = cc.iz * Nb + cc.iR;
    const double w00 = (1 - cc.fR) * (1 - cc.fz), w10 = (cc.fR) * (1 - cc.fz), w01 = (1 - cc.fR) * (cc.fz),
                 w11 = (cc.fR) * (cc.fz);
    const double *c = stk + (size_t) gi[a] * Ns + off;
    // committed value, plus w * dv at the four corners of the cell
    auto fin = [&](int i) {
      const double x = c[i];
      return i == c00 ? x + w00 * dv
                      : (i == c00 + 1 ? x + w10 * dv : (i == c00 + Nb ? x + w01 * dv : (i == c00 + Nb + 1 ? x + w11 * dv : x)));
    };
    stack_smooth_cta_from(sm, L, fin);
    v = stack_diff_cta_from(sm, fin, tg + ti[a] * Ns, stk + (size_t) GALIC_GRID_MASS_I * Ns, tg + T_EGM * Ns,
                            nullptr, f.thr_e[type], 1, 0, L, f.R200_20, f.LowerDispLimit);
  }
  if(threadIdx.x == 0) R.F[(2 * k + which) * NTERM + term] = v;
}

// the committed instantaneous misfit of each present type: terms 5-8 of
// every base evaluation of the repetition (see k_eval_terms)
__global__ void __launch_bounds__(512) k_base_inst(RepArgs R, FitArgs f)
{
  extern __shared__ double sm[];
  const int type = blockIdx.x >> 2, a = blockIdx.x & 3;
  if(type < 1 || !f.present[type]) return;
  const int L = f.L, Ns = f.Nstack;
  const int off = ((1 << (2 * L)) - 1) / 3;
  const double *stk = f.stacks + (size_t) type * NG_COMMITTED * Ns;
  const double *tg = f.targets + (size_t) type * NT_TARGET * Ns;
  const int gi[4] = {GALIC_GRID_R_I, GALIC_GRID_T_I, GALIC_GRID_P_I, GALIC_GRID_Q_I};
  const int ti[4] = {T_R, T_T, T_P, T_Q};
  const double *c = stk + (size_t) gi[a] * Ns + off;
  auto fin = [&](int i) { return c[i]; };
  stack_smooth_cta_from(sm, L, fin);
  const double v = stack_diff_cta_from(sm, fin, tg + ti[a] * Ns, stk + (size_t) GALIC_GRID_MASS_I * Ns,
                                       tg + T_EGM * Ns, nullptr, f.thr_e[type], 1, 0, L, f.R200_20, f.LowerDispLimit);
  if(threadIdx.x == 0) R.inst0[blockIdx.x] = v;
}

// F of eval_fit_mod from its nine stack terms t[] (main.c:1047, 1120, 1195-1212)
__device__ __forceinline__ double combine_terms(const DevModel &M, const RepArgs &R, const FitArgs &f, int type,
                                                const double *t)
{
  const double MT = f.MType[type];
  double value = t[0];
  value *= 1.0 / MT;
  const double value_rs = t[1] / MT, value_ts = t[2] / MT, value_qs = t[3] / MT, value_ps = t[4] / MT;
  double value_r = t[5], value_t = t[6], value_p = t[7], value_q = t[8];
  if(M.tovs[type] == 0 || type == 2) value_q = 0;  // main.c:1195
  const double *fit = f.fit + type * 7;
  return value + fit[5] / fit[6] * (value_r + value_t + value_p + value_q) +
         (R.fac_rs[type] * value_rs + R.fac_ts[type] * value_ts + R.fac_ps[type] * value_ps +
          R.fac_qs[type] * value_qs) /
             4;
}

__global__ void k_accept(DevModel M, RepArgs R, FitArgs f)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= R.count) return;
  const int n = R.idx[k];
  const int type = R.p_type[n];
  R.p_orbits[n] = R.b_norbit[2 * k];  // main.c:460 writes the old orbit's count
  atomicAdd(&R.tries[type], 1ULL);
  double tb[NTERM];
  for(int j = 0; j < 5; j++) tb[j] = R.F[(2 * k) * NTERM + j];
  for(int j = 0; j < 4; j++) tb[5 + j] = R.inst0[4 * type + j];
  const double F_base = combine_terms(M, R, f, type, tb);
  const double F_try = combine_terms(M, R, f, type, &R.F[(2 * k + 1) * NTERM]);
  const bool acc = F_try < F_base;  // main.c:468
  // mass/tall of the old and trial orbits (orbit_response.c:477-486) for
  // the commit, which reads the unscaled orbit grids
  R.fac[2 * k] = R.b_mass[2 * k] / R.b_tall[2 * k];
  R.fac[2 * k + 1] = R.b_mass[2 * k + 1] / R.b_tall[2 * k + 1];
  R.accepted[k] = acc ? 1 : 0;
  if(!acc) return;
  for(int j = 0; j < 3; j++) R.p_vel[3 * n + j] = R.vel_try[3 * k + j];
  R.p_orbits[n] = R.b_norbit[2 * k + 1];
  atomicAdd(&R.changes[type], 1ULL);
  LogConsts L = make_log_consts(M);
  double d[4];
  disp_components(M, L, type, &R.p_pos[3 * n], &R.vel_try[3 * k], d);
  double *vd = &R.p_vdisp[4 * n];
  const double mass = R.p_mass[n];
  for(int j = 0; j < 4; j++) {
    R.inst_v[4 * k + j] = (d[j] - vd[j]) * mass;
    vd[j] = d[j];
  }
  R.inst_cell[k] = energy_cell(M, L, &R.p_pos[3 * n]);
}

// the accepted positions of one repetition in increasing k (one CTA): the
// commit kernels below loop over these instead of over every position
__global__ void __launch_bounds__(1024) k_compact(RepArgs R)
{
  __shared__ int warp_sum[32];
  __shared__ int base;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  if(threadIdx.x == 0) base = 0;
  __syncthreads();
  for(int k0 = 0; k0 < R.count; k0 += blockDim.x) {
    const int k = k0 + threadIdx.x;
    const int a = (k < R.count && R.accepted[k]) ? 1 : 0;
    const unsigned m = __ballot_sync(0xffffffffu, a);
    if(lane == 0) warp_sum[wid] = __popc(m);
    __syncthreads();
    int before = 0;
    for(int w = 0; w < wid; w++) before += warp_sum[w];
    if(a) R.acc_list[base + before + __popc(m & ((1u << lane) - 1))] = k;
    __syncthreads();
    if(threadIdx.x == 0) {
      int tot = 0;
      for(int w = 0; w < (int) (blockDim.x >> 5); w++) tot += warp_sum[w];
      base += tot;
    }
    __syncthreads();
  }
  if(threadIdx.x == 0) *R.acc_n = base;
}

// per (type, field, bin): delta = sum over accepted particles, in order, of
// new - old; committed += delta
__global__ void k_delta_cols(RepArgs R, FitArgs f)
{
  const int G = f.Ngrid;
  const int na = *R.acc_n;
  const size_t total = (size_t) 4 * NF_ORBIT * G;
  for(size_t t = blockIdx.x * (size_t) blockDim.x + threadIdx.x; t < total; t += (size_t) gridDim.x * blockDim.x) {
    const int type = (int) (t / ((size_t) NF_ORBIT * G));
    const int fld = (int) ((t / G) % NF_ORBIT);
    const int i = (int) (t % G);
    if(type < 1 || !f.present[type]) continue;
    double delta = 0;
    for(int j = 0; j < na; j++) {
      const int k = R.acc_list[j];
      if(R.b_type[2 * k] != type) continue;
      const double *gold = R.grids + (size_t) (2 * k) * NF_ORBIT * G;
      const double *gnew = gold + (size_t) NF_ORBIT * G;
      // unscaled orbit grids: x mass/tall as k_scale_dense would (the
      // factors k_accept stored, the same divisions)
      delta += gnew[fld * G + i] * R.fac[2 * k + 1] - gold[fld * G + i] * R.fac[2 * k];
    }
    // orbit fields m,r,t,q,p map to committed MASS_S, R_S, T_S, Q_S, P_S
    double *dst = (double *) f.committed + ((size_t) type * NG_COMMITTED + fld) * G + i;
    *dst += delta;
  }
}

__global__ void k_inst_delta(RepArgs R, FitArgs f)
{
  const int G = f.Ngrid, Nb = 1 << f.L;
  const int na = *R.acc_n;
  const size_t total = (size_t) 4 * 4 * G;
  const int gi[4] = {GALIC_GRID_R_I, GALIC_GRID_T_I, GALIC_GRID_P_I, GALIC_GRID_Q_I};
  for(size_t t = blockIdx.x * (size_t) blockDim.x + threadIdx.x; t < total; t += (size_t) gridDim.x * blockDim.x) {
    const int type = (int) (t / ((size_t) 4 * G));
    const int a = (int) ((t / G) % 4);
    const int cidx = (int) (t % G);
    if(type < 1 || !f.present[type]) continue;
    double delta = 0;
    for(int j = 0; j < na; j++) {
      const int k = R.acc_list[j];
      if(R.b_type[2 * k] != type) continue;
      const Cell c = R.inst_cell[k];
      const int base = c.iz * Nb + c.iR;
      double w;
      if(cidx == base) w = (1 - c.fR) * (1 - c.fz);
      else if(cidx == base + 1) w = (c.fR) * (1 - c.fz);
      else if(cidx == base + Nb) w = (1 - c.fR) * (c.fz);
      else if(cidx == base + Nb + 1) w = (c.fR) * (c.fz);
      else continue;
      // inst_v holds (vr2, vt2, vp2, vq2) differences times mass
      delta += w * R.inst_v[4 * k + a];
    }
    double *dst = (double *) f.committed + ((size_t) type * NG_COMMITTED + gi[a]) * G + cidx;
    *dst += delta;
  }
}

}  // namespace

// the stack kernels keep a whole level-7 stack (171 KiB) in shared memory;
// called once per context, on the context's device
// the shared-memory opt-in of the stack kernels, once per device
cudaError_t prepare_fit_kernels()
{
  static std::mutex mu;
  static bool done[256] = {false};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e != cudaSuccess) return e;
  std::lock_guard<std::mutex> lk(mu);
  if(dev >= 0 && dev < 256 && done[dev]) return cudaSuccess;
  if((e = cudaFuncSetAttribute(k_fit_smooth, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
  if((e = cudaFuncSetAttribute(k_fit_diff, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
  if((e = cudaFuncSetAttribute(k_eval_terms, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
  if((e = cudaFuncSetAttribute(k_base_inst, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024))) return e;
  if(dev >= 0 && dev < 256) done[dev] = true;
  return cudaSuccess;
}

int launch_global_fit(const FitArgs &f, cudaStream_t s)
{
  size_t smem = (size_t) f.Nstack * sizeof(double);
  double *raw = f.fit + 4 * 7;  // scratch after the 4x7 fit block
  k_fit_smooth<<<4 * NG_COMMITTED, 1024, smem, s>>>(f);
  k_fit_diff<<<4 * 5, 1024, smem, s>>>(f, raw);
  k_fit_final<<<1, 4, 0, s>>>(f, raw);
  return 3;
}

int launch_rep_orbits(const DevModel &M, const RepArgs &R, const OrbitBatch &b, cudaStream_t s,
                      const float4 *const *quad32, const float *cellsize32)
{
  const int count = R.count;
  k_propose<<<(count + 63) / 64, 64, 0, s>>>(M, R);
  cudaMemsetAsync(b.grids, 0, (size_t) b.count * NF_ORBIT * M.DG_Ngrid * sizeof(double), s);
  if(quad32)
    launch_orbits_dense_fp32(M, quad32, cellsize32, b, s);
  else
    launch_orbits_dense(M, b, s);
  // the grids stay unscaled: the merit and commit kernels multiply by
  // mass/tall where they read them (one pass over the grids less)
  return 2;
}

int launch_rep_commit(const DevModel &M, const RepArgs &R, const FitArgs &f, cudaStream_t s)
{
  const int count = R.count;
  // levels 0 .. L-1 of a stack in shared memory (43 KiB at L = 7): four
  // CTAs of 512 threads per SM
  const size_t smem = (size_t) (((1 << (2 * f.L)) - 1) / 3) * sizeof(double);
  k_base_inst<<<16, 512, smem, s>>>(R, f);
  k_eval_terms<<<count * NLAUNCH, 512, smem, s>>>(M, R, f);
  k_accept<<<(count + 127) / 128, 128, 0, s>>>(M, R, f);
  k_compact<<<1, 1024, 0, s>>>(R);
  k_delta_cols<<<148 * 8, 256, 0, s>>>(R, f);
  k_inst_delta<<<148 * 8, 256, 0, s>>>(R, f);
  return 6 + launch_global_fit(f, s);
}

RepArgs rep_slice(const RepArgs &R, int first, int count, int G)
{
  RepArgs S = R;
  S.count = count;
  S.per_rep = 0;
  S.idx = R.idx + first;
  S.b_pos = R.b_pos + 3 * (size_t) (2 * first);
  S.b_vel = R.b_vel + 3 * (size_t) (2 * first);
  S.b_mass = R.b_mass + 2 * (size_t) first;
  S.b_time = R.b_time + 2 * (size_t) first;
  S.b_type = R.b_type + 2 * (size_t) first;
  S.b_norbit = R.b_norbit + 2 * (size_t) first;
  S.b_tall = R.b_tall + 2 * (size_t) first;
  S.fac = R.fac + 2 * (size_t) first;
  S.grids = R.grids + (size_t) (2 * first) * NF_ORBIT * G;
  S.vel_try = R.vel_try + 3 * (size_t) first;
  S.F = R.F + 2 * (size_t) NTERM * first;
  S.accepted = R.accepted + first;
  S.acc_list = R.acc_list + first;
  S.acc_n = R.acc_n + first / count;
  S.inst_v = R.inst_v + 4 * (size_t) first;
  S.inst_cell = R.inst_cell + first;
  return S;
}

int launch_rep(const DevModel &M, const RepArgs &R, const FitArgs &f, const OrbitBatch &b, cudaStream_t s,
               const float4 *const *quad32, const float *cellsize32)
{
  const int launches = launch_rep_orbits(M, R, b, s, quad32, cellsize32);
  return launches + launch_rep_commit(M, R, f, s);
}
