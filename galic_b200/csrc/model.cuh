// Device-side view of one GALIC model and the FP64 orbit integrator.
//
// Every function restates a reference routine (file:line of the reference
// tree src/) with the same operation order, so that compiled with
// --fmad=false and evaluated with gmath.h it reproduces the CPU restatement
// bit for bit.  The orbit integrator is a template over a "sink" that
// receives the deposits: a dense per-orbit grid (reference semantics) or
// the batched fixed-point accumulators.
#ifndef GALIC_MODEL_CUH
#define GALIC_MODEL_CUH

#include <stdint.h>

#include "gmath.h"

#define GALIC_STEP_CAP 100000000LL  // orbit_response.c:450

enum OrbitStatus { ORBIT_OK = 0, ORBIT_STEP_CAP = 1, ORBIT_NONFINITE = 2 };

struct DevModel {
  // All.* (allvars.h:639-836)
  double V200, M200, R200, G;
  double Halo_Mass, Halo_A, Bulge_Mass, Bulge_A;
  double f_orb, f_cc;  // TimeStepFactorOrbit, TimeStepFactorCellCross
  double LowerDispLimit, MaxVelInUnitsVesc;
  int tabulated;       // grid.c:63 / grid.c:124 condition
  int analytic_halo;   // Halo_Mass > 0 && SampleForceNhalo == 0
  int analytic_bulge;  // Bulge_Mass > 0 && SampleForceNbulge == 0
  int tovs[4];
  int vstream_zero[4]; // FG_Vstream[type] is identically +0
  // grid geometry
  int FG_Nbin, DG_Nbin, DG_L, EG_L, DG_Ngrid, DG_Nstack;
  double FG_Rmin, FG_Fac, DG_Rmin, DG_Fac, EG_Rmin, EG_Fac;
  // log(FG_Fac), log(DG_Fac), log(EG_Fac) and the correctly rounded
  // reciprocals of the orbit step's per-model divisors FG_Rmin, DG_Rmin,
  // log(FG_Fac), log(DG_Fac) (set_step_constants)
  double lfg, ldg, leg;
  double inv_FG_Rmin, inv_DG_Rmin, inv_lfg, inv_ldg;
  // tables (device pointers, reference layouts)
  const double2 *fg_acc;  // {FG_DPotDR, FG_DPotDz}[iz*FG_Nbin+iR]
  const double *fg_pot;
  const double *vstream[4];
  const double *cellsize;  // DG_CellSize
  long long step_cap;
};

// Host side: the logs of the grid factors (gm_log is the same function on
// host and device, so these equal make_log_consts' values) and the
// reciprocals div_by needs, from the same values the step divides by.
inline void set_step_constants(DevModel &M)
{
  M.lfg = gm_log(M.FG_Fac);
  M.ldg = gm_log(M.DG_Fac);
  M.leg = gm_log(M.EG_Fac);
  M.inv_FG_Rmin = 1.0 / M.FG_Rmin;
  M.inv_DG_Rmin = 1.0 / M.DG_Rmin;
  M.inv_lfg = 1.0 / M.lfg;
  M.inv_ldg = 1.0 / M.ldg;
}

// a / b for a divisor b fixed per model, given y = 1/b correctly rounded:
// q0 = a*y, then one correction q0 + (a - b*q0)*y with both steps fused
// (Markstein, IBM J. Res. Develop. 34(1), 1990).  It returns the correctly
// rounded quotient a / b whenever b, y and a/b are normal numbers: checked for
// every pair of significands at precisions 6 to 12 and on 1e8 random binary64
// pairs (tests/test_gmath.py), and by the per-orbit bit-exact parity tests.
// Where the step uses it, a tiny or subnormal quotient is added to 1.0 and an
// infinite one (NaN here) only ever fails an in-grid test, so the step's
// results are those of the division in every case.  Three dependent FP64
// operations instead of an IEEE division's iteration and range checks.
__device__ __forceinline__ double div_by(double a, double b, double y)
{
  const double q0 = a * y;
  return fma(fma(-q0, b, a), y, q0);
}

// ------------------------------------------------------------ analytic parts

// halo_get_acceleration (halo.c:76-84)
__device__ __forceinline__ void halo_acc(const DevModel &M, const double *pos, double *acc)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  double fac = M.G * M.Halo_Mass / ((r + 1.0e-6 * M.Halo_A) * (r + M.Halo_A) * (r + M.Halo_A));
  acc[0] = -fac * pos[0];
  acc[1] = -fac * pos[1];
  acc[2] = -fac * pos[2];
}
// halo_get_potential (halo.c:63-73)
__device__ __forceinline__ double halo_pot(const DevModel &M, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  return -M.G * M.Halo_Mass / (r + M.Halo_A);
}
// bulge_get_acceleration / _potential (bulge.c:63-85)
__device__ __forceinline__ void bulge_acc(const DevModel &M, const double *pos, double *acc)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  double fac = M.G * M.Bulge_Mass / ((r + 1.0e-6 * M.Bulge_A) * (r + M.Bulge_A) * (r + M.Bulge_A));
  acc[0] = -fac * pos[0];
  acc[1] = -fac * pos[1];
  acc[2] = -fac * pos[2];
}
__device__ __forceinline__ double bulge_pot(const DevModel &M, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  return -M.G * M.Bulge_Mass / (r + M.Bulge_A);
}

// Per-model constants the reference recomputes in every call (log(FG_Fac),
// log(DG_Fac)); same function, same value.
struct LogConsts {
  double lfg, ldg, leg;
};
// the same values from the parameter space, where set_step_constants put
// them (kernels whose model went through it: no registers held for them)
__device__ __forceinline__ LogConsts step_log_consts(const DevModel &M)
{
  LogConsts c;
  c.lfg = M.lfg;
  c.ldg = M.ldg;
  c.leg = M.leg;
  return c;
}
__device__ __forceinline__ LogConsts make_log_consts(const DevModel &M)
{
  LogConsts c;
  c.lfg = gm_log(M.FG_Fac);
  c.ldg = gm_log(M.DG_Fac);
  c.leg = gm_log(M.EG_Fac);
  return c;
}

// (int) conversion as the reference's x86 build performs it for finite
// in-range values; callers guard NaN and out-of-range before using indices.
__device__ __forceinline__ int trunc_int(double x) { return (int) x; }

// The FG log coordinates jdbl, idbl of grid.c:130-136 (also forcegrid_get_cell
// grid.c:20-21 and the potential grid.c:68-74): identical expressions.
struct FgCoord {
  double jdbl, idbl;
};
__device__ __forceinline__ FgCoord fg_coord(const DevModel &M, const LogConsts &L, const double *pos)
{
  FgCoord c;
  double R = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  c.jdbl = gm_log(R / M.FG_Rmin + 1.0) / L.lfg;
  c.idbl = gm_log(gm_fabs(pos[2]) / M.FG_Rmin + 1.0) / L.lfg;
  return c;
}

// forcegrid_get_acceleration (grid.c:122-197) given the FG coordinates of pos
__device__ __forceinline__ void forcegrid_acc(const DevModel &M, const FgCoord &c, const double *pos, double *acc)
{
  const int N = M.FG_Nbin;
  if(M.tabulated) {
    double jdbl = c.jdbl, idbl = c.idbl;
    // NaN or huge coordinates take the off-grid branch instead of indexing
    if(jdbl < (double) (N - 1) && idbl < (double) (N - 1)) {
      double phi = gm_atan2(pos[1], pos[0]);
      int jbin = trunc_int(jdbl);
      double jfac = jdbl - jbin;
      int ibin = trunc_int(idbl);
      double ifac = idbl - ibin;
      const double2 *T = M.fg_acc;
      double2 t00 = __ldg(&T[ibin * N + jbin]);
      double2 t01 = __ldg(&T[ibin * N + (jbin + 1)]);
      double2 t10 = __ldg(&T[(ibin + 1) * N + jbin]);
      double2 t11 = __ldg(&T[(ibin + 1) * N + (jbin + 1)]);
      double accR = t00.x * (1 - ifac) * (1 - jfac) + t01.x * (1 - ifac) * jfac + t10.x * ifac * (1 - jfac) +
                    t11.x * ifac * jfac;
      double accz = t00.y * (1 - ifac) * (1 - jfac) + t01.y * (1 - ifac) * jfac + t10.y * ifac * (1 - jfac) +
                    t11.y * ifac * jfac;
      if(pos[2] < 0) accz = -accz;
      double sp, cp;
      gm_sincos(phi, &sp, &cp);  // gm_sin(phi), gm_cos(phi)
      acc[0] = accR * cp;
      acc[1] = accR * sp;
      acc[2] = accz;
    } else {
      halo_acc(M, pos, acc);
      double fac = M.M200 / M.Halo_Mass;
      acc[0] *= fac;
      acc[1] *= fac;
      acc[2] *= fac;
    }
  } else {
    acc[0] = acc[1] = acc[2] = 0;
  }
  if(M.analytic_halo) {
    double a[3];
    halo_acc(M, pos, a);
    acc[0] += a[0];
    acc[1] += a[1];
    acc[2] += a[2];
  }
  if(M.analytic_bulge) {
    double a[3];
    bulge_acc(M, pos, a);
    acc[0] += a[0];
    acc[1] += a[1];
    acc[2] += a[2];
  }
}

// forcegrid_get_potential (grid.c:59-113)
__device__ __forceinline__ double forcegrid_pot(const DevModel &M, const LogConsts &L, const double *pos)
{
  const int N = M.FG_Nbin;
  double pot;
  if(M.tabulated) {
    FgCoord c = fg_coord(M, L, pos);
    if(c.jdbl < (double) (N - 1) && c.idbl < (double) (N - 1)) {
      int jbin = trunc_int(c.jdbl);
      double jfac = c.jdbl - jbin;
      int ibin = trunc_int(c.idbl);
      double ifac = c.idbl - ibin;
      const double *P = M.fg_pot;
      pot = __ldg(&P[ibin * N + jbin]) * (1 - ifac) * (1 - jfac) + __ldg(&P[ibin * N + (jbin + 1)]) * (1 - ifac) * jfac +
            __ldg(&P[(ibin + 1) * N + jbin]) * ifac * (1 - jfac) +
            __ldg(&P[(ibin + 1) * N + (jbin + 1)]) * ifac * jfac;
    } else
      pot = M.M200 / M.Halo_Mass * halo_pot(M, pos);
  } else
    pot = 0;
  if(M.analytic_halo) pot += halo_pot(M, pos);
  if(M.analytic_bulge) pot += bulge_pot(M, pos);
  return pot;
}

// cell (iR, iz, fR, fz) of a log grid: densitygrid_get_cell (grid.c:494-534,
// shift 0.5), energygrid_get_cell (grid.c:896-938, shift 0.5) and
// forcegrid_get_cell (grid.c:15-55, from precomputed br/bz, no shift).
struct Cell {
  int iR, iz;
  double fR, fz;
};
__device__ __forceinline__ Cell cell_from_b(double br, double bz, int nbin)
{
  Cell c;
  if(br < 0) br = 0;
  if(bz < 0) bz = 0;
  // a NaN coordinate fails both tests below and lands in the last cell with
  // weight 1: the orbit is flagged ORBIT_NONFINITE by the caller
  int binr = (br < (double) (nbin - 1)) ? trunc_int(br) : nbin - 1;
  int binz = (bz < (double) (nbin - 1)) ? trunc_int(bz) : nbin - 1;
  c.fR = br - binr;
  c.fz = bz - binz;
  if(binr >= nbin - 1) {
    binr = nbin - 2;
    c.fR = 1;
  }
  if(binz >= nbin - 1) {
    binz = nbin - 2;
    c.fz = 1;
  }
  c.iR = binr;
  c.iz = binz;
  return c;
}

__device__ __forceinline__ Cell density_cell(const DevModel &M, const LogConsts &L, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  double z = gm_fabs(pos[2]);
  double br = (gm_log(r / M.DG_Rmin + 1.0) / L.ldg) - 0.5;
  double bz = (gm_log(z / M.DG_Rmin + 1.0) / L.ldg) - 0.5;
  return cell_from_b(br, bz, M.DG_Nbin);
}

__device__ __forceinline__ Cell energy_cell(const DevModel &M, const LogConsts &L, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
  double z = gm_fabs(pos[2]);
  double br = (gm_log(r / M.EG_Rmin + 1.0) / L.leg) - 0.5;
  double bz = (gm_log(z / M.EG_Rmin + 1.0) / L.leg) - 0.5;
  return cell_from_b(br, bz, 1 << M.EG_L);
}

// get_vstream (disp_fields.c:118-132) from the FG coordinates of pos
__device__ __forceinline__ double vstream_at(const DevModel &M, const FgCoord &c, int type)
{
  if(M.vstream_zero[type]) return 0.0;
  const int N = M.FG_Nbin;
  Cell k = cell_from_b(c.jdbl, c.idbl, N);
  const double *V = M.vstream[type];
  return __ldg(&V[k.iz * N + k.iR]) * (1 - k.fR) * (1 - k.fz) + __ldg(&V[(k.iz + 1) * N + k.iR]) * (1 - k.fR) * (k.fz) +
         __ldg(&V[k.iz * N + (k.iR + 1)]) * (k.fR) * (1 - k.fz) +
         __ldg(&V[(k.iz + 1) * N + (k.iR + 1)]) * (k.fR) * (k.fz);
}

// velocity projections of orbit_response.c:222-273 (= 338-391).  Rxy is
// sqrt(x[0]*x[0] + x[1]*x[1]), which the caller has already formed: it is the
// reference's q = sqrt(q2) bit for bit whenever x is finite (with
// Z = (0, 0, -1), Q = (-x1, x0, +-0) exactly, so q2 = x1*x1 + x0*x0 + 0).
struct Proj {
  double vr2, vt2, vq2, vp2;
};
__device__ __forceinline__ Proj project(const DevModel &M, int tovs, int type, const FgCoord &fc, const double *x,
                                        const double *v, double Rxy)
{
  Proj o;
  double r2, v_dot_x, q, q2, vq, v_dot_Q, t2, v_dot_T, vstr;
  const double Z0 = 0, Z1 = 0, Z2 = -1;
  double Q0, Q1, Q2, T0, T1, T2;
  if(tovs == 2) {
    r2 = x[0] * x[0] + x[1] * x[1];
    v_dot_x = v[0] * x[0] + v[1] * x[1];
    o.vr2 = v_dot_x * v_dot_x / r2;
    Q0 = -x[1];
    Q1 = x[0];
    q2 = Q0 * Q0 + Q1 * Q1;
    v_dot_Q = v[0] * Q0 + v[1] * Q1;
    q = Rxy;  // sqrt(q2): the same sum in the other order
    vq = v_dot_Q / q;
    o.vq2 = vq * vq;
    vstr = vstream_at(M, fc, type);
    o.vp2 = (vq - vstr) * (vq - vstr);
    o.vt2 = v[2] * v[2];
  } else {
    r2 = x[0] * x[0] + x[1] * x[1] + x[2] * x[2];
    v_dot_x = v[0] * x[0] + v[1] * x[1] + v[2] * x[2];
    o.vr2 = v_dot_x * v_dot_x / r2;
    Q0 = x[1] * Z2 - x[2] * Z1;
    Q1 = x[2] * Z0 - x[0] * Z2;
    Q2 = x[0] * Z1 - x[1] * Z0;
    q2 = Q0 * Q0 + Q1 * Q1 + Q2 * Q2;
    v_dot_Q = v[0] * Q0 + v[1] * Q1 + v[2] * Q2;
    q = Rxy;
    if(!(gm_fabs(x[0] + x[1] + x[2]) < GM_INF)) q = sqrt(q2);  // non-finite (or huge) x: as the reference
    vq = v_dot_Q / q;
    o.vq2 = vq * vq;
    vstr = vstream_at(M, fc, type);
    o.vp2 = (vq - vstr) * (vq - vstr);
    T0 = x[1] * Q2 - x[2] * Q1;
    T1 = x[2] * Q0 - x[0] * Q2;
    T2 = x[0] * Q1 - x[1] * Q0;
    t2 = T0 * T0 + T1 * T1 + T2 * T2;
    v_dot_T = v[0] * T0 + v[1] * T1 + v[2] * T2;
    o.vt2 = v_dot_T * v_dot_T / t2;
  }
  return o;
}

// get_timestep (orbit_response.c:16-26)
__device__ __forceinline__ double get_timestep(const DevModel &M, const double *v, const double *a, int icell)
{
  double vv = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
  double aa = sqrt(a[0] * a[0] + a[1] * a[1] + a[2] * a[2]);
  double torbit = M.V200 / aa;
  double tcross = __ldg(&M.cellsize[icell]) / vv;
  double t1 = M.f_orb * torbit, t2 = M.f_cc * tcross;
  return t1 < t2 ? t1 : t2;  // dmin, system.c:46
}

// One deposit of orbit_response.c:277-320: the weights m[a][b] of the four
// corners of cell k, and the projections.
struct Deposit {
  int iR, iz;
  double m00, m10, m01, m11;
  Proj p;
};
__device__ __forceinline__ Deposit make_deposit(double dt, const Cell &k, const Proj &p)
{
  Deposit d;
  d.iR = k.iR;
  d.iz = k.iz;
  d.m00 = 0.5 * dt * (1 - k.fR) * (1 - k.fz);
  d.m10 = 0.5 * dt * (k.fR) * (1 - k.fz);
  d.m01 = 0.5 * dt * (1 - k.fR) * (k.fz);
  d.m11 = 0.5 * dt * (k.fR) * (k.fz);
  d.p = p;
  return d;
}

// Orbit state of produce_orbit_response_field_mod (orbit_response.c:170-209)
struct OrbitState {
  double x[3], v[3], a[3];
  double tall, timespan, E0;
  bool rad_in;  // radsign_previous < 0: all the reference reads of it
  Cell cell;
  Proj proj;
  long long steps;
  int norbit, flag, type, tovs, status;
};

// orbit_response.c:181-209: copy the initial state, first acceleration, cell,
// projections and energy
__device__ __forceinline__ void orbit_begin(const DevModel &M, const LogConsts &L, OrbitState &s, const double *pos,
                                            const double *vel, double timespan, int type, bool with_proj)
{
  for(int i = 0; i < 3; i++) {
    s.x[i] = pos[i];
    s.v[i] = vel[i];
  }
  s.tall = 0;
  s.timespan = timespan;
  s.rad_in = false;
  s.norbit = 0;
  s.flag = 0;
  s.steps = 0;
  s.type = type;
  s.tovs = M.tovs[type];
  s.status = ORBIT_OK;
  FgCoord fc = fg_coord(M, L, s.x);
  forcegrid_acc(M, fc, s.x, s.a);
  s.cell = density_cell(M, L, s.x);
  s.E0 = 0.5 * (s.v[0] * s.v[0] + s.v[1] * s.v[1] + s.v[2] * s.v[2]) + forcegrid_pot(M, L, s.x);
  if(with_proj) s.proj = project(M, s.tovs, type, fc, s.x, s.v, sqrt(s.x[0] * s.x[0] + s.x[1] * s.x[1]));
}

// One iteration of the do-loop of orbit_response.c:211-458 (with_proj) or
// orbit_response.c:61-126 (mass only).  Calls sink(deposit) twice.  Returns
// false when the orbit has ended.
template <class Sink>
__device__ __forceinline__ bool orbit_step(const DevModel &M, const LogConsts &L, OrbitState &s, bool with_proj,
                                           Sink &sink)
{
  const int Nb = M.DG_Nbin;
  double dt = get_timestep(M, s.v, s.a, s.cell.iz * Nb + s.cell.iR);
  if(0 < s.timespan)
    if(s.timespan < dt + s.tall) {
      dt = s.timespan - s.tall;
      s.flag = 1;
    }
  sink(make_deposit(dt, s.cell, s.proj));
  for(int i = 0; i < 3; i++) s.v[i] += 0.5 * dt * s.a[i];
  for(int i = 0; i < 3; i++) s.x[i] += dt * s.v[i];
  // the four log coordinates of the new position (force grid: grid.c:130-136;
  // density grid: grid.c:494-534) in one block, so that their independent
  // chains interleave; the same expressions as fg_coord and density_cell
  const double Rxy = sqrt(s.x[0] * s.x[0] + s.x[1] * s.x[1]), az = gm_fabs(s.x[2]);
  const double lf0 = gm_log(div_by(Rxy, M.FG_Rmin, M.inv_FG_Rmin) + 1.0);
  const double lf1 = gm_log(div_by(az, M.FG_Rmin, M.inv_FG_Rmin) + 1.0);
  const double ld0 = gm_log(div_by(Rxy, M.DG_Rmin, M.inv_DG_Rmin) + 1.0);
  const double ld1 = gm_log(div_by(az, M.DG_Rmin, M.inv_DG_Rmin) + 1.0);
  FgCoord fc;
  fc.jdbl = div_by(lf0, L.lfg, M.inv_lfg);
  fc.idbl = div_by(lf1, L.lfg, M.inv_lfg);
  forcegrid_acc(M, fc, s.x, s.a);
  for(int i = 0; i < 3; i++) s.v[i] += 0.5 * dt * s.a[i];
  s.cell = cell_from_b(div_by(ld0, L.ldg, M.inv_ldg) - 0.5, div_by(ld1, L.ldg, M.inv_ldg) - 0.5, M.DG_Nbin);
  if(with_proj) s.proj = project(M, s.tovs, s.type, fc, s.x, s.v, Rxy);
  sink(make_deposit(dt, s.cell, s.proj));
  s.tall += dt;
  double radsign = s.v[0] * s.x[0] + s.v[1] * s.x[1] + s.v[2] * s.x[2];
  if(radsign > 0 && s.rad_in) s.norbit++;
  s.rad_in = radsign < 0;
  s.steps++;
  if(!(s.tall == s.tall) || !(dt == dt)) {
    s.status = ORBIT_NONFINITE;
    return false;
  }
  if(s.steps > M.step_cap) {
    s.status = ORBIT_STEP_CAP;
    return false;
  }
  // (timespan == 0 && norbit < Norbits) continues until the step cap, as in
  // the reference (Norbits = 1e8)
  return (s.timespan == 0 && s.norbit < 100000000) || (s.timespan != 0 && s.flag == 0);
}

// orbit_response.c:460-462: relative energy error of the finished orbit
__device__ __forceinline__ double orbit_energy_error(const DevModel &M, const LogConsts &L, const OrbitState &s)
{
  double E1 = 0.5 * (s.v[0] * s.v[0] + s.v[1] * s.v[1] + s.v[2] * s.v[2]) + forcegrid_pot(M, L, s.x);
  return gm_fabs((E1 - s.E0) / s.E0);
}
// the same, with E0 formed again from the orbit's initial position and
// velocity (orbit_begin's expression, so the same value), for kernels that
// would rather not hold E0 for the whole orbit
__device__ __forceinline__ double orbit_energy_error_from(const DevModel &M, const LogConsts &L, const OrbitState &s,
                                                          const double *pos0, const double *vel0)
{
  const double E0 = 0.5 * (vel0[0] * vel0[0] + vel0[1] * vel0[1] + vel0[2] * vel0[2]) + forcegrid_pot(M, L, pos0);
  double E1 = 0.5 * (s.v[0] * s.v[0] + s.v[1] * s.v[1] + s.v[2] * s.v[2]) + forcegrid_pot(M, L, s.x);
  return gm_fabs((E1 - E0) / E0);
}

// calc_disp_components_for_particle (disp_fields.c:200-372); out = vr2, vt2, vp2, vq2
__device__ __forceinline__ void disp_components(const DevModel &M, const LogConsts &L, int type, const double *pos,
                                                const double *vel, double *out)
{
  int tovs = M.tovs[type];
  if(tovs == 0 || tovs == 1 || tovs == 3) {
    double phi = gm_atan2(pos[1], pos[0]);
    double theta = gm_acos(pos[2] / sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]));
    double st, ct, sp, cp;
    gm_sincos(theta, &st, &ct);
    gm_sincos(phi, &sp, &cp);
    double er0 = st * cp, er1 = st * sp, er2 = ct;
    double ep0 = -sp, ep1 = cp, ep2 = 0;
    double et0 = -ct * cp, et1 = -ct * sp, et2 = st;
    double vr = vel[0] * er0 + vel[1] * er1 + vel[2] * er2;
    double vphi = vel[0] * ep0 + vel[1] * ep1 + vel[2] * ep2;
    double vtheta = vel[0] * et0 + vel[1] * et1 + vel[2] * et2;
    double vstr = 0;
    if(tovs == 1 || tovs == 3) vstr = vstream_at(M, fg_coord(M, L, pos), type);
    out[0] = vr * vr;
    out[1] = vtheta * vtheta;
    out[2] = (vphi - vstr) * (vphi - vstr);
    out[3] = vphi * vphi;
  } else if(tovs == 2) {
    double phi = gm_atan2(pos[1], pos[0]);
    double cp, sp;
    gm_sincos(phi, &sp, &cp);
    double eR0 = cp, eR1 = sp, eR2 = 0;
    double ep0 = -sp, ep1 = cp, ep2 = 0;
    double ez0 = 0, ez1 = 0, ez2 = 1;
    double vR = vel[0] * eR0 + vel[1] * eR1 + vel[2] * eR2;
    double vphi = vel[0] * ep0 + vel[1] * ep1 + vel[2] * ep2;
    double vZ = vel[0] * ez0 + vel[1] * ez1 + vel[2] * ez2;
    double vstr = vstream_at(M, fg_coord(M, L, pos), type);
    out[0] = vR * vR;
    out[1] = vZ * vZ;
    out[2] = (vphi - vstr) * (vphi - vstr);
    out[3] = vphi * vphi;
  } else {
    out[0] = out[1] = out[2] = out[3] = 0;
  }
}

#endif
