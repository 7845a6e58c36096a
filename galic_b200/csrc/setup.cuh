// Device code shared by the set-up kernels (sampling.cu, particles.cu): the
// coordinate samplers of halo.c / disk.c / bulge.c and get_disp_rtp with its
// table lookups (disp_fields.c).  Every expression keeps the reference's
// operation order; built with --fmad=false and gmath.h's functions.
#ifndef GALIC_SETUP_CUH
#define GALIC_SETUP_CUH

#include "gmath.h"
#include "model.cuh"

namespace {

constexpr int NEWTON_CAP = 10000;               // disk.c:27-36 converges in < 30 steps; bounds the loop
constexpr double kPi = 3.14159265358979323846;  // M_PI

struct Shape {
  double Rmax, Halo_A, HaloStretch, Disk_Z0, Disk_H, Bulge_A, BulgeStretch;
};

// get_disp_rtp's tables and constants for one type (disp_fields.c:26-198, 375-398)
struct DispTab {
  const double *disp_r, *dispz, *dispphi, *tvr2, *tvz2, *vstream;  // FG_Nbin^2 each
  int tovs;
  double beta, beta_a;  // Halo/BulgeBetaParameter and the matching scale radius
  double FG_Rmin, lfg;
  int FG_Nbin;
};

// ---------------------------------------------------------------- samplers

// halo.c:21-39, one pass of the loop body from the draws (q, azimuth, polar);
// true when the point is kept (the loop's exit test)
__device__ __forceinline__ bool halo_draw(const Shape &S, double q, double uphi, double uth, double *pos)
{
  double r;
  if(q > 0)
    r = S.Halo_A * (q + sqrt(q)) / (1 - q);
  else
    r = 0;
  double phi = uphi * kPi * 2;
  double theta = gm_acos(uth * 2 - 1);
  pos[0] = r * gm_sin(theta) * gm_cos(phi);
  pos[1] = r * gm_sin(theta) * gm_sin(phi);
  pos[2] = r * gm_cos(theta) / S.HaloStretch;
  r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  return !(r > S.Rmax);
}

// disk.c:21-47, one pass of the loop body from the draws (height, radius, azimuth)
__device__ __forceinline__ bool disk_draw(const Shape &S, double q1, double q2, double uphi, double *pos)
{
  pos[2] = S.Disk_Z0 / 2 * gm_log(q1 / (1 - q1));
  double R = 1.0, Rold, f, f_;
  int it = 0;
  do {
    const double e = gm_exp(-R);  // the reference evaluates exp(-R) twice: same value
    f = (1 + R) * e + q2 - 1;
    f_ = -R * e;
    Rold = R;
    R = R - f / f_;
  } while(gm_fabs(R - Rold) / R > 1e-7 && ++it < NEWTON_CAP);
  R *= S.Disk_H;
  double phi = uphi * kPi * 2;
  pos[0] = R * gm_cos(phi);
  pos[1] = R * gm_sin(phi);
  double R2 = pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2];
  return !(R2 > S.Rmax * S.Rmax);
}

// bulge.c:19-28: the radius of draw q (redrawn while beyond Rmax)
__device__ __forceinline__ double bulge_radius(const Shape &S, double q)
{
  if(q > 0) return S.Bulge_A * (q + sqrt(q)) / (1 - q);
  return 0;
}
// bulge.c:30-36
__device__ __forceinline__ void bulge_place(const Shape &S, double r, double uphi, double uth, double *pos)
{
  double phi = uphi * kPi * 2;
  double theta = gm_acos(uth * 2 - 1);
  pos[0] = r * gm_sin(theta) * gm_cos(phi);
  pos[1] = r * gm_sin(theta) * gm_sin(phi);
  pos[2] = r * gm_cos(theta) / S.BulgeStretch;
}

// ---------------------------------------------------------------- dispersions

__device__ __forceinline__ double interp_fg(const double *T, const Cell &k, int N)
{
  return T[k.iz * N + k.iR] * (1 - k.fR) * (1 - k.fz) + T[(k.iz + 1) * N + k.iR] * (1 - k.fR) * (k.fz) +
         T[k.iz * N + (k.iR + 1)] * (k.fR) * (1 - k.fz) + T[(k.iz + 1) * N + (k.iR + 1)] * (k.fR) * (k.fz);
}

// get_radial_disp_spherical (disp_fields.c:375-398)
__device__ __forceinline__ double radial_disp(const DispTab &D, const double *pos)
{
  double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
  double br = (gm_log(r / D.FG_Rmin + 1.0) / D.lfg);
  const int N = D.FG_Nbin;
  if(br < 0) br = 0;
  int binr = (br < (double) (N - 1)) ? (int) br : N - 1;
  double fR = br - binr;
  if(binr >= N - 1) {
    binr = N - 2;
    fR = 1;
  }
  return D.disp_r[binr] * (1 - fR) + D.disp_r[binr + 1] * (fR);
}

// get_beta_of_type (disp_fields.c:26-60): D.beta is the type's parameter
// (0 for the disk), D.beta_a the matching scale radius
__device__ __forceinline__ double beta_of(const DispTab &D, const double *pos)
{
  double beta = D.beta;
  if(beta >= 1) {
    double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    double dlogrhodr = -1.0 - 3.0 * r / (r + D.beta_a);
    beta = -0.15 - 0.20 * dlogrhodr;
  }
  return beta;
}

// get_disp_rtp (disp_fields.c:66-115)
__device__ __forceinline__ void disp_rtp(const DispTab &D, const double *pos, double *d)
{
  if(D.tovs == 0) {
    d[0] = radial_disp(D, pos);
    d[1] = d[2] = d[3] = d[0];
  } else if(D.tovs == 1) {
    d[0] = radial_disp(D, pos);
    d[1] = (1 - beta_of(D, pos)) * d[0];
    d[2] = d[3] = d[1];
  } else {
    // forcegrid_get_cell (grid.c:15-55)
    double R = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
    double jdbl = gm_log(R / D.FG_Rmin + 1.0) / D.lfg;
    double idbl = gm_log(gm_fabs(pos[2]) / D.FG_Rmin + 1.0) / D.lfg;
    Cell k = cell_from_b(jdbl, idbl, D.FG_Nbin);
    const int N = D.FG_Nbin;
    double vstr = D.vstream ? interp_fg(D.vstream, k, N) : 0.0;
    if(D.tovs == 2) {
      d[1] = interp_fg(D.dispz, k, N);
      d[0] = d[1];
      d[2] = interp_fg(D.dispphi, k, N);
    } else {
      d[0] = interp_fg(D.tvr2, k, N);
      d[1] = interp_fg(D.tvz2, k, N);
      d[2] = interp_fg(D.dispphi, k, N);
    }
    d[3] = d[2] + vstr * vstr;
  }
}

}  // namespace

#endif
