// Host-side grid geometry of GALIC (set-up code the hot path consumes).
//
// galic_grid_geometry    forcedensitygrid_create, grid.c:329-480
// galic_density_geometry DGs_Distance grid.c:381-416, DG_CellSize/Vol grid.c:830-850
// galic_smooth_stack     smooth_stack, grid.c:1247-1265
//
// These run once per model on the host and feed the device tables; they use
// the host libm (std::log/pow/exp), as the reference does.
#include <cmath>
#include <vector>

#include "galic_gpu.h"

namespace {

inline int stack_offset(int l, int i, int j) { return (((1 << (2 * l)) - 1) / 3) + i * (1 << l) + j; }

// Newton solve for the log-grid spacing factor: the outer edge of bin nbin
// sits at y times the inner edge (grid.c:358-372, 429-443, 461-475).
bool solve_spacing(double y, int nbin, double *out)
{
  double fac = 1.02, dfac;
  int iter = 0;
  do {
    double f = std::log((std::pow(fac, nbin) - 1.0) / (y * (fac - 1.0)));
    double df = nbin / (fac - 1.0 / std::pow(fac, nbin - 1)) - 1.0 / (fac - 1.0);
    dfac = -f / df;
    fac += dfac;
    if(++iter > 1000) return false;
  } while(std::fabs(dfac) > 1.0e-8 * fac);
  // Started from 1.02 the iteration can settle on the spurious root below 1
  // when nbin is large compared with log(y) (e.g. 256 bins for y = 233); the
  // reference then runs with a negative Rmin.  Reject that geometry.
  if(!(fac > 1.0)) return false;
  *out = fac;
  return true;
}

}  // namespace

extern "C" int galic_grid_geometry(double halo_a, double outer_frac, double inner_frac, int fg_nbin,
                                   int dg_maxlevel, int eg_maxlevel, double *out)
{
  if(!out || !(halo_a > 0) || !(outer_frac > 0 && outer_frac < 1) || !(inner_frac > 0 && inner_frac < outer_frac) ||
     fg_nbin < 2 || dg_maxlevel < 1 || dg_maxlevel > 12 || eg_maxlevel < 1 || eg_maxlevel > 12)
    return GALIC_ERR_INVALID_ARGUMENT;
  // Hernquist radius enclosing a mass fraction f: a (f + sqrt f) / (1 - f)
  double rmax = halo_a * (outer_frac + std::sqrt(outer_frac)) / (1 - outer_frac);
  double rin = halo_a * (inner_frac + std::sqrt(inner_frac)) / (1 - inner_frac);
  double dgf, fgf, egf;
  if(!solve_spacing(rmax / rin, 1 << dg_maxlevel, &dgf) || !solve_spacing(rmax / rin, fg_nbin, &fgf) ||
     !solve_spacing(rmax / rin, 1 << eg_maxlevel, &egf))
    return GALIC_ERR_INVALID_ARGUMENT;
  out[0] = rmax;
  out[1] = rin;
  out[2] = dgf;
  out[3] = rin / (dgf - 1.0);
  out[4] = fgf;
  out[5] = rin / (fgf - 1.0);
  out[6] = egf;
  out[7] = rin / (egf - 1.0);
  return GALIC_OK;
}

extern "C" void galic_smooth_stack(double *data, int maxlevel)
{
  for(int l = maxlevel - 1; l >= 0; l--) {
    int n = 1 << l;
    for(int i = 0; i < n; i++)
      for(int j = 0; j < n; j++)
        data[stack_offset(l, i, j)] = data[stack_offset(l + 1, 2 * i, 2 * j)] +
                                      data[stack_offset(l + 1, 2 * i + 1, 2 * j)] +
                                      data[stack_offset(l + 1, 2 * i, 2 * j + 1)] +
                                      data[stack_offset(l + 1, 2 * i + 1, 2 * j + 1)];
  }
}

extern "C" int galic_density_geometry(int L, double rmin, double fac, double *dist, double *cellsize,
                                      double *cellvol)
{
  if(L < 1 || L > 12 || !(rmin > 0) || !(fac > 1) || !dist || !cellsize || !cellvol)
    return GALIC_ERR_INVALID_ARGUMENT;
  const int nbin = 1 << L, nstack = ((1 << (2 + 2 * L)) - 1) / 3;
  std::vector<double> logR(nstack), logZ(nstack);
  // log of the centre coordinates of every finest cell, averaged up the stack
  for(int k = 0; k < nbin; k++)
    for(int j = 0; j < nbin; j++) {
      double z = rmin * 0.5 * (std::pow(fac, k) + std::pow(fac, k + 1) - 2.0);
      double R = rmin * 0.5 * (std::pow(fac, j) + std::pow(fac, j + 1) - 2.0);
      logR[stack_offset(L, k, j)] = std::log(R);
      logZ[stack_offset(L, k, j)] = std::log(z);
    }
  galic_smooth_stack(logR.data(), L);
  galic_smooth_stack(logZ.data(), L);
  for(int l = L - 1; l >= 0; l--) {
    int n = 1 << l, f = 1 << (L - l);
    for(int i = 0; i < n; i++)
      for(int j = 0; j < n; j++) {
        logR[stack_offset(l, i, j)] /= (f * f);
        logZ[stack_offset(l, i, j)] /= (f * f);
      }
  }
  for(int l = L; l >= 0; l--) {
    int n = 1 << l;
    for(int i = 0; i < n; i++)
      for(int j = 0; j < n; j++) {
        int s = stack_offset(l, i, j);
        dist[s] = std::sqrt(std::pow(std::exp(logR[s]), 2) + std::pow(std::exp(logZ[s]), 2));
      }
  }
  for(int k = 0; k < nbin; k++)
    for(int j = 0; j < nbin; j++) {
      int i = k * nbin + j;
      double r1 = rmin * (std::pow(fac, j) - 1.0), r2 = rmin * (std::pow(fac, j + 1) - 1.0);
      double z1 = rmin * (std::pow(fac, k) - 1.0), z2 = rmin * (std::pow(fac, k + 1) - 1.0);
      double vol = M_PI * (r2 * r2 - r1 * r1) * (z2 - z1) * 2;  // both sides of z = 0
      cellsize[i] = (r2 - r1 > z2 - z1) ? r2 - r1 : z2 - z1;
      cellvol[i] = vol;
    }
  return GALIC_OK;
}
