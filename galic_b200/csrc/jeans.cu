// calculate_dispfield (disp_fields.c:502-1049) on the GPU: the Jeans tables
// FG_Disp_r, FG_DispZ, FG_DispPhi, FG_Vstream and, for velocity structure 3,
// FG_tilted_*.
//
// The reference's solvers march sequentially (outer radius to centre, top
// row to mid-plane), but every density, anisotropy, tilt factor and force
// they evaluate depends only on the grid point, never on the running
// solution.  So each part splits into a wide kernel that evaluates all of
// those coefficients in parallel and a narrow kernel that runs the
// recurrence in the reference's order with the coefficients it would have
// computed:
//  * spherical Jeans (disp_fields.c:512-570): coefficients of the 50 Heun
//    steps of all N+1 radial intervals (k_sph_coef), then one thread per
//    type runs the steps (k_sph_march), then the division by the density;
//  * axisymmetric f(E, Lz) (disp_fields.c:575-729): the integrand at the 51
//    points of every z interval of every column (k_axi_points), then one
//    thread per column sums the trapezoids in the reference's order
//    (k_axi_march), then DispPhi / Vstream per grid point (k_axi_stream);
//  * tilted f(E, Lz, I3) (disp_fields.c:733-1044): the coefficients of the
//    100 method-of-lines substeps of every row (k_tilt_coef, 313 MB at
//    N = 256), then one CTA, a thread per column, steps the rows with the
//    neighbour exchange in shared memory (k_tilt_march); then the tilted
//    tables and the VER_1_1 streaming velocity per grid point.
// Every expression keeps the reference's operation order and the file is
// built with --fmad=false, so the tables are bit-identical to the CPU
// restatement with gmath.h's functions.  The grid radii
// FG_Rmin (FG_Fac^j - 1) come from the C library's pow on the host.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <vector>

#include "context.cuh"
#include "galic_gpu.h"
#include "model.cuh"

#include <cuda_pipeline.h>

namespace {

constexpr double kPi = 3.14159265358979323846;  // M_PI
constexpr double MIN_DENSITY = 1e-25;           // allvars.h:201
constexpr int SPH_STEPS = 50;                   // disp_fields.c:458
constexpr int AXI_STEPS = 50;                   // disp_fields.c:429
constexpr int TILT_STEPS = 100;                 // disp_fields.c:784
constexpr int NTAB = 8;  // disp_r, dispz, dispphi, vstream, tilted_vz2, tilted_vR2, tilted_vz2_prime, tilted_vR2_prime

struct JeansArgs {
  DevModel M;
  const double *Rg;  // FG_Rmin * (pow(FG_Fac, j) - 1.0), j = 0 .. 2N + 2
  int N, type;
  double HaloStretch, Halo_Mass, Halo_A, Disk_Mass, Disk_H, Disk_Z0, Bulge_Mass, Bulge_A, BulgeStretch;
  double beta, beta_a;  // get_beta_of_type's parameter and scale radius for this type
  double f, kpar;       // DispersionRoverZratio, StreamingVelocityParameter of this type
  double *tab;          // [NTAB][N * N] of this type
};

__device__ __forceinline__ double tan_(double x) { return gm_sin(x) / gm_cos(x); }
__device__ __forceinline__ double atan_(double x) { return gm_atan2(x, 1.0); }

// get_density_of_type (disp_fields.c:11-24; halo.c:43-54, disk.c:53-69, bulge.c:39-48)
__device__ double density(const JeansArgs &J, const double *pos)
{
  double rho;
  if(J.type == 1) {
    double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + J.HaloStretch * J.HaloStretch * pos[2] * pos[2]);
    const double ra = r + J.Halo_A;
    rho = J.HaloStretch * J.Halo_Mass / (2 * kPi) * J.Halo_A / (r + 1.0e-6 * J.Halo_A) / (ra * ra * ra);
  } else if(J.type == 2) {
    if(!(J.Disk_Mass > 0)) return 0;
    double R = sqrt(pos[0] * pos[0] + pos[1] * pos[1]);
    double z = pos[2];
    const double s = 2 / (gm_exp(z / J.Disk_Z0) + gm_exp(-z / J.Disk_Z0));
    rho = J.Disk_Mass / (4 * kPi * J.Disk_H * J.Disk_H * J.Disk_Z0) * gm_exp(-R / J.Disk_H) * (s * s);
  } else {
    double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    const double ra = r + J.Bulge_A;
    rho = J.BulgeStretch * J.Bulge_Mass / (2 * kPi) * J.Bulge_Mass / (r + 1.0e-6 * J.Bulge_A) / (ra * ra * ra);
  }
  if(gm_fabs(rho) < MIN_DENSITY) rho = 0;
  return rho;
}

// get_beta_of_type (disp_fields.c:26-60)
__device__ __forceinline__ double beta_of(const JeansArgs &J, const double *pos)
{
  double beta = J.beta;
  if(J.type != 2 && beta >= 1) {
    double r = sqrt(pos[0] * pos[0] + pos[1] * pos[1] + pos[2] * pos[2]);
    double dlogrhodr = -1.0 - 3.0 * r / (r + J.beta_a);
    beta = -0.15 - 0.20 * dlogrhodr;
  }
  return beta;
}

// forcegrid_get_acceleration (grid.c:122-197)
__device__ __forceinline__ void fg_acc(const JeansArgs &J, const LogConsts &L, const double *pos, double *acc)
{
  FgCoord c = fg_coord(J.M, L, pos);
  forcegrid_acc(J.M, c, pos, acc);
}

__device__ __forceinline__ double tilt_den(double f, double alpha)
{
  const double c = gm_cos(alpha), s = gm_sin(alpha);
  return c * c - f * (s * s) + (1.0 + f) / 2.0 * gm_sin(2 * alpha) * tan_(2 * alpha);
}

// h_factor (disp_fields.c:1051-1077)
__device__ double h_factor(const JeansArgs &J, double R, double z)
{
  double fac;
  if(R <= 1.0e-12 * z || R == 0)
    fac = 0;
  else {
    double alpha = atan_(z / R);
    fac = ((J.f - 1) / 2 * tan_(2 * alpha)) / tilt_den(J.f, alpha);
  }
  return fac;
}

// h_over_R (disp_fields.c:1079-1105); z > 0 on every call
__device__ double h_over_r(const JeansArgs &J, double R, double z)
{
  double fac;
  if(R <= 1.0e-12 * z || R == 0)
    fac = (J.f - 1) / J.f;
  else {
    double alpha = atan_(z / R);
    fac = ((J.f - 1) / 2 * tan_(alpha) * tan_(2 * alpha)) / tilt_den(J.f, alpha);
  }
  return fac / z;
}

__device__ __forceinline__ double *table(const JeansArgs &J, int w) { return J.tab + (size_t) w * J.N * J.N; }

// ---------------------------------------------------------------- spherical

struct SphCoef {
  double a0, c0, a1, c1, dr;
  int flag;  // 2: Heun step, 1: Euler step, 0: no change (disp_fields.c:488-496)
};

// interval m: 0 is [R(N+2) -> R(N)], m >= 1 is [R(j+1) -> R(j)] with j = N - m
__global__ void k_sph_coef(const JeansArgs J, SphCoef *coef)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  if(t >= (J.N + 1) * SPH_STEPS) return;
  const int m = t / SPH_STEPS, i = t - m * SPH_STEPS;
  const int N = J.N;
  const double rstart = (m == 0) ? J.Rg[N + 2] : J.Rg[N - m + 1];
  const double rend = (m == 0) ? J.Rg[N] : J.Rg[N - m];
  const LogConsts L = make_log_consts(J.M);
  // integrate_spherical_jeans_beta (disp_fields.c:456-499), step i
  double dr = (rend - rstart) / SPH_STEPS;
  double r0 = rstart + i * dr;
  double r1 = rstart + (i + 1) * dr;
  double pos0[3] = {r0, 0, 0};
  double pos1[3] = {r1, 0, 0};
  double beta0 = beta_of(J, pos0);
  double beta1 = beta_of(J, pos1);
  double acc[3];
  double dens0 = density(J, pos0);
  fg_acc(J, L, pos0, acc);
  double acc0 = acc[0];
  double dens1 = density(J, pos1);
  fg_acc(J, L, pos1, acc);
  double acc1 = acc[0];
  SphCoef c;
  c.a0 = dens0 * acc0;
  c.c0 = 2 * beta0 / r0;
  c.a1 = dens1 * acc1;
  c.c1 = 2 * beta1 / r1;
  c.dr = dr;
  c.flag = (r1 > gm_fabs(dr) && r0 > gm_fabs(dr)) ? 2 : (r0 > gm_fabs(dr) ? 1 : 0);
  coef[t] = c;
}

// One thread runs the recurrence; the other threads of the CTA stage the
// next chunk of coefficients in shared memory meanwhile.
constexpr int SPH_CHUNK = 256;

__global__ void __launch_bounds__(256) k_sph_march(const JeansArgs J, const SphCoef *coef)
{
  __shared__ SphCoef buf[2][SPH_CHUNK];
  const int total = (J.N + 1) * SPH_STEPS;
  double *disp_r = table(J, 0);
  for(int t = threadIdx.x; t < SPH_CHUNK && t < total; t += blockDim.x) buf[0][t] = coef[t];
  __syncthreads();
  double y = 0.0;
  int b = 0;
  for(int c0 = 0; c0 < total; c0 += SPH_CHUNK, b ^= 1) {
    const int n1 = c0 + SPH_CHUNK;
    if(threadIdx.x > 0) {
      for(int t = threadIdx.x - 1; t < SPH_CHUNK && n1 + t < total; t += blockDim.x - 1) buf[b ^ 1][t] = coef[n1 + t];
    } else {
      for(int t = 0; t < SPH_CHUNK && c0 + t < total; t++) {
        const SphCoef c = buf[b][t];
        if(c.flag == 2) {
          double ypred = y + c.dr * (c.a0 - c.c0 * y);
          y += c.dr * 0.5 * ((c.a0 - c.c0 * y) + (c.a1 - c.c1 * ypred));
        } else if(c.flag == 1) {
          y += c.dr * (c.a0 - c.c0 * y);
        }
        const int g = c0 + t;
        if((g + 1) % SPH_STEPS == 0) {
          const int m = g / SPH_STEPS;
          if(m >= 1) disp_r[J.N - m] = y;
        }
      }
    }
    __syncthreads();
  }
}

__global__ void k_sph_divide(const JeansArgs J)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if(j >= J.N) return;
  double *disp_r = table(J, 0);
  double pos[3] = {J.Rg[j], 0, 0};
  double dens = density(J, pos);
  if(dens > 0)
    disp_r[j] /= dens;
  else
    disp_r[j] = 0;
}

// ---------------------------------------------------------------- axisymmetric

// interval m of column j: 0 is [R(N), R(2N)], m >= 1 is [R(k), R(k+1)] with k = N - m
__device__ __forceinline__ void axi_interval(const JeansArgs &J, int m, double *zstart, double *zend)
{
  const int N = J.N;
  *zstart = (m == 0) ? J.Rg[N] : J.Rg[N - m];
  *zend = (m == 0) ? J.Rg[2 * N] : J.Rg[N - m + 1];
}

// integrate_axisymmetric_jeans (disp_fields.c:427-453): the integrand at the
// 51 points zstart + i dz (point i + 1 is the reference's z1 of step i and z0
// of step i + 1: the same expression, the same value)
__global__ void k_axi_points(const JeansArgs J, double *Y)
{
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  const int P = AXI_STEPS + 1;
  const long long total = (long long) J.N * (J.N + 1) * P;
  if(t >= total) return;
  // Y[(j * (N + 1) + m) * P + i]: one column's points are contiguous
  const int i = (int) (t % P);
  const long long cm = t / P;
  const int m = (int) (cm % (J.N + 1));
  const int j = (int) (cm / (J.N + 1));
  double zstart, zend;
  axi_interval(J, m, &zstart, &zend);
  const LogConsts L = make_log_consts(J.M);
  double dz = (zend - zstart) / AXI_STEPS;
  double z = zstart + i * dz;
  double pos[3] = {J.Rg[j], 0, z};
  double acc[3];
  fg_acc(J, L, pos, acc);
  Y[t] = -acc[2] * density(J, pos);
}

__global__ void k_axi_march(const JeansArgs J, const double *Y)
{
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if(j >= J.N) return;
  const int N = J.N, P = AXI_STEPS + 1;
  double *dispz = table(J, 1);
  const double R = J.Rg[j];
  double integ = 0;
  for(int m = 0; m <= N; m++) {
    double zstart, zend;
    axi_interval(J, m, &zstart, &zend);
    double dz = (zend - zstart) / AXI_STEPS;
    // the interval's 51 points are loaded together, then summed in order
    const double *y = Y + ((size_t) j * (N + 1) + m) * P;
    double v[AXI_STEPS + 1];
#pragma unroll
    for(int i = 0; i <= AXI_STEPS; i++) v[i] = y[i];
    double sum = 0;
#pragma unroll
    for(int i = 0; i < AXI_STEPS; i++) sum += 0.5 * (v[i] + v[i + 1]) * dz;
    if(m == 0) {
      integ = sum;
    } else {
      const int k = N - m;
      integ += sum;
      double pos[3] = {R, 0, J.Rg[k]};
      double dens = density(J, pos);
      dispz[k * N + j] = (dens > 0) ? integ / dens : 0;
    }
  }
}

// disp_fields.c:638-698: DispPhi and Vstream from FG_DispZ
__global__ void k_axi_stream(const JeansArgs J)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = J.N;
  if(t >= N * N) return;
  const int k = t / N, j = t - k * N;
  const double *DispZ = table(J, 1);
  double *DispPhi = table(J, 2), *Vstream = table(J, 3);
  const LogConsts L = make_log_consts(J.M);
  double z = J.Rg[k];
  double R = J.Rg[j];
  double pos[3], acc[3], R1, R2;
  int i1, i2;
  pos[0] = R;
  pos[1] = 0;
  pos[2] = z;
  fg_acc(J, L, pos, acc);
  const int i = k * N + j;
  if(j > 1 && j < N - 1) {
    R1 = J.Rg[j - 1];
    i1 = k * N + j - 1;
    R2 = J.Rg[j + 1];
    i2 = k * N + j + 1;
  } else if(j == 1) {
    R1 = J.Rg[j];
    i1 = k * N + j;
    R2 = J.Rg[j + 1];
    i2 = k * N + j + 1;
  } else if(j == 0) {
    R1 = J.Rg[j + 1];
    i1 = k * N + j + 1;
    R2 = J.Rg[j + 2];
    i2 = k * N + j + 2;
  } else {
    R1 = J.Rg[j - 1];
    i1 = k * N + j - 1;
    R2 = J.Rg[j];
    i2 = k * N + j;
  }
  pos[0] = R1;
  double dens1 = density(J, pos);
  pos[0] = R2;
  double dens2 = density(J, pos);
  double dlog = 0;
  if(dens1 * DispZ[i1] > 0 && dens2 * DispZ[i2] > 0)
    dlog = gm_log((dens2 * DispZ[i2]) / (dens1 * DispZ[i1])) / gm_log(R2 / R1);
  double Vphi2 = DispZ[i] + R * (-acc[0]) + DispZ[i] * dlog;
  if(Vphi2 > 0) {
    double vstr = 0;
    if(Vphi2 >= DispZ[i]) vstr = J.kpar * sqrt((Vphi2 - DispZ[i]));
    DispPhi[i] = Vphi2 - vstr * vstr;
    Vstream[i] = vstr;
  } else {
    DispPhi[i] = 0;
    Vstream[i] = 0;
  }
}

// ---------------------------------------------------------------- tilted

struct alignas(16) TiltCoef {
  double p, h1, h2, dR, hor;
  int nb;  // neighbour column of dqdR, -1: dqdR = 0
  int pad;
};
static_assert(sizeof(TiltCoef) == 48, "three 16-byte copies per coefficient");

// rows k in [k_lo, k_hi] (all < N - 1), substep st, column j
// (disp_fields.c:775-835)
__global__ void k_tilt_coef(const JeansArgs J, int k_lo, int k_hi, TiltCoef *coef)
{
  const int N = J.N;
  const long long t = (long long) blockIdx.x * blockDim.x + threadIdx.x;
  const long long per_row = (long long) TILT_STEPS * N;
  if(t >= per_row * (k_hi - k_lo + 1)) return;
  const int r = (int) (t / per_row);
  const int rem = (int) (t - r * per_row);
  const int st = rem / N, j = rem - st * N;
  const int k = k_hi - r;  // rows in marching order
  const LogConsts L = make_log_consts(J.M);
  double z0 = J.Rg[k + 1];
  double z1 = J.Rg[k];
  double dz = (z1 - z0);
  double z = z0 + (dz / TILT_STEPS) * st;
  double R1 = J.Rg[j];
  TiltCoef c;
  c.h1 = h_factor(J, R1, z);
  double pos[3] = {R1, 0, z}, acc[3];
  double dens = density(J, pos);
  fg_acc(J, L, pos, acc);
  c.p = -dens * acc[2];
  c.h2 = c.dR = c.hor = 0;
  if(c.h1 > 0)
    c.nb = (j == N - 1) ? -1 : j + 1;
  else
    c.nb = (j == 0) ? j + 1 : j - 1;
  if(c.nb >= 0) {
    double R2 = J.Rg[c.nb];
    c.h2 = h_factor(J, R2, z);
    c.dR = R2 - R1;
    c.hor = h_over_r(J, R1, z);
  }
  coef[t] = c;
}

// one CTA, a thread per column (N <= blockDim.x): the substeps of rows
// k_hi .. k_lo (disp_fields.c:775-839); FG_q holds the row above on entry.
// Each thread streams its own coefficients D substeps ahead into a ring in
// shared memory with asynchronous copies (only the thread that reads a slot
// writes it, so no barrier guards the ring); the row alternates between two
// shared buffers, one barrier per substep.
template <int MAXT, int D>
__global__ void __launch_bounds__(MAXT) k_tilt_march(const JeansArgs J, int k_lo, int k_hi, const TiltCoef *coef,
                                                     double *FG_q)
{
  extern __shared__ __align__(16) unsigned char smem[];
  const int N = J.N, j = threadIdx.x;
  const bool active = j < N;
  TiltCoef *ring = reinterpret_cast<TiltCoef *>(smem);     // [D][N]
  double *qb = reinterpret_cast<double *>(ring + (size_t) D * N);  // [2][N]
  const int steps = (k_hi - k_lo + 1) * TILT_STEPS;
  if(active) qb[j] = FG_q[(size_t) (k_hi + 1) * N + j];
#pragma unroll
  for(int u = 0; u < D; u++) {
    if(active && u < steps) {
      const char *src = reinterpret_cast<const char *>(coef + (size_t) u * N + j);
      char *dst = reinterpret_cast<char *>(ring + (size_t) u * N + j);
      __pipeline_memcpy_async(dst, src, 16);
      __pipeline_memcpy_async(dst + 16, src + 16, 16);
      __pipeline_memcpy_async(dst + 32, src + 32, 16);
    }
    __pipeline_commit();
  }
  __syncthreads();
  int cur = 0;
  double step = 0;
  for(int g = 0; g < steps; g++) {
    const int k = k_hi - g / TILT_STEPS, st = g - (g / TILT_STEPS) * TILT_STEPS;
    if(st == 0) step = (J.Rg[k] - J.Rg[k + 1]) / TILT_STEPS;  // dz / nsteps
    __pipeline_wait_prior(D - 1);  // this thread's copy of substep g has landed
    const int slot = g % D;
    if(active) {
      const TiltCoef c = ring[(size_t) slot * N + j];
      const double *qp = qb + cur * N;
      double dqdR;
      if(c.nb < 0)
        dqdR = 0;
      else
        dqdR = (c.h2 * qp[c.nb] - c.h1 * qp[j]) / (c.dR) + qp[j] * c.hor;
      qb[(cur ^ 1) * N + j] = qp[j] + (-c.p - dqdR) * step;
      if(g + D < steps) {
        const char *src = reinterpret_cast<const char *>(coef + (size_t) (g + D) * N + j);
        char *dst = reinterpret_cast<char *>(ring + (size_t) slot * N + j);
        __pipeline_memcpy_async(dst, src, 16);
        __pipeline_memcpy_async(dst + 16, src + 16, 16);
        __pipeline_memcpy_async(dst + 32, src + 32, 16);
      }
    }
    __pipeline_commit();
    __syncthreads();
    cur ^= 1;
    if(active && st == TILT_STEPS - 1) FG_q[(size_t) k * N + j] = qb[cur * N + j];
  }
}

// disp_fields.c:849-898: tilted_vz2 = q / rho and the tilted rotation
__global__ void k_tilt_tables(const JeansArgs J, const double *FG_q)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = J.N;
  if(t >= N * N) return;
  const int k = t / N, j = t - k * N;
  double *tvz2 = table(J, 4), *tvR2 = table(J, 5), *tvz2p = table(J, 6), *tvR2p = table(J, 7);
  double R = J.Rg[j];
  double z = J.Rg[k];
  double pos[3] = {R, 0, z};
  double dens = density(J, pos);
  const double vz2 = (dens > 0) ? FG_q[t] / dens : 0;
  tvz2[t] = vz2;
  const double f = J.f;
  if(j > 0) {
    double alpha = atan_(z / R);
    const double c = gm_cos(alpha), s = gm_sin(alpha);
    const double den = tilt_den(f, alpha);
    double vrvz = vz2 * ((f - 1) / 2 * tan_(2 * alpha)) / den;
    double vr2 = vz2 * (f * (c * c) - s * s + (1.0 + f) / 2.0 * gm_sin(2 * alpha) * tan_(2 * alpha)) / den;
    double vr2_prime = vr2 * (c * c) + 2 * vrvz * s * c + vz2 * (s * s);
    double vz2_prime = vr2 * (s * s) - 2 * vrvz * s * c + vz2 * (c * c);
    tvR2[t] = vr2;
    tvz2p[t] = vz2_prime;
    tvR2p[t] = vr2_prime;
  } else {
    tvR2[t] = vz2 / f;
    tvz2p[t] = tvR2[t];
    tvR2p[t] = vz2;
  }
}

// disp_fields.c:902-988 (VER_1_1): DispPhi and Vstream from the tilted tables
__global__ void k_tilt_stream(const JeansArgs J)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int N = J.N;
  if(t >= N * N) return;
  const int k = t / N, j = t - k * N;
  const double *tvz2 = table(J, 4), *tvR2 = table(J, 5);
  double *DispPhi = table(J, 2), *Vstream = table(J, 3);
  const LogConsts L = make_log_consts(J.M);
  double z = J.Rg[k];
  double R = J.Rg[j];
  double pos[3] = {R, 0, z}, acc[3];
  double dens = density(J, pos);
  fg_acc(J, L, pos, acc);
  const int i = t;
  double Vphi2 = 0;
  if(dens > 0) {
    int j1 = (0 < j ? j - 1 : j);
    int j2 = (j < N - 1 ? j + 1 : j);
    int i1 = k * N + j1;
    int i2 = k * N + j2;
    double R1 = J.Rg[j1];
    double R2 = J.Rg[j2];
    pos[0] = R1;
    double dens1 = density(J, pos);
    pos[0] = R2;
    double dens2 = density(J, pos);
    Vphi2 = tvR2[i] + R / dens * (dens2 * tvR2[i2] - dens1 * tvR2[i1]) / (R2 - R1) + R * (-acc[0]) +
            R / dens * (dens2 * h_factor(J, R2, z) * tvz2[i2] - dens1 * h_factor(J, R1, z) * tvz2[i1]) / (R2 - R1);
  }
  if(Vphi2 > 0) {
    double vstr = 0;
    if(Vphi2 >= tvR2[i]) vstr = J.kpar * sqrt((Vphi2 - tvR2[i]));
    DispPhi[i] = Vphi2 - vstr * vstr;
    Vstream[i] = vstr;
  } else {
    DispPhi[i] = 0;
    Vstream[i] = 0;
  }
}

#define JCK(call)                                                                             \
  do {                                                                                        \
    cudaError_t e_ = (call);                                                                  \
    if(e_ != cudaSuccess) {                                                                   \
      fprintf(stderr, "galic_cuda: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                      \
      rc = GALIC_ERR_CUDA;                                                                    \
      goto done;                                                                              \
    }                                                                                         \
  } while(0)

int jfail(galic_ctx *ctx, int st)
{
  if(ctx) ctx->status = st;
  return st;
}

inline int blocks(long long n, int b) { return (int) ((n + b - 1) / b); }

size_t march_smem(int N, int D) { return (size_t) D * N * sizeof(TiltCoef) + 2 * (size_t) N * sizeof(double); }

// the marches' shared-memory ceiling, once per device
cudaError_t prepare_march()
{
  static bool done[256];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if(e || (dev >= 0 && dev < 256 && done[dev])) return e;
  if((e = cudaFuncSetAttribute(k_tilt_march<512, 8>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int) march_smem(512, 8))))
    return e;
  if((e = cudaFuncSetAttribute(k_tilt_march<1024, 4>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               (int) march_smem(1024, 4))))
    return e;
  if(dev >= 0 && dev < 256) done[dev] = true;
  return cudaSuccess;
}

}  // namespace

extern "C" int galic_calculate_dispfield(galic_ctx *ctx, const galic_sample_params_t *sp,
                                         const galic_jeans_params_t *jp, galic_jeans_tables_t *out)
{
  if(!ctx) return GALIC_ERR_INVALID_ARGUMENT;
  if(!sp || !jp) return jfail(ctx, GALIC_ERR_INVALID_ARGUMENT);
  if(!ctx->have_fg) return jfail(ctx, GALIC_ERR_STATE);
  const galic_params_t &p = ctx->prm;
  const int N = p.FG_Nbin;
  if(N < 3 || N > 1024) return jfail(ctx, GALIC_ERR_UNSUPPORTED);
  for(int t = 1; t <= 3; t++)
    if(p.NType[t] > 0 && p.TypeOfVelocityStructure[t] == 3 && jp->DispersionRoverZratio[t] == 0)
      return jfail(ctx, GALIC_ERR_UNSUPPORTED);  // disp_fields.c:743-750 terminate()
  if(cudaSetDevice(ctx->device)) return jfail(ctx, GALIC_ERR_CUDA);
  cudaStream_t s = ctx->stream;
  const size_t G = (size_t) N * N;
  int rc = GALIC_OK, launches = 0;
  double *d_Rg = nullptr, *d_tab = nullptr, *d_Y = nullptr, *d_q = nullptr;
  SphCoef *d_sph = nullptr;
  TiltCoef *d_tilt = nullptr;
  // rows of tilted coefficients per block: all of them within 512 MiB
  const int tilt_rows =
      (int) std::max<size_t>(1, std::min<size_t>(N - 1, (512ull << 20) / ((size_t) TILT_STEPS * N * sizeof(TiltCoef))));
  std::vector<double> Rg(2 * N + 3), h_tab;
  for(int j = 0; j < 2 * N + 3; j++) Rg[j] = p.FG_Rmin * (std::pow(p.FG_Fac, j) - 1.0);
  bool any_tilt = false;
  JeansArgs J{};
  J.M = ctx->dm;
  J.N = N;
  J.HaloStretch = p.HaloStretch;
  J.Halo_Mass = p.Halo_Mass;
  J.Halo_A = p.Halo_A;
  J.Disk_Mass = p.Disk_Mass;
  J.Disk_H = sp->Disk_H;
  J.Disk_Z0 = sp->Disk_Z0;
  J.Bulge_Mass = p.Bulge_Mass;
  J.Bulge_A = p.Bulge_A;
  J.BulgeStretch = p.BulgeStretch;
  for(int t = 1; t <= 3; t++) any_tilt |= (p.NType[t] > 0 && p.TypeOfVelocityStructure[t] == 3);
  JCK(cudaMallocAsync((void **) &d_Rg, Rg.size() * sizeof(double), s));
  JCK(cudaMallocAsync((void **) &d_tab, 4 * NTAB * G * sizeof(double), s));
  JCK(cudaMallocAsync((void **) &d_sph, (size_t) (N + 1) * SPH_STEPS * sizeof(SphCoef), s));
  JCK(cudaMallocAsync((void **) &d_Y, (size_t) N * (N + 1) * (AXI_STEPS + 1) * sizeof(double), s));
  if(any_tilt) {
    JCK(cudaMallocAsync((void **) &d_q, G * sizeof(double), s));
    JCK(cudaMallocAsync((void **) &d_tilt, (size_t) tilt_rows * TILT_STEPS * N * sizeof(TiltCoef), s));
    JCK(prepare_march());
  }
  JCK(cudaMemcpyAsync(d_Rg, Rg.data(), Rg.size() * sizeof(double), cudaMemcpyHostToDevice, s));
  JCK(cudaMemsetAsync(d_tab, 0, 4 * NTAB * G * sizeof(double), s));
  J.Rg = d_Rg;
  // spherical (disp_fields.c:512-570)
  for(int t = 1; t <= 3; t++) {
    if(p.NType[t] == 0) continue;
    J.type = t;
    J.beta = (t == 1) ? sp->HaloBetaParameter : (t == 3 ? sp->BulgeBetaParameter : 0.0);
    J.beta_a = (t == 1) ? p.Halo_A : p.Bulge_A;
    J.tab = d_tab + (size_t) t * NTAB * G;
    k_sph_coef<<<blocks((long long) (N + 1) * SPH_STEPS, 256), 256, 0, s>>>(J, d_sph);
    k_sph_march<<<1, 256, 0, s>>>(J, d_sph);
    k_sph_divide<<<blocks(N, 256), 256, 0, s>>>(J);
    launches += 3;
    JCK(cudaGetLastError());
  }
  // axisymmetric f(E, Lz) (disp_fields.c:575-729)
  for(int t = 1; t <= 3; t++) {
    if(p.NType[t] == 0) continue;
    J.type = t;
    J.kpar = jp->StreamingVelocityParameter[t];
    J.tab = d_tab + (size_t) t * NTAB * G;
    k_axi_points<<<blocks((long long) N * (N + 1) * (AXI_STEPS + 1), 256), 256, 0, s>>>(J, d_Y);
    k_axi_march<<<blocks(N, 32), 32, 0, s>>>(J, d_Y);
    k_axi_stream<<<blocks((long long) G, 256), 256, 0, s>>>(J);
    launches += 3;
    JCK(cudaGetLastError());
  }
  // tilted f(E, Lz, I3) (disp_fields.c:733-1044)
  for(int t = 1; t <= 3; t++) {
    if(p.NType[t] == 0 || p.TypeOfVelocityStructure[t] != 3) continue;
    J.type = t;
    J.f = jp->DispersionRoverZratio[t];
    J.kpar = jp->StreamingVelocityParameter[t];
    J.beta = (t == 1) ? sp->HaloBetaParameter : (t == 3 ? sp->BulgeBetaParameter : 0.0);
    J.beta_a = (t == 1) ? p.Halo_A : p.Bulge_A;
    J.tab = d_tab + (size_t) t * NTAB * G;
    JCK(cudaMemsetAsync(d_q + (size_t) (N - 1) * N, 0, N * sizeof(double), s));  // the top row is 0
    const int mthreads = ((N + 31) / 32) * 32;
    for(int k_hi = N - 2; k_hi >= 0; k_hi -= tilt_rows) {
      const int k_lo = std::max(0, k_hi - tilt_rows + 1);
      const long long n = (long long) (k_hi - k_lo + 1) * TILT_STEPS * N;
      k_tilt_coef<<<blocks(n, 256), 256, 0, s>>>(J, k_lo, k_hi, d_tilt);
      if(mthreads <= 512)
        k_tilt_march<512, 8><<<1, mthreads, march_smem(N, 8), s>>>(J, k_lo, k_hi, d_tilt, d_q);
      else
        k_tilt_march<1024, 4><<<1, mthreads, march_smem(N, 4), s>>>(J, k_lo, k_hi, d_tilt, d_q);
      launches += 2;
    }
    k_tilt_tables<<<blocks((long long) G, 256), 256, 0, s>>>(J, d_q);
    k_tilt_stream<<<blocks((long long) G, 256), 256, 0, s>>>(J);
    launches += 2;
    JCK(cudaGetLastError());
  }
  h_tab.resize(4 * NTAB * G);
  JCK(cudaMemcpyAsync(h_tab.data(), d_tab, 4 * NTAB * G * sizeof(double), cudaMemcpyDeviceToHost, s));
  JCK(cudaStreamSynchronize(s));
done:
  if(d_Rg) cudaFreeAsync(d_Rg, s);
  if(d_tab) cudaFreeAsync(d_tab, s);
  if(d_sph) cudaFreeAsync(d_sph, s);
  if(d_Y) cudaFreeAsync(d_Y, s);
  if(d_q) cudaFreeAsync(d_q, s);
  if(d_tilt) cudaFreeAsync(d_tilt, s);
  if(rc != GALIC_OK) {
    cudaStreamSynchronize(s);
    return jfail(ctx, rc);
  }
  ctx->last_launches = launches;
  // install into the context (as galic_set_vstream / galic_set_dispersion
  // would) and copy out
  for(int t = 1; t <= 3; t++) {
    if(p.NType[t] == 0) continue;
    const double *T = h_tab.data() + (size_t) t * NTAB * G;
    if((rc = galic_set_vstream(ctx, t, T + 3 * G)) != GALIC_OK) return rc;
    if((rc = galic_set_dispersion(ctx, t, T, T + G, T + 2 * G, T + 7 * G, T + 6 * G)) != GALIC_OK) return rc;
    if(out) {
      double *dst[NTAB] = {out[t].disp_r,     out[t].dispz,      out[t].dispphi,          out[t].vstream,
                           out[t].tilted_vz2, out[t].tilted_vR2, out[t].tilted_vz2_prime, out[t].tilted_vR2_prime};
      for(int w = 0; w < NTAB; w++)
        if(dst[w]) std::copy(T + (size_t) w * G, T + (size_t) (w + 1) * G, dst[w]);
    }
  }
  return jfail(ctx, GALIC_OK);
}
