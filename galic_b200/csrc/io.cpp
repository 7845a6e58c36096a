// GALIC's output files, written from host copies of the device state:
//   galic_write_snapshot        write_file (io.c:906-1243) for one rank and one
//                               file, SnapFormat 1 or 2, single-precision
//                               blocks POS, VEL, ID, MASS, VELT
//   galic_write_forcefield      forcefield.dat (grid.c:789-823) with the
//                               analytic-halo columns of grid.c:766-786
//   galic_write_density_field   densfield_<type>_<num>.dat (io.c:36-460)
//   galic_output_density_field  the same for every type, from a context
// The byte layout, the order of the blocks and every computed value (grid
// coordinates through the C library's pow, the variable-resolution
// smoothing) follow the reference, so the files are byte-identical.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "galic_gpu.h"

namespace {

// struct io_header (allvars.h:998-1031): 256 bytes, no padding
#pragma pack(push, 1)
struct SnapHeader {
  int npart[6];
  double mass[6];
  double time, redshift;
  int flag_sfr, flag_feedback;
  unsigned int npartTotal[6];
  int flag_cooling, num_files;
  double BoxSize, Omega0, OmegaLambda, HubbleParam;
  int flag_stellarage, flag_metals;
  unsigned int npartTotalHighWord[6];
  int flag_entropy_instead_u, flag_doubleprecision, flag_lpt_ics;
  float lpt_scalingfactor;
  int flag_tracer_field, composition_vector_length;
  char fill[40];
};
#pragma pack(pop)
static_assert(sizeof(SnapHeader) == 256, "the Gadget header is 256 bytes");

struct File {
  FILE *f = nullptr;
  bool ok = true;
  explicit File(const char *name) : f(std::fopen(name, "wb")) { ok = f != nullptr; }
  ~File()
  {
    if(f) std::fclose(f);
  }
  void put(const void *p, size_t size, size_t n)
  {
    if(ok && n && std::fwrite(p, size, n, f) != n) ok = false;
  }
  void put_int(int v) { put(&v, sizeof(int), 1); }
  bool close()
  {
    if(f && std::fclose(f) != 0) ok = false;
    f = nullptr;
    return ok;
  }
};

int stack_off(int l) { return ((1 << (2 * l)) - 1) / 3; }

// eval_smoothed_stack / calc_smoothed_stack (grid.c:1217-1243)
double eval_smoothed(const double *din, int l, int i, int j, int maxlevel, const double *ref, double thresh)
{
  const double scale = std::pow((double) (1 << (maxlevel - l)), 2);
  if(l == 0) return din[stack_off(l) + i * (1 << l) + j] / scale;
  if(ref[stack_off(l - 1) + (i / 2) * (1 << (l - 1)) + j / 2] > thresh)
    return din[stack_off(l) + i * (1 << l) + j] / scale;
  return eval_smoothed(din, l - 1, i / 2, j / 2, maxlevel, ref, thresh);
}

void calc_smoothed(const double *din, double *dout, int maxlevel, const double *ref, double thresh)
{
  const int n = 1 << maxlevel;
  for(int i = 0; i < n; i++)
    for(int j = 0; j < n; j++) dout[i * n + j] = eval_smoothed(din, maxlevel, i, j, maxlevel, ref, thresh);
}

// a smoothed stack from its finest level: calc_global_fit copies the
// committed grid into the stack's finest level and smooths it (main.c:259-289)
std::vector<double> stack_from_grid(const double *grid, int L)
{
  std::vector<double> st(stack_off(L + 1), 0.0);
  std::memcpy(st.data() + stack_off(L), grid, sizeof(double) * ((size_t) 1 << (2 * L)));
  galic_smooth_stack(st.data(), L);
  return st;
}

}  // namespace

extern "C" int galic_write_snapshot(const char *fname, int snap_format, int n, const double *pos, const double *vel,
                                    const double *vel_theo, const double *mass, const int *id, const int *type,
                                    const double *mass_table)
{
  if(!fname || (snap_format != 1 && snap_format != 2) || n < 0 ||
     (n > 0 && (!pos || !vel || !vel_theo || !mass || !id || !type)))
    return GALIC_ERR_INVALID_ARGUMENT;
  for(int i = 0; i < n; i++)
    if(type[i] < 0 || type[i] > 5) return GALIC_ERR_INVALID_ARGUMENT;
  SnapHeader h;
  std::memset(&h, 0, sizeof(h));
  double mt[6] = {0, 0, 0, 0, 0, 0};
  if(mass_table)
    for(int t = 0; t < 6; t++) mt[t] = mass_table[t];
  for(int i = 0; i < n; i++) h.npart[type[i]]++;
  for(int t = 0; t < 6; t++) {
    h.npartTotal[t] = (unsigned int) h.npart[t];
    h.mass[t] = mt[t];
  }
  h.num_files = 1;
  File f(fname);
  if(!f.ok) return GALIC_ERR_INVALID_ARGUMENT;
  if(snap_format == 2) {
    f.put_int(8);
    f.put("HEAD", 1, 4);
    f.put_int((int) sizeof(h) + 8);
    f.put_int(8);
  }
  f.put_int((int) sizeof(h));
  f.put(&h, sizeof(h), 1);
  f.put_int((int) sizeof(h));
  // IO_POS, IO_VEL, IO_ID, IO_MASS, IO_VELTHEO (allvars.h:1035-1044)
  const char *labels[5] = {"POS ", "VEL ", "ID  ", "MASS", "VELT"};
  const int per[5] = {3, 3, 1, 1, 3};
  std::vector<float> fb;
  std::vector<unsigned int> ib;
  for(int b = 0; b < 5; b++) {
    bool in_block[6];
    long long npart = 0;
    for(int t = 0; t < 6; t++) {
      in_block[t] = h.npart[t] > 0 && (b != 3 || mt[t] == 0);
      if(in_block[t]) npart += h.npart[t];
    }
    if(npart == 0) continue;
    const int bytes = per[b] * 4;  // single-precision values, unsigned int IDs
    if(snap_format == 2) {
      f.put_int(8);
      f.put(labels[b], 1, 4);
      f.put_int((int) (npart * bytes + 8));
      f.put_int(8);
    }
    f.put_int((int) (npart * bytes));
    for(int t = 0; t < 6; t++) {
      if(!in_block[t]) continue;
      fb.clear();
      ib.clear();
      for(int i = 0; i < n; i++) {
        if(type[i] != t) continue;
        if(b == 0)
          for(int k = 0; k < 3; k++) fb.push_back((float) pos[3 * i + k]);
        else if(b == 1)
          for(int k = 0; k < 3; k++) fb.push_back((float) vel[3 * i + k]);
        else if(b == 4)
          for(int k = 0; k < 3; k++) fb.push_back((float) vel_theo[3 * i + k]);
        else if(b == 3)
          fb.push_back((float) mass[i]);
        else
          ib.push_back((unsigned int) id[i]);
      }
      if(b == 2)
        f.put(ib.data(), sizeof(unsigned int), ib.size());
      else
        f.put(fb.data(), sizeof(float), fb.size());
    }
    f.put_int((int) (npart * bytes));
  }
  return f.close() ? GALIC_OK : GALIC_ERR_INVALID_ARGUMENT;
}

extern "C" int galic_write_forcefield(const char *fname, const galic_params_t *prm, const double *dpotdr,
                                      const double *dpotdz, const double *pot)
{
  if(!fname || !prm || !dpotdr || !dpotdz || !pot || prm->FG_Nbin < 1) return GALIC_ERR_INVALID_ARGUMENT;
  const int N = prm->FG_Nbin;
  const size_t G = (size_t) N * N;
  std::vector<double> pe(G), re(G), ze(G), tR(G), tz(G);
  for(int k = 0; k < N; k++)
    for(int j = 0; j < N; j++) {
      const size_t i = (size_t) k * N + j;
      const double r1 = prm->FG_Rmin * (std::pow(prm->FG_Fac, j) - 1.0);
      const double z1 = prm->FG_Rmin * (std::pow(prm->FG_Fac, k) - 1.0);
      const double p[3] = {r1, 0, z1};
      // halo_get_potential / halo_get_acceleration (halo.c:63-84)
      const double r = std::sqrt(p[0] * p[0] + p[1] * p[1] + p[2] * p[2]);
      pe[i] = -prm->G * prm->Halo_Mass / (r + prm->Halo_A);
      const double fac = prm->G * prm->Halo_Mass / ((r + 1.0e-6 * prm->Halo_A) * (r + prm->Halo_A) * (r + prm->Halo_A));
      re[i] = -fac * p[0];
      ze[i] = -fac * p[2];
    }
  for(int k = 0; k < N; k++) {
    const double z = prm->FG_Rmin * (std::pow(prm->FG_Fac, k) - 1.0);
    for(int j = 0; j < N; j++) {
      const double R = prm->FG_Rmin * (std::pow(prm->FG_Fac, j) - 1.0);
      tR[(size_t) k * N + j] = R;
      tz[(size_t) k * N + j] = z;
    }
  }
  File f(fname);
  if(!f.ok) return GALIC_ERR_INVALID_ARGUMENT;
  f.put_int(N);
  const double *cols[8] = {dpotdr, dpotdz, pot, re.data(), ze.data(), pe.data(), tR.data(), tz.data()};
  for(const double *c : cols) f.put(c, sizeof(double), G);
  return f.close() ? GALIC_OK : GALIC_ERR_INVALID_ARGUMENT;
}

extern "C" int galic_write_density_field(const char *fname, const galic_params_t *prm, int type,
                                         const double *dgs_target, const double *egs_targets,
                                         const double *dg_mass_loc, const double *eg_loc)
{
  if(!fname || !prm || type < 1 || type > 3 || !dgs_target || !egs_targets || !dg_mass_loc || !eg_loc ||
     prm->DG_MaxLevel < 1 || prm->DG_MaxLevel > 12 || prm->EG_MaxLevel < 1 || prm->EG_MaxLevel > 12 ||
     prm->NType[type] <= 0)
    return GALIC_ERR_INVALID_ARGUMENT;
  const int DL = prm->DG_MaxLevel, EL = prm->EG_MaxLevel;
  const int DN = 1 << DL, EN = 1 << EL;
  const size_t DG = (size_t) DN * DN, EG = (size_t) EN * EN, ENs = (size_t) stack_off(EL + 1);
  const double thrD = prm->MinParticlesPerBinForDensityMeasurement * prm->MType[type] / prm->NType[type];
  const double thrE = prm->MinParticlesPerBinForDispersionMeasurement * prm->MType[type] / prm->NType[type];
  const std::vector<double> dgs_resp = stack_from_grid(dg_mass_loc, DL);
  std::vector<double> egs_resp[5];
  for(int k = 0; k < 5; k++) egs_resp[k] = stack_from_grid(eg_loc + (size_t) k * EG, EL);
  File f(fname);
  if(!f.ok) return GALIC_ERR_INVALID_ARGUMENT;
  // io.c:60-95: the target stack level by level, the variable-resolution
  // target and response, the fine response
  f.put_int(DL);
  for(int lev = DL; lev >= 0; lev--) {
    const int nbin = 1 << lev;
    f.put_int(nbin);
    f.put(dgs_target + stack_off(lev), sizeof(double), (size_t) nbin * nbin);
  }
  std::vector<double> dout(DG);
  calc_smoothed(dgs_target, dout.data(), DL, dgs_target, thrD);
  f.put_int(DN);
  f.put(dout.data(), sizeof(double), DG);
  calc_smoothed(dgs_resp.data(), dout.data(), DL, dgs_target, thrD);
  f.put_int(DN);
  f.put(dout.data(), sizeof(double), DG);
  f.put_int(DN);
  f.put(dgs_resp.data() + stack_off(DL), sizeof(double), DG);
  // io.c:286-343: cell centres of the density and energy grids
  for(int g = 0; g < 2; g++) {
    const int nb = g ? EN : DN;
    const double rmin = g ? prm->EG_Rmin : prm->DG_Rmin, fac = g ? prm->EG_Fac : prm->DG_Fac;
    std::vector<double> tR((size_t) nb * nb), tz((size_t) nb * nb);
    for(int k = 0; k < nb; k++) {
      const double z = rmin * 0.5 * (std::pow(fac, k) + std::pow(fac, k + 1) - 2.0);
      for(int j = 0; j < nb; j++) {
        const double R = rmin * 0.5 * (std::pow(fac, j) + std::pow(fac, j + 1) - 2.0);
        tR[(size_t) k * nb + j] = R;
        tz[(size_t) k * nb + j] = z;
      }
    }
    f.put_int(nb);
    f.put(tR.data(), sizeof(double), tR.size());
    f.put_int(nb);
    f.put(tz.data(), sizeof(double), tz.size());
  }
  // io.c:347-455: target and response of the energy-grid mass and of r, t, p, q
  std::vector<double> eout(EG);
  const double *emass_resp = egs_resp[0].data();
  for(int k = 0; k < 5; k++) {
    calc_smoothed(egs_targets + (size_t) k * ENs, eout.data(), EL, emass_resp, thrE);
    f.put_int(EN);
    f.put(eout.data(), sizeof(double), EG);
    calc_smoothed(egs_resp[k].data(), eout.data(), EL, emass_resp, thrE);
    f.put_int(EN);
    f.put(eout.data(), sizeof(double), EG);
  }
  return f.close() ? GALIC_OK : GALIC_ERR_INVALID_ARGUMENT;
}

extern "C" int galic_output_density_field(galic_ctx *ctx, const char *outdir, int num)
{
  if(!ctx || !outdir || num < 0) return GALIC_ERR_INVALID_ARGUMENT;
  galic_params_t prm;
  std::memset(&prm, 0, sizeof(prm));
  int st = galic_get_params(ctx, &prm);
  if(st != GALIC_OK) return st;
  const int L = prm.DG_MaxLevel;
  const size_t G = (size_t) 1 << (2 * L), Ns = (size_t) stack_off(L + 1);
  for(int t = 1; t <= 3; t++) {
    if(prm.NType[t] == 0) continue;
    std::vector<double> tg(6 * Ns), loc(6 * G);
    if((st = galic_get_targets(ctx, t, tg.data(), tg.data() + Ns, tg.data() + 2 * Ns, tg.data() + 3 * Ns,
                                tg.data() + 4 * Ns, tg.data() + 5 * Ns)) != GALIC_OK)
      return st;
    // the committed grids: DG mass (time averaged), EG mass, r, t, p, q (instantaneous)
    const int which[6] = {GALIC_GRID_MASS_S, GALIC_GRID_MASS_I, GALIC_GRID_R_I, GALIC_GRID_T_I, GALIC_GRID_P_I,
                          GALIC_GRID_Q_I};
    for(int k = 0; k < 6; k++)
      if((st = galic_get_response(ctx, t, which[k], loc.data() + (size_t) k * G)) != GALIC_OK) return st;
    char name[4096];
    std::snprintf(name, sizeof(name), "%s/densfield_%d_%03d.dat", outdir, t, num);
    if((st = galic_write_density_field(name, &prm, t, tg.data(), tg.data() + Ns, loc.data(), loc.data() + G)) !=
       GALIC_OK)
      return st;
  }
  return GALIC_OK;
}
