// Force-grid fill: the tree-force part of forcedensitygrid_calculate
// (grid.c:621-750), i.e. GALIC's gravity() (gravtree.c:35-50) evaluated at
// the FG_Nbin^2 x FG_SECTIONS probe points and averaged over the sections.
//
// Built with --fmad=false (device) and -ffp-contract=off (host); the result is
// bit-identical to the single-rank reference because every step reproduces
// its arithmetic and its order:
//  * probe positions and section angles use the host libm, as grid.c:680-704
//    and grid.c:733-737 do;
//  * the domain cube (domain_box.c:20-65), the 21-bit domain coordinates and
//    Peano-Hilbert keys (domain.c:155-164, peano.c:331-347) and the stable key
//    order of all points (peano.c:63-104) are computed on the GPU;
//  * the oct-tree (forcetree.c:139-495) is the set of cubes that belong to the
//    top-level domain tree (domain_toplevel.c:18-171: the root and every cube
//    holding more than a fraction 1/(TopNodeFactor*MultipleDomains) of all
//    points, probes included, are split) or contain at least two mass
//    particles.  It is laid out in depth-first order with children in Morton
//    order (x bit 0, y bit 1, z bit 2), which is the reference's threaded
//    nextnode/sibling order (forcetree.c:591-722): the first child of item i
//    is item i+1 and `skip` is the item after i's subtree;
//  * node moments are summed over the children in that order
//    (forcetree.c:622-690; force_treeupdate_toplevel forcetree.c:817-890
//    recomputes the top nodes with the same sums);
//  * the walk (forcetree_walk.c:12-222) opens a node when
//    (float) len*len > r2*theta*theta, with the side length held as a float
//    (allvars.h:1096), and uses the reference's spline-softened kernel;
//  * the section values of each grid cell are added in the points' key order
//    (grid.c:720-750).
//
// The walk runs one probe per lane with the probes in key order, so a warp
// holds 32 neighbouring probes.  Every lane's walk visits items in increasing
// index order, so the warp steps through the minimum of its lanes' next
// items: that item is loaded once for the warp (a broadcast), the lanes whose
// walk is at it evaluate it, and each lane still sees exactly its own item
// sequence, in the reference's order.
#include <cuda_runtime.h>
#include <cub/cub.cuh>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "galic_gpu.h"

namespace {

constexpr int kSections = 8;       // FG_SECTIONS (allvars.h:123)
constexpr int kBits = 21;          // BITS_PER_DIMENSION (allvars.h:213)
constexpr int kMaxTreeLevel = 30;  // MAX_TREE_LEVEL (forcetree.h:16)
constexpr int kWalkBlock = 256;

// Peano-Hilbert state machine of peano.c:226-330: next state (kRot) and key
// digit (kSub) for each state 0..47 and octant pix = 4*x + 2*y + z.  The
// tables must be identical for the keys to be.
const char *const kRot[48] = {
    "\x24\x1c\x19\x1b\x0a\x0a\x19\x1b", "\x1d\x0b\x18\x18\x25\x0b\x1a\x1a", "\x08\x08\x19\x1b\x1e\x26\x19\x1b",
    "\x09\x27\x18\x18\x09\x1f\x1a\x1a", "\x28\x18\x2c\x20\x28\x06\x2c\x06", "\x19\x07\x21\x07\x29\x29\x2d\x2d",
    "\x04\x2a\x04\x2e\x1a\x2a\x22\x2e", "\x2b\x2b\x2f\x2f\x05\x1b\x05\x23", "\x21\x23\x24\x1c\x21\x23\x02\x02",
    "\x20\x20\x1d\x03\x22\x22\x25\x03", "\x21\x23\x00\x00\x21\x23\x1e\x26", "\x20\x20\x01\x27\x22\x22\x01\x1f",
    "\x18\x2a\x20\x2e\x0e\x2a\x0e\x2e", "\x2b\x2b\x2f\x2f\x19\x0f\x21\x0f", "\x28\x0c\x2c\x0c\x28\x1a\x2c\x22",
    "\x0d\x1b\x0d\x23\x29\x29\x2d\x2d", "\x1c\x29\x1c\x16\x26\x2b\x26\x16", "\x2a\x28\x17\x17\x1d\x27\x1d\x27",
    "\x29\x24\x14\x24\x2b\x1e\x14\x1e", "\x25\x1f\x25\x1f\x2a\x28\x15\x15", "\x1c\x12\x1c\x2d\x26\x12\x26\x2f",
    "\x13\x13\x2e\x2c\x1d\x27\x1d\x27", "\x10\x24\x2d\x24\x10\x1e\x2f\x1e", "\x25\x1f\x25\x1f\x11\x11\x2e\x2c",
    "\x0c\x04\x01\x03\x22\x22\x01\x03", "\x05\x23\x00\x00\x0d\x23\x02\x02", "\x20\x20\x01\x03\x06\x0e\x01\x03",
    "\x21\x0f\x00\x00\x21\x07\x02\x02", "\x10\x00\x14\x08\x10\x1e\x14\x1e", "\x01\x1f\x09\x1f\x11\x11\x15\x15",
    "\x1c\x12\x1c\x16\x02\x12\x0a\x16", "\x13\x13\x17\x17\x1d\x03\x1d\x0b", "\x09\x0b\x0c\x04\x09\x0b\x1a\x1a",
    "\x08\x08\x05\x1b\x0a\x0a\x0d\x1b", "\x09\x0b\x18\x18\x09\x0b\x06\x0e", "\x08\x08\x19\x0f\x0a\x0a\x19\x07",
    "\x00\x12\x08\x16\x26\x12\x26\x16", "\x13\x13\x17\x17\x01\x27\x09\x27", "\x10\x24\x14\x24\x10\x02\x14\x0a",
    "\x25\x03\x25\x0b\x11\x11\x15\x15", "\x04\x11\x04\x2e\x0e\x13\x0e\x2e", "\x12\x10\x2f\x2f\x05\x0f\x05\x0f",
    "\x11\x0c\x2c\x0c\x13\x06\x2c\x06", "\x0d\x07\x0d\x07\x12\x10\x2d\x2d", "\x04\x2a\x04\x15\x0e\x2a\x0e\x17",
    "\x2b\x2b\x16\x14\x05\x0f\x05\x0f", "\x28\x0c\x15\x0c\x28\x06\x17\x06", "\x0d\x07\x0d\x07\x29\x29\x16\x14"};
const char *const kSub[48] = {
    "07163425", "74650312", "43527061", "30214756", "10672354", "03741265", "32450176", "21563047",
    "61705243", "12036574", "25341607", "56472130", "76014532", "65127403", "54236710", "47305621",
    "67541023", "70436152", "01327645", "16250734", "23105467", "34072516", "45763201", "52614370",
    "70614352", "03127465", "34250716", "47563021", "67105423", "74036512", "45327601", "56214730",
    "16072534", "65741203", "52436170", "21305647", "01763245", "12650374", "23541067", "30472156",
    "10236754", "07341625", "76450132", "61527043", "54672310", "43705261", "32014576", "25163407"};

struct PhTables {
  unsigned char rot[48][8], sub[48][8];
};

const PhTables &host_tables()
{
  static PhTables t;
  static std::once_flag once;
  std::call_once(once, [] {
    for(int r = 0; r < 48; r++)
      for(int c = 0; c < 8; c++) {
        t.rot[r][c] = (unsigned char) kRot[r][c];
        t.sub[r][c] = (unsigned char) (kSub[r][c] - '0');
      }
  });
  return t;
}

__constant__ PhTables c_ph;

// One tree item, 48 bytes: a node (len >= 0: centre of mass, mass, float side
// length) or a single mass particle (len < 0: position, mass).
struct __align__(16) FillItem {
  double x, y, z, mass;
  float len;
  int skip;  // next item when this one is not opened; -1 ends the walk
  int pad[2];
};

// force_double_to_int (forcetree.h:33-38): the 52 mantissa bits
__host__ __device__ __forceinline__ unsigned long long mantissa52(double d)
{
  union {
    double d;
    unsigned long long u;
  } v;
  v.d = d;
  return v.u & 0xFFFFFFFFFFFFFull;
}

// 52-bit tree coordinate of one axis (forcetree.c:192-194); the top 21 bits
// are domain_double_to_int (domain.c:155-164)
__host__ __device__ __forceinline__ unsigned long long int_coord(double p, double corner, double inv_len)
{
  return mantissa52(((p - corner) * inv_len) + 1.0);
}

__host__ __device__ __forceinline__ unsigned long long ph_key(int x, int y, int z, int bits, const PhTables &t)
{
  unsigned char rotation = 0;
  unsigned long long key = 0;
  for(int mask = 1 << (bits - 1); mask > 0; mask >>= 1) {
    const unsigned char pix = ((x & mask) ? 4 : 0) | ((y & mask) ? 2 : 0) | ((z & mask) ? 1 : 0);
    key = (key << 3) | t.sub[rotation][pix];
    rotation = t.rot[rotation][pix];
  }
  return key;
}

// domain_determineTopTree (domain_toplevel.c:22-32): keys of all points
__global__ void k_keys(int n, const double *__restrict__ pos, double cx, double cy, double cz, double inv_len,
                       unsigned long long *__restrict__ key, int *__restrict__ idx)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  const int x = (int) (int_coord(pos[3 * (size_t) i + 0], cx, inv_len) >> (52 - kBits));
  const int y = (int) (int_coord(pos[3 * (size_t) i + 1], cy, inv_len) >> (52 - kBits));
  const int z = (int) (int_coord(pos[3 * (size_t) i + 2], cz, inv_len) >> (52 - kBits));
  key[i] = ph_key(x, y, z, kBits, c_ph);
  idx[i] = i;
}

// force_treeevaluate (forcetree_walk.c:12-222), mode 0, one probe per lane.
// probes: SoA [3][np] in key order; res: SoA [4][np] (acc x, y, z, pot) * G.
__global__ void __launch_bounds__(kWalkBlock) k_walk(const FillItem *__restrict__ items, int nitems, int np,
                                                    const double *__restrict__ probes, double hmax,
                                                    double theta, double G, double *__restrict__ res,
                                                    unsigned long long *__restrict__ counts)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool live = t < np;
  double px = 0, py = 0, pz = 0;
  if(live) {
    px = probes[t];
    py = probes[np + t];
    pz = probes[2 * (size_t) np + t];
  }
  double acc_x = 0, acc_y = 0, acc_z = 0, pot = 0;
  unsigned next = live ? 0u : 0xFFFFFFFFu;  // 0xFFFFFFFF: walk finished
  const double h_inv = 1.0 / hmax;
  const double h3_inv = h_inv * h_inv * h_inv;
  unsigned n_int = 0, n_test = 0;
  for(;;) {
    const unsigned cur = __reduce_min_sync(0xFFFFFFFFu, next);
    if(cur == 0xFFFFFFFFu) break;
    if(next != cur) continue;
    const FillItem it = items[cur];
    const double dx = it.x - px;
    const double dy = it.y - py;
    const double dz = it.z - pz;
    const double r2 = dx * dx + dy * dy + dz * dz;
    if(it.len >= 0.f) {
      n_test++;
      const float len2 = it.len * it.len;
      if((double) len2 > r2 * theta * theta) {
        // open: the first daughter follows; a node without daughters is
        // followed by its skip item, which is the end for the last item
        next = (cur + 1 < (unsigned) nitems) ? cur + 1 : 0xFFFFFFFFu;
        continue;
      }
    }
    next = it.skip < 0 ? 0xFFFFFFFFu : (unsigned) it.skip;
    const double mass = it.mass;
    if(mass != 0.0) {
      n_int++;
      const double r = sqrt(r2);
      double fac, wp;
      if(r >= hmax) {
        fac = mass / (r2 * r);
        wp = -mass / r;
      } else {
        const double u = r * h_inv;
        if(u < 0.5) {
          fac = mass * h3_inv * (10.666666666667 + u * u * (32.0 * u - 38.4));
          wp = mass * h_inv * (-2.8 + u * u * (5.333333333333 + u * u * (6.4 * u - 9.6)));
        } else {
          fac = mass * h3_inv *
                (21.333333333333 - 48.0 * u + 38.4 * u * u - 10.666666666667 * u * u * u - 0.066666666667 / (u * u * u));
          wp = mass * h_inv *
               (-3.2 + 0.066666666667 / u + u * u * (10.666666666667 + u * (-16.0 + u * (9.6 - 2.133333333333 * u))));
        }
      }
      acc_x += dx * fac;
      acc_y += dy * fac;
      acc_z += dz * fac;
      pot += wp;
    }
  }
  // diagnostics: one atomic pair per warp
  unsigned long long a = n_int, b = n_test;
  for(int o = 16; o > 0; o >>= 1) {
    a += __shfl_xor_sync(0xFFFFFFFFu, a, o);
    b += __shfl_xor_sync(0xFFFFFFFFu, b, o);
  }
  if((threadIdx.x & 31) == 0) {
    atomicAdd(&counts[0], a);
    atomicAdd(&counts[1], b);
  }
  if(live) {  // gravtree.c:456-463
    res[t] = acc_x * G;
    res[np + t] = acc_y * G;
    res[2 * (size_t) np + t] = acc_z * G;
    res[3 * (size_t) np + t] = pot * G;
  }
}

// grid.c:720-750: the FG_SECTIONS values of a grid cell are added in the
// points' key order, then divided by FG_SECTIONS.  rank[s][cell] is the
// position of probe (s, cell) in the key order of the probes.
__global__ void k_readout(int NN, int np, const int *__restrict__ rank, const double *__restrict__ res,
                          const double *__restrict__ trig, double *__restrict__ out)
{
  const int cell = blockIdx.x * blockDim.x + threadIdx.x;
  if(cell >= NN) return;
  int rk[kSections], sec[kSections];
  for(int s = 0; s < kSections; s++) {
    rk[s] = rank[s * NN + cell];
    sec[s] = s;
  }
  for(int a = 1; a < kSections; a++)  // insertion sort of the sections by rank
    for(int b = a; b > 0 && rk[b] < rk[b - 1]; b--) {
      int tmp = rk[b];
      rk[b] = rk[b - 1];
      rk[b - 1] = tmp;
      tmp = sec[b];
      sec[b] = sec[b - 1];
      sec[b - 1] = tmp;
    }
  double r = 0, z = 0, p = 0;
  for(int a = 0; a < kSections; a++) {
    const int q = rk[a], s = sec[a];
    r += res[q] * trig[s] + res[np + q] * trig[kSections + s];
    z += res[2 * (size_t) np + q];
    p += res[3 * (size_t) np + q];
  }
  out[cell] = r / kSections;
  out[NN + cell] = z / kSections;
  out[2 * NN + cell] = p / kSections;
}

// ------------------------------------------------------------------ host tree

struct TreeBuilder {
  const unsigned long long *ix, *iy, *iz;  // 52-bit coordinates of the mass particles
  const double *pos, *mass;
  const unsigned long long *keys;          // sorted keys of all points
  size_t nkeys;
  double fac_load, limit, len;
  const PhTables *ph;
  std::vector<FillItem> items;
  std::vector<int> scratch;
  bool too_deep = false;

  // number of points whose key starts with the level-`level` prefix
  size_t count_prefix(unsigned long long prefix, int level) const
  {
    const int sh = 3 * (kBits - level);
    const unsigned long long lo = prefix << sh, hi = (prefix + 1) << sh;
    const unsigned long long *a = std::lower_bound(keys, keys + nkeys, lo);
    const unsigned long long *b = (level == 0) ? keys + nkeys : std::lower_bound(keys, keys + nkeys, hi);
    return (size_t) (b - a);
  }

  // Node for the cube at `level` with coordinate prefix (x52, y52, z52) that
  // holds the mass particles list[0..cnt).  `top`: the cube is a node of the
  // top-level tree, with Peano-Hilbert prefix `php` and curve state `rot`;
  // centre: its float centre (forcetree.c:543-547), the node's position when
  // it holds no mass (forcetree.c:684-689).
  void build(int level, int *list, int cnt, unsigned long long x52, unsigned long long y52, unsigned long long z52,
             const float centre[3], bool top, int rot, unsigned long long php)
  {
    const int me = (int) items.size();
    items.push_back(FillItem{});
    FillItem node{};
    node.len = (float) (len * std::ldexp(1.0, -level));
    if(level >= 52) {  // coincident particles: unreachable below MAX_TREE_LEVEL
      too_deep = true;
      node.skip = (int) items.size();
      items[me] = node;
      return;
    }
    const bool refined =
        top && (level == 0 || (level < kBits && fac_load * (double) count_prefix(php, level) > limit));
    const int bit = 51 - level;
    int count[8] = {0, 0, 0, 0, 0, 0, 0, 0}, start[9];
    auto digit = [&](int p) {
      return (int) (((ix[p] >> bit) & 1) | (((iy[p] >> bit) & 1) << 1) | (((iz[p] >> bit) & 1) << 2));
    };
    for(int k = 0; k < cnt; k++) count[digit(list[k])]++;
    start[0] = 0;
    for(int d = 0; d < 8; d++) start[d + 1] = start[d] + count[d];
    if(cnt > 1) {
      int fill[8];
      for(int d = 0; d < 8; d++) fill[d] = start[d];
      std::copy(list, list + cnt, scratch.begin());
      for(int k = 0; k < cnt; k++) list[fill[digit(scratch[k])]++] = scratch[k];
    }
    const double lenhalf = 0.25 * (double) node.len;
    double m = 0, s[3] = {0, 0, 0};
    for(int d = 0; d < 8; d++) {
      const int n = count[d];
      if(refined || n >= 2) {
        if(!refined && level + 1 > kMaxTreeLevel) too_deep = true;
        const int xb = d & 1, yb = (d >> 1) & 1, zb = (d >> 2) & 1;
        const int pix = (xb << 2) | (yb << 1) | zb;
        float cc[3];
        cc[0] = (float) (centre[0] + (2 * xb - 1) * lenhalf);
        cc[1] = (float) (centre[1] + (2 * yb - 1) * lenhalf);
        cc[2] = (float) (centre[2] + (2 * zb - 1) * lenhalf);
        const int child = (int) items.size();
        build(level + 1, list + start[d], n, x52 | ((unsigned long long) xb << bit),
              y52 | ((unsigned long long) yb << bit), z52 | ((unsigned long long) zb << bit), cc, refined,
              ph->rot[rot][pix], (php << 3) | ph->sub[rot][pix]);
        const FillItem &c = items[child];
        m += c.mass;
        s[0] += c.mass * c.x;
        s[1] += c.mass * c.y;
        s[2] += c.mass * c.z;
      } else if(n == 1) {
        const int p = list[start[d]];
        FillItem leaf{};
        leaf.x = pos[3 * (size_t) p + 0];
        leaf.y = pos[3 * (size_t) p + 1];
        leaf.z = pos[3 * (size_t) p + 2];
        leaf.mass = mass[p];
        leaf.len = -1.f;
        leaf.skip = (int) items.size() + 1;
        items.push_back(leaf);
        m += leaf.mass;
        s[0] += leaf.mass * leaf.x;
        s[1] += leaf.mass * leaf.y;
        s[2] += leaf.mass * leaf.z;
      }
    }
    if(m) {
      s[0] /= m;
      s[1] /= m;
      s[2] /= m;
    } else {
      s[0] = centre[0];
      s[1] = centre[1];
      s[2] = centre[2];
    }
    node.x = s[0];
    node.y = s[1];
    node.z = s[2];
    node.mass = m;
    node.skip = (int) items.size();
    items[me] = node;
  }
};

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() { cudaFree(p); }
  template <class T> T *as() { return static_cast<T *>(p); }
};

bool upload_tables()
{
  static std::once_flag once;
  static cudaError_t err = cudaSuccess;
  std::call_once(once, [] { err = cudaMemcpyToSymbol(c_ph, &host_tables(), sizeof(PhTables)); });
  return err == cudaSuccess;
}

}  // namespace

extern "C" uint64_t galic_peano_hilbert_key(int x, int y, int z, int bits)
{
  if(bits < 1 || bits > kBits) return 0;
  return ph_key(x, y, z, bits, host_tables());
}

#define FCK(call)                                                                                      \
  do {                                                                                                 \
    cudaError_t e_ = (call);                                                                           \
    if(e_ != cudaSuccess) {                                                                            \
      fprintf(stderr, "galic_cuda: %s failed: %s (%s:%d)\n", #call, cudaGetErrorString(e_), __FILE__, \
              __LINE__);                                                                               \
      return GALIC_ERR_CUDA;                                                                           \
    }                                                                                                  \
  } while(0)

extern "C" int galic_force_grid_fill(const galic_fill_params_t *fp, int n, const double *pos, const double *mass,
                                     double *fg_dpotdr, double *fg_dpotdz, double *fg_pot, galic_fill_stats_t *stats)
{
  const auto t_start = std::chrono::steady_clock::now();
  if(!fp || n < 1 || !pos || !mass || !fg_dpotdr || !fg_dpotdz || !fg_pot || fp->FG_Nbin < 2 ||
     fp->FG_Nbin > 4096 || !(fp->FG_Fac > 1) || !(fp->FG_Rmin > 0) || !(fp->ErrTolTheta > 0) ||
     !(fp->ForceSoftening > 0) || fp->MultipleDomains < 1 || !(fp->TopNodeFactor > 0) ||
     n > (1 << 30) - fp->FG_Nbin * fp->FG_Nbin * kSections)
    return GALIC_ERR_INVALID_ARGUMENT;
  const int N = fp->FG_Nbin, NN = N * N, np = NN * kSections, ntot = n + np;

  // probe points (grid.c:680-704), in the reference's point order: mass
  // particles, then s, k (z), j (R)
  std::vector<double> P(3 * (size_t) ntot);
  std::memcpy(P.data(), pos, 3 * (size_t) n * sizeof(double));
  std::vector<double> r1(N), z1(N);
  for(int j = 0; j < N; j++) r1[j] = fp->FG_Rmin * (std::pow(fp->FG_Fac, j) - 1.0);
  for(int k = 0; k < N; k++) z1[k] = fp->FG_Rmin * (std::pow(fp->FG_Fac, k) - 1.0);
  double trig[2 * kSections];
  for(int s = 0; s < kSections; s++) {
    const double phi = 2 * M_PI / kSections * s;
    trig[s] = std::cos(phi);
    trig[kSections + s] = std::sin(phi);
    for(int k = 0; k < N; k++)
      for(int j = 0; j < N; j++) {
        const size_t q = (size_t) n + (size_t) s * NN + (size_t) k * N + j;
        P[3 * q + 0] = r1[j] * trig[s];
        P[3 * q + 1] = r1[j] * trig[kSections + s];
        P[3 * q + 2] = z1[k];
      }
  }
  // domain_findExtent (domain_box.c:20-65)
  double xmin[3] = {1e306, 1e306, 1e306}, xmax[3] = {-1e306, -1e306, -1e306};
  for(size_t i = 0; i < (size_t) ntot; i++)
    for(int j = 0; j < 3; j++) {
      const double v = P[3 * i + j];
      if(xmin[j] > v) xmin[j] = v;
      if(xmax[j] < v) xmax[j] = v;
    }
  double len = 0;
  for(int j = 0; j < 3; j++)
    if(xmax[j] - xmin[j] > len) len = xmax[j] - xmin[j];
  len *= 1.00001;
  double centre[3], corner[3];
  for(int j = 0; j < 3; j++) {
    centre[j] = 0.5 * (xmin[j] + xmax[j]);
    corner[j] = 0.5 * (xmin[j] + xmax[j]) - 0.5 * len;
  }
  const double inv_len = 1.0 / len;
  if(!(len > 0) || !std::isfinite(inv_len)) return GALIC_ERR_INVALID_ARGUMENT;

  if(!upload_tables()) {
    fprintf(stderr, "galic_cuda: Peano-Hilbert table upload failed\n");
    return GALIC_ERR_CUDA;
  }
  // keys of all points and their stable key order (peano.c:63-104)
  DevBuf d_pos, d_key, d_key2, d_idx, d_idx2, d_tmp;
  FCK(cudaMalloc(&d_pos.p, 3 * (size_t) ntot * sizeof(double)));
  FCK(cudaMalloc(&d_key.p, (size_t) ntot * sizeof(unsigned long long)));
  FCK(cudaMalloc(&d_key2.p, (size_t) ntot * sizeof(unsigned long long)));
  FCK(cudaMalloc(&d_idx.p, (size_t) ntot * sizeof(int)));
  FCK(cudaMalloc(&d_idx2.p, (size_t) ntot * sizeof(int)));
  FCK(cudaMemcpy(d_pos.p, P.data(), 3 * (size_t) ntot * sizeof(double), cudaMemcpyHostToDevice));
  k_keys<<<(ntot + 255) / 256, 256>>>(ntot, d_pos.as<double>(), corner[0], corner[1], corner[2], inv_len,
                                      d_key.as<unsigned long long>(), d_idx.as<int>());
  FCK(cudaGetLastError());
  size_t tmp_bytes = 0;
  FCK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_key.as<unsigned long long>(),
                                      d_key2.as<unsigned long long>(), d_idx.as<int>(), d_idx2.as<int>(), ntot, 0,
                                      3 * kBits));
  FCK(cudaMalloc(&d_tmp.p, tmp_bytes));
  FCK(cub::DeviceRadixSort::SortPairs(d_tmp.p, tmp_bytes, d_key.as<unsigned long long>(),
                                      d_key2.as<unsigned long long>(), d_idx.as<int>(), d_idx2.as<int>(), ntot, 0,
                                      3 * kBits));
  std::vector<unsigned long long> keys(ntot);
  std::vector<int> order(ntot);
  FCK(cudaMemcpy(keys.data(), d_key2.p, (size_t) ntot * sizeof(unsigned long long), cudaMemcpyDeviceToHost));
  FCK(cudaMemcpy(order.data(), d_idx2.p, (size_t) ntot * sizeof(int), cudaMemcpyDeviceToHost));

  // oct-tree of the mass particles (forcetree.c:139-722)
  std::vector<unsigned long long> ix(n), iy(n), iz(n);
  for(int i = 0; i < n; i++) {
    ix[i] = int_coord(pos[3 * (size_t) i + 0], corner[0], inv_len);
    iy[i] = int_coord(pos[3 * (size_t) i + 1], corner[1], inv_len);
    iz[i] = int_coord(pos[3 * (size_t) i + 2], corner[2], inv_len);
  }
  TreeBuilder tb;
  tb.ix = ix.data();
  tb.iy = iy.data();
  tb.iz = iz.data();
  tb.pos = pos;
  tb.mass = mass;
  tb.keys = keys.data();
  tb.nkeys = keys.size();
  tb.fac_load = 1.0 / (double) ntot;                              // domain.c:149
  tb.limit = 1.0 / (fp->TopNodeFactor * fp->MultipleDomains * 1);  // one rank
  tb.len = len;
  tb.ph = &host_tables();
  tb.scratch.resize(n);
  tb.items.reserve(2 * (size_t) n + 64);
  {
    std::vector<int> list(n);
    for(int i = 0; i < n; i++) list[i] = i;
    const float c0[3] = {(float) centre[0], (float) centre[1], (float) centre[2]};
    tb.build(0, list.data(), n, 0, 0, 0, c0, true, 0, 0);
  }
  if(tb.too_deep) return GALIC_ERR_UNSUPPORTED;
  const int nitems = (int) tb.items.size();
  for(auto &it : tb.items)
    if(it.skip >= nitems) it.skip = -1;

  // probes in key order (SoA) and the key-order rank of each probe
  std::vector<double> probes(3 * (size_t) np);
  std::vector<int> rank(np);
  for(int r = 0, t = 0; r < ntot; r++) {
    const int id = order[r] - n;
    if(id < 0) continue;
    rank[id] = t;
    for(int j = 0; j < 3; j++) probes[(size_t) j * np + t] = P[3 * ((size_t) n + id) + j];
    t++;
  }
  DevBuf d_items, d_probes, d_res, d_rank, d_trig, d_out, d_counts;
  FCK(cudaMalloc(&d_items.p, (size_t) nitems * sizeof(FillItem)));
  FCK(cudaMalloc(&d_probes.p, 3 * (size_t) np * sizeof(double)));
  FCK(cudaMalloc(&d_res.p, 4 * (size_t) np * sizeof(double)));
  FCK(cudaMalloc(&d_rank.p, (size_t) np * sizeof(int)));
  FCK(cudaMalloc(&d_trig.p, sizeof(trig)));
  FCK(cudaMalloc(&d_out.p, 3 * (size_t) NN * sizeof(double)));
  FCK(cudaMalloc(&d_counts.p, 2 * sizeof(unsigned long long)));
  FCK(cudaMemset(d_counts.p, 0, 2 * sizeof(unsigned long long)));
  FCK(cudaMemcpy(d_items.p, tb.items.data(), (size_t) nitems * sizeof(FillItem), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_probes.p, probes.data(), 3 * (size_t) np * sizeof(double), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_rank.p, rank.data(), (size_t) np * sizeof(int), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_trig.p, trig, sizeof(trig), cudaMemcpyHostToDevice));

  cudaEvent_t e0, e1;
  FCK(cudaEventCreate(&e0));
  FCK(cudaEventCreate(&e1));
  FCK(cudaEventRecord(e0));
  k_walk<<<(np + kWalkBlock - 1) / kWalkBlock, kWalkBlock>>>(d_items.as<FillItem>(), nitems, np, d_probes.as<double>(),
                                                             fp->ForceSoftening, fp->ErrTolTheta, fp->G,
                                                             d_res.as<double>(),
                                                             d_counts.as<unsigned long long>());
  cudaError_t e = cudaGetLastError();
  cudaEventRecord(e1);
  if(e == cudaSuccess) {
    k_readout<<<(NN + 127) / 128, 128>>>(NN, np, d_rank.as<int>(), d_res.as<double>(), d_trig.as<double>(),
                                         d_out.as<double>());
    e = cudaGetLastError();
  }
  if(e == cudaSuccess) e = cudaDeviceSynchronize();
  float ms = 0;
  if(e == cudaSuccess) e = cudaEventElapsedTime(&ms, e0, e1);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  FCK(e);
  unsigned long long counts[2];
  FCK(cudaMemcpy(counts, d_counts.p, sizeof(counts), cudaMemcpyDeviceToHost));
  FCK(cudaMemcpy(fg_dpotdr, d_out.p, (size_t) NN * sizeof(double), cudaMemcpyDeviceToHost));
  FCK(cudaMemcpy(fg_dpotdz, d_out.as<double>() + NN, (size_t) NN * sizeof(double), cudaMemcpyDeviceToHost));
  FCK(cudaMemcpy(fg_pot, d_out.as<double>() + 2 * (size_t) NN, (size_t) NN * sizeof(double),
                 cudaMemcpyDeviceToHost));
  if(stats) {
    stats->ms_walk = ms;
    stats->ms_total =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t_start).count();
    stats->tree_items = nitems;
    stats->tree_nodes = nitems - n;
    stats->interactions = (long long) counts[0];
    stats->node_tests = (long long) counts[1];
  }
  return GALIC_OK;
}
