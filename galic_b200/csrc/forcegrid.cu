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
//    points, probes included, are split; built on the host, a few hundred
//    cubes) or contain at least two mass particles (built on the GPU from the
//    particles' Morton order).  It is laid out in depth-first order with
//    children in Morton order (x bit 0, y bit 1, z bit 2), which is the
//    reference's threaded nextnode/sibling order (forcetree.c:591-722): the
//    first child of item i is item i+1 and `skip` is the item after i's
//    subtree;
//  * node moments are summed over the children in that order, one level at a
//    time from the deepest (forcetree.c:622-690; force_treeupdate_toplevel
//    forcetree.c:817-890 recomputes the top nodes with the same sums);
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

#include "context.cuh"
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
    if(next <= cur) next = 0xFFFFFFFFu;  // skips always point forward; never loop
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

// ------------------------------------------------------------- tree on the GPU
//
// The oct-tree below the top-level tree is built from the mass particles in
// Morton order.  Particle k's Morton key holds the digits
// x_bit | y_bit << 1 | z_bit << 2 of levels 1..31 of its 52-bit coordinates
// (levels 1..21 in `hi`, 22..31 in `lo`).  With lam[k] the number of leading
// levels particles k and k+1 share, the cubes holding >= 2 particles that
// start at particle k are the levels in (max(lam[k-1], L), lam[k]], L the
// level of the particle's top leaf; they precede particle k's leaf item in
// the depth-first order, shallowest first.  So every item's position follows
// from a prefix sum, and a node's `skip` is the first item of the first
// particle after its cube.

constexpr int kTreeLevels = kMaxTreeLevel + 1;  // a cube of this level with two particles is refused

__global__ void k_morton(int n, const double *__restrict__ pos, double cx, double cy, double cz, double inv_len,
                         unsigned long long *__restrict__ hi, unsigned long long *__restrict__ lo,
                         int *__restrict__ idx)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= n) return;
  const unsigned long long x = int_coord(pos[3 * (size_t) i + 0], cx, inv_len);
  const unsigned long long y = int_coord(pos[3 * (size_t) i + 1], cy, inv_len);
  const unsigned long long z = int_coord(pos[3 * (size_t) i + 2], cz, inv_len);
  unsigned long long h = 0, l = 0;
  for(int lev = 1; lev <= kTreeLevels; lev++) {
    const int b = 52 - lev;
    const unsigned long long d = ((x >> b) & 1) | (((y >> b) & 1) << 1) | (((z >> b) & 1) << 2);
    if(lev <= kBits)
      h = (h << 3) | d;
    else
      l = (l << 3) | d;
  }
  hi[i] = h;
  lo[i] = l;
  idx[i] = i;
}

template <class T>
__global__ void k_gather(int n, const T *__restrict__ src, const int *__restrict__ idx, T *__restrict__ dst)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k < n) dst[k] = src[idx[k]];
}

// levels shared by particles k and k+1 (kTreeLevels: identical keys)
__device__ __forceinline__ int shared_levels(unsigned long long h0, unsigned long long l0, unsigned long long h1,
                                             unsigned long long l1)
{
  if(h0 != h1) return (__clzll((long long) (h0 ^ h1)) - 1) / 3;
  if(l0 != l1) return kBits + (__clzll((long long) (l0 ^ l1)) - (64 - 3 * (kTreeLevels - kBits))) / 3;
  return kTreeLevels;
}

// top leaf of each particle (leaves sorted by their first Morton key), the
// nodes that start at it and its item count; flags a level-31 pair
__global__ void k_particle_nodes(int n, const unsigned long long *__restrict__ hi, const unsigned long long *__restrict__ lo,
                                 int nleaves, const unsigned long long *__restrict__ leaf_start,
                                 const int *__restrict__ leaf_level, int *__restrict__ leaf_of, int *__restrict__ lo_lev,
                                 int *__restrict__ nitem, int *__restrict__ too_deep)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= n) return;
  const unsigned long long h = hi[k];
  int a = 0, b = nleaves;  // last leaf whose start <= h
  while(b - a > 1) {
    const int m = (a + b) >> 1;
    if(leaf_start[m] <= h)
      a = m;
    else
      b = m;
  }
  const int L = leaf_level[a];
  const int next = (k + 1 < n) ? shared_levels(h, lo[k], hi[k + 1], lo[k + 1]) : -1;
  const int prev = (k > 0) ? shared_levels(hi[k - 1], lo[k - 1], h, lo[k]) : -1;
  if(next >= kTreeLevels) *too_deep = 1;
  const int lo_l = max(prev, L);
  const int c = next > lo_l ? next - lo_l : 0;  // next > L implies k+1 is in the same leaf
  leaf_of[k] = a;
  lo_lev[k] = lo_l;
  nitem[k] = c + 1;
}

// first item offset (exclusive scan) of each top leaf's first particle and
// the end offset of its last particle
__global__ void k_leaf_ranges(int n, const int *__restrict__ leaf_of, const int *__restrict__ off,
                              const int *__restrict__ nitem, int *__restrict__ leaf_first, int *__restrict__ leaf_off0,
                              int *__restrict__ leaf_off1)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= n) return;
  const int T = leaf_of[k];
  if(k == 0 || leaf_of[k - 1] != T) {
    leaf_first[T] = k;
    leaf_off0[T] = off[k];
  }
  if(k == n - 1 || leaf_of[k + 1] != T) leaf_off1[T] = off[k] + nitem[k];
}

// the items of particle k: its nodes (levels lo_lev+1 .. lo_lev+c) and its leaf
__global__ void k_particle_items(int n, int nitems, double dom_len, const unsigned long long *__restrict__ hi,
                                 const unsigned long long *__restrict__ lo, const int *__restrict__ sorted,
                                 const double *__restrict__ pos, const double *__restrict__ mass,
                                 const int *__restrict__ leaf_of, const int *__restrict__ lo_lev,
                                 const int *__restrict__ nitem, const int *__restrict__ off,
                                 const int *__restrict__ leaf_item, const int *__restrict__ leaf_skip,
                                 const int *__restrict__ leaf_off0, FillItem *__restrict__ items)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k >= n) return;
  const int T = leaf_of[k];
  const int first_item = leaf_item[T] + 1 - leaf_off0[T];  // item of offset o is first_item + o
  const int base = first_item + off[k];
  const int c = nitem[k] - 1;
  const int p = sorted[k];
  const unsigned long long h = hi[k], l = lo[k];
  for(int j = 0; j < c; j++) {
    const int lev = lo_lev[k] + 1 + j;
    // end of the cube: first particle after k outside it (binary search in
    // the particles of the same leaf, which follow k in Morton order)
    int a = k, b = n;  // a inside, b outside
    while(b - a > 1) {
      const int m = (a + b) >> 1;
      const bool inside = leaf_of[m] == T && shared_levels(h, l, hi[m], lo[m]) >= lev;
      if(inside)
        a = m;
      else
        b = m;
    }
    const int g = b;
    const int skip = (g < n && leaf_of[g] == T) ? first_item + off[g] : leaf_skip[T];
    FillItem it;
    it.x = pos[3 * (size_t) p + 0];  // replaced by the centre of mass (the node holds >= 2 particles)
    it.y = pos[3 * (size_t) p + 1];
    it.z = pos[3 * (size_t) p + 2];
    it.mass = 0;
    it.len = (float) ldexp(dom_len, -lev);
    it.skip = skip < nitems ? skip : -1;
    it.pad[0] = lev;
    it.pad[1] = 0;
    items[base + j] = it;
  }
  FillItem leaf;
  leaf.x = pos[3 * (size_t) p + 0];
  leaf.y = pos[3 * (size_t) p + 1];
  leaf.z = pos[3 * (size_t) p + 2];
  leaf.mass = mass[p];
  leaf.len = -1.f;
  leaf.skip = base + c + 1 < nitems ? base + c + 1 : -1;
  leaf.pad[0] = -1;
  leaf.pad[1] = 0;
  items[base + c] = leaf;
}

__global__ void k_scatter_items(int count, const int *__restrict__ at, const FillItem *__restrict__ src,
                                FillItem *__restrict__ items)
{
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if(k < count) items[at[k]] = src[k];
}

// force_update_node_recursive (forcetree.c:622-690) for the nodes of one
// level: mass and centre of mass summed over the daughters in Morton order
// (the daughters follow the node, linked by their skips); a node without
// mass keeps the centre it was written with
__global__ void k_moments(int nitems, int level, FillItem *__restrict__ items)
{
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if(i >= nitems || items[i].pad[0] != level) return;
  const int end = items[i].skip < 0 ? nitems : items[i].skip;
  double m = 0, s0 = 0, s1 = 0, s2 = 0;
  for(int c = i + 1; c < end;) {
    const FillItem d = items[c];
    m += d.mass;
    s0 += d.mass * d.x;
    s1 += d.mass * d.y;
    s2 += d.mass * d.z;
    const int nx = (d.len < 0.f) ? c + 1 : (d.skip < 0 ? nitems : d.skip);
    c = nx > c ? nx : nitems;  // skips always point forward; never loop
  }
  if(m) {
    items[i].x = s0 / m;
    items[i].y = s1 / m;
    items[i].z = s2 / m;
  }
  items[i].mass = m;
}

// ------------------------------------------------------------- point set on the GPU

// probe points of grid.c:680-704 from the host's r1[j], z1[k], cos/sin of the
// section angles (glibc values): one IEEE product per coordinate, as there
__global__ void k_probe_points(int n, int N, const double *__restrict__ r1, const double *__restrict__ z1,
                               const double *__restrict__ trig, double *__restrict__ pos)
{
  const int NN = N * N;
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if(q >= kSections * NN) return;
  const int sct = q / NN, rem = q - sct * NN, k = rem / N, j = rem - k * N;
  double *P = pos + 3 * ((size_t) n + q);
  P[0] = r1[j] * trig[sct];
  P[1] = r1[j] * trig[kSections + sct];
  P[2] = z1[k];
}

// per-block minimum and maximum of each axis (domain_box.c:27-39); the host
// finishes the reduction.  Extremes are order independent (a +0/-0 tie
// leaves the length, centre and corner unchanged).
__global__ void __launch_bounds__(256) k_extent(int ntot, const double *__restrict__ pos, double *__restrict__ part)
{
  __shared__ double sh[6][256];
  double mn[3] = {1e306, 1e306, 1e306}, mx[3] = {-1e306, -1e306, -1e306};
  for(int i = blockIdx.x * blockDim.x + threadIdx.x; i < ntot; i += gridDim.x * blockDim.x)
#pragma unroll
    for(int j = 0; j < 3; j++) {
      const double v = pos[3 * (size_t) i + j];
      if(mn[j] > v) mn[j] = v;
      if(mx[j] < v) mx[j] = v;
    }
#pragma unroll
  for(int j = 0; j < 3; j++) {
    sh[j][threadIdx.x] = mn[j];
    sh[3 + j][threadIdx.x] = mx[j];
  }
  __syncthreads();
  for(int h = 128; h > 0; h >>= 1) {
    if(threadIdx.x < h)
#pragma unroll
      for(int j = 0; j < 3; j++) {
        if(sh[j][threadIdx.x] > sh[j][threadIdx.x + h]) sh[j][threadIdx.x] = sh[j][threadIdx.x + h];
        if(sh[3 + j][threadIdx.x] < sh[3 + j][threadIdx.x + h]) sh[3 + j][threadIdx.x] = sh[3 + j][threadIdx.x + h];
      }
    __syncthreads();
  }
  if(threadIdx.x < 6) part[6 * blockIdx.x + threadIdx.x] = sh[threadIdx.x][0];
}

// number of points whose key lies in each queried cube (Peano-Hilbert
// prefix of `level` digits), by binary search in the sorted keys
__global__ void k_count_prefix(int nq, const unsigned long long *__restrict__ prefix, const int *__restrict__ level,
                               const unsigned long long *__restrict__ keys, int nkeys, int *__restrict__ count)
{
  const int q = blockIdx.x * blockDim.x + threadIdx.x;
  if(q >= nq) return;
  const int sh = 3 * (kBits - level[q]);
  const unsigned long long lo = prefix[q] << sh, hi = (prefix[q] + 1) << sh;
  int a = 0, b = nkeys;
  while(a < b) {
    const int m = (a + b) >> 1;
    if(keys[m] < lo)
      a = m + 1;
    else
      b = m;
  }
  int c = a, d = nkeys;
  while(c < d) {
    const int m = (c + d) >> 1;
    if(keys[m] < hi)
      c = m + 1;
    else
      d = m;
  }
  count[q] = c - a;
}

// probes in key order (SoA) and the key-order rank of every probe; before[r]
// is the number of probes at sorted positions below r
__global__ void k_probe_order(int ntot, int n, int np, const int *__restrict__ order, const int *__restrict__ before,
                              const double *__restrict__ pos, double *__restrict__ probes, int *__restrict__ rank)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if(r >= ntot) return;
  const int i = order[r];
  if(i < n) return;
  const int t = before[r];
  rank[i - n] = t;
  probes[t] = pos[3 * (size_t) i + 0];
  probes[np + t] = pos[3 * (size_t) i + 1];
  probes[2 * (size_t) np + t] = pos[3 * (size_t) i + 2];
}

__global__ void k_is_probe(int ntot, int n, const int *__restrict__ order, int *__restrict__ flag)
{
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if(r < ntot) flag[r] = order[r] >= n ? 1 : 0;
}

// ------------------------------------------------------------------ host: top tree
//
// domain_determineTopTree / domain_do_local_refine (domain_toplevel.c:18-190)
// with one rank: the root is split; a cube is split when it holds more than
// 1/(TopNodeFactor * MultipleDomains) of all points (probes included) and is
// above level 21.  Cubes are enumerated depth first with daughters in Morton
// order; their float centres follow force_create_empty_nodes
// (forcetree.c:543-547).

struct TopCube {
  int level;
  bool refined;
  unsigned long long mort;  // Morton prefix of `level` digits
  float centre[3];
  float len;
  int item = 0, skip = 0, size = 0;  // set once the leaves' particle items are known
  int leaf = -1;                     // index among the leaves
};

struct TopTree {
  double fac_load, limit, len;
  const PhTables *ph;
  std::vector<TopCube> cubes;  // depth-first order

  // counts(prefixes, levels) -> point counts of those cubes.  Cubes are
  // created level by level (a cube's split depends only on its own count)
  // and then listed depth first.
  template <class Counts>
  int build(const float centre0[3], Counts counts)
  {
    struct Node {
      TopCube c;
      int rot;
      unsigned long long php;
      int child0 = -1;  // first of 8 daughters in Morton order
    };
    std::vector<Node> all(1);
    all[0].c.level = 0;
    all[0].c.mort = 0;
    all[0].c.len = (float) len;
    for(int j = 0; j < 3; j++) all[0].c.centre[j] = centre0[j];
    all[0].c.refined = true;  // the root is always split (domain_toplevel.c:43-46)
    all[0].rot = 0;
    all[0].php = 0;
    std::vector<int> frontier{0};
    while(!frontier.empty()) {
      std::vector<int> fresh;
      for(int f : frontier) {
        all[f].child0 = (int) all.size();
        const Node par = all[f];
        const double lenhalf = 0.25 * (double) par.c.len;
        for(int d = 0; d < 8; d++) {
          const int xb = d & 1, yb = (d >> 1) & 1, zb = (d >> 2) & 1;
          const int pix = (xb << 2) | (yb << 1) | zb;
          Node ch;
          ch.c.level = par.c.level + 1;
          ch.c.mort = (par.c.mort << 3) | (unsigned long long) d;
          ch.c.len = (float) (len * std::ldexp(1.0, -ch.c.level));
          ch.c.centre[0] = (float) (par.c.centre[0] + (2 * xb - 1) * lenhalf);
          ch.c.centre[1] = (float) (par.c.centre[1] + (2 * yb - 1) * lenhalf);
          ch.c.centre[2] = (float) (par.c.centre[2] + (2 * zb - 1) * lenhalf);
          ch.c.refined = false;
          ch.rot = ph->rot[par.rot][pix];
          ch.php = (par.php << 3) | ph->sub[par.rot][pix];
          fresh.push_back((int) all.size());
          all.push_back(ch);
        }
      }
      // a daughter is split when fac_load * Count > limit and it can be
      // (domain_toplevel.c:146-178)
      std::vector<unsigned long long> pre;
      std::vector<int> lev, idx;
      for(int k : fresh)
        if(all[k].c.level < kBits) {
          pre.push_back(all[k].php);
          lev.push_back(all[k].c.level);
          idx.push_back(k);
        }
      std::vector<int> cnt(pre.size(), 0);
      if(!pre.empty()) {
        const int st = counts(pre, lev, cnt);
        if(st) return st;
      }
      frontier.clear();
      for(size_t q = 0; q < idx.size(); q++)
        if(fac_load * (double) cnt[q] > limit) {
          all[idx[q]].c.refined = true;
          frontier.push_back(idx[q]);
        }
    }
    // depth-first listing, daughters in Morton order
    cubes.clear();
    std::vector<int> stack{0};
    while(!stack.empty()) {
      const int k = stack.back();
      stack.pop_back();
      cubes.push_back(all[k].c);
      if(all[k].c.refined)
        for(int d = 7; d >= 0; d--) stack.push_back(all[k].child0 + d);
    }
    return 0;
  }

  // item index, subtree size and skip of every cube, given each leaf's
  // particle item count; returns the item count of the whole tree
  int layout(const std::vector<int> &leaf_items)
  {
    int next = 0;
    // depth-first order = the order of `cubes`; a cube's subtree ends where
    // the next cube of its level or shallower starts
    for(auto &c : cubes) {
      c.item = next++;
      if(!c.refined) next += leaf_items[c.leaf];
    }
    const int total = next;
    std::vector<int> stack;  // open cubes
    for(int i = 0; i < (int) cubes.size(); i++) {
      while(!stack.empty() && cubes[stack.back()].level >= cubes[i].level) {
        cubes[stack.back()].skip = cubes[i].item;
        stack.pop_back();
      }
      stack.push_back(i);
    }
    for(int i : stack) cubes[i].skip = total;
    return total;
  }
};

// Scratch comes from the device's stream-ordered pool (kept mapped between
// calls), allocated and released in the calling thread's default stream: a
// fill allocates some thirty buffers, and plain cudaMalloc / cudaFree (which
// synchronises the device) cost more than the walk.  The kernels run in the
// legacy default stream, which orders itself with the per-thread stream.
inline cudaError_t dmalloc(void **p, size_t bytes) { return cudaMallocAsync(p, bytes, cudaStreamPerThread); }
inline void dfree_async(void *&p)
{
  if(p) cudaFreeAsync(p, cudaStreamPerThread);
  p = nullptr;
}

struct DevBuf {
  void *p = nullptr;
  ~DevBuf() { dfree_async(p); }
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
  // particles, then s, k (z), j (R); the glibc values r1[j], z1[k] and the
  // section angles' cos/sin come from the host, the products from the GPU
  std::vector<double> r1(N), z1(N);
  for(int j = 0; j < N; j++) r1[j] = fp->FG_Rmin * (std::pow(fp->FG_Fac, j) - 1.0);
  for(int k = 0; k < N; k++) z1[k] = fp->FG_Rmin * (std::pow(fp->FG_Fac, k) - 1.0);
  double trig[2 * kSections];
  for(int s = 0; s < kSections; s++) {
    const double phi = 2 * M_PI / kSections * s;
    trig[s] = std::cos(phi);
    trig[kSections + s] = std::sin(phi);
  }
  {
    int dev = 0;
    if(cudaGetDevice(&dev) != cudaSuccess || galic_internal::keep_device_pool(dev) != cudaSuccess)
      return GALIC_ERR_CUDA;
  }
  if(!upload_tables()) {
    fprintf(stderr, "galic_cuda: Peano-Hilbert table upload failed\n");
    return GALIC_ERR_CUDA;
  }
  DevBuf d_pos, d_key, d_key2, d_idx, d_idx2, d_tmp, d_r1, d_z1, d_trig, d_part;
  FCK(dmalloc(&d_pos.p, 3 * (size_t) ntot * sizeof(double)));
  FCK(dmalloc(&d_r1.p, N * sizeof(double)));
  FCK(dmalloc(&d_z1.p, N * sizeof(double)));
  FCK(dmalloc(&d_trig.p, sizeof(trig)));
  FCK(cudaMemcpy(d_pos.p, pos, 3 * (size_t) n * sizeof(double), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_r1.p, r1.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_z1.p, z1.data(), N * sizeof(double), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_trig.p, trig, sizeof(trig), cudaMemcpyHostToDevice));
  k_probe_points<<<(np + 255) / 256, 256>>>(n, N, d_r1.as<double>(), d_z1.as<double>(), d_trig.as<double>(),
                                            d_pos.as<double>());
  FCK(cudaGetLastError());
  // domain_findExtent (domain_box.c:20-65)
  const int EB = 592;
  FCK(dmalloc(&d_part.p, 6 * EB * sizeof(double)));
  k_extent<<<EB, 256>>>(ntot, d_pos.as<double>(), d_part.as<double>());
  std::vector<double> part(6 * EB);
  FCK(cudaMemcpy(part.data(), d_part.p, part.size() * sizeof(double), cudaMemcpyDeviceToHost));
  double xmin[3] = {1e306, 1e306, 1e306}, xmax[3] = {-1e306, -1e306, -1e306};
  for(int b = 0; b < EB; b++)
    for(int j = 0; j < 3; j++) {
      if(xmin[j] > part[6 * b + j]) xmin[j] = part[6 * b + j];
      if(xmax[j] < part[6 * b + 3 + j]) xmax[j] = part[6 * b + 3 + j];
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

  // keys of all points and their stable key order (peano.c:63-104)
  FCK(dmalloc(&d_key.p, (size_t) ntot * sizeof(unsigned long long)));
  FCK(dmalloc(&d_key2.p, (size_t) ntot * sizeof(unsigned long long)));
  FCK(dmalloc(&d_idx.p, (size_t) ntot * sizeof(int)));
  FCK(dmalloc(&d_idx2.p, (size_t) ntot * sizeof(int)));
  k_keys<<<(ntot + 255) / 256, 256>>>(ntot, d_pos.as<double>(), corner[0], corner[1], corner[2], inv_len,
                                      d_key.as<unsigned long long>(), d_idx.as<int>());
  FCK(cudaGetLastError());
  size_t tmp_bytes = 0;
  FCK(cub::DeviceRadixSort::SortPairs(nullptr, tmp_bytes, d_key.as<unsigned long long>(),
                                      d_key2.as<unsigned long long>(), d_idx.as<int>(), d_idx2.as<int>(), ntot, 0,
                                      3 * kBits));
  FCK(dmalloc(&d_tmp.p, tmp_bytes));
  FCK(cub::DeviceRadixSort::SortPairs(d_tmp.p, tmp_bytes, d_key.as<unsigned long long>(),
                                      d_key2.as<unsigned long long>(), d_idx.as<int>(), d_idx2.as<int>(), ntot, 0,
                                      3 * kBits));

  // top-level tree (host, a few hundred cubes; counts from the sorted keys)
  TopTree tt;
  tt.fac_load = 1.0 / (double) ntot;                              // domain.c:149
  tt.limit = 1.0 / (fp->TopNodeFactor * fp->MultipleDomains * 1);  // one rank
  tt.len = len;
  tt.ph = &host_tables();
  {
    DevBuf d_qp, d_ql, d_qc;
    size_t cap = 0;
    auto counts = [&](const std::vector<unsigned long long> &pre, const std::vector<int> &lev,
                      std::vector<int> &cnt) -> int {
      const size_t nq = pre.size();
      if(nq > cap) {
        dfree_async(d_qp.p);
        dfree_async(d_ql.p);
        dfree_async(d_qc.p);
        d_qp.p = d_ql.p = d_qc.p = nullptr;
        cap = std::max<size_t>(nq, 4096);
        FCK(dmalloc(&d_qp.p, cap * sizeof(unsigned long long)));
        FCK(dmalloc(&d_ql.p, cap * sizeof(int)));
        FCK(dmalloc(&d_qc.p, cap * sizeof(int)));
      }
      FCK(cudaMemcpy(d_qp.p, pre.data(), nq * sizeof(unsigned long long), cudaMemcpyHostToDevice));
      FCK(cudaMemcpy(d_ql.p, lev.data(), nq * sizeof(int), cudaMemcpyHostToDevice));
      k_count_prefix<<<((int) nq + 127) / 128, 128>>>((int) nq, d_qp.as<unsigned long long>(), d_ql.as<int>(),
                                                      d_key2.as<unsigned long long>(), ntot, d_qc.as<int>());
      FCK(cudaGetLastError());
      FCK(cudaMemcpy(cnt.data(), d_qc.p, nq * sizeof(int), cudaMemcpyDeviceToHost));
      return 0;
    };
    const float c0[3] = {(float) centre[0], (float) centre[1], (float) centre[2]};
    const int st = tt.build(c0, counts);
    if(st) return st;
  }
  std::vector<unsigned long long> leaf_start;
  std::vector<int> leaf_level;
  for(auto &c : tt.cubes)
    if(!c.refined) {
      c.leaf = (int) leaf_start.size();
      leaf_start.push_back(c.mort << (63 - 3 * c.level));
      leaf_level.push_back(c.level);
    }
  const int nleaves = (int) leaf_start.size();

  // oct-tree of the mass particles below the top leaves (forcetree.c:139-722),
  // built on the GPU from their Morton order
  DevBuf d_mass, d_hi, d_lo, d_hi2, d_lo2, d_pidx, d_pidx2, d_pidx3, d_lstart, d_llevel, d_leaf_of, d_lolev, d_nitem,
      d_off, d_flag, d_loff0, d_loff1, d_lfirst, d_litem, d_lskip, d_tmp2;
  const int TB = 256, TG = (n + TB - 1) / TB;
  FCK(dmalloc(&d_mass.p, (size_t) n * sizeof(double)));
  FCK(cudaMemcpy(d_mass.p, mass, (size_t) n * sizeof(double), cudaMemcpyHostToDevice));
  for(DevBuf *b : {&d_hi, &d_lo, &d_hi2, &d_lo2}) FCK(dmalloc(&b->p, (size_t) n * sizeof(unsigned long long)));
  for(DevBuf *b : {&d_pidx, &d_pidx2, &d_pidx3, &d_leaf_of, &d_lolev, &d_nitem, &d_off})
    FCK(dmalloc(&b->p, (size_t) n * sizeof(int)));
  FCK(dmalloc(&d_lstart.p, nleaves * sizeof(unsigned long long)));
  FCK(dmalloc(&d_llevel.p, nleaves * sizeof(int)));
  for(DevBuf *b : {&d_loff0, &d_loff1, &d_lfirst, &d_litem, &d_lskip}) FCK(dmalloc(&b->p, nleaves * sizeof(int)));
  FCK(dmalloc(&d_flag.p, sizeof(int)));
  FCK(cudaMemset(d_flag.p, 0, sizeof(int)));
  FCK(cudaMemset(d_loff0.p, 0, nleaves * sizeof(int)));
  FCK(cudaMemset(d_loff1.p, 0, nleaves * sizeof(int)));
  FCK(cudaMemcpy(d_lstart.p, leaf_start.data(), nleaves * sizeof(unsigned long long), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_llevel.p, leaf_level.data(), nleaves * sizeof(int), cudaMemcpyHostToDevice));
  k_morton<<<TG, TB>>>(n, d_pos.as<double>(), corner[0], corner[1], corner[2], inv_len,
                       d_hi.as<unsigned long long>(), d_lo.as<unsigned long long>(), d_pidx.as<int>());
  FCK(cudaGetLastError());
  {
    // Morton order: stable sorts by the low digits, then by the high digits
    size_t b1 = 0, b2 = 0, b3 = 0;
    FCK(cub::DeviceRadixSort::SortPairs(nullptr, b1, d_lo.as<unsigned long long>(), d_lo2.as<unsigned long long>(),
                                        d_pidx.as<int>(), d_pidx2.as<int>(), n, 0, 3 * (kTreeLevels - kBits)));
    FCK(cub::DeviceRadixSort::SortPairs(nullptr, b2, d_hi2.as<unsigned long long>(), d_hi.as<unsigned long long>(),
                                        d_pidx2.as<int>(), d_pidx3.as<int>(), n, 0, 3 * kBits));
    FCK(cub::DeviceScan::ExclusiveSum(nullptr, b3, d_nitem.as<int>(), d_off.as<int>(), n));
    FCK(dmalloc(&d_tmp2.p, std::max(b1, std::max(b2, b3))));
    size_t bb = b1;
    FCK(cub::DeviceRadixSort::SortPairs(d_tmp2.p, bb, d_lo.as<unsigned long long>(), d_lo2.as<unsigned long long>(),
                                        d_pidx.as<int>(), d_pidx2.as<int>(), n, 0, 3 * (kTreeLevels - kBits)));
    k_gather<<<TG, TB>>>(n, d_hi.as<unsigned long long>(), d_pidx2.as<int>(), d_hi2.as<unsigned long long>());
    bb = b2;
    FCK(cub::DeviceRadixSort::SortPairs(d_tmp2.p, bb, d_hi2.as<unsigned long long>(), d_hi.as<unsigned long long>(),
                                        d_pidx2.as<int>(), d_pidx3.as<int>(), n, 0, 3 * kBits));
    // d_hi: high digits in Morton order; the low digits follow them
    k_gather<<<TG, TB>>>(n, d_lo.as<unsigned long long>(), d_pidx3.as<int>(), d_lo2.as<unsigned long long>());
    k_particle_nodes<<<TG, TB>>>(n, d_hi.as<unsigned long long>(), d_lo2.as<unsigned long long>(), nleaves,
                                 d_lstart.as<unsigned long long>(), d_llevel.as<int>(), d_leaf_of.as<int>(),
                                 d_lolev.as<int>(), d_nitem.as<int>(), d_flag.as<int>());
    bb = b3;
    FCK(cub::DeviceScan::ExclusiveSum(d_tmp2.p, bb, d_nitem.as<int>(), d_off.as<int>(), n));
    k_leaf_ranges<<<TG, TB>>>(n, d_leaf_of.as<int>(), d_off.as<int>(), d_nitem.as<int>(), d_lfirst.as<int>(),
                              d_loff0.as<int>(), d_loff1.as<int>());
    FCK(cudaGetLastError());
  }
  int too_deep = 0;
  FCK(cudaMemcpy(&too_deep, d_flag.p, sizeof(int), cudaMemcpyDeviceToHost));
  if(too_deep) return GALIC_ERR_UNSUPPORTED;  // particles closer than DomainLen / 2^30
  std::vector<int> loff0(nleaves), loff1(nleaves), leaf_items(nleaves);
  FCK(cudaMemcpy(loff0.data(), d_loff0.p, nleaves * sizeof(int), cudaMemcpyDeviceToHost));
  FCK(cudaMemcpy(loff1.data(), d_loff1.p, nleaves * sizeof(int), cudaMemcpyDeviceToHost));
  for(int T = 0; T < nleaves; T++) leaf_items[T] = loff1[T] - loff0[T];
  const int nitems = tt.layout(leaf_items);
  std::vector<int> litem(nleaves), lskip(nleaves), at;
  std::vector<FillItem> top_items;
  for(const auto &c : tt.cubes) {
    if(!c.refined) {
      litem[c.leaf] = c.item;
      lskip[c.leaf] = c.skip;
    }
    FillItem it{};
    it.x = c.centre[0];
    it.y = c.centre[1];
    it.z = c.centre[2];
    it.mass = 0;
    it.len = c.len;
    it.skip = c.skip < nitems ? c.skip : -1;
    it.pad[0] = c.level;
    top_items.push_back(it);
    at.push_back(c.item);
  }
  DevBuf d_items, d_top, d_at;
  FCK(dmalloc(&d_items.p, (size_t) nitems * sizeof(FillItem)));
  FCK(dmalloc(&d_top.p, top_items.size() * sizeof(FillItem)));
  FCK(dmalloc(&d_at.p, at.size() * sizeof(int)));
  FCK(cudaMemcpy(d_top.p, top_items.data(), top_items.size() * sizeof(FillItem), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_at.p, at.data(), at.size() * sizeof(int), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_litem.p, litem.data(), nleaves * sizeof(int), cudaMemcpyHostToDevice));
  FCK(cudaMemcpy(d_lskip.p, lskip.data(), nleaves * sizeof(int), cudaMemcpyHostToDevice));
  k_scatter_items<<<((int) at.size() + 127) / 128, 128>>>((int) at.size(), d_at.as<int>(), d_top.as<FillItem>(),
                                                          d_items.as<FillItem>());
  k_particle_items<<<TG, TB>>>(n, nitems, len, d_hi.as<unsigned long long>(), d_lo2.as<unsigned long long>(),
                               d_pidx3.as<int>(), d_pos.as<double>(), d_mass.as<double>(), d_leaf_of.as<int>(),
                               d_lolev.as<int>(), d_nitem.as<int>(), d_off.as<int>(), d_litem.as<int>(),
                               d_lskip.as<int>(), d_loff0.as<int>(), d_items.as<FillItem>());
  for(int lev = kTreeLevels - 1; lev >= 0; lev--)
    k_moments<<<(nitems + 255) / 256, 256>>>(nitems, lev, d_items.as<FillItem>());
  FCK(cudaGetLastError());

  // probes in key order (SoA) and the key-order rank of each probe
  DevBuf d_probes, d_res, d_rank, d_out, d_counts, d_flag2, d_before;
  FCK(dmalloc(&d_probes.p, 3 * (size_t) np * sizeof(double)));
  FCK(dmalloc(&d_res.p, 4 * (size_t) np * sizeof(double)));
  FCK(dmalloc(&d_rank.p, (size_t) np * sizeof(int)));
  FCK(dmalloc(&d_out.p, 3 * (size_t) NN * sizeof(double)));
  FCK(dmalloc(&d_flag2.p, (size_t) ntot * sizeof(int)));
  FCK(dmalloc(&d_before.p, (size_t) ntot * sizeof(int)));
  k_is_probe<<<(ntot + 255) / 256, 256>>>(ntot, n, d_idx2.as<int>(), d_flag2.as<int>());
  {
    size_t b = 0;
    FCK(cub::DeviceScan::ExclusiveSum(nullptr, b, d_flag2.as<int>(), d_before.as<int>(), ntot));
    DevBuf d_t3;
    FCK(dmalloc(&d_t3.p, b));
    FCK(cub::DeviceScan::ExclusiveSum(d_t3.p, b, d_flag2.as<int>(), d_before.as<int>(), ntot));
  }
  k_probe_order<<<(ntot + 255) / 256, 256>>>(ntot, n, np, d_idx2.as<int>(), d_before.as<int>(), d_pos.as<double>(),
                                             d_probes.as<double>(), d_rank.as<int>());
  FCK(cudaGetLastError());
  FCK(dmalloc(&d_counts.p, 2 * sizeof(unsigned long long)));
  FCK(cudaMemset(d_counts.p, 0, 2 * sizeof(unsigned long long)));

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
