/*
 * oracle_forcegrid.c - CPU restatement of GALIC's tree force-grid fill.
 * TEST INFRASTRUCTURE (the checker of galic_force_grid_fill); see
 * galic_oracle.h.
 *
 * Follows the single-rank reference step by step: probe placement
 * (grid.c:680-704), domain cube (domain_box.c:20-65), 21-bit coordinates and
 * Peano-Hilbert keys (domain.c:155-164, peano.c:331-347), top-level tree by
 * key segments (domain_toplevel.c:18-171), stable key order (peano.c:63-104,
 * 653-705), empty top nodes (forcetree.c:510-564), one-by-one particle
 * insertion (forcetree.c:184-495), recursive moments (forcetree.c:591-722),
 * the walk (forcetree_walk.c:12-222), G scaling (gravtree.c:456-463) and the
 * readout (grid.c:720-750).  The tree is built by insertion, as the reference
 * does, and walked by recursion over the daughters in Morton order, which
 * visits the same items in the same order as the reference's threaded walk.
 * Build with -ffp-contract=off.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "galic_oracle.h"

#define ORC_SECTIONS 8 /* FG_SECTIONS, allvars.h:123 */
#define ORC_BITS 21    /* BITS_PER_DIMENSION, allvars.h:213 */
#define ORC_MAXLEVEL 30 /* MAX_TREE_LEVEL, forcetree.h:16 */

/* Peano-Hilbert state machine (peano.c:226-330): next state and key digit
 * for state 0..47 and octant 4x+2y+z; must equal the reference's tables. */
static const unsigned char ph_next[48][8] = {
    {36, 28, 25, 27, 10, 10, 25, 27}, {29, 11, 24, 24, 37, 11, 26, 26}, {8, 8, 25, 27, 30, 38, 25, 27},
    {9, 39, 24, 24, 9, 31, 26, 26},   {40, 24, 44, 32, 40, 6, 44, 6},   {25, 7, 33, 7, 41, 41, 45, 45},
    {4, 42, 4, 46, 26, 42, 34, 46},   {43, 43, 47, 47, 5, 27, 5, 35},   {33, 35, 36, 28, 33, 35, 2, 2},
    {32, 32, 29, 3, 34, 34, 37, 3},   {33, 35, 0, 0, 33, 35, 30, 38},   {32, 32, 1, 39, 34, 34, 1, 31},
    {24, 42, 32, 46, 14, 42, 14, 46}, {43, 43, 47, 47, 25, 15, 33, 15}, {40, 12, 44, 12, 40, 26, 44, 34},
    {13, 27, 13, 35, 41, 41, 45, 45}, {28, 41, 28, 22, 38, 43, 38, 22}, {42, 40, 23, 23, 29, 39, 29, 39},
    {41, 36, 20, 36, 43, 30, 20, 30}, {37, 31, 37, 31, 42, 40, 21, 21}, {28, 18, 28, 45, 38, 18, 38, 47},
    {19, 19, 46, 44, 29, 39, 29, 39}, {16, 36, 45, 36, 16, 30, 47, 30}, {37, 31, 37, 31, 17, 17, 46, 44},
    {12, 4, 1, 3, 34, 34, 1, 3},      {5, 35, 0, 0, 13, 35, 2, 2},      {32, 32, 1, 3, 6, 14, 1, 3},
    {33, 15, 0, 0, 33, 7, 2, 2},      {16, 0, 20, 8, 16, 30, 20, 30},   {1, 31, 9, 31, 17, 17, 21, 21},
    {28, 18, 28, 22, 2, 18, 10, 22},  {19, 19, 23, 23, 29, 3, 29, 11},  {9, 11, 12, 4, 9, 11, 26, 26},
    {8, 8, 5, 27, 10, 10, 13, 27},    {9, 11, 24, 24, 9, 11, 6, 14},    {8, 8, 25, 15, 10, 10, 25, 7},
    {0, 18, 8, 22, 38, 18, 38, 22},   {19, 19, 23, 23, 1, 39, 9, 39},   {16, 36, 20, 36, 16, 2, 20, 10},
    {37, 3, 37, 11, 17, 17, 21, 21},  {4, 17, 4, 46, 14, 19, 14, 46},   {18, 16, 47, 47, 5, 15, 5, 15},
    {17, 12, 44, 12, 19, 6, 44, 6},   {13, 7, 13, 7, 18, 16, 45, 45},   {4, 42, 4, 21, 14, 42, 14, 23},
    {43, 43, 22, 20, 5, 15, 5, 15},   {40, 12, 21, 12, 40, 6, 23, 6},   {13, 7, 13, 7, 41, 41, 22, 20}};
static const unsigned char ph_digit[48][8] = {
    {0, 7, 1, 6, 3, 4, 2, 5}, {7, 4, 6, 5, 0, 3, 1, 2}, {4, 3, 5, 2, 7, 0, 6, 1}, {3, 0, 2, 1, 4, 7, 5, 6},
    {1, 0, 6, 7, 2, 3, 5, 4}, {0, 3, 7, 4, 1, 2, 6, 5}, {3, 2, 4, 5, 0, 1, 7, 6}, {2, 1, 5, 6, 3, 0, 4, 7},
    {6, 1, 7, 0, 5, 2, 4, 3}, {1, 2, 0, 3, 6, 5, 7, 4}, {2, 5, 3, 4, 1, 6, 0, 7}, {5, 6, 4, 7, 2, 1, 3, 0},
    {7, 6, 0, 1, 4, 5, 3, 2}, {6, 5, 1, 2, 7, 4, 0, 3}, {5, 4, 2, 3, 6, 7, 1, 0}, {4, 7, 3, 0, 5, 6, 2, 1},
    {6, 7, 5, 4, 1, 0, 2, 3}, {7, 0, 4, 3, 6, 1, 5, 2}, {0, 1, 3, 2, 7, 6, 4, 5}, {1, 6, 2, 5, 0, 7, 3, 4},
    {2, 3, 1, 0, 5, 4, 6, 7}, {3, 4, 0, 7, 2, 5, 1, 6}, {4, 5, 7, 6, 3, 2, 0, 1}, {5, 2, 6, 1, 4, 3, 7, 0},
    {7, 0, 6, 1, 4, 3, 5, 2}, {0, 3, 1, 2, 7, 4, 6, 5}, {3, 4, 2, 5, 0, 7, 1, 6}, {4, 7, 5, 6, 3, 0, 2, 1},
    {6, 7, 1, 0, 5, 4, 2, 3}, {7, 4, 0, 3, 6, 5, 1, 2}, {4, 5, 3, 2, 7, 6, 0, 1}, {5, 6, 2, 1, 4, 7, 3, 0},
    {1, 6, 0, 7, 2, 5, 3, 4}, {6, 5, 7, 4, 1, 2, 0, 3}, {5, 2, 4, 3, 6, 1, 7, 0}, {2, 1, 3, 0, 5, 6, 4, 7},
    {0, 1, 7, 6, 3, 2, 4, 5}, {1, 2, 6, 5, 0, 3, 7, 4}, {2, 3, 5, 4, 1, 0, 6, 7}, {3, 0, 4, 7, 2, 1, 5, 6},
    {1, 0, 2, 3, 6, 7, 5, 4}, {0, 7, 3, 4, 1, 6, 2, 5}, {7, 6, 4, 5, 0, 1, 3, 2}, {6, 1, 5, 2, 7, 0, 4, 3},
    {5, 4, 6, 7, 2, 3, 1, 0}, {4, 3, 7, 0, 5, 2, 6, 1}, {3, 2, 0, 1, 4, 5, 7, 6}, {2, 5, 1, 6, 3, 4, 0, 7}};

uint64_t orc_peano_key(int x, int y, int z, int bits) /* peano.c:331-347 */
{
  int state = 0, b;
  uint64_t key = 0;
  for(b = bits - 1; b >= 0; b--) {
    int oct = (((x >> b) & 1) << 2) | (((y >> b) & 1) << 1) | ((z >> b) & 1);
    key = (key << 3) | ph_digit[state][oct];
    state = ph_next[state][oct];
  }
  return key;
}

static uint64_t mant52(double d) /* force_double_to_int, forcetree.h:33-38 */
{
  uint64_t u;
  memcpy(&u, &d, sizeof(u));
  return u & 0xFFFFFFFFFFFFFull;
}

/* ------------------------------------------------------------- top tree */

typedef struct {
  uint64_t start, size; /* key range [start, start + size) */
  long first, count;    /* points in the sorted key array */
  int daughter;         /* first of 8 daughters in key order, or -1 */
} orc_top;

typedef struct {
  orc_top *t;
  int n, cap;
} orc_toplist;

static int top_add(orc_toplist *L)
{
  if(L->n == L->cap) {
    L->cap = L->cap ? 2 * L->cap : 64;
    L->t = (orc_top *) realloc(L->t, (size_t) L->cap * sizeof(orc_top));
  }
  return L->n++;
}

/* domain_do_local_refine (domain_toplevel.c:69-190), one rank: the root is
 * split; a daughter is split when fac_load * Count > limit and it can be */
static void top_refine(orc_toplist *L, int node, const uint64_t *keys, double fac_load, double limit)
{
  int j, d0 = top_add(L);
  for(j = 1; j < 8; j++) top_add(L);
  L->t[node].daughter = d0;
  long p = L->t[node].first, end = L->t[node].first + L->t[node].count;
  for(j = 0; j < 8; j++) {
    orc_top *c = &L->t[d0 + j];
    c->size = L->t[node].size >> 3;
    c->start = L->t[node].start + (uint64_t) j * c->size;
    c->daughter = -1;
    c->first = p;
    while(p < end && keys[p] < c->start + c->size) p++;
    c->count = p - c->first;
  }
  for(j = 0; j < 8; j++) {
    double work = fac_load * L->t[d0 + j].count;
    if(work > limit && L->t[d0 + j].size >= 8) top_refine(L, d0 + j, keys, fac_load, limit);
  }
}

/* --------------------------------------------------------------- oct-tree */

typedef struct {
  int suns[8]; /* -1 empty, 0..n-1 particle, n+k node k */
  double s[3], mass;
  float center[3], len;
} orc_node;

typedef struct {
  orc_node *nd;
  int n, cap, npart;
} orc_tree;

static int node_add(orc_tree *T)
{
  if(T->n == T->cap) {
    T->cap = T->cap ? 2 * T->cap : 1024;
    T->nd = (orc_node *) realloc(T->nd, (size_t) T->cap * sizeof(orc_node));
  }
  int k = T->n++, j;
  for(j = 0; j < 8; j++) T->nd[k].suns[j] = -1;
  return k;
}

/* force_create_empty_nodes (forcetree.c:510-564): daughters of every split
 * top node, in Morton order i + 2j + 4k, with float centres */
static void empty_nodes(orc_tree *T, int node, const orc_toplist *L, int top, int bits, int x, int y, int z)
{
  int i, j, k;
  if(L->t[top].daughter < 0) return;
  for(i = 0; i < 2; i++)
    for(j = 0; j < 2; j++)
      for(k = 0; k < 2; k++) {
        int sub = (int) (7 & orc_peano_key((x << 1) + i, (y << 1) + j, (z << 1) + k, bits));
        int c = node_add(T);
        orc_node *p = &T->nd[node], *q = &T->nd[c];
        double half = 0.25 * p->len;
        q->len = 0.5 * p->len;
        q->center[0] = p->center[0] + (2 * i - 1) * half;
        q->center[1] = p->center[1] + (2 * j - 1) * half;
        q->center[2] = p->center[2] + (2 * k - 1) * half;
        p->suns[i + 2 * j + 4 * k] = T->npart + c;
        empty_nodes(T, c, L, L->t[top].daughter + sub, bits + 1, 2 * x + i, 2 * y + j, 2 * z + k);
      }
}

static int octant(const uint64_t *ip, int level)
{
  int b = 51 - level;
  return (int) (((ip[0] >> b) & 1) | (((ip[1] >> b) & 1) << 1) | (((ip[2] >> b) & 1) << 2));
}

/* force_treebuild_insert_single_point (forcetree.c:361-495) from the root;
 * returns 1 when the MAX_TREE_LEVEL case (forcetree.c:400-416) is met */
static int insert(orc_tree *T, int p, const uint64_t *ipos, double corner[3], double bigfac)
{
  int node = 0, level = 0;
  for(;;) {
    int sub = octant(&ipos[3 * p], level);
    level++;
    int c = T->nd[node].suns[sub];
    if(c >= 0 && level > ORC_MAXLEVEL) return 1; /* the slot shift would reshape the tree */
    if(c < 0) {
      T->nd[node].suns[sub] = p;
      return 0;
    }
    if(c >= T->npart) {
      node = c - T->npart;
      continue;
    }
    /* a particle occupies the slot: a new node for the level-`level` cube */
    int k = node_add(T), j;
    orc_node *q = &T->nd[k];
    uint64_t mask = (uint64_t) 1 << (51 - level), cmask = ~((mask << 1) - 1) & 0xFFFFFFFFFFFFFull;
    q->len = (float) ((double) (mask << 1) * bigfac);
    for(j = 0; j < 3; j++) q->center[j] = (float) ((double) ((ipos[3 * p + j] & cmask) | mask) * bigfac + corner[j]);
    q->suns[octant(&ipos[3 * c], level)] = c;
    T->nd[node].suns[sub] = T->npart + k;
    node = k;
  }
}

/* force_update_node_recursive (forcetree.c:591-722): moments over suns 0..7 */
static void moments(orc_tree *T, int node, const double *pos, const double *mass)
{
  double s[3] = {0, 0, 0}, m = 0;
  int j;
  for(j = 0; j < 8; j++) {
    int c = T->nd[node].suns[j];
    if(c < 0) continue;
    if(c < T->npart) {
      m += mass[c];
      s[0] += mass[c] * pos[3 * c + 0];
      s[1] += mass[c] * pos[3 * c + 1];
      s[2] += mass[c] * pos[3 * c + 2];
    } else {
      int k = c - T->npart;
      moments(T, k, pos, mass);
      m += T->nd[k].mass;
      s[0] += T->nd[k].mass * T->nd[k].s[0];
      s[1] += T->nd[k].mass * T->nd[k].s[1];
      s[2] += T->nd[k].mass * T->nd[k].s[2];
    }
  }
  orc_node *q = &T->nd[node];
  if(m) {
    q->s[0] = s[0] / m;
    q->s[1] = s[1] / m;
    q->s[2] = s[2] / m;
  } else {
    q->s[0] = q->center[0];
    q->s[1] = q->center[1];
    q->s[2] = q->center[2];
  }
  q->mass = m;
}

typedef struct {
  double px, py, pz, h, theta;
  double ax, ay, az, pot;
} orc_walker;

/* the interaction of forcetree_walk.c:156-196 */
static void interact(orc_walker *w, double dx, double dy, double dz, double r2, double mass)
{
  double r, u, fac, wp, h_inv, h3_inv;
  if(!mass) return;
  r = sqrt(r2);
  if(r >= w->h) {
    fac = mass / (r2 * r);
    wp = -mass / r;
  } else {
    h_inv = 1.0 / w->h;
    h3_inv = h_inv * h_inv * h_inv;
    u = r * h_inv;
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
  w->ax += dx * fac;
  w->ay += dy * fac;
  w->az += dz * fac;
  w->pot += wp;
}

/* force_treeevaluate (forcetree_walk.c:12-222): a node is opened when its
 * float len squared exceeds r2 theta^2, then its daughters are visited in
 * suns order */
static void walk(const orc_tree *T, int node, orc_walker *w, const double *pos, const double *mass)
{
  const orc_node *q = &T->nd[node];
  double dx = q->s[0] - w->px, dy = q->s[1] - w->py, dz = q->s[2] - w->pz;
  double r2 = dx * dx + dy * dy + dz * dz;
  if(q->len * q->len > r2 * w->theta * w->theta) {
    int j;
    for(j = 0; j < 8; j++) {
      int c = q->suns[j];
      if(c < 0) continue;
      if(c >= T->npart)
        walk(T, c - T->npart, w, pos, mass);
      else {
        double ex = pos[3 * c + 0] - w->px, ey = pos[3 * c + 1] - w->py, ez = pos[3 * c + 2] - w->pz;
        interact(w, ex, ey, ez, ex * ex + ey * ey + ez * ez, mass[c]);
      }
    }
    return;
  }
  interact(w, dx, dy, dz, r2, q->mass);
}

typedef struct {
  uint64_t key;
  long idx;
} orc_keyed;

static void merge_sort(orc_keyed *a, long n, orc_keyed *tmp) /* stable, as peano.c:653-690 */
{
  long n1 = n / 2, i = 0, j = n1, k = 0;
  if(n <= 1) return;
  merge_sort(a, n1, tmp);
  merge_sort(a + n1, n - n1, tmp);
  while(i < n1 && j < n) tmp[k++] = (a[i].key <= a[j].key) ? a[i++] : a[j++];
  while(i < n1) tmp[k++] = a[i++];
  memcpy(a, tmp, (size_t) k * sizeof(orc_keyed));
}

int orc_force_grid_fill(const galic_fill_params_t *fp, int n, const double *pos_in, const double *mass_in,
                        double *dpotdr, double *dpotdz, double *potgrid)
{
  const int N = fp->FG_Nbin, NN = N * N, np = NN * ORC_SECTIONS, ntot = n + np;
  double *P = (double *) malloc(3 * (size_t) ntot * sizeof(double));
  double *M = (double *) calloc((size_t) ntot, sizeof(double));
  int *ID = (int *) malloc((size_t) ntot * sizeof(int));
  int i, j, k, s, status = 0;
  memcpy(P, pos_in, 3 * (size_t) n * sizeof(double));
  memcpy(M, mass_in, (size_t) n * sizeof(double));
  for(i = 0; i < n; i++) ID[i] = -1;
  /* grid.c:680-704 */
  for(s = 0, i = n; s < ORC_SECTIONS; s++)
    for(k = 0; k < N; k++)
      for(j = 0; j < N; j++, i++) {
        double phi = 2 * M_PI / ORC_SECTIONS * s;
        double r1 = fp->FG_Rmin * (pow(fp->FG_Fac, j) - 1.0);
        double z1 = fp->FG_Rmin * (pow(fp->FG_Fac, k) - 1.0);
        ID[i] = s * NN + k * N + j;
        P[3 * i + 0] = r1 * cos(phi);
        P[3 * i + 1] = r1 * sin(phi);
        P[3 * i + 2] = z1;
      }
  /* domain_box.c:20-65 */
  double xmin[3], xmax[3], len = 0, corner[3], centre[3];
  for(j = 0; j < 3; j++) {
    xmin[j] = 1.0e306;
    xmax[j] = -1.0e306;
  }
  for(i = 0; i < ntot; i++)
    for(j = 0; j < 3; j++) {
      if(xmin[j] > P[3 * i + j]) xmin[j] = P[3 * i + j];
      if(xmax[j] < P[3 * i + j]) xmax[j] = P[3 * i + j];
    }
  for(j = 0; j < 3; j++)
    if(xmax[j] - xmin[j] > len) len = xmax[j] - xmin[j];
  len *= 1.00001;
  for(j = 0; j < 3; j++) {
    centre[j] = 0.5 * (xmin[j] + xmax[j]);
    corner[j] = 0.5 * (xmin[j] + xmax[j]) - 0.5 * len;
  }
  double inv_len = 1.0 / len, bigfac = len / ((long long) 1 << 52);
  /* keys and the stable key order */
  orc_keyed *ord = (orc_keyed *) malloc((size_t) ntot * sizeof(orc_keyed));
  orc_keyed *tmp = (orc_keyed *) malloc((size_t) ntot * sizeof(orc_keyed));
  for(i = 0; i < ntot; i++) {
    int c[3];
    for(j = 0; j < 3; j++) c[j] = (int) (mant52(((P[3 * i + j] - corner[j]) * inv_len) + 1.0) >> (52 - ORC_BITS));
    ord[i].key = orc_peano_key(c[0], c[1], c[2], ORC_BITS);
    ord[i].idx = i;
  }
  merge_sort(ord, ntot, tmp);
  free(tmp);
  uint64_t *keys = (uint64_t *) malloc((size_t) ntot * sizeof(uint64_t));
  for(i = 0; i < ntot; i++) keys[i] = ord[i].key;
  /* the points in key order (peano_hilbert_order reorders P) */
  double *Ps = (double *) malloc(3 * (size_t) ntot * sizeof(double));
  double *Ms = (double *) malloc((size_t) ntot * sizeof(double));
  int *IDs = (int *) malloc((size_t) ntot * sizeof(int));
  for(i = 0; i < ntot; i++) {
    long o = ord[i].idx;
    memcpy(&Ps[3 * i], &P[3 * o], 3 * sizeof(double));
    Ms[i] = M[o];
    IDs[i] = ID[o];
  }
  /* top-level tree */
  orc_toplist L = {0, 0, 0};
  int root = top_add(&L);
  L.t[root].start = 0;
  L.t[root].size = (uint64_t) 1 << (3 * ORC_BITS);
  L.t[root].first = 0;
  L.t[root].count = ntot;
  L.t[root].daughter = -1;
  top_refine(&L, root, keys, 1.0 / ntot, 1.0 / (fp->TopNodeFactor * fp->MultipleDomains * 1));
  /* oct-tree over the mass particles of the key-ordered points */
  int nm = 0;
  int *midx = (int *) malloc((size_t) ntot * sizeof(int));
  for(i = 0; i < ntot; i++)
    if(IDs[i] < 0) midx[nm++] = i;
  double *mp = (double *) malloc(3 * (size_t) (nm ? nm : 1) * sizeof(double));
  double *mm = (double *) malloc((size_t) (nm ? nm : 1) * sizeof(double));
  uint64_t *ip = (uint64_t *) malloc(3 * (size_t) (nm ? nm : 1) * sizeof(uint64_t));
  for(i = 0; i < nm; i++) {
    memcpy(&mp[3 * i], &Ps[3 * midx[i]], 3 * sizeof(double));
    mm[i] = Ms[midx[i]];
    for(j = 0; j < 3; j++) ip[3 * i + j] = mant52(((mp[3 * i + j] - corner[j]) * inv_len) + 1.0);
  }
  orc_tree T = {0, 0, 0, nm};
  int r0 = node_add(&T);
  T.nd[r0].len = len;
  for(j = 0; j < 3; j++) T.nd[r0].center[j] = centre[j];
  empty_nodes(&T, r0, &L, root, 1, 0, 0, 0);
  for(i = 0; i < nm && !status; i++) status = insert(&T, i, ip, corner, bigfac);
  if(!status) {
    moments(&T, r0, mp, mm);
    double *acc = (double *) calloc(3 * (size_t) NN, sizeof(double));
    /* walk for every probe in key order, readout in that order */
    for(i = 0; i < ntot; i++) {
      if(IDs[i] < 0) continue;
      orc_walker w = {Ps[3 * i + 0], Ps[3 * i + 1], Ps[3 * i + 2], fp->ForceSoftening, fp->ErrTolTheta, 0, 0, 0, 0};
      walk(&T, r0, &w, mp, mm);
      double gx = w.ax * fp->G, gy = w.ay * fp->G, gz = w.az * fp->G, gp = w.pot * fp->G;
      int id = IDs[i], sec = id / NN, cell = id - sec * NN;
      double phi = 2 * M_PI / ORC_SECTIONS * sec;
      acc[cell] += gx * cos(phi) + gy * sin(phi);
      acc[NN + cell] += gz;
      acc[2 * NN + cell] += gp;
    }
    for(i = 0; i < NN; i++) {
      dpotdr[i] = acc[i] / ORC_SECTIONS;
      dpotdz[i] = acc[NN + i] / ORC_SECTIONS;
      potgrid[i] = acc[2 * NN + i] / ORC_SECTIONS;
    }
    free(acc);
  }
  free(T.nd);
  free(L.t);
  free(ip);
  free(mm);
  free(mp);
  free(midx);
  free(IDs);
  free(Ms);
  free(Ps);
  free(keys);
  free(ord);
  free(ID);
  free(M);
  free(P);
  return status ? GALIC_ERR_UNSUPPORTED : GALIC_OK;
}
