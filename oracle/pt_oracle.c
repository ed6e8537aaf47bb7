/*
 * pt_oracle.c -- CPU oracle for ParaTreeT's Barnes-Hut gravity path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the "port"
 * CPU baseline.  The product never links, loads or calls this file.
 *
 * A plain-C, structure-of-arrays restatement of the reference path, FP64
 * throughout, compiled with -ffp-contract=off so that every expression is
 * evaluated exactly as the reference (built -DUSE_DOUBLE_FP) evaluates it.
 * Arithmetic expressions that decide bit-exact parity keep the reference's
 * association order; each block cites the reference lines it restates.
 */
#include "pt_oracle.h"
#include "pt_sfc.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define PTO_MAX_DEPTH 21 /* 63 key bits / 3 */
#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif
#ifndef M_1_PI
#define M_1_PI 0.31830988618379067154
#endif

typedef struct {
  double mass, cm[3], soft, radius;
  double xx, xy, xz, yy, yz, zz;
  double lo[3], hi[3];
  int count;
} pto_mom;

struct pto_sim {
  int n, bucket, threads;
  double theta, dt_max, last_dt;
  /* particles, current (key-sorted after a build) order */
  double *x, *y, *z, *vx, *vy, *vz, *m, *soft;
  double *ax, *ay, *az, *pot, *potf;
  int* order;
  uint64_t* key;
  double ulo[3], uhi[3];
  /* tree */
  long nnodes, cap;
  uint64_t* nkey;
  int *ntype, *ndepth, *npstart, *nnp, *nparent, *nchild, *nwait;
  pto_mom* mom;
  int *leaves, *empties;
  long nleaves, nempties, leafcap, emptycap;
  /* interaction lists of the last evaluation */
  long *list_off;
  uint64_t* list_key;
  int* list_kind;
  long list_total, list_cap;
  unsigned long long n_pp, n_pc, n_open;
  unsigned long long n_mono; /* node() calls that took the monopole fallback */
  double t_build, t_trav;
  /* periodic cube (examples/Gravity.C:34-50, examples/Ewald.{h,C}) */
  int periodic, n_replicas;
  /* 0: TransposedDownTraverser (startDown), 1: BasicDownTraverser (startBasicDown) */
  int basic_down;
  double period, ewald_rcut, ewald_hcut;
};

static double wall(void) {
#ifdef _OPENMP
  return omp_get_wtime();
#else
  return 0.0;
#endif
}

/* ---------------------------------------------------------------- universe
 * src/Driver.h:67-80 (remakeUniverse): cube centred on the bbox centre with
 * half-side (1 + 1.91e-6) * 0.5 * longest side. */
static void remake_universe(pto_sim* s, const double blo[3], const double bhi[3]) {
  double sx = bhi[0] - blo[0], sy = bhi[1] - blo[1], sz = bhi[2] - blo[2];
  double mx = (sx > sy) ? sx : sy;
  mx = (mx > sz) ? mx : sz;
  double c[3];
  for (int d = 0; d < 3; d++) c[d] = (blo[d] + bhi[d]) / 2.0;
  const double fEps = 1.0 + 1.91e-6;
  double h = fEps * 0.5 * mx;
  for (int d = 0; d < 3; d++) {
    s->ulo[d] = c[d] - h;
    s->uhi[d] = c[d] + h;
  }
}

static void particle_bbox(const pto_sim* s, double lo[3], double hi[3]) {
  lo[0] = lo[1] = lo[2] = 1.7976931348623157e308;
  hi[0] = hi[1] = hi[2] = -1.7976931348623157e308;
  for (int i = 0; i < s->n; i++) {
    double p[3] = {s->x[i], s->y[i], s->z[i]};
    for (int d = 0; d < 3; d++) {
      if (p[d] < lo[d]) lo[d] = p[d];
      if (p[d] > hi[d]) hi[d] = p[d];
    }
  }
}

/* src/Decomposition.C:58-64: key = SFC key | placeholder bit 63. */
static void assign_keys(pto_sim* s) {
  for (int i = 0; i < s->n; i++)
    s->key[i] = pt_morton_key(s->x[i], s->y[i], s->z[i], s->ulo, s->uhi) | PT_KEY_PLACEHOLDER;
}

/* ---------------------------------------------------------------- sort
 * src/Subtree.h:281 sorts the particles by key (Particle::operator<,
 * src/Particle.C:61-79).  Stable LSD radix sort here: equal keys keep their
 * current order. */
static void permute_d(double* a, const int* perm, double* tmp, int n) {
  for (int i = 0; i < n; i++) tmp[i] = a[perm[i]];
  memcpy(a, tmp, sizeof(double) * (size_t)n);
}

static void sort_particles(pto_sim* s) {
  int n = s->n;
  int* idx = (int*)malloc(sizeof(int) * (size_t)n);
  int* idx2 = (int*)malloc(sizeof(int) * (size_t)n);
  uint64_t* k2 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  uint64_t* k1 = (uint64_t*)malloc(sizeof(uint64_t) * (size_t)n);
  for (int i = 0; i < n; i++) { idx[i] = i; k1[i] = s->key[i]; }
  for (int pass = 0; pass < 8; pass++) {
    int shift = pass * 8;
    long cnt[257];
    memset(cnt, 0, sizeof(cnt));
    for (int i = 0; i < n; i++) cnt[((k1[i] >> shift) & 0xff) + 1]++;
    for (int b = 0; b < 256; b++) cnt[b + 1] += cnt[b];
    for (int i = 0; i < n; i++) {
      long d = cnt[(k1[i] >> shift) & 0xff]++;
      k2[d] = k1[i];
      idx2[d] = idx[i];
    }
    uint64_t* tk = k1; k1 = k2; k2 = tk;
    int* ti = idx; idx = idx2; idx2 = ti;
  }
  double* tmp = (double*)malloc(sizeof(double) * (size_t)n);
  permute_d(s->x, idx, tmp, n);
  permute_d(s->y, idx, tmp, n);
  permute_d(s->z, idx, tmp, n);
  permute_d(s->vx, idx, tmp, n);
  permute_d(s->vy, idx, tmp, n);
  permute_d(s->vz, idx, tmp, n);
  permute_d(s->m, idx, tmp, n);
  permute_d(s->soft, idx, tmp, n);
  for (int i = 0; i < n; i++) idx2[i] = s->order[idx[i]];
  memcpy(s->order, idx2, sizeof(int) * (size_t)n);
  memcpy(s->key, k1, sizeof(uint64_t) * (size_t)n);
  free(tmp); free(idx); free(idx2); free(k1); free(k2);
}

/* ---------------------------------------------------------------- moments
 * Leaf data: CentroidData(particles, n, depth), examples/CentroidData.h:41-59,
 * accumulating MultipoleMoments::operator+=(Particle) in particle order,
 * examples/MultipoleMoments.h:274-353 (non-HEXADECAPOLE branch), then
 * calculateRadiusBox (:473-482) or radius 1.0 for count <= 1. */
static void mom_clear(pto_mom* q) {
  memset(q, 0, sizeof(*q));
  for (int d = 0; d < 3; d++) {
    q->lo[d] = 1.7976931348623157e308;
    q->hi[d] = -1.7976931348623157e308;
  }
}

static void mom_add_particle(pto_mom* q, double px, double py, double pz, double pm, double ps) {
  double m1 = q->mass;
  q->mass += pm;
  if (q->mass == 0.0) {
    q->soft = 0.5 * (q->soft + ps);
    q->cm[0] = 0.5 * (q->cm[0] + px);
    q->cm[1] = 0.5 * (q->cm[1] + py);
    q->cm[2] = 0.5 * (q->cm[2] + pz);
    return;
  }
  q->soft = (m1 * q->soft + pm * ps) / q->mass;
  double c1[3] = {q->cm[0], q->cm[1], q->cm[2]};
  q->cm[0] = (m1 * q->cm[0] + pm * px) / q->mass;
  q->cm[1] = (m1 * q->cm[1] + pm * py) / q->mass;
  q->cm[2] = (m1 * q->cm[2] + pm * pz) / q->mass;
  double d0 = c1[0] - q->cm[0], d1 = c1[1] - q->cm[1], d2 = c1[2] - q->cm[2];
  q->xx += m1 * d0 * d0;
  q->yy += m1 * d1 * d1;
  q->zz += m1 * d2 * d2;
  q->xy += m1 * d0 * d1;
  q->xz += m1 * d0 * d2;
  q->yz += m1 * d1 * d2;
  d0 = px - q->cm[0];
  d1 = py - q->cm[1];
  d2 = pz - q->cm[2];
  q->xx += pm * d0 * d0;
  q->yy += pm * d1 * d1;
  q->zz += pm * d2 * d2;
  q->xy += pm * d0 * d1;
  q->xz += pm * d0 * d2;
  q->yz += pm * d1 * d2;
}

static void box_grow_pt(double lo[3], double hi[3], const double p[3]) {
  for (int d = 0; d < 3; d++) {
    if (p[d] < lo[d]) lo[d] = p[d];
    if (p[d] > hi[d]) hi[d] = p[d];
  }
}

static void leaf_moments(pto_sim* s, pto_mom* q, int start, int cnt) {
  mom_clear(q);
  for (int i = start; i < start + cnt; i++) {
    mom_add_particle(q, s->x[i], s->y[i], s->z[i], s->m[i], s->soft[i]);
    double p[3] = {s->x[i], s->y[i], s->z[i]};
    box_grow_pt(q->lo, q->hi, p);
  }
  q->count = cnt;
  if (q->count > 1) {
    double dx = q->hi[0] - q->lo[0], dy = q->hi[1] - q->lo[1], dz = q->hi[2] - q->lo[2];
    q->radius = 0.5 * sqrt(dx * dx + dy * dy + dz * dz);
  } else {
    q->radius = 1.0;
  }
}

/* Upward combine: CentroidData::operator+=, examples/CentroidData.h:61-73,
 * with MultipoleMoments::operator+=(MultipoleMoments) (parallel axis),
 * examples/MultipoleMoments.h:204-221 and :253-271, and
 * calculateRadiusFarthestCorner, :458-469. */
static void mom_combine(pto_mom* q, const pto_mom* c) {
  for (int d = 0; d < 3; d++) {
    if (c->lo[d] < q->lo[d]) q->lo[d] = c->lo[d];
    if (c->hi[d] > q->hi[d]) q->hi[d] = c->hi[d];
  }
  double m1 = q->mass;
  q->mass += c->mass;
  if (q->mass == 0.0) {
    q->soft = 0.5 * (q->soft + c->soft);
    for (int d = 0; d < 3; d++) q->cm[d] = 0.5 * (q->cm[d] + c->cm[d]);
  } else if (m1 == 0.0) {
    double lo[3], hi[3];
    int cnt = q->count;
    memcpy(lo, q->lo, sizeof(lo));
    memcpy(hi, q->hi, sizeof(hi));
    *q = *c;
    q->count = cnt;
    memcpy(q->lo, lo, sizeof(lo));
    memcpy(q->hi, hi, sizeof(hi));
  } else if (c->mass != 0.0) {
    q->soft = (m1 * q->soft + c->mass * c->soft) / q->mass;
    double c1[3] = {q->cm[0], q->cm[1], q->cm[2]};
    for (int d = 0; d < 3; d++) q->cm[d] = (m1 * q->cm[d] + c->mass * c->cm[d]) / q->mass;
    double d0 = c1[0] - q->cm[0], d1 = c1[1] - q->cm[1], d2 = c1[2] - q->cm[2];
    q->xx += m1 * d0 * d0;
    q->yy += m1 * d1 * d1;
    q->zz += m1 * d2 * d2;
    q->xy += m1 * d0 * d1;
    q->xz += m1 * d0 * d2;
    q->yz += m1 * d1 * d2;
    d0 = c->cm[0] - q->cm[0];
    d1 = c->cm[1] - q->cm[1];
    d2 = c->cm[2] - q->cm[2];
    q->xx += c->xx + c->mass * d0 * d0;
    q->yy += c->yy + c->mass * d1 * d1;
    q->zz += c->zz + c->mass * d2 * d2;
    q->xy += c->xy + c->mass * d0 * d1;
    q->xz += c->xz + c->mass * d0 * d2;
    q->yz += c->yz + c->mass * d1 * d2;
  }
  q->count += c->count;
  if (q->count > 1) {
    double e[3];
    for (int d = 0; d < 3; d++) {
      double a = q->cm[d] - q->lo[d], b = q->hi[d] - q->cm[d];
      e[d] = (a > b) ? a : b;
    }
    q->radius = sqrt(e[0] * e[0] + e[1] * e[1] + e[2] * e[2]);
  } else {
    q->radius = 1.0;
  }
}

/* ---------------------------------------------------------------- build */
static long new_node(pto_sim* s) {
  if (s->nnodes == s->cap) {
    long nc = s->cap ? 2 * s->cap : 1024;
    s->nkey = (uint64_t*)realloc(s->nkey, sizeof(uint64_t) * nc);
    s->ntype = (int*)realloc(s->ntype, sizeof(int) * nc);
    s->ndepth = (int*)realloc(s->ndepth, sizeof(int) * nc);
    s->npstart = (int*)realloc(s->npstart, sizeof(int) * nc);
    s->nnp = (int*)realloc(s->nnp, sizeof(int) * nc);
    s->nparent = (int*)realloc(s->nparent, sizeof(int) * nc);
    s->nchild = (int*)realloc(s->nchild, sizeof(int) * nc);
    s->nwait = (int*)realloc(s->nwait, sizeof(int) * nc);
    s->mom = (pto_mom*)realloc(s->mom, sizeof(pto_mom) * nc);
    s->cap = nc;
  }
  return s->nnodes++;
}

static void push_int(int** a, long* len, long* cap, int v) {
  if (*len == *cap) {
    *cap = *cap ? 2 * *cap : 1024;
    *a = (int*)realloc(*a, sizeof(int) * (*cap));
  }
  (*a)[(*len)++] = v;
}

/* src/Subtree.h:263-267 (getType), with depth 21 forced to Leaf. */
static int node_type(long n, int bucket, int depth) {
  if (n == 0) return PTO_EMPTY;
  if (n <= bucket || depth >= PTO_MAX_DEPTH) return PTO_LEAF;
  return PTO_INTERNAL;
}

static int key_depth(uint64_t k) {
  int pos = 63 - __builtin_clzll(k);
  return pos / 3;
}

/* Utility::removeLeadingZeros, src/Utility.h:127-130 with :91-93. */
static uint64_t left_align(uint64_t k) { return k << (63 - 3 * key_depth(k)); }

/* first index in [lo, hi) whose key >= v (Utility::binarySearchComp,
 * src/Utility.h:33-50 with OctTree::findChildsLastParticle,
 * src/Modularization.C:60-65). */
static int first_ge(const uint64_t* keys, int lo, int hi, uint64_t v) {
  while (lo < hi) {
    int mid = lo + ((hi - lo) >> 1);
    if (keys[mid] >= v) hi = mid;
    else lo = mid + 1;
  }
  return lo;
}

static void make_node(pto_sim* s, long id, uint64_t key, int type, int depth, int pstart, int np, int parent) {
  s->nkey[id] = key;
  s->ntype[id] = type;
  s->ndepth[id] = depth;
  s->npstart[id] = pstart;
  s->nnp[id] = np;
  s->nparent[id] = parent;
  s->nchild[id] = -1;
  s->nwait[id] = (type == PTO_INTERNAL) ? 8 : 0;
  if (type == PTO_LEAF) {
    leaf_moments(s, &s->mom[id], pstart, np);
    push_int(&s->leaves, &s->nleaves, &s->leafcap, (int)id);
  } else {
    mom_clear(&s->mom[id]);
    s->mom[id].radius = 0.0;
    if (type == PTO_EMPTY) push_int(&s->empties, &s->nempties, &s->emptycap, (int)id);
  }
}

/* src/Subtree.h:314-349 (recursiveBuild); children of a node are allocated
 * as one contiguous group of 8. */
static void recursive_build(pto_sim* s, long node) {
  uint64_t ck = s->nkey[node] << 3;
  int start = s->npstart[node];
  int finish = start + s->nnp[node];
  long first = -1;
  for (int i = 0; i < 8; i++) {
    long c = new_node(s);
    if (i == 0) first = c;
  }
  s->nchild[node] = (int)first;
  int depth = s->ndepth[node] + 1;
  for (int i = 0; i < 8; i++) {
    int fge = finish;
    if (i < 7) fge = first_ge(s->key, start, finish, left_align(ck + 1));
    int cn = fge - start;
    long c = first + i;
    make_node(s, c, ck, node_type(cn, s->bucket, depth), depth, start, cn, (int)node);
    if (s->ntype[c] == PTO_INTERNAL) recursive_build(s, c);
    start = fge;
    ck++;
  }
}

/* src/Subtree.h:352-384 (populateTree): leaves (DFS order), then empty
 * leaves, through a FIFO; a parent joins the queue when its last child is
 * popped, and combines its children in pop order. */
static void populate(pto_sim* s) {
  long total = s->nleaves + s->nempties;
  long qcap = s->nnodes + 1, head = 0, tail = 0;
  int* q = (int*)malloc(sizeof(int) * qcap);
  for (long i = 0; i < s->nleaves; i++) q[tail++] = s->leaves[i];
  for (long i = 0; i < s->nempties; i++) q[tail++] = s->empties[i];
  (void)total;
  while (head < tail) {
    int nd = q[head++];
    if (nd == 0) continue; /* the root */
    int p = s->nparent[nd];
    mom_combine(&s->mom[p], &s->mom[nd]);
    if (--s->nwait[p] == 0) q[tail++] = p;
  }
  free(q);
}

static void build_tree(pto_sim* s) {
  sort_particles(s);
  s->nnodes = 0;
  s->nleaves = s->nempties = 0;
  long root = new_node(s);
  make_node(s, root, 1, node_type(s->n, s->bucket, 0), 0, 0, s->n, -1);
  if (s->ntype[root] == PTO_INTERNAL) recursive_build(s, root);
  populate(s);
}

/* ---------------------------------------------------------------- visitor
 * examples/GravityVisitor.h.  Offsets are zero (no periodic replicas). */
static const double kOpenGeom = 4.0 / 3.0; /* :14 */

/* SPLINE, GravityVisitor.h:87-120 (a: potential term, b: force term) */
static void spline(double r2, double twoh, double* a, double* b) {
  double r = sqrt(r2);
  if (r < twoh) {
    double dih = 2.0 / twoh;
    double u = r * dih;
    if (u < 1.0) {
      *a = dih * (7.0 / 5.0 - 2.0 / 3.0 * u * u + 3.0 / 10.0 * u * u * u * u - 1.0 / 10.0 * u * u * u * u * u);
      *b = dih * dih * dih * (4.0 / 3.0 - 6.0 / 5.0 * u * u + 1.0 / 2.0 * u * u * u);
    } else {
      double dir = 1.0 / r;
      *a = -1.0 / 15.0 * dir +
           dih * (8.0 / 5.0 - 4.0 / 3.0 * u * u + u * u * u - 3.0 / 10.0 * u * u * u * u + 1.0 / 30.0 * u * u * u * u * u);
      *b = -1.0 / 15.0 * dir * dir * dir + dih * dih * dih * (8.0 / 3.0 - 3.0 * u + 6.0 / 5.0 * u * u - 1.0 / 6.0 * u * u * u);
    }
  } else {
    *a = 1.0 / r;
    *b = *a * *a * *a;
  }
}

/* SPLINEQ, GravityVisitor.h:37-80, kept exactly as the reference evaluates
 * it (including its softened-branch grouping). */
static void splineq(double invr, double r2, double twoh, double* a, double* b, double* c, double* d) {
  double dir = invr;
  if (r2 < twoh * twoh) {
    double dih = 2.0 / twoh;
    double u = dih / dir;
    if (u < 1.0) {
      *a = dih * (7.0) / 5.0 - 2.0 / 3.0 * u * u + 3.0 / 10.0 * u * u * u * u - 1.0 / 10.0 * u * u * u * u * u;
      *b = dih * dih * dih * (4.0) / 3.0 - 6.0 / 5.0 * u * u + 1.0 / 2.0 * u * u * u;
      *c = dih * dih * dih * dih * dih * (12.0) / 5.0 - 3.0 / 2.0 * u;
      *d = 3.0 / 2.0 * dih * dih * dih * dih * dih * dih * dir;
    } else {
      *a = -1.0 / 15.0 * dir + dih * (8.0 / 5.0) - 4.0 / 3.0 * u * u + u * u * u - 3.0 / 10.0 * u * u * u * u +
           1.0 / 30.0 * u * u * u * u * u;
      *b = -1.0 / 15.0 * dir * dir * dir + dih * dih * dih * (8.0) / 3.0 - 3.0 * u + 6.0 / 5.0 * u * u -
           1.0 / 6.0 * u * u * u;
      *c = -1.0 / 5.0 * dir * dir * dir * dir * dir + 3.0 * dih * dih * dih * dih * dir +
           dih * dih * dih * dih * dih * (-12.0) / 5.0 + 1.0 / 2.0 * u;
      *d = -dir * dir * dir * dir * dir * dir * dir + 3.0 * dih * dih * dih * dih * dir * dir * dir -
           1.0 / 2.0 * dih * dih * dih * dih * dih * dih * dir;
    }
  } else {
    *a = dir;
    *b = *a * *a * *a;
    *c = 3.0 * *b * *a * *a;
    *d = 5.0 * *c * *a * *a;
  }
}

/* box/sphere test of the stand-in Space::intersect (x, y, z order; <=). */
static int box_sphere(const double lo[3], const double hi[3], const double c[3], double rsq) {
  double dsq = 0.0, d;
  for (int k = 0; k < 3; k++) {
    if ((d = lo[k] - c[k]) > 0) dsq += d * d;
    else if ((d = c[k] - hi[k]) > 0) dsq += d * d;
  }
  return dsq <= rsq;
}

/* GravityVisitor::open, :162-182 (non-HEXADECAPOLE :180). */
static int visit_open(const pto_mom* src, const pto_mom* tgt, double gfac, const double off[3]) {
  if (src->count <= 6) return 1;
  double rsq = src->radius * src->radius * gfac;
  double c[3] = {src->cm[0] + off[0], src->cm[1] + off[1], src->cm[2] + off[2]};
  return box_sphere(tgt->lo, tgt->hi, c, rsq);
}

/* GravityVisitor::openSoftening, :122-128. */
static int open_softening(const pto_mom* src, const pto_mom* tgt, const double off[3]) {
  double r1 = 2.0 * src->soft, r2 = 2.0 * tgt->soft;
  double c[3] = {src->cm[0] + off[0], src->cm[1] + off[1], src->cm[2] + off[2]};
  double dx = c[0] - tgt->cm[0], dy = c[1] - tgt->cm[1], dz = c[2] - tgt->cm[2];
  double rs = r1 + r2;
  if (dx * dx + dy * dy + dz * dz <= rs * rs) return 1;
  return box_sphere(tgt->lo, tgt->hi, c, r1 * r1);
}

/* GravityVisitor::leaf, :144-160 -- P2P; the per-source-leaf sum is formed
 * first and then added (applyAcceleration).  pot_full additionally sums
 * -m_j * a (the reference's leaf() does not touch the potential). */
static void visit_leaf(pto_sim* s, int src, int tgt, const double off[3]) {
  int s0 = s->npstart[src], sn = s->nnp[src];
  int t0 = s->npstart[tgt], tn = s->nnp[tgt];
  for (int i = t0; i < t0 + tn; i++) {
    double ax = 0.0, ay = 0.0, az = 0.0, pf = 0.0;
    for (int j = s0; j < s0 + sn; j++) {
      double dx = (s->x[j] + off[0]) - s->x[i];
      double dy = (s->y[j] + off[1]) - s->y[i];
      double dz = (s->z[j] + off[2]) - s->z[i];
      double rsq = dx * dx + dy * dy + dz * dz;
      double twoh = s->soft[j] + s->soft[i];
      if (rsq != 0) {
        double a, b;
        spline(rsq, twoh, &a, &b);
        double bm = b * s->m[j];
        ax += dx * bm;
        ay += dy * bm;
        az += dz * bm;
        pf += -s->m[j] * a;
      }
    }
    s->ax[i] += ax;
    s->ay[i] += ay;
    s->az[i] += az;
    s->potf[i] += pf;
  }
}

/* GravityVisitor::node, :184-224 (non-HEXADECAPOLE :207-221), with the
 * unsoftened monopole fallback addGravity, :130-139.  Returns 1 when the
 * monopole fallback was taken. */
static int visit_node(pto_sim* s, int src, int tgt, const double off[3]) {
  const pto_mom* q = &s->mom[src];
  const pto_mom* t = &s->mom[tgt];
  if (q->count == 0) return 0;
  int t0 = s->npstart[tgt], tn = s->nnp[tgt];
  if (open_softening(q, t, off)) {
    for (int i = t0; i < t0 + tn; i++) {
      double dx = (q->cm[0] + off[0]) - s->x[i];
      double dy = (q->cm[1] + off[1]) - s->y[i];
      double dz = (q->cm[2] + off[2]) - s->z[i];
      double rsq = dx * dx + dy * dy + dz * dz;
      if (rsq != 0) {
        double f = q->mass / (rsq * sqrt(rsq));
        s->ax[i] += dx * f;
        s->ay[i] += dy * f;
        s->az[i] += dz * f;
        s->potf[i] += -q->mass / sqrt(rsq);
      }
    }
    return 1;
  }
  for (int i = t0; i < t0 + tn; i++) {
    double rx = (s->x[i] - q->cm[0]) - off[0];
    double ry = (s->y[i] - q->cm[1]) - off[1];
    double rz = (s->z[i] - q->cm[2]) - off[2];
    double rsq = rx * rx + ry * ry + rz * rz;
    double dir = 1.0 / sqrt(rsq);
    double twoh = q->soft + s->soft[i];
    double a, b, c, d;
    splineq(dir, rsq, twoh, &a, &b, &c, &d);
    double qx = q->xx * rx + q->xy * ry + q->xz * rz;
    double qy = q->xy * rx + q->yy * ry + q->yz * rz;
    double qz = q->xz * rx + q->yz * ry + q->zz * rz;
    double qir = 0.5 * (qx * rx + qy * ry + qz * rz);
    double tr = 0.5 * (q->xx + q->yy + q->zz);
    double qir3 = b * q->mass + d * qir - c * tr;
    double p = -q->mass * a - c * qir + b * tr;
    s->pot[i] += p;
    s->potf[i] += p;
    s->ax[i] += -qir3 * rx + c * qx;
    s->ay[i] += -qir3 * ry + c * qy;
    s->az[i] += -qir3 * rz + c * qz;
  }
}

/* EwaldData::EwaldInit (examples/Ewald.C:80-163) and LeafEwaldFn
 * (examples/Ewald.h:3-199), non-HEXADECAPOLE branch, restated: the root
 * cell's monopole + quadrupole summed over real-space images (erfc; -erf for
 * images inside the replica hole, which the tree walked) and over the
 * reciprocal table; alpha = 2/L. */
typedef struct { double h[3], c; } pto_ewt;

static void ewald_correction(pto_sim* s) {
  const pto_mom* R = &s->mom[0];
  const double L = s->period;
  const int hReps = (int)ceil(s->ewald_hcut);
  const double alpha = 2.0 / L, alpha2 = alpha * alpha;
  const double k4 = M_PI * M_PI / (alpha * alpha * L * L);
  int cap = (2 * hReps + 1) * (2 * hReps + 1) * (2 * hReps + 1), nh = 0;
  pto_ewt* ewt = (pto_ewt*)malloc(sizeof(pto_ewt) * (size_t)cap);
  for (int hx = -hReps; hx <= hReps; ++hx)
    for (int hy = -hReps; hy <= hReps; ++hy)
      for (int hz = -hReps; hz <= hReps; ++hz) {
        int h2 = hx * hx + hy * hy + hz * hz;
        if (h2 == 0 || h2 > s->ewald_hcut * s->ewald_hcut) continue;
        double g0 = exp(-k4 * h2) / (M_PI * h2 * L);
        double g1 = 2 * M_PI / L * g0;
        double g2 = -2 * M_PI / L * g1;
        double qx = (1.0 / 1.0) * (R->xz * hz + R->xy * hy + R->xx * hx);
        double qy = (1.0 / 1.0) * (R->yz * hz + R->xy * hx + R->yy * hy);
        double qz = (1.0 / 1.0) * (R->yz * hy + R->xz * hx + R->zz * hz);
        double qm = (1.0 / 2.0) * (qx * hx + qy * hy + qz * hz);
        double c = 0.0;
        c -= g2 * qm;
        c -= g0 * R->mass;
        ewt[nh].h[0] = 2 * M_PI / L * hx;
        ewt[nh].h[1] = 2 * M_PI / L * hy;
        ewt[nh].h[2] = 2 * M_PI / L * hz;
        ewt[nh].c = c;
        nh++;
      }
  const double Q2 = 0.5 * (R->xx + R->yy + R->zz);
  int nEw = (int)ceil(s->ewald_rcut);
  if (s->n_replicas > nEw) nEw = s->n_replicas;
  const double cut2 = s->ewald_rcut * s->ewald_rcut * L * L, inner2 = 1.2e-3 * L * L;
  const double k1 = M_PI / (alpha2 * L * L * L), ka = 2.0 * alpha / sqrt(M_PI);
  const int nr = s->n_replicas;
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(s->threads)
#endif
  for (int i = 0; i < s->n; i++) {
    double pot = R->mass * k1, ax = 0.0, ay = 0.0, az = 0.0;
    double dx = s->x[i] - R->cm[0], dy = s->y[i] - R->cm[1], dz = s->z[i] - R->cm[2];
    for (int ix = -nEw; ix <= nEw; ++ix)
      for (int iy = -nEw; iy <= nEw; ++iy)
        for (int iz = -nEw; iz <= nEw; ++iz) {
          int hole = ix >= -nr && ix <= nr && iy >= -nr && iy <= nr && iz >= -nr && iz <= nr;
          double x = dx + ix * L, y = dy + iy * L, z = dz + iz * L;
          double r2 = x * x + y * y + z * z, g0, g1, g2, g3;
          if (r2 > cut2 && !hole) continue;
          if (r2 < inner2) {
            double an = ka;
            r2 *= alpha2;
            g0 = an * ((1.0 / 3.0) * r2 - 1.0);
            an *= 2 * alpha2;
            g1 = an * ((1.0 / 5.0) * r2 - (1.0 / 3.0));
            an *= 2 * alpha2;
            g2 = an * ((1.0 / 7.0) * r2 - (1.0 / 5.0));
            an *= 2 * alpha2;
            g3 = an * ((1.0 / 9.0) * r2 - (1.0 / 7.0));
          } else {
            double dir = 1 / sqrt(r2), dir2 = dir * dir;
            double a = exp(-r2 * alpha2);
            a *= ka * dir2;
            g0 = hole ? -erf(alpha / dir) : erfc(alpha / dir);
            g0 *= dir;
            g1 = g0 * dir2 + a;
            double an = 2 * alpha2;
            g2 = 3 * g1 * dir2 + an * a;
            an *= 2 * alpha2;
            g3 = 5 * g2 * dir2 + an * a;
          }
          double mx = R->xx * x + R->xy * y + R->xz * z;
          double my = R->xy * x + R->yy * y + R->yz * z;
          double mz = R->xz * x + R->yz * y + R->zz * z;
          double mir = 0.5 * (mx * x + my * y + mz * z);
          double qta = g1 * R->mass - g2 * Q2 + g3 * mir;
          pot -= g0 * R->mass - g1 * Q2 + g2 * mir;
          ax += g2 * (mx) - x * qta;
          ay += g2 * (my) - y * qta;
          az += g2 * (mz) - z * qta;
        }
    for (int h = 0; h < nh; ++h) {
      double hx = ewt[h].h[0] * dx + ewt[h].h[1] * dy + ewt[h].h[2] * dz;
      double c = cos(hx), sn = sin(hx);
      pot += ewt[h].c * c;
      ax += ewt[h].h[0] * (ewt[h].c * sn);
      ay += ewt[h].h[1] * (ewt[h].c * sn);
      az += ewt[h].h[2] * (ewt[h].c * sn);
    }
    s->pot[i] += pot;
    s->potf[i] += pot;
    s->ax[i] += ax;
    s->ay[i] += ay;
    s->az[i] += az;
  }
  free(ewt);
}

static void list_push(pto_sim* s, uint64_t key, int kind) {
  if (s->list_total == s->list_cap) {
    s->list_cap = s->list_cap ? 2 * s->list_cap : 4096;
    s->list_key = (uint64_t*)realloc(s->list_key, sizeof(uint64_t) * s->list_cap);
    s->list_kind = (int*)realloc(s->list_kind, sizeof(int) * s->list_cap);
  }
  s->list_key[s->list_total] = key;
  s->list_kind[s->list_total] = kind;
  s->list_total++;
}

/* src/Traverser.h:154-217 for one bucket: pre-order DFS; Leaf -> leaf()
 * (self included, CallSelfLeaf), Internal -> open() ? children : node(),
 * EmptyLeaf -> nothing. */
static void walk(pto_sim* s, int tgt, double gfac, int record, unsigned long long* cnt, const double off[3]) {
  int stack[8 * (PTO_MAX_DEPTH + 2)];
  int sp = 0;
  stack[sp++] = 0;
  while (sp) {
    int nd = stack[--sp];
    int ty = s->ntype[nd];
    if (ty == PTO_LEAF) {
      visit_leaf(s, nd, tgt, off);
      cnt[0] += (unsigned long long)s->nnp[nd] * (unsigned long long)s->nnp[tgt];
      if (record) list_push(s, s->nkey[nd], 0);
    } else if (ty == PTO_INTERNAL) {
      cnt[2]++;
      if (visit_open(&s->mom[nd], &s->mom[tgt], gfac, off)) {
        int c0 = s->nchild[nd];
        for (int c = 7; c >= 0; c--) stack[sp++] = c0 + c;
      } else {
        cnt[3] += (unsigned long long)visit_node(s, nd, tgt, off);
        cnt[1] += (unsigned long long)s->nnp[tgt];
        if (record) list_push(s, s->nkey[nd], 1);
      }
    }
  }
}

/* BasicDownTraverser::doTrav (src/Traverser.h:296-330): a deque used first in,
 * first out -- children pushed at the front in index order, nodes taken from
 * the back -- so one bucket's nodes are visited breadth first. */
static void walk_bfs(pto_sim* s, int tgt, double gfac, int record, unsigned long long* cnt, const double off[3],
                     int* queue) {
  long head = 0, tail = 0;
  queue[tail++] = 0;
  while (head < tail) {
    int nd = queue[head++];
    int ty = s->ntype[nd];
    if (ty == PTO_LEAF) {
      visit_leaf(s, nd, tgt, off);
      cnt[0] += (unsigned long long)s->nnp[nd] * (unsigned long long)s->nnp[tgt];
      if (record) list_push(s, s->nkey[nd], 0);
    } else if (ty == PTO_INTERNAL) {
      cnt[2]++;
      if (visit_open(&s->mom[nd], &s->mom[tgt], gfac, off)) {
        int c0 = s->nchild[nd];
        for (int c = 0; c < 8; c++) queue[tail++] = c0 + c;
      } else {
        cnt[3] += (unsigned long long)visit_node(s, nd, tgt, off);
        cnt[1] += (unsigned long long)s->nnp[tgt];
        if (record) list_push(s, s->nkey[nd], 1);
      }
    }
  }
}

static void walk_any(pto_sim* s, int tgt, double gfac, int record, unsigned long long* cnt, const double off[3]) {
  if (!s->basic_down) {
    walk(s, tgt, gfac, record, cnt, off);
    return;
  }
  int* queue = (int*)malloc(sizeof(int) * (size_t)(s->nnodes + 1));
  walk_bfs(s, tgt, gfac, record, cnt, off, queue);
  free(queue);
}

void pto_set_traversal(pto_sim* s, int basic_down) { s->basic_down = basic_down; }

static void traverse(pto_sim* s, int record) {
  double gfac = kOpenGeom / (s->theta * s->theta);
  memset(s->ax, 0, sizeof(double) * s->n);
  memset(s->ay, 0, sizeof(double) * s->n);
  memset(s->az, 0, sizeof(double) * s->n);
  memset(s->pot, 0, sizeof(double) * s->n);
  memset(s->potf, 0, sizeof(double) * s->n);
  unsigned long long pp = 0, pc = 0, op = 0, mo = 0;
  const double zero[3] = {0.0, 0.0, 0.0};
  if (record) {
    free(s->list_off);
    s->list_off = (long*)malloc(sizeof(long) * (s->nleaves + 1));
    s->list_total = 0;
    for (long b = 0; b < s->nleaves; b++) {
      unsigned long long c[4] = {0, 0, 0, 0};
      s->list_off[b] = s->list_total;
      walk_any(s, s->leaves[b], gfac, 1, c, zero);
      pp += c[0]; pc += c[1]; op += c[2]; mo += c[3];
    }
    s->list_off[s->nleaves] = s->list_total;
  } else {
    /* examples/Gravity.C:32-46: one walk, or (2n+1)^3 replica walks */
    const int nr = s->periodic ? s->n_replicas : 0;
    for (int X = -nr; X <= nr; X++)
      for (int Y = -nr; Y <= nr; Y++)
        for (int Z = -nr; Z <= nr; Z++) {
          const double off[3] = {X * s->period, Y * s->period, Z * s->period};
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : pp, pc, op, mo) num_threads(s->threads)
#endif
          for (long b = 0; b < s->nleaves; b++) {
            unsigned long long c[4] = {0, 0, 0, 0};
            walk_any(s, s->leaves[b], gfac, 0, c, s->periodic ? off : zero);
            pp += c[0]; pc += c[1]; op += c[2]; mo += c[3];
          }
        }
    if (s->periodic) ewald_correction(s);
  }
  s->n_pp = pp;
  s->n_pc = pc;
  s->n_open = op;
  s->n_mono = mo;
}

/* ---------------------------------------------------------------- API */
static double* dup_d(const double* a, int n) {
  double* p = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  if (n > 0) memcpy(p, a, sizeof(double) * (size_t)n);
  return p;
}

void pto_set_periodic(pto_sim* s, int periodic, double L, int n_replicas, double rcut, double hcut) {
  s->periodic = periodic;
  s->period = L;
  s->n_replicas = n_replicas;
  s->ewald_rcut = rcut;
  s->ewald_hcut = hcut;
}

pto_sim* pto_create(int n, const double* x, const double* y, const double* z, const double* vx,
                    const double* vy, const double* vz, const double* m, const double* soft, int bucket,
                    double theta, double dt_max, int threads) {
  pto_sim* s = (pto_sim*)calloc(1, sizeof(pto_sim));
  s->n = n;
  s->bucket = bucket;
  s->theta = theta;
  s->dt_max = dt_max;
  s->threads = threads > 0 ? threads : 1;
  s->x = dup_d(x, n); s->y = dup_d(y, n); s->z = dup_d(z, n);
  s->vx = dup_d(vx, n); s->vy = dup_d(vy, n); s->vz = dup_d(vz, n);
  s->m = dup_d(m, n); s->soft = dup_d(soft, n);
  s->ax = (double*)calloc((size_t)n + 1, sizeof(double));
  s->ay = (double*)calloc((size_t)n + 1, sizeof(double));
  s->az = (double*)calloc((size_t)n + 1, sizeof(double));
  s->pot = (double*)calloc((size_t)n + 1, sizeof(double));
  s->potf = (double*)calloc((size_t)n + 1, sizeof(double));
  s->order = (int*)malloc(sizeof(int) * ((size_t)n + 1));
  s->key = (uint64_t*)malloc(sizeof(uint64_t) * ((size_t)n + 1));
  for (int i = 0; i < n; i++) s->order[i] = i;
  double lo[3], hi[3];
  particle_bbox(s, lo, hi);
  remake_universe(s, lo, hi);
  assign_keys(s);
  return s;
}

void pto_destroy(pto_sim* s) {
  if (!s) return;
  free(s->x); free(s->y); free(s->z); free(s->vx); free(s->vy); free(s->vz); free(s->m); free(s->soft);
  free(s->ax); free(s->ay); free(s->az); free(s->pot); free(s->potf); free(s->order); free(s->key);
  free(s->nkey); free(s->ntype); free(s->ndepth); free(s->npstart); free(s->nnp); free(s->nparent);
  free(s->nchild); free(s->nwait); free(s->mom); free(s->leaves); free(s->empties);
  free(s->list_off); free(s->list_key); free(s->list_kind);
  free(s);
}

int pto_forces(pto_sim* s, int record_lists) {
  double t0 = wall();
  build_tree(s);
  double t1 = wall();
  traverse(s, record_lists);
  double t2 = wall();
  s->t_build = t1 - t0;
  s->t_trav = t2 - t1;
  return 0;
}

/* examples/Gravity.C:63-67 with v_max from src/Subtree.h:164-170. */
static double timestep(const pto_sim* s) {
  double v2 = 0.0;
  for (int i = 0; i < s->n; i++) {
    double w = s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i];
    if (w > v2) v2 = w;
  }
  double vmax = sqrt(v2);
  double len = s->uhi[0] - s->ulo[0];
  double t = len / vmax / cbrt((double)s->n);
  return t < s->dt_max ? t : s->dt_max;
}

/* src/Driver.h:183-251 iteration: forces, Particle::kick (src/Particle.C:7-9)
 * for all particles, then Particle::perturb (:11-21) with the new bbox,
 * remakeUniverse and rekey (src/Partition.h:382-387). */
int pto_run(pto_sim* s, int nsteps) {
  if (nsteps <= 0) return pto_forces(s, 0);
  for (int it = 0; it < nsteps; it++) {
    pto_forces(s, 0);
    double dt = timestep(s);
    s->last_dt = dt;
    for (int i = 0; i < s->n; i++) {
      s->vx[i] += s->ax[i] * dt / 2;
      s->vy[i] += s->ay[i] * dt / 2;
      s->vz[i] += s->az[i] * dt / 2;
    }
    for (int i = 0; i < s->n; i++) {
      s->vx[i] += (s->ax[i] * dt / 2);
      s->vy[i] += (s->ay[i] * dt / 2);
      s->vz[i] += (s->az[i] * dt / 2);
      s->x[i] += (s->vx[i] * dt);
      s->y[i] += (s->vy[i] * dt);
      s->z[i] += (s->vz[i] * dt);
    }
    double lo[3], hi[3];
    particle_bbox(s, lo, hi);
    remake_universe(s, lo, hi);
    assign_keys(s);
  }
  return 0;
}

void pto_get_acc(const pto_sim* s, double* ax, double* ay, double* az, double* pot, double* pot_full) {
  for (int i = 0; i < s->n; i++) {
    int o = s->order[i];
    if (ax) ax[o] = s->ax[i];
    if (ay) ay[o] = s->ay[i];
    if (az) az[o] = s->az[i];
    if (pot) pot[o] = s->pot[i];
    if (pot_full) pot_full[o] = s->potf[i];
  }
}

void pto_get_keys(const pto_sim* s, uint64_t* keys) {
  for (int i = 0; i < s->n; i++) keys[s->order[i]] = s->key[i];
}

void pto_get_state(const pto_sim* s, double* x, double* y, double* z, double* vx, double* vy, double* vz) {
  for (int i = 0; i < s->n; i++) {
    int o = s->order[i];
    x[o] = s->x[i]; y[o] = s->y[i]; z[o] = s->z[i];
    vx[o] = s->vx[i]; vy[o] = s->vy[i]; vz[o] = s->vz[i];
  }
}

void pto_get_universe(const pto_sim* s, double* lo3, double* hi3) {
  for (int d = 0; d < 3; d++) { lo3[d] = s->ulo[d]; hi3[d] = s->uhi[d]; }
}

void pto_get_counters(const pto_sim* s, unsigned long long* out4, double* times2, double* last_dt) {
  out4[0] = s->n_pp; out4[1] = s->n_pc; out4[2] = s->n_open; out4[3] = (unsigned long long)s->nleaves;
  times2[0] = s->t_build; times2[1] = s->t_trav;
  *last_dt = s->last_dt;
}

long pto_num_nodes(const pto_sim* s) { return s->nnodes; }

unsigned long long pto_get_mono(const pto_sim* s) { return s->n_mono; }

void pto_get_nodes(const pto_sim* s, uint64_t* keys, int* ints4, double* d18) {
  for (long i = 0; i < s->nnodes; i++) {
    const pto_mom* q = &s->mom[i];
    keys[i] = s->nkey[i];
    ints4[4 * i + 0] = s->ntype[i];
    ints4[4 * i + 1] = s->ndepth[i];
    ints4[4 * i + 2] = q->count;
    ints4[4 * i + 3] = s->ntype[i] == PTO_INTERNAL ? 8 : 0;
    double* d = d18 + 18 * i;
    d[0] = q->mass; d[1] = q->cm[0]; d[2] = q->cm[1]; d[3] = q->cm[2]; d[4] = q->soft; d[5] = q->radius;
    d[6] = q->xx; d[7] = q->xy; d[8] = q->xz; d[9] = q->yy; d[10] = q->yz; d[11] = q->zz;
    d[12] = q->lo[0]; d[13] = q->lo[1]; d[14] = q->lo[2];
    d[15] = q->hi[0]; d[16] = q->hi[1]; d[17] = q->hi[2];
  }
}

long pto_num_buckets(const pto_sim* s) { return s->nleaves; }

void pto_get_bucket_keys(const pto_sim* s, uint64_t* keys) {
  for (long b = 0; b < s->nleaves; b++) keys[b] = s->nkey[s->leaves[b]];
}

long pto_list_total(const pto_sim* s) { return s->list_off ? s->list_total : 0; }

void pto_get_lists(const pto_sim* s, long* offsets, uint64_t* keys, int* kinds) {
  if (!s->list_off) return;
  for (long b = 0; b <= s->nleaves; b++) offsets[b] = s->list_off[b];
  memcpy(keys, s->list_key, sizeof(uint64_t) * s->list_total);
  memcpy(kinds, s->list_kind, sizeof(int) * s->list_total);
}

/* FP64 isolated direct sum with the reference's spline kernel. */
void pto_direct(int n, const double* x, const double* y, const double* z, const double* m,
                const double* soft, int nt, const int* targets, double* ax, double* ay, double* az,
                double* pot, int threads) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads > 0 ? threads : 1)
#endif
  for (int t = 0; t < nt; t++) {
    int i = targets[t];
    double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
    for (int j = 0; j < n; j++) {
      double dx = x[j] - x[i], dy = y[j] - y[i], dz = z[j] - z[i];
      double rsq = dx * dx + dy * dy + dz * dz;
      if (rsq != 0) {
        double a, b;
        spline(rsq, soft[j] + soft[i], &a, &b);
        double bm = b * m[j];
        sx += dx * bm;
        sy += dy * bm;
        sz += dz * bm;
        sp += -m[j] * a;
      }
    }
    ax[t] = sx; ay[t] = sy; az[t] = sz; pot[t] = sp;
  }
  (void)threads;
}

/* FP64 periodic (Ewald) direct sum with the spline kernel for the nearest
 * image within soft_i + soft_j: alpha = 4/L, real-space images within 1.5 L,
 * reciprocal |h|^2 <= 64, background and self terms in the potential. */
void pto_ewald_direct(int n, const double* x, const double* y, const double* z, const double* m,
                      const double* soft, double L, int nt, const int* targets, double* ax, double* ay,
                      double* az, double* pot, int threads) {
  const double V = L * L * L, alpha = 4.0 / L, rc = 1.5 * L, rc2 = rc * rc;
  const double ka = 2.0 * alpha / sqrt(M_PI);
  const int hmax = 8, nimg = 2;
  int cap = (2 * hmax + 1) * (2 * hmax + 1) * (2 * hmax + 1), nk = 0;
  double* kv = (double*)malloc(sizeof(double) * 4 * (size_t)cap);
  for (int hx = -hmax; hx <= hmax; hx++)
    for (int hy = -hmax; hy <= hmax; hy++)
      for (int hz = -hmax; hz <= hmax; hz++) {
        int h2 = hx * hx + hy * hy + hz * hz;
        if (h2 == 0 || h2 > hmax * hmax) continue;
        double kx = 2 * M_PI / L * hx, ky = 2 * M_PI / L * hy, kz = 2 * M_PI / L * hz;
        double k2 = kx * kx + ky * ky + kz * kz;
        kv[4 * nk] = kx; kv[4 * nk + 1] = ky; kv[4 * nk + 2] = kz;
        kv[4 * nk + 3] = 4 * M_PI / V * exp(-k2 / (4 * alpha * alpha)) / k2;
        nk++;
      }
  double* S = (double*)calloc(2 * (size_t)nk, sizeof(double));
  double M = 0.0;
  for (int j = 0; j < n; j++) M += m[j];
#ifdef _OPENMP
#pragma omp parallel for schedule(static) num_threads(threads > 0 ? threads : 1)
#endif
  for (int k = 0; k < nk; k++) {
    double sc = 0.0, ss = 0.0;
    for (int j = 0; j < n; j++) {
      double ph = kv[4 * k] * x[j] + kv[4 * k + 1] * y[j] + kv[4 * k + 2] * z[j];
      sc += m[j] * cos(ph);
      ss += m[j] * sin(ph);
    }
    S[2 * k] = sc;
    S[2 * k + 1] = ss;
  }
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 4) num_threads(threads > 0 ? threads : 1)
#endif
  for (int t = 0; t < nt; t++) {
    int i = targets[t];
    double sx = 0.0, sy = 0.0, sz = 0.0, sp = 0.0;
    for (int j = 0; j < n; j++) {
      double d0x = x[j] - x[i], d0y = y[j] - y[i], d0z = z[j] - z[i];
      d0x -= L * rint(d0x / L);
      d0y -= L * rint(d0y / L);
      d0z -= L * rint(d0z / L);
      for (int a = -nimg; a <= nimg; a++)
        for (int b = -nimg; b <= nimg; b++)
          for (int c = -nimg; c <= nimg; c++) {
            double dx = d0x + a * L, dy = d0y + b * L, dz = d0z + c * L;
            double r2 = dx * dx + dy * dy + dz * dz;
            if (r2 > rc2 || r2 == 0.0) continue;
            double r = sqrt(r2), ec = erfc(alpha * r);
            double f = (ec + ka * r * exp(-alpha * alpha * r2)) / (r2 * r);
            sx += m[j] * f * dx;
            sy += m[j] * f * dy;
            sz += m[j] * f * dz;
            sp -= m[j] * ec / r;
          }
      double r2 = d0x * d0x + d0y * d0y + d0z * d0z, twoh = soft[j] + soft[i];
      if (r2 != 0.0 && r2 < twoh * twoh) {
        double a, b, r = sqrt(r2);
        spline(r2, twoh, &a, &b);
        double corr = b - 1.0 / (r2 * r);
        sx += m[j] * corr * d0x;
        sy += m[j] * corr * d0y;
        sz += m[j] * corr * d0z;
        sp -= m[j] * (a - 1.0 / r);
      }
    }
    sp += M_PI * M / (alpha * alpha * V) + ka * m[i];
    for (int k = 0; k < nk; k++) {
      double ph = kv[4 * k] * x[i] + kv[4 * k + 1] * y[i] + kv[4 * k + 2] * z[i];
      double sn = sin(ph), cs = cos(ph), w = kv[4 * k + 3];
      double f = w * (sn * S[2 * k] - cs * S[2 * k + 1]);
      sx -= f * kv[4 * k];
      sy -= f * kv[4 * k + 1];
      sz -= f * kv[4 * k + 2];
      sp -= w * (cs * S[2 * k] + sn * S[2 * k + 1]);
    }
    ax[t] = sx; ay[t] = sy; az[t] = sz; pot[t] = sp;
  }
  free(kv);
  free(S);
}

/* SPH density of the reference's SPH example (examples/SPH.C:11-37 DensityFn,
 * examples/DensityVisitor.h leaf(), kernelM4 examples/SPHUtils.h:20-26): the
 * k nearest neighbours of every particle, itself included, found here by
 * brute force; rsq = the k-th distance^2; density = sum_j kernelM4(d2_j * 4 /
 * rsq) m_j / (pi/8 rsq^1.5).  d2 = dx*dx + dy*dy + dz*dz with dx = x_i - x_j,
 * as Vector3D::lengthSquared.  Neighbours (caller order) sorted by (d2, index);
 * the density is summed in that order. */
static double kernel_m4(double ar2) {
  double ak = 2.0 - sqrt(ar2);
  if (ar2 < 1.0) ak = (1.0 - 0.75 * ak * ar2);
  else ak = 0.25 * ak * ak * ak;
  return ak;
}

void pto_sph_density(int n, const double* x, const double* y, const double* z, const double* m, int k,
                     int threads, double* density, double* ballsq, int* nbr, double* nd2) {
#ifdef _OPENMP
#pragma omp parallel for schedule(dynamic, 16) num_threads(threads > 0 ? threads : 1)
#endif
  for (int i = 0; i < n; i++) {
    double bd[64];
    int bi[64];
    int cnt = 0;
    const int kk = k < 64 ? k : 64;
    for (int j = 0; j < n; j++) {
      double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
      double d2 = dx * dx + dy * dy + dz * dz;
      if (cnt == kk && !(d2 < bd[kk - 1] || (d2 == bd[kk - 1] && j < bi[kk - 1]))) continue;
      int p = cnt < kk ? cnt++ : kk - 1;
      while (p > 0 && (bd[p - 1] > d2 || (bd[p - 1] == d2 && bi[p - 1] > j))) {
        bd[p] = bd[p - 1];
        bi[p] = bi[p - 1];
        p--;
      }
      bd[p] = d2;
      bi[p] = j;
    }
    const double rsq = bd[cnt - 1], fBall = sqrt(rsq), ih2 = 4.0 / rsq;
    double dens = 0.0;
    for (int q = 0; q < cnt; q++) dens += kernel_m4(bd[q] * ih2) * m[bi[q]];
    dens /= (0.125 * M_PI * (rsq * fBall));
    density[i] = dens;
    ballsq[i] = rsq;
    for (int q = 0; q < k; q++) {
      nbr[(size_t)i * k + q] = q < cnt ? bi[q] : -1;
      nd2[(size_t)i * k + q] = q < cnt ? bd[q] : -1.0;
    }
  }
}

/* dkernelM4 (examples/SPHUtils.h:40-49): scaled gradient of the M4 kernel. */
static double dkernel_m4(double ar2) {
  double adk = sqrt(ar2);
  if (ar2 < 1.0) adk = -3 + 2.25 * adk;
  else adk = -0.75 * (2.0 - adk) * (2.0 - adk) / adk;
  return adk;
}

/* The SPH example's pressure pass after pto_sph_density (examples/SPH.C:39-64
 * ForceFn and :87-101; doSPHCalc examples/SPHUtils.h:64-133 with visc = 0,
 * aFac = vFac = 1, H = 0, gammam1 = 2/3): every neighbour within the ball
 * (the k nearest; nbr from pto_sph_density, in that order), the divv
 * corrector, then per neighbour the particle's pressure acceleration and PdV
 * work and the opposite reaction on the neighbour, added after the pass.
 * v*: velocities (= velocity_predicted), u: internal energy (= u_predicted). */
void pto_sph_pressure(int n, const double* x, const double* y, const double* z, const double* vx,
                      const double* vy, const double* vz, const double* m, const double* u, const double* density,
                      const double* ballsq, const int* nbr, const double* nd2, int k, double* ax, double* ay,
                      double* az, double* pdv) {
  const double gammam1 = 5.0 / 3.0 - 1.;
  double* oa = (double*)calloc(4 * (size_t)n, sizeof(double));
  for (int i = 0; i < n; i++) {
    const double rsq = ballsq[i], fBall = sqrt(rsq), ih2 = 4.0 / rsq;
    double divvi = 0, divvj = 0;
    for (int e = 0; e < k; e++) {
      const int q = nbr[(size_t)i * k + e];
      if (q < 0) break;
      const double fDist2 = nd2[(size_t)i * k + e];
      double rs1 = dkernel_m4(fDist2 * ih2);
      rs1 *= fDist2 * m[q];
      divvi += rs1;
      divvj += rs1 / density[q];
    }
    divvi /= density[i];
    const double corr = (divvj != 0.0 ? divvi / divvj : 1.0);
    double sax = 0.0, say = 0.0, saz = 0.0, spdv = 0.0;
    for (int e = 0; e < k; e++) {
      const int q = nbr[(size_t)i * k + e];
      if (q < 0) break;
      const double ph = 0.5 * fBall, ih2b = 4. / (fBall * fBall);
      const double fNorm1 = 0.5 * M_1_PI * ih2b * ih2b / ph;
      const double dx = x[q] - x[i], dy = y[q] - y[i], dz = z[q] - z[i];
      const double fDist2 = dx * dx + dy * dy + dz * dz;
      double rs1 = dkernel_m4(fDist2 * ih2b);
      rs1 *= fNorm1;
      rs1 *= corr;
      const double aR = rs1 * m[i], bR = rs1 * m[q];
      const double dvx = vx[q] - vx[i], dvy = vy[q] - vy[i], dvz = vz[q] - vz[i];
      const double dvdotdr = 1.0 * (dvx * dx + dvy * dy + dvz * dz) + fDist2 * 0.0;
      const double aP = u[i] * gammam1 / density[q], bP = u[q] * gammam1 / density[i];
      const double visc = 0.0;
      double PdV = bR * 0.5 * visc * dvdotdr;
      PdV += bR * aP * dvdotdr;
      spdv += PdV;
      const double acc = (aP + bP) + visc;
      const double s = acc * bR;
      sax += s * dx;
      say += s * dy;
      saz += s * dz;
      PdV = aR * 0.5 * visc * dvdotdr;
      PdV += aR * aP * dvdotdr;
      const double so = -acc * aR;
      oa[4 * (size_t)q + 0] += so * dx;
      oa[4 * (size_t)q + 1] += so * dy;
      oa[4 * (size_t)q + 2] += so * dz;
      oa[4 * (size_t)q + 3] += PdV;
    }
    ax[i] = sax;
    ay[i] = say;
    az[i] = saz;
    pdv[i] = spdv;
  }
  for (int i = 0; i < n; i++) {
    ax[i] += oa[4 * (size_t)i + 0];
    ay[i] += oa[4 * (size_t)i + 1];
    az[i] += oa[4 * (size_t)i + 2];
    pdv[i] += oa[4 * (size_t)i + 3];
  }
  free(oa);
}
