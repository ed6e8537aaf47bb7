/*
 * pt_oracle.h -- CPU oracle for the Barnes-Hut gravity path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a plain-C restatement of ParaTreeT's
 * gravity path (keys, sort, octree build, FIFO upward pass, transposed
 * traversal with GravityVisitor, kick/perturb) used as the checker for the
 * CUDA path and as the timed CPU baseline.  Nothing in the product links or
 * calls it.  Each function in pt_oracle.c cites the reference lines it follows.
 */
#ifndef PT_ORACLE_H_
#define PT_ORACLE_H_

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct pto_sim pto_sim;

/* Node types, numbered as Node<Data>::Type in src/Node.h:82-95. */
enum { PTO_LEAF = 1, PTO_EMPTY = 2, PTO_INTERNAL = 6 };

pto_sim* pto_create(int n, const double* x, const double* y, const double* z, const double* vx,
                    const double* vy, const double* vz, const double* m, const double* soft, int bucket,
                    double theta, double dt_max, int threads);
void pto_destroy(pto_sim* s);
/* One force evaluation (keys -> traversal); record_lists keeps the per-bucket
 * interaction lists of this evaluation. */
int pto_forces(pto_sim* s, int record_lists);
/* nsteps iterations of forces -> kick -> perturb -> new universe -> rekey. */
int pto_run(pto_sim* s, int nsteps);

void pto_get_acc(const pto_sim* s, double* ax, double* ay, double* az, double* pot, double* pot_full);
void pto_get_keys(const pto_sim* s, uint64_t* keys);
void pto_get_state(const pto_sim* s, double* x, double* y, double* z, double* vx, double* vy, double* vz);
void pto_get_universe(const pto_sim* s, double* lo3, double* hi3);
/* counters: n_pp, n_pc, n_open, n_buckets; times: build, traverse seconds */
void pto_get_counters(const pto_sim* s, unsigned long long* out4, double* times2, double* last_dt);
unsigned long long pto_get_mono(const pto_sim* s);
long pto_num_nodes(const pto_sim* s);
/* Same layout as the reference-side dump: ints [type, depth, count, n_children],
 * 18 doubles [mass, cm3, soft, radius, xx, xy, xz, yy, yz, zz, lo3, hi3]. */
void pto_get_nodes(const pto_sim* s, uint64_t* keys, int* ints4, double* dbls18);
long pto_num_buckets(const pto_sim* s);
void pto_get_bucket_keys(const pto_sim* s, uint64_t* keys);
long pto_list_total(const pto_sim* s);
void pto_get_lists(const pto_sim* s, long* offsets, uint64_t* keys, int* kinds);

/* 0: the transposed down traversal (Partition::startDown, pre-order per
 * bucket); 1: the basic down traversal (Partition::startBasicDown,
 * breadth first per bucket) -- the same interactions in another order. */
void pto_set_traversal(pto_sim* s, int basic_down);
/* Periodic cube of side L: (2n+1)^3 replica walks and the reference's Ewald
 * correction with real-space radius rcut*L and reciprocal cut |h| <= hcut. */
void pto_set_periodic(pto_sim* s, int periodic, double L, int n_replicas, double rcut, double hcut);
/* FP64 periodic (Ewald) direct sum; see pt_oracle.c. */
void pto_ewald_direct(int n, const double* x, const double* y, const double* z, const double* m,
                      const double* soft, double L, int nt, const int* targets, double* ax, double* ay,
                      double* az, double* pot, int threads);

/* SPH density of the reference's SPH example: k nearest neighbours (itself
 * included, brute force) and the M4-kernel density; see pt_oracle.c. */
void pto_sph_density(int n, const double* x, const double* y, const double* z, const double* m, int k,
                     int threads, double* density, double* ballsq, int* nbr, double* nd2);

/* The SPH example's pressure pass after pto_sph_density: pressure
 * accelerations and PdV work with the opposite reactions added; see
 * pt_oracle.c. */
void pto_sph_pressure(int n, const double* x, const double* y, const double* z, const double* vx,
                      const double* vy, const double* vz, const double* m, const double* u, const double* density,
                      const double* ballsq, const int* nbr, const double* nd2, int k, double* ax, double* ay,
                      double* az, double* pdv);

/* FP64 direct sum (spline softening, twoh = soft_i + soft_j, G = 1) over
 * all n sources for nt target indices; isolated (no periodic images). */
void pto_direct(int n, const double* x, const double* y, const double* z, const double* m,
                const double* soft, int nt, const int* targets, double* ax, double* ay, double* az,
                double* pot, int threads);

#ifdef __cplusplus
}
#endif

#endif
