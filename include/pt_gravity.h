/*
 * pt_gravity.h -- C ABI of the B200 Barnes-Hut gravity path.
 *
 * Drop-in replacement for the path ParaTreeT's Gravity example runs once per
 * iteration: universe + SFC keys, key sort, octree build, upward pass of
 * CentroidData / MultipoleMoments, the TransposedDownTraverser walk with
 * GravityVisitor (open / node / leaf), and the kick / perturb integrator.
 *
 * Conventions
 *   - Every function returns an int status: PT_OK (0) or a negative PT_E*
 *     code; pt_last_error() gives the text.  Nothing throws across the ABI.
 *   - Host arrays are FP64 structure-of-arrays in the caller's particle order
 *     (the reference's Particle::order, src/Reader.C:89).  Outputs are always
 *     returned in that order.
 *   - Device memory is owned by the handle.  One host thread per handle.
 *     Work is issued on the handle's stream (pt_set_stream) and every call
 *     that returns host data synchronises that stream.
 *   - Nodes and buckets are reported in the layouts documented at each
 *     getter; node keys are the reference's (root 1, child = key<<3 | c;
 *     src/Subtree.h:325, src/Utility.h:105-108).
 */
#ifndef PT_GRAVITY_H_
#define PT_GRAVITY_H_

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PT_ABI_VERSION 2

enum {
  PT_OK = 0,
  PT_E_ARG = -1,        /* bad argument */
  PT_E_CUDA = -2,       /* CUDA runtime error */
  PT_E_NOMEM = -3,      /* device allocation failed */
  PT_E_STATE = -4,      /* call out of order (e.g. no particles) */
  PT_E_DEVICE = -5,     /* a kernel reported an error status */
  PT_E_NONFINITE = -6,  /* NaN/Inf in particle positions */
  PT_E_UNSUPPORTED = -7 /* feature not built in this library */
};

/* Arithmetic of the traversal. */
enum {
  PT_FP64 = 0,  /* reference-exact FP64 (bit-identical to the reference built
                   with -DUSE_DOUBLE_FP) */
  PT_MIXED = 1,  /* FP64 positions, tree and opening tests; FP32 P2P / P2C
                   interactions on bucket-relative offsets with compensated
                   FP32 accumulation */
  PT_FP64_LISTS = 2  /* the mixed form's two-phase traversal (same lists, same
                        work layout) with FP64 interactions: the FP64
                        comparator of PT_MIXED; equal to PT_FP64 up to the
                        order of each particle's sums (not bit-exact) */
};

/* Traverser of the FP64 form (the interaction set is the same; the order in
 * which a bucket's interactions are summed, and so the last bits, differ). */
enum {
  PT_TRANSPOSED_DOWN = 0,  /* Partition::startDown: TransposedDownTraverser, pre-order
                              per bucket (src/Partition.h:129-134, src/Traverser.h:154-217) */
  PT_BASIC_DOWN = 1        /* Partition::startBasicDown: BasicDownTraverser, breadth first
                              per bucket (src/Partition.h:148-152, src/Traverser.h:296-330) */
};

/* Integrator of pt_step. */
enum {
  PT_KKD = 0,  /* the reference's iteration (src/Driver.h:218-250,
                  src/Particle.C:7-21): forces(x_n); v += a dt/2; v += a dt/2;
                  x += v dt */
  PT_KDK = 1   /* textbook leapfrog: v += a(x_n) dt/2; x += v dt; forces(x_{n+1});
                  v += a dt/2 */
};

typedef struct pt_config {
  double theta;      /* opening angle: GravityVisitor(offset, theta),
                        examples/GravityVisitor.h:16-20, examples/Main.C:55 */
  int bucket;        /* max particles per leaf: Configuration::
                        max_particles_per_leaf (-l), examples/Main.C:29 */
  int precision;     /* PT_FP64 or PT_MIXED */
  int integrator;    /* PT_KKD or PT_KDK */
  double dt_max;     /* max_timestep (-j), examples/Main.C:57,77; the step is
                        min(L / v_max / cbrt(N), dt_max), examples/Gravity.C:63-67 */
  int device;        /* CUDA device ordinal */
  int record_lists;  /* keep per-bucket interaction lists of every force pass */
  /* Periodic cube (Configuration::periodic / fPeriod / nReplicas,
     src/Configuration.h:118-148; examples/Gravity.C:32-48): the tree is walked
     for (2 n_replicas + 1)^3 replica offsets, then the Ewald correction of
     examples/Ewald.{h,C} (root monopole + quadrupole; real-space images within
     ewald_rcut * period, reciprocal vectors |h| <= ewald_hcut) is added.
     Excludes record_lists. */
  int periodic;
  int n_replicas;     /* 0..8 */
  double period;      /* cube side L (> 0) */
  double ewald_rcut;  /* fEwCut, examples/Ewald.h:26 (default 2.6) */
  double ewald_hcut;  /* dEwhCut, examples/Ewald.C:86 (default 2.8) */
  int traversal;      /* PT_TRANSPOSED_DOWN (default) or PT_BASIC_DOWN */
  int reserved[7];
} pt_config;

typedef struct pt_handle pt_handle;

typedef struct pt_counters {
  uint64_t n_pp;       /* P2P pairs, n_src * n_tgt per leaf() (src/Traverser.h:27) */
  uint64_t n_pc;       /* P2C evaluations, n_tgt per node() (src/Traverser.h:35) */
  uint64_t n_open;     /* open() tests */
  int64_t n_nodes;
  int64_t n_buckets;
  int32_t depth;       /* deepest level */
  int32_t launches;    /* kernels this library launched for the pass */
  /* device milliseconds of the last force pass, by phase */
  float ms_keys;       /* bbox + universe + keys */
  float ms_sort;       /* radix sort + permute */
  float ms_build;      /* octree build + bucket order */
  float ms_upward;     /* leaf moments + upward pass */
  float ms_traverse;   /* traversal (the dominant kernel) */
  float ms_total;
} pt_counters;

/* Library / handle ------------------------------------------------------- */
int pt_abi_version(void);
/* Fills the reference's defaults for the Gravity example with the octree:
 * theta 0.7, bucket 16, FP64, KKD, dt_max 1e-5, device 0; not periodic
 * (period 1, 0 replica shells, Ewald cuts 2.6 and 2.8). */
int pt_config_default(pt_config* cfg);
/* Replaces paratreet::initialize<CentroidData> (src/Paratreet.h:220-239) for
 * this path: allocates the device state of one simulation. */
int pt_create(const pt_config* cfg, pt_handle** out);
int pt_destroy(pt_handle* h);
const char* pt_last_error(const pt_handle* h);
/* cudaStream_t as void*; NULL = the handle's own stream. */
int pt_set_stream(pt_handle* h, void* stream);
int pt_set_theta(pt_handle* h, double theta);
int pt_set_precision(pt_handle* h, int precision);
/* Failure-path control of the key sort, for tests.  Each digit pass of the
 * onesweep radix sort (the replacement of std::sort at src/Subtree.h:281)
 * resolves its tile's offsets by looking back at the tiles before it; a look-
 * back polls a tile that has not yet published its counts at most `polls`
 * times (default 2^21, which is never reached in practice) and then gives up.
 * The force pass then stops before it permutes the particles and returns
 * PT_E_DEVICE ("radix sort look-back timed out"); the handle keeps its last
 * consistent state and the next call sorts afresh.  0 gives up at the first
 * poll of an unpublished tile.  polls < 0 is PT_E_ARG. */
int pt_set_sort_spin_limit(pt_handle* h, int64_t polls);

/* Entries per warp region of the two-phase list pools (PT_MIXED and
 * PT_FP64_LISTS; default 32768).  Each warp of the list walk reserves regions
 * of this size; a bucket's list that outgrows what is left of its region
 * moves to a new region of at least twice its length, so smaller regions move
 * lists more often (the lists and results are the same).  A tuning and testing
 * knob; entries < 64 is PT_E_ARG. */
int pt_set_list_region(pt_handle* h, int64_t entries);

/* Particles -------------------------------------------------------------- */
/* Replaces Reader::load + the universe reduction (src/Reader.C:11-107,
 * src/Driver.h:96-107): copies FP64 host SoA to the device.  soft is the
 * per-particle softening (Particle::soft, the Tipsy eps). */
int pt_set_particles(pt_handle* h, int64_t n, const double* x, const double* y, const double* z,
                     const double* vx, const double* vy, const double* vz, const double* m,
                     const double* soft);
/* Same from device pointers (FP64, n elements each); copied device-to-device. */
int pt_set_particles_device(pt_handle* h, int64_t n, const double* x, const double* y,
                            const double* z, const double* vx, const double* vy, const double* vz,
                            const double* m, const double* soft);
int64_t pt_num_particles(const pt_handle* h);

/* Force pass ------------------------------------------------------------- */
/* One force evaluation: universe (src/Driver.h:67-80), keys
 * (src/Decomposition.C:58-64), sort + build + upward (src/Subtree.h:276-384),
 * and Partition::startDown<GravityVisitor> over every bucket
 * (src/Partition.h:129-134, src/Traverser.h:154-217,
 * examples/Gravity.C:29-33). */
int pt_compute_forces(pt_handle* h);
/* Only the buckets [b0, b1) of the DFS-ordered bucket list are traversed
 * (multi-GPU sharding of one system); the tree is still built in full. */
int pt_compute_forces_range(pt_handle* h, int64_t b0, int64_t b1);
/* Accelerations and potentials of the last force pass, caller order.
 * pot: the reference's potential (quadrupole node() terms only,
 * examples/GravityVisitor.h:218); pot_full: every interaction's potential
 * (P2P spline, quadrupole, monopole).  The mixed form's fused fallback
 * (taken only when the interaction-list pools cannot be allocated) leaves
 * pot at zero.  Any pointer may be NULL. */
int pt_get_accel(pt_handle* h, double* ax, double* ay, double* az, double* pot, double* pot_full);
/* Device pointers (sorted order, FP64) of the last force pass, and the
 * sorted-to-caller permutation (int32 order[i] = caller index of sorted i).
 * The arrays may be changed in place before pt_advance / pt_get_accel: the
 * ranks of a sharded run, which build identical trees and so share the sorted
 * order, sum their pt_compute_forces_range results there (outside the range
 * every array is zero).  Any pointer may be NULL. */
int pt_device_accel(pt_handle* h, double** ax, double** ay, double** az, double** pot, double** pot_full,
                    const int32_t** order);

/* Integration ------------------------------------------------------------ */
/* nsteps iterations of src/Driver.h:183-251 (PT_KKD) or leapfrog (PT_KDK).
 * dt = min(L / v_max / cbrt(N), dt_max) per step. */
int pt_step(pt_handle* h, int nsteps);
/* The integrator half of one Driver::run iteration without its force pass:
 * dt = min(L / v_max / cbrt(N), dt_max), then Partition::kick + perturb
 * (src/Partition.h:329-379, src/Particle.C:7-21) with the accelerations now on
 * the device (pt_device_accel), e.g. after the ranks of a sharded run have
 * summed their pt_compute_forces_range results.  Needs a force pass at the
 * current positions; dt may be NULL. */
int pt_advance(pt_handle* h, double* dt);
int pt_get_state(pt_handle* h, double* x, double* y, double* z, double* vx, double* vy, double* vz);
int pt_last_dt(const pt_handle* h, double* dt);

/* Parity / inspection ---------------------------------------------------- */
/* SFC keys of the last pass with the placeholder bit (caller order). */
int pt_get_keys(pt_handle* h, uint64_t* keys);
int pt_get_universe(pt_handle* h, double* lo3, double* hi3);
int pt_get_tree_size(pt_handle* h, int64_t* n_nodes, int64_t* n_buckets);
/* Node dump, breadth-first order.  ints4: [type (1 Leaf, 2 EmptyLeaf,
 * 6 Internal; src/Node.h:82-95), depth, count, n_children]; dbls18:
 * [mass, cm x/y/z, soft, radius, xx, xy, xz, yy, yz, zz, box lo x/y/z,
 * box hi x/y/z] (CentroidData + MultipoleMoments,
 * examples/CentroidData.h:24-38, examples/MultipoleMoments.h:161-184). */
int pt_get_tree(pt_handle* h, uint64_t* keys, int32_t* ints4, double* dbls18);
/* Keys of the buckets (leaves) in DFS order (Subtree::leaves). */
int pt_get_bucket_keys(pt_handle* h, uint64_t* keys);
/* Interaction lists of the last pass (needs record_lists): CSR over buckets
 * in DFS order; entries are node keys, kinds 0 = leaf() P2P, 1 = node() P2C.
 * PT_FP64 records them in the reference's traversal order; the two-phase
 * forms (PT_MIXED, PT_FP64_LISTS) record the lists their walk wrote (per
 * bucket its leaves, then its nodes) -- the same sets. */
int pt_get_lists_size(pt_handle* h, int64_t* total);
int pt_get_lists(pt_handle* h, int64_t* offsets, uint64_t* keys, int32_t* kinds);
/* Per bucket (DFS order), an order-independent 64-bit digest of its
 * interaction list in the last pass and the list's length: the sum mod 2^64
 * of a mix of (node, class) over the entries, class 0 = leaf() P2P,
 * 1 = node() quadrupole P2C, 2 = node() monopole P2C (addGravity).  which = 0:
 * the recorded lists (record_lists, the FP64 walk in the reference's order);
 * which = 1: the lists that the mixed form's two-phase walk wrote and
 * evaluated in its last pass (non-periodic, every bucket).  Equal digests of
 * the two show that both forms make the same interactions (the traversal of
 * src/Traverser.h:154-217 with GravityVisitor::open / node / leaf) without
 * copying the lists to the host.  PT_E_STATE if the lists are not there. */
int pt_get_list_digests(pt_handle* h, int which, uint64_t* digest, int64_t* count);
int pt_get_counters(pt_handle* h, pt_counters* c);
/* P2P pairs + P2C evaluations of each bucket (DFS order, pt_get_tree_size
 * buckets) in the last force pass, replicas included; 0 for buckets outside
 * the traversed range.  The cost model for splitting buckets over ranks
 * (the work the reference's decompositions balance, src/Decomposition.C). */
int pt_get_bucket_work(pt_handle* h, uint64_t* work);

/* Differentiation ---------------------------------------------------------
 * No reference counterpart (ParaTreeT has no gradients).  All three need a
 * force pass over every bucket with config.record_lists set, and work on its
 * interaction lists: a "fixed interaction list" is the set of leaf() and
 * node() interactions of each bucket that the pass recorded. */
/* Re-evaluates the recorded lists in FP64 after replacing positions and/or
 * masses (caller order, host; NULL keeps the current values) while keeping
 * the tree topology and the lists: moments are recomputed, nothing is
 * re-walked.  Results via pt_get_accel. */
int pt_forces_frozen(pt_handle* h, const double* x, const double* y, const double* z, const double* m);
/* Gradient of sum_i cot_i . a_i with respect to every position and mass for
 * the recorded lists (FP64; tidal tensors through leaf() and node(), and the
 * upward pass in closed form).  Host arrays in caller order. */
int pt_adjoint(pt_handle* h, const double* cot_ax, const double* cot_ay, const double* cot_az, double* gx,
               double* gy, double* gz, double* gm);
/* Loss L = 0.5 sum_i |x_i(T) - y_i|^2 after nsteps leapfrog (KDK) steps of
 * fixed dt from the handle's current particles, and its gradient with respect
 * to the initial positions, velocities and masses.  (x, v) are checkpointed
 * every ckpt_every steps (<= 0: round(sqrt(nsteps))); each segment is
 * recomputed forward during the backward sweep.  Forces use the handle's
 * precision, the adjoint is FP64.  Host arrays in caller order; any gradient
 * pointer may be NULL.  The handle is left at the initial state. */
int pt_chain_grad(pt_handle* h, int nsteps, double dt, int ckpt_every, const double* yx, const double* yy,
                  const double* yz, double* loss, double* gx, double* gy, double* gz, double* gvx,
                  double* gvy, double* gvz, double* gm);

/* SPH density ---------------------------------------------------------------
 * The density pass of the reference's SPH example on the same tree:
 * startUpAndDown<DensityVisitor> (examples/SPH.C:77-86, examples/
 * DensityVisitor.h: the k = 32 nearest neighbours of every particle, the
 * particle itself included) and DensityFn (examples/SPH.C:11-37): ball_sq =
 * the 32nd smallest d2, density = sum_j kernelM4(4 d2_j / ball_sq) m_j /
 * (pi/8 ball_sq^1.5) with kernelM4 of examples/SPHUtils.h.  FP64; the tree is
 * rebuilt from the current positions (an earlier force pass's results are
 * dropped).  Caller order; any output may be NULL except that nbr and nbr_d2
 * go together: 32 neighbours per particle (caller indices, -1 past N) sorted
 * by (d2, index), and their d2. */
int pt_sph_density(pt_handle* h, double* density, double* ball_sq, int32_t* nbr, double* nbr_d2);

/* SPH pressure ---------------------------------------------------------------
 * The pressure pass of the SPH example after its density pass
 * (examples/SPH.C:87-101): startDown<PressureVisitor>, then ForceFn
 * (examples/SPH.C:39-64) with doSPHCalc (examples/SPHUtils.h:64-133; visc = 0,
 * aFac = vFac = 1, H = 0, gamma = 5/3) over each particle's 32 neighbours from
 * pt_sph_density's pass (run here first on the current positions), then the
 * opposite reactions (applyAccumulatedOpposingEffects).  u: internal energy
 * per particle (u_predicted; velocity_predicted = the handle's velocities).
 * Outputs: pressure accelerations and PdV work; density optional.  FP64; the
 * reactions are summed by atomic adds, so their order (the last bits) is not
 * fixed.  A term that fails doSPHCalc's isfinite(acc) assertion (examples/
 * SPHUtils.h:122; a ball of zero radius, as with N = 1 or coincident
 * particles) returns PT_E_DEVICE.  Caller order; any output may be NULL. */
int pt_sph_pressure(pt_handle* h, const double* u, double* density, double* ax, double* ay, double* az,
                    double* pdv);

/* SPH step ------------------------------------------------------------------
 * nsteps iterations of the SPH example's Driver::run loop (src/Driver.h:
 * 183-251 with examples/SPH.C:74-111): tree build, the density pass, the
 * pressure pass (as pt_sph_pressure, reading u_pred as u_predicted and
 * vpx/vpy/vpz as velocity_predicted), then Particle::kick and
 * Particle::perturb with their SPH updates (src/Particle.C:7-21):
 * v += a dt/2 twice, v_pred = v + a dt, x += v dt, u -= PdV 0.5e-7 dt,
 * u_pred = u - PdV 0.5e-7 dt.  dt = config.dt_max (the SPH example's
 * getTimestep returns max_timestep).  u, u_pred and v_pred are in/out host
 * arrays in caller order (start them as u and the velocities, as
 * src/Reader.C:90-91 does); positions and velocities stay in the handle
 * (pt_get_state).  FP64; the pressure pass's reactions are atomic adds, so
 * trajectories match the reference to rounding, not bit for bit.  A step whose
 * pressure pass fails (as pt_sph_pressure) returns its error before the kick,
 * with the particles of the steps before it. */
int pt_sph_step(pt_handle* h, int nsteps, double* u, double* u_pred, double* vpx, double* vpy, double* vpz);

/* FP64 direct sum (the force-error yardstick) ------------------------------
 * Isolated spline-softened sum over all particles for nt caller indices,
 * the kernel of examples/GravityVisitor.h:87-120 with twoh = soft_i + soft_j. */
int pt_direct_sum(pt_handle* h, int64_t nt, const int32_t* targets, double* ax, double* ay,
                  double* az, double* pot);

/* FP64 periodic (Ewald) direct sum, the yardstick of the periodic pass: the
 * Ewald sum of the cube of side config.period (alpha = 4/L, real-space images
 * within 1.5 L, reciprocal |h|^2 <= 64), with the spline kernel for the
 * nearest image within soft_i + soft_j, for nt caller indices.  Potentials
 * include the uniform-background and self terms.  No reference counterpart. */
int pt_ewald_direct_sum(pt_handle* h, int64_t nt, const int32_t* targets, double* ax, double* ay,
                        double* az, double* pot);

/* No counterpart in the reference.  The same FP64 direct sum for callers that
 * cannot allocate device memory (their buffers come from a pool or budget of
 * their own, and cudaMalloc / cudaFree would also synchronise the device):
 * every pointer except errbuf is DEVICE memory supplied by the caller
 * (sources x..soft of n particles, nt int32 target indices into them, nt
 * outputs per array; any output may be NULL).  Nothing is allocated: the only
 * scratch is a fixed 8 MiB array inside the library, held by every GPU that
 * loads it until exit, which limits nt to 262,136 (larger nt is rejected with
 * PT_E_ARG).  Works on the current device; the first call on a device looks up
 * the array's address (make that call before any stream capture).  Issued on
 * `stream` (cudaStream_t, NULL = default); every call copies a status word to
 * host memory and synchronises `stream` before it returns.  A target index
 * outside [0, n) is found on the device and returned as PT_E_ARG with nothing
 * written to the outputs.  Calls that overlap on the GPU share the array and
 * race.  On error a message is written to errbuf (errlen bytes, may be NULL). */
int pt_direct_sum_noalloc(int64_t n, const double* x, const double* y, const double* z,
                          const double* m, const double* soft, int64_t nt, const int32_t* targets,
                          double* ax, double* ay, double* az, double* pot, void* stream,
                          char* errbuf, size_t errlen);

#ifdef __cplusplus
}
#endif

#endif /* PT_GRAVITY_H_ */
