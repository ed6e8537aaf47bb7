// pt_launch.h -- host-side launchers of the kernels in k_*.cu.
#pragma once

#include <cstddef>
#include <cstdint>
#include <cuda_runtime.h>

#include "pt_internal.cuh"

namespace pt {

// k_keys.cu
void launch_bbox(const double* x, const double* y, const double* z, int64_t n, double* partial, int nblocks,
                 double* uni, unsigned* status, cudaStream_t st);
void launch_keys(const double* x, const double* y, const double* z, int64_t n, const double* uni, uint64_t* key,
                 uint32_t* idx, int grid, cudaStream_t st);
void launch_vmax2(const double* vx, const double* vy, const double* vz, int64_t n, unsigned long long* out,
                  int grid, cudaStream_t st);

// k_sort.cu
size_t scan_scratch_bytes(int64_t n);
void scan_exclusive(const uint32_t* in, uint32_t* out, int64_t n, uint32_t* scratch, uint32_t* total,
                    cudaStream_t st);
size_t sort_scratch_bytes(int64_t n);
// 0 on success, -1 if the kernel attribute could not be set; spin_limit =
// polls of an unpublished tile before the look-back gives up (kErrSort)
int radix_sort_pairs(uint64_t* k0, uint32_t* v0, uint64_t* k1, uint32_t* v1, int64_t n, void* scratch,
                     unsigned* status, int sms, long long spin_limit, cudaStream_t st);
void gather_f64(const double* in, double* out, const uint32_t* idx, int64_t n, int grid, cudaStream_t st);
void gather_i32(const int32_t* in, int32_t* out, const uint32_t* idx, int64_t n, int grid, cudaStream_t st);

// k_build.cu
void launch_init_root(Nodes nd, int64_t n, int bucket, cudaStream_t st);
void launch_flag_internal(const int32_t* type, int64_t begin, int64_t count, uint32_t* flags, cudaStream_t st);
void launch_build_children(Nodes nd, const uint64_t* keys, int64_t begin, int64_t count, const uint32_t* rank,
                           int64_t next_begin, int bucket, int64_t cap, unsigned* status, cudaStream_t st);
void launch_count_subtree(Nodes nd, int64_t begin, int64_t count, cudaStream_t st);
void launch_base_topdown(Nodes nd, int64_t begin, int64_t count, cudaStream_t st);
void launch_assign_buckets(Nodes nd, int64_t nnodes, int32_t* buckets, int nleaves, cudaStream_t st);

// k_fp64.cu
void launch_leaf_moments(Nodes nd, int64_t nnodes, Particles p, cudaStream_t st);
void launch_upward_level(Nodes nd, int64_t begin, int64_t count, cudaStream_t st);
void launch_finalize(Nodes nd, int64_t nnodes, double gfac, int want_f32, cudaStream_t st);
void launch_traverse_f64(const TravParams& P, const Mom* mom, int grid, cudaStream_t st);
void launch_replay_f64(const TravParams& P, int grid, cudaStream_t st);
void launch_kick_perturb(Particles p, int64_t n, double dt, int grid, cudaStream_t st);
void launch_kick_half(Particles p, int64_t n, double dt, int grid, cudaStream_t st);
void launch_drift(Particles p, int64_t n, double dt, int grid, cudaStream_t st);
void launch_direct_sum(const double* x, const double* y, const double* z, const double* m, const double* soft,
                       int64_t n, const int32_t* tgt, int64_t nt, int nsplit, double* part, cudaStream_t st);

// k_mixed.cu
void launch_prep_sources(const int32_t* buckets, int64_t nbuckets, const WalkRec* walk, Particles p, float4* srcf,
                         float* softf, cudaStream_t st);
void launch_traverse_mixed(const TravParams& P, const Mom* mom, int grid, cudaStream_t st);

// k_ewald.cu
void launch_ewald_correction(Particles p, int64_t i0, int64_t i1, const EwaldRoot& R, const double4* htab,
                             cudaStream_t st);
void launch_ewald_structure(const double* x, const double* y, const double* z, const double* m, int64_t n,
                            const double4* kv, int nk, double* S, cudaStream_t st);
void launch_ewald_real(const double* x, const double* y, const double* z, const double* m, const double* soft,
                       int64_t n, const int32_t* tgt, int64_t nt, int nsplit, double L, double alpha, double rcut,
                       double* part, cudaStream_t st);
void launch_ewald_recip(const double* x, const double* y, const double* z, const double* m, const int32_t* tgt,
                        int64_t nt, const double4* kv, int nk, const double* S, double alpha, double V, double* out,
                        cudaStream_t st);

// k_mixed2.cu
int walk_lists_grid(int sms);
void launch_walk_lists(const TravParams& P, const ListParams& L, const Mom* mom, int grid, cudaStream_t st);
// eval_p2c (store or add per P.accumulate) then eval_p2p (add); each takes its
// bucket queue from P.work and work2 respectively (zeroed by the caller)
void launch_eval_lists(const TravParams& P, const ListParams& L, const Mom* mom, int grid, cudaStream_t st,
                       unsigned* work2);
// k_f64lists.cu
void launch_eval_lists_f64(const TravParams& P, const ListParams& L, const Mom* mom, int grid, cudaStream_t st,
                           unsigned* work2);

// k_sph.cu
int sph_k();
void launch_sph_pressure(Particles p, const double* density, const double* ballsq, const double* u,
                         const int32_t* nbr, const double* nd2, int64_t n, double* ax, double* ay, double* az,
                         double* pdv, unsigned* status, int grid, cudaStream_t st);
void launch_sph_kick_perturb(Particles p, const double* ax, const double* ay, const double* az, const double* pdv,
                             double* u, double* u_pred, double* vpx, double* vpy, double* vpz, int64_t n, double dt,
                             int grid, cudaStream_t st);
int sph_knn_slots(int grid);
void launch_sph_density(Particles p, int64_t n, const Mom* mom, const WalkRec* walk, const int32_t* buckets,
                        int64_t nbuckets, int64_t nnodes, double* density, double* ballsq, int32_t* nbr, double* nd2,
                        double* lists_d, int32_t* lists_i, unsigned* work, unsigned* status, int grid,
                        cudaStream_t st);

// k_adjoint.cu
void launch_adjoint(const AdjParams& A, int grid, cudaStream_t st);

// k_util.cu
void launch_pools_to_csr(const int32_t* pc_pool, const int32_t* pp_pool, const int64_t* pc_start,
                         const int32_t* pc_count, const int64_t* pp_start, const int32_t* pp_count, int64_t nb,
                         const int64_t* off, int32_t* node, int8_t* kind, cudaStream_t st);
void launch_digest_recorded(const int64_t* off, const int32_t* node, const int8_t* kind, int64_t nb,
                            unsigned long long* dig, int64_t* cnt, cudaStream_t st);
void launch_digest_two_phase(const int32_t* pc_pool, const int32_t* pp_pool, const int64_t* pc_start,
                             const int32_t* pc_count, const int64_t* pp_start, const int32_t* pp_count, int64_t nb,
                             unsigned long long* dig, int64_t* cnt, cudaStream_t st);
void launch_scatter_f64(const double* in, double* out, const int32_t* order, int64_t n, int grid, cudaStream_t st);
void launch_scatter_u64(const uint64_t* in, uint64_t* out, const int32_t* order, int64_t n, int grid,
                        cudaStream_t st);
void launch_iota_i32(int32_t* out, int64_t n, int grid, cudaStream_t st);
void launch_inverse_perm(const int32_t* order, int32_t* inv, int64_t n, int grid, cudaStream_t st);
void launch_map_index(const int32_t* inv, const int32_t* in, int32_t* out, int64_t n, cudaStream_t st);
void launch_axpy1(int64_t n, double alpha, const double* x, double* y, int grid, cudaStream_t st);
void launch_axpy3(int64_t n, double alpha, const double* x0, const double* x1, const double* x2, double* y0,
                  double* y1, double* y2, int grid, cudaStream_t st);
void launch_gather_by_order(const double* in, double* out, const int32_t* order, int64_t n, int grid,
                            cudaStream_t st);

}  // namespace pt
