/*
 * voxneus_b200: the VoxNeuS geometry-and-rendering hot path for NVIDIA B200 (sm_100a).
 *
 * C ABI: plain pointers, sizes and host scalars. Every pointer named as an array of tensor
 * data is DEVICE memory (float32 / int64 / uint8 / uint32 as stated); `res`, `xyz_min`,
 * `xyz_max`, `eps` and other 3-element arrays are HOST memory. `stream` is a cudaStream_t
 * (NULL = legacy default stream). No call synchronises the host with the device and no call
 * allocates device memory: scratch buffers (partials, counters, block scratch) are passed
 * in by the caller, with the size queried from the matching *_blocks / *_words function.
 * Counters passed as `counter` must be zero before their first use; the kernels leave them
 * at zero when they finish.
 *
 * Return value: VX_OK (0) or an error code; vx_last_error() then describes the failure
 * (thread-local). Arguments are validated before any launch.
 *
 * Grid layout: a dense float32 SDF volume (X, Y, Z) with z fastest, linear index
 * (x * Y + y) * Z + z; at most 2^31 - 1 voxels. World bounds xyz_min / xyz_max; voxel size
 * eps = (xyz_max - xyz_min) / (res - 1).
 *
 * Reference paths below are inside Code/ of rishidevde/VoxNeus.
 */
#ifndef VOXNEUS_B200_H
#define VOXNEUS_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VX_OK 0
#define VX_ERR_INVALID 1
#define VX_ERR_CUDA 2

/* ---------------------------------------------------------------- library ---------------- */
const char* vx_last_error(void);
const char* vx_version(void);
/* Number of kernel launches issued by this library since load (for launch accounting). */
uint64_t vx_launch_count(void);

/* ------------------------------------------- reference extension interface ---------------- *
 * Drop-in equivalents of the pybind module voxneus.cuda._backend (voxneus/cuda/adam_upd.cpp:118-125).
 * The voxel size is passed as host floats instead of a device tensor read with .item(). */

/* gradient_interp_forward (voxneus/cuda/gradient_interp.cu:154-183): Eq.7 interpolated gradient at
 * grid-index coordinates coords (n,3) -> out_grad (n,3). */
int vx_gradient_interp_forward(const float* grid, const int32_t res[3], const float* coords, int64_t n,
                               const float eps[3], float* out_grad, void* stream);

/* gradient_interp_backward (voxneus/cuda/gradient_interp.cu:185-212): accumulates the adjoint of
 * Eq.7 into grad_grid (X,Y,Z). */
int vx_gradient_interp_backward(const float* grad_out, const float* coords, int64_t n, float* grad_grid,
                                const int32_t res[3], const float eps[3], void* stream);

/* Blocks used by the list-form regularizers; partials must hold 3 doubles per block. */
int vx_reg_list_blocks(int64_t n_verts);

/* eikonal_grad (voxneus/cuda/eikonal_grad.cu:71-101): closed-form eikonal gradient of the listed
 * vertices (n_verts,3) accumulated into grad_grid (nullable: loss only), scale 2/n_verts * weight.
 * losses (device, nullable) receives [mean (|n|-1)^2 over interior vertices, 0]. */
int vx_eikonal_grad(const float* grid, const int32_t res[3], const int64_t* verts, int64_t n_verts, float* grad_grid,
                    const float eps[3], float weight, double* partials, int n_partials, unsigned int* counter,
                    float* losses, void* stream);

/* curvature_grad (voxneus/cuda/curvature_grad.cu:73-103): closed-form Laplacian curvature gradient;
 * losses receives [0, mean(Lx^2+Ly^2+Lz^2) over interior vertices]. */
int vx_curvature_grad(const float* grid, const int32_t res[3], const int64_t* verts, int64_t n_verts,
                      float* grad_grid, const float eps[3], float weight, double* partials, int n_partials,
                      unsigned int* counter, float* losses, void* stream);

/* adam_upd / masked_adam_upd (voxneus/cuda/adam_upd_kernel.cu:40-82): in-place Adam over n elements;
 * the masked form skips elements whose gradient is exactly 0. */
int vx_adam_upd(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, int step, float beta1,
                float beta2, float lr, float eps, void* stream);
int vx_masked_adam_upd(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n, int step,
                       float beta1, float beta2, float lr, float eps, void* stream);

/* torch.optim.Adam's update (no counterpart in the reference extension: the reference steps its
 * network parameters, training/optimizer.py:119-154, with torch.optim.Adam):
 * m = b1 m + (1-b1) g, v = b2 v + (1-b2) g^2, p -= (lr / (1 - b1^t)) m / (sqrt(v) / sqrt(1 - b2^t) + eps),
 * over several tensors, each with its own step count t and learning rate (its parameter group's),
 * one launch per 8 tensors. All segments are updated in place. */
typedef struct vx_adam_segment {
  float* param;
  const float* grad;
  float* exp_avg;
  float* exp_avg_sq;
  int64_t n;
  int64_t step;
  float lr;
  /* Optional, for launches replayed from a CUDA graph: device floats {lr / (1 - b1^t),
   * 1 / sqrt(1 - b2^t), the step size to use when *lr_flag is nonzero}, written before each replay
   * (vx_adam_torch_step_scalars); step and lr are then ignored. lr_flag may be NULL. */
  const float* step_scalars;
  const int* lr_flag;
} vx_adam_segment;
int vx_adam_torch(const vx_adam_segment* segs, int n_segs, float beta1, float beta2, float eps, void* stream);

/* SparseGridAdam's vectorised torch path (training/optimizer.py:86-113, the plain-PyTorch mode of
 * the grid optimizer): the torch formula above, and elements whose gradient is exactly 0 keep p, m
 * and v. Same segments as vx_adam_torch (step_scalars/lr_flag optional). */
int vx_masked_adam_torch(const vx_adam_segment* segs, int n_segs, float beta1, float beta2, float eps,
                         void* stream);

/* Host helpers giving exactly the scalars the updates above compute from (step, lr): the
 * reference formula's step size lr * sqrt(1 - b2^t) / (1 - b1^t) in float, and torch's
 * {lr / (1 - b1^t), 1 / sqrt(1 - b2^t)} in double rounded to float. */
float vx_adam_reference_step_size(int step, float beta1, float beta2, float lr);
void vx_adam_torch_step_scalars(int64_t step, float beta1, float beta2, float lr, float out[2]);

/* vx_masked_adam_upd with its step size read from device memory (*step_size, from
 * vx_adam_reference_step_size), for launches replayed from a CUDA graph. */
int vx_masked_adam_upd_dev(float* param, const float* grad, float* exp_avg, float* exp_avg_sq, int64_t n,
                           const float* step_size, float beta1, float beta2, float eps, void* stream);

/* ------------------------------------------------------------ field queries --------------- */

/* DenseSDFGrid.query_sdf (models/sdf_grid.py:90-120) and query_normals (:122-160) in one pass over
 * world points xyz (n,3). Outputs, each nullable: sdf (n), grad (n,3) (Eq.7, unnormalised),
 * normal (n,3), corners (n,8,3) int64, weights (n,8) (geometry/coordinates.py:55-124). */
int vx_field_query(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                   const float* xyz, int64_t n, float* sdf, float* grad, float* normal, int64_t* corners,
                   float* weights, void* stream);

/* vx_field_query's sdf, grad and normal outputs (models/sdf_grid.py:90-160) for a large batch of
 * scattered points, computed in spatial order: the points are sorted by the Morton code of their
 * grid cell, queried in that order and each result is written at the point's own index, so the
 * outputs are bit-identical to vx_field_query's. For grids larger than the L2 cache, where
 * scattered points read every stencil from a different DRAM row. n < 2^31; workspace: at least
 * vx_field_query_sorted_workspace(n, res) bytes, 256-byte aligned (0 when the size query fails,
 * which needs a CUDA device). */
int64_t vx_field_query_sorted_workspace(int64_t n, const int32_t res[3]);
int vx_field_query_sorted(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                          const float* xyz, int64_t n, float* sdf, float* grad, float* normal, void* workspace,
                          int64_t workspace_bytes, void* stream);

/* Adjoint of vx_field_query: accumulates dL/dgrid from d_sdf (n), d_grad (n,3), d_normal (n,3)
 * (each nullable) into grad_grid. */
int vx_field_query_backward(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                            const float* xyz, int64_t n, const float* d_sdf, const float* d_grad,
                            const float* d_normal, float* grad_grid, void* stream);

/* get_voxel_corners_and_weights (geometry/coordinates.py:55-124) at grid-index coordinates (n,3):
 * corners (n,8,3) int64 and weights (n,8), each nullable. */
int vx_corners_weights(const float* coords, int64_t n, const int32_t res[3], int64_t* corners, float* weights,
                       void* stream);

/* SDF + Eq.7 normal on a regular lattice (lattice[0] x lattice[1] x lattice[2] points spanning
 * [lat_min, lat_max] per axis, z fastest, torch.linspace spacing); positions are implicit. The
 * batched query of geometry/mesh.py:80-114 on a lattice. sdf (N) and normal (N,3) nullable. */
int vx_field_query_lattice(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                           const int32_t lattice[3], const float lat_min[3], const float lat_max[3], float* sdf,
                           float* normal, void* stream);

/* ------------------------------------------------------------------ sampler ---------------- */

/* near_far_from_sphere (rendering/rays.py:102-128). */
int vx_near_far_from_sphere(const float* rays_o, const float* rays_d, int64_t n, float radius, float* near_out,
                            float* far_out, void* stream);

/* RaySampler.sample_multistep_sdf (rendering/sampler.py:127-204): stratified samples, then
 * up_sample_steps NeuS upsampling steps (inv_s = 64 * 2^i) with the occupancy modulation of
 * up_sample, each merged into the sorted sample list; outputs z (nullable), dists and mid, each
 * (n_rays, n_samples + n_importance). near/far nullable (computed from the unit sphere).
 * t_lin: torch.linspace(0, 1, n_samples); u_det: the deterministic sample_pdf uniforms
 * linspace(0.5/k, 1-0.5/k, k), k = n_importance / up_sample_steps; with perturb, t_rand
 * (n_rays, n_samples) and u (up_sample_steps, n_rays, k) are the uniforms the reference draws
 * (sampler.py:117, :44). occupancy: (occ_res^3) bool mask or NULL. k <= 32; total <= 256. */
int vx_sample_multistep(const float* grid, const int32_t res[3], const float xyz_min[3], const float xyz_max[3],
                        const float* rays_o, const float* rays_d, const float* near_in, const float* far_in,
                        int64_t n_rays, int n_samples, int n_importance, int up_sample_steps, int perturb,
                        const float* t_lin, const float* t_rand, const float* u, const float* u_det,
                        const uint8_t* occupancy, int occ_res, const float occ_min[3], const float occ_max[3],
                        float* z_out, float* dists_out, float* mid_out, void* stream);

/* up_sample (rendering/sampler.py:243-292): one NeuS upsampling step on sorted z (n_rays, n) with
 * SDF values sdf (n_rays, n) -> out (n_rays, n_importance) in sample_pdf order. u (n_rays,
 * n_importance) or NULL with u_det (deterministic). */
int vx_up_sample(const float* rays_o, const float* rays_d, const float* z, const float* sdf, int64_t n_rays, int n,
                 int n_importance, float inv_s, const float* u, const float* u_det, const uint8_t* occupancy,
                 int occ_res, const float occ_min[3], const float occ_max[3], float* out, void* stream);

/* sample_pdf (rendering/sampler.py:11-66): bins (n_rays, n_bins), weights (n_rays, n_bins-1) -> out
 * (n_rays, n_samples); idx_out (nullable) receives the searchsorted(right=True) indices. With cdf
 * (n_rays, n_bins) given, weights are ignored and that CDF is inverted as is. */
int vx_sample_pdf(const float* bins, const float* weights, const float* cdf, int64_t n_rays, int n_bins,
                  int n_samples, const float* u, const float* u_det, float* out, int64_t* idx_out, void* stream);

/* The sort-and-carry of cat_z_vals (rendering/sampler.py:295-320): per ray, the depths z_old
 * (n_rays, n_old) and z_new (n_rays, n_new; need not be sorted) concatenated and sorted ascending
 * as torch.sort orders floats (NaN last) into z_out (n_rays, n_old + n_new); with sdf_out given,
 * the SDF values sdf_old / sdf_new move with their depths (the reference's gather by the sort's
 * indices). Equal depths keep concatenation order. n_old + n_new <= 8192. */
int vx_cat_z_vals(const float* z_old, const float* z_new, const float* sdf_old, const float* sdf_new, int64_t n_rays,
                  int n_old, int n_new, float* z_out, float* sdf_out, void* stream);

/* ---------------------------------------------------------- render (per sample) ------------ */

/* Pass-2 geometry of VoxNeuS.render (models/voxneus.py:226-236 -> forward_points :115-167):
 * positions o + d*mid for (n_rays, n_samples) midpoints, trilinear SDF, Eq.7 gradient and normal;
 * sdf (nullable), normal (required), grad (nullable); vr_bitmap (nullable) receives the 8 Eq.7
 * corners of every sample (the V_R of regularization/active_vertices.py:12-50). */
int vx_render_geometry_forward(const float* grid, const int32_t res[3], const float xyz_min[3],
                               const float xyz_max[3], const float* rays_o, const float* rays_d, const float* mid,
                               int64_t n_rays, int n_samples, float* sdf, float* normal, float* grad,
                               uint32_t* vr_bitmap, void* stream);

/* Adjoint of vx_render_geometry_forward: recomputes positions and normals and accumulates into
 * grid_grad the SDF term (d_sdf) and the Eq.7 term from d_normal (n,3) + d_normal2 (row stride
 * ld2, e.g. the normal columns of the radiance-MLP input gradient) + d_grad; each nullable.
 * grad_fwd: the forward's `grad` output (n,3), read instead of recomputing the Eq.7 gradient for
 * the normalisation's adjoint (the same values), or NULL. */
int vx_render_geometry_backward(const float* grid, const int32_t res[3], const float xyz_min[3],
                                const float xyz_max[3], const float* rays_o, const float* rays_d, const float* mid,
                                int64_t n_rays, int n_samples, const float* d_sdf, const float* d_normal,
                                const float* d_normal2, int64_t ld2, const float* d_grad, const float* grad_fwd,
                                float* grid_grad, void* stream);

/* Radiance-MLP input rows (models/voxneus.py:147-157): hash features (models/radiance_hash.py:71-166,
 * 2 per level, NeuS2 level weights level_weights (nullable = all 1)) in columns [0, 2L), degree-4 SH
 * of the view direction (models/embedder.py:55-87) at sh_col (-1: none), the normal copied to
 * normal_col (-1: none), pad_col zeroed (-1: none). Points are either normalised pts_norm (n,3), or
 * world positions o + d*mid of (rays, n_samples) normalised by xyz_min/xyz_max; both are clamped to
 * [0,1] (radiance_hash.py:213). dirs (row stride dir_stride) or, when NULL, rays_d per ray. table
 * NULL skips the hash columns. */
int vx_appearance_forward(const float* table, int n_levels, int log2_size, int n_features, const int32_t* level_res,
                          const float* level_weights, const float* pts_norm, const float* rays_o, const float* rays_d,
                          const float* mid, int n_samples, const float xyz_min[3], const float xyz_max[3],
                          int64_t n_points, float* out, int64_t ld, int sh_col, const float* dirs,
                          int64_t dir_stride, int normal_col, const float* normals, int pad_col, void* stream);

/* Adjoint of the hash columns: accumulates into table_grad (L, 2^log2_size, 2) from the row
 * gradients d_out (row stride ld_d, hash columns first). */
int vx_hash_encode_backward(float* table_grad, int n_levels, int log2_size, int n_features, const int32_t* level_res,
                            const float* level_weights, const float* pts_norm, const float* rays_o,
                            const float* rays_d, const float* mid, int n_samples, const float xyz_min[3],
                            const float xyz_max[3], int64_t n_points, const float* d_out, int64_t ld_d,
                            void* stream);

/* Deterministic variants of the two scatter adjoints (vx_render_geometry_backward,
 * vx_hash_encode_backward): every contribution is emitted as a (destination, value) pair at a
 * fixed slot, stably radix-sorted by destination and summed per destination in slot order, so the
 * gradient is bitwise reproducible. The caller provides a workspace of the size the *_workspace
 * query returns (0 = sizes out of range). Hash variant: level_res_dev / level_weights_dev are
 * device arrays of n_levels int32 / float32. */
size_t vx_geometry_backward_det_workspace(int64_t n_rays, int n_samples, const int32_t res[3]);
int vx_render_geometry_backward_det(const float* grid, const int32_t res[3], const float xyz_min[3],
                                    const float xyz_max[3], const float* rays_o, const float* rays_d, const float* mid,
                                    int64_t n_rays, int n_samples, const float* d_sdf, const float* d_normal,
                                    const float* d_normal2, int64_t ld2, float* grid_grad, void* workspace,
                                    size_t workspace_bytes, void* stream);
size_t vx_hash_backward_det_workspace(int64_t n_points, int n_levels, int log2_size);
int vx_hash_encode_backward_det(float* table_grad, int n_levels, int log2_size, int n_features,
                                const int32_t* level_res_dev, const float* level_weights_dev, const float* pts_norm,
                                const float* rays_o, const float* rays_d, const float* mid, int n_samples,
                                const float xyz_min[3], const float xyz_max[3], int64_t n_points, const float* d_out,
                                int64_t ld_d, void* workspace, size_t workspace_bytes, void* stream);

/* Radiance MLP (models/radiance_mlp.py:42-53,81-98): rows x (n_points, in_dim) with row stride
 * ldx -> Linear(51,64) -> ReLU -> Linear(64,3) -> Sigmoid -> colors (n_points, 3). W0 (64,51),
 * b0 (64), W1 (3,64), b1 (3) as nn.Linear stores them. Only the 51 -> 64 -> 3 shape is fused. */
int vx_radiance_mlp_forward(const float* x, int64_t ldx, int64_t n_points, int in_dim, int hidden, int out_dim,
                            const float* W0, const float* b0, const float* W1, const float* b1, float* colors,
                            void* stream);

/* Appearance branch + MLP in one pass (models/voxneus.py:147-157): hash features of o + d*mid
 * (16 levels x 2), SH of the ray direction and the normal are built in shared memory and fed to
 * the 51-64-3 MLP; writes colors (n,3) and, when rows is given, the MLP input rows (row stride
 * ld_rows >= 52, multiple of 4, 16-byte aligned; the adjoint's input). ld_rows == 36 stores the
 * compact rows of vx_appearance_mlp_backward instead: [hash 32 | normal 3 | pad], without the 16
 * SH(d) columns, which the MLP takes from rays_d (folded into a per-ray hidden bias when n_samples
 * is a multiple of 128, as vx_appearance_mlp_backward describes). */
int vx_appearance_mlp_forward(const float* table, int n_levels, int log2_size, int n_features,
                              const int32_t* level_res, const float* level_weights, const float* rays_o,
                              const float* rays_d, const float* mid, int n_samples, const float xyz_min[3],
                              const float xyz_max[3], int64_t n_points, const float* normals, const float* W0,
                              const float* b0, const float* W1, const float* b1, float* colors, float* rows,
                              int64_t ld_rows, void* stream);

/* Inference form of vx_appearance_mlp_forward (models/voxneus.py:147-157 under no_grad, the path
 * of scripts/render.py:35-54; no rows kept for an adjoint): the same colours,
 * computed chunk by chunk of whole rays through the caller's scratch rows (scratch_count x 36
 * floats, 16-byte aligned; at least n_samples rows): each chunk's compact rows [hash 32 | normal 3 |
 * pad] are gathered into the scratch and the MLP reads them back with SH(d) recomputed from rays_d
 * (the gather and the MLP each at their own best occupancy).
 * Fewer, larger chunks cost less: each chunk adds two launches and their tails. n_points must be a
 * multiple of n_samples (whole rays). */
int vx_appearance_mlp_forward_chunked(const float* table, int n_levels, int log2_size, int n_features,
                                      const int32_t* level_res, const float* level_weights, const float* rays_o,
                                      const float* rays_d, const float* mid, int n_samples, const float xyz_min[3],
                                      const float xyz_max[3], int64_t n_points, const float* normals,
                                      const float* W0, const float* b0, const float* W1, const float* b1,
                                      float* colors, float* scratch_rows, int64_t scratch_count, void* stream);

/* Blocks of vx_radiance_mlp_backward and the floats of one block's weight-gradient partial. */
int vx_mlp_blocks(int64_t n_points);
int vx_mlp_partial_floats(void);

/* The three MLP kernels run on the tcgen05 tensor cores (kind::tf32, hi/lo split for FP32-level
 * accuracy) and wait on the tensor core with bounded mbarrier polls. Returns how many blocks gave
 * up on such a wait since the last call (their outputs are invalid) and resets the count; -1 on
 * a CUDA error. Synchronises the device (diagnostic only). No counterpart in the reference. */
int vx_tensor_core_timeouts(void);

/* The wait policy of this thread's later MLP launches (vx_radiance_mlp_forward/backward,
 * vx_appearance_mlp_forward[_chunked]): at most wait_polls mbarrier polls per wait on the tensor
 * core (negative: the default, 2^22), and a device int (status, may be NULL) that every block
 * which gave up on a wait increments atomically, so the caller can test its step's status without
 * a synchronisation. A block that gives up lets the copy or MMA it waited for finish (bounded)
 * before it frees tensor memory and exits; its outputs are invalid. The arguments are baked into
 * launches captured in a CUDA graph. Thread-local; no counterpart in the reference. */
int vx_tc_guard(int* status, int64_t wait_polls);

/* Adjoint of vx_radiance_mlp_forward (recomputes the hidden layer): d_colors (n,3) -> d_hash (n,32)
 * (gradient of input columns 0..31), d_normal (n,3) (columns 48..50), and the weight gradients
 * dW0, db0, dW1, db1 (written, not accumulated; summed over blocks in a fixed order).
 * colors: the forward's outputs (n,3) for the sigmoid's derivative, or NULL to recompute them
 * (the same bits either way). partials: >= vx_mlp_blocks(n) * vx_mlp_partial_floats() floats. */
int vx_radiance_mlp_backward(const float* x, int64_t ldx, int64_t n_points, int in_dim, int hidden, int out_dim,
                             const float* W0, const float* b0, const float* W1, const float* b1, const float* d_colors,
                             const float* colors, float* d_hash, float* d_normal, float* dW0, float* db0, float* dW1,
                             float* db1, float* partials, int64_t n_partial_floats, void* stream);

/* The adjoint of the fused appearance path on its compact rows: n_points rows of 36 floats
 * [hash 32 | normal 3 | pad] (16-byte aligned, contiguous) whose SH(d) features come from rays_d
 * of the sample's ray (sample i belongs to ray i / n_samples): the 16 columns of a full row that
 * depend on the ray only (models/embedder.py:55-87). Outputs and partials as
 * vx_radiance_mlp_backward. When n_samples is a multiple of 128 (every 128-sample tile inside one
 * ray: the training and serving shapes) the MLP is folded: SH(d) enters as a per-ray bias of the
 * hidden layer (b0 + W0[:, 32:48] SH(d)) and the SH columns of dW0 come from per-tile column sums
 * of dL/dz, so the results agree with the full rows within FP32 rounding; otherwise SH(d) is
 * rebuilt per sample and they are the same bits. vx_appearance_mlp_forward folds on the same
 * condition. */
int vx_appearance_mlp_backward(const float* rows, const float* rays_d, int n_samples, int64_t n_points,
                               const float* W0, const float* b0, const float* W1, const float* b1,
                               const float* d_colors, const float* colors, float* d_hash, float* d_normal, float* dW0,
                               float* db0, float* dW1, float* db1, float* partials, int64_t n_partial_floats,
                               void* stream);

/* ---------------------------------------------------------- render (per ray) --------------- */

/* Blocks used by the per-ray kernels; vx_composite_backward's partials hold one double per block. */
int vx_composite_workspace_blocks(int64_t n_rays);

/* volume_render_from_samples (rendering/volume_render.py:57-153) with compute_neus_alpha
 * (rendering/neus_alpha.py:12-81) and composite_weights (volume_render.py:12-40) fused: one warp per
 * ray. colors/normals (n_rays, n_samples, 3), sdf/z_vals/dists (n_rays, n_samples); direction of
 * sample (r,i) at dirs + r*dir_ray_stride + i*dir_sample_stride; the inside-sphere mask
 * (sphere_radius > 0) uses pts (n_rays, n_samples, 3) or rebuilds o + d*z from rays_o. s_ptr points
 * at s, or at the variance parameter v when s_is_variance (s = clamp(exp(10 v), 1e-4, s_max),
 * models/variance.py:38-41). background: (3) or (n_rays,3) when background_per_ray, or NULL.
 * Outputs (each nullable): rgb (n,3), depth (n), normal (n,3), opacity (n), weights, alpha,
 * transmittance (n, n_samples). */
int vx_composite_forward(const float* colors, const float* sdf, const float* normals, const float* dirs,
                         int64_t dir_ray_stride, int64_t dir_sample_stride, const float* z_vals, const float* dists,
                         const float* pts, const float* rays_o, const float* s_ptr, int s_is_variance, float s_max,
                         float sphere_radius, const float* background, int background_per_ray, int use_iter_cos,
                         float cos_anneal_ratio, int64_t n_rays, int n_samples, float* rgb, float* depth,
                         float* normal, float* opacity, float* weights, float* alpha, float* transmittance,
                         void* stream);

/* Adjoint of vx_composite_forward. Output gradients g_* nullable (zero). Writes d_colors, d_sdf,
 * d_normals (each nullable) and the scalar d_s (device): dL/ds, or dL/dv when s_is_variance, in
 * which case a negative dL/dv is multiplied by amplify_k when amplify_k > 0 (the k=5 rule of
 * training/scheduler.py:14-33) and *amplified (nullable) is set to 1 or 0. partials: >=
 * vx_composite_workspace_blocks(n_rays) doubles. */
int vx_composite_backward(const float* colors, const float* sdf, const float* normals, const float* dirs,
                          int64_t dir_ray_stride, int64_t dir_sample_stride, const float* z_vals, const float* dists,
                          const float* pts, const float* rays_o, const float* s_ptr, int s_is_variance, float s_max,
                          float sphere_radius, const float* background, int background_per_ray, int use_iter_cos,
                          float cos_anneal_ratio, int64_t n_rays, int n_samples, const float* g_rgb,
                          const float* g_depth, const float* g_normal, const float* g_opacity, const float* g_weights,
                          const float* g_alpha, const float* g_transmittance, float* d_colors, float* d_sdf,
                          float* d_normals, double* partials, int n_partials, unsigned int* counter, float* d_s,
                          float amplify_k, int* amplified, void* stream);

/* compute_neus_alpha (rendering/neus_alpha.py:12-81) elementwise, with its adjoint when d_alpha is
 * given (d_s_elems receives the per-element dL/ds terms). */
int vx_neus_alpha(const float* sdf, const float* normals, const float* dirs, int64_t dir_ray_stride,
                  int64_t dir_sample_stride, const float* dists, const float* s_ptr, int use_iter_cos,
                  float cos_anneal_ratio, int64_t n_rays, int n_samples, float* alpha, const float* d_alpha,
                  float* d_sdf, float* d_normals, float* d_s_elems, void* stream);

/* composite_weights (rendering/volume_render.py:12-40), and its adjoint when d_alpha is given. */
int vx_composite_weights(const float* alpha, int64_t n_rays, int n_samples, float* weights, float* transmittance,
                         const float* d_weights, const float* d_transmittance, float* d_alpha, void* stream);

/* ------------------------------------------------------------------ colour loss ----------- */

/* Blocks of vx_huber_loss (one double partial each). */
int vx_huber_loss_blocks(int64_t n);

/* NeuS2 Huber colour loss (rendering/volume_render.py:43-54, compute_huber_color_loss): *loss =
 * mean over n elements of (d < delta ? 0.5 d^2 / delta : d - 0.5 delta), d = |pred - target|;
 * grad (optional, n floats) = d(loss)/d(pred). partials: >= vx_huber_loss_blocks(n) doubles. */
int vx_huber_loss(const float* pred, const float* target, int64_t n, float delta, float* loss, float* grad,
                  double* partials, int64_t n_partials, void* stream);

/* ------------------------------------------------ active vertices and regularizers -------- */

/* 32-bit words of a V_R bitmap for the grid; blocks of block scratch vx_vr_compact needs. */
int64_t vx_vr_bitmap_words(const int32_t res[3]);
int64_t vx_vr_compact_blocks(const int32_t res[3]);

/* Marks explicit corner indices (n_corners,3) int64, clamped to the grid, in a V_R bitmap. */
int vx_vr_mark_corners(const int64_t* corners, int64_t n_corners, const int32_t res[3], uint32_t* bitmap,
                       void* stream);

/* Counts V_R (counts[4] device uint64, zeroed by the caller): [all, relax, band, relax & band] with
 * relax = |xyz_min + idx*eps| < relax_radius (training/trainer.py:262-266; <= 0 disables) and
 * band = |f| < band (<= 0 disables). filtered (nullable, 2 x vx_vr_bitmap_words words) receives
 * the bitmaps bits & band and bits & band & relax (the regularizer's input). */
int vx_vr_count(const uint32_t* bitmap, const float* grid, const int32_t res[3], const float xyz_min[3],
                const float xyz_max[3], float relax_radius, float band, unsigned long long* counts,
                uint32_t* filtered, void* stream);

/* Writes the V_R list in ascending linear order (torch.unique order): verts (V,3) and linear (V),
 * each nullable, up to capacity entries. The relax filter applies only when counts[1] > 0. */
int vx_vr_compact(const uint32_t* bitmap, const float* grid, const int32_t res[3], const float xyz_min[3],
                  const float xyz_max[3], float relax_radius, float band, const unsigned long long* counts,
                  int* block_scratch, int64_t n_block_scratch, int64_t* verts_out, int64_t* linear_out,
                  int64_t capacity, void* stream);

/* vx_vr_compact without caller scratch. No counterpart in the reference. For callers that
 * cannot allocate device memory when they call in: embedders whose device memory belongs to
 * another runtime's pool (no allocation hook reaches this library) and plugin hosts that forbid
 * device allocation after start-up. Identical arguments and output to vx_vr_compact minus the
 * block scratch, which lives in a 16 KiB file-scope device array held by every GPU that loads the
 * library until exit. Limit: grids of at most 2^27 voxels (4096 compaction blocks, e.g. 512^3);
 * larger grids are rejected with VX_ERR_INVALID before any launch. Allocates nothing (no
 * cudaMalloc, cudaFree or allocating library call). The first call on each device looks up the
 * array's device address with that device current and keeps it for the life of the process;
 * make that first call before any stream capture. The kept address assumes the device's
 * primary context is never reset (cudaDeviceReset reloads the library's device code and may move
 * the array; do not call this entry point after one). All calls share the one array: calls that overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller. */
int vx_vr_compact_noalloc(const uint32_t* bitmap, const float* grid, const int32_t res[3], const float xyz_min[3],
                          const float xyz_max[3], float relax_radius, float band, const unsigned long long* counts,
                          int64_t* verts_out, int64_t* linear_out, int64_t capacity, void* stream);

/* Blocks of the fused regularizer, and the doubles of its workspace (3 loss partials per block,
 * then one flag byte per 32x4x4 tile). */
int64_t vx_reg_stencil_blocks(const int32_t res[3]);
int64_t vx_reg_stencil_workspace(const int32_t res[3]);

/* Fused eikonal + curvature closed forms (regularization/eikonal.py:13-171 and curvature.py:13-165 as
 * called by training/trainer.py:268-319), gather form (deterministic, no atomics), accumulated into
 * grad_grid with weights w_eik and w_curv and scale 2/|V_R|. bitmap is the filtered pair written by
 * vx_vr_count; counts selects its relax half (the reference applies the relax filter only when a
 * vertex passes it) and gives |V_R|. band is applied by vx_vr_count (here it only selects which
 * count n_active reports); counter is unused (may be NULL). partials: >=
 * vx_reg_stencil_workspace(res) doubles. losses (device float[2], nullable) receives the monitoring
 * losses; n_active (device int64, nullable) |V_R| after the relax and band filters. */
int vx_reg_stencil(const float* grid, const uint32_t* bitmap, const int32_t res[3], const float xyz_min[3],
                   const float xyz_max[3], float relax_radius, float band, const unsigned long long* counts,
                   float w_eik, float w_curv, float* grad_grid, double* partials, int64_t n_partials,
                   unsigned int* counter, float* losses, int64_t* n_active, void* stream);

/* ------------------------------------------------------------ occupancy grid ------------- */

/* Bytes of the workspace vx_occupancy_update needs for n drawn cells (8 per cell, 16-byte padded). */
int64_t vx_occupancy_workspace(int64_t n);

/* World-space centres of the drawn cells (n,3) of an occ_res^3 grid spanning [occ_min, occ_max]:
 * xyz_min + ((idx + 0.5) / res) * (xyz_max - xyz_min) (rendering/occupancy_grid.py:85-98), for a
 * caller that evaluates its own SDF function at them. */
int vx_occupancy_points(int32_t occ_res, const float occ_min[3], const float occ_max[3], const int64_t* idx_x,
                        const int64_t* idx_y, const int64_t* idx_z, int64_t n, float* pts, void* stream);

/* OccupancyGrid.is_occupied (rendering/occupancy_grid.py:121-147) for world points pts (n,3):
 * occupied_out[i] = 1 when the point lies inside [occ_min, occ_max] and its cell of the occ_res^3
 * mask is set (the lookup the sampler applies to interval midpoints), else 0. */
int vx_occupancy_query(const uint8_t* mask, int32_t occ_res, const float occ_min[3], const float occ_max[3],
                       const float* pts, int64_t n, uint8_t* occupied_out, void* stream);

/* OccupancyGrid.update_from_sdf (rendering/occupancy_grid.py:62-119) at caller-drawn cells
 * (idx_x, idx_y, idx_z: n int64 each, as torch.randint draws them, :81-83). The SDF comes from the
 * dense grid (sdf_grid with res / sdf_min / sdf_max, the trilinear query of models/sdf_grid.py:90-120
 * at the cell centres) or, when sdf_grid is NULL, from sdf_values (n). s (device scalar) is s, or the
 * variance parameter v when s_is_variance (s = clamp(exp(10 v), 1e-4, s_max)). Density
 * s*sig*(1-sig), sig = sigmoid(s*sdf); floor 2*threshold where |sdf| < 2*|(xyz_max-xyz_min)/occ_res|;
 * unless first, max with decay * previous density; density (occ_res^3 float) and mask (occ_res^3
 * bytes, 0/1; a torch.bool tensor) are written at the drawn cells. A cell drawn several times gets
 * the value computed from its density before this update. Cells outside [0, occ_res) are skipped and
 * counted into *n_invalid (device, nullable). workspace: >= vx_occupancy_workspace(n) bytes, 16-byte
 * aligned. Two launches on stream. */
int vx_occupancy_update(const float* sdf_grid, const int32_t res[3], const float sdf_min[3], const float sdf_max[3],
                        const float* sdf_values, int32_t occ_res, const float occ_min[3], const float occ_max[3],
                        const int64_t* idx_x, const int64_t* idx_y, const int64_t* idx_z, int64_t n,
                        const float* s, int s_is_variance, float s_max, int first, float decay, float threshold,
                        float* density, uint8_t* mask, void* workspace, int64_t workspace_bytes,
                        unsigned int* n_invalid, void* stream);

/* -------------------------------------------------------------- grid upsampling ----------- */

/* upsample_sdf_grid (geometry/upsample.py:12-39): trilinear, align_corners=True, src (res_in) ->
 * dst (res_out); dst 16-byte aligned. */
int vx_grid_upsample(const float* src, const int32_t res_in[3], float* dst, const int32_t res_out[3], void* stream);

#ifdef __cplusplus
}
#endif

#endif /* VOXNEUS_B200_H */
